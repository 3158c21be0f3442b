"""Shared helpers for the parity tests."""

import numpy as np

# fields compared after full steps: the state the next step reads, plus phi
STATE_FIELDS = ("c_new", "u_new", "v_new", "w_new", "phi", "u_pg", "v_pg",
                "w_pg", "c_hn", "u_hn", "v_hn", "w_hn")


def rel_maxnorm(a: np.ndarray, b: np.ndarray) -> float:
    """max|a-b| / max|b| (0 when both are zero)."""
    den = float(np.abs(b).max())
    num = float(np.abs(a - b).max())
    if den == 0.0:
        return num
    return num / den


# components measured against the vector's scale: a flow that is nearly
# two-dimensional has |w| ~ 1e-8 |u| on the small test grids, where the
# per-component ratio measures rounding noise of exp(), not the solver
VECTOR_OF = {
    "u_new": ("u_new", "v_new", "w_new"), "v_new": ("u_new", "v_new", "w_new"),
    "w_new": ("u_new", "v_new", "w_new"), "u_old": ("u_old", "v_old", "w_old"),
    "v_old": ("u_old", "v_old", "w_old"), "w_old": ("u_old", "v_old", "w_old"),
    "u_pg": ("u_pg", "v_pg", "w_pg"), "v_pg": ("u_pg", "v_pg", "w_pg"),
    "w_pg": ("u_pg", "v_pg", "w_pg"), "u_hn": ("u_hn", "v_hn", "w_hn"),
    "v_hn": ("u_hn", "v_hn", "w_hn"), "w_hn": ("u_hn", "v_hn", "w_hn"),
}


def rel_vector(get_a, get_b, name: str) -> float:
    """max|a-b| over the field / max-norm of the reference vector field it
    belongs to (the field itself for scalars)."""
    a, b = get_a(name), get_b(name)
    comps = VECTOR_OF.get(name, (name,))
    den = max(float(np.abs(get_b(c)).max()) for c in comps)
    num = float(np.abs(a - b).max())
    return num / den if den > 0 else num
