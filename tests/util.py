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
