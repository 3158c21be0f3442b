"""Algorithmic-traffic model of the step, for roofline fractions.

Per kernel: FP64 words per cell that the stage must move at minimum - each
distinct input field read once and each output field written once; ghost
layers and the Thomas scratch (c', eliminated rhs) are not counted.  The
whole-step figure is the 303 words per cell-step of the reference-structured
model (100 words per RK substep plus 3 for the CFL scan), i.e. 2424 bytes per
cell-step in FP64.
"""

STEP_WORDS_PER_CELL = 303
WORD_BYTES = {"fp64": 8, "fp32": 4}

KERNEL_WORDS = {
    # explicit operator + rhs: q, three velocities, mu_old (3 arrays for the
    # momentum components), c_new (u, v body force), pg, H_old ; H, S
    "explicit_c": 7,
    "explicit_u": 11,
    "explicit_v": 11,
    "explicit_w": 10,
    # y / z line solves: rhs in, rhs out (+ one viscosity array for momentum)
    "adi_y_c": 2, "adi_z_c": 2,
    "adi_y_u": 3, "adi_z_u": 3,
    "adi_y_v": 3, "adi_z_v": 3,
    "adi_y_w": 3, "adi_z_w": 3,
    # x line solve + update: rhs, q_old (+ viscosity) ; q_new
    "adi_x_c": 3,
    "adi_x_u": 4, "adi_x_v": 4, "adi_x_w": 4,
    "viscosity": 5,      # c ; 4 viscosity families
    "div_rhs": 4,        # u, v, w ; rhs
    "dct_gemm": 2,       # one dense pass: in ; out (per launch)
    "poisson_x": 2,
    "project": 17,       # u v w phi mu(4) pg(3) ; u v w pg(3)
    "cfl": 3,
}


def kernel_bytes_per_launch(label: str, cells: int, precision: str = "fp64") -> float:
    """Algorithmic bytes one launch of `label` moves on a grid of `cells`."""
    return KERNEL_WORDS[label] * cells * WORD_BYTES[precision]


def step_bytes(cells: int, precision: str = "fp64") -> float:
    return STEP_WORDS_PER_CELL * cells * WORD_BYTES[precision]
