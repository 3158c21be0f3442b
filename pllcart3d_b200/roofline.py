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
    "dct_umma": 2,
    "dct_fft": 2,        # one FFT pass: in ; out
    "poisson_x": 2,
    "project": 17,       # u v w phi mu(4) pg(3) ; u v w pg(3)
    "cfl": 3,
}


# kernel families (one CUDA kernel template each) of the per-launch labels in
# the FP64 and mixed64 forms (explicit="tma", the default on these forms)
FAMILY = {
    "explicit_c": "k_explicit_tma", "explicit_u": "k_explicit_tma", "explicit_v": "k_explicit_tma",
    "explicit_w": "k_explicit_tma",
    "adi_y_c": "k_line_seg (y)", "adi_y_u": "k_line_pf (y)", "adi_y_v": "k_line_pf (y)",
    "adi_y_w": "k_line_pf (y)",
    "adi_z_c": "k_adi_z_part", "adi_z_u": "k_adi_z_part", "adi_z_v": "k_adi_z_part",
    "adi_z_w": "k_adi_z_part",
    "adi_x_c": "k_line_pf (x)", "adi_x_u": "k_line_pf (x)", "adi_x_v": "k_line_pf (x)",
    "adi_x_w": "k_line_pf (x)",
    "viscosity": "k_viscosity2", "div_rhs": "k_div_rhs2", "dct_fft": "k_dct_fft",
    "poisson_x": "k_poisson_x", "project": "k_project2", "cfl": "k_cfl",
}

# the exact FP64 form's kernels where they differ (bit-reproducible order of
# operations: no paired-cell kernels, DMMA DCT, tiled z solve)
FAMILY_EXACT = dict(FAMILY, **{
    "explicit_c": "k_explicit", "explicit_u": "k_explicit", "explicit_v": "k_explicit",
    "explicit_w": "k_explicit", "adi_y_c": "k_line_pf (y)",
    "adi_z_c": "k_adi_z_tiled", "adi_z_u": "k_adi_z_tiled", "adi_z_v": "k_adi_z_tiled",
    "adi_z_w": "k_adi_z_tiled",
    "viscosity": "k_viscosity", "div_rhs": "k_div_rhs", "dct_gemm": "k_gemm_dmma", "project": "k_project"})

# the precision form's kernels where they differ from the FP64 form's
FAMILY_FP32 = {
    "explicit_c": "k_explicit2", "explicit_u": "k_explicit2", "explicit_v": "k_explicit2",
    "explicit_w": "k_explicit2",
    "adi_y_c": "k_line_seg (y)", "adi_y_u": "k_line_seg (y)", "adi_y_v": "k_line_seg (y)",
    "adi_y_w": "k_line_seg (y)",
    "adi_z_c": "k_adi_z_part", "adi_z_u": "k_adi_z_part", "adi_z_v": "k_adi_z_part", "adi_z_w": "k_adi_z_part",
    "adi_x_c": "k_line_seg (x)", "adi_x_u": "k_line_seg (x)", "adi_x_v": "k_line_seg (x)",
    "adi_x_w": "k_line_seg (x)",
    "viscosity": "k_viscosity2", "div_rhs": "k_div_rhs2", "dct_umma": "k_dct_umma_p",
    "poisson_x": "k_poisson_x2", "project": "k_project2", "cfl": "k_cfl2",
}


def family(label: str, precision: str = "fp64", form: str = None, explicit: str = "auto"):
    """Kernel (family) that runs `label` in the given form, or None.  `form`
    is "fp64x" for the exact form; `explicit` is the Solver's explicit_kernel
    ("direct" runs the FP64 forms' explicit operator as k_explicit)."""
    if precision == "fp32" and label in FAMILY_FP32:
        if explicit == "tma" and label.startswith("explicit_"):
            return "k_explicit_tma"
        return FAMILY_FP32[label]
    if form == "fp64x":
        return FAMILY_EXACT.get(label)
    if explicit == "direct" and label.startswith("explicit_"):
        return "k_explicit"
    return FAMILY.get(label)


# tensor-core kernels: products per DCT pass (one dense product of 2 n flops
# per cell for a pass of length n; the precision form's split-TF32 passes
# issue 3: hi*hi, hi*lo, lo*hi)
TENSOR_PASS_FLOPS = {"dct_gemm": 1, "dct_umma": 3}


def kernel_bytes_per_launch(label: str, cells: int, precision: str = "fp64") -> float:
    """Algorithmic bytes one launch of `label` moves on a grid of `cells`."""
    return KERNEL_WORDS[label] * cells * WORD_BYTES[precision]


def step_bytes(cells: int, precision: str = "fp64") -> float:
    return STEP_WORDS_PER_CELL * cells * WORD_BYTES[precision]
