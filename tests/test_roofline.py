"""The algorithmic-traffic model behind bench.py's roofline fields (host
logic, no GPU): every per-launch label has a word count and a kernel family
in both forms, the precision form names its own kernels, and the per-cell
figures add up as the model states."""

from pllcart3d_b200 import roofline

LABELS = [f"{s}_{v}" for s in ("explicit", "adi_y", "adi_z", "adi_x") for v in "cuvw"] + [
    "viscosity", "div_rhs", "poisson_x", "project", "cfl"]


def test_every_label_has_words_and_family():
    for lab in LABELS:
        assert roofline.KERNEL_WORDS[lab] > 0, lab
        assert roofline.family(lab, "fp64"), lab
        assert roofline.family(lab, "fp32"), lab


def test_precision_form_names_its_kernels():
    assert roofline.family("explicit_u", "fp64") == "k_explicit"
    assert roofline.family("explicit_u", "fp32") == "k_explicit2"
    assert roofline.family("adi_x_c", "fp32") == "k_line_seg (x)"
    assert roofline.family("adi_z_w", "fp32") == "k_adi_z_part"
    assert roofline.family("dct_gemm", "fp32") == "k_gemm_dmma"   # no precision-form override
    assert roofline.family("not_a_label", "fp32") is None


def test_bytes_scale_with_cells_and_word_size():
    cells = 1 << 20
    assert roofline.kernel_bytes_per_launch("project", cells, "fp64") == 17 * cells * 8
    assert roofline.kernel_bytes_per_launch("project", cells, "fp32") == 17 * cells * 4
    assert roofline.step_bytes(cells, "fp64") == 2 * roofline.step_bytes(cells, "fp32") == 2424 * cells
