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
        assert roofline.family(lab, "fp64", "fp64x"), lab
        assert roofline.family(lab, "fp32"), lab


def test_each_form_names_its_kernels():
    assert roofline.family("explicit_u", "fp64") == "k_explicit_tma"
    assert roofline.family("explicit_u", "fp64", "mixed64", "direct") == "k_explicit"
    assert roofline.family("explicit_u", "fp64", "fp64x") == "k_explicit"
    assert roofline.family("adi_z_u", "fp64") == "k_adi_z_part"
    assert roofline.family("adi_z_u", "fp64", "fp64x") == "k_adi_z_tiled"
    assert roofline.family("adi_y_c", "fp64") == "k_line_seg (y)"
    assert roofline.family("dct_fft", "fp64") == "k_dct_fft"
    assert roofline.family("dct_gemm", "fp64", "fp64x") == "k_gemm_dmma"
    assert roofline.family("explicit_u", "fp32") == "k_explicit2"
    assert roofline.family("explicit_u", "fp32", "mixed", "tma") == "k_explicit_tma"
    assert roofline.family("adi_x_c", "fp32") == "k_line_seg (x)"
    assert roofline.family("adi_z_w", "fp32") == "k_adi_z_part"
    assert roofline.family("dct_gemm", "fp32", "fp64x") == "k_gemm_dmma"   # no precision-form override
    assert roofline.family("not_a_label", "fp32") is None


def test_bytes_scale_with_cells_and_word_size():
    cells = 1 << 20
    assert roofline.kernel_bytes_per_launch("project", cells, "fp64") == 17 * cells * 8
    assert roofline.kernel_bytes_per_launch("project", cells, "fp32") == 17 * cells * 4
    assert roofline.step_bytes(cells, "fp64") == 2 * roofline.step_bytes(cells, "fp32") == 2424 * cells


def test_bench_roofline_picks_the_largest_family():
    """bench.py's roofline field from a synthetic per-label timing table: the
    family with the largest total time wins, its achieved bandwidth is its
    algorithmic bytes over its mean launch time, traffic uses the ncu ratio."""
    import bench

    cells = 1 << 20
    kernels = {
        "explicit_u": {"ms_total": 6.0, "launches": 6},
        "explicit_v": {"ms_total": 6.0, "launches": 6},
        "project": {"ms_total": 3.0, "launches": 3},
        "viscosity": {"ms_total": 1.0, "launches": 3},
    }
    r = bench.roofline_of(kernels, 2, cells, "fp32")
    assert r["kernel"] == "k_explicit2" and r["labels"] == ["explicit_u", "explicit_v"]
    assert r["bound"] == "hbm" and r["avg_launch_ms"] == 1.0
    alg = roofline.kernel_bytes_per_launch("explicit_u", cells, "fp32")
    assert abs(r["achieved"] - alg / 1e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert abs(r["traffic"] - bench.TRAFFIC_RATIO[("k_explicit2", "fp32")] * alg) < 1.0
    assert abs(r["share_of_step"] - 12.0 / 16.0) < 1e-12
    r64 = bench.roofline_of(kernels, 2, cells, "fp64", form="mixed64")
    assert r64["kernel"] == "k_explicit_tma"
    assert abs(r64["traffic"] - bench.TRAFFIC_RATIO[("k_explicit_tma", "fp64")]
               * roofline.kernel_bytes_per_launch("explicit_u", cells, "fp64")) < 1.0


def test_bench_states_its_l2_figures():
    """The bench line's config.l2 note follows the run's own sizes: field
    size in the form's word and the step's modelled traffic against L2."""
    import bench
    from pllcart3d_b200.params import workload

    p = workload("fingering-512x256x256").params
    assert bench.l2_note(p, "mixed64").startswith("no L2 flush: each field 276 MB, each step moves 81.3 GB")
    assert "each field 138 MB" in bench.l2_note(p, "mixed")
    small = workload("fingering-256x128x128").params
    assert "each field 35 MB" in bench.l2_note(small, "fp64")
