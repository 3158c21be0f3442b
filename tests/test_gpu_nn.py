"""The surrogate's BF16 tensor-core kernels against the CPU oracle
(oracle/nn_ref.py, itself checked against finite differences), the full
network gradient, Adam, and a short training run that must beat the method
without the network (persistence) on held-out data."""

import numpy as np
import pytest

from oracle import nn_ref

pytestmark = pytest.mark.gpu


def _bf16(a):
    """Round an FP32/FP64 array to BF16 (round to nearest even) in FP64."""
    import torch

    return torch.tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float64).numpy()


def _t(a, dtype):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("k,ci,co,vol", [(3, 16, 32, (2, 6, 8, 10)), (3, 64, 128, (1, 4, 4, 8)),
                                         (3, 384, 128, (1, 4, 6, 4)), (1, 32, 16, (1, 8, 8, 8))])
def test_conv_forward_and_gradients(k, ci, co, vol):
    import torch

    from pllcart3d_b200 import surrogate as S

    rng = np.random.default_rng(k * 1000 + ci)
    x = _bf16(rng.standard_normal(vol + (ci,)))
    w = _bf16(rng.standard_normal((co, k ** 3, ci)) / np.sqrt(k ** 3 * ci))
    b = rng.standard_normal(co).astype(np.float32)
    c = S.Conv("t", ci, co, k, 1, np.random.default_rng(0))
    c.w32.copy_(_t(w, torch.float32))
    c.b32.copy_(_t(b, torch.float32))
    c.refresh()
    x16 = _t(x.reshape(-1, ci), torch.bfloat16)
    y16 = c.forward(x16, vol)
    z_ref = nn_ref.conv_fwd(x, w, b.astype(np.float64), k)
    assert _relerr(c.z.cpu().numpy().reshape(z_ref.shape), z_ref) < 1e-5
    y_ref = nn_ref.leaky(z_ref, S.SLOPE)
    assert _relerr(y16.float().cpu().numpy().reshape(y_ref.shape), y_ref) < 1e-2
    gy = rng.standard_normal(z_ref.shape).astype(np.float32)
    z_gpu = c.z.cpu().numpy().reshape(z_ref.shape)
    dx = c.backward(_t(gy.reshape(-1, co), torch.float32)).cpu().numpy()
    # the kernels round dL/dz to BF16 before both gradient GEMMs
    gz = _bf16(nn_ref.leaky_bwd(z_gpu, gy, np.float32(S.SLOPE)))
    dx_ref, dw_ref, db_ref = nn_ref.conv_bwd(x, w, gz, k)
    assert _relerr(dx.reshape(dx_ref.shape), dx_ref) < 1e-4
    assert _relerr(c.gw.cpu().numpy(), dw_ref) < 1e-4
    # the bias gradient sums the unrounded FP32 values
    assert _relerr(c.gb.cpu().numpy(), nn_ref.leaky_bwd(z_gpu, gy, np.float32(S.SLOPE)).reshape(-1, co).sum(0)) < 1e-4


def test_pool_up_cat_adam():
    import torch

    from pllcart3d_b200 import surrogate as S

    L, st = S.nnlib(), S._stream()
    rng = np.random.default_rng(3)
    x = _bf16(rng.standard_normal((2, 4, 6, 8, 16)))
    x16 = _t(x.reshape(-1, 16), torch.bfloat16)
    y = torch.empty((2 * 2 * 3 * 4, 16), dtype=torch.bfloat16, device="cuda")
    assert L.pllnn_pool_fwd(S._p(x16), 2, 4, 6, 8, 16, S._p(y), st) == 0
    assert _relerr(y.float().cpu().numpy().reshape(2, 2, 3, 4, 16), nn_ref.pool(x)) < 1e-2
    g = rng.standard_normal((2, 2, 3, 4, 16))
    dx = torch.zeros((2 * 4 * 6 * 8, 16), dtype=torch.float32, device="cuda")
    assert L.pllnn_pool_bwd(S._p(_t(g.reshape(-1, 16), torch.float32)), 2, 4, 6, 8, 16, S._p(dx), 1, st) == 0
    assert _relerr(dx.cpu().numpy().reshape(x.shape), nn_ref.pool_bwd(g)) < 1e-6
    u = torch.empty((2 * 8 * 12 * 16, 16), dtype=torch.bfloat16, device="cuda")
    assert L.pllnn_up_fwd(S._p(x16), 2, 4, 6, 8, 16, S._p(u), st) == 0
    assert np.array_equal(u.float().cpu().numpy().reshape(2, 8, 12, 16, 16), nn_ref.up(x))
    gu = rng.standard_normal((2, 8, 12, 16, 16))
    du = torch.empty((2 * 4 * 6 * 8, 16), dtype=torch.float32, device="cuda")
    assert L.pllnn_up_bwd(S._p(_t(gu.reshape(-1, 16), torch.float32)), 2, 4, 6, 8, 16, S._p(du), 0, st) == 0
    assert _relerr(du.cpu().numpy().reshape(x.shape), nn_ref.up_bwd(gu)) < 1e-5
    # Adam, three steps
    w = rng.standard_normal(1000)
    w32 = _t(w, torch.float32)
    m = torch.zeros_like(w32)
    v = torch.zeros_like(w32)
    mr, vr, wr = np.zeros(1000), np.zeros(1000), w.copy()
    for t in range(1, 4):
        gr = rng.standard_normal(1000)
        assert L.pllnn_adam(S._p(w32), S._p(_t(gr, torch.float32)), S._p(m), S._p(v), 1000, 1e-2, 0.9, 0.999, 1e-8,
                            t, None, None, 0.0, st) == 0
        wr, mr, vr = nn_ref.adam(wr, gr, mr, vr, 1e-2, 0.9, 0.999, 1e-8, t)
    assert _relerr(w32.cpu().numpy(), wr) < 1e-5


def test_unet_gradient_matches_oracle():
    import torch

    from pllcart3d_b200 import surrogate as S

    net = S.UNet(seed=5)
    params = {}
    for name, c in net.layers.items():
        w = _bf16(c.w32.cpu().numpy())
        c.w32.copy_(_t(w, torch.float32))
        b = (np.random.default_rng(7).standard_normal(c.cout) * 0.05).astype(np.float32)
        c.b32.copy_(_t(b, torch.float32))
        c.refresh()
        params[name] = (w, b.astype(np.float64))
    rng = np.random.default_rng(9)
    x = _bf16(rng.standard_normal((1, 8, 8, 8, 16)))
    tgt = rng.standard_normal((1, 8, 8, 8, 16))
    out = net.forward(_t(x.reshape(-1, 16), torch.bfloat16), (1, 8, 8, 8))
    out_ref, cache = nn_ref.unet_forward(params, x, S.SLOPE)
    # BF16 activations between layers: agreement to a few BF16 ulps
    assert _relerr(out.cpu().numpy().reshape(out_ref.shape), out_ref) < 5e-2
    g = 2 * (out.cpu().numpy().reshape(out_ref.shape) - tgt)
    net.zero_grad()
    net.backward(_t(g.reshape(-1, 16), torch.float32))
    grads = nn_ref.unet_backward(params, cache, g, S.SLOPE)
    for name, c in net.layers.items():
        gw = c.gw.cpu().numpy()
        ref = grads[name][0]
        cos = float((gw * ref).sum() / (np.linalg.norm(gw) * np.linalg.norm(ref)))
        assert cos > 0.995, (name, cos)
        assert abs(np.linalg.norm(gw) / np.linalg.norm(ref) - 1) < 0.05, name


def test_training_beats_persistence():
    """What the trained network gains over the method without it: its
    8-step prediction error on a held-out run against predicting no change."""
    from pllcart3d_b200 import surrogate as S

    ds, wls = S.generate_data(n_runs=4, grid=(32, 32, 32), steps=160, precision="mixed", seed=77)
    per_run = len(ds.a) // 4
    train = np.arange(0, 3 * per_run)
    held = list(range(3 * per_run, 4 * per_run))
    net = S.UNet(seed=1)
    tr = S.Trainer(net, ds, batch=4, lr=1e-3)
    before, persist = tr.eval_loss(held)
    for _ in range(300):
        tr.step(tr.rng.choice(train, 4))
    after, persist2 = tr.eval_loss(held)
    assert persist == pytest.approx(persist2, rel=1e-5)   # FP32 atomics: order varies
    assert after < 0.5 * persist, (before, after, persist)


@pytest.mark.parametrize("k,ci,co,vol", [
    (3, 16, 32, (1, 8, 16, 64)),    # the first encoder level: 128-voxel tiles of two w rows
    (3, 64, 64, (1, 8, 32, 32)),
    (3, 384, 128, (2, 8, 16, 16)),  # a decoder level (concatenated channels)
    (3, 128, 256, (1, 16, 8, 8)),   # tiles spanning two d slices; two column tiles
    (3, 96, 32, (1, 4, 16, 64)),
    (1, 32, 16, (1, 8, 16, 64)),    # the 1x1x1 output convolution
])
def test_tcgen05_conv_matches_mma_sync(k, ci, co, vol):
    """The tcgen05 convolution (TMA-staged operands, zero padding from the
    TMA out-of-bounds fill, TMEM accumulator) against the mma.sync kernel on
    the same BF16 inputs: FP32 sums of the same products in another order."""
    import torch

    from pllcart3d_b200 import surrogate as S

    L = S.nnlib()
    rng = np.random.default_rng(ci * 7 + co)
    x = _t(_bf16(rng.standard_normal(vol + (ci,))).reshape(-1, ci), torch.bfloat16)
    w = _t(_bf16(rng.standard_normal((co, k ** 3, ci)) / np.sqrt(k ** 3 * ci)), torch.bfloat16)
    b = _t(rng.standard_normal(co), torch.float32)
    V = int(np.prod(vol))
    outs = []
    try:
        for path in (1, 2):
            L.pllnn_set_conv_path(path)
            z = torch.full((V, co), float("nan"), dtype=torch.float32, device="cuda")
            y = torch.empty((V, co), dtype=torch.bfloat16, device="cuda")
            assert L.pllnn_conv_fwd(S._p(x), *vol, ci, S._p(w), S._p(b), co, k, S._p(z), S._p(y), 1, S.SLOPE,
                                    S._stream()) == 0
            torch.cuda.synchronize()
            outs.append((z.cpu().numpy(), y.float().cpu().numpy()))
    finally:
        L.pllnn_set_conv_path(0)
    assert L.pllnn_status() == 0
    assert np.isfinite(outs[1][0]).all()
    assert _relerr(outs[1][0], outs[0][0]) < 1e-5
    assert _relerr(outs[1][1], outs[0][1]) < 1e-2
