"""Learned surrogate of the fingering step: a 3-d convolutional U-Net that
advances the cell-centred state (c, u, v, w) of a run by 8 steps, followed by
the solver's own DCT pressure projection, inside a rollout judged by the
plain FP64 solver.

Network (channels-last, BF16 weights and activations, FP32 accumulation):

    input 16 ch = (c, u, v, w) normalised, R/3, log(Pe/500)/log(10), 10 zeros
    e1 conv3 16->32   e2 conv3 32->64   e3 conv3 64->128   e4 conv3 128->256
      (each after a 2x average pooling of the previous level's output)
    d3 conv3 (up(e4) | e3) 384->128   d2 conv3 (up(d3) | e2) 192->64
    d1 conv3 (up(d2) | e1) 96->32     out conv1 32->16 (channels 0-3 used)
    leaky ReLU (slope 0.1) after every 3x3x3 convolution; 2.9 M parameters

The output is the 8-step change of (c, u, v, w) over its per-channel scale.
Every operation runs in pllcart3d_b200/csrc/nn.cu (libpllnn.so): the
convolutions' forward, input-gradient and weight-gradient passes on the BF16
tensor cores, pooling, upsampling, concatenation, loss and Adam; torch only
allocates the device buffers.  Training data: snapshots every 8 steps of an
ensemble of runs (pllcart3d_b200.ensemble).

Rollout protocol: windows of 8 steps; the network advances the state, the
solver projects it (``Solver.project``).  Every 4th window the plain FP64
solver re-runs the window from the same start (a second context with the
same state, ``copy_state_from``); the surrogate window is rejected, and the
solver's state taken, when its mass or mixing length differs from the
solver's by more than 1e-3 (relative).

    python -m pllcart3d_b200.surrogate [--train-steps N] [--rollout 2000] ...
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NNLIB = os.path.join(HERE, "libpllnn.so")
SLOPE = 0.1
WINDOW = 8

_nn = None


def nnlib():
    """The kernel library; there is no fallback when it is missing."""
    global _nn
    if _nn is None:
        if not os.path.exists(NNLIB):
            raise ImportError(f"{NNLIB} not built (python -m pllcart3d_b200.build)")
        L = ctypes.CDLL(NNLIB)
        P, I, F, Lg = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_long
        L.pllnn_conv_fwd.argtypes = [P, I, I, I, I, I, P, P, I, I, P, P, I, F, P]
        L.pllnn_conv_wgrad.argtypes = [P, P, I, I, I, I, I, I, I, P, P]
        L.pllnn_flip.argtypes = [P, I, I, I, P, P]
        L.pllnn_act_bwd.argtypes = [P, P, Lg, I, I, F, P, P, P]
        L.pllnn_pool_fwd.argtypes = [P, I, I, I, I, I, P, P]
        L.pllnn_pool_bwd.argtypes = [P, I, I, I, I, I, P, I, P]
        L.pllnn_up_fwd.argtypes = [P, I, I, I, I, I, P, P]
        L.pllnn_up_bwd.argtypes = [P, I, I, I, I, I, P, I, P]
        L.pllnn_cat_fwd.argtypes = [P, I, P, I, Lg, P, P]
        L.pllnn_cat_bwd.argtypes = [P, I, I, Lg, P, I, P, I, P]
        L.pllnn_mse.argtypes = [P, P, Lg, F, P, P, P]
        L.pllnn_adam.argtypes = [P, P, P, P, Lg, F, F, F, F, I, P, P, F, P]
        L.pllnn_sumsq.argtypes = [P, Lg, P, P]
        L.pllnn_cast.argtypes = [P, Lg, P, P]
        L.pllnn_pack_input.argtypes = [P, Lg, F, F, P, P, P]
        L.pllnn_pack_target.argtypes = [P, P, Lg, P, P, P]
        L.pllnn_apply_delta.argtypes = [P, P, Lg, P, P, P]
        L.pllnn_set_conv_path.argtypes = [I]
        L.pllnn_status.argtypes = []
        _nn = L
    return _nn


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _ok(code, what):
    if code != 0:
        raise RuntimeError(f"{what} failed ({code})")


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Conv:
    """One convolution (3x3x3 or 1x1x1) with bias and optional leaky ReLU."""

    def __init__(self, name, cin, cout, k, act, rng, device="cuda"):
        import torch

        self.name, self.cin, self.cout, self.k, self.act = name, cin, cout, k, act
        fan = k ** 3 * cin
        w = rng.standard_normal((cout, k ** 3, cin)) * math.sqrt(2.0 / fan)
        if not act:
            w *= 0.1   # output layer starts near zero change
        self.w32 = torch.tensor(w, dtype=torch.float32, device=device).contiguous()
        self.b32 = torch.zeros(cout, dtype=torch.float32, device=device)
        self.w16 = torch.empty(self.w32.shape, dtype=torch.bfloat16, device=device)
        self.wf16 = torch.empty((cin, k ** 3, cout), dtype=torch.bfloat16, device=device)
        self.gw = torch.zeros_like(self.w32)
        self.gb = torch.zeros_like(self.b32)
        self.mw, self.vw = torch.zeros_like(self.w32), torch.zeros_like(self.w32)
        self.mb, self.vb = torch.zeros_like(self.b32), torch.zeros_like(self.b32)
        self.refresh()

    def refresh(self):
        L, st = nnlib(), _stream()
        _ok(L.pllnn_cast(_p(self.w32), self.w32.numel(), _p(self.w16), st), "cast")
        _ok(L.pllnn_flip(_p(self.w16), self.cout, self.k ** 3, self.cin, _p(self.wf16), st), "flip")

    def forward(self, x16, vol):
        import torch

        V = vol[0] * vol[1] * vol[2] * vol[3]
        z = torch.empty((V, self.cout), dtype=torch.float32, device=x16.device)
        y = torch.empty((V, self.cout), dtype=torch.bfloat16, device=x16.device) if self.act else None
        _ok(nnlib().pllnn_conv_fwd(_p(x16), *vol, self.cin, _p(self.w16), _p(self.b32), self.cout, self.k, _p(z),
                                   _p(y), int(self.act), SLOPE, _stream()), f"{self.name} forward")
        self.x, self.z, self.vol = x16, z, vol
        return y if self.act else z

    def backward(self, gy32, need_dx=True):
        import torch

        L, st = nnlib(), _stream()
        V = self.z.shape[0]
        dz = torch.empty((V, self.cout), dtype=torch.bfloat16, device=gy32.device)
        _ok(L.pllnn_act_bwd(_p(gy32), _p(self.z), V, self.cout, int(self.act), SLOPE, _p(dz), _p(self.gb), st),
            "act backward")
        _ok(L.pllnn_conv_wgrad(_p(dz), _p(self.x), *self.vol, self.cin, self.cout, self.k, _p(self.gw), st),
            "weight gradient")
        if not need_dx:
            return None
        dx = torch.empty((V, self.cin), dtype=torch.float32, device=gy32.device)
        _ok(L.pllnn_conv_fwd(_p(dz), *self.vol, self.cout, _p(self.wf16), None, self.cin, self.k, _p(dx), None, 0,
                             SLOPE, st), "input gradient")
        return dx

    def params(self):
        return [(self.w32, self.gw, self.mw, self.vw), (self.b32, self.gb, self.mb, self.vb)]


LAYERS = (("e1", 16, 32, 3, 1), ("e2", 32, 64, 3, 1), ("e3", 64, 128, 3, 1), ("e4", 128, 256, 3, 1),
          ("d3", 384, 128, 3, 1), ("d2", 192, 64, 3, 1), ("d1", 96, 32, 3, 1), ("out", 32, 16, 1, 0))


class UNet:
    def __init__(self, seed=0, device="cuda"):
        rng = np.random.default_rng(seed)
        self.layers = {n: Conv(n, ci, co, k, a, rng, device) for n, ci, co, k, a in LAYERS}
        self.t = 0

    def n_params(self):
        return sum(c.w32.numel() + c.b32.numel() for c in self.layers.values())

    def forward(self, x16, vol):
        import torch

        L, st = nnlib(), _stream()
        B, D, H, W = vol
        l = self.layers
        dev = x16.device
        vols = [(B, D >> s, H >> s, W >> s) for s in range(4)]
        Vs = [v[0] * v[1] * v[2] * v[3] for v in vols]

        def pool(x, s, C):
            y = torch.empty((Vs[s + 1], C), dtype=torch.bfloat16, device=dev)
            _ok(L.pllnn_pool_fwd(_p(x), *vols[s], C, _p(y), st), "pool")
            return y

        def upcat(x, s, C, skip, CS):
            u = torch.empty((Vs[s - 1], C), dtype=torch.bfloat16, device=dev)
            _ok(L.pllnn_up_fwd(_p(x), *vols[s], C, _p(u), st), "up")
            y = torch.empty((Vs[s - 1], C + CS), dtype=torch.bfloat16, device=dev)
            _ok(L.pllnn_cat_fwd(_p(u), C, _p(skip), CS, Vs[s - 1], _p(y), st), "cat")
            return y

        e1 = l["e1"].forward(x16, vols[0])
        e2 = l["e2"].forward(pool(e1, 0, 32), vols[1])
        e3 = l["e3"].forward(pool(e2, 1, 64), vols[2])
        e4 = l["e4"].forward(pool(e3, 2, 128), vols[3])
        d3 = l["d3"].forward(upcat(e4, 3, 256, e3, 128), vols[2])
        d2 = l["d2"].forward(upcat(d3, 2, 128, e2, 64), vols[1])
        d1 = l["d1"].forward(upcat(d2, 1, 64, e1, 32), vols[0])
        self._vols, self._Vs = vols, Vs
        return l["out"].forward(d1, vols[0])

    def backward(self, gout):
        import torch

        L, st = nnlib(), _stream()
        l, vols, Vs = self.layers, self._vols, self._Vs
        dev = gout.device

        def cat_up_bwd(gc, s, C, CS, gskip):
            """gc over (up(x) | skip) at level s-1 -> grad of x (level s);
            the skip's share goes into gskip (overwritten)."""
            gu = torch.empty((Vs[s - 1], C), dtype=torch.float32, device=dev)
            _ok(L.pllnn_cat_bwd(_p(gc), C, CS, Vs[s - 1], _p(gu), 0, _p(gskip), 0, st), "cat backward")
            gx = torch.empty((Vs[s], C), dtype=torch.float32, device=dev)
            _ok(L.pllnn_up_bwd(_p(gu), *vols[s], C, _p(gx), 0, st), "up backward")
            return gx

        def pool_bwd_acc(g, s, C, into):
            _ok(L.pllnn_pool_bwd(_p(g), *vols[s], C, _p(into), 1, st), "pool backward")

        ge1 = torch.empty((Vs[0], 32), dtype=torch.float32, device=dev)
        ge2 = torch.empty((Vs[1], 64), dtype=torch.float32, device=dev)
        ge3 = torch.empty((Vs[2], 128), dtype=torch.float32, device=dev)
        gd1 = l["out"].backward(gout)
        gc1 = l["d1"].backward(gd1)
        gd2 = cat_up_bwd(gc1, 1, 64, 32, ge1)
        gc2 = l["d2"].backward(gd2)
        gd3 = cat_up_bwd(gc2, 2, 128, 64, ge2)
        gc3 = l["d3"].backward(gd3)
        ge4 = cat_up_bwd(gc3, 3, 256, 128, ge3)
        pool_bwd_acc(l["e4"].backward(ge4), 2, 128, ge3)
        pool_bwd_acc(l["e3"].backward(ge3), 1, 64, ge2)
        pool_bwd_acc(l["e2"].backward(ge2), 0, 32, ge1)
        l["e1"].backward(ge1, need_dx=False)

    def zero_grad(self):
        for c in self.layers.values():
            c.gw.zero_()
            c.gb.zero_()

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8, clip=1.0):
        """One Adam step with global gradient-norm clipping at `clip`
        (norm reduced on the device; a non-finite norm skips the step)."""
        import torch

        L, st = nnlib(), _stream()
        self.t += 1
        if not hasattr(self, "_sumsq"):
            self._sumsq = torch.zeros(1, dtype=torch.float32, device="cuda")
        self._sumsq.zero_()
        for c in self.layers.values():
            for (w, g, m, v) in c.params():
                _ok(L.pllnn_sumsq(_p(g), g.numel(), _p(self._sumsq), st), "sumsq")
        for c in self.layers.values():
            for (w, g, m, v), w16 in zip(c.params(), (c.w16, None)):
                _ok(L.pllnn_adam(_p(w), _p(g), _p(m), _p(v), w.numel(), lr, b1, b2, eps, self.t, _p(w16),
                                 _p(self._sumsq), clip, st), "adam")
            _ok(L.pllnn_flip(_p(c.w16), c.cout, c.k ** 3, c.cin, _p(c.wf16), st), "flip")

    def state_dict(self):
        return {n: (c.w32.cpu().numpy(), c.b32.cpu().numpy()) for n, c in self.layers.items()}

    def load_state_dict(self, sd):
        import torch

        for n, (w, b) in sd.items():
            c = self.layers[n]
            c.w32.copy_(torch.tensor(w))
            c.b32.copy_(torch.tensor(b))
            c.refresh()


# ---- data ------------------------------------------------------------------

def const_channels(R, Pe):
    return float(R / 3.0), float(math.log(Pe / 500.0) / math.log(10.0))


class Dataset:
    """(state_t, state_t+8) pairs of cell arrays [V][4] (u, v, w, c) FP32 on
    the device, with each run's (R, Pe)."""

    def __init__(self):
        self.a, self.b, self.rp, self.vol = [], [], [], None

    def add_run(self, snaps, R, Pe):
        for s0, s1 in zip(snaps[:-1], snaps[1:]):
            self.a.append(s0)
            self.b.append(s1)
            self.rp.append(const_channels(R, Pe))

    def stats(self, nsample=64):
        """Input mean / std and target scale per channel (c, u, v, w)."""
        idx = np.linspace(0, len(self.a) - 1, min(nsample, len(self.a))).astype(int)
        A = np.stack([self.a[i].cpu().numpy() for i in idx])   # [n][V][4] (u,v,w,c)
        Bm = np.stack([self.b[i].cpu().numpy() for i in idx])
        order = [3, 0, 1, 2]
        mean = A.reshape(-1, 4).mean(0)[order]
        std = A.reshape(-1, 4).std(0)[order] + 1e-6
        dsc = (Bm - A).reshape(-1, 4).std(0)[order] + 1e-9
        return np.concatenate([mean, std]).astype(np.float32), dsc.astype(np.float32)


def generate_data(n_runs=8, grid=(128, 64, 64), steps=400, precision="mixed", seed=4321, every=WINDOW):
    """Ensemble runs (pllcart3d_b200.ensemble) snapshotted every `every` steps."""
    import torch

    from .ensemble import Ensemble, random_members

    wls = random_members(n_runs * 4, seed)
    wls = [w for w in wls if (w.params.nx, w.params.ny, w.params.nz) == tuple(grid)][:n_runs]
    while len(wls) < n_runs:   # draw more members of this grid
        seed += 1
        wls += [w for w in random_members(16, seed) if (w.params.nx, w.params.ny, w.params.nz) == tuple(grid)]
        wls = wls[:n_runs]
    ens = Ensemble(wls, precision=precision)
    ens.load_ics()
    V = grid[0] * grid[1] * grid[2]
    snaps = [[] for _ in wls]

    def grab():
        for i, m in enumerate(ens.members):
            t = torch.empty((V, 4), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            m.pack_cells(t.data_ptr())
            snaps[i].append(t)

    grab()
    for _ in range(steps // every):
        ens.step(every)
        grab()
    ds = Dataset()
    ds.vol = tuple(grid)
    for s, w in zip(snaps, wls):
        ds.add_run(s, -w.params.Vratio, w.params.Pe)
    ens.close()
    return ds, wls


class Trainer:
    def __init__(self, net: UNet, ds: Dataset, batch=8, lr=3e-4, seed=0):
        import torch

        self.net, self.ds, self.batch, self.lr = net, ds, batch, lr
        self.norm, self.dscale = ds.stats()
        self.norm_t = torch.tensor(self.norm, device="cuda")
        self.dscale_t = torch.tensor(self.dscale, device="cuda")
        self.rng = np.random.default_rng(seed)
        D, H, W = ds.vol
        self.V = D * H * W
        self.x16 = torch.empty((batch * self.V, 16), dtype=torch.bfloat16, device="cuda")
        self.tgt = torch.empty((batch * self.V, 16), dtype=torch.float32, device="cuda")
        self.grad = torch.empty_like(self.tgt)
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")

    def pack(self, idx, x16, tgt):
        L, st = nnlib(), _stream()
        V = self.V
        for k, i in enumerate(idx):
            r, p = self.ds.rp[i]
            _ok(L.pllnn_pack_input(_p(self.ds.a[i]), V, r, p, _p(self.norm_t), _p(x16[k * V:(k + 1) * V]), st),
                "pack input")
            if tgt is not None:
                _ok(L.pllnn_pack_target(_p(self.ds.a[i]), _p(self.ds.b[i]), V, _p(self.dscale_t),
                                        _p(tgt[k * V:(k + 1) * V]), st), "pack target")

    def step(self, idx=None):
        L, st = nnlib(), _stream()
        if idx is None:
            idx = self.rng.integers(0, len(self.ds.a), self.batch)
        self.pack(idx, self.x16, self.tgt)
        D, H, W = self.ds.vol
        out = self.net.forward(self.x16, (len(idx), D, H, W))
        self.net.zero_grad()
        n = len(idx) * self.V * 16
        _ok(L.pllnn_mse(_p(out), _p(self.tgt), n, 1.0 / (len(idx) * self.V * 4), _p(self.grad), _p(self.loss), st),
            "mse")
        self.net.backward(self.grad)
        self.net.adam(self.lr)

    def eval_loss(self, idx):
        """Mean squared normalised error of the network and of persistence
        (predicting no change) on samples idx."""
        import torch

        L, st = nnlib(), _stream()
        D, H, W = self.ds.vol
        tot = tot0 = 0.0
        for i in idx:
            self.pack([i], self.x16, self.tgt)
            out = self.net.forward(self.x16[:self.V], (1, D, H, W))
            self.loss.zero_()
            _ok(L.pllnn_mse(_p(out), _p(self.tgt[:self.V]), self.V * 16, 1.0 / (self.V * 4), None, _p(self.loss),
                            st), "mse")
            tot += float(self.loss.item())
            zero = torch.zeros_like(out)
            self.loss.zero_()
            _ok(L.pllnn_mse(_p(zero), _p(self.tgt[:self.V]), self.V * 16, 1.0 / (self.V * 4), None, _p(self.loss),
                            st), "mse")
            tot0 += float(self.loss.item())
        return tot / len(idx), tot0 / len(idx)


# ---- rollout ---------------------------------------------------------------

MASS_FIX_MIN_ZONE = 0.005   # the mixing zone's share of the cells below which c is left as predicted
MASS_FIX_MAX_SHIFT = 0.02   # largest change of c per zone cell the mass correction applies

class Surrogate:
    """Network + normalisation of one grid, acting on a Solver's state."""

    def __init__(self, net: UNet, norm, dscale, grid):
        import torch

        self.net = net
        self.norm_t = torch.tensor(norm, device="cuda")
        self.dscale_t = torch.tensor(dscale, device="cuda")
        self.grid = tuple(grid)
        self.V = grid[0] * grid[1] * grid[2]
        self.cells = torch.empty((self.V, 4), dtype=torch.float32, device="cuda")
        self.next = torch.empty_like(self.cells)
        self.x16 = torch.empty((self.V, 16), dtype=torch.bfloat16, device="cuda")

    def advance(self, solver, R, Pe, mass_target=None, dV=None):
        """One window: network prediction, then the solver's projection.
        With `mass_target` (and the cell volume dV) the predicted c is made
        to carry that mass: the difference is spread evenly over the cells
        of the mixing zone (0.01 < c < 0.99), leaving the pure-fluid regions
        as predicted; skipped when the zone is under MASS_FIX_MIN_ZONE of the
        cells or the shift would exceed MASS_FIX_MAX_SHIFT."""
        import torch

        L, st = nnlib(), _stream()
        torch.cuda.synchronize()
        solver.pack_cells(self.cells.data_ptr())
        r, p = const_channels(R, Pe)
        _ok(L.pllnn_pack_input(_p(self.cells), self.V, r, p, _p(self.norm_t), _p(self.x16), st), "pack input")
        out = self.net.forward(self.x16, (1,) + self.grid)
        _ok(L.pllnn_apply_delta(_p(self.cells), _p(out), self.V, _p(self.dscale_t), _p(self.next), st), "apply")
        if mass_target is not None:
            c = self.next[:, 3]   # cells are (u, v, w, c)
            zone = (c > 0.01) & (c < 0.99)
            n = int(zone.sum().item())
            # only while the mixing zone is a real part of the volume and the
            # shift stays small: once the displaced fluid has left the box
            # the zone is a few cells and the mass history no longer a guide
            if n >= MASS_FIX_MIN_ZONE * self.V:
                m = float(c.double().sum().item()) * dV
                shift = (mass_target - m) / (n * dV)
                if abs(shift) <= MASS_FIX_MAX_SHIFT:
                    c[zone] += float(shift)
        torch.cuda.synchronize()
        solver.unpack_cells(self.next.data_ptr())
        solver.project()


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def rollout(sur: Surrogate, wl, steps=2000, judge_every=4, tol=1e-3, precision="fp64", mass_fix=True):
    """Surrogate + judge rollout of `steps` steps; returns a report.

    Windows of 8 steps.  Every `judge_every`-th window the plain solver runs
    the same window from the same start on a second context; the surrogate
    window is rejected when mass or mixing length differ by more than `tol`
    (or the solver cannot step from that start).  A rejection, or a
    non-finite prediction anywhere, sends the rollout back to the last state
    a judge verified, and the solver runs every window since: the state is
    verified at every judged window.

    mass_fix: the network's c is corrected to the mass the run had at the
    window's start plus the mass change of the previous window (the inflow
    adds mass at a nearly constant rate); the judge's own result is never
    used for it."""
    import torch

    from . import _lib
    from .ic import workload_fields
    from .solver import Solver

    R, Pe = -wl.params.Vratio, wl.params.Pe
    ic = workload_fields(wl)
    S = Solver(wl.params, precision=precision)       # the rollout state
    J = Solver(wl.params, precision=precision)       # the judge
    Sgood = Solver(wl.params, precision=precision)   # last verified state
    for x in (S, J, Sgood):
        x.load_ic(ic)
    wgood = 0
    nwin = steps // WINDOW
    judged = rejected = failed = broken = 0
    trace = []

    def solver_window(start):
        """The solver's window from `start` into J; False when the start
        state makes the solver fail (NaN/Inf)."""
        J.copy_state_from(start)
        try:
            J.step(WINDOW)
            return True
        except _lib.PllGpuError:
            J.clear_status()
            return False

    def fall_back(w):
        """Rejection: back to the last verified state; the solver runs every
        window since (the result is verified by construction)."""
        nonlocal wgood
        J.copy_state_from(Sgood)
        J.step(WINDOW * (w + 1 - wgood))
        S.copy_state_from(J)
        Sgood.copy_state_from(S)
        wgood = w + 1

    dV = wl.params.dx * wl.params.dy * wl.params.dz
    m_prev = None   # mass at the previous window's start
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for w in range(nwin):
        judge = (w % judge_every) == judge_every - 1
        judged_ok = solver_window(S) if judge else False
        m_now = S.diagnostics()["mass"] if mass_fix else None
        target = (2.0 * m_now - m_prev) if (mass_fix and m_prev is not None) else None
        sur.advance(S, R, Pe, target, dV)
        m_prev = m_now
        ds = S.diagnostics()
        finite = all(math.isfinite(x) for x in ds.values())
        if not finite:
            failed += 1
        if not judge:
            if not finite:
                fall_back(w)
            continue
        judged += 1
        if not judged_ok or not finite:
            broken += int(not judged_ok)
            rejected += 1
            fall_back(w)
            continue
        dj = J.diagnostics()
        if len(trace) < 16:
            trace.append({"window": w, "mass_rel": rel(ds["mass"], dj["mass"]),
                          "ml": ds["mixing_length"], "ml_solver": dj["mixing_length"]})
        if rel(ds["mass"], dj["mass"]) > tol or rel(ds["mixing_length"], dj["mixing_length"]) > tol:
            rejected += 1
            fall_back(w)
        else:
            Sgood.copy_state_from(S)
            wgood = w + 1
    torch.cuda.synchronize()
    t_roll = time.perf_counter() - t0
    # the plain FP64 run of the same steps
    P = Solver(wl.params, precision=precision)
    P.load_ic(ic)
    P.step(2)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    P.step(steps - 2)
    torch.cuda.synchronize()
    t_plain = (time.perf_counter() - t1) * steps / (steps - 2)
    ds, dp = S.diagnostics(), P.diagnostics()
    c_err = float(np.abs(S.get("c_new") - P.get("c_new")).max())
    return {"steps": steps, "windows": nwin, "judged": judged, "rejected": rejected,
            "accepted_fraction_of_judged": (judged - rejected) / max(judged, 1),
            "nonfinite_windows": failed, "judge_failed_windows": broken, "judge_trace": trace,
            "mixing_length": ds["mixing_length"], "mixing_length_plain": dp["mixing_length"],
            "mixing_length_rel_error": rel(ds["mixing_length"], dp["mixing_length"]),
            "mass_rel_error": rel(ds["mass"], dp["mass"]), "c_maxnorm_error": c_err,
            "wall_s_rollout": t_roll, "wall_s_plain": t_plain, "speedup": t_plain / t_roll}


def bench_conv(batch=8, grid=(128, 64, 64), reps=10):
    """Forward convolution of every U-Net layer at its own level, on the
    tcgen05 kernel and on the mma.sync kernel: mean ms per launch (CUDA
    events) and TFLOP/s (2 x voxels x taps x Cin x Cout per launch)."""
    import torch

    L, st = nnlib(), _stream()
    rng = np.random.default_rng(0)
    levels = {"e1": 0, "e2": 1, "e3": 2, "e4": 3, "d3": 2, "d2": 1, "d1": 0, "out": 0}
    rows = []
    for n, ci, co, k, a in LAYERS:
        s_ = levels[n]
        vol = (batch, grid[0] >> s_, grid[1] >> s_, grid[2] >> s_)
        V = int(np.prod(vol))
        x = torch.tensor(rng.standard_normal((V, ci)), dtype=torch.bfloat16, device="cuda")
        w = torch.tensor(rng.standard_normal((co, k ** 3, ci)) * 0.05, dtype=torch.bfloat16, device="cuda")
        b = torch.zeros(co, dtype=torch.float32, device="cuda")
        z = torch.empty((V, co), dtype=torch.float32, device="cuda")
        y = torch.empty((V, co), dtype=torch.bfloat16, device="cuda")
        flops = 2.0 * V * k ** 3 * ci * co
        row = {"layer": n, "vol": list(vol), "cin": ci, "cout": co, "k": k}
        for path, name in ((2, "tcgen05"), (1, "mma_sync")):
            L.pllnn_set_conv_path(path)
            code = L.pllnn_conv_fwd(_p(x), *vol, ci, _p(w), _p(b), co, k, _p(z), _p(y), a, SLOPE, st)
            if code:
                row[name] = None
                continue
            torch.cuda.synchronize()
            e0, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                L.pllnn_conv_fwd(_p(x), *vol, ci, _p(w), _p(b), co, k, _p(z), _p(y), a, SLOPE, st)
            e1_.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1_) / reps
            row[name] = {"ms": ms, "tflops": flops / (ms / 1e3) / 1e12}
        L.pllnn_set_conv_path(0)
        rows.append(row)
    tot = {name: sum(r[name]["ms"] for r in rows if r.get(name)) for name in ("tcgen05", "mma_sync")}
    fl = sum(2.0 * np.prod(r["vol"]) * r["k"] ** 3 * r["cin"] * r["cout"] for r in rows)
    return {"batch": batch, "grid": list(grid), "layers": rows,
            "forward_ms": tot, "forward_tflops": {k_: fl / (v / 1e3) / 1e12 for k_, v in tot.items()},
            "status": L.pllnn_status()}


def main(argv=None) -> int:
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=8)
    ap.add_argument("--data-steps", type=int, default=400)
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-4)
    ap.add_argument("--rollout", type=int, default=2000)
    ap.add_argument("--grid", default="128x64x64")
    ap.add_argument("--save", default=None)
    ap.add_argument("--load", default=None, help="a network saved by --save: skip training")
    ap.add_argument("--data-precision", default="fp64", choices=["fp64", "mixed64", "mixed"],
                    help="form of the runs that make the training data (the judge runs the FP64 form)")
    ap.add_argument("--no-mass-fix", action="store_true")
    ap.add_argument("--out", default=None, help="also write the report JSON to this file")
    ap.add_argument("--bench-conv", action="store_true",
                    help="only time every layer's forward convolution on both kernels")
    args = ap.parse_args(argv)
    grid = tuple(int(t) for t in args.grid.split("x"))
    if args.bench_conv:
        rep = bench_conv(args.batch, grid)
        print(json.dumps(rep))
        if args.out:
            with open(args.out, "w") as f:
                json.dump(rep, f, indent=1)
        return 0
    t0 = time.perf_counter()
    ds, wls = generate_data(args.runs, grid, args.data_steps, precision=args.data_precision)
    t_data = time.perf_counter() - t0
    # hold out the last run for evaluation and the rollout
    per_run = len(ds.a) // args.runs
    held = list(range(len(ds.a) - per_run, len(ds.a)))
    train_idx = np.arange(0, len(ds.a) - per_run)
    net = UNet(seed=0)
    tr = Trainer(net, ds, batch=args.batch, lr=args.lr)
    if args.load:
        z = np.load(args.load)
        net.load_state_dict({n: (z[f"{n}_w"], z[f"{n}_b"]) for n in net.layers})
        tr.norm, tr.dscale = z["norm"], z["dscale"]
        tr.norm_t.copy_(torch.tensor(tr.norm))
        tr.dscale_t.copy_(torch.tensor(tr.dscale))
        args.train_steps = 0
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    curve = []
    for s in range(args.train_steps):
        log = s % 250 == 0 or s == args.train_steps - 1
        if log:
            tr.loss.zero_()
        tr.step(tr.rng.choice(train_idx, args.batch))
        if log:
            curve.append((s, float(tr.loss.item())))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    loss, loss0 = tr.eval_loss(held[::max(1, len(held) // 8)])
    if args.save:
        sd = net.state_dict()
        np.savez(args.save, norm=tr.norm, dscale=tr.dscale, **{f"{n}_w": w for n, (w, b) in sd.items()},
                 **{f"{n}_b": b for n, (w, b) in sd.items()})
    print(json.dumps({"phase": "trained", "train_s": t_train, "heldout_mse": loss,
                      "heldout_mse_persistence": loss0, "loss_curve": curve}), flush=True)
    sur = Surrogate(net, tr.norm, tr.dscale, grid)
    rep = rollout(sur, wls[-1], args.rollout, mass_fix=not args.no_mass_fix)
    rep.update({"grid": list(grid), "params": net.n_params(), "train_steps": args.train_steps,
                "data_precision": args.data_precision, "mass_fix": not args.no_mass_fix, "runs": args.runs,
                "data_steps": args.data_steps,
                "batch": args.batch, "train_s": t_train, "train_ms_per_step": 1e3 * t_train / max(1, args.train_steps),
                "data_s": t_data, "samples": len(ds.a), "heldout_mse": loss, "heldout_mse_persistence": loss0,
                "loss_curve": curve})
    print(json.dumps(rep))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
