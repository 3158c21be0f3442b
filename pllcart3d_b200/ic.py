"""Seeded synthetic initial condition for viscous-fingering runs.

The reference's own ``initial_condition`` (pllcart3d.c:493-552) is an erf
interface with a Poiseuille inlet and a fluid at rest.  The measured
workloads instead start from a perturbed interface in a uniform stream, built
once on the host in FP64 and handed identically to every implementation
(reference, CPU restatement and GPU), so no random-number implementation can
affect parity:

* pseudo-random numbers: splitmix64 (Steele, Lea, Flood 2014) from ``seed``;
  a uniform double is ``(x >> 11) * 2**-53``;
* ``modes`` Fourier modes, each with a wavenumber pair ``(ky, kz)`` drawn
  uniformly from ``{0..4}^2 \\ {(0,0)}`` and phases ``phi, psi`` uniform in
  ``[0, 2 pi)``, drawn in that order per mode;
* ``eta(y,z) = sum_m A cos(2 pi ky (y-Y1)/Ly + phi) cos(2 pi kz (z-Z1)/Lz + psi)``;
* ``c = 0.5 (1 - tanh((x - Inf_pos - eta) / Inf_thick))`` on every cell of the
  padded box (ghosts included, as pllcart3d.c:501-508 fills its IC);
* ``u = 1`` on every u face of the padded box, ``v = w = 0``.

Cell centres follow ``mesh_generation`` for one rank (pllcart3d.c:442-455).
Arrays are ``(nx_max, ny_max, nz_max)`` float64, z fastest, the reference's
``[i][j][k]`` order.
"""

from __future__ import annotations

import numpy as np

from .params import PI, Params, Workload

_MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & _MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)


def cell_centres(p: Params):
    """Xc, Yc, Zc over the padded box (pllcart3d.c:442-455, one rank)."""
    nxm, nym, nzm = p.shape
    dx, dy, dz = p.dx, p.dy, p.dz
    istart, jstart, kstart = p.Nx_ghost, p.Ny_ghost, p.Nz_ghost
    xstart = p.X1 + (0 - istart) * dx + (dx / 2.0)
    ystart = p.Y1 - jstart * dy + (dy / 2.0)
    zstart = p.Z1 - kstart * dz + (dz / 2.0)
    xc = np.array([xstart + i * dx for i in range(nxm)], dtype=np.float64)
    yc = np.array([ystart + j * dy for j in range(nym)], dtype=np.float64)
    zc = np.array([zstart + k * dz for k in range(nzm)], dtype=np.float64)
    return xc, yc, zc


def interface_modes(modes: int, seed: int):
    """(ky, kz, phi, psi) for each mode, in draw order."""
    rng = SplitMix64(seed)
    pairs = [(a, b) for a in range(5) for b in range(5) if (a, b) != (0, 0)]
    out = []
    for _ in range(modes):
        ky, kz = pairs[rng.next_u64() % len(pairs)]
        phi = 2.0 * PI * rng.uniform()
        psi = 2.0 * PI * rng.uniform()
        out.append((ky, kz, phi, psi))
    return out


def initial_fields(p: Params, modes: int = 8, amplitude: float = 0.01,
                   seed: int = 20240611):
    """Return dict(c, u, v, w) of padded float64 arrays."""
    xc, yc, zc = cell_centres(p)
    ly, lz = p.Y2 - p.Y1, p.Z2 - p.Z1
    eta = np.zeros((yc.size, zc.size), dtype=np.float64)
    for ky, kz, phi, psi in interface_modes(modes, seed):
        fy = np.cos(2.0 * PI * ky * (yc - p.Y1) / ly + phi)
        fz = np.cos(2.0 * PI * kz * (zc - p.Z1) / lz + psi)
        eta += amplitude * fy[:, None] * fz[None, :]
    arg = (xc[:, None, None] - p.Inf_pos - eta[None, :, :]) / p.Inf_thick
    c = 0.5 * (1.0 - np.tanh(arg))
    shape = p.shape
    u = np.ones(shape, dtype=np.float64)
    v = np.zeros(shape, dtype=np.float64)
    w = np.zeros(shape, dtype=np.float64)
    return {"c": np.ascontiguousarray(c), "u": u, "v": v, "w": w}


def workload_fields(wl: Workload):
    return initial_fields(wl.params, wl.modes, wl.amplitude, wl.seed)
