"""Run parameters in the reference's ``param.input`` format.

``param.input`` is positional: 34 values, each on the line after a caption
line, read in this order by ``input()`` (pllcart3d.c:271-350).  The derived
globals follow ``simulation_setup`` (pllcart3d.c:394-433: ``M = Vratio``,
``Vnorm = 0``) and ``grid_setup`` (pllcart3d.c:353-392, one rank: the whole
x-range is one slab).

The named workloads at the bottom are the synthetic fingering cases this
project measures; their interface perturbation is described in :mod:`ic`.
"""

from __future__ import annotations

import dataclasses
import math
import os
from dataclasses import dataclass, field

# (name, type, caption) in the order of pllcart3d.c:279-346
PARAM_FIELDS = [
    ("Nx_cell_global", int, "Nx_cell_global - No. of cells in x globally"),
    ("Ny_cell_global", int, "Ny_cell_global - No. of cells in y globally"),
    ("Nz_cell_global", int, "Nz_cell_global - No. of cells in z globally"),
    ("Nx_ghost", int, "Nx_ghost - No. of ghost cells in x"),
    ("Ny_ghost", int, "Ny_ghost - No. of ghost cells in y"),
    ("Nz_ghost", int, "Nz_ghost - No. of ghost cells in z"),
    ("Initial", int, "Initial ?Start from initial cond(1) or intermediate(0)"),
    ("Ugrid", int, "Ugrid? uniform grid(1) or not(0)"),
    ("Niter_print", int, "Niter_print: No. of screen printing interval"),
    ("Out_mid", float, "Out_mid: time interval before storing midfield"),
    ("X1", float, "X1: left end of domain"),
    ("X2", float, "X2: right end of domain"),
    ("Y1", float, "Y1:bottom end of domain"),
    ("Y2", float, "Y2:top end of domain"),
    ("Z1", float, "Z1:side end of domain"),
    ("Z2", float, "Z2:side domain"),
    ("Timemax", float, "Timemax: Maximum simulation time"),
    ("Timestep", float, "Timestep: time marching step"),
    ("Re", float, "Re: Reynolds number"),
    ("Pe", float, "Pe: Peclet number"),
    ("Vratio", float, "Vratio: viscosity ratio(M)-log(mu2/mu1)"),
    ("Fx", float, "Fx: Density parameter in x-dir"),
    ("Fy", float, "Fy: Density parameter in y-dir"),
    ("Inf_pos", float, "Inf_pos: Initial interface position"),
    ("Inf_thick", float, "Inf_thick: Initial interface thickness"),
    ("CFLmax", float, "CFLmax: Maximum bound for CFL number"),
    ("Out_inter", float, "Out_inter: output time interval for writing to file for plotting"),
    ("Wavpert", int, "Wavpert ? add wave perturbation in the spanwise direction (1) or not (0)"),
    ("Ampli", float, "Ampli: amplitude of Wavpert"),
    ("Lamb", float, "Lamb: wavelength of Wavpert"),
    ("Subharm", int, "Subharm: ? add sub-harmonic perturbation (1) or not (0)"),
    ("Nmvp", int, "Nmvp: ? use non-monotonic viscosity profile (1) or exponential correlation (0)"),
    ("Mum", float, "Mum: maximum viscosity of non-monotonic viscosity profile"),
    ("Lambda", float, "Lambda: parameter that relates end point slopes of nm viscosity profile"),
]


@dataclass
class Params:
    """The 34 ``param.input`` values (pllcart3d.c:271-350)."""

    Nx_cell_global: int = 64
    Ny_cell_global: int = 32
    Nz_cell_global: int = 32
    Nx_ghost: int = 3
    Ny_ghost: int = 1
    Nz_ghost: int = 1
    Initial: int = 1
    Ugrid: int = 1
    Niter_print: int = 1000000
    Out_mid: float = 1.0e9
    X1: float = 0.0
    X2: float = 4.0
    Y1: float = -0.5
    Y2: float = 0.5
    Z1: float = -0.5
    Z2: float = 0.5
    Timemax: float = 1.0e9
    Timestep: float = 1.0
    Re: float = 100.0
    Pe: float = 1000.0
    Vratio: float = -2.0
    Fx: float = 0.0
    Fy: float = 0.0
    Inf_pos: float = 1.0
    Inf_thick: float = 0.02
    CFLmax: float = 0.5
    Out_inter: float = 1.0e9
    Wavpert: int = 0
    Ampli: float = 0.1
    Lamb: float = 3.0
    Subharm: int = 0
    Nmvp: int = 0
    Mum: float = 1.5
    Lambda: float = 0.0

    # ---- derived quantities (one rank) -------------------------------------
    @property
    def nx(self) -> int:
        return self.Nx_cell_global

    @property
    def ny(self) -> int:
        return self.Ny_cell_global

    @property
    def nz(self) -> int:
        return self.Nz_cell_global

    @property
    def shape(self) -> tuple:
        """Padded array shape (nx_max, ny_max, nz_max), pllcart3d.c:361-363."""
        return (self.nx + 2 * self.Nx_ghost, self.ny + 2 * self.Ny_ghost,
                self.nz + 2 * self.Nz_ghost)

    @property
    def dx(self) -> float:
        return (self.X2 - self.X1) / float(self.Nx_cell_global)

    @property
    def dy(self) -> float:
        return (self.Y2 - self.Y1) / float(self.Ny_cell_global)

    @property
    def dz(self) -> float:
        return (self.Z2 - self.Z1) / float(self.Nz_cell_global)

    @property
    def M(self) -> float:
        """Viscosity exponent, ``M = Vratio`` (pllcart3d.c:400)."""
        return self.Vratio

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def timestep_cap(self) -> float:
        """``Timestep`` after the diffusive cap of pllcart3d.c:150-154."""
        dmin = self.dx if self.dx < self.dy else self.dy
        dmin = dmin if dmin < self.dz else self.dz
        diff_dt = 0.1 * self.Pe * dmin * dmin
        return diff_dt if diff_dt < self.Timestep else self.Timestep

    def validate(self) -> None:
        """Reject settings the reference's stencils cannot run with."""
        if (self.Nx_ghost, self.Ny_ghost, self.Nz_ghost) != (3, 1, 1):
            raise ValueError("the stencils need Nx_ghost=3, Ny_ghost=Nz_ghost=1")
        if min(self.nx, self.ny, self.nz) < 4:
            raise ValueError("each direction needs at least 4 interior cells")
        if self.Nmvp not in (0, 1):
            raise ValueError("Nmvp must be 0 or 1")

    # ---- file format --------------------------------------------------------
    def to_text(self) -> str:
        lines = []
        for name, typ, caption in PARAM_FIELDS:
            val = getattr(self, name)
            lines.append("//" + caption)
            lines.append(str(int(val)) if typ is int else repr(float(val)))
        return "\n".join(lines) + "\n"

    def write(self, path: str) -> str:
        """Write ``param.input``; *path* is a directory or a file name."""
        if os.path.isdir(path):
            path = os.path.join(path, "param.input")
        with open(path, "w") as f:
            f.write(self.to_text())
        return path

    @classmethod
    def read(cls, path: str) -> "Params":
        """Parse ``param.input`` the way ``input()`` does: caption, value, ..."""
        if os.path.isdir(path):
            path = os.path.join(path, "param.input")
        with open(path) as f:
            lines = [ln.strip() for ln in f.read().splitlines()]
        vals = {}
        pos = 0
        for name, typ, _ in PARAM_FIELDS:
            pos += 1  # caption line
            while pos < len(lines) and lines[pos] == "":
                pos += 1
            if pos >= len(lines):
                raise ValueError(f"param.input ends before {name}")
            tok = lines[pos].split()[0]
            vals[name] = int(tok) if typ is int else float(tok)
            pos += 1
        return cls(**vals)

    def replace(self, **kw) -> "Params":
        return dataclasses.replace(self, **kw)


@dataclass
class Workload:
    """A named synthetic fingering case: run parameters + interface recipe."""

    name: str
    params: Params
    modes: int = 8
    amplitude: float = 0.01
    steps: int = 200
    seed: int = 20240611
    precision: str = "fp64"


def workload(name: str) -> Workload:
    """Named cases.

    ``fingering-64x32x32``: plain FP64, R=2 (Vratio=-2), Re=100, Pe=1000,
    8 modes of amplitude 0.01, interface width 0.02, 200 steps at CFL 0.5.
    ``fingering-256x128x128``: R=3, Re=500, Pe=2000, 16 modes of amplitude
    0.005, width 0.01, 1000 steps.
    ``fingering-512x256x256``: R=2.5, Re=1000, Pe=5000, density contrast with
    Atwood number 0.05 acting along -y through the reference's ``Fy`` term
    (the reference has body forces along x and y only, pllcart3d.c:984,1141,
    1293); ``Fy = 2 At Re`` for g L / U^2 = 1.
    """
    base = Params()
    if name in ("fingering-64x32x32", "cfg0"):
        return Workload("fingering-64x32x32", base, modes=8, amplitude=0.01,
                        steps=200)
    if name in ("fingering-256x128x128", "cfg1"):
        p = base.replace(Nx_cell_global=256, Ny_cell_global=128,
                         Nz_cell_global=128, Vratio=-3.0, Re=500.0, Pe=2000.0,
                         Inf_thick=0.01)
        return Workload("fingering-256x128x128", p, modes=16, amplitude=0.005,
                        steps=1000)
    if name in ("fingering-512x256x256", "cfg2"):
        at = 0.05
        p = base.replace(Nx_cell_global=512, Ny_cell_global=256,
                         Nz_cell_global=256, Vratio=-2.5, Re=1000.0,
                         Pe=5000.0, Inf_thick=0.01, Fy=2.0 * at * 1000.0)
        return Workload("fingering-512x256x256", p, modes=16, amplitude=0.005,
                        steps=1000, precision="mixed")
    m = _parse_small(name)
    if m is not None:
        return m
    raise KeyError(name)


def _parse_small(name: str):
    """``fingering-NXxNYxNZ`` for any size, with the 64x32x32 physics."""
    if not name.startswith("fingering-"):
        return None
    try:
        nx, ny, nz = (int(t) for t in name[len("fingering-"):].split("x"))
    except ValueError:
        return None
    p = Params().replace(Nx_cell_global=nx, Ny_cell_global=ny,
                         Nz_cell_global=nz)
    return Workload(name, p, modes=8, amplitude=0.01, steps=200)


PI = 4.0 * math.atan(1.0)  # pllcart3d.c:397
