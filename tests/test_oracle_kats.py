"""Known-answer checks of the CPU restatement's numerics (no reference
needed): FFTW DCT definitions, the manufactured Poisson source of
pllcart3d.c:2029, Thomas against a dense solve, WENO5 exactness."""

import ctypes

import numpy as np
import pytest

from oracle.pyref import ORACLE_LIB, OracleRun
from pllcart3d_b200.params import PI, Params

P = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def olib():
    L = ctypes.CDLL(ORACLE_LIB)
    L.orc_weno.restype = ctypes.c_double
    L.orc_weno.argtypes = [P, ctypes.c_int, ctypes.c_int]
    L.orc_thomas_serial.argtypes = [ctypes.c_int, P, P, P, P]
    L.orc_thomas_pll.argtypes = [ctypes.c_int, P, P, P, P]
    L.pll_dct_matrix.argtypes = [ctypes.c_int, ctypes.c_int, P]
    L.pll_dct2d_fast.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
    return L


def p(a):
    return a.ctypes.data_as(P)


def dct_matrix(L, kind, n):
    T = np.zeros((n, n))
    L.pll_dct_matrix(kind, n, p(T))
    return T


@pytest.mark.parametrize("n", [4, 7, 16, 32])
def test_dct_definitions(olib, n):
    x = np.random.default_rng(n).standard_normal(n)
    j = np.arange(n)
    k = j[:, None]
    ref2 = 2.0 * (np.cos(PI * (2 * j[None, :] + 1) * k / (2 * n)) * x).sum(1)
    ref3 = x[0] + 2.0 * (np.cos(PI * j[None, 1:] * (2 * k + 1) / (2 * n)) * x[1:]).sum(1)
    assert np.allclose(dct_matrix(olib, 0, n) @ x, ref2, rtol=1e-13, atol=1e-13)
    assert np.allclose(dct_matrix(olib, 1, n) @ x, ref3, rtol=1e-13, atol=1e-13)
    # REDFT01(REDFT10(x)) = 2n x
    rt = dct_matrix(olib, 1, n) @ (dct_matrix(olib, 0, n) @ x)
    assert np.allclose(rt / (2 * n), x, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("n0,n1", [(8, 16), (32, 32)])
def test_fast_dct_matches_definition(olib, n0, n1):
    x = np.random.default_rng(1).standard_normal((n0, n1))
    for kind in (0, 1):
        out = np.zeros_like(x)
        tmp = np.zeros_like(x)
        olib.pll_dct2d_fast(kind, n0, n1, p(x), p(out), p(tmp))
        ref = dct_matrix(olib, kind, n0) @ x @ dct_matrix(olib, kind, n1).T
        assert np.allclose(out, ref, rtol=1e-12, atol=1e-11)


def test_thomas_matches_dense(olib):
    rng = np.random.default_rng(3)
    n = 37
    a = rng.uniform(-1, -0.1, n)
    c = rng.uniform(-1, -0.1, n)
    b = 3.0 + rng.uniform(0, 1, n)
    r = rng.standard_normal(n)
    A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
    x = np.linalg.solve(A, r)
    r1 = r.copy()
    olib.orc_thomas_serial(n, p(a), p(b.copy()), p(c.copy()), p(r1))
    assert np.allclose(r1, x, rtol=1e-12)
    r2, b2, c2 = r.copy(), b.copy(), c.copy()
    olib.orc_thomas_pll(n, p(a), p(b2), p(c2), p(r2))
    assert np.array_equal(r1, r2)


def test_weno_exact_on_quadratics(olib):
    # divided differences of a quadratic are linear: WENO5 reproduces the
    # derivative at the upwind-biased point to rounding
    h = 0.1
    xs = np.arange(-6, 7) * h
    q = 0.3 * xs ** 2 - 1.2 * xs + 0.7
    d1 = np.diff(q) / h
    m = 6  # derivative location index
    for sign in (1, -1):
        kk = m - 3 if sign == 1 else m + 2
        val = olib.orc_weno(p(d1), kk, sign)
        # the candidate stencils are consistent; at x_m the exact derivative
        assert abs(val - (0.6 * xs[m] - 1.2)) < 1e-12


def test_manufactured_poisson_source():
    """pllcart3d.c:2029: source -8 pi^2 cos(2 pi y) cos(2 pi z) on a y-z
    periodic-in-cosines box gives phi = cos(2 pi y)cos(2 pi z) / lambda_h
    scaled by the discrete eigenvalue; checked through the restated
    phisolver with the divergence field set to the source."""
    prm = Params().replace(Nx_cell_global=8, Ny_cell_global=16, Nz_cell_global=16)
    o = OracleRun(prm)
    nx, ny, nz = prm.nx, prm.ny, prm.nz
    NX, NY, NZ = prm.shape
    yc = prm.Y1 + (np.arange(NY) - 1 + 0.5) * prm.dy
    zc = prm.Z1 + (np.arange(NZ) - 1 + 0.5) * prm.dz
    mode = np.cos(2 * PI * yc)[:, None] * np.cos(2 * PI * zc)[None, :]
    div = np.zeros(prm.shape)
    div[3:nx + 3, 1:ny + 1, 1:nz + 1] = (-8 * PI * PI * mode[1:ny + 1, 1:nz + 1])[None]
    o.set("div", div)
    dt, g, r = 1.0, 1.0, 0.0   # fac = Re/(dt*alpha) = Re
    o.call("phisolver", dt, g, r)
    phi = o.get("phi")[3:nx + 3, 1:ny + 1, 1:nz + 1]
    lam = (2 * (np.cos(2 * PI * prm.dy) - 1) / prm.dy ** 2
           + 2 * (np.cos(2 * PI * prm.dz) - 1) / prm.dz ** 2)
    expect = prm.Re * (-8 * PI * PI) / lam * mode[1:ny + 1, 1:nz + 1]
    assert np.allclose(phi, expect[None], rtol=1e-10, atol=1e-10)
