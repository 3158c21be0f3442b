"""CPU restatement of the reference's output formats (test infrastructure).

Each function returns the bytes (or text) the reference writes, from numpy
arrays over the padded box (nx+6, ny+2, nz+2) in [i][j][k] order:

* ``snapshot``   write_to_file, pllcart3d.c:3047-3092
* ``middata`` / ``midfield``   midfield, pllcart3d.c:3121-3178
* ``read_midfield``            intermediate, pllcart3d.c:3181-3228
* ``conc_average``             conc_average, pllcart3d.c:3635-3728
* ``wmax_record``              find_wmax, pllcart3d.c:3606-3632
* ``find_max_text``            find_max, pllcart3d.c:3539-3603

Only tests import this module; the GPU library has its own device kernels.
"""

from __future__ import annotations

import numpy as np

MID_FIELDS = ("c_old", "c_hnm1", "u_old", "u_new", "u_hnm1", "u_pg", "v_old", "v_new",
              "v_hnm1", "v_pg", "w_old", "w_new", "w_hnm1", "w_pg")   # L3160-3173


def interior(shape):
    """Index ranges of one rank (simulation_setup, pllcart3d.c:405-431)."""
    nx, ny, nz = shape[0] - 6, shape[1] - 2, shape[2] - 2
    return (3, nx + 2), (1, ny), (1, nz)


def snapshot(u, v, w, c, subsample=None) -> bytes:
    """float32 (u, v, w at cell centres, c) per interior cell in i-j-k order;
    above 2e7 cells only the cells whose padded i, j, k are all even."""
    (i0, i1), (j0, j1), (k0, k1) = interior(c.shape)
    ncell = (i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1)
    if subsample is None:
        subsample = ncell > 2e7
    I = slice(i0, i1 + 1)
    J = slice(j0, j1 + 1)
    K = slice(k0, k1 + 1)
    uc = 0.5 * (u[I, J, K] + u[i0 + 1:i1 + 2, J, K])
    vc = 0.5 * (v[I, J, K] + v[I, j0 + 1:j1 + 2, K])
    wc = 0.5 * (w[I, J, K] + w[I, J, k0 + 1:k1 + 2])
    rec = np.stack([uc, vc, wc, c[I, J, K]], axis=-1).astype(np.float32)
    if subsample:
        ii = np.arange(i0, i1 + 1) % 2 == 0
        jj = np.arange(j0, j1 + 1) % 2 == 0
        kk = np.arange(k0, k1 + 1) % 2 == 0
        rec = rec[ii][:, jj][:, :, kk]
    return rec.tobytes()


def middata(tstep, fileno, tval, outtime, outmid, cavgtime) -> str:
    return "%d\n%d\n%f\n%f\n%f\n%f\n" % (tstep, fileno, tval, outtime, outmid, cavgtime)


def midfield(fields: dict) -> bytes:
    """For every (i, j) of the padded box, the 14 rows of nz_max doubles."""
    stack = np.stack([np.asarray(fields[f], dtype=np.float64) for f in MID_FIELDS], axis=2)
    return np.ascontiguousarray(stack).tobytes()


def read_midfield(data: bytes, shape) -> dict:
    a = np.frombuffer(data, dtype=np.float64).reshape(shape[0], shape[1], len(MID_FIELDS), shape[2])
    return {f: a[:, :, n, :].copy() for n, f in enumerate(MID_FIELDS)}


def _seq_sum(a, axis):
    """Sequential FP64 sum along `axis` in increasing index order."""
    a = np.moveaxis(np.asarray(a, dtype=np.float64), axis, 0)
    s = np.zeros(a.shape[1:])
    for x in a:
        s = s + x
    return s


def conc_average(c, tval):
    """(cavgy, cavgz, cavgyz) record bytes appended by one call."""
    (i0, i1), (j0, j1), (k0, k1) = interior(c.shape)
    ci = c[i0:i1 + 1, j0:j1 + 1, k0:k1 + 1]
    ny, nz = ci.shape[1], ci.shape[2]
    avgy = (_seq_sum(ci, 1) / ny).astype(np.float32)          # [i][k]
    avgz = (_seq_sum(ci, 2) / nz).astype(np.float32)          # [i][j]
    flat = ci.reshape(ci.shape[0], ny * nz)                   # j outer, k inner
    avgyz = (_seq_sum(flat, 1) / (ny * nz)).astype(np.float32)
    return avgy.tobytes(), avgz.tobytes(), np.float32(tval).tobytes() + avgyz.tobytes()


def wmax_record(w, tval) -> bytes:
    (i0, i1), (j0, j1), (k0, k1) = interior(w.shape)
    m = max(0.0, float(np.nanmax(w[i0:i1 + 1, j0:j1 + 1, k0:k1 + 1])))
    return np.array([m, tval], dtype=np.float32).tobytes()


def _last_absmax(a):
    """Signed value and (i, j, k) of the last element, in i-j-k order, whose
    |x| is the largest (fabs(max) <= fabs(x) keeps later ties)."""
    flat = np.abs(a).ravel()
    m = np.nanmax(flat)
    t = int(np.nonzero(flat == m)[0][-1])
    return float(a.ravel()[t]), np.unravel_index(t, a.shape)


def find_max_text(u, v, w, c) -> str:
    parts = []
    for a in (u, v, w, c):
        val, (i, j, k) = _last_absmax(a)
        parts.append("  %2d %2d %2d %f\n" % (i, j, k, val))
    return "max\n" + "".join(parts) + "\n"
