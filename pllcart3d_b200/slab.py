"""x-slab decomposition of the step across ranks: the pieces each rank of a
multi-GPU run needs, over torch.distributed (NCCL between GPUs, gloo on
CPU).

The reference splits x into slabs, one per MPI rank (grid_setup,
pllcart3d.c:357-378), exchanges 3 ghost planes with each neighbour after
every stage that changes a field (e.g. exchange_conc_boundary,
pllcart3d.c:2230-2300), solves every x-tridiagonal system with a Thomas
sweep pipelined over the ranks one line at a time (pll_tridiag.c:49-149, one
2-double message per line per rank boundary), and reduces the CFL maximum
with MPI_Allreduce (L3113).  Here:

* ``slab_ranges``      - the reference's slab sizes and offsets;
* ``halo_exchange``    - the ghost planes from the neighbours' edge planes
                         (point-to-point, both directions at once);
* ``reduce_scalars``   - the step's scalars in one MAX all-reduce: the CFL
                         maximum, and values only one rank computes (the
                         inflow flux on the first slab, the outflow flux and
                         the outflow speed on the last) travelling as the
                         only finite entry;
* ``partitioned_tridiag`` - every x system at once by the partition method:
                         each rank eliminates its block's interior rows in
                         terms of its first row and the next block's first
                         row, the ranks exchange one small separator
                         equation per line (an all-gather), every rank
                         solves the P-row separator system and finishes its
                         own rows.  One collective per sweep instead of
                         pll_tridiag's 2 messages per line per boundary.

The same elimination runs inside one GPU in the precision form's segmented
line solve (``k_line_seg``).  Nothing in this module is wired into the GPU
step: every GPU run available to this project has one device.
"""

from __future__ import annotations

import math

import torch
import torch.distributed as dist


def slab_ranges(nx: int, size: int):
    """(offset, cells) of each rank's slab: rank r gets
    (nx + size - r - 1) // size cells after the cells of ranks 0..r-1
    (grid_setup, pllcart3d.c:357, 376-379)."""
    out, off = [], 0
    for r in range(size):
        n = (nx + size - r - 1) // size
        out.append((off, n))
        off += n
    return out


def halo_exchange(f: torch.Tensor, width: int = 3, group=None) -> None:
    """Fill the `width` ghost planes at each x end of this rank's padded
    slab f[(width + n + width), ...] from the neighbours' edge planes; the
    outer ghosts of the first and last ranks are left alone (their
    boundary closures own them)."""
    rank, size = dist.get_rank(group), dist.get_world_size(group)
    n = f.shape[0] - 2 * width
    if n < width:
        raise ValueError("a slab needs at least as many planes as the halo is wide")
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, f[width:2 * width].contiguous(), rank - 1, group))
        left = torch.empty_like(f[:width])
        ops.append(dist.P2POp(dist.irecv, left, rank - 1, group))
    if rank < size - 1:
        ops.append(dist.P2POp(dist.isend, f[n:n + width].contiguous(), rank + 1, group))
        right = torch.empty_like(f[:width])
        ops.append(dist.P2POp(dist.irecv, right, rank + 1, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    if rank > 0:
        f[:width].copy_(left)
    if rank < size - 1:
        f[n + width:].copy_(right)


def reduce_scalars(cfl_local: float, qin=None, qout=None, vbulk=None, group=None, device="cpu"):
    """One MAX all-reduce for the step's scalars: the CFL maximum over all
    ranks, and the inflow flux (first rank), outflow flux and outflow speed
    (last rank), which travel as the only finite entry of their slot."""
    neg = -math.inf
    t = torch.tensor([cfl_local, neg if qin is None else qin, neg if qout is None else qout,
                      neg if vbulk is None else vbulk], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return tuple(float(x) for x in t)


def partitioned_tridiag(a: torch.Tensor, b: torch.Tensor, c: torch.Tensor, r: torch.Tensor, group=None):
    """Solve N tridiagonal systems a_i x_{i-1} + b_i x_i + c_i x_{i+1} = r_i
    whose rows are split over the ranks in order: this rank holds rows
    [lines, m] (m >= 1) of every system; a of the global first row and c of
    the global last row are ignored.  Returns this rank's x [lines, m].
    Diagonally dominant systems (the ADI operators); FP64 throughout."""
    rank, size = dist.get_rank(group), dist.get_world_size(group)
    N, m = r.shape
    a = a.clone()
    c = c.clone()
    if rank == 0:
        a[:, 0] = 0
    if rank == size - 1:
        c[:, -1] = 0
    zero = torch.zeros(N, dtype=r.dtype, device=r.device)
    # interior rows 1..m-1 in terms of S (this block's row 0) and T (the next
    # block's row 0): x_e = g_e - v_e S - w_e T
    g = torch.zeros((N, m), dtype=r.dtype, device=r.device)
    v = torch.zeros_like(g)
    w = torch.zeros_like(g)
    if m > 1:
        # top-down: x_e = rh_e - ah_e S - ch_e x_{e+1}
        rh = torch.zeros_like(g)
        ah = torch.zeros_like(g)
        ch = torch.zeros_like(g)
        d = b[:, 1]
        rh[:, 1], ah[:, 1], ch[:, 1] = r[:, 1] / d, a[:, 1] / d, c[:, 1] / d
        for e in range(2, m):
            d = b[:, e] - a[:, e] * ch[:, e - 1]
            rh[:, e] = (r[:, e] - a[:, e] * rh[:, e - 1]) / d
            ah[:, e] = -a[:, e] * ah[:, e - 1] / d
            ch[:, e] = c[:, e] / d
        # bottom-up: substitute x_{e+1}
        g[:, m - 1], v[:, m - 1], w[:, m - 1] = rh[:, m - 1], ah[:, m - 1], ch[:, m - 1]
        for e in range(m - 2, 0, -1):
            g[:, e] = rh[:, e] - ch[:, e] * g[:, e + 1]
            v[:, e] = ah[:, e] - ch[:, e] * v[:, e + 1]
            w[:, e] = -ch[:, e] * w[:, e + 1]
        last = (g[:, m - 1], v[:, m - 1], w[:, m - 1])
        first = (g[:, 1], v[:, 1], w[:, 1])
    else:
        # a one-row block: its last row is row 0 itself (x = S), and row 0's
        # right neighbour is T directly
        last = (zero, -torch.ones_like(zero), zero)
        first = None
    # the separator equation of this block needs the previous block's last
    # row; every rank gathers every block's pieces
    mine = torch.stack([last[0], last[1], last[2], a[:, 0], b[:, 0], c[:, 0], r[:, 0],
                        first[0] if first is not None else zero, first[1] if first is not None else zero,
                        first[2] if first is not None else zero,
                        torch.full_like(zero, 1.0 if first is not None else 0.0)])
    allp = [torch.empty_like(mine) for _ in range(size)]
    dist.all_gather(allp, mine, group=group)
    # separator system: al_l S_{l-1} + be_l S_l + ga_l S_{l+1} = rho_l
    al, be, ga, rho = [], [], [], []
    for l in range(size):
        p = allp[l]
        a0, b0, c0, r0 = p[3], p[4], p[5], p[6]
        if l > 0:
            gp, vp, wp = allp[l - 1][0], allp[l - 1][1], allp[l - 1][2]
        else:
            gp = vp = wp = torch.zeros_like(a0)
        interior = p[10] > 0
        g1 = torch.where(interior, p[7], torch.zeros_like(a0))
        v1 = torch.where(interior, p[8], torch.zeros_like(a0))
        w1 = torch.where(interior, p[9], torch.zeros_like(a0))
        # x_1 = g1 - v1 S - w1 T, or T itself for a one-row block
        al.append(-a0 * vp)
        be.append(b0 - a0 * wp - c0 * v1)
        ga.append(torch.where(interior, -c0 * w1, c0))
        rho.append(r0 - a0 * gp - c0 * g1)
    # Thomas over the P separators of every line
    cp = [None] * size
    rp = [None] * size
    cp[0] = ga[0] / be[0]
    rp[0] = rho[0] / be[0]
    for l in range(1, size):
        d = be[l] - al[l] * cp[l - 1]
        cp[l] = ga[l] / d
        rp[l] = (rho[l] - al[l] * rp[l - 1]) / d
    S = [None] * size
    S[size - 1] = rp[size - 1]
    for l in range(size - 2, -1, -1):
        S[l] = rp[l] - cp[l] * S[l + 1]
    Sl = S[rank]
    Tl = S[rank + 1] if rank + 1 < size else torch.zeros_like(Sl)
    x = g - v * Sl[:, None] - w * Tl[:, None]
    x[:, 0] = Sl
    return x
