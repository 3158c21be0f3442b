// Shared device-side types for the pllcart3d B200 step.
//
// Device layout: every field is one array over the padded box
// (nx+6) x (ny+2) x (nz+2) in the reference's [i][j][k] order with k
// contiguous (allocate_3d_calloc.h:46-64), but contiguous in HBM with a row
// pitch `sy` >= nz+2 (a multiple of 8 elements) and a plane pitch
// `sx` = (ny+2)*sy.  Index ranges follow grid_setup / simulation_setup for
// one rank (pllcart3d.c:357-431): interior i in [3, nx+2], j in [1, ny],
// k in [1, nz]; the u unknowns start at i=4, v at j=2, w at k=2.
#pragma once

#include <cstdint>

namespace pll {

struct Geo {
    int nx, ny, nz;   // interior cells
    int NX, NY, NZ;   // padded logical extents
    long sx, sy;      // element strides of i and j (k stride is 1)
    double dx, dy, dz;
};

struct Rng {
    int is, ie, js, je, ks, ke;
};

struct Phys {
    double Re, Pe, M, Vnorm, Fx, Fy, CFLmax;
    double Y1, Y2, Z1, Z2;
    double Mum, PI;
    int nmvp;
};

enum Var { VC = 0, VU = 1, VV = 2, VW = 3 };

// device scalar slots (one small array per context)
enum Scal {
    S_DT = 0,        // time step of the current step
    S_VBULK = 1,     // outflow convective speed of the current substep
    S_DEFICIT = 2,   // inflow - outflow mass-flux deficit per unit area
    S_CFLMAX = 3,    // max over cells of |u|/dx+|v|/dy+|w|/dz (as bits)
    S_TIMESTEP = 4,  // Timestep after the diffusive cap
    S_CM = 5,        // slope parameter of the non-monotonic viscosity law
    S_QIN = 6,
    S_QOUT = 7,
    // 8..11: non-monotonic viscosity coefficients (aux_kernels.cuh)
    S_TVAL = 12,     // simulated time
    S_CFLDT = 13,    // CFLmax / max, find_cfl's return value
    S_COUNT = 16
};

// sticky status bits
enum StatusBits {
    ST_NAN = 1,       // a NaN/Inf met in the CFL scan
    ST_NOCONV = 2,    // slope-parameter bisection did not converge
    ST_BOUNDS = 4,    // a kernel's self-check found a bad index
    ST_TIMEOUT = 8,   // a bounded device wait ran out
};

// ---------------------------------------------------------------------------
// constants shared by the stencil kernels (host-precomputed, exact as in the
// reference: each is the same IEEE expression the reference evaluates)
// ---------------------------------------------------------------------------
struct Consts {
    double hx, hy, hz;            // dx, dy, dz
    double ihx, ihy, ihz;         // 1/dx ... (used only when pow2)
    double i2hx, i2hy, i2hz;      // 1/(2 dx) ... (used only when pow2)
    int pow2;                     // all spacings are exact powers of two
    double cdx, cdy, cdz;         // 1/(Pe h^2), A_conc (pllcart3d.c:1421-1433)
    double d1x, d1y, d1z;         // 1/(Re h)
    double d2x, d2y, d2z;         // 2/(Re h)
    double xuv, xuw;              // 1/(Re dy dx), 1/(Re dz dx)  (Hu_op)
    double xvu, xvw;              // 1/(Re dx dy), 1/(Re dz dy)  (Hv_op)
    double xwu, xwv;              // 1/(Re dx dz), 1/(Re dy dz)  (Hw_op)
    double FxRe, FyRe;            // -(Fx/Re), -(Fy/Re)
    double Re;
    double area;                  // (Y2-Y1)*(Z2-Z1)
    double dx2i;                  // 1/(dx*dx) (phisolver_dct)
    double CFLmax;
    double M, Vnorm;
};

// the four viscosity arrays of one time level (cell centres and edges)
template <typename real>
struct MuPtrs {
    const real* cell;
    const real* xy;
    const real* xz;
    const real* yz;
};

// launch-shape variants the autotuner chooses among; every variant computes
// each cell (explicit operators) or line (line solves) with the same
// arithmetic, so the choice changes timing only, never a bit of the result
// Scratch of the multi-block reductions: the flux row sums of both x
// planes (2 NY) and the bulk-velocity block partials (value and index,
// BULK_BLOCKS each).
constexpr int BULK_BLOCKS = 128;
inline long red_doubles(const Geo& G) { return 2L * G.NY + 2L * BULK_BLOCKS; }

constexpr int NTUNE_EXP = 4, NTUNE_LINE = 3;
inline void tune_exp_block(int v, int& bx, int& by)
{
    static const int t[NTUNE_EXP][2] = {{32, 4}, {64, 2}, {128, 1}, {32, 2}};
    bx = t[v][0];
    by = t[v][1];
}
inline int tune_line_block(int v)
{
    static const int t[NTUNE_LINE] = {32, 64, 128};
    return t[v];
}

}  // namespace pll
