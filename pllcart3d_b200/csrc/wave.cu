// Spanwise wave perturbation of the interface (shift_conc, pllcart3d.c:
// 3231-3277, with spline L3280-3344): every x line of c_old, over the whole
// padded box, is re-sampled at x - meshdx(z) by a natural cubic spline whose
// second derivatives solve the (1, 4, 1) system of pll_tridiag's one-rank
// arithmetic.  One thread per (j, k) line, consecutive threads on
// consecutive k (coalesced); the line's eliminated coefficients and the
// spline values go to FP64 scratch laid out [position][line].  The interval
// of each sample point is found directly (uniform mesh) and checked with
// the reference's comparisons, keeping its rule that the last interval
// [x_i, x_{i+1}] containing the point wins and its end-point overrides.
#include <cuda_runtime.h>

#include <cmath>

#include "../../include/pllcart3d_gpu.h"
#include "forms.h"
#include "host_common.cuh"

using namespace pll;

namespace pll {
namespace {

struct WaveArgs {
    double xstart, zstart, dx, dz;   // mesh_generation, pllcart3d.c:442-454
    double ampli, lamb, pi;
    int subharm;
};

// mesh x of padded index i (grid->Xc, L444)
__device__ __forceinline__ double xc(const WaveArgs& W, int i) { return W.xstart + i * W.dx; }

template <typename real>
__global__ void k_shift_conc(Geo G, WaveArgs W, real* __restrict__ c, double* __restrict__ cp,
                             double* __restrict__ rp, double* __restrict__ yy)
{
    const int nl = G.NY * G.NZ;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nl) return;
    const int j = t / G.NZ, k = t % G.NZ;
    const long base = (long)j * G.sy + k;
    const int N = G.NX, n = N - 2;
    const double delta = W.dx;
    auto y = [&](int i) { return (double)c[base + (long)i * G.sx]; };

    // mesh translation of this z (L3246-3252)
    const double beta = 2 * W.pi / W.lamb;
    const double zc = W.zstart + k * W.dz;
    double meshdx;
    if (W.subharm == 0)
        meshdx = W.ampli * cos(beta * zc);
    else
        meshdx = W.ampli * cos(beta * (zc + W.lamb / 2)) + W.ampli * cos(beta / 2 * (zc + W.lamb / 2));

    // second derivatives: a = c = 1, b = 4, r = 6/d/d (y[i+1] - 2 y[i] + y[i-1])
    // for i = 1 .. N-2 (L3295-3301), pll_tridiag's one-rank recurrences
    double cprev = 0, rprev = 0;
    for (int m = 0; m < n; ++m) {
        const int i = m + 1;
        const double la = 1.0, lc = 1.0;
        double lb = 4.0;
        const double lr = 6.0 / delta / delta * (y(i + 1) - 2.0 * y(i) + y(i - 1));
        double cm, rm;
        if (m == 0) {
            lb = lb - 0.0 * la;
            cm = lc / lb;
            rm = (lr - 0.0 * la) / lb;
        } else {
            lb = (lb - cprev * la);
            cm = lc / lb;
            rm = (lr - rprev * la) / lb;
        }
        cp[(long)m * nl + t] = cm;
        rp[(long)m * nl + t] = rm;
        cprev = cm;
        rprev = rm;
    }
    // fpp[i] = solution[i-1] for i in 1..N-2, kept in rp; fpp[0] = fpp[N-1] = 0
    double xnext = rprev - cprev * 0.0;
    rp[(long)(n - 1) * nl + t] = xnext;
    for (int m = n - 2; m >= 0; --m) {
        const double x = rp[(long)m * nl + t] - cp[(long)m * nl + t] * xnext;
        rp[(long)m * nl + t] = x;
        xnext = x;
    }
    auto fpp = [&](int i) { return (i <= 0 || i >= N - 1) ? 0.0 : rp[(long)(i - 1) * nl + t]; };

    // evaluation (L3320-3341), into yy
    const double xlast = xc(W, N - 1), x1 = xc(W, 1);
    for (int ii = 0; ii < N; ++ii) {
        const double xx = xc(W, ii) - meshdx;
        double v = 0.0;
        bool have = false;
        // the last i in [0, N-2] with x[i] <= xx <= x[i+1]
        int i0 = (int)floor((xx - W.xstart) / W.dx);
        i0 = i0 < 0 ? 0 : (i0 > N - 2 ? N - 2 : i0);
        while (i0 < N - 2 && xc(W, i0 + 1) <= xx) ++i0;
        while (i0 > 0 && xc(W, i0) > xx) --i0;
        if (xc(W, i0) <= xx && xx <= xc(W, i0 + 1)) {
            const int i = i0;
            const double xi = xc(W, i), xi1 = xc(W, i + 1);
            const double fi = fpp(i), fi1 = fpp(i + 1);
            v = fi * (xi1 - xx) * (xi1 - xx) * (xi1 - xx) / (6 * delta) +
                fi1 * (xx - xi) * (xx - xi) * (xx - xi) / (6 * delta) + (y(i) / delta - delta / 6 * fi) * (xi1 - xx) +
                (y(i + 1) / delta - delta / 6 * fi1) * (xx - xi);
            have = true;
        }
        if (xx > xlast) {
            v = y(N - 1);
            have = true;
        } else if (xx < x1) {
            v = y(0);
            have = true;
        }
        // every point lies in [x0, x_{N-1}] or beyond an end: `have` holds
        yy[(long)ii * nl + t] = have ? v : y(ii);
    }
    for (int ii = 0; ii < N; ++ii) c[base + (long)ii * G.sx] = (real)yy[(long)ii * nl + t];
}

}  // namespace
}  // namespace pll

extern "C" int pllgpu_shift_conc(pllgpu_ctx* ctx, double ampli, double lamb, int subharm)
{
    if (!ctx || lamb == 0.0 || (subharm != 0 && subharm != 1)) return PLLGPU_EINVAL;
    CK(cudaSetDevice(ctx->dev));
    // the reference's c->new == c->old here (update_old_conc); make the
    // ping-pong buffers hold that before c_old alone is shifted
    if (int e = materialize(ctx)) return e;
    void* c = field_ptr(ctx, PLLGPU_C_OLD, true);
    if (!c) return fail(ctx, PLLGPU_ECUDA);
    const Geo& G = ctx->G;
    WaveArgs W;
    W.dx = G.dx;
    W.dz = G.dz;
    W.xstart = ctx->P.X1 + (0 - ctx->Rg.is) * G.dx + (G.dx / 2.0);
    W.zstart = ctx->P.Z1 - ctx->Rg.ks * G.dz + (G.dz / 2.0);
    W.ampli = ampli;
    W.lamb = lamb;
    W.pi = 4.0 * std::atan(1.0);   // pllcart3d.c:397
    W.subharm = subharm;
    const long nl = (long)G.NY * G.NZ;
    double* scratch = nullptr;
    CK(cudaMallocAsync((void**)&scratch, sizeof(double) * 3 * nl * G.NX, ctx->st));
    const unsigned blocks = (unsigned)((nl + 127) / 128);
    if (ctx->mixed)
        k_shift_conc<float><<<blocks, 128, 0, ctx->st>>>(G, W, (float*)c, scratch, scratch + nl * G.NX,
                                                         scratch + 2 * nl * G.NX);
    else
        k_shift_conc<double><<<blocks, 128, 0, ctx->st>>>(G, W, (double*)c, scratch, scratch + nl * G.NX,
                                                          scratch + 2 * nl * G.NX);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(scratch, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    // c_new keeps the unshifted field, as the reference's c->new does; the
    // next substep's update_old_conc brings its never-written entries into
    // c_old (the same one-time copy as after a restart)
    ctx->resync_c = true;
    return PLLGPU_OK;
}
