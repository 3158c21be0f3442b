// The surrogate's 3x3x3 / 1x1x1 convolution on the 5th-generation tensor
// cores: an implicit GEMM (rows = 128 voxels, columns = BN output channels,
// K = taps x input channels) issued with tcgen05.mma.kind::f16 (BF16
// operands, FP32 accumulator in tensor memory), operands staged in shared
// memory by TMA.
//
// The A tile of one (tap, channel chunk) is a single 5-d tiled TMA load of
// the channels-last activations [n][d][h][w][c]: box (CK channels, the whole
// W row, hb rows of h, db slices of d) at the coordinates of the tile's
// voxels shifted by the tap's offset.  TMA fills the box elements that fall
// outside the volume with zeros, which is exactly the convolution's zero
// padding, so no gather or boundary code runs on the SMs.  The swizzle of
// the box rows (CK * 2 bytes: 128, 64 or 32) is the K-major layout tcgen05
// reads.  The B tile (BN output channels x CK input channels of one tap) is
// a 3-d TMA load of the weights [cout][tap][cin].  No multicast.
//
// CTA: 128 voxels x BN channels; four pipeline stages.
//   warp 0      TMA producer (one thread)
//   warp 1      TMEM owner and MMA issuer (one thread)
//   warps 2..5  epilogue: TMEM lanes 32*(warp%4) .. +31 = tile rows; bias,
//               leaky ReLU, FP32 pre-activation and BF16 activation stores
// Every mbarrier wait is bounded (about one second of SM clock); a wait that
// runs out raises the kernel's abort flag and the library's status word,
// the other roles stop at their next wait, the producer drains its copies
// and the tensor memory is freed before the CTA returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int CU_BM = 128;
constexpr int CU_STAGES = 4;
constexpr int CU_THREADS = 192;
constexpr long long CU_WAIT_CYCLES = 2000000000LL;

__device__ int g_nn_status;   // bit 8: a bounded wait of a tcgen05 convolution ran out

template <int BN, int CK>
struct CuSmem {
    static constexpr uint32_t A_BYTES = CU_BM * CK * 2;
    static constexpr uint32_t B_BYTES = BN * CK * 2;
    static constexpr uint32_t STAGE = ((A_BYTES + B_BYTES) + 1023) / 1024 * 1024;
    static constexpr uint32_t BAR_OFF = CU_STAGES * STAGE;
    static constexpr uint32_t TOTAL = BAR_OFF + 128;
    static constexpr uint32_t DYN = TOTAL + 1024;   // slack for 1024-byte alignment
    static constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
};

// shared-memory matrix descriptor (sm_100, version 1), K-major rows of CK
// BF16 with the swizzle of their width; 8-row groups SBO bytes apart
template <int CK>
__device__ __forceinline__ uint64_t cu_desc(uint32_t saddr)
{
    constexpr uint64_t layout = CK == 64 ? 2 : CK == 32 ? 4 : 6;   // SWIZZLE_128B / 64B / 32B
    constexpr uint64_t sbo = 8 * CK * 2;
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (sbo >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= layout << 61;
    return d;
}

// instruction descriptor, kind::f16: D = F32, A = B = BF16, both K-major,
// M = 128, N = BN
template <int BN>
__device__ __forceinline__ uint32_t cu_idesc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(CU_BM >> 4) << 24);
}

__device__ __forceinline__ uint32_t cu_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cu_bar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(cu_smem(b)), "r"(count) : "memory");
}

__device__ __forceinline__ bool cu_try_wait(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(cu_smem(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __noinline__ bool cu_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, bool honor_abort)
{
    if (cu_try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (true) {
        if (cu_try_wait(b, parity)) return true;
        if (honor_abort && *abort_flag) return false;
        if (clock64() - t0 > CU_WAIT_CYCLES) {
            *abort_flag = 1;
            return false;
        }
    }
}

__device__ __forceinline__ void cu_tma_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c, int w, int h, int d,
                                          int n)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
        "%6, %7}], [%2];\n" ::"r"(cu_smem(dst)),
        "l"((uint64_t)map), "r"(cu_smem(bar)), "r"(c), "r"(w), "r"(h), "r"(d), "r"(n)
        : "memory");
}

__device__ __forceinline__ void cu_tma_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];\n" ::"r"(cu_smem(dst)),
        "l"((uint64_t)map), "r"(cu_smem(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void cu_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::
            "r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void cu_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(cu_smem(bar))
                 : "memory");
}

__device__ __forceinline__ void cu_ld16(uint32_t taddr, uint32_t* r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// the voxel box of one tile: 128 voxels = W x hb x db (every tile starts a
// whole w row; hb rows of h; db slices of d)
struct CuGeom {
    int N, D, H, W;
    int hb, db;
    int Cin, Cout, ksize;
};

template <int BN, int CK>
__global__ void __launch_bounds__(CU_THREADS, 1)
    k_conv_umma(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW, CuGeom g,
                const float* __restrict__ bias, float* __restrict__ Y32, __nv_bfloat16* __restrict__ Y16, int act,
                float slope)
{
    using L = CuSmem<BN, CK>;
    extern __shared__ uint8_t cu_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)cu_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(sm + L::BAR_OFF);
    uint64_t* full = bars;
    uint64_t* empty = bars + CU_STAGES;
    uint64_t* done = bars + 2 * CU_STAGES;
    volatile uint32_t* tmem_slot = (volatile uint32_t*)(bars + 2 * CU_STAGES + 1);
    volatile int* abort_flag = (volatile int*)(bars + 2 * CU_STAGES + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long m0 = (long)blockIdx.x * CU_BM;
    const int n0 = blockIdx.y * BN;
    // the tile's first voxel (whole w rows): row index r0 = (n D + d) H + h
    const long r0 = m0 / g.W;
    const int h0 = (int)(r0 % g.H), d0 = (int)((r0 / g.H) % g.D), nn = (int)(r0 / ((long)g.H * g.D));
    const int ntaps = g.ksize * g.ksize * g.ksize;
    const int nch = g.Cin / CK;
    const int nk = ntaps * nch;

    if (threadIdx.x == 0) {
        for (int s = 0; s < CU_STAGES; ++s) {
            cu_bar_init(&full[s], 1);
            cu_bar_init(&empty[s], 1);
        }
        cu_bar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         cu_smem((const void*)tmem_slot)),
                     "r"(L::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int last[CU_STAGES];
#pragma unroll
            for (int s = 0; s < CU_STAGES; ++s) last[s] = -1;
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % CU_STAGES;
                if (kc >= CU_STAGES && !cu_wait(&empty[s], (kc / CU_STAGES + 1) & 1, abort_flag, true)) break;
                const int tap = kc / nch, c0 = (kc - tap * nch) * CK;
                int dz = 0, dy = 0, dx = 0;
                if (g.ksize == 3) {
                    dz = tap / 9 - 1;
                    dy = (tap / 3) % 3 - 1;
                    dx = tap % 3 - 1;
                }
                uint8_t* st = sm + s * L::STAGE;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(cu_smem(&full[s])),
                             "r"(L::A_BYTES + L::B_BYTES)
                             : "memory");
                cu_tma_5d(st, &tmX, &full[s], c0, dx, h0 + dy, d0 + dz, nn);
                cu_tma_3d(st + L::A_BYTES, &tmW, &full[s], c0, tap, n0);
                last[s] = kc;
            }
            // drain: no copy may still be landing when the CTA leaves
            for (int s = 0; s < CU_STAGES; ++s)
                if (last[s] >= 0) cu_wait(&full[s], (last[s] / CU_STAGES) & 1, abort_flag, false);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = cu_idesc<BN>();
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % CU_STAGES;
                if (!cu_wait(&full[s], (kc / CU_STAGES) & 1, abort_flag, true)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t st = cu_smem(sm + s * L::STAGE);
                const uint64_t da = cu_desc<CK>(st), db = cu_desc<CK>(st + L::A_BYTES);
#pragma unroll
                for (int kk = 0; kk < CK / 16; ++kk) {
                    // K step of 16 BF16 = 32 bytes inside the swizzle row
                    const uint64_t o = (uint64_t)(kk * 32) >> 4;
                    cu_mma(tmem, da + o, db + o, idesc, (kc | kk) ? 1u : 0u);
                }
                cu_commit(&empty[s]);
            }
            cu_commit(done);   // tracks every MMA issued above, also after an abort
        }
        __syncwarp();
    } else {
        const bool ok = cu_wait(done, 0, abort_flag, false) && !*abort_flag;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int q = warp & 3;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
        const long row = m0 + 32 * q + lane;
        if (ok) {
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 16) {
                uint32_t v[16];
                cu_ld16(trow + c0, v);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                float y[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) y[j] = __uint_as_float(v[j]) + (bias ? bias[n0 + c0 + j] : 0.f);
                const long o = row * g.Cout + n0 + c0;
                if (Y32) {
#pragma unroll
                    for (int j = 0; j < 16; j += 4) *(float4*)(Y32 + o + j) = make_float4(y[j], y[j + 1], y[j + 2], y[j + 3]);
                }
                if (Y16) {
                    __align__(16) __nv_bfloat16 b[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const float a = act ? (y[j] > 0.f ? y[j] : slope * y[j]) : y[j];
                        b[j] = __float2bfloat16(a);
                    }
                    *(uint4*)(Y16 + o) = *(const uint4*)&b[0];
                    *(uint4*)(Y16 + o + 8) = *(const uint4*)&b[8];
                }
            }
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(L::TMEM_COLS));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicOr(&g_nn_status, 0x100);
}

}  // namespace
