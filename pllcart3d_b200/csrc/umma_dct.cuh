// The DCT passes of the precision form on the 5th-generation tensor cores:
// split-TF32 (3-term compensated) GEMMs issued with tcgen05.mma, operands
// staged in shared memory by TMA (cp.async.bulk.tensor, 64-byte swizzle),
// the FP32 accumulator in tensor memory and read back with tcgen05.ld.
//
// Every pass of the 2-d DCT-II / DCT-III over an x-plane (fftw_3d.h:45-106
// as called by phisolver_dct pllcart3d.c:2035, 2104) is one GEMM over all
// planes at once, contracting the array's contiguous axis:
//
//     C[r][n] = sum_k A[r][k] * T[n][k]        r = (plane, row), k contiguous
//
// with T the dense cosine matrix of that pass (FFTW's documented REDFT10 /
// REDFT01 definitions).  The epilogue writes C either row-major (the next
// consumer contracts n) or transposed within the plane (the next pass
// contracts the other axis, which then becomes contiguous), so every pass
// reads a K-major operand and no transpose kernel runs.
//
// Split-TF32: x = hi + lo with hi = rna_tf32(x), lo = rna_tf32(x - hi); the
// product is lo*Thi + hi*Tlo + hi*Thi accumulated in FP32 (the lo*lo term,
// 2^-22 relative, is dropped).  T's halves are split once on the host; the
// data tile is split in shared memory by the converter warps after TMA
// lands it (in place for hi, beside it for lo; the swizzle is a permutation
// of positions, so elementwise conversion preserves it).
//
// CTA: 128 rows x BN columns (BN = the whole transform length, 128 or 256),
// K in chunks of 16 (one 64-byte swizzle row), four pipeline stages.
//   warp 0      TMA producer (one thread)
//   warp 1      TMEM owner and MMA issuer (one thread)
//   warps 2..5  converters, then the epilogue (TMEM lanes 32*(warp%4)...)
// Every mbarrier wait is bounded (about one second of SM clock); a wait that
// runs out sets ST_TIMEOUT in the context's status word, the other roles
// stop at their next wait, and the CTA still drains its copies and MMAs in
// flight (bounded as well) and frees its tensor memory before returning.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace pll {
namespace {

constexpr int UM_BM = 128;       // rows per CTA (tcgen05 M)
constexpr int UM_BK = 16;        // K chunk: 16 fp32 = one 64-byte swizzle row
constexpr int UM_STAGES = 4;
constexpr int UM_THREADS = 192;
constexpr long long UM_WAIT_CYCLES = 2000000000LL;   // ~1 s at 1.9 GHz

struct UmmaEpi {
    long rows_per_plane;   // P: output row r maps to (r / P, r % P)
    long ob, oq, on;       // element strides of plane, row-in-plane, column
    float scale;
    int scale_mode;        // 0 none, 1 multiply, 2 divide
    int transposed;        // oq == 1: columns are strided, rows contiguous
};

template <int BN>
struct UmmaSmem {
    static constexpr uint32_t A_BYTES = UM_BM * UM_BK * 4;
    static constexpr uint32_t B_BYTES = BN * UM_BK * 4;
    static constexpr uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr uint32_t BAR_OFF = UM_STAGES * STAGE;
    // full[2], conv[2], empty[2], done, then the TMEM address and abort flag
    static constexpr uint32_t TOTAL = BAR_OFF + 256;
    static constexpr uint32_t DYN = TOTAL + 1024;   // slack for 1024-byte alignment
};

__device__ __forceinline__ uint32_t um_smem(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void um_bar_init(uint64_t* b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(um_smem(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void um_arrive_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(um_smem(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void um_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(um_smem(b)) : "memory");
}

__device__ __forceinline__ bool um_try_wait(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(um_smem(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity`.  With honor_abort, returns
// false at once when another role has given up; a wait that runs out of
// time raises the abort flag.
__device__ __noinline__ bool um_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag, bool honor_abort)
{
    if (um_try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (true) {
        if (um_try_wait(b, parity)) return true;
        if (honor_abort && *abort_flag) return false;
        if (clock64() - t0 > UM_WAIT_CYCLES) {
            *abort_flag = 1;
            return false;
        }
    }
}

__device__ __forceinline__ void um_tma_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];\n" ::"r"(um_smem(dst)),
        "l"((uint64_t)map), "r"(um_smem(bar)), "r"(x), "r"(y)
        : "memory");
}

// shared-memory matrix descriptor: K-major, 64-byte swizzle, rows of 64 B
// packed (8-row groups 512 B apart), descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t um_desc_sw64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);   // start address, bits 0-13
    d |= (uint64_t)1 << 16;                      // leading byte offset (unused here)
    d |= (uint64_t)(512 >> 4) << 32;             // stride byte offset, bits 32-45
    d |= (uint64_t)1 << 46;                      // version
    d |= (uint64_t)4 << 61;                      // SWIZZLE_64B
    return d;
}

// instruction descriptor, kind::tf32: D = F32, A = B = TF32, both K-major
template <int BN>
__device__ __forceinline__ uint32_t um_idesc_tf32()
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(UM_BM >> 4) << 24);
}

__device__ __forceinline__ void um_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::
            "r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void um_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     um_smem(bar))
                 : "memory");
}

__device__ __forceinline__ void um_ld16(uint32_t taddr, uint32_t* r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Row-major epilogue: element offset of (row 32 q, column lane) of the tile
// starting at output row m0.  A plane holds 128 or 256 rows (a multiple of
// the 128-row tile), so all rows of a tile lie in one plane and their offsets
// are this origin plus rr * oq + column * on.
__device__ __forceinline__ long tile_origin(const UmmaEpi& e, long m0, int q, int lane)
{
    const long plane = m0 / e.rows_per_plane, prow = m0 % e.rows_per_plane + 32 * q;
    return plane * e.ob + prow * e.oq + (long)lane * e.on;
}

__device__ __forceinline__ float um_rna_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

template <int BN>
__global__ void __launch_bounds__(UM_THREADS, 1)
    k_dct_umma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmBh,
               const __grid_constant__ CUtensorMap tmBl, int K, UmmaEpi e, float* __restrict__ out,
               int* __restrict__ status)
{
    using L = UmmaSmem<BN>;
    extern __shared__ uint8_t um_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)um_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(sm + L::BAR_OFF);
    uint64_t* full = bars;                    // TMA landed (A fp32, T hi, T lo)
    uint64_t* conv = bars + UM_STAGES;        // A split into hi / lo
    uint64_t* empty = bars + 2 * UM_STAGES;   // MMAs of the stage retired
    uint64_t* done = bars + 3 * UM_STAGES;    // accumulator complete
    volatile uint32_t* tmem_slot = (volatile uint32_t*)(bars + 3 * UM_STAGES + 1);
    volatile int* abort_flag = (volatile int*)(bars + 3 * UM_STAGES + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * UM_BM;
    const int nk = K / UM_BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < UM_STAGES; ++s) {
            um_bar_init(&full[s], 1);
            um_bar_init(&conv[s], 128);
            um_bar_init(&empty[s], 1);
        }
        um_bar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         um_smem((const void*)tmem_slot)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int last[UM_STAGES];
#pragma unroll
            for (int s = 0; s < UM_STAGES; ++s) last[s] = -1;
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % UM_STAGES;
                if (kc >= UM_STAGES && !um_wait(&empty[s], (kc / UM_STAGES + 1) & 1, abort_flag, true)) break;
                uint8_t* st = sm + s * L::STAGE;
                um_arrive_tx(&full[s], L::A_BYTES + 2 * L::B_BYTES);
                um_tma_2d(st, &tmA, &full[s], kc * UM_BK, m0);
                um_tma_2d(st + 2 * L::A_BYTES, &tmBh, &full[s], kc * UM_BK, 0);
                um_tma_2d(st + 2 * L::A_BYTES + L::B_BYTES, &tmBl, &full[s], kc * UM_BK, 0);
                last[s] = kc;
            }
            // drain: no copy may still be landing when the CTA leaves
            for (int s = 0; s < UM_STAGES; ++s)
                if (last[s] >= 0) um_wait(&full[s], (last[s] / UM_STAGES) & 1, abort_flag, false);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = um_idesc_tf32<BN>();
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % UM_STAGES;
                if (!um_wait(&conv[s], (kc / UM_STAGES) & 1, abort_flag, true)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t st = um_smem(sm + s * L::STAGE);
                const uint64_t dh = um_desc_sw64(st);
                const uint64_t dl = um_desc_sw64(st + L::A_BYTES);
                const uint64_t bh = um_desc_sw64(st + 2 * L::A_BYTES);
                const uint64_t bl = um_desc_sw64(st + 2 * L::A_BYTES + L::B_BYTES);
#pragma unroll
                for (int kk = 0; kk < UM_BK / 8; ++kk) {
                    // K step of 8 tf32 = 32 bytes inside the swizzle row
                    const uint64_t o = (uint64_t)(kk * 32) >> 4;
                    um_mma(tmem, dl + o, bh + o, idesc, (kc | kk) ? 1u : 0u);
                    um_mma(tmem, dh + o, bl + o, idesc, 1u);
                    um_mma(tmem, dh + o, bh + o, idesc, 1u);
                }
                um_commit(&empty[s]);
            }
            // tracks every MMA issued above, also after an abort
            um_commit(done);
        }
        __syncwarp();
    } else {
        const int ct = threadIdx.x - 64;   // 0..127
        for (int kc = 0; kc < nk; ++kc) {
            const int s = kc % UM_STAGES;
            if (!um_wait(&full[s], (kc / UM_STAGES) & 1, abort_flag, true)) break;
            float4* a = (float4*)(sm + s * L::STAGE);
            float4* lo = (float4*)(sm + s * L::STAGE + L::A_BYTES);
#pragma unroll 4
            for (int i = ct; i < (int)(L::A_BYTES / 16); i += 128) {
                float4 x = a[i], h, l;
                h.x = um_rna_tf32(x.x); l.x = um_rna_tf32(x.x - h.x);
                h.y = um_rna_tf32(x.y); l.y = um_rna_tf32(x.y - h.y);
                h.z = um_rna_tf32(x.z); l.z = um_rna_tf32(x.z - h.z);
                h.w = um_rna_tf32(x.w); l.w = um_rna_tf32(x.w - h.w);
                a[i] = h;
                lo[i] = l;
            }
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            um_arrive(&conv[s]);
        }
        // epilogue: this warp owns TMEM lanes 32*(warp%4) .. +31 = tile rows
        const bool ok = um_wait(done, 0, abort_flag, false) && !*abort_flag;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const int q = warp & 3;
        const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
        if (ok) {
            if (e.transposed) {
                const long r = m0 + 32 * q + lane;
                float* o = out + (r / e.rows_per_plane) * e.ob + (r % e.rows_per_plane) * e.oq;
                for (int c0 = 0; c0 < BN; c0 += 16) {
                    uint32_t v[16];
                    um_ld16(trow + c0, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        float x = __uint_as_float(v[j]);
                        if (e.scale_mode == 1) x = x * e.scale;
                        else if (e.scale_mode == 2) x = x / e.scale;
                        o[(long)(c0 + j) * e.on] = x;   // lanes = consecutive rows
                    }
                }
            } else {
                // row-major output: transpose 32x32 blocks through shared
                // memory (the pipeline stages are idle now) so that a warp
                // stores 32 consecutive columns of one row at a time
                float* buf = (float*)sm + (warp - 2) * 32 * 33;
                float* o = out + tile_origin(e, m0, q, lane);
                for (int c0 = 0; c0 < BN; c0 += 32) {
                    uint32_t v[32];
                    um_ld16(trow + c0, v);
                    um_ld16(trow + c0 + 16, v + 16);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 32; ++j) buf[lane * 33 + j] = __uint_as_float(v[j]);
                    __syncwarp();
#pragma unroll 8
                    for (int rr = 0; rr < 32; ++rr) {
                        float x = buf[rr * 33 + lane];
                        if (e.scale_mode == 1) x = x * e.scale;
                        else if (e.scale_mode == 2) x = x / e.scale;
                        o[(long)rr * e.oq + (long)c0 * e.on] = x;
                    }
                    __syncwarp();
                }
            }
        }
    }

    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicOr(status, (int)ST_TIMEOUT);
}

// ---------------------------------------------------------------------------
// Persistent form of the same pass: one CTA per SM walks tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...; the TMA / convert / MMA pipeline
// runs on across tile boundaries, and two TMEM accumulators (2 x BN columns)
// let the epilogue of one tile overlap the main loop of the next.  The
// arithmetic of every tile (MMA order, epilogue) is that of k_dct_umma, so
// the two kernels give identical results.
//   warp 0      TMA producer         warp 1      TMEM owner, MMA issuer
//   warps 2..5  converters           warps 6..9  epilogue (TMEM lanes 32*(warp%4))
// ---------------------------------------------------------------------------
constexpr int UMP_THREADS = 320;

template <int BN>
struct UmmaPSmem {
    static constexpr uint32_t A_BYTES = UM_BM * UM_BK * 4;
    static constexpr uint32_t B_BYTES = BN * UM_BK * 4;
    static constexpr uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr uint32_t EPI_OFF = UM_STAGES * STAGE;            // 4 x 32x33 floats
    static constexpr uint32_t BAR_OFF = EPI_OFF + 4 * 32 * 33 * 4;
    // full[2] conv[2] empty[2] tfull[2] tempty[2] done, TMEM address, abort
    static constexpr uint32_t TOTAL = BAR_OFF + 256;
    static constexpr uint32_t DYN = TOTAL + 1024;
};

template <int BN>
__global__ void __launch_bounds__(UMP_THREADS, 1)
    k_dct_umma_p(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmBh,
                 const __grid_constant__ CUtensorMap tmBl, int K, int ntiles, UmmaEpi e, float* __restrict__ out,
                 int* __restrict__ status)
{
    using L = UmmaPSmem<BN>;
    extern __shared__ uint8_t ump_raw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)ump_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(sm + L::BAR_OFF);
    uint64_t* full = bars;
    uint64_t* conv = bars + UM_STAGES;
    uint64_t* empty = bars + 2 * UM_STAGES;
    uint64_t* tfull = bars + 3 * UM_STAGES;
    uint64_t* tempty = bars + 3 * UM_STAGES + 2;
    uint64_t* done = bars + 3 * UM_STAGES + 4;
    volatile uint32_t* tmem_slot = (volatile uint32_t*)(bars + 3 * UM_STAGES + 5);
    volatile int* abort_flag = (volatile int*)(bars + 3 * UM_STAGES + 6);
    constexpr uint32_t TCOLS = 2 * BN;   // two accumulators

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = K / UM_BK;
    // tiles of this CTA: blockIdx.x + it * gridDim.x, it < nmine
    const int nmine = blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < UM_STAGES; ++s) {
            um_bar_init(&full[s], 1);
            um_bar_init(&conv[s], 128);
            um_bar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            um_bar_init(&tfull[a], 1);
            um_bar_init(&tempty[a], 128);
        }
        um_bar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         um_smem((const void*)tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int total = nmine * nk;   // k-chunks this CTA streams

    if (warp == 0) {
        if (lane == 0) {
            int last[UM_STAGES];
#pragma unroll
            for (int s = 0; s < UM_STAGES; ++s) last[s] = -1;
            for (int g = 0; g < total; ++g) {
                const int s = g % UM_STAGES, kc = g % nk;
                const int m0 = ((int)blockIdx.x + (g / nk) * (int)gridDim.x) * UM_BM;
                if (g >= UM_STAGES && !um_wait(&empty[s], (g / UM_STAGES + 1) & 1, abort_flag, true)) break;
                uint8_t* st = sm + s * L::STAGE;
                um_arrive_tx(&full[s], L::A_BYTES + 2 * L::B_BYTES);
                um_tma_2d(st, &tmA, &full[s], kc * UM_BK, m0);
                um_tma_2d(st + 2 * L::A_BYTES, &tmBh, &full[s], kc * UM_BK, 0);
                um_tma_2d(st + 2 * L::A_BYTES + L::B_BYTES, &tmBl, &full[s], kc * UM_BK, 0);
                last[s] = g;
            }
            for (int s = 0; s < UM_STAGES; ++s)
                if (last[s] >= 0) um_wait(&full[s], (last[s] / UM_STAGES) & 1, abort_flag, false);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = um_idesc_tf32<BN>();
            bool ok = true;
            for (int it = 0; it < nmine && ok; ++it) {
                const int a = it & 1;
                if (it >= 2 && !um_wait(&tempty[a], ((it >> 1) + 1) & 1, abort_flag, true)) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(a * BN);
                for (int kc = 0; kc < nk; ++kc) {
                    const int g = it * nk + kc, s = g % UM_STAGES;
                    if (!um_wait(&conv[s], (g / UM_STAGES) & 1, abort_flag, true)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                    const uint32_t st = um_smem(sm + s * L::STAGE);
                    const uint64_t dh = um_desc_sw64(st);
                    const uint64_t dl = um_desc_sw64(st + L::A_BYTES);
                    const uint64_t bh = um_desc_sw64(st + 2 * L::A_BYTES);
                    const uint64_t bl = um_desc_sw64(st + 2 * L::A_BYTES + L::B_BYTES);
#pragma unroll
                    for (int kk = 0; kk < UM_BK / 8; ++kk) {
                        const uint64_t o = (uint64_t)(kk * 32) >> 4;
                        um_mma(acc, dl + o, bh + o, idesc, (kc | kk) ? 1u : 0u);
                        um_mma(acc, dh + o, bl + o, idesc, 1u);
                        um_mma(acc, dh + o, bh + o, idesc, 1u);
                    }
                    um_commit(&empty[s]);
                }
                if (ok) um_commit(&tfull[a]);
            }
            um_commit(done);   // tracks every MMA issued above
        }
        __syncwarp();
    } else if (warp < 6) {
        const int ct = threadIdx.x - 64;   // 0..127
        for (int g = 0; g < total; ++g) {
            const int s = g % UM_STAGES;
            if (!um_wait(&full[s], (g / UM_STAGES) & 1, abort_flag, true)) break;
            float4* a = (float4*)(sm + s * L::STAGE);
            float4* lo = (float4*)(sm + s * L::STAGE + L::A_BYTES);
#pragma unroll 4
            for (int i = ct; i < (int)(L::A_BYTES / 16); i += 128) {
                float4 x = a[i], h, l;
                h.x = um_rna_tf32(x.x); l.x = um_rna_tf32(x.x - h.x);
                h.y = um_rna_tf32(x.y); l.y = um_rna_tf32(x.y - h.y);
                h.z = um_rna_tf32(x.z); l.z = um_rna_tf32(x.z - h.z);
                h.w = um_rna_tf32(x.w); l.w = um_rna_tf32(x.w - h.w);
                a[i] = h;
                lo[i] = l;
            }
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            um_arrive(&conv[s]);
        }
    } else {
        // epilogue warps 6..9: TMEM lane quadrant q = warp % 4
        const int q = warp & 3;
        float* buf = (float*)(sm + L::EPI_OFF) + (warp - 6) * 32 * 33;
        for (int it = 0; it < nmine; ++it) {
            const int a = it & 1;
            if (!um_wait(&tfull[a], (it >> 1) & 1, abort_flag, true)) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t trow = tmem + (uint32_t)(a * BN) + ((uint32_t)(32 * q) << 16);
            const long m0 = ((long)blockIdx.x + (long)it * gridDim.x) * UM_BM;
            if (e.transposed) {
                const long r = m0 + 32 * q + lane;
                float* o = out + (r / e.rows_per_plane) * e.ob + (r % e.rows_per_plane) * e.oq;
                for (int c0 = 0; c0 < BN; c0 += 16) {
                    uint32_t v[16];
                    um_ld16(trow + c0, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        float x = __uint_as_float(v[j]);
                        if (e.scale_mode == 1) x = x * e.scale;
                        else if (e.scale_mode == 2) x = x / e.scale;
                        o[(long)(c0 + j) * e.on] = x;
                    }
                }
            } else {
                float* o = out + tile_origin(e, m0, q, lane);
                for (int c0 = 0; c0 < BN; c0 += 32) {
                    uint32_t v[32];
                    um_ld16(trow + c0, v);
                    um_ld16(trow + c0 + 16, v + 16);
                    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 32; ++j) buf[lane * 33 + j] = __uint_as_float(v[j]);
                    __syncwarp();
#pragma unroll 8
                    for (int rr = 0; rr < 32; ++rr) {
                        float x = buf[rr * 33 + lane];
                        if (e.scale_mode == 1) x = x * e.scale;
                        else if (e.scale_mode == 2) x = x / e.scale;
                        o[(long)rr * e.oq + (long)c0 * e.on] = x;
                    }
                    __syncwarp();
                }
            }
            // this accumulator is read out: the MMA warp may overwrite it
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            um_arrive(&tempty[a]);
        }
    }

    // every role: the MMAs issued (also after an abort) retire before TMEM goes
    um_wait(done, 0, abort_flag, false);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicOr(status, (int)ST_TIMEOUT);
}

}  // namespace
}  // namespace pll
