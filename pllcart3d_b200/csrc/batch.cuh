// Launch recording and member-batched launches (ensembles).
//
// Every step kernel is written as a body, NAME_run(blockIdx, gridDim, ...),
// whose first two parameters shadow the built-ins, the __global__ NAME that
// calls it with the real ones, and a spec NAME_b (body + launch bounds).
// Stage launchers hand kernel, shape and arguments to go(): normally it
// launches NAME; while a context records (an ensemble building its graphs)
// it stores the launch instead.  Members whose recorded steps match launch
// for launch (same kernels, shapes and shared memory) form a class, and the
// ensemble issues each of the class's launches once: k_members runs the
// same body over a grid whose z extent is the class size times the
// member's, member m = blockIdx.z / gz reading its own arguments from a
// device table.  Each member so computes exactly what it computes alone.
// Kernels whose arguments hold a tensor map (passed as __grid_constant__)
// have no spec and replay one launch per member.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

namespace pll {

// argument pack with one layout on host and device
template <typename... P>
struct Tup {};
template <typename H, typename... T>
struct Tup<H, T...> {
    H h;
    Tup<T...> t;
};

template <size_t I>
struct TupAt {
    template <typename H, typename... T>
    __host__ __device__ static const auto& get(const Tup<H, T...>& x)
    {
        return TupAt<I - 1>::get(x.t);
    }
};
template <>
struct TupAt<0> {
    template <typename H, typename... T>
    __host__ __device__ static const H& get(const Tup<H, T...>& x)
    {
        return x.h;
    }
};

inline void tup_fill(Tup<>&) {}
template <typename H, typename... T, typename A, typename... B>
void tup_fill(Tup<H, T...>& x, A&& a, B&&... b)
{
    x.h = H(std::forward<A>(a));
    tup_fill(x.t, std::forward<B>(b)...);
}

// one recorded launch of one member (the interface the ensemble sees)
struct LaunchRec {
    const void* fn = nullptr;   // the member's own kernel: identity of the launch
    dim3 grid, blk;
    size_t smem = 0;
    virtual ~LaunchRec() {}
    virtual bool batchable() const = 0;
    virtual size_t arg_bytes() const = 0;
    virtual const void* arg_data() const = 0;
    virtual void one(cudaStream_t st) const = 0;
    // before a capture: the batched kernel's shared-memory opt-in
    virtual cudaError_t prepare() const = 0;
    // n members of a class at once, member m's argument pack at tab + m * stride
    virtual cudaError_t many(const unsigned char* tab, size_t stride, unsigned n, cudaStream_t st) const = 0;
    bool same_launch(const LaunchRec& o) const
    {
        return fn == o.fn && grid.x == o.grid.x && grid.y == o.grid.y && grid.z == o.grid.z && blk.x == o.blk.x &&
               blk.y == o.blk.y && blk.z == o.blk.z && smem == o.smem && arg_bytes() == o.arg_bytes();
    }
};

namespace {

template <auto RUN, typename... P, size_t... I>
__device__ __forceinline__ void member_run(const Tup<P...>& t, uint3 b, dim3 g, std::index_sequence<I...>)
{
    RUN(b, g, TupAt<I>::get(t)...);
}

// the body over members: grid.z = gz x members
template <auto RUN, typename... P>
__global__ void k_members(const unsigned char* __restrict__ tab, unsigned stride, unsigned gz)
{
    const unsigned m = blockIdx.z / gz;
    const Tup<P...>& t = *reinterpret_cast<const Tup<P...>*>(tab + (size_t)m * stride);
    member_run<RUN, P...>(t, make_uint3(blockIdx.x, blockIdx.y, blockIdx.z - m * gz),
                          dim3(gridDim.x, gridDim.y, gz), std::index_sequence_for<P...>{});
}
template <auto RUN, int MAXT, typename... P>
__global__ void __launch_bounds__(MAXT) k_members_b1(const unsigned char* __restrict__ tab, unsigned stride,
                                                     unsigned gz)
{
    const unsigned m = blockIdx.z / gz;
    const Tup<P...>& t = *reinterpret_cast<const Tup<P...>*>(tab + (size_t)m * stride);
    member_run<RUN, P...>(t, make_uint3(blockIdx.x, blockIdx.y, blockIdx.z - m * gz),
                          dim3(gridDim.x, gridDim.y, gz), std::index_sequence_for<P...>{});
}
template <auto RUN, int MAXT, int MINB, typename... P>
__global__ void __launch_bounds__(MAXT, MINB) k_members_b2(const unsigned char* __restrict__ tab, unsigned stride,
                                                           unsigned gz)
{
    const unsigned m = blockIdx.z / gz;
    const Tup<P...>& t = *reinterpret_cast<const Tup<P...>*>(tab + (size_t)m * stride);
    member_run<RUN, P...>(t, make_uint3(blockIdx.x, blockIdx.y, blockIdx.z - m * gz),
                          dim3(gridDim.x, gridDim.y, gz), std::index_sequence_for<P...>{});
}

// minimum blocks per SM of a batched copy: the spec's bminb where it has
// one (a body that reads its arguments from memory holds more registers
// than the kernel that finds them in its parameter bank), else its minb
template <typename B, typename = void>
struct BatchMinb {
    static constexpr int value = B::minb;
};
template <typename B>
struct BatchMinb<B, std::void_t<decltype(B::bminb)>> {
    static constexpr int value = B::bminb;
};

// no body: replayed one launch per member
struct NoBatch {
    static constexpr auto run = nullptr;
    static constexpr int maxt = 0, minb = 0;
};

template <typename B, typename... P>
struct LaunchRecT : LaunchRec {
    void (*k)(P...) = nullptr;
    Tup<P...> a;
    bool batchable() const override { return !std::is_same<B, NoBatch>::value; }
    size_t arg_bytes() const override { return sizeof(Tup<P...>); }
    const void* arg_data() const override { return &a; }
    template <size_t... I>
    void one_(cudaStream_t st, std::index_sequence<I...>) const
    {
        k<<<grid, blk, smem, st>>>(TupAt<I>::get(a)...);
    }
    void one(cudaStream_t st) const override { one_(st, std::index_sequence_for<P...>{}); }
    const void* batched_kernel() const
    {
        if constexpr (std::is_same<B, NoBatch>::value) return nullptr;
        else if constexpr (B::maxt == 0) return (const void*)k_members<B::run, P...>;
        else if constexpr (BatchMinb<B>::value == 0) return (const void*)k_members_b1<B::run, B::maxt, P...>;
        else return (const void*)k_members_b2<B::run, B::maxt, BatchMinb<B>::value, P...>;
    }
    cudaError_t prepare() const override
    {
        // static and dynamic shared memory together above 48 KB need the
        // opt-in, which is a per-device attribute: set on every build (a
        // host call, once per recorded launch, never per step)
        const void* kb = batched_kernel();
        if (kb && smem > 0)
            return cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return cudaSuccess;
    }
    cudaError_t many(const unsigned char* tab, size_t stride, unsigned n, cudaStream_t st) const override
    {
        const void* kb = batched_kernel();
        if (!kb) return cudaErrorInvalidValue;
        unsigned st_ = (unsigned)stride, gz = grid.z;
        const dim3 g(grid.x, grid.y, grid.z * n);
        void* args[3] = {(void*)&tab, (void*)&st_, (void*)&gz};
        return cudaLaunchKernel(kb, g, blk, args, smem, st);
    }
};

}  // namespace
}  // namespace pll
