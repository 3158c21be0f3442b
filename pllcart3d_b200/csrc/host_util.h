// Host-side helpers shared by the runtime and the stand-alone primitives.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace pll {

inline bool is_pow2(double h)
{
    int e;
    const double m = std::frexp(h, &e);
    return m == 0.5;
}

// FFTW REDFT10 (kind 0) / REDFT01 (kind 1) as dense matrices T[k*n+j]
// (FFTW 3 manual, "1d Real-even DFTs (DCTs)"); the argument is reduced
// mod 4n exactly
template <typename T>
inline void dct_matrix(int kind, int n, T* out)
{
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j) {
            double v;
            if (kind == 0) {
                const long m = ((long)(2 * j + 1) * (long)k) % (4L * n);
                v = 2.0 * std::cos(pi * (double)m / (2.0 * n));
            } else if (j == 0) {
                v = 1.0;
            } else {
                const long m = ((long)j * (long)(2 * k + 1)) % (4L * n);
                v = 2.0 * std::cos(pi * (double)m / (2.0 * n));
            }
            out[(long)k * n + j] = (T)v;
        }
}

// owning device buffer released on scope exit
struct DevBuf {
    void* p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    bool alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 8) == cudaSuccess; }
    double* d() { return (double*)p; }
};

}  // namespace pll
