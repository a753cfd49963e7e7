// Shared definitions for the riptide_b200 CUDA library (sm_100a).
//
// Conventions
//  * All arithmetic that must reproduce the reference bit for bit is written with explicit
//    rounding intrinsics (__fadd_rn, __fmul_rn, __fmaf_rn, __fdiv_rn, ...), so that the
//    compiler cannot contract or reorder it. The library is built without --use_fast_math.
//  * Plan arithmetic (downsampling factors, row counts, trial periods) is double precision
//    and follows cpp/periodogram.hpp and cpp/downsample.hpp of the reference.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <math.h>

#include "../../include/riptide_b200.h"

#define RT_HD __host__ __device__ __forceinline__

namespace rt {

// ------------------------------------------------------------------------------------
// Error state (host side). Messages are thread-local; codes mirror include/riptide_b200.h.
// ------------------------------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* where);

#define RT_TRY_CUDA(expr)                                                   \
    do {                                                                    \
        cudaError_t _e = (expr);                                            \
        if (_e != cudaSuccess) return ::rt::check_cuda(_e, #expr);          \
    } while (0)

#define RT_TRY(expr)                                                        \
    do {                                                                    \
        int _s = (expr);                                                    \
        if (_s != RT_OK) return _s;                                         \
    } while (0)

// ------------------------------------------------------------------------------------
// Plan arithmetic shared by host and device. cpp/downsample.hpp:21-38,
// cpp/periodogram.hpp:54-57,135-141,175-183.
// ------------------------------------------------------------------------------------
RT_HD size_t downsampled_size(size_t num_samples, double f)
{
    return (size_t)floor((double)num_samples / f);
}

// downsample.hpp:29-38; pow(v, 2) of the reference is an exact square for the
// integer-valued k-1 and a correctly rounded square for x, written here as v * v.
RT_HD double downsampled_variance(size_t num_samples, double f)
{
    const double k = floor(f);
    const double r = f - k;
    const double x = (double)downsampled_size(num_samples, f) * r;
    if (x > 1) return f - 1.0 / 3.0;
    return (k - 1) * (k - 1) + 2.0 / 3.0 * (x * x) - x + 1.0;
}

RT_HD size_t ceilshift(size_t rows, size_t cols, double pmax)
{
    return (size_t)ceil((double)cols * (rows - 1.0) * (1.0 - (double)cols / pmax));
}

RT_HD size_t rows_to_evaluate(size_t rows, size_t bins, double period_max_samples)
{
    const double period_ceil = period_max_samples < bins + 1.0 ? period_max_samples : bins + 1.0;
    const size_t cs = ceilshift(rows, bins, period_ceil);
    return rows < cs ? rows : cs;
}

// periodogram.hpp:192, with bins*bins evaluated first as the reference build does
// (-fassociative-math); exact in double.
RT_HD double trial_period(double tau, size_t bins, size_t s, size_t rows)
{
    return tau * ((double)bins * (double)bins) / ((double)bins - (double)s / (rows - 1.0));
}

// FFA merge row indices, transforms.hpp:17-24: float32 slope, h = size_t(kh*s + 0.5f),
// evaluated as one fused multiply-add like the reference build (-march=native, GCC's
// default -ffp-contract=fast).
struct MergeCoef {
    float kh, kt;
};

__device__ __forceinline__ MergeCoef merge_coef(int rows)
{
    const int mh = rows >> 1, mt = rows - mh;
    MergeCoef c;
    c.kh = __fdiv_rn((float)mh - 1.0f, (float)rows - 1.0f);
    c.kt = __fdiv_rn((float)mt - 1.0f, (float)rows - 1.0f);
    return c;
}

__device__ __forceinline__ int merge_row(float k, int s)
{
    return (int)__fmaf_rn(k, (float)s, 0.5f);
}

// Host copy of the same index arithmetic (used by the planners). std::fma is correctly
// rounded, identical to __fmaf_rn.
inline void merge_coef_host(int rows, float* kh, float* kt)
{
    const int mh = rows >> 1, mt = rows - mh;
    volatile float num_h = (float)mh - 1.0f, num_t = (float)mt - 1.0f, den = (float)rows - 1.0f;
    *kh = num_h / den;
    *kt = num_t / den;
}

inline int merge_row_host(float k, int s) { return (int)fmaf(k, (float)s, 0.5f); }

// ------------------------------------------------------------------------------------
// Misc
// ------------------------------------------------------------------------------------
RT_HD int ceil_div(int a, int b) { return (a + b - 1) / b; }
RT_HD size_t ceil_div_z(size_t a, size_t b) { return (a + b - 1) / b; }

// Order-preserving map float -> uint32 (for atomicMax on floats of any sign).
__device__ __forceinline__ unsigned float_to_ordered(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(unsigned u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

}  // namespace rt
