// Boxcar S/N of folded profiles held in shared memory (cpp/snr.hpp:37-65).
//
// Per profile x of b bins the reference computes the circular prefix sum
//     C[j] = float(sum_{i<=j} x[i])  (double accumulator),  C[b+j] = C[j] + float(total)
// (cpp/kernels.hpp:73-101) and, for every trial width w,
//     dmax = max_i (C[i+w] - C[i]),  h = sqrt((b-w)/(b*w)),  beta = w/(b-w)*h,
//     S/N = ((h + beta) * dmax - beta * C[b-1]) / stdnoise
// (snr.hpp:49-52; the reference build fuses the first product and the subtraction, which is
// reproduced with __fmaf_rn). Everything below follows that arithmetic exactly; the only
// change of order is the prefix sum, done as a warp scan in double: identical to the
// reference's sequential double sum whenever the double sums are exact (float inputs whose
// magnitudes within one profile span less than 2^29).
//
// Work split: one warp computes C for a profile; then TPR threads share one profile, each
// holding a window C[i .. i+SB+WMAX) in registers so that every width reads registers only.
#pragma once
#include "common.cuh"

namespace rt {

// Trial widths generate_width_trials(bmin, ducy_max=0.2, wtsp=1.5) begin with these ten
// for every bmin >= 210 (ffautils.py:4-11). They get the register-window fast path.
struct FastWidths10 {
    static constexpr int NW = 10;
    static constexpr int WMAX = 42;
    __host__ __device__ static constexpr int w(int k)
    {
        return k == 0 ? 1 : k == 1 ? 2 : k == 2 ? 3 : k == 3 ? 4 : k == 4 ? 6 : k == 5 ? 9
             : k == 6 ? 13 : k == 7 ? 19 : k == 8 ? 28 : 42;
    }
};

constexpr int kMaxWidths = 64;

// Per-call width data, placed in shared memory by the caller.
struct SnrParams {
    int nw;                  // number of trial widths
    int nfast;               // leading widths handled by the register window (0 or 10)
    int wmax;                // largest width
    int w[kMaxWidths];
    float hb[kMaxWidths];    // h + beta (per width, for the current b)
    float beta[kMaxWidths];  // beta
};

// Boxcar coefficients for profile length b (snr.hpp:49-50).
__device__ __forceinline__ void boxcar_coefs(int b, int w, float* hb, float* beta)
{
    const float h = __fsqrt_rn(__fdiv_rn((float)(b - w), (float)((size_t)b * (size_t)w)));
    const float be = __fmul_rn(__fdiv_rn((float)w, (float)(b - w)), h);
    *hb = __fadd_rn(h, be);
    *beta = be;
}

__device__ inline void snr_params_fill(SnrParams& S, const int* widths, int nw, int nfast, int b)
{
    if (threadIdx.x == 0) {
        S.nw = nw;
        S.nfast = nfast;
        int wm = 0;
        for (int k = 0; k < nw; ++k) wm = widths[k] > wm ? widths[k] : wm;
        S.wmax = wm;
    }
    for (int k = threadIdx.x; k < nw; k += blockDim.x) {
        S.w[k] = widths[k];
        boxcar_coefs(b, widths[k], &S.hb[k], &S.beta[k]);
    }
    __syncthreads();
}

// Circular prefix sums of `nrows` profiles (rows of `x`, stride xs) into C (stride cs, each row
// b + wmax entries). One warp per profile.
__device__ inline void prefix_rows(const float* x, int xs, int nrows, int b, int wmax, float* C, int cs)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw_ = blockDim.x >> 5;
    const int K = ((b + 31) >> 5) | 1;  // odd chunk: the 32 lanes hit distinct banks
    for (int r = warp; r < nrows; r += nw_) {
        const float* xr = x + (size_t)r * xs;
        float* cr = C + (size_t)r * cs;
        const int c0 = lane * K;
        const int c1 = min(b, c0 + K);
        double local = 0.0;
        for (int c = c0; c < c1; ++c) local += (double)xr[c];
        double incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        double run = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) run = 0.0;
        for (int c = c0; c < c1; ++c) {
            run += (double)xr[c];
            cr[c] = __double2float_rn(run);
        }
        const double total = __shfl_sync(0xffffffffu, incl, 31);
        const float sumx = __double2float_rn(total);
        __syncwarp();
        for (int j = lane; j < wmax; j += 32) cr[b + j] = __fadd_rn(cr[j], sumx);
        __syncwarp();
    }
}

// Max over phases of C[i+w] - C[i] for the fast widths, register window. Each thread covers
// phases [i0, i1) of one profile.
template <class WS, int SB>
__device__ __forceinline__ void window_max(const float* cr, int i0, int i1, int climit,
                                           float (&mx)[WS::NW])
{
    for (int base = i0; base < i1; base += SB) {
        float win[SB + WS::WMAX];
#pragma unroll
        for (int j = 0; j < SB + WS::WMAX; ++j) win[j] = cr[min(base + j, climit)];
        const int nvalid = i1 - base;
#pragma unroll
        for (int j = 0; j < SB; ++j) {
            if (j < nvalid) {
#pragma unroll
                for (int k = 0; k < WS::NW; ++k)
                    mx[k] = fmaxf(mx[k], __fsub_rn(win[j + WS::w(k)], win[j]));
            }
        }
    }
}

// S/N of `nrows` profiles whose prefix sums are rows of C; writes out[r * out_stride + k].
// TPR threads per profile. `stdnoise` is the same for all rows.
template <int TPR, int SB>
__device__ void snr_rows_from_prefix(const float* C, int cs, int nrows, int b, const SnrParams& S,
                                     float stdnoise, float* __restrict__ out, size_t out_stride)
{
    const int tid = threadIdx.x;
    const int rows_per_pass = blockDim.x / TPR;
    const int g = tid / TPR, t = tid - g * TPR;
    const int P = ((b + TPR - 1) / TPR) | 1;  // odd: threads of a profile hit distinct banks
    const int i0 = min(b, t * P), i1 = min(b, i0 + P);
    const int climit = b + S.wmax - 1;
    for (int r0 = 0; r0 < nrows; r0 += rows_per_pass) {
        const int r = r0 + g;
        const bool active = r < nrows;  // whole TPR groups share `active`
        const float* cr = C + (size_t)(active ? r : 0) * cs;
        float mx[FastWidths10::NW];
#pragma unroll
        for (int k = 0; k < FastWidths10::NW; ++k) mx[k] = -INFINITY;
        if (active && S.nfast == FastWidths10::NW)
            window_max<FastWidths10, SB>(cr, i0, i1, climit, mx);
#pragma unroll
        for (int k = 0; k < FastWidths10::NW; ++k) {
#pragma unroll
            for (int o = TPR / 2; o > 0; o >>= 1)
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
        const float sum = active ? cr[b - 1] : 0.f;
        if (active) {
            float* orow = out + (size_t)r * out_stride;
            for (int k = t; k < S.nfast; k += TPR) {
                float dm = mx[0];
#pragma unroll
                for (int q = 1; q < FastWidths10::NW; ++q) dm = (k == q) ? mx[q] : dm;
                orow[k] = __fdiv_rn(__fmaf_rn(S.hb[k], dm, -__fmul_rn(S.beta[k], sum)), stdnoise);
            }
        }
        // remaining widths: direct shared-memory reads, one width per pass
        for (int k = S.nfast; k < S.nw; ++k) {
            const int w = S.w[k];
            float m = -INFINITY;
            if (active)
                for (int i = i0; i < i1; ++i) m = fmaxf(m, __fsub_rn(cr[i + w], cr[i]));
#pragma unroll
            for (int o = TPR / 2; o > 0; o >>= 1)
                m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (active && t == 0)
                out[(size_t)r * out_stride + k] =
                    __fdiv_rn(__fmaf_rn(S.hb[k], m, -__fmul_rn(S.beta[k], sum)), stdnoise);
        }
    }
}

// Row stride for prefix-sum rows: >= b + wmax and = TPR (mod 32), so that with an odd
// per-thread phase count the TPR threads of a profile and the 32/TPR profiles of a warp read
// distinct banks.
RT_HD int prefix_stride(int b, int wmax, int tpr)
{
    int s = b + wmax;
    s = (s + 31) & ~31;
    return s + tpr;
}

RT_HD int snr_tpr(int b) { return b <= 264 ? 8 : 16; }

}  // namespace rt
