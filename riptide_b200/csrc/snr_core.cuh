// Boxcar S/N of folded profiles held in shared memory (cpp/snr.hpp:37-65).
//
// Per profile x of b bins the reference computes the circular prefix sum
//     C[j] = float(sum_{i<=j} x[i])  (double accumulator),  C[b+j] = C[j] + float(total)
// (cpp/kernels.hpp:73-101) and, for every trial width w,
//     dmax = max_i (C[i+w] - C[i]),  h = sqrt((b-w)/(b*w)),  beta = w/(b-w)*h,
//     S/N = ((h + beta) * dmax - beta * C[b-1]) / stdnoise
// (snr.hpp:49-52; the reference build fuses the first product and the subtraction, which is
// reproduced with __fmaf_rn). Everything below follows that arithmetic exactly; the only
// change of order is the prefix sum: the TPR threads of a profile sum their segments (in
// double), scan the segment totals and accumulate their running prefixes (in double-float
// pairs), which is identical to the reference's sequential double sum whenever the sums are
// exact (float inputs whose magnitudes within one profile span less than about 2^24).
//
// Work split: TPR threads share one profile; each builds its segment of C, then holds a
// window C[i .. i+SB+WMAX) in registers so that every width reads registers only.
#pragma once
#include "common.cuh"
#include "ffa_core.cuh"

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
    for (int k = threadIdx.x; k < nw; k += kThreads) {
        S.w[k] = widths[k];
        boxcar_coefs(b, widths[k], &S.hb[k], &S.beta[k]);
    }
    cta_sync();
}

// The same parameters filled by one warp (no CTA barrier).
__device__ inline void snr_params_fill_warp(SnrParams& S, const int* widths, int nw, int nfast,
                                            int b)
{
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        S.nw = nw;
        S.nfast = nfast;
        int wm = 0;
        for (int k = 0; k < nw; ++k) wm = widths[k] > wm ? widths[k] : wm;
        S.wmax = wm;
    }
    for (int k = lane; k < nw; k += 32) {
        S.w[k] = widths[k];
        boxcar_coefs(b, widths[k], &S.hb[k], &S.beta[k]);
    }
    __syncwarp();
}

// Double-float accumulation (Knuth's TwoSum): (hi, lo) holds a sum exactly while it needs no
// more than about 48 significant bits -- the float32 counterpart of the reference's double
// accumulator (kernels.hpp:75-83), which is exact up to 53 bits. round(hi + lo) is then the
// correctly rounded prefix, i.e. the reference's float(acc). Pure FP32 adds: no conversions.
__device__ __forceinline__ void df_add(float& hi, float& lo, float x)
{
    const float s = __fadd_rn(hi, x);
    const float bp = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(x, bp));
    hi = s;
    lo = __fadd_rn(lo, e);
}

__device__ __forceinline__ void df_add2(float& hi, float& lo, float bhi, float blo)
{
    const float s = __fadd_rn(hi, bhi);
    const float bp = __fsub_rn(s, hi);
    const float e = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bp)), __fsub_rn(bhi, bp));
    hi = s;
    lo = __fadd_rn(__fadd_rn(lo, blo), e);
}

__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Max over SB consecutive phases [start, start + SB) of C[i+w] - C[i], for the fast widths,
// from a register window (start + SB <= b, so every phase is a real phase of the profile).
// Threads of one profile may cover overlapping phases: a maximum does not mind duplicates.
template <class WS, int SB>
__device__ __forceinline__ void window_max(const float* cr, int start, float (&mx)[WS::NW])
{
    static_assert(SB % 2 == 0, "phase pairs");
    float win[SB + WS::WMAX];
#pragma unroll
    for (int j = 0; j < SB + WS::WMAX; ++j) win[j] = cr[start + j];
#pragma unroll
    for (int j = 0; j < SB; j += 2) {
#pragma unroll
        for (int k = 0; k < WS::NW; ++k) {
            if (WS::w(k) % 2 == 0) {
                // even width: both phases' differences in one packed subtraction (two
                // round-to-nearest float32 subtractions, as __fsub_rn)
                float d0, d1;
                asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
                    " sub.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
                    : "=f"(d0), "=f"(d1)
                    : "f"(win[j + WS::w(k)]), "f"(win[j + 1 + WS::w(k)]), "f"(win[j]), "f"(win[j + 1]));
                mx[k] = fmax3(mx[k], d0, d1);
            } else {
                mx[k] = fmax3(mx[k], __fsub_rn(win[j + WS::w(k)], win[j]),
                              __fsub_rn(win[j + 1 + WS::w(k)], win[j + 1]));
            }
        }
    }
}

// Boxcar S/N of `nrows` folded profiles (rows of X, stride xs) straight from the FFA output:
// TPR threads per profile build its circular prefix sum (double accumulation, group scan) in
// the scratch rows C (stride cs), then take the width maxima from a register window. Only
// warp-level synchronisation: a profile's TPR threads are lanes of one warp. Writes
// out[r * out_stride + k]. `groups` profiles are processed at a time (C holds `groups` rows).
// Phases per thread of a TPR-thread profile for which the prefix passes are unrolled (the
// thread's values held in registers): bins up to 264 with 8 threads, up to 544 with 16.
template <int TPR>
constexpr int snr_unrolled_phases() { return TPR == 8 ? 33 : 35; }

template <int TPR, int SB, bool kUnrolled>
__device__ void snr_rows_impl(const float* X, int xs, int nrows, int b, const SnrParams& S,
                              float stdnoise, float* __restrict__ out, size_t out_stride,
                              float* C, int cs, int groups)
{
    constexpr int PMAX = kUnrolled ? snr_unrolled_phases<TPR>() : 1;
    const int tid = threadIdx.x;
    const int g = tid / TPR, t = tid - g * TPR;
    const int ngroups = min(groups, kThreads / TPR);
    const int P = ((b + TPR - 1) / TPR) | 1;  // odd: threads of a profile hit distinct banks
    const int i0 = min(b, t * P), i1 = min(b, i0 + P);
    const unsigned gmask = (TPR == 32) ? 0xffffffffu : (((1u << TPR) - 1u) << ((tid & 31) & ~(TPR - 1)));
    if (g >= ngroups) return;  // whole groups leave together
    float* cr = C + (size_t)g * cs;
    for (int r = g; r < nrows; r += ngroups) {
        const float* xr = X + (size_t)r * xs;
        // prefix sums (kernels.hpp:73-101): exact sums, float stores. The thread's segment
        // total is summed in double (cheaper here than double-float pairs) and split into a
        // double-float pair for the scan; the running prefix is accumulated in double-float.
        // With at most PMAX phases per thread, the thread's values are loaded once into
        // registers.
        constexpr bool unrolled = kUnrolled;
        float v[PMAX];
        double seg = 0.0;
        if (unrolled) {
#pragma unroll
            for (int j = 0; j < PMAX; ++j) v[j] = (j < i1 - i0) ? xr[i0 + j] : 0.0f;
#pragma unroll
            for (int j = 0; j < PMAX; ++j) seg = __dadd_rn(seg, (double)v[j]);
        } else {
            for (int i = i0; i < i1; ++i) seg = __dadd_rn(seg, (double)xr[i]);
        }
        const float lh = __double2float_rn(seg);
        const float ll = __double2float_rn(__dsub_rn(seg, (double)lh));
        float ih = lh, il = ll;  // inclusive scan over the TPR segments
#pragma unroll
        for (int o = 1; o < TPR; o <<= 1) {
            const float yh = __shfl_up_sync(gmask, ih, o, TPR);
            const float yl = __shfl_up_sync(gmask, il, o, TPR);
            if (t >= o) {
                // (earlier segments) + (this range), in order of increasing phase
                float nh = yh, nl = yl;
                df_add2(nh, nl, ih, il);
                ih = nh;
                il = nl;
            }
        }
        float rh = __shfl_up_sync(gmask, ih, 1, TPR), rl = __shfl_up_sync(gmask, il, 1, TPR);
        if (t == 0) rh = rl = 0.f;
        if (unrolled) {
#pragma unroll
            for (int j = 0; j < PMAX; ++j) {
                df_add(rh, rl, v[j]);  // adding the zero padding changes nothing stored
                if (j < i1 - i0) cr[i0 + j] = __fadd_rn(rh, rl);
            }
        } else {
            for (int i = i0; i < i1; ++i) {
                df_add(rh, rl, xr[i]);
                cr[i] = __fadd_rn(rh, rl);
            }
        }
        const float th = __shfl_sync(gmask, ih, TPR - 1, TPR), tl = __shfl_sync(gmask, il, TPR - 1, TPR);
        const float sumx = __fadd_rn(th, tl);
        __syncwarp(gmask);
        for (int j = t; j < S.wmax; j += TPR) cr[b + j] = __fadd_rn(cr[j], sumx);
        __syncwarp(gmask);
        const float sum = cr[b - 1];
        float mx[FastWidths10::NW];
#pragma unroll
        for (int k = 0; k < FastWidths10::NW; ++k) mx[k] = -INFINITY;
        if (S.nfast == FastWidths10::NW) {
            if (b >= SB && P <= SB) {
                window_max<FastWidths10, SB>(cr, min(i0, b - SB), mx);
            } else {
                for (int i = i0; i < i1; ++i)
#pragma unroll
                    for (int k = 0; k < FastWidths10::NW; ++k)
                        mx[k] = fmaxf(mx[k], __fsub_rn(cr[i + FastWidths10::w(k)], cr[i]));
            }
        }
#pragma unroll
        for (int k = 0; k < FastWidths10::NW; ++k) {
#pragma unroll
            for (int o = TPR / 2; o > 0; o >>= 1)
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(gmask, mx[k], o, TPR));
        }
        float* orow = out + (size_t)r * out_stride;
        for (int k = t; k < S.nfast; k += TPR) {
            float dm = mx[0];
#pragma unroll
            for (int q = 1; q < FastWidths10::NW; ++q) dm = (k == q) ? mx[q] : dm;
            orow[k] = __fdiv_rn(__fmaf_rn(S.hb[k], dm, -__fmul_rn(S.beta[k], sum)), stdnoise);
        }
        // remaining widths (63 and 94 for bins_min 480), two at a time straight from shared
        // memory: each phase's C[i] is loaded once for both widths, eight phases per step
        for (int k = S.nfast; k < S.nw; k += 2) {
            const bool two = k + 1 < S.nw;
            const int w1 = S.w[k], w2 = two ? S.w[k + 1] : w1;
            float m1 = -INFINITY, m2 = -INFINITY;
            int i = i0;
            for (; i + 8 <= i1; i += 8) {
                float a[8], p[8], q[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    a[j] = cr[i + j];
                    p[j] = cr[i + j + w1];
                    q[j] = cr[i + j + w2];
                }
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    m1 = fmax3(m1, __fsub_rn(p[j], a[j]), __fsub_rn(p[j + 1], a[j + 1]));
                    m2 = fmax3(m2, __fsub_rn(q[j], a[j]), __fsub_rn(q[j + 1], a[j + 1]));
                }
            }
            for (; i < i1; ++i) {
                const float a = cr[i];
                m1 = fmaxf(m1, __fsub_rn(cr[i + w1], a));
                m2 = fmaxf(m2, __fsub_rn(cr[i + w2], a));
            }
#pragma unroll
            for (int o = TPR / 2; o > 0; o >>= 1) {
                m1 = fmaxf(m1, __shfl_xor_sync(gmask, m1, o, TPR));
                m2 = fmaxf(m2, __shfl_xor_sync(gmask, m2, o, TPR));
            }
            if (t == 0) {
                orow[k] = __fdiv_rn(__fmaf_rn(S.hb[k], m1, -__fmul_rn(S.beta[k], sum)), stdnoise);
                if (two)
                    orow[k + 1] =
                        __fdiv_rn(__fmaf_rn(S.hb[k + 1], m2, -__fmul_rn(S.beta[k + 1], sum)), stdnoise);
            }
        }
        __syncwarp(gmask);  // cr is rewritten for the next profile
    }
}

template <int TPR, int SB>
__device__ __forceinline__ void snr_rows(const float* X, int xs, int nrows, int b,
                                         const SnrParams& S, float stdnoise,
                                         float* __restrict__ out, size_t out_stride, float* C,
                                         int cs, int groups)
{
    if ((((b + TPR - 1) / TPR) | 1) <= snr_unrolled_phases<TPR>())
        snr_rows_impl<TPR, SB, true>(X, xs, nrows, b, S, stdnoise, out, out_stride, C, cs, groups);
    else
        snr_rows_impl<TPR, SB, false>(X, xs, nrows, b, S, stdnoise, out, out_stride, C, cs, groups);
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
