// Building-block kernels and their host launchers: the drop-ins for the reference's
// `libcpp` functions (cpp/python_bindings.cpp:44-222) and the plain per-(cycle, bins)
// periodogram, which issues one launch per step of the reference's loop nest
// (cpp/periodogram.hpp:153-200). The batched engine (engine.cu) reuses the device code.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "ffa_core.cuh"
#include "snr_core.cuh"
#include "kernels.cuh"

namespace rt {

// ------------------------------------------------------------------------------------
// Error state
// ------------------------------------------------------------------------------------
static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int check_cuda(cudaError_t e, const char* where)
{
    if (e == cudaSuccess) return RT_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_error(RT_ENOMEM, "CUDA out of memory in %s", where);
    }
    return set_error(RT_ECUDA, "CUDA error %s (%s) in %s", cudaGetErrorName(e),
                     cudaGetErrorString(e), where);
}

const char* last_error() { return g_err; }

// ------------------------------------------------------------------------------------
// Elementwise helpers (kernels.hpp:19-38, 73-101)
// ------------------------------------------------------------------------------------
__global__ void k_rollback(const float* __restrict__ x, size_t size, size_t p,
                           float* __restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < size;
         i += (size_t)gridDim.x * blockDim.x) {
        size_t j = i + p;
        if (j >= size) j -= size;
        out[i] = x[j];
    }
}

__global__ void k_fused_rollback_add(const float* __restrict__ x, const float* __restrict__ y,
                                     size_t size, size_t p, float* __restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < size;
         i += (size_t)gridDim.x * blockDim.x) {
        size_t j = i + p;
        if (j >= size) j -= size;
        out[i] = __fadd_rn(x[i], y[j]);
    }
}

static int grid_for(size_t n, int threads)
{
    size_t g = (n + threads - 1) / threads;
    return (int)std::min<size_t>(std::max<size_t>(g, 1), 148 * 32);
}

int rollback(const float* x, size_t size, size_t shift, float* out, cudaStream_t st)
{
    if (size == 0) return RT_OK;
    k_rollback<<<grid_for(size, 256), 256, 0, st>>>(x, size, shift % size, out);
    return check_cuda(cudaGetLastError(), "rollback");
}

int fused_rollback_add(const float* x, const float* y, size_t size, size_t shift, float* out,
                       cudaStream_t st)
{
    if (size == 0) return RT_OK;
    k_fused_rollback_add<<<grid_for(size, 256), 256, 0, st>>>(x, y, size, shift % size, out);
    return check_cuda(cudaGetLastError(), "fused_rollback_add");
}

// circular_prefix_sum (kernels.hpp:73-101). The first min(size, nsum) sums are the
// reference's: one double accumulator taking the values in order, each partial sum rounded
// to float. That order is kept exactly (a parallel scan rounds differently whenever a partial
// sum is not representable in double, which random data of a few hundred thousand values
// already reaches): one CTA stages chunks of x in shared memory, thread 0 runs the sequential
// double sum over them, and the CTA writes the rounded sums back.
constexpr int kCpsChunk = 4096;

__global__ void __launch_bounds__(256) k_cps_head(const float* __restrict__ x, size_t jmax,
                                                  float* __restrict__ out)
{
    __shared__ float sx[kCpsChunk];
    double acc = 0.0;  // thread 0 only
    for (size_t c0 = 0; c0 < jmax; c0 += kCpsChunk) {
        const int n = (int)min((size_t)kCpsChunk, jmax - c0);
        for (int i = threadIdx.x; i < n; i += blockDim.x) sx[i] = x[c0 + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int i = 0; i < n; ++i) {
                acc = __dadd_rn(acc, (double)sx[i]);
                sx[i] = __double2float_rn(acc);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) out[c0 + i] = sx[i];
        __syncthreads();
    }
}

// The wraps beyond the first `size` sums (kernels.hpp:85-100): out[i*size + j] =
// out[j] + float(i) * sumx with sumx = float(total) = out[size - 1]; full wraps and the last
// partial one use the same formula.
__global__ void k_cps_wraps(size_t size, size_t nsum, float* __restrict__ out)
{
    const float sumx = out[size - 1];
    for (size_t k = size + blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nsum;
         k += (size_t)gridDim.x * blockDim.x) {
        const size_t i = k / size, j = k - i * size;
        out[k] = __fadd_rn(out[j], __fmul_rn(__ull2float_rn((unsigned long long)i), sumx));
    }
}

int circular_prefix_sum(const float* x, size_t size, size_t nsum, float* out, cudaStream_t st)
{
    if (nsum == 0) return RT_OK;
    if (size == 0) return set_error(RT_EINVAL, "input array must not be empty");
    k_cps_head<<<1, 256, 0, st>>>(x, std::min(size, nsum), out);
    RT_TRY_CUDA(cudaGetLastError());
    if (nsum > size) {
        k_cps_wraps<<<grid_for(nsum - size, 256), 256, 0, st>>>(size, nsum, out);
        RT_TRY_CUDA(cudaGetLastError());
    }
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// FFA stage kernel: one CTA per job; root rows written to dst.
// ------------------------------------------------------------------------------------
constexpr size_t kStageTreeBytes = (sizeof(JobTree) + 255) & ~size_t(255);

int ffa_cap_rows(int b) { return ffa_cap_rows_for(kFfaSmemBytes, kStageTreeBytes, b); }

__global__ void __launch_bounds__(kThreads, 1)
    k_ffa_stage(const float* __restrict__ src, float* __restrict__ dst, int m, int b,
                int rows_out, StagePlan P, int stage, int cap_rows, int* err)
{
    extern __shared__ __align__(16) unsigned char smem[];
    JobTree& T = *reinterpret_cast<JobTree*>(smem);
    const FfaSmem L = ffa_smem(smem + kStageTreeBytes, cap_rows, b);
    const int stride = ffa_stride(b);
    const JobSpec J = stage_job(m, rows_out, P, stage, blockIdx.x);
    if (J.hi <= J.lo) return;
    build_job_tree(T, J, cap_rows);
    if (T.error) {
        if (threadIdx.x == 0) atomicExch(err, RT_EINTERNAL);
        return;
    }
    LevelIO io;
    io.src = src;
    io.src_stride = b;
    io.root_dst = root_rows_dst(T, b, dst);
    io.root_stride = b;
    run_job_levels(T, b, L.buf0, L.buf1, stride, L.ops, io);
}

bool plan_stages(int m, int rows_out, int cap_rows, StagePlan* P, int max_depth)
{
    memset(P, 0, sizeof(*P));
    max_depth = std::max(0, std::min(max_depth, kMaxJobDepth));
    if (m <= cap_rows && full_depth(m) <= max_depth) {
        P->nstages = 1;
        P->D[0] = 0;
        P->R[0] = rows_out;
        P->jobs[0] = 1;
        P->jobs_per_node[0] = 1;
        return true;
    }
    int D = 0;
    while ((((m + (1 << D) - 1) >> D) > cap_rows) || full_depth((m + (1 << D) - 1) >> D) > max_depth) {
        ++D;
        if (D > 20) return false;
    }
    int ns = 0;
    P->D[0] = D;
    P->R[0] = (m + (1 << D) - 1) >> D;
    P->jobs[0] = 1 << D;
    P->jobs_per_node[0] = 1;
    ns = 1;
    while (D > 0) {
        if (ns >= kMaxStages) return false;
        // largest step e such that R = cap - 3 * 2^(e-1) stays >= cap / 2 (at least 1 level)
        int e = std::min(D, max_depth + 1);
        int R = 0;
        for (; e >= 1; --e) {
            R = cap_rows - 3 * (1 << (e - 1));
            if (R >= cap_rows / 2 || e == 1) break;
        }
        if (R < 1) return false;
        const int Dn = D - e;
        const int node_rows = (m + (1 << Dn) - 1) >> Dn;
        const int need = (Dn == 0) ? rows_out : node_rows;
        P->D[ns] = Dn;
        P->R[ns] = R;
        P->jobs_per_node[ns] = std::max(1, (need + R - 1) / R);
        P->jobs[ns] = P->jobs_per_node[ns] << Dn;
        ++ns;
        D = Dn;
    }
    P->nstages = ns;
    return true;
}

int ffa_transform(const float* in, int m, int b, int rows_out, float* out, float* scratch,
                  int* d_err, cudaStream_t st)
{
    const int cap = ffa_cap_rows(b);
    StagePlan P;
    if (cap < 4 || !plan_stages(m, rows_out, cap, &P))
        return set_error(RT_EINVAL, "FFA transform of %d x %d does not fit the device plan", m, b);
    if (P.nstages > 1 && scratch == nullptr)
        return set_error(RT_EINTERNAL, "FFA transform of %d x %d needs scratch memory", m, b);
    RT_TRY_CUDA(cudaFuncSetAttribute(k_ffa_stage, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kFfaSmemBytes));
    const float* src = in;
    for (int s = 0; s < P.nstages; ++s) {
        float* dst = (s == P.nstages - 1) ? out : scratch + (size_t)(s & 1) * m * b;
        k_ffa_stage<<<P.jobs[s], kThreads, kFfaSmemBytes, st>>>(src, dst, m, b, rows_out, P, s,
                                                               cap, d_err);
        RT_TRY_CUDA(cudaGetLastError());
        src = dst;
    }
    return RT_OK;
}

size_t ffa_scratch_floats(int m, int b)
{
    // multi-stage plans (too many rows, or too deep for one job) need two scratch copies
    StagePlan P;
    if (!plan_stages(m, m, ffa_cap_rows(b), &P) || P.nstages == 1) return 0;
    return 2 * (size_t)m * b;
}

// ------------------------------------------------------------------------------------
// S/N of rows in global memory (snr.hpp:58-65)
// ------------------------------------------------------------------------------------
template <int TPR>
__global__ void __launch_bounds__(kThreads, 1)
    k_snr2(const float* __restrict__ x, int rows, int b, const int* __restrict__ widths, int nw,
           int nfast, float stdnoise, float* __restrict__ out, int tile_rows)
{
    extern __shared__ __align__(16) unsigned char smem[];
    SnrParams& S = *reinterpret_cast<SnrParams*>(smem);
    float* C = reinterpret_cast<float*>(smem + ((sizeof(SnrParams) + 255) & ~size_t(255)));
    snr_params_fill(S, widths, nw, nfast, b);
    const int cs = prefix_stride(b, S.wmax, TPR);
    const int groups = min(tile_rows, kThreads / TPR);
    for (int r0 = blockIdx.x * tile_rows; r0 < rows; r0 += gridDim.x * tile_rows) {
        const int nr = min(tile_rows, rows - r0);
        snr_rows<TPR, 34>(x + (size_t)r0 * b, b, nr, b, S, stdnoise, out + (size_t)r0 * nw, nw,
                          C, cs, groups);
    }
}

int snr_tile_rows(int b, int wmax)
{
    const size_t avail = kFfaSmemBytes - ((sizeof(SnrParams) + 255) & ~size_t(255));
    return (int)(avail / (sizeof(float) * prefix_stride(b, wmax, snr_tpr(b))));
}

int detect_fast_widths(const int* w, int nw)
{
    if (nw < FastWidths10::NW) return 0;
    for (int k = 0; k < FastWidths10::NW; ++k)
        if (w[k] != FastWidths10::w(k)) return 0;
    return FastWidths10::NW;
}

int snr2(const float* x, size_t rows, size_t cols, const int* d_widths, const int* h_widths,
         int nw, float stdnoise, float* out, cudaStream_t st)
{
    if (rows == 0 || nw == 0) return RT_OK;
    int wmax = 0;
    for (int k = 0; k < nw; ++k) wmax = std::max(wmax, h_widths[k]);
    const int nfast = detect_fast_widths(h_widths, nw);
    const int tile = std::min<int>(snr_tile_rows((int)cols, wmax), 1024);
    if (tile < 1) return set_error(RT_EINVAL, "profiles of %zu bins are too long", cols);
    const int grid = (int)std::min<size_t>((rows + tile - 1) / tile, 148 * 4);
    if (nw > kMaxWidths) return set_error(RT_EINVAL, "at most %d trial widths are supported", kMaxWidths);
    const int tpr = snr_tpr((int)cols);
    if (tpr == 8) {
        RT_TRY_CUDA(cudaFuncSetAttribute(k_snr2<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFfaSmemBytes));
        k_snr2<8><<<grid, kThreads, kFfaSmemBytes, st>>>(x, (int)rows, (int)cols, d_widths, nw,
                                                         nfast, stdnoise, out, tile);
    } else {
        RT_TRY_CUDA(cudaFuncSetAttribute(k_snr2<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kFfaSmemBytes));
        k_snr2<16><<<grid, kThreads, kFfaSmemBytes, st>>>(x, (int)rows, (int)cols, d_widths, nw,
                                                          nfast, stdnoise, out, tile);
    }
    return check_cuda(cudaGetLastError(), "snr2");
}

// ------------------------------------------------------------------------------------
// Downsampling by a real factor (downsample.hpp:44-82).
//
// One CTA owns the output samples whose first input sample imin = floor(k f) falls in its
// segment [seg0, seg0 + seg). It stages kDsStage samples from seg0 (the segment plus a halo
// of at least f + 1 samples for the largest factor f of the run) in shared memory with
// an exclusive prefix sum in double, so each output costs O(1):
//   out[k] = wmin*z[imin] + (P[imax] - P[imin+1]) + wmax*z[imax]
// with the reference's FP64 sample bounds and float32 edge weights; the sum is formed in
// double and rounded once. When the series is normalised on the way ((v - mean) / norm,
// time_series.py:84-93), the weighted sum of the raw values is normalised instead:
// (acc - mean * W) / norm with W the total weight, one rounding instead of one per sample.
// All cycles of a search are produced in the same pass, so the series is read once.
// Factors with f + 2 > kDsHalo use k_downsample_wide instead.
//
// Layout of the work: a lane owns 4 consecutive staged samples of each 128-sample chunk of
// its warp's 512, read as 16-byte vectors (realigned in registers when the segment does not
// start on a 16-byte boundary, so the staged values and the order of the prefix sums do not
// depend on where the series lies in memory). The prefix is a 4-sample scan in the lane and a
// shuffle scan of the lanes' totals. Outputs of all cycles form one index range; a table gives
// the cycle of each 32-output chunk's first index.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ size_t first_k_at_or_after(size_t i0, double f)
{
    // smallest k with floor(k * f) >= i0
    size_t k = (size_t)ceil((double)i0 / f);
    while (k > 0 && floor((double)(k - 1) * f) >= (double)i0) --k;
    while (floor((double)k * f) < (double)i0) ++k;
    return k;
}

constexpr int kDsThreads = 512;
constexpr int kDsWarps = kDsThreads / 32;
constexpr int kDsPerWarp = kDsStage / kDsWarps;  // staged samples per warp
constexpr int kDsQuads = kDsPerWarp / 128;       // 128-sample chunks per warp, 4 samples a lane
constexpr int kDsTab = 1024;                     // 32-output chunks with a tabulated cycle
static_assert(kDsPerWarp % 128 == 0, "whole chunks");
static_assert(kDsMaxCycles <= 256, "cycle numbers are stored in bytes");

// The 16-byte-aligned group A[j .. j+3] (j a multiple of 4), zero outside [lo, hi).
__device__ __forceinline__ float4 ds_group(const float* A, int j, int lo, int hi)
{
    if (j >= lo && j + 4 <= hi) return __ldg(reinterpret_cast<const float4*>(A + j));
    float4 v;
    v.x = (j >= lo && j < hi) ? __ldg(A + j) : 0.0f;
    v.y = (j + 1 >= lo && j + 1 < hi) ? __ldg(A + j + 1) : 0.0f;
    v.z = (j + 2 >= lo && j + 2 < hi) ? __ldg(A + j + 2) : 0.0f;
    v.w = (j + 3 >= lo && j + 3 < hi) ? __ldg(A + j + 3) : 0.0f;
    return v;
}

__device__ __forceinline__ float ds_normalised(float x, double mean, double inv)
{
    return __double2float_rn(__ddiv_rn(__dsub_rn((double)x, mean), inv));
}

__global__ void __launch_bounds__(kDsThreads, 2)
    k_downsample_segments(DsJob job)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double* P = reinterpret_cast<double*>(smem);                    // kDsStage + 1 (+1 pad)
    float* zs = reinterpret_cast<float*>(P + kDsStage + 2);          // kDsStage
    __shared__ int s_cnt[kDsMaxCycles + 1];
    __shared__ long long s_kb[kDsMaxCycles];  // first output of the cycle here, minus its offset
    __shared__ double s_f[kDsMaxCycles];
    __shared__ float* s_o[kDsMaxCycles];
    __shared__ double s_part[kDsWarps];
    __shared__ unsigned char s_tab[kDsTab];

    const int trial = blockIdx.y;
    const size_t N = job.lengths[trial];
    const int seg = job.seg;
    const size_t seg0 = (size_t)blockIdx.x * seg;
    if (seg0 >= N) return;
    const float* z = job.in + job.in_off[trial] + seg0;
    const int L = (int)std::min<size_t>(kDsStage, N - seg0);
    const double mean = job.mean ? job.mean[trial] : 0.0;
    const double inv = job.norm ? job.norm[trial] : 1.0;
    const bool affine = job.mean != nullptr;
    float* zout = job.norm_out ? job.norm_out + job.in_off[trial] + seg0 : nullptr;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nc = job.ncycles;

    // per-cycle output ranges whose first sample imin = floor(k f) lies in the segment
    const size_t seg1 = std::min(N, seg0 + (size_t)seg);
    if (tid < nc) {
        const int c = tid;
        const double f = job.f[c];
        const size_t n = downsampled_size(N, f);
        int cnt = 0;
        size_t k0 = 0;
        if (job.use_seg[c] && n > 0) {
            k0 = first_k_at_or_after(seg0, f);
            size_t k1 = (seg1 >= N) ? n : first_k_at_or_after(seg1, f);
            k1 = std::min(k1, n);
            cnt = k1 > k0 ? (int)(k1 - k0) : 0;
        }
        s_cnt[c] = cnt;
        s_kb[c] = (long long)k0;
        s_f[c] = f;
        s_o[c] = job.out + job.out_off[(size_t)trial * nc + c];
    }

    // Stage the segment + halo. A = z - sh is 16-byte aligned; staged sample i is A[i + sh].
    const int sh = (int)((reinterpret_cast<uintptr_t>(z) >> 2) & 3);
    const float* A = z - sh;
    const int lo = sh, hi = sh + L;
    float4 v[kDsQuads];
    if (sh == 0) {
#pragma unroll
        for (int q = 0; q < kDsQuads; ++q)
            v[q] = ds_group(A, warp * kDsPerWarp + q * 128 + 4 * lane, lo, hi);
    } else {
        float4 a[kDsQuads], b[kDsQuads];
#pragma unroll
        for (int q = 0; q < kDsQuads; ++q) {
            const int i = warp * kDsPerWarp + q * 128 + 4 * lane;
            a[q] = ds_group(A, i, lo, hi);
            b[q] = ds_group(A, i + 4, lo, hi);
        }
#pragma unroll
        for (int q = 0; q < kDsQuads; ++q) {
            v[q].x = sh == 1 ? a[q].y : sh == 2 ? a[q].z : a[q].w;
            v[q].y = sh == 1 ? a[q].z : sh == 2 ? a[q].w : b[q].x;
            v[q].z = sh == 1 ? a[q].w : sh == 2 ? b[q].x : b[q].y;
            v[q].w = sh == 1 ? b[q].x : sh == 2 ? b[q].y : b[q].z;
        }
    }
    double wsum = 0.0;
#pragma unroll
    for (int q = 0; q < kDsQuads; ++q) {
        const int i = warp * kDsPerWarp + q * 128 + 4 * lane;
        *reinterpret_cast<float4*>(zs + i) = v[q];
        wsum += ((double)v[q].x + (double)v[q].y) + ((double)v[q].z + (double)v[q].w);
        if (zout) {  // the normalised copy of the segment's own samples
            const int m = min(L, seg) - i;
            if (m > 0) zout[i] = ds_normalised(v[q].x, mean, inv);
            if (m > 1) zout[i + 1] = ds_normalised(v[q].y, mean, inv);
            if (m > 2) zout[i + 2] = ds_normalised(v[q].z, mean, inv);
            if (m > 3) zout[i + 3] = ds_normalised(v[q].w, mean, inv);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if (lane == 0) s_part[warp] = wsum;
    __syncthreads();

    if (warp == kDsWarps - 1) {
        // output offsets of the cycles (exclusive scan of the counts) and the chunk table
        int run = 0;
        for (int c0 = 0; c0 < nc; c0 += 32) {
            const int c = c0 + lane;
            const int cnt = c < nc ? s_cnt[c] : 0;
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int off = run + incl - cnt;
            if (c < nc) {
                s_cnt[c] = off;
                s_kb[c] -= off;
                for (int j = (off + 31) >> 5; j < min((int)kDsTab, (off + cnt + 31) >> 5); ++j)
                    s_tab[j] = (unsigned char)c;
            }
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) s_cnt[nc] = run;
    }

    // exclusive prefix in double: the preceding warps' totals, then per chunk the lane's
    // 4-sample scan and a shuffle scan of the lanes' totals
    double carry = lane < warp ? s_part[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) carry += __shfl_xor_sync(0xffffffffu, carry, o);
#pragma unroll
    for (int q = 0; q < kDsQuads; ++q) {
        const int i = warp * kDsPerWarp + q * 128 + 4 * lane;
        const double a0 = (double)v[q].x;
        const double a1 = a0 + (double)v[q].y;
        const double a2 = a1 + (double)v[q].z;
        const double a3 = a2 + (double)v[q].w;
        double incl = a3;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        double ex = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) ex = 0.0;
        const double e = carry + ex;
        *reinterpret_cast<double2*>(P + i) = make_double2(e, e + a0);
        *reinterpret_cast<double2*>(P + i + 2) = make_double2(e + a1, e + a2);
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (tid == kDsThreads - 1) P[kDsStage] = carry;
    __syncthreads();

    // Outputs, in chunks of 32 consecutive indices of the range of all cycles (balanced across
    // warps). A lane starts from the cycle of its chunk's first index and steps forward across
    // the cycle boundaries inside the chunk. Sample positions are made relative to seg0:
    // start - seg0 and end - seg0 are exact (seg0 is an integer at most start), so floor,
    // weights and clamping give the same values as the absolute FP64 bounds of
    // downsample.hpp:58-72.
    const double seg0d = (double)seg0;
    const double lastd = (double)(N - 1 - seg0);
    const double rinv = 1.0 / inv;
    const int total = s_cnt[nc];
    for (int base = warp * 32; base < total; base += kDsThreads) {
        int c;
        if ((base >> 5) < kDsTab) {
            c = s_tab[base >> 5];
        } else {
            c = 0;
            for (int c0 = 1; c0 < nc; c0 += 32) {
                const int cc = c0 + lane;
                c += __popc(__ballot_sync(0xffffffffu, cc < nc && s_cnt[cc] <= base));
            }
        }
        const int q = base + lane;
        if (q >= total) continue;
        while (s_cnt[c + 1] <= q) ++c;
        const double f = s_f[c];
        const size_t k = (size_t)(s_kb[c] + q);
        const double start = (double)k * f;
        const double end = start + f;
        const double sr = start - seg0d, er = end - seg0d;
        // floors of values in [0, 2^13) as doubles; their integer values via the 2^52 + 2^51
        // rounding constant (exact for integral doubles below 2^51)
        const double fl = floor(sr);
        const double fu = fmin(floor(er), lastd);
        const int li = __double2loint(fl + 6755399441055744.0);
        const int ui = __double2loint(fu + 6755399441055744.0);
        const float wmin = __double2float_rn((fl + 1.0) - sr);
        const float wmax = __double2float_rn(er - fu);
        double acc = (double)wmin * (double)zs[li] + (P[ui] - P[li + 1]) +
                     (double)wmax * (double)zs[ui];
        if (affine)  // sum of (v - mean) / norm over the same weights, W = their total
            acc = (acc - mean * ((double)wmin + (fu - fl - 1.0) + (double)wmax)) * rinv;
        s_o[c][k] = __double2float_rn(acc);
    }
}

// Wide factors: one warp per output sample, deterministic warp tree in double.
__global__ void k_downsample_wide(DsJob job, int cycle)
{
    const int trial = blockIdx.y;
    const size_t N = job.lengths[trial];
    const double f = job.f[cycle];
    const size_t n = downsampled_size(N, f);
    const float* z = job.in + job.in_off[trial];
    const double mean = job.mean ? job.mean[trial] : 0.0;
    const double inv = job.norm ? job.norm[trial] : 1.0;
    const double rinv = 1.0 / inv;
    const bool affine = job.mean != nullptr;
    float* o = job.out + job.out_off[(size_t)trial * job.ncycles + cycle];
    const int lane = threadIdx.x & 31;
    const size_t wid = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nwarp = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t k = wid; k < n; k += nwarp) {
        const double start = (double)k * f;
        const double end = start + f;
        const size_t imin = (size_t)floor(start);
        const double fe = floor(end);
        const size_t imax = (size_t)(fe < (double)N - 1.0 ? fe : (double)N - 1.0);
        double acc = 0.0;
        for (size_t i = imin + 1 + lane; i < imax; i += 32) acc += (double)__ldg(z + i);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (lane == 0) {
            const float a = __ldg(z + imin), bb = __ldg(z + imax);
            const float wmin = __double2float_rn((double)(imin + 1) - start);
            const float wmax = __double2float_rn(end - (double)imax);
            double r = (double)wmin * a + acc + (double)wmax * bb;
            if (affine)  // as in k_downsample_segments
                r = (r - mean * ((double)wmin + (double)(imax - imin - 1) + (double)wmax)) * rinv;
            o[k] = __double2float_rn(r);
        }
    }
}

int launch_downsample(const DsJob& job_in, int ntrials, size_t max_len, cudaStream_t st)
{
    DsJob job = job_in;
    if (reinterpret_cast<uintptr_t>(job.in) & 3)
        return set_error(RT_EINVAL, "the series to downsample is not 4-byte aligned");
    bool any_seg = job.norm_out != nullptr;  // the segment pass also writes the normalised copy
    double fmax = 0.0;
    for (int c = 0; c < job.ncycles; ++c) {
        if (job.use_seg_host[c]) fmax = std::max(fmax, job.f_host[c]);
        any_seg |= job.use_seg_host[c] != 0;
    }
    // halo >= f + 1 for every segment factor (ds_use_segments: f + 2 <= kDsHalo), in whole warps
    const int halo = std::min(kDsHalo, ((int)ceil(fmax) + 2 + 31) & ~31);
    job.seg = kDsStage - halo;
    if (any_seg) {
        const size_t smem = (kDsStage + 2) * sizeof(double) + kDsStage * sizeof(float);
        RT_TRY_CUDA(cudaFuncSetAttribute(k_downsample_segments,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        dim3 grid((unsigned)((max_len + job.seg - 1) / job.seg), (unsigned)ntrials);
        k_downsample_segments<<<grid, kDsThreads, smem, st>>>(job);
        RT_TRY_CUDA(cudaGetLastError());
    }
    for (int c = 0; c < job.ncycles; ++c) {
        if (job.use_seg_host[c] || job.skip_host[c]) continue;
        dim3 grid(148 * 2, (unsigned)ntrials);
        k_downsample_wide<<<grid, 256, 0, st>>>(job, c);
        RT_TRY_CUDA(cudaGetLastError());
    }
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// Running median (running_median.hpp:100-132): exact order statistic of rank width/2 of the
// edge-padded window. Counting selection over a shared-memory tile.
// ------------------------------------------------------------------------------------
__global__ void k_running_median(const float* __restrict__ x, const size_t* __restrict__ lengths,
                                 const size_t* __restrict__ offsets, int width,
                                 float* __restrict__ out, int tile)
{
    extern __shared__ float sx[];
    const int trial = blockIdx.y;
    const size_t N = lengths[trial];
    const float* xr = x + offsets[trial];
    float* orow = out + offsets[trial];
    const int half = width / 2;
    const size_t t0 = (size_t)blockIdx.x * tile;
    if (t0 >= N) return;
    const int span = tile + 2 * half;
    for (int i = threadIdx.x; i < span; i += blockDim.x) {
        long long g = (long long)t0 + i - half;
        g = g < 0 ? 0 : (g >= (long long)N ? (long long)N - 1 : g);
        sx[i] = xr[g];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < tile; i += blockDim.x) {
        const size_t gi = t0 + i;
        if (gi >= N) break;
        const float* win = sx + i;
        float med = win[0];
        for (int j = 0; j < width; ++j) {
            const float cand = win[j];
            int less = 0, leq = 0;
            for (int q = 0; q < width; ++q) {
                const float v = win[q];
                less += v < cand;
                leq += v <= cand;
            }
            if (less <= half && half < leq) {
                med = cand;
                break;
            }
        }
        orow[gi] = med;
    }
}

// Running median through a sorted tile: a CTA sorts the tile + w - 1 (edge-padded) values of
// its windows once, by (value, position); the median of the window starting at t is the
// (w / 2 + 1)-th entry of that order whose position lies in [t, t + w). The same order
// statistic as the counting kernel above, found in ~(w / 2) * (tile + w) / w steps.
constexpr int kRmedSortTile = 256;
constexpr int kRmedSortSpan = 512;  // tile + width - 1 <= span

__global__ void __launch_bounds__(kRmedSortTile)
    k_running_median_sorted(const float* __restrict__ x, const size_t* __restrict__ lengths,
                            const size_t* __restrict__ offsets, int width,
                            float* __restrict__ out)
{
    __shared__ float sv[kRmedSortSpan];
    __shared__ short sp[kRmedSortSpan];
    const int trial = blockIdx.y;
    const size_t N = lengths[trial];
    const size_t t0 = (size_t)blockIdx.x * kRmedSortTile;
    if (t0 >= N) return;
    const float* xr = x + offsets[trial];
    const int half = width / 2;
    const int span = kRmedSortTile + width - 1;
    for (int i = threadIdx.x; i < kRmedSortSpan; i += blockDim.x) {
        if (i < span) {
            long long g = (long long)t0 + i - half;
            g = g < 0 ? 0 : (g >= (long long)N ? (long long)N - 1 : g);
            sv[i] = xr[g];
            sp[i] = (short)i;
        } else {
            sv[i] = INFINITY;
            sp[i] = (short)kRmedSortSpan;
        }
    }
    __syncthreads();
    // bitonic sort by (value, position)
    for (int k = 2; k <= kRmedSortSpan; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < kRmedSortSpan; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const float a = sv[i], b = sv[l];
                    const short pa = sp[i], pb = sp[l];
                    const bool gt = (a > b) || (a == b && pa > pb);
                    if (gt == up) {
                        sv[i] = b;
                        sv[l] = a;
                        sp[i] = pb;
                        sp[l] = pa;
                    }
                }
            }
            __syncthreads();
        }
    }
    const int t = threadIdx.x;
    if (t0 + t >= N) return;
    int cnt = 0;
    float med = 0.0f;
    for (int k = 0; k < span; ++k) {
        const int q = sp[k];
        if (q >= t && q < t + width && ++cnt == half + 1) {
            med = sv[k];
            break;
        }
    }
    out[offsets[trial] + t0 + t] = med;
}

int launch_running_median(const float* x, const size_t* d_lengths, const size_t* d_offsets,
                          int ntrials, size_t max_len, int width, float* out, cudaStream_t st)
{
    if (width >= 1 && kRmedSortTile + width - 1 <= kRmedSortSpan) {
        dim3 grid((unsigned)((max_len + kRmedSortTile - 1) / kRmedSortTile), (unsigned)ntrials);
        k_running_median_sorted<<<grid, kRmedSortTile, 0, st>>>(x, d_lengths, d_offsets, width, out);
        return check_cuda(cudaGetLastError(), "running_median");
    }
    int tile = 256;
    size_t smem = (tile + width) * sizeof(float);
    if (smem > kFfaSmemBytes)
        return set_error(RT_EINVAL, "running median width %d is larger than supported", width);
    if (smem > 48 * 1024)
        RT_TRY_CUDA(cudaFuncSetAttribute(k_running_median,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)((max_len + tile - 1) / tile), (unsigned)ntrials);
    k_running_median<<<grid, 256, smem, st>>>(x, d_lengths, d_offsets, width, out, tile);
    return check_cuda(cudaGetLastError(), "running_median");
}

// ------------------------------------------------------------------------------------
// Trial periods / fold bins of one transform (periodogram.hpp:190-194)
// ------------------------------------------------------------------------------------
__global__ void k_periods(double* __restrict__ periods, uint32_t* __restrict__ foldbins,
                          size_t rows_eval, double tau, int bins, size_t rows)
{
    for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < rows_eval;
         s += (size_t)gridDim.x * blockDim.x) {
        periods[s] = trial_period(tau, bins, s, rows);
        foldbins[s] = (uint32_t)bins;
    }
}

int launch_periods(double* periods, uint32_t* foldbins, size_t rows_eval, double tau, int bins,
                   size_t rows, cudaStream_t st)
{
    if (rows_eval == 0) return RT_OK;
    k_periods<<<grid_for(rows_eval, 256), 256, 0, st>>>(periods, foldbins, rows_eval, tau, bins,
                                                        rows);
    return check_cuda(cudaGetLastError(), "periods");
}

}  // namespace rt
