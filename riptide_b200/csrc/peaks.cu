// Peak detection on the device (peak_detection.py:38-240 of the reference): the per-segment
// S/N statistics that the dynamic threshold is fitted to, and the selection of the
// periodogram points above that threshold, for every (trial, width) of a batch of
// periodograms at once. The threshold fit itself (a degree-2 polynomial in log f over a few
// hundred control points) and the clustering of the selected points run on the host, in the
// reference's own numpy calls (riptide_b200/peaks.py).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace rt {

constexpr int kSegMaxPoints = 16384;       // points per segment, sorted on chip
constexpr size_t kSegColsSmem = 112 * 1024;  // shared memory of the all-widths segment kernel

// In-place ascending bitonic sort of n (a power of two) values in shared memory. Each
// compare-exchange stage is n/2 independent pairs (i, i + j), i with bit j clear, dealt to
// the threads so that none idles; padding values are +inf.
template <typename T>
__device__ void bitonic_sort(T* a, int n)
{
    const int half = n >> 1;
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int q = threadIdx.x; q < half; q += blockDim.x) {
                const int i = ((q & ~(j - 1)) << 1) | (q & (j - 1));  // a 0 at bit j
                const bool up = (i & k) == 0;
                const T x = a[i], y = a[i + j];
                if ((x > y) == up) {
                    a[i] = y;
                    a[i + j] = x;
                }
            }
            __syncthreads();
        }
    }
}

// numpy's linear interpolation between two order statistics (numpy _lerp) of float64
// values: the reference takes the percentiles of each width's S/N after casting them to
// float64 (peak_detection.py:205), so the difference b - a is a float64 one.
__device__ __forceinline__ double np_lerp(double a, double b, double t)
{
    const double d = __dsub_rn(b, a);
    return (t >= 0.5) ? __dsub_rn(b, __dmul_rn(d, __dsub_rn(1.0, t))) : __dadd_rn(a, __dmul_rn(d, t));
}


struct SegTrial {
    unsigned long long row0;  // first periodogram row of the trial
    int seg0, m, p, pad;      // first global segment, segments, points per segment
};

// One CTA per (segment, width): sc = median + nstd * IQR / 1.349 of the segment's S/N
// (segment_stats, peak_detection.py:38-86), the S/N sorted as float32 (their type). CTAs of
// width 0 also write the segment's median frequency fc (sorted as float64). `n2`: the sort
// size of the launch, a power of two >= every segment's length.
template <typename T>
__device__ __forceinline__ double np_percentile_sorted(const T* a, int n, double q);

// np.percentile(x, q), method 'linear', of n sorted float32 S/N values cast to float64 (their
// order is the same either way)
template <>
__device__ __forceinline__ double np_percentile_sorted<float>(const float* a, int n, double q)
{
    const double v = __dmul_rn((double)(n - 1), q);
    const double prev = floor(v);
    const int i0 = (int)prev;
    const int i1 = min(i0 + 1, n - 1);
    return np_lerp((double)a[i0], (double)a[i1], __dsub_rn(v, prev));
}

__global__ void __launch_bounds__(1024)
    k_peak_segments(const double* __restrict__ periods, const float* __restrict__ snrs, int nw,
                    const SegTrial* __restrict__ trials, int ntrials, double nstd, int n2,
                    double* __restrict__ fc, double* __restrict__ sc)
{
    extern __shared__ double sv[];
    float* vf = reinterpret_cast<float*>(sv);
    const int seg = blockIdx.x, iw = blockIdx.y;
    int lo = 0, hi = ntrials - 1;  // trial of this segment
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (trials[mid].seg0 <= seg) lo = mid;
        else hi = mid - 1;
    }
    const SegTrial T = trials[lo];
    const int j = seg - T.seg0, p = T.p;
    const size_t r0 = T.row0 + (size_t)j * p;
    for (int i = threadIdx.x; i < n2; i += blockDim.x)
        vf[i] = (i < p) ? snrs[(r0 + i) * nw + iw] : INFINITY;
    __syncthreads();
    bitonic_sort(vf, n2);
    if (threadIdx.x == 0) {
        const double s25 = np_percentile_sorted(vf, p, 0.25);
        const double s50 = np_percentile_sorted(vf, p, 0.5);
        const double s75 = np_percentile_sorted(vf, p, 0.75);
        const double sstd = __ddiv_rn(__dsub_rn(s75, s25), 1.349);
        sc[(size_t)seg * nw + iw] = __dadd_rn(s50, __dmul_rn(nstd, sstd));
    }
    if (iw != 0) return;
    __syncthreads();
    for (int i = threadIdx.x; i < n2; i += blockDim.x)
        sv[i] = (i < p) ? __ddiv_rn(1.0, periods[r0 + i]) : INFINITY;
    __syncthreads();
    bitonic_sort(sv, n2);
    if (threadIdx.x == 0)  // np.median: the middle value, or the mean of the middle two
        fc[seg] = (p & 1) ? sv[p / 2] : __ddiv_rn(__dadd_rn(sv[p / 2 - 1], sv[p / 2]), 2.0);
}

// In-place ascending bitonic sorts of `ncols` columns of n values each (column c at a + c*n),
// all columns advancing through the same network together: more independent
// compare-exchanges per thread and per barrier than one column at a time.
template <typename T>
__device__ void bitonic_sort_cols(T* a, int n, int ncols)
{
    const int half = n >> 1;
    int lh = 0;
    while ((1 << lh) < half) ++lh;
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int q = threadIdx.x; q < ncols * half; q += blockDim.x) {
                const int col = q >> lh, qq = q & (half - 1);
                const int i = ((qq & ~(j - 1)) << 1) | (qq & (j - 1));
                T* c = a + (size_t)col * n;
                const bool up = (i & k) == 0;
                const T x = c[i], y = c[i + j];
                if ((x > y) == up) {
                    c[i] = y;
                    c[i + j] = x;
                }
            }
            __syncthreads();
        }
    }
}

// One CTA per segment for every width at once: the segment's nw S/N columns sorted together
// (float32), then its frequencies (float64); the same statistics as k_peak_segments.
__global__ void __launch_bounds__(512)
    k_peak_segments_cols(const double* __restrict__ periods, const float* __restrict__ snrs,
                         int nw, const SegTrial* __restrict__ trials, int ntrials, double nstd,
                         int n2, double* __restrict__ fc, double* __restrict__ sc)
{
    extern __shared__ double sv[];                        // n2 frequencies
    float* vf = reinterpret_cast<float*>(sv + n2);        // nw columns of n2 S/N values
    const int seg = blockIdx.x;
    int lo = 0, hi = ntrials - 1;  // trial of this segment
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (trials[mid].seg0 <= seg) lo = mid;
        else hi = mid - 1;
    }
    const SegTrial T = trials[lo];
    const int j = seg - T.seg0, p = T.p;
    const size_t r0 = T.row0 + (size_t)j * p;
    for (int e = threadIdx.x; e < nw * n2; e += blockDim.x) {
        const int i = e / nw, iw = e - i * nw;  // row-major reads of the periodogram
        if (i < n2) vf[(size_t)iw * n2 + i] = (i < p) ? snrs[(r0 + i) * nw + iw] : INFINITY;
    }
    for (int i = threadIdx.x; i < n2; i += blockDim.x)
        sv[i] = (i < p) ? __ddiv_rn(1.0, periods[r0 + i]) : INFINITY;
    __syncthreads();
    bitonic_sort_cols(vf, n2, nw);
    bitonic_sort_cols(sv, n2, 1);
    for (int iw = threadIdx.x; iw < nw; iw += blockDim.x) {
        const float* c = vf + (size_t)iw * n2;
        const double s25 = np_percentile_sorted(c, p, 0.25);
        const double s50 = np_percentile_sorted(c, p, 0.5);
        const double s75 = np_percentile_sorted(c, p, 0.75);
        const double sstd = __ddiv_rn(__dsub_rn(s75, s25), 1.349);
        sc[(size_t)seg * nw + iw] = __dadd_rn(s50, __dmul_rn(nstd, sstd));
    }
    if (threadIdx.x == 0)  // np.median: the middle value, or the mean of the middle two
        fc[seg] = (p & 1) ? sv[p / 2] : __ddiv_rn(__dadd_rn(sv[p / 2 - 1], sv[p / 2]), 2.0);
}

// First and last period of every trial's periodogram (the segment layout's frequency span).
__global__ void k_period_ends(const double* __restrict__ periods,
                              const unsigned long long* __restrict__ row_offsets, int ntrials,
                              double* __restrict__ ends)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntrials) return;
    ends[2 * t] = periods[row_offsets[t]];
    ends[2 * t + 1] = periods[row_offsets[t + 1] - 1];
}

// Points above the dynamic threshold poly(log f) and above smin (find_peaks_single,
// peak_detection.py:112-146), as (row * nw + iw), in any order.
__global__ void k_peak_select(const double* __restrict__ periods, const float* __restrict__ snrs,
                              int nw, const unsigned long long* __restrict__ row_trial_end,
                              int ntrials, const double* __restrict__ coef, int ncoef,
                              double smin, unsigned long long rows,
                              unsigned long long* __restrict__ sel, unsigned long long cap,
                              unsigned long long* __restrict__ count)
{
    for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         e < rows * nw; e += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long r = e / nw;
        const int iw = (int)(e - r * nw);
        const double s = (double)snrs[e];
        if (!(s > smin)) continue;
        int lo = 0, hi = ntrials - 1;  // first trial whose end is beyond r
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (row_trial_end[mid] > r) hi = mid;
            else lo = mid + 1;
        }
        const double x = log(__ddiv_rn(1.0, periods[r]));
        const double* c = coef + ((size_t)lo * nw + iw) * ncoef;
        double y = 0.0;  // np.polyval: y = y * x + c_k, no fused multiply-add
        for (int k = 0; k < ncoef; ++k) y = __dadd_rn(__dmul_rn(y, x), c[k]);
        if (s > y) {
            const unsigned long long slot = atomicAdd(count, 1ull);
            if (slot < cap) sel[slot] = e;
        }
    }
}

}  // namespace rt

using namespace rt;

extern "C" int rt_peak_segments(const double* d_periods, const float* d_snrs, size_t num_widths,
                                const uint64_t* h_row_offsets, size_t ntrials,
                                const double* h_tobs, double segwidth, double nstd,
                                uint64_t* h_seg_offsets, double* d_fc, double* d_sc, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_periods || !h_row_offsets || !h_tobs || !h_seg_offsets)
        return set_error(RT_EINVAL, "null argument");
    if (num_widths == 0 || num_widths > 65535) return set_error(RT_EINVAL, "bad number of widths");
    // segment layout of every trial: m = ceil(|f[-1] - f[0]| / w), p = rows // m; the first
    // and last period of every trial gathered on the device and copied back at once
    if (ntrials == 0) return set_error(RT_EINVAL, "no periodograms");
    for (size_t t = 0; t < ntrials; ++t)
        if (h_row_offsets[t + 1] <= h_row_offsets[t])
            return set_error(RT_EINVAL, "periodogram %zu is empty", t);
    std::vector<double> ends(2 * ntrials);
    {
        unsigned long long* d_ro = nullptr;
        double* d_ends = nullptr;
        const size_t ro_bytes = (ntrials + 1) * sizeof(uint64_t);
        const size_t ro_room = (ro_bytes + 15) & ~size_t(15);
        RT_TRY_CUDA(cudaMallocAsync((void**)&d_ro, ro_room + 2 * ntrials * sizeof(double), st));
        d_ends = reinterpret_cast<double*>(reinterpret_cast<char*>(d_ro) + ro_room);
        cudaError_t e = cudaMemcpyAsync(d_ro, h_row_offsets, ro_bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_period_ends<<<(unsigned)((ntrials + 255) / 256), 256, 0, st>>>(d_periods, d_ro,
                                                                            (int)ntrials, d_ends);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ends.data(), d_ends, 2 * ntrials * sizeof(double),
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFreeAsync(d_ro, st);
        if (e != cudaSuccess) return check_cuda(e, "peak_segments layout");
    }
    std::vector<SegTrial> tr(ntrials);
    uint64_t seg = 0, pmax = 1;
    h_seg_offsets[0] = 0;
    for (size_t t = 0; t < ntrials; ++t) {
        const double w = segwidth / h_tobs[t];
        const double span = std::fabs(1.0 / ends[2 * t + 1] - 1.0 / ends[2 * t]);
        const double mf = std::ceil(span / w);
        if (!(mf >= 1.0) || !std::isfinite(mf))
            return set_error(RT_EINVAL, "periodogram %zu spans no frequency segment", t);
        const uint64_t rows = h_row_offsets[t + 1] - h_row_offsets[t];
        const uint64_t m = (uint64_t)mf;
        const uint64_t p = rows / m;
        if (p == 0) return set_error(RT_EINVAL, "periodogram %zu has fewer rows than segments", t);
        if (p > (uint64_t)kSegMaxPoints)
            return set_error(RT_EINVAL, "segments of %llu points exceed the device limit (%d)",
                             (unsigned long long)p, kSegMaxPoints);
        pmax = std::max(pmax, p);
        tr[t].row0 = h_row_offsets[t];
        tr[t].seg0 = (int)seg;
        tr[t].m = (int)m;
        tr[t].p = (int)p;
        tr[t].pad = 0;
        seg += m;
        h_seg_offsets[t + 1] = seg;
    }
    if (!d_fc || !d_sc) return RT_OK;  // layout only
    if (!d_snrs) return set_error(RT_EINVAL, "null argument");
    if (seg >= (1ull << 31)) return set_error(RT_EINVAL, "too many segments");
    SegTrial* d_tr = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_tr, ntrials * sizeof(SegTrial), st));
    int s = check_cuda(cudaMemcpyAsync(d_tr, tr.data(), ntrials * sizeof(SegTrial),
                                       cudaMemcpyHostToDevice, st), "peak_segments");
    int n2 = 2;
    while ((uint64_t)n2 < pmax) n2 <<= 1;
    const int threads = std::max(32, std::min(1024, n2 / 2));
    const size_t smem = (size_t)n2 * sizeof(double);
    if (s == RT_OK && smem > 48 * 1024)
        s = check_cuda(cudaFuncSetAttribute(k_peak_segments,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(kSegMaxPoints * sizeof(double))),
                       "peak_segments");
    // all widths of a segment in one CTA when they fit two CTAs per SM's shared memory
    const size_t smem_cols = (size_t)n2 * (sizeof(double) + num_widths * sizeof(float));
    if (s == RT_OK && seg > 0 && smem_cols <= kSegColsSmem) {
        if (smem_cols > 48 * 1024)
            s = check_cuda(cudaFuncSetAttribute(k_peak_segments_cols,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)kSegColsSmem),
                           "peak_segments");
        if (s == RT_OK) {
            const int tc = (int)std::max<size_t>(
                32, std::min<size_t>(512, (num_widths * (size_t)n2 / 2 + 31) / 32 * 32));
            k_peak_segments_cols<<<(unsigned)seg, tc, smem_cols, st>>>(
                d_periods, d_snrs, (int)num_widths, d_tr, (int)ntrials, nstd, n2, d_fc, d_sc);
            s = check_cuda(cudaGetLastError(), "peak_segments");
        }
    } else if (s == RT_OK && seg > 0) {
        dim3 grid((unsigned)seg, (unsigned)num_widths);
        k_peak_segments<<<grid, threads, smem, st>>>(d_periods, d_snrs, (int)num_widths, d_tr,
                                                     (int)ntrials, nstd, n2, d_fc, d_sc);
        s = check_cuda(cudaGetLastError(), "peak_segments");
    }
    cudaFreeAsync(d_tr, st);
    return s;
}

extern "C" int rt_peak_select(const double* d_periods, const float* d_snrs, size_t num_widths,
                              const uint64_t* h_row_offsets, size_t ntrials, const double* d_coef,
                              size_t num_coef, double smin, uint64_t* d_sel, size_t capacity,
                              size_t* h_count, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!d_periods || !d_snrs || !h_row_offsets || !d_coef || !d_sel || !h_count)
        return set_error(RT_EINVAL, "null argument");
    if (num_coef == 0 || num_widths == 0) return set_error(RT_EINVAL, "bad coefficient count");
    const uint64_t rows = h_row_offsets[ntrials];
    unsigned long long* d_aux = nullptr;  // [ntrials] trial row ends, then the counter
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_aux, (ntrials + 1) * sizeof(unsigned long long), st));
    int s = check_cuda(cudaMemcpyAsync(d_aux, h_row_offsets + 1, ntrials * sizeof(uint64_t),
                                       cudaMemcpyHostToDevice, st), "peak_select");
    if (s == RT_OK)
        s = check_cuda(cudaMemsetAsync(d_aux + ntrials, 0, sizeof(unsigned long long), st), "peak_select");
    if (s == RT_OK && rows > 0) {
        const size_t work = (size_t)rows * num_widths;
        const int grid = (int)std::min<size_t>((work + 255) / 256, 148 * 32);
        k_peak_select<<<grid, 256, 0, st>>>(d_periods, d_snrs, (int)num_widths, d_aux,
                                            (int)ntrials, d_coef, (int)num_coef, smin, rows,
                                            (unsigned long long*)d_sel, capacity, d_aux + ntrials);
        s = check_cuda(cudaGetLastError(), "peak_select");
    }
    unsigned long long count = 0;
    if (s == RT_OK)
        s = check_cuda(cudaMemcpyAsync(&count, d_aux + ntrials, sizeof(count),
                                       cudaMemcpyDeviceToHost, st), "peak_select");
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "peak_select");
    cudaFreeAsync(d_aux, st);
    if (s != RT_OK) return s;
    *h_count = (size_t)count;
    if (count > capacity)
        return set_error(RT_EINVAL, "%llu points pass the threshold (capacity %zu)", count, capacity);
    return RT_OK;
}
