// Folding of a time series at trial periods (TimeSeries.fold / folding.py:21-85 of the
// reference), for one period or a batch of candidates of the same series.
//
// The reference downsamples the series by tbin / tsamp (tbin = period / bins), reshapes the
// first m * bins samples to (m, bins), multiplies by (m * factor)^-1/2 in float32, and either
// sums the rows (subints = 1, or m = 1), returns the rows (subints = None or m), or downsamples
// each phase column by m / subints (downsample_vertical, folding.py:6-18). Here one thread
// computes one output value: the downsampled samples it needs are formed straight from the raw
// series (FP64 sum of the window, rounded once, as rt_downsample forms them), scaled, and then
// summed or column-downsampled in the reference's order, so no downsampled copy of the series
// is written.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace rt {

enum FoldMode : int { kFoldSum = 0, kFoldRows = 1, kFoldColumns = 2 };

struct FoldJob {
    double f;          // time downsampling factor tbin / tsamp
    double vf;         // column downsampling factor m / subints (kFoldColumns)
    size_t out_off;    // first output value
    int bins, m;       // phase bins, rows of the folded block
    int rows;          // output rows (1 for kFoldSum)
    int mode;
    float scale;       // float32((m * factor) ** -0.5)
    int pad;
};

struct FoldShape {
    int mode;
    size_t m, rows;
    double f, vf;
    float scale;
};

// Sample k of the series downsampled by f (downsample.hpp:44-82): the window sum in FP64,
// rounded once to float32.
__device__ __forceinline__ float ds_value(const float* __restrict__ x, size_t N, double f, size_t k)
{
    const double start = (double)k * f;
    const double end = start + f;
    const size_t imin = (size_t)floor(start);
    const double fe = floor(end);
    const size_t imax = (size_t)(fe < (double)N - 1.0 ? fe : (double)N - 1.0);
    double acc = 0.0;
    for (size_t i = imin + 1; i < imax; ++i) acc += (double)__ldg(x + i);
    const float wmin = __double2float_rn((double)(imin + 1) - start);
    const float wmax = __double2float_rn(end - (double)imax);
    return __double2float_rn((double)wmin * __ldg(x + imin) + acc + (double)wmax * __ldg(x + imax));
}

// Folded value (row i, phase j): downsampled sample i * bins + j times the float32 scale.
__device__ __forceinline__ float folded(const float* x, size_t N, const FoldJob& J, size_t i, int j)
{
    return __fmul_rn(ds_value(x, N, J.f, i * (size_t)J.bins + j), J.scale);
}

__global__ void k_fold(const float* __restrict__ x, size_t N, const FoldJob* __restrict__ jobs,
                       float* __restrict__ out)
{
    const FoldJob J = jobs[blockIdx.y];
    const size_t total = (size_t)J.rows * J.bins;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < total;
         o += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(o % J.bins);
        const size_t r = o / J.bins;
        float v;
        if (J.mode == kFoldRows) {
            v = folded(x, N, J, r, j);
        } else if (J.mode == kFoldSum) {
            // numpy's sum over axis 0: the rows accumulated in order in float32
            v = J.m > 0 ? folded(x, N, J, 0, j) : 0.0f;
            for (int i = 1; i < J.m; ++i) v = __fadd_rn(v, folded(x, N, J, i, j));
        } else {
            // column j downsampled by vf (downsample_vertical): window sum in FP64, rounded once
            const double start = (double)r * J.vf;
            const double end = start + J.vf;
            const size_t imin = (size_t)floor(start);
            const double fe = floor(end);
            const size_t imax = (size_t)(fe < (double)J.m - 1.0 ? fe : (double)J.m - 1.0);
            double acc = 0.0;
            for (size_t i = imin + 1; i < imax; ++i) acc += (double)folded(x, N, J, i, j);
            const float wmin = __double2float_rn((double)(imin + 1) - start);
            const float wmax = __double2float_rn(end - (double)imax);
            v = __double2float_rn((double)wmin * folded(x, N, J, imin, j) + acc +
                                  (double)wmax * folded(x, N, J, imax, j));
        }
        out[J.out_off + o] = v;
    }
}

// The reference's argument checks and output shape (folding.py:21-85; TimeSeries.downsample
// checks the factor, downsample.hpp:11-19; downsample_vertical checks its factor, :7-14).
// subints < 0 stands for None.
static int fold_shape(size_t size, double tsamp, double period, size_t bins, long long subints,
                      FoldShape& s)
{
    if (!(tsamp > 0)) return set_error(RT_EINVAL, "tsamp must be > 0");
    if (bins < 1) return set_error(RT_EINVAL, "bins must be >= 1");
    const double length = (double)size * tsamp;
    if (period > length) return set_error(RT_EINVAL, "Period exceeds data length");
    const double tbin = period / (double)bins;
    if (!(tbin > tsamp)) return set_error(RT_EINVAL, "Bin width is shorter than sampling time");
    if (subints == 0) return set_error(RT_EINVAL, "subints must be >= 1 or None");
    if (subints > 0) {
        const double full_periods = length / period;
        if ((double)subints > full_periods)
            return set_error(RT_EINVAL,
                             "subints (%lld) exceeds the number of signal periods that fit in the data (%g)",
                             subints, full_periods);
    }
    const double f = tbin / tsamp;
    if (!(f > 1.0) || f > (double)size)
        return set_error(RT_EINVAL, "Downsampling factor must be > 1 and <= input size");
    const size_t n = downsampled_size(size, f);
    const size_t m = n / bins;
    if (m == 0) return set_error(RT_EINVAL, "the downsampled series holds no full period");
    s.f = f;
    s.m = m;
    s.vf = 0.0;
    s.scale = (float)std::pow((double)m * f, -0.5);
    if (subints == 1 || m == 1) {
        s.mode = kFoldSum;
        s.rows = 1;
    } else if (subints < 0 || (size_t)subints == m) {
        s.mode = kFoldRows;
        s.rows = m;
    } else {
        const double vf = (double)m / (double)subints;
        if (!(vf > 1.0)) return set_error(RT_EINVAL, "factor must be > 1");
        if (!(vf < (double)m))
            return set_error(RT_EINVAL, "factor must be strictly smaller than the number of input lines");
        s.mode = kFoldColumns;
        s.vf = vf;
        s.rows = downsampled_size(m, vf);
    }
    if (m > (size_t)INT32_MAX || bins > (size_t)INT32_MAX)
        return set_error(RT_EINVAL, "fold too large");
    return RT_OK;
}

}  // namespace rt

using namespace rt;

extern "C" int rt_fold_shape(size_t size, double tsamp, double period, size_t bins,
                             long long subints, size_t* rows, int* ndim)
{
    FoldShape s;
    RT_TRY(fold_shape(size, tsamp, period, bins, subints, s));
    if (rows) *rows = s.rows;
    if (ndim) *ndim = s.mode == kFoldSum ? 1 : 2;
    return RT_OK;
}

extern "C" int rt_fold_batched(const float* d_in, size_t size, double tsamp,
                               const double* h_periods, const size_t* h_bins,
                               const long long* h_subints, size_t count,
                               const uint64_t* h_out_offsets, float* d_out, void* stream_)
{
    cudaStream_t stream = (cudaStream_t)stream_;
    if (count == 0) return RT_OK;
    if (!d_in || !d_out || !h_periods || !h_bins || !h_subints || !h_out_offsets)
        return set_error(RT_EINVAL, "null argument");
    if (count > 65535) return set_error(RT_EINVAL, "at most 65535 folds per call");
    std::vector<FoldJob> jobs(count);
    size_t most = 0;
    for (size_t c = 0; c < count; ++c) {
        FoldShape s;
        RT_TRY(fold_shape(size, tsamp, h_periods[c], h_bins[c], h_subints[c], s));
        FoldJob& J = jobs[c];
        J.f = s.f;
        J.vf = s.vf;
        J.out_off = h_out_offsets[c];
        J.bins = (int)h_bins[c];
        J.m = (int)s.m;
        J.rows = (int)s.rows;
        J.mode = s.mode;
        J.scale = s.scale;
        J.pad = 0;
        most = std::max(most, s.rows * h_bins[c]);
    }
    if (most == 0) return RT_OK;
    FoldJob* d_jobs = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_jobs, count * sizeof(FoldJob), stream));
    cudaError_t e = cudaMemcpyAsync(d_jobs, jobs.data(), count * sizeof(FoldJob),
                                    cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        const int threads = 128;
        const size_t bx = std::min<size_t>((most + threads - 1) / threads, 4096);
        k_fold<<<dim3((unsigned)bx, (unsigned)count), threads, 0, stream>>>(d_in, size, d_jobs, d_out);
        e = cudaGetLastError();
    }
    // a copy from pageable memory has read `jobs` when cudaMemcpyAsync returns
    cudaFreeAsync(d_jobs, stream);
    if (e != cudaSuccess) return check_cuda(e, "k_fold");
    return RT_OK;
}

extern "C" int rt_fold(const float* d_in, size_t size, double tsamp, double period, size_t bins,
                       long long subints, float* d_out, void* stream)
{
    const uint64_t off = 0;
    return rt_fold_batched(d_in, size, tsamp, &period, &bins, &subints, 1, &off, d_out, stream);
}
