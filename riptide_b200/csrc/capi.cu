// C ABI entry points: drop-ins for the reference's riptide.libcpp functions
// (cpp/python_bindings.cpp) on device buffers.
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "snr_core.cuh"

using namespace rt;

extern "C" const char* rt_last_error(void) { return rt::last_error(); }
extern "C" int rt_version(void) { return 100; }

extern "C" int rt_rollback(const float* d_x, size_t size, size_t shift, float* d_out,
                           void* stream)
{
    return rt::rollback(d_x, size, shift, d_out, (cudaStream_t)stream);
}

extern "C" int rt_fused_rollback_add(const float* d_x, const float* d_y, size_t size,
                                     size_t shift, float* d_out, void* stream)
{
    return rt::fused_rollback_add(d_x, d_y, size, shift, d_out, (cudaStream_t)stream);
}

extern "C" int rt_circular_prefix_sum(const float* d_x, size_t size, size_t nsum, float* d_out,
                                      void* stream)
{
    return rt::circular_prefix_sum(d_x, size, nsum, d_out, (cudaStream_t)stream);
}

// ------------------------------------------------------------------------------------
// ffa2
// ------------------------------------------------------------------------------------
static int ffa2_impl(const float* d_in, size_t rows, size_t cols, float* d_out, cudaStream_t st,
                     bool sync)
{
    if (rows == 0 || cols == 0) return RT_OK;
    if (rows >= (1u << 24) || cols > 4096)
        return set_error(RT_EINVAL, "ffa2 input of %zu x %zu is larger than supported", rows, cols);
    const int m = (int)rows, b = (int)cols;
    float* scratch = nullptr;
    int* d_err = nullptr;
    const size_t sf = ffa_scratch_floats(m, b);
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_err, sizeof(int), st));
    RT_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    if (sf) {
        cudaError_t e = cudaMallocAsync((void**)&scratch, sf * sizeof(float), st);
        if (e != cudaSuccess) {
            cudaFreeAsync(d_err, st);
            return check_cuda(e, "ffa2 scratch");
        }
    }
    int s = ffa_transform(d_in, m, b, m, d_out, scratch, d_err, st);
    int herr = 0;
    if (s == RT_OK) {
        cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    if (scratch) cudaFreeAsync(scratch, st);
    cudaFreeAsync(d_err, st);
    if (s != RT_OK) return s;
    (void)sync;
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) return set_error(RT_EINTERNAL, "ffa2 device plan check failed (%d)", herr);
    return RT_OK;
}

extern "C" int rt_ffa2(const float* d_in, size_t rows, size_t cols, float* d_out, void* stream)
{
    return ffa2_impl(d_in, rows, cols, d_out, (cudaStream_t)stream, true);
}

extern "C" int rt_benchmark_ffa2(size_t rows, size_t cols, size_t loops, double* h_seconds)
{
    if (!h_seconds) return set_error(RT_EINVAL, "null argument");
    if (rows == 0 || cols == 0 || loops == 0) {
        *h_seconds = 0.0;
        return RT_OK;
    }
    const int m = (int)rows, b = (int)cols;
    float *in = nullptr, *out = nullptr, *scratch = nullptr;
    int* d_err = nullptr;
    const size_t n = rows * cols, sf = ffa_scratch_floats(m, b);
    RT_TRY_CUDA(cudaMalloc((void**)&in, n * sizeof(float)));
    RT_TRY_CUDA(cudaMalloc((void**)&out, n * sizeof(float)));
    RT_TRY_CUDA(cudaMalloc((void**)&d_err, sizeof(int)));
    if (sf) RT_TRY_CUDA(cudaMalloc((void**)&scratch, sf * sizeof(float)));
    RT_TRY_CUDA(cudaMemset(in, 0, n * sizeof(float)));
    RT_TRY_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int s = ffa_transform(in, m, b, m, out, scratch, d_err, 0);  // warm-up
    cudaEventRecord(e0, 0);
    for (size_t i = 0; i < loops && s == RT_OK; ++i) s = ffa_transform(in, m, b, m, out, scratch, d_err, 0);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(in);
    cudaFree(out);
    cudaFree(d_err);
    if (scratch) cudaFree(scratch);
    if (s != RT_OK) return s;
    *h_seconds = (double)ms * 1e-3 / (double)loops;
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// snr2
// ------------------------------------------------------------------------------------
static int check_widths(const uint64_t* w, size_t nw, size_t bins, std::vector<int>& out)
{
    out.clear();
    for (size_t i = 0; i < nw; ++i) {
        // snr.hpp:21-31
        if (!((w[i] > 0) & (w[i] < bins)))
            return set_error(RT_EINVAL, "trial widths must be all > 0 and < columns");
        out.push_back((int)w[i]);
    }
    if (nw > (size_t)kMaxWidths)
        return set_error(RT_EINVAL, "at most %d trial widths are supported", kMaxWidths);
    return RT_OK;
}

extern "C" int rt_snr2(const float* d_in, size_t rows, size_t cols, const uint64_t* h_widths,
                       size_t num_widths, float stdnoise, float* d_out, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!(stdnoise > 0)) return set_error(RT_EINVAL, "stdnoise must be > 0");  // snr.hpp:14-18
    std::vector<int> w;
    RT_TRY(check_widths(h_widths, num_widths, cols, w));
    if (rows == 0 || num_widths == 0) return RT_OK;
    if (cols > 4096) return set_error(RT_EINVAL, "profiles longer than 4096 bins are not supported");
    int* d_w = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_w, w.size() * sizeof(int), st));
    cudaMemcpyAsync(d_w, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    int s = rt::snr2(d_in, rows, cols, d_w, w.data(), (int)w.size(), stdnoise, d_out, st);
    cudaFreeAsync(d_w, st);
    if (s != RT_OK) return s;
    RT_TRY_CUDA(cudaStreamSynchronize(st));  // h_widths staging must outlive the copy
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// downsample
// ------------------------------------------------------------------------------------
extern "C" size_t rt_downsampled_size(size_t size, double f) { return downsampled_size(size, f); }

static int downsample_one(const float* d_in, size_t size, double f, float* d_out, cudaStream_t st)
{
    // device-side descriptor arrays for one series, one factor
    struct Hdr {
        size_t in_off, len, out_off;
        double f;
        int use_seg;
    };
    Hdr h{0, size, 0, f, ds_use_segments(f) ? 1 : 0};
    unsigned char* d = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d, sizeof(Hdr), st));
    RT_TRY_CUDA(cudaMemcpyAsync(d, &h, sizeof(Hdr), cudaMemcpyHostToDevice, st));
    Hdr* dh = reinterpret_cast<Hdr*>(d);
    DsJob job;
    job.in = d_in;
    job.in_off = &dh->in_off;
    job.lengths = &dh->len;
    job.mean = nullptr;
    job.norm = nullptr;
    job.norm_out = nullptr;
    job.f = &dh->f;
    job.use_seg = &dh->use_seg;
    job.out = d_out;
    job.out_off = &dh->out_off;
    job.ncycles = 1;
    const int use_seg = h.use_seg, skip = 0;
    job.use_seg_host = &use_seg;
    job.f_host = &f;
    job.skip_host = &skip;
    int s = launch_downsample(job, 1, size, st);
    cudaFreeAsync(d, st);
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "downsample");
    return s;
}

extern "C" int rt_downsample(const float* d_in, size_t size, double f, float* d_out,
                             void* stream)
{
    // downsample.hpp:11-16
    if (!((f > 1.0) & (f <= (double)size)))
        return set_error(RT_EINVAL, "Downsampling factor must verify: 1 < f <= size");
    return downsample_one(d_in, size, f, d_out, (cudaStream_t)stream);
}

// ------------------------------------------------------------------------------------
// running median
// ------------------------------------------------------------------------------------
extern "C" int rt_running_median(const float* d_in, size_t size, size_t width, float* d_out,
                                 void* stream)
{
    // running_median.hpp:103-107
    if (!(width % 2)) return set_error(RT_EINVAL, "width must be an odd number");
    if (!(width < size)) return set_error(RT_EINVAL, "width must be < size");
    cudaStream_t st = (cudaStream_t)stream;
    size_t* d = nullptr;
    const size_t hv[2] = {size, 0};
    RT_TRY_CUDA(cudaMallocAsync((void**)&d, sizeof(hv), st));
    RT_TRY_CUDA(cudaMemcpyAsync(d, hv, sizeof(hv), cudaMemcpyHostToDevice, st));
    int s = launch_running_median(d_in, d, d + 1, 1, size, (int)width, d_out, st);
    cudaFreeAsync(d, st);
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "running_median");
    return s;
}

// ------------------------------------------------------------------------------------
// periodogram
// ------------------------------------------------------------------------------------
extern "C" int rt_periodogram_length(size_t size, double tsamp, double period_min,
                                     double period_max, size_t bins_min, size_t bins_max,
                                     size_t* h_length)
{
    if (!h_length) return set_error(RT_EINVAL, "null argument");
    if (!(tsamp > 0)) return set_error(RT_EINVAL, "tsamp must be > 0");
    if (!(period_min > 0)) return set_error(RT_EINVAL, "period_min must be > 0");
    if (!(period_max > period_min)) return set_error(RT_EINVAL, "period_max must be > period_min");
    if (!(bins_min > 1)) return set_error(RT_EINVAL, "bins_min must be > 1");
    if (!(bins_max >= bins_min)) return set_error(RT_EINVAL, "bins_max must be >= bins_min");
    if (!(period_min >= tsamp * bins_min))
        return set_error(RT_EINVAL, "Must have: period_min >= tsamp * bins_min ");
    const double ds_ini = period_min / (tsamp * bins_min);
    const double ds_geo = (bins_max + 1.0) / bins_min;
    const size_t nds = (size_t)ceil(log(period_max / period_min) / log(ds_geo));
    size_t len = 0;
    for (size_t ids = 0; ids < nds; ++ids) {
        const double f = ds_ini * pow(ds_geo, (double)ids);
        const double tau = f * tsamp;
        const double pms = period_max / tau;
        const size_t n = downsampled_size(size, f);
        const size_t bstop = std::min({bins_max, n, (size_t)pms});
        for (size_t b = bins_min; b <= bstop; ++b) len += rows_to_evaluate(n / b, b, pms);
    }
    *h_length = len;
    return RT_OK;
}

extern "C" int rt_search_plan_create(const uint64_t*, size_t, const rt_search_config*,
                                     const uint64_t*, size_t, rt_search_plan**);
extern "C" int rt_search_run(rt_search_plan*, const float*, float*, double*, uint32_t*, float*,
                             void*);
extern "C" int rt_search_check(rt_search_plan*, void*);
extern "C" void rt_search_plan_destroy(rt_search_plan*);

// Plans of the single-series periodogram, cached by geometry (a series length and search
// parameters reused across calls is the common case: all DM trials of one observation).
namespace {
struct PgKey {
    size_t size;
    double tsamp, pmin, pmax;
    size_t bmin, bmax;
    std::vector<uint64_t> widths;
    bool operator<(const PgKey& o) const
    {
        return std::tie(size, tsamp, pmin, pmax, bmin, bmax, widths) <
               std::tie(o.size, o.tsamp, o.pmin, o.pmax, o.bmin, o.bmax, o.widths);
    }
};
std::mutex g_pg_mutex;
std::map<PgKey, rt_search_plan*> g_pg_cache;
}  // namespace

extern "C" int rt_periodogram(const float* d_data, size_t size, double tsamp,
                              const uint64_t* h_widths, size_t num_widths, double period_min,
                              double period_max, size_t bins_min, size_t bins_max,
                              double* d_periods, uint32_t* d_foldbins, float* d_snrs,
                              void* stream)
{
    size_t L = 0;
    RT_TRY(rt_periodogram_length(size, tsamp, period_min, period_max, bins_min, bins_max, &L));
    if (L == 0) return RT_OK;
    std::lock_guard<std::mutex> lock(g_pg_mutex);
    PgKey key{size, tsamp, period_min, period_max, bins_min, bins_max,
              std::vector<uint64_t>(h_widths, h_widths + num_widths)};
    rt_search_plan* plan = nullptr;
    auto it = g_pg_cache.find(key);
    if (it != g_pg_cache.end()) {
        plan = it->second;
    } else {
        rt_search_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.tsamp = tsamp;
        cfg.period_min = period_min;
        cfg.period_max = period_max;
        cfg.bins_min = bins_min;
        cfg.bins_max = bins_max;
        cfg.deredden = 0;
        cfg.already_normalised = 1;
        const uint64_t len = size;
        RT_TRY(rt_search_plan_create(&len, 1, &cfg, h_widths, num_widths, &plan));
        if (g_pg_cache.size() >= 8) {
            rt_search_plan_destroy(g_pg_cache.begin()->second);
            g_pg_cache.erase(g_pg_cache.begin());
        }
        g_pg_cache[key] = plan;
    }
    RT_TRY(rt_search_run(plan, d_data, nullptr, d_periods, d_foldbins, d_snrs, stream));
    return rt_search_check(plan, stream);
}

extern "C" int rt_periodogram_plain(const float* d_data, size_t size, double tsamp,
                                    const uint64_t* h_widths, size_t num_widths,
                                    double period_min, double period_max, size_t bins_min,
                                    size_t bins_max, double* d_periods, uint32_t* d_foldbins,
                                    float* d_snrs, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    size_t L = 0;
    RT_TRY(rt_periodogram_length(size, tsamp, period_min, period_max, bins_min, bins_max, &L));
    std::vector<int> w;
    RT_TRY(check_widths(h_widths, num_widths, bins_min, w));
    if (L == 0) return RT_OK;
    const double ds_ini = period_min / (tsamp * bins_min);
    const double ds_geo = (bins_max + 1.0) / bins_min;
    const size_t nds = (size_t)ceil(log(period_max / period_min) / log(ds_geo));
    const size_t bufsize = downsampled_size(size, ds_ini);
    float *input = nullptr, *ffaout = nullptr, *scratch = nullptr;
    int *d_w = nullptr, *d_err = nullptr;
    size_t scratch_floats = 0;
    for (size_t b = bins_min; b <= bins_max && b <= bufsize; ++b)
        scratch_floats = std::max(scratch_floats, ffa_scratch_floats((int)(bufsize / b), (int)b));
    RT_TRY_CUDA(cudaMallocAsync((void**)&input, std::max<size_t>(bufsize, 1) * sizeof(float), st));
    RT_TRY_CUDA(cudaMallocAsync((void**)&ffaout, std::max<size_t>(bufsize, 1) * sizeof(float), st));
    RT_TRY_CUDA(cudaMallocAsync((void**)&scratch, std::max<size_t>(scratch_floats, 1) * sizeof(float), st));
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_w, w.size() * sizeof(int), st));
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_err, sizeof(int), st));
    RT_TRY_CUDA(cudaMemcpyAsync(d_w, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    RT_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    int s = RT_OK;
    double* periods = d_periods;
    uint32_t* foldbins = d_foldbins;
    float* snr = d_snrs;
    for (size_t ids = 0; ids < nds && s == RT_OK; ++ids) {
        const double f = ds_ini * pow(ds_geo, (double)ids);
        const double tau = f * tsamp;
        const double pms = period_max / tau;
        const size_t n = downsampled_size(size, f);
        const float* in = d_data;
        if (f != 1) {
            if (!((f > 1.0) & (f <= (double)size))) {
                s = set_error(RT_EINVAL, "Downsampling factor must verify: 1 < f <= size");
                break;
            }
            s = downsample_one(d_data, size, f, input, st);
            in = input;
        }
        const size_t bstop = std::min({bins_max, n, (size_t)pms});
        for (size_t b = bins_min; b <= bstop && s == RT_OK; ++b) {
            const size_t rows = n / b;
            const float stdnoise = (float)sqrt((double)rows * downsampled_variance(size, f));
            const size_t re = rows_to_evaluate(rows, b, pms);
            if (re == 0) continue;
            s = ffa_transform(in, (int)rows, (int)b, (int)rows, ffaout, scratch, d_err, st);
            if (s != RT_OK) break;
            s = rt::snr2(ffaout, re, b, d_w, w.data(), (int)w.size(), stdnoise, snr, st);
            if (s != RT_OK) break;
            s = launch_periods(periods, foldbins, re, tau, (int)b, rows, st);
            snr += re * w.size();
            periods += re;
            foldbins += re;
        }
    }
    int herr = 0;
    cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(input, st);
    cudaFreeAsync(ffaout, st);
    cudaFreeAsync(scratch, st);
    cudaFreeAsync(d_w, st);
    cudaFreeAsync(d_err, st);
    if (s != RT_OK) return s;
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) return set_error(RT_EINTERNAL, "FFA device plan check failed (%d)", herr);
    return RT_OK;
}
