// Adjoints (transposed Jacobians) of the search steps, for gradients of a loss of the
// periodogram with respect to the searched series. The reference's search is not
// differentiable; these follow its forward arithmetic (snr.hpp:37-65, transforms.hpp:13-61,
// downsample.hpp:44-82, time_series.py:67-93) so that the gradient is the one of the function
// the forward computes.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "snr_core.cuh"

namespace rt {

// ------------------------------------------------------------------------------------
// Boxcar S/N: S/N_w = ((h+b) dmax_w - b sum) / sigma, dmax_w = max_i C[i+w] - C[i] with C the
// circular prefix sum. d S/N_w / d x_q = (h+b)/sigma on the w phases after the first
// maximising i, minus b/sigma on every phase.
// ------------------------------------------------------------------------------------
constexpr int kSnrBwdMaxWidths = 64;

__global__ void k_snr2_backward(const float* __restrict__ x, int rows, int b,
                                const int* __restrict__ widths, int nw, float stdnoise,
                                const float* __restrict__ gsnr, float* __restrict__ gx, int wmax)
{
    extern __shared__ float sC[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    float* C = sC + (size_t)wib * (b + wmax + 1);
    __shared__ int s_best[32][kSnrBwdMaxWidths];
    for (int r = blockIdx.x * wpb + wib; r < rows; r += gridDim.x * wpb) {
        const float* xr = x + (size_t)r * b;
        // circular prefix: float of the double running sum (kernels.hpp:73-101), as the
        // forward stores it; the wrap-around part as cr[j] + float(sum)
        double carry = 0.0;
        for (int c0 = 0; c0 < b; c0 += 32) {
            const int c = c0 + lane;
            const double v = (c < b) ? (double)xr[c] : 0.0;
            double incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (c < b) C[c] = (float)(carry + incl);
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
        const float sumx = (float)carry;
        for (int j = lane; j < wmax; j += 32) C[b + j] = __fadd_rn(C[j], sumx);
        __syncwarp();
        // first maximising phase per width
        for (int k = 0; k < nw; ++k) {
            const int w = widths[k];
            float best = -INFINITY;
            int bi = b;
            for (int i = lane; i < b; i += 32) {
                const float d = __fsub_rn(C[i + w], C[i]);
                if (d > best) {
                    best = d;
                    bi = i;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (lane == 0) s_best[wib][k] = bi;
        }
        __syncwarp();
        // gradient of the row
        const float* g = gsnr + (size_t)r * nw;
        double base = 0.0;
        for (int k = 0; k < nw; ++k) {
            float hb, be;
            boxcar_coefs(b, widths[k], &hb, &be);
            base -= (double)g[k] * (double)be / (double)stdnoise;
        }
        for (int q = lane; q < b; q += 32) {
            double acc = base;
            for (int k = 0; k < nw; ++k) {
                const int w = widths[k];
                int off = q - s_best[wib][k] - 1;  // position of q in the window
                off += (off < 0) ? b : 0;
                if (off < w) {
                    float hb, be;
                    boxcar_coefs(b, w, &hb, &be);
                    acc += (double)g[k] * (double)hb / (double)stdnoise;
                }
            }
            gx[(size_t)r * b + q] = (float)acc;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------
// FFA transpose. The forward merges node (row0, n) from its head (rows row0 + [0, n/2)) and
// tail (the rest): out[s] = head[h(s)] + roll(tail[t(s)], -(s - t(s))). The transpose, level by
// level from the root: a head row j gathers the rows s with h(s) = j; a tail row j gathers the
// rows s with t(s) = j, rolled back by s - t(s). Rows of nodes that no longer split are copied.
// ------------------------------------------------------------------------------------
struct TRow {
    int row0, n, kind, j;  // parent node; kind 0 copy, 1 head row j, 2 tail row j
};

// first s in [0, n) with merge_row(k, s) >= v (merge_row is non-decreasing in s)
__device__ __forceinline__ int first_at_least(float k, int n, int v)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (merge_row(k, mid) >= v) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__global__ void k_ffa_transpose_level(const float* __restrict__ gp, float* __restrict__ gc,
                                      const TRow* __restrict__ tab, int m, int b)
{
    const int lane = threadIdx.x & 31;
    for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m;
         r += (gridDim.x * blockDim.x) >> 5) {
        const TRow e = tab[r];
        float* out = gc + (size_t)r * b;
        if (e.kind == 0) {
            for (int c = lane; c < b; c += 32) out[c] = gp[(size_t)r * b + c];
            continue;
        }
        const MergeCoef mc = merge_coef(e.n);
        const float k = (e.kind == 1) ? mc.kh : mc.kt;
        const int s0 = first_at_least(k, e.n, e.j), s1 = first_at_least(k, e.n, e.j + 1);
        for (int c = lane; c < b; c += 32) {
            float acc = 0.0f;
            for (int s = s0; s < s1; ++s) {
                const float* src = gp + (size_t)(e.row0 + s) * b;
                if (e.kind == 1) {
                    acc = __fadd_rn(acc, src[c]);
                } else {
                    const int t = merge_row(mc.kt, s);
                    int idx = c - (s - t) % b;
                    idx += (idx < 0) ? b : 0;
                    acc = __fadd_rn(acc, src[idx]);
                }
            }
            out[c] = acc;
        }
    }
}

// Transition tables, root level first: tab[l][r] maps row r of level l + 1 to level l.
static int ffa_transpose_tables(int m, std::vector<TRow>& tabs, int* nlevels)
{
    std::vector<int2> nodes{make_int2(0, m)};
    tabs.clear();
    int L = 0;
    while (true) {
        bool split = false;
        for (const int2& nd : nodes) split |= nd.y >= 2;
        if (!split) break;
        std::vector<int2> next;
        const size_t base = tabs.size();
        tabs.resize(base + (size_t)m);
        for (const int2& nd : nodes) {
            if (nd.y < 2) {
                tabs[base + nd.x] = TRow{nd.x, 1, 0, 0};
                next.push_back(nd);
                continue;
            }
            const int nh = nd.y >> 1;
            for (int j = 0; j < nh; ++j) tabs[base + nd.x + j] = TRow{nd.x, nd.y, 1, j};
            for (int j = 0; j < nd.y - nh; ++j)
                tabs[base + nd.x + nh + j] = TRow{nd.x, nd.y, 2, j};
            next.push_back(make_int2(nd.x, nh));
            next.push_back(make_int2(nd.x + nh, nd.y - nh));
        }
        nodes.swap(next);
        ++L;
        if (L > 64) return set_error(RT_EINTERNAL, "FFA transpose: too many levels");
    }
    *nlevels = L;
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// Downsampling adjoint: out[k] = wmin x[imin] + sum_{imin < i < imax} x[i] + wmax x[imax]
// (written as a prefix difference, so imax == imin gives (wmin + wmax - 1) x[imin]).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double ds_coef(size_t k, double f, size_t N, size_t i)
{
    const double start = (double)k * f;
    const double end = start + f;
    const size_t imin = (size_t)floor(start);
    const double fe = floor(end);
    const size_t imax = (size_t)(fe < (double)N - 1.0 ? fe : (double)N - 1.0);
    const float wmin = __double2float_rn((double)(imin + 1) - start);
    const float wmax = __double2float_rn(end - (double)imax);
    double c = 0.0;
    if (i == imin) c += (double)wmin;
    if (i == imax) c += (double)wmax;
    if (i > imin && i < imax) c += 1.0;
    if (imax == imin && i == imin) c -= 1.0;
    return c;
}

__global__ void k_downsample_adjoint(const float* __restrict__ gout, size_t N, double f,
                                     size_t n, float* __restrict__ gin)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        const double q = floor((double)i / f);
        const size_t k0 = q >= 1.0 ? (size_t)q - 1 : 0;
        const size_t k1 = std::min(n, (size_t)floor((double)(i + 1) / f) + 2);
        double acc = 0.0;
        for (size_t k = k0; k < k1; ++k) {
            const double c = ds_coef(k, f, N, i);
            if (c != 0.0) acc += c * (double)gout[k];
        }
        if (acc != 0.0) gin[i] = __fadd_rn(gin[i], (float)acc);
    }
}

// ------------------------------------------------------------------------------------
// Normalisation adjoint (population statistics)
// ------------------------------------------------------------------------------------
constexpr int kNormBwdThreads = 256;

__global__ void k_norm_adj_sums(const float* __restrict__ g, const float* __restrict__ z,
                                size_t N, double* __restrict__ part)
{
    double s1 = 0.0, s2 = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        s1 += (double)g[i];
        s2 += (double)g[i] * (double)z[i];
    }
    __shared__ double r1[kNormBwdThreads], r2[kNormBwdThreads];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int o = kNormBwdThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            r1[threadIdx.x] += r1[threadIdx.x + o];
            r2[threadIdx.x] += r2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = r1[0];
        part[2 * blockIdx.x + 1] = r2[0];
    }
}

__global__ void k_norm_adj_apply(const float* __restrict__ g, const float* __restrict__ z,
                                 size_t N, const double* __restrict__ part, int nblocks,
                                 double inv_std, float* __restrict__ gy)
{
    __shared__ double s_m1, s_m2;
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int k = 0; k < nblocks; ++k) {
            a += part[2 * k];
            c += part[2 * k + 1];
        }
        s_m1 = a / (double)N;
        s_m2 = c / (double)N;
    }
    __syncthreads();
    const double m1 = s_m1, m2 = s_m2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x)
        gy[i] = (float)(((double)g[i] - m1 - (double)z[i] * m2) * inv_std);
}

}  // namespace rt

using namespace rt;

extern "C" int rt_snr2_backward(const float* d_in, size_t rows, size_t cols,
                                const uint64_t* h_widths, size_t num_widths, float stdnoise,
                                const float* d_gsnr, float* d_gin, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (rows == 0) return RT_OK;
    if (!d_in || !d_gin || !d_gsnr || (!h_widths && num_widths))
        return set_error(RT_EINVAL, "null argument");
    if (num_widths > (size_t)kSnrBwdMaxWidths)
        return set_error(RT_EINVAL, "at most %d trial widths are supported", kSnrBwdMaxWidths);
    std::vector<int> w(num_widths);
    int wmax = 1;
    for (size_t k = 0; k < num_widths; ++k) {
        if (!(h_widths[k] > 0 && h_widths[k] < cols))  // snr.hpp:21-31
            return set_error(RT_EINVAL, "trial widths must be all > 0 and < columns");
        w[k] = (int)h_widths[k];
        wmax = std::max(wmax, w[k]);
    }
    if (!(stdnoise > 0.0f)) return set_error(RT_EINVAL, "stdnoise must be > 0");
    const size_t per_warp = (cols + wmax + 1) * sizeof(float);
    int wpb = (int)std::min<size_t>(8, (160 * 1024) / per_warp);
    if (wpb < 1) return set_error(RT_EINVAL, "profiles of %zu bins are too long", cols);
    int* d_w = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_w, std::max<size_t>(num_widths, 1) * sizeof(int), st));
    int s = check_cuda(cudaMemcpyAsync(d_w, w.data(), num_widths * sizeof(int),
                                       cudaMemcpyHostToDevice, st), "snr2_backward");
    const size_t smem = (size_t)wpb * per_warp;
    if (s == RT_OK && smem > 48 * 1024)
        s = check_cuda(cudaFuncSetAttribute(k_snr2_backward,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                       "snr2_backward");
    if (s == RT_OK) {
        const int grid = (int)std::min<size_t>((rows + wpb - 1) / wpb, 148 * 16);
        k_snr2_backward<<<grid, 32 * wpb, smem, st>>>(d_in, (int)rows, (int)cols, d_w,
                                                     (int)num_widths, stdnoise, d_gsnr, d_gin, wmax);
        s = check_cuda(cudaGetLastError(), "snr2_backward");
    }
    cudaFreeAsync(d_w, st);
    return s;
}

extern "C" int rt_ffa2_transpose(const float* d_gout, size_t rows, size_t cols, float* d_gin,
                                 void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (rows == 0 || cols == 0) return RT_OK;
    if (!d_gout || !d_gin) return set_error(RT_EINVAL, "null argument");
    if (rows >= (1u << 24) || cols >= (1u << 24))
        return set_error(RT_EINVAL, "a %zu x %zu block is too large", rows, cols);
    const int m = (int)rows, b = (int)cols;
    std::vector<TRow> tabs;
    int L = 0;
    RT_TRY(ffa_transpose_tables(m, tabs, &L));
    if (L == 0)
        return check_cuda(cudaMemcpyAsync(d_gin, d_gout, rows * cols * sizeof(float),
                                          cudaMemcpyDeviceToDevice, st), "ffa2_transpose");
    TRow* d_tab = nullptr;
    float* tmp = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_tab, tabs.size() * sizeof(TRow), st));
    int s = check_cuda(cudaMallocAsync((void**)&tmp, rows * cols * sizeof(float), st), "ffa2_transpose");
    if (s == RT_OK)
        s = check_cuda(cudaMemcpyAsync(d_tab, tabs.data(), tabs.size() * sizeof(TRow),
                                       cudaMemcpyHostToDevice, st), "ffa2_transpose");
    // ping-pong so that the last level lands in d_gin
    const float* src = d_gout;
    for (int l = 0; l < L && s == RT_OK; ++l) {
        float* dst = ((L - 1 - l) % 2 == 0) ? d_gin : tmp;
        const int grid = (int)std::min<size_t>(((size_t)m * 32 + 255) / 256, 148 * 8);
        k_ffa_transpose_level<<<grid, 256, 0, st>>>(src, dst, d_tab + (size_t)l * m, m, b);
        s = check_cuda(cudaGetLastError(), "ffa2_transpose");
        src = dst;
    }
    cudaFreeAsync(tmp, st);
    cudaFreeAsync(d_tab, st);
    return s;
}

extern "C" int rt_downsample_adjoint(const float* d_gout, size_t size, double f, float* d_gin,
                                     void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (!((f > 1.0) && (f <= (double)size)))  // downsample.hpp:11-16
        return set_error(RT_EINVAL, "Downsampling factor must verify: 1 < f <= size");
    if (!d_gout || !d_gin) return set_error(RT_EINVAL, "null argument");
    const size_t n = downsampled_size(size, f);
    const int grid = (int)std::min<size_t>((size + 255) / 256, 148 * 16);
    k_downsample_adjoint<<<grid, 256, 0, st>>>(d_gout, size, f, n, d_gin);
    return check_cuda(cudaGetLastError(), "downsample_adjoint");
}

extern "C" int rt_normalise_adjoint(const float* d_g, const float* d_z, size_t size,
                                    double std_, float* d_gy, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (size == 0) return RT_OK;
    if (!d_g || !d_z || !d_gy) return set_error(RT_EINVAL, "null argument");
    if (!(std_ > 0.0)) return set_error(RT_EINVAL, "std must be > 0");
    const int blocks = (int)std::min<size_t>((size + kNormBwdThreads - 1) / kNormBwdThreads, 512);
    double* part = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&part, (size_t)blocks * 2 * sizeof(double), st));
    k_norm_adj_sums<<<blocks, kNormBwdThreads, 0, st>>>(d_g, d_z, size, part);
    int s = check_cuda(cudaGetLastError(), "normalise_adjoint");
    if (s == RT_OK) {
        k_norm_adj_apply<<<blocks, kNormBwdThreads, 0, st>>>(d_g, d_z, size, part, blocks,
                                                             1.0 / std_, d_gy);
        s = check_cuda(cudaGetLastError(), "normalise_adjoint");
    }
    cudaFreeAsync(part, st);
    return s;
}
