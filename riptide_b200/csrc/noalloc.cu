// rt_ffa2_noalloc: the FFA transform of rt_ffa2 for callers that must not allocate device
// memory, with its scratch in a fixed array that every GPU loading this library holds.
//
// Who needs it: search pipelines whose device memory is reserved up front by another
// framework's pool (so a cudaMalloc of a few MiB can fail mid-run even though the pool has
// room), and real-time search loops that forbid allocation after start-up because
// cudaMalloc / cudaFree can block on the whole device and stall other streams.
//
// Limits and behaviour (also stated in include/riptide_b200.h):
//  * rows * cols must not exceed kNoAllocMaxValues (1 Mi values, i.e. 4 MiB per copy; the
//    transform keeps two copies of intermediate results when it needs several passes);
//    larger inputs are rejected with RT_EINVAL before anything is launched;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress)
//    with that device current and caches it for the life of the process; make that first
//    call before any stream capture. cudaDeviceReset after the first call is not supported:
//    the module is loaded again at a new address and the cached one is stale;
//  * all calls share the array and its contents stay from the last call; the error word is
//    cleared at the start of each call, and every scratch row a call reads was written
//    earlier in the same call, so nothing else needs clearing; calls that overlap on the GPU
//    (different streams, or several host threads) race on the array and must not be issued.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr size_t kNoAllocMaxValues = size_t(1) << 20;
constexpr size_t kNoAllocHeaderFloats = 64;  // error word, padded to 256 bytes
constexpr size_t kNoAllocFloats = kNoAllocHeaderFloats + 2 * kNoAllocMaxValues;

static __device__ __align__(256) float g_noalloc_scratch[kNoAllocFloats];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
float* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device (set up on first use).
int noalloc_scratch(float** out)
{
    int dev = 0;
    RT_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return rt::set_error(RT_EINVAL, "device %d is out of the supported range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        float* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return rt::check_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return RT_OK;
}

}  // namespace

extern "C" int rt_ffa2_noalloc(const float* d_in, size_t rows, size_t cols, float* d_out,
                               void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (rows == 0 || cols == 0) return RT_OK;
    if (rows >= (1u << 24) || cols > 4096 || rows * cols > kNoAllocMaxValues)
        return rt::set_error(RT_EINVAL,
                             "rt_ffa2_noalloc: a %zu x %zu block exceeds the fixed scratch "
                             "(at most %zu values, cols <= 4096)",
                             rows, cols, kNoAllocMaxValues);
    float* base = nullptr;
    RT_TRY(noalloc_scratch(&base));
    int* d_err = reinterpret_cast<int*>(base);
    float* scratch = base + kNoAllocHeaderFloats;
    RT_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    RT_TRY(rt::ffa_transform(d_in, (int)rows, (int)cols, (int)rows, d_out, scratch, d_err, st));
    int herr = 0;
    RT_TRY_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    if (herr) return rt::set_error(RT_EINTERNAL, "rt_ffa2_noalloc: device plan check failed (%d)", herr);
    return RT_OK;
}
