// Ingest of dedispersed time series files into device memory (the data side of
// TimeSeries.from_presto_inf / from_sigproc, time_series.py:300-379, reading/presto.py:148-152
// of the reference). File payloads are read with parallel pread into page-locked host memory,
// copied to the device in double-buffered chunks while the next chunk is read, and widened to
// float32 on the device: an 8-bit payload crosses PCIe as bytes, a quarter of the float32
// volume, and is converted exactly as numpy's astype(np.float32) converts it.
#include <errno.h>
#include <fcntl.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "common.cuh"

namespace rt {

static size_t sample_bytes(int encoding)
{
    return encoding == RT_SAMPLES_F32 ? 4 : 1;
}

// Four samples per thread: one 32-bit load of the bytes, four float stores. `src` is 4-byte
// aligned (the staging buffer's chunks start at multiples of the page size).
template <bool kSigned>
__global__ void k_widen8(const uint8_t* __restrict__ src, size_t n, float* __restrict__ dst)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; 4 * q < n; q += stride) {
        const size_t i = 4 * q;
        if (i + 4 <= n) {
            const uint32_t v = *reinterpret_cast<const uint32_t*>(src + i);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t byte = (v >> (8 * k)) & 0xffu;
                dst[i + k] = kSigned ? (float)(int8_t)byte : (float)byte;
            }
        } else {
            for (size_t j = i; j < n; ++j)
                dst[j] = kSigned ? (float)(int8_t)src[j] : (float)src[j];
        }
    }
}

static int launch_widen8(const void* src, int encoding, size_t n, float* dst, cudaStream_t st)
{
    if (n == 0) return RT_OK;
    const size_t quads = (n + 3) / 4;
    const int threads = 256;
    const size_t want = (quads + threads - 1) / threads;
    const int blocks = (int)std::min<size_t>(want, (size_t)148 * 16);
    if (encoding == RT_SAMPLES_I8)
        k_widen8<true><<<blocks, threads, 0, st>>>((const uint8_t*)src, n, dst);
    else
        k_widen8<false><<<blocks, threads, 0, st>>>((const uint8_t*)src, n, dst);
    RT_TRY_CUDA(cudaGetLastError());
    return RT_OK;
}

// pread of [offset, offset + nbytes) of an open file into dst, split over `threads` threads.
static int pread_parallel(int fd, const char* path, uint64_t offset, uint64_t nbytes, void* dst,
                          int threads)
{
    const uint64_t kMinSlice = 1ull << 20;
    int nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)std::max(threads, 1),
                                                           nbytes / kMinSlice));
    std::vector<int> err(nt, 0);
    std::vector<uint64_t> got(nt, 0);
    auto work = [&](int t) {
        const uint64_t a = nbytes * t / nt, b = nbytes * (t + 1) / nt;
        uint64_t pos = a;
        while (pos < b) {
            const ssize_t r = pread(fd, (char*)dst + pos, (size_t)std::min<uint64_t>(b - pos, 1ull << 30),
                                    (off_t)(offset + pos));
            if (r < 0) {
                if (errno == EINTR) continue;
                err[t] = errno;
                return;
            }
            if (r == 0) break;
            pos += (uint64_t)r;
        }
        got[t] = pos - a;
    };
    if (nt == 1) {
        work(0);
    } else {
        std::vector<std::thread> pool;
        pool.reserve(nt);
        for (int t = 0; t < nt; ++t) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (int t = 0; t < nt; ++t) {
        if (err[t]) return set_error(RT_EIO, "reading %s: %s", path, strerror(err[t]));
        const uint64_t want = nbytes * (t + 1) / nt - nbytes * t / nt;
        if (got[t] != want)
            return set_error(RT_EIO, "%s holds fewer than %llu bytes after offset %llu", path,
                             (unsigned long long)nbytes, (unsigned long long)offset);
    }
    return RT_OK;
}

namespace {
struct Fd {
    int fd = -1;
    ~Fd()
    {
        if (fd >= 0) close(fd);
    }
};
}  // namespace

static int open_file(const char* path, Fd& f)
{
    if (!path) return set_error(RT_EINVAL, "file path is null");
    f.fd = open(path, O_RDONLY | O_CLOEXEC);
    if (f.fd < 0) return set_error(RT_EIO, "cannot open %s: %s", path, strerror(errno));
    return RT_OK;
}

}  // namespace rt

using namespace rt;

extern "C" int rt_file_size(const char* path, uint64_t* size)
{
    if (!path || !size) return set_error(RT_EINVAL, "null argument");
    struct stat sb;
    if (stat(path, &sb) != 0) return set_error(RT_EIO, "cannot stat %s: %s", path, strerror(errno));
    *size = (uint64_t)sb.st_size;
    return RT_OK;
}

extern "C" int rt_read_file(const char* path, uint64_t offset, uint64_t nbytes, void* dst,
                            int threads)
{
    if (nbytes && !dst) return set_error(RT_EINVAL, "destination is null");
    Fd f;
    RT_TRY(open_file(path, f));
    if (!nbytes) return RT_OK;
    return pread_parallel(f.fd, path, offset, nbytes, dst, threads);
}

extern "C" int rt_samples_to_f32(const void* d_src, int encoding, size_t n, float* d_dst,
                                 void* stream_)
{
    cudaStream_t stream = (cudaStream_t)stream_;
    if (encoding != RT_SAMPLES_F32 && encoding != RT_SAMPLES_U8 && encoding != RT_SAMPLES_I8)
        return set_error(RT_EINVAL, "unknown sample encoding %d", encoding);
    if (n && (!d_src || !d_dst)) return set_error(RT_EINVAL, "null pointer");
    if (n == 0) return RT_OK;
    if (encoding == RT_SAMPLES_F32) {
        if (d_src != d_dst)
            RT_TRY_CUDA(cudaMemcpyAsync(d_dst, d_src, n * 4, cudaMemcpyDeviceToDevice, stream));
        return RT_OK;
    }
    if ((uintptr_t)d_src % 4) return set_error(RT_EINVAL, "8-bit source must be 4-byte aligned");
    return launch_widen8(d_src, encoding, n, d_dst, stream);
}

extern "C" int rt_ingest_files(const char* const* paths, const uint64_t* offsets,
                               const uint64_t* nsamples, const int* encodings, size_t nfiles,
                               float* d_out, void* h_staging, size_t staging_bytes, int threads,
                               void* stream_)
{
    cudaStream_t stream = (cudaStream_t)stream_;
    if (nfiles && (!paths || !offsets || !nsamples || !encodings))
        return set_error(RT_EINVAL, "null file table");
    const size_t kPage = 4096;
    const size_t half = (staging_bytes / 2) / kPage * kPage;
    if (!h_staging || half < 16 * kPage)
        return set_error(RT_EINVAL, "staging buffer must hold at least %zu bytes", 32 * kPage);
    bool any8 = false;
    uint64_t total = 0;
    for (size_t i = 0; i < nfiles; ++i) {
        const int e = encodings[i];
        if (e != RT_SAMPLES_F32 && e != RT_SAMPLES_U8 && e != RT_SAMPLES_I8)
            return set_error(RT_EINVAL, "file %zu: unknown sample encoding %d", i, e);
        any8 = any8 || e != RT_SAMPLES_F32;
        total += nsamples[i];
    }
    if (total && !d_out) return set_error(RT_EINVAL, "output is null");
    if (!total) return RT_OK;

    char* hbuf[2] = {(char*)h_staging, (char*)h_staging + half};
    uint8_t* dstage = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    int status = RT_OK;
    auto fail_cuda = [&](cudaError_t e, const char* what) {
        status = check_cuda(e, what);
    };
    for (int h = 0; h < 2 && status == RT_OK; ++h) {
        cudaError_t e = cudaEventCreateWithFlags(&ev[h], cudaEventDisableTiming);
        if (e != cudaSuccess) fail_cuda(e, "cudaEventCreateWithFlags");
    }
    if (status == RT_OK && any8) {
        cudaError_t e = cudaMallocAsync((void**)&dstage, 2 * half, stream);
        if (e != cudaSuccess) fail_cuda(e, "cudaMallocAsync");
    }
    uint64_t out_pos = 0;
    int k = 0;
    for (size_t i = 0; i < nfiles && status == RT_OK; ++i) {
        const int enc = encodings[i];
        const uint64_t esz = sample_bytes(enc);
        const uint64_t bytes = nsamples[i] * esz;
        Fd f;
        if (bytes) status = open_file(paths[i], f);
        // chunks hold whole samples: half is a multiple of 4
        for (uint64_t off = 0; off < bytes && status == RT_OK; off += half, ++k) {
            const int h = k & 1;
            const uint64_t c = std::min<uint64_t>(half, bytes - off);
            if (used[h]) {
                cudaError_t e = cudaEventSynchronize(ev[h]);
                if (e != cudaSuccess) {
                    fail_cuda(e, "cudaEventSynchronize");
                    break;
                }
            }
            status = pread_parallel(f.fd, paths[i], offsets[i] + off, c, hbuf[h], threads);
            if (status != RT_OK) break;
            float* dst = d_out + out_pos + off / esz;
            cudaError_t e;
            if (enc == RT_SAMPLES_F32) {
                e = cudaMemcpyAsync(dst, hbuf[h], c, cudaMemcpyHostToDevice, stream);
            } else {
                uint8_t* ds = dstage + (size_t)h * half;
                e = cudaMemcpyAsync(ds, hbuf[h], c, cudaMemcpyHostToDevice, stream);
                if (e == cudaSuccess) {
                    status = launch_widen8(ds, enc, c, dst, stream);
                    if (status != RT_OK) break;
                }
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[h], stream);
            if (e != cudaSuccess) {
                fail_cuda(e, "cudaMemcpyAsync");
                break;
            }
            used[h] = true;
        }
        out_pos += nsamples[i];
    }
    // the staging buffer must not be reused before its last copy has left it
    for (int h = 0; h < 2; ++h) {
        if (ev[h]) {
            if (used[h]) {
                cudaError_t e = cudaEventSynchronize(ev[h]);
                if (e != cudaSuccess && status == RT_OK) fail_cuda(e, "cudaEventSynchronize");
            }
            cudaEventDestroy(ev[h]);
        }
    }
    if (dstage) {
        cudaError_t e = cudaFreeAsync(dstage, stream);
        if (e != cudaSuccess && status == RT_OK) fail_cuda(e, "cudaFreeAsync");
    }
    return status;
}
