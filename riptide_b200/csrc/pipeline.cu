// Host-buffer search pipeline: the batched search of series held in host memory, with the
// host -> device copies of the input and the device -> host copies of the periodograms
// overlapped with the search kernels.
//
// The reference searches DM trials from host memory, one worker process per trial
// (pipeline/worker_pool.py:35-68 calling search.py:11-93). Here the trials are cut into
// chunks of consecutive trials, each with its own plan; two chunks of device buffers are in
// flight. Three streams: copies in, search, copies out. Chunk i:
//   in-stream:     wait until chunk i-2's search is done with input buffer (i & 1),
//                  copy its series in, record "input ready"
//   search-stream: wait for "input ready" and for chunk i-2's results to have left output
//                  buffer (i & 1), run the chunk's plan, record "search done"
//   out-stream:    wait for "search done", copy periods / foldbins / S/N out, record
//                  "output free"
// so the search of chunk i runs while chunk i+1 comes in and chunk i-1 goes out. Copies
// overlap only when the host buffers are page-locked (cudaHostAlloc / cudaHostRegister);
// with pageable memory the results are the same, the copies just do not overlap.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "../../include/riptide_b200.h"

namespace {

struct Chunk {
    rt_search_plan* plan = nullptr;
    size_t t0 = 0, nt = 0;        // first trial, number of trials
    size_t s0 = 0, ns = 0;        // first sample, number of samples
    size_t r0 = 0, nr = 0;        // first periodogram row, number of rows
};

}  // namespace

struct rt_search_pipeline {
    std::vector<Chunk> chunks;
    std::vector<uint64_t> rows;   // ntrials + 1 row offsets
    size_t nw = 0;
    int device = 0;
    float* d_in[2] = {nullptr, nullptr};
    double* d_periods[2] = {nullptr, nullptr};
    uint32_t* d_foldbins[2] = {nullptr, nullptr};
    float* d_snrs[2] = {nullptr, nullptr};
    cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_run_done[2] = {nullptr, nullptr};
    cudaEvent_t ev_out_free[2] = {nullptr, nullptr};
};

static void pipeline_free(rt_search_pipeline* P)
{
    if (!P) return;
    for (Chunk& c : P->chunks)
        if (c.plan) rt_search_plan_destroy(c.plan);
    for (int j = 0; j < 2; ++j) {
        if (P->d_in[j]) cudaFree(P->d_in[j]);
        if (P->d_periods[j]) cudaFree(P->d_periods[j]);
        if (P->d_foldbins[j]) cudaFree(P->d_foldbins[j]);
        if (P->d_snrs[j]) cudaFree(P->d_snrs[j]);
        if (P->ev_in_ready[j]) cudaEventDestroy(P->ev_in_ready[j]);
        if (P->ev_run_done[j]) cudaEventDestroy(P->ev_run_done[j]);
        if (P->ev_out_free[j]) cudaEventDestroy(P->ev_out_free[j]);
    }
    if (P->ev_begin) cudaEventDestroy(P->ev_begin);
    if (P->ev_end) cudaEventDestroy(P->ev_end);
    if (P->s_in) cudaStreamDestroy(P->s_in);
    if (P->s_run) cudaStreamDestroy(P->s_run);
    if (P->s_out) cudaStreamDestroy(P->s_out);
    delete P;
}

static int pipeline_build(rt_search_pipeline* P, const uint64_t* lengths, size_t ntrials,
                          const rt_search_config* cfg, const uint64_t* widths, size_t nw,
                          size_t chunk_trials)
{
    P->nw = nw;
    RT_TRY_CUDA(cudaGetDevice(&P->device));
    P->rows.assign(ntrials + 1, 0);
    // chunk sizes: a quarter chunk first and last, so that the copy-in before the first
    // search and the copy-out after the last one (the parts of the pipeline that overlap
    // nothing) are short; full chunks in between
    std::vector<size_t> sizes;
    const size_t q = std::max<size_t>(1, chunk_trials / 4);
    if (ntrials <= chunk_trials + 2 * q) {
        for (size_t t0 = 0; t0 < ntrials; t0 += chunk_trials)
            sizes.push_back(std::min(chunk_trials, ntrials - t0));
    } else {
        sizes.push_back(q);
        size_t left = ntrials - 2 * q;
        while (left > 0) {
            const size_t n = std::min(chunk_trials, left);
            sizes.push_back(n);
            left -= n;
        }
        sizes.push_back(q);
    }
    size_t s = 0, t0 = 0;
    for (size_t ci = 0; ci < sizes.size(); t0 += sizes[ci], ++ci) {
        Chunk c;
        c.t0 = t0;
        c.nt = sizes[ci];
        c.s0 = s;
        for (size_t i = 0; i < c.nt; ++i) s += lengths[t0 + i];
        c.ns = s - c.s0;
        RT_TRY(rt_search_plan_create(lengths + t0, c.nt, cfg, widths, nw, &c.plan));
        P->chunks.push_back(c);  // owned by P from here on (freed on error)
        std::vector<uint64_t> r(c.nt + 1);
        RT_TRY(rt_search_plan_rows(c.plan, r.data()));
        Chunk& cc = P->chunks.back();
        cc.r0 = P->rows[t0];
        cc.nr = r[c.nt];
        for (size_t i = 0; i < c.nt; ++i) P->rows[t0 + i + 1] = cc.r0 + r[i + 1];
        RT_TRY(rt_search_plan_prepare(cc.plan));
        RT_TRY(rt_search_set_graph(cc.plan, 1));  // each chunk always uses the same buffers
    }
    size_t max_s = 1, max_r = 1;
    for (const Chunk& c : P->chunks) {
        max_s = std::max(max_s, c.ns);
        max_r = std::max(max_r, c.nr);
    }
    for (int j = 0; j < 2 && j < (int)P->chunks.size(); ++j) {
        RT_TRY_CUDA(cudaMalloc((void**)&P->d_in[j], max_s * sizeof(float)));
        RT_TRY_CUDA(cudaMalloc((void**)&P->d_periods[j], max_r * sizeof(double)));
        RT_TRY_CUDA(cudaMalloc((void**)&P->d_foldbins[j], max_r * sizeof(uint32_t)));
        RT_TRY_CUDA(cudaMalloc((void**)&P->d_snrs[j], max_r * std::max<size_t>(nw, 1) * sizeof(float)));
    }
    RT_TRY_CUDA(cudaStreamCreateWithFlags(&P->s_in, cudaStreamNonBlocking));
    RT_TRY_CUDA(cudaStreamCreateWithFlags(&P->s_run, cudaStreamNonBlocking));
    RT_TRY_CUDA(cudaStreamCreateWithFlags(&P->s_out, cudaStreamNonBlocking));
    RT_TRY_CUDA(cudaEventCreateWithFlags(&P->ev_begin, cudaEventDisableTiming));
    RT_TRY_CUDA(cudaEventCreateWithFlags(&P->ev_end, cudaEventDisableTiming));
    for (int j = 0; j < 2; ++j) {
        RT_TRY_CUDA(cudaEventCreateWithFlags(&P->ev_in_ready[j], cudaEventDisableTiming));
        RT_TRY_CUDA(cudaEventCreateWithFlags(&P->ev_run_done[j], cudaEventDisableTiming));
        RT_TRY_CUDA(cudaEventCreateWithFlags(&P->ev_out_free[j], cudaEventDisableTiming));
    }
    return RT_OK;
}

extern "C" int rt_search_pipeline_create(const uint64_t* h_lengths, size_t ntrials,
                                         const rt_search_config* cfg, const uint64_t* h_widths,
                                         size_t num_widths, size_t chunk_trials,
                                         rt_search_pipeline** out)
{
    if (!out || !cfg || !h_lengths || ntrials == 0)
        return rt::set_error(RT_EINVAL, "null argument or no trials");
    if (chunk_trials == 0) return rt::set_error(RT_EINVAL, "chunk_trials must be positive");
    *out = nullptr;
    rt_search_pipeline* P = new rt_search_pipeline();
    const int rc = pipeline_build(P, h_lengths, ntrials, cfg, h_widths, num_widths, chunk_trials);
    if (rc != RT_OK) {
        pipeline_free(P);
        return rc;
    }
    *out = P;
    return RT_OK;
}

extern "C" int rt_search_pipeline_rows(const rt_search_pipeline* P, uint64_t* h_row_offsets)
{
    if (!P || !h_row_offsets) return rt::set_error(RT_EINVAL, "null argument");
    std::copy(P->rows.begin(), P->rows.end(), h_row_offsets);
    return RT_OK;
}

extern "C" int rt_search_pipeline_chunks(const rt_search_pipeline* P, size_t* h_nchunks)
{
    if (!P || !h_nchunks) return rt::set_error(RT_EINVAL, "null argument");
    *h_nchunks = P->chunks.size();
    return RT_OK;
}

extern "C" int rt_search_pipeline_run(rt_search_pipeline* P, const float* h_data,
                                      double* h_periods, uint32_t* h_foldbins, float* h_snrs,
                                      void* stream)
{
    if (!P || !h_data || !h_periods || !h_foldbins || !h_snrs)
        return rt::set_error(RT_EINVAL, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    RT_TRY_CUDA(cudaGetDevice(&dev));
    if (dev != P->device)
        return rt::set_error(RT_EINVAL, "the pipeline was created on device %d, current is %d",
                             P->device, dev);
    // everything enqueued here runs after the work already in `stream`
    RT_TRY_CUDA(cudaEventRecord(P->ev_begin, st));
    RT_TRY_CUDA(cudaStreamWaitEvent(P->s_in, P->ev_begin, 0));
    RT_TRY_CUDA(cudaStreamWaitEvent(P->s_run, P->ev_begin, 0));
    RT_TRY_CUDA(cudaStreamWaitEvent(P->s_out, P->ev_begin, 0));
    const size_t nw = P->nw;
    for (size_t i = 0; i < P->chunks.size(); ++i) {
        const Chunk& c = P->chunks[i];
        const int j = (int)(i & 1);
        if (i >= 2) RT_TRY_CUDA(cudaStreamWaitEvent(P->s_in, P->ev_run_done[j], 0));
        RT_TRY_CUDA(cudaMemcpyAsync(P->d_in[j], h_data + c.s0, c.ns * sizeof(float),
                                    cudaMemcpyHostToDevice, P->s_in));
        RT_TRY_CUDA(cudaEventRecord(P->ev_in_ready[j], P->s_in));

        RT_TRY_CUDA(cudaStreamWaitEvent(P->s_run, P->ev_in_ready[j], 0));
        if (i >= 2) RT_TRY_CUDA(cudaStreamWaitEvent(P->s_run, P->ev_out_free[j], 0));
        RT_TRY(rt_search_run(c.plan, P->d_in[j], nullptr, P->d_periods[j], P->d_foldbins[j],
                             P->d_snrs[j], P->s_run));
        RT_TRY_CUDA(cudaEventRecord(P->ev_run_done[j], P->s_run));

        RT_TRY_CUDA(cudaStreamWaitEvent(P->s_out, P->ev_run_done[j], 0));
        RT_TRY_CUDA(cudaMemcpyAsync(h_periods + c.r0, P->d_periods[j], c.nr * sizeof(double),
                                    cudaMemcpyDeviceToHost, P->s_out));
        RT_TRY_CUDA(cudaMemcpyAsync(h_foldbins + c.r0, P->d_foldbins[j], c.nr * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, P->s_out));
        RT_TRY_CUDA(cudaMemcpyAsync(h_snrs + c.r0 * nw, P->d_snrs[j], c.nr * nw * sizeof(float),
                                    cudaMemcpyDeviceToHost, P->s_out));
        RT_TRY_CUDA(cudaEventRecord(P->ev_out_free[j], P->s_out));
    }
    // the last copies out follow every search, which follow every copy in
    RT_TRY_CUDA(cudaEventRecord(P->ev_end, P->s_out));
    RT_TRY_CUDA(cudaStreamWaitEvent(st, P->ev_end, 0));
    return RT_OK;
}

extern "C" int rt_search_pipeline_check(rt_search_pipeline* P, void* stream)
{
    if (!P) return rt::set_error(RT_EINVAL, "null argument");
    RT_TRY_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    for (const Chunk& c : P->chunks) RT_TRY(rt_search_check(c.plan, P->s_run));
    return RT_OK;
}

extern "C" void rt_search_pipeline_destroy(rt_search_pipeline* P)
{
    if (P) cudaDeviceSynchronize();
    pipeline_free(P);
}
