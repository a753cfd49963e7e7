// Batched FFA search engine: many DM trials of uneven length searched in one pass.
//
// Stream of work for one run (all stream-ordered, capturable in a CUDA graph):
//   1. deredden (time_series.py:95-124 / running_medians.py:40-85): mean-scrunch, exact
//      running median of the scrunched series, linear interpolation back, subtraction;
//   2. normalise (time_series.py:67-93): FP64 mean / variance per trial;
//   3. one pass over every series producing the downsampled copy for every octave cycle
//      (normalisation applied on the fly, cpp/periodogram.hpp:153-168);
//   4. one persistent kernel that walks a precomputed list of FFA jobs (ffa_core.cuh) for all
//      (trial, cycle, bins) transforms and writes the periodogram rows (S/N fused).
// Transforms too large for one CTA are split in stages; jobs of a stage wait for the previous
// stage through per-transform counters, and stage-0 jobs wait until their scratch slot is
// released. Every wait is bounded and reports RT_ETIMEOUT instead of hanging.
#include <string.h>

#include <algorithm>
#include <deque>
#include <map>
#include <set>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "ffa_core.cuh"
#include "kernels.cuh"
#include "snr_core.cuh"

namespace rt {

struct XformRec {
    unsigned long long src_off;  // row 0 of the folded series (offset in its arena)
    unsigned long long out_row;  // first periodogram row of this transform
    double tau;                  // sampling time of the folded series
    int b, m, rows_eval;
    float stdnoise;
    int plan;                    // index into the stage-plan table
    int seq;                     // multi-stage sequence number, -1 for single-stage transforms
    int src_norm;                // 1: src is in the normalised series arena, 0: downsampled arena
    int tune;                    // rows per job (low 16 bits), S/N threads per profile (high)
};

struct WorkItem {
    int xform;
    int stage_job;       // stage << 24 | job
};

// Shared-memory layout of the persistent kernel: per item slot (static) a job tree and the
// boxcar coefficients; the dynamic part holds the row operations and two level buffers.
constexpr size_t kEngineTreeBytes = (sizeof(JobTree) + 255) & ~size_t(255);
constexpr size_t kEngineSnrBytes = (sizeof(SnrParams) + 255) & ~size_t(255);
constexpr size_t kEngineDynBytes = kFfaSmemBytes - 2 * (kEngineTreeBytes + kEngineSnrBytes);
RT_HD int engine_cap_rows(int b)
{
    return ffa_cap_rows_for(kEngineDynBytes, 0, b);
}

constexpr int kSlots = 256;          // scratch slots for multi-stage transforms
constexpr size_t kLagItems = 640;    // work items emitted between two stages of a transform
constexpr long long kSpinLimit = 20000000LL;  // default bound of the waits (about 2-20 s with backoff)

struct EngineArgs {
    const float* ds;         // downsampled series arena
    const float* norm;       // normalised series arena (cycles with f == 1)
    float* snrs;
    double* periods;
    uint32_t* foldbins;
    const XformRec* xforms;
    const WorkItem* items;
    long long nitems;
    const StagePlan* plans;
    const int* widths;
    int nw, nfast;
    float* scratch;          // kSlots * 2 * slot_floats
    size_t slot_floats;
    int* done;               // [nseq * kMaxStages]
    int* slot_release;       // [kSlots]
    unsigned long long* ticket;
    int* error;              // RT_OK or an error code
    unsigned long long* phase_cycles;  // optional [kPhases] SM-cycle totals (thread 0 of each CTA)
    long long spin_limit;    // polls before a wait gives up with RT_ETIMEOUT
    int dep_bias;            // added to later-stage dependency targets (fault injection; 0)
};

// Phases of one work item, for the optional in-kernel profile.
enum { kPhFetch = 0, kPhWait, kPhTree, kPhLevels, kPhSnr, kPhStore, kPhases = 8 };
// extra counters after the phases: blocked on a scratch slot, blocked on a previous stage,
// items claimed, scheduler polls that found nothing ready
constexpr int kCounters = 16;

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <int TPR>
__device__ void final_stage_outputs(const JobTree& T, const XformRec& X, const EngineArgs& A,
                                    const SnrParams& S, float* buf0, float* buf1, int fstride,
                                    int cap_rows)
{
    const Node r = T.nodes[0];
    const int b = X.b;
    const int cs = prefix_stride(b, S.wmax, TPR);
    const int groups = (int)(((size_t)cap_rows * fstride) / cs);
    snr_rows<TPR, 34>(buf0, fstride, r.hi - r.lo, b, S, X.stdnoise,
                      A.snrs + ((size_t)X.out_row + r.lo) * S.nw, S.nw, buf1, cs, groups);
    double* per_out = A.periods + X.out_row;
    uint32_t* fb_out = A.foldbins + X.out_row;
    for (int s = r.lo + threadIdx.x; s < r.hi; s += kThreads) {
        per_out[s] = trial_period(X.tau, b, s, X.m);
        fb_out[s] = (uint32_t)b;
    }
}

// The persistent kernel has kThreads compute threads and one scheduling warp. The scheduler
// claims the next ticket, loads its descriptors into one of two shared slots and waits for
// its dependencies while the compute threads work on the other slot; slot hand-over uses
// named barriers (full: scheduler -> compute, empty: compute -> scheduler), one pair per slot.
constexpr int kEngineThreads = kThreads + 32;
constexpr int kBarFull = 2;   // + slot
constexpr int kBarEmpty = 4;  // + slot

struct ItemSlot {
    long long ticket;   // >= nitems: no more work
    int ok;             // 0: a wait failed, stop
    int done_ok;        // set by the compute threads: 0 if the item failed
    int stage, last, cap_rows, jobs_of_stage;
    JobSpec J;
    XformRec X;
};

__device__ __forceinline__ void named_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int n)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Per-slot count of compute warps done with the slot's item: each warp adds 1 with release
// semantics at CTA scope; the scheduling warp reads it with acquire semantics.
__device__ __forceinline__ void warp_done_release(unsigned* counter)
{
    asm volatile("red.release.cta.shared::cta.add.u32 [%0], 1;" ::"r"(smem_u32(counter))
                 : "memory");
}
__device__ __forceinline__ unsigned warps_done_acquire(const unsigned* counter)
{
    unsigned v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(counter))
                 : "memory");
    return v;
}

// Completion of an item for the other CTAs: its stage counter and, after the last job of the
// last stage, the release of the transform's scratch slot. Called by one thread after every
// compute warp of the CTA has released the item (CTA scope); the fence makes their global
// writes visible at GPU scope before the counters.
__device__ __forceinline__ void signal_item_done(const EngineArgs& A, const ItemSlot& P)
{
    if (P.X.seq < 0 || !P.done_ok) return;
    __threadfence();
    int* d = A.done + (size_t)P.X.seq * kMaxStages + P.stage;
    const int prev = atomicAdd(d, 1);
    if (P.last && prev + 1 == P.jobs_of_stage) {
        __threadfence();
        atomicAdd(A.slot_release + (P.X.seq % kSlots), 1);
    }
}

// Scheduler-side view of a claimed item: its slot contents and its dependency.
struct SchedItem {
    ItemSlot slot;
    const int* dep;     // counter to wait for (null: no dependency)
    int target;         // ... until it reaches this value
};

__device__ __forceinline__ bool sched_ready(const SchedItem& it)
{
    return it.dep == nullptr || ld_acquire(it.dep) >= it.target;
}

__device__ void sched_decode(const EngineArgs& A, long long t, SchedItem& it)
{
    ItemSlot& L = it.slot;
    const WorkItem W = A.items[t];
    const XformRec X = A.xforms[W.xform];
    const StagePlan P = A.plans[X.plan];
    const int stage = W.stage_job >> 24, job = W.stage_job & 0xffffff;
    const JobSpec J = stage_job(X.m, X.rows_eval, P, stage, job);
    L.ticket = t;
    L.ok = 1;
    L.X = X;
    L.J = J;
    L.stage = stage;
    L.last = stage == P.nstages - 1;
    L.jobs_of_stage = P.jobs[stage];
    L.cap_rows = X.tune & 0xffff;
    it.dep = nullptr;
    it.target = 0;
    if (J.hi > J.lo && X.seq >= 0) {
        const int seq = X.seq;
        if (stage == 0) {
            it.dep = A.slot_release + (seq % kSlots);
            it.target = seq / kSlots;
        } else {
            it.dep = A.done + (size_t)seq * kMaxStages + stage - 1;
            it.target = P.jobs[stage - 1] + A.dep_bias;
        }
    }
}

// Hands the compute threads one ready item per slot. Items whose dependency is not met yet
// are parked (up to kParked) while later tickets are tried, so a waiting stage does not stall
// the CTA. Progress: the smallest unfinished ticket has all its dependencies finished (they
// have smaller tickets), so whichever scheduler holds it hands it over; every wait is bounded.
constexpr int kParked = 4;

__device__ void scheduler_warp(const EngineArgs& A, ItemSlot* slots, JobTree* trees,
                               SnrParams* snr, unsigned* finished)
{
    const int lane = threadIdx.x & 31;
    SchedItem parked[kParked];
    int nparked = 0;
    bool exhausted = false;
    // items handed over whose completion is not signalled yet (lane 0): signalled as soon as
    // every compute warp has released them, also while this warp waits for a dependency (an
    // item it waits for may be the one running here)
    bool pending[2] = {false, false};
    auto try_signal = [&](int s) {
        if (pending[s] && warps_done_acquire(finished + s) >= (unsigned)kWarps) {
            signal_item_done(A, slots[s]);
            pending[s] = false;
        }
    };
    int k = 0;
    for (;; ++k) {
        const int s = k & 1;
        if (k >= 2) named_sync(kBarEmpty + s, kEngineThreads);  // compute is done with item k-2
        if (lane == 0) {
            try_signal(s);  // item k-2
            ItemSlot& L = slots[s];
            const long long w0 = clock64();
            bool chosen = false;
            unsigned ns = 32;
            for (long long spin = 0; !chosen; ++spin) {
                try_signal(s ^ 1);  // item k-1, running
                for (int i = 0; i < nparked && !chosen; ++i) {
                    if (sched_ready(parked[i])) {
                        L = parked[i].slot;
                        for (int q = i; q + 1 < nparked; ++q) parked[q] = parked[q + 1];
                        --nparked;
                        chosen = true;
                    }
                }
                if (chosen) break;
                if (ld_acquire(A.error) != RT_OK) exhausted = true;
                if (!exhausted && nparked < kParked) {
                    const long long t = (long long)atomicAdd(A.ticket, 1ull);
                    if (t >= A.nitems) {
                        exhausted = true;
                    } else {
                        SchedItem it;
                        sched_decode(A, t, it);
                        if (A.phase_cycles) atomicAdd(A.phase_cycles + 10, 1ull);
                        if (sched_ready(it)) {
                            L = it.slot;
                            chosen = true;
                        } else {
                            if (A.phase_cycles)
                                atomicAdd(A.phase_cycles + (it.slot.stage == 0 ? 8 : 9), 1ull);
                            parked[nparked++] = it;
                        }
                    }
                    continue;
                }
                if (exhausted && (nparked == 0 || ld_acquire(A.error) != RT_OK)) {
                    L.ticket = A.nitems;  // no more work
                    L.ok = 1;
                    chosen = true;
                    break;
                }
                if (spin > A.spin_limit) {
                    atomicExch(A.error, RT_ETIMEOUT);
                    L.ticket = A.nitems;
                    L.ok = 0;
                    chosen = true;
                    break;
                }
                if (A.phase_cycles) atomicAdd(A.phase_cycles + 11, 1ull);
                __nanosleep(ns);
                if (ns < 1024) ns <<= 1;
            }
            if (A.phase_cycles) atomicAdd(A.phase_cycles + 7, (unsigned long long)(clock64() - w0));
            L.done_ok = 1;
            finished[s] = 0;
            __threadfence_block();
        }
        __syncwarp();
        const bool stop = slots[s].ticket >= A.nitems || !slots[s].ok;
        // the job tree and boxcar coefficients of the item, prepared while the compute threads
        // run the previous item
        if (!stop && slots[s].J.hi > slots[s].J.lo) {
            build_job_tree_warp(trees[s], slots[s].J, slots[s].cap_rows, slots[s].stage > 0);
            if (slots[s].last) snr_params_fill_warp(snr[s], A.widths, A.nw, A.nfast, slots[s].X.b);
        }
        named_arrive(kBarFull + s, kEngineThreads);
        if (stop) break;
        if (lane == 0) pending[s] = true;
    }
    // the compute threads still hand back the slot of item k-1
    if (k >= 1) {
        named_sync(kBarEmpty + ((k - 1) & 1), kEngineThreads);
        if (lane == 0) try_signal((k - 1) & 1);
    }
}

// BC: the bins class of the plan's transforms (which unrolled level loops the instance holds);
// TPRS: the S/N threads per profile its transforms use (bit 0: 8, bit 1: 16). The host picks
// the instance (search_kernel_for).
template <int BC, int TPRS>
__global__ void __launch_bounds__(kEngineThreads, 1) k_search_persistent(EngineArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char* layout = smem;
    __shared__ ItemSlot slots[2];
    __shared__ JobTree trees[2];
    __shared__ SnrParams snr[2];
    __shared__ unsigned finished[2];
    __shared__ __align__(8) uint64_t s_bar;  // completion of the bulk copy of a job's rows

    if (threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (threadIdx.x >= kThreads) {
        scheduler_warp(A, slots, trees, snr, finished);
        return;
    }
    uint32_t bar_phase = 0;
    const bool prof = A.phase_cycles != nullptr;
    unsigned long long ph[kPhases] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long cnt[4] = {0, 0, 0, 0};  // counters 12..15
    long long tprev = prof ? clock64() : 0;
    auto mark = [&](int phase) {
        if (prof && threadIdx.x == 0) {
            const long long t = clock64();
            ph[phase] += (unsigned long long)(t - tprev);
            tprev = t;
        }
    };
    for (int k = 0;; ++k) {
        const int sl = k & 1;
        named_sync(kBarFull + sl, kEngineThreads);
        mark(kPhWait);
        const ItemSlot& L = slots[sl];
        const JobTree& T = trees[sl];
        const SnrParams& S = snr[sl];
        if (L.ticket >= A.nitems || !L.ok) break;
        const XformRec X = L.X;
        const JobSpec J = L.J;
        const int stage = L.stage;
        const bool last = L.last != 0;
        const int b = X.b;
        const int fstride = ffa_stride(b);
        const int cap_rows = L.cap_rows;
        const FfaSmem Lay = ffa_smem(layout, cap_rows, b);
        float* slot = (X.seq >= 0) ? A.scratch + (size_t)(X.seq % kSlots) * 2 * A.slot_floats
                                   : nullptr;
        mark(6);
        mark(kPhFetch);
        bool failed = false;
        if (J.hi > J.lo) {
            const float* src =
                (stage == 0) ? (X.src_norm ? A.norm : A.ds) + X.src_off
                             : slot + (size_t)((stage - 1) & 1) * A.slot_floats;
            LevelIO io;
            io.src = src;
            io.src_stride = (stage == 0) ? b : fstride;  // stage outputs: level stride
            io.bar = &s_bar;
            io.phase = &bar_phase;
            // Level G's source rows are copied (bulk copies) into the level buffer that level G
            // does not write, in the background of the row-operation build: for stage-0 jobs
            // (whole subtrees) one contiguous block of the downsampled arena (padded); for
            // later stages the blocks of the previous stage's output that the cone needs.
            float* sbuf = (J.G & 1) ? Lay.buf0 : Lay.buf1;
            const bool staged0 = stage == 0 && !X.src_norm && J.root_rows <= cap_rows &&
                                 (size_t)J.root_rows * b + 8 <= (size_t)cap_rows * fstride;
            const bool staged = staged0 || (stage > 0 && T.pstaged && !T.error);
            if (staged0) {
                __shared__ int s_delta;
                if (threadIdx.x == 0)
                    s_delta = stage_rows_async(sbuf, src + (size_t)J.root_row0 * b,
                                               (size_t)J.root_rows * b, &s_bar);
                cta_sync();
                io.staged = sbuf + s_delta - (ptrdiff_t)J.root_row0 * b;
            } else if (staged) {
                if (threadIdx.x < 32) stage_source_rows_async(T, src, fstride, sbuf, &s_bar);
                io.staged = sbuf;
                io.staged_rows = true;
            }
            failed = T.error != 0;
            if (failed) {
                if (threadIdx.x == 0) atomicExch(A.error, RT_EINTERNAL);
                if (staged) {  // still let the copy land before the buffer is reused
                    mbar_wait(&s_bar, bar_phase);
                    bar_phase ^= 1u;
                }
            } else {
                mark(kPhTree);
                if (prof && threadIdx.x == 0) {
                    for (int d = 0; d <= T.depth; ++d)
                        cnt[0] += (unsigned long long)T.level_rows[d] * b;
                    cnt[1] += T.depth + 1;
                    cnt[2] += J.hi - J.lo;
                    cnt[3] += stage > 0;
                }
                // stage outputs other than the last are written by the root level itself
                if (!last) {
                    io.root_dst =
                        root_rows_dst(T, fstride, slot + (size_t)(stage & 1) * A.slot_floats);
                    io.root_stride = fstride;
                }
                if (!run_job_levels<BC>(T, b, Lay.buf0, Lay.buf1, fstride, Lay.ops, io)) {
                    if (threadIdx.x == 0) atomicExch(A.error, RT_ETIMEOUT);
                }
                mark(kPhLevels);
                if (last) {
                    if constexpr (TPRS == 1)
                        final_stage_outputs<8>(T, X, A, S, Lay.buf0, Lay.buf1, fstride, cap_rows);
                    else if constexpr (TPRS == 2)
                        final_stage_outputs<16>(T, X, A, S, Lay.buf0, Lay.buf1, fstride, cap_rows);
                    else if ((X.tune >> 16) == 8)
                        final_stage_outputs<8>(T, X, A, S, Lay.buf0, Lay.buf1, fstride, cap_rows);
                    else
                        final_stage_outputs<16>(T, X, A, S, Lay.buf0, Lay.buf1, fstride, cap_rows);
                    mark(kPhSnr);
                }
            }
        }
        // hand the item back: the scheduling warp signals its completion to the other CTAs
        // once every compute warp has released it
        if (threadIdx.x == 0 && failed) slots[sl].done_ok = 0;
        __syncwarp();
        if ((threadIdx.x & 31) == 0) warp_done_release(finished + sl);
        mark(kPhStore);
        named_arrive(kBarEmpty + sl, kEngineThreads);
    }
    if (prof && threadIdx.x == 0)
        for (int i = 0; i < kPhases; ++i) atomicAdd(A.phase_cycles + i, ph[i]);
    if (prof && threadIdx.x == 0)
        for (int i = 0; i < 4; ++i) atomicAdd(A.phase_cycles + 12 + i, cnt[i]);
}

// ------------------------------------------------------------------------------------
// Deredden / normalise (batched)
// ------------------------------------------------------------------------------------
struct TrialArrays {
    const size_t* len;       // [T]
    const size_t* off;       // [T] offsets into the packed series
    const size_t* lo_len;    // [T] scrunched lengths
    const size_t* lo_off;    // [T] offsets into the packed scrunched series
};

// ---- numpy's pairwise summation -----------------------------------------------------
// The reference's scrunch is `data[:N].reshape(-1, k).mean(axis=1)` on float32 data
// (running_medians.py:40-46). numpy reduces each contiguous row with its pairwise sum in the
// input type (numpy/_core/src/umath/loops_utils.h.src, pairwise_sum): a block of n < 8
// values is summed in turn from -0.0; a block of 8 <= n <= 128 values in eight strided
// accumulators r[j] = a[j] + a[j+8] + ... over its first n - n%8 values, combined as
// ((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), with the n%8 trailing values then added in turn; a
// longer block is split at n2 = n/2 - (n/2)%8 and the two halves' sums are added. The mean is
// that float32 sum divided by k, correctly rounded (numpy divides in float64 and casts; a
// float64 quotient of float32 operands rounds to float32 exactly as a float32 division).
// Reproduced here in the same order, so the scrunched series is bit-identical.
constexpr int kPwLeaf = 128;

// Leaves (blocks of <= 128 values) of the recursion over n values, left to right.
static int pw_num_leaves(long long n)
{
    if (n <= kPwLeaf) return 1;
    long long n2 = n / 2;
    n2 -= n2 % 8;
    return pw_num_leaves(n2) + pw_num_leaves(n - n2);
}

// Fills leaves[] with (start, length) in recursion (left to right) order; explicit stack.
__device__ void pw_leaf_table(int n, int2* leaves)
{
    int st_s[40], st_n[40];
    int sp = 0, nl = 0;
    st_s[sp] = 0;
    st_n[sp++] = n;
    while (sp > 0) {
        --sp;
        const int s = st_s[sp], m = st_n[sp];
        if (m <= kPwLeaf) {
            leaves[nl++] = make_int2(s, m);
            continue;
        }
        int m2 = m / 2;
        m2 -= m2 % 8;
        // right half pushed first, so the left half is popped (and emitted) first
        st_s[sp] = s + m2;
        st_n[sp++] = m - m2;
        st_s[sp] = s;
        st_n[sp++] = m2;
    }
}

// Adds the leaf sums up the recursion tree of n values in numpy's order (left + right at
// every split); leaf sums are consumed left to right.
__device__ float pw_combine(const float* leaf_sums, int n)
{
    int fn[40], fstate[40];
    float fleft[40];
    int sp = 0, li = 0;
    float ret = 0.0f;
    fn[0] = n;
    fstate[0] = 0;
    sp = 1;
    while (sp > 0) {
        const int t = sp - 1;
        const int m = fn[t];
        if (m <= kPwLeaf) {
            ret = leaf_sums[li++];
            --sp;
            continue;
        }
        int m2 = m / 2;
        m2 -= m2 % 8;
        if (fstate[t] == 0) {  // descend left
            fstate[t] = 1;
            fn[sp] = m2;
            fstate[sp++] = 0;
        } else if (fstate[t] == 1) {  // left done: descend right
            fleft[t] = ret;
            fstate[t] = 2;
            fn[sp] = m - m2;
            fstate[sp++] = 0;
        } else {  // both done
            ret = __fadd_rn(fleft[t], ret);
            --sp;
        }
    }
    return ret;
}

// The additions of the recursion tree of n values as a program: nodes 0 .. L-1 are the leaves
// (left to right), node L + q = node prog[q].x + node prog[q].y, in the order numpy adds
// them (children before parents); the root is node 2L - 2 (node 0 when L = 1).
__device__ void pw_program(int n, int2* prog)
{
    int fn[40], fstate[40], fleft[40];
    int sp = 1, li = 0, q = 0, ret = 0;
    fn[0] = n;
    fstate[0] = 0;
    int nleaves = 0;
    // first pass: count leaves (node ids of internal nodes start after them)
    {
        int gn[40], gs[40], gp = 1;
        gn[0] = n;
        gs[0] = 0;
        while (gp > 0) {
            const int t = gp - 1, m = gn[t];
            if (m <= kPwLeaf) {
                ++nleaves;
                --gp;
                continue;
            }
            int m2 = m / 2;
            m2 -= m2 % 8;
            if (gs[t] == 0) {
                gs[t] = 1;
                gn[gp] = m2;
                gs[gp++] = 0;
            } else if (gs[t] == 1) {
                gs[t] = 2;
                gn[gp] = m - m2;
                gs[gp++] = 0;
            } else {
                --gp;
            }
        }
    }
    while (sp > 0) {
        const int t = sp - 1;
        const int m = fn[t];
        if (m <= kPwLeaf) {
            ret = li++;
            --sp;
            continue;
        }
        int m2 = m / 2;
        m2 -= m2 % 8;
        if (fstate[t] == 0) {
            fstate[t] = 1;
            fn[sp] = m2;
            fstate[sp++] = 0;
        } else if (fstate[t] == 1) {
            fleft[t] = ret;
            fstate[t] = 2;
            fn[sp] = m - m2;
            fstate[sp++] = 0;
        } else {
            prog[q] = make_int2(fleft[t], ret);
            ret = nleaves + q;
            ++q;
            --sp;
        }
    }
}

// Scrunch for factors whose recursion has at most 32 leaves (k up to a few thousand): a warp
// takes 32 scrunched points at a time; its four 8-lane groups compute their leaves (one leaf
// per group per step, one strided accumulator per lane), then every lane adds up one
// point's leaves along the program above, so the additions of 32 points run side by side.
// Dynamic shared memory: leaf table, program, and per warp 32 points x (2L - 1) node values.
constexpr int kScrunchBatchLeaves = 32;

__global__ void k_scrunch_batched(const float* __restrict__ x, TrialArrays A, int k, int nleaves,
                                  float* __restrict__ lores)
{
    extern __shared__ __align__(16) unsigned char sm_scb[];
    int2* leaves = reinterpret_cast<int2*>(sm_scb);
    int2* prog = leaves + nleaves;
    const int nn = 2 * nleaves - 1, vs = nn | 1;  // odd per-point stride: no bank conflicts
    float* V = reinterpret_cast<float*>(prog + nleaves) + (threadIdx.x >> 5) * 32 * vs;
    if (threadIdx.x == 0) {
        pw_leaf_table(k, leaves);
        pw_program(k, prog);
    }
    __syncthreads();
    const int trial = blockIdx.y;
    const size_t nl = A.lo_len[trial];
    const float* xr = x + A.off[trial];
    float* o = lores + A.lo_off[trial];
    const int lane = threadIdx.x & 31;
    const int grp = lane >> 3, c = lane & 7;
    const size_t w0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nwarp = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t p0 = w0 * 32; p0 < nl; p0 += nwarp * 32) {
        const int np = (int)min((size_t)32, nl - p0);
        const int tasks = np * nleaves;
        for (int u0 = 0; u0 < tasks; u0 += 4) {
            const int u = u0 + grp;
            const bool ok = u < tasks;
            const int pt = ok ? u / nleaves : 0, l = ok ? u - pt * nleaves : 0;
            const float* a = xr + (p0 + pt) * (size_t)k;
            float v = 0.0f;
            int2 lf = make_int2(0, 0);
            if (ok) {
                lf = leaves[l];
                if (lf.y >= 8) {
                    const int full = lf.y - lf.y % 8;
                    v = __ldg(a + lf.x + c);
                    for (int i = 8; i < full; i += 8) v = __fadd_rn(v, __ldg(a + lf.x + i + c));
                }
            }
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 1));
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 2));
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 4));
            if (ok && c == 0) {
                int i = lf.y - lf.y % 8;
                if (lf.y < 8) {
                    v = -0.0f;
                    i = 0;
                }
                for (; i < lf.y; ++i) v = __fadd_rn(v, __ldg(a + lf.x + i));
                V[pt * vs + l] = v;
            }
        }
        __syncwarp();
        if (lane < np) {
            float* Vp = V + lane * vs;
            for (int q = 0; q + 1 < nleaves; ++q) {
                const int2 ab = prog[q];
                Vp[nleaves + q] = __fadd_rn(Vp[ab.x], Vp[ab.y]);
            }
            o[p0 + lane] = __fdiv_rn(Vp[nn - 1], (float)k);
        }
        __syncwarp();
    }
}

// lores[j] = float32 mean of x[j*k .. (j+1)*k), numpy's pairwise order (see above).
// One warp per scrunched value; the warp's four 8-lane groups take one leaf each, a lane
// one of the eight strided accumulators; lane 0 adds the leaf sums up the tree.
// Dynamic shared memory: the leaf table (int2 per leaf) and one leaf-sum row per warp.
__global__ void k_scrunch(const float* __restrict__ x, TrialArrays A, int k, int nleaves,
                          float* __restrict__ lores)
{
    extern __shared__ __align__(16) unsigned char sm_scrunch[];
    int2* leaves = reinterpret_cast<int2*>(sm_scrunch);
    float* sums = reinterpret_cast<float*>(leaves + nleaves) + (threadIdx.x >> 5) * nleaves;
    if (threadIdx.x == 0) pw_leaf_table(k, leaves);
    __syncthreads();
    const int trial = blockIdx.y;
    const size_t nl = A.lo_len[trial];
    const float* xr = x + A.off[trial];
    float* o = lores + A.lo_off[trial];
    const int lane = threadIdx.x & 31;
    const int grp = lane >> 3, c = lane & 7;
    const size_t w0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nwarp = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t j = w0; j < nl; j += nwarp) {
        const float* a = xr + j * (size_t)k;
        for (int l0 = 0; l0 < nleaves; l0 += 4) {
            const int l = l0 + grp;
            float v = 0.0f;
            int2 lf = make_int2(0, 0);
            if (l < nleaves) {
                lf = leaves[l];
                if (lf.y >= 8) {
                    const int full = lf.y - lf.y % 8;
                    v = __ldg(a + lf.x + c);
                    for (int i = 8; i < full; i += 8) v = __fadd_rn(v, __ldg(a + lf.x + i + c));
                }
            }
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 1));
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 2));
            v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, 4));
            if (l < nleaves && c == 0) {
                int i = lf.y - lf.y % 8;
                if (lf.y < 8) {
                    v = -0.0f;
                    i = 0;
                }
                for (; i < lf.y; ++i) v = __fadd_rn(v, __ldg(a + lf.x + i));
                sums[l] = v;
            }
        }
        __syncwarp();
        if (lane == 0) o[j] = __fdiv_rn(pw_combine(sums, k), (float)k);
        __syncwarp();
    }
}

// Launch shape of k_scrunch for factor k: 256 threads while the leaf table and eight
// leaf-sum rows fit 48 KB, fewer warps above that (up to the opt-in shared-memory size).
static int launch_scrunch(const float* x, const TrialArrays& A, int k, int ntrials,
                          size_t max_lo, float* lores, cudaStream_t st)
{
    const int nleaves = pw_num_leaves(k);
    if (nleaves <= kScrunchBatchLeaves) {
        // 8 warps, each with 32 points x (2L - 1) node values
        const size_t smem = 2 * (size_t)nleaves * sizeof(int2) +
                            8 * 32 * (size_t)((2 * nleaves - 1) | 1) * sizeof(float);
        const size_t per_trial = std::max<size_t>(8, 4096 / (size_t)std::max(ntrials, 1));
        dim3 g((unsigned)std::max<size_t>(1, std::min<size_t>((max_lo + 255) / 256, per_trial)),
               (unsigned)ntrials);
        if (smem > 48 * 1024)
            RT_TRY_CUDA(cudaFuncSetAttribute(k_scrunch_batched,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_scrunch_batched<<<g, 256, smem, st>>>(x, A, k, nleaves, lores);
        return check_cuda(cudaGetLastError(), "scrunch");
    }
    const size_t per_warp = (size_t)nleaves * sizeof(float);
    const size_t table = (size_t)nleaves * sizeof(int2);
    int warps = 8;
    while (warps > 1 && table + warps * per_warp > 48 * 1024) warps >>= 1;
    const size_t smem = table + warps * per_warp;
    if (smem > 200 * 1024) return set_error(RT_EINVAL, "scrunch factor too large");
    if (smem > 48 * 1024)
        RT_TRY_CUDA(cudaFuncSetAttribute(k_scrunch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    const unsigned threads = 32u * warps;
    // every CTA builds the leaf table first, so CTAs are few and long-lived: about 8192 in
    // all (at least 16 per series), each warp taking many points
    const size_t per_trial = std::max<size_t>(16, 8192 / (size_t)std::max(ntrials, 1));
    dim3 g((unsigned)std::max<size_t>(1, std::min<size_t>((max_lo + 63) / 64, per_trial)),
           (unsigned)ntrials);
    k_scrunch<<<g, threads, smem, st>>>(x, A, k, nleaves, lores);
    return check_cuda(cudaGetLastError(), "scrunch");
}

constexpr int kStatThreads = 256;

// Unsigned 32-bit division by an invariant divisor d >= 1 with one multiply-high
// (Granlund & Montgomery, "Division by invariant integers using multiplication", PLDI 1994,
// figure 4.1): l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// q = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0) with t = mulhi(m, n); exact for every
// 32-bit n.
struct DivMagic {
    unsigned m;
    int sh1, sh2;
};

inline DivMagic div_magic(unsigned d)
{
    int l = 0;
    while ((1ull << l) < d) ++l;
    DivMagic g;
    g.m = (unsigned)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    g.sh1 = l < 1 ? l : 1;
    g.sh2 = l - 1 > 0 ? l - 1 : 0;
    return g;
}

__device__ __forceinline__ unsigned div_by_magic(unsigned n, const DivMagic& g)
{
    const unsigned t = __umulhi(g.m, n);
    return (t + ((n - t) >> g.sh1)) >> g.sh2;
}

// np.interp coefficients of the scrunched running median (running_medians.py:82-85):
// coef[j] = (fp[j], (fp[j+1] - fp[j]) / k) in float64, so that the interpolated value at
// x = j*k + (k-1)/2 + dx is fp[j] + slope * dx as numpy evaluates it.
__global__ void k_interp_coef(TrialArrays A, int k, const float* __restrict__ rmed,
                              double2* __restrict__ coef)
{
    const int trial = blockIdx.y;
    const size_t nl = A.lo_len[trial];
    const float* fp = rmed + A.lo_off[trial];
    double2* c = coef + A.lo_off[trial];
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < nl;
         j += (size_t)gridDim.x * blockDim.x) {
        const double a = (double)fp[j];
        const double s = (j + 1 < nl) ? __ddiv_rn(__dsub_rn((double)fp[j + 1], a), (double)k) : 0.0;
        c[j] = make_double2(a, s);
    }
}

// y = float32(x - running median); per-block shifted sums for the statistics.
// k > 1: rmed = np.interp(i, j*k + (k-1)/2, rmed_lores) in float64 (running_medians.py:82-85),
// from the coefficients of k_interp_coef; with v = 2i - (k-1) = 2k*j + 2*dx, the segment j
// and the offset dx = v mod 2k / 2 come from one invariant division (exact in 32 bits while
// 2N < 2^32; longer series take 64-bit division);
// k == 1: rmed is the full-resolution float32 running median (float32 subtraction).
__global__ void __launch_bounds__(kStatThreads)
    k_dered(const float* __restrict__ x, TrialArrays A, int k, DivMagic g2k,
            const float* __restrict__ rmed, const double2* __restrict__ coef,
            float* __restrict__ y, double* __restrict__ part, int blocks_per_trial)
{
    const int trial = blockIdx.y;
    const size_t N = A.len[trial];
    const float* xr = x + A.off[trial];
    float* yr = y + A.off[trial];
    const float* fp = rmed + (k > 1 ? A.lo_off[trial] : A.off[trial]);
    const double2* cf = coef + (k > 1 ? A.lo_off[trial] : 0);
    const size_t nl = A.lo_len[trial];
    double s1 = 0.0, s2 = 0.0;
    const float shift = xr[0];
    float shift_y;
    {
        // shift for the sums: y[0]
        double r0;
        if (k > 1) r0 = (double)fp[0];  // x = 0 <= xp[0]
        else r0 = 0.0;
        shift_y = (k > 1) ? __double2float_rn((double)shift - r0) : __fsub_rn(shift, fp[0]);
    }
    const double shift_yd = (double)shift_y;
    // v = 2i - (k-1) ranges: v < 0 is left of xp[0]; v >= 2k(nl-1) is at or right of xp[-1]
    const long long vlast = 2LL * k * (long long)(nl - 1);
    const bool small = 2 * (unsigned long long)N < (1ull << 32);
    const double first = (k > 1) ? (double)fp[0] : 0.0;
    const double last = (k > 1) ? (double)fp[nl - 1] : 0.0;
    auto body = [&](size_t i, float xv) {
        float yv;
        if (k > 1) {
            const long long v = 2LL * (long long)i - (k - 1);
            double r;
            if (v < 0) {
                r = first;
            } else if (v >= vlast) {
                r = last;
            } else {
                long long j;
                if (small) j = (long long)div_by_magic((unsigned)v, g2k);
                else j = v / (2LL * k);
                const int twodx = (int)(v - j * 2LL * k);  // 2 (x - xp[j]), 0 <= . < 2k
                const double2 c = cf[j];
                // x - xp[j] is exact in double; numpy's interp returns fp[j] at x == xp[j]
                r = (twodx == 0) ? c.x : __dadd_rn(__dmul_rn(c.y, 0.5 * (double)twodx), c.x);
            }
            yv = __double2float_rn(__dsub_rn((double)xv, r));
        } else {
            yv = __fsub_rn(xv, fp[i]);
        }
        yr[i] = yv;
        const double d = (double)yv - shift_yd;
        s1 += d;
        s2 += d * d;
    };
    // four grid-stride steps per pass with their loads issued first; the sums keep the
    // order of the plain loop
    const size_t stride = (size_t)blocks_per_trial * blockDim.x;
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    for (; i + 3 * stride < N; i += 4 * stride) {
        float xv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) xv[q] = xr[i + q * stride];
#pragma unroll
        for (int q = 0; q < 4; ++q) body(i + q * stride, xv[q]);
    }
    for (; i < N; i += stride) body(i, xr[i]);
    // block reduction (fixed order)
    __shared__ double r1[kStatThreads], r2[kStatThreads];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int o = kStatThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            r1[threadIdx.x] += r1[threadIdx.x + o];
            r2[threadIdx.x] += r2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* p = part + ((size_t)trial * blocks_per_trial + blockIdx.x) * 3;
        p[0] = r1[0];
        p[1] = r2[0];
        p[2] = (double)shift_y;
    }
}

// Same statistics without deredden (normalise only).
__global__ void __launch_bounds__(kStatThreads)
    k_sums(const float* __restrict__ x, TrialArrays A, double* __restrict__ part,
           int blocks_per_trial)
{
    const int trial = blockIdx.y;
    const size_t N = A.len[trial];
    const float* xr = x + A.off[trial];
    const float shift = xr[0];
    double s1 = 0.0, s2 = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)blocks_per_trial * blockDim.x) {
        const double d = (double)xr[i] - (double)shift;
        s1 += d;
        s2 += d * d;
    }
    __shared__ double r1[kStatThreads], r2[kStatThreads];
    r1[threadIdx.x] = s1;
    r2[threadIdx.x] = s2;
    __syncthreads();
    for (int o = kStatThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            r1[threadIdx.x] += r1[threadIdx.x + o];
            r2[threadIdx.x] += r2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double* p = part + ((size_t)trial * blocks_per_trial + blockIdx.x) * 3;
        p[0] = r1[0];
        p[1] = r2[0];
        p[2] = (double)shift;
    }
}

// mean and standard deviation per trial (population variance, ddof = 0).
__global__ void k_stats(const double* __restrict__ part, const size_t* __restrict__ len,
                        int blocks_per_trial, int ntrials, double* __restrict__ mean,
                        double* __restrict__ norm)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntrials) return;
    double s1 = 0.0, s2 = 0.0, shift = 0.0;
    for (int b = 0; b < blocks_per_trial; ++b) {
        const double* p = part + ((size_t)t * blocks_per_trial + b) * 3;
        s1 += p[0];
        s2 += p[1];
        shift = p[2];
    }
    const double N = (double)len[t];
    const double d = s1 / N;
    const double var = s2 / N - d * d;
    mean[t] = shift + d;
    norm[t] = sqrt(var);
}

// fast_running_median output (running_medians.py:82-85): float64 interpolation of the
// scrunched running median back to every sample.
__global__ void k_interp_rmed(TrialArrays A, int k, const float* __restrict__ rmed,
                              double* __restrict__ out)
{
    const int trial = blockIdx.y;
    const size_t N = A.len[trial];
    const float* fp = rmed + A.lo_off[trial];
    const size_t nl = A.lo_len[trial];
    double* o = out + A.off[trial];
    const double half = 0.5 * (double)(k - 1);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        const double xi = (double)i;
        const double xl = (double)(nl - 1) * k + half;
        double r;
        if (xi < half) {
            r = (double)fp[0];
        } else if (xi >= xl) {
            r = (double)fp[nl - 1];
        } else {
            const long long j = (2LL * (long long)i - (k - 1)) / (2LL * k);
            const double xj = (double)j * k + half;
            if (xj == xi) {
                r = (double)fp[j];
            } else {
                const double slope =
                    __ddiv_rn(__dsub_rn((double)fp[j + 1], (double)fp[j]), (double)k);
                r = __dadd_rn(__dmul_rn(slope, __dsub_rn(xi, xj)), (double)fp[j]);
            }
        }
        o[i] = r;
    }
}

// z = float32((x - mean) / norm) in float64 (time_series.py:91-93).
__global__ void k_normalise(const float* __restrict__ x, TrialArrays A, const double* mean,
                            const double* norm, float* __restrict__ z)
{
    const int trial = blockIdx.y;
    const size_t N = A.len[trial];
    const float* xr = x + A.off[trial];
    float* zr = z + A.off[trial];
    const double m = mean[trial], s = norm[trial];
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x)
        zr[i] = __double2float_rn(__ddiv_rn(__dsub_rn((double)xr[i], m), s));
}

// ------------------------------------------------------------------------------------
// Plan
// ------------------------------------------------------------------------------------
struct SearchPlan {
    // configuration
    rt_search_config cfg;
    rt_search_tuning tuning = {1.0, 0, 0, 0.0};
    std::vector<rt_tile_rule> rules;    // per (rows, bins) tile choices, first match wins
    std::vector<int> widths;
    int nfast = 0;
    int bins_used[2] = {1 << 30, 0};  // smallest and largest b of the transforms
    int tpr_mask = 0;                 // S/N threads per profile used: bit 0 = 8, bit 1 = 16
    std::vector<size_t> lengths, offsets;
    size_t total_len = 0, max_len = 0;
    // cycles (cpp/periodogram.hpp:135-158)
    std::vector<double> f, tau, pms;
    std::vector<int> use_seg, skip;
    // per trial
    std::vector<size_t> out_rows_off;   // [T+1]
    std::vector<size_t> ds_off;         // [T * C] offsets into the downsample arena
    size_t ds_total = 0;
    bool has_unit_factor = false;       // a cycle folds the series itself (f == 1)
    // deredden
    int scrunch = 1, rmed_width = 0;
    std::vector<size_t> lo_len, lo_off;
    size_t lo_total = 0, max_lo = 0;
    // work
    std::vector<StagePlan> plans;
    std::vector<XformRec> xforms;
    std::vector<int2> xform_tc;          // (trial, cycle) of each transform
    std::vector<WorkItem> items;
    int nseq = 0;
    size_t slot_floats = 0;
    // device buffers
    bool dev_ready = false;
    int* d_widths = nullptr;
    XformRec* d_xforms = nullptr;
    WorkItem* d_items = nullptr;
    StagePlan* d_plans = nullptr;
    float* d_scratch = nullptr;
    int* d_counters = nullptr;          // done + slot_release + error
    unsigned long long* d_ticket = nullptr;
    float* d_ds = nullptr;
    float* d_y = nullptr;               // dereddened series
    float* d_norm = nullptr;            // normalised copy (when a cycle has f == 1)
    float* d_lores = nullptr;
    double2* d_coef = nullptr;          // interpolation coefficients of the running median
    float* d_rmed = nullptr;
    double* d_part = nullptr;
    double* d_mean = nullptr;
    double* d_normv = nullptr;
    size_t* d_len = nullptr;
    size_t* d_off = nullptr;
    size_t* d_lo_len = nullptr;
    size_t* d_lo_off = nullptr;
    double* d_f = nullptr;
    int* d_useseg = nullptr;
    size_t* d_dsoff = nullptr;
    int stat_blocks = 64;
    // optional per-stage CUDA-event timing: deredden+normalise, downsample, FFA + S/N
    bool timing = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    unsigned long long* d_phase = nullptr;  // in-kernel phase profile (optional)
    int launches_last_run = 0;
    // replay of the whole run as one CUDA graph (optional); the graph is keyed on the
    // run's device pointers and captured again when they change
    bool use_graph = false;
    // bounded waits and fault injection (rt_search_set_wait_limit, rt_search_inject_fault)
    long long spin_limit = kSpinLimit;
    int dep_bias = 0;
    int alloc_fail_at = 0;   // 1-based device allocation that fails; 0: none
    int alloc_calls = 0;
    cudaGraphExec_t gexec = nullptr;
    cudaStream_t cap_stream = nullptr;
    const void* gkey[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int graph_captures = 0;
};

static int plan_cycles(SearchPlan& P)
{
    const rt_search_config& c = P.cfg;
    // periodogram.hpp:25-40, same messages and order
    if (!(c.tsamp > 0)) return set_error(RT_EINVAL, "tsamp must be > 0");
    if (!(c.period_min > 0)) return set_error(RT_EINVAL, "period_min must be > 0");
    if (!(c.period_max > c.period_min)) return set_error(RT_EINVAL, "period_max must be > period_min");
    if (!(c.bins_min > 1)) return set_error(RT_EINVAL, "bins_min must be > 1");
    if (!(c.bins_max >= c.bins_min)) return set_error(RT_EINVAL, "bins_max must be >= bins_min");
    if (!(c.period_min >= c.tsamp * c.bins_min))
        return set_error(RT_EINVAL, "Must have: period_min >= tsamp * bins_min ");
    if (c.bins_max > 4096) return set_error(RT_EINVAL, "bins_max above 4096 is not supported");
    const double ds_ini = c.period_min / (c.tsamp * c.bins_min);
    const double ds_geo = (c.bins_max + 1.0) / c.bins_min;
    const size_t nds = (size_t)ceil(log(c.period_max / c.period_min) / log(ds_geo));
    if (nds > (size_t)kDsMaxCycles)
        return set_error(RT_EINVAL, "too many downsampling cycles (%zu)", nds);
    for (size_t i = 0; i < nds; ++i) {
        const double f = ds_ini * pow(ds_geo, (double)i);
        P.f.push_back(f);
        P.tau.push_back(f * c.tsamp);
        P.pms.push_back(c.period_max / (f * c.tsamp));
        P.skip.push_back(f == 1 ? 1 : 0);
        P.use_seg.push_back((f != 1 && ds_use_segments(f)) ? 1 : 0);
        if (f == 1) P.has_unit_factor = true;
    }
    return RT_OK;
}

// Emits the work items of all transforms. Order: (trial, cycle, bins). For a transform that
// needs several stages, stage s + 1 is emitted at least kLagItems items after stage s, so that
// by the time a CTA takes it the previous stage has usually completed; the transform that
// reuses a scratch slot starts only after every stage of the previous occupant is emitted.
static int plan_build(SearchPlan& P)
{
    RT_TRY(plan_cycles(P));
    const rt_search_config& c = P.cfg;
    const int T = (int)P.lengths.size();
    const int C = (int)P.f.size();
    P.out_rows_off.assign(T + 1, 0);
    P.ds_off.assign((size_t)T * C, 0);
    std::map<std::pair<int, long long>, int> plan_index;
    const size_t lag_items = P.tuning.lag_items > 0 ? (size_t)P.tuning.lag_items : kLagItems;
    std::set<std::tuple<size_t, int, int>> deferred;  // (due item count, xform, stage)
    std::vector<int> seq_xform;                        // xform of each multi-stage sequence
    std::vector<std::tuple<size_t, int, int>> seq_pending;  // its deferred entry, if any
    std::vector<char> seq_has_pending;

    auto emit_stage = [&](int xi, int stage) {
        const StagePlan& sp = P.plans[P.xforms[xi].plan];
        for (int j = 0; j < sp.jobs[stage]; ++j) P.items.push_back({xi, (stage << 24) | j});
        const int seq = P.xforms[xi].seq;
        if (seq >= 0) {
            if (stage + 1 < sp.nstages) {
                auto e = std::make_tuple(P.items.size() + lag_items, xi, stage + 1);
                deferred.insert(e);
                seq_pending[seq] = e;
                seq_has_pending[seq] = 1;
            } else {
                seq_has_pending[seq] = 0;
            }
        }
    };
    auto flush = [&]() {
        while (!deferred.empty() && std::get<0>(*deferred.begin()) <= P.items.size()) {
            const auto e = *deferred.begin();
            deferred.erase(deferred.begin());
            emit_stage(std::get<1>(e), std::get<2>(e));
        }
    };
    auto finish_seq = [&](int seq) {  // emit all remaining stages of `seq` now
        while (seq_has_pending[seq]) {
            const auto e = seq_pending[seq];
            deferred.erase(e);
            emit_stage(std::get<1>(e), std::get<2>(e));
        }
    };

    size_t ds_total = 0;
    for (int t = 0; t < T; ++t) {
        const size_t N = P.lengths[t];
        size_t rows_total = 0;
        for (int ci = 0; ci < C; ++ci) {
            const double f = P.f[ci];
            const size_t n = downsampled_size(N, f);
            if (f != 1) {
                // downsample.hpp:11-16 (the reference downsamples every cycle)
                if (!((f > 1.0) && (f <= (double)N)))
                    return set_error(RT_EINVAL, "Downsampling factor must verify: 1 < f <= size");
                P.ds_off[(size_t)t * C + ci] = ds_total;
                ds_total += n;
            }
            const size_t bstop = std::min({(size_t)c.bins_max, n, (size_t)P.pms[ci]});
            for (size_t b = c.bins_min; b <= bstop; ++b) {
                const size_t rows = n / b;
                const size_t re = rows_to_evaluate(rows, b, P.pms[ci]);
                if (re == 0) continue;
                if (rows >= (1u << 24))
                    return set_error(RT_EINVAL, "transform of %zu rows is too large", rows);
                // rows per job: the shared-memory capacity, scaled by the tuning (its own
                // fraction for transforms of more than 8 jobs' worth of rows)
                const int cap_full = engine_cap_rows((int)b);
                double frac = P.tuning.rows_fraction > 0 ? std::min(1.0, P.tuning.rows_fraction) : 1.0;
                if (rows > 8 * (size_t)cap_full && P.tuning.rows_fraction_deep > 0)
                    frac = std::min(1.0, P.tuning.rows_fraction_deep);
                int tune_tpr = P.tuning.snr_threads, max_depth = kMaxJobDepth;
                for (const rt_tile_rule& R : P.rules) {
                    if (rows < R.rows_min || rows > R.rows_max || b < R.bins_min || b > R.bins_max)
                        continue;
                    if (R.rows_fraction > 0) frac = std::min(1.0, R.rows_fraction);
                    if (R.snr_threads) tune_tpr = R.snr_threads;
                    if (R.max_levels) max_depth = R.max_levels - 1;
                    break;
                }
                const int capr = std::max(4, (int)((double)cap_full * frac));
                // S/N threads per profile: 8 where the register window allows it, unless tuned
                const int tpr = (tune_tpr == 16) ? 16 : snr_tpr((int)b);
                const auto key = std::make_pair((int)rows, (long long)re * 8192 + (long long)b);
                int pi;
                auto itp = plan_index.find(key);
                if (itp == plan_index.end()) {
                    StagePlan sp;
                    // a rule's level count that needs more stages than a plan holds falls back
                    // to the default depth
                    if (capr < 4 || (!plan_stages((int)rows, (int)re, capr, &sp, max_depth) &&
                                     !plan_stages((int)rows, (int)re, capr, &sp)))
                        return set_error(RT_EINVAL, "no device plan for a %zu x %zu transform", rows, b);
                    pi = (int)P.plans.size();
                    P.plans.push_back(sp);
                    plan_index[key] = pi;
                } else {
                    pi = itp->second;
                }
                XformRec X;
                memset(&X, 0, sizeof(X));
                const bool multi = P.plans[pi].nstages > 1;
                X.src_off = (f != 1) ? P.ds_off[(size_t)t * C + ci] : P.offsets[t];
                X.src_norm = (f != 1) ? 0 : 1;
                X.out_row = P.out_rows_off[t] + rows_total;
                X.tau = P.tau[ci];
                X.b = (int)b;
                X.m = (int)rows;
                X.rows_eval = (int)re;
                X.stdnoise = (float)sqrt((double)rows * downsampled_variance(N, f));
                X.plan = pi;
                X.seq = -1;
                X.tune = capr | (tpr << 16);
                const int xi = (int)P.xforms.size();
                if (multi) {
                    X.seq = P.nseq++;
                    // stage outputs use the level stride (16-byte aligned rows)
                    P.slot_floats = std::max(P.slot_floats, rows * (size_t)ffa_stride((int)b));
                    seq_xform.push_back(xi);
                    seq_pending.emplace_back();
                    seq_has_pending.push_back(0);
                    if (X.seq >= kSlots) finish_seq(X.seq - kSlots);
                }
                P.xforms.push_back(X);
                P.bins_used[0] = std::min(P.bins_used[0], (int)b);
                P.bins_used[1] = std::max(P.bins_used[1], (int)b);
                P.tpr_mask |= (tpr == 8) ? 1 : 2;
                P.xform_tc.push_back(make_int2(t, ci));
                rows_total += re;
                emit_stage(xi, 0);
                flush();
            }
        }
        P.out_rows_off[t + 1] = P.out_rows_off[t] + rows_total;
    }
    while (!deferred.empty()) {
        const auto e = *deferred.begin();
        deferred.erase(deferred.begin());
        emit_stage(std::get<1>(e), std::get<2>(e));
    }
    P.ds_total = ds_total;

    // deredden geometry (time_series.py:119, running_medians.py:72-80)
    P.lo_len.assign(T, 0);
    P.lo_off.assign(T, 0);
    if (c.deredden) {
        const double ws = nearbyint(c.rmed_width / c.tsamp);  // Python round(): half to even
        if (!(ws >= 1)) return set_error(RT_EINVAL, "rmed_width is shorter than one sample");
        P.rmed_width = (int)ws;
        if (!(c.rmed_minpts % 2)) return set_error(RT_EINVAL, "min_points must be an odd number");
        const double sf = std::max(1.0, ws / (double)c.rmed_minpts);
        P.scrunch = (int)sf;
        const int w = P.scrunch == 1 ? P.rmed_width : (int)c.rmed_minpts;
        if (!(w % 2)) return set_error(RT_EINVAL, "width must be an odd number");
        size_t lo_total = 0;
        for (int t = 0; t < T; ++t) {
            const size_t nl = P.scrunch == 1 ? P.lengths[t] : P.lengths[t] / P.scrunch;
            if (!((size_t)w < nl)) return set_error(RT_EINVAL, "width must be < size");
            P.lo_len[t] = nl;
            P.lo_off[t] = lo_total;
            lo_total += nl;
            P.max_lo = std::max(P.max_lo, nl);
        }
        P.lo_total = lo_total;
    }
    return RT_OK;
}

template <class T>
static void dfree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

static void plan_free_device(SearchPlan& P)
{
    dfree(P.d_widths); dfree(P.d_xforms); dfree(P.d_items); dfree(P.d_plans);
    dfree(P.d_scratch); dfree(P.d_counters); dfree(P.d_ticket); dfree(P.d_ds); dfree(P.d_y);
    dfree(P.d_norm); dfree(P.d_lores); dfree(P.d_coef); dfree(P.d_rmed); dfree(P.d_part);
    dfree(P.d_mean); dfree(P.d_normv); dfree(P.d_len); dfree(P.d_off); dfree(P.d_lo_len);
    dfree(P.d_lo_off); dfree(P.d_f); dfree(P.d_useseg); dfree(P.d_dsoff);
    P.dev_ready = false;
}

// Device allocation of one of the plan's buffers. With an injected allocation fault
// (rt_search_inject_fault, RT_FAULT_ALLOC) the chosen call fails as cudaMalloc would.
template <class T>
static int dalloc(SearchPlan& P, T** p, size_t n)
{
    if (n == 0) n = 1;
    ++P.alloc_calls;
    if (P.alloc_fail_at > 0 && P.alloc_calls == P.alloc_fail_at)
        return set_error(RT_ENOMEM, "device allocation %d of the plan failed (injected)",
                         P.alloc_calls);
    RT_TRY_CUDA(cudaMalloc((void**)p, n * sizeof(T)));
    return RT_OK;
}

template <class T>
static int upload(SearchPlan& P, T** p, const std::vector<T>& v)
{
    RT_TRY(dalloc(P, p, v.size()));
    if (!v.empty())
        RT_TRY_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return RT_OK;
}

static int plan_alloc_device(SearchPlan& P);

// Allocates and fills the plan's device buffers once. On failure every buffer allocated so
// far is released again, so a failed call leaks nothing and can be retried.
static int plan_prepare_device(SearchPlan& P)
{
    if (P.dev_ready) return RT_OK;
    P.alloc_calls = 0;
    const int s = plan_alloc_device(P);
    if (s != RT_OK) {
        plan_free_device(P);
        return s;
    }
    P.dev_ready = true;
    return RT_OK;
}

static int plan_alloc_device(SearchPlan& P)
{
    const int T = (int)P.lengths.size();
    RT_TRY(upload(P, &P.d_widths, P.widths));
    RT_TRY(upload(P, &P.d_items, P.items));
    RT_TRY(upload(P, &P.d_plans, P.plans));
    RT_TRY(upload(P, &P.d_xforms, P.xforms));
    RT_TRY(dalloc(P, &P.d_scratch, (size_t)kSlots * 2 * std::max<size_t>(P.slot_floats, 1)));
    RT_TRY(dalloc(P, &P.d_counters, (size_t)P.nseq * kMaxStages + kSlots + 1));
    RT_TRY(dalloc(P, &P.d_ticket, 1));
    // + 16 floats: bulk copies read whole 16-byte units around a block of rows
    RT_TRY(dalloc(P, &P.d_ds, P.ds_total + 16));
    if (P.cfg.deredden) {
        RT_TRY(dalloc(P, &P.d_y, P.total_len));
        RT_TRY(dalloc(P, &P.d_rmed, P.scrunch > 1 ? P.lo_total : P.total_len));
        if (P.scrunch > 1) {
            RT_TRY(dalloc(P, &P.d_lores, P.lo_total));
            RT_TRY(dalloc(P, &P.d_coef, P.lo_total));
        }
    }
    if (P.has_unit_factor) RT_TRY(dalloc(P, &P.d_norm, P.total_len));
    RT_TRY(dalloc(P, &P.d_part, (size_t)T * P.stat_blocks * 3));
    RT_TRY(dalloc(P, &P.d_mean, T));
    RT_TRY(dalloc(P, &P.d_normv, T));
    RT_TRY(upload(P, &P.d_len, P.lengths));
    RT_TRY(upload(P, &P.d_off, P.offsets));
    RT_TRY(upload(P, &P.d_lo_len, P.lo_len));
    RT_TRY(upload(P, &P.d_lo_off, P.lo_off));
    RT_TRY(upload(P, &P.d_f, P.f));
    RT_TRY(upload(P, &P.d_useseg, P.use_seg));
    RT_TRY(upload(P, &P.d_dsoff, P.ds_off));
    return RT_OK;
}

// The instance of k_search_persistent for a plan whose transforms have bins in
// [bmin, bmax] and use the S/N thread counts of tpr_mask (bit 0: 8, bit 1: 16). Plans of bins
// 449-544 with 16 S/N threads (the bins 480-520 searches) get the instance without the
// 256-bin loops and the 8-thread S/N: 2.0% faster on the large sweep. An instance for bins
// 225-288 measured 3.6-3.8% slower than the full one on the 240-260 searches (with both S/N
// thread counts or with 8 only), so those keep the full instance.
static void (*search_kernel_for(int bmin, int bmax, int tpr_mask))(EngineArgs)
{
    if (bins_class(bmin, bmax) == kBins512 && tpr_mask == 2)
        return k_search_persistent<kBins512, 2>;
    return k_search_persistent<kBinsAny, 3>;
}

static int engine_grid(void (*kernel)(EngineArgs))
{
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kEngineThreads, kEngineDynBytes);
    return std::max(1, sms * std::max(per, 1));
}

// Launches the whole search of the plan on `st`. data: packed input series (device).
static int plan_run(SearchPlan& P, const float* data, float* normalised_out, double* periods,
                    uint32_t* foldbins, float* snrs, cudaStream_t st)
{
    RT_TRY(plan_prepare_device(P));
    const int T = (int)P.lengths.size();
    const int C = (int)P.f.size();
    TrialArrays TA{P.d_len, P.d_off, P.d_lo_len, P.d_lo_off};
    const float* series = data;  // series before normalisation
    int launches = 0;
    if (P.timing) RT_TRY_CUDA(cudaEventRecord(P.ev[0], st));
    if (P.cfg.deredden) {
        const int k = P.scrunch;
        if (k > 1) {
            RT_TRY(launch_scrunch(data, TA, k, T, P.max_lo, P.d_lores, st));
            RT_TRY(launch_running_median(P.d_lores, P.d_lo_len, P.d_lo_off, T, P.max_lo,
                                         (int)P.cfg.rmed_minpts, P.d_rmed, st));
            dim3 gc((unsigned)std::min<size_t>((P.max_lo + 255) / 256, 1024), (unsigned)T);
            k_interp_coef<<<gc, 256, 0, st>>>(TA, k, P.d_rmed, P.d_coef);
            RT_TRY_CUDA(cudaGetLastError());
            launches += 3;
        } else {
            RT_TRY(launch_running_median(data, P.d_len, P.d_off, T, P.max_len, P.rmed_width,
                                         P.d_rmed, st));
            launches += 1;
        }
        dim3 g((unsigned)P.stat_blocks, (unsigned)T);
        k_dered<<<g, kStatThreads, 0, st>>>(data, TA, k, div_magic(2u * (unsigned)k), P.d_rmed,
                                            P.d_coef, P.d_y, P.d_part, P.stat_blocks);
        RT_TRY_CUDA(cudaGetLastError());
        launches += 1;
        series = P.d_y;
    } else if (!P.cfg.already_normalised) {
        dim3 g((unsigned)P.stat_blocks, (unsigned)T);
        k_sums<<<g, kStatThreads, 0, st>>>(data, TA, P.d_part, P.stat_blocks);
        RT_TRY_CUDA(cudaGetLastError());
        launches += 1;
    }
    const bool affine = !P.cfg.already_normalised;
    if (affine) {
        k_stats<<<(T + 127) / 128, 128, 0, st>>>(P.d_part, P.d_len, P.stat_blocks, T, P.d_mean,
                                                 P.d_normv);
        RT_TRY_CUDA(cudaGetLastError());
        launches += 1;
    }
    if (P.timing) RT_TRY_CUDA(cudaEventRecord(P.ev[1], st));
    // The normalised series is materialised by the downsampler when the caller wants it or
    // when a cycle folds it directly (f == 1); without normalisation it is `series` itself.
    float* zdst = normalised_out ? normalised_out : (P.has_unit_factor && affine ? P.d_norm : nullptr);
    const float* zsrc = affine ? (zdst ? zdst : series) : series;
    if (!affine && normalised_out && normalised_out != series)
        RT_TRY_CUDA(cudaMemcpyAsync(normalised_out, series, P.total_len * sizeof(float),
                                    cudaMemcpyDeviceToDevice, st));
    DsJob job;
    job.in = series;
    job.in_off = P.d_off;
    job.lengths = P.d_len;
    job.mean = affine ? P.d_mean : nullptr;
    job.norm = affine ? P.d_normv : nullptr;
    job.norm_out = affine ? zdst : nullptr;
    job.f = P.d_f;
    job.use_seg = P.d_useseg;
    job.out = P.d_ds;
    job.out_off = P.d_dsoff;
    job.ncycles = C;
    job.use_seg_host = P.use_seg.data();
    job.f_host = P.f.data();
    job.skip_host = P.skip.data();
    RT_TRY(launch_downsample(job, T, P.max_len, st));
    {
        bool seg = job.norm_out != nullptr;
        for (int c = 0; c < C; ++c) {
            seg |= P.use_seg[c] != 0;
            launches += (!P.use_seg[c] && !P.skip[c]) ? 1 : 0;
        }
        launches += seg ? 1 : 0;
    }
    if (P.timing) RT_TRY_CUDA(cudaEventRecord(P.ev[2], st));
    // counters
    const size_t ncounters = (size_t)P.nseq * kMaxStages + kSlots + 1;
    RT_TRY_CUDA(cudaMemsetAsync(P.d_counters, 0, ncounters * sizeof(int), st));
    RT_TRY_CUDA(cudaMemsetAsync(P.d_ticket, 0, sizeof(unsigned long long), st));
    EngineArgs A;
    A.ds = P.d_ds;
    A.norm = zsrc;
    A.snrs = snrs;
    A.periods = periods;
    A.foldbins = foldbins;
    A.xforms = P.d_xforms;
    A.items = P.d_items;
    A.nitems = (long long)P.items.size();
    A.plans = P.d_plans;
    A.widths = P.d_widths;
    A.nw = (int)P.widths.size();
    A.nfast = P.nfast;
    A.scratch = P.d_scratch;
    A.slot_floats = P.slot_floats;
    A.done = P.d_counters;
    A.slot_release = P.d_counters + (size_t)P.nseq * kMaxStages;
    A.error = A.slot_release + kSlots;
    A.ticket = P.d_ticket;
    A.phase_cycles = P.d_phase;
    A.spin_limit = P.spin_limit;
    A.dep_bias = P.dep_bias;
    void (*kernel)(EngineArgs) = search_kernel_for(P.bins_used[0], P.bins_used[1], P.tpr_mask);
    RT_TRY_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kEngineDynBytes));
    if (A.nitems > 0) {
        kernel<<<engine_grid(kernel), kEngineThreads, kEngineDynBytes, st>>>(A);
        RT_TRY_CUDA(cudaGetLastError());
        launches += 1;
    }
    if (P.timing) RT_TRY_CUDA(cudaEventRecord(P.ev[3], st));
    P.launches_last_run = launches;
    return RT_OK;
}

static int plan_check_error(SearchPlan& P, cudaStream_t st)
{
    int err = 0;
    RT_TRY_CUDA(cudaMemcpyAsync(&err, P.d_counters + (size_t)P.nseq * kMaxStages + kSlots,
                                sizeof(int), cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    if (err == RT_ETIMEOUT)
        return set_error(RT_ETIMEOUT, "a bounded wait in the search kernel ran out");
    if (err != RT_OK) return set_error(err, "the search kernel reported error %d", err);
    return RT_OK;
}

// ------------------------------------------------------------------------------------
// Sparse-row backward of a run: the gradient with respect to the searched (normalised)
// series of sum(gsnr * snrs), for gradients on few periodogram rows (a max-S/N loss has one
// per trial). Output row s of a transform is a sum of every input row i rolled by a total
// shift sigma_i(s) (the tail shifts met on the way from the root to leaf i); the row is
// recomputed from the downsampled series that the run left in its arena, its boxcar S/N is
// differentiated (the max routed to the first maximising phase), and the row gradient is
// scattered back through the same shifts, then through the downsampling.
// ------------------------------------------------------------------------------------
struct BwdJob {
    int m, b, s, pad;
    float stdnoise;
    int pad2;
    unsigned long long grow;  // row index into gsnr
};

struct BwdGroup {
    unsigned long long src;   // float offset of the folded series (arena or z)
    unsigned long long gds;   // float offset of this group's downsampled gradient
    unsigned long long gz;    // float offset of the trial's series in the packed gradient
    unsigned long long sig;   // int offset of this group's shift table
    int job0, njobs, src_is_z, pad;
    size_t n_ds, N;
    double f;
};

constexpr int kBwdThreads = 256;
constexpr int kBwdMaxBins = 4096;

__global__ void __launch_bounds__(kBwdThreads)
    k_rows_backward(const BwdGroup* __restrict__ groups, const BwdJob* __restrict__ jobs,
                    const float* __restrict__ arena, const float* __restrict__ z,
                    const float* __restrict__ gsnr, const int* __restrict__ widths, int nw,
                    int wmax, float* __restrict__ gds_all, int* __restrict__ sig_all)
{
    extern __shared__ float sm[];
    float* F = sm;                       // kBwdMaxBins
    float* C = F + kBwdMaxBins;          // b + wmax
    __shared__ float s_g[kBwdMaxBins];
    __shared__ int s_best[64];
    const BwdGroup G = groups[blockIdx.x];
    const float* src = (G.src_is_z ? z : arena) + G.src;
    float* gds = gds_all + G.gds;
    int* sig = sig_all + G.sig;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int q = 0; q < G.njobs; ++q) {
        const BwdJob J = jobs[G.job0 + q];
        const int m = J.m, b = J.b;
        // total shift of every input row for output row s
        for (int i = tid; i < m; i += kBwdThreads) {
            int row0 = 0, n = m, r = J.s, sg = 0;
            while (n > 1) {
                const int nh = n >> 1;
                const MergeCoef mc = merge_coef(n);
                const int h = merge_row(mc.kh, r), t = merge_row(mc.kt, r);
                if (i < row0 + nh) {
                    n = nh;
                    r = h;
                } else {
                    sg += (r - t) % b;
                    sg -= (sg >= b) ? b : 0;
                    row0 += nh;
                    n -= nh;
                    r = t;
                }
            }
            sig[i] = sg;
        }
        __syncthreads();
        // the output row
        for (int c = tid; c < b; c += kBwdThreads) {
            float acc = 0.0f;
            for (int i = 0; i < m; ++i) {
                int idx = c + sig[i];
                idx -= (idx >= b) ? b : 0;
                acc = __fadd_rn(acc, src[(size_t)i * b + idx]);
            }
            F[c] = acc;
        }
        __syncthreads();
        // boxcar S/N backward of the row (one warp)
        if (tid < 32) {
            double carry = 0.0;
            for (int c0 = 0; c0 < b; c0 += 32) {
                const int c = c0 + lane;
                const double v = (c < b) ? (double)F[c] : 0.0;
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
                if (lane == 0) s_best[k] = bi;
            }
        }
        __syncthreads();
        const float* g = gsnr + (size_t)J.grow * nw;
        for (int c = tid; c < b; c += kBwdThreads) {
            double acc = 0.0;
            for (int k = 0; k < nw; ++k) {
                float hb, be;
                boxcar_coefs(b, widths[k], &hb, &be);
                acc -= (double)g[k] * (double)be;
                int off = c - s_best[k] - 1;
                off += (off < 0) ? b : 0;
                if (off < widths[k]) acc += (double)g[k] * (double)hb;
            }
            s_g[c] = (float)(acc / (double)J.stdnoise);
        }
        __syncthreads();
        // back through the shifts: row i reads the row gradient at c - sigma_i
        for (size_t e = tid; e < (size_t)m * b; e += kBwdThreads) {
            const int i = (int)(e / b), c = (int)(e - (size_t)i * b);
            int idx = c - sig[i];
            idx += (idx < 0) ? b : 0;
            gds[e] = __fadd_rn(gds[e], s_g[idx]);
        }
        __syncthreads();
    }
}

// Downsampling adjoint of the groups of one wave (each trial at most once per wave).
__global__ void k_groups_ds_adjoint(const BwdGroup* __restrict__ groups, const int* __restrict__ wave,
                                    const float* __restrict__ gds_all, float* __restrict__ gz_all)
{
    const BwdGroup G = groups[wave[blockIdx.y]];
    const float* gout = gds_all + G.gds;
    float* gin = gz_all + G.gz;
    const size_t N = G.N, n = G.n_ds;
    const double f = G.f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x) {
        if (G.src_is_z) {  // the cycle folds the series itself
            if (i < n) gin[i] = __fadd_rn(gin[i], gout[i]);
            continue;
        }
        const double qf = floor((double)i / f);
        const size_t k0 = qf >= 1.0 ? (size_t)qf - 1 : 0;
        const size_t k1 = min(n, (size_t)floor((double)(i + 1) / f) + 2);
        double acc = 0.0;
        for (size_t k = k0; k < k1; ++k) {
            const double start = (double)k * f;
            const double end = start + f;
            const size_t imin = (size_t)floor(start);
            const double fe = floor(end);
            const size_t imax = (size_t)(fe < (double)N - 1.0 ? fe : (double)N - 1.0);
            double c = 0.0;
            if (i == imin) c += (double)__double2float_rn((double)(imin + 1) - start);
            if (i == imax) c += (double)__double2float_rn(end - (double)imax);
            if (i > imin && i < imax) c += 1.0;
            if (imax == imin && i == imin) c -= 1.0;
            if (c != 0.0) acc += c * (double)gout[k];
        }
        if (acc != 0.0) gin[i] = __fadd_rn(gin[i], (float)acc);
    }
}

__global__ void k_live_rows(const float* __restrict__ g, size_t rows, int nw,
                            unsigned long long* __restrict__ list, unsigned long long cap,
                            unsigned long long* __restrict__ count)
{
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < rows;
         r += (size_t)gridDim.x * blockDim.x) {
        bool live = false;
        for (int k = 0; k < nw; ++k) live |= g[r * nw + k] != 0.0f;
        if (live) {
            const unsigned long long slot = atomicAdd(count, 1ull);
            if (slot < cap) list[slot] = r;
        }
    }
}

static int plan_backward(SearchPlan& P, const float* d_z, const float* d_gsnr, float* d_gz,
                         size_t max_rows, cudaStream_t st)
{
    if (!P.dev_ready) return set_error(RT_EINVAL, "the plan has not run");
    const size_t L = P.out_rows_off.back();
    const int nw = (int)P.widths.size();
    RT_TRY_CUDA(cudaMemsetAsync(d_gz, 0, P.total_len * sizeof(float), st));
    if (L == 0 || nw == 0) return RT_OK;
    // rows that carry a gradient
    unsigned long long *d_list = nullptr, *d_count = nullptr;
    RT_TRY_CUDA(cudaMallocAsync((void**)&d_list, (max_rows + 1) * sizeof(unsigned long long), st));
    d_count = d_list + max_rows;
    RT_TRY_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st));
    k_live_rows<<<(unsigned)std::min<size_t>((L + 255) / 256, 148 * 16), 256, 0, st>>>(
        d_gsnr, L, nw, d_list, max_rows, d_count);
    unsigned long long count = 0;
    RT_TRY_CUDA(cudaMemcpyAsync(&count, d_count, sizeof(count), cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    if (count > max_rows) {
        cudaFreeAsync(d_list, st);
        return set_error(RT_EINVAL, "%llu periodogram rows carry a gradient (at most %zu)", count,
                         max_rows);
    }
    std::vector<unsigned long long> rows(count);
    if (count)
        RT_TRY_CUDA(cudaMemcpyAsync(rows.data(), d_list, count * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    cudaFreeAsync(d_list, st);
    if (count == 0) return RT_OK;
    std::sort(rows.begin(), rows.end());
    // rows -> (transform, s), grouped by (trial, cycle) in plan order
    const int C = (int)P.f.size();
    std::vector<BwdJob> jobs;
    std::vector<BwdGroup> groups;
    std::vector<int> group_trial;
    size_t xi = 0, gds_total = 0, sig_total = 0;
    int last_tc = -1;
    for (unsigned long long r : rows) {
        while (xi + 1 < P.xforms.size() && P.xforms[xi + 1].out_row <= r) ++xi;
        const XformRec& X = P.xforms[xi];
        if (r < X.out_row || r >= X.out_row + (unsigned long long)X.rows_eval) continue;
        if (X.b > kBwdMaxBins || X.b + (size_t)*std::max_element(P.widths.begin(), P.widths.end()) > 2 * kBwdMaxBins)
            return set_error(RT_EINVAL, "profiles of %d bins are too long for the backward", X.b);
        const int t = P.xform_tc[xi].x, c = P.xform_tc[xi].y;
        const int tc = t * C + c;
        if (tc != last_tc) {
            BwdGroup G;
            const double f = P.f[c];
            const size_t N = P.lengths[t];
            G.src_is_z = (f == 1) ? 1 : 0;
            G.src = G.src_is_z ? P.offsets[t] : P.ds_off[(size_t)tc];
            G.n_ds = G.src_is_z ? N : downsampled_size(N, f);
            G.N = N;
            G.f = f;
            G.gds = gds_total;
            gds_total += (G.n_ds + 3) & ~size_t(3);
            G.gz = P.offsets[t];
            G.sig = sig_total;
            G.job0 = (int)jobs.size();
            G.njobs = 0;
            G.pad = 0;
            groups.push_back(G);
            group_trial.push_back(t);
            last_tc = tc;
        }
        BwdGroup& G = groups.back();
        BwdJob J;
        J.m = X.m;
        J.b = X.b;
        J.s = (int)(r - X.out_row);
        J.stdnoise = X.stdnoise;
        J.grow = r;
        J.pad = J.pad2 = 0;
        jobs.push_back(J);
        ++G.njobs;
        sig_total = std::max<size_t>(sig_total, (size_t)G.sig + (size_t)X.m);
    }
    if (jobs.empty()) return RT_OK;
    // waves: the k-th group of every trial (a trial's groups accumulate into one series)
    std::vector<std::vector<int>> waves;
    {
        std::map<int, int> seen;
        for (size_t g = 0; g < groups.size(); ++g) {
            const int k = seen[group_trial[g]]++;
            if ((int)waves.size() <= k) waves.emplace_back();
            waves[k].push_back((int)g);
        }
    }
    int wmax = 1;
    for (int w : P.widths) wmax = std::max(wmax, w);
    unsigned char* blob = nullptr;
    const size_t nwave = groups.size();
    const size_t bytes = groups.size() * sizeof(BwdGroup) + jobs.size() * sizeof(BwdJob) +
                         nwave * sizeof(int) + (gds_total + 4) * sizeof(float) +
                         (sig_total + 4) * sizeof(int) + 64;
    RT_TRY_CUDA(cudaMallocAsync((void**)&blob, bytes, st));
    BwdGroup* d_groups = reinterpret_cast<BwdGroup*>(blob);
    BwdJob* d_jobs = reinterpret_cast<BwdJob*>(d_groups + groups.size());
    int* d_wave = reinterpret_cast<int*>(d_jobs + jobs.size());
    float* d_gds = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(d_wave + nwave) + 15) & ~uintptr_t(15));
    int* d_sig = reinterpret_cast<int*>(d_gds + gds_total + 4);
    int s = RT_OK;
    auto ck = [&](cudaError_t e) { if (s == RT_OK && e != cudaSuccess) s = check_cuda(e, "search backward"); };
    ck(cudaMemcpyAsync(d_groups, groups.data(), groups.size() * sizeof(BwdGroup),
                       cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(BwdJob), cudaMemcpyHostToDevice, st));
    ck(cudaMemsetAsync(d_gds, 0, gds_total * sizeof(float), st));
    const size_t smem = (size_t)(2 * kBwdMaxBins + wmax) * sizeof(float);
    ck(cudaFuncSetAttribute(k_rows_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (s == RT_OK) {
        k_rows_backward<<<(unsigned)groups.size(), kBwdThreads, smem, st>>>(
            d_groups, d_jobs, P.d_ds, d_z, d_gsnr, P.d_widths, nw, wmax, d_gds, d_sig);
        ck(cudaGetLastError());
    }
    // every group of a kernel call uses its own shift table: the groups run concurrently
    (void)sig_total;
    for (const auto& w : waves) {
        if (s != RT_OK) break;
        ck(cudaMemcpyAsync(d_wave, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        dim3 grid(64, (unsigned)w.size());
        k_groups_ds_adjoint<<<grid, 256, 0, st>>>(d_groups, d_wave, d_gds, d_gz);
        ck(cudaGetLastError());
    }
    cudaFreeAsync(blob, st);
    return s;
}

}  // namespace rt

// ====================================================================================
// C ABI
// ====================================================================================
using namespace rt;

struct rt_search_plan {
    SearchPlan p;
};

static int plan_create(const uint64_t* lengths, size_t ntrials, const rt_search_config* cfg,
                       const uint64_t* widths, size_t num_widths,
                       const rt_search_tuning* tuning, rt_search_plan** out,
                       const rt_tile_rule* rules = nullptr, size_t num_rules = 0)
{
    if (!out || !cfg || (!lengths && ntrials) || (!widths && num_widths))
        return set_error(RT_EINVAL, "null argument");
    *out = nullptr;
    if (ntrials == 0) return set_error(RT_EINVAL, "at least one time series is required");
    if (num_widths == 0 || num_widths > (size_t)kMaxWidths)
        return set_error(RT_EINVAL, "between 1 and %d trial widths are supported", kMaxWidths);
    rt_search_plan* h = new (std::nothrow) rt_search_plan();
    if (!h) return set_error(RT_ENOMEM, "out of host memory");
    SearchPlan& P = h->p;
    P.cfg = *cfg;
    if (tuning) P.tuning = *tuning;
    if (rules) P.rules.assign(rules, rules + num_rules);
    for (size_t i = 0; i < num_widths; ++i) {
        // snr.hpp:21-31
        if (!(widths[i] > 0 && widths[i] < cfg->bins_min)) {
            delete h;
            return set_error(RT_EINVAL, "trial widths must be all > 0 and < columns");
        }
        P.widths.push_back((int)widths[i]);
    }
    P.nfast = detect_fast_widths(P.widths.data(), (int)P.widths.size());
    if (P.nfast && P.widths.size() > 10 && cfg->bins_min <= 42) P.nfast = 0;
    for (size_t t = 0; t < ntrials; ++t) {
        if (lengths[t] == 0 || lengths[t] >= (1ull << 40)) {
            delete h;
            return set_error(RT_EINVAL, "time series %zu has an unsupported length", t);
        }
        P.lengths.push_back((size_t)lengths[t]);
        P.offsets.push_back(P.total_len);
        P.total_len += lengths[t];
        P.max_len = std::max(P.max_len, (size_t)lengths[t]);
    }
    int s = plan_build(P);
    if (s != RT_OK) {
        delete h;
        return s;
    }
    *out = h;
    return RT_OK;
}

extern "C" int rt_search_plan_create(const uint64_t* lengths, size_t ntrials,
                                     const rt_search_config* cfg, const uint64_t* widths,
                                     size_t num_widths, rt_search_plan** out)
{
    return plan_create(lengths, ntrials, cfg, widths, num_widths, nullptr, out);
}

static int check_tuning(const rt_search_tuning* tuning)
{
    if (tuning && !(tuning->rows_fraction >= 0.0 && tuning->rows_fraction <= 1.0))
        return set_error(RT_EINVAL, "rows_fraction must be in [0, 1]");
    if (tuning && !(tuning->rows_fraction_deep >= 0.0 && tuning->rows_fraction_deep <= 1.0))
        return set_error(RT_EINVAL, "rows_fraction_deep must be in [0, 1]");
    if (tuning && tuning->snr_threads != 0 && tuning->snr_threads != 8 && tuning->snr_threads != 16)
        return set_error(RT_EINVAL, "snr_threads must be 0, 8 or 16");
    if (tuning && tuning->lag_items < 0) return set_error(RT_EINVAL, "lag_items must be >= 0");
    return RT_OK;
}

extern "C" int rt_search_plan_create_tuned(const uint64_t* lengths, size_t ntrials,
                                           const rt_search_config* cfg, const uint64_t* widths,
                                           size_t num_widths, const rt_search_tuning* tuning,
                                           rt_search_plan** out)
{
    RT_TRY(check_tuning(tuning));
    return plan_create(lengths, ntrials, cfg, widths, num_widths, tuning, out);
}

extern "C" int rt_search_plan_create_rules(const uint64_t* lengths, size_t ntrials,
                                           const rt_search_config* cfg, const uint64_t* widths,
                                           size_t num_widths, const rt_search_tuning* tuning,
                                           const rt_tile_rule* rules, size_t num_rules,
                                           rt_search_plan** plan)
{
    if (num_rules && !rules) return set_error(RT_EINVAL, "null argument");
    for (size_t i = 0; i < num_rules; ++i) {
        const rt_tile_rule& R = rules[i];
        if (R.rows_min > R.rows_max || R.bins_min > R.bins_max)
            return set_error(RT_EINVAL, "tile rule %zu: empty rows or bins range", i);
        if (!(R.rows_fraction >= 0.0 && R.rows_fraction <= 1.0))
            return set_error(RT_EINVAL, "tile rule %zu: rows_fraction must be in [0, 1]", i);
        if (R.snr_threads != 0 && R.snr_threads != 8 && R.snr_threads != 16)
            return set_error(RT_EINVAL, "tile rule %zu: snr_threads must be 0, 8 or 16", i);
        if (R.max_levels < 0 || R.max_levels > kMaxJobDepth + 1)
            return set_error(RT_EINVAL, "tile rule %zu: max_levels must be in [0, %d]", i,
                             kMaxJobDepth + 1);
    }
    RT_TRY(check_tuning(tuning));
    return plan_create(lengths, ntrials, cfg, widths, num_widths, tuning, plan, rules, num_rules);
}

extern "C" int rt_search_plan_rows(const rt_search_plan* plan, uint64_t* row_offsets)
{
    if (!plan || !row_offsets) return set_error(RT_EINVAL, "null argument");
    for (size_t i = 0; i < plan->p.out_rows_off.size(); ++i) row_offsets[i] = plan->p.out_rows_off[i];
    return RT_OK;
}

extern "C" int rt_search_plan_stats(const rt_search_plan* plan, rt_search_plan_stats_t* st)
{
    if (!plan || !st) return set_error(RT_EINVAL, "null argument");
    const SearchPlan& P = plan->p;
    memset(st, 0, sizeof(*st));
    st->num_trials = P.lengths.size();
    st->num_cycles = P.f.size();
    st->num_transforms = P.xforms.size();
    st->num_work_items = P.items.size();
    st->num_multistage = (uint64_t)P.nseq;
    st->total_rows = P.out_rows_off.back();
    st->total_samples = P.total_len;
    st->downsampled_samples = P.ds_total;
    uint64_t fold = 0;
    for (const XformRec& X : P.xforms) fold += (uint64_t)X.m * X.b;
    st->folded_samples = fold;
    st->scrunch_factor = (uint64_t)P.scrunch;
    return RT_OK;
}

// Graph replay of plan_run: captured on the plan's own stream (the legacy default stream
// cannot be captured), launched on the caller's.
static int plan_run_graph(SearchPlan& P, const float* data, float* normalised_out,
                          double* periods, uint32_t* foldbins, float* snrs, cudaStream_t st)
{
    const void* key[5] = {data, normalised_out, periods, foldbins, snrs};
    bool same = P.gexec != nullptr;
    for (int i = 0; i < 5; ++i) same = same && key[i] == P.gkey[i];
    if (!same) {
        RT_TRY(plan_prepare_device(P));  // allocations happen outside the capture
        if (!P.cap_stream)
            RT_TRY_CUDA(cudaStreamCreateWithFlags(&P.cap_stream, cudaStreamNonBlocking));
        if (P.gexec) {
            cudaGraphExecDestroy(P.gexec);
            P.gexec = nullptr;
        }
        RT_TRY_CUDA(cudaStreamBeginCapture(P.cap_stream, cudaStreamCaptureModeThreadLocal));
        const int rc = plan_run(P, data, normalised_out, periods, foldbins, snrs, P.cap_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(P.cap_stream, &g);
        if (rc != RT_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ec != cudaSuccess) return check_cuda(ec, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&P.gexec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            P.gexec = nullptr;
            return check_cuda(ei, "cudaGraphInstantiate");
        }
        for (int i = 0; i < 5; ++i) P.gkey[i] = key[i];
        ++P.graph_captures;
    }
    RT_TRY_CUDA(cudaGraphLaunch(P.gexec, st));
    return RT_OK;
}

extern "C" int rt_search_run(rt_search_plan* plan, const float* data, float* normalised_out,
                             double* periods, uint32_t* foldbins, float* snrs, void* stream)
{
    if (!plan || !data || !periods || !foldbins || !snrs) return set_error(RT_EINVAL, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    SearchPlan& P = plan->p;
    if (P.use_graph && !P.timing)
        return plan_run_graph(P, data, normalised_out, periods, foldbins, snrs, st);
    return plan_run(P, data, normalised_out, periods, foldbins, snrs, st);
}

extern "C" int rt_search_set_graph(rt_search_plan* plan, int enable)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    P.use_graph = enable != 0;
    if (!P.use_graph && P.gexec) {
        RT_TRY_CUDA(cudaGraphExecDestroy(P.gexec));
        P.gexec = nullptr;
    }
    return RT_OK;
}

extern "C" int rt_search_graph_captures(const rt_search_plan* plan, int* h_count)
{
    if (!plan || !h_count) return set_error(RT_EINVAL, "null argument");
    *h_count = plan->p.graph_captures;
    return RT_OK;
}

extern "C" int rt_search_plan_transforms(const rt_search_plan* plan, rt_search_transform* h_out)
{
    if (!plan || !h_out) return set_error(RT_EINVAL, "null argument");
    const SearchPlan& P = plan->p;
    for (size_t i = 0; i < P.xforms.size(); ++i) {
        const XformRec& X = P.xforms[i];
        rt_search_transform& o = h_out[i];
        o.trial = (uint32_t)P.xform_tc[i].x;
        o.cycle = (uint32_t)P.xform_tc[i].y;
        o.bins = (uint32_t)X.b;
        o.rows = (uint32_t)X.m;
        o.rows_eval = (uint32_t)X.rows_eval;
        o.out_row = X.out_row;
        o.factor = P.f[P.xform_tc[i].y];
        o.tau = X.tau;
        o.stdnoise = X.stdnoise;
    }
    return RT_OK;
}

extern "C" int rt_search_normalisation(rt_search_plan* plan, double* h_mean, double* h_std,
                                       void* stream)
{
    if (!plan || !h_mean || !h_std) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    const size_t T = P.lengths.size();
    if (!P.dev_ready || P.cfg.already_normalised) {
        for (size_t t = 0; t < T; ++t) {
            h_mean[t] = 0.0;
            h_std[t] = 1.0;
        }
        return RT_OK;
    }
    cudaStream_t st = (cudaStream_t)stream;
    RT_TRY_CUDA(cudaMemcpyAsync(h_mean, P.d_mean, T * sizeof(double), cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaMemcpyAsync(h_std, P.d_normv, T * sizeof(double), cudaMemcpyDeviceToHost, st));
    RT_TRY_CUDA(cudaStreamSynchronize(st));
    return RT_OK;
}

extern "C" int rt_search_backward_rows(rt_search_plan* plan, const float* d_z,
                                       const float* d_gsnr, float* d_gz, size_t max_rows,
                                       void* stream)
{
    if (!plan || !d_z || !d_gsnr || !d_gz) return set_error(RT_EINVAL, "null argument");
    if (max_rows == 0) return set_error(RT_EINVAL, "max_rows must be positive");
    return plan_backward(plan->p, d_z, d_gsnr, d_gz, max_rows, (cudaStream_t)stream);
}

extern "C" int rt_search_plan_prepare(rt_search_plan* plan)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    return plan_prepare_device(plan->p);
}

extern "C" int rt_search_check(rt_search_plan* plan, void* stream)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    if (!plan->p.dev_ready) return RT_OK;
    return plan_check_error(plan->p, (cudaStream_t)stream);
}

// The kernel arguments and buffers are baked into a captured graph: drop it.
static void plan_drop_graph(SearchPlan& P)
{
    if (P.gexec) cudaGraphExecDestroy(P.gexec);
    P.gexec = nullptr;
    for (int i = 0; i < 5; ++i) P.gkey[i] = nullptr;
}

extern "C" int rt_search_set_wait_limit(rt_search_plan* plan, long long polls)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    if (polls < 1) return set_error(RT_EINVAL, "the wait limit must be at least one poll");
    cudaDeviceSynchronize();
    plan->p.spin_limit = polls;
    plan_drop_graph(plan->p);
    return RT_OK;
}

extern "C" int rt_search_inject_fault(rt_search_plan* plan, int kind, int arg)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    cudaDeviceSynchronize();
    switch (kind) {
        case RT_FAULT_NONE:
            P.dep_bias = 0;
            P.alloc_fail_at = 0;
            break;
        case RT_FAULT_STAGE_WAIT:
            P.dep_bias = 1;
            break;
        case RT_FAULT_ALLOC:
            if (arg < 1) return set_error(RT_EINVAL, "the failing allocation is numbered from 1");
            P.alloc_fail_at = arg;
            plan_free_device(P);  // the next run allocates again
            break;
        default:
            return set_error(RT_EINVAL, "unknown fault kind %d", kind);
    }
    plan_drop_graph(P);
    return RT_OK;
}

extern "C" int rt_search_set_timing(rt_search_plan* plan, int enable)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    if (enable && !P.ev[0])
        for (int i = 0; i < 4; ++i) RT_TRY_CUDA(cudaEventCreate(&P.ev[i]));
    P.timing = enable != 0;
    return RT_OK;
}

extern "C" int rt_search_last_timing(rt_search_plan* plan, float* h_ms, int* h_launches)
{
    if (!plan || !h_ms) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    if (!P.timing || !P.ev[0]) return set_error(RT_EINVAL, "timing is not enabled on this plan");
    RT_TRY_CUDA(cudaEventSynchronize(P.ev[3]));
    for (int i = 0; i < 3; ++i) RT_TRY_CUDA(cudaEventElapsedTime(&h_ms[i], P.ev[i], P.ev[i + 1]));
    if (h_launches) *h_launches = P.launches_last_run;
    return RT_OK;
}

extern "C" int rt_search_set_profiling(rt_search_plan* plan, int enable)
{
    if (!plan) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    if (enable && !P.d_phase) {
        RT_TRY_CUDA(cudaMalloc((void**)&P.d_phase, kCounters * sizeof(unsigned long long)));
        RT_TRY_CUDA(cudaMemset(P.d_phase, 0, kCounters * sizeof(unsigned long long)));
    } else if (!enable && P.d_phase) {
        cudaFree(P.d_phase);
        P.d_phase = nullptr;
    }
    return RT_OK;
}

extern "C" int rt_search_phase_cycles(rt_search_plan* plan, uint64_t* h_counters, int reset)
{
    if (!plan || !h_counters) return set_error(RT_EINVAL, "null argument");
    SearchPlan& P = plan->p;
    if (!P.d_phase) return set_error(RT_EINVAL, "profiling is not enabled on this plan");
    RT_TRY_CUDA(cudaDeviceSynchronize());
    RT_TRY_CUDA(cudaMemcpy(h_counters, P.d_phase, kCounters * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    if (reset) RT_TRY_CUDA(cudaMemset(P.d_phase, 0, kCounters * sizeof(unsigned long long)));
    return RT_OK;
}

extern "C" void rt_search_plan_destroy(rt_search_plan* plan)
{
    if (!plan) return;
    cudaDeviceSynchronize();
    if (plan->p.d_phase) cudaFree(plan->p.d_phase);
    if (plan->p.gexec) cudaGraphExecDestroy(plan->p.gexec);
    if (plan->p.cap_stream) cudaStreamDestroy(plan->p.cap_stream);
    for (int i = 0; i < 4; ++i)
        if (plan->p.ev[i]) cudaEventDestroy(plan->p.ev[i]);
    plan_free_device(plan->p);
    delete plan;
}

// ------------------------------------------------------------------------------------
// Single-series deredden / normalise (TimeSeries.deredden / normalise, fast_running_median)
// ------------------------------------------------------------------------------------
namespace {
struct OneSeries {
    size_t v[4];  // len, off, lo_len, lo_off
};
}  // namespace

static int one_series_arrays(size_t N, size_t nl, size_t** d, cudaStream_t st, TrialArrays* A)
{
    OneSeries h{{N, 0, nl, 0}};
    RT_TRY_CUDA(cudaMallocAsync((void**)d, sizeof(h), st));
    RT_TRY_CUDA(cudaMemcpyAsync(*d, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    A->len = *d;
    A->off = *d + 1;
    A->lo_len = *d + 2;
    A->lo_off = *d + 3;
    return RT_OK;
}

// width_samples / min_points -> (scrunch factor, running-median width, scrunched length)
static int rmed_geometry(size_t N, size_t width_samples, size_t minpts, int* k, int* w, size_t* nl)
{
    // running_medians.py:72-80
    if (!(minpts % 2)) return set_error(RT_EINVAL, "min_points must be an odd number");
    *k = (int)std::max(1.0, (double)width_samples / (double)minpts);
    *w = (*k == 1) ? (int)width_samples : (int)minpts;
    *nl = (*k == 1) ? N : N / (size_t)*k;
    // running_median.hpp:103-107
    if (!(*w % 2)) return set_error(RT_EINVAL, "width must be an odd number");
    if (!((size_t)*w < *nl)) return set_error(RT_EINVAL, "width must be < size");
    return RT_OK;
}

extern "C" int rt_fast_running_median(const float* d_x, size_t size, size_t width_samples,
                                      size_t min_points, double* d_out, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    int k, w;
    size_t nl;
    RT_TRY(rmed_geometry(size, width_samples, min_points, &k, &w, &nl));
    size_t* d = nullptr;
    TrialArrays A;
    RT_TRY(one_series_arrays(size, nl, &d, st, &A));
    float *lores = nullptr, *rmed = nullptr;
    int s = RT_OK;
    if (k > 1) {
        RT_TRY_CUDA(cudaMallocAsync((void**)&lores, nl * sizeof(float), st));
        RT_TRY_CUDA(cudaMallocAsync((void**)&rmed, nl * sizeof(float), st));
        s = launch_scrunch(d_x, A, k, 1, nl, lores, st);
        if (s == RT_OK) s = launch_running_median(lores, A.lo_len, A.lo_off, 1, nl, w, rmed, st);
        if (s == RT_OK) {
            k_interp_rmed<<<dim3(std::max(1, (int)std::min<size_t>((size + 255) / 256, 4096)), 1), 256, 0, st>>>(
                A, k, rmed, d_out);
            s = check_cuda(cudaGetLastError(), "fast_running_median");
        }
    } else {
        // no scrunching: the exact running median (float32), widened to float64
        RT_TRY_CUDA(cudaMallocAsync((void**)&rmed, size * sizeof(float), st));
        s = launch_running_median(d_x, A.len, A.off, 1, size, w, rmed, st);
        if (s == RT_OK) {
            k_interp_rmed<<<dim3(std::max(1, (int)std::min<size_t>((size + 255) / 256, 4096)), 1), 256, 0, st>>>(
                TrialArrays{A.len, A.off, A.len, A.off}, 1, rmed, d_out);
            s = check_cuda(cudaGetLastError(), "fast_running_median");
        }
    }
    if (lores) cudaFreeAsync(lores, st);
    if (rmed) cudaFreeAsync(rmed, st);
    cudaFreeAsync(d, st);
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "fast_running_median");
    return s;
}

extern "C" int rt_deredden(const float* d_x, size_t size, double tsamp, double width,
                           size_t min_points, float* d_out, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const double ws = nearbyint(width / tsamp);  // int(round(width / tsamp)), half to even
    if (!(ws >= 1)) return set_error(RT_EINVAL, "width is shorter than one sample");
    int k, w;
    size_t nl;
    RT_TRY(rmed_geometry(size, (size_t)ws, min_points, &k, &w, &nl));
    size_t* d = nullptr;
    TrialArrays A;
    RT_TRY(one_series_arrays(size, nl, &d, st, &A));
    float *lores = nullptr, *rmed = nullptr;
    double2* coef = nullptr;
    double* part = nullptr;
    int s = RT_OK;
    const int blocks = 64;
    RT_TRY_CUDA(cudaMallocAsync((void**)&part, blocks * 3 * sizeof(double), st));
    if (k > 1) {
        RT_TRY_CUDA(cudaMallocAsync((void**)&lores, nl * sizeof(float), st));
        RT_TRY_CUDA(cudaMallocAsync((void**)&rmed, nl * sizeof(float), st));
        RT_TRY_CUDA(cudaMallocAsync((void**)&coef, nl * sizeof(double2), st));
        s = launch_scrunch(d_x, A, k, 1, nl, lores, st);
        if (s == RT_OK) s = launch_running_median(lores, A.lo_len, A.lo_off, 1, nl, w, rmed, st);
        if (s == RT_OK) {
            k_interp_coef<<<dim3((unsigned)std::min<size_t>((nl + 255) / 256, 1024), 1), 256, 0, st>>>(
                A, k, rmed, coef);
            s = check_cuda(cudaGetLastError(), "deredden");
        }
    } else {
        RT_TRY_CUDA(cudaMallocAsync((void**)&rmed, size * sizeof(float), st));
        s = launch_running_median(d_x, A.len, A.off, 1, size, w, rmed, st);
    }
    if (s == RT_OK) {
        k_dered<<<dim3(blocks, 1), kStatThreads, 0, st>>>(d_x, A, k, div_magic(2u * (unsigned)k),
                                                          rmed, coef, d_out, part, blocks);
        s = check_cuda(cudaGetLastError(), "deredden");
    }
    if (coef) cudaFreeAsync(coef, st);
    if (lores) cudaFreeAsync(lores, st);
    if (rmed) cudaFreeAsync(rmed, st);
    cudaFreeAsync(part, st);
    cudaFreeAsync(d, st);
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "deredden");
    return s;
}

extern "C" int rt_normalise(const float* d_x, size_t size, float* d_out, void* stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    if (size == 0) return RT_OK;
    size_t* d = nullptr;
    TrialArrays A;
    RT_TRY(one_series_arrays(size, 0, &d, st, &A));
    double* part = nullptr;
    const int blocks = 64;
    RT_TRY_CUDA(cudaMallocAsync((void**)&part, (blocks * 3 + 2) * sizeof(double), st));
    double* mean = part + blocks * 3;
    double* norm = mean + 1;
    k_sums<<<dim3(blocks, 1), kStatThreads, 0, st>>>(d_x, A, part, blocks);
    k_stats<<<1, 32, 0, st>>>(part, A.len, blocks, 1, mean, norm);
    k_normalise<<<dim3(std::max(1, (int)std::min<size_t>((size + 255) / 256, 4096)), 1), 256, 0, st>>>(
        d_x, A, mean, norm, d_out);
    int s = check_cuda(cudaGetLastError(), "normalise");
    cudaFreeAsync(part, st);
    cudaFreeAsync(d, st);
    if (s == RT_OK) s = check_cuda(cudaStreamSynchronize(st), "normalise");
    return s;
}
