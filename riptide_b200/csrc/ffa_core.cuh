// FFA transform core: one CTA executes one "tree job" of an FFA transform in shared memory.
//
// The reference computes the transform of an m x b block (cpp/transforms.hpp:30-50) by
// recursive halving: head = rows >> 1 (cpp/block.hpp:30-31), tail = the rest, then
//     out[s] = head[h] + roll(tail[t], -(s - t)),   h = int(kh*s + .5f), t = int(kt*s + .5f)
// (transforms.hpp:13-27; the shift h + b_s of the reference equals s - t).
//
// Here the recursion tree is cut into jobs that fit one CTA's shared memory:
//   * a job has a root node (a subtree of the transform: first row, row count), the range of
//     root output rows it must produce, and a depth G: nodes at depth G below the root are
//     computed straight from a global source array whose row j holds the output of a node
//     at depth G+1 (or, for full-depth jobs, raw input row j);
//   * going down the tree, a contiguous output range of a node needs a contiguous range of
//     rows of each child, so every level is a list of (node, row range) stored back to back
//     in a shared-memory buffer; two buffers alternate between levels;
//   * the root rows are then either written to global memory (to feed a job higher in the
//     tree, or as the ffa2 result) or turned into boxcar S/N (snr_core.cuh).
// Additions are float32 and performed in exactly the reference's order, so the result is
// bit-identical to cpp/transforms.hpp.
#pragma once
#include "common.cuh"
#include "bulk_copy.cuh"

namespace rt {

constexpr int kMaxJobDepth = 7;      // levels computed inside one job (<= 128 nodes at the bottom)
constexpr int kMaxJobNodes = 256;    // total nodes of all levels of one job
constexpr int kThreads = 480;        // compute threads per CTA of every FFA kernel (1 CTA per SM)
constexpr int kWarps = kThreads / 32;

// Barrier of the compute threads only (named barrier 1). The persistent search kernel adds a
// scheduling warp that does not take part; in the other kernels every thread computes.
__device__ __forceinline__ void cta_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory");
}

struct Node {
    int row0;   // first row of the node in the transform
    int rows;   // node size
    int lo;     // first needed output row (node-local)
    int hi;     // one past the last needed output row
    int off;    // row of `lo` inside this level's shared buffer
};

struct JobTree {
    Node nodes[kMaxJobNodes];
    int level_start[kMaxJobDepth + 2];  // index of the first node of each level
    int level_rows[kMaxJobDepth + 2];   // rows stored for each level
    int op_start[kMaxJobDepth + 2];     // first row operation of each level
    int depth;                          // G: nodes at this level read the global source
    int error;                          // nonzero if the job does not fit
    // Source rows of level G staged in shared memory (jobs of later stages, whose source is
    // the previous stage's output with 16-byte aligned rows; G <= kMaxStagedDepth): node i
    // of level G reads its head child's source rows src_rng[i].x + [0, src_rng[i].y) from
    // staged rows src_off[i] + ..., and its tail child's rows src_rng[i].z + [0, .w) right
    // after them. pstaged = 0: level G reads global rows.
    int pstaged;
    int src_off[33];
    int4 src_rng[32];
};
constexpr int kMaxStagedDepth = 5;

// Description of one job, produced by the planners (host).
struct JobSpec {
    int root_row0, root_rows;  // root node
    int lo, hi;                // root output range
    int G;                     // relative depth of the level computed from the global source
};

// Full-depth job: G = smallest depth d with ceil(M / 2^d) <= 2 (all nodes there have 1 or
// 2 rows, whose children are single input rows).
RT_HD int full_depth(int rows)
{
    int d = 0;
    while (((rows + (1 << d) - 1) >> d) > 2) ++d;
    return d;
}

// Builds the per-level node lists of a job (all threads of the CTA, 3 barriers).
// Node q of the flat array is node i = q - (2^d - 1) of level d; its row range follows from
// the root range by applying the head/tail row maps along the bits of i.
__device__ inline void build_job_tree(JobTree& T, const JobSpec& J, int cap_rows)
{
    const int tid = threadIdx.x;
    const int G = J.G;
    const bool bad = (G > kMaxJobDepth || (2 << G) - 1 > kMaxJobNodes);
    if (tid == 0) {
        T.depth = G;
        T.error = bad ? 1 : 0;
        T.pstaged = 0;
    }
    if (bad) {
        cta_sync();
        return;
    }
    const int nnodes = (2 << G) - 1;
    for (int q = tid; q < nnodes; q += kThreads) {
        const int d = 31 - __clz(q + 1);
        const int i = q + 1 - (1 << d);
        int row0 = J.root_row0, rows = J.root_rows, lo = J.lo, hi = J.hi;
        for (int k = d - 1; k >= 0; --k) {
            const int mh = rows >> 1;
            const MergeCoef c = merge_coef(rows);
            if ((i >> k) & 1) {
                const int nlo = merge_row(c.kt, lo), nhi = merge_row(c.kt, hi - 1) + 1;
                row0 += mh;
                rows -= mh;
                lo = nlo;
                hi = nhi;
            } else {
                const int nlo = merge_row(c.kh, lo), nhi = merge_row(c.kh, hi - 1) + 1;
                rows = mh;
                lo = nlo;
                hi = nhi;
            }
        }
        Node nd;
        nd.row0 = row0;
        nd.rows = rows;
        nd.lo = lo;
        nd.hi = hi;
        nd.off = 0;
        T.nodes[q] = nd;
    }
    if (tid <= G) T.level_start[tid] = (1 << tid) - 1;
    cta_sync();
    // one warp per level: exclusive prefix of the row counts -> buffer offsets
    const int warp = tid >> 5, lane = tid & 31;
    if (warp <= G) {
        const int d = warp, n = 1 << d, base = (1 << d) - 1;
        int carry = 0;
        for (int b0 = 0; b0 < n; b0 += 32) {
            const int i = b0 + lane;
            const int v = (i < n) ? (T.nodes[base + i].hi - T.nodes[base + i].lo) : 0;
            int incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (i < n) T.nodes[base + i].off = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            T.level_rows[d] = carry;
            if (carry > cap_rows) T.error = 2;
        }
    }
    cta_sync();
    if (tid == 0) {
        int acc = 0;
        for (int d = 0; d <= G; ++d) {
            T.op_start[d] = acc;
            acc += T.level_rows[d];
        }
        T.op_start[G + 1] = acc;
    }
    cta_sync();
}

// The same job tree built by one warp (no CTA barrier), level by level: node i of level d is
// the head (i even) or tail (i odd) child of node i >> 1 of level d - 1, which gives the
// node list of build_job_tree.
// With stage_source, also lays out the level-G source rows for staging (src_off, pstaged):
// set when every level-G node has two children and the rows fit the level buffer.
__device__ inline void build_job_tree_warp(JobTree& T, const JobSpec& J, int cap_rows,
                                           bool stage_source = false)
{
    const int lane = threadIdx.x & 31;
    const int G = J.G;
    const bool bad = (G > kMaxJobDepth || (2 << G) - 1 > kMaxJobNodes);
    if (lane == 0) {
        T.depth = G;
        T.error = bad ? 1 : 0;
        T.pstaged = 0;
    }
    if (bad) {
        __syncwarp();
        return;
    }
    if (lane == 0) {
        Node nd;
        nd.row0 = J.root_row0;
        nd.rows = J.root_rows;
        nd.lo = J.lo;
        nd.hi = J.hi;
        nd.off = 0;
        T.nodes[0] = nd;
    }
    __syncwarp();
    for (int d = 1; d <= G; ++d) {
        const int base = (1 << d) - 1, pbase = (1 << (d - 1)) - 1;
        for (int i = lane; i < (1 << d); i += 32) {
            const Node p = T.nodes[pbase + (i >> 1)];
            const int mh = p.rows >> 1;
            const MergeCoef c = merge_coef(p.rows);
            Node nd;
            if (i & 1) {
                nd.row0 = p.row0 + mh;
                nd.rows = p.rows - mh;
                nd.lo = merge_row(c.kt, p.lo);
                nd.hi = merge_row(c.kt, p.hi - 1) + 1;
            } else {
                nd.row0 = p.row0;
                nd.rows = mh;
                nd.lo = merge_row(c.kh, p.lo);
                nd.hi = merge_row(c.kh, p.hi - 1) + 1;
            }
            nd.off = 0;
            T.nodes[base + i] = nd;
        }
        __syncwarp();
    }
    // per level: exclusive prefix of the row counts -> buffer offsets; then op_start
    int acc = 0;
    for (int d = 0; d <= G; ++d) {
        const int n = 1 << d, base = n - 1;
        int carry = 0;
        for (int b0 = 0; b0 < n; b0 += 32) {
            const int i = b0 + lane;
            const int v = (i < n) ? (T.nodes[base + i].hi - T.nodes[base + i].lo) : 0;
            int incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (i < n) T.nodes[base + i].off = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) {
            T.level_start[d] = base;
            T.level_rows[d] = carry;
            T.op_start[d] = acc;
            if (carry > cap_rows) T.error = 2;
        }
        acc += carry;
    }
    if (lane == 0) T.op_start[G + 1] = acc;
    if (stage_source && G <= kMaxStagedDepth) {
        // rows each level-G node needs from its two children, as consecutive staged blocks
        // (one lane per node: at most 32 nodes)
        const int n = 1 << G, base = n - 1;
        const int i = lane;
        int v = 0;
        bool two = true;
        if (i < n) {
            const Node nd = T.nodes[base + i];
            int4 rg = make_int4(nd.row0, 0, nd.row0 + (nd.rows >> 1), 0);
            if (nd.rows < 2) {
                two = false;
            } else if (nd.hi > nd.lo) {
                const MergeCoef c = merge_coef(nd.rows);
                const int hlo = merge_row(c.kh, nd.lo), tlo = merge_row(c.kt, nd.lo);
                rg.x += hlo;
                rg.y = merge_row(c.kh, nd.hi - 1) + 1 - hlo;
                rg.z += tlo;
                rg.w = merge_row(c.kt, nd.hi - 1) + 1 - tlo;
            }
            v = rg.y + rg.w;
            T.src_rng[i] = rg;
        }
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (i < n) T.src_off[i] = incl - v;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        two = __all_sync(0xffffffffu, two);
        if (lane == 0) {
            T.src_off[n] = total;
            T.pstaged = (two && total <= cap_rows) ? 1 : 0;
        }
    }
    __syncwarp();
}

// Index of the node holding buffer row r at a level (nodes sorted by `off`).
__device__ __forceinline__ int find_node(const Node* nodes, int n, int r)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (nodes[mid].off <= r) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Level rows in shared memory: b values, 16-byte aligned rows. For the bins ranges of the
// usual searches (bins_min 240 or 480) the level loops are unrolled for exactly ceil(b / 64)
// two-column chunks per lane (4, 5, 8, 9) and the global level for ceil(b / 32) columns
// (8, 9, 15, 16, 17).
RT_HD bool halo_mode(int b) { return (b >= 225 && b <= 288) || (b >= 449 && b <= 544); }
RT_HD int ffa_stride(int b) { return (b + 3) & ~3; }

// One output row of a level: out = row h + roll(row t, -shift) of the level below.
// For the level read from global memory, h and t are global row indices; t < 0 marks a
// single-row node (out = row h).
struct RowOp {
    int h, t, shift;
};

// Row operation of buffer row r of level d.
__device__ __forceinline__ RowOp make_row_op(const JobTree& T, int d, int r, int b)
{
    const Node* lvl = T.nodes + T.level_start[d];
    const int i = find_node(lvl, 1 << d, r);
    const Node nd = lvl[i];
    const int s = nd.lo + (r - nd.off);
    RowOp op;
    if (nd.rows == 1) {
        op.h = nd.row0;
        op.t = -1;
        op.shift = 0;
    } else {
        const MergeCoef c = merge_coef(nd.rows);
        const int h = merge_row(c.kh, s), t = merge_row(c.kt, s);
        op.shift = (s - t) % b;
        if (d == T.depth && T.pstaged) {
            const int4 rg = T.src_rng[i];
            op.h = T.src_off[i] + (nd.row0 + h - rg.x);
            op.t = T.src_off[i] + rg.y + (nd.row0 + (nd.rows >> 1) + t - rg.z);
        } else if (d == T.depth) {
            op.h = nd.row0 + h;
            op.t = nd.row0 + (nd.rows >> 1) + t;
        } else {
            const Node* child = T.nodes + T.level_start[d + 1];
            const Node hn = child[2 * i], tn = child[2 * i + 1];
            op.h = hn.off + h - hn.lo;
            op.t = tn.off + t - tn.lo;
        }
    }
    return op;
}

// Row operations of every level of the job (one thread per output row, all levels at once).
// Call after build_job_tree; the caller synchronises before using `ops`.
__device__ inline void build_all_ops(const JobTree& T, int b, RowOp* ops)
{
    const int total = T.op_start[T.depth + 1];
    for (int g = threadIdx.x; g < total; g += kThreads) {
        int d = 0;
        while (T.op_start[d + 1] <= g) ++d;
        ops[g] = make_row_op(T, d, g - T.op_start[d], b);
    }
}

// Computes the rows of one level, one warp per row, NIT = ceil(b / 32) columns per lane.
// kGlobal: operands are rows of the global source (packed, stride b).
template <int NIT, bool kGlobal>
__device__ __forceinline__ void level_rows_unrolled(const RowOp* ops, int nrows,
                                                    const float* __restrict__ src, int sstride,
                                                    float* __restrict__ dst, int stride, int b)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < nrows; r += kWarps) {
        const RowOp op = ops[r];
        float* out = dst + (size_t)r * stride;
        const float* H = src + (size_t)op.h * sstride;
        float v[NIT];
        if (op.t < 0) {
#pragma unroll
            for (int j = 0; j < NIT; ++j) {
                const int c = lane + 32 * j;
                if (j < NIT - 1 || c < b) v[j] = kGlobal ? __ldcg(H + c) : H[c];
            }
        } else {
            // column c reads the rolled row at c + shift, or c + shift - b past the wrap
            // (c + shift < 2 b): the test 32 j >= b - shift - lane picks the base pointer
            const float* T0 = src + (size_t)op.t * sstride + op.shift + lane;
            const float* T1 = T0 - b;
            const int thr = b - op.shift - lane;
#pragma unroll
            for (int j = 0; j < NIT; j += 2) {
                const int c = lane + 32 * j;
                const float* p = (32 * j >= thr) ? T1 : T0;
                if (j + 1 < NIT - 1) {
                    // two columns, both inside the row: one packed f32x2 addition
                    const float* q = (32 * j + 32 >= thr) ? T1 : T0;
                    asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
                        " add.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
                        : "=f"(v[j]), "=f"(v[j + 1])
                        : "f"(kGlobal ? __ldcg(H + c) : H[c]), "f"(kGlobal ? __ldcg(H + c + 32) : H[c + 32]),
                          "f"(kGlobal ? __ldcg(p + 32 * j) : p[32 * j]),
                          "f"(kGlobal ? __ldcg(q + 32 * j + 32) : q[32 * j + 32]));
                } else {
                    if (j < NIT - 1 || c < b)
                        v[j] = __fadd_rn(kGlobal ? __ldcg(H + c) : H[c],
                                         kGlobal ? __ldcg(p + 32 * j) : p[32 * j]);
                    if (j + 1 < NIT) {
                        const float* q = (32 * j + 32 >= thr) ? T1 : T0;
                        if (c + 32 < b)
                            v[j + 1] = __fadd_rn(kGlobal ? __ldcg(H + c + 32) : H[c + 32],
                                                 kGlobal ? __ldcg(q + 32 * j + 32) : q[32 * j + 32]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            const int c = lane + 32 * j;
            if (j < NIT - 1 || c < b) out[c] = v[j];
        }
    }
}

// Shared-memory level for the usual bins ranges: in each 64-column chunk a lane computes
// columns c = 64 j + lane and c + 32, so every load and store of the warp touches 32
// consecutive words (mod b). Column c reads the rolled row at c + shift before the wrap and
// at c + shift - b after it (c + shift < 2 b: one wrap at most); with c = 64 j + lane (+ 32)
// the wrap test is 64 j (+ 32) >= b - shift - lane, an immediate compared with one register
// per row, and picks one of two base pointers: one compare and one select per element, and
// no dependency chain from chunk to chunk.
template <int NIT2>
__device__ __forceinline__ void level_rows_pairs(const RowOp* ops, int nrows,
                                                 const float* __restrict__ src, int sstride,
                                                 float* __restrict__ dst, int stride, int b)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < nrows; r += kWarps) {
        const RowOp op = ops[r];
        float* out = dst + (size_t)r * stride + lane;
        const float* H = src + (size_t)op.h * sstride + lane;
        const float* T0 = src + (size_t)op.t * sstride + op.shift + lane;
        const float* T1 = T0 - b;
        const int thr = b - op.shift - lane;
#pragma unroll
        for (int j = 0; j < NIT2; ++j) {
            const int c = 64 * j + lane;
            const float* p0 = (64 * j >= thr) ? T1 : T0;
            const float* p1 = (64 * j + 32 >= thr) ? T1 : T0;
            if (j < NIT2 - 1) {
                // both columns' adds in one packed f32x2 addition
                float s0, s1;
                asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
                    " add.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
                    : "=f"(s0), "=f"(s1)
                    : "f"(H[64 * j]), "f"(H[64 * j + 32]), "f"(p0[64 * j]), "f"(p1[64 * j + 32]));
                out[64 * j] = s0;
                out[64 * j + 32] = s1;
            } else {
                if (c < b) out[64 * j] = __fadd_rn(H[64 * j], p0[64 * j]);
                // the last chunk's second half (columns from 64 (NIT2 - 1) + 32) is empty for
                // every b of the 5- and 9-chunk ranges (b <= 288 and b <= 544)
                constexpr bool kHalf2 = NIT2 != 5 && NIT2 != 9;
                if (kHalf2 && c + 32 < b) out[64 * j + 32] = __fadd_rn(H[64 * j + 32], p1[64 * j + 32]);
            }
        }
    }
}

// Any b: per-element wrap, no unrolling.
template <bool kGlobal>
__device__ __forceinline__ void level_rows_generic(const RowOp* ops, int nrows,
                                                   const float* __restrict__ src, int sstride,
                                                   float* __restrict__ dst, int stride, int b)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < nrows; r += kWarps) {
        const RowOp op = ops[r];
        float* out = dst + (size_t)r * stride;
        const float* H = src + (size_t)op.h * sstride;
        const float* Tr = src + (size_t)(op.t < 0 ? 0 : op.t) * sstride;
        for (int c = lane; c < b; c += 32) {
            float v;
            if (op.t < 0) {
                v = kGlobal ? __ldcg(H + c) : H[c];
            } else {
                int idx = c + op.shift;
                idx -= (idx >= b) ? b : 0;
                v = kGlobal ? __fadd_rn(__ldcg(H + c), __ldcg(Tr + idx)) : __fadd_rn(H[c], Tr[idx]);
            }
            out[c] = v;
        }
    }
}

// Bins classes of a kernel instance: which unrolled level loops it contains. A kernel that
// only ever sees b in [225, 288] (kBins256) or in [449, 544] (kBins512) leaves out the loops of
// the other range (smaller code); kBinsAny has all of them. Any b still runs correctly in any
// class (the generic loop), only slower.
enum BinsClass { kBinsAny = 0, kBins256 = 1, kBins512 = 2 };

RT_HD int bins_class(int bmin, int bmax)
{
    if (bmin >= 225 && bmax <= 288) return kBins256;
    if (bmin >= 449 && bmax <= 544) return kBins512;
    return kBinsAny;
}

template <bool kGlobal, int BC = kBinsAny>
__device__ __forceinline__ void level_rows(const RowOp* ops, int nrows, const float* src,
                                           int sstride, float* dst, int stride, int b)
{
    constexpr bool k256 = BC != kBins512, k512 = BC != kBins256;
    // each case runs its unrolled loop and returns when the class holds it, else falls
    // through to the generic loop below
#define RT_PAIRS_CASE(N, K)                                                   \
    case N:                                                                   \
        if constexpr (K) {                                                    \
            level_rows_pairs<N>(ops, nrows, src, sstride, dst, stride, b);    \
            return;                                                           \
        }                                                                     \
        break;
    if (!kGlobal && halo_mode(b)) {
        switch ((b + 63) >> 6) {
            RT_PAIRS_CASE(4, k256)
            RT_PAIRS_CASE(5, k256)
            RT_PAIRS_CASE(8, k512)
            default:  // 9
                if constexpr (k512) {
                    level_rows_pairs<9>(ops, nrows, src, sstride, dst, stride, b);
                    return;
                }
                break;
        }
    }
#undef RT_PAIRS_CASE
#define RT_NIT_CASE(N, K)                                                              \
    case N:                                                                            \
        if constexpr (K) {                                                             \
            level_rows_unrolled<N, kGlobal>(ops, nrows, src, sstride, dst, stride, b); \
            return;                                                                    \
        }                                                                              \
        break;
    switch ((b + 31) >> 5) {
        // bins 225-288 and 449-544 cover the usual searches (bins_min 240 / 480)
        RT_NIT_CASE(8, k256)
        RT_NIT_CASE(9, k256)
        RT_NIT_CASE(15, k512)
        RT_NIT_CASE(16, k512)
        RT_NIT_CASE(17, k512)
        default: break;
    }
#undef RT_NIT_CASE
    level_rows_generic<kGlobal>(ops, nrows, src, sstride, dst, stride, b);
}

// Level computed from source rows staged in shared memory (packed, stride b): same loop as
// the global level, plain loads.
template <int BC = kBinsAny>
__device__ __forceinline__ void level_rows_staged(const RowOp* ops, int nrows, const float* src,
                                                  float* dst, int stride, int b)
{
    constexpr bool k256 = BC != kBins512, k512 = BC != kBins256;
#define RT_NIT_CASE(N, K)                                                         \
    case N:                                                                       \
        if constexpr (K) {                                                        \
            level_rows_unrolled<N, false>(ops, nrows, src, b, dst, stride, b);    \
            return;                                                               \
        }                                                                         \
        break;
    switch ((b + 31) >> 5) {
        RT_NIT_CASE(8, k256)
        RT_NIT_CASE(9, k256)
        RT_NIT_CASE(15, k512)
        RT_NIT_CASE(16, k512)
        RT_NIT_CASE(17, k512)
        default: break;
    }
#undef RT_NIT_CASE
    level_rows_generic<false>(ops, nrows, src, b, dst, stride, b);
}

// Where a job's levels read and write outside the two level buffers.
struct LevelIO {
    const float* src = nullptr;     // global source: row j at src + j * src_stride
    int src_stride = 0;
    const float* staged = nullptr;  // optional source rows being copied into shared memory
    bool staged_rows = false;       // staged: true = rows of the layout in JobTree::src_off
                                    // (stride = the level stride); false = global row j at
                                    // staged + j * b
    uint64_t* bar = nullptr;        // the copy completes on phase *phase of bar
    uint32_t* phase = nullptr;
    float* root_dst = nullptr;      // optional: root rows go to root_dst + i * root_stride
    int root_stride = 0;
};

// Runs all levels of the job. On return, the root rows [lo, hi) are in buf0 (stride
// `stride`, row i of the buffer = root output row lo + i), or in global memory if
// io.root_dst is given. `ops` has room for the largest level. Returns false if the wait for
// staged rows ran out.
template <int BC = kBinsAny>
__device__ inline bool run_job_levels(const JobTree& T, int b, float* buf0, float* buf1,
                                      int stride, RowOp* ops, const LevelIO& io)
{
    build_all_ops(T, b, ops);
    cta_sync();
    bool ok = true;
    if (io.staged) {
        ok = mbar_wait(io.bar, *io.phase);
        *io.phase ^= 1u;
    }
    for (int d = T.depth; d >= 0; --d) {
        // the root level goes straight to global memory when the caller wants it there
        const bool out_global = d == 0 && io.root_dst != nullptr;
        float* dst = out_global ? io.root_dst : ((d & 1) ? buf1 : buf0);
        const int dstride = out_global ? io.root_stride : stride;
        const RowOp* lops = ops + T.op_start[d];
        // one call site per level loop kind (the loops are large once unrolled)
        const bool first = d == T.depth;
        if (first && !io.staged) {
            level_rows<true, BC>(lops, T.level_rows[d], io.src, io.src_stride, dst, dstride, b);
        } else if (first && !io.staged_rows) {
            level_rows_staged<BC>(lops, T.level_rows[d], io.staged, dst, dstride, b);
        } else {
            // shared-memory source: level d + 1, or the staged rows of level G's children
            const float* from = first ? io.staged : ((d & 1) ? buf0 : buf1);
            level_rows<false, BC>(lops, T.level_rows[d], from, stride, dst, dstride, b);
        }
        cta_sync();
    }
    return ok;
}

// Global address of the root rows of a job in a stage output (row stride `rstride`).
__device__ __forceinline__ float* root_rows_dst(const JobTree& T, int rstride, float* dst)
{
    const Node r = T.nodes[0];
    return dst + (size_t)(r.row0 + r.lo) * rstride;
}

// Issued by one warp: bulk copies of the level-G source rows of a job laid out by
// build_job_tree_warp (pstaged), from a global source of 16-byte aligned rows of `stride`
// floats into `sbuf` (same stride), completing on `bar` (one arrival with the byte count).
__device__ inline void stage_source_rows_async(const JobTree& T, const float* src, int stride,
                                               float* sbuf, uint64_t* bar)
{
    const int lane = threadIdx.x & 31;
    const int n = 1 << T.depth;
    const size_t row_bytes = (size_t)stride * sizeof(float);
    // the source was written by other CTAs (generic proxy) before they signalled it
    asm volatile("fence.proxy.async.global;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)(T.src_off[n] * row_bytes));
    __syncwarp();
    constexpr uint32_t kChunk = 32768;
    for (int i = lane; i < n; i += 32) {
        const int4 rg = T.src_rng[i];
        const int r0[2] = {rg.x, rg.z};
        const int cnt[2] = {rg.y, rg.w};
        int off = T.src_off[i];
        for (int h = 0; h < 2; ++h) {
            const unsigned char* from =
                reinterpret_cast<const unsigned char*>(src + (size_t)r0[h] * stride);
            unsigned char* to = reinterpret_cast<unsigned char*>(sbuf + (size_t)off * stride);
            const size_t bytes = (size_t)cnt[h] * row_bytes;
            for (size_t o = 0; o < bytes; o += kChunk) {
                const uint32_t nb = (uint32_t)(bytes - o < kChunk ? bytes - o : kChunk);
                bulk_g2s(to + o, from + o, nb, bar);
            }
            off += cnt[h];
        }
    }
}

// Shared-memory layout of a CTA running FFA jobs: [fixed part][ops][buf0][buf1].
// Rows per level buffer for `smem_bytes` with `fixed_bytes` already used.
constexpr int kOpsPerCapRow = kMaxJobDepth + 1;  // row operations of all levels of a job

RT_HD int ffa_cap_rows_for(size_t smem_bytes, size_t fixed_bytes, int b)
{
    const size_t per_row =
        2 * (size_t)ffa_stride(b) * sizeof(float) + kOpsPerCapRow * sizeof(RowOp);
    return (int)((smem_bytes - fixed_bytes - 64) / per_row);
}

struct FfaSmem {
    RowOp* ops;
    float* buf0;
    float* buf1;
};

__device__ __forceinline__ FfaSmem ffa_smem(unsigned char* base, int cap_rows, int b)
{
    FfaSmem L;
    L.ops = reinterpret_cast<RowOp*>(base);
    size_t off = ((size_t)cap_rows * kOpsPerCapRow * sizeof(RowOp) + 63) & ~size_t(63);
    L.buf0 = reinterpret_cast<float*>(base + off);
    L.buf1 = L.buf0 + (size_t)cap_rows * ffa_stride(b);
    return L;
}

// ------------------------------------------------------------------------------------
// Host-side planning of the stages of one transform.
//
// Stage 0 computes nodes at depth D[0] fully (full-depth jobs from the raw rows); stage k
// computes the needed rows of nodes at depth D[k] from the outputs of depth D[k-1]; the
// last stage has D = 0 (the root) and produces rows [0, rows_out).
// ------------------------------------------------------------------------------------
constexpr int kMaxStages = 4;

struct StagePlan {
    int nstages;
    int D[kMaxStages];      // node depth produced by each stage
    int R[kMaxStages];      // output rows per job (per node) of each stage
    int jobs[kMaxStages];   // number of jobs of each stage
    int jobs_per_node[kMaxStages];
};

// Plans the stages of a transform with m rows whose root output is [0, rows_out), for
// level buffers of cap_rows rows. Uses the bound: a job whose root range has R rows holds at
// most R + 3 * 2^G rows at any level (a child range of an L-row range has <= (L + 3) / 2
// rows, since kh, kt <= 1/2).
// max_depth: the largest depth G of a job (G + 1 levels computed in shared memory); smaller
// values cut deep transforms into more stages, whose outputs pass through L2.
bool plan_stages(int m, int rows_out, int cap_rows, StagePlan* P, int max_depth = kMaxJobDepth);
// Job k of stage s of a transform (host or device).
RT_HD void node_at(int m, int d, int i, int* row0, int* rows)
{
    int r0 = 0, rr = m;
    for (int k = d - 1; k >= 0; --k) {
        const int mh = rr >> 1;
        if ((i >> k) & 1) {
            r0 += mh;
            rr -= mh;
        } else {
            rr = mh;
        }
    }
    *row0 = r0;
    *rows = rr;
}

RT_HD JobSpec stage_job(int m, int rows_out, const StagePlan& P, int stage, int job)
{
    JobSpec J;
    const int d = P.D[stage];
    if (stage == 0) {
        int r0, rr;
        node_at(m, d, job, &r0, &rr);
        J.root_row0 = r0;
        J.root_rows = rr;
        J.lo = 0;
        J.hi = (P.nstages == 1) ? rows_out : rr;
        J.G = full_depth(rr);
        return J;
    }
    const int node = job / P.jobs_per_node[stage];
    const int part = job - node * P.jobs_per_node[stage];
    int r0, rr;
    node_at(m, d, node, &r0, &rr);
    const int hi_node = (stage == P.nstages - 1) ? rows_out : rr;
    J.root_row0 = r0;
    J.root_rows = rr;
    J.lo = part * P.R[stage];
    J.hi = J.lo + P.R[stage] < hi_node ? J.lo + P.R[stage] : hi_node;
    J.G = P.D[stage - 1] - d - 1;
    return J;
}

}  // namespace rt
