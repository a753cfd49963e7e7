/*
 * riptide_b200.h -- C ABI of the B200 (sm_100a) implementation of riptide's FFA search.
 *
 * Every function returns an int status (RT_OK on success); on failure rt_last_error()
 * returns a message for the calling thread. RT_EINVAL corresponds to the reference raising
 * std::invalid_argument (ValueError in Python) with the same message text.
 *
 * Pointers named d_* are CUDA device pointers; h_* are host pointers. `stream` is a
 * cudaStream_t passed as void* (NULL = the legacy default stream). Kernels are enqueued
 * asynchronously on `stream`; functions that need host results synchronise it themselves.
 *
 * Each entry point cites the reference interface it replaces (paths relative to the
 * reference project: src/riptide/cpp/python_bindings.cpp is the pybind11 module
 * `riptide.libcpp`).
 */
#ifndef RIPTIDE_B200_H
#define RIPTIDE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RT_OK 0
#define RT_EINVAL 1     /* invalid argument (ValueError)                   */
#define RT_ECUDA 2      /* CUDA runtime error                              */
#define RT_ENOMEM 3     /* device or host allocation failed                */
#define RT_ETIMEOUT 4   /* a bounded wait inside a persistent kernel ran out */
#define RT_EINTERNAL 5  /* a device-side plan check failed                 */
#define RT_EIO 6        /* a file could not be opened or read (OSError)    */

/* Message of the last failing call on this thread. */
const char* rt_last_error(void);
/* Library version, 100 * major + minor. */
int rt_version(void);

/* ---------------------------------------------------------------------------------
 * Drop-ins for the riptide.libcpp functions (device buffers).
 * -------------------------------------------------------------------------------*/

/* rollback: out = roll(x, -shift). Replaces python_bindings.cpp:44-52 (kernels.hpp:32-38). */
int rt_rollback(const float* d_x, size_t size, size_t shift, float* d_out, void* stream);

/* fused_rollback_add: out = x + roll(y, -shift). Replaces python_bindings.cpp:55-70
 * (kernels.hpp:19-25). */
int rt_fused_rollback_add(const float* d_x, const float* d_y, size_t size, size_t shift,
                          float* d_out, void* stream);

/* circular_prefix_sum over nsum elements, double accumulator. Replaces
 * python_bindings.cpp:73-81 (kernels.hpp:73-101). d_out holds nsum floats. */
int rt_circular_prefix_sum(const float* d_x, size_t size, size_t nsum, float* d_out,
                           void* stream);

/* ffa2: FFA transform of a rows x cols C-order block, bit-identical to the reference.
 * Replaces python_bindings.cpp:84-96 (transforms.hpp:53-61). Allocates its own scratch for
 * blocks larger than one CTA's shared memory. */
int rt_ffa2(const float* d_in, size_t rows, size_t cols, float* d_out, void* stream);

/* ffa2 without any device allocation, for callers that cannot allocate: pipelines whose
 * device memory is reserved up front by another framework's pool, and real-time loops that
 * forbid cudaMalloc/cudaFree after start-up (they can block the whole device). No counterpart
 * in the reference. Scratch is a fixed 8 MiB array in this library, held by every GPU that
 * loads it: rows * cols <= 1048576 (cols <= 4096), else RT_EINVAL. The first call on a device
 * looks the array up (cudaGetSymbolAddress) and should come before any stream capture; the
 * address is kept for the life of the process, so cudaDeviceReset after that first call is
 * not supported. Calls share the array: calls that overlap on the GPU race and must not be
 * issued. */
int rt_ffa2_noalloc(const float* d_in, size_t rows, size_t cols, float* d_out, void* stream);

/* benchmark_ffa2: seconds per transform of a zero rows x cols block over `loops` runs
 * (CUDA events). Replaces python_bindings.cpp:99-118. */
int rt_benchmark_ffa2(size_t rows, size_t cols, size_t loops, double* h_seconds);

/* snr2: boxcar S/N of `rows` profiles of `cols` bins for num_widths trial widths (host
 * array). Output rows x num_widths. Replaces python_bindings.cpp:141-160 (snr.hpp:58-65);
 * snr1 is the rows == 1 case (python_bindings.cpp:121-138). */
int rt_snr2(const float* d_in, size_t rows, size_t cols, const uint64_t* h_widths,
            size_t num_widths, float stdnoise, float* d_out, void* stream);

/* downsample by a real factor 1 < f <= size; output floor(size / f) samples. d_in must be
 * 4-byte aligned (any float array is); RT_EINVAL otherwise, before any launch.
 * Replaces python_bindings.cpp:163-177 (downsample.hpp:44-82). */
int rt_downsample(const float* d_in, size_t size, double f, float* d_out, void* stream);

/* floor(size / f) (downsample.hpp:21-24), host only. */
size_t rt_downsampled_size(size_t size, double f);

/* running_median of odd width < size with edge padding, exact. Replaces
 * python_bindings.cpp:212-222 (running_median.hpp:100-132). */
int rt_running_median(const float* d_in, size_t size, size_t width, float* d_out,
                      void* stream);

/* fast_running_median: approximate running median of a series (float64 output): mean-
 * scrunch by int(max(1, width_samples / min_points)), exact running median of width
 * min_points, linear interpolation back. Replaces running_medians.py:49-85. */
int rt_fast_running_median(const float* d_in, size_t size, size_t width_samples,
                           size_t min_points, double* d_out, void* stream);

/* TimeSeries.deredden: out = float32(x - fast_running_median(x, round(width / tsamp),
 * min_points)). Replaces time_series.py:95-124. */
int rt_deredden(const float* d_in, size_t size, double tsamp, double width, size_t min_points,
                float* d_out, void* stream);

/* TimeSeries.normalise: out = float32((x - mean) / std), float64 statistics, population
 * variance. Replaces time_series.py:67-93. */
int rt_normalise(const float* d_in, size_t size, float* d_out, void* stream);

/* Number of periodogram rows (periodogram.hpp:63-109), host only. */
int rt_periodogram_length(size_t size, double tsamp, double period_min, double period_max,
                          size_t bins_min, size_t bins_max, size_t* h_length);

/* periodogram of one normalised series, through the batched engine (one trial).
 * Replaces python_bindings.cpp:180-209 (periodogram.hpp:117-201). Outputs hold
 * rt_periodogram_length() rows: periods (f64), foldbins (u32), snrs (rows x num_widths). */
int rt_periodogram(const float* d_data, size_t size, double tsamp, const uint64_t* h_widths,
                   size_t num_widths, double period_min, double period_max, size_t bins_min,
                   size_t bins_max, double* d_periods, uint32_t* d_foldbins, float* d_snrs,
                   void* stream);

/* The same periodogram computed the plain way: one downsample launch per octave cycle and,
 * per bins value, separate FFA, S/N and period launches with the FFA output in global
 * memory -- the loop nest of periodogram.hpp:153-200 moved to the GPU as it stands. */
int rt_periodogram_plain(const float* d_data, size_t size, double tsamp,
                         const uint64_t* h_widths, size_t num_widths, double period_min,
                         double period_max, size_t bins_min, size_t bins_max,
                         double* d_periods, uint32_t* d_foldbins, float* d_snrs, void* stream);

/* ---------------------------------------------------------------------------------
 * Batched search: ffa_search (search.py:11-93) over many DM trials of uneven length.
 * A plan holds everything that depends only on the lengths and the parameters.
 * -------------------------------------------------------------------------------*/
typedef struct rt_search_config {
    double tsamp;          /* sampling time (s)                                   */
    double period_min;     /* s                                                   */
    double period_max;     /* s                                                   */
    uint64_t bins_min;
    uint64_t bins_max;
    int deredden;          /* subtract the running median (time_series.py:95-124) */
    double rmed_width;     /* running median width (s)                            */
    uint64_t rmed_minpts;  /* odd                                                 */
    int already_normalised;
} rt_search_config;

typedef struct rt_search_plan_stats_t {
    uint64_t num_trials, num_cycles, num_transforms, num_work_items, num_multistage;
    uint64_t total_rows;           /* periodogram rows of all trials              */
    uint64_t total_samples;        /* input samples of all trials                 */
    uint64_t downsampled_samples;  /* samples of all downsampled series           */
    uint64_t folded_samples;       /* sum over transforms of rows * bins          */
    uint64_t scrunch_factor;
} rt_search_plan_stats_t;

typedef struct rt_search_plan rt_search_plan;

/* Builds the plan (host work only). widths: trial boxcar widths (all > 0, < bins_min). */
int rt_search_plan_create(const uint64_t* h_lengths, size_t ntrials,
                          const rt_search_config* cfg, const uint64_t* h_widths,
                          size_t num_widths, rt_search_plan** plan);
/* Engine tile choices (0 = default), as picked by an autotuner:
 *   rows_fraction       rows per job as a fraction (0, 1] of what the shared memory holds,
 *                       for transforms of up to 8 jobs' worth of rows;
 *   snr_threads         threads per profile in the S/N: 8 (bins <= 264 only) or 16;
 *   lag_items           work items between two stages of a multi-stage transform (640);
 *   rows_fraction_deep  the same fraction for transforms of more rows than that (0: the
 *                       value of rows_fraction).
 * Results do not depend on these; only the speed does. No counterpart in the reference. */
typedef struct rt_search_tuning {
    double rows_fraction;
    int snr_threads;
    int lag_items;
    double rows_fraction_deep;
} rt_search_tuning;
int rt_search_plan_create_tuned(const uint64_t* h_lengths, size_t ntrials,
                                const rt_search_config* cfg, const uint64_t* h_widths,
                                size_t num_widths, const rt_search_tuning* tuning,
                                rt_search_plan** plan);
/* Tile choices for the transforms of a range of rows and bins, as an autotuner picks them
 * (riptide_b200.tuning): the first rule whose ranges hold a transform's (rows, bins) sets
 * its choices; a field left 0 keeps the plan-wide value of `tuning`.
 *   rows_fraction  rows per job, as a fraction of what shared memory holds at these bins;
 *   snr_threads    threads per profile in the S/N: 8 (bins <= 264 only) or 16;
 *   max_levels     levels a job computes in shared memory (1..8, default 8): fewer levels cut
 *                  a deep transform into more stages, whose outputs pass through L2.
 * Results do not depend on these; only the speed does. No counterpart in the reference. */
typedef struct rt_tile_rule {
    uint32_t rows_min, rows_max;
    uint32_t bins_min, bins_max;
    double rows_fraction;
    int snr_threads;
    int max_levels;
} rt_tile_rule;
int rt_search_plan_create_rules(const uint64_t* h_lengths, size_t ntrials,
                                const rt_search_config* cfg, const uint64_t* h_widths,
                                size_t num_widths, const rt_search_tuning* tuning,
                                const rt_tile_rule* rules, size_t num_rules,
                                rt_search_plan** plan);
/* Row offsets of each trial in the packed outputs: ntrials + 1 entries. */
int rt_search_plan_rows(const rt_search_plan* plan, uint64_t* h_row_offsets);
int rt_search_plan_stats(const rt_search_plan* plan, rt_search_plan_stats_t* stats);
/* Description of one (trial, octave cycle, bins) transform of a plan: its periodogram rows
 * are out_row + [0, rows_eval) of the packed outputs; the series is downsampled by `factor`
 * (1: not downsampled) and folded into rows x bins. num_transforms entries (plan stats). */
typedef struct rt_search_transform {
    uint32_t trial, cycle, bins, rows, rows_eval;
    uint64_t out_row;
    double factor;
    double tau;
    float stdnoise;
} rt_search_transform;
int rt_search_plan_transforms(const rt_search_plan* plan, rt_search_transform* h_out);
/* Per-trial mean and (population) standard deviation of the series the last run normalised
 * (after deredden); 0 and 1 when the plan does not normalise. Synchronises `stream`. */
int rt_search_normalisation(rt_search_plan* plan, double* h_mean, double* h_std, void* stream);
/* Allocates and uploads the plan's device buffers now (otherwise the first run does it;
 * cudaMalloc synchronises the device, so do this before timing or overlapping work). */
int rt_search_plan_prepare(rt_search_plan* plan);
/* Enqueues the search. d_data: the series packed back to back (plan order). Outputs are
 * packed by trial (rt_search_plan_rows). d_normalised (optional, may be NULL) receives the
 * dereddened + normalised series actually searched. Device buffers of the plan are
 * allocated on the first run. Not reentrant per plan. */
int rt_search_run(rt_search_plan* plan, const float* d_data, float* d_normalised,
                  double* d_periods, uint32_t* d_foldbins, float* d_snrs, void* stream);
/* Synchronises `stream` and reports a device-side failure of the last run. */
int rt_search_check(rt_search_plan* plan, void* stream);
/* Replays every later run as one CUDA graph (the run's launches and memsets, captured on
 * the first run with these device pointers, and again when the pointers change); the graph
 * is launched on the run's stream. Runs with stage timing enabled are not replayed. */
int rt_search_set_graph(rt_search_plan* plan, int enable);
/* Number of graph captures made so far (for checking that replays reuse the graph). */
int rt_search_graph_captures(const rt_search_plan* plan, int* h_count);
/* Per-stage CUDA-event timing of rt_search_run (events recorded on the run's stream). */
int rt_search_set_timing(rt_search_plan* plan, int enable);
/* Milliseconds of the last timed run: h_ms[0] deredden + normalise statistics,
 * h_ms[1] downsampling of all cycles, h_ms[2] the persistent FFA + S/N kernel; also the number
 * of kernel launches the run made. Synchronises with the run. */
int rt_search_last_timing(rt_search_plan* plan, float* h_ms, int* h_launches);
/* In-kernel profile of the persistent FFA kernel (16 entries): summed SM cycles of compute
 * thread 0 of every CTA in each phase of a work item (0 boxcar setup, 1 slot hand-over wait,
 * 2 job tree, 3 FFA levels, 4 S/N + periodogram rows, 5 stage output + counters, 6 item
 * decode), 7 cycles the scheduling warps spent choosing items; counts: 8 items blocked on a
 * scratch slot, 9 items blocked on a previous stage, 10 items claimed, 11 empty polls,
 * 12 values computed by FFA levels (rows x bins), 13 FFA levels run, 14 root rows produced,
 * 15 items of stages after the first. */
int rt_search_set_profiling(rt_search_plan* plan, int enable);
int rt_search_phase_cycles(rt_search_plan* plan, uint64_t* h_counters16, int reset);
/* Bound of every wait inside the search kernel (a later stage of a transform waiting for
 * the earlier one, a transform waiting for its scratch slot), in polls with a backoff of up
 * to ~1 us between polls; default 20,000,000. A wait that runs out makes every CTA leave and
 * the run report RT_ETIMEOUT (rt_search_check); the context stays usable. No counterpart in
 * the reference, whose search has no device waits. */
int rt_search_set_wait_limit(rt_search_plan* plan, long long polls);
/* Host-side fault injection for tests of the error paths (no GPU fault is raised):
 * RT_FAULT_STAGE_WAIT: later-stage work items wait for one job more than their previous
 * stage has, a count that is never reached, so the run ends with RT_ETIMEOUT after the wait
 * limit; RT_FAULT_ALLOC: the plan's device buffers are released and allocation number `arg`
 * (from 1) of the next run fails with RT_ENOMEM (everything allocated before it is released
 * again); RT_FAULT_NONE clears both. No counterpart in the reference. */
#define RT_FAULT_NONE 0
#define RT_FAULT_STAGE_WAIT 1
#define RT_FAULT_ALLOC 2
int rt_search_inject_fault(rt_search_plan* plan, int kind, int arg);
void rt_search_plan_destroy(rt_search_plan* plan);

/* ---------------------------------------------------------------------------------
 * Host-buffer pipeline: the batched search of series in host memory, the way the
 * reference's worker pool searches DM trials from host memory (pipeline/worker_pool.py:35-68
 * calling search.py:11-93), with the copies in and out overlapped with the search. The
 * trials are cut into chunks of at most `chunk_trials` consecutive trials (one plan each;
 * the first and last chunks hold a quarter of that when there are enough trials, so that the
 * copies that overlap no search are short); while chunk i is searched, chunk i+1 is copied
 * in and chunk i-1's periodograms are copied out. Host buffers must be page-locked for the
 * copies to overlap.
 * -------------------------------------------------------------------------------*/
typedef struct rt_search_pipeline rt_search_pipeline;

int rt_search_pipeline_create(const uint64_t* h_lengths, size_t ntrials,
                              const rt_search_config* cfg, const uint64_t* h_widths,
                              size_t num_widths, size_t chunk_trials,
                              rt_search_pipeline** pipeline);
/* Row offsets of each trial in the packed host outputs: ntrials + 1 entries. */
int rt_search_pipeline_rows(const rt_search_pipeline* pipeline, uint64_t* h_row_offsets);
int rt_search_pipeline_chunks(const rt_search_pipeline* pipeline, size_t* h_nchunks);
/* Enqueues the search of h_data (series packed back to back) into the host outputs, packed
 * by trial: h_periods f64[L], h_foldbins u32[L], h_snrs f32[L * num_widths]. The work runs
 * after what is already queued on `stream`, and `stream` waits for its end. Returns once
 * enqueued; the host outputs are complete after rt_search_pipeline_check. */
int rt_search_pipeline_run(rt_search_pipeline* pipeline, const float* h_data,
                           double* h_periods, uint32_t* h_foldbins, float* h_snrs,
                           void* stream);
/* Synchronises `stream` and reports a device-side failure of any chunk. */
int rt_search_pipeline_check(rt_search_pipeline* pipeline, void* stream);
void rt_search_pipeline_destroy(rt_search_pipeline* pipeline);

/* ---------------------------------------------------------------------------------
 * Peak detection (peak_detection.py:38-146): the device parts of find_peaks for a batch of
 * periodograms packed by trial (h_row_offsets: ntrials + 1 entries).
 * -------------------------------------------------------------------------------*/
/* Segment statistics of segment_stats (peak_detection.py:38-86): per trial the frequency
 * range is cut into m = ceil(|f[-1] - f[0]| T / segwidth) segments of p = rows // m points;
 * h_seg_offsets (ntrials + 1, output) gives each trial's first segment. With d_fc and d_sc
 * given: d_fc[seg] = median frequency, d_sc[seg * num_widths + iw] = median S/N + nstd *
 * IQR / 1.349 (np.median / np.percentile 'linear'). At most 16384 points per segment. */
int rt_peak_segments(const double* d_periods, const float* d_snrs, size_t num_widths,
                     const uint64_t* h_row_offsets, size_t ntrials, const double* h_tobs,
                     double segwidth, double nstd, uint64_t* h_seg_offsets, double* d_fc,
                     double* d_sc, void* stream);
/* Points whose S/N exceeds both smin and the polynomial threshold in log f (coefficients
 * d_coef[(trial * num_widths + iw) * num_coef + k], highest power first, evaluated as
 * np.polyval), listed in d_sel as row * num_widths + iw in no particular order; *h_count =
 * their number (RT_EINVAL when above `capacity`). Synchronises `stream`. */
int rt_peak_select(const double* d_periods, const float* d_snrs, size_t num_widths,
                   const uint64_t* h_row_offsets, size_t ntrials, const double* d_coef,
                   size_t num_coef, double smin, uint64_t* d_sel, size_t capacity,
                   size_t* h_count, void* stream);

/* ---------------------------------------------------------------------------------
 * Adjoints of the search steps, for gradients of a loss of the periodogram with respect to
 * the searched series (differentiable search; no counterpart in the reference, whose search
 * is not differentiable). Each computes the transpose of the Jacobian of the forward step
 * named, applied to an output gradient.
 * -------------------------------------------------------------------------------*/
/* snr2 (snr.hpp:37-65): gradient with respect to the rows x cols profiles d_in, given the
 * gradient d_gsnr (rows x num_widths) of the S/N. The max over phases is routed to its first
 * maximising phase (per row and width); sum and dmax as the forward computes them. */
int rt_snr2_backward(const float* d_in, size_t rows, size_t cols, const uint64_t* h_widths,
                     size_t num_widths, float stdnoise, const float* d_gsnr, float* d_gin,
                     void* stream);
/* ffa2 (transforms.hpp:13-61): d_gin = FFA^T d_gout for a rows x cols block (the transposed
 * butterfly: each level's gradient gathered from the rows that read it, rolls reversed). */
int rt_ffa2_transpose(const float* d_gout, size_t rows, size_t cols, float* d_gin, void* stream);
/* downsample (downsample.hpp:44-82): d_gin[i] += sum_k w(k, i) d_gout[k] over the
 * floor(size / f) outputs, the same FP64 bounds and float32 edge weights as the forward.
 * Accumulates into d_gin (size values). */
int rt_downsample_adjoint(const float* d_gout, size_t size, double f, float* d_gin,
                          void* stream);
/* Gradient with respect to the searched series of sum(d_gsnr * snrs) for the last run of
 * `plan`, when few periodogram rows carry a gradient (a max-S/N loss: one row per trial):
 * each such row is recomputed from the downsampled series the run left in the plan (so the
 * plan must not have run again since), its boxcar S/N differentiated, and the row gradient
 * taken back through the FFA's shifts and the downsampling. d_z: the normalised series the
 * run searched (rt_search_run's d_normalised); d_gsnr: L x num_widths; d_gz (output, packed
 * like the input) is the gradient with respect to d_z. RT_EINVAL when more than max_rows
 * rows carry a gradient (use the per-transform adjoints instead). */
int rt_search_backward_rows(rt_search_plan* plan, const float* d_z, const float* d_gsnr,
                            float* d_gz, size_t max_rows, void* stream);
/* normalise (time_series.py:67-93), z = (y - mean) / std with population std:
 * d_gy = (g - mean(g) - z * mean(g z)) / std, with d_z the normalised series. */
int rt_normalise_adjoint(const float* d_g, const float* d_z, size_t size, double std_,
                         float* d_gy, void* stream);

/* ---------------------------------------------------------------------------------------
 * Time series files into device memory: the data side of TimeSeries.from_presto_inf /
 * from_sigproc (time_series.py:300-379; reading/presto.py:148-152 reads a .dat as float32;
 * time_series.py:366-377 reads SIGPROC 8-bit data as int8 / uint8 and casts to float32).
 * Headers are parsed by the caller (riptide_b200/reading); these calls move the payload.
 * --------------------------------------------------------------------------------------- */
#define RT_SAMPLES_F32 0 /* float32 samples                                  */
#define RT_SAMPLES_U8 1  /* unsigned 8-bit samples (SIGPROC nbits=8, signed=0) */
#define RT_SAMPLES_I8 2  /* signed 8-bit samples (SIGPROC nbits=8, signed=1)   */

/* Size of a file in bytes. RT_EIO if it cannot be examined. */
int rt_file_size(const char* path, uint64_t* size);
/* Read nbytes at `offset` of a file into host memory dst, split over `threads` parallel
 * pread calls (slices of at least 1 MiB). RT_EIO if the file cannot be opened or holds fewer
 * bytes. */
int rt_read_file(const char* path, uint64_t offset, uint64_t nbytes, void* dst, int threads);
/* Widen n device samples of `encoding` to float32 (astype(np.float32): exact for every 8-bit
 * value). 8-bit sources must be 4-byte aligned. */
int rt_samples_to_f32(const void* d_src, int encoding, size_t n, float* d_dst, void* stream);
/* Load nfiles payloads (nsamples[i] samples of encodings[i] at byte offsets[i] of paths[i])
 * into d_out, packed back to back as float32 (the layout rt_search_run takes). Each file is
 * read in chunks into one half of the page-locked host buffer h_staging (staging_bytes
 * >= 128 KiB) with `threads` parallel reads, while the other half's chunk is copied to
 * the device; 8-bit chunks are copied as bytes and widened on the device. Returns when the
 * last chunk has left h_staging; the conversion may still be running on `stream`. */
int rt_ingest_files(const char* const* paths, const uint64_t* offsets, const uint64_t* nsamples,
                    const int* encodings, size_t nfiles, float* d_out, void* h_staging,
                    size_t staging_bytes, int threads, void* stream);

/* ---------------------------------------------------------------------------------------
 * Folding (TimeSeries.fold, folding.py:21-85): downsample by (period / bins) / tsamp, take
 * the first m * bins samples as m rows of `bins` phases scaled by (m * factor)^-1/2, then
 * sum the rows (subints == 1 or m == 1: one profile), keep them (subints < 0, standing for
 * None, or subints == m), or downsample each phase column by m / subints
 * (downsample_vertical, folding.py:6-18). RT_EINVAL with the reference's messages for a
 * period longer than the data, a bin shorter than tsamp, subints == 0, or subints above the
 * number of periods in the data.
 * --------------------------------------------------------------------------------------- */
/* Output rows (1 when ndim == 1) and ndim of fold(size samples, ...), host only. */
int rt_fold_shape(size_t size, double tsamp, double period, size_t bins, long long subints,
                  size_t* rows, int* ndim);
/* fold of d_in (size float32 samples) into d_out (rows x bins, rt_fold_shape). */
int rt_fold(const float* d_in, size_t size, double tsamp, double period, size_t bins,
            long long subints, float* d_out, void* stream);
/* `count` folds of the same series in one launch (candidate folding): fold c at h_periods[c]
 * with h_bins[c] bins and h_subints[c], written at d_out + h_out_offsets[c]. */
int rt_fold_batched(const float* d_in, size_t size, double tsamp, const double* h_periods,
                    const size_t* h_bins, const long long* h_subints, size_t count,
                    const uint64_t* h_out_offsets, float* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RIPTIDE_B200_H */
