// Declarations shared by the kernel files of riptide_b200.
#pragma once
#include "common.cuh"
#include "ffa_core.cuh"

namespace rt {

// Dynamic shared memory of the FFA / S/N kernels (one CTA per SM).
constexpr size_t kFfaSmemBytes = 226 * 1024;

int ffa_cap_rows(int b);
size_t ffa_scratch_floats(int m, int b);
int detect_fast_widths(const int* w, int nw);
const char* last_error();

// FFA transform of an m x b block (device pointers). rows_out <= m root rows are produced
// (the reference's ffa2 uses rows_out = m). `scratch` holds ffa_scratch_floats(m, b)
// floats. Errors of the device plan are reported through d_err.
int ffa_transform(const float* in, int m, int b, int rows_out, float* out, float* scratch,
                  int* d_err, cudaStream_t st);

int snr2(const float* x, size_t rows, size_t cols, const int* d_widths, const int* h_widths,
         int nw, float stdnoise, float* out, cudaStream_t st);
int rollback(const float* x, size_t size, size_t shift, float* out, cudaStream_t st);
int fused_rollback_add(const float* x, const float* y, size_t size, size_t shift, float* out,
                       cudaStream_t st);
int circular_prefix_sum(const float* x, size_t size, size_t nsum, float* out, cudaStream_t st);
int launch_periods(double* periods, uint32_t* foldbins, size_t rows_eval, double tau, int bins,
                   size_t rows, cudaStream_t st);
int launch_running_median(const float* x, const size_t* d_lengths, const size_t* d_offsets,
                          int ntrials, size_t max_len, int width, float* out, cudaStream_t st);

// Downsampling of many series by many factors in one pass (device arrays).
constexpr int kDsStage = 8192;        // input samples staged per CTA (segment + halo)
constexpr int kDsHalo = 4096;         // largest halo: factors up to kDsHalo - 2
constexpr int kDsMaxCycles = 256;

struct DsJob {
    const float* in;            // packed input series
    const size_t* in_off;       // [ntrials] offset of each series
    const size_t* lengths;      // [ntrials]
    const double* mean;         // [ntrials] or null: values are normalised as (v - mean) / norm
    const double* norm;         // [ntrials] or null
    float* norm_out;            // packed normalised series (optional)
    const double* f;            // [ncycles] factors
    const int* use_seg;         // [ncycles] 1: segment kernel, 0: wide kernel
    float* out;                 // packed outputs
    const size_t* out_off;      // [ntrials * ncycles]
    int ncycles;
    int seg;                    // output ownership segment (input samples), set by the launcher
    // host copies for the launcher
    const double* f_host;       // [ncycles]
    const int* use_seg_host;
    const int* skip_host;       // [ncycles] cycles with nothing to produce (f == 1)
};

int launch_downsample(const DsJob& job, int ntrials, size_t max_len, cudaStream_t st);

inline bool ds_use_segments(double f) { return f + 2.0 <= (double)kDsHalo; }

}  // namespace rt
