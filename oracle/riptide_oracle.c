/*
 * riptide_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's FFA search path (riptide `libcpp`), used as the
 * checker by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.
 * It is never linked into, loaded by, or called from the product library
 * (riptide_b200/_riptide_b200.so).
 *
 * Parity pinning: tests/test_oracle_pins.py checks this file against the reference's
 * own known-answer tests (FFA_OUT_88 from tests/test_ffa_base_functions.py:25-36, the
 * boxcar top-hat from tests/test_snr.py:62-78, the naive running median from
 * tests/test_running_median.py:7-17) and against golden fixtures produced by the
 * reference's `libcpp` compiled from its own sources (tests/golden/make_golden.py).
 *
 * Every function cites the reference lines it restates (paths relative to the
 * reference project root). Two numeric variants are built from one body:
 *   ORA_T = float  -> the reference's arithmetic (ora_* symbols)
 *   ORA_T = double -> an FP64 restatement (ora64_* symbols), used to state the
 *                     error of each output against FP64.
 * Compiled with -O2 and no fast-math: sums are sequential, in the order the
 * reference source writes them. (The reference build adds -fassociative-math and
 * -march=native, setup.py:13-20,34, which lets GCC reorder the downsample sum; the
 * parity tests therefore use a tolerance for downsample and S/N.)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORA_T
#define ORA_T float
#define ORA(name) ora_##name
#define ORA_IS_F32 1
#else
#define ORA_IS_F32 0
#endif

/* ---------------------------------------------------------------------------------
 * Error reporting: 0 = ok, nonzero = invalid argument (the reference raises
 * std::invalid_argument -> ValueError with these messages).
 * -------------------------------------------------------------------------------*/
#if ORA_IS_F32
static const char* g_ora_err = "";
const char* ora_last_error(void) { return g_ora_err; }
static int ora_fail(const char* msg) { g_ora_err = msg; return 1; }
#else
static int ora_fail(const char* msg) { (void)msg; return 1; }
size_t ora_downsampled_size(size_t num_samples, double f);
double ora_downsampled_variance(size_t num_samples, double f);
size_t ora_ceilshift(size_t rows, size_t cols, double pmax);
int ora_periodogram_check_arguments(size_t size, double tsamp, double period_min,
                                    double period_max, size_t bins_min, size_t bins_max);
#endif

static size_t ora_min3(size_t a, size_t b, size_t c)
{
    size_t m = a < b ? a : b;
    return m < c ? m : c;
}

/* ---------------------------------------------------------------------------------
 * Plan helpers (shared, always double). cpp/downsample.hpp:21-24, 29-38;
 * cpp/periodogram.hpp:54-57, 25-40.
 * -------------------------------------------------------------------------------*/
#if ORA_IS_F32
size_t ora_downsampled_size(size_t num_samples, double f)
{
    return (size_t)floor(num_samples / f); /* downsample.hpp:21-24 */
}

double ora_downsampled_variance(size_t num_samples, double f)
{
    /* downsample.hpp:29-38 */
    const double k = floor(f);
    const double r = f - k;
    const double x = ora_downsampled_size(num_samples, f) * r;
    if (x > 1)
        return f - 1.0 / 3.0;
    return pow(k - 1, 2) + 2.0 / 3.0 * pow(x, 2) - x + 1.0;
}

size_t ora_ceilshift(size_t rows, size_t cols, double pmax)
{
    return (size_t)ceil(cols * (rows - 1.0) * (1.0 - cols / pmax)); /* periodogram.hpp:54-57 */
}

int ora_periodogram_check_arguments(size_t size, double tsamp, double period_min,
                                    double period_max, size_t bins_min, size_t bins_max)
{
    (void)size;
    /* periodogram.hpp:25-40, same messages and order */
    if (!(tsamp > 0)) return ora_fail("tsamp must be > 0");
    if (!(period_min > 0)) return ora_fail("period_min must be > 0");
    if (!(period_max > period_min)) return ora_fail("period_max must be > period_min");
    if (!(bins_min > 1)) return ora_fail("bins_min must be > 1");
    if (!(bins_max >= bins_min)) return ora_fail("bins_max must be >= bins_min");
    if (!(period_min >= tsamp * bins_min))
        return ora_fail("Must have: period_min >= tsamp * bins_min ");
    return 0;
}

int ora_periodogram_length(size_t size, double tsamp, double period_min, double period_max,
                           size_t bins_min, size_t bins_max, size_t* length)
{
    /* periodogram.hpp:63-109 */
    if (ora_periodogram_check_arguments(size, tsamp, period_min, period_max, bins_min, bins_max))
        return 1;
    const double ds_ini = period_min / (tsamp * bins_min);
    const double ds_geo = (bins_max + 1.0) / bins_min;
    const size_t num_downsamplings = (size_t)ceil(log(period_max / period_min) / log(ds_geo));
    size_t len = 0;
    for (size_t ids = 0; ids < num_downsamplings; ++ids) {
        const double f = ds_ini * pow(ds_geo, ids);
        const double tau = f * tsamp;
        const double period_max_samples = period_max / tau;
        const size_t n = ora_downsampled_size(size, f);
        const size_t bstart = bins_min;
        const size_t bstop = ora_min3(bins_max, n, (size_t)period_max_samples);
        for (size_t bins = bstart; bins <= bstop; ++bins) {
            const size_t rows = n / bins;
            const double period_ceil =
                period_max_samples < bins + 1.0 ? period_max_samples : bins + 1.0;
            const size_t cs = ora_ceilshift(rows, bins, period_ceil);
            len += rows < cs ? rows : cs;
        }
    }
    *length = len;
    return 0;
}
#endif

/* ---------------------------------------------------------------------------------
 * Elementwise kernels. cpp/kernels.hpp
 * -------------------------------------------------------------------------------*/
static void ORA(add)(const ORA_T* x, const ORA_T* y, size_t size, ORA_T* z)
{
    for (size_t i = 0; i < size; ++i) z[i] = x[i] + y[i]; /* kernels.hpp:9-13 */
}

void ORA(fused_rollback_add)(const ORA_T* x, const ORA_T* y, size_t size, size_t shift, ORA_T* z)
{
    /* kernels.hpp:19-25: z = x + roll(y, -shift) */
    const size_t p = shift % size;
    const size_t q = size - p;
    ORA(add)(x, y + p, q, z);
    ORA(add)(x + q, y, p, z + q);
}

void ORA(rollback)(const ORA_T* x, size_t size, size_t shift, ORA_T* out)
{
    /* kernels.hpp:32-38 */
    const size_t p = shift % size;
    const size_t q = size - p;
    memcpy(out, x + p, q * sizeof(ORA_T));
    memcpy(out + q, x, p * sizeof(ORA_T));
}

void ORA(circular_prefix_sum)(const ORA_T* x, size_t size, size_t nsum, ORA_T* out)
{
    /* kernels.hpp:73-101: double accumulator, then wraps added in working precision */
    double acc = 0;
    const size_t jmax = size < nsum ? size : nsum;
    for (size_t j = 0; j < jmax; ++j) {
        acc += x[j];
        out[j] = (ORA_T)acc;
    }
    if (nsum <= size) return;
    const ORA_T sumx = (ORA_T)acc;
    const size_t q = nsum / size;
    const size_t r = nsum % size;
    for (size_t i = 1; i < q; ++i)
        for (size_t j = 0; j < size; ++j) out[i * size + j] = out[j] + (ORA_T)i * sumx;
    for (size_t j = 0; j < r; ++j) out[q * size + j] = out[j] + (ORA_T)q * sumx;
}

/* ---------------------------------------------------------------------------------
 * FFA transform. cpp/transforms.hpp:13-61, cpp/block.hpp:30-43
 * A block is (data, rows, cols); head = first rows>>1 rows, tail = the rest.
 * -------------------------------------------------------------------------------*/
static void ORA(merge)(const ORA_T* head, size_t head_rows, const ORA_T* tail, size_t tail_rows,
                       ORA_T* out, size_t m, size_t p)
{
    /* transforms.hpp:13-27. Row indices use float32 arithmetic; the reference build
     * (-O3 -march=native, GCC's default -ffp-contract=fast) evaluates kh*s+0.5f as one
     * fused multiply-add, restated here with fmaf. */
    const float kh = ((float)head_rows - 1.0f) / ((float)m - 1.0f);
    const float kt = ((float)tail_rows - 1.0f) / ((float)m - 1.0f);
    for (size_t s = 0; s < m; ++s) {
        const size_t h = (size_t)fmaf(kh, (float)s, 0.5f);
        const size_t t = (size_t)fmaf(kt, (float)s, 0.5f);
        const size_t b = s - (h + t);
        ORA(fused_rollback_add)(head + h * p, tail + t * p, p, h + b, out + s * p);
    }
}

static void ORA(transform_rec)(const ORA_T* in, ORA_T* temp, ORA_T* out, size_t m, size_t p)
{
    /* transforms.hpp:30-50 */
    if (m == 2) {
        ORA(add)(in, in + p, p, out);
        ORA(fused_rollback_add)(in, in + p, p, 1, out + p);
        return;
    } else if (m == 1) {
        memcpy(out, in, p * sizeof(ORA_T));
        return;
    }
    const size_t h = m >> 1;
    /* transform(input.head(), out.head(), temp.head()) : the roles of temp/out swap */
    ORA(transform_rec)(in, out, temp, h, p);
    ORA(transform_rec)(in + h * p, out + h * p, temp + h * p, m - h, p);
    ORA(merge)(temp, h, temp + h * p, m - h, out, m, p);
}

void ORA(transform)(const ORA_T* in, size_t rows, size_t cols, ORA_T* temp, ORA_T* out)
{
    ORA(transform_rec)(in, temp, out, rows, cols); /* transforms.hpp:53-61 */
}

int ORA(ffa2)(const ORA_T* in, size_t rows, size_t cols, ORA_T* out)
{
    /* python_bindings.cpp:84-96: allocate temp, transform */
    if (rows == 0 || cols == 0) return 0;
    ORA_T* temp = (ORA_T*)malloc(rows * cols * sizeof(ORA_T));
    if (!temp) return ora_fail("out of memory");
    ORA(transform)(in, rows, cols, temp, out);
    free(temp);
    return 0;
}

/* ---------------------------------------------------------------------------------
 * Boxcar S/N. cpp/snr.hpp
 * -------------------------------------------------------------------------------*/
static ORA_T ORA(diff_max)(const ORA_T* x, const ORA_T* y, size_t size)
{
    /* kernels.hpp:50-60 */
    ORA_T dmax = x[0] - y[0];
    for (size_t i = 1; i < size; ++i) {
        const ORA_T d = x[i] - y[i];
        if (d > dmax) dmax = d;
    }
    return dmax;
}

int ORA(check_snr_args)(const uint64_t* widths, size_t num_widths, size_t bins, float stdnoise)
{
    /* snr.hpp:14-31 */
    if (!(stdnoise > 0)) return ora_fail("stdnoise must be > 0");
    for (size_t i = 0; i < num_widths; ++i)
        if (!((widths[i] > 0) & (widths[i] < bins)))
            return ora_fail("trial widths must be all > 0 and < columns");
    return 0;
}

void ORA(snr1)(const ORA_T* arr, size_t size, const uint64_t* widths, size_t num_widths,
               ORA_T stdnoise, ORA_T* out)
{
    /* snr.hpp:37-55 */
    size_t wmax = 0;
    for (size_t i = 0; i < num_widths; ++i) if (widths[i] > wmax) wmax = widths[i];
    ORA_T* cpfsum = (ORA_T*)malloc((size + wmax) * sizeof(ORA_T));
    ORA(circular_prefix_sum)(arr, size, size + wmax, cpfsum);
    const ORA_T sum = cpfsum[size - 1];
    for (size_t iw = 0; iw < num_widths; ++iw) {
        const size_t w = widths[iw];
#if ORA_IS_F32
        const float h = sqrtf((size - w) / (float)(size * w));
        const float b = w / (float)(size - w) * h;
#else
        const double h = sqrt((size - w) / (double)(size * w));
        const double b = w / (double)(size - w) * h;
#endif
        const ORA_T dmax = ORA(diff_max)(cpfsum + w, cpfsum, size);
        /* snr.hpp:52 ((h + b) * dmax - b * sum) / stdnoise. The reference build contracts
         * the first product and the subtraction into one fused multiply-add; restated
         * with fma so that this file reproduces the built reference bit for bit. */
#if ORA_IS_F32
        out[iw] = fmaf(h + b, dmax, -(b * sum)) / stdnoise;
#else
        out[iw] = fma(h + b, dmax, -(b * sum)) / stdnoise;
#endif
    }
    free(cpfsum);
}

void ORA(snr2)(const ORA_T* block, size_t rows, size_t cols, const uint64_t* widths,
               size_t num_widths, ORA_T stdnoise, ORA_T* out)
{
    for (size_t i = 0; i < rows; ++i) /* snr.hpp:58-65 */
        ORA(snr1)(block + i * cols, cols, widths, num_widths, stdnoise, out + i * num_widths);
}

/* ---------------------------------------------------------------------------------
 * Downsampling by a real factor. cpp/downsample.hpp:11-82
 * -------------------------------------------------------------------------------*/
int ORA(downsample)(const ORA_T* in, size_t size, double f, ORA_T* out)
{
    if (!((f > 1.0) & (f <= size))) /* downsample.hpp:11-16 */
        return ora_fail("Downsampling factor must verify: 1 < f <= size");
    const size_t N = size;
    const size_t n = ora_downsampled_size(N, f);
    for (size_t k = 0; k < n; ++k) { /* downsample.hpp:54-81 */
        const double start = k * f;
        const double end = start + f;
        const size_t imin = (size_t)floor(start);
        const double fe = floor(end);
        const size_t imax = (size_t)(fe < N - 1.0 ? fe : N - 1.0);
        const ORA_T wmin = (ORA_T)((imin + 1) - start);
        const ORA_T wmax = (ORA_T)(end - imax);
        ORA_T acc = wmin * in[imin];
        for (size_t i = imin + 1; i < imax; ++i) acc += in[i];
        acc += wmax * in[imax];
        out[k] = acc;
    }
    return 0;
}

/* ---------------------------------------------------------------------------------
 * Periodogram. cpp/periodogram.hpp:117-201
 * -------------------------------------------------------------------------------*/
int ORA(periodogram)(const ORA_T* data, size_t size, double tsamp, const uint64_t* widths,
                     size_t num_widths, double period_min, double period_max, size_t bins_min,
                     size_t bins_max, double* periods, uint32_t* foldbins, ORA_T* snr)
{
    if (ora_periodogram_check_arguments(size, tsamp, period_min, period_max, bins_min, bins_max))
        return 1;
    const double ds_ini = period_min / (tsamp * bins_min);
    const double ds_geo = (bins_max + 1.0) / bins_min;
    const size_t num_downsamplings = (size_t)ceil(log(period_max / period_min) / log(ds_geo));
    const size_t bufsize = ora_downsampled_size(size, ds_ini);
    ORA_T* input_mem = (ORA_T*)malloc((bufsize ? bufsize : 1) * sizeof(ORA_T));
    ORA_T* ffabuf = (ORA_T*)malloc((bufsize ? bufsize : 1) * sizeof(ORA_T));
    ORA_T* ffaout = (ORA_T*)malloc((bufsize ? bufsize : 1) * sizeof(ORA_T));
    for (size_t ids = 0; ids < num_downsamplings; ++ids) {
        const double f = ds_ini * pow(ds_geo, ids);
        const double tau = f * tsamp;
        const double period_max_samples = period_max / tau;
        const size_t n = ora_downsampled_size(size, f);
        const ORA_T* input;
        if (f == 1) {
            input = data;
        } else {
            if (ORA(downsample)(data, size, f, input_mem)) { /* throws in the reference */
                free(input_mem);
                free(ffabuf);
                free(ffaout);
                return 1;
            }
            input = input_mem;
        }
        const size_t bstart = bins_min;
        const size_t bstop = ora_min3(bins_max, n, (size_t)period_max_samples);
        for (size_t bins = bstart; bins <= bstop; ++bins) {
            const size_t rows = n / bins;
            const ORA_T stdnoise = (ORA_T)sqrt(rows * ora_downsampled_variance(size, f));
            const double period_ceil =
                period_max_samples < bins + 1.0 ? period_max_samples : bins + 1.0;
            const size_t cs = ora_ceilshift(rows, bins, period_ceil);
            const size_t rows_eval = rows < cs ? rows : cs;
            ORA(transform)(input, rows, bins, ffabuf, ffaout);
            ORA(snr2)(ffaout, rows_eval, bins, widths, num_widths, stdnoise, snr);
            for (size_t s = 0; s < rows_eval; ++s) {
                /* periodogram.hpp:192 tau * bins * bins / (...). The reference build's
                 * -fassociative-math evaluates bins * bins first (exact in double). */
                periods[s] = tau * ((double)bins * bins) / (bins - s / (rows - 1.0));
                foldbins[s] = (uint32_t)bins;
            }
            snr += rows_eval * num_widths;
            periods += rows_eval;
            foldbins += rows_eval;
        }
    }
    free(input_mem);
    free(ffabuf);
    free(ffaout);
    return 0;
}

/* ---------------------------------------------------------------------------------
 * Running median. cpp/running_median.hpp:13-132 (float only)
 * -------------------------------------------------------------------------------*/
#if ORA_IS_F32
static void ora_swap(float* a, float* b) { float t = *a; *a = *b; *b = t; }

static size_t ora_partition(float* data, size_t start, size_t end, size_t ipiv)
{
    /* running_median.hpp:13-35 */
    const float pivot = data[ipiv];
    ora_swap(&data[ipiv], &data[end]);
    size_t j = start;
    for (size_t i = start; i < end; ++i) {
        if (data[i] < pivot) {
            ora_swap(&data[i], &data[j]);
            ++j;
        }
    }
    ora_swap(&data[j], &data[end]);
    return j;
}

static float ora_nth_element(float* data, size_t start, size_t end, size_t n)
{
    /* running_median.hpp:39-56, iterative form of the same recursion */
    for (;;) {
        if (start == end) return data[start];
        const size_t j = ora_partition(data, start, end, end);
        if (j == n) return data[j];
        if (j < n) start = j + 1;
        else end = j - 1;
    }
}

typedef struct {
    size_t width, writepos;
    float* ring;
    float* buffer;
} ora_rmed_t;

static float ora_rmed_push(ora_rmed_t* r, float val)
{
    /* running_median.hpp:72-95 */
    r->ring[r->writepos] = val;
    if (++r->writepos >= r->width) r->writepos = 0;
    memcpy(r->buffer, r->ring, r->width * sizeof(float));
    return ora_nth_element(r->buffer, 0, r->width - 1, r->width / 2);
}

int ora_running_median(const float* data, size_t size, size_t width, float* out)
{
    /* running_median.hpp:100-132 */
    if (!(width % 2)) return ora_fail("width must be an odd number");
    if (!(width < size)) return ora_fail("width must be < size");
    const size_t half = width / 2;
    ora_rmed_t r;
    r.width = width;
    r.writepos = 0;
    r.ring = (float*)calloc(width, sizeof(float));
    r.buffer = (float*)calloc(width, sizeof(float));
    for (size_t i = 0; i < half + 1; ++i) ora_rmed_push(&r, data[0]);
    for (size_t i = 1; i < half; ++i) ora_rmed_push(&r, data[i]);
    for (size_t i = half; i < size; ++i) out[i - half] = ora_rmed_push(&r, data[i]);
    for (size_t i = 0; i < half; ++i) out[size - half + i] = ora_rmed_push(&r, data[size - 1]);
    free(r.ring);
    free(r.buffer);
    return 0;
}
#endif
