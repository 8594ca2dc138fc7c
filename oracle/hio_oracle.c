/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker or the timed CPU baseline.
 *
 * CPU restatement of the reference's fixed-support hybrid input-output with
 * a random initial phase, imresh::libs::hybridInputOutput and addRandomPhase
 * (src/imresh/libs/hybridInputOutput.cpp:126-184, 193-306), in float (the
 * reference's arithmetic: separate multiply and add, float division) and in
 * double (the FP64 yardstick), over the project FFT (imro_fft.c).  The random
 * field comes from the C library's own srand()/rand(), the generator the
 * reference calls.
 *
 * Pinning: tests/test_oracle.py compares imro_hio_f32 with the reference's own
 * hybridInputOutput compiled from its sources into oracle/_ref (bit for bit).
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "imro.h"

/* addRandomPhase (cpp:126-184): phase of the 2D FFT of a rand()/RAND_MAX
 * field, applied to the modulus.  std::arg of a complex<float> is atan2f;
 * the unqualified cos/sin of that float resolve to the double functions, and
 * the float modulus times the double cosine is rounded to float on store. */
static void hio_random_phase_f32(const float *mod, float *cur, long n, int W, int H, unsigned seed)
{
    float *tmp = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    srand(seed);                                                               /* cpp:160 */
    for (long i = 0; i < n; ++i) {                                             /* cpp:161-165 */
        tmp[2 * i] = (float)rand() / RAND_MAX;
        tmp[2 * i + 1] = 0;
    }
    imro_c2c_2d_f32(tmp, H, W, -1);                                            /* cpp:167-171 */
    for (long i = 0; i < n; ++i) {                                             /* cpp:175-182 */
        const float phase = atan2f(tmp[2 * i + 1], tmp[2 * i]);
        cur[2 * i] = (float)((double)mod[i] * cos((double)phase));
        cur[2 * i + 1] = (float)((double)mod[i] * sin((double)phase));
    }
    free(tmp);
}

static void hio_random_phase_f64(const double *mod, double *cur, long n, int W, int H, unsigned seed)
{
    double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    srand(seed);
    for (long i = 0; i < n; ++i) {
        tmp[2 * i] = (double)((float)rand() / RAND_MAX);
        tmp[2 * i + 1] = 0;
    }
    imro_c2c_2d_f64(tmp, H, W, -1);
    for (long i = 0; i < n; ++i) {
        const double phase = atan2(tmp[2 * i + 1], tmp[2 * i]);
        cur[2 * i] = mod[i] * cos(phase);
        cur[2 * i + 1] = mod[i] * sin(phase);
    }
    free(tmp);
}

void imro_random_phase_f32(const float *mod, float *out, unsigned W, unsigned H, unsigned seed)
{
    hio_random_phase_f32(mod, out, (long)W * (long)H, (int)W, (int)H, seed);
}

static void hio_trace_error(imro_hio_trace *trace, unsigned k, float err)
{
    if (!trace) return;
    trace->last_error = err;
    if (trace->errors && (long)k < (long)trace->errors_cap) trace->errors[k] = err;
}

/* hybridInputOutput (cpp:193-306). */
int imro_hio_f32(float *io, const unsigned char *mask, unsigned W, unsigned H, unsigned nCycles,
                 float targetError, float beta, unsigned seed, imro_hio_trace *trace)
{
    if (io == NULL || mask == NULL) return 1;                                  /* cpp:205 */
    if (nCycles == 0) nCycles = UINT_MAX;                                      /* cpp:208 */
    if (beta <= 0) beta = 0.9f;                                                /* cpp:209 */
    const long n = (long)W * (long)H;
    float *cur = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    float *gprev = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    hio_random_phase_f32(io, cur, n, (int)W, (int)H, seed);                    /* cpp:227 */
    unsigned k = 0;
    for (;;) {
        imro_c2c_2d_f32(cur, (int)H, (int)W, +1);                              /* cpp:233 */
        if (k == 0) memcpy(gprev, cur, sizeof(float) * 2 * (size_t)n);         /* cpp:238-239 */
        const int test = targetError > 0;
        if (test || k >= nCycles) {
            double t = 0, c = 0;
            for (long i = 0; i < n; ++i) {                                     /* calculateHioError */
                const float re = cur[2 * i], im = cur[2 * i + 1];
                t += (double)mask[i] * (double)sqrtf(re * re + im * im);
                c += (double)mask[i];
            }
            hio_trace_error(trace, k, (float)(sqrt(t) / c));
            if (test && (float)(sqrt(t) / c) < targetError) break;            /* cpp:242-245 */
        }
        if (k >= nCycles) break;                                               /* cpp:246-247 */
        for (long i = 0; i < n; ++i) {                                         /* cpp:250-258 */
            if (mask[i] == 1 || cur[2 * i] < 0) {
                cur[2 * i] = gprev[2 * i] - beta * cur[2 * i];
                cur[2 * i + 1] = gprev[2 * i + 1] - beta * cur[2 * i + 1];
            }
        }
        memcpy(gprev, cur, sizeof(float) * 2 * (size_t)n);                     /* cpp:259 */
        imro_c2c_2d_f32(cur, (int)H, (int)W, -1);                              /* cpp:262 */
        for (long i = 0; i < n; ++i) {                                         /* cpp:281-289 */
            const float re = cur[2 * i], im = cur[2 * i + 1];
            const float f = io[i] / sqrtf(re * re + im * im);
            cur[2 * i] = re * f;
            cur[2 * i + 1] = im * f;
        }
        ++k;
    }
    if (trace) trace->iterations = (int)k;
    for (long i = 0; i < n; ++i) io[i] = cur[2 * i];                           /* cpp:294-296 */
    free(cur);
    free(gprev);
    return 0;
}

int imro_hio_f64(double *io, const unsigned char *mask, unsigned W, unsigned H, unsigned nCycles,
                 float targetError, float beta, unsigned seed, imro_hio_trace *trace)
{
    if (io == NULL || mask == NULL) return 1;
    if (nCycles == 0) nCycles = UINT_MAX;
    if (beta <= 0) beta = 0.9f;
    const double b = beta;
    const long n = (long)W * (long)H;
    double *cur = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *gprev = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    hio_random_phase_f64(io, cur, n, (int)W, (int)H, seed);
    unsigned k = 0;
    for (;;) {
        imro_c2c_2d_f64(cur, (int)H, (int)W, +1);
        if (k == 0) memcpy(gprev, cur, sizeof(double) * 2 * (size_t)n);
        const int test = targetError > 0;
        if (test || k >= nCycles) {
            double t = 0, c = 0;
            for (long i = 0; i < n; ++i) {
                t += (double)mask[i] * sqrt(cur[2 * i] * cur[2 * i] + cur[2 * i + 1] * cur[2 * i + 1]);
                c += (double)mask[i];
            }
            hio_trace_error(trace, k, (float)(sqrt(t) / c));
            if (test && (float)(sqrt(t) / c) < targetError) break;
        }
        if (k >= nCycles) break;
        for (long i = 0; i < n; ++i) {
            if (mask[i] == 1 || cur[2 * i] < 0) {
                cur[2 * i] = gprev[2 * i] - b * cur[2 * i];
                cur[2 * i + 1] = gprev[2 * i + 1] - b * cur[2 * i + 1];
            }
        }
        memcpy(gprev, cur, sizeof(double) * 2 * (size_t)n);
        imro_c2c_2d_f64(cur, (int)H, (int)W, -1);
        for (long i = 0; i < n; ++i) {
            const double re = cur[2 * i], im = cur[2 * i + 1];
            const double f = io[i] / sqrt(re * re + im * im);
            cur[2 * i] = re * f;
            cur[2 * i + 1] = im * f;
        }
        ++k;
    }
    if (trace) trace->iterations = (int)k;
    for (long i = 0; i < n; ++i) io[i] = cur[2 * i];
    free(cur);
    free(gprev);
    return 0;
}
