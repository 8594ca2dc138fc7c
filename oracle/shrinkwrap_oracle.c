/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker or the timed CPU baseline.
 *
 * CPU restatement of the reference's CPU shrink-wrap path, written from the
 * reference's behaviour (file:line cited per function), in float (same
 * arithmetic as the reference's FFTW-float build: separate multiply and add,
 * float accumulators, double-computed Gaussian weights) and in double (the
 * FP64 oracle).  The FFT underneath is the project-written one (imro_fft.c);
 * FFTW is not installed here.
 *
 * Pinning: tests/test_oracle.py checks this file against (1) the known-answer
 * tests of the reference's own test suite (Dirac-delta blur, constant-image
 * invariance, planted maximum, Pythagorean HIO error) and (2) the reference's
 * own shrinkWrap built from its sources in oracle/_ref (bit-for-bit on the
 * output, the FFT being shared).
 */
#define _GNU_SOURCE
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include "imro.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846264338327950288
#endif

/* ---- Gaussian weights: src/imresh/libs/calcGaussianKernel.cpp:42-91 ----- */
static int imro_ntaps(double sigma)
{
    int half = (int)ceil(2.884402748387961466 * sigma - 0.5);   /* cpp:63 */
    return 2 * half + 1;
}

int imro_gaussian_weights_f32(double sigma, float *w, int cap)
{
    const int K = imro_ntaps(sigma);
    const int half = (K - 1) / 2;
    if (w == NULL || K > cap) return K;
    const double a = 1.0 / (sqrt(2.0 * M_PI) * sigma);
    const double b = -1.0 / (2.0 * sigma * sigma);
    double sum = 0;
    for (int i = -half; i <= half; ++i) {
        float v = (float)(a * exp(i * i * b));   /* rounded to float first (cpp:84) */
        w[half + i] = v;
        sum += v;
    }
    for (int i = 0; i < K; ++i) w[i] = (float)((double)w[i] / sum);   /* cpp:88 */
    return K;
}

int imro_gaussian_weights_f64(double sigma, double *w, int cap)
{
    const int K = imro_ntaps(sigma);
    const int half = (K - 1) / 2;
    if (w == NULL || K > cap) return K;
    const double a = 1.0 / (sqrt(2.0 * M_PI) * sigma);
    const double b = -1.0 / (2.0 * sigma * sigma);
    double sum = 0;
    for (int i = -half; i <= half; ++i) {
        w[half + i] = a * exp(i * i * b);
        sum += w[half + i];
    }
    for (int i = 0; i < K; ++i) w[i] /= sum;
    return K;
}

/* ---- separable blur with clamp-to-edge border ----------------------------
 * Horizontal: applyKernel (src/imresh/libs/gaussian.cpp:51-163): for every
 * pixel, sum = 0; sum += v[clamp(x-N+k)] * w[k] for k = 0..K-1, in that order.
 * Vertical: gaussianBlurVertical (gaussian.cpp:559-734), same tap order with
 * rows clamped to [0, H-1].  gaussianBlur = horizontal then vertical
 * (gaussian.cpp:737-749). */
#define IMRO_MAXTAPS 127

void imro_blur_h_f32(float *data, int W, int H, double sigma)
{
    float w[IMRO_MAXTAPS];
    const int K = imro_gaussian_weights_f32(sigma, w, IMRO_MAXTAPS);
    if (K > IMRO_MAXTAPS) return;
    const int N = (K - 1) / 2;
    float *row = (float *)malloc(sizeof(float) * (size_t)W);
    for (int y = 0; y < H; ++y) {
        float *d = data + (size_t)y * W;
        memcpy(row, d, sizeof(float) * (size_t)W);
        for (int x = 0; x < W; ++x) {
            float sum = 0;
            for (int k = 0; k < K; ++k) {
                int xs = x - N + k;
                xs = xs < 0 ? 0 : (xs > W - 1 ? W - 1 : xs);
                sum += row[xs] * w[k];
            }
            d[x] = sum;
        }
    }
    free(row);
}

void imro_blur_v_f32(float *data, int W, int H, double sigma)
{
    float w[IMRO_MAXTAPS];
    const int K = imro_gaussian_weights_f32(sigma, w, IMRO_MAXTAPS);
    if (K > IMRO_MAXTAPS) return;
    const int N = (K - 1) / 2;
    float *src = (float *)malloc(sizeof(float) * (size_t)W * (size_t)H);
    memcpy(src, data, sizeof(float) * (size_t)W * (size_t)H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            float sum = 0;
            for (int k = -N; k <= N; ++k) {
                int ys = y + k;
                ys = ys < 0 ? 0 : (ys > H - 1 ? H - 1 : ys);
                sum += src[(size_t)ys * W + x] * w[N + k];
            }
            data[(size_t)y * W + x] = sum;
        }
    free(src);
}

void imro_blur_f32(float *data, int W, int H, double sigma)
{
    imro_blur_h_f32(data, W, H, sigma);
    imro_blur_v_f32(data, W, H, sigma);
}

void imro_blur_f64(double *data, int W, int H, double sigma)
{
    double w[IMRO_MAXTAPS];
    const int K = imro_gaussian_weights_f64(sigma, w, IMRO_MAXTAPS);
    if (K > IMRO_MAXTAPS) return;
    const int N = (K - 1) / 2;
    double *src = (double *)malloc(sizeof(double) * (size_t)W * (size_t)H);
    memcpy(src, data, sizeof(double) * (size_t)W * (size_t)H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            double sum = 0;
            for (int k = 0; k < K; ++k) {
                int xs = x - N + k;
                xs = xs < 0 ? 0 : (xs > W - 1 ? W - 1 : xs);
                sum += src[(size_t)y * W + xs] * w[k];
            }
            data[(size_t)y * W + x] = sum;
        }
    memcpy(src, data, sizeof(double) * (size_t)W * (size_t)H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            double sum = 0;
            for (int k = -N; k <= N; ++k) {
                int ys = y + k;
                ys = ys < 0 ? 0 : (ys > H - 1 ? H - 1 : ys);
                sum += src[(size_t)ys * W + x] * w[N + k];
            }
            data[(size_t)y * W + x] = sum;
        }
    free(src);
}

/* ---- reductions and element-wise steps ----------------------------------- */
/* vectorMax (src/imresh/algorithms/vectorReduce.cpp:73-87): start at the
 * lowest float, keep the larger value. */
float imro_vector_max_f32(const float *data, long n)
{
    float m = -FLT_MAX;
    for (long i = 0; i < n; ++i) m = data[i] > m ? data[i] : m;
    return m;
}

/* calculateHioError (src/imresh/libs/hybridInputOutput.cpp:67-103):
 * total = sum mask*|g'|, count = sum mask, error = sqrt(total)/count.
 * Sums are kept in double here (the reference sums in float). */
double imro_hio_error_f64sum(const float *gp, const float *mask, long n,
                             double *total, double *count)
{
    double t = 0, c = 0;
    for (long i = 0; i < n; ++i) {
        double re = gp[2 * i], im = gp[2 * i + 1];
        t += (double)mask[i] * sqrt(re * re + im * im);
        c += mask[i];
    }
    if (total) *total = t;
    if (count) *count = c;
    return sqrt(t) / c;
}

/* applyComplexModulus (src/imresh/algorithms/vectorElementwise.cpp:59-81):
 * G <- G * M/|G|, with |G| = 0 replaced by 1. */
void imro_apply_modulus_f32(float *d, const float *mod, long n)
{
    for (long i = 0; i < n; ++i) {
        float re = d[2 * i], im = d[2 * i + 1];
        float norm = sqrtf(re * re + im * im);
        if (norm == 0) norm = 1;
        float f = mod[i] / norm;
        d[2 * i] = re * f;
        d[2 * i + 1] = im * f;
    }
}

/* ---- shrinkWrap: src/imresh/algorithms/shrinkWrap.cpp:111-361 ----------- */
#define SW_DEFAULTS()                                                        \
    do {                                                                     \
        if (targetError <= 0) targetError = 1e-5f;     /* cpp:134 */         \
        if (nHio == 0) nHio = 20;                       /* cpp:135 */         \
        if (beta <= 0) beta = 0.9f;                     /* cpp:136 */         \
        if (cutAuto <= 0) cutAuto = 0.04f;              /* cpp:137 */         \
        if (cut <= 0) cut = 0.2f;                       /* cpp:138 */         \
        if (sigma0 <= 0) sigma0 = 3.0f;                 /* cpp:139 */         \
        if (sigmaChange <= 0) sigmaChange = 0.01f;      /* cpp:140 */         \
    } while (0)

int imro_shrinkwrap_f32(float *io, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta, float cutAuto, float cut,
                        float sigma0, float sigmaChange, unsigned nHio,
                        imro_sw_trace *trace)
{
    if (io == NULL) return 1;
    SW_DEFAULTS();
    const long n = (long)W * (long)H;
    float sigma = sigma0;
    float *cur = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    float *gprev = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    float *mask = (float *)malloc(sizeof(float) * (size_t)n);
    if (trace) trace->cycles_run = 0;

    for (long i = 0; i < n; ++i) { cur[2 * i] = io[i]; cur[2 * i + 1] = 0; }   /* cpp:158-163 */
    imro_c2c_2d_f32(cur, (int)H, (int)W, +1);                                   /* cpp:164 */
    memcpy(gprev, cur, sizeof(float) * 2 * (size_t)n);                          /* cpp:173-178 */

    for (unsigned c = 0; c < nCycles; ++c) {
        for (long i = 0; i < n; ++i) {                                          /* cpp:191 */
            float re = cur[2 * i], im = cur[2 * i + 1];
            mask[i] = sqrtf(re * re + im * im);
        }
        imro_blur_f32(mask, (int)W, (int)H, (double)sigma);                     /* cpp:206 */
        float thr = imro_vector_max_f32(mask, n);                               /* cpp:234 */
        thr *= (c == 0) ? cutAuto : cut;                                        /* cpp:235-239 */
        for (long i = 0; i < n; ++i) mask[i] = mask[i] < thr ? 1.0f : 0.0f;    /* cpp:240-242 */
        sigma = (float)fmax(1.5, (double)((1 - sigmaChange) * sigma));          /* cpp:245 */

        for (unsigned it = 0; it < nHio; ++it) {
            for (long i = 0; i < n; ++i) {                                      /* cpp:263-276 */
                if (mask[i] == 1 || cur[2 * i] < 0) {
                    gprev[2 * i] -= beta * cur[2 * i];
                    gprev[2 * i + 1] -= beta * cur[2 * i + 1];
                } else {
                    gprev[2 * i] = cur[2 * i];
                    gprev[2 * i + 1] = cur[2 * i + 1];
                }
            }
            memcpy(cur, gprev, sizeof(float) * 2 * (size_t)n);                  /* out-of-place FORWARD */
            imro_c2c_2d_f32(cur, (int)H, (int)W, -1);                           /* cpp:279 */
            imro_apply_modulus_f32(cur, io, n);                                 /* cpp:282 */
            imro_c2c_2d_f32(cur, (int)H, (int)W, +1);                           /* cpp:301 */
        }
        float err = (float)imro_hio_error_f64sum(cur, mask, n, NULL, NULL);     /* cpp:322 */
        if (trace) {
            trace->cycles_run = (int)c + 1;
            if (trace->errors) trace->errors[c] = err;
        }
        if (targetError > 0 && err < targetError) break;                        /* cpp:328-329 */
    }
    if (trace && trace->mask)
        for (long i = 0; i < n; ++i) trace->mask[i] = (unsigned char)mask[i];
    if (trace && trace->gprime) memcpy(trace->gprime, cur, sizeof(float) * 2 * (size_t)n);
    for (long i = 0; i < n; ++i) io[i] = cur[2 * i];                            /* cpp:349-351 */
    free(cur);
    free(gprev);
    free(mask);
    return 0;
}

int imro_shrinkwrap_f64(double *io, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta, float cutAuto, float cut,
                        float sigma0, float sigmaChange, unsigned nHio,
                        imro_sw_trace *trace)
{
    if (io == NULL) return 1;
    SW_DEFAULTS();
    const long n = (long)W * (long)H;
    float sigma = sigma0;
    double *cur = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *gprev = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *mask = (double *)malloc(sizeof(double) * (size_t)n);
    const double b = beta;
    if (trace) trace->cycles_run = 0;

    for (long i = 0; i < n; ++i) { cur[2 * i] = io[i]; cur[2 * i + 1] = 0; }
    imro_c2c_2d_f64(cur, (int)H, (int)W, +1);
    memcpy(gprev, cur, sizeof(double) * 2 * (size_t)n);

    for (unsigned c = 0; c < nCycles; ++c) {
        for (long i = 0; i < n; ++i) mask[i] = sqrt(cur[2 * i] * cur[2 * i] + cur[2 * i + 1] * cur[2 * i + 1]);
        imro_blur_f64(mask, (int)W, (int)H, (double)sigma);
        double mx = -DBL_MAX;
        for (long i = 0; i < n; ++i) mx = mask[i] > mx ? mask[i] : mx;
        const double thr = mx * (double)((c == 0) ? cutAuto : cut);
        for (long i = 0; i < n; ++i) mask[i] = mask[i] < thr ? 1.0 : 0.0;
        sigma = (float)fmax(1.5, (double)((1 - sigmaChange) * sigma));

        for (unsigned it = 0; it < nHio; ++it) {
            for (long i = 0; i < n; ++i) {
                if (mask[i] == 1 || cur[2 * i] < 0) {
                    gprev[2 * i] -= b * cur[2 * i];
                    gprev[2 * i + 1] -= b * cur[2 * i + 1];
                } else {
                    gprev[2 * i] = cur[2 * i];
                    gprev[2 * i + 1] = cur[2 * i + 1];
                }
            }
            memcpy(cur, gprev, sizeof(double) * 2 * (size_t)n);
            imro_c2c_2d_f64(cur, (int)H, (int)W, -1);
            for (long i = 0; i < n; ++i) {
                double re = cur[2 * i], im = cur[2 * i + 1];
                double norm = sqrt(re * re + im * im);
                if (norm == 0) norm = 1;
                double f = io[i] / norm;
                cur[2 * i] = re * f;
                cur[2 * i + 1] = im * f;
            }
            imro_c2c_2d_f64(cur, (int)H, (int)W, +1);
        }
        double t = 0, cnt = 0;
        for (long i = 0; i < n; ++i) {
            t += mask[i] * sqrt(cur[2 * i] * cur[2 * i] + cur[2 * i + 1] * cur[2 * i + 1]);
            cnt += mask[i];
        }
        float err = (float)(sqrt(t) / cnt);
        if (trace) {
            trace->cycles_run = (int)c + 1;
            if (trace->errors) trace->errors[c] = err;
        }
        if (targetError > 0 && err < targetError) break;
    }
    if (trace && trace->mask)
        for (long i = 0; i < n; ++i) trace->mask[i] = (unsigned char)mask[i];
    if (trace && trace->gprime)
        for (long i = 0; i < 2 * n; ++i) trace->gprime[i] = (float)cur[i];
    for (long i = 0; i < n; ++i) io[i] = cur[2 * i];
    free(cur);
    free(gprev);
    free(mask);
    return 0;
}
