/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * C API of liboracle.so: a CPU restatement of the reference's CPU shrink-wrap
 * path (src/imresh/algorithms/shrinkWrap.cpp:111-361 and the functions it
 * calls), in float (mirrors the reference's FFTW-float build) and in double
 * (the FP64 oracle), plus the project-written FFT it runs on.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as
 * the checker / the timed CPU baseline.
 */
#ifndef IMRO_H
#define IMRO_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- FFT (unnormalised; sign -1 forward, +1 backward) ------------------- */
/* row-major [H][W] interleaved complex, in place, rows then columns */
void imro_c2c_2d_f32(float *data, int H, int W, int sign);
void imro_c2c_2d_f64(double *data, int H, int W, int sign);
/* `howmany` contiguous sequences of length n, in place */
void imro_c2c_rows_f32(float *data, int n, int howmany, int sign);
void imro_c2c_rows_f64(double *data, int n, int howmany, int sign);
/* along the columns of a row-major [H][W] array, in place */
void imro_c2c_cols_f32(float *data, int H, int W, int sign);
void imro_c2c_cols_f64(double *data, int H, int W, int sign);

/* ---- kernel-level restatements ------------------------------------------ */
/* calcGaussianKernel (src/imresh/libs/calcGaussianKernel.cpp:42-91):
 * returns the tap count K = 2*ceil(2.884402748387961466*sigma - 0.5) + 1 and,
 * when K <= cap, writes the normalised float weights. */
int imro_gaussian_weights_f32(double sigma, float *w, int cap);
int imro_gaussian_weights_f64(double sigma, double *w, int cap);
/* gaussianBlurHorizontal / gaussianBlurVertical / gaussianBlur, clamp border
 * (src/imresh/libs/gaussian.cpp:51-163, 180-197, 559-749) */
void imro_blur_h_f32(float *data, int W, int H, double sigma);
void imro_blur_v_f32(float *data, int W, int H, double sigma);
void imro_blur_f32(float *data, int W, int H, double sigma);
void imro_blur_f64(double *data, int W, int H, double sigma);
/* vectorMax (src/imresh/algorithms/vectorReduce.cpp:73-87) */
float imro_vector_max_f32(const float *data, long n);
/* calculateHioError (src/imresh/libs/hybridInputOutput.cpp:67-103) with the
 * two sums accumulated in double; returns sqrt(total)/count. */
double imro_hio_error_f64sum(const float *gprime, const float *mask, long n,
                             double *total, double *count);
/* applyComplexModulus (src/imresh/algorithms/vectorElementwise.cpp:59-81) */
void imro_apply_modulus_f32(float *data, const float *modulus, long n);

/* ---- the full path -------------------------------------------------------- */
typedef struct imro_sw_trace {
    int cycles_run;        /* cycles whose HIO block completed            */
    float *errors;         /* [nCycles] error after each cycle, or NULL   */
    unsigned char *mask;   /* [W*H] mask of the last cycle run, or NULL   */
    float *gprime;         /* [2*W*H] final g' (complex), or NULL          */
} imro_sw_trace;

/* shrinkWrap (src/imresh/algorithms/shrinkWrap.cpp:111-361) with its default
 * substitution for arguments <= 0 (cpp:133-140).  io: W*H modulus in, W*H
 * Re(g') out.  Returns 0, or 1 for a NULL buffer as the reference does. */
int imro_shrinkwrap_f32(float *io, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta, float cutAuto, float cut,
                        float sigma0, float sigmaChange, unsigned nHio,
                        imro_sw_trace *trace);
/* Same algorithm with every array and every arithmetic step in double (the
 * FP64 oracle).  The sigma schedule stays in float as in the reference. */
int imro_shrinkwrap_f64(double *io, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta, float cutAuto, float cut,
                        float sigma0, float sigmaChange, unsigned nHio,
                        imro_sw_trace *trace);

/* ---- fixed-support HIO with a random initial phase ------------------------
 * hybridInputOutput / addRandomPhase (src/imresh/libs/hybridInputOutput.cpp:126-306):
 * io: W*H modulus in, Re(g') out; mask: W*H bytes, 1 = outside the support.
 * nCycles 0 = unbounded, beta <= 0 = 0.9, targetError <= 0 = no error test.
 * The random field is the C library's rand() after srand(seed). */
typedef struct imro_hio_trace {
    int iterations;        /* HIO updates applied before the returned g'   */
    float last_error;      /* last error evaluated                         */
    float *errors;         /* [errors_cap] error of each tested g', or NULL */
    int errors_cap;
} imro_hio_trace;
int imro_hio_f32(float *io, const unsigned char *mask, unsigned W, unsigned H, unsigned nCycles,
                 float targetError, float beta, unsigned seed, imro_hio_trace *trace);
int imro_hio_f64(double *io, const unsigned char *mask, unsigned W, unsigned H, unsigned nCycles,
                 float targetError, float beta, unsigned seed, imro_hio_trace *trace);
/* addRandomPhase alone: out = W*H interleaved complex M e^{i phase}. */
void imro_random_phase_f32(const float *mod, float *out, unsigned W, unsigned H, unsigned seed);

#ifdef __cplusplus
}
#endif
#endif
