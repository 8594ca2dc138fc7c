/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * Float and double instances of the project-written FFT in fft_impl.h, with a
 * small C API used by the FFTW shim (fftw_shim.c), by the C restatement of the
 * reference CPU path (shrinkwrap_oracle.c) and by the tests.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "imro.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846264338327950288
#endif

#define R float
#define SUF f32
#include "fft_impl.h"
#undef R
#undef SUF

#define R double
#define SUF f64
#include "fft_impl.h"
#undef R
#undef SUF

void imro_c2c_2d_f32(float *d, int H, int W, int s) { imro_fft2d_f32(d, H, W, s); }
void imro_c2c_2d_f64(double *d, int H, int W, int s) { imro_fft2d_f64(d, H, W, s); }
void imro_c2c_rows_f32(float *d, int n, int m, int s) { imro_fft_rows_f32(d, n, m, s); }
void imro_c2c_rows_f64(double *d, int n, int m, int s) { imro_fft_rows_f64(d, n, m, s); }
void imro_c2c_cols_f32(float *d, int H, int W, int s) { imro_fft_cols_f32(d, H, W, s); }
void imro_c2c_cols_f64(double *d, int H, int W, int s) { imro_fft_cols_f64(d, H, W, s); }
