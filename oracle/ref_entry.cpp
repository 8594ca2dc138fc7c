/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * C-linkage entry points into the reference's own CPU implementation,
 * compiled unmodified from its sources (see oracle/Makefile) into
 * oracle/_ref/libimresh_ref.so, so that Python tests and the CPU-baseline leg
 * of bench.py can call it through ctypes.  Each wrapper forwards to exactly
 * one reference function:
 *   imro_ref_shrinkwrap      -> imresh::algorithms::shrinkWrap
 *                               (src/imresh/algorithms/shrinkWrap.cpp:111-361)
 *   imro_ref_blur{,_h,_v}    -> imresh::libs::gaussianBlur{,Horizontal,Vertical}<float>
 *                               (src/imresh/libs/gaussian.cpp:180-197, 559-749)
 *   imro_ref_weights         -> imresh::libs::calcGaussianKernel<float>
 *                               (src/imresh/libs/calcGaussianKernel.cpp:42-91)
 *   imro_ref_vector_max      -> imresh::algorithms::vectorMax<float>
 *                               (src/imresh/algorithms/vectorReduce.cpp:73-87)
 *   imro_ref_hio_error       -> imresh::libs::calculateHioError<fftwf_complex,float>
 *                               (src/imresh/libs/hybridInputOutput.cpp:67-103)
 *   imro_ref_hio             -> imresh::libs::hybridInputOutput
 *                               (src/imresh/libs/hybridInputOutput.cpp:193-306);
 *                               rSize = {H, W}: the FFTW plan's slow then fast
 *                               dimension (cpp:219-222); rnCores = 0 leaves the
 *                               process's OpenMP thread count alone
 */
#include <fftw3.h>
#include "algorithms/shrinkWrap.hpp"
#include "algorithms/vectorReduce.hpp"
#include "libs/gaussian.hpp"
#include "libs/calcGaussianKernel.hpp"
#include "libs/hybridInputOutput.hpp"

extern "C" {

int imro_ref_shrinkwrap(float *io, unsigned W, unsigned H, unsigned nCycles,
                        float targetError, float beta, float cutAuto, float cut,
                        float sigma0, float sigmaChange, unsigned nHio)
{
    return imresh::algorithms::shrinkWrap(io, W, H, nCycles, targetError, beta,
                                          cutAuto, cut, sigma0, sigmaChange, nHio);
}

void imro_ref_blur(float *d, unsigned W, unsigned H, double sigma)
{
    imresh::libs::gaussianBlur<float>(d, W, H, sigma);
}

void imro_ref_blur_h(float *d, unsigned W, unsigned H, double sigma)
{
    imresh::libs::gaussianBlurHorizontal<float>(d, W, H, sigma);
}

void imro_ref_blur_v(float *d, unsigned W, unsigned H, double sigma)
{
    imresh::libs::gaussianBlurVertical<float>(d, W, H, sigma);
}

int imro_ref_weights(double sigma, float *w, unsigned cap)
{
    return imresh::libs::calcGaussianKernel<float>(sigma, w, cap);
}

float imro_ref_vector_max(const float *d, unsigned n)
{
    return imresh::algorithms::vectorMax<float>(d, n);
}

float imro_ref_hio_error(const float *gp, const float *mask, unsigned n,
                         float *total, float *count)
{
    return imresh::libs::calculateHioError<fftwf_complex, float>(
        (const fftwf_complex *)gp, mask, n, false, total, count);
}

int imro_ref_hio(float *io, const unsigned char *mask, unsigned W, unsigned H, unsigned nCycles,
                 float targetError, float beta)
{
    return imresh::libs::hybridInputOutput(io, mask, std::vector<unsigned>{H, W}, nCycles,
                                           targetError, beta, 0);
}

}
