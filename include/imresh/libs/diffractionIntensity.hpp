/*
 * Drop-in declaration of the reference's forward model (the cuFFT variant,
 * src/imresh/libs/diffractionIntensity.hpp): replaces the real image in
 * rpIoData (HOST buffer, width*height floats) by the modulus |FFT2| of it,
 * unnormalised, zero frequency at index 0 -- the input cudaShrinkWrap
 * expects.  Implemented by libimresh_b200.so on its own FFT; synchronous.
 */
#pragma once
#include <cuda_runtime_api.h>

namespace imresh
{
namespace libs
{
    void diffractionIntensity
    (
        float * const      rpIoData,
        unsigned int const rImageWidth,
        unsigned int const rImageHeight,
        cudaStream_t const rStream = cudaStream_t(0),
        bool               rAsync  = false
    );
} // namespace libs
} // namespace imresh
