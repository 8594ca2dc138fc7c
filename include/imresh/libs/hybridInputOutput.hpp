/*
 * Drop-in declarations of the reference's fixed-support HIO header
 * (src/imresh/libs/hybridInputOutput.hpp).
 *
 * hybridInputOutput (hpp:81-90, cpp:193-306): rIoData is a HOST buffer of
 * rSize[0]*rSize[1] floats, the Fourier modulus in and Re(g') out; rSize[0]
 * is the slow (row) dimension and rSize[1] the contiguous one, as the
 * reference's FFTW plan takes them.  rMask: 1 = outside the support.  Runs on
 * the GPU (libimresh_b200.so: random initial phase from srand(2623091912)
 * drawn on the device, fused HIO passes); synchronous.  Returns 0 on success,
 * 1 for a wrong dimension count or a NULL buffer (as the reference), else an
 * imr_status code.  rnCores is accepted and ignored.
 *
 * calculateHioError (hpp:59-79, cpp:67-103): the CPU error of g' against a
 * mask in HOST memory, sqrt(sum m*|g'|) / sum m, m = mask or 1 - mask.
 */
#pragma once
#include <climits>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace imresh
{
namespace libs
{
    template< class T_COMPLEX, class T_MASK_ELEMENT >
    float calculateHioError
    (
        T_COMPLEX      const * const __restrict__ gPrime,
        T_MASK_ELEMENT const * const __restrict__ rIsMasked,
        unsigned int const nElements,
        bool const rInvertMask = false,
        float * const __restrict__ rpTotalError    = NULL,
        float * const __restrict__ rpnMaskedPixels = NULL
    )
    {
        float total = 0, count = 0;
        for ( unsigned int i = 0; i < nElements; ++i )
        {
            float const w = rInvertMask ? 1 - (float) rIsMasked[i] : (float) rIsMasked[i];
            float const re = gPrime[i][0], im = gPrime[i][1];
            total += w * std::sqrt( re * re + im * im );
            count += w;
        }
        if ( rpTotalError    != NULL ) *rpTotalError    = total;
        if ( rpnMaskedPixels != NULL ) *rpnMaskedPixels = count;
        return std::sqrt( total ) / count;
    }

    int hybridInputOutput
    (
        float * const rIoData,
        uint8_t const * const rMask,
        std::vector<unsigned int> const rSize,
        unsigned int rnCycles = UINT_MAX,
        float rTargetError = 1e-6,
        float rBeta = 0.9,
        unsigned int rnCores = 0
    );
} // namespace libs
} // namespace imresh
