/*
 * Drop-in declaration of imresh::algorithms::cuda::cudaShrinkWrap, same
 * signature and defaults as the reference
 * (src/imresh/algorithms/cuda/cudaShrinkWrap.hpp:114-130), implemented by
 * libimresh_b200.so over its C ABI (include/imresh_b200.h).
 *
 * rIoData: HOST buffer of rImageWidth*rImageHeight floats, the Fourier
 * modulus on entry, Re(g') of the reconstruction on return.  Synchronous.
 * Arguments <= 0 select the reference's CUDA defaults (20 cycles,
 * targetError 1e-5, beta 0.9, autocorrelation cutoff 0.02, cutoff 0.2,
 * sigma0 3, sigma change 0.01, 20 HIO iterations).  rnBlocks / rnThreads are
 * accepted and ignored (the engine picks its own launch shapes).
 * Returns 0 on success, else an imr_status code; unlike the reference it
 * never calls exit() on a CUDA error.
 */
#pragma once
#include <cuda_runtime_api.h>

namespace imresh
{
namespace algorithms
{
namespace cuda
{
    int cudaShrinkWrap
    (
        float * const       rIoData,
        unsigned int const  rImageWidth,
        unsigned int const  rImageHeight,
        cudaStream_t const  rStream                     = 0,
        unsigned int        rnBlocks                    = 256,
        unsigned int        rnThreads                   = 256,
        unsigned int        rnCycles                    = 0,
        float               rTargetError                = 0,
        float               rHioBeta                    = 0,
        float               rIntensityCutOffAutoCorel   = 0,
        float               rIntensityCutOff            = 0,
        float               rSigma0                     = 0,
        float               rSigmaChange                = 0,
        unsigned int        rnHioCycles                 = 0
    );
} // namespace cuda
} // namespace algorithms
} // namespace imresh
