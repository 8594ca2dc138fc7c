/*
 * Drop-in declarations of the reference's device reductions on the
 * shrink-wrap path (src/imresh/algorithms/cuda/cudaVectorReduce.hpp):
 *   cudaVectorMax<float>   (hpp:88-94, cu:229-239)
 *   cudaCalculateHioError  (hpp:160-170, cu:357-403) for complex64 data with a
 *                          float or 8-bit mask (the reference instantiates
 *                          <cufftComplex, float>; its test also feeds byte masks)
 * Device buffers in, host results out; synchronous on rStream.  Implemented
 * over the C ABI of libimresh_b200.so (imr_vector_max, imr_calculate_hio_error).
 * On a library error the result is NaN and the message goes to stderr (the
 * reference exits the process instead).
 */
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <type_traits>
#include <cuda_runtime_api.h>
#include "imresh_b200.h"

namespace imresh
{
namespace algorithms
{
namespace cuda
{
    template< class T_PREC >
    T_PREC cudaVectorMax
    (
        T_PREC const * const rdpData,
        unsigned int const rnElements,
        cudaStream_t rStream = 0
    )
    {
        static_assert( std::is_same< T_PREC, float >::value, "cudaVectorMax: float data only" );
        float m = 0;
        int const rc = imr_vector_max( rdpData, rnElements, &m, (void *) rStream );
        if ( rc != IMR_SUCCESS )
        {
            fprintf( stderr, "imresh_b200 cudaVectorMax: %s\n", imr_status_string( rc ) );
            return std::numeric_limits< float >::quiet_NaN();
        }
        return m;
    }

    template< class T_COMPLEX, class T_MASK >
    float cudaCalculateHioError
    (
        T_COMPLEX const * const rdpData,
        T_MASK const * const rdpIsMasked,
        unsigned int const rnElements,
        bool const rInvertMask = false,
        cudaStream_t rStream = 0,
        float * const rpTotalError = NULL,
        float * const rpnMaskedPixels = NULL
    )
    {
        static_assert( sizeof( T_COMPLEX ) == 2 * sizeof( float ), "complex64 data expected" );
        static_assert( std::is_same< T_MASK, float >::value || sizeof( T_MASK ) == 1,
                       "float or 8-bit mask expected" );
        int const kind = std::is_same< T_MASK, float >::value ? IMR_MASK_F32 : IMR_MASK_U8;
        float total = 0, count = 0, error = 0;
        int const rc = imr_calculate_hio_error( rdpData, rdpIsMasked, kind, rnElements,
                                                rInvertMask ? 1 : 0, &total, &count, &error,
                                                (void *) rStream );
        if ( rc != IMR_SUCCESS )
        {
            fprintf( stderr, "imresh_b200 cudaCalculateHioError: %s\n", imr_status_string( rc ) );
            return std::numeric_limits< float >::quiet_NaN();
        }
        if ( rpTotalError    != NULL ) *rpTotalError    = total;
        if ( rpnMaskedPixels != NULL ) *rpnMaskedPixels = count;
        return error;
    }
} // namespace cuda
} // namespace algorithms
} // namespace imresh
