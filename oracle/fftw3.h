/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * Declarations-only stand-in for the six FFTW3 entry points the reference's
 * CPU sources use (src/imresh/algorithms/shrinkWrap.cpp:146-155,164,279,301,
 * 354-357; src/imresh/libs/diffractionIntensity.cpp:61-68;
 * src/imresh/libs/hybridInputOutput.cpp:172-183).  FFTW itself is not
 * installed on this image; fftw_shim.c implements these names on the
 * project-written FFT so the reference's CPU translation units compile
 * unmodified into oracle/_ref/libimresh_ref.so.  Types and sign constants
 * follow FFTW3's published API.
 */
#ifndef IMRO_FFTW3_SHIM_H
#define IMRO_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct imro_fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft(int rank, const int *n, fftwf_complex *in,
                          fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in,
                             fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
fftwf_complex *fftwf_alloc_complex(size_t n);
void fftwf_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
