/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.
 *
 * The six FFTW3 float entry points (see fftw3.h) over the project-written
 * FFT.  Semantics kept from FFTW3's documented API: planning stores the
 * pointers and never touches the data (FFTW_ESTIMATE), transforms are
 * unnormalised, an out-of-place c2c execute leaves the input intact, and
 * rank-d arrays are row-major with the last dimension contiguous.  Like the
 * reference build (which never calls fftwf_init_threads) it runs on one
 * thread.
 */
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include "fftw3.h"
#include "imro.h"

struct imro_fftwf_plan_s {
    int rank;
    int n[3];
    float *in;
    float *out;
    int sign;
};

fftwf_plan fftwf_plan_dft(int rank, const int *n, fftwf_complex *in,
                          fftwf_complex *out, int sign, unsigned flags)
{
    (void)flags;
    if (rank < 1 || rank > 2) {
        fprintf(stderr, "fftw shim: rank %d not supported\n", rank);
        return NULL;
    }
    struct imro_fftwf_plan_s *p = (struct imro_fftwf_plan_s *)calloc(1, sizeof(*p));
    p->rank = rank;
    for (int i = 0; i < rank; ++i) p->n[i] = n[i];
    p->in = (float *)in;
    p->out = (float *)out;
    p->sign = sign;
    return p;
}

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in,
                             fftwf_complex *out, int sign, unsigned flags)
{
    int n[2] = {n0, n1};
    return fftwf_plan_dft(2, n, in, out, sign, flags);
}

void fftwf_execute(const fftwf_plan p)
{
    if (!p) return;
    size_t total = 1;
    for (int i = 0; i < p->rank; ++i) total *= (size_t)p->n[i];
    if (p->in != p->out) memcpy(p->out, p->in, sizeof(float) * 2 * total);
    if (p->rank == 1)
        imro_c2c_rows_f32(p->out, p->n[0], 1, p->sign);
    else
        imro_c2c_2d_f32(p->out, p->n[0], p->n[1], p->sign);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }

fftwf_complex *fftwf_alloc_complex(size_t n)
{
    void *ptr = NULL;
    if (posix_memalign(&ptr, 64, sizeof(fftwf_complex) * (n ? n : 1)) != 0) return NULL;
    return (fftwf_complex *)ptr;
}

void fftwf_free(void *p) { free(p); }
