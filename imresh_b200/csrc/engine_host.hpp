// Host-side helpers shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "imresh_b200.h"
#include "engine.cuh"

namespace imr {

constexpr unsigned kMaxSide = 4096;
constexpr int kMaxRuntimeSide = 2048;

void set_error(const char *what, cudaError_t e);
bool factor_len(int n, std::vector<int> &rad);
int make_fft_plan(int n, FftPlanDev &p);
int gaussian_weights(double sigma, float *w, int cap);
int ensure_kernel_attributes();
void resolve_params(const imr_params *in, imr_params &out);
int build_weight_table(const imr_params &p, std::vector<float> &w, std::vector<int> &taps);

// Kernels and launch shape of the row passes for one row length.
struct RowKernels {
    void (*hio_first)(const JobDev *, const WorkItem *);
    void (*hio)(const JobDev *, const WorkItem *);
    void (*finish)(const JobDev *, const WorkItem *, float2 *);
    void (*fft_fwd)(float2 *, FftPlanDev, int, int);
    void (*fft_inv)(float2 *, FftPlanDev, int, int);
    int nb;        // rows per CTA
    int threads;
};
// Kernels and launch shape of the column passes for one column length.
struct ColKernels {
    void (*col)(const JobDev *, const WorkItem *);
    void (*init)(const JobDev *, const WorkItem *);
    void (*fft_fwd)(float2 *, FftPlanDev, int, int);
    void (*fft_inv)(float2 *, FftPlanDev, int, int);
    int nb;        // columns per CTA
    int threads;
};
RowKernels row_kernels(int N);
ColKernels col_kernels(int N);
int plan_cache_acquire(unsigned W, unsigned H, const imr_params *params, imr_plan **out);
void plan_cache_release(imr_plan *P);

}  // namespace imr
