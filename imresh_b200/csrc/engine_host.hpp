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
    int smem;      // dynamic shared memory of the FFT kernels (bytes); 0: nb*N*8
    // pipelined (persistent, TMA) row passes; null when the length has none
    void (*p_hio_first)(const JobDev *, const WorkItem *, int);
    void (*p_hio)(const JobDev *, const WorkItem *, int);
    int p_smem_first, p_smem;
};
// Kernels and launch shape of the column passes for one column length.
struct ColKernels {
    void (*col)(const JobDev *, const WorkItem *);
    void (*init)(const JobDev *, const WorkItem *);
    void (*fft_fwd)(float2 *, FftPlanDev, int, int);
    void (*fft_inv)(float2 *, FftPlanDev, int, int);
    int nb;        // columns per CTA
    int threads;
    int smem;      // dynamic shared memory (bytes); 0: nb*N*8
    void (*p_col)(const JobDev *, const WorkItem *, int);   // pipelined column pass or null
    int p_smem;
    int p_box_rows;  // rows per 2D TMA box
    int p_tma_m;     // 1: the modulus tile also arrives by TMA
};
RowKernels row_kernels(int N);
ColKernels col_kernels(int N);
// Persistent grid size for a pipelined kernel (CTAs per SM x SMs, <= items).
int persistent_grid(const void *kernel, int threads, int smem, int items);
// 2D tensor map over a row-major [H][W] array of `elem`-byte elements with a
// (box_w, box_h) box; returns false when the shape cannot be described.
bool encode_tensor_map(CUtensorMap *map, const void *base, int W, int H, int elem, int box_w, int box_h);
int plan_cache_acquire(unsigned W, unsigned H, const imr_params *params, imr_plan **out);
void plan_cache_release(imr_plan *P);

}  // namespace imr
