// Host-side helpers shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "imresh_b200.h"
#include "engine.cuh"

namespace imr {

constexpr unsigned kMaxSide = 4096;
constexpr int kMaxRuntimeSide = 2048;

extern thread_local char g_last_error[256];   // imr_last_error() text
void set_error(const char *what, cudaError_t e);
bool factor_len(int n, std::vector<int> &rad);
bool length_supported(int n);
int bluestein_m(int n);
int make_fft_plan(int n, FftPlanDev &p);
int gaussian_weights(double sigma, float *w, int cap);
int ensure_kernel_attributes();
void resolve_params(const imr_params *in, imr_params &out);
int build_weight_table(const imr_params &p, std::vector<float> &w, std::vector<int> &taps);

// Kernels and launch shape of the row passes for one row length.
struct RowKernels {
    void (*hio_first)(const JobDev *, const WorkList *);
    void (*hio)(const JobDev *, const WorkList *);
    void (*finish)(const JobDev *, const WorkList *, float2 *);
    void (*fft_fwd)(float2 *, FftPlanDev, int, int);
    void (*fft_inv)(float2 *, FftPlanDev, int, int);
    int nb;        // rows per CTA
    int threads;
    int smem;      // dynamic shared memory of the FFT kernels (bytes); 0: nb*N*8
    // pipelined (persistent, TMA) row passes; null when the length has none
    void (*p_hio_first)(const JobDev *, const WorkList *);
    void (*p_hio)(const JobDev *, const WorkList *);
    int p_smem_first, p_smem;
    int bs_m;      // Bluestein work length (0: direct transform)
    // fixed-support HIO row passes (libs::hybridInputOutput): per-tile kernel
    // and, where the length has one, the pipelined kernel (shared memory p_smem)
    void (*hio_fix)(const JobDev *, const WorkList *);
    void (*p_hio_fix)(const JobDev *, const WorkList *);
    // pipelined once-per-cycle pass (g', out, error sums, row blur) or null
    void (*p_finish)(const JobDev *, const WorkList *, float2 *);
    int p_smem_fin;
};
// Kernels and launch shape of the column passes for one column length.
struct ColKernels {
    void (*col)(const JobDev *, const WorkList *);
    void (*init)(const JobDev *, const WorkList *);
    void (*fft_fwd)(float2 *, FftPlanDev, int, int);
    void (*fft_inv)(float2 *, FftPlanDev, int, int);
    int nb;        // columns per CTA
    int threads;
    int smem;      // dynamic shared memory (bytes); 0: nb*N*8
    void (*p_col)(const JobDev *, const WorkList *);   // pipelined column pass or null
    int p_smem;
    int p_box_rows;  // rows per 2D TMA box
    int p_tma_m;     // 1: the modulus tile also arrives by TMA
    int p_threads;   // threads of the pipelined column pass
    int bs_m;        // Bluestein work length (0: direct transform)
    int p_nb;        // columns per tile of the pipelined pass (its TMA box width)
    int p_mt;        // 1: the pipelined pass reads the modulus from JobDev::Mt when set
    // split-precision tensor-core column passes ([0] BF16 hi+lo, [1] FP16 hi+lo;
    // same launch shape as p_col) and their stand-alone forward / inverse
    // column transforms; null where the length has none
    void (*p_col_tc[2])(const JobDev *, const WorkList *);
    void (*fft_tc[2][2])(const JobDev *, const WorkList *);   // [precision][0 forward, 1 inverse]
    int p_smem_tc;   // their dynamic shared memory
    void (*p_col_split)(const JobDev *, const WorkList *);   // p_col running WorkList::n_split
                                                              // tiles as half tiles (JobDev::tmXh), or null
};
RowKernels row_kernels(int N);
ColKernels col_kernels(int N);
// Plain 2D transform passes (axes: 1 rows, 2 columns, 3 both).
int fft_passes(float2 *d, int W, int H, int sign, int axes, const FftPlanDev &pr, const FftPlanDev &pc,
               cudaStream_t s);
// Persistent grid size for a pipelined kernel (CTAs per SM x SMs, <= items).
int persistent_grid(const void *kernel, int threads, int smem, int items);
// Launch the once-per-cycle row pass over `items` row tiles: the pipelined
// persistent kernel where the row length has one, else one CTA per tile.
// grid_pct: the persistent grid at this percentage of the occupancy limit.
int launch_finish(const RowKernels &rk, int items, size_t smem_fin, cudaStream_t s, const JobDev *dj,
                  const WorkList *L, float2 *dbg, int grid_pct = 100);
// Persistent grid scaled to grid_pct % of the occupancy limit (at least 1 CTA, at most `items`).
int scaled_grid(const void *kernel, int threads, int smem, int items, int grid_pct);
// WorkList::n_split of a persistent column launch of n_tiles tiles with at
// most g_max CTAs resident (its grid: min(g_max, n_tiles + n_split)): every
// tile when their halves fit the resident CTAs, else none.
int col_split(int n_tiles, int g_max);
// 2D tensor map over a row-major [H][W] array of `elem`-byte elements with a
// (box_w, box_h) box; returns false when the shape cannot be described.
bool encode_tensor_map(CUtensorMap *map, const void *base, int W, int H, int elem, int box_w, int box_h);

// Host description of one reconstruction's device layout and kernels.
struct JobShape {
    RowKernels rk{};
    ColKernels ck{};
    bool p_rows = false, p_cols = false;
    bool p_half = false;   // JobDev::tmXh encoded: the column pass may run half tiles
    size_t smem_row = 0, smem_fin = 0, smem_col = 0;
    size_t bytes = 0;   // arena bytes (JobState not included)
    size_t oX = 0, oG = 0, oM = 0, oMt = 0, oHB = 0, oVB = 0, oOut = 0, oMask = 0, oW = 0, oT = 0, oEP = 0, oErr = 0;
    std::vector<float> wt;
    std::vector<int> taps;
};
int job_prepare(unsigned W, unsigned H, const imr_params &p, JobDev &J, JobShape &S);
void job_bind(JobDev &J, JobShape &S, char *arena, JobState *st);
int job_upload(const JobDev &J, const JobShape &S, char *arena, JobDev *dj, cudaStream_t s);
// Fill JobDev::Mt from the modulus (stream-ordered; nothing to do when Mt is
// null).  Called whenever the modulus has been (re)written.
int job_modulus_tiles(const JobDev &J, cudaStream_t s);
int plan_cache_acquire(unsigned W, unsigned H, const imr_params *params, imr_plan **out);
void plan_cache_release(imr_plan *P);

}  // namespace imr
