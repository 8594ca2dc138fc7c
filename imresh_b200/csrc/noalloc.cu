// Shrink-wrap reconstruction that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while its memory is
// owned by a fixed arena or a framework allocator, real-time loops that must
// not take the driver's allocation locks, and processes whose device memory
// is fully reserved up front.  imr_shrink_wrap_noalloc serves them: the
// caller passes the modulus and the output buffer, and everything else the
// reconstruction needs (a copy of the modulus and its column tiles, iterate,
// g_prev, mask, blur buffers, FFT twiddles, Gaussian weights, reduction
// partials, job state) lives in one file-scope device array,
// g_noalloc_scratch, of kNoAllocScratchBytes.  Every GPU that loads the
// library holds that array until the process exits.  Because the modulus is
// copied in first, the caller may pass one buffer as both modulus and output,
// as the reference's cudaShrinkWrap works in place.
//
// The array's name in host code is a host-side stand-in, not a device
// address, so the first call on each device (with that device current) looks
// up the real address with cudaGetSymbolAddress; that first call also sets
// kernel attributes and must come before any stream capture.  All calls share
// the array and it keeps the previous call's contents: the job state, the
// error log and the mask are cleared at the start of each call, everything
// else is written before it is read.  Calls whose work overlaps on the GPU
// (different streams, or host threads without ordering) race on the array;
// issue them on one stream, one after another.  imr_shrink_wrap_noalloc_stats
// reads the last call's cycle count, errors and device-wait status back.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "imresh_b200.h"
#include "kernels.cuh"
#include "engine_host.hpp"

namespace imr {

constexpr size_t kNoAllocMaxPixels = 512 * 512;
constexpr unsigned kNoAllocMaxCycles = 1024;
constexpr size_t kNoAllocTableBytes = 1u << 20;   // state, errors, weights, taps, twiddles, partials, lists
// per pixel: X, g_prev (8 + 8), the modulus copy and its column tiles (4 + 4;
// the tiles round the width up to whole 16-column tiles: at most 15 columns
// of the largest side more), the blur buffers (4 + 4), the mask (1)
constexpr size_t kNoAllocTileSlack = 15 * 4096 * 4;
constexpr size_t kNoAllocScratchBytes = kNoAllocMaxPixels * 33 + kNoAllocTileSlack + 8 * 256 + kNoAllocTableBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Fixed places at the start of the array (the same for every image size), so
// that imr_shrink_wrap_noalloc_stats finds the last call's state.
constexpr size_t kNaState = 0;                                             // JobState
constexpr size_t kNaErrors = 256;                                          // float[kNoAllocMaxCycles + 1]
constexpr size_t kNaJob = kNaErrors + ((kNoAllocMaxCycles + 1) * 4 + 255) / 256 * 256;   // JobDev
constexpr size_t kNaLists = kNaJob + (sizeof(JobDev) + 255) / 256 * 256;  // WorkList[3]
constexpr size_t kNaVar = kNaLists + 256;                                 // everything sized by the call

static std::mutex g_na_mu;
static void *g_na_ptr[64];        // device address of g_noalloc_scratch per device
static int g_na_cycles[64];       // nCycles of the last call on each device

static int noalloc_setup(int dev, char **out)
{
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (dev < 0 || dev >= 64) return IMR_ERR_INVALID_VALUE;
    if (!g_na_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
            return IMR_ERR_CUDA;
        }
        g_na_ptr[dev] = p;
    }
    *out = (char *)g_na_ptr[dev];
    return IMR_SUCCESS;
}

// host staging for the tables (per host thread; no heap allocation per call)
struct NoAllocStage {
    float2 tw_row[4096], tw_col[4096];
    float weights[(kNoAllocMaxCycles + 1) * kTapStride];
    int taps[kNoAllocMaxCycles + 1];
    JobDev J;
    WorkList lists[3];
};
static thread_local NoAllocStage t_stage;

// the radix schedule of factor_len(), without its std::vector
static bool radices(int n, FftPlanDev &p, const float2 *tw)
{
    if (n < 1 || n > (int)kMaxSide || (n > kMaxRuntimeSide && n != 3072 && n != 4096)) return false;
    const RadixList L = radix_list(n);
    if (L.n < 0) return false;
    memset(&p, 0, sizeof(p));
    p.n = n;
    p.nrad = L.n;
    for (int i = 0; i < L.n; ++i) p.rad[i] = L.r[i];
    p.tw = tw;
    return true;
}

static void fill_twiddles(float2 *h, int n)
{
    for (int t = 0; t < n; ++t) {
        const double a = -2.0 * M_PI * (double)t / (double)n;
        h[t] = make_float2((float)cos(a), (float)sin(a));
    }
}

static bool ranges_overlap(const void *a, const void *b, size_t bytes)
{
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + bytes && y < x + bytes;
}

}  // namespace imr

using namespace imr;

#define CKN(call)                      \
    do {                               \
        cudaError_t e_ = (call);       \
        if (e_ != cudaSuccess) {       \
            set_error(#call, e_);      \
            return IMR_ERR_CUDA;       \
        }                              \
    } while (0)

extern "C" int imr_shrink_wrap_noalloc(const float *d_modulus, float *d_out, unsigned W, unsigned H,
                                       const imr_params *params, void *stream)
{
    if (!d_modulus || !d_out || W == 0 || H == 0) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: null buffer or zero size");
        return IMR_ERR_INVALID_VALUE;
    }
    imr_params p;
    resolve_params(params, p);
    if ((size_t)W * H > kNoAllocMaxPixels) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "imr_shrink_wrap_noalloc: %ux%u exceeds the static scratch (at most %zu pixels)", W, H,
                 kNoAllocMaxPixels);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    if (p.nCycles > kNoAllocMaxCycles) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: at most %u cycles", kNoAllocMaxCycles);
        return IMR_ERR_INVALID_VALUE;
    }
    // direct transforms only: Bluestein lengths need device tables that are
    // allocated per length
    if (radix_list((int)W).n < 0 || radix_list((int)H).n < 0) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "imr_shrink_wrap_noalloc: %ux%u: sides must be 2^a 3^b 5^c 7^d (no Bluestein lengths)", W, H);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    const size_t N = (size_t)W * H;
    int dev = 0;
    CKN(cudaGetDevice(&dev));
    char *base = nullptr;
    int rc = noalloc_setup(dev, &base);
    if (rc) return rc;
    if ((rc = ensure_kernel_attributes())) return rc;

    // ---- job description (host side, no allocation)
    NoAllocStage &S = t_stage;
    JobDev &J = S.J;
    memset(&J, 0, sizeof(J));
    J.W = (int)W;
    J.H = (int)H;
    const RowKernels rk = row_kernels(J.W);
    const ColKernels ck = col_kernels(J.H);
    J.rpc = rk.nb < J.H ? rk.nb : J.H;
    J.cpc = ck.nb < J.W ? ck.nb : J.W;
    const bool p_rows = rk.p_hio != nullptr;
    bool p_cols = ck.p_col != nullptr && J.W % 4 == 0 && J.W >= ck.p_nb;
    const int tile_w = p_cols ? ck.p_nb : 1;
    const size_t mt_bytes = (p_cols && ck.p_mt) ? (size_t)((J.W + tile_w - 1) / tile_w) * tile_w * J.H * 4 : 0;

    // ---- layout inside the scratch array: fixed tables first, then the images
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    JobState *d_st = (JobState *)(base + kNaState);
    float *d_err = (float *)(base + kNaErrors);
    JobDev *d_j = (JobDev *)(base + kNaJob);
    WorkList *d_l = (WorkList *)(base + kNaLists);
    size_t off = kNaVar;
    float2 *d_twr = (float2 *)(base + off); off += al(sizeof(float2) * W);
    float2 *d_twc = (float2 *)(base + off); off += al(sizeof(float2) * H);
    float *d_w = (float *)(base + off);     off += al(sizeof(float) * (p.nCycles + 1) * kTapStride);
    int *d_taps = (int *)(base + off);      off += al(sizeof(int) * (p.nCycles + 1));
    const int n_row_tiles = (J.H + J.rpc - 1) / J.rpc;
    double *d_ep = (double *)(base + off);  off += al(sizeof(double) * 2 * n_row_tiles);
    char *X = base + off;    off += al(N * 8);
    char *G = base + off;    off += al(N * 8);
    char *M = base + off;    off += al(N * 4);
    char *Mt = base + off;   off += al(mt_bytes);
    char *hb = base + off;   off += al(N * 4);
    char *vb = base + off;   off += al(N * 4);
    char *mask = base + off; off += al(N);
    if (off > kNoAllocScratchBytes) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "imr_shrink_wrap_noalloc: %ux%u with %u cycles needs %zu bytes of the %zu-byte static scratch", W, H,
                 p.nCycles, off, kNoAllocScratchBytes);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    // the caller's buffers must not lie inside the library's own array
    if (ranges_overlap(d_modulus, base, kNoAllocScratchBytes) || ranges_overlap(d_out, base, kNoAllocScratchBytes)) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: buffer inside the library's scratch");
        return IMR_ERR_INVALID_VALUE;
    }

    if (!radices((int)W, J.prow, d_twr) || !radices((int)H, J.pcol, d_twc)) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: %ux%u: unsupported side", W, H);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    float sigma = p.sigma0;
    for (unsigned c = 0; c <= p.nCycles; ++c) {
        float *w = S.weights + (size_t)c * kTapStride;
        memset(w, 0, sizeof(float) * kTapStride);
        const int K = gaussian_weights((double)sigma, w, kMaxTaps);
        if (K > kMaxTaps) {
            snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: sigma %g needs %d taps (at most %d)",
                     (double)sigma, K, kMaxTaps);
            return IMR_ERR_INVALID_VALUE;
        }
        S.taps[c] = K;
        sigma = fmaxf(1.5f, (1.0f - p.sigmaChange) * sigma);
    }
    fill_twiddles(S.tw_row, (int)W);
    fill_twiddles(S.tw_col, (int)H);
    J.X = (float2 *)X;
    J.G = (float2 *)G;
    J.M = (const float *)M;   // a copy: d_modulus and d_out may be one buffer
    J.Mt = nullptr;
    J.hb = (float *)hb;
    J.vb = (float *)vb;
    J.out = d_out;
    J.mask = (uint8_t *)mask;
    J.weights = d_w;
    J.ntaps = d_taps;
    J.err_part = d_ep;
    J.errors = d_err;
    J.st = d_st;
    if (p_cols) {
        J.cpc = ck.p_nb;
        p_cols = encode_tensor_map(&J.tmX, J.X, J.W, J.H, 8, ck.p_nb, ck.p_box_rows) &&
                 (!ck.p_tma_m || encode_tensor_map(&J.tmM, J.M, J.W, J.H, 4, ck.p_nb, ck.p_box_rows));
        if (!p_cols) J.cpc = ck.nb < J.W ? ck.nb : J.W;
        else if (ck.p_mt) J.Mt = (const float *)Mt;
    }
    J.use_tma_cols = p_cols ? 1 : 0;
    J.n_row_tiles = n_row_tiles;
    J.n_col_tiles = (J.W + J.cpc - 1) / J.cpc;
    J.vb_tiles_x = (J.W + kVbTileX - 1) / kVbTileX;
    J.n_vb_tiles = J.vb_tiles_x * ((J.H + kVbTileY - 1) / kVbTileY);
    J.beta = p.hioBeta;
    J.cut_auto = p.intensityCutOffAutoCorel;
    J.cut = p.intensityCutOff;
    J.target = p.targetError;
    J.n_cycles = (int)p.nCycles;
    J.n_hio = (int)p.nHioCycles;
    S.lists[0] = WorkList{nullptr, J.n_row_tiles};
    S.lists[1] = WorkList{nullptr, J.n_col_tiles};
    S.lists[2] = WorkList{nullptr, J.n_vb_tiles};
    size_t smem_row, smem_fin;
    if (rk.smem) {
        smem_row = smem_fin = (size_t)rk.smem;
    } else {
        smem_row = (size_t)rk.nb * J.W * sizeof(float2);
        smem_fin = smem_row + (size_t)rk.nb * J.W * sizeof(float);
    }
    const size_t smem_col = ck.smem ? (size_t)ck.smem : (size_t)ck.nb * J.H * sizeof(float2);

    // ---- upload tables, copy the modulus, clear what must start at zero (stream-ordered)
    cudaStream_t s = (cudaStream_t)stream;
    CKN(cudaMemcpyAsync(d_twr, S.tw_row, sizeof(float2) * W, cudaMemcpyHostToDevice, s));
    CKN(cudaMemcpyAsync(d_twc, S.tw_col, sizeof(float2) * H, cudaMemcpyHostToDevice, s));
    CKN(cudaMemcpyAsync(d_w, S.weights, sizeof(float) * (p.nCycles + 1) * kTapStride, cudaMemcpyHostToDevice, s));
    CKN(cudaMemcpyAsync(d_taps, S.taps, sizeof(int) * (p.nCycles + 1), cudaMemcpyHostToDevice, s));
    CKN(cudaMemcpyAsync(d_j, &J, sizeof(JobDev), cudaMemcpyHostToDevice, s));
    CKN(cudaMemcpyAsync(d_l, S.lists, sizeof(S.lists), cudaMemcpyHostToDevice, s));
    CKN(cudaMemsetAsync(d_st, 0, sizeof(JobState), s));
    CKN(cudaMemsetAsync(d_err, 0, sizeof(float) * (kNoAllocMaxCycles + 1), s));
    CKN(cudaMemsetAsync(mask, 0, N, s));
    CKN(cudaMemcpyAsync(M, d_modulus, N * 4, cudaMemcpyDeviceToDevice, s));
    if ((rc = job_modulus_tiles(J, s))) return rc;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        g_na_cycles[dev] = (int)p.nCycles;
    }

    // ---- the reconstruction: column init, cycles, final error pass
    const int g_row_first = p_rows ? persistent_grid((const void *)rk.p_hio_first, rk.threads, rk.p_smem_first,
                                                     J.n_row_tiles) : 0;
    const int g_row = p_rows ? persistent_grid((const void *)rk.p_hio, rk.threads, rk.p_smem, J.n_row_tiles) : 0;
    const int g_col = p_cols ? persistent_grid((const void *)ck.p_col, ck.p_threads, ck.p_smem, J.n_col_tiles) : 0;
    ck.init<<<J.n_col_tiles, ck.threads, smem_col, s>>>(d_j, d_l + 1);
    for (int c = 0; c <= J.n_cycles; ++c) {
        if (int rc = launch_finish(rk, J.n_row_tiles, smem_fin, s, d_j, d_l, nullptr)) return rc;
        k_vblur<<<J.n_vb_tiles, kVbThreads, 0, s>>>(d_j, d_l + 2);
        if (c == J.n_cycles) break;   // final pass: error and stop test only
        for (int i = 0; i < J.n_hio; ++i) {
            if (p_rows) {
                if (i == 0) rk.p_hio_first<<<g_row_first, rk.threads, rk.p_smem_first, s>>>(d_j, d_l);
                else rk.p_hio<<<g_row, rk.threads, rk.p_smem, s>>>(d_j, d_l);
            } else {
                (i == 0 ? rk.hio_first : rk.hio)<<<J.n_row_tiles, rk.threads, smem_row, s>>>(d_j, d_l);
            }
            if (p_cols) ck.p_col<<<g_col, ck.p_threads, ck.p_smem, s>>>(d_j, d_l + 1);
            else ck.col<<<J.n_col_tiles, ck.threads, smem_col, s>>>(d_j, d_l + 1);
        }
    }
    CKN(cudaGetLastError());
    return IMR_SUCCESS;
}

extern "C" int imr_shrink_wrap_noalloc_stats(void *stream, int *cycles_done, float *errors, int cap)
{
    int dev = 0;
    CKN(cudaGetDevice(&dev));
    char *base = nullptr;
    int rc = noalloc_setup(dev, &base);
    if (rc) return rc;
    int n_cycles;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        n_cycles = g_na_cycles[dev];
    }
    CKN(cudaStreamSynchronize((cudaStream_t)stream));
    JobState st;
    CKN(cudaMemcpy(&st, base + kNaState, sizeof(JobState), cudaMemcpyDeviceToHost));
    if (cycles_done) *cycles_done = st.cycles_done;
    if (errors && cap > 0) {
        const int n = cap < n_cycles ? cap : n_cycles;
        if (n > 0) CKN(cudaMemcpy(errors, base + kNaErrors, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    if (st.err) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_shrink_wrap_noalloc: a device-side copy wait timed out");
        return IMR_ERR_DEVICE_TIMEOUT;
    }
    return IMR_SUCCESS;
}
