// Fixed-support hybrid input-output with a random initial phase -- the GPU
// counterpart of imresh::libs::hybridInputOutput
// (src/imresh/libs/hybridInputOutput.cpp:193-306, hpp:81-90) -- on the
// engine's fused passes, and the standalone HIO error of cudaCalculateHioError
// (src/imresh/algorithms/cuda/cudaVectorReduce.cu:357-403).
//
// One execution:
//   X = rand() field (k_rand_field) -> forward 2D FFT -> X = M e^{i arg X}
//   (k_random_phase) -> inverse column FFT; then for k = 0, 1, ...:
//     row pass    inverse row FFT -> g'_k; error terms and out = Re(g'_k);
//                 the job's last tile forms E_k and applies the stop tests;
//                 HIO update with the caller's mask; forward row FFT
//     column pass forward column FFT -> G*M/|G| (no |G| = 0 guard, as in
//                 cpp:281-289) -> inverse column FFT
//   until E_k < target (target > 0) or k == nCycles; the result is Re(g'_k).
// Iterations run as a captured graph of up to kHioChunk iterations, replayed;
// the host reads the device stop flag one replay behind, and the passes of a
// finished job return at once.
#include <cuda_runtime.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <vector>

#include "imresh_b200.h"
#include "kernels.cuh"
#include "engine_host.hpp"

namespace imr {

constexpr int kHioChunk = 16;
constexpr int kRandPowTable = 24;   // B^(2^j), j < 24: up to 2^24 chunks
constexpr int kHioMaxErrors = 1 << 16;

#define HCK(call)                                 \
    do {                                          \
        cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) {                  \
            set_error(#call, e_);                 \
            return IMR_ERR_CUDA;                  \
        }                                         \
    } while (0)

// ---------------------------------------------------------------- rand() stream
// glibc's srand/rand (TYPE_3 state, degree 31, separation 3): seeding fills
// r[0] = seed (0 acts as 1), r[i] = 16807 r[i-1] mod (2^31 - 1) for i < 31,
// r[31..33] = r[0..2]; afterwards r[i] = r[i-31] + r[i-3] mod 2^32 and rand()
// number k is r[k + 344] >> 1 (srand discards the first 310 sums).
using RandMat = std::array<uint32_t, kRandLag * kRandLag>;

static RandMat rand_mul(const RandMat &a, const RandMat &b)
{
    RandMat c{};
    for (int i = 0; i < kRandLag; ++i)
        for (int m = 0; m < kRandLag; ++m) {
            const uint32_t aim = a[i * kRandLag + m];
            if (!aim) continue;
            for (int j = 0; j < kRandLag; ++j) c[i * kRandLag + j] += aim * b[m * kRandLag + j];
        }
    return c;
}

// One step of the state (r[i-31..i-1]) -> (r[i-30..i]).
static RandMat rand_step()
{
    RandMat a{};
    for (int j = 0; j + 1 < kRandLag; ++j) a[j * kRandLag + j + 1] = 1u;
    a[(kRandLag - 1) * kRandLag + 0] = 1u;              // r[i-31]
    a[(kRandLag - 1) * kRandLag + kRandLag - 3] = 1u;   // r[i-3]
    return a;
}

static RandBase rand_base(unsigned seed)
{
    uint32_t r[344];
    const int32_t s0 = (int32_t)(seed ? seed : 1u);
    r[0] = (uint32_t)s0;
    for (int i = 1; i < 31; ++i) {
        long long v = (16807LL * (long long)(int32_t)r[i - 1]) % 2147483647LL;
        if (v < 0) v += 2147483647LL;
        r[i] = (uint32_t)v;
    }
    for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
    for (int i = 34; i < 344; ++i) r[i] = r[i - 31] + r[i - 3];
    RandBase b;
    for (int q = 0; q < kRandLag; ++q) b.s[q] = r[344 - kRandLag + q];
    return b;
}

static std::mutex g_rand_mu;
static std::map<int, uint32_t *> g_rand_pow;   // device -> kRandPowTable matrices

// Device table B^(2^j), B = (step matrix)^kRandChunk; seed independent.
static int rand_pow_table(uint32_t **out)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_rand_mu);
    auto it = g_rand_pow.find(dev);
    if (it != g_rand_pow.end()) {
        *out = it->second;
        return IMR_SUCCESS;
    }
    RandMat a = rand_step(), b{};
    for (int i = 0; i < kRandLag; ++i) b[i * kRandLag + i] = 1u;
    for (unsigned e = kRandChunk; e; e >>= 1) {   // b = a^kRandChunk
        if (e & 1u) b = rand_mul(b, a);
        a = rand_mul(a, a);
    }
    std::vector<uint32_t> tab((size_t)kRandPowTable * kRandLag * kRandLag);
    for (int j = 0; j < kRandPowTable; ++j) {
        memcpy(&tab[(size_t)j * kRandLag * kRandLag], b.data(), sizeof(uint32_t) * kRandLag * kRandLag);
        b = rand_mul(b, b);
    }
    uint32_t *d = nullptr;
    HCK(cudaMalloc((void **)&d, tab.size() * sizeof(uint32_t)));
    cudaError_t e = cudaMemcpy(d, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        set_error("rand table upload", e);
        return IMR_ERR_CUDA;
    }
    g_rand_pow[dev] = d;
    *out = d;
    return IMR_SUCCESS;
}

// X = rand() field of n numbers (seeded as srand(seed)).
static int launch_rand_field(float2 *X, long n, unsigned seed, cudaStream_t s)
{
    uint32_t *pow = nullptr;
    int rc = rand_pow_table(&pow);
    if (rc) return rc;
    const long chunks = (n + kRandChunk - 1) / kRandChunk;
    int n_pow = 0;
    while ((1L << n_pow) < chunks) ++n_pow;
    if (n_pow > kRandPowTable) return IMR_ERR_UNSUPPORTED_SIZE;
    const long blocks = (chunks + kRandThreads - 1) / kRandThreads;
    k_rand_field<<<(unsigned)blocks, kRandThreads, 0, s>>>(X, n, rand_base(seed), pow, n_pow);
    HCK(cudaGetLastError());
    return IMR_SUCCESS;
}

}  // namespace imr

using namespace imr;

// ==================================================================== plans
struct imr_hio_plan {
    int dev = 0;
    int W = 0, H = 0;
    JobDev hj{};
    JobDev *dj = nullptr;
    JobState *st = nullptr;
    void *arena = nullptr;
    WorkList *Lrow = nullptr, *Lcol = nullptr;
    RowKernels rk{};
    ColKernels ck{};
    bool p_rows = false, p_cols = false;
    int g_row = 0, g_col = 0;
    size_t smem_row = 0, smem_col = 0;
    int chunk = 0;   // iterations per graph replay
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int *h_stop = nullptr;   // pinned, one per replay parity
    cudaEvent_t ev[2] = {nullptr, nullptr};
};

static int hio_launch_iteration(imr_hio_plan *P, cudaStream_t s)
{
    const JobDev &J = P->hj;
    if (P->p_rows)
        P->rk.p_hio_fix<<<P->g_row, P->rk.threads, P->rk.p_smem, s>>>(P->dj, P->Lrow);
    else
        P->rk.hio_fix<<<J.n_row_tiles, P->rk.threads, P->smem_row, s>>>(P->dj, P->Lrow);
    if (P->p_cols)
        P->ck.p_col<<<P->g_col, P->ck.p_threads, P->ck.p_smem, s>>>(P->dj, P->Lcol);
    else
        P->ck.col<<<J.n_col_tiles, P->ck.threads, P->smem_col, s>>>(P->dj, P->Lcol);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("kernel launch", e);
        return IMR_ERR_CUDA;
    }
    return IMR_SUCCESS;
}

extern "C" {

int imr_hio_plan_destroy(imr_hio_plan *P)
{
    if (!P) return IMR_SUCCESS;
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->graph) cudaGraphDestroy(P->graph);
    for (auto &e : P->ev)
        if (e) cudaEventDestroy(e);
    if (P->h_stop) cudaFreeHost(P->h_stop);
    if (P->arena) cudaFree(P->arena);
    delete P;
    return IMR_SUCCESS;
}

int imr_hio_plan_create(imr_hio_plan **out, unsigned W, unsigned H, unsigned nCycles, float targetError,
                        float beta)
{
    if (!out || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    *out = nullptr;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    // parameter defaults of hybridInputOutput.cpp:208-213; the iteration
    // count is kept below INT_MAX (UINT_MAX in the reference: both unbounded
    // in practice)
    if (nCycles == 0) nCycles = UINT_MAX;
    if (!(beta > 0)) beta = 0.9f;
    const int n_cycles = nCycles >= (unsigned)INT_MAX ? INT_MAX - 1 : (int)nCycles;
    imr_hio_plan *P = new imr_hio_plan();
    cudaGetDevice(&P->dev);
    P->W = (int)W;
    P->H = (int)H;
    imr_params p{};
    resolve_params(nullptr, p);
    JobDev &J = P->hj;
    JobShape S;
    if ((rc = job_prepare(W, H, p, J, S))) {
        delete P;
        return rc;
    }
    J.mode = kModeHio;
    J.n_cycles = n_cycles;
    J.n_hio = 0;
    J.target = targetError;
    J.beta = beta;
    J.n_err = n_cycles < kHioMaxErrors ? n_cycles + 1 : kHioMaxErrors;
    S.bytes = S.oErr + ((size_t)J.n_err * 4 + 255) / 256 * 256;
    const size_t sst = (sizeof(JobState) + 255) / 256 * 256, sdj = (sizeof(JobDev) + 255) / 256 * 256;
    cudaError_t e = cudaMalloc(&P->arena, S.bytes + sst + sdj + 256);
    if (e != cudaSuccess) {
        set_error("cudaMalloc HIO plan arena", e);
        delete P;
        return IMR_ERR_OUT_OF_MEMORY;
    }
    char *a = (char *)P->arena;
    JobState *st = (JobState *)(a + S.bytes);
    P->dj = (JobDev *)(a + S.bytes + sst);
    P->Lrow = (WorkList *)(a + S.bytes + sst + sdj);
    P->Lcol = P->Lrow + 1;
    job_bind(J, S, a, st);
    P->st = st;
    P->rk = S.rk;
    P->ck = S.ck;
    P->p_rows = S.rk.p_hio_fix != nullptr;
    P->p_cols = S.p_cols;
    P->smem_row = S.smem_row;
    P->smem_col = S.smem_col;
    if (P->p_rows)
        P->g_row = persistent_grid((const void *)P->rk.p_hio_fix, P->rk.threads, P->rk.p_smem, J.n_row_tiles);
    int n_split = 0;
    if (P->p_cols) {
        int g_max = persistent_grid((const void *)P->ck.p_col, P->ck.p_threads, P->ck.p_smem, 1 << 30);
        if (S.p_half && col_split(J.n_col_tiles, g_max)) {   // the half-tile variant of the pass
            P->ck.p_col = P->ck.p_col_split;
            g_max = persistent_grid((const void *)P->ck.p_col, P->ck.p_threads, P->ck.p_smem, 1 << 30);
            n_split = col_split(J.n_col_tiles, g_max);
        }
        P->g_col = std::min(g_max, J.n_col_tiles + n_split);
    }
    const WorkList lists[2] = {{nullptr, J.n_row_tiles, 0}, {nullptr, J.n_col_tiles, n_split}};
    e = cudaMemcpy(P->Lrow, lists, sizeof(lists), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = job_upload(J, S, a, P->dj, 0) ? cudaErrorUnknown : cudaSuccess;
    if (e == cudaSuccess) e = cudaHostAlloc((void **)&P->h_stop, 2 * sizeof(int), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev[0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&P->ev[1], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error("HIO plan upload", e);
        imr_hio_plan_destroy(P);
        return IMR_ERR_CUDA;
    }
    P->chunk = n_cycles + 1 < kHioChunk ? n_cycles + 1 : kHioChunk;
    cudaStream_t cs;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int i = 0; i < P->chunk && rc == IMR_SUCCESS; ++i) rc = hio_launch_iteration(P, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &P->graph);
        if (rc == IMR_SUCCESS && e2 == cudaSuccess)
            e = cudaGraphInstantiate(&P->gexec, P->graph, 0);
        else if (e2 != cudaSuccess)
            e = e2;
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess || rc != IMR_SUCCESS) {
        if (e != cudaSuccess) set_error("graph capture", e);
        imr_hio_plan_destroy(P);
        return rc ? rc : IMR_ERR_CUDA;
    }
    *out = P;
    return IMR_SUCCESS;
}

// Random phase, then the iterations; M and the mask are already in place.
static int hio_run(imr_hio_plan *P, unsigned seed, cudaStream_t s)
{
    const JobDev &J = P->hj;
    const long N = (long)P->W * P->H;
    HCK(cudaMemsetAsync(P->st, 0, sizeof(JobState), s));
    int rc = job_modulus_tiles(J, s);
    if (rc) return rc;
    if ((rc = launch_rand_field(J.X, N, seed, s))) return rc;
    if ((rc = fft_passes(J.X, P->W, P->H, -1, 3, J.prow, J.pcol, s))) return rc;
    const int g = (int)std::min<long>((N + 255) / 256, 148L * 16);
    k_random_phase<<<g, 256, 0, s>>>(J.X, J.M, N);
    HCK(cudaGetLastError());
    if ((rc = fft_passes(J.X, P->W, P->H, +1, 2, J.prow, J.pcol, s))) return rc;
    // k = 0 .. n_cycles: n_cycles + 1 row passes at most
    const long replays = ((long)J.n_cycles + 1 + P->chunk - 1) / P->chunk;
    const bool poll = J.target > 0.f && replays > 1;
    for (long c = 0; c < replays; ++c) {
        HCK(cudaGraphLaunch(P->gexec, s));
        if (!poll) continue;
        HCK(cudaMemcpyAsync(&P->h_stop[c & 1], &P->st->stop, sizeof(int), cudaMemcpyDeviceToHost, s));
        HCK(cudaEventRecord(P->ev[c & 1], s));
        if (c >= 1) {
            HCK(cudaEventSynchronize(P->ev[(c - 1) & 1]));
            if (P->h_stop[(c - 1) & 1]) break;
        }
    }
    return IMR_SUCCESS;
}

int imr_hio_plan_execute(imr_hio_plan *P, const float *d_modulus, const uint8_t *d_mask, float *d_out,
                         unsigned seed, void *stream)
{
    if (!P || !d_modulus || !d_mask || !d_out) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    const JobDev &J = P->hj;
    const size_t N = (size_t)P->W * P->H;
    HCK(cudaMemcpyAsync((void *)J.M, d_modulus, N * 4, cudaMemcpyDeviceToDevice, s));
    HCK(cudaMemcpyAsync(J.mask, d_mask, N, cudaMemcpyDeviceToDevice, s));
    int rc = hio_run(P, seed, s);
    if (rc) return rc;
    HCK(cudaMemcpyAsync(d_out, J.out, N * 4, cudaMemcpyDeviceToDevice, s));
    return IMR_SUCCESS;
}

int imr_hio_plan_execute_host(imr_hio_plan *P, const float *h_modulus, const uint8_t *h_mask, float *h_out,
                              unsigned seed, void *stream)
{
    if (!P || !h_modulus || !h_mask || !h_out) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    const JobDev &J = P->hj;
    const size_t N = (size_t)P->W * P->H;
    HCK(cudaMemcpyAsync((void *)J.M, h_modulus, N * 4, cudaMemcpyHostToDevice, s));
    HCK(cudaMemcpyAsync(J.mask, h_mask, N, cudaMemcpyHostToDevice, s));
    int rc = hio_run(P, seed, s);
    if (rc) return rc;
    HCK(cudaMemcpyAsync(h_out, J.out, N * 4, cudaMemcpyDeviceToHost, s));
    HCK(cudaStreamSynchronize(s));
    return IMR_SUCCESS;
}

int imr_hio_plan_stats(imr_hio_plan *P, void *stream, int *iterations, float *last_error, float *errors,
                       int cap)
{
    if (!P || cap < 0) return IMR_ERR_INVALID_VALUE;
    HCK(cudaStreamSynchronize((cudaStream_t)stream));
    JobState st;
    HCK(cudaMemcpy(&st, P->st, sizeof(JobState), cudaMemcpyDeviceToHost));
    if (st.err) {
        snprintf(g_last_error, sizeof(g_last_error), "a device-side copy wait timed out");
        return IMR_ERR_DEVICE_TIMEOUT;
    }
    if (iterations) *iterations = st.cycles_done;
    if (last_error) *last_error = st.last_error;
    if (errors && cap > 0) {
        int n = st.cycles_done + 1 < P->hj.n_err ? st.cycles_done + 1 : P->hj.n_err;
        if (n > cap) n = cap;
        HCK(cudaMemcpy(errors, P->hj.errors, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }
    return IMR_SUCCESS;
}

// ------------------------------------------------------------ drop-in
int imr_hybrid_input_output(float *io, const uint8_t *mask, unsigned W, unsigned H, unsigned nCycles,
                            float targetError, float beta, void *stream)
{
    if (!io || !mask || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    if (!length_supported((int)W) || !length_supported((int)H)) return IMR_ERR_UNSUPPORTED_SIZE;
    imr_hio_plan *P = nullptr;
    int rc = imr_hio_plan_create(&P, W, H, nCycles, targetError, beta);
    if (rc) return rc;
    rc = imr_hio_plan_execute_host(P, io, mask, io, IMR_HIO_SEED, stream);
    imr_hio_plan_destroy(P);
    return rc;
}

int imr_rand_field(void *d_out, size_t n, unsigned seed, void *stream)
{
    if (n == 0) return IMR_SUCCESS;
    if (!d_out) return IMR_ERR_INVALID_VALUE;
    return launch_rand_field((float2 *)d_out, (long)n, seed, (cudaStream_t)stream);
}

// ------------------------------------------------------------ HIO error
int imr_calculate_hio_error(const void *d_data, const void *d_mask, int mask_type, size_t n, int invert_mask,
                            float *h_total, float *h_count, float *h_error, void *stream)
{
    if (!d_data || !d_mask || (mask_type != IMR_MASK_F32 && mask_type != IMR_MASK_U8)) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    double res[2] = {0.0, 0.0};
    if (n > 0) {
        const long grid = std::min<long>(((long)n + 255) / 256, 148L * 4);
        char *buf = nullptr;
        const size_t pb = (size_t)grid * 2 * sizeof(double);
        HCK(cudaMallocAsync((void **)&buf, pb + 256, s));
        double *part = (double *)buf;
        double *dres = (double *)(buf + pb);
        unsigned *counter = (unsigned *)(buf + pb + 2 * sizeof(double));
        HCK(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
        if (mask_type == IMR_MASK_F32)
            k_hio_error<float><<<(unsigned)grid, 256, 0, s>>>((const float2 *)d_data, (const float *)d_mask, (long)n,
                                                              invert_mask, part, counter, dres);
        else
            k_hio_error<uint8_t><<<(unsigned)grid, 256, 0, s>>>((const float2 *)d_data, (const uint8_t *)d_mask,
                                                                (long)n, invert_mask, part, counter, dres);
        HCK(cudaGetLastError());
        HCK(cudaMemcpyAsync(res, dres, sizeof(res), cudaMemcpyDeviceToHost, s));
        HCK(cudaFreeAsync(buf, s));
        HCK(cudaStreamSynchronize(s));
    }
    const float total = (float)res[0], count = (float)res[1];
    if (h_total) *h_total = total;
    if (h_count) *h_count = count;
    if (h_error) *h_error = sqrtf(total) / count;
    return IMR_SUCCESS;
}

}  // extern "C"
