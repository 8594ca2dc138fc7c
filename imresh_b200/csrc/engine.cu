// Host side of the engine: FFT plans, reconstruction plans (device buffers +
// captured CUDA graph of one shrink-wrap cycle) and the C ABI declared in
// include/imresh_b200.h.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "imresh_b200.h"
#include "kernels.cuh"
#include "engine_host.hpp"
#include <cudaTypedefs.h>

namespace imr {

thread_local char g_last_error[256] = "";

void set_error(const char *what, cudaError_t e)
{
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------- lengths
// Radix schedule: 8s first (4,4 or 4 or 2 for the remaining power of two),
// then 3s, 5s and 7s.  Supported lengths: every 2^a 3^b 5^c 7^d up to
// kMaxRuntimeSide (runtime-length kernels hold 8 values x 256 threads), and
// the compile-time lengths 3072 and 4096 above it.
bool factor_len(int n, std::vector<int> &rad)
{
    rad.clear();
    if (n < 1 || n > (int)kMaxSide) return false;
    if (n > kMaxRuntimeSide && n != 3072 && n != 4096) return false;
    int m = n, k = 0;
    while (m % 2 == 0) { m /= 2; ++k; }
    while (k >= 3 && !(k == 4)) { rad.push_back(8); k -= 3; }
    if (k == 4) { rad.push_back(4); rad.push_back(4); }
    else if (k == 2) rad.push_back(4);
    else if (k == 1) rad.push_back(2);
    for (int p : {3, 5, 7})
        while (m % p == 0) { rad.push_back(p); m /= p; }
    return m == 1 && (int)rad.size() <= 14;
}

// Supported image sides: every length 1..kMaxRuntimeSide (direct mixed-radix
// transforms when the length factors into 2, 3, 5, 7; Bluestein otherwise),
// plus the compile-time lengths 3072 and 4096.
int bluestein_m(int n)
{
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    return m;
}

bool length_supported(int n)
{
    std::vector<int> rad;
    if (factor_len(n, rad)) return true;
    return n >= 1 && n <= kMaxRuntimeSide;
}

// in-place radix-2 FFT in double (host; Bluestein kernel spectra)
static void host_fft_pow2(std::vector<double> &re, std::vector<double> &im, int sign)
{
    const int n = (int)re.size();
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        for (int i = 0; i < n; i += len)
            for (int k = 0; k < len / 2; ++k) {
                const double a = sign * 2.0 * M_PI * (double)k / (double)len;
                const double wr = cos(a), wi = sin(a);
                const double ur = re[i + k], ui = im[i + k];
                const double xr = re[i + k + len / 2], xi = im[i + k + len / 2];
                const double vr = xr * wr - xi * wi, vi = xr * wi + xi * wr;
                re[i + k] = ur + vr;
                im[i + k] = ui + vi;
                re[i + k + len / 2] = ur - vr;
                im[i + k + len / 2] = ui - vi;
            }
    }
}

// Twiddle tables exp(-2 pi i t/L), t < L, computed in double; one per
// (device, n), kept for the life of the process.  Bluestein lengths also
// keep their chirp and kernel spectra in the same allocation.
static std::mutex g_tw_mu;
static std::map<std::pair<int, int>, float2 *> g_tw;

static int make_bluestein_plan(int n, FftPlanDev &p)
{
    const int M = bluestein_m(n);
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_tw_mu);
    auto key = std::make_pair(dev, -n);
    float2 *d = nullptr;
    auto it = g_tw.find(key);
    if (it == g_tw.end()) {
        std::vector<float2> h((size_t)M + n + 2 * (size_t)M);
        for (int t = 0; t < M; ++t) {
            const double a = -2.0 * M_PI * (double)t / (double)M;
            h[t] = make_float2((float)cos(a), (float)sin(a));
        }
        std::vector<double> cre(n), cim(n);
        for (int j = 0; j < n; ++j) {
            const long long q = ((long long)j * j) % (2LL * n);   // j^2 mod 2n: exact angle
            const double a = -M_PI * (double)q / (double)n;
            cre[j] = cos(a);
            cim[j] = sin(a);
            h[M + j] = make_float2((float)cre[j], (float)cim[j]);
        }
        for (int dir = 0; dir < 2; ++dir) {   // 0: forward (S = -1), 1: inverse (S = +1)
            std::vector<double> kr(M, 0.0), ki(M, 0.0);
            for (int j = 0; j < n; ++j) {
                // kernel conj(c_j) with c_j = exp(S i pi j^2/n), wrapped for negative j
                const double br = cre[j], bi = dir == 0 ? -cim[j] : cim[j];
                kr[j] = br;
                ki[j] = bi;
                if (j) {
                    kr[M - j] = br;
                    ki[M - j] = bi;
                }
            }
            host_fft_pow2(kr, ki, -1);
            for (int t = 0; t < M; ++t)
                h[(size_t)M + n + (size_t)dir * M + t] = make_float2((float)(kr[t] / M), (float)(ki[t] / M));
        }
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * h.size());
        if (e != cudaSuccess) { set_error("cudaMalloc Bluestein tables", e); return IMR_ERR_OUT_OF_MEMORY; }
        e = cudaMemcpy(d, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { set_error("cudaMemcpy Bluestein tables", e); return IMR_ERR_CUDA; }
        g_tw[key] = d;
    } else {
        d = it->second;
    }
    memset(&p, 0, sizeof(p));
    p.n = n;
    p.bs_m = M;
    p.tw = d;
    p.chirp = d + M;
    p.bspec_f = d + M + n;
    p.bspec_b = d + M + n + M;
    return IMR_SUCCESS;
}

int make_fft_plan(int n, FftPlanDev &p)
{
    std::vector<int> rad;
    if (!factor_len(n, rad)) return length_supported(n) ? make_bluestein_plan(n, p) : IMR_ERR_UNSUPPORTED_SIZE;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_tw_mu);
    auto key = std::make_pair(dev, n);
    auto it = g_tw.find(key);
    float2 *d = nullptr;
    if (it == g_tw.end()) {
        std::vector<float2> h(n);
        for (int t = 0; t < n; ++t) {
            double a = -2.0 * M_PI * (double)t / (double)n;
            h[t] = make_float2((float)cos(a), (float)sin(a));
        }
        cudaError_t e = cudaMalloc(&d, sizeof(float2) * n);
        if (e != cudaSuccess) { set_error("cudaMalloc twiddles", e); return IMR_ERR_OUT_OF_MEMORY; }
        e = cudaMemcpy(d, h.data(), sizeof(float2) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { set_error("cudaMemcpy twiddles", e); return IMR_ERR_CUDA; }
        g_tw[key] = d;
    } else {
        d = it->second;
    }
    memset(&p, 0, sizeof(p));
    p.n = n;
    p.nrad = (int)rad.size();
    for (size_t i = 0; i < rad.size(); ++i) p.rad[i] = rad[i];
    p.tw = d;
    return IMR_SUCCESS;
}

// calcGaussianKernel<float> (src/imresh/libs/calcGaussianKernel.cpp:42-91):
// half width ceil(2.884402748387961466*sigma - 0.5); weights a*exp(i*i*b)
// rounded to float, normalised by their double sum.
int gaussian_weights(double sigma, float *w, int cap)
{
    const int half = (int)ceil(2.884402748387961466 * sigma - 0.5);
    const int K = 2 * half + 1;
    if (w == nullptr || K > cap) return K;
    const double a = 1.0 / (sqrt(2.0 * M_PI) * sigma);
    const double b = -1.0 / (2.0 * sigma * sigma);
    double sum = 0;
    for (int i = -half; i <= half; ++i) {
        float v = (float)(a * exp(i * i * b));
        w[half + i] = v;
        sum += v;
    }
    for (int i = 0; i < K; ++i) w[i] = (float)((double)w[i] / sum);
    return K;
}

// ---------------------------------------------------------------- dispatch
// Kernels specialised at compile time for the lengths below; any other
// supported length runs the runtime-length FFT (N = 0 instantiation).
template <int N>
static RowKernels row_set()
{
    RowKernels k{};
    if constexpr (N >= 16 && is_pow2(N)) {
        k = RowKernels{k_row_hio_r<true, N>, k_row_hio_r<false, N>, k_row_finish_r<N>,
                       k_fft_rows_r<-1, N>, k_fft_rows_r<+1, N>, rrow_nb(N), rrow_threads(N),
                       rrow_smem(N), k_row_hio_p<true, N>, k_row_hio_p<false, N>,
                       prow_smem<true, N>(), prow_smem<false, N>(), 0};
        k.hio_fix = k_row_hio_r<false, N, true>;
        k.p_hio_fix = k_row_hio_p<false, N, true>;
        k.p_finish = k_row_finish_p<N>;
        k.p_smem_fin = pfin_smem<N>();
    } else if constexpr (N >= 8 && is_pow2(N)) {
        k = RowKernels{k_row_hio_r<true, N>, k_row_hio_r<false, N>, k_row_finish_r<N>,
                       k_fft_rows_r<-1, N>, k_fft_rows_r<+1, N>, rrow_nb(N), rrow_threads(N),
                       rrow_smem(N), nullptr, nullptr, 0, 0, 0};
        k.hio_fix = k_row_hio_r<false, N, true>;
    } else if constexpr (is_3pow2(N)) {   // per-tile kernels + pipelined 12-value register passes
        k = RowKernels{k_row_hio<true, N>, k_row_hio<false, N>, k_row_finish<N>, k_fft_rows<-1, N>,
                       k_fft_rows<+1, N>, row_nb(N), row_threads(N), 0, k_row_hio_p<true, N>,
                       k_row_hio_p<false, N>, prow_smem<true, N>(), prow_smem<false, N>(), 0};
        k.hio_fix = k_row_hio<false, N, true>;
        k.p_hio_fix = k_row_hio_p<false, N, true>;
        k.p_finish = k_row_finish_p<N>;
        k.p_smem_fin = pfin_smem<N>();
    } else if constexpr (N < 0 && -N >= 256) {   // Bluestein lengths, 16 values per thread
        constexpr int M = -N;
        k = RowKernels{k_row_hio_bs16<true, M>, k_row_hio_bs16<false, M>, k_row_finish_bs16<M>,
                       k_fft_rows_bs16<-1, M>, k_fft_rows_bs16<+1, M>, bs16_rows(M), bs16_row_threads(M),
                       bs16_row_smem(M), nullptr, nullptr, 0, 0, M};
        k.hio_fix = k_row_hio_bs16<false, M, true>;
    } else if constexpr (N < 0 && -N >= 8) {   // Bluestein lengths: register chirp-z transforms
        constexpr int M = -N;
        k = RowKernels{k_row_hio_bs<true, M>, k_row_hio_bs<false, M>, k_row_finish_bs<M>, k_fft_rows_bs<-1, M>,
                       k_fft_rows_bs<+1, M>, rrow_nb(M), rrow_threads(M), rrow_smem(M), nullptr, nullptr, 0, 0,
                       M};
        k.hio_fix = k_row_hio_bs<false, M, true>;
    } else {
        k = RowKernels{k_row_hio<true, N>, k_row_hio<false, N>, k_row_finish<N>, k_fft_rows<-1, N>,
                       k_fft_rows<+1, N>, row_nb(N), row_threads(N), 0, nullptr, nullptr, 0, 0,
                       N < 0 ? -N : 0};
        k.hio_fix = k_row_hio<false, N, true>;
    }
    return k;
}
template <int N>
static ColKernels col_set()
{
    if constexpr (N >= 128 && N <= 4096 && is_pow2(N)) {   // 16 values per thread in the pipelined pass
        constexpr int T = pcol16_nbt(N);
        ColKernels k{k_col_r<N>, k_col_init_r<N>, k_fft_cols_r<-1, N>, k_fft_cols_r<+1, N>,
                     rcol_nb(N), rcol_threads(N), rcol_smem(N), k_col_p16<N, T, false>, pcol16_smem<N, T>(),
                     pcol_box_rows(N), 0, pcol16_threads(N, T), 0, T, 1};
        if constexpr (N >= 256) {   // split-precision tensor-core variants
            k.p_col_tc[0] = k_col_tc<N, T, kPrecBf16x3, 0>;
            k.p_col_tc[1] = k_col_tc<N, T, kPrecFp16x3, 0>;
            k.fft_tc[0][0] = k_col_tc<N, T, kPrecBf16x3, 1>;
            k.fft_tc[0][1] = k_col_tc<N, T, kPrecBf16x3, 2>;
            k.fft_tc[1][0] = k_col_tc<N, T, kPrecFp16x3, 1>;
            k.fft_tc[1][1] = k_col_tc<N, T, kPrecFp16x3, 2>;
            k.p_smem_tc = pcol_tc_smem<N, T>();
        }
        if constexpr (T >= 4) k.p_col_split = k_col_p16<N, T, true>;   // half tiles of >= 2 columns (16-byte TMA rows)
        return k;
    } else if constexpr (N >= 16 && is_pow2(N))
        return ColKernels{k_col_r<N>, k_col_init_r<N>, k_fft_cols_r<-1, N>, k_fft_cols_r<+1, N>,
                          rcol_nb(N), rcol_threads(N), rcol_smem(N), k_col_p<N>, pcol_smem<N>(),
                          pcol_box_rows(N), pcol_tma_m(N) ? 1 : 0, pcol_threads(N), 0, rcol_nb(N)};
    else if constexpr (N >= 8 && is_pow2(N))
        return ColKernels{k_col_r<N>, k_col_init_r<N>, k_fft_cols_r<-1, N>, k_fft_cols_r<+1, N>,
                          rcol_nb(N), rcol_threads(N), rcol_smem(N), nullptr, 0, 0, 0, 0, 0};
    else if constexpr (is_3pow2(N))
        return ColKernels{k_col<N>, k_col_init<N>, k_fft_cols<-1, N>, k_fft_cols<+1, N>, col_nb(N),
                          col_threads(N), 0, k_col_p<N>, pcol_smem<N>(), pcol_box_rows(N),
                          pcol_tma_m(N) ? 1 : 0, pcol_threads(N), 0, rcol_nb(N)};
    else if constexpr (N < 0 && -N >= 256)   // Bluestein lengths, 16 values per thread
        return ColKernels{k_col_bs16<-N, 0>, k_col_bs16<-N, 1>, k_fft_cols_bs16<-1, -N>, k_fft_cols_bs16<+1, -N>,
                          rcol_nb(-N), bs16_col_threads(-N), bs16_col_smem(-N), nullptr, 0, 0, 0, 0, -N, 0};
    else if constexpr (N < 0 && -N >= 8)   // Bluestein lengths: register chirp-z transforms
        return ColKernels{k_col_bs<-N>, k_col_init_bs<-N>, k_fft_cols_bs<-1, -N>, k_fft_cols_bs<+1, -N>,
                          rcol_nb(-N), rcol_threads(-N), rcol_smem(-N), nullptr, 0, 0, 0, 0, -N, 0};
    else
        return ColKernels{k_col<N>, k_col_init<N>, k_fft_cols<-1, N>, k_fft_cols<+1, N>, col_nb(N),
                          col_threads(N), 0, nullptr, 0, 0, 0, 0, N < 0 ? -N : 0};
}

// Resident CTAs per SM of a kernel at a launch shape, asked of the occupancy
// calculator once per (device, kernel, shape): the engine launches hundreds
// of persistent passes per step.
struct OccKey {
    int dev;
    const void *k;
    int threads, smem;
    bool operator<(const OccKey &o) const
    {
        return std::tie(dev, k, threads, smem) < std::tie(o.dev, o.k, o.threads, o.smem);
    }
};
static std::mutex g_occ_mu;
static std::map<OccKey, std::pair<int, int>> g_occ;   // -> (CTAs per SM, SMs)

int persistent_grid(const void *kernel, int threads, int smem, int items)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const OccKey key{dev, kernel, threads, smem};
    std::pair<int, int> occ;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(key);
        if (it != g_occ.end()) {
            occ = it->second;
        } else {
            int sms = 148, per_sm = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            occ = {per_sm, sms};
            g_occ[key] = occ;
        }
    }
    const long g = (long)occ.first * occ.second;
    return (int)(g < items ? g : items);
}

// A persistent column pass runs one tile per CTA at a time.  When the tiles
// fill at most half of the resident CTAs (256^2: 16 tiles, 512^2: 32, on 148
// SMs) every tile runs as two half tiles on two CTAs (bit-identical results):
// measured 5.6 -> 5.1 us at 256^2 and 8.8 -> 6.9 us at 512^2.  Beyond that a
// half tile, at ~79 % of a whole tile's time, loses: splitting each CTA's first
// and last tile at 2048^2 took the pass from 33.3 to 37.6 us, and all tiles at
// 1024^2 (two rounds of halves) from 9.8 to 12.7 us.
int col_split(int n_tiles, int g_max)
{
    return (n_tiles > 0 && 2 * n_tiles <= g_max) ? n_tiles : 0;
}

int scaled_grid(const void *kernel, int threads, int smem, int items, int grid_pct)
{
    const int g = persistent_grid(kernel, threads, smem, 1 << 30);   // the occupancy limit
    const long want = std::max(1L, (long)g * grid_pct / 100);
    return (int)std::min<long>(want, std::max(items, 1));
}

int launch_finish(const RowKernels &rk, int items, size_t smem_fin, cudaStream_t s, const JobDev *dj,
                  const WorkList *L, float2 *dbg, int grid_pct)
{
    if (rk.p_finish)
        rk.p_finish<<<scaled_grid((const void *)rk.p_finish, rk.threads, rk.p_smem_fin, items, grid_pct), rk.threads,
                      rk.p_smem_fin, s>>>(dj, L, dbg);
    else
        rk.finish<<<items, rk.threads, smem_fin, s>>>(dj, L, dbg);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("finish launch", e);
        return IMR_ERR_CUDA;
    }
    return IMR_SUCCESS;
}

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

bool encode_tensor_map(CUtensorMap *map, const void *base, int W, int H, int elem, int box_w, int box_h)
{
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    if (((size_t)W * elem) % 16 != 0 || ((uintptr_t)base & 15) != 0 || (box_w * elem) % 16 != 0) return false;
    if (box_w > 256 || box_h > 256 || box_w > W || box_h > H) return false;
    cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
    cuuint64_t strides[1] = {(cuuint64_t)W * elem};
    cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                          const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

#define IMR_SIZES(X) X(64) X(128) X(192) X(256) X(384) X(512) X(768) X(1024) X(1536) X(2048) X(3072) X(4096)
// Bluestein transform lengths M (power of two >= 2n - 1 for n <= 2048)
#define IMR_BS_SIZES(X) X(-8) X(-16) X(-32) X(-64) X(-128) X(-256) X(-512) X(-1024) X(-2048) X(-4096)

RowKernels row_kernels(int N)
{
    std::vector<int> rad;
    if (!factor_len(N, rad) && length_supported(N)) N = -bluestein_m(N);
    switch (N) {
#define ROWCASE(n) case n: return row_set<n>();
        IMR_SIZES(ROWCASE)
        IMR_BS_SIZES(ROWCASE)
#undef ROWCASE
    default: {
        RowKernels k = row_set<0>();
        k.nb = (kRowVpt * kRowThreads) / N;
        if (k.nb < 1) k.nb = 1;
        return k;
    }
    }
}

ColKernels col_kernels(int N)
{
    std::vector<int> rad;
    if (!factor_len(N, rad) && length_supported(N)) N = -bluestein_m(N);
    switch (N) {
#define COLCASE(n) case n: return col_set<n>();
        IMR_SIZES(COLCASE)
        IMR_BS_SIZES(COLCASE)
#undef COLCASE
    default: {
        ColKernels k = col_set<0>();
        k.nb = (kColVpt * kColThreads) / N;
        if (k.nb > 8) k.nb = 8;
        if (k.nb < 1) k.nb = 1;
        return k;
    }
    }
}

static std::mutex g_attr_mu;
static std::vector<int> g_attr_done;

// Opt every kernel into the device's largest dynamic shared-memory size
// (opt-in limit minus the kernel's static shared memory).
static int g_optin_smem = 0;

template <class F>
static cudaError_t allow_smem(F f)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)f);
    if (e != cudaSuccess) return e;
    const int dyn = g_optin_smem - (int)fa.sharedSizeBytes;
    return cudaFuncSetAttribute((const void *)f, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
}

int ensure_kernel_attributes()
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (int d : g_attr_done)
        if (d == dev) return IMR_SUCCESS;
    cudaError_t e = cudaDeviceGetAttribute(&g_optin_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    std::vector<int> sizes = {0};
#define PUSH(n) sizes.push_back(n);
    IMR_SIZES(PUSH)
#undef PUSH
    std::vector<RowKernels> rks;
    std::vector<ColKernels> cks;
    for (int n : sizes) {
        rks.push_back(n ? row_kernels(n) : row_set<0>());
        cks.push_back(n ? col_kernels(n) : col_set<0>());
    }
#define PUSHBS(n) rks.push_back(row_set<n>()); cks.push_back(col_set<n>());
    IMR_BS_SIZES(PUSHBS)
#undef PUSHBS
    for (size_t q = 0; q < rks.size(); ++q) {
        RowKernels r = rks[q];
        ColKernels c = cks[q];
        if (e == cudaSuccess) e = allow_smem(r.hio_first);
        if (e == cudaSuccess) e = allow_smem(r.hio);
        if (e == cudaSuccess) e = allow_smem(r.finish);
        if (e == cudaSuccess) e = allow_smem(r.fft_fwd);
        if (e == cudaSuccess) e = allow_smem(r.fft_inv);
        if (e == cudaSuccess) e = allow_smem(c.col);
        if (e == cudaSuccess) e = allow_smem(c.init);
        if (e == cudaSuccess) e = allow_smem(c.fft_fwd);
        if (e == cudaSuccess) e = allow_smem(c.fft_inv);
        if (e == cudaSuccess && r.p_hio) e = allow_smem(r.p_hio);
        if (e == cudaSuccess && r.p_hio_first) e = allow_smem(r.p_hio_first);
        if (e == cudaSuccess) e = allow_smem(r.hio_fix);
        if (e == cudaSuccess && r.p_hio_fix) e = allow_smem(r.p_hio_fix);
        if (e == cudaSuccess && r.p_finish) e = allow_smem(r.p_finish);
        if (e == cudaSuccess && c.p_col) e = allow_smem(c.p_col);
        if (e == cudaSuccess && c.p_col_split) e = allow_smem(c.p_col_split);
        for (int pr = 0; pr < 2; ++pr) {
            if (e == cudaSuccess && c.p_col_tc[pr]) e = allow_smem(c.p_col_tc[pr]);
            for (int d = 0; d < 2; ++d)
                if (e == cudaSuccess && c.fft_tc[pr][d]) e = allow_smem(c.fft_tc[pr][d]);
        }
    }
    if (e == cudaSuccess) e = allow_smem(k_hblur);
    if (e != cudaSuccess) {
        set_error("cudaFuncSetAttribute", e);
        return IMR_ERR_CUDA;
    }
    g_attr_done.push_back(dev);
    return IMR_SUCCESS;
}

void resolve_params(const imr_params *in, imr_params &p)
{
    // Defaults of the reference's CUDA driver (cudaShrinkWrap.cu:193-200).
    if (in) p = *in;
    else memset(&p, 0, sizeof(p));
    if (p.nCycles == 0) p.nCycles = 20;
    if (!(p.targetError > 0)) p.targetError = 1e-5f;
    if (!(p.hioBeta > 0)) p.hioBeta = 0.9f;
    if (!(p.intensityCutOffAutoCorel > 0)) p.intensityCutOffAutoCorel = 0.02f;
    if (!(p.intensityCutOff > 0)) p.intensityCutOff = 0.2f;
    if (!(p.sigma0 > 0)) p.sigma0 = 3.0f;
    if (!(p.sigmaChange > 0)) p.sigmaChange = 0.01f;
    if (p.nHioCycles == 0) p.nHioCycles = 20;
}

// Sigma of every cycle (sigma <- max(1.5, (1 - change)*sigma) after each
// mask, in float: cudaShrinkWrap.cu:294) and its Gaussian weights.  Entry
// n_cycles serves the final error-only pass.
int build_weight_table(const imr_params &p, std::vector<float> &w, std::vector<int> &taps)
{
    w.assign((size_t)(p.nCycles + 1) * kTapStride, 0.f);
    taps.assign(p.nCycles + 1, 1);
    float sigma = p.sigma0;
    for (unsigned c = 0; c <= p.nCycles; ++c) {
        int K = gaussian_weights((double)sigma, &w[(size_t)c * kTapStride], kMaxTaps);
        if (K > kMaxTaps) return IMR_ERR_INVALID_VALUE;
        taps[c] = K;
        sigma = fmaxf(1.5f, (1.0f - p.sigmaChange) * sigma);
    }
    return IMR_SUCCESS;
}

// Unnormalised 2D transform passes over a [H][W] complex array with the
// plain FFT kernels: axes bit 1 = rows, bit 2 = columns; sign -1 runs rows
// then columns, +1 columns then rows.
int fft_passes(float2 *d, int W, int H, int sign, int axes, const FftPlanDev &pr, const FftPlanDev &pc,
               cudaStream_t s)
{
    const RowKernels rk = row_kernels(W);
    const ColKernels ck = col_kernels(H);
    const int rpc = rk.nb, cpc = ck.nb;
    const int nrt = (H + rpc - 1) / rpc, nct = (W + cpc - 1) / cpc;
    const size_t sr = rk.smem ? (size_t)rk.smem : ((size_t)rpc * W + rk.bs_m) * 8;
    const size_t sc = ck.smem ? (size_t)ck.smem : ((size_t)H + ck.bs_m) * cpc * 8;
    if (sign < 0) {
        if (axes & 1) rk.fft_fwd<<<nrt, rk.threads, sr, s>>>(d, pr, H, rpc);
        if (axes & 2) ck.fft_fwd<<<nct, ck.threads, sc, s>>>(d, pc, W, cpc);
    } else {
        if (axes & 2) ck.fft_inv<<<nct, ck.threads, sc, s>>>(d, pc, W, cpc);
        if (axes & 1) rk.fft_inv<<<nrt, rk.threads, sr, s>>>(d, pr, H, rpc);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("fft launch", e);
        return IMR_ERR_CUDA;
    }
    return IMR_SUCCESS;
}

}  // namespace imr

using namespace imr;

// ==================================================================== plans
constexpr int kPlanGraphCycles = 64;   // shrink-wrap cycles per captured graph

struct imr_plan {
    int dev = 0;
    int W = 0, H = 0;
    imr_params p{};
    JobDev hj{};
    JobDev *dj = nullptr;
    JobState *st = nullptr;
    void *arena = nullptr;
    size_t smem_row = 0, smem_fin = 0, smem_col = 0;
    // the cycles of one execution as at most two captured graphs: `chunk`
    // cycles replayed n_chunks times, then the remaining cycles
    cudaGraphExec_t gexec = nullptr, gexec_rem = nullptr;
    cudaGraph_t graph = nullptr, graph_rem = nullptr;
    int chunk = 0, n_chunks = 0;
    float2 *dbg_gprime = nullptr;
    RowKernels rk{};
    ColKernels ck{};
    bool p_rows = false, p_cols = false;   // pipelined passes in use
    int g_row_first = 0, g_row = 0, g_col = 0;
    WorkList *Lrow = nullptr, *Lcol = nullptr, *Lvb = nullptr;   // device
    int prec = 0;   // column pass: 0 FP32, 1 BF16 hi+lo tensor cores, 2 FP16 hi+lo tensor cores
    int g_col_tc = 0;
};

// The pipelined column pass of the plan's precision.
static void (*plan_col_kernel(const imr_plan *P))(const JobDev *, const WorkList *)
{
    return P->prec ? P->ck.p_col_tc[P->prec - 1] : P->ck.p_col;
}

static int plan_launch_cycle(imr_plan *P, cudaStream_t s)
{
    const JobDev &J = P->hj;
    const RowKernels &rk = P->rk;
    const ColKernels &ck = P->ck;
    int rc = launch_finish(rk, J.n_row_tiles, P->smem_fin, s, P->dj, P->Lrow, P->dbg_gprime);
    if (rc) return rc;
    k_vblur<<<J.n_vb_tiles, kVbThreads, 0, s>>>(P->dj, P->Lvb);
    for (int i = 0; i < J.n_hio; ++i) {
        if (P->p_rows) {
            if (i == 0)
                rk.p_hio_first<<<P->g_row_first, rk.threads, rk.p_smem_first, s>>>(P->dj, P->Lrow);
            else
                rk.p_hio<<<P->g_row, rk.threads, rk.p_smem, s>>>(P->dj, P->Lrow);
        } else {
            (i == 0 ? rk.hio_first : rk.hio)<<<J.n_row_tiles, rk.threads, P->smem_row, s>>>(P->dj, P->Lrow);
        }
        if (P->p_cols)
            plan_col_kernel(P)<<<P->prec ? P->g_col_tc : P->g_col, ck.p_threads,
                                 P->prec ? ck.p_smem_tc : ck.p_smem, s>>>(P->dj, P->Lcol);
        else
            ck.col<<<J.n_col_tiles, ck.threads, P->smem_col, s>>>(P->dj, P->Lcol);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("kernel launch", e);
        return IMR_ERR_CUDA;
    }
    return IMR_SUCCESS;
}

#define CK(call)                                  \
    do {                                          \
        cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) {                  \
            set_error(#call, e_);                 \
            return IMR_ERR_CUDA;                  \
        }                                         \
    } while (0)

namespace imr {

// ---------------------------------------------------------------- one job
// Host description of one reconstruction's device layout (shared by plans
// and the batched engine).  Arena layout, 256-byte aligned pieces:
// X, G (c64) | M, hb, vb, out (f32) | mask (u8) | weights | taps | error
// partials | per-cycle errors.  The JobState lives wherever the caller puts
// it (plans: after the arena; the engine: in one array for all jobs).
int job_prepare(unsigned W, unsigned H, const imr_params &p, JobDev &J, JobShape &S)
{
    int rc;
    memset(&J, 0, sizeof(J));
    J.W = (int)W;
    J.H = (int)H;
    if ((rc = make_fft_plan((int)W, J.prow)) || (rc = make_fft_plan((int)H, J.pcol))) return rc;
    if ((rc = build_weight_table(p, S.wt, S.taps))) return rc;
    S.rk = row_kernels(J.W);
    S.ck = col_kernels(J.H);
    J.rpc = S.rk.nb < J.H ? S.rk.nb : J.H;
    J.cpc = S.ck.nb < J.W ? S.ck.nb : J.W;
    S.p_rows = S.rk.p_hio != nullptr;
    S.p_cols = S.ck.p_col != nullptr && J.W % 4 == 0 && J.W >= S.ck.p_nb;
    if (S.p_cols) J.cpc = S.ck.p_nb;
    J.n_row_tiles = (J.H + J.rpc - 1) / J.rpc;
    J.n_col_tiles = (J.W + J.cpc - 1) / J.cpc;
    J.vb_tiles_x = (J.W + kVbTileX - 1) / kVbTileX;
    J.n_vb_tiles = J.vb_tiles_x * ((J.H + kVbTileY - 1) / kVbTileY);
    J.beta = p.hioBeta;
    J.cut_auto = p.intensityCutOffAutoCorel;
    J.cut = p.intensityCutOff;
    J.target = p.targetError;
    J.n_cycles = (int)p.nCycles;
    J.n_hio = (int)p.nHioCycles;
    // shared memory sized for the compile-time tile (NB sequences), even when
    // the image has fewer rows / columns than NB
    if (S.rk.smem) {
        S.smem_row = S.smem_fin = (size_t)S.rk.smem;   // norms reuse the FFT buffers
    } else if (S.rk.bs_m) {   // row + Bluestein work area (the norms reuse the work area)
        S.smem_row = S.smem_fin = ((size_t)J.W + S.rk.bs_m) * sizeof(float2);
    } else {
        S.smem_row = (size_t)S.rk.nb * J.W * sizeof(float2);
        S.smem_fin = S.smem_row + (size_t)S.rk.nb * J.W * sizeof(float);
    }
    S.smem_col = S.ck.smem ? (size_t)S.ck.smem
                 : S.ck.bs_m ? ((size_t)J.H + S.ck.bs_m) * S.ck.nb * sizeof(float2)
                             : (size_t)S.ck.nb * J.H * sizeof(float2);
    const size_t N = (size_t)W * H;
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t off = 0;
    S.oX = off; off += al(N * 8);
    S.oG = off; off += al(N * 8);
    S.oM = off; off += al(N * 4);
    if (S.p_cols && S.ck.p_mt) {
        S.oMt = off;
        off += al((size_t)((W + S.ck.p_nb - 1) / S.ck.p_nb) * S.ck.p_nb * H * 4);
    }
    S.oHB = off; off += al(N * 4);
    S.oVB = off; off += al(N * 4);
    S.oOut = off; off += al(N * 4);
    S.oMask = off; off += al(N);
    S.oW = off; off += al(S.wt.size() * 4);
    S.oT = off; off += al(S.taps.size() * 4);
    S.oEP = off; off += al((size_t)2 * J.n_row_tiles * 8);
    S.oErr = off; off += al((size_t)(J.n_cycles + 1) * 4);
    S.bytes = off;
    return IMR_SUCCESS;
}

void job_bind(JobDev &J, JobShape &S, char *a, JobState *st)
{
    J.X = (float2 *)(a + S.oX);
    J.G = (float2 *)(a + S.oG);
    J.M = (const float *)(a + S.oM);
    J.Mt = nullptr;
    J.hb = (float *)(a + S.oHB);
    J.vb = (float *)(a + S.oVB);
    J.out = (float *)(a + S.oOut);
    J.mask = (uint8_t *)(a + S.oMask);
    J.weights = (const float *)(a + S.oW);
    J.ntaps = (const int *)(a + S.oT);
    J.err_part = (double *)(a + S.oEP);
    J.errors = (float *)(a + S.oErr);
    J.st = st;
    J.use_tma_cols = 0;
    if (S.p_cols) {
        const int br = S.ck.p_box_rows;
        bool okm = encode_tensor_map(&J.tmX, J.X, J.W, J.H, 8, S.ck.p_nb, br);
        if (okm && S.ck.p_tma_m) okm = encode_tensor_map(&J.tmM, J.M, J.W, J.H, 4, S.ck.p_nb, br);
        if (!okm) {   // shape the TMA unit cannot describe: per-tile column pass
            S.p_cols = false;
            J.cpc = S.ck.nb < J.W ? S.ck.nb : J.W;
            J.n_col_tiles = (J.W + J.cpc - 1) / J.cpc;
        }
        J.use_tma_cols = S.p_cols ? 1 : 0;
        if (S.p_cols && S.ck.p_mt) J.Mt = (const float *)(a + S.oMt);
        S.p_half = S.p_cols && S.ck.p_col_split && encode_tensor_map(&J.tmXh, J.X, J.W, J.H, 8, S.ck.p_nb / 2, br);
    }
}

int job_modulus_tiles(const JobDev &J, cudaStream_t s)
{
    if (!J.Mt) return IMR_SUCCESS;
    const size_t n = (size_t)J.n_col_tiles * J.cpc * J.H;
    k_modulus_tiles<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(J.M, const_cast<float *>(J.Mt), J.W, J.H, J.cpc, n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("modulus tiles", e);
        return IMR_ERR_CUDA;
    }
    return IMR_SUCCESS;
}

int job_upload(const JobDev &J, const JobShape &S, char *a, JobDev *dj, cudaStream_t s)
{
    const size_t N = (size_t)J.W * J.H;
    CK(cudaMemcpyAsync(a + S.oW, S.wt.data(), S.wt.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(a + S.oT, S.taps.data(), S.taps.size() * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dj, &J, sizeof(JobDev), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(a + S.oMask, 0, N, s));
    const size_t n_err = J.mode == kModeHio ? (size_t)J.n_err : (size_t)J.n_cycles + 1;   // allocated length
    CK(cudaMemsetAsync(a + S.oErr, 0, n_err * 4, s));
    return IMR_SUCCESS;
}
}  // namespace imr

extern "C" {

const char *imr_status_string(int s)
{
    switch (s) {
    case IMR_SUCCESS: return "success";
    case IMR_ERR_INVALID_VALUE: return "invalid value";
    case IMR_ERR_UNSUPPORTED_SIZE: return "unsupported image size";
    case IMR_ERR_OUT_OF_MEMORY: return "out of memory";
    case IMR_ERR_CUDA: return "CUDA error";
    case IMR_ERR_NOT_INITIALIZED: return "not initialised";
    case IMR_ERR_QUEUE: return "task queue error";
    case IMR_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case IMR_ERR_CANCELLED: return "cancelled";
    default: return "unknown status";
    }
}

const char *imr_last_error(void) { return g_last_error; }

unsigned imr_max_side(void) { return kMaxSide; }

int imr_side_supported(unsigned n) { return length_supported((int)n) ? 1 : 0; }

int imr_gaussian_weights(double sigma, float *h_w, int cap)
{
    if (!(sigma > 0)) return -1;
    return gaussian_weights(sigma, h_w, cap);
}

int imr_plan_destroy(imr_plan *P)
{
    if (!P) return IMR_SUCCESS;
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->gexec_rem) cudaGraphExecDestroy(P->gexec_rem);
    if (P->graph_rem) cudaGraphDestroy(P->graph_rem);
    if (P->arena) cudaFree(P->arena);
    if (P->dbg_gprime) cudaFree(P->dbg_gprime);
    delete P;
    return IMR_SUCCESS;
}

// Capture the cycles as graphs: up to kPlanGraphCycles cycles per graph, so a
// reconstruction is one or a few graph launches (no host work between
// cycles), plus one graph for the remainder.  Replaces earlier graphs.
static int plan_capture(imr_plan *P)
{
    if (P->gexec) cudaGraphExecDestroy(P->gexec);
    if (P->graph) cudaGraphDestroy(P->graph);
    if (P->gexec_rem) cudaGraphExecDestroy(P->gexec_rem);
    if (P->graph_rem) cudaGraphDestroy(P->graph_rem);
    P->gexec = P->gexec_rem = nullptr;
    P->graph = P->graph_rem = nullptr;
    const JobDev &J = P->hj;
    P->chunk = J.n_cycles < kPlanGraphCycles ? J.n_cycles : kPlanGraphCycles;
    P->n_chunks = P->chunk ? J.n_cycles / P->chunk : 0;
    const int rem = P->chunk ? J.n_cycles % P->chunk : 0;
    int rc = IMR_SUCCESS;
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int g = 0; g < 2 && e == cudaSuccess && rc == IMR_SUCCESS; ++g) {
        const int cycles = g == 0 ? P->chunk : rem;
        if (cycles == 0) continue;
        cudaGraph_t &gr = g == 0 ? P->graph : P->graph_rem;
        cudaGraphExec_t &gx = g == 0 ? P->gexec : P->gexec_rem;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) break;
        for (int c = 0; c < cycles && rc == IMR_SUCCESS; ++c) rc = plan_launch_cycle(P, cs);
        cudaError_t e2 = cudaStreamEndCapture(cs, &gr);
        if (rc == IMR_SUCCESS && e2 == cudaSuccess)
            e = cudaGraphInstantiate(&gx, gr, 0);
        else if (e2 != cudaSuccess)
            e = e2;
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        set_error("graph capture", e);
        return rc ? rc : IMR_ERR_CUDA;
    }
    return rc;
}

int imr_plan_create(imr_plan **out, unsigned W, unsigned H, const imr_params *params)
{
    if (!out || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    *out = nullptr;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    imr_plan *P = new imr_plan();
    cudaGetDevice(&P->dev);
    P->W = (int)W;
    P->H = (int)H;
    resolve_params(params, P->p);
    JobDev &J = P->hj;
    JobShape S;
    if ((rc = job_prepare(W, H, P->p, J, S))) {
        delete P;
        return rc;
    }
    const size_t extra = (sizeof(JobState) + 255) / 256 * 256 + (sizeof(JobDev) + 255) / 256 * 256 +
                         (3 * sizeof(WorkList) + 255) / 256 * 256;
    cudaError_t e = cudaMalloc(&P->arena, S.bytes + extra);
    if (e != cudaSuccess) {
        set_error("cudaMalloc plan arena", e);
        delete P;
        return IMR_ERR_OUT_OF_MEMORY;
    }
    char *a = (char *)P->arena;
    char *tail = a + S.bytes;
    JobState *st = (JobState *)tail;
    P->dj = (JobDev *)(tail + (sizeof(JobState) + 255) / 256 * 256);
    P->Lrow = (WorkList *)((char *)P->dj + (sizeof(JobDev) + 255) / 256 * 256);
    P->Lcol = P->Lrow + 1;
    P->Lvb = P->Lrow + 2;
    job_bind(J, S, a, st);
    P->st = J.st;
    P->rk = S.rk;
    P->ck = S.ck;
    P->p_rows = S.p_rows;
    P->p_cols = S.p_cols;
    P->smem_row = S.smem_row;
    P->smem_fin = S.smem_fin;
    P->smem_col = S.smem_col;
    if (P->p_rows) {
        P->g_row_first = persistent_grid((const void *)P->rk.p_hio_first, P->rk.threads, P->rk.p_smem_first,
                                         J.n_row_tiles);
        P->g_row = persistent_grid((const void *)P->rk.p_hio, P->rk.threads, P->rk.p_smem, J.n_row_tiles);
    }
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
    const WorkList lists[3] = {{nullptr, J.n_row_tiles, 0}, {nullptr, J.n_col_tiles, n_split},
                               {nullptr, J.n_vb_tiles, 0}};
    e = cudaMemcpy(P->Lrow, lists, sizeof(lists), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = job_upload(J, S, a, P->dj, 0) ? cudaErrorUnknown : cudaSuccess;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        set_error("plan upload", e);
        imr_plan_destroy(P);
        return IMR_ERR_CUDA;
    }
    if ((rc = plan_capture(P))) {
        imr_plan_destroy(P);
        return rc;
    }
    *out = P;
    return IMR_SUCCESS;
}

int imr_plan_launches(imr_plan *P, long *launches)
{
    if (!P || !launches) return IMR_ERR_INVALID_VALUE;
    *launches = (P->hj.Mt ? 2 : 1) + (long)P->hj.n_cycles * (2 + 2L * P->hj.n_hio) + 2;
    return IMR_SUCCESS;
}

int imr_plan_execute(imr_plan *P, const float *d_modulus, float *d_out, void *stream)
{
    if (!P || !d_modulus || !d_out) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    const JobDev &J = P->hj;
    const size_t N = (size_t)P->W * P->H;
    CK(cudaMemcpyAsync((void *)J.M, d_modulus, N * 4, cudaMemcpyDeviceToDevice, s));
    if (int rc = job_modulus_tiles(J, s)) return rc;
    CK(cudaMemsetAsync(P->st, 0, sizeof(JobState), s));
    P->ck.init<<<J.n_col_tiles, P->ck.threads, P->smem_col, s>>>(P->dj, P->Lcol);
    CK(cudaGetLastError());
    for (int c = 0; c < P->n_chunks; ++c) CK(cudaGraphLaunch(P->gexec, s));
    if (P->gexec_rem) CK(cudaGraphLaunch(P->gexec_rem, s));
    if (int rc = launch_finish(P->rk, J.n_row_tiles, P->smem_fin, s, P->dj, P->Lrow, P->dbg_gprime)) return rc;
    k_vblur<<<J.n_vb_tiles, kVbThreads, 0, s>>>(P->dj, P->Lvb);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(d_out, J.out, N * 4, cudaMemcpyDeviceToDevice, s));
    return IMR_SUCCESS;
}

int imr_plan_execute_host(imr_plan *P, const float *h_modulus, float *h_out, void *stream)
{
    if (!P || !h_modulus || !h_out) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    const JobDev &J = P->hj;
    const size_t N = (size_t)P->W * P->H;
    CK(cudaMemcpyAsync((void *)J.M, h_modulus, N * 4, cudaMemcpyHostToDevice, s));
    if (int rc = job_modulus_tiles(J, s)) return rc;
    CK(cudaMemsetAsync(P->st, 0, sizeof(JobState), s));
    P->ck.init<<<J.n_col_tiles, P->ck.threads, P->smem_col, s>>>(P->dj, P->Lcol);
    CK(cudaGetLastError());
    for (int c = 0; c < P->n_chunks; ++c) CK(cudaGraphLaunch(P->gexec, s));
    if (P->gexec_rem) CK(cudaGraphLaunch(P->gexec_rem, s));
    if (int rc = launch_finish(P->rk, J.n_row_tiles, P->smem_fin, s, P->dj, P->Lrow, P->dbg_gprime)) return rc;
    k_vblur<<<J.n_vb_tiles, kVbThreads, 0, s>>>(P->dj, P->Lvb);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_out, J.out, N * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return IMR_SUCCESS;
}

int imr_plan_stats(imr_plan *P, void *stream, int *cycles_done, float *errors)
{
    if (!P) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaStreamSynchronize(s));
    JobState st;
    CK(cudaMemcpy(&st, P->st, sizeof(JobState), cudaMemcpyDeviceToHost));
    if (cycles_done) *cycles_done = st.cycles_done;
    if (st.err) {
        snprintf(g_last_error, sizeof(g_last_error), "a device-side copy wait timed out");
        return IMR_ERR_DEVICE_TIMEOUT;
    }
    if (errors) CK(cudaMemcpy(errors, P->hj.errors, sizeof(float) * P->hj.n_cycles, cudaMemcpyDeviceToHost));
    return IMR_SUCCESS;
}

int imr_plan_copy_state(imr_plan *P, int what, void *h_dst, void *stream)
{
    if (!P || !h_dst) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t N = (size_t)P->W * P->H;
    const void *src = nullptr;
    size_t bytes = 0;
    switch (what) {
    case 0: src = P->hj.mask; bytes = N; break;
    case 1: src = P->hj.X; bytes = N * 8; break;
    case 2: src = P->hj.G; bytes = N * 8; break;
    case 3: src = P->hj.vb; bytes = N * 4; break;
    default: return IMR_ERR_INVALID_VALUE;
    }
    CK(cudaMemcpyAsync(h_dst, src, bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return IMR_SUCCESS;
}

// One replay of `iters` (row pass, column pass) pairs captured into a graph;
// with `split`, an event record node after every pass (ev[0..2*iters]),
// else only before and after the pairs (ev[0], ev[1]).  External records: a
// plain record inside a capture only orders streams.
static cudaError_t profile_replay(imr_plan *P, int iters, bool split, cudaStream_t s, std::vector<cudaEvent_t> &ev)
{
    const JobDev &J = P->hj;
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    cudaGraph_t gr = nullptr;
    cudaGraphExec_t gx = nullptr;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        int k = 0;
        cudaEventRecordWithFlags(ev[k++], cs, cudaEventRecordExternal);
        for (int i = 0; i < iters; ++i) {
            if (P->p_rows)
                P->rk.p_hio<<<P->g_row, P->rk.threads, P->rk.p_smem, cs>>>(P->dj, P->Lrow);
            else
                P->rk.hio<<<J.n_row_tiles, P->rk.threads, P->smem_row, cs>>>(P->dj, P->Lrow);
            if (split) cudaEventRecordWithFlags(ev[k++], cs, cudaEventRecordExternal);
            if (P->p_cols)
                plan_col_kernel(P)<<<P->prec ? P->g_col_tc : P->g_col, P->ck.p_threads,
                                     P->prec ? P->ck.p_smem_tc : P->ck.p_smem, cs>>>(P->dj, P->Lcol);
            else
                P->ck.col<<<J.n_col_tiles, P->ck.threads, P->smem_col, cs>>>(P->dj, P->Lcol);
            if (split || i == iters - 1) cudaEventRecordWithFlags(ev[k++], cs, cudaEventRecordExternal);
        }
        const cudaError_t e2 = cudaStreamEndCapture(cs, &gr);
        e = e2 != cudaSuccess ? e2 : cudaGraphInstantiate(&gx, gr, 0);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(P->st, 0, sizeof(JobState), s);
    if (e == cudaSuccess) e = cudaGraphLaunch(gx, s);   // warm-up
    if (e == cudaSuccess) e = cudaGraphLaunch(gx, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (gx) cudaGraphExecDestroy(gx);
    if (gr) cudaGraphDestroy(gr);
    cudaStreamDestroy(cs);
    return e;
}

int imr_plan_profile(imr_plan *P, int iters, void *stream, float *ms_row, float *ms_col)
{
    if (!P || iters < 1 || !ms_row || !ms_col) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    // The pair time comes from a graph of `iters` pairs with no event inside
    // (kernel after kernel, as a reconstruction runs them: an event between
    // two kernels drains the GPU and adds that gap to the pass); its split
    // between the two passes from a replay with an event after every pass.
    std::vector<cudaEvent_t> ev(2 * iters + 1, nullptr);
    for (auto &x : ev) CK(cudaEventCreate(&x));
    cudaError_t e = profile_replay(P, iters, false, s, ev);
    float pair = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&pair, ev[0], ev[1]);
    if (e == cudaSuccess) e = profile_replay(P, iters, true, s, ev);
    double tr = 0, tc = 0;
    for (int i = 0; i < iters && e == cudaSuccess; ++i) {
        float a = 0, b = 0;
        e = cudaEventElapsedTime(&a, ev[2 * i], ev[2 * i + 1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&b, ev[2 * i + 1], ev[2 * i + 2]);
        tr += a;
        tc += b;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) {
        set_error("imr_plan_profile", e);
        return IMR_ERR_CUDA;
    }
    const double per_pair = (double)pair / iters, frac_row = tr + tc > 0 ? tr / (tr + tc) : 0.5;
    *ms_row = (float)(per_pair * frac_row);
    *ms_col = (float)(per_pair * (1.0 - frac_row));
    return IMR_SUCCESS;
}

int imr_plan_pass_bytes(imr_plan *P, double *row_bytes, double *col_bytes)
{
    if (!P || !row_bytes || !col_bytes) return IMR_ERR_INVALID_VALUE;
    const double N = (double)P->W * P->H;
    *row_bytes = 33.0 * N;
    *col_bytes = 20.0 * N;
    return IMR_SUCCESS;
}

int imr_plan_set_wait_limit(imr_plan *P, unsigned long long limit_ns)
{
    if (!P) return IMR_ERR_INVALID_VALUE;
    P->hj.wait_ns = limit_ns;
    // the captured graphs read the job description from device memory: no re-capture
    CK(cudaMemcpy(P->dj, &P->hj, sizeof(JobDev), cudaMemcpyHostToDevice));
    return IMR_SUCCESS;
}

int imr_plan_set_precision(imr_plan *P, int precision)
{
    if (!P || precision < IMR_PREC_FP32 || precision > IMR_PREC_FP16X3) return IMR_ERR_INVALID_VALUE;
    if (precision != IMR_PREC_FP32 && !(P->p_cols && P->ck.p_col_tc[precision - 1])) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "split-precision column pass: height %d is not a power of two in 256..4096 with a pipelined "
                 "column pass", P->H);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    if (precision == P->prec) return IMR_SUCCESS;
    P->prec = precision;
    if (precision != IMR_PREC_FP32)
        P->g_col_tc = persistent_grid((const void *)P->ck.p_col_tc[precision - 1], P->ck.p_threads, P->ck.p_smem_tc,
                                      P->hj.n_col_tiles);
    CK(cudaDeviceSynchronize());
    return plan_capture(P);
}

int imr_fft2d_split(void *d_data, unsigned W, unsigned H, int sign, int precision, void *stream)
{
    if (!d_data || W == 0 || H == 0 || (sign != 1 && sign != -1) || precision < IMR_PREC_BF16X3 ||
        precision > IMR_PREC_FP16X3)
        return IMR_ERR_INVALID_VALUE;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    const ColKernels ck = col_kernels((int)H);
    auto kcol = ck.fft_tc[precision - 1][sign < 0 ? 0 : 1];
    if (!kcol || W % (unsigned)ck.p_nb != 0 || ((uintptr_t)d_data & 15)) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "imr_fft2d_split: H must be a power of two in 256..4096 and W a multiple of %d", ck.p_nb);
        return IMR_ERR_UNSUPPORTED_SIZE;
    }
    FftPlanDev pr, pc;
    if ((rc = make_fft_plan((int)W, pr)) || (rc = make_fft_plan((int)H, pc))) return rc;
    JobDev J;
    memset(&J, 0, sizeof(J));
    J.W = (int)W;
    J.H = (int)H;
    J.X = (float2 *)d_data;
    J.pcol = pc;
    J.cpc = ck.p_nb;
    J.n_col_tiles = (int)W / ck.p_nb;
    if (!encode_tensor_map(&J.tmX, d_data, J.W, J.H, 8, ck.p_nb, ck.p_box_rows)) return IMR_ERR_UNSUPPORTED_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    char *dev = nullptr;
    const size_t jb = (sizeof(JobDev) + 255) / 256 * 256;
    CK(cudaMallocAsync((void **)&dev, jb + 256 + 256, s));
    JobDev *dj = (JobDev *)dev;
    WorkList *dl = (WorkList *)(dev + jb);
    JobState *dst = (JobState *)(dev + jb + 256);
    J.st = dst;
    const WorkList wl{nullptr, J.n_col_tiles};
    CK(cudaMemcpyAsync(dj, &J, sizeof(JobDev), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dl, &wl, sizeof(WorkList), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(dst, 0, sizeof(JobState), s));
    const int grid = persistent_grid((const void *)kcol, ck.p_threads, ck.p_smem_tc, J.n_col_tiles);
    if (sign < 0) {
        if ((rc = fft_passes((float2 *)d_data, (int)W, (int)H, -1, 1, pr, pc, s))) return rc;
        kcol<<<grid, ck.p_threads, ck.p_smem_tc, s>>>(dj, dl);
    } else {
        kcol<<<grid, ck.p_threads, ck.p_smem_tc, s>>>(dj, dl);
        if ((rc = fft_passes((float2 *)d_data, (int)W, (int)H, +1, 1, pr, pc, s))) return rc;
    }
    CK(cudaGetLastError());
    JobState st;
    CK(cudaMemcpyAsync(&st, dst, sizeof(JobState), cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(dev, s));
    CK(cudaStreamSynchronize(s));
    if (st.err) {
        snprintf(g_last_error, sizeof(g_last_error), "imr_fft2d_split: a device-side copy wait timed out");
        return IMR_ERR_DEVICE_TIMEOUT;
    }
    return IMR_SUCCESS;
}

int imr_bounded_wait_check(unsigned long long limit_ns, unsigned long long *elapsed_ns, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    k_wait_probe<<<1, 32, 0, s>>>(limit_ns);
    CK(cudaGetLastError());
    unsigned long long r[2] = {0, 0};
    CK(cudaMemcpyFromSymbolAsync(r, g_wait_probe, sizeof(r), 0, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (elapsed_ns) *elapsed_ns = r[1];
    if (r[0] == 0) {
        snprintf(g_last_error, sizeof(g_last_error), "bounded wait gave up after %llu ns", r[1]);
        return IMR_ERR_DEVICE_TIMEOUT;
    }
    return IMR_SUCCESS;
}

// ------------------------------------------------------------ drop-in
int imr_cuda_shrink_wrap(float *io, unsigned W, unsigned H, void *stream, unsigned nBlocks,
                         unsigned nThreads, unsigned nCycles, float targetError, float hioBeta,
                         float cutAuto, float cut, float sigma0, float sigmaChange,
                         unsigned nHio)
{
    (void)nBlocks;
    (void)nThreads;
    if (!io || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    imr_params p{nCycles, targetError, hioBeta, cutAuto, cut, sigma0, sigmaChange, nHio};
    imr_plan *P = nullptr;
    int rc = plan_cache_acquire(W, H, &p, &P);
    if (rc) return rc;
    rc = imr_plan_execute_host(P, io, io, stream);
    plan_cache_release(P);
    return rc;
}

// ------------------------------------------------------------ kernel-level
int imr_fft2d(void *d_data, unsigned W, unsigned H, int sign, void *stream)
{
    if (!d_data || W == 0 || H == 0 || (sign != 1 && sign != -1)) return IMR_ERR_INVALID_VALUE;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    FftPlanDev pr, pc;
    if ((rc = make_fft_plan((int)W, pr)) || (rc = make_fft_plan((int)H, pc))) return rc;
    return fft_passes((float2 *)d_data, (int)W, (int)H, sign, 3, pr, pc, (cudaStream_t)stream);
}

int imr_gaussian_blur(float *d_data, float *d_tmp, unsigned W, unsigned H, double sigma, int axes,
                      void *stream)
{
    if (!d_data || W == 0 || H == 0 || !(sigma > 0) || axes < 1 || axes > 3) return IMR_ERR_INVALID_VALUE;
    if ((axes & 2) && !d_tmp) return IMR_ERR_INVALID_VALUE;
    if (W > 65536 || H > 65536) return IMR_ERR_UNSUPPORTED_SIZE;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    Taps t;
    memset(&t, 0, sizeof(t));
    const int K = gaussian_weights(sigma, t.w, kMaxTaps);
    if (K > kMaxTaps) return IMR_ERR_INVALID_VALUE;
    cudaStream_t s = (cudaStream_t)stream;
    if (axes & 1) k_hblur<<<H, kRowThreads, (size_t)W * 4, s>>>(d_data, (int)W, (int)H, t, K);
    if (axes & 2) {
        const int nt = (int)(((W + kVbTileX - 1) / kVbTileX) * ((H + kVbTileY - 1) / kVbTileY));
        k_vblur_plain<<<nt, kVbThreads, 0, s>>>(d_data, d_tmp, (int)W, (int)H, t, K, nullptr);
        CK(cudaMemcpyAsync(d_data, d_tmp, (size_t)W * H * 4, cudaMemcpyDeviceToDevice, s));
    }
    CK(cudaGetLastError());
    return IMR_SUCCESS;
}

int imr_diffraction_intensity(float *h_io, unsigned W, unsigned H, void *stream)
{
    if (!h_io || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    if (!length_supported((int)W) || !length_supported((int)H)) return IMR_ERR_UNSUPPORTED_SIZE;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t N = (size_t)W * H;
    float2 *d = nullptr;
    float *f = nullptr;
    CK(cudaMallocAsync((void **)&d, N * 8, s));
    CK(cudaMallocAsync((void **)&f, N * 4, s));
    CK(cudaMemcpyAsync(f, h_io, N * 4, cudaMemcpyHostToDevice, s));
    const int g = (int)std::min<size_t>((N + 255) / 256, 148 * 16);
    k_real_to_complex<<<g, 256, 0, s>>>(f, d, (long)N);
    int rc = imr_fft2d(d, W, H, -1, stream);
    if (rc) return rc;
    k_complex_norm<<<g, 256, 0, s>>>(d, f, (long)N);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_io, f, N * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(d, s));
    CK(cudaFreeAsync(f, s));
    CK(cudaStreamSynchronize(s));
    return IMR_SUCCESS;
}

int imr_vector_max(const float *d, size_t n, float *h_max, void *stream)
{
    if (!d || !h_max) return IMR_ERR_INVALID_VALUE;
    if (n == 0) {
        *h_max = -FLT_MAX;
        return IMR_SUCCESS;
    }
    cudaStream_t s = (cudaStream_t)stream;
    unsigned *dk = nullptr;
    CK(cudaMallocAsync((void **)&dk, sizeof(unsigned), s));
    CK(cudaMemsetAsync(dk, 0, sizeof(unsigned), s));
    long blocks = (long)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_vector_max<<<(unsigned)blocks, 256, 0, s>>>(d, (long)n, dk);
    CK(cudaGetLastError());
    unsigned key = 0;
    CK(cudaMemcpyAsync(&key, dk, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CK(cudaFreeAsync(dk, s));
    CK(cudaStreamSynchronize(s));
    unsigned u = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    memcpy(h_max, &u, 4);
    return IMR_SUCCESS;
}

}  // extern "C"

// ------------------------------------------------------------ plan cache
// Idle plans keyed by (device, W, H, parameters), so repeated drop-in calls
// of one size reuse buffers and the captured graph.  Concurrent callers of
// the same size get separate plans.
namespace imr {
struct PlanKey {
    int dev;
    unsigned W, H;
    imr_params p;
    bool operator<(const PlanKey &o) const { return memcmp(this, &o, sizeof(PlanKey)) < 0; }
};
static std::mutex g_cache_mu;
static std::multimap<PlanKey, imr_plan *> g_idle;

int plan_cache_acquire(unsigned W, unsigned H, const imr_params *params, imr_plan **out)
{
    PlanKey k;
    memset(&k, 0, sizeof(k));
    cudaGetDevice(&k.dev);
    k.W = W;
    k.H = H;
    resolve_params(params, k.p);
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto it = g_idle.find(k);
        if (it != g_idle.end()) {
            *out = it->second;
            g_idle.erase(it);
            return IMR_SUCCESS;
        }
    }
    return imr_plan_create(out, W, H, &k.p);
}

void plan_cache_release(imr_plan *P)
{
    PlanKey k;
    memset(&k, 0, sizeof(k));
    k.dev = P->dev;
    k.W = (unsigned)P->W;
    k.H = (unsigned)P->H;
    k.p = P->p;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    g_idle.insert(std::make_pair(k, P));
}
}  // namespace imr
