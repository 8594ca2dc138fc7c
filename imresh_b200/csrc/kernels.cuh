// Fused kernels of the shrink-wrap / HIO engine (sm_100a).
//
// Per HIO iteration the reference runs four full-image launches
// (src/imresh/algorithms/cuda/cudaShrinkWrap.cu:311-365): the HIO domain
// constraint, a 2D forward cuFFT, the modulus projection and a 2D inverse
// cuFFT.  Here one iteration is two passes over HBM:
//   row pass    (k_row_hio):  X rows -> inverse row FFT -> g' -> HIO update
//                             with g_prev and the support mask -> g_prev :=
//                             g -> forward row FFT -> X rows
//   column pass (k_col):      X columns -> forward column FFT -> modulus
//                             projection -> inverse column FFT -> X columns
// so X holds the column-inverse-transformed iterate between iterations and
// g' = IFFT2(...) is completed by the next row pass.
//
// Once per shrink-wrap cycle:
//   k_row_finish  inverse row FFT -> g'; Re(g') -> out; |g'| -> error sums
//                 against the previous cycle's mask; |g'| blurred along rows
//   k_vblur       blur along columns, block max -> device max; the last CTA
//                 finalises the error, the stop test and the next threshold
// and the first row pass of a cycle builds the uint8 mask from the blurred
// image and the threshold.
#pragma once
#include "engine.cuh"
#include "fft_reg.cuh"
#include "tma.cuh"

namespace imr {


// Item i of a work list (a null item array means job 0, tile i).
__device__ __forceinline__ WorkItem item_at(const WorkList *L, int i)
{
    if (L->items) return L->items[i];
    return WorkItem{0, i};
}

// Kernel wrapper: the CTAs stride over the list's items, so one launch with a
// fixed grid serves any number of items (the count lives in device memory and
// may change between replays of a captured graph).
#define IMR_ITEM_LOOP(BODY_CALL)                                        \
    do {                                                                \
        const int n_items_ = L->n;                                      \
        for (int it_ = blockIdx.x; it_ < n_items_; it_ += gridDim.x) {  \
            const WorkItem wi = item_at(L, it_);                        \
            BODY_CALL;                                                  \
            __syncthreads();                                            \
        }                                                               \
    } while (0)

// ---- launch shapes ---------------------------------------------------------
// Row passes: NB rows of length N per CTA, T threads.  Column passes: NB
// columns of length N per CTA (one tile row = NB contiguous complex values),
// T threads.  N = 0 selects the runtime-length FFT.
// N < 0: Bluestein on the power-of-two length M = -N (one row per CTA;
// column tiles of 8192/M columns).
__host__ __device__ constexpr int row_nb(int N)
{
    return N == 0 ? 0 : (N < 0 ? 1 : (N % 3 == 0 ? (N <= 3072 ? 3072 / N : 1) : (N <= 2048 ? 2048 / N : 1)));
}
__host__ __device__ constexpr int row_threads(int N)
{
    return N == 0 ? kRowThreads : (N < 0 ? (-N / 8 < 64 ? 64 : -N / 8) : 256);
}
__host__ __device__ constexpr int col_nb(int N)
{
    return N == 0 ? 0
                  : (N < 0 ? (8192 / -N > 8 ? 8 : (8192 / -N < 1 ? 1 : 8192 / -N))
                           : (N % 3 == 0 ? (N <= 384 ? 16 : (6144 / N < 2 ? 2 : 6144 / N)) : (N <= 2048 ? 8 : 4)));
}
__host__ __device__ constexpr int col_len(int N) { return N < 0 ? -N : N; }
__host__ __device__ constexpr int col_threads(int N)
{
    return N == 0 ? kColThreads
                  : ((col_nb(N) * col_len(N) / 16 + 31) / 32 * 32 < 64 ? 64
                     : ((col_nb(N) * col_len(N) / 16 + 31) / 32 * 32 > 1024
                            ? 1024
                            : (col_nb(N) * col_len(N) / 16 + 31) / 32 * 32));
}

// Rows in shared memory at b*n + e; a Bluestein transform works in the
// region after the row_nb(N) rows (M complex per row).
template <int N, int S>
__device__ __forceinline__ void fft_rows(float2 *sm, int nr, const FftPlanDev &p)
{
    if constexpr (N > 0) ct_fft<N, row_nb(N), row_threads(N), S, false>(sm, nr, p.tw);
    else if constexpr (N < 0)
        bluestein<-N, 1, row_threads(N), S, false>(sm, p.n, 1, sm + (size_t)row_nb(N) * p.n, nr, p);
    else fft_smem<S, kRowVpt>(sm, p, nr, p.n, 1, false, threadIdx.x, kRowThreads);
}

// Column tiles in shared memory at e*col_nb(N) + b; a Bluestein transform
// works in the region after the tile (M * col_nb(N) complex).
template <int N, int S>
__device__ __forceinline__ void fft_cols(float2 *sm, int nc, const FftPlanDev &p)
{
    if constexpr (N > 0) ct_fft<N, col_nb(N), col_threads(N), S, true>(sm, nc, p.tw);
    else if constexpr (N < 0)
        bluestein<-N, col_nb(N), col_threads(N), S, true>(sm, 1, col_nb(N), sm + (size_t)col_nb(N) * p.n, nc,
                                                          p);
    else fft_smem<S, kColVpt>(sm, p, nc, 1, nc, true, threadIdx.x, kColThreads);
}

// |z| exactly as the reference computes it: sqrtf(re*re + im*im) with a
// separate multiply and add (vectorElementwise.cpp:52-54).
__device__ __forceinline__ float cnorm_ref(float2 z)
{
    return sqrtf(__fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y)));
}

// The modulus projection factor mod / |z| with the reference's rounding
// (cnorm_ref, then an IEEE division), |z| = 0 taken as 1 when `guard` (the
// shrink-wrap update; fixed-support HIO divides by the zero).  A zero modulus
// over a finite nonzero norm is its own quotient, so that case skips the
// square root and the division: most pixels of a measured diffraction pattern
// are zero counts (80 % of the 2048^2 benchmark pattern).
__device__ __forceinline__ float modulus_factor(float mod, float2 z, bool guard)
{
    const float ss = __fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y));
    if (mod == 0.f && ss > 0.f && ss < __int_as_float(0x7f800000)) return mod;
    float nrm = sqrtf(ss);
    if (nrm == 0.f && guard) nrm = 1.f;
    return __fdiv_rn(mod, nrm);
}

// Block-wide sum of two doubles, fixed reduction order (deterministic).
template <int NT>
__device__ __forceinline__ void block_sum2(double &a, double &b, double *scratch)
{
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        scratch[2 * warp] = a;
        scratch[2 * warp + 1] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0, sb = 0;
        for (int w = 0; w < NT / 32; ++w) {
            sa += scratch[2 * w];
            sb += scratch[2 * w + 1];
        }
        a = sa;
        b = sb;
    }
    __syncthreads();
}

// Fixed-support HIO (libs::hybridInputOutput, src/imresh/libs/hybridInputOutput.cpp:237-292):
// every row pass makes g'_k.  Each tile's sums (sum mask*|g'|, sum mask) are
// stored per tile; the CTA that completes the job's last tile of the pass
// forms E_k = sqrt(sum)/count (calculateHioError, cpp:67-103, summed in double
// in a fixed order), applies the stop tests E_k < target (cpp:251-254) and
// k == nCycles (cpp:255-256), and moves the job to iteration k + 1.
template <int T>
__device__ __forceinline__ void hio_tile_done(const JobDev &J, int tile, double tot, double cnt)
{
    __shared__ double red[2 * (T / 32 > 1 ? T / 32 : 1)];
    __shared__ int s_last;
    JobState *st = J.st;
    block_sum2<T>(tot, cnt, red);
    if (threadIdx.x == 0) {
        J.err_part[2 * tile] = tot;
        J.err_part[2 * tile + 1] = cnt;
        __threadfence();
        s_last = atomicAdd(&st->counter, 1u) == (unsigned)J.n_row_tiles - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    tot = 0.0;
    cnt = 0.0;
    const volatile double *ep = J.err_part;
    for (int t = threadIdx.x; t < J.n_row_tiles; t += T) {
        tot += ep[2 * t];
        cnt += ep[2 * t + 1];
    }
    block_sum2<T>(tot, cnt, red);
    if (threadIdx.x == 0) {
        const int k = st->cycle;
        int stop = k >= J.n_cycles;
        if (J.target > 0.f || stop) {
            const float E = (float)(sqrt(tot) / cnt);
            st->last_error = E;
            if (k < J.n_err) J.errors[k] = E;
            if (J.target > 0.f && E < J.target) stop = 1;
        }
        st->cycles_done = k;
        st->cycle = k + 1;
        st->counter = 0u;
        if (stop) st->stop = 1;
        __threadfence();
    }
}

// Per-element part of the fixed-support HIO row pass: error terms of g' and
// out = Re(g') when this iteration is tested (or is the last).
__device__ __forceinline__ void hio_track(float *out, size_t idx, float2 gp1, uint8_t m, double &tot, double &cnt)
{
    if (m) {
        tot += (double)m * (double)cnorm_ref(gp1);
        cnt += (double)m;
    }
    out[idx] = gp1.x;
}

template <int NT>
__device__ __forceinline__ float block_max(float v, float *scratch)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    float r = v;
    if (threadIdx.x == 0) {
        r = scratch[0];
        for (int w = 1; w < NT / 32; ++w) r = fmaxf(r, scratch[w]);
    }
    __syncthreads();
    return r;
}

// Horizontal clamp-border convolution of nr rows of length W held in shared
// memory, tap order k = 0..K-1 as in applyKernel (src/imresh/libs/gaussian.cpp:139-148).
__device__ __forceinline__ float hblur_at(const float *row, int W, int x, const float *w, int K)
{
    const int N = (K - 1) / 2;
    float sum = 0.f;
    for (int k = 0; k < K; ++k) {
        int xs = x - N + k;
        xs = xs < 0 ? 0 : (xs > W - 1 ? W - 1 : xs);
        sum = __fadd_rn(sum, __fmul_rn(row[xs], w[k]));
    }
    return sum;
}

// Vertical clamp-border convolution of a kVbTileY x kVbTileX tile of src
// (row-major [H][W]) into dst; returns the tile's max of the outputs.
// Tap order k = -N..N as in gaussianBlurVertical (src/imresh/libs/gaussian.cpp:706-712).
__device__ __forceinline__ float vblur_tile(const float *src, float *dst, int W, int H, int x0,
                                            int y0, const float *w, int K, float *tile)
{
    const int N = (K - 1) / 2;
    const int rows_in = kVbTileY + 2 * N;
    const int tx = threadIdx.x & (kVbTileX - 1);
    const int ty = threadIdx.x / kVbTileX;
    const int x = x0 + tx;
    // all of a thread's tile rows are requested before any is stored, so the
    // loads' latencies overlap (rows_in <= kVbTileY + 62 for K <= 63 taps)
    constexpr int RS0 = kVbThreads / kVbTileX, NLD = (kVbTileY + 62 + RS0 - 1) / RS0;
    float ld[NLD];
#pragma unroll
    for (int i = 0; i < NLD; ++i) {
        const int r = ty + i * RS0;
        int ys = y0 - N + r;
        ys = ys < 0 ? 0 : (ys > H - 1 ? H - 1 : ys);
        ld[i] = r < rows_in && x < W ? __ldg(src + (size_t)ys * W + x) : 0.f;
    }
#pragma unroll
    for (int i = 0; i < NLD; ++i) {
        const int r = ty + i * RS0;
        if (r < rows_in) tile[r * kVbTileX + tx] = ld[i];
    }
    __syncthreads();
    // RPT outputs per thread, accumulated side by side (independent chains);
    // each output still sums its taps in order k = 0..K-1
    constexpr int RS = kVbThreads / kVbTileX, RPT = kVbTileY / RS;
    float sum[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) sum[j] = 0.f;
    for (int k = 0; k < K; ++k) {
        const float wk = w[k];
#pragma unroll
        for (int j = 0; j < RPT; ++j) sum[j] = __fadd_rn(sum[j], __fmul_rn(tile[(ty + j * RS + k) * kVbTileX + tx], wk));
    }
    float mx = 0.f;
    if (x < W) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int y = y0 + ty + j * RS;
            if (y < H) {
                dst[(size_t)y * W + x] = sum[j];
                mx = fmaxf(mx, sum[j]);
            }
        }
    }
    return mx;
}

// ---------------------------------------------------------------- init
// X := inverse column FFT of (M, 0): the column half of g'_0 = IFFT2(M)
// (cudaShrinkWrap.cu:229-232: CopyToRealPart then an in-place inverse FFT).
template <int N>
__device__ __forceinline__ void b_col_init(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const JobDev &J = jobs[wi.job];
    const int W = J.W, H = J.H;
    const int x0 = wi.tile * J.cpc;
    const int nc = min(J.cpc, W - x0);
    constexpr int T = col_threads(N);
    const int es = N != 0 ? col_nb(N) : nc;   // smem row stride of the tile
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        sm[y * es + c] = make_float2(J.M[(size_t)y * W + x0 + c], 0.f);
    }
    __syncthreads();
    fft_cols<N, +1>(sm, nc, J.pcol);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        J.X[(size_t)y * W + x0 + c] = sm[y * es + c];
    }
}
template <int N>
__global__ void __launch_bounds__(col_threads(N)) k_col_init(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col_init<N>(jobs, wi)));
}

// ---------------------------------------------------------------- column pass
// Forward column FFT, G <- G * M/|G| (|G| = 0 -> 1; applyComplexModulus,
// src/imresh/algorithms/cuda/cudaVectorElementwise.cu:168-195), inverse
// column FFT.  Fixed-support HIO jobs divide without the |G| = 0 guard, as
// libs::hybridInputOutput does (src/imresh/libs/hybridInputOutput.cpp:281-289).
template <int N>
__device__ __forceinline__ void b_col(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const JobDev &J = jobs[wi.job];
    if (J.st->stop) return;
    const int W = J.W, H = J.H;
    const int x0 = wi.tile * J.cpc;
    const int nc = min(J.cpc, W - x0);
    constexpr int T = col_threads(N);
    const int es = N != 0 ? col_nb(N) : nc;
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        sm[y * es + c] = J.X[(size_t)y * W + x0 + c];
    }
    __syncthreads();
    fft_cols<N, -1>(sm, nc, J.pcol);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        const float2 g = sm[y * es + c];
        const float f = modulus_factor(J.M[(size_t)y * W + x0 + c], g, J.mode == kModeShrinkWrap);
        sm[y * es + c] = make_float2(__fmul_rn(g.x, f), __fmul_rn(g.y, f));
    }
    __syncthreads();
    fft_cols<N, +1>(sm, nc, J.pcol);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        J.X[(size_t)y * W + x0 + c] = sm[y * es + c];
    }
}
template <int N>
__global__ void __launch_bounds__(col_threads(N)) k_col(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col<N>(jobs, wi)));
}

// ---------------------------------------------------------------- row pass
// Inverse row FFT -> g'; HIO domain constraint
//   if mask == 1 or Re(g') < 0:  g = g_prev - beta*g'  else  g = g'
// (cudaKernelApplyHioDomainConstraints, cudaVectorElementwise.cu:42-72);
// g_prev := g; forward row FFT of g -> X.
// FIRST: first iteration of a cycle -- builds the uint8 mask from the blurred
// image (mask = blurred < threshold, cudaKernelCutOff, cudaVectorElementwise.cu:198-219)
// and, on cycle 0, takes g_prev = g'_0 (cudaShrinkWrap.cu:304-309).
// FIX: fixed-support HIO of libs::hybridInputOutput -- the caller's mask
// (HIO where mask == 1, error weight = mask value, hybridInputOutput.cpp:262-269),
// g_prev = g'_0 on iteration 0 (cpp:245-246), error terms and out = Re(g')
// on every tested iteration, no update on the last one (hio_tile_done).
template <bool FIRST, int N, bool FIX = false>
__device__ __forceinline__ void b_row_hio(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int W = J.W, H = J.H;
    const int y0 = wi.tile * J.rpc;
    const int nr = min(J.rpc, H - y0);
    const int n = nr * W;
    const size_t base = (size_t)y0 * W;
    constexpr int T = row_threads(N);
    for (int i = threadIdx.x; i < n; i += T) sm[i] = J.X[base + i];
    __syncthreads();
    fft_rows<N, +1>(sm, nr, J.prow);
    const float beta = J.beta;
    const float thr = st->thr;
    const int k = FIX ? st->cycle : 0;
    const bool init_gprev = FIX ? k == 0 : FIRST && st->hio_cycle == 0;
    const bool fin = FIX && k >= J.n_cycles;
    const bool track = FIX && (J.target > 0.f || fin);
    double tot = 0.0, cnt = 0.0;
    for (int i = threadIdx.x; i < n; i += T) {
        const size_t idx = base + i;
        const float2 gp1 = sm[i];   // g'
        uint8_t m;
        if (FIRST) {
            m = J.vb[idx] < thr ? 1 : 0;
            J.mask[idx] = m;
        } else {
            m = J.mask[idx];
        }
        if (FIX) {
            if (track) hio_track(J.out, idx, gp1, m, tot, cnt);
            if (fin) continue;
        }
        const float2 gp = init_gprev ? gp1 : J.G[idx];
        float2 g;
        if ((FIX ? m == 1 : m != 0) || gp1.x < 0.f)
            g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)),
                            __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
        else
            g = gp1;
        J.G[idx] = g;
        sm[i] = g;
    }
    if (!fin) {
        __syncthreads();
        fft_rows<N, -1>(sm, nr, J.prow);
        for (int i = threadIdx.x; i < n; i += T) J.X[base + i] = sm[i];
    }
    if (FIX) hio_tile_done<T>(J, wi.tile, tot, cnt);
}
template <bool FIRST, int N, bool FIX = false>
__global__ void __launch_bounds__(row_threads(N)) k_row_hio(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_row_hio<FIRST, N, FIX>(jobs, wi)));
}

// Once per cycle: inverse row FFT -> g'; out = Re(g') (CopyFromRealPart,
// cudaVectorElementwise.cu:98-117); error sums against the previous cycle's
// mask (cudaKernelCalculateHioError, cudaVectorReduce.cu:284-355, summed in
// double here); |g'| (cudaKernelComplexNormElementwise) blurred along rows.
template <int N>
__device__ __forceinline__ void b_row_finish(const JobDev *jobs, const WorkItem wi, float2 *dbg_gprime)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int T = row_threads(N);
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32];
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int c = st->cycle;
    if (wi.tile == 0 && threadIdx.x == 0) st->max_bits = 0u;
    const int W = J.W, H = J.H;
    const int y0 = wi.tile * J.rpc;
    const int nr = min(J.rpc, H - y0);
    const int n = nr * W;
    const size_t base = (size_t)y0 * W;
    float *nrm = reinterpret_cast<float *>(sm + J.rpc * W);
    const int K = J.ntaps[c];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
    for (int i = threadIdx.x; i < n; i += T) sm[i] = J.X[base + i];
    __syncthreads();
    fft_rows<N, +1>(sm, nr, J.prow);
    double tot = 0.0, cnt = 0.0;
    for (int i = threadIdx.x; i < n; i += T) {
        const size_t idx = base + i;
        const float2 g = sm[i];
        J.out[idx] = g.x;
        if (dbg_gprime) dbg_gprime[idx] = g;
        const float v = cnorm_ref(g);
        nrm[i] = v;
        if (c > 0 && J.mask[idx]) {
            tot += (double)v;
            cnt += 1.0;
        }
    }
    block_sum2<T>(tot, cnt, red);   // includes __syncthreads
    if (threadIdx.x == 0) {
        J.err_part[2 * wi.tile] = tot;
        J.err_part[2 * wi.tile + 1] = cnt;
    }
    for (int i = threadIdx.x; i < n; i += T) {
        const int r = i / W, x = i - r * W;
        J.hb[base + i] = hblur_at(nrm + r * W, W, x, wsm, K);
    }
}
template <int N>
__global__ void __launch_bounds__(row_threads(N)) k_row_finish(const JobDev *jobs, const WorkList *L, float2 *dbg_gprime)
{
    IMR_ITEM_LOOP((b_row_finish<N>(jobs, wi, dbg_gprime)));
}

// Once per cycle: vertical blur hb -> vb and the global max; the last CTA
// of the job finalises the cycle: error E = sqrt(sum mask*|g'|)/sum mask of
// the previous cycle (cudaVectorReduce.cu:357-403) and the stop test
// E < target (cudaShrinkWrap.cu:374-375), then the threshold
// (cycle 0 ? cutOffAutoCorel : cutOff) * max (cudaShrinkWrap.cu:274-276).
__device__ __forceinline__ void b_vblur(const JobDev *jobs, const WorkItem wi)
{
    __shared__ float tile[(kVbTileY + 2 * 31) * kVbTileX];
    __shared__ float wsm[kTapStride];
    __shared__ float fred[kVbThreads / 32];
    __shared__ double red[2 * kVbThreads / 32];
    __shared__ int s_last;
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int c = st->cycle;
    const int K = J.ntaps[c];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
    const int tx = wi.tile % J.vb_tiles_x, ty = wi.tile / J.vb_tiles_x;
    __syncthreads();
    float mx = vblur_tile(J.hb, J.vb, J.W, J.H, tx * kVbTileX, ty * kVbTileY, wsm, K, tile);
    mx = block_max<kVbThreads>(mx, fred);
    if (threadIdx.x == 0) {
        atomicMax(&st->max_bits, __float_as_uint(mx));
        __threadfence();
        const unsigned prev = atomicAdd(&st->counter, 1u);
        s_last = (prev == (unsigned)J.n_vb_tiles - 1u);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double tot = 0.0, cnt = 0.0;
    const volatile double *ep = J.err_part;
    for (int t = threadIdx.x; t < J.n_row_tiles; t += kVbThreads) {
        tot += ep[2 * t];
        cnt += ep[2 * t + 1];
    }
    block_sum2<kVbThreads>(tot, cnt, red);
    if (threadIdx.x == 0) {
        int stop = 0;
        if (c > 0) {
            const float E = (float)(sqrt(tot) / cnt);
            J.errors[c - 1] = E;
            st->last_error = E;
            st->cycles_done = c;
            if (J.target > 0.f && E < J.target) stop = 1;
        }
        if (c >= J.n_cycles) stop = 1;
        const float gmax = __uint_as_float(atomicAdd(&st->max_bits, 0u));
        st->thr = (c == 0 ? J.cut_auto : J.cut) * gmax;
        st->hio_cycle = c;
        st->cycle = c + 1;
        st->counter = 0u;
        if (stop) st->stop = 1;
        __threadfence();
    }
}
static __global__ void __launch_bounds__(kVbThreads) k_vblur(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_vblur(jobs, wi)));
}

// ---------------------------------------------------------------- plain FFT
// Stand-alone 2D transform passes (used by the kernel-level API and tests).
template <int S, int N>
__global__ void __launch_bounds__(row_threads(N)) k_fft_rows(float2 *data, FftPlanDev p, int H, int rpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int T = row_threads(N);
    const int W = p.n;
    const int y0 = blockIdx.x * rpc;
    const int nr = min(rpc, H - y0);
    const int n = nr * W;
    const size_t base = (size_t)y0 * W;
    for (int i = threadIdx.x; i < n; i += T) sm[i] = data[base + i];
    __syncthreads();
    fft_rows<N, S>(sm, nr, p);
    for (int i = threadIdx.x; i < n; i += T) data[base + i] = sm[i];
}

template <int S, int N>
__global__ void __launch_bounds__(col_threads(N)) k_fft_cols(float2 *data, FftPlanDev p, int W, int cpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int T = col_threads(N);
    const int H = p.n;
    const int x0 = blockIdx.x * cpc;
    const int nc = min(cpc, W - x0);
    const int es = N != 0 ? col_nb(N) : nc;
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        sm[y * es + c] = data[(size_t)y * W + x0 + c];
    }
    __syncthreads();
    fft_cols<N, S>(sm, nc, p);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        data[(size_t)y * W + x0 + c] = sm[y * es + c];
    }
}

// Stand-alone separable blur (kernel-level API): rows in place, then columns.
struct Taps {
    float w[kTapStride];
};

static __global__ void __launch_bounds__(kRowThreads) k_hblur(float *data, int W, int H, Taps w, int K)
{
    extern __shared__ float4 smem4[];
    float *row = reinterpret_cast<float *>(smem4);
    __shared__ float wsm[kTapStride];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = w.w[threadIdx.x];
    const size_t base = (size_t)blockIdx.x * W;
    for (int x = threadIdx.x; x < W; x += kRowThreads) row[x] = data[base + x];
    __syncthreads();
    for (int x = threadIdx.x; x < W; x += kRowThreads) data[base + x] = hblur_at(row, W, x, wsm, K);
}

static __global__ void __launch_bounds__(kVbThreads) k_vblur_plain(const float *src, float *dst, int W, int H,
                                                           Taps w, int K, unsigned *max_bits)
{
    __shared__ float tile[(kVbTileY + 2 * 31) * kVbTileX];
    __shared__ float wsm[kTapStride];
    __shared__ float fred[kVbThreads / 32];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = w.w[threadIdx.x];
    __syncthreads();
    const int tiles_x = (W + kVbTileX - 1) / kVbTileX;
    const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    float mx = vblur_tile(src, dst, W, H, tx * kVbTileX, ty * kVbTileY, wsm, K, tile);
    mx = block_max<kVbThreads>(mx, fred);
    if (threadIdx.x == 0 && max_bits) atomicMax(max_bits, __float_as_uint(mx));
}

// (x, 0) <-> |z| helpers of the forward model
static __global__ void k_real_to_complex(const float *src, float2 *dst, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = make_float2(src[i], 0.f);
}
static __global__ void k_complex_norm(const float2 *src, float *dst, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = cnorm_ref(src[i]);
}

// ---------------------------------------------------------------- random phase
// The C library's rand() stream as libs::addRandomPhase draws it after
// srand(2623091912) (src/imresh/libs/hybridInputOutput.cpp:160-167): glibc's
// additive feedback generator, r[i] = r[i-31] + r[i-3] (mod 2^32) for i >= 34,
// rand() number k = r[k + 344] >> 1.  Thread c makes the numbers
// [c*kRandChunk, (c+1)*kRandChunk): its 31-word state (r[i-31..i-1]) starts
// from the base state at i = 344 and jumps by B^c, B = A^kRandChunk the
// recurrence's 31x31 step matrix over Z/2^32 raised to the chunk length,
// composed from the table pow[j] = B^(2^j); then it runs the recurrence.
// Element k of X becomes ((float)rand_k / RAND_MAX, 0) (cpp:163-167).
constexpr int kRandLag = 31;
constexpr int kRandChunk = 31 * 32;
constexpr int kRandThreads = 128;
struct RandBase {
    uint32_t s[kRandLag];
};
static __global__ void __launch_bounds__(kRandThreads) k_rand_field(float2 *X, long n, RandBase base,
                                                                    const uint32_t *pow, int n_pow)
{
    __shared__ uint32_t P[kRandLag * kRandLag];
    const long c = (long)blockIdx.x * kRandThreads + threadIdx.x;
    uint32_t s[kRandLag];
#pragma unroll
    for (int i = 0; i < kRandLag; ++i) s[i] = base.s[i];
    for (int j = 0; j < n_pow; ++j) {
        __syncthreads();
        for (int i = threadIdx.x; i < kRandLag * kRandLag; i += kRandThreads)
            P[i] = pow[(size_t)j * kRandLag * kRandLag + i];
        __syncthreads();
        if ((c >> j) & 1) {
            uint32_t t[kRandLag];
#pragma unroll
            for (int i = 0; i < kRandLag; ++i) {
                uint32_t a = 0;
#pragma unroll
                for (int m = 0; m < kRandLag; ++m) a += P[i * kRandLag + m] * s[m];
                t[i] = a;
            }
#pragma unroll
            for (int i = 0; i < kRandLag; ++i) s[i] = t[i];
        }
    }
    const long k0 = c * kRandChunk;
    if (k0 >= n) return;
    const long kend = min(n, k0 + kRandChunk);
    for (int o = 0; o < kRandChunk / kRandLag; ++o) {
#pragma unroll
        for (int q = 0; q < kRandLag; ++q) {
            const uint32_t r = s[q] + s[(q + kRandLag - 3) % kRandLag];   // r[i-31] + r[i-3]
            s[q] = r;
            const long k = k0 + (long)o * kRandLag + q;
            if (k < kend) X[k] = make_float2(__fdiv_rn((float)(int)(r >> 1), 2147483648.0f), 0.f);
        }
    }
}

// X = M * (cos phase, sin phase), phase = arg(X) of the transformed random
// field (addRandomPhase, hybridInputOutput.cpp:170-180).  The reference's
// unqualified cos/sin of a float resolve to the double functions, so the
// products are formed in double and rounded to float, as there.
static __global__ void k_random_phase(float2 *X, const float *M, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float2 z = X[i];
        const float ph = atan2f(z.y, z.x);
        double sn, cs;
        sincos((double)ph, &sn, &cs);
        const double m = (double)M[i];
        X[i] = make_float2((float)(m * cs), (float)(m * sn));
    }
}

// cudaCalculateHioError (src/imresh/algorithms/cuda/cudaVectorReduce.cu:284-403):
// sums of w*|z| and of w, w = (mask != 0) xor invert.  Block sums in double;
// the last block folds them in block order (deterministic) into res[0..1].
template <class TM>
static __global__ void __launch_bounds__(256) k_hio_error(const float2 *d, const TM *mask, long n, int invert,
                                                          double *part, unsigned *counter, double *res)
{
    __shared__ double red[16];
    __shared__ int s_last;
    double tot = 0.0, cnt = 0.0;
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
        const bool w = (mask[i] != TM(0)) != (invert != 0);
        if (w) {
            tot += (double)cnorm_ref(d[i]);
            cnt += 1.0;
        }
    }
    block_sum2<256>(tot, cnt, red);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = tot;
        part[2 * blockIdx.x + 1] = cnt;
        __threadfence();
        s_last = atomicAdd(counter, 1u) == gridDim.x - 1u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    tot = 0.0;
    cnt = 0.0;
    const volatile double *vp = part;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 256) {
        tot += vp[2 * b];
        cnt += vp[2 * b + 1];
    }
    block_sum2<256>(tot, cnt, red);
    if (threadIdx.x == 0) {
        res[0] = tot;
        res[1] = cnt;
        *counter = 0u;
    }
}

// Self-check of the bounded wait every pipelined pass relies on: one thread
// waits on an mbarrier whose transaction nothing will complete (an expected
// 16 bytes that no copy delivers), so the wait must give up after limit_ns
// and report it; no copy is in flight, so returning is safe.
// g_wait_probe = {completed (1) or gave up (0), nanoseconds waited}.
static __device__ unsigned long long g_wait_probe[2];
static __global__ void k_wait_probe(unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_fence_init();
    mbar_arrive_expect_tx(&bar, 16u);
    const uint64_t t0 = global_ns();
    const bool ok = mbar_wait(&bar, 0u, limit_ns);
    g_wait_probe[1] = global_ns() - t0;
    g_wait_probe[0] = ok ? 1ull : 0ull;
    mbar_inval(&bar);
}

// Global max of a float array (vectorMax; cudaVectorReduce.cu:229-239):
// signed floats ordered through an order-preserving integer key.
__device__ __forceinline__ unsigned f2key(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
static __global__ void __launch_bounds__(256) k_vector_max(const float *d, long n, unsigned *key)
{
    __shared__ unsigned s[8];
    unsigned m = 0u;   // key of the lowest value
    for (long i = blockIdx.x * 256L + threadIdx.x; i < n; i += (long)gridDim.x * 256L) {
        unsigned k = f2key(d[i]);
        m = k > m ? k : m;
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) m = max(m, s[w]);
        atomicMax(key, m);
    }
}

}  // namespace imr

// ============================================================================
// Power-of-two lengths: the same passes on the register-resident FFT
// (fft_reg.cuh).  Thread (b, l) owns positions l + m*N/8 of sequence b.
// ============================================================================
namespace imr {

// power-of-two lengths (8 values per thread); 3 * 2^k lengths (12 values per
// thread) share their tile shapes with the per-tile kernels (row_nb, col_nb)
__host__ __device__ constexpr int rrow_nb(int N) { return N % 3 == 0 ? row_nb(N) : (N <= 2048 ? 2048 / N : 1); }
__host__ __device__ constexpr int rrow_threads(int N) { return rrow_nb(N) * N / reg_v(N); }
__host__ __device__ constexpr int rcol_nb(int N)
{
    return N % 3 == 0 ? col_nb(N) : (N <= 1024 ? (8192 / N < 16 ? 8192 / N : 16) : (N == 2048 ? 4 : 2));
}
__host__ __device__ constexpr int rcol_threads(int N) { return rcol_nb(N) * N / reg_v(N); }
__host__ __device__ constexpr int rrow_smem(int N) { return reg_smem_bytes(N, rrow_nb(N)); }
__host__ __device__ constexpr int rcol_smem(int N) { return reg_smem_bytes(N, rcol_nb(N)); }

// X := inverse column FFT of (M, 0)
template <int N>
__device__ __forceinline__ void b_col_init_r(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(N), Q = N / 8;
    const JobDev &J = jobs[wi.job];
    const int W = J.W;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = wi.tile * J.cpc + b;
    const bool ok = b < J.cpc && x < W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m)
        v[m] = make_float2(ok ? J.M[(size_t)(l + m * Q) * W + x] : 0.f, 0.f);
    reg_fft<N, NB, true, +1>(v, sm, b, l, J.pcol.tw);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) J.X[(size_t)(l + m * Q) * W + x] = v[m];
    }
}
template <int N>
__global__ void __launch_bounds__(rcol_threads(N)) k_col_init_r(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col_init_r<N>(jobs, wi)));
}

// column pass: forward column FFT, modulus projection, inverse column FFT
template <int N>
__device__ __forceinline__ void b_col_r(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(N), Q = N / 8;
    const JobDev &J = jobs[wi.job];
    if (J.st->stop) return;
    const int W = J.W;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = wi.tile * J.cpc + b;
    const bool ok = b < J.cpc && x < W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? J.X[(size_t)(l + m * Q) * W + x] : make_float2(0.f, 0.f);
    reg_fft<N, NB, true, -1>(v, sm, b, l, J.pcol.tw);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const float mod = ok ? J.M[(size_t)(l + m * Q) * W + x] : 0.f;
        const float f = modulus_factor(mod, v[m], J.mode == kModeShrinkWrap);
        v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
    }
    reg_fft<N, NB, true, +1>(v, sm, b, l, J.pcol.tw);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) J.X[(size_t)(l + m * Q) * W + x] = v[m];
    }
}
template <int N>
__global__ void __launch_bounds__(rcol_threads(N)) k_col_r(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col_r<N>(jobs, wi)));
}

// row pass: inverse row FFT, HIO update, forward row FFT (see k_row_hio)
template <bool FIRST, int N, bool FIX = false>
__device__ __forceinline__ void b_row_hio_r(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = N / 8;
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = wi.tile * J.rpc + b;
    const bool ok = b < J.rpc && y < J.H;
    const size_t base = (size_t)y * N;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? J.X[base + l + m * Q] : make_float2(0.f, 0.f);
    reg_fft<N, rrow_nb(N), false, +1>(v, sm, b, l, J.prow.tw);
    const float beta = J.beta;
    const float thr = st->thr;
    const int k = FIX ? st->cycle : 0;
    const bool init_gprev = FIX ? k == 0 : FIRST && st->hio_cycle == 0;
    const bool fin = FIX && k >= J.n_cycles;
    const bool track = FIX && (J.target > 0.f || fin);
    double tot = 0.0, cnt = 0.0;
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const size_t idx = base + l + m * Q;
            const float2 gp1 = v[m];
            uint8_t msk;
            if (FIRST) {
                msk = J.vb[idx] < thr ? 1 : 0;
                J.mask[idx] = msk;
            } else {
                msk = J.mask[idx];
            }
            if (FIX && track) hio_track(J.out, idx, gp1, msk, tot, cnt);
            if (fin) continue;
            const float2 gp = init_gprev ? gp1 : J.G[idx];
            float2 g;
            if ((FIX ? msk == 1 : msk != 0) || gp1.x < 0.f)
                g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)),
                                __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
            else
                g = gp1;
            J.G[idx] = g;
            v[m] = g;
        }
    }
    if (!fin) {
        reg_fft<N, rrow_nb(N), false, -1>(v, sm, b, l, J.prow.tw);
        if (ok) {
#pragma unroll
            for (int m = 0; m < 8; ++m) J.X[base + l + m * Q] = v[m];
        }
    }
    if (FIX) hio_tile_done<rrow_threads(N)>(J, wi.tile, tot, cnt);
}
template <bool FIRST, int N, bool FIX = false>
__global__ void __launch_bounds__(rrow_threads(N)) k_row_hio_r(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_row_hio_r<FIRST, N, FIX>(jobs, wi)));
}

// once per cycle: inverse row FFT -> g'; out, error sums, |g'| blurred along rows
template <int N>
__device__ __forceinline__ void b_row_finish_r(const JobDev *jobs, const WorkItem wi, float2 *dbg_gprime)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int T = rrow_threads(N), Q = N / 8;
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32 > 2 ? 2 * T / 32 : 2];
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int c = st->cycle;
    if (wi.tile == 0 && threadIdx.x == 0) st->max_bits = 0u;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = wi.tile * J.rpc + b;
    const bool ok = b < J.rpc && y < J.H;
    const size_t base = (size_t)y * N;
    const int K = J.ntaps[c];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? J.X[base + l + m * Q] : make_float2(0.f, 0.f);
    reg_fft<N, rrow_nb(N), false, +1>(v, sm, b, l, J.prow.tw);
    float *nrow = reinterpret_cast<float *>(sm) + b * N;   // buffers are free after reg_fft
    double tot = 0.0, cnt = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int e = l + m * Q;
        const float nv = cnorm_ref(v[m]);
        nrow[e] = nv;
        if (ok) {
            const size_t idx = base + e;
            J.out[idx] = v[m].x;
            if (dbg_gprime) dbg_gprime[idx] = v[m];
            if (c > 0 && J.mask[idx]) {
                tot += (double)nv;
                cnt += 1.0;
            }
        }
    }
    block_sum2<T>(tot, cnt, red);   // includes barriers: nrow complete after it
    if (threadIdx.x == 0) {
        J.err_part[2 * wi.tile] = tot;
        J.err_part[2 * wi.tile + 1] = cnt;
    }
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int e = l + m * Q;
            J.hb[base + e] = hblur_at(nrow, N, e, wsm, K);
        }
    }
}
template <int N>
__global__ void __launch_bounds__(rrow_threads(N)) k_row_finish_r(const JobDev *jobs, const WorkList *L, float2 *dbg_gprime)
{
    IMR_ITEM_LOOP((b_row_finish_r<N>(jobs, wi, dbg_gprime)));
}

// plain 2D transform passes
template <int S, int N>
__global__ void __launch_bounds__(rrow_threads(N)) k_fft_rows_r(float2 *data, FftPlanDev p, int H, int rpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = N / 8;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = blockIdx.x * rpc + b;
    const bool ok = b < rpc && y < H;
    const size_t base = (size_t)y * N;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? data[base + l + m * Q] : make_float2(0.f, 0.f);
    reg_fft<N, rrow_nb(N), false, S>(v, sm, b, l, p.tw);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) data[base + l + m * Q] = v[m];
    }
}

template <int S, int N>
__global__ void __launch_bounds__(rcol_threads(N)) k_fft_cols_r(float2 *data, FftPlanDev p, int W, int cpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(N), Q = N / 8;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = blockIdx.x * cpc + b;
    const bool ok = b < cpc && x < W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = ok ? data[(size_t)(l + m * Q) * W + x] : make_float2(0.f, 0.f);
    reg_fft<N, NB, true, S>(v, sm, b, l, p.tw);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) data[(size_t)(l + m * Q) * W + x] = v[m];
    }
}

// ---------------------------------------------------------------- Bluestein, in registers
// Lengths n with a prime factor > 7 run Bluestein's chirp-z transform on the
// power-of-two work length M >= 2n - 1 (x_j c_j, c the chirp -- conjugated
// for inverse transforms -- zero-padded to M; FFT_M; times the kernel
// spectrum; inverse FFT_M; times c_j).  Here the whole chain stays in
// registers at the positions j = l + m*M/8 of the register FFT, so a row pass
// keeps g' in registers from the inverse transform through the HIO update to
// the forward transform, as for power-of-two lengths.  Positions j >= n carry
// nothing on output.
template <int M, int NB, bool COLS, int S>
__device__ __forceinline__ void reg_bluestein(float2 (&v)[8], float2 *sm, int b, int l, const FftPlanDev &p)
{
    constexpr int Q = M / 8;
    const int n = p.n;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        if (j < n) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            v[m] = cmul(v[m], c);
        } else {
            v[m] = make_float2(0.f, 0.f);
        }
    }
    reg_fft<M, NB, COLS, -1>(v, sm, b, l, p.tw);
    const float2 *spec = S < 0 ? p.bspec_f : p.bspec_b;
#pragma unroll
    for (int m = 0; m < 8; ++m) v[m] = cmul(v[m], __ldg(spec + l + m * Q));
    reg_fft<M, NB, COLS, +1>(v, sm, b, l, p.tw);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        if (j < n) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            v[m] = cmul(v[m], c);
        }
    }
}

// row pass (see k_row_hio) on Bluestein row lengths: NB rows of length W per CTA
template <bool FIRST, int M, bool FIX = false>
__device__ __forceinline__ void b_row_hio_bs(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rrow_nb(M), Q = M / 8;
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int W = J.W;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = wi.tile * J.rpc + b;
    const bool ok = b < J.rpc && y < J.H;
    const size_t base = (size_t)y * W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < W ? J.X[base + j] : make_float2(0.f, 0.f);
    }
    reg_bluestein<M, NB, false, +1>(v, sm, b, l, J.prow);
    const float beta = J.beta;
    const float thr = st->thr;
    const int k = FIX ? st->cycle : 0;
    const bool init_gprev = FIX ? k == 0 : FIRST && st->hio_cycle == 0;
    const bool fin = FIX && k >= J.n_cycles;
    const bool track = FIX && (J.target > 0.f || fin);
    double tot = 0.0, cnt = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        if (!ok || j >= W) continue;
        const size_t idx = base + j;
        const float2 gp1 = v[m];
        uint8_t msk;
        if (FIRST) {
            msk = J.vb[idx] < thr ? 1 : 0;
            J.mask[idx] = msk;
        } else {
            msk = J.mask[idx];
        }
        if (FIX && track) hio_track(J.out, idx, gp1, msk, tot, cnt);
        if (fin) continue;
        const float2 gp = init_gprev ? gp1 : J.G[idx];
        float2 g;
        if ((FIX ? msk == 1 : msk != 0) || gp1.x < 0.f)
            g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)), __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
        else
            g = gp1;
        J.G[idx] = g;
        v[m] = g;
    }
    if (!fin) {
        reg_bluestein<M, NB, false, -1>(v, sm, b, l, J.prow);
        if (ok) {
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int j = l + m * Q;
                if (j < W) J.X[base + j] = v[m];
            }
        }
    }
    if (FIX) hio_tile_done<rrow_threads(M)>(J, wi.tile, tot, cnt);
}
template <bool FIRST, int M, bool FIX = false>
__global__ void __launch_bounds__(rrow_threads(M)) k_row_hio_bs(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_row_hio_bs<FIRST, M, FIX>(jobs, wi)));
}

// once per cycle (see k_row_finish) on Bluestein row lengths
template <int M>
__device__ __forceinline__ void b_row_finish_bs(const JobDev *jobs, const WorkItem wi, float2 *dbg_gprime)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rrow_nb(M), T = rrow_threads(M), Q = M / 8;
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32 > 2 ? 2 * T / 32 : 2];
    const JobDev &J = jobs[wi.job];
    JobState *st = J.st;
    if (st->stop) return;
    const int c = st->cycle;
    if (wi.tile == 0 && threadIdx.x == 0) st->max_bits = 0u;
    const int W = J.W;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = wi.tile * J.rpc + b;
    const bool ok = b < J.rpc && y < J.H;
    const size_t base = (size_t)y * W;
    const int K = J.ntaps[c];
    if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < W ? J.X[base + j] : make_float2(0.f, 0.f);
    }
    reg_bluestein<M, NB, false, +1>(v, sm, b, l, J.prow);   // ends with a barrier: sm is free
    float *nrow = reinterpret_cast<float *>(sm) + b * M;
    double tot = 0.0, cnt = 0.0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        if (j >= W) continue;
        const float nv = cnorm_ref(v[m]);
        nrow[j] = nv;
        if (ok) {
            const size_t idx = base + j;
            J.out[idx] = v[m].x;
            if (dbg_gprime) dbg_gprime[idx] = v[m];
            if (c > 0 && J.mask[idx]) {
                tot += (double)nv;
                cnt += 1.0;
            }
        }
    }
    block_sum2<T>(tot, cnt, red);   // includes barriers: nrow complete after it
    if (threadIdx.x == 0) {
        J.err_part[2 * wi.tile] = tot;
        J.err_part[2 * wi.tile + 1] = cnt;
    }
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int j = l + m * Q;
            if (j < W) J.hb[base + j] = hblur_at(nrow, W, j, wsm, K);
        }
    }
}
template <int M>
__global__ void __launch_bounds__(rrow_threads(M)) k_row_finish_bs(const JobDev *jobs, const WorkList *L,
                                                                   float2 *dbg_gprime)
{
    IMR_ITEM_LOOP((b_row_finish_bs<M>(jobs, wi, dbg_gprime)));
}

// X := inverse column transform of (M, 0), Bluestein column lengths
template <int M>
__device__ __forceinline__ void b_col_init_bs(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(M), Q = M / 8;
    const JobDev &J = jobs[wi.job];
    const int W = J.W, H = J.H;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = wi.tile * J.cpc + b;
    const bool ok = b < J.cpc && x < W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = make_float2(ok && j < H ? J.M[(size_t)j * W + x] : 0.f, 0.f);
    }
    reg_bluestein<M, NB, true, +1>(v, sm, b, l, J.pcol);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int j = l + m * Q;
            if (j < H) J.X[(size_t)j * W + x] = v[m];
        }
    }
}
template <int M>
__global__ void __launch_bounds__(rcol_threads(M)) k_col_init_bs(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col_init_bs<M>(jobs, wi)));
}

// column pass (see k_col) on Bluestein column lengths
template <int M>
__device__ __forceinline__ void b_col_bs(const JobDev *jobs, const WorkItem wi)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(M), Q = M / 8;
    const JobDev &J = jobs[wi.job];
    if (J.st->stop) return;
    const int W = J.W, H = J.H;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = wi.tile * J.cpc + b;
    const bool ok = b < J.cpc && x < W;
    const bool guard = J.mode == kModeShrinkWrap;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < H ? J.X[(size_t)j * W + x] : make_float2(0.f, 0.f);
    }
    reg_bluestein<M, NB, true, -1>(v, sm, b, l, J.pcol);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        const float mod = ok && j < H ? J.M[(size_t)j * W + x] : 0.f;
        const float f = modulus_factor(mod, v[m], guard);
        v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
    }
    reg_bluestein<M, NB, true, +1>(v, sm, b, l, J.pcol);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int j = l + m * Q;
            if (j < H) J.X[(size_t)j * W + x] = v[m];
        }
    }
}
template <int M>
__global__ void __launch_bounds__(rcol_threads(M)) k_col_bs(const JobDev *jobs, const WorkList *L)
{
    IMR_ITEM_LOOP((b_col_bs<M>(jobs, wi)));
}

// plain 2D transform passes on Bluestein lengths (rows of length p.n)
template <int S, int M>
__global__ void __launch_bounds__(rrow_threads(M)) k_fft_rows_bs(float2 *data, FftPlanDev p, int H, int rpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = M / 8;
    const int n = p.n;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = blockIdx.x * rpc + b;
    const bool ok = b < rpc && y < H;
    const size_t base = (size_t)y * n;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < n ? data[base + j] : make_float2(0.f, 0.f);
    }
    reg_bluestein<M, rrow_nb(M), false, S>(v, sm, b, l, p);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int j = l + m * Q;
            if (j < n) data[base + j] = v[m];
        }
    }
}

template <int S, int M>
__global__ void __launch_bounds__(rcol_threads(M)) k_fft_cols_bs(float2 *data, FftPlanDev p, int W, int cpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(M), Q = M / 8;
    const int n = p.n;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = blockIdx.x * cpc + b;
    const bool ok = b < cpc && x < W;
    float2 v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < n ? data[(size_t)j * W + x] : make_float2(0.f, 0.f);
    }
    reg_bluestein<M, NB, true, S>(v, sm, b, l, p);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int j = l + m * Q;
            if (j < n) data[(size_t)j * W + x] = v[m];
        }
    }
}

// ---- Bluestein with 16 values per thread (work lengths M >= 256) ------------
// The same chain as reg_bluestein on the 16-value register FFT: two
// exchanges per length-M transform up to M = 4096 instead of three, and
// twiddle powers in registers (loaded once per CTA; every job of a launch has
// the same work length).  Rows: 4096/M rows per CTA (256 threads); column
// tiles: rcol_nb(M) columns (512 threads for M >= 512).
__host__ __device__ constexpr int bs16_rows(int M) { return M >= 4096 ? 1 : 4096 / M; }
__host__ __device__ constexpr int bs16_row_threads(int M) { return bs16_rows(M) * M / 16; }
__host__ __device__ constexpr int bs16_row_smem(int M) { return bs16_rows(M) * M * 8; }
__host__ __device__ constexpr int bs16_col_threads(int M) { return rcol_nb(M) * M / 16; }
__host__ __device__ constexpr int bs16_col_smem(int M) { return rcol_nb(M) * M * 8; }

template <int M, class LAYOUT, int S>
__device__ __forceinline__ void reg16_bluestein(float2 (&v)[16], float2 *sm, int b, int l, const RegTw16<M> &tw,
                                                const FftPlanDev &p)
{
    constexpr int Q = M / 16;
    const int n = p.n;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int j = l + m * Q;
        if (j < n) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            v[m] = cmul(v[m], c);
        } else {
            v[m] = make_float2(0.f, 0.f);
        }
    }
    reg16_fft<M, LAYOUT, -1>(v, sm, b, l, tw);
    const float2 *spec = S < 0 ? p.bspec_f : p.bspec_b;
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = cmul(v[m], __ldg(spec + l + m * Q));
    reg16_fft<M, LAYOUT, +1>(v, sm, b, l, tw);
    __syncthreads();   // the last exchange's reads are done before the buffer is written again
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int j = l + m * Q;
        if (j < n) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            v[m] = cmul(v[m], c);
        }
    }
}

template <bool FIRST, int M, bool FIX = false>
__global__ void __launch_bounds__(bs16_row_threads(M), 2) k_row_hio_bs16(const JobDev *jobs, const WorkList *L)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = M / 16, T = bs16_row_threads(M);
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int n_items = L->n;
    if ((int)blockIdx.x >= n_items) return;
    RegTw16<M> rtw;
    rtw.load(jobs[item_at(L, blockIdx.x).job].prow.tw, l);
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const WorkItem wi = item_at(L, it);
        const JobDev &J = jobs[wi.job];
        JobState *st = J.st;
        if (st->stop) continue;
        const int W = J.W;
        const int y = wi.tile * J.rpc + b;
        const bool ok = b < J.rpc && y < J.H;
        const size_t base = (size_t)y * W;
        float2 v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            v[m] = ok && j < W ? J.X[base + j] : make_float2(0.f, 0.f);
        }
        reg16_bluestein<M, RowSwz16<M>, +1>(v, sm, b, l, rtw, J.prow);
        const float beta = J.beta;
        const float thr = st->thr;
        const int k = FIX ? st->cycle : 0;
        const bool init_gprev = FIX ? k == 0 : FIRST && st->hio_cycle == 0;
        const bool fin = FIX && k >= J.n_cycles;
        const bool track = FIX && (J.target > 0.f || fin);
        double tot = 0.0, cnt = 0.0;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            if (!ok || j >= W) continue;
            const size_t idx = base + j;
            const float2 gp1 = v[m];
            uint8_t msk;
            if (FIRST) {
                msk = J.vb[idx] < thr ? 1 : 0;
                J.mask[idx] = msk;
            } else {
                msk = J.mask[idx];
            }
            if (FIX && track) hio_track(J.out, idx, gp1, msk, tot, cnt);
            if (fin) continue;
            const float2 gp = init_gprev ? gp1 : J.G[idx];
            float2 g;
            if ((FIX ? msk == 1 : msk != 0) || gp1.x < 0.f)
                g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)), __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
            else
                g = gp1;
            J.G[idx] = g;
            v[m] = g;
        }
        if (!fin) {
            reg16_bluestein<M, RowSwz16<M>, -1>(v, sm, b, l, rtw, J.prow);
            if (ok) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int j = l + m * Q;
                    if (j < W) J.X[base + j] = v[m];
                }
            }
        }
        if (FIX) hio_tile_done<T>(J, wi.tile, tot, cnt);
        __syncthreads();
    }
}

template <int M>
__global__ void __launch_bounds__(bs16_row_threads(M), 2) k_row_finish_bs16(const JobDev *jobs, const WorkList *L,
                                                                         float2 *dbg_gprime)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = M / 16, T = bs16_row_threads(M);
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32 > 2 ? 2 * T / 32 : 2];
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int n_items = L->n;
    if ((int)blockIdx.x >= n_items) return;
    RegTw16<M> rtw;
    rtw.load(jobs[item_at(L, blockIdx.x).job].prow.tw, l);
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const WorkItem wi = item_at(L, it);
        const JobDev &J = jobs[wi.job];
        JobState *st = J.st;
        if (st->stop) continue;
        const int c = st->cycle;
        if (wi.tile == 0 && threadIdx.x == 0) st->max_bits = 0u;
        const int W = J.W;
        const int y = wi.tile * J.rpc + b;
        const bool ok = b < J.rpc && y < J.H;
        const size_t base = (size_t)y * W;
        const int K = J.ntaps[c];
        if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
        float2 v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            v[m] = ok && j < W ? J.X[base + j] : make_float2(0.f, 0.f);
        }
        reg16_bluestein<M, RowSwz16<M>, +1>(v, sm, b, l, rtw, J.prow);   // ends with a barrier: sm is free
        float *nrow = reinterpret_cast<float *>(sm) + b * M;
        double tot = 0.0, cnt = 0.0;
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            if (j >= W) continue;
            const float nv = cnorm_ref(v[m]);
            nrow[j] = nv;
            if (ok) {
                const size_t idx = base + j;
                J.out[idx] = v[m].x;
                if (dbg_gprime) dbg_gprime[idx] = v[m];
                if (c > 0 && J.mask[idx]) {
                    tot += (double)nv;
                    cnt += 1.0;
                }
            }
        }
        block_sum2<T>(tot, cnt, red);   // includes barriers: nrow complete after it
        if (threadIdx.x == 0) {
            J.err_part[2 * wi.tile] = tot;
            J.err_part[2 * wi.tile + 1] = cnt;
        }
        if (ok) {
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int j = l + m * Q;
                if (j < W) J.hb[base + j] = hblur_at(nrow, W, j, wsm, K);
            }
        }
        __syncthreads();
    }
}

// column kernels: mode 0 column pass (fwd, modulus, inv), 1 column init
// (inverse of (M, 0)), 2 plain forward, 3 plain inverse
template <int M, int MODE>
__device__ __forceinline__ void col_bs16_tile(float2 *X, const float *Mod, int W, int H, int x0, int cpc,
                                              const FftPlanDev &p, const RegTw16<M> &rtw, bool guard)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int NB = rcol_nb(M), Q = M / 16;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int x = x0 + b;
    const bool ok = b < cpc && x < W;
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int j = l + m * Q;
        if (MODE == 1) v[m] = make_float2(ok && j < H ? Mod[(size_t)j * W + x] : 0.f, 0.f);
        else v[m] = ok && j < H ? X[(size_t)j * W + x] : make_float2(0.f, 0.f);
    }
    if (MODE == 0) {
        reg16_bluestein<M, ColSwz16<M, NB>, -1>(v, sm, b, l, rtw, p);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            const float mod = ok && j < H ? Mod[(size_t)j * W + x] : 0.f;
            const float f = modulus_factor(mod, v[m], guard);
            v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
        }
    }
    reg16_bluestein<M, ColSwz16<M, NB>, MODE == 2 ? -1 : +1>(v, sm, b, l, rtw, p);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            if (j < H) X[(size_t)j * W + x] = v[m];
        }
    }
}

template <int M, int MODE>
__global__ void __launch_bounds__(bs16_col_threads(M)) k_col_bs16(const JobDev *jobs, const WorkList *L)
{
    constexpr int NB = rcol_nb(M);
    const int n_items = L->n;
    if ((int)blockIdx.x >= n_items) return;
    RegTw16<M> rtw;
    rtw.load(jobs[item_at(L, blockIdx.x).job].pcol.tw, threadIdx.x / NB);
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const WorkItem wi = item_at(L, it);
        const JobDev &J = jobs[wi.job];
        if (MODE == 0 && J.st->stop) continue;
        col_bs16_tile<M, MODE>(J.X, J.M, J.W, J.H, wi.tile * J.cpc, J.cpc, J.pcol, rtw,
                               J.mode == kModeShrinkWrap);
        __syncthreads();
    }
}

template <int S, int M>
__global__ void __launch_bounds__(bs16_row_threads(M), 2) k_fft_rows_bs16(float2 *data, FftPlanDev p, int H, int rpc)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int Q = M / 16;
    const int n = p.n;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int y = blockIdx.x * rpc + b;
    const bool ok = b < rpc && y < H;
    const size_t base = (size_t)y * n;
    RegTw16<M> rtw;
    rtw.load(p.tw, l);
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int j = l + m * Q;
        v[m] = ok && j < n ? data[base + j] : make_float2(0.f, 0.f);
    }
    reg16_bluestein<M, RowSwz16<M>, S>(v, sm, b, l, rtw, p);
    if (ok) {
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int j = l + m * Q;
            if (j < n) data[base + j] = v[m];
        }
    }
}

template <int S, int M>
__global__ void __launch_bounds__(bs16_col_threads(M)) k_fft_cols_bs16(float2 *data, FftPlanDev p, int W, int cpc)
{
    constexpr int NB = rcol_nb(M);
    RegTw16<M> rtw;
    rtw.load(p.tw, threadIdx.x / NB);
    col_bs16_tile<M, S < 0 ? 2 : 3>(data, nullptr, W, p.n, blockIdx.x * cpc, cpc, p, rtw, true);
}

}  // namespace imr

// ============================================================================
// Pipelined (persistent) passes for power-of-two lengths.
//
// Each CTA loops over its work items (blockIdx.x, + gridDim.x, ...).  Two
// shared-memory stages alternate: while the CTA transforms item i in one
// stage, the TMA engine copies item i+1 into the other (1D bulk copies for
// rows, 2D tensor-map tiles for columns), so HBM traffic stays in flight
// across the compute.  The FFT exchanges reuse the stage the item arrived
// in (swizzled, see fft_reg.cuh).
// ============================================================================
namespace imr {

__host__ __device__ constexpr int round16(int b) { return (b + 15) & ~15; }
__host__ __device__ constexpr int round128(int b) { return (b + 127) & ~127; }

// ---- rows -------------------------------------------------------------------
// stage: X rows (complex) | G rows (complex) | mask rows (u8) or blurred rows (f32)
template <bool FIRST, int N>
__host__ __device__ constexpr int prow_stage_bytes()
{
    return round128(2 * rrow_nb(N) * N * 8 + (FIRST ? rrow_nb(N) * N * 4 : round16(rrow_nb(N) * N)));
}
template <bool FIRST, int N>
__host__ __device__ constexpr int prow_smem() { return 128 + 2 * prow_stage_bytes<FIRST, N>(); }
// Three 8-warp CTAs per SM for the every-iteration shrink-wrap pass at
// power-of-two lengths (its stages fit three times in shared memory; 80
// registers per thread, no spills), two at lengths 3 * 2^k (stages of up to
// 52 KB; left free, the compiler took up to 246 registers, one CTA per SM)
// and two for the first pass of a cycle at powers of two (150 registers free,
// 0-28 B of spills at 128; 2048^2: 3.22 -> 3.05 ms for 24 cycles x 1 HIO).
// Other variants keep their registers.
__host__ __device__ constexpr int prow_min_blocks(bool FIRST, bool FIX, int N)
{
    return !FIRST && !FIX && is_pow2(N) && N <= 2048 ? 3 : (!FIX && (N % 3 == 0 ? !FIRST : is_pow2(N) && N <= 2048) ? 2 : 1);
}

__device__ __forceinline__ bool job_live(const JobDev *jobs, const WorkList *L, int item)
{
    const WorkItem wi = item_at(L, item);
    return jobs[wi.job].st->stop == 0;
}

// A persistent CTA's walk over its work items (stride gridDim.x), skipping
// items of stopped jobs.  A job's stop flag does not change during a launch
// (only the once-per-cycle kernels write it), so the liveness of the last job
// looked at is kept: a CTA whose consecutive items belong to one job (always,
// for a one-job list) pays no dependent global loads per item.
struct LiveWalker {
    const JobDev *jobs;
    const WorkItem *items;
    int n, job = -1;
    bool live = false;
    __device__ LiveWalker(const JobDev *j, const WorkList *L) : jobs(j), items(L->items), n(L->n) {}
    __device__ __forceinline__ int next(int it)
    {
        for (; it < n; it += gridDim.x) {
            const int jb = items ? items[it].job : 0;
            if (jb != job) {
                job = jb;
                live = jobs[jb].st->stop == 0;
            }
            if (live) break;
        }
        return it;
    }
    __device__ __forceinline__ WorkItem at(int it) const { return items ? items[it] : WorkItem{0, it}; }
};

// FIX: fixed-support HIO iteration (see b_row_hio)
template <bool FIRST, int N, bool FIX = false>
__global__ void __launch_bounds__(rrow_threads(N), prow_min_blocks(FIRST, FIX, N)) k_row_hio_p(const JobDev *jobs, const WorkList *L)
{
    extern __shared__ __align__(128) unsigned char sbuf[];
    constexpr int NB = rrow_nb(N), V = reg_v(N), Q = N / V;
    constexpr int XB = NB * N * 8;
    constexpr int STAGE = prow_stage_bytes<FIRST, N>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(sbuf);
    unsigned char *stages = sbuf + 128;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int n_items = L->n;

    LiveWalker walk(jobs, L);
    auto next_live = [&](int it) { return walk.next(it); };
    auto issue = [&](int item, int s) {   // one thread
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        const int y0 = wi.tile * J.rpc;
        const int nr = min(J.rpc, J.H - y0);
        const uint32_t xb = (uint32_t)(nr * N * 8);
        const uint32_t mb = FIRST ? (uint32_t)(nr * N * 4) : (uint32_t)round16(nr * N);
        unsigned char *st = stages + s * STAGE;
        mbar_arrive_expect_tx(&bars[s], 2 * xb + mb);
        tma_load_1d(st, J.X + (size_t)y0 * N, xb, &bars[s]);
        tma_load_1d(st + XB, J.G + (size_t)y0 * N, xb, &bars[s]);
        if (FIRST) tma_load_1d(st + 2 * XB, J.vb + (size_t)y0 * N, mb, &bars[s]);
        else tma_load_1d(st + 2 * XB, J.mask + (size_t)y0 * N, mb, &bars[s]);
    };

    __shared__ int s_next[2];   // next item, found by thread 0 (double-buffered by iteration parity)
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    int item = next_live(blockIdx.x);
    if (threadIdx.x == 0 && item < n_items) issue(item, 0);
    // every job of this launch has row length N: one twiddle set for all items
    RegTw<N> rtw;
    if (item < n_items) rtw.load(jobs[walk.at(item).job].prow.tw, l);
    for (int k = 0; item < n_items; ++k) {
        const int s = k & 1;
        int nxt = n_items;
        if (threadIdx.x == 0) {
            nxt = next_live(item + gridDim.x);
            s_next[s] = nxt;
            if (nxt < n_items) {
                fence_proxy_async_smem();
                issue(nxt, s ^ 1);
            }
        }
        // this item's job fields, loaded before the wait so that their latency overlaps it
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        JobState *const st = J.st;
        float2 *const Xg = J.X;
        float2 *const Gg = J.G;
        uint8_t *const Mk = J.mask;
        float *const outp = J.out;
        const int rpc = J.rpc, H = J.H;
        const float beta = J.beta;
        const float thr = FIRST ? st->thr : 0.f;
        const bool first_cycle = FIRST && st->hio_cycle == 0;
        const int kit = FIX ? st->cycle : 0;
        const bool fin = FIX && kit >= J.n_cycles;
        const bool tested = FIX && (J.target > 0.f || fin);
        const bool landed = mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), J.wait_ns);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicExch(&st->err, 1);
                // the copies still in flight (this item's, the next item's) land before the CTA exits
                mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), kDrainNs);
                if (nxt < n_items) mbar_wait(&bars[s ^ 1], (uint32_t)(((k + 1) >> 1) & 1), kDrainNs);
            }
            return;
        }
        unsigned char *stg = stages + s * STAGE;
        float2 *sX = reinterpret_cast<float2 *>(stg);
        const float2 *sG = reinterpret_cast<const float2 *>(stg + XB);
        const int y = wi.tile * rpc + b;
        const bool ok = b < rpc && y < H;
        const size_t base = (size_t)y * N;
        float2 v[V];
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = sX[b * N + l + m * Q];
        reg_fft_1buf<N, RowSwz<N, NB>, +1>(v, sX, b, l, rtw);
        const bool init_gprev = FIX ? kit == 0 : first_cycle;
        const bool track = tested && ok;
        double tot = 0.0, cnt = 0.0;
#pragma unroll
        for (int m = 0; m < V; ++m) {
            const int e = b * N + l + m * Q;
            const float2 gp1 = v[m];
            uint8_t msk;
            if constexpr (FIRST) msk = reinterpret_cast<const float *>(stg + 2 * XB)[e] < thr ? 1 : 0;
            else msk = (stg + 2 * XB)[e];
            if constexpr (FIX) {
                if (track) hio_track(outp, base + l + m * Q, gp1, msk, tot, cnt);
            }
            const float2 gp = init_gprev ? gp1 : sG[e];
            float2 g;
            if ((FIX ? msk == 1 : msk != 0) || gp1.x < 0.f)
                g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)),
                                __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
            else
                g = gp1;
            if (ok && !fin) {
                Gg[base + l + m * Q] = g;
                if constexpr (FIRST) Mk[base + l + m * Q] = msk;
            }
            v[m] = g;
        }
        if (!fin) {
            reg_fft_1buf<N, RowSwz<N, NB>, -1>(v, sX, b, l, rtw);
            if (ok) {
#pragma unroll
                for (int m = 0; m < V; ++m) Xg[base + l + m * Q] = v[m];
            }
        }
        if constexpr (FIX) hio_tile_done<rrow_threads(N)>(J, wi.tile, tot, cnt);
        fence_proxy_async_smem();
        __syncthreads();   // stage s is free for the copy issued next iteration; s_next[s] is visible
        item = s_next[s];
    }
}

// ---- once per cycle, pipelined ----------------------------------------------
// The work of b_row_finish_r on the persistent, TMA-fed skeleton of the row
// pass: inverse row FFT -> g'; out = Re(g'); error sums of |g'| against the
// previous cycle's mask; |g'| blurred along the row -> hb.  Stage: X rows and
// mask rows; the X region holds the row norms for the blur once the FFT is
// done with it.
template <int N>
__host__ __device__ constexpr int pfin_stage_bytes() { return round128(rrow_nb(N) * N * 8 + round16(rrow_nb(N) * N)); }
template <int N>
__host__ __device__ constexpr int pfin_smem() { return 128 + 2 * pfin_stage_bytes<N>(); }

template <int N>
__global__ void __launch_bounds__(rrow_threads(N)) k_row_finish_p(const JobDev *jobs, const WorkList *L, float2 *dbg_gprime)
{
    extern __shared__ __align__(128) unsigned char sbuf[];
    constexpr int NB = rrow_nb(N), V = reg_v(N), Q = N / V, T = rrow_threads(N);
    constexpr int XB = NB * N * 8;
    constexpr int STAGE = pfin_stage_bytes<N>();
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32 > 2 ? 2 * T / 32 : 2];
    __shared__ int s_next[2];
    uint64_t *bars = reinterpret_cast<uint64_t *>(sbuf);
    unsigned char *stages = sbuf + 128;
    const int b = threadIdx.x / Q, l = threadIdx.x % Q;
    const int n_items = L->n;

    LiveWalker walk(jobs, L);
    auto next_live = [&](int it) { return walk.next(it); };
    auto issue = [&](int item, int s) {   // one thread
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        const int y0 = wi.tile * J.rpc;
        const int nr = min(J.rpc, J.H - y0);
        const uint32_t xb = (uint32_t)(nr * N * 8), mb = (uint32_t)round16(nr * N);
        unsigned char *st = stages + s * STAGE;
        mbar_arrive_expect_tx(&bars[s], xb + mb);
        tma_load_1d(st, J.X + (size_t)y0 * N, xb, &bars[s]);
        tma_load_1d(st + XB, J.mask + (size_t)y0 * N, mb, &bars[s]);
    };

    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    int item = next_live(blockIdx.x);
    if (threadIdx.x == 0 && item < n_items) issue(item, 0);
    RegTw<N> rtw;
    if (item < n_items) rtw.load(jobs[walk.at(item).job].prow.tw, l);
    for (int k = 0; item < n_items; ++k) {
        const int s = k & 1;
        int nxt = n_items;
        if (threadIdx.x == 0) {
            nxt = next_live(item + gridDim.x);
            s_next[s] = nxt;
            if (nxt < n_items) {
                fence_proxy_async_smem();
                issue(nxt, s ^ 1);
            }
        }
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        JobState *const st = J.st;
        float *const outp = J.out;
        float *const hbp = J.hb;
        const int rpc = J.rpc, H = J.H;
        const int c = st->cycle;
        const int K = J.ntaps[c];
        if (threadIdx.x < kTapStride) wsm[threadIdx.x] = J.weights[(size_t)c * kTapStride + threadIdx.x];
        if (wi.tile == 0 && threadIdx.x == 0) st->max_bits = 0u;
        const bool landed = mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), J.wait_ns);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicExch(&st->err, 1);
                // the copies still in flight (this item's, the next item's) land before the CTA exits
                mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), kDrainNs);
                if (nxt < n_items) mbar_wait(&bars[s ^ 1], (uint32_t)(((k + 1) >> 1) & 1), kDrainNs);
            }
            return;
        }
        unsigned char *stg = stages + s * STAGE;
        float2 *sX = reinterpret_cast<float2 *>(stg);
        const uint8_t *sM = stg + XB;
        const int y = wi.tile * rpc + b;
        const bool ok = b < rpc && y < H;
        const size_t base = (size_t)y * N;
        float2 v[V];
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = sX[b * N + l + m * Q];
        reg_fft_1buf<N, RowSwz<N, NB>, +1>(v, sX, b, l, rtw);
        __syncthreads();   // the FFT's last reads of the X region are done: it now holds the norms
        float *nrow = reinterpret_cast<float *>(sX) + b * N;
        double tot = 0.0, cnt = 0.0;
#pragma unroll
        for (int m = 0; m < V; ++m) {
            const int e = l + m * Q;
            const float nv = cnorm_ref(v[m]);
            nrow[e] = nv;
            if (ok) {
                outp[base + e] = v[m].x;
                if (dbg_gprime) dbg_gprime[base + e] = v[m];
                if (c > 0 && sM[b * N + e]) {
                    tot += (double)nv;
                    cnt += 1.0;
                }
            }
        }
        block_sum2<T>(tot, cnt, red);   // includes barriers: nrow complete after it
        if (threadIdx.x == 0) {
            J.err_part[2 * wi.tile] = tot;
            J.err_part[2 * wi.tile + 1] = cnt;
        }
        if (ok) {
            // the V outputs' tap sums side by side (independent chains), each
            // in the tap order of hblur_at
            const int hw = (K - 1) / 2;
            float sum[V];
#pragma unroll
            for (int m = 0; m < V; ++m) sum[m] = 0.f;
            for (int k = 0; k < K; ++k) {
                const float wk = wsm[k];
#pragma unroll
                for (int m = 0; m < V; ++m) {
                    int xs = l + m * Q - hw + k;
                    xs = xs < 0 ? 0 : (xs > N - 1 ? N - 1 : xs);
                    sum[m] = __fadd_rn(sum[m], __fmul_rn(nrow[xs], wk));
                }
            }
#pragma unroll
            for (int m = 0; m < V; ++m) hbp[base + l + m * Q] = sum[m];
        }
        fence_proxy_async_smem();
        __syncthreads();   // stage s is free for the copy issued next iteration; s_next[s] is visible
        item = s_next[s];
    }
}

// ---- columns ------------------------------------------------------------------
// stage: X tile [N][NB] complex | M tile [N][NB] float (when NB*4 >= 16)
// rows per 2D TMA box: must divide N (boxes tile the column exactly)
__host__ __device__ constexpr int pcol_box_rows(int N) { return N <= 256 ? N : (N % 3 == 0 ? 192 : 256); }
__host__ __device__ constexpr bool pcol_tma_m(int N) { return rcol_nb(N) * 4 >= 16; }
__host__ __device__ constexpr int pcol_threads(int N) { return rcol_threads(N); }
template <int N>
__host__ __device__ constexpr int pcol_stage_bytes()
{
    return round128(rcol_nb(N) * N * 8 + (pcol_tma_m(N) ? rcol_nb(N) * N * 4 : 0));
}
// barriers | 2 stages | twiddle table (N complex)
template <int N>
__host__ __device__ constexpr int pcol_smem() { return 128 + 2 * pcol_stage_bytes<N>() + N * 8; }

template <int N>
__global__ void __launch_bounds__(rcol_threads(N)) k_col_p(const JobDev *jobs, const WorkList *L)
{
    extern __shared__ __align__(128) unsigned char sbuf[];
    constexpr int NB = rcol_nb(N), V = reg_v(N), Q = N / V;
    constexpr int XB = NB * N * 8;
    constexpr int BR = pcol_box_rows(N);
    constexpr bool TM = pcol_tma_m(N);
    constexpr int STAGE = pcol_stage_bytes<N>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(sbuf);
    unsigned char *stages = sbuf + 128;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int n_items = L->n;

    LiveWalker walk(jobs, L);
    auto next_live = [&](int it) { return walk.next(it); };
    auto issue = [&](int item, int s) {
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        unsigned char *st = stages + s * STAGE;
        const int x0 = wi.tile * NB;
        mbar_arrive_expect_tx(&bars[s], (uint32_t)(XB + (TM ? NB * N * 4 : 0)));
        for (int r0 = 0; r0 < N; r0 += BR) {
            tma_load_2d(st + (size_t)r0 * NB * 8, &J.tmX, x0, r0, &bars[s]);
            if constexpr (TM) tma_load_2d(st + XB + (size_t)r0 * NB * 4, &J.tmM, x0, r0, &bars[s]);
        }
    };

    // the column length is N for every job of this launch: one twiddle table,
    // kept in shared memory (the stages leave little L1 for it)
    float2 *stw = reinterpret_cast<float2 *>(stages + 2 * STAGE);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_fence_init();
    }
    int item = next_live(blockIdx.x);
    if (item < n_items) {
        const float2 *gtw = jobs[walk.at(item).job].pcol.tw;
        for (int i = threadIdx.x; i < N; i += rcol_threads(N)) stw[i] = gtw[i];
    }
    __syncthreads();
    if (threadIdx.x == 0 && item < n_items) issue(item, 0);
    for (int k = 0; item < n_items; ++k) {
        const int nxt = next_live(item + gridDim.x);
        const int s = k & 1;
        if (threadIdx.x == 0 && nxt < n_items) {
            bulk_wait_read0();   // the tile stored from stage s^1 last iteration has left it
            fence_proxy_async_smem();
            issue(nxt, s ^ 1);
        }
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        const bool landed = mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), J.wait_ns);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicExch(&J.st->err, 1);
                // the copies still in flight (this tile's, the next tile's) land before the CTA exits
                mbar_wait(&bars[s], (uint32_t)((k >> 1) & 1), kDrainNs);
                if (nxt < n_items) mbar_wait(&bars[s ^ 1], (uint32_t)(((k + 1) >> 1) & 1), kDrainNs);
                bulk_wait0();
            }
            return;
        }
        unsigned char *stg = stages + s * STAGE;
        float2 *sX = reinterpret_cast<float2 *>(stg);
        const int W = J.W;
        const int x = wi.tile * NB + b;
        const bool ok = x < W;
        float2 v[V];
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = sX[(l + m * Q) * NB + b];
        reg_fft_1buf<N, ColSwz<N, NB>, -1, true>(v, sX, b, l, stw);
#pragma unroll
        for (int m = 0; m < V; ++m) {
            float mod;
            if constexpr (TM) mod = reinterpret_cast<const float *>(stg + XB)[(l + m * Q) * NB + b];
            else mod = ok ? J.M[(size_t)(l + m * Q) * W + x] : 0.f;
            const float f = modulus_factor(mod, v[m], J.mode == kModeShrinkWrap);
            v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
        }
        reg_fft_1buf<N, ColSwz<N, NB>, +1, true>(v, sX, b, l, stw);
        // the result goes back into the stage (tile layout) and leaves by TMA
        __syncthreads();
#pragma unroll
        for (int m = 0; m < V; ++m) sX[(l + m * Q) * NB + b] = v[m];
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            const int x0 = wi.tile * NB;
            for (int r0 = 0; r0 < N; r0 += BR) tma_store_2d(&J.tmX, x0, r0, sX + (size_t)r0 * NB);
            bulk_commit();
        }
        item = nxt;
    }
    if (threadIdx.x == 0) bulk_wait0();
}

// ---- columns, 16 values per thread (powers of two >= 128) ----------------------
// The X tiles and TMA traffic of k_col_p; each thread holds 16 values of its
// column (a length-2048 transform is three passes, two exchanges), and its
// twiddle powers stay in registers for the whole persistent loop, so no
// shared-memory twiddle table (whose strided reads were the pass's bank
// conflicts) remains.  The modulus comes from the job's column-tiled copy
// (JobDev::Mt: one contiguous block per tile) into registers.  Three stages:
// tile k+2 is requested after the forward FFT of tile k into the stage of
// tile k-1, whose bulk store has had a whole forward FFT to read it.
// (Measured at 2048^2 and kept out: 2-column tiles with two CTAs per SM, 15 %
// slower; the modulus by TMA from the row-major array, 4 % slower.)
// The modulus in column tiles (JobDev::Mt): element i of the tiled array is
// tile t = i / (H*NB), row r = (i / NB) % H, column t*NB + i % NB (zero past W).
static __global__ void k_modulus_tiles(const float *__restrict__ M, float *__restrict__ Mt, int W, int H, int NB, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t t = i / ((size_t)H * NB);
    const int r = (int)((i / NB) % H), x = (int)(t * NB) + (int)(i % NB);
    Mt[i] = x < W ? M[(size_t)r * W + x] : 0.f;
}

__host__ __device__ constexpr int pcol16_threads(int N, int NBT) { return NBT * N / 16; }
__host__ __device__ constexpr int pcol16_nbt(int N) { return rcol_nb(N); }
// A stage holds one X tile; the modulus goes straight to registers.  Three
// stages where they fit (all lengths up to 4096: 64 KB tiles), so tile k+2 is
// requested while tile k is transformed.
template <int N, int NBT>
__host__ __device__ constexpr int pcol16_stage_bytes() { return round128(NBT * N * 8); }
template <int N, int NBT>
__host__ __device__ constexpr int pcol16_stages()
{
    return 128 + 3 * pcol16_stage_bytes<N, NBT>() <= 227 * 1024 ? 3 : 2;
}
template <int N, int NBT>
__host__ __device__ constexpr int pcol16_smem() { return 128 + pcol16_stages<N, NBT>() * pcol16_stage_bytes<N, NBT>(); }
__host__ __device__ constexpr int pcol16_min_blocks(int N, int NBT) { return NBT * N / 16 <= 256 ? 2 : 1; }

// Item v of a column launch with n tiles of which the first S run as halves
// (WorkList::n_split): v < S is half 0 of tile v, S <= v < n tile v whole,
// n <= v < n + S half 1 of tile v - n.
struct ColItem {
    int tile, half;   // half: -1 the whole tile, else 0 / 1
};
__device__ __forceinline__ ColItem col_item(int v, int n, int S)
{
    if (v < S) return ColItem{v, 0};
    if (v < n) return ColItem{v, -1};
    return ColItem{v - n, 1};
}

// SPLIT: the variant that runs WorkList::n_split tiles as half tiles (plans
// whose tiles fill at most half of the resident CTAs); the other keeps the
// registers and code of whole tiles alone.
template <int N, int NBT, bool SPLIT>
__global__ void __launch_bounds__(pcol16_threads(N, NBT), pcol16_min_blocks(N, NBT))
k_col_p16(const JobDev *jobs, const WorkList *L)
{
    extern __shared__ __align__(128) unsigned char sbuf[];
    constexpr int NB = NBT, V = 16, Q = N / V;
    constexpr int XB = NB * N * 8;
    constexpr int BR = pcol_box_rows(N);
    constexpr int STAGE = pcol16_stage_bytes<N, NBT>();
    constexpr int NST = pcol16_stages<N, NBT>();
    constexpr int HNB = NB / 2;                      // columns of a half tile
    constexpr bool HALVES = SPLIT && HNB * 8 >= 16;  // half-tile rows are whole 16-byte TMA units
    uint64_t *bars = reinterpret_cast<uint64_t *>(sbuf);   // NST barriers in the first 128 bytes
    unsigned char *stages = sbuf + 128;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int n_tiles = L->n;
    const int n_split = (HALVES && L->items == nullptr) ? L->n_split : 0;
    const int n_items = n_tiles + n_split;
    __shared__ int s_item[NST];   // item whose tile each stage receives (n_items: none); thread 0 writes

    LiveWalker walk(jobs, L);
    walk.n = n_items;
    auto issue = [&](int item, int s) {   // one thread
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        unsigned char *st = stages + s * STAGE;
        const ColItem ci = col_item(item, n_tiles, n_split);
        if (!HALVES || ci.half < 0) {
            const int x0 = wi.tile * NB;   // items == nullptr: the item is the tile
            mbar_arrive_expect_tx(&bars[s], (uint32_t)XB);
            for (int r0 = 0; r0 < N; r0 += BR) tma_load_2d(st + (size_t)r0 * NB * 8, &J.tmX, x0, r0, &bars[s]);
        } else {
            const int x0 = ci.tile * NB + ci.half * HNB;
            mbar_arrive_expect_tx(&bars[s], (uint32_t)(XB / 2));
            for (int r0 = 0; r0 < N; r0 += BR) tma_load_2d(st + (size_t)r0 * HNB * 8, &J.tmXh, x0, r0, &bars[s]);
        }
    };

    int item = walk.next(blockIdx.x);
    // the column length is N for every job of this launch: one set of twiddles
    RegTw16<N> rtw;
    if (item < n_items) rtw.load(jobs[walk.at(item).job].pcol.tw, l);
    int it_next = n_items;   // thread 0: the next item to request
    if (threadIdx.x == 0) {
        for (int t = 0; t < NST; ++t) mbar_init(&bars[t], 1);
        mbar_fence_init();
        int it = item;
        for (int t = 0; t < NST - 1; ++t) {   // the first NST - 1 tiles
            s_item[t] = it;
            if (it < n_items) {
                issue(it, t);
                it = walk.next(it + gridDim.x);
            }
        }
        it_next = it;
    }
    __syncthreads();
    // thread 0, after the forward transform of item k: request the next item
    // into the stage of item k - 1, free once the store committed after it
    // has read it
    auto request_next = [&](int k) {
        const int t = (k + NST - 1) % NST;
        s_item[t] = it_next;
        if (it_next < n_items) {
            bulk_wait_read0();
            fence_proxy_async_smem();
            issue(it_next, t);
            it_next = walk.next(it_next + gridDim.x);
        }
    };
    // a wait that gave up: this item and the items already requested beyond it
    // land before the CTA exits (thread 0)
    auto drain = [&](int k, const JobDev &J) {
        atomicExch(&J.st->err, 1);
        for (int d = 0; d < NST - 1; ++d) {
            const int t = (k + d) % NST;
            if (d == 0 || s_item[t] < n_items) mbar_wait(&bars[t], (uint32_t)(((k + d) / NST) & 1), kDrainNs);
        }
        bulk_wait0();
    };
    for (int k = 0; item < n_items; ++k) {
        const int s = k % NST;
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        const int W = J.W;
        const bool guard = J.mode == kModeShrinkWrap;
        const ColItem ci = col_item(item, n_tiles, n_split);
        float *const sX0 = reinterpret_cast<float *>(stages + s * STAGE);
        if (!HALVES || ci.half < 0) {
            const int tile = wi.tile;
            const int x = tile * NB + b;
            const bool ok = x < W;
            // the modulus goes straight to registers, its latency hidden by the
            // tile wait and the forward FFT: from the tiled copy (one 128-byte
            // line per warp and value) when the job has one
            float mod[V];
            if (const float *mt = J.Mt) {
                mt += (size_t)tile * NB * N + b;
#pragma unroll
                for (int m = 0; m < V; ++m) mod[m] = __ldg(mt + (size_t)(l + m * Q) * NB);
            } else {
#pragma unroll
                for (int m = 0; m < V; ++m) mod[m] = ok ? __ldg(J.M + (size_t)(l + m * Q) * W + x) : 0.f;
            }
            const bool landed = mbar_wait(&bars[s], (uint32_t)((k / NST) & 1), J.wait_ns);
            if (__syncthreads_or(!landed)) {
                if (threadIdx.x == 0) drain(k, J);
                return;
            }
            float2 *sX = reinterpret_cast<float2 *>(sX0);
            float2 v[V];
#pragma unroll
            for (int m = 0; m < V; ++m) v[m] = sX[(l + m * Q) * NB + b];
            reg16_fft<N, ColSwz16<N, NB>, -1>(v, sX, b, l, rtw);
            if (threadIdx.x == 0) request_next(k);
#pragma unroll
            for (int m = 0; m < V; ++m) {
                const float f = modulus_factor(mod[m], v[m], guard);
                v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
            }
            reg16_fft<N, ColSwz16<N, NB>, +1>(v, sX, b, l, rtw);
            // the result goes back into the stage (tile layout) and leaves by TMA
            __syncthreads();
#pragma unroll
            for (int m = 0; m < V; ++m) sX[(l + m * Q) * NB + b] = v[m];
            fence_proxy_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int r0 = 0; r0 < N; r0 += BR) tma_store_2d(&J.tmX, tile * NB, r0, sX + (size_t)r0 * NB);
                bulk_commit();
            }
        } else if constexpr (HALVES) {
            // a half tile: two threads per sequence position, each with the
            // values of one parity (reg16h_fft), h uniform over a warp; the
            // stage's second half holds the radix-16 trades (forward, inverse)
            const int h = (threadIdx.x >> 5) & 1;
            const int pair = (threadIdx.x & 31) | ((threadIdx.x >> 6) << 5);
            constexpr int npairs = pcol16_threads(N, NBT) / 2;
            const int hb = pair % HNB, hl = pair / HNB;
            const int tile = ci.tile;
            const int x0 = tile * NB + ci.half * HNB;
            const int x = x0 + hb;
            const bool ok = x < W;
            RegTw16<N> htw;
            htw.load(J.pcol.tw, hl);
            float mod[8];
            if (const float *mt = J.Mt) {
                mt += (size_t)tile * NB * N + ci.half * HNB + hb;
#pragma unroll
                for (int j = 0; j < 8; ++j) mod[j] = __ldg(mt + (size_t)(hl + (2 * j + h) * Q) * NB);
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j) mod[j] = ok ? __ldg(J.M + (size_t)(hl + (2 * j + h) * Q) * W + x) : 0.f;
            }
            const bool landed = mbar_wait(&bars[s], (uint32_t)((k / NST) & 1), J.wait_ns);
            if (__syncthreads_or(!landed)) {
                if (threadIdx.x == 0) drain(k, J);
                return;
            }
            float2 *sX = reinterpret_cast<float2 *>(sX0);
            float2 *mid = sX + N * HNB;   // 2 x 8 * npairs values
            float2 v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = sX[(hl + (2 * j + h) * Q) * HNB + hb];
            reg16h_fft<N, ColSwz16<N, HNB>, -1>(v, sX, mid, hb, hl, h, pair, npairs, htw);
            if (threadIdx.x == 0) request_next(k);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float f = modulus_factor(mod[j], v[j], guard);
                v[j] = make_float2(__fmul_rn(v[j].x, f), __fmul_rn(v[j].y, f));
            }
            reg16h_fft<N, ColSwz16<N, HNB>, +1>(v, sX, mid + 8 * npairs, hb, hl, h, pair, npairs, htw);
            __syncthreads();
#pragma unroll
            for (int j = 0; j < 8; ++j) sX[(hl + (2 * j + h) * Q) * HNB + hb] = v[j];
            fence_proxy_async_smem();
            __syncthreads();
            if (threadIdx.x == 0) {
                if (x0 < W)
                    for (int r0 = 0; r0 < N; r0 += BR) tma_store_2d(&J.tmXh, x0, r0, sX + (size_t)r0 * HNB);
                bulk_commit();
            }
        }
        item = s_item[(k + 1) % NST];   // written before the barriers above
    }
    if (threadIdx.x == 0) bulk_wait0();
}

}  // namespace imr

#include "kernels_tc.cuh"
