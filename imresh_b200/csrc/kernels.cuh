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

namespace imr {

__device__ __forceinline__ WorkItem get_work(const WorkItem *wl)
{
    if (wl) return wl[blockIdx.x];
    return WorkItem{0, (int)blockIdx.x};
}

// ---- launch shapes ---------------------------------------------------------
// Row passes: NB rows of length N per CTA, T threads.  Column passes: NB
// columns of length N per CTA (one tile row = NB contiguous complex values),
// T threads.  N = 0 selects the runtime-length FFT.
__host__ __device__ constexpr int row_nb(int N) { return N == 0 ? 0 : (N <= 2048 ? 2048 / N : 1); }
__host__ __device__ constexpr int row_threads(int N) { return N == 0 ? kRowThreads : 256; }
__host__ __device__ constexpr int col_nb(int N) { return N == 0 ? 0 : (N <= 2048 ? 8 : 4); }
__host__ __device__ constexpr int col_threads(int N)
{
    return N == 0 ? kColThreads
                  : ((col_nb(N) * N / 16 + 31) / 32 * 32 < 64 ? 64
                     : ((col_nb(N) * N / 16 + 31) / 32 * 32 > 1024 ? 1024 : (col_nb(N) * N / 16 + 31) / 32 * 32));
}

template <int N, int S>
__device__ __forceinline__ void fft_rows(float2 *sm, int nr, const FftPlanDev &p)
{
    if constexpr (N > 0) ct_fft<N, row_nb(N), row_threads(N), S, false>(sm, nr, p.tw);
    else fft_smem<S, kRowVpt>(sm, p, nr, p.n, 1, false, threadIdx.x, kRowThreads);
}

template <int N, int S>
__device__ __forceinline__ void fft_cols(float2 *sm, int nc, const FftPlanDev &p)
{
    if constexpr (N > 0) ct_fft<N, col_nb(N), col_threads(N), S, true>(sm, nc, p.tw);
    else fft_smem<S, kColVpt>(sm, p, nc, 1, nc, true, threadIdx.x, kColThreads);
}

// |z| exactly as the reference computes it: sqrtf(re*re + im*im) with a
// separate multiply and add (vectorElementwise.cpp:52-54).
__device__ __forceinline__ float cnorm_ref(float2 z)
{
    return sqrtf(__fadd_rn(__fmul_rn(z.x, z.x), __fmul_rn(z.y, z.y)));
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
    for (int r = ty; r < rows_in; r += kVbThreads / kVbTileX) {
        int ys = y0 - N + r;
        ys = ys < 0 ? 0 : (ys > H - 1 ? H - 1 : ys);
        tile[r * kVbTileX + tx] = x < W ? src[(size_t)ys * W + x] : 0.f;
    }
    __syncthreads();
    float mx = 0.f;
    if (x < W) {
        for (int r = ty; r < kVbTileY; r += kVbThreads / kVbTileX) {
            const int y = y0 + r;
            if (y >= H) break;
            float sum = 0.f;
            for (int k = 0; k < K; ++k)
                sum = __fadd_rn(sum, __fmul_rn(tile[(r + k) * kVbTileX + tx], w[k]));
            dst[(size_t)y * W + x] = sum;
            mx = fmaxf(mx, sum);
        }
    }
    return mx;
}

// ---------------------------------------------------------------- init
// X := inverse column FFT of (M, 0): the column half of g'_0 = IFFT2(M)
// (cudaShrinkWrap.cu:229-232: CopyToRealPart then an in-place inverse FFT).
template <int N>
__global__ void __launch_bounds__(col_threads(N)) k_col_init(const JobDev *jobs, const WorkItem *wl)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const WorkItem wi = get_work(wl);
    const JobDev &J = jobs[wi.job];
    const int W = J.W, H = J.H;
    const int x0 = wi.tile * J.cpc;
    const int nc = min(J.cpc, W - x0);
    constexpr int T = col_threads(N);
    const int es = N > 0 ? col_nb(N) : nc;   // smem row stride of the tile
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

// ---------------------------------------------------------------- column pass
// Forward column FFT, G <- G * M/|G| (|G| = 0 -> 1; applyComplexModulus,
// src/imresh/algorithms/cuda/cudaVectorElementwise.cu:168-195), inverse
// column FFT.
template <int N>
__global__ void __launch_bounds__(col_threads(N)) k_col(const JobDev *jobs, const WorkItem *wl)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const WorkItem wi = get_work(wl);
    const JobDev &J = jobs[wi.job];
    if (J.st->stop) return;
    const int W = J.W, H = J.H;
    const int x0 = wi.tile * J.cpc;
    const int nc = min(J.cpc, W - x0);
    constexpr int T = col_threads(N);
    const int es = N > 0 ? col_nb(N) : nc;
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        sm[y * es + c] = J.X[(size_t)y * W + x0 + c];
    }
    __syncthreads();
    fft_cols<N, -1>(sm, nc, J.pcol);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        const float2 g = sm[y * es + c];
        float nrm = cnorm_ref(g);
        if (nrm == 0.f) nrm = 1.f;
        const float f = __fdiv_rn(J.M[(size_t)y * W + x0 + c], nrm);
        sm[y * es + c] = make_float2(__fmul_rn(g.x, f), __fmul_rn(g.y, f));
    }
    __syncthreads();
    fft_cols<N, +1>(sm, nc, J.pcol);
    for (int i = threadIdx.x; i < H * nc; i += T) {
        const int y = i / nc, c = i - y * nc;
        J.X[(size_t)y * W + x0 + c] = sm[y * es + c];
    }
}

// ---------------------------------------------------------------- row pass
// Inverse row FFT -> g'; HIO domain constraint
//   if mask == 1 or Re(g') < 0:  g = g_prev - beta*g'  else  g = g'
// (cudaKernelApplyHioDomainConstraints, cudaVectorElementwise.cu:42-72);
// g_prev := g; forward row FFT of g -> X.
// FIRST: first iteration of a cycle -- builds the uint8 mask from the blurred
// image (mask = blurred < threshold, cudaKernelCutOff, cudaVectorElementwise.cu:198-219)
// and, on cycle 0, takes g_prev = g'_0 (cudaShrinkWrap.cu:304-309).
template <bool FIRST, int N>
__global__ void __launch_bounds__(row_threads(N)) k_row_hio(const JobDev *jobs, const WorkItem *wl)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    const WorkItem wi = get_work(wl);
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
    const bool init_gprev = FIRST && st->hio_cycle == 0;
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
        const float2 gp = init_gprev ? gp1 : J.G[idx];
        float2 g;
        if (m || gp1.x < 0.f)
            g = make_float2(__fsub_rn(gp.x, __fmul_rn(beta, gp1.x)),
                            __fsub_rn(gp.y, __fmul_rn(beta, gp1.y)));
        else
            g = gp1;
        J.G[idx] = g;
        sm[i] = g;
    }
    __syncthreads();
    fft_rows<N, -1>(sm, nr, J.prow);
    for (int i = threadIdx.x; i < n; i += T) J.X[base + i] = sm[i];
}

// Once per cycle: inverse row FFT -> g'; out = Re(g') (CopyFromRealPart,
// cudaVectorElementwise.cu:98-117); error sums against the previous cycle's
// mask (cudaKernelCalculateHioError, cudaVectorReduce.cu:284-355, summed in
// double here); |g'| (cudaKernelComplexNormElementwise) blurred along rows.
template <int N>
__global__ void __launch_bounds__(row_threads(N)) k_row_finish(const JobDev *jobs, const WorkItem *wl,
                                                              float2 *dbg_gprime)
{
    extern __shared__ float4 smem4[];
    float2 *sm = reinterpret_cast<float2 *>(smem4);
    constexpr int T = row_threads(N);
    __shared__ float wsm[kTapStride];
    __shared__ double red[2 * T / 32];
    const WorkItem wi = get_work(wl);
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

// Once per cycle: vertical blur hb -> vb and the global max; the last CTA
// of the job finalises the cycle: error E = sqrt(sum mask*|g'|)/sum mask of
// the previous cycle (cudaVectorReduce.cu:357-403) and the stop test
// E < target (cudaShrinkWrap.cu:374-375), then the threshold
// (cycle 0 ? cutOffAutoCorel : cutOff) * max (cudaShrinkWrap.cu:274-276).
__global__ void __launch_bounds__(kVbThreads) k_vblur(const JobDev *jobs, const WorkItem *wl)
{
    __shared__ float tile[(kVbTileY + 2 * 31) * kVbTileX];
    __shared__ float wsm[kTapStride];
    __shared__ float fred[kVbThreads / 32];
    __shared__ double red[2 * kVbThreads / 32];
    __shared__ int s_last;
    const WorkItem wi = get_work(wl);
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
    const int es = N > 0 ? col_nb(N) : nc;
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

__global__ void __launch_bounds__(kRowThreads) k_hblur(float *data, int W, int H, Taps w, int K)
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

__global__ void __launch_bounds__(kVbThreads) k_vblur_plain(const float *src, float *dst, int W, int H,
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

// Global max of a float array (vectorMax; cudaVectorReduce.cu:229-239):
// signed floats ordered through an order-preserving integer key.
__device__ __forceinline__ unsigned f2key(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__global__ void __launch_bounds__(256) k_vector_max(const float *d, long n, unsigned *key)
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
