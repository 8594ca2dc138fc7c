// Split-precision tensor-core column pass (sm_100a).
//
// The column pass of kernels.cuh (forward column FFT -> modulus projection ->
// inverse column FFT, the cuFFT pair of cudaShrinkWrap.cu:319,343 around
// cudaKernelApplyComplexModulus) with its radix-16 stages computed as DFT
// matrix products on the tensor cores.  A column of length N = 16*16*R3
// (256..4096) is transformed in Stockham passes of radix 16, 16 and R3
// (exactly the decomposition of the FP32 pass); a radix-16 pass over the
// tile's NB*N/16 groups is the product
//     [Yr | Yi] = [Xr | Xi] * [[C, +-S], [-+S, C]]          (K = N = 32)
// with C = cos(2 pi p s/16), S = sin(2 pi p s/16) and the sign of the
// direction, one matrix row per group (16 groups per m16n8k16 tile).  The
// FP32 inputs are split into a 16-bit high part and a 16-bit remainder
// (x = hi + lo + O(2^-17 |x|) in BF16, O(2^-22 |x|) in FP16), the DFT
// matrix likewise, and three products -- lo*hi, hi*lo, hi*hi, smallest
// first -- accumulate in FP32 ("hi+lo compensated" products; lo*lo is below
// the FP32 rounding of the sum).  Twiddles between passes are FP32 complex
// products on the CUDA cores, as is a last pass of radix 2, 4 or 8 and the
// modulus projection.  FP16 inputs are scaled per DFT-16 (per matrix row) by
// a power of two that puts the row's largest magnitude near 2^14 (exact;
// undone on the same row of the product), so the 5-bit exponent range is
// neither exceeded nor wasted on rows far below the tile's largest.
//
// Fragment layout (mma.sync m16n8k16, row.col): lane (g = lane/4, t = lane%4)
// holds, of the A tile (16 groups x 16 points), points {2t, 2t+1, 2t+8, 2t+9}
// of groups g and g+8; the accumulator tile of a 16-column block holds outputs
// {2t, 2t+1} of groups g and g+8 -- so a lane's eight complex outputs of one
// DFT-16 sit at the same (group, index) places as its eight inputs, and the
// last forward pass, the modulus and the first inverse pass chain in
// registers whenever the last pass is a radix-16 one (N = 256, 4096).
#pragma once
#include <cuda_fp16.h>

namespace imr {

constexpr int kPrecFp32 = 0;    // CUDA-core FFT (kernels.cuh)
constexpr int kPrecBf16x3 = 1;  // BF16 hi+lo, three products, FP32 accumulation
constexpr int kPrecFp16x3 = 2;  // FP16 hi+lo (scaled), three products, FP32 accumulation

// hi + lo split of (a, b) into packed 16-bit pairs, a in the low half
template <int PREC>
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    if constexpr (PREC == kPrecBf16x3) {
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(hi) : "f"(b), "f"(a));
        const float ha = __uint_as_float(hi << 16), hb = __uint_as_float(hi & 0xffff0000u);
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(lo) : "f"(__fsub_rn(b, hb)), "f"(__fsub_rn(a, ha)));
    } else {
        asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(hi) : "f"(b), "f"(a));
        const float2 h = __half22float2(*reinterpret_cast<const __half2 *>(&hi));
        asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(lo) : "f"(__fsub_rn(b, h.y)), "f"(__fsub_rn(a, h.x)));
    }
}

template <int PREC>
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    if constexpr (PREC == kPrecBf16x3)
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
                     "{%8,%9}, {%0,%1,%2,%3};"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    else
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
                     "{%8,%9}, {%0,%1,%2,%3};"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// The DFT-16 matrices C and S as this lane's B fragments (k = point p,
// n = output s), hi and lo parts, both 8-column blocks; -S is S with the
// sign bits of both halves flipped (exact).
template <int PREC>
struct Dft16B {
    uint32_t c[2][2][2], s[2][2][2];   // [hi/lo][n block][register]

    __device__ __forceinline__ void init(int lane)
    {
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int nb = 0; nb < 2; ++nb) {
            const int sc = g + 8 * nb;
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int k0 = 2 * t + 8 * r, k1 = k0 + 1;
                double s0, c0, s1, c1;
                sincospi((double)((k0 * sc) & 15) / 8.0, &s0, &c0);
                sincospi((double)((k1 * sc) & 15) / 8.0, &s1, &c1);
                split2<PREC>((float)c0, (float)c1, c[0][nb][r], c[1][nb][r]);
                split2<PREC>((float)s0, (float)s1, s[0][nb][r], s[1][nb][r]);
            }
        }
    }
};

// One DFT-16 tile: x (this lane's eight complex inputs, fragment order
// i -> group g + 8*((i>>1)&1), point 2t + (i&1) + 8*(i>>2)) -> y in the same
// order.  FP16: each matrix row (group) is scaled by the power of two that
// puts its largest component in [2^13, 2^14) -- a row scale of A scales the
// same row of the product, so it is undone exactly afterwards -- found over
// the four lanes that share the row.
template <int PREC, int S>
__device__ __forceinline__ void dft16_tc(const float2 (&x)[8], float2 (&y)[8], const Dft16B<PREC> &B)
{
    float sc[2] = {1.f, 1.f}, un[2] = {1.f, 1.f};   // rows g, g + 8
    if constexpr (PREC == kPrecFp16x3) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float m = 0.f;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (((i >> 1) & 1) == h) m = fmaxf(m, fmaxf(fabsf(x[i].x), fabsf(x[i].y)));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
            int e = 0;
            if (m > 0.f && m < __int_as_float(0x7f800000)) frexpf(m, &e);   // m = f 2^e, f in [0.5, 1)
            const int sh = min(max(14 - e, -120), 120);
            sc[h] = ldexpf(1.f, sh);
            un[h] = ldexpf(1.f, -sh);
        }
    }
    uint32_t ar[2][4], ai[2][4];   // [hi/lo][register]
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float2 u0 = x[2 * q], u1 = x[2 * q + 1];
        if constexpr (PREC == kPrecFp16x3) {
            const float f = sc[q & 1];
            u0 = make_float2(u0.x * f, u0.y * f);
            u1 = make_float2(u1.x * f, u1.y * f);
        }
        split2<PREC>(u0.x, u1.x, ar[0][q], ar[1][q]);
        split2<PREC>(u0.y, u1.y, ai[0][q], ai[1][q]);
    }
    // forward: yr = xr C + xi S, yi = -xr S + xi C; inverse: the signs of S swapped
    constexpr uint32_t kFlipX = S < 0 ? 0u : 0x80008000u;   // xi -> yr: S or -S
    constexpr uint32_t kFlipY = S < 0 ? 0x80008000u : 0u;   // xr -> yi: -S or S
    float yr[2][4], yi[2][4];
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
        uint32_t bx[2][2], by[2][2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                bx[h][r] = B.s[h][nb][r] ^ kFlipX;
                by[h][r] = B.s[h][nb][r] ^ kFlipY;
            }
#pragma unroll
        for (int e = 0; e < 4; ++e) yr[nb][e] = yi[nb][e] = 0.f;
        mma16816<PREC>(yr[nb], ar[1], B.c[0][nb]);
        mma16816<PREC>(yr[nb], ai[1], bx[0]);
        mma16816<PREC>(yr[nb], ar[0], B.c[1][nb]);
        mma16816<PREC>(yr[nb], ai[0], bx[1]);
        mma16816<PREC>(yr[nb], ar[0], B.c[0][nb]);
        mma16816<PREC>(yr[nb], ai[0], bx[0]);
        mma16816<PREC>(yi[nb], ar[1], by[0]);
        mma16816<PREC>(yi[nb], ai[1], B.c[0][nb]);
        mma16816<PREC>(yi[nb], ar[0], by[1]);
        mma16816<PREC>(yi[nb], ai[0], B.c[1][nb]);
        mma16816<PREC>(yi[nb], ar[0], by[0]);
        mma16816<PREC>(yi[nb], ai[0], B.c[0][nb]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float re = yr[i >> 2][i & 3], im = yi[i >> 2][i & 3];
        if constexpr (PREC == kPrecFp16x3) {
            const float f = un[(i >> 1) & 1];
            re *= f;
            im *= f;
        }
        y[i] = make_float2(re, im);
    }
}

// Positions of this lane's fragment elements within a radix-16 pass: m-tile
// mt of warp w covers rows 16*(2w+mt) .. +15 of the tile's NB*Q groups, row r
// = column b * Q + group j.
template <int N, int NB>
struct TcTile {
    static constexpr int Q = N / 16;
    int b, j0;   // column and first group of the m-tile
    __device__ __forceinline__ TcTile(int warp, int mt)
    {
        const int row0 = 16 * (2 * warp + mt);
        b = row0 / Q;
        j0 = row0 % Q;
    }
    __device__ __forceinline__ int group(int lane, int i) const { return j0 + (lane >> 2) + 8 * ((i >> 1) & 1); }
    __device__ __forceinline__ static int point(int lane, int i) { return 2 * (lane & 3) + (i & 1) + 8 * (i >> 2); }
};

// Plain tile layout (as the TMA copies it): element e of column b at e*NB + b.
template <int NB>
struct PlainLayout {
    __device__ __forceinline__ static int at(int b, int e) { return e * NB + b; }
};

// One radix-16 Stockham pass (NS = product of the earlier radices) on the
// tensor cores: loads from IN (or, !LOAD, takes y as the input), twiddles,
// DFT-16, and -- unless KEEP -- the barrier and the stores to OUT.  KEEP
// leaves the results in y (the caller chains them; no barrier is passed).
template <int N, int NB, int PREC, int S, int NS, class IN, class OUT, bool KEEP = false, bool LOAD = true>
__device__ __forceinline__ void tc_pass16(float2 *buf, const float2 *__restrict__ tw, const Dft16B<PREC> &B,
                                          float2 (&y)[2][8])
{
    constexpr int Q = N / 16;
    constexpr int STEP = N / (NS * 16);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const TcTile<N, NB> T(warp, mt);
        float2 x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int j = T.group(lane, i), p = TcTile<N, NB>::point(lane, i);
            float2 v = LOAD ? buf[IN::at(T.b, j + p * Q)] : y[mt][i];
            if constexpr (NS > 1) {
                const int k = j % NS;
                float2 w = tw[(k * STEP * p) & (N - 1)];   // the shared-memory copy of the table
                if (S > 0) w.y = -w.y;
                v = cmul(v, w);
            }
            x[i] = v;
        }
        dft16_tc<PREC, S>(x, y[mt], B);
    }
    if constexpr (!KEEP) {
        __syncthreads();   // all loads of buf are complete
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const TcTile<N, NB> T(warp, mt);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int j = T.group(lane, i), q = TcTile<N, NB>::point(lane, i);
                const int k = j % NS;
                buf[OUT::at(T.b, (j - k) * 16 + k + q * NS)] = y[mt][i];
            }
        }
        __syncthreads();
    }
}

// Dynamic shared memory of k_col_tc: the stages of k_col_p16 and the
// length-N twiddle table.
template <int N, int NBT>
__host__ __device__ constexpr int pcol_tc_smem() { return pcol16_smem<N, NBT>() + N * 8; }

// Column pass with split-precision tensor-core stages.  MODE 0: forward
// FFT, modulus projection, inverse FFT (the shrink-wrap / HIO column pass);
// MODE 1: forward FFT only; MODE 2: inverse FFT only (kernel-level
// transforms).  Tile pipeline, modulus source and bounded waits as k_col_p16.
template <int N, int NBT, int PREC, int MODE>
__global__ void __launch_bounds__(pcol16_threads(N, NBT), 1) k_col_tc(const JobDev *jobs, const WorkList *L)
{
    extern __shared__ __align__(128) unsigned char sbuf[];
    constexpr int NB = NBT, V = 16, Q = N / V;
    constexpr int XB = NB * N * 8;
    constexpr int BR = pcol_box_rows(N);
    constexpr int STAGE = pcol16_stage_bytes<N, NBT>();
    constexpr int NST = pcol16_stages<N, NBT>();
    constexpr RadixList RL = reg16_radix_list(N);
    constexpr int R3 = RL.n > 2 ? RL.r[2] : 0;   // 0: two radix-16 passes only
    constexpr bool LAST16 = R3 == 0 || R3 == 16;
    static_assert(RL.n >= 2 && RL.r[0] == 16 && RL.r[1] == 16, "split-precision pass: N = 256 .. 4096");
    // NB*Q rows of groups, 16 per m-tile, 32 threads per warp: two m-tiles per warp
    static_assert(pcol16_threads(N, NBT) == NB * Q && (NB * Q) % 32 == 0 && Q % 16 == 0, "tile shape");
    using SWZ = ColSwz16<N, NB>;
    using PLN = PlainLayout<NB>;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sbuf);
    unsigned char *stages = sbuf + 128;
    const int b = threadIdx.x % NB, l = threadIdx.x / NB;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n_items = L->n;
    __shared__ int s_item[NST];

    LiveWalker walk(jobs, L);
    auto issue = [&](int item, int s) {   // one thread
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        unsigned char *st = stages + s * STAGE;
        const int x0 = wi.tile * NB;
        mbar_arrive_expect_tx(&bars[s], (uint32_t)XB);
        for (int r0 = 0; r0 < N; r0 += BR) tma_load_2d(st + (size_t)r0 * NB * 8, &J.tmX, x0, r0, &bars[s]);
    };

    int item = walk.next(blockIdx.x);
    Dft16B<PREC> B;
    B.init(lane);
    RegTw16<N> rtw;   // twiddles of the CUDA-core last pass
    float2 *tw = reinterpret_cast<float2 *>(stages + NST * STAGE);   // the table, copied once per CTA
    if (item < n_items) {
        const float2 *gtw = jobs[walk.at(item).job].pcol.tw;
        for (int i = threadIdx.x; i < N; i += pcol16_threads(N, NBT)) tw[i] = __ldg(gtw + i);
        if constexpr (!LAST16) rtw.load(gtw, l);
    }
    int it_next = n_items;
    if (threadIdx.x == 0) {
        for (int t = 0; t < NST; ++t) mbar_init(&bars[t], 1);
        mbar_fence_init();
        int it = item;
        for (int t = 0; t < NST - 1; ++t) {
            s_item[t] = it;
            if (it < n_items) {
                issue(it, t);
                it = walk.next(it + gridDim.x);
            }
        }
        it_next = it;
    }
    __syncthreads();
    for (int k = 0; item < n_items; ++k) {
        const int s = k % NST;
        const WorkItem wi = walk.at(item);
        const JobDev &J = jobs[wi.job];
        const bool guard = J.mode == kModeShrinkWrap;
        const bool landed = mbar_wait(&bars[s], (uint32_t)((k / NST) & 1), J.wait_ns);
        if (__syncthreads_or(!landed)) {
            if (threadIdx.x == 0) {
                atomicExch(&J.st->err, 1);
                for (int d = 0; d < NST - 1; ++d) {
                    const int t = (k + d) % NST;
                    if (d == 0 || s_item[t] < n_items) mbar_wait(&bars[t], (uint32_t)(((k + d) / NST) & 1), kDrainNs);
                }
                bulk_wait0();
            }
            return;
        }
        float2 *sX = reinterpret_cast<float2 *>(stages + s * STAGE);
        float2 y[2][8];
        float2 v[V];
        constexpr int SF = MODE == 2 ? +1 : -1;   // sign of the first transform
        // ---- first transform: two radix-16 passes on the tensor cores, then R3
        tc_pass16<N, NB, PREC, SF, 1, PLN, SWZ>(sX, tw, B, y);
        if constexpr (R3 == 0) {
            tc_pass16<N, NB, PREC, SF, 16, SWZ, SWZ, true>(sX, tw, B, y);
        } else if constexpr (R3 == 16) {
            tc_pass16<N, NB, PREC, SF, 16, SWZ, SWZ>(sX, tw, B, y);
            tc_pass16<N, NB, PREC, SF, 256, SWZ, SWZ, true>(sX, tw, B, y);
        } else {
            tc_pass16<N, NB, PREC, SF, 16, SWZ, SWZ>(sX, tw, B, y);
#pragma unroll
            for (int m = 0; m < V; ++m) v[m] = sX[SWZ::at(b, l + m * Q)];
            if constexpr (SF < 0) reg16_passes<N, SWZ, -1, 2, 256>(v, sX, b, l, rtw);
            else reg16_passes<N, SWZ, +1, 2, 256>(v, sX, b, l, rtw);
        }
        if (threadIdx.x == 0) {   // the stage of tile k - 1 is free: request tile k + NST - 1 there
            const int t = (k + NST - 1) % NST;
            s_item[t] = it_next;
            if (it_next < n_items) {
                bulk_wait_read0();
                fence_proxy_async_smem();
                issue(it_next, t);
                it_next = walk.next(it_next + gridDim.x);
            }
        }
        if constexpr (MODE == 0) {
            // ---- modulus projection (FP32), then the inverse transform
            const float *mt_base = J.Mt ? J.Mt + (size_t)wi.tile * NB * N : nullptr;
            const int W = J.W;
            if constexpr (LAST16) {
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    const TcTile<N, NB> T(warp, mt);
                    const int x = wi.tile * NB + T.b;
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int e = T.group(lane, i) + TcTile<N, NB>::point(lane, i) * Q;
                        const float mod = mt_base ? __ldg(mt_base + (size_t)e * NB + T.b)
                                                  : (x < W ? __ldg(J.M + (size_t)e * W + x) : 0.f);
                        const float f = modulus_factor(mod, y[mt][i], guard);
                        y[mt][i] = make_float2(__fmul_rn(y[mt][i].x, f), __fmul_rn(y[mt][i].y, f));
                    }
                }
                tc_pass16<N, NB, PREC, +1, 1, SWZ, SWZ, false, false>(sX, tw, B, y);
            } else {
                const int x = wi.tile * NB + b;
#pragma unroll
                for (int m = 0; m < V; ++m) {
                    const int e = l + m * Q;
                    const float mod = mt_base ? __ldg(mt_base + (size_t)e * NB + b)
                                              : (x < W ? __ldg(J.M + (size_t)e * W + x) : 0.f);
                    const float f = modulus_factor(mod, v[m], guard);
                    v[m] = make_float2(__fmul_rn(v[m].x, f), __fmul_rn(v[m].y, f));
                }
                __syncthreads();   // the last pass's loads of sX are complete
#pragma unroll
                for (int m = 0; m < V; ++m) sX[SWZ::at(b, l + m * Q)] = v[m];
                __syncthreads();
                tc_pass16<N, NB, PREC, +1, 1, SWZ, SWZ>(sX, tw, B, y);
            }
        }
        if constexpr (MODE == 0) {
            // second radix-16 pass and the last one of the inverse transform
            if constexpr (LAST16) {
                if constexpr (R3 == 16) {
                    tc_pass16<N, NB, PREC, +1, 16, SWZ, SWZ>(sX, tw, B, y);
                    tc_pass16<N, NB, PREC, +1, 256, SWZ, SWZ, true>(sX, tw, B, y);
                } else {
                    tc_pass16<N, NB, PREC, +1, 16, SWZ, SWZ, true>(sX, tw, B, y);
                }
            } else {
                tc_pass16<N, NB, PREC, +1, 16, SWZ, SWZ>(sX, tw, B, y);
#pragma unroll
                for (int m = 0; m < V; ++m) v[m] = sX[SWZ::at(b, l + m * Q)];
                reg16_passes<N, SWZ, +1, 2, 256>(v, sX, b, l, rtw);
            }
        }
        // ---- the result into the stage (plain tile layout), out by TMA
        __syncthreads();
        if constexpr (LAST16) {
            constexpr int NSL = N / 16;   // NS of the last radix-16 pass
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const TcTile<N, NB> T(warp, mt);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int j = T.group(lane, i), q = TcTile<N, NB>::point(lane, i);
                    sX[PLN::at(T.b, j + q * NSL)] = y[mt][i];
                }
            }
        } else {
#pragma unroll
            for (int m = 0; m < V; ++m) sX[PLN::at(b, l + m * Q)] = v[m];
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            const int x0 = wi.tile * NB;
            for (int r0 = 0; r0 < N; r0 += BR) tma_store_2d(&J.tmX, x0, r0, sX + (size_t)r0 * NB);
            bulk_commit();
        }
        item = s_item[(k + 1) % NST];
    }
    if (threadIdx.x == 0) bulk_wait0();
}

}  // namespace imr
