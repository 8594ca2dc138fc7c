// Device-side building blocks of the hand-written FFT for sm_100a.
//
// The transform is the unnormalised DFT
//     X[k] = sum_j x[j] * exp(S * 2*pi*i * j*k / n),  S = -1 forward, +1 inverse,
// i.e. what the reference obtains from cufftExecC2C(CUFFT_FORWARD / CUFFT_INVERSE)
// (src/imresh/algorithms/cuda/cudaShrinkWrap.cu:232,319,343) without any 1/n.
//
// Algorithm: Stockham autosort over mixed radices {8,4,2,3,5,7}, one pass per
// radix, natural order in and out.  Pass with radix R and current sub-length Ns:
//     v[q]  = buf[j + q*n/R] * w^(q*(j mod Ns)),   w = exp(S*2*pi*i/(Ns*R))
//     v     = DFT_R(v)
//     buf'[(j/Ns)*Ns*R + (j mod Ns) + q*Ns] = v[q]
// Each pass runs in place in shared memory: every thread first loads all of
// its butterflies' inputs into registers, the block synchronises, then every
// thread writes its outputs.  A thread owns at most VPT complex values per pass.
//
// Shared-memory layout of a batch of sequences: element e of sequence b lives
// at b*bs + e*es.  Row tiles use (bs = n, es = 1); column tiles use
// (bs = 1, es = ncols) so that one row of the tile is contiguous.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace imr {

struct FftPlanDev {
    int n;           // transform length
    int nrad;        // number of radix passes
    int rad[14];     // radices, first pass first
    const float2 *tw;  // exp(-2*pi*i*t/L), t < L, computed in double on the host; L = n, or bs_m
    // Bluestein (lengths with a prime factor > 7): the length-n DFT runs as a
    // convolution on the power-of-two length bs_m >= 2n - 1
    int bs_m;                // 0: direct transform
    const float2 *chirp;     // n entries: exp(-i*pi*j^2/n)
    const float2 *bspec_f;   // bs_m entries: FFT of the kernel for forward transforms, / bs_m
    const float2 *bspec_b;   // bs_m entries: the same for inverse transforms
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Complex add and subtract as one packed two-lane FP32 instruction each
// (add/sub.rn.f32x2 of sm_100): per lane the same IEEE round-to-nearest
// operation as the scalar form, half the instructions.
__device__ __forceinline__ unsigned long long f2pack(float2 a)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f2unpack(unsigned long long r)
{
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(r);
}
__device__ __forceinline__ float2 csub(float2 a, float2 b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(r);
}
// a + S*i*d and a - S*i*d: (a.x -+ S d.y, a.y +- S d.x), one packed fma with
// exact +-1 factors each (a single rounding, as the scalar subtraction).
template <int S>
__device__ __forceinline__ void cadd_sub_si(float2 a, float2 d, float2 &plus, float2 &minus)
{
    const unsigned long long sw = f2pack(make_float2(d.y, d.x)), pa = f2pack(a);
    const unsigned long long kp = f2pack(make_float2((float)-S, (float)S)), km = f2pack(make_float2((float)S, (float)-S));
    unsigned long long rp, rm;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rp) : "l"(sw), "l"(kp), "l"(pa));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(rm) : "l"(sw), "l"(km), "l"(pa));
    plus = f2unpack(rp);
    minus = f2unpack(rm);
}
// multiply by S*i
template <int S>
__device__ __forceinline__ float2 mul_si(float2 a) { return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }

// ---- radix-R DFTs on registers, sign S --------------------------------------
template <int S>
__device__ __forceinline__ void dft2(float2 *v)
{
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <int S>
__device__ __forceinline__ void dft4(float2 *v)
{
    float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    float2 a2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    cadd_sub_si<S>(a1, d, v[1], v[3]);   // a1 +- S i d
}

template <int S>
__device__ __forceinline__ void dft8(float2 *v)
{
    const float c = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<S>(e);
    dft4<S>(o);
    // w^1 = c*(1 + S i), w^2 = S i, w^3 = c*(-1 + S i)
    float2 o1 = make_float2(c * (o[1].x - S * o[1].y), c * (S * o[1].x + o[1].y));
    float2 o3 = make_float2(c * (-o[3].x - S * o[3].y), c * (S * o[3].x - o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    cadd_sub_si<S>(e[2], o[2], v[2], v[6]);   // e2 +- S i o2
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
}

// 16 points as 4 x 4: DFT4 over n1 of x[4 n1 + n2], twiddle W16^(n2 k1),
// DFT4 over n2; output k1 + 4 k2.
template <int S>
__device__ __forceinline__ void dft16(float2 *v)
{
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;   // cos, sin(pi/8)
    const float h = 0.70710678118654752440f;
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        float2 a[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
        dft4<S>(a);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = a[k1];
    }
    // W16^e = cos(2 pi e/16) + S i sin(2 pi e/16), e = n2*k1 in {1,2,3,4,6,9}
    y[1][1] = cmul(y[1][1], make_float2(c1, S * s1));
    y[1][2] = make_float2(h * (y[1][2].x - S * y[1][2].y), h * (S * y[1][2].x + y[1][2].y));
    y[1][3] = cmul(y[1][3], make_float2(s1, S * c1));
    y[2][1] = make_float2(h * (y[2][1].x - S * y[2][1].y), h * (S * y[2][1].x + y[2][1].y));
    y[2][2] = mul_si<S>(y[2][2]);
    y[2][3] = make_float2(h * (-y[2][3].x - S * y[2][3].y), h * (S * y[2][3].x - y[2][3].y));
    y[3][1] = cmul(y[3][1], make_float2(s1, S * c1));
    y[3][2] = make_float2(h * (-y[3][2].x - S * y[3][2].y), h * (S * y[3][2].x - y[3][2].y));
    y[3][3] = cmul(y[3][3], make_float2(-c1, -S * s1));
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 b[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
        dft4<S>(b);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = b[k2];
    }
}

// The twiddle W16^(n2 k1) of element (n2, k1) of dft16's 4 x 4 step, by the
// same expression dft16 uses for it (identity for n2 = 0 or k1 = 0).
template <int S, int N2, int K1>
__device__ __forceinline__ float2 dft16_tw(float2 y)
{
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;   // cos, sin(pi/8)
    const float h = 0.70710678118654752440f;
    if constexpr (N2 == 0 || K1 == 0) return y;
    else if constexpr (N2 * K1 == 1) return cmul(y, make_float2(c1, S * s1));
    else if constexpr (N2 * K1 == 2) return make_float2(h * (y.x - S * y.y), h * (S * y.x + y.y));
    else if constexpr (N2 * K1 == 3) return cmul(y, make_float2(s1, S * c1));
    else if constexpr (N2 * K1 == 4) return mul_si<S>(y);
    else if constexpr (N2 * K1 == 6) return make_float2(h * (-y.x - S * y.y), h * (S * y.x - y.y));
    else return cmul(y, make_float2(-c1, -S * s1));   // 9
}

// dft16 split over two threads, H = 0 or 1: the thread holds u[j] = v[2j + H]
// of dft16's v and ends holding the outputs v'[2j + H].  Part A: the DFT-4s
// over n1 of rows n2 = H and H + 2 (inputs 4 n1 + n2 = 2j + H); their values in
// the other parity's columns k1 = 1 - H, 3 - H go to the partner through `out`
// (4 slots, `stride` apart) before twiddling.  Part B (after a barrier): the
// partner's rows at columns k1 = H, H + 2 come from `in`; every element of
// those columns is twiddled here, in the thread that sums it, as dft16 does,
// and the DFT-4s over n2 give the outputs k1 + 4 k2 = 2j + H.
template <int S, int H>
__device__ __forceinline__ void dft16_half_a(const float2 (&u)[8], float2 (&ya)[4], float2 (&yb)[4], float2 *out,
                                             int stride)
{
    ya[0] = u[0]; ya[1] = u[2]; ya[2] = u[4]; ya[3] = u[6];   // row n2 = H
    yb[0] = u[1]; yb[1] = u[3]; yb[2] = u[5]; yb[3] = u[7];   // row n2 = H + 2
    dft4<S>(ya);
    dft4<S>(yb);
    out[0] = ya[1 - H];
    out[stride] = ya[3 - H];
    out[2 * stride] = yb[1 - H];
    out[3 * stride] = yb[3 - H];
}
template <int S, int H, int T>
__device__ __forceinline__ void dft16_half_col(float2 (&u)[8], const float2 (&ya)[4], const float2 (&yb)[4],
                                               float2 pa, float2 pb)
{
    constexpr int K1 = H + 2 * T;
    float2 b[4];
    if constexpr (H == 0) {
        b[0] = ya[K1];
        b[1] = dft16_tw<S, 1, K1>(pa);
        b[2] = dft16_tw<S, 2, K1>(yb[K1]);
        b[3] = dft16_tw<S, 3, K1>(pb);
    } else {
        b[0] = pa;
        b[1] = dft16_tw<S, 1, K1>(ya[K1]);
        b[2] = dft16_tw<S, 2, K1>(pb);
        b[3] = dft16_tw<S, 3, K1>(yb[K1]);
    }
    dft4<S>(b);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) u[T + 2 * k2] = b[k2];
}
template <int S, int H>
__device__ __forceinline__ void dft16_half_b(float2 (&u)[8], const float2 (&ya)[4], const float2 (&yb)[4],
                                             const float2 *in, int stride)
{
    // the partner's rows n2 = 1 - H (pa) and 3 - H (pb) at columns H, H + 2
    const float2 pa0 = in[0], pa1 = in[stride], pb0 = in[2 * stride], pb1 = in[3 * stride];
    dft16_half_col<S, H, 0>(u, ya, yb, pa0, pb0);
    dft16_half_col<S, H, 1>(u, ya, yb, pa1, pb1);
}

template <int S>
__device__ __forceinline__ void dft3(float2 *v)
{
    const float h = 0.86602540378443864676f;  // sin(2pi/3)
    float2 t = cadd(v[1], v[2]);
    float2 d = csub(v[1], v[2]);
    float2 y0 = cadd(v[0], t);
    float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    float2 r = mul_si<S>(make_float2(h * d.x, h * d.y));
    v[0] = y0;
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

template <int S>
__device__ __forceinline__ void dft5(float2 *v)
{
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 d1 = csub(v[1], v[4]), d2 = csub(v[2], v[3]);
    float2 y0 = cadd(v[0], cadd(t1, t2));
    float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 b1 = mul_si<S>(make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y));
    float2 b2 = mul_si<S>(make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y));
    v[0] = y0;
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
}

template <int S>
__device__ __forceinline__ void dft7(float2 *v)
{
    // cos(2 pi k/7), sin(2 pi k/7), k = 1..3
    const float c[3] = {0.62348980185873353053f, -0.22252093395631440429f, -0.90096886790241912624f};
    const float s[3] = {0.78183148246802980871f, 0.97492791218182360702f, 0.43388373911755812048f};
    float2 t[3], d[3];
    for (int k = 0; k < 3; ++k) {
        t[k] = cadd(v[1 + k], v[6 - k]);
        d[k] = csub(v[1 + k], v[6 - k]);
    }
    float2 y[7];
    y[0] = cadd(v[0], cadd(t[0], cadd(t[1], t[2])));
#pragma unroll
    for (int m = 1; m <= 3; ++m) {
        float2 a = v[0], b = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            int idx = (m * k) % 7;               // angle 2 pi m k / 7
            float cc = idx <= 3 ? c[idx - 1] : c[7 - idx - 1];
            float ss = idx <= 3 ? s[idx - 1] : -s[7 - idx - 1];
            a.x += cc * t[k - 1].x;
            a.y += cc * t[k - 1].y;
            b.x += ss * d[k - 1].x;
            b.y += ss * d[k - 1].y;
        }
        float2 r = mul_si<S>(b);
        y[m] = cadd(a, r);
        y[7 - m] = csub(a, r);
    }
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = y[k];
}

// 12 points by the prime-factor (Good-Thomas) split 3 x 4, which needs no
// twiddles: input index n = (4 n1 + 3 n2) mod 12, DFT-3 over n1, DFT-4 over n2,
// output index k = (4 k1 + 9 k2) mod 12 (k1 = k mod 3, k2 = k mod 4), since
// n k = 4 n1 k1 + 3 n2 k2 (mod 12).
template <int S>
__device__ __forceinline__ void dft12(float2 *v)
{
    float2 A[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        float2 a[3] = {v[(3 * n2) % 12], v[(4 + 3 * n2) % 12], v[(8 + 3 * n2) % 12]};
        dft3<S>(a);
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) A[n2][k1] = a[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
        float2 b[4] = {A[0][k1], A[1][k1], A[2][k1], A[3][k1]};
        dft4<S>(b);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[(4 * k1 + 9 * k2) % 12] = b[k2];
    }
}

template <int R, int S>
__device__ __forceinline__ void dftR(float2 *v)
{
    if constexpr (R == 2) dft2<S>(v);
    else if constexpr (R == 3) dft3<S>(v);
    else if constexpr (R == 4) dft4<S>(v);
    else if constexpr (R == 5) dft5<S>(v);
    else if constexpr (R == 7) dft7<S>(v);
    else if constexpr (R == 16) dft16<S>(v);
    else if constexpr (R == 12) dft12<S>(v);
    else dft8<S>(v);
}

// ---- one Stockham pass, in place in shared memory ---------------------------
// nb sequences; butterfly u -> (sequence b, index j).  seq_fast: adjacent
// threads take adjacent sequences (column tiles); otherwise adjacent j (rows).
template <int R, int S, int VPT>
__device__ __forceinline__ void stockham_pass(float2 *buf, const FftPlanDev &p, int Ns, int nb,
                                              int bs, int es, bool seq_fast, int tid, int nthr)
{
    constexpr int BPT = (VPT + R - 1) / R;
    const int n = p.n;
    const int m = n / R;
    const int total = nb * m;
    const int step = n / (Ns * R);
    float2 v[BPT][R];
    int dst[BPT];
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        const int u = tid + i * nthr;
        dst[i] = -1;
        if (u < total) {
            int b, j;
            if (seq_fast) { b = u % nb; j = u / nb; }
            else          { j = u % m;  b = u / m; }
            const int k = j % Ns;
            const float2 *src = buf + b * bs + j * es;
#pragma unroll
            for (int q = 0; q < R; ++q) v[i][q] = src[q * m * es];
            if (k != 0) {
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    float2 w = __ldg(p.tw + q * k * step);
                    if (S > 0) w.y = -w.y;
                    v[i][q] = cmul(v[i][q], w);
                }
            }
            dftR<R, S>(v[i]);
            dst[i] = b * bs + ((j - k) * R + k) * es;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        if (dst[i] >= 0) {
#pragma unroll
            for (int q = 0; q < R; ++q) buf[dst[i] + q * Ns * es] = v[i][q];
        }
    }
    __syncthreads();
}

// ---- compile-time schedule -------------------------------------------------
// Radix schedule of length N: 8s first (then 4,4 / 4 / 2 for the remaining
// power of two), then 3s, 5s, 7s.  Must match factor_len() on the host.
struct RadixList {
    int n;
    int r[14];
};
__host__ __device__ constexpr RadixList radix_list(int N)
{
    RadixList L{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    int m = N, k = 0;
    while (m % 2 == 0) { m /= 2; ++k; }
    while (k >= 3 && k != 4) { L.r[L.n++] = 8; k -= 3; }
    if (k == 4) { L.r[L.n++] = 4; L.r[L.n++] = 4; }
    else if (k == 2) L.r[L.n++] = 4;
    else if (k == 1) L.r[L.n++] = 2;
    while (m % 3 == 0) { L.r[L.n++] = 3; m /= 3; }
    while (m % 5 == 0) { L.r[L.n++] = 5; m /= 5; }
    while (m % 7 == 0) { L.r[L.n++] = 7; m /= 7; }
    if (m != 1) L.n = -1;
    return L;
}

// One Stockham pass with every size known at compile time.  NB sequences of
// length N, T threads; SEQ_FAST selects the column-tile layout (es = NB).
template <int N, int NB, int T, int R, int NS, int S, bool SEQ_FAST>
__device__ __forceinline__ void ct_pass(float2 *buf, int nb, const float2 *__restrict__ tw)
{
    constexpr int M = N / R;
    constexpr int TOTAL = NB * M;
    constexpr int BPT = (TOTAL + T - 1) / T;
    constexpr int STEP = N / (NS * R);
    constexpr int BS = SEQ_FAST ? 1 : N;
    constexpr int ES = SEQ_FAST ? NB : 1;
    float2 v[BPT][R];
    int dst[BPT];
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        const int u = threadIdx.x + i * T;
        dst[i] = -1;
        int b, j;
        if (SEQ_FAST) { b = u % NB; j = u / NB; }
        else          { j = u % M;  b = u / M; }
        if ((TOTAL % T == 0 || u < TOTAL) && b < nb) {
            const int k = j % NS;
            const float2 *src = buf + b * BS + j * ES;
#pragma unroll
            for (int q = 0; q < R; ++q) v[i][q] = src[q * M * ES];
            if (NS > 1 && k != 0) {
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    float2 w = __ldg(tw + q * k * STEP);
                    if (S > 0) w.y = -w.y;
                    v[i][q] = cmul(v[i][q], w);
                }
            }
            dftR<R, S>(v[i]);
            dst[i] = b * BS + ((j - k) * R + k) * ES;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        if (dst[i] >= 0) {
#pragma unroll
            for (int q = 0; q < R; ++q) buf[dst[i] + q * NS * ES] = v[i][q];
        }
    }
    __syncthreads();
}

template <int N, int NB, int T, int S, bool SEQ_FAST, int P, int NS>
__device__ __forceinline__ void ct_passes(float2 *buf, int nb, const float2 *__restrict__ tw)
{
    constexpr RadixList L = radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        ct_pass<N, NB, T, R, NS, S, SEQ_FAST>(buf, nb, tw);
        ct_passes<N, NB, T, S, SEQ_FAST, P + 1, NS * R>(buf, nb, tw);
    }
}

// Transform of nb <= NB sequences of compile-time length N in shared memory:
// rows (SEQ_FAST = false): element e of sequence b at b*N + e;
// column tiles (SEQ_FAST = true): element e of sequence b at e*NB + b.
// Ends with a __syncthreads().
template <int N, int NB, int T, int S, bool SEQ_FAST>
__device__ __forceinline__ void ct_fft(float2 *buf, int nb, const float2 *__restrict__ tw)
{
    static_assert(radix_list(N).n > 0, "length must factor into 2, 3, 5, 7");
    ct_passes<N, NB, T, S, SEQ_FAST, 0, 1>(buf, nb, tw);
}

// ---- Bluestein -------------------------------------------------------------
// X[k] = c_k * sum_j (x_j c_j) conj(c_{k-j}),  c_j = exp(S*i*pi*j^2/n)
//      = c_k * IFFT_M( FFT_M(a) * FFT_M(b) )[k],  a_j = x_j c_j (zero padded),
// b the kernel conj(c_j) wrapped on the M grid; FFT_M(b)/M is precomputed
// (bspec_f for S = -1, bspec_b for S = +1).  nb sequences: data element
// (b, j) at b*dbs + j*des, work element (b, j) at the compile-time layout of
// ct_fft<M, NB, T, ., SEQ_FAST>.  Ends with a barrier.
template <int M, int NB, int T, int S, bool SEQ_FAST>
__device__ __forceinline__ void bluestein(float2 *data, int dbs, int des, float2 *work, int nb,
                                          const FftPlanDev &p)
{
    const int n = p.n;
    constexpr int WBS = SEQ_FAST ? 1 : M;
    constexpr int WES = SEQ_FAST ? NB : 1;
    for (int idx = threadIdx.x; idx < NB * M; idx += T) {
        int b, j;
        if (SEQ_FAST) { b = idx % NB; j = idx / NB; }
        else          { j = idx % M;  b = idx / M; }
        float2 v = make_float2(0.f, 0.f);
        if (b < nb && j < n) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            v = cmul(data[b * dbs + j * des], c);
        }
        work[b * WBS + j * WES] = v;
    }
    __syncthreads();
    ct_fft<M, NB, T, -1, SEQ_FAST>(work, nb, p.tw);
    const float2 *spec = S < 0 ? p.bspec_f : p.bspec_b;
    for (int idx = threadIdx.x; idx < NB * M; idx += T) {
        int b, j;
        if (SEQ_FAST) { b = idx % NB; j = idx / NB; }
        else          { j = idx % M;  b = idx / M; }
        work[b * WBS + j * WES] = cmul(work[b * WBS + j * WES], __ldg(spec + j));
    }
    __syncthreads();
    ct_fft<M, NB, T, +1, SEQ_FAST>(work, nb, p.tw);
    for (int idx = threadIdx.x; idx < NB * n; idx += T) {
        int b, j;
        if (SEQ_FAST) { b = idx % NB; j = idx / NB; }
        else          { j = idx % n;  b = idx / n; }
        if (b < nb) {
            float2 c = __ldg(p.chirp + j);
            if (S > 0) c.y = -c.y;
            data[b * dbs + j * des] = cmul(work[b * WBS + j * WES], c);
        }
    }
    __syncthreads();
}

// Full transform of nb sequences held in shared memory (see layout above).
// Requires nb * n <= VPT * nthr.  Ends with a __syncthreads().
template <int S, int VPT>
__device__ void fft_smem(float2 *buf, const FftPlanDev &p, int nb, int bs, int es, bool seq_fast,
                         int tid, int nthr)
{
    int Ns = 1;
    for (int i = 0; i < p.nrad; ++i) {
        const int R = p.rad[i];
        switch (R) {
        case 8: stockham_pass<8, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        case 4: stockham_pass<4, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        case 2: stockham_pass<2, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        case 3: stockham_pass<3, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        case 5: stockham_pass<5, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        default: stockham_pass<7, S, VPT>(buf, p, Ns, nb, bs, es, seq_fast, tid, nthr); break;
        }
        Ns *= R;
    }
}

}  // namespace imr
