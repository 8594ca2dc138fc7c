// Register-resident FFT for power-of-two lengths (sm_100a).
//
// A sequence of length N is owned by Q = N/8 threads; thread l holds the
// eight values at positions l + m*Q (m = 0..7) in v[m], before and after the
// transform (natural order).  Each Stockham pass (radix R in {8,4,2}) runs
// 8/R butterflies per thread entirely in registers; between passes the
// values go through shared memory once (store, barrier, load), so a length
// 2048 transform (radices 8,8,8,4) costs three shared-memory exchanges.
// Because input and output sit at the same positions l + m*Q, an inverse
// transform, a point-wise update and a forward transform chain in registers,
// and global loads / stores are coalesced across the Q threads.
//
// Shared memory: two buffers (ping-pong, one barrier per exchange) of
// padded length N + N/8 per sequence; the pad of one element per eight
// spreads the strided stores of the early passes over all banks.
#pragma once
#include "fft_dev.cuh"

namespace imr {

__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Lengths the pipelined register FFT handles: powers of two (8 values per
// thread, radices 8/4/2) and 3 * 2^k (12 values per thread, radices 12/4/2).
__host__ __device__ constexpr bool is_3pow2(int n) { return n >= 48 && n % 3 == 0 && is_pow2(n / 3); }
__host__ __device__ constexpr int reg_v(int n) { return is_pow2(n) ? 8 : 12; }
__host__ __device__ constexpr RadixList reg_radix_list(int n)
{
    if (is_pow2(n)) return radix_list(n);
    RadixList L{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    int k = 0, m = n % 12 == 0 ? n / 12 : n / 3;
    while (m > 1) { m >>= 1; ++k; }
    // 3*2^k >= 12: a first, twiddle-free radix-12 pass (prime-factor 3 x 4),
    // then radix 4 and at most one radix 2 -- one pass, and one shared-memory
    // exchange, fewer than radix 4 ... 4, 3
    if (n % 12 == 0) L.r[L.n++] = 12;
    for (; k >= 2; k -= 2) L.r[L.n++] = 4;
    if (k == 1) L.r[L.n++] = 2;
    if (n % 12 != 0) L.r[L.n++] = 3;
    return L;
}

// padded index of element e
__device__ __forceinline__ int pad8(int e) { return e + (e >> 3); }

// Layout of NB sequences in one shared-memory buffer.
//  rows:    sequence b at b*(N + N/8), element e at pad8(e)
//  columns: element e of sequence b at pad8(e)*NB + b (one tile row contiguous)
template <int N, int NB, bool COLS>
struct SmemLayout {
    static constexpr int kBuf = NB * (N + N / 8);   // float2 per buffer
    __device__ __forceinline__ static int at(int b, int e)
    {
        if constexpr (COLS) return pad8(e) * NB + b;
        else return b * (N + N / 8) + pad8(e);
    }
};

// v[i] *= w^i for i = 1..R-1, w = table[t] (conjugated for S > 0); w^2 and
// w^4 come from the table, the other powers from one product each.
template <int R, int S, bool SMEM_TW = false>
__device__ __forceinline__ void twiddle(float2 *u, const float2 *__restrict__ tw, int t, int n)
{
    if (t == 0) return;
    auto ld = [&](int idx) {
        float2 w = SMEM_TW ? tw[idx] : __ldg(tw + idx);
        if (S > 0) w.y = -w.y;
        return w;
    };
    const float2 w1 = ld(t);
    if constexpr (R == 2) {
        u[1] = cmul(u[1], w1);
    } else if constexpr (R == 3) {
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], ld(2 * t));
    } else if constexpr (R == 4) {
        const float2 w2 = ld(2 * t);
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], cmul(w1, w2));
    } else {
        const float2 w2 = ld(2 * t), w4 = ld(4 * t);
        const float2 w3 = cmul(w1, w2);
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], w3);
        u[4] = cmul(u[4], w4);
        u[5] = cmul(u[5], cmul(w1, w4));
        u[6] = cmul(u[6], cmul(w2, w4));
        u[7] = cmul(u[7], cmul(w3, w4));
    }
    (void)n;
}

template <int N, int NB, bool COLS, int S, int P, int NS>
__device__ __forceinline__ void reg_passes(float2 (&v)[8], float2 *buf0, float2 *buf1, int b, int l,
                                           const float2 *__restrict__ tw)
{
    constexpr RadixList L = radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        constexpr int BPT = 8 / R;
        constexpr int Q = N / 8;
        constexpr int STEP = N / (NS * R);
        static_assert(R == 2 || R == 4 || R == 8, "power-of-two radices only");
        int kk[BPT];
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int j = l + i * Q;
            const int k = j & (NS - 1);
            kk[i] = k;
            float2 u[R];
#pragma unroll
            for (int q = 0; q < R; ++q) u[q] = v[i + q * BPT];
            if constexpr (NS > 1) twiddle<R, S>(u, tw, k * STEP, N);
            dftR<R, S>(u);
#pragma unroll
            for (int q = 0; q < R; ++q) v[i + q * BPT] = u[q];
        }
        if constexpr (P + 1 < L.n) {
            using A = SmemLayout<N, NB, COLS>;
            float2 *buf = (P & 1) ? buf1 : buf0;
#pragma unroll
            for (int i = 0; i < BPT; ++i) {
                const int j = l + i * Q;
                const int base = (j - kk[i]) * R + kk[i];
#pragma unroll
                for (int q = 0; q < R; ++q) buf[A::at(b, base + q * NS)] = v[i + q * BPT];
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < 8; ++m) v[m] = buf[A::at(b, l + m * Q)];
            reg_passes<N, NB, COLS, S, P + 1, NS * R>(v, buf0, buf1, b, l, tw);
        }
    }
}

// Unnormalised transform of the sequence held in v (see top of file).
// Ends with a barrier, so the buffers may be reused right after.
template <int N, int NB, bool COLS, int S>
__device__ __forceinline__ void reg_fft(float2 (&v)[8], float2 *smem, int b, int l,
                                        const float2 *__restrict__ tw)
{
    static_assert(is_pow2(N) && N >= 8, "register FFT needs a power-of-two length >= 8");
    float2 *buf0 = smem;
    float2 *buf1 = smem + SmemLayout<N, NB, COLS>::kBuf;
    reg_passes<N, NB, COLS, S, 0, 1>(v, buf0, buf1, b, l, tw);
    __syncthreads();
}

// ---- single-buffer variant with XOR-swizzled layouts -------------------------
// Used by the pipelined kernels, whose exchange buffer is the TMA stage the
// data arrived in.  Swizzles chosen by simulating the bank pattern of every
// exchange (all power-of-two lengths, 8-byte accesses served per half warp):
// conflict-free, no padding.
//  rows:    sequence b at b*N, element e at e ^ ((e >> 3) & 15)
//  columns: element e of sequence b at (e ^ ((e >> 3) & (16/NB - 1)))*NB + b
template <int N, int NB>
struct RowSwz {
    __device__ __forceinline__ static int at(int b, int e) { return b * N + (e ^ ((e >> 3) & 15)); }
};
template <int N, int NB>
struct ColSwz {
    static_assert(NB >= 1 && NB <= 16 && 16 % NB == 0, "column tile width must divide 16");
    __device__ __forceinline__ static int at(int b, int e) { return (e ^ ((e >> 3) & (16 / NB - 1))) * NB + b; }
};

// ---- per-thread twiddles, loaded once per kernel ----------------------------
// In pass P (sub-length NS) butterfly i of thread l uses powers of
// w = tw[((l + i*N/8) mod NS) * N/(NS*R)].  When NS divides N/8 the base does
// not depend on i, otherwise each of the 8/R butterflies has its own.  A
// persistent kernel keeps the bases in registers for all its work items and
// forms w^2..w^7 by products (see twiddle_reg).
__host__ __device__ constexpr int tw_slots_upto(int N, int P)
{
    RadixList L = reg_radix_list(N);
    const int V = reg_v(N), Q = N / reg_v(N);
    int slots = 0, ns = 1;
    for (int p = 0; p < P && p < L.n; ++p) {
        if (p > 0) slots += (Q % ns == 0) ? 1 : V / L.r[p];
        ns *= L.r[p];
    }
    return slots;
}
__host__ __device__ constexpr int tw_slots(int N) { return tw_slots_upto(N, reg_radix_list(N).n); }

template <int N>
struct RegTw {
    float2 w[tw_slots(N) > 0 ? tw_slots(N) : 1];

    template <int P, int NS>
    __device__ __forceinline__ void load_pass(const float2 *__restrict__ tw, int l)
    {
        constexpr RadixList L = reg_radix_list(N);
        if constexpr (P < L.n) {
            constexpr int R = L.r[P];
            constexpr int V = reg_v(N);
            constexpr int Q = N / V;
            if constexpr (P > 0) {
                constexpr int off = tw_slots_upto(N, P);
                constexpr int STEP = N / (NS * R);
                if constexpr (Q % NS == 0) {
                    w[off] = __ldg(tw + (l % NS) * STEP);
                } else {
#pragma unroll
                    for (int i = 0; i < V / R; ++i) w[off + i] = __ldg(tw + ((l + i * Q) % NS) * STEP);
                }
            }
            load_pass<P + 1, NS * R>(tw, l);
        }
    }
    __device__ __forceinline__ void load(const float2 *__restrict__ tw, int l) { load_pass<0, 1>(tw, l); }
};

// u[q] *= w^q, q = 1..R-1, from the base w (conjugated for S > 0).  The
// empty asm makes the base opaque at each use, so the compiler recomputes
// the powers instead of hoisting all of them out of the work-item loop
// (which would keep ~50 more values live per thread).
template <int R, int S>
__device__ __forceinline__ void twiddle_reg(float2 *u, float2 w1)
{
    asm volatile("" : "+f"(w1.x), "+f"(w1.y));
    if (S > 0) w1.y = -w1.y;
    if constexpr (R == 2) {
        u[1] = cmul(u[1], w1);
    } else if constexpr (R == 3) {
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], cmul(w1, w1));
    } else if constexpr (R == 4) {
        const float2 w2 = cmul(w1, w1);
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], cmul(w1, w2));
    } else {
        const float2 w2 = cmul(w1, w1), w4 = cmul(w2, w2);
        const float2 w3 = cmul(w1, w2);
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], w3);
        u[4] = cmul(u[4], w4);
        u[5] = cmul(u[5], cmul(w1, w4));
        u[6] = cmul(u[6], cmul(w2, w4));
        u[7] = cmul(u[7], cmul(w3, w4));
    }
}

template <int N, class LAYOUT, int S, int P, int NS>
__device__ __forceinline__ void reg_passes_1buf_rt(float2 (&v)[reg_v(N)], float2 *buf, int b, int l,
                                                   const RegTw<N> &tw)
{
    constexpr RadixList L = reg_radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        constexpr int V = reg_v(N);
        constexpr int BPT = V / R;
        constexpr int Q = N / V;
        int kk[BPT];
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int j = l + i * Q;
            const int k = j % NS;
            kk[i] = k;
            float2 u[R];
#pragma unroll
            for (int q = 0; q < R; ++q) u[q] = v[i + q * BPT];
            if constexpr (NS > 1) {
                constexpr int off = tw_slots_upto(N, P);
                twiddle_reg<R, S>(u, tw.w[off + (Q % NS == 0 ? 0 : i)]);
            }
            dftR<R, S>(u);
#pragma unroll
            for (int q = 0; q < R; ++q) v[i + q * BPT] = u[q];
        }
        if constexpr (P + 1 < L.n) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < BPT; ++i) {
                const int j = l + i * Q;
                const int base = (j - kk[i]) * R + kk[i];
#pragma unroll
                for (int q = 0; q < R; ++q) buf[LAYOUT::at(b, base + q * NS)] = v[i + q * BPT];
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < V; ++m) v[m] = buf[LAYOUT::at(b, l + m * Q)];
            reg_passes_1buf_rt<N, LAYOUT, S, P + 1, NS * R>(v, buf, b, l, tw);
        }
    }
}

// As reg_fft_1buf, with the twiddles already in registers.
template <int N, class LAYOUT, int S>
__device__ __forceinline__ void reg_fft_1buf(float2 (&v)[reg_v(N)], float2 *buf, int b, int l,
                                             const RegTw<N> &tw)
{
    static_assert((is_pow2(N) && N >= 16) || is_3pow2(N), "pipelined FFT length: 2^k >= 16 or 3*2^k >= 48");
    reg_passes_1buf_rt<N, LAYOUT, S, 0, 1>(v, buf, b, l, tw);
}

template <int N, class LAYOUT, int S, int P, int NS, bool SMEM_TW>
__device__ __forceinline__ void reg_passes_1buf(float2 (&v)[reg_v(N)], float2 *buf, int b, int l,
                                                const float2 *__restrict__ tw)
{
    constexpr RadixList L = reg_radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        constexpr int V = reg_v(N);
        constexpr int BPT = V / R;
        constexpr int Q = N / V;
        constexpr int STEP = N / (NS * R);
        int kk[BPT];
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int j = l + i * Q;
            const int k = j % NS;
            kk[i] = k;
            float2 u[R];
#pragma unroll
            for (int q = 0; q < R; ++q) u[q] = v[i + q * BPT];
            if constexpr (NS > 1) twiddle<R, S, SMEM_TW>(u, tw, k * STEP, N);
            dftR<R, S>(u);
#pragma unroll
            for (int q = 0; q < R; ++q) v[i + q * BPT] = u[q];
        }
        if constexpr (P + 1 < L.n) {
            __syncthreads();   // earlier reads of buf are complete
#pragma unroll
            for (int i = 0; i < BPT; ++i) {
                const int j = l + i * Q;
                const int base = (j - kk[i]) * R + kk[i];
#pragma unroll
                for (int q = 0; q < R; ++q) buf[LAYOUT::at(b, base + q * NS)] = v[i + q * BPT];
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < V; ++m) v[m] = buf[LAYOUT::at(b, l + m * Q)];
            reg_passes_1buf<N, LAYOUT, S, P + 1, NS * R, SMEM_TW>(v, buf, b, l, tw);
        }
    }
}

// tw: the length-N twiddle table, in global memory or (SMEM_TW) shared memory.
template <int N, class LAYOUT, int S, bool SMEM_TW = false>
__device__ __forceinline__ void reg_fft_1buf(float2 (&v)[reg_v(N)], float2 *buf, int b, int l,
                                             const float2 *__restrict__ tw)
{
    static_assert((is_pow2(N) && N >= 16) || is_3pow2(N), "pipelined FFT length: 2^k >= 16 or 3*2^k >= 48");
    reg_passes_1buf<N, LAYOUT, S, 0, 1, SMEM_TW>(v, buf, b, l, tw);
}

// ---- 16 values per thread (powers of two >= 128) -----------------------------
// Thread l of a sequence holds positions l + m*N/16, m = 0..15; passes of
// radix 16 first, then one pass of the remaining 2, 4 or 8.  A length-2048
// transform (16, 16, 8) costs two shared-memory exchanges instead of the
// three of the 8-value form, and a third fewer barriers.
__host__ __device__ constexpr RadixList reg16_radix_list(int n)
{
    RadixList L{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
    int k = 0;
    while ((1 << k) < n) ++k;
    for (; k >= 4; k -= 4) L.r[L.n++] = 16;
    if (k > 0) L.r[L.n++] = 1 << k;
    return L;
}
__host__ __device__ constexpr int tw16_slots_upto(int N, int P)
{
    RadixList L = reg16_radix_list(N);
    const int Q = N / 16;
    int slots = 0, ns = 1;
    for (int p = 0; p < P && p < L.n; ++p) {
        if (p > 0) slots += (Q % ns == 0) ? 1 : 16 / L.r[p];
        ns *= L.r[p];
    }
    return slots;
}
__host__ __device__ constexpr int tw16_slots(int N) { return tw16_slots_upto(N, reg16_radix_list(N).n); }

// Per-thread twiddle powers w, w^2, w^4, w^8 of every butterfly base, read
// from the length-N table once per kernel (they depend only on l).
template <int N>
struct RegTw16 {
    float2 w[tw16_slots(N) > 0 ? tw16_slots(N) : 1][4];

    template <int P, int NS>
    __device__ __forceinline__ void load_pass(const float2 *__restrict__ tw, int l)
    {
        constexpr RadixList L = reg16_radix_list(N);
        if constexpr (P < L.n) {
            constexpr int R = L.r[P];
            constexpr int Q = N / 16;
            if constexpr (P > 0) {
                constexpr int off = tw16_slots_upto(N, P);
                constexpr int STEP = N / (NS * R);
                constexpr int NSL = (Q % NS == 0) ? 1 : 16 / R;
#pragma unroll
                for (int i = 0; i < NSL; ++i) {
                    const int t = ((l + i * Q) % NS) * STEP;   // t < N/R: 8t < N for R = 16
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        w[off + i][e] = (R >> e) > 1 ? __ldg(tw + (((1 << e) * t) & (N - 1))) : make_float2(1.f, 0.f);
                }
            }
            load_pass<P + 1, NS * R>(tw, l);
        }
    }
    __device__ __forceinline__ void load(const float2 *__restrict__ tw, int l) { load_pass<0, 1>(tw, l); }
};

// u[q] *= w^q, q = 1..R-1, from the table powers p = (w, w^2, w^4, w^8)
// (conjugated for S > 0); the remaining powers are products of at most three
// of them.  The empty asm keeps the compiler from hoisting the products out of
// a work-item loop.
template <int R, int S>
__device__ __forceinline__ void twiddle_pow(float2 *u, const float2 (&p)[4])
{
    float2 w1 = p[0], w2 = p[1], w4 = p[2], w8 = p[3];
    asm volatile("" : "+f"(w1.x), "+f"(w1.y), "+f"(w2.x), "+f"(w2.y), "+f"(w4.x), "+f"(w4.y), "+f"(w8.x),
                 "+f"(w8.y));
    if (S > 0) {
        w1.y = -w1.y;
        w2.y = -w2.y;
        w4.y = -w4.y;
        w8.y = -w8.y;
    }
    if constexpr (R == 2) {
        u[1] = cmul(u[1], w1);
    } else if constexpr (R == 4) {
        u[1] = cmul(u[1], w1);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], cmul(w1, w2));
    } else {
        const float2 w3 = cmul(w1, w2);
        float2 pw[8] = {make_float2(1.f, 0.f), w1, w2, w3, w4, cmul(w1, w4), cmul(w2, w4), cmul(w3, w4)};
#pragma unroll
        for (int q = 1; q < 8; ++q) u[q] = cmul(u[q], pw[q]);
        if constexpr (R == 16) {
            u[8] = cmul(u[8], w8);
#pragma unroll
            for (int q = 1; q < 8; ++q) u[8 + q] = cmul(u[8 + q], cmul(pw[q], w8));
        }
    }
}

// Swizzle of the 16-value exchanges (column tiles): element e of sequence b
// at (e ^ ((e >> 4) & (16/NB - 1)))*NB + b; conflict-free for every exchange
// of the 16-value passes (8-byte accesses per half warp).
template <int N, int NB>
struct ColSwz16 {
    static_assert(NB >= 1 && NB <= 16 && 16 % NB == 0, "column tile width must divide 16");
    __device__ __forceinline__ static int at(int b, int e) { return (e ^ ((e >> 4) & (16 / NB - 1))) * NB + b; }
};

// Row layout of the 16-value exchanges: sequence b at b*N, element e at
// e ^ ((e >> 4) & 15) (the column-tile swizzle with one column per tile).
template <int N>
struct RowSwz16 {
    __device__ __forceinline__ static int at(int b, int e) { return b * N + (e ^ ((e >> 4) & 15)); }
};

template <int N, class LAYOUT, int S, int P, int NS>
__device__ __forceinline__ void reg16_passes(float2 (&v)[16], float2 *buf, int b, int l, const RegTw16<N> &tw)
{
    constexpr RadixList L = reg16_radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        constexpr int BPT = 16 / R;
        constexpr int Q = N / 16;
        int kk[BPT];
#pragma unroll
        for (int i = 0; i < BPT; ++i) {
            const int j = l + i * Q;
            const int k = j % NS;
            kk[i] = k;
            float2 u[R];
#pragma unroll
            for (int q = 0; q < R; ++q) u[q] = v[i + q * BPT];
            if constexpr (NS > 1) {
                constexpr int off = tw16_slots_upto(N, P);
                twiddle_pow<R, S>(u, tw.w[off + (Q % NS == 0 ? 0 : i)]);
            }
            dftR<R, S>(u);
#pragma unroll
            for (int q = 0; q < R; ++q) v[i + q * BPT] = u[q];
        }
        if constexpr (P + 1 < L.n) {
            __syncthreads();   // earlier reads of buf are complete
#pragma unroll
            for (int i = 0; i < BPT; ++i) {
                const int j = l + i * Q;
                const int base = (j - kk[i]) * R + kk[i];
#pragma unroll
                for (int q = 0; q < R; ++q) buf[LAYOUT::at(b, base + q * NS)] = v[i + q * BPT];
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = buf[LAYOUT::at(b, l + m * Q)];
            reg16_passes<N, LAYOUT, S, P + 1, NS * R>(v, buf, b, l, tw);
        }
    }
}

template <int N, class LAYOUT, int S>
__device__ __forceinline__ void reg16_fft(float2 (&v)[16], float2 *buf, int b, int l, const RegTw16<N> &tw)
{
    static_assert(is_pow2(N) && N >= 128 && N <= 4096, "16-value FFT length: 2^k, 128..4096");
    reg16_passes<N, LAYOUT, S, 0, 1>(v, buf, b, l, tw);
}

// ---- half of each 16-value sequence per thread (half tiles) --------------------
// Two threads share a sequence position l: thread h (0 or 1) holds v[2j + h],
// j = 0..7, of the 16-value form and performs the operations reg16_passes
// performs on those values, so the pair's results are reg16_fft's bit for bit.
// A radix-16 butterfly trades four values with the partner through `mid`
// (dft16_half_a / dft16_half_b; 8 * npairs values, `pair` indexing the
// thread's (b, l)); the butterflies i of the smaller radices use values of one
// parity (i + q*BPT = i mod 2), so thread h takes i = h, h + 2, ...  h must be
// uniform over each warp; every barrier is in code that all threads run.

// twiddle_pow<16, S> on the values of parity H (the same products)
template <int S, int H>
__device__ __forceinline__ void twiddle_pow16_half(float2 (&u)[8], const float2 (&p)[4])
{
    float2 w1 = p[0], w2 = p[1], w4 = p[2], w8 = p[3];
    asm volatile("" : "+f"(w1.x), "+f"(w1.y), "+f"(w2.x), "+f"(w2.y), "+f"(w4.x), "+f"(w4.y), "+f"(w8.x),
                 "+f"(w8.y));
    if (S > 0) {
        w1.y = -w1.y;
        w2.y = -w2.y;
        w4.y = -w4.y;
        w8.y = -w8.y;
    }
    const float2 w3 = cmul(w1, w2);
    float2 pw[8] = {make_float2(1.f, 0.f), w1, w2, w3, w4, cmul(w1, w4), cmul(w2, w4), cmul(w3, w4)};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int q = 2 * j + H;
        if (q == 0) continue;
        if (q < 8) u[j] = cmul(u[j], pw[q]);
        else if (q == 8) u[j] = cmul(u[j], w8);
        else u[j] = cmul(u[j], cmul(pw[q - 8], w8));
    }
}

template <int N, class LAYOUT, int S, int P, int NS>
__device__ __forceinline__ void reg16h_passes(float2 (&v)[8], float2 *buf, float2 *mid, int b, int l, int h,
                                              int pair, int npairs, const RegTw16<N> &tw)
{
    constexpr RadixList L = reg16_radix_list(N);
    if constexpr (P < L.n) {
        constexpr int R = L.r[P];
        constexpr int BPT = 16 / R;
        constexpr int HB = BPT / 2 > 0 ? BPT / 2 : 1;   // butterflies per thread (R < 16)
        constexpr int Q = N / 16;
        constexpr int off = tw16_slots_upto(N, P);
        int kk[HB];
        if constexpr (R == 16) {
            kk[0] = l % NS;
            if constexpr (NS > 1) {
                if (h) twiddle_pow16_half<S, 1>(v, tw.w[off]);
                else twiddle_pow16_half<S, 0>(v, tw.w[off]);
            }
            float2 ya[4], yb[4];
            if (h) dft16_half_a<S, 1>(v, ya, yb, mid + 4 * npairs + pair, npairs);
            else dft16_half_a<S, 0>(v, ya, yb, mid + pair, npairs);
            __syncthreads();
            if (h) dft16_half_b<S, 1>(v, ya, yb, mid + pair, npairs);
            else dft16_half_b<S, 0>(v, ya, yb, mid + 4 * npairs + pair, npairs);
        } else {
#pragma unroll
            for (int t = 0; t < HB; ++t) {
                const int i = 2 * t + h;
                const int j = l + i * Q;
                const int k = j % NS;
                kk[t] = k;
                float2 u[R];
#pragma unroll
                for (int q = 0; q < R; ++q) u[q] = v[t + q * HB];
                if constexpr (NS > 1) {
                    if constexpr (Q % NS == 0) {
                        twiddle_pow<R, S>(u, tw.w[off]);
                    } else {
                        float2 p[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) p[e] = h ? tw.w[off + 2 * t + 1][e] : tw.w[off + 2 * t][e];
                        twiddle_pow<R, S>(u, p);
                    }
                }
                dftR<R, S>(u);
#pragma unroll
                for (int q = 0; q < R; ++q) v[t + q * HB] = u[q];
            }
        }
        if constexpr (P + 1 < L.n) {
            __syncthreads();   // earlier reads of buf are complete
            if constexpr (R == 16) {
                const int base = (l - kk[0]) * 16 + kk[0];
#pragma unroll
                for (int j = 0; j < 8; ++j) buf[LAYOUT::at(b, base + (2 * j + h) * NS)] = v[j];
            } else {
#pragma unroll
                for (int t = 0; t < HB; ++t) {
                    const int j = l + (2 * t + h) * Q;
                    const int base = (j - kk[t]) * R + kk[t];
#pragma unroll
                    for (int q = 0; q < R; ++q) buf[LAYOUT::at(b, base + q * NS)] = v[t + q * HB];
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = buf[LAYOUT::at(b, l + (2 * j + h) * Q)];
            reg16h_passes<N, LAYOUT, S, P + 1, NS * R>(v, buf, mid, b, l, h, pair, npairs, tw);
        }
    }
}

// reg16_fft on the values of parity h (see above); `mid` holds 8 * npairs values
template <int N, class LAYOUT, int S>
__device__ __forceinline__ void reg16h_fft(float2 (&v)[8], float2 *buf, float2 *mid, int b, int l, int h, int pair,
                                           int npairs, const RegTw16<N> &tw)
{
    static_assert(is_pow2(N) && N >= 128 && N <= 4096, "16-value FFT length: 2^k, 128..4096");
    reg16h_passes<N, LAYOUT, S, 0, 1>(v, buf, mid, b, l, h, pair, npairs, tw);
}

// shared memory (bytes) a register-FFT kernel needs
__host__ __device__ constexpr int reg_smem_bytes(int N, int NB) { return 2 * NB * (N + N / 8) * 8; }

}  // namespace imr
