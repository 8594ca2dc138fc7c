/*
 * ORACLE / TEST INFRASTRUCTURE -- not part of the product.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Project-written complex FFT, instantiated twice (float and double) by
 * oracle/imro_fft.c.  It stands in for FFTW3 (an un-vendored, unpinned system
 * dependency of the reference: cmake/FindFFTW.cmake, CMakeLists.txt:20-22)
 * and restates the published DFT definition
 *     X[k] = sum_j x[j] * exp(sign * 2*pi*i * j*k / n),   sign = -1 forward,
 *                                                          sign = +1 backward,
 * unnormalised in both directions, exactly what the reference's calls
 * fftwf_plan_dft(..., FFTW_FORWARD/FFTW_BACKWARD, FFTW_ESTIMATE) compute
 * (src/imresh/algorithms/shrinkWrap.cpp:151-155).
 *
 * Algorithm: Stockham autosort (ping-pong, natural order in and out) over
 * mixed radices 4, 2, 3, 5, 7 and generic small odd primes <= 61; lengths
 * with a larger prime factor go through Bluestein's chirp-z convolution on a
 * power-of-two grid.  Twiddles and chirps are computed in double and rounded
 * to the working precision, so the float instance behaves like FFTW's float
 * library: float arithmetic, accurate twiddles.
 *
 * Data layout inside a 1D call is batch-inner: element t of sequence b is at
 * complex index t*B + b, so the inner loops vectorise over the batch.
 *
 * Expected macros: R (float|double), SUF (token suffix).
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)

typedef struct FN(imro_fft_plan_) {
    int n;
    int nrad;
    int rad[40];
    R *tw;          /* 2*n: exp(-2*pi*i*t/n), t = 0..n-1                   */
    R *roots;       /* per generic radix p: exp(-2*pi*i*t/p), packed         */
    int bluestein;  /* 1: length n via chirp-z on length m                  */
    int m;
    R *chirp;       /* 2*n: exp(-pi*i*j^2/n)                                 */
    R *bfft_fwd;    /* 2*m: FFT_m of the kernel conj(c_j) for sign -1        */
    R *bfft_bwd;    /* 2*m: FFT_m of the kernel conj(c_j) for sign +1        */
    struct FN(imro_fft_plan_) *sub; /* power-of-two plan of length m        */
} FN(imro_fft_plan_);

static int FN(imro_factor_)(int n, int *rad)
{
    int k = 0;
    while (n % 4 == 0) { rad[k++] = 4; n /= 4; }
    while (n % 2 == 0) { rad[k++] = 2; n /= 2; }
    for (int p = 3; p <= 61 && n > 1; p += 2) {
        while (n % p == 0) { rad[k++] = p; n /= p; }
    }
    return n == 1 ? k : -1;   /* -1: a prime factor > 61 remains */
}

static void FN(imro_fft_batched_)(const FN(imro_fft_plan_) *p, R *data, R *work, int B, int sign);

static FN(imro_fft_plan_) *FN(imro_fft_plan_create_)(int n)
{
    FN(imro_fft_plan_) *p = (FN(imro_fft_plan_) *)calloc(1, sizeof(*p));
    p->n = n;
    int rad[40];
    int nr = FN(imro_factor_)(n, rad);
    if (nr >= 0) {
        p->nrad = nr;
        memcpy(p->rad, rad, sizeof(int) * (size_t)nr);
        p->tw = (R *)malloc(sizeof(R) * 2 * (size_t)n);
        for (int t = 0; t < n; ++t) {
            /* reduce t/n exactly before scaling: keeps twiddles accurate */
            double a = -2.0 * M_PI * (double)t / (double)n;
            p->tw[2 * t] = (R)cos(a);
            p->tw[2 * t + 1] = (R)sin(a);
        }
        int tot = 0;
        for (int i = 0; i < nr; ++i) if (rad[i] != 2 && rad[i] != 4) tot += rad[i];
        p->roots = (R *)malloc(sizeof(R) * 2 * (size_t)(tot + 1));
        int off = 0;
        for (int i = 0; i < nr; ++i) {
            int r = rad[i];
            if (r == 2 || r == 4) continue;
            for (int t = 0; t < r; ++t) {
                double a = -2.0 * M_PI * (double)t / (double)r;
                p->roots[2 * (off + t)] = (R)cos(a);
                p->roots[2 * (off + t) + 1] = (R)sin(a);
            }
            off += r;
        }
        return p;
    }
    /* Bluestein: X_k = c_k * sum_j (x_j c_j) conj(c_{k-j}),  c_j = e^{s*pi*i*j^2/n} */
    p->bluestein = 1;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->sub = FN(imro_fft_plan_create_)(m);
    p->chirp = (R *)malloc(sizeof(R) * 2 * (size_t)n);
    double *cre = (double *)malloc(sizeof(double) * (size_t)n);
    double *cim = (double *)malloc(sizeof(double) * (size_t)n);
    for (int j = 0; j < n; ++j) {
        /* j^2 mod 2n keeps the angle argument small and exact */
        long long q = ((long long)j * (long long)j) % (2LL * n);
        double a = -M_PI * (double)q / (double)n;
        cre[j] = cos(a);
        cim[j] = sin(a);
        p->chirp[2 * j] = (R)cre[j];
        p->chirp[2 * j + 1] = (R)cim[j];
    }
    p->bfft_fwd = (R *)calloc(2 * (size_t)m, sizeof(R));
    p->bfft_bwd = (R *)calloc(2 * (size_t)m, sizeof(R));
    for (int j = 0; j < n; ++j) {
        /* forward (sign -1): c_j = e^{-i pi j^2/n} = chirp; kernel conj(c) */
        p->bfft_fwd[2 * j] = (R)cre[j];
        p->bfft_fwd[2 * j + 1] = (R)(-cim[j]);
        p->bfft_bwd[2 * j] = (R)cre[j];
        p->bfft_bwd[2 * j + 1] = (R)cim[j];
        if (j > 0) {
            p->bfft_fwd[2 * (m - j)] = (R)cre[j];
            p->bfft_fwd[2 * (m - j) + 1] = (R)(-cim[j]);
            p->bfft_bwd[2 * (m - j)] = (R)cre[j];
            p->bfft_bwd[2 * (m - j) + 1] = (R)cim[j];
        }
    }
    free(cre);
    free(cim);
    {
        R *tmp = (R *)malloc(sizeof(R) * 2 * (size_t)m);
        FN(imro_fft_batched_)(p->sub, p->bfft_fwd, tmp, 1, -1);
        FN(imro_fft_batched_)(p->sub, p->bfft_bwd, tmp, 1, -1);
        free(tmp);
    }
    return p;
}

static void FN(imro_fft_plan_destroy_)(FN(imro_fft_plan_) *p)
{
    if (!p) return;
    free(p->tw);
    free(p->roots);
    free(p->chirp);
    free(p->bfft_fwd);
    free(p->bfft_bwd);
    if (p->sub) FN(imro_fft_plan_destroy_)(p->sub);
    free(p);
}

/* One Stockham pass of radix r over B interleaved sequences of length n:
 *   for j in [0, n/r): v[q] = in[j + q*n/r] * w^(q*(j mod Ns)), w = e^{s 2pi i/(Ns r)}
 *                      v = DFT_r(v);  out[(j/Ns)*Ns*r + (j mod Ns) + q*Ns] = v[q] */
static void FN(imro_pass_)(const FN(imro_fft_plan_) *p, const R *roots, int r, int Ns,
                           const R *in, R *out, int B, int sign)
{
    const int n = p->n;
    const int mq = n / r;
    const int twstep = n / (Ns * r);
    R vr[64], vi[64];
    for (int j = 0; j < mq; ++j) {
        const int k = j % Ns;
        const int base = (j / Ns) * Ns * r + k;
        for (int b = 0; b < B; ++b) {
            for (int q = 0; q < r; ++q) {
                const R *s = in + 2 * ((size_t)(j + q * mq) * B + b);
                R xr = s[0], xi = s[1];
                if (q && k) {
                    int t = q * k * twstep;       /* < n */
                    R wr = p->tw[2 * t], wi = p->tw[2 * t + 1] * (R)(-sign);
                    R tr = xr * wr - xi * wi;
                    xi = xr * wi + xi * wr;
                    xr = tr;
                }
                vr[q] = xr;
                vi[q] = xi;
            }
            if (r == 2) {
                R ar = vr[0] + vr[1], ai = vi[0] + vi[1];
                R br = vr[0] - vr[1], bi = vi[0] - vi[1];
                vr[0] = ar; vi[0] = ai; vr[1] = br; vi[1] = bi;
            } else if (r == 4) {
                R s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
                R d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
                R s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
                R d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
                /* w = e^{s*i*pi/2} = s*i, so Y1 = d0 + w*d1, Y3 = d0 - w*d1 */
                R jr = -(R)sign * d1i, ji = (R)sign * d1r;
                vr[0] = s0r + s1r; vi[0] = s0i + s1i;
                vr[2] = s0r - s1r; vi[2] = s0i - s1i;
                vr[1] = d0r + jr;  vi[1] = d0i + ji;
                vr[3] = d0r - jr;  vi[3] = d0i - ji;
            } else {
                R yr[64], yi[64];
                for (int kk = 0; kk < r; ++kk) {
                    R ar = 0, ai = 0;
                    for (int q = 0; q < r; ++q) {
                        int t = (q * kk) % r;
                        R wr = roots[2 * t], wi = roots[2 * t + 1] * (R)(-sign);
                        ar += vr[q] * wr - vi[q] * wi;
                        ai += vr[q] * wi + vi[q] * wr;
                    }
                    yr[kk] = ar;
                    yi[kk] = ai;
                }
                for (int q = 0; q < r; ++q) { vr[q] = yr[q]; vi[q] = yi[q]; }
            }
            for (int q = 0; q < r; ++q) {
                R *d = out + 2 * ((size_t)(base + q * Ns) * B + b);
                d[0] = vr[q];
                d[1] = vi[q];
            }
        }
    }
}

/* In-place batched 1D transform; data holds n*B complex, batch-inner.
 * work must hold at least n*B complex (Bluestein: 2*m*B complex). */
static void FN(imro_fft_batched_)(const FN(imro_fft_plan_) *p, R *data, R *work, int B, int sign)
{
    const int n = p->n;
    if (n == 1) return;
    if (!p->bluestein) {
        R *a = data, *b = work;
        int Ns = 1, off = 0;
        for (int i = 0; i < p->nrad; ++i) {
            int r = p->rad[i];
            const R *roots = (r == 2 || r == 4) ? NULL : p->roots + 2 * off;
            if (roots) off += r;
            FN(imro_pass_)(p, roots, r, Ns, a, b, B, sign);
            Ns *= r;
            R *t = a; a = b; b = t;
        }
        if (a != data) memcpy(data, a, sizeof(R) * 2 * (size_t)n * (size_t)B);
        return;
    }
    const int m = p->m;
    R *A = work;                              /* m*B complex */
    R *W2 = work + 2 * (size_t)m * B;         /* m*B complex scratch */
    memset(A, 0, sizeof(R) * 2 * (size_t)m * B);
    for (int j = 0; j < n; ++j) {
        R cr = p->chirp[2 * j], ci = p->chirp[2 * j + 1] * (R)(-sign);  /* c_j for this sign */
        for (int b = 0; b < B; ++b) {
            const R *s = data + 2 * ((size_t)j * B + b);
            R *d = A + 2 * ((size_t)j * B + b);
            d[0] = s[0] * cr - s[1] * ci;
            d[1] = s[0] * ci + s[1] * cr;
        }
    }
    FN(imro_fft_batched_)(p->sub, A, W2, B, -1);
    const R *Kf = sign < 0 ? p->bfft_fwd : p->bfft_bwd;   /* already in frequency space */
    for (int t = 0; t < m; ++t) {
        R kr = Kf[2 * t], ki = Kf[2 * t + 1];
        for (int b = 0; b < B; ++b) {
            R *d = A + 2 * ((size_t)t * B + b);
            R xr = d[0] * kr - d[1] * ki;
            d[1] = d[0] * ki + d[1] * kr;
            d[0] = xr;
        }
    }
    FN(imro_fft_batched_)(p->sub, A, W2, B, +1);
    const R inv_m = (R)(1.0 / (double)m);
    for (int k = 0; k < n; ++k) {
        R cr = p->chirp[2 * k], ci = p->chirp[2 * k + 1] * (R)(-sign);
        for (int b = 0; b < B; ++b) {
            const R *s = A + 2 * ((size_t)k * B + b);
            R yr = s[0] * inv_m, yi = s[1] * inv_m;
            R *d = data + 2 * ((size_t)k * B + b);
            d[0] = yr * cr - yi * ci;
            d[1] = yr * ci + yi * cr;
        }
    }
}

#define IMRO_FFT_BATCH 16

/* Unnormalised 1D transform of `howmany` contiguous sequences of length n
 * (sequence s at data + 2*s*n), in place. */
static void FN(imro_fft_rows_)(R *data, int n, int howmany, int sign)
{
    if (n <= 1 || howmany <= 0) return;
    FN(imro_fft_plan_) *p = FN(imro_fft_plan_create_)(n);
    size_t wn = p->bluestein ? (size_t)4 * p->m : (size_t)2 * n;
    R *buf = (R *)malloc(sizeof(R) * 2 * (size_t)n * IMRO_FFT_BATCH);
    R *work = (R *)malloc(sizeof(R) * wn * IMRO_FFT_BATCH);
    for (int r0 = 0; r0 < howmany; r0 += IMRO_FFT_BATCH) {
        int B = howmany - r0 < IMRO_FFT_BATCH ? howmany - r0 : IMRO_FFT_BATCH;
        for (int b = 0; b < B; ++b)
            for (int x = 0; x < n; ++x) {
                buf[2 * ((size_t)x * B + b)] = data[2 * ((size_t)(r0 + b) * n + x)];
                buf[2 * ((size_t)x * B + b) + 1] = data[2 * ((size_t)(r0 + b) * n + x) + 1];
            }
        FN(imro_fft_batched_)(p, buf, work, B, sign);
        for (int b = 0; b < B; ++b)
            for (int x = 0; x < n; ++x) {
                data[2 * ((size_t)(r0 + b) * n + x)] = buf[2 * ((size_t)x * B + b)];
                data[2 * ((size_t)(r0 + b) * n + x) + 1] = buf[2 * ((size_t)x * B + b) + 1];
            }
    }
    free(buf);
    free(work);
    FN(imro_fft_plan_destroy_)(p);
}

/* Unnormalised 1D transform along the columns of a row-major [H][W] array. */
static void FN(imro_fft_cols_)(R *data, int H, int W, int sign)
{
    if (H <= 1 || W <= 0) return;
    FN(imro_fft_plan_) *p = FN(imro_fft_plan_create_)(H);
    size_t wn = p->bluestein ? (size_t)4 * p->m : (size_t)2 * H;
    R *buf = (R *)malloc(sizeof(R) * 2 * (size_t)H * IMRO_FFT_BATCH);
    R *work = (R *)malloc(sizeof(R) * wn * IMRO_FFT_BATCH);
    for (int c0 = 0; c0 < W; c0 += IMRO_FFT_BATCH) {
        int B = W - c0 < IMRO_FFT_BATCH ? W - c0 : IMRO_FFT_BATCH;
        for (int y = 0; y < H; ++y)
            for (int b = 0; b < B; ++b) {
                buf[2 * ((size_t)y * B + b)] = data[2 * ((size_t)y * W + c0 + b)];
                buf[2 * ((size_t)y * B + b) + 1] = data[2 * ((size_t)y * W + c0 + b) + 1];
            }
        FN(imro_fft_batched_)(p, buf, work, B, sign);
        for (int y = 0; y < H; ++y)
            for (int b = 0; b < B; ++b) {
                data[2 * ((size_t)y * W + c0 + b)] = buf[2 * ((size_t)y * B + b)];
                data[2 * ((size_t)y * W + c0 + b) + 1] = buf[2 * ((size_t)y * B + b) + 1];
            }
    }
    free(buf);
    free(work);
    FN(imro_fft_plan_destroy_)(p);
}

/* Unnormalised 2D transform of a row-major [H][W] complex array, in place:
 * rows first, then columns. */
static void FN(imro_fft2d_)(R *data, int H, int W, int sign)
{
    FN(imro_fft_rows_)(data, W, H, sign);
    FN(imro_fft_cols_)(data, H, W, sign);
}

#undef FN
#undef CAT
#undef CAT2
