// FP64 fast Fourier transforms of the PME mesh (hand-written; no library):
// the forward real-to-complex and the inverse complex-to-real 3D transforms of
// an n0 x n1 x n2 mesh (n2 fastest; half spectrum n0 x n1 x (n2 / 2 + 1)),
// each built from 1D passes over lines held in shared memory.
//
// A line of length n = 2^a 3^b (n <= kFftMax) is transformed by the
// self-sorting Stockham algorithm, decimation in frequency: with the remaining
// length l (initially n) and the stride s (initially 1, l s = n), a radix-r
// stage maps x to y by
//     y[q + s (r p + k)] = w_l^(p k) sum_j x[q + s (p + j l / r)] w_r^(j k),
// p < l / r, q < s, k < r, w_m = exp(-+ 2 pi i / m), and continues on y with
// l / r and r s; the output is in natural order.  Sign -1: forward
// (exp(-2 pi i k x / n)), +1: inverse, unnormalised.  The twiddles come from
// sincospi in FP64.
//
// The line transform (fft_line) is a __host__ __device__ function over a
// "thread" index range, so the host test build runs the same arithmetic.
#pragma once
#include <cuda_runtime.h>

namespace gcmc {

constexpr int kFftMax = 256;   // longest line
constexpr int kFftLines = 8;   // lines per CTA in the batched passes
constexpr int kFftThreads = 256;

__host__ __device__ inline bool fft_size_ok(int n) {
    if (n < 1 || n > kFftMax) return false;
    while (n % 2 == 0) n /= 2;
    while (n % 3 == 0) n /= 3;
    return n == 1;
}

// The radices of n, radix 2 first, then 3 (stored in r[], returns the count).
__host__ __device__ inline int fft_radices(int n, int r[16]) {
    int c = 0;
    while (n % 2 == 0) { r[c++] = 2; n /= 2; }
    while (n % 3 == 0) { r[c++] = 3; n /= 3; }
    return c;
}

__host__ __device__ inline double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(sign 2 pi i num / den)
__host__ __device__ inline double2 twiddle(int num, int den, int sign) {
    double sn, cs;
#ifdef __CUDA_ARCH__
    sincospi(2.0 * (double)num / (double)den, &sn, &cs);
#else
    sn = sin(2.0 * 3.14159265358979323846 * (double)num / (double)den);
    cs = cos(2.0 * 3.14159265358979323846 * (double)num / (double)den);
#endif
    return make_double2(cs, sign * sn);
}

// One Stockham stage on `nl` lines of length n (line b at x + b * ld), work
// items t in [t0, t1) step dt (t = line * (n / r) + butterfly).
__host__ __device__ inline void fft_stage(const double2* x, double2* y, int ld, int nl, int n, int l, int s, int r,
                                          int sign, int t0, int dt) {
    const int m = l / r;
    const int per = n / r;  // butterflies per line (m * s)
    for (int t = t0; t < nl * per; t += dt) {
        const int b = t / per, u = t - b * per;
        const int p = u / s, q = u - p * s;
        const double2* xb = x + (size_t)b * ld;
        double2* yb = y + (size_t)b * ld;
        if (r == 2) {
            const double2 a = xb[q + s * p], c = xb[q + s * (p + m)];
            const double2 w = twiddle(p, l, sign);
            yb[q + s * (2 * p)] = make_double2(a.x + c.x, a.y + c.y);
            yb[q + s * (2 * p + 1)] = cmul(make_double2(a.x - c.x, a.y - c.y), w);
        } else {  // r == 3
            const double2 a = xb[q + s * p], c = xb[q + s * (p + m)], d = xb[q + s * (p + 2 * m)];
            // w3 = exp(sign 2 pi i / 3) = -1/2 + sign i sqrt(3)/2
            const double h = 0.86602540378443864676 * sign;
            const double2 cd = make_double2(c.x + d.x, c.y + d.y);
            const double2 cm = make_double2(c.x - d.x, c.y - d.y);  // (c - d)
            const double2 t0v = make_double2(a.x + cd.x, a.y + cd.y);
            const double2 base = make_double2(a.x - 0.5 * cd.x, a.y - 0.5 * cd.y);
            // i h (c - d)
            const double2 rot = make_double2(-h * cm.y, h * cm.x);
            const double2 t1v = make_double2(base.x + rot.x, base.y + rot.y);
            const double2 t2v = make_double2(base.x - rot.x, base.y - rot.y);
            const double2 w1 = twiddle(p, l, sign);
            const double2 w2 = twiddle(2 * p, l, sign);
            yb[q + s * (3 * p)] = t0v;
            yb[q + s * (3 * p + 1)] = cmul(t1v, w1);
            yb[q + s * (3 * p + 2)] = cmul(t2v, w2);
        }
    }
}

#ifdef __CUDACC__
// nl lines of length n in shared memory (buf0, buf1: nl * ld each), whole
// CTA; returns the buffer holding the result.
__device__ __forceinline__ double2* fft_lines_block(double2* buf0, double2* buf1, int ld, int nl, int n, int sign) {
    int rad[16];
    const int nr = fft_radices(n, rad);
    double2 *x = buf0, *y = buf1;
    int l = n, s = 1;
    for (int st = 0; st < nr; ++st) {
        __syncthreads();
        fft_stage(x, y, ld, nl, n, l, s, rad[st], sign, threadIdx.x, blockDim.x);
        l /= rad[st];
        s *= rad[st];
        double2* t = x; x = y; y = t;
    }
    __syncthreads();
    return x;
}
#endif

// Host reference of one line (test build): returns the transform of x in x.
inline void fft_line_host(double2* x, int n, int sign) {
    double2 y[kFftMax];
    int rad[16];
    const int nr = fft_radices(n, rad);
    double2 *a = x, *b = y;
    int l = n, s = 1;
    for (int st = 0; st < nr; ++st) {
        fft_stage(a, b, n, 1, n, l, s, rad[st], sign, 0, 1);
        l /= rad[st];
        s *= rad[st];
        double2* t = a; a = b; b = t;
    }
    if (a != x)
        for (int i = 0; i < n; ++i) x[i] = a[i];
}

}  // namespace gcmc
