// Shared device definitions: constants, exact-rounding float helpers, the
// counter-based RNG, the deterministic sin/cos, pose construction and the two
// FP32 distance forms.  Everything a proposal or an inclusion decision depends
// on is built from correctly rounded operations (explicit __f*_rn intrinsics,
// which the compiler never fuses or reorders), so every result here is
// reproducible bit for bit by a CPU implementation of the same formulas.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gcmc_b200.h"

namespace gcmc {

// gcmc/cpp/gcmc.h:28-41
constexpr double kBeta = 1.0 / (0.0083115 * 300.0);
constexpr double kMolesToMolecules = 0.0006023;
constexpr double kKcalToKJ = 4.184;
constexpr float kCoulomb = 1388.431112f;  // gcmc/cpp/gcmc_energy.h:137
constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr int kMaxSites = 20;
constexpr int kMaxPoses = 1024;  // poses per step (confBias limit)
constexpr int kMaxWords = kMaxPoses / 32;

// RNG purposes: high half of the third counter word.
enum : uint32_t { RP_INSERT = 1, RP_DELETE = 2, RP_MOVE = 3, RP_CLUSTER = 4, RP_PERM = 5, RP_GUMBEL = 6, RP_FB = 7 };
// force-bias tilt lambda (Pangali, Rao and Berne): density ~ exp(lambda beta f . d) in the step cube
constexpr float kFbLambda = 0.5f;
enum : int { MV_NONE = -1, MV_INSERT = 0, MV_DELETE = 1, MV_TRANSLATE = 2, MV_ROTATE = 3 };
enum : int {
    ERR_CELL_OVERFLOW = 1, ERR_IMAGE = 2, ERR_SLOT = 4, ERR_POSES = 8, ERR_SITE_TYPE = 16, ERR_SYNC = 32,
    ERR_GRID_BITS = 64
};

// ---------------------------------------------------------------------------
// exact-rounding float helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float ffma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }

// fast_round of gcmc/cpp/gcmc_energy.h:110-112: round half away from zero via
// truncation to int, returned as float.
__device__ __forceinline__ float fast_round(float a) {
    return a >= 0.0f ? __int2float_rn(__float2int_rz(fadd(a, 0.5f)))
                     : __int2float_rn(__float2int_rz(fsub(a, 0.5f)));
}

// Group-inclusion distance: the reference's device distanceP
// (gcmc/cpp/gcmc_energy.h:115-122) with its multiply-adds fused.
__device__ __forceinline__ float dist_group(float ax, float ay, float az, float bx, float by, float bz,
                                            const float* L) {
    float dx = fsub(ax, bx), dy = fsub(ay, by), dz = fsub(az, bz);
    dx = ffma(-fast_round(fdiv(dx, L[0])), L[0], dx);
    dy = ffma(-fast_round(fdiv(dy, L[1])), L[1], dy);
    dz = ffma(-fast_round(fdiv(dz, L[2])), L[2], dz);
    float s = fmul(dx, dx);
    s = ffma(dy, dy, s);
    s = ffma(dz, dz, s);
    return fsqrt(s);
}

// Clustering distance: the reference's host distanceP (unfused), used by the
// pose clustering of gcmc/cpp/gcmc_move_add.h:129 and gcmc_move_trn.h:180.
__device__ __forceinline__ float dist_host(float ax, float ay, float az, float bx, float by, float bz,
                                           const float* L) {
    float dx = fsub(ax, bx), dy = fsub(ay, by), dz = fsub(az, bz);
    dx = fsub(dx, fmul(fast_round(fdiv(dx, L[0])), L[0]));
    dy = fsub(dy, fmul(fast_round(fdiv(dy, L[1])), L[1]));
    dz = fsub(dz, fmul(fast_round(fdiv(dz, L[2])), L[2]));
    float s = fadd(fmul(dx, dx), fmul(dy, dy));
    s = fadd(s, fmul(dz, dz));
    return fsqrt(s);
}

// Inclusion test equal to dist_group(...) <= cutoff.  When R.fast_incl is set
// (cutoff below half of every box edge) a multiply-based squared distance
// decides every case outside +-1e-4 of the cutoff: there both forms pick the
// same periodic image (they can differ only at |d| ~ L/2, beyond the cutoff)
// and their distances agree to a few ulps; only candidates inside the band take
// the exact division form.
template <bool Host>
__device__ __forceinline__ bool within_cutoff(float ax, float ay, float az, float bx, float by, float bz,
                                              const float* L, const float* invL, float cutoff, float lo2,
                                              float hi2, bool fast) {
    if (fast) {
        float dx = ax - bx, dy = ay - by, dz = az - bz;
        dx = fmaf(-rintf(dx * invL[0]), L[0], dx);
        dy = fmaf(-rintf(dy * invL[1]), L[1], dy);
        dz = fmaf(-rintf(dz * invL[2]), L[2], dz);
        const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        if (r2 < lo2) return true;
        if (r2 > hi2) return false;
    }
    return (Host ? dist_host(ax, ay, az, bx, by, bz, L) : dist_group(ax, ay, az, bx, by, bz, L)) <= cutoff;
}

// Programmatic dependent launch (PTX griddepcontrol): a kernel launched as a
// programmatic dependent of the kernel before it in its stream may start while
// that kernel runs; pdl_wait blocks until the prerequisite grid has completed
// and its memory operations are visible (it returns at once when the kernel
// was launched normally), and pdl_trigger lets this grid's dependents be
// scheduled once every CTA of it has triggered or exited.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): counter (step, index,
// purpose<<16 | draw, 0), key (seed, replica).
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                     uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return {c0, c1, c2, c3};
}

__device__ __forceinline__ U4 rng(uint32_t seed, uint32_t replica, uint32_t step, uint32_t index,
                                  uint32_t purpose, uint32_t draw) {
    return philox(step, index, (purpose << 16) | draw, 0u, seed, replica);
}

__device__ __forceinline__ float u01_oc(uint32_t x) { return fmul(__uint2float_rn((x >> 8) + 1u), 5.9604644775390625e-08f); }
__device__ __forceinline__ float u01_co(uint32_t x) { return fmul(__uint2float_rn(x >> 8), 5.9604644775390625e-08f); }
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
    unsigned long long m = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
    return (double)m * 1.1102230246251565e-16;
}
__device__ __forceinline__ double u53_open(uint32_t a, uint32_t b) {
    unsigned long long m = ((unsigned long long)(a >> 5) << 26) | (unsigned long long)(b >> 6);
    return ((double)m + 0.5) * 1.1102230246251565e-16;
}

// ---------------------------------------------------------------------------
// Deterministic sin/cos: reduction by pi/2 with a two-part constant, then the
// Taylor polynomials of sin (through r^9) and cos (through r^10) on
// |r| <= pi/4; absolute error below 4e-7 on [-2pi, 2pi].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void det_sincos(float x, float& s_out, float& c_out) {
    const float two_over_pi = 0.636619772367581343f;
    const float pio2_hi = 1.57079637050628662109375f;
    const float pio2_lo = -4.37113900018624283e-8f;
    float kf = rintf(fmul(x, two_over_pi));
    float r = ffma(-kf, pio2_hi, x);
    r = ffma(-kf, pio2_lo, r);
    float r2 = fmul(r, r);
    float ps = ffma(r2, 2.75573192239858925e-6f, -1.98412698412698413e-4f);
    ps = ffma(r2, ps, 8.33333333333333333e-3f);
    ps = ffma(r2, ps, -1.66666666666666667e-1f);
    float sr = ffma(fmul(r, r2), ps, r);
    float pc = ffma(r2, -2.75573192239858925e-7f, 2.48015873015873016e-5f);
    pc = ffma(r2, pc, -1.38888888888888889e-3f);
    pc = ffma(r2, pc, 4.16666666666666667e-2f);
    pc = ffma(r2, pc, -0.5f);
    float cr = ffma(r2, pc, 1.0f);
    int q = __float2int_rz(kf) & 3;
    float s, c;
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = -sr; }
    else if (q == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
    s_out = s;
    c_out = c;
}

struct Mat3 { float m[3][3]; };

// Rodrigues rotation about a (normalised here) by the angle with (sn, cs);
// gcmc/cpp/gcmc_energy.h:39-58 with the fused form fixed.
__device__ __forceinline__ Mat3 rodrigues(float a0, float a1, float a2, float sn, float cs) {
    float nn = fmul(a0, a0);
    nn = ffma(a1, a1, nn);
    nn = ffma(a2, a2, nn);
    float norm = fsqrt(nn);
    a0 = fdiv(a0, norm); a1 = fdiv(a1, norm); a2 = fdiv(a2, norm);
    float C = fsub(1.0f, cs);
    Mat3 R;
    R.m[0][0] = ffma(fmul(a0, a0), C, cs);
    R.m[0][1] = ffma(fmul(a0, a1), C, -fmul(a2, sn));
    R.m[0][2] = ffma(fmul(a0, a2), C, fmul(a1, sn));
    R.m[1][0] = ffma(fmul(a1, a0), C, fmul(a2, sn));
    R.m[1][1] = ffma(fmul(a1, a1), C, cs);
    R.m[1][2] = ffma(fmul(a1, a2), C, -fmul(a0, sn));
    R.m[2][0] = ffma(fmul(a2, a0), C, -fmul(a1, sn));
    R.m[2][1] = ffma(fmul(a2, a1), C, fmul(a0, sn));
    R.m[2][2] = ffma(fmul(a2, a2), C, cs);
    return R;
}

// Uniform random rotation from three uniforms (Shoemake, Graphics Gems III, 1992).
__device__ __forceinline__ Mat3 shoemake(float u1, float u2, float u3) {
    float s2, c2, s3, c3;
    det_sincos(fmul(u2, kTwoPiF), s2, c2);
    det_sincos(fmul(u3, kTwoPiF), s3, c3);
    float r1 = fsqrt(fsub(1.0f, u1)), r2 = fsqrt(u1);
    float x = fmul(r1, s2), y = fmul(r1, c2), z = fmul(r2, s3), w = fmul(r2, c3);
    float xx = fmul(x, x), yy = fmul(y, y), zz = fmul(z, z);
    float xy = fmul(x, y), xz = fmul(x, z), yz = fmul(y, z), xw = fmul(x, w), yw = fmul(y, w), zw = fmul(z, w);
    Mat3 R;
    R.m[0][0] = fsub(1.0f, fmul(2.0f, fadd(yy, zz)));
    R.m[0][1] = fmul(2.0f, fsub(xy, zw));
    R.m[0][2] = fmul(2.0f, fadd(xz, yw));
    R.m[1][0] = fmul(2.0f, fadd(xy, zw));
    R.m[1][1] = fsub(1.0f, fmul(2.0f, fadd(xx, zz)));
    R.m[1][2] = fmul(2.0f, fsub(yz, xw));
    R.m[2][0] = fmul(2.0f, fsub(xz, yw));
    R.m[2][1] = fmul(2.0f, fadd(yz, xw));
    R.m[2][2] = fsub(1.0f, fmul(2.0f, fadd(xx, yy)));
    return R;
}

// p' = R p in the accumulation order of gcmc/cpp/gcmc_energy.h:62-71, fused.
__device__ __forceinline__ void rotate(const Mat3& R, float p0, float p1, float p2, float& o0, float& o1,
                                       float& o2) {
    float x = fmul(p0, R.m[0][0]); x = ffma(p1, R.m[0][1], x); x = ffma(p2, R.m[0][2], x);
    float y = fmul(p0, R.m[1][0]); y = ffma(p1, R.m[1][1], y); y = ffma(p2, R.m[1][2], y);
    float z = fmul(p0, R.m[2][0]); z = ffma(p1, R.m[2][1], z); z = ffma(p2, R.m[2][2], z);
    o0 = x; o1 = y; o2 = z;
}

// Own natural logarithm for x > 0 (finite, normal), identical on the host
// oracle: x = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s) with
// s = (m - 1) / (m + 1) summed as the odd series s (1 + s^2/3 + ... + s^10/11)
// (|s| <= 0.1716, truncation < 1e-9 relative), ln x = e ln2_hi + (e ln2_lo + ln m).
__device__ __forceinline__ float det_log(float x) {
    const uint32_t b = __float_as_uint(x);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421356f) {
        m = fmul(m, 0.5f);
        e += 1;
    }
    const float s = fdiv(fsub(m, 1.0f), fadd(m, 1.0f));
    const float s2 = fmul(s, s);
    float p = fadd(fmul(s2, 0.0909090936f), 0.111111112f);  // 1/11, 1/9
    p = fadd(fmul(s2, p), 0.142857149f);                      // 1/7
    p = fadd(fmul(s2, p), 0.200000003f);                      // 1/5
    p = fadd(fmul(s2, p), 0.333333343f);                      // 1/3
    p = fadd(fmul(s2, p), 1.0f);
    const float lnm = fmul(fmul(2.0f, s), p);
    const float ef = (float)e;
    return fadd(fmul(ef, 0.693145751953125f), fadd(fmul(ef, 1.42860677e-06f), lnm));
}

// Own exponential for x <= 0 (0 below -87), identical on the host oracle:
// x = k ln2 + r with |r| <= ln2 / 2 (Cody-Waite split of ln2), e^r by its
// Taylor polynomial to r^7 (truncation < 3e-9 relative), times 2^k.
__device__ __forceinline__ float det_exp_neg(float x) {
    if (!(x > -87.0f)) return 0.0f;
    const float kf = floorf(fadd(fmul(x, 1.44269502f), 0.5f));
    const float r = fsub(fsub(x, fmul(kf, 0.693145751953125f)), fmul(kf, 1.42860677e-06f));
    float p = fadd(fmul(r, 1.98412701e-04f), 1.38888892e-03f);  // 1/5040, 1/720
    p = fadd(fmul(r, p), 8.33333377e-03f);                      // 1/120
    p = fadd(fmul(r, p), 4.16666679e-02f);                      // 1/24
    p = fadd(fmul(r, p), 0.166666672f);                         // 1/6
    p = fadd(fmul(r, p), 0.5f);
    p = fadd(fmul(r, p), 1.0f);
    p = fadd(fmul(r, p), 1.0f);
    const int k = (int)kf;  // in [-126, 0]
    return fmul(p, __int_as_float((k + 127) << 23));
}

// One tilted-uniform draw on [-h, h] with density a e^{a x} / (2 sinh(a h))
// (the force-bias proposal of Pangali, Rao and Berne, Chem. Phys. Lett. 55
// (1978) 413, per axis with a = lambda beta f), by inverting its CDF in the
// overflow-free forms  x = h + ln(u + (1 - u) e^{-2ah}) / a  (a > 0) and
// x = -h + ln(1 - u + u e^{2ah}) / a  (a < 0); uniform when |a| h < 1e-4.
__device__ __forceinline__ float fb_tilted(float a, float h, float u) {
    const float ah = fmul(a, h);
    if (fabsf(ah) < 1e-4f) return fmul(h, fsub(fmul(2.0f, u), 1.0f));
    if (a > 0.0f) {
        const float t = det_exp_neg(fmul(-2.0f, ah));
        return fadd(h, fdiv(det_log(fadd(u, fmul(fsub(1.0f, u), t))), a));
    }
    const float t = det_exp_neg(fmul(2.0f, ah));
    return fadd(-h, fdiv(det_log(fadd(fsub(1.0f, u), fmul(u, t))), a));
}

// ln of the tilted-uniform normaliser a / (2 sinh(a h)) (even in a):
// -ln(2h) - (ah)^2/6 + (ah)^4/180 for |a| h < 1e-2, else
// ln|a| - |a| h - ln(1 - e^{-2|a| h}).
__device__ __forceinline__ float fb_lnorm(float a, float h) {
    const float b = fabsf(fmul(a, h));
    if (b < 1e-2f) {
        const float b2 = fmul(b, b);
        return fadd(fsub(-det_log(fmul(2.0f, h)), fdiv(b2, 6.0f)), fdiv(fmul(b2, b2), 180.0f));
    }
    return fsub(fsub(det_log(fabsf(a)), b), det_log(fsub(1.0f, det_exp_neg(fmul(-2.0f, b)))));
}


// Keyed permutation of [0,n) (4-round Feistel on 2h bits, cycle walking;
// round function = the MurmurHash3 32-bit finaliser).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}
__device__ __forceinline__ int perm_slot(const U4& rk, int h, int i, int n) {
    uint32_t mask = (1u << h) - 1u;
    uint32_t x = (uint32_t)i;
    do {
        uint32_t Lh = x >> h, Rh = x & mask;
        uint32_t nl;
        nl = Rh; Rh = Lh ^ (fmix32(Rh ^ rk.x) & mask); Lh = nl;
        nl = Rh; Rh = Lh ^ (fmix32(Rh ^ rk.y) & mask); Lh = nl;
        nl = Rh; Rh = Lh ^ (fmix32(Rh ^ rk.z) & mask); Lh = nl;
        nl = Rh; Rh = Lh ^ (fmix32(Rh ^ rk.w) & mask); Lh = nl;
        x = (Lh << h) | Rh;
    } while (x >= (uint32_t)n);
    return (int)x;
}
__host__ __device__ __forceinline__ int perm_bits(int n) {
    int h = 1;
    while ((1u << (2 * h)) < (uint32_t)n) ++h;
    return h;
}

// ---------------------------------------------------------------------------
// device-resident state
// ---------------------------------------------------------------------------
struct FragDev {
    int startRes, maxNum, confBias, nsites;
    double B;                  // beta*muex_eff + ln(V*conc*6.023e-4)
    double qnet;               // sum of the site charges (Ewald background term)
    float4 site[kMaxSites];    // template x, y, z, charge
    int stype[kMaxSites];      // template type
};

struct StepDesc {
    int step;      // step index this descriptor describes
    int move;      // MV_*
    int ftype;
    int k;         // poses
    int n;         // totalNum at the start of the step
    int nvar;      // 1, or 2 for translate/rotate (new, old)
    int nslab;     // work items per pose variant (item z takes window cells z, z + nslab, ...)
    int nw;        // neighbour-row words (0 = no clustering)
    int items;     // k * nvar * nslab (force-biased and dual steps: k * nslab; tiled: tiles)
    int del_slot;
    int perm_h;
    int fb;        // 1: force-biased translate/rotate (old-pose forces first, then new poses)
    int items_pre; // force-biased steps: k * nslab old-pose items of the first launch; else 0
    int dual;      // translate / rotate in the pairwise-difference form: items k * nslab, each
                   // writing the slab's energy change in the new variant's partial and 0 in the old's
    int margin;    // cells the window reaches beyond R (dual translate steps)
    int varslab;   // 1: the per-pose-warp kernel's items come from pitem, each pose variant split
                   // into pnslab ranges in proportion to its window's work (nslab: their maximum)
    int pad2[3];
    int queue[2];  // pose-energy work counters of a launch whose first replica this is: [0] plain or
                   // all items, [1] difference-form items; each launch's last CTA resets its counter
    int done[2];   //   and this count of finished CTAs to 0
    U4 perm_key;
};

// One cell-list entry: the group's centre, id and atom range, so that the
// cell walk tests a candidate group and expands it into atoms from this one
// record (no further loads of the group's centre or atom range).
struct __align__(16) CellEnt {
    float4 c;   // group centre x, y, z; w: the group id (int bits)
    int2 span;  // atomStart, atomNum
    int2 pad;
};

struct RepDev {
    // geometry and physics
    float L[3], start[3];
    float invLc[3];
    int nc[3];          // cells per axis
    int span[3];        // cells visited per axis (min(2R+1, nc))
    int range;          // R
    int split_items;    // target work items per step (pose splits = target / poses)
    int max_split;      // splits per pose cap (window cells / 8)
    int cap;            // cell capacity
    float cutoff, grid_dx, trn_step, rot_max;
    double lncav;
    int proposal;
    int pair_image;     // 1: per-pair minimum image (small boxes); 0: per-group image shift
    int fast_incl;      // 1: multiply-based prefilter decides away from the cutoff (cutoff < L/2)
    float invL[3];
    float cut2_lo, cut2_hi;  // (cutoff*(1-1e-4))^2, (cutoff*(1+1e-4))^2
    int nfixed, ntypes, ffX, ffY, G;
    int mcsteps;
    uint32_t seed, replica;
    uint32_t step_base; // RNG step counter = step_base + local step (resume from a checkpoint)
    int run_end;        // steps below this index are executed
    int log_cap, log_kmax;
    // force-biased translate/rotate (proposal 2): each component of the
    // displacement (rotation vector) lies in [-h, h] with density ~ exp(a d),
    // a = lambda beta f, f the force (torque) at the old pose
    int fb;
    float fb_at, fb_ht;  // translate: lambda beta [mol/kJ], half-width h_t [A]
    float fb_ar, fb_hr;  // rotate: lambda beta [mol/kJ], half-width h_r [rad]
    // state
    float4* xyzq;       // atom x, y, z, charge
    int* atype;         // atom type (column of the LJ table)
    float4* gcen;       // group centre
    int2* gspan;        // (atomStart, atomNum)
    int* cell_count;
    CellEnt* cell_ent;  // [ncell * cap] entries of each cell, in increasing group id
    int* gcell;         // [ngroups] cell*cap + position, or -1
    float4* grid;       // insertion base points
    float2* lj;         // [ffX * ffY] (100*sigma^2 [nm^2 -> A^2], 4*eps)
    const int* moves;
    FragDev* frag;
    int* totalNum;      // [ntypes]
    // per-step scratch.  A replica advanced speculatively has two descriptors
    // whose scratch alternates by step parity (other: the second one); otherwise
    // other is the descriptor itself.
    const RepDev* other;
    int* valid;                         // speculating: this copy's step was prepared and evaluated
                                        // while the previous step accepted nothing
    unsigned long long* pairs_pending;  // speculating: pair count of that evaluation
    int* abort;                         // speculating: the step whose evaluation is void (the
                                        // step before it accepted a move); set while it runs
    int* spec_step;                     // speculating: the step this copy holds
    StepDesc* desc;
    float4* pcen;       // [kMaxPoses] pose centres (w unused)
    int* pslot;         // [kMaxPoses]
    double* epart;      // [kMaxPoses * 2 * nslab_max]
    uint32_t* nbr;      // [kMaxPoses * kMaxWords]
    // logs and counters
    gcmc_step_log* log;
    double* logE;
    unsigned long long* counters;  // steps, poses, pairs, then 8 accept-kernel phase cycle sums
    int* err;
    double* energy;     // running sum of the accepted moves' energy changes (FP64)
    float4* psite;      // [kMaxPoses * kMaxSites] trial sites (x, y, z, charge) of pose i, new variant
    double* pgum;       // [kMaxPoses] -ln(-ln u) Gumbel draw of pose i (clustering moves)
    double* plnu;       // [kMaxPoses] ln u of the acceptance draw of the cluster seeded by pose i
    // force-biased moves
    float* fpart;       // [kMaxPoses * 2 * nslab_max * 6] per-item force and torque partials
    float4* fbprop;     // [kMaxPoses * 2] (d or v, invalid flag), (a0, a1, a2, 0) of the old pose
    int* fbcnt;         // [kMaxPoses] old-pose items finished (reset by the last one)
    float* logF;        // [log_cap * log_kmax * 12] F_old, tau_old, F_new, tau_new used
    // tiled pose energies (k_energy_tiles): pose blocks of tblk^3 cells, nbk blocks
    // per axis, windows of tspan cells per axis (min(tblk + 2 range, nc); a translate
    // step's windows reach dmargin cells further); per step the preparation bins the
    // pose entries by block (pbin) and cuts the blocks into tiles (block, first entry
    // in pbin, entry count, entry count of the block's largest tile)
    int tiled;
    int tblk;
    int nbk[3];
    int tspan[3];
    int* pbin;          // [2 * kMaxPoses]
    int4* tiles;        // [2 * kMaxPoses]
    // per-pose splits of the per-pose-warp kernel: each cell's window work (atoms of the fixed
    // groups in the cells within R of it), and per step the ranges of each pose variant
    // (entry e = i * nvar + v) and the item list (e << 8 | range)
    const int* wcost;   // [ncell]
    int* pnslab;        // [2 * kMaxPoses]
    int* pitem;         // [2 * kMaxPoses * slab cap]
    // translate / rotate energy changes in the pairwise-difference form (dual = 1):
    // one work item per pose evaluates the old and the new pose together over the
    // groups within the cutoff of either centre; a translate's new centre lies
    // within dmargin cells of the old one's, so its windows reach dmargin cells further
    int dual;
    int dmargin;
    // Ewald electrostatics by smooth PME (pme = 1): real-space Coulomb erfc(alpha r)/r,
    // the reciprocal-space potential phi of the current state on a mesh (FP64),
    // interpolated at trial sites with order-4 B-splines
    int pme;
    float pme_alpha;
    int pme_n[3];
    const double* pme_phi;  // [n0 * n1 * n2] theta_rec * Q (kJ/mol/e)
    double* pme_q;          // [n0 * n1 * n2] spread charges of the current state
    double2* pme_spec;      // [n0 * n1 * (n2 / 2 + 1)] transform workspace
    const double* pme_g;    // [n0 * n1 * (n2 / 2 + 1)] influence function
    int* pme_dirty;         // 1: Q changed since phi was computed
    double pme_bgc;         // K pi / (2 V alpha^2): background energy -bgc Q^2
    double pme_qfix;        // total charge of the fixed atoms
};

__device__ __forceinline__ int wrapi(int c, int n) {
    c %= n;
    return c < 0 ? c + n : c;
}
__device__ __forceinline__ int cell_coord(float x, float start, float invLc, int nc) {
    const int c = __float2int_rd(fmul(fsub(x, start), invLc));
    return (unsigned)c < (unsigned)nc ? c : wrapi(c, nc);
}
__device__ __forceinline__ int cell_of(const RepDev& R, float x, float y, float z) {
    int cx = cell_coord(x, R.start[0], R.invLc[0], R.nc[0]);
    int cy = cell_coord(y, R.start[1], R.invLc[1], R.nc[1]);
    int cz = cell_coord(z, R.start[2], R.invLc[2], R.nc[2]);
    return (cz * R.nc[1] + cy) * R.nc[0] + cx;
}

// Centre of insertion pose i (gcmc/cpp/gcmc_energy.h:82-93): grid point + U(0,1]*dx.
__device__ __forceinline__ void insert_centre(const RepDev& R, int step, int i, float& x, float& y,
                                              float& z) {
    U4 r0 = rng(R.seed, R.replica, R.step_base + (uint32_t)step, (uint32_t)i, RP_INSERT, 0);
    int g = (int)(r0.x % (uint32_t)R.G);
    float4 gp = R.grid[g];
    x = fadd(fmul(u01_oc(r0.y), R.grid_dx), gp.x);
    y = fadd(fmul(u01_oc(r0.z), R.grid_dx), gp.y);
    z = fadd(fmul(u01_oc(r0.w), R.grid_dx), gp.z);
}

__device__ __forceinline__ Mat3 insert_rotation(const RepDev& R, int step, int i) {
    U4 r1 = rng(R.seed, R.replica, R.step_base + (uint32_t)step, (uint32_t)i, RP_INSERT, 1);
    if (R.proposal == 0) {
        float sn, cs;
        det_sincos(fmul(u01_oc(r1.w), kTwoPiF), sn, cs);
        return rodrigues(u01_oc(r1.x), u01_oc(r1.y), u01_oc(r1.z), sn, cs);
    }
    return shoemake(u01_co(r1.x), u01_co(r1.y), u01_co(r1.z));
}

// Translate shift of pose i with the box wrap of gcmc/cpp/gcmc_move_trn.h:57-66.
__device__ __forceinline__ float trn_shift(const RepDev& R, uint32_t r, int axis, float c) {
    float sh = R.proposal == 0 ? fmul(u01_oc(r), R.grid_dx) : fmul(fsub(u01_co(r), 0.5f), R.trn_step);
    float hi = fadd(R.L[axis], R.start[axis]);
    if (fadd(c, sh) > hi) sh = fsub(sh, R.L[axis]);
    if (fadd(c, sh) < R.start[axis]) sh = fadd(sh, R.L[axis]);
    return sh;
}

__device__ __forceinline__ Mat3 move_rotation(const RepDev& R, const U4& r) {
    if (R.proposal == 0) {
        float sn, cs;
        det_sincos(fmul(u01_oc(r.w), kTwoPiF), sn, cs);
        return rodrigues(u01_oc(r.x), u01_oc(r.y), u01_oc(r.z), sn, cs);
    }
    float z = fsub(fmul(2.0f, u01_co(r.x)), 1.0f);
    float sp, cp;
    det_sincos(fmul(u01_co(r.y), kTwoPiF), sp, cp);
    float rxy = fsqrt(fmaxf(0.0f, fsub(1.0f, fmul(z, z))));
    float theta = fmul(R.rot_max, fsub(fmul(2.0f, u01_co(r.z)), 1.0f));
    float sn, cs;
    det_sincos(theta, sn, cs);
    return rodrigues(fmul(rxy, cp), fmul(rxy, sp), z, sn, cs);
}

}  // namespace gcmc
