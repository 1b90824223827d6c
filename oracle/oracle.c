/*
 * CPU oracle for the GCMC hot path -- TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Compiled with -ffp-contract=off so every float operation written below is
 * rounded exactly once, as written; the places where the reference's CUDA
 * build fuses a multiply-add are written as explicit fmaf() calls.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Physical constants of the reference (gcmc/cpp/gcmc.h:28-41). */
#define OR_TEMPERATURE 300.0
#define OR_BOLTZMANN 0.0083115
#define OR_BETA (1.0 / (OR_BOLTZMANN * OR_TEMPERATURE))
#define OR_MOLES_TO_MOLECULES 0.0006023
#define OR_KCAL_TO_KJ 4.184
#define OR_COULOMB 1388.431112 /* gcmc/cpp/gcmc_energy.h:137 */
#define OR_TWO_PI_F 6.28318530717958647692f
#define OR_PI 3.14159265358979323846

/* RNG purposes (third counter word, high half). */
enum { RP_INSERT = 1, RP_DELETE = 2, RP_MOVE = 3, RP_CLUSTER = 4, RP_PERM = 5, RP_GUMBEL = 6, RP_FB = 7 };

/* ------------------------------------------------------------------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as    */
/* easy as 1, 2, 3", SC'11).                                                  */
/* ------------------------------------------------------------------------- */
void or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void rng(uint32_t seed, uint32_t replica, uint32_t step, uint32_t index, uint32_t purpose,
                uint32_t draw, uint32_t out[4]) {
    uint32_t ctr[4] = {step, index, (purpose << 16) | draw, 0u};
    uint32_t key[2] = {seed, replica};
    or_philox(ctr, key, out);
}

/* uniform float in (0,1] and [0,1) from the top 24 bits */
static inline float u01_oc(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f; }
static inline float u01_co(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }
/* uniform double in [0,1) from 53 bits of two words */
static inline double u53(uint32_t a, uint32_t b) {
    uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return (double)m * 1.1102230246251565e-16;
}
/* uniform double in (0,1) */
static inline double u53_open(uint32_t a, uint32_t b) {
    uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return ((double)m + 0.5) * 1.1102230246251565e-16;
}

/* ------------------------------------------------------------------------- */
/* Deterministic sin/cos: two-constant reduction by pi/2, then the Taylor     */
/* polynomials of sin (to r^9) and cos (to r^10) on |r| <= pi/4.  Only         */
/* correctly rounded operations, so CPU and GPU agree bit for bit.            */
/* ------------------------------------------------------------------------- */
void or_det_sincos(float x, float* s_out, float* c_out) {
    const float two_over_pi = 0.636619772367581343f;
    const float pio2_hi = 1.57079637050628662109375f;     /* float(pi/2)          */
    const float pio2_lo = -4.37113900018624283e-8f;       /* pi/2 - float(pi/2)   */
    float kf = rintf(x * two_over_pi);
    float r = fmaf(-kf, pio2_hi, x);
    r = fmaf(-kf, pio2_lo, r);
    float r2 = r * r;
    float ps = fmaf(r2, 2.75573192239858925e-6f, -1.98412698412698413e-4f);
    ps = fmaf(r2, ps, 8.33333333333333333e-3f);
    ps = fmaf(r2, ps, -1.66666666666666667e-1f);
    float sr = fmaf(r * r2, ps, r);
    float pc = fmaf(r2, -2.75573192239858925e-7f, 2.48015873015873016e-5f);
    pc = fmaf(r2, pc, -1.38888888888888889e-3f);
    pc = fmaf(r2, pc, 4.16666666666666667e-2f);
    pc = fmaf(r2, pc, -0.5f);
    float cr = fmaf(r2, pc, 1.0f);
    int q = ((int)kf) & 3;
    float s, c;
    switch (q) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
    *s_out = s;
    *c_out = c;
}

/* Own natural logarithm (engine: det_log in common.cuh): x = m 2^e with m in
 * [sqrt(1/2), sqrt(2)), ln m = 2 atanh((m-1)/(m+1)) as an odd series. */
float or_det_log(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    int e = (int)((b >> 23) & 0xffu) - 127;
    uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
    float m;
    memcpy(&m, &mb, 4);
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = s2 * 0.0909090936f + 0.111111112f;
    p = s2 * p + 0.142857149f;
    p = s2 * p + 0.200000003f;
    p = s2 * p + 0.333333343f;
    p = s2 * p + 1.0f;
    const float lnm = (2.0f * s) * p;
    const float ef = (float)e;
    return ef * 0.693145751953125f + (ef * 1.42860677e-06f + lnm);
}

/* Own exponential for x <= 0 (engine: det_exp_neg). */
float or_det_exp_neg(float x) {
    if (!(x > -87.0f)) return 0.0f;
    const float kf = floorf(x * 1.44269502f + 0.5f);
    const float r = (x - kf * 0.693145751953125f) - kf * 1.42860677e-06f;
    float p = r * 1.98412701e-04f + 1.38888892e-03f;
    p = r * p + 8.33333377e-03f;
    p = r * p + 4.16666679e-02f;
    p = r * p + 0.166666672f;
    p = r * p + 0.5f;
    p = r * p + 1.0f;
    p = r * p + 1.0f;
    const int k = (int)kf;
    const uint32_t sb = (uint32_t)(k + 127) << 23;
    float sc;
    memcpy(&sc, &sb, 4);
    return p * sc;
}

/* Tilted-uniform draw on [-h, h] with density a e^{ax} / (2 sinh(ah)) (force
 * bias of Pangali, Rao and Berne 1978; engine: fb_tilted). */
static float fb_tilted(float a, float h, float u) {
    const float ah = a * h;
    if (fabsf(ah) < 1e-4f) return h * (2.0f * u - 1.0f);
    if (a > 0.0f) {
        const float t = or_det_exp_neg(-2.0f * ah);
        return h + or_det_log(u + (1.0f - u) * t) / a;
    }
    const float t = or_det_exp_neg(2.0f * ah);
    return -h + or_det_log((1.0f - u) + u * t) / a;
}

/* ln(a / (2 sinh(ah))) (engine: fb_lnorm). */
static float fb_lnorm(float a, float h) {
    const float b = fabsf(a * h);
    if (b < 1e-2f) {
        const float b2 = b * b;
        return (-or_det_log(2.0f * h) - b2 / 6.0f) + (b2 * b2) / 180.0f;
    }
    return (or_det_log(fabsf(a)) - b) - or_det_log(1.0f - or_det_exp_neg(-2.0f * b));
}

/* Rodrigues matrix about axis a (normalised here) by angle with (sin, cos);
 * formulas of gcmc/cpp/gcmc_energy.h:39-58 with the fused form fixed. */
static void rodrigues(const float axis[3], float sn, float cs, float R[3][3]) {
    float a0 = axis[0], a1 = axis[1], a2 = axis[2];
    float nn = a0 * a0;
    nn = fmaf(a1, a1, nn);
    nn = fmaf(a2, a2, nn);
    float norm = sqrtf(nn);
    a0 = a0 / norm; a1 = a1 / norm; a2 = a2 / norm;
    float C = 1.0f - cs;
    R[0][0] = fmaf(a0 * a0, C, cs);
    R[0][1] = fmaf(a0 * a1, C, -(a2 * sn));
    R[0][2] = fmaf(a0 * a2, C, a1 * sn);
    R[1][0] = fmaf(a1 * a0, C, a2 * sn);
    R[1][1] = fmaf(a1 * a1, C, cs);
    R[1][2] = fmaf(a1 * a2, C, -(a0 * sn));
    R[2][0] = fmaf(a2 * a0, C, -(a1 * sn));
    R[2][1] = fmaf(a2 * a1, C, a0 * sn);
    R[2][2] = fmaf(a2 * a2, C, cs);
}

/* Uniform rotation from three uniforms (Shoemake, "Uniform random rotations",
 * Graphics Gems III, 1992): unit quaternion -> matrix. */
static void shoemake(float u1, float u2, float u3, float R[3][3]) {
    float s2, c2, s3, c3;
    or_det_sincos(u2 * OR_TWO_PI_F, &s2, &c2);
    or_det_sincos(u3 * OR_TWO_PI_F, &s3, &c3);
    float r1 = sqrtf(1.0f - u1), r2 = sqrtf(u1);
    float x = r1 * s2, y = r1 * c2, z = r2 * s3, w = r2 * c3;
    float xx = x * x, yy = y * y, zz = z * z;
    float xy = x * y, xz = x * z, yz = y * z, xw = x * w, yw = y * w, zw = z * w;
    R[0][0] = 1.0f - 2.0f * (yy + zz);
    R[0][1] = 2.0f * (xy - zw);
    R[0][2] = 2.0f * (xz + yw);
    R[1][0] = 2.0f * (xy + zw);
    R[1][1] = 1.0f - 2.0f * (xx + zz);
    R[1][2] = 2.0f * (yz - xw);
    R[2][0] = 2.0f * (xz - yw);
    R[2][1] = 2.0f * (yz + xw);
    R[2][2] = 1.0f - 2.0f * (xx + yy);
}

/* p' = R p (gcmc/cpp/gcmc_energy.h:62-71 accumulation order, fused) */
static inline void rotate(const float R[3][3], const float p[3], float out[3]) {
    for (int j = 0; j < 3; ++j) {
        float x = p[0] * R[j][0];
        x = fmaf(p[1], R[j][1], x);
        x = fmaf(p[2], R[j][2], x);
        out[j] = x;
    }
}

/* ------------------------------------------------------------------------- */
/* Distances (gcmc/cpp/gcmc_energy.h:110-122).                                */
/* ------------------------------------------------------------------------- */
static inline float fast_round_f(float a) {
    return a >= 0.0f ? (float)(int)(a + 0.5f) : (float)(int)(a - 0.5f);
}
static inline double fast_round_d(double a) {
    return a >= 0.0 ? trunc(a + 0.5) : trunc(a - 0.5);
}

float or_dist_group(const float a[3], const float b[3], const float L[3]) {
    float d[3];
    for (int i = 0; i < 3; ++i) {
        float x = a[i] - b[i];
        float r = fast_round_f(x / L[i]);
        d[i] = fmaf(-r, L[i], x);
    }
    float s = d[0] * d[0];
    s = fmaf(d[1], d[1], s);
    s = fmaf(d[2], d[2], s);
    return sqrtf(s);
}

float or_dist_host(const float a[3], const float b[3], const float L[3]) {
    float d[3];
    for (int i = 0; i < 3; ++i) {
        float x = a[i] - b[i];
        float r = fast_round_f(x / L[i]);
        d[i] = x - r * L[i];
    }
    float s = d[0] * d[0] + d[1] * d[1];
    s = s + d[2] * d[2];
    return sqrtf(s);
}

/* ------------------------------------------------------------------------- */
/* Pose energy (gcmc/cpp/gcmc_energy.h:142-204).                              */
/* ------------------------------------------------------------------------- */
static double group_pairs64a(const or_info* info, const or_atom* atoms, const float* ff, int a0,
                             int na, const float (*sx)[3], const float* sq, const int32_t* st,
                             int ns, double* l1, double alpha) {
    const double L[3] = {info->cryst[0], info->cryst[1], info->cryst[2]};
    double e = 0.0;
    for (int a = a0; a < a0 + na; ++a) {
        const or_atom* A = &atoms[a];
        for (int s = 0; s < ns; ++s) {
            double d2 = 0.0;
            for (int i = 0; i < 3; ++i) {
                double d = (double)A->position[i] - (double)sx[s][i];
                d -= fast_round_d(d / L[i]) * L[i];
                d2 += d * d;
            }
            int tij = st[s] * info->ffYNum + A->type;
            double sig = ff[2 * tij], eps = ff[2 * tij + 1];
            double s2 = sig * sig * 100.0 / d2;
            double s6 = s2 * s2 * s2;
            double lj = 4.0 * eps * (s6 * s6 - s6);
            double el = OR_COULOMB * (double)sq[s] * (double)A->charge / sqrt(d2);
            if (alpha > 0.0) el *= erfc(alpha * sqrt(d2));  /* Ewald real-space kernel */
            e += lj + el;
            *l1 += fabs(lj) + fabs(el);
        }
    }
    return e;
}

static double group_pairs64(const or_info* info, const or_atom* atoms, const float* ff, int a0, int na,
                            const float (*sx)[3], const float* sq, const int32_t* st, int ns, double* l1) {
    return group_pairs64a(info, atoms, ff, a0, na, sx, sq, st, ns, l1, 0.0);
}

/* FP32 mirror of one reference thread's pair work on one group. */
static float group_pairs32(const or_info* info, const or_atom* atoms, const float* ff, int a0, int na,
                           const float (*sx)[3], const float* sq, const int32_t* st, int ns,
                           float acc) {
    for (int a = a0; a < a0 + na; ++a) {
        const or_atom* A = &atoms[a];
        for (int s = 0; s < ns; ++s) {
            float dist = or_dist_group(A->position, sx[s], info->cryst);
            int tij = st[s] * info->ffYNum + A->type;
            float sigma = ff[2 * tij], epsilon = ff[2 * tij + 1];
            float sigma_sqrd = sigma * sigma * 100.0f;
            float sd = sigma_sqrd / (dist * dist);
            float vdw = 4.0f * epsilon * (powf(sd, 6.0f) - powf(sd, 3.0f));
            acc = acc + vdw;
            double el = OR_COULOMB * (double)(sq[s] * A->charge) / (double)dist;
            acc = (float)((double)acc + el);
        }
    }
    return acc;
}

double or_pose_energy(const or_info* info, const or_atomarray* frag, const or_residue* res,
                      const or_atom* atoms, const float* ff, const float (*sx)[3],
                      const float* sq, const int32_t* st, int32_t ns, const float centre[3],
                      int32_t self, int32_t mode, int32_t* n_groups, int64_t* pairs) {
    return or_pose_energy_l1(info, frag, res, atoms, ff, sx, sq, st, ns, centre, self, mode, n_groups, pairs,
                             NULL);
}

/* FP64 real-space pose energy with the Ewald real-space kernel erfc(alpha r)/r
 * for Coulomb (alpha = 0: plain 1/r, calcEnergy's form). */
static double pose_energy64a(const or_info* info, const or_atomarray* frag, const or_residue* res,
                             const or_atom* atoms, const float* ff, const float (*sx)[3], const float* sq,
                             const int32_t* st, int32_t ns, const float centre[3], int32_t self, double alpha,
                             double* l1_out) {
    double e = 0.0, l1 = 0.0;
    for (int t = -1; t < info->fragTypeNum; ++t) {
        const int g0 = t < 0 ? 0 : frag[t].startRes;
        const int g1 = t < 0 ? frag[0].startRes : g0 + frag[t].totalNum;
        for (int g = g0; g < g1; ++g) {
            if (g == self) continue;
            if (or_dist_group(centre, res[g].position, info->cryst) <= info->cutoff)
                e += group_pairs64a(info, atoms, ff, res[g].atomStart, res[g].atomNum, sx, sq, st, ns, &l1, alpha);
        }
    }
    if (l1_out) *l1_out = l1;
    return e;
}

double or_pose_energy_l1(const or_info* info, const or_atomarray* frag, const or_residue* res,
                         const or_atom* atoms, const float* ff, const float (*sx)[3],
                         const float* sq, const int32_t* st, int32_t ns, const float centre[3],
                         int32_t self, int32_t mode, int32_t* n_groups, int64_t* pairs, double* l1_out) {
    int ng = 0;
    int64_t np = 0;
    double l1 = 0.0;
    const int nfixed = frag[0].startRes;
    if (mode == 0) {
        double e = 0.0;
        for (int g = 0; g < nfixed; ++g) {
            if (or_dist_group(centre, res[g].position, info->cryst) <= info->cutoff) {
                e += group_pairs64(info, atoms, ff, res[g].atomStart, res[g].atomNum, sx, sq, st, ns, &l1);
                ng++;
                np += (int64_t)res[g].atomNum * ns;
            }
        }
        for (int t = 0; t < info->fragTypeNum; ++t) {
            int g0 = frag[t].startRes, g1 = g0 + frag[t].totalNum;
            for (int g = g0; g < g1; ++g) {
                if (g == self) continue;
                if (or_dist_group(centre, res[g].position, info->cryst) <= info->cutoff) {
                    e += group_pairs64(info, atoms, ff, res[g].atomStart, res[g].atomNum, sx, sq, st, ns, &l1);
                    ng++;
                    np += (int64_t)res[g].atomNum * ns;
                }
            }
        }
        if (n_groups) *n_groups = ng;
        if (pairs) *pairs = np;
        if (l1_out) *l1_out = l1;
        return e;
    }
    /* FP32 mirror: 128 virtual threads, strided group loops, tree reduction */
    float sh[128];
    for (int tid = 0; tid < 128; ++tid) {
        float acc = 0.0f;
        for (int g = tid; g < nfixed; g += 128) {
            if (or_dist_group(centre, res[g].position, info->cryst) <= info->cutoff) {
                acc = group_pairs32(info, atoms, ff, res[g].atomStart, res[g].atomNum, sx, sq, st, ns, acc);
                ng++;
                np += (int64_t)res[g].atomNum * ns;
            }
        }
        for (int t = 0; t < info->fragTypeNum; ++t) {
            int g0 = frag[t].startRes, g1 = g0 + frag[t].totalNum;
            for (int g = tid + g0; g < g1; g += 128) {
                if (g != self && or_dist_group(centre, res[g].position, info->cryst) <= info->cutoff) {
                    acc = group_pairs32(info, atoms, ff, res[g].atomStart, res[g].atomNum, sx, sq, st, ns, acc);
                    ng++;
                    np += (int64_t)res[g].atomNum * ns;
                }
            }
        }
        sh[tid] = acc;
    }
    for (int s = 64; s > 0; s >>= 1)
        for (int tid = 0; tid < s; ++tid) sh[tid] += sh[tid + s];
    if (n_groups) *n_groups = ng;
    if (pairs) *pairs = np;
    return (double)sh[0];
}

/* ------------------------------------------------------------------------- */
/* Proposals (gcmc/cpp/gcmc_energy.h:75-107, gcmc_move_trn.h:54-75,           */
/* gcmc_move_rot.h:62-101).                                                  */
/* ------------------------------------------------------------------------- */
void or_insert_pose(const or_info* info, const or_atomarray* frag, const float* grid,
                    const or_options* opt, int32_t ftype, int32_t step, int32_t i,
                    float (*xyz)[3], float centre[3]) {
    uint32_t r0[4], r1[4];
    rng(info->seed, opt->replica, (uint32_t)step, (uint32_t)i, RP_INSERT, 0, r0);
    rng(info->seed, opt->replica, (uint32_t)step, (uint32_t)i, RP_INSERT, 1, r1);
    int g = (int)(r0[0] % (uint32_t)info->totalGridNum);
    float t[3];
    for (int j = 0; j < 3; ++j) {
        float off = u01_oc(r0[1 + j]) * info->grid_dx;
        t[j] = off + grid[3 * g + j];
    }
    float R[3][3];
    if (opt->proposal == 0) {
        float axis[3] = {u01_oc(r1[0]), u01_oc(r1[1]), u01_oc(r1[2])};
        float phi = u01_oc(r1[3]) * OR_TWO_PI_F;
        float sn, cs;
        or_det_sincos(phi, &sn, &cs);
        rodrigues(axis, sn, cs, R);
    } else {
        shoemake(u01_co(r1[0]), u01_co(r1[1]), u01_co(r1[2]), R);
    }
    const or_atomarray* F = &frag[ftype];
    for (int s = 0; s < F->num_atoms; ++s) {
        float p[3];
        rotate(R, F->atoms[s].position, p);
        for (int j = 0; j < 3; ++j) xyz[s][j] = p[j] + t[j];
    }
    for (int j = 0; j < 3; ++j) centre[j] = t[j];
}

void or_move_pose(const or_info* info, const or_atomarray* frag, const or_residue* res,
                  const or_atom* atoms, const or_options* opt, int32_t ftype, int32_t move,
                  int32_t step, int32_t i, int32_t slot, float (*xyz)[3], float centre[3]) {
    const or_atomarray* F = &frag[ftype];
    const or_residue* Rs = &res[F->startRes + slot];
    const int ns = F->num_atoms;
    uint32_t r[4];
    rng(info->seed, opt->replica, (uint32_t)step, (uint32_t)i, RP_MOVE, 0, r);
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < 3; ++j) xyz[s][j] = atoms[Rs->atomStart + s].position[j];
    if (move == 2) {
        for (int j = 0; j < 3; ++j) {
            float sh = opt->proposal == 0 ? u01_oc(r[j]) * info->grid_dx
                                          : (u01_co(r[j]) - 0.5f) * opt->trn_step;
            float c = Rs->position[j];
            float hi = info->cryst[j] + info->startxyz[j];
            if (c + sh > hi) sh = sh - info->cryst[j];
            if (c + sh < info->startxyz[j]) sh = sh + info->cryst[j];
            centre[j] = c + sh;
            for (int s = 0; s < ns; ++s) xyz[s][j] = xyz[s][j] + sh;
        }
        return;
    }
    /* rotate about the unweighted centroid; residue centre unchanged */
    float R[3][3];
    if (opt->proposal == 0) {
        float axis[3] = {u01_oc(r[0]), u01_oc(r[1]), u01_oc(r[2])};
        float phi = u01_oc(r[3]) * OR_TWO_PI_F;
        float sn, cs;
        or_det_sincos(phi, &sn, &cs);
        rodrigues(axis, sn, cs, R);
    } else {
        float z = 2.0f * u01_co(r[0]) - 1.0f;
        float sp, cp;
        or_det_sincos(u01_co(r[1]) * OR_TWO_PI_F, &sp, &cp);
        float rxy = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float axis[3] = {rxy * cp, rxy * sp, z};
        float theta = opt->rot_max * (2.0f * u01_co(r[2]) - 1.0f);
        float sn, cs;
        or_det_sincos(theta, &sn, &cs);
        rodrigues(axis, sn, cs, R);
    }
    float cen[3] = {0.0f, 0.0f, 0.0f};
    for (int j = 0; j < 3; ++j)
        for (int s = 0; s < ns; ++s) cen[j] = cen[j] + xyz[s][j] / (float)ns;
    for (int s = 0; s < ns; ++s) {
        float q[3] = {xyz[s][0] - cen[0], xyz[s][1] - cen[1], xyz[s][2] - cen[2]};
        float p[3];
        rotate(R, q, p);
        for (int j = 0; j < 3; ++j) xyz[s][j] = p[j] + cen[j];
    }
    for (int j = 0; j < 3; ++j) centre[j] = Rs->position[j];
}

/* Keyed permutation of [0,n): 4-round Feistel network on the smallest even
 * bit width covering n, with cycle walking; round function = murmur3 fmix32. */
static inline uint32_t fmix32(uint32_t h) {
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
    return h;
}
int32_t or_perm_slot(const or_options* opt, uint32_t seed, int32_t step, int32_t i, int32_t n) {
    uint32_t rk[4];
    rng(seed, opt->replica, (uint32_t)step, 0u, RP_PERM, 0, rk);
    int h = 1;
    while ((1u << (2 * h)) < (uint32_t)n) ++h;
    uint32_t mask = (1u << h) - 1u;
    uint32_t x = (uint32_t)i;
    do {
        uint32_t Lh = x >> h, Rh = x & mask;
        for (int r = 0; r < 4; ++r) {
            uint32_t nl = Rh;
            Rh = Lh ^ (fmix32(Rh ^ rk[r]) & mask);
            Lh = nl;
        }
        x = (Lh << h) | Rh;
    } while (x >= (uint32_t)n);
    return (int32_t)x;
}

/* ------------------------------------------------------------------------- */
/* Cluster / Rosenbluth / acceptance pass (gcmc_move_add.h:107-191,           */
/* gcmc_move_trn.h:160-244).                                                  */
/* ------------------------------------------------------------------------- */
/* Decision margins (test statistics): for every acceptance decision, the
 * distance |ln u - ln p| / beta of the draw from the threshold in energy units,
 * against the largest per-trial tolerance max(1e-5 |E|, 1e-4 kcal/mol) of the
 * energies the decision depends on (ln p moves by at most beta times the
 * largest error of those energies: ln W is a log-sum-exp).  A decision inside
 * that band may legitimately differ between two evaluations of the energies
 * that both meet the per-trial criterion. */
static long long g_dec_total = 0, g_dec_band = 0;
static double g_dec_min_ratio = INFINITY;

static void note_decision(double lnp, double u, double tol) {
    if (isnan(lnp) || !(tol > 0.0)) return;
    g_dec_total++;
    /* accepted for sure when lnp >= 0: its margin is lnp itself */
    const double m = (lnp >= 0.0 ? lnp : fabs(log(u) - lnp)) / OR_BETA;
    if (m <= tol) g_dec_band++;
    if (m / tol < g_dec_min_ratio) g_dec_min_ratio = m / tol;
}

static double trial_tol(double e) { return fmax(1e-5 * fabs(e), 1e-4 * 4.184); }

void or_decision_stats(int32_t reset, int64_t* total, int64_t* band, double* min_ratio) {
    if (total) *total = g_dec_total;
    if (band) *band = g_dec_band;
    if (min_ratio) *min_ratio = g_dec_min_ratio;
    if (reset) {
        g_dec_total = 0;
        g_dec_band = 0;
        g_dec_min_ratio = INFINITY;
    }
}

typedef struct {
    int kind;        /* 0 insert, 1 translate/rotate */
    double lncav;    /* insert: ln(cavityFactor)     */
    double B;        /* insert: beta*muex + ln(Nbar) */
    int* n;          /* insert: running totalNum     */
    int maxNum;
} cluster_par;

static int cluster_pass(const or_info* info, const or_options* opt, int step, int k,
                        const double* E, const float (*c)[3], const cluster_par* P,
                        int* accepted, int* inserted, int* n_acc, int* first_accept) {
    const double beta = OR_BETA;
    unsigned char* U = (unsigned char*)malloc((size_t)k);
    int* mem = (int*)malloc(sizeof(int) * (size_t)k);
    memset(U, 1, (size_t)k);
    int nclus = 0, na = 0;
    *first_accept = -1;
    for (int s = 0; s < k; ++s) {
        if (!U[s]) continue;
        nclus++;
        int nm = 0;
        mem[nm++] = s; /* the seed is always a member */
        for (int i = s + 1; i < k; ++i)
            if (U[i] && or_dist_host(c[s], c[i], info->cryst) <= info->cutoff) mem[nm++] = i;
        double emin = INFINITY;
        for (int m = 0; m < nm; ++m)
            if (isfinite(E[mem[m]]) && E[mem[m]] < emin) emin = E[mem[m]];
        int chosen = s;
        int acc = 0;
        if (isfinite(emin)) {
            double W = 0.0, best = -INFINITY;
            for (int m = 0; m < nm; ++m) {
                int i = mem[m];
                if (!isfinite(E[i])) continue;
                W += exp(-beta * (E[i] - emin));
                uint32_t g[4];
                rng(info->seed, opt->replica, (uint32_t)step, (uint32_t)i, RP_GUMBEL, 0, g);
                double key = -beta * E[i] - log(-log(u53_open(g[0], g[1])));
                if (key > best) { best = key; chosen = i; }
            }
            double lnp = log(W) - log((double)nm) - beta * emin;
            if (P->kind == 0) lnp += P->lncav + P->B - log((double)(*P->n) + 1.0);
            uint32_t ua[4];
            rng(info->seed, opt->replica, (uint32_t)step, (uint32_t)s, RP_CLUSTER, 0, ua);
            double u = u53(ua[0], ua[1]);
            acc = !isnan(lnp) && (lnp >= 0.0 || u < exp(lnp));
            double tol = 0.0;
            for (int m = 0; m < nm; ++m)
                if (isfinite(E[mem[m]])) tol = fmax(tol, trial_tol(E[mem[m]]));
            note_decision(lnp, u, tol);
        }
        for (int m = 0; m < nm; ++m) U[mem[m]] = 0;
        if (acc) {
            for (int i = s + 1; i < k; ++i)
                if (U[i] && or_dist_host(c[chosen], c[i], info->cryst) <= info->cutoff) U[i] = 0;
            if (*first_accept < 0) *first_accept = chosen;
            int ins = 1;
            if (P->kind == 0) {
                if (*P->n < P->maxNum) (*P->n)++;
                else ins = 0;
            }
            accepted[na] = chosen;
            inserted[na] = ins;
            na++;
        }
    }
    free(U);
    free(mem);
    *n_acc = na;
    return nclus;
}

/* ------------------------------------------------------------------------- */
/* FP64 inputs and analytic gradients of calcEnergy's pair sum.               */
/*                                                                            */
/* Same group inclusion as or_pose_energy (the FP32 group-centre distance of  */
/* gcmc_energy.h:160-176 against the float pose centre), but sites, site      */
/* charges and the pair table are double, so that central finite differences  */
/* of these energies resolve steps of 1e-4 A / 1e-5 relative.  The gradient    */
/* of each pair term (minimum-image d = atom - site, d2 = |d|^2):             */
/*   U = 4 eps (s6^2 - s6) + K q_s q_a / r,  s6 = (100 sigma^2 / d2)^3         */
/*   dU/dd2 = -12 eps s6 (2 s6 - 1) / d2 - U_el / (2 d2)                      */
/*   dU/dx_s = -2 dU/dd2 d,  dU/dq_s = K q_a / r,                             */
/*   dU/dsigma = 24 eps (2 s6 - 1) s6 / sigma,  dU/deps = 4 (s6^2 - s6).        */
/* ------------------------------------------------------------------------- */
typedef struct {
    const or_info* info;
    const or_atomarray* frag;
    const or_residue* res;
    const or_atom* atoms;
    const double* ff;
    const double (*sx)[3];
    const double* sq;
    const int32_t* st;
    int ns;
    double alpha;  /* > 0: Ewald real-space Coulomb K q q erfc(alpha r) / r */
} pose64;

/* Visit every included group of a pose (fixed groups, then occupied slots). */
#define OR_FOR_INCLUDED(P, centre, self, ...)                                          \
    do {                                                                               \
        const int nfixed_ = (P)->frag[0].startRes;                                     \
        for (int t_ = -1; t_ < (P)->info->fragTypeNum; ++t_) {                         \
            const int g0_ = t_ < 0 ? 0 : (P)->frag[t_].startRes;                       \
            const int g1_ = t_ < 0 ? nfixed_ : g0_ + (P)->frag[t_].totalNum;          \
            for (int g = g0_; g < g1_; ++g) {                                          \
                if (g == (self)) continue;                                             \
                if (or_dist_group((centre), (P)->res[g].position, (P)->info->cryst) >   \
                    (P)->info->cutoff)                                                 \
                    continue;                                                          \
                __VA_ARGS__                                                            \
            }                                                                          \
        }                                                                              \
    } while (0)

static double pose_energy64(const pose64* P, const float centre[3], int self, int32_t* ngroups) {
    const double L[3] = {P->info->cryst[0], P->info->cryst[1], P->info->cryst[2]};
    double e = 0.0;
    int ng = 0;
    OR_FOR_INCLUDED(P, centre, self, {
        ng++;
        for (int a = P->res[g].atomStart; a < P->res[g].atomStart + P->res[g].atomNum; ++a) {
            const or_atom* A = &P->atoms[a];
            for (int s = 0; s < P->ns; ++s) {
                double d2 = 0.0;
                for (int i = 0; i < 3; ++i) {
                    double d = (double)A->position[i] - P->sx[s][i];
                    d -= fast_round_d(d / L[i]) * L[i];
                    d2 += d * d;
                }
                const int tij = P->st[s] * P->info->ffYNum + A->type;
                const double sig = P->ff[2 * tij], eps = P->ff[2 * tij + 1];
                const double s2 = sig * sig * 100.0 / d2, s6 = s2 * s2 * s2;
                e += 4.0 * eps * (s6 * s6 - s6) + OR_COULOMB * P->sq[s] * (double)A->charge / sqrt(d2);
            }
        }
    });
    if (ngroups) *ngroups = ng;
    return e;
}

/* gxyz[ns*3], gq[ns] of one pose; gff (+= w * dE/dff) and the l1 scales
 * (sums of |terms|: per site over its three components, per site charge, per
 * table entry). */
static void pose_grad64(const pose64* P, const float centre[3], int self, double w, double* gxyz, double* gq,
                        double* gff, double* gxyz_l1, double* gq_l1, double* gff_l1) {
    const double L[3] = {P->info->cryst[0], P->info->cryst[1], P->info->cryst[2]};
    for (int s = 0; s < P->ns; ++s) {
        gxyz[3 * s] = gxyz[3 * s + 1] = gxyz[3 * s + 2] = 0.0;
        gq[s] = 0.0;
        if (gxyz_l1) gxyz_l1[s] = 0.0;
        if (gq_l1) gq_l1[s] = 0.0;
    }
    OR_FOR_INCLUDED(P, centre, self, {
        for (int a = P->res[g].atomStart; a < P->res[g].atomStart + P->res[g].atomNum; ++a) {
            const or_atom* A = &P->atoms[a];
            for (int s = 0; s < P->ns; ++s) {
                double d[3], d2 = 0.0;
                for (int i = 0; i < 3; ++i) {
                    d[i] = (double)A->position[i] - P->sx[s][i];
                    d[i] -= fast_round_d(d[i] / L[i]) * L[i];
                    d2 += d[i] * d[i];
                }
                const int tij = P->st[s] * P->info->ffYNum + A->type;
                const double sig = P->ff[2 * tij], eps = P->ff[2 * tij + 1];
                const double s2 = sig * sig * 100.0 / d2, s6 = s2 * s2 * s2;
                const double r = sqrt(d2);
                double el = OR_COULOMB * P->sq[s] * (double)A->charge / r, gel = el, kr = 1.0 / r;
                if (P->alpha > 0.0) { /* d/d(d2) of K q q erfc(a r) / r */
                    const double ec = erfc(P->alpha * r);
                    el *= ec;
                    kr *= ec;
                    gel = el + OR_COULOMB * P->sq[s] * (double)A->charge * 2.0 * P->alpha / sqrt(OR_PI) *
                                   exp(-P->alpha * P->alpha * d2);
                }
                const double dd2 = -12.0 * eps * s6 * (2.0 * s6 - 1.0) / d2 - 0.5 * gel / d2;
                for (int i = 0; i < 3; ++i) {
                    const double gi = -2.0 * dd2 * d[i];
                    gxyz[3 * s + i] += gi;
                    if (gxyz_l1) gxyz_l1[s] += fabs(gi);
                }
                const double gqi = OR_COULOMB * (double)A->charge * kr;
                gq[s] += gqi;
                if (gq_l1) gq_l1[s] += fabs(gqi);
                if (gff) {
                    /* dU/dsigma = 24 eps s6 (2 s6 - 1) / sigma, written without the division */
                    const double c3 = 100.0 / d2 * (100.0 / d2) * (100.0 / d2);
                    const double s5 = sig * sig * sig * sig * sig;
                    const double gs = w * 4.0 * eps * (2.0 * s6 - 1.0) * 6.0 * s5 * c3;
                    const double ge = w * 4.0 * (s6 * s6 - s6);
                    gff[2 * tij] += gs;
                    gff[2 * tij + 1] += ge;
                    if (gff_l1) {
                        gff_l1[2 * tij] += fabs(gs);
                        gff_l1[2 * tij + 1] += fabs(ge);
                    }
                }
            }
        }
    });
}

/* ------------------------------------------------------------------------- */
/* Ewald electrostatics (not in the reference): exact reciprocal-space        */
/* potential by a direct k-space sum, for checking the engine's smooth PME.   */
/* ------------------------------------------------------------------------- */
typedef struct {
    int nk, n[3];
    int* idx;       /* [nk*3] integer wave vector (half space)                 */
    double* coef;   /* [nk] 2 K exp(-pi^2 m^2/alpha^2) / (pi V m^2)            */
    double* sre;    /* [nk] Re S(m)                                             */
    double* sim;    /* [nk] Im S(m)                                             */
    double L[3];
} ewald_t;

static void ewald_free(ewald_t* E) {
    free(E->idx); free(E->coef); free(E->sre); free(E->sim);
    memset(E, 0, sizeof(*E));
}

static int ewald_init(ewald_t* E, const or_info* info, double alpha) {
    memset(E, 0, sizeof(*E));
    const double mmax = alpha * sqrt(-log(1e-13)) / OR_PI;
    const double V = (double)info->cryst[0] * info->cryst[1] * info->cryst[2];
    for (int d = 0; d < 3; ++d) {
        E->L[d] = info->cryst[d];
        E->n[d] = (int)ceil(mmax * E->L[d]);
    }
    const size_t cap = (size_t)(E->n[0] + 1) * (2 * E->n[1] + 1) * (2 * E->n[2] + 1);
    E->idx = malloc(sizeof(int) * 3 * cap);
    E->coef = malloc(sizeof(double) * cap);
    if (!E->idx || !E->coef) return -1;
    for (int a = 0; a <= E->n[0]; ++a)
        for (int b = -E->n[1]; b <= E->n[1]; ++b)
            for (int c = -E->n[2]; c <= E->n[2]; ++c) {
                if (a == 0 && (b < 0 || (b == 0 && c <= 0))) continue; /* half space, m != 0 */
                const double m[3] = {a / E->L[0], b / E->L[1], c / E->L[2]};
                const double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                if (m2 > mmax * mmax) continue;
                E->idx[3 * E->nk] = a; E->idx[3 * E->nk + 1] = b; E->idx[3 * E->nk + 2] = c;
                E->coef[E->nk] = 2.0 * OR_COULOMB * exp(-OR_PI * OR_PI * m2 / (alpha * alpha)) / (OR_PI * V * m2);
                E->nk++;
            }
    E->sre = calloc((size_t)E->nk, sizeof(double));
    E->sim = calloc((size_t)E->nk, sizeof(double));
    return (E->sre && E->sim) ? 0 : -1;
}

/* e^{2 pi i n x / L} for n = -N..N by repeated multiplication */
static void ewald_powers(double x, double L, int N, double* re, double* im) {
    const double th = 2.0 * OR_PI * x / L;
    const double c = cos(th), s2 = sin(th);
    re[N] = 1.0; im[N] = 0.0;
    for (int k = 1; k <= N; ++k) {
        re[N + k] = re[N + k - 1] * c - im[N + k - 1] * s2;
        im[N + k] = re[N + k - 1] * s2 + im[N + k - 1] * c;
        re[N - k] = re[N + k]; im[N - k] = -im[N + k];
    }
}

static void ewald_term(const ewald_t* E, const double r[3], double* wre, double* wim, double* tmp) {
    /* tmp: 6 * (2N+1) doubles; (wre, wim)[k] = e^{2 pi i m_k . r} */
    const int N0 = E->n[0], N1 = E->n[1], N2 = E->n[2];
    double *xr = tmp, *xi = xr + 2 * N0 + 1, *yr = xi + 2 * N0 + 1, *yi = yr + 2 * N1 + 1, *zr = yi + 2 * N1 + 1,
           *zi = zr + 2 * N2 + 1;
    ewald_powers(r[0], E->L[0], N0, xr, xi);
    ewald_powers(r[1], E->L[1], N1, yr, yi);
    ewald_powers(r[2], E->L[2], N2, zr, zi);
    for (int k = 0; k < E->nk; ++k) {
        const int a = E->idx[3 * k] + N0, b = E->idx[3 * k + 1] + N1, c = E->idx[3 * k + 2] + N2;
        const double pr = xr[a] * yr[b] - xi[a] * yi[b], pi = xr[a] * yi[b] + xi[a] * yr[b];
        wre[k] = pr * zr[c] - pi * zi[c];
        wim[k] = pr * zi[c] + pi * zr[c];
    }
}

static int ewald_tmp_size(const ewald_t* E) { return 2 * (2 * E->n[0] + 1 + 2 * E->n[1] + 1 + 2 * E->n[2] + 1); }

/* S(m) of the fixed atoms and occupied slots */
static void ewald_structure(ewald_t* E, const or_info* info, const or_atomarray* frag, const or_residue* res,
                            const or_atom* atoms, int threads) {
    memset(E->sre, 0, sizeof(double) * E->nk);
    memset(E->sim, 0, sizeof(double) * E->nk);
    const int nfix = frag[0].startRes;
    /* atom list of the occupied groups */
    int na = 0;
    for (int t = -1; t < info->fragTypeNum; ++t) {
        const int g0 = t < 0 ? 0 : frag[t].startRes, g1 = t < 0 ? nfix : g0 + frag[t].totalNum;
        for (int g = g0; g < g1; ++g) na += res[g].atomNum;
    }
    int* list = malloc(sizeof(int) * (size_t)(na > 0 ? na : 1));
    na = 0;
    for (int t = -1; t < info->fragTypeNum; ++t) {
        const int g0 = t < 0 ? 0 : frag[t].startRes, g1 = t < 0 ? nfix : g0 + frag[t].totalNum;
        for (int g = g0; g < g1; ++g)
            for (int a = 0; a < res[g].atomNum; ++a) list[na++] = res[g].atomStart + a;
    }
#pragma omp parallel num_threads(threads)
    {
        double* wre = malloc(sizeof(double) * E->nk);
        double* wim = malloc(sizeof(double) * E->nk);
        double* tmp = malloc(sizeof(double) * ewald_tmp_size(E));
        double* are = calloc((size_t)E->nk, sizeof(double));
        double* aim = calloc((size_t)E->nk, sizeof(double));
#pragma omp for schedule(static)
        for (int j = 0; j < na; ++j) {
            const or_atom* A = &atoms[list[j]];
            const double r[3] = {A->position[0], A->position[1], A->position[2]};
            ewald_term(E, r, wre, wim, tmp);
            for (int k = 0; k < E->nk; ++k) {
                are[k] += A->charge * wre[k];
                aim[k] += A->charge * wim[k];
            }
        }
#pragma omp critical
        for (int k = 0; k < E->nk; ++k) {
            E->sre[k] += are[k];
            E->sim[k] += aim[k];
        }
        free(wre); free(wim); free(tmp); free(are); free(aim);
    }
    free(list);
}

/* phi(r) = sum_half coef (Re S cos th + Im S sin th), th = 2 pi m.r; work: 2*nk + tmp */
static double ewald_phi(const ewald_t* E, const double r[3], double* work) {
    double* wre = work;
    double* wim = work + E->nk;
    ewald_term(E, r, wre, wim, work + 2 * E->nk);
    double p = 0.0;
    for (int k = 0; k < E->nk; ++k) p += E->coef[k] * (E->sre[k] * wre[k] + E->sim[k] * wim[k]);
    return p;
}

/* grad phi(r): d/dr_d of sum coef (Re S cos th + Im S sin th) = sum coef (Im S cos th - Re S sin th) 2 pi m_d / L_d */
static void ewald_grad(const ewald_t* E, const double r[3], double* work, double g[3]) {
    double* wre = work;
    double* wim = work + E->nk;
    ewald_term(E, r, wre, wim, work + 2 * E->nk);
    g[0] = g[1] = g[2] = 0.0;
    for (int k = 0; k < E->nk; ++k) {
        const double c = E->coef[k] * (E->sim[k] * wre[k] - E->sre[k] * wim[k]);
        for (int d = 0; d < 3; ++d) g[d] += c * E->idx[3 * k + d];
    }
    for (int d = 0; d < 3; ++d) g[d] *= 2.0 * OR_PI / E->L[d];
}

void or_ewald_potential(const or_info* info, const or_atomarray* frag, const or_residue* res, const or_atom* atoms,
                        double alpha, const double* pts, int32_t n, double* out, int32_t threads) {
    if (threads <= 0) threads = 1;
    ewald_t E;
    if (ewald_init(&E, info, alpha) != 0) { ewald_free(&E); return; }
    ewald_structure(&E, info, frag, res, atoms, threads);
#pragma omp parallel num_threads(threads)
    {
        double* work = malloc(sizeof(double) * (2 * E.nk + ewald_tmp_size(&E)));
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n; ++i) out[i] = ewald_phi(&E, pts + 3 * i, work);
        free(work);
    }
    ewald_free(&E);
}

/* g(r) = erf(alpha r) / r, g(0) = 2 alpha / sqrt(pi) */
static inline double ewald_g(double r, double alpha) {
    return r < 1e-10 ? 2.0 * alpha / sqrt(OR_PI) : erf(alpha * r) / r;
}

/* Reciprocal-space and molecular terms of a pose energy (see the engine's
 * PME description): sum_s q_s phi(r_s), minus, when the pose replaces the
 * occupied group `self`, K sum_{s,t} q_s q_t g(|r_s - x_t|) over that group's
 * current atoms x_t (minimum image). */
static double ewald_pose_terms(const ewald_t* E, const or_info* info, const or_residue* res, const or_atom* atoms,
                               const float (*sx)[3], const float* sq, int ns, int self, double alpha, double* work) {
    double e = 0.0;
    for (int s2 = 0; s2 < ns; ++s2) {
        const double r[3] = {sx[s2][0], sx[s2][1], sx[s2][2]};
        e += (double)sq[s2] * ewald_phi(E, r, work);
    }
    if (self >= 0) {
        const or_residue* R = &res[self];
        double m = 0.0;
        for (int s2 = 0; s2 < ns; ++s2)
            for (int t = 0; t < R->atomNum; ++t) {
                const or_atom* A = &atoms[R->atomStart + t];
                double d2 = 0.0;
                for (int c = 0; c < 3; ++c) {
                    double d = (double)sx[s2][c] - (double)A->position[c];
                    d -= fast_round_d(d / info->cryst[c]) * info->cryst[c];
                    d2 += d * d;
                }
                m += (double)sq[s2] * (double)A->charge * ewald_g(sqrt(d2), alpha);
            }
        e -= OR_COULOMB * m;
    }
    return e;
}

/* Total charge of the fixed atoms and occupied slots. */
static double total_charge(const or_info* info, const or_atomarray* frag, const or_residue* res,
                           const or_atom* atoms) {
    double Q = 0.0;
    for (int t = -1; t < info->fragTypeNum; ++t) {
        const int g0 = t < 0 ? 0 : frag[t].startRes, g1 = t < 0 ? frag[0].startRes : g0 + frag[t].totalNum;
        for (int g = g0; g < g1; ++g)
            for (int a = 0; a < res[g].atomNum; ++a) Q += atoms[res[g].atomStart + a].charge;
    }
    return Q;
}

/* ------------------------------------------------------------------------- */
/* Moves and the step loop.                                                   */
/* ------------------------------------------------------------------------- */
typedef struct {
    const or_info* info;
    or_atomarray* frag;
    or_residue* res;
    or_atom* atoms;
    const float* grid;
    const float* ff;
    const or_options* opt;
    /* or_run_ext extensions (per call; the step pointers are advanced per step) */
    double* e_total;
    double* forces;
    double* fscale;
    const float* replay_forces;
    /* Ewald electrostatics (opt->pme): structure factors of the step's state */
    ewald_t* ew;
} sysref;

/* A trial pose's energy: real space (erfc kernel under Ewald) plus, under
 * Ewald, the reciprocal-space and molecular terms; *l1 = sum of |real-space
 * pair terms| plus sum |q_s phi(r_s)| and |molecular terms|. */
static double step_pose_energy(const sysref* S, const float (*sx)[3], const float* sq, const int32_t* st, int ns,
                               const float centre[3], int self, double* l1) {
    const or_info* info = S->info;
    if (!S->opt->pme)
        return or_pose_energy_l1(info, S->frag, S->res, S->atoms, S->ff, sx, sq, st, ns, centre, self, 0, NULL, NULL,
                                 l1);
    const double alpha = S->opt->pme_alpha;
    double lr = 0.0;
    double e = pose_energy64a(info, S->frag, S->res, S->atoms, S->ff, sx, sq, st, ns, centre, self, alpha, &lr);
    double* work = malloc(sizeof(double) * (2 * S->ew->nk + ewald_tmp_size(S->ew)));
    const double er = ewald_pose_terms(S->ew, info, S->res, S->atoms, sx, sq, ns, self, alpha, work);
    free(work);
    if (l1) *l1 = lr + fabs(er);
    return e + er;
}

/* Change of the neutralising-background energy -K pi Q^2 / (2 V alpha^2) when the
 * total charge goes from Q to Q + dq. */
static double background_change(const sysref* S, double Q, double dq) {
    const or_info* info = S->info;
    const double V = (double)info->cryst[0] * info->cryst[1] * info->cryst[2];
    const double a = S->opt->pme_alpha;
    return -OR_COULOMB * OR_PI * ((Q + dq) * (Q + dq) - Q * Q) / (2.0 * V * a * a);
}

/* FP64 force and torque (about the site centroid) on a pose of float sites:
 * f = (F, tau) with F = -sum_s dE/dx_s, tau = -sum_s (x_s - m) x dE/dx_s;
 * sc = (sum of |force terms|, sum of |x_s - m| |force terms of s|). */
static void pose_force64(const sysref* S, const double* ff64, const float (*sx)[3], const float* sq,
                         const int32_t* st, int ns, const float centre[3], int self, double f[6], double sc[2]) {
    double x64[20][3], q64[20], g[60], gq[20], gl1[20];
    for (int s = 0; s < ns; ++s) {
        for (int j = 0; j < 3; ++j) x64[s][j] = sx[s][j];
        q64[s] = sq[s];
    }
    pose64 P = {S->info, S->frag, S->res, S->atoms, ff64, (const double (*)[3])x64, q64, st, ns,
                S->opt->pme ? (double)S->opt->pme_alpha : 0.0};
    pose_grad64(&P, centre, self, 1.0, g, gq, NULL, gl1, NULL, NULL);
    if (S->opt->pme) { /* reciprocal-space and molecular terms (ewald_pose_terms) */
        const double alpha = S->opt->pme_alpha, c = 2.0 * alpha / sqrt(OR_PI);
        double* work = malloc(sizeof(double) * (2 * S->ew->nk + ewald_tmp_size(S->ew)));
        for (int s = 0; s < ns; ++s) {
            double gp[3];
            ewald_grad(S->ew, x64[s], work, gp);
            for (int j = 0; j < 3; ++j) {
                g[3 * s + j] += q64[s] * gp[j];
                gl1[s] += fabs(q64[s] * gp[j]);
            }
            if (self >= 0) {
                const or_residue* R = &S->res[self];
                for (int t = 0; t < R->atomNum; ++t) {
                    const or_atom* A = &S->atoms[R->atomStart + t];
                    double d[3], d2 = 0.0;
                    for (int j = 0; j < 3; ++j) {
                        d[j] = x64[s][j] - (double)A->position[j];
                        d[j] -= fast_round_d(d[j] / S->info->cryst[j]) * S->info->cryst[j];
                        d2 += d[j] * d[j];
                    }
                    const double r = sqrt(d2);
                    const double gpr = r < 1e-4 ? -(2.0 / 3.0) * c * alpha * alpha
                                                : (c * exp(-alpha * alpha * d2) * r - erf(alpha * r)) / (r * d2);
                    const double w = -OR_COULOMB * q64[s] * (double)A->charge * gpr;
                    for (int j = 0; j < 3; ++j) {
                        g[3 * s + j] += w * d[j];
                        gl1[s] += fabs(w * d[j]);
                    }
                }
            }
        }
        free(work);
    }
    double m[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < ns; ++s)
        for (int j = 0; j < 3; ++j) m[j] += x64[s][j] / ns;
    for (int c = 0; c < 6; ++c) f[c] = 0.0;
    sc[0] = sc[1] = 0.0;
    for (int s = 0; s < ns; ++s) {
        const double r[3] = {x64[s][0] - m[0], x64[s][1] - m[1], x64[s][2] - m[2]};
        const double* gs = g + 3 * s;
        f[0] -= gs[0]; f[1] -= gs[1]; f[2] -= gs[2];
        f[3] -= r[1] * gs[2] - r[2] * gs[1];
        f[4] -= r[2] * gs[0] - r[0] * gs[2];
        f[5] -= r[0] * gs[1] - r[1] * gs[0];
        sc[0] += gl1[s];
        sc[1] += sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) * gl1[s];
    }
}

/* Force-biased proposal steps (engine: fb_* in energy.cuh). */
static inline float fb_shift(const or_info* info, float d, int axis, float c) {
    const float invL = 1.0f / info->cryst[axis];
    const float k = floorf(((c + d) - info->startxyz[axis]) * invL);
    return d - k * info->cryst[axis];
}
static void fb_params(const or_options* opt, int trn, float* lb, float* h) {
    const float ht = opt->fb_trn > 0.0f ? opt->fb_trn : 0.5f;
    const float hr = opt->fb_rot > 0.0f ? opt->fb_rot : (float)(10.0 * 3.14159265358979323846 / 180.0);
    *h = trn ? ht : hr;
    *lb = (float)(0.5 * OR_BETA);
}
/* sum over components of g(a') - g(a) - (a' + a) d (engine: fb_ln_ratio) */
static double fb_ln_ratio(const float d[3], const float ao[3], const float* gn, float lb, float h) {
    double s2 = 0.0;
    for (int c = 0; c < 3; ++c) {
        const float an = lb * gn[c];
        const double t = ((double)fb_lnorm(an, h) - (double)fb_lnorm(ao[c], h)) - ((double)an + (double)ao[c]) * (double)d[c];
        s2 = s2 + t;
    }
    return s2;
}

static double beta_muex(const or_options* opt, const or_atomarray* F) {
    double mu = (double)F->muex;
    if (opt->muex_kcal) mu *= OR_KCAL_TO_KJ;
    return OR_BETA * mu;
}

static double ln_nbar(const or_info* info, const or_atomarray* F) {
    double V = (double)info->cryst[0] * (double)info->cryst[1] * (double)info->cryst[2];
    return log(V * (double)F->conc * OR_MOLES_TO_MOLECULES);
}

static void template_sites(const or_atomarray* F, float* q, int32_t* t) {
    for (int s = 0; s < F->num_atoms; ++s) { q[s] = F->atoms[s].charge; t[s] = F->atoms[s].type; }
}

static int32_t do_step(const sysref* S, const int32_t* moves, int step, or_step_log* L, double* Eout,
                       double* Escale, const double* Ereplay, int kmax, int threads) {
    const or_info* info = S->info;
    int mv = moves[step];
    int f = mv / 4, m = mv % 4;
    or_atomarray* F = &S->frag[f];
    const int ns = F->num_atoms;
    float sq[20];
    int32_t st[20];
    template_sites(F, sq, st);
    int n0 = F->totalNum;
    if (L) {
        memset(L, 0, sizeof(*L));
        L->step = step; L->move = m; L->ftype = f; L->n_before = n0;
        L->first_accept = -1; L->slot = -1;
    }
    int k = 0;
    if (m == 0) {
        if (F->totalNum == F->maxNum) goto done;
        k = F->confBias;
        if (Eout && k > kmax) return -3;
        float (*xyz)[20][3] = malloc(sizeof(float) * 60 * (size_t)k);
        float (*cen)[3] = malloc(sizeof(float) * 3 * (size_t)k);
        double* E = malloc(sizeof(double) * (size_t)k);
        double* l1 = malloc(sizeof(double) * (size_t)k);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 4)
        for (int i = 0; i < k; ++i) {
            or_insert_pose(info, S->frag, S->grid, S->opt, f, step, i, xyz[i], cen[i]);
            E[i] = step_pose_energy(S, (const float (*)[3])xyz[i], sq, st, ns, cen[i], -1, &l1[i]);
        }
        if (S->opt->pme) {  /* neutralising background: Q -> Q + q_fragment */
            double qf = 0.0;
            for (int s2 = 0; s2 < ns; ++s2) qf += sq[s2];
            const double bg = background_change(S, total_charge(info, S->frag, S->res, S->atoms), qf);
            for (int i = 0; i < k; ++i) E[i] += bg;
        }
        double esum = 0.0;
        for (int i = 0; i < k; ++i) {
            esum += E[i];
            if (Eout) Eout[i] = E[i];
            if (Escale) Escale[i] = l1[i];
        }
        free(l1);
        const double* Ed = Ereplay ? Ereplay : E;
        int n = F->totalNum;
        cluster_par P = {0, log((double)info->cavityFactor), beta_muex(S->opt, F) + ln_nbar(info, F), &n,
                         F->maxNum};
        int* acc = malloc(sizeof(int) * (size_t)k);
        int* ins = malloc(sizeof(int) * (size_t)k);
        int na = 0, fa = -1;
        int nc = cluster_pass(info, S->opt, step, k, Ed, (const float (*)[3])cen, &P, acc, ins, &na, &fa);
        for (int a = 0; a < na; ++a) {
            if (!ins[a]) continue;
            int i = acc[a];
            if (S->e_total) *S->e_total += Ed[i];
            int slot = F->totalNum++;
            or_residue* R = &S->res[F->startRes + slot];
            for (int j = 0; j < 3; ++j) R->position[j] = cen[i][j];
            for (int s = 0; s < ns; ++s) {
                or_atom* A = &S->atoms[R->atomStart + s];
                for (int j = 0; j < 3; ++j) A->position[j] = xyz[i][s][j];
                A->charge = F->atoms[s].charge;
                A->type = F->atoms[s].type;
            }
        }
        if (L) { L->n_clusters = nc; L->n_accept = na; L->first_accept = fa; L->e_sum = esum; }
        free(acc); free(ins); free(xyz); free(cen); free(E);
    } else if (m == 1) {
        if (F->totalNum == 0) goto done; /* the reference divides by zero here */
        k = 1;
        uint32_t r[4];
        rng(info->seed, S->opt->replica, (uint32_t)step, 0u, RP_DELETE, 0, r);
        int slot = (int)(r[0] % (uint32_t)F->totalNum);
        or_residue* R = &S->res[F->startRes + slot];
        float xyz[20][3];
        for (int s = 0; s < ns; ++s)
            for (int j = 0; j < 3; ++j) xyz[s][j] = S->atoms[R->atomStart + s].position[j];
        double l1 = 0.0;
        double E = step_pose_energy(S, (const float (*)[3])xyz, sq, st, ns, R->position, F->startRes + slot, &l1);
        if (S->opt->pme) {  /* the removal changes Q by -q_fragment; E is minus the system's change */
            double qf = 0.0;
            for (int s2 = 0; s2 < ns; ++s2) qf += sq[s2];
            E -= background_change(S, total_charge(info, S->frag, S->res, S->atoms), -qf);
        }
        if (Eout) Eout[0] = E;
        if (Escale) Escale[0] = l1;
        double Ed = Ereplay ? Ereplay[0] : E;
        int n = F->totalNum;
        double lnp = log((double)n) - (beta_muex(S->opt, F) + ln_nbar(info, F)) + OR_BETA * Ed;
        double u = u53(r[1], r[2]);
        int acc = !isnan(lnp) && (lnp >= 0.0 || u < exp(lnp));
        if (isfinite(Ed)) note_decision(lnp, u, trial_tol(Ed));
        if (acc) {
            int last = n - 1;
            or_residue* RL = &S->res[F->startRes + last];
            for (int j = 0; j < 3; ++j) R->position[j] = RL->position[j];
            for (int s = 0; s < R->atomNum; ++s)
                for (int j = 0; j < 3; ++j)
                    S->atoms[R->atomStart + s].position[j] = S->atoms[RL->atomStart + s].position[j];
            F->totalNum -= 1;
            if (S->e_total) *S->e_total -= Ed;
        }
        if (L) {
            L->n_clusters = 1; L->n_accept = acc; L->first_accept = acc ? 0 : -1;
            L->slot = slot; L->e_sum = E;
        }
    } else if (S->opt->proposal == 2) {
        /* force-biased translate/rotate with the Metropolis-Hastings correction */
        int n = F->totalNum;
        k = F->confBias < n ? F->confBias : n;
        if (k == 0) goto done;
        if (Eout && k > kmax) return -3;
        const int trn = (m == 2);
        float lb, hh;
        fb_params(S->opt, trn, &lb, &hh);
        const size_t nff = (size_t)2 * info->ffXNum * info->ffYNum;
        double* ff64 = malloc(sizeof(double) * nff);
        for (size_t j = 0; j < nff; ++j) ff64[j] = S->ff[j];
        float (*xyz)[20][3] = malloc(sizeof(float) * 60 * (size_t)k);
        float (*cen)[3] = malloc(sizeof(float) * 3 * (size_t)k);
        float (*pd)[3] = malloc(sizeof(float) * 3 * (size_t)k);
        float (*pa)[3] = malloc(sizeof(float) * 3 * (size_t)k);
        float (*fnu)[6] = malloc(sizeof(float) * 6 * (size_t)k);
        int* okv = malloc(sizeof(int) * (size_t)k);
        int* slots = malloc(sizeof(int) * (size_t)k);
        double* dE = malloc(sizeof(double) * (size_t)k);
        double* sc = malloc(sizeof(double) * (size_t)k);
        double* Eeff = malloc(sizeof(double) * (size_t)k);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 2)
        for (int i = 0; i < k; ++i) {
            int slot = or_perm_slot(S->opt, info->seed, step, i, n);
            slots[i] = slot;
            const int self = F->startRes + slot;
            const or_residue* R = &S->res[self];
            float old[20][3];
            for (int s2 = 0; s2 < ns; ++s2)
                for (int j = 0; j < 3; ++j) old[s2][j] = S->atoms[R->atomStart + s2].position[j];
            double lo = 0.0, ln = 0.0, fo64[6], fn64[6], so[2], sn2[2];
            double Eo = step_pose_energy(S, (const float (*)[3])old, sq, st, ns, R->position, self, &lo);
            pose_force64(S, ff64, (const float (*)[3])old, sq, st, ns, R->position, self, fo64, so);
            float fo[6];
            for (int c = 0; c < 6; ++c)
                fo[c] = S->replay_forces ? S->replay_forces[(size_t)i * 12 + c] : (float)fo64[c];
            uint32_t ru[4];
            rng(info->seed, S->opt->replica, (uint32_t)step, (uint32_t)i, RP_FB, 0, ru);
            const float* g = trn ? fo : fo + 3;
            const int ok = isfinite(g[0]) && isfinite(g[1]) && isfinite(g[2]);
            okv[i] = ok;
            for (int a = 0; a < 3; ++a) {
                pa[i][a] = ok ? lb * g[a] : 0.0f;
                pd[i][a] = fb_tilted(pa[i][a], hh, u01_co(ru[a]));
            }
            if (trn) {
                for (int j = 0; j < 3; ++j) {
                    const float sh = fb_shift(info, pd[i][j], j, R->position[j]);
                    cen[i][j] = R->position[j] + sh;
                    for (int s2 = 0; s2 < ns; ++s2) xyz[i][s2][j] = old[s2][j] + sh;
                }
            } else {
                for (int s2 = 0; s2 < ns; ++s2)
                    for (int j = 0; j < 3; ++j) xyz[i][s2][j] = old[s2][j];
                for (int j = 0; j < 3; ++j) cen[i][j] = R->position[j];
                const float* d = pd[i];
                float nn = d[0] * d[0];
                nn = fmaf(d[1], d[1], nn);
                nn = fmaf(d[2], d[2], nn);
                if (nn > 0.0f) {
                    float ang = sqrtf(nn);
                    ang = ang - floorf(ang * 0.159154943f) * OR_TWO_PI_F;
                    float sn, cs, Rm[3][3];
                    or_det_sincos(ang, &sn, &cs);
                    rodrigues(d, sn, cs, Rm);
                    float mc[3] = {0.0f, 0.0f, 0.0f};
                    for (int j = 0; j < 3; ++j)
                        for (int s2 = 0; s2 < ns; ++s2) mc[j] = mc[j] + xyz[i][s2][j] / (float)ns;
                    for (int s2 = 0; s2 < ns; ++s2) {
                        float q[3] = {xyz[i][s2][0] - mc[0], xyz[i][s2][1] - mc[1], xyz[i][s2][2] - mc[2]};
                        float pr[3];
                        rotate(Rm, q, pr);
                        for (int j = 0; j < 3; ++j) xyz[i][s2][j] = pr[j] + mc[j];
                    }
                }
            }
            double En = step_pose_energy(S, (const float (*)[3])xyz[i], sq, st, ns, cen[i], self, &ln);
            pose_force64(S, ff64, (const float (*)[3])xyz[i], sq, st, ns, cen[i], self, fn64, sn2);
            for (int c = 0; c < 6; ++c)
                fnu[i][c] = S->replay_forces ? S->replay_forces[(size_t)i * 12 + 6 + c] : (float)fn64[c];
            if (S->forces)
                for (int c = 0; c < 6; ++c) {
                    S->forces[(size_t)i * 12 + c] = fo64[c];
                    S->forces[(size_t)i * 12 + 6 + c] = fn64[c];
                }
            if (S->fscale) {
                S->fscale[(size_t)i * 4] = so[0]; S->fscale[(size_t)i * 4 + 1] = so[1];
                S->fscale[(size_t)i * 4 + 2] = sn2[0]; S->fscale[(size_t)i * 4 + 3] = sn2[1];
            }
            dE[i] = En - Eo;
            sc[i] = ln + lo;
        }
        double esum = 0.0;
        for (int i = 0; i < k; ++i) {
            esum += dE[i];
            if (Eout) Eout[i] = dE[i];
            if (Escale) Escale[i] = sc[i];
        }
        const double* Ed = Ereplay ? Ereplay : dE;
        for (int i = 0; i < k; ++i) {
            const float* gn = trn ? fnu[i] : fnu[i] + 3;
            Eeff[i] = (!okv[i] || !isfinite(Ed[i])) ? INFINITY
                                                    : Ed[i] - fb_ln_ratio(pd[i], pa[i], gn, lb, hh) / OR_BETA;
        }
        cluster_par P = {1, 0.0, 0.0, NULL, 0};
        int* acc = malloc(sizeof(int) * (size_t)k);
        int* ins = malloc(sizeof(int) * (size_t)k);
        int na = 0, fa = -1;
        int nc = cluster_pass(info, S->opt, step, k, Eeff, (const float (*)[3])cen, &P, acc, ins, &na, &fa);
        for (int a = 0; a < na; ++a) {
            int i = acc[a];
            or_residue* R = &S->res[F->startRes + slots[i]];
            for (int j = 0; j < 3; ++j) R->position[j] = cen[i][j];
            for (int s2 = 0; s2 < ns; ++s2)
                for (int j = 0; j < 3; ++j) S->atoms[R->atomStart + s2].position[j] = xyz[i][s2][j];
            if (S->e_total) *S->e_total += Ed[i];
        }
        if (L) { L->n_clusters = nc; L->n_accept = na; L->first_accept = fa; L->e_sum = esum; }
        free(acc); free(ins); free(xyz); free(cen); free(pd); free(pa); free(fnu); free(okv); free(slots);
        free(dE); free(sc); free(Eeff); free(ff64);
    } else {
        int n = F->totalNum;
        k = F->confBias < n ? F->confBias : n;
        if (k == 0) goto done;
        if (Eout && k > kmax) return -3;
        float (*xyz)[20][3] = malloc(sizeof(float) * 60 * (size_t)k);
        float (*cen)[3] = malloc(sizeof(float) * 3 * (size_t)k);
        int* slots = malloc(sizeof(int) * (size_t)k);
        double* dE = malloc(sizeof(double) * (size_t)k);
        double* sc = malloc(sizeof(double) * (size_t)k);
#pragma omp parallel for num_threads(threads) schedule(dynamic, 2)
        for (int i = 0; i < k; ++i) {
            int slot = or_perm_slot(S->opt, info->seed, step, i, n);
            slots[i] = slot;
            const or_residue* R = &S->res[F->startRes + slot];
            float old[20][3];
            for (int s = 0; s < ns; ++s)
                for (int j = 0; j < 3; ++j) old[s][j] = S->atoms[R->atomStart + s].position[j];
            double lo = 0.0, ln = 0.0;
            double Eo = step_pose_energy(S, (const float (*)[3])old, sq, st, ns, R->position, F->startRes + slot,
                                         &lo);
            or_move_pose(info, S->frag, S->res, S->atoms, S->opt, f, m, step, i, slot, xyz[i], cen[i]);
            double En = step_pose_energy(S, (const float (*)[3])xyz[i], sq, st, ns, cen[i], F->startRes + slot,
                                         &ln);
            dE[i] = En - Eo;
            sc[i] = ln + lo;
        }
        double esum = 0.0;
        for (int i = 0; i < k; ++i) {
            esum += dE[i];
            if (Eout) Eout[i] = dE[i];
            if (Escale) Escale[i] = sc[i];
        }
        const double* Ed = Ereplay ? Ereplay : dE;
        cluster_par P = {1, 0.0, 0.0, NULL, 0};
        int* acc = malloc(sizeof(int) * (size_t)k);
        int* ins = malloc(sizeof(int) * (size_t)k);
        int na = 0, fa = -1;
        int nc = cluster_pass(info, S->opt, step, k, Ed, (const float (*)[3])cen, &P, acc, ins, &na, &fa);
        for (int a = 0; a < na; ++a) {
            int i = acc[a];
            or_residue* R = &S->res[F->startRes + slots[i]];
            for (int j = 0; j < 3; ++j) R->position[j] = cen[i][j];
            for (int s = 0; s < ns; ++s)
                for (int j = 0; j < 3; ++j) S->atoms[R->atomStart + s].position[j] = xyz[i][s][j];
            if (S->e_total) *S->e_total += Ed[i];
        }
        if (L) { L->n_clusters = nc; L->n_accept = na; L->first_accept = fa; L->e_sum = esum; }
        free(acc); free(ins); free(xyz); free(cen); free(slots); free(dE); free(sc);
    }
done:
    if (L) { L->k = k; L->n_after = F->totalNum; L->e_total = S->e_total ? *S->e_total : 0.0; }
    return 0;
}

int32_t or_run(const or_info* info, or_atomarray* frag, or_residue* res, or_atom* atoms,
               const float* grid, const float* ff, const int32_t* moves, const or_options* opt,
               int32_t step0, int32_t nsteps, or_step_log* log, double* energies, double* escale,
               const double* replay, int32_t kmax, int32_t threads) {
    return or_run_ext(info, frag, res, atoms, grid, ff, moves, opt, step0, nsteps, log, energies, escale, replay,
                      kmax, threads, NULL, NULL, NULL, NULL);
}

int32_t or_run_ext(const or_info* info, or_atomarray* frag, or_residue* res, or_atom* atoms,
                   const float* grid, const float* ff, const int32_t* moves, const or_options* opt,
                   int32_t step0, int32_t nsteps, or_step_log* log, double* energies, double* escale,
                   const double* replay, int32_t kmax, int32_t threads, double* e_total,
                   double* forces, double* fscale, const float* replay_forces) {
    if (threads <= 0) threads = 1;
    ewald_t ew;
    memset(&ew, 0, sizeof(ew));
    if (opt->pme && ewald_init(&ew, info, opt->pme_alpha) != 0) {
        ewald_free(&ew);
        return -5;
    }
    int rc = 0;
    for (int s = 0; s < nsteps && rc == 0; ++s) {
        int step = step0 + s;
        if (opt->pme) ewald_structure(&ew, info, frag, res, atoms, threads);
        sysref S = {info, frag, res, atoms, grid, ff, opt, e_total,
                    forces ? forces + (size_t)s * kmax * 12 : NULL, fscale ? fscale + (size_t)s * kmax * 4 : NULL,
                    replay_forces ? replay_forces + (size_t)s * kmax * 12 : NULL, opt->pme ? &ew : NULL};
        rc = do_step(&S, moves, step, log ? &log[s] : NULL, energies ? energies + (size_t)s * kmax : NULL,
                     escale ? escale + (size_t)s * kmax : NULL, replay ? replay + (size_t)s * kmax : NULL,
                     kmax, threads);
    }
    ewald_free(&ew);
    return rc;
}

int64_t or_energy_batch(const or_info* info, const or_atomarray* frag, const or_residue* res,
                        const or_atom* atoms, const float* ff, const float* poses_xyz,
                        const float* site_q, const int32_t* site_type, int32_t nsites,
                        const float* centres, const int32_t* self, int32_t nposes, int32_t mode,
                        double* out, int32_t* n_groups, double* l1, int32_t threads) {
    if (threads <= 0) threads = 1;
    int64_t total = 0;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 4) reduction(+ : total)
    for (int p = 0; p < nposes; ++p) {
        int32_t ng = 0;
        int64_t np = 0;
        double m1 = 0.0;
        out[p] = or_pose_energy_l1(info, frag, res, atoms, ff,
                                   (const float (*)[3])(poses_xyz + (size_t)p * nsites * 3), site_q,
                                   site_type, nsites, centres + 3 * p, self ? self[p] : -1, mode, &ng, &np,
                                   &m1);
        if (l1) l1[p] = m1;
        if (n_groups) n_groups[p] = ng;
        total += np;
    }
    return total;
}

int64_t or_energy_batch64(const or_info* info, const or_atomarray* frag, const or_residue* res,
                          const or_atom* atoms, const double* ff64, const double* xyz64, const double* q64,
                          const int32_t* site_type, int32_t nsites, const float* centres, const int32_t* self,
                          int32_t nposes, double* out, int32_t* n_groups, int32_t threads) {
    if (threads <= 0) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 4)
    for (int p = 0; p < nposes; ++p) {
        pose64 P = {info, frag, res, atoms, ff64, (const double (*)[3])(xyz64 + (size_t)p * nsites * 3), q64,
                    site_type, nsites};
        int32_t ng = 0;
        out[p] = pose_energy64(&P, centres + 3 * p, self ? self[p] : -1, &ng);
        if (n_groups) n_groups[p] = ng;
    }
    return 0;
}

int64_t or_grad_batch(const or_info* info, const or_atomarray* frag, const or_residue* res, const or_atom* atoms,
                      const double* ff64, const double* xyz64, const double* q64, const int32_t* site_type,
                      int32_t nsites, const float* centres, const int32_t* self, int32_t nposes,
                      const double* gout, double* gxyz, double* gq, double* gff, double* gxyz_l1, double* gq_l1,
                      double* gff_l1, int32_t threads) {
    if (threads <= 0) threads = 1;
    const size_t nff = (size_t)2 * info->ffXNum * info->ffYNum;
    double* tff = NULL;
    double* tff1 = NULL;
    if (gff) {
        tff = calloc(nff * (size_t)threads, sizeof(double));
        tff1 = calloc(nff * (size_t)threads, sizeof(double));
        if (!tff || !tff1) {
            free(tff);
            free(tff1);
            return -1;
        }
    }
#pragma omp parallel num_threads(threads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 4)
        for (int p = 0; p < nposes; ++p) {
            pose64 P = {info, frag, res, atoms, ff64, (const double (*)[3])(xyz64 + (size_t)p * nsites * 3), q64,
                        site_type, nsites};
            pose_grad64(&P, centres + 3 * p, self ? self[p] : -1, gout ? gout[p] : 1.0,
                        gxyz + (size_t)p * nsites * 3, gq + (size_t)p * nsites, tff ? tff + nff * tid : NULL,
                        gxyz_l1 ? gxyz_l1 + (size_t)p * nsites : NULL, gq_l1 ? gq_l1 + (size_t)p * nsites : NULL,
                        tff1 ? tff1 + nff * tid : NULL);
        }
    }
    if (gff) {
        for (size_t j = 0; j < nff; ++j) {
            double a = 0.0, b = 0.0;
            for (int t = 0; t < threads; ++t) {
                a += tff[nff * t + j];
                b += tff1[nff * t + j];
            }
            gff[j] = a;
            if (gff_l1) gff_l1[j] = b;
        }
    }
    free(tff);
    free(tff1);
    return 0;
}

/* Rotation of one point by the Rodrigues matrix of (axis, angle) -- exposes the
 * pose rotation for the known-answer test of the reference notebook. */
void or_rotate_point(const float axis[3], float angle, const float p[3], float out[3], float R_out[9]) {
    float sn, cs, R[3][3];
    or_det_sincos(angle, &sn, &cs);
    rodrigues(axis, sn, cs, R);
    rotate(R, p, out);
    if (R_out)
        for (int i = 0; i < 9; ++i) R_out[i] = R[i / 3][i % 3];
}
