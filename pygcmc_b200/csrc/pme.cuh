// Ewald electrostatics by smooth particle-mesh Ewald (Essmann et al., J. Chem.
// Phys. 103 (1995) 8577), FP64 mesh; not in the reference, whose calcEnergy
// uses a plain cutoff.
//
// Each replica keeps its spread charges Q on the mesh: the fixed atoms and the
// occupied fragment atoms spread with order-4 cardinal B-splines once at
// set-up; afterwards the accept kernel spreads the change of every accepted
// move (-q at a molecule's old sites, +q at its new ones) and marks the mesh
// dirty.  Before a step's pose energies, a dirty mesh's potential is
// recomputed, phi_mesh = IFFT(G * FFT(Q)) with G(m) = K exp(-pi^2 m^2 /
// alpha^2) B(m) / (pi V m^2), B the B-spline moduli, by the hand-written FP64
// transforms of fft.cuh (five passes: rows real-to-complex, axis 1, axis 0
// with the G product between its forward and inverse transforms, axis 1,
// rows complex-to-real); after a step that accepted nothing every pass
// returns at once.  The potential at a point is the same B-spline
// interpolation of phi_mesh.
//
// Energy of a trial pose p (sites r_s, charges q_s) under Ewald:
//   E(p) = sum_{pairs in the group cutoff} [LJ + K q_s q_a erfc(alpha r) / r]
//        + sum_s q_s phi(r_s)
//        - [p replaces occupied group M]  K sum_{s, t in M} q_s q_t g(|r_s - x_t|)
//        (+ the neutralising-background change for insert / delete, added by
//         the accept kernel), g(r) = erf(alpha r) / r, g(0) = 2 alpha / sqrt(pi).
// The molecule's self and intramolecular terms cancel exactly for an insertion
// (its own Coulomb pairs are excluded); the g term removes a moving or
// leaving molecule's own field from phi.  Neglected: the molecule's
// interaction with its own periodic images beyond erf(alpha r)/r (a smooth
// term of order q^2 / L^3 for these box sizes).
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace gcmc {

// order-4 B-spline weights of the four mesh points floor(u) - j, j = 0..3
__device__ __forceinline__ void bspline4(double w, double m[4]) {
    const double w2 = w * w, w3 = w2 * w, c = 1.0 - w;
    m[0] = w3 / 6.0;
    m[1] = (-3.0 * w3 + 3.0 * w2 + 3.0 * w + 1.0) / 6.0;
    m[2] = (3.0 * w3 - 6.0 * w2 + 4.0) / 6.0;
    m[3] = c * c * c / 6.0;
}

__device__ __forceinline__ int wrapm(int k, int n) {
    k %= n;
    return k < 0 ? k + n : k;
}

// mesh coordinate of x along axis a
__device__ __forceinline__ double mesh_u(const RepDev& R, double x, int a) {
    return ((x - (double)R.start[a]) / (double)R.L[a]) * (double)R.pme_n[a];
}

// spread charge q at (x, y, z) onto Q (atomic FP64 adds)
__device__ __forceinline__ void pme_spread_one(const RepDev& R, double* Q, double x, double y, double z, double q) {
    double mx[4], my[4], mz[4];
    const double ux = mesh_u(R, x, 0), uy = mesh_u(R, y, 1), uz = mesh_u(R, z, 2);
    const double fx = floor(ux), fy = floor(uy), fz = floor(uz);
    bspline4(ux - fx, mx);
    bspline4(uy - fy, my);
    bspline4(uz - fz, mz);
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], n2 = R.pme_n[2];
    for (int a = 0; a < 4; ++a) {
        const int i0 = wrapm((int)fx - a, n0);
        for (int b = 0; b < 4; ++b) {
            const int i1 = wrapm((int)fy - b, n1);
            const double wab = q * mx[a] * my[b];
            double* row = Q + ((size_t)i0 * n1 + i1) * n2;
            for (int c = 0; c < 4; ++c) atomicAdd(row + wrapm((int)fz - c, n2), wab * mz[c]);
        }
    }
}

// derivatives of bspline4's weights with respect to w
__device__ __forceinline__ void bspline4_d(double w, double d[4]) {
    const double c = 1.0 - w;
    d[0] = 0.5 * w * w;
    d[1] = 0.5 * (-3.0 * w * w + 2.0 * w + 1.0);
    d[2] = 0.5 * (3.0 * w * w - 4.0 * w);
    d[3] = -0.5 * c * c;
}

// phi at a point by the same interpolation
__device__ __forceinline__ double pme_phi_at(const RepDev& R, double x, double y, double z) {
    double mx[4], my[4], mz[4];
    const double ux = mesh_u(R, x, 0), uy = mesh_u(R, y, 1), uz = mesh_u(R, z, 2);
    const double fx = floor(ux), fy = floor(uy), fz = floor(uz);
    bspline4(ux - fx, mx);
    bspline4(uy - fy, my);
    bspline4(uz - fz, mz);
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], n2 = R.pme_n[2];
    double p = 0.0;
    for (int a = 0; a < 4; ++a) {
        const int i0 = wrapm((int)fx - a, n0);
        for (int b = 0; b < 4; ++b) {
            const int i1 = wrapm((int)fy - b, n1);
            const double* row = R.pme_phi + ((size_t)i0 * n1 + i1) * n2;
            double t = 0.0;
            for (int c = 0; c < 4; ++c) t += mz[c] * __ldg(row + wrapm((int)fz - c, n2));
            p += mx[a] * my[b] * t;
        }
    }
    return p;
}

// Atoms [a0, a1) of the replica spread onto Q (the fixed atoms, once).
__global__ void k_pme_spread_range(const RepDev* __restrict__ rep, double* Q, int a0, int a1) {
    const RepDev& R = *rep;
    for (int a = a0 + blockIdx.x * blockDim.x + threadIdx.x; a < a1; a += gridDim.x * blockDim.x) {
        const float4 p = R.xyzq[a];
        if (p.w != 0.0f) pme_spread_one(R, Q, p.x, p.y, p.z, p.w);
    }
}

// The occupied fragment atoms of every type spread onto Q.
__global__ void k_pme_spread_frag(const RepDev* __restrict__ rep, double* Q) {
    const RepDev& R = *rep;
    for (int t = 0; t < R.ntypes; ++t) {
        const FragDev& F = R.frag[t];
        const int n = R.totalNum[t] * F.nsites;
        const int a0 = R.gspan[F.startRes].x;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const float4 p = R.xyzq[a0 + i];
            if (p.w != 0.0f) pme_spread_one(R, Q, p.x, p.y, p.z, p.w);
        }
    }
}

// ---- the mesh transforms (dynamic shared memory: 2 * kFftLines * n * 16 B,
// n the pass's line length) ----

__device__ __forceinline__ bool pme_clean(const RepDev& R) {
    return *reinterpret_cast<const volatile int*>(R.pme_dirty) == 0;
}

// Rows along axis 2: Q (real, n2 per row) -> spectrum rows (n2 / 2 + 1).
__global__ void __launch_bounds__(kFftThreads) k_pme_rows_r2c(const RepDev* __restrict__ rep) {
    const RepDev& R = *rep;
    if (pme_clean(R)) return;
    extern __shared__ __align__(16) double2 fbuf[];
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], n2 = R.pme_n[2], M = n2 / 2 + 1;
    const int rows = n0 * n1;
    double2 *b0 = fbuf, *b1 = fbuf + kFftLines * n2;
    for (int r0 = blockIdx.x * kFftLines; r0 < rows; r0 += gridDim.x * kFftLines) {
        const int nl = min(kFftLines, rows - r0);
        __syncthreads();
        for (int e = threadIdx.x; e < nl * n2; e += blockDim.x)
            b0[e] = make_double2(R.pme_q[(size_t)r0 * n2 + e], 0.0);
        const double2* out = fft_lines_block(b0, b1, n2, nl, n2, -1);
        for (int e = threadIdx.x; e < nl * M; e += blockDim.x) {
            const int b = e / M, k = e - b * M;
            R.pme_spec[(size_t)(r0 + b) * M + k] = out[b * n2 + k];
        }
    }
}

// Lines along axis `axis` (0 or 1) of the half spectrum, kFftLines consecutive
// k2 per CTA: sign -1 forward, +1 inverse; fuse_g: forward, times G, inverse.
__global__ void __launch_bounds__(kFftThreads) k_pme_axis(const RepDev* __restrict__ rep, int axis, int sign,
                                                          int fuse_g) {
    const RepDev& R = *rep;
    if (pme_clean(R)) return;
    extern __shared__ __align__(16) double2 fbuf[];
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], M = R.pme_n[2] / 2 + 1;
    const int n = axis == 0 ? n0 : n1, other = axis == 0 ? n1 : n0;
    const size_t stride = axis == 0 ? (size_t)n1 * M : (size_t)M;
    const int kb = (M + kFftLines - 1) / kFftLines;
    double2 *b0 = fbuf, *b1 = fbuf + kFftLines * n;
    for (int w = blockIdx.x; w < other * kb; w += gridDim.x) {
        const int o = w / kb, k0 = (w - o * kb) * kFftLines;
        const int nl = min(kFftLines, M - k0);
        const size_t base = (axis == 0 ? (size_t)o * M : (size_t)o * n1 * M) + k0;
        __syncthreads();
        for (int e = threadIdx.x; e < n * kFftLines; e += blockDim.x) {  // consecutive threads: consecutive k2
            const int i = e / kFftLines, b = e - i * kFftLines;
            if (b < nl) b0[b * n + i] = R.pme_spec[base + (size_t)i * stride + b];
        }
        double2* out = fft_lines_block(b0, b1, n, nl, n, fuse_g ? -1 : sign);
        if (fuse_g) {
            for (int e = threadIdx.x; e < n * kFftLines; e += blockDim.x) {
                const int i = e / kFftLines, b = e - i * kFftLines;
                if (b < nl) {
                    const double g = R.pme_g[base + (size_t)i * stride + b];
                    double2& v = out[b * n + i];
                    v.x *= g;
                    v.y *= g;
                }
            }
            double2* other_buf = out == b0 ? b1 : b0;
            out = fft_lines_block(out, other_buf, n, nl, n, 1);
        }
        for (int e = threadIdx.x; e < n * kFftLines; e += blockDim.x) {
            const int i = e / kFftLines, b = e - i * kFftLines;
            if (b < nl) R.pme_spec[base + (size_t)i * stride + b] = out[b * n + i];
        }
    }
}

// Rows along axis 2: half spectrum -> phi (real): the row's full Hermitian
// extension, inverse transform, real part.
__global__ void __launch_bounds__(kFftThreads) k_pme_rows_c2r(const RepDev* __restrict__ rep) {
    const RepDev& R = *rep;
    if (pme_clean(R)) return;
    extern __shared__ __align__(16) double2 fbuf[];
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], n2 = R.pme_n[2], M = n2 / 2 + 1;
    const int rows = n0 * n1;
    double2 *b0 = fbuf, *b1 = fbuf + kFftLines * n2;
    double* phi = const_cast<double*>(R.pme_phi);
    for (int r0 = blockIdx.x * kFftLines; r0 < rows; r0 += gridDim.x * kFftLines) {
        const int nl = min(kFftLines, rows - r0);
        __syncthreads();
        for (int e = threadIdx.x; e < nl * n2; e += blockDim.x) {
            const int b = e / n2, k = e - b * n2;
            const double2* row = R.pme_spec + (size_t)(r0 + b) * M;
            double2 v;
            if (k < M) {
                v = row[k];
            } else {
                v = row[n2 - k];
                v.y = -v.y;
            }
            b0[e] = v;
        }
        const double2* out = fft_lines_block(b0, b1, n2, nl, n2, 1);
        for (int e = threadIdx.x; e < nl * n2; e += blockDim.x) phi[(size_t)r0 * n2 + e] = out[e].x;
    }
}

// The mesh potential is current again.
__global__ void k_pme_done(const RepDev* __restrict__ rep) {
    if (threadIdx.x == 0) *rep->pme_dirty = 0;
}

// Spread the change of an accepted move's site: charge q leaves (x0, y0, z0)
// and arrives at (x1, y1, z1) (either side skipped when its flag is false).
__device__ __forceinline__ void pme_move_site(const RepDev& R, bool from, float x0, float y0, float z0, bool to,
                                              float x1, float y1, float z1, float q) {
    if (q == 0.0f) return;
    if (from) pme_spread_one(R, R.pme_q, x0, y0, z0, -(double)q);
    if (to) pme_spread_one(R, R.pme_q, x1, y1, z1, (double)q);
}

// phi at caller points (diagnostics)
__global__ void k_pme_phi_points(const RepDev* __restrict__ rep, const double* __restrict__ pts, int n,
                                 double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = pme_phi_at(*rep, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}

__device__ __forceinline__ float ewald_g(float r, float alpha) {
    return r < 1e-6f ? 2.0f * alpha * 0.564189584f : erff(alpha * r) / r;
}

// Reciprocal-space and molecular terms of a pose for lane `lane` (< ns; 0
// otherwise): q_s phi(r_s) - K q_s sum_t q_t g(|r_s - x_t|) (the latter when
// the pose replaces group `self`).  Sites at absolute positions (sx, sy, sz).
__device__ __forceinline__ double pme_pose_lane(const RepDev& R, int ns, int lane, float sx, float sy, float sz,
                                                float q, int self) {
    if (lane >= ns) return 0.0;
    double e = (double)q * pme_phi_at(R, sx, sy, sz);
    if (self >= 0) {
        const int2 sp = R.gspan[self];
        float m = 0.0f;
        for (int t = 0; t < sp.y; ++t) {
            const float4 a = R.xyzq[sp.x + t];
            float dx = sx - a.x, dy = sy - a.y, dz = sz - a.z;
            dx -= rintf(dx * R.invL[0]) * R.L[0];
            dy -= rintf(dy * R.invL[1]) * R.L[1];
            dz -= rintf(dz * R.invL[2]) * R.L[2];
            m += a.w * ewald_g(sqrtf(dx * dx + dy * dy + dz * dz), R.pme_alpha);
        }
        e -= (double)kCoulomb * (double)q * (double)m;
    }
    return e;
}

// Gradient of pme_pose_lane's terms with respect to lane `lane`'s site
// position (< ns; zero otherwise): q grad phi(r_s) from the derivative of the
// B-spline interpolation (d/dx = (n / L) d/du), minus K q sum_t q_t g'(d) d/|d|
// over the replaced group's atoms (d = r_s - x_t, minimum image).
__device__ __forceinline__ void pme_grad_lane(const RepDev& R, int ns, int lane, float sx, float sy, float sz,
                                              float q, int self, float& gx, float& gy, float& gz) {
    gx = gy = gz = 0.0f;
    if (lane >= ns || q == 0.0f) return;
    double mx[4], my[4], mz[4], dx[4], dy[4], dz[4];
    const double ux = mesh_u(R, sx, 0), uy = mesh_u(R, sy, 1), uz = mesh_u(R, sz, 2);
    const double fx = floor(ux), fy = floor(uy), fz = floor(uz);
    bspline4(ux - fx, mx);
    bspline4(uy - fy, my);
    bspline4(uz - fz, mz);
    bspline4_d(ux - fx, dx);
    bspline4_d(uy - fy, dy);
    bspline4_d(uz - fz, dz);
    const int n0 = R.pme_n[0], n1 = R.pme_n[1], n2 = R.pme_n[2];
    double px = 0.0, py = 0.0, pz = 0.0;
    for (int a = 0; a < 4; ++a) {
        const int i0 = wrapm((int)fx - a, n0);
        for (int b = 0; b < 4; ++b) {
            const int i1 = wrapm((int)fy - b, n1);
            const double* row = R.pme_phi + ((size_t)i0 * n1 + i1) * n2;
            double t = 0.0, tz = 0.0;
            for (int c = 0; c < 4; ++c) {
                const double v = row[wrapm((int)fz - c, n2)];
                t += mz[c] * v;
                tz += dz[c] * v;
            }
            px += dx[a] * my[b] * t;
            py += mx[a] * dy[b] * t;
            pz += mx[a] * my[b] * tz;
        }
    }
    double g0 = (double)q * px * n0 / (double)R.L[0];
    double g1 = (double)q * py * n1 / (double)R.L[1];
    double g2 = (double)q * pz * n2 / (double)R.L[2];
    if (self >= 0) {  // d/dr_s of -K q sum_t q_t g(|r_s - x_t|), g(r) = erf(alpha r) / r
        const int2 sp = R.gspan[self];
        const double al = (double)R.pme_alpha, c = 1.1283791670955126 * al;  // 2 alpha / sqrt(pi)
        for (int t = 0; t < sp.y; ++t) {
            const float4 at = R.xyzq[sp.x + t];
            double ex = (double)sx - at.x, ey = (double)sy - at.y, ez = (double)sz - at.z;
            ex -= rint(ex / (double)R.L[0]) * (double)R.L[0];
            ey -= rint(ey / (double)R.L[1]) * (double)R.L[1];
            ez -= rint(ez / (double)R.L[2]) * (double)R.L[2];
            const double r = sqrt(ex * ex + ey * ey + ez * ez);
            // g'(r) / r (a smooth even function: -(4/3) alpha^3 / sqrt(pi) at r = 0)
            const double gp = r < 1e-4 ? -(2.0 / 3.0) * c * al * al
                                       : (c * exp(-al * al * r * r) * r - erf(al * r)) / (r * r * r);
            const double w = -(double)kCoulomb * q * at.w * gp;
            g0 += w * ex;
            g1 += w * ey;
            g2 += w * ez;
        }
    }
    gx = (float)g0;
    gy = (float)g1;
    gz = (float)g2;
}

}  // namespace gcmc
