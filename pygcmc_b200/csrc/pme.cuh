// Ewald electrostatics by smooth particle-mesh Ewald (Essmann et al., J. Chem.
// Phys. 103 (1995) 8577), FP64 mesh; not in the reference, whose calcEnergy
// uses a plain cutoff.
//
// Per MC step, before the pose energies, each replica's mesh potential is
// rebuilt: Q = Q_fixed (the fixed atoms' spread charges, made once) + the
// occupied fragment atoms spread with order-4 cardinal B-splines;
// phi_mesh = IFFT(G * FFT(Q)) with G(m) = K exp(-pi^2 m^2 / alpha^2) B(m) /
// (pi V m^2), B the B-spline moduli (cuFFT D2Z / Z2D).  The potential at a
// point is the same B-spline interpolation of phi_mesh.
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

// spectrum *= G (half spectrum, n0 * n1 * (n2/2 + 1) complex values)
__global__ void k_pme_scale(double2* __restrict__ spec, const double* __restrict__ G, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double g = G[i];
        double2 v = spec[i];
        v.x *= g;
        v.y *= g;
        spec[i] = v;
    }
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

}  // namespace gcmc
