// Pose-energy kernel: the batched, cell-listed form of calcEnergy
// (gcmc/cpp/gcmc_energy.h:142-204).
//
// Work item = (pose, variant, z-slab), or for a translate / rotate step in the
// pairwise-difference form (StepDesc.dual) (pose, z-slab) with both poses.
// One warp per item:
//   1. builds the pose's sites in shared memory (insertion pose from the RNG,
//      or the slot's current / moved atoms),
//   2. walks the cells of its z-slab within R cells of the pose centre, tests
//      every group centre with the bit-exact FP32 inclusion distance and
//      compacts the included groups (ballot + popc),
//   3. flattens the included groups' atoms into a shared list and evaluates
//      all atom x site pairs with FP32 math (one atom per lane, sites
//      broadcast from shared memory), summing each atom's <= 20 site terms in
//      FP32 and the per-atom sums in FP64,
//   4. warp-reduces the FP64 partial and writes it to epart (no atomics: the
//      accept kernel sums the slabs in a fixed order),
//   5. for clustering moves, also writes its share of the pose's row of the
//      pose-pose "within cutoff" bit matrix (host distance form, bit-exact).
#pragma once
#include "common.cuh"
#include "pme.cuh"

namespace gcmc {

constexpr int kWarpsE = 8;
constexpr int kGCap = 128;
constexpr int kACap = 512;
constexpr unsigned kFull = 0xffffffffu;

// Sites 2p and 2p+1 of a pose, component-interleaved for the packed (f32x2)
// pair loop: negated centre-relative coordinates and Coulomb constant * charge.
struct SitePair {
    float2 nx, ny, nz, kq;
};

// Site s of a translate / rotate pose in the pairwise-difference form: the
// negated offsets so, sn of its old and its new position from the old pose
// centre (x: old, y: new; the new one in the old centre's periodic frame);
// twice its displacement delta = sn - so (from the absolute positions, rounded
// once) with the Coulomb constant * charge; and c = delta.(so + sn) =
// |sn|^2 - |so|^2 (FP64, rounded once), so that for an atom at offset A
// r_o^2 - r_n^2 = delta.(d_o + d_n) = 2 delta.A - c.
struct DualSite {
    float2 nx, ny, nz;
    float4 dk;
    float c, pad;
};

struct WarpBuf {
    float4 site[kMaxSites];  // x, y, z relative to the pose centre, Coulomb constant * charge
    int srow[kMaxSites];     // template type * ffY
    SitePair spair[kMaxSites / 2];
    DualSite dsite[kMaxSites];  // dual items (translate / rotate in the difference form)
    uint2 glist[kGCap];      // included group: (atomStart | image code << 26, atomNum)
    uint32_t alist[kACap];   // atom id  | image code << 26
    float cs_hi[3][4];       // pose centre + image shift (code 0: 0, 1: +L, 2: -L), high part
    float cs_lo[3][4];       //   and its exact rounding error (TwoSum)
    float4 site_abs[kMaxSites];  // absolute site position, raw charge (Ewald terms)
    int cbase[32];           // cell gather: entry base of each of the batch's cells
    int cexcl[32];           //   and the exclusive prefix of their entry counts
};

// Exact split of c + t into hi + lo (Knuth's TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& hi, float& lo) {
    hi = __fadd_rn(a, b);
    const float bb = __fsub_rn(hi, a);
    lo = __fadd_rn(__fsub_rn(a, __fsub_rn(hi, bb)), __fsub_rn(b, bb));
}

// Per item: the pose centre plus each periodic image shift as an exact
// (hi, lo) pair, so an atom's centre-relative offset (a - hi) - lo carries a
// single rounding of the offset itself.
template <class Buf>
__device__ __forceinline__ void set_centre(const RepDev& R, Buf& B, float cx, float cy, float cz, int lane) {
    if (lane < 9) {
        const int ax = lane / 3, code = lane - 3 * (lane / 3);
        const float c = ax == 0 ? cx : (ax == 1 ? cy : cz);
        const float t = code == 0 ? 0.0f : (code == 1 ? R.L[ax] : -R.L[ax]);
        float hi, lo;
        two_sum(c, t, hi, lo);
        B.cs_hi[ax][code] = hi;
        B.cs_lo[ax][code] = lo;
    }
    __syncwarp();
}

// Site s of the pose (centre-relative x, y, z and K q) into B.site and its
// slot of the interleaved pair layout.
template <class Buf>
__device__ __forceinline__ void put_site(Buf& B, int s, float x, float y, float z, float kq) {
    B.site[s] = make_float4(x, y, z, kq);
    float* p = reinterpret_cast<float*>(&B.spair[s >> 1]) + (s & 1);
    p[0] = -x;
    p[2] = -y;
    p[4] = -z;
    p[6] = kq;
}

__device__ __forceinline__ float image_shift(uint32_t code2, float L) {
    return code2 == 1u ? L : (code2 == 2u ? -L : 0.0f);
}

// Pair energies of the atoms buffered in B.alist[0, na) with the pose sites.
// Geometry is centre-relative: an atom's offset from the pose centre (with its
// group's periodic image) is (a - hi) - lo with hi + lo = centre + image
// exactly, i.e. one rounding of the offset, and the sites in B.site are stored
// relative to the same centre, so the FP32 pair differences carry ~1e-7 A of
// rounding instead of the ~1e-6 A of absolute-coordinate differences.
// PairImage = false: the atom takes its group's image (exact when every pair
// of an included group lies within half a box, checked at set-up); true:
// per-pair minimum image as in gcmc_energy.h:115-122.  1/r is rsqrt refined by
// one Newton step; each atom's site terms are summed in FP32, atoms in FP64.
template <bool PairImage, bool Ewald>
__device__ __forceinline__ void flush_atoms_t(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                              double& acc);

// Plain Coulomb: two sites per step with Blackwell's packed FP32 operations
// (__fadd2_rn / __fmul2_rn / __ffma2_rn: one instruction for both lanes of a
// float2, each lane correctly rounded as its scalar counterpart).  The per-pair
// arithmetic is the scalar form's; only the order of the per-atom FP32 site sum
// differs (even and odd sites in two partial sums, then added, then a last odd
// site).
template <bool PairImage>
__device__ __forceinline__ void flush_atoms_packed(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                                   double& acc) {
    const int np = ns >> 1;
    const float2 mhalf = make_float2(-0.5f, -0.5f), three_half = make_float2(1.5f, 1.5f);
    for (int f = lane; f < na; f += 32) {
        const uint32_t u = B.alist[f];
        const int idx = (int)(u & 0x3FFFFFFu);
        const float4 a = R.xyzq[idx];
        const int ta = R.atype[idx];
        uint32_t c0, c1, c2;
        if (PairImage) {
            const float kx = rintf((a.x - B.cs_hi[0][0]) * R.invL[0]);
            const float ky = rintf((a.y - B.cs_hi[1][0]) * R.invL[1]);
            const float kz = rintf((a.z - B.cs_hi[2][0]) * R.invL[2]);
            c0 = kx > 0.0f ? 1u : (kx < 0.0f ? 2u : 0u);
            c1 = ky > 0.0f ? 1u : (ky < 0.0f ? 2u : 0u);
            c2 = kz > 0.0f ? 1u : (kz < 0.0f ? 2u : 0u);
        } else {
            const uint32_t code = u >> 26;
            c0 = code & 3u; c1 = (code >> 2) & 3u; c2 = (code >> 4) & 3u;
        }
        const float ax = (a.x - B.cs_hi[0][c0]) - B.cs_lo[0][c0];
        const float ay = (a.y - B.cs_hi[1][c1]) - B.cs_lo[1][c1];
        const float az = (a.z - B.cs_hi[2][c2]) - B.cs_lo[2][c2];
        const float2 Ax = make_float2(ax, ax), Ay = make_float2(ay, ay), Az = make_float2(az, az);
        const float2 Aq = make_float2(a.w, a.w);
        float2 e2 = make_float2(0.0f, 0.0f);
#pragma unroll 2
        for (int p = 0; p < np; ++p) {
            const SitePair sp = B.spair[p];
            float2 dx = __fadd2_rn(Ax, sp.nx), dy = __fadd2_rn(Ay, sp.ny), dz = __fadd2_rn(Az, sp.nz);
            if (PairImage) {
                dx.x = fmaf(-rintf(dx.x * R.invL[0]), R.L[0], dx.x);
                dx.y = fmaf(-rintf(dx.y * R.invL[0]), R.L[0], dx.y);
                dy.x = fmaf(-rintf(dy.x * R.invL[1]), R.L[1], dy.x);
                dy.y = fmaf(-rintf(dy.y * R.invL[1]), R.L[1], dy.y);
                dz.x = fmaf(-rintf(dz.x * R.invL[2]), R.L[2], dz.x);
                dz.y = fmaf(-rintf(dz.y * R.invL[2]), R.L[2], dz.y);
            }
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
            float2 ir = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
            ir = __fmul2_rn(ir, __ffma2_rn(__fmul2_rn(__fmul2_rn(mhalf, r2), ir), ir, three_half));
            const float2 ir2 = __fmul2_rn(ir, ir);
            const float2 p0 = __ldg(&R.lj[B.srow[2 * p] + ta]);
            const float2 p1 = __ldg(&R.lj[B.srow[2 * p + 1] + ta]);
            const float2 s2 = __fmul2_rn(make_float2(p0.x, p1.x), ir2);
            const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
            e2 = __ffma2_rn(make_float2(p0.y, p1.y), __ffma2_rn(s6, s6, make_float2(-s6.x, -s6.y)), e2);
            e2 = __ffma2_rn(__fmul2_rn(sp.kq, Aq), ir, e2);
        }
        float e = e2.x + e2.y;
        if (ns & 1) {  // last site of an odd count
            const float4 sp = B.site[ns - 1];
            float dx = ax - sp.x, dy = ay - sp.y, dz = az - sp.z;
            if (PairImage) {
                dx = fmaf(-rintf(dx * R.invL[0]), R.L[0], dx);
                dy = fmaf(-rintf(dy * R.invL[1]), R.L[1], dy);
                dz = fmaf(-rintf(dz * R.invL[2]), R.L[2], dz);
            }
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            float ir = rsqrtf(r2);
            ir = ir * fmaf(-0.5f * r2 * ir, ir, 1.5f);
            const float ir2 = ir * ir;
            const float2 pp = __ldg(&R.lj[B.srow[ns - 1] + ta]);
            const float s2 = pp.x * ir2;
            const float s6 = s2 * s2 * s2;
            e = fmaf(pp.y, fmaf(s6, s6, -s6), e);
            e = fmaf(sp.w * a.w, ir, e);
        }
        acc += (double)e;
    }
}

template <bool PairImage, bool Ewald>
__device__ __forceinline__ void flush_atoms_t(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                              double& acc) {
    for (int f = lane; f < na; f += 32) {
        const uint32_t u = B.alist[f];
        const int idx = (int)(u & 0x3FFFFFFu);
        const float4 a = R.xyzq[idx];
        const int ta = R.atype[idx];
        uint32_t c0, c1, c2;
        if (PairImage) {  // the atom's image nearest the pose centre
            const float kx = rintf((a.x - B.cs_hi[0][0]) * R.invL[0]);
            const float ky = rintf((a.y - B.cs_hi[1][0]) * R.invL[1]);
            const float kz = rintf((a.z - B.cs_hi[2][0]) * R.invL[2]);
            c0 = kx > 0.0f ? 1u : (kx < 0.0f ? 2u : 0u);
            c1 = ky > 0.0f ? 1u : (ky < 0.0f ? 2u : 0u);
            c2 = kz > 0.0f ? 1u : (kz < 0.0f ? 2u : 0u);
        } else {
            const uint32_t code = u >> 26;
            c0 = code & 3u; c1 = (code >> 2) & 3u; c2 = (code >> 4) & 3u;
        }
        const float ax = (a.x - B.cs_hi[0][c0]) - B.cs_lo[0][c0];
        const float ay = (a.y - B.cs_hi[1][c1]) - B.cs_lo[1][c1];
        const float az = (a.z - B.cs_hi[2][c2]) - B.cs_lo[2][c2];
        float e = 0.0f;
#pragma unroll 4
        for (int s = 0; s < ns; ++s) {
            const float4 sp = B.site[s];
            float dx = ax - sp.x, dy = ay - sp.y, dz = az - sp.z;
            if (PairImage) {
                dx = fmaf(-rintf(dx * R.invL[0]), R.L[0], dx);
                dy = fmaf(-rintf(dy * R.invL[1]), R.L[1], dy);
                dz = fmaf(-rintf(dz * R.invL[2]), R.L[2], dz);
            }
            const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            float ir = rsqrtf(r2);
            ir = ir * fmaf(-0.5f * r2 * ir, ir, 1.5f);
            const float ir2 = ir * ir;
            const float2 p = __ldg(&R.lj[B.srow[s] + ta]);
            const float s2 = p.x * ir2;
            const float s6 = s2 * s2 * s2;
            e = fmaf(p.y, fmaf(s6, s6, -s6), e);
            if (Ewald) e = fmaf(sp.w * a.w * erfcf(R.pme_alpha * (r2 * ir)), ir, e);
            else e = fmaf(sp.w * a.w, ir, e);
        }
        acc += (double)e;
    }
}

// This lane's FP64 sum of the pair energies of the buffered atoms.  (Inlined:
// an out-of-line copy shared by the call sites measured slower, as the call
// makes the kernels spill around it.)
// Ew = 0: the replica never runs Ewald electrostatics (the Ewald loops are not
// compiled in: they add registers to the kernel around them).
template <int Ew = 1>
__device__ __forceinline__ double flush_atoms(const RepDev& R, const WarpBuf& B, int na, int ns, int lane) {
    double acc = 0.0;
    if (Ew && R.pme) {
        if (R.pair_image) flush_atoms_t<true, true>(R, B, na, ns, lane, acc);
        else flush_atoms_t<false, true>(R, B, na, ns, lane, acc);
    } else {
        if (R.pair_image) flush_atoms_packed<true>(R, B, na, ns, lane, acc);
        else flush_atoms_packed<false>(R, B, na, ns, lane, acc);
    }
    return acc;
}

// One atom's contribution to the energy change E_new - E_old of a translate /
// rotate pose, sites in the difference form (DualSite), the atom at (ax, ay,
// az) relative to the old pose centre.  fl bit 0: the atom's group lies within
// the cutoff of the old centre, bit 1: of the new one.  Both: per site the LJ
// change lj(new) - lj(old) and the Coulomb change k q_s q_a (1/r_n - 1/r_o),
// with 1/r_n - 1/r_o = (r_o^2 - r_n^2) / (r_o r_n (r_o + r_n)) and
// r_o^2 - r_n^2 = (d_o - d_n).(d_o + d_n) = delta.(d_o + d_n): the change comes
// out to a few ulp of itself instead of as the difference of two terms that
// are each an order of magnitude larger (under a per-pair minimum image whose
// old and new shifts differ, 1/r_n - 1/r_o directly).  One side only: +E_new or
// -E_old terms.  Each pair is the packed (f32x2) form of the single-pose pair
// energy, x the old pose and y the new one.
template <bool PairImage>
__device__ __forceinline__ float dual_atom_e(const RepDev& R, const DualSite* ds, const int* srow, int ns, float ax,
                                             float ay, float az, float q, int ta, uint32_t fl, const float2* lj) {
    const float2 mhalf = make_float2(-0.5f, -0.5f), three_half = make_float2(1.5f, 1.5f);
    const float2 Ax = make_float2(ax, ax), Ay = make_float2(ay, ay), Az = make_float2(az, az);
    float e = 0.0f;
#pragma unroll 2
    for (int s = 0; s < ns; ++s) {
        const DualSite d = ds[s];
        float2 dx = __fadd2_rn(Ax, d.nx), dy = __fadd2_rn(Ay, d.ny), dz = __fadd2_rn(Az, d.nz);
        bool same = true;
        if (PairImage) {
            const float kox = rintf(dx.x * R.invL[0]), knx = rintf(dx.y * R.invL[0]);
            const float koy = rintf(dy.x * R.invL[1]), kny = rintf(dy.y * R.invL[1]);
            const float koz = rintf(dz.x * R.invL[2]), knz = rintf(dz.y * R.invL[2]);
            dx = make_float2(fmaf(-kox, R.L[0], dx.x), fmaf(-knx, R.L[0], dx.y));
            dy = make_float2(fmaf(-koy, R.L[1], dy.x), fmaf(-kny, R.L[1], dy.y));
            dz = make_float2(fmaf(-koz, R.L[2], dz.x), fmaf(-knz, R.L[2], dz.y));
            same = kox == knx && koy == kny && koz == knz;
        }
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        float2 ir = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
        ir = __fmul2_rn(ir, __ffma2_rn(__fmul2_rn(__fmul2_rn(mhalf, r2), ir), ir, three_half));
        const float2 ir2 = __fmul2_rn(ir, ir);
        const float2 p = lj[srow[s] + ta];
        const float2 s2 = __fmul2_rn(make_float2(p.x, p.x), ir2);
        const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
        const float2 l = __fmul2_rn(make_float2(p.y, p.y), __ffma2_rn(s6, s6, make_float2(-s6.x, -s6.y)));
        const float kqq = d.dk.w * q;
        if (fl == 3u) {
            float dinv;
            if (same) {
                // r_o^2 - r_n^2: 2 delta.A - c (group image), or delta.(d_o + d_n) under a
                // per-pair image (the same shift for both, so the pair's own offsets)
                const float D = PairImage ? 0.5f * fmaf(d.dk.z, dz.x + dz.y, fmaf(d.dk.y, dy.x + dy.y,
                                                                                d.dk.x * (dx.x + dx.y)))
                                          : fmaf(d.dk.z, az, fmaf(d.dk.y, ay, fmaf(d.dk.x, ax, -d.c)));
                // 1/r_n - 1/r_o = D / (r_o r_n (r_o + r_n)) = D (ir_o ir_n)^2 / (ir_o + ir_n)
                dinv = __fdividef(D * (ir2.x * ir2.y), ir.x + ir.y);
            } else {
                dinv = ir.y - ir.x;
            }
            e += fmaf(kqq, dinv, l.y - l.x);
        } else if (fl == 2u) {
            e += fmaf(kqq, ir.y, l.y);
        } else {
            e -= fmaf(kqq, ir.x, l.x);
        }
    }
    return e;
}

// The buffered atoms B.alist[0, na) of a dual item: atom id in bits 0-23, the
// inclusion flags (dual_atom_e) in bits 24-25, the group's image code relative
// to the old centre in bits 26-31.
template <bool PairImage>
__device__ __forceinline__ void flush_dual(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                           double& acc) {
    for (int f = lane; f < na; f += 32) {
        const uint32_t u = B.alist[f];
        const int idx = (int)(u & 0xFFFFFFu);
        const float4 a = R.xyzq[idx];
        const int ta = R.atype[idx];
        uint32_t c0, c1, c2;
        if (PairImage) {  // the atom's image nearest the old pose centre
            const float kx = rintf((a.x - B.cs_hi[0][0]) * R.invL[0]);
            const float ky = rintf((a.y - B.cs_hi[1][0]) * R.invL[1]);
            const float kz = rintf((a.z - B.cs_hi[2][0]) * R.invL[2]);
            c0 = kx > 0.0f ? 1u : (kx < 0.0f ? 2u : 0u);
            c1 = ky > 0.0f ? 1u : (ky < 0.0f ? 2u : 0u);
            c2 = kz > 0.0f ? 1u : (kz < 0.0f ? 2u : 0u);
        } else {
            const uint32_t code = u >> 26;
            c0 = code & 3u; c1 = (code >> 2) & 3u; c2 = (code >> 4) & 3u;
        }
        const float ax = (a.x - B.cs_hi[0][c0]) - B.cs_lo[0][c0];
        const float ay = (a.y - B.cs_hi[1][c1]) - B.cs_lo[1][c1];
        const float az = (a.z - B.cs_hi[2][c2]) - B.cs_lo[2][c2];
        acc += (double)dual_atom_e<PairImage>(R, B.dsite, B.srow, ns, ax, ay, az, a.w, ta, (u >> 24) & 3u, R.lj);
    }
}

// What the cell walk does with each buffer of included atoms: the energy
// sink sums pair energies; the gradient kernel supplies its own sink.
template <int Ew = 1>
struct EnergySink {
    double acc = 0.0;
    __device__ __forceinline__ void flush(const RepDev& R, WarpBuf& B, int na, int ns, int lane) {
        acc += flush_atoms<Ew>(R, B, na, ns, lane);
    }
};

// The sink of a dual item: sums the pairwise energy changes.
struct DualSink {
    double acc = 0.0;
    __device__ __forceinline__ void flush(const RepDev& R, WarpBuf& B, int na, int ns, int lane) {
        if (R.pair_image) flush_dual<true>(R, B, na, ns, lane, acc);
        else flush_dual<false>(R, B, na, ns, lane, acc);
    }
};

// The new centre of a dual item: its exact coordinates (for the inclusion
// test) and the same point in the old centre's periodic frame (for the image
// codes of the groups included for it); the item's window: per axis the first
// cell (before wrapping) and the cell count, covering R cells around both
// centres' cells.
struct DualCentre {
    float nx, ny, nz;
    float ux, uy, uz;
    int w0[3], ws[3];
};

// Image code of a group centre g relative to a pose centre c (2 bits per
// axis: 0, 1 = +L, 2 = -L); sets *bad if the image lies more than one box away.
__device__ __forceinline__ uint32_t image_code(const RepDev& R, float gx, float gy, float gz, float cx, float cy,
                                               float cz, bool* bad) {
    const float rx = rintf((gx - cx) * R.invL[0]);
    const float ry = rintf((gy - cy) * R.invL[1]);
    const float rz = rintf((gz - cz) * R.invL[2]);
    *bad = fabsf(rx) > 1.0f || fabsf(ry) > 1.0f || fabsf(rz) > 1.0f;
    return (rx > 0.0f ? 1u : (rx < 0.0f ? 2u : 0u)) | ((ry > 0.0f ? 1u : (ry < 0.0f ? 2u : 0u)) << 2) |
           ((rz > 0.0f ? 1u : (rz < 0.0f ? 2u : 0u)) << 4);
}

// The window of a dual item along axis a: R cells around the cells of both
// centres (old cell po, new cell pn), the whole axis when that reaches around.
__device__ __forceinline__ void dual_window(const RepDev& R, int a, int po, int pn, int& w0, int& ws) {
    const int nc = R.nc[a];
    int dd = wrapi(pn - po, nc);
    if (dd > nc / 2) dd -= nc;
    ws = abs(dd) + 2 * R.range + 1;
    w0 = po + min(dd, 0) - R.range;
    if (ws >= nc) {
        ws = nc;
        w0 = 0;
    }
}

// Expand included groups B.glist[0, ng) into atoms and evaluate them.  Each
// lane takes one group of a batch of 32, a warp scan of the atom counts gives
// the write offsets; groups larger than the buffer are streamed in pieces.
template <class Sink>
__device__ __forceinline__ void process_groups(const RepDev& R, WarpBuf& B, int ng, int ns, int lane,
                                               Sink& sink, long long& npair) {
    int na = 0;
    for (int base = 0; base < ng; base += 32) {
        const int gi = base + lane;
        int start = 0, cnt = 0;
        uint32_t code = 0;
        if (gi < ng) {
            const uint2 ge = B.glist[gi];
            start = (int)(ge.x & 0x3FFFFFFu);
            cnt = (int)ge.y;
            code = ge.x >> 26;
        }
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        npair += (long long)total * ns;  // warp-uniform: atom x site pairs of this batch's groups
        const int maxcnt = __reduce_max_sync(kFull, (unsigned)cnt);
        if (maxcnt <= kACap / 2) {
            if (na + total > kACap) {
                __syncwarp();
                sink.flush(R, B, na, ns, lane);
                __syncwarp();
                na = 0;
            }
            if (total <= kACap) {
                const int off0 = na + incl - cnt;
                for (int j = 0; j < cnt; ++j) B.alist[off0 + j] = (uint32_t)(start + j) | (code << 26);
                na += total;
                continue;
            }
        }
        // large groups: one group at a time, in buffer-sized pieces
        for (int l = 0; l < 32; ++l) {
            const int s0 = __shfl_sync(kFull, start, l), c0 = __shfl_sync(kFull, cnt, l);
            const uint32_t cd = __shfl_sync(kFull, code, l);
            int done = 0;
            while (done < c0) {
                const int take = min(c0 - done, kACap - na);
                if (take == 0) {
                    __syncwarp();
                    sink.flush(R, B, na, ns, lane);
                    __syncwarp();
                    na = 0;
                    continue;
                }
                for (int j = lane; j < take; j += 32) B.alist[na + j] = (uint32_t)(s0 + done + j) | (cd << 26);
                na += take;
                done += take;
            }
        }
    }
    __syncwarp();
    sink.flush(R, B, na, ns, lane);
    __syncwarp();
}

// Energy of the pose in B.site against the groups whose cells lie in the
// window cells c0, c0 + stride, ... below c1 around the pose centre (flattened as
// ((z * span1) + y) * span0 + x), handed to the sink in buffers of atoms;
// ngroups (warp-uniform) counts the included groups.  Cells are visited 32 at
// a time: a warp scan of their entry counts numbers the batch's candidates,
// and lane t of each round of 32 finds its candidate's cell by binary search
// over the exclusive prefix, loads the entry (centre, id, atom range; one
// record) and tests it with the bit-exact inclusion distance.
__device__ __forceinline__ int wrap_near(int c, int n) {  // c in (-n, 2n)
    return c < 0 ? c + n : (c >= n ? c - n : c);
}
//
// Dual (dc set): a translate / rotate pose with old centre (cx, cy, cz) and new
// centre dc; the window is dc's (around both centres' cells), every group within
// the cutoff of either centre is listed with its inclusion flags in bits 24-25
// of the atom start (dual_atom_e; atom ids stay below 2^24), and a group
// included for both whose image codes relative to the two centres differ is
// listed twice, once for each side.
template <class Sink, bool Dual = false>
__device__ __forceinline__ void walk_cells(const RepDev& R, WarpBuf& B, int ns, float cx, float cy, float cz,
                                           int self, int c0, int c1, int lane, Sink& sink, int& ngroups,
                                           long long& npair, const int* stop = nullptr, int stop_at = 0,
                                           int stride = 1, const DualCentre* dc = nullptr) {
    set_centre(R, B, cx, cy, cz, lane);
    const int pcx = cell_coord(cx, R.start[0], R.invLc[0], R.nc[0]);
    const int pcy = cell_coord(cy, R.start[1], R.invLc[1], R.nc[1]);
    const int pcz = cell_coord(cz, R.start[2], R.invLc[2], R.nc[2]);
    const int sp0 = Dual ? dc->ws[0] : R.span[0], sp1 = Dual ? dc->ws[1] : R.span[1];
    const int sp2 = Dual ? dc->ws[2] : R.span[2];
    const int lo0 = Dual ? dc->w0[0] : pcx - R.range, lo1 = Dual ? dc->w0[1] : pcy - R.range;
    const int lo2 = Dual ? dc->w0[2] : pcz - R.range;
    const int sxy = sp0 * sp1;
    const float inv_s0 = 1.0f / (float)sp0, inv_sxy = 1.0f / (float)sxy;
    const unsigned lt = (1u << lane) - 1u;
    int ng = 0;
    long long both_atoms = 0;  // dual: atoms listed once for both poses (their pairs count twice)
    for (int base = c0; base < c1; base += 32 * stride) {  // window cells c0, c0 + stride, ... < c1
        const int j = base + lane * stride;
        int cell = 0, cnt = 0;
        if (j < c1) {
            const int jz = (int)(((float)j + 0.5f) * inv_sxy), jxy = j - jz * sxy;
            const int jy = (int)(((float)jxy + 0.5f) * inv_s0), jx = jxy - jy * sp0;
            const int x = (sp0 == R.nc[0]) ? jx : wrap_near(lo0 + jx, R.nc[0]);
            const int y = (sp1 == R.nc[1]) ? jy : wrap_near(lo1 + jy, R.nc[1]);
            const int z = (sp2 == R.nc[2]) ? jz : wrap_near(lo2 + jz, R.nc[2]);
            cell = (z * R.nc[1] + y) * R.nc[0] + x;
            cnt = R.cell_count[cell];
        }
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        B.cbase[lane] = cell * R.cap;
        B.cexcl[lane] = incl - cnt;
        __syncwarp();
        for (int t0 = 0; t0 < total; t0 += 32) {
            if (stop) {  // a speculative evaluation that has become void ends early
                int v = 0;
                if (lane == 0) v = *reinterpret_cast<const volatile int*>(stop);
                if (__shfl_sync(kFull, v, 0) == stop_at) { c1 = base; ng = -1; break; }
            }
            const int t = t0 + lane;
            bool inc = false, inc2 = false;
            uint2 packed = make_uint2(0u, 0u), packed2 = make_uint2(0u, 0u);
            if (t < total) {
                int lo = 0, hi = 31;  // the last cell whose exclusive prefix is <= t
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (B.cexcl[mid] <= t) lo = mid; else hi = mid - 1;
                }
                const CellEnt* e = R.cell_ent + B.cbase[lo] + (t - B.cexcl[lo]);
                // plain loads (not the read-only path) for the state: a speculative walk reads
                // records that the accept kernel may be writing meanwhile, and the persistent
                // step loop reads them after its own accept phase rewrote them
                const float4 gc = e->c;
                const int2 sp = e->span;
                if (Dual) {
                    if (__float_as_int(gc.w) != self) {
                        const bool io = within_cutoff<false>(cx, cy, cz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff,
                                                             R.cut2_lo, R.cut2_hi, R.fast_incl);
                        const bool in = within_cutoff<false>(dc->nx, dc->ny, dc->nz, gc.x, gc.y, gc.z, R.L, R.invL,
                                                             R.cutoff, R.cut2_lo, R.cut2_hi, R.fast_incl);
                        uint32_t co = 0u, cn = 0u;
                        bool bo = false, bn = false;
                        if (!R.pair_image) {
                            if (io) co = image_code(R, gc.x, gc.y, gc.z, cx, cy, cz, &bo);
                            if (in) cn = image_code(R, gc.x, gc.y, gc.z, dc->ux, dc->uy, dc->uz, &bn);
                        }
                        if (bo || bn) {
                            atomicOr(R.err, ERR_IMAGE);
                        } else if (io || in) {
                            // first entry: both sides if their images agree, else the old side
                            // (or the new one alone); second: the new side of a split group
                            const bool split = io && in && co != cn;
                            const uint32_t fl1 = split ? 1u : ((io ? 1u : 0u) | (in ? 2u : 0u));
                            inc = true;
                            packed = make_uint2((uint32_t)sp.x | (fl1 << 24) | ((io ? co : cn) << 26), (uint32_t)sp.y);
                            if (split) {
                                inc2 = true;
                                packed2 = make_uint2((uint32_t)sp.x | (2u << 24) | (cn << 26), (uint32_t)sp.y);
                            }
                            if (fl1 == 3u) both_atoms += sp.y;
                        }
                    }
                } else if (__float_as_int(gc.w) != self) {
                    inc = within_cutoff<false>(cx, cy, cz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                               R.cut2_hi, R.fast_incl);
                    if (inc) {
                        packed = make_uint2((uint32_t)sp.x, (uint32_t)sp.y);
                        if (!R.pair_image) {  // the group's periodic image relative to the pose centre
                            const float rx = rintf((gc.x - cx) * R.invL[0]);
                            const float ry = rintf((gc.y - cy) * R.invL[1]);
                            const float rz = rintf((gc.z - cz) * R.invL[2]);
                            if (fabsf(rx) > 1.0f || fabsf(ry) > 1.0f || fabsf(rz) > 1.0f) {
                                atomicOr(R.err, ERR_IMAGE);
                                inc = false;
                            } else {
                                const uint32_t code = (rx > 0.0f ? 1u : (rx < 0.0f ? 2u : 0u)) |
                                                      ((ry > 0.0f ? 1u : (ry < 0.0f ? 2u : 0u)) << 2) |
                                                      ((rz > 0.0f ? 1u : (rz < 0.0f ? 2u : 0u)) << 4);
                                packed.x |= code << 26;
                            }
                        }
                    }
                }
            }
            const unsigned m = __ballot_sync(kFull, inc);
            if (inc) B.glist[ng + __popc(m & lt)] = packed;
            ng += __popc(m);
            ngroups += __popc(m);
            if (Dual) {
                const unsigned m2 = __ballot_sync(kFull, inc2);
                if (inc2) B.glist[ng + __popc(m2 & lt)] = packed2;
                ng += __popc(m2);
            }
            if (ng > kGCap - (Dual ? 64 : 32)) {
                __syncwarp();
                process_groups(R, B, ng, ns, lane, sink, npair);
                ng = 0;
            }
        }
        __syncwarp();  // cbase / cexcl are rewritten by the next batch
    }
    __syncwarp();
    if (ng >= 0) process_groups(R, B, ng, ns, lane, sink, npair);  // ng < 0: stopped
    if (Dual) npair += (long long)__reduce_add_sync(kFull, (unsigned)both_atoms) * ns;
}

template <int Ew = 1>
__device__ __forceinline__ void energy_cells(const RepDev& R, WarpBuf& B, int ns, float cx, float cy, float cz,
                                             int self, int c0, int c1, int lane, double& acc, int& ngroups,
                                             long long& npair, const int* stop = nullptr, int stop_at = 0,
                                             int stride = 1) {
    EnergySink<Ew> sink;
    sink.acc = acc;
    walk_cells(R, B, ns, cx, cy, cz, self, c0, c1, lane, sink, ngroups, npair, stop, stop_at, stride);
    acc = sink.acc;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    return v;
}

// New site of lane `lane` for translate/rotate pose i (slot atoms from xyzq);
// identical arithmetic to build_pose's moved variant.
__device__ __forceinline__ void moved_site(const RepDev& R, const StepDesc& D, int i, const float4& gc,
                                           int ns, int lane, float& px, float& py, float& pz) {
    U4 r = rng(R.seed, R.replica, R.step_base + (uint32_t)D.step, (uint32_t)i, RP_MOVE, 0);
    if (D.move == MV_TRANSLATE) {
        px = fadd(px, trn_shift(R, r.x, 0, gc.x));
        py = fadd(py, trn_shift(R, r.y, 1, gc.y));
        pz = fadd(pz, trn_shift(R, r.z, 2, gc.z));
        return;
    }
    Mat3 Rm = move_rotation(R, r);
    const float nsf = (float)ns;
    float mx = 0.f, my = 0.f, mz = 0.f;
    for (int s = 0; s < ns; ++s) {
        mx = fadd(mx, fdiv(__shfl_sync(kFull, px, s), nsf));
        my = fadd(my, fdiv(__shfl_sync(kFull, py, s), nsf));
        mz = fadd(mz, fdiv(__shfl_sync(kFull, pz, s), nsf));
    }
    float x, y, z;
    rotate(Rm, fsub(px, mx), fsub(py, my), fsub(pz, mz), x, y, z);
    px = fadd(x, mx);
    py = fadd(y, my);
    pz = fadd(z, mz);
}

// ---- force-biased translate/rotate (proposal 2) ----
//
// Pose i's displacement d (translate) or rotation vector v (rotate, about the
// site centroid) has independent components on [-h, h] with densities
// a e^{a x} / (2 sinh(a h)), a = lambda beta f from the force (torque) f at the
// old pose (fb_tilted).  A translate moves the sites by d wrapped so the new
// centre lies in the box.  The reverse move is -d from the new pose with its
// own force, and the ratio of the two proposal densities enters the
// acceptance (fb_ln_ratio).  All float steps are explicit round-to-nearest
// operations so the host oracle reproduces them bit for bit.

// Force and torque partials of pose i, variant v, summed over the slabs in
// order (FP64) and rounded to float.  cg: read through L2 only (partials
// written by other CTAs of the running launch).
__device__ __forceinline__ void fb_force(const RepDev& R, const StepDesc& D, int i, int v, float f[6], bool cg) {
    for (int c = 0; c < 6; ++c) {
        double a = 0.0;
        for (int z = 0; z < D.nslab; ++z) {
            const float* p = R.fpart + ((size_t)(i * 2 + v) * D.nslab + z) * 6 + c;
            a += (double)(cg ? __ldcg(p) : *p);
        }
        f[c] = (float)a;
    }
}

// Shift of the centre coordinate c by d, wrapped into [start, start + L).
__device__ __forceinline__ float fb_shift(const RepDev& R, float d, int axis, float c) {
    const float k = floorf(fmul(fsub(fadd(c, d), R.start[axis]), R.invL[axis]));
    return fsub(d, fmul(k, R.L[axis]));
}

// Proposal of pose i from its old-pose force/torque f and group centre gc:
// prop[0] = (d, invalid), prop[1] = (a, 0); returns the new centre.
__device__ __forceinline__ float4 fb_propose(const RepDev& R, const StepDesc& D, int i, const float f[6],
                                             float4 gc, float4* prop) {
    const U4 r = rng(R.seed, R.replica, R.step_base + (uint32_t)D.step, (uint32_t)i, RP_FB, 0);
    const float u[3] = {u01_co(r.x), u01_co(r.y), u01_co(r.z)};
    const bool trn = D.move == MV_TRANSLATE;
    const float* g = trn ? f : f + 3;
    const bool ok = isfinite(g[0]) && isfinite(g[1]) && isfinite(g[2]);
    const float lb = trn ? R.fb_at : R.fb_ar, h = trn ? R.fb_ht : R.fb_hr;
    float d[3], a[3];
    for (int c = 0; c < 3; ++c) {
        a[c] = ok ? fmul(lb, g[c]) : 0.0f;
        d[c] = fb_tilted(a[c], h, u[c]);
    }
    prop[0] = make_float4(d[0], d[1], d[2], ok ? 0.0f : 1.0f);
    prop[1] = make_float4(a[0], a[1], a[2], 0.0f);
    if (!trn) return gc;
    return make_float4(fadd(gc.x, fb_shift(R, d[0], 0, gc.x)), fadd(gc.y, fb_shift(R, d[1], 1, gc.y)),
                       fadd(gc.z, fb_shift(R, d[2], 2, gc.z)), 0.0f);
}

// New site of lane `lane` (old site p) under pose i's stored proposal.
__device__ __forceinline__ void fb_moved_site(const RepDev& R, const StepDesc& D, int i, const float4& gc, int ns,
                                              int lane, float& px, float& py, float& pz) {
    const float4 d = R.fbprop[2 * i];
    if (D.move == MV_TRANSLATE) {
        px = fadd(px, fb_shift(R, d.x, 0, gc.x));
        py = fadd(py, fb_shift(R, d.y, 1, gc.y));
        pz = fadd(pz, fb_shift(R, d.z, 2, gc.z));
        return;
    }
    float nn = fmul(d.x, d.x);
    nn = ffma(d.y, d.y, nn);
    nn = ffma(d.z, d.z, nn);
    if (!(nn > 0.0f)) return;
    float ang = fsqrt(nn);
    ang = fsub(ang, fmul(floorf(fmul(ang, 0.159154943f)), kTwoPiF));  // same rotation, angle in [0, 2 pi)
    float sn, cs;
    det_sincos(ang, sn, cs);
    const Mat3 Rm = rodrigues(d.x, d.y, d.z, sn, cs);
    const float nsf = (float)ns;
    float mx = 0.f, my = 0.f, mz = 0.f;
    for (int s = 0; s < ns; ++s) {
        mx = fadd(mx, fdiv(__shfl_sync(kFull, px, s), nsf));
        my = fadd(my, fdiv(__shfl_sync(kFull, py, s), nsf));
        mz = fadd(mz, fdiv(__shfl_sync(kFull, pz, s), nsf));
    }
    float x, y, z;
    rotate(Rm, fsub(px, mx), fsub(py, my), fsub(pz, mz), x, y, z);
    px = fadd(x, mx);
    py = fadd(y, my);
    pz = fadd(z, mz);
}

// ln q(new -> old) - ln q(old -> new) for pose i: per component
// g(a') - g(a) - (a' + a) d with g = fb_lnorm, a (stored) the old tilt and
// a' = lambda beta f' from the new pose's force/torque fn; the rotation-vector
// Jacobian is even in v and cancels.  Float terms, FP64 sum.
__device__ __forceinline__ double fb_ln_ratio(const RepDev& R, const StepDesc& D, const float4& d, const float4& a,
                                              const float fn[6]) {
    const bool trn = D.move == MV_TRANSLATE;
    const float* g = trn ? fn : fn + 3;
    const float lb = trn ? R.fb_at : R.fb_ar, h = trn ? R.fb_ht : R.fb_hr;
    const float dd[3] = {d.x, d.y, d.z}, ao[3] = {a.x, a.y, a.z};
    double s = 0.0;
    for (int c = 0; c < 3; ++c) {
        const float an = fmul(lb, g[c]);
        const double t = __dsub_rn(__dsub_rn((double)fb_lnorm(an, h), (double)fb_lnorm(ao[c], h)),
                                   __dmul_rn(__dadd_rn((double)an, (double)ao[c]), (double)dd[c]));
        s = __dadd_rn(s, t);
    }
    return s;
}

// Load the pose of item (i, variant v) of step D into B.site; returns the
// pose centre and the residue to skip.
template <class Buf>
__device__ __forceinline__ void build_pose(const RepDev& R, const StepDesc& D, int i, int v, Buf& B,
                                           int lane, float& cx, float& cy, float& cz, int& self) {
    const FragDev& F = R.frag[D.ftype];
    const int ns = F.nsites;
    if (D.move == MV_INSERT) {
        float4 c = R.pcen[i];
        cx = c.x; cy = c.y; cz = c.z;
        self = -1;
        Mat3 Rm = insert_rotation(R, D.step, i);
        if (lane < ns) {
            float4 t = F.site[lane];
            float x, y, z;
            rotate(Rm, t.x, t.y, t.z, x, y, z);
            // absolute site (bit-exact, as written to the slot on acceptance), stored centre-relative
            const float sx = fadd(x, cx), sy = fadd(y, cy), sz = fadd(z, cz);
            put_site(B, lane, (float)((double)sx - (double)cx), (float)((double)sy - (double)cy),
                     (float)((double)sz - (double)cz), kCoulomb * t.w);
            B.site_abs[lane] = make_float4(sx, sy, sz, t.w);
            B.srow[lane] = F.stype[lane] * R.ffY;
        }
        __syncwarp();
        return;
    }
    const int slot = (D.move == MV_DELETE) ? D.del_slot : R.pslot[i];
    const int res = F.startRes + slot;
    self = res;
    const int2 sp = R.gspan[res];
    const float4 gc = R.gcen[res];
    float px = 0.f, py = 0.f, pz = 0.f;
    if (lane < ns) {
        float4 a = R.xyzq[sp.x + lane];
        px = a.x; py = a.y; pz = a.z;
        B.srow[lane] = F.stype[lane] * R.ffY;
    }
    if (D.move == MV_DELETE || v == 1 || D.move == MV_ROTATE) {  // centre unchanged
        cx = gc.x; cy = gc.y; cz = gc.z;
    } else {  // translated centre, computed by prepare_step with the same shift
        const float4 c = R.pcen[i];
        cx = c.x; cy = c.y; cz = c.z;
    }
    if (D.move != MV_DELETE && v == 0) {
        if (D.fb) fb_moved_site(R, D, i, gc, ns, lane, px, py, pz);
        else moved_site(R, D, i, gc, ns, lane, px, py, pz);
    }
    if (lane < ns) {
        put_site(B, lane, (float)((double)px - (double)cx), (float)((double)py - (double)cy),
                 (float)((double)pz - (double)cz), kCoulomb * F.site[lane].w);
        B.site_abs[lane] = make_float4(px, py, pz, F.site[lane].w);
    }
    __syncwarp();
}

// The first item of pose i's new variant keeps its trial sites (absolute
// position, charge) for the accept kernel, which writes an accepted pose from
// them instead of rebuilding it.
template <class Buf>
__device__ __forceinline__ void keep_sites(const RepDev& R, const StepDesc& D, const Buf& B, int i, int v, int zi,
                                           int lane) {
    if (v == 0 && zi == 0 && D.move != MV_DELETE && lane < R.frag[D.ftype].nsites)
        R.psite[i * kMaxSites + lane] = B.site_abs[lane];
}

// Translate / rotate pose i of step D in the difference form (one item for
// both poses): B.dsite, B.srow and the new sites in B.site_abs (for
// keep_sites); returns the old centre o (the group's centre, the frame of the
// site offsets), the new one in dc (exact, and unwrapped into o's periodic
// frame, with the window around both centres' cells) and the residue to skip.
// The new sites are moved_site's, as in build_pose; offsets and displacements
// are formed in FP64 from the absolute FP32 positions and rounded once.
template <class Buf>
__device__ __forceinline__ void build_pose_dual(const RepDev& R, const StepDesc& D, int i, Buf& B, int lane,
                                                float& ox, float& oy, float& oz, DualCentre& dc, int& self) {
    const FragDev& F = R.frag[D.ftype];
    const int ns = F.nsites;
    const int res = F.startRes + R.pslot[i];
    self = res;
    const int2 sp = R.gspan[res];
    const float4 gc = R.gcen[res];
    ox = gc.x; oy = gc.y; oz = gc.z;
    if (D.move == MV_TRANSLATE) {
        const float4 c = R.pcen[i];
        dc.nx = c.x; dc.ny = c.y; dc.nz = c.z;
    } else {
        dc.nx = gc.x; dc.ny = gc.y; dc.nz = gc.z;
    }
    dc.ux = dc.nx - R.L[0] * rintf((dc.nx - ox) * R.invL[0]);
    dc.uy = dc.ny - R.L[1] * rintf((dc.ny - oy) * R.invL[1]);
    dc.uz = dc.nz - R.L[2] * rintf((dc.nz - oz) * R.invL[2]);
    dual_window(R, 0, cell_coord(ox, R.start[0], R.invLc[0], R.nc[0]),
                cell_coord(dc.nx, R.start[0], R.invLc[0], R.nc[0]), dc.w0[0], dc.ws[0]);
    dual_window(R, 1, cell_coord(oy, R.start[1], R.invLc[1], R.nc[1]),
                cell_coord(dc.ny, R.start[1], R.invLc[1], R.nc[1]), dc.w0[1], dc.ws[1]);
    dual_window(R, 2, cell_coord(oz, R.start[2], R.invLc[2], R.nc[2]),
                cell_coord(dc.nz, R.start[2], R.invLc[2], R.nc[2]), dc.w0[2], dc.ws[2]);
    float px = 0.f, py = 0.f, pz = 0.f;
    if (lane < ns) {
        const float4 a = R.xyzq[sp.x + lane];
        px = a.x; py = a.y; pz = a.z;
        B.srow[lane] = F.stype[lane] * R.ffY;
    }
    const float qx = px, qy = py, qz = pz;
    moved_site(R, D, i, gc, ns, lane, px, py, pz);
    if (lane < ns) {
        const double dox = (double)qx - (double)ox, doy = (double)qy - (double)oy, doz = (double)qz - (double)oz;
        double dnx = (double)px - (double)ox, dny = (double)py - (double)oy, dnz = (double)pz - (double)oz;
        dnx -= (double)R.L[0] * rint(dnx / (double)R.L[0]);  // a translate wrapped across the box
        dny -= (double)R.L[1] * rint(dny / (double)R.L[1]);
        dnz -= (double)R.L[2] * rint(dnz / (double)R.L[2]);
        DualSite d;
        d.nx = make_float2(-(float)dox, -(float)dnx);
        d.ny = make_float2(-(float)doy, -(float)dny);
        d.nz = make_float2(-(float)doz, -(float)dnz);
        d.dk = make_float4((float)(2.0 * (dnx - dox)), (float)(2.0 * (dny - doy)), (float)(2.0 * (dnz - doz)),
                           kCoulomb * F.site[lane].w);
        d.c = (float)((dnx * dnx + dny * dny + dnz * dnz) - (dox * dox + doy * doy + doz * doz));
        d.pad = 0.0f;
        B.dsite[lane] = d;
        B.site_abs[lane] = make_float4(px, py, pz, F.site[lane].w);
    }
    __syncwarp();
}

// The draws of pose i that do not depend on energies, made once per pose by
// the pose-energy kernels (off the single-CTA accept kernel's critical path):
// the Gumbel perturbation -ln(-ln u) and ln u of the cluster acceptance draw.
__device__ __forceinline__ void pose_draws(const RepDev& R, const StepDesc& D, int i) {
    const U4 g = rng(R.seed, R.replica, R.step_base + (uint32_t)D.step, (uint32_t)i, RP_GUMBEL, 0);
    R.pgum[i] = -log(-log(u53_open(g.x, g.y)));
    const U4 ua = rng(R.seed, R.replica, R.step_base + (uint32_t)D.step, (uint32_t)i, RP_CLUSTER, 0);
    R.plnu[i] = log(u53(ua.x, ua.y));
}

// Words [zi nw / nslab, (zi + 1) nw / nslab) of pose i's row of the pose-pose
// "within cutoff" bit matrix (host distance form, bit-exact).  The row of pose
// 32 w also makes the energy-independent draws of the 32 poses of word w, one
// per lane.
__device__ __forceinline__ void nbr_rows(const RepDev& R, const StepDesc& D, int i, int zi, int nsl, int lane) {
    const int w0 = zi * D.nw / nsl, w1 = (zi + 1) * D.nw / nsl;
    const float4 ci = R.pcen[i];
    for (int w = w0; w < w1; ++w) {
        const int j = 32 * w + lane;
        if (i == 32 * w && j < D.k) pose_draws(R, D, j);
        bool b = false;
        if (j < D.k) {
            const float4 cj = R.pcen[j];
            b = within_cutoff<true>(ci.x, ci.y, ci.z, cj.x, cj.y, cj.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                    R.cut2_hi, R.fast_incl);
        }
        const unsigned m = __ballot_sync(kFull, b);
        if (lane == 0) R.nbr[i * D.nw + w] = m;
    }
}

// Transpose of a 32 x 32 bit block held one row per lane (bit c of lane r =
// entry (r, c)): afterwards lane c holds column c (bit r = entry (r, c)).
// Five rounds of exchanging the off-diagonal s x s sub-blocks between lanes
// l and l ^ s (s = 16, 8, 4, 2, 1).
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
    const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        const int sft = 16 >> t;
        const uint32_t M = masks[t];
        const uint32_t y = __shfl_xor_sync(kFull, x, sft);
        x = (lane & sft) ? ((x & ~M) | ((y >> sft) & M)) : ((x & M) | ((y & M) << sft));
    }
    return x;
}

// Block task p (upper triangle in row order) of the pose-pose "within cutoff"
// bit matrix, whose 32 x 32 blocks (I, J), I <= J, cover all of it: the matrix
// is symmetric bit for bit (both distance forms are odd in the difference and
// round symmetrically), so lane c tests pose 32 J + c against the block's 32
// row poses (centres broadcast by shuffles), the row words of (I, J) come from
// ballots and those of the mirror block (J, I) from their transpose.  A
// diagonal block also makes the energy-independent draws of its 32 poses.
__device__ __forceinline__ void nbr_block(const RepDev& R, const StepDesc& D, int p, int lane) {
    const int k = D.k, nw = D.nw;
    int I = 0, rem = p;
    while (rem >= nw - I) {
        rem -= nw - I;
        ++I;
    }
    const int J = I + rem;
    const int jc = 32 * J + lane, ir = 32 * I + lane;
    if (I == J && jc < k) pose_draws(R, D, jc);
    float4 cj = make_float4(0.f, 0.f, 0.f, 0.f), cr = cj;
    if (jc < k) cj = R.pcen[jc];
    if (ir < k) cr = R.pcen[ir];
    const int nrow = min(32, k - 32 * I);
    uint32_t mine = 0u;  // lane r: word J of row 32 I + r
    for (int r = 0; r < nrow; ++r) {
        const float x = __shfl_sync(kFull, cr.x, r), y = __shfl_sync(kFull, cr.y, r), z = __shfl_sync(kFull, cr.z, r);
        const bool b = jc < k && within_cutoff<true>(x, y, z, cj.x, cj.y, cj.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                                     R.cut2_hi, R.fast_incl);
        const unsigned m = __ballot_sync(kFull, b);
        if (lane == r) mine = m;
    }
    if (ir < k) R.nbr[ir * nw + J] = mine;
    if (I != J) {
        const uint32_t t = transpose32(mine, lane);  // lane c: word I of row 32 J + c
        if (jc < k) R.nbr[jc * nw + I] = t;
    }
}

// New-variant item (i, zi)'s share of the bit matrix.  A launch with more
// items than resident warps is throughput-bound: there the first
// nw (nw + 1) / 2 items compute a block each (half the distance tests);
// otherwise every item computes its slab's share of pose i's row, which keeps
// each item's latency short.  Both give the same matrix.
// (i, zi): the item's pose and range of nsl; task: its index among the step's
// new-variant items (at least k of them, more than the nw (nw + 1) / 2 blocks).
__device__ __forceinline__ void nbr_share(const RepDev& R, const StepDesc& D, int i, int zi, int nsl, int task,
                                          int lane, bool sym) {
    if (sym) {
        if (task < D.nw * (D.nw + 1) / 2) nbr_block(R, D, task, lane);
    } else {
        nbr_rows(R, D, i, zi, nsl, lane);
    }
}

// pre[r] = work items of the replicas before r, pre[nrep] = all of them,
// computed by the whole block (one replica per thread, warp scans, then the
// warp totals) so that no thread walks the replica list alone.
template <class Items>
__device__ __forceinline__ void items_prefix(int nrep, int* pre, int* wtot, Items items) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
    int carry = 0;
    for (int base = 0; base < nrep; base += blockDim.x) {
        const int r = base + tid;
        const int v = r < nrep ? items(r) : 0;
        int inc = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int t = __shfl_up_sync(kFull, inc, off);
            if (lane >= off) inc += t;
        }
        if (lane == 31) wtot[warp] = inc;
        __syncthreads();
        int before = 0, tot = 0;
        for (int w = 0; w < nwarp; ++w) {
            const int t = wtot[w];
            if (w < warp) before += t;
            tot += t;
        }
        if (r < nrep) pre[r] = carry + before + inc - v;
        carry += tot;
        __syncthreads();
    }
    if (tid == 0) pre[nrep] = carry;
    __syncthreads();
}

// One item of a pose-energy launch (whole warp): item `it` of the replicas'
// items numbered by the prefix pre (pre[r] = items of the replicas before r).
// sym: more items than warps (throughput-bound; see nbr_share).  Which: the
// kinds of items this code path handles (-1 both, 0 / 1 the steps not in / in
// the difference form).
template <int Which, int Ew>
__device__ __forceinline__ void energy_item(const RepDev* __restrict__ reps, int nrep, int mode, WarpBuf& B,
                                            const int* pre, int it, int lane, bool sym) {
    int lo = 0, hi = nrep;  // find r with pre[r] <= it < pre[r+1]
    while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (pre[mid] <= it) lo = mid; else hi = mid; }
    const RepDev& R = reps[lo];
    const StepDesc D = *R.desc;
    const int local = it - pre[lo];
    int i, v, zi, nsl;
    if (D.varslab) {  // the preparation's list: pose variant e's range zi of pnslab[e]
        const int pk = R.pitem[local];
        const int e = pk >> 8;
        zi = pk & 255;
        i = e / D.nvar;
        v = e - i * D.nvar;
        nsl = R.pnslab[e];
    } else {
        // pose fastest: the ranges of one pose go to different CTAs (and SMs), so the
        // items of a heavy pose do not share one SM's issue slots
        const int q = local / max(1, D.k);
        i = local - q * D.k;
        v = q / D.nslab;
        zi = q - v * D.nslab;
        nsl = D.nslab;
    }
    float cx, cy, cz;
    int self;
    double acc = 0.0;
    int ng = 0;
    long long npair = 0;
    if (Which != 0 && D.dual) {  // translate / rotate: the energy change of both poses in one walk
        DualCentre dc;
        build_pose_dual(R, D, i, B, lane, cx, cy, cz, dc, self);
        keep_sites(R, D, B, i, 0, zi, lane);
        const int nwin = dc.ws[0] * dc.ws[1] * dc.ws[2];
        DualSink sink;
        walk_cells<DualSink, true>(R, B, R.frag[D.ftype].nsites, cx, cy, cz, self, zi, nwin, lane, sink, ng,
                                   npair, mode == 1 ? R.abort : nullptr, D.step, nsl, &dc);
        acc = sink.acc;
    } else if (Which != 1) {
        build_pose(R, D, i, v, B, lane, cx, cy, cz, self);
        keep_sites(R, D, B, i, v, zi, lane);
        const int nwin = R.span[0] * R.span[1] * R.span[2];
        // range zi of the pose's window: cells zi, zi + nslab, ... (interleaved, so that every
        // range samples the whole cutoff sphere and the ranges of a pose take equal time)
        energy_cells<Ew>(R, B, R.frag[D.ftype].nsites, cx, cy, cz, self, zi, nwin, lane, acc, ng, npair,
                         mode == 1 ? R.abort : nullptr, D.step, nsl);
        if (Ew && R.pme && zi == 0) {
            const float4 a = B.site_abs[lane < kMaxSites ? lane : 0];
            acc += pme_pose_lane(R, R.frag[D.ftype].nsites, lane, a.x, a.y, a.z, a.w, self);
        }
    }
    acc = warp_sum(acc);
    if (lane == 0) {
        R.epart[(i * D.nvar + v) * D.nslab + zi] = acc;
        if (D.dual) R.epart[(i * D.nvar + 1) * D.nslab + zi] = 0.0;  // the old variant's share
        atomicAdd(mode == 1 ? R.pairs_pending : &R.counters[2], (unsigned long long)npair);
    }
    if (v == 0 && D.nw > 0) {
        int stop = 0;
        if (mode == 1 && lane == 0) stop = *reinterpret_cast<const volatile int*>(R.abort) == D.step;
        if (!__shfl_sync(kFull, stop, 0))
            nbr_share(R, D, i, zi, nsl, D.varslab ? local : i * D.nslab + zi, lane, sym);
    }
}

// One launch per MC step: every replica's (pose, variant, slab) items.
// Two register budgets of the same kernel, picked per context (gcmc_options.
// energy_variant, autotuned): MinBlocks = 3 CTAs per SM (up to 85 registers,
// fewer spills; best for a single replica whose step is latency-bound) or 4
// (64 registers, more warps in flight; best for large batches).
//
// mode 0: every item; mode 1 (speculative, nrep = 1): pair count into
// pairs_pending, and the walks end early once the step has been voided (the
// accept kernel of the step before accepted a move); mode 2 (completion,
// nrep = 1): nothing if the speculative evaluation of this step stands (the
// accept kernel books its pair count), else mode 0.
// The items of one pose-energy launch, whole CTA: warp w of the CTA is warp
// gw0 + w of the nwarps that share the items; B: this warp's buffer; pre,
// wtot: 257 and 32 ints of shared memory.  The body of k_energy_t and of the
// persistent step loop.  Which: -1 every replica's items; 0 only the items of
// steps not in the difference form, 1 only those of steps in it (the
// persistent step loop runs the two kinds one after the other, so that an SM
// holds one code path's instructions at a time; a batched launch runs both
// kinds SM-affine, energy_items_affine).
// queue (optional): a counter, zero before the launch, from which warps take
// their next item (the items' results do not depend on which warp takes them);
// without it warp g takes items g, g + nwarps, ...
template <int Which, int Ew = 1>
__device__ __forceinline__ void energy_items(const RepDev* __restrict__ reps, int nrep, int mode, int gw0,
                                             int nwarps, WarpBuf& B, int* pre, int* wtot, int* queue = nullptr) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    items_prefix(nrep, pre, wtot, [&](int r) {
        const StepDesc* d = reps[r].desc;
        return (Which < 0 || (Which == 1) == (d->dual != 0)) ? d->items : 0;
    });
    const int total = pre[nrep];
    const bool sym = total > nwarps;  // more items than warps: throughput-bound
    auto next_item = [&](int prev) {
        if (!queue) return prev < 0 ? gw0 + warp : prev + nwarps;
        int v = 0;
        if (lane == 0) v = atomicAdd(queue, 1);
        return __shfl_sync(kFull, v, 0);
    };
    for (int it = next_item(-1); it < total; it = next_item(it)) {
        energy_item<Which, Ew>(reps, nrep, mode, B, pre, it, lane, sym);
        __syncwarp();
    }
}

// Both kinds of items in one launch (a batch whose replicas' steps lie in and
// out of the difference form): the warps of an SM take the kind its SM index
// selects, the SMs split between the kinds in proportion to their item counts,
// so that an SM fetches one code path's instructions; a warp whose kind has run
// out then takes the other kind's remaining items.  Items come from the
// counters queue[0] (steps not in the difference form) and queue[1] (steps in
// it), zero before the launch; pre0 / pre1: 257 ints of shared memory each.
template <int Ew>
__device__ __forceinline__ void energy_items_affine(const RepDev* __restrict__ reps, int nrep, int mode, int nwarps,
                                                    WarpBuf& B, int* pre0, int* pre1, int* wtot, int* queue) {
    const int lane = threadIdx.x & 31;
    items_prefix(nrep, pre0, wtot, [&](int r) {
        const StepDesc* d = reps[r].desc;
        return d->dual ? 0 : d->items;
    });
    items_prefix(nrep, pre1, wtot, [&](int r) {
        const StepDesc* d = reps[r].desc;
        return d->dual ? d->items : 0;
    });
    const int t0 = pre0[nrep], t1 = pre1[nrep];
    const bool sym = t0 + t1 > nwarps;
    unsigned smid, nsm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    asm volatile("mov.u32 %0, %%nsmid;" : "=r"(nsm));
    int kind = ((long long)smid * (t0 + t1) < (long long)t0 * nsm) ? 0 : 1;
    for (int pass = 0; pass < 2; ++pass, kind ^= 1) {
        const int total = kind ? t1 : t0;
        for (;;) {
            int v = 0;
            if (lane == 0) v = atomicAdd(&queue[kind], 1);
            const int it = __shfl_sync(kFull, v, 0);
            if (it >= total) break;
            if (kind == 0) energy_item<0, Ew>(reps, nrep, mode, B, pre0, it, lane, sym);
            else energy_item<1, Ew>(reps, nrep, mode, B, pre1, it, lane, sym);
            __syncwarp();
        }
    }
}

template <int MinBlocks, int Which, int Ew>
__global__ void __launch_bounds__(kWarpsE * 32, MinBlocks) k_energy_t(const RepDev* __restrict__ reps, int nrep,
                                                                      int mode) {
    __shared__ WarpBuf bufs[kWarpsE];
    __shared__ int pre[257];
    __shared__ int wtot[32];
    // the completion launch of a speculating graph is a programmatic dependent of the step's
    // re-preparation: a standing step (valid, set by the accept kernel of the step before,
    // which completed before the re-preparation began) returns at once; otherwise wait for
    // the re-preparation's results.  Then the accept kernel may be scheduled.
    if (mode == 2 && *reps[0].valid) return;
    pdl_wait();
    pdl_trigger();
    // several replicas (throughput-bound launches): warps take items from a counter, which
    // balances uneven items; one replica (latency-bound, about one item per warp): a fixed
    // stride, which saves the counter's round trip per item
    StepDesc* d0 = reps[0].desc;
    const int q = Which == 1 ? 1 : 0;
    if (Which == 2) {  // both kinds, SM-affine (batches only)
        __shared__ int pre1[257];
        energy_items_affine<Ew>(reps, nrep, mode, gridDim.x * kWarpsE, bufs[threadIdx.x >> 5], pre, pre1, wtot,
                                d0->queue);
    } else {
        energy_items<Which, Ew>(reps, nrep, mode, blockIdx.x * kWarpsE, gridDim.x * kWarpsE,
                                bufs[threadIdx.x >> 5], pre, wtot, nrep > 1 ? &d0->queue[q] : nullptr);
    }
    if (nrep == 1) return;
    // the last CTA to finish resets the counter for the next launch (every warp has taken
    // its last item once its CTA arrives here)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&d0->done[q], 1) == (int)gridDim.x - 1) {
            d0->queue[q] = 0;
            if (Which == 2) d0->queue[1] = 0;
            d0->done[q] = 0;
            __threadfence();
        }
    }
}

template __global__ void k_energy_t<3, -1, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<4, -1, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<3, 0, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<4, 0, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<3, 1, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<4, 1, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<3, 2, 0>(const RepDev* __restrict__, int, int);  // both kinds, SM-affine
template __global__ void k_energy_t<4, 2, 0>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_t<3, -1, 1>(const RepDev* __restrict__, int, int);  // Ewald contexts
template __global__ void k_energy_t<4, -1, 1>(const RepDev* __restrict__, int, int);

// Energies of caller-supplied poses (gcmc_energy_poses): item = (pose, slab).
// The replica descriptor is passed by value so that callers can substitute
// the pair table (R.lj).
__global__ void __launch_bounds__(kWarpsE * 32)
    k_energy_explicit(__grid_constant__ const RepDev R, const float* __restrict__ xyz,
                      const float* __restrict__ q, const int* __restrict__ type, int ns,
                      const float* __restrict__ centres, const int* __restrict__ self, int nposes,
                      int nslab, double* __restrict__ out, int* __restrict__ ngout) {
    __shared__ WarpBuf bufs[kWarpsE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpBuf& B = bufs[warp];
    const int total = nposes * nslab;
    for (int it = blockIdx.x * kWarpsE + warp; it < total; it += gridDim.x * kWarpsE) {
        const int p = it / nslab, z = it - p * nslab;
        // a site type outside the pair table's rows would index past it: flag the
        // input error (reported by the next gcmc_sync) and give the pose NaN
        const bool bad_type = lane < ns && (unsigned)type[lane] >= (unsigned)R.ffX;
        if (__any_sync(kFull, bad_type)) {
            if (lane == 0) {
                atomicOr(R.err, ERR_SITE_TYPE);
                out[it] = __longlong_as_double(0x7ff8000000000000ll);
                ngout[it] = 0;
            }
            __syncwarp();
            continue;
        }
        if (lane < ns) {
            const float* s = xyz + ((size_t)p * ns + lane) * 3;
            const double c0 = centres[3 * p], c1 = centres[3 * p + 1], c2 = centres[3 * p + 2];
            put_site(B, lane, (float)((double)s[0] - c0), (float)((double)s[1] - c1), (float)((double)s[2] - c2),
                     kCoulomb * q[lane]);
            B.site_abs[lane] = make_float4(s[0], s[1], s[2], q[lane]);
            B.srow[lane] = type[lane] * R.ffY;
        }
        __syncwarp();
        double acc = 0.0;
        int ng = 0;
        long long npair = 0;
        const int nwin = R.span[0] * R.span[1] * R.span[2];
        energy_cells(R, B, ns, centres[3 * p], centres[3 * p + 1], centres[3 * p + 2], self ? self[p] : -1,
                     z * nwin / nslab, (z + 1) * nwin / nslab, lane, acc, ng, npair);
        if (R.pme && z == 0) {
            const float4 a = B.site_abs[lane < kMaxSites ? lane : 0];
            acc += pme_pose_lane(R, ns, lane, a.x, a.y, a.z, a.w, self ? self[p] : -1);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            out[it] = acc;
            ngout[it] = ng;
        }
        __syncwarp();
    }
}

}  // namespace gcmc
