// Pose-energy kernel: the batched, cell-listed form of calcEnergy
// (gcmc/cpp/gcmc_energy.h:142-204).
//
// Work item = (pose, variant, z-slab).  One warp per item:
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

namespace gcmc {

constexpr int kWarpsE = 8;
constexpr int kGCap = 128;
constexpr int kACap = 512;
constexpr unsigned kFull = 0xffffffffu;

struct WarpBuf {
    float4 site[kMaxSites];  // x, y, z, Coulomb constant * charge
    int srow[kMaxSites];     // template type * ffY
    uint32_t glist[kGCap];   // group id | image code << 26
    uint32_t alist[kACap];   // atom id  | image code << 26
};

__device__ __forceinline__ float image_shift(uint32_t code2, float L) {
    return code2 == 1u ? L : (code2 == 2u ? -L : 0.0f);
}

// Pair energies of the atoms buffered in B.alist[0, na) with the pose sites.
// Geometry is centre-relative: each atom's offset from the pose centre is
// formed in FP64 (including its periodic image) and rounded once to FP32, and
// the sites in B.site are stored relative to the same centre, so the FP32
// pair differences carry ~1e-7 A of rounding instead of the ~1e-6 A of
// absolute-coordinate differences.  PairImage = false: the atom takes its
// group's image (exact when every pair of an included group lies within half
// a box, checked at set-up); true: per-pair minimum image as in
// gcmc_energy.h:115-122.  1/r is rsqrt refined by one Newton step.
template <bool PairImage>
__device__ __forceinline__ void flush_atoms_t(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                              double cx, double cy, double cz, double& acc) {
    for (int f = lane; f < na; f += 32) {
        uint32_t u = B.alist[f];
        int idx = (int)(u & 0x3FFFFFFu);
        uint32_t code = u >> 26;
        float4 a = __ldg(&R.xyzq[idx]);
        int ta = __ldg(&R.atype[idx]);
        double ox = (double)a.x - cx, oy = (double)a.y - cy, oz = (double)a.z - cz;
        if (PairImage) {
            ox -= (double)R.L[0] * rint(ox * (double)R.invL[0]);
            oy -= (double)R.L[1] * rint(oy * (double)R.invL[1]);
            oz -= (double)R.L[2] * rint(oz * (double)R.invL[2]);
        } else {
            ox -= (double)image_shift(code & 3u, R.L[0]);
            oy -= (double)image_shift((code >> 2) & 3u, R.L[1]);
            oz -= (double)image_shift((code >> 4) & 3u, R.L[2]);
        }
        const float ax = (float)ox, ay = (float)oy, az = (float)oz;
        float e = 0.0f;
#pragma unroll 4
        for (int s = 0; s < ns; ++s) {
            float4 sp = B.site[s];
            float dx = ax - sp.x, dy = ay - sp.y, dz = az - sp.z;
            if (PairImage) {
                dx = fmaf(-rintf(dx * R.invL[0]), R.L[0], dx);
                dy = fmaf(-rintf(dy * R.invL[1]), R.L[1], dy);
                dz = fmaf(-rintf(dz * R.invL[2]), R.L[2], dz);
            }
            float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            float ir = rsqrtf(r2);
            ir = ir * fmaf(-0.5f * r2 * ir, ir, 1.5f);
            float ir2 = ir * ir;
            float2 p = __ldg(&R.lj[B.srow[s] + ta]);
            float s2 = p.x * ir2;
            float s6 = s2 * s2 * s2;
            e = fmaf(p.y, fmaf(s6, s6, -s6), e);
            e = fmaf(sp.w * a.w, ir, e);
        }
        acc += (double)e;
    }
}

__device__ __forceinline__ void flush_atoms(const RepDev& R, const WarpBuf& B, int na, int ns, int lane,
                                            double cx, double cy, double cz, double& acc) {
    if (R.pair_image) flush_atoms_t<true>(R, B, na, ns, lane, cx, cy, cz, acc);
    else flush_atoms_t<false>(R, B, na, ns, lane, cx, cy, cz, acc);
}

// Expand included groups B.glist[0, ng) into atoms and evaluate them.  Each
// lane takes one group of a batch of 32, a warp scan of the atom counts gives
// the write offsets; groups larger than the buffer are streamed in pieces.
__device__ __forceinline__ void process_groups(const RepDev& R, WarpBuf& B, int ng, int ns, int lane,
                                               double cx, double cy, double cz, double& acc, long long& npair) {
    int na = 0;
    for (int base = 0; base < ng; base += 32) {
        const int gi = base + lane;
        int start = 0, cnt = 0;
        uint32_t code = 0;
        if (gi < ng) {
            const uint32_t ge = B.glist[gi];
            const int2 sp = __ldg(&R.gspan[(int)(ge & 0x3FFFFFFu)]);
            start = sp.x;
            cnt = sp.y;
            code = ge >> 26;
        }
        npair += (long long)cnt * ns;
        int incl = cnt;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, off);
            if (lane >= off) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        const int maxcnt = __reduce_max_sync(kFull, (unsigned)cnt);
        if (maxcnt <= kACap / 2) {
            if (na + total > kACap) {
                __syncwarp();
                flush_atoms(R, B, na, ns, lane, cx, cy, cz, acc);
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
                    flush_atoms(R, B, na, ns, lane, cx, cy, cz, acc);
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
    flush_atoms(R, B, na, ns, lane, cx, cy, cz, acc);
    __syncwarp();
}

// Energy of the pose in B.site against the groups whose cells lie in z-slab
// `slab` around the pose centre; returns this lane's FP64 partial.  ngroups
// (warp-uniform) counts the included groups.
__device__ __noinline__ void energy_slab(const RepDev& R, WarpBuf& B, int ns, float cx, float cy, float cz,
                                         int self, int slab, int lane, double& acc, int& ngroups,
                                         long long& npair) {
    const int pcx = cell_coord(cx, R.start[0], R.invLc[0], R.nc[0]);
    const int pcy = cell_coord(cy, R.start[1], R.invLc[1], R.nc[1]);
    const int pcz = cell_coord(cz, R.start[2], R.invLc[2], R.nc[2]);
    const int z = (R.span[2] == R.nc[2]) ? slab : wrapi(pcz - R.range + slab, R.nc[2]);
    const int nxy = R.span[0] * R.span[1];
    const unsigned lt = (1u << lane) - 1u;
    int ng = 0;
    for (int base = 0; base < nxy; base += 32) {
        int j = base + lane;
        int cell = 0, cnt = 0;
        if (j < nxy) {
            int jx = j % R.span[0], jy = j / R.span[0];
            int x = (R.span[0] == R.nc[0]) ? jx : wrapi(pcx - R.range + jx, R.nc[0]);
            int y = (R.span[1] == R.nc[1]) ? jy : wrapi(pcy - R.range + jy, R.nc[1]);
            cell = (z * R.nc[1] + y) * R.nc[0] + x;
            cnt = R.cell_count[cell];
        }
        int maxc = __reduce_max_sync(kFull, cnt);
        for (int e = 0; e < maxc; ++e) {
            bool inc = false;
            uint32_t packed = 0;
            if (e < cnt) {
                int g = R.cell_ent[cell * R.cap + e];
                if (g != self) {
                    float4 gc = R.gcen[g];
                    inc = within_cutoff<false>(cx, cy, cz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                               R.cut2_hi, R.fast_incl);
                    if (inc) {
                        // image of the group relative to the pose (same rounding as dist_group)
                        float rx = fast_round(fdiv(fsub(gc.x, cx), R.L[0]));
                        float ry = fast_round(fdiv(fsub(gc.y, cy), R.L[1]));
                        float rz = fast_round(fdiv(fsub(gc.z, cz), R.L[2]));
                        if (R.pair_image) {
                            packed = (uint32_t)g;
                        } else if (fabsf(rx) > 1.0f || fabsf(ry) > 1.0f || fabsf(rz) > 1.0f) {
                            atomicOr(R.err, ERR_IMAGE);
                            inc = false;
                        } else {
                            uint32_t code = (rx > 0.0f ? 1u : (rx < 0.0f ? 2u : 0u)) |
                                            ((ry > 0.0f ? 1u : (ry < 0.0f ? 2u : 0u)) << 2) |
                                            ((rz > 0.0f ? 1u : (rz < 0.0f ? 2u : 0u)) << 4);
                            packed = (uint32_t)g | (code << 26);
                        }
                    }
                }
            }
            unsigned m = __ballot_sync(kFull, inc);
            if (inc) B.glist[ng + __popc(m & lt)] = packed;
            ng += __popc(m);
            ngroups += __popc(m);
            if (ng > kGCap - 32) {
                __syncwarp();
                process_groups(R, B, ng, ns, lane, (double)cx, (double)cy, (double)cz, acc, npair);
                ng = 0;
            }
        }
    }
    __syncwarp();
    process_groups(R, B, ng, ns, lane, (double)cx, (double)cy, (double)cz, acc, npair);
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
    U4 r = rng(R.seed, R.replica, (uint32_t)D.step, (uint32_t)i, RP_MOVE, 0);
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

// Load the pose of item (i, variant v) of step D into B.site; returns the
// pose centre and the residue to skip.
__device__ __forceinline__ void build_pose(const RepDev& R, const StepDesc& D, int i, int v, WarpBuf& B,
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
            B.site[lane] = make_float4((float)((double)sx - (double)cx), (float)((double)sy - (double)cy),
                                       (float)((double)sz - (double)cz), kCoulomb * t.w);
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
    if (D.move != MV_DELETE && v == 0) moved_site(R, D, i, gc, ns, lane, px, py, pz);
    if (lane < ns)
        B.site[lane] = make_float4((float)((double)px - (double)cx), (float)((double)py - (double)cy),
                                   (float)((double)pz - (double)cz), kCoulomb * F.site[lane].w);
    __syncwarp();
}

// One launch per MC step: every replica's (pose, variant, slab) items.
__global__ void __launch_bounds__(kWarpsE * 32, 3) k_energy(const RepDev* __restrict__ reps, int nrep) {
    __shared__ WarpBuf bufs[kWarpsE];
    __shared__ int pre[257];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int r = 0; r < nrep; ++r) { pre[r] = acc; acc += reps[r].desc->items; }
        pre[nrep] = acc;
    }
    __syncthreads();
    const int total = pre[nrep];
    WarpBuf& B = bufs[warp];
    for (int it = blockIdx.x * kWarpsE + warp; it < total; it += gridDim.x * kWarpsE) {
        int lo = 0, hi = nrep;  // find r with pre[r] <= it < pre[r+1]
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (pre[mid] <= it) lo = mid; else hi = mid; }
        const RepDev& R = reps[lo];
        const StepDesc D = *R.desc;
        const int local = it - pre[lo];
        const int per_pose = D.nvar * D.nslab;
        const int i = local / per_pose;
        const int rem = local - i * per_pose;
        const int v = rem / D.nslab, z = rem - v * D.nslab;
        float cx, cy, cz;
        int self;
        build_pose(R, D, i, v, B, lane, cx, cy, cz, self);
        double acc = 0.0;
        int ng = 0;
        long long npair = 0;
        energy_slab(R, B, R.frag[D.ftype].nsites, cx, cy, cz, self, z, lane, acc, ng, npair);
        acc = warp_sum(acc);
        if (lane == 0) {
            R.epart[(i * D.nvar + v) * D.nslab + z] = acc;
            atomicAdd(&R.counters[2], (unsigned long long)npair);
        }
        if (v == 0 && D.nw > 0) {  // this slab's share of the neighbour row of pose i
            const int w0 = z * D.nw / D.nslab, w1 = (z + 1) * D.nw / D.nslab;
            const float4 ci = R.pcen[i];
            for (int w = w0; w < w1; ++w) {
                int j = 32 * w + lane;
                bool b = false;
                if (j < D.k) {
                    float4 cj = R.pcen[j];
                    b = within_cutoff<true>(ci.x, ci.y, ci.z, cj.x, cj.y, cj.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                            R.cut2_hi, R.fast_incl);
                }
                unsigned m = __ballot_sync(kFull, b);
                if (lane == 0) R.nbr[i * D.nw + w] = m;
            }
        }
        __syncwarp();
    }
}

// Energies of caller-supplied poses (gcmc_energy_poses): item = (pose, slab).
__global__ void __launch_bounds__(kWarpsE * 32)
    k_energy_explicit(const RepDev* __restrict__ rep, const float* __restrict__ xyz,
                      const float* __restrict__ q, const int* __restrict__ type, int ns,
                      const float* __restrict__ centres, const int* __restrict__ self, int nposes,
                      int nslab, double* __restrict__ out, int* __restrict__ ngout) {
    __shared__ WarpBuf bufs[kWarpsE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const RepDev& R = *rep;
    WarpBuf& B = bufs[warp];
    const int total = nposes * nslab;
    for (int it = blockIdx.x * kWarpsE + warp; it < total; it += gridDim.x * kWarpsE) {
        const int p = it / nslab, z = it - p * nslab;
        if (lane < ns) {
            const float* s = xyz + ((size_t)p * ns + lane) * 3;
            const double c0 = centres[3 * p], c1 = centres[3 * p + 1], c2 = centres[3 * p + 2];
            B.site[lane] = make_float4((float)((double)s[0] - c0), (float)((double)s[1] - c1),
                                       (float)((double)s[2] - c2), kCoulomb * q[lane]);
            B.srow[lane] = type[lane] * R.ffY;
        }
        __syncwarp();
        double acc = 0.0;
        int ng = 0;
        long long npair = 0;
        energy_slab(R, B, ns, centres[3 * p], centres[3 * p + 1], centres[3 * p + 2], self ? self[p] : -1, z,
                    lane, acc, ng, npair);
        acc = warp_sum(acc);
        if (lane == 0) {
            out[it] = acc;
            ngout[it] = ng;
        }
        __syncwarp();
    }
}

}  // namespace gcmc
