// Tiled pose-energy kernel: calcEnergy (gcmc/cpp/gcmc_energy.h:142-204) for all
// of a step's trial poses, organised around the environment they share.
//
// The step's pose entries (pose i, variant v: the new pose, and for a
// translate / rotate also the old one; a translate / rotate step in the
// pairwise-difference form has one entry per pose for both) are binned by the
// preparation kernel (bin_entries) into pose blocks of B x B x B cells of the
// cell grid, and each block into work items ("tiles") of at most kTilePoses
// entries.  One CTA per tile:
//   1. builds the tile's poses (one warp each; insertion poses from the RNG,
//      moved poses from the slot's atoms), keeping new-variant sites for the
//      accept kernel;
//   2. stages the block's window -- the cells within R cells of the block
//      (R + margin for a translate step, whose new centres lie within margin
//      cells of the old ones), which hold every group within the cutoff of any
//      pose in it -- into
//      shared memory: the window's cell counts, the cells' records (group
//      centre, id, atom range) and then the groups' atoms (x, y, z, charge,
//      type), coalesced, once for all the tile's poses (windows larger than the
//      staging buffers are staged in rounds);
//   3. evaluates every pose against the staged groups: warps split the poses,
//      and when the tile has fewer poses than warps, each pose's groups (a
//      fixed split given the pose count), testing every staged centre with the
//      bit-exact FP32 inclusion distance, compacting the included groups
//      (ballot) and their atoms, and evaluating atom x site pairs with the
//      packed FP32 arithmetic of flush_atoms_packed, or of dual_atom_e for a
//      pose pair in the difference form (atoms and the pair table read from
//      shared memory);
//   4. sums each pose's per-warp FP64 partials in warp order into epart (one
//      entry per pose variant) and, for clustering moves, fills the tile's
//      poses' rows of the pose-pose bit matrix and the per-pose draws.
// Energies depend only on the state and the entry count of the pose's block
// (the staging order is the cells' sorted order, and every tile of a block
// splits its poses' groups alike), so the speculative and the sequential
// evaluation of a step are bit-identical.
#pragma once
#include "energy.cuh"

namespace gcmc {

constexpr int kWarpsT = 16;       // warps per tile CTA
constexpr int kTilePoses = 16;    // pose entries per tile at most
constexpr int kTileAtoms = 5120;  // atoms staged per round
constexpr int kTileGroups = 1024; // group records staged per round
constexpr int kTileCells = 1024;  // window cells at most
constexpr int kTileLJ = 2048;     // pair-table entries kept in shared memory (larger tables: global)
constexpr int kTileGList = 128;   // per-warp included-group buffer
constexpr int kTileAList = 256;   // per-warp included-atom buffer
constexpr int kTileMaxGroupAtoms = kTileAtoms / 4;  // groups larger than this are not tiled
constexpr int kMaxBlocks = 4096;  // pose blocks per replica at most
constexpr int kBinScratchBytes = 2 * kMaxBlocks * (int)sizeof(int);

struct PoseBuf {
    float4 site[kMaxSites];  // x, y, z relative to the pose centre, Coulomb constant * charge
    int srow[kMaxSites];     // template type * ffY
    SitePair spair[kMaxSites / 2];
    DualSite dsite[kMaxSites];  // dual entries: both poses' sites in the difference form
    float cs_hi[3][4];       // pose centre + image shift, high part and TwoSum error
    float cs_lo[3][4];
    float4 site_abs[kMaxSites];
    float cx, cy, cz;        // pose centre (dual: the old one)
    float nx, ny, nz;        // dual: the new centre, exact
    float ux, uy, uz;        //   and in the old centre's periodic frame
    int self;
};

struct TileSmem {
    float4 atom[kTileAtoms];       // staged atoms: x, y, z, charge
    float4 gc[kTileGroups];        // staged groups: centre, w = group id bits
    int2 gs[kTileGroups];          // staged groups: (first staged atom, atom count)
    int2 gsrc[kTileGroups];        // staged groups: (atomStart, atomNum) in the state
    float2 lj[kTileLJ];            // pair table (100 sigma^2, 4 eps)
    PoseBuf pose[kTilePoses];
    uint2 glist[kWarpsT][kTileGList];      // included group: (staged start | image code << 26, count)
    uint32_t alist[kWarpsT][kTileAList];   // staged atom | image code << 26
    double part[kTilePoses][kWarpsT];      // per-pose, per-part FP64 partial sums
    int cell[kTileCells];          // window cells
    int cpre[kTileCells + 1];      // exclusive prefix of their record counts
    short atype[kTileAtoms];       // staged atoms' types
    int entry[kTilePoses];
    long long npair[kWarpsT];
    int wtot[32];
    int flag;
};

// Exclusive prefix sum over a[0, n) in place (whole block); returns the total.
__device__ __forceinline__ int block_excl_scan(int* a, int n, int* wtot) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int per = (n + nt - 1) / nt, lo = min(n, tid * per), hi = min(n, lo + per);
    int s = 0;
    for (int x = lo; x < hi; ++x) s += a[x];
    int inc = s;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(kFull, inc, off);
        if (lane >= off) inc += t;
    }
    if (lane == 31) wtot[warp] = inc;
    __syncthreads();
    int before = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
        const int t = wtot[w];
        if (w < warp) before += t;
        tot += t;
    }
    int run = before + inc - s;
    for (int x = lo; x < hi; ++x) {
        const int v = a[x];
        a[x] = run;
        run += v;
    }
    __syncthreads();
    return tot;
}

// Pose block of a centre: its cell coordinates divided by the block edge.
__device__ __forceinline__ int pose_block(const RepDev& R, float x, float y, float z) {
    const int bx = cell_coord(x, R.start[0], R.invLc[0], R.nc[0]) / R.tblk;
    const int by = cell_coord(y, R.start[1], R.invLc[1], R.nc[1]) / R.tblk;
    const int bz = cell_coord(z, R.start[2], R.invLc[2], R.nc[2]) / R.tblk;
    return (bz * R.nbk[1] + by) * R.nbk[0] + bx;
}

// Bin the step's pose entries (e = i * nvar + v) by pose block and cut each
// block's entries into tiles of at most kTilePoses: R.pbin (entries by block),
// R.tiles (block, first entry in pbin, count).  Whole CTA; scratch: 2 x
// kMaxBlocks ints of shared memory.  Returns the tile count.  The order of the
// entries within a block follows the atomic ranks and does not matter: every
// entry of a block is evaluated against the same staged window.
__device__ int bin_entries(const RepDev& R, const StepDesc& D, int* scratch, int* wtot) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nblk = R.nbk[0] * R.nbk[1] * R.nbk[2];
    const int ne = D.k * D.nvar;
    int* cnt = scratch;
    int* chunks = scratch + kMaxBlocks;
    for (int b = tid; b < nblk; b += nt) cnt[b] = 0;
    __syncthreads();
    constexpr int kPer = (2 * kMaxPoses + 1023) / 1024;
    int myb[kPer > 0 ? kPer : 1], myr[kPer > 0 ? kPer : 1];
    const int startRes = D.move == MV_INSERT ? 0 : R.frag[D.ftype].startRes;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int e = tid + q * nt;
        myb[q] = -1;
        if (e < ne && q * nt < 2 * kMaxPoses) {
            const int i = e / D.nvar, v = e - i * D.nvar;
            if (D.dual && v == 1) continue;  // dual: one entry per pose (v = 0), binned by its old centre
            float4 c;
            if (D.move == MV_INSERT || D.move == MV_DELETE || (v == 0 && !D.dual)) c = R.pcen[i];
            else c = R.gcen[startRes + R.pslot[i]];  // old pose of a translate / rotate
            myb[q] = pose_block(R, c.x, c.y, c.z);
            myr[q] = atomicAdd(&cnt[myb[q]], 1);
        }
    }
    __syncthreads();
    for (int b = tid; b < nblk; b += nt) chunks[b] = (cnt[b] + kTilePoses - 1) / kTilePoses;
    __syncthreads();
    // entries by block: cnt becomes each block's first entry
    const int nbinned = block_excl_scan(cnt, nblk, wtot);
    const int ntiles = block_excl_scan(chunks, nblk, wtot);
#pragma unroll
    for (int q = 0; q < kPer; ++q)
        if (myb[q] >= 0) R.pbin[cnt[myb[q]] + myr[q]] = tid + q * nt;
    // a block of c entries becomes ceil(c / kTilePoses) tiles of near-equal size, all
    // evaluated with the warp split of the largest (w = its entry count): a pose's
    // energy then depends on its block's entry count only, not on which tile the
    // atomic ranks above put it in
    for (int b = tid; b < nblk; b += nt) {
        const int first = cnt[b], end = (b + 1 < nblk) ? cnt[b + 1] : nbinned, c = end - first;
        if (c == 0) continue;
        const int nt_b = (c + kTilePoses - 1) / kTilePoses, base = c / nt_b, extra = c - base * nt_b;
        const int pmax = base + (extra > 0 ? 1 : 0);
        for (int j = 0; j < nt_b; ++j)
            R.tiles[chunks[b] + j] = make_int4(b, first + j * base + min(j, extra), base + (j < extra ? 1 : 0), pmax);
    }
    __syncthreads();
    return ntiles;
}

// Pair energies of the staged atoms in alist[0, na) with pose P: the
// arithmetic of flush_atoms_packed, with atoms and the pair table read from
// shared memory.
template <bool PairImage>
__device__ __forceinline__ void flush_staged(const RepDev& R, const TileSmem& T, const PoseBuf& P,
                                             const uint32_t* alist, int na, int ns, int lane, const float2* lj,
                                             double& acc) {
    const int np = ns >> 1;
    const float2 mhalf = make_float2(-0.5f, -0.5f), three_half = make_float2(1.5f, 1.5f);
    for (int f = lane; f < na; f += 32) {
        const uint32_t u = alist[f];
        const int idx = (int)(u & 0x3FFFFFFu);
        const float4 a = T.atom[idx];
        const int ta = T.atype[idx];
        uint32_t c0, c1, c2;
        if (PairImage) {
            const float kx = rintf((a.x - P.cs_hi[0][0]) * R.invL[0]);
            const float ky = rintf((a.y - P.cs_hi[1][0]) * R.invL[1]);
            const float kz = rintf((a.z - P.cs_hi[2][0]) * R.invL[2]);
            c0 = kx > 0.0f ? 1u : (kx < 0.0f ? 2u : 0u);
            c1 = ky > 0.0f ? 1u : (ky < 0.0f ? 2u : 0u);
            c2 = kz > 0.0f ? 1u : (kz < 0.0f ? 2u : 0u);
        } else {
            const uint32_t code = u >> 26;
            c0 = code & 3u; c1 = (code >> 2) & 3u; c2 = (code >> 4) & 3u;
        }
        const float ax = (a.x - P.cs_hi[0][c0]) - P.cs_lo[0][c0];
        const float ay = (a.y - P.cs_hi[1][c1]) - P.cs_lo[1][c1];
        const float az = (a.z - P.cs_hi[2][c2]) - P.cs_lo[2][c2];
        const float2 Ax = make_float2(ax, ax), Ay = make_float2(ay, ay), Az = make_float2(az, az);
        const float2 Aq = make_float2(a.w, a.w);
        float2 e2 = make_float2(0.0f, 0.0f);
#pragma unroll 2
        for (int p = 0; p < np; ++p) {
            const SitePair sp = P.spair[p];
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
            const float2 p0 = lj[P.srow[2 * p] + ta];
            const float2 p1 = lj[P.srow[2 * p + 1] + ta];
            const float2 s2 = __fmul2_rn(make_float2(p0.x, p1.x), ir2);
            const float2 s6 = __fmul2_rn(__fmul2_rn(s2, s2), s2);
            e2 = __ffma2_rn(make_float2(p0.y, p1.y), __ffma2_rn(s6, s6, make_float2(-s6.x, -s6.y)), e2);
            e2 = __ffma2_rn(__fmul2_rn(sp.kq, Aq), ir, e2);
        }
        float e = e2.x + e2.y;
        if (ns & 1) {  // last site of an odd count
            const float4 sp = P.site[ns - 1];
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
            const float2 pp = lj[P.srow[ns - 1] + ta];
            const float s2 = pp.x * ir2;
            const float s6 = s2 * s2 * s2;
            e = fmaf(pp.y, fmaf(s6, s6, -s6), e);
            e = fmaf(sp.w * a.w, ir, e);
        }
        acc += (double)e;
    }
}

// Energy changes of the staged atoms in alist[0, na) with the dual pose P
// (atoms: staged index in bits 0-23, inclusion flags in bits 24-25, image
// code in bits 26-31).
template <bool PairImage>
__device__ __forceinline__ void flush_staged_dual(const RepDev& R, const TileSmem& T, const PoseBuf& P,
                                                  const uint32_t* alist, int na, int ns, int lane, const float2* lj,
                                                  double& acc) {
    for (int f = lane; f < na; f += 32) {
        const uint32_t u = alist[f];
        const int idx = (int)(u & 0xFFFFFFu);
        const float4 a = T.atom[idx];
        const int ta = T.atype[idx];
        uint32_t c0, c1, c2;
        if (PairImage) {
            const float kx = rintf((a.x - P.cs_hi[0][0]) * R.invL[0]);
            const float ky = rintf((a.y - P.cs_hi[1][0]) * R.invL[1]);
            const float kz = rintf((a.z - P.cs_hi[2][0]) * R.invL[2]);
            c0 = kx > 0.0f ? 1u : (kx < 0.0f ? 2u : 0u);
            c1 = ky > 0.0f ? 1u : (ky < 0.0f ? 2u : 0u);
            c2 = kz > 0.0f ? 1u : (kz < 0.0f ? 2u : 0u);
        } else {
            const uint32_t code = u >> 26;
            c0 = code & 3u; c1 = (code >> 2) & 3u; c2 = (code >> 4) & 3u;
        }
        const float ax = (a.x - P.cs_hi[0][c0]) - P.cs_lo[0][c0];
        const float ay = (a.y - P.cs_hi[1][c1]) - P.cs_lo[1][c1];
        const float az = (a.z - P.cs_hi[2][c2]) - P.cs_lo[2][c2];
        acc += (double)dual_atom_e<PairImage>(R, P.dsite, P.srow, ns, ax, ay, az, a.w, ta, (u >> 24) & 3u, lj);
    }
}

// Expand the included groups glist[0, ng) into staged-atom entries and
// evaluate them (warp-collective; the staged form of process_groups).
template <bool PairImage, bool Dual>
__device__ __forceinline__ void flush_any(const RepDev& R, const TileSmem& T, const PoseBuf& P, const uint32_t* alist,
                                          int na, int ns, int lane, const float2* lj, double& acc) {
    if (Dual) flush_staged_dual<PairImage>(R, T, P, alist, na, ns, lane, lj, acc);
    else flush_staged<PairImage>(R, T, P, alist, na, ns, lane, lj, acc);
}

template <bool PairImage, bool Dual>
__device__ __forceinline__ void process_staged(const RepDev& R, TileSmem& T, const PoseBuf& P, int warp, int ng,
                                               int ns, int lane, const float2* lj, double& acc, long long& npair) {
    uint32_t* alist = T.alist[warp];
    const uint2* glist = T.glist[warp];
    int na = 0;
    for (int base = 0; base < ng; base += 32) {
        const int gi = base + lane;
        int start = 0, cnt = 0;
        uint32_t code = 0;
        if (gi < ng) {
            const uint2 ge = glist[gi];
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
        npair += (long long)total * ns;
        const int maxcnt = __reduce_max_sync(kFull, (unsigned)cnt);
        if (maxcnt <= kTileAList / 2) {
            if (na + total > kTileAList) {
                __syncwarp();
                flush_any<PairImage, Dual>(R, T, P, alist, na, ns, lane, lj, acc);
                __syncwarp();
                na = 0;
            }
            if (total <= kTileAList) {
                const int off0 = na + incl - cnt;
                for (int j = 0; j < cnt; ++j) alist[off0 + j] = (uint32_t)(start + j) | (code << 26);
                na += total;
                continue;
            }
        }
        for (int l = 0; l < 32; ++l) {  // large groups: one at a time, in buffer-sized pieces
            const int s0 = __shfl_sync(kFull, start, l), c0 = __shfl_sync(kFull, cnt, l);
            const uint32_t cd = __shfl_sync(kFull, code, l);
            int done = 0;
            while (done < c0) {
                const int take = min(c0 - done, kTileAList - na);
                if (take == 0) {
                    __syncwarp();
                    flush_any<PairImage, Dual>(R, T, P, alist, na, ns, lane, lj, acc);
                    __syncwarp();
                    na = 0;
                    continue;
                }
                for (int j = lane; j < take; j += 32) alist[na + j] = (uint32_t)(s0 + done + j) | (cd << 26);
                na += take;
                done += take;
            }
        }
    }
    __syncwarp();
    flush_any<PairImage, Dual>(R, T, P, alist, na, ns, lane, lj, acc);
    __syncwarp();
}

// Pose P against the staged groups [g0, g1) (warp-collective).  Dual: every
// group within the cutoff of either centre, with its inclusion flags, listed
// as in walk_cells.
template <bool PairImage, bool Dual>
__device__ __forceinline__ void eval_staged(const RepDev& R, TileSmem& T, const PoseBuf& P, int warp, int g0, int g1,
                                            int ns, int lane, const float2* lj, double& acc, long long& npair) {
    uint2* glist = T.glist[warp];
    const unsigned lt = (1u << lane) - 1u;
    int ng = 0;
    long long both_atoms = 0;
    for (int base = g0; base < g1; base += 32) {
        const int gi = base + lane;
        bool inc = false, inc2 = false;
        uint2 packed = make_uint2(0u, 0u), packed2 = make_uint2(0u, 0u);
        if (Dual && gi < g1) {
            const float4 gc = T.gc[gi];
            if (__float_as_int(gc.w) != P.self) {
                const bool io = within_cutoff<false>(P.cx, P.cy, P.cz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff,
                                                     R.cut2_lo, R.cut2_hi, R.fast_incl);
                const bool in = within_cutoff<false>(P.nx, P.ny, P.nz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff,
                                                     R.cut2_lo, R.cut2_hi, R.fast_incl);
                uint32_t co = 0u, cn = 0u;
                bool bo = false, bn = false;
                if (!PairImage) {
                    if (io) co = image_code(R, gc.x, gc.y, gc.z, P.cx, P.cy, P.cz, &bo);
                    if (in) cn = image_code(R, gc.x, gc.y, gc.z, P.ux, P.uy, P.uz, &bn);
                }
                if (bo || bn) {
                    atomicOr(R.err, ERR_IMAGE);
                } else if (io || in) {
                    const int2 sg = T.gs[gi];
                    const bool split = io && in && co != cn;
                    const uint32_t fl1 = split ? 1u : ((io ? 1u : 0u) | (in ? 2u : 0u));
                    inc = true;
                    packed = make_uint2((uint32_t)sg.x | (fl1 << 24) | ((io ? co : cn) << 26), (uint32_t)sg.y);
                    if (split) {
                        inc2 = true;
                        packed2 = make_uint2((uint32_t)sg.x | (2u << 24) | (cn << 26), (uint32_t)sg.y);
                    }
                    if (fl1 == 3u) both_atoms += sg.y;
                }
            }
        } else if (gi < g1) {
            const float4 gc = T.gc[gi];
            if (__float_as_int(gc.w) != P.self) {
                inc = within_cutoff<false>(P.cx, P.cy, P.cz, gc.x, gc.y, gc.z, R.L, R.invL, R.cutoff, R.cut2_lo,
                                           R.cut2_hi, R.fast_incl);
                if (inc) {
                    const int2 sg = T.gs[gi];
                    packed = make_uint2((uint32_t)sg.x, (uint32_t)sg.y);
                    if (!PairImage) {  // the group's periodic image relative to the pose centre
                        const float rx = rintf((gc.x - P.cx) * R.invL[0]);
                        const float ry = rintf((gc.y - P.cy) * R.invL[1]);
                        const float rz = rintf((gc.z - P.cz) * R.invL[2]);
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
        if (inc) glist[ng + __popc(m & lt)] = packed;
        ng += __popc(m);
        if (Dual) {
            const unsigned m2 = __ballot_sync(kFull, inc2);
            if (inc2) glist[ng + __popc(m2 & lt)] = packed2;
            ng += __popc(m2);
        }
        if (ng > kTileGList - (Dual ? 64 : 32)) {
            __syncwarp();
            process_staged<PairImage, Dual>(R, T, P, warp, ng, ns, lane, lj, acc, npair);
            ng = 0;
        }
    }
    __syncwarp();
    process_staged<PairImage, Dual>(R, T, P, warp, ng, ns, lane, lj, acc, npair);
    if (Dual) npair += (long long)__reduce_add_sync(kFull, (unsigned)both_atoms) * ns;
}

// A speculative evaluation that has become void (the accept kernel of the step
// before accepted a move) ends at its next check; whole block.
__device__ __forceinline__ bool tile_voided(const RepDev& R, const StepDesc& D, int mode, TileSmem& T) {
    if (mode != 1) return false;
    __syncthreads();
    if (threadIdx.x == 0) T.flag = *reinterpret_cast<const volatile int*>(R.abort) == D.step;
    __syncthreads();
    return T.flag != 0;
}

// One tile (whole block).
template <bool PairImage>
__device__ void tile_item(const RepDev& R, const StepDesc& D, int li, TileSmem& T, int mode, bool sym) {
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
    if (tile_voided(R, D, mode, T)) return;
    const int4 tile = R.tiles[li];
    const int b = tile.x, P = tile.z;
    if (tid < P) T.entry[tid] = R.pbin[tile.y + tid];
    // window cells: the block's cells and R (+ margin) cells around them
    const int nb01 = R.nbk[0] * R.nbk[1];
    const int bz = b / nb01, bxy = b - bz * nb01, by = bxy / R.nbk[0], bx = bxy - by * R.nbk[0];
    const int reach = R.range + D.margin;
    const int o[3] = {bx * R.tblk - reach, by * R.tblk - reach, bz * R.tblk - reach};
    const int W0 = min(R.tblk + 2 * reach, R.nc[0]), W1 = min(R.tblk + 2 * reach, R.nc[1]);
    const int W2 = min(R.tblk + 2 * reach, R.nc[2]), W01 = W0 * W1;
    const int nwin = W01 * W2;
    for (int t = tid; t < nwin; t += nt) {
        const int jz = t / W01, jxy = t - jz * W01, jy = jxy / W0, jx = jxy - jy * W0;
        const int x = (W0 == R.nc[0]) ? jx : wrapi(o[0] + jx, R.nc[0]);
        const int y = (W1 == R.nc[1]) ? jy : wrapi(o[1] + jy, R.nc[1]);
        const int z = (W2 == R.nc[2]) ? jz : wrapi(o[2] + jz, R.nc[2]);
        const int cell = (z * R.nc[1] + y) * R.nc[0] + x;
        T.cell[t] = cell;
        T.cpre[t] = min(R.cell_count[cell], R.cap);
    }
    const int nlj = R.ffX * R.ffY;
    const bool lj_smem = nlj <= kTileLJ;
    if (lj_smem)
        for (int x = tid; x < nlj; x += nt) T.lj[x] = R.lj[x];
    __syncthreads();
    // the tile's poses, one warp each (overlapping the count loads above)
    const int ns = R.frag[D.ftype].nsites;
    for (int p = warp; p < P; p += kWarpsT) {
        const int e = T.entry[p];
        const int i = e / D.nvar, v = e - i * D.nvar;
        PoseBuf& Pb = T.pose[p];
        float cx, cy, cz;
        int self;
        if (D.dual) {
            DualCentre dc;
            build_pose_dual(R, D, i, Pb, lane, cx, cy, cz, dc, self);
            if (lane == 0) {
                Pb.nx = dc.nx; Pb.ny = dc.ny; Pb.nz = dc.nz;
                Pb.ux = dc.ux; Pb.uy = dc.uy; Pb.uz = dc.uz;
            }
        } else {
            build_pose(R, D, i, v, Pb, lane, cx, cy, cz, self);
        }
        keep_sites(R, D, Pb, i, v, 0, lane);
        set_centre(R, Pb, cx, cy, cz, lane);
        if (lane == 0) {
            Pb.cx = cx;
            Pb.cy = cy;
            Pb.cz = cz;
            Pb.self = self;
        }
    }
    const int nrec = block_excl_scan(T.cpre, nwin, T.wtot);
    if (tid == 0) T.cpre[nwin] = nrec;
    // warp w evaluates pose w / S over part w % S of each round's groups; S follows the
    // block's largest tile (tile.w), so every tile of a block splits its poses alike
    const int S = max(1, kWarpsT / max(1, tile.w));
    const int mp = warp / S, mj = warp - mp * S;
    const bool active = mp < P;
    double acc = 0.0;
    long long npair = 0;
    const float2* lj = lj_smem ? T.lj : R.lj;
    for (int r0 = 0; r0 < nrec;) {
        const int nr = min(nrec - r0, kTileGroups);
        // records r0 .. r0 + nr (cell by binary search over the prefix); their atom
        // counts go to an int scratch (the alist area, free between evaluations)
        int* cnts = reinterpret_cast<int*>(&T.alist[0][0]);
        for (int q = tid; q < nr; q += nt) {
            const int rec = r0 + q;
            int lo = 0, hi = nwin - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (T.cpre[mid] <= rec) lo = mid; else hi = mid - 1;
            }
            const CellEnt* ce = R.cell_ent + (size_t)T.cell[lo] * R.cap + (rec - T.cpre[lo]);
            const float4 c = ce->c;
            int2 sp = ce->span;
            sp.y = min(max(sp.y, 0), kTileMaxGroupAtoms);
            T.gc[q] = c;
            T.gsrc[q] = sp;
            cnts[q] = sp.y;
        }
        __syncthreads();
        block_excl_scan(cnts, nr, T.wtot);
        // the round takes the longest prefix of records whose atoms fit (offsets are monotone)
        if (tid == 0) T.flag = 0;
        int fit_local = 0;
        for (int q = tid; q < nr; q += nt) {
            const int off = cnts[q], c = T.gsrc[q].y;
            T.gs[q] = make_int2(off, c);
            fit_local += (off + c <= kTileAtoms) ? 1 : 0;
        }
        __syncthreads();
        if (fit_local) atomicAdd(&T.flag, fit_local);
        __syncthreads();
        const int nfit = T.flag;
        // atoms of records [0, nfit): a warp per record, lanes over its atoms
        for (int q = warp; q < nfit; q += kWarpsT) {
            const int2 src = T.gsrc[q];
            const int dst = T.gs[q].x;
            for (int a = lane; a < src.y; a += 32) {
                T.atom[dst + a] = R.xyzq[src.x + a];
                T.atype[dst + a] = (short)R.atype[src.x + a];
            }
        }
        __syncthreads();
        if (active) {
            const int g0 = mj * nfit / S, g1 = (mj + 1) * nfit / S;
            if (D.dual) eval_staged<PairImage, true>(R, T, T.pose[mp], warp, g0, g1, ns, lane, lj, acc, npair);
            else eval_staged<PairImage, false>(R, T, T.pose[mp], warp, g0, g1, ns, lane, lj, acc, npair);
        }
        r0 += nfit;
        if (tile_voided(R, D, mode, T)) return;
        __syncthreads();
        if (nfit == 0) break;  // cannot happen: a single group's atoms always fit
    }
    acc = warp_sum(acc);
    if (lane == 0) {
        if (active) T.part[mp][mj] = acc;
        T.npair[warp] = active ? npair : 0;
    }
    __syncthreads();
    if (tid < P) {
        double e = 0.0;
        for (int j = 0; j < S; ++j) e += T.part[tid][j];
        R.epart[T.entry[tid]] = e;
        if (D.dual) R.epart[T.entry[tid] + 1] = 0.0;  // the old variant's share of the change
    }
    if (tid == 0) {
        long long np = 0;
        for (int w = 0; w < kWarpsT; ++w) np += T.npair[w];
        atomicAdd(mode == 1 ? R.pairs_pending : &R.counters[2], (unsigned long long)np);
    }
    // clustering moves: the bit matrix and the per-pose draws
    if (D.nw > 0) {
        if (sym) {
            const int ntask = D.nw * (D.nw + 1) / 2;
            for (int q = li * kWarpsT + warp; q < ntask; q += D.items * kWarpsT) nbr_block(R, D, q, lane);
        } else {
            for (int p = warp; p < P; p += kWarpsT) {
                const int e = T.entry[p];
                const int i = e / D.nvar, v = e - i * D.nvar;
                if (v == 0) nbr_rows(R, D, i, 0, 1, lane);
            }
        }
    }
    __syncthreads();
}

// One launch per MC step: every replica's tiles, one CTA per tile (a grid
// stride loop over them).  mode as k_energy_t: 0 every tile; 1 speculative
// (pairs into pairs_pending, ends early once voided); 2 completion (nothing
// if the speculative evaluation stands).
__global__ void __launch_bounds__(kWarpsT * 32, 1) k_energy_tiles(const RepDev* __restrict__ reps, int nrep,
                                                                  int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem& T = *reinterpret_cast<TileSmem*>(smem_raw);
    __shared__ int pre[257];
    if (mode == 2 && *reps[0].valid) return;
    items_prefix(nrep, pre, T.wtot, [&](int r) { return reps[r].desc->items; });
    const int total = pre[nrep];
    const bool sym = total > (int)gridDim.x;  // more tiles than CTAs: throughput-bound
    for (int it = blockIdx.x; it < total; it += gridDim.x) {
        int lo = 0, hi = nrep;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (pre[mid] <= it) lo = mid; else hi = mid;
        }
        const RepDev& R = reps[lo];
        const StepDesc D = *R.desc;
        if (R.pair_image) tile_item<true>(R, D, it - pre[lo], T, mode, sym);
        else tile_item<false>(R, D, it - pre[lo], T, mode, sym);
    }
}

}  // namespace gcmc
