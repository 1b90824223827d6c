// Backward of the pose energy: gradients of E(pose) with respect to the site
// coordinates, the site charges and the LJ pair table, for explicit poses.
//
// Same cell walk and group inclusion as the pose-energy kernel (the included
// atoms reach this sink in the same buffers); the pair arithmetic of each
// (site, atom) term is the forward's (centre-relative offsets, rsqrt + one
// Newton step, s6 = (sigma2 / r2)^3) followed by its analytic derivatives:
//   G      = dU/dr2   = -(3 E4 (2 s6^2 - s6) + U_el / 2) / r2
//   dU/dx_s           = -2 G d             (d = atom - site)
//   dU/dq_s           = K q_a / r
//   dU/dsigma2        = 3 E4 s2^2 (2 s6 - 1) / r2      (sigma2 = 100 sigma^2)
//   dU/dE4            = s6^2 - s6                      (E4 = 4 eps)
// Lanes are (site, atom subset) pairs: lane = sub * ns + s with
// nsub = 32 / ns subsets, so each lane keeps its site's four gradient sums in
// registers while it walks its share of a staged batch of atoms; the subsets
// are summed in a fixed order at the end of the item.  Table gradients,
// weighted by the caller's dL/dE of the pose, go to a per-block shared array
// [ns][ffY][2] and from there to global FP64 sums.
#pragma once
#include "energy.cuh"

namespace gcmc {

constexpr int kWarpsG = 4;
constexpr int kGStage = 128;

struct GradStage {
    float4 a[kGStage];  // atom offset from the pose centre (x, y, z), charge
    int t[kGStage];     // atom type
    float4 red[32];     // per-lane site sums for the end-of-item reduction
};

template <bool WithE>
struct GradSinkT {
    GradStage* st;
    float* gtab;   // block shared [ns][ffY][2] (nullptr: no table gradient)
    float w;       // dL/dE of the current pose
    int ffY;
    float gx = 0.f, gy = 0.f, gz = 0.f, gq = 0.f;
    float e = 0.f;  // WithE: this lane's FP32 sum of its pair energies

    template <bool PairImage>
    __device__ __forceinline__ void flush_t(const RepDev& R, WarpBuf& B, int na, int ns, int lane) {
        const int s = lane % ns, sub = lane / ns, nsub = 32 / ns;
        const bool active = sub < nsub;
        float4 sp = make_float4(0.f, 0.f, 0.f, 0.f);
        int row = 0;
        if (active) {
            sp = B.site[s];
            row = B.srow[s];
        }
        for (int base = 0; base < na; base += kGStage) {
            const int m = min(kGStage, na - base);
            for (int f = lane; f < m; f += 32) {  // stage: the forward's centre-relative offsets
                const uint32_t u = B.alist[base + f];
                const int idx = (int)(u & 0x3FFFFFFu);
                const float4 a = __ldg(&R.xyzq[idx]);
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
                st->a[f] = make_float4((a.x - B.cs_hi[0][c0]) - B.cs_lo[0][c0],
                                       (a.y - B.cs_hi[1][c1]) - B.cs_lo[1][c1],
                                       (a.z - B.cs_hi[2][c2]) - B.cs_lo[2][c2], a.w);
                st->t[f] = __ldg(&R.atype[idx]);
            }
            __syncwarp();
            if (active) {
                for (int f = sub; f < m; f += nsub) {
                    const float4 a = st->a[f];
                    const int ta = st->t[f];
                    float dx = a.x - sp.x, dy = a.y - sp.y, dz = a.z - sp.z;
                    if (PairImage) {
                        dx = fmaf(-rintf(dx * R.invL[0]), R.L[0], dx);
                        dy = fmaf(-rintf(dy * R.invL[1]), R.L[1], dy);
                        dz = fmaf(-rintf(dz * R.invL[2]), R.L[2], dz);
                    }
                    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                    float ir = rsqrtf(r2);
                    ir = ir * fmaf(-0.5f * r2 * ir, ir, 1.5f);
                    const float ir2 = ir * ir;
                    const float2 p = __ldg(&R.lj[row + ta]);
                    const float s2 = p.x * ir2;
                    const float s6 = s2 * s2 * s2;
                    float uel = sp.w * a.w * ir;
                    float gel = uel;  // -2 r^2 d(U_el)/d(r^2)
                    float cq = ir;    // d(U_el)/d(K q_s q_a)
                    if (R.pme) {      // Ewald real space: K q q erfc(alpha r) / r
                        const float ar = R.pme_alpha * (r2 * ir);
                        const float ec = erfcf(ar);
                        uel *= ec;
                        cq *= ec;
                        gel = uel + sp.w * a.w * (1.12837917f * R.pme_alpha) * expf(-ar * ar);
                    }
                    const float t6 = fmaf(2.0f * s6, s6, -s6);
                    const float G = -fmaf(3.0f * p.y, t6, 0.5f * gel) * ir2;
                    const float m2 = -2.0f * G;
                    gx = fmaf(m2, dx, gx);  // dU/dx_s = -2 G (atom - site)
                    gy = fmaf(m2, dy, gy);
                    gz = fmaf(m2, dz, gz);
                    gq = fmaf(kCoulomb * a.w, cq, gq);
                    if (WithE) e = fmaf(p.y, fmaf(s6, s6, -s6), e) + uel;
                    if (gtab) {
                        float* g = gtab + ((size_t)s * ffY + ta) * 2;
                        atomicAdd(g, w * (3.0f * p.y * s2 * s2 * ir2 * fmaf(2.0f, s6, -1.0f)));
                        atomicAdd(g + 1, w * fmaf(s6, s6, -s6));
                    }
                }
            }
            __syncwarp();
        }
    }
    __device__ __forceinline__ void flush(const RepDev& R, WarpBuf& B, int na, int ns, int lane) {
        if (R.pair_image) flush_t<true>(R, B, na, ns, lane);
        else flush_t<false>(R, B, na, ns, lane);
    }
};
using GradSink = GradSinkT<false>;

// item = (pose, slab) as in k_energy_explicit; part[(item * ns + s)] =
// (dE/dx, dE/dy, dE/dz, dE/dq) of site s from this slab's atoms.
// Dynamic shared memory: ns * ffY * 2 floats when glj != nullptr.
__global__ void __launch_bounds__(kWarpsG * 32)
    k_energy_grad(const RepDev R, const float* __restrict__ xyz, const float* __restrict__ q,
                  const int* __restrict__ type, int ns, const float* __restrict__ centres,
                  const int* __restrict__ self, int nposes, int nslab, const double* __restrict__ gout,
                  float4* __restrict__ part, double* __restrict__ glj) {
    extern __shared__ float gtab[];
    __shared__ WarpBuf bufs[kWarpsG];
    __shared__ GradStage stages[kWarpsG];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntab = glj ? ns * R.ffY * 2 : 0;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) gtab[i] = 0.0f;
    __syncthreads();
    WarpBuf& B = bufs[warp];
    const int total = nposes * nslab;
    for (int it = blockIdx.x * kWarpsG + warp; it < total; it += gridDim.x * kWarpsG) {
        const int p = it / nslab, z = it - p * nslab;
        if (lane < ns) {
            const float* sx = xyz + ((size_t)p * ns + lane) * 3;
            const double c0 = centres[3 * p], c1 = centres[3 * p + 1], c2 = centres[3 * p + 2];
            B.site[lane] = make_float4((float)((double)sx[0] - c0), (float)((double)sx[1] - c1),
                                       (float)((double)sx[2] - c2), kCoulomb * q[lane]);
            B.srow[lane] = type[lane] * R.ffY;
        }
        __syncwarp();
        GradSink sink;
        sink.st = &stages[warp];
        sink.gtab = glj ? gtab : nullptr;
        sink.w = gout ? (float)gout[p] : 1.0f;
        sink.ffY = R.ffY;
        int ng = 0;
        long long npair = 0;
        const int nwin = R.span[0] * R.span[1] * R.span[2];
        walk_cells(R, B, ns, centres[3 * p], centres[3 * p + 1], centres[3 * p + 2], self ? self[p] : -1,
                   z * nwin / nslab, (z + 1) * nwin / nslab, lane, sink, ng, npair);
        // sum the atom subsets of each site in a fixed order
        stages[warp].red[lane] = make_float4(sink.gx, sink.gy, sink.gz, sink.gq);
        __syncwarp();
        if (lane < ns) {
            const int nsub = 32 / ns;
            float4 acc = stages[warp].red[lane];
            for (int k = 1; k < nsub; ++k) {
                const float4 v = stages[warp].red[k * ns + lane];
                acc.x += v.x; acc.y += v.y; acc.z += v.z; acc.w += v.w;
            }
            part[(size_t)it * ns + lane] = acc;
        }
        __syncwarp();
    }
    __syncthreads();
    if (glj) {  // block sums -> global, rows mapped to the sites' table rows
        for (int i = threadIdx.x; i < ntab; i += blockDim.x) {
            const float v = gtab[i];
            if (v != 0.0f) {
                const int s = i / (2 * R.ffY), rem = i - s * 2 * R.ffY;
                atomicAdd(&glj[(size_t)type[s] * R.ffY * 2 + rem], (double)v);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Pose energies with forces for force-biased translate/rotate steps.
//
// phase 1: items (pose i, slab) of the OLD poses of force-biased steps:
//          energy partial (variant 1) and force/torque partials; the last item
//          of a pose to finish (a per-pose counter after a fence) sums them in
//          slab order and draws the pose's proposal (new centre, d, z).  The
//          ordinary items of the other steps (insert / delete), which depend on
//          no proposal, run here too.
// phase 2: items (pose i, slab) of the NEW poses (variant 0) of force-biased
//          steps, with forces.
// Several replicas: warps take items from a counter per phase (the step
// descriptor of the first replica; the launch's last CTA resets it), which
// balances uneven items; one replica: a fixed stride.
// ---------------------------------------------------------------------------
// (Five CTAs per SM: at most 102 registers a thread, the budget that keeps
// 20 warps per SM resident.)
// Mixed: the replicas' move schedules differ, so that one launch can hold both
// kinds of first-launch items (the SM-affine split below is compiled in only then).
template <bool Mixed>
__global__ void __launch_bounds__(kWarpsG * 32, 5) k_energy_fb(const RepDev* __restrict__ reps, int nrep, int phase) {
    __shared__ WarpBuf bufs[kWarpsG];
    __shared__ GradStage stages[kWarpsG];
    __shared__ int pre[257];
    __shared__ int pre2[257];
    __shared__ int wtot[kWarpsG];
    __shared__ int kinds;  // bit 0: old poses of force-biased steps, bit 1: ordinary items
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // A batch's first launch can hold two kinds of items, the old poses of force-biased
    // steps (gradient sink) and the ordinary items of the other steps: then each SM's warps
    // take the kind their SM index selects (SMs split in proportion to the kinds' item
    // counts, one counter per kind), then the other kind's remainder, so that an SM fetches
    // one code path's instructions at a time.  Otherwise one kind, one counter (one
    // replica: a fixed stride).
    if (threadIdx.x == 0) kinds = 0;
    __syncthreads();
    items_prefix(nrep, pre, wtot, [&](int r) {
        const StepDesc* d = reps[r].desc;
        const int n = phase == 1 ? (d->fb ? d->items_pre : d->items) : (d->fb ? d->items : 0);
        if (Mixed && phase == 1 && n > 0) atomicOr(&kinds, d->fb ? 1 : 2);
        return n;
    });
    const bool affine = Mixed && phase == 1 && nrep > 1 && kinds == 3;
    if (affine) {
        items_prefix(nrep, pre, wtot, [&](int r) {
            const StepDesc* d = reps[r].desc;
            return d->fb ? d->items_pre : 0;
        });
        items_prefix(nrep, pre2, wtot, [&](int r) {
            const StepDesc* d = reps[r].desc;
            return d->fb ? 0 : d->items;
        });
    }
    const int t0 = pre[nrep], t1 = affine ? pre2[nrep] : 0;
    const int nwarps = (int)(gridDim.x * kWarpsG);
    const bool sym = t0 + t1 > nwarps;
    WarpBuf& B = bufs[warp];
    StepDesc* d0 = reps[0].desc;
    const int qi = phase == 1 ? 0 : 1;
    int kind = 0;  // affine: 0 old poses of force-biased steps (queue[0]), 1 ordinary items (queue[1])
    if (affine) {
        unsigned smid, nsm;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        asm volatile("mov.u32 %0, %%nsmid;" : "=r"(nsm));
        kind = ((long long)smid * (t0 + t1) < (long long)t0 * nsm) ? 0 : 1;
    }
    for (int pass = 0; pass < (affine ? 2 : 1); ++pass, kind ^= 1) {
    const int* P = kind ? pre2 : pre;
    const int total = kind ? t1 : t0;
    int* queue = &d0->queue[affine ? kind : qi];
    auto next_item = [&](int prev) {
        if (nrep == 1) return prev < 0 ? (int)blockIdx.x * kWarpsG + warp : prev + nwarps;
        int v = 0;
        if (lane == 0) v = atomicAdd(queue, 1);
        return __shfl_sync(kFull, v, 0);
    };
    for (int it = next_item(-1); it < total; it = next_item(it)) {
        int lo = 0, hi = nrep;
        while (hi - lo > 1) { int mid = (lo + hi) >> 1; if (P[mid] <= it) lo = mid; else hi = mid; }
        const RepDev& R = reps[lo];
        const StepDesc D = *R.desc;
        const int local = it - P[lo];
        const bool fbitem = D.fb != 0;
        const int q = local / max(1, D.k);  // pose fastest, as in k_energy_t
        const int i = local - q * D.k;
        const int v = fbitem ? (phase == 1 ? 1 : 0) : q / D.nslab;
        const int zi = fbitem ? q : q - v * D.nslab;
        float cx, cy, cz;
        int self;
        build_pose(R, D, i, v, B, lane, cx, cy, cz, self);
        if (!(phase == 1 && fbitem)) keep_sites(R, D, B, i, v, zi, lane);
        const int ns = R.frag[D.ftype].nsites;
        const int nwin = R.span[0] * R.span[1] * R.span[2];
        const int c0 = zi, c1 = nwin;  // interleaved range: cells zi, zi + nslab, ...
        const int stride = D.nslab;
        int ng = 0;
        long long npair = 0;
        double acc = 0.0;
        if (!fbitem) {
            EnergySink<> sink;
            walk_cells(R, B, ns, cx, cy, cz, self, c0, c1, lane, sink, ng, npair, nullptr, 0, stride);
            acc = warp_sum(sink.acc);
        } else {
            GradSinkT<true> sink;
            sink.st = &stages[warp];
            sink.gtab = nullptr;
            sink.w = 1.0f;
            sink.ffY = R.ffY;
            walk_cells(R, B, ns, cx, cy, cz, self, c0, c1, lane, sink, ng, npair, nullptr, 0, stride);
            double epme = 0.0;
            float pgx = 0.f, pgy = 0.f, pgz = 0.f;
            if (R.pme && zi == 0) {  // Ewald reciprocal and molecular terms of the pose, once (slab 0)
                const float4 a = B.site_abs[lane < kMaxSites ? lane : 0];
                epme = pme_pose_lane(R, ns, lane, a.x, a.y, a.z, a.w, self);
                pme_grad_lane(R, ns, lane, a.x, a.y, a.z, a.w, self, pgx, pgy, pgz);
            }
            acc = warp_sum((double)sink.e + epme);
            // per-site gradient (lanes < ns after summing the atom subsets), then
            // force -sum g_s and torque -sum (x_s - m) x g_s about the site centroid
            stages[warp].red[lane] = make_float4(sink.gx, sink.gy, sink.gz, 0.0f);
            __syncwarp();
            float g0 = 0.f, g1 = 0.f, g2 = 0.f, r0 = 0.f, r1 = 0.f, r2 = 0.f;
            if (lane < ns) {
                const int nsub = 32 / ns;
                float4 gsum = stages[warp].red[lane];
                for (int k = 1; k < nsub; ++k) {
                    const float4 t = stages[warp].red[k * ns + lane];
                    gsum.x += t.x; gsum.y += t.y; gsum.z += t.z;
                }
                g0 = gsum.x + pgx; g1 = gsum.y + pgy; g2 = gsum.z + pgz;
                float mx = 0.f, my = 0.f, mz = 0.f;
                for (int s = 0; s < ns; ++s) { mx += B.site[s].x; my += B.site[s].y; mz += B.site[s].z; }
                const float inv = 1.0f / (float)ns;
                r0 = B.site[lane].x - mx * inv;
                r1 = B.site[lane].y - my * inv;
                r2 = B.site[lane].z - mz * inv;
            }
            float f[6] = {-g0, -g1, -g2, -(r1 * g2 - r2 * g1), -(r2 * g0 - r0 * g2), -(r0 * g1 - r1 * g0)};
#pragma unroll
            for (int c = 0; c < 6; ++c)
                for (int off = 16; off > 0; off >>= 1) f[c] += __shfl_xor_sync(kFull, f[c], off);
            if (lane == 0) {
                float* out = R.fpart + ((size_t)(i * 2 + v) * D.nslab + zi) * 6;
                for (int c = 0; c < 6; ++c) out[c] = f[c];
            }
        }
        if (lane == 0) {
            R.epart[(i * D.nvar + v) * D.nslab + zi] = acc;
            atomicAdd(&R.counters[2], (unsigned long long)npair);
        }
        if (phase == 1 && fbitem) {  // the last item of pose i draws its proposal
            int last = 0;
            if (lane == 0) {
                __threadfence();
                const int done = atomicAdd(&R.fbcnt[i], 1);
                last = done == D.nslab - 1;
                if (last) R.fbcnt[i] = 0;
            }
            last = __shfl_sync(kFull, last, 0);
            if (last && lane == 0) {
                __threadfence();
                float fo[6];
                fb_force(R, D, i, 1, fo, true);
                const float4 gc = R.gcen[R.frag[D.ftype].startRes + R.pslot[i]];
                R.pcen[i] = fb_propose(R, D, i, fo, gc, R.fbprop + 2 * i);
            }
        } else if (v == 0 && D.nw > 0) {  // this item's share of the neighbour bit matrix
            nbr_share(R, D, i, zi, D.nslab, i * D.nslab + zi, lane, sym);
        }
        __syncwarp();
    }
    }
    if (nrep == 1) return;
    // the last CTA to finish resets the counters for the next launch
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&d0->done[qi], 1) == (int)gridDim.x - 1) {
            d0->queue[qi] = 0;
            if (affine) d0->queue[1] = 0;
            d0->done[qi] = 0;
            __threadfence();
        }
    }
}

template __global__ void k_energy_fb<false>(const RepDev* __restrict__, int, int);
template __global__ void k_energy_fb<true>(const RepDev* __restrict__, int, int);

// gxyz[p][s][3], gq[p][s] = the slabs' partial sums in slab order (FP64).
__global__ void k_sum_grad(const float4* __restrict__ part, int nposes, int nslab, int ns,
                           double* __restrict__ gxyz, double* __restrict__ gq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // p * ns + s
    if (i >= nposes * ns) return;
    const int p = i / ns, s = i - p * ns;
    double x = 0.0, y = 0.0, zz = 0.0, w = 0.0;
    for (int z = 0; z < nslab; ++z) {
        const float4 v = part[((size_t)p * nslab + z) * ns + s];
        x += v.x; y += v.y; zz += v.z; w += v.w;
    }
    if (gxyz) {
        gxyz[3 * (size_t)i] = x;
        gxyz[3 * (size_t)i + 1] = y;
        gxyz[3 * (size_t)i + 2] = zz;
    }
    if (gq) gq[i] = w;
}

// The pair table of the kernels, (100 sigma^2, 4 eps), from the reference's
// (sigma [nm], eps [kJ/mol]) layout: the same float operations as the
// context set-up (gcmc_energy.h:128-130).
__global__ void k_ff_to_lj(const float* __restrict__ ff, float2* __restrict__ lj, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float sigma = ff[2 * i], eps = ff[2 * i + 1];
    lj[i] = make_float2(sigma * sigma * 100.0f, 4.0f * eps);
}

// d/d(sigma, eps) from d/d(sigma2, E4): dsigma2/dsigma = 200 sigma, dE4/deps = 4.
__global__ void k_glj_to_gff(const double* __restrict__ glj, const float* __restrict__ ff,
                             double* __restrict__ gff, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    gff[2 * i] += glj[2 * i] * 200.0 * (double)ff[2 * i];
    gff[2 * i + 1] += glj[2 * i + 1] * 4.0;
}

}  // namespace gcmc
