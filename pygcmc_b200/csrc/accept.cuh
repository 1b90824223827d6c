// Accept/update kernel: the host halves of move_add / move_del / move_trn /
// move_rot (gcmc/cpp/gcmc_move_add.h:103-198, gcmc_move_del.h:97-187,
// gcmc_move_trn.h:159-250, gcmc_move_rot.h:151-275) moved onto the device,
// plus the preparation of the next step's proposals.
//
// One CTA per replica.  For clustering moves the CTA
//   1. sums each pose's slab partials (FP64) and precomputes per pose the
//      log-weight -beta*E and the Gumbel key -beta*E + G (Gumbel-max picks
//      pose i with probability w_i / sum w, the law of the reference's
//      roulette selection); the per-pose draws and the pose-pose bit matrix
//      are staged in shared memory;
//   2. the clusters are walked in pose-index order: seed = lowest unused
//      pose, members = unused poses within the cutoff of the seed (one 32-bit
//      word per lane), the argmax key and the Rosenbluth / Metropolis
//      acceptance in FP64 (decided from bounds on ln W where they settle it);
//      an accepted cluster also removes the unused poses within the cutoff of
//      its chosen pose;
//   3. all warps write the accepted poses into their slots, then one thread
//      applies the cell-list and count updates in acceptance order.
#pragma once
#include "tiles.cuh"

namespace gcmc {

constexpr int kAcceptThreads = 1024;
constexpr int kNbHalf = kMaxPoses * kMaxWords / 2;  // words

struct AcceptSmem {
    double E[kMaxPoses];      // energy entering the acceptance (force-biased: dE - ln(q ratio) / beta)
    double ephys[kMaxPoses];  // the pose's energy (insert/delete) or energy change (translate/rotate)
    double a[kMaxPoses];      // log-weight -beta E of pose i (-inf if E is not finite)
    unsigned long long key[kMaxPoses];  // order-preserving encoding of the Gumbel key
    alignas(16) double lnu[kMaxPoses];  // ln of the acceptance draw of the cluster seeded by pose i
    alignas(16) double gum[kMaxPoses];  // Gumbel draw -ln(-ln u) of pose i
    double lnn[kMaxPoses + 1];          // insertion: ln(n + 1) for n = D.n .. D.n + k
    alignas(16) float4 c[kMaxPoses];
    alignas(16) uint32_t nb[kMaxPoses * kMaxWords];
    int acc_list[kMaxPoses];
    int acc_slot[kMaxPoses];
    double red[32];
    int misc[8];
    // one round of speculative clusters (seeded in order assuming no acceptance)
    uint32_t spec_mask[32][kMaxWords];
    uint32_t spec_us[33][kMaxWords];  // unused words after the round's first c seeds (c = 0..32)
    int spec_seed[32];
    int spec_cnt[32];
    int spec_chosen[32];  // Gumbel argmax, -1 if no member has a finite energy
    double spec_lnq[32];  // exact ln(W) - ln(cnt) (W = sum over members of exp(-beta E)) when spec_dec = 0
    int spec_dec[32];     // +1 / -1: accepted / rejected for every K the round can reach; 0: compare with lnq
    double kr[2];         // K range of the round: the lowest K the step can reach, K at the round's start
    int spec_n;
};

// ---- asynchronous 16-byte global -> shared copies (cp.async) ----
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(__cvta_generic_to_global(gmem))
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---- cell list maintenance (single thread) ----
// Each cell keeps its entries in increasing group id, so a cell's content (and
// with it the order in which the energy kernels visit groups and sum their
// terms) depends only on the current state, not on the history of moves: a
// context rebuilt from a checkpoint evaluates bit-identical energies.  An
// entry carries the group's centre and atom range (from R.gcen / R.gspan at
// insertion; translated groups that stay in their cell are refreshed in place).
__device__ __forceinline__ int ent_id(const CellEnt& e) { return __float_as_int(e.c.w); }
__device__ __forceinline__ CellEnt make_ent(const RepDev& R, int g) {
    const float4 c = R.gcen[g];
    CellEnt e;
    e.c = make_float4(c.x, c.y, c.z, __int_as_float(g));
    e.span = R.gspan[g];
    e.pad = make_int2(0, 0);
    return e;
}
__device__ __forceinline__ void cell_insert(const RepDev& R, int c, int g) {
    const int n = R.cell_count[c];
    if (n >= R.cap) {
        atomicOr(R.err, ERR_CELL_OVERFLOW);
        R.gcell[g] = -1;
        return;
    }
    CellEnt* ent = R.cell_ent + (size_t)c * R.cap;
    int p = n;
    while (p > 0 && ent_id(ent[p - 1]) > g) {  // shift larger ids up by one
        const CellEnt h = ent[p - 1];
        ent[p] = h;
        R.gcell[ent_id(h)] = c * R.cap + p;
        --p;
    }
    ent[p] = make_ent(R, g);
    R.cell_count[c] = n + 1;
    R.gcell[g] = c * R.cap + p;
}
__device__ __forceinline__ void cell_add(const RepDev& R, int g, float x, float y, float z) {
    cell_insert(R, cell_of(R, x, y, z), g);
}
__device__ __forceinline__ void cell_remove(const RepDev& R, int g) {
    const int cp = R.gcell[g];
    if (cp < 0) return;
    const int c = cp / R.cap;
    const int n = R.cell_count[c];
    CellEnt* ent = R.cell_ent + (size_t)c * R.cap;
    for (int p = cp - c * R.cap; p + 1 < n; ++p) {  // shift the rest down by one
        const CellEnt h = ent[p + 1];
        ent[p] = h;
        R.gcell[ent_id(h)] = c * R.cap + p;
    }
    R.cell_count[c] = n - 1;
    R.gcell[g] = -1;
}
// the cell entry of group `from` now stands for group `to` (same cell; R.gcen[to] already set)
__device__ __forceinline__ void cell_rename(const RepDev& R, int from, int to) {
    const int cp = R.gcell[from];
    if (cp < 0) {
        R.gcell[to] = -1;
        return;
    }
    const int c = cp / R.cap;
    cell_remove(R, from);
    cell_insert(R, c, to);
}

// Cell-list moves of up to 32 groups by one warp: lane l (active) takes group
// g out of its current cell (rem) and/or inserts it into cell `cnew` (cnew < 0:
// no insertion).  All removals run before all insertions; lanes touching the
// same cell take turns (lowest lane first), different cells are independent,
// and since cells are kept sorted their content does not depend on the order.
__device__ __forceinline__ void warp_cell_moves(const RepDev& R, int lane, bool active, int g, bool rem,
                                                int cnew) {
    int cold = -1;
    if (active && rem) {
        const int cp = R.gcell[g];
        cold = cp >= 0 ? cp / R.cap : -1;
    }
    bool pend = active && cold >= 0;
    while (__any_sync(kFull, pend)) {
        const unsigned grp = __match_any_sync(kFull, pend ? cold : -2 - lane);
        if (pend && __ffs(grp) - 1 == lane) {
            cell_remove(R, g);
            pend = false;
        }
        __syncwarp();
    }
    pend = active && cnew >= 0;
    while (__any_sync(kFull, pend)) {
        const unsigned grp = __match_any_sync(kFull, pend ? cnew : -2 - lane);
        if (pend && __ffs(grp) - 1 == lane) {
            cell_insert(R, cnew, g);
            pend = false;
        }
        __syncwarp();
    }
}

// Order-preserving map of a double to uint64 (larger key -> larger integer);
// 0 is reserved for "no candidate".
__device__ __forceinline__ bool normal_positive(double a) { return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e308; }

__device__ __forceinline__ unsigned long long key_order(double d) {
    const long long b = __double_as_longlong(d);
    return b >= 0 ? ((unsigned long long)b | 0x8000000000000000ull) : ~(unsigned long long)b;
}

// ---- block reductions ----
__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    return v;
}

// Per-pose ranges of the per-pose-warp kernel in proportion to each pose
// variant's work, estimated as the fixed atoms in the windows of its centre's
// cell (wcost) plus kCellWork atoms' worth per window cell: the poses inside a
// dense protein get more, and shorter, ranges than those in the open box, so
// that the items of one launch take similar times.  Whole CTA; scratch: 2 *
// kMaxPoses ints.  Slots s = v k + i (the new variants first, so that the
// new-variant items are the list's first ones; a step in the difference form has
// v = 0 only); entry e = i nvar + v.  The total stays the uniform split's
// `budget` items (up to rounding).  Writes pnslab and pitem; returns the item
// count and the largest split in *nmax.
constexpr int kCellWork = 4;
__device__ int split_entries(const RepDev& R, const StepDesc& D, int budget, int* scratch, int* wtot, int* nmax_sh) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nv = D.dual ? 1 : D.nvar;
    const int nslots = D.k * nv;
    const int startRes = D.move == MV_INSERT ? 0 : R.frag[D.ftype].startRes;
    const int nwin = R.span[0] * R.span[1] * R.span[2];
    const int cap = min(255, R.max_split * (D.dual ? 2 : 1));
    auto cost = [&](int s) {
        const int v = s / D.k, i = s - v * D.k;
        float4 c;
        if (D.move == MV_INSERT || D.move == MV_DELETE || (v == 0 && !D.dual)) c = R.pcen[i];
        else c = R.gcen[startRes + R.pslot[i]];
        return R.wcost[cell_of(R, c.x, c.y, c.z)] + kCellWork * nwin;
    };
    for (int s = tid; s < nslots; s += nt) scratch[s] = cost(s);
    if (tid == 0) *nmax_sh = 1;
    __syncthreads();
    const double total = (double)block_excl_scan(scratch, nslots, wtot);
    for (int s = tid; s < nslots; s += nt) {
        const int n = max(1, min(cap, (int)((double)budget * (double)cost(s) / total + 0.5)));
        scratch[s] = n;
        const int v = s / D.k, i = s - v * D.k;
        const int e = i * D.nvar + v;
        R.pnslab[e] = n;
        if (D.dual) R.pnslab[e + 1] = n;  // the old variant's zero partials
        atomicMax(nmax_sh, n);
    }
    __syncthreads();
    const int items = block_excl_scan(scratch, nslots, wtot);
    for (int s = tid; s < nslots; s += nt) {
        const int v = s / D.k, i = s - v * D.k;
        const int e = i * D.nvar + v;
        const int off = scratch[s], n = (s + 1 < nslots ? scratch[s + 1] : items) - off;
        for (int z = 0; z < n; ++z) R.pitem[off + z] = (e << 8) | z;
    }
    __syncthreads();
    return items;
}

// ---- next-step preparation (whole CTA) ----
// scratch: kBinScratchBytes of shared memory for the tiled contexts' pose binning.
__device__ void prepare_step(const RepDev& R, int step, int* scratch) {
    __shared__ StepDesc Dsh;
    __shared__ int wtot_sh[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        StepDesc D{};
        D.step = step;
        D.move = MV_NONE;
        D.del_slot = -1;
        D.nslab = 1;
        if (step < R.run_end && step < R.mcsteps) {
            const int mv = R.moves[step];
            D.ftype = mv >> 2;
            D.move = mv & 3;
            const FragDev& F = R.frag[D.ftype];
            const int n = R.totalNum[D.ftype];
            D.n = n;
            if (D.move == MV_INSERT) {
                D.k = (n >= F.maxNum) ? 0 : F.confBias;
                D.nvar = 1;
            } else if (D.move == MV_DELETE) {
                D.k = n > 0 ? 1 : 0;
                D.nvar = 1;
                if (n > 0) {
                    U4 r = rng(R.seed, R.replica, R.step_base + (uint32_t)step, 0u, RP_DELETE, 0);
                    D.del_slot = (int)(r.x % (uint32_t)n);
                }
            } else {
                D.k = min(F.confBias, n);
                D.nvar = 2;
                D.perm_key = rng(R.seed, R.replica, R.step_base + (uint32_t)step, 0u, RP_PERM, 0);
                D.perm_h = perm_bits(n);
                D.fb = R.fb;
            }
            if (D.k > kMaxPoses) {
                atomicOr(R.err, ERR_POSES);
                D.k = 0;
            }
            D.nw = (D.move == MV_DELETE) ? 0 : (D.k + 31) >> 5;
            // translate / rotate in the pairwise-difference form: one item per pose (and slab)
            D.dual = (R.dual && !D.fb && (D.move == MV_TRANSLATE || D.move == MV_ROTATE)) ? 1 : 0;
            D.margin = (D.dual && D.move == MV_TRANSLATE) ? R.dmargin : 0;
            // split each pose's cell window so a step has at most split_items work items
            // (at least one range per pose, at most max_split)
            const int kv = max(1, D.k * (D.dual ? 1 : D.nvar));
            // tiled contexts: one energy per pose variant (per pose when dual), items = tiles
            // (set below)
            // (a dual item carries both poses' pairs: up to twice as many ranges per pose)
            D.nslab = R.tiled ? 1 : max(1, min(R.max_split * (D.dual ? 2 : 1), R.split_items / kv));
            D.items = R.tiled ? 0 : ((D.fb || D.dual) ? D.k * D.nslab : D.k * D.nvar * D.nslab);
            D.items_pre = D.fb ? D.k * D.nslab : 0;
        }
        Dsh = D;
    }
    __syncthreads();
    const StepDesc D = Dsh;
    if (D.move == MV_INSERT) {
        for (int i = tid; i < D.k; i += nt) {
            float x, y, z;
            insert_centre(R, step, i, x, y, z);
            R.pcen[i] = make_float4(x, y, z, 0.0f);
        }
    } else if (D.move == MV_DELETE) {
        if (tid == 0 && D.k > 0) R.pcen[0] = R.gcen[R.frag[D.ftype].startRes + D.del_slot];
    } else if (D.move != MV_NONE) {
        const int startRes = R.frag[D.ftype].startRes;
        for (int i = tid; i < D.k; i += nt) {
            const int slot = perm_slot(D.perm_key, D.perm_h, i, D.n);
            R.pslot[i] = slot;
            float4 c = R.gcen[startRes + slot];
            if (D.move == MV_TRANSLATE && !D.fb) {  // force-biased: set by the old-pose launch
                U4 r = rng(R.seed, R.replica, R.step_base + (uint32_t)step, (uint32_t)i, RP_MOVE, 0);
                c.x = fadd(c.x, trn_shift(R, r.x, 0, c.x));
                c.y = fadd(c.y, trn_shift(R, r.y, 1, c.y));
                c.z = fadd(c.z, trn_shift(R, r.z, 2, c.z));
            }
            c.w = 0.0f;
            R.pcen[i] = c;
        }
    }
    __shared__ int nmax_sh;
    if (R.tiled && D.move != MV_NONE && D.k > 0) {
        __syncthreads();  // centres and slots written above
        const int ntiles = bin_entries(R, D, scratch, wtot_sh);
        if (tid == 0) Dsh.items = ntiles;
    } else if (R.wcost && D.move != MV_NONE && D.k > 0 && !R.fb) {  // (the force-bias kernel splits alike)
        __syncthreads();  // centres and slots written above
        const int items = split_entries(R, D, D.items, scratch, wtot_sh, &nmax_sh);
        if (tid == 0) {
            Dsh.items = items;
            Dsh.nslab = nmax_sh;
            Dsh.varslab = 1;
        }
    }
    if (tid == 0) {
        StepDesc Dw = D;
        Dw.items = Dsh.items;
        Dw.nslab = Dsh.nslab;
        Dw.varslab = Dsh.varslab;
        *R.desc = Dw;
    }
    __syncthreads();
}

// The preparation kernels take kBinScratchBytes of dynamic shared memory when
// the context is tiled (the pose binning's scratch).
__global__ void __launch_bounds__(kAcceptThreads) k_prepare(const RepDev* __restrict__ reps, int nrep) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const RepDev& R = reps[blockIdx.x];
    const StepDesc D = *R.desc;
    __syncthreads();
    if (D.move == MV_NONE) prepare_step(R, D.step, reinterpret_cast<int*>(smem_raw));
}

// Prepare step `step` in one descriptor (a run's first step, whichever copy holds it).
__global__ void __launch_bounds__(kAcceptThreads) k_prepare_at(const RepDev* __restrict__ rep, int step) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    prepare_step(*rep, step, reinterpret_cast<int*>(smem_raw));
}

__global__ void k_set_run_end(RepDev* reps, int nrep, int nsteps) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nrep) {
        long long e = (long long)reps[r].run_end + nsteps;
        reps[r].run_end = (int)(e < reps[r].mcsteps ? e : reps[r].mcsteps);
        if (reps[r].other != &reps[r]) {  // the speculating copy: same run end, no standing speculation
            RepDev* o = const_cast<RepDev*>(reps[r].other);
            o->run_end = reps[r].run_end;
            *reps[r].valid = 0;
            *o->valid = 0;
            *reps[r].abort = -1;
            *o->abort = -1;
        }
    }
}

// Speculative step preparation (one CTA, nrep = 1).  mode 0: prepare in this
// copy the step after the other copy's, from the state after the step before
// that (as if the other copy's step accepts nothing); mode 1: prepare this
// copy's step again from the current state unless its speculation stands.
__global__ void __launch_bounds__(kAcceptThreads) k_prep_spec(const RepDev* __restrict__ reps, int mode) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_trigger();  // the completion pose-energy launch may start (it waits for this grid's results)
    int* scratch = reinterpret_cast<int*>(smem_raw);
    const RepDev& R = reps[0];
    if (mode == 0) {
        const int step = *R.other->spec_step + 1;
        if (threadIdx.x == 0) {
            *R.pairs_pending = 0ull;
            *R.spec_step = step;
        }
        prepare_step(R, step, scratch);
    } else {
        const int valid = *R.valid;
        const int step = *R.spec_step;
        __syncthreads();
        if (!valid) prepare_step(R, step, scratch);
    }
}

// The step a speculating run starts at, in the copy that holds it.
__global__ void k_spec_start(const RepDev* __restrict__ rep, int step) {
    if (threadIdx.x == 0) *rep->spec_step = step;
}

// Initial cell lists in two parallel passes (grid.y = replica): every present
// group (fixed, or an occupied fragment slot) appends its record to its cell
// at a slot from an atomic counter, then each cell is ordered by group id and
// the groups' record slots are noted -- the same lists as inserting the groups
// one by one.  A cell that overflows keeps cap records and raises the error
// flag; the groups left out keep gcell = -1.
__global__ void k_fill_cells(const RepDev* __restrict__ reps) {
    const RepDev& R = reps[blockIdx.y];
    const FragDev& Fl = R.frag[R.ntypes - 1];
    const int ng = Fl.startRes + Fl.maxNum;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        bool present = g < R.nfixed;
        for (int t = 0; !present && t < R.ntypes; ++t) {
            const int s = g - R.frag[t].startRes;
            if (s >= 0 && s < R.frag[t].maxNum) {
                present = s < R.totalNum[t];
                break;
            }
        }
        if (!present) continue;
        const float4 c = R.gcen[g];
        const int cell = cell_of(R, c.x, c.y, c.z);
        const int p = atomicAdd(&R.cell_count[cell], 1);
        if (p < R.cap) R.cell_ent[(size_t)cell * R.cap + p] = make_ent(R, g);
        else atomicOr(R.err, ERR_CELL_OVERFLOW);
    }
}

__global__ void k_sort_cells(const RepDev* __restrict__ reps) {
    const RepDev& R = reps[blockIdx.y];
    const int ncell = R.nc[0] * R.nc[1] * R.nc[2];
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) {
        int n = R.cell_count[c];
        if (n > R.cap) {
            n = R.cap;
            R.cell_count[c] = n;
        }
        CellEnt* ent = R.cell_ent + (size_t)c * R.cap;
        for (int i = 1; i < n; ++i) {  // insertion sort by group id
            const CellEnt e = ent[i];
            int j = i;
            while (j > 0 && ent_id(ent[j - 1]) > ent_id(e)) {
                ent[j] = ent[j - 1];
                --j;
            }
            ent[j] = e;
        }
        for (int i = 0; i < n; ++i) R.gcell[ent_id(ent[i])] = c * R.cap + i;
    }
}

__device__ __forceinline__ double key_value(unsigned long long k) {  // inverse of key_order
    return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

// Evaluation of the cluster with member words m (lane = word) and seed draw
// ln u, warp-collective.  Results: member count, the Gumbel argmax (-1 if no
// member has a finite energy) and the decision of "ln u < lnq + K" with
//   lnq = ln(W') + M - ln(cnt),  W' = sum over members of exp(a_i - M),
// a_i = -beta E_i, M = max a_i, for every K of the round's range [Klo, Khi]:
// dec = +1 (accepted for all of them), -1 (rejected for all), or 0 with lnq
// computed (then the commit compares with its K).  The max term of W' is
// exactly 1 and the others lie in [0, 1], so ln W' lies in [0, ln cnt] and
// lnq in [M - ln cnt, M]; dec is decided from that range (ln cnt bounded above
// by ln 2 * ceil(log2 cnt), a margin above the rounding of the exact form),
// and exp / log are evaluated only when ln u falls inside it.
__device__ __forceinline__ void eval_cluster(const AcceptSmem& S, uint32_t m, int lane, double lnu, double Klo,
                                             double Khi, int& cnt_out, int& chosen_out, int& dec_out,
                                             double& lnq_out) {
    const int cnt = __reduce_add_sync(kFull, (unsigned)__popc(m));
    unsigned long long best = 0ull, amax = 0ull;
    int bi = -1;
    for (uint32_t mm = m; mm; mm &= mm - 1u) {
        const int i = 32 * lane + __ffs(mm) - 1;
        const unsigned long long kk = S.key[i];
        if (kk > best) { best = kk; bi = i; }
        const double ai = S.a[i];
        if (ai > -INFINITY) {
            const unsigned long long ak = key_order(ai);
            if (ak > amax) amax = ak;
        }
    }
    // Gumbel argmax (keys are distinct integers; ties cannot occur between members)
    const unsigned hi = (unsigned)(best >> 32);
    const unsigned mhi = __reduce_max_sync(kFull, hi);
    const unsigned lo = (hi == mhi) ? (unsigned)best : 0u;
    const unsigned mlo = __reduce_max_sync(kFull, lo);
    const unsigned win = __ballot_sync(kFull, best != 0ull && hi == mhi && (unsigned)best == mlo);
    const int chosen = win ? __shfl_sync(kFull, bi, __ffs(win) - 1) : -1;
    // M = max a_i over the members with a finite energy
    const unsigned ahi = (unsigned)(amax >> 32);
    const unsigned mahi = __reduce_max_sync(kFull, ahi);
    const unsigned alo = (ahi == mahi) ? (unsigned)amax : 0u;
    const unsigned malo = __reduce_max_sync(kFull, alo);
    int dec = -1;
    double lnq = -INFINITY;
    if (chosen >= 0) {
        const double M = key_value(((unsigned long long)mahi << 32) | malo);
        const double lnc_hi = 0.6931471805599453 * (double)(32 - __clz(cnt - 1));  // >= ln(cnt)
        const double eps = 1e-9 * (1.0 + fabs(M) + fabs(Klo) + fabs(Khi) + fabs(lnu));
        if (lnu < (M - lnc_hi) + Klo - eps) {
            dec = 1;
        } else if (lnu > M + Khi + eps) {
            dec = -1;
        } else {
            double w = 0.0;
            for (uint32_t mm = m; mm; mm &= mm - 1u) w += exp(S.a[32 * lane + __ffs(mm) - 1] - M);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) w += __shfl_xor_sync(kFull, w, off);
            lnq = (log(w) + M) - log((double)cnt);
            dec = 0;
        }
    }
    cnt_out = cnt;
    chosen_out = chosen;
    dec_out = dec;
    lnq_out = lnq;
}

// Void the speculative evaluation of step `step` (the other descriptor copy's):
// its walks stop at their next batch of candidate groups.
__device__ __forceinline__ void void_next(const RepDev& R, int step) {
    *reinterpret_cast<volatile int*>(R.other->abort) = step;
    __threadfence();
}

// spec (one replica, speculating): the step's pose energies may come from the
// speculative launch (booked here); as soon as a move is accepted the
// speculative evaluation of the next step is voided, and at the end the next
// step is marked as standing when nothing was accepted.
// One replica's step, whole CTA (kAcceptThreads threads); smem_raw: an
// AcceptSmem.  The body of k_accept and of the persistent step loop.
// Pme: the replica may run Ewald electrostatics (the background term and the
// mesh charge updates are compiled in only then; they add registers to every
// phase of the kernel).
template <bool Pme>
__device__ __forceinline__ void accept_step(const RepDev& R, int spec, unsigned char* smem_raw) {
    AcceptSmem& S = *reinterpret_cast<AcceptSmem*>(smem_raw);
    const StepDesc D = *R.desc;
    if (D.move == MV_NONE) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nt = blockDim.x, nwarps = nt >> 5;
    if (spec && tid == 0 && *R.valid) {  // energies evaluated beside the previous step's accept kernel
        R.counters[2] += *R.pairs_pending;
        R.counters[13] += 1ull;
    }
    const FragDev& F = R.frag[D.ftype];
    const int k = D.k, ns = F.nsites;
    long long t_start = clock64(), t_mark = t_start;
    // Clustering moves: the per-pose inputs of the walk (centres, Gumbel and
    // acceptance draws, neighbour bit rows; written by the pose-energy launch)
    // are copied into shared memory asynchronously, issued first so that they
    // arrive while the energies are summed.  Sizes are rounded up to whole
    // 16-byte chunks; the sources hold kMaxPoses entries (kMaxPoses x kMaxWords
    // words), so the rounding stays inside them.
    // The slab partials of the pose energies follow when they fit in the upper
    // half of the bit-matrix array beside the step's rows (translate/rotate
    // steps: few poses, many slabs each).
    double* const Ep = reinterpret_cast<double*>(&S.nb[kNbHalf]);
    const int npart = k * D.nvar * D.nslab;
    const bool stage_e = D.move != MV_DELETE && k > 0 && ((k * D.nw + 3) & ~3) <= kNbHalf && npart <= kNbHalf / 2;
    if (D.move != MV_DELETE && k > 0) {
        const int nb16 = (k * D.nw + 3) >> 2, d16 = (k + 1) >> 1;
        if (stage_e)  // the source holds kMaxPoses * 2 * (max slabs) partials: an even count
            for (int x = tid; x < (npart + 1) >> 1; x += nt) cp_async16(&Ep[2 * x], R.epart + 2 * x);
        for (int x = tid; x < nb16; x += nt) cp_async16(&S.nb[4 * x], R.nbr + 4 * x);
        for (int x = tid; x < k; x += nt) cp_async16(&S.c[x], R.pcen + x);
        for (int x = tid; x < d16; x += nt) {
            cp_async16(&S.gum[2 * x], R.pgum + 2 * x);
            cp_async16(&S.lnu[2 * x], R.plnu + 2 * x);
        }
        cp_async_commit();
    }
    // phase cycle sums (thread 0): 0 energies, 1 per-pose precompute, 2 cluster walk, 3 apply, 4 prepare
#define PHASE(i)                                                                  \
    do {                                                                          \
        if (tid == 0) {                                                           \
            long long t_ = clock64();                                             \
            atomicAdd(&R.counters[4 + (i)], (unsigned long long)(t_ - t_mark));   \
            t_mark = t_;                                                          \
        }                                                                         \
    } while (0)

    // ---- phase 0: pose energies (sum of slab partials; dE for translate/rotate)
    const bool logging = R.log != nullptr && D.step < R.log_cap;
    double bg = 0.0;  // Ewald: change of the neutralising-background energy -bgc Q^2
    if (Pme && R.pme && (D.move == MV_INSERT || D.move == MV_DELETE)) {
        double Q = R.pme_qfix;
        for (int t = 0; t < R.ntypes; ++t) Q += (double)R.totalNum[t] * R.frag[t].qnet;
        const double dq = D.move == MV_INSERT ? F.qnet : -F.qnet;
        const double change = -R.pme_bgc * ((Q + dq) * (Q + dq) - Q * Q);
        bg = D.move == MV_INSERT ? change : -change;  // a deletion's E is minus the system's change
    }
    if (stage_e) {
        cp_async_wait_all();
        __syncthreads();
    }
    const double* ep = stage_e ? Ep : R.epart;
    for (int i = tid; i < k; i += nt) {
        double e = 0.0;
        const int n0 = D.varslab ? R.pnslab[i * D.nvar] : D.nslab;
        for (int z = 0; z < n0; ++z) e += ep[(i * D.nvar) * D.nslab + z];
        if (D.nvar == 2) {
            const int n1 = D.varslab ? R.pnslab[i * 2 + 1] : D.nslab;
            double eo = 0.0;
            for (int z = 0; z < n1; ++z) eo += ep[(i * 2 + 1) * D.nslab + z];
            e = e - eo;
        }
        e += bg;
        S.ephys[i] = e;
        if (D.fb) {  // Metropolis-Hastings: exp(-beta dE) q(new -> old) / q(old -> new)
            float fo[6], fn[6];
            fb_force(R, D, i, 1, fo, false);
            fb_force(R, D, i, 0, fn, false);
            const float4 d = R.fbprop[2 * i], ao = R.fbprop[2 * i + 1];
            double eff = INFINITY;
            if (d.w == 0.0f && isfinite(e)) eff = __dsub_rn(e, __ddiv_rn(fb_ln_ratio(R, D, d, ao, fn), kBeta));
            S.E[i] = eff;
            if (logging && R.logF && i < R.log_kmax) {
                float* o = R.logF + ((size_t)D.step * R.log_kmax + i) * 12;
                for (int c = 0; c < 6; ++c) { o[c] = fo[c]; o[6 + c] = fn[c]; }
            }
        } else {
            S.E[i] = e;
        }
    }
    if (tid == 0) { S.misc[0] = 0; S.misc[1] = 0; S.misc[2] = -1; S.misc[3] = D.n; }
    __syncthreads();
    PHASE(0);
    double esum = 0.0;
    if (logging) {
        double v = 0.0;
        for (int i = tid; i < k; i += nt) v += S.ephys[i];
        esum = block_sum(v, S.red);
        const int kl = min(k, R.log_kmax);
        for (int i = tid; i < kl; i += nt) R.logE[(size_t)D.step * R.log_kmax + i] = S.ephys[i];
    }

    if (D.move == MV_DELETE) {
        if (tid == 0 && k == 1) {
            const double E = S.E[0];
            const int n = D.n;
            const double lnp = log((double)n) - F.B + kBeta * E;
            const U4 r = rng(R.seed, R.replica, R.step_base + (uint32_t)D.step, 0u, RP_DELETE, 0);
            const double u = u53(r.y, r.z);
            const bool acc = !isnan(lnp) && (lnp >= 0.0 || u < exp(lnp));
            if (acc) {
                if (spec) void_next(R, D.step + 1);
                const int slot = D.del_slot, last = n - 1;
                const int gs = F.startRes + slot, gl = F.startRes + last;
                if (Pme && R.pme) {  // the leaving molecule's charges leave the mesh
                    const int2 sd = R.gspan[gs];
                    for (int s = 0; s < ns; ++s) {
                        const float4 a = R.xyzq[sd.x + s];
                        pme_move_site(R, true, a.x, a.y, a.z, false, 0.f, 0.f, 0.f, a.w);
                    }
                    *R.pme_dirty = 1;
                }
                cell_remove(R, gs);
                if (slot != last) {
                    const int2 ss = R.gspan[gs], sl = R.gspan[gl];
                    for (int s = 0; s < ns; ++s) {
                        float4 a = R.xyzq[sl.x + s];
                        float4 b = R.xyzq[ss.x + s];
                        R.xyzq[ss.x + s] = make_float4(a.x, a.y, a.z, b.w);
                    }
                    R.gcen[gs] = R.gcen[gl];
                    cell_rename(R, gl, gs);
                }
                R.totalNum[D.ftype] = n - 1;
                *R.energy -= E;
            }
            S.misc[0] = acc ? 1 : 0;
            S.misc[1] = 1;
            S.misc[2] = acc ? 0 : -1;
            S.misc[3] = acc ? n - 1 : n;
        }
    } else if (k > 0) {
        // ---- phase 1: per-pose weights, Gumbel keys, acceptance draws, bit rows
        cp_async_wait_all();  // this thread's staged copies
        __syncthreads();      // everyone's
        for (int i = tid; i < k; i += nt) {
            const double e = S.E[i];
            const bool fin = isfinite(e);
            S.a[i] = fin ? -kBeta * e : -INFINITY;
            S.key[i] = fin ? key_order(-kBeta * e + S.gum[i]) : 0ull;  // Gumbel-max key
        }
        const int nw = D.nw;
        if (D.move == MV_INSERT)  // ln(n + 1) for every count the walk can reach
            for (int j = tid; j <= k && D.n + j <= F.maxNum; j += nt) S.lnn[j] = log((double)(D.n + j) + 1.0);
        __syncthreads();
        PHASE(1);

        // ---- phase 2: cluster walk in speculative rounds
        // The sequential definition: seed = lowest unused pose, members = unused
        // poses within the cutoff of the seed, decision, then the members (and on
        // acceptance the unused poses within the cutoff of the chosen pose) leave
        // the unused set.  Each round, warp 0 seeds up to 32 clusters ahead
        // assuming no acceptance; all warps evaluate them in parallel (member
        // count, Gumbel argmax and the decision for the round's range of K, see
        // eval_cluster); warp 0 then commits them in order.  A speculative cluster is exactly
        // the sequential one while its seed and all its members are still unused
        // (removing other poses can neither lower the seed nor change the member
        // set); at the first cluster that fails this test the round ends and the
        // next one reseeds from there.  The commit accepts iff
        // ln u < ln(W) - ln(cnt) + K(n), K = ln(cavityFactor) + B - ln(n+1) for
        // insertions and 0 for translate/rotate -- u < min(1, exp(lnp)) in log form.
        const bool ins = (D.move == MV_INSERT);
        uint32_t u = 0u;  // warp 0: unused-pose word `lane`
        if (warp == 0 && lane < nw) {
            const int rem = k - 32 * lane;
            u = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
        }
        int wn = D.n, wna = 0, wnc = 0, wfa = -1;
        const double K0 = ins ? (R.lncav + F.B) : 0.0;
        double K = ins ? K0 - S.lnn[0] : 0.0;
        // K only decreases (one ln(n+1) step per accepted insertion), down to Klo
        const double Klo = ins ? K0 - S.lnn[min(k, F.maxNum - D.n)] : 0.0;
        int nrounds = 0;
        int depth = 32;  // speculation depth: halves after a round cut short, doubles after a full one
        for (int round = 0; round <= k; ++round) {
            ++nrounds;
            if (warp == 0) {  // speculative seeding
                uint32_t us = u;
                int nb = 0;
                S.spec_us[0][lane] = us;
                while (nb < depth) {
                    // lowest unused pose: minimum over the lanes' lowest set bits
                    const unsigned low = us ? (unsigned)(32 * lane + __ffs(us) - 1) : 0xffffffffu;
                    const unsigned sdu = __reduce_min_sync(kFull, low);
                    if (sdu == 0xffffffffu) break;
                    const int sd = (int)sdu;
                    uint32_t m = (lane < nw) ? (us & S.nb[sd * nw + lane]) : 0u;
                    if (lane == (sd >> 5)) m |= 1u << (sd & 31);
                    us &= ~m;
                    S.spec_mask[nb][lane] = m;
                    S.spec_us[nb + 1][lane] = us;
                    if (lane == 0) S.spec_seed[nb] = sd;
                    ++nb;
                }
                if (lane == 0) {
                    S.spec_n = nb;
                    S.kr[0] = Klo;
                    S.kr[1] = K;
                }
            }
            __syncthreads();
            const int nb = S.spec_n;
            if (nb == 0) break;
            if (warp < nb) {  // evaluation, one warp per speculative cluster
                const int sd = S.spec_seed[warp];
                int cnt, chosen, dec;
                double lnq;
                eval_cluster(S, S.spec_mask[warp][lane], lane, S.lnu[sd], S.kr[0], S.kr[1], cnt, chosen, dec, lnq);
                if (lane == 0) {
                    S.spec_cnt[warp] = cnt;
                    S.spec_lnq[warp] = lnq;
                    S.spec_chosen[warp] = chosen;
                    S.spec_dec[warp] = dec;
                }
            }
            __syncthreads();
            if (warp == 0) {  // in-order commit
                // Lane j holds speculative cluster j's scalars.  The decision of a
                // cluster depends only on its own scalars and on K, which changes only
                // at an acceptance, so the decisions of all clusters after the last
                // acceptance are made at once and the clusters before the first
                // accepting one are committed together: u keeps only the unused
                // words after their seeding (spec_us).  A cluster is exact while none
                // of its poses has left u, and only an acceptance (the unused poses
                // within the cutoff of its chosen pose) removes poses of later
                // clusters.  A removed pose's cluster is the first c whose seeding
                // took it out of spec_us (binary search over c), and the earliest
                // such cluster is where the round ends.
                const int my_seed = lane < nb ? S.spec_seed[lane] : 0;
                const int my_chosen = lane < nb ? S.spec_chosen[lane] : -1;
                const int my_dec = lane < nb ? S.spec_dec[lane] : -1;
                const double my_lnq = lane < nb ? S.spec_lnq[lane] : 0.0;
                const double my_lnu = lane < nb ? S.lnu[my_seed] : 0.0;
                int j = 0;
                int cut = nb + 1;  // first cluster that lost a pose to an acceptance (nb + 1: none)
                while (j < nb) {
                    const unsigned am = __ballot_sync(
                        kFull, lane >= j && lane < nb && my_chosen >= 0 &&
                                   (my_dec > 0 || (my_dec == 0 && my_lnu < my_lnq + K)));
                    const int ja = am ? __ffs(am) - 1 : nb;  // first accepting cluster (nb: none)
                    const int jstop = min(ja, cut);          // clusters [j, jstop) are rejected
                    u &= S.spec_us[jstop][lane];
                    wnc += jstop - j;
                    j = jstop;
                    if (j >= nb || j == cut) break;
                    // cluster j accepts its chosen pose
                    const int chosen = __shfl_sync(kFull, my_chosen, j);
                    u &= S.spec_us[j + 1][lane];
                    const uint32_t row = lane < nw ? S.nb[chosen * nw + lane] : 0u;
                    const uint32_t lost = u & row;
                    u &= ~row;
                    unsigned first = 0xffffffffu;
                    for (uint32_t mm = lost; mm; mm &= mm - 1u) {
                        const int b = __ffs(mm) - 1;
                        if ((S.spec_us[nb][lane] >> b) & 1u) continue;  // in no cluster of this round
                        int lo = j + 2, hi = nb;  // first t with the bit cleared in spec_us[t]: cluster t - 1
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if ((S.spec_us[mid][lane] >> b) & 1u) lo = mid + 1; else hi = mid;
                        }
                        first = min(first, (unsigned)(lo - 1));
                    }
                    first = __reduce_min_sync(kFull, first);
                    if (first != 0xffffffffu) cut = min(cut, (int)first);
                    int slot = 0;
                    if (ins) {
                        if (wn < F.maxNum) {
                            slot = wn;
                            ++wn;
                            K = K0 - S.lnn[wn - D.n];
                        } else {
                            slot = -1;
                        }
                    }
                    if (lane == 0) { S.acc_list[wna] = chosen; S.acc_slot[wna] = slot; }
                    ++wna;
                    if (wfa < 0) wfa = chosen;
                    ++wnc;
                    ++j;
                }
                depth = (j < nb) ? max(1, min(depth, 2 * j) / 2 + 1) : min(32, 2 * depth);
            }
            // no barrier here: warp 0 seeds the next round next, and the other warps
            // read its results only after the barrier that follows the seeding
        }
        if (tid == 0) {
            if (spec && wna > 0) void_next(R, D.step + 1);
            S.misc[0] = wna; S.misc[1] = wnc; S.misc[2] = wfa; S.misc[3] = wn;
            atomicAdd(&R.counters[12], (unsigned long long)nrounds);
        }
        __syncthreads();
        PHASE(2);

        // ---- phase 3: write accepted poses, then cell lists and counts
        const int na = S.misc[0];
        if (ins) {
            for (int a = warp; a < na; a += nwarps) {
                const int slot = S.acc_slot[a];
                if (slot < 0) continue;
                const int i = S.acc_list[a];
                const int res = F.startRes + slot;
                const int2 sp = R.gspan[res];
                const float4 c = S.c[i];
                if (lane < ns) {  // the pose's sites as built by the pose-energy kernel
                    const float4 p = R.psite[i * kMaxSites + lane];
                    R.xyzq[sp.x + lane] = p;
                    R.atype[sp.x + lane] = F.stype[lane];
                    if (Pme && R.pme) pme_move_site(R, false, 0.f, 0.f, 0.f, true, p.x, p.y, p.z, p.w);
                }
                if (lane == 0) R.gcen[res] = make_float4(c.x, c.y, c.z, 0.0f);
            }
            __syncthreads();
            if (warp == 0) {
                for (int a0 = 0; a0 < na; a0 += 32) {
                    const int a = a0 + lane;
                    const bool act = a < na && S.acc_slot[a] >= 0;
                    int g = 0, cn = -1;
                    if (act) {
                        const float4 c = S.c[S.acc_list[a]];
                        g = F.startRes + S.acc_slot[a];
                        cn = cell_of(R, c.x, c.y, c.z);
                    }
                    warp_cell_moves(R, lane, act, g, false, cn);
                }
                if (lane == 0) R.totalNum[D.ftype] = S.misc[3];
            }
        } else {
            for (int a = warp; a < na; a += nwarps) {
                const int i = S.acc_list[a];
                const int res = F.startRes + R.pslot[i];
                const int2 sp = R.gspan[res];
                if (lane < ns) {  // moved sites as built by the pose-energy kernel; the charge stays
                    const float4 p = R.psite[i * kMaxSites + lane];
                    float* dst = reinterpret_cast<float*>(R.xyzq + sp.x + lane);
                    if (Pme && R.pme) {
                        const float4 o = R.xyzq[sp.x + lane];
                        pme_move_site(R, true, o.x, o.y, o.z, true, p.x, p.y, p.z, o.w);
                    }
                    dst[0] = p.x;
                    dst[1] = p.y;
                    dst[2] = p.z;
                }
            }
            __syncthreads();
            if (warp == 0 && D.move == MV_TRANSLATE) {
                for (int a0 = 0; a0 < na; a0 += 32) {
                    const int a = a0 + lane;
                    bool act = a < na;
                    int res = 0, cn = -1;
                    float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (act) {
                        const int i = S.acc_list[a];
                        res = F.startRes + R.pslot[i];
                        c = S.c[i];
                        R.gcen[res] = make_float4(c.x, c.y, c.z, 0.0f);
                        cn = cell_of(R, c.x, c.y, c.z);
                        const int cp = R.gcell[res];
                        act = cp < 0 || cp / R.cap != cn;  // only groups that change cell
                    }
                    warp_cell_moves(R, lane, act, res, true, cn);
                    // groups that stay in their cell: new centre in their entry (wherever
                    // the moves above have shifted it)
                    if (a < na && !act) {
                        const int cp = R.gcell[res];
                        if (cp >= 0) R.cell_ent[cp].c = make_float4(c.x, c.y, c.z, __int_as_float(res));
                    }
                    __syncwarp();
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        if (Pme && R.pme && D.move != MV_DELETE && S.misc[0] > 0) *R.pme_dirty = 1;  // the mesh charges moved
        if (D.move != MV_DELETE) {  // running energy: accepted moves in commit order
            double et = *R.energy;
            const int na = S.misc[0];
            for (int a = 0; a < na; ++a)
                if (D.move != MV_INSERT || S.acc_slot[a] >= 0) et += S.ephys[S.acc_list[a]];
            *R.energy = et;
        }
        R.counters[0] += 1ull;
        R.counters[1] += (unsigned long long)(k * D.nvar);
        if (logging) {
            gcmc_step_log L;
            L.step = D.step;
            L.move = D.move;
            L.ftype = D.ftype;
            L.k = k;
            L.n_before = D.n;
            L.n_after = S.misc[3];
            L.n_clusters = S.misc[1];
            L.n_accept = S.misc[0];
            L.first_accept = S.misc[2];
            L.slot = (D.move == MV_DELETE && k > 0) ? D.del_slot : -1;
            L.e_sum = esum;
            L.e_total = *R.energy;
            R.log[D.step] = L;
        }
    }
    __syncthreads();
    PHASE(3);
    if (spec) {  // the next step's speculation stands iff this step accepted nothing
        if (tid == 0) *R.other->valid = S.misc[0] == 0 ? 1 : 0;
    } else {
        prepare_step(R, D.step + 1, reinterpret_cast<int*>(S.nb));  // the bit matrix is dead here
    }
    PHASE(4);
#undef PHASE
}

template <bool Pme>
__global__ void __launch_bounds__(kAcceptThreads, 1) k_accept(const RepDev* __restrict__ reps, int nrep, int spec) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    pdl_wait();  // a speculating graph launches this kernel as a dependent of the pose energies
    accept_step<Pme>(reps[blockIdx.x], spec, smem_raw);
}
template __global__ void k_accept<false>(const RepDev* __restrict__, int, int);
template __global__ void k_accept<true>(const RepDev* __restrict__, int, int);

}  // namespace gcmc
