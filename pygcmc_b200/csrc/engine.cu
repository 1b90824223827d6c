// Host engine and C ABI (include/gcmc_b200.h).
//
// A context owns the device-resident state of nrep independent replicas
// (structure-of-arrays, float4 atoms and group centres, a cell grid over group
// centres) and a CUDA graph of `kGraphSteps` MC steps; each step is one
// k_energy launch (every replica's pose items) and one k_accept launch (one
// CTA per replica) that also prepares the next step, so the whole step loop
// runs without host round trips.  A one-replica context speculates instead
// (build_spec_graph): the next step is prepared and its pose energies
// evaluated beside the accept kernel, and kept when the step accepts nothing.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>


#include "accept.cuh"
#include "grad.cuh"
#include "persist.cuh"

using namespace gcmc;

namespace {

constexpr int kGraphSteps = 32;
static_assert(kGraphSteps % 2 == 0, "a speculating graph ends on its start parity");
constexpr int kMaxRep = 256;
thread_local int g_last_status = GCMC_OK;

// GCMC_B200_TRACE=1 (read once): every drop-in call (gcmc_run_gcmc,
// runGCMC_cuda, gcmc_run_batch) prints its phases' host wall times to stderr.
bool trace_on() {
    static const bool on = [] {
        const char* e = std::getenv("GCMC_B200_TRACE");
        return e && *e && *e != '0';
    }();
    return on;
}
double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// phase stamps of the current call (refill: validated, host set-up done, set-up enqueued)
thread_local double g_trace[4];
// host set-up split, host time summed over the call's replicas (and threads):
// layout and cell sizing, allocations, per-cell work table and PME host set-up,
// uploads enqueued
std::atomic<long long> g_setup_ns[4];

// fn(r) for r in [0, n) on up to 16 host threads (inline for one replica or
// one hardware thread); a worker first selects `device` (>= 0) for its CUDA
// calls.  Returns the first failing replica's status.
template <class F>
int for_each_rep(int n, int device, F fn) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nt = std::min(n, std::min(hw, 16));
    std::vector<int> st(n, GCMC_OK);
    if (nt <= 1) {
        for (int r = 0; r < n; ++r)
            if ((st[r] = fn(r)) != GCMC_OK) return st[r];
        return GCMC_OK;
    }
    std::vector<std::thread> pool;
    pool.reserve(nt);
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            if (device >= 0 && cudaSetDevice(device) != cudaSuccess) {
                cudaGetLastError();
                for (int r = t; r < n; r += nt) st[r] = GCMC_ERR_CUDA;
                return;
            }
            for (int r = t; r < n; r += nt) st[r] = fn(r);
        });
    for (auto& th : pool) th.join();
    for (int r = 0; r < n; ++r)
        if (st[r] != GCMC_OK) return st[r];
    return GCMC_OK;
}

struct RepHost {
    int natoms = 0, ngroups = 0, ncell = 0, cap = 0, ntypes = 0, G = 0, ffX = 0, ffY = 0, mcsteps = 0;
    int nslab = 0, log_cap = 0, log_kmax = 0;
    int slab_cap = 0;  // per-variant slab partials allocated per pose (>= the largest step split)
    int host_end = 0;
    int2 frag_atoms = make_int2(0, 0);  // atom range of the fragment slots (the caller's layout)
    std::vector<int> startRes, maxNum, moves_host;
    // allocated element count of each device buffer, keyed by the offset of its
    // pointer member (grown on demand, reused on refill)
    std::map<size_t, size_t> capn;
    // device allocations (owned)
    float4* xyzq = nullptr;
    int* atype = nullptr;
    float4* gcen = nullptr;
    int2* gspan = nullptr;
    int* cell_count = nullptr;
    CellEnt* cell_ent = nullptr;
    Atom* raw_atoms = nullptr;      // the caller's arrays as uploaded, unpacked on the device
    residue* raw_groups = nullptr;
    float* raw_grid = nullptr;
    uint32_t* raw_bits = nullptr;   // gcmc_grid_bits words as uploaded
    int* bits_blk = nullptr;        // per-block marked-voxel counts, then offsets (+ total)
    int* gcell = nullptr;
    float4* grid = nullptr;
    float2* lj = nullptr;
    int* moves = nullptr;
    FragDev* frag = nullptr;
    int* totalNum = nullptr;
    StepDesc* desc = nullptr;
    float4* pcen = nullptr;
    int* pslot = nullptr;
    double* epart = nullptr;
    uint32_t* nbr = nullptr;
    gcmc_step_log* log = nullptr;
    double* logE = nullptr;
    unsigned long long* counters = nullptr;
    int* err = nullptr;
    double* energy = nullptr;
    float4* psite = nullptr;
    // per-step scratch of the speculating copy (single-replica contexts)
    StepDesc* desc2 = nullptr;
    float4* pcen2 = nullptr;
    int* pslot2 = nullptr;
    double* epart2 = nullptr;
    uint32_t* nbr2 = nullptr;
    double* pgum2 = nullptr;
    double* plnu2 = nullptr;
    float4* psite2 = nullptr;
    int* valid2 = nullptr;                  // [2] per copy
    int* abort2 = nullptr;                  // [2] per copy
    int* sstep2 = nullptr;                  // [2] per copy
    unsigned long long* pending2 = nullptr; // [2] per copy
    double* pgum = nullptr;
    double* plnu = nullptr;
    int* pbin = nullptr;       // tiled contexts: the step's pose entries by block
    int4* tiles = nullptr;     //   and its tiles
    int* pbin2 = nullptr;      //   (the speculating copy's)
    int4* tiles2 = nullptr;
    int* wcost = nullptr;      // per-pose-warp kernel: each cell's window work (fixed atoms)
    int* pnslab = nullptr;     //   the step's ranges per pose variant
    int* pitem = nullptr;      //   and its item list
    int* pnslab2 = nullptr;    //   (the speculating copy's)
    int* pitem2 = nullptr;
    float* fpart = nullptr;
    float4* fbprop = nullptr;
    int* fbcnt = nullptr;
    float* logF = nullptr;
    // smooth PME (Ewald runs)
    int pme = 0;
    int pme_n[3] = {0, 0, 0};
    int nfix_atoms = 0;
    double* pme_q = nullptr;      // this step's spread charges
    double* pme_phi = nullptr;    // potential on the mesh
    double2* pme_spec = nullptr;  // half spectrum
    double* pme_g = nullptr;      // influence function on the half spectrum
    int* pme_dirty = nullptr;     // 1: the spread charges changed since phi was computed
    double pme_key[7] = {0, 0, 0, 0, 0, 0, 0};  // mesh, box and alpha the influence function in pme_g is for
    const double* pme_g_for = nullptr;          // the buffer it was written to
};

}  // namespace

struct gcmc_ctx {
    int nrep = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<RepHost> reps;
    std::vector<RepDev> repdev;
    RepDev* d_reps = nullptr;
    cudaGraphExec_t gexec = nullptr;
    // speculation (one replica, one branch, no PME, no force bias): the next step's pose
    // energies run beside the accept kernel; a second descriptor copy holds every other
    // step's scratch, and the step loop has one graph per parity of its first step
    bool spec = false;
    RepDev repdev_b{};
    RepDev* d_reps_b = nullptr;
    cudaGraphExec_t gexec_spec[2] = {nullptr, nullptr};
    int per_sm_e = 1;      // pose-energy CTAs per SM
    int gridE = 0;       // pose-energy CTAs for all replicas
    int branches = 1;    // independent chains in the captured step loop
    int ebps = 0;        // requested pose-energy CTAs per SM (0 = occupancy limit)
    int evar = 0;        // pose-energy kernel variant: 0 = 3 CTAs per SM, 1 = 4 CTAs per SM
    int fb = 0;          // force-biased moves: two pose-energy launches per step (k_energy_fb)
    bool fb_mixed = false;  // several replicas whose move schedules differ
    bool tiled = false;  // pose energies by k_energy_tiles (every replica allows it)
    bool pme_any = false; // some replica runs Ewald electrostatics
    bool dual_any = false; // some replica evaluates translate / rotate changes in the difference form
    bool persist = false;   // the step loop as one cooperative launch (k_persist) instead of a graph
    GridSync* d_sync = nullptr;
    int grid_persist = 0;   // k_persist CTAs (one per SM)
    long long spin_cap = kPersistSpinCap;
    int gridF = 0;       // k_energy_fb CTAs
    std::vector<int> br_off;  // branch b holds replicas [br_off[b], br_off[b+1])
    // ordering of calls that launch on a caller's stream against the context's
    // stream (created once, so such calls allocate nothing): ev_ctx marks the
    // context's work so far, ev_call the caller's launches
    cudaEvent_t ev_ctx = nullptr, ev_call = nullptr;
};

namespace {

#define CK(call)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            std::fprintf(stderr, "gcmc_b200: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return GCMC_ERR_CUDA;                                                       \
        }                                                                               \
    } while (0)

template <typename T>
int dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    CK(cudaMalloc((void**)p, n * sizeof(T)));
    return GCMC_OK;
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

// (Re)allocate *p for n elements unless it already holds at least n.
template <typename T>
int ensure(T** p, size_t* cap, size_t n) {
    if (n == 0) n = 1;
    if (*p && *cap >= n) return GCMC_OK;
    dfree(*p);
    *cap = 0;
    int st = dalloc(p, n);
    if (st == GCMC_OK) *cap = n;
    return st;
}

void free_rep(RepHost& h) {
    dfree(h.xyzq); dfree(h.atype); dfree(h.gcen); dfree(h.gspan); dfree(h.cell_count); dfree(h.cell_ent);
    dfree(h.gcell); dfree(h.grid); dfree(h.lj); dfree(h.moves); dfree(h.frag); dfree(h.totalNum);
    dfree(h.desc); dfree(h.pcen); dfree(h.pslot); dfree(h.epart); dfree(h.nbr); dfree(h.log);
    dfree(h.logE); dfree(h.counters); dfree(h.err);
    dfree(h.energy); dfree(h.pgum); dfree(h.psite);
    dfree(h.raw_atoms); dfree(h.raw_groups); dfree(h.raw_grid); dfree(h.raw_bits); dfree(h.bits_blk);
    dfree(h.desc2); dfree(h.pcen2); dfree(h.pslot2); dfree(h.epart2); dfree(h.nbr2); dfree(h.pgum2); dfree(h.plnu2);
    dfree(h.psite2); dfree(h.valid2); dfree(h.abort2); dfree(h.sstep2); dfree(h.pending2); dfree(h.plnu); dfree(h.fpart); dfree(h.fbprop); dfree(h.fbcnt); dfree(h.logF);
    dfree(h.pme_q); dfree(h.pme_phi); dfree(h.pme_spec); dfree(h.pme_g); dfree(h.pme_dirty);
    dfree(h.pbin); dfree(h.tiles); dfree(h.pbin2); dfree(h.tiles2);
    dfree(h.wcost); dfree(h.pnslab); dfree(h.pitem); dfree(h.pnslab2); dfree(h.pitem2);
    h.capn.clear();
}

// Host copy of the device cell index function (floor((x - start) * invLc) mod nc),
// used only to size the cell capacity.
int host_cell(float x, float start, float invLc, int nc) {
    volatile float d = x - start;
    volatile float f = d * invLc;
    int c = (int)std::floor((float)f);
    c %= nc;
    return c < 0 ? c + nc : c;
}

// frag_atoms (optional): the atom range [x, y) the fragment slots cover (empty: x >= y)
int validate(const gcmc_replica_in& in, int2* frag_atoms = nullptr) {
    const InfoStruct* I = in.info;
    if (!I || !in.fragmentInfo || !in.residueInfo || !in.atomInfo || !in.ff) return GCMC_ERR_ARG;
    if (I->fragTypeNum < 1 || I->totalResNum < 0 || I->totalAtomNum < 0 || I->mcsteps < 0) return GCMC_ERR_ARG;
    if (I->mcsteps > 0 && !in.moveArray) return GCMC_ERR_ARG;
    if (!(I->cutoff > 0.0f) || !(I->grid_dx > 0.0f)) return GCMC_ERR_ARG;
    for (int d = 0; d < 3; ++d)
        if (!(I->cryst[d] > 0.0f)) return GCMC_ERR_ARG;
    if (I->ffXNum < 1 || I->ffYNum < 1) return GCMC_ERR_ARG;
    if (I->totalAtomNum >= (1 << 26) || I->totalResNum >= (1 << 26)) return GCMC_ERR_LIMIT;
    const AtomArray* F = in.fragmentInfo;
    const residue* R = in.residueInfo;
    int prev_end = F[0].startRes;
    if (prev_end < 0) return GCMC_ERR_ARG;
    bool any_insert = false;
    int alo = I->totalAtomNum, ahi = 0;
    for (int t = 0; t < I->fragTypeNum; ++t) {
        const AtomArray& f = F[t];
        if (f.num_atoms < 1 || f.num_atoms > kMaxSites) return GCMC_ERR_LIMIT;
        if (f.confBias < 1) return GCMC_ERR_ARG;
        if (f.confBias > kMaxPoses) return GCMC_ERR_LIMIT;
        if (f.totalNum < 0 || f.maxNum < f.totalNum) return GCMC_ERR_ARG;
        if (f.startRes != prev_end || f.startRes + f.maxNum > I->totalResNum) return GCMC_ERR_ARG;
        prev_end = f.startRes + f.maxNum;
        for (int s = 0; s < f.num_atoms; ++s)
            if (f.atoms[s].type < 0 || f.atoms[s].type >= I->ffXNum) return GCMC_ERR_ARG;
        for (int j = 0; j < f.maxNum; ++j) {
            const residue& r = R[f.startRes + j];
            if (r.atomNum != f.num_atoms || r.atomStart < 0 || r.atomStart + r.atomNum > I->totalAtomNum)
                return GCMC_ERR_ARG;
            alo = std::min(alo, r.atomStart);
            ahi = std::max(ahi, r.atomStart + r.atomNum);
        }
        for (int j = 0; j < f.totalNum; ++j) {
            const residue& r = R[f.startRes + j];
            for (int s = 0; s < r.atomNum; ++s) {
                int ty = in.atomInfo[r.atomStart + s].type;
                if (ty < 0 || ty >= I->ffYNum) return GCMC_ERR_ARG;
            }
        }
    }
    for (int g = 0; g < F[0].startRes; ++g) {
        const residue& r = R[g];
        if (r.atomNum < 0 || r.atomStart < 0 || r.atomStart + r.atomNum > I->totalAtomNum) return GCMC_ERR_ARG;
        for (int s = 0; s < r.atomNum; ++s) {
            int ty = in.atomInfo[r.atomStart + s].type;
            if (ty < 0 || ty >= I->ffYNum) return GCMC_ERR_ARG;
        }
    }
    for (int s = 0; s < I->mcsteps; ++s) {
        int mv = in.moveArray[s];
        if (mv < 0 || mv >= 4 * I->fragTypeNum) return GCMC_ERR_ARG;
        if ((mv & 3) == 0) any_insert = true;
    }
    if (any_insert && (I->totalGridNum < 1 || !in.grid)) return GCMC_ERR_ARG;
    if (frag_atoms) *frag_atoms = make_int2(alo, ahi);
    return GCMC_OK;
}

// smallest n' >= n whose prime factors are 2 and 3 (the mesh transforms' line
// lengths; 0 when that exceeds kFftMax)
int smooth_size(int n) {
    for (int m = std::max(n, 1); m <= kFftMax; ++m)
        if (fft_size_ok(m)) return m;
    return 0;
}

// Smooth-PME influence function on the half spectrum (FP64):
// G(m) = K exp(-pi^2 m^2 / alpha^2) / (pi V m^2) * prod_d |b_d(k_d)|^2, G(0) = 0,
// |b(k)|^2 = 1 / |sum_{j=0}^{2} M4(j + 1) e^{2 pi i k j / n}|^2 (order-4 B-spline moduli).
void pme_influence(const int n[3], const float cryst[3], double alpha, double* G) {
    const double V = (double)cryst[0] * cryst[1] * cryst[2];
    const double M4[3] = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
    std::vector<double> bm[3];
    for (int a = 0; a < 3; ++a) {
        bm[a].resize(n[a]);
        for (int k = 0; k < n[a]; ++k) {
            double re = 0.0, im = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double th = 2.0 * M_PI * k * j / n[a];
                re += M4[j] * std::cos(th);
                im += M4[j] * std::sin(th);
            }
            bm[a][k] = 1.0 / (re * re + im * im);
        }
    }
    const int nh = n[2] / 2 + 1;
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            for (int k = 0; k < nh; ++k) {
                const double m0 = (i <= n[0] / 2 ? i : i - n[0]) / (double)cryst[0];
                const double m1 = (j <= n[1] / 2 ? j : j - n[1]) / (double)cryst[1];
                const double m2 = k / (double)cryst[2];
                const double mm = m0 * m0 + m1 * m1 + m2 * m2;
                double g = 0.0;
                if (mm > 0.0)
                    g = (double)kCoulomb * std::exp(-M_PI * M_PI * mm / (alpha * alpha)) / (M_PI * V * mm) *
                        bm[0][i] * bm[1][j] * bm[2][k];
                G[((size_t)i * n[1] + j) * nh + k] = g;
            }
}

// The caller's arrays (uploaded unchanged) into the engine's layout: atoms ->
// (x, y, z, charge) + type, residues -> centre + (atomStart, atomNum), cavity
// grid points -> float4.
__global__ void k_unpack_atoms(const Atom* __restrict__ in, float4* __restrict__ xyzq, int* __restrict__ atype,
                               int n) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const Atom A = in[a];
        xyzq[a] = make_float4(A.position[0], A.position[1], A.position[2], A.charge);
        atype[a] = A.type;
    }
}
__global__ void k_unpack_groups(const residue* __restrict__ in, float4* __restrict__ gcen, int2* __restrict__ gspan,
                                int n) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const residue R = in[g];
        gcen[g] = make_float4(R.position[0], R.position[1], R.position[2], 0.0f);
        gspan[g] = make_int2(R.atomStart, R.atomNum);
    }
}
__global__ void k_unpack_grid(const float* __restrict__ in, float4* __restrict__ grid, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        grid[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.0f);
}

// Cavity grid from a gcmc_grid_bits record: base point k = the k-th marked
// voxel.  Three launches, one word per thread: marked voxels per block of
// kBitsThreads words (k_bits_count), an exclusive scan of the block counts with
// the total checked against the expected point count (k_bits_scan), and the
// points of each word at its offset (k_bits_expand).
constexpr int kBitsThreads = 256;
constexpr long long kIntMax = 0x7fffffffll;

// the marked bits of word w (bits past the last voxel cleared)
__device__ __forceinline__ uint32_t bits_word(const uint32_t* words, long long w, long long nvox) {
    uint32_t b = words[w];
    const long long rest = nvox - w * 32;
    if (rest < 32) b &= (1u << rest) - 1u;
    return b;
}

// Exclusive prefix of v over the block (kBitsThreads threads); *total = the sum.
__device__ __forceinline__ int bits_block_scan(int v, int* total) {
    __shared__ int warp_sum[kBitsThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    int before = 0, all = 0;
    for (int w = 0; w < kBitsThreads / 32; ++w) {
        if (w < wid) before += warp_sum[w];
        all += warp_sum[w];
    }
    __syncthreads();
    *total = all;
    return before + x - v;
}

__global__ void __launch_bounds__(kBitsThreads) k_bits_count(const uint32_t* __restrict__ words, long long nwords,
                                                              long long nvox, int* __restrict__ blk) {
    const long long w = (long long)blockIdx.x * kBitsThreads + threadIdx.x;
    const int c = w < nwords ? __popc(bits_word(words, w, nvox)) : 0;
    int total = 0;
    bits_block_scan(c, &total);
    if (threadIdx.x == 0) blk[blockIdx.x] = total;
}

// One CTA: blk[0, nblk) -> exclusive offsets; blk[nblk] = total; error bit when total != expect.
__global__ void __launch_bounds__(kBitsThreads) k_bits_scan(int* __restrict__ blk, int nblk, int expect,
                                                             int* __restrict__ err) {
    long long carry = 0;
    for (int b0 = 0; b0 < nblk; b0 += kBitsThreads) {
        const int b = b0 + threadIdx.x;
        const int v = b < nblk ? blk[b] : 0;
        int total = 0;
        const int ex = bits_block_scan(v, &total);
        if (b < nblk) blk[b] = (int)(carry + ex < kIntMax ? carry + ex : kIntMax);
        carry += total;
    }
    if (threadIdx.x == 0) {
        blk[nblk] = (int)(carry < kIntMax ? carry : kIntMax);
        if (carry != expect) atomicOr(err, ERR_GRID_BITS);
    }
}

__global__ void __launch_bounds__(kBitsThreads) k_bits_expand(const uint32_t* __restrict__ words, long long nwords,
                                                               long long nvox, const int* __restrict__ blk, int n1,
                                                               int n2, double s0, double s1, double s2, double dx,
                                                               float4* __restrict__ grid, int npts) {
    const long long w = (long long)blockIdx.x * kBitsThreads + threadIdx.x;
    uint32_t b = w < nwords ? bits_word(words, w, nvox) : 0u;
    int total = 0;
    long long k = (long long)blk[blockIdx.x] + bits_block_scan(__popc(b), &total);
    if (!b) return;
    // voxel of the word's first bit, then walk z (and carry into y, x) bit by bit
    const long long plane = (long long)n1 * n2, v0 = w * 32;
    long long x = v0 / plane;
    const long long r0 = v0 - x * plane;
    int y = (int)(r0 / n2), z = (int)(r0 - (long long)y * n2);
    int at = 0;
    while (b) {
        const int bit = __ffs(b) - 1;
        b &= b - 1u;
        for (; at < bit; ++at)
            if (++z == n2) {
                z = 0;
                if (++y == n1) {
                    y = 0;
                    ++x;
                }
            }
        if (k < npts)
            grid[k] = make_float4(__double2float_rn(__dadd_rn(__dmul_rn((double)x, dx), s0)),
                                  __double2float_rn(__dadd_rn(__dmul_rn((double)y, dx), s1)),
                                  __double2float_rn(__dadd_rn(__dmul_rn((double)z, dx), s2)), 0.0f);
        ++k;
    }
}
int unpack_blocks(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

int energy_warps(int device, int evar, int ebps, int spare_sms);

// Speculation applies to one replica on one branch, without PME or force bias.
bool spec_eligible(int nrep, const gcmc_replica_in* ins, const gcmc_options& opt) {
    const bool pme = opt.pme > 0 || (opt.pme == 0 && ins[0].info->PME != 0);
    return nrep == 1 && opt.speculate >= 0 && opt.proposal != 2 && opt.branches <= 1 && !pme;
}

int setup_rep(gcmc_ctx* ctx, int r, const gcmc_replica_in& in, const gcmc_options& opt) {
    const bool trace = trace_on();
    double tp = trace ? now_ms() : 0.0;
    auto stamp = [&](int k) {
        if (!trace) return;
        const double t = now_ms();
        g_setup_ns[k] += (long long)((t - tp) * 1e6);
        tp = t;
    };
    const InfoStruct* I = in.info;
    RepHost& h = ctx->reps[r];
    RepDev& d = ctx->repdev[r];
    std::memset(&d, 0, sizeof(d));
    h.startRes.clear();
    h.maxNum.clear();
    h.host_end = 0;
    h.natoms = I->totalAtomNum;
    h.ngroups = I->totalResNum;
    h.ntypes = I->fragTypeNum;
    // no grid array (accepted when the schedule holds no insertion): no base points
    h.G = (in.grid && I->totalGridNum > 0) ? I->totalGridNum : 0;
    h.ffX = I->ffXNum;
    h.ffY = I->ffYNum;
    h.mcsteps = I->mcsteps;

    // geometry: cells of edge >= cutoff/R, with a 1e-4 margin so rounding in the
    // cell index can never push an included group outside the +-R window
    const int Rc = opt.cells_per_cutoff > 0 ? opt.cells_per_cutoff : 2;
    for (int a = 0; a < 3; ++a) {
        d.L[a] = I->cryst[a];
        d.start[a] = I->startxyz[a];
        int nc = (int)std::floor((double)I->cryst[a] * Rc / I->cutoff * (1.0 - 1e-4));
        nc = std::max(1, nc);
        d.nc[a] = nc;
        d.invLc[a] = (float)nc / I->cryst[a];
        d.span[a] = std::min(2 * Rc + 1, nc);
    }
    d.range = Rc;
    d.max_split = std::max(1, d.span[0] * d.span[1] * d.span[2] / 8);
    // default: one wave of the pose-energy grid (its resident warps), the most items a
    // step can have without a second round of warps (speculating: without the SM that
    // the accept kernel holds meanwhile)
    d.split_items = opt.split_items > 0 ? opt.split_items
                                        : energy_warps(ctx->device, opt.energy_variant == 1 ? 1 : 0,
                                                       opt.energy_blocks_per_sm, ctx->spec ? 1 : 0);
    h.nslab = std::max(d.span[2], d.max_split);
    h.slab_cap = std::max(h.nslab, 2 * d.max_split);  // a dual step may split its poses twice as finely
    h.ncell = d.nc[0] * d.nc[1] * d.nc[2];
    const bool pme_on = opt.pme > 0 || (opt.pme == 0 && I->PME != 0);
    // translate / rotate energy changes in the pairwise-difference form (atom ids
    // below 2^24 leave bits 24-25 of an atom entry for the inclusion flags); a
    // translate moves the centre by at most grid_dx (reference proposals) or
    // trn_step / 2 (symmetric) per axis, i.e. within dmargin cells
    d.dual = (opt.pair_delta >= 0 && !pme_on && opt.proposal != 2 && I->totalAtomNum < (1 << 24)) ? 1 : 0;
    {
        const double shift = opt.proposal == 0 ? (double)I->grid_dx : 0.5 * (double)opt.trn_step;
        int m = 0;
        for (int a = 0; a < 3; ++a)
            m = std::max(m, (int)std::ceil(shift * (1.0 + 1e-6) / ((double)I->cryst[a] / d.nc[a])));
        d.dmargin = m;
    }
    // tiled pose energies: blocks of B^3 cells, windows of B + 2R cells per axis (a
    // translate step's: B + 2 (R + dmargin))
    {
        const int B = std::max(1, opt.tile_cells > 0 ? opt.tile_cells : Rc);
        d.tblk = B;
        long long nblk = 1, nwin = 1;
        for (int a = 0; a < 3; ++a) {
            d.nbk[a] = (d.nc[a] + B - 1) / B;
            d.tspan[a] = std::min(B + 2 * Rc, d.nc[a]);
            nblk *= d.nbk[a];
            nwin *= std::min(B + 2 * (Rc + (d.dual ? d.dmargin : 0)), d.nc[a]);
        }
        int maxga = 0;
        for (int g = 0; g < in.fragmentInfo[0].startRes; ++g) maxga = std::max(maxga, in.residueInfo[g].atomNum);
        for (int t = 0; t < I->fragTypeNum; ++t) maxga = std::max(maxga, in.fragmentInfo[t].num_atoms);
        d.tiled = (opt.energy_kernel > 0 && !pme_on && opt.proposal != 2 && nblk <= kMaxBlocks &&
                   nwin <= kTileCells && maxga <= kTileMaxGroupAtoms) ? 1 : 0;
    }
    d.cutoff = I->cutoff;
    d.grid_dx = I->grid_dx;
    d.trn_step = opt.trn_step;
    d.rot_max = opt.rot_max;
    d.proposal = opt.proposal;
    d.fb = opt.proposal == 2 ? 1 : 0;
    d.fb_ht = opt.fb_trn > 0.0f ? opt.fb_trn : 0.5f;
    d.fb_hr = opt.fb_rot > 0.0f ? opt.fb_rot : (float)(10.0 * M_PI / 180.0);
    d.fb_at = d.fb_ar = (float)((double)kFbLambda * kBeta);
    d.lncav = std::log((double)I->cavityFactor);
    d.nfixed = in.fragmentInfo[0].startRes;
    d.ntypes = I->fragTypeNum;
    d.ffX = I->ffXNum;
    d.ffY = I->ffYNum;
    d.G = h.G;
    d.mcsteps = I->mcsteps;
    d.seed = I->seed;
    d.replica = opt.replica + (uint32_t)r;
    d.step_base = opt.step_offset;
    d.run_end = 0;

    // the per-group periodic image is exact when every pair of an included
    // group lies within half a box: cutoff + group radius + fragment radius < L/2
    double rg = 0.0, rf = 0.0;
    for (int g = 0; g < d.nfixed; ++g) {
        const residue& rs = in.residueInfo[g];
        for (int s = 0; s < rs.atomNum; ++s) {
            const Atom& a = in.atomInfo[rs.atomStart + s];
            double dx = a.position[0] - rs.position[0], dy = a.position[1] - rs.position[1],
                   dz = a.position[2] - rs.position[2];
            rg = std::max(rg, std::sqrt(dx * dx + dy * dy + dz * dz));
        }
    }
    for (int t = 0; t < h.ntypes; ++t) {
        const AtomArray& f = in.fragmentInfo[t];
        for (int s = 0; s < f.num_atoms; ++s) {
            double x = f.atoms[s].position[0], y = f.atoms[s].position[1], z = f.atoms[s].position[2];
            rf = std::max(rf, std::sqrt(x * x + y * y + z * z));
        }
    }
    rf += 0.5;
    const double reach = (double)I->cutoff + std::max(rg, rf) + rf;
    d.pair_image = 0;
    d.fast_incl = 1;
    for (int a = 0; a < 3; ++a) {
        d.invL[a] = 1.0f / I->cryst[a];
        if (reach >= 0.5 * I->cryst[a]) d.pair_image = 1;
        if ((double)I->cutoff * (1.0 + 1e-3) >= 0.5 * I->cryst[a]) d.fast_incl = 0;
    }
    d.cut2_lo = (float)(((double)I->cutoff * (1.0 - 1e-4)) * ((double)I->cutoff * (1.0 - 1e-4)));
    d.cut2_hi = (float)(((double)I->cutoff * (1.0 + 1e-4)) * ((double)I->cutoff * (1.0 + 1e-4)));

    // cell capacity from the initial occupancy
    std::vector<int> counts(h.ncell, 0);
    auto cell_host = [&](const float* p) {
        int cx = host_cell(p[0], d.start[0], d.invLc[0], d.nc[0]);
        int cy = host_cell(p[1], d.start[1], d.invLc[1], d.nc[1]);
        int cz = host_cell(p[2], d.start[2], d.invLc[2], d.nc[2]);
        return (cz * d.nc[1] + cy) * d.nc[0] + cx;
    };
    int maxcount = 0;
    for (int g = 0; g < d.nfixed; ++g) maxcount = std::max(maxcount, ++counts[cell_host(in.residueInfo[g].position)]);
    for (int t = 0; t < h.ntypes; ++t)
        for (int j = 0; j < in.fragmentInfo[t].totalNum; ++j)
            maxcount = std::max(maxcount, ++counts[cell_host(in.residueInfo[in.fragmentInfo[t].startRes + j].position)]);
    int cap = 32;
    while (cap < 2 * maxcount + 16) cap *= 2;
    if (cap > 4096) return GCMC_ERR_LIMIT;
    h.cap = d.cap = cap;

    // atoms, groups and cavity grid points are uploaded as the caller holds them
    // and unpacked on the device (k_unpack_*): no host-side copies of the
    // large arrays
    std::vector<float2> lj((size_t)h.ffX * h.ffY);
    for (size_t x = 0; x < lj.size(); ++x) {
        float sigma = in.ff[2 * x], eps = in.ff[2 * x + 1];
        lj[x] = make_float2(sigma * sigma * 100.0f, 4.0f * eps);  // gcmc_energy.h:128-130
    }
    std::vector<FragDev> frag(h.ntypes);
    std::vector<int> tot(h.ntypes);
    const double V = (double)I->cryst[0] * (double)I->cryst[1] * (double)I->cryst[2];
    for (int t = 0; t < h.ntypes; ++t) {
        const AtomArray& f = in.fragmentInfo[t];
        FragDev& F = frag[t];
        std::memset(&F, 0, sizeof(F));
        F.startRes = f.startRes;
        F.maxNum = f.maxNum;
        F.confBias = f.confBias;
        F.nsites = f.num_atoms;
        double mu = (double)f.muex * (opt.muex_kcal ? kKcalToKJ : 1.0);
        F.B = kBeta * mu + std::log(V * (double)f.conc * kMolesToMolecules);
        for (int s = 0; s < f.num_atoms; ++s) {
            F.site[s] = make_float4(f.atoms[s].position[0], f.atoms[s].position[1], f.atoms[s].position[2],
                                    f.atoms[s].charge);
            F.stype[s] = f.atoms[s].type;
            F.qnet += (double)f.atoms[s].charge;
        }
        tot[t] = f.totalNum;
        h.startRes.push_back(f.startRes);
        h.maxNum.push_back(f.maxNum);
    }

    stamp(0);
    int st;
#define AL(ptr, n)                                                                          \
    do {                                                                                    \
        const size_t key_ = (size_t)((const char*)&(ptr) - (const char*)&h);                \
        if ((st = ensure(&(ptr), &h.capn[key_], (size_t)(n))) != GCMC_OK) return st;        \
    } while (0)
    AL(h.xyzq, h.natoms); AL(h.atype, h.natoms); AL(h.gcen, h.ngroups); AL(h.gspan, h.ngroups);
    AL(h.cell_count, h.ncell); AL(h.cell_ent, (size_t)h.ncell * cap); AL(h.gcell, h.ngroups);
    AL(h.grid, h.G); AL(h.lj, lj.size()); AL(h.moves, h.mcsteps); AL(h.frag, h.ntypes);
    AL(h.totalNum, h.ntypes); AL(h.desc, 1); AL(h.pcen, kMaxPoses); AL(h.pslot, kMaxPoses);
    AL(h.epart, (size_t)kMaxPoses * 2 * h.slab_cap); AL(h.nbr, (size_t)kMaxPoses * kMaxWords);
    AL(h.counters, 16); AL(h.err, 1);
    AL(h.energy, 1); AL(h.fpart, (size_t)kMaxPoses * 2 * h.slab_cap * 6); AL(h.fbprop, (size_t)kMaxPoses * 2);
    AL(h.fbcnt, kMaxPoses); AL(h.pgum, kMaxPoses); AL(h.plnu, kMaxPoses);
    AL(h.psite, (size_t)kMaxPoses * kMaxSites);
    AL(h.pbin, 2 * kMaxPoses); AL(h.tiles, 2 * kMaxPoses);
    AL(h.wcost, h.ncell); AL(h.pnslab, 2 * kMaxPoses); AL(h.pitem, (size_t)2 * kMaxPoses * h.slab_cap);
    AL(h.raw_atoms, h.natoms); AL(h.raw_groups, h.ngroups);
    // the cavity grid as the caller holds it: the reference's float list, or a voxel bit set
    gcmc_grid_bits gb{};
    long long nvox = 0, nwords = 0;
    int nblk = 0;
    if (opt.grid_bits && h.G > 0) {
        std::memcpy(&gb, in.grid, sizeof(gb));
        if (!(gb.dx > 0.0) || !std::isfinite(gb.dx)) return GCMC_ERR_ARG;
        nvox = 1;
        for (int a = 0; a < 3; ++a) {
            if (gb.n[a] < 1 || !std::isfinite(gb.start[a])) return GCMC_ERR_ARG;
            nvox *= gb.n[a];
            if (nvox > (1ll << 36)) return GCMC_ERR_LIMIT;
        }
        if (h.G > nvox) return GCMC_ERR_ARG;
        nwords = (nvox + 31) / 32;
        nblk = (int)((nwords + kBitsThreads - 1) / kBitsThreads);
        AL(h.raw_bits, (size_t)nwords); AL(h.bits_blk, (size_t)nblk + 1); AL(h.raw_grid, 1);
    } else {
        AL(h.raw_grid, (size_t)3 * h.G);
    }
    if (ctx->spec) {
        AL(h.desc2, 1); AL(h.pcen2, kMaxPoses); AL(h.pslot2, kMaxPoses); AL(h.epart2, (size_t)kMaxPoses * 2 * h.slab_cap);
        AL(h.nbr2, (size_t)kMaxPoses * kMaxWords); AL(h.pgum2, kMaxPoses); AL(h.plnu2, kMaxPoses);
        AL(h.psite2, (size_t)kMaxPoses * kMaxSites); AL(h.valid2, 2); AL(h.abort2, 2); AL(h.sstep2, 2);
        AL(h.pending2, 2); AL(h.pbin2, 2 * kMaxPoses); AL(h.tiles2, 2 * kMaxPoses);
        AL(h.pnslab2, 2 * kMaxPoses); AL(h.pitem2, (size_t)2 * kMaxPoses * h.slab_cap);
    }
    stamp(1);
    // each cell's window work: the fixed atoms in the cells within R of it (box sums along
    // each axis, periodic; the whole axis where the window spans it)
    if (opt.pose_split > 0) {
        const int n0 = d.nc[0], n1 = d.nc[1], n2 = d.nc[2];
        std::vector<int> cnt((size_t)h.ncell, 0), tmp((size_t)h.ncell, 0);
        for (int g = 0; g < d.nfixed; ++g) {
            int c[3];
            for (int a = 0; a < 3; ++a) {
                const double u = ((double)in.residueInfo[g].position[a] - (double)d.start[a]) * (double)d.invLc[a];
                int x = (int)std::floor(u);
                x %= d.nc[a];
                c[a] = x < 0 ? x + d.nc[a] : x;
            }
            cnt[((size_t)c[2] * n1 + c[1]) * n0 + c[0]] += in.residueInfo[g].atomNum;
        }
        auto box = [&](std::vector<int>& src, std::vector<int>& dst, int a) {
            const int n = d.nc[a], R = d.range;
            const bool whole = d.span[a] == n;
            for (int z = 0; z < n2; ++z)
                for (int y = 0; y < n1; ++y)
                    for (int x = 0; x < n0; ++x) {
                        int co[3] = {x, y, z};
                        long long sum = 0;
                        const int lo = whole ? 0 : co[a] - R, hi = whole ? n - 1 : co[a] + R;
                        for (int t = lo; t <= hi; ++t) {
                            int q[3] = {x, y, z};
                            q[a] = ((t % n) + n) % n;
                            sum += src[((size_t)q[2] * n1 + q[1]) * n0 + q[0]];
                        }
                        dst[((size_t)z * n1 + y) * n0 + x] = (int)std::min<long long>(sum, 1ll << 30);
                    }
        };
        box(cnt, tmp, 0);
        box(tmp, cnt, 1);
        box(cnt, tmp, 2);
        // (a copy from pageable memory is staged before the call returns: tmp may go)
        CK(cudaMemcpyAsync(h.wcost, tmp.data(), sizeof(int) * h.ncell, cudaMemcpyHostToDevice, ctx->stream));
    }
    // smooth PME: mesh and influence function
    h.pme = opt.pme > 0 || (opt.pme == 0 && I->PME != 0);
    d.pme = h.pme ? 1 : 0;
    h.nfix_atoms = d.nfixed > 0 ? in.residueInfo[d.nfixed - 1].atomStart + in.residueInfo[d.nfixed - 1].atomNum : 0;
    if (h.pme) {
        const double alpha = opt.pme_alpha > 0.0f ? opt.pme_alpha : 0.32;
        d.pme_alpha = (float)alpha;
        int n[3];
        for (int a = 0; a < 3; ++a) {
            n[a] = opt.pme_grid[a] > 0 ? opt.pme_grid[a] : smooth_size((int)std::ceil(I->cryst[a] / 1.2));
            if (n[a] == 0) return GCMC_ERR_LIMIT;      // box edge over 1.2 kFftMax A
            if (n[a] < 8) return GCMC_ERR_ARG;
            if (!fft_size_ok(n[a])) return GCMC_ERR_LIMIT;  // a mesh size that is not 2^a 3^b <= kFftMax
            d.pme_n[a] = n[a];
        }
        const size_t nr = (size_t)n[0] * n[1] * n[2], nh = (size_t)n[0] * n[1] * (n[2] / 2 + 1);
        AL(h.pme_q, nr); AL(h.pme_phi, nr); AL(h.pme_spec, nh); AL(h.pme_g, nh); AL(h.pme_dirty, 1);
        // the influence function depends only on the mesh, the box and alpha: kept between refills
        const double key[7] = {(double)n[0], (double)n[1], (double)n[2], (double)I->cryst[0], (double)I->cryst[1],
                               (double)I->cryst[2], alpha};
        if (h.pme_g_for != h.pme_g || std::memcmp(key, h.pme_key, sizeof(key)) != 0) {
            std::vector<double> G(nh);
            pme_influence(n, I->cryst, alpha, G.data());
            CK(cudaMemcpyAsync(h.pme_g, G.data(), sizeof(double) * nh, cudaMemcpyHostToDevice, ctx->stream));
            std::memcpy(h.pme_key, key, sizeof(key));
            h.pme_g_for = h.pme_g;
        }
        CK(cudaMemsetAsync(h.pme_phi, 0, sizeof(double) * nr, ctx->stream));
        const int fft_smem = 2 * kFftLines * kFftMax * (int)sizeof(double2);
        CK(cudaFuncSetAttribute(k_pme_rows_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, fft_smem));
        CK(cudaFuncSetAttribute(k_pme_axis, cudaFuncAttributeMaxDynamicSharedMemorySize, fft_smem));
        CK(cudaFuncSetAttribute(k_pme_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, fft_smem));
        for (int a = 0; a < 3; ++a) h.pme_n[a] = n[a];
        d.pme_phi = h.pme_phi;
        d.pme_q = h.pme_q;
        d.pme_spec = h.pme_spec;
        d.pme_g = h.pme_g;
        d.pme_dirty = h.pme_dirty;
        d.pme_bgc = (double)kCoulomb * M_PI / (2.0 * V * alpha * alpha);
        double qf = 0.0;
        for (int a = 0; a < h.nfix_atoms; ++a) qf += (double)in.atomInfo[a].charge;
        d.pme_qfix = qf;
    }
    h.log_cap = std::max(0, std::min(opt.log_steps, h.mcsteps));
    h.log_kmax = std::max(1, std::min(opt.log_kmax > 0 ? opt.log_kmax : 1, kMaxPoses));
    if (h.log_cap > 0) {
        AL(h.log, h.log_cap);
        AL(h.logE, (size_t)h.log_cap * h.log_kmax);
        if (d.fb) AL(h.logF, (size_t)h.log_cap * h.log_kmax * 12);
    }
#undef AL
    stamp(2);
    cudaStream_t s = ctx->stream;
    if (h.natoms > 0) {
        CK(cudaMemcpyAsync(h.raw_atoms, in.atomInfo, sizeof(Atom) * h.natoms, cudaMemcpyHostToDevice, s));
        k_unpack_atoms<<<unpack_blocks(h.natoms), 256, 0, s>>>(h.raw_atoms, h.xyzq, h.atype, h.natoms);
    }
    if (h.ngroups > 0) {
        CK(cudaMemcpyAsync(h.raw_groups, in.residueInfo, sizeof(residue) * h.ngroups, cudaMemcpyHostToDevice, s));
        k_unpack_groups<<<unpack_blocks(h.ngroups), 256, 0, s>>>(h.raw_groups, h.gcen, h.gspan, h.ngroups);
    }
    CK(cudaMemsetAsync(h.cell_count, 0, sizeof(int) * h.ncell, s));
    CK(cudaMemsetAsync(h.gcell, 0xff, sizeof(int) * std::max(1, h.ngroups), s));
    if (h.G > 0 && !opt.grid_bits) {
        CK(cudaMemcpyAsync(h.raw_grid, in.grid, sizeof(float) * 3 * (size_t)h.G, cudaMemcpyHostToDevice, s));
        k_unpack_grid<<<unpack_blocks(h.G), 256, 0, s>>>(h.raw_grid, h.grid, h.G);
    } else if (h.G == 0) {
        CK(cudaMemsetAsync(h.grid, 0, sizeof(float4), s));
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h.lj, lj.data(), sizeof(float2) * lj.size(), cudaMemcpyHostToDevice, s));
    if (h.mcsteps > 0) {
        CK(cudaMemcpyAsync(h.moves, in.moveArray, sizeof(int) * h.mcsteps, cudaMemcpyHostToDevice, s));
        h.moves_host.assign(in.moveArray, in.moveArray + h.mcsteps);
    }
    CK(cudaMemcpyAsync(h.frag, frag.data(), sizeof(FragDev) * h.ntypes, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(h.totalNum, tot.data(), sizeof(int) * h.ntypes, cudaMemcpyHostToDevice, s));
    StepDesc d0{};
    d0.step = 0;
    d0.move = MV_NONE;
    CK(cudaMemcpyAsync(h.desc, &d0, sizeof(StepDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(h.counters, 0, sizeof(unsigned long long) * 16, s));
    CK(cudaMemsetAsync(h.err, 0, sizeof(int), s));
    if (h.log_cap > 0) {  // entries past a step's pose count read as zeros
        CK(cudaMemsetAsync(h.logE, 0, sizeof(double) * (size_t)h.log_cap * h.log_kmax, s));
        if (d.fb) CK(cudaMemsetAsync(h.logF, 0, sizeof(float) * (size_t)h.log_cap * h.log_kmax * 12, s));
    }
    if (nblk > 0) {  // after the error word is cleared: the scan reports a count mismatch there
        CK(cudaMemcpyAsync(h.raw_bits, reinterpret_cast<const char*>(in.grid) + sizeof(gcmc_grid_bits),
                           sizeof(uint32_t) * (size_t)nwords, cudaMemcpyHostToDevice, s));
        k_bits_count<<<nblk, kBitsThreads, 0, s>>>(h.raw_bits, nwords, nvox, h.bits_blk);
        k_bits_scan<<<1, kBitsThreads, 0, s>>>(h.bits_blk, nblk, h.G, h.err);
        k_bits_expand<<<nblk, kBitsThreads, 0, s>>>(h.raw_bits, nwords, nvox, h.bits_blk, gb.n[1], gb.n[2],
                                                    gb.start[0], gb.start[1], gb.start[2], gb.dx, h.grid, h.G);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(h.epart, 0, sizeof(double) * kMaxPoses * 2 * h.slab_cap, s));
    CK(cudaMemsetAsync(h.energy, 0, sizeof(double), s));
    CK(cudaMemsetAsync(h.fpart, 0, sizeof(float) * kMaxPoses * 2 * h.slab_cap * 6, s));
    CK(cudaMemsetAsync(h.fbprop, 0, sizeof(float4) * kMaxPoses * 2, s));
    CK(cudaMemsetAsync(h.fbcnt, 0, sizeof(int) * kMaxPoses, s));
    if (ctx->spec) {
        // a speculative evaluation may read a cell while the accept kernel edits it:
        // every record slot then holds a span of real atoms (or none)
        CK(cudaMemsetAsync(h.cell_ent, 0, sizeof(CellEnt) * (size_t)h.ncell * cap, s));
        CK(cudaMemcpyAsync(h.desc2, &d0, sizeof(StepDesc), cudaMemcpyHostToDevice, s));
        CK(cudaMemsetAsync(h.epart2, 0, sizeof(double) * kMaxPoses * 2 * h.slab_cap, s));
        CK(cudaMemsetAsync(h.valid2, 0, sizeof(int) * 2, s));
        CK(cudaMemsetAsync(h.abort2, 0xff, sizeof(int) * 2, s));  // -1: no step voided
        CK(cudaMemsetAsync(h.sstep2, 0, sizeof(int) * 2, s));
        CK(cudaMemsetAsync(h.pending2, 0, sizeof(unsigned long long) * 2, s));
    }

    stamp(3);
    d.xyzq = h.xyzq; d.atype = h.atype; d.gcen = h.gcen; d.gspan = h.gspan;
    d.cell_count = h.cell_count; d.cell_ent = h.cell_ent; d.gcell = h.gcell;
    d.grid = h.grid; d.lj = h.lj; d.moves = h.moves; d.frag = h.frag; d.totalNum = h.totalNum;
    d.desc = h.desc; d.pcen = h.pcen; d.pslot = h.pslot; d.epart = h.epart; d.nbr = h.nbr;
    d.log = h.log; d.logE = h.logE; d.log_cap = h.log_cap; d.log_kmax = h.log_kmax;
    d.counters = h.counters; d.err = h.err;
    d.energy = h.energy; d.pgum = h.pgum; d.psite = h.psite; d.plnu = h.plnu; d.fpart = h.fpart; d.fbprop = h.fbprop; d.fbcnt = h.fbcnt;
    d.logF = (h.log_cap > 0 && d.fb) ? h.logF : nullptr;
    d.pbin = h.pbin; d.tiles = h.tiles;
    d.wcost = opt.pose_split > 0 ? h.wcost : nullptr;
    d.pnslab = h.pnslab; d.pitem = h.pitem;
    if (ctx->spec) {
        RepDev& b = ctx->repdev_b;
        b = d;
        b.desc = h.desc2; b.pcen = h.pcen2; b.pslot = h.pslot2; b.epart = h.epart2; b.nbr = h.nbr2;
        b.pgum = h.pgum2; b.plnu = h.plnu2; b.psite = h.psite2; b.pbin = h.pbin2; b.tiles = h.tiles2;
        b.pnslab = h.pnslab2; b.pitem = h.pitem2;
        d.valid = h.valid2; d.pairs_pending = h.pending2; d.abort = h.abort2; d.spec_step = h.sstep2;
        b.valid = h.valid2 + 1; b.pairs_pending = h.pending2 + 1; b.abort = h.abort2 + 1; b.spec_step = h.sstep2 + 1;
    }
    return GCMC_OK;
}

// Link each descriptor to its partner (itself unless speculating) and upload.
int upload_reps(gcmc_ctx* ctx) {
    if (ctx->spec && !ctx->d_reps_b) CK(cudaMalloc(&ctx->d_reps_b, sizeof(RepDev)));
    for (int r = 0; r < ctx->nrep; ++r) ctx->repdev[r].other = ctx->d_reps + r;
    if (ctx->spec) {
        ctx->repdev[0].other = ctx->d_reps_b;
        ctx->repdev_b.other = ctx->d_reps;
        CK(cudaMemcpyAsync(ctx->d_reps_b, &ctx->repdev_b, sizeof(RepDev), cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaMemcpyAsync(ctx->d_reps, ctx->repdev.data(), sizeof(RepDev) * ctx->nrep, cudaMemcpyHostToDevice,
                       ctx->stream));
    return GCMC_OK;
}

using EnergyKernel = void (*)(const RepDev*, int, int);
// which: -1 every item; 0 / 1 the items of steps not in / in the difference form;
// ew: the Ewald code paths compiled in (contexts with a replica under Ewald)
EnergyKernel energy_kernel(int variant, int which = -1, bool ew = false) {
    if (ew) return variant == 1 ? k_energy_t<4, -1, 1> : k_energy_t<3, -1, 1>;
    if (which == 0) return variant == 1 ? k_energy_t<4, 0, 0> : k_energy_t<3, 0, 0>;
    if (which == 1) return variant == 1 ? k_energy_t<4, 1, 0> : k_energy_t<3, 1, 0>;
    if (which == 2) return variant == 1 ? k_energy_t<4, 2, 0> : k_energy_t<3, 2, 0>;
    return variant == 1 ? k_energy_t<4, -1, 0> : k_energy_t<3, -1, 0>;
}

// One pose-energy launch over replicas reps[0, n) in `mode` on `grid` CTAs:
// the tiled kernel when the context is tiled, else the per-pose-warp kernel.
void launch_energy(const gcmc_ctx* ctx, const RepDev* reps, int n, int mode, int grid, cudaStream_t s) {
    if (ctx->tiled) {
        k_energy_tiles<<<grid, kWarpsT * 32, sizeof(TileSmem), s>>>(reps, n, mode);
    } else if (n > 1 && ctx->dual_any && !ctx->pme_any) {
        // a batch mixes the two kinds of items: one launch whose SMs each take one kind
        // (an SM that ran both code paths at once stalled on instruction fetch)
        energy_kernel(ctx->evar, 2)<<<grid, kWarpsE * 32, 0, s>>>(reps, n, mode);
    } else {
        energy_kernel(ctx->evar, -1, ctx->pme_any)<<<grid, kWarpsE * 32, 0, s>>>(reps, n, mode);
    }
}

// The accept kernel of the context: with the Ewald code paths when a replica
// runs Ewald electrostatics.
using AcceptKernel = void (*)(const RepDev*, int, int);
AcceptKernel accept_kernel(const gcmc_ctx* ctx) { return ctx->pme_any ? k_accept<true> : k_accept<false>; }

// Dynamic shared memory of the preparation kernels (the pose binning's or the
// per-pose split's scratch).
size_t prep_smem(const gcmc_ctx*) { return (size_t)kBinScratchBytes; }

// The context is tiled when every replica allows it; otherwise no replica is.
void finalize_tiling(gcmc_ctx* ctx) {
    bool all = true;
    for (const auto& d : ctx->repdev) all = all && d.tiled;
    ctx->tiled = all;
    for (auto& d : ctx->repdev) d.tiled = all ? 1 : 0;
    ctx->repdev_b.tiled = all ? 1 : 0;
    bool pme = false;
    for (const auto& h : ctx->reps) pme = pme || h.pme;
    ctx->pme_any = pme;
    bool dual = false;
    for (const auto& d : ctx->repdev) dual = dual || d.dual;
    ctx->dual_any = dual;
}

// Resident warps of the pose-energy grid for this register variant and CTA cap.
int energy_warps(int device, int evar, int ebps, int spare_sms) {
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, energy_kernel(evar), kWarpsE * 32, 0) != cudaSuccess) {
        cudaGetLastError();
        return 2048;
    }
    per_sm = std::max(1, per_sm);
    if (ebps > 0) per_sm = std::min(per_sm, ebps);
    return std::max(1, sms - spare_sms) * per_sm * kWarpsE;
}


// Replica r's PME mesh potential from its spread charges on stream s, when
// they changed since the last update (every pass returns at once otherwise):
// rows real-to-complex, axis 1, axis 0 with the influence function between
// its forward and inverse transforms, axis 1 inverse, rows complex-to-real.
int pme_update(gcmc_ctx* ctx, int r, cudaStream_t s) {
    RepHost& h = ctx->reps[r];
    if (!h.pme) return GCMC_OK;
    const RepDev* rep = ctx->d_reps + r;
    const int n0 = h.pme_n[0], n1 = h.pme_n[1], n2 = h.pme_n[2], M = n2 / 2 + 1;
    const int kb = (M + kFftLines - 1) / kFftLines;
    const int rows = (n0 * n1 + kFftLines - 1) / kFftLines;
    const size_t sm2 = 2 * kFftLines * (size_t)n2 * sizeof(double2);
    const size_t sm1 = 2 * kFftLines * (size_t)n1 * sizeof(double2);
    const size_t sm0 = 2 * kFftLines * (size_t)n0 * sizeof(double2);
    k_pme_rows_r2c<<<std::min(rows, 4096), kFftThreads, sm2, s>>>(rep);
    k_pme_axis<<<std::min(n0 * kb, 4096), kFftThreads, sm1, s>>>(rep, 1, -1, 0);
    k_pme_axis<<<std::min(n1 * kb, 4096), kFftThreads, sm0, s>>>(rep, 0, 0, 1);
    k_pme_axis<<<std::min(n0 * kb, 4096), kFftThreads, sm1, s>>>(rep, 1, 1, 0);
    k_pme_rows_c2r<<<std::min(rows, 4096), kFftThreads, sm2, s>>>(rep);
    k_pme_done<<<1, 32, 0, s>>>(rep);
    CK(cudaGetLastError());
    return GCMC_OK;
}

// The spread charges of the current state (the fixed atoms and the occupied
// fragment slots; once per set-up, needs d_reps uploaded), marked dirty.
int pme_init_fixed(gcmc_ctx* ctx) {
    for (int r = 0; r < ctx->nrep; ++r) {
        RepHost& h = ctx->reps[r];
        if (!h.pme) continue;
        const size_t nr = (size_t)h.pme_n[0] * h.pme_n[1] * h.pme_n[2];
        CK(cudaMemsetAsync(h.pme_q, 0, sizeof(double) * nr, ctx->stream));
        if (h.nfix_atoms > 0)
            k_pme_spread_range<<<296, 256, 0, ctx->stream>>>(ctx->d_reps + r, h.pme_q, 0, h.nfix_atoms);
        k_pme_spread_frag<<<148, 256, 0, ctx->stream>>>(ctx->d_reps + r, h.pme_q);
        CK(cudaMemsetAsync(h.pme_dirty, 1, sizeof(int), ctx->stream));
        CK(cudaGetLastError());
    }
    return GCMC_OK;
}

// The force-bias pose-energy kernel: with the SM-affine split of its first launch
// when the replicas' move schedules differ (a launch may then hold both kinds of
// items), without it otherwise.
using FbKernel = void (*)(const RepDev*, int, int);
FbKernel fb_kernel(const gcmc_ctx* ctx) { return ctx->fb_mixed ? k_energy_fb<true> : k_energy_fb<false>; }

// Whether the replicas' move schedules differ (over the steps all of them hold).
void find_mixed_moves(gcmc_ctx* ctx) {
    bool mixed = false;
    const auto& m0 = ctx->reps[0].moves_host;
    for (int r = 1; r < ctx->nrep && !mixed; ++r) {
        const auto& m = ctx->reps[r].moves_host;
        const size_t n = std::min(m.size(), m0.size());
        mixed = m.size() != m0.size() || !std::equal(m.begin(), m.begin() + n, m0.begin());
    }
    ctx->fb_mixed = mixed;
}

// Pose-energy grid: SMs x min(occupancy limit, requested CTAs per SM).
int set_energy_grid(gcmc_ctx* ctx, int ebps) {
    int sms = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (ctx->tiled) {
        CK(cudaFuncSetAttribute(k_energy_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem)));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_energy_tiles, kWarpsT * 32, sizeof(TileSmem)));
    } else {
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, energy_kernel(ctx->evar), kWarpsE * 32, 0));
    }
    per_sm = std::max(1, per_sm);
    if (ebps > 0) per_sm = std::min(per_sm, ebps);
    ctx->ebps = ebps;
    ctx->per_sm_e = per_sm;
    ctx->gridE = std::max(1, sms) * per_sm;
    int per_sm_f = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, fb_kernel(ctx), kWarpsG * 32, 0));
    ctx->gridF = std::max(1, sms) * std::max(1, per_sm_f);
    return GCMC_OK;
}

// Cell lists of every replica from its current centres and counts (cell_count
// zeroed and gcell = -1 beforehand).
void build_cells(gcmc_ctx* ctx) {
    int ng = 1, nc = 1;
    for (const auto& h : ctx->reps) {
        ng = std::max(ng, h.ngroups);
        nc = std::max(nc, h.ncell);
    }
    const dim3 gf((unsigned)std::min((ng + 255) / 256, 148 * 4), (unsigned)ctx->nrep);
    const dim3 gs((unsigned)std::min((nc + 255) / 256, 148 * 4), (unsigned)ctx->nrep);
    k_fill_cells<<<gf, 256, 0, ctx->stream>>>(ctx->d_reps);
    k_sort_cells<<<gs, 256, 0, ctx->stream>>>(ctx->d_reps);
}

// Split the replicas into `nb` contiguous groups of about equal atom count.
void split_branches(gcmc_ctx* ctx, int nb) {
    nb = std::max(1, std::min(nb, ctx->nrep));
    std::vector<double> pre(ctx->nrep + 1, 0.0);
    for (int r = 0; r < ctx->nrep; ++r) pre[r + 1] = pre[r] + (double)ctx->reps[r].natoms + 1.0;
    ctx->br_off.assign(nb + 1, 0);
    ctx->br_off[nb] = ctx->nrep;
    for (int b = 1; b < nb; ++b) {
        const double target = pre[ctx->nrep] * b / nb;
        int r = ctx->br_off[b - 1] + 1;
        while (r < ctx->nrep - (nb - b) && pre[r] < target) ++r;
        ctx->br_off[b] = r;
    }
    ctx->branches = nb;
}

// kGraphSteps MC steps.  With several branches, each branch is its own chain
// of (pose-energy, accept) launches over its replicas, forked from and joined
// to the context's stream, so one branch's accept kernel (a CTA per replica)
// overlaps another's pose energies; each branch gets a share of the
// pose-energy grid in proportion to its atoms.
// Speculating (one replica): step j (descriptor copy j & 1) is, on the
// context's stream, F_p (prepare it again unless its speculation stands), F_e
// (its pose energies unless they stand) and A (accept).  On a second stream P
// prepares step j + 1 in the other copy as soon as A of step j - 1 is done (as
// if step j accepts nothing), and on a third S evaluates its pose energies
// once P and F_e are done, on the SMs that A leaves free, stopping early when
// A accepts a move.  F_p of step j + 1 waits for A and S.  One graph per
// parity of the run's first step (kGraphSteps is even).
// Launch of `kernel` on s as a programmatic dependent of the kernel before it in
// s: it may be scheduled once every CTA of that kernel has triggered (pdl_trigger)
// and waits in pdl_wait for that kernel's results, so its launch latency overlaps
// the kernel before it.
template <class... Args, class... Act>
cudaError_t launch_dependent(void (*kernel)(Args...), int grid, int block, size_t smem, cudaStream_t s,
                             Act... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// pdl: the step's completion pose-energy launch and accept kernel as programmatic
// dependents of the kernels before them (F_p -> F_e -> accept).
int build_spec_graph(gcmc_ctx* ctx, int parity, bool pdl) {
    cudaStream_t sp = nullptr, ss = nullptr;
    cudaEvent_t ev[4 * kGraphSteps + 1] = {};
    int st = GCMC_OK;
    if (cudaStreamCreateWithFlags(&sp, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking) != cudaSuccess)
        st = GCMC_ERR_CUDA;
    for (auto& e : ev)
        if (st == GCMC_OK && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) st = GCMC_ERR_CUDA;
    cudaGraph_t graph = nullptr;
    if (st == GCMC_OK && cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        st = GCMC_ERR_CUDA;
    if (st == GCMC_OK) {
        const int grid_s = std::max(1, ctx->gridE - ctx->per_sm_e);
        cudaEvent_t* evF = ev;                    // F_e of step j done
        cudaEvent_t* evA = ev + kGraphSteps;      // A of step j done
        cudaEvent_t* evP = ev + 2 * kGraphSteps;  // P of step j + 1 done
        cudaEvent_t* evS = ev + 3 * kGraphSteps;  // S of step j + 1 done
        cudaError_t e = cudaEventRecord(ev[4 * kGraphSteps], ctx->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sp, ev[4 * kGraphSteps], 0);
        for (int i = 0; i < kGraphSteps && e == cudaSuccess; ++i) {
            const RepDev* cur = ((parity + i) & 1) ? ctx->d_reps_b : ctx->d_reps;
            const RepDev* nxt = ((parity + i) & 1) ? ctx->d_reps : ctx->d_reps_b;
            if (i > 0) e = cudaStreamWaitEvent(ctx->stream, evS[i - 1], 0);
            k_prep_spec<<<1, kAcceptThreads, prep_smem(ctx), ctx->stream>>>(cur, 1);
            if (pdl && !ctx->tiled) {
                if (e == cudaSuccess)
                    e = launch_dependent(energy_kernel(ctx->evar, -1, ctx->pme_any), ctx->gridE, kWarpsE * 32, 0,
                                         ctx->stream, cur, 1, 2);
            } else {
                launch_energy(ctx, cur, 1, 2, ctx->gridE, ctx->stream);
            }
            if (e == cudaSuccess) e = cudaEventRecord(evF[i], ctx->stream);
            if (pdl) {  // (speculating: no Ewald)
                if (e == cudaSuccess)
                    e = launch_dependent(k_accept<false>, 1, kAcceptThreads, sizeof(AcceptSmem), ctx->stream, cur, 1,
                                         1);
            } else {
                k_accept<false><<<1, kAcceptThreads, sizeof(AcceptSmem), ctx->stream>>>(cur, 1, 1);
            }
            if (e == cudaSuccess) e = cudaEventRecord(evA[i], ctx->stream);
            if (i > 0 && e == cudaSuccess) e = cudaStreamWaitEvent(sp, evA[i - 1], 0);
            k_prep_spec<<<1, kAcceptThreads, prep_smem(ctx), sp>>>(nxt, 0);
            if (e == cudaSuccess) e = cudaEventRecord(evP[i], sp);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(ss, evP[i], 0);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(ss, evF[i], 0);
            launch_energy(ctx, nxt, 1, 1, grid_s, ss);
            if (e == cudaSuccess) e = cudaEventRecord(evS[i], ss);
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, evS[kGraphSteps - 1], 0);
        if (e == cudaSuccess) e = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            std::fprintf(stderr, "gcmc_b200: graph capture failed: %s\n",
                         cudaGetErrorString(e != cudaSuccess ? e : e2));
            st = GCMC_ERR_CUDA;
        }
    }
    if (st == GCMC_OK && cudaGraphInstantiate(&ctx->gexec_spec[parity], graph, 0) != cudaSuccess) st = GCMC_ERR_CUDA;
    if (graph) cudaGraphDestroy(graph);
    if (sp) cudaStreamDestroy(sp);
    if (ss) cudaStreamDestroy(ss);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (st != GCMC_OK) cudaGetLastError();
    return st;
}

int build_graph(gcmc_ctx* ctx) {
    if (ctx->gexec) {
        cudaGraphExecDestroy(ctx->gexec);
        ctx->gexec = nullptr;
    }
    for (auto& g : ctx->gexec_spec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    if (ctx->spec) {
        int st = build_spec_graph(ctx, 0, true);
        if (st == GCMC_OK) st = build_spec_graph(ctx, 1, true);
        if (st != GCMC_OK) {  // a driver that cannot capture programmatic launches: plain launches
            for (auto& g : ctx->gexec_spec)
                if (g) {
                    cudaGraphExecDestroy(g);
                    g = nullptr;
                }
            cudaGetLastError();
            st = build_spec_graph(ctx, 0, false);
            if (st == GCMC_OK) st = build_spec_graph(ctx, 1, false);
        }
        return st;
    }
    const int nb = ctx->branches;
    std::vector<cudaStream_t> side(nb, nullptr);
    std::vector<cudaEvent_t> ev(nb, nullptr);
    int st = GCMC_OK;
    for (int b = 1; b < nb && st == GCMC_OK; ++b)
        if (cudaStreamCreateWithFlags(&side[b], cudaStreamNonBlocking) != cudaSuccess) st = GCMC_ERR_CUDA;
    for (int b = 0; b < nb && st == GCMC_OK; ++b)
        if (cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming) != cudaSuccess) st = GCMC_ERR_CUDA;
    cudaGraph_t graph = nullptr;
    if (st == GCMC_OK && cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        st = GCMC_ERR_CUDA;
    if (st == GCMC_OK) {
        side[0] = ctx->stream;
        cudaError_t e = cudaEventRecord(ev[0], ctx->stream);
        for (int b = 1; b < nb && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(side[b], ev[0], 0);
        for (int b = 0; b < nb && e == cudaSuccess; ++b) {
            const int r0 = ctx->br_off[b], cnt = ctx->br_off[b + 1] - r0;
            // every branch's pose-energy launch on the whole grid: its warps take items from
            // the branch's own counter, so a branch whose neighbour sits in its accept kernel
            // (one CTA per replica) spreads over the SMs left free (a grid in proportion to
            // the branch's atoms left them idle: 358 against 306 us per 64-replica step)
            const int grid = ctx->gridE;
            const int gridf = ctx->gridF;
            for (int s = 0; s < kGraphSteps && e == cudaSuccess; ++s) {
                for (int r = r0; r < r0 + cnt; ++r)
                    if (pme_update(ctx, r, side[b]) != GCMC_OK) e = cudaErrorUnknown;
                if (ctx->fb) {
                    fb_kernel(ctx)<<<gridf, kWarpsG * 32, 0, side[b]>>>(ctx->d_reps + r0, cnt, 1);
                    fb_kernel(ctx)<<<gridf, kWarpsG * 32, 0, side[b]>>>(ctx->d_reps + r0, cnt, 2);
                } else {
                    launch_energy(ctx, ctx->d_reps + r0, cnt, 0, grid, side[b]);
                }
                accept_kernel(ctx)<<<cnt, kAcceptThreads, sizeof(AcceptSmem), side[b]>>>(ctx->d_reps + r0, cnt, 0);
            }
            if (e == cudaSuccess) e = cudaGetLastError();
        }
        for (int b = 1; b < nb && e == cudaSuccess; ++b) {
            e = cudaEventRecord(ev[b], side[b]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ev[b], 0);
        }
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &graph);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            std::fprintf(stderr, "gcmc_b200: graph capture failed: %s\n",
                         cudaGetErrorString(e != cudaSuccess ? e : e2));
            st = GCMC_ERR_CUDA;
        }
    }
    if (st == GCMC_OK && cudaGraphInstantiate(&ctx->gexec, graph, 0) != cudaSuccess) st = GCMC_ERR_CUDA;
    if (graph) cudaGraphDestroy(graph);
    for (int b = 1; b < nb; ++b)
        if (side[b]) cudaStreamDestroy(side[b]);
    for (int b = 0; b < nb; ++b)
        if (ev[b]) cudaEventDestroy(ev[b]);
    if (st != GCMC_OK) cudaGetLastError();
    return st;
}

int destroy_impl(gcmc_ctx* ctx) {
    if (!ctx) return GCMC_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    for (auto g : ctx->gexec_spec)
        if (g) cudaGraphExecDestroy(g);
    for (auto& h : ctx->reps) free_rep(h);
    if (ctx->d_reps) cudaFree(ctx->d_reps);
    if (ctx->d_reps_b) cudaFree(ctx->d_reps_b);
    if (ctx->d_sync) cudaFree(ctx->d_sync);
    if (ctx->ev_ctx) cudaEventDestroy(ctx->ev_ctx);
    if (ctx->ev_call) cudaEventDestroy(ctx->ev_call);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return GCMC_OK;
}

// The persistent step loop where it was asked for and the context allows it:
// no speculation (one-replica contexts speculate instead), no PME (its mesh
// mesh update runs between steps), proposal 0 or 1, the per-pose-warp
// pose-energy kernel, and one k_persist CTA resident on every SM.
int setup_persist(gcmc_ctx* ctx, const gcmc_options& opt) {
    ctx->persist = false;
    ctx->spin_cap = opt.persist_spin_cap > 0 ? (long long)opt.persist_spin_cap : kPersistSpinCap;
    if (opt.persistent <= 0 || ctx->spec || ctx->pme_any || ctx->fb || ctx->tiled) return GCMC_OK;
    int sms = 0, per_sm = 0, coop = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
    if (!coop) return GCMC_OK;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CK(cudaFuncSetAttribute(k_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AcceptSmem)));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist, kAcceptThreads, sizeof(AcceptSmem)));
    if (per_sm < 1) return GCMC_OK;
    if (!ctx->d_sync) CK(cudaMalloc(&ctx->d_sync, sizeof(GridSync)));
    ctx->grid_persist = sms;
    ctx->persist = true;
    return GCMC_OK;
}

int create_impl(int nrep, const gcmc_replica_in* ins, const gcmc_options* optp, void* stream, gcmc_ctx** out) {
    if (!out || !ins || nrep < 1) return GCMC_ERR_ARG;
    if (nrep > kMaxRep) return GCMC_ERR_LIMIT;
    *out = nullptr;
    gcmc_options opt;
    if (optp) opt = *optp; else gcmc_default_options(&opt);
    if (opt.proposal < 0 || opt.proposal > 2) return GCMC_ERR_ARG;
    std::vector<int2> frag_atoms(nrep);
    {
        const int st = for_each_rep(nrep, -1, [&](int r) { return validate(ins[r], &frag_atoms[r]); });
        if (st != GCMC_OK) return st;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return GCMC_ERR_NODEVICE;
    }
    gcmc_ctx* ctx = new gcmc_ctx();
    ctx->nrep = nrep;
    cudaGetDevice(&ctx->device);
    int st = GCMC_OK;
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return GCMC_ERR_CUDA;
        }
        ctx->own_stream = true;
    }
    if (cudaEventCreateWithFlags(&ctx->ev_ctx, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_call, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        destroy_impl(ctx);
        return GCMC_ERR_CUDA;
    }
    ctx->reps.resize(nrep);
    ctx->repdev.resize(nrep);
    for (int r = 0; r < nrep; ++r) ctx->reps[r].frag_atoms = frag_atoms[r];
    ctx->spec = spec_eligible(nrep, ins, opt);
    if (st == GCMC_OK) st = for_each_rep(nrep, ctx->device, [&](int r) { return setup_rep(ctx, r, ins[r], opt); });
    if (st == GCMC_OK) {
        finalize_tiling(ctx);
        find_mixed_moves(ctx);
    }
    if (st == GCMC_OK && cudaMalloc(&ctx->d_reps, sizeof(RepDev) * nrep) != cudaSuccess) st = GCMC_ERR_CUDA;
    if (st == GCMC_OK) st = upload_reps(ctx);
    if (st == GCMC_OK) {
        if (cudaFuncSetAttribute(k_accept<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(AcceptSmem)) != cudaSuccess ||
            cudaFuncSetAttribute(k_accept<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(AcceptSmem)) != cudaSuccess)
            st = GCMC_ERR_CUDA;
    }
    ctx->fb = opt.proposal == 2 ? 1 : 0;
    ctx->evar = opt.energy_variant == 1 ? 1 : 0;
    if (st == GCMC_OK) st = set_energy_grid(ctx, opt.energy_blocks_per_sm);
    if (st == GCMC_OK) {
        split_branches(ctx, opt.branches > 0 ? opt.branches : 1);
        build_cells(ctx);
        if (cudaGetLastError() != cudaSuccess) st = GCMC_ERR_CUDA;
    }
    if (st == GCMC_OK) st = pme_init_fixed(ctx);
    if (st == GCMC_OK) st = setup_persist(ctx, opt);
    if (st == GCMC_OK && !ctx->persist) st = build_graph(ctx);
    if (st == GCMC_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) st = GCMC_ERR_CUDA;
    if (st == GCMC_OK) {
        int32_t err = 0;
        gcmc_device_error(ctx, &err);
        if (err) st = (err & ERR_GRID_BITS) ? GCMC_ERR_ARG : GCMC_ERR_DEVICE;
    }
    if (st != GCMC_OK) {
        cudaGetLastError();
        destroy_impl(ctx);
        return st;
    }
    *out = ctx;
    return GCMC_OK;
}

// Load new inputs (same replica count) into an existing context: buffers are
// reused where large enough, the captured graph is kept when the launch shape
// is unchanged (kernels reach every buffer through d_reps), cells are rebuilt
// and the run state reset.
int refill_impl(gcmc_ctx* ctx, int nrep, const gcmc_replica_in* ins, const gcmc_options* optp) {
    if (ctx->nrep != nrep) return GCMC_ERR_ARG;
    gcmc_options opt;
    if (optp) opt = *optp; else gcmc_default_options(&opt);
    if (opt.proposal < 0 || opt.proposal > 2) return GCMC_ERR_ARG;
    int st = GCMC_OK;
    std::vector<int2> frag_atoms(nrep);
    st = for_each_rep(nrep, -1, [&](int r) { return validate(ins[r], &frag_atoms[r]); });
    if (st != GCMC_OK) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int r = 0; r < nrep; ++r) ctx->reps[r].frag_atoms = frag_atoms[r];
    if (trace_on()) g_trace[0] = now_ms();
    const bool spec = spec_eligible(nrep, ins, opt);
    const bool spec_changed = spec != ctx->spec;
    ctx->spec = spec;
    const bool tiled_before = ctx->tiled, pme_before = ctx->pme_any, dual_before = ctx->dual_any;
    st = for_each_rep(nrep, ctx->device, [&](int r) { return setup_rep(ctx, r, ins[r], opt); });
    if (st != GCMC_OK) return st;
    if (trace_on()) g_trace[1] = now_ms();
    finalize_tiling(ctx);
    const bool mixed_before = ctx->fb_mixed;
    find_mixed_moves(ctx);
    st = upload_reps(ctx);
    if (st != GCMC_OK) return st;
    build_cells(ctx);
    CK(cudaGetLastError());
    st = pme_init_fixed(ctx);
    if (st != GCMC_OK) return st;
    const int nb = std::max(1, std::min(opt.branches > 0 ? opt.branches : 1, nrep));
    const int fb = opt.proposal == 2 ? 1 : 0;
    const int evar = opt.energy_variant == 1 ? 1 : 0;
    const bool persist_before = ctx->persist;
    const bool had_graph = ctx->gexec || ctx->gexec_spec[0];
    const bool shape_changed = spec_changed || nb != ctx->branches || opt.energy_blocks_per_sm != ctx->ebps ||
                               fb != ctx->fb || evar != ctx->evar || ctx->tiled != tiled_before ||
                               ctx->pme_any != pme_before || ctx->dual_any != dual_before ||
                               ctx->fb_mixed != mixed_before;
    ctx->fb = fb;
    ctx->evar = evar;
    st = setup_persist(ctx, opt);
    if (st != GCMC_OK) return st;
    if (shape_changed || ctx->persist != persist_before) {
        st = set_energy_grid(ctx, opt.energy_blocks_per_sm);
        if (st != GCMC_OK) return st;
        split_branches(ctx, nb);
        if (!ctx->persist && (shape_changed || !had_graph)) {
            st = build_graph(ctx);
            if (st != GCMC_OK) return st;
        }
    }
    if (trace_on()) g_trace[2] = now_ms();
    CK(cudaStreamSynchronize(ctx->stream));
    int32_t err = 0;
    gcmc_device_error(ctx, &err);
    return err ? ((err & ERR_GRID_BITS) ? GCMC_ERR_ARG : GCMC_ERR_DEVICE) : GCMC_OK;
}

// The contexts kept by gcmc_run_gcmc / runGCMC_cuda (one replica) and by
// gcmc_run_batch between calls.
std::mutex g_cache_mutex;
gcmc_ctx* g_cache = nullptr;
gcmc_ctx* g_batch = nullptr;

// What a run can change in the caller's arrays, written back in place: the
// fragment types' counts, the fragment residues' centres and the atoms of the
// fragment slots (fixed groups and atoms never move, so their entries already
// hold the device's values).  k_pack_moved writes the current state in the
// caller's layout into the upload buffers (which hold the caller's arrays as
// uploaded, so the fields a run never changes keep the caller's values), and
// one copy per range lands it in place.
__global__ void k_pack_moved(const float4* __restrict__ gcen, residue* __restrict__ groups, int g0, int g1,
                             const float4* __restrict__ xyzq, const int* __restrict__ atype, Atom* __restrict__ atoms,
                             int a0, int a1) {
    const int ng = g1 - g0, na = a1 - a0, n = ng > na ? ng : na;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < ng) {
            const float4 c = gcen[g0 + i];
            residue& R = groups[g0 + i];
            R.position[0] = c.x;
            R.position[1] = c.y;
            R.position[2] = c.z;
        }
        if (i < na) {
            const float4 p = xyzq[a0 + i];
            Atom& A = atoms[a0 + i];
            A.position[0] = p.x;
            A.position[1] = p.y;
            A.position[2] = p.z;
            A.charge = p.w;
            A.type = atype[a0 + i];
        }
    }
}

// Every replica's changes into the caller's arrays (one stream sync).
int download_moved(gcmc_ctx* ctx, int nrep, const gcmc_replica_in* ins) {
    cudaStream_t s = ctx->stream;
    std::vector<std::vector<int>> tot(nrep);
    for (int r = 0; r < nrep; ++r) {
        RepHost& h = ctx->reps[r];
        const gcmc_replica_in& in = ins[r];
        tot[r].resize(h.ntypes);
        CK(cudaMemcpyAsync(tot[r].data(), h.totalNum, sizeof(int) * h.ntypes, cudaMemcpyDeviceToHost, s));
        const int g0 = in.fragmentInfo[0].startRes, g1 = h.ngroups;
        const int a0 = h.frag_atoms.x, a1 = h.frag_atoms.y;
        if (g1 <= g0 && a1 <= a0) continue;
        const int n = std::max(g1 - g0, a1 - a0);
        k_pack_moved<<<unpack_blocks(n), 256, 0, s>>>(h.gcen, h.raw_groups, g0, g1, h.xyzq, h.atype, h.raw_atoms,
                                                      a0, a1);
        CK(cudaGetLastError());
        if (g1 > g0)
            CK(cudaMemcpyAsync(const_cast<residue*>(in.residueInfo) + g0, h.raw_groups + g0,
                               sizeof(residue) * (g1 - g0), cudaMemcpyDeviceToHost, s));
        if (a1 > a0)
            CK(cudaMemcpyAsync(const_cast<Atom*>(in.atomInfo) + a0, h.raw_atoms + a0, sizeof(Atom) * (a1 - a0),
                               cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    for (int r = 0; r < nrep; ++r) {
        AtomArray* frag = const_cast<AtomArray*>(ins[r].fragmentInfo);
        for (int t = 0; t < ctx->reps[r].ntypes; ++t) frag[t].totalNum = tot[r][t];
    }
    return GCMC_OK;
}

// Refill *slot (or create it) for these inputs, run every replica's mcsteps
// steps and download the results in place.  Called under g_cache_mutex.
int cached_run(gcmc_ctx** slot, int nrep, const gcmc_replica_in* ins, const gcmc_options* opt) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return GCMC_ERR_NODEVICE;
    }
    int st = GCMC_OK;
    const bool trace = trace_on();
    const double t0 = trace ? now_ms() : 0.0;
    bool refilled = false;
    if (trace) {
        g_trace[0] = g_trace[1] = g_trace[2] = t0;
        for (auto& x : g_setup_ns) x = 0;
    }
    if (*slot && (*slot)->device == dev && (*slot)->nrep == nrep) {
        refilled = true;
        st = refill_impl(*slot, nrep, ins, opt);
        if (st != GCMC_OK) {  // drop the cached context and start afresh
            destroy_impl(*slot);
            *slot = nullptr;
            if (st == GCMC_ERR_ARG || st == GCMC_ERR_LIMIT) return st;
        }
    } else if (*slot) {
        destroy_impl(*slot);
        *slot = nullptr;
    }
    if (!*slot) {
        st = create_impl(nrep, ins, opt, nullptr, slot);
        if (st != GCMC_OK) {
            *slot = nullptr;
            return st;
        }
    }
    const double t1 = trace ? now_ms() : 0.0;
    int most = 0;
    for (int r = 0; r < nrep; ++r) most = std::max(most, (int)ins[r].info->mcsteps);
    st = gcmc_run(*slot, most);
    if (st == GCMC_OK) st = gcmc_sync(*slot);
    const double t2 = trace ? now_ms() : 0.0;
    if (st == GCMC_OK) st = download_moved(*slot, nrep, ins);
    if (trace) {
        const double t3 = now_ms();
        if (refilled)
            std::fprintf(stderr,
                         "gcmc_b200 trace: %d replicas, %d steps: validate %.3f ms, host set-up %.3f ms "
                         "(host time over threads: layout %.3f, allocations %.3f, tables %.3f, uploads %.3f), "
                         "enqueue %.3f ms, device set-up %.3f ms, run %.3f ms, download %.3f ms\n",
                         nrep, most, g_trace[0] - t0, g_trace[1] - g_trace[0], g_setup_ns[0] * 1e-6,
                         g_setup_ns[1] * 1e-6, g_setup_ns[2] * 1e-6, g_setup_ns[3] * 1e-6, g_trace[2] - g_trace[1],
                         t1 - g_trace[2], t2 - t1, t3 - t2);
        else
            std::fprintf(stderr,
                         "gcmc_b200 trace: %d replicas, %d steps: new context %.3f ms, run %.3f ms, "
                         "download %.3f ms\n",
                         nrep, most, t1 - t0, t2 - t1, t3 - t2);
    }
    if (st != GCMC_OK) {
        destroy_impl(*slot);
        *slot = nullptr;
    }
    return st;
}

// ---------------------------------------------------------------------------
// Allocation-free pose energies (gcmc_energy_poses_noalloc).
//
// The per-(pose, split) partial sums live in this file-scope device array
// instead of a cudaMalloc'd buffer.  It is reserved when the library is loaded
// and stays resident on every GPU that loads the library until the process
// exits.  In host code `g_noalloc_scratch` names a host-side stand-in, not the
// device array, so its device address is looked up once per device with
// cudaGetSymbolAddress and cached.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = 2u << 20;  // 2 MiB
constexpr int kNoAllocPartBytes = sizeof(double) + sizeof(int);
constexpr int kNoAllocMaxParts = (int)(kNoAllocScratchBytes / kNoAllocPartBytes);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (set up on first use).
int noalloc_scratch(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) return GCMC_ERR_LIMIT;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "gcmc_b200: cudaGetSymbolAddress(scratch) failed on device %d: %s\n", device,
                         cudaGetErrorString(e));
            return GCMC_ERR_CUDA;
        }
        g_noalloc_addr[device] = p;
    }
    *out = g_noalloc_addr[device];
    return GCMC_OK;
}

// out[p] = sum of the pose's split partials in split order (the order the
// host-side sum of gcmc_energy_poses uses), ngroups[p] likewise.
__global__ void k_sum_parts(const double* __restrict__ part, const int* __restrict__ ngpart, int nposes, int nslab,
                            double* __restrict__ out, int* __restrict__ ngroups) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nposes) return;
    double e = 0.0;
    int ng = 0;
    for (int z = 0; z < nslab; ++z) {
        e += part[(size_t)p * nslab + z];
        ng += ngpart[(size_t)p * nslab + z];
    }
    out[p] = e;
    if (ngroups) ngroups[p] = ng;
}

// A call that launches on a caller's stream s reads the context's state (cell
// lists, positions) and, with Ewald, rewrites its mesh buffers: it must not
// overlap a run on the context's stream.  Before its launches s waits for the
// context's work so far; after them the context's stream waits for s.  Both
// are event records and waits on events the context created once.
int order_before(gcmc_ctx* ctx, cudaStream_t s) {
    if (s == ctx->stream) return GCMC_OK;
    CK(cudaEventRecord(ctx->ev_ctx, ctx->stream));
    CK(cudaStreamWaitEvent(s, ctx->ev_ctx, 0));
    return GCMC_OK;
}
int order_after(gcmc_ctx* ctx, cudaStream_t s) {
    if (s == ctx->stream) return GCMC_OK;
    CK(cudaEventRecord(ctx->ev_call, s));
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_call, 0));
    return GCMC_OK;
}

}  // namespace

extern "C" {

void gcmc_default_options(gcmc_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->proposal = 0;
    opt->muex_kcal = 0;
    opt->trn_step = 1.0f;
    opt->rot_max = 15.0f * 3.14159265358979f / 180.0f;
    opt->replica = 0;
    opt->cells_per_cutoff = 2;
    opt->log_steps = 0;
    opt->log_kmax = 1;
    opt->split_items = 0;
    opt->branches = 1;
    opt->energy_blocks_per_sm = 0;
    opt->fb_trn = 0.5f;
    opt->fb_rot = (float)(10.0 * M_PI / 180.0);
}

const char* gcmc_status_string(int status) {
    switch (status) {
        case GCMC_OK: return "ok";
        case GCMC_ERR_CUDA: return "CUDA runtime error";
        case GCMC_ERR_ARG: return "invalid or inconsistent input";
        case GCMC_ERR_LIMIT: return "a size limit of the engine is exceeded";
        case GCMC_ERR_DEVICE: return "the device raised an error flag";
        case GCMC_ERR_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

int gcmc_create(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* opt, void* stream,
                gcmc_ctx** out) {
    return create_impl(nrep, reps, opt, stream, out);
}

int gcmc_destroy(gcmc_ctx* ctx) { return destroy_impl(ctx); }

int gcmc_autotune(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* base, int32_t trial_steps,
                  gcmc_options* best, gcmc_tune_trial* trials, int32_t max_trials, int32_t* ntrials) {
    if (!reps || nrep < 1 || !best || trial_steps < 1) return GCMC_ERR_ARG;
    if (nrep > kMaxRep) return GCMC_ERR_LIMIT;
    constexpr int kWarm = 8;
    int avail = INT32_MAX;
    for (int r = 0; r < nrep; ++r) {
        if (!reps[r].info) return GCMC_ERR_ARG;
        avail = std::min(avail, (int)reps[r].info->mcsteps - kWarm);
    }
    const int steps = std::min(trial_steps, avail);
    if (steps < 1) return GCMC_ERR_ARG;
    gcmc_options opt;
    if (base) opt = *base; else gcmc_default_options(&opt);
    if (opt.cells_per_cutoff <= 0) opt.cells_per_cutoff = 2;
    if (opt.branches <= 0) opt.branches = 1;
    opt.log_steps = 0;
    int n = 0;
    float best_ms = INFINITY;
    gcmc_options cur = opt;
    // time one candidate on a fresh context: kWarm steps, then the best of two runs of `steps`
    auto trial = [&](gcmc_options o, float* ms) -> int {
        gcmc_ctx* c = nullptr;
        int st = create_impl(nrep, reps, &o, nullptr, &c);
        if (st != GCMC_OK) return st;
        cudaEvent_t a = nullptr, b = nullptr;
        float t = INFINITY;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) st = GCMC_ERR_CUDA;
        if (st == GCMC_OK) st = gcmc_run(c, kWarm);
        const int half = std::max(1, steps / 2);
        for (int k = 0; k < 2 && st == GCMC_OK; ++k) {
            cudaEventRecord(a, c->stream);
            st = gcmc_run(c, half);
            cudaEventRecord(b, c->stream);
            if (st == GCMC_OK) st = gcmc_sync(c);
            float x = 0.f;
            if (st == GCMC_OK && cudaEventElapsedTime(&x, a, b) == cudaSuccess) t = std::min(t, x / half);
        }
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        destroy_impl(c);
        *ms = t;
        return st;
    };
    auto consider = [&](gcmc_options o) -> int {
        float ms = INFINITY;
        int st = trial(o, &ms);
        if (st != GCMC_OK) return st;
        if (trials && n < max_trials)
            trials[n] = gcmc_tune_trial{o.cells_per_cutoff, o.split_items,   o.branches,     o.energy_blocks_per_sm,
                                        o.energy_variant,   ms,              o.energy_kernel, o.tile_cells,
                                        o.persistent};
        ++n;
        if (ms < best_ms) {
            best_ms = ms;
            cur = o;
        }
        return GCMC_OK;
    };
    int st = GCMC_OK;
    // coordinate descent: pose-energy kernel x cell grid; then the tiled kernel's
    // pose-block edge, or the per-pose-warp kernel's work split, register budget
    // and CTAs per SM, whichever kernel won; then graph branches; then (several
    // replicas) the persistent step loop in place of the graph
    {
        const gcmc_options base0 = cur;
        for (int kern : {0, 1})
            for (int R : {1, 2, 3}) {
                gcmc_options o = base0;
                o.energy_kernel = kern;
                o.cells_per_cutoff = R;
                o.tile_cells = 0;
                if (st == GCMC_OK) st = consider(o);
            }
    }
    if (cur.energy_kernel > 0) {
        const int base_b = cur.tile_cells > 0 ? cur.tile_cells : cur.cells_per_cutoff;
        for (int B : {1, 2, 3}) {
            if (B == base_b) continue;
            gcmc_options o = cur;
            o.tile_cells = B;
            if (st == GCMC_OK) st = consider(o);
        }
    } else {
        const int base_split = cur.split_items;
        for (int sp : {512, 1024, 2048, 4096, 8192}) {
            if (sp == base_split) continue;
            gcmc_options o = cur;
            o.split_items = sp;
            if (st == GCMC_OK) st = consider(o);
        }
        {
            gcmc_options o = cur;
            o.energy_variant = cur.energy_variant == 1 ? 0 : 1;
            if (st == GCMC_OK) st = consider(o);
        }
        const int base_e = cur.energy_blocks_per_sm;
        for (int e : {0, 2, 1}) {
            if (e == base_e) continue;
            gcmc_options o = cur;
            o.energy_blocks_per_sm = e;
            if (st == GCMC_OK) st = consider(o);
        }
        {
            gcmc_options o = cur;
            o.pose_split = cur.pose_split > 0 ? 0 : 1;
            if (st == GCMC_OK) st = consider(o);
        }
    }
    const int base_br = cur.branches;
    for (int nb : {1, 2, 4}) {
        if (nb == base_br || nb > nrep) continue;
        gcmc_options o = cur;
        o.branches = nb;
        if (st == GCMC_OK) st = consider(o);
    }
    // several replicas with the per-pose-warp kernel: the persistent step loop
    if (nrep > 1 && cur.energy_kernel == 0 && cur.persistent <= 0) {
        gcmc_options o = cur;
        o.persistent = 1;
        o.branches = 1;
        if (st == GCMC_OK) st = consider(o);
    }
    if (ntrials) *ntrials = n;
    if (st != GCMC_OK) return st;
    cur.log_steps = base ? base->log_steps : 0;
    *best = cur;
    return GCMC_OK;
}

void* gcmc_stream(gcmc_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int gcmc_run(gcmc_ctx* ctx, int32_t nsteps) {
    if (!ctx) return GCMC_ERR_ARG;
    if (nsteps <= 0) return GCMC_OK;
    const int first = ctx->reps[0].host_end;
    int need = 0;
    for (auto& h : ctx->reps) {
        long long e = std::min<long long>((long long)h.host_end + nsteps, h.mcsteps);
        need = std::max(need, (int)(e - h.host_end));
        h.host_end = (int)e;
    }
    if (need == 0) return GCMC_OK;
    k_set_run_end<<<(ctx->nrep + 127) / 128, 128, 0, ctx->stream>>>(ctx->d_reps, ctx->nrep, nsteps);
    if (ctx->spec) {  // step `first` lives in descriptor copy first & 1
        k_spec_start<<<1, 32, 0, ctx->stream>>>((first & 1) ? ctx->d_reps_b : ctx->d_reps, first);
        CK(cudaGetLastError());
        for (int done = 0; done < need; done += kGraphSteps)
            CK(cudaGraphLaunch(ctx->gexec_spec[first & 1], ctx->stream));
        return GCMC_OK;
    }
    k_prepare<<<ctx->nrep, kAcceptThreads, prep_smem(ctx), ctx->stream>>>(ctx->d_reps, ctx->nrep);
    CK(cudaGetLastError());
    if (ctx->persist) {  // the whole step range in one cooperative launch
        CK(cudaMemsetAsync(ctx->d_sync, 0, sizeof(GridSync), ctx->stream));
        const RepDev* reps = ctx->d_reps;
        int nrep = ctx->nrep, nst = need;
        GridSync* gs = ctx->d_sync;
        long long cap = ctx->spin_cap;
        void* args[] = {(void*)&reps, (void*)&nrep, (void*)&nst, (void*)&gs, (void*)&cap};
        CK(cudaLaunchCooperativeKernel((const void*)k_persist, dim3(ctx->grid_persist), dim3(kAcceptThreads), args,
                                       sizeof(AcceptSmem), ctx->stream));
        return GCMC_OK;
    }
    for (int done = 0; done < need; done += kGraphSteps) CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    return GCMC_OK;
}

int gcmc_run_profiled(gcmc_ctx* ctx, int32_t nsteps, float* ms_energy, float* ms_accept, int32_t* move) {
    if (!ctx || nsteps < 0) return GCMC_ERR_ARG;
    if (nsteps == 0) return GCMC_OK;
    const int first = ctx->reps[0].host_end;
    int need = 0;
    for (auto& h : ctx->reps) {
        long long e = std::min<long long>((long long)h.host_end + nsteps, h.mcsteps);
        need = std::max(need, (int)(e - h.host_end));
        h.host_end = (int)e;
    }
    if (need == 0) return GCMC_OK;
    k_set_run_end<<<(ctx->nrep + 127) / 128, 128, 0, ctx->stream>>>(ctx->d_reps, ctx->nrep, nsteps);
    if (ctx->spec)  // timed one step after another: the first descriptor copy only
        k_prepare_at<<<1, kAcceptThreads, prep_smem(ctx), ctx->stream>>>(ctx->d_reps, first);
    else
        k_prepare<<<ctx->nrep, kAcceptThreads, prep_smem(ctx), ctx->stream>>>(ctx->d_reps, ctx->nrep);
    CK(cudaGetLastError());
    std::vector<cudaEvent_t> ev(3 * (size_t)need);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int i = 0; i < need; ++i) {
        for (int r = 0; r < ctx->nrep; ++r) {
            const int st = pme_update(ctx, r, ctx->stream);
            if (st != GCMC_OK) return st;
        }
        CK(cudaEventRecord(ev[3 * i], ctx->stream));
        if (ctx->fb) {
            fb_kernel(ctx)<<<ctx->gridF, kWarpsG * 32, 0, ctx->stream>>>(ctx->d_reps, ctx->nrep, 1);
            fb_kernel(ctx)<<<ctx->gridF, kWarpsG * 32, 0, ctx->stream>>>(ctx->d_reps, ctx->nrep, 2);
        } else {
            launch_energy(ctx, ctx->d_reps, ctx->nrep, 0, ctx->gridE, ctx->stream);
        }
        CK(cudaEventRecord(ev[3 * i + 1], ctx->stream));
        accept_kernel(ctx)<<<ctx->nrep, kAcceptThreads, sizeof(AcceptSmem), ctx->stream>>>(ctx->d_reps, ctx->nrep, 0);
        CK(cudaEventRecord(ev[3 * i + 2], ctx->stream));
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < need; ++i) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
        if (ms_energy) ms_energy[i] = a;
        if (ms_accept) ms_accept[i] = b;
        if (move) {
            const auto& mh = ctx->reps[0].moves_host;
            move[i] = (first + i < (int)mh.size()) ? mh[first + i] : -1;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return GCMC_OK;
}

int gcmc_device_error(gcmc_ctx* ctx, int32_t* err) {
    if (!ctx || !err) return GCMC_ERR_ARG;
    int acc = 0;
    for (auto& h : ctx->reps) {
        int e = 0;
        CK(cudaMemcpy(&e, h.err, sizeof(int), cudaMemcpyDeviceToHost));
        acc |= e;
    }
    *err = acc;
    return GCMC_OK;
}

int gcmc_sync(gcmc_ctx* ctx) {
    if (!ctx) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    int32_t err = 0;
    int st = gcmc_device_error(ctx, &err);
    if (st) return st;
    if (err) {
        std::fprintf(stderr, "gcmc_b200: device error flags 0x%x\n", err);
        return GCMC_ERR_DEVICE;
    }
    return GCMC_OK;
}

int gcmc_download(gcmc_ctx* ctx, int32_t rep, AtomArray* fragmentInfo, residue* residueInfo, Atom* atomInfo) {
    if (!ctx || rep < 0 || rep >= ctx->nrep) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    RepHost& h = ctx->reps[rep];
    std::vector<int> tot(h.ntypes);
    CK(cudaMemcpy(tot.data(), h.totalNum, sizeof(int) * h.ntypes, cudaMemcpyDeviceToHost));
    if (fragmentInfo)
        for (int t = 0; t < h.ntypes; ++t) fragmentInfo[t].totalNum = tot[t];
    if (residueInfo && h.ngroups > 0) {
        std::vector<float4> gcen(h.ngroups);
        CK(cudaMemcpy(gcen.data(), h.gcen, sizeof(float4) * h.ngroups, cudaMemcpyDeviceToHost));
        for (int g = 0; g < h.ngroups; ++g) {
            residueInfo[g].position[0] = gcen[g].x;
            residueInfo[g].position[1] = gcen[g].y;
            residueInfo[g].position[2] = gcen[g].z;
        }
    }
    if (atomInfo && h.natoms > 0) {
        std::vector<float4> xyzq(h.natoms);
        std::vector<int> atype(h.natoms);
        CK(cudaMemcpy(xyzq.data(), h.xyzq, sizeof(float4) * h.natoms, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(atype.data(), h.atype, sizeof(int) * h.natoms, cudaMemcpyDeviceToHost));
        for (int a = 0; a < h.natoms; ++a) {
            atomInfo[a].position[0] = xyzq[a].x;
            atomInfo[a].position[1] = xyzq[a].y;
            atomInfo[a].position[2] = xyzq[a].z;
            atomInfo[a].charge = xyzq[a].w;
            atomInfo[a].type = atype[a];
        }
    }
    return GCMC_OK;
}

int gcmc_get_logs(gcmc_ctx* ctx, int32_t rep, gcmc_step_log* logs, double* energies, int32_t max_steps,
                  int32_t* n_steps) {
    if (!ctx || rep < 0 || rep >= ctx->nrep) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    RepHost& h = ctx->reps[rep];
    int n = std::min(std::min(max_steps, h.log_cap), h.host_end);
    if (n_steps) *n_steps = n;
    if (n <= 0) return GCMC_OK;
    if (logs) CK(cudaMemcpy(logs, h.log, sizeof(gcmc_step_log) * n, cudaMemcpyDeviceToHost));
    if (energies) CK(cudaMemcpy(energies, h.logE, sizeof(double) * (size_t)n * h.log_kmax, cudaMemcpyDeviceToHost));
    return GCMC_OK;
}

int gcmc_get_forces(gcmc_ctx* ctx, int32_t rep, float* forces, int32_t max_steps, int32_t* n_steps) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !forces) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    RepHost& h = ctx->reps[rep];
    const int n = std::min(std::min(max_steps, h.log_cap), h.host_end);
    if (n_steps) *n_steps = std::max(0, n);
    if (n <= 0 || !ctx->repdev[rep].logF) return GCMC_OK;
    CK(cudaMemcpy(forces, h.logF, sizeof(float) * (size_t)n * h.log_kmax * 12, cudaMemcpyDeviceToHost));
    return GCMC_OK;
}

int gcmc_energy_total(gcmc_ctx* ctx, int32_t rep, double* e_total) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !e_total) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaMemcpy(e_total, ctx->reps[rep].energy, sizeof(double), cudaMemcpyDeviceToHost));
    return GCMC_OK;
}

int gcmc_pme_potential(gcmc_ctx* ctx, int32_t rep, const double* pts, int32_t n, double* out) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || n < 0 || (n > 0 && (!pts || !out))) return GCMC_ERR_ARG;
    if (!ctx->reps[rep].pme) return GCMC_ERR_ARG;
    if (n == 0) return GCMC_OK;
    int st = pme_update(ctx, rep, ctx->stream);
    if (st != GCMC_OK) return st;
    double *dp = nullptr, *dout = nullptr;
    if ((st = dalloc(&dp, (size_t)3 * n)) || (st = dalloc(&dout, (size_t)n))) {
        dfree(dp);
        return st;
    }
    cudaStream_t s = ctx->stream;
    if (cudaMemcpyAsync(dp, pts, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s) != cudaSuccess) st = GCMC_ERR_CUDA;
    if (st == GCMC_OK) {
        k_pme_phi_points<<<(n + 127) / 128, 128, 0, s>>>(ctx->d_reps + rep, dp, n, dout);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            st = GCMC_ERR_CUDA;
    }
    dfree(dp);
    dfree(dout);
    return st;
}

int gcmc_counters(gcmc_ctx* ctx, int32_t rep, int64_t* steps, int64_t* poses, int64_t* pairs) {
    if (!ctx || rep < 0 || rep >= ctx->nrep) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long c[4];
    CK(cudaMemcpy(c, ctx->reps[rep].counters, sizeof(c), cudaMemcpyDeviceToHost));
    if (steps) *steps = (int64_t)c[0];
    if (poses) *poses = (int64_t)c[1];
    if (pairs) *pairs = (int64_t)c[2];
    return GCMC_OK;
}

int gcmc_phase_cycles(gcmc_ctx* ctx, int32_t rep, int64_t* out8) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !out8) return GCMC_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long c[16];
    CK(cudaMemcpy(c, ctx->reps[rep].counters, sizeof(c), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 5; ++i) out8[i] = (int64_t)c[4 + i];
    out8[5] = (int64_t)c[12];  // speculative cluster rounds
    out8[6] = (int64_t)c[13];  // steps whose pose energies were evaluated in advance and kept
    out8[7] = 0;
    return GCMC_OK;
}

int gcmc_energy_poses(gcmc_ctx* ctx, int32_t rep, const float* xyz, const float* site_q,
                      const int32_t* site_type, int32_t nsites, const float* centres, const int32_t* self,
                      int32_t nposes, double* out, int32_t* n_groups) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !xyz || !site_q || !site_type || !centres || !out) return GCMC_ERR_ARG;
    if (nsites < 1 || nsites > kMaxSites) return GCMC_ERR_LIMIT;
    if (nposes <= 0) return GCMC_OK;
    RepHost& h = ctx->reps[rep];
    for (int s = 0; s < nsites; ++s)
        if (site_type[s] < 0 || site_type[s] >= h.ffX) return GCMC_ERR_ARG;
    const int nslab = h.nslab;
    float *dxyz = nullptr, *dq = nullptr, *dc = nullptr;
    int *dt = nullptr, *dself = nullptr, *dng = nullptr;
    double* dout = nullptr;
    int st = GCMC_OK;
    std::vector<int> selfv(nposes, -1);
    if (self) std::copy(self, self + nposes, selfv.begin());
    std::vector<double> part((size_t)nposes * nslab);
    std::vector<int> ngp((size_t)nposes * nslab);
    do {
        if ((st = dalloc(&dxyz, (size_t)nposes * nsites * 3)) || (st = dalloc(&dq, nsites)) ||
            (st = dalloc(&dt, nsites)) || (st = dalloc(&dc, (size_t)nposes * 3)) || (st = dalloc(&dself, nposes)) ||
            (st = dalloc(&dout, (size_t)nposes * nslab)) || (st = dalloc(&dng, (size_t)nposes * nslab)))
            break;
        cudaStream_t s = ctx->stream;
        if (cudaMemcpyAsync(dxyz, xyz, sizeof(float) * nposes * nsites * 3, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(dq, site_q, sizeof(float) * nsites, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(dt, site_type, sizeof(int) * nsites, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(dc, centres, sizeof(float) * nposes * 3, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(dself, selfv.data(), sizeof(int) * nposes, cudaMemcpyHostToDevice, s)) {
            st = GCMC_ERR_CUDA;
            break;
        }
        if ((st = pme_update(ctx, rep, s)) != GCMC_OK) break;
        k_energy_explicit<<<ctx->gridE, kWarpsE * 32, 0, s>>>(ctx->repdev[rep], dxyz, dq, dt, nsites, dc, dself,
                                                              nposes, nslab, dout, dng);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(part.data(), dout, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s) ||
            cudaMemcpyAsync(ngp.data(), dng, sizeof(int) * ngp.size(), cudaMemcpyDeviceToHost, s) ||
            cudaStreamSynchronize(s)) {
            st = GCMC_ERR_CUDA;
            break;
        }
        for (int p = 0; p < nposes; ++p) {
            double e = 0.0;
            int ng = 0;
            for (int z = 0; z < nslab; ++z) {
                e += part[(size_t)p * nslab + z];
                ng += ngp[(size_t)p * nslab + z];
            }
            out[p] = e;
            if (n_groups) n_groups[p] = ng;
        }
    } while (0);
    dfree(dxyz); dfree(dq); dfree(dt); dfree(dc); dfree(dself); dfree(dout); dfree(dng);
    if (st == GCMC_OK) {
        int32_t err = 0;
        gcmc_device_error(ctx, &err);
        if (err) st = GCMC_ERR_DEVICE;
    }
    return st;
}

int gcmc_energy_grad(gcmc_ctx* ctx, int32_t rep, const float* d_xyz, const float* d_site_q,
                     const int32_t* d_site_type, const int32_t* site_type, int32_t nsites, const float* d_centres,
                     const int32_t* d_self, int32_t nposes, const float* d_ff, const double* d_gout,
                     double* d_energy, double* d_gxyz, double* d_gq, double* d_gff, void* stream) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !d_xyz || !d_site_q || !d_site_type || !site_type || !d_centres)
        return GCMC_ERR_ARG;
    if (nsites < 1 || nsites > kMaxSites) return GCMC_ERR_LIMIT;
    if (d_gff && (!d_ff || !d_gout)) return GCMC_ERR_ARG;
    if (nposes <= 0) return GCMC_OK;
    RepHost& h = ctx->reps[rep];
    if (h.pme) return GCMC_ERR_ARG;  // gradients are of the plain-cutoff energy
    for (int s = 0; s < nsites; ++s)
        if (site_type[s] < 0 || site_type[s] >= h.ffX) return GCMC_ERR_ARG;
    const int nslab = h.nslab;
    const size_t ntab = (size_t)h.ffX * h.ffY;
    const size_t tab_smem = d_gff ? (size_t)nsites * h.ffY * 2 * sizeof(float) : 0;
    if (tab_smem > 160 * 1024) return GCMC_ERR_LIMIT;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    {
        const int ost = order_before(ctx, s);
        if (ost != GCMC_OK) return ost;
    }
    RepDev R = ctx->repdev[rep];
    float2* lj = nullptr;
    double *epart = nullptr, *glj = nullptr;
    int* ngpart = nullptr;
    float4* gpart = nullptr;
    int st = GCMC_OK;
    auto amalloc = [&](void** p, size_t bytes) {
        if (st == GCMC_OK && cudaMallocAsync(p, bytes, s) != cudaSuccess) st = GCMC_ERR_CUDA;
    };
    if (d_ff) {
        amalloc((void**)&lj, sizeof(float2) * ntab);
        if (st == GCMC_OK) {
            k_ff_to_lj<<<(int)((ntab + 255) / 256), 256, 0, s>>>(d_ff, lj, (int)ntab);
            R.lj = lj;
        }
    }
    if (d_energy) {
        amalloc((void**)&epart, sizeof(double) * nposes * nslab);
        amalloc((void**)&ngpart, sizeof(int) * nposes * nslab);
        if (st == GCMC_OK) {
            k_energy_explicit<<<ctx->gridE, kWarpsE * 32, 0, s>>>(R, d_xyz, d_site_q, d_site_type, nsites, d_centres,
                                                                  d_self, nposes, nslab, epart, ngpart);
            k_sum_parts<<<(nposes + 255) / 256, 256, 0, s>>>(epart, ngpart, nposes, nslab, d_energy, nullptr);
        }
    }
    if (d_gxyz || d_gq || d_gff) {
        amalloc((void**)&gpart, sizeof(float4) * nposes * nslab * nsites);
        if (d_gff) {
            amalloc((void**)&glj, sizeof(double) * ntab * 2);
            if (st == GCMC_OK && cudaMemsetAsync(glj, 0, sizeof(double) * ntab * 2, s) != cudaSuccess)
                st = GCMC_ERR_CUDA;
        }
        if (st == GCMC_OK && tab_smem > 0 &&
            cudaFuncSetAttribute(k_energy_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tab_smem) !=
                cudaSuccess)
            st = GCMC_ERR_CUDA;
        if (st == GCMC_OK) {
            int sms = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
            k_energy_grad<<<std::max(1, sms) * 4, kWarpsG * 32, tab_smem, s>>>(
                R, d_xyz, d_site_q, d_site_type, nsites, d_centres, d_self, nposes, nslab, d_gout, gpart, glj);
            if (d_gxyz || d_gq)
                k_sum_grad<<<(nposes * nsites + 255) / 256, 256, 0, s>>>(gpart, nposes, nslab, nsites, d_gxyz, d_gq);
            if (d_gff) k_glj_to_gff<<<(int)((ntab + 255) / 256), 256, 0, s>>>(glj, d_ff, d_gff, (int)ntab);
        }
    }
    if (st == GCMC_OK && cudaGetLastError() != cudaSuccess) st = GCMC_ERR_CUDA;
    if (lj) cudaFreeAsync(lj, s);
    if (epart) cudaFreeAsync(epart, s);
    if (ngpart) cudaFreeAsync(ngpart, s);
    if (gpart) cudaFreeAsync(gpart, s);
    if (glj) cudaFreeAsync(glj, s);
    if (st == GCMC_OK) st = order_after(ctx, s);
    return st;
}

int gcmc_run_gcmc(const InfoStruct* info, AtomArray* fragmentInfo, residue* residueInfo, Atom* atomInfo,
                  const float* grid, const float* ff, const int* moveArray, const gcmc_options* opt) {
    if (!info) return GCMC_ERR_ARG;
    gcmc_replica_in in{info, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray};
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    return cached_run(&g_cache, 1, &in, opt);
}

int gcmc_run_batch(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* opt) {
    if (!reps || nrep < 1) return GCMC_ERR_ARG;
    if (nrep > kMaxRep) return GCMC_ERR_LIMIT;
    for (int r = 0; r < nrep; ++r)
        if (!reps[r].info) return GCMC_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    return cached_run(&g_batch, nrep, reps, opt);
}

int gcmc_release_cache(void) {
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    if (g_cache) destroy_impl(g_cache);
    if (g_batch) destroy_impl(g_batch);
    g_cache = nullptr;
    g_batch = nullptr;
    return GCMC_OK;
}

void runGCMC_cuda(const InfoStruct* info, AtomArray* fragmentInfo, residue* residueInfo, Atom* atomInfo,
                  const float* grid, const float* ff, const int* moveArray) {
    g_last_status = gcmc_run_gcmc(info, fragmentInfo, residueInfo, atomInfo, grid, ff, moveArray, nullptr);
}

int gcmc_last_status(void) { return g_last_status; }

int gcmc_energy_poses_noalloc(gcmc_ctx* ctx, int32_t rep, const float* d_xyz, const float* d_site_q,
                              const int32_t* d_site_type, int32_t nsites, const float* d_centres,
                              const int32_t* d_self, int32_t nposes, double* d_out, int32_t* d_ngroups,
                              void* stream) {
    if (!ctx || rep < 0 || rep >= ctx->nrep || !d_xyz || !d_site_q || !d_site_type || !d_centres || !d_out)
        return GCMC_ERR_ARG;
    if (nsites < 1 || nsites > kMaxSites) return GCMC_ERR_LIMIT;
    if (nposes <= 0) return GCMC_OK;
    const int nslab = ctx->reps[rep].nslab;
    if ((long long)nposes * nslab > kNoAllocMaxParts) {
        std::fprintf(stderr,
                     "gcmc_b200: gcmc_energy_poses_noalloc: %d poses x %d splits exceed the %d partials of its "
                     "fixed %zu-byte scratch (at most %d poses per call for this context)\n",
                     nposes, nslab, kNoAllocMaxParts, kNoAllocScratchBytes, kNoAllocMaxParts / nslab);
        return GCMC_ERR_LIMIT;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev != ctx->device) return GCMC_ERR_ARG;
    void* scratch = nullptr;
    int st = noalloc_scratch(dev, &scratch);
    if (st != GCMC_OK) return st;
    double* part = reinterpret_cast<double*>(scratch);
    int* ngpart = reinterpret_cast<int*>(part + kNoAllocMaxParts);
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    if ((st = order_before(ctx, s)) != GCMC_OK) return st;
    {
        const int pst = pme_update(ctx, rep, s);
        if (pst != GCMC_OK) return pst;
    }
    k_energy_explicit<<<ctx->gridE, kWarpsE * 32, 0, s>>>(ctx->repdev[rep], d_xyz, d_site_q, d_site_type, nsites,
                                                          d_centres, d_self, nposes, nslab, part, ngpart);
    k_sum_parts<<<(nposes + 255) / 256, 256, 0, s>>>(part, ngpart, nposes, nslab, d_out, d_ngroups);
    CK(cudaGetLastError());
    return order_after(ctx, s);
}

}  // extern "C"
