/*
 * gcmc_b200 -- C ABI of the B200 GCMC engine (fragment-environment LJ+Coulomb
 * trial-move energies, cavity-bias insertion, on-device accept/update).
 *
 * The structs are byte-identical to pyGCMC's (gcmc/cpp/gcmc.h:47-100; numpy
 * mirror gcmc/python/values.py:18-62), so the caller's numpy structured arrays
 * are passed as plain pointers, exactly as the reference binding does
 * (gcmc/cpp/gcmc.cpp:176-182).
 *
 * Every entry point except runGCMC_cuda returns a gcmc_status (0 = success).
 * Pointers are host pointers unless stated otherwise; the library owns all
 * device memory it allocates and frees it in gcmc_destroy / before returning.
 */
#ifndef GCMC_B200_H
#define GCMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- state structs (gcmc/cpp/gcmc.h:47-100) ---------------- */
typedef struct { float position[3]; float charge; int32_t type; } Atom;          /* 20 B  */
typedef struct {
    char name[4];
    int32_t startRes;   /* first residue (slot) of this fragment type            */
    float muex;         /* excess chemical potential (see gcmc_options.muex_kcal) */
    float conc;         /* bulk concentration, mol/L                             */
    int32_t confBias;   /* trial poses per insertion / max fragments per move    */
    float mcTime;
    int32_t totalNum;   /* occupied slots [startRes, startRes+totalNum)           */
    int32_t maxNum;     /* slot capacity                                          */
    int32_t num_atoms;  /* sites per fragment, <= 20                              */
    Atom atoms[20];     /* template, centred at the origin                        */
} AtomArray;                                                                      /* 436 B */
typedef struct {
    int32_t mcsteps;
    float cutoff;        /* group-centre cutoff, A                                */
    float grid_dx;       /* cavity grid spacing and reference translate step, A  */
    float startxyz[3];   /* box origin                                            */
    float cryst[3];      /* box edges (orthorhombic, periodic)                    */
    int32_t showInfo;
    float cavityFactor;  /* empty voxels / all voxels                             */
    int32_t fragTypeNum;
    int32_t totalGridNum;
    int32_t totalResNum;
    int32_t totalAtomNum;
    int32_t ffXNum;      /* fragment atom types (rows of ff)                      */
    int32_t ffYNum;      /* all atom types (columns of ff)                        */
    int32_t PME;
    uint32_t seed;
} InfoStruct;                                                                     /* 76 B  */
typedef struct { float position[3]; int32_t atomNum; int32_t atomStart; } residue; /* 20 B */

/* ---------------- status codes ---------------- */
typedef enum {
    GCMC_OK = 0,
    GCMC_ERR_CUDA = 1,      /* a CUDA runtime call failed                          */
    GCMC_ERR_ARG = 2,       /* inconsistent or out-of-range input                  */
    GCMC_ERR_LIMIT = 3,     /* a documented size limit is exceeded                 */
    GCMC_ERR_DEVICE = 4,    /* the device raised an error flag (see gcmc_device_error) */
    GCMC_ERR_NODEVICE = 5   /* no CUDA device is visible                           */
} gcmc_status;

/* Engine options.  gcmc_default_options() gives the reference's semantics. */
typedef struct {
    int32_t proposal;    /* 0: reference proposals -- insertion axis in the positive
                            octant, translate by U(0,grid_dx] per axis (gcmc_energy.h:84,
                            gcmc_move_trn.h:58); 1: symmetric -- uniform SO(3)
                            insertion, translate in a cube of edge trn_step,
                            rotate about a uniform axis by up to rot_max;
                            2: force-biased (no counterpart in the reference) --
                            uniform SO(3) insertion; translate by d and rotate by
                            the rotation vector v (about the site centroid) whose
                            components lie in [-h, h] with density
                            ~ exp(beta f_c x / 2), f the force / torque at the old
                            pose (Pangali, Rao and Berne 1978), accepted with the
                            Metropolis-Hastings ratio of the proposal densities
                            (forces at the old and at the new pose)              */
    int32_t muex_kcal;   /* 0: beta*muex with beta in mol/kJ and muex as given
                            (gcmc_move_add.h:105); 1: muex in kcal/mol (x4.184)     */
    float trn_step;      /* symmetric translate cube edge, A                        */
    float rot_max;       /* symmetric rotate max angle, rad                         */
    uint32_t replica;    /* RNG stream id (the key's second word)                   */
    int32_t cells_per_cutoff; /* cell-grid resolution R (cells of >= cutoff/R); 0 = 2 */
    int32_t log_steps;   /* record per-step logs for this many steps (0 = off)      */
    int32_t log_kmax;    /* per-step pose energies recorded (<= 1024)               */
    int32_t split_items; /* pose-energy work items per step at most: each pose's cell
                            window is split into floor(split_items / poses) ranges (1 to
                            window cells / 8); 0 = one wave of the pose-energy grid (its
                            resident warps) */
    int32_t branches;    /* independent chains of the captured step loop: the
                            replicas are split into this many contiguous groups
                            (balanced by atom count) whose kernels run
                            concurrently; 0 = 1                                     */
    int32_t energy_blocks_per_sm; /* pose-energy kernel CTAs per SM (0 = the
                            occupancy limit)                                        */
    float fb_trn;        /* proposal 2: translate half-width h_t, A (0 = 0.5)        */
    float fb_rot;        /* proposal 2: rotation half-width h_r, rad (0 = 10 degrees)*/
    uint32_t step_offset; /* the RNG counts steps from this value: a context created
                            from a checkpoint taken after s steps, with moveArray
                            starting at step s and step_offset = s, continues the
                            same chain (0 for a fresh run)                         */
    int32_t pme;         /* Ewald electrostatics by smooth PME (no counterpart in the
                            reference): 1 on, -1 off, 0 = InfoStruct.PME decides.
                            Real-space Coulomb erfc(alpha r)/r in the group cutoff,
                            the reciprocal potential of the state on an FP64 mesh
                            rebuilt every step, order-4 B-splines; not with
                            proposal 2                                           */
    float pme_alpha;     /* Ewald splitting parameter, 1/A (0 = 0.32)              */
    int32_t pme_grid[3]; /* mesh points per axis (0 = box edge / 1.2 A rounded up to
                            a 2-3-5-7-smooth size)                                 */
    int32_t energy_variant; /* pose-energy kernel register budget: 0 = 3 CTAs per SM,
                            1 = 4 CTAs per SM (autotuned)                           */
    int32_t speculate;   /* one-replica contexts with one branch, no PME and proposal
                            0 or 1: each step's successor is prepared and its pose
                            energies evaluated while the step's accept kernel runs,
                            and kept when the step accepts nothing (the state is then
                            unchanged, so the results are those of the sequential
                            order); 0 = on, -1 = off                               */
    int32_t energy_kernel; /* 0: one warp per pose (variant) and cell range;
                            1: tiled pose energies where the context allows them
                            (no PME, proposal 0 or 1): the step's poses are binned
                            into blocks of tile_cells^3 cells and each block's window
                            of groups and atoms is staged in shared memory once for
                            all its poses (autotuned)                               */
    int32_t tile_cells;  /* tiled kernel: pose-block edge in cells (0 = cells_per_cutoff) */
    int32_t pair_delta;  /* 0: a translate / rotate step's energy changes in the
                            pairwise-difference form where the context allows it
                            (no PME, proposal 0 or 1): one evaluation per pose over
                            the groups within the cutoff of either centre, each
                            atom-site pair contributing its own change (the Coulomb
                            change from r_o^2 - r_n^2 = delta.(d_o + d_n)), so the
                            change carries the rounding of itself rather than of the
                            two pose energies; -1: E_new - E_old from two
                            evaluations                                         */
    int32_t persistent;  /* 1: run the step loop of a context without speculation,
                            PME or force bias, with the per-pose-warp pose-energy
                            kernel, as one cooperative launch (one CTA per SM: per
                            step all CTAs evaluate every replica's pose energies,
                            a grid barrier, CTA r accepts replica r's moves and
                            prepares its next step, a grid barrier) instead of a
                            captured graph of per-step launches; 0 = the graph   */
    int32_t persist_spin_cap; /* polls a CTA waits at the persistent loop's grid
                            barrier before it gives up, raises device error bit 5
                            and ends the launch (0 = 2^24, over a second)        */
    int32_t pose_split;  /* per-pose-warp kernel: 0 = every pose's cell window split into
                            the same number of ranges; 1 = each pose's window split in
                            proportion to its estimated work (the fixed atoms in the
                            windows of its centre's cell), the same total (an
                            autotuner candidate; slower than 0 on one replica)      */
    int32_t grid_bits;   /* 0 = the `grid` argument of the run entry points is the
                            reference's float list of insertion base points (x, y, z
                            per point); 1 = it is a gcmc_grid_bits record: the same
                            points as a voxel bit set, 1 bit per voxel instead of
                            12 bytes per point, expanded on the device (no
                            counterpart in the reference)                         */
} gcmc_options;

/* Cavity grid as a voxel bit set (gcmc_options.grid_bits = 1): this header,
 * followed directly by ceil(n[0] n[1] n[2] / 32) uint32 words; bit (v % 32) of
 * word v / 32 marks voxel v = (x n[1] + y) n[2] + z.  Insertion base point k is
 * the k-th marked voxel in increasing v, at ((float)(x dx + start[0]), ...),
 * each coordinate an FP64 product and sum rounded once to float -- the points
 * and the order gcmc_cavity_grid writes, so both forms give the same chains.
 * InfoStruct.totalGridNum must equal the number of marked voxels (else device
 * error bit 6 and GCMC_ERR_ARG); bits past the last voxel are ignored. */
typedef struct {
    double start[3];     /* lower corner of voxel (0, 0, 0)                         */
    double dx;           /* voxel edge                                              */
    int32_t n[3];        /* voxels per axis                                         */
    int32_t pad;
} gcmc_grid_bits;        /* 48 B */

/* One autotuner trial (gcmc_autotune). */
typedef struct {
    int32_t cells_per_cutoff, split_items, branches, energy_blocks_per_sm, energy_variant;
    float ms_per_step;   /* device time per MC step (all replicas)                  */
    int32_t energy_kernel, tile_cells, persistent;
} gcmc_tune_trial;

/* One per-step record (56 bytes). */
typedef struct {
    int32_t step, move, ftype, k;
    int32_t n_before, n_after, n_clusters, n_accept;
    int32_t first_accept;  /* pose index of the first accepted cluster, -1 if none */
    int32_t slot;          /* delete: chosen slot; otherwise -1                     */
    double e_sum;          /* sum of pose E (insert/delete) or dE (translate/rotate) */
    double e_total;        /* running sum of the accepted energy changes since the
                              context was created (kJ/mol, FP64), after this step   */
} gcmc_step_log;

typedef struct gcmc_ctx gcmc_ctx;

/* One replica's input (the reference's seven arrays, gcmc/cpp/gcmc.cu:21). */
typedef struct {
    const InfoStruct* info;
    const AtomArray* fragmentInfo;
    const residue* residueInfo;
    const Atom* atomInfo;
    const float* grid;
    const float* ff;
    const int32_t* moveArray;
} gcmc_replica_in;

/* Drop-in for runGCMC_cuda (gcmc/cpp/gcmc.cu:21, declared gcmc/cpp/gcmc.cpp:159):
 * runs info->mcsteps steps of moveArray and writes fragmentInfo[].totalNum,
 * residueInfo[] and atomInfo[] back in place.  Same void signature; the status
 * of the call is available from gcmc_last_status(). */
void runGCMC_cuda(const InfoStruct* info, AtomArray* fragmentInfo, residue* residueInfo,
                  Atom* atomInfo, const float* grid, const float* ff, const int* moveArray);

/* Same as runGCMC_cuda with options, returning the status.  Unlike the
 * reference (which allocates and frees all device buffers on every call,
 * gcmc/cpp/gcmc.cu:31-43,107-115), the device context of the last call is
 * kept and refilled by the next call on the same device (buffers grown only
 * when a larger system arrives); gcmc_release_cache() frees it.  Calls are
 * serialised by a lock. */
int gcmc_run_gcmc(const InfoStruct* info, AtomArray* fragmentInfo, residue* residueInfo,
                  Atom* atomInfo, const float* grid, const float* ff, const int* moveArray,
                  const gcmc_options* opt);
/* Free the device contexts kept between runGCMC_cuda / gcmc_run_gcmc /
 * gcmc_run_batch calls. */
int gcmc_release_cache(void);

/* Batched drop-in (no counterpart in the reference, which runs one system per
 * runGCMC_cuda call): runs each replica's info->mcsteps steps in ONE device
 * context -- all replicas advance together, one pose-energy launch and one
 * accept launch per MC step (a single replica speculates instead, see
 * gcmc_options.speculate) -- and writes every replica's totalNum,
 * residueInfo and atomInfo back in place (the arrays behind reps[r] are
 * written although the struct holds const pointers).  The context is kept
 * between calls with the same replica count, like gcmc_run_gcmc's. */
int gcmc_run_batch(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* opt);

/* Status of the last runGCMC_cuda call in this thread. */
int gcmc_last_status(void);
const char* gcmc_status_string(int status);
void gcmc_default_options(gcmc_options* opt);

/* ---- device-resident contexts (replaces the per-call allocation of
 *      gcmc/cpp/gcmc.cu:31-43; one context holds nrep independent replicas) ---- */
/* stream: a cudaStream_t to launch on (NULL = the library creates one). */
int gcmc_create(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* opt, void* stream,
                gcmc_ctx** out);
/* Advance every replica by nsteps steps of its move schedule (asynchronous). */
int gcmc_run(gcmc_ctx* ctx, int32_t nsteps);
/* Same as gcmc_run but launches each step's two kernels individually (no
 * graph) with CUDA events around them: per step, the pose-energy kernel time,
 * the accept kernel time (ms) and replica 0's move code.  Synchronous. */
int gcmc_run_profiled(gcmc_ctx* ctx, int32_t nsteps, float* ms_energy, float* ms_accept, int32_t* move);
/* Wait for the context's stream and report device-side errors. */
int gcmc_sync(gcmc_ctx* ctx);
/* Copy replica `rep`'s state back into the caller's arrays (sizes as created). */
int gcmc_download(gcmc_ctx* ctx, int32_t rep, AtomArray* fragmentInfo, residue* residueInfo,
                  Atom* atomInfo);
/* Per-step logs recorded since creation (needs opt.log_steps > 0).  energies
 * (optional) receives log_kmax doubles per step. */
int gcmc_get_logs(gcmc_ctx* ctx, int32_t rep, gcmc_step_log* logs, double* energies,
                  int32_t max_steps, int32_t* n_steps);
/* Ewald runs: the reciprocal-space potential (kJ/mol/e) of replica rep's
 * current state at n points (host arrays pts[3n], out[n]); rebuilds the mesh
 * first.  Synchronous. */
int gcmc_pme_potential(gcmc_ctx* ctx, int32_t rep, const double* pts, int32_t n, double* out);
/* Force-biased runs with logs: per step, log_kmax x 12 floats -- the force and
 * torque at the old pose, then at the new pose, of each translate/rotate pose
 * (as used by the proposal and the acceptance). */
int gcmc_get_forces(gcmc_ctx* ctx, int32_t rep, float* forces, int32_t max_steps, int32_t* n_steps);
/* Running sum of the accepted moves' energy changes since creation (FP64). */
int gcmc_energy_total(gcmc_ctx* ctx, int32_t rep, double* e_total);
/* Counters: steps done, pose energies evaluated, atom-site pairs evaluated. */
int gcmc_counters(gcmc_ctx* ctx, int32_t rep, int64_t* steps, int64_t* poses, int64_t* pairs);
/* SM cycles spent by replica `rep`'s accept kernel in its phases, summed over
 * steps: [0] pose energies, [1] per-pose weights and bit rows, [2] cluster
 * walk, [3] state update, [4] next-step preparation; [5] number of
 * speculative cluster rounds; [6] steps whose pose energies were evaluated
 * beside the previous step's accept kernel and kept (gcmc_options.speculate);
 * [7] reserved. */
int gcmc_phase_cycles(gcmc_ctx* ctx, int32_t rep, int64_t* out8);
/* Device error word (bit 0 cell overflow, bit 1 periodic image > 1 box,
 * bit 2 slot overflow, bit 3 pose limit, bit 4 an explicit pose's site type
 * outside the pair table -- gcmc_energy_poses_noalloc, whose device inputs the
 * host does not read; such a pose's energy is NaN; bit 5 the persistent step
 * loop's grid barrier waited longer than gcmc_options.persist_spin_cap, in
 * replica 0's word; bit 6 a gcmc_grid_bits record whose marked voxels do not
 * number InfoStruct.totalGridNum -- the run entry points report it as
 * GCMC_ERR_ARG). */
int gcmc_device_error(gcmc_ctx* ctx, int32_t* err);
/* The cudaStream_t the context launches on. */
void* gcmc_stream(gcmc_ctx* ctx);
int gcmc_destroy(gcmc_ctx* ctx);

/* Launch-shape autotuner (no counterpart in the reference).  For the given
 * replicas, times trial_steps MC steps (after 8 warm-up steps) on temporary
 * contexts for a coordinate-descent sequence of candidates -- pose-energy
 * kernel (energy_kernel 0 / 1) x cell-grid resolution (cells_per_cutoff 1..3);
 * then the tiled kernel's pose-block edge, or the per-pose-warp kernel's work
 * split (split_items 512..8192), register budget (energy_variant) and CTAs per
 * SM; graph branches (1, 2, 4); for several replicas the persistent step loop
 * -- and writes the base options with the fastest shape into *best.  trials
 * (optional, max_trials entries) receives each trial; *ntrials their number.
 * The inputs are not modified; the trajectories of a context created with
 * *best are the same MC chain up to FP32 summation order. */
int gcmc_autotune(int32_t nrep, const gcmc_replica_in* reps, const gcmc_options* base, int32_t trial_steps,
                  gcmc_options* best, gcmc_tune_trial* trials, int32_t max_trials, int32_t* ntrials);

/* Energies of explicit poses against replica `rep`'s current state
 * (the calcEnergy of gcmc/cpp/gcmc_energy.h:142-204, batched).
 * xyz[p*nsites*3], centres[p*3], self[p] (residue to skip, -1 = none);
 * site charges/types are shared by all poses.  out[p] in kJ/mol;
 * n_groups (optional) = groups inside the cutoff per pose. */
int gcmc_energy_poses(gcmc_ctx* ctx, int32_t rep, const float* xyz, const float* site_q,
                      const int32_t* site_type, int32_t nsites, const float* centres,
                      const int32_t* self, int32_t nposes, double* out, int32_t* n_groups);

/* Pose energies and their gradients (no counterpart in the reference, whose
 * calcEnergy, gcmc/cpp/gcmc_energy.h:142-204, has no derivative).  All arrays
 * are DEVICE pointers except site_type, a host copy of d_site_type used for
 * validation; launches on `stream` (NULL = the context's stream) and returns
 * without waiting (scratch comes from the stream-ordered allocator).  A
 * caller's stream first waits for the work queued on the context's stream, and
 * the context's stream then waits for the call's launches, so the call never
 * overlaps a gcmc_run of the same context.
 *   d_xyz[p*nsites*3], d_centres[p*3], d_self[p] (optional), d_site_q /
 *   d_site_type[nsites]: as gcmc_energy_poses;
 *   d_ff: pair table in the reference's layout (sigma [nm], eps [kJ/mol] per
 *     (site type, atom type), ffX*ffY*2 floats) used instead of the
 *     context's; NULL = the context's table;
 *   d_energy[p] (optional): E_p with that table (FP64 sums of FP32 terms, the
 *     arithmetic of gcmc_energy_poses);
 *   d_gxyz[p*nsites*3] (optional): dE_p / dx_{p,s};
 *   d_gq[p*nsites] (optional): dE_p / dq_s;
 *   d_gff[ffX*ffY*2] (optional; needs d_ff and d_gout): ADDS
 *     sum_p d_gout[p] * dE_p / dff.
 * Gradients are FP32 pair terms summed per lane in FP32 and across lanes and
 * cell ranges in FP64 (the table gradient per block in FP32).  Group
 * inclusion is by pose centre, as in the energy, so E is piecewise smooth in
 * the site coordinates and the centre carries no gradient. */
int gcmc_energy_grad(gcmc_ctx* ctx, int32_t rep, const float* d_xyz, const float* d_site_q,
                     const int32_t* d_site_type, const int32_t* site_type, int32_t nsites, const float* d_centres,
                     const int32_t* d_self, int32_t nposes, const float* d_ff, const double* d_gout,
                     double* d_energy, double* d_gxyz, double* d_gq, double* d_gff, void* stream);

/* Allocation-free variant of gcmc_energy_poses (no counterpart in the reference).
 *
 * For callers that cannot allocate GPU memory at the point where they need
 * trial energies: a host program that hands the whole device budget to its own
 * memory pool and forbids allocations by third-party code, or one running an
 * asynchronous pipeline that must not stall -- cudaMalloc/cudaFree (which
 * gcmc_energy_poses uses for its staging buffers) can block or synchronise the
 * device.  This entry point takes DEVICE pointers the caller already owns
 * (inputs as in gcmc_energy_poses; out[nposes] doubles; ngroups[nposes] ints,
 * optional; self optional = none skipped), launches on `stream` (NULL = the
 * context's stream), returns without waiting, and calls no allocator.  The
 * site types are device data the host does not read: a type outside the pair
 * table's rows gives that pose a NaN energy and sets bit 4 of the device error
 * word, which the next gcmc_sync reports as GCMC_ERR_DEVICE.  A caller's
 * stream first waits (an event wait) for the work queued on the context's
 * stream, and the context's stream then waits for the call's launches, so the
 * call never overlaps a gcmc_run of the same context; with Ewald the call
 * rebuilds the context's mesh on the caller's stream in that order.
 *
 * Its intermediate per-(pose, split) sums live in a fixed 2 MiB device array
 * inside the library, reserved on every GPU that loads the library until the
 * process exits.  Limit: nposes x splits <= 174762, where splits is the
 * context's number of work items per pose (at most ~11,600 poses for the
 * default cell grid); larger requests return GCMC_ERR_LIMIT and launch
 * nothing.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the one array and it keeps the last call's contents; every
 * entry a call reads is first written by that call, so nothing needs clearing,
 * but calls that overlap on the GPU (different streams, or different contexts
 * on the same device) race on it and must be serialised by the caller.
 * Device-side error flags are reported by the next gcmc_sync. */
int gcmc_energy_poses_noalloc(gcmc_ctx* ctx, int32_t rep, const float* d_xyz, const float* d_site_q,
                              const int32_t* d_site_type, int32_t nsites, const float* d_centres,
                              const int32_t* d_self, int32_t nposes, double* d_out, int32_t* d_ngroups,
                              void* stream);

/* ---- synthetic fixed-atom generators (host) ---- */
int gcmc_synth_chain_sphere(int n, const float centre[3], float radius, float step, float excl,
                            uint64_t seed, float* out_xyz, int* n_breaks);
int gcmc_synth_chain_slab(int n, float lo0, float hi0, float lo1, float hi1, float zc, float half,
                          float px, float py, float pore, float step, float excl, uint64_t seed,
                          float* out_xyz, int* n_breaks);
/* ---- host-side system assembly (the reference's input builders, C++) ---- */
/* get_grid (gcmc/python/dataset.py:21-139): box origin start[3] (centre of the
 * atoms' bounding box minus cryst/2), the lower corners of the empty voxels of
 * edge grid_dx in lexicographic (x, y, z) order (all voxels of a 1 A grid
 * without cavity bias) and the cavity factor.  pts == NULL: count only
 * (*npts); else pts[3 * cap].  GCMC_ERR_ARG when the factor is below 0.05,
 * where the reference exits (dataset.py:95-97). */
int gcmc_cavity_grid(int32_t n, const double* xyz, const double* cryst, double grid_dx, int32_t cavity_bias,
                     double* start, float* pts, int64_t cap, int64_t* npts, double* factor);
/* The same grid as a gcmc_grid_bits record (no counterpart in the reference):
 * *hdr and words[cap_words] (words == NULL: header and counts only); *nwords =
 * ceil(voxels / 32), *npts = marked voxels.  Errors as gcmc_cavity_grid. */
int gcmc_cavity_bits(int32_t n, const double* xyz, const double* cryst, double grid_dx, int32_t cavity_bias,
                     gcmc_grid_bits* hdr, uint32_t* words, int64_t cap_words, int64_t* nwords, int64_t* npts);
/* set_fixCut (gcmc/python/dataset.py:175-188): group id per atom (a new group
 * starts more than fix_cutoff from the current group's first atom); returns the
 * number of groups. */
int32_t gcmc_fix_groups(int32_t n, const double* xyz, double fix_cutoff, int32_t* group);
/* Unweighted centres of groups [starts[g], starts[g] + counts[g]) with the
 * reference's arithmetic (float32 running sums of float64 additions). */
int gcmc_group_centres(int32_t ngroups, const double* xyz, const int64_t* starts, const int32_t* counts,
                       float* out);
/* update_data's residue and atom arrays (gcmc/python/dataset.py:190-373): fixed
 * atoms grouped by fixed_group (contiguous runs), then per fragment type
 * max_num slots of num_atoms atoms, the first n_initial holding the given
 * copies (initial_xyz, concatenated by type) with the type's template charges
 * and types (tpl_q / tpl_type concatenated by type); start_res[f] out. */
int gcmc_fill_layout(int32_t nfix, const double* fixed_xyz, const double* fixed_q, const int32_t* fixed_type,
                     const int32_t* fixed_group, int32_t nfrag, const int32_t* max_num, const int32_t* num_atoms,
                     const float* tpl_q, const int32_t* tpl_type, const int32_t* n_initial,
                     const double* initial_xyz, int32_t total_res, int64_t total_atoms, residue* res, Atom* atoms,
                     int32_t* start_res);

/* get_data's fragment PDB records (gcmc/python/dataset.py:393-408): an ATOM line
 * per atom of every occupied slot (type, then slot order), serials / residue
 * numbers from serial0 / resnum0 wrapping at 99999 / 9999; atom_names holds 20
 * names of 4 chars per type.  Returns the bytes written, or, when out is NULL
 * or cap is short, the capacity to provide; -1 on bad input. */
int64_t gcmc_pdb_fragment_lines(int32_t nfrag, const AtomArray* fragmentInfo, const residue* residueInfo,
                                const Atom* atomInfo, const char* atom_names, int64_t serial0, int64_t resnum0,
                                char* out, int64_t cap);

/* count random non-clashing copies (sites >= min_dist from all atoms) of a rigid
 * template in the periodic box [lo, lo+L); out_xyz[count*nsites*3]. */
int gcmc_synth_place(int n_existing, const float* existing_xyz, const float lo[3], const float L[3],
                     const float* tpl_xyz, int nsites, int count, float min_dist, uint64_t seed,
                     float* out_xyz);

#ifdef __cplusplus
}
#endif
#endif
