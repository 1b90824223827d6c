/*
 * CPU oracle for the GCMC hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is a plain-C restatement of the reference's energy routine and
 * move/accept logic.  Only the test suite, the smoke check and the CPU-baseline
 * leg of the benchmark may load it; the product never links or calls it.
 *
 * What it restates (paths relative to the pyGCMC source tree):
 *   - ABI structs ........................ gcmc/cpp/gcmc.h:47-100
 *   - calcEnergy / distanceP / fast_round  gcmc/cpp/gcmc_energy.h:110-204
 *   - randomFragment / rotate_atoms_shared gcmc/cpp/gcmc_energy.h:29-107
 *   - move_add   (cluster + Rosenbluth) .. gcmc/cpp/gcmc_move_add.h:86-201
 *   - move_del   (GC deletion) ........... gcmc/cpp/gcmc_move_del.h:97-187
 *   - move_trn / move_rot ................ gcmc/cpp/gcmc_move_trn.h:125-253,
 *                                          gcmc/cpp/gcmc_move_rot.h:151-275
 *   - step loop .......................... gcmc/cpp/gcmc.cu:77-98
 *
 * Random numbers: the reference draws from cuRAND XORWOW and glibc rand(); this
 * oracle (and the CUDA engine it checks) draws from a counter-based
 * Philox4x32-10 stream keyed by (seed, replica) with counter (step, index,
 * purpose, draw), so both make the same proposals and decisions.
 */
#ifndef GCMC_ORACLE_H
#define GCMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference ABI (gcmc/cpp/gcmc.h:47-100), packed 20/436/76/20 bytes ---- */
typedef struct { float position[3]; float charge; int32_t type; } or_atom;
typedef struct {
    char name[4];
    int32_t startRes;
    float muex;
    float conc;
    int32_t confBias;
    float mcTime;
    int32_t totalNum;
    int32_t maxNum;
    int32_t num_atoms;
    or_atom atoms[20];
} or_atomarray;
typedef struct {
    int32_t mcsteps;
    float cutoff;
    float grid_dx;
    float startxyz[3];
    float cryst[3];
    int32_t showInfo;
    float cavityFactor;
    int32_t fragTypeNum;
    int32_t totalGridNum;
    int32_t totalResNum;
    int32_t totalAtomNum;
    int32_t ffXNum;
    int32_t ffYNum;
    int32_t PME;
    uint32_t seed;
} or_info;
typedef struct { float position[3]; int32_t atomNum; int32_t atomStart; } or_residue;

/* ---- engine options (same meaning as gcmc_options in include/gcmc_b200.h) ---- */
typedef struct {
    int32_t proposal;   /* 0: reference, 1: symmetric, 2: force-biased proposals */
    int32_t muex_kcal;  /* 0: beta*muex with muex as given, 1: muex in kcal/mol */
    float trn_step;     /* symmetric translate: cube edge (A)                   */
    float rot_max;      /* symmetric rotate: max angle (rad)                    */
    uint32_t replica;   /* RNG stream id                                        */
    float fb_trn;       /* proposal 2: translate half-width (A)                 */
    float fb_rot;       /* proposal 2: rotation half-width (rad)                */
    int32_t pme;        /* 1: Ewald electrostatics (erfc real space, exact k-space
                           potential of the environment, background term)       */
    float pme_alpha;    /* Ewald splitting parameter (1/A)                      */
} or_options;

/* Per-step record; identical layout to gcmc_step_log in include/gcmc_b200.h. */
typedef struct {
    int32_t step, move, ftype, k;
    int32_t n_before, n_after, n_clusters, n_accept;
    int32_t first_accept;   /* pose index of the first accepted cluster, -1 if none */
    int32_t slot;           /* delete: chosen slot; otherwise -1                    */
    double e_sum;           /* sum over poses of E (insert/delete) or dE (trn/rot)  */
    double e_total;         /* running sum of accepted energy changes after the step */
} or_step_log;

/* Counter-based RNG: Philox4x32-10. */
void or_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Own sin/cos (Taylor polynomials, Cody-Waite reduction) -- identical to the engine's. */
void or_det_sincos(float x, float* s, float* c);

/* Bit-exact FP32 group-inclusion distance (device distanceP form) and the
 * clustering distance (host distanceP form). */
float or_dist_group(const float a[3], const float b[3], const float L[3]);
float or_dist_host(const float a[3], const float b[3], const float L[3]);

/* Energy of one pose against the state.  mode 0: FP64, mode 1: FP32 mirror of
 * the reference kernel's arithmetic and summation order.  self = residue index
 * to skip (-1 for none).  n_groups/pairs (optional) return the included group
 * count and the number of atom-site pairs evaluated. */
double or_pose_energy(const or_info* info, const or_atomarray* frag, const or_residue* res,
                      const or_atom* atoms, const float* ff, const float (*site_xyz)[3],
                      const float* site_q, const int32_t* site_type, int32_t nsites,
                      const float centre[3], int32_t self, int32_t mode,
                      int32_t* n_groups, int64_t* pairs);

/* Same, also returning l1 = sum over pairs of |LJ| + |Coulomb| (FP64 only):
 * the condition of the energy sum, to which its relative tolerance refers. */
double or_pose_energy_l1(const or_info* info, const or_atomarray* frag, const or_residue* res,
                         const or_atom* atoms, const float* ff, const float (*site_xyz)[3],
                         const float* site_q, const int32_t* site_type, int32_t nsites,
                         const float centre[3], int32_t self, int32_t mode,
                         int32_t* n_groups, int64_t* pairs, double* l1);

/* Build the pose of insertion trial i at step t (sites and centre). */
void or_insert_pose(const or_info* info, const or_atomarray* frag, const float* grid,
                    const or_options* opt, int32_t ftype, int32_t step, int32_t i,
                    float (*xyz)[3], float centre[3]);
/* Trial t/r move of the fragment in slot `slot` (pose index i). */
void or_move_pose(const or_info* info, const or_atomarray* frag, const or_residue* res,
                  const or_atom* atoms, const or_options* opt, int32_t ftype, int32_t move,
                  int32_t step, int32_t i, int32_t slot, float (*xyz)[3], float centre[3]);
/* Slot picked for translate/rotate pose i (keyed permutation of [0,n)). */
int32_t or_perm_slot(const or_options* opt, uint32_t seed, int32_t step, int32_t i, int32_t n);

/* Rodrigues rotation of one point (axis normalised internally); R_out optional (row-major). */
void or_rotate_point(const float axis[3], float angle, const float p[3], float out[3], float R_out[9]);

/* Run steps [step0, step0+nsteps) of the move schedule in place.
 * energies (optional): per step, k doubles (E for insert/delete, dE for
 * translate/rotate) at energies[s*kmax + i]; replay_energies (optional): same
 * layout -- when given, decisions use these energies (replay of another
 * engine's energies) while the oracle's own FP64 energies go to `energies`.
 * escale (optional, same layout): the l1 magnitude (sum of |pair terms|) of
 * each insert/delete energy, and l1(new) + l1(old) for translate/rotate --
 * the magnitude the relative energy tolerance refers to.  Returns 0, or a negative error code. */
int32_t or_run(const or_info* info, or_atomarray* frag, or_residue* res, or_atom* atoms,
               const float* grid, const float* ff, const int32_t* moves, const or_options* opt,
               int32_t step0, int32_t nsteps, or_step_log* log, double* energies, double* escale,
               const double* replay_energies, int32_t kmax, int32_t threads);

/* or_run with the force-biased (proposal 2) and running-energy extensions:
 * e_total (in/out, optional): running sum of the accepted moves' energy
 * changes (the energies decisions use); forces (optional, [s*kmax + i][12]):
 * the oracle's FP64 force and torque at the old and at the new pose of each
 * force-biased translate/rotate pose; fscale ([s*kmax + i][4], optional): their
 * l1 scales (sum of |pair terms| of the force, and of |r| times them for the
 * torque); replay_forces ([s*kmax + i][12], optional): forces to use instead
 * of the oracle's own (as float, the values another engine used). */
/* Counts of the acceptance decisions made since the last reset and of those
 * whose draw lies within the per-trial energy tolerance of the threshold, and
 * the smallest margin / tolerance seen. */
void or_decision_stats(int32_t reset, int64_t* total, int64_t* band, double* min_ratio);

int32_t or_run_ext(const or_info* info, or_atomarray* frag, or_residue* res, or_atom* atoms,
                   const float* grid, const float* ff, const int32_t* moves, const or_options* opt,
                   int32_t step0, int32_t nsteps, or_step_log* log, double* energies, double* escale,
                   const double* replay_energies, int32_t kmax, int32_t threads, double* e_total,
                   double* forces, double* fscale, const float* replay_forces);

/* Ewald reciprocal-space potential of the current state (fixed atoms and
 * occupied slots) at n points: phi(r) = (K / (pi V)) sum_{m != 0}
 * exp(-pi^2 m^2 / alpha^2) / m^2 Re[S(m) exp(-2 pi i m.r)], S(m) = sum_j q_j
 * exp(2 pi i m.r_j), summed over all m with exp(-pi^2 m^2 / alpha^2) > 1e-13. */
void or_ewald_potential(const or_info* info, const or_atomarray* frag, const or_residue* res, const or_atom* atoms,
                        double alpha, const double* pts, int32_t n, double* out, int32_t threads);

/* Own float log and exp(x <= 0), identical to the engine's (force-biased proposals). */
float or_det_log(float x);
float or_det_exp_neg(float x);

/* Energies of many explicit poses (OpenMP over poses): poses_xyz[p*nsites*3],
 * centres[p*3], self[p]; returns pair count. */
int64_t or_energy_batch(const or_info* info, const or_atomarray* frag, const or_residue* res,
                        const or_atom* atoms, const float* ff, const float* poses_xyz,
                        const float* site_q, const int32_t* site_type, int32_t nsites,
                        const float* centres, const int32_t* self, int32_t nposes,
                        int32_t mode, double* out, int32_t* n_groups, double* l1, int32_t threads);

/* FP64 energies of explicit poses with FP64 sites, charges and pair table
 * (same inclusion as or_energy_batch; for finite differences). */
int64_t or_energy_batch64(const or_info* info, const or_atomarray* frag, const or_residue* res,
                          const or_atom* atoms, const double* ff64, const double* xyz64, const double* q64,
                          const int32_t* site_type, int32_t nsites, const float* centres, const int32_t* self,
                          int32_t nposes, double* out, int32_t* n_groups, int32_t threads);

/* FP64 analytic gradients of those energies: gxyz[p][s][3] = dE_p/dx_s,
 * gq[p][s] = dE_p/dq_s, gff[ffX*ffY*2] = sum_p gout[p] dE_p/dff (sigma, eps)
 * (gff optional; gout NULL = all ones), with the l1 scales of each (sums of
 * |pair terms|; optional). */
int64_t or_grad_batch(const or_info* info, const or_atomarray* frag, const or_residue* res, const or_atom* atoms,
                      const double* ff64, const double* xyz64, const double* q64, const int32_t* site_type,
                      int32_t nsites, const float* centres, const int32_t* self, int32_t nposes,
                      const double* gout, double* gxyz, double* gq, double* gff, double* gxyz_l1, double* gq_l1,
                      double* gff_l1, int32_t threads);

#ifdef __cplusplus
}
#endif
#endif
