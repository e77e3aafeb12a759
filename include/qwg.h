/*
 * qwg.h -- C-ABI of the B200 walker engine for QWalk VMC/DMC.
 *
 * One opaque context = one system (deck) + one resident walker population on
 * one GPU, bound to one CUDA stream.  All entry points return an int status
 * (QWG_OK or a negative error class); qwg_last_error() gives the text.  No C++
 * exceptions cross this boundary.  Host buffers are caller-owned; device
 * memory is owned by the context.
 *
 * Reference interfaces each entry point replaces (QWalk/mainline src/):
 *   qwg_create          System / Pseudopotential / Wavefunction_data factories
 *                       driven by the input file: allocate(System)
 *                       system/System.cpp:29-49, System::generatePseudo
 *                       system/System.cpp:145-149, allocate(Wavefunction_data)
 *                       wavefunction/Wavefunction_data.cpp:32-59 (module chosen
 *                       by the first word of each section, same grammar as
 *                       program_utils/qmc_io.cpp:280-345).
 *   qwg_set_walkers /   Config_save_point::restorePos / savePos
 *   qwg_get_walkers     system/Sample_point.cpp:61-85 (walker positions, 3N
 *                       doubles each).
 *   qwg_eval            Slat_Jastrow::updateLap + getVal + getLap for every
 *                       electron (wavefunction/Slat_Jastrow.cpp:101-123,
 *                       235-381), System::calcKinetic (system/System.cpp:105-140),
 *                       System::calcLoc (system/Molecular_system.cpp:209-287)
 *                       and Pseudopotential::calcNonlocWithTest in its
 *                       deterministic mode (system/Pseudopotential.cpp:412-424,
 *                       596-815), batched over walkers.
 *   qwg_ratio           Sample_point::setElectronPos + Wavefunction::updateLap +
 *                       getVal/getLap for one electron per walker
 *                       (wavefunction/Slat_wf.h:1145-1172, Jastrow2_wf.cpp:988-1157).
 *   qwg_vmc_block       Vmc_method::runWithVariables, one block
 *                       (method/Vmc_method.cpp:389-536) with the Split_sampler
 *                       depth-1 move (method/Split_sample.cpp:380-540).
 *   qwg_dmc_block       Dmc_method::runWithVariables, one block
 *                       (method/Dmc_method.cpp:373-552): moves, gatherData,
 *                       getWeight (:801-824), updateEtrial (:780-797),
 *                       calcBranch/match_walkers (:961-1156).
 *   qwg_dmc_init        Dmc_method::restorecheckpoint tail: gatherData for every
 *                       walker, find_cutoffs (:262-300), updateEtrial.
 */
#ifndef QWG_H
#define QWG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QWG_OK 0
#define QWG_ERR_ARG -1      /* bad argument / size beyond a limit */
#define QWG_ERR_INPUT -2    /* deck or orbital file could not be read/understood */
#define QWG_ERR_CUDA -3     /* CUDA runtime error */
#define QWG_ERR_STATE -4    /* call made in the wrong state (e.g. no walkers) */
#define QWG_ERR_NUMERIC -5  /* non-finite walker or singular determinant */

#define QWG_FP64 0          /* all arithmetic in double precision */
#define QWG_MIXED 1         /* FP32 basis/MO/ratios/inverse; FP64 LU refresh,
                               log|det|, energies and weights */

typedef struct qwg_ctx qwg_ctx;

typedef struct {
  int nelec, nup, ndown, natoms, nbasis, nshell, nmo_up, nmo_down;
  int has_pseudo;      /* 1 if any atom carries a PSEUDO section */
  int max_walkers;
  int precision;
  int walkers_per_cta; /* launch shape picked at create time */
  double ion_ion;      /* constant ion-ion energy */
  unsigned long long device_bytes; /* device memory a context of max_walkers holds */
  int complex_orbitals; /* 1: complex-orbital kernels (CORBITALS, or a nonzero KPOINT) */
} qwg_info;

/* Per-walker outputs of qwg_eval (host arrays, caller-owned, sized by nw). */
typedef struct {
  double* logpsi;      /* [nw]          ln|psi|                        */
  double* sign;        /* [nw]          sign of psi; complex orbitals: arg psi (radians) */
  double* grad;        /* [nw][nelec][3] grad ln|psi| per electron     */
  double* lap;         /* [nw][nelec]   Re (lap psi)/psi per electron  */
  double* kinetic;     /* [nw]  -1/2 sum_e lap                         */
  double* potential;   /* [nw]  Coulomb e-e, e-i, i-i                  */
  double* nonlocal;    /* [nw]  pseudopotential (local + nonlocal)     */
} qwg_eval_out;

/* Block statistics (weighted averages over steps x walkers in the block,
 * Properties_manager::endBlock, properties/Properties.cpp:578-652). */
typedef struct {
  double energy, kinetic, potential, nonlocal;
  double weight;          /* average walker weight                      */
  double energy_var;      /* weighted variance of E_L over the block    */
  double acceptance;      /* accepted / attempted single-electron moves */
  double etrial;          /* E_T after the block                        */
  double block_ms;        /* device time of the block (CUDA events)     */
  int nsteps, nwalkers;
  int nonfinite;          /* walkers whose E_L or weight went non-finite */
  /* Point statistics of the block as Properties_manager::endBlock keeps them
   * for the log (properties/Properties.cpp:574-640): npoints = walker-steps,
   * var_* = unweighted sample variance over those points, n/(n-1) corrected. */
  double npoints;
  double var_energy, var_kinetic, var_potential, var_nonlocal, var_weight;
} qwg_block_stats;

/* DMC parameters (Dmc_method::read defaults, method/Dmc_method.cpp:33-160). */
typedef struct {
  double timestep;        /* TIMESTEP                                   */
  int nstep;              /* steps per block (default 1/tau)            */
  int feedback_interval;  /* FEEDBACK_INTERVAL (5)                      */
  double feedback;        /* FEEDBACK (1.0)                             */
  double max_poss_weight; /* MAX_POSS_WEIGHT (7.0)                      */
  double branch_start_cutoff; /* BRANCH_START_CUTOFF (10); stop = 1.5x  */
  int refresh_interval;   /* steps between full recomputes (MIXED: LU refresh) */
  int deterministic_pp;   /* 1: evaluate every pair inside the cutoff   */
  uint64_t seed;
  int tmoves;             /* 0: locality approximation; 1: TMOVES (one T-move per
                             walker per step); 2: TMOVESSC (size-consistent, one per
                             electron) -- Dmc_method::doTmove, method/Dmc_method.cpp:850-906 */
} qwg_dmc_params;

const char* qwg_version(void);
const char* qwg_last_error(const qwg_ctx* ctx);

/* Build a context from a QWalk input file.  stream may be NULL (the context
 * then creates its own) or a cudaStream_t the caller owns.  On failure *out is
 * NULL and qwg_last_error(NULL) returns the reason (per calling thread). */
int qwg_create(const char* deck_path, int precision, int max_walkers, void* stream, qwg_ctx** out);
int qwg_destroy(qwg_ctx* ctx);
int qwg_get_info(const qwg_ctx* ctx, qwg_info* info);

/* Host-side table check without a GPU: parse the deck and build the device
 * tables on the host only; returns sizes through info.  Used by CPU tests. */
int qwg_inspect_deck(const char* deck_path, qwg_info* info, char* err, int errlen);
/* Device memory (bytes) qwg_create would hold for this deck, precision and
 * walker count, computed on the host from the same layout (tables, walker
 * state, scratch, DMC buffers).  No counterpart in the reference, which has
 * no device memory; used for admission control. */
int qwg_footprint(const char* deck_path, int precision, int max_walkers, unsigned long long* bytes);
/* Radial spline table of basis shell s (host copy, [npts][4]); npts returned. */
int qwg_inspect_spline(const char* deck_path, int shell, double* coef, int maxpts, int* npts,
                       double* spacing, double* cutoff);

/* Walker positions: R is [nw][nelec][3] doubles.  Host buffers. */
int qwg_set_walkers(qwg_ctx* ctx, const double* R, int nw);
int qwg_get_walkers(qwg_ctx* ctx, double* R, int nw);
/* Device-buffer variants (pointers in device memory, stream-ordered). */
int qwg_set_walkers_device(qwg_ctx* ctx, const double* dR, int nw);
/* Per-walker scalars after the last VMC/DMC step: local energy and DMC weight
 * (1 in VMC) of each walker, as Dmc_point keeps them (method/Dmc_method.h:62-82:
 * prop.energy, weight).  energy / weight: host arrays of nw doubles, either
 * may be NULL.  QWG_ERR_STATE before any block has run on these walkers. */
int qwg_get_walker_scalars(qwg_ctx* ctx, double* energy, double* weight, int nw);

/* Full evaluation of every resident walker.  rot: [nw][3][3] quadrature
 * rotations (rows x,y,z; Pseudopotential::rotateQuadrature) or NULL for the
 * unrotated points.  The pseudopotential is evaluated deterministically. */
int qwg_eval(qwg_ctx* ctx, const double* rot, qwg_eval_out* out);

/* Single-electron move per walker: electron e[w] to Rnew[w][3].  Returns
 * ln|psi'|-ln|psi|, sign ratio (complex orbitals: the phase change
 * arg(psi'/psi) in radians), grad ln|psi'| [nw][3] and Re lap psi'/psi' of
 * the moved electron. */
int qwg_ratio(qwg_ctx* ctx, const int* e, const double* Rnew, double* dlogpsi, double* sign,
              double* grad, double* lap);

/* VMC move dynamics, the DYNAMICS { SPLIT DEPTH d DIVIDER x } section of a
 * VMC method (method/Vmc_method.cpp:75-82, Split_sampler::split_driver,
 * method/Split_sample.cpp:380-478).  depth 2 (the default, with divider 2):
 * a rejected move is retried from the same point with timestep tau/divider
 * and the delayed-rejection acceptance (Split_sample.cpp:302-373); depth 1:
 * one attempt.  DMC always uses depth 1, as the reference does. */
int qwg_set_vmc_dynamics(qwg_ctx* ctx, int depth, double divider);

/* VMC block on the resident walkers: nstep sweeps (each = one drift-diffusion
 * Metropolis move per electron + one local energy).  stochastic PP unless
 * deterministic_pp. */
int qwg_vmc_block(qwg_ctx* ctx, int nstep, double timestep, uint64_t seed, int deterministic_pp,
                  qwg_block_stats* stats);

/* DMC: initialise (energies of the resident walkers, E_ref, branch cut-offs,
 * E_T), then run blocks on the device-resident population. */
int qwg_dmc_init(qwg_ctx* ctx, const qwg_dmc_params* p);
int qwg_dmc_block(qwg_ctx* ctx, qwg_block_stats* stats);
/* The same block split in two: _async enqueues it on the context's stream
 * (one CUDA graph launch: every feedback interval, branching and the E_ref/E_T
 * update run on the device) and returns at once; _wait blocks until it is
 * done and returns its statistics.  Blocks of several contexts on different
 * streams overlap on the GPU (Dmc_method::runWithVariables, one block). */
int qwg_dmc_block_async(qwg_ctx* ctx);
int qwg_dmc_block_wait(qwg_ctx* ctx, qwg_block_stats* stats);
/* 1 when the block in flight has finished (qwg_dmc_block_wait returns at
 * once), 0 while it runs; negative error code otherwise.  Does not block. */
int qwg_dmc_block_ready(qwg_ctx* ctx);

/* VMC block that allocates no device memory.
 *
 * No counterpart in the reference: QWalk's walker loop runs on the CPU.
 *
 * For callers that must not allocate device memory while they run: a serving
 * loop that has already divided HBM among the jobs it admitted, a host that
 * works inside a fixed device-memory budget owned by another allocator, or
 * code with kernels of other jobs in flight that must not wait on the
 * device-wide synchronisation cudaMalloc/cudaFree can cause.  The context
 * (tables) is built beforehand with qwg_create; this call then only launches.
 *
 * It runs the same kernel as qwg_vmc_block, but the walkers' resident state
 * and the block accumulators live in one file-scope device array of
 * QWG_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU loading the library holds
 * until the process exits.  nw * (per-walker state bytes) + 256 must fit in
 * it; systems with more than 32 orbitals per spin keep their per-walker
 * scratch there too, so for them nw * (state + scratch bytes) + 256 must fit.
 * Otherwise QWG_ERR_ARG (qwg_last_error names the largest nw that fits).
 * Buffers are the caller's device memory, ordered on the context's stream:
 *   d_R       [nw][nelec][3] walker positions, read and overwritten
 *   d_energy  [nw] local energy of each walker after the last step (or NULL)
 *   d_sums    [10] block sums: sum w, sum wE, sum wT, sum wV, sum wV_NL,
 *             sum wE^2, accepted moves, attempted moves, non-finite, points
 * The first call on a device looks up that device's address of the array
 * (cudaGetSymbolAddress, with that device current) and keeps it for the rest
 * of the process; make that first call before any stream capture.  A
 * cudaDeviceReset by the host invalidates the kept address: do not call this
 * entry point again on a device after resetting it.  These calls count their
 * own steps for the random streams (a separate counter from qwg_vmc_block and
 * the DMC calls), so they do not shift the streams or the refresh schedule of
 * the context's regular walkers.  All calls share the one array and it keeps the
 * last call's contents: the accumulators are cleared on every call, and calls
 * whose work overlaps on the GPU (other streams, other contexts) race on it. */
#define QWG_NOALLOC_SCRATCH_BYTES (16u << 20)
int qwg_vmc_block_noalloc(qwg_ctx* ctx, double* d_R, int nw, int nstep, double timestep, uint64_t seed,
                          int deterministic_pp, double* d_energy, double* d_sums);

/* MO value, gradient and Laplacian of every orbital of one spin at npos
 * positions: out[p][j][0..4] = (phi_j, d/dx, d/dy, d/dz, lap) at pos[p][0..2]
 * (host arrays; periodic systems wrap the positions into the cell).
 * Templated_MO_matrix::updateLap (orbitals/MO_matrix.h:101-118) for a batch of
 * positions, the product of MO_matrix_blas::updateLap
 * (orbitals/MO_matrix_blas.h:411-491).  QWG_FP64 contexts contract on CUDA
 * cores in FP64; QWG_MIXED contexts contract all positions in one
 * tensor-core GEMM (tcgen05, split TF32 with FP32 accumulation, TMA-staged
 * tiles).  Real orbitals only (QWG_ERR_ARG for complex ones). */
int qwg_mo_eval(qwg_ctx* ctx, const double* pos, int npos, int spin, double* out);

/* Walker-kernel phase counters (no counterpart in the reference: a profiling
 * aid).  In the profiling build libqwg_phases.so every walker's warp adds the
 * clock cycles it spends in each phase: out[0] MO rows of proposals, [1] rest
 * of a proposal (ratio, drift, Jastrow), [2] Sherman-Morrison updates, [3]
 * kinetic energy, [4] Coulomb/Ewald, [5] quadrature Jastrow values, [6]
 * quadrature pairs, [7] projected coefficients, [8] quadrature points, [9]
 * full recomputes, [10] whole step-mode launches; n <= 16 counters are
 * copied, reset != 0 clears them.  The regular library returns
 * QWG_ERR_STATE. */
int qwg_phase_counters(qwg_ctx* ctx, unsigned long long* out, int n, int reset);

/* Batched uneven systems: one CUDA graph holding one DMC block of every
 * context (each on its own stream, forked and joined inside the graph), so a
 * single graph launch advances all systems concurrently.  Every context must
 * have had qwg_dmc_init.  qwg_batch_block launches the graph, waits, and
 * fills stats[i] for context i.  (Dmc_method::runWithVariables per system;
 * QWalk runs independent systems as separate MPI groups, ooqmc.cpp:69-84.) */
typedef struct qwg_batch qwg_batch;
int qwg_batch_create(qwg_ctx* const* ctxs, int n, qwg_batch** out);
int qwg_batch_block(qwg_batch* b, qwg_block_stats* stats);
int qwg_batch_destroy(qwg_batch* b);

/* Launch-shape autotuner: times the full evaluation of the resident walkers
 * for each walkers-per-CTA choice that fits shared memory and keeps the
 * fastest (call before qwg_dmc_init).  Returns the chosen value. */
int qwg_autotune(qwg_ctx* ctx, int* walkers_per_cta);

/* QWalk log files (runid.log), host only.  qwg_log_header appends the run
 * banner of Dmc_method::run / Vmc_method::run (method/Dmc_method.cpp:307-317,
 * method/Vmc_method.cpp:333-340) and the "init" entry of
 * Properties_manager::initializeLog (properties/Properties.cpp:1022-1036);
 * qwg_log_block appends one "block { ... }" entry with the fields and
 * precision of Properties_manager::endBlock + Properties_block::storeToLog
 * (properties/Properties.cpp:628-636, properties/Properties_block.cpp:73-136),
 * so the reference's gosling analyser reads and reblocks engine runs.
 * method: "DMC" or "VMC"; label: the block label (e.g. "dmc"); nconfig and
 * nstep appear in the VMC banner only. */
int qwg_log_header(const char* path, const char* method, const char* label, double timestep, int nconfig,
                   int nstep);
int qwg_log_block(const char* path, const char* label, const qwg_block_stats* stats);

/* Walker configuration files (STORECONFIG / READCONFIG), host only, in the
 * text layout of write_configurations / read_configurations
 * (program_utils/qmc_io.h:371-470) with Config_save_point positions
 * (system/Sample_point.cpp:120-148) and, for DMC, the Dmc_point weight and
 * sign section (method/Dmc_method.cpp:1228-1267).  qwg_write_configs renames
 * an existing file to <path>.backup first, as the reference does; weight NULL
 * writes VMC walkers (positions only), sign NULL writes sign 1.
 * qwg_read_configs fills up to maxw walkers (weight and sign 1 where a walker
 * has no DMC section) and fails with QWG_ERR_INPUT on a malformed file or an
 * electron count other than nelec.  qwg_store_configs writes the context's
 * resident walkers (with weights and signs if dmc != 0). */
int qwg_write_configs(const char* path, const double* R, const double* weight, const double* sign, int nw,
                      int nelec);
int qwg_count_configs(const char* path, int* nw, int* nelec);
int qwg_read_configs(const char* path, double* R, double* weight, double* sign, int maxw, int nelec, int* nw_read);
int qwg_store_configs(qwg_ctx* ctx, const char* path, int dmc);

/* T-move selection without moving (Pseudopotential::calcNonlocTmove +
 * the selection of Dmc_method::doTmove, system/Pseudopotential.cpp:371-389,
 * method/Dmc_method.cpp:850-906) for the resident walkers, with the
 * deterministic pseudopotential and the quadrature rotations rot ([nw][3][3]
 * or NULL): mode 1 or 2 as qwg_dmc_params.tmoves, tau the time step.  For
 * electron e of walker w, moved[w][e] = 1 and pos[w][e][0..2] its target when
 * a move is selected, else moved = 0. */
int qwg_tmove_select(qwg_ctx* ctx, const double* rot, int mode, double tau, uint64_t seed, int* moved,
                     double* pos);

/* Kernel timing for rooflines: runs nstep DMC steps of the resident
 * population as individual launches of the move kernel and the local-energy
 * kernel (no branching; the walk and the weights advance) with CUDA events
 * around each launch, and returns the mean duration of each in ms.  Requires
 * qwg_dmc_init and no block in flight. */
int qwg_time_kernels(qwg_ctx* ctx, int nstep, double* sweep_ms, double* eloc_ms);

/* Number of kernel launches the context issued since the last reset. */
long long qwg_launch_count(const qwg_ctx* ctx);
void qwg_reset_launch_count(qwg_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif
