/*
 * gpufoam_b200 — C ABI of the B200 (sm_100a) per-cell detailed-chemistry solver.
 *
 * This is the drop-in seam for the OpenFOAM `gpuChemistryModel` plugin of gpuFoam.
 * The plugin keeps its OpenFOAM side (dictionary loaders, field gather/scatter,
 * `solve(deltaT)` contract); everything below `FoamGpu::GpuKernelEvaluator` is
 * replaced by the entry points declared here.
 *
 * Conventions
 *   - Plain C types, pointers and sizes only. Every function returns an int
 *     status (GF_OK == 0); no exception ever crosses this boundary.
 *   - All arithmetic is IEEE FP64 (the reference's gScalar = double,
 *     gpu_utils/common/gpu_constants.H:8); indices are int (gLabel).
 *   - nEqns = nSpecie + 2; a cell state is [Y_0 .. Y_{nS-1}, T, p], cell-major
 *     (the reference's Yvf layout, gpuChemistryModel.C:33-53).
 *   - `stream` arguments are cudaStream_t passed as void* (0 = legacy default).
 *
 * Reference interfaces replaced (paths relative to the gpuFoam repository):
 *   gf_thermo_from_nasa      makeGpuThermo            gpu_chemistry/src/gpuThermo/makeGpuThermo.H:16-48
 *   gf_reaction_thermo       set_reaction_thermo      gpu_chemistry/src/gpuReaction/makeGpuReactions.H:18-59
 *   gf_mech_create           thermosAndReactions ctor gpu_chemistry/src/gpuKernelEvaluator/gpuKernelEvaluator/thermosAndReactions.cu:10-24
 *   gf_solver_create         GpuKernelEvaluator ctor  gpu_chemistry/src/gpuKernelEvaluator/gpuKernelEvaluator/gpuKernelEvaluator.cu:14-33
 *                            + make_gpuODESolver      gpu_chemistry/src/gpuOde/makeGpuOdeSolver.H:13-31
 *   gf_compute_rr            GpuKernelEvaluator::computeRR   gpuKernelEvaluator.cu:65-97
 *   gf_compute_ynew          GpuKernelEvaluator::computeYNew gpuKernelEvaluator.cu:35-63
 *   gf_solve                 computeYNew + computeRR on device memory (same contract, no host staging)
 *   gf_rates                 gpuODESystem::derivatives      gpu_chemistry/src/gpuOde/gpuODESystem.H:164-196
 *   gf_jacobian              gpuODESystem::jacobian         gpu_chemistry/src/gpuOde/gpuODESystem.H:198-281
 *   gf_lu_decompose          LUDecompose                    gpu_chemistry/src/gpuOde/ludecompose.H:9-92
 *   gf_lu_backsubstitute     LUBacksubstitute               gpu_chemistry/src/gpuOde/ludecompose.H:94-130
 *   gf_lu_factor_solve       LUDecompose + LUBacksubstitute ludecompose.H:9-130 (the solve kernels' forms)
 */
#ifndef GPUFOAM_B200_H
#define GPUFOAM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define GF_ABI_VERSION 1

/* Longest side of a reaction (reference MAX_REACTION_WIDTH, gpuReaction.H:12). */
#define GF_MAX_REACTION_WIDTH 10
/* Largest mechanism the kernels accept (nSpecie). The reference's third-body
 * efficiency arrays hold 300 species (gpuThirdBodyEfficiencies.H:10). */
#define GF_MAX_SPECIES 300

/* ---- status codes ------------------------------------------------------ */
enum gf_status {
    GF_OK = 0,
    GF_ERR_INVALID_ARGUMENT = 1,  /* null pointer, negative size, bad enum      */
    GF_ERR_UNKNOWN_SOLVER = 2,    /* ode name not Rosenbrock12/23/34
                                     (reference throws logic_error, makeGpuOdeSolver.H:28) */
    GF_ERR_UNSUPPORTED = 3,       /* mechanism outside the kernels' limits        */
    GF_ERR_MASS_IMBALANCE = 4,    /* |lhs - rhs| > 0.1 kg/kmol (makeGpuReactions.H:48-54) */
    GF_ERR_CUDA = 5,              /* a CUDA runtime call failed                   */
    GF_ERR_NO_DEVICE = 6,         /* no CUDA device visible                       */
    GF_ERR_OUT_OF_MEMORY = 7,
    GF_ERR_CELL_FAILURE = 8       /* at least one cell ended with a non-OK cell status */
};

/* Per-cell integration status (written to the optional `status` array). The
 * reference traps on step underflow (gpuAdaptiveSolver.H:111-114) and returns
 * silently on maxSteps (gpuODESolverBase.H:80-111); here both are reported. */
enum gf_cell_status {
    GF_CELL_OK = 0,
    GF_CELL_STEP_UNDERFLOW = 1,   /* dx < vSmall during step rejection           */
    GF_CELL_MAX_STEPS = 2,        /* maxSteps substeps taken before reaching deltaT */
    GF_CELL_NONFINITE = 3,        /* NaN/Inf in the integrated state             */
    GF_CELL_SKIPPED = 4,          /* T <= Treact: chemistry not solved (not an error) */
    GF_CELL_BAD_MECHANISM = 5     /* mech_id outside the solver's mechanisms: not integrated */
};

/* Reaction-rate kinds (gpuReactionRate variant, gpuReactionRate.H:16-28). */
enum gf_rate_type {
    GF_RATE_ARRHENIUS = 0,             /* gpuArrheniusReactionRate              */
    GF_RATE_THIRD_BODY_ARRHENIUS = 1,  /* gpuThirdBodyArrheniusReactionRate     */
    GF_RATE_LINDEMANN_FALLOFF = 2,     /* gpuFallOffReactionRate<Arrhenius, Lindemann> */
    GF_RATE_TROE_FALLOFF = 3           /* gpuFallOffReactionRate<Arrhenius, Troe>      */
};

enum gf_ode_kind { GF_ROSENBROCK12 = 12, GF_ROSENBROCK23 = 23, GF_ROSENBROCK34 = 34 };

/* ---- mechanism description ---------------------------------------------- */

/* One gpuThermo (gpuThermo.H:9-62): perfect gas (Y, W) + JANAF/NASA-7 with
 * coefficients ALREADY multiplied by R = RR/W, as makeGpuThermo produces. */
typedef struct gf_thermo {
    double Y;
    double W;
    double Tlow, Thigh, Tcommon;
    double high[7];
    double low[7];
} gf_thermo;

/* gpuSpecieCoeffs (gpuReaction.H:25-37). `integer_exponent` != 0 selects the
 * integerPow path with exponent (int)exponent (gpuSpecieExponent.H:103-110). */
typedef struct gf_specie_coeff {
    int index;
    int integer_exponent;
    double stoich;
    double exponent;
} gf_specie_coeff;

/* One gpuReaction (gpuReaction.H:43-98). `thermo` is the reaction ΔThermo
 * (the gpuThermo base of gpuReaction, set by set_reaction_thermo). */
typedef struct gf_reaction {
    gf_thermo thermo;
    int n_lhs, n_rhs;
    gf_specie_coeff lhs[GF_MAX_REACTION_WIDTH];
    gf_specie_coeff rhs[GF_MAX_REACTION_WIDTH];
    int rate_type;           /* enum gf_rate_type                                */
    int irreversible;
    /* Arrhenius, third-body Arrhenius, or the k0 of a fall-off rate */
    double A, beta, Ta;
    /* kInf of a fall-off rate (ignored otherwise) */
    double Ainf, betainf, Tainf;
    /* Troe F (gpuTroeFallOffFunction.H:10-25): alpha, T***, T*, T** */
    double troe_alpha, troe_Tsss, troe_Ts, troe_Tss;
    /* third-body efficiencies, nSpecie values; NULL for plain Arrhenius */
    const double* efficiencies;
    /* temperature limits of the rate (gpuReaction::Tlow/Thigh) */
    double Tlow, Thigh;
} gf_reaction;

typedef struct gf_mech_desc {
    int n_species;
    int n_reactions;
    const gf_thermo* thermos;       /* n_species   */
    const gf_reaction* reactions;   /* n_reactions */
} gf_mech_desc;

/* gpuODESolverInputs (gpuODESolverInputs.H:9-23) with the solver name as an enum. */
typedef struct gf_ode_inputs {
    int solver;              /* enum gf_ode_kind */
    double absTol, relTol;
    int maxSteps;
    double safeScale, alphaInc, alphaDec, minScale, maxScale;
} gf_ode_inputs;

/* Kernel launch form. kind: 0 = plain (one thread per cell, one launch over all
 * cells, the reference's launch model); 1 = persistent work queue. */
typedef struct gf_launch_config {
    int kind;
    int threads_per_cell;    /* persistent only: 1, 2, 4, 8, 16, 32 (groups inside a
                                warp) or 64, 96, 128, 256 (one cell per CTA)     */
    int scratch_in_shared;   /* 1: per-cell workspace in shared memory           */
    int cells_per_block;     /* groups per CTA (persistent, threads_per_cell <= 32;
                                CTAs have at most 128 threads)                   */
    int blocks_per_sm;       /* 0 = as many as fit                               */
    int register_budget;     /* persistent only: 0 = up to 255 registers per thread,
                                1 = at most 128 (more resident cell groups)      */
    int lu_panel;            /* persistent, 32/64/96/128 threads per cell: columns per LU
                                panel, 4, 8 or 16 (0 = 8; see gf_solver_set_launch) */
    int specialize;          /* persistent, 32/64/96/128 threads per cell: 1 = the kernel
                                compiled for the matrix size of the solver's
                                mechanisms (10, 53 or 100 species; all the same)  */
} gf_launch_config;

typedef struct gf_stats {
    long long accepted_steps;   /* summed over cells */
    long long attempts;         /* accepted + rejected Rosenbrock attempts       */
    long long failed_cells;     /* cells with a status other than OK/SKIPPED     */
    double min_delta_t;         /* min over cells of deltaTChemNew before clamping */
} gf_stats;

typedef struct gf_mech gf_mech;
typedef struct gf_solver gf_solver;

/* ---- host helpers: the reference's mechanism loader arithmetic ---------- */

/* makeGpuThermo (makeGpuThermo.H:16-48): coefficients × R where R = RR/W. */
int gf_thermo_from_nasa(double Y, double W, double Tlow, double Thigh, double Tcommon,
                        const double high_raw[7], const double low_raw[7], gf_thermo* out);

/* set_reaction_thermo (makeGpuReactions.H:18-59): the reaction ΔThermo from the
 * species thermos, with the same operator sequence (gpuThermo.H:352-470,
 * gpuPerfectGas.H:100-117,280-325). Returns GF_ERR_MASS_IMBALANCE when the
 * reference would raise its FatalError. */
int gf_reaction_thermo(const gf_thermo* species, int n_species,
                       int n_lhs, const gf_specie_coeff* lhs,
                       int n_rhs, const gf_specie_coeff* rhs, gf_thermo* out);

/* ---- mechanism / solver objects ----------------------------------------- */

/* Copies the description into device tables on the current device. */
int gf_mech_create(const gf_mech_desc* desc, gf_mech** out);
void gf_mech_destroy(gf_mech* mech);
int gf_mech_info(const gf_mech* mech, int* n_species, int* n_reactions, long long* device_bytes);

/* One or more mechanisms (mixed batches address them by a per-cell id). */
int gf_solver_create(const gf_mech* const* mechs, int n_mechs, const gf_ode_inputs* inputs,
                     double Treact, gf_solver** out);
void gf_solver_destroy(gf_solver* solver);
/* GF_ERR_UNSUPPORTED for a form the library does not compile: lu_panel 4/16 or
 * specialize need 32, 64 or 128 threads per cell with register_budget 1 for
 * 128 threads and 0 otherwise; without specialize, lu_panel 4/16 needs
 * scratch_in_shared; specialize needs a solver whose mechanisms share 10, 53 or
 * 100 species, with lu_panel 8 (or 0), or 4 for 53 species. */
int gf_solver_set_launch(gf_solver* solver, const gf_launch_config* cfg);
int gf_solver_get_launch(const gf_solver* solver, gf_launch_config* cfg);
/* The per-cell workspace of the solve kernels (doubles: in shared memory or
 * HBM, by the launch form), the widest state row (nEqns) and the number of
 * mechanisms; any output may be NULL. */
int gf_solver_info(const gf_solver* solver, int* ws_doubles_per_cell, int* max_neq, int* n_mechs);

/* ---- the per-flow-step solve --------------------------------------------- */

/* Device-memory form of computeYNew + computeRR. All pointers are device pointers.
 *   n_cells
 *   deltaT         flow time step (used when deltaT_cell is NULL)
 *   deltaT_cell    per-cell time step [n_cells] or NULL (local time stepping)
 *   deltaTChemMax  clamp for the returned chemistry time steps
 *   mech_id        per-cell mechanism index [n_cells] or NULL (all mechanism 0); a cell whose
 *                  id is outside 0 .. n_mechs-1 is not integrated (GF_CELL_BAD_MECHANISM):
 *                  its Ynew row is a copy of its Y0 row, its RR row zero, its counters
 *                  zero, its deltaTChem unchanged, and it counts as a failed cell
 *   rho            old-time density [n_cells] (may be NULL when RR is NULL)
 *   Y0             input states [n_cells][nEqns of the cell's mechanism], row stride ld_y
 *   Ynew           output states, same layout (may alias Y0, may be NULL)
 *   deltaTChem     in: chemistry time steps; out: new, clamped ≤ deltaTChemMax
 *   RR             output rho*(Ynew-Y0)/deltaT [n_cells][ld_rr] or NULL
 *   status         per-cell gf_cell_status [n_cells] or NULL
 *   counters       per-cell accepted/attempt counts [n_cells][2] (int) or NULL
 *   stats          host struct filled after the solve, or NULL (no host sync)
 */
int gf_solve(gf_solver* solver, int n_cells, double deltaT, const double* deltaT_cell,
             double deltaTChemMax, const int* mech_id, const double* rho,
             const double* Y0, int ld_y, double* Ynew, double* deltaTChem,
             double* RR, int ld_rr, int* status, int* counters, gf_stats* stats,
             void* stream);

/* ---- graph-captured solve (no counterpart in the reference) ------------- */

typedef struct gf_solve_graph gf_solve_graph;

/* Captures one gf_solve with these arguments (device pointers; no stats) into
 * an executable CUDA graph: the work-queue reset, the solve kernel and a copy of
 * the step totals to pinned host memory. The graph owns its workspaces and
 * queue, so later calls on the solver leave it valid; the solver's launch form
 * is the one set at capture. Every launch reads and writes the arrays given
 * here: the caller refills Y0 and deltaTChem in place between launches. The
 * solver and its mechanisms must outlive the graph. Nothing runs at capture. */
int gf_solve_graph_create(gf_solver* solver, int n_cells, double deltaT, const double* deltaT_cell,
                          double deltaTChemMax, const int* mech_id, const double* rho,
                          const double* Y0, int ld_y, double* Ynew, double* deltaTChem,
                          double* RR, int ld_rr, int* status, int* counters, gf_solve_graph** out);
/* New flow time step for later launches (the kernel node is updated in place). */
int gf_solve_graph_set_delta_t(gf_solve_graph* graph, double deltaT);
/* Enqueues one solve on stream. */
int gf_solve_graph_launch(gf_solve_graph* graph, void* stream);
/* Step totals of the last launch; valid once its stream has synchronized. */
int gf_solve_graph_stats(const gf_solve_graph* graph, gf_stats* stats);
void gf_solve_graph_destroy(gf_solve_graph* graph);

/* Host-memory mirror of GpuKernelEvaluator::computeRR (single mechanism):
 * RR [n_cells][nSpecie], deltaTChemNew [n_cells] (clamped), *minDeltaT (before
 * clamping). The host arrays are copied to and from device staging buffers
 * that the solver allocates on first use (cudaMalloc) and keeps; the copies
 * run at pageable-memory speed unless the caller's arrays are pinned. */
int gf_compute_rr(gf_solver* solver, int n_cells, double deltaT, double deltaTChemMax,
                  const double* rho, const double* deltaTChem, const double* Y,
                  double* RR, double* deltaTChemNew, double* minDeltaT);

/* gf_compute_rr with a flow time step per cell, deltaT [n_cells] (host): the
 * local time stepping that gpuChemistryModel::solve(const scalarField& deltaT)
 * rejects in the reference (gpuChemistryModel.C:328-333). RR uses each cell's
 * own deltaT. */
int gf_compute_rr_lts(gf_solver* solver, int n_cells, const double* deltaT, double deltaTChemMax,
                      const double* rho, const double* deltaTChem, const double* Y,
                      double* RR, double* deltaTChemNew, double* minDeltaT);

/* Host-memory mirror of GpuKernelEvaluator::computeYNew: Ynew [n_cells][nEqns]
 * and deltaTChemNew [n_cells] (not clamped, as in the reference). */
int gf_compute_ynew(gf_solver* solver, int n_cells, double deltaT, double deltaTChemMax,
                    const double* deltaTChem, const double* Y, double* Ynew,
                    double* deltaTChemNew);

/* ---- the plugin's field gather and rate scatter ---------------------------
 * The plugin packs OpenFOAM's per-species fields into cell-major states on the
 * host (getY0, gpu_chemistry/src/gpuChemistryModels/gpuChemistryModel/
 * gpuChemistryModel.C:33-53) and unpacks the cell-major rates into per-species
 * fields after the solve (computeRRAndChemDeltaT, gpuChemistryModel.C:351-356).
 * With the fields in device memory both run on the GPU. Y_fields and RR_fields
 * are host arrays of n_species device pointers (one field of n_cells values
 * each); 1 <= n_species <= GF_MAX_SPECIES.
 *   gf_gather_states   y[c][i] = Y_fields[i][c], y[c][nS] = T[c], y[c][nS+1] = p[c]
 *                      (row stride ld_y >= n_species + 2)
 *   gf_scatter_rates   RR_fields[i][c] = RR[c][i] (row stride ld_rr >= n_species) */
int gf_gather_states(int n_cells, int n_species, const double* const* Y_fields, const double* T,
                     const double* p, double* y, int ld_y, void* stream);
int gf_scatter_rates(int n_cells, int n_species, const double* RR, int ld_rr, double* const* RR_fields,
                     void* stream);

/* ---- the plugin's per-cell side paths ------------------------------------
 * gpuChemistryModel computes these on the CPU through OpenFOAM's reactions
 * (gpu_chemistry/src/gpuChemistryModels/gpuChemistryModel/gpuChemistryModel.C);
 * here they run on the GPU with the solve's rate code. Concentrations are
 * c_i = rho Y_i / W_i with the thermo's density rho [n_cells] (:163-166);
 * y [n_cells][ld_y] = (Y, T, p); device pointers. */

/*   gf_cell_rates       calculate()   gpuChemistryModel.C:145-186  RR [n][ld_rr] = W_i dN_i/dt / V
 *                       tc()          gpuChemistryModel.C:366-427  tc [n], the chemical time scale
 * Either output may be NULL. GF_ERR_UNSUPPORTED if one cell's rate data
 * (about (2 nS + n_third_body + 4 nR) doubles) exceeds the shared memory of a CTA. */
int gf_cell_rates(const gf_mech* mech, int n_cells, const double* rho, const double* y, int ld_y,
                  double* RR, int ld_rr, double* tc, void* stream);

/*   gf_reaction_rates   reactionRR(r)        gpuChemistryModel.C:188-229  omega [n] of reaction r
 *                       specieReactionRR(r)  gpuChemistryModel.C:231-298  RR [n][ld_rr] of reaction r alone
 * reaction in mechanism order; either output may be NULL. */
int gf_reaction_rates(const gf_mech* mech, int n_cells, int reaction, const double* rho, const double* y,
                      int ld_y, double* omega, double* RR, int ld_rr, void* stream);

/*   gf_qdot             Qdot()        gpuChemistryModel.C:429-450  qdot [n] = -sum_i hf_i RR[c][i]
 * from species mass rates RR (of gf_solve, gf_compute_rr or gf_cell_rates),
 * hf_i the enthalpy of formation (gpuThermo::Hf); summed in species order. */
int gf_qdot(const gf_mech* mech, int n_cells, const double* RR, int ld_rr, double* qdot, void* stream);

/* ---- differentiation (no counterpart in the reference) ------------------ */

/* gf_solve (single mechanism, one flow step deltaT, no RR) that also records
 * the trajectory for gf_adjoint: for accepted step k of cell c,
 * traj[(c * traj_cap + k) * (nS + 2) + 0 .. nS] = the state (Y, T) at the step's
 * start and [nS + 1] = its size. status and counters [n][2] (accepted,
 * attempts) are required. A cell with more than traj_cap accepted steps stops
 * with status GF_CELL_MAX_STEPS. Device pointers. */
int gf_solve_record(gf_solver* solver, int n_cells, double deltaT, const double* Y0, int ld_y,
                    double* Ynew, double* deltaTChem, int* status, int* counters,
                    double* traj, int traj_cap, void* stream);

/* Discrete adjoint of the recorded integration (step sequence frozen): given
 * the loss gradient Ybar w.r.t. the final states Ynew, writes the gradient
 * w.r.t. the initial states Y0 (Y and T; p gets 0) and, per cell,
 * theta_bar[c][3 r + 0..2] = dL/d ln|A|, dL/d beta, dL/d Ta of reaction r
 * (mechanism order; the k rate, k0 for fall-off reactions; Ta = Ea / R).
 * traj, counters and fwd_status come from gf_solve_record with the same
 * solver; status gets 0 per cell, or the recording's failure status (the
 * cell's gradient is then 0). GF_ERR_UNSUPPORTED for reactions with more
 * than 4 species on a side. Device pointers. */
int gf_adjoint(gf_solver* solver, int n_cells, const double* traj, int traj_cap,
               const int* counters, const int* fwd_status, const double* Y0, const double* Ynew,
               const double* Ybar, int ld_y, double* Y0bar, double* theta_bar, int* status,
               void* stream);

/* Size of the static device scratch of gf_solve_noalloc (32 MiB per GPU). */
#define GF_NOALLOC_SCRATCH_BYTES (32ll * 1024 * 1024)

/* gf_solve without any device allocation — no counterpart in the reference.
 * For callers that cannot call cudaMalloc: a host code whose device memory
 * belongs to another allocator (a caching pool that has reserved the free
 * memory, or a host application that requires every allocation to go through
 * its own memory manager), or a real-time loop that forbids allocation once it
 * has started. The mechanism (gf_mech_create, on the current device) is
 * set-up-time input; inputs and outputs are the caller's device arrays, as in
 * gf_solve. The per-cell workspaces and work-queue counters live in a static
 * device array of GF_NOALLOC_SCRATCH_BYTES that every GPU loading the library
 * holds until exit; the number of cells integrated at once is capped so their
 * workspaces fit (GF_ERR_UNSUPPORTED if not even one cell's does). The first
 * call on each device resolves the array's address (cudaGetSymbolAddress) and
 * should come before any stream capture. All calls share the array: calls
 * whose kernels overlap on one GPU race and must not be issued. With stats !=
 * NULL the call copies the step totals to the host and waits for the stream;
 * it returns GF_ERR_INVALID_ARGUMENT for a stream that is being captured. */
int gf_solve_noalloc(const gf_mech* mech, const gf_ode_inputs* inputs, double Treact, int n_cells, double deltaT,
                     const double* deltaT_cell, double deltaTChemMax, const double* rho, const double* Y0, int ld_y,
                     double* Ynew, double* deltaTChem, double* RR, int ld_rr, int* status, int* counters,
                     gf_stats* stats, void* stream);

/* ---- parity entry points (one thread group per state, device pointers) --- */

/* dydx [n_states][nEqns] = derivatives(y [n_states][nEqns]). */
int gf_rates(const gf_mech* mech, int n_states, const double* y, double* dydx, void* stream);

/* dfdx [n_states][nEqns] and J [n_states][nEqns][nEqns] = jacobian(y). */
int gf_jacobian(const gf_mech* mech, int n_states, const double* y, double* dfdx,
                double* J, void* stream);

/* In-place LU of n_mats matrices [n_mats][m][m] with pivots [n_mats][m]. */
int gf_lu_decompose(int n_mats, int m, double* A, int* pivots, void* stream);
/* In-place solve of b [n_mats][m] with the factors from gf_lu_decompose. */
int gf_lu_backsubstitute(int n_mats, int m, const double* LU, const int* pivots,
                         double* b, void* stream);

/* LUDecompose + LUBacksubstitute (ludecompose.H:9-130) as the solve kernels
 * run them, with threads_per_matrix (1, 4, 8, 16, 32, 64, 96, 128 or 256) threads
 * per matrix: after the implicit row scaling, the register-panel factorisation
 * for 32 or more threads and m <= 64, the blocked one otherwise; solves by
 * reciprocal pivots for 16 or more threads. exact != 0 rounds every
 * elimination update a - l u twice (no FMA contraction), as the reference's
 * CPU build computes its Crout sums, so the factors can be compared bit for
 * bit. A [n_mats][m][m] (in place: the factors), pivots [n_mats][m],
 * b [n_mats][n_rhs][m] (in place: the solutions); m <= 160; device pointers. */
int gf_lu_factor_solve(int n_mats, int m, double* A, int* pivots, double* b, int n_rhs,
                       int threads_per_matrix, int exact, void* stream);

/* ---- measurement (no reference counterpart) -------------------------------- */

/* FP64 FMA throughput of the current device, measured with independent DFMA
 * chains for about `ms` milliseconds: the roofline denominator of the kernels
 * above, which run on the FP64 CUDA-core pipe. */
int gf_measure_fp64_peak(double ms, double* tflops);

/* ---- misc --------------------------------------------------------------- */
const char* gf_strerror(int status);
int gf_abi_version(void);
/* CUDA error text of the last GF_ERR_CUDA on this thread. */
const char* gf_last_cuda_error(void);

#ifdef __cplusplus
}
#endif
#endif /* GPUFOAM_B200_H */
