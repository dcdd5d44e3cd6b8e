/*
 * axisim_b200.h -- C ABI of the B200-native SIMPLE pressure-velocity solver.
 *
 * A drop-in for AxiSim's solver path (Luippe/AxiSim-Software): the structs below
 * are plain-old-data mirrors of the reference's case, mesh and boundary types,
 * and the verbs mirror Solver's solve / continue / stop entry points. Every entry
 * point takes plain pointers and sizes, returns an int status (never aborts),
 * and leaves a message for axisim_last_error().
 *
 * Reference interface each declaration replaces is cited beside it
 * (path:line inside the reference project).
 */
#ifndef AXISIM_B200_H
#define AXISIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AXISIM_ABI_VERSION 1

/* ---- status codes (the reference aborts in CUDA_CHECK, gpu_utils.h:5-11) ---- */
enum axisim_status {
    AXISIM_OK = 0,
    AXISIM_E_ARG = 1,       /* null pointer, bad size, unknown name */
    AXISIM_E_CONFIG = 2,    /* Solver::runCheck rejections (solver.cpp:530-661) */
    AXISIM_E_MESH = 3,      /* inconsistent packed mesh */
    AXISIM_E_CUDA = 4,      /* CUDA runtime error or no usable device */
    AXISIM_E_DIVERGED = 5,  /* NaN/Inf residual */
    AXISIM_E_STOPPED = 6,   /* axisim_request_stop() ended the run */
    AXISIM_E_STATE = 7,     /* verb called in the wrong state (e.g. solve before set_mesh) */
    AXISIM_E_TIMEOUT = 8    /* a device wait ran out of its iteration budget */
};

/* ---- enums: same numbering as the reference's uint8_t enums ---- */
/* BCType (structs/boundary_struct.h:90-99) */
enum { AXISIM_BC_DIRICHLET = 0, AXISIM_BC_NEUMANN = 1, AXISIM_BC_FULLY_DEVELOPED = 2,
       AXISIM_BC_MICHAELIS_MENTEN = 3, AXISIM_BC_HILL = 4, AXISIM_BC_NONE = 5, AXISIM_BC_PULSATILE = 6 };
/* BoundaryType (structs/boundary_struct.h:342-348) */
enum { AXISIM_WALL = 0, AXISIM_VELOCITY_INLET = 1, AXISIM_PRESSURE_OUTLET = 2, AXISIM_SYMMETRY = 3,
       AXISIM_FAR_FIELD = 4 };
/* BoundaryVariable (structs/boundary_struct.h:44-53): StaticTemperature and
 * Concentration are the transported scalars */
enum { AXISIM_VAR_U = 0, AXISIM_VAR_V = 1, AXISIM_VAR_P = 2, AXISIM_VAR_T = 3, AXISIM_VAR_C = 4 };
/* MeshType (structs/boundary_struct.h:382-385) */
enum { AXISIM_MESH_STRUCTURED = 0, AXISIM_MESH_UNSTRUCTURED = 1 };
/* Precision of the pressure-correction multigrid (new; no reference counterpart) */
enum { AXISIM_PREC_FP64 = 0, AXISIM_PREC_MIXED = 1 };
/* Method of the pressure-correction solve (new; no reference counterpart) */
enum { AXISIM_PSOLVE_VCYCLES = 0, AXISIM_PSOLVE_FCG = 1 };

/* Mirror of FVMeshHostPacked (structs/solver_struct.h:400-429). */
typedef struct axisim_mesh_packed {
    int32_t nCells;
    int32_t nFaces;
    const int32_t* faceOwner;
    const int32_t* faceNeighbor;          /* -1 on a boundary face */
    const double* faceNormalZ;            /* unit, owner -> neighbour / outward */
    const double* faceNormalR;
    const double* faceCenterZ;
    const double* faceCenterR;
    const double* faceArea;               /* revolved area 2 pi r_f L */
    const int32_t* faceBoundaryGroupID;   /* -1 = unassigned */
    const double* cellCenterZ;
    const double* cellCenterR;
    const double* cellArea2D;
    const double* cellVolume;             /* revolved volume 2 pi r_c A */
    const int32_t* cellFaceStart;         /* nCells + 1 */
    const int32_t* cellFaceIDs;           /* cellFaceStart[nCells] */
} axisim_mesh_packed;

/* Mirror of BoundaryFieldHost (structs/solver_struct.h:464-476) for one
 * variable. lengthByGroup holds the group's float totalLength widened to
 * double (structs/boundary_struct.h:515). The three pulsatile arrays are new:
 * the reference re-derives them from BoundarySegmentGroup each time step
 * (solver.cpp:375-424); here a group flagged pulsatile is a Dirichlet value
 * valueByGroup * (1 + amplitude sin(2 pi frequency t)). Any may be NULL. */
typedef struct axisim_bc_field {
    int32_t nGroups;
    const uint8_t* typeByGroup;
    const uint8_t* boundaryTypeByGroup;
    const double* valueByGroup;
    const double* lengthByGroup;
    const uint8_t* pulsatileByGroup;
    const double* amplitudeByGroup;
    const double* frequencyByGroup;
} axisim_bc_field;

/* Mirror of ConfigSolver (structs/solver_struct.h:203-238), byte-compatible:
 * sizeof == 40 like the reference's static_assert. */
typedef struct axisim_config_solver {
    uint8_t velocitySolver;     /* 0 SIMPLE */
    uint8_t convectionScheme;   /* 0 UPWIND 1 CENTRAL 2 SECOND_ORDER_UPWIND 3 QUICK (-> upwind) */
    uint8_t gradientScheme;     /* 0 GREEN_GAUSS 1 LSQ */
    uint8_t type;               /* linear solver: 0 JACOBI 1 GS_RB (multicolour) */
    uint8_t timeScheme;         /* 0 first order 1 BDF2 */
    uint8_t pad_[3];
    int32_t linearMaxIter;
    uint8_t useMultigrid;
    uint8_t addConvectionTerm;
    uint8_t transient;
    uint8_t useNonOrthCorrector;
    double dt;
    double tEnd;
    int32_t saveKeyFrameIter;
    int32_t pad2_;
} axisim_config_solver;

/* Mirror of ConfigSimple (structs/solver_struct.h:158-165), sizeof == 24. */
typedef struct axisim_config_simple {
    int32_t maxIter;
    int32_t checkConv;
    double momTol;   /* carried, unread (as in the reference) */
    double ppTol;    /* carried, unread (as in the reference) */
} axisim_config_simple;

/* Mirror of ConfigMultigrid (structs/solver_struct.h:167-190). */
typedef struct axisim_config_multigrid {
    int32_t maxIter;
    double weight;
    int32_t linearSweep;
    int32_t linearPreSweep;
    int32_t linearPostSweep;
} axisim_config_multigrid;

/* ConfigResidual without its device pointers (structs/solver_struct.h:240-258). */
typedef struct axisim_config_residual {
    uint8_t type;        /* 0 SCALED 1 RAW 2 RMS (informational, as in the reference) */
    uint8_t normType;    /* 0 L1 1 L2 2 LINF */
    uint8_t scaleType;   /* 0 NONE 1 N 2 SQRT_N 3 DIAGONAL 4 CONTINUITY(unused) */
    uint8_t enabled;
    double tol;
} axisim_config_residual;

/* Mirror of FluidPropertyConfig (src/header/setting.cuh:60-71). */
typedef struct axisim_fluid {
    double rho;
    double mu;
    double cp;
    double k;
    double D;
} axisim_fluid;

/* Result of a solve (Console::addCompletionTime + residual line, solver.cpp:1266-1323). */
typedef struct axisim_result {
    int32_t iterations;        /* SIMPLE iterations executed in this call */
    int32_t totalIterations;   /* currentIteration after the call */
    int32_t converged;
    int32_t timeSteps;
    double residual[3];        /* last U, V, Continuity residual */
    double solveMs;            /* CUDA-event time of the time + SIMPLE loops */
} axisim_result;

typedef struct axisim_handle axisim_handle;

/* Per-iteration residual callback, replacing ResidualPlot::add / Console line
 * (solver.cpp:1267-1268). Called after each check with five values: U, V,
 * Continuity, Temperature, Concentration (the last two 0 unless monitored). */
typedef void (*axisim_residual_fn)(void* ctx, int32_t iteration, const double* residuals);
typedef void (*axisim_log_fn)(void* ctx, const char* line);

/* ---- lifetime ---- */
int axisim_abi_version(void);
/* Solver::Solver(Config&) (solver.cpp:104-114) on CUDA device 0. */
int axisim_create(const axisim_fluid* fluid, axisim_handle** out);
/* The same on a chosen CUDA device (one handle per GPU; the reference has a
 * single device and stream per Solver, solver.cpp:110). */
int axisim_create_on(int32_t device, const axisim_fluid* fluid, axisim_handle** out);
/* Solver::reset + free (solver.cpp:118-144); frees every device allocation. */
int axisim_destroy(axisim_handle* h);
const char* axisim_last_error(const axisim_handle* h);
int axisim_set_log(axisim_handle* h, axisim_log_fn log, axisim_residual_fn residual, void* ctx);

/* ---- case ---- */
/* Mesh::getFVMesh + createFVMeshDevice (solver.cpp:774-785, memory_manger.cpp:679-689):
 * copies the packed mesh to the device and precomputes the geometry on the GPU. */
int axisim_set_mesh(axisim_handle* h, const axisim_mesh_packed* mesh);
/* Mesh::currentMeshType of the handle's mesh (AXISIM_MESH_*), which
 * Solver::runCheck reads (solver.cpp:548-555): a solve on a STRUCTURED mesh
 * clears configSolver.useNonOrthCorrector (and it stays cleared), as the
 * reference does. axisim_set_mesh resets it to UNSTRUCTURED. */
int axisim_set_mesh_type(axisim_handle* h, int32_t meshType);
/* createBoundarySolverDevice (memory_manger.cpp:191-237) for one variable
 * (AXISIM_VAR_*). MICHAELIS_MENTEN and HILL are accepted for T and C only; a
 * PULSATILE T or C group is a Dirichlet value at its mean (only u and v are
 * updated per time step, solver.cpp:1038-1055). */
int axisim_set_bc(axisim_handle* h, int32_t variable, const axisim_bc_field* bc);
/* Wall kinetics of a scalar's MICHAELIS_MENTEN / HILL groups: the vmax, km,
 * n, m, k2, v2 and Rtot arrays of BoundaryFieldHost (solver_struct.h:469-475)
 * as createBoundaryFieldHost fills them (memory_manger.cpp:110-145): rate
 * J(c) = Vmax c / (Km + c) or Vmax c^n / (Km^n + c^n), times
 * 1 - V2 c^m / (K2^m + c^m) when V2 != 0, through the series wall
 * resistance Rtot. Any array may be NULL (defaults Vmax = Km = K2 = V2 =
 * Rtot = 0, n = m = 1); groups at or past nGroups take the defaults. */
typedef struct axisim_kinetics {
    int32_t nGroups;
    const double* vmaxByGroup;
    const double* kmByGroup;
    const double* nByGroup;
    const double* mByGroup;
    const double* k2ByGroup;
    const double* v2ByGroup;
    const double* RtotByGroup;
} axisim_kinetics;
/* variable is AXISIM_VAR_T or AXISIM_VAR_C; kin = NULL restores the defaults. */
int axisim_set_kinetics(axisim_handle* h, int32_t variable, const axisim_kinetics* kin);
/* SolverFieldOption (solver_struct.h:9-12) and the "Temperature" /
 * "Concentration" ConfigResidual entries (res2[0], res2[1]; NULL keeps them;
 * the reference creates both disabled, solver.cpp:88-100). A solved scalar is
 * assembled and solved after the velocity / pressure corrections of every
 * SIMPLE iteration (solver.cpp:1218-1238): energy with the diffusivity
 * k / (rho cp) and the momentum relaxation factor, concentration with D,
 * unrelaxed; both convect with mDot / rho. Both start from zero, like the
 * reference's fields. An enabled entry joins the convergence test. With BDF2
 * the scalar step reads the time levels as the reference does: through the
 * names tempOld / tempOld2 as they stood when the run started, which the
 * per-step shift keeps exchanging (solver.cpp:985-1009, 1066-1095). */
int axisim_set_scalars(axisim_handle* h, int32_t solveEnergy, int32_t solveConcentration,
                       const axisim_config_residual* res2);
/* Temperature and Concentration residuals of the last check (out2[2]). */
int axisim_scalar_residuals(const axisim_handle* h, double* out2);
/* Solver's public config members configSolver / configSimple / configMultigrid /
 * cfg / simple.{momentum,pressure}Relaxation (solver.h:83-133). res[3] = U, V,
 * Continuity. */
int axisim_set_config(axisim_handle* h, const axisim_config_solver* solver,
                      const axisim_config_simple* simple, const axisim_config_multigrid* mg,
                      const axisim_config_residual* res3, double alphaU, double alphaP);
int axisim_set_fluid(axisim_handle* h, const axisim_fluid* fluid);
/* New: precision of the pressure-correction solve (AXISIM_PREC_*). */
int axisim_set_precision(axisim_handle* h, int32_t mode);
/* New: method of the pressure-correction solve when configSolver.useMultigrid
 * is set (AXISIM_PSOLVE_*). VCYCLES is the reference's configMultigrid.maxIter
 * V-cycles (multigrid.cu:794-798); FCG runs up to configMultigrid.maxIter
 * iterations of flexible conjugate gradients in FP64 with one FP32 V-cycle as
 * the preconditioner of each, in either precision mode, stopping once
 * ||b - A p'||_2 <= relTol ||b||_2 (relTol = 0: always maxIter iterations).
 * prolongScale multiplies the coarse-level corrections inside that V-cycle
 * (1 = the reference's injection; > 1 over-corrects, which offsets the weak
 * coarse correction of piecewise-constant aggregation). */
int axisim_set_pressure_solver(axisim_handle* h, int32_t mode, double relTol, double prolongScale);
/* New: Krylov p' solves started and iterations completed since the handle's
 * mesh was set. */
int axisim_pressure_stats(axisim_handle* h, int64_t* solves, int64_t* iterations);
/* New (the reference launches every multigrid phase as its own kernel or
 * graph node, multigrid.cu:607-662): how the V-cycle below the finest level
 * runs. AXISIM_VCYCLE_PER_PHASE (the default): one launch per phase, chained
 * by programmatic dependent launch inside the captured graph.
 * AXISIM_VCYCLE_RESIDENT: one cooperative kernel, one CTA per SM, runs every
 * phase of the coarser levels in order with a grid-wide barrier between
 * phases (the same per-cell arithmetic, so the same results bit for bit; on a
 * B200 it measured slower than the launches it replaces); a barrier that
 * waits longer than a second ends the solve with AXISIM_E_TIMEOUT. */
#define AXISIM_VCYCLE_PER_PHASE 0
#define AXISIM_VCYCLE_RESIDENT 1
int axisim_set_vcycle_kernel(axisim_handle* h, int32_t mode);
/* New (the reference launches one kernel per Jacobi sweep of each momentum
 * component, linear_solver.cu:91-146): how many of the u/v momentum Jacobi
 * sweeps one launch runs (1..8, default 1). Above 1 the cells are cut into
 * tiles along a space-filling curve of their centres; a launch loads a
 * tile's coefficients once, keeps the iterate of the tile and its halo in
 * shared memory and repeats the sweep there, each sweep on a halo one layer
 * thinner, so the tile's own cells end with the values of that many
 * whole-mesh sweeps (the same arithmetic, so the same results bit for bit).
 * threads is the CTA size of those launches (256, 512 or 1024; 0 = 1024).
 * Meshes with more than four faces on a cell, and the Gauss-Seidel momentum
 * solver, always run one launch per sweep. On a B200 the tiled launches cut
 * the sweeps' DRAM bytes about threefold but measured no faster in a captured
 * iteration: one launch per sweep keeps the 874k-cell working set in L2
 * between sweeps, and the tile kernel waits on its loads (one CTA of 1024
 * threads per SM); FP32 sweeps on 2M cells and more gained 3-4 %, FP64 lost
 * 2-4 %, and the host builds the tiles in about 30 ms per million cells. */
int axisim_set_momentum_sweeps(axisim_handle* h, int32_t sweepsPerLaunch, int32_t threads);
/* New: the number of tiles the sweeps of the last captured solve ran on (0 =
 * one launch per sweep). */
int axisim_sweep_tiles(axisim_handle* h, int32_t* nTiles);
/* Test hook for the failure path above: on = 1 makes every grid-wide barrier
 * of the resident V-cycle expect one arrival that never comes, so its waits
 * run out (after one second), the solve returns AXISIM_E_TIMEOUT and the
 * handle stays usable (no continue; the next solve starts fresh). on = 0
 * restores normal barriers. */
int axisim_test_barrier_timeout(axisim_handle* h, int32_t on);
/* New (no reference counterpart; the reference launches every multigrid kernel
 * with fixed shapes): enable = 1 tunes, before the next solve captures its
 * graph, the threads per CTA (64, 128 or 256) of the smoothing, residual,
 * restriction and prolongation kernels of each multigrid level the V-cycle
 * launches kernels on (the levels solved inside the one-CTA tail are not
 * tuned), by timing that level's Jacobi sweep at each size on scratch inputs
 * and keeping 256 unless another size is more than 3 % faster. Results are
 * unchanged (every cell's arithmetic is the same at any shape). enable = 0
 * returns to 256. */
int axisim_set_autotune(axisim_handle* h, int32_t enable);
/* The tuned block size per level (0: not tuned, or a level solved inside the
 * one-CTA tail) and, with usPerCandidate, the measured sweep time in
 * microseconds per level and candidate (3 per level: 64, 128, 256 threads).
 * Returns the level count. */
int axisim_autotune_report(const axisim_handle* h, int32_t* blockPerLevel, double* usPerCandidate,
                           int32_t maxLevels);

/* ---- learned p' preconditioner (new; no reference counterpart) ----
 * A U-Net over the multigrid's agglomeration hierarchy maps a p' residual r to
 * a correction y. It is trained on (p' right-hand side, converged p') pairs
 * that the solver's own FCG + V-cycle solve produces, with the energy-norm
 * error left after the best scaling of y as the loss. In the first FCG
 * iteration of a p' solve the preconditioner becomes
 * z = a y + V(r - a A y), a = (y, r) / (y, A y): the network's step, scaled
 * for the least energy error, then a V-cycle on the residual it leaves. Each solve is scored
 * by its mean log reduction of the FP64 residual per Krylov iteration; with
 * FIRST_STEP the network is used while its running score is at least as good
 * as the plain V-cycle's, else the solve falls back to the V-cycle (every 16th
 * solve probes each method so both scores stay current); ALWAYS uses it on
 * every solve. */
enum { AXISIM_LEARNED_OFF = 0, AXISIM_LEARNED_FIRST_STEP = 1, AXISIM_LEARNED_ALWAYS = 2 };
/* Sample store of `capacity` samples (0 keeps the current store) and harvest
 * of one sample every `every` SIMPLE iterations (0 = off) during solves; a
 * harvested sample is the p' system of that iteration after its solve, so run
 * the FCG solver with a tight relTol while harvesting. */
int axisim_learned_harvest(axisim_handle* h, int32_t every, int32_t capacity);
int axisim_learned_sample_count(axisim_handle* h, int32_t* count);
/* Host arrays: right-hand side, target p' (A p' = b), A_C diagonal and
 * boundary deficit 1 - sum|A_F| / A_C (nCells floats each), and the
 * off-diagonals A_F in the mesh's slot order (cellFaceStart[nCells] floats, 0
 * on boundary slots). */
int axisim_learned_add_sample(axisim_handle* h, const float* b, const float* target, const float* acDiag,
                              const float* deficit, const float* afSlots);
/* Any output may be NULL; relResidual = ||b - A p'|| / ||b|| of the solve that
 * produced it (-1 when added by hand). */
int axisim_learned_get_sample(axisim_handle* h, int32_t index, float* b, float* target, float* acDiag,
                              float* deficit, float* afSlots, float* relResidual);
/* (Re)initialises the network for the handle's mesh (AXISIM_NET_*): weights
 * and activations in FP32, both in BF16, or BF16 weights with FP32
 * activations; products always accumulate in FP32. */
enum { AXISIM_NET_FP32 = 0, AXISIM_NET_BF16 = 1, AXISIM_NET_BF16_WEIGHTS = 2 };
int axisim_learned_init(axisim_handle* h, int32_t precision, uint64_t seed, int64_t* nParams);
/* Reads (set = 0) or writes (set = 1) the n FP32 master parameters. */
int axisim_learned_params(axisim_handle* h, float* params, int64_t n, int32_t set);
/* Loss 1 - (y.b)^2 / ((y.A y)(b.p')) of the network output y on stored
 * sample `sample` (the energy-norm error left after the best scaling of y,
 * which is what one Krylov step along y removes) and its gradient with respect
 * to the parameters; grad may be NULL. */
int axisim_learned_grad(axisim_handle* h, int32_t sample, float* loss, float* grad, int64_t n);
/* `steps` Adam steps (learning rate lr) on samples drawn from store entries
 * [first, first + count) (count <= 0: to the end) with a seeded generator;
 * lossOut[steps] (may be NULL) receives each step's loss. */
int axisim_learned_train(axisim_handle* h, int32_t steps, float lr, uint64_t seed, int32_t first, int32_t count,
                         float* lossOut);
/* The network's correction out[nCells] (its output times rms(r / A_C)) for a
 * residual r, A_C diagonal and boundary deficit (host arrays). */
int axisim_learned_predict(axisim_handle* h, const float* r, const float* acDiag, const float* deficit, float* out);
/* AXISIM_LEARNED_*; takes effect in the FCG pressure solver. */
int axisim_learned_enable(axisim_handle* h, int32_t mode);
/* Solves that used the network, solves that fell back to the V-cycle because
 * its score was better, and the two running scores (mean log residual
 * reduction per Krylov iteration; more negative is better). */
int axisim_learned_stats(axisim_handle* h, int64_t* applied, int64_t* fallbacks, double* scoreNet,
                         double* scoreVcycle);

/* ---- solve / continue / stop ---- */
/* Solver::run + runSimple (solver.cpp:146-173, 753-1396), synchronous on the
 * caller's thread. continueRun mirrors Solver::continueSolver: the device fields
 * are reused as the initial guess when axisim_can_continue() holds. */
int axisim_solve(axisim_handle* h, int32_t continueRun, axisim_result* result);
/* Solver::canContinue (solver.cpp:469-528). Returns 1 if a continue is possible,
 * 0 otherwise (reason written to `reason`), or a negative status. */
int axisim_can_continue(const axisim_handle* h, char* reason, size_t reasonLen);
/* Solver::requestStop (solver.cpp:175-184): thread-safe; the running solve stops
 * at the top of its next SIMPLE iteration with the fields consistent. */
int axisim_request_stop(axisim_handle* h);

/* ---- fields ---- */
/* Solver::solutions (solver.cpp:186-219) plus solver internals for checking:
 * "u" "v" "p" "pp" "mDot" "DU" "DV" "gradPZ" "gradPR" "gradUZ" "gradUR"
 * "gradVZ" "gradVR" "AC_u" "b_u" "AF_u" "invAC_u" (and _v, _pp; AF in the
 * reference's CSR slot order) "res_U" "res_V" "res_Continuity" "continuity"
 * (per-cell mass imbalance, Solver::getMassImbalance) and the geometry
 * "invDPN" "wP" "dPB" "length2D" "lsqWZ" "lsqWR" "invA2D" "lsqInvZZ"
 * "lsqInvZR" "lsqInvRR"; with a solved scalar "T" / "C", "gradTZ" "gradTR"
 * "gradCZ" "gradCR", "AC_T" "b_T" "AF_T" "invAC_T" (and _C), "TOld" "TOld2"
 * "COld" "COld2", "res_T" "res_C", and per face the wall concentration "cw"
 * and wall consumption "ocrWall" of reactive walls (mesh.faces.cw / ocrWall).
 * Returns the element count written, or -status. */
int64_t axisim_get_field(const axisim_handle* h, const char* name, double* out, size_t n);
/* Initial state for u v p mDot (and uOld vOld for a transient restart; T C
 * TOld COld TOld2 COld2 for a solved scalar). */
int64_t axisim_set_field(axisim_handle* h, const char* name, const double* in, size_t n);

/* ---- batches (new: the reference solves one case per Solver, solver.h:18-185) ---- */
/* Declares the packed mesh to be nCases independent problems occupying the
 * contiguous cell ranges [caseCellStart[c], caseCellStart[c+1]) (no face may
 * join two ranges; boundary group ids are per case). Every kernel and every
 * graph node then advances all cases at once; residuals are formed and
 * normalised per case and the solve ends when every case has converged.
 * nCases = 0 returns to a single problem. */
int axisim_set_batch(axisim_handle* h, int32_t nCases, const int32_t* caseCellStart);
/* Per case: the first SIMPLE iteration at which it met the tolerances (-1 if
 * not yet) and its last U, V, Continuity residuals (3 per case). */
int axisim_batch_status(const axisim_handle* h, int32_t* convergedAt, double* residuals, int32_t n);

/* ---- multigrid hierarchy (MultigridSolver::describeHierarchy, multigrid.cu:727-764) ---- */
int axisim_mg_levels(const axisim_handle* h, int32_t* cellsPerLevel, int32_t maxLevels);
/* fine->coarse maps of level `level` (GridLevel::cellToCoarse / fineSlotToCoarseSlot,
 * multigrid.cuh:29-68) and the coarse CSR; returns the coarse slot count. */
int64_t axisim_mg_level_maps(const axisim_handle* h, int32_t level, int32_t* cellToCoarse,
                             int32_t* fineSlotToCoarseSlot, int32_t* coarseFaceStart,
                             int32_t* coarseFaceNeighbor);
/* MeshColoring (solver_struct.h:122-154): colour per cell; returns nColors. */
int axisim_coloring(const axisim_handle* h, int32_t* colorOut, size_t n);
/* The same hierarchy and colouring computed on the host from a packed mesh,
 * with no handle and no device (MultigridSolver::buildLevels,
 * multigrid.cu:298-325; buildMeshColoring, memory_manger.cpp:334-409): the
 * results of the three calls above for a handle holding that mesh. Each call
 * rebuilds what it reports. A mesh whose connectivity fails axisim_set_mesh's
 * checks gives -AXISIM_E_MESH. */
int axisim_mg_levels_host(const axisim_mesh_packed* mesh, int32_t* cellsPerLevel, int32_t maxLevels);
/* New: the hierarchy a batch solve uses (axisim_set_batch with these case
 * ranges): each case coarsened alone as MultigridSolver::buildLevels does for
 * a mesh of its own (multigrid.cu:298-325), merged level by level. Per level,
 * the cells of all cases and the cells of the cases whose coarsest level it is
 * (0 on the deepest level). Returns the number of levels or -status. */
int axisim_mg_batch_levels_host(const axisim_mesh_packed* mesh, int32_t nCases, const int32_t* caseCellStart,
                                int32_t* cellsPerLevel, int32_t* terminalCellsPerLevel, int32_t maxLevels);
int64_t axisim_mg_level_maps_host(const axisim_mesh_packed* mesh, int32_t level, int32_t* cellToCoarse,
                                  int32_t* fineSlotToCoarseSlot, int32_t* coarseFaceStart,
                                  int32_t* coarseFaceNeighbor);
int axisim_coloring_host(const axisim_mesh_packed* mesh, int32_t* colorOut, size_t n);
/* New: the tiles of several momentum sweeps per launch (see
 * axisim_set_momentum_sweeps) for a mesh of at most four faces per cell:
 * S halo layers, at most cap local cells a tile (< 65535), runs of tileCells
 * curve positions. Writes *nTiles and returns the total local cells (>= 0) or
 * -status; when every array is given and capacity >= that total, also fills
 * tileStart (nTiles + 1 offsets), layerEnd (S + 1 cumulative layer sizes per
 * tile), gid (mesh cell of each local cell) and lnb (slot j's local neighbour
 * in bits 16j..16j+15, 0xFFFF for none). nTiles = 0 when some cell with its
 * halo exceeds cap. */
int64_t axisim_sweep_tiles_host(const axisim_mesh_packed* mesh, int32_t S, int32_t cap, int32_t tileCells,
                                int32_t* nTiles, int32_t* tileStart, int32_t* layerEnd, int32_t* gid, uint64_t* lnb,
                                int64_t capacity);

/* ---- measurement ---- */
/* Per-kernel statistics of the profiled iterations: launches, summed CUDA-event
 * time between consecutive launches and the algorithmic bytes (each array
 * element the kernel's arithmetic needs, counted once per launch). */
typedef struct axisim_kernel_stat {
    char name[32];
    int32_t launches;
    double ms;
    double bytes;
} axisim_kernel_stat;
/* New (the reference times only the whole solve, solver.cpp:907-908,1318-1323):
 * runs `iterations` SIMPLE iterations eagerly from the current state, with an
 * event recorded after every kernel on the solver's stream. */
int axisim_profile_iteration(axisim_handle* h, int32_t iterations, axisim_kernel_stat* out, int32_t maxOut,
                             int32_t* nOut);
/* As axisim_profile_iteration, with every multigrid launch (smoothing,
 * residual, restriction, prolongation, Galerkin, the one-CTA tail) named
 * "<kernel>@<level>" for a per-level breakdown of the V-cycle. */
int axisim_profile_levels(axisim_handle* h, int32_t iterations, axisim_kernel_stat* out, int32_t maxOut,
                          int32_t* nOut);
/* New (the reference logs no set-up timings): host-clock cost of the handle's
 * set-up stages (mesh validation, upload, GPU precompute, multigrid hierarchy,
 * level build, graph capture / instantiate / upload, state reset, the solve's
 * iteration loop), summed per stage since creation or the last reset. Each
 * entry reuses axisim_kernel_stat: `launches` counts the stage's calls, `ms`
 * is their total, `bytes` is 0. reset != 0 clears the record after reading. */
int axisim_setup_profile(axisim_handle* h, axisim_kernel_stat* out, int32_t maxOut, int32_t* nOut, int32_t reset);
/* New; no counterpart in the reference. The mesh's 32-cell segments (cells
 * 32s .. 32s + 31) as set_mesh classified them for the kernels on its slots:
 * nOffsetSegments have every slot's neighbour at one offset from the cell for
 * all 32 cells (no boundary slot), so the sweeps form the neighbour indices
 * instead of loading them; nFaceSegments of those also number each slot's face
 * affinely (stride 1 or 2) with the cell on the same side of it, so the
 * assembly kernels form the face, owner and neighbour too. inUse is 0 when the
 * tables are not used: a mesh with more than four faces per cell, or with
 * fewer than half its segments regular. Any argument may be NULL. */
int axisim_mesh_segments(axisim_handle* h, int32_t* nSegments, int32_t* nOffsetSegments, int32_t* nFaceSegments,
                         int32_t* inUse);

/* New; no counterpart in the reference. The SIMPLE residuals of caller-owned
 * device arrays, computed with the same arithmetic as a solve's residual step
 * (residualAll + continuityResidual, residuals.cu:5-100) but with NO device
 * allocation: for callers that cannot allocate at that point -- a host whose
 * GPU memory is all held by another allocator or capped, or a monitoring hook
 * inside a time-critical loop where cudaMalloc/cudaFree would stall the device.
 * The reduction scratch is a fixed file-scope device array sized for at most
 * AXISIM_STATIC_MAX_CELLS cells; larger nCells is rejected with AXISIM_E_ARG.
 * Inputs, all device pointers on the current device, in the reference's CSR
 * slot order: cellFaceStart[nCells + 1], cellFaceIDs[nSlots],
 * faceOwner/faceNeighbor/mDot[nFaces], AF[nSlots] (u and v share it),
 * ACu/ACv/bu/bv/u/v[nCells]; normU/normV 0 = L1, 1 = L2, 2 = LINF.
 * Outputs: resU/resV = |b - A x| and resC = the signed mass imbalance per cell,
 * sums[5] = the U statistic (sum, sum of squares or max by norm), sum |AC_u u|,
 * the V statistic, sum |AC_v v| and sum |imbalance| -- the values before
 * residualAllHost's scaling. The per-cell arrays equal a solve's bit for bit;
 * the sums are deterministic but reduced in a different order (256-cell block
 * partials, then a 256-wide tree), so they agree with the solve's to rounding,
 * not bit for bit. Runs on the calling thread's current device, on `stream` (a
 * cudaStream_t; NULL = default stream), and returns once the results are
 * written: every call ends with a blocking read-back, so NO call may be made
 * while `stream` is being captured into a CUDA graph (AXISIM_E_ARG). Pointers
 * into another GPU's memory are rejected (AXISIM_E_ARG). Out-of-range indices
 * are skipped and reported as AXISIM_E_MESH with their count. All calls share
 * the scratch: calls that overlap in time (other threads, or other streams
 * still running) race and give wrong sums.
 * Messages go to err[errLen] (may be NULL). */
#define AXISIM_STATIC_MAX_CELLS 4194304
int axisim_residual_static(int32_t nCells, int32_t nFaces, int32_t nSlots, const int32_t* cellFaceStart,
                           const int32_t* cellFaceIDs, const int32_t* faceOwner, const int32_t* faceNeighbor,
                           const double* AF, const double* ACu, const double* ACv, const double* bu,
                           const double* bv, const double* u, const double* v, const double* mDot,
                           int32_t normU, int32_t normV, double* resU, double* resV, double* resC, double* sums,
                           void* stream, char* err, size_t errLen);

/* ---- host case preparation ---- */
/* Multiblock structured mesh (structs/multiblock.h): makeRectBlock +
 * autoDetectInterfaces + assignGlobalNumbering + toPackedMesh. */
typedef struct axisim_block_spec {
    double z0, r0;
    double axialLength;  int32_t axialCells;  int32_t axialGrading;  double axialCoef;
    double radialLength; int32_t radialCells; int32_t radialGrading; double radialCoef;
    int32_t edgeGroup[4];  /* West, East, South, North; -1 = default group */
} axisim_block_spec;

typedef struct axisim_mesh axisim_mesh;
/* status_out: 0 ok, 1 non-conformal seam (interfaces dropped, as mesh.cpp:2742-2745) */
int axisim_multiblock_build(int32_t nBlocks, const axisim_block_spec* blocks, double tol,
                            int32_t defaultGroup, axisim_mesh** out, int32_t* seamStatus);
int axisim_mesh_sizes(const axisim_mesh* m, int32_t* nCells, int32_t* nFaces, int32_t* nRefs);
/* fills `view` with pointers into the mesh object (valid until axisim_mesh_free) */
int axisim_mesh_view(const axisim_mesh* m, axisim_mesh_packed* view);
int axisim_mesh_free(axisim_mesh* m);

/* The domain outline as Mesh keeps it (BoundaryVertex / BoundaryEdge,
 * structs/boundary_struct.h:408-490): vertex positions and the edges between
 * them, each with its boundary group (-1 = unassigned). Obstacle loops are
 * more edges of the same outline. */
typedef struct axisim_outline {
    int32_t nVertices;
    const double* vertexZ;
    const double* vertexR;
    int32_t nEdges;
    const int32_t* edgeV0;
    const int32_t* edgeV1;
    const int32_t* edgeGroup;
} axisim_outline;
/* Mesh::buildStructuredMultiBlock + createMultiBlockFVMesh (mesh.cpp:2717-2762,
 * 2364-2462): trellis lines zLines[nZLines] and rLines[nRLines] (ascending)
 * cut the domain into cells; each trellis cell whose centre lies inside the
 * outline (even-odd ray cast, Mesh::pointInsideDomain, mesh.cpp:1177-1205)
 * becomes a uniform block of zBandCells[i] x rBandCells[j] cells; with none
 * inside, one nz x nr block covers [0, L] x [0, R]. Blocks are joined and
 * packed as axisim_multiblock_build does, then every external face takes the
 * group of the nearest grouped outline edge within 1e-4 max(L, R, 1)
 * (Mesh::classifyBoundaryFaces, mesh.cpp:1835-1846). */
int axisim_trellis_build(int32_t nZLines, const double* zLines, int32_t nRLines, const double* rLines,
                         const int32_t* zBandCells, const int32_t* rBandCells, const axisim_outline* outline,
                         double L, double R, int32_t nz, int32_t nr, axisim_mesh** out, int32_t* seamStatus);
/* Mesh::createUnstructuredMesh (mesh.cpp:1848-2002): nTriangles triangles
 * (3 point ids each) over nPoints shared points; cell centre the vertex mean,
 * volume 2 pi r_c A; faces created per triangle in edge order (v0 v1),
 * (v1 v2), (v2 v0), owned by the first triangle to reach them, normal away
 * from the owner, area 2 pi r_f L; external faces classified as above.
 * An edge shared by more than two triangles is rejected (AXISIM_E_MESH). */
int axisim_triangle_mesh_build(int32_t nPoints, const double* pointZ, const double* pointR, int32_t nTriangles,
                               const int32_t* triangles, const axisim_outline* outline, double L, double R,
                               axisim_mesh** out);
/* Mesh::classifyBoundaryFaces on a packed mesh the caller holds: rewrites
 * faceBoundaryGroupID[f] for every face with faceNeighbor[f] < 0. */
int axisim_classify_boundary_faces(int32_t nFaces, const int32_t* faceNeighbor, const double* faceCenterZ,
                                   const double* faceCenterR, const axisim_outline* outline, double L, double R,
                                   int32_t* faceBoundaryGroupID);

/* BoundaryDefaults::getEffectiveBC + createBoundaryFieldHost for one group and
 * one variable (boundary_func.cpp:104-201, 333-378; memory_manger.cpp:96-109):
 * given the group's BoundaryType and the user's BC (hasUser = 0 for none),
 * writes the effective BCType (PULSATILE mapped to DIRICHLET) and value. */
int axisim_resolve_bc(int32_t boundaryType, int32_t variable, int32_t hasUser,
                      int32_t userType, double userValue, uint8_t* typeOut, double* valueOut,
                      uint8_t* pulsatileOut);

#ifdef __cplusplus
}
#endif
#endif
