/*
 * axisim_oracle.h -- CPU restatement of AxiSim's SIMPLE pressure-velocity loop.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the parity checker for the CUDA
 * path in axisim-software_b200/. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it; the product never links it.
 *
 * Every routine restates one piece of the reference (Luippe/AxiSim-Software) and
 * cites the file:line it follows. Arithmetic is FP64 in the same operation
 * order as the reference kernels so the two agree to rounding (the reference's
 * multigrid Galerkin build and restriction use atomicAdd, which this oracle
 * replaces with an ascending-cell-order sum).
 *
 * Parity of this restatement is pinned by fixtures produced by the reference's
 * own solver (compiled headless from its sources, oracle/ref_build) and by the
 * analytic Hagen-Poiseuille solution (tools/validation.py:180-274).
 */
#ifndef AXISIM_ORACLE_H
#define AXISIM_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirror of FVMeshHostPacked (structs/solver_struct.h:400-429). */
typedef struct orc_mesh {
    int32_t nCells;
    int32_t nFaces;
    const int32_t* faceOwner;
    const int32_t* faceNeighbor;
    const double* faceNormalZ;
    const double* faceNormalR;
    const double* faceCenterZ;
    const double* faceCenterR;
    const double* faceArea;
    const int32_t* faceBoundaryGroupID;
    const double* cellCenterZ;
    const double* cellCenterR;
    const double* cellArea2D;
    const double* cellVolume;
    const int32_t* cellFaceStart; /* nCells + 1 */
    const int32_t* cellFaceIDs;   /* cellFaceStart[nCells] */
} orc_mesh;

/* Mirror of the solver-facing part of BoundaryFieldHost
 * (structs/solver_struct.h:464-476). lengthByGroup carries the group's float
 * totalLength widened to double (boundary_struct.h:515). */
typedef struct orc_bc_field {
    int32_t nGroups;
    const uint8_t* typeByGroup;          /* BCType: 0 DIRICHLET 1 NEUMANN 2 FULLY_DEVELOPED ... */
    const uint8_t* boundaryTypeByGroup;  /* BoundaryType: 0 WALL 1 INLET 2 OUTLET 3 SYMMETRY 4 FAR_FIELD */
    const double* valueByGroup;
    const double* lengthByGroup;
    /* Pulsatile inlet (boundary_struct.h:112-115, 150-158): per group flag and
     * parameters; NULL when the run has none. */
    const uint8_t* pulsatileByGroup;
    const double* amplitudeByGroup;
    const double* frequencyByGroup;
    /* Michaelis-Menten / Hill wall kinetics per group (BoundaryFieldHost
     * vmax..Rtot, solver_struct.h:469-475, filled by memory_manger.cpp:110-145);
     * NULL = the defaults vmax = km = k2 = v2 = Rtot = 0, n = m = 1. */
    const double* vmaxByGroup;
    const double* kmByGroup;
    const double* nByGroup;
    const double* mByGroup;
    const double* k2ByGroup;
    const double* v2ByGroup;
    const double* RtotByGroup;
} orc_bc_field;

/* Flattened ConfigSolver / ConfigSimple / ConfigMultigrid / ConfigResidual /
 * FluidPropertyConfig / relaxation (solver_struct.h:158-313, setting.cuh:60-71). */
typedef struct orc_config {
    /* ConfigSolver */
    int convectionScheme;   /* 0 UPWIND 1 CENTRAL 2 SOU 3 QUICK(->upwind) */
    int gradientScheme;     /* 0 GREEN_GAUSS 1 LSQ */
    int linearType;         /* 0 JACOBI 1 GS_RB (multicolour) */
    int timeScheme;         /* 0 BDF1 1 BDF2 */
    int linearMaxIter;
    int useMultigrid;
    int addConvectionTerm;
    int transient;
    int useNonOrthCorrector;
    double dt;
    double tEnd;
    /* ConfigSimple */
    int maxIter;
    int checkConv;
    /* ConfigMultigrid */
    int mgMaxIter;
    double mgWeight;
    int mgLinearSweep;
    int mgPreSweep;
    int mgPostSweep;
    /* fluid */
    double rho;
    double mu;
    /* VariablesSimple relaxation */
    double alphaU;
    double alphaP;
    /* ConfigResidual for U, V, Continuity: norm 0 L1 1 L2 2 LINF;
     * scale 0 NONE 1 N 2 SQRT_N 3 DIAGONAL */
    int resNorm[3];
    int resScale[3];
    int resEnabled[3];
    double resTol[3];
    /* scalar transport: SolverFieldOption (solver_struct.h:9-12), the
     * FluidPropertyConfig cp, k, D (setting.cuh:61-71) and the ConfigResidual
     * entries "Temperature", "Concentration" (index 0 T, 1 C) */
    int solveEnergy;
    int solveConcentration;
    double cp;
    double k;
    double D;
    int scalarResNorm[2];
    int scalarResScale[2];
    int scalarResEnabled[2];
    double scalarResTol[2];
    /* Mesh::currentMeshType == Structured (boundary_struct.h:382-385) */
    int structuredMesh;
} orc_config;

typedef struct orc_solver orc_solver;

/* --- multiblock structured mesh builder (structs/multiblock.h) ----------- */
typedef struct orc_block_spec {
    double z0, r0;
    double axialLength;  int axialCells;  int axialGrading;  double axialCoef;
    double radialLength; int radialCells; int radialGrading; double radialCoef;
    int edgeGroup[4];    /* West, East, South, North */
} orc_block_spec;

typedef struct orc_packed orc_packed;
orc_packed* orc_mb_build(int nBlocks, const orc_block_spec* blocks, double tol,
                         int defaultGroup, int* status);
void orc_mb_sizes(const orc_packed* p, int32_t* nCells, int32_t* nFaces, int32_t* nRefs);
/* fills every array of a caller-allocated mesh (non-const cast of orc_mesh) */
void orc_mb_copy(const orc_packed* p,
                 int32_t* faceOwner, int32_t* faceNeighbor,
                 double* faceNormalZ, double* faceNormalR,
                 double* faceCenterZ, double* faceCenterR, double* faceArea,
                 int32_t* faceBoundaryGroupID,
                 double* cellCenterZ, double* cellCenterR,
                 double* cellArea2D, double* cellVolume,
                 int32_t* cellFaceStart, int32_t* cellFaceIDs);
void orc_mb_free(orc_packed* p);

/* --- solver ---------------------------------------------------------------- */
orc_solver* orc_create(const orc_mesh* mesh, const orc_bc_field* bcU,
                       const orc_bc_field* bcV, const orc_bc_field* bcP,
                       const orc_config* cfg);
/* The same with the temperature and concentration boundary fields (each may be
 * NULL when cfg does not solve that field). */
orc_solver* orc_create_ex(const orc_mesh* mesh, const orc_bc_field* bcU,
                          const orc_bc_field* bcV, const orc_bc_field* bcP,
                          const orc_bc_field* bcT, const orc_bc_field* bcC,
                          const orc_config* cfg);
/* Runs Solver::runSimple's time + SIMPLE loops (solver.cpp:1034-1298).
 * Returns the SIMPLE iterations executed; *converged set if the residual test
 * passed. continueRun keeps currentIteration / continuity scale / time offset. */
int orc_run(orc_solver* s, int continueRun, int* converged);
/* Fields: u v p pp mDot DU DV gradPZ gradPR gradUZ gradUR gradVZ gradVR
 *         AC_u b_u AF_u invAC_u (and _v, _pp) res_U res_V res_Continuity
 *         T C gradTZ gradTR gradCZ gradCR AC_T b_T AF_T invAC_T (and _C)
 *         TOld COld TOld2 COld2 res_T res_C cw ocrWall (per face) */
int orc_get(const orc_solver* s, const char* name, double* out, size_t n);
int orc_set(orc_solver* s, const char* name, const double* in, size_t n);
/* residual history: resVal for U, V, Continuity of the last check */
void orc_last_residuals(const orc_solver* s, double out[3]);
/* resVal of the Temperature and Concentration entries of the last check */
void orc_scalar_residuals(const orc_solver* s, double out[2]);
int orc_iterations(const orc_solver* s);
/* multigrid hierarchy description: level count and cells per level */
int orc_mg_levels(const orc_solver* s, int32_t* cellsPerLevel, int maxLevels);
int orc_mg_level_maps(const orc_solver* s, int level, int32_t* cellToCoarse,
                      int32_t* fineSlotToCoarseSlot, int32_t* coarseFaceStart,
                      int32_t* coarseFaceNeighbor);
/* greedy colouring (memory_manger.cpp:334-409): colour per cell, returns nColors */
int orc_coloring(const orc_solver* s, int32_t* colorOut);
void orc_destroy(orc_solver* s);
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
