// device.cuh -- device-side data layout of the B200 SIMPLE solver.
//
// Layout in HBM (structure of arrays):
//   * faces:  owner, neighbor, group, normal, centre, area and the precomputed
//             geometry (invDPN, wP, dPB, length2D, lsqW) as one array each;
//   * cells:  centre, volume, invA2D, LSQ inverse matrix, fields;
//   * slots:  a cell's faces in the reference's CSR order, stored as an ELL
//             block [W][N] (slot j of cell n at j*N + n), so the per-cell face
//             loops and the smoother sweeps read coalesced columns. W is the
//             largest face count of any cell (4 on quads, 3 on triangles);
//             unused slots carry face -1 and neighbour -1.
// The momentum off-diagonals are identical for u and v in the reference
// (diffusion -mu A/d plus min(F,0) on the same faces), so one AF block serves
// both momentum systems.
#pragma once

#include <cstdint>
#include <utility>

#include <cuda_runtime.h>

namespace axisim {

// Programmatic dependent launch: every kernel of the SIMPLE iteration is
// launched with programmatic stream serialisation, so its launch and CTA
// scheduling overlap the tail of the kernel before it. Each kernel waits for
// its predecessor's results (griddepcontrol.wait) before reading anything,
// then lets its own successor be scheduled (griddepcontrol.launch_dependents);
// a successor's CTAs only start once the last CTA of this grid has started.
__device__ __forceinline__ void pdlEnter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Set on the host thread before a launch whose predecessor in the captured
// graph is not a kernel (the first kernel of a conditional node's body, the
// first kernel after that node): the next launchPDL then goes without the
// programmatic attribute, and clears the flag.
inline thread_local bool tNextLaunchPlain = false;

template <typename... KArgs, typename... Args>
inline cudaError_t launchPDL(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = tNextLaunchPlain ? 0 : 1;
    tNextLaunchPlain = false;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int kMaxHist = 128;   // residual history ring (>= largest graph batch)

struct MeshDev {
    int N = 0, F = 0, W = 0;
    const int32_t* owner = nullptr;
    const int32_t* neighbor = nullptr;
    const int32_t* group = nullptr;
    const double* nZ = nullptr;
    const double* nR = nullptr;
    const double* fcZ = nullptr;
    const double* fcR = nullptr;
    const double* area = nullptr;
    const double* invDPN = nullptr;
    const double* wP = nullptr;
    const double* dPB = nullptr;
    const double* length2D = nullptr;
    const double* lsqWZ = nullptr;
    const double* lsqWR = nullptr;
    const double* ccZ = nullptr;
    const double* ccR = nullptr;
    const double* vol = nullptr;
    const double* invA2D = nullptr;
    const double* lsqIZZ = nullptr;
    const double* lsqIZR = nullptr;
    const double* lsqIRR = nullptr;
    const int32_t* sface = nullptr;  // [W][N]
    const int32_t* snb = nullptr;    // [W][N]
    const int4* sseg = nullptr;      // [(N + 31) / 32] slot offsets by segment (segNeighbours); null: none
    const int4* ssegF = nullptr;     // [(N + 31) / 32] face of each slot at the segment's first cell (slotFaces)
    const int* ssegM = nullptr;      // [(N + 31) / 32] face strides and owner sides (slotFaces); < 0: none
};

// Slot neighbours by 32-cell segment. Where all 32 cells n = 32s .. 32s + 31
// of a segment have every slot's neighbour at the same offset,
// snb[j][n] = n + d_j (the interior of a structured block), sseg[s] holds
// d_0 .. d_3 and the sweeps form the neighbours without reading snb; every
// other segment (a boundary, a block seam, a partial last segment, an
// irregular numbering) holds kSegIrregular in .x and its cells read snb. A
// warp is one segment, so its lanes take the same branch and the segment's
// entry is one broadcast load. The neighbours, and so every result, are the
// same either way.
constexpr int kSegIrregular = (int)0x80000000;

template <int WC>
__device__ __forceinline__ void segNeighbours(const int4* __restrict__ seg, const int32_t* __restrict__ snb, int N,
                                              int n, int (&k)[WC]) {
    static_assert(WC >= 1 && WC <= 4, "segment offsets cover four slots");
    int4 d = make_int4(kSegIrregular, 0, 0, 0);
    if (seg) d = __ldg(seg + (n >> 5));
    if (d.x != kSegIrregular) {
        const int dd[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
        for (int j = 0; j < WC; j++) k[j] = n + dd[j];
    } else {
#pragma unroll
        for (int j = 0; j < WC; j++) k[j] = snb[(size_t)j * N + n];
    }
}

// The face, owner and neighbour of each of a cell's WC slots. Where the
// cell's segment numbers its faces affinely (ssegM[s] >= 0; on the
// structured blocks every segment with slot offsets does): slot j's face is
// ssegF[s].j + t_j (n - 32s) with stride t_j = 1 or 2 (bit j of ssegM[s]), and
// the cell is that face's owner throughout the segment (bit 4 + j) or its
// neighbour, the other cell being n + d_j. Elsewhere from sface, owner and
// neighbor; a slot beyond the cell's faces gets face -1, and the owner and
// neighbour read for it (face 0's) are never used. Either way the values are
// those the face arrays hold.
template <int WC>
__device__ __forceinline__ void slotFaces(const MeshDev& m, int n, int (&f)[WC], int (&own)[WC], int (&nb)[WC]) {
    static_assert(WC >= 1 && WC <= 4, "segment faces cover four slots");
    const int s = n >> 5;
    // the segment's three entries are loaded together (the tables exist as a
    // set), so the test below does not put a second load round trip ahead of
    // the face numbers
    int meta = -1;
    int4 d = make_int4(0, 0, 0, 0), b = make_int4(0, 0, 0, 0);
    if (m.ssegM) {
        meta = __ldg(m.ssegM + s);
        d = __ldg(m.sseg + s);
        b = __ldg(m.ssegF + s);
    }
    if (meta >= 0) {
        const int r = n & 31;
        const int dd[4] = {d.x, d.y, d.z, d.w}, bb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int j = 0; j < WC; j++) {
            f[j] = bb[j] + (((meta >> j) & 1) ? 2 * r : r);
            const bool o = (meta >> (4 + j)) & 1;
            own[j] = o ? n : n + dd[j];
            nb[j] = o ? n + dd[j] : n;
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < WC; j++) f[j] = m.sface[(size_t)j * m.N + n];
#pragma unroll
    for (int j = 0; j < WC; j++) {
        const int g = f[j] >= 0 ? f[j] : 0;
        own[j] = m.owner[g];
        nb[j] = m.neighbor[g];
    }
}

struct BCDev {
    int nGroups = 0;
    const uint8_t* type = nullptr;
    const double* value = nullptr;
    const double* length = nullptr;
    // wall kinetics of a transported scalar, [9][nGroups]: Vmax, Km, n, m, K2,
    // V2, Rtot, Km^n, K2^m (null for u, v, p)
    const double* kin = nullptr;
};

// Control block: one per solver, in device memory. Kernels of an iteration
// return at entry once `done` is set, so a captured iteration graph can be
// replayed past convergence without changing the result.
struct Ctl {
    int done;             // 0 running, 1 converged, 2 stopped, 3 iteration budget, 4 non-finite residual,
                          // 5 a grid barrier of the resident V-cycle gave up
    int k;                // SIMPLE iteration within the current time step
    int currentIteration; // run-global iteration counter (continues across continue runs)
    int maxIter;
    int checkConv;
    int transient;
    int bdf2;             // BDF2 active in this time step
    int converged;        // result of the last check
    int checked;          // a residual check ran this iteration
    int itersThisCall;
    int pad0, pad1;
    double resVal[3];     // U, V, Continuity
    double scaleVal[3];
    double tol[3];
    int resNorm[3];
    int resScale[3];
    int resEnabled[3];
    int histCount;        // entries written since the host last drained
    double hist[kMaxHist][6];  // iteration, U, V, Continuity, Temperature, Concentration
    // batch of independent cases packed into one mesh (nCases = 0: one case)
    int nCases;
    int casesConverged;
    // Krylov p' solve: set once its residual meets the tolerance, so the
    // remaining kernels of that solve (cycles included) return at entry;
    // cleared when the solve ends
    int ppSkip;
    int ppPad;
    long long ppSolves;      // Krylov solves started
    long long ppIterations;  // Krylov iterations completed
    // monitored residuals of the transported scalars (0 Temperature, 1 Concentration)
    double resValS[2];
    double scaleValS[2];
    double tolS[2];
    int resNormS[2];
    int resScaleS[2];
    int resEnabledS[2];
    int solvedS[2];       // the scalar is solved (an unsolved one has an all-zero system)
    // grid-wide barrier of the resident V-cycle kernel: arrivals, generation;
    // mgErr is set when a wait gives up (the next iteration then ends the run);
    // mgPhantom extra arrivals are expected per barrier (0; 1 in a test that
    // makes a wait run out)
    unsigned int mgBar[2];
    int mgErr;
    int mgPhantom;
};

// One transported scalar (energy or concentration) in the fused assembly.
struct ScalarDev {
    BCDev bc;
    const double* phi;
    const double* gZ;
    const double* gR;
    const double* old;
    const double* old2;
    double* AF;  // [W][N]
    double* AC;
    double* b;
    double* inv;
    double* wall;  // per face: c_w of this scalar's reactive wall faces
    double gamma;  // kinematic diffusivity
    double alpha;  // under-relaxation factor
};

struct ScalarArgs {
    ScalarDev s[2];
    const double* mDot;
    double* cw;    // wall concentration per face
    double* ocr;   // wall consumption per face
    double fluxScale, dt;
    int conv, scheme, nonOrtho, transient;
};

// The learned first Krylov step: which p' solves use it, and the running means
// the choice is made from (device memory, one per solver). Each solve's score
// is its mean log residual reduction per Krylov iteration, log(||r_end|| /
// ||r_0||) / iterations, from the FP64 residual.
struct NetStats {
    long long applied;    // solves whose first step used the network
    long long fallbacks;  // solves that ran the plain V-cycle because its score was better
    double logRhoNet;     // running mean score of solves with the network
    double logRhoV;       // running mean score of solves without it
    long long nNet, nV;   // solves in those means
    long long solveIdx;   // learned-enabled solves so far (probe schedule)
    int curNet;           // this solve uses the network
    int pad;
};

// Per-case monitoring of a batch: raw sums per case and the reference's
// residual arithmetic (residuals.cu:37-100) applied case by case.
struct BatchDev {
    int nCases = 0;
    const int32_t* cellStart = nullptr;  // nCases + 1
    double* raw = nullptr;               // 5 per case: |rU|, scaleU, |rV|, scaleV, |continuity|
    double* resVal = nullptr;            // 3 per case
    double* scaleVal = nullptr;          // 3 per case
    int32_t* convergedAt = nullptr;      // first converged iteration, -1 before
};

struct MomentumArgs {
    const double* mDot;
    const double* u;
    const double* v;
    const double* gUZ;
    const double* gUR;
    const double* gVZ;
    const double* gVR;
    const double* gPZ;
    const double* gPR;
    const double* uOld;
    const double* vOld;
    const double* uOld2;
    const double* vOld2;
    double* AF;     // [W][N] shared by u and v
    double* ACu;
    double* ACv;
    double* bu;
    double* bv;
    double* invACu;
    double* invACv;
    double* DU;
    double* DV;
    double mu, rho, dt, alpha;
    int conv, scheme, nonOrtho, transient;
    // mixed precision: FP32 copies of AF and 1/AC for the correction sweeps (null on the FP64 path)
    float* AF32;
    float* invU32;
    float* invV32;
};

}  // namespace axisim
