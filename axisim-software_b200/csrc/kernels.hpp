// kernels.hpp -- host launchers for the sm_100a kernels of the SIMPLE path.
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace axisim {

// One multigrid level on the device, values of type T (double on the FP64
// path, float for the mixed-precision cycle). Level 0 aliases the p' system
// and uses the mesh's [W][N] slot block; coarser levels use sliced ELL:
// 32-row slices, slot j of cell n at sliceOff[n/32] + 32 j + n%32, slice width
// (sliceOff[s+1] - sliceOff[s]) / 32, unused slots with neighbour -1 and
// coefficient 0. Topology and transfer lists are shared by both precisions.
template <class T>
struct LevelT {
    int N = 0, W = 0;
    int totalSlots = 0;
    const int32_t* sliceOff = nullptr;  // null: [W][N] layout
    int32_t* nb = nullptr;
    const int4* seg = nullptr;  // finest level: the mesh's segment offsets (segNeighbours); null elsewhere
    T* AF = nullptr;
    T* AC = nullptr;
    T* b = nullptr;
    T* x = nullptr;
    T* xNew = nullptr;
    T* res = nullptr;          // fine residual (N)
    int32_t* c2c = nullptr;    // fine -> coarse (null on the coarsest level)
    // restriction / Galerkin gathers, stored on the COARSE level:
    int32_t* mStart = nullptr;  // [N+1] members of each coarse cell
    int32_t* mList = nullptr;   // fine cell ids, ascending
    int32_t* gStart = nullptr;  // [totalSlots+1] fine slots feeding each coarse slot
    int32_t* gList = nullptr;   // fine slot positions, ascending fine cell then slot
    uint32_t* internalMask = nullptr;  // on the FINE level: slots folding into the coarse diagonal
    int block = 0;  // threads per CTA of this level's smoothing, residual and transfer kernels (0: 256)
    // batch with per-case hierarchies: the cases whose coarsest level this is
    // (not the deepest level), as [begin, end) cell ranges; their cells have
    // c2c = -1, keep their values through the level's sweeps and transfers,
    // and are solved by the coarsest-level sweeps of launchMGTerminal
    int nTerm = 0;
    int termMax = 0;                // cells of the largest terminal range
    const int32_t* term = nullptr;  // [2 nTerm]
};
using LevelDev = LevelT<double>;
using LevelF = LevelT<float>;

// Levels at and below `first` solved inside one CTA (V-cycle tail).
constexpr int kMaxTail = 8;
template <class T>
struct TailArgsT {
    int first = 0, count = 0;
    LevelT<T> lv[kMaxTail];
    int smemOff[kMaxTail];   // elements of T: x, y, b, r per level
    const T* resFine = nullptr;
    T* xOut = nullptr;
    T w = T(0.6);
    T prolongScale = T(1);  // coarse correction x += s P e (1 in the reference's cycle)
    int pre = 1, post = 1, coarseSweeps = 30;
};
using TailArgs = TailArgsT<double>;

// The V-cycle below the finest level run as ONE resident (cooperative) kernel:
// the phases the per-phase launches would run, recorded in order at capture
// time, each followed by a grid-wide barrier. Every phase keeps the per-cell
// arithmetic of its separate kernel, so results are the same bit for bit.
enum MgOpType : int {
    kOpSmooth = 1,      // y = sweep(x) on the level              p0 = x, p1 = y
    kOpSmoothBlock,     // ival sweeps of the level in one CTA    p0 = x (in place)
    kOpResidual,        // res = b - A x                          p0 = x
    kOpGather,          // b = restricted finer residual; x = 0 or first sweep (ival) p0 = xCur, p1 = xAlt
    kOpTerminal,        // terminal cases' coarsest sweeps (ival) p0 = x
    kOpProlong,         // x += scale * P xc                      p0 = x (fine), p1 = xc
    kOpTail,            // the one-CTA tail (ResidentArgsT::tail)
    kOpGatherRes,       // kOpGather with the finer residual formed on the fly  p2 = fine x
    kOpProlongSmooth,   // y = sweep(x + scale * P xc)           p0 = x, p1 = xc, p2 = y
};
struct MgOp {
    int type = 0, level = 0, ival = 0, pad = 0;
    void* p0 = nullptr;
    void* p1 = nullptr;
    void* p2 = nullptr;
    double scale = 0.0;
};
constexpr int kMaxResidentLevels = 12;
constexpr int kMaxResidentOps = 64;
template <class T>
struct ResidentArgsT {
    int nOps = 0, first = 0, nLevels = 0;
    T w = T(0);
    LevelT<T> lv[kMaxResidentLevels];  // levels first .. first + nLevels - 1
    MgOp ops[kMaxResidentOps];
    TailArgsT<T> tail;
    size_t smem = 0;  // dynamic shared memory the phases need
};

// ---- setup ----
void launchPrecompute(const MeshDev& m, const int32_t* cfs, const int32_t* cfi, double* lsqDZ, double* lsqDR,
                      cudaStream_t s);
void launchBuildEll(int N, int W, const int32_t* cfs, const int32_t* cfi, const int32_t* owner,
                    const int32_t* neighbor, int32_t* sface, int32_t* snb, cudaStream_t s);
// the segment tables of segNeighbours and slotFaces; adds the segments without
// slot offsets to nIrregular[0], those without affine faces to nIrregular[1]
void launchBuildSegments(const MeshDev& m, int4* seg, int4* segF, int* segM, int* nIrregular, cudaStream_t s);

// Tiles of the momentum Jacobi sweeps run several per launch from shared
// memory (SweepTiles in host_prep.hpp, kernel in sweep_tiles.cuh): one CTA of
// `threads` per tile, cap = K threads local cells, K = kSweepK32 (FP32) or
// kSweepK64 (FP64); lnb holds four 16-bit local neighbour indices per cell.
struct SweepTilesDev {
    int nTiles = 0, S = 0, cap = 0, threads = 0;
    const int32_t* tileStart = nullptr;
    const int32_t* layerEnd = nullptr;
    const int32_t* gid = nullptr;
    const uint2* lnb = nullptr;
};
constexpr int kSweepK32 = 4;
constexpr int kSweepK64 = 2;
constexpr int kMaxSweepsPerLaunch = 8;

// ---- one SIMPLE iteration ----
void launchIterBegin(Ctl* ctl, const volatile int* hostStop, cudaStream_t s);
// gradients of up to five fields (u, v, p, T, C) with their boundary fields
void launchGradient(const MeshDev& m, const Ctl* ctl, int nFields, const double* const* phi, const BCDev* bc,
                    double* const* gZ, double* const* gR, int scheme, cudaStream_t s);
void launchMomentum(const MeshDev& m, const Ctl* ctl, const BCDev& bcU, const BCDev& bcV,
                    const MomentumArgs& a, cudaStream_t s);
void launchJacobiUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* bu, const double* bv,
                    const double* invu, const double* invv, const double* xu, const double* xv, double* yu,
                    double* yv, cudaStream_t s);
// `sweeps` (<= t.S) Jacobi sweeps of u and v from x to y on tiles (W 3 or 4)
void launchJacobiUVTiles(const MeshDev& m, const Ctl* ctl, const SweepTilesDev& t, int sweeps, const double* AF,
                         const double* bu, const double* bv, const double* invu, const double* invv,
                         const double* xu, const double* xv, double* yu, double* yv, cudaStream_t s);
// the shared-memory size of the FP64 tile kernels (before the first launch)
cudaError_t allowJacobiUVTiles(int cap);
void launchGaussSeidelUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* bu, const double* bv,
                         const double* invu, const double* invv, double* xu, double* xv, const int32_t* order,
                         int begin, int count, cudaStream_t s);
// p' system + inverse diagonal + Rhie-Chow face mass flux (owner writes each face)
void launchPressureSystem(const MeshDev& m, const Ctl* ctl, const BCDev& bcU, const BCDev& bcV,
                          const BCDev& bcP, double rho, const double* u, const double* v, const double* p,
                          const double* gPZ, const double* gPR, const double* DU, const double* DV,
                          double* AFpp, double* ACpp, double* invACpp, double* mDot, float* AF32, float* AC32,
                          cudaStream_t s);
void launchPressureRhs(const MeshDev& m, const Ctl* ctl, double rho, const double* mDot, const double* DU,
                       const double* DV, const double* gZ, const double* gR, int cross, int zeroPP, double* bpp,
                       double* pp, cudaStream_t s);
// p' linear solve without multigrid (Jacobi ping-pong or colour sweep on one field)
void launchJacobi1(const MeshDev& m, const Ctl* ctl, const double* AF, const double* b, const double* inv,
                   const double* x, double* y, cudaStream_t s);
void launchGaussSeidel1(const MeshDev& m, const Ctl* ctl, const double* AF, const double* b, const double* inv,
                        double* x, const int32_t* order, int begin, int count, cudaStream_t s);
void launchCorrect(const MeshDev& m, const Ctl* ctl, const BCDev& bcP, double rho, double alphaP, int nonOrtho,
                   const double* pp, const double* gZ, const double* gR, const double* DU, const double* DV,
                   double* u, double* v, double* p, double* mDot, cudaStream_t s);
void launchResiduals(const MeshDev& m, const Ctl* ctl, const double* AF, const double* ACu, const double* ACv,
                     const double* bu, const double* bv, const double* u, const double* v, const double* mDot,
                     double* resU, double* resV, double* resC, double* scaleU, double* scaleV, double* partial,
                     int* nBlocksOut, cudaStream_t s);
// partialS: per block {stat_T, |diag_T|, stat_C, |diag_C|} of the scalar
// residual pass (null when no scalar residual is monitored)
void launchIterEnd(Ctl* ctl, const double* partial, const double* partialS, int nBlocks, int N, cudaStream_t s);
// batch: per-case reduction of the per-cell residual arrays, then per-case norms + convergence
void launchBatchIterEnd(Ctl* ctl, const BatchDev& b, const double* resU, const double* resV, const double* resC,
                        const double* scaleU, const double* scaleV, cudaStream_t s);
void launchCopy(const Ctl* ctl, double* dst, const double* src, int n, cudaStream_t s);

// ---- transported scalars (scalar.cu) ----
// wall concentration of the reactive boundary faces faces[0..nFaces) (before the assembly)
void launchScalarWall(const MeshDev& m, const Ctl* ctl, int ns, const ScalarArgs& a, const int32_t* faces,
                      int nFaces, cudaStream_t s);
// assembly of ns = 1 or 2 scalars (a.s[0..ns)) after the corrections
void launchScalarAssembly(const MeshDev& m, const Ctl* ctl, int ns, const ScalarArgs& a, cudaStream_t s);

// residualRaw of ns solved scalars, the first of monitoring entry `first`
// (0 Temperature, 1 Concentration), and the first reduction pass into
// partial[4 per block]
void launchScalarResidual(const MeshDev& m, const Ctl* ctl, int ns, int first, const double* const* AF,
                          const double* const* AC, const double* const* b, const double* const* x,
                          double* const* res, double* const* scale, double* partial, cudaStream_t s);

// ---- multigrid (mg.cu), T = double or float ----
// Galerkin P^T A P from a fine level of type TF into a coarse level of type TC
template <class TF, class TC>
void launchGalerkin(const Ctl* ctl, const LevelT<TF>& fine, const LevelT<TC>& coarse, cudaStream_t s);
// Galerkin of a chain of small levels (lv[i] -> lv[i+1], i < count - 1) in one
// single-CTA launch, level by level: the coarse operators of the V-cycle
// tail, each at most 1024 cells, without a launch per level.
template <class T>
struct GalChainArgsT {
    int count = 0;
    LevelT<T> lv[kMaxTail + 1];
};
template <class T>
void launchGalerkinChain(const Ctl* ctl, const GalChainArgsT<T>& a, cudaStream_t s);
template <class T>
void launchMGSmooth(const Ctl* ctl, const LevelT<T>& L, const T* x, T* y, T w, cudaStream_t s);
template <class T>
void launchMGSmoothBlock(const Ctl* ctl, const LevelT<T>& L, T* x, T w, int sweeps, cudaStream_t s);
template <class T>
void launchMGResidual(const Ctl* ctl, const LevelT<T>& L, const T* x, cudaStream_t s);
// b_c = sum of the fine residuals of each agglomerate; x_c = 0, or with
// firstSweep the result of one Jacobi sweep from zero written to xAlt
template <class T>
void launchMGGather(const Ctl* ctl, const LevelT<T>& fine, const LevelT<T>& coarse, T* xCur, T* xAlt,
                    int firstSweep, T w, cudaStream_t s);
template <class T>
void launchMGProlong(const Ctl* ctl, const LevelT<T>& fine, T* xFine, const T* xCoarse, T scale, cudaStream_t s);
// the restriction with the fine residual formed per member (no residual pass)
template <class T>
void launchMGGatherRes(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const LevelT<T>& coarse, T* xCur,
                       T* xAlt, int firstSweep, T w, cudaStream_t s);
// prolongation fused into the first post-smoothing sweep, any level layout
template <class T>
void launchMGProlongSmoothAny(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const T* xCoarse, T* y, T w,
                              T scale, cudaStream_t s);
// prolongation fused into the first post-smoothing sweep (ELL levels with
// W = 3 or 4): y = smooth(x + s P e), and upd[n] += (double)y[n] when upd is
// given; returns false when not applicable
template <class T>
bool launchMGProlongSmooth(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const T* xCoarse, T* y, T w,
                           T scale, cudaStream_t s, double* upd = nullptr);
// the coarsest-level solve of each terminal case of a level: `sweeps` Jacobi
// sweeps from zero, one CTA per case, written to x (cells of other cases untouched)
template <class T>
void launchMGTerminal(const Ctl* ctl, const LevelT<T>& L, T* x, T w, int sweeps, cudaStream_t s);
// the resident V-cycle kernel: one CTA of 1024 threads per SM (cooperative
// launch, no programmatic serialisation on either side); false when the
// device cannot hold the grid or the program does not fit
template <class T>
bool launchMGResident(Ctl* ctl, const ResidentArgsT<T>& a, cudaStream_t s);
template <class T>
size_t tailSharedBytes(const TailArgsT<T>& a);
template <class T>
void launchMGTail(const Ctl* ctl, const TailArgsT<T>& a, cudaStream_t s);

// ---- mixed precision (kernels_mixed.cu) ----
// p' cycle as iterative refinement: r = b - A x in FP64, stored as FP32 with
// the first Jacobi sweep of the correction (from zero); x += e after the cycle.
void launchIRResidualPP(const Ctl* ctl, const LevelDev& L0, float* r32, float* eFirst, double w, int firstSweep,
                        cudaStream_t s);
void launchIRUpdatePP(const Ctl* ctl, int N, double* x, const float* e, cudaStream_t s);
// momentum in correction form: r = b - A u (FP64) -> FP32, first Jacobi sweep
// delta = r / AC; FP32 sweeps on delta; u += delta
void launchIRResidualUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* ACu, const double* ACv,
                        const double* bu, const double* bv, const double* u, const double* v, const float* iu32,
                        const float* iv32, float* ru, float* rv, float* du, float* dv, cudaStream_t s);
void launchJacobiUV32(const MeshDev& m, const Ctl* ctl, const float* AF32, const float* ru, const float* rv,
                      const float* iu32, const float* iv32, const float* du, const float* dv, float* du2, float* dv2,
                      cudaStream_t s);
void launchJacobiUV32Tiles(const MeshDev& m, const Ctl* ctl, const SweepTilesDev& t, int sweeps, const float* AF32,
                           const float* ru, const float* rv, const float* iu32, const float* iv32, const float* du,
                           const float* dv, float* du2, float* dv2, cudaStream_t s);
cudaError_t allowJacobiUV32Tiles(int cap);
void launchIRUpdateUV(const Ctl* ctl, int N, double* u, double* v, const float* du, const float* dv, cudaStream_t s);

// ---- flexible CG on the p' system, FP32 V-cycle preconditioner (krylov.cu) ----
// partial: one FP64 pair per block of 256 cells; counter[2] start at zero;
// scalars[0] = (r, z), [1] = (z, q_prev), [2] and [3] = (p, q) of alternate
// iterations, [4] = (b, b), [5] = (r, r), [6] = Krylov iteration counter at
// the solve's start, [7] = (r0, r0), [8..10] = learned step scale and its dots.
struct FcgScratch {
    double* partial = nullptr;
    unsigned int* counter = nullptr;
    double* scalars = nullptr;
};
void launchFcgInit(Ctl* ctl, const LevelDev& L0, const double* x, double* r, float* r32, float* eFirst, double w,
                   int firstSweep, double relTol, FcgScratch& f, cudaStream_t s);
void launchFcgDots(const Ctl* ctl, int N, const float* e, const double* r, const double* q, int useQ, FcgScratch& f,
                   cudaStream_t s);
void launchFcgSpmv(const Ctl* ctl, const LevelDev& L0, const float* e, const double* pOld, double* pNew, double* q,
                   int first, int pqOld, int pqNew, FcgScratch& f, cudaStream_t s);
// next: 0 = x only, 1 = also r and (r, r), 2 = also the first sweep; the
// solve stops (Ctl::ppSkip) at relTol or after maxIt iterations
void launchFcgUpdate(Ctl* ctl, const LevelDev& L0, double* x, double* r, const double* p, const double* q,
                     FcgScratch& f, int pqSlot, float* r32, float* eFirst, double w, int next, double relTol,
                     int maxIt, cudaStream_t s);
// condition of the conditional WHILE node that repeats the Krylov iterations
// in a captured graph: head (before the node) resets the body count, tail
// (last kernel of the body) counts one; both set run = solve not stopped and
// fewer than maxBodies bodies run
void launchFcgLoop(Ctl* ctl, FcgScratch& f, cudaGraphConditionalHandle h, int head, int maxBodies, cudaStream_t s);
// per-solve choice between the learned first preconditioner and the V-cycle;
// the learned one is z = alpha y + V-cycle(r - alpha A y), y the network's
// output and alpha = (y, r) / (y, A y) its best scale (scalars [8..10])
void launchFcgGate(Ctl* ctl, NetStats* ns, int always, cudaStream_t s);
void launchFcgUngate(Ctl* ctl, cudaStream_t s);
void launchNnResidual(const Ctl* ctl, const LevelDev& L0, const double* r, const float* y, double* Ay,
                      FcgScratch& f, float* r32, float* eFirst, double w, int firstSweep, cudaStream_t s);
void launchNnCombine(const Ctl* ctl, const NetStats* ns, int N, const float* y, const FcgScratch& f, float* e,
                     cudaStream_t s);
// clears Ctl::ppSkip after the solve; with ns, scores the solve
void launchFcgEnd(Ctl* ctl, const FcgScratch& f, NetStats* ns, cudaStream_t s);

}  // namespace axisim
