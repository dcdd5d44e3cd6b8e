// mg.cu -- agglomeration multigrid V-cycle for the pressure correction (sm_100a).
//
// Same algorithm as MultigridSolver (solver/source/multigrid.cu:350-662):
// Galerkin coarse operator P^T A P with piecewise-constant P, restriction by
// summing fine residuals per agglomerate, prolongation by injection,
// weighted-Jacobi smoothing (jacobiRow, multigrid.cu:447-484). B200 design:
//   * no atomics: the Galerkin sums and the restriction are gathers over
//     host-built member / slot lists in ascending fine order (bit-reproducible);
//   * the fine residual is a coalesced pass over the fine level; the gather of
//     the coarse right-hand side also performs the coarse level's first
//     pre-smoothing sweep (from x = 0 it needs no neighbour values);
//   * every level at or below 1024 cells runs as ONE single-CTA kernel holding
//     x, the Jacobi partner, b and the residual in shared memory, with the
//     coefficients L1-resident and the coarsest rows in registers (the
//     reference launches three to four kernels per level per cycle there).
// Every kernel is a template on the value type: double for the FP64 path
// (compiled with --fmad=false, bit-exact with the CPU oracle), float for the
// inner cycles of the mixed-precision path.
#include <cmath>

#include "kernels.hpp"

namespace axisim {

namespace {

constexpr int kThreads = 256;
constexpr int kTailThreads = 1024;  // tail levels hold at most this many cells: one row per thread
constexpr int kRegW = 16;

inline int blocksFor(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }
// Threads per CTA for a level's kernels: its tuned block size, else kThreads
// (the kernels' launch bound).
template <class T>
inline int tpb(const LevelT<T>& L) {
    return (L.block >= 32 && L.block <= kThreads && L.block % 32 == 0) ? L.block : kThreads;
}

template <class T>
__device__ __forceinline__ T tiny();
template <>
__device__ __forceinline__ double tiny<double>() {
    return 1.0e-30;
}
template <>
__device__ __forceinline__ float tiny<float>() {
    return 1.0e-30f;
}

struct Slots {
    int base, stride, width;
};

template <class T>
__device__ __forceinline__ Slots slotsOf(const LevelT<T>& L, int n) {
    if (L.sliceOff) {
        const int s = n >> 5;
        const int o = L.sliceOff[s];
        return Slots{o + (n & 31), 32, (L.sliceOff[s + 1] - o) >> 5};
    }
    return Slots{n, L.N, L.W};
}

// A row's A x in the reference's order (AC x_n first, then the slots in
// order; jacobiTest: a slot counts when its neighbour is not -1, as jacobiRow
// tests it, else when it is >= 0, as residualRaw does). Every slot's neighbour
// and coefficient, and then every neighbour value, is loaded before the sum
// starts, eight slots at a time, so a row waits for two or three load
// latencies instead of one per slot; the arithmetic is unchanged.
template <class T>
__device__ __forceinline__ T axEager(const LevelT<T>& L, int n, const T* x, bool jacobiTest) {
    const Slots sl = slotsOf(L, n);
    T Ax = L.AC[n] * x[n];
    constexpr int kU = 8;
    for (int j0 = 0; j0 < sl.width; j0 += kU) {
        int k[kU];
        T a[kU], g[kU];
#pragma unroll
        for (int j = 0; j < kU; j++) {
            if (j0 + j < sl.width) {
                const int p = sl.base + (j0 + j) * sl.stride;
                k[j] = __ldg(L.nb + p);
                a[j] = __ldg(L.AF + p);
            } else {
                k[j] = -1;
                a[j] = T(0);
            }
        }
#pragma unroll
        for (int j = 0; j < kU; j++) g[j] = x[k[j] >= 0 ? k[j] : n];
#pragma unroll
        for (int j = 0; j < kU; j++)
            if (jacobiTest ? (k[j] != -1) : (k[j] >= 0)) Ax += a[j] * g[j];
    }
    return Ax;
}

// Weighted Jacobi row, jacobiRow (multigrid.cu:447-484).
template <class T>
__device__ __forceinline__ T jacobiRow(const LevelT<T>& L, int n, const T* xo, T w, T bn) {
    const T ac = L.AC[n];
    if (fabs(ac) < tiny<T>()) return xo[n];
    const T Ax = axEager(L, n, xo, true);
    return xo[n] + w * (bn - Ax) / ac;
}

// residualRaw with sign (residuals.cuh:17-48)
template <class T>
__device__ __forceinline__ T residualRow(const LevelT<T>& L, int n, const T* x, T bn) {
    return bn - axEager(L, n, x, false);
}

template <class T>
__device__ __forceinline__ T jacobiRowT(const LevelT<T>& L, int n, const T* xo, T w, T bn) {
    return jacobiRow(L, n, xo, w, bn);
}

// Level 0 ([W][N] slots, W fixed at compile time): loads issued before gathers.
template <class T, int WC>
__device__ __forceinline__ T ellAx(const LevelT<T>& L, int n, const T* x, bool jacobiTest) {
    int k[WC];
    T a[WC], g[WC];
    segNeighbours<WC>(L.seg, L.nb, L.N, n, k);
#pragma unroll
    for (int j = 0; j < WC; j++) a[j] = L.AF[(size_t)j * L.N + n];
#pragma unroll
    for (int j = 0; j < WC; j++) g[j] = x[k[j] >= 0 ? k[j] : n];
    T Ax = L.AC[n] * x[n];
#pragma unroll
    for (int j = 0; j < WC; j++)
        if (jacobiTest ? (k[j] != -1) : (k[j] >= 0)) Ax += a[j] * g[j];
    return Ax;
}

template <class T, int WC>
__global__ void __launch_bounds__(kThreads) k_mg_smooth_ell(const Ctl* ctl, LevelT<T> L, const T* __restrict__ x,
                                                            T* __restrict__ y, T w) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const T ac = L.AC[n];
    if (fabs(ac) < tiny<T>()) {
        y[n] = x[n];
        return;
    }
    const T Ax = ellAx<T, WC>(L, n, x, true);
    y[n] = x[n] + w * (L.b[n] - Ax) / ac;
}

// Prolongation fused into the first post-smoothing sweep on an ELL level:
// x' = x + s P e is formed on the fly for the cell and its neighbours, and
// y = x' + w (b - A x') / A_C, with the expressions and their order of the
// separate prolongation and sweep kernels, so the result is the same bit for
// bit; x' itself is never stored (one pass over x instead of three).
// With upd (the mixed cycle's last finest-level pass), the FP64 iterate the
// cycle corrects is updated in the same pass, upd[n] += (double)y[n], the
// arithmetic of the separate refinement update.
template <class T, int WC>
__global__ void __launch_bounds__(kThreads) k_mg_prolong_smooth_ell(const Ctl* ctl, LevelT<T> L,
                                                                    const T* __restrict__ x,
                                                                    const T* __restrict__ xc, T* __restrict__ y,
                                                                    T w, T scale, double* __restrict__ upd) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const int32_t* __restrict__ c2c = L.c2c;
    const T xn = x[n] + scale * xc[c2c[n]];
    const T ac = L.AC[n];
    if (fabs(ac) < tiny<T>()) {
        y[n] = xn;
        if (upd) upd[n] += (double)xn;
        return;
    }
    int k[WC];
    T a[WC], g[WC];
    segNeighbours<WC>(L.seg, L.nb, L.N, n, k);
#pragma unroll
    for (int j = 0; j < WC; j++) a[j] = L.AF[(size_t)j * L.N + n];
#pragma unroll
    for (int j = 0; j < WC; j++) {
        const int m = k[j] >= 0 ? k[j] : n;
        g[j] = x[m] + scale * xc[c2c[m]];
    }
    T Ax = L.AC[n] * xn;
#pragma unroll
    for (int j = 0; j < WC; j++)
        if (k[j] != -1) Ax += a[j] * g[j];
    const T yn = xn + w * (L.b[n] - Ax) / ac;
    y[n] = yn;
    if (upd) upd[n] += (double)yn;
}

template <class T, int WC>
__global__ void __launch_bounds__(kThreads) k_mg_residual_ell(const Ctl* ctl, LevelT<T> L, const T* __restrict__ x) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    L.res[n] = L.b[n] - ellAx<T, WC>(L, n, x, false);
}

// A terminal cell of a batch level (its case's coarsest level) keeps its value.
template <class T>
__device__ __forceinline__ bool frozen(const LevelT<T>& L, int n) {
    return L.nTerm > 0 && L.c2c[n] < 0;
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_smooth(const Ctl* ctl, LevelT<T> L, const T* __restrict__ x,
                                                        T* __restrict__ y, T w) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    y[n] = frozen(L, n) ? x[n] : jacobiRow(L, n, x, w, L.b[n]);
}

// Coarsest-level sweeps of the terminal cases of a batch level, one CTA per
// case: from zero, `sweeps` weighted-Jacobi sweeps (jacobiRow's arithmetic)
// with both iterates in shared memory, as the case's standalone coarsest
// level runs them. A case's neighbours all lie inside its range.
template <class T>
__device__ __forceinline__ void terminalBody(const LevelT<T>& L, T* x, T w, int sweeps, int r, unsigned char* smraw) {
    const int s0 = L.term[2 * r], n1 = L.term[2 * r + 1];
    const int m = n1 - s0;
    T* xo = reinterpret_cast<T*>(smraw);
    T* xn = xo + m;
    for (int i = threadIdx.x; i < m; i += blockDim.x) xo[i] = T(0);
    __syncthreads();
    for (int it = 0; it < sweeps; it++) {
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const int n = s0 + i;
            const T ac = L.AC[n];
            if (fabs(ac) < tiny<T>()) {
                xn[i] = xo[i];
                continue;
            }
            T Ax = ac * xo[i];
            const Slots sl = slotsOf(L, n);
            constexpr int kU = 8;
            for (int j0 = 0; j0 < sl.width; j0 += kU) {  // loads first, sums in slot order
                int k[kU];
                T a[kU], g[kU];
#pragma unroll
                for (int j = 0; j < kU; j++) {
                    if (j0 + j < sl.width) {
                        const int p = sl.base + (j0 + j) * sl.stride;
                        k[j] = __ldg(L.nb + p);
                        a[j] = __ldg(L.AF + p);
                    } else {
                        k[j] = -1;
                        a[j] = T(0);
                    }
                }
#pragma unroll
                for (int j = 0; j < kU; j++) g[j] = xo[k[j] >= 0 ? k[j] - s0 : i];
#pragma unroll
                for (int j = 0; j < kU; j++)
                    if (k[j] != -1) Ax += a[j] * g[j];
            }
            xn[i] = xo[i] + w * (L.b[n] - Ax) / ac;
        }
        __syncthreads();
        T* t = xo;
        xo = xn;
        xn = t;
    }
    for (int i = threadIdx.x; i < m; i += blockDim.x) x[s0 + i] = xo[i];
}

template <class T>
__global__ void k_mg_terminal(const Ctl* ctl, LevelT<T> L, T* x, T w, int sweeps) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    terminalBody(L, x, w, sweeps, (int)blockIdx.x, smraw);
}

// `sweeps` sweeps of a whole level inside one CTA, both iterates in shared memory.
template <class T>
__device__ __forceinline__ void smoothBlockBody(const LevelT<T>& L, T* x, T w, int sweeps, unsigned char* smraw) {
    T* xo = reinterpret_cast<T*>(smraw);
    T* xn = xo + L.N;
    for (int n = threadIdx.x; n < L.N; n += blockDim.x) xo[n] = x[n];
    __syncthreads();
    for (int it = 0; it < sweeps; it++) {
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) xn[n] = frozen(L, n) ? xo[n] : jacobiRow(L, n, xo, w, L.b[n]);
        __syncthreads();
        T* t = xo;
        xo = xn;
        xn = t;
    }
    for (int n = threadIdx.x; n < L.N; n += blockDim.x) x[n] = xo[n];
}

template <class T>
__global__ void k_mg_smooth_block(const Ctl* ctl, LevelT<T> L, T* x, T w, int sweeps) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    smoothBlockBody(L, x, w, sweeps, smraw);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_residual(const Ctl* ctl, LevelT<T> L, const T* __restrict__ x) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    L.res[n] = residualRow(L, n, x, L.b[n]);
}

// Restriction (multigrid.cu:398-410) as a gather; optionally the coarse
// level's first Jacobi sweep from x = 0: x1 = 0 + w (b - A 0) / AC.
template <class T>
__device__ __forceinline__ void gatherFinish(int c, const LevelT<T>& C, T* xCur, T* xAlt, int firstSweep, T w, T sum);

template <class T>
__device__ __forceinline__ void gatherCell(int c, const T* __restrict__ resFine, const LevelT<T>& C, T* xCur, T* xAlt,
                                           int firstSweep, T w) {
    T sum = T(0);
    for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += resFine[C.mList[q]];
    gatherFinish(c, C, xCur, xAlt, firstSweep, w, sum);
}

// The same restriction with each member's residual formed on the fly
// (residualRow's arithmetic, summed in ascending member order), so no
// separate residual pass over the fine level is needed.
template <class T>
__device__ __forceinline__ void gatherResCell(int c, const LevelT<T>& F, const T* __restrict__ xf, const LevelT<T>& C,
                                              T* xCur, T* xAlt, int firstSweep, T w) {
    T sum = T(0);
    const int q0 = C.mStart[c], q1 = C.mStart[c + 1];
    for (int q = q0; q < q1; q += 2) {  // two members' rows at once, summed in member order
        T r[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int m = (q + u < q1) ? C.mList[q + u] : -1;
            r[u] = (m >= 0) ? residualRow(F, m, xf, F.b[m]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 2; u++)
            if (q + u < q1) sum += r[u];
    }
    gatherFinish(c, C, xCur, xAlt, firstSweep, w, sum);
}

template <class T>
__device__ __forceinline__ void gatherFinish(int c, const LevelT<T>& C, T* xCur, T* xAlt, int firstSweep, T w, T sum) {
    C.b[c] = sum;
    if (!firstSweep) {
        xCur[c] = T(0);
        return;
    }
    const T ac = C.AC[c];
    xAlt[c] = (fabs(ac) < tiny<T>()) ? T(0) : T(0) + w * (sum - ac * T(0)) / ac;
}

// The restriction with residual, four lanes per coarse cell (aggregates hold
// four members almost everywhere): lane u of the cell's group forms the
// residual row of member q0 + 4k + u in round k, so the members' load chains
// run side by side instead of one after another. Every lane of the group then
// adds the four residuals in ascending member order to its own running sum,
// the order of gatherResCell, so the sum is the same bit for bit, and the
// group's first lane finishes the cell. Rounds are warp-uniform so every lane
// takes part in every shuffle. (The plain restriction of a stored residual
// keeps one thread per coarse cell: its two loads per member pipeline well.)
template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_gather_res4(const Ctl* ctl, LevelT<T> F, const T* __restrict__ xf,
                                                             LevelT<T> C, T* xCur, T* xAlt, int firstSweep, T w) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t >> 2, u = t & 3;
    const bool live = c < C.N;
    const int q0 = live ? C.mStart[c] : 0;
    const int q1 = live ? C.mStart[c + 1] : 0;
    const int rounds = __reduce_max_sync(0xFFFFFFFFu, (q1 - q0 + 3) >> 2);
    T sum = T(0);
    for (int k = 0; k < rounds; k++) {
        const int q = q0 + 4 * k + u;
        T r = T(0);
        if (q < q1) {
            const int m = C.mList[q];
            r = residualRow(F, m, xf, F.b[m]);
        }
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const T rv = __shfl_sync(0xFFFFFFFFu, r, v, 4);
            if (q0 + 4 * k + v < q1) sum += rv;
        }
    }
    if (live && u == 0) gatherFinish(c, C, xCur, xAlt, firstSweep, w, sum);
}

// Prolongation fused into the first post-smoothing sweep on any level layout:
// x' = x + s P e formed on the fly for the cell and its neighbours, then the
// weighted-Jacobi row of jacobiRow, so the result equals the separate
// prolongation and sweep bit for bit. A batch's terminal cell keeps its value.
template <class T>
__device__ __forceinline__ T prolongSmoothRow(const LevelT<T>& L, int n, const T* x, const T* xc, T w, T scale) {
    const int cn = L.c2c[n];
    if (cn < 0) return x[n];
    const T xn = x[n] + scale * xc[cn];
    const T ac = L.AC[n];
    if (fabs(ac) < tiny<T>()) return xn;
    T Ax = ac * xn;
    const Slots sl = slotsOf(L, n);
    constexpr int kU = 8;
    for (int j0 = 0; j0 < sl.width; j0 += kU) {  // loads first, eight slots at a time; sums in slot order
        int k[kU], ck[kU];
        T a[kU], gx[kU], gc[kU];
#pragma unroll
        for (int j = 0; j < kU; j++) {
            if (j0 + j < sl.width) {
                const int p = sl.base + (j0 + j) * sl.stride;
                k[j] = __ldg(L.nb + p);
                a[j] = __ldg(L.AF + p);
            } else {
                k[j] = -1;
                a[j] = T(0);
            }
        }
#pragma unroll
        for (int j = 0; j < kU; j++) {
            const int m = k[j] >= 0 ? k[j] : n;
            ck[j] = L.c2c[m];
            gx[j] = x[m];
        }
#pragma unroll
        for (int j = 0; j < kU; j++) gc[j] = xc[ck[j] >= 0 ? ck[j] : 0];
#pragma unroll
        for (int j = 0; j < kU; j++)
            if (k[j] != -1) Ax += a[j] * (ck[j] >= 0 ? gx[j] + scale * gc[j] : gx[j]);
    }
    return xn + w * (L.b[n] - Ax) / ac;
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_prolong_smooth(const Ctl* ctl, LevelT<T> L, const T* __restrict__ x,
                                                                const T* __restrict__ xc, T* __restrict__ y, T w,
                                                                T scale) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    y[n] = prolongSmoothRow(L, n, x, xc, w, scale);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_gather(const Ctl* ctl, const T* __restrict__ resFine, LevelT<T> C,
                                                        T* xCur, T* xAlt, int firstSweep, T w) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C.N) return;
    gatherCell(c, resFine, C, xCur, xAlt, firstSweep, w);
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_mg_prolong(const Ctl* ctl, int N, const int32_t* __restrict__ c2c, T* x,
                                                         const T* __restrict__ xc, T scale) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int c = c2c[n];
    if (c >= 0) x[n] += scale * xc[c];  // a batch's terminal cells have no coarse parent
}

// Galerkin (multigrid.cu:350-389) as gathers, one launch per level: thread t
// sums the fine slots feeding coarse slot t, and the first N threads also sum
// their members' diagonal contributions, each member's AC plus its
// agglomerate-internal off-diagonals in slot order (multigrid.cu:371-386).
// Sums run in the fine type and are stored in the coarse type.
template <class TF, bool NC = true>
__device__ __forceinline__ TF galDiag(const LevelT<TF>& F, int n) {
    TF diag = F.AC[n];
    const uint32_t mask = F.internalMask[n];
    const Slots sl = slotsOf(F, n);
    constexpr int kU = 8;
    for (int j0 = 0; j0 < sl.width; j0 += kU) {  // the slots' loads first, sums in slot order
        TF a[kU];
#pragma unroll
        for (int j = 0; j < kU; j++) {
            const TF* p = F.AF + sl.base + (j0 + j) * sl.stride;
            a[j] = (j0 + j < sl.width) ? (NC ? __ldg(p) : *p) : TF(0);
        }
#pragma unroll
        for (int j = 0; j < kU; j++)
            if (j0 + j < 32 && ((mask >> (j0 + j)) & 1u)) diag += a[j];
    }
    return diag;
}

// NC: the fine level's coefficients were written by an earlier kernel, so
// they may go through the read-only cache
template <class TF, class TC, bool NC>
__device__ __forceinline__ void galCoarseCell(const LevelT<TF>& F, const LevelT<TC>& C, int t) {
    if (t < C.totalSlots) {
        TF af = TF(0);
        for (int q = C.gStart[t]; q < C.gStart[t + 1]; q++) af += F.AF[C.gList[q]];
        C.AF[t] = (TC)af;
    }
    if (t < C.N) {
        TF ac = TF(0);
        const int q0 = C.mStart[t], q1 = C.mStart[t + 1];
        for (int q = q0; q < q1; q += 4) {  // four members' contributions at once, summed in member order
            TF d[4];
#pragma unroll
            for (int u = 0; u < 4; u++) d[u] = (q + u < q1) ? galDiag<TF, NC>(F, C.mList[q + u]) : TF(0);
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (q + u < q1) ac += d[u];
        }
        C.AC[t] = (TC)ac;
    }
}

template <class TF, class TC>
__global__ void __launch_bounds__(kThreads) k_gal_coarse(const Ctl* ctl, LevelT<TF> F, LevelT<TC> C) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    galCoarseCell<TF, TC, true>(F, C, blockIdx.x * blockDim.x + threadIdx.x);
}

// The tail levels' Galerkin in one CTA: a coarse level's operator is read as
// the next pair's fine level after the barrier (plain loads: it was written
// in this launch).
template <class T>
__global__ void __launch_bounds__(kTailThreads) k_gal_chain(const Ctl* ctl, GalChainArgsT<T> a) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    for (int i = 0; i + 1 < a.count; i++) {
        const LevelT<T>& F = a.lv[i];
        const LevelT<T>& C = a.lv[i + 1];
        const int n = C.totalSlots > C.N ? C.totalSlots : C.N;
        for (int t = threadIdx.x; t < n; t += blockDim.x) galCoarseCell<T, T, false>(F, C, t);
        __syncthreads();
    }
}

// ---------------- V-cycle tail inside one CTA ----------------
template <class T>
__device__ __forceinline__ void tailSmooth(const LevelT<T>& L, T*& xo, T*& xn, const T* b, T w, int sweeps) {
    for (int it = 0; it < sweeps; it++) {
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) xn[n] = jacobiRowT(L, n, xo, w, b[n]);
        __syncthreads();
        T* t = xo;
        xo = xn;
        xn = t;
    }
}

// Barrier of the first `threads` threads of the CTA (a multiple of 32):
// named barrier 1, or the warp's own barrier for a single warp.
__device__ __forceinline__ void groupSync(int threads) {
    if (threads <= 32) __syncwarp();
    else asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

template <class T, int RW>
__device__ __forceinline__ void tailCoarsestGroup(const LevelT<T>& L, T*& xo, T*& xn, const T* b, T w, int sweeps,
                                                  int group);

// Coarsest level with one row per thread held in registers. Only the warps
// that hold rows take part in the sweeps, synchronising among themselves (a
// CTA-wide barrier per sweep would wait on every warp of the CTA); the others
// go straight to the closing CTA barrier.
template <class T>
__device__ __forceinline__ void tailCoarsest(const LevelT<T>& L, T*& xo, T*& xn, const T* b, T w, int sweeps) {
    const int n = threadIdx.x;
    const int group = ((L.N + 31) / 32) * 32;  // threads of the warps holding rows (whole warps)
    if (n < group) {
        if (L.W <= 8) tailCoarsestGroup<T, 8>(L, xo, xn, b, w, sweeps, group);
        else tailCoarsestGroup<T, kRegW>(L, xo, xn, b, w, sweeps, group);
    }
    else if (sweeps & 1) {  // the same buffer roles as the sweeping warps end with
        T* t = xo;
        xo = xn;
        xn = t;
    }
    __syncthreads();
}

// RW register slots per row (the level's width at most). With eight, every
// neighbour value of a sweep is read before the row's ordered sum; with
// sixteen the reads stay inside the sum (the registers run out otherwise).
template <class T, int RW>
__device__ __forceinline__ void tailCoarsestGroup(const LevelT<T>& L, T*& xo, T*& xn, const T* b, T w, int sweeps,
                                                  int group) {
    const int n = threadIdx.x;
    const bool active = n < L.N;
    T af[RW];
    int nb[RW];
    int width = 0;
    T ac = T(0), bn = T(0);
    if (active) {
        const Slots sl = slotsOf(L, n);
        width = sl.width;
        for (int j = 0; j < RW; j++) {
            if (j < width) {
                af[j] = L.AF[sl.base + j * sl.stride];
                nb[j] = L.nb[sl.base + j * sl.stride];
            } else {
                af[j] = T(0);
                nb[j] = -1;
            }
        }
        ac = L.AC[n];
        bn = b[n];
    }
    const bool empty = fabs(ac) < tiny<T>();
    for (int it = 0; it < sweeps; it++) {
        if (active) {
            if (empty) {
                xn[n] = xo[n];
            } else {
                T Ax = ac * xo[n];
                if (RW <= 8) {
                    T g[RW];
#pragma unroll
                    for (int j = 0; j < RW; j++) g[j] = xo[nb[j] >= 0 ? nb[j] : n];
#pragma unroll
                    for (int j = 0; j < RW; j++)
                        if (j < width && nb[j] != -1) Ax += af[j] * g[j];
                } else {
#pragma unroll
                    for (int j = 0; j < RW; j++)
                        if (j < width && nb[j] != -1) Ax += af[j] * xo[nb[j]];
                }
                xn[n] = xo[n] + w * (bn - Ax) / ac;
            }
        }
        groupSync(group);
        T* t = xo;
        xo = xn;
        xn = t;
    }
}

template <class T>
__device__ __forceinline__ void tailBody(const TailArgsT<T>& a, unsigned char* smraw) {
    T* sm = reinterpret_cast<T*>(smraw);
    T* X[kMaxTail];
    T* Y[kMaxTail];
    T* B[kMaxTail];
    T* R[kMaxTail];
    for (int i = 0; i < a.count; i++) {
        const int N = a.lv[i].N;
        X[i] = sm + a.smemOff[i];
        Y[i] = X[i] + N;
        B[i] = Y[i] + N;
        R[i] = B[i] + N;
    }
    // restriction into the first tail level from the finer level's residual
    {
        const LevelT<T>& C = a.lv[0];
        for (int c = threadIdx.x; c < C.N; c += blockDim.x) {
            T sum = T(0);
            for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += a.resFine[C.mList[q]];
            B[0][c] = sum;
            X[0][c] = T(0);
        }
        __syncthreads();
    }
    const int last = a.count - 1;
    for (int i = 0; i < last; i++) {
        const LevelT<T>& L = a.lv[i];
        tailSmooth(L, X[i], Y[i], B[i], a.w, a.pre);
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) R[i][n] = B[i][n] - axEager(L, n, X[i], false);
        __syncthreads();
        const LevelT<T>& C = a.lv[i + 1];
        for (int c = threadIdx.x; c < C.N; c += blockDim.x) {
            T sum = T(0);
            for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += R[i][C.mList[q]];
            B[i + 1][c] = sum;
            X[i + 1][c] = T(0);
        }
        __syncthreads();
    }
    {
        const LevelT<T>& L = a.lv[last];
        if (L.N <= (int)blockDim.x && L.W <= kRegW) tailCoarsest(L, X[last], Y[last], B[last], a.w, a.coarseSweeps);
        else tailSmooth(L, X[last], Y[last], B[last], a.w, a.coarseSweeps);
    }
    for (int i = last - 1; i >= 0; i--) {
        const LevelT<T>& L = a.lv[i];
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) X[i][n] += a.prolongScale * X[i + 1][L.c2c[n]];
        __syncthreads();
        tailSmooth(L, X[i], Y[i], B[i], a.w, a.post);
    }
    for (int n = threadIdx.x; n < a.lv[0].N; n += blockDim.x) a.xOut[n] = X[0][n];
}

template <class T>
__global__ void __launch_bounds__(kTailThreads) k_mg_tail(const Ctl* ctl, TailArgsT<T> a) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    tailBody(a, smraw);
}

// ---------------- resident V-cycle (one cooperative kernel) ----------------
__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a cooperative grid: arrivals counted in Ctl::mgBar[0],
// the last arrival resets the count and advances the generation mgBar[1] that
// the others wait on. A wait gives up after one second of the GPU's global
// timer (sets Ctl::mgErr, and every later wait of the grid returns at once),
// so a grid whose CTAs do not all arrive ends with an error instead of
// hanging. Ctl::mgPhantom extra arrivals are expected (0; a test sets 1 to
// make the wait run out).
__device__ __forceinline__ void gridSync(Ctl* ctl) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = &ctl->mgBar[1];
        volatile int* err = &ctl->mgErr;
        const unsigned int g = *gen;
        __threadfence();
        if (atomicAdd(&ctl->mgBar[0], 1u) == gridDim.x - 1 + (unsigned int)ctl->mgPhantom) {
            atomicExch(&ctl->mgBar[0], 0u);
            __threadfence();
            atomicAdd(&ctl->mgBar[1], 1u);
        } else {
            const unsigned long long t0 = globalTimerNs();
            while (*gen == g && !*err) {
                if (globalTimerNs() - t0 > 1000000000ull) {
                    atomicExch(&ctl->mgErr, 1);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <class T>
__global__ void __launch_bounds__(kTailThreads, 1) k_mg_resident(Ctl* ctl, const __grid_constant__ ResidentArgsT<T> a) {
    // launched after its predecessor completes, and never lets its successor
    // start early: every CTA of this grid holds an SM until the last barrier
    if (ctl->done || ctl->ppSkip || ctl->mgErr) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (int i = 0; i < a.nOps; i++) {
        const MgOp& op = a.ops[i];
        const LevelT<T>& L = a.lv[op.level - a.first];
        switch (op.type) {
            case kOpSmooth: {
                const T* x = static_cast<const T*>(op.p0);
                T* y = static_cast<T*>(op.p1);
                for (int n = tid; n < L.N; n += stride) y[n] = frozen(L, n) ? x[n] : jacobiRow(L, n, x, a.w, L.b[n]);
                break;
            }
            case kOpSmoothBlock:
                if (blockIdx.x == 0) smoothBlockBody(L, static_cast<T*>(op.p0), a.w, op.ival, smraw);
                break;
            case kOpResidual: {
                const T* x = static_cast<const T*>(op.p0);
                for (int n = tid; n < L.N; n += stride) L.res[n] = residualRow(L, n, x, L.b[n]);
                break;
            }
            case kOpGather: {
                const T* resFine = a.lv[op.level - 1 - a.first].res;
                for (int c = tid; c < L.N; c += stride)
                    gatherCell(c, resFine, L, static_cast<T*>(op.p0), static_cast<T*>(op.p1), op.ival, a.w);
                break;
            }
            case kOpTerminal:
                for (int r = blockIdx.x; r < L.nTerm; r += gridDim.x)
                    terminalBody(L, static_cast<T*>(op.p0), a.w, op.ival, r, smraw);
                break;
            case kOpProlong: {
                T* x = static_cast<T*>(op.p0);
                const T* xc = static_cast<const T*>(op.p1);
                const T sc = (T)op.scale;
                for (int n = tid; n < L.N; n += stride) {
                    const int c = L.c2c[n];
                    if (c >= 0) x[n] += sc * xc[c];
                }
                break;
            }
            case kOpGatherRes: {
                const LevelT<T>& F = a.lv[op.level - 1 - a.first];
                for (int c = tid; c < L.N; c += stride)
                    gatherResCell(c, F, static_cast<const T*>(op.p2), L, static_cast<T*>(op.p0),
                                  static_cast<T*>(op.p1), op.ival, a.w);
                break;
            }
            case kOpProlongSmooth: {
                const T* x = static_cast<const T*>(op.p0);
                const T* xc = static_cast<const T*>(op.p1);
                T* y = static_cast<T*>(op.p2);
                const T sc = (T)op.scale;
                for (int n = tid; n < L.N; n += stride) y[n] = prolongSmoothRow(L, n, x, xc, a.w, sc);
                break;
            }
            case kOpTail:
                if (blockIdx.x == 0) tailBody(a.tail, smraw);
                break;
            default:
                break;
        }
        if (i + 1 < a.nOps) gridSync(ctl);
    }
}

}  // namespace

template <class TF, class TC>
void launchGalerkin(const Ctl* ctl, const LevelT<TF>& fine, const LevelT<TC>& coarse, cudaStream_t s) {
    const int n = coarse.totalSlots > coarse.N ? coarse.totalSlots : coarse.N;
    launchPDL(k_gal_coarse<TF, TC>, dim3(blocksFor(n)), dim3(kThreads), 0, s, ctl, fine, coarse);
}

template <class T>
void launchGalerkinChain(const Ctl* ctl, const GalChainArgsT<T>& a, cudaStream_t s) {
    launchPDL(k_gal_chain<T>, dim3(1), dim3(kTailThreads), 0, s, ctl, a);
}

template <class T>
void launchMGSmooth(const Ctl* ctl, const LevelT<T>& L, const T* x, T* y, T w, cudaStream_t s) {
    const int t = tpb(L);
    if (!L.sliceOff && L.W == 4) launchPDL(k_mg_smooth_ell<T, 4>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x, y, w);
    else if (!L.sliceOff && L.W == 3) launchPDL(k_mg_smooth_ell<T, 3>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x, y, w);
    else launchPDL(k_mg_smooth<T>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x, y, w);
}

template <class T>
void launchMGSmoothBlock(const Ctl* ctl, const LevelT<T>& L, T* x, T w, int sweeps, cudaStream_t s) {
    const int threads = L.N < 1024 ? ((L.N + 31) / 32) * 32 : 1024;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mg_smooth_block<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    launchPDL(k_mg_smooth_block<T>, dim3(1), dim3(threads), 2 * (size_t)L.N * sizeof(T), s, ctl, L, x, w, sweeps);
}

template <class T>
void launchMGResidual(const Ctl* ctl, const LevelT<T>& L, const T* x, cudaStream_t s) {
    const int t = tpb(L);
    if (!L.sliceOff && L.W == 4) launchPDL(k_mg_residual_ell<T, 4>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x);
    else if (!L.sliceOff && L.W == 3) launchPDL(k_mg_residual_ell<T, 3>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x);
    else launchPDL(k_mg_residual<T>, dim3(blocksFor(L.N, t)), dim3(t), 0, s, ctl, L, x);
}

template <class T>
void launchMGGather(const Ctl* ctl, const LevelT<T>& fine, const LevelT<T>& coarse, T* xCur, T* xAlt, int firstSweep,
                    T w, cudaStream_t s) {
    const int t = tpb(coarse);
    launchPDL(k_mg_gather<T>, dim3(blocksFor(coarse.N, t)), dim3(t), 0, s, ctl, fine.res, coarse, xCur, xAlt,
              firstSweep, w);
}

template <class T>
void launchMGGatherRes(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const LevelT<T>& coarse, T* xCur,
                       T* xAlt, int firstSweep, T w, cudaStream_t s) {
    const int t = tpb(coarse);  // a multiple of 32: a cell's four lanes share a warp
    launchPDL(k_mg_gather_res4<T>, dim3(blocksFor(4LL * coarse.N, t)), dim3(t), 0, s, ctl, fine, xFine, coarse, xCur,
              xAlt, firstSweep, w);
}

template <class T>
void launchMGProlongSmoothAny(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const T* xCoarse, T* y, T w,
                              T scale, cudaStream_t s) {
    const int t = tpb(fine);
    launchPDL(k_mg_prolong_smooth<T>, dim3(blocksFor(fine.N, t)), dim3(t), 0, s, ctl, fine, xFine, xCoarse, y, w,
              scale);
}

template <class T>
void launchMGProlong(const Ctl* ctl, const LevelT<T>& fine, T* xFine, const T* xCoarse, T scale, cudaStream_t s) {
    const int t = tpb(fine);
    launchPDL(k_mg_prolong<T>, dim3(blocksFor(fine.N, t)), dim3(t), 0, s, ctl, fine.N, fine.c2c, xFine, xCoarse,
              scale);
}

template <class T>
bool launchMGProlongSmooth(const Ctl* ctl, const LevelT<T>& fine, const T* xFine, const T* xCoarse, T* y, T w,
                           T scale, cudaStream_t s, double* upd) {
    if (fine.sliceOff || !fine.c2c) return false;
    const int t = tpb(fine);
    if (fine.W == 4)
        launchPDL(k_mg_prolong_smooth_ell<T, 4>, dim3(blocksFor(fine.N, t)), dim3(t), 0, s, ctl, fine, xFine,
                  xCoarse, y, w, scale, upd);
    else if (fine.W == 3)
        launchPDL(k_mg_prolong_smooth_ell<T, 3>, dim3(blocksFor(fine.N, t)), dim3(t), 0, s, ctl, fine, xFine,
                  xCoarse, y, w, scale, upd);
    else
        return false;
    return true;
}

template <class T>
void launchMGTerminal(const Ctl* ctl, const LevelT<T>& L, T* x, T w, int sweeps, cudaStream_t s) {
    if (L.nTerm <= 0) return;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mg_terminal<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    const int threads = L.termMax < 256 ? ((L.termMax + 31) / 32) * 32 : 256;
    launchPDL(k_mg_terminal<T>, dim3(L.nTerm), dim3(threads), 2 * (size_t)L.termMax * sizeof(T), s, ctl, L, x, w,
              sweeps);
}

template <class T>
bool launchMGResident(Ctl* ctl, const ResidentArgsT<T>& a, cudaStream_t s) {
    if (a.nOps <= 0 || a.smem > 200 * 1024) return false;
    static int grid = -1;
    if (grid < 0) {
        grid = 0;
        int dev = 0, sms = 0, coop = 0, perSM = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
            cudaFuncSetAttribute(k_mg_resident<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
                cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_mg_resident<T>, kTailThreads, 200 * 1024) ==
                cudaSuccess &&
            perSM >= 1)
            grid = sms;  // one CTA per SM: every CTA resident at once
        cudaGetLastError();
    }
    if (grid <= 0) return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = a.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    tNextLaunchPlain = false;
    return cudaLaunchKernelEx(&cfg, k_mg_resident<T>, ctl, a) == cudaSuccess;
}

template <class T>
size_t tailSharedBytes(const TailArgsT<T>& a) {
    size_t d = 0;
    for (int i = 0; i < a.count; i++) d += 4 * (size_t)a.lv[i].N;
    return d * sizeof(T);
}

template <class T>
void launchMGTail(const Ctl* ctl, const TailArgsT<T>& a, cudaStream_t s) {
    const size_t smem = tailSharedBytes(a);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mg_tail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    launchPDL(k_mg_tail<T>, dim3(1), dim3(kTailThreads), smem, s, ctl, a);
}

// explicit instantiations: FP64 path, mixed-precision cycle
template void launchGalerkin<double, double>(const Ctl*, const LevelT<double>&, const LevelT<double>&, cudaStream_t);
template void launchGalerkin<double, float>(const Ctl*, const LevelT<double>&, const LevelT<float>&, cudaStream_t);
template void launchGalerkin<float, float>(const Ctl*, const LevelT<float>&, const LevelT<float>&, cudaStream_t);
template void launchGalerkinChain<double>(const Ctl*, const GalChainArgsT<double>&, cudaStream_t);
template void launchGalerkinChain<float>(const Ctl*, const GalChainArgsT<float>&, cudaStream_t);
#define AXISIM_MG_INSTANTIATE(T)                                                                               \
    template void launchMGSmooth<T>(const Ctl*, const LevelT<T>&, const T*, T*, T, cudaStream_t);               \
    template void launchMGSmoothBlock<T>(const Ctl*, const LevelT<T>&, T*, T, int, cudaStream_t);               \
    template void launchMGResidual<T>(const Ctl*, const LevelT<T>&, const T*, cudaStream_t);                    \
    template void launchMGGather<T>(const Ctl*, const LevelT<T>&, const LevelT<T>&, T*, T*, int, T, cudaStream_t); \
    template void launchMGProlong<T>(const Ctl*, const LevelT<T>&, T*, const T*, T, cudaStream_t);                 \
    template bool launchMGProlongSmooth<T>(const Ctl*, const LevelT<T>&, const T*, const T*, T*, T, T, cudaStream_t, \
                                           double*);                                                             \
    template void launchMGTerminal<T>(const Ctl*, const LevelT<T>&, T*, T, int, cudaStream_t);                  \
    template bool launchMGResident<T>(Ctl*, const ResidentArgsT<T>&, cudaStream_t);                              \
    template void launchMGGatherRes<T>(const Ctl*, const LevelT<T>&, const T*, const LevelT<T>&, T*, T*, int, T,     \
                                       cudaStream_t);                                                            \
    template void launchMGProlongSmoothAny<T>(const Ctl*, const LevelT<T>&, const T*, const T*, T*, T, T,          \
                                              cudaStream_t);                                                     \
    template size_t tailSharedBytes<T>(const TailArgsT<T>&);                                                   \
    template void launchMGTail<T>(const Ctl*, const TailArgsT<T>&, cudaStream_t);
AXISIM_MG_INSTANTIATE(double)
AXISIM_MG_INSTANTIATE(float)
#undef AXISIM_MG_INSTANTIATE

}  // namespace axisim
