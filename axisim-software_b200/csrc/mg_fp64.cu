// mg_fp64.cu -- agglomeration multigrid V-cycle for the pressure correction (FP64, sm_100a).
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
// Compiled with --fmad=false like the rest of the FP64 path.
#include <cmath>

#include "kernels.hpp"

namespace axisim {

namespace {

constexpr int kThreads = 256;
constexpr int kTailThreads = 1024;
// tail levels are at most kTailThreads cells: one row per thread
constexpr int kRegW = 16;

inline int blocksFor(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

struct Slots {
    int base, stride, width;
};

__device__ __forceinline__ Slots slotsOf(const LevelDev& L, int n) {
    if (L.sliceOff) {
        const int s = n >> 5;
        const int o = L.sliceOff[s];
        return Slots{o + (n & 31), 32, (L.sliceOff[s + 1] - o) >> 5};
    }
    return Slots{n, L.N, L.W};
}

// Weighted Jacobi row, jacobiRow (multigrid.cu:447-484). Slot loads are
// issued before the neighbour gathers; a slot without a neighbour reads the
// cell itself and is skipped in the sum.
__device__ __forceinline__ double jacobiRowT(const LevelDev& L, int n, const double* xo, double w, double bn) {
    const double ac = L.AC[n];
    if (fabs(ac) < 1.0e-30) return xo[n];
    const Slots sl = slotsOf(L, n);
    double Ax = ac * xo[n];
    constexpr int kU = 8;
    for (int j0 = 0; j0 < sl.width; j0 += kU) {
        int k[kU];
        double a[kU], g[kU];
#pragma unroll
        for (int j = 0; j < kU; j++) {
            if (j0 + j < sl.width) {
                const int p = sl.base + (j0 + j) * sl.stride;
                k[j] = __ldg(L.nb + p);
                a[j] = __ldg(L.AF + p);
            } else {
                k[j] = -1;
                a[j] = 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < kU; j++) g[j] = xo[k[j] != -1 ? k[j] : n];
#pragma unroll
        for (int j = 0; j < kU; j++)
            if (k[j] != -1) Ax += a[j] * g[j];
    }
    return xo[n] + w * (bn - Ax) / ac;
}

// residualRaw with sign (residuals.cuh:17-48)
__device__ __forceinline__ double residualRowT(const LevelDev& L, int n, const double* x, double bn) {
    const Slots sl = slotsOf(L, n);
    double Ax = L.AC[n] * x[n];
    constexpr int kU = 8;
    for (int j0 = 0; j0 < sl.width; j0 += kU) {
        int k[kU];
        double a[kU], g[kU];
#pragma unroll
        for (int j = 0; j < kU; j++) {
            if (j0 + j < sl.width) {
                const int p = sl.base + (j0 + j) * sl.stride;
                k[j] = __ldg(L.nb + p);
                a[j] = __ldg(L.AF + p);
            } else {
                k[j] = -1;
                a[j] = 0.0;
            }
        }
#pragma unroll
        for (int j = 0; j < kU; j++) g[j] = x[k[j] >= 0 ? k[j] : n];
#pragma unroll
        for (int j = 0; j < kU; j++)
            if (k[j] >= 0) Ax += a[j] * g[j];
    }
    return bn - Ax;
}

// Plain rows for the multi-CTA sweeps (bandwidth-bound: occupancy first).
__device__ __forceinline__ double jacobiRow(const LevelDev& L, int n, const double* xo, double w, double bn) {
    const double ac = L.AC[n];
    if (fabs(ac) < 1.0e-30) return xo[n];
    double Ax = ac * xo[n];
    const Slots sl = slotsOf(L, n);
    for (int j = 0; j < sl.width; j++) {
        const int p = sl.base + j * sl.stride;
        const int k = L.nb[p];
        if (k != -1) Ax += L.AF[p] * xo[k];
    }
    return xo[n] + w * (bn - Ax) / ac;
}

__device__ __forceinline__ double residualRow(const LevelDev& L, int n, const double* x, double bn) {
    double Ax = L.AC[n] * x[n];
    const Slots sl = slotsOf(L, n);
    for (int j = 0; j < sl.width; j++) {
        const int p = sl.base + j * sl.stride;
        const int k = L.nb[p];
        if (k >= 0) Ax += L.AF[p] * x[k];
    }
    return bn - Ax;
}

// Level 0 ([W][N] slots, W fixed at compile time): loads issued before gathers.
template <int WC>
__device__ __forceinline__ double ellAx(const LevelDev& L, int n, const double* x, bool jacobiTest) {
    int k[WC];
    double a[WC], g[WC];
#pragma unroll
    for (int j = 0; j < WC; j++) {
        k[j] = L.nb[(size_t)j * L.N + n];
        a[j] = L.AF[(size_t)j * L.N + n];
    }
#pragma unroll
    for (int j = 0; j < WC; j++) g[j] = x[k[j] >= 0 ? k[j] : n];
    double Ax = L.AC[n] * x[n];
#pragma unroll
    for (int j = 0; j < WC; j++)
        if (jacobiTest ? (k[j] != -1) : (k[j] >= 0)) Ax += a[j] * g[j];
    return Ax;
}

template <int WC>
__global__ void __launch_bounds__(kThreads) k_mg_smooth_ell(const Ctl* ctl, LevelDev L, const double* __restrict__ x,
                                                            double* __restrict__ y, double w) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const double ac = L.AC[n];
    if (fabs(ac) < 1.0e-30) {
        y[n] = x[n];
        return;
    }
    const double Ax = ellAx<WC>(L, n, x, true);
    y[n] = x[n] + w * (L.b[n] - Ax) / ac;
}

template <int WC>
__global__ void __launch_bounds__(kThreads) k_mg_residual_ell(const Ctl* ctl, LevelDev L, const double* __restrict__ x) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    L.res[n] = L.b[n] - ellAx<WC>(L, n, x, false);
}

__global__ void __launch_bounds__(kThreads) k_mg_smooth(const Ctl* ctl, LevelDev L, const double* __restrict__ x,
                                                        double* __restrict__ y, double w) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    y[n] = jacobiRow(L, n, x, w, L.b[n]);
}

__global__ void k_mg_smooth_block(const Ctl* ctl, LevelDev L, double* x, double w, int sweeps) {
    if (ctl->done) return;
    extern __shared__ double sx[];
    double* xo = sx;
    double* xn = sx + L.N;
    for (int n = threadIdx.x; n < L.N; n += blockDim.x) xo[n] = x[n];
    __syncthreads();
    for (int it = 0; it < sweeps; it++) {
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) xn[n] = jacobiRow(L, n, xo, w, L.b[n]);
        __syncthreads();
        double* t = xo;
        xo = xn;
        xn = t;
    }
    for (int n = threadIdx.x; n < L.N; n += blockDim.x) x[n] = xo[n];
}

__global__ void __launch_bounds__(kThreads) k_mg_residual(const Ctl* ctl, LevelDev L, const double* __restrict__ x) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    L.res[n] = residualRow(L, n, x, L.b[n]);
}

// Restriction (multigrid.cu:398-410) as a gather; optionally the coarse
// level's first Jacobi sweep from x = 0: x1 = 0 + w (b - A 0) / AC.
__global__ void __launch_bounds__(kThreads) k_mg_gather(const Ctl* ctl, const double* __restrict__ resFine,
                                                        LevelDev C, double* xCur, double* xAlt, int firstSweep,
                                                        double w) {
    if (ctl->done) return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C.N) return;
    double sum = 0.0;
    for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += resFine[C.mList[q]];
    C.b[c] = sum;
    if (!firstSweep) {
        xCur[c] = 0.0;
        return;
    }
    const double ac = C.AC[c];
    xAlt[c] = (fabs(ac) < 1.0e-30) ? 0.0 : 0.0 + w * (sum - ac * 0.0) / ac;
}

__global__ void __launch_bounds__(kThreads) k_mg_prolong(const Ctl* ctl, int N, const int32_t* __restrict__ c2c,
                                                         double* x, const double* __restrict__ xc) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    x[n] += xc[c2c[n]];
}

// Galerkin, step 1 (coalesced over fine cells): each row's contribution to
// its coarse diagonal, AC plus the agglomerate-internal off-diagonals in slot
// order (multigrid.cu:371-386).
__global__ void __launch_bounds__(kThreads) k_gal_diag(const Ctl* ctl, LevelDev F) {
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= F.N) return;
    double diag = F.AC[n];
    uint32_t mask = F.internalMask[n];
    const Slots sl = slotsOf(F, n);
    while (mask) {
        const int j = __ffs(mask) - 1;
        mask &= mask - 1;
        diag += F.AF[sl.base + j * sl.stride];
    }
    F.res[n] = diag;
}

// Galerkin, step 2: one thread per coarse slot sums its feeding fine slots;
// the first N threads also sum their members' diagonal contributions.
__global__ void __launch_bounds__(kThreads) k_gal_coarse(const Ctl* ctl, LevelDev F, LevelDev C) {
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < C.totalSlots) {
        double af = 0.0;
        for (int q = C.gStart[t]; q < C.gStart[t + 1]; q++) af += F.AF[C.gList[q]];
        C.AF[t] = af;
    }
    if (t < C.N) {
        double ac = 0.0;
        for (int q = C.mStart[t]; q < C.mStart[t + 1]; q++) ac += F.res[C.mList[q]];
        C.AC[t] = ac;
    }
}

// ---------------- V-cycle tail inside one CTA ----------------
__device__ __forceinline__ void tailSmooth(const LevelDev& L, double*& xo, double*& xn, const double* b, double w,
                                           int sweeps) {
    for (int it = 0; it < sweeps; it++) {
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) xn[n] = jacobiRowT(L, n, xo, w, b[n]);
        __syncthreads();
        double* t = xo;
        xo = xn;
        xn = t;
    }
}

// Coarsest level with one row per thread held in registers.
__device__ __forceinline__ void tailCoarsest(const LevelDev& L, double*& xo, double*& xn, const double* b, double w,
                                             int sweeps) {
    const int n = threadIdx.x;
    const bool active = n < L.N;
    double af[kRegW];
    int nb[kRegW];
    int width = 0;
    double ac = 0.0, bn = 0.0;
    if (active) {
        const Slots sl = slotsOf(L, n);
        width = sl.width;
        for (int j = 0; j < kRegW; j++) {
            if (j < width) {
                af[j] = L.AF[sl.base + j * sl.stride];
                nb[j] = L.nb[sl.base + j * sl.stride];
            } else {
                af[j] = 0.0;
                nb[j] = -1;
            }
        }
        ac = L.AC[n];
        bn = b[n];
    }
    const bool empty = fabs(ac) < 1.0e-30;
    for (int it = 0; it < sweeps; it++) {
        if (active) {
            if (empty) {
                xn[n] = xo[n];
            } else {
                double Ax = ac * xo[n];
#pragma unroll
                for (int j = 0; j < kRegW; j++)
                    if (j < width && nb[j] != -1) Ax += af[j] * xo[nb[j]];
                xn[n] = xo[n] + w * (bn - Ax) / ac;
            }
        }
        __syncthreads();
        double* t = xo;
        xo = xn;
        xn = t;
    }
}

__global__ void __launch_bounds__(kTailThreads) k_mg_tail(const Ctl* ctl, TailArgs a) {
    if (ctl->done) return;
    extern __shared__ double sm[];
    double* X[kMaxTail];
    double* Y[kMaxTail];
    double* B[kMaxTail];
    double* R[kMaxTail];
    for (int i = 0; i < a.count; i++) {
        const int N = a.lv[i].N;
        X[i] = sm + a.smemOff[i];
        Y[i] = X[i] + N;
        B[i] = Y[i] + N;
        R[i] = B[i] + N;
    }
    // restriction into the first tail level from the finer level's residual
    {
        const LevelDev& C = a.lv[0];
        for (int c = threadIdx.x; c < C.N; c += blockDim.x) {
            double sum = 0.0;
            for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += a.resFine[C.mList[q]];
            B[0][c] = sum;
            X[0][c] = 0.0;
        }
        __syncthreads();
    }
    const int last = a.count - 1;
    for (int i = 0; i < last; i++) {
        const LevelDev& L = a.lv[i];
        tailSmooth(L, X[i], Y[i], B[i], a.w, a.pre);
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) R[i][n] = residualRowT(L, n, X[i], B[i][n]);
        __syncthreads();
        const LevelDev& C = a.lv[i + 1];
        for (int c = threadIdx.x; c < C.N; c += blockDim.x) {
            double sum = 0.0;
            for (int q = C.mStart[c]; q < C.mStart[c + 1]; q++) sum += R[i][C.mList[q]];
            B[i + 1][c] = sum;
            X[i + 1][c] = 0.0;
        }
        __syncthreads();
    }
    {
        const LevelDev& L = a.lv[last];
        if (L.N <= (int)blockDim.x && L.W <= kRegW) tailCoarsest(L, X[last], Y[last], B[last], a.w, a.coarseSweeps);
        else tailSmooth(L, X[last], Y[last], B[last], a.w, a.coarseSweeps);
    }
    for (int i = last - 1; i >= 0; i--) {
        const LevelDev& L = a.lv[i];
        for (int n = threadIdx.x; n < L.N; n += blockDim.x) X[i][n] += X[i + 1][L.c2c[n]];
        __syncthreads();
        tailSmooth(L, X[i], Y[i], B[i], a.w, a.post);
    }
    for (int n = threadIdx.x; n < a.lv[0].N; n += blockDim.x) a.xOut[n] = X[0][n];
}

}  // namespace

void launchGalerkin(const Ctl* ctl, const LevelDev& fine, const LevelDev& coarse, cudaStream_t s) {
    k_gal_diag<<<blocksFor(fine.N), kThreads, 0, s>>>(ctl, fine);
    const int n = coarse.totalSlots > coarse.N ? coarse.totalSlots : coarse.N;
    k_gal_coarse<<<blocksFor(n), kThreads, 0, s>>>(ctl, fine, coarse);
}

void launchMGSmooth(const Ctl* ctl, const LevelDev& L, const double* x, double* y, double w, cudaStream_t s) {
    if (!L.sliceOff && L.W == 4) k_mg_smooth_ell<4><<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x, y, w);
    else if (!L.sliceOff && L.W == 3) k_mg_smooth_ell<3><<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x, y, w);
    else k_mg_smooth<<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x, y, w);
}

void launchMGSmoothBlock(const Ctl* ctl, const LevelDev& L, double* x, double w, int sweeps, cudaStream_t s) {
    const int threads = L.N < 1024 ? ((L.N + 31) / 32) * 32 : 1024;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mg_smooth_block, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    k_mg_smooth_block<<<1, threads, 2 * (size_t)L.N * sizeof(double), s>>>(ctl, L, x, w, sweeps);
}

void launchMGResidual(const Ctl* ctl, const LevelDev& L, const double* x, cudaStream_t s) {
    if (!L.sliceOff && L.W == 4) k_mg_residual_ell<4><<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x);
    else if (!L.sliceOff && L.W == 3) k_mg_residual_ell<3><<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x);
    else k_mg_residual<<<blocksFor(L.N), kThreads, 0, s>>>(ctl, L, x);
}

void launchMGGather(const Ctl* ctl, const LevelDev& fine, const LevelDev& coarse, double* xCur, double* xAlt,
                    int firstSweep, double w, cudaStream_t s) {
    k_mg_gather<<<blocksFor(coarse.N), kThreads, 0, s>>>(ctl, fine.res, coarse, xCur, xAlt, firstSweep, w);
}

void launchMGProlong(const Ctl* ctl, const LevelDev& fine, double* xFine, const double* xCoarse, cudaStream_t s) {
    k_mg_prolong<<<blocksFor(fine.N), kThreads, 0, s>>>(ctl, fine.N, fine.c2c, xFine, xCoarse);
}

size_t tailSharedBytes(const TailArgs& a) {
    size_t d = 0;
    for (int i = 0; i < a.count; i++) d += 4 * (size_t)a.lv[i].N;
    return d * sizeof(double);
}

void launchMGTail(const Ctl* ctl, const TailArgs& a, cudaStream_t s) {
    const size_t smem = tailSharedBytes(a);
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_mg_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        configured = true;
    }
    k_mg_tail<<<1, kTailThreads, smem, s>>>(ctl, a);
}

}  // namespace axisim
