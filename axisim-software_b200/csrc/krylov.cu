// krylov.cu -- flexible preconditioned conjugate gradients for the pressure
// correction, with the FP32 agglomeration V-cycle as preconditioner.
//
// New relative to the reference, which applies a fixed number of V-cycles
// (multigrid.cu:794-798). The p' matrix is symmetric (each face coefficient
// rho A Df / d is the same seen from either cell) with a positive diagonal
// that dominates, so CG applies. The FP32 V-cycle is not exactly a fixed
// linear operator, so directions are kept A-orthogonal with the flexible
// choice beta = -(z, q_prev) / (p_prev, q_prev) (Notay, "Flexible conjugate
// gradients", SIAM J. Sci. Comput. 22, 2000). Vectors and scalars are FP64 and
// never leave the device: each dot product is a per-block partial sum that the
// last block to finish adds up in block order (deterministic), so one
// iteration is
//   V-cycle(r) -> e ; dots (r,e),(e,q) ; p = e + beta p, q = A p, (p,q) ;
//   x += alpha p, r -= alpha q (and r in FP32 for the next V-cycle)
// with no host round trip, inside the captured SIMPLE iteration. The solve
// stops early once ||r||_2 <= relTol ||b||_2, or at its iteration cap: the
// kernel that finds it sets Ctl::ppSkip, every later kernel of the solve (the
// V-cycle's included) returns at entry, and k_fcg_end clears the flag. In a
// captured graph of a solve with a tolerance and a cap of 8 or more, the
// iterations after the first are the body of a conditional WHILE node (two
// iterations per body), so a solve that stops early launches at most one
// iteration's kernels past that point instead of running every remaining
// iteration's kernels up to the cap as early returns; a solve without a
// tolerance always runs to its cap and keeps its iterations unrolled.
#include <cmath>

#include "kernels.hpp"

namespace axisim {

namespace {

constexpr int kThreads = 256;
inline int blocksFor(int n) { return (n + kThreads - 1) / kThreads; }

__device__ __forceinline__ double opAx(const LevelDev& L, int n, const double* __restrict__ x) {
    double Ax = L.AC[n] * x[n];
    for (int j = 0; j < L.W; j++) {
        const size_t s = (size_t)j * L.N + n;
        const int k = L.nb[s];
        if (k >= 0) Ax += L.AF[s] * x[k];
    }
    return Ax;
}

// Block sums of NQ values -> partial[block][NQ]; the last block to arrive adds
// all partials in block order and writes out[0..NQ). counter starts at 0 and is
// returned to 0 by the last block.
// Returns true in thread 0 of the last block, after out[] is written.
template <int NQ>
__device__ __forceinline__ bool gridSum(const double (&v)[NQ], double* __restrict__ partial,
                                        unsigned int* counter, double* out) {
    __shared__ double sh[kThreads / 32][NQ];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            double x = 0.0;
            for (int w = 0; w < kThreads / 32; w++) x += sh[w][q];
            partial[(size_t)blockIdx.x * NQ + q] = x;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) acc[q] = 0.0;
    // fixed assignment of partials to threads and a fixed tree: deterministic
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads)
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] += ((volatile double*)partial)[(size_t)i * NQ + q];
    __shared__ double tr[kThreads][NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) tr[threadIdx.x][q] = acc[q];
    __syncthreads();
    for (int st = kThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
#pragma unroll
            for (int q = 0; q < NQ; q++) tr[threadIdx.x][q] += tr[threadIdx.x + st][q];
        __syncthreads();
    }
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int q = 0; q < NQ; q++) out[q] = tr[0][q];
    *counter = 0u;
    return true;
}

// r = b - A x in FP64, r in FP32 for the V-cycle and, when firstSweep, the
// V-cycle's first weighted Jacobi sweep from zero.
// s[4] = (b, b), s[5] = (r, r), s[7] = (r0, r0), s[6] = iteration counter; a solve that
// already meets the tolerance (b = 0 included) is skipped whole.
__global__ void __launch_bounds__(kThreads) k_fcg_init(Ctl* ctl, LevelDev L, const double* __restrict__ x,
                                                       double* __restrict__ r, float* __restrict__ r32,
                                                       float* __restrict__ eFirst, double w, int firstSweep,
                                                       double relTol, double* __restrict__ partial,
                                                       unsigned int* counter, double* s) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (n < L.N) {
        const double bv = L.b[n];
        const double rv = bv - opAx(L, n, x);
        r[n] = rv;
        r32[n] = (float)rv;
        if (firstSweep) {
            const double ac = L.AC[n];
            eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * rv / ac);
        }
        acc[0] = bv * bv;
        acc[1] = rv * rv;
    }
    if (gridSum<2>(acc, partial, counter, s + 4)) {
        ctl->ppSolves++;
        s[6] = (double)ctl->ppIterations;  // Krylov iterations before this solve
        s[7] = s[5];                       // (r0, r0)
        if (s[5] <= relTol * relTol * s[4]) ctl->ppSkip = 1;
    }
}

// s[0] = (r, e), s[1] = (e, q_prev) (useQ) with e the V-cycle's output.
__global__ void __launch_bounds__(kThreads) k_fcg_dots(const Ctl* ctl, int N, const float* __restrict__ e,
                                                       const double* __restrict__ r, const double* __restrict__ q,
                                                       int useQ, double* __restrict__ partial, unsigned int* counter,
                                                       double* s) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (n < N) {
        const double z = (double)e[n];
        acc[0] = r[n] * z;
        if (useQ) acc[1] = z * q[n];
    }
    gridSum<2>(acc, partial, counter, s);
}

// p_new = e + beta p_old (beta = -s[1] / s[pqOld], 0 on the first iteration),
// q = A p_new, s[pqNew] = (p_new, q). Neighbours' p_new are formed from their
// e and p_old on the fly, so the direction update needs no pass of its own.
__global__ void __launch_bounds__(kThreads) k_fcg_spmv(const Ctl* ctl, LevelDev L, const float* __restrict__ e,
                                                       const double* __restrict__ pOld, double* __restrict__ pNew,
                                                       double* __restrict__ q, double* s, int first, int pqOld,
                                                       int pqNew, double* __restrict__ partial,
                                                       unsigned int* counter) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double beta = 0.0;
    if (!first) {
        const double pq = s[pqOld];
        beta = (pq != 0.0 && isfinite(pq)) ? -s[1] / pq : 0.0;
    }
    double acc[1] = {0.0};
    if (n < L.N) {
        const double pn = first ? (double)e[n] : (double)e[n] + beta * pOld[n];
        double Ap = L.AC[n] * pn;
        for (int j = 0; j < L.W; j++) {
            const size_t sl = (size_t)j * L.N + n;
            const int k = L.nb[sl];
            if (k >= 0) {
                const double pk = first ? (double)e[k] : (double)e[k] + beta * pOld[k];
                Ap += L.AF[sl] * pk;
            }
        }
        pNew[n] = pn;
        q[n] = Ap;
        acc[0] = pn * Ap;
    }
    gridSum<1>(acc, partial, counter, s + pqNew);
}

// alpha = s[0] / s[pq]; x += alpha p; r -= alpha q; r in FP32 (and the first
// sweep) for the next V-cycle; s[5] = (r, r) and the stopping test.
__global__ void __launch_bounds__(kThreads) k_fcg_update(Ctl* ctl, LevelDev L, double* __restrict__ x,
                                                         double* __restrict__ r, const double* __restrict__ p,
                                                         const double* __restrict__ q, double* s, int pqSlot,
                                                         float* __restrict__ r32, float* __restrict__ eFirst, double w,
                                                         int next, double relTol, int maxIt,
                                                         double* __restrict__ partial, unsigned int* counter) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const double pq = s[pqSlot];
    const double alpha = (pq != 0.0 && isfinite(pq)) ? s[0] / pq : 0.0;
    double acc[1] = {0.0};
    if (n < L.N) {
        x[n] += alpha * p[n];
        if (next) {
            const double rv = r[n] - alpha * q[n];
            r[n] = rv;
            r32[n] = (float)rv;
            if (next > 1) {
                const double ac = L.AC[n];
                eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * rv / ac);
            }
            acc[0] = rv * rv;
        }
    }
    if (!next) {
        if (n == 0) {
            ctl->ppIterations++;
            if (ctl->ppIterations - (long long)s[6] >= maxIt) ctl->ppSkip = 1;
        }
        return;
    }
    if (gridSum<1>(acc, partial, counter, s + 5)) {
        ctl->ppIterations++;
        if (s[5] <= relTol * relTol * s[4] || ctl->ppIterations - (long long)s[6] >= maxIt) ctl->ppSkip = 1;
    }
}

// Condition of the WHILE node over the Krylov iterations; s[15] counts the
// bodies run in this solve, so the loop ends after maxBodies bodies even if
// the iteration cap in k_fcg_update were never reached.
__global__ void k_fcg_loop(const Ctl* ctl, double* s, cudaGraphConditionalHandle h, int head, int maxBodies) {
    pdlEnter();
    s[15] = head ? 0.0 : s[15] + 1.0;
    const bool run = !ctl->done && !ctl->ppSkip && s[15] < (double)maxBodies;
    cudaGraphSetConditional(h, run ? 1u : 0u);
}

// Chooses, for this solve, between the learned first preconditioner and the
// plain V-cycle: the network when its running score is at least as good as
// the V-cycle's (or either has no score yet), with every 16th solve a probe of
// the V-cycle and every 16th + 8 a probe of the network so both scores stay
// current (always: the network on every solve). Using the network sets
// Ctl::ppSkip = 2 for the network's kernels and k_nn_residual; k_fcg_ungate
// then clears it before the V-cycle on the remaining residual.
__global__ void k_fcg_gate(Ctl* ctl, NetStats* ns, int always) {
    pdlEnter();
    if (ctl->done) return;
    const long long k = ns->solveIdx++ % 16;
    int use;
    if (always) use = 1;
    else if (k == 0) use = 0;
    else if (k == 8) use = 1;
    else use = (ns->nNet == 0 || ns->nV == 0 || ns->logRhoNet <= ns->logRhoV) ? 1 : 0;
    ns->curNet = use && ctl->ppSkip == 0;
    if (use) ns->applied++;
    else if (k != 0) ns->fallbacks++;
    if (use && ctl->ppSkip == 0) ctl->ppSkip = 2;
}

// With the network's step (ppSkip == 2), step 1: Ay = A y (FP64) and the
// best scale of y in the energy norm, alpha = (y, r) / (y, A y), in sn[0].
__global__ void __launch_bounds__(kThreads) k_nn_scale(const Ctl* ctl, LevelDev L, const double* __restrict__ r,
                                                       const float* __restrict__ y, double* __restrict__ Ay,
                                                       double* __restrict__ partial, unsigned int* counter,
                                                       double* sn) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip != 2) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0.0, 0.0};
    if (n < L.N) {
        const double yn = (double)y[n];
        double a = L.AC[n] * yn;
        for (int j = 0; j < L.W; j++) {
            const size_t s = (size_t)j * L.N + n;
            const int k = L.nb[s];
            if (k >= 0) a += L.AF[s] * (double)y[k];
        }
        Ay[n] = a;
        acc[0] = yn * r[n];
        acc[1] = yn * a;
    }
    if (gridSum<2>(acc, partial, counter, sn + 1)) sn[0] = (sn[2] > 0.0 && isfinite(sn[1])) ? sn[1] / sn[2] : 0.0;
}

// Step 2: r' = r - alpha A y in FP64, r' in FP32 for the V-cycle that follows,
// and that V-cycle's first sweep from zero.
__global__ void __launch_bounds__(kThreads) k_nn_residual(const Ctl* ctl, LevelDev L, const double* __restrict__ r,
                                                          const double* __restrict__ Ay, const double* sn,
                                                          float* __restrict__ r32, float* __restrict__ eFirst,
                                                          double w, int firstSweep) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip != 2) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const double rv = r[n] - sn[0] * Ay[n];
    r32[n] = (float)rv;
    if (firstSweep) {
        const double ac = L.AC[n];
        eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * rv / ac);
    }
}

// z = alpha y + V-cycle(r - alpha A y) when this solve uses the network.
__global__ void __launch_bounds__(kThreads) k_nn_combine(const Ctl* ctl, const NetStats* ns, int N,
                                                         const float* __restrict__ y, const double* sn,
                                                         float* __restrict__ e) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip || !ns->curNet) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) e[n] = (float)((double)e[n] + sn[0] * (double)y[n]);
}

__global__ void k_fcg_ungate(Ctl* ctl) {
    pdlEnter();
    if (ctl->ppSkip == 2) ctl->ppSkip = 0;
}

// Ends the solve: clears Ctl::ppSkip and, with ns, adds the solve's score to
// the running mean (window 32) of the method it used.
__global__ void k_fcg_end(Ctl* ctl, const double* s, NetStats* ns) {
    pdlEnter();
    ctl->ppSkip = 0;
    if (!ns || ctl->done) return;
    const double iters = (double)ctl->ppIterations - s[6];
    if (!(iters >= 1.0) || !(s[7] > 0.0) || !(s[5] > 0.0) || !isfinite(s[5])) return;
    const double score = 0.5 * log(s[5] / s[7]) / iters;
    if (ns->curNet) {
        const long long m = ns->nNet < 32 ? ns->nNet + 1 : 32;
        ns->logRhoNet += (score - ns->logRhoNet) / (double)m;
        ns->nNet++;
    } else {
        const long long m = ns->nV < 32 ? ns->nV + 1 : 32;
        ns->logRhoV += (score - ns->logRhoV) / (double)m;
        ns->nV++;
    }
}


}  // namespace

void launchFcgInit(Ctl* ctl, const LevelDev& L0, const double* x, double* r, float* r32, float* eFirst, double w,
                   int firstSweep, double relTol, FcgScratch& f, cudaStream_t s) {
    launchPDL(k_fcg_init, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, x, r, r32, eFirst, w, firstSweep,
              relTol, f.partial, f.counter, f.scalars);
}

void launchFcgDots(const Ctl* ctl, int N, const float* e, const double* r, const double* q, int useQ, FcgScratch& f,
                   cudaStream_t s) {
    launchPDL(k_fcg_dots, dim3(blocksFor(N)), dim3(kThreads), 0, s, ctl, N, e, r, q, useQ, f.partial, f.counter,
              f.scalars);
}

void launchFcgSpmv(const Ctl* ctl, const LevelDev& L0, const float* e, const double* pOld, double* pNew, double* q,
                   int first, int pqOld, int pqNew, FcgScratch& f, cudaStream_t s) {
    launchPDL(k_fcg_spmv, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, e, pOld, pNew, q, f.scalars, first,
              pqOld, pqNew, f.partial, f.counter + 1);
}

void launchFcgUpdate(Ctl* ctl, const LevelDev& L0, double* x, double* r, const double* p, const double* q,
                     FcgScratch& f, int pqSlot, float* r32, float* eFirst, double w, int next, double relTol,
                     int maxIt, cudaStream_t s) {
    launchPDL(k_fcg_update, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, x, r, p, q, f.scalars, pqSlot, r32,
              eFirst, w, next, relTol, maxIt, f.partial, f.counter + 1);
}

void launchFcgLoop(Ctl* ctl, FcgScratch& f, cudaGraphConditionalHandle h, int head, int maxBodies, cudaStream_t s) {
    launchPDL(k_fcg_loop, dim3(1), dim3(1), 0, s, (const Ctl*)ctl, f.scalars, h, head, maxBodies);
}

void launchFcgGate(Ctl* ctl, NetStats* ns, int always, cudaStream_t s) {
    launchPDL(k_fcg_gate, dim3(1), dim3(1), 0, s, ctl, ns, always);
}

void launchNnResidual(const Ctl* ctl, const LevelDev& L0, const double* r, const float* y, double* Ay,
                      FcgScratch& f, float* r32, float* eFirst, double w, int firstSweep, cudaStream_t s) {
    double* sn = f.scalars + 8;
    launchPDL(k_nn_scale, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, r, y, Ay, f.partial, f.counter,
              sn);
    launchPDL(k_nn_residual, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, r, (const double*)Ay,
              (const double*)sn, r32, eFirst, w, firstSweep);
}

void launchNnCombine(const Ctl* ctl, const NetStats* ns, int N, const float* y, const FcgScratch& f, float* e,
                     cudaStream_t s) {
    launchPDL(k_nn_combine, dim3(blocksFor(N)), dim3(kThreads), 0, s, ctl, ns, N, y, (const double*)(f.scalars + 8),
              e);
}

void launchFcgUngate(Ctl* ctl, cudaStream_t s) { launchPDL(k_fcg_ungate, dim3(1), dim3(1), 0, s, ctl); }

void launchFcgEnd(Ctl* ctl, const FcgScratch& f, NetStats* ns, cudaStream_t s) {
    launchPDL(k_fcg_end, dim3(1), dim3(1), 0, s, ctl, (const double*)f.scalars, ns);
}

}  // namespace axisim
