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
// stops early once ||r||_2 <= relTol ||b||_2: the kernel that finds it sets
// Ctl::ppSkip, every later kernel of the solve (the V-cycle's included) returns
// at entry, and k_fcg_end clears the flag.
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
// s[4] = (b, b), s[5] = (r, r), s[7] = (r0, r0), s[6] = 0; a solve that
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
        s[6] = 0.0;   // restart flag (set when a learned step is rolled back)
        s[7] = s[5];  // (r0, r0)
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
    const bool withQ = useQ && s[6] == 0.0;  // after a rollback the search restarts
    double acc[2] = {0.0, 0.0};
    if (n < N) {
        const double z = (double)e[n];
        acc[0] = r[n] * z;
        if (withQ) acc[1] = z * q[n];
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
                                                         int next, double relTol, double* __restrict__ partial,
                                                         unsigned int* counter, NetStats* ns) {
    pdlEnter();
    if (ctl->done || ctl->ppSkip) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const double rrOld = s[5];
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
        if (n == 0) ctl->ppIterations++;
        return;
    }
    if (gridSum<1>(acc, partial, counter, s + 5)) {
        ctl->ppIterations++;
        if (ns && rrOld > 0.0 && s[5] > 0.0 && isfinite(s[5])) {
            // running mean of the V-cycle step's log residual reduction (window ~100)
            const double lr = 0.5 * log(s[5] / rrOld);
            const long long k = ns->vSteps < 100 ? ns->vSteps + 1 : 100;
            ns->logRhoV += (lr - ns->logRhoV) / (double)k;
            ns->vSteps++;
        }
        if (s[5] <= relTol * relTol * s[4]) ctl->ppSkip = 1;
    }
}

// After a first step preconditioned by the learned network: keep it when its
// residual reduction ||r1|| / ||r0|| is at least as good as the V-cycle's
// running mean, else undo it (x -= alpha p, r += alpha q, r in FP32 and the
// first sweep again) and flag a restart of the search directions.
__global__ void __launch_bounds__(kThreads) k_fcg_judge(Ctl* ctl, LevelDev L, double* __restrict__ x,
                                                        double* __restrict__ r, const double* __restrict__ p,
                                                        const double* __restrict__ q, double* s, int pqSlot,
                                                        float* __restrict__ r32, float* __restrict__ eFirst, double w,
                                                        int firstSweep, NetStats* ns) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const double rr0 = s[7], rr1 = s[5];
    const double lr = (rr0 > 0.0 && rr1 >= 0.0) ? 0.5 * log(rr1 / rr0) : 0.0;
    const bool ok = isfinite(rr1) && (ns->vSteps == 0 || lr <= ns->logRhoV);
    if (n == 0) {
        ns->applied++;
        if (!ok) {
            ns->fallbacks++;
            s[6] = 1.0;
            s[5] = rr0;
            ctl->ppSkip = 0;
        }
    }
    if (ok || n >= L.N) return;
    const double pq = s[pqSlot];
    const double alpha = (pq != 0.0 && isfinite(pq)) ? s[0] / pq : 0.0;
    x[n] -= alpha * p[n];
    const double rv = r[n] + alpha * q[n];
    r[n] = rv;
    r32[n] = (float)rv;
    if (firstSweep) {
        const double ac = L.AC[n];
        eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * rv / ac);
    }
}

__global__ void k_fcg_end(Ctl* ctl) {
    pdlEnter();
    ctl->ppSkip = 0;
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
                     NetStats* ns, cudaStream_t s) {
    launchPDL(k_fcg_update, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, x, r, p, q, f.scalars, pqSlot, r32,
              eFirst, w, next, relTol, f.partial, f.counter + 1, ns);
}

void launchFcgJudge(Ctl* ctl, const LevelDev& L0, double* x, double* r, const double* p, const double* q,
                    FcgScratch& f, int pqSlot, float* r32, float* eFirst, double w, int firstSweep, NetStats* ns,
                    cudaStream_t s) {
    launchPDL(k_fcg_judge, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, x, r, p, q, f.scalars, pqSlot, r32,
              eFirst, w, firstSweep, ns);
}

void launchFcgEnd(Ctl* ctl, cudaStream_t s) { launchPDL(k_fcg_end, dim3(1), dim3(1), 0, s, ctl); }

}  // namespace axisim
