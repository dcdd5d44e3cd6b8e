// learned.cu -- forward, backward and Adam kernels of the learned p'
// preconditioner (network described in learned.hpp), its host driver, and the
// harvest of training samples from the captured SIMPLE iteration.
//
// Every layer is the same fused operation over the rows of one level:
//   Y = act(Z W + b [+ add]),  Z = [T_1(X_1), T_2(X_2)]
// where each input transform T is the identity, the mean over the cell's
// neighbours, the mean over an agglomerate's members (pool) or the copy from
// the cell's agglomerate (unpool). The backward pass of a layer is
//   G = dY * act'(Y);  dW = Z^T G;  db = sum G;  dZ = G W^T
// followed by the adjoint of each transform, which accumulates dZ into the
// gradient of its source tensor: identity, neighbour-mean transposed (a
// gather over the same symmetric graph), pool transposed (copy back to the
// members), unpool transposed (sum over the members). All reductions over
// rows (dW, db, the loss) run as per-block partials summed in a fixed order,
// so a training step is deterministic.
//
// The dense products are small (K <= 256 inputs, <= 128 outputs per row) and
// run on the FP32 pipes with BF16 storage: at the finest level, where nearly
// all rows are, a layer moves ~100 bytes and does ~1 kFLOP per row, far below
// the ridge point of either the FP32 pipes or the tensor cores, so the layer is
// bound by memory traffic, not by the multiply-adds.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>

#include <cuda_bf16.h>
#include <type_traits>

#include "host_prep.hpp"
#include "learned.hpp"

namespace axisim {

namespace {

constexpr int kThreads = 256;
inline int blocksFor(size_t n, int t = kThreads) { return (int)((n + t - 1) / t); }

#define NCK(x)                                                                                                \
    do {                                                                                                      \
        cudaError_t e_ = (x);                                                                                 \
        if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_));      \
    } while (0)

using bfloat = __nv_bfloat16;

// FP32 -> TF32 (round to nearest, ties away), as the tensor cores read it
__device__ __forceinline__ uint32_t toTf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// d += a b for one m16n8k8 block (A row-major 16 x 8, B column-major 8 x 8, FP32 accumulators)
__device__ __forceinline__ void mmaTf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float ldv(const float* p, size_t i) { return p[i]; }
__device__ __forceinline__ float ldv(const bfloat* p, size_t i) { return __bfloat162float(p[i]); }
__device__ __forceinline__ void stv(float* p, size_t i, float v) { p[i] = v; }
__device__ __forceinline__ void stv(bfloat* p, size_t i, float v) { p[i] = __float2bfloat16_rn(v); }

// Inference kernels run inside the captured p' solve: ungated they return while
// the solve is done or skipped (ppSkip != 0); gated they run only while
// ppSkip == 2, the state in which the solve uses the network's step.
__device__ __forceinline__ bool idle(const Ctl* ctl, int gated) {
    if (!ctl) return false;
    return ctl->done || (gated ? ctl->ppSkip != 2 : ctl->ppSkip != 0);
}

// Sums NQ doubles over the grid: block partials, then the last block to arrive
// adds them in block order. Returns true in thread 0 of that block.
template <int NQ>
__device__ bool gridSumD(const double (&v)[NQ], double* partial, unsigned int* counter, double* out) {
    __shared__ double sh[kThreads / 32][NQ];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < NQ; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
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
    __shared__ double tr[kThreads][NQ];
    double acc[NQ];
    for (int q = 0; q < NQ; q++) acc[q] = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads)
        for (int q = 0; q < NQ; q++) acc[q] += ((volatile double*)partial)[(size_t)i * NQ + q];
    for (int q = 0; q < NQ; q++) tr[threadIdx.x][q] = acc[q];
    __syncthreads();
    for (int st = kThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int q = 0; q < NQ; q++) tr[threadIdx.x][q] += tr[threadIdx.x + st][q];
        __syncthreads();
    }
    if (threadIdx.x != 0) return false;
    for (int q = 0; q < NQ; q++) out[q] = tr[0][q];
    *counter = 0u;
    return true;
}

// ---------------- features ----------------

// scal[0] = mean (r / AC)^2 (sigma^2)
template <class TR>
__global__ void __launch_bounds__(kThreads) k_sigma(const Ctl* ctl, int gated, int N, const TR* r, const TR* AC, double* partial,
                                                    unsigned int* counter, double* scal) {
    if (idle(ctl, gated)) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[1] = {0.0};
    if (n < N) {
        const double ac = (double)AC[n];
        const double q = ac != 0.0 ? (double)r[n] / ac : 0.0;
        acc[0] = q * q;
    }
    if (gridSumD<1>(acc, partial, counter, scal)) scal[0] /= (double)N;
}

// feat[n] = [r / (AC sigma), deficit]; deficit from the ELL matrix (AF != null)
// or given.
template <class TA, class TR>
__global__ void __launch_bounds__(kThreads) k_features(const Ctl* ctl, int gated, int N, const TR* r, const TR* AC,
                                                       const double* AF, const int32_t* nb, int W,
                                                       const float* deficit, const double* scal, TA* feat) {
    if (idle(ctl, gated)) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const double sigma = sqrt(scal[0]);
    const double ac = (double)AC[n];
    const double x = (ac != 0.0 && sigma > 0.0) ? (double)r[n] / (ac * sigma) : 0.0;
    float d;
    if (AF) {
        double s = 0.0;
        for (int j = 0; j < W; j++) {
            const size_t sl = (size_t)j * N + n;
            if (nb[sl] >= 0) s += fabs(AF[sl]);
        }
        d = ac != 0.0 ? (float)(1.0 - s / ac) : 0.f;
    } else {
        d = deficit[n];
    }
    stv(feat, (size_t)n * 2, (float)x);
    stv(feat, (size_t)n * 2 + 1, d);
}

// ---------------- layer forward ----------------

template <class TA>
__device__ __forceinline__ void gatherInput(const NetIn& I, int n, float* z) {
    const TA* x = (const TA*)I.x;
    const int C = I.C;
    if (I.xf == NX_ID) {
        for (int c = 0; c < C; c++) z[c] = ldv(x, (size_t)n * C + c);
    } else if (I.xf == NX_UNPOOL) {
        const int k = I.map[n];
        for (int c = 0; c < C; c++) z[c] = ldv(x, (size_t)k * C + c);
    } else {  // NBMEAN or POOL: mean over a CSR list
        for (int c = 0; c < C; c++) z[c] = 0.f;
        for (int q = I.s[n]; q < I.s[n + 1]; q++) {
            const int k = I.list[q];
            for (int c = 0; c < C; c++) z[c] += ldv(x, (size_t)k * C + c);
        }
        const float w = I.inv[n];
        for (int c = 0; c < C; c++) z[c] *= w;
    }
}

// One row per thread; the row's concatenated input Z lives in shared memory
// (stride K + 1: conflict-free across the warp), weights are broadcast loads.
template <class TA, class TW, int OCH>
__global__ void k_layer_fwd(const Ctl* ctl, int gated, NetLayer L, const TW* __restrict__ P) {
    if (idle(ctl, gated)) return;
    extern __shared__ float zsm[];
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const int K = L.K, Cout = L.Cout;
    float* z = zsm + (size_t)threadIdx.x * (K + 1);
    int off = 0;
    for (int i = 0; i < L.nIn; i++) {
        gatherInput<TA>(L.in[i], n, z + off);
        off += L.in[i].C;
    }
    if (L.Z) {
        TA* Z = (TA*)L.Z;
        for (int k = 0; k < K; k++) stv(Z, (size_t)n * K + k, z[k]);
    }
    const TW* W = P + L.wOff;
    const TW* B = W + (size_t)K * Cout;
    const TA* add = (const TA*)L.add;
    TA* Y = (TA*)L.Y;
    for (int o0 = 0; o0 < Cout; o0 += OCH) {
        float acc[OCH];
#pragma unroll
        for (int j = 0; j < OCH; j++) acc[j] = (o0 + j < Cout) ? ldv(B, o0 + j) : 0.f;
        for (int k = 0; k < K; k++) {
            const float zk = z[k];
            const TW* wr = W + (size_t)k * Cout + o0;
#pragma unroll
            for (int j = 0; j < OCH; j++)
                if (o0 + j < Cout) acc[j] = fmaf(zk, ldv(wr, j), acc[j]);
        }
#pragma unroll
        for (int j = 0; j < OCH; j++) {
            if (o0 + j >= Cout) break;
            float v = acc[j];
            if (add) v += ldv(add, (size_t)n * Cout + o0 + j);
            if (L.relu) v = fmaxf(v, 0.f);
            stv(Y, (size_t)n * Cout + o0 + j, v);
        }
    }
}

// Tiled layers: a block computes a 64-row tile of Y = act(Z W + b [+ add])
// for all Cout = 16 CPT outputs. The tile's Z (64 x K, FP32) is gathered into
// shared memory (lanes along the channels, so source rows load coalesced),
// W is staged in 32-row chunks, and each of the 256 threads accumulates a
// 4-row x CPT-column register block (columns tx + 16 j: conflict-free
// weight reads, broadcast Z reads).
constexpr int kTileRows = 64;
constexpr int kChunk = 32;

// Every channel count here divides 256, so thread t handles channel t % C of
// rows t / C, t / C + 256 / C, ... of each input (no per-element division).
// For a mean over a CSR list, the tile's list bounds are first staged in
// shared memory (idx: TR + 1 ints) so the C threads of a row do not each
// re-read them.
template <class TA, int TR>
__device__ __forceinline__ void gatherTile(const NetLayer& L, int row0, float* zs, int ldz, int* idx) {
    int off = 0;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        if (i >= L.nIn) break;
        const NetIn& I = L.in[i];
        const int C = I.C;
        const int c = threadIdx.x % C, rstep = blockDim.x / C;
        const TA* x = (const TA*)I.x;
        const bool mean = I.xf == NX_NBMEAN || I.xf == NX_POOL;
        if (mean) {
            __syncthreads();
            for (int r = threadIdx.x; r <= TR; r += blockDim.x) idx[r] = I.s[min(row0 + r, L.N)];
            __syncthreads();
        }
        for (int r = threadIdx.x / C; r < TR; r += rstep) {
            const int n = row0 + r;
            float v = 0.f;
            if (n < L.N) {
                if (I.xf == NX_ID) v = ldv(x, (size_t)n * C + c);
                else if (I.xf == NX_UNPOOL) v = ldv(x, (size_t)I.map[n] * C + c);
                else {
                    // four independent list loads, then four independent row
                    // loads: coarse levels have long lists and few rows, so
                    // the loop is bound by load latency, not bandwidth
                    int q = idx[r];
                    const int q1 = idx[r + 1];
                    for (; q + 4 <= q1; q += 4) {
                        const int k0 = __ldg(I.list + q), k1 = __ldg(I.list + q + 1);
                        const int k2 = __ldg(I.list + q + 2), k3 = __ldg(I.list + q + 3);
                        const float a0 = ldv(x, (size_t)k0 * C + c), a1 = ldv(x, (size_t)k1 * C + c);
                        const float a2 = ldv(x, (size_t)k2 * C + c), a3 = ldv(x, (size_t)k3 * C + c);
                        v += (a0 + a1) + (a2 + a3);
                    }
                    for (; q < q1; q++) v += ldv(x, (size_t)__ldg(I.list + q) * C + c);
                    v *= __ldg(I.inv + n);
                }
            }
            zs[r * ldz + off + c] = v;
        }
        off += C;
    }
}

template <class TA, class TW, int CPT, int RPT>
__global__ void __launch_bounds__(256) k_layer_tile(const Ctl* ctl, int gated, NetLayer L, const TW* __restrict__ P) {
    if (idle(ctl, gated)) return;
    constexpr int COUT = 16 * CPT;
    constexpr int TR = 16 * RPT;  // rows per tile
    extern __shared__ float sm[];
    const int K = L.K;
    const int ldz = K + 1;
    float* zs = sm;                   // [TR][K + 1]
    float* ws = sm + TR * ldz;        // [32][COUT]
    const int row0 = blockIdx.x * TR;
    gatherTile<TA, TR>(L, row0, zs, ldz, (int*)(ws + kChunk * COUT));
    __syncthreads();
    if (L.Z) {
        TA* Z = (TA*)L.Z;
        const int k = threadIdx.x % K, rstep = blockDim.x / K;
        for (int r = threadIdx.x / K; r < TR; r += rstep)
            if (row0 + r < L.N) stv(Z, (size_t)(row0 + r) * K + k, zs[r * ldz + k]);
    }
    // Tensor cores: the TR x COUT tile is (TR/16) x (COUT/8) mma.sync
    // m16n8k8 TF32 blocks with FP32 accumulators, dealt round-robin to the 8
    // warps. The FP32 activations are split into a TF32 high part and the
    // TF32 rounding of the remainder, and both are multiplied: close to FP32
    // accuracy. BF16 weights are exact in TF32; FP32 weights (the gradient
    // check's mode) are split the same way, adding a third product.
    constexpr int NRB = RPT, NCB = 2 * CPT;
    constexpr int TPW = (NRB * NCB + 7) / 8;  // blocks per warp
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t4 = lane & 3;
    const TW* W = P + L.wOff;
    float acc[TPW][4];
#pragma unroll
    for (int q = 0; q < TPW; q++) {
        const int blk = warp + 8 * q;
        const int cb = blk % NCB;
        const float b0 = blk < NRB * NCB ? ldv(W + (size_t)K * COUT, cb * 8 + 2 * t4) : 0.f;
        const float b1 = blk < NRB * NCB ? ldv(W + (size_t)K * COUT, cb * 8 + 2 * t4 + 1) : 0.f;
        acc[q][0] = b0;
        acc[q][1] = b1;
        acc[q][2] = b0;
        acc[q][3] = b1;
    }
    for (int k0 = 0; k0 < K; k0 += kChunk) {
        const int kn = min(kChunk, K - k0);
        // the chunk's weights: all of a thread's loads issued before any
        // shared-memory store, so they are in flight together
        constexpr int PER = kChunk * COUT / 256;
        float wv[PER];
#pragma unroll
        for (int u = 0; u < PER; u++) {
            const int idx = threadIdx.x + 256 * u;
            wv[u] = idx < kn * COUT ? ldv(W, (size_t)k0 * COUT + idx) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PER; u++) ws[threadIdx.x + 256 * u] = wv[u];
        __syncthreads();
        for (int kk = 0; kk < kn; kk += 8) {
            // columns past the chunk (K below 8) read as zero, never the next row
            const bool c0ok = kk + t4 < kn, c1ok = kk + t4 + 4 < kn;
#pragma unroll
            for (int q = 0; q < TPW; q++) {
                const int blk = warp + 8 * q;
                if (blk >= NRB * NCB) break;
                const int rb = blk / NCB, cb = blk % NCB;
                const float* zr0 = zs + (rb * 16 + g) * ldz + k0 + kk;
                const float* zr1 = zr0 + 8 * ldz;
                const float a[4] = {c0ok ? zr0[t4] : 0.f, c0ok ? zr1[t4] : 0.f, c1ok ? zr0[t4 + 4] : 0.f,
                                    c1ok ? zr1[t4 + 4] : 0.f};
                const float bw[2] = {ws[(kk + t4) * COUT + cb * 8 + g], ws[(kk + t4 + 4) * COUT + cb * 8 + g]};
                uint32_t ahi[4], alo[4], bhi[2];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    ahi[e] = toTf32(a[e]);
                    alo[e] = toTf32(a[e] - __uint_as_float(ahi[e]));
                }
#pragma unroll
                for (int e = 0; e < 2; e++) bhi[e] = toTf32(bw[e]);
                if constexpr (std::is_same<TW, float>::value) {
                    uint32_t blo[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) blo[e] = toTf32(bw[e] - __uint_as_float(bhi[e]));
                    mmaTf32(acc[q], ahi, blo);
                }
                mmaTf32(acc[q], alo, bhi);
                mmaTf32(acc[q], ahi, bhi);
            }
        }
    }
    const TA* add = (const TA*)L.add;
    TA* Y = (TA*)L.Y;
#pragma unroll
    for (int q = 0; q < TPW; q++) {
        const int blk = warp + 8 * q;
        if (blk >= NRB * NCB) break;
        const int rb = blk / NCB, cb = blk % NCB;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int n = row0 + rb * 16 + g + (e >= 2 ? 8 : 0);
            const int o = cb * 8 + 2 * t4 + (e & 1);
            if (n >= L.N) continue;
            float v = acc[q][e];
            if (add) v += ldv(add, (size_t)n * COUT + o);
            if (L.relu) v = fmaxf(v, 0.f);
            stv(Y, (size_t)n * COUT + o, v);
        }
    }
}

// Tiled backward: G = gY * act'(Y) for a 64-row tile (kept in shared memory
// and written out for the weight gradient), then dZ = G W^T for K = 16 KPT
// columns, W^T staged in 32-output chunks.
template <class TA, class TW, int KPT>
__global__ void __launch_bounds__(256) k_layer_dz_tile(NetLayer L, const TW* __restrict__ P, float* __restrict__ G,
                                                       float* __restrict__ dZ) {
    constexpr int KD = 16 * KPT;
    extern __shared__ float sm[];
    const int Cout = L.Cout;
    const int ldg = Cout + 1;
    float* gs = sm;                       // [64][Cout + 1]
    float* wt = sm + kTileRows * ldg;     // [32][KD]: W^T chunk
    const int row0 = blockIdx.x * kTileRows;
    const TA* Y = (const TA*)L.Y;
    const int o = threadIdx.x % Cout, rstep = blockDim.x / Cout;  // Cout divides 256
    for (int r = threadIdx.x / Cout; r < kTileRows; r += rstep) {
        const int n = row0 + r;
        float v = 0.f;
        if (n < L.N) {
            v = L.gY[(size_t)n * Cout + o];
            if (L.relu && ldv(Y, (size_t)n * Cout + o) <= 0.f) v = 0.f;
            G[(size_t)n * Cout + o] = v;
        }
        gs[r * ldg + o] = v;
    }
    if (!dZ) return;
    // tensor cores: the 64 x KD tile of dZ is 4 x (KD/8) mma.sync m16n8k8
    // TF32 blocks dealt to the 8 warps; G split into TF32 high and low parts,
    // W exact (BF16) or split (FP32)
    constexpr int NCB = 2 * KPT, NBLK = 4 * NCB, TPW = (NBLK + 7) / 8;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const TW* W = P + L.wOff;
    float acc[TPW][4];
#pragma unroll
    for (int q = 0; q < TPW; q++)
#pragma unroll
        for (int e = 0; e < 4; e++) acc[q][e] = 0.f;
    for (int o0 = 0; o0 < Cout; o0 += kChunk) {
        const int on = min(kChunk, Cout - o0);
        constexpr int PER = kChunk * KD / 256;
        float wv[PER];
#pragma unroll
        for (int u = 0; u < PER; u++) {
            const int idx = threadIdx.x + 256 * u;
            const int oo = idx / KD, k = idx % KD;
            wv[u] = oo < on ? ldv(W, (size_t)k * Cout + o0 + oo) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PER; u++) wt[threadIdx.x + 256 * u] = wv[u];
        __syncthreads();
        for (int oo = 0; oo < on; oo += 8) {
            const bool c0ok = oo + t4 < on, c1ok = oo + t4 + 4 < on;
#pragma unroll
            for (int q = 0; q < TPW; q++) {
                const int blk = warp + 8 * q;
                if (blk >= NBLK) break;
                const int rb = blk / NCB, cb = blk % NCB;
                const float* g0 = gs + (rb * 16 + g) * ldg + o0 + oo;
                const float* g1 = g0 + 8 * ldg;
                const float a[4] = {c0ok ? g0[t4] : 0.f, c0ok ? g1[t4] : 0.f, c1ok ? g0[t4 + 4] : 0.f,
                                    c1ok ? g1[t4 + 4] : 0.f};
                const float bw[2] = {wt[(oo + t4) * KD + cb * 8 + g], wt[(oo + t4 + 4) * KD + cb * 8 + g]};
                uint32_t ahi[4], alo[4], bhi[2];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    ahi[e] = toTf32(a[e]);
                    alo[e] = toTf32(a[e] - __uint_as_float(ahi[e]));
                }
#pragma unroll
                for (int e = 0; e < 2; e++) bhi[e] = toTf32(bw[e]);
                if constexpr (std::is_same<TW, float>::value) {
                    uint32_t blo[2];
#pragma unroll
                    for (int e = 0; e < 2; e++) blo[e] = toTf32(bw[e] - __uint_as_float(bhi[e]));
                    mmaTf32(acc[q], ahi, blo);
                }
                mmaTf32(acc[q], alo, bhi);
                mmaTf32(acc[q], ahi, bhi);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < TPW; q++) {
        const int blk = warp + 8 * q;
        if (blk >= NBLK) break;
        const int rb = blk / NCB, cb = blk % NCB;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int n = row0 + rb * 16 + g + (e >= 2 ? 8 : 0);
            if (n < L.N) dZ[(size_t)n * KD + cb * 8 + 2 * t4 + (e & 1)] = acc[q][e];
        }
    }
}

// e = sigma * y
template <class TA>
__global__ void __launch_bounds__(kThreads) k_scale_out(const Ctl* ctl, int gated, int N, const TA* y, const double* scal,
                                                        float* e) {
    if (idle(ctl, gated)) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    e[n] = (float)(sqrt(scal[0]) * (double)ldv(y, n));
}

// ---------------- loss ----------------

// Loss: the A-norm (energy) error left after the best scaling of the output,
//   loss = min_a ||a y - t||_A^2 / ||t||_A^2 = 1 - (y.b)^2 / ((y.A y)(b.t)),
// with A t = b. The Krylov solve applies the network's output with its own
// line search, which minimises exactly this error, so only y's direction in
// the energy norm matters. scal[1..3] = y.b, y.Ay, b.t.
template <class TA>
__global__ void __launch_bounds__(kThreads) k_loss_spmv(int N, int W, const int32_t* __restrict__ nb,
                                                        const float* __restrict__ AF, const float* __restrict__ AC,
                                                        const TA* y, const float* b, const float* t, float* Ay,
                                                        double* partial, unsigned int* counter, double* scal) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[3] = {0.0, 0.0, 0.0};
    if (n < N) {
        const double yn = (double)ldv(y, n);
        double a = (double)AC[n] * yn;
        for (int j = 0; j < W; j++) {
            const size_t sl = (size_t)j * N + n;
            const int k = nb[sl];
            if (k >= 0) a += (double)AF[sl] * (double)ldv(y, k);
        }
        Ay[n] = (float)a;
        acc[0] = yn * (double)b[n];
        acc[1] = yn * a;
        acc[2] = (double)b[n] * (double)t[n];
    }
    gridSumD<3>(acc, partial, counter, scal + 1);
}

// d loss / d y = -2 c / (E_y E_t) b + 2 c^2 / (E_y^2 E_t) A y,  c = y.b,
// E_y = y.Ay, E_t = b.t (A symmetric)
__global__ void __launch_bounds__(kThreads) k_loss_grad(int N, const float* b, const float* Ay, const double* scal,
                                                        float* gy, float* lossOut) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const double c = scal[1], ey = scal[2] > 0.0 ? scal[2] : 1e-300, et = scal[3] > 0.0 ? scal[3] : 1.0;
    if (n == 0) *lossOut = (float)(1.0 - c * c / (ey * et));
    if (n >= N) return;
    gy[n] = (float)(-2.0 * c / (ey * et) * (double)b[n] + 2.0 * c * c / (ey * ey * et) * (double)Ay[n]);
}

// ---------------- layer backward ----------------

// G = gY * act'(Y) ; dZ = G W^T (dZ may be null)
template <class TA, class TW, int KCH>
__global__ void __launch_bounds__(kThreads) k_layer_dz(NetLayer L, const TW* __restrict__ P, float* __restrict__ G,
                                                       float* __restrict__ dZ) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    const int K = L.K, Cout = L.Cout;
    const TA* Y = (const TA*)L.Y;
    for (int o = 0; o < Cout; o++) {
        float g = L.gY[(size_t)n * Cout + o];
        if (L.relu && ldv(Y, (size_t)n * Cout + o) <= 0.f) g = 0.f;
        G[(size_t)n * Cout + o] = g;
    }
    if (!dZ) return;
    const TW* W = P + L.wOff;
    for (int k0 = 0; k0 < K; k0 += KCH) {
        float acc[KCH];
#pragma unroll
        for (int j = 0; j < KCH; j++) acc[j] = 0.f;
        for (int o = 0; o < Cout; o++) {
            const float g = G[(size_t)n * Cout + o];
#pragma unroll
            for (int j = 0; j < KCH; j++)
                if (k0 + j < K) acc[j] = fmaf(g, ldv(W, (size_t)(k0 + j) * Cout + o), acc[j]);
        }
#pragma unroll
        for (int j = 0; j < KCH; j++)
            if (k0 + j < K) dZ[(size_t)n * K + k0 + j] = acc[j];
    }
}

// partial[split][K*Cout + Cout] = (Z^T G, sum G) over the split's rows.
// Block: a 32 x 32 tile of (k, o); 256 threads, 4 k per thread.
template <class TA>
__global__ void __launch_bounds__(kThreads) k_wgrad(int N, int K, int Cout, int tilesO, int rowsPerSplit,
                                                    const TA* __restrict__ Z, const float* __restrict__ G,
                                                    float* __restrict__ partial) {
    __shared__ float zs[64][33];
    __shared__ float gs[64][33];
    const int tk = blockIdx.x / tilesO, to = blockIdx.x % tilesO;
    const int k0 = tk * 32, o0 = to * 32;
    const int split = blockIdx.y;
    const int r0 = split * rowsPerSplit;
    const int r1 = min(N, r0 + rowsPerSplit);
    // tensor cores: the 32 x 32 tile of dW = Z^T G is 2 x 4 mma.sync m16n8k8
    // TF32 blocks, one per warp, reduced over the rows 8 at a time; FP32
    // operands split into TF32 high and low parts (BF16 activations are exact)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
    const int mb = warp >> 2, nb = warp & 3;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    float bacc = 0.f;
    for (int rc = r0; rc < r1; rc += 64) {
        for (int i = threadIdx.x; i < 64 * 32; i += kThreads) {
            const int rr = i >> 5, cc = i & 31;
            const int n = rc + rr;
            zs[rr][cc] = (n < r1 && k0 + cc < K) ? ldv(Z, (size_t)n * K + k0 + cc) : 0.f;
            gs[rr][cc] = (n < r1 && o0 + cc < Cout) ? G[(size_t)n * Cout + o0 + cc] : 0.f;
        }
        __syncthreads();
#pragma unroll 2
        for (int kk = 0; kk < 64; kk += 8) {
            const float a[4] = {zs[kk + t4][mb * 16 + g], zs[kk + t4][mb * 16 + g + 8], zs[kk + t4 + 4][mb * 16 + g],
                                zs[kk + t4 + 4][mb * 16 + g + 8]};
            const float b[2] = {gs[kk + t4][nb * 8 + g], gs[kk + t4 + 4][nb * 8 + g]};
            uint32_t ahi[4], bhi[2], blo[2];
#pragma unroll
            for (int e = 0; e < 4; e++) ahi[e] = toTf32(a[e]);
#pragma unroll
            for (int e = 0; e < 2; e++) {
                bhi[e] = toTf32(b[e]);
                blo[e] = toTf32(b[e] - __uint_as_float(bhi[e]));
            }
            if constexpr (std::is_same<TA, float>::value) {
                uint32_t alo[4];
#pragma unroll
                for (int e = 0; e < 4; e++) alo[e] = toTf32(a[e] - __uint_as_float(ahi[e]));
                mmaTf32(acc, alo, bhi);
            }
            mmaTf32(acc, ahi, blo);
            mmaTf32(acc, ahi, bhi);
        }
        if (warp == 0)
            for (int rr = 0; rr < 64; rr++) bacc += gs[rr][lane];
        __syncthreads();
    }
    const size_t stride = (size_t)K * Cout + Cout;
    float* out = partial + (size_t)split * stride;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int k = k0 + mb * 16 + g + (e >= 2 ? 8 : 0);
        const int o = o0 + nb * 8 + 2 * t4 + (e & 1);
        if (k < K && o < Cout) out[(size_t)k * Cout + o] = acc[e];
    }
    if (tk == 0 && warp == 0 && o0 + lane < Cout) out[(size_t)K * Cout + o0 + lane] = bacc;
}

__global__ void __launch_bounds__(kThreads) k_wgrad_reduce(int entries, int splits, const float* __restrict__ partial,
                                                           float* __restrict__ grad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= entries) return;
    float s = 0.f;
    for (int i = 0; i < splits; i++) s += partial[(size_t)i * entries + e];
    grad[e] += s;
}

// adjoints: accumulate segment [off, off + C) of dZ (row stride K) into gX
__global__ void __launch_bounds__(kThreads) k_adj_id(int N, int C, int off, int K, const float* __restrict__ dZ,
                                                     float* __restrict__ gX) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)N * C) return;
    const size_t n = i / C, c = i % C;
    gX[i] += dZ[n * K + off + c];
}

// neighbour mean transposed: gX[k] += sum_{n in nb(k)} invDeg[n] dZ[n]
__global__ void __launch_bounds__(kThreads) k_adj_nbmean(int N, int C, int off, int K, const int32_t* __restrict__ s,
                                                         const int32_t* __restrict__ list,
                                                         const float* __restrict__ inv, const float* __restrict__ dZ,
                                                         float* __restrict__ gX) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)N * C) return;
    const int k = (int)(i / C), c = (int)(i % C);
    float acc = 0.f;
    for (int q = s[k]; q < s[k + 1]; q++) {
        const int n = list[q];
        acc = fmaf(inv[n], dZ[(size_t)n * K + off + c], acc);
    }
    gX[i] += acc;
}

// pool transposed: gX[m] += invCnt[c] dZ[c], c = c2c[m] (m over the fine rows)
__global__ void __launch_bounds__(kThreads) k_adj_pool(int Nf, int C, int off, int K, const int32_t* __restrict__ c2c,
                                                       const float* __restrict__ invCnt, const float* __restrict__ dZ,
                                                       float* __restrict__ gX) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Nf * C) return;
    const int m = (int)(i / C), c = (int)(i % C);
    const int cc = c2c[m];
    gX[i] += invCnt[cc] * dZ[(size_t)cc * K + off + c];
}

// unpool transposed: gX[c] += sum_{m in members(c)} dZ[m] (c over the coarse rows)
__global__ void __launch_bounds__(kThreads) k_adj_unpool(int Nc, int C, int off, int K, const int32_t* __restrict__ ms,
                                                         const int32_t* __restrict__ ml, const float* __restrict__ dZ,
                                                         float* __restrict__ gX) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Nc * C) return;
    const int c = (int)(i / C), cc = (int)(i % C);
    float acc = 0.f;
    for (int q = ms[c]; q < ms[c + 1]; q++) acc += dZ[(size_t)ml[q] * K + off + cc];
    gX[i] += acc;
}

// ---------------- optimiser ----------------

template <class TW>
__global__ void __launch_bounds__(kThreads) k_adam(size_t n, float* __restrict__ p, const float* __restrict__ g,
                                                   float* __restrict__ m, float* __restrict__ v, TW* low, float lr,
                                                   float b1, float b2, float eps, float c1, float c2) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    stv(low, i, pi);
}

template <class TW>
__global__ void __launch_bounds__(kThreads) k_to_low(size_t n, const float* __restrict__ p, TW* __restrict__ low) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) stv(low, i, p[i]);
}

// Appends (b, x, A_C, deficit, A_F) of this iteration's p' system to the sample
// store (FP32, [4 + W][N] per sample, A_F as ELL [W][N]) when the iteration
// counter is a multiple of `every` and the store has room; fs (nullable) holds
// the Krylov solve's (b, b) and (r, r) for the sample's relative residual.
__global__ void __launch_bounds__(kThreads) k_harvest(const Ctl* ctl, int N, int every, int cap, const double* b,
                                                      const double* x, const double* AC, const double* AF,
                                                      const int32_t* nb, int W, const double* fs, float* store,
                                                      int* count, float* relres, unsigned int* counter) {
    if (ctl->done || every <= 0 || (ctl->currentIteration % every) != 0) return;
    const int slot = *(volatile int*)count;
    if (slot >= cap) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) {
        float* base = store + (size_t)slot * (4 + W) * N;
        const double ac = AC[n];
        double sum = 0.0;
        for (int j = 0; j < W; j++) {
            const size_t sl = (size_t)j * N + n;
            const bool in = nb[sl] >= 0;
            if (in) sum += fabs(AF[sl]);
            base[(size_t)(4 + j) * N + n] = in ? (float)AF[sl] : 0.f;
        }
        base[n] = (float)b[n];
        base[(size_t)N + n] = (float)x[n];
        base[2 * (size_t)N + n] = (float)ac;
        base[3 * (size_t)N + n] = ac != 0.0 ? (float)(1.0 - sum / ac) : 0.f;
    }
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        relres[slot] = (fs && fs[4] > 0.0) ? (float)sqrt(fs[5] / fs[4]) : -1.f;
        *count = slot + 1;
        *counter = 0u;
    }
}

// ---------------- host helpers ----------------

// Opts a kernel into more than 48 KB of dynamic shared memory, once per device.
template <class F>
void allowSmem(F* f, size_t bytes) {
    if (bytes <= 48 * 1024) return;
    static std::mutex mu;
    static std::vector<std::pair<int, const void*>> done;
    int dev = 0;
    NCK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    for (auto& d : done)
        if (d.first == dev && d.second == (const void*)f) return;
    NCK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    done.push_back({dev, (const void*)f});
}

template <class TA, class TW, int CPT, int RPT>
void launchTileR(const Ctl* ctl, int gated, const NetLayer& L, const void* P, cudaStream_t s) {
    const size_t smem =
        ((size_t)16 * RPT * (L.K + 1) + (size_t)kChunk * 16 * CPT + 16 * RPT + 1) * sizeof(float);
    allowSmem(k_layer_tile<TA, TW, CPT, RPT>, smem);
    k_layer_tile<TA, TW, CPT, RPT><<<blocksFor(L.N, 16 * RPT), 256, smem, s>>>(ctl, gated, L, (const TW*)P);
}

// 64-row tiles on large levels; 16-row tiles (4 x the blocks, 1/4 the work
// per thread) where a level has too few rows to fill the GPU.
template <class TA, class TW, int CPT>
void launchTile(const Ctl* ctl, int gated, const NetLayer& L, const void* P, cudaStream_t s) {
    if (L.N >= 148 * 64 * 4) launchTileR<TA, TW, CPT, 4>(ctl, gated, L, P, s);
    else launchTileR<TA, TW, CPT, 1>(ctl, gated, L, P, s);
}

template <class TA, class TW, int KPT>
void launchDzTile(const NetLayer& L, const void* P, float* G, float* dZ, cudaStream_t s) {
    const size_t smem = ((size_t)kTileRows * (L.Cout + 1) + (size_t)kChunk * 16 * KPT) * sizeof(float);
    allowSmem(k_layer_dz_tile<TA, TW, KPT>, smem);
    k_layer_dz_tile<TA, TW, KPT><<<blocksFor(L.N, kTileRows), 256, smem, s>>>(L, (const TW*)P, G, dZ);
}

// The tiled kernels assume every channel count divides their 256 threads.
inline bool tileable(const NetLayer& L) {
    if (L.K > 256 || 256 % L.K != 0 || L.Cout > 256 || 256 % L.Cout != 0) return false;
    for (int i = 0; i < L.nIn; i++)
        if (256 % L.in[i].C != 0) return false;
    return true;
}

template <class TA, class TW>
void launchLayerFwd(const Ctl* ctl, int gated, const NetLayer& L, const void* P, cudaStream_t s) {
    switch (tileable(L) ? L.Cout : 0) {
        case 16: launchTile<TA, TW, 1>(ctl, gated, L, P, s); return;
        case 32: launchTile<TA, TW, 2>(ctl, gated, L, P, s); return;
        case 64: launchTile<TA, TW, 4>(ctl, gated, L, P, s); return;
        case 128: launchTile<TA, TW, 8>(ctl, gated, L, P, s); return;
        default: break;
    }
    const int rows = L.K <= 64 ? 128 : 32;
    const size_t smem = (size_t)rows * (L.K + 1) * sizeof(float);
    const dim3 grid(blocksFor(L.N, rows));
    const TW* p = (const TW*)P;
    if (L.Cout >= 32) k_layer_fwd<TA, TW, 32><<<grid, rows, smem, s>>>(ctl, gated, L, p);
    else if (L.Cout >= 16) k_layer_fwd<TA, TW, 16><<<grid, rows, smem, s>>>(ctl, gated, L, p);
    else k_layer_fwd<TA, TW, 1><<<grid, rows, smem, s>>>(ctl, gated, L, p);
}

template <class TA, class TW>
void launchLayerDz(const NetLayer& L, const void* P, float* G, float* dZ, cudaStream_t s) {
    if (dZ && tileable(L)) {
        switch (L.K) {
            case 16: launchDzTile<TA, TW, 1>(L, P, G, dZ, s); return;
            case 32: launchDzTile<TA, TW, 2>(L, P, G, dZ, s); return;
            case 64: launchDzTile<TA, TW, 4>(L, P, G, dZ, s); return;
            case 128: launchDzTile<TA, TW, 8>(L, P, G, dZ, s); return;
            case 256: launchDzTile<TA, TW, 16>(L, P, G, dZ, s); return;
            default: break;
        }
    }
    k_layer_dz<TA, TW, 16><<<blocksFor(L.N), kThreads, 0, s>>>(L, (const TW*)P, G, dZ);
}

template <class T>
T* devAlloc(std::vector<void*>& list, size_t n) {
    void* p = nullptr;
    NCK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    list.push_back(p);
    NCK(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    return static_cast<T*>(p);
}

template <class T>
T* devUpload(std::vector<void*>& list, const std::vector<T>& h) {
    T* d = devAlloc<T>(list, h.size());
    if (!h.empty()) NCK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

inline int wgradSplits(int rows) { return std::min(512, std::max(1, (rows + 2047) / 2048)); }

}  // namespace

void launchHarvest(const Ctl* ctl, int N, int every, int cap, const double* b, const double* x, const double* AC,
                   const double* AF, const int32_t* nb, int W, const double* fcgScalars, float* store, int* count,
                   float* relres, unsigned int* counter, cudaStream_t s) {
    k_harvest<<<blocksFor(N), kThreads, 0, s>>>(ctl, N, every, cap, b, x, AC, AF, nb, W, fcgScalars, store, count,
                                                relres, counter);
}

// ---------------- LearnedNet ----------------

LearnedNet::~LearnedNet() { release(); }

void LearnedNet::release() {
    for (void* p : allocs_) cudaFree(p);
    allocs_.clear();
    g_.clear();
    layers_.clear();
    N0_ = 0;
    L_ = 0;
    nParams_ = 0;
}

void LearnedNet::init(const std::vector<GridLevel>& hier, const int32_t* nb, int W, int precision, uint64_t seed,
                      cudaStream_t s) {
    release();
    if (hier.empty()) throw std::runtime_error("learned preconditioner needs the multigrid hierarchy");
    nb0_ = nb;
    W0_ = W;
    // precision: 0 FP32 throughout, 1 BF16 weights and activations, 2 BF16
    // weights with FP32 activations
    actBf16_ = precision == 1 ? 1 : 0;
    wBf16_ = precision == 1 || precision == 2 ? 1 : 0;
    L_ = std::min<int>((int)hier.size(), 16);
    N0_ = hier[0].nCells;
    g_.assign((size_t)L_, NetGraphLevel{});
    C_.assign((size_t)L_, 128);
    const int chan[3] = {16, 32, 64};
    for (int l = 0; l < L_ && l < 3; l++) C_[(size_t)l] = chan[l];
    for (int l = 0; l < L_; l++) {
        const GridLevel& h = hier[(size_t)l];
        NetGraphLevel& G = g_[(size_t)l];
        G.N = h.nCells;
        std::vector<int32_t> ns((size_t)h.nCells + 1, 0), nl;
        std::vector<float> inv((size_t)h.nCells, 0.f);
        for (int c = 0; c < h.nCells; c++) {
            for (int q = h.faceStart[(size_t)c]; q < h.faceStart[(size_t)c + 1]; q++) {
                const int k = h.faceNeighbor[(size_t)q];
                if (k >= 0 && k != c) nl.push_back(k);
            }
            ns[(size_t)c + 1] = (int32_t)nl.size();
            const int d = ns[(size_t)c + 1] - ns[(size_t)c];
            inv[(size_t)c] = d > 0 ? 1.f / (float)d : 0.f;
        }
        G.nStart = devUpload(allocs_, ns);
        G.nList = devUpload(allocs_, nl);
        G.invDeg = devUpload(allocs_, inv);
        if (l + 1 < L_) G.c2c = devUpload(allocs_, h.cellToCoarse);
        if (l > 0) {
            const GridLevel& f = hier[(size_t)l - 1];
            std::vector<int32_t> ms((size_t)h.nCells + 1, 0), ml((size_t)f.nCells);
            for (int m = 0; m < f.nCells; m++) ms[(size_t)f.cellToCoarse[(size_t)m] + 1]++;
            for (int c = 0; c < h.nCells; c++) ms[(size_t)c + 1] += ms[(size_t)c];
            std::vector<int32_t> fill(ms.begin(), ms.end() - 1);
            for (int m = 0; m < f.nCells; m++) ml[(size_t)fill[(size_t)f.cellToCoarse[(size_t)m]]++] = m;
            std::vector<float> ic((size_t)h.nCells, 0.f);
            for (int c = 0; c < h.nCells; c++) {
                const int d = ms[(size_t)c + 1] - ms[(size_t)c];
                ic[(size_t)c] = d > 0 ? 1.f / (float)d : 0.f;
            }
            G.mStart = devUpload(allocs_, ms);
            G.mList = devUpload(allocs_, ml);
            G.invCnt = devUpload(allocs_, ic);
        }
    }
    buildLayers();
    // He-uniform weights, zero biases, from a fixed seed
    std::vector<float> hp(nParams_, 0.f);
    std::mt19937_64 rng(seed);
    std::vector<char> done(nParams_, 0);
    for (const NetLayer& L : layers_) {
        if (done[L.wOff]) continue;
        done[L.wOff] = 1;
        const float a = L.relu ? std::sqrt(6.f / (float)L.K) : std::sqrt(3.f / (float)L.K);
        std::uniform_real_distribution<float> U(-a, a);
        for (size_t i = 0; i < (size_t)L.K * L.Cout; i++) hp[L.wOff + i] = U(rng);
    }
    NCK(cudaMemcpy(params_, hp.data(), nParams_ * sizeof(float), cudaMemcpyHostToDevice));
    syncLowPrecision(s);
    NCK(cudaStreamSynchronize(s));
}

void LearnedNet::buildLayers() {
    const size_t tsz = actBf16_ ? sizeof(bfloat) : sizeof(float);
    auto act = [&](size_t n) { return (void*)devAlloc<unsigned char>(allocs_, n * tsz); };
    auto grd = [&](size_t n) { return devAlloc<float>(allocs_, n); };
    const int L = L_;
    std::vector<void*> H((size_t)L), E((size_t)L), S((size_t)L), D((size_t)L);
    std::vector<float*> gH((size_t)L), gE((size_t)L), gS((size_t)L), gD((size_t)L);
    for (int l = 0; l < L; l++) {
        const size_t n = (size_t)g_[(size_t)l].N * C_[(size_t)l];
        H[(size_t)l] = act(n);
        E[(size_t)l] = act(n);
        S[(size_t)l] = act(n);
        D[(size_t)l] = act(n);
        gH[(size_t)l] = grd(n);
        gE[(size_t)l] = grd(n);
        gS[(size_t)l] = grd(n);
        gD[(size_t)l] = grd(n);
    }
    feat_ = act((size_t)N0_ * 2);
    out_ = act((size_t)N0_);
    gOut_ = grd((size_t)N0_);
    // weight groups, allocated in first-use order
    std::vector<std::pair<std::string, size_t>> groups;
    size_t total = 0;
    auto group = [&](const std::string& key, int K, int Cout) -> size_t {
        for (auto& g : groups)
            if (g.first == key) return g.second;
        const size_t off = total;
        total += (size_t)K * Cout + Cout;
        groups.push_back({key, off});
        return off;
    };
    auto idIn = [&](const void* x, int C, int rows) {
        NetIn I;
        I.x = x;
        I.C = C;
        I.xf = NX_ID;
        I.srcRows = rows;
        return I;
    };
    auto mp = [&](const std::string& key, int l, void* X, float* gX, void* Y, float* gY) {
        NetLayer Ly;
        Ly.N = g_[(size_t)l].N;
        Ly.K = 2 * C_[(size_t)l];
        Ly.Cout = C_[(size_t)l];
        Ly.wOff = group(key, Ly.K, Ly.Cout);
        Ly.in[0] = idIn(X, C_[(size_t)l], Ly.N);
        NetIn I;
        I.x = X;
        I.C = C_[(size_t)l];
        I.xf = NX_NBMEAN;
        I.s = g_[(size_t)l].nStart;
        I.list = g_[(size_t)l].nList;
        I.inv = g_[(size_t)l].invDeg;
        I.srcRows = Ly.N;
        Ly.in[1] = I;
        Ly.nIn = 2;
        Ly.Y = Y;
        Ly.gY = gY;
        Ly.gIn[0] = gX;
        Ly.gIn[1] = gX;
        return Ly;
    };
    layers_.clear();
    {  // input
        NetLayer Ly;
        Ly.N = N0_;
        Ly.K = 2;
        Ly.Cout = C_[0];
        Ly.wOff = group("in", 2, C_[0]);
        Ly.in[0] = idIn(feat_, 2, N0_);
        Ly.nIn = 1;
        Ly.Y = H[0];
        Ly.gY = gH[0];
        layers_.push_back(Ly);
    }
    layers_.push_back(mp("enc0", 0, H[0], gH[0], E[0], gE[0]));
    for (int l = 1; l < L; l++) {
        NetLayer Ly;
        Ly.N = g_[(size_t)l].N;
        Ly.K = C_[(size_t)l - 1];
        Ly.Cout = C_[(size_t)l];
        Ly.wOff = group("down" + std::to_string(std::min(l, 4)), Ly.K, Ly.Cout);
        NetIn I;
        I.x = E[(size_t)l - 1];
        I.C = C_[(size_t)l - 1];
        I.xf = NX_POOL;
        I.s = g_[(size_t)l].mStart;
        I.list = g_[(size_t)l].mList;
        I.inv = g_[(size_t)l].invCnt;
        I.map = g_[(size_t)l - 1].c2c;
        I.srcRows = g_[(size_t)l - 1].N;
        Ly.in[0] = I;
        Ly.nIn = 1;
        Ly.Y = H[(size_t)l];
        Ly.gY = gH[(size_t)l];
        Ly.gIn[0] = gE[(size_t)l - 1];
        layers_.push_back(Ly);
        layers_.push_back(mp("enc" + std::to_string(std::min(l, 3)), l, H[(size_t)l], gH[(size_t)l], E[(size_t)l],
                             gE[(size_t)l]));
    }
    layers_.push_back(mp("mid" + std::to_string(std::min(L - 1, 3)), L - 1, E[(size_t)L - 1], gE[(size_t)L - 1],
                         D[(size_t)L - 1], gD[(size_t)L - 1]));
    for (int l = L - 2; l >= 0; l--) {
        NetLayer Ly;
        Ly.N = g_[(size_t)l].N;
        Ly.K = C_[(size_t)l + 1];
        Ly.Cout = C_[(size_t)l];
        Ly.wOff = group("up" + std::to_string(std::min(l, 3)), Ly.K, Ly.Cout);
        NetIn I;
        I.x = D[(size_t)l + 1];
        I.C = C_[(size_t)l + 1];
        I.xf = NX_UNPOOL;
        I.map = g_[(size_t)l].c2c;
        I.s = g_[(size_t)l + 1].mStart;
        I.list = g_[(size_t)l + 1].mList;
        I.srcRows = g_[(size_t)l + 1].N;
        Ly.in[0] = I;
        Ly.nIn = 1;
        Ly.add = E[(size_t)l];
        Ly.gAdd = gE[(size_t)l];
        Ly.Y = S[(size_t)l];
        Ly.gY = gS[(size_t)l];
        Ly.gIn[0] = gD[(size_t)l + 1];
        layers_.push_back(Ly);
        layers_.push_back(mp("dec" + std::to_string(std::min(l, 3)), l, S[(size_t)l], gS[(size_t)l], D[(size_t)l],
                             gD[(size_t)l]));
    }
    {  // output
        NetLayer Ly;
        Ly.N = N0_;
        Ly.K = C_[0];
        Ly.Cout = 1;
        Ly.relu = 0;
        Ly.wOff = group("out", C_[0], 1);
        Ly.in[0] = idIn(D[0], C_[0], N0_);
        Ly.nIn = 1;
        Ly.Y = out_;
        Ly.gY = gOut_;
        Ly.gIn[0] = gD[0];
        layers_.push_back(Ly);
    }
    nParams_ = total;
    params_ = devAlloc<float>(allocs_, nParams_);
    paramsLow_ = wBf16_ ? (void*)devAlloc<bfloat>(allocs_, nParams_) : (void*)params_;
    grad_ = devAlloc<float>(allocs_, nParams_);
    adamM_ = devAlloc<float>(allocs_, nParams_);
    adamV_ = devAlloc<float>(allocs_, nParams_);
    // training buffers: Z per layer, scratch for G and dZ, wgrad partials
    size_t maxG = 0, maxZ = 0, maxPart = 0;
    for (NetLayer& Ly : layers_) {
        Ly.Z = act((size_t)Ly.N * Ly.K);
        maxG = std::max(maxG, (size_t)Ly.N * Ly.Cout);
        maxZ = std::max(maxZ, (size_t)Ly.N * Ly.K);
        maxPart = std::max(maxPart, (size_t)wgradSplits(Ly.N) * ((size_t)Ly.K * Ly.Cout + Ly.Cout));
    }
    gpre_ = grd(maxG);
    dZ_ = grd(maxZ);
    wgPartial_ = grd(maxPart);
    Ay_ = grd((size_t)N0_);
    scal_ = devAlloc<double>(allocs_, 8);
    red_ = devAlloc<double>(allocs_, 3 * (size_t)blocksFor(N0_) + 8);
    counter_ = devAlloc<unsigned int>(allocs_, 4);
}

void LearnedNet::syncLowPrecision(cudaStream_t s) {
    if (!wBf16_) return;
    k_to_low<bfloat><<<blocksFor(nParams_), kThreads, 0, s>>>(nParams_, params_, (bfloat*)paramsLow_);
    NCK(cudaGetLastError());
}

void LearnedNet::forward(const Ctl* ctl, int gated, bool keepZ, cudaStream_t s) {
    for (NetLayer L : layers_) {
        if (!keepZ) L.Z = nullptr;
        if (actBf16_) launchLayerFwd<bfloat, bfloat>(ctl, gated, L, paramsLow_, s);
        else if (wBf16_) launchLayerFwd<float, bfloat>(ctl, gated, L, paramsLow_, s);
        else launchLayerFwd<float, float>(ctl, gated, L, paramsLow_, s);
    }
}

void LearnedNet::infer(const Ctl* ctl, int gated, const double* r, const double* AC, const double* AF,
                       const int32_t* nb, int W, float* e, cudaStream_t s) {
    const int nb0 = blocksFor(N0_);
    k_sigma<double><<<nb0, kThreads, 0, s>>>(ctl, gated, N0_, r, AC, red_, counter_, scal_);
    if (actBf16_)
        k_features<bfloat, double><<<nb0, kThreads, 0, s>>>(ctl, gated, N0_, r, AC, AF, nb, W, nullptr, scal_,
                                                             (bfloat*)feat_);
    else
        k_features<float, double><<<nb0, kThreads, 0, s>>>(ctl, gated, N0_, r, AC, AF, nb, W, nullptr, scal_,
                                                            (float*)feat_);
    forward(ctl, gated, false, s);
    if (actBf16_) k_scale_out<bfloat><<<nb0, kThreads, 0, s>>>(ctl, gated, N0_, (const bfloat*)out_, scal_, e);
    else k_scale_out<float><<<nb0, kThreads, 0, s>>>(ctl, gated, N0_, (const float*)out_, scal_, e);
}

void LearnedNet::backward(cudaStream_t s) {
    for (int i = (int)layers_.size() - 1; i >= 0; i--) {
        const NetLayer& L = layers_[(size_t)i];
        const bool needDz = L.gIn[0] != nullptr;
        if (actBf16_) launchLayerDz<bfloat, bfloat>(L, paramsLow_, gpre_, needDz ? dZ_ : nullptr, s);
        else if (wBf16_) launchLayerDz<float, bfloat>(L, paramsLow_, gpre_, needDz ? dZ_ : nullptr, s);
        else launchLayerDz<float, float>(L, paramsLow_, gpre_, needDz ? dZ_ : nullptr, s);
        // dW, db
        const int splits = wgradSplits(L.N);
        const int rowsPerSplit = (L.N + splits - 1) / splits;
        const int tilesK = (L.K + 31) / 32, tilesO = (L.Cout + 31) / 32;
        const dim3 grid((unsigned)(tilesK * tilesO), (unsigned)splits);
        if (actBf16_)
            k_wgrad<bfloat><<<grid, kThreads, 0, s>>>(L.N, L.K, L.Cout, tilesO, rowsPerSplit, (const bfloat*)L.Z, gpre_,
                                                      wgPartial_);
        else
            k_wgrad<float><<<grid, kThreads, 0, s>>>(L.N, L.K, L.Cout, tilesO, rowsPerSplit, (const float*)L.Z, gpre_,
                                                     wgPartial_);
        const int entries = L.K * L.Cout + L.Cout;
        k_wgrad_reduce<<<blocksFor(entries), kThreads, 0, s>>>(entries, splits, wgPartial_, grad_ + L.wOff);
        // adjoints of the inputs
        int off = 0;
        for (int q = 0; q < L.nIn; q++) {
            const NetIn& I = L.in[q];
            float* gX = L.gIn[q];
            if (gX) {
                const size_t n = (size_t)I.srcRows * I.C;
                switch (I.xf) {
                    case NX_ID:
                        k_adj_id<<<blocksFor(n), kThreads, 0, s>>>(I.srcRows, I.C, off, L.K, dZ_, gX);
                        break;
                    case NX_NBMEAN:
                        k_adj_nbmean<<<blocksFor(n), kThreads, 0, s>>>(I.srcRows, I.C, off, L.K, I.s, I.list, I.inv,
                                                                      dZ_, gX);
                        break;
                    case NX_POOL:
                        k_adj_pool<<<blocksFor(n), kThreads, 0, s>>>(I.srcRows, I.C, off, L.K, I.map, I.inv, dZ_, gX);
                        break;
                    default:
                        k_adj_unpool<<<blocksFor(n), kThreads, 0, s>>>(I.srcRows, I.C, off, L.K, I.s, I.list, dZ_, gX);
                        break;
                }
            }
            off += I.C;
        }
        if (L.gAdd) {
            const size_t n = (size_t)L.N * L.Cout;
            k_adj_id<<<blocksFor(n), kThreads, 0, s>>>(L.N, L.Cout, 0, L.Cout, gpre_, L.gAdd);
        }
    }
    NCK(cudaGetLastError());
}

void LearnedNet::lossAndGrad(const Sample& smp, float* lossOut, cudaStream_t s) {
    const int nb0 = blocksFor(N0_);
    k_sigma<float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, smp.b, smp.AC, red_, counter_, scal_);
    if (actBf16_)
        k_features<bfloat, float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, smp.b, smp.AC, nullptr, nullptr, 0,
                                                           smp.deficit, scal_, (bfloat*)feat_);
    else
        k_features<float, float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, smp.b, smp.AC, nullptr, nullptr, 0,
                                                          smp.deficit, scal_, (float*)feat_);
    forward(nullptr, 0, true, s);
    if (actBf16_)
        k_loss_spmv<bfloat><<<nb0, kThreads, 0, s>>>(N0_, W0_, nb0_, smp.AF, smp.AC, (const bfloat*)out_, smp.b,
                                                     smp.target, Ay_, red_, counter_, scal_);
    else
        k_loss_spmv<float><<<nb0, kThreads, 0, s>>>(N0_, W0_, nb0_, smp.AF, smp.AC, (const float*)out_, smp.b,
                                                    smp.target, Ay_, red_, counter_, scal_);
    k_loss_grad<<<nb0, kThreads, 0, s>>>(N0_, smp.b, Ay_, scal_, gOut_, lossOut);
    // zero every activation gradient except the output's, and the parameter gradient
    for (const NetLayer& L : layers_)
        if (L.gY != gOut_) NCK(cudaMemsetAsync(L.gY, 0, (size_t)L.N * L.Cout * sizeof(float), s));
    NCK(cudaMemsetAsync(grad_, 0, nParams_ * sizeof(float), s));
    backward(s);
}

void LearnedNet::predict(const float* r, const float* AC, const float* deficit, float* out, cudaStream_t s) {
    const int nb0 = blocksFor(N0_);
    k_sigma<float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, r, AC, red_, counter_, scal_);
    if (actBf16_) {
        k_features<bfloat, float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, r, AC, nullptr, nullptr, 0, deficit, scal_,
                                                           (bfloat*)feat_);
        forward(nullptr, 0, false, s);
        k_scale_out<bfloat><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, (const bfloat*)out_, scal_, out);
    } else {
        k_features<float, float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, r, AC, nullptr, nullptr, 0, deficit, scal_,
                                                          (float*)feat_);
        forward(nullptr, 0, false, s);
        k_scale_out<float><<<nb0, kThreads, 0, s>>>(nullptr, 0, N0_, (const float*)out_, scal_, out);
    }
    NCK(cudaGetLastError());
}

void LearnedNet::trainStep(const Sample& smp, float lr, int t, float* lossOut, cudaStream_t s) {
    lossAndGrad(smp, lossOut, s);
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)t), c2 = 1.f - std::pow(b2, (float)t);
    if (wBf16_)
        k_adam<bfloat><<<blocksFor(nParams_), kThreads, 0, s>>>(nParams_, params_, grad_, adamM_, adamV_,
                                                                (bfloat*)paramsLow_, lr, b1, b2, 1e-8f, c1, c2);
    else
        k_adam<float><<<blocksFor(nParams_), kThreads, 0, s>>>(nParams_, params_, grad_, adamM_, adamV_, params_, lr,
                                                               b1, b2, 1e-8f, c1, c2);
    NCK(cudaGetLastError());
}

}  // namespace axisim
