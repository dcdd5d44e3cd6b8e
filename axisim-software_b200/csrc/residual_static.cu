// residual_static.cu -- the SIMPLE residuals (momentum u, v and continuity) of
// caller-owned device arrays, computed without allocating any memory.
//
// Same arithmetic as the solver's residual kernel (residualAll +
// continuityResidual, residuals.cu:5-100): per cell |b - A x| for u and v,
// A_C x as the DIAGONAL scale, and the signed mass imbalance; then one block
// partial per 256 cells and a final pass in block order, so results do not
// depend on scheduling.
//
// Why: some callers cannot allocate device memory at the point where they want
// residuals -- a host that has handed the whole GPU to a caching allocator or
// runs under a hard memory cap, or a monitoring hook inside a time-critical
// loop where cudaMalloc/cudaFree would stall (cudaFree synchronises the whole
// device). This entry point therefore keeps its reduction scratch in a
// fixed-size file-scope device array instead of the solver's arena.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "axisim_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kQ = 5;  // stat_u, scale_u, stat_v, scale_v, continuity
constexpr int kMaxBlocks = AXISIM_STATIC_MAX_CELLS / kThreads;
constexpr int kPartialDoubles = kMaxBlocks * kQ;
constexpr int kWordDoubles = 32;  // 256 bytes of counters after the partials
constexpr int kMaxDevices = 64;

static_assert(AXISIM_STATIC_MAX_CELLS % kThreads == 0, "limit must be whole blocks");

// Partials of up to kMaxBlocks blocks, then the counters: [0] arrival ticket,
// [1] number of out-of-range indices met. 640 KiB + 256 B per device.
static __device__ __align__(256) double g_residualScratch[kPartialDoubles + kWordDoubles];

__device__ __forceinline__ double combine(double a, double b, int isMax) { return isMax ? fmax(a, b) : a + b; }

__global__ void __launch_bounds__(kThreads)
k_residual_static(int N, int F, int S, const int32_t* __restrict__ cellFaceStart,
                  const int32_t* __restrict__ cellFaceIDs, const int32_t* __restrict__ faceOwner,
                  const int32_t* __restrict__ faceNeighbor, const double* __restrict__ AF,
                  const double* __restrict__ ACu, const double* __restrict__ ACv, const double* __restrict__ bu,
                  const double* __restrict__ bv, const double* __restrict__ u, const double* __restrict__ v,
                  const double* __restrict__ mDot, int normU, int normV, double* __restrict__ resU,
                  double* __restrict__ resV, double* __restrict__ resC, double* __restrict__ sums,
                  double* scratch) {
    unsigned int* words = reinterpret_cast<unsigned int*>(scratch + kPartialDoubles);
    const int isMax[kQ] = {normU == 2, 0, normV == 2, 0, 0};
    double acc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[q] = isMax[q] ? -INFINITY : 0.0;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) {
        double Axu = ACu[n] * u[n];
        double Axv = ACv[n] * v[n];
        const double su = Axu, sv = Axv;
        double imb = 0.0;
        int bad = 0;
        const int k0 = cellFaceStart[n], k1 = cellFaceStart[n + 1];
        if (k0 < 0 || k1 < k0 || k1 > S) {
            bad = 1;
        } else {
            for (int k = k0; k < k1; k++) {
                const int f = cellFaceIDs[k];
                if (f < 0 || f >= F) {
                    bad = 1;
                    continue;
                }
                const int own = faceOwner[f], nbr = faceNeighbor[f];
                if (own < 0 || own >= N || nbr < -1 || nbr >= N) {
                    bad = 1;
                    continue;
                }
                if (nbr >= 0) {
                    const int c = (own == n) ? nbr : own;
                    const double a = AF[k];
                    Axu += a * u[c];
                    Axv += a * v[c];
                }
                const double md = mDot[f];
                if (own == n) imb += md;
                else if (nbr == n) imb -= md;
            }
        }
        if (bad) atomicAdd(&words[1], 1u);
        const double ru = fabs(bu[n] - Axu);
        const double rv = fabs(bv[n] - Axv);
        resU[n] = ru;
        resV[n] = rv;
        resC[n] = imb;
        acc[0] = normU == 1 ? ru * ru : ru;
        acc[1] = fabs(su);
        acc[2] = normV == 1 ? rv * rv : rv;
        acc[3] = fabs(sv);
        acc[4] = fabs(imb);
    }
    // block partial
    __shared__ double sh[kThreads / 32][kQ];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kQ; q++) {
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1) x = combine(x, __shfl_down_sync(0xffffffffu, x, o), isMax[q]);
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            double x = sh[0][q];
            for (int w = 1; w < kThreads / 32; w++) x = combine(x, sh[w][q], isMax[q]);
            scratch[(size_t)blockIdx.x * kQ + q] = x;
        }
        __threadfence();
        last = atomicAdd(&words[0], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block to arrive adds the partials in block order
    __threadfence();
    __shared__ double tr[kThreads][kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) acc[q] = isMax[q] ? -INFINITY : 0.0;
    const volatile double* part = scratch;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads)
#pragma unroll
        for (int q = 0; q < kQ; q++) acc[q] = combine(acc[q], part[(size_t)i * kQ + q], isMax[q]);
#pragma unroll
    for (int q = 0; q < kQ; q++) tr[threadIdx.x][q] = acc[q];
    __syncthreads();
    for (int st = kThreads / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
#pragma unroll
            for (int q = 0; q < kQ; q++) tr[threadIdx.x][q] = combine(tr[threadIdx.x][q], tr[threadIdx.x + st][q], isMax[q]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kQ; q++) sums[q] = tr[0][q];
    }
}

// Per-device address of the scratch array, looked up once per device.
std::mutex g_setupMu;
double* g_scratchPtr[kMaxDevices] = {};

void setError(char* err, size_t errLen, const char* msg) {
    if (!err || errLen == 0) return;
    std::snprintf(err, errLen, "%s", msg);
}

// Device memory of device `dev`, or managed memory (reachable from any device).
// A pointer into another GPU's memory is rejected: without peer access the
// kernel would fault on it.
bool isDevicePointerOn(const void* p, int dev) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" int axisim_residual_static(int32_t nCells, int32_t nFaces, int32_t nSlots, const int32_t* cellFaceStart,
                                      const int32_t* cellFaceIDs, const int32_t* faceOwner,
                                      const int32_t* faceNeighbor, const double* AF, const double* ACu,
                                      const double* ACv, const double* bu, const double* bv, const double* u,
                                      const double* v, const double* mDot, int32_t normU, int32_t normV,
                                      double* resU, double* resV, double* resC, double* sums, void* stream,
                                      char* err, size_t errLen) {
    char msg[160];
    if (nCells <= 0 || nFaces <= 0 || nSlots <= 0) {
        setError(err, errLen, "nCells, nFaces and nSlots must be positive");
        return AXISIM_E_ARG;
    }
    if (nCells > AXISIM_STATIC_MAX_CELLS) {
        std::snprintf(msg, sizeof msg, "nCells %d exceeds the static scratch limit of %d cells", nCells,
                      AXISIM_STATIC_MAX_CELLS);
        setError(err, errLen, msg);
        return AXISIM_E_ARG;
    }
    if (normU < 0 || normU > 2 || normV < 0 || normV > 2) {
        setError(err, errLen, "norm type must be 0 (L1), 1 (L2) or 2 (LINF)");
        return AXISIM_E_ARG;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        setError(err, errLen, "no current CUDA device");
        return AXISIM_E_CUDA;
    }
    const void* ptrs[] = {cellFaceStart, cellFaceIDs, faceOwner, faceNeighbor, AF, ACu, ACv, bu, bv, u, v, mDot,
                          resU, resV, resC, sums};
    for (const void* p : ptrs)
        if (!p || !isDevicePointerOn(p, dev)) {
            setError(err, errLen, "every array must be a device pointer on the current device");
            return AXISIM_E_ARG;
        }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // every call ends with a blocking read-back of the bad-index count, which
    // a capturing stream cannot do: refuse before touching the stream
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof msg, "cudaStreamIsCapturing: %s", cudaGetErrorString(e));
        setError(err, errLen, msg);
        return AXISIM_E_CUDA;
    }
    if (cap != cudaStreamCaptureStatusNone) {
        setError(err, errLen, "cannot be called while the stream is being captured (it reads its status back)");
        return AXISIM_E_ARG;
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setupMu);
        if (!g_scratchPtr[dev]) {
            e = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_scratchPtr[dev]), g_residualScratch);
            if (e != cudaSuccess) {
                g_scratchPtr[dev] = nullptr;
                std::snprintf(msg, sizeof msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                setError(err, errLen, msg);
                return AXISIM_E_CUDA;
            }
        }
        scratch = g_scratchPtr[dev];
    }
    unsigned int* words = reinterpret_cast<unsigned int*>(scratch + kPartialDoubles);
    // the arrival ticket and the bad-index count must start at zero
    e = cudaMemsetAsync(words, 0, kWordDoubles * sizeof(double), s);
    if (e == cudaSuccess) {
        const int blocks = (nCells + kThreads - 1) / kThreads;
        k_residual_static<<<blocks, kThreads, 0, s>>>(nCells, nFaces, nSlots, cellFaceStart, cellFaceIDs, faceOwner,
                                                      faceNeighbor, AF, ACu, ACv, bu, bv, u, v, mDot, normU, normV,
                                                      resU, resV, resC, sums, scratch);
        e = cudaGetLastError();
    }
    unsigned int bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, words + 1, sizeof bad, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        std::snprintf(msg, sizeof msg, "CUDA: %s", cudaGetErrorString(e));
        setError(err, errLen, msg);
        return AXISIM_E_CUDA;
    }
    if (bad) {
        std::snprintf(msg, sizeof msg, "%u cells met an out-of-range slot, face or cell index (skipped)", bad);
        setError(err, errLen, msg);
        return AXISIM_E_MESH;
    }
    setError(err, errLen, "");
    return AXISIM_OK;
}
