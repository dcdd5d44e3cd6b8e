// sweep_tiles.cuh -- several Jacobi sweeps of the fused u/v momentum systems
// (linear_solver.cu:9-33, u and v in one pass) per launch, out of shared
// memory. Included by kernels_fp64.cu (FP64, compiled without FMA
// contraction, bit for bit the per-sweep kernel) and kernels_mixed.cu (the
// FP32 correction sweeps).
//
// One CTA per tile (SweepTiles in host_prep.hpp). Local cell c of a tile is
// kept by thread c % blockDim.x, register slot c / blockDim.x (< K): its slot
// coefficients, right-hand sides, inverse diagonals and the local indices of
// its neighbours are loaded once; the iterate of every local cell lives in
// shared memory, two buffers of `cap` (u, v) pairs and a zero entry. A launch of s sweeps loads
// the iterate of layers 0..s, runs sweep k over layers 0..s-k and writes
// layer 0 back: per launch each coefficient crosses HBM once instead of s
// times, and the halo layers are the only cells loaded twice.
#pragma once

#include "kernels.hpp"

namespace axisim {

template <class T>
struct SweepVec;
template <>
struct SweepVec<float> {
    using type = float2;
    // the per-sweep FP32 kernel's update, contraction pinned so both kernels agree bit for bit
    static __device__ __forceinline__ float sub(float v, float a, float x) { return __fmaf_rn(-a, x, v); }
};
template <>
struct SweepVec<double> {
    using type = double2;
    // FP64: a separate multiply and subtract, as the oracle does
    static __device__ __forceinline__ double sub(double v, double a, double x) { return __dsub_rn(v, __dmul_rn(a, x)); }
};

template <class T, int WC, int K>
__global__ void __launch_bounds__(1024) k_jacobi_uv_tiles(const Ctl* ctl, SweepTilesDev t, int sweeps, int N,
                                                          const T* __restrict__ AF, const T* __restrict__ bu,
                                                          const T* __restrict__ bv, const T* __restrict__ iu,
                                                          const T* __restrict__ iv, const T* __restrict__ xu,
                                                          const T* __restrict__ xv, T* __restrict__ yu,
                                                          T* __restrict__ yv) {
    using V = typename SweepVec<T>::type;
    extern __shared__ __align__(16) unsigned char sweepSmem[];
    // two buffers of cap + 1 (u, v) pairs; entry cap of each stays zero and
    // stands in for every missing neighbour (its slot coefficient is zeroed,
    // so the update subtracts +0 * +0 = +0, which leaves every value -- -0
    // and NaN included -- exactly as skipping the slot does)
    V* X0 = reinterpret_cast<V*>(sweepSmem);
    V* X1 = X0 + (t.cap + 1);
    pdlEnter();
    if (ctl->done) return;
    const int base = t.tileStart[blockIdx.x];
    const int* le = t.layerEnd + (size_t)blockIdx.x * (t.S + 1);
    const int nX = le[sweeps], nA = le[sweeps - 1], n0 = le[0];
    const unsigned none = (unsigned)t.cap;
    T a[K][WC], cu[K], cv[K], du[K], dv[K];
    unsigned nb[K][(WC + 1) / 2];  // two local neighbour indices per word, 16 bits each
    if (threadIdx.x == 0) {
        V z;
        z.x = z.y = T(0);
        X0[t.cap] = z;
        X1[t.cap] = z;
    }
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int c = threadIdx.x + i * blockDim.x;
        cu[i] = cv[i] = du[i] = dv[i] = T(0);
#pragma unroll
        for (int j = 0; j < WC; j++) a[i][j] = T(0);
#pragma unroll
        for (int h = 0; h < (WC + 1) / 2; h++) nb[i][h] = none | (none << 16);
        if (c < nX) {
            const int g = t.gid[base + c];
            V x;
            x.x = xu[g];
            x.y = xv[g];
            X0[c] = x;
            if (c < nA) {
                const uint2 w = t.lnb[base + c];
#pragma unroll
                for (int j = 0; j < WC; j++) {
                    const unsigned raw = ((j < 2 ? w.x : w.y) >> (16 * (j & 1))) & 0xFFFFu;
                    const bool has = raw != 0xFFFFu;
                    const unsigned l = has ? raw : none;
                    nb[i][j / 2] = (j & 1) ? ((nb[i][j / 2] & 0xFFFFu) | (l << 16)) : ((nb[i][j / 2] & 0xFFFF0000u) | l);
                    a[i][j] = has ? AF[(size_t)j * N + g] : T(0);
                }
                cu[i] = bu[g];
                cv[i] = bv[g];
                du[i] = iu[g];
                dv[i] = iv[g];
            }
        }
    }
    __syncthreads();
    for (int s = 1; s <= sweeps; s++) {
        const int n = le[sweeps - s];
        const V* src = (s & 1) ? X0 : X1;
        V* dst = (s & 1) ? X1 : X0;
#pragma unroll
        for (int i = 0; i < K; i++) {
            const int c = threadIdx.x + i * blockDim.x;
            if (c < n) {
                V g[WC];
#pragma unroll
                for (int j = 0; j < WC; j++) g[j] = src[(nb[i][j / 2] >> (16 * (j & 1))) & 0xFFFFu];
                T vu = cu[i], vv = cv[i];
#pragma unroll
                for (int j = 0; j < WC; j++) {
                    vu = SweepVec<T>::sub(vu, a[i][j], g[j].x);
                    vv = SweepVec<T>::sub(vv, a[i][j], g[j].y);
                }
                const V own = src[c];
                V y;
                y.x = (du[i] != T(0)) ? vu * du[i] : own.x;
                y.y = (dv[i] != T(0)) ? vv * dv[i] : own.y;
                dst[c] = y;
            }
        }
        __syncthreads();
    }
    const V* res = (sweeps & 1) ? X1 : X0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        const int c = threadIdx.x + i * blockDim.x;
        if (c < n0) {
            const int g = t.gid[base + c];
            const V y = res[c];
            yu[g] = y.x;
            yv[g] = y.y;
        }
    }
}

template <class T, int K>
cudaError_t allowJacobiUVTilesSmem(int cap) {
    const int bytes = 2 * (cap + 1) * (int)sizeof(typename SweepVec<T>::type);
    cudaError_t e = cudaFuncSetAttribute(k_jacobi_uv_tiles<T, 4, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_jacobi_uv_tiles<T, 3, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

template <class T, int K>
void launchJacobiUVTilesT(const MeshDev& m, const Ctl* ctl, const SweepTilesDev& t, int sweeps, const T* AF,
                          const T* bu, const T* bv, const T* iu, const T* iv, const T* xu, const T* xv, T* yu, T* yv,
                          cudaStream_t s) {
    const size_t smem = 2 * ((size_t)t.cap + 1) * sizeof(typename SweepVec<T>::type);
    if (m.W == 4)
        launchPDL(k_jacobi_uv_tiles<T, 4, K>, dim3(t.nTiles), dim3(t.threads), smem, s, ctl, t, sweeps, m.N, AF, bu,
                  bv, iu, iv, xu, xv, yu, yv);
    else
        launchPDL(k_jacobi_uv_tiles<T, 3, K>, dim3(t.nTiles), dim3(t.threads), smem, s, ctl, t, sweeps, m.N, AF, bu,
                  bv, iu, iv, xu, xv, yu, yv);
}

}  // namespace axisim
