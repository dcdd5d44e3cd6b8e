// kernels_mixed.cu -- mixed-precision inner solves with FP64 iterative refinement.
//
// Momentum: the reference's 20 Jacobi sweeps (linear_solver.cu:9-33) rewritten
// in correction form, u_k = u_0 + d_k with d_{k+1} = D^-1 (r - N d_k) and
// r = b - A u_0. Jacobi is linear, so in exact arithmetic this is the same
// iterate; here r is formed once in FP64 and the sweeps on d run in FP32 over
// an FP32 copy of the off-diagonals (64 instead of 112 bytes per cell and
// sweep for u and v), then u += d in FP64. Cells whose 1/AC is zero keep d = 0,
// as the reference keeps x.
//
// Pressure correction: each V-cycle is one refinement step, r = b - A x in FP64,
// an FP32 V-cycle for the correction from zero (its first Jacobi sweep fused
// here), then x += e in FP64 (kernels in mg.cu, instantiated for float).
#include <cmath>

#include "kernels.hpp"
#include "sweep_tiles.cuh"

namespace axisim {

namespace {

constexpr int kThreads = 256;
inline int blocksFor(int n) { return (n + kThreads - 1) / kThreads; }

template <int WC>
__global__ void __launch_bounds__(kThreads) k_ir_residual_pp(const Ctl* ctl, LevelDev L, float* __restrict__ r32,
                                                             float* __restrict__ eFirst, double w, int firstSweep) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    int k[WC];
    segNeighbours<WC>(L.seg, L.nb, L.N, n, k);
    double Ax = L.AC[n] * L.x[n];
#pragma unroll
    for (int j = 0; j < WC; j++)
        if (k[j] >= 0) Ax += L.AF[(size_t)j * L.N + n] * L.x[k[j]];
    const double r = L.b[n] - Ax;
    r32[n] = (float)r;
    if (firstSweep) {
        const double ac = L.AC[n];
        eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * r / ac);
    }
}

__global__ void __launch_bounds__(kThreads) k_ir_residual_pp_gen(const Ctl* ctl, LevelDev L, float* __restrict__ r32,
                                                                 float* __restrict__ eFirst, double w,
                                                                 int firstSweep) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= L.N) return;
    double Ax = L.AC[n] * L.x[n];
    for (int j = 0; j < L.W; j++) {
        const size_t s = (size_t)j * L.N + n;
        const int k = L.nb[s];
        if (k >= 0) Ax += L.AF[s] * L.x[k];
    }
    const double r = L.b[n] - Ax;
    r32[n] = (float)r;
    if (firstSweep) {
        const double ac = L.AC[n];
        eFirst[n] = (fabs(ac) < 1.0e-30) ? 0.f : (float)(w * r / ac);
    }
}

__global__ void __launch_bounds__(kThreads) k_ir_update(const Ctl* ctl, int N, double* __restrict__ x,
                                                        const float* __restrict__ e) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) x[n] += (double)e[n];
}

template <int WC>
__global__ void __launch_bounds__(kThreads) k_ir_residual_uv(int N, int W, const int32_t* __restrict__ snb,
                                                             const int4* __restrict__ seg,
                                                             const Ctl* ctl, const double* __restrict__ AF,
                                                             const double* __restrict__ ACu,
                                                             const double* __restrict__ ACv,
                                                             const double* __restrict__ bu,
                                                             const double* __restrict__ bv,
                                                             const double* __restrict__ u,
                                                             const double* __restrict__ v,
                                                             const float* __restrict__ iu,
                                                             const float* __restrict__ iv, float* __restrict__ ru,
                                                             float* __restrict__ rv, float* __restrict__ du,
                                                             float* __restrict__ dv) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double Au = ACu[n] * u[n], Av = ACv[n] * v[n];
    if (WC > 0) {
        int k[WC > 0 ? WC : 1];
        segNeighbours<(WC > 0 ? WC : 1)>(seg, snb, N, n, k);
#pragma unroll
        for (int j = 0; j < WC; j++)
            if (k[j] >= 0) {
                const double a = AF[(size_t)j * N + n];
                Au += a * u[k[j]];
                Av += a * v[k[j]];
            }
    } else {
        for (int j = 0; j < W; j++) {
            const size_t s = (size_t)j * N + n;
            const int k = snb[s];
            if (k >= 0) {
                const double a = AF[s];
                Au += a * u[k];
                Av += a * v[k];
            }
        }
    }
    const float r_u = (float)(bu[n] - Au), r_v = (float)(bv[n] - Av);
    ru[n] = r_u;
    rv[n] = r_v;
    // first Jacobi sweep from d = 0: d1 = (r - N 0) / AC, or 0 where 1/AC is zero
    const float a_u = iu[n], a_v = iv[n];
    du[n] = (a_u != 0.f) ? r_u * a_u : 0.f;
    dv[n] = (a_v != 0.f) ? r_v * a_v : 0.f;
}

template <int WC>
__global__ void __launch_bounds__(kThreads) k_jacobi_uv32(int N, int W, const int32_t* __restrict__ snb,
                                                          const int4* __restrict__ seg,
                                                          const Ctl* ctl, const float* __restrict__ AF,
                                                          const float* __restrict__ ru, const float* __restrict__ rv,
                                                          const float* __restrict__ iu, const float* __restrict__ iv,
                                                          const float* __restrict__ xu, const float* __restrict__ xv,
                                                          float* __restrict__ yu, float* __restrict__ yv) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    if (WC > 0) {
        int k[WC > 0 ? WC : 1];
        float a[WC > 0 ? WC : 1], gu[WC > 0 ? WC : 1], gv[WC > 0 ? WC : 1];
        segNeighbours<(WC > 0 ? WC : 1)>(seg, snb, N, n, k);
#pragma unroll
        for (int j = 0; j < WC; j++) a[j] = AF[(size_t)j * N + n];
#pragma unroll
        for (int j = 0; j < WC; j++) {
            const int c = k[j] >= 0 ? k[j] : n;
            gu[j] = xu[c];
            gv[j] = xv[c];
        }
        float vu = ru[n], vv = rv[n];
#pragma unroll
        for (int j = 0; j < WC; j++)
            if (k[j] >= 0) {  // one rounding per slot, as the tile kernel (sweep_tiles.cuh)
                vu = __fmaf_rn(-a[j], gu[j], vu);
                vv = __fmaf_rn(-a[j], gv[j], vv);
            }
        const float au = iu[n], av = iv[n];
        yu[n] = (au != 0.f) ? vu * au : xu[n];
        yv[n] = (av != 0.f) ? vv * av : xv[n];
    } else {
        float vu = ru[n], vv = rv[n];
        for (int j = 0; j < W; j++) {
            const size_t s = (size_t)j * N + n;
            const int k = snb[s];
            if (k >= 0) {
                vu = __fmaf_rn(-AF[s], xu[k], vu);
                vv = __fmaf_rn(-AF[s], xv[k], vv);
            }
        }
        const float au = iu[n], av = iv[n];
        yu[n] = (au != 0.f) ? vu * au : xu[n];
        yv[n] = (av != 0.f) ? vv * av : xv[n];
    }
}

__global__ void __launch_bounds__(kThreads) k_ir_update_uv(const Ctl* ctl, int N, double* __restrict__ u,
                                                           double* __restrict__ v, const float* __restrict__ du,
                                                           const float* __restrict__ dv) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < N) {
        u[n] += (double)du[n];
        v[n] += (double)dv[n];
    }
}

}  // namespace

void launchIRResidualPP(const Ctl* ctl, const LevelDev& L0, float* r32, float* eFirst, double w, int firstSweep,
                        cudaStream_t s) {
    if (L0.W == 4) launchPDL(k_ir_residual_pp<4>, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, r32, eFirst, w, firstSweep);
    else if (L0.W == 3) launchPDL(k_ir_residual_pp<3>, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, r32, eFirst, w, firstSweep);
    else launchPDL(k_ir_residual_pp_gen, dim3(blocksFor(L0.N)), dim3(kThreads), 0, s, ctl, L0, r32, eFirst, w, firstSweep);
}

void launchIRUpdatePP(const Ctl* ctl, int N, double* x, const float* e, cudaStream_t s) {
    launchPDL(k_ir_update, dim3(blocksFor(N)), dim3(kThreads), 0, s, ctl, N, x, e);
}

void launchIRResidualUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* ACu, const double* ACv,
                        const double* bu, const double* bv, const double* u, const double* v, const float* iu32,
                        const float* iv32, float* ru, float* rv, float* du, float* dv, cudaStream_t s) {
    if (m.W == 4)
        launchPDL(k_ir_residual_uv<4>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF, ACu, ACv, bu, bv, u, v, iu32,
                                                               iv32, ru, rv, du, dv);
    else if (m.W == 3)
        launchPDL(k_ir_residual_uv<3>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF, ACu, ACv, bu, bv, u, v, iu32,
                                                               iv32, ru, rv, du, dv);
    else
        launchPDL(k_ir_residual_uv<0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF, ACu, ACv, bu, bv, u, v, iu32,
                                                               iv32, ru, rv, du, dv);
}

void launchJacobiUV32(const MeshDev& m, const Ctl* ctl, const float* AF32, const float* ru, const float* rv,
                      const float* iu32, const float* iv32, const float* du, const float* dv, float* du2, float* dv2,
                      cudaStream_t s) {
    if (m.W == 4)
        launchPDL(k_jacobi_uv32<4>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF32, ru, rv, iu32, iv32, du, dv,
                                                            du2, dv2);
    else if (m.W == 3)
        launchPDL(k_jacobi_uv32<3>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF32, ru, rv, iu32, iv32, du, dv,
                                                            du2, dv2);
    else
        launchPDL(k_jacobi_uv32<0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF32, ru, rv, iu32, iv32, du, dv,
                                                            du2, dv2);
}

void launchJacobiUV32Tiles(const MeshDev& m, const Ctl* ctl, const SweepTilesDev& t, int sweeps, const float* AF32,
                           const float* ru, const float* rv, const float* iu32, const float* iv32, const float* du,
                           const float* dv, float* du2, float* dv2, cudaStream_t s) {
    launchJacobiUVTilesT<float, kSweepK32>(m, ctl, t, sweeps, AF32, ru, rv, iu32, iv32, du, dv, du2, dv2, s);
}

cudaError_t allowJacobiUV32Tiles(int cap) { return allowJacobiUVTilesSmem<float, kSweepK32>(cap); }

void launchIRUpdateUV(const Ctl* ctl, int N, double* u, double* v, const float* du, const float* dv, cudaStream_t s) {
    launchPDL(k_ir_update_uv, dim3(blocksFor(N)), dim3(kThreads), 0, s, ctl, N, u, v, du, dv);
}

}  // namespace axisim
