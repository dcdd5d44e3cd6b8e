// scalar.cu -- energy and species transport for sm_100a (FP64, --fmad=false).
//
// After the velocity / pressure corrections of a SIMPLE iteration the
// reference solves one transport equation per enabled scalar
// (solver.cpp:976-1009, 1218-1238): temperature with the thermal diffusivity
// k / (rho cp), relaxed by the momentum factor, and concentration with the
// mass diffusivity D, unrelaxed. Both convect with the volumetric flux
// mDot / rho and take capacity 1 in the unsteady term. A wall group may
// carry a Michaelis-Menten or Hill consumption law; its wall concentration
// c_w then comes from a per-face Newton solve of h (c_P - c_w) = J(c_w)
// (concentration_equation.cu:6-160) and the wall enters the row as the
// conductance A h with source A h c_w (solver_util.cu:388-411).
//
// k_scalar_wall solves the wall concentration of every reactive boundary
// face (one thread per face of a host-built list, before the assembly). k_scalar fuses, for up to
// two scalars in one pass over the cells' slots, clearAllCoefficients +
// addTransportCoefficients + addTransientCoefficient + underRelaxEquation +
// buildInverseDiagonal, each row's arithmetic in the reference's order; a
// reactive face enters it through the c_w k_scalar_wall stored. Keeping the
// Newton iteration (and pow) out of the assembly keeps its register count,
// and so its occupancy, at the level of the momentum assembly.
// k_scalar_residual is residualRaw for the scalars plus the first reduction
// pass of their monitored residuals.
#include <cmath>

#include "face.cuh"
#include "kernels.hpp"

namespace axisim {

namespace {

constexpr int kThreads = 256;

inline int blocksFor(int n) { return (n + kThreads - 1) / kThreads; }

// kinetics parameters of group g (BCDev::kin, [9][G])
struct Kin {
    double vmax, km, n, m, k2, v2, Rtot, kmN, k2M;
};

__device__ __forceinline__ Kin kinOf(const BCDev& bc, int g) {
    const int G = bc.nGroups;
    const double* k = bc.kin;
    return Kin{k[g], k[G + g], k[2 * G + g], k[3 * G + g], k[4 * G + g], k[5 * G + g], k[6 * G + g], k[7 * G + g],
               k[8 * G + g]};
}

// MichaelisMenten, dMichaelisMenten, Inhibition, dInhibition, Hill, dHill
// (concentration_equation.cu:6-88)
__device__ __forceinline__ double kinMM(const Kin& k, double c) { return (k.vmax * c) / (k.km + c); }
__device__ __forceinline__ double kinDMM(const Kin& k, double c) {
    const double inv = 1.0 / (k.km + c);
    return k.vmax * k.km * inv * inv;
}
__device__ __forceinline__ double kinInhib(const Kin& k, double c) {
    if (k.v2 == 0.0) return 1.0;
    const double cm = pow(c, k.m);
    return (1.0 - (k.v2 * cm / (k.k2M + cm)));
}
__device__ __forceinline__ double kinDInhib(const Kin& k, double c) {
    if (k.v2 == 0.0) return 0.0;
    const double cm = pow(c, k.m);
    const double cm1 = pow(c, k.m - 1.0);
    return (-(k.m * k.v2 * k.k2M) * (cm1) / ((k.k2M + cm) * (k.k2M + cm)));
}
__device__ __forceinline__ double kinHill(const Kin& k, double c) {
    const double cn = pow(c, k.n);
    return (k.vmax * cn) / (k.kmN + cn);
}
__device__ __forceinline__ double kinDHill(const Kin& k, double c) {
    const double cn = pow(c, k.n);
    const double cn1 = pow(c, k.n - 1.0);
    return ((k.n * k.vmax * k.kmN) * (cn1) / ((k.kmN + cn) * (k.kmN + cn)));
}

// wallConcentrationMichaelisMenten / wallConcentrationHill
// (concentration_equation.cu:90-160): Newton from c_w = c_P, clipped at zero,
// mixed step tolerance, at most 100 steps.
__device__ double wallConcentration(const Kin& k, bool hill, double cp, double h) {
    double cw = cp;
    const double relTol = 1e-10, absTol = 1e-14;
#pragma unroll 1
    for (int i = 0; i < 100; i++) {
        const double rate = hill ? kinHill(k, cw) : kinMM(k, cw);
        const double inhib = kinInhib(k, cw);
        const double J = rate * inhib;
        const double drate = hill ? kinDHill(k, cw) : kinDMM(k, cw);
        const double dJ = rate * kinDInhib(k, cw) + drate * inhib;
        const double F = h * (cp - cw) - J;
        const double dF = -h - dJ;
        const double step = F / dF;
        cw -= step;
        cw = fmax(0.0, cw);
        if (fabs(step) < absTol + relTol * fabs(cw)) break;
    }
    return cw;
}

// Boundary face of one scalar: the diffusion branch of addTransportCoefficients
// (solver_util.cu:355-413), reactive walls included, then first-order
// convection (solver_util.cuh:817-864).
__device__ __forceinline__ void scalarBoundary(const MeshDev& m, int n, int f, double area, double F,
                                               const ScalarDev& q, double& AC, double& b) {
    const BCDev& bc = q.bc;
    const int g = m.group[f];
    const bool valid = g >= 0 && g < bc.nGroups;
    if (valid) {
        const uint8_t t = bc.type[g];
        const double val = bc.value[g];
        const double nz = m.nZ[f], nr = m.nR[f];
        const double dPF = fabs((m.fcZ[f] - m.ccZ[n]) * nz + (m.fcR[f] - m.ccR[n]) * nr);
        const double K = q.gamma * area / dPF;
        if (t == BC_DIRICHLET) {
            AC += K;
            b += K * val;
        } else if (t == BC_NEUMANN) {
            b += q.gamma * area * val;
        } else if (t == BC_FULLY_DEVELOPED) {
            AC += K;
            b += K * prescribed(m, f, t, val, bc.length[g]);
        } else if (t == BC_MICHAELIS_MENTEN || t == BC_HILL) {
            // c_w from k_scalar_wall, which used the same h
            const double Rtot = (dPF / q.gamma) + bc.kin[6 * bc.nGroups + g];
            const double h = 1 / Rtot;
            const double cw = q.wall[f];
            AC += area * h;
            b += area * h * cw;
        }
    }
    if (F != 0.0) {
        if (!valid) {
            AC += F;
            return;
        }
        const uint8_t t = bc.type[g];
        const double val = bc.value[g];
        if (t == BC_DIRICHLET) {
            if (F < 0.0) b += -F * val;
            else AC += F;
        } else if (t == BC_NEUMANN) {
            AC += F;
        } else if (t == BC_FULLY_DEVELOPED) {
            if (F < 0.0) b += -F * prescribed(m, f, t, val, bc.length[g]);
            else AC += F;
        }
    }
}

// Reactive wall faces (solver_util.cu:388-411 with the wall solves of
// concentration_equation.cu:90-160): c_w from the owner cell's current value,
// the wall consumption A J(c_w), and c_w kept per scalar for the assembly.
// A face reactive for both scalars leaves the second one's c_w and consumption
// in cw / ocr, as the reference's shared mesh.faces arrays do.
template <int NS>
__global__ void __launch_bounds__(kThreads) k_scalar_wall(MeshDev m, const Ctl* ctl, ScalarArgs a,
                                                          const int32_t* __restrict__ faces, int nFaces) {
    pdlEnter();
    if (ctl->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nFaces) return;
    const int f = faces[i];
    const int g = m.group[f];
    const int n = m.owner[f];
#pragma unroll
    for (int q = 0; q < NS; q++) {
        const ScalarDev& sc = a.s[q];
        const BCDev& bc = sc.bc;
        if (g < 0 || g >= bc.nGroups) continue;
        const uint8_t t = bc.type[g];
        if (t != BC_MICHAELIS_MENTEN && t != BC_HILL) continue;
        const bool hill = t == BC_HILL;
        const double nz = m.nZ[f], nr = m.nR[f];
        const double dPF = fabs((m.fcZ[f] - m.ccZ[n]) * nz + (m.fcR[f] - m.ccR[n]) * nr);
        const Kin k = kinOf(bc, g);
        const double Rtot = (dPF / sc.gamma) + k.Rtot;
        const double h = 1 / Rtot;
        const double cw = wallConcentration(k, hill, sc.phi[n], h);
        sc.wall[f] = cw;
        a.cw[f] = cw;
        a.ocr[f] = m.area[f] * (hill ? kinHill(k, cw) : kinMM(k, cw)) * kinInhib(k, cw);
    }
}

template <int NS>
__global__ void __launch_bounds__(kThreads, 4) k_scalar(MeshDev m, const Ctl* ctl, ScalarArgs a) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    double AC[NS], b[NS];
    for (int q = 0; q < NS; q++) AC[q] = b[q] = 0.0;
    double netF = 0.0;
    for (int j = 0; j < m.W; j++) {
        const size_t s = (size_t)j * N + n;
        const int f = m.sface[s];
        if (f < 0) break;
        const int own = m.owner[f], nb = m.neighbor[f];
        const double area = m.area[f];
        double F = 0.0;
        if (a.conv) {
            const double Fo = a.mDot[f] * a.fluxScale;
            if (own == n) F = Fo;
            else if (nb == n) F = -Fo;
            if (fabs(F) <= 1.0e-30) F = 0.0;
            netF += F;
        }
        if (nb >= 0) {
            const int o = (own == n) ? nb : own;
            const double invD = m.invDPN[f];
#pragma unroll
            for (int q = 0; q < NS; q++) {
                const ScalarDev& sc = a.s[q];
                const double K = sc.gamma * area * invD;
                AC[q] += K;
                double af = 0.0 - K;
                if (a.nonOrtho) b[q] += nonOrthoFlux(m, n, f, own, nb, sc.gZ, sc.gR, sc.gamma);
                if (F != 0.0) {
                    AC[q] += fmax(F, 0.0);
                    af += fmin(F, 0.0);
                    if (a.scheme != CONV_UPWIND) {
                        const double ud = (F > 0.0) ? sc.phi[n] : sc.phi[o];
                        const double ho = higherOrder(m, n, o, f, a.scheme, F, ud, sc.phi, sc.gZ, sc.gR);
                        b[q] -= F * (ho - ud);
                    }
                }
                sc.AF[s] = af;
            }
        } else {
#pragma unroll
            for (int q = 0; q < NS; q++) {
                a.s[q].AF[s] = 0.0;
                scalarBoundary(m, n, f, area, F, a.s[q], AC[q], b[q]);
            }
        }
    }
    const double V = m.vol[n];
#pragma unroll
    for (int q = 0; q < NS; q++) {
        const ScalarDev& sc = a.s[q];
        double ac = AC[q], bb = b[q];
        if (a.conv) ac -= netF;
        if (a.transient && a.dt > 0.0) {  // addTransientCoefficient with capacity 1 (solver_util.cu:536-578)
            const double cV = 1.0 * V;
            if (ctl->bdf2) {
                const double c2 = cV / (2.0 * a.dt);
                ac += 3.0 * c2;
                bb += c2 * (4.0 * sc.old[n] - sc.old2[n]);
            } else {
                const double c1 = cV / a.dt;
                ac += c1;
                bb += c1 * sc.old[n];
            }
        }
        const double al = sc.alpha;  // underRelaxEquation (solver_util.cu:582-600)
        if (!(fabs(ac) < 1.0e-30)) {
            const double ACo = ac;
            ac = ACo / al;
            bb += ((1.0 - al) / al) * ACo * sc.phi[n];
        }
        sc.AC[n] = ac;
        sc.b[n] = bb;
        sc.inv[n] = (fabs(ac) < 1.0e-30) ? 0.0 : 1.0 / ac;  // buildInverseDiagonal
    }
}

// residualRaw (residuals.cuh:17-48) of the solved scalars and the first pass
// of their reductions: per block {stat_T, sum |diag_T|, stat_C, sum |diag_C|}
// (stat: |r|, r^2 or max |r| by the entry's norm). Entry FIRST + q is scalar q.
struct ScalarResArgs {
    const double* AF[2];
    const double* AC[2];
    const double* b[2];
    const double* x[2];
    double* res[2];
    double* scale[2];
};

template <int NS, int FIRST>
__global__ void __launch_bounds__(kThreads) k_scalar_residual(int N, int W, const int32_t* __restrict__ snb,
                                                              const Ctl* ctl, ScalarResArgs a, double* partial) {
    pdlEnter();
    if (ctl->done || !ctl->checked) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    bool isMax[4] = {false, false, false, false};
#pragma unroll
    for (int q = 0; q < NS; q++) {
        isMax[2 * (FIRST + q)] = ctl->resNormS[FIRST + q] == 2;
        if (isMax[2 * (FIRST + q)]) acc[2 * (FIRST + q)] = -INFINITY;
    }
    if (n < N) {
#pragma unroll
        for (int q = 0; q < NS; q++) {
            const int e = FIRST + q;
            const double* x = a.x[q];
            double Ax = a.AC[q][n] * x[n];
            const double sc = Ax;
            for (int j = 0; j < W; j++) {
                const size_t s = (size_t)j * N + n;
                const int nb = snb[s];
                if (nb >= 0) Ax += a.AF[q][s] * x[nb];
            }
            const double r = fabs(a.b[q][n] - Ax);
            a.res[q][n] = r;
            a.scale[q][n] = sc;
            acc[2 * e] = ctl->resNormS[e] == 1 ? r * r : r;
            acc[2 * e + 1] = fabs(sc);
        }
    }
    __shared__ double sh[kThreads / 32][4];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            x = isMax[q] ? fmax(x, y) : x + y;
        }
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 4; q++) {
            double x = sh[0][q];
            for (int w = 1; w < kThreads / 32; w++) x = isMax[q] ? fmax(x, sh[w][q]) : x + sh[w][q];
            partial[(size_t)blockIdx.x * 4 + q] = x;
        }
    }
}

}  // namespace

void launchScalarWall(const MeshDev& m, const Ctl* ctl, int ns, const ScalarArgs& a, const int32_t* faces,
                      int nFaces, cudaStream_t s) {
    if (nFaces <= 0) return;
    if (ns == 2) launchPDL(k_scalar_wall<2>, dim3(blocksFor(nFaces)), dim3(kThreads), 0, s, m, ctl, a, faces, nFaces);
    else launchPDL(k_scalar_wall<1>, dim3(blocksFor(nFaces)), dim3(kThreads), 0, s, m, ctl, a, faces, nFaces);
}

void launchScalarAssembly(const MeshDev& m, const Ctl* ctl, int ns, const ScalarArgs& a, cudaStream_t s) {
    if (ns == 2) launchPDL(k_scalar<2>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, a);
    else launchPDL(k_scalar<1>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, a);
}

void launchScalarResidual(const MeshDev& m, const Ctl* ctl, int ns, int first, const double* const* AF,
                          const double* const* AC, const double* const* b, const double* const* x,
                          double* const* res, double* const* scale, double* partial, cudaStream_t s) {
    ScalarResArgs a{};
    for (int q = 0; q < ns; q++) {
        a.AF[q] = AF[q];
        a.AC[q] = AC[q];
        a.b[q] = b[q];
        a.x[q] = x[q];
        a.res[q] = res[q];
        a.scale[q] = scale[q];
    }
    const dim3 g(blocksFor(m.N)), t(kThreads);
    if (ns == 2) launchPDL(k_scalar_residual<2, 0>, g, t, 0, s, m.N, m.W, m.snb, ctl, a, partial);
    else if (first == 0) launchPDL(k_scalar_residual<1, 0>, g, t, 0, s, m.N, m.W, m.snb, ctl, a, partial);
    else launchPDL(k_scalar_residual<1, 1>, g, t, 0, s, m.N, m.W, m.snb, ctl, a, partial);
}

}  // namespace axisim
