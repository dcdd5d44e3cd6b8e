// kernels_fp64.cu -- FP64 kernels of the SIMPLE iteration for sm_100a.
//
// Compiled with --fmad=false: every a*b+c is two rounded operations, in the
// order the reference kernels write them, so this path reproduces the CPU
// oracle bit for bit. The kernels are HBM-bound (stencil / CSR work well under
// 1 flop/byte); the layout they read is described in device.cuh.
//
// Fusions relative to the reference launch sequence (solver.cpp:1116-1266):
//   k_momentum   clearAllCoefficients + addTransportCoefficients(u) and (v)
//                + addRadialMomentumCylindricalSource + addTransientCoefficient
//                + createMomentumPressureRhs + underRelaxEquation + buildInverseDiagonal
//                + getCorrectionCoefficients (per-cell arithmetic order unchanged)
//   k_jacobi_uv  the u and v Jacobi sweeps in one pass over the shared AF
//   k_pressure   createPPCoeff + buildInverseDiagonal(pp) + computeFaceMassFluxRhieChow
//   k_pp_rhs     createPPRhs + the p' reset
//   k_correct    updateMomentumPressure + updateMassFlux
//   k_residual   residualAll + continuityResidual + first reduction pass
// The multigrid kernels live in mg_fp64.cu.
#include <cmath>
#include <cstdio>

#include "face.cuh"
#include "kernels.hpp"
#include "sweep_tiles.cuh"

namespace axisim {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kThreads = 256;

inline int blocksFor(int n, int t = kThreads) { return (n + t - 1) / t; }

// ---------------- face helpers (solver_util.cuh:56-297) ----------------

__device__ __forceinline__ double normalCorr(const double* DU, const double* DV, double nz, double nr, int c) {
    return DU[c] * nz * nz + DV[c] * nr * nr;
}

// interpolateNormalCorrectionCoeffToFace (solver_util.cuh:126-161)
__device__ __forceinline__ double interpCorr(const MeshDev& m, const double* DU, const double* DV, int c, int f,
                                             int own, int nb) {
    const double nz = m.nZ[f], nr = m.nR[f];
    const double DP = normalCorr(DU, DV, nz, nr, c);
    if (nb < 0) return DP;
    const int o = (own == c) ? nb : own;
    const double DN = normalCorr(DU, DV, nz, nr, o);
    const double w = (own == c) ? m.wP[f] : 1.0 - m.wP[f];
    return w * DP + (1.0 - w) * DN;
}

// ---------------- set-up kernels ----------------
// preComputeVariables, face part (memory_manger.cpp:528-591)
__global__ void k_precompute_faces(MeshDev m, double* invDPN, double* wP, double* dPB, double* length2D,
                                   double* lsqWZ, double* lsqWR, double* lsqDZ, double* lsqDR) {
    pdlEnter();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.F) return;
    length2D[f] = m.area[f] / (2 * kPi * m.fcR[f]);
    const int nb = m.neighbor[f], o = m.owner[f];
    const double dzPF = m.fcZ[f] - m.ccZ[o];
    const double drPF = m.fcR[f] - m.ccR[o];
    if (nb < 0) {
        dPB[f] = fabs(dzPF * m.nZ[f] + drPF * m.nR[f]);
        invDPN[f] = 0.0;
        wP[f] = 0.0;
    } else {
        const double dzNF = m.fcZ[f] - m.ccZ[nb];
        const double drNF = m.fcR[f] - m.ccR[nb];
        const double dzPN = m.ccZ[nb] - m.ccZ[o];
        const double drPN = m.ccR[nb] - m.ccR[o];
        const double dPF = fabs(dzPF * m.nZ[f] + drPF * m.nR[f]);
        const double dNF = fabs(dzNF * m.nZ[f] + drNF * m.nR[f]);
        const double dPN = sqrt(dzPN * dzPN + drPN * drPN);
        const double denom = dPF + dNF;
        invDPN[f] = 1.0 / dPN;
        wP[f] = dNF / denom;
        dPB[f] = 0.0;
    }
    const double dz = (nb >= 0 ? m.ccZ[nb] : m.fcZ[f]) - m.ccZ[o];
    const double dr = (nb >= 0 ? m.ccR[nb] : m.fcR[f]) - m.ccR[o];
    const double w = 1.0 / (dz * dz + dr * dr);
    lsqDZ[f] = dz;
    lsqDR[f] = dr;
    lsqWZ[f] = w * dz;
    lsqWR[f] = w * dr;
}

// preComputeVariables, cell part (memory_manger.cpp:524-526, 593-613)
__global__ void k_precompute_cells(MeshDev m, const int32_t* cfs, const int32_t* cfi, const double* lsqDZ,
                                   const double* lsqDR, double* invA2D, double* IZZ, double* IZR, double* IRR) {
    pdlEnter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.N) return;
    invA2D[c] = 2.0 * kPi * m.ccR[c] / m.vol[c];
    double Szz = 0.0, Szr = 0.0, Srr = 0.0;
    for (int k = cfs[c]; k < cfs[c + 1]; k++) {
        const int f = cfi[k];
        Szz += m.lsqWZ[f] * lsqDZ[f];
        Szr += m.lsqWZ[f] * lsqDR[f];
        Srr += m.lsqWR[f] * lsqDR[f];
    }
    const double det = Szz * Srr - Szr * Szr;
    if (fabs(det) <= 1.0e-30) {
        IZZ[c] = 0.0;
        IZR[c] = 0.0;
        IRR[c] = 0.0;
        return;
    }
    IZZ[c] = Srr / det;
    IZR[c] = -Szr / det;
    IRR[c] = Szz / det;
}

// buildCellFaceCSR (memory_manger.cpp:287-323) into the [W][N] slot block
__global__ void k_build_ell(int N, int W, const int32_t* cfs, const int32_t* cfi, const int32_t* owner,
                            const int32_t* neighbor, int32_t* sface, int32_t* snb) {
    pdlEnter();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int k0 = cfs[n], deg = cfs[n + 1] - k0;
    for (int j = 0; j < W; j++) {
        int f = -1, nb = -1;
        if (j < deg) {
            f = cfi[k0 + j];
            if (owner[f] == n) nb = neighbor[f];
            else if (neighbor[f] == n) nb = owner[f];
        }
        sface[(size_t)j * N + n] = f;
        snb[(size_t)j * N + n] = nb;
    }
}

// The segment tables of segNeighbours and slotFaces (device.cuh), one thread
// per 32-cell segment; the segments without slot offsets are counted in
// nIrregular[0], those without affine faces in nIrregular[1].
__global__ void k_build_seg(int N, int W, const int32_t* __restrict__ snb, const int32_t* __restrict__ sface,
                            const int32_t* __restrict__ owner, const int32_t* __restrict__ neighbor,
                            int4* __restrict__ seg, int4* __restrict__ segF, int* __restrict__ segM,
                            int* nIrregular) {
    pdlEnter();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= (N + 31) / 32) return;
    const int a = 32 * s;
    int d[4] = {0, 0, 0, 0};
    bool ok = a + 32 <= N && W >= 1 && W <= 4;
    for (int j = 0; ok && j < W; j++) {
        d[j] = snb[(size_t)j * N + a] - a;
        for (int c = a; c < a + 32; c++) {
            const int k = snb[(size_t)j * N + c];
            if (k < 0 || k - c != d[j]) {
                ok = false;
                break;
            }
        }
    }
    int meta = ok ? 0 : -1;
    int fb[4] = {0, 0, 0, 0};
    for (int j = 0; meta >= 0 && j < W; j++) {
        const int f0 = sface[(size_t)j * N + a], t = sface[(size_t)j * N + a + 1] - f0;
        const bool o = f0 >= 0 && owner[f0] == a;
        bool aff = f0 >= 0 && (t == 1 || t == 2);
        for (int c = a; aff && c < a + 32; c++) {
            const int f = sface[(size_t)j * N + c];
            aff = f == f0 + t * (c - a) && (o ? (owner[f] == c && neighbor[f] == c + d[j])
                                              : (owner[f] == c + d[j] && neighbor[f] == c));
        }
        if (!aff) {
            meta = -1;
        } else {
            fb[j] = f0;
            meta |= (t == 2 ? 1 : 0) << j;
            meta |= (o ? 1 : 0) << (4 + j);
        }
    }
    seg[s] = ok ? make_int4(d[0], d[1], d[2], d[3]) : make_int4(kSegIrregular, 0, 0, 0);
    segF[s] = make_int4(fb[0], fb[1], fb[2], fb[3]);
    segM[s] = meta;
    if (!ok) atomicAdd(nIrregular, 1);
    if (meta < 0) atomicAdd(nIrregular + 1, 1);
}

// ---------------- iteration control ----------------
__global__ void k_iter_begin(Ctl* ctl, const volatile int* hostStop) {
    pdlEnter();
    if (ctl->done) return;
    if (hostStop && *hostStop) {
        ctl->done = 2;
        return;
    }
    if (ctl->mgErr) {  // a grid barrier of the resident V-cycle gave up
        ctl->done = 5;
        return;
    }
    if (ctl->k >= ctl->maxIter) {
        ctl->done = 3;
        return;
    }
    ctl->checked = (ctl->k % ctl->checkConv) == 0;
}

// ---------------- gradients (solver_util.cu:146-169, cuh:458-588) ----------------
struct GradArgs {
    const double* phi[5];
    BCDev bc[5];
    double* gZ[5];
    double* gR[5];
};

// Bounded to 4 resident CTAs per SM for one field (64 registers, no spills);
// two to five fields keep 3 (85 registers: the four face chains of the
// least-squares loop and their other-cell values are loaded ahead, in
// registers, with a few spills from three fields up, which measured faster
// than 2 CTAs per SM without spills).
// SCH: the scheme at compile time (0 Green-Gauss, 1 least squares) so the
// other scheme's registers stay out, or 2 to read it from `scheme`.
template <int NF, int SCH>
__global__ void __launch_bounds__(kThreads, NF == 1 ? 4 : 3) k_gradient(MeshDev m, const Ctl* ctl, GradArgs a,
                                                                       int scheme) {
    pdlEnter();
    if (ctl && ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    if (SCH == 2 ? scheme == 0 : SCH == 0) {
        double gz[NF], gr[NF], axisPhi[NF];
        double clZ = 0.0, clR = 0.0;
        bool hasAxis = false;
        for (int q = 0; q < NF; q++) gz[q] = gr[q] = axisPhi[q] = 0.0;
        for (int j = 0; j < m.W; j++) {
            const int f = m.sface[(size_t)j * N + n];
            if (f < 0) break;
            const int own = m.owner[f], nb = m.neighbor[f];
            double nz = m.nZ[f], nr = m.nR[f];
            if (nb == n) {
                nz = -nz;
                nr = -nr;
            }
            double phiF[NF];
            if (nb >= 0) {
                const int o = (own == n) ? nb : own;
                const double w = (own == n) ? m.wP[f] : 1.0 - m.wP[f];
                for (int q = 0; q < NF; q++) phiF[q] = w * a.phi[q][n] + (1.0 - w) * a.phi[q][o];
            } else {
                for (int q = 0; q < NF; q++) phiF[q] = boundaryFaceValue(m, f, a.bc[q], a.phi[q][n]);
            }
            const double rf = m.fcR[f];
            if (rf > 1.0e-30) {
                const double L = m.length2D[f];
                for (int q = 0; q < NF; q++) {
                    gz[q] += phiF[q] * nz * L;
                    gr[q] += phiF[q] * nr * L;
                }
                clZ += nz * L;
                clR += nr * L;
            } else {
                hasAxis = true;
                for (int q = 0; q < NF; q++) axisPhi[q] = phiF[q];
            }
        }
        const double inv = m.invA2D[n];
        for (int q = 0; q < NF; q++) {
            if (hasAxis) {
                gz[q] += axisPhi[q] * (-clZ);
                gr[q] += axisPhi[q] * (-clR);
            }
            a.gZ[q][n] = gz[q] * inv;
            a.gR[q][n] = gr[q] * inv;
        }
    } else if (SCH == 2 ? scheme == 1 : SCH == 1) {
        double bz[NF], br[NF], phiP[NF];
        for (int q = 0; q < NF; q++) {
            bz[q] = br[q] = 0.0;
            phiP[q] = a.phi[q][n];
        }
        // pre: the other cell's values of the NF fields, loaded ahead (null: load here)
        auto face = [&](int f, int own, int nb, double wz, double wr, const double* pre) {
            for (int q = 0; q < NF; q++) {
                double dphi;
                if (nb >= 0) {
                    const bool isOwner = (own == n);
                    const double phiNb = pre ? pre[q] : a.phi[q][isOwner ? nb : own];
                    dphi = isOwner ? (phiNb - phiP[q]) : (phiP[q] - phiNb);
                } else {
                    dphi = boundaryFaceValue(m, f, a.bc[q], phiP[q]) - phiP[q];
                }
                bz[q] += wz * dphi;
                br[q] += wr * dphi;
            }
        };
        // the first four slots' face id, owner, neighbour and weights are
        // loaded before any arithmetic, so those chains are in flight together
        int pf[4], po[4], pn[4];
        double pz[4], pr[4];
        if (m.W == 4) {
            slotFaces<4>(m, n, pf, po, pn);
        } else if (m.W == 3) {
            int f3[3], o3[3], n3[3];
            slotFaces<3>(m, n, f3, o3, n3);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                pf[j] = f3[j];
                po[j] = o3[j];
                pn[j] = n3[j];
            }
            pf[3] = -1;
            po[3] = pn[3] = -1;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) pf[j] = j < m.W ? m.sface[(size_t)j * N + n] : -1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int f = pf[j] >= 0 ? pf[j] : 0;
                po[j] = m.owner[f];
                pn[j] = m.neighbor[f];
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int f = pf[j] >= 0 ? pf[j] : 0;
            pz[j] = m.lsqWZ[f];
            pr[j] = m.lsqWR[f];
        }
        // and so are those slots' other-cell values of every field (a boundary
        // or missing slot loads the cell's own values and does not use them)
        double pv[4][NF];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int o = (pf[j] >= 0 && pn[j] >= 0) ? (po[j] == n ? pn[j] : po[j]) : n;
#pragma unroll
            for (int q = 0; q < NF; q++) pv[j][q] = a.phi[q][o];
        }
        bool more = true;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (pf[j] < 0) {
                more = false;
                break;
            }
            face(pf[j], po[j], pn[j], pz[j], pr[j], pv[j]);
        }
        for (int j = 4; more && j < m.W; j++) {
            const int f = m.sface[(size_t)j * N + n];
            if (f < 0) break;
            face(f, m.owner[f], m.neighbor[f], m.lsqWZ[f], m.lsqWR[f], nullptr);
        }
        const double izz = m.lsqIZZ[n], izr = m.lsqIZR[n], irr = m.lsqIRR[n];
        for (int q = 0; q < NF; q++) {
            a.gZ[q][n] = izz * bz[q] + izr * br[q];
            a.gR[q][n] = izr * bz[q] + irr * br[q];
        }
    } else {
        for (int q = 0; q < NF; q++) {
            a.gZ[q][n] = 0.0;
            a.gR[q][n] = 0.0;
        }
    }
}

// ---------------- momentum assembly ----------------
// Boundary face of one momentum component: diffusion BC (solver_util.cu:355-413)
// and first-order convection (solver_util.cuh:817-864).
__device__ __forceinline__ void momentumBoundary(const MeshDev& m, int n, int f, double area, double F, double mu,
                                                 const BCDev& bc, double& AC, double& b) {
    const int g = m.group[f];
    const bool valid = g >= 0 && g < bc.nGroups;
    if (valid) {
        const uint8_t t = bc.type[g];
        const double val = bc.value[g];
        const double nz = m.nZ[f], nr = m.nR[f];
        const double dPF = fabs((m.fcZ[f] - m.ccZ[n]) * nz + (m.fcR[f] - m.ccR[n]) * nr);
        const double K = mu * area / dPF;
        if (t == BC_DIRICHLET) {
            AC += K;
            b += K * val;
        } else if (t == BC_NEUMANN) {
            b += mu * area * val;
        } else if (t == BC_FULLY_DEVELOPED) {
            AC += K;
            b += K * prescribed(m, f, t, val, bc.length[g]);
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

// WC > 0: the mesh's slot count, known at compile time. Every slot's face id,
// then every face's owner, neighbour, area, 1/d_PN and mass flux are loaded
// before the per-face arithmetic (which keeps the reference's order), so the
// slot -> face -> value chains of the cell's faces are in flight together
// instead of one after another. WC = 0: any slot count, loads as needed.
template <int WC>
__global__ void __launch_bounds__(kThreads, 4) k_momentum(MeshDev m, const Ctl* ctl, BCDev bcU, BCDev bcV,
                                                       MomentumArgs a) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    constexpr int P = WC > 0 ? WC : 1;
    int pf[P], po[P], pn[P];
    double pa[P], pd[P], pm[P];
    if (WC > 0) {
        slotFaces<P>(m, n, pf, po, pn);
#pragma unroll
        for (int j = 0; j < P; j++) {
            const int f = pf[j] >= 0 ? pf[j] : 0;
            pa[j] = m.area[f];
            pd[j] = m.invDPN[f];
            pm[j] = a.conv ? a.mDot[f] : 0.0;
        }
    }
    double ACu = 0.0, ACv = 0.0, bu = 0.0, bv = 0.0, netF = 0.0;
    // WC > 0: the slots' coefficients are stored after the loop, so no store
    // sits between one slot's loads and the next's
    double afv[P];
    bool wr[P];
#pragma unroll
    for (int j = 0; j < P; j++) wr[j] = false;
#pragma unroll
    for (int j = 0; j < (WC > 0 ? WC : 32); j++) {
        if (WC == 0 && j >= m.W) break;
        const size_t s = (size_t)j * N + n;
        const int f = WC > 0 ? pf[j] : m.sface[s];
        if (f < 0) break;
        const int own = WC > 0 ? po[j] : m.owner[f], nb = WC > 0 ? pn[j] : m.neighbor[f];
        const double area = WC > 0 ? pa[j] : m.area[f];
        double F = 0.0;
        if (a.conv) {
            const double Fo = (WC > 0 ? pm[j] : a.mDot[f]) * 1.0;
            if (own == n) F = Fo;
            else if (nb == n) F = -Fo;
            if (fabs(F) <= 1.0e-30) F = 0.0;
            netF += F;
        }
        if (nb >= 0) {
            const int o = (own == n) ? nb : own;
            const double K = a.mu * area * (WC > 0 ? pd[j] : m.invDPN[f]);
            ACu += K;
            ACv += K;
            double af = 0.0 - K;
            if (a.nonOrtho) {
                bu += nonOrthoFlux(m, n, f, own, nb, a.gUZ, a.gUR, a.mu);
                bv += nonOrthoFlux(m, n, f, own, nb, a.gVZ, a.gVR, a.mu);
            }
            if (F != 0.0) {
                ACu += fmax(F, 0.0);
                ACv += fmax(F, 0.0);
                af += fmin(F, 0.0);
                if (a.scheme != CONV_UPWIND) {
                    const double udU = (F > 0.0) ? a.u[n] : a.u[o];
                    const double hoU = higherOrder(m, n, o, f, a.scheme, F, udU, a.u, a.gUZ, a.gUR);
                    bu -= F * (hoU - udU);
                    const double udV = (F > 0.0) ? a.v[n] : a.v[o];
                    const double hoV = higherOrder(m, n, o, f, a.scheme, F, udV, a.v, a.gVZ, a.gVR);
                    bv -= F * (hoV - udV);
                }
            }
            if (WC > 0) {
                afv[j] = af;
                wr[j] = true;
            } else {
                a.AF[s] = af;
                if (a.AF32) a.AF32[s] = (float)af;
            }
        } else {
            if (WC > 0) {
                afv[j] = 0.0;
                wr[j] = true;
            } else {
                a.AF[s] = 0.0;
                if (a.AF32) a.AF32[s] = 0.f;
            }
            momentumBoundary(m, n, f, area, F, a.mu, bcU, ACu, bu);
            momentumBoundary(m, n, f, area, F, a.mu, bcV, ACv, bv);
        }
    }
    if (WC > 0) {
#pragma unroll
        for (int j = 0; j < P; j++)
            if (wr[j]) {
                const size_t s = (size_t)j * N + n;
                a.AF[s] = afv[j];
                if (a.AF32) a.AF32[s] = (float)afv[j];
            }
    }
    if (a.conv) {
        ACu -= netF;
        ACv -= netF;
    }
    const double V = m.vol[n];
    const double r = m.ccR[n];
    ACv += a.mu * V / (r * r);  // hoop term, solver_util.cu:454-470
    if (a.transient && a.dt > 0.0) {  // solver_util.cu:536-578
        const double cV = a.rho * V;
        if (ctl->bdf2) {
            const double c2 = cV / (2.0 * a.dt);
            ACu += 3.0 * c2;
            bu += c2 * (4.0 * a.uOld[n] - a.uOld2[n]);
            ACv += 3.0 * c2;
            bv += c2 * (4.0 * a.vOld[n] - a.vOld2[n]);
        } else {
            const double c1 = cV / a.dt;
            ACu += c1;
            bu += c1 * a.uOld[n];
            ACv += c1;
            bv += c1 * a.vOld[n];
        }
    }
    bu += -V * a.gPZ[n];  // simple.cu:144-164
    bv += -V * a.gPR[n];
    const double al = a.alpha;  // solver_util.cu:582-600
    if (!(fabs(ACu) < 1.0e-30)) {
        const double ACo = ACu;
        ACu = ACo / al;
        bu += ((1.0 - al) / al) * ACo * a.u[n];
    }
    if (!(fabs(ACv) < 1.0e-30)) {
        const double ACo = ACv;
        ACv = ACo / al;
        bv += ((1.0 - al) / al) * ACo * a.v[n];
    }
    const double iu = (fabs(ACu) < 1.0e-30) ? 0.0 : 1.0 / ACu;  // solver_util.cu:602-612
    const double iv = (fabs(ACv) < 1.0e-30) ? 0.0 : 1.0 / ACv;
    a.ACu[n] = ACu;
    a.ACv[n] = ACv;
    a.bu[n] = bu;
    a.bv[n] = bv;
    a.invACu[n] = iu;
    a.invACv[n] = iv;
    a.DU[n] = V * iu;  // solver_util.cu:127-144
    a.DV[n] = V * iv;
    if (a.invU32) {
        a.invU32[n] = (float)iu;
        a.invV32[n] = (float)iv;
    }
}

// ---------------- momentum sweeps (linear_solver.cu:9-72) ----------------
template <int WC>
__global__ void __launch_bounds__(kThreads) k_jacobi_uv(int N, int W, const int32_t* __restrict__ snb,
                                                        const int4* __restrict__ seg,
                                                        const Ctl* ctl, const double* __restrict__ AF,
                                                        const double* __restrict__ bu, const double* __restrict__ bv,
                                                        const double* __restrict__ iu, const double* __restrict__ iv,
                                                        const double* __restrict__ xu, const double* __restrict__ xv,
                                                        double* __restrict__ yu, double* __restrict__ yv) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    // All slot loads are issued before any neighbour gather (no load waits on
    // the neighbour test); a boundary slot reads its own cell and is skipped.
    int nbs[WC];
    double af[WC];
    segNeighbours<WC>(seg, snb, N, n, nbs);
#pragma unroll
    for (int j = 0; j < WC; j++) af[j] = AF[(size_t)j * N + n];
    double gu[WC], gv[WC];
#pragma unroll
    for (int j = 0; j < WC; j++) {
        const int k = nbs[j] >= 0 ? nbs[j] : n;
        gu[j] = xu[k];
        gv[j] = xv[k];
    }
    double vu = bu[n], vv = bv[n];
#pragma unroll
    for (int j = 0; j < WC; j++) {
        if (nbs[j] >= 0) {
            vu -= af[j] * gu[j];
            vv -= af[j] * gv[j];
        }
    }
    const double au = iu[n], av = iv[n];
    yu[n] = (au != 0.0) ? vu * au : xu[n];
    yv[n] = (av != 0.0) ? vv * av : xv[n];
}

// General-width fallback (cells with more than 8 faces).
__global__ void __launch_bounds__(kThreads) k_jacobi_uv_wide(int N, int W, const int32_t* __restrict__ snb,
                                                             const Ctl* ctl, const double* __restrict__ AF,
                                                             const double* __restrict__ bu,
                                                             const double* __restrict__ bv,
                                                             const double* __restrict__ iu,
                                                             const double* __restrict__ iv,
                                                             const double* __restrict__ xu,
                                                             const double* __restrict__ xv, double* __restrict__ yu,
                                                             double* __restrict__ yv) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double vu = bu[n], vv = bv[n];
    for (int j = 0; j < W; j++) {
        const size_t s = (size_t)j * N + n;
        const int nb = snb[s];
        if (nb >= 0) {
            const double a = AF[s];
            vu -= a * xu[nb];
            vv -= a * xv[nb];
        }
    }
    const double au = iu[n], av = iv[n];
    yu[n] = (au != 0.0) ? vu * au : xu[n];
    yv[n] = (av != 0.0) ? vv * av : xv[n];
}

__global__ void __launch_bounds__(kThreads) k_gs_uv(int N, int W, const int32_t* __restrict__ snb, const Ctl* ctl,
                                                    const double* __restrict__ AF, const double* __restrict__ bu,
                                                    const double* __restrict__ bv, const double* __restrict__ iu,
                                                    const double* __restrict__ iv, double* xu, double* xv,
                                                    const int32_t* __restrict__ order, int begin, int count) {
    pdlEnter();
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int n = order[begin + t];
    double vu = bu[n], vv = bv[n];
    for (int j = 0; j < W; j++) {
        const size_t s = (size_t)j * N + n;
        const int nb = snb[s];
        if (nb >= 0) {
            const double a = AF[s];
            vu -= a * xu[nb];
            vv -= a * xv[nb];
        }
    }
    const double au = iu[n], av = iv[n];
    xu[n] = (au != 0.0) ? vu * au : xu[n];
    xv[n] = (av != 0.0) ? vv * av : xv[n];
}

__global__ void __launch_bounds__(kThreads) k_jacobi1(int N, int W, const int32_t* __restrict__ snb, const Ctl* ctl,
                                                      const double* __restrict__ AF, const double* __restrict__ b,
                                                      const double* __restrict__ inv, const double* __restrict__ x,
                                                      double* __restrict__ y) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    double v = b[n];
    for (int j = 0; j < W; j++) {
        const size_t s = (size_t)j * N + n;
        const int nb = snb[s];
        if (nb >= 0) v -= AF[s] * x[nb];
    }
    const double a = inv[n];
    y[n] = (a != 0.0) ? v * a : x[n];
}

__global__ void __launch_bounds__(kThreads) k_gs1(int N, int W, const int32_t* __restrict__ snb, const Ctl* ctl,
                                                  const double* __restrict__ AF, const double* __restrict__ b,
                                                  const double* __restrict__ inv, double* x,
                                                  const int32_t* __restrict__ order, int begin, int count) {
    pdlEnter();
    if (ctl->done) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int n = order[begin + t];
    double v = b[n];
    for (int j = 0; j < W; j++) {
        const size_t s = (size_t)j * N + n;
        const int nb = snb[s];
        if (nb >= 0) v -= AF[s] * x[nb];
    }
    const double a = inv[n];
    x[n] = (a != 0.0) ? v * a : x[n];
}

// ---------------- pressure correction system + Rhie-Chow ----------------
struct PressureArgs {
    double rho;
    const double* u;
    const double* v;
    const double* p;
    const double* gPZ;
    const double* gPR;
    const double* DU;
    const double* DV;
    double* AFpp;
    double* ACpp;
    double* invACpp;
    double* mDot;
    float* AF32;  // FP32 copies for the mixed-precision cycle (null on the FP64 path)
    float* AC32;
};

// WC > 0: the mesh's slot count; every slot's face, owner and neighbour come
// first (slotFaces), the per-face work then runs in slot order as for WC = 0.
template <int WC>
__global__ void __launch_bounds__(kThreads) k_pressure(MeshDev m, const Ctl* ctl, BCDev bcU, BCDev bcV, BCDev bcP,
                                                       PressureArgs a) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    const double rho = a.rho;
    constexpr int P = WC > 0 ? WC : 1;
    int pf[P], po[P], pn[P];
    if (WC > 0) slotFaces<P>(m, n, pf, po, pn);
    double AC = 0.0;
#pragma unroll
    for (int j = 0; j < (WC > 0 ? WC : 32); j++) {
        if (WC == 0 && j >= m.W) break;
        const size_t s = (size_t)j * N + n;
        const int f = WC > 0 ? pf[j] : m.sface[s];
        if (f < 0) break;
        const int own = WC > 0 ? po[j] : m.owner[f], nb = WC > 0 ? pn[j] : m.neighbor[f];
        const double area = m.area[f];
        const double nz = m.nZ[f], nr = m.nR[f];
        const double Df = interpCorr(m, a.DU, a.DV, n, f, own, nb);
        // createPPCoeff (simple.cu:7-88)
        if (nb >= 0) {
            const double K = rho * area * Df * m.invDPN[f];
            AC += K;
            a.AFpp[s] = 0.0 - K;
            if (a.AF32) a.AF32[s] = (float)(0.0 - K);
        } else {
            a.AFpp[s] = 0.0;
            if (a.AF32) a.AF32[s] = 0.f;
            const int g = m.group[f];
            if (g >= 0 && g < bcP.nGroups && bcP.type[g] == BC_DIRICHLET) {
                const double K = rho * area * Df / m.dPB[f];
                AC += K;
            }
        }
        // Rhie-Chow face mass flux, computed once per face by its owner
        // (solver_util.cu:171-203, solver_util.cuh:590-713)
        if (own != n) continue;
        if (area <= 1.0e-30) {
            a.mDot[f] = 0.0;
            continue;
        }
        double uF, vF;
        if (nb >= 0) {
            const double w = m.wP[f];
            uF = w * a.u[n] + (1.0 - w) * a.u[nb];
            vF = w * a.v[n] + (1.0 - w) * a.v[nb];
        } else {
            uF = boundaryFaceValue(m, f, bcU, a.u[n]);
            vF = boundaryFaceValue(m, f, bcV, a.v[n]);
        }
        const double unLin = uF * nz + vF * nr;
        double un;
        if (nb < 0) {
            const int g = m.group[f];
            if (g < 0 || g >= bcP.nGroups || bcP.type[g] != BC_DIRICHLET) {
                un = unLin;
            } else {
                const double gc = (bcP.value[g] - a.p[n]) / m.dPB[f];
                const double gn = a.gPZ[n] * nz + a.gPR[n] * nr;
                un = unLin - Df * (gc - gn);
            }
        } else {
            const double gpn = (a.p[nb] - a.p[n]) * m.invDPN[f];
            const double w = m.wP[f];
            const double gzf = w * a.gPZ[n] + (1.0 - w) * a.gPZ[nb];
            const double grf = w * a.gPR[n] + (1.0 - w) * a.gPR[nb];
            const double gfn = gzf * nz + grf * nr;
            un = unLin - Df * (gpn - gfn);
        }
        a.mDot[f] = rho * un * area;
    }
    a.ACpp[n] = AC;
    a.invACpp[n] = (fabs(AC) < 1.0e-30) ? 0.0 : 1.0 / AC;
    if (a.AC32) a.AC32[n] = (float)AC;
}

// createPPRhs (simple.cu:90-142) + the p' reset before the corrector loop
// NO: the cross-diffusion (non-orthogonal) term off (0) or on (1) at compile
// time, or read from the arguments (2); the fixed forms leave the other
// branch's registers out (32 instead of 60 registers on quads without it).
template <int WC, int NO>
__global__ void __launch_bounds__(kThreads) k_pp_rhs(MeshDev m, const Ctl* ctl, double rho, const double* mDot,
                                                     const double* DU, const double* DV, const double* gZ,
                                                     const double* gR, int cross, int zeroPP, double* bpp,
                                                     double* pp) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    constexpr int P = WC > 0 ? WC : 1;
    int pf[P], po[P], pn[P];
    if (WC > 0) slotFaces<P>(m, n, pf, po, pn);
    double imb = 0.0, crossSum = 0.0;
#pragma unroll
    for (int j = 0; j < (WC > 0 ? WC : 32); j++) {
        if (WC == 0 && j >= m.W) break;
        const int f = WC > 0 ? pf[j] : m.sface[(size_t)j * N + n];
        if (f < 0) break;
        const int own = WC > 0 ? po[j] : m.owner[f], nb = WC > 0 ? pn[j] : m.neighbor[f];
        const double md = mDot[f];
        if (own == n) imb += md;
        else if (nb == n) imb -= md;
        if (NO == 2 ? cross != 0 : NO == 1) {
            const double Df = interpCorr(m, DU, DV, n, f, own, nb);
            crossSum += nonOrthoFlux(m, n, f, own, nb, gZ, gR, rho * Df);
        }
    }
    bpp[n] = -imb + crossSum;
    if (zeroPP) pp[n] = 0.0;
}

// updateMomentumPressure + updateMassFlux (simple.cu:166-258); the owner of
// each face updates its mass flux.
struct CorrectArgs {
    double rho, alphaP;
    int nonOrtho;
    const double* pp;
    const double* gZ;
    const double* gR;
    const double* DU;
    const double* DV;
    double* u;
    double* v;
    double* p;
    double* mDot;
};

// WC > 0: the slot count at compile time; every slot's face id, owner,
// neighbour and area are loaded before the first store.
template <int WC, int NO>  // NO as k_pp_rhs's, for the non-orthogonal flux correction
__global__ void __launch_bounds__(kThreads) k_correct(MeshDev m, const Ctl* ctl, BCDev bcP, CorrectArgs a) {
    pdlEnter();
    if (ctl->done) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= m.N) return;
    const int N = m.N;
    constexpr int P = WC > 0 ? WC : 1;
    int pf[P], po[P], pn[P];
    double pa[P];
    if (WC > 0) {
        slotFaces<P>(m, n, pf, po, pn);
#pragma unroll
        for (int j = 0; j < P; j++) pa[j] = m.area[pf[j] >= 0 ? pf[j] : 0];
    }
    a.u[n] -= a.DU[n] * a.gZ[n];
    a.v[n] -= a.DV[n] * a.gR[n];
    a.p[n] += a.alphaP * a.pp[n];
    const double rho = a.rho;
#pragma unroll
    for (int j = 0; j < (WC > 0 ? WC : 32); j++) {
        if (WC == 0 && j >= m.W) break;
        const int f = WC > 0 ? pf[j] : m.sface[(size_t)j * N + n];
        if (f < 0) break;
        const int own = WC > 0 ? po[j] : m.owner[f];
        if (own != n) continue;
        const int nb = WC > 0 ? pn[j] : m.neighbor[f];
        const double area = WC > 0 ? pa[j] : m.area[f];
        if (area <= 1.0e-30) {
            a.mDot[f] = 0.0;
            continue;
        }
        const double Df = interpCorr(m, a.DU, a.DV, n, f, own, nb);
        if (nb >= 0) {
            double md = a.mDot[f];
            md -= rho * area * Df * (a.pp[nb] - a.pp[n]) * m.invDPN[f];
            if (NO == 2 ? a.nonOrtho != 0 : NO == 1) md -= nonOrthoFlux(m, n, f, own, nb, a.gZ, a.gR, rho * Df);
            a.mDot[f] = md;
            continue;
        }
        const int g = m.group[f];
        if (g < 0 || g >= bcP.nGroups) continue;
        if (bcP.type[g] == BC_DIRICHLET) {
            const double nz = m.nZ[f], nr = m.nR[f];
            const double dPB = fabs((m.fcZ[f] - m.ccZ[n]) * nz + (m.fcR[f] - m.ccR[n]) * nr);
            const double ppB = 0.0;
            a.mDot[f] -= rho * area * Df * (ppB - a.pp[n]) / dPB;
        }
    }
}

// ---------------- residuals (residuals.cuh:17-60, residuals.cu:5-100) ----------------
constexpr int kResQ = 5;  // |r_u| stat, scale_u, |r_v| stat, scale_v, continuity

__device__ __forceinline__ double normStat(double r, int norm) {
    return norm == 1 ? r * r : r;  // r is already |r|
}

__device__ __forceinline__ double combine(double a, double b, int isMax) { return isMax ? fmax(a, b) : a + b; }

template <int NT>
__device__ __forceinline__ void blockReduce(double (&v)[kResQ], const int (&isMax)[kResQ], double* out) {
    __shared__ double sh[NT / 32][kResQ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < kResQ; q++) {
        double x = v[q];
        for (int o = 16; o > 0; o >>= 1) x = combine(x, __shfl_down_sync(0xffffffffu, x, o), isMax[q]);
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < kResQ; q++) {
            double x = sh[0][q];
            for (int w = 1; w < NT / 32; w++) x = combine(x, sh[w][q], isMax[q]);
            out[q] = x;
        }
    }
}

// WC > 0: the slot count at compile time; the neighbour and face ids of
// every slot are loaded first, then every value they point to.
template <int WC>
__global__ void __launch_bounds__(kThreads) k_residual(MeshDev m, const Ctl* ctl, const double* AF, const double* ACu,
                                                       const double* ACv, const double* bu, const double* bv,
                                                       const double* u, const double* v, const double* mDot,
                                                       double* resU, double* resV, double* resC, double* scaleU,
                                                       double* scaleV, double* partial) {
    pdlEnter();
    if (ctl->done || !ctl->checked) return;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int N = m.N;
    const int normU = ctl->resNorm[0], normV = ctl->resNorm[1];
    const int isMax[kResQ] = {normU == 2, 0, normV == 2, 0, 0};
    double acc[kResQ];
    for (int q = 0; q < kResQ; q++) acc[q] = isMax[q] ? -INFINITY : 0.0;
    if (n < N) {
        double Axu = ACu[n] * u[n];
        double Axv = ACv[n] * v[n];
        const double su = Axu, sv = Axv;
        double imb = 0.0;
        if (WC > 0) {
            constexpr int P = WC > 0 ? WC : 1;
            int pb[P], pf[P], po[P], pn[P];
            double pa[P], pu[P], pv[P], pm[P];
            segNeighbours<P>(m.sseg, m.snb, N, n, pb);
            slotFaces<P>(m, n, pf, po, pn);
#pragma unroll
            for (int j = 0; j < P; j++) {
                const int c = pb[j] >= 0 ? pb[j] : n;
                const int f = pf[j] >= 0 ? pf[j] : 0;
                pa[j] = AF[(size_t)j * N + n];
                pu[j] = u[c];
                pv[j] = v[c];
                pm[j] = mDot[f];
            }
#pragma unroll
            for (int j = 0; j < P; j++) {
                if (pb[j] >= 0) {
                    Axu += pa[j] * pu[j];
                    Axv += pa[j] * pv[j];
                }
                if (pf[j] >= 0) {
                    if (po[j] == n) imb += pm[j];
                    else if (pn[j] == n) imb -= pm[j];
                }
            }
        } else {
            for (int j = 0; j < m.W; j++) {
                const size_t s = (size_t)j * N + n;
                const int nb = m.snb[s];
                if (nb >= 0) {
                    const double a = AF[s];
                    Axu += a * u[nb];
                    Axv += a * v[nb];
                }
                const int f = m.sface[s];
                if (f >= 0) {
                    const double md = mDot[f];
                    if (m.owner[f] == n) imb += md;
                    else if (m.neighbor[f] == n) imb -= md;
                }
            }
        }
        const double ru = fabs(bu[n] - Axu);
        const double rv = fabs(bv[n] - Axv);
        resU[n] = ru;
        resV[n] = rv;
        resC[n] = imb;
        scaleU[n] = su;
        scaleV[n] = sv;
        acc[0] = normStat(ru, normU);
        acc[1] = fabs(su);
        acc[2] = normStat(rv, normV);
        acc[3] = fabs(sv);
        acc[4] = fabs(imb);
    }
    blockReduce<kThreads>(acc, isMax, partial + (size_t)blockIdx.x * kResQ);
}

// Second reduction pass + residualAllHost's host arithmetic + convergence test
// + iteration counters, all on the device (no host synchronisation).
constexpr int kResS = 4;  // stat_T, |diag_T|, stat_C, |diag_C|

__global__ void __launch_bounds__(kThreads) k_iter_end(Ctl* ctl, const double* partial, const double* partialS,
                                                       int nBlocks, int N) {
    pdlEnter();
    if (ctl->done) return;
    constexpr int NQ = kResQ + kResS;
    __shared__ double sh[kThreads][NQ];
    if (ctl->checked) {
        const int isMax[NQ] = {ctl->resNorm[0] == 2, 0, ctl->resNorm[1] == 2, 0, 0,
                               ctl->resNormS[0] == 2, 0, ctl->resNormS[1] == 2, 0};
        double acc[NQ];
        for (int q = 0; q < NQ; q++) acc[q] = isMax[q] ? -INFINITY : 0.0;
#pragma unroll 4
        for (int i = threadIdx.x; i < nBlocks; i += blockDim.x) {  // unrolled: the loads of four rows in flight
            for (int q = 0; q < kResQ; q++) acc[q] = combine(acc[q], partial[(size_t)i * kResQ + q], isMax[q]);
            if (partialS)
                for (int q = 0; q < kResS; q++)
                    acc[kResQ + q] = combine(acc[kResQ + q], partialS[(size_t)i * kResS + q], isMax[kResQ + q]);
        }
        for (int q = 0; q < NQ; q++) sh[threadIdx.x][q] = acc[q];
        __syncthreads();
        for (int st = blockDim.x / 2; st > 0; st >>= 1) {
            if ((int)threadIdx.x < st)
                for (int q = 0; q < NQ; q++)
                    sh[threadIdx.x][q] = combine(sh[threadIdx.x][q], sh[threadIdx.x + st][q], isMax[q]);
            __syncthreads();
        }
    }
    if (threadIdx.x != 0) return;
    if (ctl->checked) {
        const double raw[3] = {sh[0][0], sh[0][2], sh[0][4]};
        const double diag[2] = {sh[0][1], sh[0][3]};
        const int scaleIteration = ctl->transient ? ctl->k : ctl->currentIteration;
        for (int i = 0; i < 3; i++) {
            if (!ctl->resEnabled[i]) continue;
            ctl->resVal[i] = raw[i];
            if (i < 2) {
                switch (ctl->resScale[i]) {
                    case 0: ctl->scaleVal[i] = 1.0; break;
                    case 1: ctl->scaleVal[i] = (double)N; break;
                    case 2: ctl->scaleVal[i] = sqrt((double)N); break;
                    case 3: ctl->scaleVal[i] = diag[i]; break;
                    default: break;
                }
            }
        }
        bool finite = true;
        for (int i = 0; i < 3; i++) {
            if (!ctl->resEnabled[i]) continue;
            if (i == 2 && scaleIteration < 5) ctl->scaleVal[i] = fmax(ctl->resVal[i], 0.0);
            if (ctl->scaleVal[i] == 0.0) continue;
            if (ctl->resNorm[i] == 1) ctl->resVal[i] = sqrt(ctl->resVal[i]);
            ctl->resVal[i] /= ctl->scaleVal[i];
        }
        // Temperature and Concentration entries (an unsolved scalar's system is all zero)
        for (int e = 0; e < 2; e++) {
            if (!ctl->resEnabledS[e]) continue;
            const double raw = ctl->solvedS[e] ? sh[0][kResQ + 2 * e] : 0.0;
            const double diag = ctl->solvedS[e] ? sh[0][kResQ + 2 * e + 1] : 0.0;
            ctl->resValS[e] = raw;
            switch (ctl->resScaleS[e]) {
                case 0: ctl->scaleValS[e] = 1.0; break;
                case 1: ctl->scaleValS[e] = (double)N; break;
                case 2: ctl->scaleValS[e] = sqrt((double)N); break;
                case 3: ctl->scaleValS[e] = diag; break;
                default: break;
            }
            if (ctl->scaleValS[e] == 0.0) continue;
            if (ctl->resNormS[e] == 1) ctl->resValS[e] = sqrt(ctl->resValS[e]);
            ctl->resValS[e] /= ctl->scaleValS[e];
        }
        bool any = false, conv = true;
        for (int i = 0; i < 3; i++) {
            if (!ctl->resEnabled[i]) continue;
            any = true;
            if (!(ctl->resVal[i] <= ctl->tol[i])) conv = false;
            if (!isfinite(ctl->resVal[i])) finite = false;
        }
        for (int e = 0; e < 2; e++) {
            if (!ctl->resEnabledS[e]) continue;
            any = true;
            if (!(ctl->resValS[e] <= ctl->tolS[e])) conv = false;
            if (!isfinite(ctl->resValS[e])) finite = false;
        }
        ctl->converged = any && conv;
        const int h = ctl->histCount % kMaxHist;
        ctl->hist[h][0] = (double)ctl->currentIteration;
        ctl->hist[h][1] = ctl->resVal[0];
        ctl->hist[h][2] = ctl->resVal[1];
        ctl->hist[h][3] = ctl->resVal[2];
        ctl->hist[h][4] = ctl->resValS[0];
        ctl->hist[h][5] = ctl->resValS[1];
        ctl->histCount++;
        if (ctl->converged) ctl->done = 1;
        else if (!finite) ctl->done = 4;
    }
    ctl->k++;
    ctl->currentIteration++;
    ctl->itersThisCall++;
}

// One CTA per case: sums over the case's cell range of the per-cell residual
// arrays k_residual wrote (fixed strided order, deterministic).
__global__ void __launch_bounds__(kThreads) k_case_reduce(const Ctl* ctl, BatchDev b, const double* resU,
                                                          const double* resV, const double* resC,
                                                          const double* scaleU, const double* scaleV) {
    pdlEnter();
    if (ctl->done || !ctl->checked) return;
    const int c = blockIdx.x;
    const int n0 = b.cellStart[c], n1 = b.cellStart[c + 1];
    const int normU = ctl->resNorm[0], normV = ctl->resNorm[1];
    const int isMax[kResQ] = {normU == 2, 0, normV == 2, 0, 0};
    double acc[kResQ];
    for (int q = 0; q < kResQ; q++) acc[q] = isMax[q] ? -INFINITY : 0.0;
    for (int n = n0 + (int)threadIdx.x; n < n1; n += blockDim.x) {
        acc[0] = combine(acc[0], normStat(resU[n], normU), isMax[0]);
        acc[1] += fabs(scaleU[n]);
        acc[2] = combine(acc[2], normStat(resV[n], normV), isMax[2]);
        acc[3] += fabs(scaleV[n]);
        acc[4] += fabs(resC[n]);
    }
    blockReduce<kThreads>(acc, isMax, b.raw + (size_t)c * kResQ);
}

// residualAllHost's arithmetic and the convergence test, case by case; the
// batch is done once every case has converged.
__global__ void __launch_bounds__(kThreads) k_batch_iter_end(Ctl* ctl, BatchDev b, int N) {
    pdlEnter();
    if (ctl->done) return;
    __shared__ int nConv, nBad;
    if (threadIdx.x == 0) {
        nConv = 0;
        nBad = 0;
    }
    __syncthreads();
    if (ctl->checked) {
        const int scaleIteration = ctl->transient ? ctl->k : ctl->currentIteration;
        for (int c = threadIdx.x; c < b.nCases; c += blockDim.x) {
            const double* raw = b.raw + (size_t)c * kResQ;
            double* rv = b.resVal + (size_t)c * 3;
            double* sv = b.scaleVal + (size_t)c * 3;
            const double rawv[3] = {raw[0], raw[2], raw[4]};
            const double diag[2] = {raw[1], raw[3]};
            const double Nc = (double)(b.cellStart[c + 1] - b.cellStart[c]);
            for (int i = 0; i < 3; i++) {
                if (!ctl->resEnabled[i]) continue;
                rv[i] = rawv[i];
                if (i < 2) {
                    switch (ctl->resScale[i]) {
                        case 0: sv[i] = 1.0; break;
                        case 1: sv[i] = Nc; break;
                        case 2: sv[i] = sqrt(Nc); break;
                        case 3: sv[i] = diag[i]; break;
                        default: break;
                    }
                }
            }
            bool any = false, conv = true, finite = true;
            for (int i = 0; i < 3; i++) {
                if (!ctl->resEnabled[i]) continue;
                if (i == 2 && scaleIteration < 5) sv[i] = fmax(rv[i], 0.0);
                if (sv[i] != 0.0) {
                    if (ctl->resNorm[i] == 1) rv[i] = sqrt(rv[i]);
                    rv[i] /= sv[i];
                }
                any = true;
                if (!(rv[i] <= ctl->tol[i])) conv = false;
                if (!isfinite(rv[i])) finite = false;
            }
            if (any && conv) {
                atomicAdd(&nConv, 1);
                if (b.convergedAt[c] < 0) b.convergedAt[c] = ctl->currentIteration;
            }
            if (!finite) atomicAdd(&nBad, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (ctl->checked) {
        ctl->casesConverged = nConv;
        ctl->converged = nConv == b.nCases;
        for (int i = 0; i < 3; i++) ctl->resVal[i] = b.resVal[i];  // first case, for the summary line
        const int h = ctl->histCount % kMaxHist;
        ctl->hist[h][0] = (double)ctl->currentIteration;
        ctl->hist[h][1] = b.resVal[0];
        ctl->hist[h][2] = b.resVal[1];
        ctl->hist[h][3] = b.resVal[2];
        ctl->hist[h][4] = 0.0;
        ctl->hist[h][5] = 0.0;
        ctl->histCount++;
        if (ctl->converged) ctl->done = 1;
        else if (nBad) ctl->done = 4;
    }
    ctl->k++;
    ctl->currentIteration++;
    ctl->itersThisCall++;
    (void)N;
}

__global__ void k_copy(const Ctl* ctl, double* dst, const double* src, int n) {
    pdlEnter();
    if (ctl && ctl->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

}  // namespace

// ---------------- launchers ----------------
void launchPrecompute(const MeshDev& m, const int32_t* cfs, const int32_t* cfi, double* lsqDZ, double* lsqDR,
                      cudaStream_t s) {
    launchPDL(k_precompute_faces, dim3(blocksFor(m.F)), dim3(kThreads), 0, s, m, const_cast<double*>(m.invDPN), const_cast<double*>(m.wP),
                                                            const_cast<double*>(m.dPB), const_cast<double*>(m.length2D),
                                                            const_cast<double*>(m.lsqWZ), const_cast<double*>(m.lsqWR),
                                                            lsqDZ, lsqDR);
    launchPDL(k_precompute_cells, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, cfs, cfi, lsqDZ, lsqDR, const_cast<double*>(m.invA2D),
                                                            const_cast<double*>(m.lsqIZZ), const_cast<double*>(m.lsqIZR),
                                                            const_cast<double*>(m.lsqIRR));
}

void launchBuildEll(int N, int W, const int32_t* cfs, const int32_t* cfi, const int32_t* owner,
                    const int32_t* neighbor, int32_t* sface, int32_t* snb, cudaStream_t s) {
    launchPDL(k_build_ell, dim3(blocksFor(N)), dim3(kThreads), 0, s, N, W, cfs, cfi, owner, neighbor, sface, snb);
}

void launchBuildSegments(const MeshDev& m, int4* seg, int4* segF, int* segM, int* nIrregular, cudaStream_t s) {
    launchPDL(k_build_seg, dim3(blocksFor((m.N + 31) / 32)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sface, m.owner,
              m.neighbor, seg, segF, segM, nIrregular);
}

void launchIterBegin(Ctl* ctl, const volatile int* hostStop, cudaStream_t s) {
    launchPDL(k_iter_begin, dim3(1), dim3(1), 0, s, ctl, hostStop);
}

void launchGradient(const MeshDev& m, const Ctl* ctl, int nFields, const double* const* phi, const BCDev* bc,
                    double* const* gZ, double* const* gR, int scheme, cudaStream_t s) {
    GradArgs a{};
    for (int q = 0; q < nFields; q++) {
        a.phi[q] = phi[q];
        a.bc[q] = bc[q];
        a.gZ[q] = gZ[q];
        a.gR[q] = gR[q];
    }
    const int b = blocksFor(m.N);
#define AXISIM_GRAD(NF)                                                                                         \
    (scheme == 1   ? launchPDL(k_gradient<NF, 1>, dim3(b), dim3(kThreads), 0, s, m, ctl, a, scheme)                 \
     : scheme == 0 ? launchPDL(k_gradient<NF, 0>, dim3(b), dim3(kThreads), 0, s, m, ctl, a, scheme)                 \
                   : launchPDL(k_gradient<NF, 2>, dim3(b), dim3(kThreads), 0, s, m, ctl, a, scheme))
    if (nFields == 1) AXISIM_GRAD(1);
    else if (nFields == 2) AXISIM_GRAD(2);
    else if (nFields == 3) AXISIM_GRAD(3);
    else if (nFields == 4) AXISIM_GRAD(4);
    else AXISIM_GRAD(5);
#undef AXISIM_GRAD
}

void launchMomentum(const MeshDev& m, const Ctl* ctl, const BCDev& bcU, const BCDev& bcV, const MomentumArgs& a,
                    cudaStream_t s) {
    if (m.W == 4) launchPDL(k_momentum<4>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, a);
    else if (m.W == 3) launchPDL(k_momentum<3>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, a);
    else launchPDL(k_momentum<0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, a);
}

void launchJacobiUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* bu, const double* bv,
                    const double* iu, const double* iv, const double* xu, const double* xv, double* yu, double* yv,
                    cudaStream_t s) {
    if (m.W == 4) launchPDL(k_jacobi_uv<4>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF, bu, bv, iu, iv, xu, xv, yu, yv);
    else if (m.W == 3) launchPDL(k_jacobi_uv<3>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, m.sseg, ctl, AF, bu, bv, iu, iv, xu, xv, yu, yv);
    else launchPDL(k_jacobi_uv_wide, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, ctl, AF, bu, bv, iu, iv, xu, xv, yu, yv);
}

void launchJacobiUVTiles(const MeshDev& m, const Ctl* ctl, const SweepTilesDev& t, int sweeps, const double* AF,
                         const double* bu, const double* bv, const double* invu, const double* invv,
                         const double* xu, const double* xv, double* yu, double* yv, cudaStream_t s) {
    launchJacobiUVTilesT<double, kSweepK64>(m, ctl, t, sweeps, AF, bu, bv, invu, invv, xu, xv, yu, yv, s);
}

cudaError_t allowJacobiUVTiles(int cap) { return allowJacobiUVTilesSmem<double, kSweepK64>(cap); }

void launchGaussSeidelUV(const MeshDev& m, const Ctl* ctl, const double* AF, const double* bu, const double* bv,
                         const double* iu, const double* iv, double* xu, double* xv, const int32_t* order, int begin,
                         int count, cudaStream_t s) {
    launchPDL(k_gs_uv, dim3(blocksFor(count)), dim3(kThreads), 0, s, m.N, m.W, m.snb, ctl, AF, bu, bv, iu, iv, xu, xv, order, begin,
                                                  count);
}

void launchPressureSystem(const MeshDev& m, const Ctl* ctl, const BCDev& bcU, const BCDev& bcV, const BCDev& bcP,
                          double rho, const double* u, const double* v, const double* p, const double* gPZ,
                          const double* gPR, const double* DU, const double* DV, double* AFpp, double* ACpp,
                          double* invACpp, double* mDot, float* AF32, float* AC32, cudaStream_t s) {
    PressureArgs a{rho, u, v, p, gPZ, gPR, DU, DV, AFpp, ACpp, invACpp, mDot, AF32, AC32};
    if (m.W == 4) launchPDL(k_pressure<4>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, bcP, a);
    else if (m.W == 3) launchPDL(k_pressure<3>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, bcP, a);
    else launchPDL(k_pressure<0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, bcU, bcV, bcP, a);
}

void launchPressureRhs(const MeshDev& m, const Ctl* ctl, double rho, const double* mDot, const double* DU,
                       const double* DV, const double* gZ, const double* gR, int cross, int zeroPP, double* bpp,
                       double* pp, cudaStream_t s) {
    if (m.W == 4)
        cross ? launchPDL(k_pp_rhs<4, 1>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, rho, mDot, DU, DV, gZ, gR, cross,
                          zeroPP, bpp, pp)
              : launchPDL(k_pp_rhs<4, 0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, rho, mDot, DU, DV, gZ, gR, cross,
                          zeroPP, bpp, pp);
    else if (m.W == 3)
        cross ? launchPDL(k_pp_rhs<3, 1>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, rho, mDot, DU, DV, gZ, gR, cross,
                          zeroPP, bpp, pp)
              : launchPDL(k_pp_rhs<3, 0>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, rho, mDot, DU, DV, gZ, gR, cross,
                          zeroPP, bpp, pp);
    else
        launchPDL(k_pp_rhs<0, 2>, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m, ctl, rho, mDot, DU, DV, gZ, gR, cross, zeroPP, bpp, pp);
}

void launchJacobi1(const MeshDev& m, const Ctl* ctl, const double* AF, const double* b, const double* inv,
                   const double* x, double* y, cudaStream_t s) {
    launchPDL(k_jacobi1, dim3(blocksFor(m.N)), dim3(kThreads), 0, s, m.N, m.W, m.snb, ctl, AF, b, inv, x, y);
}

void launchGaussSeidel1(const MeshDev& m, const Ctl* ctl, const double* AF, const double* b, const double* inv,
                        double* x, const int32_t* order, int begin, int count, cudaStream_t s) {
    launchPDL(k_gs1, dim3(blocksFor(count)), dim3(kThreads), 0, s, m.N, m.W, m.snb, ctl, AF, b, inv, x, order, begin, count);
}

void launchCorrect(const MeshDev& m, const Ctl* ctl, const BCDev& bcP, double rho, double alphaP, int nonOrtho,
                   const double* pp, const double* gZ, const double* gR, const double* DU, const double* DV, double* u,
                   double* v, double* p, double* mDot, cudaStream_t s) {
    CorrectArgs a{rho, alphaP, nonOrtho, pp, gZ, gR, DU, DV, u, v, p, mDot};
    const dim3 g(blocksFor(m.N)), t(kThreads);
    if (m.W == 4 && nonOrtho) launchPDL(k_correct<4, 1>, g, t, 0, s, m, ctl, bcP, a);
    else if (m.W == 4) launchPDL(k_correct<4, 0>, g, t, 0, s, m, ctl, bcP, a);
    else if (m.W == 3 && nonOrtho) launchPDL(k_correct<3, 1>, g, t, 0, s, m, ctl, bcP, a);
    else if (m.W == 3) launchPDL(k_correct<3, 0>, g, t, 0, s, m, ctl, bcP, a);
    else launchPDL(k_correct<0, 2>, g, t, 0, s, m, ctl, bcP, a);
}

void launchResiduals(const MeshDev& m, const Ctl* ctl, const double* AF, const double* ACu, const double* ACv,
                     const double* bu, const double* bv, const double* u, const double* v, const double* mDot,
                     double* resU, double* resV, double* resC, double* scaleU, double* scaleV, double* partial,
                     int* nBlocksOut, cudaStream_t s) {
    const int b = blocksFor(m.N);
    *nBlocksOut = b;
    if (m.W == 4) launchPDL(k_residual<4>, dim3(b), dim3(kThreads), 0, s, m, ctl, AF, ACu, ACv, bu, bv, u, v, mDot, resU, resV, resC, scaleU, scaleV,
                                      partial);
    else if (m.W == 3) launchPDL(k_residual<3>, dim3(b), dim3(kThreads), 0, s, m, ctl, AF, ACu, ACv, bu, bv, u, v, mDot, resU, resV, resC, scaleU, scaleV,
                                      partial);
    else launchPDL(k_residual<0>, dim3(b), dim3(kThreads), 0, s, m, ctl, AF, ACu, ACv, bu, bv, u, v, mDot, resU, resV, resC, scaleU, scaleV,
                                      partial);
}

void launchIterEnd(Ctl* ctl, const double* partial, const double* partialS, int nBlocks, int N, cudaStream_t s) {
    launchPDL(k_iter_end, dim3(1), dim3(kThreads), 0, s, ctl, partial, partialS, nBlocks, N);
}

void launchBatchIterEnd(Ctl* ctl, const BatchDev& b, const double* resU, const double* resV, const double* resC,
                        const double* scaleU, const double* scaleV, cudaStream_t s) {
    launchPDL(k_case_reduce, dim3(b.nCases), dim3(kThreads), 0, s, ctl, b, resU, resV, resC, scaleU, scaleV);
    launchPDL(k_batch_iter_end, dim3(1), dim3(kThreads), 0, s, ctl, b, 0);
}

void launchCopy(const Ctl* ctl, double* dst, const double* src, int n, cudaStream_t s) {
    launchPDL(k_copy, dim3(blocksFor(n)), dim3(kThreads), 0, s, ctl, dst, src, n);
}

}  // namespace axisim
