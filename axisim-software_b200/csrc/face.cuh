// face.cuh -- per-face discretisation helpers shared by the FP64 assembly
// kernels (momentum in kernels_fp64.cu, the transported scalars in scalar.cu).
// Compiled with --fmad=false in both, so every a*b+c stays two rounded
// operations in the reference's order.
#pragma once

#include <cstdint>

#include "device.cuh"

namespace axisim {

// BCType (structs/boundary_struct.h:88-97) and ConvectionScheme values
constexpr uint8_t BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_FULLY_DEVELOPED = 2, BC_MICHAELIS_MENTEN = 3, BC_HILL = 4;
constexpr int CONV_UPWIND = 0, CONV_CENTRAL = 1, CONV_SOU = 2;

// prescribedBoundaryFaceValue (solver_util.cuh:223-238)
__device__ __forceinline__ double prescribed(const MeshDev& m, int f, uint8_t type, double value, double len) {
    if (type != BC_FULLY_DEVELOPED) return value;
    const double nz = m.nZ[f], nr = m.nR[f];
    const double along = m.fcR[f] * nz * nz + m.fcZ[f] * nr * nr;
    const double x = along / len;
    return value * (1.0 - x * x);
}

// interpolateFieldToFace, boundary branch (solver_util.cuh:264-296)
__device__ __forceinline__ double boundaryFaceValue(const MeshDev& m, int f, const BCDev& bc, double phiP) {
    const int g = m.group[f];
    if (g < 0 || g >= bc.nGroups) return phiP;
    const uint8_t t = bc.type[g];
    const double val = bc.value[g];
    if (t == BC_DIRICHLET || t == BC_FULLY_DEVELOPED) return prescribed(m, f, t, val, bc.length[g]);
    if (t == BC_NEUMANN) return phiP + val * m.dPB[f];
    return phiP;
}

// nonOrthoScalarDiffusionFlux (solver_util.cuh:383-430)
__device__ __forceinline__ double nonOrthoFlux(const MeshDev& m, int c, int f, int own, int nb, const double* gZ,
                                               const double* gR, double gamma) {
    if (nb < 0) return 0.0;
    const int o = (own == c) ? nb : own;
    double nz = m.nZ[f], nr = m.nR[f];
    if (nb == c) {
        nz = -nz;
        nr = -nr;
    }
    const double a = m.area[f];
    const double dz = m.ccZ[o] - m.ccZ[c];
    const double dr = m.ccR[o] - m.ccR[c];
    const double aOverNd = a * m.invDPN[f];
    const double Tz = a * nz - aOverNd * dz;
    const double Tr = a * nr - aOverNd * dr;
    const double w = (own == c) ? m.wP[f] : 1.0 - m.wP[f];
    const double gfz = w * gZ[c] + (1.0 - w) * gZ[o];
    const double gfr = w * gR[c] + (1.0 - w) * gR[o];
    return gamma * (Tz * gfz + Tr * gfr);
}

// Higher-order face value of the deferred correction (solver_util.cuh:724-768)
__device__ __forceinline__ double higherOrder(const MeshDev& m, int n, int o, int f, int scheme, double F, double phiUD,
                                              const double* phi, const double* gZ, const double* gR) {
    if (scheme == CONV_CENTRAL) {
        const double w = (m.owner[f] == n) ? m.wP[f] : 1.0 - m.wP[f];
        return w * phi[n] + (1.0 - w) * phi[o];
    }
    if (scheme == CONV_SOU) {
        const int up = (F > 0.0) ? n : o;
        const double dz = m.fcZ[f] - m.ccZ[up];
        const double dr = m.fcR[f] - m.ccR[up];
        const double ho = phi[up] + gZ[up] * dz + gR[up] * dr;
        const double lo = fmin(phi[n], phi[o]);
        const double hi = fmax(phi[n], phi[o]);
        return fmin(fmax(ho, lo), hi);
    }
    return phiUD;
}

}  // namespace axisim
