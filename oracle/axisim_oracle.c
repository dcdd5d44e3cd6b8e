/*
 * axisim_oracle.c -- CPU restatement of AxiSim's SIMPLE loop (TEST INFRASTRUCTURE).
 *
 * This file is the parity oracle for the CUDA path. It is loaded only by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py, never by the
 * product. It follows the reference sources cited beside each routine:
 *
 *   solver/source/solver.cpp:1034-1298      order of operations (time + SIMPLE loop)
 *   solver/source/solver_util.cu:127-612    discretisation kernels
 *   solver/header/solver_util.cuh:56-865    face helpers
 *   solver/source/simple.cu:7-258           p' assembly, Rhie-Chow, corrections
 *   solver/source/multigrid.cu:79-325       hierarchy construction
 *   solver/source/multigrid.cu:350-662      Galerkin, transfers, smoothers, V-cycle
 *   solver/source/linear_solver.cu:9-146    Jacobi / multicolour Gauss-Seidel
 *   solver/source/residuals.cu:5-100        monitored residuals
 *   manager/source/memory_manger.cpp:287-617 CSR, colouring, geometry precompute
 *   structs/multiblock.h:59-444             multiblock mesh packing
 *
 * Per-cell and per-face loops are OpenMP-parallel (each iteration writes only
 * its own outputs, as the reference's one-thread-per-cell kernels do), so the
 * result does not depend on the thread count. Sums that the reference does with
 * atomicAdd or a tree reduction are done here in ascending index order.
 */
#include "axisim_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

enum { BC_DIRICHLET = 0, BC_NEUMANN = 1, BC_FULLY_DEVELOPED = 2, BC_MICHAELIS_MENTEN = 3, BC_HILL = 4 };
enum { CONV_UPWIND = 0, CONV_CENTRAL = 1, CONV_SOU = 2, CONV_QUICK = 3 };
enum { GRAD_GG = 0, GRAD_LSQ = 1 };
enum { NORM_L1 = 0, NORM_L2 = 1, NORM_LINF = 2 };
enum { SCALE_NONE = 0, SCALE_N = 1, SCALE_SQRT_N = 2, SCALE_DIAG = 3 };

void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static void* xcalloc(size_t n, size_t sz) {
    void* p = calloc(n ? n : 1, sz);
    if (!p) abort();
    return p;
}

/* ======================================================================
 * Multiblock packer -- structs/multiblock.h:59-444
 * ====================================================================== */
typedef struct { double z, r; } node2;

typedef struct {
    int nr, nz, globalOffset;
    node2* nodes; /* (nr+1)*(nz+1), index I*(nz+1)+J */
    int edgeGroup[4];
} mb_block;

struct orc_packed {
    int nCells, nFaces, nRefs;
    int cap;
    int32_t *faceOwner, *faceNeighbor, *faceGroup;
    double *faceNZ, *faceNR, *faceCZ, *faceCR, *faceArea;
    double *cellCZ, *cellCR, *cellA2D, *cellVol;
    int32_t *cellFaceStart, *cellFaceIDs;
};

/* multiblock.h:59-80 generateFaces */
static double* mb_generate_faces(double length, int n, int grading, double coef, double start) {
    double* faces = (double*)xcalloc((size_t)n + 1, sizeof(double));
    double* d = (double*)xcalloc((size_t)n, sizeof(double));
    for (int k = 0; k < n; k++) d[k] = length / n;
    if (grading == 1 && n > 1 && coef > 0.0 && coef != 1.0) {
        const double d0 = length * (coef - 1.0) / (pow(coef, n) - 1.0);
        for (int k = 0; k < n; k++) d[k] = d0 * pow(coef, k);
    }
    double x = start;
    faces[0] = start;
    for (int k = 0; k < n; k++) { x += d[k]; faces[k + 1] = x; }
    free(d);
    return faces;
}

static inline node2 mb_node(const mb_block* b, int I, int J) { return b->nodes[I * (b->nz + 1) + J]; }
static inline int mb_cell(const mb_block* b, int i, int j) { return b->globalOffset + i * b->nz + j; }

/* multiblock.h:180-187 edgeCorners; Edge order West, East, South, North */
static void mb_edge_corners(const mb_block* b, int e, node2* s, node2* t) {
    switch (e) {
    case 0: *s = mb_node(b, 0, 0);     *t = mb_node(b, b->nr, 0);     break;
    case 1: *s = mb_node(b, 0, b->nz); *t = mb_node(b, b->nr, b->nz); break;
    case 2: *s = mb_node(b, 0, 0);     *t = mb_node(b, 0, b->nz);     break;
    default:*s = mb_node(b, b->nr, 0); *t = mb_node(b, b->nr, b->nz); break;
    }
}
static inline int mb_edge_count(const mb_block* b, int e) { return (e <= 1) ? b->nr : b->nz; }

/* multiblock.h:298-306 edgeFace */
static void mb_edge_face(const mb_block* b, int e, int k, int* local, node2* n0, node2* n1) {
    switch (e) {
    case 0: *local = k * b->nz;                 *n0 = mb_node(b, k, 0);     *n1 = mb_node(b, k + 1, 0);     break;
    case 1: *local = k * b->nz + b->nz - 1;     *n0 = mb_node(b, k, b->nz); *n1 = mb_node(b, k + 1, b->nz); break;
    case 2: *local = k;                         *n0 = mb_node(b, 0, k);     *n1 = mb_node(b, 0, k + 1);     break;
    default:*local = (b->nr - 1) * b->nz + k;   *n0 = mb_node(b, b->nr, k); *n1 = mb_node(b, b->nr, k + 1); break;
    }
}
/* multiblock.h:168-177 edgeCells */
static int mb_edge_cell(const mb_block* b, int e, int k) {
    switch (e) {
    case 0: return k * b->nz;
    case 1: return k * b->nz + b->nz - 1;
    case 2: return k;
    default: return (b->nr - 1) * b->nz + k;
    }
}

/* multiblock.h:272-295 quadCentroidArea */
static void mb_quad(node2 p0, node2 p1, node2 p2, node2 p3, double* cz, double* cr, double* area) {
    node2 p[4] = { p0, p1, p2, p3 };
    double A = 0.0, Cz = 0.0, Cr = 0.0;
    for (int k = 0; k < 4; k++) {
        node2 a = p[k], b = p[(k + 1) & 3];
        double cross = a.z * b.r - b.z * a.r;
        A += cross;
        Cz += (a.z + b.z) * cross;
        Cr += (a.r + b.r) * cross;
    }
    A *= 0.5;
    if (fabs(A) < 1e-30) {
        *cz = 0.25 * (p0.z + p1.z + p2.z + p3.z);
        *cr = 0.25 * (p0.r + p1.r + p2.r + p3.r);
        *area = 0.0;
        return;
    }
    *cz = Cz / (6.0 * A);
    *cr = Cr / (6.0 * A);
    *area = fabs(A);
}

typedef struct { int* data; int n, cap; } ivec;
static void ivec_push(ivec* v, int x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 4; v->data = (int*)realloc(v->data, (size_t)v->cap * sizeof(int)); }
    v->data[v->n++] = x;
}

static void mb_emit(orc_packed* o, ivec* cellFaces, int owner, int nb, node2 a, node2 b, int gid) {
    if (o->nFaces == o->cap) {
        o->cap = o->cap ? 2 * o->cap : 1024;
        size_t c = (size_t)o->cap;
        o->faceOwner = (int32_t*)realloc(o->faceOwner, c * 4);
        o->faceNeighbor = (int32_t*)realloc(o->faceNeighbor, c * 4);
        o->faceGroup = (int32_t*)realloc(o->faceGroup, c * 4);
        o->faceNZ = (double*)realloc(o->faceNZ, c * 8);
        o->faceNR = (double*)realloc(o->faceNR, c * 8);
        o->faceCZ = (double*)realloc(o->faceCZ, c * 8);
        o->faceCR = (double*)realloc(o->faceCR, c * 8);
        o->faceArea = (double*)realloc(o->faceArea, c * 8);
    }
    const int fid = o->nFaces++;
    const double dz = b.z - a.z, dr = b.r - a.r;
    const double L = sqrt(dz * dz + dr * dr);
    const double fz = 0.5 * (a.z + b.z), fr = 0.5 * (a.r + b.r);
    double nz_ = (L > 0.0) ? dr / L : 0.0;
    double nr_ = (L > 0.0) ? -dz / L : 0.0;
    double tz, tr;
    if (nb >= 0) { tz = o->cellCZ[nb] - o->cellCZ[owner]; tr = o->cellCR[nb] - o->cellCR[owner]; }
    else { tz = fz - o->cellCZ[owner]; tr = fr - o->cellCR[owner]; }
    if (nz_ * tz + nr_ * tr < 0.0) { nz_ = -nz_; nr_ = -nr_; }
    o->faceOwner[fid] = owner;
    o->faceNeighbor[fid] = nb;
    o->faceNZ[fid] = nz_;
    o->faceNR[fid] = nr_;
    o->faceCZ[fid] = fz;
    o->faceCR[fid] = fr;
    o->faceArea[fid] = 2.0 * ORC_PI * fabs(fr) * L;
    o->faceGroup[fid] = gid;
    ivec_push(&cellFaces[owner], fid);
    if (nb >= 0) ivec_push(&cellFaces[nb], fid);
}

orc_packed* orc_mb_build(int nBlocks, const orc_block_spec* spec, double tol, int defaultGroup, int* status) {
    *status = 0;
    mb_block* blk = (mb_block*)xcalloc((size_t)nBlocks, sizeof(mb_block));
    int total = 0;
    /* multiblock.h:118-136 makeRectBlock + 210-214 assignGlobalNumbering */
    for (int bi = 0; bi < nBlocks; bi++) {
        const orc_block_spec* s = &spec[bi];
        double* zf = mb_generate_faces(s->axialLength, s->axialCells, s->axialGrading, s->axialCoef, s->z0);
        double* rf = mb_generate_faces(s->radialLength, s->radialCells, s->radialGrading, s->radialCoef, s->r0);
        mb_block* b = &blk[bi];
        b->nz = s->axialCells;
        b->nr = s->radialCells;
        b->nodes = (node2*)xcalloc((size_t)(b->nr + 1) * (b->nz + 1), sizeof(node2));
        for (int I = 0; I <= b->nr; I++)
            for (int J = 0; J <= b->nz; J++) {
                b->nodes[I * (b->nz + 1) + J].z = zf[J];
                b->nodes[I * (b->nz + 1) + J].r = rf[I];
            }
        for (int e = 0; e < 4; e++) b->edgeGroup[e] = s->edgeGroup[e];
        b->globalOffset = total;
        total += b->nr * b->nz;
        free(zf);
        free(rf);
    }
    /* multiblock.h:220-251 autoDetectInterfaces */
    typedef struct { int a, b, ea, eb, rev; } itf_t;
    itf_t* itf = NULL;
    int nItf = 0, capItf = 0;
    const double tol2 = tol * tol;
    for (int a = 0; a < nBlocks; a++)
        for (int b = a + 1; b < nBlocks; b++)
            for (int ea = 0; ea < 4; ea++)
                for (int eb = 0; eb < 4; eb++) {
                    node2 as, ae, bs, be;
                    mb_edge_corners(&blk[a], ea, &as, &ae);
                    mb_edge_corners(&blk[b], eb, &bs, &be);
#define CO(p, q) (((p).z - (q).z) * ((p).z - (q).z) + ((p).r - (q).r) * ((p).r - (q).r) <= tol2)
                    const int aligned = CO(as, bs) && CO(ae, be);
                    const int reversed = CO(as, be) && CO(ae, bs);
#undef CO
                    if (!aligned && !reversed) continue;
                    if (mb_edge_count(&blk[a], ea) != mb_edge_count(&blk[b], eb)) {
                        /* non-conformal seam: the reference clears every interface
                         * (mesh.cpp:2742-2745) */
                        *status = 1;
                        nItf = 0;
                        goto interfaces_done;
                    }
                    if (nItf == capItf) { capItf = capItf ? 2 * capItf : 8; itf = (itf_t*)realloc(itf, (size_t)capItf * sizeof(itf_t)); }
                    itf[nItf].a = a; itf[nItf].b = b; itf[nItf].ea = ea; itf[nItf].eb = eb; itf[nItf].rev = reversed;
                    nItf++;
                }
interfaces_done:;
    orc_packed* o = (orc_packed*)xcalloc(1, sizeof(orc_packed));
    o->nCells = total;
    o->cellCZ = (double*)xcalloc((size_t)total, 8);
    o->cellCR = (double*)xcalloc((size_t)total, 8);
    o->cellA2D = (double*)xcalloc((size_t)total, 8);
    o->cellVol = (double*)xcalloc((size_t)total, 8);
    /* multiblock.h:320-338 cells */
    for (int bi = 0; bi < nBlocks; bi++) {
        const mb_block* b = &blk[bi];
        for (int i = 0; i < b->nr; i++)
            for (int j = 0; j < b->nz; j++) {
                const int g = mb_cell(b, i, j);
                double cz, cr, area;
                mb_quad(mb_node(b, i, j), mb_node(b, i, j + 1), mb_node(b, i + 1, j + 1), mb_node(b, i + 1, j), &cz, &cr, &area);
                o->cellCZ[g] = cz;
                o->cellCR[g] = cr;
                o->cellA2D[g] = area;
                o->cellVol[g] = 2.0 * ORC_PI * fabs(cr) * area;
            }
    }
    ivec* cellFaces = (ivec*)xcalloc((size_t)total, sizeof(ivec));
    /* 2a intra-block faces, multiblock.h:382-394 */
    for (int bi = 0; bi < nBlocks; bi++) {
        const mb_block* b = &blk[bi];
        for (int i = 0; i < b->nr; i++)
            for (int j = 0; j < b->nz; j++) {
                const int owner = mb_cell(b, i, j);
                if (j + 1 < b->nz) mb_emit(o, cellFaces, owner, mb_cell(b, i, j + 1), mb_node(b, i, j + 1), mb_node(b, i + 1, j + 1), -1);
                if (i + 1 < b->nr) mb_emit(o, cellFaces, owner, mb_cell(b, i + 1, j), mb_node(b, i + 1, j), mb_node(b, i + 1, j + 1), -1);
            }
    }
    /* 2b interface faces, multiblock.h:397-414 */
    char* claimed = (char*)xcalloc((size_t)nBlocks * 4, 1);
    for (int t = 0; t < nItf; t++) {
        claimed[itf[t].a * 4 + itf[t].ea] = 1;
        claimed[itf[t].b * 4 + itf[t].eb] = 1;
        const mb_block* A = &blk[itf[t].a];
        const mb_block* B = &blk[itf[t].b];
        const int count = mb_edge_count(A, itf[t].ea);
        for (int k = 0; k < count; k++) {
            int localA; node2 n0, n1;
            mb_edge_face(A, itf[t].ea, k, &localA, &n0, &n1);
            const int kb = itf[t].rev ? (count - 1 - k) : k;
            mb_emit(o, cellFaces, A->globalOffset + localA, B->globalOffset + mb_edge_cell(B, itf[t].eb, kb), n0, n1, -1);
        }
    }
    /* 2c external faces, multiblock.h:417-432 */
    for (int bi = 0; bi < nBlocks; bi++) {
        const mb_block* b = &blk[bi];
        for (int e = 0; e < 4; e++) {
            if (claimed[bi * 4 + e]) continue;
            const int gid = (b->edgeGroup[e] >= 0) ? b->edgeGroup[e] : defaultGroup;
            const int count = mb_edge_count(b, e);
            for (int k = 0; k < count; k++) {
                int local; node2 n0, n1;
                mb_edge_face(b, e, k, &local, &n0, &n1);
                mb_emit(o, cellFaces, b->globalOffset + local, -1, n0, n1, gid);
            }
        }
    }
    /* 3 CSR, multiblock.h:435-441 */
    o->cellFaceStart = (int32_t*)xcalloc((size_t)total + 1, 4);
    for (int c = 0; c < total; c++) o->cellFaceStart[c + 1] = o->cellFaceStart[c] + cellFaces[c].n;
    o->nRefs = o->cellFaceStart[total];
    o->cellFaceIDs = (int32_t*)xcalloc((size_t)o->nRefs, 4);
    for (int c = 0; c < total; c++) {
        memcpy(o->cellFaceIDs + o->cellFaceStart[c], cellFaces[c].data, (size_t)cellFaces[c].n * 4);
        free(cellFaces[c].data);
    }
    free(cellFaces);
    free(claimed);
    free(itf);
    for (int bi = 0; bi < nBlocks; bi++) free(blk[bi].nodes);
    free(blk);
    return o;
}

void orc_mb_sizes(const orc_packed* p, int32_t* nCells, int32_t* nFaces, int32_t* nRefs) {
    *nCells = p->nCells; *nFaces = p->nFaces; *nRefs = p->nRefs;
}

void orc_mb_copy(const orc_packed* p, int32_t* faceOwner, int32_t* faceNeighbor, double* faceNormalZ,
                 double* faceNormalR, double* faceCenterZ, double* faceCenterR, double* faceArea,
                 int32_t* faceBoundaryGroupID, double* cellCenterZ, double* cellCenterR, double* cellArea2D,
                 double* cellVolume, int32_t* cellFaceStart, int32_t* cellFaceIDs) {
    const size_t F = (size_t)p->nFaces, N = (size_t)p->nCells;
    memcpy(faceOwner, p->faceOwner, F * 4);
    memcpy(faceNeighbor, p->faceNeighbor, F * 4);
    memcpy(faceNormalZ, p->faceNZ, F * 8);
    memcpy(faceNormalR, p->faceNR, F * 8);
    memcpy(faceCenterZ, p->faceCZ, F * 8);
    memcpy(faceCenterR, p->faceCR, F * 8);
    memcpy(faceArea, p->faceArea, F * 8);
    memcpy(faceBoundaryGroupID, p->faceGroup, F * 4);
    memcpy(cellCenterZ, p->cellCZ, N * 8);
    memcpy(cellCenterR, p->cellCR, N * 8);
    memcpy(cellArea2D, p->cellA2D, N * 8);
    memcpy(cellVolume, p->cellVol, N * 8);
    memcpy(cellFaceStart, p->cellFaceStart, (N + 1) * 4);
    memcpy(cellFaceIDs, p->cellFaceIDs, (size_t)p->nRefs * 4);
}

void orc_mb_free(orc_packed* p) {
    if (!p) return;
    free(p->faceOwner); free(p->faceNeighbor); free(p->faceGroup);
    free(p->faceNZ); free(p->faceNR); free(p->faceCZ); free(p->faceCR); free(p->faceArea);
    free(p->cellCZ); free(p->cellCR); free(p->cellA2D); free(p->cellVol);
    free(p->cellFaceStart); free(p->cellFaceIDs);
    free(p);
}

/* ======================================================================
 * Solver state
 * ====================================================================== */
typedef struct {
    int nGroups;
    uint8_t* type;
    uint8_t* btype;
    double* value;   /* current value (pulsatile groups updated per step) */
    double* mean;    /* value at t = 0 */
    double* length;
    uint8_t* puls;
    double* amp;
    double* freq;
    /* wall kinetics (BoundaryFieldDevice, solver_struct.h:436-451) with the
     * host-precomputed Km^n and K2^m (memory_manger.cpp:122-136) */
    double *vmax, *km, *nexp, *mexp, *k2, *v2, *Rtot, *kmN, *k2M;
} bcf;

typedef struct {
    int N, S;
    double *AC, *b, *invAC, *AF;
    const int32_t* faceStart;     /* shared with the mesh CSR */
    const int32_t* faceNeighbor;
} coeffs;

typedef struct {
    int N, S;
    int32_t *faceStart, *faceNeighbor;
    int32_t *cellToCoarse, *fineSlotToCoarseSlot; /* NULL on the coarsest level */
    double *AC, *AF, *b, *x, *xNew, *res;
} mglevel;

struct orc_solver {
    orc_config cfg;
    int N, F, S;
    /* mesh (owned copies) */
    int32_t *owner, *neighbor, *group, *cfs, *cfi;
    double *nZ, *nR, *fcZ, *fcR, *area, *ccZ, *ccR, *vol;
    /* precompute, memory_manger.cpp:512-617 */
    double *invDPN, *wP, *dPB, *invA2D, *length2D, *lsqWZ, *lsqWR, *lsqIZZ, *lsqIZR, *lsqIRR;
    /* level-0 CSR neighbour, memory_manger.cpp:287-323 */
    int32_t* slotNb;
    bcf bcU, bcV, bcP, bcPP, bcT, bcC;
    coeffs cu, cv, cpp, ct, cc;
    double *u, *v, *p, *pp, *uTemp, *vTemp, *ppTemp, *DU, *DV;
    double *gradPZ, *gradPR, *gradUZ, *gradUR, *gradVZ, *gradVR;
    double *uOld, *vOld, *uOld2, *vOld2, *mDot;
    double *resU, *resV, *resC, *scaleU, *scaleV;
    double resVal[3], scaleVal[3];
    /* scalar transport: temperature, concentration, their work and old levels,
     * gradients, residuals; wall concentration and consumption per face */
    double *T, *C, *TTemp, *CTemp, *TOld, *COld, *TOld2, *COld2, *gradTZ, *gradTR, *gradCZ, *gradCR;
    double *resT, *resCc, *scaleT, *scaleCc, *cw, *ocrWall;
    double resValS[2], scaleValS[2];
    int currentIteration;
    double simTime;
    /* multigrid */
    int nLevels;
    mglevel* lv;
    /* colouring */
    int nColors;
    int32_t *color, *colorStart, *cellOrder;
};

/* ---------------- face helpers, solver_util.cuh:56-238 ---------------- */
static inline double face_weight(const orc_solver* s, int c, int f) {
    const double w = s->wP[f];
    return (s->owner[f] == c) ? w : 1.0 - w;
}

static inline double normal_corr(const orc_solver* s, int c, int f) {
    const double nz = s->nZ[f], nr = s->nR[f];
    return s->DU[c] * nz * nz + s->DV[c] * nr * nr;
}

/* solver_util.cuh:126-161 */
static inline double interp_corr(const orc_solver* s, int c, int f) {
    const int own = s->owner[f], nb = s->neighbor[f];
    const double DP = normal_corr(s, c, f);
    if (nb < 0) return DP;
    const int o = (own == c) ? nb : own;
    const double DN = normal_corr(s, o, f);
    const double w = face_weight(s, c, f);
    return w * DP + (1.0 - w) * DN;
}

/* solver_util.cuh:223-238 */
static inline double prescribed(const orc_solver* s, int f, int type, double value, double len) {
    if (type != BC_FULLY_DEVELOPED) return value;
    const double nz = s->nZ[f], nr = s->nR[f];
    const double along = s->fcR[f] * nz * nz + s->fcZ[f] * nr * nr;
    const double x = along / len;
    return value * (1.0 - x * x);
}

/* solver_util.cuh:240-297 */
static inline double interp_face(const orc_solver* s, int c, int f, const bcf* bc, const double* phi) {
    const int own = s->owner[f], nb = s->neighbor[f];
    const double phiP = phi[c];
    if (nb >= 0) {
        const int o = (own == c) ? nb : own;
        const double w = face_weight(s, c, f);
        return w * phiP + (1.0 - w) * phi[o];
    }
    const int g = s->group[f];
    if (g < 0 || g >= bc->nGroups) return phiP;
    const int t = bc->type[g];
    const double val = bc->value[g];
    if (t == BC_DIRICHLET || t == BC_FULLY_DEVELOPED) return prescribed(s, f, t, val, bc->length[g]);
    if (t == BC_NEUMANN) return phiP + val * s->dPB[f];
    return phiP;
}

/* solver_util.cuh:383-430 */
static inline double nonortho_flux(const orc_solver* s, int c, int f, const double* gZ, const double* gR, double gamma) {
    const int own = s->owner[f], nb = s->neighbor[f];
    if (nb < 0) return 0.0;
    const int o = (own == c) ? nb : own;
    double nz = s->nZ[f], nr = s->nR[f];
    if (nb == c) { nz = -nz; nr = -nr; }
    const double a = s->area[f];
    const double dz = s->ccZ[o] - s->ccZ[c];
    const double dr = s->ccR[o] - s->ccR[c];
    const double invD = s->invDPN[f];
    const double aOverNd = a * invD;
    const double Tz = a * nz - aOverNd * dz;
    const double Tr = a * nr - aOverNd * dr;
    const double w = face_weight(s, c, f);
    const double gfz = w * gZ[c] + (1.0 - w) * gZ[o];
    const double gfr = w * gR[c] + (1.0 - w) * gR[o];
    return gamma * (Tz * gfz + Tr * gfr);
}

/* ---------------- gradients, solver_util.cu:146-169, cuh:458-588 ---------------- */
static void compute_gradient(const orc_solver* s, const bcf* bc, const double* phi, double* gZ, double* gR) {
    const int scheme = s->cfg.gradientScheme;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        if (scheme == GRAD_GG) {
            double gz = 0.0, gr = 0.0, clZ = 0.0, clR = 0.0, axisPhi = 0.0;
            int hasAxis = 0;
            for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
                const int f = s->cfi[k];
                double nz = s->nZ[f], nr = s->nR[f];
                if (s->neighbor[f] == n) { nz = -nz; nr = -nr; }
                const double phiF = interp_face(s, n, f, bc, phi);
                const double rf = s->fcR[f];
                if (rf > 1.0e-30) {
                    const double L = s->length2D[f];
                    gz += phiF * nz * L;
                    gr += phiF * nr * L;
                    clZ += nz * L;
                    clR += nr * L;
                } else {
                    hasAxis = 1;
                    axisPhi = phiF;
                }
            }
            if (hasAxis) {
                gz += axisPhi * (-clZ);
                gr += axisPhi * (-clR);
            }
            const double inv = s->invA2D[n];
            gZ[n] = gz * inv;
            gR[n] = gr * inv;
        } else if (scheme == GRAD_LSQ) {
            const double phiP = phi[n];
            double bz = 0.0, br = 0.0;
            for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
                const int f = s->cfi[k];
                const int own = s->owner[f], nb = s->neighbor[f];
                double dphi;
                if (nb >= 0) {
                    const int isOwner = (own == n);
                    const double phiNb = phi[isOwner ? nb : own];
                    dphi = isOwner ? (phiNb - phiP) : (phiP - phiNb);
                } else {
                    dphi = interp_face(s, n, f, bc, phi) - phiP;
                }
                bz += s->lsqWZ[f] * dphi;
                br += s->lsqWR[f] * dphi;
            }
            const double izr = s->lsqIZR[n];
            gZ[n] = s->lsqIZZ[n] * bz + izr * br;
            gR[n] = izr * bz + s->lsqIRR[n] * br;
        } else {
            gZ[n] = 0.0;
            gR[n] = 0.0;
        }
    }
}

/* ---------------- wall kinetics, concentration_equation.cu:6-160 ---------------- */
static inline double kin_mm(const bcf* bc, int g, double c) { return (bc->vmax[g] * c) / (bc->km[g] + c); }
static inline double kin_dmm(const bcf* bc, int g, double c) {
    const double inv = 1.0 / (bc->km[g] + c);
    return bc->vmax[g] * bc->km[g] * inv * inv;
}
static inline double kin_inhib(const bcf* bc, int g, double c) {
    const double V2 = bc->v2[g];
    if (V2 == 0.0) return 1.0;
    const double cm = pow(c, bc->mexp[g]);
    return (1.0 - (V2 * cm / (bc->k2M[g] + cm)));
}
static inline double kin_dinhib(const bcf* bc, int g, double c) {
    const double V2 = bc->v2[g];
    if (V2 == 0.0) return 0.0;
    const double m = bc->mexp[g], K2m = bc->k2M[g];
    const double cm = pow(c, m);
    const double cm1 = pow(c, m - 1.0);
    return (-(m * V2 * K2m) * (cm1) / ((K2m + cm) * (K2m + cm)));
}
static inline double kin_hill(const bcf* bc, int g, double c) {
    const double cn = pow(c, bc->nexp[g]);
    return (bc->vmax[g] * cn) / (bc->kmN[g] + cn);
}
static inline double kin_dhill(const bcf* bc, int g, double c) {
    const double n = bc->nexp[g], Kmn = bc->kmN[g];
    const double cn = pow(c, n);
    const double cn1 = pow(c, n - 1.0);
    return ((n * bc->vmax[g] * Kmn) * (cn1) / ((Kmn + cn) * (Kmn + cn)));
}
/* wallConcentrationMichaelisMenten / wallConcentrationHill: Newton on
 * h (c_P - c_w) = J(c_w), from c_w = c_P, clipped at 0, at most 100 steps. */
static double wall_concentration(const bcf* bc, int g, int hill, double cp, double h) {
    double cw = cp;
    const double relTol = 1e-10, absTol = 1e-14;
    for (int i = 0; i < 100; i++) {
        const double rate = hill ? kin_hill(bc, g, cw) : kin_mm(bc, g, cw);
        const double inhib = kin_inhib(bc, g, cw);
        const double J = rate * inhib;
        const double drate = hill ? kin_dhill(bc, g, cw) : kin_dmm(bc, g, cw);
        const double dJ = rate * kin_dinhib(bc, g, cw) + drate * inhib;
        const double F = h * (cp - cw) - J;
        const double dF = -h - dJ;
        const double step = F / dF;
        cw -= step;
        cw = fmax(0.0, cw);
        if (fabs(step) < absTol + relTol * fabs(cw)) break;
    }
    return cw;
}

/* ---------------- momentum assembly, solver_util.cu:218-448, cuh:715-865 ---------------- */
static void add_transport(orc_solver* s, coeffs* c, const bcf* bc, const double* phi,
                          const double* gZ, const double* gR, int nonOrtho, double gamma, int conv,
                          int scheme, double fluxScale) {
    double *AC = c->AC, *b = c->b, *AF = c->AF;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        double netF = 0.0;
        for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
            const int f = s->cfi[k];
            const int own = s->owner[f], nb = s->neighbor[f];
            const double a = s->area[f];
            double F = 0.0;
            if (conv) {
                const double Fo = s->mDot[f] * fluxScale;
                if (own == n) F = Fo;
                else if (nb == n) F = -Fo;
                if (fabs(F) <= 1.0e-30) F = 0.0;
                netF += F;
            }
            if (nb >= 0) {
                const double K = gamma * a * s->invDPN[f];
                AC[n] += K;
                AF[k] -= K;
                if (nonOrtho) b[n] += nonortho_flux(s, n, f, gZ, gR, gamma);
                if (F != 0.0) {
                    const int o = (own == n) ? nb : own;
                    AC[n] += fmax(F, 0.0);
                    AF[k] += fmin(F, 0.0);
                    if (scheme != CONV_UPWIND && phi) {
                        const double phiUD = (F > 0.0) ? phi[n] : phi[o];
                        double phiHO = phiUD;
                        if (scheme == CONV_CENTRAL) {
                            phiHO = interp_face(s, n, f, bc, phi);
                        } else if (scheme == CONV_SOU) {
                            const int up = (F > 0.0) ? n : o;
                            const double dz = s->fcZ[f] - s->ccZ[up];
                            const double dr = s->fcR[f] - s->ccR[up];
                            const double ho = phi[up] + gZ[up] * dz + gR[up] * dr;
                            const double lo = fmin(phi[n], phi[o]);
                            const double hi = fmax(phi[n], phi[o]);
                            phiHO = fmin(fmax(ho, lo), hi);
                        }
                        b[n] -= F * (phiHO - phiUD);
                    }
                }
            } else {
                const int g = s->group[f];
                const double nz = s->nZ[f], nr = s->nR[f];
                if (g >= 0 && g < bc->nGroups) {
                    const int t = bc->type[g];
                    const double val = bc->value[g];
                    const double len = bc->length[g];
                    const double dPF = fabs((s->fcZ[f] - s->ccZ[n]) * nz + (s->fcR[f] - s->ccR[n]) * nr);
                    const double K = gamma * a / dPF;
                    if (t == BC_DIRICHLET) {
                        AC[n] += K;
                        b[n] += K * val;
                    } else if (t == BC_NEUMANN) {
                        b[n] += gamma * a * val;
                    } else if (t == BC_FULLY_DEVELOPED) {
                        AC[n] += K;
                        b[n] += K * prescribed(s, f, t, val, len);
                    } else if (t == BC_MICHAELIS_MENTEN || t == BC_HILL) {
                        /* solver_util.cu:388-411 reactive wall */
                        const int hill = t == BC_HILL;
                        const double Rtot = (dPF / gamma) + bc->Rtot[g];
                        const double h = 1 / Rtot;
                        const double cw = wall_concentration(bc, g, hill, phi[n], h);
                        s->cw[f] = cw;
                        s->ocrWall[f] = a * (hill ? kin_hill(bc, g, cw) : kin_mm(bc, g, cw)) * kin_inhib(bc, g, cw);
                        AC[n] += a * h;
                        b[n] += a * h * cw;
                    }
                }
                if (F != 0.0) {
                    /* addConvectionContribution, boundary branch (solver_util.cuh:817-864) */
                    if (g < 0 || g >= bc->nGroups) {
                        AC[n] += F;
                    } else {
                        const int t = bc->type[g];
                        const double val = bc->value[g];
                        if (t == BC_DIRICHLET) {
                            if (F < 0.0) b[n] += -F * val;
                            else AC[n] += F;
                        } else if (t == BC_NEUMANN) {
                            AC[n] += F;
                        } else if (t == BC_FULLY_DEVELOPED) {
                            if (F < 0.0) b[n] += -F * prescribed(s, f, t, val, bc->length[g]);
                            else AC[n] += F;
                        }
                    }
                }
            }
        }
        if (conv) AC[n] -= netF;
    }
}

/* ---------------- SIMPLE kernels, simple.cu ---------------- */
static void create_pp_coeff(orc_solver* s) {
    double *AC = s->cpp.AC, *AF = s->cpp.AF;
    const double rho = s->cfg.rho;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
            const int f = s->cfi[k];
            const int nb = s->neighbor[f];
            const double a = s->area[f];
            const double Df = interp_corr(s, n, f);
            if (nb >= 0) {
                const double K = rho * a * Df * s->invDPN[f];
                AC[n] += K;
                AF[k] -= K;
            } else {
                const int g = s->group[f];
                if (g < 0 || g >= s->bcP.nGroups) continue;
                if (s->bcP.type[g] == BC_DIRICHLET) {
                    const double K = rho * a * Df / s->dPB[f];
                    AC[n] += K;
                }
            }
        }
    }
}

static void create_pp_rhs(orc_solver* s, int applyNonOrtho) {
    const double rho = s->cfg.rho;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        double imb = 0.0, cross = 0.0;
        for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
            const int f = s->cfi[k];
            const double m = s->mDot[f];
            if (s->owner[f] == n) imb += m;
            else if (s->neighbor[f] == n) imb -= m;
            if (applyNonOrtho) {
                const double Df = interp_corr(s, n, f);
                cross += nonortho_flux(s, n, f, s->gradPZ, s->gradPR, rho * Df);
            }
        }
        s->cpp.b[n] = -imb + cross;
    }
}

/* solver_util.cu:171-203, cuh:590-713 */
static void rhie_chow(orc_solver* s) {
    const double rho = s->cfg.rho;
#pragma omp parallel for schedule(static)
    for (int f = 0; f < s->F; f++) {
        const int P = s->owner[f], nb = s->neighbor[f];
        const double a = s->area[f];
        if (a <= 1.0e-30) { s->mDot[f] = 0.0; continue; }
        const double nz = s->nZ[f], nr = s->nR[f];
        const double uF = interp_face(s, P, f, &s->bcU, s->u);
        const double vF = interp_face(s, P, f, &s->bcV, s->v);
        const double unLin = uF * nz + vF * nr;
        double un;
        if (nb < 0) {
            const int g = s->group[f];
            if (g < 0 || g >= s->bcP.nGroups || s->bcP.type[g] != BC_DIRICHLET) {
                un = unLin;
            } else {
                const double dPB = s->dPB[f];
                const double DfB = interp_corr(s, P, f);
                const double gc = (s->bcP.value[g] - s->p[P]) / dPB;
                const double gn = s->gradPZ[P] * nz + s->gradPR[P] * nr;
                un = unLin - DfB * (gc - gn);
            }
        } else {
            const double gpn = (s->p[nb] - s->p[P]) * s->invDPN[f];
            const double w = face_weight(s, P, f);
            const double gzf = w * s->gradPZ[P] + (1.0 - w) * s->gradPZ[nb];
            const double grf = w * s->gradPR[P] + (1.0 - w) * s->gradPR[nb];
            const double gfn = gzf * nz + grf * nr;
            const double Df = interp_corr(s, P, f);
            un = unLin - Df * (gpn - gfn);
        }
        s->mDot[f] = rho * un * a;
    }
}

/* simple.cu:181-258 */
static void update_mass_flux(orc_solver* s, int applyNonOrtho) {
    const double rho = s->cfg.rho;
#pragma omp parallel for schedule(static)
    for (int f = 0; f < s->F; f++) {
        const int P = s->owner[f], nb = s->neighbor[f];
        const double a = s->area[f];
        if (a <= 1.0e-30) { s->mDot[f] = 0.0; continue; }
        const double nz = s->nZ[f], nr = s->nR[f];
        const double Df = interp_corr(s, P, f);
        if (nb >= 0) {
            s->mDot[f] -= rho * a * Df * (s->pp[nb] - s->pp[P]) * s->invDPN[f];
            if (applyNonOrtho) s->mDot[f] -= nonortho_flux(s, P, f, s->gradPZ, s->gradPR, rho * Df);
            continue;
        }
        const int g = s->group[f];
        if (g < 0 || g >= s->bcP.nGroups) continue;
        if (s->bcP.type[g] == BC_DIRICHLET) {
            const double dPB = fabs((s->fcZ[f] - s->ccZ[P]) * nz + (s->fcR[f] - s->ccR[P]) * nr);
            const double ppB = 0.0;
            s->mDot[f] -= rho * a * Df * (ppB - s->pp[P]) / dPB;
        }
    }
}

/* ---------------- linear solvers, linear_solver.cu:9-146 ---------------- */
static void jacobi_sweeps(const orc_solver* s, const coeffs* c, double* x, double* xTmp, int iters) {
    double* live = x;
    double* spare = xTmp;
    for (int it = 0; it < iters; it++) {
#pragma omp parallel for schedule(static)
        for (int n = 0; n < c->N; n++) {
            const double inv = c->invAC[n];
            double val = c->b[n];
            for (int k = c->faceStart[n]; k < c->faceStart[n + 1]; k++) {
                const int nb = c->faceNeighbor[k];
                if (nb >= 0) val -= c->AF[k] * live[nb];
            }
            spare[n] = (inv != 0.0) ? val * inv : live[n];
        }
        double* t = live; live = spare; spare = t;
    }
    if (live != x) memcpy(x, live, (size_t)c->N * sizeof(double));
    (void)s;
}

static void gs_sweeps(const orc_solver* s, const coeffs* c, double* x, int iters) {
    for (int it = 0; it < iters; it++) {
        for (int col = 0; col < s->nColors; col++) {
            const int b0 = s->colorStart[col], b1 = s->colorStart[col + 1];
#pragma omp parallel for schedule(static)
            for (int t = b0; t < b1; t++) {
                const int n = s->cellOrder[t];
                const double inv = c->invAC[n];
                double val = c->b[n];
                for (int k = c->faceStart[n]; k < c->faceStart[n + 1]; k++) {
                    const int nb = c->faceNeighbor[k];
                    if (nb >= 0) val -= c->AF[k] * x[nb];
                }
                x[n] = (inv != 0.0) ? val * inv : x[n];
            }
        }
    }
}

static void linear_solve(const orc_solver* s, const coeffs* c, double* x, double* xTmp) {
    const int useGS = (s->cfg.linearType == 1) && s->nColors > 0;
    if (useGS) gs_sweeps(s, c, x, s->cfg.linearMaxIter);
    else jacobi_sweeps(s, c, x, xTmp, s->cfg.linearMaxIter);
}

/* ---------------- multigrid, multigrid.cu ---------------- */
static int cmp_ref(const void* a, const void* b) {
    const int* x = (const int*)a;
    const int* y = (const int*)b;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
    return 0;
}

/* multigrid.cu:79-194 buildAgglomerationMap */
static int agglomerate(const mglevel* fine, int32_t* c2c) {
    const int target = 4;
    const int N = fine->N;
    for (int n = 0; n < N; n++) c2c[n] = -1;
    int nCoarse = 0;
    int members[4];
    for (int n = 0; n < N; n++) {
        if (c2c[n] >= 0) continue;
        const int c = nCoarse++;
        c2c[n] = c;
        int nm = 0;
        members[nm++] = n;
        for (int m = 0; m < nm && nm < target; m++) {
            const int cell = members[m];
            for (int k = fine->faceStart[cell]; k < fine->faceStart[cell + 1] && nm < target; k++) {
                const int nb = fine->faceNeighbor[k];
                if (nb < 0) continue;
                if (c2c[nb] >= 0) continue;
                c2c[nb] = c;
                members[nm++] = nb;
            }
        }
    }
    int* size = (int*)xcalloc((size_t)nCoarse, sizeof(int));
    for (int n = 0; n < N; n++) size[c2c[n]]++;
    for (int n = 0; n < N; n++) {
        const int c = c2c[n];
        if (size[c] != 1) continue;
        int best = -1, bestSize = 0;
        for (int k = fine->faceStart[n]; k < fine->faceStart[n + 1]; k++) {
            const int nb = fine->faceNeighbor[k];
            if (nb < 0) continue;
            const int cnb = c2c[nb];
            if (cnb == c) continue;
            if (best < 0 || size[cnb] < bestSize) { best = cnb; bestSize = size[cnb]; }
        }
        if (best < 0) continue;
        c2c[n] = best;
        size[best]++;
        size[c] = 0;
    }
    int* remap = (int*)xcalloc((size_t)nCoarse, sizeof(int));
    for (int c = 0; c < nCoarse; c++) remap[c] = -1;
    int nCompact = 0;
    for (int n = 0; n < N; n++) {
        const int c = c2c[n];
        if (remap[c] < 0) remap[c] = nCompact++;
        c2c[n] = remap[c];
    }
    free(size);
    free(remap);
    return nCompact;
}

/* multigrid.cu:196-287 coarsenGrid; returns the coarse level (topology only) */
static mglevel coarsen(mglevel* fine) {
    mglevel coarse;
    memset(&coarse, 0, sizeof(coarse));
    fine->cellToCoarse = (int32_t*)xcalloc((size_t)fine->N, 4);
    const int nC = agglomerate(fine, fine->cellToCoarse);
    coarse.N = nC;
    int* refs = (int*)xcalloc((size_t)fine->S * 3, sizeof(int));
    int nr = 0;
    for (int n = 0; n < fine->N; n++) {
        const int cn = fine->cellToCoarse[n];
        for (int k = fine->faceStart[n]; k < fine->faceStart[n + 1]; k++) {
            const int nb = fine->faceNeighbor[k];
            if (nb < 0) continue;
            const int cnb = fine->cellToCoarse[nb];
            if (cnb != cn) { refs[3 * nr] = cn; refs[3 * nr + 1] = cnb; refs[3 * nr + 2] = k; nr++; }
        }
    }
    qsort(refs, (size_t)nr, 3 * sizeof(int), cmp_ref);
    fine->fineSlotToCoarseSlot = (int32_t*)xcalloc((size_t)fine->S, 4);
    for (int k = 0; k < fine->S; k++) fine->fineSlotToCoarseSlot[k] = -1;
    coarse.faceStart = (int32_t*)xcalloc((size_t)nC + 1, 4);
    coarse.faceNeighbor = (int32_t*)xcalloc((size_t)(nr ? nr : 1), 4);
    int S = 0;
    for (int i = 0; i < nr; i++) {
        const int newEntry = (i == 0) || refs[3 * i] != refs[3 * (i - 1)] || refs[3 * i + 1] != refs[3 * (i - 1) + 1];
        if (newEntry) {
            coarse.faceNeighbor[S++] = refs[3 * i + 1];
            coarse.faceStart[refs[3 * i] + 1]++;
        }
        fine->fineSlotToCoarseSlot[refs[3 * i + 2]] = S - 1;
    }
    for (int c = 0; c < nC; c++) coarse.faceStart[c + 1] += coarse.faceStart[c];
    coarse.S = S;
    free(refs);
    return coarse;
}

static void alloc_level_data(mglevel* l) {
    l->AC = (double*)xcalloc((size_t)l->N, 8);
    l->AF = (double*)xcalloc((size_t)(l->S ? l->S : 1), 8);
    l->b = (double*)xcalloc((size_t)l->N, 8);
    l->x = (double*)xcalloc((size_t)l->N, 8);
    l->xNew = (double*)xcalloc((size_t)l->N, 8);
    l->res = (double*)xcalloc((size_t)l->N, 8);
}

/* multigrid.cu:298-325 buildLevels */
static void build_levels(orc_solver* s) {
    const int minCoarseCells = 64;
    const double maxShrink = 0.8;
    int cap = 8;
    s->lv = (mglevel*)xcalloc((size_t)cap, sizeof(mglevel));
    s->nLevels = 0;
    mglevel fine;
    memset(&fine, 0, sizeof(fine));
    fine.N = s->N;
    fine.S = s->S;
    fine.faceStart = (int32_t*)xcalloc((size_t)s->N + 1, 4);
    memcpy(fine.faceStart, s->cfs, ((size_t)s->N + 1) * 4);
    fine.faceNeighbor = (int32_t*)xcalloc((size_t)(s->S ? s->S : 1), 4);
    memcpy(fine.faceNeighbor, s->slotNb, (size_t)s->S * 4);
    for (;;) {
        if (fine.N <= minCoarseCells) break;
        mglevel coarse = coarsen(&fine);
        if (coarse.N >= (int)(fine.N * maxShrink)) {
            free(fine.cellToCoarse); fine.cellToCoarse = NULL;
            free(fine.fineSlotToCoarseSlot); fine.fineSlotToCoarseSlot = NULL;
            free(coarse.faceStart); free(coarse.faceNeighbor);
            break;
        }
        if (s->nLevels == cap) { cap *= 2; s->lv = (mglevel*)realloc(s->lv, (size_t)cap * sizeof(mglevel)); }
        alloc_level_data(&fine);
        s->lv[s->nLevels++] = fine;
        fine = coarse;
    }
    if (s->nLevels == cap) { cap *= 2; s->lv = (mglevel*)realloc(s->lv, (size_t)cap * sizeof(mglevel)); }
    alloc_level_data(&fine);
    s->lv[s->nLevels++] = fine;
}

/* multigrid.cu:447-493 jacobiRow / jacobiFused; 501-541 single block (same math) */
static void mg_smooth(mglevel* l, int iters, double w) {
    if (l->N <= 0 || iters <= 0) return;
    for (int it = 0; it < iters; it++) {
        const double* xo = l->x;
        double* xn = l->xNew;
#pragma omp parallel for schedule(static) if (l->N > 4096)
        for (int n = 0; n < l->N; n++) {
            const double AC = l->AC[n];
            if (fabs(AC) < 1.0e-30) { xn[n] = xo[n]; continue; }
            double Ax = AC * xo[n];
            for (int k = l->faceStart[n]; k < l->faceStart[n + 1]; k++) {
                const int nb = l->faceNeighbor[k];
                if (nb != -1) Ax += l->AF[k] * xo[nb];
            }
            xn[n] = xo[n] + w * (l->b[n] - Ax) / AC;
        }
        double* t = l->x; l->x = l->xNew; l->xNew = t;
    }
}

/* residuals.cuh:17-48 with sign = true */
static void mg_residual(mglevel* l) {
#pragma omp parallel for schedule(static) if (l->N > 4096)
    for (int n = 0; n < l->N; n++) {
        double Ax = l->AC[n] * l->x[n];
        for (int k = l->faceStart[n]; k < l->faceStart[n + 1]; k++) {
            const int nb = l->faceNeighbor[k];
            if (nb >= 0) Ax += l->AF[k] * l->x[nb];
        }
        l->res[n] = l->b[n] - Ax;
    }
}

/* multigrid.cu:607-662 vCycle */
static void vcycle(orc_solver* s, int l) {
    if (l < 0 || l >= s->nLevels) return;
    mglevel* L = &s->lv[l];
    const double w = s->cfg.mgWeight;
    if (L->cellToCoarse == NULL) {
        mg_smooth(L, s->cfg.mgLinearSweep, w);
        return;
    }
    mg_smooth(L, s->cfg.mgPreSweep, w);
    mg_residual(L);
    mglevel* C = &s->lv[l + 1];
    memset(C->b, 0, (size_t)C->N * 8);
    for (int n = 0; n < L->N; n++) C->b[L->cellToCoarse[n]] += L->res[n];
    memset(C->x, 0, (size_t)C->N * 8);
    vcycle(s, l + 1);
    for (int n = 0; n < L->N; n++) L->x[n] += C->x[L->cellToCoarse[n]];
    mg_smooth(L, s->cfg.mgPostSweep, w);
}

/* multigrid.cu:766-811 enqueueRun (copy-in, Galerkin per level, cycles, copy-out) */
static void mg_run(orc_solver* s) {
    mglevel* L0 = &s->lv[0];
    memcpy(L0->x, s->pp, (size_t)s->N * 8);
    memcpy(L0->AC, s->cpp.AC, (size_t)s->N * 8);
    memcpy(L0->b, s->cpp.b, (size_t)s->N * 8);
    memcpy(L0->AF, s->cpp.AF, (size_t)s->S * 8);
    /* multigrid.cu:350-389 Galerkin, ascending fine-cell order */
    for (int l = 1; l < s->nLevels; l++) {
        mglevel* f = &s->lv[l - 1];
        mglevel* c = &s->lv[l];
        memset(c->AC, 0, (size_t)c->N * 8);
        memset(c->AF, 0, (size_t)(c->S ? c->S : 1) * 8);
        for (int n = 0; n < f->N; n++) {
            double diag = f->AC[n];
            for (int k = f->faceStart[n]; k < f->faceStart[n + 1]; k++) {
                const int nb = f->faceNeighbor[k];
                if (nb < 0) continue;
                const int slot = f->fineSlotToCoarseSlot[k];
                if (slot >= 0) c->AF[slot] += f->AF[k];
                else diag += f->AF[k];
            }
            c->AC[f->cellToCoarse[n]] += diag;
        }
    }
    const int nCycles = s->cfg.mgMaxIter > 1 ? s->cfg.mgMaxIter : 1;
    for (int cyc = 0; cyc < nCycles; cyc++) vcycle(s, 0);
    memcpy(s->pp, L0->x, (size_t)s->N * 8);
}

/* ---------------- residuals, residuals.cu / residuals.cuh ---------------- */
static void residual_raw(const orc_solver* s, const coeffs* c, const double* x, double* res, double* scale, int diag) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < c->N; n++) {
        double Ax = c->AC[n] * x[n];
        if (diag) scale[n] = Ax;
        for (int k = c->faceStart[n]; k < c->faceStart[n + 1]; k++) {
            const int nb = c->faceNeighbor[k];
            if (nb >= 0) Ax += c->AF[k] * x[nb];
        }
        res[n] = fabs(c->b[n] - Ax);
    }
    (void)s;
}

/* Fixed-chunk sums so the value does not depend on the thread count. */
#define RCHUNK 4096
static double reduce(const double* v, int N, int method /*0 none 1 abs 2 sq*/, int op /*0 sum 1 max*/) {
    const int nChunks = (N + RCHUNK - 1) / RCHUNK;
    double* part = (double*)xcalloc((size_t)(nChunks ? nChunks : 1), 8);
#pragma omp parallel for schedule(static)
    for (int ch = 0; ch < nChunks; ch++) {
        const int a = ch * RCHUNK, b = (a + RCHUNK < N) ? a + RCHUNK : N;
        double acc = op ? -INFINITY : 0.0;
        for (int i = a; i < b; i++) {
            double x = v[i];
            if (method == 1) x = fabs(x);
            else if (method == 2) x = x * x;
            acc = op ? fmax(acc, x) : acc + x;
        }
        part[ch] = acc;
    }
    double acc = op ? -INFINITY : 0.0;
    for (int ch = 0; ch < nChunks; ch++) acc = op ? fmax(acc, part[ch]) : acc + part[ch];
    free(part);
    return acc;
}

static void continuity_residual(orc_solver* s) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        double imb = 0.0;
        for (int k = s->cfs[n]; k < s->cfs[n + 1]; k++) {
            const int f = s->cfi[k];
            const double m = s->mDot[f];
            if (s->owner[f] == n) imb += m;
            else if (s->neighbor[f] == n) imb -= m;
        }
        s->resC[n] = imb;
    }
}

/* residuals.cu:37-100 residualAllHost: U, V, Continuity, Temperature,
 * Concentration (entries 3 and 4 read the scalar settings). */
static void residual_host(orc_solver* s, int scaleIteration) {
    const orc_config* c = &s->cfg;
    double* res[5] = { s->resU, s->resV, s->resC, s->resT, s->resCc };
    double* scl[5] = { s->scaleU, s->scaleV, NULL, s->scaleT, s->scaleCc };
    double* val[5] = { &s->resVal[0], &s->resVal[1], &s->resVal[2], &s->resValS[0], &s->resValS[1] };
    double* sv[5] = { &s->scaleVal[0], &s->scaleVal[1], &s->scaleVal[2], &s->scaleValS[0], &s->scaleValS[1] };
    const int norm[5] = { c->resNorm[0], c->resNorm[1], c->resNorm[2], c->scalarResNorm[0], c->scalarResNorm[1] };
    const int scale[5] = { c->resScale[0], c->resScale[1], c->resScale[2], c->scalarResScale[0], c->scalarResScale[1] };
    const int en[5] = { c->resEnabled[0], c->resEnabled[1], c->resEnabled[2], c->scalarResEnabled[0],
                        c->scalarResEnabled[1] };
    const int N = s->N;
    for (int i = 0; i < 5; i++) {
        if (!en[i]) continue;
        if (i == 2) {
            *val[i] = reduce(res[i], N, 1, 0);
        } else {
            switch (norm[i]) {
            case NORM_L1: *val[i] = reduce(res[i], N, 1, 0); break;
            case NORM_L2: *val[i] = reduce(res[i], N, 2, 0); break;
            case NORM_LINF: *val[i] = reduce(res[i], N, 1, 1); break;
            }
            switch (scale[i]) {
            case SCALE_NONE: *sv[i] = 1.0; break;
            case SCALE_N: *sv[i] = N; break;
            case SCALE_SQRT_N: *sv[i] = sqrt((double)N); break;
            case SCALE_DIAG: *sv[i] = reduce(scl[i], N, 1, 0); break;
            }
        }
    }
    for (int i = 0; i < 5; i++) {
        if (!en[i]) continue;
        if (i == 2 && scaleIteration < 5) *sv[i] = fmax(*val[i], 0.0);
        if (*sv[i] == 0.0) continue;
        if (norm[i] == NORM_L2) *val[i] = sqrt(*val[i]);
        *val[i] /= *sv[i];
    }
}

/* solver.cpp:59-72 residualsConverged */
static int residuals_converged(const orc_solver* s) {
    const orc_config* c = &s->cfg;
    const int en[5] = { c->resEnabled[0], c->resEnabled[1], c->resEnabled[2], c->scalarResEnabled[0],
                        c->scalarResEnabled[1] };
    const double val[5] = { s->resVal[0], s->resVal[1], s->resVal[2], s->resValS[0], s->resValS[1] };
    const double tol[5] = { c->resTol[0], c->resTol[1], c->resTol[2], c->scalarResTol[0], c->scalarResTol[1] };
    int any = 0;
    for (int i = 0; i < 5; i++) {
        if (!en[i]) continue;
        any = 1;
        if (!(val[i] <= tol[i])) return 0;
    }
    return any;
}

/* ---------------- set-up ---------------- */
static void copy_bc(bcf* d, const orc_bc_field* h, int zeroValues) {
    memset(d, 0, sizeof(*d));
    if (!h || h->nGroups <= 0) return;
    const int G = h->nGroups;
    d->nGroups = G;
    /* memory_manger.cpp:72-83 defaults, 110-136 kinetics and Km^n, K2^m */
    double** kin[9] = { &d->vmax, &d->km, &d->nexp, &d->mexp, &d->k2, &d->v2, &d->Rtot, &d->kmN, &d->k2M };
    for (int i = 0; i < 9; i++) *kin[i] = (double*)xcalloc((size_t)G, 8);
    for (int g = 0; g < G; g++) {
        d->vmax[g] = h->vmaxByGroup ? h->vmaxByGroup[g] : 0.0;
        d->km[g] = h->kmByGroup ? h->kmByGroup[g] : 0.0;
        d->nexp[g] = h->nByGroup ? h->nByGroup[g] : 1.0;
        d->mexp[g] = h->mByGroup ? h->mByGroup[g] : 1.0;
        d->k2[g] = h->k2ByGroup ? h->k2ByGroup[g] : 0.0;
        d->v2[g] = h->v2ByGroup ? h->v2ByGroup[g] : 0.0;
        d->Rtot[g] = h->RtotByGroup ? h->RtotByGroup[g] : 0.0;
        d->kmN[g] = pow(d->km[g], d->nexp[g]);
        d->k2M[g] = pow(d->k2[g], d->mexp[g]);
    }
    d->type = (uint8_t*)xcalloc((size_t)G, 1);
    d->btype = (uint8_t*)xcalloc((size_t)G, 1);
    d->value = (double*)xcalloc((size_t)G, 8);
    d->mean = (double*)xcalloc((size_t)G, 8);
    d->length = (double*)xcalloc((size_t)G, 8);
    d->puls = (uint8_t*)xcalloc((size_t)G, 1);
    d->amp = (double*)xcalloc((size_t)G, 8);
    d->freq = (double*)xcalloc((size_t)G, 8);
    memcpy(d->type, h->typeByGroup, (size_t)G);
    if (h->boundaryTypeByGroup) memcpy(d->btype, h->boundaryTypeByGroup, (size_t)G);
    for (int g = 0; g < G; g++) {
        d->value[g] = zeroValues ? 0.0 : h->valueByGroup[g];
        d->mean[g] = d->value[g];
        d->length[g] = h->lengthByGroup ? h->lengthByGroup[g] : 0.0;
        if (h->pulsatileByGroup && h->pulsatileByGroup[g]) {
            d->puls[g] = 1;
            d->amp[g] = h->amplitudeByGroup[g];
            d->freq[g] = h->frequencyByGroup[g];
        }
    }
}
static void free_bc(bcf* d) {
    free(d->type); free(d->btype); free(d->value); free(d->mean); free(d->length);
    free(d->puls); free(d->amp); free(d->freq);
    free(d->vmax); free(d->km); free(d->nexp); free(d->mexp); free(d->k2); free(d->v2); free(d->Rtot);
    free(d->kmN); free(d->k2M);
}

#define DUP(dst, src, n, T) do { dst = (T*)xcalloc((size_t)(n) ? (size_t)(n) : 1, sizeof(T)); memcpy(dst, src, (size_t)(n) * sizeof(T)); } while (0)

/* memory_manger.cpp:325-409 buildMeshColoring (greedy) */
static void build_coloring(orc_solver* s) {
    const int N = s->N;
    s->color = (int32_t*)xcalloc((size_t)N, 4);
    for (int c = 0; c < N; c++) s->color[c] = -1;
    int stampCap = 16;
    int* stamp = (int*)xcalloc((size_t)stampCap, sizeof(int));
    int stampSize = 0;
    int nColors = 0;
    for (int c = 0; c < N; c++) {
        for (int k = s->cfs[c]; k < s->cfs[c + 1]; k++) {
            const int nb = s->slotNb[k];
            if (nb < 0 || s->color[nb] < 0) continue;
            const int cl = s->color[nb];
            if (cl >= stampSize) {
                if (cl + 1 > stampCap) { while (cl + 1 > stampCap) stampCap *= 2; stamp = (int*)realloc(stamp, (size_t)stampCap * sizeof(int)); }
                for (int q = stampSize; q <= cl; q++) stamp[q] = -1;
                stampSize = cl + 1;
            }
            stamp[cl] = c;
        }
        int pick = 0;
        while (pick < stampSize && stamp[pick] == c) pick++;
        s->color[c] = pick;
        if (pick >= nColors) nColors = pick + 1;
    }
    free(stamp);
    s->nColors = nColors;
    s->colorStart = (int32_t*)xcalloc((size_t)nColors + 1, 4);
    for (int c = 0; c < N; c++) s->colorStart[s->color[c] + 1]++;
    for (int k = 0; k < nColors; k++) s->colorStart[k + 1] += s->colorStart[k];
    s->cellOrder = (int32_t*)xcalloc((size_t)N, 4);
    int32_t* fill = (int32_t*)xcalloc((size_t)nColors + 1, 4);
    memcpy(fill, s->colorStart, ((size_t)nColors + 1) * 4);
    for (int c = 0; c < N; c++) s->cellOrder[fill[s->color[c]]++] = c;
    free(fill);
}

orc_solver* orc_create(const orc_mesh* m, const orc_bc_field* bu, const orc_bc_field* bv,
                       const orc_bc_field* bp, const orc_config* cfg) {
    return orc_create_ex(m, bu, bv, bp, NULL, NULL, cfg);
}

orc_solver* orc_create_ex(const orc_mesh* m, const orc_bc_field* bu, const orc_bc_field* bv,
                          const orc_bc_field* bp, const orc_bc_field* bt, const orc_bc_field* bcc,
                          const orc_config* cfg) {
    if (!m || m->nCells <= 0 || !cfg) return NULL;
    if ((cfg->solveEnergy && !bt) || (cfg->solveConcentration && !bcc)) return NULL;
    /* solver.cpp:887-889: both scalars are divided through by rho */
    if ((cfg->solveEnergy || cfg->solveConcentration) && !(cfg->rho > 0.0)) return NULL;
    orc_solver* s = (orc_solver*)xcalloc(1, sizeof(orc_solver));
    s->cfg = *cfg;
    /* solver.cpp:537-547 runCheck clamps */
    if (s->cfg.maxIter < 1) s->cfg.maxIter = 50;
    if (s->cfg.checkConv < 1) s->cfg.checkConv = 1;
    if (s->cfg.linearMaxIter < 1) s->cfg.linearMaxIter = 20;
    /* solver.cpp:548-555: no non-orthogonal corrector on a structured mesh */
    if (s->cfg.structuredMesh) s->cfg.useNonOrthCorrector = 0;
    const int N = m->nCells, F = m->nFaces;
    s->N = N;
    s->F = F;
    s->S = m->cellFaceStart[N];
    DUP(s->owner, m->faceOwner, F, int32_t);
    DUP(s->neighbor, m->faceNeighbor, F, int32_t);
    DUP(s->group, m->faceBoundaryGroupID, F, int32_t);
    DUP(s->nZ, m->faceNormalZ, F, double);
    DUP(s->nR, m->faceNormalR, F, double);
    DUP(s->fcZ, m->faceCenterZ, F, double);
    DUP(s->fcR, m->faceCenterR, F, double);
    DUP(s->area, m->faceArea, F, double);
    DUP(s->ccZ, m->cellCenterZ, N, double);
    DUP(s->ccR, m->cellCenterR, N, double);
    DUP(s->vol, m->cellVolume, N, double);
    DUP(s->cfs, m->cellFaceStart, N + 1, int32_t);
    DUP(s->cfi, m->cellFaceIDs, s->S, int32_t);

    /* memory_manger.cpp:512-617 preComputeVariables */
    s->invDPN = (double*)xcalloc((size_t)F, 8);
    s->wP = (double*)xcalloc((size_t)F, 8);
    s->dPB = (double*)xcalloc((size_t)F, 8);
    s->length2D = (double*)xcalloc((size_t)F, 8);
    s->invA2D = (double*)xcalloc((size_t)N, 8);
    s->lsqWZ = (double*)xcalloc((size_t)F, 8);
    s->lsqWR = (double*)xcalloc((size_t)F, 8);
    s->lsqIZZ = (double*)xcalloc((size_t)N, 8);
    s->lsqIZR = (double*)xcalloc((size_t)N, 8);
    s->lsqIRR = (double*)xcalloc((size_t)N, 8);
    for (int c = 0; c < N; c++) s->invA2D[c] = 2.0 * ORC_PI * s->ccR[c] / s->vol[c];
    double* lsqDZ = (double*)xcalloc((size_t)F, 8);
    double* lsqDR = (double*)xcalloc((size_t)F, 8);
    for (int f = 0; f < F; f++) {
        s->length2D[f] = s->area[f] / (2 * ORC_PI * s->fcR[f]);
        const int nb = s->neighbor[f], o = s->owner[f];
        const double dzPF = s->fcZ[f] - s->ccZ[o];
        const double drPF = s->fcR[f] - s->ccR[o];
        if (nb < 0) {
            s->dPB[f] = fabs(dzPF * s->nZ[f] + drPF * s->nR[f]);
        } else {
            const double dzNF = s->fcZ[f] - s->ccZ[nb];
            const double drNF = s->fcR[f] - s->ccR[nb];
            const double dzPN = s->ccZ[nb] - s->ccZ[o];
            const double drPN = s->ccR[nb] - s->ccR[o];
            const double dPF = fabs(dzPF * s->nZ[f] + drPF * s->nR[f]);
            const double dNF = fabs(dzNF * s->nZ[f] + drNF * s->nR[f]);
            const double dPN = sqrt(dzPN * dzPN + drPN * drPN);
            const double denom = dPF + dNF;
            s->invDPN[f] = 1.0 / dPN;
            s->wP[f] = dNF / denom;
        }
        const double dz = (nb >= 0 ? s->ccZ[nb] : s->fcZ[f]) - s->ccZ[o];
        const double dr = (nb >= 0 ? s->ccR[nb] : s->fcR[f]) - s->ccR[o];
        const double w = 1.0 / (dz * dz + dr * dr);
        lsqDZ[f] = dz;
        lsqDR[f] = dr;
        s->lsqWZ[f] = w * dz;
        s->lsqWR[f] = w * dr;
    }
    for (int c = 0; c < N; c++) {
        double Szz = 0.0, Szr = 0.0, Srr = 0.0;
        for (int k = s->cfs[c]; k < s->cfs[c + 1]; k++) {
            const int f = s->cfi[k];
            Szz += s->lsqWZ[f] * lsqDZ[f];
            Szr += s->lsqWZ[f] * lsqDR[f];
            Srr += s->lsqWR[f] * lsqDR[f];
        }
        const double det = Szz * Srr - Szr * Szr;
        if (fabs(det) <= 1.0e-30) continue;
        s->lsqIZZ[c] = Srr / det;
        s->lsqIZR[c] = -Szr / det;
        s->lsqIRR[c] = Szz / det;
    }
    free(lsqDZ);
    free(lsqDR);

    /* memory_manger.cpp:287-323 buildCellFaceCSR */
    s->slotNb = (int32_t*)xcalloc((size_t)(s->S ? s->S : 1), 4);
    for (int c = 0; c < N; c++)
        for (int k = s->cfs[c]; k < s->cfs[c + 1]; k++) {
            const int f = s->cfi[k];
            int nb = -1;
            if (f >= 0 && f < F) {
                if (s->owner[f] == c) nb = s->neighbor[f];
                else if (s->neighbor[f] == c) nb = s->owner[f];
            }
            s->slotNb[k] = nb;
        }

    copy_bc(&s->bcU, bu, 0);
    copy_bc(&s->bcV, bv, 0);
    copy_bc(&s->bcP, bp, 0);
    copy_bc(&s->bcPP, bp, 1); /* solver.cpp:791-795: p types, zero values */
    if (cfg->solveEnergy) copy_bc(&s->bcT, bt, 0);
    if (cfg->solveConcentration) copy_bc(&s->bcC, bcc, 0);

    coeffs* cs[5] = { &s->cu, &s->cv, &s->cpp, &s->ct, &s->cc };
    for (int i = 0; i < 5; i++) {
        cs[i]->N = N;
        cs[i]->S = s->S;
        cs[i]->AC = (double*)xcalloc((size_t)N, 8);
        cs[i]->b = (double*)xcalloc((size_t)N, 8);
        cs[i]->invAC = (double*)xcalloc((size_t)N, 8);
        cs[i]->AF = (double*)xcalloc((size_t)(s->S ? s->S : 1), 8);
        cs[i]->faceStart = s->cfs;
        cs[i]->faceNeighbor = s->slotNb;
    }
#define AL(p, n) p = (double*)xcalloc((size_t)(n) ? (size_t)(n) : 1, 8)
    AL(s->u, N); AL(s->v, N); AL(s->p, N); AL(s->pp, N); AL(s->uTemp, N); AL(s->vTemp, N); AL(s->ppTemp, N);
    AL(s->DU, N); AL(s->DV, N); AL(s->gradPZ, N); AL(s->gradPR, N); AL(s->gradUZ, N); AL(s->gradUR, N);
    AL(s->gradVZ, N); AL(s->gradVR, N); AL(s->uOld, N); AL(s->vOld, N); AL(s->uOld2, N); AL(s->vOld2, N);
    AL(s->mDot, F); AL(s->resU, N); AL(s->resV, N); AL(s->resC, N); AL(s->scaleU, N); AL(s->scaleV, N);
    AL(s->T, N); AL(s->C, N); AL(s->TTemp, N); AL(s->CTemp, N); AL(s->TOld, N); AL(s->COld, N);
    AL(s->TOld2, N); AL(s->COld2, N); AL(s->gradTZ, N); AL(s->gradTR, N); AL(s->gradCZ, N); AL(s->gradCR, N);
    AL(s->resT, N); AL(s->resCc, N); AL(s->scaleT, N); AL(s->scaleCc, N); AL(s->cw, F); AL(s->ocrWall, F);
#undef AL
    if (s->cfg.linearType == 1) build_coloring(s);
    if (s->cfg.useMultigrid) build_levels(s);
    return s;
}

static void clear_coeffs(coeffs* c) {
    memset(c->AC, 0, (size_t)c->N * 8);
    memset(c->b, 0, (size_t)c->N * 8);
    memset(c->AF, 0, (size_t)c->S * 8);
}

static void under_relax(orc_solver* s, coeffs* c, const double* x, double alpha) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        const double ACo = c->AC[n];
        if (fabs(ACo) < 1.0e-30) continue;
        c->AC[n] = ACo / alpha;
        c->b[n] += ((1.0 - alpha) / alpha) * ACo * x[n];
    }
}

static void inverse_diag(coeffs* c) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < c->N; n++) {
        const double AC = c->AC[n];
        c->invAC[n] = (fabs(AC) < 1.0e-30) ? 0.0 : 1.0 / AC;
    }
}

static void add_transient(orc_solver* s, coeffs* c, const double* old, const double* old2, double cap, double dt) {
    if (!old || dt <= 0.0) return;
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        const double cV = cap * s->vol[n];
        if (old2) {
            const double a = cV / (2.0 * dt);
            c->AC[n] += 3.0 * a;
            c->b[n] += a * (4.0 * old[n] - old2[n]);
        } else {
            const double a = cV / dt;
            c->AC[n] += a;
            c->b[n] += a * old[n];
        }
    }
}

/* solver.cpp:375-424 updatePulsatileBoundaryValues */
static void update_pulsatile(bcf* bc, double t) {
    for (int g = 0; g < bc->nGroups; g++) {
        if (!bc->puls[g]) continue;
        const double twoPi = 2.0 * ORC_PI;
        bc->value[g] = bc->mean[g] * (1.0 + bc->amp[g] * sin(twoPi * bc->freq[g] * t));
    }
}

/* One transported scalar after the corrections (solver.cpp:1218-1238): the
 * volumetric flux mDot / rho convects it, `gamma` is its kinematic
 * diffusivity, the unsteady term has capacity 1. */
static void scalar_transport(orc_solver* s, coeffs* cf, const bcf* bc, double* phi, double* phiTemp, double* gZ,
                             double* gR, const double* old, const double* old2, double gamma, double alpha) {
    const orc_config* c = &s->cfg;
    const int applyNonOrtho = c->useNonOrthCorrector ? 1 : 0;
    const int conv = c->addConvectionTerm ? 1 : 0;
    const int convNeedsGrad = conv && (c->convectionScheme == CONV_SOU || c->convectionScheme == CONV_QUICK);
    if (applyNonOrtho || convNeedsGrad) compute_gradient(s, bc, phi, gZ, gR);
    add_transport(s, cf, bc, phi, gZ, gR, applyNonOrtho, gamma, conv, c->convectionScheme, 1.0 / c->rho);
    if (c->transient) add_transient(s, cf, old, old2, 1.0, c->dt);
    under_relax(s, cf, phi, alpha);
    inverse_diag(cf);
    linear_solve(s, cf, phi, phiTemp);
}

/* One SIMPLE iteration, solver.cpp:1116-1238. sOld / sOld2 are the scalar
 * time levels the scalar step reads (T, C); see orc_run for which buffers. */
static void simple_iteration(orc_solver* s, const double* uOld2, const double* vOld2, int bdf2,
                             const double* const sOld[2], const double* const sOld2[2]) {
    const orc_config* c = &s->cfg;
    const int applyNonOrtho = c->useNonOrthCorrector ? 1 : 0;
    const int conv = c->addConvectionTerm ? 1 : 0;
    const int convNeedsGrad = conv && (c->convectionScheme == CONV_SOU || c->convectionScheme == CONV_QUICK);
    clear_coeffs(&s->cu);
    clear_coeffs(&s->cv);
    clear_coeffs(&s->cpp);
    if (c->solveEnergy) clear_coeffs(&s->ct);
    if (c->solveConcentration) clear_coeffs(&s->cc);
    if (applyNonOrtho || convNeedsGrad) {
        compute_gradient(s, &s->bcU, s->u, s->gradUZ, s->gradUR);
        compute_gradient(s, &s->bcV, s->v, s->gradVZ, s->gradVR);
    }
    add_transport(s, &s->cu, &s->bcU, s->u, s->gradUZ, s->gradUR, applyNonOrtho, c->mu, conv, c->convectionScheme, 1.0);
    add_transport(s, &s->cv, &s->bcV, s->v, s->gradVZ, s->gradVR, applyNonOrtho, c->mu, conv, c->convectionScheme, 1.0);
    /* solver_util.cu:454-470 hoop term */
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        const double r = s->ccR[n];
        s->cv.AC[n] += c->mu * s->vol[n] / (r * r);
    }
    if (c->transient) {
        add_transient(s, &s->cu, s->uOld, uOld2, c->rho, c->dt);
        add_transient(s, &s->cv, s->vOld, vOld2, c->rho, c->dt);
    }
    compute_gradient(s, &s->bcP, s->p, s->gradPZ, s->gradPR);
    /* simple.cu:144-164 */
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        const double V = s->vol[n];
        s->cu.b[n] += -V * s->gradPZ[n];
        s->cv.b[n] += -V * s->gradPR[n];
    }
    under_relax(s, &s->cu, s->u, c->alphaU);
    under_relax(s, &s->cv, s->v, c->alphaU);
    inverse_diag(&s->cu);
    inverse_diag(&s->cv);
    /* solver_util.cu:127-144 */
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        s->DU[n] = s->vol[n] * s->cu.invAC[n];
        s->DV[n] = s->vol[n] * s->cv.invAC[n];
    }
    linear_solve(s, &s->cu, s->u, s->uTemp);
    linear_solve(s, &s->cv, s->v, s->vTemp);
    create_pp_coeff(s);
    inverse_diag(&s->cpp);
    rhie_chow(s);
    memset(s->pp, 0, (size_t)s->N * 8);
    for (int corr = 0; corr <= applyNonOrtho; corr++) {
        const int cross = corr > 0;
        if (cross) compute_gradient(s, &s->bcPP, s->pp, s->gradPZ, s->gradPR);
        create_pp_rhs(s, cross);
        if (c->useMultigrid) mg_run(s);
        else linear_solve(s, &s->cpp, s->pp, s->ppTemp);
    }
    compute_gradient(s, &s->bcPP, s->pp, s->gradPZ, s->gradPR);
    /* simple.cu:166-179 */
#pragma omp parallel for schedule(static)
    for (int n = 0; n < s->N; n++) {
        s->u[n] -= s->DU[n] * s->gradPZ[n];
        s->v[n] -= s->DV[n] * s->gradPR[n];
        s->p[n] += c->alphaP * s->pp[n];
    }
    update_mass_flux(s, applyNonOrtho);
    /* energy (k / (rho cp), relaxed with alphaU) then concentration (D, unrelaxed) */
    if (c->solveEnergy)
        scalar_transport(s, &s->ct, &s->bcT, s->T, s->TTemp, s->gradTZ, s->gradTR, sOld[0], bdf2 ? sOld2[0] : NULL,
                         c->k / (c->rho * c->cp), c->alphaU);
    if (c->solveConcentration)
        scalar_transport(s, &s->cc, &s->bcC, s->C, s->CTemp, s->gradCZ, s->gradCR, sOld[1], bdf2 ? sOld2[1] : NULL,
                         c->D, 1.0);
}

int orc_run(orc_solver* s, int continueRun, int* converged) {
    const orc_config* c = &s->cfg;
    if (!continueRun) {
        s->simTime = 0.0;
    }
    const double timeOffset = (c->transient && continueRun) ? s->simTime : 0.0;
    const int useBDF2 = c->transient && c->timeScheme == 1;
    const int numSteps = c->transient ? (int)ceil(c->tEnd / c->dt) : 1;
    /* solver.cpp:985-1009: the scalar step reads the time levels through
     * pointers taken from simple.tempOld / tempOld2 (concOld / concOld2) once,
     * before the time loop, while the BDF2 shift below swaps the names
     * simple.tempOld <-> tempOld2 every step. The scalar step therefore keeps
     * reading the same two buffers: correct levels on odd steps, the two
     * levels exchanged on even steps from the third on. Reproduced as is. */
    const double* const sOld[2] = { s->TOld, s->COld };
    const double* const sOld2[2] = { s->TOld2, s->COld2 };
    int iters = 0;
    int conv = 0;
    for (int t = 0; t < numSteps; t++) {
        if (c->transient) {
            const double stepTime = timeOffset + (double)(t + 1) * c->dt;
            update_pulsatile(&s->bcU, stepTime);
            update_pulsatile(&s->bcV, stepTime);
            if (useBDF2) {
                double* tmp;
                tmp = s->uOld2; s->uOld2 = s->uOld; s->uOld = tmp;
                tmp = s->vOld2; s->vOld2 = s->vOld; s->vOld = tmp;
                tmp = s->TOld2; s->TOld2 = s->TOld; s->TOld = tmp;
                tmp = s->COld2; s->COld2 = s->COld; s->COld = tmp;
            }
            memcpy(s->uOld, s->u, (size_t)s->N * 8);
            memcpy(s->vOld, s->v, (size_t)s->N * 8);
            if (c->solveEnergy) memcpy(s->TOld, s->T, (size_t)s->N * 8);
            if (c->solveConcentration) memcpy(s->COld, s->C, (size_t)s->N * 8);
        }
        const int bdf2 = useBDF2 && t > 0;
        conv = 0;
        for (int k = 0; k < c->maxIter; k++) {
            simple_iteration(s, bdf2 ? s->uOld2 : NULL, bdf2 ? s->vOld2 : NULL, bdf2, sOld, sOld2);
            if (k % c->checkConv == 0) {
                residual_raw(s, &s->cu, s->u, s->resU, s->scaleU, c->resScale[0] == SCALE_DIAG);
                residual_raw(s, &s->cv, s->v, s->resV, s->scaleV, c->resScale[1] == SCALE_DIAG);
                /* unsolved scalars keep all-zero systems and residuals */
                if (c->solveEnergy)
                    residual_raw(s, &s->ct, s->T, s->resT, s->scaleT, c->scalarResScale[0] == SCALE_DIAG);
                if (c->solveConcentration)
                    residual_raw(s, &s->cc, s->C, s->resCc, s->scaleCc, c->scalarResScale[1] == SCALE_DIAG);
                continuity_residual(s);
                residual_host(s, c->transient ? k : s->currentIteration);
                conv = residuals_converged(s);
            }
            s->currentIteration++;
            iters++;
            if (conv) break;
        }
        if (c->transient) s->simTime = timeOffset + (double)(t + 1) * c->dt;
    }
    /* solver.cpp:1330-1332: final gradients of u, v, p for the solution fields */
    compute_gradient(s, &s->bcU, s->u, s->gradUZ, s->gradUR);
    compute_gradient(s, &s->bcV, s->v, s->gradVZ, s->gradVR);
    compute_gradient(s, &s->bcP, s->p, s->gradPZ, s->gradPR);
    if (c->solveEnergy) compute_gradient(s, &s->bcT, s->T, s->gradTZ, s->gradTR);
    if (c->solveConcentration) compute_gradient(s, &s->bcC, s->C, s->gradCZ, s->gradCR);
    if (converged) *converged = conv;
    return iters;
}

/* ---------------- accessors ---------------- */
static double* field_ptr(const orc_solver* s, const char* name, size_t* len) {
    const size_t N = (size_t)s->N, F = (size_t)s->F, S = (size_t)s->S;
    struct { const char* n; double* p; size_t l; } t[] = {
        { "u", s->u, N }, { "v", s->v, N }, { "p", s->p, N }, { "pp", s->pp, N }, { "mDot", s->mDot, F },
        { "DU", s->DU, N }, { "DV", s->DV, N }, { "gradPZ", s->gradPZ, N }, { "gradPR", s->gradPR, N },
        { "gradUZ", s->gradUZ, N }, { "gradUR", s->gradUR, N }, { "gradVZ", s->gradVZ, N }, { "gradVR", s->gradVR, N },
        { "AC_u", s->cu.AC, N }, { "b_u", s->cu.b, N }, { "AF_u", s->cu.AF, S }, { "invAC_u", s->cu.invAC, N },
        { "AC_v", s->cv.AC, N }, { "b_v", s->cv.b, N }, { "AF_v", s->cv.AF, S }, { "invAC_v", s->cv.invAC, N },
        { "AC_pp", s->cpp.AC, N }, { "b_pp", s->cpp.b, N }, { "AF_pp", s->cpp.AF, S }, { "invAC_pp", s->cpp.invAC, N },
        { "res_U", s->resU, N }, { "res_V", s->resV, N }, { "res_Continuity", s->resC, N },
        { "uOld", s->uOld, N }, { "vOld", s->vOld, N }, { "uOld2", s->uOld2, N }, { "vOld2", s->vOld2, N },
        { "invDPN", s->invDPN, F }, { "wP", s->wP, F }, { "dPB", s->dPB, F }, { "length2D", s->length2D, F },
        { "lsqWZ", s->lsqWZ, F }, { "lsqWR", s->lsqWR, F }, { "invA2D", s->invA2D, N },
        { "lsqInvZZ", s->lsqIZZ, N }, { "lsqInvZR", s->lsqIZR, N }, { "lsqInvRR", s->lsqIRR, N },
        { "T", s->T, N }, { "C", s->C, N }, { "gradTZ", s->gradTZ, N }, { "gradTR", s->gradTR, N },
        { "gradCZ", s->gradCZ, N }, { "gradCR", s->gradCR, N },
        { "AC_T", s->ct.AC, N }, { "b_T", s->ct.b, N }, { "AF_T", s->ct.AF, S }, { "invAC_T", s->ct.invAC, N },
        { "AC_C", s->cc.AC, N }, { "b_C", s->cc.b, N }, { "AF_C", s->cc.AF, S }, { "invAC_C", s->cc.invAC, N },
        { "TOld", s->TOld, N }, { "COld", s->COld, N }, { "TOld2", s->TOld2, N }, { "COld2", s->COld2, N },
        { "res_T", s->resT, N }, { "res_C", s->resCc, N }, { "cw", s->cw, F }, { "ocrWall", s->ocrWall, F },
    };
    for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); i++)
        if (strcmp(t[i].n, name) == 0) { *len = t[i].l; return t[i].p; }
    return NULL;
}

int orc_get(const orc_solver* s, const char* name, double* out, size_t n) {
    size_t len = 0;
    double* p = field_ptr(s, name, &len);
    if (!p || n < len) return -1;
    memcpy(out, p, len * 8);
    return (int)len;
}

int orc_set(orc_solver* s, const char* name, const double* in, size_t n) {
    size_t len = 0;
    double* p = field_ptr(s, name, &len);
    if (!p || n < len) return -1;
    memcpy(p, in, len * 8);
    return (int)len;
}

void orc_last_residuals(const orc_solver* s, double out[3]) {
    for (int i = 0; i < 3; i++) out[i] = s->resVal[i];
}

void orc_scalar_residuals(const orc_solver* s, double out[2]) {
    out[0] = s->resValS[0];
    out[1] = s->resValS[1];
}

int orc_iterations(const orc_solver* s) { return s->currentIteration; }

int orc_mg_levels(const orc_solver* s, int32_t* cells, int maxLevels) {
    for (int l = 0; l < s->nLevels && l < maxLevels; l++) cells[l] = s->lv[l].N;
    return s->nLevels;
}

int orc_mg_level_maps(const orc_solver* s, int level, int32_t* c2c, int32_t* f2c, int32_t* cfs, int32_t* cfn) {
    if (level < 0 || level >= s->nLevels - 1) return -1;
    const mglevel* f = &s->lv[level];
    const mglevel* c = &s->lv[level + 1];
    if (c2c) memcpy(c2c, f->cellToCoarse, (size_t)f->N * 4);
    if (f2c) memcpy(f2c, f->fineSlotToCoarseSlot, (size_t)f->S * 4);
    if (cfs) memcpy(cfs, c->faceStart, ((size_t)c->N + 1) * 4);
    if (cfn) memcpy(cfn, c->faceNeighbor, (size_t)c->S * 4);
    return c->S;
}

int orc_coloring(const orc_solver* s, int32_t* out) {
    if (!s->color) return 0;
    memcpy(out, s->color, (size_t)s->N * 4);
    return s->nColors;
}

void orc_destroy(orc_solver* s) {
    if (!s) return;
    free(s->owner); free(s->neighbor); free(s->group); free(s->cfs); free(s->cfi);
    free(s->nZ); free(s->nR); free(s->fcZ); free(s->fcR); free(s->area); free(s->ccZ); free(s->ccR); free(s->vol);
    free(s->invDPN); free(s->wP); free(s->dPB); free(s->invA2D); free(s->length2D);
    free(s->lsqWZ); free(s->lsqWR); free(s->lsqIZZ); free(s->lsqIZR); free(s->lsqIRR); free(s->slotNb);
    free_bc(&s->bcU); free_bc(&s->bcV); free_bc(&s->bcP); free_bc(&s->bcPP); free_bc(&s->bcT); free_bc(&s->bcC);
    coeffs* cs[5] = { &s->cu, &s->cv, &s->cpp, &s->ct, &s->cc };
    for (int i = 0; i < 5; i++) { free(cs[i]->AC); free(cs[i]->b); free(cs[i]->invAC); free(cs[i]->AF); }
    double* sc[] = { s->T, s->C, s->TTemp, s->CTemp, s->TOld, s->COld, s->TOld2, s->COld2, s->gradTZ, s->gradTR,
                     s->gradCZ, s->gradCR, s->resT, s->resCc, s->scaleT, s->scaleCc, s->cw, s->ocrWall };
    for (size_t i = 0; i < sizeof(sc) / sizeof(sc[0]); i++) free(sc[i]);
    free(s->u); free(s->v); free(s->p); free(s->pp); free(s->uTemp); free(s->vTemp); free(s->ppTemp);
    free(s->DU); free(s->DV); free(s->gradPZ); free(s->gradPR); free(s->gradUZ); free(s->gradUR);
    free(s->gradVZ); free(s->gradVR); free(s->uOld); free(s->vOld); free(s->uOld2); free(s->vOld2);
    free(s->mDot); free(s->resU); free(s->resV); free(s->resC); free(s->scaleU); free(s->scaleV);
    for (int l = 0; l < s->nLevels; l++) {
        mglevel* L = &s->lv[l];
        free(L->faceStart); free(L->faceNeighbor); free(L->cellToCoarse); free(L->fineSlotToCoarseSlot);
        free(L->AC); free(L->AF); free(L->b); free(L->x); free(L->xNew); free(L->res);
    }
    free(s->lv);
    free(s->color); free(s->colorStart); free(s->cellOrder);
    free(s);
}
