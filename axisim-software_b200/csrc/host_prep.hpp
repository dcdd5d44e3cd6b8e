// host_prep.hpp -- host-side case preparation for the B200 SIMPLE solver.
//
// Pieces of the reference that run once per solve on the CPU: the multiblock
// packer (structs/multiblock.h), the trellis builder and boundary-face
// classification of Mesh (solver/source/mesh.cpp), the triangle-mesh builder,
// the agglomeration hierarchy
// (solver/source/multigrid.cu:79-325), the greedy colouring
// (manager/source/memory_manger.cpp:325-409) and the boundary defaults
// (manager/source/boundary_func.cpp:104-201, 333-378).
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

namespace axisim {

// fn(begin, end) over [0, n) split into contiguous ranges, one per host
// thread (up to 16); small ranges run on the calling thread. Each index is
// handled by exactly one call, so results do not depend on the split.
template <class Fn>
void parallelFor(int n, Fn&& fn, int grain = 16384) {
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = std::max(1, std::min({(int)(hw ? hw : 1), 16, n / std::max(grain, 1)}));
    if (nt <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve((size_t)nt - 1);
    const int chunk = (n + nt - 1) / nt;
    for (int t = 1; t < nt; t++) {
        const int b = t * chunk, e = std::min(n, b + chunk);
        if (b < e) pool.emplace_back([&fn, b, e] { fn(b, e); });
    }
    fn(0, std::min(n, chunk));
    for (std::thread& th : pool) th.join();
}

// Packed face-based mesh (FVMeshHostPacked, structs/solver_struct.h:400-429).
struct PackedMesh {
    int nCells = 0;
    int nFaces = 0;
    std::vector<int32_t> faceOwner, faceNeighbor, faceBoundaryGroupID;
    std::vector<double> faceNormalZ, faceNormalR, faceCenterZ, faceCenterR, faceArea;
    std::vector<double> cellCenterZ, cellCenterR, cellArea2D, cellVolume;
    std::vector<int32_t> cellFaceStart, cellFaceIDs;
};

struct BlockSpec {
    double z0 = 0, r0 = 0;
    double axialLength = 0;  int axialCells = 0;  int axialGrading = 0;  double axialCoef = 1;
    double radialLength = 0; int radialCells = 0; int radialGrading = 0; double radialCoef = 1;
    int edgeGroup[4] = {-1, -1, -1, -1};
};

// makeRectBlock + autoDetectInterfaces + assignGlobalNumbering + toPackedMesh.
// seamStatus = 1 when a non-conformal seam made every interface drop.
PackedMesh buildMultiblock(const std::vector<BlockSpec>& blocks, double tol, int defaultGroup,
                           int& seamStatus);

// Domain outline as Mesh keeps it (BoundaryVertex / BoundaryEdge,
// structs/boundary_struct.h:408-490): vertex positions and edges between
// them, each edge with its boundary group (-1 = unassigned).
struct Outline {
    std::vector<double> vz, vr;
    std::vector<int32_t> e0, e1, group;
};

// Mesh::pointInsideDomain (mesh.cpp:1177-1205): even-odd ray cast along +z
// against every edge, so obstacle loops make holes.
bool pointInsideDomain(const Outline& o, double z, double r);
// groupAtPoint (manager/source/math_func.cpp:175-196): the group of the
// nearest grouped edge closer than tol, else -1.
int groupAtPoint(const Outline& o, double z, double r, double tol);
// Mesh::classifyBoundaryFaces (mesh.cpp:1835-1846): every external face takes
// the group of the nearest outline edge, tolerance 1e-4 max(L, R, 1).
void classifyBoundaryFaces(PackedMesh& m, const Outline& o, double L, double R);
// Mesh::buildStructuredMultiBlock (mesh.cpp:2717-2762) from trellis lines and
// band cell counts (a uniform block per trellis cell whose centre lies inside
// the outline; one nz x nr block over [0, L] x [0, R] when none does), packed,
// then classified as createMultiBlockFVMesh does (mesh.cpp:2458-2460).
PackedMesh buildTrellis(const std::vector<double>& zLines, const std::vector<double>& rLines,
                        const std::vector<int>& zCells, const std::vector<int>& rCells, const Outline& o, double L,
                        double R, int nz, int nr, int& seamStatus);
// Mesh::createUnstructuredMesh (mesh.cpp:1848-2002): triangles (3 vertex ids
// each) over shared points, faces in triangle-edge order, then classified.
PackedMesh buildTriangleMesh(const std::vector<double>& pz, const std::vector<double>& pr,
                             const std::vector<int32_t>& tri, const Outline& o, double L, double R);

// One multigrid level's graph, CSR exactly as GridLevel (multigrid.cuh:29-68).
struct GridLevel {
    int nCells = 0;
    std::vector<int32_t> faceStart;
    std::vector<int32_t> faceNeighbor;
    std::vector<int32_t> cellToCoarse;          // empty on the coarsest level
    std::vector<int32_t> fineSlotToCoarseSlot;  // empty on the coarsest level
    int nFaceRefs() const { return (int)faceNeighbor.size(); }
    bool isCoarsest() const { return cellToCoarse.empty(); }
};

// buildCellFaceCSR (memory_manger.cpp:287-323) from a packed mesh.
GridLevel finestLevel(int nCells, int nFaces, const int32_t* cellFaceStart, const int32_t* cellFaceIDs,
                      const int32_t* faceOwner, const int32_t* faceNeighbor);

// buildLevels (multigrid.cu:298-325): coarsen until <= 64 cells or a pass
// shrinks by less than 0.8.
std::vector<GridLevel> buildHierarchy(GridLevel finest);

// A batch of independent cases packed into one mesh (cells
// [caseStart[c], caseStart[c+1]) of case c, no face between cases): each
// case's hierarchy built alone with buildHierarchy, then merged level by level
// (level l holds, in case order, the level-l cells of every case that has a
// level l). A case whose coarsest level is l < the deepest level has
// cellToCoarse = fineSlotToCoarseSlot = -1 there; its cells are that level's
// terminal cells, listed per level as [begin, end) pairs in terminal[l].
// Every level of every case is then exactly its standalone level.
std::vector<GridLevel> buildBatchHierarchy(const GridLevel& finest, const std::vector<int32_t>& caseStart,
                                           std::vector<std::vector<int32_t>>& terminal);

// Tiles for running several momentum Jacobi sweeps (linear_solver.cu:9-33)
// per launch out of shared memory. Cells are ordered along a Morton curve of
// their centres (one scale for both axes) and cut into runs of `tileCells`
// curve positions; a tile lists its own cells (layer 0) and then halo layers
// 1..S, layer k holding the neighbours of layer k-1 not listed before it, each
// layer in ascending cell order. Sweep s of a launch of s' <= S sweeps updates
// layers 0..s'-s from the values of layers 0..s'-s+1, so layer 0 ends with
// exactly the values of s' whole-mesh sweeps. A run whose cells and halo
// exceed `cap` local cells is halved until it fits. nb is the slot
// neighbour block [W][N] (-1 for a boundary or unused slot), W <= 4.
struct SweepTiles {
    int S = 0, cap = 0;
    std::vector<int32_t> tileStart;  // nTiles + 1 offsets into gid / lnb
    std::vector<int32_t> layerEnd;   // S + 1 per tile: local cells in layers 0..k
    std::vector<int32_t> gid;        // the mesh cell of each local cell
    std::vector<uint64_t> lnb;       // slot j's local neighbour in bits 16j..16j+15, 0xFFFF for none
    int nTiles() const { return (int)tileStart.size() - 1; }
};
// The slot neighbour block [W][N] of a packed mesh as the device builds it
// (slot j of cell n: the other cell of its j-th face, -1 for a boundary face
// or j beyond the cell's face count).
std::vector<int32_t> slotNeighbours(int nCells, int W, const int32_t* cellFaceStart, const int32_t* cellFaceIDs,
                                    const int32_t* faceOwner, const int32_t* faceNeighbor);
// With nCases > 0 the cells of case c are [caseStart[c], caseStart[c+1]) and
// the curve runs case by case, so a tile mixes cases only where one ends.
// Empty tiles (tileStart = {0}) when some cell with its S-layer halo alone
// exceeds cap.
SweepTiles buildSweepTiles(int nCells, int W, const int32_t* nb, const double* cz, const double* cr, int S, int cap,
                           int tileCells, const int32_t* caseStart = nullptr, int nCases = 0);

// buildMeshColoring (memory_manger.cpp:334-409): greedy colour per cell.
int greedyColoring(const GridLevel& g, std::vector<int32_t>& color);

// Launch-shape autotuning: the index of the candidate block size to use for a
// level, given each candidate's measured time. The default candidate is kept
// unless the fastest one beats it by more than the relative tolerance tol, so
// timing noise does not move a level off the default shape; a candidate with a
// non-finite or non-positive time is never picked.
int pickBlock(const std::vector<int>& candidates, const std::vector<double>& timeUs, int defaultIndex, double tol);

// Boundary defaults: effective BC for a group type and variable.
uint8_t defaultBCType(int boundaryType, int variable);
bool variableEditable(int variable, int boundaryType);

}  // namespace axisim
