// Headless stand-in for solver/header/mesh.h: only the members Solver reads
// (refreshFVMesh, getFVMesh, isReady, currentMeshType, boundaryGroups,
// boundaryEdges). The driver fills the FVMesh from the reference's own
// multiblock packer.
#pragma once
#include <vector>

#include "boundary_struct.h"
#include "multiblock.h"

class Mesh {
public:
    bool isReady = false;
    MeshType currentMeshType = MeshType::Structured;
    std::vector<BoundarySegmentGroup> boundaryGroups;
    std::vector<BoundaryEdge> boundaryEdges;
    FVMesh fvMesh;
    const FVMesh& getFVMesh() const { return fvMesh; }
    const FVMesh& refreshFVMesh() { return fvMesh; }
};
