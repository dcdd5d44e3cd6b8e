// foam_driver.cpp -- headless driver of the reference's OWN OpenFOAM case export.
//
// TEST INFRASTRUCTURE ONLY (pins axisim/foam.py). Links the reference's
// manager/source/file_converter.cpp and boundary_func.cpp, compiled unchanged
// from their sources (see Makefile), and lays a case out the way
// saveFoamCase does (manager/source/file_manager.cpp:1153-1258):
//   structured   : MultiBlockMesh from makeRectBlock + autoDetectInterfaces
//                  (structs/multiblock.h), blockMeshDictFromMultiblock,
//                  writeBlockMeshDict, initialFieldsFromDict
//   unstructured : points + triangles + the FVMesh faces given in the spec,
//                  polyMeshFromUnstructured, writePolyMesh, initialFieldsFromPolyMesh
// then the controlDict / fvSchemes / fvSolution / transportProperties /
// turbulenceProperties writers and writeInitialFields.
//
// Usage: foam_ref <spec.txt> <case-dir>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "boundary_func.h"
#include "boundary_struct.h"
#include "file_converter.h"
#include "file_struct.h"
#include "multiblock.h"

namespace {

BoundaryVariable varOf(const std::string& v) {
    if (v == "u") return BoundaryVariable::UVelocity;
    if (v == "v") return BoundaryVariable::VVelocity;
    if (v == "T") return BoundaryVariable::StaticTemperature;
    if (v == "C") return BoundaryVariable::Concentration;
    return BoundaryVariable::Pressure;
}

BoundaryCondition makeBC(int type, double value, double amp, double freq) {
    BoundaryCondition bc{};
    switch (type) {
        case 0: bc.params = DirichletParams{value}; break;
        case 1: bc.params = NeumannParams{value}; break;
        case 2: bc.params = FullyDevelopedParams{value}; break;
        case 6: {
            PulsatileParams p;
            p.value = value;
            p.amplitude = amp;
            p.frequency = freq;
            bc.params = p;
            break;
        }
        default: bc.params = NoneParams{value}; break;
    }
    return bc;
}

std::string fromHex(const std::string& h) {
    std::string s;
    if (h == "-") return s;
    for (size_t i = 0; i + 1 < h.size(); i += 2) s.push_back((char)std::stoi(h.substr(i, 2), nullptr, 16));
    return s;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s spec.txt case-dir\n", argv[0]);
        return 2;
    }
    std::ifstream in(argv[1]);
    if (!in) return 2;
    MultiBlockMesh mb;
    std::vector<BoundarySegmentGroup> groups;
    std::vector<BoundaryVertex> bverts;
    std::vector<BoundaryEdge> bedges;
    std::vector<Vec2> points;
    std::vector<Triangle> tris;
    std::vector<FVFace> faces;
    FoamCaseSetup setup;
    double tol = 1e-9, wedge = 5.0;
    std::string key;
    while (in >> key) {
        if (key == "tol") {
            in >> tol;
        } else if (key == "wedge") {
            in >> wedge;
        } else if (key == "block") {
            double z0, r0, axL, axC, rdL, rdC;
            int axN, axG, rdN, rdG, e[4];
            in >> z0 >> r0 >> axL >> axN >> axG >> axC >> rdL >> rdN >> rdG >> rdC >> e[0] >> e[1] >> e[2] >> e[3];
            MeshZone ax{axL, axN, axG == 1 ? Grading::Progression : Grading::Uniform, axC};
            MeshZone rd{rdL, rdN, rdG == 1 ? Grading::Progression : Grading::Uniform, rdC};
            Block b = makeRectBlock((int)mb.blocks.size() + 1, z0, r0, ax, rd);
            for (int k = 0; k < 4; k++) b.edgeGroup[k] = e[k];
            mb.blocks.push_back(b);
        } else if (key == "group") {
            int id, btype, nbc;
            float len;
            std::string name;
            in >> id >> btype >> len >> name >> nbc;
            BoundarySegmentGroup g;
            g.id = id;
            g.type = (BoundaryType)btype;
            g.totalLength = len;
            g.name = fromHex(name);
            for (int i = 0; i < nbc; i++) {
                std::string var;
                int type;
                double value, amp, freq;
                in >> var >> type >> value >> amp >> freq;
                g.bcs[varOf(var)] = makeBC(type, value, amp, freq);
            }
            groups.push_back(g);
        } else if (key == "kin") {
            int id, type, inhib;
            std::string var;
            double vmax, km, n, m, k2, v2;
            in >> id >> var >> type >> vmax >> km >> n >> inhib >> m >> k2 >> v2;
            for (BoundarySegmentGroup& g : groups) {
                if (g.id != id) continue;
                BoundaryCondition bc{};
                if (type == 3) {
                    MichaelisMentenParams p;
                    p.Vmax = vmax; p.Km = km; p.inhibition = inhib != 0; p.m = m; p.K2 = k2; p.V2 = v2;
                    bc.params = p;
                } else {
                    HillParams p;
                    p.Vmax = vmax; p.Km = km; p.n = n; p.inhibition = inhib != 0; p.m = m; p.K2 = k2; p.V2 = v2;
                    bc.params = p;
                }
                g.bcs[varOf(var)] = bc;
            }
        } else if (key == "vertex") {
            BoundaryVertex v;
            in >> v.pos.z >> v.pos.r;
            v.id = (int)bverts.size();
            bverts.push_back(v);
        } else if (key == "edge") {
            BoundaryEdge e;
            in >> e.v0 >> e.v1 >> e.groupID;
            e.id = (int)bedges.size();
            bedges.push_back(e);
        } else if (key == "point") {
            Vec2 p;
            in >> p.z >> p.r;
            points.push_back(p);
        } else if (key == "tri") {
            Triangle t;
            in >> t.v0 >> t.v1 >> t.v2;
            tris.push_back(t);
        } else if (key == "face") {
            FVFace f;
            in >> f.v0 >> f.v1 >> f.owner >> f.neighbor >> f.normal.z >> f.normal.r >> f.boundaryGroupID;
            faces.push_back(f);
        } else if (key == "set") {
            std::string name;
            double v;
            in >> name >> v;
            if (name == "rho") setup.rho = v;
            else if (name == "mu") setup.mu = v;
            else if (name == "D") setup.D = v;
            else if (name == "cp") setup.cp = v;
            else if (name == "k") setup.k = v;
            else if (name == "solveEnergy") setup.solveEnergy = v != 0;
            else if (name == "solveConcentration") setup.solveConcentration = v != 0;
            else if (name == "transient") setup.transient = v != 0;
            else if (name == "secondOrderTime") setup.secondOrderTime = v != 0;
            else if (name == "dt") setup.dt = v;
            else if (name == "tEnd") setup.tEnd = v;
            else if (name == "steadyIterations") setup.steadyIterations = (int)v;
            else if (name == "convection") setup.convection = (FoamConvection)(int)v;
            else if (name == "leastSquaresGradient") setup.leastSquaresGradient = v != 0;
            else if (name == "addConvection") setup.addConvection = v != 0;
            else if (name == "nonOrthCorrector") setup.nonOrthCorrector = v != 0;
            else if (name == "momentumRelaxation") setup.momentumRelaxation = v;
            else if (name == "pressureRelaxation") setup.pressureRelaxation = v;
            else if (name == "concentrationRelaxation") setup.concentrationRelaxation = v;
        }
    }
    const std::filesystem::path dir(argv[2]);
    const std::filesystem::path systemDir = dir / "system", constantDir = dir / "constant", zeroDir = dir / "0";
    for (const auto& sub : {systemDir, constantDir, zeroDir}) std::filesystem::create_directories(sub);
    std::vector<FoamField> fields;
    if (tris.empty()) {
        std::string reason;
        if (!autoDetectInterfaces(mb, reason, tol)) mb.interfaces.clear();
        mb.assignGlobalNumbering();
        const BlockMeshDict dict = blockMeshDictFromMultiblock(mb, groups, bedges, bverts);
        if (!writeBlockMeshDict(systemDir / "blockMeshDict", dict)) return 3;
        fields = initialFieldsFromDict(dict, groups, setup);
    } else {
        FVMesh fv;
        fv.cells.resize(tris.size());
        fv.faces = faces;
        const PolyMesh poly = polyMeshFromUnstructured(points, tris, fv, groups, wedge);
        if (!writePolyMesh(constantDir / "polyMesh", poly)) return 3;
        fields = initialFieldsFromPolyMesh(poly, groups, setup);
    }
    if (!writeControlDict(systemDir / "controlDict", setup) || !writeFvSchemes(systemDir / "fvSchemes", setup) ||
        !writeFvSolution(systemDir / "fvSolution", setup) ||
        !writeTransportProperties(constantDir / "transportProperties", setup) ||
        !writeTurbulenceProperties(constantDir / "turbulenceProperties"))
        return 3;
    if (!writeInitialFields(zeroDir, fields)) return 3;
    return 0;
}
