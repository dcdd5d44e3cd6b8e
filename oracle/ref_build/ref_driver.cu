// ref_driver.cu -- headless driver of the reference's OWN SIMPLE solver.
//
// TEST INFRASTRUCTURE ONLY (pins the CPU oracle). Links the reference's solver
// translation units compiled unchanged from their sources (see Makefile) and
// drives Solver::run exactly as SolverGUI does (solver_gui.cpp:898-933):
//   mesh  : the reference's multiblock packer (structs/multiblock.h) turned into
//           an FVMesh the way Mesh::createMultiBlockFVMesh does (mesh.cpp:2366-2393),
//           or (spec key `packed <file>`) packed arrays of an unstructured mesh read
//           from a file in FVMeshHostPacked order, with MeshType::Unstructured
//   groups: BoundarySegmentGroup with per-variable BoundaryCondition
//   run   : Solver::run + Solver::shutdown (joins the worker thread)
// and writes the solution fields and the residual history to a binary file.
//
// Usage: axisim_ref <spec.txt> <out.bin>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "console.h"
#include "mesh.h"
#include "residual_plot.h"
#include "solver.h"
#include "solver_struct.h"

void ResidualPlot::add(int currentIteration, const std::unordered_map<std::string, ConfigResidual>& cfg) {
    Row r{currentIteration, *cfg.at("U").resVal, *cfg.at("V").resVal, *cfg.at("Continuity").resVal,
          *cfg.at("Temperature").resVal, *cfg.at("Concentration").resVal};
    rows.push_back(r);
}

namespace {

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

BoundaryVariable varOf(const std::string& v) {
    if (v == "u") return BoundaryVariable::UVelocity;
    if (v == "v") return BoundaryVariable::VVelocity;
    if (v == "T") return BoundaryVariable::StaticTemperature;
    if (v == "C") return BoundaryVariable::Concentration;
    return BoundaryVariable::Pressure;
}

// Packed mesh file: int32 nCells, nFaces, nRefs, then the FVMeshHostPacked
// arrays in declaration order (int32 or float64 as declared).
bool readPacked(const std::string& path, FVMeshHostPacked& p) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    int32_t h[3];
    if (!f.read(reinterpret_cast<char*>(h), sizeof(h)) || h[0] <= 0 || h[1] <= 0 || h[2] < 0) return false;
    p.nCells = h[0];
    p.nFaces = h[1];
    const size_t N = (size_t)h[0], F = (size_t)h[1], S = (size_t)h[2];
    auto ints = [&](std::vector<int>& v, size_t n) {
        std::vector<int32_t> t(n);
        f.read(reinterpret_cast<char*>(t.data()), (std::streamsize)(n * sizeof(int32_t)));
        v.assign(t.begin(), t.end());
    };
    auto reals = [&](std::vector<double>& v, size_t n) {
        v.resize(n);
        f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(double)));
    };
    ints(p.faceOwner, F);
    ints(p.faceNeighbor, F);
    reals(p.faceNormalZ, F);
    reals(p.faceNormalR, F);
    reals(p.faceCenterZ, F);
    reals(p.faceCenterR, F);
    reals(p.faceArea, F);
    ints(p.faceBoundaryGroupID, F);
    reals(p.cellCenterZ, N);
    reals(p.cellCenterR, N);
    reals(p.cellArea2D, N);
    reals(p.cellVolume, N);
    ints(p.cellFaceStart, N + 1);
    ints(p.cellFaceIDs, S);
    return (bool)f && p.cellFaceStart[0] == 0 && (size_t)p.cellFaceStart[N] == S;
}

BoundarySegmentGroup* groupOf(Mesh& mesh, int id) {
    for (BoundarySegmentGroup& g : mesh.boundaryGroups)
        if (g.id == id) return &g;
    return nullptr;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s spec.txt out.bin\n", argv[0]);
        return 2;
    }
    std::ifstream in(argv[1]);
    if (!in) {
        std::fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    MultiBlockMesh mb;
    Mesh mesh;
    double tol = 1e-9;
    Config config{};
    Solver* solverPtr = nullptr;
    std::vector<std::pair<std::string, double>> settings;
    FVMeshHostPacked packed{};
    bool fromFile = false;
    std::string key;
    while (in >> key) {
        if (key == "tol") {
            in >> tol;
        } else if (key == "packed") {
            std::string path;
            in >> path;
            if (!readPacked(path, packed)) {
                std::fprintf(stderr, "cannot read packed mesh %s\n", path.c_str());
                return 2;
            }
            fromFile = true;
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
            in >> id >> btype >> len >> nbc;
            BoundarySegmentGroup g;
            g.id = id;
            g.type = (BoundaryType)btype;
            g.totalLength = len;
            for (int i = 0; i < nbc; i++) {
                std::string var;
                int type;
                double value, amp, freq;
                in >> var >> type >> value >> amp >> freq;
                g.bcs[varOf(var)] = makeBC(type, value, amp, freq);
            }
            mesh.boundaryGroups.push_back(g);
        } else if (key == "kin") {
            // kin <group> <var> <3 MM | 4 Hill> <Vmax> <Km> <n> <inhibition> <m> <K2> <V2>
            int id, type, inhib;
            std::string var;
            double vmax, km, n, m, k2, v2;
            in >> id >> var >> type >> vmax >> km >> n >> inhib >> m >> k2 >> v2;
            BoundarySegmentGroup* g = groupOf(mesh, id);
            if (!g) return 2;
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
            g->bcs[varOf(var)] = bc;
        } else if (key == "layer") {
            // layer <group> <var> <k> <d>
            int id;
            std::string var;
            double k, d;
            in >> id >> var >> k >> d;
            BoundarySegmentGroup* g = groupOf(mesh, id);
            if (!g) return 2;
            Layer l{};
            l.k = k;
            l.d = d;
            g->layers[varOf(var)].push_back(l);
        } else if (key == "set") {
            std::string name;
            double value;
            in >> name >> value;
            settings.emplace_back(name, value);
        }
    }
    if (!fromFile) {
        std::string reason;
        if (!autoDetectInterfaces(mb, reason, tol)) mb.interfaces.clear();
        mb.assignGlobalNumbering();
        toPackedMesh(mb, packed);
    }
    // FVMesh from the packed arrays, as Mesh::createMultiBlockFVMesh does
    FVMesh& fv = mesh.fvMesh;
    fv.cells.resize((size_t)packed.nCells);
    for (int c = 0; c < packed.nCells; c++) {
        FVCell& cell = fv.cells[(size_t)c];
        cell.center = Vec2{packed.cellCenterZ[(size_t)c], packed.cellCenterR[(size_t)c]};
        cell.volume = packed.cellVolume[(size_t)c];
        cell.area2D = packed.cellArea2D[(size_t)c];
        for (int k = packed.cellFaceStart[(size_t)c]; k < packed.cellFaceStart[(size_t)c + 1]; k++)
            cell.faceIDs.push_back(packed.cellFaceIDs[(size_t)k]);
    }
    fv.faces.resize((size_t)packed.nFaces);
    for (int f = 0; f < packed.nFaces; f++) {
        FVFace& face = fv.faces[(size_t)f];
        face.owner = packed.faceOwner[(size_t)f];
        face.neighbor = packed.faceNeighbor[(size_t)f];
        face.normal = Vec2{packed.faceNormalZ[(size_t)f], packed.faceNormalR[(size_t)f]};
        face.center = Vec2{packed.faceCenterZ[(size_t)f], packed.faceCenterR[(size_t)f]};
        face.area = packed.faceArea[(size_t)f];
        face.boundaryGroupID = packed.faceBoundaryGroupID[(size_t)f];
    }
    mesh.isReady = true;
    mesh.currentMeshType = fromFile ? MeshType::Unstructured : MeshType::Structured;

    Console console;
    ResidualPlot plot;
    Solver solver(config);
    solverPtr = &solver;
    solver.console = &console;
    solver.residualPlot = &plot;
    for (auto& [name, v] : settings) {
        ConfigSolver& cs = solver.configSolver;
        if (name == "convectionScheme") cs.convectionScheme = (ConvectionScheme)(int)v;
        else if (name == "gradientScheme") cs.gradientScheme = (GradientScheme)(int)v;
        else if (name == "linearType") cs.type = (LinearSolverType)(int)v;
        else if (name == "timeScheme") cs.timeScheme = (TimeScheme)(int)v;
        else if (name == "linearMaxIter") cs.linearMaxIter = (int)v;
        else if (name == "useMultigrid") cs.useMultigrid = v != 0;
        else if (name == "addConvectionTerm") cs.addConvectionTerm = v != 0;
        else if (name == "transient") cs.transient = v != 0;
        else if (name == "useNonOrthCorrector") cs.useNonOrthCorrector = v != 0;
        else if (name == "dt") cs.dt = v;
        else if (name == "tEnd") cs.tEnd = v;
        else if (name == "maxIter") solver.configSimple.maxIter = (int)v;
        else if (name == "checkConv") solver.configSimple.checkConv = (int)v;
        else if (name == "mgMaxIter") solver.configMultigrid.maxIter = (int)v;
        else if (name == "mgWeight") solver.configMultigrid.weight = v;
        else if (name == "mgLinearSweep") solver.configMultigrid.linearSweep = (int)v;
        else if (name == "mgPreSweep") solver.configMultigrid.linearPreSweep = (int)v;
        else if (name == "mgPostSweep") solver.configMultigrid.linearPostSweep = (int)v;
        else if (name == "rho") solver.f.rho = v;
        else if (name == "mu") solver.f.mu = v;
        else if (name == "cp") solver.f.cp = v;
        else if (name == "k") solver.f.k = v;
        else if (name == "D") solver.f.D = v;
        else if (name == "solveEnergy") solver.fieldOption.solveEnergy = v != 0;
        else if (name == "solveConcentration") solver.fieldOption.solveConcentration = v != 0;
        else if (name == "alphaU") solver.simple.momentumRelaxation = v;
        else if (name == "alphaP") solver.simple.pressureRelaxation = v;
        else {
            const char* names[5] = {"U", "V", "Continuity", "Temperature", "Concentration"};
            for (int i = 0; i < 5; i++) {
                ConfigResidual& r = solver.cfg.at(names[i]);
                const std::string sfx = std::to_string(i);
                if (name == "resNorm" + sfx) r.normType = (ResidualNormType)(int)v;
                if (name == "resScale" + sfx) r.scaleType = (ResidualScalingType)(int)v;
                if (name == "resEnabled" + sfx) r.enabled = v != 0;
                if (name == "resTol" + sfx) r.tol = v;
            }
        }
    }
    solver.run(mesh);
    solver.shutdown();
    (void)solverPtr;

    const int N = packed.nCells;
    int iterations = 0, converged = 0;
    for (const std::string& l : console.lines) {
        if (l.rfind("Converged:", 0) == 0) {
            converged = 1;
            std::sscanf(l.c_str(), "Converged: all residuals below tolerance at iteration %d", &iterations);
        }
    }
    if (!converged && !plot.rows.empty()) iterations = plot.rows.back().iteration + 1;
    std::FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 3;
    const int32_t hdr[4] = {N, iterations, converged, (int32_t)plot.rows.size()};
    std::fwrite(hdr, sizeof(int32_t), 4, out);
    const char* fields[] = {"Axial Velocity", "Radial Velocity", "Pressure", "Continuity", "dP/dz", "dP/dr",
                            "dU/dz", "dU/dr", "dV/dz", "dV/dr"};
    for (const char* name : fields) {
        const std::vector<double>& f = solver.solutions.at(name).field;
        std::fwrite(f.data(), sizeof(double), (size_t)N, out);
    }
    for (const ResidualPlot::Row& r : plot.rows) {
        const double row[6] = {(double)r.iteration, r.u, r.v, r.continuity, r.temperature, r.concentration};
        std::fwrite(row, sizeof(double), 6, out);
    }
    // scalar fields of the solved scalars (flags, then each field's value and gradients)
    const int32_t flags[2] = {solver.fieldOption.solveEnergy ? 1 : 0, solver.fieldOption.solveConcentration ? 1 : 0};
    std::fwrite(flags, sizeof(int32_t), 2, out);
    const char* tFields[] = {"Temperature", "dT/dz", "dT/dr"};
    const char* cFields[] = {"Concentration", "dC/dz", "dC/dr"};
    for (int sIdx = 0; sIdx < 2; sIdx++) {
        if (!flags[sIdx]) continue;
        for (const char* name : (sIdx == 0 ? tFields : cFields)) {
            const std::vector<double>& f = solver.solutions.at(name).field;
            std::fwrite(f.data(), sizeof(double), (size_t)N, out);
        }
    }
    std::fclose(out);
    std::printf("reference solver: %d cells, %d iterations, converged %d, %.3f ms\n", N, iterations, converged,
                console.completionMs);
    for (const std::string& l : console.lines)
        if (l.find("Multigrid") != std::string::npos) std::printf("%s", l.c_str());
    return 0;
}
