// axisim_solver.hpp -- C++ adapter with the reference Solver's member names over
// the C ABI in axisim_b200.h, so a manager written against AxiSim's Solver
// (solver/header/solver.h:18-185) can call the B200 library instead.
//
// Header-only. What it mirrors:
//   Solver::run(Mesh&)         -> run(): solve on a worker thread (solver.cpp:146-173)
//   Solver::requestStop()      -> requestStop()                   (solver.cpp:175-184)
//   Solver::shutdown()         -> shutdown(): join the worker      (solver.cpp:663-667)
//   Solver::canContinue(...)   -> canContinue(reason)              (solver.cpp:469-528)
//   continueSolver, fieldOption, configSolver, configSimple, configMultigrid,
//   relaxation, cfg (U, V, Continuity, Temperature, Concentration), solutions
//   (solver.h:37-133)
// The case (packed mesh + per-variable boundary fields) is handed over with
// setCase(); the reference derives both from its Mesh (mesh.cpp, memory_manger.cpp).
#pragma once

#include <atomic>
#include <map>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "axisim_b200.h"

namespace axisim_b200 {

class Solver {
public:
    explicit Solver(const axisim_fluid& fluid, int device = 0) : f(fluid) {
        if (axisim_create_on(device, &f, &h_) != AXISIM_OK) throw std::runtime_error("axisim_create_on failed");
        configSolver = axisim_config_solver{};
        configSolver.gradientScheme = 1;
        configSolver.linearMaxIter = 20;
        configSolver.useMultigrid = 1;
        configSolver.addConvectionTerm = 1;
        configSolver.dt = 0.1;
        configSolver.tEnd = 2.0;
        configSolver.saveKeyFrameIter = 2;
        configSimple = axisim_config_simple{50, 1, 1e-8, 1e-5};
        configMultigrid = axisim_config_multigrid{3, 0.6, 30, 1, 1};
        for (auto& r : cfg) r = axisim_config_residual{0, 0, 3, 1, 1e-3};
        cfg[3].enabled = cfg[4].enabled = 0;  // solver.cpp:88-100
    }
    ~Solver() {
        shutdown();
        axisim_destroy(h_);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    // Public configuration, as on the reference Solver.
    axisim_fluid f;
    axisim_config_solver configSolver;
    axisim_config_simple configSimple;
    axisim_config_multigrid configMultigrid;
    axisim_config_residual cfg[5];  // U, V, Continuity, Temperature, Concentration
    struct FieldOption {            // SolverFieldOption (solver_struct.h:9-12)
        bool solveEnergy = false;
        bool solveConcentration = false;
    } fieldOption;
    double momentumRelaxation = 0.7;
    double pressureRelaxation = 0.3;
    bool continueSolver = false;
    std::atomic<bool> solverRunning{false};
    std::map<std::string, std::vector<double>> solutions;
    axisim_result lastResult{};
    int lastStatus = AXISIM_OK;

    // Mesh + boundary fields (what Mesh / createBoundarySolverDevice provide).
    // meshType: Mesh::currentMeshType (AXISIM_MESH_*)
    int setCase(const axisim_mesh_packed& mesh, const axisim_bc_field& u, const axisim_bc_field& v,
                const axisim_bc_field& p, int meshType = AXISIM_MESH_UNSTRUCTURED) {
        int st = axisim_set_mesh(h_, &mesh);
        if (st == AXISIM_OK) st = axisim_set_mesh_type(h_, meshType);
        if (st == AXISIM_OK) st = axisim_set_bc(h_, AXISIM_VAR_U, &u);
        if (st == AXISIM_OK) st = axisim_set_bc(h_, AXISIM_VAR_V, &v);
        if (st == AXISIM_OK) st = axisim_set_bc(h_, AXISIM_VAR_P, &p);
        nCells_ = mesh.nCells;
        return st;
    }
    // Temperature / concentration boundary fields and their wall kinetics
    // (kin may be null); variable AXISIM_VAR_T or AXISIM_VAR_C.
    int setScalarBC(int variable, const axisim_bc_field& bc, const axisim_kinetics* kin = nullptr) {
        int st = axisim_set_bc(h_, variable, &bc);
        if (st == AXISIM_OK) st = axisim_set_kinetics(h_, variable, kin);
        return st;
    }

    bool canContinue(std::string* reason = nullptr) const {
        char buf[256] = {0};
        const int r = axisim_can_continue(h_, buf, sizeof(buf));
        if (reason) *reason = buf;
        return r == 1;
    }

    // Synchronous solve on the caller's thread (Solver::runSimple).
    int runSimple() {
        axisim_set_fluid(h_, &f);
        axisim_set_config(h_, &configSolver, &configSimple, &configMultigrid, cfg, momentumRelaxation,
                          pressureRelaxation);
        axisim_set_scalars(h_, fieldOption.solveEnergy ? 1 : 0, fieldOption.solveConcentration ? 1 : 0, cfg + 3);
        lastStatus = axisim_solve(h_, continueSolver ? 1 : 0, &lastResult);
        if (lastStatus == AXISIM_OK || lastStatus == AXISIM_E_STOPPED) createSolutions();
        return lastStatus;
    }

    // Asynchronous solve on a worker thread (Solver::run).
    void run() {
        shutdown();
        solverRunning = true;
        worker_ = std::thread([this] {
            runSimple();
            solverRunning = false;
        });
    }

    void requestStop() { axisim_request_stop(h_); }

    void shutdown() {
        if (worker_.joinable()) worker_.join();
    }

    const char* lastError() const { return axisim_last_error(h_); }
    axisim_handle* handle() { return h_; }

private:
    axisim_handle* h_ = nullptr;
    std::thread worker_;
    int nCells_ = 0;

    // Solver::createSolutions (solver.cpp:186-219): the same field names.
    void createSolutions() {
        const std::pair<const char*, const char*> names[] = {
            {"Axial Velocity", "u"}, {"Radial Velocity", "v"}, {"Pressure", "p"}, {"dU/dz", "gradUZ"},
            {"dU/dr", "gradUR"},     {"dV/dz", "gradVZ"},     {"dV/dr", "gradVR"}, {"dP/dz", "gradPZ"},
            {"dP/dr", "gradPR"},     {"Continuity", "continuity"}};
        for (const auto& [label, field] : names) {
            std::vector<double> v((size_t)nCells_);
            if (axisim_get_field(h_, field, v.data(), v.size()) >= 0) solutions[label] = std::move(v);
        }
        const std::pair<const char*, const char*> tNames[] = {
            {"Temperature", "T"}, {"dT/dz", "gradTZ"}, {"dT/dr", "gradTR"}};
        const std::pair<const char*, const char*> cNames[] = {
            {"Concentration", "C"}, {"dC/dz", "gradCZ"}, {"dC/dr", "gradCR"}};
        for (int q = 0; q < 2; q++) {
            if (!(q == 0 ? fieldOption.solveEnergy : fieldOption.solveConcentration)) continue;
            const auto* list = q == 0 ? tNames : cNames;
            for (int i = 0; i < 3; i++) {
                std::vector<double> v((size_t)nCells_);
                if (axisim_get_field(h_, list[i].second, v.data(), v.size()) >= 0) solutions[list[i].first] = std::move(v);
            }
        }
    }
};

}  // namespace axisim_b200
