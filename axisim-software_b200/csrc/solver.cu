// solver.cu -- host orchestration of the B200 SIMPLE solver and its C ABI.
//
// Follows Solver::runSimple (solver/source/solver.cpp:753-1396): same set-up,
// time loop, SIMPLE iteration and convergence rules. Differences by design:
//   * one SIMPLE iteration is captured ONCE as a CUDA graph (the reference
//     captures only the linear solves) and replayed in batches; convergence is
//     decided on the device, so there is no host synchronisation per iteration
//     (the reference syncs in residualAllHost, residuals.cu:79);
//   * the multigrid hierarchy operators live in the same graph;
//   * errors come back as status codes, never abort().
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/axisim_b200.h"
#include "host_prep.hpp"
#include "kernels.hpp"
#include "learned.hpp"

namespace axisim {

namespace {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) check((x), #x)

struct StatusError : std::runtime_error {
    int status;
    StatusError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

}  // namespace

// Every device allocation of a solver; freed together. Buffers are carved,
// 256-byte aligned and zero-filled, out of a few large chunks (one cudaMalloc
// and one memset per chunk instead of per buffer: set-up makes about a hundred
// buffers per mesh).
// Host arrays filled right after they are sized: no zero fill, and the copy
// runs on all host threads (first touch of the pages included).
template <class T>
struct UninitAlloc : std::allocator<T> {
    using std::allocator<T>::allocator;
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};
using HostI32 = std::vector<int32_t, UninitAlloc<int32_t>>;

template <class V, class T>
void copyParallel(V& v, const T* src, size_t n) {
    v.resize(n);
    T* d = v.data();
    axisim::parallelFor((int)std::min<size_t>(n, (size_t)INT32_MAX), [&](int b, int e) {
        std::memcpy(d + b, src + b, (size_t)(e - b) * sizeof(T));
    });
}

class Arena {
public:
    ~Arena() { release(); }
    template <class T>
    T* alloc(size_t n) {
        const size_t bytes = (std::max<size_t>(n, 1) * sizeof(T) + 255) & ~size_t(255);
        if (chunks_.empty() || used_ + bytes > cap_) {
            // chunks grow from 1 MiB to 64 MiB, so a small arena stays small
            const size_t cap = std::max(bytes, next_);
            next_ = std::min(next_ * 2, kChunkMax);
            void* p = nullptr;
            CK(cudaMalloc(&p, cap));
            chunks_.push_back(p);
            CK(cudaMemset(p, 0, cap));
            cap_ = cap;
            used_ = 0;
        }
        void* p = static_cast<char*>(chunks_.back()) + used_;
        used_ += bytes;
        return static_cast<T*>(p);
    }
    // at least `bytes` of room for the next buffers in one chunk (one
    // cudaMalloc for a set-up whose size is known instead of a chain of them)
    void reserve(size_t bytes) {
        bytes = (bytes + 255) & ~size_t(255);
        if (!chunks_.empty() && used_ + bytes <= cap_) return;
        void* p = nullptr;
        CK(cudaMalloc(&p, bytes));
        chunks_.push_back(p);
        CK(cudaMemset(p, 0, bytes));
        cap_ = bytes;
        used_ = 0;
    }
    template <class T>
    T* upload(const T* h, size_t n) {
        T* d = alloc<T>(n);
        if (n) CK(cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice));
        return d;
    }
    void release() {
        for (void* p : chunks_) cudaFree(p);
        chunks_.clear();
        cap_ = used_ = 0;
        next_ = kChunkMin;
    }

private:
    static constexpr size_t kChunkMin = size_t(1) << 20, kChunkMax = size_t(64) << 20;
    std::vector<void*> chunks_;
    size_t cap_ = 0, used_ = 0, next_ = kChunkMin;
};

struct HostBC {
    int nGroups = 0;
    std::vector<uint8_t> type, btype, puls;
    std::vector<double> value, length, amp, freq;
};

class Solver {
public:
    Solver(int device, const axisim_fluid& f) : fluid_(f), device_(device) {
        CK(cudaSetDevice(device_));
        // A blocking stream: set-up work (cudaMalloc'd buffers zeroed by
        // cudaMemset, uploads by cudaMemcpy from pageable memory, which may
        // return before the DMA lands) runs on the legacy default stream, and
        // the solver's kernels must be ordered after it.
        CK(cudaStreamCreate(&stream_));
        CK(cudaHostAlloc(&hostStop_, sizeof(int), cudaHostAllocMapped));
        *hostStop_ = 0;
        CK(cudaHostGetDevicePointer((void**)&hostStopDev_, (void*)hostStop_, 0));
        CK(cudaEventCreate(&ev0_));
        CK(cudaEventCreate(&ev1_));
        defaults();
    }
    ~Solver() {
        destroyGraph();
        if (stream_) cudaStreamSynchronize(stream_);
        meshArena_.release();
        segArena_.release();
        mgArena_.release();
        bcArena_.release();
        if (hostStop_) cudaFreeHost((void*)hostStop_);
        if (hostBCStage_) cudaFreeHost(hostBCStage_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (stream_) cudaStreamDestroy(stream_);
        if (loopStream_) cudaStreamDestroy(loopStream_);
        if (galStream_) cudaStreamDestroy(galStream_);
        if (evFork_) cudaEventDestroy(evFork_);
        for (cudaEvent_t e : evGal_) cudaEventDestroy(e);
    }

    // Every entry point makes the handle's device current on the calling thread.
    void activate() const { CK(cudaSetDevice(device_)); }

    std::string lastError;
    axisim_log_fn logFn = nullptr;
    axisim_residual_fn resFn = nullptr;
    void* cbCtx = nullptr;

    void defaults() {
        std::memset(&cs_, 0, sizeof(cs_));
        cs_.convectionScheme = 0;
        cs_.gradientScheme = 1;
        cs_.type = 0;
        cs_.linearMaxIter = 20;
        cs_.useMultigrid = 1;
        cs_.addConvectionTerm = 1;
        cs_.dt = 0.1;
        cs_.tEnd = 2.0;
        cs_.saveKeyFrameIter = 2;
        csim_ = axisim_config_simple{50, 1, 1e-8, 1e-5};
        cmg_ = axisim_config_multigrid{3, 0.6, 30, 1, 1};
        for (int i = 0; i < 3; i++) cres_[i] = axisim_config_residual{0, 0, 3, 1, 1e-3};
        for (int i = 0; i < 2; i++) sres_[i] = axisim_config_residual{0, 0, 3, 0, 1e-3};
        alphaU_ = 0.7;
        alphaP_ = 0.3;
    }

    void setFluid(const axisim_fluid& f) {
        fluid_ = f;
        destroyGraph();
    }

    void setPrecision(int mode) {
        if (mode != AXISIM_PREC_FP64 && mode != AXISIM_PREC_MIXED) throw StatusError(AXISIM_E_ARG, "unknown precision mode");
        precision_ = mode;
        destroyGraph();
    }

    void setPressureSolver(int mode, double relTol, double prolongScale) {
        if (mode != AXISIM_PSOLVE_VCYCLES && mode != AXISIM_PSOLVE_FCG)
            throw StatusError(AXISIM_E_ARG, "unknown pressure solver mode");
        if (!(relTol >= 0.0 && relTol < 1.0)) throw StatusError(AXISIM_E_ARG, "relTol must be in [0, 1)");
        if (!(prolongScale > 0.0 && prolongScale <= 4.0)) throw StatusError(AXISIM_E_ARG, "prolongScale must be in (0, 4]");
        psolve_ = mode;
        psolveTol_ = relTol;
        prolongScale_ = prolongScale;
        destroyGraph();
    }

    void pressureStats(int64_t* solves, int64_t* iterations) {
        Ctl h;
        CK(cudaMemcpy(&h, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost));
        if (solves) *solves = h.ppSolves;
        if (iterations) *iterations = h.ppIterations;
    }

    void resetLearned() {
        net_.reset();
        learnedMode_ = 0;
        adamT_ = 0;
        sampleArena_.release();
        harvestEvery_ = 0;
        sampleCap_ = 0;
        samples_ = nullptr;
        sampleCount_ = nullptr;
        sampleRelres_ = nullptr;
        harvestCounter_ = nullptr;
    }

    // ---------------- learned preconditioner ----------------
    void learnedHarvest(int every, int capacity) {
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
        if (every < 0 || capacity < 0) throw StatusError(AXISIM_E_ARG, "every and capacity must be >= 0");
        if (capacity > 0 && capacity != sampleCap_) {
            sampleArena_.release();
            samples_ = sampleArena_.alloc<float>((size_t)capacity * sampleStride());
            sampleCount_ = sampleArena_.alloc<int>(1);
            sampleRelres_ = sampleArena_.alloc<float>((size_t)capacity);
            harvestCounter_ = sampleArena_.alloc<unsigned int>(1);
            sampleCap_ = capacity;
        }
        harvestEvery_ = samples_ ? every : 0;
        destroyGraph();
    }

    int learnedSampleCount() {
        if (!sampleCount_) return 0;
        int c = 0;
        CK(cudaMemcpy(&c, sampleCount_, sizeof(int), cudaMemcpyDeviceToHost));
        return c;
    }

    size_t sampleStride() const { return (size_t)(4 + W_) * (size_t)N_; }

    // A_F in the mesh's CSR slot order (cellFaceStart) <-> ELL [W][N]
    std::vector<float> csrToEll(const float* csr) const {
        std::vector<float> ell((size_t)W_ * N_, 0.f);
        for (int n = 0; n < N_; n++)
            for (int k = hCfs_[(size_t)n], j = 0; k < hCfs_[(size_t)n + 1]; k++, j++)
                ell[(size_t)j * N_ + n] = csr[(size_t)k];
        return ell;
    }

    void learnedAddSample(const float* b, const float* t, const float* ac, const float* d, const float* afCsr) {
        if (!samples_) throw StatusError(AXISIM_E_STATE, "no sample store: call axisim_learned_harvest with a capacity");
        if (!b || !t || !ac || !d || !afCsr) throw StatusError(AXISIM_E_ARG, "sample array is null");
        const int c = learnedSampleCount();
        if (c >= sampleCap_) throw StatusError(AXISIM_E_ARG, "sample store is full");
        float* base = samples_ + (size_t)c * sampleStride();
        const float* src[4] = {b, t, ac, d};
        for (int k = 0; k < 4; k++)
            CK(cudaMemcpy(base + (size_t)k * N_, src[k], (size_t)N_ * sizeof(float), cudaMemcpyHostToDevice));
        const std::vector<float> ell = csrToEll(afCsr);
        CK(cudaMemcpy(base + 4 * (size_t)N_, ell.data(), ell.size() * sizeof(float), cudaMemcpyHostToDevice));
        const float rr = -1.f;
        const int c1 = c + 1;
        CK(cudaMemcpy(sampleRelres_ + c, &rr, sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(sampleCount_, &c1, sizeof(int), cudaMemcpyHostToDevice));
    }

    void learnedGetSample(int idx, float* b, float* t, float* ac, float* d, float* afCsr, float* relres) {
        if (idx < 0 || idx >= learnedSampleCount()) throw StatusError(AXISIM_E_ARG, "sample index out of range");
        const float* base = samples_ + (size_t)idx * sampleStride();
        float* dst[4] = {b, t, ac, d};
        for (int k = 0; k < 4; k++)
            if (dst[k])
                CK(cudaMemcpy(dst[k], base + (size_t)k * N_, (size_t)N_ * sizeof(float), cudaMemcpyDeviceToHost));
        if (afCsr) {
            std::vector<float> ell((size_t)W_ * N_);
            CK(cudaMemcpy(ell.data(), base + 4 * (size_t)N_, ell.size() * sizeof(float), cudaMemcpyDeviceToHost));
            for (int n = 0; n < N_; n++)
                for (int k = hCfs_[(size_t)n], j = 0; k < hCfs_[(size_t)n + 1]; k++, j++)
                    afCsr[(size_t)k] = ell[(size_t)j * N_ + n];
        }
        if (relres) CK(cudaMemcpy(relres, sampleRelres_ + idx, sizeof(float), cudaMemcpyDeviceToHost));
    }

    size_t learnedInit(int precision, uint64_t seed) {
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
        if (precision < 0 || precision > 2) throw StatusError(AXISIM_E_ARG, "unknown network precision");
        ensureHierarchy();
        if (!termRanges_.empty())
            throw StatusError(AXISIM_E_CONFIG, "the learned preconditioner needs one hierarchy over the whole mesh "
                                               "(not a batch of per-case hierarchies)");
        net_.init(hier_, mesh_.snb, W_, precision, seed, stream_);
        adamT_ = 0;
        destroyGraph();
        return net_.numParams();
    }

    void requireNet() const {
        if (!net_.ready()) throw StatusError(AXISIM_E_STATE, "network not initialised (axisim_learned_init)");
    }

    void learnedParams(float* host, int64_t n, int set) {
        requireNet();
        if (!host || n != (int64_t)net_.numParams()) throw StatusError(AXISIM_E_ARG, "parameter count mismatch");
        if (set) {
            CK(cudaMemcpy(net_.params(), host, (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
            net_.syncLowPrecision(stream_);
            CK(cudaStreamSynchronize(stream_));
        } else {
            CK(cudaMemcpy(host, net_.params(), (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
        }
    }

    LearnedNet::Sample sample(int idx) const {
        const float* base = samples_ + (size_t)idx * sampleStride();
        const size_t N = (size_t)N_;
        return LearnedNet::Sample{base, base + N, base + 2 * N, base + 3 * N, base + 4 * N};
    }

    float learnedGrad(int idx, float* grad, int64_t n) {
        requireNet();
        if (idx < 0 || idx >= learnedSampleCount()) throw StatusError(AXISIM_E_ARG, "sample index out of range");
        if (grad && n != (int64_t)net_.numParams()) throw StatusError(AXISIM_E_ARG, "parameter count mismatch");
        Arena tmp;
        float* loss = tmp.alloc<float>(1);
        net_.lossAndGrad(sample(idx), loss, stream_);
        CK(cudaStreamSynchronize(stream_));
        float h = 0.f;
        CK(cudaMemcpy(&h, loss, sizeof(float), cudaMemcpyDeviceToHost));
        if (grad) CK(cudaMemcpy(grad, net_.grad(), (size_t)n * sizeof(float), cudaMemcpyDeviceToHost));
        return h;
    }

    // Adam on samples [first, first + count) drawn uniformly (with replacement)
    // by a seeded linear congruential generator.
    void learnedTrain(int steps, float lr, uint64_t seed, int first, int count, float* lossHost) {
        requireNet();
        const int have = learnedSampleCount();
        if (count <= 0) count = have - first;
        if (first < 0 || count <= 0 || first + count > have)
            throw StatusError(AXISIM_E_ARG, "sample range outside the store");
        if (steps <= 0 || !(lr > 0.f)) throw StatusError(AXISIM_E_ARG, "steps and lr must be positive");
        Arena tmp;
        float* loss = tmp.alloc<float>((size_t)steps);
        uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
        for (int i = 0; i < steps; i++) {
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            const int idx = first + (int)((st >> 33) % (uint64_t)count);
            net_.trainStep(sample(idx), lr, ++adamT_, loss + i, stream_);
        }
        CK(cudaStreamSynchronize(stream_));
        if (lossHost) CK(cudaMemcpy(lossHost, loss, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost));
    }

    void learnedPredict(const float* r, const float* ac, const float* d, float* out) {
        requireNet();
        if (!r || !ac || !d || !out) throw StatusError(AXISIM_E_ARG, "array is null");
        Arena tmp;
        float* dev = tmp.alloc<float>(4 * (size_t)N_);
        const float* src[3] = {r, ac, d};
        for (int k = 0; k < 3; k++)
            CK(cudaMemcpy(dev + (size_t)k * N_, src[k], (size_t)N_ * sizeof(float), cudaMemcpyHostToDevice));
        net_.predict(dev, dev + N_, dev + 2 * (size_t)N_, dev + 3 * (size_t)N_, stream_);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(out, dev + 3 * (size_t)N_, (size_t)N_ * sizeof(float), cudaMemcpyDeviceToHost));
    }

    void learnedEnable(int mode) {
        if (mode != AXISIM_LEARNED_OFF && mode != AXISIM_LEARNED_FIRST_STEP && mode != AXISIM_LEARNED_ALWAYS)
            throw StatusError(AXISIM_E_ARG, "unknown learned mode");
        if (mode != AXISIM_LEARNED_OFF) requireNet();
        learnedMode_ = mode;
        destroyGraph();
    }

    void learnedStats(int64_t* applied, int64_t* fallbacks, double* scoreNet, double* scoreV) {
        NetStats h{};
        if (netStats_) CK(cudaMemcpy(&h, netStats_, sizeof(NetStats), cudaMemcpyDeviceToHost));
        if (applied) *applied = h.applied;
        if (fallbacks) *fallbacks = h.fallbacks;
        if (scoreNet) *scoreNet = h.logRhoNet;
        if (scoreV) *scoreV = h.logRhoV;
    }

    void ensureNetStats() {
        if (netStats_) return;
        netStats_ = netArena_.alloc<NetStats>(1);
        nnY_ = netArena_.alloc<float>((size_t)N_);
        nnAy_ = netArena_.alloc<double>((size_t)N_);
    }

    // ---------------- mesh ----------------
    void setMesh(const axisim_mesh_packed& pm) {
        std::unique_ptr<PhaseTimer> ph(new PhaseTimer(*this, "mesh_validate"));
        const int N = pm.nCells, F = pm.nFaces;
        if (N <= 0 || F <= 0) throw StatusError(AXISIM_E_MESH, "mesh needs cells and faces");
        const void* req[] = {pm.faceOwner, pm.faceNeighbor, pm.faceNormalZ, pm.faceNormalR, pm.faceCenterZ,
                             pm.faceCenterR, pm.faceArea, pm.faceBoundaryGroupID, pm.cellCenterZ, pm.cellCenterR,
                             pm.cellVolume, pm.cellFaceStart, pm.cellFaceIDs};
        for (const void* p : req)
            if (!p) throw StatusError(AXISIM_E_ARG, "mesh array is null");
        if (pm.cellFaceStart[0] != 0) throw StatusError(AXISIM_E_MESH, "cellFaceStart[0] must be 0");
        // range checks in parallel; each range reports its largest face count
        // and a violation flag (1 order, 2 slot face id, 3 owner, 4 neighbour)
        std::atomic<int> W{0}, bad{0};
        auto note = [&](int code) {
            int z = 0;
            bad.compare_exchange_strong(z, code);
        };
        parallelFor(N, [&](int c0, int c1) {
            int w = 0;
            for (int c = c0; c < c1; c++) {
                const int d = pm.cellFaceStart[c + 1] - pm.cellFaceStart[c];
                if (d < 0) note(1);
                w = std::max(w, d);
            }
            int cur = W.load();
            while (w > cur && !W.compare_exchange_weak(cur, w)) {
            }
        });
        if (bad == 1) throw StatusError(AXISIM_E_MESH, "cellFaceStart is not monotone");
        if (W > 32) throw StatusError(AXISIM_E_MESH, "a cell has more than 32 faces");
        const int S = pm.cellFaceStart[N];
        parallelFor(S, [&](int k0, int k1) {
            for (int k = k0; k < k1; k++)
                if (pm.cellFaceIDs[k] < 0 || pm.cellFaceIDs[k] >= F) note(2);
        });
        if (bad == 2) throw StatusError(AXISIM_E_MESH, "cellFaceIDs out of range");
        parallelFor(F, [&](int f0, int f1) {
            for (int f = f0; f < f1; f++) {
                if (pm.faceOwner[f] < 0 || pm.faceOwner[f] >= N) note(3);
                if (pm.faceNeighbor[f] >= N) note(4);
            }
        });
        if (bad == 3) throw StatusError(AXISIM_E_MESH, "faceOwner out of range");
        if (bad == 4) throw StatusError(AXISIM_E_MESH, "faceNeighbor out of range");
        destroyGraph();
        batchArena_.release();
        batch_ = BatchDev{};
        mixArena_.release();
        levels32_.clear();
        AF32m_ = nullptr;
        fcgR_ = nullptr;
        netArena_.release();
        netStats_ = nullptr;
        nnY_ = nullptr;
        nnAy_ = nullptr;
        resetLearned();
        mgArena_.release();
        levels_.clear();
        hier_.clear();
        haveHierarchy_ = false;
        colorN_ = 0;
        releaseScalarBuffers();
        meshArena_.release();
        segArena_.release();
        meshType_ = AXISIM_MESH_UNSTRUCTURED;
        N_ = N;
        F_ = F;
        S_ = S;
        W_ = W;
        copyParallel(hCfs_, pm.cellFaceStart, (size_t)N + 1);
        copyParallel(hCfi_, pm.cellFaceIDs, (size_t)S);
        copyParallel(hOwner_, pm.faceOwner, (size_t)F);
        copyParallel(hNeighbor_, pm.faceNeighbor, (size_t)F);
        dropSweepTiles();
        ph.reset(new PhaseTimer(*this, "mesh_upload"));
        Arena& A = meshArena_;
        // the mesh, its precomputed geometry and the fields below, in one
        // chunk: 13 face arrays of 8 bytes and 3 of 4, 7 cell arrays of 8 and
        // ~35 field and system arrays of 8, 4 [W][N] blocks of 8, the slot ids
        A.reserve((size_t)F * (13 * 8 + 3 * 4 + 8) + (size_t)N * (7 * 8 + 4 + 35 * 8) +
                  (size_t)W * N * (4 * 8 + 2 * 4) + (size_t)S * 4 + (size_t)64 * 256);
        MeshDev& m = mesh_;
        m.N = N;
        m.F = F;
        m.W = W;
        m.owner = A.upload(pm.faceOwner, F);
        m.neighbor = A.upload(pm.faceNeighbor, F);
        m.group = A.upload(pm.faceBoundaryGroupID, F);
        m.nZ = A.upload(pm.faceNormalZ, F);
        m.nR = A.upload(pm.faceNormalR, F);
        m.fcZ = A.upload(pm.faceCenterZ, F);
        m.fcR = A.upload(pm.faceCenterR, F);
        m.area = A.upload(pm.faceArea, F);
        m.ccZ = A.upload(pm.cellCenterZ, N);
        m.ccR = A.upload(pm.cellCenterR, N);
        m.vol = A.upload(pm.cellVolume, N);
        m.invDPN = A.alloc<double>(F);
        m.wP = A.alloc<double>(F);
        m.dPB = A.alloc<double>(F);
        m.length2D = A.alloc<double>(F);
        m.lsqWZ = A.alloc<double>(F);
        m.lsqWR = A.alloc<double>(F);
        m.invA2D = A.alloc<double>(N);
        m.lsqIZZ = A.alloc<double>(N);
        m.lsqIZR = A.alloc<double>(N);
        m.lsqIRR = A.alloc<double>(N);
        int32_t* dCfs = A.upload(pm.cellFaceStart, (size_t)N + 1);
        int32_t* dCfi = A.upload(pm.cellFaceIDs, (size_t)S);
        int32_t* sface = A.alloc<int32_t>((size_t)W * N);
        int32_t* snb = A.alloc<int32_t>((size_t)W * N);
        m.sface = sface;
        m.snb = snb;
        double* tz = A.alloc<double>(F);
        double* tr = A.alloc<double>(F);
        ph.reset(new PhaseTimer(*this, "mesh_precompute_ell"));
        launchPrecompute(m, dCfs, dCfi, tz, tr, stream_);
        launchBuildEll(N, W, dCfs, dCfi, m.owner, m.neighbor, sface, snb, stream_);
        segCounts_[0] = segCounts_[1] = (N + 31) / 32;
        nSeg_ = (N + 31) / 32;
        m.sseg = nullptr;
        m.ssegF = nullptr;
        m.ssegM = nullptr;
        if (W == 3 || W == 4) {
            Arena& B = segArena_;
            B.reserve((size_t)nSeg_ * (16 + 16 + 4) + 3 * 256);
            int4* seg = B.alloc<int4>((size_t)nSeg_);
            int4* segF = B.alloc<int4>((size_t)nSeg_);
            int* segM = B.alloc<int>((size_t)nSeg_ + 2);
            int* nIrr = segM + nSeg_;  // [0] without slot offsets, [1] without affine faces
            CK(cudaMemsetAsync(nIrr, 0, 2 * sizeof(int), stream_));
            launchBuildSegments(m, seg, segF, segM, nIrr, stream_);
            CK(cudaMemcpyAsync(segCounts_, nIrr, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream_));
            m.sseg = seg;
            m.ssegF = segF;
            m.ssegM = segM;
        }
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(stream_));
        segIrregular_ = m.sseg ? segCounts_[0] : nSeg_;
        if (m.sseg && 2 * segIrregular_ > nSeg_) {
            // mostly irregular numbering (unstructured cells): the segment test
            // would only put a load ahead of every slot neighbour read
            m.sseg = nullptr;
            m.ssegF = nullptr;
            m.ssegM = nullptr;
            segArena_.release();
        }
        ph.reset(new PhaseTimer(*this, "fields_alloc"));
        // fields and coefficient systems (allocateSimple / allocateCoefficients)
        const size_t WN = (size_t)W * N;
        u_ = A.alloc<double>(N); v_ = A.alloc<double>(N); p_ = A.alloc<double>(N); pp_ = A.alloc<double>(N);
        uT_ = A.alloc<double>(N); vT_ = A.alloc<double>(N); ppT_ = A.alloc<double>(N);
        DU_ = A.alloc<double>(N); DV_ = A.alloc<double>(N);
        gPZ_ = A.alloc<double>(N); gPR_ = A.alloc<double>(N);
        gUZ_ = A.alloc<double>(N); gUR_ = A.alloc<double>(N); gVZ_ = A.alloc<double>(N); gVR_ = A.alloc<double>(N);
        uOld_ = A.alloc<double>(N); vOld_ = A.alloc<double>(N); uOld2_ = A.alloc<double>(N); vOld2_ = A.alloc<double>(N);
        mDot_ = A.alloc<double>(F);
        AFm_ = A.alloc<double>(WN);
        ACu_ = A.alloc<double>(N); ACv_ = A.alloc<double>(N); bu_ = A.alloc<double>(N); bv_ = A.alloc<double>(N);
        iu_ = A.alloc<double>(N); iv_ = A.alloc<double>(N);
        AFpp_ = A.alloc<double>(WN); ACpp_ = A.alloc<double>(N); bpp_ = A.alloc<double>(N); ipp_ = A.alloc<double>(N);
        resU_ = A.alloc<double>(N); resV_ = A.alloc<double>(N); resC_ = A.alloc<double>(N);
        scU_ = A.alloc<double>(N); scV_ = A.alloc<double>(N);
        partial_ = A.alloc<double>((size_t)((N + 255) / 256) * 5 + 5);
        ctl_ = A.alloc<Ctl>(1);
        CK(cudaStreamSynchronize(stream_));
        haveMesh_ = true;
        isReady_ = false;
    }

    // Cases [caseStart[c], caseStart[c+1]) of the packed mesh are independent
    // problems monitored and converged separately (nCases = 0 clears).
    void setBatch(int nCases, const int32_t* caseStart) {
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "set the mesh before the batch layout");
        if (nCases < 0 || (nCases > 0 && !caseStart)) throw StatusError(AXISIM_E_ARG, "bad batch layout");
        if (nCases > 0) {
            if (caseStart[0] != 0 || caseStart[nCases] != N_) throw StatusError(AXISIM_E_ARG, "case ranges must cover the mesh");
            for (int c = 0; c < nCases; c++)
                if (caseStart[c + 1] <= caseStart[c]) throw StatusError(AXISIM_E_ARG, "empty or decreasing case range");
            // no face may connect two cases
            for (int f = 0; f < F_; f++) {
                const int nb = hNeighbor_[(size_t)f];
                if (nb < 0) continue;
                const int co = (int)(std::upper_bound(caseStart, caseStart + nCases + 1, hOwner_[(size_t)f]) - caseStart);
                const int cn = (int)(std::upper_bound(caseStart, caseStart + nCases + 1, nb) - caseStart);
                if (co != cn) throw StatusError(AXISIM_E_MESH, "a face connects two cases");
            }
        }
        destroyGraph();
        batchArena_.release();
        batch_ = BatchDev{};
        dropSweepTiles();  // the tile curve runs case by case
        // the multigrid hierarchy depends on the case layout (one per case)
        if (haveHierarchy_ && (nCases > 0 || !termRanges_.empty())) {
            mixArena_.release();
            levels32_.clear();
            AF32m_ = nullptr;
            fcgR_ = nullptr;
            netArena_.release();
            netStats_ = nullptr;
            nnY_ = nullptr;
            nnAy_ = nullptr;
            resetLearned();
            mgArena_.release();
            levels_.clear();
            hier_.clear();
            termRanges_.clear();
            haveHierarchy_ = false;
        }
        hCaseStart_.clear();
        if (nCases == 0) return;
        hCaseStart_.assign(caseStart, caseStart + nCases + 1);
        batch_.nCases = nCases;
        batch_.cellStart = batchArena_.upload(caseStart, (size_t)nCases + 1);
        batch_.raw = batchArena_.alloc<double>((size_t)nCases * 5);
        batch_.resVal = batchArena_.alloc<double>((size_t)nCases * 3);
        batch_.scaleVal = batchArena_.alloc<double>((size_t)nCases * 3);
        batch_.convergedAt = batchArena_.alloc<int32_t>((size_t)nCases);
        std::vector<int32_t> neg((size_t)nCases, -1);
        CK(cudaMemcpy(batch_.convergedAt, neg.data(), neg.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }

    int batchStatus(int32_t* convergedAt, double* residuals, int n) const {
        if (batch_.nCases == 0) throw StatusError(AXISIM_E_STATE, "no batch layout set");
        if (n < batch_.nCases) throw StatusError(AXISIM_E_ARG, "buffer too small");
        CK(cudaStreamSynchronize(stream_));
        if (convergedAt)
            CK(cudaMemcpy(convergedAt, batch_.convergedAt, sizeof(int32_t) * (size_t)batch_.nCases, cudaMemcpyDeviceToHost));
        if (residuals)
            CK(cudaMemcpy(residuals, batch_.resVal, sizeof(double) * 3 * (size_t)batch_.nCases, cudaMemcpyDeviceToHost));
        return batch_.nCases;
    }

    void setBC(int var, const axisim_bc_field& b) {
        if (var < 0 || var > 4) throw StatusError(AXISIM_E_ARG, "variable must be 0 (u), 1 (v), 2 (p), 3 (T) or 4 (C)");
        if (b.nGroups < 0 || (b.nGroups > 0 && (!b.typeByGroup || !b.valueByGroup)))
            throw StatusError(AXISIM_E_ARG, "bc arrays are null");
        HostBC h;
        const int G = b.nGroups;
        h.nGroups = G;
        h.type.assign(b.typeByGroup, b.typeByGroup + G);
        h.btype = b.boundaryTypeByGroup ? std::vector<uint8_t>(b.boundaryTypeByGroup, b.boundaryTypeByGroup + G)
                                        : std::vector<uint8_t>((size_t)G, 0);
        h.value.assign(b.valueByGroup, b.valueByGroup + G);
        h.length = b.lengthByGroup ? std::vector<double>(b.lengthByGroup, b.lengthByGroup + G)
                                   : std::vector<double>((size_t)G, 0.0);
        h.puls.assign((size_t)G, 0);
        h.amp.assign((size_t)G, 0.0);
        h.freq.assign((size_t)G, 0.0);
        for (int g = 0; g < G; g++) {
            const uint8_t t = h.type[(size_t)g];
            if (var < 3 && (t == AXISIM_BC_MICHAELIS_MENTEN || t == AXISIM_BC_HILL))
                throw StatusError(AXISIM_E_CONFIG, "Michaelis-Menten and Hill conditions apply to T and C only");
            if (t == AXISIM_BC_PULSATILE) h.type[(size_t)g] = AXISIM_BC_DIRICHLET;
            // only u and v follow the pulsatile law in time (solver.cpp:1038-1055)
            if (var < 2 && b.pulsatileByGroup && b.pulsatileByGroup[g]) {
                h.puls[(size_t)g] = 1;
                h.amp[(size_t)g] = b.amplitudeByGroup ? b.amplitudeByGroup[g] : 0.0;
                h.freq[(size_t)g] = b.frequencyByGroup ? b.frequencyByGroup[g] : 0.0;
            }
        }
        if (var < 3) {
            hbc_[var] = h;
            haveBC_[var] = true;
        } else {
            hbcS_[var - 3] = h;
            haveBCS_[var - 3] = true;
        }
        bcDirty_ = true;
    }

    void setMeshType(int t) {
        if (t != AXISIM_MESH_STRUCTURED && t != AXISIM_MESH_UNSTRUCTURED)
            throw StatusError(AXISIM_E_ARG, "mesh type must be 0 (structured) or 1 (unstructured)");
        meshType_ = t;
    }

    // Wall kinetics of T (var 3) or C (var 4); null restores the defaults.
    void setKinetics(int var, const axisim_kinetics* k) {
        if (var != 3 && var != 4) throw StatusError(AXISIM_E_ARG, "kinetics apply to variable 3 (T) or 4 (C)");
        std::vector<double>& kin = hkin_[var - 3];
        kin.clear();
        if (k) {
            if (k->nGroups < 0) throw StatusError(AXISIM_E_ARG, "kinetics nGroups < 0");
            const int G = k->nGroups;
            const double* src[7] = {k->vmaxByGroup, k->kmByGroup, k->nByGroup, k->mByGroup,
                                    k->k2ByGroup, k->v2ByGroup, k->RtotByGroup};
            const double dflt[7] = {0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0};
            kin.assign((size_t)7 * G, 0.0);
            for (int j = 0; j < 7; j++)
                for (int g = 0; g < G; g++) kin[(size_t)j * G + g] = src[j] ? src[j][g] : dflt[j];
            hkinG_[var - 3] = G;
        } else {
            hkinG_[var - 3] = 0;
        }
        bcDirty_ = true;
    }

    // SolverFieldOption and the Temperature / Concentration residual entries.
    void setScalars(int energy, int concentration, const axisim_config_residual* r2) {
        const int next[2] = {energy ? 1 : 0, concentration ? 1 : 0};
        bool baked = next[0] != solveS_[0] || next[1] != solveS_[1];
        if (r2)
            for (int q = 0; q < 2; q++) {
                baked |= r2[q].enabled != sres_[q].enabled;
                sres_[q] = r2[q];
            }
        solveS_[0] = next[0];
        solveS_[1] = next[1];
        if (baked) {
            wallFacesReady_ = false;
            destroyGraph();
        }
    }

    void scalarResiduals(double* out) const {
        out[0] = lastResS_[0];
        out[1] = lastResS_[1];
    }

    void setConfig(const axisim_config_solver* s, const axisim_config_simple* sim, const axisim_config_multigrid* mg,
                   const axisim_config_residual* r3, double aU, double aP) {
        // maxIter, checkConv and the residual settings are read from the device
        // control block at run time; only settings baked into the captured
        // iteration graph force a recapture.
        bool baked = false;
        if (s) {
            baked |= std::memcmp(&cs_, s, sizeof(cs_)) != 0;
            cs_ = *s;
        }
        if (sim) csim_ = *sim;
        if (mg) {
            baked |= std::memcmp(&cmg_, mg, sizeof(cmg_)) != 0;
            cmg_ = *mg;
        }
        if (r3)
            for (int i = 0; i < 3; i++) cres_[i] = r3[i];
        baked |= alphaU_ != aU || alphaP_ != aP;
        alphaU_ = aU;
        alphaP_ = aP;
        if (baked) destroyGraph();
    }

    bool canContinue(std::string* reason) const {
        auto why = [&](const char* t) {
            if (reason) *reason = t;
            return false;
        };
        if (running_) return why("Solver is already running.");
        if (!isReady_) return why("Run the solver once before continuing.");
        if (timedOut_) return why("The last run ended when a multigrid barrier gave up waiting.");
        if (!haveMesh_) return why("Generate a valid mesh first.");
        // solver.cpp:485-493
        if (solveS_[0] != ranS_[0]) return why("Energy field selection changed.");
        if (solveS_[1] != ranS_[1]) return why("Concentration field selection changed.");
        return true;
    }

    void requestStop() {
        if (running_) __atomic_store_n(hostStop_, 1, __ATOMIC_SEQ_CST);
    }

    int solve(int continueRun, axisim_result* res);

    int64_t getField(const std::string& name, double* out, size_t n) const;
    int64_t setField(const std::string& name, const double* in, size_t n);

    int mgLevels(int32_t* cells, int maxL) {
        ensureHierarchy();
        for (int l = 0; l < (int)hier_.size() && l < maxL; l++) cells[l] = hier_[(size_t)l].nCells;
        return (int)hier_.size();
    }
    int64_t mgLevelMaps(int level, int32_t* c2c, int32_t* f2c, int32_t* cfs, int32_t* cfn) {
        ensureHierarchy();
        if (level < 0 || level + 1 >= (int)hier_.size()) throw StatusError(AXISIM_E_ARG, "level out of range");
        const GridLevel& f = hier_[(size_t)level];
        const GridLevel& c = hier_[(size_t)level + 1];
        if (c2c) std::copy(f.cellToCoarse.begin(), f.cellToCoarse.end(), c2c);
        if (f2c) std::copy(f.fineSlotToCoarseSlot.begin(), f.fineSlotToCoarseSlot.end(), f2c);
        if (cfs) std::copy(c.faceStart.begin(), c.faceStart.end(), cfs);
        if (cfn) std::copy(c.faceNeighbor.begin(), c.faceNeighbor.end(), cfn);
        return c.nFaceRefs();
    }
    int coloring(int32_t* out, size_t n) {
        ensureColoring();
        if (n < (size_t)N_) throw StatusError(AXISIM_E_ARG, "buffer too small");
        std::copy(hColor_.begin(), hColor_.end(), out);
        return colorN_;
    }

private:
    axisim_fluid fluid_;
    int device_ = 0;
    axisim_config_solver cs_;
    axisim_config_simple csim_;
    axisim_config_multigrid cmg_;
    axisim_config_residual cres_[3];
    double alphaU_ = 0.7, alphaP_ = 0.3;
    int meshType_ = AXISIM_MESH_UNSTRUCTURED;  // Mesh::currentMeshType
    // transported scalars, index 0 temperature, 1 concentration: which are
    // solved (and were in the last run), their residual entries, boundary
    // fields, user kinetics [7][G] (Vmax Km n m K2 V2 Rtot), device buffers
    int solveS_[2] = {0, 0};
    int ranS_[2] = {0, 0};
    axisim_config_residual sres_[2];
    double lastResS_[2] = {0.0, 0.0};
    HostBC hbcS_[2];
    bool haveBCS_[2] = {false, false};
    std::vector<double> hkin_[2];
    int hkinG_[2] = {0, 0};
    BCDev bcS_[2];
    // lvl[0], lvl[1] are the reference's simple.tempOld / tempOld2 buffers as
    // first allocated; `swapped` says the BDF2 shift has exchanged the two
    // names an odd number of times (simple.tempOld is then lvl[1]).
    struct ScalarBuf {
        double *phi = nullptr, *tmp = nullptr, *lvl[2] = {nullptr, nullptr}, *gZ = nullptr, *gR = nullptr;
        double *AF = nullptr, *AC = nullptr, *b = nullptr, *inv = nullptr, *res = nullptr, *scale = nullptr;
        double* wall = nullptr;  // per face: c_w of this scalar's reactive faces
        int swapped = 0;
        double* old() const { return lvl[swapped]; }       // simple.tempOld
        double* old2() const { return lvl[1 - swapped]; }  // simple.tempOld2
    } sb_[2];
    // the `swapped` state at the start of the run the graph was captured for:
    // the scalar step reads the levels through the names as they stood then
    int graphSwapS_[2] = {0, 0};
    Arena scalarArena_;
    double *cw_ = nullptr, *ocr_ = nullptr, *partialS_ = nullptr;
    Arena wallArena_;
    int32_t* wallFaces_ = nullptr;  // reactive boundary faces of the solved scalars
    int nWallFaces_ = 0;
    bool wallFacesReady_ = false;
    int precision_ = AXISIM_PREC_FP64;
    int psolve_ = AXISIM_PSOLVE_VCYCLES;
    double psolveTol_ = 0.0;
    double prolongScale_ = 1.0;  // coarse-correction scale inside the FCG preconditioner
    double curProlong_ = 1.0;    // scale of the cycle being captured

    cudaStream_t stream_ = nullptr;
    cudaStream_t loopStream_ = nullptr;  // captures the body of the Krylov loop's WHILE node
    // the coarse operators of the p' solve are built on a second stream of the
    // captured graph, beside the right-hand side and the finest level's
    // residual, and joined before the first restriction reads them
    cudaStream_t galStream_ = nullptr;
    cudaEvent_t evFork_ = nullptr;
    std::vector<cudaEvent_t> evGal_;  // recorded after each coarse level's operator is built
    std::vector<int> galEvOf_;        // level -> the event that covers it (the chain covers several)
    bool galerkinForked_ = false;     // this solve's Galerkin is on galStream_
    int galJoined_ = 0;               // stream_ has waited for the operators of levels 1..galJoined_
    volatile int* hostStop_ = nullptr;
    int* hostStopDev_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    std::atomic<bool> running_{false};
    bool isReady_ = false;
    double simTime_ = 0.0;

    // mesh
    bool haveMesh_ = false;
    int N_ = 0, F_ = 0, S_ = 0, W_ = 0;
    int nSeg_ = 0, segIrregular_ = 0;  // 32-cell segments of the mesh; those without shared slot offsets
    int segCounts_[2] = {0, 0};        // segments without slot offsets, without affine faces
    HostI32 hCfs_, hCfi_, hOwner_, hNeighbor_;
    Arena meshArena_, mgArena_, bcArena_;
    Arena segArena_;  // the mesh's segment tables, kept only when the kernels use them
    // momentum Jacobi sweeps per launch out of shared memory (1: one launch
    // per sweep), CTA size of those launches, and the tiles they run on
    int sweepsPerLaunch_ = 1;
    int sweepThreads_ = 1024;
    SweepTilesDev tiles_;
    int tilesKey_ = 0;  // cap * 8 + S the tiles were built for, 0 = none
    Arena tileArena_;
    MeshDev mesh_;
    double *u_ = nullptr, *v_ = nullptr, *p_ = nullptr, *pp_ = nullptr, *uT_ = nullptr, *vT_ = nullptr, *ppT_ = nullptr;
    double *DU_ = nullptr, *DV_ = nullptr, *gPZ_ = nullptr, *gPR_ = nullptr, *gUZ_ = nullptr, *gUR_ = nullptr;
    double *gVZ_ = nullptr, *gVR_ = nullptr, *uOld_ = nullptr, *vOld_ = nullptr, *uOld2_ = nullptr, *vOld2_ = nullptr;
    double *mDot_ = nullptr, *AFm_ = nullptr, *ACu_ = nullptr, *ACv_ = nullptr, *bu_ = nullptr, *bv_ = nullptr;
    double *iu_ = nullptr, *iv_ = nullptr, *AFpp_ = nullptr, *ACpp_ = nullptr, *bpp_ = nullptr, *ipp_ = nullptr;
    double *resU_ = nullptr, *resV_ = nullptr, *resC_ = nullptr, *scU_ = nullptr, *scV_ = nullptr, *partial_ = nullptr;
    Ctl* ctl_ = nullptr;

    // boundary conditions
    HostBC hbc_[3];
    bool haveBC_[3] = {false, false, false};
    bool bcDirty_ = true;
    BCDev bc_[4];  // u, v, p, p'
    double* bcValueDev_[2] = {nullptr, nullptr};
    double* hostBCStage_ = nullptr;

    // multigrid / colouring
    std::vector<GridLevel> hier_;
    // batch with per-case hierarchies: per level, the [begin, end) ranges of
    // the cases whose coarsest level it is (empty: one joint hierarchy)
    std::vector<std::vector<int32_t>> termRanges_;
    static constexpr int kMaxTerminalCells = 12 * 1024;  // a terminal case's shared-memory sweeps
    bool haveHierarchy_ = false;
    int autotune_ = 0;             // tune the level launch shapes before capturing the graph
    std::vector<double> tuneUs_;   // measured sweep time per level and candidate (us)
    std::vector<LevelDev> levels_;
    // mixed precision: FP32 copies of the hierarchy and the inner-solve vectors
    Arena mixArena_;
    std::vector<LevelF> levels32_;
    float *AF32m_ = nullptr, *iu32_ = nullptr, *iv32_ = nullptr, *ru32_ = nullptr, *rv32_ = nullptr;
    float *du32_[2] = {nullptr, nullptr}, *dv32_[2] = {nullptr, nullptr};
    float *AF32pp_ = nullptr, *AC32pp_ = nullptr, *r32pp_ = nullptr, *e32_[2] = {nullptr, nullptr}, *res32_ = nullptr;
    // flexible CG on the p' system: FP64 residual, directions (two, alternating), A p
    double *fcgR_ = nullptr, *fcgP_[2] = {nullptr, nullptr}, *fcgQ_ = nullptr;
    FcgScratch fcg_;
    // counters of the Krylov steps (V-cycle reduction, learned-step outcomes)
    Arena netArena_;
    NetStats* netStats_ = nullptr;
    float* nnY_ = nullptr;    // the network's output in the first Krylov iteration
    double* nnAy_ = nullptr;  // A times it
    // learned preconditioner and its harvested (b, p', A_C, deficit, A_F)
    // training samples, FP32 [cap][4 + W][N] (A_F as ELL)
    LearnedNet net_;
    int learnedMode_ = 0;
    int adamT_ = 0;
    Arena sampleArena_;
    int harvestEvery_ = 0, sampleCap_ = 0;
    float* samples_ = nullptr;
    int* sampleCount_ = nullptr;
    float* sampleRelres_ = nullptr;
    unsigned int* harvestCounter_ = nullptr;
    std::vector<int32_t> hColor_, hColorStart_;
    int colorN_ = 0;
    int32_t* dCellOrder_ = nullptr;

    // per-kernel profiling (eager replay of one iteration with an event after each launch)
    struct Mark {
        std::string name;
        cudaEvent_t ev;
        double bytes;
    };
    bool profiling_ = false;
    bool profileByLevel_ = false;  // multigrid marks carry "@<level>"
    std::vector<Mark> marks_;
    // a multigrid launch on `level`
    void markL(const std::string& name, int level, double bytes) {
        if (!profiling_) return;
        mark(profileByLevel_ ? (name + "@" + std::to_string(level)).c_str() : name.c_str(), bytes);
    }
    void mark(const char* name, double bytes) {
        if (!profiling_) return;
        Mark m{name, nullptr, bytes};
        CK(cudaEventCreate(&m.ev));
        CK(cudaEventRecord(m.ev, stream_));
        marks_.push_back(m);
    }

    // host-clock cost of each set-up stage (set_mesh, hierarchy, graph
    // capture, ...), summed per stage name since the handle was created
    struct Phase {
        std::string name;
        int calls;
        double ms;
    };
    std::vector<Phase> phases_;
    struct PhaseTimer {
        Solver& s;
        const char* name;
        std::chrono::steady_clock::time_point t0;
        PhaseTimer(Solver& so, const char* n) : s(so), name(n), t0(std::chrono::steady_clock::now()) {}
        ~PhaseTimer() {
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            s.addPhase(name, ms);
        }
    };
    void addPhase(const char* name, double ms) {
        for (Phase& p : phases_)
            if (p.name == name) {
                p.calls++;
                p.ms += ms;
                return;
            }
        phases_.push_back(Phase{name, 1, ms});
    }

public:
    // The 32-cell segment tables of the mesh (segNeighbours / slotFaces).
    void meshSegments(int32_t* nSeg, int32_t* nOffsets, int32_t* nFaces, int32_t* inUse) const {
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
        if (nSeg) *nSeg = nSeg_;
        if (nOffsets) *nOffsets = nSeg_ - segCounts_[0];
        if (nFaces) *nFaces = nSeg_ - segCounts_[1];
        if (inUse) *inUse = mesh_.sseg ? 1 : 0;
    }

    int setupProfile(axisim_kernel_stat* out, int maxOut, int reset) {
        const int n = (int)phases_.size();
        for (int i = 0; i < n && i < maxOut; i++) {
            axisim_kernel_stat st{};
            std::snprintf(st.name, sizeof(st.name), "%s", phases_[(size_t)i].name.c_str());
            st.launches = phases_[(size_t)i].calls;
            st.ms = phases_[(size_t)i].ms;
            st.bytes = 0.0;
            out[i] = st;
        }
        if (reset) phases_.clear();
        return n;
    }

private:
    // batch of independent cases packed into one mesh
    Arena batchArena_;
    BatchDev batch_;
    std::vector<int32_t> hCaseStart_;

    // graph
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    int residualBlocks_ = 0;

    void destroyGraph() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
    }

    void log(const std::string& s) {
        if (logFn) logFn(cbCtx, s.c_str());
    }

    void uploadBC() {
        if (!bcDirty_) return;
        PhaseTimer ph(*this, "bc_upload");
        bcArena_.release();
        wallFacesReady_ = false;
        for (int var = 0; var < 3; var++) {
            const HostBC& h = hbc_[var];
            BCDev d;
            d.nGroups = h.nGroups;
            d.type = bcArena_.upload(h.type.data(), h.type.size());
            d.value = bcArena_.upload(h.value.data(), h.value.size());
            d.length = bcArena_.upload(h.length.data(), h.length.size());
            bc_[var] = d;
            if (var < 2) bcValueDev_[var] = const_cast<double*>(d.value);
        }
        // p' boundary field: p's types with every value zero (solver.cpp:788-795)
        BCDev pp = bc_[2];
        std::vector<double> zeros((size_t)std::max(hbc_[2].nGroups, 1), 0.0);
        pp.value = bcArena_.upload(zeros.data(), zeros.size());
        bc_[3] = pp;
        // T and C: kinetics [9][G] = Vmax Km n m K2 V2 Rtot, then Km^n and K2^m
        // precomputed on the host (memory_manger.cpp:72-83, 110-136)
        for (int q = 0; q < 2; q++) {
            const HostBC& h = hbcS_[q];
            BCDev d;
            d.nGroups = h.nGroups;
            if (h.nGroups > 0) {
                const int G = h.nGroups;
                d.type = bcArena_.upload(h.type.data(), h.type.size());
                d.value = bcArena_.upload(h.value.data(), h.value.size());
                d.length = bcArena_.upload(h.length.data(), h.length.size());
                std::vector<double> kin((size_t)9 * G, 0.0);
                const double dflt[7] = {0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0};
                for (int j = 0; j < 7; j++)
                    for (int g = 0; g < G; g++)
                        kin[(size_t)j * G + g] = g < hkinG_[q] ? hkin_[q][(size_t)j * hkinG_[q] + g] : dflt[j];
                for (int g = 0; g < G; g++) {
                    kin[(size_t)7 * G + g] = std::pow(kin[(size_t)1 * G + g], kin[(size_t)2 * G + g]);
                    kin[(size_t)8 * G + g] = std::pow(kin[(size_t)4 * G + g], kin[(size_t)3 * G + g]);
                }
                d.kin = bcArena_.upload(kin.data(), kin.size());
            }
            bcS_[q] = d;
        }
        int maxG = std::max(hbc_[0].nGroups, hbc_[1].nGroups);
        if (hostBCStage_) cudaFreeHost(hostBCStage_);
        hostBCStage_ = nullptr;
        CK(cudaHostAlloc((void**)&hostBCStage_, sizeof(double) * 2 * (size_t)std::max(maxG, 1), cudaHostAllocDefault));
        bcDirty_ = false;
        destroyGraph();
    }

    // Buffers of the solved scalars (zeroed on allocation, as allocateSimple
    // zero-fills temp / conc, memory_manger.cpp:740-772).
    void ensureScalarBuffers() {
        const size_t N = (size_t)N_, WN = (size_t)W_ * N_;
        for (int q = 0; q < 2; q++) {
            if (!solveS_[q] || sb_[q].phi) continue;
            ScalarBuf& b = sb_[q];
            Arena& A = scalarArena_;
            b.phi = A.alloc<double>(N); b.tmp = A.alloc<double>(N); b.lvl[0] = A.alloc<double>(N);
            b.lvl[1] = A.alloc<double>(N); b.gZ = A.alloc<double>(N); b.gR = A.alloc<double>(N);
            b.AF = A.alloc<double>(WN); b.AC = A.alloc<double>(N); b.b = A.alloc<double>(N);
            b.inv = A.alloc<double>(N); b.res = A.alloc<double>(N); b.scale = A.alloc<double>(N);
            b.wall = A.alloc<double>((size_t)F_);
            b.swapped = 0;
        }
        if ((solveS_[0] || solveS_[1]) && !cw_) {
            cw_ = scalarArena_.alloc<double>((size_t)F_);
            ocr_ = scalarArena_.alloc<double>((size_t)F_);
            partialS_ = scalarArena_.alloc<double>((size_t)((N_ + 255) / 256) * 4 + 4);
        }
    }
    void releaseScalarBuffers() {
        scalarArena_.release();
        sb_[0] = ScalarBuf{};
        sb_[1] = ScalarBuf{};
        cw_ = ocr_ = partialS_ = nullptr;
        wallFaces_ = nullptr;
        nWallFaces_ = 0;
        wallFacesReady_ = false;
        ranS_[0] = ranS_[1] = 0;
    }

    void ensureHierarchy() {
        if (haveHierarchy_) return;
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
        PhaseTimer ph(*this, "hierarchy_host");
        GridLevel fine = finestLevel(N_, F_, hCfs_.data(), hCfi_.data(), hOwner_.data(), hNeighbor_.data());
        termRanges_.clear();
        if (hCaseStart_.size() > 2) {
            // each case coarsened alone; a case with one level only would be
            // terminal on the finest level, which the fine-level kernels do
            // not support: such a batch keeps one joint hierarchy
            std::vector<std::vector<int32_t>> term;
            std::vector<GridLevel> h = buildBatchHierarchy(fine, hCaseStart_, term);
            size_t biggest = 0;
            for (const auto& t : term)
                for (size_t i = 0; i + 1 < t.size(); i += 2) biggest = std::max(biggest, (size_t)(t[i + 1] - t[i]));
            if (term.empty() || !term[0].empty() || biggest > kMaxTerminalCells) {
                log("batch: a case has a single multigrid level or a coarsest level above " +
                    std::to_string(kMaxTerminalCells) + " cells; the batch shares one hierarchy\n");
                hier_ = buildHierarchy(std::move(fine));
            } else {
                hier_ = std::move(h);
                termRanges_ = std::move(term);
            }
        } else {
            hier_ = buildHierarchy(std::move(fine));
        }
        haveHierarchy_ = true;
        levels_.clear();
        levels32_.clear();
        mgArena_.release();
    }

    void ensureColoring() {
        if (colorN_ > 0) return;
        PhaseTimer ph(*this, "coloring_host");
        GridLevel g = finestLevel(N_, F_, hCfs_.data(), hCfi_.data(), hOwner_.data(), hNeighbor_.data());
        colorN_ = greedyColoring(g, hColor_);
        hColorStart_.assign((size_t)colorN_ + 1, 0);
        for (int c = 0; c < N_; c++) hColorStart_[(size_t)hColor_[(size_t)c] + 1]++;
        for (int k = 0; k < colorN_; k++) hColorStart_[(size_t)k + 1] += hColorStart_[(size_t)k];
        std::vector<int32_t> order((size_t)N_);
        std::vector<int32_t> fill(hColorStart_);
        for (int c = 0; c < N_; c++) order[(size_t)fill[(size_t)hColor_[(size_t)c]]++] = c;
        dCellOrder_ = meshArena_.upload(order.data(), order.size());
    }

    // Device copies of the hierarchy: level 0 aliases the p' system; coarser
    // levels in sliced ELL; member lists and fine->coarse slot gathers for the
    // restriction and the Galerkin build; the V-cycle tail for small levels.
    void ensureDeviceLevels() {
        ensureHierarchy();
        if (!levels_.empty()) return;
        PhaseTimer ph(*this, "levels_build_upload");
        const int L = (int)hier_.size();
        levels_.resize((size_t)L);
        std::vector<std::vector<int32_t>> sliceOffH((size_t)L);
        auto pos = [&](int l, int c, int j) -> int {
            if (l == 0) return j * N_ + c;
            return sliceOffH[(size_t)l][(size_t)(c >> 5)] + 32 * j + (c & 31);
        };
        for (int l = 0; l < L; l++) {
            const GridLevel& g = hier_[(size_t)l];
            LevelDev& d = levels_[(size_t)l];
            d.N = g.nCells;
            if (l == 0) {
                d.W = W_;
                d.totalSlots = W_ * N_;
                d.nb = const_cast<int32_t*>(mesh_.snb);
                d.seg = mesh_.sseg;
                d.AF = AFpp_;
                d.AC = ACpp_;
                d.b = bpp_;
                d.x = pp_;
                d.xNew = ppT_;
            } else {
                const int nS = (g.nCells + 31) / 32;
                std::vector<int32_t>& off = sliceOffH[(size_t)l];
                off.assign((size_t)nS + 1, 0);
                int W = 0;
                for (int sI = 0; sI < nS; sI++) {
                    int w = 0;
                    for (int c = sI * 32; c < std::min(g.nCells, sI * 32 + 32); c++)
                        w = std::max(w, g.faceStart[(size_t)c + 1] - g.faceStart[(size_t)c]);
                    off[(size_t)sI + 1] = off[(size_t)sI] + 32 * w;
                    W = std::max(W, w);
                }
                d.W = W;
                d.totalSlots = off[(size_t)nS];
                std::vector<int32_t> nb((size_t)std::max(d.totalSlots, 1), -1);
                parallelFor(g.nCells, [&](int c0, int c1) {
                    for (int c = c0; c < c1; c++)
                        for (int k = g.faceStart[(size_t)c], j = 0; k < g.faceStart[(size_t)c + 1]; k++, j++)
                            nb[(size_t)pos(l, c, j)] = g.faceNeighbor[(size_t)k];
                });
                d.sliceOff = mgArena_.upload(off.data(), off.size());
                d.nb = mgArena_.upload(nb.data(), nb.size());
                d.AF = mgArena_.alloc<double>(nb.size());
                d.AC = mgArena_.alloc<double>((size_t)g.nCells);
                d.b = mgArena_.alloc<double>((size_t)g.nCells);
                d.x = mgArena_.alloc<double>((size_t)g.nCells);
                d.xNew = mgArena_.alloc<double>((size_t)g.nCells);
            }
            if (!g.isCoarsest()) {
                d.c2c = mgArena_.upload(g.cellToCoarse.data(), g.cellToCoarse.size());
                d.res = mgArena_.alloc<double>((size_t)g.nCells);
            }
        }
        for (int l = 1; l < L; l++) {
            const GridLevel& f = hier_[(size_t)l - 1];
            const GridLevel& c = hier_[(size_t)l];
            LevelDev& fd = levels_[(size_t)l - 1];
            LevelDev& cd = levels_[(size_t)l];
            // members of each coarse cell (a batch's terminal cells have no coarse cell)
            std::vector<int32_t> mStart((size_t)c.nCells + 1, 0), mList;
            for (int n = 0; n < f.nCells; n++)
                if (f.cellToCoarse[(size_t)n] >= 0) mStart[(size_t)f.cellToCoarse[(size_t)n] + 1]++;
            for (int k = 0; k < c.nCells; k++) mStart[(size_t)k + 1] += mStart[(size_t)k];
            mList.resize((size_t)std::max(mStart[(size_t)c.nCells], 1));
            {
                std::vector<int32_t> fill(mStart);
                for (int n = 0; n < f.nCells; n++)
                    if (f.cellToCoarse[(size_t)n] >= 0) mList[(size_t)fill[(size_t)f.cellToCoarse[(size_t)n]]++] = n;
            }
            std::vector<int32_t> coarsePos((size_t)std::max(c.nFaceRefs(), 1));
            parallelFor(c.nCells, [&](int c0, int c1) {
                for (int cc = c0; cc < c1; cc++)
                    for (int k = c.faceStart[(size_t)cc], j = 0; k < c.faceStart[(size_t)cc + 1]; k++, j++)
                        coarsePos[(size_t)k] = pos(l, cc, j);
            });
            // Each coarse slot is fed only by members of its own coarse cell, so
            // the counts and lists are built per coarse cell in parallel; its
            // members in ascending order keep every list in ascending fine order.
            std::vector<int32_t> gCount((size_t)cd.totalSlots + 1, 0);
            std::vector<uint32_t> mask((size_t)f.nCells, 0u);
            parallelFor(f.nCells, [&](int n0, int n1) {
                for (int n = n0; n < n1; n++)
                    for (int k = f.faceStart[(size_t)n], j = 0; k < f.faceStart[(size_t)n + 1]; k++, j++)
                        if (f.faceNeighbor[(size_t)k] >= 0 && f.fineSlotToCoarseSlot[(size_t)k] < 0)
                            mask[(size_t)n] |= (1u << j);
            });
            auto eachSource = [&](int cc, auto&& fn) {
                for (int q = mStart[(size_t)cc]; q < mStart[(size_t)cc + 1]; q++) {
                    const int n = mList[(size_t)q];
                    for (int k = f.faceStart[(size_t)n], j = 0; k < f.faceStart[(size_t)n + 1]; k++, j++) {
                        if (f.faceNeighbor[(size_t)k] < 0) continue;
                        const int sI = f.fineSlotToCoarseSlot[(size_t)k];
                        if (sI >= 0) fn(coarsePos[(size_t)sI], n, j);
                    }
                }
            };
            parallelFor(c.nCells, [&](int c0, int c1) {
                for (int cc = c0; cc < c1; cc++) eachSource(cc, [&](int p, int, int) { gCount[(size_t)p + 1]++; });
            });
            std::vector<int32_t> gStart(gCount.size(), 0);
            for (size_t i = 1; i < gCount.size(); i++) gStart[i] = gStart[i - 1] + gCount[i];
            std::vector<int32_t> gList((size_t)std::max(gStart.back(), 1));
            {
                std::vector<int32_t> fill(gStart);
                parallelFor(c.nCells, [&](int c0, int c1) {
                    for (int cc = c0; cc < c1; cc++)
                        eachSource(cc, [&](int p, int n, int j) { gList[(size_t)fill[(size_t)p]++] = pos(l - 1, n, j); });
                });
            }
            cd.mStart = mgArena_.upload(mStart.data(), mStart.size());
            cd.mList = mgArena_.upload(mList.data(), mList.size());
            cd.gStart = mgArena_.upload(gStart.data(), gStart.size());
            cd.gList = mgArena_.upload(gList.data(), gList.size());
            fd.internalMask = mgArena_.upload(mask.data(), mask.size());
        }
        int lastTerminal = -1;
        for (int l = 0; l < (int)termRanges_.size() && l < L; l++) {
            const std::vector<int32_t>& t = termRanges_[(size_t)l];
            if (t.empty()) continue;
            LevelDev& d = levels_[(size_t)l];
            d.nTerm = (int)t.size() / 2;
            d.termMax = 0;
            for (size_t i = 0; i + 1 < t.size(); i += 2) d.termMax = std::max(d.termMax, t[i + 1] - t[i]);
            d.term = mgArena_.upload(t.data(), t.size());
            lastTerminal = l;
        }
        // V-cycle tail: the deepest levels that all fit one CTA's shared memory
        tailStart_ = -1;
        for (int t = std::max(1, lastTerminal + 1); t < L; t++) {
            if (L - t > kMaxTail) continue;
            bool fits = true;
            size_t bytes = 0;
            for (int l = t; l < L; l++) {
                fits = fits && levels_[(size_t)l].N <= 1024;
                bytes += 4 * (size_t)levels_[(size_t)l].N * sizeof(double);
            }
            if (fits && bytes <= 200 * 1024) {
                tailStart_ = t;
                break;
            }
        }
    }
    int tailStart_ = -1;
    bool galerkinThisSolve_ = true;  // false: the coarse operators of this p' solve are already built
    double* irUpdate_ = nullptr;     // set during a mixed refinement cycle: the FP64 iterate it corrects
    bool irUpdated_ = false;         // the cycle's last finest-level pass applied the correction

    // FP32 p' hierarchy: used by the mixed-precision cycle and as the
    // preconditioner of the flexible CG solve in either precision
    bool fp32PressureCycle() const {
        return cs_.useMultigrid && (precision_ == AXISIM_PREC_MIXED || psolve_ == AXISIM_PSOLVE_FCG);
    }

    void dropSweepTiles() {
        tileArena_.release();
        tiles_ = SweepTilesDev{};
        tilesKey_ = 0;
    }

    // Tiles for several momentum sweeps per launch (SweepTiles), built for
    // the precision of the sweeps: cap = K x CTA size local cells. Runs of the
    // cell curve are sized so the tiles fill whole waves of resident CTAs;
    // where no tiling fits (a cell whose halo alone exceeds cap) the sweeps
    // stay one launch each.
    void ensureSweepTiles() {
        const bool fp32 = precision_ == AXISIM_PREC_MIXED && cs_.type != 1;
        const int S = sweepsPerLaunch_;
        if (S <= 1 || cs_.type == 1 || W_ < 3 || W_ > 4 || cs_.linearMaxIter < 2) {
            dropSweepTiles();
            return;
        }
        const int cap = (fp32 ? kSweepK32 : kSweepK64) * sweepThreads_;
        const int key = cap * 8 + S;
        if (tilesKey_ == key) return;
        PhaseTimer ph(*this, "sweep_tiles");
        dropSweepTiles();
        const std::vector<int32_t> nb =
            slotNeighbours(N_, W_, hCfs_.data(), hCfi_.data(), hOwner_.data(), hNeighbor_.data());
        int sms = 148;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
        const int slots = sms * std::max(1, 1024 / sweepThreads_);  // 64 registers a thread: 1024 threads per SM
        const int l0max = std::max(32, (int)(cap / (1.0 + 0.1 * S)));
        // whole waves of tiles when that costs at most 15 % of the tile size
        const long long per = (long long)slots * l0max;
        const int waves = (int)std::max(1LL, ((long long)N_ + per - 1) / per);
        int tileCells = (int)(((long long)N_ + (long long)waves * slots - 1) / ((long long)waves * slots));
        if (tileCells < l0max * 85 / 100) tileCells = l0max;
        const int nCases = hCaseStart_.empty() ? 0 : (int)hCaseStart_.size() - 1;
        std::vector<double> cz((size_t)N_), cr((size_t)N_);  // the cell centres, for the tile curve
        CK(cudaMemcpy(cz.data(), mesh_.ccZ, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(cr.data(), mesh_.ccR, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToHost));
        SweepTiles t = buildSweepTiles(N_, W_, nb.data(), cz.data(), cr.data(), S, cap, tileCells,
                                       nCases ? hCaseStart_.data() : nullptr, nCases);
        tilesKey_ = key;
        if (t.nTiles() == 0) return;
        CK(fp32 ? allowJacobiUV32Tiles(cap) : allowJacobiUVTiles(cap));
        Arena& A = tileArena_;
        tiles_.nTiles = t.nTiles();
        tiles_.S = S;
        tiles_.cap = cap;
        tiles_.threads = sweepThreads_;
        tiles_.tileStart = A.upload(t.tileStart.data(), t.tileStart.size());
        tiles_.layerEnd = A.upload(t.layerEnd.data(), t.layerEnd.size());
        tiles_.gid = A.upload(t.gid.data(), t.gid.size());
        tiles_.lnb = reinterpret_cast<const uint2*>(A.upload(t.lnb.data(), t.lnb.size()));
        tileLocal_ = (double)t.gid.size();
    }
    double tileLocal_ = 0.0;  // local cells of all tiles (layer 0 and halo)

    void ensureMixedBuffers() {
        if (precision_ != AXISIM_PREC_MIXED && !fp32PressureCycle()) return;
        PhaseTimer ph(*this, "mixed_buffers");
        if (psolve_ == AXISIM_PSOLVE_FCG && !fcgR_) {
            const size_t N = (size_t)N_;
            Arena& A = mixArena_;
            fcgR_ = A.alloc<double>(N);
            fcgP_[0] = A.alloc<double>(N);
            fcgP_[1] = A.alloc<double>(N);
            fcgQ_ = A.alloc<double>(N);
            fcg_.partial = A.alloc<double>((N + 255) / 256 * 2);
            fcg_.counter = A.alloc<unsigned int>(2);
            fcg_.scalars = A.alloc<double>(16);
        }
        if (!AF32m_) {
            const size_t N = (size_t)N_, WN = (size_t)W_ * N;
            Arena& A = mixArena_;
            AF32m_ = A.alloc<float>(WN);
            iu32_ = A.alloc<float>(N); iv32_ = A.alloc<float>(N);
            ru32_ = A.alloc<float>(N); rv32_ = A.alloc<float>(N);
            for (int i = 0; i < 2; i++) {
                du32_[i] = A.alloc<float>(N);
                dv32_[i] = A.alloc<float>(N);
                e32_[i] = A.alloc<float>(N);
            }
            AF32pp_ = A.alloc<float>(WN);
            AC32pp_ = A.alloc<float>(N);
            r32pp_ = A.alloc<float>(N);
            res32_ = A.alloc<float>(N);
        }
        if (!cs_.useMultigrid || !levels32_.empty()) return;
        // FP32 hierarchy: the same topology and transfer lists as levels_
        const int L = (int)levels_.size();
        levels32_.resize((size_t)L);
        for (int l = 0; l < L; l++) {
            const LevelDev& d = levels_[(size_t)l];
            LevelF& f = levels32_[(size_t)l];
            f.N = d.N;
            f.W = d.W;
            f.totalSlots = d.totalSlots;
            f.sliceOff = d.sliceOff;
            f.nb = d.nb;
            f.seg = d.seg;
            f.c2c = d.c2c;
            f.mStart = d.mStart;
            f.mList = d.mList;
            f.gStart = d.gStart;
            f.gList = d.gList;
            f.internalMask = d.internalMask;
            f.nTerm = d.nTerm;
            f.termMax = d.termMax;
            f.term = d.term;
            if (l == 0) {
                f.AF = AF32pp_;
                f.AC = AC32pp_;
                f.b = r32pp_;
                f.x = e32_[0];
                f.xNew = e32_[1];
                f.res = res32_;
            } else {
                f.AF = mixArena_.alloc<float>((size_t)std::max(d.totalSlots, 1));
                f.AC = mixArena_.alloc<float>((size_t)d.N);
                f.b = mixArena_.alloc<float>((size_t)d.N);
                f.x = mixArena_.alloc<float>((size_t)d.N);
                f.xNew = mixArena_.alloc<float>((size_t)d.N);
                f.res = d.c2c ? mixArena_.alloc<float>((size_t)d.N) : nullptr;
            }
        }
    }

    // ---------- capture of one SIMPLE iteration (solver.cpp:1109-1284) ----------
    template <class T>
    void smoothT(std::vector<LevelT<T>>& lv, int l, int sweeps, std::vector<T*>& cur, std::vector<T*>& alt) {
        LevelT<T>& L = lv[(size_t)l];
        if (L.N <= 0 || sweeps <= 0) return;
        const T w = (T)cmg_.weight;
        const char* tag = sizeof(T) == 8 ? "" : "32";
        if (sweeps > 1 && L.N <= 4096) {
            T* x = cur[(size_t)l];
            emit<T>(kOpSmoothBlock, l, x, nullptr, sweeps, 0.0, 2 * (size_t)L.N * sizeof(T),
                    std::string("mg_smooth_block") + tag,
                    (double)L.N * ((4.0 + 2 * sizeof(T)) * L.W + 4.0 * sizeof(T)),
                    [&] { launchMGSmoothBlock<T>(ctl_, L, x, w, sweeps, stream_); });
            return;
        }
        for (int i = 0; i < sweeps; i++) {
            T* x = cur[(size_t)l];
            T* y = alt[(size_t)l];
            emit<T>(kOpSmooth, l, x, y, 0, 0.0, 0, std::string(l == 0 ? "mg_smooth_l0" : "mg_smooth") + tag,
                    (double)L.N * ((double)sizeof(T) * L.W + 4.0 * sizeof(T)) + slotIndexBytes(L),
                    [&] { launchMGSmooth<T>(ctl_, L, x, y, w, stream_); });
            std::swap(cur[(size_t)l], alt[(size_t)l]);
        }
    }

    // The V-cycle below the finest level as one resident kernel: while a
    // program is being recorded, emit() appends the phase instead of
    // launching it (the launch and its profile mark happen otherwise).
    ResidentArgsT<double>* rec64_ = nullptr;
    ResidentArgsT<float>* rec32_ = nullptr;
    double recBytes_ = 0.0;
    int residentVcycle_ = 0;
    // coarse levels up to this size fuse residual + restriction and
    // prolongation + first post-sweep (beyond it the fused forms, one thread
    // per row gathering its neighbours' corrections, run slower than two
    // coalesced passes)
    static constexpr int kFuseMaxCells = 65536;
    int barrierPhantom_ = 0;  // test hook: extra arrivals each grid barrier expects
    bool timedOut_ = false;   // the last run ended on a barrier that gave up
    template <class T>
    ResidentArgsT<T>*& recSlot() {
        if constexpr (std::is_same_v<T, double>) return rec64_;
        else return rec32_;
    }
    template <class T, class Launch>
    void emit(int type, int level, void* p0, void* p1, int ival, double scale, size_t smem, const std::string& name,
              double bytes, Launch&& launch, void* p2 = nullptr) {
        ResidentArgsT<T>* r = recSlot<T>();
        if (!r) {
            launch();
            markL(name, level, bytes);
            return;
        }
        if (r->nOps < kMaxResidentOps) {
            MgOp& o = r->ops[r->nOps];
            o.type = type;
            o.level = level;
            o.ival = ival;
            o.p0 = p0;
            o.p1 = p1;
            o.p2 = p2;
            o.scale = scale;
        }
        r->nOps++;  // a count past the capacity drops the program (per-phase launches instead)
        r->smem = std::max(r->smem, smem);
        recBytes_ += bytes;
    }

    // One V-cycle from level l (multigrid.cu:607-662). firstDone: the gather
    // (or, on level 0 of the mixed cycle, the refinement residual) that
    // produced this level's right-hand side already ran its first
    // pre-smoothing sweep.
    template <class T>
    void vcycleT(std::vector<LevelT<T>>& lv, int l, std::vector<T*>& cur, std::vector<T*>& alt, bool firstDone) {
        const int L = (int)lv.size();
        if (l < 0 || l >= L) return;
        const T w = (T)cmg_.weight;
        const char* tag = sizeof(T) == 8 ? "" : "32";
        const double vb = (double)sizeof(T);
        if (hier_[(size_t)l].isCoarsest()) {
            smoothT<T>(lv, l, cmg_.linearSweep - (firstDone ? 1 : 0), cur, alt);
            return;
        }
        smoothT<T>(lv, l, cmg_.linearPreSweep - (firstDone ? 1 : 0), cur, alt);
        LevelT<T>& F = lv[(size_t)l];
        LevelT<T>& C = lv[(size_t)l + 1];
        // on a small coarse level the restriction forms its members' residuals
        // itself (one launch instead of two where launches dominate); larger
        // levels, the finest one (coalesced [W][N] rows) and the level above
        // the tail (whose residual the tail reads) keep the separate pass
        const bool gatherRes = F.sliceOff != nullptr && F.N <= kFuseMaxCells && l + 1 != tailStart_;
        if (!gatherRes) {
            T* x = cur[(size_t)l];
            emit<T>(kOpResidual, l, x, nullptr, 0, 0.0, 0, std::string("mg_residual") + tag,
                    (double)F.N * (vb * F.W + 4.0 * vb) + slotIndexBytes(F),
                    [&] { launchMGResidual<T>(ctl_, F, x, stream_); });
        }
        // level l + 1's operator is read from here on; the tail reads every
        // level below it as well
        joinGalerkin(l + 1 == tailStart_ ? L - 1 : l + 1);
        if (l + 1 == tailStart_) {
            TailArgsT<T> a;
            a.first = l + 1;
            a.count = L - (l + 1);
            size_t off = 0;
            for (int i = 0; i < a.count; i++) {
                a.lv[i] = lv[(size_t)(l + 1 + i)];
                a.smemOff[i] = (int)off;
                off += 4 * (size_t)a.lv[i].N;
            }
            a.resFine = F.res;
            a.xOut = cur[(size_t)l + 1];
            a.w = w;
            a.pre = cmg_.linearPreSweep;
            a.post = cmg_.linearPostSweep;
            a.coarseSweeps = cmg_.linearSweep;
            a.prolongScale = (T)curProlong_;
            double tb = 0.0;
            for (int i = 0; i < a.count; i++) tb += (double)a.lv[i].N * ((4.0 + vb) * a.lv[i].W + 4.0 * vb);
            if (ResidentArgsT<T>* r = recSlot<T>()) r->tail = a;
            emit<T>(kOpTail, l + 1, nullptr, nullptr, 0, 0.0, tailSharedBytes<T>(a), std::string("mg_tail") + tag, tb,
                    [&] { launchMGTail<T>(ctl_, a, stream_); });
        } else {
            const bool coarseIsCoarsest = hier_[(size_t)l + 1].isCoarsest();
            const int sweepsBelow = coarseIsCoarsest ? cmg_.linearSweep : cmg_.linearPreSweep;
            const bool fuse = sweepsBelow >= 1;
            {
                T* xc = cur[(size_t)l + 1];
                T* xa = alt[(size_t)l + 1];
                if (gatherRes) {
                    T* xf = cur[(size_t)l];
                    emit<T>(kOpGatherRes, l + 1, xc, xa, fuse ? 1 : 0, 0.0, 0, std::string("mg_gather_res") + tag,
                            (double)F.N * ((4.0 + vb) * F.W + 4.0 * vb) + 4.0 * F.N + 4.0 * vb * C.N,
                            [&] { launchMGGatherRes<T>(ctl_, F, xf, C, xc, xa, fuse ? 1 : 0, w, stream_); }, xf);
                } else {
                    emit<T>(kOpGather, l + 1, xc, xa, fuse ? 1 : 0, 0.0, 0, std::string("mg_gather") + tag,
                            (4.0 + vb) * F.N + 4.0 * vb * C.N,
                            [&] { launchMGGather<T>(ctl_, F, C, xc, xa, fuse ? 1 : 0, w, stream_); });
                }
            }
            if (fuse) std::swap(cur[(size_t)l + 1], alt[(size_t)l + 1]);
            if (C.nTerm > 0) {  // the cases whose coarsest level this is: their coarsest-level sweeps
                T* x = cur[(size_t)l + 1];
                const int sw = cmg_.linearSweep;
                emit<T>(kOpTerminal, l + 1, x, nullptr, sw, 0.0, 2 * (size_t)C.termMax * sizeof(T),
                        std::string("mg_terminal") + tag, (double)C.N * ((4.0 + vb) * C.W + 3.0 * vb),
                        [&] { launchMGTerminal<T>(ctl_, C, x, w, sw, stream_); });
            }
            if (l == 0 && residentVcycle_ && !recSlot<T>() && L - 1 <= kMaxResidentLevels) {
                // every level below the finest in one resident kernel; if the
                // program does not fit or the device cannot hold the grid, the
                // same phases are launched one by one
                std::unique_ptr<ResidentArgsT<T>> prog(new ResidentArgsT<T>());
                prog->first = 1;
                prog->nLevels = L - 1;
                prog->w = w;
                for (int i = 1; i < L; i++) prog->lv[i - 1] = lv[(size_t)i];
                const std::vector<T*> cur0 = cur, alt0 = alt;
                recBytes_ = 0.0;
                recSlot<T>() = prog.get();
                try {
                    vcycleT<T>(lv, l + 1, cur, alt, fuse);
                } catch (...) {
                    recSlot<T>() = nullptr;
                    throw;
                }
                recSlot<T>() = nullptr;
                if (prog->nOps <= kMaxResidentOps && launchMGResident<T>(ctl_, *prog, stream_)) {
                    markL(std::string("mg_resident") + tag, 1, recBytes_);
                } else {
                    cur = cur0;
                    alt = alt0;
                    vcycleT<T>(lv, l + 1, cur, alt, fuse);
                }
            } else {
                vcycleT<T>(lv, l + 1, cur, alt, fuse);
            }
        }
        const int post = cmg_.linearPostSweep;
        const bool blockSmoother = post > 1 && F.N <= 4096;
        // the prolongation fused into the first post-smoothing sweep: the
        // [W][N] kernel on the finest level (W = 3 or 4; never recorded), the
        // layout-generic one on coarse levels
        const bool fusedEll = post >= 1 && !blockSmoother && !F.sliceOff && F.c2c && (F.W == 3 || F.W == 4) &&
                              !recSlot<T>();
        const bool fusedAny = post >= 1 && !blockSmoother && F.sliceOff && F.c2c && F.N <= kFuseMaxCells;
        if (fusedAny) {
            T* x = cur[(size_t)l];
            T* xc = cur[(size_t)l + 1];
            T* y = alt[(size_t)l];
            const T sc = (T)curProlong_;
            emit<T>(kOpProlongSmooth, l, x, xc, 0, (double)sc, 0, std::string("mg_prolong_smooth") + tag,
                    (double)F.N * (vb * F.W + 4.0 + 4.0 * vb) + slotIndexBytes(F) + vb * C.N,
                    [&] { launchMGProlongSmoothAny<T>(ctl_, F, x, xc, y, w, sc, stream_); }, y);
            std::swap(cur[(size_t)l], alt[(size_t)l]);
            smoothT<T>(lv, l, post - 1, cur, alt);
        } else if (fusedEll && launchMGProlongSmooth<T>(ctl_, F, cur[(size_t)l], cur[(size_t)l + 1], alt[(size_t)l], w,
                                                        (T)curProlong_, stream_,
                                                        (l == 0 && post == 1) ? irUpdate_ : nullptr)) {
            const bool ir = l == 0 && post == 1 && irUpdate_;
            markL(std::string(ir ? "mg_prolong_smooth_ir" : "mg_prolong_smooth") + tag, l,
                 (double)F.N * (vb * F.W + 4.0 + 4.0 * vb + (ir ? 16.0 : 0.0)) + slotIndexBytes(F) + vb * C.N);
            if (ir) irUpdated_ = true;
            std::swap(cur[(size_t)l], alt[(size_t)l]);
            smoothT<T>(lv, l, post - 1, cur, alt);
        } else {
            T* x = cur[(size_t)l];
            T* xc = cur[(size_t)l + 1];
            const T sc = (T)curProlong_;
            emit<T>(kOpProlong, l, x, xc, 0, (double)sc, 0, std::string("mg_prolong") + tag,
                    (4.0 + 2 * vb) * F.N + vb * C.N, [&] { launchMGProlong<T>(ctl_, F, x, xc, sc, stream_); });
            smoothT<T>(lv, l, post, cur, alt);
        }
    }

    // After level l's operator on galStream_: the event the V-cycle waits for.
    void galerkinBuilt(cudaStream_t st, int l, int last) {
        if (st != galStream_ || !galerkinForked_) return;
        CK(cudaEventRecord(evGal_[(size_t)l], st));
        for (int k = l; k <= last; k++) galEvOf_[(size_t)k] = l;
    }

    void enqueueGalerkin64(cudaStream_t st) {
        if (!galerkinThisSolve_) return;
        const int L = (int)levels_.size();
        const int chain = galerkinChainStart(L);
        for (int l = 1; l < chain; l++) {
            const LevelDev& f = levels_[(size_t)l - 1];
            const LevelDev& c = levels_[(size_t)l];
            launchGalerkin(ctl_, f, c, st);
            markL("mg_galerkin", l, galerkinBytes(f, c));
            galerkinBuilt(st, l, l);
        }
        if (chain < L) {
            enqueueGalerkinChain<double>(levels_, chain, "mg_galerkin", st);
            galerkinBuilt(st, chain, L - 1);
        }
    }

    void enqueueGalerkin32(cudaStream_t st) {
        if (!galerkinThisSolve_) return;
        const int L = (int)levels_.size();
        if (L > 1) {
            launchGalerkin<double, float>(ctl_, levels_[0], levels32_[1], st);
            markL("mg_galerkin", 1, (double)levels_[0].N * (20.0 + 8.0 * levels_[0].W) + 12.0 * levels32_[1].totalSlots);
            galerkinBuilt(st, 1, 1);
        }
        const int chain = galerkinChainStart(L);
        for (int l = 2; l < chain; l++) {
            launchGalerkin<float, float>(ctl_, levels32_[(size_t)l - 1], levels32_[(size_t)l], st);
            markL("mg_galerkin32", l, galerkinBytes(levels32_[(size_t)l - 1], levels32_[(size_t)l]));
            galerkinBuilt(st, l, l);
        }
        if (chain < L) {
            enqueueGalerkinChain<float>(levels32_, chain, "mg_galerkin32", st);
            galerkinBuilt(st, chain, L - 1);
        }
    }

    // Forks this p' solve's Galerkin onto galStream_ (captured graph only: the
    // per-kernel profile keeps one stream so every launch has its own events).
    // The V-cycle waits for level l's operator just before it first restricts
    // into level l, so the finer levels' phases overlap the coarser builds.
    void forkGalerkin() {
        const bool mixed = fp32PressureCycle();
        if (profiling_ || !cs_.useMultigrid || psolve_ == AXISIM_PSOLVE_FCG || residentVcycle_ ||
            levels_.size() < 2 || !galerkinThisSolve_)
            return;
        if (!galStream_) CK(cudaStreamCreateWithFlags(&galStream_, cudaStreamNonBlocking));
        if (!evFork_) CK(cudaEventCreateWithFlags(&evFork_, cudaEventDisableTiming));
        const size_t L = levels_.size();
        while (evGal_.size() < L) {
            cudaEvent_t e = nullptr;
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            evGal_.push_back(e);
        }
        galEvOf_.assign(L, -1);
        CK(cudaEventRecord(evFork_, stream_));
        CK(cudaStreamWaitEvent(galStream_, evFork_, 0));
        tNextLaunchPlain = true;  // its first kernel follows an event, not a kernel
        galerkinForked_ = true;
        galJoined_ = 0;
        if (mixed) enqueueGalerkin32(galStream_);
        else enqueueGalerkin64(galStream_);
    }
    // stream_ waits for the operators of levels up to l (no-op unless forked)
    void joinGalerkin(int l) {
        if (!galerkinForked_) return;
        l = std::min(l, (int)galEvOf_.size() - 1);
        if (l <= galJoined_) return;
        const int e = galEvOf_[(size_t)l];
        if (e < 0) return;
        CK(cudaStreamWaitEvent(stream_, evGal_[(size_t)e], 0));
        int covered = l;  // the event also covers the levels its launch built
        while (covered + 1 < (int)galEvOf_.size() && galEvOf_[(size_t)covered + 1] == e) covered++;
        galJoined_ = covered;
        tNextLaunchPlain = true;  // the next kernel follows the join
    }

    // The Galerkin steps into the tail levels (at most 1024 cells each) run in
    // one single-CTA launch; returns the first coarse level of that chain (L:
    // none). The chain starts at level 2 or deeper, so its first fine level is
    // one of the cycle's own levels in either precision.
    int galerkinChainStart(int L) const {
        if (tailStart_ < 2 || L - tailStart_ + 1 > kMaxTail + 1) return L;
        return tailStart_;
    }
    // Neighbour-index bytes one pass over the mesh's slots reads: the segment
    // offsets plus the slot neighbours of the irregular segments where the
    // mesh has segment offsets, else the whole [W][N] block.
    double meshSlotIndexBytes() const {
        if (!mesh_.sseg) return 4.0 * W_ * N_;
        return 16.0 * nSeg_ + 4.0 * W_ * 32.0 * segIrregular_;
    }
    // Face-id, owner and neighbour bytes an assembly pass (momentum, pressure,
    // p' right-hand side, correction, residual, least-squares gradient) does
    // not read where the segment tables give them (slotFaces): the slot's face
    // id and its half of the face's owner and neighbour, for every slot of the
    // segments with affine faces, less the tables' 36 bytes per segment.
    double faceIndexSaving() const {
        if (!mesh_.ssegM) return 0.0;
        return 8.0 * W_ * 32.0 * (nSeg_ - segCounts_[1]) - 36.0 * nSeg_;
    }
    template <class T>
    double slotIndexBytes(const LevelT<T>& L) const {
        return L.seg ? meshSlotIndexBytes() : 4.0 * L.W * L.N;
    }
    template <class T>
    static double galerkinBytes(const LevelT<T>& f, const LevelT<T>& c) {
        return (double)f.N * ((double)sizeof(T) * (1.0 + f.W) + 4.0) + (12.0 + sizeof(T)) * c.totalSlots +
               (8.0 + sizeof(T)) * c.N;
    }
    template <class T>
    void enqueueGalerkinChain(const std::vector<LevelT<T>>& lv, int chain, const char* name, cudaStream_t st) {
        GalChainArgsT<T> a;
        const int L = (int)lv.size();
        a.count = L - chain + 1;
        double bytes = 0.0;
        for (int i = 0; i < a.count; i++) {
            a.lv[i] = lv[(size_t)chain - 1 + i];
            if (i > 0) bytes += galerkinBytes(a.lv[i - 1], a.lv[i]);
        }
        launchGalerkinChain<T>(ctl_, a, st);
        markL(name, chain, bytes);
    }

    // Mixed precision: every V-cycle is one refinement step on the FP64 system
    // (residual and update in FP64, the cycle for the correction in FP32).
    void enqueueMultigridMixed() {
        if (!galerkinForked_) enqueueGalerkin32(stream_);
        const int L = (int)levels_.size();
        const bool coarsest0 = hier_[0].isCoarsest();
        const int first = coarsest0 ? cmg_.linearSweep : cmg_.linearPreSweep;
        const bool firstSweep = first >= 1;
        const int cycles = cmg_.maxIter > 1 ? cmg_.maxIter : 1;
        for (int c = 0; c < cycles; c++) {
            std::vector<float*> cur((size_t)L), alt((size_t)L);
            for (int l = 0; l < L; l++) {
                cur[(size_t)l] = levels32_[(size_t)l].x;
                alt[(size_t)l] = levels32_[(size_t)l].xNew;
            }
            launchIRResidualPP(ctl_, levels_[0], r32pp_, cur[0], cmg_.weight, firstSweep ? 1 : 0, stream_);
            mark("ir_residual_pp", (double)N_ * (8.0 * W_ + 32.0 + 8.0) + slotIndexBytes(levels_[0]));
            // the cycle's last finest-level pass, when it is the fused
            // prolongation and sweep, also adds the correction to p'
            irUpdate_ = pp_;
            irUpdated_ = false;
            vcycleT<float>(levels32_, 0, cur, alt, firstSweep);
            irUpdate_ = nullptr;
            if (!irUpdated_) {
                launchIRUpdatePP(ctl_, N_, pp_, cur[0], stream_);
                mark("ir_update_pp", 20.0 * N_);
            }
        }
    }

    // Flexible CG on the FP64 p' system with one FP32 V-cycle (from zero) as the
    // preconditioner of each iteration; at most cmg_.maxIter iterations. Inside a
    // stream capture of a solve with a tolerance, iterations 1.. are the body of
    // a conditional WHILE node (two iterations per body, so the direction
    // buffers keep their parity), and the kernels of iterations past the
    // stopping point are never launched.
    void enqueuePressureFcg() {
        enqueueGalerkin32(stream_);
        curProlong_ = prolongScale_;
        const bool firstSweep = (hier_[0].isCoarsest() ? cmg_.linearSweep : cmg_.linearPreSweep) >= 1;
        const int iters = cmg_.maxIter > 1 ? cmg_.maxIter : 1;
        const int nextSweep = firstSweep ? 2 : 1;
        const double vb = 4.0;
        launchFcgInit(ctl_, levels_[0], pp_, fcgR_, r32pp_, levels32_[0].x, cmg_.weight, firstSweep ? 1 : 0,
                      psolveTol_, fcg_, stream_);
        mark("fcg_init", (double)N_ * (12.0 * W_ + 8.0 + 8.0 + 8.0 + 8.0 + vb + (firstSweep ? vb : 0.0)));
        const bool useNet = learnedMode_ != AXISIM_LEARNED_OFF && net_.ready();
        fcgIteration(0, iters > 1 ? nextSweep : 1, iters, firstSweep, useNet);
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        CK(cudaStreamIsCapturing(stream_, &cap));
        // the loop pays (two kernels per body, one edge without overlap) only
        // where a solve can stop before its cap: a tolerance and a cap of 8 or more
        if (iters >= 8 && psolveTol_ > 0.0 && cap == cudaStreamCaptureStatusActive) {
            cudaGraph_t g = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nDeps = 0;
            cudaGraphConditionalHandle h;
            CK(cudaStreamGetCaptureInfo(stream_, &cap, nullptr, &g, &deps, &nDeps));
            CK(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
            const int maxBodies = iters / 2;  // iterations 1 .. iters-1, two per body
            launchFcgLoop(ctl_, fcg_, h, 1, maxBodies, stream_);
            CK(cudaStreamGetCaptureInfo(stream_, &cap, nullptr, &g, &deps, &nDeps));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            CK(cudaGraphAddNode(&node, g, deps, nDeps, &cp));
            CK(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
            if (!loopStream_) CK(cudaStreamCreateWithFlags(&loopStream_, cudaStreamNonBlocking));
            CK(cudaStreamBeginCaptureToGraph(loopStream_, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
            std::swap(stream_, loopStream_);
            try {
                tNextLaunchPlain = true;
                fcgIteration(1, nextSweep, iters, firstSweep, false);
                fcgIteration(2, nextSweep, iters, firstSweep, false);
                launchFcgLoop(ctl_, fcg_, h, 0, maxBodies, stream_);
            } catch (...) {
                std::swap(stream_, loopStream_);
                cudaGraph_t body = nullptr;
                cudaStreamEndCapture(loopStream_, &body);
                tNextLaunchPlain = false;
                throw;
            }
            std::swap(stream_, loopStream_);
            cudaGraph_t body = nullptr;
            CK(cudaStreamEndCapture(loopStream_, &body));
            tNextLaunchPlain = true;
        } else {
            for (int it = 1; it < iters; it++) fcgIteration(it, it + 1 < iters ? nextSweep : 1, iters, firstSweep, false);
        }
        launchFcgEnd(ctl_, fcg_, useNet ? netStats_ : nullptr, stream_);
        mark("fcg_end", 0.0);
        curProlong_ = 1.0;
    }

    // Krylov iteration `it` (its parity picks the direction buffers; 0 starts
    // the directions and, with netStep, may take the learned step): V-cycle(r),
    // dots, direction and A p, update of x and r.
    void fcgIteration(int it, int next, int iters, bool firstSweep, bool netStep) {
        const int L = (int)levels_.size();
        const double vb = 4.0;
        std::vector<float*> cur((size_t)L), alt((size_t)L);
        for (int l = 0; l < L; l++) {
            cur[(size_t)l] = levels32_[(size_t)l].x;
            alt[(size_t)l] = levels32_[(size_t)l].xNew;
        }
        // with the network, the gate picks the learned preconditioner
        // z = alpha y + V-cycle(r - alpha A y), y = network(r), whose kernels run
        // while ppSkip == 2, or the plain V-cycle
        if (netStep) {
            launchFcgGate(ctl_, netStats_, learnedMode_ == AXISIM_LEARNED_ALWAYS ? 1 : 0, stream_);
            net_.infer(ctl_, 1, fcgR_, ACpp_, AFpp_, mesh_.snb, W_, nnY_, stream_);
            mark("nn_infer", 0.0);
            launchNnResidual(ctl_, levels_[0], fcgR_, nnY_, nnAy_, fcg_, r32pp_, levels32_[0].x, cmg_.weight,
                             firstSweep ? 1 : 0, stream_);
            mark("nn_residual", (double)N_ * (12.0 * W_ + 8.0 + 4.0 * W_ + 8.0 + 8.0 + 8.0 + 8.0 + 4.0 + 4.0));
            launchFcgUngate(ctl_, stream_);
        }
        vcycleT<float>(levels32_, 0, cur, alt, firstSweep);
        const float* e = cur[0];
        if (netStep) {
            launchNnCombine(ctl_, netStats_, N_, nnY_, fcg_, cur[0], stream_);
            mark("nn_combine", 12.0 * N_);
        }
        launchFcgDots(ctl_, N_, e, fcgR_, fcgQ_, it > 0 ? 1 : 0, fcg_, stream_);
        mark("fcg_dots", (double)N_ * (vb + 8.0 + (it > 0 ? 8.0 : 0.0)));
        double* pOld = fcgP_[(it + 1) & 1];
        double* pNew = fcgP_[it & 1];
        const int pqOld = 2 + ((it + 1) & 1), pqNew = 2 + (it & 1);
        launchFcgSpmv(ctl_, levels_[0], e, pOld, pNew, fcgQ_, it == 0 ? 1 : 0, pqOld, pqNew, fcg_, stream_);
        mark("fcg_spmv", (double)N_ * (12.0 * W_ + 8.0 + vb + (it > 0 ? 8.0 : 0.0) + 16.0));
        launchFcgUpdate(ctl_, levels_[0], pp_, fcgR_, pNew, fcgQ_, fcg_, pqNew, r32pp_, levels32_[0].x, cmg_.weight,
                        next, psolveTol_, iters, stream_);
        mark("fcg_update", (double)N_ * (24.0 + 24.0 + vb + (next > 1 ? 8.0 + vb : 0.0)));
    }

    void enqueueMultigrid() {
        if (psolve_ == AXISIM_PSOLVE_FCG) {
            enqueuePressureFcg();
            return;
        }
        if (precision_ == AXISIM_PREC_MIXED) {
            enqueueMultigridMixed();
            return;
        }
        const int L = (int)levels_.size();
        if (!galerkinForked_) enqueueGalerkin64(stream_);
        std::vector<double*> cur((size_t)L), alt((size_t)L);
        for (int l = 0; l < L; l++) {
            cur[(size_t)l] = levels_[(size_t)l].x;
            alt[(size_t)l] = levels_[(size_t)l].xNew;
        }
        const int cycles = cmg_.maxIter > 1 ? cmg_.maxIter : 1;
        for (int c = 0; c < cycles; c++) vcycleT<double>(levels_, 0, cur, alt, false);
        if (cur[0] != pp_) {
            launchCopy(ctl_, pp_, cur[0], N_, stream_);
            mark("copy", 16.0 * N_);
        }
    }

    // The linear solver of one system (LinearSolver::run); `tag` names its
    // launches in the profile ("pp" or the scalar's).
    void enqueueLinear(double* x, double* xT, const double* AF, const double* b, const double* inv,
                       const char* tag = "pp") {
        const int iters = cs_.linearMaxIter;
        if (cs_.type == 1 && colorN_ > 0) {
            for (int k = 0; k < iters; k++)
                for (int c = 0; c < colorN_; c++) {
                    const int b0 = hColorStart_[(size_t)c], cnt = hColorStart_[(size_t)c + 1] - b0;
                    if (cnt > 0) {
                        launchGaussSeidel1(mesh_, ctl_, AF, b, inv, x, dCellOrder_, b0, cnt, stream_);
                        mark((std::string("gs_") + tag).c_str(), (double)cnt * (12.0 * W_ + 28.0));
                    }
                }
            return;
        }
        double *live = x, *spare = xT;
        for (int k = 0; k < iters; k++) {
            launchJacobi1(mesh_, ctl_, AF, b, inv, live, spare, stream_);
            mark((std::string("jacobi_") + tag).c_str(), (double)N_ * (12.0 * W_ + 32.0));
            std::swap(live, spare);
        }
        if (live != x) {
            launchCopy(ctl_, x, live, N_, stream_);
            mark("copy", 16.0 * N_);
        }
    }

    // Boundary faces in a Michaelis-Menten or Hill group of a solved scalar,
    // ascending (uploaded with the scalar buffers; rebuilt when those are).
    void ensureWallFaces() {
        if (wallFacesReady_) return;
        std::vector<int32_t> list;
        std::vector<int32_t> grp((size_t)F_);
        CK(cudaMemcpy(grp.data(), mesh_.group, (size_t)F_ * sizeof(int32_t), cudaMemcpyDeviceToHost));
        for (int f = 0; f < F_; f++) {
            if (hNeighbor_[(size_t)f] >= 0) continue;
            const int g = grp[(size_t)f];
            bool reactive = false;
            for (int q = 0; q < 2; q++) {
                if (!solveS_[q] || g < 0 || g >= hbcS_[q].nGroups) continue;
                const uint8_t t = hbcS_[q].type[(size_t)g];
                reactive |= t == AXISIM_BC_MICHAELIS_MENTEN || t == AXISIM_BC_HILL;
            }
            if (reactive) list.push_back(f);
        }
        wallArena_.release();
        nWallFaces_ = (int)list.size();
        wallFaces_ = nWallFaces_ ? wallArena_.upload(list.data(), list.size()) : nullptr;
        wallFacesReady_ = true;
    }

    void enqueueIteration() {
        const int scheme = cs_.convectionScheme;
        const int conv = cs_.addConvectionTerm ? 1 : 0;
        const int nonOrtho = cs_.useNonOrthCorrector ? 1 : 0;
        const bool convNeedsGrad = conv && (scheme == 2 || scheme == 3);
        const int grad = cs_.gradientScheme;
        launchIterBegin(ctl_, hostStopDev_, stream_);
        mark("iter_begin", 0.0);
        // gradients of u, v (when SOU / non-orthogonal) and p in one pass; the
        // solved scalars' gradients join it: the reference takes them just
        // before each scalar's assembly (solver.cpp:1224-1226), and nothing
        // writes T or C between the start of the iteration and that point
        {
            const double* phi[5];
            BCDev bc[5];
            double* gz[5];
            double* gr[5];
            int nf = 0;
            if (nonOrtho || convNeedsGrad) {
                phi[nf] = u_; bc[nf] = bc_[0]; gz[nf] = gUZ_; gr[nf] = gUR_; nf++;
                phi[nf] = v_; bc[nf] = bc_[1]; gz[nf] = gVZ_; gr[nf] = gVR_; nf++;
            }
            phi[nf] = p_; bc[nf] = bc_[2]; gz[nf] = gPZ_; gr[nf] = gPR_; nf++;
            if (nonOrtho || convNeedsGrad)
                for (int q = 0; q < 2; q++)
                    if (solveS_[q]) {
                        phi[nf] = sb_[q].phi; bc[nf] = bcS_[q]; gz[nf] = sb_[q].gZ; gr[nf] = sb_[q].gR; nf++;
                    }
            launchGradient(mesh_, ctl_, nf, phi, bc, gz, gr, grad, stream_);
            mark("gradient", gradBytes(nf, grad) - (grad == 1 ? faceIndexSaving() : 0.0));
        }
        MomentumArgs a{};
        a.mDot = mDot_; a.u = u_; a.v = v_; a.gUZ = gUZ_; a.gUR = gUR_; a.gVZ = gVZ_; a.gVR = gVR_;
        a.gPZ = gPZ_; a.gPR = gPR_; a.uOld = uOld_; a.vOld = vOld_; a.uOld2 = uOld2_; a.vOld2 = vOld2_;
        a.AF = AFm_; a.ACu = ACu_; a.ACv = ACv_; a.bu = bu_; a.bv = bv_; a.invACu = iu_; a.invACv = iv_;
        a.DU = DU_; a.DV = DV_; a.mu = fluid_.mu; a.rho = fluid_.rho; a.dt = cs_.dt; a.alpha = alphaU_;
        a.conv = conv; a.scheme = (scheme == 3) ? 0 : scheme; a.nonOrtho = nonOrtho; a.transient = cs_.transient ? 1 : 0;
        const bool mixedMomentum = precision_ == AXISIM_PREC_MIXED && cs_.type != 1;
        a.AF32 = mixedMomentum ? AF32m_ : nullptr;
        a.invU32 = mixedMomentum ? iu32_ : nullptr;
        a.invV32 = mixedMomentum ? iv32_ : nullptr;
        launchMomentum(mesh_, ctl_, bc_[0], bc_[1], a, stream_);
        {
            double face = 32.0 + (scheme == 1 ? 8.0 : scheme == 2 ? 16.0 : 0.0);
            double cell = 4.0 * W_ + 16.0 + 16.0 + 16.0 + 8.0 * W_ + 64.0 + (scheme == 2 ? 40.0 : 0.0);
            if (cs_.transient) cell += 32.0;
            mark("momentum", face * F_ + cell * N_ - faceIndexSaving());
        }
        // momentum solves (LinearSolver::run for u then v; fused, identical arithmetic)
        const int iters = cs_.linearMaxIter;
        if (cs_.type == 1 && colorN_ > 0) {
            for (int k = 0; k < iters; k++)
                for (int c = 0; c < colorN_; c++) {
                    const int b0 = hColorStart_[(size_t)c], cnt = hColorStart_[(size_t)c + 1] - b0;
                    if (cnt > 0) {
                        launchGaussSeidelUV(mesh_, ctl_, AFm_, bu_, bv_, iu_, iv_, u_, v_, dCellOrder_, b0, cnt, stream_);
                        mark("gs_uv", (double)cnt * (12.0 * W_ + 52.0));
                    }
                }
        } else if (mixedMomentum) {
            // correction form: FP64 residual, FP32 Jacobi sweeps on the correction, FP64 update
            launchIRResidualUV(mesh_, ctl_, AFm_, ACu_, ACv_, bu_, bv_, u_, v_, iu32_, iv32_, ru32_, rv32_, du32_[0],
                               dv32_[0], stream_);
            mark("ir_residual_uv", (double)N_ * (8.0 * W_ + 64.0 + 24.0) + meshSlotIndexBytes());
            int c = 0;
            const int rest = iters - 1;
            if (tiles_.nTiles > 0 && rest > 1) {
                // the remaining sweeps in launches of at most S, as even as possible
                const int L = (rest + tiles_.S - 1) / tiles_.S;
                for (int q = 0; q < L; q++) {
                    const int k = rest / L + (q < rest % L ? 1 : 0);
                    launchJacobiUV32Tiles(mesh_, ctl_, tiles_, k, AF32m_, ru32_, rv32_, iu32_, iv32_, du32_[c],
                                          dv32_[c], du32_[1 - c], dv32_[1 - c], stream_);
                    mark("jacobi_uv32_tiles", (double)N_ * (4.0 * W_ + 32.0));
                    c = 1 - c;
                }
            } else {
                for (int k = 1; k < iters; k++) {
                    launchJacobiUV32(mesh_, ctl_, AF32m_, ru32_, rv32_, iu32_, iv32_, du32_[c], dv32_[c],
                                     du32_[1 - c], dv32_[1 - c], stream_);
                    mark("jacobi_uv32", (double)N_ * (4.0 * W_ + 32.0) + meshSlotIndexBytes());
                    c = 1 - c;
                }
            }
            launchIRUpdateUV(ctl_, N_, u_, v_, du32_[c], dv32_[c], stream_);
            mark("ir_update_uv", 40.0 * N_);
        } else {
            double *lu = u_, *su = uT_, *lv = v_, *sv = vT_;
            if (tiles_.nTiles > 0 && iters > 1) {
                const int L = (iters + tiles_.S - 1) / tiles_.S;
                for (int q = 0; q < L; q++) {
                    const int k = iters / L + (q < iters % L ? 1 : 0);
                    launchJacobiUVTiles(mesh_, ctl_, tiles_, k, AFm_, bu_, bv_, iu_, iv_, lu, lv, su, sv, stream_);
                    mark("jacobi_uv_tiles", (double)N_ * (8.0 * W_ + 64.0));
                    std::swap(lu, su);
                    std::swap(lv, sv);
                }
            } else {
                for (int k = 0; k < iters; k++) {
                    launchJacobiUV(mesh_, ctl_, AFm_, bu_, bv_, iu_, iv_, lu, lv, su, sv, stream_);
                    mark("jacobi_uv", (double)N_ * (8.0 * W_ + 64.0) + meshSlotIndexBytes());
                    std::swap(lu, su);
                    std::swap(lv, sv);
                }
            }
            if (lu != u_) {
                launchCopy(ctl_, u_, lu, N_, stream_);
                launchCopy(ctl_, v_, lv, N_, stream_);
                mark("copy", 32.0 * N_);
            }
        }
        const bool mixedPP = fp32PressureCycle();
        launchPressureSystem(mesh_, ctl_, bc_[0], bc_[1], bc_[2], fluid_.rho, u_, v_, p_, gPZ_, gPR_, DU_, DV_, AFpp_,
                             ACpp_, ipp_, mDot_, mixedPP ? AF32pp_ : nullptr, mixedPP ? AC32pp_ : nullptr, stream_);
        mark("pressure_rhiechow", 56.0 * F_ + (12.0 * W_ + 72.0) * N_ - faceIndexSaving());
        for (int corr = 0; corr <= nonOrtho; corr++) {
            const int cross = corr > 0;
            if (cross) {
                const double* phi[1] = {pp_};
                double* gz[1] = {gPZ_};
                double* gr[1] = {gPR_};
                launchGradient(mesh_, ctl_, 1, phi, &bc_[3], gz, gr, grad, stream_);
                mark("gradient_pp", gradBytes(1, grad) - (grad == 1 ? faceIndexSaving() : 0.0));
            }
            galerkinThisSolve_ = corr == 0;
            forkGalerkin();
            launchPressureRhs(mesh_, ctl_, fluid_.rho, mDot_, DU_, DV_, gPZ_, gPR_, cross, corr == 0, bpp_, pp_, stream_);
            mark("pp_rhs", 16.0 * F_ + (4.0 * W_ + 16.0) * N_ - faceIndexSaving());
            // the non-orthogonal corrector's pass solves the same p' operator
            // with a new right-hand side: its coarse operators are the ones
            // the first pass built
            if (cs_.useMultigrid) enqueueMultigrid();
            else enqueueLinear(pp_, ppT_, AFpp_, bpp_, ipp_);
            joinGalerkin((int)levels_.size() - 1);  // whatever the solve did not wait for
            galerkinForked_ = false;
            galerkinThisSolve_ = true;
        }
        if (harvestEvery_ > 0 && samples_) {
            launchHarvest(ctl_, N_, harvestEvery_, sampleCap_, bpp_, pp_, ACpp_, AFpp_, mesh_.snb, W_,
                          psolve_ == AXISIM_PSOLVE_FCG ? fcg_.scalars : nullptr, samples_, sampleCount_, sampleRelres_,
                          harvestCounter_, stream_);
            mark("harvest", 0.0);
        }
        {
            const double* phi[1] = {pp_};
            double* gz[1] = {gPZ_};
            double* gr[1] = {gPR_};
            launchGradient(mesh_, ctl_, 1, phi, &bc_[3], gz, gr, grad, stream_);
            mark("gradient_pp", gradBytes(1, grad) - (grad == 1 ? faceIndexSaving() : 0.0));
        }
        launchCorrect(mesh_, ctl_, bc_[2], fluid_.rho, alphaP_, nonOrtho, pp_, gPZ_, gPR_, DU_, DV_, u_, v_, p_, mDot_,
                      stream_);
        mark("correct_massflux", 64.0 * F_ + (88.0 + 4.0 * W_) * N_ - faceIndexSaving());
        // energy and concentration (solver.cpp:1218-1238): both assembled in one
        // pass (each system depends only on its own field, mDot and the mesh),
        // then each solved with the momentum linear solver
        int ns = 0, firstS = -1;
        for (int q = 0; q < 2; q++)
            if (solveS_[q]) {
                if (firstS < 0) firstS = q;
                ns++;
            }
        if (ns > 0) {
            ScalarArgs sa{};
            int k = 0;
            for (int q = 0; q < 2; q++) {
                if (!solveS_[q]) continue;
                ScalarDev& d = sa.s[k++];
                const ScalarBuf& b = sb_[q];
                d.bc = bcS_[q];
                // the names simple.tempOld / tempOld2 as they stood when the run
                // started (solver.cpp:985-1009 caches them before the time loop)
                d.phi = b.phi; d.gZ = b.gZ; d.gR = b.gR;
                d.old = b.lvl[graphSwapS_[q]];
                d.old2 = b.lvl[1 - graphSwapS_[q]];
                d.AF = b.AF; d.AC = b.AC; d.b = b.b; d.inv = b.inv; d.wall = b.wall;
                d.gamma = q == 0 ? fluid_.k / (fluid_.rho * fluid_.cp) : fluid_.D;
                d.alpha = q == 0 ? alphaU_ : 1.0;
            }
            sa.mDot = mDot_;
            sa.cw = cw_;
            sa.ocr = ocr_;
            sa.fluxScale = 1.0 / fluid_.rho;
            sa.dt = cs_.dt;
            sa.conv = conv;
            sa.scheme = (scheme == 3) ? 0 : scheme;
            sa.nonOrtho = nonOrtho;
            sa.transient = cs_.transient ? 1 : 0;
            if (nWallFaces_ > 0) {
                launchScalarWall(mesh_, ctl_, ns, sa, wallFaces_, nWallFaces_, stream_);
                mark("scalar_wall", 100.0 * nWallFaces_);
            }
            launchScalarAssembly(mesh_, ctl_, ns, sa, stream_);
            {
                double face = 32.0 + (scheme == 1 ? 8.0 : scheme == 2 ? 16.0 : 0.0);
                double cell = 4.0 * W_ + 16.0 + ns * (8.0 * W_ + 8.0 + 24.0 + (cs_.transient ? 16.0 : 0.0));
                mark("scalar", face * F_ + cell * N_);
            }
            // temperature's sweeps, then concentration's: each system's working
            // set stays in L2 across its own consecutive sweeps
            for (int q = 0; q < 2; q++)
                if (solveS_[q]) enqueueLinear(sb_[q].phi, sb_[q].tmp, sb_[q].AF, sb_[q].b, sb_[q].inv, q == 0 ? "T" : "C");
        }
        launchResiduals(mesh_, ctl_, AFm_, ACu_, ACv_, bu_, bv_, u_, v_, mDot_, resU_, resV_, resC_, scU_, scV_,
                        partial_, &residualBlocks_, stream_);
        mark("residual", 16.0 * F_ + (12.0 * W_ + 88.0) * N_ + meshSlotIndexBytes() - 16.0 * nSeg_ * (mesh_.sseg ? 1 : 0) -
                             faceIndexSaving());
        const bool monitorS = (solveS_[0] && sres_[0].enabled) || (solveS_[1] && sres_[1].enabled);
        if (monitorS) {
            const double* AF[2];
            const double* AC[2];
            const double* bb[2];
            const double* x[2];
            double* res[2];
            double* sc[2];
            int k = 0;
            for (int q = 0; q < 2; q++) {
                if (!solveS_[q]) continue;
                AF[k] = sb_[q].AF; AC[k] = sb_[q].AC; bb[k] = sb_[q].b; x[k] = sb_[q].phi;
                res[k] = sb_[q].res; sc[k] = sb_[q].scale;
                k++;
            }
            launchScalarResidual(mesh_, ctl_, ns, firstS, AF, AC, bb, x, res, sc, partialS_, stream_);
            mark("scalar_residual", ns * (8.0 * W_ + 48.0) * N_ + 4.0 * W_ * N_);
        }
        if (batch_.nCases > 0) {
            launchBatchIterEnd(ctl_, batch_, resU_, resV_, resC_, scU_, scV_, stream_);
            mark("batch_iter_end", 40.0 * N_);
        } else {
            launchIterEnd(ctl_, partial_, monitorS ? partialS_ : nullptr, residualBlocks_, N_, stream_);
            mark("iter_end", 40.0 * residualBlocks_);
        }
    }

    // Algorithmic bytes of one gradient launch: every array element counted once.
    double gradBytes(int nf, int scheme) const {
        const double face = scheme == 1 ? 24.0 : 48.0;
        const double cell = 4.0 * W_ + 8.0 * nf + (scheme == 1 ? 24.0 : 8.0) + 16.0 * nf;
        return face * F_ + cell * N_;
    }

public:
    // Runs `iters` SIMPLE iterations eagerly from the current state with an
    // event after every launch; returns per-kernel launches, time and bytes.
    int profile(int iters, axisim_kernel_stat* out, int maxOut, bool byLevel = false) {
        if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
        uploadBC();
        buildGraph();
        Ctl h;
        CK(cudaMemcpy(&h, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost));
        const Ctl saved = h;
        h.done = 0;
        h.k = 0;
        h.maxIter = 1 << 30;
        h.checkConv = std::max(1, csim_.checkConv);
        h.transient = cs_.transient ? 1 : 0;
        for (int i = 0; i < 3; i++) {
            h.tol[i] = -1.0;  // never converges: every profiled iteration runs in full
            h.resNorm[i] = cres_[i].normType;
            h.resScale[i] = cres_[i].scaleType;
            h.resEnabled[i] = cres_[i].enabled;
        }
        for (int q = 0; q < 2; q++) {
            h.tolS[q] = -1.0;
            h.resNormS[q] = sres_[q].normType;
            h.resScaleS[q] = sres_[q].scaleType;
            h.resEnabledS[q] = sres_[q].enabled;
            h.solvedS[q] = solveS_[q];
        }
        CK(cudaMemcpyAsync(ctl_, &h, sizeof(Ctl), cudaMemcpyHostToDevice, stream_));
        CK(cudaStreamSynchronize(stream_));
        profiling_ = true;
        profileByLevel_ = byLevel;
        marks_.clear();
        cudaEvent_t start;
        CK(cudaEventCreate(&start));
        CK(cudaEventRecord(start, stream_));
        try {
            for (int i = 0; i < iters; i++) enqueueIteration();
        } catch (...) {
            profiling_ = false;
            profileByLevel_ = false;
            throw;
        }
        profiling_ = false;
        profileByLevel_ = false;
        CK(cudaStreamSynchronize(stream_));
        std::vector<axisim_kernel_stat> acc;
        cudaEvent_t prev = start;
        for (Mark& m : marks_) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, prev, m.ev));
            auto it = std::find_if(acc.begin(), acc.end(),
                                   [&](const axisim_kernel_stat& s) { return m.name == s.name; });
            if (it == acc.end()) {
                axisim_kernel_stat s{};
                std::snprintf(s.name, sizeof(s.name), "%s", m.name.c_str());
                acc.push_back(s);
                it = acc.end() - 1;
            }
            it->launches++;
            it->ms += ms;
            it->bytes += m.bytes;
            prev = m.ev;
        }
        for (Mark& m : marks_) cudaEventDestroy(m.ev);
        marks_.clear();
        cudaEventDestroy(start);
        // restore the run's control block (iteration counters advanced by the profiled iterations)
        Ctl after;
        CK(cudaMemcpy(&after, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost));
        Ctl restored = saved;
        restored.currentIteration = after.currentIteration;
        CK(cudaMemcpy(ctl_, &restored, sizeof(Ctl), cudaMemcpyHostToDevice));
        const int n = (int)acc.size();
        for (int i = 0; i < n && i < maxOut; i++) out[i] = acc[(size_t)i];
        return n;
    }

private:
    // Launch-shape autotuner: for every level the V-cycle launches kernels on
    // (the tail's levels run inside one CTA and are skipped), time the weighted
    // Jacobi sweep at each candidate block size and keep pickBlock's choice in
    // LevelT::block, which the level's smoothing, residual, restriction and
    // prolongation launches use. The sweeps run on scratch inputs (unit
    // diagonal, zero right-hand side and iterate, a zeroed control block), so
    // the solution and the level's own vectors are untouched; only the sparsity
    // pattern and coefficient storage are the level's.
    static constexpr int kTuneCandidates[3] = {64, 128, 256};
    template <class T>
    void tuneLevels(std::vector<LevelT<T>>& lv) {
        const int L = (int)lv.size();
        const int upto = tailStart_ > 0 ? std::min(tailStart_, L) : L;
        int nMax = 1;
        for (int l = 0; l < upto; l++) nMax = std::max(nMax, lv[(size_t)l].N);
        Arena scratch;
        Ctl* ctl = scratch.alloc<Ctl>(1);
        const std::vector<T> ones((size_t)nMax, T(1));
        T* ac = scratch.upload(ones.data(), ones.size());
        T* b = scratch.alloc<T>((size_t)nMax);
        T* x = scratch.alloc<T>((size_t)nMax);
        T* y = scratch.alloc<T>((size_t)nMax);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        const std::vector<int> cand(std::begin(kTuneCandidates), std::end(kTuneCandidates));
        const int nc = (int)cand.size(), def = nc - 1, reps = 8;
        tuneUs_.assign((size_t)L * nc, 0.0);
        try {
            for (int l = 0; l < upto; l++) {
                LevelT<T> t = lv[(size_t)l];
                t.AC = ac;
                t.b = b;
                std::vector<double> us((size_t)nc, 0.0);
                for (int c = 0; c < nc; c++) {
                    t.block = cand[(size_t)c];
                    for (int r = 0; r < 2; r++) launchMGSmooth<T>(ctl, t, x, y, (T)cmg_.weight, stream_);
                    CK(cudaEventRecord(e0, stream_));
                    for (int r = 0; r < reps; r++) launchMGSmooth<T>(ctl, t, x, y, (T)cmg_.weight, stream_);
                    CK(cudaEventRecord(e1, stream_));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    us[(size_t)c] = 1e3 * (double)ms / reps;
                    tuneUs_[(size_t)l * nc + c] = us[(size_t)c];
                }
                lv[(size_t)l].block = cand[(size_t)pickBlock(cand, us, def, 0.03)];
            }
            CK(cudaGetLastError());
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            for (auto& v : lv) v.block = 0;
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }

public:
    void testBarrierTimeout(int on) { barrierPhantom_ = on ? 1 : 0; }
    void setMomentumSweeps(int sweepsPerLaunch, int threads) {
        if (sweepsPerLaunch < 1 || sweepsPerLaunch > kMaxSweepsPerLaunch)
            throw StatusError(AXISIM_E_ARG, "sweeps per launch must be 1..8");
        if (threads != 0 && threads != 256 && threads != 512 && threads != 1024)
            throw StatusError(AXISIM_E_ARG, "sweep CTA size must be 256, 512 or 1024 (0: default)");
        sweepsPerLaunch_ = sweepsPerLaunch;
        sweepThreads_ = threads ? threads : 1024;
        dropSweepTiles();
        destroyGraph();
    }
    int tileCount() const { return tiles_.nTiles; }

    void setVcycleKernel(int mode) {
        if (mode != AXISIM_VCYCLE_PER_PHASE && mode != AXISIM_VCYCLE_RESIDENT)
            throw StatusError(AXISIM_E_ARG, "V-cycle kernel mode must be 0 (one launch per phase) or 1 (resident)");
        residentVcycle_ = mode;
        destroyGraph();
    }
    void setAutotune(int on) {
        autotune_ = on ? 1 : 0;
        destroyGraph();
        for (auto& v : levels_) v.block = 0;
        for (auto& v : levels32_) v.block = 0;
        tuneUs_.clear();
    }
    // Block size per level of the set the V-cycle uses (0: not tuned, or a
    // tail level) and, with us, the measured sweep time per candidate.
    int autotuneReport(int32_t* blocks, double* us, int maxL) const {
        const bool f32 = fp32PressureCycle();
        const int L = f32 ? (int)levels32_.size() : (int)levels_.size();
        const int nc = (int)(sizeof(kTuneCandidates) / sizeof(int));
        for (int l = 0; l < L && l < maxL; l++) {
            if (blocks) blocks[l] = f32 ? levels32_[(size_t)l].block : levels_[(size_t)l].block;
            for (int c = 0; c < nc && us; c++)
                us[(size_t)l * nc + c] = (size_t)l * nc + c < tuneUs_.size() ? tuneUs_[(size_t)l * nc + c] : 0.0;
        }
        return L;
    }

private:
    void buildGraph() {
        if (exec_) return;
        ensureScalarBuffers();
        if (solveS_[0] || solveS_[1]) ensureWallFaces();  // host copies: before the capture
        if (cs_.useMultigrid) ensureDeviceLevels();
        ensureMixedBuffers();
        if (cs_.useMultigrid && psolve_ == AXISIM_PSOLVE_FCG) ensureNetStats();
        if (cs_.type == 1) ensureColoring();
        ensureSweepTiles();
        if (autotune_ && cs_.useMultigrid) {  // launch shapes are fixed in the graph: tune first
            if (fp32PressureCycle()) {
                if (!levels32_.empty() && levels32_[0].block == 0) tuneLevels(levels32_);
            } else if (!levels_.empty() && levels_[0].block == 0) {
                tuneLevels(levels_);
            }
        }
        std::unique_ptr<PhaseTimer> ph(new PhaseTimer(*this, "graph_capture"));
        CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            enqueueIteration();
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        CK(cudaStreamEndCapture(stream_, &graph_));
        ph.reset(new PhaseTimer(*this, "graph_instantiate"));
        CK(cudaGraphInstantiate(&exec_, graph_, 0));
        ph.reset(new PhaseTimer(*this, "graph_upload"));
        CK(cudaGraphUpload(exec_, stream_));
        CK(cudaStreamSynchronize(stream_));
    }

    void zeroState() {
        const size_t N = (size_t)N_;
        double* fields[] = {u_, v_, p_, pp_, uT_, vT_, ppT_, DU_, DV_, gPZ_, gPR_, gUZ_, gUR_, gVZ_, gVR_,
                            uOld_, vOld_, uOld2_, vOld2_};
        for (double* f : fields) CK(cudaMemsetAsync(f, 0, N * sizeof(double), stream_));
        for (int q = 0; q < 2; q++) {
            ScalarBuf& b = sb_[q];
            double* sf[] = {b.phi, b.tmp, b.lvl[0], b.lvl[1], b.gZ, b.gR};
            for (double* f : sf)
                if (f) CK(cudaMemsetAsync(f, 0, N * sizeof(double), stream_));
            b.swapped = 0;  // allocateSimple hands out fresh tempOld / tempOld2
        }
        if (cw_) {
            CK(cudaMemsetAsync(cw_, 0, (size_t)F_ * sizeof(double), stream_));
            CK(cudaMemsetAsync(ocr_, 0, (size_t)F_ * sizeof(double), stream_));
        }
        CK(cudaMemsetAsync(mDot_, 0, (size_t)F_ * sizeof(double), stream_));
        CK(cudaMemsetAsync(ctl_, 0, sizeof(Ctl), stream_));
    }

    friend int64_t getFieldImpl(const Solver&, const std::string&, double*, size_t);
};

int Solver::solve(int continueRun, axisim_result* res) {
    if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "set a mesh before solving");
    for (int v = 0; v < 3; v++)
        if (!haveBC_[v]) throw StatusError(AXISIM_E_STATE, "set boundary conditions for u, v and p before solving");
    for (int q = 0; q < 2; q++)
        if (solveS_[q] && !haveBCS_[q])
            throw StatusError(AXISIM_E_STATE, q == 0 ? "set boundary conditions for T before solving energy"
                                                     : "set boundary conditions for C before solving concentration");
    if (batch_.nCases > 0 && ((solveS_[0] && sres_[0].enabled) || (solveS_[1] && sres_[1].enabled)))
        throw StatusError(AXISIM_E_CONFIG, "a batch monitors U, V and Continuity only; disable the scalar residuals");
    // Solver::runCheck (solver.cpp:530-661)
    if (running_) throw StatusError(AXISIM_E_STATE, "Solver still running");
    if (csim_.maxIter < 1) csim_.maxIter = 50;
    if (csim_.checkConv < 1) csim_.checkConv = 1;
    if (cs_.linearMaxIter < 1) cs_.linearMaxIter = 20;
    if (cs_.saveKeyFrameIter < 1) cs_.saveKeyFrameIter = 1;
    // a structured mesh is orthogonal by construction: no corrector (solver.cpp:548-555)
    if (meshType_ == AXISIM_MESH_STRUCTURED && cs_.useNonOrthCorrector) {
        cs_.useNonOrthCorrector = 0;
        destroyGraph();
    }
    const bool transient = cs_.transient != 0;
    if (transient) {
        if (!std::isfinite(cs_.dt) || cs_.dt <= 0.0) throw StatusError(AXISIM_E_CONFIG, "Transient run needs a positive time step.");
        if (!std::isfinite(cs_.tEnd) || cs_.tEnd <= 0.0) throw StatusError(AXISIM_E_CONFIG, "Transient run needs a positive end time.");
    }
    bool anyPuls = false;
    for (int var = 0; var < 2; var++) {
        const HostBC& h = hbc_[var];
        for (int g = 0; g < h.nGroups; g++) {
            if (!h.puls[(size_t)g]) continue;
            anyPuls = true;
            if (!std::isfinite(h.value[(size_t)g]) || !std::isfinite(h.amp[(size_t)g]) || h.amp[(size_t)g] < 0.0 ||
                !std::isfinite(h.freq[(size_t)g]) || h.freq[(size_t)g] <= 0.0)
                throw StatusError(AXISIM_E_CONFIG, "Pulsatile inlet needs a finite mean velocity, A >= 0, and f > 0 Hz.");
        }
    }
    if (anyPuls && !transient) throw StatusError(AXISIM_E_CONFIG, "Pulsatile inlet requires Transient Solver to be enabled.");
    if (!std::isfinite(fluid_.rho) || !std::isfinite(fluid_.mu) || fluid_.rho <= 0.0 || fluid_.mu <= 0.0)
        throw StatusError(AXISIM_E_CONFIG, "Solver needs positive density and viscosity.");
    if (solveS_[0] && !(std::isfinite(fluid_.cp) && std::isfinite(fluid_.k) && fluid_.cp > 0.0 && fluid_.k >= 0.0))
        throw StatusError(AXISIM_E_CONFIG, "Energy equation needs a positive heat capacity and a conductivity >= 0.");
    if (solveS_[1] && !(std::isfinite(fluid_.D) && fluid_.D >= 0.0))
        throw StatusError(AXISIM_E_CONFIG, "Concentration equation needs a mass diffusivity >= 0.");
    bool cont = continueRun != 0;
    timedOut_ = false;
    if (cont) {
        std::string why;
        if (!canContinue(&why)) {
            log("Continue Solver disabled: " + why + " Starting from a fresh solve.\n");
            cont = false;
        }
    }
    uploadBC();
    ensureScalarBuffers();
    running_ = true;
    struct Guard {
        std::atomic<bool>& r;
        ~Guard() { r = false; }
    } guard{running_};
    *hostStop_ = 0;
    if (!cont) {
        PhaseTimer ph(*this, "zero_state");
        zeroState();
        simTime_ = 0.0;
        if (batch_.nCases > 0) {
            std::vector<int32_t> neg((size_t)batch_.nCases, -1);
            CK(cudaMemcpyAsync(batch_.convergedAt, neg.data(), neg.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                               stream_));
            CK(cudaMemsetAsync(batch_.scaleVal, 0, sizeof(double) * 3 * (size_t)batch_.nCases, stream_));
            CK(cudaStreamSynchronize(stream_));
        }
    }
    // the scalar step reads the time levels through the names tempOld /
    // tempOld2 as they stand at the start of the run (solver.cpp:985-1009)
    bool regraph = false;
    for (int q = 0; q < 2; q++)
        if (graphSwapS_[q] != sb_[q].swapped) {
            graphSwapS_[q] = sb_[q].swapped;
            regraph = true;
        }
    if (regraph) destroyGraph();
    buildGraph();
    // control block: settings for this run
    Ctl h;
    CK(cudaMemcpyAsync(&h, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    h.maxIter = csim_.maxIter;
    h.checkConv = csim_.checkConv;
    h.transient = transient ? 1 : 0;
    h.itersThisCall = 0;
    h.mgPhantom = barrierPhantom_;
    for (int i = 0; i < 3; i++) {
        h.tol[i] = cres_[i].tol;
        h.resNorm[i] = cres_[i].normType;
        h.resScale[i] = cres_[i].scaleType;
        h.resEnabled[i] = cres_[i].enabled;
    }
    for (int q = 0; q < 2; q++) {
        h.tolS[q] = sres_[q].tol;
        h.resNormS[q] = sres_[q].normType;
        h.resScaleS[q] = sres_[q].scaleType;
        h.resEnabledS[q] = sres_[q].enabled;
        h.solvedS[q] = solveS_[q];
    }
    const double timeOffset = (transient && cont) ? simTime_ : 0.0;
    const int numSteps = transient ? (int)std::ceil(cs_.tEnd / cs_.dt) : 1;
    const bool bdf2 = transient && cs_.timeScheme == 1;
    std::unique_ptr<PhaseTimer> ph(new PhaseTimer(*this, "solve_iterations"));
    CK(cudaEventRecord(ev0_, stream_));
    int stepsDone = 0;
    int status = AXISIM_OK;
    int totalIters = 0;
    bool converged = false;
    for (int t = 0; t < numSteps; t++) {
        if (transient) {
            const double stepTime = timeOffset + (double)(t + 1) * cs_.dt;
            for (int var = 0; var < 2; var++) {
                const HostBC& hb = hbc_[var];
                bool any = false;
                for (int g = 0; g < hb.nGroups; g++) {
                    double val = hb.value[(size_t)g];
                    if (hb.puls[(size_t)g]) {
                        any = true;
                        const double twoPi = 2.0 * 3.14159265358979323846;
                        val = hb.value[(size_t)g] * (1.0 + hb.amp[(size_t)g] * std::sin(twoPi * hb.freq[(size_t)g] * stepTime));
                    }
                    hostBCStage_[(size_t)var * std::max(std::max(hbc_[0].nGroups, hbc_[1].nGroups), 1) + (size_t)g] = val;
                }
                if (any) {
                    // the previous step's kernels have finished (we synchronised below)
                    CK(cudaMemcpy(bcValueDev_[var],
                                  hostBCStage_ + (size_t)var * std::max(std::max(hbc_[0].nGroups, hbc_[1].nGroups), 1),
                                  sizeof(double) * (size_t)hb.nGroups, cudaMemcpyHostToDevice));
                }
            }
            if (bdf2) {
                CK(cudaMemcpyAsync(uOld2_, uOld_, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
                CK(cudaMemcpyAsync(vOld2_, vOld_, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
            }
            CK(cudaMemcpyAsync(uOld_, u_, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
            CK(cudaMemcpyAsync(vOld_, v_, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
            for (int q = 0; q < 2; q++) {  // solver.cpp:1076-1095: swap the names, copy into tempOld
                if (!solveS_[q]) continue;
                ScalarBuf& b = sb_[q];
                if (bdf2) b.swapped ^= 1;
                CK(cudaMemcpyAsync(b.old(), b.phi, (size_t)N_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
            }
        }
        h.done = 0;
        h.k = 0;
        h.bdf2 = (bdf2 && t > 0) ? 1 : 0;
        h.converged = 0;
        h.histCount = 0;
        const int startIters = h.itersThisCall;
        CK(cudaMemcpyAsync(ctl_, &h, sizeof(Ctl), cudaMemcpyHostToDevice, stream_));
        int batch = 4;
        int launched = 0;
        int drained = 0;
        for (;;) {
            const int nb = std::min(batch, std::max(1, csim_.maxIter - launched + 1));
            for (int i = 0; i < nb; i++) CK(cudaGraphLaunch(exec_, stream_));
            launched += nb;
            CK(cudaMemcpyAsync(&h, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            if (resFn) {
                for (int q = drained; q < h.histCount; q++) {
                    const double* e = h.hist[q % kMaxHist];
                    resFn(cbCtx, (int32_t)e[0], e + 1);  // U, V, Continuity, Temperature, Concentration
                }
            }
            drained = h.histCount;
            if (h.done) break;
            batch = std::min(batch * 2, 64);
        }
        totalIters += h.itersThisCall - startIters;
        converged = h.converged != 0;
        stepsDone++;
        if (transient) simTime_ = timeOffset + (double)(t + 1) * cs_.dt;
        if (h.done == 2) {
            status = AXISIM_E_STOPPED;
            break;
        }
        if (h.done == 4) {
            status = AXISIM_E_DIVERGED;
            break;
        }
        if (h.done == 5) {
            status = AXISIM_E_TIMEOUT;
            timedOut_ = true;
            break;
        }
    }
    CK(cudaEventRecord(ev1_, stream_));
    ph.reset(new PhaseTimer(*this, "solve_final_gradients"));
    // final gradients of u, v, p for the solution fields (solver.cpp:1330-1332)
    {
        const double* phi[3] = {u_, v_, p_};
        double* gz[3] = {gUZ_, gVZ_, gPZ_};
        double* gr[3] = {gUR_, gVR_, gPR_};
        BCDev bc[3] = {bc_[0], bc_[1], bc_[2]};
        launchGradient(mesh_, nullptr, 3, phi, bc, gz, gr, cs_.gradientScheme, stream_);
    }
    // and of the solved scalars (solver.cpp:1334-1336)
    for (int q = 0; q < 2; q++) {
        if (!solveS_[q]) continue;
        const double* phi[1] = {sb_[q].phi};
        double* gz[1] = {sb_[q].gZ};
        double* gr[1] = {sb_[q].gR};
        launchGradient(mesh_, nullptr, 1, phi, &bcS_[q], gz, gr, cs_.gradientScheme, stream_);
    }
    ranS_[0] = solveS_[0];
    ranS_[1] = solveS_[1];
    lastResS_[0] = h.resValS[0];
    lastResS_[1] = h.resValS[1];
    CK(cudaStreamSynchronize(stream_));
    CK(cudaGetLastError());
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
    isReady_ = true;
    if (res) {
        res->iterations = totalIters;
        res->totalIterations = h.currentIteration;
        res->converged = converged ? 1 : 0;
        res->timeSteps = stepsDone;
        for (int i = 0; i < 3; i++) res->residual[i] = h.resVal[i];
        res->solveMs = ms;
    }
    if (status == AXISIM_E_STOPPED) lastError = "Solver stopped by user";
    if (status == AXISIM_E_TIMEOUT) lastError = "a grid-wide barrier of the resident multigrid kernel gave up waiting";
    if (status == AXISIM_E_DIVERGED) lastError = "non-finite residual: the solve diverged";
    return status;
}

// Field access (Solver::createSolutions, solver.cpp:186-219, plus internals).
int64_t Solver::getField(const std::string& name, double* out, size_t n) const {
    if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
    const size_t N = (size_t)N_, F = (size_t)F_, S = (size_t)S_;
    struct E {
        const char* n;
        const double* p;
        size_t len;
        int ell;
    };
    const E tab[] = {
        {"u", u_, N, 0}, {"v", v_, N, 0}, {"p", p_, N, 0}, {"pp", pp_, N, 0}, {"mDot", mDot_, F, 0},
        {"DU", DU_, N, 0}, {"DV", DV_, N, 0}, {"gradPZ", gPZ_, N, 0}, {"gradPR", gPR_, N, 0},
        {"gradUZ", gUZ_, N, 0}, {"gradUR", gUR_, N, 0}, {"gradVZ", gVZ_, N, 0}, {"gradVR", gVR_, N, 0},
        {"AC_u", ACu_, N, 0}, {"b_u", bu_, N, 0}, {"AF_u", AFm_, S, 1}, {"invAC_u", iu_, N, 0},
        {"AC_v", ACv_, N, 0}, {"b_v", bv_, N, 0}, {"AF_v", AFm_, S, 1}, {"invAC_v", iv_, N, 0},
        {"AC_pp", ACpp_, N, 0}, {"b_pp", bpp_, N, 0}, {"AF_pp", AFpp_, S, 1}, {"invAC_pp", ipp_, N, 0},
        {"res_U", resU_, N, 0}, {"res_V", resV_, N, 0}, {"res_Continuity", resC_, N, 0},
        {"uOld", uOld_, N, 0}, {"vOld", vOld_, N, 0}, {"uOld2", uOld2_, N, 0}, {"vOld2", vOld2_, N, 0},
        {"invDPN", mesh_.invDPN, F, 0}, {"wP", mesh_.wP, F, 0}, {"dPB", mesh_.dPB, F, 0},
        {"length2D", mesh_.length2D, F, 0}, {"lsqWZ", mesh_.lsqWZ, F, 0}, {"lsqWR", mesh_.lsqWR, F, 0},
        {"invA2D", mesh_.invA2D, N, 0}, {"lsqInvZZ", mesh_.lsqIZZ, N, 0}, {"lsqInvZR", mesh_.lsqIZR, N, 0},
        {"lsqInvRR", mesh_.lsqIRR, N, 0},
        // transported scalars (null until the scalar is solved)
        {"T", sb_[0].phi, N, 0}, {"gradTZ", sb_[0].gZ, N, 0}, {"gradTR", sb_[0].gR, N, 0},
        {"AC_T", sb_[0].AC, N, 0}, {"b_T", sb_[0].b, N, 0}, {"AF_T", sb_[0].AF, S, 1}, {"invAC_T", sb_[0].inv, N, 0},
        {"TOld", sb_[0].old(), N, 0}, {"TOld2", sb_[0].old2(), N, 0}, {"res_T", sb_[0].res, N, 0},
        {"C", sb_[1].phi, N, 0}, {"gradCZ", sb_[1].gZ, N, 0}, {"gradCR", sb_[1].gR, N, 0},
        {"AC_C", sb_[1].AC, N, 0}, {"b_C", sb_[1].b, N, 0}, {"AF_C", sb_[1].AF, S, 1}, {"invAC_C", sb_[1].inv, N, 0},
        {"COld", sb_[1].old(), N, 0}, {"COld2", sb_[1].old2(), N, 0}, {"res_C", sb_[1].res, N, 0},
        {"cw", cw_, F, 0}, {"ocrWall", ocr_, F, 0},
    };
    if (name == "continuity") {
        // Solver::getMassImbalance (solver.cpp:298-331): per-cell net outflow
        // of the final face mass fluxes.
        if (!out || n < N) throw StatusError(AXISIM_E_ARG, "output buffer too small for continuity");
        CK(cudaStreamSynchronize(stream_));
        std::vector<double> md(F);
        CK(cudaMemcpy(md.data(), mDot_, F * sizeof(double), cudaMemcpyDeviceToHost));
        for (int c = 0; c < N_; c++) {
            double imb = 0.0;
            for (int k = hCfs_[(size_t)c]; k < hCfs_[(size_t)c + 1]; k++) {
                const int f = hCfi_[(size_t)k];
                if (hOwner_[(size_t)f] == c) imb += md[(size_t)f];
                else if (hNeighbor_[(size_t)f] == c) imb -= md[(size_t)f];
            }
            out[c] = imb;
        }
        return (int64_t)N;
    }
    for (const E& e : tab) {
        if (name != e.n) continue;
        if (!e.p) throw StatusError(AXISIM_E_STATE, name + " is not available: its scalar is not solved");
        if (!out || n < e.len) throw StatusError(AXISIM_E_ARG, "output buffer too small for " + name);
        CK(cudaStreamSynchronize(stream_));
        if (!e.ell) {
            CK(cudaMemcpy(out, e.p, e.len * sizeof(double), cudaMemcpyDeviceToHost));
        } else {
            std::vector<double> ell((size_t)W_ * N);
            CK(cudaMemcpy(ell.data(), e.p, ell.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int c = 0; c < N_; c++)
                for (int k = hCfs_[(size_t)c], j = 0; k < hCfs_[(size_t)c + 1]; k++, j++)
                    out[k] = ell[(size_t)j * N + (size_t)c];
        }
        return (int64_t)e.len;
    }
    throw StatusError(AXISIM_E_ARG, "unknown field " + name);
}

int64_t Solver::setField(const std::string& name, const double* in, size_t n) {
    if (!haveMesh_) throw StatusError(AXISIM_E_STATE, "no mesh");
    const size_t N = (size_t)N_, F = (size_t)F_;
    struct E {
        const char* n;
        double* p;
        size_t len;
    };
    if (solveS_[0] || solveS_[1]) ensureScalarBuffers();
    const E tab[] = {{"u", u_, N}, {"v", v_, N}, {"p", p_, N}, {"mDot", mDot_, F}, {"uOld", uOld_, N},
                     {"vOld", vOld_, N}, {"uOld2", uOld2_, N}, {"vOld2", vOld2_, N},
                     {"T", sb_[0].phi, N}, {"TOld", sb_[0].old(), N}, {"TOld2", sb_[0].old2(), N},
                     {"C", sb_[1].phi, N}, {"COld", sb_[1].old(), N}, {"COld2", sb_[1].old2(), N}};
    for (const E& e : tab) {
        if (name != e.n) continue;
        if (!e.p) throw StatusError(AXISIM_E_STATE, name + " is not available: its scalar is not solved");
        if (!in || n < e.len) throw StatusError(AXISIM_E_ARG, "input buffer too small for " + name);
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(e.p, in, e.len * sizeof(double), cudaMemcpyHostToDevice));
        isReady_ = true;  // a seeded state can be continued from
        return (int64_t)e.len;
    }
    throw StatusError(AXISIM_E_ARG, "field is not settable: " + name);
}

}  // namespace axisim

// ====================================================================== C ABI
using axisim::Solver;
using axisim::StatusError;

struct axisim_handle {
    std::unique_ptr<Solver> s;
    std::string err;
    std::mutex mu;
};

struct axisim_mesh {
    axisim::PackedMesh m;
};

namespace {

template <class Fn>
int guarded(axisim_handle* h, Fn&& fn) {
    if (!h) return AXISIM_E_ARG;
    try {
        h->s->activate();
        return fn();
    } catch (const StatusError& e) {
        h->err = e.what();
        return e.status;
    } catch (const std::exception& e) {
        h->err = e.what();
        return AXISIM_E_CUDA;
    } catch (...) {
        h->err = "unknown error";
        return AXISIM_E_CUDA;
    }
}

}  // namespace

extern "C" {

int axisim_abi_version(void) { return AXISIM_ABI_VERSION; }

int axisim_create_on(int32_t device, const axisim_fluid* fluid, axisim_handle** out) {
    if (!out) return AXISIM_E_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        return AXISIM_E_CUDA;
    }
    if (device < 0 || device >= n) return AXISIM_E_ARG;
    try {
        axisim_fluid f{998.0, 0.0010518, 4180.0, 0.6, 3.0277e-9};
        if (fluid) f = *fluid;
        auto* h = new axisim_handle;
        h->s.reset(new Solver(device, f));
        *out = h;
        return AXISIM_OK;
    } catch (...) {
        return AXISIM_E_CUDA;
    }
}

int axisim_create(const axisim_fluid* fluid, axisim_handle** out) { return axisim_create_on(0, fluid, out); }

int axisim_destroy(axisim_handle* h) {
    if (!h) return AXISIM_E_ARG;
    delete h;
    return AXISIM_OK;
}

const char* axisim_last_error(const axisim_handle* h) { return h ? h->err.c_str() : "null handle"; }

int axisim_set_log(axisim_handle* h, axisim_log_fn log, axisim_residual_fn residual, void* ctx) {
    return guarded(h, [&] {
        h->s->logFn = log;
        h->s->resFn = residual;
        h->s->cbCtx = ctx;
        return AXISIM_OK;
    });
}

int axisim_set_mesh(axisim_handle* h, const axisim_mesh_packed* mesh) {
    return guarded(h, [&] {
        if (!mesh) throw StatusError(AXISIM_E_ARG, "mesh is null");
        h->s->setMesh(*mesh);
        return AXISIM_OK;
    });
}

int axisim_set_bc(axisim_handle* h, int32_t variable, const axisim_bc_field* bc) {
    return guarded(h, [&] {
        if (!bc) throw StatusError(AXISIM_E_ARG, "bc is null");
        h->s->setBC(variable, *bc);
        return AXISIM_OK;
    });
}

int axisim_set_mesh_type(axisim_handle* h, int32_t meshType) {
    return guarded(h, [&] {
        h->s->setMeshType(meshType);
        return AXISIM_OK;
    });
}

int axisim_set_kinetics(axisim_handle* h, int32_t variable, const axisim_kinetics* kin) {
    return guarded(h, [&] {
        h->s->setKinetics(variable, kin);
        return AXISIM_OK;
    });
}

int axisim_set_scalars(axisim_handle* h, int32_t solveEnergy, int32_t solveConcentration,
                       const axisim_config_residual* res2) {
    return guarded(h, [&] {
        h->s->setScalars(solveEnergy, solveConcentration, res2);
        return AXISIM_OK;
    });
}

int axisim_scalar_residuals(const axisim_handle* h, double* out2) {
    if (!h || !out2) return AXISIM_E_ARG;
    h->s->scalarResiduals(out2);
    return AXISIM_OK;
}

int axisim_set_config(axisim_handle* h, const axisim_config_solver* solver, const axisim_config_simple* simple,
                      const axisim_config_multigrid* mg, const axisim_config_residual* res3, double alphaU,
                      double alphaP) {
    return guarded(h, [&] {
        h->s->setConfig(solver, simple, mg, res3, alphaU, alphaP);
        return AXISIM_OK;
    });
}

int axisim_set_fluid(axisim_handle* h, const axisim_fluid* fluid) {
    return guarded(h, [&] {
        if (!fluid) throw StatusError(AXISIM_E_ARG, "fluid is null");
        h->s->setFluid(*fluid);
        return AXISIM_OK;
    });
}

int axisim_set_precision(axisim_handle* h, int32_t mode) {
    return guarded(h, [&] {
        h->s->setPrecision(mode);
        return AXISIM_OK;
    });
}

int axisim_set_pressure_solver(axisim_handle* h, int32_t mode, double relTol, double prolongScale) {
    return guarded(h, [&] {
        h->s->setPressureSolver(mode, relTol, prolongScale);
        return AXISIM_OK;
    });
}

int axisim_set_vcycle_kernel(axisim_handle* h, int32_t mode) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        h->s->setVcycleKernel(mode);
        return AXISIM_OK;
    });
}

int axisim_set_momentum_sweeps(axisim_handle* h, int32_t sweepsPerLaunch, int32_t threads) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        h->s->setMomentumSweeps(sweepsPerLaunch, threads);
        return AXISIM_OK;
    });
}

int axisim_sweep_tiles(axisim_handle* h, int32_t* nTiles) {
    if (!h || !nTiles) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        *nTiles = h->s->tileCount();
        return AXISIM_OK;
    });
}

int axisim_test_barrier_timeout(axisim_handle* h, int32_t on) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        h->s->testBarrierTimeout(on);
        return AXISIM_OK;
    });
}

int axisim_set_autotune(axisim_handle* h, int32_t enable) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        h->s->setAutotune(enable);
        return AXISIM_OK;
    });
}

int axisim_autotune_report(const axisim_handle* h, int32_t* blockPerLevel, double* usPerCandidate,
                           int32_t maxLevels) {
    auto* hh = const_cast<axisim_handle*>(h);
    if (maxLevels < 0) return -AXISIM_E_ARG;
    int r = 0;
    const int st = guarded(hh, [&] {
        r = hh->s->autotuneReport(blockPerLevel, usPerCandidate, maxLevels);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int axisim_learned_harvest(axisim_handle* h, int32_t every, int32_t capacity) {
    return guarded(h, [&] {
        h->s->learnedHarvest(every, capacity);
        return AXISIM_OK;
    });
}

int axisim_learned_sample_count(axisim_handle* h, int32_t* count) {
    return guarded(h, [&] {
        if (!count) throw StatusError(AXISIM_E_ARG, "count is null");
        *count = h->s->learnedSampleCount();
        return AXISIM_OK;
    });
}

int axisim_learned_add_sample(axisim_handle* h, const float* b, const float* target, const float* acDiag,
                              const float* deficit, const float* afSlots) {
    return guarded(h, [&] {
        h->s->learnedAddSample(b, target, acDiag, deficit, afSlots);
        return AXISIM_OK;
    });
}

int axisim_learned_get_sample(axisim_handle* h, int32_t index, float* b, float* target, float* acDiag,
                              float* deficit, float* afSlots, float* relResidual) {
    return guarded(h, [&] {
        h->s->learnedGetSample(index, b, target, acDiag, deficit, afSlots, relResidual);
        return AXISIM_OK;
    });
}

int axisim_learned_init(axisim_handle* h, int32_t precision, uint64_t seed, int64_t* nParams) {
    return guarded(h, [&] {
        const size_t n = h->s->learnedInit(precision, seed);
        if (nParams) *nParams = (int64_t)n;
        return AXISIM_OK;
    });
}

int axisim_learned_params(axisim_handle* h, float* params, int64_t n, int32_t set) {
    return guarded(h, [&] {
        h->s->learnedParams(params, n, set);
        return AXISIM_OK;
    });
}

int axisim_learned_grad(axisim_handle* h, int32_t sample, float* loss, float* grad, int64_t n) {
    return guarded(h, [&] {
        const float l = h->s->learnedGrad(sample, grad, n);
        if (loss) *loss = l;
        return AXISIM_OK;
    });
}

int axisim_learned_train(axisim_handle* h, int32_t steps, float lr, uint64_t seed, int32_t first, int32_t count,
                         float* lossOut) {
    return guarded(h, [&] {
        h->s->learnedTrain(steps, lr, seed, first, count, lossOut);
        return AXISIM_OK;
    });
}

int axisim_learned_predict(axisim_handle* h, const float* r, const float* acDiag, const float* deficit, float* out) {
    return guarded(h, [&] {
        h->s->learnedPredict(r, acDiag, deficit, out);
        return AXISIM_OK;
    });
}

int axisim_learned_enable(axisim_handle* h, int32_t mode) {
    return guarded(h, [&] {
        h->s->learnedEnable(mode);
        return AXISIM_OK;
    });
}

int axisim_learned_stats(axisim_handle* h, int64_t* applied, int64_t* fallbacks, double* scoreNet,
                         double* scoreVcycle) {
    return guarded(h, [&] {
        h->s->learnedStats(applied, fallbacks, scoreNet, scoreVcycle);
        return AXISIM_OK;
    });
}

int axisim_pressure_stats(axisim_handle* h, int64_t* solves, int64_t* iterations) {
    return guarded(h, [&] {
        h->s->pressureStats(solves, iterations);
        return AXISIM_OK;
    });
}

int axisim_solve(axisim_handle* h, int32_t continueRun, axisim_result* result) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] { return h->s->solve(continueRun, result); });
}

int axisim_can_continue(const axisim_handle* h, char* reason, size_t reasonLen) {
    if (!h) return -AXISIM_E_ARG;
    std::string why;
    const bool ok = h->s->canContinue(&why);
    if (!ok && reason && reasonLen) {
        std::snprintf(reason, reasonLen, "%s", why.c_str());
    }
    return ok ? 1 : 0;
}

int axisim_request_stop(axisim_handle* h) {
    if (!h) return AXISIM_E_ARG;
    h->s->requestStop();
    return AXISIM_OK;
}

int64_t axisim_get_field(const axisim_handle* h, const char* name, double* out, size_t n) {
    auto* hh = const_cast<axisim_handle*>(h);
    int64_t r = 0;
    const int st = guarded(hh, [&] {
        if (!name) throw StatusError(AXISIM_E_ARG, "name is null");
        r = h->s->getField(name, out, n);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int64_t axisim_set_field(axisim_handle* h, const char* name, const double* in, size_t n) {
    int64_t r = 0;
    const int st = guarded(h, [&] {
        if (!name) throw StatusError(AXISIM_E_ARG, "name is null");
        r = h->s->setField(name, in, n);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int axisim_mg_levels(const axisim_handle* h, int32_t* cellsPerLevel, int32_t maxLevels) {
    auto* hh = const_cast<axisim_handle*>(h);
    int r = 0;
    const int st = guarded(hh, [&] {
        r = hh->s->mgLevels(cellsPerLevel, maxLevels);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int64_t axisim_mg_level_maps(const axisim_handle* h, int32_t level, int32_t* cellToCoarse,
                             int32_t* fineSlotToCoarseSlot, int32_t* coarseFaceStart, int32_t* coarseFaceNeighbor) {
    auto* hh = const_cast<axisim_handle*>(h);
    int64_t r = 0;
    const int st = guarded(hh, [&] {
        r = hh->s->mgLevelMaps(level, cellToCoarse, fineSlotToCoarseSlot, coarseFaceStart, coarseFaceNeighbor);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int axisim_coloring(const axisim_handle* h, int32_t* colorOut, size_t n) {
    auto* hh = const_cast<axisim_handle*>(h);
    int r = 0;
    const int st = guarded(hh, [&] {
        r = hh->s->coloring(colorOut, n);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

namespace {
// The connectivity checks of axisim_set_mesh: false for a mesh whose indices
// would read outside its arrays.
bool connectivityOk(const axisim_mesh_packed* pm) {
    if (!pm || pm->nCells <= 0 || pm->nFaces <= 0 || !pm->cellFaceStart || !pm->cellFaceIDs || !pm->faceOwner ||
        !pm->faceNeighbor || pm->cellFaceStart[0] != 0)
        return false;
    const int N = pm->nCells, F = pm->nFaces;
    for (int c = 0; c < N; c++) {
        const int d = pm->cellFaceStart[c + 1] - pm->cellFaceStart[c];
        if (d < 0 || d > 32) return false;
    }
    for (int k = 0; k < pm->cellFaceStart[N]; k++)
        if (pm->cellFaceIDs[k] < 0 || pm->cellFaceIDs[k] >= F) return false;
    for (int f = 0; f < F; f++)
        if (pm->faceOwner[f] < 0 || pm->faceOwner[f] >= N || pm->faceNeighbor[f] >= N) return false;
    return true;
}

axisim::GridLevel hostFinest(const axisim_mesh_packed* pm) {
    return axisim::finestLevel(pm->nCells, pm->nFaces, pm->cellFaceStart, pm->cellFaceIDs, pm->faceOwner,
                               pm->faceNeighbor);
}
}  // namespace

int axisim_mg_levels_host(const axisim_mesh_packed* mesh, int32_t* cellsPerLevel, int32_t maxLevels) {
    if (maxLevels < 0 || (maxLevels > 0 && !cellsPerLevel)) return -AXISIM_E_ARG;
    if (!connectivityOk(mesh)) return -AXISIM_E_MESH;
    try {
        const std::vector<axisim::GridLevel> h = axisim::buildHierarchy(hostFinest(mesh));
        for (int l = 0; l < (int)h.size() && l < maxLevels; l++) cellsPerLevel[l] = h[(size_t)l].nCells;
        return (int)h.size();
    } catch (...) {
        return -AXISIM_E_MESH;
    }
}

int axisim_mg_batch_levels_host(const axisim_mesh_packed* mesh, int32_t nCases, const int32_t* caseCellStart,
                                int32_t* cellsPerLevel, int32_t* terminalCellsPerLevel, int32_t maxLevels) {
    if (maxLevels < 0 || (maxLevels > 0 && (!cellsPerLevel || !terminalCellsPerLevel))) return -AXISIM_E_ARG;
    if (nCases < 1 || !caseCellStart) return -AXISIM_E_ARG;
    if (!connectivityOk(mesh)) return -AXISIM_E_MESH;
    if (caseCellStart[0] != 0 || caseCellStart[nCases] != mesh->nCells) return -AXISIM_E_ARG;
    for (int c = 0; c < nCases; c++)
        if (caseCellStart[c + 1] <= caseCellStart[c]) return -AXISIM_E_ARG;
    try {
        std::vector<std::vector<int32_t>> term;
        const std::vector<int32_t> start(caseCellStart, caseCellStart + nCases + 1);
        const std::vector<axisim::GridLevel> h = axisim::buildBatchHierarchy(hostFinest(mesh), start, term);
        for (int l = 0; l < (int)h.size() && l < maxLevels; l++) {
            cellsPerLevel[l] = h[(size_t)l].nCells;
            int t = 0;
            for (size_t i = 0; i + 1 < term[(size_t)l].size(); i += 2) t += term[(size_t)l][i + 1] - term[(size_t)l][i];
            terminalCellsPerLevel[l] = t;
        }
        return (int)h.size();
    } catch (...) {
        return -AXISIM_E_MESH;
    }
}

int64_t axisim_mg_level_maps_host(const axisim_mesh_packed* mesh, int32_t level, int32_t* cellToCoarse,
                                  int32_t* fineSlotToCoarseSlot, int32_t* coarseFaceStart,
                                  int32_t* coarseFaceNeighbor) {
    if (!connectivityOk(mesh)) return -AXISIM_E_MESH;
    try {
        const std::vector<axisim::GridLevel> h = axisim::buildHierarchy(hostFinest(mesh));
        if (level < 0 || level + 1 >= (int)h.size()) return -AXISIM_E_ARG;
        const axisim::GridLevel& f = h[(size_t)level];
        const axisim::GridLevel& c = h[(size_t)level + 1];
        if (cellToCoarse) std::copy(f.cellToCoarse.begin(), f.cellToCoarse.end(), cellToCoarse);
        if (fineSlotToCoarseSlot)
            std::copy(f.fineSlotToCoarseSlot.begin(), f.fineSlotToCoarseSlot.end(), fineSlotToCoarseSlot);
        if (coarseFaceStart) std::copy(c.faceStart.begin(), c.faceStart.end(), coarseFaceStart);
        if (coarseFaceNeighbor) std::copy(c.faceNeighbor.begin(), c.faceNeighbor.end(), coarseFaceNeighbor);
        return c.nFaceRefs();
    } catch (...) {
        return -AXISIM_E_MESH;
    }
}

int64_t axisim_sweep_tiles_host(const axisim_mesh_packed* mesh, int32_t S, int32_t cap, int32_t tileCells,
                                int32_t* nTiles, int32_t* tileStart, int32_t* layerEnd, int32_t* gid, uint64_t* lnb,
                                int64_t capacity) {
    if (!nTiles || S < 1 || S > axisim::kMaxSweepsPerLaunch || cap < 1 || cap >= 0xFFFF || tileCells < 1)
        return -AXISIM_E_ARG;
    if (!connectivityOk(mesh)) return -AXISIM_E_MESH;
    const int N = mesh->nCells;
    int W = 0;
    for (int c = 0; c < N; c++) W = std::max(W, mesh->cellFaceStart[c + 1] - mesh->cellFaceStart[c]);
    if (W < 1 || W > 4) return -AXISIM_E_MESH;
    if (!mesh->cellCenterZ || !mesh->cellCenterR) return -AXISIM_E_ARG;
    try {
        const std::vector<int32_t> nb = axisim::slotNeighbours(N, W, mesh->cellFaceStart, mesh->cellFaceIDs,
                                                               mesh->faceOwner, mesh->faceNeighbor);
        const axisim::SweepTiles t =
            axisim::buildSweepTiles(N, W, nb.data(), mesh->cellCenterZ, mesh->cellCenterR, S, cap, tileCells);
        *nTiles = t.nTiles();
        const int64_t local = (int64_t)t.gid.size();
        if (tileStart && layerEnd && gid && lnb && capacity >= local) {
            std::copy(t.tileStart.begin(), t.tileStart.end(), tileStart);
            std::copy(t.layerEnd.begin(), t.layerEnd.end(), layerEnd);
            std::copy(t.gid.begin(), t.gid.end(), gid);
            std::copy(t.lnb.begin(), t.lnb.end(), lnb);
        }
        return local;
    } catch (...) {
        return -AXISIM_E_MESH;
    }
}

int axisim_coloring_host(const axisim_mesh_packed* mesh, int32_t* colorOut, size_t n) {
    if (!colorOut) return -AXISIM_E_ARG;
    if (!connectivityOk(mesh)) return -AXISIM_E_MESH;
    if (n < (size_t)mesh->nCells) return -AXISIM_E_ARG;
    try {
        std::vector<int32_t> color;
        const int nc = axisim::greedyColoring(hostFinest(mesh), color);
        std::copy(color.begin(), color.end(), colorOut);
        return nc;
    } catch (...) {
        return -AXISIM_E_MESH;
    }
}

int axisim_profile_iteration(axisim_handle* h, int32_t iterations, axisim_kernel_stat* out, int32_t maxOut,
                             int32_t* nOut) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        if (iterations < 1 || !out || maxOut < 1) throw StatusError(AXISIM_E_ARG, "bad profile arguments");
        const int n = h->s->profile(iterations, out, maxOut);
        if (nOut) *nOut = n;
        return AXISIM_OK;
    });
}

int axisim_profile_levels(axisim_handle* h, int32_t iterations, axisim_kernel_stat* out, int32_t maxOut,
                          int32_t* nOut) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        if (iterations < 1 || !out || maxOut < 1) throw StatusError(AXISIM_E_ARG, "bad profile arguments");
        const int n = h->s->profile(iterations, out, maxOut, true);
        if (nOut) *nOut = n;
        return AXISIM_OK;
    });
}

int axisim_setup_profile(axisim_handle* h, axisim_kernel_stat* out, int32_t maxOut, int32_t* nOut, int32_t reset) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        if (!out || maxOut < 1) throw StatusError(AXISIM_E_ARG, "bad setup profile arguments");
        const int n = h->s->setupProfile(out, maxOut, reset);
        if (nOut) *nOut = n;
        return AXISIM_OK;
    });
}

int axisim_mesh_segments(axisim_handle* h, int32_t* nSegments, int32_t* nOffsetSegments, int32_t* nFaceSegments,
                         int32_t* inUse) {
    if (!h) return AXISIM_E_ARG;
    std::lock_guard<std::mutex> lk(h->mu);
    return guarded(h, [&] {
        h->s->meshSegments(nSegments, nOffsetSegments, nFaceSegments, inUse);
        return AXISIM_OK;
    });
}

int axisim_set_batch(axisim_handle* h, int32_t nCases, const int32_t* caseCellStart) {
    return guarded(h, [&] {
        h->s->setBatch(nCases, caseCellStart);
        return AXISIM_OK;
    });
}

int axisim_batch_status(const axisim_handle* h, int32_t* convergedAt, double* residuals, int32_t n) {
    auto* hh = const_cast<axisim_handle*>(h);
    int r = 0;
    const int st = guarded(hh, [&] {
        r = hh->s->batchStatus(convergedAt, residuals, n);
        return AXISIM_OK;
    });
    return st == AXISIM_OK ? r : -st;
}

int axisim_multiblock_build(int32_t nBlocks, const axisim_block_spec* blocks, double tol, int32_t defaultGroup,
                            axisim_mesh** out, int32_t* seamStatus) {
    if (!out || nBlocks <= 0 || !blocks) return AXISIM_E_ARG;
    try {
        std::vector<axisim::BlockSpec> spec((size_t)nBlocks);
        for (int i = 0; i < nBlocks; i++) {
            const axisim_block_spec& b = blocks[i];
            if (b.axialCells <= 0 || b.radialCells <= 0) return AXISIM_E_ARG;
            axisim::BlockSpec& s = spec[(size_t)i];
            s.z0 = b.z0; s.r0 = b.r0;
            s.axialLength = b.axialLength; s.axialCells = b.axialCells; s.axialGrading = b.axialGrading; s.axialCoef = b.axialCoef;
            s.radialLength = b.radialLength; s.radialCells = b.radialCells; s.radialGrading = b.radialGrading; s.radialCoef = b.radialCoef;
            for (int e = 0; e < 4; e++) s.edgeGroup[e] = b.edgeGroup[e];
        }
        int seam = 0;
        auto* m = new axisim_mesh;
        m->m = axisim::buildMultiblock(spec, tol, defaultGroup, seam);
        if (seamStatus) *seamStatus = seam;
        *out = m;
        return AXISIM_OK;
    } catch (...) {
        return AXISIM_E_MESH;
    }
}

namespace {
// Copies and checks an outline; false when an array it needs is missing.
bool outlineFrom(const axisim_outline* o, axisim::Outline& d) {
    if (!o || o->nVertices < 0 || o->nEdges < 0) return false;
    if (o->nVertices > 0 && (!o->vertexZ || !o->vertexR)) return false;
    if (o->nEdges > 0 && (!o->edgeV0 || !o->edgeV1 || !o->edgeGroup)) return false;
    d.vz.assign(o->vertexZ, o->vertexZ + o->nVertices);
    d.vr.assign(o->vertexR, o->vertexR + o->nVertices);
    d.e0.assign(o->edgeV0, o->edgeV0 + o->nEdges);
    d.e1.assign(o->edgeV1, o->edgeV1 + o->nEdges);
    d.group.assign(o->edgeGroup, o->edgeGroup + o->nEdges);
    return true;
}
}  // namespace

int axisim_trellis_build(int32_t nZLines, const double* zLines, int32_t nRLines, const double* rLines,
                         const int32_t* zBandCells, const int32_t* rBandCells, const axisim_outline* outline,
                         double L, double R, int32_t nz, int32_t nr, axisim_mesh** out, int32_t* seamStatus) {
    if (!out || nZLines < 0 || nRLines < 0) return AXISIM_E_ARG;
    if ((nZLines > 0 && (!zLines || !zBandCells)) || (nRLines > 0 && (!rLines || !rBandCells))) return AXISIM_E_ARG;
    axisim::Outline o;
    if (!outlineFrom(outline, o)) return AXISIM_E_ARG;
    for (int i = 0; i + 1 < nZLines; i++)
        if (!(zLines[i + 1] > zLines[i])) return AXISIM_E_ARG;
    for (int j = 0; j + 1 < nRLines; j++)
        if (!(rLines[j + 1] > rLines[j])) return AXISIM_E_ARG;
    try {
        std::vector<double> zL(zLines, zLines + nZLines), rL(rLines, rLines + nRLines);
        std::vector<int> zc(zBandCells, zBandCells + std::max(nZLines - 1, 0));
        std::vector<int> rc(rBandCells, rBandCells + std::max(nRLines - 1, 0));
        int seam = 0;
        auto* m = new axisim_mesh;
        m->m = axisim::buildTrellis(zL, rL, zc, rc, o, L, R, nz, nr, seam);
        if (seamStatus) *seamStatus = seam;
        *out = m;
        return AXISIM_OK;
    } catch (...) {
        return AXISIM_E_MESH;
    }
}

int axisim_triangle_mesh_build(int32_t nPoints, const double* pointZ, const double* pointR, int32_t nTriangles,
                               const int32_t* triangles, const axisim_outline* outline, double L, double R,
                               axisim_mesh** out) {
    if (!out || nPoints <= 0 || nTriangles <= 0 || !pointZ || !pointR || !triangles) return AXISIM_E_ARG;
    axisim::Outline o;
    if (!outlineFrom(outline, o)) return AXISIM_E_ARG;
    try {
        std::vector<double> pz(pointZ, pointZ + nPoints), pr(pointR, pointR + nPoints);
        std::vector<int32_t> tri(triangles, triangles + 3 * (size_t)nTriangles);
        auto* m = new axisim_mesh;
        try {
            m->m = axisim::buildTriangleMesh(pz, pr, tri, o, L, R);
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
        return AXISIM_OK;
    } catch (...) {
        return AXISIM_E_MESH;
    }
}

int axisim_classify_boundary_faces(int32_t nFaces, const int32_t* faceNeighbor, const double* faceCenterZ,
                                   const double* faceCenterR, const axisim_outline* outline, double L, double R,
                                   int32_t* faceBoundaryGroupID) {
    if (nFaces < 0 || (nFaces > 0 && (!faceNeighbor || !faceCenterZ || !faceCenterR || !faceBoundaryGroupID)))
        return AXISIM_E_ARG;
    axisim::Outline o;
    if (!outlineFrom(outline, o)) return AXISIM_E_ARG;
    const double tol = 1e-4 * std::max(std::max(L, R), 1.0);
    for (int f = 0; f < nFaces; f++)
        if (faceNeighbor[f] < 0) faceBoundaryGroupID[f] = axisim::groupAtPoint(o, faceCenterZ[f], faceCenterR[f], tol);
    return AXISIM_OK;
}

int axisim_mesh_sizes(const axisim_mesh* m, int32_t* nCells, int32_t* nFaces, int32_t* nRefs) {
    if (!m) return AXISIM_E_ARG;
    if (nCells) *nCells = m->m.nCells;
    if (nFaces) *nFaces = m->m.nFaces;
    if (nRefs) *nRefs = (int32_t)m->m.cellFaceIDs.size();
    return AXISIM_OK;
}

int axisim_mesh_view(const axisim_mesh* m, axisim_mesh_packed* v) {
    if (!m || !v) return AXISIM_E_ARG;
    const axisim::PackedMesh& p = m->m;
    v->nCells = p.nCells;
    v->nFaces = p.nFaces;
    v->faceOwner = p.faceOwner.data();
    v->faceNeighbor = p.faceNeighbor.data();
    v->faceNormalZ = p.faceNormalZ.data();
    v->faceNormalR = p.faceNormalR.data();
    v->faceCenterZ = p.faceCenterZ.data();
    v->faceCenterR = p.faceCenterR.data();
    v->faceArea = p.faceArea.data();
    v->faceBoundaryGroupID = p.faceBoundaryGroupID.data();
    v->cellCenterZ = p.cellCenterZ.data();
    v->cellCenterR = p.cellCenterR.data();
    v->cellArea2D = p.cellArea2D.data();
    v->cellVolume = p.cellVolume.data();
    v->cellFaceStart = p.cellFaceStart.data();
    v->cellFaceIDs = p.cellFaceIDs.data();
    return AXISIM_OK;
}

int axisim_mesh_free(axisim_mesh* m) {
    delete m;
    return AXISIM_OK;
}

int axisim_resolve_bc(int32_t boundaryType, int32_t variable, int32_t hasUser, int32_t userType, double userValue,
                      uint8_t* typeOut, double* valueOut, uint8_t* pulsatileOut) {
    if (!typeOut || !valueOut || variable < 0 || variable > 4) return AXISIM_E_ARG;
    int t;
    double v;
    if (hasUser && axisim::variableEditable(variable, boundaryType)) {
        t = userType;
        v = userValue;
    } else {
        t = axisim::defaultBCType(boundaryType, variable);
        v = 0.0;
    }
    if (pulsatileOut) *pulsatileOut = (t == AXISIM_BC_PULSATILE) ? 1 : 0;
    *typeOut = (uint8_t)(t == AXISIM_BC_PULSATILE ? AXISIM_BC_DIRICHLET : t);
    *valueOut = v;
    return AXISIM_OK;
}

}  // extern "C"
