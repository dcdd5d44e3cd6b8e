// learned.hpp -- the learned pressure-correction preconditioner: a U-Net over
// the agglomeration multigrid's own hierarchy, trained on the GPU by the
// kernels in learned.cu.
//
// In the solver the network is the preconditioner of the first flexible-CG
// iteration of a p' solve, whose line search scales it; per solve, a device
// gate picks it or the plain V-cycle by their running residual-reduction
// scores (k_fcg_gate in krylov.cu).
//
// Network (levels l = 0 .. L-1 of the hierarchy, channels C_l = 16, 32, 64,
// then 128 on every coarser level; "mp" is a message-passing layer
// relu([h, mean_nb(h)] W + b) over the level's cell graph):
//   level 0:  h0 = relu(x W_in + b),  x = [r / (A_C sigma), 1 - sum|A_F| / A_C]
//             e0 = mp(h0)
//   level l:  h_l = relu(pool(e_{l-1}) W_down + b)   (pool: mean over the
//             agglomerate's members),  e_l = mp(h_l)
//   bottom:   d_{L-1} = mp(e_{L-1})
//   level l:  s_l = relu(unpool(d_{l+1}) W_up + b + e_l)  (unpool: copy from
//             the agglomerate),  d_l = mp(s_l)
//   output:   y = d_0 W_out + b,  correction = sigma y
// sigma = rms(r / A_C) makes the map scale-equivariant. Weights of levels >= 3
// (>= 4 for the down projections, whose input width changes at level 3) are
// shared, so one set of parameters serves hierarchies of any depth and the
// receptive field reaches the coarsest level (the whole domain). On a
// structured block the neighbour mean is a 5-point stencil and pool/unpool
// follow the 2 x 2 agglomerates, so there the network is a convolutional
// U-Net; on an unstructured mesh the same layers are message passing.
// Weights are BF16 copies of FP32 masters and every product accumulates in
// FP32; activations are FP32 by default, because the energy norm the network
// is trained and used in differences neighbouring values of its smooth output
// (BF16 storage, also available, loses most of that); a full-FP32 mode serves
// the gradient check.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "device.cuh"

namespace axisim {

struct GridLevel;

// One level of the network's graph, device arrays.
struct NetGraphLevel {
    int N = 0;
    const int32_t* nStart = nullptr;  // neighbours of each cell, CSR
    const int32_t* nList = nullptr;
    const float* invDeg = nullptr;    // 1 / neighbour count (0 when none)
    const int32_t* c2c = nullptr;     // to level l + 1 (null on the last level)
    const int32_t* mStart = nullptr;  // members of each cell in level l - 1 (null on level 0)
    const int32_t* mList = nullptr;
    const float* invCnt = nullptr;
};

enum NetXform { NX_ID = 0, NX_NBMEAN = 1, NX_POOL = 2, NX_UNPOOL = 3 };

struct NetIn {
    const void* x = nullptr;  // activations [rows of the source level][C]
    int C = 0;
    int xf = NX_ID;
    // NBMEAN: the level's neighbour CSR; POOL: the coarse cells' member CSR +
    // the fine level's c2c (adjoint); UNPOOL: c2c (forward) + member CSR (adjoint)
    const int32_t* s = nullptr;
    const int32_t* list = nullptr;
    const float* inv = nullptr;
    const int32_t* map = nullptr;
    int srcRows = 0;
};

struct NetLayer {
    int N = 0, K = 0, Cout = 0, relu = 1;
    size_t wOff = 0;  // weights [K][Cout] then bias [Cout] in the flat parameter vector
    NetIn in[2];
    int nIn = 0;
    const void* add = nullptr;  // [N][Cout] added before the activation
    void* Y = nullptr;          // [N][Cout]
    void* Z = nullptr;          // [N][K] concatenated input (training only)
    float* gY = nullptr;        // gradient of Y
    float* gIn[2] = {nullptr, nullptr};
    float* gAdd = nullptr;
};

// Training-sample harvest from the captured SIMPLE iteration (learned.cu).
void launchHarvest(const Ctl* ctl, int N, int every, int cap, const double* b, const double* x, const double* AC,
                   const double* AF, const int32_t* nb, int W, const double* fcgScalars, float* store, int* count,
                   float* relres, unsigned int* counter, cudaStream_t s);

class LearnedNet {
public:
    LearnedNet() = default;
    ~LearnedNet();
    LearnedNet(const LearnedNet&) = delete;
    LearnedNet& operator=(const LearnedNet&) = delete;

    // Builds the graph from the hierarchy (host CSR + maps) and allocates
    // weights and activations for meshes of hier[0].nCells cells; nb [W][N0]
    // is the finest level's ELL neighbour array (the training loss applies the
    // sample's matrix with it).
    // precision: 0 FP32 weights and activations, 1 BF16 weights and
    // activations, 2 BF16 weights with FP32 activations (always FP32
    // accumulation and FP32 master weights).
    void init(const std::vector<GridLevel>& hier, const int32_t* nb, int W, int precision, uint64_t seed,
              cudaStream_t s);
    bool ready() const { return N0_ > 0; }
    void reset() { release(); }
    int levels() const { return L_; }
    size_t numParams() const { return nParams_; }

    // Inference: correction e (FP32, [N0]) of residual r (FP64) for the matrix
    // (AF [W][N0] ELL with neighbours nb, AC). With ctl, the kernels return at
    // entry while ctl->done is set, and otherwise unless ctl->ppSkip is 2
    // (gated) or 0 (not gated).
    void infer(const Ctl* ctl, int gated, const double* r, const double* AC, const double* AF, const int32_t* nb,
               int W, float* e, cudaStream_t s);

    // A training sample: right-hand side b, converged p' (target), the
    // matrix (diagonal AC, off-diagonals AF as ELL [W][N0]) and the boundary
    // deficit, FP32 device arrays.
    struct Sample {
        const float *b, *target, *AC, *deficit, *AF;
    };
    // One training step on one sample: forward, energy-norm loss, backward,
    // Adam. The loss is the A-norm error left after the best scaling of the
    // output y,  1 - (y.b)^2 / ((y.A y)(b.target)),  which is what one
    // Krylov step along y removes. The loss of the step is written to lossOut
    // (device). t = Adam step count (1-based).
    void trainStep(const Sample& smp, float lr, int t, float* lossOut, cudaStream_t s);
    // Forward only on FP32 arrays (training-path features): out = sigma y.
    void predict(const float* r, const float* AC, const float* deficit, float* out, cudaStream_t s);
    // Forward + backward only: loss (device scalar) and the flat gradient.
    void lossAndGrad(const Sample& smp, float* lossOut, cudaStream_t s);

    // flat FP32 master parameters / gradient (device)
    float* params() { return params_; }
    const float* grad() const { return grad_; }
    void syncLowPrecision(cudaStream_t s);  // BF16 copies from the masters

private:
    void release();
    void buildLayers();
    void forward(const Ctl* ctl, int gated, bool keepZ, cudaStream_t s);
    void backward(cudaStream_t s);

    int N0_ = 0, L_ = 0, actBf16_ = 1, wBf16_ = 1;
    size_t nParams_ = 0;
    std::vector<void*> allocs_;
    std::vector<NetGraphLevel> g_;
    std::vector<int> C_;
    std::vector<NetLayer> layers_;
    // parameters
    float* params_ = nullptr;
    void* paramsLow_ = nullptr;  // BF16 copies (or the FP32 masters in FP32 mode)
    float* grad_ = nullptr;
    float* adamM_ = nullptr;
    float* adamV_ = nullptr;
    float* wgPartial_ = nullptr;
    // activations
    void* feat_ = nullptr;  // [N0][2]
    void* out_ = nullptr;   // [N0]
    float* gOut_ = nullptr;
    float* gpre_ = nullptr;
    float* dZ_ = nullptr;
    const int32_t* nb0_ = nullptr;  // finest level ELL neighbours [W0][N0]
    int W0_ = 0;
    float* Ay_ = nullptr;           // A y of the training loss
    double* scal_ = nullptr;        // [0] sigma^2, [1..3] y.b, y.Ay, b.t
    double* red_ = nullptr;   // block partials
    unsigned int* counter_ = nullptr;
};

}  // namespace axisim
