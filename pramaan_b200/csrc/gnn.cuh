// gnn.cuh — the learned warm start: a bipartite constraint-variable graph
// network that predicts a primal point x, a dual point y and the primal
// weight omega of every LP of a batch, trained on the GPU by hand-written
// forward and backward kernels.
//
// Graph.  The K LPs are packed block-diagonally (as in the batched solver).
// Variable j and constraint i are nodes; every non-zero A_ij is an edge.
// Per LP k the host computes scales s_a (RMS of the non-zeros), s_b (RMS of
// the finite row bounds), s_c (RMS of the minimisation cost) and the
// reference weight omega_ref = ||c|| / ||b|| (1 when either is zero).
//
// Node features (9 per node, FP32):
//   variable j:   c_j/s_c, [l_j finite], [u_j finite], clip(l_j s_a/s_b),
//                 clip(u_j s_a/s_b), log(1+deg_j)/4, mean|A_.j|/s_a,
//                 [hint x given], clip(xh_j s_a/s_b)
//   constraint i: [l_i == u_i], [l_i finite], [u_i finite], clip(l_i/s_b),
//                 clip(u_i/s_b), log(1+deg_i)/4, mean|A_i.|/s_a,
//                 [hint y given], clip(yh_i s_a/s_c)
// (clip to [-10, 10]; a missing bound or hint gives 0).  A hint (xh, yh) is
// an optional prior guess of the LP's solution given by the caller — for a
// rolling-horizon stream, the previous window's solution shifted by one
// period — and the x / y heads predict a correction to it.
//
// Network (hidden width 64, BF16 weights and activations, FP32 sums):
//   h_v0 = relu(W_vin f_v + b_vin)          h_c0 = relu(W_cin f_c + b_cin)
//   for l = 1..3:
//     agg_c[i] = sum_j A_ij / (s_a max(1, deg_i)) h_v[j]
//     h_c      = relu(W_c^l [h_c ; agg_c] + b_c^l)          (64 x 128 GEMM)
//     agg_v[j] = sum_i A_ij / (s_a max(1, deg_j)) h_c[i]     (new h_c)
//     h_v      = relu(W_v^l [h_v ; agg_v] + b_v^l)
//   xhat_j = xh_j s_a/s_b + w_x . h_v[j] + b_x,
//   yhat_i = yh_i s_a/s_c + w_y . h_c[i] + b_y   (hint terms 0 without a hint),
//   rho_k  = w_w . [mean_{j in k} h_v ; mean_{i in k} h_c] + b_w
//   prediction: x_j = clamp(xhat_j s_b/s_a, l_j, u_j), y_i = yhat_i s_c/s_a,
//               omega_k = omega_ref_k exp(clamp(rho_k, -10, 10)).
// Every BF16 rounding point (weights, h, agg, dz) is part of the definition:
// the NumPy restatement rounds at the same points.
//
// Loss against a solved point (x*, y*, omega*), with scaled targets
// tx_j = x*_j s_a/s_b, ty_i = y*_i s_a/s_c, tw_k = log(omega*_k / omega_ref_k):
//   L = 1/K sum_k [ sum_{j in k} (xhat_j - tx_j)^2 / (n_k (mean_{j in k} tx_j^2 + d))
//                 + sum_{i in k} (yhat_i - ty_i)^2 / (m_k (mean_{i in k} ty_i^2 + d))
//                 + (rho_k - tw_k)^2 ],   d = kLossFloor,
// i.e. each LP's squared error relative to the size of its own solution, so
// that LPs with large duals do not dominate.
//
// The six 64 x 128 layers run on the tensor cores (tcgen05.mma, operands
// staged by TMA with the 128-byte swizzle, FP32 accumulators in tensor
// memory): forward H = relu(X W^T + b), input gradient dX = dZ W and weight
// gradient dW^T = X^T dZ (MN-major operands, per-CTA partials reduced in a
// fixed order).  The aggregations are warp-per-node gathers over the CSR of
// A and of its transpose, so the backward pass is a gather too and every
// reduction is deterministic.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>
#include <vector>

#include "csr_device.cuh"

namespace pb {

constexpr int kGnnHidden = 64;
constexpr int kGnnFeat = 9;
constexpr int kGnnLayers = 3;
constexpr int kGnnChunk = 256;   // nodes per reduction chunk (chunks never straddle two LPs)
constexpr double kLossFloor = 1e-2;   // added to each LP's mean squared target in the loss weights

// Offsets into the flat FP32 parameter vector.
struct GnnParams {
    static constexpr int kVinW = 0;                          // [64][9]
    static constexpr int kVinB = kVinW + 64 * kGnnFeat;      // [64]
    static constexpr int kCinW = kVinB + 64;                 // [64][9]
    static constexpr int kCinB = kCinW + 64 * kGnnFeat;      // [64]
    static constexpr int kLayer0 = kCinB + 64;
    static constexpr int kDenseW = 64 * 128;                 // one layer's W [64 out][128 in]
    static constexpr int kLayerStride = 2 * (kDenseW + 64);  // W_c, b_c, W_v, b_v
    static constexpr int layer_w(int l, int side) { return kLayer0 + l * kLayerStride + side * (kDenseW + 64); }
    static constexpr int layer_b(int l, int side) { return layer_w(l, side) + kDenseW; }
    static constexpr int kHeadX = kLayer0 + kGnnLayers * kLayerStride;   // w_x [64], b_x
    static constexpr int kHeadY = kHeadX + 65;                           // w_y [64], b_y
    static constexpr int kHeadW = kHeadY + 65;                           // w_w [128], b_w
    static constexpr int kCount = kHeadW + 129;
};

// A packed batch of LPs prepared for the network (device resident).
class GnnGraph {
public:
    GnnGraph(const pramaan_lp* lps, int count, const pramaan_warm_start* hints, const pramaan_warm_start* targets,
             int device);
    ~GnnGraph();
    GnnGraph(const GnnGraph&) = delete;
    GnnGraph& operator=(const GnnGraph&) = delete;

    int device = 0;
    int count = 0;                 // LPs given by the caller
    int K = 0, m = 0, n = 0, nnz = 0;
    bool has_targets = false;
    std::vector<int> index;        // packed LP q -> caller's index
    std::vector<int> r0, c0;       // packed row / column start of each LP (size K + 1)
    std::vector<double> s_a, s_b, s_c, omega_ref;
    cudaStream_t st = nullptr;

    DevBuf<int> rp, ci, tp, ti;                   // CSR of A and of A^T
    DevBuf<float> coef_r, coef_c;                 // A order: A_ij/(s_a deg_i), A_ij/(s_a deg_j)
    DevBuf<float> tcoef_r, tcoef_c;               // A^T order, the same two coefficients
    DevBuf<float> fv, fc;                         // node features [n][9], [m][9]
    DevBuf<float> base_x, base_y;                 // scaled hints added to the heads ([n], [m])
    DevBuf<int> lp_col, lp_row;                   // LP of each node
    DevBuf<float> lp_scale;                       // [K][4]: s_a, s_b, s_c, 1/K
    DevBuf<double> vlo, vhi;                      // variable bounds
    std::vector<double> h_vlo, h_vhi;             // host copies (prediction clamp)
    DevBuf<float> tx, ty, tw;                     // scaled targets
    DevBuf<float> lw_x, lw_y;                     // per-LP loss weights (see the loss)
    // chunk tables: chunk c covers nodes [begin[c], begin[c+1]); lp_first[k]..lp_first[k+1]
    int cchunks = 0, rchunks = 0;
    DevBuf<int> cchunk_begin, rchunk_begin, cchunk_lp, rchunk_lp, clp_first, rlp_first;
    DevBuf<float> inv_n, inv_m;                   // per LP: 1/n_k, 1/m_k (0 when m_k = 0)
};

class GnnModel {
public:
    GnnModel(int device, uint64_t seed);
    ~GnnModel();
    GnnModel(const GnnModel&) = delete;
    GnnModel& operator=(const GnnModel&) = delete;

    static int num_params() { return GnnParams::kCount; }
    void get_params(float* host) const;
    void set_params(const float* host);
    // Forward pass; activations are kept for backward() / trace().
    void forward(const GnnGraph& g);
    // Loss of the last forward pass against g's targets; with `grad` the
    // gradient is left in grad_ (device).
    double backward(const GnnGraph& g, bool grad);
    void adam_step(float lr);
    void copy_grad(float* host) const;
    // x, y, omega in the original units of each LP (forward() first).
    void predict(const GnnGraph& g, double* const* x, double* const* y, double* omega);
    // Every stored activation as FP32, in the order documented at
    // pramaan_gnn_forward_trace.
    size_t trace_size(const GnnGraph& g) const;
    void trace(const GnnGraph& g, float* host) const;

private:
    void refresh_weights();
    void ensure_workspace(const GnnGraph& g);

    int dev_ = 0;
    cudaStream_t st_ = nullptr;
    long long adam_t_ = 0;
    DevBuf<float> p_, g_, am_, av_;        // FP32 master, gradient, Adam moments
    DevBuf<float> pr_;                     // parameters rounded to BF16 (as FP32)
    DevBuf<__nv_bfloat16> w_, wt_;         // per dense layer: W [64][128], W^T [128][64]
    DevBuf<int> status_;
    // workspace (grown to the largest graph seen)
    size_t cap_m_ = 0, cap_n_ = 0, cap_k_ = 0, cap_chunks_ = 0;
    DevBuf<__nv_bfloat16> xc_[kGnnLayers], xv_[kGnnLayers];   // [rows][128] = [h_prev ; agg]
    DevBuf<__nv_bfloat16> hc3_, hv3_;                           // [rows][64]
    DevBuf<__nv_bfloat16> dz_;                                  // [max(m,n)][64]
    DevBuf<float> dhc_, dhv_, dagg_;                            // [rows][64]
    DevBuf<float> xhat_, yhat_, pooled_, rho_;
    DevBuf<float> part_, lp_sums_, wpart_;
    const GnnGraph* last_ = nullptr;
};

}  // namespace pb
