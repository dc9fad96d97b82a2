// learned.cuh -- the learned edge rating: a small message-passing network
// that predicts, per edge, the probability that a partition cuts it; its
// complement replaces expansion*^2 (edge_ratings.cpp:171-183) as the matching
// rating.  The reference has no learned component; this is new.
//
// Network (BF16 weights and activations, FP32 accumulation):
//   node input  x_v = [log2(1+deg v)/8, log2(max(c(v),1))/8]
//   edge input  f_e = [log2(max(w_e,1))/8, log2(1+r_e)/8], r_e = expansion*^2
//   h0 = relu(W0 x + b0)                                      2 -> 64
//   h_l = relu(W_l [h_{l-1} | mean_w(h_{l-1} over N(v))] + b_l)  128 -> 64, l = 1..3
//   z  = Wz h3 + bz                                           64 -> 32
//   s_e = bo + wo . relu(z_u + z_v + Wf f_e),  p_e = sigmoid(s_e)
// s_e is symmetric in (u, v) bit for bit (z_u + z_v commutes exactly), so
// both directed entries of an edge get the same rating.
#pragma once

#include "lp.cuh"

namespace kb {

// Flat FP32 parameter layout (offsets in floats).
namespace rm {
constexpr int H = 64, Z = 32;
constexpr int W0 = 0, B0 = W0 + H * 2;
constexpr int W1 = B0 + H, B1 = W1 + H * 2 * H;
constexpr int W2 = B1 + H, B2 = W2 + H * 2 * H;
constexpr int W3 = B2 + H, B3 = W3 + H * 2 * H;
constexpr int WZ = B3 + H, BZ = WZ + Z * H;
constexpr int WF = BZ + Z, WO = WF + Z * 2, BO = WO + Z;
constexpr int kParams = BO + 1;  // 27137
constexpr int layer_w(int l) { return l == 1 ? W1 : l == 2 ? W2 : W3; }
constexpr int layer_b(int l) { return l == 1 ? B1 : l == 2 ? B2 : B3; }
}  // namespace rm

// Rating of every directed entry of g with model `params` (device FP32,
// rm::kParams floats): prob[e] = p_e (may be null), rating[e] =
// floor((1 - p_e) * 2^24) (may be null).  use_tc: the layer GEMMs run on
// the tensor cores (tcgen05, fused with the neighbour gather); otherwise on
// the CUDA cores (the training path's forward).
void rating_infer(Ctx& ctx, const DevGraph& g, const float* params, float* prob, uint32_t* rating, bool use_tc);

// One training graph: device CSR plus one 0/1 label per directed entry.
struct TrainGraph {
    DevGraph g;
    const uint8_t* label;
};

// Adam training of `params` (device FP32, in/out) on the graphs, one graph
// per step in round-robin order; loss_out[step] (host) = weighted BCE.
void rating_train(Ctx& ctx, const TrainGraph* graphs, int count, int steps, float lr, float* params,
                  float* loss_out);

// Loss (host out) and gradient G[kParams] (device out) of one graph at
// `params`, without an update.
void rating_grad(Ctx& ctx, const TrainGraph& tg, const float* params, float* G, float* loss);

}  // namespace kb
