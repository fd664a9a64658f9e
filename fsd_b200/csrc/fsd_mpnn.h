// Message-passing network that predicts a correction to the two-hop sparse
// approximate inverse G ~ (R_FU^pruned + D)^-1 used by FSD_PRECOND_LEARNED
// (mpnn.cu).
//
// Graph: particles, and a directed edge c -> s for every member s != c of
// c's two-hop set (the pattern of G).  Inputs are rotation invariants of each
// pair (gap, inverse distance, the tabulated resistance scalars and whether
// the pair is in direct contact range); outputs are scalar coefficients of an
// axisymmetric tensor basis built from the pair's unit vector, so the
// correction rotates with the configuration by construction:
//   dG_cs = J_c B(o_cs, r_cs)                       (s != c)
//   dG_cc = J_c (diag(c_t I3, c_r I3) + sum_s B(q_cs, r_cs))
// with J_c = (A_cc)^-1 the inverse diagonal block of A = R_FU^pruned + D and
//   B(o, r) = [ o0 rr + o1 (I - rr)   o2 [r]x          ]
//             [ o3 [r]x               o4 rr + o5 (I - rr) ]
// ([r]x the cross-product matrix).  o = out[0:6], q = out[6:12] of the edge
// head; (c_t, c_r) from the node head.
//
// Network (width 64, three message-passing layers, ReLU):
//   e0 = relu(W_in x + b_in)                    x: 16 edge features
//   h0_i = mean_j e0_ij
//   layer l = 1..3:
//     m = relu(W_m [e, h_src, h_dst] + b_m);  e <- e + m
//     h <- h + relu(W_h [h, mean_j m_ij] + b_h)
//   edge head  o_ij = W_o [e, h_src, h_dst] + b_o   (12 used of 16)
//   node head  c_i  = W_n h_i + b_n                 (2 used of 16)
#pragma once

#include <cstddef>

namespace fsd {

constexpr int kMpWidth = 64;
constexpr int kMpLayers = 3;
constexpr int kMpFeat = 16;     // edge input features
constexpr int kMpHeadE = 16;    // edge head outputs (12 used)
constexpr int kMpHeadN = 16;    // node head outputs (2 used)

// Offsets of the parameter blocks in the flat fp32 weight vector.  Matrices
// are row-major [out x in].
struct MpLayout {
    static constexpr int W_in = 0;
    static constexpr int b_in = W_in + kMpWidth * kMpFeat;
    static constexpr int layer0 = b_in + kMpWidth;
    static constexpr int W_m = 0;                                   // [64 x 192]
    static constexpr int b_m = W_m + kMpWidth * 3 * kMpWidth;
    static constexpr int W_h = b_m + kMpWidth;                      // [64 x 128]
    static constexpr int b_h = W_h + kMpWidth * 2 * kMpWidth;
    static constexpr int layer_size = b_h + kMpWidth;
    static constexpr int W_o = layer0 + kMpLayers * layer_size;     // [16 x 192]
    static constexpr int b_o = W_o + kMpHeadE * 3 * kMpWidth;
    static constexpr int W_n = b_o + kMpHeadE;                      // [16 x 64]
    static constexpr int b_n = W_n + kMpHeadN * kMpWidth;
    static constexpr int total = b_n + kMpHeadN;
    static constexpr int layer(int l) { return layer0 + l * layer_size; }
};

}  // namespace fsd
