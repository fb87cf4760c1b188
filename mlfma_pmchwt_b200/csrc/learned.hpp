// Learned right preconditioner for flexible GMRES: a message-passing network
// over the octree's leaf boxes that corrects the near-field preconditioner's
// output (learned.cu). No counterpart in the reference, whose GMRES is
// unpreconditioned (Code/GMRES.h:65-217).
//
// For a Krylov vector v (complex128 [2N], J then M) and z = P_near v:
//   y_c[i] = z_c[i] + sum_t G[i][c][t] u_t[i]        c in {J, M}, t < 8
//   u = (z_J, z_M, d_i.Z2_J, d_i.Z2_M, d_i.Zb_J, d_i.Zb_M, d_i.Zn_J, d_i.Zn_M)
// d_i: RWG dipole l_i (c+ - c-), normalised to mean length 1; Zb_c[b]: mean
// of z_c d over box b's RWGs; Zn_c[b]: mean of Zb_c over b and its near
// neighbours; Z2_c[b]: the same mean of Zn_c. The complex gains G come from
// 16 static features per RWG (geometry and material) through
//   encoder  a_i = relu(We f_i + be)                       (16 -> 64)
//   pool     h0_b = mean over the box's RWGs of a_i
//   3 layers h_{l+1} = h_l + relu(Ws h_l + Wn mean_nbr(h_l) + Wg mean_all(h_l) + c)
//   decoder  q_i = relu(Wd1 [h3_box(i); a_i] + d1);  G_i = Wd2 q_i + d2   (128 -> 64 -> 32)
// so y = (I + L) z with a fixed linear L per body. Weights are bfloat16 on
// the device, arithmetic FP32. Parameters are one float vector in the order
// We, be, (Ws, Wn, Wg, c) x 3, Wd1, d1, Wd2, d2.
#pragma once
#include <cuda_bf16.h>

#include <memory>

#include "plan.hpp"

namespace mlfma {

constexpr int kLpF = 16;      // features per RWG
constexpr int kLpH = 64;      // width
constexpr int kLpT = 8;       // linear terms
constexpr int kLpG = 32;      // real gain outputs: 2 outputs x 8 terms x (re, im)
constexpr int kLpLayers = 3;
constexpr int kLpOffBe = kLpH * kLpF;
constexpr int kLpOffLayer0 = kLpOffBe + kLpH;
constexpr int kLpLayerSize = 3 * kLpH * kLpH + kLpH;  // Ws, Wn, Wg, c
constexpr int kLpOffWd1 = kLpOffLayer0 + kLpLayers * kLpLayerSize;
constexpr int kLpOffD1 = kLpOffWd1 + kLpH * 2 * kLpH;
constexpr int kLpOffWd2 = kLpOffD1 + kLpH;
constexpr int kLpOffD2 = kLpOffWd2 + kLpG * kLpH;
constexpr int kLpParams = kLpOffD2 + kLpG;  // 48,480

struct LearnedWork;

// Static tables and work arrays, allocated on first use (not inside a graph capture).
LearnedWork& lp_work(Plan& P);
// y = z + correction (y may alias z). w: bfloat16 parameters on the device.
// train: also keep what lp_backward needs.
void lp_forward(Plan& P, const __nv_bfloat16* w, const double2* v, const double2* z, double2* y, bool train,
                cudaStream_t s);
// After lp_forward(train) with output y: adds to grad (float [kLpParams]) the
// parameter gradient of sum |y - e|^2 / sum |e|^2 (gy null; the loss is
// added to *loss), or of a loss whose gradient with respect to y is given,
// gy = dL/dRe(y) + j dL/dIm(y) (e and loss unused).
void lp_backward(Plan& P, const __nv_bfloat16* w, const double2* y, const double2* e, const double2* gy, float* grad,
                 float* loss, cudaStream_t s);
// float -> bfloat16 (nearest, ties to even)
void lp_to_bf16(const float* in, __nv_bfloat16* out, int n, cudaStream_t s);
// One Adam step on float parameters with float moments; grad is multiplied by grad_scale.
void lp_adam(int n, float* theta, const float* grad, float* m, float* v, float lr, float b1, float b2, float eps,
             int step, float grad_scale, cudaStream_t s);
// The network the solves apply after the near-field preconditioner (host
// parameters; n = 0 detaches), and the bfloat16 copy the solves use (null
// when none is attached).
void lp_attach(Plan& P, const float* params, int n);
const __nv_bfloat16* lp_attached(const Plan& P);
// A scratch bfloat16 parameter buffer of the plan (for training calls).
__nv_bfloat16* lp_scratch_weights(Plan& P);

}  // namespace mlfma
