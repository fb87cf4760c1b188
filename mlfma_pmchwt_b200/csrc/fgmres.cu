// Flexible GMRES with a near-field preconditioner.
//
// The right preconditioner of the MLFMA system A x = b is an approximate
// solve with the near-field part of A alone (the same Z_near rows the matvec
// uses, Code/Zmartix.h:541-643): a fixed number of GMRES steps from zero on
// Z_near z = v. Because that inner solve changes from one outer step to the
// next, the outer iteration is flexible GMRES (Saad 1993): it keeps the
// preconditioned directions Z and updates x = x0 + Z y. The outer loop keeps
// MGMRES's arguments, stopping rule, true residual per cycle and divergence
// abort (Code/GMRES.h:65-217). With inner_its = 0 the preconditioner is the
// identity and the iteration is the reference's GMRES.
#include <chrono>
#include <cmath>
#include <complex>

#include "blas1.cuh"
#include "solver.hpp"

namespace mlfma {

namespace {

using C = std::complex<double>;

template <class Z>
struct NearArg {
  const int* leaf_rwg;
  const int* rwg_box;
  const int* leaf_ptr;
  const int* near_sptr;
  const int* near_src;
  const long long* near_zoff;
  const Z* near_z;
  const double2* x;
  double2* w;
  int N;
};

// w = Z_near x: rows t and N + t of the near field, one warp per RWG; the
// entries and the arithmetic in the storage type Z (complex128 or complex64).
template <class Z>
__global__ void __launch_bounds__(128) near_apply_kernel(NearArg<Z> a) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= a.N) return;
  const int id = a.leaf_rwg[r];
  const int b = a.rwg_box[id];
  const int s0 = a.near_sptr[b], ns = a.near_sptr[b + 1] - s0;
  const int tl = r - a.leaf_ptr[b];
  const Z* Zr = a.near_z + 3 * (a.near_zoff[b] + static_cast<long long>(tl) * ns);
  Z nJ = Cx<Z>::zero(), nM = Cx<Z>::zero();
  for (int j = lane; j < ns; j += 32) {
    const int s = a.near_src[s0 + j];
    const Z xJ = Cx<Z>::from(a.x[s]), xM = Cx<Z>::from(a.x[a.N + s]);
    const Z z11 = Zr[3 * j], z12 = Zr[3 * j + 1], z22 = Zr[3 * j + 2];
    nJ = cfma(z11, xJ, cfma(z12, xM, nJ));
    nM = cfma(z22, xM, csub(nM, cmul(z12, xJ)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nJ.x += __shfl_xor_sync(0xffffffffu, nJ.x, o);
    nJ.y += __shfl_xor_sync(0xffffffffu, nJ.y, o);
    nM.x += __shfl_xor_sync(0xffffffffu, nM.x, o);
    nM.y += __shfl_xor_sync(0xffffffffu, nM.y, o);
  }
  if (lane == 0) {
    a.w[id] = Cx<Z>::to64(nJ);
    a.w[a.N + id] = Cx<Z>::to64(nM);
  }
}

// Upper-triangular solve of the rotated least-squares system (Code/GMRES.h:165-182).
void back_substitute(const std::vector<C>& H, int ld, const std::vector<C>& s, int m, std::vector<C>& y) {
  const double eps = 1e-16;
  y.assign(m, C(0.0));
  for (int i = m - 1; i >= 0; --i) {
    y[i] = s[i];
    for (int j = i + 1; j < m; ++j) y[i] -= H[i + j * ld] * y[j];
    if (std::abs(H[i + i * ld]) > eps)
      y[i] /= H[i + i * ld];
    else
      y[i] = C(0.0);
  }
}

}  // namespace

void near_apply(Plan& P, const double2* x, double2* w, cudaStream_t s, int prec) {
  if (prec == 1) {
    if (P.d_near_z32 == nullptr) throw std::invalid_argument("plan holds no complex64 near field");
    NearArg<float2> a{P.d_leaf_rwg,  P.d_rwg_leafbox, P.d_leaf_ptr, P.d_near_sptr, P.d_near_src,
                      P.d_near_zoff, P.d_near_z32,    x,            w,             P.N};
    near_apply_kernel<float2><<<(P.N + 3) / 4, 128, 0, s>>>(a);
  } else {
    NearArg<double2> a{P.d_leaf_rwg,  P.d_rwg_leafbox, P.d_leaf_ptr, P.d_near_sptr, P.d_near_src,
                       P.d_near_zoff, P.d_near_z,      x,            w,             P.N};
    near_apply_kernel<double2><<<(P.N + 3) / 4, 128, 0, s>>>(a);
  }
  MLFMA_CUDA(cudaGetLastError());
}

bool fgmres_solve(Plan& P, double* xh, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                  int inner_its, SolveStats& st, std::vector<double>& history, int prec) {
  if (prec == 1 && P.precision != 1) throw std::invalid_argument("plan was not created with mixed precision");
  auto op_apply = [&](const double2* in, double2* out, cudaStream_t s) {
    if (prec == 1)
      apply_mixed_device(P, in, out, s);
    else
      apply_device(P, in, out, s);
  };
  if (mr < 1 || mr + 1 > blas1::kMaxBasis) throw std::invalid_argument("mr must be in 1..63");
  if (inner_its < 0 || inner_its + 1 > blas1::kMaxBasis) throw std::invalid_argument("inner_its must be in 0..63");
  const auto t0 = std::chrono::steady_clock::now();
  MLFMA_CUDA(cudaSetDevice(P.device));
  cudaStream_t s = P.stream;
  const long long n = 2LL * P.N;
  blas1::Work g;
  const int ldp = blas1::kMaxBasis + 2;
  double2* x = g.get(n);
  double2* b = g.get(n);
  double2* r = g.get(n);
  double2* w = g.get(n);
  double2* V = g.get(static_cast<size_t>(mr + 1) * n);
  double2* Zd = inner_its > 0 ? g.get(static_cast<size_t>(mr) * n) : V;
  double2* Q = inner_its > 0 ? g.get(static_cast<size_t>(inner_its + 1) * n) : nullptr;
  double2* y = g.get(blas1::kMaxBasis);
  blas1::Ops ops{s, n, g.get(static_cast<size_t>(blas1::kBlocks) * ldp), ldp, g.get(2 * ldp + 2)};
  MLFMA_CUDA(cudaMemcpyAsync(x, xh, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(b, rhs, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  st = SolveStats();
  history.clear();
  std::vector<C> hcol;

  auto true_residual = [&]() {
    op_apply(x, w, s);
    st.matvecs++;
    return ops.residual(b, w, r);
  };
  auto finish = [&](bool ok, double err) {
    MLFMA_CUDA(cudaMemcpyAsync(xh, x, n * sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    st.rel_residual = err;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return ok;
  };
  // z = approximate solution of Z_near z = v by inner_its GMRES steps from
  // zero, with the complex64 copy of Z_near (the outer flexible GMRES admits
  // any preconditioner; its operator and residuals stay at the solve's
  // precision)
  std::vector<C> Hi(static_cast<size_t>(inner_its + 1) * std::max(inner_its, 1)), ci(inner_its + 1),
      si(inner_its + 1), gi(inner_its + 1), yi;
  auto precondition = [&](const double2* v, double2* z) {
    const double beta = ops.norm(v);
    blas1::scale<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(v, 1.0 / beta, Q, n);
    const int ld = inner_its + 1;
    std::fill(Hi.begin(), Hi.end(), C(0.0));
    std::fill(gi.begin(), gi.end(), C(0.0));
    gi[0] = beta;
    int used = 0;
    for (int j = 0; j < inner_its; ++j) {
      double2* u = Q + static_cast<long long>(j + 1) * n;
      near_apply(P, Q + static_cast<long long>(j) * n, u, s, 1);
      st.near_products++;
      const double hn = ops.orthogonalise(Q, j + 1, u, hcol);
      for (int i = 0; i <= j; ++i) Hi[i + j * ld] = hcol[i];
      Hi[j + 1 + j * ld] = hn;
      used = j + 1;
      if (hn < 1e-14 * beta) break;
      blas1::scale<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(u, 1.0 / hn, u, n);
      for (int i = 0; i < j; ++i) blas1::givens_apply(Hi[i + j * ld], Hi[i + 1 + j * ld], ci[i], si[i]);
      blas1::givens_make(Hi[j + j * ld], Hi[j + 1 + j * ld], ci[j], si[j]);
      blas1::givens_apply(Hi[j + j * ld], Hi[j + 1 + j * ld], ci[j], si[j]);
      Hi[j + 1 + j * ld] = C(0.0);
      blas1::givens_apply(gi[j], gi[j + 1], ci[j], si[j]);
    }
    back_substitute(Hi, ld, gi, used, yi);
    MLFMA_CUDA(cudaMemcpyAsync(y, yi.data(), used * sizeof(double2), cudaMemcpyHostToDevice, s));
    blas1::combine<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, used, y, z, 0);
  };

  const double eps = 1e-16;
  double rnorm = true_residual();
  double bnorm = ops.norm(b);
  if (bnorm < eps) bnorm = 1.0;
  double error = rnorm / bnorm;
  if (error < tol_rel || error < tol_abs) return finish(true, error);

  const int ld = mr + 1;
  std::vector<C> H(static_cast<size_t>(ld) * mr), cs(mr), sn(mr), sv(mr + 1), yy;
  int total = 0;
  for (int cycle = 1; cycle <= itr_max; ++cycle) {
    st.restarts = cycle;
    blas1::scale<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(r, 1.0 / rnorm, V, n);
    std::fill(sv.begin(), sv.end(), C(0.0));
    sv[0] = rnorm;
    std::fill(H.begin(), H.end(), C(0.0));
    int k_used = 0;
    for (int k = 0; k < mr; ++k) {
      if (total >= itr_max) break;
      ++total;
      k_used = k + 1;
      const double2* vk = V + static_cast<long long>(k) * n;
      double2* zk = Zd + static_cast<long long>(k) * n;
      if (inner_its > 0) precondition(vk, zk);
      op_apply(zk, w, s);
      st.matvecs++;
      const double h_next = ops.orthogonalise(V, k + 1, w, hcol);
      for (int j = 0; j <= k; ++j) H[j + static_cast<size_t>(k) * ld] = hcol[j];
      H[k + 1 + static_cast<size_t>(k) * ld] = h_next;
      if (h_next < eps * rnorm) break;
      blas1::scale<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(w, 1.0 / h_next, V + static_cast<long long>(k + 1) * n, n);
      for (int j = 0; j < k; ++j) blas1::givens_apply(H[j + k * ld], H[j + 1 + k * ld], cs[j], sn[j]);
      blas1::givens_make(H[k + k * ld], H[k + 1 + k * ld], cs[k], sn[k]);
      blas1::givens_apply(H[k + k * ld], H[k + 1 + k * ld], cs[k], sn[k]);
      H[k + 1 + k * ld] = C(0.0);
      blas1::givens_apply(sv[k], sv[k + 1], cs[k], sn[k]);
      error = std::abs(sv[k + 1]) / bnorm;
      history.push_back(error);
      if (error < tol_rel || error < tol_abs) break;
    }
    const int m = std::min(k_used, mr);
    back_substitute(H, ld, sv, m, yy);
    if (m > 0) {
      MLFMA_CUDA(cudaMemcpyAsync(y, yy.data(), m * sizeof(double2), cudaMemcpyHostToDevice, s));
      blas1::combine<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Zd, n, m, y, x, 1);
    }
    rnorm = true_residual();
    error = rnorm / bnorm;
    st.iterations = total;
    if (error < tol_rel || error < tol_abs) return finish(true, error);
    if (total >= itr_max) return finish(false, error);
    if (error > 100.0 * tol_rel && cycle > 8 && error > 1000.0 * tol_rel) return finish(false, error);
  }
  st.iterations = total;
  return finish(false, error);
}

}  // namespace mlfma
