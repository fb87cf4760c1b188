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
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>

#include "blas1.cuh"
#include "learned.hpp"
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

// Device state of the preconditioner's inner GMRES: its Hessenberg matrix,
// rotations and right-hand side live on the GPU, so that the inner steps run
// without a host round trip.
struct InnerDev {
  double2* H;   // [(inner + 1) x inner], column-major, ld = inner + 1
  double2* cs;  // [inner] rotations
  double2* sn;
  double2* g;   // [inner + 1] rotated right-hand side
  double2* y;   // [inner] solution of the triangular system
  double2* h1;  // [inner + 1] coefficients of the two Gram-Schmidt passes
  double2* h2;
  double2* hn2; // [1] ||u||^2 after the projections (real part)
  double* sc;   // [0] beta, [1] scale of the next basis vector, [2] 1 / beta
  int* flags;   // [0] breakdown, [1] columns in use
};

// beta = ||v|| from the norm partials; g = (beta, 0, ...); flags cleared
__global__ void inner_begin(const double2* partial, int nblk, InnerDev d, int inner) {
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += partial[b].x;
  const double beta = sqrt(s);
  d.sc[0] = beta;
  d.sc[2] = beta > 0.0 ? 1.0 / beta : 0.0;
  for (int i = 0; i <= inner; ++i) d.g[i] = c2(i == 0 ? beta : 0.0, 0.0);
  d.flags[0] = 0;
  d.flags[1] = 0;
}

// column j of H from the Gram-Schmidt coefficients, its rotations, and the
// scale of the next basis vector (0 after a breakdown)
__global__ void inner_step(InnerDev d, int j, int ld) {
  if (d.flags[0]) {
    d.sc[1] = 0.0;
    return;
  }
  double2* Hj = d.H + static_cast<long long>(j) * ld;
  for (int i = 0; i <= j; ++i) Hj[i] = cadd(d.h1[i], d.h2[i]);
  const double hn = sqrt(d.hn2[0].x);
  Hj[j + 1] = c2(hn, 0.0);
  for (int i = 0; i < j; ++i) blas1::dgivens_apply(Hj[i], Hj[i + 1], d.cs[i], d.sn[i]);
  d.flags[1] = j + 1;
  if (hn < 1e-14 * d.sc[0]) {
    d.flags[0] = 1;
    d.sc[1] = 0.0;
    return;
  }
  d.sc[1] = 1.0 / hn;
  blas1::dgivens_make(Hj[j], Hj[j + 1], d.cs[j], d.sn[j]);
  blas1::dgivens_apply(Hj[j], Hj[j + 1], d.cs[j], d.sn[j]);
  Hj[j + 1] = c2(0.0, 0.0);
  blas1::dgivens_apply(d.g[j], d.g[j + 1], d.cs[j], d.sn[j]);
}

// y = R^{-1} g over the columns in use (Code/GMRES.h:165-182); zero beyond
__global__ void inner_end(InnerDev d, int ld, int inner) {
  const int m = d.flags[1];
  const double eps = 1e-16;
  for (int i = inner - 1; i >= 0; --i) {
    if (i >= m) {
      d.y[i] = c2(0.0, 0.0);
      continue;
    }
    double2 yi = d.g[i];
    for (int j = i + 1; j < m; ++j) yi = csub(yi, cmul(d.H[i + static_cast<long long>(j) * ld], d.y[j]));
    const double2 hii = d.H[i + static_cast<long long>(i) * ld];
    d.y[i] = sqrt(hii.x * hii.x + hii.y * hii.y) > eps ? cdiv(yi, hii) : c2(0.0, 0.0);
  }
}

// dst = src * s[0]; dst may be src (the inner step scales its vector in place)
__global__ void scale_by(const double2* src, const double* s, double2* dst, long long n) {
  const double a = *s;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = cscale(src[i], a);
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

namespace {

// z = approximate solution of Z_near z = v by inner_its GMRES steps from
// zero, with the complex64 copy of Z_near (the outer flexible GMRES admits
// any preconditioner; its operator and residuals stay at the solve's
// precision). The inner Hessenberg matrix, rotations and triangular solve
// stay on the GPU: the inner steps run without a host round trip. Buffers
// come from the caller's Work; the reduction scratch is the caller's Ops.
struct NearPrecond {
  Plan& P;
  cudaStream_t s;
  long long n;
  int inner_its, ldi;
  blas1::Ops ops;
  double2* Q = nullptr;
  InnerDev idv{};
  NearPrecond(Plan& P_, cudaStream_t s_, int inner, blas1::Work& g, const blas1::Ops& o)
      : P(P_), s(s_), n(2LL * P_.N), inner_its(inner), ldi(inner + 1), ops(o) {
    if (inner_its <= 0) return;
    Q = g.get(static_cast<size_t>(inner_its + 1) * n);
    idv.H = g.get(static_cast<size_t>(ldi) * inner_its);
    idv.cs = g.get(inner_its);
    idv.sn = g.get(inner_its);
    idv.g = g.get(ldi);
    idv.y = g.get(inner_its);
    idv.h1 = g.get(ldi);
    idv.h2 = g.get(ldi);
    idv.hn2 = g.get(1);
    idv.sc = reinterpret_cast<double*>(g.get(2));
    idv.flags = reinterpret_cast<int*>(g.get(1));
  }
  void launch(const double2* v, double2* z) {
    blas1::norm2<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(nullptr, v, nullptr, n, ops.part);
    inner_begin<<<1, 1, 0, s>>>(ops.part, blas1::kBlocks, idv, inner_its);
    scale_by<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(v, idv.sc + 2, Q, n);
    for (int j = 0; j < inner_its; ++j) {
      const double2* q = Q + static_cast<long long>(j) * n;
      double2* u = Q + static_cast<long long>(j + 1) * n;
      near_apply(P, q, u, s, 1);
      const int nv = j + 1;
      blas1::dots<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, nv, u, ops.part, ops.ldp);
      blas1::reduce<<<(nv + 63) / 64, 64, 0, s>>>(ops.part, blas1::kBlocks, ops.ldp, nv, idv.h1);
      blas1::project_out<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, nv, idv.h1, u, 0, ops.part, ops.ldp);
      blas1::dots<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, nv, u, ops.part, ops.ldp);
      blas1::reduce<<<(nv + 63) / 64, 64, 0, s>>>(ops.part, blas1::kBlocks, ops.ldp, nv, idv.h2);
      blas1::project_out<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, nv, idv.h2, u, 1, ops.part, ops.ldp);
      blas1::reduce<<<1, 64, 0, s>>>(ops.part, blas1::kBlocks, ops.ldp, 1, idv.hn2);
      inner_step<<<1, 1, 0, s>>>(idv, j, ldi);
      scale_by<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(u, idv.sc + 1, u, n);
    }
    inner_end<<<1, 1, 0, s>>>(idv, ldi, inner_its);
    blas1::combine<<<blas1::kBlocks, blas1::kThreads, 0, s>>>(Q, n, inner_its, idv.y, z, 0);
    MLFMA_CUDA(cudaGetLastError());
  }
};

}  // namespace

void near_precondition(Plan& P, int inner_its, const double2* v, double2* z, cudaStream_t s) {
  if (inner_its < 1 || inner_its + 1 > blas1::kMaxBasis) throw std::invalid_argument("inner_its must be in 1..63");
  MLFMA_CUDA(cudaSetDevice(P.device));
  blas1::Work g;
  const int ldp = blas1::kMaxBasis + 2;
  blas1::Ops ops{s, 2LL * P.N, g.get(static_cast<size_t>(blas1::kBlocks) * ldp), ldp, g.get(2 * ldp + 2)};
  NearPrecond np(P, s, inner_its, g, ops);
  np.launch(v, z);
  MLFMA_CUDA(cudaStreamSynchronize(s));  // the work arrays are freed on return
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
  NearPrecond np(P, s, inner_its, g, ops);
  auto precondition_launch = [&](const double2* v, double2* z) {
    np.launch(v, z);
    // a learned correction of z, when a network is attached to the plan
    if (const __nv_bfloat16* wl = lp_attached(P)) lp_forward(P, wl, v, z, z, false, s);
  };
  // The preconditioner's ~10 launches per inner step are captured once per
  // solve as a CUDA graph on solve-owned input / output vectors (v copied in,
  // z out): the same graph serves every basis vector.
  double2* pv = inner_its > 0 ? g.get(n) : nullptr;
  double2* pz = inner_its > 0 ? g.get(n) : nullptr;
  cudaGraphExec_t pgraph = nullptr;
  struct GraphGuard {
    cudaGraphExec_t& e;
    ~GraphGuard() {
      if (e) cudaGraphExecDestroy(e);
    }
  } pguard{pgraph};
  auto precondition = [&](const double2* v, double2* z) {
    st.near_products += inner_its;
    if (!P.tuning.graph) return precondition_launch(v, z);
    MLFMA_CUDA(cudaMemcpyAsync(pv, v, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if (pgraph == nullptr) {
      MLFMA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        precondition_launch(pv, pz);
      } catch (...) {
        cudaGraph_t gr = nullptr;
        cudaStreamEndCapture(s, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
      }
      cudaGraph_t gr = nullptr;
      MLFMA_CUDA(cudaStreamEndCapture(s, &gr));
      const cudaError_t e = cudaGraphInstantiate(&pgraph, gr, 0);
      cudaGraphDestroy(gr);
      MLFMA_CUDA(e);
    }
    MLFMA_CUDA(cudaGraphLaunch(pgraph, s));
    MLFMA_CUDA(cudaMemcpyAsync(z, pz, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  };

  const double eps = 1e-16;
  // a zero initial guess has r = b without an apply
  const bool from_zero = std::all_of(xh, xh + 2 * n, [](double v) { return v == 0.0; });
  double rnorm;
  if (from_zero) {
    MLFMA_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    rnorm = ops.norm(b);
  } else {
    rnorm = true_residual();
  }
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
