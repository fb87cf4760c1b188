// Mixed-precision solves: FP64 iterative refinement around the complex64
// operator. Each refinement step computes the true residual r = b - A x with
// the FP64 operator (the plain path, which reproduces the reference's
// matvec), solves the correction equation A d = r with FGMRES on the plan's
// complex64 copies (patterns, transfer factors, shifts, near field and
// workspaces in complex64, FP32 arithmetic; Krylov vectors, Gram-Schmidt and
// Givens rotations in FP64) to a relative tolerance aimed at the target, and
// updates x += d. The stopping test is always the FP64 residual.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <vector>

#include "blas1.cuh"
#include "solver.hpp"

namespace mlfma {

namespace {

using C = std::complex<double>;

// Relative tolerance of one correction solve: enough for the FP64 residual
// to fall under the target (half of it, for margin), bounded below by what a
// complex64 operator can deliver and above so that every step gains.
double inner_tolerance(double err, double tol_rel) {
  return std::min(0.5, std::max(1e-5, 0.5 * tol_rel / err));
}

double norm2(const C* v, long long n) {
  double s = 0.0;
  for (long long i = 0; i < n; ++i) s += std::norm(v[i]);
  return std::sqrt(s);
}

// r_q = b_q - A x_q with the FP64 operator for the listed systems (rows of
// host arrays), through device rows of up to kBatchSlots; returns ||r_q||.
std::vector<double> fp64_residuals(Plan& P, const std::vector<int>& list, const C* X, const C* B, C* Rr,
                                   double2* Xd, double2* Wd) {
  const long long n = 2LL * P.N;
  std::vector<double> out;
  for (size_t g0 = 0; g0 < list.size(); g0 += kBatchSlots) {
    const int rn = static_cast<int>(std::min<size_t>(kBatchSlots, list.size() - g0));
    for (int j = 0; j < rn; ++j)
      MLFMA_CUDA(cudaMemcpyAsync(Xd + j * n, X + list[g0 + j] * n, n * sizeof(double2), cudaMemcpyHostToDevice,
                                 P.stream));
    for (int j = 0; j < rn; ++j) apply_device(P, Xd + j * n, Wd + j * n, P.stream);
    std::vector<C> w(static_cast<size_t>(rn) * n);
    MLFMA_CUDA(cudaMemcpyAsync(w.data(), Wd, w.size() * sizeof(double2), cudaMemcpyDeviceToHost, P.stream));
    fetch_device_status(P, P.stream);
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    raise_device_status(P);
    for (int j = 0; j < rn; ++j) {
      const int q = list[g0 + j];
      for (long long i = 0; i < n; ++i) Rr[q * n + i] = B[q * n + i] - w[j * n + i];
      out.push_back(norm2(Rr + q * n, n));
    }
  }
  return out;
}

// fp64_residuals for a refinement's starting point: systems whose x is all
// zero take r = b without an apply (applied[q] = 0); the others are applied.
std::vector<double> start_residuals(Plan& P, const std::vector<int>& list, const C* X, const C* B, C* Rr,
                                    double2* Xd, double2* Wd, std::vector<char>& applied) {
  const long long n = 2LL * P.N;
  std::vector<double> out(list.size());
  std::vector<int> nz;
  std::vector<size_t> at;
  applied.assign(list.size(), 0);
  for (size_t a = 0; a < list.size(); ++a) {
    const int q = list[a];
    const bool zero = std::all_of(X + q * n, X + (q + 1) * n, [](const C& c) { return c == C(0.0); });
    if (zero) {
      std::copy(B + q * n, B + (q + 1) * n, Rr + q * n);
      out[a] = norm2(B + q * n, n);
    } else {
      nz.push_back(q);
      at.push_back(a);
      applied[a] = 1;
    }
  }
  if (!nz.empty()) {
    const std::vector<double> r = fp64_residuals(P, nz, X, B, Rr, Xd, Wd);
    for (size_t k = 0; k < nz.size(); ++k) out[at[k]] = r[k];
  }
  return out;
}

}  // namespace

bool mixed_solve(Plan& P, double* xh, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                 int inner_its, int refine_max, SolveStats& st, std::vector<double>& history) {
  if (P.precision != 1) throw std::invalid_argument("plan was not created with mixed precision");
  if (refine_max < 0) throw std::invalid_argument("refine_max must be non-negative");
  const auto t0 = std::chrono::steady_clock::now();
  MLFMA_CUDA(cudaSetDevice(P.device));
  MLFMA_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int), P.stream));
  const long long n = 2LL * P.N;
  C* x = reinterpret_cast<C*>(xh);
  const C* b = reinterpret_cast<const C*>(rhs);
  st = SolveStats();
  history.clear();
  std::vector<C> r(n), d(n);
  double bnorm = norm2(b, n);
  if (bnorm < 1e-16) bnorm = 1.0;
  const std::vector<int> one{0};
  std::vector<char> applied;
  double err = start_residuals(P, one, x, b, r.data(), P.d_x, P.d_w, applied)[0] / bnorm;
  st.matvecs += applied[0];
  history.push_back(err);
  bool ok = err < tol_rel || err < tol_abs;
  for (int step = 0; !ok && step < refine_max && st.iterations < itr_max; ++step) {
    std::fill(d.begin(), d.end(), C(0.0));
    SolveStats si;
    std::vector<double> hi;
    fgmres_solve(P, reinterpret_cast<double*>(d.data()), reinterpret_cast<const double*>(r.data()),
                 itr_max - st.iterations, mr, 0.0, inner_tolerance(err, tol_rel), inner_its, si, hi, 1);
    st.iterations += si.iterations;
    st.matvecs += si.matvecs;
    st.near_products += si.near_products;
    st.restarts++;
    for (long long i = 0; i < n; ++i) x[i] += d[i];
    err = fp64_residuals(P, one, x, b, r.data(), P.d_x, P.d_w)[0] / bnorm;
    st.matvecs++;
    history.push_back(err);
    ok = err < tol_rel || err < tol_abs;
  }
  st.rel_residual = err;
  st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return ok;
}

std::vector<char> mixed_batch_solve(Plan& P, int R, double* xh, const double* rhs, int itr_max, int mr,
                                    double tol_abs, double tol_rel, int inner_its, int refine_max,
                                    std::vector<SolveStats>& st, double& seconds) {
  if (P.precision != 1) throw std::invalid_argument("plan was not created with mixed precision");
  if (R < 1) throw std::invalid_argument("R must be positive");
  if (refine_max < 0) throw std::invalid_argument("refine_max must be non-negative");
  const auto t0 = std::chrono::steady_clock::now();
  MLFMA_CUDA(cudaSetDevice(P.device));
  MLFMA_CUDA(cudaMemsetAsync(P.d_status, 0, sizeof(int), P.stream));
  reserve_batch(P, R, false);
  reserve_batch_staging(P);  // the FP64 residuals' device rows
  const long long n = 2LL * P.N;
  C* X = reinterpret_cast<C*>(xh);
  const C* B = reinterpret_cast<const C*>(rhs);
  double2* Xd = P.d_xb;
  double2* Wd = P.d_wb;
  std::vector<C> Rr(static_cast<size_t>(R) * n);
  st.assign(R, SolveStats());
  std::vector<double> bnorm(R), err(R);
  std::vector<int> all(R);
  for (int q = 0; q < R; ++q) {
    all[q] = q;
    bnorm[q] = norm2(B + q * n, n);
    if (bnorm[q] < 1e-16) bnorm[q] = 1.0;
  }
  std::vector<char> applied;
  std::vector<double> rn = start_residuals(P, all, X, B, Rr.data(), Xd, Wd, applied);
  std::vector<char> ok(R, 0);
  std::vector<int> live;
  for (int q = 0; q < R; ++q) {
    st[q].matvecs += applied[q];
    err[q] = rn[q] / bnorm[q];
    ok[q] = err[q] < tol_rel || err[q] < tol_abs;
    if (!ok[q]) live.push_back(q);
  }
  for (int step = 0; !live.empty() && step < refine_max; ++step) {
    const int Rl = static_cast<int>(live.size());
    double worst = 0.0;
    std::vector<C> rb(static_cast<size_t>(Rl) * n), d(static_cast<size_t>(Rl) * n, C(0.0));
    for (int a = 0; a < Rl; ++a) {
      std::copy(Rr.begin() + live[a] * n, Rr.begin() + (live[a] + 1) * n, rb.begin() + a * n);
      worst = std::max(worst, err[live[a]]);
    }
    std::vector<SolveStats> si;
    std::vector<std::vector<double>> hi;
    double sec = 0.0;
    int budget = itr_max;
    for (int q : live) budget = std::min(budget, itr_max - st[q].iterations);
    if (budget <= 0) break;
    fgmres_batch_solve(P, Rl, reinterpret_cast<double*>(d.data()), reinterpret_cast<const double*>(rb.data()), budget,
                       mr, 0.0, inner_tolerance(worst, tol_rel), inner_its, si, hi, sec, 1);
    for (int a = 0; a < Rl; ++a) {
      const int q = live[a];
      st[q].iterations += si[a].iterations;
      st[q].matvecs += si[a].matvecs + 1;
      st[q].near_products += si[a].near_products;
      st[q].restarts++;
      for (long long i = 0; i < n; ++i) X[q * n + i] += d[a * n + i];
    }
    rn = fp64_residuals(P, live, X, B, Rr.data(), Xd, Wd);
    std::vector<int> keep;
    for (int a = 0; a < Rl; ++a) {
      const int q = live[a];
      err[q] = rn[a] / bnorm[q];
      ok[q] = err[q] < tol_rel || err[q] < tol_abs;
      if (!ok[q]) keep.push_back(q);
    }
    live = keep;
  }
  seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int q = 0; q < R; ++q) {
    st[q].rel_residual = err[q];
    st[q].seconds = seconds;
  }
  return ok;
}

}  // namespace mlfma
