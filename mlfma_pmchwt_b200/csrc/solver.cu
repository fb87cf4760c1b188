// Restarted GMRES on the device (Code/GMRES.h:65-217), plane-wave
// excitation (Code/Vm.h:150-203) and far field (Code/RCS.h:116-192).
//
// GMRES: the Krylov basis, the iterate and all length-2N vector work live on
// the GPU; the (mr+1) x mr Hessenberg matrix, the complex Givens rotations
// and the triangular solve run on the host exactly as the reference's
// (generate_givens / apply_givens, Code/GMRES.h:22-48). Orthogonalisation is
// classical Gram-Schmidt applied twice (one projection, one re-projection),
// the block form of the reference's modified Gram-Schmidt plus one
// re-orthogonalisation pass (Code/GMRES.h:119-131); the Hessenberg column is
// the sum of both passes' coefficients, as in the reference. Reductions are
// two-stage and deterministic.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <mutex>
#include <string>

#include "cplx.cuh"
#include "solver.hpp"

namespace mlfma {

namespace {

constexpr int kRB = 592;   // reduction blocks (4 per SM)
constexpr int kRT = 256;   // threads per reduction block
constexpr int kJT = 8;     // basis vectors per pass of dots_kernel

__device__ __forceinline__ double2 block_sum(double2 v, double2* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (blockDim.x >> 5) ? sh[lane] : c2(0.0, 0.0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
  }
  return v;  // valid in thread 0
}

// partial[blk * ldp + j] = sum over this block's rows of conj(V_j) w, j < nv
__global__ void __launch_bounds__(kRT) dots_kernel(const double2* __restrict__ V, long long n, int nv,
                                                   const double2* __restrict__ w, double2* __restrict__ partial,
                                                   int ldp) {
  __shared__ double2 sh[kRT / 32];
  for (int j0 = 0; j0 < nv; j0 += kJT) {
    double2 acc[kJT];
#pragma unroll
    for (int q = 0; q < kJT; ++q) acc[q] = c2(0.0, 0.0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
      const double2 wi = w[i];
#pragma unroll
      for (int q = 0; q < kJT; ++q)
        if (j0 + q < nv) {
          const double2 v = V[(long long)(j0 + q) * n + i];
          // conj(v) * wi
          acc[q].x = fma(v.x, wi.x, fma(v.y, wi.y, acc[q].x));
          acc[q].y = fma(v.x, wi.y, fma(-v.y, wi.x, acc[q].y));
        }
    }
#pragma unroll
    for (int q = 0; q < kJT; ++q)
      if (j0 + q < nv) {
        const double2 s = block_sum(acc[q], sh);
        if (threadIdx.x == 0) partial[(long long)blockIdx.x * ldp + j0 + q] = s;
      }
  }
}

// out[j] = sum over blocks of partial[blk * ldp + j] (+ add[j] if add != null)
__global__ void reduce_kernel(const double2* __restrict__ partial, int nblk, int ldp, int nv, double2* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nv) return;
  double2 s = c2(0.0, 0.0);
  for (int b = 0; b < nblk; ++b) s = cadd(s, partial[(long long)b * ldp + j]);
  out[j] = s;
}

// w -= sum_j V_j h[j]; with norm != 0 also per-block partial ||w||^2 into partial[blk*ldp]
__global__ void __launch_bounds__(kRT) update_kernel(const double2* __restrict__ V, long long n, int nv,
                                                     const double2* __restrict__ h, double2* __restrict__ w,
                                                     int want_norm, double2* __restrict__ partial, int ldp) {
  __shared__ double2 hs[64];
  __shared__ double2 sh[kRT / 32];
  for (int j = threadIdx.x; j < nv; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  double2 nrm = c2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 wi = w[i];
    for (int j = 0; j < nv; ++j) wi = csub(wi, cmul(hs[j], V[(long long)j * n + i]));
    w[i] = wi;
    nrm.x = fma(wi.x, wi.x, fma(wi.y, wi.y, nrm.x));
  }
  if (want_norm) {
    const double2 s = block_sum(nrm, sh);
    if (threadIdx.x == 0) partial[(long long)blockIdx.x * ldp] = s;
  }
}

// r = b - w, partial ||r||^2
__global__ void __launch_bounds__(kRT) residual_kernel(const double2* __restrict__ b, const double2* __restrict__ w,
                                                       double2* __restrict__ r, long long n,
                                                       double2* __restrict__ partial) {
  __shared__ double2 sh[kRT / 32];
  double2 nrm = c2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = csub(b[i], w[i]);
    r[i] = v;
    nrm.x = fma(v.x, v.x, fma(v.y, v.y, nrm.x));
  }
  const double2 s = block_sum(nrm, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void norm_kernel(const double2* __restrict__ v, long long n, double2* __restrict__ partial) {
  __shared__ double2 sh[kRT / 32];
  double2 nrm = c2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 a = v[i];
    nrm.x = fma(a.x, a.x, fma(a.y, a.y, nrm.x));
  }
  const double2 s = block_sum(nrm, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void scale_kernel(const double2* __restrict__ src, double inv, double2* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = cscale(src[i], inv);
}

// x += sum_j V_j y[j]
__global__ void combine_kernel(const double2* __restrict__ V, long long n, int m, const double2* __restrict__ y,
                               double2* __restrict__ x) {
  __shared__ double2 ys[64];
  for (int j = threadIdx.x; j < m; j += blockDim.x) ys[j] = y[j];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 xi = x[i];
    for (int j = 0; j < m; ++j) xi = cfma(ys[j], V[(long long)j * n + i], xi);
    x[i] = xi;
  }
}

using C = std::complex<double>;

// Code/GMRES.h:22-40
void givens_make(C a, C b, C& c, C& s) {
  const double eps = 1e-16;
  const double an = std::abs(a), bn = std::abs(b);
  if (bn < eps) {
    c = 1.0;
    s = 0.0;
  } else if (an < eps) {
    c = 0.0;
    s = 1.0;
  } else {
    const double r = std::sqrt(std::real(a * std::conj(a) + b * std::conj(b)));
    c = a / r;
    s = b / r;
  }
}
// Code/GMRES.h:43-48
void givens_apply(C& x, C& y, C c, C s) {
  const C t = std::conj(c) * x + std::conj(s) * y;
  y = -s * x + c * y;
  x = t;
}

struct GmresWork {
  double2 *x = nullptr, *b = nullptr, *r = nullptr, *w = nullptr, *V = nullptr, *h = nullptr, *part = nullptr,
          *y = nullptr;
  std::vector<void*> owned;
  ~GmresWork() {
    for (void* p : owned) cudaFree(p);
  }
  double2* get(size_t count) {
    void* p = nullptr;
    MLFMA_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(double2)));
    owned.push_back(p);
    return static_cast<double2*>(p);
  }
};

}  // namespace

bool gmres_solve(Plan& P, double* xh, const double* rhs, int itr_max, int mr, double tol_abs, double tol_rel,
                 SolveStats& st, std::vector<double>& history) {
  if (mr > 63) throw std::invalid_argument("mr above 63 is not supported");
  const auto t0 = std::chrono::steady_clock::now();
  MLFMA_CUDA(cudaSetDevice(P.device));
  cudaStream_t s = P.stream;
  const long long n = 2LL * P.N;
  const int ldp = mr + 2;
  GmresWork g;
  g.x = g.get(n);
  g.b = g.get(n);
  g.r = g.get(n);
  g.w = g.get(n);
  g.V = g.get(static_cast<size_t>(mr + 1) * n);
  g.h = g.get(2 * (mr + 2));
  g.part = g.get(static_cast<size_t>(kRB) * ldp);
  g.y = g.get(mr + 1);
  MLFMA_CUDA(cudaMemcpyAsync(g.x, xh, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(g.b, rhs, n * sizeof(double2), cudaMemcpyHostToDevice, s));
  st = SolveStats();
  history.clear();

  auto norm_of = [&](const double2* v) {
    norm_kernel<<<kRB, kRT, 0, s>>>(v, n, g.part);
    reduce_kernel<<<1, 64, 0, s>>>(g.part, kRB, 1, 1, g.h);
    C out;
    MLFMA_CUDA(cudaMemcpyAsync(&out, g.h, sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(out.real());
  };
  auto true_residual = [&]() {
    apply_device(P, g.x, g.w, s);
    st.matvecs++;
    residual_kernel<<<kRB, kRT, 0, s>>>(g.b, g.w, g.r, n, g.part);
    reduce_kernel<<<1, 64, 0, s>>>(g.part, kRB, 1, 1, g.h);
    C out;
    MLFMA_CUDA(cudaMemcpyAsync(&out, g.h, sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(out.real());
  };
  auto finish = [&](bool ok, double err) {
    MLFMA_CUDA(cudaMemcpyAsync(xh, g.x, n * sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    st.rel_residual = err;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return ok;
  };

  const double eps = 1e-16;
  double rnorm = true_residual();
  double bnorm = norm_of(g.b);
  if (bnorm < eps) bnorm = 1.0;
  double error = rnorm / bnorm;
  if (error < tol_rel || error < tol_abs) return finish(true, error);

  const int ld = mr + 1;
  std::vector<C> H(static_cast<size_t>(ld) * mr), cs(mr), sn(mr), sv(mr + 1), y(mr);
  std::vector<C> h1, h2;
  int total = 0;
  for (int cycle = 1; cycle <= itr_max; ++cycle) {
    st.restarts = cycle;
    scale_kernel<<<kRB, kRT, 0, s>>>(g.r, 1.0 / rnorm, g.V, n);
    std::fill(sv.begin(), sv.end(), C(0.0));
    sv[0] = rnorm;
    std::fill(H.begin(), H.end(), C(0.0));
    std::fill(cs.begin(), cs.end(), C(0.0));
    std::fill(sn.begin(), sn.end(), C(0.0));
    int k_used = 0;
    for (int k = 0; k < mr; ++k) {
      if (total >= itr_max) break;
      ++total;
      k_used = k + 1;
      apply_device(P, g.V + static_cast<long long>(k) * n, g.w, s);
      st.matvecs++;
      const int nv = k + 1;
      // first projection
      dots_kernel<<<kRB, kRT, 0, s>>>(g.V, n, nv, g.w, g.part, ldp);
      reduce_kernel<<<(nv + 63) / 64, 64, 0, s>>>(g.part, kRB, ldp, nv, g.h);
      update_kernel<<<kRB, kRT, 0, s>>>(g.V, n, nv, g.h, g.w, 0, g.part, ldp);
      h1.resize(nv);
      MLFMA_CUDA(cudaMemcpyAsync(h1.data(), g.h, nv * sizeof(double2), cudaMemcpyDeviceToHost, s));
      // re-projection
      dots_kernel<<<kRB, kRT, 0, s>>>(g.V, n, nv, g.w, g.part, ldp);
      reduce_kernel<<<(nv + 63) / 64, 64, 0, s>>>(g.part, kRB, ldp, nv, g.h + ldp);
      update_kernel<<<kRB, kRT, 0, s>>>(g.V, n, nv, g.h + ldp, g.w, 1, g.part, ldp);
      reduce_kernel<<<1, 64, 0, s>>>(g.part, kRB, ldp, 1, g.h + 2 * ldp - 1);
      h2.resize(nv + 1);
      MLFMA_CUDA(cudaMemcpyAsync(h2.data(), g.h + ldp, nv * sizeof(double2), cudaMemcpyDeviceToHost, s));
      MLFMA_CUDA(cudaMemcpyAsync(&h2[nv], g.h + 2 * ldp - 1, sizeof(double2), cudaMemcpyDeviceToHost, s));
      MLFMA_CUDA(cudaStreamSynchronize(s));
      for (int j = 0; j <= k; ++j) H[j + static_cast<size_t>(k) * ld] = h1[j] + h2[j];
      const double h_next = std::sqrt(h2[nv].real());
      H[k + 1 + static_cast<size_t>(k) * ld] = h_next;
      if (h_next < eps * rnorm) break;  // Krylov space exhausted (Code/GMRES.h:136-139)
      scale_kernel<<<kRB, kRT, 0, s>>>(g.w, 1.0 / h_next, g.V + static_cast<long long>(k + 1) * n, n);
      for (int j = 0; j < k; ++j) givens_apply(H[j + k * ld], H[j + 1 + k * ld], cs[j], sn[j]);
      givens_make(H[k + k * ld], H[k + 1 + k * ld], cs[k], sn[k]);
      givens_apply(H[k + k * ld], H[k + 1 + k * ld], cs[k], sn[k]);
      H[k + 1 + k * ld] = C(0.0);
      givens_apply(sv[k], sv[k + 1], cs[k], sn[k]);
      error = std::abs(sv[k + 1]) / bnorm;
      history.push_back(error);
      if (error < tol_rel || error < tol_abs) break;
    }
    // upper-triangular solve (Code/GMRES.h:165-182)
    const int m = std::min(k_used, mr);
    for (int i = m - 1; i >= 0; --i) {
      y[i] = sv[i];
      for (int j = i + 1; j < m; ++j) y[i] -= H[i + j * ld] * y[j];
      if (std::abs(H[i + i * ld]) > eps)
        y[i] /= H[i + i * ld];
      else
        y[i] = C(0.0);
    }
    if (m > 0) {
      MLFMA_CUDA(cudaMemcpyAsync(g.y, y.data(), m * sizeof(double2), cudaMemcpyHostToDevice, s));
      combine_kernel<<<kRB, kRT, 0, s>>>(g.V, n, m, g.y, g.x);
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

// ------------------------------------------------------------------- RHS ----

namespace {

struct RhsArg {
  const double* xyz;
  const int* face_v;
  const int* fpos;
  const int* fneg;
  const int* vpos;
  const int* vneg;
  const double* len;
  int nq;
  double l1[16], l2[16], l3[16], w[16];
  double kinc[3], einc[3], hinc[3];
  double2 k1;
  int N;
};

__global__ void rhs_kernel(RhsArg a, double2* __restrict__ V) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.N) return;
  const double lm = a.len[m];
  double2 ve = c2(0, 0), vh = c2(0, 0);
  for (int i = 0; i < a.nq; ++i) {
    for (int side = 0; side < 2; ++side) {
      const int f = side ? a.fneg[m] : a.fpos[m];
      const double* A = &a.xyz[3 * a.face_v[3 * f]];
      const double* B = &a.xyz[3 * a.face_v[3 * f + 1]];
      const double* Cc = &a.xyz[3 * a.face_v[3 * f + 2]];
      const double* fv = &a.xyz[3 * (side ? a.vneg[m] : a.vpos[m])];
      double rr[3], rho[3];
      for (int c = 0; c < 3; ++c) {
        rr[c] = a.l1[i] * A[c] + a.l2[i] * B[c] + a.l3[i] * Cc[c];
        rho[c] = side ? fv[c] - rr[c] : rr[c] - fv[c];
      }
      const double2 e = cexp_mjkt(a.k1, a.kinc[0] * rr[0] + a.kinc[1] * rr[1] + a.kinc[2] * rr[2]);
      const double de = a.einc[0] * rho[0] + a.einc[1] * rho[1] + a.einc[2] * rho[2];
      const double dh = a.hinc[0] * rho[0] + a.hinc[1] * rho[1] + a.hinc[2] * rho[2];
      ve = cadd(ve, cscale(e, lm * a.w[i] * de));
      vh = cadd(vh, cscale(e, lm * a.w[i] * dh));
    }
  }
  V[m] = ve;
  V[a.N + m] = vh;
}

struct RcsArg {
  const double* xyz;
  const int* face_v;
  const int* fpos;
  const int* fneg;
  const int* vpos;
  const int* vneg;
  const double* len;
  int nq;
  double l1[16], l2[16], l3[16], w[16];
  double2 k1;
  int N;
};

// one block per direction; threads over RWGs; out[3] complex per direction
__global__ void __launch_bounds__(256) rcs_kernel(RcsArg a, const double* __restrict__ rdir,
                                                  const double2* __restrict__ I, double2* __restrict__ out) {
  __shared__ double2 sh[8];
  const double r[3] = {rdir[3 * blockIdx.x], rdir[3 * blockIdx.x + 1], rdir[3 * blockIdx.x + 2]};
  const double2 coeff = c2(a.k1.y, -a.k1.x);  // -j k1
  double2 acc[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
  for (int m = threadIdx.x; m < a.N; m += blockDim.x) {
    const double ln = a.len[m];
    double2 FJ[3] = {c2(0, 0), c2(0, 0), c2(0, 0)}, FM[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
    for (int i = 0; i < a.nq; ++i) {
      for (int side = 0; side < 2; ++side) {
        const int f = side ? a.fneg[m] : a.fpos[m];
        const double* A = &a.xyz[3 * a.face_v[3 * f]];
        const double* B = &a.xyz[3 * a.face_v[3 * f + 1]];
        const double* Cc = &a.xyz[3 * a.face_v[3 * f + 2]];
        const double* fv = &a.xyz[3 * (side ? a.vneg[m] : a.vpos[m])];
        double p[3], rho[3];
        for (int c = 0; c < 3; ++c) {
          p[c] = a.l1[i] * A[c] + a.l2[i] * B[c] + a.l3[i] * Cc[c];
          rho[c] = side ? fv[c] - p[c] : p[c] - fv[c];
        }
        // exp(+j k1 rhat.p)
        const double t = p[0] * r[0] + p[1] * r[1] + p[2] * r[2];
        const double2 e = cexp(make_double2(-a.k1.y * t, a.k1.x * t));
        const double rr = r[0] * rho[0] + r[1] * rho[1] + r[2] * rho[2];
        const double Ft[3] = {rho[0] - r[0] * rr, rho[1] - r[1] * rr, rho[2] - r[2] * rr};
        const double Fm[3] = {r[1] * rho[2] - r[2] * rho[1], r[2] * rho[0] - r[0] * rho[2],
                              r[0] * rho[1] - r[1] * rho[0]};
        const double wf = ln * a.w[i];
        for (int c = 0; c < 3; ++c) {
          FJ[c] = cadd(FJ[c], cscale(e, wf * Ft[c]));
          FM[c] = cadd(FM[c], cscale(e, wf * Fm[c]));
        }
      }
    }
    const double2 IJ = I[m], IM = I[a.N + m];
    for (int c = 0; c < 3; ++c) {
      acc[c] = csub(acc[c], cmul(cmul(coeff, FJ[c]), IJ));
      acc[c] = cadd(acc[c], cmul(cmul(coeff, FM[c]), IM));
    }
  }
  for (int c = 0; c < 3; ++c) {
    const double2 v = block_sum(acc[c], sh);
    if (threadIdx.x == 0) out[3 * blockIdx.x + c] = v;
  }
}

template <class A>
void fill_common(const Plan& P, A& a) {
  a.xyz = P.d_xyz;
  a.face_v = P.d_face_v;
  a.fpos = P.d_rwg_fpos;
  a.fneg = P.d_rwg_fneg;
  a.vpos = P.d_rwg_vpos;
  a.vneg = P.d_rwg_vneg;
  a.len = P.d_rwg_len;
  a.nq = P.quad.n;
  for (int i = 0; i < P.quad.n; ++i) {
    a.l1[i] = P.quad.l1[i];
    a.l2[i] = P.quad.l2[i];
    a.l3[i] = P.quad.l3[i];
    a.w[i] = P.quad.w[i];
  }
  a.k1 = make_double2(P.k1.real(), P.k1.imag());
  a.N = P.N;
}

}  // namespace

void rhs_pmchwt(Plan& P, const double kinc[3], const double einc[3], const double hinc[3], double* V) {
  MLFMA_CUDA(cudaSetDevice(P.device));
  RhsArg a{};
  fill_common(P, a);
  for (int c = 0; c < 3; ++c) {
    a.kinc[c] = kinc[c];
    a.einc[c] = einc[c];
    a.hinc[c] = hinc[c];
  }
  // into the plan's staging vector for host-pointer applies (one call in flight per plan)
  rhs_kernel<<<(P.N + 127) / 128, 128, 0, P.stream>>>(a, P.d_w);
  MLFMA_CUDA(cudaGetLastError());
  MLFMA_CUDA(cudaMemcpyAsync(V, P.d_w, 2 * static_cast<size_t>(P.N) * sizeof(double2), cudaMemcpyDeviceToHost,
                             P.stream));
  MLFMA_CUDA(cudaStreamSynchronize(P.stream));
}

void rcs_pmchwt(Plan& P, const double* I, int n_angles, const double* theta_deg, const double* phi_deg,
                double* field, double* rcs_db) {
  if (n_angles == 0) return;
  MLFMA_CUDA(cudaSetDevice(P.device));
  RcsArg a{};
  fill_common(P, a);
  std::vector<double> rdir(3 * static_cast<size_t>(n_angles));
  for (int i = 0; i < n_angles; ++i) {
    // Code/RCS.h:120-123
    const double th = (theta_deg[i] / 180.0) * kPi, ph = (phi_deg[i] / 180.0) * kPi;
    rdir[3 * i] = std::sin(th) * std::cos(ph);
    rdir[3 * i + 1] = std::sin(th) * std::sin(ph);
    rdir[3 * i + 2] = std::cos(th);
  }
  double *d_r = nullptr;
  double2 *d_I = nullptr, *d_o = nullptr;
  MLFMA_CUDA(cudaMalloc(&d_r, rdir.size() * sizeof(double)));
  MLFMA_CUDA(cudaMalloc(&d_I, 2 * static_cast<size_t>(P.N) * sizeof(double2)));
  MLFMA_CUDA(cudaMalloc(&d_o, 3 * static_cast<size_t>(n_angles) * sizeof(double2)));
  std::vector<double2> out(3 * static_cast<size_t>(n_angles));
  cudaError_t e = cudaMemcpyAsync(d_r, rdir.data(), rdir.size() * sizeof(double), cudaMemcpyHostToDevice, P.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_I, I, 2 * static_cast<size_t>(P.N) * sizeof(double2), cudaMemcpyHostToDevice, P.stream);
  if (e == cudaSuccess) {
    rcs_kernel<<<n_angles, 256, 0, P.stream>>>(a, d_r, d_I, d_o);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out.data(), d_o, out.size() * sizeof(double2), cudaMemcpyDeviceToHost, P.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(P.stream);
  cudaFree(d_r);
  cudaFree(d_I);
  cudaFree(d_o);
  MLFMA_CUDA(e);
  for (int i = 0; i < n_angles; ++i) {
    if (field)
      for (int c = 0; c < 3; ++c) {
        field[6 * i + 2 * c] = out[3 * i + c].x;
        field[6 * i + 2 * c + 1] = out[3 * i + c].y;
      }
    if (rcs_db) {
      // theta-hat / phi-hat of EMSource::initPW (Code/EMSource.cpp:34-59):
      // degrees to radians with |a| < 1e-6 snapped to 0, components snapped too.
      auto snap = [](double v) { return std::abs(v) < 1e-6 ? 0.0 : v; };
      const double th = snap(theta_deg[i] * kPi / 180.0), ph = snap(phi_deg[i] * kPi / 180.0);
      const double vt[3] = {snap(-std::cos(th) * std::cos(ph)), snap(-std::cos(th) * std::sin(ph)), snap(std::sin(th))};
      const double vp[3] = {snap(-std::sin(ph)), snap(std::cos(ph)), 0.0};
      const C E[3] = {C(out[3 * i].x, out[3 * i].y), C(out[3 * i + 1].x, out[3 * i + 1].y),
                      C(out[3 * i + 2].x, out[3 * i + 2].y)};
      const C Ev = vt[0] * E[0] + vt[1] * E[1] + vt[2] * E[2];
      const C Eh = vp[0] * E[0] + vp[1] * E[1] + vp[2] * E[2];
      rcs_db[3 * i] = 10.0 * std::log10((std::norm(Ev) + std::norm(Eh)) / (4.0 * kPi));
      rcs_db[3 * i + 1] = 10.0 * std::log10(std::norm(Ev) / (4.0 * kPi));
      rcs_db[3 * i + 2] = 10.0 * std::log10(std::norm(Eh) / (4.0 * kPi));
    }
  }
}

}  // namespace mlfma

// ------------------------------------------------ far field without allocation
//
// mlfma_rcs_pmchwt_noalloc: the far-field evaluation for callers that cannot
// allocate device memory while they run. Examples are an application that
// reserves all device memory up front in its own pool, and a real-time loop
// where a cudaMalloc/cudaFree (and the device synchronisation it can imply)
// is not allowed. Its only scratch is the angle table below, a file-scope
// device array that every GPU loading this library holds until exit.
namespace mlfma {
namespace {

constexpr int kNoAllocMaxAngles = 8192;  // 2 x 8192 doubles = 128 KiB

// [0, max): theta in degrees, [max, 2 max): phi in degrees
static __device__ __align__(256) double g_rcs_angle_scratch[2 * kNoAllocMaxAngles];

// Host-side device address of g_rcs_angle_scratch, looked up once per device
// with that device current (the symbol's name on the host is only a
// stand-in, not a device address).
double* g_rcs_scratch_addr[64] = {nullptr};
std::mutex g_rcs_scratch_mutex;

__global__ void __launch_bounds__(256) rcs_angles_kernel(RcsArg a, const double* __restrict__ angles, int max_angles,
                                                         const double2* __restrict__ I, double2* __restrict__ out);

// Set-up on the first call on a device (that device current): the address,
// and the kernel's function attributes, which makes a lazily loading runtime
// load the kernel now rather than at the first launch with angles.
double* rcs_scratch_address(int device) {
  if (device < 0 || device >= 64) throw std::invalid_argument("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_rcs_scratch_mutex);
  if (!g_rcs_scratch_addr[device]) {
    void* p = nullptr;
    MLFMA_CUDA(cudaGetSymbolAddress(&p, g_rcs_angle_scratch));
    cudaFuncAttributes fa{};
    MLFMA_CUDA(cudaFuncGetAttributes(&fa, rcs_angles_kernel));
    g_rcs_scratch_addr[device] = static_cast<double*>(p);
  }
  return g_rcs_scratch_addr[device];
}

// Makes a device current for the lifetime of the object and gives the
// caller's current device back afterwards.
class CurrentDevice {
 public:
  explicit CurrentDevice(int device) {
    MLFMA_CUDA(cudaGetDevice(&prev_));
    if (prev_ != device) MLFMA_CUDA(cudaSetDevice(device));
  }
  ~CurrentDevice() { cudaSetDevice(prev_); }
  CurrentDevice(const CurrentDevice&) = delete;
  CurrentDevice& operator=(const CurrentDevice&) = delete;

 private:
  int prev_ = 0;
};

// Same accumulation as rcs_kernel; the direction of block b is formed from
// the angles held in the scratch array.
__global__ void __launch_bounds__(256) rcs_angles_kernel(RcsArg a, const double* __restrict__ angles, int max_angles,
                                                         const double2* __restrict__ I, double2* __restrict__ out) {
  __shared__ double2 sh[8];
  const double th = (angles[blockIdx.x] / 180.0) * 3.14159265358979323846;
  const double ph = (angles[max_angles + blockIdx.x] / 180.0) * 3.14159265358979323846;
  const double r[3] = {sin(th) * cos(ph), sin(th) * sin(ph), cos(th)};
  const double2 coeff = c2(a.k1.y, -a.k1.x);  // -j k1
  double2 acc[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
  for (int m = threadIdx.x; m < a.N; m += blockDim.x) {
    const double ln = a.len[m];
    double2 FJ[3] = {c2(0, 0), c2(0, 0), c2(0, 0)}, FM[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
    for (int i = 0; i < a.nq; ++i) {
      for (int side = 0; side < 2; ++side) {
        const int f = side ? a.fneg[m] : a.fpos[m];
        const double* A = &a.xyz[3 * a.face_v[3 * f]];
        const double* B = &a.xyz[3 * a.face_v[3 * f + 1]];
        const double* Cc = &a.xyz[3 * a.face_v[3 * f + 2]];
        const double* fv = &a.xyz[3 * (side ? a.vneg[m] : a.vpos[m])];
        double p[3], rho[3];
        for (int c = 0; c < 3; ++c) {
          p[c] = a.l1[i] * A[c] + a.l2[i] * B[c] + a.l3[i] * Cc[c];
          rho[c] = side ? fv[c] - p[c] : p[c] - fv[c];
        }
        const double t = p[0] * r[0] + p[1] * r[1] + p[2] * r[2];
        const double2 e = cexp(make_double2(-a.k1.y * t, a.k1.x * t));
        const double rr = r[0] * rho[0] + r[1] * rho[1] + r[2] * rho[2];
        const double Ft[3] = {rho[0] - r[0] * rr, rho[1] - r[1] * rr, rho[2] - r[2] * rr};
        const double Fm[3] = {r[1] * rho[2] - r[2] * rho[1], r[2] * rho[0] - r[0] * rho[2],
                              r[0] * rho[1] - r[1] * rho[0]};
        const double wf = ln * a.w[i];
        for (int c = 0; c < 3; ++c) {
          FJ[c] = cadd(FJ[c], cscale(e, wf * Ft[c]));
          FM[c] = cadd(FM[c], cscale(e, wf * Fm[c]));
        }
      }
    }
    const double2 IJ = I[m], IM = I[a.N + m];
    for (int c = 0; c < 3; ++c) {
      acc[c] = csub(acc[c], cmul(cmul(coeff, FJ[c]), IJ));
      acc[c] = cadd(acc[c], cmul(cmul(coeff, FM[c]), IM));
    }
  }
  for (int c = 0; c < 3; ++c) {
    const double2 v = block_sum(acc[c], sh);
    if (threadIdx.x == 0) out[3 * blockIdx.x + c] = v;
  }
}

}  // namespace

int rcs_noalloc_max_angles() { return kNoAllocMaxAngles; }

void rcs_pmchwt_noalloc(Plan& P, const double2* I_dev, int n_angles, const double* theta_deg,
                        const double* phi_deg, double2* field_dev, cudaStream_t s) {
  if (n_angles < 0 || n_angles > kNoAllocMaxAngles)
    throw std::invalid_argument("n_angles must be between 0 and " + std::to_string(kNoAllocMaxAngles) +
                                " (size of the fixed angle scratch)");
  CurrentDevice current(P.device);
  double* scratch = rcs_scratch_address(P.device);
  if (n_angles == 0) return;
  MLFMA_CUDA(cudaMemcpyAsync(scratch, theta_deg, n_angles * sizeof(double), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(scratch + kNoAllocMaxAngles, phi_deg, n_angles * sizeof(double),
                             cudaMemcpyHostToDevice, s));
  RcsArg a{};
  fill_common(P, a);
  rcs_angles_kernel<<<n_angles, 256, 0, s>>>(a, scratch, kNoAllocMaxAngles, I_dev, field_dev);
  MLFMA_CUDA(cudaGetLastError());
}

}  // namespace mlfma
