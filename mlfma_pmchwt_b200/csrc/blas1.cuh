// Length-n complex128 vector kernels (internal linkage: one copy per including
// file) for the Krylov solvers: Gram-Schmidt
// projections against a block of basis vectors, updates, norms. Reductions
// are two-stage (per-block partials, then one deterministic sum), so results
// do not depend on scheduling.
#pragma once
#include <cuda_runtime.h>

#include <complex>
#include <vector>

#include "cplx.cuh"
#include "plan.hpp"

namespace mlfma {
namespace blas1 {

constexpr int kBlocks = 592;   // 4 per SM
constexpr int kThreads = 256;
constexpr int kTile = 8;       // basis vectors per pass of dots
constexpr int kMaxBasis = 64;  // largest basis a projection may use

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

// partial[blk * ldp + j] = sum over the block's rows of conj(V_j) w, j < nv
static __global__ void __launch_bounds__(kThreads) dots(const double2* __restrict__ V, long long n, int nv,
                                                 const double2* __restrict__ w, double2* __restrict__ partial,
                                                 int ldp) {
  __shared__ double2 sh[kThreads / 32];
  for (int j0 = 0; j0 < nv; j0 += kTile) {
    double2 acc[kTile];
#pragma unroll
    for (int q = 0; q < kTile; ++q) acc[q] = c2(0.0, 0.0);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
      const double2 wi = w[i];
#pragma unroll
      for (int q = 0; q < kTile; ++q)
        if (j0 + q < nv) {
          const double2 v = V[(long long)(j0 + q) * n + i];
          acc[q].x = fma(v.x, wi.x, fma(v.y, wi.y, acc[q].x));
          acc[q].y = fma(v.x, wi.y, fma(-v.y, wi.x, acc[q].y));
        }
    }
#pragma unroll
    for (int q = 0; q < kTile; ++q)
      if (j0 + q < nv) {
        const double2 s = block_sum(acc[q], sh);
        if (threadIdx.x == 0) partial[(long long)blockIdx.x * ldp + j0 + q] = s;
      }
  }
}

// out[j] = sum over blocks of partial[blk * ldp + j]
static __global__ void reduce(const double2* __restrict__ partial, int nblk, int ldp, int nv, double2* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nv) return;
  double2 s = c2(0.0, 0.0);
  for (int b = 0; b < nblk; ++b) s = cadd(s, partial[(long long)b * ldp + j]);
  out[j] = s;
}

// w -= sum_j V_j h[j]; optionally the block partials of ||w||^2 into partial[blk * ldp]
static __global__ void __launch_bounds__(kThreads) project_out(const double2* __restrict__ V, long long n, int nv,
                                                        const double2* __restrict__ h, double2* __restrict__ w,
                                                        int want_norm, double2* __restrict__ partial, int ldp) {
  __shared__ double2 hs[kMaxBasis];
  __shared__ double2 sh[kThreads / 32];
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

// block partials of ||v||^2 (or of ||b - w||^2 with r = b - w written when b != null)
static __global__ void __launch_bounds__(kThreads) norm2(const double2* __restrict__ b, const double2* __restrict__ w,
                                                  double2* __restrict__ r, long long n, double2* __restrict__ partial) {
  __shared__ double2 sh[kThreads / 32];
  double2 nrm = c2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 v = w[i];
    if (b) {
      v = csub(b[i], v);
      r[i] = v;
    }
    nrm.x = fma(v.x, v.x, fma(v.y, v.y, nrm.x));
  }
  const double2 s = block_sum(nrm, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

static __global__ void scale(const double2* __restrict__ src, double a, double2* __restrict__ dst, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = cscale(src[i], a);
}

// x (+)= sum_j V_j y[j]   (accumulate != 0: add to x, else overwrite)
static __global__ void combine(const double2* __restrict__ V, long long n, int m, const double2* __restrict__ y,
                        double2* __restrict__ x, int accumulate) {
  __shared__ double2 ys[kMaxBasis];
  for (int j = threadIdx.x; j < m; j += blockDim.x) ys[j] = y[j];
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 xi = accumulate ? x[i] : c2(0.0, 0.0);
    for (int j = 0; j < m; ++j) xi = cfma(ys[j], V[(long long)j * n + i], xi);
    x[i] = xi;
  }
}

// Device work arrays owned by one solve.
struct Work {
  std::vector<void*> owned;
  ~Work() {
    for (void* p : owned) cudaFree(p);
  }
  double2* get(size_t count) {
    void* p = nullptr;
    MLFMA_CUDA(cudaMalloc(&p, (count ? count : 1) * sizeof(double2)));
    owned.push_back(p);
    return static_cast<double2*>(p);
  }
};

// Host side of two-stage reductions and Gram-Schmidt, on one stream.
struct Ops {
  cudaStream_t s;
  long long n;
  double2* part;   // [kBlocks * ldp]
  int ldp;
  double2* h;      // device scratch for reduced values, >= 2 * ldp + 2

  // ||v||
  double norm(const double2* v) {
    norm2<<<kBlocks, kThreads, 0, s>>>(nullptr, v, nullptr, n, part);
    reduce<<<1, 64, 0, s>>>(part, kBlocks, 1, 1, h);
    std::complex<double> o;
    MLFMA_CUDA(cudaMemcpyAsync(&o, h, sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(o.real());
  }
  // r = b - w, returns ||r||
  double residual(const double2* b, const double2* w, double2* r) {
    norm2<<<kBlocks, kThreads, 0, s>>>(b, w, r, n, part);
    reduce<<<1, 64, 0, s>>>(part, kBlocks, 1, 1, h);
    std::complex<double> o;
    MLFMA_CUDA(cudaMemcpyAsync(&o, h, sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(o.real());
  }
  // Classical Gram-Schmidt twice of w against V[0..nv): hcol[j] = sum of both
  // passes' coefficients, returns ||w|| after projection.
  double orthogonalise(const double2* V, int nv, double2* w, std::vector<std::complex<double>>& hcol) {
    dots<<<kBlocks, kThreads, 0, s>>>(V, n, nv, w, part, ldp);
    reduce<<<(nv + 63) / 64, 64, 0, s>>>(part, kBlocks, ldp, nv, h);
    project_out<<<kBlocks, kThreads, 0, s>>>(V, n, nv, h, w, 0, part, ldp);
    dots<<<kBlocks, kThreads, 0, s>>>(V, n, nv, w, part, ldp);
    reduce<<<(nv + 63) / 64, 64, 0, s>>>(part, kBlocks, ldp, nv, h + ldp);
    project_out<<<kBlocks, kThreads, 0, s>>>(V, n, nv, h + ldp, w, 1, part, ldp);
    reduce<<<1, 64, 0, s>>>(part, kBlocks, ldp, 1, h + 2 * ldp);
    std::vector<std::complex<double>> buf(2 * ldp + 1);
    MLFMA_CUDA(cudaMemcpyAsync(buf.data(), h, (2 * ldp + 1) * sizeof(double2), cudaMemcpyDeviceToHost, s));
    MLFMA_CUDA(cudaStreamSynchronize(s));
    hcol.resize(nv);
    for (int j = 0; j < nv; ++j) hcol[j] = buf[j] + buf[ldp + j];
    return std::sqrt(buf[2 * ldp].real());
  }
};

}  // namespace blas1
}  // namespace mlfma

namespace mlfma {
namespace blas1 {

// Complex Givens rotation as MGMRES builds and applies it (Code/GMRES.h:22-48).
inline void givens_make(std::complex<double> a, std::complex<double> b, std::complex<double>& c,
                        std::complex<double>& s) {
  const double eps = 1e-16;
  if (std::abs(b) < eps) {
    c = 1.0;
    s = 0.0;
  } else if (std::abs(a) < eps) {
    c = 0.0;
    s = 1.0;
  } else {
    const double r = std::sqrt(std::real(a * std::conj(a) + b * std::conj(b)));
    c = a / r;
    s = b / r;
  }
}
inline void givens_apply(std::complex<double>& x, std::complex<double>& y, std::complex<double> c,
                         std::complex<double> s) {
  const std::complex<double> t = std::conj(c) * x + std::conj(s) * y;
  y = -s * x + c * y;
  x = t;
}

// The same rotations on the device, for the inner GMRES steps that run
// without a host round trip.
__device__ __forceinline__ double2 dconj(double2 a) { return c2(a.x, -a.y); }
__device__ inline void dgivens_make(double2 a, double2 b, double2& c, double2& s) {
  const double eps = 1e-16;
  if (sqrt(b.x * b.x + b.y * b.y) < eps) {
    c = c2(1.0, 0.0);
    s = c2(0.0, 0.0);
  } else if (sqrt(a.x * a.x + a.y * a.y) < eps) {
    c = c2(0.0, 0.0);
    s = c2(1.0, 0.0);
  } else {
    const double r = sqrt(a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y);
    c = c2(a.x / r, a.y / r);
    s = c2(b.x / r, b.y / r);
  }
}
__device__ inline void dgivens_apply(double2& x, double2& y, double2 c, double2 s) {
  const double2 t = cadd(cmul(dconj(c), x), cmul(dconj(s), y));
  y = cadd(cmul(c2(-s.x, -s.y), x), cmul(c, y));
  x = t;
}

}  // namespace blas1
}  // namespace mlfma
