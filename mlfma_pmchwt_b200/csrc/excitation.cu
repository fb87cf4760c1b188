// Many incidences at once: the plane-wave excitation of R incidences
// (RHS::computeV_PMCHWT, Code/Vm.h:150-203, with the incident vectors of
// EMSource::initPW, Code/EMSource.cpp:34-72) and the far field of R current
// vectors, bistatic (Code/RCS.h:116-192 per solution and angle, the
// dual-static study Code/RCS.h:345-425) or monostatic (each solution seen
// from its own backscatter angle, the mono-static loop Code/RCS.h:436-494).
//
// The reference runs these once per incidence inside its study loops; here
// one launch covers a chunk of incidences. The incidence and angle tables
// travel in the kernel parameters (read at launch), so the entry points
// allocate nothing and accept pageable or pinned host tables alike.
// Quadrature points are formed once per (RWG, point) and reused for every
// incidence of a chunk.
#include <cmath>
#include <stdexcept>

#include "cplx.cuh"
#include "solver.hpp"

namespace mlfma {
namespace {

constexpr int kRhsChunk = 128;   // incidences per excitation launch (9 KB of parameters)
constexpr int kRhsTile = 8;      // incidences per thread (grid.y tiles)
constexpr int kFarChunk = 256;   // angles per bistatic launch (6 KB of parameters)
constexpr int kFarTile = 4;      // solutions per block of the bistatic far field

struct Geo {
  const double* xyz;
  const int* face_v;
  const int* fpos;
  const int* fneg;
  const int* vpos;
  const int* vneg;
  const double* len;
  int nq, N;
  double l1[16], l2[16], l3[16], w[16];
  double2 k1;
};

Geo geo(const Plan& P) {
  Geo g{};
  g.xyz = P.d_xyz;
  g.face_v = P.d_face_v;
  g.fpos = P.d_rwg_fpos;
  g.fneg = P.d_rwg_fneg;
  g.vpos = P.d_rwg_vpos;
  g.vneg = P.d_rwg_vneg;
  g.len = P.d_rwg_len;
  g.nq = P.quad.n;
  g.N = P.N;
  for (int i = 0; i < P.quad.n; ++i) {
    g.l1[i] = P.quad.l1[i];
    g.l2[i] = P.quad.l2[i];
    g.l3[i] = P.quad.l3[i];
    g.w[i] = P.quad.w[i];
  }
  g.k1 = make_double2(P.k1.real(), P.k1.imag());
  return g;
}

// Quadrature point i of side `side` (0: T+, 1: T-) of RWG m: position p and
// the RWG vector rho (p - free vertex on T+, free vertex - p on T-).
__device__ __forceinline__ void rwg_point(const Geo& g, int m, int side, int i, double p[3], double rho[3]) {
  const int f = side ? g.fneg[m] : g.fpos[m];
  const double* A = &g.xyz[3 * g.face_v[3 * f]];
  const double* B = &g.xyz[3 * g.face_v[3 * f + 1]];
  const double* Cc = &g.xyz[3 * g.face_v[3 * f + 2]];
  const double* fv = &g.xyz[3 * (side ? g.vneg[m] : g.vpos[m])];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    p[c] = g.l1[i] * A[c] + g.l2[i] * B[c] + g.l3[i] * Cc[c];
    rho[c] = side ? fv[c] - p[c] : p[c] - fv[c];
  }
}

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

struct RhsBatchArg {
  Geo g;
  double inc[kRhsChunk][9];  // per incidence: kinc, einc, hinc
  int R;
  double2* V;                // [R][2N] for this chunk
};

// thread per RWG, kRhsTile incidences (blockIdx.y tile): V[r][m], V[r][N + m]
__global__ void __launch_bounds__(128) rhs_batch_kernel(const __grid_constant__ RhsBatchArg a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int r0 = blockIdx.y * kRhsTile;
  const Geo& g = a.g;
  if (m >= g.N) return;
  const int nr = min(kRhsTile, a.R - r0);
  const double lm = g.len[m];
  double2 ve[kRhsTile], vh[kRhsTile];
#pragma unroll
  for (int q = 0; q < kRhsTile; ++q) ve[q] = vh[q] = c2(0.0, 0.0);
  for (int i = 0; i < g.nq; ++i) {
    for (int side = 0; side < 2; ++side) {
      double p[3], rho[3];
      rwg_point(g, m, side, i, p, rho);
      const double wl = lm * g.w[i];
#pragma unroll
      for (int q = 0; q < kRhsTile; ++q) {
        if (q < nr) {
          const double* d = a.inc[r0 + q];
          const double2 e = cexp_mjkt(g.k1, d[0] * p[0] + d[1] * p[1] + d[2] * p[2]);
          const double de = d[3] * rho[0] + d[4] * rho[1] + d[5] * rho[2];
          const double dh = d[6] * rho[0] + d[7] * rho[1] + d[8] * rho[2];
          ve[q] = cadd(ve[q], cscale(e, wl * de));
          vh[q] = cadd(vh[q], cscale(e, wl * dh));
        }
      }
    }
  }
  const size_t n = 2 * static_cast<size_t>(g.N);
#pragma unroll
  for (int q = 0; q < kRhsTile; ++q)
    if (q < nr) {
      a.V[(r0 + q) * n + m] = ve[q];
      a.V[(r0 + q) * n + g.N + m] = vh[q];
    }
}

// The far-field factors of RWG m in direction r: F_J = sum l w (I - r r) rho
// e^{+j k1 r.p} and F_M = sum l w (r x rho) e^{+j k1 r.p} (Code/RCS.h:140-170).
__device__ __forceinline__ void far_factors(const Geo& g, int m, const double r[3], double2 FJ[3], double2 FM[3]) {
  const double ln = g.len[m];
#pragma unroll
  for (int c = 0; c < 3; ++c) FJ[c] = FM[c] = c2(0.0, 0.0);
  for (int i = 0; i < g.nq; ++i) {
    for (int side = 0; side < 2; ++side) {
      double p[3], rho[3];
      rwg_point(g, m, side, i, p, rho);
      const double t = p[0] * r[0] + p[1] * r[1] + p[2] * r[2];
      const double2 e = cexp(make_double2(-g.k1.y * t, g.k1.x * t));
      const double rr = r[0] * rho[0] + r[1] * rho[1] + r[2] * rho[2];
      const double Ft[3] = {rho[0] - r[0] * rr, rho[1] - r[1] * rr, rho[2] - r[2] * rr};
      const double Fm[3] = {r[1] * rho[2] - r[2] * rho[1], r[2] * rho[0] - r[0] * rho[2],
                            r[0] * rho[1] - r[1] * rho[0]};
      const double wf = ln * g.w[i];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        FJ[c] = cadd(FJ[c], cscale(e, wf * Ft[c]));
        FM[c] = cadd(FM[c], cscale(e, wf * Fm[c]));
      }
    }
  }
}

struct FarBatchArg {
  Geo g;
  double dir[kFarChunk][3];
  int n_angles, angle0, n_total_angles, R;
  const double2* I;  // [R][2N]
  double2* out;      // [R][n_total_angles][3]
};

// block per (angle, tile of kFarTile solutions): E = -j k1 (F_J . I_J - F_M . I_M)
__global__ void __launch_bounds__(256) far_batch_kernel(const __grid_constant__ FarBatchArg a) {
  __shared__ double2 sh[8];
  const Geo& g = a.g;
  const int ang = blockIdx.x;
  const int r0 = blockIdx.y * kFarTile;
  const int nr = min(kFarTile, a.R - r0);
  const double r[3] = {a.dir[ang][0], a.dir[ang][1], a.dir[ang][2]};
  const size_t n = 2 * static_cast<size_t>(g.N);
  double2 acc[kFarTile][3];
#pragma unroll
  for (int q = 0; q < kFarTile; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[q][c] = c2(0.0, 0.0);
  for (int m = threadIdx.x; m < g.N; m += blockDim.x) {
    double2 FJ[3], FM[3];
    far_factors(g, m, r, FJ, FM);
#pragma unroll
    for (int q = 0; q < kFarTile; ++q) {
      if (q < nr) {
        const double2 IJ = a.I[(r0 + q) * n + m], IM = a.I[(r0 + q) * n + g.N + m];
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[q][c] = cadd(acc[q][c], csub(cmul(FM[c], IM), cmul(FJ[c], IJ)));
      }
    }
  }
  const double2 coeff = c2(g.k1.y, -g.k1.x);  // -j k1 ... applied as -j k1 (-F_J I_J + F_M I_M)
#pragma unroll
  for (int q = 0; q < kFarTile; ++q)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 v = block_sum(acc[q][c], sh);
      if (threadIdx.x == 0 && q < nr)
        a.out[((r0 + q) * static_cast<size_t>(a.n_total_angles) + a.angle0 + ang) * 3 + c] = cmul(coeff, v);
    }
}

struct FarMonoArg {
  Geo g;
  double dir[kFarChunk][3];
  int r0;            // first solution of this chunk
  const double2* I;  // [R][2N]
  double2* out;      // [R][3]
};

// block per solution of the chunk, observed in its own direction
__global__ void __launch_bounds__(256) far_mono_kernel(const __grid_constant__ FarMonoArg a) {
  __shared__ double2 sh[8];
  const Geo& g = a.g;
  const int q = blockIdx.x;
  const double r[3] = {a.dir[q][0], a.dir[q][1], a.dir[q][2]};
  const double2* I = a.I + (a.r0 + q) * 2 * static_cast<size_t>(g.N);
  double2 acc[3] = {c2(0.0, 0.0), c2(0.0, 0.0), c2(0.0, 0.0)};
  for (int m = threadIdx.x; m < g.N; m += blockDim.x) {
    double2 FJ[3], FM[3];
    far_factors(g, m, r, FJ, FM);
    const double2 IJ = I[m], IM = I[g.N + m];
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = cadd(acc[c], csub(cmul(FM[c], IM), cmul(FJ[c], IJ)));
  }
  const double2 coeff = c2(g.k1.y, -g.k1.x);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 v = block_sum(acc[c], sh);
    if (threadIdx.x == 0) a.out[(a.r0 + q) * 3 + c] = cmul(coeff, v);
  }
}

// Code/RCS.h:120-123: observation direction of (theta, phi) in degrees
void direction(double theta_deg, double phi_deg, double r[3]) {
  const double th = (theta_deg / 180.0) * kPi, ph = (phi_deg / 180.0) * kPi;
  r[0] = std::sin(th) * std::cos(ph);
  r[1] = std::sin(th) * std::sin(ph);
  r[2] = std::cos(th);
}

}  // namespace

void rhs_pmchwt_batch(Plan& P, int R, const double* kinc, const double* einc, const double* hinc, double2* V_dev,
                      cudaStream_t s) {
  if (R <= 0) return;
  MLFMA_CUDA(cudaSetDevice(P.device));
  RhsBatchArg a{};
  a.g = geo(P);
  for (int c0 = 0; c0 < R; c0 += kRhsChunk) {
    a.R = std::min(kRhsChunk, R - c0);
    for (int q = 0; q < a.R; ++q)
      for (int c = 0; c < 3; ++c) {
        a.inc[q][c] = kinc[3 * (c0 + q) + c];
        a.inc[q][3 + c] = einc[3 * (c0 + q) + c];
        a.inc[q][6 + c] = hinc[3 * (c0 + q) + c];
      }
    a.V = V_dev + static_cast<size_t>(c0) * 2 * P.N;
    const dim3 grid((P.N + 127) / 128, (a.R + kRhsTile - 1) / kRhsTile);
    rhs_batch_kernel<<<grid, 128, 0, s>>>(a);
    MLFMA_CUDA(cudaGetLastError());
  }
}

void rcs_pmchwt_batch(Plan& P, int R, const double2* I_dev, int n_angles, const double* theta_deg,
                      const double* phi_deg, double2* field_dev, cudaStream_t s) {
  if (R <= 0 || n_angles <= 0) return;
  MLFMA_CUDA(cudaSetDevice(P.device));
  FarBatchArg a{};
  a.g = geo(P);
  a.R = R;
  a.I = I_dev;
  a.out = field_dev;
  a.n_total_angles = n_angles;
  for (int c0 = 0; c0 < n_angles; c0 += kFarChunk) {
    a.n_angles = std::min(kFarChunk, n_angles - c0);
    a.angle0 = c0;
    for (int q = 0; q < a.n_angles; ++q) direction(theta_deg[c0 + q], phi_deg[c0 + q], a.dir[q]);
    const dim3 grid(a.n_angles, (R + kFarTile - 1) / kFarTile);
    far_batch_kernel<<<grid, 256, 0, s>>>(a);
    MLFMA_CUDA(cudaGetLastError());
  }
}

void rcs_pmchwt_mono(Plan& P, int R, const double2* I_dev, const double* theta_deg, const double* phi_deg,
                     double2* field_dev, cudaStream_t s) {
  if (R <= 0) return;
  MLFMA_CUDA(cudaSetDevice(P.device));
  FarMonoArg a{};
  a.g = geo(P);
  a.I = I_dev;
  a.out = field_dev;
  for (int c0 = 0; c0 < R; c0 += kFarChunk) {
    const int nr = std::min(kFarChunk, R - c0);
    a.r0 = c0;
    for (int q = 0; q < nr; ++q) direction(theta_deg[c0 + q], phi_deg[c0 + q], a.dir[q]);
    far_mono_kernel<<<nr, 256, 0, s>>>(a);
    MLFMA_CUDA(cudaGetLastError());
  }
}

void rcs_db(int n_angles, const double* theta_deg, const double* phi_deg, const double* field, double* out) {
  for (int i = 0; i < n_angles; ++i) {
    // theta-hat / phi-hat of EMSource::initPW (Code/EMSource.cpp:34-59):
    // degrees to radians with |a| < 1e-6 snapped to 0, components snapped too;
    // dB as the dual-static study forms them (Code/RCS.h:391-410).
    auto snap = [](double v) { return std::abs(v) < 1e-6 ? 0.0 : v; };
    const double th = snap(theta_deg[i] * kPi / 180.0), ph = snap(phi_deg[i] * kPi / 180.0);
    const double vt[3] = {snap(-std::cos(th) * std::cos(ph)), snap(-std::cos(th) * std::sin(ph)), snap(std::sin(th))};
    const double vp[3] = {snap(-std::sin(ph)), snap(std::cos(ph)), 0.0};
    const cplx E[3] = {cplx(field[6 * i], field[6 * i + 1]), cplx(field[6 * i + 2], field[6 * i + 3]),
                       cplx(field[6 * i + 4], field[6 * i + 5])};
    const cplx Ev = vt[0] * E[0] + vt[1] * E[1] + vt[2] * E[2];
    const cplx Eh = vp[0] * E[0] + vp[1] * E[1] + vp[2] * E[2];
    out[3 * i] = 10.0 * std::log10((std::norm(Ev) + std::norm(Eh)) / (4.0 * kPi));
    out[3 * i + 1] = 10.0 * std::log10(std::norm(Ev) / (4.0 * kPi));
    out[3 * i + 2] = 10.0 * std::log10(std::norm(Eh) / (4.0 * kPi));
  }
}

}  // namespace mlfma
