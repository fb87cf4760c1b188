// Learned leaf-box preconditioner: forward pass (inference inside flexible
// GMRES), backward pass and Adam step (training). The network and its
// parameter layout are described in learned.hpp.
//
// Layout: per-RWG arrays in the plan's leaf order (position p; the RWG id is
// leaf_rwg[p], its box pos_box[p]) and per-box arrays in leaf-box order,
// both row-major [row][channel] so that a box's rows are contiguous.
// Sizes: N RWGs, B leaf boxes; everything is O(N * 64) floats.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

#include "cplx.cuh"
#include "learned.hpp"

namespace mlfma {

namespace {

constexpr int kRedBlocks = 256;
constexpr int kColParts = 64;     // partial column sums over boxes
constexpr int kLayerBoxes = 32;   // boxes per CTA in the layer kernels
constexpr int kDecRows = 32;      // RWGs per CTA in the decoder kernels
constexpr int kWgRows = 256;      // rows per CTA in the weight-gradient kernel

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }
__device__ __forceinline__ float2 f2(double2 a) {
  return make_float2(static_cast<float>(a.x), static_cast<float>(a.y));
}

// sum |a_k|^2 over k < n: per-block partials
__global__ void lp_sumsq_kernel(const double2* __restrict__ a, long long n, double* __restrict__ part) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += 256LL * gridDim.x)
    acc += a[i].x * a[i].x + a[i].y * a[i].y;
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// out[j] = sum of part[j * nblk .. (j + 1) * nblk), j < count
__global__ void lp_finalize_kernel(const double* __restrict__ part, int nblk, int count, double* __restrict__ out) {
  __shared__ double red[256];
  for (int j = 0; j < count; ++j) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < nblk; i += 256) acc += part[j * nblk + i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = red[0];
    __syncthreads();
  }
}

struct Tabs {
  int N, B;
  const int* ids;       // [N] leaf position -> RWG id
  const int* leaf_ptr;  // [B + 1]
  const int* pos_box;   // [N]
  const float* dip;     // [N][3] by leaf position
  const int* nb_ptr;    // [B + 1]: the box itself and its near neighbours
  const int* nb_idx;
  const float* fs;      // [N][16] static features by leaf position
};

// Zb[b][c][k] = mean over the box's RWGs of z_c d_k
__global__ void lp_boxz_kernel(Tabs t, const double2* __restrict__ z, float2* __restrict__ zb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= t.B) return;
  const int p0 = t.leaf_ptr[b], p1 = t.leaf_ptr[b + 1];
  float2 acc[6];
  for (int j = 0; j < 6; ++j) acc[j] = make_float2(0.f, 0.f);
  for (int p = p0; p < p1; ++p) {
    const int id = t.ids[p];
    const float2 zj = f2(z[id]), zm = f2(z[t.N + id]);
    for (int k = 0; k < 3; ++k) {
      const float d = t.dip[3 * p + k];
      acc[k] = make_float2(fmaf(zj.x, d, acc[k].x), fmaf(zj.y, d, acc[k].y));
      acc[3 + k] = make_float2(fmaf(zm.x, d, acc[3 + k].x), fmaf(zm.y, d, acc[3 + k].y));
    }
  }
  const float inv = p1 > p0 ? 1.f / static_cast<float>(p1 - p0) : 0.f;
  for (int j = 0; j < 6; ++j) zb[6 * b + j] = cscale(acc[j], inv);
}

// Zn[b] = mean of Zb over the box and its near neighbours (and, applied to
// Zn, the two-ring mean Z2)
__global__ void lp_boxn_kernel(Tabs t, const float2* __restrict__ zb, float2* __restrict__ zn) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= t.B) return;
  const int q0 = t.nb_ptr[b], q1 = t.nb_ptr[b + 1];
  float2 acc[6];
  for (int j = 0; j < 6; ++j) acc[j] = make_float2(0.f, 0.f);
  for (int q = q0; q < q1; ++q) {
    const int c = t.nb_idx[q];
    for (int j = 0; j < 6; ++j) acc[j] = cadd(acc[j], zb[6 * c + j]);
  }
  const float inv = 1.f / static_cast<float>(q1 - q0);
  for (int j = 0; j < 6; ++j) zn[6 * b + j] = cscale(acc[j], inv);
}

__device__ __forceinline__ float2 dot3(const float* d, const float2* zv) {
  return make_float2(d[0] * zv[0].x + d[1] * zv[1].x + d[2] * zv[2].x, d[0] * zv[0].y + d[1] * zv[1].y + d[2] * zv[2].y);
}

struct EncArg {
  Tabs t;
  const double2* z;
  const float2* zb;    // box, one-ring and two-ring dipole means of z
  const float2* zn;
  const float2* z2;
  const __nv_bfloat16* w;
  float2* u;           // [N][8]
  float* a;            // [N][64]
};

// Per RWG: the linear terms and the encoder layer (on the static features).
__global__ void __launch_bounds__(128) lp_encode_kernel(EncArg e) {
  __shared__ float We[kLpH * kLpF], be[kLpH];
  for (int i = threadIdx.x; i < kLpH * kLpF; i += blockDim.x) We[i] = bf(e.w, i);
  for (int i = threadIdx.x; i < kLpH; i += blockDim.x) be[i] = bf(e.w, kLpOffBe + i);
  __syncthreads();
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= e.t.N) return;
  const int N = e.t.N, id = e.t.ids[p], b = e.t.pos_box[p];
  const float d[3] = {e.t.dip[3 * p], e.t.dip[3 * p + 1], e.t.dip[3 * p + 2]};
  float2 u[kLpT];
  u[0] = f2(e.z[id]);
  u[1] = f2(e.z[N + id]);
  u[2] = dot3(d, e.z2 + 6 * b);
  u[3] = dot3(d, e.z2 + 6 * b + 3);
  u[4] = dot3(d, e.zb + 6 * b);
  u[5] = dot3(d, e.zb + 6 * b + 3);
  u[6] = dot3(d, e.zn + 6 * b);
  u[7] = dot3(d, e.zn + 6 * b + 3);
  for (int k = 0; k < kLpT; ++k) e.u[kLpT * p + k] = u[k];
  float f[kLpF];
  for (int k = 0; k < kLpF; ++k) f[k] = e.t.fs[kLpF * p + k];
  float* ar = e.a + static_cast<size_t>(kLpH) * p;
  for (int o = 0; o < kLpH; o += 4) {
    float4 r;
    float* rr = &r.x;
    for (int j = 0; j < 4; ++j) {
      float acc = be[o + j];
      for (int k = 0; k < kLpF; ++k) acc = fmaf(We[(o + j) * kLpF + k], f[k], acc);
      rr[j] = fmaxf(acc, 0.f);
    }
    *reinterpret_cast<float4*>(ar + o) = r;
  }
}

// h0[b] = mean over the box's RWGs of a; warp per box, 2 channels per lane
__global__ void lp_pool_kernel(Tabs t, const float* __restrict__ a, float* __restrict__ h0) {
  const int b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (b >= t.B) return;
  const int p0 = t.leaf_ptr[b], p1 = t.leaf_ptr[b + 1];
  float s0 = 0.f, s1 = 0.f;
  for (int p = p0; p < p1; ++p) {
    s0 += a[kLpH * p + lane];
    s1 += a[kLpH * p + 32 + lane];
  }
  const float inv = p1 > p0 ? 1.f / static_cast<float>(p1 - p0) : 0.f;
  h0[kLpH * b + lane] = s0 * inv;
  h0[kLpH * b + 32 + lane] = s1 * inv;
}

// part[blk][o] = sum over this CTA's boxes of x[b][o] (kColParts CTAs, 256 threads)
__global__ void lp_colpart_kernel(const float* __restrict__ x, int B, float* __restrict__ part) {
  __shared__ float red[4][kLpH];
  const int o = threadIdx.x & 63, sub = threadIdx.x >> 6;
  const int per = (B + gridDim.x - 1) / gridDim.x;
  const int b0 = blockIdx.x * per, b1 = min(B, b0 + per);
  float acc = 0.f;
  for (int b = b0 + sub; b < b1; b += 4) acc += x[kLpH * b + o];
  red[sub][o] = acc;
  __syncthreads();
  if (sub == 0) part[kLpH * blockIdx.x + o] = red[0][o] + red[1][o] + red[2][o] + red[3][o];
}

struct LayerArg {
  Tabs t;
  const __nv_bfloat16* w;  // the layer's block: Ws, Wn, Wg, c
  const float* h;          // [B][64] input
  const float* gpart;      // [kColParts][64] column partial sums of h
  float* hout;             // [B][64]
  float* m;                // [B][64] neighbourhood means (kept for the backward pass)
  float* P;                // [B][64] pre-activations (kept)
  float* g;                // [64] the global mean (kept; written by CTA 0)
};

// One message-passing layer for kLayerBoxes boxes per CTA (256 threads:
// box r = tid / 8, channels 8 (tid % 8) .. + 8).
__global__ void __launch_bounds__(256) lp_layer_kernel(LayerArg L) {
  extern __shared__ float sm[];
  float* WsT = sm;                       // [k][o]
  float* WnT = WsT + kLpH * kLpH;
  float* cg = WnT + kLpH * kLpH;         // c + Wg g
  float* gs = cg + kLpH;
  float* X = gs + kLpH;                  // [kLayerBoxes][2 * 64 + 1]: h, m
  constexpr int ldx = 2 * kLpH + 1;
  const int tid = threadIdx.x, B = L.t.B;
  for (int i = tid; i < kLpH * kLpH; i += 256) {
    const int o = i / kLpH, k = i % kLpH;
    WsT[k * kLpH + o] = bf(L.w, i);
    WnT[k * kLpH + o] = bf(L.w, kLpH * kLpH + i);
  }
  if (tid < kLpH) {
    float s = 0.f;
    for (int j = 0; j < kColParts; ++j) s += L.gpart[kLpH * j + tid];
    gs[tid] = s / static_cast<float>(B);
    if (blockIdx.x == 0) L.g[tid] = gs[tid];
  }
  __syncthreads();
  if (tid < kLpH) {
    float acc = bf(L.w, 3 * kLpH * kLpH + tid);
    for (int k = 0; k < kLpH; ++k) acc = fmaf(bf(L.w, 2 * kLpH * kLpH + tid * kLpH + k), gs[k], acc);
    cg[tid] = acc;
  }
  const int r = tid >> 3, o0 = (tid & 7) * 8;
  const int b = blockIdx.x * kLayerBoxes + r;
  if (b < B) {
    float hm[8], mm[8];
    for (int j = 0; j < 8; ++j) {
      hm[j] = L.h[kLpH * b + o0 + j];
      mm[j] = 0.f;
    }
    const int q0 = L.t.nb_ptr[b], q1 = L.t.nb_ptr[b + 1];
    for (int q = q0; q < q1; ++q) {
      const float* hr = L.h + kLpH * L.t.nb_idx[q] + o0;
      for (int j = 0; j < 8; ++j) mm[j] += hr[j];
    }
    const float inv = 1.f / static_cast<float>(q1 - q0);
    for (int j = 0; j < 8; ++j) {
      X[r * ldx + o0 + j] = hm[j];
      X[r * ldx + kLpH + o0 + j] = mm[j] * inv;
    }
  }
  __syncthreads();
  if (b >= B) return;
  float acc[8];
  for (int j = 0; j < 8; ++j) acc[j] = cg[o0 + j];
  for (int k = 0; k < kLpH; ++k) {
    const float xh = X[r * ldx + k], xm = X[r * ldx + kLpH + k];
    for (int j = 0; j < 8; ++j) acc[j] = fmaf(WsT[k * kLpH + o0 + j], xh, fmaf(WnT[k * kLpH + o0 + j], xm, acc[j]));
  }
  for (int j = 0; j < 8; ++j) {
    const int o = o0 + j;
    L.P[kLpH * b + o] = acc[j];
    L.m[kLpH * b + o] = X[r * ldx + kLpH + o];
    L.hout[kLpH * b + o] = X[r * ldx + o] + fmaxf(acc[j], 0.f);
  }
}

struct DecArg {
  Tabs t;
  const __nv_bfloat16* w;
  const float* h3;     // [B][64]
  const float* a;      // [N][64]
  const float2* u;     // [N][8]
  const double2* z;
  double2* y;          // may alias z
  float* q;            // [N][64] decoder hidden layer (training; null otherwise)
};

// Decoder and output for kDecRows RWGs per CTA (128 threads: RWG r = tid / 4).
__global__ void __launch_bounds__(128) lp_decode_kernel(DecArg D) {
  extern __shared__ float sm[];
  float* W1T = sm;                     // [128][64]
  float* W2T = W1T + 2 * kLpH * kLpH;  // [64][32]
  float* d1 = W2T + kLpH * kLpG;
  float* d2 = d1 + kLpH;
  float* X = d2 + kLpG;                // [32][129]
  float* Q = X + kDecRows * (2 * kLpH + 1);  // [32][65]
  float* Gs = Q + kDecRows * (kLpH + 1);     // [32][33]
  const int tid = threadIdx.x, N = D.t.N;
  for (int i = tid; i < 2 * kLpH * kLpH; i += 128) {
    const int o = i / (2 * kLpH), k = i % (2 * kLpH);
    W1T[k * kLpH + o] = bf(D.w, kLpOffWd1 + i);
  }
  for (int i = tid; i < kLpG * kLpH; i += 128) {
    const int j = i / kLpH, o = i % kLpH;
    W2T[o * kLpG + j] = bf(D.w, kLpOffWd2 + i);
  }
  if (tid < kLpH) d1[tid] = bf(D.w, kLpOffD1 + tid);
  if (tid < kLpG) d2[tid] = bf(D.w, kLpOffD2 + tid);
  const int p0 = blockIdx.x * kDecRows;
  for (int i = tid; i < kDecRows * kLpH; i += 128) {
    const int r = i / kLpH, k = i % kLpH, p = p0 + r;
    float xh = 0.f, xa = 0.f;
    if (p < N) {
      xh = D.h3[kLpH * D.t.pos_box[p] + k];
      xa = D.a[kLpH * p + k];
    }
    X[r * (2 * kLpH + 1) + k] = xh;
    X[r * (2 * kLpH + 1) + kLpH + k] = xa;
  }
  __syncthreads();
  const int r = tid >> 2, c4 = tid & 3, p = p0 + r;
  {
    float acc[16];
    for (int j = 0; j < 16; ++j) acc[j] = d1[c4 * 16 + j];
    for (int k = 0; k < 2 * kLpH; ++k) {
      const float x = X[r * (2 * kLpH + 1) + k];
      for (int j = 0; j < 16; ++j) acc[j] = fmaf(W1T[k * kLpH + c4 * 16 + j], x, acc[j]);
    }
    for (int j = 0; j < 16; ++j) {
      const float qv = fmaxf(acc[j], 0.f);
      Q[r * (kLpH + 1) + c4 * 16 + j] = qv;
      if (D.q && p < N) D.q[kLpH * p + c4 * 16 + j] = qv;
    }
  }
  __syncthreads();
  {
    float acc[8];
    for (int j = 0; j < 8; ++j) acc[j] = d2[c4 * 8 + j];
    for (int o = 0; o < kLpH; ++o) {
      const float qv = Q[r * (kLpH + 1) + o];
      for (int j = 0; j < 8; ++j) acc[j] = fmaf(W2T[o * kLpG + c4 * 8 + j], qv, acc[j]);
    }
    for (int j = 0; j < 8; ++j) Gs[r * (kLpG + 1) + c4 * 8 + j] = acc[j];
  }
  __syncthreads();
  if (tid < 2 * kDecRows) {
    const int rr = tid >> 1, c = tid & 1, pp = p0 + rr;
    if (pp < N) {
      const int id = D.t.ids[pp];
      float2 dl = make_float2(0.f, 0.f);
      for (int t = 0; t < kLpT; ++t) {
        const float2 g = make_float2(Gs[rr * (kLpG + 1) + c * 16 + 2 * t], Gs[rr * (kLpG + 1) + c * 16 + 2 * t + 1]);
        dl = cfma(g, D.u[kLpT * pp + t], dl);
      }
      const double2 zc = D.z[c * N + id];
      D.y[c * N + id] = make_double2(zc.x + static_cast<double>(dl.x), zc.y + static_cast<double>(dl.y));
    }
  }
}

struct DecBwdArg {
  Tabs t;
  const __nv_bfloat16* w;
  const double2* y;    // with e: the loss sum |y - e|^2 / sum |e|^2
  const double2* e;
  const double* esum;  // sum |e|^2
  const double2* gy;   // or, when not null, a given dL/dRe(y) + j dL/dIm(y)
  const float2* u;
  const float* q;      // [N][64]
  float* dG;           // [N][32]
  float* dq;           // [N][64]
  float* dx;           // [N][128]: d/d[h3_box; a]
  float* loss;
};

__global__ void __launch_bounds__(128) lp_decode_bwd_kernel(DecBwdArg D) {
  extern __shared__ float sm[];
  float* W2 = sm;                      // [32][64] as stored (j, o)
  float* W1 = W2 + kLpG * kLpH;        // [64][128] as stored (o, k)
  float* DG = W1 + 2 * kLpH * kLpH;    // [32][33]
  float* DQ = DG + kDecRows * (kLpG + 1);  // [32][65]
  __shared__ float red[128];
  const int tid = threadIdx.x, N = D.t.N;
  for (int i = tid; i < kLpG * kLpH; i += 128) W2[i] = bf(D.w, kLpOffWd2 + i);
  for (int i = tid; i < 2 * kLpH * kLpH; i += 128) W1[i] = bf(D.w, kLpOffWd1 + i);
  const int p0 = blockIdx.x * kDecRows;
  const float sc = D.gy ? 0.f : static_cast<float>(2.0 / D.esum[0]);
  float lsum = 0.f;
  if (tid < 2 * kDecRows) {
    const int r = tid >> 1, c = tid & 1, p = p0 + r;
    float g[2 * kLpT];
    for (int j = 0; j < 2 * kLpT; ++j) g[j] = 0.f;
    if (p < N) {
      const int id = D.t.ids[p];
      float2 gv;  // dL/dRe(y) + j dL/dIm(y)
      if (D.gy) {
        gv = f2(D.gy[c * N + id]);
      } else {
        const double2 yy = D.y[c * N + id], ee = D.e[c * N + id];
        const float2 res = make_float2(static_cast<float>(yy.x - ee.x), static_cast<float>(yy.y - ee.y));
        lsum = (res.x * res.x + res.y * res.y) * (0.5f * sc);
        gv = cscale(res, sc);
      }
      for (int t = 0; t < kLpT; ++t) {
        const float2 uu = D.u[kLpT * p + t];
        // d/dgr = Re(conj(gv) u), d/dgi = -Im(conj(gv) u)
        g[2 * t] = gv.x * uu.x + gv.y * uu.y;
        g[2 * t + 1] = -(gv.x * uu.y - gv.y * uu.x);
      }
      for (int j = 0; j < 2 * kLpT; ++j) D.dG[kLpG * p + c * 16 + j] = g[j];
    }
    for (int j = 0; j < 2 * kLpT; ++j) DG[r * (kLpG + 1) + c * 16 + j] = g[j];
  }
  red[tid] = lsum;
  __syncthreads();
  for (int wdt = 64; wdt > 0; wdt >>= 1) {
    if (tid < wdt) red[tid] += red[tid + wdt];
    __syncthreads();
  }
  if (tid == 0 && D.loss) atomicAdd(D.loss, red[0]);
  const int r = tid >> 2, c4 = tid & 3, p = p0 + r;
  {
    float acc[16];
    for (int j = 0; j < 16; ++j) acc[j] = 0.f;
    for (int jj = 0; jj < kLpG; ++jj) {
      const float g = DG[r * (kLpG + 1) + jj];
      for (int j = 0; j < 16; ++j) acc[j] = fmaf(W2[jj * kLpH + c4 * 16 + j], g, acc[j]);
    }
    for (int j = 0; j < 16; ++j) {
      const int o = c4 * 16 + j;
      const float v = (p < N && D.q[kLpH * p + o] > 0.f) ? acc[j] : 0.f;
      DQ[r * (kLpH + 1) + o] = v;
      if (p < N) D.dq[kLpH * p + o] = v;
    }
  }
  __syncthreads();
  if (p < N) {
    float acc[32];
    for (int j = 0; j < 32; ++j) acc[j] = 0.f;
    for (int o = 0; o < kLpH; ++o) {
      const float g = DQ[r * (kLpH + 1) + o];
      for (int j = 0; j < 32; ++j) acc[j] = fmaf(W1[o * 2 * kLpH + c4 * 32 + j], g, acc[j]);
    }
    for (int j = 0; j < 32; ++j) D.dx[2 * kLpH * p + c4 * 32 + j] = acc[j];
  }
}

// dh[b] = sum over the box's RWGs of dx[p][0..64)
__global__ void lp_box_dxsum_kernel(Tabs t, const float* __restrict__ dx, float* __restrict__ dh) {
  const int b = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (b >= t.B) return;
  float s0 = 0.f, s1 = 0.f;
  for (int p = t.leaf_ptr[b]; p < t.leaf_ptr[b + 1]; ++p) {
    s0 += dx[2 * kLpH * p + lane];
    s1 += dx[2 * kLpH * p + 32 + lane];
  }
  dh[kLpH * b + lane] = s0;
  dh[kLpH * b + 32 + lane] = s1;
}

// dP = dh * [P > 0], and per-CTA column partial sums of dP
__global__ void lp_dp_kernel(const float* __restrict__ dh, const float* __restrict__ P, int B, float* __restrict__ dP,
                             float* __restrict__ part) {
  __shared__ float red[4][kLpH];
  const int o = threadIdx.x & 63, sub = threadIdx.x >> 6;
  const int per = (B + gridDim.x - 1) / gridDim.x;
  const int b0 = blockIdx.x * per, b1 = min(B, b0 + per);
  float acc = 0.f;
  for (int b = b0 + sub; b < b1; b += 4) {
    const float v = P[kLpH * b + o] > 0.f ? dh[kLpH * b + o] : 0.f;
    dP[kLpH * b + o] = v;
    acc += v;
  }
  red[sub][o] = acc;
  __syncthreads();
  if (sub == 0) part[kLpH * blockIdx.x + o] = red[0][o] + red[1][o] + red[2][o] + red[3][o];
}

struct LayerBwdArg {
  Tabs t;
  const __nv_bfloat16* w;  // the layer's block
  const float* dh;         // [B][64] gradient at the layer's output
  const float* dP;         // [B][64]
  const float* spart;      // [kColParts][64] partial column sums of dP
  float* tmp;              // [B][64]: dh + Ws^T dP + Wg^T S / B
  float* dm;               // [B][64]: Wn^T dP / |nbr(b)|
  float* S;                // [64] column sums of dP (written by CTA 0)
};

__global__ void __launch_bounds__(256) lp_layer_bwd_kernel(LayerBwdArg L) {
  extern __shared__ float sm[];
  float* Ws = sm;                  // [o][k] as stored
  float* Wn = Ws + kLpH * kLpH;
  float* dg = Wn + kLpH * kLpH;
  float* Ss = dg + kLpH;
  float* D = Ss + kLpH;            // [kLayerBoxes][65]
  const int tid = threadIdx.x, B = L.t.B;
  for (int i = tid; i < kLpH * kLpH; i += 256) {
    Ws[i] = bf(L.w, i);
    Wn[i] = bf(L.w, kLpH * kLpH + i);
  }
  if (tid < kLpH) {
    float s = 0.f;
    for (int j = 0; j < kColParts; ++j) s += L.spart[kLpH * j + tid];
    Ss[tid] = s;
    if (blockIdx.x == 0) L.S[tid] = s;
  }
  const int r = tid >> 3, k0 = (tid & 7) * 8;
  const int b = blockIdx.x * kLayerBoxes + r;
  for (int j = 0; j < 8; ++j) D[r * (kLpH + 1) + k0 + j] = b < B ? L.dP[kLpH * b + k0 + j] : 0.f;
  __syncthreads();
  if (tid < kLpH) {
    float acc = 0.f;
    for (int o = 0; o < kLpH; ++o) acc = fmaf(bf(L.w, 2 * kLpH * kLpH + o * kLpH + tid), Ss[o], acc);
    dg[tid] = acc / static_cast<float>(B);
  }
  __syncthreads();
  if (b >= B) return;
  float ts[8], tn[8];
  for (int j = 0; j < 8; ++j) ts[j] = tn[j] = 0.f;
  for (int o = 0; o < kLpH; ++o) {
    const float g = D[r * (kLpH + 1) + o];
    for (int j = 0; j < 8; ++j) {
      ts[j] = fmaf(Ws[o * kLpH + k0 + j], g, ts[j]);
      tn[j] = fmaf(Wn[o * kLpH + k0 + j], g, tn[j]);
    }
  }
  const float inv = 1.f / static_cast<float>(L.t.nb_ptr[b + 1] - L.t.nb_ptr[b]);
  for (int j = 0; j < 8; ++j) {
    const int k = k0 + j;
    L.tmp[kLpH * b + k] = L.dh[kLpH * b + k] + ts[j] + dg[k];
    L.dm[kLpH * b + k] = tn[j] * inv;
  }
}

// dh_in[b] = tmp[b] + sum over the box's neighbourhood of dm (the
// neighbourhoods are symmetric: b' in nbr(b) iff b in nbr(b'))
__global__ void lp_nbr_sum_kernel(Tabs t, const float* __restrict__ tmp, const float* __restrict__ dm,
                                  float* __restrict__ dh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.B * kLpH) return;
  const int b = i / kLpH, k = i % kLpH;
  float acc = tmp[i];
  for (int q = t.nb_ptr[b]; q < t.nb_ptr[b + 1]; ++q) acc += dm[kLpH * t.nb_idx[q] + k];
  dh[i] = acc;
}

// dWg[o][k] += S[o] g[k]
__global__ void lp_outer_kernel(const float* __restrict__ S, const float* __restrict__ g, float* __restrict__ dW) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kLpH * kLpH) dW[i] += S[i / kLpH] * g[i % kLpH];
}

// The encoder's input gradient: da = (dx[p][64..128) + dh0[box] / n_box) * [a > 0], in place
__global__ void lp_unpool_kernel(Tabs t, const float* __restrict__ dh0, const float* __restrict__ a,
                                 float* __restrict__ dx) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i >= static_cast<long long>(t.N) * kLpH) return;
  const int p = static_cast<int>(i / kLpH), o = static_cast<int>(i % kLpH), b = t.pos_box[p];
  const float nb = static_cast<float>(t.leaf_ptr[b + 1] - t.leaf_ptr[b]);
  float* d = dx + 2 * kLpH * static_cast<long long>(p) + kLpH + o;
  *d = a[i] > 0.f ? *d + dh0[kLpH * b + o] / nb : 0.f;
}

struct WgArg {
  const float* A;    // A[row * lda + o], o < O (<= 64)
  int lda, O;
  const float* X;    // X[(xmap ? xmap[row] : row) * ldx + k], k < K (16 or 64)
  int ldx, K;
  const int* xmap;
  int rows;
  float* dW;         // dW[o * ldw + k] +=
  int ldw;
  float* db;         // db[o] += sum_rows A (optional)
};

// dW += A^T X over the rows: kWgRows rows per CTA, 256 threads, thread
// (o = tid / 4, k = tid % 4 + 4 j).
__global__ void __launch_bounds__(256) lp_wgrad_kernel(WgArg g) {
  __shared__ float As[32][kLpH + 1];
  __shared__ float Xs[32][kLpH + 1];
  const int tid = threadIdx.x, o = tid >> 2, kq = tid & 3;
  const int r0 = blockIdx.x * kWgRows, r1 = min(g.rows, r0 + kWgRows);
  const int nk = g.K / 4;
  float acc[16], accb = 0.f;
  for (int j = 0; j < 16; ++j) acc[j] = 0.f;
  for (int rb = r0; rb < r1; rb += 32) {
    for (int i = tid; i < 32 * kLpH; i += 256) {
      const int rr = i / kLpH, c = i % kLpH, row = rb + rr;
      const bool in = row < r1;
      As[rr][c] = (in && c < g.O) ? g.A[static_cast<long long>(row) * g.lda + c] : 0.f;
      Xs[rr][c] = (in && c < g.K) ? g.X[static_cast<long long>(g.xmap ? g.xmap[row] : row) * g.ldx + c] : 0.f;
    }
    __syncthreads();
    for (int rr = 0; rr < 32; ++rr) {
      const float a = As[rr][o];
      accb += a;
      for (int j = 0; j < nk; ++j) acc[j] = fmaf(a, Xs[rr][kq + 4 * j], acc[j]);
    }
    __syncthreads();
  }
  if (o < g.O) {
    for (int j = 0; j < nk; ++j) atomicAdd(g.dW + o * g.ldw + kq + 4 * j, acc[j]);
    if (g.db && kq == 0) atomicAdd(g.db + o, accb);
  }
}

__global__ void lp_bf16_kernel(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

__global__ void lp_adam_kernel(int n, float* __restrict__ th, const float* __restrict__ gr, float* __restrict__ m,
                               float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                               float gs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = gr[i] * gs;
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  th[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

struct LearnedWork {
  int N = 0, B = 0;
  Tabs t{};
  double* part = nullptr;   // [kRedBlocks] partial sums of |e|^2
  double* esum = nullptr;   // sum |e|^2
  float2 *zb = nullptr, *zn = nullptr, *z2 = nullptr, *u = nullptr;
  float *a = nullptr, *q = nullptr, *dG = nullptr, *dq = nullptr, *dx = nullptr;
  float* h[kLpLayers + 1] = {};
  float* m[kLpLayers] = {};
  float* P[kLpLayers] = {};
  float* g[kLpLayers] = {};
  float *cpart = nullptr, *dh = nullptr, *dh2 = nullptr, *dP = nullptr, *dm = nullptr, *tmp = nullptr, *S = nullptr;
  __nv_bfloat16* w_attached = nullptr;  // null until a network is attached
  __nv_bfloat16* w_scratch = nullptr;
  __nv_bfloat16* w_store = nullptr;     // storage behind w_attached
};

static size_t layer_smem() { return (2 * kLpH * kLpH + 2 * kLpH + kLayerBoxes * (2 * kLpH + 1)) * sizeof(float); }
static size_t dec_smem() {
  return (2 * kLpH * kLpH + kLpH * kLpG + kLpH + kLpG + kDecRows * (2 * kLpH + 1) + kDecRows * (kLpH + 1) +
          kDecRows * (kLpG + 1)) *
         sizeof(float);
}
static size_t dec_bwd_smem() {
  return (kLpG * kLpH + 2 * kLpH * kLpH + kDecRows * (kLpG + 1) + kDecRows * (kLpH + 1)) * sizeof(float);
}
static size_t layer_bwd_smem() { return (2 * kLpH * kLpH + 2 * kLpH + kLayerBoxes * (kLpH + 1)) * sizeof(float); }

LearnedWork& lp_work(Plan& P) {
  if (P.lp) return *P.lp;
  MLFMA_CUDA(cudaSetDevice(P.device));
  auto w = std::make_shared<LearnedWork>();
  const Tree& T = P.tree;
  const int N = P.N, B = static_cast<int>(T.leaf_ptr.size()) - 1;
  w->N = N;
  w->B = B;
  // neighbourhoods: the box and its near-field neighbours at the leaf level
  const Level& L = T.lv[T.maxLevel];
  if (L.size() != B) throw std::runtime_error("leaf level and leaf lists disagree");
  std::vector<int> nb_ptr(B + 1, 0), nb_idx;
  for (int b = 0; b < B; ++b) {
    std::vector<int> s(L.near_idx.begin() + L.near_ptr[b], L.near_idx.begin() + L.near_ptr[b + 1]);
    s.push_back(b);
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
    nb_idx.insert(nb_idx.end(), s.begin(), s.end());
    nb_ptr[b + 1] = static_cast<int>(nb_idx.size());
  }
  for (int b = 0; b < B; ++b)  // the backward pass relies on symmetric neighbourhoods
    for (int q = nb_ptr[b]; q < nb_ptr[b + 1]; ++q) {
      const int c = nb_idx[q];
      if (!std::binary_search(nb_idx.begin() + nb_ptr[c], nb_idx.begin() + nb_ptr[c + 1], b))
        throw std::runtime_error("leaf neighbourhoods are not symmetric");
    }
  std::vector<int> pos_box(N);
  for (int b = 0; b < B; ++b)
    for (int p = T.leaf_ptr[b]; p < T.leaf_ptr[b + 1]; ++p) pos_box[p] = b;
  // RWG dipoles l (c+ - c-), normalised to mean length 1, by leaf position
  auto centroid = [&](int f, int k) {
    double s = 0.0;
    for (int j = 0; j < 3; ++j) s += P.mesh.xyz[3 * P.mesh.face_v[3 * f + j] + k];
    return s / 3.0;
  };
  std::vector<double> dd(3 * static_cast<size_t>(N));
  double mean = 0.0;
  for (int i = 0; i < N; ++i) {
    double nn = 0.0;
    for (int k = 0; k < 3; ++k) {
      dd[3 * i + k] = P.rwg.len[i] * (centroid(P.rwg.fpos[i], k) - centroid(P.rwg.fneg[i], k));
      nn += dd[3 * i + k] * dd[3 * i + k];
    }
    mean += std::sqrt(nn);
  }
  mean /= N;
  std::vector<float> dip(3 * static_cast<size_t>(N));
  for (int p = 0; p < N; ++p)
    for (int k = 0; k < 3; ++k) dip[3 * p + k] = static_cast<float>(dd[3 * T.leaf_rwg[p] + k] / mean);
  // static features per leaf position: edge length, the two triangle
  // areas, the cosine between their normals, the dipole length, box fill,
  // neighbourhood size, dipole coherence of the box, and the material
  std::vector<double> area(P.mesh.face_v.size() / 3), nrm(P.mesh.face_v.size());
  double area_mean = 0.0, len_mean = 0.0;
  for (size_t f = 0; f < area.size(); ++f) {
    const double* p0 = &P.mesh.xyz[3 * P.mesh.face_v[3 * f]];
    const double* p1 = &P.mesh.xyz[3 * P.mesh.face_v[3 * f + 1]];
    const double* p2 = &P.mesh.xyz[3 * P.mesh.face_v[3 * f + 2]];
    const double a[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    const double b[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    const double cn = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    area[f] = 0.5 * cn;
    for (int k = 0; k < 3; ++k) nrm[3 * f + k] = c[k] / cn;
    area_mean += area[f];
  }
  area_mean /= static_cast<double>(area.size());
  for (int i = 0; i < N; ++i) len_mean += P.rwg.len[i];
  len_mean /= N;
  std::vector<double> coh(B);
  for (int b = 0; b < B; ++b) {
    double s3[3] = {0, 0, 0};
    for (int p = T.leaf_ptr[b]; p < T.leaf_ptr[b + 1]; ++p)
      for (int k = 0; k < 3; ++k) s3[k] += dd[3 * T.leaf_rwg[p] + k] / mean;
    coh[b] = std::sqrt(s3[0] * s3[0] + s3[1] * s3[1] + s3[2] * s3[2]) / (T.leaf_ptr[b + 1] - T.leaf_ptr[b]);
  }
  const double er = P.epsr.real();
  std::vector<float> fs(static_cast<size_t>(kLpF) * N, 0.f);
  for (int p = 0; p < N; ++p) {
    const int i = T.leaf_rwg[p], b = pos_box[p], fp = P.rwg.fpos[i], fn = P.rwg.fneg[i];
    const double nb = T.leaf_ptr[b + 1] - T.leaf_ptr[b];
    double dl = 0.0;
    for (int k = 0; k < 3; ++k) dl += (dd[3 * i + k] / mean) * (dd[3 * i + k] / mean);
    float* f = &fs[static_cast<size_t>(kLpF) * p];
    f[0] = static_cast<float>(P.rwg.len[i] / len_mean);
    f[1] = static_cast<float>(area[fp] / area_mean);
    f[2] = static_cast<float>(area[fn] / area_mean);
    f[3] = static_cast<float>(nrm[3 * fp] * nrm[3 * fn] + nrm[3 * fp + 1] * nrm[3 * fn + 1] +
                              nrm[3 * fp + 2] * nrm[3 * fn + 2]);
    f[4] = static_cast<float>(std::sqrt(dl));
    f[5] = static_cast<float>(nb / 16.0);
    f[6] = static_cast<float>((nb_ptr[b + 1] - nb_ptr[b]) / 27.0);
    f[7] = static_cast<float>(coh[b]);
    f[8] = static_cast<float>(std::log(er));
    f[9] = static_cast<float>(std::abs(P.epsr.imag()) / er);
    f[10] = static_cast<float>(std::sqrt(er) / 2.0);
  }
  w->t.N = N;
  w->t.B = B;
  w->t.ids = P.d_leaf_rwg;
  w->t.leaf_ptr = P.d_leaf_ptr;
  w->t.pos_box = P.upload(pos_box);
  w->t.dip = P.upload(dip);
  w->t.nb_ptr = P.upload(nb_ptr);
  w->t.nb_idx = P.upload(nb_idx);
  w->t.fs = P.upload(fs);
  w->part = P.alloc<double>(kRedBlocks);
  w->esum = P.alloc<double>(1);
  w->zb = P.alloc<float2>(6 * static_cast<size_t>(B));
  w->zn = P.alloc<float2>(6 * static_cast<size_t>(B));
  w->z2 = P.alloc<float2>(6 * static_cast<size_t>(B));
  w->u = P.alloc<float2>(static_cast<size_t>(kLpT) * N);
  w->a = P.alloc<float>(static_cast<size_t>(kLpH) * N);
  w->q = P.alloc<float>(static_cast<size_t>(kLpH) * N);
  w->dG = P.alloc<float>(static_cast<size_t>(kLpG) * N);
  w->dq = P.alloc<float>(static_cast<size_t>(kLpH) * N);
  w->dx = P.alloc<float>(static_cast<size_t>(2 * kLpH) * N);
  for (auto& x : w->h) x = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  for (auto& x : w->m) x = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  for (auto& x : w->P) x = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  for (auto& x : w->g) x = P.alloc<float>(kLpH);
  w->cpart = P.alloc<float>(static_cast<size_t>(kColParts) * kLpH);
  w->dh = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  w->dh2 = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  w->dP = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  w->dm = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  w->tmp = P.alloc<float>(static_cast<size_t>(kLpH) * B);
  w->S = P.alloc<float>(kLpH);
  w->w_scratch = P.alloc<__nv_bfloat16>(kLpParams);
  w->w_store = P.alloc<__nv_bfloat16>(kLpParams);
  // the tables above are uploaded on the plan's stream; the learned kernels
  // may run on a caller's stream
  MLFMA_CUDA(cudaStreamSynchronize(P.stream));
  MLFMA_CUDA(cudaFuncSetAttribute(lp_layer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(layer_smem())));
  MLFMA_CUDA(cudaFuncSetAttribute(lp_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dec_smem())));
  MLFMA_CUDA(cudaFuncSetAttribute(lp_decode_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dec_bwd_smem())));
  MLFMA_CUDA(cudaFuncSetAttribute(lp_layer_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(layer_bwd_smem())));
  P.lp = w;
  return *w;
}

static const __nv_bfloat16* layer_w(const __nv_bfloat16* w, int l) { return w + kLpOffLayer0 + l * kLpLayerSize; }

void lp_forward(Plan& P, const __nv_bfloat16* w, const double2* /* v: enters through z */, const double2* z,
                double2* y, bool train, cudaStream_t s) {
  LearnedWork& W = lp_work(P);
  const int N = W.N, B = W.B;
  lp_boxz_kernel<<<(B + 127) / 128, 128, 0, s>>>(W.t, z, W.zb);
  lp_boxn_kernel<<<(B + 127) / 128, 128, 0, s>>>(W.t, W.zb, W.zn);
  lp_boxn_kernel<<<(B + 127) / 128, 128, 0, s>>>(W.t, W.zn, W.z2);
  EncArg e{W.t, z, W.zb, W.zn, W.z2, w, W.u, W.a};
  lp_encode_kernel<<<(N + 127) / 128, 128, 0, s>>>(e);
  lp_pool_kernel<<<(B + 7) / 8, 256, 0, s>>>(W.t, W.a, W.h[0]);
  for (int l = 0; l < kLpLayers; ++l) {
    lp_colpart_kernel<<<kColParts, 256, 0, s>>>(W.h[l], B, W.cpart);
    LayerArg la{W.t, layer_w(w, l), W.h[l], W.cpart, W.h[l + 1], W.m[l], W.P[l], W.g[l]};
    lp_layer_kernel<<<(B + kLayerBoxes - 1) / kLayerBoxes, 256, layer_smem(), s>>>(la);
  }
  DecArg d{W.t, w, W.h[kLpLayers], W.a, W.u, z, y, train ? W.q : nullptr};
  lp_decode_kernel<<<(N + kDecRows - 1) / kDecRows, 128, dec_smem(), s>>>(d);
  MLFMA_CUDA(cudaGetLastError());
}

static void wgrad(const float* A, int lda, int O, const float* X, int ldx, int K, const int* xmap, int rows, float* dW,
                  int ldw, float* db, cudaStream_t s) {
  WgArg g{A, lda, O, X, ldx, K, xmap, rows, dW, ldw, db};
  lp_wgrad_kernel<<<(rows + kWgRows - 1) / kWgRows, 256, 0, s>>>(g);
}

void lp_backward(Plan& P, const __nv_bfloat16* w, const double2* y, const double2* e, const double2* gy, float* grad,
                 float* loss, cudaStream_t s) {
  LearnedWork& W = lp_work(P);
  const int N = W.N, B = W.B;
  if (!gy) {
    lp_sumsq_kernel<<<kRedBlocks, 256, 0, s>>>(e, 2LL * N, W.part);
    lp_finalize_kernel<<<1, 256, 0, s>>>(W.part, kRedBlocks, 1, W.esum);
  }
  DecBwdArg d{W.t, w, y, e, W.esum, gy, W.u, W.q, W.dG, W.dq, W.dx, gy ? nullptr : loss};
  lp_decode_bwd_kernel<<<(N + kDecRows - 1) / kDecRows, 128, dec_bwd_smem(), s>>>(d);
  wgrad(W.dG, kLpG, kLpG, W.q, kLpH, kLpH, nullptr, N, grad + kLpOffWd2, kLpH, grad + kLpOffD2, s);
  wgrad(W.dq, kLpH, kLpH, W.h[kLpLayers], kLpH, kLpH, W.t.pos_box, N, grad + kLpOffWd1, 2 * kLpH, grad + kLpOffD1, s);
  wgrad(W.dq, kLpH, kLpH, W.a, kLpH, kLpH, nullptr, N, grad + kLpOffWd1 + kLpH, 2 * kLpH, nullptr, s);
  lp_box_dxsum_kernel<<<(B + 7) / 8, 256, 0, s>>>(W.t, W.dx, W.dh);
  float* dh = W.dh;
  float* dh_next = W.dh2;
  for (int l = kLpLayers - 1; l >= 0; --l) {
    float* gl = grad + kLpOffLayer0 + l * kLpLayerSize;
    lp_dp_kernel<<<kColParts, 256, 0, s>>>(dh, W.P[l], B, W.dP, W.cpart);
    LayerBwdArg lb{W.t, layer_w(w, l), dh, W.dP, W.cpart, W.tmp, W.dm, W.S};
    lp_layer_bwd_kernel<<<(B + kLayerBoxes - 1) / kLayerBoxes, 256, layer_bwd_smem(), s>>>(lb);
    wgrad(W.dP, kLpH, kLpH, W.h[l], kLpH, kLpH, nullptr, B, gl, kLpH, gl + 3 * kLpH * kLpH, s);
    wgrad(W.dP, kLpH, kLpH, W.m[l], kLpH, kLpH, nullptr, B, gl + kLpH * kLpH, kLpH, nullptr, s);
    lp_outer_kernel<<<(kLpH * kLpH + 255) / 256, 256, 0, s>>>(W.S, W.g[l], gl + 2 * kLpH * kLpH);
    lp_nbr_sum_kernel<<<(B * kLpH + 255) / 256, 256, 0, s>>>(W.t, W.tmp, W.dm, dh_next);
    std::swap(dh, dh_next);
  }
  lp_unpool_kernel<<<static_cast<int>((static_cast<long long>(N) * kLpH + 255) / 256), 256, 0, s>>>(W.t, dh, W.a,
                                                                                                     W.dx);
  wgrad(W.dx + kLpH, 2 * kLpH, kLpH, W.t.fs, kLpF, kLpF, nullptr, N, grad, kLpF, grad + kLpOffBe, s);
  MLFMA_CUDA(cudaGetLastError());
}

void lp_to_bf16(const float* in, __nv_bfloat16* out, int n, cudaStream_t s) {
  lp_bf16_kernel<<<(n + 255) / 256, 256, 0, s>>>(in, out, n);
  MLFMA_CUDA(cudaGetLastError());
}

void lp_adam(int n, float* theta, const float* grad, float* m, float* v, float lr, float b1, float b2, float eps,
             int step, float grad_scale, cudaStream_t s) {
  const float c1 = 1.f - std::pow(b1, static_cast<float>(step));
  const float c2 = 1.f - std::pow(b2, static_cast<float>(step));
  lp_adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, theta, grad, m, v, lr, b1, b2, eps, c1, c2, grad_scale);
  MLFMA_CUDA(cudaGetLastError());
}

void lp_attach(Plan& P, const float* params, int n) {
  if (n == 0) {
    if (P.lp) P.lp->w_attached = nullptr;
    return;
  }
  if (n != kLpParams) throw std::invalid_argument("learned preconditioner: wrong parameter count");
  LearnedWork& W = lp_work(P);
  std::vector<__nv_bfloat16> h(kLpParams);
  for (int i = 0; i < kLpParams; ++i) h[i] = __float2bfloat16_rn(params[i]);
  // complete before the weights are used, on any stream
  MLFMA_CUDA(cudaMemcpyAsync(W.w_store, h.data(), kLpParams * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice,
                             P.stream));
  MLFMA_CUDA(cudaStreamSynchronize(P.stream));
  W.w_attached = W.w_store;
}

const __nv_bfloat16* lp_attached(const Plan& P) { return P.lp ? P.lp->w_attached : nullptr; }

__nv_bfloat16* lp_scratch_weights(Plan& P) { return lp_work(P).w_scratch; }

}  // namespace mlfma
