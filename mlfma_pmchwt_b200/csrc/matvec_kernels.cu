// The PMCHWT MLFMA matvec on the GPU, FP64 (the `ax` closure of
// Code/MLFMM.cpp:189-368). J and M currents share the tree and the tables,
// so every stage processes both (6 complex components per direction) in one
// pass over the tables; media k1 and k2 run as separate launches.
//
//   agg      leaf aggregation           Code/ProcessMLFMM.h:33-56   (mexp)
//   up       interpolation + shift up   Code/ProcessMLFMM.h:61-107  (m2m)
//   down     translation over the interaction list plus the parent's
//            anterpolated, shifted incoming pattern
//                                       Code/ProcessMLFMM.h:112-147 (m2l)
//                                       Code/ProcessMLFMM.h:152-202 (l2l)
//   leaf_out receive-pattern testing of both media and the near-field rows,
//            written once per unknown   Code/MLFMM.cpp:285-366
// No stage accumulates into memory written by another launch of the same
// matvec, so no clearing pass (Code/ProcessMLFMM.h:14-28) is needed.
#include "cplx.cuh"
#include "plan.hpp"

namespace mlfma {

namespace {

constexpr int kThreads = 128;

__global__ void __launch_bounds__(kThreads) agg_kernel(const double2* __restrict__ Vs,
                                                       const int* __restrict__ leaf_ptr,
                                                       const int* __restrict__ leaf_rwg,
                                                       const double2* __restrict__ x, int N, int K,
                                                       double2* __restrict__ S) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  if (kk >= K) return;
  double2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = c2(0.0, 0.0);
  const int r1 = leaf_ptr[b + 1];
  for (int r = leaf_ptr[b]; r < r1; ++r) {
    const int id = leaf_rwg[r];
    const double2 xJ = x[id], xM = x[N + id];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double2 v = Vs[(static_cast<size_t>(r) * 3 + c) * K + kk];
      acc[c] = cfma(v, xJ, acc[c]);
      acc[3 + c] = cfma(v, xM, acc[3 + c]);
    }
  }
  double2* out = S + static_cast<size_t>(b) * 6 * K + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * K] = acc[c];
}

struct UpArg {
  const double2* Sc;   // child level patterns [Bc][6][Kc]
  double2* Sp;         // parent level patterns [Bp][6][Kp]
  const int* child_begin;
  const int* octant;   // of child boxes
  const int* tidx;
  const double* lt;
  const int* pidx;
  const double* lp;
  const double2* ph_up;
  int Kp, nphp, Kc, nphc;
};

__global__ void __launch_bounds__(kThreads) up_kernel(UpArg a) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  if (kk >= a.Kp) return;
  const int t = kk / a.nphp, p = kk - t * a.nphp;
  int ti[3], pi[3];
  double wt[3], wp[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    ti[i] = a.tidx[3 * t + i] * a.nphc;
    wt[i] = a.lt[3 * t + i];
    pi[i] = a.pidx[3 * p + i];
    wp[i] = a.lp[3 * p + i];
  }
  double2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = c2(0.0, 0.0);
  const int c1 = a.child_begin[b + 1];
  for (int ch = a.child_begin[b]; ch < c1; ++ch) {
    const double2 e = a.ph_up[a.octant[ch] * a.Kp + kk];
    const double2* src = a.Sc + static_cast<size_t>(ch) * 6 * a.Kc;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const double2* sc = src + static_cast<size_t>(c) * a.Kc;
      double2 v = c2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) v = cfmas(wt[i] * wp[j], sc[ti[i] + pi[j]], v);
      acc[c] = cfma(e, v, acc[c]);
    }
  }
  double2* out = a.Sp + static_cast<size_t>(b) * 6 * a.Kp + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * a.Kp] = acc[c];
}

struct DownArg {
  const double2* S;     // this level's aggregated patterns
  double2* Bm;          // this level's incoming patterns (written)
  const int* far_ptr;
  const int* far_idx;
  const int* far_off;
  const int* off2vec;
  const double2* tfw;
  int K;
  // parent contribution (null Bp at the top level)
  const double2* Bp;
  const int* parent;
  const int* octant;
  const double2* ph_dn;  // parent level table [8][Kp]
  const int* tr_ptr;
  const int* tr_kp;
  const double* tr_w;
  int Kp;
};

__global__ void __launch_bounds__(kThreads) down_kernel(DownArg a) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  if (kk >= a.K) return;
  double2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = c2(0.0, 0.0);
  const int e1 = a.far_ptr[b + 1];
  for (int e = a.far_ptr[b]; e < e1; ++e) {
    const int s = a.far_idx[e];
    const double2 tf = a.tfw[static_cast<size_t>(a.off2vec[a.far_off[e]]) * a.K + kk];
    const double2* src = a.S + static_cast<size_t>(s) * 6 * a.K + kk;
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = cfma(tf, src[static_cast<size_t>(c) * a.K], acc[c]);
  }
  if (a.Bp) {
    const int P = a.parent[b];
    const double2* ph = a.ph_dn + a.octant[b] * a.Kp;
    const double2* bp = a.Bp + static_cast<size_t>(P) * 6 * a.Kp;
    const int t1 = a.tr_ptr[kk + 1];
    for (int e = a.tr_ptr[kk]; e < t1; ++e) {
      const int kp = a.tr_kp[e];
      const double2 f = cscale(ph[kp], a.tr_w[e]);
#pragma unroll
      for (int c = 0; c < 6; ++c) acc[c] = cfma(f, bp[static_cast<size_t>(c) * a.Kp + kp], acc[c]);
    }
  }
  double2* out = a.Bm + static_cast<size_t>(b) * 6 * a.K + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * a.K] = acc[c];
}

struct LeafArg {
  const double2* Vf[2];
  const double2* Bm[2];
  const double* khat[2];
  int K[2];
  const int* leaf_rwg;
  const int* rwg_box;     // leaf box of each RWG id
  const int* leaf_ptr;
  const int* near_sptr;
  const int* near_src;
  const long long* near_zoff;
  const double2* near_z;
  const double2* x;
  double2* w;
  int N;
  double2 c1, c2, etai;
};

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// One warp per RWG (leaf order).
__global__ void __launch_bounds__(kThreads) leaf_out_kernel(LeafArg a) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= a.N) return;
  const int id = a.leaf_rwg[r];
  const int b = a.rwg_box[id];
  double2 res[8];  // L1J K1J L1M K1M L2J K2J L2M K2M
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int K = a.K[m];
    const double2* V = a.Vf[m] + static_cast<size_t>(r) * 3 * K;
    const double2* B = a.Bm[m] + static_cast<size_t>(b) * 6 * K;
    const double* kh = a.khat[m];
    double2 LJ = c2(0, 0), KJ = c2(0, 0), LM = c2(0, 0), KM = c2(0, 0);
    for (int kk = lane; kk < K; kk += 32) {
      const double2 v0 = V[kk], v1 = V[K + kk], v2 = V[2 * K + kk];
      const double2 j0 = B[kk], j1 = B[K + kk], j2 = B[2 * K + kk];
      const double2 m0 = B[3 * K + kk], m1 = B[4 * K + kk], m2 = B[5 * K + kk];
      // (-khat) x V
      const double ax = -kh[kk], ay = -kh[K + kk], az = -kh[2 * K + kk];
      const double2 w0 = csub(cscale(v2, ay), cscale(v1, az));
      const double2 w1 = csub(cscale(v0, az), cscale(v2, ax));
      const double2 w2 = csub(cscale(v1, ax), cscale(v0, ay));
      LJ = cfma(v0, j0, cfma(v1, j1, cfma(v2, j2, LJ)));
      LM = cfma(v0, m0, cfma(v1, m1, cfma(v2, m2, LM)));
      KJ = cfma(w0, j0, cfma(w1, j1, cfma(w2, j2, KJ)));
      KM = cfma(w0, m0, cfma(w1, m1, cfma(w2, m2, KM)));
    }
    res[4 * m + 0] = warp_sum(LJ);
    res[4 * m + 1] = warp_sum(KJ);
    res[4 * m + 2] = warp_sum(LM);
    res[4 * m + 3] = warp_sum(KM);
  }
  // near-field rows t and N + t
  const int s0 = a.near_sptr[b], ns = a.near_sptr[b + 1] - s0;
  const int tl = r - a.leaf_ptr[b];
  const double2* Z = a.near_z + 3 * (a.near_zoff[b] + static_cast<long long>(tl) * ns);
  double2 nJ = c2(0, 0), nM = c2(0, 0);
  for (int j = lane; j < ns; j += 32) {
    const int s = a.near_src[s0 + j];
    const double2 xJ = a.x[s], xM = a.x[a.N + s];
    const double2 z11 = Z[3 * j], z12 = Z[3 * j + 1], z22 = Z[3 * j + 2];
    nJ = cfma(z11, xJ, cfma(z12, xM, nJ));
    nM = cfma(z22, xM, csub(nM, cmul(z12, xJ)));
  }
  nJ = warp_sum(nJ);
  nM = warp_sum(nM);
  if (lane == 0) {
    // w[t]   = c1 (L1J - K1M) + c2 (etai L2J - K2M) + near
    // w[N+t] = c1 (K1J + L1M) + c2 (K2J + L2M / etai) + near
    const double2 L2M_eta = cdiv(res[6], a.etai);
    double2 wj = cmul(a.c1, csub(res[0], res[3]));
    wj = cadd(wj, cmul(a.c2, csub(cmul(a.etai, res[4]), res[7])));
    double2 wm = cmul(a.c1, cadd(res[1], res[2]));
    wm = cadd(wm, cmul(a.c2, cadd(res[5], L2M_eta)));
    a.w[id] = cadd(wj, nJ);
    a.w[a.N + id] = cadd(wm, nM);
  }
}

}  // namespace

void apply_device(Plan& P, const double2* x, double2* w, cudaStream_t s) {
  const int L = P.maxL;
  cudaEvent_t* ev = nullptr;
  if (P.prof.on) {
    if (P.prof.used == P.prof.sets.size()) {
      if (P.prof.sets.size() >= 4096) throw std::runtime_error("stage profiler: read it at least every 4096 applies");
      std::array<cudaEvent_t, StageProfiler::kEvents> set{};
      for (auto& e : set) MLFMA_CUDA(cudaEventCreate(&e));
      P.prof.sets.push_back(set);
    }
    ev = P.prof.sets[P.prof.used++].data();
    MLFMA_CUDA(cudaEventRecord(ev[0], s));
  }
  for (int m = 0; m < 2; ++m) {
    const MediumLevel& leaf = P.ml[m][L];
    dim3 g(P.lv[L].B, (leaf.K + kThreads - 1) / kThreads);
    agg_kernel<<<g, kThreads, 0, s>>>(P.d_Vs[m], P.d_leaf_ptr, P.d_leaf_rwg, x, P.N, leaf.K, leaf.S);
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[1 + 3 * m], s));
    for (int l = L - 1; l >= 2; --l) {
      const MediumLevel& pm = P.ml[m][l];
      const MediumLevel& cm = P.ml[m][l + 1];
      UpArg a{cm.S, pm.S, P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx, pm.lp,
              pm.ph_up, pm.K, pm.nph, cm.K, cm.nph};
      dim3 gu(P.lv[l].B, (pm.K + kThreads - 1) / kThreads);
      up_kernel<<<gu, kThreads, 0, s>>>(a);
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[2 + 3 * m], s));
    for (int l = 2; l <= L; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      DownArg a{};
      a.S = cm.S;
      a.Bm = cm.Bm;
      a.far_ptr = P.lv[l].far_ptr;
      a.far_idx = P.lv[l].far_idx;
      a.far_off = P.lv[l].far_off;
      a.off2vec = cm.off2vec;
      a.tfw = cm.tfw;
      a.K = cm.K;
      if (l > 2) {
        const MediumLevel& pm = P.ml[m][l - 1];
        a.Bp = pm.Bm;
        a.parent = P.lv[l].parent;
        a.octant = P.lv[l].octant;
        a.ph_dn = pm.ph_dn;
        a.tr_ptr = cm.tr_ptr;
        a.tr_kp = cm.tr_kp;
        a.tr_w = cm.tr_w;
        a.Kp = pm.K;
      }
      dim3 gd(P.lv[l].B, (cm.K + kThreads - 1) / kThreads);
      down_kernel<<<gd, kThreads, 0, s>>>(a);
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[3 + 3 * m], s));
  }
  LeafArg a{};
  for (int m = 0; m < 2; ++m) {
    a.Vf[m] = P.d_Vf[m];
    a.Bm[m] = P.ml[m][L].Bm;
    a.khat[m] = P.ml[m][L].khat;
    a.K[m] = P.ml[m][L].K;
  }
  a.leaf_rwg = P.d_leaf_rwg;
  a.rwg_box = P.d_rwg_leafbox;
  a.leaf_ptr = P.d_leaf_ptr;
  a.near_sptr = P.d_near_sptr;
  a.near_src = P.d_near_src;
  a.near_zoff = P.d_near_zoff;
  a.near_z = P.d_near_z;
  a.x = x;
  a.w = w;
  a.N = P.N;
  const cplx c1 = P.k1 * P.k1 / (16.0 * kPi * kPi);
  const cplx c2v = P.k2 * P.k2 / (16.0 * kPi * kPi);
  a.c1 = c2(c1.real(), c1.imag());
  a.c2 = c2(c2v.real(), c2v.imag());
  a.etai = c2(P.etai.real(), P.etai.imag());
  const int warps = kThreads / 32;
  leaf_out_kernel<<<(P.N + warps - 1) / warps, kThreads, 0, s>>>(a);
  MLFMA_CUDA(cudaGetLastError());
  if (ev) MLFMA_CUDA(cudaEventRecord(ev[7], s));
}

}  // namespace mlfma

namespace mlfma {
// Sums the recorded stage times (ms) since the last read: out[0] aggregation,
// out[1] interpolation up, out[2] translation + anterpolation down,
// out[3] leaf testing + near field. Returns the number of applies covered.
int read_stage_times(Plan& P, double out[4]) {
  for (int i = 0; i < 4; ++i) out[i] = 0.0;
  const int n = static_cast<int>(P.prof.used);
  for (int a = 0; a < n; ++a) {
    auto& e = P.prof.sets[a];
    MLFMA_CUDA(cudaEventSynchronize(e[7]));
    float t[7];
    for (int i = 0; i < 7; ++i) MLFMA_CUDA(cudaEventElapsedTime(&t[i], e[i], e[i + 1]));
    out[0] += t[0] + t[3];
    out[1] += t[1] + t[4];
    out[2] += t[2] + t[5];
    out[3] += t[6];
  }
  P.prof.used = 0;
  return n;
}
}  // namespace mlfma
