// The PMCHWT MLFMA matvec on the GPU, FP64 (the `ax` closure of
// Code/MLFMM.cpp:189-368). J and M currents share the tree and the tables,
// so every stage processes both (6 complex components per direction) in one
// pass over the tables; media k1 and k2 run as separate launches.
//
//   agg      leaf aggregation           Code/ProcessMLFMM.h:33-56   (mexp)
//   up       interpolation + shift up   Code/ProcessMLFMM.h:61-107  (m2m)
//   m2l      translation over the interaction list   Code/ProcessMLFMM.h:112-147
//   l2l      the parent's incoming pattern, shifted and anterpolated onto
//            the child grid, added                    Code/ProcessMLFMM.h:152-202
//   leaf_out receive-pattern testing of both media and the near-field rows,
//            written once per unknown   Code/MLFMM.cpp:285-366
// Every stage writes its output before anything accumulates into it (l2l adds
// onto the Bm that m2l of the same level has just written), so no clearing
// pass (Code/ProcessMLFMM.h:14-28) is needed.
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

// One thread per (parent box, parent direction, component): the 9-tap
// separable interpolation of each child's pattern, times the child's shift
// phase, summed over the children. One component per thread keeps the
// register count low enough for the occupancy this gather needs.
__global__ void __launch_bounds__(kThreads) up_kernel(UpArg a) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  const int c = blockIdx.z;
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
  double2 acc = c2(0.0, 0.0);
  const int c1 = a.child_begin[b + 1];
  for (int ch = a.child_begin[b]; ch < c1; ++ch) {
    const double2 e = a.ph_up[a.octant[ch] * a.Kp + kk];
    const double2* sc = a.Sc + (static_cast<size_t>(ch) * 6 + c) * a.Kc;
    double2 v = c2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) v = cfmas(wt[i] * wp[j], __ldg(sc + ti[i] + pi[j]), v);
    acc = cfma(e, v, acc);
  }
  a.Sp[(static_cast<size_t>(b) * 6 + c) * a.Kp + kk] = acc;
}

struct M2lArg {
  const double2* S;     // this level's aggregated patterns
  double2* Bm;          // this level's incoming patterns (written)
  const int* far_ptr;
  const int* far_idx;
  const int* far_off;
  const int* off2vec;
  const double2* tfw;
  int K;
};

// Translation (m2l): one thread per (box, direction); the 6 components of
// each interaction-list source are applied with one transfer-factor load.
// Writes Bm (no accumulation into an earlier value).
__global__ void __launch_bounds__(kThreads) m2l_kernel(M2lArg a) {
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
  double2* out = a.Bm + static_cast<size_t>(b) * 6 * a.K + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * a.K] = acc[c];
}

struct M2lTileArg {
  const double2* S;
  double2* Bm;
  const int* child_begin;  // parent level: range of children (the targets)
  const int* usrc_ptr;     // per parent: union of its children's interaction sources
  const int* usrc;
  const int* coord;        // [3 * B] integer box coordinates at this level
  const int* off2vec;
  const double2* tfw;
  int K;
};

constexpr int kTileDirs = 32;   // directions per CTA (one per lane)
constexpr int kTileWarps = 8;   // one warp per child slot of the parent
constexpr int kTileBatch = 14;  // sources staged per round (static shared memory < 48 KB)

// Translation by sibling groups: one CTA per (parent box, 32-direction
// chunk), one warp per child. The union of the children's interaction
// sources (children of the parent's 27-neighbourhood) is staged through
// shared memory in batches, so each source pattern crosses L2 once per
// sibling group instead of once per target. Each warp then applies the
// sources that interact with its child (Chebyshev distance >= 2 in box
// units), in the same ascending source order as m2l_kernel.
__global__ void __launch_bounds__(kTileDirs * kTileWarps) m2l_tile_kernel(M2lTileArg a) {
  __shared__ double2 sS[kTileBatch][6][kTileDirs];
  __shared__ int sSrc[kTileBatch][4];  // x, y, z, box
  __shared__ int sVec[343];
  const int P = blockIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int kk = blockIdx.y * kTileDirs + lane;
  for (int i = threadIdx.x; i < 343; i += blockDim.x) sVec[i] = a.off2vec[i];
  const int c0 = a.child_begin[P], nc = a.child_begin[P + 1] - c0;
  const int t = c0 + w;
  const bool active = w < nc;
  int tx = 0, ty = 0, tz = 0;
  if (active) {
    tx = a.coord[3 * t];
    ty = a.coord[3 * t + 1];
    tz = a.coord[3 * t + 2];
  }
  double2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = c2(0.0, 0.0);
  const int u0 = a.usrc_ptr[P], nu = a.usrc_ptr[P + 1] - u0;
  for (int base = 0; base < nu; base += kTileBatch) {
    const int nb = min(kTileBatch, nu - base);
    __syncthreads();
    if (threadIdx.x < nb) {
      const int sb = a.usrc[u0 + base + threadIdx.x];
      sSrc[threadIdx.x][0] = a.coord[3 * sb];
      sSrc[threadIdx.x][1] = a.coord[3 * sb + 1];
      sSrc[threadIdx.x][2] = a.coord[3 * sb + 2];
      sSrc[threadIdx.x][3] = sb;
    }
    // stage nb sources x 6 components x 32 directions (one 512-byte row per warp load)
    for (int row = w; row < nb * 6; row += kTileWarps) {
      const int j = row / 6, c = row - 6 * j;
      const int sb = a.usrc[u0 + base + j];
      sS[j][c][lane] = kk < a.K ? a.S[(static_cast<size_t>(sb) * 6 + c) * a.K + kk] : c2(0.0, 0.0);
    }
    __syncthreads();
    if (active && kk < a.K) {
      for (int j = 0; j < nb; ++j) {
        const int dx = tx - sSrc[j][0], dy = ty - sSrc[j][1], dz = tz - sSrc[j][2];
        if (max(abs(dx), max(abs(dy), abs(dz))) < 2) continue;  // near: not translated
        const int v = sVec[(dx + 3) * 49 + (dy + 3) * 7 + (dz + 3)];
        const double2 tf = __ldg(a.tfw + static_cast<size_t>(v) * a.K + kk);
#pragma unroll
        for (int c = 0; c < 6; ++c) acc[c] = cfma(tf, sS[j][c][lane], acc[c]);
      }
    }
  }
  if (active && kk < a.K) {
    double2* out = a.Bm + static_cast<size_t>(t) * 6 * a.K + kk;
#pragma unroll
    for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * a.K] = acc[c];
  }
}

struct L2lArg {
  double2* Bm;           // child level (accumulated into)
  const double2* Bp;     // parent level
  const int* parent;     // of child boxes
  const int* octant;     // of child boxes
  const double2* ph_dn;  // parent level table [8][Kp]
  const int* tr_ptr;     // child direction -> (parent direction, weight)
  const int* tr_kp;
  const double* tr_w;
  int K, Kp;
};

// Anterpolation (l2l): one thread per (child box, child direction,
// component) adds the parent's incoming pattern, shifted to the child centre
// and interpolated transposed onto the child grid.
__global__ void __launch_bounds__(kThreads) l2l_kernel(L2lArg a) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  const int c = blockIdx.z;
  if (kk >= a.K) return;
  const double2* ph = a.ph_dn + a.octant[b] * a.Kp;
  const double2* bp = a.Bp + (static_cast<size_t>(a.parent[b]) * 6 + c) * a.Kp;
  double2 acc = c2(0.0, 0.0);
  const int t1 = a.tr_ptr[kk + 1];
  for (int e = a.tr_ptr[kk]; e < t1; ++e) {
    const int kp = __ldg(a.tr_kp + e);
    acc = cfma(cscale(__ldg(ph + kp), __ldg(a.tr_w + e)), __ldg(bp + kp), acc);
  }
  double2* out = a.Bm + (static_cast<size_t>(b) * 6 + c) * a.K + kk;
  *out = cadd(*out, acc);
}

struct L2lSepArg {
  double2* Bm;           // child level (accumulated into)
  const double2* Bp;     // parent level
  const int* parent;     // of child boxes
  const int* octant;     // of child boxes
  const double2* ph_dn;  // parent level table [8][Kp]
  const int* th_ptr;     // child theta row -> (parent theta row, Lagrange weight)
  const int* th_src;
  const double* th_w;
  const int* ph_ptr;     // child phi column -> (parent phi column, Lagrange weight)
  const int* ph_src;
  const double* ph_w;
  int ntc, npc, ntp, npp;
};

constexpr int kL2lRows = 8;        // child theta rows per band at most
constexpr int kL2lBand = 2944;     // band entries in shared memory (46 KiB)
constexpr int kL2lMaxPhi = kL2lBand;

// Anterpolation (l2l), separable: the parent's incoming pattern is shifted to
// the child centre, then spread onto the child grid by the transposed
// theta interpolation (into a shared-memory band of child rows x parent phi
// columns) and the transposed phi interpolation. One CTA per (child box,
// component); the reference's 9-tap weight of a (parent, child) direction
// pair is the product of the two 1-D weights used here (Code/AlgoMLFMM.h:347-351).
__global__ void __launch_bounds__(256) l2l_sep_kernel(L2lSepArg a) {
  __shared__ double2 band[kL2lBand];
  const int b = blockIdx.x, c = blockIdx.y;
  const int band_rows = max(1, min(kL2lRows, kL2lBand / a.npp));
  const int Kp = a.ntp * a.npp, Kc = a.ntc * a.npc;
  const double2* ph = a.ph_dn + a.octant[b] * Kp;
  const double2* bp = a.Bp + (static_cast<size_t>(a.parent[b]) * 6 + c) * Kp;
  double2* out = a.Bm + (static_cast<size_t>(b) * 6 + c) * Kc;
  for (int tc0 = 0; tc0 < a.ntc; tc0 += band_rows) {
    const int rows = min(band_rows, a.ntc - tc0);
    __syncthreads();
    for (int e = threadIdx.x; e < rows * a.npp; e += blockDim.x) {
      const int r = e / a.npp, pp = e - r * a.npp;
      const int tc = tc0 + r;
      double2 v = c2(0.0, 0.0);
      for (int q = a.th_ptr[tc]; q < a.th_ptr[tc + 1]; ++q) {
        const int kp = a.th_src[q] * a.npp + pp;
        v = cfmas(a.th_w[q], cmul(__ldg(ph + kp), __ldg(bp + kp)), v);
      }
      band[r * a.npp + pp] = v;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rows * a.npc; e += blockDim.x) {
      const int r = e / a.npc, pc = e - r * a.npc;
      double2 v = c2(0.0, 0.0);
      for (int q = a.ph_ptr[pc]; q < a.ph_ptr[pc + 1]; ++q) v = cfmas(a.ph_w[q], band[r * a.npp + a.ph_src[q]], v);
      double2* o = out + (tc0 + r) * a.npc + pc;
      *o = cadd(*o, v);
    }
  }
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
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[1 + 4 * m], s));
    for (int l = L - 1; l >= 2; --l) {
      const MediumLevel& pm = P.ml[m][l];
      const MediumLevel& cm = P.ml[m][l + 1];
      UpArg a{cm.S, pm.S, P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx, pm.lp,
              pm.ph_up, pm.K, pm.nph, cm.K, cm.nph};
      dim3 gu(P.lv[l].B, (pm.K + kThreads - 1) / kThreads, 6);
      up_kernel<<<gu, kThreads, 0, s>>>(a);
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[2 + 4 * m], s));
    // translations of every level (independent of each other) ...
    for (int l = 2; l <= L; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      if (P.tuning.m2l_variant == 1) {
        M2lTileArg a{cm.S, cm.Bm, P.lv[l - 1].child_begin, P.lv[l].usrc_ptr, P.lv[l].usrc, P.lv[l].coord,
                     cm.off2vec, cm.tfw, cm.K};
        dim3 gd(P.lv[l - 1].B, (cm.K + kTileDirs - 1) / kTileDirs);
        m2l_tile_kernel<<<gd, kTileDirs * kTileWarps, 0, s>>>(a);
      } else {
        M2lArg a{cm.S, cm.Bm, P.lv[l].far_ptr, P.lv[l].far_idx, P.lv[l].far_off, cm.off2vec, cm.tfw, cm.K};
        dim3 gd(P.lv[l].B, (cm.K + kThreads - 1) / kThreads);
        m2l_kernel<<<gd, kThreads, 0, s>>>(a);
      }
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[3 + 4 * m], s));
    // ... then the downward chain: level l receives level l-1 once that is final
    for (int l = 3; l <= L; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      const MediumLevel& pm = P.ml[m][l - 1];
      if (P.tuning.l2l_variant == 1 && pm.nph <= kL2lMaxPhi) {
        L2lSepArg b{cm.Bm,      pm.Bm,     P.lv[l].parent, P.lv[l].octant, pm.ph_dn, cm.thT_ptr,
                    cm.thT_src, cm.thT_w,  cm.phT_ptr,     cm.phT_src,     cm.phT_w, cm.nth,
                    cm.nph,     pm.nth,    pm.nph};
        l2l_sep_kernel<<<dim3(P.lv[l].B, 6), 256, 0, s>>>(b);
      } else {
        L2lArg b{cm.Bm, pm.Bm, P.lv[l].parent, P.lv[l].octant, pm.ph_dn, cm.tr_ptr, cm.tr_kp, cm.tr_w, cm.K, pm.K};
        dim3 gl(P.lv[l].B, (cm.K + kThreads - 1) / kThreads, 6);
        l2l_kernel<<<gl, kThreads, 0, s>>>(b);
      }
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[4 + 4 * m], s));
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
  if (ev) MLFMA_CUDA(cudaEventRecord(ev[9], s));
}

}  // namespace mlfma

namespace mlfma {
// Sums the recorded stage times (ms) since the last read: out[0] aggregation,
// out[1] interpolation up, out[2] translation, out[3] anterpolation down,
// out[4] leaf testing + near field. Returns the number of applies covered.
int read_stage_times(Plan& P, double out[kStages]) {
  for (int i = 0; i < kStages; ++i) out[i] = 0.0;
  const int n = static_cast<int>(P.prof.used);
  for (int a = 0; a < n; ++a) {
    auto& e = P.prof.sets[a];
    MLFMA_CUDA(cudaEventSynchronize(e[StageProfiler::kEvents - 1]));
    float t[StageProfiler::kEvents - 1];
    for (int i = 0; i + 1 < StageProfiler::kEvents; ++i) MLFMA_CUDA(cudaEventElapsedTime(&t[i], e[i], e[i + 1]));
    for (int m = 0; m < 2; ++m)
      for (int k = 0; k < 4; ++k) out[k] += t[4 * m + k];
    out[4] += t[8];
  }
  P.prof.used = 0;
  return n;
}
}  // namespace mlfma
