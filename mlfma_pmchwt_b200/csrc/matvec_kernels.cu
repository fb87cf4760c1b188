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
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>

#include "agg_tc.hpp"
#include "bulk.cuh"
#include "cplx.cuh"
#include "plan.hpp"
#include "solver.hpp"

namespace mlfma {

namespace {

constexpr int kThreads = 128;

// Aggregation: thread per (leaf box, direction), J and M from one pattern load.
template <class C>
__global__ void __launch_bounds__(kThreads) agg_kernel(const C* __restrict__ Vs, const int* __restrict__ leaf_ptr,
                                                       const int* __restrict__ leaf_rwg,
                                                       const double2* __restrict__ x, int N, int K,
                                                       C* __restrict__ S) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  if (kk >= K) return;
  C acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = Cx<C>::zero();
  const int r1 = leaf_ptr[b + 1];
  for (int r = leaf_ptr[b]; r < r1; ++r) {
    const int id = leaf_rwg[r];
    const C xJ = Cx<C>::from(x[id]), xM = Cx<C>::from(x[N + id]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const C v = Vs[(static_cast<size_t>(r) * 3 + c) * K + kk];
      acc[c] = cfma(v, xJ, acc[c]);
      acc[3 + c] = cfma(v, xM, acc[3 + c]);
    }
  }
  C* out = S + static_cast<size_t>(b) * 6 * K + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * K] = acc[c];
}

struct AggBoxArg {
  const double2* Vs[2];  // radiation patterns per medium [N][3][K] (leaf order)
  double2* S[2];         // leaf-level patterns per medium [Bleaf][6][K]
  int K[2];
  const int* leaf_ptr;
  const int* leaf_rwg;
  const double2* x;
  int N;
};

// Aggregation, CTA per (leaf box, medium): the box's radiation patterns are
// one contiguous block [n_b][3K] in leaf order, streamed by threads over its
// 3K entries, two columns per thread (J components land at S[b][0..2], M at
// S[b][3..5]). The box's currents are staged in shared memory first (boxes
// of more than kAggStage RWGs read them from global memory).
constexpr int kAggStage = 64;

__global__ void __launch_bounds__(kThreads) agg_box_kernel(AggBoxArg a) {
  __shared__ double2 sx[2][kAggStage];
  const int b = blockIdx.x, m = blockIdx.y;
  const int K3 = 3 * a.K[m];
  const int r0 = a.leaf_ptr[b], nb = a.leaf_ptr[b + 1] - r0;
  const bool staged = nb <= kAggStage;
  if (staged)
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
      const int id = a.leaf_rwg[r0 + i];
      sx[0][i] = a.x[id];
      sx[1][i] = a.x[a.N + id];
    }
  __syncthreads();
  const double2* V = a.Vs[m] + static_cast<size_t>(r0) * K3;
  double2* out = a.S[m] + static_cast<size_t>(b) * 2 * K3;
  for (int e0 = threadIdx.x; e0 < K3; e0 += 2 * blockDim.x) {
    const int e1 = e0 + blockDim.x;
    const bool two = e1 < K3;
    double2 aJ0 = c2(0.0, 0.0), aM0 = c2(0.0, 0.0), aJ1 = c2(0.0, 0.0), aM1 = c2(0.0, 0.0);
    const double2* v = V + e0;
#pragma unroll 4
    for (int r = 0; r < nb; ++r, v += K3) {
      double2 xJ, xM;
      if (staged) {
        xJ = sx[0][r];
        xM = sx[1][r];
      } else {
        const int id = __ldg(a.leaf_rwg + r0 + r);
        xJ = __ldg(a.x + id);
        xM = __ldg(a.x + a.N + id);
      }
      const double2 s0 = __ldg(v);
      const double2 s1 = two ? __ldg(v + blockDim.x) : c2(0.0, 0.0);
      aJ0 = cfma(s0, xJ, aJ0);
      aM0 = cfma(s0, xM, aM0);
      aJ1 = cfma(s1, xJ, aJ1);
      aM1 = cfma(s1, xM, aM1);
    }
    out[e0] = aJ0;
    out[K3 + e0] = aM0;
    if (two) {
      out[e1] = aJ1;
      out[K3 + e1] = aM1;
    }
  }
}

template <class C>
struct UpArg {
  const C* Sc;   // child level patterns [Bc][6][Kc]
  C* Sp;               // parent level patterns [Bp][6][Kp]
  const int* child_begin;
  const int* octant;   // of child boxes
  const int* tidx;
  const double* lt;
  const int* pidx;
  const double* lp;
  const C* ph_up;
  int Kp, nphp, Kc, nphc;
  long long slot_c = 0, slot_p = 0;  // element strides between right-hand-side slots (grid.z = 6 x slots)
};

// One thread per (parent box, parent direction, component): the 9-tap
// separable interpolation of each child's pattern, times the child's shift
// phase, summed over the children. One component per thread keeps the
// register count low enough for the occupancy this gather needs.
// kSlots: grid.z = 6 x slots with the slot offsets of the batched tree; the
// single apply instantiates without them.
// kT: threads per CTA (a tile of kT parent directions of one box and component)
template <class C, bool kSlots = false, int kT = kThreads>
__global__ void __launch_bounds__(kT) up_kernel(UpArg<C> a) {
  using R = typename Cx<C>::real;
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  const int slot = kSlots ? blockIdx.z / 6 : 0;
  const int c = blockIdx.z - 6 * slot;
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
  C acc = Cx<C>::zero();
  const int c1 = a.child_begin[b + 1];
  for (int ch = a.child_begin[b]; ch < c1; ++ch) {
    const C e = __ldg(a.ph_up + a.octant[ch] * a.Kp + kk);
    const C* sc = (kSlots ? a.Sc + slot * a.slot_c : a.Sc) + (static_cast<size_t>(ch) * 6 + c) * a.Kc;
    C v = Cx<C>::zero();
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) v = cfmas(static_cast<R>(wt[i] * wp[j]), __ldg(sc + ti[i] + pi[j]), v);
    acc = cfma(e, v, acc);
  }
  (kSlots ? a.Sp + slot * a.slot_p : a.Sp)[(static_cast<size_t>(b) * 6 + c) * a.Kp + kk] = acc;
}

// grid: (parent boxes, direction tiles of t, zdim = 6 components x slots)
template <class C, bool kSlots>
void launch_up(int t, int boxes, int K, int zdim, const UpArg<C>& a, cudaStream_t s) {
  const dim3 g(boxes, (K + t - 1) / t, zdim);
  if (t == 64)
    up_kernel<C, kSlots, 64><<<g, 64, 0, s>>>(a);
  else if (t == 256)
    up_kernel<C, kSlots, 256><<<g, 256, 0, s>>>(a);
  else
    up_kernel<C, kSlots, 128><<<g, 128, 0, s>>>(a);
}

// Interpolation (m2m), one thread per (parent box, parent direction) for all
// 6 components: the stencil (3 theta x 3 phi taps and weights) and the
// child's shift phase are loaded once per child and applied to the 6
// component rows, 54 independent loads per child in flight.
__global__ void __launch_bounds__(kThreads) up6_kernel(UpArg<double2> a) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int b = blockIdx.x;
  if (kk >= a.Kp) return;
  const int t = kk / a.nphp, p = kk - t * a.nphp;
  int ti[3], pi[3];
  double wt[3], wp[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    ti[i] = __ldg(a.tidx + 3 * t + i) * a.nphc;
    wt[i] = __ldg(a.lt + 3 * t + i);
    pi[i] = __ldg(a.pidx + 3 * p + i);
    wp[i] = __ldg(a.lp + 3 * p + i);
  }
  double2 acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = c2(0.0, 0.0);
  const int c1 = a.child_begin[b + 1];
  for (int ch = a.child_begin[b]; ch < c1; ++ch) {
    const double2 e = __ldg(a.ph_up + a.octant[ch] * a.Kp + kk);
    const double2* sc = a.Sc + static_cast<size_t>(ch) * 6 * a.Kc;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const double2* sr = sc + static_cast<size_t>(c) * a.Kc;
      double2 v = c2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) v = cfmas(wt[i] * wp[j], __ldg(sr + ti[i] + pi[j]), v);
      acc[c] = cfma(e, v, acc[c]);
    }
  }
  double2* out = a.Sp + static_cast<size_t>(b) * 6 * a.Kp + kk;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * a.Kp] = acc[c];
}

// Interpolation (m2m), separable in registers: thread per (parent box, band
// of kUpColBand parent theta rows, component, parent phi column). For each
// child it interpolates in phi each child theta row the band needs (3 taps;
// kept in the thread's own shared-memory slots, so no barrier), then forms
// the band's parent directions from 3 theta taps each, times the child's
// shift phase, accumulated over the children. About 5.5 loads per output
// against 10 for the 9-tap gather.
template <class C>
struct UpColArg {
  const C* Sc;
  C* Sp;
  const int* child_begin;
  const int* octant;
  const int* pidx;
  const double* lp;
  const double* lt;
  const int* row_ptr;  // per band: the child theta rows it needs
  const int* row;
  const int* tpos;     // [nthp][3]: band row of each theta tap
  const C* ph_up;
  int nthp, nphp, nphc, Kc;
};

template <class C>
__global__ void __launch_bounds__(kThreads) up_col_kernel(UpColArg<C> a) {
  using R = typename Cx<C>::real;
  __shared__ C rv[kUpColRows][kThreads];
  const int P = blockIdx.x, bi = blockIdx.y;
  const int q = blockIdx.z * blockDim.x + threadIdx.x;
  if (q >= 6 * a.nphp) return;
  const int c = q / a.nphp, p = q - c * a.nphp;
  const int t0 = bi * kUpColBand, nt = min(kUpColBand, a.nthp - t0);
  const int r0 = a.row_ptr[bi], nr = a.row_ptr[bi + 1] - r0;
  int pj[3];
  R wp[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    pj[j] = __ldg(a.pidx + 3 * p + j);
    wp[j] = static_cast<R>(__ldg(a.lp + 3 * p + j));
  }
  int tp[kUpColBand][3];
  R wt[kUpColBand][3];
#pragma unroll
  for (int t = 0; t < kUpColBand; ++t)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const bool in = t < nt;
      tp[t][i] = in ? __ldg(a.tpos + 3 * (t0 + t) + i) : 0;
      wt[t][i] = in ? static_cast<R>(__ldg(a.lt + 3 * (t0 + t) + i)) : R(0);
    }
  int rowoff[kUpColRows];
#pragma unroll
  for (int r = 0; r < kUpColRows; ++r) rowoff[r] = r < nr ? __ldg(a.row + r0 + r) * a.nphc : 0;
  C acc[kUpColBand];
#pragma unroll
  for (int t = 0; t < kUpColBand; ++t) acc[t] = Cx<C>::zero();
  const int Kp = a.nthp * a.nphp;
  C(*mine)[kThreads] = rv;
  const int me = threadIdx.x;
  const int c1 = a.child_begin[P + 1];
  for (int ch = a.child_begin[P]; ch < c1; ++ch) {
    const C* sc = a.Sc + (static_cast<size_t>(ch) * 6 + c) * a.Kc;
#pragma unroll
    for (int r = 0; r < kUpColRows; ++r) {
      if (r < nr) {
        const C* srow = sc + rowoff[r];
        C v = cscale(__ldg(srow + pj[0]), wp[0]);
        v = cfmas(wp[1], __ldg(srow + pj[1]), v);
        v = cfmas(wp[2], __ldg(srow + pj[2]), v);
        mine[r][me] = v;
      }
    }
    const C* ph = a.ph_up + a.octant[ch] * Kp + t0 * a.nphp + p;
#pragma unroll
    for (int t = 0; t < kUpColBand; ++t) {
      if (t < nt) {
        C v = cscale(mine[tp[t][0]][me], wt[t][0]);
        v = cfmas(wt[t][1], mine[tp[t][1]][me], v);
        v = cfmas(wt[t][2], mine[tp[t][2]][me], v);
        acc[t] = cfma(__ldg(ph + t * a.nphp), v, acc[t]);
      }
    }
  }
  C* out = a.Sp + (static_cast<size_t>(P) * 6 + c) * Kp + t0 * a.nphp + p;
#pragma unroll
  for (int t = 0; t < kUpColBand; ++t)
    if (t < nt) out[t * a.nphp] = acc[t];
}

struct UpSepArg {
  const double2* Sc;   // child level patterns [Bc][6][Kc]
  double2* Sp;         // parent level patterns [Bp][6][Kp]
  const int* child_begin;
  const int* octant;   // of child boxes
  const int* pidx;     // [nphp][3] into the child phi grid
  const double* lp;
  const double* lt;    // [nthp][3]
  const int* row_ptr;  // per band: child theta rows it needs
  const int* row;
  const int* tpos;     // [nthp][3]: band row of each theta tap
  const double2* ph_up;
  int nthp, nphp, nphc, Kc, R;
};

// Interpolation (m2m), separable: CTA per (parent box, component, band of R
// parent theta rows). For each child, the phi interpolation of the child
// rows the band needs goes to shared memory (3 taps), then each parent
// direction takes its 3 theta taps from there, times the child's shift
// phase, accumulated over the children in registers. The reference's 9-tap
// weight is the product of the two 1-D weights (Code/AlgoMLFMM.h:347-351).
__global__ void __launch_bounds__(256) up_sep_kernel(UpSepArg a) {
  __shared__ double2 T[kUpBandEntries];
  const int P = blockIdx.x, c = blockIdx.y, bi = blockIdx.z;
  const int t0 = bi * a.R;
  const int nout = min(a.R, a.nthp - t0) * a.nphp;
  const int r0 = a.row_ptr[bi], nr = a.row_ptr[bi + 1] - r0;
  const int Kp = a.nthp * a.nphp;
  constexpr int kPer = kUpBandOut / 256;
  double2 acc[kPer];
#pragma unroll
  for (int q = 0; q < kPer; ++q) acc[q] = c2(0.0, 0.0);
  const int ch1 = a.child_begin[P + 1];
  for (int ch = a.child_begin[P]; ch < ch1; ++ch) {
    const double2* sc = a.Sc + (static_cast<size_t>(ch) * 6 + c) * a.Kc;
    __syncthreads();
    for (int e = threadIdx.x; e < nr * a.nphp; e += blockDim.x) {
      const int r = e / a.nphp, p = e - r * a.nphp;
      const double2* srow = sc + __ldg(a.row + r0 + r) * a.nphc;
      double2 v = cscale(__ldg(srow + __ldg(a.pidx + 3 * p)), __ldg(a.lp + 3 * p));
      v = cfmas(__ldg(a.lp + 3 * p + 1), __ldg(srow + __ldg(a.pidx + 3 * p + 1)), v);
      v = cfmas(__ldg(a.lp + 3 * p + 2), __ldg(srow + __ldg(a.pidx + 3 * p + 2)), v);
      T[e] = v;
    }
    __syncthreads();
    const double2* ph = a.ph_up + a.octant[ch] * Kp + t0 * a.nphp;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int e = threadIdx.x + q * 256;
      if (e < nout) {
        const int r = e / a.nphp, p = e - r * a.nphp;
        const int t = t0 + r;
        double2 v = cscale(T[__ldg(a.tpos + 3 * t) * a.nphp + p], __ldg(a.lt + 3 * t));
        v = cfmas(__ldg(a.lt + 3 * t + 1), T[__ldg(a.tpos + 3 * t + 1) * a.nphp + p], v);
        v = cfmas(__ldg(a.lt + 3 * t + 2), T[__ldg(a.tpos + 3 * t + 2) * a.nphp + p], v);
        acc[q] = cfma(__ldg(ph + e), v, acc[q]);
      }
    }
  }
  double2* out = a.Sp + (static_cast<size_t>(P) * 6 + c) * Kp + t0 * a.nphp;
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    const int e = threadIdx.x + q * 256;
    if (e < nout) out[e] = acc[q];
  }
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

// Translation by octant registers, all levels of one medium in one launch.
// A CTA takes one parent box and 64 directions; thread (direction, half,
// group) keeps the incoming patterns of 4 of the parent's 8 octant children
// (group 0: octants 0-3, group 1: 4-7) for the J (half 0) or M (half 1)
// components in registers. The union of the children's interaction-list
// sources is staged in shared memory; each source pattern is loaded once per
// thread (the next one prefetched) and applied to every child of the group
// whose list holds it (octant mask), with that child's transfer factor.
constexpr int kM2lDirs = 64;
constexpr int kM2lThreads = 4 * kM2lDirs;
constexpr int kM2lMaxSeg = 14;  // levels 2..15
constexpr int kM2lStage = 512;  // union entries staged per round

struct M2lSeg {
  const double2* S;
  double2* Bm;
  const double2* tfw;
  const int* off2vec;
  const int* ufar_ptr;
  const int* ufar;
  const int* upack;
  const int* child_begin;  // parent level
  const int* octant;       // this level
  int K, nchunk, cta_begin;
};
struct M2lOctArg {
  M2lSeg seg[kM2lMaxSeg];
  int nseg;
};

__global__ void __launch_bounds__(kM2lThreads, 2) m2l_oct_kernel(const __grid_constant__ M2lOctArg a) {
  __shared__ int sVec[343];
  __shared__ int sChild[8];
  __shared__ int sSrc[kM2lStage];
  __shared__ int sPack[kM2lStage];
  int si = 0;
  while (si + 1 < a.nseg && static_cast<int>(blockIdx.x) >= a.seg[si + 1].cta_begin) ++si;
  const M2lSeg& g = a.seg[si];
  const int local = blockIdx.x - g.cta_begin;
  const int P = local / g.nchunk;
  const int k = (local - P * g.nchunk) * kM2lDirs + (threadIdx.x & (kM2lDirs - 1));
  const int h = (threadIdx.x / kM2lDirs) & 1;   // J or M
  const int grp = threadIdx.x / (2 * kM2lDirs);  // octants 4 grp .. 4 grp + 3
  const int K = g.K;
  const bool live = k < K;
  const int kq = live ? k : K - 1;
  for (int i = threadIdx.x; i < 343; i += blockDim.x) sVec[i] = g.off2vec[i];
  if (threadIdx.x < 8) sChild[threadIdx.x] = -1;
  __syncthreads();
  const int c0 = g.child_begin[P], c1 = g.child_begin[P + 1];
  if (threadIdx.x < c1 - c0) sChild[g.octant[c0 + threadIdx.x]] = c0 + threadIdx.x;
  double2 acc[4][3];
#pragma unroll
  for (int o = 0; o < 4; ++o)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[o][c] = c2(0.0, 0.0);
  const double2* Sbase = g.S + static_cast<size_t>(3 * h) * K + kq;
  const int u0 = g.ufar_ptr[P], nu = g.ufar_ptr[P + 1] - u0;
  for (int base = 0; base < nu; base += kM2lStage) {
    const int nb = min(kM2lStage, nu - base);
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
      sSrc[i] = g.ufar[u0 + base + i];
      sPack[i] = g.upack[u0 + base + i];
    }
    __syncthreads();
    const double2* src = Sbase + static_cast<size_t>(sSrc[0]) * 6 * K;
    double2 n0 = __ldg(src), n1 = __ldg(src + K), n2 = __ldg(src + 2 * K);
    for (int j = 0; j < nb; ++j) {
      const double2 s0 = n0, s1 = n1, s2 = n2;
      if (j + 1 < nb) {
        src = Sbase + static_cast<size_t>(sSrc[j + 1]) * 6 * K;
        n0 = __ldg(src);
        n1 = __ldg(src + K);
        n2 = __ldg(src + 2 * K);
      }
      const int pk = sPack[j];
      const int enc0 = pk & 511;
      const int mask = (pk >> (9 + 4 * grp)) & 15;
      double2 tf[4];
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        const int oo = 4 * grp + o;
        const int v = sVec[enc0 + (oo & 1) * 49 + ((oo >> 1) & 1) * 7 + (oo >> 2)];
        tf[o] = (mask >> o) & 1 ? __ldg(g.tfw + static_cast<size_t>(max(v, 0)) * K + kq) : c2(0.0, 0.0);
      }
#pragma unroll
      for (int o = 0; o < 4; ++o) {
        if ((mask >> o) & 1) {
          acc[o][0] = cfma(tf[o], s0, acc[o][0]);
          acc[o][1] = cfma(tf[o], s1, acc[o][1]);
          acc[o][2] = cfma(tf[o], s2, acc[o][2]);
        }
      }
    }
  }
  __syncthreads();
  if (!live) return;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const int t = sChild[4 * grp + o];
    if (t >= 0) {
      double2* out = g.Bm + (static_cast<size_t>(t) * 6 + 3 * h) * K + k;
      out[0] = acc[o][0];
      out[static_cast<size_t>(K)] = acc[o][1];
      out[2 * static_cast<size_t>(K)] = acc[o][2];
    }
  }
}

// Translation, warp per box: a CTA takes 8 Morton-consecutive boxes (one
// warp each) and 32 directions; every level of a medium in one launch. Each
// lane accumulates its box's 6 components over the box's interaction list,
// with one transfer-factor load per entry. Neighbouring boxes' lists hold
// largely the same sources in the same (ascending) order, so the 8 warps
// read the same source patterns at about the same time and L1 serves the
// repeats.
constexpr int kWarpBoxes = 8;

template <class C>
struct M2lWarpSeg {
  const C* S;
  C* Bm;
  const C* tfw;
  const int* far_ptr;
  const int* far_idx;
  const int* far_vec;
  int B, K, nchunk, cta_begin;
};
template <class C>
struct M2lWarpArg {
  M2lWarpSeg<C> seg[kM2lMaxSeg];
  int nseg;
};

template <class C>
__global__ void __launch_bounds__(32 * kWarpBoxes) m2l_warp_kernel(const __grid_constant__ M2lWarpArg<C> a) {
  int si = 0;
  while (si + 1 < a.nseg && static_cast<int>(blockIdx.x) >= a.seg[si + 1].cta_begin) ++si;
  const M2lWarpSeg<C>& g = a.seg[si];
  const int local = blockIdx.x - g.cta_begin;
  const int grp = local / g.nchunk;
  const int b = grp * kWarpBoxes + (threadIdx.x >> 5);
  const int k = (local - grp * g.nchunk) * 32 + (threadIdx.x & 31);
  const int K = g.K;
  if (b >= g.B || k >= K) return;
  C acc[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) acc[c] = Cx<C>::zero();
  const int e1 = g.far_ptr[b + 1];
  int e = g.far_ptr[b];
  for (; e + 1 < e1; e += 2) {
    const int s0 = __ldg(g.far_idx + e), s1 = __ldg(g.far_idx + e + 1);
    const C t0 = __ldg(g.tfw + static_cast<size_t>(__ldg(g.far_vec + e)) * K + k);
    const C t1 = __ldg(g.tfw + static_cast<size_t>(__ldg(g.far_vec + e + 1)) * K + k);
    const C* p0 = g.S + static_cast<size_t>(s0) * 6 * K + k;
    const C* p1 = g.S + static_cast<size_t>(s1) * 6 * K + k;
    C v0[6], v1[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      v0[c] = __ldg(p0 + static_cast<size_t>(c) * K);
      v1[c] = __ldg(p1 + static_cast<size_t>(c) * K);
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = cfma(t1, v1[c], cfma(t0, v0[c], acc[c]));
  }
  if (e < e1) {
    const int s0 = __ldg(g.far_idx + e);
    const C t0 = __ldg(g.tfw + static_cast<size_t>(__ldg(g.far_vec + e)) * K + k);
    const C* p0 = g.S + static_cast<size_t>(s0) * 6 * K + k;
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = cfma(t0, __ldg(p0 + static_cast<size_t>(c) * K), acc[c]);
  }
  C* out = g.Bm + static_cast<size_t>(b) * 6 * K + k;
#pragma unroll
  for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * K] = acc[c];
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

// Translation, warp per box pair: a CTA takes 4 pairs of Morton-consecutive
// boxes (2g, 2g+1; mostly siblings) and 32 directions. A lane walks the
// pair's merged, source-ordered interaction lists: each source pattern is
// loaded once and applied to whichever of the two boxes lists it, with that
// box's transfer factor. Each box still sums its sources in ascending order.
constexpr int kPairWarps = 4;

template <class C>
struct M2lPairSeg {
  const C* S;
  C* Bm;
  const C* tfw;
  const int* pair_ptr;
  const int* pair_src;
  const int2* pair_vec;
  int B, K, nchunk, cta_begin;
  long long slot_S = 0, slot_B = 0;  // element strides between right-hand-side slots (grid.y = slots)
};
template <class C>
struct M2lPairArg {
  M2lPairSeg<C> seg[kM2lMaxSeg];
  int nseg;
};

// kSlots: the slot offsets of the batched tree (grid.y = slot); the single
// apply instantiates without them (two registers fewer: 96 rather than 98 in
// FP64, which keeps five CTAs per SM).
// kW: box pairs (warps) per CTA.
template <class C, bool kSlots = false, int kW = kPairWarps>
__global__ void __launch_bounds__(32 * kW) m2l_pair_kernel(const __grid_constant__ M2lPairArg<C> a) {
  int si = 0;
  while (si + 1 < a.nseg && static_cast<int>(blockIdx.x) >= a.seg[si + 1].cta_begin) ++si;
  const M2lPairSeg<C>& g = a.seg[si];
  const int local = blockIdx.x - g.cta_begin;
  const int grp = local / g.nchunk;
  const int pg = grp * kW + (threadIdx.x >> 5);
  const int k = (local - grp * g.nchunk) * 32 + (threadIdx.x & 31);
  const int K = g.K;
  if (2 * pg >= g.B || k >= K) return;
  const C* const Sl = kSlots ? g.S + blockIdx.y * g.slot_S : g.S;
  C* const Bl = kSlots ? g.Bm + blockIdx.y * g.slot_B : g.Bm;
  C a0[6], a1[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) a0[c] = a1[c] = Cx<C>::zero();
  const int e1 = g.pair_ptr[pg + 1];
  for (int e = g.pair_ptr[pg]; e < e1; ++e) {
    const int src = __ldg(g.pair_src + e);
    const int2 v = __ldg(g.pair_vec + e);
    const C* p = Sl + static_cast<size_t>(src) * 6 * K + k;
    C sv[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) sv[c] = __ldg(p + static_cast<size_t>(c) * K);
    if (v.x >= 0) {
      const C t = __ldg(g.tfw + static_cast<size_t>(v.x) * K + k);
#pragma unroll
      for (int c = 0; c < 6; ++c) a0[c] = cfma(t, sv[c], a0[c]);
    }
    if (v.y >= 0) {
      const C t = __ldg(g.tfw + static_cast<size_t>(v.y) * K + k);
#pragma unroll
      for (int c = 0; c < 6; ++c) a1[c] = cfma(t, sv[c], a1[c]);
    }
  }
  C* out0 = Bl + static_cast<size_t>(2 * pg) * 6 * K + k;
#pragma unroll
  for (int c = 0; c < 6; ++c) out0[static_cast<size_t>(c) * K] = a0[c];
  if (2 * pg + 1 < g.B) {
    C* out1 = Bl + static_cast<size_t>(2 * pg + 1) * 6 * K + k;
#pragma unroll
    for (int c = 0; c < 6; ++c) out1[static_cast<size_t>(c) * K] = a1[c];
  }
}

// The same walk with each pair's J and M halves on two warps: a CTA of 8
// warps takes 4 pairs x {J, M}; a lane keeps 3 components of both boxes
// (half the registers of m2l_pair_kernel, twice the resident warps), and
// the transfer factors the two halves both load come from L1.
template <class C>
__global__ void __launch_bounds__(64 * kPairWarps) m2l_pairh_kernel(const __grid_constant__ M2lPairArg<C> a) {
  int si = 0;
  while (si + 1 < a.nseg && static_cast<int>(blockIdx.x) >= a.seg[si + 1].cta_begin) ++si;
  const M2lPairSeg<C>& g = a.seg[si];
  const int local = blockIdx.x - g.cta_begin;
  const int grp = local / g.nchunk;
  const int w = threadIdx.x >> 5;
  const int pg = grp * kPairWarps + (w >> 1), h = w & 1;
  const int k = (local - grp * g.nchunk) * 32 + (threadIdx.x & 31);
  const int K = g.K;
  if (2 * pg >= g.B || k >= K) return;
  C a0[3], a1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) a0[c] = a1[c] = Cx<C>::zero();
  const int e1 = g.pair_ptr[pg + 1];
  for (int e = g.pair_ptr[pg]; e < e1; ++e) {
    const int src = __ldg(g.pair_src + e);
    const int2 v = __ldg(g.pair_vec + e);
    const C* p = g.S + (static_cast<size_t>(src) * 6 + 3 * h) * K + k;
    C sv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) sv[c] = __ldg(p + static_cast<size_t>(c) * K);
    if (v.x >= 0) {
      const C t = __ldg(g.tfw + static_cast<size_t>(v.x) * K + k);
#pragma unroll
      for (int c = 0; c < 3; ++c) a0[c] = cfma(t, sv[c], a0[c]);
    }
    if (v.y >= 0) {
      const C t = __ldg(g.tfw + static_cast<size_t>(v.y) * K + k);
#pragma unroll
      for (int c = 0; c < 3; ++c) a1[c] = cfma(t, sv[c], a1[c]);
    }
  }
  C* out0 = g.Bm + (static_cast<size_t>(2 * pg) * 6 + 3 * h) * K + k;
#pragma unroll
  for (int c = 0; c < 3; ++c) out0[static_cast<size_t>(c) * K] = a0[c];
  if (2 * pg + 1 < g.B) {
    C* out1 = g.Bm + (static_cast<size_t>(2 * pg + 1) * 6 + 3 * h) * K + k;
#pragma unroll
    for (int c = 0; c < 3; ++c) out1[static_cast<size_t>(c) * K] = a1[c];
  }
}

// Tile shapes chosen at run time (tuning keys "m2l.pair_warps", "up.threads").
inline int pair_warps(const Plan& P) { return 2 << P.tuning.m2l_pair_warps; }
inline int up_threads(const Plan& P) { return 64 << P.tuning.up_threads; }

template <class C, bool kSlots>
void launch_m2l_pair(int w, dim3 grid, const M2lPairArg<C>& a, cudaStream_t st) {
  if (w == 2)
    m2l_pair_kernel<C, kSlots, 2><<<grid, 64, 0, st>>>(a);
  else if (w == 8)
    m2l_pair_kernel<C, kSlots, 8><<<grid, 256, 0, st>>>(a);
  else
    m2l_pair_kernel<C, kSlots, 4><<<grid, 128, 0, st>>>(a);
}

// Translation with staged sources: a CTA takes a group of 8 Morton-
// consecutive boxes and 32 directions. The group's interaction lists are
// merged into one source-ordered union whose entries carry the transfer-
// factor row of each member that lists the source. A producer warp stages,
// per union entry, the source's 6 pattern rows (one tiled TMA copy of a
// 6-row box) and the listed members' transfer-factor rows (two tile::gather4
// copies of 4 rows each) for 32 directions into a ring of shared-memory
// stages, completing on the stage's mbarrier, kGrpStages entries ahead of the
// arithmetic. kGrpBoxes / kBW compute warps, one direction per lane, apply
// every staged entry to their kBW boxes from shared memory only: no compute
// warp waits on a global load. A source pattern crosses L2 once per group
// instead of once per box pair. Each box still sums its sources in ascending
// order.
constexpr int kGrpBoxes = 8;
constexpr int kGrpDirs = 32;
constexpr int kGrpStages = 6;
constexpr int kGrpRows = 6 + kGrpBoxes;  // staged rows per entry: 6 pattern components, 8 transfer factors
constexpr int kGrpMaxSeg = 8;            // levels per launch

template <class C>
struct M2lGrpSeg {
  CUtensorMap smap;  // the level's patterns as rows [B * 6][2K] of scalars, box 2 * kGrpDirs x 6
  const C* S;
  const C* tfw;
  C* Bm;
  const int* grp_ptr;
  const int* grp_src;
  const int4* grp_code;
  int B, K, G, nchunk, cta_begin;
};
template <class C>
struct M2lGrpArg {
  M2lGrpSeg<C> seg[kGrpMaxSeg];
  int nseg;
  int* status;
};

template <class C>
constexpr size_t grp_smem_bytes() {
  return static_cast<size_t>(kGrpStages) * kGrpRows * kGrpDirs * sizeof(C) + kGrpStages * sizeof(int4) +
         2 * kGrpStages * sizeof(uint64_t);
}

__device__ __forceinline__ int grp_field(const int4& w, int j) {
  const int v = (j >> 1) == 0 ? w.x : (j >> 1) == 1 ? w.y : (j >> 1) == 2 ? w.z : w.w;
  return (j & 1) ? (v >> 16) : static_cast<int>(static_cast<short>(v & 0xffff));
}

template <class C, int kBW, bool kTmaS>
__global__ void __launch_bounds__(32 * (kGrpBoxes / kBW + 1)) m2l_grp_kernel(const __grid_constant__ M2lGrpArg<C> a) {
  constexpr int kCW = kGrpBoxes / kBW;  // compute warps; warp kCW is the producer
  constexpr uint32_t kRowBytes = kGrpDirs * sizeof(C);
  extern __shared__ __align__(128) unsigned char smem[];
  C* stage = reinterpret_cast<C*>(smem);  // [kGrpStages][kGrpRows][kGrpDirs]
  int4* codes = reinterpret_cast<int4*>(smem + static_cast<size_t>(kGrpStages) * kGrpRows * kRowBytes);
  uint64_t* full = reinterpret_cast<uint64_t*>(codes + kGrpStages);
  uint64_t* empty = full + kGrpStages;

  int si = 0;
  while (si + 1 < a.nseg && static_cast<int>(blockIdx.x) >= a.seg[si + 1].cta_begin) ++si;
  const M2lGrpSeg<C>& g = a.seg[si];
  const int local = blockIdx.x - g.cta_begin;
  const int chunk = local / g.G, grp = local - chunk * g.G;
  const int k0 = chunk * kGrpDirs;
  const int nk = min(kGrpDirs, g.K - k0);
  const int e0 = g.grp_ptr[grp], n = g.grp_ptr[grp + 1] - e0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (status_now(a.status) != 0) return;  // an earlier wait ran out: the output is void anyway
  if (threadIdx.x == 0) {
    for (int i = 0; i < kGrpStages; ++i) {
      mbar_init(full + i, 33);  // the producer's 32 lanes after their copies, and lane 0 with the codes
      mbar_init(empty + i, kCW);
    }
    mbar_init_fence();
  }
  __syncthreads();

  if (warp == kCW) {  // producer
    if (kTmaS && lane == 0) tma_prefetch_map(&g.smap);
    bool ok = true;
    int i = 0;
    for (int base = 0; base < n && ok; base += 32) {
      int src = 0;
      int4 cd = make_int4(-1, -1, -1, -1);
      if (base + lane < n) {
        src = __ldg(g.grp_src + e0 + base + lane);
        cd = __ldg(g.grp_code + e0 + base + lane);
      }
      const int cnt = min(32, n - base);
      for (int j = 0; j < cnt; ++j, ++i) {
        const int sj = __shfl_sync(0xffffffffu, src, j);
        const int4 cj = make_int4(__shfl_sync(0xffffffffu, cd.x, j), __shfl_sync(0xffffffffu, cd.y, j),
                                  __shfl_sync(0xffffffffu, cd.z, j), __shfl_sync(0xffffffffu, cd.w, j));
        const int st = i % kGrpStages;
        const bool waited =
            i < kGrpStages || mbar_wait(empty + st, ((i / kGrpStages) - 1) & 1, a.status, true, kStatusM2lGrp);
        if (!__all_sync(0xffffffffu, waited)) {
          ok = false;
          break;
        }
        C* dst = stage + st * kGrpRows * kGrpDirs;
        if (lane == 0) {  // the codes, released to the compute warps by this arrival
          codes[st] = cj;
          if (kTmaS) {
            mbar_arrive_expect_tx(full + st, 6 * kRowBytes);
            tma_load_2d(dst, &g.smap, 2 * k0, 6 * sj, full + st);
          } else {
            mbar_arrive(full + st);
          }
        }
        if (lane < nk) {
          if (!kTmaS) {
            const C* p = g.S + static_cast<size_t>(sj) * 6 * g.K + k0 + lane;
#pragma unroll
            for (int c = 0; c < 6; ++c) cp_async_ca<sizeof(C)>(dst + c * kGrpDirs + lane, p + static_cast<size_t>(c) * g.K);
          }
#pragma unroll
          for (int b = 0; b < kGrpBoxes; ++b) {
            const int code = grp_field(cj, b);
            if (code >= 0)
              cp_async_ca<sizeof(C)>(dst + (6 + b) * kGrpDirs + lane, g.tfw + static_cast<size_t>(code) * g.K + k0 + lane);
          }
        }
        cp_async_arrive(full + st);
      }
    }
    // the copies still in flight land before the producer leaves, so that the
    // CTA never ends (a compute warp may give up after a failed wait) with a
    // copy into its shared memory outstanding
    if (lane == 0)
      for (int q = max(0, i - kGrpStages); q < i; ++q)
        mbar_wait(full + q % kGrpStages, (q / kGrpStages) & 1, a.status, false, kStatusM2lGrp);
    return;
  }

  const int k = k0 + lane;
  C acc[kBW][6];
#pragma unroll
  for (int j = 0; j < kBW; ++j)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[j][c] = Cx<C>::zero();
  bool ok = true;
  for (int i = 0; i < n; ++i) {
    const int st = i % kGrpStages;
    if (!mbar_wait(full + st, (i / kGrpStages) & 1, a.status, true, kStatusM2lGrp)) {
      ok = false;
      break;
    }
    const int4 cw = codes[st];
    const C* sp = stage + st * kGrpRows * kGrpDirs + lane;
    unsigned mask = 0;  // this warp's boxes that list the source (warp-uniform)
#pragma unroll
    for (int j = 0; j < kBW; ++j) mask |= (grp_field(cw, warp * kBW + j) >= 0 ? 1u : 0u) << j;
    if (mask != 0) {
      C sv[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) sv[c] = sp[c * kGrpDirs];
#pragma unroll
      for (int j = 0; j < kBW; ++j) {
        if (mask & (1u << j)) {
          const C t = sp[(6 + warp * kBW + j) * kGrpDirs];
#pragma unroll
          for (int c = 0; c < 6; ++c) acc[j][c] = cfma(t, sv[c], acc[j][c]);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + st);
  }
  if (!ok || lane >= nk) return;
#pragma unroll
  for (int j = 0; j < kBW; ++j) {
    const int b = grp * kGrpBoxes + warp * kBW + j;
    if (b < g.B) {
      C* out = g.Bm + static_cast<size_t>(b) * 6 * g.K + k;
#pragma unroll
      for (int c = 0; c < 6; ++c) out[static_cast<size_t>(c) * g.K] = acc[j][c];
    }
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    MLFMA_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || p == nullptr)
      throw std::runtime_error("cuTensorMapEncodeTiled is not available from the driver");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// A 2-D tensor map over rows of K complex values (2K scalars each) with a
// box of 2 * kGrpDirs scalars by box_rows rows.
template <class C>
CUtensorMap rows_tensor_map(const C* base, int K, long long rows, int box_rows) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (static_cast<size_t>(K) * sizeof(C)) % 16 != 0)
    throw std::runtime_error("tensor map: rows not 16-byte aligned");
  CUtensorMap m;
  const cuuint64_t dims[2] = {2ull * static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(K) * sizeof(C)};
  const cuuint32_t box[2] = {2 * kGrpDirs, static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(
      &m, sizeof(C) == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
      const_cast<C*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed: " + std::to_string(r));
  return m;
}

// Segments (levels lo..hi) of staged-group translation launches, at most
// kGrpMaxSeg levels per launch. tf_at(l) gives the level's transfer-factor
// table and row count.
template <class C, class SAt, class BAt, class TfAt>
void launch_m2l_grp(Plan& P, int lo, int hi, int bw, bool tma_s, SAt S_at, BAt B_at, TfAt tf_at, cudaStream_t s) {
  static_assert(grp_smem_bytes<double2>() <= 48 * 1024, "staged translation needs the opt-in shared memory size");
  constexpr size_t smem = grp_smem_bytes<C>();
  for (int l0 = lo; l0 <= hi; l0 += kGrpMaxSeg) {
    M2lGrpArg<C> a{};
    a.status = P.d_status;
    int ctas = 0;
    for (int l = l0; l <= std::min(hi, l0 + kGrpMaxSeg - 1); ++l) {
      const auto tf = tf_at(l);  // (table, rows, K)
      M2lGrpSeg<C>& g = a.seg[a.nseg++];
      if (tma_s) g.smap = rows_tensor_map<C>(S_at(l), std::get<2>(tf), 6LL * P.lv[l].B, 6);
      g.S = S_at(l);
      g.tfw = std::get<0>(tf);
      g.Bm = B_at(l);
      g.grp_ptr = P.lv[l].grp_ptr;
      g.grp_src = P.lv[l].grp_src;
      g.grp_code = P.lv[l].grp_code;
      g.B = P.lv[l].B;
      g.K = std::get<2>(tf);
      g.G = (P.lv[l].B + kGrpBoxes - 1) / kGrpBoxes;
      g.nchunk = (g.K + kGrpDirs - 1) / kGrpDirs;
      g.cta_begin = ctas;
      ctas += g.G * g.nchunk;
    }
    if (tma_s)
      m2l_grp_kernel<C, 4, true><<<ctas, 32 * (kGrpBoxes / 4 + 1), smem, s>>>(a);
    else if (bw == 4)
      m2l_grp_kernel<C, 4, false><<<ctas, 32 * (kGrpBoxes / 4 + 1), smem, s>>>(a);
    else
      m2l_grp_kernel<C, 2, false><<<ctas, 32 * (kGrpBoxes / 2 + 1), smem, s>>>(a);
    MLFMA_CUDA(cudaGetLastError());
  }
}

template <class C>
struct L2lSepArg {
  C* Bm;                 // child level (accumulated into)
  const C* Bp;     // parent level
  const int* parent;     // of child boxes
  const int* octant;     // of child boxes
  const C* ph_dn;        // parent level table [8][Kp]
  const int* th_ptr;     // child theta row -> (parent theta row, Lagrange weight)
  const int* th_src;
  const double* th_w;
  const int* ph_ptr;     // child phi column -> (parent phi column, Lagrange weight)
  const int* ph_src;
  const double* ph_w;
  int ntc, npc, ntp, npp;
  long long slot_c = 0, slot_p = 0;  // element strides between right-hand-side slots (grid.z = slots)
};

constexpr int kL2lBand = 2944;     // band entries in shared memory (46 KiB), all 6 components

// child theta rows per band of the separable anterpolation
__host__ __device__ __forceinline__ int l2l_band_rows(int ntc, int npp) {
  return max(1, min(ntc, kL2lBand / (6 * npp)));
}

// CTAs per child box: one per band on levels with few boxes (so that the
// level fills the GPU), else one CTA walks all the bands of its box.
constexpr int kL2lSplitBoxes = 1024;
inline int l2l_grid_y(int boxes, int ntc, int npp) {
  const int nband = (ntc + l2l_band_rows(ntc, npp) - 1) / l2l_band_rows(ntc, npp);
  return boxes < kL2lSplitBoxes ? nband : 1;
}

// Anterpolation (l2l), separable: a CTA per child box (and, on levels with few
// boxes, per band of child theta rows) does all 6 components. The parent's incoming pattern is shifted to the child centre
// and spread onto the child grid by the transposed theta interpolation (into
// a shared-memory band of child rows x parent phi columns x 6 components),
// then by the transposed phi interpolation, and added to the child's Bm. The
// reference's 9-tap weight of a (parent, child) direction pair is the
// product of the two 1-D weights used here (Code/AlgoMLFMM.h:347-351).
// (4 CTAs per SM: 64 registers, up from 3 CTAs at 80.)
// kSlots: grid.z = slots with the slot offsets of the batched tree; the single
// apply instantiates without them.
template <class C, bool kSlots = false>
__global__ void __launch_bounds__(256, 4) l2l_sep_kernel(L2lSepArg<C> a) {
  using R = typename Cx<C>::real;
  __shared__ C band[kL2lBand];
  const int b = blockIdx.x;
  const int band_rows = l2l_band_rows(a.ntc, a.npp);
  const int Kp = a.ntp * a.npp, Kc = a.ntc * a.npc;
  const C* ph = a.ph_dn + a.octant[b] * Kp;
  const C* bp = (kSlots ? a.Bp + blockIdx.z * a.slot_p : a.Bp) + static_cast<size_t>(a.parent[b]) * 6 * Kp;
  C* out = (kSlots ? a.Bm + blockIdx.z * a.slot_c : a.Bm) + static_cast<size_t>(b) * 6 * Kc;
  for (int tc0 = blockIdx.y * band_rows; tc0 < a.ntc; tc0 += gridDim.y * band_rows) {
    const int rows = min(band_rows, a.ntc - tc0);
    const int stride = rows * a.npp;
    __syncthreads();
    for (int e = threadIdx.x; e < stride; e += blockDim.x) {
      const int r = e / a.npp, pp = e - r * a.npp;
      const int tc = tc0 + r;
      C v[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) v[c] = Cx<C>::zero();
      const int q1 = __ldg(a.th_ptr + tc + 1);
      for (int q = __ldg(a.th_ptr + tc); q < q1; ++q) {
        const int kp = __ldg(a.th_src + q) * a.npp + pp;
        const C f = cscale(__ldg(ph + kp), static_cast<R>(__ldg(a.th_w + q)));
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = cfma(f, __ldg(bp + static_cast<size_t>(c) * Kp + kp), v[c]);
      }
#pragma unroll
      for (int c = 0; c < 6; ++c) band[c * stride + e] = v[c];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rows * a.npc; e += blockDim.x) {
      const int r = e / a.npc, pc = e - r * a.npc;
      C v[6];
#pragma unroll
      for (int c = 0; c < 6; ++c) v[c] = Cx<C>::zero();
      const int q1 = __ldg(a.ph_ptr + pc + 1);
      for (int q = __ldg(a.ph_ptr + pc); q < q1; ++q) {
        const R w = static_cast<R>(__ldg(a.ph_w + q));
        const int src = r * a.npp + __ldg(a.ph_src + q);
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = cfmas(w, band[c * stride + src], v[c]);
      }
      C* o = out + (tc0 + r) * a.npc + pc;
#pragma unroll
      for (int c = 0; c < 6; ++c) o[static_cast<size_t>(c) * Kc] = cadd(o[static_cast<size_t>(c) * Kc], v[c]);
    }
  }
}

template <class C>
struct LeafArg {
  const C* Vf[2];
  const C* Bm[2];
  const double* khat[2];
  int K[2];
  const int* leaf_rwg;
  const int* rwg_box;     // leaf box of each RWG id
  const int* leaf_ptr;
  const int* near_sptr;
  const int* near_src;
  const long long* near_zoff;
  const C* near_z;
  const double2* x;
  double2* w;
  int N;
  C c1, c2, etai;
};

template <class C>
__device__ __forceinline__ C warp_sum(C v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// One warp per RWG (leaf order).
// kNear = false: the far-field testing only, added to the near-field product
// already in w (computed concurrently by near_apply).
template <class C, bool kNear = true>
__global__ void __launch_bounds__(kThreads) leaf_out_kernel(LeafArg<C> a) {
  using R = typename Cx<C>::real;
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= a.N) return;
  const int id = a.leaf_rwg[r];
  const int b = a.rwg_box[id];
  C res[8];  // L1J K1J L1M K1M L2J K2J L2M K2M
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const int K = a.K[m];
    const C* V = a.Vf[m] + static_cast<size_t>(r) * 3 * K;
    const C* B = a.Bm[m] + static_cast<size_t>(b) * 6 * K;
    const double* kh = a.khat[m];
    C LJ = Cx<C>::zero(), KJ = Cx<C>::zero(), LM = Cx<C>::zero(), KM = Cx<C>::zero();
#pragma unroll 2
    for (int kk = lane; kk < K; kk += 32) {
      const C v0 = V[kk], v1 = V[K + kk], v2 = V[2 * K + kk];
      const C j0 = B[kk], j1 = B[K + kk], j2 = B[2 * K + kk];
      const C m0 = B[3 * K + kk], m1 = B[4 * K + kk], m2 = B[5 * K + kk];
      // (-khat) x V
      const R ax = static_cast<R>(-kh[kk]), ay = static_cast<R>(-kh[K + kk]), az = static_cast<R>(-kh[2 * K + kk]);
      const C w0 = csub(cscale(v2, ay), cscale(v1, az));
      const C w1 = csub(cscale(v0, az), cscale(v2, ax));
      const C w2 = csub(cscale(v1, ax), cscale(v0, ay));
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
  C nJ = Cx<C>::zero(), nM = Cx<C>::zero();
  if constexpr (kNear) {
    const int s0 = a.near_sptr[b], ns = a.near_sptr[b + 1] - s0;
    const int tl = r - a.leaf_ptr[b];
    const C* Z = a.near_z + 3 * (a.near_zoff[b] + static_cast<long long>(tl) * ns);
#pragma unroll 2
    for (int j = lane; j < ns; j += 32) {
      const int s = a.near_src[s0 + j];
      const C xJ = Cx<C>::from(a.x[s]), xM = Cx<C>::from(a.x[a.N + s]);
      const C z11 = Z[3 * j], z12 = Z[3 * j + 1], z22 = Z[3 * j + 2];
      nJ = cfma(z11, xJ, cfma(z12, xM, nJ));
      nM = cfma(z22, xM, csub(nM, cmul(z12, xJ)));
    }
    nJ = warp_sum(nJ);
    nM = warp_sum(nM);
  }
  if (lane == 0) {
    // w[t]   = c1 (L1J - K1M) + c2 (etai L2J - K2M) + near
    // w[N+t] = c1 (K1J + L1M) + c2 (K2J + L2M / etai) + near
    const C L2M_eta = cdiv(res[6], a.etai);
    C wj = cmul(a.c1, csub(res[0], res[3]));
    wj = cadd(wj, cmul(a.c2, csub(cmul(a.etai, res[4]), res[7])));
    C wm = cmul(a.c1, cadd(res[1], res[2]));
    wm = cadd(wm, cmul(a.c2, cadd(res[5], L2M_eta)));
    if constexpr (kNear) {
      a.w[id] = Cx<C>::to64(cadd(wj, nJ));
      a.w[a.N + id] = Cx<C>::to64(cadd(wm, nM));
    } else {
      a.w[id] = cadd(a.w[id], Cx<C>::to64(wj));
      a.w[a.N + id] = cadd(a.w[a.N + id], Cx<C>::to64(wm));
    }
  }
}

// ---------------------------------------------------------------- batched
// Several right-hand sides per pass over the leaf tables: the aggregation and
// the leaf testing + near field read each radiation / receive pattern and
// each near-field entry once for a group of right-hand sides. Accumulation
// orders are those of agg_box_kernel and leaf_out_kernel, so each right-hand
// side of a batch gets the single apply's result.
template <class C>
struct AggBatchArg {
  const C* Vs[2];
  C* S[2][kBatchSlots];  // leaf-level S of each slot
  int K[2];
  const int* leaf_ptr;
  const int* leaf_rwg;
  const double2* X;            // right-hand side j at X + j * ldx
  long long ldx;
  int N, R;
};

template <class C, int RB>
__global__ void __launch_bounds__(kThreads) agg_batch_kernel(AggBatchArg<C> a) {
  const int b = blockIdx.x, m = blockIdx.y;
  const int j0 = blockIdx.z * RB, jn = min(RB, a.R - j0);
  const int K3 = 3 * a.K[m];
  const int r0 = a.leaf_ptr[b], r1 = a.leaf_ptr[b + 1];
  const C* V = a.Vs[m] + static_cast<size_t>(r0) * K3;
  for (int e = threadIdx.x; e < K3; e += blockDim.x) {
    C aJ[RB], aM[RB];
#pragma unroll
    for (int j = 0; j < RB; ++j) aJ[j] = aM[j] = Cx<C>::zero();
    const C* v = V + e;
    for (int r = r0; r < r1; ++r, v += K3) {
      const int id = __ldg(a.leaf_rwg + r);
      const C s = __ldg(v);
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j < jn) {
          const double2* x = a.X + (j0 + j) * a.ldx;
          aJ[j] = cfma(s, Cx<C>::from(__ldg(x + id)), aJ[j]);
          aM[j] = cfma(s, Cx<C>::from(__ldg(x + a.N + id)), aM[j]);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < RB; ++j) {
      if (j < jn) {
        C* out = a.S[m][j0 + j] + static_cast<size_t>(b) * 2 * K3;
        out[e] = aJ[j];
        out[K3 + e] = aM[j];
      }
    }
  }
}

template <class C>
struct LeafBatchArg {
  const C* Vf[2];
  const C* Bm[2][kBatchSlots];  // leaf-level Bm of each slot
  const double* khat[2];
  int K[2];
  const int* leaf_rwg;
  const int* rwg_box;
  const int* leaf_ptr;
  const int* near_sptr;
  const int* near_src;
  const long long* near_zoff;
  const C* near_z;
  const double2* X;
  long long ldx;
  double2* W;
  long long ldw;
  int N, R;
  C c1, c2, etai;
};

// One warp per (RWG, group of RB right-hand sides).
// kFar = false: the near-field rows alone (the far field is added by the
// tensor-core testing kernel).
template <class C, int RB, bool kFar = true>
__global__ void __launch_bounds__(kThreads) leaf_out_batch_kernel(LeafBatchArg<C> a) {
  using Rl = typename Cx<C>::real;
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (r >= a.N) return;
  const int j0 = blockIdx.y * RB, jn = min(RB, a.R - j0);
  const int id = a.leaf_rwg[r];
  const int b = a.rwg_box[id];
  C wj[RB], wm[RB];
#pragma unroll
  for (int j = 0; j < RB; ++j) wj[j] = wm[j] = Cx<C>::zero();
#pragma unroll
  for (int m = 0; m < (kFar ? 2 : 0); ++m) {
    const int K = a.K[m];
    const C* V = a.Vf[m] + static_cast<size_t>(r) * 3 * K;
    const double* kh = a.khat[m];
    C acc[RB][4];  // LJ KJ LM KM
#pragma unroll
    for (int j = 0; j < RB; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[j][q] = Cx<C>::zero();
    for (int kk = lane; kk < K; kk += 32) {
      const C v0 = V[kk], v1 = V[K + kk], v2 = V[2 * K + kk];
      // (-khat) x V
      const Rl ax = static_cast<Rl>(-kh[kk]), ay = static_cast<Rl>(-kh[K + kk]), az = static_cast<Rl>(-kh[2 * K + kk]);
      const C w0 = csub(cscale(v2, ay), cscale(v1, az));
      const C w1 = csub(cscale(v0, az), cscale(v2, ax));
      const C w2 = csub(cscale(v1, ax), cscale(v0, ay));
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j < jn) {
          const C* B = a.Bm[m][j0 + j] + static_cast<size_t>(b) * 6 * K;
          const C b0 = B[kk], b1 = B[K + kk], b2 = B[2 * K + kk];
          const C m0 = B[3 * K + kk], m1 = B[4 * K + kk], m2 = B[5 * K + kk];
          acc[j][0] = cfma(v0, b0, cfma(v1, b1, cfma(v2, b2, acc[j][0])));
          acc[j][2] = cfma(v0, m0, cfma(v1, m1, cfma(v2, m2, acc[j][2])));
          acc[j][1] = cfma(w0, b0, cfma(w1, b1, cfma(w2, b2, acc[j][1])));
          acc[j][3] = cfma(w0, m0, cfma(w1, m1, cfma(w2, m2, acc[j][3])));
        }
      }
    }
#pragma unroll
    for (int j = 0; j < RB; ++j) {
      const C LJ = warp_sum(acc[j][0]), KJ = warp_sum(acc[j][1]);
      const C LM = warp_sum(acc[j][2]), KM = warp_sum(acc[j][3]);
      if (m == 0) {
        wj[j] = cmul(a.c1, csub(LJ, KM));
        wm[j] = cmul(a.c1, cadd(KJ, LM));
      } else {
        wj[j] = cadd(wj[j], cmul(a.c2, csub(cmul(a.etai, LJ), KM)));
        wm[j] = cadd(wm[j], cmul(a.c2, cadd(KJ, cdiv(LM, a.etai))));
      }
    }
  }
  const int s0 = a.near_sptr[b], ns = a.near_sptr[b + 1] - s0;
  const int tl = r - a.leaf_ptr[b];
  const C* Z = a.near_z + 3 * (a.near_zoff[b] + static_cast<long long>(tl) * ns);
  C nJ[RB], nM[RB];
#pragma unroll
  for (int j = 0; j < RB; ++j) nJ[j] = nM[j] = Cx<C>::zero();
  for (int q = lane; q < ns; q += 32) {
    const int src = a.near_src[s0 + q];
    const C z11 = Z[3 * q], z12 = Z[3 * q + 1], z22 = Z[3 * q + 2];
#pragma unroll
    for (int j = 0; j < RB; ++j) {
      if (j < jn) {
        const double2* x = a.X + (j0 + j) * a.ldx;
        const C xJ = Cx<C>::from(x[src]), xM = Cx<C>::from(x[a.N + src]);
        nJ[j] = cfma(z11, xJ, cfma(z12, xM, nJ[j]));
        nM[j] = cfma(z22, xM, csub(nM[j], cmul(z12, xJ)));
      }
    }
  }
#pragma unroll
  for (int j = 0; j < RB; ++j) {
    const C sJ = warp_sum(nJ[j]), sM = warp_sum(nM[j]);
    if (lane == 0 && j < jn) {
      double2* w = a.W + (j0 + j) * a.ldw;
      w[id] = Cx<C>::to64(cadd(wj[j], sJ));
      w[a.N + id] = Cx<C>::to64(cadd(wm[j], sM));
    }
  }
}

// Leaf-level pattern arrays of a tree pass: the plan's own, or one RHS slot
// of a batched apply. Levels above the leaf always use the plan's arrays.
struct LeafView {
  const double2* S;
  double2* B;
};

const double2* level_S(const Plan& P, int m, int l, const LeafView& v) { return l == P.maxL ? v.S : P.ml[m][l].S; }
double2* level_B(const Plan& P, int m, int l, const LeafView& v) { return l == P.maxL ? v.B : P.ml[m][l].Bm; }

// Interpolation up the tree (levels L-1 .. 2) of medium m.
void launch_up(Plan& P, int m, const LeafView& v, cudaStream_t s) {
  const int L = P.maxL;
  for (int l = L - 1; l >= 2; --l) {
    const MediumLevel& pm = P.ml[m][l];
    const MediumLevel& cm = P.ml[m][l + 1];
    const double2* Sc = level_S(P, m, l + 1, v);
    if (P.tuning.up_variant == 3 && pm.up4_row_ptr) {
      UpColArg<double2> a{Sc,     pm.S,           P.lv[l].child_begin, P.lv[l + 1].octant, pm.pidx, pm.lp,
                          pm.lt,  pm.up4_row_ptr, pm.up4_row,          pm.up4_tpos,        pm.ph_up, pm.nth,
                          pm.nph, cm.nph,         cm.K};
      up_col_kernel<double2>
          <<<dim3(P.lv[l].B, pm.up4_nband, (6 * pm.nph + kThreads - 1) / kThreads), kThreads, 0, s>>>(a);
    } else if (P.tuning.up_variant == 2) {
      UpArg<double2> a{Sc, pm.S, P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx, pm.lp,
                       pm.ph_up, pm.K, pm.nph, cm.K, cm.nph};
      up6_kernel<<<dim3(P.lv[l].B, (pm.K + kThreads - 1) / kThreads), kThreads, 0, s>>>(a);
    } else if (P.tuning.up_variant == 1 && pm.up_rows > 0) {
      UpSepArg a{Sc,    pm.S,     P.lv[l].child_begin, P.lv[l + 1].octant, pm.pidx,
                 pm.lp, pm.lt,    pm.up_row_ptr,       pm.up_row,          pm.up_tpos,
                 pm.ph_up, pm.nth, pm.nph,             cm.nph,             cm.K,
                 pm.up_rows};
      up_sep_kernel<<<dim3(P.lv[l].B, 6, pm.up_nband), 256, 0, s>>>(a);
    } else {
      UpArg<double2> a{Sc, pm.S, P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx, pm.lp,
                       pm.ph_up, pm.K, pm.nph, cm.K, cm.nph};
      launch_up<double2, false>(up_threads(P), P.lv[l].B, pm.K, 6, a, s);
    }
  }
}

// Translations of levels lo..hi of medium m (independent of each other).
void launch_m2l(Plan& P, int m, const LeafView& v, cudaStream_t s, int lo, int hi) {
  if (lo > hi) return;
  if (P.tuning.m2l_variant >= 6 && P.tuning.m2l_variant <= 8) {
    launch_m2l_grp<double2>(
        P, lo, hi, P.tuning.m2l_variant == 6 ? 2 : 4, P.tuning.m2l_variant == 8,
        [&](int l) { return level_S(P, m, l, v); },
        [&](int l) { return level_B(P, m, l, v); },
        [&](int l) {
          return std::make_tuple(static_cast<const double2*>(P.ml[m][l].tfw), P.ml[m][l].nvec, P.ml[m][l].K);
        },
        s);
    return;
  }
  if (P.tuning.m2l_variant == 4 || P.tuning.m2l_variant == 5) {
    if (hi - lo + 1 > kM2lMaxSeg) throw std::runtime_error("m2l: more levels than one launch takes");
    M2lPairArg<double2> a{};
    int ctas = 0;
    for (int l = lo; l <= hi; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      M2lPairSeg<double2>& g = a.seg[a.nseg++];
      g = M2lPairSeg<double2>{level_S(P, m, l, v), level_B(P, m, l, v), cm.tfw, P.lv[l].pair_ptr, P.lv[l].pair_src,
                              P.lv[l].pair_vec,    P.lv[l].B,           cm.K,   (cm.K + 31) / 32,  ctas};
      const int G = (P.lv[l].B + 1) / 2;
      const int w = P.tuning.m2l_variant == 5 ? kPairWarps : pair_warps(P);
      ctas += ((G + w - 1) / w) * g.nchunk;
    }
    if (P.tuning.m2l_variant == 5)
      m2l_pairh_kernel<double2><<<ctas, 64 * kPairWarps, 0, s>>>(a);
    else
      launch_m2l_pair<double2, false>(pair_warps(P), dim3(ctas), a, s);
    return;
  }
  if (P.tuning.m2l_variant == 3) {
    if (hi - lo + 1 > kM2lMaxSeg) throw std::runtime_error("m2l: more levels than one launch takes");
    M2lWarpArg<double2> a{};
    int ctas = 0;
    for (int l = lo; l <= hi; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      M2lWarpSeg<double2>& g = a.seg[a.nseg++];
      g = M2lWarpSeg<double2>{level_S(P, m, l, v), level_B(P, m, l, v), cm.tfw, P.lv[l].far_ptr, P.lv[l].far_idx,
                     P.lv[l].far_vec, P.lv[l].B, cm.K, (cm.K + 31) / 32, ctas};
      ctas += ((P.lv[l].B + kWarpBoxes - 1) / kWarpBoxes) * g.nchunk;
    }
    m2l_warp_kernel<double2><<<ctas, 32 * kWarpBoxes, 0, s>>>(a);
    return;
  }
  if (P.tuning.m2l_variant == 2) {
    if (hi - lo + 1 > kM2lMaxSeg) throw std::runtime_error("m2l: more levels than one launch takes");
    M2lOctArg a{};
    int ctas = 0;
    for (int l = lo; l <= hi; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      M2lSeg& g = a.seg[a.nseg++];
      g = M2lSeg{level_S(P, m, l, v), level_B(P, m, l, v), cm.tfw, cm.off2vec, P.lv[l].ufar_ptr, P.lv[l].ufar,
                 P.lv[l].upack, P.lv[l - 1].child_begin, P.lv[l].octant, cm.K, (cm.K + kM2lDirs - 1) / kM2lDirs,
                 ctas};
      ctas += P.lv[l - 1].B * g.nchunk;
    }
    m2l_oct_kernel<<<ctas, kM2lThreads, 0, s>>>(a);
    return;
  }
  for (int l = lo; l <= hi; ++l) {
    const MediumLevel& cm = P.ml[m][l];
    if (P.tuning.m2l_variant == 1) {
      M2lTileArg a{level_S(P, m, l, v), level_B(P, m, l, v), P.lv[l - 1].child_begin, P.lv[l].usrc_ptr,
                   P.lv[l].usrc,        P.lv[l].coord,       cm.off2vec,              cm.tfw,
                   cm.K};
      dim3 gd(P.lv[l - 1].B, (cm.K + kTileDirs - 1) / kTileDirs);
      m2l_tile_kernel<<<gd, kTileDirs * kTileWarps, 0, s>>>(a);
    } else {
      M2lArg a{level_S(P, m, l, v), level_B(P, m, l, v), P.lv[l].far_ptr, P.lv[l].far_idx, P.lv[l].far_off,
               cm.off2vec,          cm.tfw,              cm.K};
      dim3 gd(P.lv[l].B, (cm.K + kThreads - 1) / kThreads);
      m2l_kernel<<<gd, kThreads, 0, s>>>(a);
    }
  }
}

// Anterpolation down the tree: level l receives level l-1 once that is final.
void launch_l2l(Plan& P, int m, const LeafView& v, cudaStream_t s) {
  const int L = P.maxL;
  for (int l = 3; l <= L; ++l) {
    const MediumLevel& cm = P.ml[m][l];
    const MediumLevel& pm = P.ml[m][l - 1];
    double2* Bc = level_B(P, m, l, v);
    if (P.tuning.l2l_variant == 1 && 6 * pm.nph <= kL2lBand) {
      L2lSepArg<double2> b{Bc,         pm.Bm,    P.lv[l].parent, P.lv[l].octant, pm.ph_dn, cm.thT_ptr,
                  cm.thT_src, cm.thT_w, cm.phT_ptr,     cm.phT_src,     cm.phT_w, cm.nth,
                  cm.nph,     pm.nth,   pm.nph};
      l2l_sep_kernel<double2><<<dim3(P.lv[l].B, l2l_grid_y(P.lv[l].B, cm.nth, pm.nph)), 256, 0, s>>>(b);
    } else {
      L2lArg b{Bc, pm.Bm, P.lv[l].parent, P.lv[l].octant, pm.ph_dn, cm.tr_ptr, cm.tr_kp, cm.tr_w, cm.K, pm.K};
      dim3 gl(P.lv[l].B, (cm.K + kThreads - 1) / kThreads, 6);
      l2l_kernel<<<gl, kThreads, 0, s>>>(b);
    }
  }
}

template <class Arg>
void fill_leaf_common(const Plan& P, Arg& a) {
  using C = std::remove_reference_t<decltype(a.c1)>;
  a.leaf_rwg = P.d_leaf_rwg;
  a.rwg_box = P.d_rwg_leafbox;
  a.leaf_ptr = P.d_leaf_ptr;
  a.near_sptr = P.d_near_sptr;
  a.near_src = P.d_near_src;
  a.near_zoff = P.d_near_zoff;
  a.near_z = Store<C>::near_z(P);
  a.N = P.N;
  const cplx c1 = P.k1 * P.k1 / (16.0 * kPi * kPi);
  const cplx c2v = P.k2 * P.k2 / (16.0 * kPi * kPi);
  a.c1 = Cx<C>::from(c2(c1.real(), c1.imag()));
  a.c2 = Cx<C>::from(c2(c2v.real(), c2v.imag()));
  a.etai = Cx<C>::from(c2(P.etai.real(), P.etai.imag()));
}

// Medium 1's tree passes go to the plan's second stream, forked from and
// joined back into s; with stage profiling on, both media stay on s so that
// the stage events bracket one medium at a time.
struct MediumStreams {
  Plan& P;
  cudaStream_t s;
  bool two;
  MediumStreams(Plan& P_, cudaStream_t s_, bool concurrent) : P(P_), s(s_), two(concurrent && P_.stream2) {
    if (two) {
      MLFMA_CUDA(cudaEventRecord(P.ev_fork, s));
      MLFMA_CUDA(cudaStreamWaitEvent(P.stream2, P.ev_fork, 0));
    }
  }
  cudaStream_t of(int m) const { return two && m == 1 ? P.stream2 : s; }
  void join() {
    if (two) {
      MLFMA_CUDA(cudaEventRecord(P.ev_join, P.stream2));
      MLFMA_CUDA(cudaStreamWaitEvent(s, P.ev_join, 0));
      two = false;
    }
  }
};

// The near-field rows need only x: with leaf variant 1 they start at the
// beginning of the apply on their own stream (writing w), and the leaf
// kernel adds the far-field testing once they are done.
struct NearAhead {
  Plan& P;
  cudaStream_t s;
  bool on;
  NearAhead(Plan& P_, cudaStream_t s_, bool on_, const double2* x, double2* w, int prec) : P(P_), s(s_), on(on_) {
    if (!on) return;
    MLFMA_CUDA(cudaEventRecord(P.ev_start, s));
    MLFMA_CUDA(cudaStreamWaitEvent(P.stream_near, P.ev_start, 0));
    near_apply(P, x, w, P.stream_near, prec);
    MLFMA_CUDA(cudaEventRecord(P.ev_near, P.stream_near));
  }
  void join() {
    if (on) MLFMA_CUDA(cudaStreamWaitEvent(s, P.ev_near, 0));
  }
};

cudaEvent_t* profiler_events(Plan& P, cudaStream_t s) {
  if (!P.prof.on) return nullptr;
  if (P.prof.used == P.prof.sets.size()) {
    if (P.prof.sets.size() >= 4096) throw std::runtime_error("stage profiler: read it at least every 4096 applies");
    std::array<cudaEvent_t, StageProfiler::kEvents> set{};
    for (auto& e : set) MLFMA_CUDA(cudaEventCreate(&e));
    P.prof.sets.push_back(set);
  }
  cudaEvent_t* ev = P.prof.sets[P.prof.used++].data();
  MLFMA_CUDA(cudaEventRecord(ev[0], s));
  return ev;
}

// The tree passes of medium m with fixed kernel choices (interpolation 0,
// translation 4, anterpolation 1) for either storage type; leafS / leafB are
// the leaf-level arrays (the plan's own or one batch slot). With a leaf
// stream sx, the leaf level's translation runs there after the aggregation
// (ev_agg) while the interpolation climbs the tree on s; s waits for it
// (ev_leaf) before the anterpolation chain.
template <class C>
void tree_pass_fixed(Plan& P, int m, C* leafS, C* leafB, cudaStream_t s, cudaStream_t sx = nullptr,
                     cudaEvent_t ev_agg = nullptr, cudaEvent_t ev_leaf = nullptr) {
  const int L = P.maxL;
  auto S_at = [&](int l) -> C* { return l == L ? leafS : Store<C>::S(P.ml[m][l]); };
  auto B_at = [&](int l) -> C* { return l == L ? leafB : Store<C>::Bm(P.ml[m][l]); };
  auto translate = [&](int lo, int hi, cudaStream_t st) {
    if (lo > hi) return;
    if (P.tuning.m2l_variant >= 6 && P.tuning.m2l_variant <= 8) {
      launch_m2l_grp<C>(
          P, lo, hi, P.tuning.m2l_variant == 6 ? 2 : 4, P.tuning.m2l_variant == 8, S_at, B_at,
          [&](int l) {
            return std::make_tuple(static_cast<const C*>(Store<C>::tfw(P.ml[m][l])), P.ml[m][l].nvec, P.ml[m][l].K);
          },
          st);
      return;
    }
    if (hi - lo + 1 > kM2lMaxSeg) throw std::runtime_error("m2l: more levels than one launch takes");
    M2lPairArg<C> t{};
    int ctas = 0;
    for (int l = lo; l <= hi; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      M2lPairSeg<C>& g = t.seg[t.nseg++];
      g = M2lPairSeg<C>{S_at(l),          B_at(l),   Store<C>::tfw(cm), P.lv[l].pair_ptr, P.lv[l].pair_src,
                        P.lv[l].pair_vec, P.lv[l].B, cm.K,              (cm.K + 31) / 32, ctas};
      ctas += (((P.lv[l].B + 1) / 2 + pair_warps(P) - 1) / pair_warps(P)) * g.nchunk;
    }
    launch_m2l_pair<C, false>(pair_warps(P), dim3(ctas), t, st);
  };
  if (sx) {
    MLFMA_CUDA(cudaEventRecord(ev_agg, s));
    MLFMA_CUDA(cudaStreamWaitEvent(sx, ev_agg, 0));
    translate(L, L, sx);
    MLFMA_CUDA(cudaEventRecord(ev_leaf, sx));
  }
  for (int l = L - 1; l >= 2; --l) {
    const MediumLevel& pm = P.ml[m][l];
    const MediumLevel& cm = P.ml[m][l + 1];
    UpArg<C> a{S_at(l + 1), S_at(l), P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx, pm.lp,
               Store<C>::ph_up(pm), pm.K, pm.nph, cm.K, cm.nph};
    launch_up<C, false>(up_threads(P), P.lv[l].B, pm.K, 6, a, s);
  }
  if (sx) {
    translate(2, L - 1, s);
    MLFMA_CUDA(cudaStreamWaitEvent(s, ev_leaf, 0));
  } else {
    translate(2, L, s);
  }
  for (int l = 3; l <= L; ++l) {
    const MediumLevel& cm = P.ml[m][l];
    const MediumLevel& pm = P.ml[m][l - 1];
    if (6 * pm.nph > kL2lBand) throw std::runtime_error("anterpolation band: phi grid too large for this precision");
    L2lSepArg<C> b{B_at(l),    B_at(l - 1), P.lv[l].parent, P.lv[l].octant, Store<C>::ph_dn(pm), cm.thT_ptr,
                   cm.thT_src, cm.thT_w,    cm.phT_ptr,     cm.phT_src,     cm.phT_w,            cm.nth,
                   cm.nph,     pm.nth,      pm.nph};
    l2l_sep_kernel<C><<<dim3(P.lv[l].B, l2l_grid_y(P.lv[l].B, cm.nth, pm.nph)), 256, 0, s>>>(b);
  }
}

// The tree passes of medium m for rn right-hand-side slots at once (mixed
// plans): every level's interpolation, translation and anterpolation is one
// launch over all slots of the slot-major arrays btS / btB (the slot is a grid
// dimension), with the kernels of tree_pass_fixed. The leaf level's
// translation runs on sx beside the interpolation chain, as there.
void tree_pass_slots(Plan& P, int m, int rn, cudaStream_t s, cudaStream_t sx, cudaEvent_t ev_agg,
                     cudaEvent_t ev_leaf) {
  using C = float2;
  const int L = P.maxL;
  auto stride = [&](int l) { return static_cast<long long>(P.lv[l].B) * 6 * P.ml[m][l].K; };
  auto translate = [&](int lo, int hi, cudaStream_t st) {
    if (lo > hi) return;
    if (hi - lo + 1 > kM2lMaxSeg) throw std::runtime_error("m2l: more levels than one launch takes");
    M2lPairArg<C> t{};
    int ctas = 0;
    for (int l = lo; l <= hi; ++l) {
      const MediumLevel& cm = P.ml[m][l];
      M2lPairSeg<C>& g = t.seg[t.nseg++];
      g = M2lPairSeg<C>{P.btS[m][l],      P.btB[m][l], cm.tfw32,          P.lv[l].pair_ptr, P.lv[l].pair_src,
                        P.lv[l].pair_vec, P.lv[l].B,   cm.K,              (cm.K + 31) / 32, ctas,
                        stride(l),        stride(l)};
      ctas += (((P.lv[l].B + 1) / 2 + pair_warps(P) - 1) / pair_warps(P)) * g.nchunk;
    }
    launch_m2l_pair<C, true>(pair_warps(P), dim3(ctas, rn), t, st);
    MLFMA_CUDA(cudaGetLastError());
  };
  MLFMA_CUDA(cudaEventRecord(ev_agg, s));
  MLFMA_CUDA(cudaStreamWaitEvent(sx, ev_agg, 0));
  translate(L, L, sx);
  MLFMA_CUDA(cudaEventRecord(ev_leaf, sx));
  for (int l = L - 1; l >= 2; --l) {
    const MediumLevel& pm = P.ml[m][l];
    const MediumLevel& cm = P.ml[m][l + 1];
    UpArg<C> a{P.btS[m][l + 1], P.btS[m][l], P.lv[l].child_begin, P.lv[l + 1].octant, pm.tidx, pm.lt, pm.pidx,
               pm.lp,           pm.ph_up32,  pm.K,                 pm.nph,              cm.K,    cm.nph,
               stride(l + 1),   stride(l)};
    launch_up<C, true>(up_threads(P), P.lv[l].B, pm.K, 6 * rn, a, s);
  }
  translate(2, L - 1, s);
  MLFMA_CUDA(cudaStreamWaitEvent(s, ev_leaf, 0));
  for (int l = 3; l <= L; ++l) {
    const MediumLevel& cm = P.ml[m][l];
    const MediumLevel& pm = P.ml[m][l - 1];
    if (6 * pm.nph > kL2lBand) throw std::runtime_error("anterpolation band: phi grid too large for this precision");
    L2lSepArg<C> b{P.btB[m][l], P.btB[m][l - 1], P.lv[l].parent, P.lv[l].octant, pm.ph_dn32, cm.thT_ptr,
                   cm.thT_src,  cm.thT_w,        cm.phT_ptr,     cm.phT_src,     cm.phT_w,   cm.nth,
                   cm.nph,      pm.nth,          pm.nph,         stride(l),      stride(l - 1)};
    l2l_sep_kernel<C, true><<<dim3(P.lv[l].B, l2l_grid_y(P.lv[l].B, cm.nth, pm.nph), rn), 256, 0, s>>>(b);
  }
  MLFMA_CUDA(cudaGetLastError());
}

template <class C>
void apply_fixed(Plan& P, const double2* x, double2* w, cudaStream_t s) {
  const int L = P.maxL;
  LeafArg<C> a{};
  const bool split_near = P.tuning.leaf_variant == 1;
  NearAhead near(P, s, split_near, x, w, std::is_same<C, float2>::value ? 1 : 0);
  MediumStreams ms(P, s, true);
  for (int m = 0; m < 2; ++m) {
    const cudaStream_t sm = ms.of(m);
    const MediumLevel& leaf = P.ml[m][L];
    agg_kernel<C><<<dim3(P.lv[L].B, (leaf.K + kThreads - 1) / kThreads), kThreads, 0, sm>>>(
        Store<C>::Vs(P, m), P.d_leaf_ptr, P.d_leaf_rwg, x, P.N, leaf.K, Store<C>::S(leaf));
    tree_pass_fixed<C>(P, m, Store<C>::S(leaf), Store<C>::Bm(leaf), sm, P.stream_leaf[m], P.ev_agg[m], P.ev_leaf[m]);
    a.Vf[m] = Store<C>::Vf(P, m);
    a.Bm[m] = Store<C>::Bm(leaf);
    a.khat[m] = leaf.khat;
    a.K[m] = leaf.K;
  }
  ms.join();
  fill_leaf_common(P, a);
  a.x = x;
  a.w = w;
  const int warps = kThreads / 32;
  if (split_near) {
    near.join();
    leaf_out_kernel<C, false><<<(P.N + warps - 1) / warps, kThreads, 0, s>>>(a);
  } else {
    leaf_out_kernel<C><<<(P.N + warps - 1) / warps, kThreads, 0, s>>>(a);
  }
  MLFMA_CUDA(cudaGetLastError());
}

template <class C>
void apply_batch_fixed(Plan& P, int R, const double2* X, long long ldx, double2* W, long long ldw, cudaStream_t s) {
  const int L = P.maxL;
  if (std::is_same<C, float2>::value ? P.bS32[0].empty() : P.batch_cap < std::min(R, kBatchSlots))
    throw std::runtime_error("batched apply: slots not reserved");
  constexpr int kAggRB = 8, kLeafRB = 4;
  for (int g0 = 0; g0 < R; g0 += kBatchSlots) {
    const int rn = std::min(kBatchSlots, R - g0);
    AggBatchArg<C> ag{};
    for (int m = 0; m < 2; ++m) {
      ag.Vs[m] = Store<C>::Vs(P, m);
      ag.K[m] = P.ml[m][L].K;
      for (int j = 0; j < rn; ++j) ag.S[m][j] = Store<C>::bS(P, m, j);
    }
    ag.leaf_ptr = P.d_leaf_ptr;
    ag.leaf_rwg = P.d_leaf_rwg;
    ag.X = X + g0 * ldx;
    ag.ldx = ldx;
    ag.N = P.N;
    ag.R = rn;
    bool on_tensor_cores = false;
    if constexpr (std::is_same<C, float2>::value) {
      if (P.tuning.batch_tc == 1 && agg_tc_supported(P, rn)) {
        AggTcArg t{};
        for (int m = 0; m < 2; ++m) {
          t.Vs[m] = reinterpret_cast<const float*>(ag.Vs[m]);
          t.K[m] = ag.K[m];
          for (int j = 0; j < rn; ++j) t.S[m][j] = ag.S[m][j];
        }
        t.leaf_ptr = ag.leaf_ptr;
        t.leaf_rwg = ag.leaf_rwg;
        t.X = ag.X;
        t.ldx = ag.ldx;
        t.N = ag.N;
        t.R = rn;
        t.kmax = (P.max_leaf_rwgs + 7) & ~7;
        t.status = P.d_status;
        launch_agg_tc(P, t, s);
        on_tensor_cores = true;
      }
    }
    if (!on_tensor_cores)
      agg_batch_kernel<C, kAggRB><<<dim3(P.lv[L].B, 2, (rn + kAggRB - 1) / kAggRB), kThreads, 0, s>>>(ag);
    {
      MediumStreams ms(P, s, true);
      if constexpr (std::is_same<C, float2>::value) {
        if (P.tuning.batch_tree == 1) {
          for (int m = 0; m < 2; ++m)
            tree_pass_slots(P, m, rn, ms.of(m), P.stream_leaf[m], P.ev_agg[m], P.ev_leaf[m]);
        } else {
          for (int j = 0; j < rn; ++j)
            for (int m = 0; m < 2; ++m)
              tree_pass_fixed<C>(P, m, Store<C>::bS(P, m, j), Store<C>::bB(P, m, j), ms.of(m));
        }
      } else {
        for (int j = 0; j < rn; ++j)
          for (int m = 0; m < 2; ++m)
            tree_pass_fixed<C>(P, m, Store<C>::bS(P, m, j), Store<C>::bB(P, m, j), ms.of(m));
      }
      ms.join();
    }
    LeafBatchArg<C> lb{};
    for (int m = 0; m < 2; ++m) {
      lb.Vf[m] = Store<C>::Vf(P, m);
      lb.khat[m] = P.ml[m][L].khat;
      lb.K[m] = P.ml[m][L].K;
      for (int j = 0; j < rn; ++j) lb.Bm[m][j] = Store<C>::bB(P, m, j);
    }
    fill_leaf_common(P, lb);
    lb.X = X + g0 * ldx;
    lb.ldx = ldx;
    lb.W = W + g0 * ldw;
    lb.ldw = ldw;
    lb.R = rn;
    const int warps = kThreads / 32;
    const dim3 grid((P.N + warps - 1) / warps, (rn + kLeafRB - 1) / kLeafRB);
    if (on_tensor_cores) {
      // near-field rows first (writing w), then the far field on the tensor cores (adding)
      leaf_out_batch_kernel<C, kLeafRB, false><<<grid, kThreads, 0, s>>>(lb);
      MLFMA_CUDA(cudaGetLastError());
      if constexpr (std::is_same<C, float2>::value) {
        LeafTcArg t{};
        for (int m = 0; m < 2; ++m) {
          t.Vf[m] = lb.Vf[m];
          t.khat[m] = lb.khat[m];
          t.K[m] = lb.K[m];
          for (int j = 0; j < rn; ++j) t.Bm[m][j] = lb.Bm[m][j];
        }
        t.leaf_ptr = P.d_leaf_ptr;
        t.leaf_rwg = P.d_leaf_rwg;
        t.W = lb.W;
        t.ldw = ldw;
        t.c1 = lb.c1;
        t.c2 = lb.c2;
        t.etai = lb.etai;
        t.N = P.N;
        t.R = rn;
        t.status = P.d_status;
        launch_leaf_tc(P, t, s);
      }
    } else {
      leaf_out_batch_kernel<C, kLeafRB><<<grid, kThreads, 0, s>>>(lb);
      MLFMA_CUDA(cudaGetLastError());
    }
  }
}

}  // namespace

void apply_direct(Plan& P, const double2* x, double2* w, cudaStream_t s) {
  const int L = P.maxL;
  cudaEvent_t* ev = profiler_events(P, s);
  const bool split_near = P.tuning.leaf_variant == 1;
  NearAhead near(P, s, split_near && ev == nullptr, x, w, 0);
  if (P.tuning.agg_variant == 1) {  // both media in one launch, timed as medium 1's aggregation
    AggBoxArg a{};
    for (int m = 0; m < 2; ++m) {
      a.Vs[m] = P.d_Vs[m];
      a.S[m] = P.ml[m][L].S;
      a.K[m] = P.ml[m][L].K;
    }
    a.leaf_ptr = P.d_leaf_ptr;
    a.leaf_rwg = P.d_leaf_rwg;
    a.x = x;
    a.N = P.N;
    agg_box_kernel<<<dim3(P.lv[L].B, 2), kThreads, 0, s>>>(a);
  }
  MediumStreams ms(P, s, ev == nullptr);
  for (int m = 0; m < 2; ++m) {
    const cudaStream_t sm = ms.of(m);
    const MediumLevel& leaf = P.ml[m][L];
    if (P.tuning.agg_variant == 0) {
      dim3 g(P.lv[L].B, (leaf.K + kThreads - 1) / kThreads);
      agg_kernel<double2><<<g, kThreads, 0, sm>>>(P.d_Vs[m], P.d_leaf_ptr, P.d_leaf_rwg, x, P.N, leaf.K, leaf.S);
    }
    if (ev) MLFMA_CUDA(cudaEventRecord(ev[1 + 4 * m], s));
    const LeafView v{leaf.S, leaf.Bm};
    if (ev) {  // one stage after the other, for the stage events
      launch_up(P, m, v, s);
      MLFMA_CUDA(cudaEventRecord(ev[2 + 4 * m], s));
      launch_m2l(P, m, v, s, 2, L);
      MLFMA_CUDA(cudaEventRecord(ev[3 + 4 * m], s));
      launch_l2l(P, m, v, s);
      MLFMA_CUDA(cudaEventRecord(ev[4 + 4 * m], s));
      continue;
    }
    // The leaf level's translation needs only the aggregation: it runs on a
    // stream of its own while the interpolation climbs the tree; the
    // anterpolation chain starts once both are done.
    const cudaStream_t sx = P.stream_leaf[m];
    MLFMA_CUDA(cudaEventRecord(P.ev_agg[m], sm));
    MLFMA_CUDA(cudaStreamWaitEvent(sx, P.ev_agg[m], 0));
    launch_m2l(P, m, v, sx, L, L);
    MLFMA_CUDA(cudaEventRecord(P.ev_leaf[m], sx));
    launch_up(P, m, v, sm);
    launch_m2l(P, m, v, sm, 2, L - 1);
    MLFMA_CUDA(cudaStreamWaitEvent(sm, P.ev_leaf[m], 0));
    launch_l2l(P, m, v, sm);
  }
  ms.join();
  LeafArg<double2> a{};
  for (int m = 0; m < 2; ++m) {
    a.Vf[m] = P.d_Vf[m];
    a.Bm[m] = P.ml[m][L].Bm;
    a.khat[m] = P.ml[m][L].khat;
    a.K[m] = P.ml[m][L].K;
  }
  fill_leaf_common(P, a);
  a.x = x;
  a.w = w;
  const int warps = kThreads / 32;
  if (split_near) {
    if (ev) near_apply(P, x, w, s, 0);  // profiled: in sequence, inside the leaf stage
    near.join();
    leaf_out_kernel<double2, false><<<(P.N + warps - 1) / warps, kThreads, 0, s>>>(a);
  } else {
    leaf_out_kernel<double2><<<(P.N + warps - 1) / warps, kThreads, 0, s>>>(a);
  }
  MLFMA_CUDA(cudaGetLastError());
  if (ev) MLFMA_CUDA(cudaEventRecord(ev[9], s));
}

void reserve_batch_staging(Plan& P) {
  if (P.xb_cap > 0) return;
  P.d_xb = P.alloc<double2>(static_cast<size_t>(kBatchSlots) * 2 * P.N);
  P.d_wb = P.alloc<double2>(static_cast<size_t>(kBatchSlots) * 2 * P.N);
  P.xb_cap = kBatchSlots;
}

void reserve_batch(Plan& P, int R, bool fp64) {
  const int want = std::min(R, kBatchSlots);
  const int L = P.maxL;
  if (P.precision == 1 && P.bS32[0].empty()) {
    // the complex64 tree of every slot at once, slot-major per level, in one
    // allocation
    size_t total = 0;
    for (int m = 0; m < 2; ++m)
      for (int l = 2; l <= L; ++l) total += 2 * kBatchSlots * static_cast<size_t>(P.lv[l].B) * 6 * P.ml[m][l].K;
    float2* p = P.alloc<float2>(total);
    for (int m = 0; m < 2; ++m) {
      for (int l = 2; l <= L; ++l) {
        const size_t cnt = static_cast<size_t>(P.lv[l].B) * 6 * P.ml[m][l].K;
        P.btS[m][l] = p;
        P.btB[m][l] = p + kBatchSlots * cnt;
        p += 2 * kBatchSlots * cnt;
      }
      const size_t cnt = static_cast<size_t>(P.lv[L].B) * 6 * P.ml[m][L].K;
      for (int j = 0; j < kBatchSlots; ++j) {
        P.bS32[m].push_back(P.btS[m][L] + j * cnt);
        P.bB32[m].push_back(P.btB[m][L] + j * cnt);
      }
    }
  }
  if (fp64 && P.batch_cap < want) {
    // the FP64 leaf arrays of the slots still missing, in one allocation
    const int add = want - P.batch_cap;
    size_t total = 0;
    for (int m = 0; m < 2; ++m) total += 2 * static_cast<size_t>(add) * P.lv[L].B * 6 * P.ml[m][L].K;
    double2* p = P.alloc<double2>(total);
    for (int m = 0; m < 2; ++m) {
      const size_t cnt = static_cast<size_t>(P.lv[L].B) * 6 * P.ml[m][L].K;
      for (int j = 0; j < add; ++j) {
        P.bS[m].push_back(p);
        P.bB[m].push_back(p + cnt);
        p += 2 * cnt;
      }
    }
    P.batch_cap = want;
  }
}

void apply_batch_device(Plan& P, int R, const double2* X, long long ldx, double2* W, long long ldw, cudaStream_t s) {
  const int L = P.maxL;
  if (P.batch_cap < std::min(R, kBatchSlots)) throw std::runtime_error("batched apply: slots not reserved");
  constexpr int kAggRB = 8, kLeafRB = 4;
  for (int g0 = 0; g0 < R; g0 += kBatchSlots) {
    const int rn = std::min(kBatchSlots, R - g0);
    AggBatchArg<double2> ag{};
    for (int m = 0; m < 2; ++m) {
      ag.Vs[m] = P.d_Vs[m];
      ag.K[m] = P.ml[m][L].K;
      for (int j = 0; j < rn; ++j) ag.S[m][j] = P.bS[m][j];
    }
    ag.leaf_ptr = P.d_leaf_ptr;
    ag.leaf_rwg = P.d_leaf_rwg;
    ag.X = X + g0 * ldx;
    ag.ldx = ldx;
    ag.N = P.N;
    ag.R = rn;
    agg_batch_kernel<double2, kAggRB><<<dim3(P.lv[L].B, 2, (rn + kAggRB - 1) / kAggRB), kThreads, 0, s>>>(ag);
    {
      MediumStreams ms(P, s, true);
      for (int j = 0; j < rn; ++j)
        for (int m = 0; m < 2; ++m) {
          const LeafView v{P.bS[m][j], P.bB[m][j]};
          launch_up(P, m, v, ms.of(m));
          launch_m2l(P, m, v, ms.of(m), 2, P.maxL);
          launch_l2l(P, m, v, ms.of(m));
        }
      ms.join();
    }
    LeafBatchArg<double2> lb{};
    for (int m = 0; m < 2; ++m) {
      lb.Vf[m] = P.d_Vf[m];
      lb.khat[m] = P.ml[m][L].khat;
      lb.K[m] = P.ml[m][L].K;
      for (int j = 0; j < rn; ++j) lb.Bm[m][j] = P.bB[m][j];
    }
    fill_leaf_common(P, lb);
    lb.X = X + g0 * ldx;
    lb.ldx = ldx;
    lb.W = W + g0 * ldw;
    lb.ldw = ldw;
    lb.R = rn;
    const int warps = kThreads / 32;
    leaf_out_batch_kernel<double2, kLeafRB><<<dim3((P.N + warps - 1) / warps, (rn + kLeafRB - 1) / kLeafRB), kThreads, 0, s>>>(lb);
    MLFMA_CUDA(cudaGetLastError());
  }
}

// Replays the captured apply of (stream, precision), capturing it on first
// use. The graph reads and writes the plan's staging vectors d_gx / d_gw, so
// that one graph serves every (x, w) pair: x is copied in and w out around
// the replay (two device copies of 2N complex values, microseconds against
// the apply), and a solver whose Krylov vectors change every iteration does
// not capture a graph per vector. Launches directly while stage profiling,
// inside another capture, or on the legacy default stream.
template <class F>
void apply_graphed(Plan& P, const double2* x, double2* w, cudaStream_t s, int precision, F&& launch) {
  if (!P.tuning.graph || P.prof.on || s == nullptr) return launch(x, w);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  MLFMA_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) return launch(x, w);
  const size_t bytes = 2 * static_cast<size_t>(P.N) * sizeof(double2);
  if (P.d_gx == nullptr) {
    P.d_gx = P.alloc<double2>(2 * static_cast<size_t>(P.N));
    P.d_gw = P.alloc<double2>(2 * static_cast<size_t>(P.N));
  }
  cudaGraphExec_t exec = nullptr;
  for (const ApplyGraph& g : P.graphs)
    if (g.s == s && g.precision == precision) exec = g.exec;
  if (exec == nullptr && P.graphs.size() >= kMaxApplyGraphs) return launch(x, w);
  if (x != P.d_gx) MLFMA_CUDA(cudaMemcpyAsync(P.d_gx, x, bytes, cudaMemcpyDeviceToDevice, s));
  if (exec == nullptr) {
    MLFMA_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      launch(P.d_gx, P.d_gw);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t graph = nullptr;
    MLFMA_CUDA(cudaStreamEndCapture(s, &graph));
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    MLFMA_CUDA(e);
    P.graphs.push_back(ApplyGraph{s, precision, exec});
  }
  MLFMA_CUDA(cudaGraphLaunch(exec, s));
  if (w != P.d_gw) MLFMA_CUDA(cudaMemcpyAsync(w, P.d_gw, bytes, cudaMemcpyDeviceToDevice, s));
}

void apply_device(Plan& P, const double2* x, double2* w, cudaStream_t s) {
  apply_graphed(P, x, w, s, 0, [&](const double2* xx, double2* ww) { apply_direct(P, xx, ww, s); });
}

void clear_graphs(Plan& P) {
  for (auto& g : P.graphs) cudaGraphExecDestroy(g.exec);
  P.graphs.clear();
}

void apply_mixed_device(Plan& P, const double2* x, double2* w, cudaStream_t s) {
  if (P.precision != 1) throw std::invalid_argument("plan was not created with mixed precision");
  apply_graphed(P, x, w, s, 1, [&](const double2* xx, double2* ww) { apply_fixed<float2>(P, xx, ww, s); });
}

void apply_batch_mixed_device(Plan& P, int R, const double2* X, long long ldx, double2* W, long long ldw,
                              cudaStream_t s) {
  if (P.precision != 1) throw std::invalid_argument("plan was not created with mixed precision");
  apply_batch_fixed<float2>(P, R, X, ldx, W, ldw, s);
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
