// Batched leaf aggregation on the 5th-generation tensor cores (tcgen05), for
// the complex64 (mixed-precision) operator.
//
// For leaf box b and medium m the batched aggregation (Code/ProcessMLFMM.h:
// 33-56, applied to R right-hand sides at once) is a complex GEMM
//     S_b[part][e][j] = sum_{r in b} Vs[r][e] * x_j[part * N + id(r)],
// e over the 3K pattern entries, part J (0) or M (1), j over the R slots.
// It runs as one real GEMM per (box, medium): the A operand is Vs^T seen as
// real rows (re and im of each entry as two rows, M = 6K in tiles of 128), the
// B operand holds the box's currents as real columns (re and im of each
// (part, j), N = 4R <= 64), and the contraction runs over the box's RWGs
// (K = n_b, padded to 8). Complex products come out of the epilogue:
//     re = D[re row][re col] - D[im row][im col],
//     im = D[re row][im col] + D[im row][re col],
// the two rows sitting in neighbouring TMEM lanes (one shuffle).
//
// Precision: the operands are split into TF32 high and low parts
// (a = a_hi + a_lo) and D accumulates a_hi b_hi + a_hi b_lo + a_lo b_hi in
// FP32, which carries the FP32 operands' precision (the dropped a_lo b_lo is
// below 2^-21 relative).
//
// Mechanics (cta_group::1): warp 0 allocates 64 TMEM columns; all threads
// write both operands into shared memory in the no-swizzle K-major canonical
// layout (8-row x 16-byte core matrices; SBO = 128 B between 8-row groups,
// LBO between the two 4-element K halves); one thread issues the MMAs of a
// tile (3 per 8 RWGs) and commits them to an mbarrier; the epilogue reads
// TMEM with tcgen05.ld (warp w owns lanes 32w..32w+31). Every wait is bounded.
#include <cuda.h>

#include <cstdint>
#include <stdexcept>

#include "agg_tc.hpp"
#include "bulk.cuh"
#include "cplx.cuh"
#include "plan.hpp"

namespace mlfma {

namespace {

constexpr int kTcRows = 128;  // M per MMA (real rows)
constexpr int kTcCols = 64;   // N per MMA = TMEM columns (4 R real columns, R <= 16)

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Byte offset of element (row, k) of a K-major operand with `rows` rows in
// the no-swizzle canonical layout: per 8 K-elements a slab of rows x 32 B;
// inside it the first 4 K-elements of every row, then the second 4 (LBO =
// rows x 16 B); 8-row core matrices of 128 B each (SBO = 128 B).
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int rows) {
  return static_cast<uint32_t>((k >> 3) * (rows * 32) + ((k >> 2) & 1) * (rows * 16) + (row >> 3) * 128 +
                               (row & 7) * 16 + (k & 3) * 4);
}

// Shared-memory matrix descriptor (sm_100): start address, LBO, SBO (all in
// 16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(128, 1) agg_tc_kernel(const __grid_constant__ AggTcArg a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int b = blockIdx.x, m = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int K3 = 3 * a.K[m], M6 = 6 * a.K[m];
  const int r0 = a.leaf_ptr[b], nb = a.leaf_ptr[b + 1] - r0;
  const int kp = (nb + 7) & ~7;  // <= a.kmax (checked on the host)
  const int R = a.R;
  uint32_t* Ahi = reinterpret_cast<uint32_t*>(smem);
  uint32_t* Alo = Ahi + kTcRows * a.kmax;
  uint32_t* Bhi = Alo + kTcRows * a.kmax;
  uint32_t* Blo = Bhi + kTcCols * a.kmax;
  uint64_t* bar = reinterpret_cast<uint64_t*>(Blo + kTcCols * a.kmax);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  int* sid = reinterpret_cast<int*>(tslot + 2);  // RWG ids of the box, [kmax]

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init_fence();
  }
  for (int k = tid; k < nb; k += blockDim.x) sid[k] = a.leaf_rwg[r0 + k];
  __syncthreads();
  // B: the box's currents, real column n = 2 * col + (0 re, 1 im) with
  // col = part * R + j; one complex current per (k, col) and thread
#pragma unroll 4
  for (int i = tid; i < (kTcCols / 2) * kp; i += blockDim.x) {
    const int col = i % (kTcCols / 2), k = i / (kTcCols / 2);
    float vr = 0.f, vi = 0.f;
    if (k < nb && col < 2 * R) {
      const int part = col / R, j = col - part * R;
      const double2 x = a.X[j * a.ldx + part * a.N + sid[k]];
      vr = static_cast<float>(x.x);
      vi = static_cast<float>(x.y);
    }
    const uint32_t hr = tf32_rna(vr), hi = tf32_rna(vi);
    const uint32_t o = kmajor_offset(2 * col, k, kTcCols) >> 2, o1 = kmajor_offset(2 * col + 1, k, kTcCols) >> 2;
    Bhi[o] = hr;
    Blo[o] = tf32_rna(vr - __uint_as_float(hr));
    Bhi[o1] = hi;
    Blo[o1] = tf32_rna(vi - __uint_as_float(hi));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_tf32(kTcRows, kTcCols);
  const float* V = a.Vs[m] + static_cast<size_t>(r0) * M6;  // the box's pattern rows, real view
  float2* const* S = a.S[m];
  uint32_t phase = 0;
  bool ok = true;
  for (int mt = 0; mt * kTcRows < M6 && ok; ++mt) {
    const int q = mt * kTcRows + tid;  // this thread's real row (A row, TMEM lane)
    for (int k0 = 0; k0 < kp; k0 += 8) {  // 8 loads in flight per thread
      float v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = k0 + u;
        v[u] = (k < nb && q < M6) ? __ldg(V + static_cast<size_t>(k) * M6 + q) : 0.f;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const uint32_t hi = tf32_rna(v[u]), lo = tf32_rna(v[u] - __uint_as_float(hi));
        const uint32_t o = kmajor_offset(tid, k0 + u, kTcRows) >> 2;
        Ahi[o] = hi;
        Alo[o] = lo;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic smem writes -> tensor-core reads
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      if (kp > 0) {
        for (int ks = 0; ks < kp / 8; ++ks) {
          const uint64_t ah = smem_desc(smem_addr(Ahi) + ks * kTcRows * 32, kTcRows * 16, 128);
          const uint64_t al = smem_desc(smem_addr(Alo) + ks * kTcRows * 32, kTcRows * 16, 128);
          const uint64_t bh = smem_desc(smem_addr(Bhi) + ks * kTcCols * 32, kTcCols * 16, 128);
          const uint64_t bl = smem_desc(smem_addr(Blo) + ks * kTcCols * 32, kTcCols * 16, 128);
          mma_tf32(tmem, ah, bh, idesc, ks > 0 ? 1u : 0u);
          mma_tf32(tmem, ah, bl, idesc, 1u);
          mma_tf32(tmem, al, bh, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(bar))
                     : "memory");
      } else {
        mbar_arrive(bar);  // a box without RWGs: nothing to wait for, the tile is zero
      }
    }
    // one verdict for the whole CTA: the TMEM loads below are warp-collective
    // and the loop's barriers must be reached by every thread
    ok = __syncthreads_and(mbar_wait(bar, phase, a.status, false, kStatusAggTc)) != 0;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      float d[kTcCols];
      if (kp > 0) {
        const uint32_t base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll
        for (int c = 0; c < kTcCols / 16; ++c) tmem_ld16(base + 16 * c, d + 16 * c);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int c = 0; c < kTcCols; ++c) d[c] = 0.f;
      }
      const int e = q >> 1;
      const bool re_row = (q & 1) == 0;
#pragma unroll
      for (int col = 0; col < kTcCols / 2; ++col) {
        const float dr = d[2 * col], di = d[2 * col + 1];
        const float pr = __shfl_xor_sync(0xffffffffu, dr, 1), pi = __shfl_xor_sync(0xffffffffu, di, 1);
        if (col < 2 * R && re_row && e < K3) {
          const int part = col / R, j = col - part * R;
          S[j][static_cast<size_t>(b) * 2 * K3 + part * K3 + e] = make_float2(dr - pi, di + pr);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM read and shared operands free before the next tile
  }
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
  }
}

// Far-field testing (see LeafTcArg). One real GEMM per (box, 32-RWG tile,
// medium): A rows 32 t + rr for RWG rr, t = 0 / 1 the real / imaginary row of
// Vf and t = 2 / 3 those of W = (-khat) x Vf, over real K = 2 x 3K (entry e
// gives columns 2e (re) and 2e + 1 (im)): a real row holds (a_re, -a_im), an
// imaginary row (a_im, a_re), so that D[real row] and D[imaginary row] are
// the real and imaginary parts of sum_e a_e b_e. B: column part * 16 + j is
// Bm_j of the box (part 0 the J half, 1 the M half), whose interleaved
// complex layout already is the real K order. The contraction runs over
// chunks of 4 directions (their 3 x 4 entries, 24 real K; a thread builds one
// RWG's Vf and W at one direction from one set of loads) through two
// shared-memory stages: the MMAs of one stage run while the threads fill the
// other.
constexpr int kLfRows = 128;      // 32 RWGs x 4 rows
constexpr int kLfCols = 32;       // 2 parts x 16 slots
constexpr int kLfDirs = 4;        // directions per stage: 3 x 4 complex entries (24 real K)
constexpr int kLfChunk = 3 * kLfDirs;
constexpr int kLfStageA = kLfRows * 2 * kLfChunk;  // tf32 values per A operand stage
constexpr int kLfStageB = kLfCols * 2 * kLfChunk;

__global__ void __launch_bounds__(128, 1) leaf_tc_kernel(const __grid_constant__ LeafTcArg a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int b = blockIdx.x, tile = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int rb0 = a.leaf_ptr[b], nb = a.leaf_ptr[b + 1] - rb0;
  const int rt0 = tile * 32;
  if (rt0 >= nb) return;
  const int nt = min(32, nb - rt0);  // RWGs of this tile
  // stage s: A high, A low, B high, B low
  uint32_t* const stage0 = reinterpret_cast<uint32_t*>(smem);
  constexpr int kStage = 2 * (kLfStageA + kLfStageB);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * 2 * (kLfStageA + kLfStageB) * sizeof(uint32_t));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(2 * kLfCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
    mbar_init_fence();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = idesc_tf32(kLfRows, kLfCols);
  const int R = a.R;
  const int t = tid & 3;  // epilogue: slots j = 4 q + t of RWG tid / 4
  float2 wj[4], wm[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) wj[q] = wm[q] = make_float2(0.f, 0.f);
  // Each chunk's MMAs start a fresh accumulator (TMEM columns 32 x stage);
  // its 32 columns are added into dacc (FP32, round to nearest) when the
  // stage comes round again or the medium ends, so that the tensor cores
  // never accumulate more than one chunk (12 MMAs) in place.
  const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
  float dacc[kLfCols];
  auto drain = [&](int stage) {
    float d[kLfCols];
    tmem_ld16(lane_base + stage * kLfCols, d);
    tmem_ld16(lane_base + stage * kLfCols + 16, d + 16);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int n = 0; n < kLfCols; ++n) dacc[n] += d[n];
  };
  int gc = 0;  // chunks issued so far (both media): stage gc & 1
  bool ok = true;
  for (int m = 0; m < 2 && ok; ++m) {
    const int K = a.K[m], K3 = 3 * K;
#pragma unroll
    for (int n = 0; n < kLfCols; ++n) dacc[n] = 0.f;
    const float2* V = a.Vf[m] + static_cast<size_t>(rb0 + rt0) * K3;
    const double* kh = a.khat[m];
    const int nchunk = (K + kLfDirs - 1) / kLfDirs;
    for (int c = 0; c < nchunk && ok; ++c, ++gc) {
      const int st = gc & 1;
      uint32_t* const Ah = stage0 + st * kStage;
      uint32_t* const Al = Ah + kLfStageA;
      uint32_t* const Bh = Ah + 2 * kLfStageA;
      uint32_t* const Bl = Bh + kLfStageB;
      if (gc >= 2)  // the stage's previous MMAs (chunk gc - 2) are done
        ok = __syncthreads_and(mbar_wait(bar + st, ((gc - 2) >> 1) & 1, a.status, false, kStatusLeafTc)) !=
             0;
      if (!ok) break;
      if (c >= 2) {  // chunk c - 2 of this medium is in the stage's accumulator
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        drain(st);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
      // stage entries: (component cc, direction k0 + kk) at complex index cc * kLfDirs + kk
      const int k0 = c * kLfDirs;
      {  // A: one (RWG, direction) per thread: the 3 components of Vf and of W = (-khat) x Vf
        const int ri = tid & 31, kk = tid >> 5, k = k0 + kk;
        float2 v[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        float2 w[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
        if (ri < nt && k < K) {
          const float2* vr = V + static_cast<size_t>(ri) * K3 + k;
          v[0] = __ldg(vr);
          v[1] = __ldg(vr + K);
          v[2] = __ldg(vr + 2 * K);
          const float ax = static_cast<float>(-__ldg(kh + k)), ay = static_cast<float>(-__ldg(kh + K + k)),
                      az = static_cast<float>(-__ldg(kh + 2 * K + k));
          w[0] = make_float2(v[2].x * ay - v[1].x * az, v[2].y * ay - v[1].y * az);
          w[1] = make_float2(v[0].x * az - v[2].x * ax, v[0].y * az - v[2].y * ax);
          w[2] = make_float2(v[1].x * ax - v[0].x * ay, v[1].y * ax - v[0].y * ay);
        }
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int ep = cc * kLfDirs + kk;
          const float val[4][2] = {{v[cc].x, -v[cc].y}, {v[cc].y, v[cc].x}, {w[cc].x, -w[cc].y}, {w[cc].y, w[cc].x}};
#pragma unroll
          for (int tt = 0; tt < 4; ++tt) {
            // row tt * 32 + ri: the 8 rows of a core matrix come from 8 neighbouring lanes
            const uint32_t h0 = tf32_rna(val[tt][0]), h1 = tf32_rna(val[tt][1]);
            const uint32_t l0 = tf32_rna(val[tt][0] - __uint_as_float(h0)), l1 = tf32_rna(val[tt][1] - __uint_as_float(h1));
            const uint32_t o = kmajor_offset(tt * 32 + ri, 2 * ep, kLfRows) >> 2;  // 8-byte aligned pair
            *reinterpret_cast<uint2*>(Ah + o) = make_uint2(h0, h1);
            *reinterpret_cast<uint2*>(Al + o) = make_uint2(l0, l1);
          }
        }
      }
      // B: 32 columns x 12 entries, 3 per thread
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const int q = tid + 128 * i;  // < 384
        const int ep = q % kLfChunk, col = q / kLfChunk;
        const int cc = ep / kLfDirs, k = k0 + (ep - cc * kLfDirs);
        const int part = col >> 4, j = col & 15;
        float2 v = make_float2(0.f, 0.f);
        if (j < R && k < K) v = __ldg(a.Bm[m][j] + static_cast<size_t>(b) * 2 * K3 + part * K3 + cc * K + k);
        const uint32_t hr = tf32_rna(v.x), hi = tf32_rna(v.y);
        const uint32_t o = kmajor_offset(col, 2 * ep, kLfCols) >> 2;  // 8-byte aligned pair
        *reinterpret_cast<uint2*>(Bh + o) = make_uint2(hr, hi);
        *reinterpret_cast<uint2*>(Bl + o) =
            make_uint2(tf32_rna(v.x - __uint_as_float(hr)), tf32_rna(v.y - __uint_as_float(hi)));
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
#pragma unroll
        for (int ks = 0; ks < 2 * kLfChunk / 8; ++ks) {
          const uint64_t ah = smem_desc(smem_addr(Ah) + ks * kLfRows * 32, kLfRows * 16, 128);
          const uint64_t al = smem_desc(smem_addr(Al) + ks * kLfRows * 32, kLfRows * 16, 128);
          const uint64_t bh = smem_desc(smem_addr(Bh) + ks * kLfCols * 32, kLfCols * 16, 128);
          const uint64_t bl = smem_desc(smem_addr(Bl) + ks * kLfCols * 32, kLfCols * 16, 128);
          const uint32_t acc = tmem + st * kLfCols;
          mma_tf32(acc, ah, bh, idesc, ks > 0 ? 1u : 0u);
          mma_tf32(acc, ah, bl, idesc, 1u);
          mma_tf32(acc, al, bh, idesc, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(bar + st))
                     : "memory");
      }
    }
    if (!ok) break;
    // the medium's last (up to) two chunks: their accumulators
    ok = __syncthreads_and(
             mbar_wait(bar + ((gc - 1) & 1), ((gc - 1) >> 1) & 1, a.status, false, kStatusLeafTc)) != 0;
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (nchunk >= 2) drain((gc - 2) & 1);
    drain((gc - 1) & 1);
    // warp tt holds row kind tt of all 32 RWGs (lane = RWG): regroup per RWG
    // through shared memory (the stages are idle), E[column][row]
    float* E = reinterpret_cast<float*>(stage0);
#pragma unroll
    for (int n = 0; n < kLfCols; ++n) E[n * kLfRows + tid] = dacc[n];
    __syncthreads();
    const int er = tid >> 2;  // RWG of this thread's outputs
    float2 LJ[4], KJ[4], LM[4], KM[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = 4 * q + t;
      LJ[q] = make_float2(E[j * kLfRows + er], E[j * kLfRows + 32 + er]);
      KJ[q] = make_float2(E[j * kLfRows + 64 + er], E[j * kLfRows + 96 + er]);
      LM[q] = make_float2(E[(16 + j) * kLfRows + er], E[(16 + j) * kLfRows + 32 + er]);
      KM[q] = make_float2(E[(16 + j) * kLfRows + 64 + er], E[(16 + j) * kLfRows + 96 + er]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (m == 0) {
        wj[q] = cmul(a.c1, csub(LJ[q], KM[q]));
        wm[q] = cmul(a.c1, cadd(KJ[q], LM[q]));
      } else {
        wj[q] = cadd(wj[q], cmul(a.c2, csub(cmul(a.etai, LJ[q]), KM[q])));
        wm[q] = cadd(wm[q], cmul(a.c2, cadd(KJ[q], cdiv(LM[q], a.etai))));
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // every warp has read TMEM before the next medium's MMAs overwrite it
  }
  if (ok) {
    const int ri = tid >> 2;
    if (ri < nt) {
      const int id = a.leaf_rwg[rb0 + rt0 + ri];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = 4 * q + t;
        if (j < R) {
          double2* w = a.W + j * a.ldw;
          w[id] = cadd(w[id], c2(static_cast<double>(wj[q].x), static_cast<double>(wj[q].y)));
          w[a.N + id] = cadd(w[a.N + id], c2(static_cast<double>(wm[q].x), static_cast<double>(wm[q].y)));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kLfCols)
                 : "memory");
  }
}

}  // namespace

size_t agg_tc_smem_bytes(int kmax) {
  return static_cast<size_t>(kTcRows + kTcCols) * kmax * 2 * sizeof(uint32_t) + 2 * sizeof(uint64_t) +
         static_cast<size_t>(kmax) * sizeof(int);
}

void launch_leaf_tc(const Plan& P, const LeafTcArg& a, cudaStream_t s) {
  if (a.R < 1 || a.R > 16) throw std::invalid_argument("tensor-core far-field testing: 1 <= R <= 16");
  const size_t smem = 2 * 2 * (kLfStageA + kLfStageB) * sizeof(uint32_t) + 4 * sizeof(uint64_t);
  MLFMA_CUDA(
      cudaFuncSetAttribute(leaf_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  const int tiles = (P.max_leaf_rwgs + 31) / 32;
  leaf_tc_kernel<<<dim3(P.lv[P.maxL].B, tiles), 128, smem, s>>>(a);
  MLFMA_CUDA(cudaGetLastError());
}

bool agg_tc_supported(const Plan& P, int R) {
  return P.precision == 1 && R >= 1 && 4 * R <= kTcCols && P.max_leaf_rwgs >= 1 && P.max_leaf_rwgs <= kAggTcMaxRwgs;
}

void launch_agg_tc(const Plan& P, const AggTcArg& a, cudaStream_t s) {
  if (a.R < 1 || 4 * a.R > kTcCols) throw std::invalid_argument("tensor-core aggregation: 1 <= R <= 16");
  if (a.kmax % 8 != 0 || a.kmax < 8 || a.kmax > kAggTcMaxRwgs)
    throw std::invalid_argument("tensor-core aggregation: leaf boxes hold too many RWGs");
  const size_t smem = agg_tc_smem_bytes(a.kmax);
  // the limit is the largest any plan uses, the same value on every call: plans
  // launched from several host threads then never lower it under another's launch
  MLFMA_CUDA(cudaFuncSetAttribute(agg_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(agg_tc_smem_bytes(kAggTcMaxRwgs))));
  agg_tc_kernel<<<dim3(P.lv[P.maxL].B, 2), 128, smem, s>>>(a);
  MLFMA_CUDA(cudaGetLastError());
}

}  // namespace mlfma
