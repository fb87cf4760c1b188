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
constexpr uint32_t idesc_tf32(int M, int N) {
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
  // B: the box's currents, real column n = 2 * (part * R + j) + (0 re, 1 im)
  for (int i = tid; i < kTcCols * kp; i += blockDim.x) {
    const int n = i % kTcCols, k = i / kTcCols;
    float v = 0.f;
    if (k < nb && n < 4 * R) {
      const int col = n >> 1, part = col / R, j = col - part * R;
      const double2 x = a.X[j * a.ldx + part * a.N + a.leaf_rwg[r0 + k]];
      v = static_cast<float>((n & 1) ? x.y : x.x);
    }
    const uint32_t hi = tf32_rna(v), lo = tf32_rna(v - __uint_as_float(hi));
    const uint32_t o = kmajor_offset(n, k, kTcCols) >> 2;
    Bhi[o] = hi;
    Blo[o] = lo;
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
    for (int k = 0; k < kp; ++k) {
      const float v = (k < nb && q < M6) ? __ldg(V + static_cast<size_t>(k) * M6 + q) : 0.f;
      const uint32_t hi = tf32_rna(v), lo = tf32_rna(v - __uint_as_float(hi));
      const uint32_t o = kmajor_offset(tid, k, kTcRows) >> 2;
      Ahi[o] = hi;
      Alo[o] = lo;
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
    ok = __syncthreads_and(mbar_wait(bar, phase, a.status)) != 0;
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

}  // namespace

size_t agg_tc_smem_bytes(int kmax) {
  return static_cast<size_t>(kTcRows + kTcCols) * kmax * 2 * sizeof(uint32_t) + 2 * sizeof(uint64_t);
}

bool agg_tc_supported(const Plan& P, int R) {
  return P.precision == 1 && R >= 1 && 4 * R <= kTcCols && P.max_leaf_rwgs >= 1 && P.max_leaf_rwgs <= kAggTcMaxRwgs;
}

void launch_agg_tc(const Plan& P, const AggTcArg& a, cudaStream_t s) {
  if (a.R < 1 || 4 * a.R > kTcCols) throw std::invalid_argument("tensor-core aggregation: 1 <= R <= 16");
  if (a.kmax % 8 != 0 || a.kmax < 8 || a.kmax > kAggTcMaxRwgs)
    throw std::invalid_argument("tensor-core aggregation: leaf boxes hold too many RWGs");
  const size_t smem = agg_tc_smem_bytes(a.kmax);
  MLFMA_CUDA(
      cudaFuncSetAttribute(agg_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  agg_tc_kernel<<<dim3(P.lv[P.maxL].B, 2), 128, smem, s>>>(a);
  MLFMA_CUDA(cudaGetLastError());
}

}  // namespace mlfma
