// Device-resident PMCHWT MLFMA operator ("plan") and the kernels that build
// and apply it. Layout in HBM (per medium m = k1 | k2, per level l):
//   S_m,l / B_m,l : [box][6][K_m,l] complex128 (J x,y,z then M x,y,z),
//                   boxes in Morton order; K directions theta-major.
//   radiation / receive leaf patterns: [rwg in leaf order][3][K_m,leaf].
//   transfer factors: [vec][K] complex128 with the quadrature weight folded in.
//   near field: per leaf box b, a dense block [n_b targets][sources of the
//               27-neighbourhood][3] complex128 (z11, z12, z22; z21 = -z12).
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "host.hpp"

namespace mlfma {

// Separable interpolation bands: outputs per band (4 per thread of a
// 256-thread CTA) and the staged child-row entries a band may hold (40 KiB).
constexpr int kUpBandOut = 1024;
constexpr int kUpBandEntries = 2560;
// Register-separable interpolation: parent theta rows per band, and the most
// child rows a band may need.
constexpr int kUpColBand = 4;
constexpr int kUpColRows = 8;

struct MediumLevel {
  int L = 0, nth = 0, nph = 0, K = 0;
  double2* S = nullptr;
  double2* Bm = nullptr;
  double2* tfw = nullptr;      // [nvec][K], weights folded in
  // complex64 copies for the mixed-precision operator (precision = mixed only)
  float2 *S32 = nullptr, *Bm32 = nullptr, *tfw32 = nullptr, *ph_up32 = nullptr, *ph_dn32 = nullptr;
  int nvec = 0;
  int* off2vec = nullptr;      // [343] -> vec index or -1
  double* khat = nullptr;      // [3][K] (x row, y row, z row)
  // this level as parent of level+1
  int* tidx = nullptr;         // [nth][3] into the child theta grid
  double* lt = nullptr;        // [nth][3]
  int* pidx = nullptr;         // [nph][3] into the child phi grid
  double* lp = nullptr;        // [nph][3]
  double2* ph_up = nullptr;    // [8][K]: exp(-j k khat.(c_parent - c_child)), child octant o
  double2* ph_dn = nullptr;    // [8][K]: exp(-j k khat.(c_child - c_parent))
  // separable interpolation in bands of up_rows theta rows of this grid:
  // band i needs the child theta rows up_row[up_row_ptr[i] .. up_row_ptr[i+1])
  // and parent row t's tap i reads band row up_tpos[3 t + i]
  int up_rows = 0, up_nband = 0, up_band_max = 0;
  int* up_row_ptr = nullptr;
  int* up_row = nullptr;
  int* up_tpos = nullptr;
  // the same for bands of kUpColBand rows (register-separable interpolation);
  // up4_row_ptr is null when a band would need more than kUpColRows child rows
  int up4_nband = 0;
  int* up4_row_ptr = nullptr;
  int* up4_row = nullptr;
  int* up4_tpos = nullptr;
  // this level as child of level-1: for each child direction, the parent
  // directions that interpolate onto it and the Lagrange weight
  int* tr_ptr = nullptr;       // [K+1]
  int* tr_kp = nullptr;
  double* tr_w = nullptr;
  // the same, separable: child theta row -> (parent theta row, weight),
  // child phi column -> (parent phi column, weight)
  int* thT_ptr = nullptr;
  int* thT_src = nullptr;
  double* thT_w = nullptr;
  int* phT_ptr = nullptr;
  int* phT_src = nullptr;
  double* phT_w = nullptr;
  // host copies
  Grid grid;
  Interp interp;               // this level from level+1 (levels 2..maxL-1)
  std::vector<int> vec_off;    // encoded offset of each vec
};

struct DevLevel {
  int B = 0;
  int* child_begin = nullptr;  // [B+1] into level+1
  int* parent = nullptr;       // [B]
  int* octant = nullptr;       // [B] position in the parent cube
  int* far_ptr = nullptr;      // [B+1]
  int* far_idx = nullptr;
  int* far_off = nullptr;
  int* far_vec = nullptr;      // transfer-factor row of each interaction-list entry
  // boxes in pairs (2g, 2g+1): the merged, source-ordered interaction lists of
  // each pair with the transfer-factor row of either member (-1: not in its list)
  int* pair_ptr = nullptr;     // [ceil(B/2) + 1]
  int* pair_src = nullptr;
  int2* pair_vec = nullptr;
  // boxes in groups of 8 (8q .. 8q+7): the merged, source-ordered union of
  // the group's interaction lists; per entry the transfer-factor row of each
  // member as 16-bit fields (member j in word j/2, bits 16*(j%2); -1: not
  // in its list)
  int* grp_ptr = nullptr;      // [ceil(B/8) + 1]
  int* grp_src = nullptr;
  int4* grp_code = nullptr;
  long long far_pairs = 0;
  int* coord = nullptr;        // [3 * B] integer box coordinates
  int* usrc_ptr = nullptr;     // per parent box (level - 1): union of its children's
  int* usrc = nullptr;         //   interaction sources at this level (ascending)
  // Per parent box (level - 1): the union of its children's interaction-list
  // sources, each with pack = enc(2 * parent - source) | (octant mask << 9);
  // bit o of the mask is set when the child in octant o has the source in
  // its interaction list. The child's offset code is enc + octant_offset(o).
  int* ufar_ptr = nullptr;
  int* ufar = nullptr;
  int* upack = nullptr;
};

// Kernel choices a plan can be tuned with (mlfma_set_tuning).
struct Tuning {
  int m2l_variant = 4;         // 0: one thread per (box, direction); 1: sibling-group tiles;
                               // 2: octant registers over the sibling union, all levels per launch;
                               // 3: warp per box, 8 Morton-consecutive boxes per CTA, all levels per launch;
                               // 4: warp per box pair (merged lists), 4 pairs per CTA, all levels per launch;
                               // 5: as 4 with the J and M halves on separate warps;
                               // 6: groups of 8 boxes, the union's source patterns staged in shared
                               //    memory by bulk asynchronous copies, 2 boxes per warp;
                               // 7: as 6 with 4 boxes per warp; 8: as 7 with the source patterns
                               //    by TMA tile copies
  int m2l_pair_warps = 1;      // box pairs (warps) per CTA of the pair translations (variants 4, 5 and the
                               //    complex64 paths): 0 = 2, 1 = 4, 2 = 8
  int l2l_variant = 1;         // 0: 2-D transposed taps per child direction; 1: separable
  int up_threads = 1;          // threads per CTA of the 9-tap interpolation (up variant 0 and the complex64
                               //    paths): 0 = 64, 1 = 128, 2 = 256
  int up_variant = 0;          // 0: 9-tap gather per parent direction; 1: separable in bands;
                               // 2: 9-tap gather, all 6 components per thread;
                               // 3: separable in registers, 4-row bands per thread
  int agg_variant = 0;         // 0: thread per (box, direction); 1: CTA per (box, medium) streaming
                               //    the box's contiguous pattern block
  int batch_tc = 1;            // batched complex64 leaf aggregation and far-field testing: 0 CUDA cores; 1 tcgen05
                               //    (3xTF32 split, TMEM accumulators)
  int batch_tree = 1;          // batched complex64 tree passes: 0 one slot after another; 1 every level
                               //    once for all slots (slot-major arrays)
  int leaf_variant = 0;        // 0: near field inside the leaf kernel; 1: near field on its own
                               //    stream from the start of the apply, the leaf kernel adds the far field
  int graph = 1;               // 1: capture each apply (per x, w, stream and precision) as a CUDA
                               //    graph on first use and replay it; 0: launch the kernels directly
};

// Captured applies, replayed when the same (x, w, stream, precision) recurs.
struct ApplyGraph {
  cudaStream_t s;
  int precision;
  cudaGraphExec_t exec;
};
constexpr size_t kMaxApplyGraphs = 16;

// Per-apply CUDA events between stage groups, recorded on the launching
// stream: [m1 agg | m1 up | m1 m2l | m1 l2l | m2 agg | m2 up | m2 m2l | m2 l2l | leaf_out].
constexpr int kStages = 5;
struct StageProfiler {
  static constexpr int kEvents = 10;
  bool on = false;
  std::vector<std::array<cudaEvent_t, kEvents>> sets;
  size_t used = 0;
};

struct LearnedWork;  // learned preconditioner tables and work arrays (learned.cu)

struct Plan {
  // ---- host description
  Mesh mesh;
  Rwg rwg;
  Tree tree;
  Quad quad;
  int N = 0;
  int maxL = 0;
  int device = 0;
  int verbose = 0;
  int tf_complex_argument = 0;
  int same_triangle_k = 0;          // PlanParams::same_triangle_k
  long long same_triangle_pairs = 0;  // pairs whose z12 the host evaluated (same_triangle_k = 1)
  int precision = 0;                // 0: FP64 operator; 1: also the complex64 operator
  cplx k1, k2, eta1, eta2, etai, epsr, mur;
  double lambda = 0.0, freq = 0.0;
  double setup_seconds = 0.0;
  std::vector<MediumLevel> ml[2];   // index = physical level (0..maxL), used 2..maxL
  std::vector<DevLevel> lv;         // index = physical level
  Tuning tuning;
  // ---- device geometry
  double* d_xyz = nullptr;          // [3 * points]
  int* d_face_v = nullptr;          // [3 * faces]
  int* d_face_id = nullptr;
  double* d_face_area = nullptr;
  double* d_face_normal = nullptr;  // [3 * faces]
  int* d_rwg_fpos = nullptr;
  int* d_rwg_fneg = nullptr;
  int* d_rwg_vpos = nullptr;
  int* d_rwg_vneg = nullptr;
  double* d_rwg_len = nullptr;
  double* d_quad = nullptr;         // [4][nq]: l1, l2, l3, w
  // ---- leaf data
  int* d_leaf_ptr = nullptr;        // [Bleaf+1] into leaf order
  int max_leaf_rwgs = 0;            // most RWGs in one leaf box
  int* d_leaf_rwg = nullptr;        // leaf order -> RWG id
  int* d_rwg_leafbox = nullptr;     // [N] leaf box of each RWG id
  double* d_leaf_center = nullptr;  // [3 * Bleaf]
  double2* d_Vs[2] = {nullptr, nullptr};   // radiation patterns [N][3][K]
  double2* d_Vf[2] = {nullptr, nullptr};   // receive patterns
  float2* d_Vs32[2] = {nullptr, nullptr};  // complex64 copies (precision = mixed)
  float2* d_Vf32[2] = {nullptr, nullptr};
  // ---- near field
  std::vector<long long> h_near_zoff;      // per leaf box, offset of its block (pairs)
  std::vector<int> h_near_sptr;            // per leaf box, offset into source list
  std::vector<int> h_near_src;             // concatenated source RWG ids per leaf box
  int* d_near_sptr = nullptr;       // [Bleaf+1]
  int* d_near_src = nullptr;        // concatenated source RWG ids per box
  long long* d_near_zoff = nullptr; // [Bleaf+1]
  double2* d_near_z = nullptr;      // [pairs][3]
  float2* d_near_z32 = nullptr;     // complex64 copy: preconditioner products, mixed operator
  long long near_pairs = 0;
  // ---- vectors
  int* d_status = nullptr;          // device status bits (a bounded wait that ran out)
  int* h_status = nullptr;          // pinned host copy, read back by the host-pointer apply
  double2* d_gx = nullptr;          // input / output vectors of the captured apply graphs
  double2* d_gw = nullptr;
  double2* d_x = nullptr;           // staging for host-pointer apply
  double2* d_w = nullptr;
  // ---- batched apply: leaf-level S / B arrays of each right-hand-side slot
  // (levels above the leaf are shared: the slots pass through them in turn)
  int batch_cap = 0;
  std::vector<double2*> bS[2], bB[2];
  std::vector<float2*> bS32[2], bB32[2];
  // Complex64 tree arrays of all kBatchSlots right-hand-side slots (mixed
  // plans), per medium and level 2..maxLevel, slot-major and contiguous:
  // [slot][B][6][K]. bS32 / bB32 point into the leaf level's arrays. The
  // batched complex64 apply runs every tree pass once per level for all slots.
  float2* btS[2][16] = {};
  float2* btB[2][16] = {};
  double2* d_xb = nullptr;          // staging for host-pointer batched apply
  double2* d_wb = nullptr;
  int xb_cap = 0;
  cudaStream_t stream = nullptr;
  // the second medium's tree passes run on stream2, forked from and joined
  // back into the caller's stream with these events
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // per medium: the leaf level's translation runs on stream_leaf[m] after
  // ev_agg[m] (aggregation done); ev_leaf[m] marks its end
  cudaStream_t stream_leaf[2] = {nullptr, nullptr};
  cudaEvent_t ev_agg[2] = {nullptr, nullptr}, ev_leaf[2] = {nullptr, nullptr};
  // the near-field product runs on stream_near from ev_start to ev_near
  cudaStream_t stream_near = nullptr;
  cudaEvent_t ev_start = nullptr, ev_near = nullptr;
  StageProfiler prof;
  std::vector<ApplyGraph> graphs;
  std::shared_ptr<LearnedWork> lp;  // allocated on first use; its device arrays are in the heap
  size_t bytes = 0;
  // Plan-lifetime device memory, carved (256-byte aligned) from chunks of
  // kChunk bytes: one driver allocation per chunk instead of one per array
  // (a driver allocation costs milliseconds, and far more on a busy node);
  // requests above kChunk / 4 get their own. Nothing goes back before the
  // plan is destroyed, so no array ever shares memory with a freed one.
  struct DeviceHeap {
    static constexpr size_t kChunk = size_t(64) << 20;
    std::vector<void*> blocks;
    char* cur = nullptr;
    size_t left = 0;
    void* get(size_t bytes);
    void release();
  } heap;
  // Device work arrays of the lockstep solve: one block, kept from one call
  // to the next and grown when a call needs more, so that a refinement's
  // repeated solves and solve after solve allocate nothing. Freed with the
  // plan, or at the end of a call when larger than kKeepBytes.
  struct SolveArena {
    static constexpr size_t kKeepBytes = size_t(16) << 30;
    char* base = nullptr;
    size_t cap = 0, used = 0;
    void reserve(size_t bytes);  // at least bytes in one block; carving restarts
    void* get(size_t bytes);     // the next 256-byte aligned piece of the reservation
    void release();
  } arena;

  ~Plan();
  void tf_inputs(int m, int l, std::vector<double>& rhat, std::vector<int>& hoff, std::vector<int>& hL,
                 std::vector<double2>& h2all) const;
  template <class T>
  T* alloc(size_t count) {
    if (count == 0) count = 1;
    void* p = heap.get(count * sizeof(T));
    bytes += count * sizeof(T);
    return static_cast<T*>(p);
  }
  // A device copy of v, ordered on the plan's stream: kernels on that stream
  // see it; other streams only after a synchronisation of it. (A blocking
  // cudaMemcpy from pageable memory may return before its DMA lands and is
  // not ordered with the plan's non-blocking streams: a kernel launched right
  // after it could read the array before the copy.) The host vector may go
  // as soon as this returns: a pageable source is staged by the call.
  template <class T>
  T* upload(const std::vector<T>& v) {
    T* p = alloc<T>(v.size());
    if (!v.empty()) {
      cudaError_t e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream);
      if (e != cudaSuccess) throw std::runtime_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
    }
    return p;
  }
};

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
void check_cuda(cudaError_t e, const char* what);
#define MLFMA_CUDA(call) ::mlfma::check_cuda((call), #call)

// Setup (plan.cu)
struct PlanParams {
  double freq = 3.0e8;
  cplx epsr{1.0, 0.0}, mur{1.0, 0.0};
  double leaf_coeff = 0.3;
  int gauss = 7;
  int device = 0;
  int verbose = 0;
  // 0: transfer factors with h2_l(|kR|), the reference's choice even for a
  // lossy (complex) k (Code/AlgoMLFMM.h:262-265). 1: h2_l(kR) with the
  // complex argument, consistent with the complex-k shifts and near field.
  int tf_complex_argument = 0;
  // 0: near-field K entries of RWG pairs sharing a triangle at the exact
  // height 0 of a field point above its own triangle (device kernel). 1: those
  // entries evaluated on the host with the reference's own arithmetic, which
  // reproduces its rounding-noise height n.(r - v_i) (Code/Operator.h:582-652)
  // and so its entries bit for bit.
  int same_triangle_k = 0;
  // 0: FP64 operator only. 1: also complex64 copies of the patterns, transfer
  // factors, shift phases, near field and workspaces, for the mixed-precision
  // apply and solves.
  int precision = 0;
};
std::unique_ptr<Plan> create_plan(Mesh&& mesh, const PlanParams& p);

// The arrays of one storage precision: double2 (the FP64 operator) or float2
// (the complex64 copies), for code templated over the kernels' storage type.
template <class C>
struct Store;
template <>
struct Store<double2> {
  static double2* S(const MediumLevel& M) { return M.S; }
  static double2* Bm(const MediumLevel& M) { return M.Bm; }
  static const double2* tfw(const MediumLevel& M) { return M.tfw; }
  static const double2* ph_up(const MediumLevel& M) { return M.ph_up; }
  static const double2* ph_dn(const MediumLevel& M) { return M.ph_dn; }
  static const double2* Vs(const Plan& P, int m) { return P.d_Vs[m]; }
  static const double2* Vf(const Plan& P, int m) { return P.d_Vf[m]; }
  static const double2* near_z(const Plan& P) { return P.d_near_z; }
  static double2* bS(const Plan& P, int m, int j) { return P.bS[m][j]; }
  static double2* bB(const Plan& P, int m, int j) { return P.bB[m][j]; }
};
template <>
struct Store<float2> {
  static float2* S(const MediumLevel& M) { return M.S32; }
  static float2* Bm(const MediumLevel& M) { return M.Bm32; }
  static const float2* tfw(const MediumLevel& M) { return M.tfw32; }
  static const float2* ph_up(const MediumLevel& M) { return M.ph_up32; }
  static const float2* ph_dn(const MediumLevel& M) { return M.ph_dn32; }
  static const float2* Vs(const Plan& P, int m) { return P.d_Vs32[m]; }
  static const float2* Vf(const Plan& P, int m) { return P.d_Vf32[m]; }
  static const float2* near_z(const Plan& P) { return P.d_near_z32; }
  static float2* bS(const Plan& P, int m, int j) { return P.bS32[m][j]; }
  static float2* bB(const Plan& P, int m, int j) { return P.bB32[m][j]; }
};

// Device work (setup_kernels.cu / matvec_kernels.cu)
void launch_patterns(Plan& P, int medium, cudaStream_t s);
// Transfer factors of one (medium, level) into out. The kernel's inputs go
// to the device in one block: from the plan's heap while the plan is built
// (in_heap), else a temporary allocation.
void launch_transfer(Plan& P, int medium, int level, const std::vector<double>& rhat,
                     const std::vector<int>& hoff, const std::vector<int>& hL,
                     const std::vector<double2>& h2, bool weighted, double2* out, cudaStream_t s,
                     bool in_heap = false);
void launch_near(Plan& P, cudaStream_t s);
// Z[3 pos[i] + 1] = z12[i] for n entries of the near field (device arrays).
void launch_near_z12_scatter(double2* Z, const long long* pos, const double2* z12, long long n, cudaStream_t s);
void apply_device(Plan& P, const double2* x, double2* w, cudaStream_t s);
void clear_graphs(Plan& P);  // after any change that alters what an apply launches
// Batched apply: W[j] = A X[j] for j < R; X[j] at X + j * ldx (ldx >= 2N),
// the same for W. Right-hand sides go through in groups of kBatchSlots.
constexpr int kBatchSlots = 16;
// Copies the plan's device status bits to its pinned host word on stream s
// (read after the caller's synchronisation of s) ...
void fetch_device_status(Plan& P, cudaStream_t s);
// ... and throws when one is set (a bounded wait in a kernel ran out: that
// apply's result is incomplete), naming the kernels.
void raise_device_status(const Plan& P);

// Allocates the complex64 slot tree (mixed plans) and, with fp64, the FP64
// leaf-level arrays of min(R, kBatchSlots) slots.
void reserve_batch(Plan& P, int R, bool fp64);
// Allocates d_xb / d_wb (kBatchSlots vectors each), the staging of
// host-pointer batched applies and of the refinement's FP64 residuals.
void reserve_batch_staging(Plan& P);
void apply_batch_device(Plan& P, int R, const double2* X, long long ldx, double2* W, long long ldw, cudaStream_t s);
// The complex64 operator (precision = mixed plans): complex128 x and w, every
// table and workspace in complex64, FP32 arithmetic. Fixed kernel choices:
// aggregation 0, interpolation 0, translation 4, anterpolation 1.
void apply_mixed_device(Plan& P, const double2* x, double2* w, cudaStream_t s);
void apply_batch_mixed_device(Plan& P, int R, const double2* X, long long ldx, double2* W, long long ldw,
                              cudaStream_t s);
// complex128 -> complex64 copy on the device
void to_c64(const double2* src, float2* dst, size_t n, cudaStream_t s);
int read_stage_times(Plan& P, double out[kStages]);

}  // namespace mlfma
