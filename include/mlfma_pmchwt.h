/*
 * mlfma_pmchwt.h -- C ABI of the B200 PMCHWT MLFMA operator and Krylov solve.
 *
 * This is the drop-in boundary for the dielectric (PMCHWT) MLFMA path of the
 * reference solver CCCCl0uD/MLFMA_PMCHWT. Every entry point names the
 * reference interface it replaces (path:line inside the reference project).
 *
 * Conventions
 *  - Complex vectors are interleaved float64 pairs (re, im), the memory layout
 *    of std::complex<double> and of C99 double _Complex.
 *  - Unknown ordering is the reference's: n = 2N for N RWG functions;
 *    x[0:N) = J coefficients, x[N:2N) = M coefficients (Code/MLFMM.cpp:239-245).
 *    RWG order is the reference's RWG numbering (Code/RWGGenerator.cpp:41-72:
 *    common edges in ascending (min vertex id, max vertex id) order).
 *  - No C++ exception crosses this boundary. Every function returns an int
 *    status: MLFMA_OK (0) or a negative code; mlfma_last_error() gives the
 *    message of the last failure on the calling thread.
 *  - One apply/solve in flight per plan (the plan owns its work arrays, as the
 *    reference's MLFMM object owns Sm/Bm, Code/MLFMM.h:60-66). Different plans
 *    may run concurrently.
 */
#ifndef MLFMA_PMCHWT_H
#define MLFMA_PMCHWT_H

#if defined(__GNUC__)
#define MLFMA_API __attribute__((visibility("default")))
#else
#define MLFMA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MLFMA_OK 0
#define MLFMA_ERR_ARG (-1)        /* bad argument: null pointer, size mismatch, n <= 0 */
#define MLFMA_ERR_MESH (-2)       /* mesh / NAS input unusable */
#define MLFMA_ERR_CUDA (-3)       /* CUDA runtime error */
#define MLFMA_ERR_NOMEM (-4)      /* device or host allocation failed */
#define MLFMA_ERR_UNSUPPORTED (-5)/* option not supported */
#define MLFMA_ERR_NOT_CONVERGED 1 /* solve ended without meeting the tolerance (not an error) */

typedef struct mlfma_plan mlfma_plan;

/* Triangle mesh in NAS terms (Code/NASReader.cpp:60-144): GRID ids with
 * coordinates, CTRIA3 ids with three GRID ids each. Faces keep file order. */
typedef struct {
  int num_points;
  const int* point_ids;        /* [num_points] GRID ids */
  const double* xyz;           /* [3*num_points] */
  int num_faces;
  const int* face_ids;         /* [num_faces] CTRIA3 ids */
  const int* face_points;      /* [3*num_faces] GRID ids of vertex1..3 */
} mlfma_mesh;

/* Physical and discretisation parameters. Defaults (mlfma_default_params):
 * the reference's EMSource / PhyConstant / main.cpp values. */
typedef struct {
  double freq_hz;              /* EMSource(freq), Code/EMSource.cpp:6-14 */
  double eps_r_re, eps_r_im;   /* EMSource::initDielectric, Code/EMSource.cpp:19-32 */
  double mu_r_re, mu_r_im;
  double leaf_coeff;           /* leaf box edge in wavelengths (Code/PhyConstant.h:14; 0.3) */
  int gauss_points;            /* triangle rule: 1,3,4,6,7,12,13,16 (Code/GaussPoints.cpp:286-299) */
  int precision;               /* MLFMA_PREC_FP64, or MLFMA_PREC_MIXED: the plan also holds
                                  complex64 copies of its tables for mlfma_apply_mixed_device
                                  and the mixed-precision solves */
  int device;                  /* CUDA device ordinal */
  int verbose;                 /* print setup summary to stderr */
  int tf_complex_argument;     /* 0 (default): transfer factors with h2_l(|kR|) as the reference
                                  (Code/AlgoMLFMM.h:262-265); 1: h2_l(kR) with complex kR, a
                                  departure from the reference for lossy media */
  int same_triangle_k;         /* near-field K entries of RWG pairs that share a triangle
                                  (Code/Operator.h:325-707, 883-1046). 0 (default): evaluated on
                                  the GPU at the exact height 0 of a field point above its own
                                  triangle. 1: evaluated on the host with the reference's own
                                  arithmetic, including its rounding-noise height n.(r - v_i),
                                  which reproduces the reference's entries bit for bit */
} mlfma_params;

#define MLFMA_PREC_FP64 0
#define MLFMA_PREC_MIXED 1

typedef struct {
  int num_rwg;                 /* N */
  int num_unknowns;            /* 2N */
  int max_level;               /* OCTree::maxLevel_ */
  int num_levels;              /* MLFMA levels 2..max_level */
  int boxes[16];               /* boxes at level 2+i */
  int L_k1[16], L_k2[16];      /* multipole order at level 2+i */
  int K_k1[16], K_k2[16];      /* directions at level 2+i */
  long long near_pairs;        /* RWG pairs in the near field */
  long long far_pairs[16];     /* interaction-list pairs at level 2+i */
  double bytes_device;         /* device bytes held by the plan */
  double setup_seconds;        /* wall time of mlfma_plan_create */
  double k1_re, k1_im, k2_re, k2_im, etai_re, etai_im, wavelength;
} mlfma_info;

typedef struct {
  int iterations;              /* inner Arnoldi steps taken (MGMRES total_iter) */
  int restarts;                /* restart cycles */
  int matvecs;                 /* operator applications */
  int converged;               /* 1 if the tolerance was met */
  double rel_residual;         /* last true residual ||b - A x|| / ||b|| */
  double seconds;              /* device time of the solve */
  int history_len;             /* entries written to history */
  int near_products;           /* near-field-only products spent in the preconditioner */
} mlfma_solve_stats;

MLFMA_API void mlfma_default_params(mlfma_params* p);
MLFMA_API const char* mlfma_last_error(void);
MLFMA_API const char* mlfma_version(void);

/* Builds the operator: RWGs (Code/RWGGenerator.cpp:39-113), octree
 * (Code/OCTree.cpp:13-32), angular grids (Code/AlgoMLFMM.h:21-138),
 * transfer factors (:192-295), interpolation (:298-368), radiation/receive
 * patterns (Code/ProcessFMM.h:217-233) and the near-field PMCHWT rows
 * (Code/Zmartix.h:541-643) -- replaces the setup half of the MLFMM
 * constructor (Code/MLFMM.cpp:15-113). Patterns, transfer factors and the
 * near field are computed on the GPU. */
MLFMA_API int mlfma_plan_create(const mlfma_mesh* mesh, const mlfma_params* params, mlfma_plan** plan);

/* Same, reading a NAS file in the dialect of Code/NASReader.cpp:60-144. */
MLFMA_API int mlfma_plan_create_nas(const char* nas_path, const mlfma_params* params, mlfma_plan** plan);

MLFMA_API int mlfma_plan_destroy(mlfma_plan* plan);
MLFMA_API int mlfma_plan_info(const mlfma_plan* plan, mlfma_info* info);

/* w = A x, the PMCHWT MLFMA matvec: the `ax` closure of
 * MLFMM::matrix_solver (Code/MLFMM.cpp:189-368), i.e. the documented
 * MLFMM::applyAx(int n, const std::complex<double>* x, std::complex<double>* w).
 * Host pointers; n must be 2N. w is overwritten. */
MLFMA_API int mlfma_apply(mlfma_plan* plan, int n, const double* x, double* w);

/* The same on device-resident vectors (complex128 [n]) on a CUDA stream
 * (cudaStream_t passed as void*; NULL = the plan's stream). Asynchronous. */
MLFMA_API int mlfma_apply_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream);

/* Device status bits of a plan after the device-pointer calls: synchronizes
 * the device and writes 0, or bit 1 when a bounded wait in a kernel ran out
 * and the output of that call is not valid, with the kernel's bit beside it:
 * 2 tensor-core aggregation, 4 tensor-core far-field testing, 8 staged
 * translation (m2l.variant 6-8). The host-pointer calls and every host
 * synchronisation of the solvers check the same bits and fail with
 * MLFMA_ERR_CUDA (the solvers clear them when they start). */
MLFMA_API int mlfma_device_status(mlfma_plan* plan, int* status);

/* Batched apply: w[j] = A x[j] for R right-hand sides stored one after the
 * other (x[j] at x + 2 n j doubles, complex128 interleaved, n = 2N each).
 * The reference applies its AxFunc (Code/GMRES.h:53-66, the ax closure of
 * Code/MLFMM.cpp:189-368) once per right-hand side; here the leaf radiation /
 * receive patterns and the near-field entries are read once per group of up
 * to 16 right-hand sides. Each w[j] equals the single apply's result.
 * The first call on a plan allocates the leaf-level workspace of min(R, 16)
 * right-hand sides (about 2 x leaf boxes x 6 x (K1+K2) x 16 bytes each) plus,
 * for the host-pointer form, 2 x 16 staging vectors. Not re-entrant per plan. */
MLFMA_API int mlfma_apply_batch(mlfma_plan* plan, int n, int R, const double* x, double* w);
/* The batched apply with the complex64 operator (a plan created with
 * MLFMA_PREC_MIXED), device vectors as in mlfma_apply_batch_device. Its leaf
 * aggregation and far-field testing run on the tensor cores (tcgen05, TF32
 * operands split into high and low parts, FP32 accumulation in TMEM) when the
 * tuning key "batch_tc.variant" is 1 and every leaf box holds at most 64 RWGs,
 * else on the CUDA cores. No counterpart in the reference. */
MLFMA_API int mlfma_apply_batch_mixed_device(mlfma_plan* plan, int n, int R, const void* x_dev, void* w_dev,
                                             void* stream);
MLFMA_API int mlfma_apply_batch_device(mlfma_plan* plan, int n, int R, const void* x_dev, void* w_dev,
                                       void* stream);

/* Stage timing (no counterpart in the reference, whose timers are
 * std::chrono prints): with on != 0 every apply records CUDA events on its
 * stream between stage groups; mlfma_profile_read sums them since the last
 * read into stage_ms[5] = {aggregation, interpolation up, translation,
 * anterpolation down, leaf testing + near field} and the number of applies. */
MLFMA_API int mlfma_profile(mlfma_plan* plan, int on);
MLFMA_API int mlfma_profile_read(mlfma_plan* plan, double* stage_ms, int* applies);

/* Kernel variants of a plan (no counterpart in the reference). Keys, values
 * and defaults (the fastest measured at 245,760 unknowns):
 *   "m2l.variant"  translation: 0 = one thread per (box, direction) over the
 *                  interaction list; 1 = sibling-group tiles staging the shared
 *                  sources in shared memory; 2 = octant registers over the
 *                  siblings' union; 3 = warp per box, 8 Morton-consecutive
 *                  boxes per CTA; 4 = warp per pair of Morton-consecutive boxes
 *                  over their merged lists, each source pattern loaded once for
 *                  both (default); 5 = as 4 with the J and M halves on separate
 *                  warps; 6 = groups of 8 Morton-consecutive boxes over the
 *                  union of their lists, each union source's patterns staged
 *                  in shared memory by bulk asynchronous copies ahead of the
 *                  arithmetic, 2 boxes per warp; 7 = as 6 with 4 boxes per
 *                  warp. 2-7 launch the leaf level and the other levels of a
 *                  medium as two launches.
 *   "m2l.pair_warps" tile shape of the pair translation (m2l variant 4 and
 *                  the complex64 paths): 0 = 2, 1 = 4 (default), 2 = 8 box
 *                  pairs (warps) per CTA.
 *   "up.variant"   interpolation: 0 = 9-tap gather per parent direction and
 *                  component (default); 1 = separable phi-then-theta in bands of
 *                  theta rows through shared memory; 2 = one thread per
 *                  (parent, direction) for all 6 components; 3 = separable in
 *                  registers, a phi column of 4 parent theta rows per thread.
 *   "up.threads"   tile shape of the 9-tap interpolation (up variant 0 and the
 *                  complex64 paths): 0 = 64, 1 = 128 (default), 2 = 256
 *                  parent directions (threads) per CTA.
 *   "l2l.variant"  anterpolation: 0 = transposed 9-tap gather per child
 *                  direction; 1 = separable transposed theta-then-phi (default).
 *   "agg.variant"  aggregation: 0 = one thread per (leaf box, direction), one
 *                  launch per medium (default); 1 = one CTA per (leaf box,
 *                  medium) streaming the box's contiguous pattern block.
 *   "batch_tc.variant" (the batched complex64 apply only) 0 = leaf aggregation
 *                  and far-field testing on the CUDA cores; 1 = on the tensor
 *                  cores (tcgen05 kind::tf32 with high/low operand splitting,
 *                  boxes of at most 64 RWGs; default).
 *   "batch_tree.variant" (the batched complex64 apply only) 0 = the tree
 *                  passes of each right-hand side in turn; 1 = every level
 *                  once for all right-hand sides on slot-major arrays (default).
 *   "leaf.variant" 0 = the near-field rows inside the leaf testing kernel (default);
 *                  1 = the near-field product on its own stream from the start
 *                  of the apply (it needs only x), overlapping the tree
 *                  passes; the leaf kernel then adds the far field.
 *   "apply.graph"  1 = the apply of each (stream, precision) is captured as a
 *                  CUDA graph on first use and replayed afterwards (default);
 *                  the graph works on plan-owned vectors, x is copied in and
 *                  w out around each replay (device copies of 2N values), so
 *                  any x, w pair reuses it; 0 = direct launches. Setting any
 *                  key drops the captured graphs. Inside a caller's own
 *                  capture the apply launches directly.
 * mlfma_autotune times the values of each key in that order (the others held
 * at their current values) over `applies` applies of the plan's own operator
 * (device vectors owned by the plan) and keeps the fastest; variant_ms (may be
 * NULL) receives the per-apply ms of every value, keys in that order
 * (31 entries: m2l 0-8, m2l.pair_warps 0-2, up 0-3, up.threads 0-2, l2l 0-1,
 * agg 0-1, leaf 0-1, batch_tc 0-1, batch_tree 0-1, graph 0-1). "batch_tc.variant" and "batch_tree.variant"
 * act on the batched complex64 apply only: autotune leaves them as set and
 * reports -1 for their entries. */
MLFMA_API int mlfma_set_tuning(mlfma_plan* plan, const char* key, int value);
MLFMA_API int mlfma_get_tuning(const mlfma_plan* plan, const char* key);
MLFMA_API int mlfma_autotune(mlfma_plan* plan, int applies, double* variant_ms);

/* Restarted GMRES(mr) with the operator -- replaces MGMRES::mgmres
 * (Code/GMRES.h:65-217) driven by MLFMM::matrix_solver (Code/MLFMM.cpp:186).
 * Same arguments and stopping rule: stop when ||r||/||b|| < tol_rel or
 * < tol_abs, or after itr_max inner steps; true residual after each cycle;
 * divergence abort after cycle 8. x holds the initial guess on entry and the
 * solution on return (host pointers). history (optional, may be NULL) receives
 * the estimated relative residual of each inner step, up to history_cap.
 * Returns MLFMA_OK when converged, MLFMA_ERR_NOT_CONVERGED otherwise. */
MLFMA_API int mlfma_gmres(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr,
                double tol_abs, double tol_rel, mlfma_solve_stats* stats, double* history,
                int history_cap);

/* Flexible GMRES(mr) with a near-field preconditioner. No direct
 * counterpart in the reference, whose only solvers are MGMRES::mgmres and
 * CGS (Code/CGS.h). Arguments, stopping rule, true residual per cycle and
 * divergence abort are those of mlfma_gmres. The right preconditioner is
 * inner_its GMRES steps from zero on the near-field matrix alone (the Z_near
 * rows of Code/Zmartix.h:541-643), whose products use the plan's complex64
 * copy of Z_near (a flexible outer iteration admits any preconditioner; the
 * operator and the true residual stay FP64); inner_its = 0 reduces to plain
 * GMRES.
 * itr_max counts outer steps; stats->near_products counts inner products. */
MLFMA_API int mlfma_fgmres(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr,
                           double tol_abs, double tol_rel, int inner_its, mlfma_solve_stats* stats,
                           double* history, int history_cap);

/* Lockstep FGMRES of R right-hand sides (x, rhs: R vectors of n = 2N
 * complex128 one after the other; x holds the initial guesses and receives
 * the solutions). Per system the iteration, stopping rule and divergence
 * abort are mlfma_fgmres's (itself MGMRES::mgmres, Code/GMRES.h:65-217, with
 * the optional near-field right preconditioner); the reference solves its
 * incidences one after the other (Code/RCS.h:467-468). Here every Arnoldi
 * step applies the operator to all systems still iterating at once
 * (mlfma_apply_batch), and the inner near-field products and the
 * Gram-Schmidt steps are batched the same way. stats: R entries (seconds =
 * the whole batch, history_len = 0). Returns MLFMA_OK when every system
 * converged, MLFMA_ERR_NOT_CONVERGED otherwise. */
MLFMA_API int mlfma_fgmres_batch(mlfma_plan* plan, int n, int R, double* x, const double* rhs, int itr_max, int mr,
                                 double tol_abs, double tol_rel, int inner_its, mlfma_solve_stats* stats);

/* Mixed precision (plans created with precision = MLFMA_PREC_MIXED; no
 * counterpart in the reference, which is FP64 throughout). The complex64
 * operator keeps complex128 x and w but holds the radiation/receive
 * patterns, transfer factors, shift phases, near field and Sm/Bm workspaces
 * in complex64 and computes in FP32; its relative difference from the FP64
 * operator is about 1e-6. */
MLFMA_API int mlfma_apply_mixed(mlfma_plan* plan, int n, const double* x, double* w);
MLFMA_API int mlfma_apply_mixed_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream);

/* FP64 iterative refinement: up to refine_max steps of
 *   r = b - A x (FP64 operator, the plain path); stop when ||r||/||b|| < tol_rel
 *   (or < tol_abs); d = FGMRES(mr) on A d = r with the complex64 operator and
 *   inner_its complex64 near-field steps as preconditioner, to the relative
 *   tolerance max(1e-5, min(0.5, tol_rel / (2 ||r||/||b||))); x += d.
 * The stopping test is always the FP64 residual. itr_max bounds the FGMRES
 * iterations summed over the steps; stats->restarts = refinement steps;
 * history[i] = FP64 relative residual after step i (entry 0: initial). */
MLFMA_API int mlfma_solve_mixed(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr,
                                double tol_abs, double tol_rel, int inner_its, int refine_max,
                                mlfma_solve_stats* stats, double* history, int history_cap);
/* The same for R right-hand sides (x, rhs: R vectors one after the other):
 * FP64 residuals by batched applies, corrections by lockstep FGMRES with the
 * complex64 operator (mlfma_fgmres_batch's iteration). stats: R entries. */
MLFMA_API int mlfma_solve_mixed_batch(mlfma_plan* plan, int n, int R, double* x, const double* rhs, int itr_max,
                                      int mr, double tol_abs, double tol_rel, int inner_its, int refine_max,
                                      mlfma_solve_stats* stats);

/* w = Z_near x on device vectors: the near-field rows alone (the product of
 * Code/MLFMM.cpp:353-366 without the far field). Asynchronous on stream. */
MLFMA_API int mlfma_apply_near_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream);

/* z = the near-field preconditioner of mlfma_fgmres applied to v (inner_its
 * GMRES steps from zero on the complex64 Z_near), device vectors; returns
 * after the result is complete. */
MLFMA_API int mlfma_near_precondition_device(mlfma_plan* plan, int n, int inner_its, const void* v_dev,
                                             void* z_dev, void* stream);

/* Learned preconditioner (no counterpart in the reference). A message-passing
 * network over the leaf boxes corrects the near-field preconditioner's
 * output: y = z + sum_t G_t u_t per RWG, with linear terms u built from z
 * (z itself and dipole projections of its box, one-ring and two-ring
 * means) and complex gains G predicted from static geometric and material
 * features, so that y = (I + L) z is linear. 3 layers of width 64, bfloat16
 * weights, FP32 arithmetic; parameters are one float vector of
 * mlfma_lp_param_count() entries (We, be, (Ws, Wn, Wg, c) x 3, Wd1, d1, Wd2,
 * d2, row-major). Training pairs are (v, z = P_near v), with e = A^-1 v for
 * the error loss.
 *
 * mlfma_lp_forward_device: y = the network's output for (v, z) with the
 * float parameters params_dev (NULL: the attached network); y may alias z.
 * It keeps the intermediates that mlfma_lp_backward_device needs.
 * mlfma_lp_backward_device: after mlfma_lp_forward_device with the same
 * parameters, adds to grad_dev the parameter gradient of any loss L(y) given
 * gy = dL/dRe(y) + j dL/dIm(y) (complex128 [2N]), e.g. the residual-space
 * loss |A y - v|^2 / |v|^2 with gy = 2 A^H (A y - v) / |v|^2. (v enters
 * the network only through z; it is passed for the interface's symmetry.)
 * mlfma_lp_loss_grad_device: y as above, and adds the loss
 * sum |y - e|^2 / sum |e|^2 to *loss_dev and its gradient with respect to
 * the parameters (taken at their bfloat16 values) to grad_dev.
 * mlfma_lp_adam_device: one Adam step on params_dev (moments m_dev, v_dev,
 * step counted from 1; the gradient is multiplied by grad_scale first).
 * mlfma_lp_attach: the network that mlfma_fgmres, mlfma_fgmres_batch and the
 * mixed-precision solves apply after the near-field preconditioner (host
 * parameters; nparams = 0 detaches). All device calls are asynchronous on
 * stream (NULL: the plan's stream). */
MLFMA_API int mlfma_lp_param_count(void);
MLFMA_API int mlfma_lp_forward_device(mlfma_plan* plan, int n, const float* params_dev, const void* v_dev,
                                      const void* z_dev, void* y_dev, void* stream);
MLFMA_API int mlfma_lp_backward_device(mlfma_plan* plan, int n, const float* params_dev, const void* gy_dev,
                                       float* grad_dev, void* stream);
MLFMA_API int mlfma_lp_loss_grad_device(mlfma_plan* plan, int n, const float* params_dev, const void* v_dev,
                                        const void* z_dev, const void* e_dev, void* y_dev, float* grad_dev,
                                        float* loss_dev, void* stream);
MLFMA_API int mlfma_lp_adam_device(int nparams, float* params_dev, const float* grad_dev, float* m_dev, float* v_dev,
                                   float lr, float beta1, float beta2, float eps, int step, float grad_scale,
                                   void* stream);
MLFMA_API int mlfma_lp_attach(mlfma_plan* plan, const float* params, int nparams);

/* Plane-wave excitation vector V (complex128 [2N]) -- RHS::computeV_PMCHWT
 * (Code/Vm.h:150-203) with the incident unit vectors of EMSource::initPW
 * (Code/EMSource.cpp:34-72): kinc (propagation), einc (E polarisation),
 * hinc (kinc x einc). Host pointers. */
MLFMA_API int mlfma_rhs_pmchwt(mlfma_plan* plan, const double kinc[3], const double einc[3],
                     const double hinc[3], double* V);

/* Far-field of currents I (complex128 [2N]) at n_angles directions
 * (degrees) -- RCSUtils::calculateRCS_PMCHWT (Code/RCS.h:116-192).
 * field (optional): 3 complex Cartesian components per angle (6 doubles).
 * rcs_db (optional): total / theta-pol / phi-pol RCS in dBsm per angle
 * (3 doubles), formed as the dual-static study does (Code/RCS.h:391-410). */
MLFMA_API int mlfma_rcs_pmchwt(mlfma_plan* plan, const double* I, int n_angles, const double* theta_deg,
                     const double* phi_deg, double* field, double* rcs_db);

/* Excitation vectors of R plane waves in one call -- RHS::computeV_PMCHWT
 * (Code/Vm.h:150-203) per incidence, as the mono-static study calls it once
 * per angle (Code/RCS.h:436-494). kinc/einc/hinc: host tables [R][3] (read
 * before the call returns); V_dev: device complex128 [R][2N]. Asynchronous on
 * `stream` (NULL = the plan's stream); allocates nothing. */
MLFMA_API int mlfma_rhs_pmchwt_batch_device(mlfma_plan* plan, int n, int R, const double* kinc, const double* einc,
                                            const double* hinc, void* V_dev, void* stream);

/* Bistatic far field of R current vectors in one call -- RCSUtils::
 * calculateRCS_PMCHWT (Code/RCS.h:116-192) for every (solution, angle), as
 * the dual-static study evaluates it (Code/RCS.h:345-425). I_dev: device
 * complex128 [R][2N]; theta_deg/phi_deg: host [n_angles] (read before the
 * call returns); field_dev: device complex128 [R][n_angles][3] (Cartesian E).
 * Asynchronous; allocates nothing. */
MLFMA_API int mlfma_rcs_pmchwt_batch_device(mlfma_plan* plan, int n, int R, const void* I_dev, int n_angles,
                                            const double* theta_deg, const double* phi_deg, void* field_dev,
                                            void* stream);

/* Monostatic far field: solution r observed at its own angle
 * (theta_deg[r], phi_deg[r]), the backscatter evaluation of the mono-static
 * loop (Code/RCS.h:436-494). field_dev: device complex128 [R][3]. */
MLFMA_API int mlfma_rcs_pmchwt_mono_device(mlfma_plan* plan, int n, int R, const void* I_dev,
                                           const double* theta_deg, const double* phi_deg, void* field_dev,
                                           void* stream);

/* RCS in dBsm from far fields (host, 6 doubles per angle): total,
 * theta-pol and phi-pol per angle, formed as Code/RCS.h:391-410 does. */
MLFMA_API int mlfma_rcs_db(int n_angles, const double* theta_deg, const double* phi_deg, const double* field,
                           double* rcs_db);

/* Far field without device allocation. No counterpart in the reference.
 * For callers that cannot allocate device memory while they run -- e.g. an
 * application that reserves all device memory up front in its own pool, or a
 * real-time loop in which cudaMalloc/cudaFree and the synchronisation they can
 * imply are not allowed. Computes the same field as mlfma_rcs_pmchwt, but I_dev
 * (complex128 [2N]) and field_dev (3 complex per angle) are device pointers
 * the caller owns, and the only scratch, the angle table, is a fixed
 * file-scope device array held by every GPU that loads this library until the
 * process exits. Limits and behaviour:
 *  - n_angles <= mlfma_rcs_noalloc_max_angles() (8192); larger counts return
 *    MLFMA_ERR_ARG with a message and launch nothing.
 *  - Calls no cudaMalloc, cudaFree or allocating library routine.
 *  - The first call on a device, with any n_angles (0 included), does the
 *    set-up: it looks up the array's device address (cudaGetSymbolAddress)
 *    with that device current and loads the kernel. Make that first call
 *    before any stream capture.
 *  - Every call shares the one array (it keeps the last call's angles):
 *    calls that overlap on the GPU, on any stream or plan, race. Order them on
 *    one stream or synchronise between them.
 *  - Asynchronous on `stream` (NULL = the plan's stream). theta_deg and
 *    phi_deg are host arrays copied into the device array by
 *    cudaMemcpyAsync on that stream. From pageable memory the copy has taken
 *    the values when the call returns (at the cost of the stream
 *    synchronisation the runtime performs for pageable copies). From pinned
 *    memory the copy reads them when the stream reaches it: such arrays must
 *    stay valid and unchanged until then.
 *  - The caller's current device is the same after the call as before. */
MLFMA_API int mlfma_rcs_pmchwt_noalloc(mlfma_plan* plan, const void* I_dev, int n_angles,
                                       const double* theta_deg, const double* phi_deg, void* field_dev,
                                       void* stream);
MLFMA_API int mlfma_rcs_noalloc_max_angles(void);

/* Copies of the plan's tables, for verification against the reference.
 * mlfma_get_rwgs: per RWG (reference order): face ids of T+ / T-, GRID ids of
 * the free vertices and of the common edge, edge length, edge midpoint
 * (RWGBase, Code/MyStruct.h:93-103). Any pointer may be NULL. */
MLFMA_API int mlfma_get_rwgs(const mlfma_plan* plan, int* face_pos, int* face_neg, int* free_pos,
                   int* free_neg, int* edge_a, int* edge_b, double* length, double* mid);

/* Boxes of one octree level (physical level 2..max_level) in the plan's
 * order (ascending Morton code): Morton codes and centres. Returns the count
 * when the pointers are NULL. */
MLFMA_API long long mlfma_get_level(const mlfma_plan* plan, int level, unsigned long long* morton,
                          double* center);

/* Stage arrays after the last apply, for stage-level comparison:
 * which 0 = aggregated pattern Sm, 1 = incoming pattern Bm; medium 1 or 2;
 * level = physical level; out: [boxes][6][K] complex (J xyz then M xyz).
 * Returns the number of complex values (or that count when out is NULL). */
MLFMA_API long long mlfma_get_stage(mlfma_plan* plan, int which, int medium, int level, double* out);

/* Leaf radiation (which 0) / receive (which 1) patterns of medium 1|2 in
 * reference RWG order: [N][K][3] complex (the layout of Vsmi/Vfmj). */
MLFMA_API long long mlfma_get_pattern(mlfma_plan* plan, int medium, int which, double* out);

/* Transfer factors of medium at a level as [vec][K] complex with the
 * integer translation offsets (target - source, in box edges) [vec][3]. */
MLFMA_API long long mlfma_get_transfer(mlfma_plan* plan, int medium, int level, int* offsets, double* tf);

/* Near-field entries: per near RWG pair (target t, source s), in the plan's
 * order: t, s (reference RWG ids) and z11, z12, z22 (Code/Zmartix.h:611-628;
 * z21 = -z12). Returns the pair count when pointers are NULL. */
MLFMA_API long long mlfma_get_near(mlfma_plan* plan, int* target, int* source, double* z11, double* z12,
                         double* z22);

/* The near pairs whose RWGs share a triangle, in the plan's near-field
 * order: t, s (reference RWG ids) and z12 = -(K(k1) + K(k2)) evaluated on the
 * host with the reference's own arithmetic (Code/Zmartix.h:605-612,
 * Code/Operator.h:325-707, 883-1046), whatever the plan's same_triangle_k.
 * Host-only plans (device < 0) answer too. Returns the pair count when the
 * pointers are NULL. */
MLFMA_API long long mlfma_get_near_same_triangle(mlfma_plan* plan, int* target, int* source, double* z12);

/* Near (26-neighbourhood, Code/OCTree.cpp:385-426) and interaction lists
 * (Code/OCTree.cpp:428-488) of a level in CSR form over the plan's box
 * order; far_off is the encoded offset target - source,
 * (dx+3)*49 + (dy+3)*7 + (dz+3). Returns the interaction-pair count. */
MLFMA_API long long mlfma_get_level_lists(const mlfma_plan* plan, int level, int* near_ptr, int* near_idx,
                                          int* far_ptr, int* far_idx, int* far_off);

/* RWG ids of each leaf box (CSR): leaf_ptr [boxes+1], leaf_rwg [N]. Returns the box count. */
MLFMA_API long long mlfma_get_leaf_rwgs(const mlfma_plan* plan, int* leaf_ptr, int* leaf_rwg);

/* Angular grid of medium 1|2 at a physical level (Code/AlgoMLFMM.h:21-138):
 * theta [L], phi [2L], Gauss-Legendre weights [L], phi weight. Returns L. */
MLFMA_API int mlfma_get_grid(const mlfma_plan* plan, int medium, int level, double* theta, double* phi,
                             double* wtheta, double* wphi);

/* Interpolation from level+1 onto level (Code/AlgoMLFMM.h:298-368), in
 * separable form: per parent theta row, three child theta indices and
 * Lagrange weights; per parent phi column, three child phi indices and
 * weights (the reference's 9 weights are the products lt * lp). */
MLFMA_API int mlfma_get_interp(const mlfma_plan* plan, int medium, int level, int* tidx, double* lt, int* pidx,
                               double* lp);

#ifdef __cplusplus
}
#endif

#endif /* MLFMA_PMCHWT_H */
