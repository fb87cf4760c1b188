// extern "C" boundary (include/mlfma_pmchwt.h). No exception crosses it:
// every entry point maps failures onto status codes and records the message
// for mlfma_last_error() on the calling thread.
#include <algorithm>
#include <cuda_runtime.h>

#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/mlfma_pmchwt.h"
#include "learned.hpp"
#include "near_same_triangle.hpp"
#include "plan.hpp"
#include "solver.hpp"

struct mlfma_plan {
  std::unique_ptr<mlfma::Plan> p;
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const mlfma::CudaError& e) {
    return fail(MLFMA_ERR_CUDA, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(MLFMA_ERR_NOMEM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return fail(MLFMA_ERR_ARG, e.what());
  } catch (const std::domain_error& e) {
    return fail(MLFMA_ERR_MESH, e.what());
  } catch (const std::exception& e) {
    const std::string w = e.what();
    if (w.find("cudaMalloc") != std::string::npos) return fail(MLFMA_ERR_NOMEM, w);
    return fail(MLFMA_ERR_CUDA, w);
  }
}

mlfma::PlanParams to_params(const mlfma_params* p) {
  mlfma::PlanParams q;
  q.freq = p->freq_hz;
  q.epsr = mlfma::cplx(p->eps_r_re, p->eps_r_im);
  q.mur = mlfma::cplx(p->mu_r_re, p->mu_r_im);
  q.leaf_coeff = p->leaf_coeff;
  q.gauss = p->gauss_points;
  q.device = p->device;
  q.verbose = p->verbose;
  q.tf_complex_argument = p->tf_complex_argument;
  q.same_triangle_k = p->same_triangle_k;
  q.precision = p->precision == MLFMA_PREC_MIXED ? 1 : 0;
  return q;
}

bool device_plan(const mlfma_plan* plan) { return plan && plan->p && plan->p->device >= 0; }

// Waits for the plan's stream and raises if a kernel recorded a device
// status bit (a bounded wait that ran out), naming the kernel.
void sync_and_check(mlfma::Plan& P) {
  mlfma::fetch_device_status(P, P.stream);
  MLFMA_CUDA(cudaStreamSynchronize(P.stream));
  mlfma::raise_device_status(P);
}

}  // namespace

extern "C" {

void mlfma_default_params(mlfma_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->freq_hz = 3.0e8;
  p->eps_r_re = 1.0;
  p->mu_r_re = 1.0;
  p->leaf_coeff = 0.3;
  p->gauss_points = 7;
  p->precision = MLFMA_PREC_FP64;
  p->device = 0;
}

const char* mlfma_last_error(void) { return g_last_error.c_str(); }

const char* mlfma_version(void) { return "mlfma_pmchwt_b200 0.2 (sm_100a, FP64 and mixed complex64/FP64)"; }

int mlfma_plan_create(const mlfma_mesh* mesh, const mlfma_params* params, mlfma_plan** plan) {
  if (!mesh || !params || !plan) return fail(MLFMA_ERR_ARG, "null argument");
  *plan = nullptr;
  return guarded([&] {
    if (params->precision != MLFMA_PREC_FP64 && params->precision != MLFMA_PREC_MIXED)
      return fail(MLFMA_ERR_ARG, "precision must be MLFMA_PREC_FP64 or MLFMA_PREC_MIXED");
    mlfma::Mesh m;
    std::string err;
    if (!mlfma::mesh_from_arrays(mesh->num_points, mesh->point_ids, mesh->xyz, mesh->num_faces, mesh->face_ids,
                                 mesh->face_points, m, err))
      return fail(MLFMA_ERR_MESH, err);
    auto p = mlfma::create_plan(std::move(m), to_params(params));
    *plan = new mlfma_plan{std::move(p)};
    return MLFMA_OK;
  });
}

int mlfma_plan_create_nas(const char* nas_path, const mlfma_params* params, mlfma_plan** plan) {
  if (!nas_path || !params || !plan) return fail(MLFMA_ERR_ARG, "null argument");
  *plan = nullptr;
  return guarded([&] {
    if (params->precision != MLFMA_PREC_FP64 && params->precision != MLFMA_PREC_MIXED)
      return fail(MLFMA_ERR_ARG, "precision must be MLFMA_PREC_FP64 or MLFMA_PREC_MIXED");
    mlfma::Mesh m;
    std::string err;
    if (!mlfma::read_nas(nas_path, m, err)) return fail(MLFMA_ERR_MESH, err);
    auto p = mlfma::create_plan(std::move(m), to_params(params));
    *plan = new mlfma_plan{std::move(p)};
    return MLFMA_OK;
  });
}

int mlfma_plan_destroy(mlfma_plan* plan) {
  if (!plan) return MLFMA_OK;
  return guarded([&] {
    delete plan;
    return MLFMA_OK;
  });
}

int mlfma_plan_info(const mlfma_plan* plan, mlfma_info* info) {
  if (!plan || !plan->p || !info) return fail(MLFMA_ERR_ARG, "null argument");
  const mlfma::Plan& P = *plan->p;
  std::memset(info, 0, sizeof(*info));
  info->num_rwg = P.N;
  info->num_unknowns = 2 * P.N;
  info->max_level = P.maxL;
  info->num_levels = P.maxL - 1;
  for (int l = 2; l <= P.maxL && l - 2 < 16; ++l) {
    info->boxes[l - 2] = P.lv[l].B;
    info->L_k1[l - 2] = P.ml[0][l].L;
    info->L_k2[l - 2] = P.ml[1][l].L;
    info->K_k1[l - 2] = P.ml[0][l].K;
    info->K_k2[l - 2] = P.ml[1][l].K;
    info->far_pairs[l - 2] = P.lv[l].far_pairs;
  }
  info->near_pairs = P.near_pairs;
  info->bytes_device = static_cast<double>(P.bytes);
  info->setup_seconds = P.setup_seconds;
  info->k1_re = P.k1.real();
  info->k1_im = P.k1.imag();
  info->k2_re = P.k2.real();
  info->k2_im = P.k2.imag();
  info->etai_re = P.etai.real();
  info->etai_im = P.etai.imag();
  info->wavelength = P.lambda;
  return MLFMA_OK;
}

int mlfma_apply(mlfma_plan* plan, int n, const double* x, double* w) {
  if (!plan || !plan->p || !x || !w) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    const size_t bytes = static_cast<size_t>(n) * sizeof(double2);
    MLFMA_CUDA(cudaMemcpyAsync(P.d_x, x, bytes, cudaMemcpyHostToDevice, P.stream));
    mlfma::apply_device(P, P.d_x, P.d_w, P.stream);
    MLFMA_CUDA(cudaMemcpyAsync(w, P.d_w, bytes, cudaMemcpyDeviceToHost, P.stream));
    sync_and_check(P);
    return MLFMA_OK;
  });
}

int mlfma_device_status(mlfma_plan* plan, int* status) {
  if (!plan || !plan->p || !status) return fail(MLFMA_ERR_ARG, "null argument");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    MLFMA_CUDA(cudaDeviceSynchronize());
    MLFMA_CUDA(cudaMemcpy(status, P.d_status, sizeof(int), cudaMemcpyDeviceToHost));
    return MLFMA_OK;
  });
}

int mlfma_apply_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream) {
  if (!plan || !plan->p || !x_dev || !w_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (x_dev == w_dev) return fail(MLFMA_ERR_ARG, "x and w must not alias");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::apply_device(P, static_cast<const double2*>(x_dev), static_cast<double2*>(w_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_apply_batch(mlfma_plan* plan, int n, int R, const double* x, double* w) {
  if (!plan || !plan->p || !x || !w) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (R <= 0) return fail(MLFMA_ERR_ARG, "R must be positive");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    mlfma::reserve_batch(P, R, true);
    mlfma::reserve_batch_staging(P);
    for (int g0 = 0; g0 < R; g0 += P.xb_cap) {
      const int rn = std::min(P.xb_cap, R - g0);
      const size_t bytes = static_cast<size_t>(rn) * n * sizeof(double2);
      MLFMA_CUDA(cudaMemcpyAsync(P.d_xb, x + 2 * static_cast<size_t>(g0) * n, bytes, cudaMemcpyHostToDevice,
                                 P.stream));
      mlfma::apply_batch_device(P, rn, P.d_xb, n, P.d_wb, n, P.stream);
      MLFMA_CUDA(cudaMemcpyAsync(w + 2 * static_cast<size_t>(g0) * n, P.d_wb, bytes, cudaMemcpyDeviceToHost,
                                 P.stream));
    }
    sync_and_check(P);
    return MLFMA_OK;
  });
}

int mlfma_apply_batch_device(mlfma_plan* plan, int n, int R, const void* x_dev, void* w_dev, void* stream) {
  if (!plan || !plan->p || !x_dev || !w_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (R <= 0) return fail(MLFMA_ERR_ARG, "R must be positive");
  if (x_dev == w_dev) return fail(MLFMA_ERR_ARG, "x and w must not alias");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    mlfma::reserve_batch(P, R, true);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::apply_batch_device(P, R, static_cast<const double2*>(x_dev), n, static_cast<double2*>(w_dev), n, s);
    return MLFMA_OK;
  });
}

int mlfma_apply_batch_mixed_device(mlfma_plan* plan, int n, int R, const void* x_dev, void* w_dev, void* stream) {
  if (!plan || !plan->p || !x_dev || !w_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (R <= 0) return fail(MLFMA_ERR_ARG, "R must be positive");
  if (x_dev == w_dev) return fail(MLFMA_ERR_ARG, "x and w must not alias");
  if (!device_plan(plan) || plan->p->precision != 1)
    return fail(MLFMA_ERR_UNSUPPORTED, "plan was not created with MLFMA_PREC_MIXED on a device");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    mlfma::reserve_batch(P, R, false);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::apply_batch_mixed_device(P, R, static_cast<const double2*>(x_dev), n, static_cast<double2*>(w_dev), n, s);
    return MLFMA_OK;
  });
}

int mlfma_profile(mlfma_plan* plan, int on) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  plan->p->prof.on = on != 0;
  plan->p->prof.used = 0;
  return MLFMA_OK;
}

int mlfma_profile_read(mlfma_plan* plan, double* stage_ms, int* applies) {
  if (!plan || !plan->p || !stage_ms) return fail(MLFMA_ERR_ARG, "null argument");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    MLFMA_CUDA(cudaSetDevice(plan->p->device));
    const int n = mlfma::read_stage_times(*plan->p, stage_ms);
    if (applies) *applies = n;
    return MLFMA_OK;
  });
}

namespace {
struct TuningKey {
  const char* name;
  int mlfma::Tuning::*field;
  int count;  // values 0 .. count-1
};
constexpr TuningKey kTuningKeys[] = {
    {"m2l.variant", &mlfma::Tuning::m2l_variant, 9},
    {"m2l.pair_warps", &mlfma::Tuning::m2l_pair_warps, 3},
    {"up.variant", &mlfma::Tuning::up_variant, 4},
    {"up.threads", &mlfma::Tuning::up_threads, 3},
    {"l2l.variant", &mlfma::Tuning::l2l_variant, 2},
    {"agg.variant", &mlfma::Tuning::agg_variant, 2},
    {"leaf.variant", &mlfma::Tuning::leaf_variant, 2},
    {"batch_tc.variant", &mlfma::Tuning::batch_tc, 2},
    {"batch_tree.variant", &mlfma::Tuning::batch_tree, 2},
    {"apply.graph", &mlfma::Tuning::graph, 2},
};
const TuningKey* find_key(const char* key) {
  for (const TuningKey& k : kTuningKeys)
    if (std::string(key) == k.name) return &k;
  return nullptr;
}
}  // namespace

int mlfma_set_tuning(mlfma_plan* plan, const char* key, int value) {
  if (!plan || !plan->p || !key) return fail(MLFMA_ERR_ARG, "null argument");
  const TuningKey* k = find_key(key);
  if (!k) return fail(MLFMA_ERR_ARG, std::string("unknown tuning key: ") + key);
  if (value < 0 || value >= k->count)
    return fail(MLFMA_ERR_ARG, std::string(key) + " must be in [0, " + std::to_string(k->count - 1) + "]");
  plan->p->tuning.*(k->field) = value;
  if (device_plan(plan)) mlfma::clear_graphs(*plan->p);
  return MLFMA_OK;
}

int mlfma_get_tuning(const mlfma_plan* plan, const char* key) {
  if (!plan || !plan->p || !key) return fail(MLFMA_ERR_ARG, "null argument");
  const TuningKey* k = find_key(key);
  if (!k) return fail(MLFMA_ERR_ARG, std::string("unknown tuning key: ") + key);
  return plan->p->tuning.*(k->field);
}

int mlfma_autotune(mlfma_plan* plan, int applies, double* variant_ms) {
  if (!plan || !plan->p || applies <= 0) return fail(MLFMA_ERR_ARG, "null plan or applies <= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaEvent_t e0, e1;
    MLFMA_CUDA(cudaEventCreate(&e0));
    MLFMA_CUDA(cudaEventCreate(&e1));
    MLFMA_CUDA(cudaMemsetAsync(P.d_x, 0, 2 * static_cast<size_t>(P.N) * sizeof(double2), P.stream));
    const bool prof = P.prof.on;
    P.prof.on = false;
    auto time_apply = [&] {
      mlfma::apply_device(P, P.d_x, P.d_w, P.stream);  // warm-up
      MLFMA_CUDA(cudaEventRecord(e0, P.stream));
      for (int i = 0; i < applies; ++i) mlfma::apply_device(P, P.d_x, P.d_w, P.stream);
      MLFMA_CUDA(cudaEventRecord(e1, P.stream));
      MLFMA_CUDA(cudaEventSynchronize(e1));
      sync_and_check(P);
      float ms = 0.f;
      MLFMA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return static_cast<double>(ms) / applies;
    };
    // one key at a time, the others held at their current (best so far) value
    int slot = 0;
    for (const TuningKey& k : kTuningKeys) {
      if (k.field == &mlfma::Tuning::batch_tc || k.field == &mlfma::Tuning::batch_tree) {  // no effect on the single apply timed here
        if (variant_ms)
          for (int v = 0; v < k.count; ++v) variant_ms[slot + v] = -1.0;
        slot += k.count;
        continue;
      }
      double best = 1e300;
      int best_v = P.tuning.*(k.field);
      for (int v = 0; v < k.count; ++v) {
        P.tuning.*(k.field) = v;
        mlfma::clear_graphs(P);
        const double per = time_apply();
        if (variant_ms) variant_ms[slot + v] = per;
        if (per < best) {
          best = per;
          best_v = v;
        }
      }
      P.tuning.*(k.field) = best_v;
      mlfma::clear_graphs(P);
      slot += k.count;
    }
    P.prof.on = prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return MLFMA_OK;
  });
}

int mlfma_gmres(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr, double tol_abs,
                double tol_rel, mlfma_solve_stats* stats, double* history, int history_cap) {
  if (!plan || !plan->p || !x || !rhs) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (mr <= 0 || itr_max < 0) return fail(MLFMA_ERR_ARG, "mr must be positive, itr_max non-negative");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::SolveStats st;
    std::vector<double> hist;
    const bool ok = mlfma::gmres_solve(*plan->p, x, rhs, itr_max, mr, tol_abs, tol_rel, st, hist);
    if (stats) {
      stats->iterations = st.iterations;
      stats->restarts = st.restarts;
      stats->matvecs = st.matvecs;
      stats->converged = ok ? 1 : 0;
      stats->rel_residual = st.rel_residual;
      stats->seconds = st.seconds;
      stats->history_len = static_cast<int>(std::min<size_t>(hist.size(), history ? history_cap : 0));
      stats->near_products = 0;
    }
    if (history)
      for (int i = 0; i < history_cap && i < static_cast<int>(hist.size()); ++i) history[i] = hist[i];
    return ok ? MLFMA_OK : MLFMA_ERR_NOT_CONVERGED;
  });
}

int mlfma_fgmres(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr, double tol_abs,
                 double tol_rel, int inner_its, mlfma_solve_stats* stats, double* history, int history_cap) {
  if (!plan || !plan->p || !x || !rhs) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (mr <= 0 || mr > 63 || itr_max < 0 || inner_its < 0 || inner_its > 63)
    return fail(MLFMA_ERR_ARG, "need 1 <= mr <= 63, 0 <= inner_its <= 63, itr_max >= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::SolveStats st;
    std::vector<double> hist;
    const bool ok = mlfma::fgmres_solve(*plan->p, x, rhs, itr_max, mr, tol_abs, tol_rel, inner_its, st, hist);
    if (stats) {
      stats->iterations = st.iterations;
      stats->restarts = st.restarts;
      stats->matvecs = st.matvecs;
      stats->converged = ok ? 1 : 0;
      stats->rel_residual = st.rel_residual;
      stats->seconds = st.seconds;
      stats->history_len = static_cast<int>(std::min<size_t>(hist.size(), history ? history_cap : 0));
      stats->near_products = st.near_products;
    }
    if (history)
      for (int i = 0; i < history_cap && i < static_cast<int>(hist.size()); ++i) history[i] = hist[i];
    return ok ? MLFMA_OK : MLFMA_ERR_NOT_CONVERGED;
  });
}

int mlfma_fgmres_batch(mlfma_plan* plan, int n, int R, double* x, const double* rhs, int itr_max, int mr,
                       double tol_abs, double tol_rel, int inner_its, mlfma_solve_stats* stats) {
  if (!plan || !plan->p || !x || !rhs) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (R <= 0) return fail(MLFMA_ERR_ARG, "R must be positive");
  if (mr <= 0 || mr > 63 || itr_max < 0 || inner_its < 0 || inner_its > 63)
    return fail(MLFMA_ERR_ARG, "need 1 <= mr <= 63, 0 <= inner_its <= 63, itr_max >= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    std::vector<mlfma::SolveStats> st;
    std::vector<std::vector<double>> hist;
    double seconds = 0.0;
    const std::vector<char> ok =
        mlfma::fgmres_batch_solve(*plan->p, R, x, rhs, itr_max, mr, tol_abs, tol_rel, inner_its, st, hist, seconds);
    bool all = true;
    for (int q = 0; q < R; ++q) {
      all = all && ok[q];
      if (stats) {
        stats[q].iterations = st[q].iterations;
        stats[q].restarts = st[q].restarts;
        stats[q].matvecs = st[q].matvecs;
        stats[q].converged = ok[q] ? 1 : 0;
        stats[q].rel_residual = st[q].rel_residual;
        stats[q].seconds = st[q].seconds;
        stats[q].history_len = 0;
        stats[q].near_products = st[q].near_products;
      }
    }
    return all ? MLFMA_OK : MLFMA_ERR_NOT_CONVERGED;
  });
}

namespace {
bool mixed_plan(const mlfma_plan* plan) { return device_plan(plan) && plan->p->precision == 1; }
void fill_stats(mlfma_solve_stats* out, const mlfma::SolveStats& st, bool ok, int history_len) {
  out->iterations = st.iterations;
  out->restarts = st.restarts;
  out->matvecs = st.matvecs;
  out->converged = ok ? 1 : 0;
  out->rel_residual = st.rel_residual;
  out->seconds = st.seconds;
  out->history_len = history_len;
  out->near_products = st.near_products;
}
}  // namespace

int mlfma_apply_mixed(mlfma_plan* plan, int n, const double* x, double* w) {
  if (!plan || !plan->p || !x || !w) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (!mixed_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan was not created with MLFMA_PREC_MIXED on a device");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    const size_t bytes = static_cast<size_t>(n) * sizeof(double2);
    MLFMA_CUDA(cudaMemcpyAsync(P.d_x, x, bytes, cudaMemcpyHostToDevice, P.stream));
    mlfma::apply_mixed_device(P, P.d_x, P.d_w, P.stream);
    MLFMA_CUDA(cudaMemcpyAsync(w, P.d_w, bytes, cudaMemcpyDeviceToHost, P.stream));
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    return MLFMA_OK;
  });
}

int mlfma_apply_mixed_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream) {
  if (!plan || !plan->p || !x_dev || !w_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (x_dev == w_dev) return fail(MLFMA_ERR_ARG, "x and w must not alias");
  if (!mixed_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan was not created with MLFMA_PREC_MIXED on a device");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::apply_mixed_device(P, static_cast<const double2*>(x_dev), static_cast<double2*>(w_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_solve_mixed(mlfma_plan* plan, int n, double* x, const double* rhs, int itr_max, int mr, double tol_abs,
                      double tol_rel, int inner_its, int refine_max, mlfma_solve_stats* stats, double* history,
                      int history_cap) {
  if (!plan || !plan->p || !x || !rhs) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (mr <= 0 || mr > 63 || itr_max < 0 || inner_its < 0 || inner_its > 63 || refine_max < 0)
    return fail(MLFMA_ERR_ARG, "need 1 <= mr <= 63, 0 <= inner_its <= 63, itr_max >= 0, refine_max >= 0");
  if (!mixed_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan was not created with MLFMA_PREC_MIXED on a device");
  return guarded([&] {
    mlfma::SolveStats st;
    std::vector<double> hist;
    const bool ok =
        mlfma::mixed_solve(*plan->p, x, rhs, itr_max, mr, tol_abs, tol_rel, inner_its, refine_max, st, hist);
    const int len = static_cast<int>(std::min<size_t>(hist.size(), history ? history_cap : 0));
    if (stats) fill_stats(stats, st, ok, len);
    for (int i = 0; i < len; ++i) history[i] = hist[i];
    return ok ? MLFMA_OK : MLFMA_ERR_NOT_CONVERGED;
  });
}

int mlfma_solve_mixed_batch(mlfma_plan* plan, int n, int R, double* x, const double* rhs, int itr_max, int mr,
                            double tol_abs, double tol_rel, int inner_its, int refine_max, mlfma_solve_stats* stats) {
  if (!plan || !plan->p || !x || !rhs) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (R <= 0) return fail(MLFMA_ERR_ARG, "R must be positive");
  if (mr <= 0 || mr > 63 || itr_max < 0 || inner_its < 0 || inner_its > 63 || refine_max < 0)
    return fail(MLFMA_ERR_ARG, "need 1 <= mr <= 63, 0 <= inner_its <= 63, itr_max >= 0, refine_max >= 0");
  if (!mixed_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan was not created with MLFMA_PREC_MIXED on a device");
  return guarded([&] {
    std::vector<mlfma::SolveStats> st;
    double seconds = 0.0;
    const std::vector<char> ok = mlfma::mixed_batch_solve(*plan->p, R, x, rhs, itr_max, mr, tol_abs, tol_rel,
                                                          inner_its, refine_max, st, seconds);
    bool all = true;
    for (int q = 0; q < R; ++q) {
      all = all && ok[q];
      if (stats) fill_stats(&stats[q], st[q], ok[q], 0);
    }
    return all ? MLFMA_OK : MLFMA_ERR_NOT_CONVERGED;
  });
}

int mlfma_apply_near_device(mlfma_plan* plan, int n, const void* x_dev, void* w_dev, void* stream) {
  if (!plan || !plan->p || !x_dev || !w_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (x_dev == w_dev) return fail(MLFMA_ERR_ARG, "x and w must not alias");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::near_apply(P, static_cast<const double2*>(x_dev), static_cast<double2*>(w_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_near_precondition_device(mlfma_plan* plan, int n, int inner_its, const void* v_dev, void* z_dev,
                                   void* stream) {
  if (!plan || !plan->p || !v_dev || !z_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (v_dev == z_dev) return fail(MLFMA_ERR_ARG, "v and z must not alias");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::near_precondition(P, inner_its, static_cast<const double2*>(v_dev), static_cast<double2*>(z_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_lp_param_count(void) { return mlfma::kLpParams; }

int mlfma_lp_forward_device(mlfma_plan* plan, int n, const float* params_dev, const void* v_dev, const void* z_dev,
                            void* y_dev, void* stream) {
  if (!plan || !plan->p || !v_dev || !z_dev || !y_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    const __nv_bfloat16* w = nullptr;
    if (params_dev) {
      __nv_bfloat16* ws = mlfma::lp_scratch_weights(P);
      mlfma::lp_to_bf16(params_dev, ws, mlfma::kLpParams, s);
      w = ws;
    } else {
      w = mlfma::lp_attached(P);
      if (!w) throw std::invalid_argument("no parameters given and no network attached");
    }
    mlfma::lp_forward(P, w, static_cast<const double2*>(v_dev), static_cast<const double2*>(z_dev),
                      static_cast<double2*>(y_dev), true, s);
    return MLFMA_OK;
  });
}

int mlfma_lp_backward_device(mlfma_plan* plan, int n, const float* params_dev, const void* gy_dev, float* grad_dev,
                             void* stream) {
  if (!plan || !plan->p || !params_dev || !gy_dev || !grad_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    __nv_bfloat16* ws = mlfma::lp_scratch_weights(P);
    mlfma::lp_to_bf16(params_dev, ws, mlfma::kLpParams, s);
    mlfma::lp_backward(P, ws, nullptr, nullptr, static_cast<const double2*>(gy_dev), grad_dev, nullptr, s);
    return MLFMA_OK;
  });
}

int mlfma_lp_loss_grad_device(mlfma_plan* plan, int n, const float* params_dev, const void* v_dev, const void* z_dev,
                              const void* e_dev, void* y_dev, float* grad_dev, float* loss_dev, void* stream) {
  if (!plan || !plan->p || !params_dev || !v_dev || !z_dev || !e_dev || !y_dev || !grad_dev || !loss_dev)
    return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N) return fail(MLFMA_ERR_ARG, "n must be 2N");
  if (y_dev == v_dev || y_dev == z_dev || y_dev == e_dev) return fail(MLFMA_ERR_ARG, "y must not alias v, z or e");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    __nv_bfloat16* ws = mlfma::lp_scratch_weights(P);
    mlfma::lp_to_bf16(params_dev, ws, mlfma::kLpParams, s);
    mlfma::lp_forward(P, ws, static_cast<const double2*>(v_dev), static_cast<const double2*>(z_dev),
                      static_cast<double2*>(y_dev), true, s);
    mlfma::lp_backward(P, ws, static_cast<const double2*>(y_dev), static_cast<const double2*>(e_dev), nullptr,
                       grad_dev, loss_dev, s);
    return MLFMA_OK;
  });
}

int mlfma_lp_adam_device(int nparams, float* params_dev, const float* grad_dev, float* m_dev, float* v_dev, float lr,
                         float beta1, float beta2, float eps, int step, float grad_scale, void* stream) {
  if (nparams <= 0 || !params_dev || !grad_dev || !m_dev || !v_dev) return fail(MLFMA_ERR_ARG, "null argument");
  if (step < 1) return fail(MLFMA_ERR_ARG, "step counts from 1");
  return guarded([&] {
    mlfma::lp_adam(nparams, params_dev, grad_dev, m_dev, v_dev, lr, beta1, beta2, eps, step, grad_scale,
                   static_cast<cudaStream_t>(stream));
    return MLFMA_OK;
  });
}

int mlfma_lp_attach(mlfma_plan* plan, const float* params, int nparams) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  if (nparams != 0 && (!params || nparams != mlfma::kLpParams))
    return fail(MLFMA_ERR_ARG, "nparams must be 0 or mlfma_lp_param_count()");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    MLFMA_CUDA(cudaSetDevice(P.device));
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    mlfma::lp_attach(P, params, nparams);
    return MLFMA_OK;
  });
}

int mlfma_rhs_pmchwt(mlfma_plan* plan, const double kinc[3], const double einc[3], const double hinc[3],
                     double* V) {
  if (!plan || !plan->p || !kinc || !einc || !hinc || !V) return fail(MLFMA_ERR_ARG, "null argument");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::rhs_pmchwt(*plan->p, kinc, einc, hinc, V);
    return MLFMA_OK;
  });
}

int mlfma_rcs_pmchwt(mlfma_plan* plan, const double* I, int n_angles, const double* theta_deg,
                     const double* phi_deg, double* field, double* rcs_db) {
  if (!plan || !plan->p || !I || !theta_deg || !phi_deg || n_angles < 0)
    return fail(MLFMA_ERR_ARG, "null argument");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::rcs_pmchwt(*plan->p, I, n_angles, theta_deg, phi_deg, field, rcs_db);
    return MLFMA_OK;
  });
}

int mlfma_rcs_pmchwt_noalloc(mlfma_plan* plan, const void* I_dev, int n_angles, const double* theta_deg,
                              const double* phi_deg, void* field_dev, void* stream) {
  if (!plan || !plan->p || !I_dev || !field_dev || (n_angles > 0 && (!theta_deg || !phi_deg)))
    return fail(MLFMA_ERR_ARG, "null argument");
  if (n_angles < 0 || n_angles > mlfma::rcs_noalloc_max_angles())
    return fail(MLFMA_ERR_ARG, "n_angles must be between 0 and " + std::to_string(mlfma::rcs_noalloc_max_angles()) +
                                   " (size of the fixed angle scratch)");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::rcs_pmchwt_noalloc(P, static_cast<const double2*>(I_dev), n_angles, theta_deg, phi_deg,
                              static_cast<double2*>(field_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_rcs_noalloc_max_angles(void) { return mlfma::rcs_noalloc_max_angles(); }

int mlfma_rhs_pmchwt_batch_device(mlfma_plan* plan, int n, int R, const double* kinc, const double* einc,
                                  const double* hinc, void* V_dev, void* stream) {
  if (!plan || !plan->p || (R > 0 && (!kinc || !einc || !hinc || !V_dev))) return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N || R < 0) return fail(MLFMA_ERR_ARG, "n must be 2N and R >= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::rhs_pmchwt_batch(P, R, kinc, einc, hinc, static_cast<double2*>(V_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_rcs_pmchwt_batch_device(mlfma_plan* plan, int n, int R, const void* I_dev, int n_angles,
                                  const double* theta_deg, const double* phi_deg, void* field_dev, void* stream) {
  if (!plan || !plan->p || (R > 0 && n_angles > 0 && (!I_dev || !theta_deg || !phi_deg || !field_dev)))
    return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N || R < 0 || n_angles < 0) return fail(MLFMA_ERR_ARG, "n must be 2N, R and n_angles >= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::rcs_pmchwt_batch(P, R, static_cast<const double2*>(I_dev), n_angles, theta_deg, phi_deg,
                            static_cast<double2*>(field_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_rcs_pmchwt_mono_device(mlfma_plan* plan, int n, int R, const void* I_dev, const double* theta_deg,
                                 const double* phi_deg, void* field_dev, void* stream) {
  if (!plan || !plan->p || (R > 0 && (!I_dev || !theta_deg || !phi_deg || !field_dev)))
    return fail(MLFMA_ERR_ARG, "null argument");
  if (n != 2 * plan->p->N || R < 0) return fail(MLFMA_ERR_ARG, "n must be 2N and R >= 0");
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  return guarded([&] {
    mlfma::Plan& P = *plan->p;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : P.stream;
    mlfma::rcs_pmchwt_mono(P, R, static_cast<const double2*>(I_dev), theta_deg, phi_deg,
                           static_cast<double2*>(field_dev), s);
    return MLFMA_OK;
  });
}

int mlfma_rcs_db(int n_angles, const double* theta_deg, const double* phi_deg, const double* field, double* rcs_db) {
  if (n_angles < 0 || (n_angles > 0 && (!theta_deg || !phi_deg || !field || !rcs_db)))
    return fail(MLFMA_ERR_ARG, "null argument or negative count");
  mlfma::rcs_db(n_angles, theta_deg, phi_deg, field, rcs_db);
  return MLFMA_OK;
}

int mlfma_get_rwgs(const mlfma_plan* plan, int* face_pos, int* face_neg, int* free_pos, int* free_neg,
                   int* edge_a, int* edge_b, double* length, double* mid) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Plan& P = *plan->p;
  const mlfma::Rwg& R = P.rwg;
  const mlfma::Mesh& M = P.mesh;
  for (int i = 0; i < P.N; ++i) {
    if (face_pos) face_pos[i] = M.face_id[R.fpos[i]];
    if (face_neg) face_neg[i] = M.face_id[R.fneg[i]];
    if (free_pos) free_pos[i] = M.point_id[R.free_pos[i]];
    if (free_neg) free_neg[i] = M.point_id[R.free_neg[i]];
    if (edge_a) edge_a[i] = M.point_id[R.ea[i]];
    if (edge_b) edge_b[i] = M.point_id[R.eb[i]];
    if (length) length[i] = R.len[i];
    if (mid)
      for (int a = 0; a < 3; ++a) mid[3 * i + a] = R.mid[3 * i + a];
  }
  return MLFMA_OK;
}

long long mlfma_get_level(const mlfma_plan* plan, int level, unsigned long long* morton, double* center) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Plan& P = *plan->p;
  if (level < 0 || level > P.maxL) return fail(MLFMA_ERR_ARG, "level out of range");
  const mlfma::Level& L = P.tree.lv[level];
  for (int b = 0; b < L.size(); ++b) {
    if (morton) morton[b] = L.code[b];
    if (center)
      for (int a = 0; a < 3; ++a) center[3 * b + a] = L.center[3 * b + a];
  }
  return L.size();
}

long long mlfma_get_level_lists(const mlfma_plan* plan, int level, int* near_ptr, int* near_idx, int* far_ptr,
                                int* far_idx, int* far_off) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Plan& P = *plan->p;
  if (level < 0 || level > P.maxL) return fail(MLFMA_ERR_ARG, "level out of range");
  const mlfma::Level& L = P.tree.lv[level];
  auto cp = [](const std::vector<int>& v, int* o) {
    if (o) std::copy(v.begin(), v.end(), o);
  };
  cp(L.near_ptr, near_ptr);
  cp(L.near_idx, near_idx);
  cp(L.far_ptr, far_ptr);
  cp(L.far_idx, far_idx);
  cp(L.far_off, far_off);
  return static_cast<long long>(L.far_idx.size());
}

long long mlfma_get_leaf_rwgs(const mlfma_plan* plan, int* leaf_ptr, int* leaf_rwg) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Tree& T = plan->p->tree;
  if (leaf_ptr) std::copy(T.leaf_ptr.begin(), T.leaf_ptr.end(), leaf_ptr);
  if (leaf_rwg) std::copy(T.leaf_rwg.begin(), T.leaf_rwg.end(), leaf_rwg);
  return static_cast<long long>(T.leaf_ptr.size()) - 1;
}

int mlfma_get_grid(const mlfma_plan* plan, int medium, int level, double* theta, double* phi, double* wtheta,
                   double* wphi) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Plan& P = *plan->p;
  if (medium < 1 || medium > 2 || level < 2 || level > P.maxL) return fail(MLFMA_ERR_ARG, "range");
  const mlfma::Grid& g = P.ml[medium - 1][level].grid;
  if (theta) std::copy(g.theta.begin(), g.theta.end(), theta);
  if (phi) std::copy(g.phi.begin(), g.phi.end(), phi);
  if (wtheta) std::copy(g.wth.begin(), g.wth.end(), wtheta);
  if (wphi) *wphi = g.wph;
  return g.L;
}

int mlfma_get_interp(const mlfma_plan* plan, int medium, int level, int* tidx, double* lt, int* pidx,
                     double* lp) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  const mlfma::Plan& P = *plan->p;
  if (medium < 1 || medium > 2 || level < 2 || level >= P.maxL) return fail(MLFMA_ERR_ARG, "range");
  const mlfma::Interp& I = P.ml[medium - 1][level].interp;
  if (tidx) std::copy(I.tidx.begin(), I.tidx.end(), tidx);
  if (lt) std::copy(I.lt.begin(), I.lt.end(), lt);
  if (pidx) std::copy(I.pidx.begin(), I.pidx.end(), pidx);
  if (lp) std::copy(I.lp.begin(), I.lp.end(), lp);
  return MLFMA_OK;
}

long long mlfma_get_stage(mlfma_plan* plan, int which, int medium, int level, double* out) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  mlfma::Plan& P = *plan->p;
  if (medium < 1 || medium > 2 || level < 2 || level > P.maxL || which < 0 || which > 1)
    return fail(MLFMA_ERR_ARG, "range");
  const mlfma::MediumLevel& M = P.ml[medium - 1][level];
  const long long count = static_cast<long long>(P.lv[level].B) * 6 * M.K;
  if (!out) return count;
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  const int st = guarded([&] {
    MLFMA_CUDA(cudaSetDevice(P.device));
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    MLFMA_CUDA(cudaMemcpy(out, which == 0 ? M.S : M.Bm, count * sizeof(double2), cudaMemcpyDeviceToHost));
    return 0;
  });
  return st == 0 ? count : st;
}

long long mlfma_get_pattern(mlfma_plan* plan, int medium, int which, double* out) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  mlfma::Plan& P = *plan->p;
  if (medium < 1 || medium > 2 || which < 0 || which > 1) return fail(MLFMA_ERR_ARG, "range");
  const int K = P.ml[medium - 1][P.maxL].K;
  const long long count = static_cast<long long>(P.N) * K * 3;
  if (!out) return count;
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  int st = guarded([&] {
    MLFMA_CUDA(cudaSetDevice(P.device));
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    std::vector<double2> buf(static_cast<size_t>(count));
    MLFMA_CUDA(cudaMemcpy(buf.data(), which == 0 ? P.d_Vs[medium - 1] : P.d_Vf[medium - 1],
                          count * sizeof(double2), cudaMemcpyDeviceToHost));
    // device [leaf order][3][K] -> [rwg id][K][3]
    for (int r = 0; r < P.N; ++r) {
      const int id = P.tree.leaf_rwg[r];
      for (int c = 0; c < 3; ++c)
        for (int k = 0; k < K; ++k) {
          const double2 v = buf[(static_cast<size_t>(r) * 3 + c) * K + k];
          const size_t o = (static_cast<size_t>(id) * K + k) * 3 + c;
          out[2 * o] = v.x;
          out[2 * o + 1] = v.y;
        }
    }
    return 0;
  });
  return st == 0 ? count : st;
}

long long mlfma_get_transfer(mlfma_plan* plan, int medium, int level, int* offsets, double* tf) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  mlfma::Plan& P = *plan->p;
  if (medium < 1 || medium > 2 || level < 2 || level > P.maxL) return fail(MLFMA_ERR_ARG, "range");
  const mlfma::MediumLevel& M = P.ml[medium - 1][level];
  const long long count = static_cast<long long>(M.nvec) * M.K;
  if (offsets)
    for (int v = 0; v < M.nvec; ++v) {
      int dx, dy, dz;
      mlfma::decode_offset(M.vec_off[v], dx, dy, dz);
      offsets[3 * v] = dx;
      offsets[3 * v + 1] = dy;
      offsets[3 * v + 2] = dz;
    }
  if (!tf) return count;
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  int st = guarded([&] {
    MLFMA_CUDA(cudaSetDevice(P.device));
    std::vector<double> rhat;
    std::vector<int> hoff, hL;
    std::vector<double2> h2;
    P.tf_inputs(medium - 1, level, rhat, hoff, hL, h2);
    double2* tmp = nullptr;
    MLFMA_CUDA(cudaMalloc(&tmp, std::max<long long>(count, 1) * sizeof(double2)));
    mlfma::launch_transfer(P, medium - 1, level, rhat, hoff, hL, h2, false, tmp, P.stream);
    cudaError_t e = cudaMemcpy(tf, tmp, count * sizeof(double2), cudaMemcpyDeviceToHost);
    cudaFree(tmp);
    MLFMA_CUDA(e);
    return 0;
  });
  return st == 0 ? count : st;
}

long long mlfma_get_near(mlfma_plan* plan, int* target, int* source, double* z11, double* z12, double* z22) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  mlfma::Plan& P = *plan->p;
  const mlfma::Tree& T = P.tree;
  const int B = T.lv[P.maxL].size();
  if (target || source) {
    long long e = 0;
    for (int b = 0; b < B; ++b)
      for (int t = T.leaf_ptr[b]; t < T.leaf_ptr[b + 1]; ++t)
        for (int j = P.h_near_sptr[b]; j < P.h_near_sptr[b + 1]; ++j, ++e) {
          if (target) target[e] = T.leaf_rwg[t];
          if (source) source[e] = P.h_near_src[j];
        }
  }
  if (!z11 && !z12 && !z22) return P.near_pairs;
  if (!device_plan(plan)) return fail(MLFMA_ERR_UNSUPPORTED, "plan has no device operator");
  int st = guarded([&] {
    MLFMA_CUDA(cudaSetDevice(P.device));
    MLFMA_CUDA(cudaStreamSynchronize(P.stream));
    std::vector<double2> buf(3 * static_cast<size_t>(P.near_pairs));
    MLFMA_CUDA(cudaMemcpy(buf.data(), P.d_near_z, buf.size() * sizeof(double2), cudaMemcpyDeviceToHost));
    for (long long e = 0; e < P.near_pairs; ++e) {
      double* outs[3] = {z11, z12, z22};
      for (int q = 0; q < 3; ++q)
        if (outs[q]) {
          outs[q][2 * e] = buf[3 * e + q].x;
          outs[q][2 * e + 1] = buf[3 * e + q].y;
        }
    }
    return 0;
  });
  return st == 0 ? P.near_pairs : st;
}

long long mlfma_get_near_same_triangle(mlfma_plan* plan, int* target, int* source, double* z12) {
  if (!plan || !plan->p) return fail(MLFMA_ERR_ARG, "null plan");
  mlfma::Plan& P = *plan->p;
  long long count = 0;
  int st = guarded([&] {
    std::vector<long long> pos;
    std::vector<int> tgt, src;
    mlfma::same_triangle_pairs(P.rwg, P.tree, P.h_near_sptr, P.h_near_src, P.h_near_zoff, pos, tgt, src);
    count = static_cast<long long>(pos.size());
    for (long long i = 0; i < count; ++i) {
      if (target) target[i] = tgt[i];
      if (source) source[i] = src[i];
    }
    if (z12) {
      std::vector<mlfma::cplx> z;
      mlfma::same_triangle_z12(P.mesh, P.rwg, P.quad, P.k1, P.k2, tgt, src, z);
      for (long long i = 0; i < count; ++i) {
        z12[2 * i] = z[i].real();
        z12[2 * i + 1] = z[i].imag();
      }
    }
    return 0;
  });
  return st == 0 ? count : st;
}

}  // extern "C"
