/*
 * Test infrastructure (oracle only): a plain-C restatement of the reference's
 * PMCHWT MLFMA matvec stages and of its restarted GMRES, operating on flat
 * tables in the reference's own layouts. It is checked against the reference
 * compiled from its sources (oracle/_ref/libmlfma_ref.so) in
 * tests/test_restatement.py, and never linked into the product.
 *
 * Layouts (complex128 = C99 double complex):
 *   patterns / workspaces  [box or RWG][K][3]   (Complex3D per direction, Code/MyStruct.h:11-22)
 *   transfer factors       [vec][K]
 *   interpolation          per parent direction: tp[9] child direction indices, w[9]
 *                          (InterpData, Code/MyStruct.h:41-57)
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ProcessMLFMM::mexp, Code/ProcessMLFMM.h:33-56: leaf aggregation S[b] += Vs[rwg] x[off + rwg]. */
void orc_mexp(int nbox, const int* rwg_ptr, const int* rwg_ids, int K, const cplx* Vs, const cplx* x, int xoff,
              cplx* S) {
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nbox; ++b) {
    cplx* s = S + (size_t)b * K * 3;
    for (int r = rwg_ptr[b]; r < rwg_ptr[b + 1]; ++r) {
      const int id = rwg_ids[r];
      const cplx xv = x[xoff + id];
      const cplx* v = Vs + (size_t)id * K * 3;
      for (int k = 0; k < 3 * K; ++k) s[k] += v[k] * xv;
    }
  }
}

/* ProcessMLFMM::m2m, Code/ProcessMLFMM.h:61-107: parent direction k gathers the
 * 9 interpolation taps of each child, weighted, times exp(-j k khat.(c_P - c_child)). */
void orc_m2m(int nparent, const int* child_ptr, const int* child_idx, const double* vec2F, int Kp, const int* tp,
             const double* w, const double* khat, cplx kw, const cplx* Sc, int Kc, cplx* Sp) {
#pragma omp parallel for schedule(dynamic)
  for (int P = 0; P < nparent; ++P) {
    for (int e = child_ptr[P]; e < child_ptr[P + 1]; ++e) {
      const int ch = child_idx[e];
      const double* d = vec2F + 3 * (size_t)e;
      const cplx* sc = Sc + (size_t)ch * Kc * 3;
      for (int k = 0; k < Kp; ++k) {
        cplx res[3] = {0, 0, 0};
        for (int t = 0; t < 9; ++t) {
          const cplx* f = sc + 3 * (size_t)tp[9 * k + t];
          for (int c = 0; c < 3; ++c) res[c] += f[c] * w[9 * k + t];
        }
        const cplx kr = kw * (d[0] * khat[3 * k] + d[1] * khat[3 * k + 1] + d[2] * khat[3 * k + 2]);
        const cplx e_ = cexp(-I * kr);
        cplx* sp = Sp + ((size_t)P * Kp + k) * 3;
        for (int c = 0; c < 3; ++c) sp[c] += e_ * res[c];
      }
    }
  }
}

/* ProcessMLFMM::m2l, Code/ProcessMLFMM.h:112-147: B[b][k] += TF[vec][k] S[src][k]
 * w_theta(k / nph) dphi over b's interaction list. */
void orc_m2l(int nbox, const int* far_ptr, const int* far_idx, const int* far_vec, int K, int nph, const cplx* TF,
             const double* wgl, double wphi, const cplx* S, cplx* B) {
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nbox; ++b) {
    cplx* bm = B + (size_t)b * K * 3;
    for (int e = far_ptr[b]; e < far_ptr[b + 1]; ++e) {
      const cplx* tf = TF + (size_t)far_vec[e] * K;
      const cplx* sm = S + (size_t)far_idx[e] * K * 3;
      for (int k = 0; k < K; ++k) {
        const double weight = wgl[k / nph] * wphi;
        for (int c = 0; c < 3; ++c) bm[3 * k + c] += tf[k] * sm[3 * k + c] * weight;
      }
    }
  }
}

/* ProcessMLFMM::l2l, Code/ProcessMLFMM.h:152-202: parent direction k, shifted by
 * exp(-j k khat.(c_child - c_P)), scattered onto the 3x3 child taps. */
void orc_l2l(int nparent, const int* child_ptr, const int* child_idx, const double* vecC, int Kp, const int* tidx,
             const int* pidx, const double* w, int nphc, const double* khat, cplx kw, const cplx* Bp, int Kc,
             cplx* Bc) {
#pragma omp parallel for schedule(dynamic)
  for (int P = 0; P < nparent; ++P) {
    for (int e = child_ptr[P]; e < child_ptr[P + 1]; ++e) {
      const double* r = vecC + 3 * (size_t)e;
      cplx* bc = Bc + (size_t)child_idx[e] * Kc * 3;
      for (int k = 0; k < Kp; ++k) {
        const cplx kr = kw * (khat[3 * k] * r[0] + khat[3 * k + 1] * r[1] + khat[3 * k + 2] * r[2]);
        const cplx e_ = cexp(-I * kr);
        const cplx* bp = Bp + ((size_t)P * Kp + k) * 3;
        for (int tt = 0; tt < 3; ++tt)
          for (int pp = 0; pp < 3; ++pp) {
            const int idx = tidx[3 * k + tt] * nphc + pidx[3 * k + pp];
            const double wg = w[9 * k + 3 * tt + pp];
            for (int c = 0; c < 3; ++c) bc[3 * idx + c] += e_ * bp[c] * wg;
          }
      }
    }
  }
}

static cplx pair_l(const cplx* V, const cplx* B, int K) {
  cplx s = 0;
  for (int k = 0; k < K; ++k) s += V[3 * k] * B[3 * k] + V[3 * k + 1] * B[3 * k + 1] + V[3 * k + 2] * B[3 * k + 2];
  return s;
}

static cplx pair_k(const cplx* V, const cplx* B, const double* khat, int K) {
  cplx s = 0;
  for (int k = 0; k < K; ++k) {
    const double a = -khat[3 * k], b = -khat[3 * k + 1], c = -khat[3 * k + 2];
    const cplx x = b * V[3 * k + 2] - c * V[3 * k + 1];
    const cplx y = c * V[3 * k] - a * V[3 * k + 2];
    const cplx z = a * V[3 * k + 1] - b * V[3 * k];
    s += x * B[3 * k] + y * B[3 * k + 1] + z * B[3 * k + 2];
  }
  return s;
}

/* Far-field testing, Code/MLFMM.cpp:285-351: eight pairings per RWG of the
 * receive patterns with the leaf incoming patterns of both media. */
void orc_farfield(int N, const int* leaf_of_rwg, int K1, int K2, const cplx* Vf1, const cplx* Vf2,
                  const double* khat1, const double* khat2, const cplx* BJ1, const cplx* BM1, const cplx* BJ2,
                  const cplx* BM2, cplx c1, cplx c2, cplx etai, cplx* w) {
#pragma omp parallel for schedule(dynamic)
  for (int id = 0; id < N; ++id) {
    const size_t b = (size_t)leaf_of_rwg[id];
    const cplx* V1 = Vf1 + (size_t)id * K1 * 3;
    const cplx* V2 = Vf2 + (size_t)id * K2 * 3;
    const cplx L1J = pair_l(V1, BJ1 + b * K1 * 3, K1), K1J = pair_k(V1, BJ1 + b * K1 * 3, khat1, K1);
    const cplx L1M = pair_l(V1, BM1 + b * K1 * 3, K1), K1M = pair_k(V1, BM1 + b * K1 * 3, khat1, K1);
    const cplx L2J = pair_l(V2, BJ2 + b * K2 * 3, K2), K2J = pair_k(V2, BJ2 + b * K2 * 3, khat2, K2);
    const cplx L2M = pair_l(V2, BM2 + b * K2 * 3, K2), K2M = pair_k(V2, BM2 + b * K2 * 3, khat2, K2);
    w[id] += c1 * L1J;
    w[id] += -c1 * K1M;
    w[N + id] += c1 * K1J;
    w[N + id] += c1 * L1M;
    w[id] += c2 * etai * L2J;
    w[id] += -c2 * K2M;
    w[N + id] += c2 * K2J;
    w[N + id] += c2 * L2M / etai;
  }
}

/* Near field, Code/MLFMM.cpp:353-366: w[i] += sum_j Z_near[i][j] x[Z_near_id[i][j]]. */
void orc_near(int n, const int* row_ptr, const int* col, const cplx* val, const cplx* x, cplx* w) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i)
    for (int j = row_ptr[i]; j < row_ptr[i + 1]; ++j) w[i] += x[col[j]] * val[j];
}

/* ------------------------------------------------------------------ GMRES */

static cplx dot_conj(int n, const cplx* a, const cplx* b) {
  cplx s = 0;
  for (int i = 0; i < n; ++i) s += conj(a[i]) * b[i];
  return s;
}

/* Code/GMRES.h:22-40 */
static void givens_make(cplx a, cplx b, cplx* c, cplx* s) {
  const double eps = 1e-16;
  if (cabs(b) < eps) {
    *c = 1.0;
    *s = 0.0;
  } else if (cabs(a) < eps) {
    *c = 0.0;
    *s = 1.0;
  } else {
    const double r = sqrt(creal(a * conj(a) + b * conj(b)));
    *c = a / r;
    *s = b / r;
  }
}

/* Code/GMRES.h:43-48 */
static void givens_apply(cplx* x, cplx* y, cplx c, cplx s) {
  const cplx t = conj(c) * *x + conj(s) * *y;
  *y = -s * *x + c * *y;
  *x = t;
}

typedef void (*orc_ax_fn)(int n, const cplx* x, cplx* w, void* ctx);

/* MGMRES::mgmres, Code/GMRES.h:65-217: modified Gram-Schmidt with one
 * re-orthogonalisation pass, complex Givens, true residual per cycle,
 * divergence abort after cycle 8. hist receives |s_{k+1}| / ||b|| per inner
 * step. Returns 1 when converged. */
int orc_gmres(int n, cplx* x, const cplx* rhs, int itr_max, int mr, double tol_abs, double tol_rel, orc_ax_fn ax,
              void* ctx, double* hist, int hist_cap, int* n_hist) {
  const double eps = 1e-16;
  cplx* r = calloc((size_t)n, sizeof(cplx));
  cplx* w = calloc((size_t)n, sizeof(cplx));
  cplx* v = calloc((size_t)n * (mr + 1), sizeof(cplx));
  cplx* h = calloc((size_t)(mr + 1) * mr, sizeof(cplx));
  cplx* cs = calloc((size_t)mr, sizeof(cplx));
  cplx* sn = calloc((size_t)mr, sizeof(cplx));
  cplx* s = calloc((size_t)mr + 1, sizeof(cplx));
  cplx* y = calloc((size_t)mr, sizeof(cplx));
  int total = 0, nh = 0, ok = 0;
  ax(n, x, w, ctx);
  for (int i = 0; i < n; ++i) r[i] = rhs[i] - w[i];
  double bnorm = sqrt(creal(dot_conj(n, rhs, rhs)));
  if (bnorm < eps) bnorm = 1.0;
  double rnorm = sqrt(creal(dot_conj(n, r, r)));
  double error = rnorm / bnorm;
  if (error < tol_rel || error < tol_abs) {
    ok = 1;
    goto done;
  }
  for (int cycle = 1; cycle <= itr_max; ++cycle) {
    for (int i = 0; i < n; ++i) v[i] = r[i] / rnorm;
    memset(s, 0, sizeof(cplx) * (mr + 1));
    s[0] = rnorm;
    memset(h, 0, sizeof(cplx) * (mr + 1) * mr);
    memset(cs, 0, sizeof(cplx) * mr);
    memset(sn, 0, sizeof(cplx) * mr);
    int k_used = 0;
    for (int k = 0; k < mr; ++k) {
      if (total >= itr_max) break;
      total++;
      k_used = k + 1;
      ax(n, v + (size_t)k * n, w, ctx);
      for (int j = 0; j <= k; ++j) {
        h[j + k * (mr + 1)] = dot_conj(n, v + (size_t)j * n, w);
        for (int i = 0; i < n; ++i) w[i] -= h[j + k * (mr + 1)] * v[i + (size_t)j * n];
      }
      for (int j = 0; j <= k; ++j) {
        const cplx t = dot_conj(n, v + (size_t)j * n, w);
        h[j + k * (mr + 1)] += t;
        for (int i = 0; i < n; ++i) w[i] -= t * v[i + (size_t)j * n];
      }
      const double hn = sqrt(creal(dot_conj(n, w, w)));
      h[k + 1 + k * (mr + 1)] = hn;
      if (hn < eps * rnorm) break;
      for (int i = 0; i < n; ++i) v[i + (size_t)(k + 1) * n] = w[i] / hn;
      for (int j = 0; j < k; ++j) givens_apply(&h[j + k * (mr + 1)], &h[j + 1 + k * (mr + 1)], cs[j], sn[j]);
      givens_make(h[k + k * (mr + 1)], h[k + 1 + k * (mr + 1)], &cs[k], &sn[k]);
      givens_apply(&h[k + k * (mr + 1)], &h[k + 1 + k * (mr + 1)], cs[k], sn[k]);
      h[k + 1 + k * (mr + 1)] = 0.0;
      givens_apply(&s[k], &s[k + 1], cs[k], sn[k]);
      error = cabs(s[k + 1]) / bnorm;
      if (nh < hist_cap) hist[nh++] = error;
      if (error < tol_rel || error < tol_abs) break;
    }
    const int m = k_used < mr ? k_used : mr;
    for (int i = m - 1; i >= 0; --i) {
      y[i] = s[i];
      for (int j = i + 1; j < m; ++j) y[i] -= h[i + j * (mr + 1)] * y[j];
      if (cabs(h[i + i * (mr + 1)]) > eps)
        y[i] /= h[i + i * (mr + 1)];
      else
        y[i] = 0.0;
    }
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < n; ++i) x[i] += y[j] * v[i + (size_t)j * n];
    ax(n, x, w, ctx);
    for (int i = 0; i < n; ++i) r[i] = rhs[i] - w[i];
    rnorm = sqrt(creal(dot_conj(n, r, r)));
    error = rnorm / bnorm;
    if (error < tol_rel || error < tol_abs) {
      ok = 1;
      goto done;
    }
    if (total >= itr_max) goto done;
    if (error > 100.0 * tol_rel && cycle > 8 && error > 1000.0 * tol_rel) goto done;
  }
done:
  if (n_hist) *n_hist = nh;
  free(r);
  free(w);
  free(v);
  free(h);
  free(cs);
  free(sn);
  free(s);
  free(y);
  return ok;
}

/* Dense matvec callback for orc_gmres: ctx = row-major complex n x n. */
void orc_dense_ax(int n, const cplx* x, cplx* w, void* ctx) {
  const cplx* A = (const cplx*)ctx;
#pragma omp parallel for
  for (int i = 0; i < n; ++i) {
    cplx s = 0;
    for (int j = 0; j < n; ++j) s += A[(size_t)i * n + j] * x[j];
    w[i] = s;
  }
}

int orc_gmres_dense(int n, const cplx* A, cplx* x, const cplx* rhs, int itr_max, int mr, double tol_abs,
                    double tol_rel, double* hist, int hist_cap, int* n_hist) {
  return orc_gmres(n, x, rhs, itr_max, mr, tol_abs, tol_rel, orc_dense_ax, (void*)A, hist, hist_cap, n_hist);
}
