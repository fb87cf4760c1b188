// Test infrastructure (oracle only) -- never linked into the product.
//
// A C-ABI driver around the reference solver CCCCl0uD/MLFMA_PMCHWT, compiled
// from the reference's own sources (see oracle/Makefile). It builds one
// dielectric PMCHWT MLFMA operator exactly the way the reference's main
// program does (Code/main.cpp:86-175: readNasData -> RWGGenerator::GenerateRWG
// -> OCTree -> MLFMM) and then exposes, for the parity tests:
//   * the matvec w = A x, re-composed from the reference's public members and
//     ProcessMLFMM stage functions in the order of the `ax` closure
//     (Code/MLFMM.cpp:246-367); the closure itself is local to
//     MLFMM::matrix_solver and cannot be called from outside;
//   * the reference's own GMRES solve (MLFMM::matrix_solver, Code/MLFMM.cpp:186);
//   * RHS::computeV_PMCHWT (Code/Vm.h:150-203) and
//     RCSUtils::calculateRCS_PMCHWT (Code/RCS.h:116-192);
//   * every setup table (RWGs, tree, angular grids, transfer factors,
//     interpolation, radiation/receive patterns, near-field rows) and the
//     per-level Sm/Bm workspaces after the last matvec;
//   * the dense MoM PMCHWT matrix (Code/Zmartix.h:467-539) for small meshes;
//   * MGMRES::mgmres (Code/GMRES.h:65-217) on a caller-supplied dense matrix.
#include "MLFMM.h"
#include "NASReader.h"
#include "RWGGenerator.h"
#include "OCTree.h"
#include "EMSource.h"
#include "GaussPoints.h"
#include "ProcessMLFMM.h"
#include "GMRES.h"
#include "Vm.h"
#include "RCS.h"
#include "Zmartix.h"
#include <boost/math/special_functions/bessel.hpp>
#include <boost/math/special_functions/legendre.hpp>

#include <omp.h>
#include <unistd.h>
#include <fcntl.h>
#include <cstdio>
#include <cstring>
#include <complex>
#include <memory>
#include <string>
#include <vector>

using cplx = std::complex<double>;

namespace {

// Redirects stdout (fd 1) into a temporary file for the lifetime of the
// object; text() returns what was written. The reference prints progress
// bars and per-iteration residuals on stdout.
struct StdoutCapture {
  int saved = -1;
  FILE* tmp = nullptr;
  explicit StdoutCapture(bool active) {
    if (!active) return;
    fflush(stdout);
    std::cout.flush();
    tmp = tmpfile();
    if (!tmp) return;
    saved = dup(1);
    dup2(fileno(tmp), 1);
  }
  std::string finish() {
    std::string out;
    if (saved < 0) return out;
    fflush(stdout);
    std::cout.flush();
    dup2(saved, 1);
    close(saved);
    saved = -1;
    long len = ftell(tmp);
    if (len > 0) {
      out.resize(static_cast<size_t>(len));
      fseek(tmp, 0, SEEK_SET);
      size_t got = fread(&out[0], 1, out.size(), tmp);
      out.resize(got);
    }
    fclose(tmp);
    tmp = nullptr;
    return out;
  }
  ~StdoutCapture() { finish(); }
};

struct RefCase {
  std::vector<Point> points;
  std::vector<FaceElement> faces;
  std::vector<RWGBase> rwgs;
  EMSource wave;
  gaussPoints gp;
  RCSExportConfig cfg;
  std::unique_ptr<OCTree> tree;
  std::unique_ptr<MLFMM> op;
  RefCase(double freq, int ngauss) : wave(freq, 0.0), gp(ngauss) {}
};

thread_local std::string g_err;

// Wavelength handed to the OCTree so that leafCoeff_ (0.3, Code/PhyConstant.h:14)
// times it equals leaf_coeff * lambda bit for bit: OCTree only uses the
// wavelength to form leafTarget = leafCoeff_ * wavelength (Code/OCTree.cpp:188).
double tree_wavelength(double lambda, double leaf_coeff) {
  const double target = leaf_coeff * lambda;
  double w = target / leafCoeff_;
  for (int i = 0; i < 64 && leafCoeff_ * w != target; ++i)
    w = (leafCoeff_ * w < target) ? std::nextafter(w, 1e300) : std::nextafter(w, -1e300);
  return w;
}

// x, w as interleaved complex128 (layout-compatible with std::complex<double>).
void recomposed_ax(MLFMM& m, const cplx* x, cplx* w) {
  const int N = m.row;
  const int L = m.maxLevel_;
  const int leafIdx = L - 2;
  for (int i = 0; i < 2 * N; ++i) w[i] = cplx(0.0, 0.0);
  const cplx etai = m.wave.etai();
  const cplx c1 = m.wave.k1() * m.wave.k1() / (16.0 * Pi * Pi);
  const cplx c2 = m.wave.k2() * m.wave.k2() / (16.0 * Pi * Pi);

  ProcessMLFMM::clearSmBm(m.Sm_J1, m.Bm_J1);
  ProcessMLFMM::clearSmBm(m.Sm_M1, m.Bm_M1);
  ProcessMLFMM::clearSmBm(m.Sm_J2, m.Bm_J2);
  ProcessMLFMM::clearSmBm(m.Sm_M2, m.Bm_M2);

  struct Pass {
    std::vector<std::vector<std::vector<Complex3D>>>* S;
    std::vector<std::vector<std::vector<Complex3D>>>* B;
    const std::vector<std::vector<Complex3D>>* V;
    int medium;
    int off;
  };
  Pass passes[4] = {{&m.Sm_J1, &m.Bm_J1, &m.Vsmi, 1, 0},
                    {&m.Sm_M1, &m.Bm_M1, &m.Vsmi, 1, N},
                    {&m.Sm_J2, &m.Bm_J2, &m.Vsmi2, 2, 0},
                    {&m.Sm_M2, &m.Bm_M2, &m.Vsmi2, 2, N}};
  for (const Pass& p : passes) {
    const bool k1 = p.medium == 1;
    const auto& kp = k1 ? m.kp_lvl_k1 : m.kp_lvl_k2;
    const auto& itp = k1 ? m.interpol_k1 : m.interpol_k2;
    const auto& tf = k1 ? m.TF : m.TF2;
    const auto& wgl = k1 ? m.WGL_k1 : m.WGL_k2;
    const auto& wphi = k1 ? m.WGL_phi_k1 : m.WGL_phi_k2;
    const auto& phi = k1 ? m.phi_level_k1 : m.phi_level_k2;
    const cplx kw = k1 ? m.wave.k1() : m.wave.k2();
    ProcessMLFMM::mexp(*p.S, m.octreeNodes_[L], *p.V, kp[0], x, p.off, L);
    ProcessMLFMM::m2m(*p.S, m.octreeNodes_, kp, itp, L, m.levelSpan, kw);
    ProcessMLFMM::m2l(*p.S, *p.B, m.octreeNodes_, tf, kp, wgl, wphi, phi, L, m.levelSpan);
    ProcessMLFMM::l2l(*p.B, m.octreeNodes_, kp, phi, itp, L, m.levelSpan, kw);
  }

  // Far-field testing: per RWG, the bilinear pairings of the receive pattern
  // with the incoming leaf pattern (L terms) and with kappa x pattern (K terms).
  auto pairL = [](const std::vector<Complex3D>& V, const std::vector<Complex3D>& B) {
    cplx s(0.0, 0.0);
    for (size_t k = 0; k < V.size(); ++k) s += V[k].x * B[k].x + V[k].y * B[k].y + V[k].z * B[k].z;
    return s;
  };
  auto pairK = [](const std::vector<Complex3D>& V, const std::vector<Complex3D>& B,
                  const std::vector<kp_Point>& kp) {
    cplx s(0.0, 0.0);
    for (size_t k = 0; k < V.size(); ++k) {
      const double a = -kp[k].x, b = -kp[k].y, c = -kp[k].z;
      const cplx cx = b * V[k].z - c * V[k].y;
      const cplx cy = c * V[k].x - a * V[k].z;
      const cplx cz = a * V[k].y - b * V[k].x;
      s += cx * B[k].x + cy * B[k].y + cz * B[k].z;
    }
    return s;
  };
  const auto& leaves = m.octreeNodes_[L];
  const int nLeaf = static_cast<int>(leaves.size());
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nLeaf; ++b) {
    OCTree::Node* nd = leaves[b];
    const auto& BJ1 = m.Bm_J1[leafIdx][b];
    const auto& BM1 = m.Bm_M1[leafIdx][b];
    const auto& BJ2 = m.Bm_J2[leafIdx][b];
    const auto& BM2 = m.Bm_M2[leafIdx][b];
    for (RWGBase* r : nd->rwgIndices) {
      const int id = r->rwgid;
      const auto& V1 = m.Vfmj[id];
      const auto& V2 = m.Vfmj2[id];
      const cplx L1J = pairL(V1, BJ1), K1J = pairK(V1, BJ1, m.kp_lvl_k1[0]);
      const cplx L1M = pairL(V1, BM1), K1M = pairK(V1, BM1, m.kp_lvl_k1[0]);
      const cplx L2J = pairL(V2, BJ2), K2J = pairK(V2, BJ2, m.kp_lvl_k2[0]);
      const cplx L2M = pairL(V2, BM2), K2M = pairK(V2, BM2, m.kp_lvl_k2[0]);
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
  // Near field: the stored rows of Z_near against x.
#pragma omp parallel for schedule(dynamic)
  for (int b = 0; b < nLeaf; ++b) {
    for (RWGBase* r : leaves[b]->rwgIndices) {
      const int id = r->rwgid;
      for (size_t j = 0; j < m.Z_near[id].size(); ++j) w[id] += x[m.Z_near_id[id][j]] * m.Z_near[id][j];
      for (size_t j = 0; j < m.Z_near[N + id].size(); ++j)
        w[N + id] += x[m.Z_near_id[N + id][j]] * m.Z_near[N + id][j];
    }
  }
}

const std::vector<std::vector<std::vector<Complex3D>>>* stage_array(MLFMM& m, int which, int pass) {
  // which: 0 = Sm, 1 = Bm; pass: 0 = J/k1, 1 = M/k1, 2 = J/k2, 3 = M/k2
  switch (which * 4 + pass) {
    case 0: return &m.Sm_J1;
    case 1: return &m.Sm_M1;
    case 2: return &m.Sm_J2;
    case 3: return &m.Sm_M2;
    case 4: return &m.Bm_J1;
    case 5: return &m.Bm_M1;
    case 6: return &m.Bm_J2;
    case 7: return &m.Bm_M2;
  }
  return nullptr;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void ref_set_threads(int n) {
  if (n > 0) {
    omp_set_dynamic(0);
    omp_set_num_threads(n);
  }
}

// Builds the operator. leaf_coeff is the leaf box edge in wavelengths.
void* ref_create(const char* nas_path, double freq, double eps_re, double eps_im, double mu_re,
                 double mu_im, double leaf_coeff, int ngauss, int quiet) {
  try {
    auto c = std::make_unique<RefCase>(freq, ngauss);
    StdoutCapture cap(quiet != 0);
    c->wave.initDielectric(cplx(eps_re, eps_im), cplx(mu_re, mu_im));
    if (readNasData(nas_path, c->points, c->faces) != 0) {
      g_err = "readNasData failed";
      return nullptr;
    }
    if (!RWGGenerator::GenerateRWG(c->faces, c->points, c->rwgs)) {
      g_err = "GenerateRWG failed";
      return nullptr;
    }
    c->tree = std::make_unique<OCTree>(c->rwgs, tree_wavelength(c->wave.wavelength(), leaf_coeff),
                                       std::string(nas_path));
    c->op = std::make_unique<MLFMM>(c->cfg, 2, 0, std::string("none"), std::string("v"),
                                    c->tree->octreeNodes_, c->tree->octreeNodesDRvec_, c->rwgs,
                                    c->tree->maxLevel_, c->gp, 1.0, c->wave);
    return c.release();
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void ref_destroy(void* h) { delete static_cast<RefCase*>(h); }

// out: [0]=N RWGs, [1]=maxLevel, [2]=levelSpan, [3]=points, [4]=faces
void ref_sizes(void* h, int* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  out[0] = c.op->row;
  out[1] = c.op->maxLevel_;
  out[2] = c.op->levelSpan;
  out[3] = static_cast<int>(c.points.size());
  out[4] = static_cast<int>(c.faces.size());
}

// Medium constants: k1, k2, eta1, eta2, etai as 5 complex values, plus lambda.
void ref_wave(void* h, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  cplx v[5] = {c.wave.k1(), c.wave.k2(), c.wave.eta1(), c.wave.eta2(), c.wave.etai()};
  for (int i = 0; i < 5; ++i) {
    out[2 * i] = v[i].real();
    out[2 * i + 1] = v[i].imag();
  }
  out[10] = c.wave.wavelength();
}

// RWG table in unknown order: face ids of T+/T-, point ids of the free
// vertices and of the common edge, edge length, edge midpoint.
void ref_rwgs(void* h, int* face_pos, int* face_neg, int* free_pos, int* free_neg, int* edge_a,
              int* edge_b, double* length, double* mid) {
  RefCase& c = *static_cast<RefCase*>(h);
  for (size_t i = 0; i < c.rwgs.size(); ++i) {
    const RWGBase& r = c.rwgs[i];
    face_pos[i] = r.positiveFace->faceId;
    face_neg[i] = r.negativeFace->faceId;
    free_pos[i] = r.freeVertexPositive->id;
    free_neg[i] = r.freeVertexNegative->id;
    edge_a[i] = r.commonEdgeVertex1->id;
    edge_b[i] = r.commonEdgeVertex2->id;
    length[i] = r.edgeLength;
    mid[3 * i] = r.edgeCenterCenter.x;
    mid[3 * i + 1] = r.edgeCenterCenter.y;
    mid[3 * i + 2] = r.edgeCenterCenter.z;
  }
}

int ref_level_boxes(void* h, int level) {
  RefCase& c = *static_cast<RefCase*>(h);
  return static_cast<int>(c.tree->octreeNodes_[level].size());
}

// Per box at `level` (reference node order): Morton code, centre, edge length,
// RWG count, near-neighbour count, interaction-list count.
void ref_level_info(void* h, int level, unsigned long long* morton, double* center, double* len,
                    int* n_rwg, int* n_near, int* n_far) {
  RefCase& c = *static_cast<RefCase*>(h);
  const auto& nodes = c.tree->octreeNodes_[level];
  for (size_t b = 0; b < nodes.size(); ++b) {
    morton[b] = nodes[b]->mortonCode;
    center[3 * b] = nodes[b]->center.x;
    center[3 * b + 1] = nodes[b]->center.y;
    center[3 * b + 2] = nodes[b]->center.z;
    len[b] = nodes[b]->cubeLength;
    n_rwg[b] = static_cast<int>(nodes[b]->rwgIndices.size());
    n_near[b] = static_cast<int>(nodes[b]->nearNeighbors.size());
    n_far[b] = static_cast<int>(nodes[b]->distantRelatives.size());
  }
}

// Lists of one box: RWG ids, Morton codes of near neighbours and of the
// interaction list, with each interaction's translation-vector id.
void ref_box_lists(void* h, int level, int box, int* rwg, unsigned long long* near_codes,
                   unsigned long long* far_codes, int* far_vec) {
  RefCase& c = *static_cast<RefCase*>(h);
  OCTree::Node* n = c.tree->octreeNodes_[level][box];
  for (size_t i = 0; i < n->rwgIndices.size(); ++i) rwg[i] = n->rwgIndices[i]->rwgid;
  for (size_t i = 0; i < n->nearNeighbors.size(); ++i) near_codes[i] = n->nearNeighbors[i]->mortonCode;
  for (size_t i = 0; i < n->distantRelatives.size(); ++i) {
    far_codes[i] = n->distantRelatives[i]->mortonCode;
    far_vec[i] = n->dRVecId.empty() ? -1 : n->dRVecId[i];
  }
}

int ref_dr_vec_count(void* h, int level) {
  RefCase& c = *static_cast<RefCase*>(h);
  return static_cast<int>(c.tree->octreeNodesDRvec_[level - 2].size());
}

void ref_dr_vecs(void* h, int level, double* xyz) {
  RefCase& c = *static_cast<RefCase*>(h);
  const auto& v = c.tree->octreeNodesDRvec_[level - 2];
  for (size_t i = 0; i < v.size(); ++i) {
    xyz[3 * i] = v[i].x;
    xyz[3 * i + 1] = v[i].y;
    xyz[3 * i + 2] = v[i].z;
  }
}

// Angular grid of medium (1 or 2) at reversed index rev (0 = leaf level):
// returns L; fills theta (L), phi (2L), theta weights (L), phi weight (1).
int ref_grid(void* h, int medium, int rev, double* theta, double* phi, double* wtheta, double* wphi) {
  RefCase& c = *static_cast<RefCase*>(h);
  MLFMM& m = *c.op;
  const auto& Ls = medium == 1 ? m.L_k1 : m.L_k2;
  const auto& th = medium == 1 ? m.theta_level_k1 : m.theta_level_k2;
  const auto& ph = medium == 1 ? m.phi_level_k1 : m.phi_level_k2;
  const auto& wg = medium == 1 ? m.WGL_k1 : m.WGL_k2;
  const auto& wp = medium == 1 ? m.WGL_phi_k1 : m.WGL_phi_k2;
  if (theta) std::copy(th[rev].begin(), th[rev].end(), theta);
  if (phi) std::copy(ph[rev].begin(), ph[rev].end(), phi);
  if (wtheta) std::copy(wg[rev].begin(), wg[rev].end(), wtheta);
  if (wphi) *wphi = wp[rev];
  return Ls[rev];
}

// Transfer factors of medium at Sm-level index lvl (0 = level 2): [vec][K] complex.
void ref_tf(void* h, int medium, int lvl, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  const auto& tf = medium == 1 ? c.op->TF : c.op->TF2;
  size_t o = 0;
  for (const auto& row : tf[lvl])
    for (const cplx& v : row) {
      out[o++] = v.real();
      out[o++] = v.imag();
    }
}

// Interpolation table of medium at index lvl (parent = level lvl+2):
// per parent direction: tIdx[3], pIdx[3], w[9].
int ref_interp(void* h, int medium, int lvl, int* tidx, int* pidx, double* w) {
  RefCase& c = *static_cast<RefCase*>(h);
  const auto& it = medium == 1 ? c.op->interpol_k1 : c.op->interpol_k2;
  const auto& tab = it[lvl];
  if (tidx) {
    for (size_t k = 0; k < tab.size(); ++k) {
      for (int a = 0; a < 3; ++a) {
        tidx[3 * k + a] = tab[k].tIdx[a];
        pidx[3 * k + a] = tab[k].pIdx[a];
      }
      for (int a = 0; a < 9; ++a) w[9 * k + a] = tab[k].w[a];
    }
  }
  return static_cast<int>(tab.size());
}

// Leaf patterns [N][K][3] complex. which: 0 = Vsmi (radiation), 1 = Vfmj (receive).
void ref_pattern(void* h, int medium, int which, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  MLFMM& m = *c.op;
  const auto& V = medium == 1 ? (which == 0 ? m.Vsmi : m.Vfmj) : (which == 0 ? m.Vsmi2 : m.Vfmj2);
  size_t o = 0;
  for (const auto& row : V)
    for (const Complex3D& v : row) {
      const cplx e[3] = {v.x, v.y, v.z};
      for (int a = 0; a < 3; ++a) {
        out[o++] = e[a].real();
        out[o++] = e[a].imag();
      }
    }
}

// Near-field rows: row lengths (2N entries).
void ref_znear_lengths(void* h, int* len) {
  RefCase& c = *static_cast<RefCase*>(h);
  for (size_t i = 0; i < c.op->Z_near.size(); ++i) len[i] = static_cast<int>(c.op->Z_near[i].size());
}

// Near-field rows concatenated: column ids and complex values.
void ref_znear(void* h, int* ids, double* vals) {
  RefCase& c = *static_cast<RefCase*>(h);
  size_t o = 0;
  for (size_t i = 0; i < c.op->Z_near.size(); ++i)
    for (size_t j = 0; j < c.op->Z_near[i].size(); ++j) {
      ids[o] = c.op->Z_near_id[i][j];
      vals[2 * o] = c.op->Z_near[i][j].real();
      vals[2 * o + 1] = c.op->Z_near[i][j].imag();
      ++o;
    }
}

// w = A x with the reference's stage functions; x, w complex128[2N].
void ref_apply(void* h, const double* x, double* w) {
  RefCase& c = *static_cast<RefCase*>(h);
  recomposed_ax(*c.op, reinterpret_cast<const cplx*>(x), reinterpret_cast<cplx*>(w));
}

// Sm (which=0) or Bm (which=1) of pass (0 J/k1, 1 M/k1, 2 J/k2, 3 M/k2) at Sm-level
// index lvl and reference box index: [K][3] complex.
int ref_stage(void* h, int which, int pass, int lvl, int box, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  const auto* arr = stage_array(*c.op, which, pass);
  const auto& v = (*arr)[lvl][box];
  if (out) {
    size_t o = 0;
    for (const Complex3D& e : v) {
      const cplx a[3] = {e.x, e.y, e.z};
      for (int q = 0; q < 3; ++q) {
        out[o++] = a[q].real();
        out[o++] = a[q].imag();
      }
    }
  }
  return static_cast<int>(v.size());
}

// The reference's GMRES through MLFMM::matrix_solver (ax = the real closure).
// Returns the captured solver log (residual history) in `log` (truncated).
void ref_solve(void* h, const double* rhs, double* x, int itr_max, int mr, double tol_abs,
               double tol_rel, char* log, int log_len) {
  RefCase& c = *static_cast<RefCase*>(h);
  const int n = 2 * c.op->row;
  std::vector<cplx> b(reinterpret_cast<const cplx*>(rhs), reinterpret_cast<const cplx*>(rhs) + n);
  StdoutCapture cap(true);
  c.op->matrix_solver(n, reinterpret_cast<cplx*>(x), b.data(), itr_max, mr, tol_abs, tol_rel);
  std::string text = cap.finish();
  if (log && log_len > 0) {
    std::strncpy(log, text.c_str(), static_cast<size_t>(log_len - 1));
    log[log_len - 1] = '\0';
  }
}

// Plane-wave excitation vector V (2N complex) for incidence (theta, phi) in
// degrees and polarisation pol (0 = V / theta-hat, 90 = H / phi-hat), through
// EMSource::initPW (Code/EMSource.cpp:34-72) and RHS::computeV_PMCHWT.
void ref_rhs(void* h, double pol, double th, double ph, double* V, double* vecs) {
  RefCase& c = *static_cast<RefCase*>(h);
  EMSource pw;
  pw.initPW(pol, th, ph);
  double kinc[3] = {pw.vW(0), pw.vW(1), pw.vW(2)};
  double einc[3] = {pw.vE(0), pw.vE(1), pw.vE(2)};
  double hinc[3] = {pw.vH(0), pw.vH(1), pw.vH(2)};
  if (vecs)
    for (int i = 0; i < 3; ++i) {
      vecs[i] = kinc[i];
      vecs[3 + i] = einc[i];
      vecs[6 + i] = hinc[i];
    }
  RHS::computeV_PMCHWT(c.rwgs, c.gp, c.wave.k1(), kinc, einc, hinc, c.op->Vm);
  for (size_t i = 0; i < c.op->Vm.size(); ++i) {
    V[2 * i] = c.op->Vm[i].real();
    V[2 * i + 1] = c.op->Vm[i].imag();
  }
}

// Scattered far field at (th, ph) degrees from currents I (2N complex):
// out[0..5] = the 3 complex Cartesian components (RCS.h:116-192);
// out[6..8] = total / theta-pol / phi-pol RCS in dBsm as the dual-static
// study forms them (Code/RCS.h:391-410) for polarisation pol.
void ref_rcs(void* h, const double* I, double pol, double th, double ph, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  const int N = c.op->row;
  const cplx* Ic = reinterpret_cast<const cplx*>(I);
  std::vector<cplx> pre(3);
  RCSUtils::calculateRCS_PMCHWT(*c.op, Ic, Ic + N, pre, c.wave.k1(), c.wave.k2(), c.wave.eta1(),
                                c.wave.eta2(), th, ph);
  for (int i = 0; i < 3; ++i) {
    out[2 * i] = pre[i].real();
    out[2 * i + 1] = pre[i].imag();
  }
  EMSource pw;
  pw.initPW(pol, th, ph);
  const double vv[3] = {pw.vTh(0), pw.vTh(1), pw.vTh(2)};
  const double vh[3] = {pw.vPh(0), pw.vPh(1), pw.vPh(2)};
  const cplx Ev = vv[0] * pre[0] + vv[1] * pre[1] + vv[2] * pre[2];
  const cplx Eh = vh[0] * pre[0] + vh[1] * pre[1] + vh[2] * pre[2];
  out[6] = 10.0 * std::log10((std::norm(Ev) + std::norm(Eh)) / (4.0 * Pi));
  out[7] = 10.0 * std::log10(std::norm(Ev) / (4.0 * Pi));
  out[8] = 10.0 * std::log10(std::norm(Eh) / (4.0 * Pi));
}

// Dense MoM PMCHWT matrix (2N x 2N, row-major complex), Code/Zmartix.h:467-539.
void ref_mom_matrix(void* h, double* Z) {
  RefCase& c = *static_cast<RefCase*>(h);
  std::vector<std::vector<cplx>> Zm;
  StdoutCapture cap(true);
  Zmartix::computeZ_die_pmchwt(c.rwgs, c.op->row, c.wave, c.gp, Zm, false);
  const size_t n = Zm.size();
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) {
      Z[2 * (i * n + j)] = Zm[i][j].real();
      Z[2 * (i * n + j) + 1] = Zm[i][j].imag();
    }
}

// MGMRES::mgmres on a dense row-major complex matrix A (n x n). Returns 1 if
// converged; the solver log goes to `log`.
int ref_gmres_dense(int n, const double* A, const double* rhs, double* x, int itr_max, int mr,
                    double tol_abs, double tol_rel, char* log, int log_len) {
  const cplx* Ac = reinterpret_cast<const cplx*>(A);
  auto ax = [Ac](int nn, const cplx* v, cplx* w) {
    for (int i = 0; i < nn; ++i) {
      cplx s(0.0, 0.0);
      for (int j = 0; j < nn; ++j) s += Ac[static_cast<size_t>(i) * nn + j] * v[j];
      w[i] = s;
    }
  };
  StdoutCapture cap(true);
  bool ok = MGMRES::mgmres(n, reinterpret_cast<cplx*>(x), reinterpret_cast<const cplx*>(rhs),
                           itr_max, mr, tol_abs, tol_rel, ax, true);
  std::string text = cap.finish();
  if (log && log_len > 0) {
    std::strncpy(log, text.c_str(), static_cast<size_t>(log_len - 1));
    log[log_len - 1] = '\0';
  }
  return ok ? 1 : 0;
}

}  // extern "C"

// The Boost.Math stand-ins the reference was compiled with (oracle/shim),
// exported so tests can pin them against independent implementations.
extern "C" {
double ref_shim_legendre_p(int l, double x) { return boost::math::legendre_p(l, x); }
double ref_shim_legendre_p_prime(int l, double x) { return boost::math::legendre_p_prime(l, x); }
double ref_shim_sph_bessel(int n, double x) { return boost::math::sph_bessel(static_cast<unsigned>(n), x); }
double ref_shim_sph_neumann(int n, double x) { return boost::math::sph_neumann(static_cast<unsigned>(n), x); }
// GL nodes/weights of the reference (my_math::gauss_legendre, Code/OverloadAlgo.h:271-288).
void ref_gauss_legendre(int n, double* x, double* w) {
  std::vector<double> X, W;
  my_math::gauss_legendre(n, X, W);
  std::copy(X.begin(), X.end(), x);
  std::copy(W.begin(), W.end(), w);
}
}

extern "C" {
// OLK::L_operator and OLK::K_operator (Code/Operator.h:709-1046) for one RWG
// pair at wavenumber k: out = {L re, L im, K re, K im}.
void ref_lk(void* h, int fld, int src, double k_re, double k_im, double* out) {
  RefCase& c = *static_cast<RefCase*>(h);
  cplx L(0.0, 0.0), K(0.0, 0.0);
  OLK::L_operator(&c.rwgs[fld], &c.rwgs[src], cplx(k_re, k_im), c.gp, L);
  OLK::K_operator(&c.rwgs[fld], &c.rwgs[src], cplx(k_re, k_im), c.gp, K);
  out[0] = L.real();
  out[1] = L.imag();
  out[2] = K.real();
  out[3] = K.imag();
}
}
