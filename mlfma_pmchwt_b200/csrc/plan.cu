// Plan construction: host tables, device upload, device setup kernels.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <map>

#include "cplx.cuh"
#include "near_same_triangle.hpp"
#include "plan.hpp"

namespace mlfma {

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}


namespace {
constexpr size_t kAlign = 256;
size_t round_up(size_t b) { return (b + kAlign - 1) & ~(kAlign - 1); }
void* device_block(size_t bytes) {
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  return p;
}
}  // namespace

void* Plan::DeviceHeap::get(size_t bytes) {
  bytes = round_up(bytes ? bytes : 1);
  if (bytes > kChunk / 4) {
    blocks.push_back(device_block(bytes));
    return blocks.back();
  }
  if (bytes > left) {
    blocks.push_back(device_block(kChunk));
    cur = static_cast<char*>(blocks.back());
    left = kChunk;
  }
  void* p = cur;
  cur += bytes;
  left -= bytes;
  return p;
}

void Plan::DeviceHeap::release() {
  for (void* p : blocks) cudaFree(p);
  blocks.clear();
  cur = nullptr;
  left = 0;
}

void Plan::SolveArena::reserve(size_t bytes) {
  if (bytes > cap) {
    release();
    base = static_cast<char*>(device_block(bytes));
    cap = bytes;
  }
  used = 0;
}

void* Plan::SolveArena::get(size_t bytes) {
  bytes = round_up(bytes ? bytes : 1);
  if (used + bytes > cap) throw std::logic_error("solve arena: request beyond the reservation");
  void* p = base + used;
  used += bytes;
  return p;
}

void Plan::SolveArena::release() {
  if (base) cudaFree(base);
  base = nullptr;
  cap = used = 0;
}

void fetch_device_status(Plan& P, cudaStream_t s) {
  check_cuda(cudaMemcpyAsync(P.h_status, P.d_status, sizeof(int), cudaMemcpyDeviceToHost, s), "status copy");
}

void raise_device_status(const Plan& P) {
  const int v = *P.h_status;
  if (v == 0) return;
  std::string where;
  if (v & 2) where += " tensor-core aggregation,";
  if (v & 4) where += " tensor-core far-field testing,";
  if (v & 8) where += " staged translation,";
  if (!where.empty()) where.pop_back();
  throw CudaError("device status " + std::to_string(v) + ": a bounded wait ran out in" +
                  (where.empty() ? std::string(" a kernel") : where));
}

Plan::~Plan() {
  if (device >= 0) {
    cudaSetDevice(device);
    // every stream of the plan idle before its memory goes back
    for (cudaStream_t st : {stream, stream2, stream_near, stream_leaf[0], stream_leaf[1]})
      if (st) cudaStreamSynchronize(st);
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    for (auto& set : prof.sets)
      for (cudaEvent_t e : set) cudaEventDestroy(e);
    heap.release();
    arena.release();
    if (h_status) cudaFreeHost(h_status);
    if (stream) cudaStreamDestroy(stream);
    if (stream2) {
      cudaStreamSynchronize(stream2);
      cudaStreamDestroy(stream2);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (stream_near) {
      cudaStreamSynchronize(stream_near);
      cudaStreamDestroy(stream_near);
    }
    if (ev_start) cudaEventDestroy(ev_start);
    if (ev_near) cudaEventDestroy(ev_near);
    for (int m = 0; m < 2; ++m) {
      if (stream_leaf[m]) {
        cudaStreamSynchronize(stream_leaf[m]);
        cudaStreamDestroy(stream_leaf[m]);
      }
      if (ev_agg[m]) cudaEventDestroy(ev_agg[m]);
      if (ev_leaf[m]) cudaEventDestroy(ev_leaf[m]);
    }
  }
}

namespace {

std::vector<double> soa3(const std::vector<double>& aos, int K) {
  std::vector<double> out(3 * static_cast<size_t>(K));
  for (int k = 0; k < K; ++k)
    for (int a = 0; a < 3; ++a) out[static_cast<size_t>(a) * K + k] = aos[3 * static_cast<size_t>(k) + a];
  return out;
}

// exp(-j k khat.d) for the 8 child octants, d = child centre - parent centre
// (sign = +1) or parent - child (sign = -1); child edge h.
std::vector<double2> shift_table(const Grid& g, cplx k, double h, double sign) {
  std::vector<double2> t(8 * static_cast<size_t>(g.K));
  const cplx J(0.0, 1.0);
  for (int o = 0; o < 8; ++o) {
    const double d[3] = {sign * (((o & 1) ? 0.5 : -0.5) * h), sign * (((o & 2) ? 0.5 : -0.5) * h),
                         sign * (((o & 4) ? 0.5 : -0.5) * h)};
    for (int kk = 0; kk < g.K; ++kk) {
      const double* kp = &g.khat[3 * static_cast<size_t>(kk)];
      const cplx kr = k * (kp[0] * d[0] + kp[1] * d[1] + kp[2] * d[2]);
      const cplx e = std::exp(-J * kr);
      t[static_cast<size_t>(o) * g.K + kk] = make_double2(e.real(), e.imag());
    }
  }
  return t;
}

}  // namespace

std::unique_ptr<Plan> create_plan(Mesh&& mesh, const PlanParams& prm) {
  const auto t0 = std::chrono::steady_clock::now();
  auto P = std::make_unique<Plan>();
  P->device = prm.device;
  P->verbose = prm.verbose;
  P->tf_complex_argument = prm.tf_complex_argument;
  if (prm.same_triangle_k != 0 && prm.same_triangle_k != 1)
    throw std::invalid_argument("same_triangle_k must be 0 (exact height) or 1 (the reference's arithmetic)");
  P->same_triangle_k = prm.same_triangle_k;
  if (prm.precision != 0 && prm.precision != 1) throw std::invalid_argument("precision must be 0 (FP64) or 1 (mixed)");
  P->precision = prm.precision;
  P->mesh = std::move(mesh);
  if (!(prm.freq > 0) || !(prm.leaf_coeff > 0)) throw std::invalid_argument("freq and leaf_coeff must be positive");
  if (!quad_rule(prm.gauss, P->quad)) throw std::invalid_argument("unsupported triangle rule");
  std::string err;
  if (!build_rwgs(P->mesh, P->rwg, err)) throw std::domain_error(err);
  P->N = P->rwg.N;

  // Wave constants (Code/EMSource.cpp:6-32).
  P->freq = prm.freq;
  P->lambda = kC0 / prm.freq;
  const double k = 2.0 * kPi / P->lambda;
  P->epsr = prm.epsr;
  P->mur = prm.mur;
  P->k1 = cplx(k, 0.0);
  P->k2 = cplx(k, 0.0) * std::sqrt(prm.epsr * prm.mur);
  P->etai = std::sqrt(prm.mur / prm.epsr);
  P->eta1 = cplx(kEta0, 0.0);
  P->eta2 = cplx(kEta0, 0.0) * std::sqrt(prm.mur / prm.epsr);

  build_tree(P->rwg, prm.leaf_coeff * P->lambda, P->tree);
  Tree& T = P->tree;
  const int L = T.maxLevel;
  P->maxL = L;
  const double kabs[2] = {std::abs(P->k1), std::abs(P->k2)};
  const cplx kc[2] = {P->k1, P->k2};
  for (int m = 0; m < 2; ++m) {
    P->ml[m].assign(L + 1, MediumLevel());
    for (int l = 2; l <= L; ++l) {
      MediumLevel& M = P->ml[m][l];
      M.grid = build_grid(kabs[m], T.lv[l].len);
      M.L = M.grid.L;
      M.nth = M.grid.nth;
      M.nph = M.grid.nph;
      M.K = M.grid.K;
    }
    for (int l = 2; l < L; ++l) P->ml[m][l].interp = build_interp(P->ml[m][l].grid, P->ml[m][l + 1].grid);
  }
  P->lv.assign(L + 1, DevLevel());
  for (int l = 0; l <= L; ++l) {
    P->lv[l].B = T.lv[l].size();
    P->lv[l].far_pairs = static_cast<long long>(T.lv[l].far_idx.size());
  }
  // near-field source lists per leaf box: near neighbours (list order), then self
  {
    const Level& Lf = T.lv[L];
    const int B = Lf.size();
    P->h_near_sptr.assign(B + 1, 0);
    P->h_near_zoff.assign(B + 1, 0);
    P->h_near_src.clear();
    for (int b = 0; b < B; ++b) {
      for (int e = Lf.near_ptr[b]; e <= Lf.near_ptr[b + 1]; ++e) {
        const int nb = e < Lf.near_ptr[b + 1] ? Lf.near_idx[e] : b;
        for (int q = T.leaf_ptr[nb]; q < T.leaf_ptr[nb + 1]; ++q) P->h_near_src.push_back(T.leaf_rwg[q]);
      }
      P->h_near_sptr[b + 1] = static_cast<int>(P->h_near_src.size());
      const long long nt = T.leaf_ptr[b + 1] - T.leaf_ptr[b];
      const long long ns = P->h_near_sptr[b + 1] - P->h_near_sptr[b];
      P->h_near_zoff[b + 1] = P->h_near_zoff[b] + nt * ns;
    }
    P->near_pairs = P->h_near_zoff[B];
  }
  if (prm.device < 0) {  // host-only plan: tables for inspection, no device work
    P->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return P;
  }

  // ------------------------------------------------------------- device
  MLFMA_CUDA(cudaSetDevice(prm.device));
  MLFMA_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
  MLFMA_CUDA(cudaStreamCreateWithFlags(&P->stream2, cudaStreamNonBlocking));
  MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
  MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming));
  MLFMA_CUDA(cudaStreamCreateWithFlags(&P->stream_near, cudaStreamNonBlocking));
  MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_start, cudaEventDisableTiming));
  MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_near, cudaEventDisableTiming));
  for (int m = 0; m < 2; ++m) {
    MLFMA_CUDA(cudaStreamCreateWithFlags(&P->stream_leaf[m], cudaStreamNonBlocking));
    MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_agg[m], cudaEventDisableTiming));
    MLFMA_CUDA(cudaEventCreateWithFlags(&P->ev_leaf[m], cudaEventDisableTiming));
  }
  cudaStream_t s = P->stream;
  const Mesh& Me = P->mesh;
  const Rwg& R = P->rwg;
  P->d_xyz = P->upload(Me.xyz);
  P->d_face_v = P->upload(Me.face_v);
  P->d_face_id = P->upload(Me.face_id);
  P->d_face_area = P->upload(Me.area);
  P->d_face_normal = P->upload(Me.normal);
  P->d_rwg_fpos = P->upload(R.fpos);
  P->d_rwg_fneg = P->upload(R.fneg);
  P->d_rwg_vpos = P->upload(R.free_pos);
  P->d_rwg_vneg = P->upload(R.free_neg);
  P->d_rwg_len = P->upload(R.len);

  for (int l = 0; l <= L; ++l) {
    const Level& Lv = T.lv[l];
    DevLevel& D = P->lv[l];
    if (l < L) D.child_begin = P->upload(Lv.child_begin);
    D.parent = P->upload(Lv.parent);
    std::vector<int> oct(Lv.size());
    for (int b = 0; b < Lv.size(); ++b) oct[b] = (Lv.ix[b] & 1) | ((Lv.iy[b] & 1) << 1) | ((Lv.iz[b] & 1) << 2);
    D.octant = P->upload(oct);
    if (l >= 2) {
      D.far_ptr = P->upload(Lv.far_ptr);
      D.far_idx = P->upload(Lv.far_idx);
      D.far_off = P->upload(Lv.far_off);
      std::vector<int> coord(3 * static_cast<size_t>(Lv.size()));
      for (int b = 0; b < Lv.size(); ++b) {
        coord[3 * b] = Lv.ix[b];
        coord[3 * b + 1] = Lv.iy[b];
        coord[3 * b + 2] = Lv.iz[b];
      }
      D.coord = P->upload(coord);
      // per parent: children of the parent's 27-neighbourhood (itself included)
      const Level& Pl = T.lv[l - 1];
      std::vector<int> uptr(Pl.size() + 1, 0), usrc;
      std::vector<int> tmp;
      for (int p = 0; p < Pl.size(); ++p) {
        tmp.clear();
        for (int e = Pl.near_ptr[p]; e <= Pl.near_ptr[p + 1]; ++e) {
          const int q = e < Pl.near_ptr[p + 1] ? Pl.near_idx[e] : p;
          for (int c = Pl.child_begin[q]; c < Pl.child_begin[q + 1]; ++c) tmp.push_back(c);
        }
        std::sort(tmp.begin(), tmp.end());
        usrc.insert(usrc.end(), tmp.begin(), tmp.end());
        uptr[p + 1] = static_cast<int>(usrc.size());
      }
      D.usrc_ptr = P->upload(uptr);
      D.usrc = P->upload(usrc);
      // per parent: union of the children's interaction-list sources with
      // the octant mask of the children that translate each of them
      std::vector<int> fptr(Pl.size() + 1, 0), fsrc, fpack;
      std::vector<std::array<int, 3>> tagged;  // (source, octant, offset code)
      for (int p = 0; p < Pl.size(); ++p) {
        tagged.clear();
        for (int c = Pl.child_begin[p]; c < Pl.child_begin[p + 1]; ++c) {
          if ((Lv.ix[c] >> 1) != Pl.ix[p] || (Lv.iy[c] >> 1) != Pl.iy[p] || (Lv.iz[c] >> 1) != Pl.iz[p])
            throw std::runtime_error("child box coordinates are not 2 * parent + octant");
          const int o = (Lv.ix[c] & 1) | ((Lv.iy[c] & 1) << 1) | ((Lv.iz[c] & 1) << 2);
          for (int e = Lv.far_ptr[c]; e < Lv.far_ptr[c + 1]; ++e) tagged.push_back({Lv.far_idx[e], o, Lv.far_off[e]});
        }
        std::sort(tagged.begin(), tagged.end());
        for (size_t i = 0; i < tagged.size();) {
          const int sb = tagged[i][0];
          const int d0[3] = {2 * Pl.ix[p] - Lv.ix[sb], 2 * Pl.iy[p] - Lv.iy[sb], 2 * Pl.iz[p] - Lv.iz[sb]};
          for (int ax = 0; ax < 3; ++ax)
            if (d0[ax] < -3 || d0[ax] > 2) throw std::runtime_error("interaction source outside the parent neighbourhood");
          const int enc0 = encode_offset(d0[0], d0[1], d0[2]);
          int mask = 0;
          for (; i < tagged.size() && tagged[i][0] == sb; ++i) {
            const int o = tagged[i][1];
            // the kernel forms the child's offset code as enc0 + octant offset
            if (enc0 + (o & 1) * 49 + ((o >> 1) & 1) * 7 + (o >> 2) != tagged[i][2])
              throw std::runtime_error("interaction offset code mismatch");
            mask |= 1 << o;
          }
          fsrc.push_back(sb);
          fpack.push_back(enc0 | (mask << 9));
        }
        fptr[p + 1] = static_cast<int>(fsrc.size());
      }
      D.ufar_ptr = P->upload(fptr);
      D.ufar = P->upload(fsrc);
      D.upack = P->upload(fpack);
    }
  }
  for (int m = 0; m < 2; ++m) {
    for (int l = 2; l <= L; ++l) {
      MediumLevel& M = P->ml[m][l];
      const int B = P->lv[l].B;
      M.khat = P->upload(soa3(M.grid.khat, M.K));
      M.S = P->alloc<double2>(static_cast<size_t>(B) * 6 * M.K);
      M.Bm = P->alloc<double2>(static_cast<size_t>(B) * 6 * M.K);
      if (l < L) {
        const Interp& I = M.interp;
        M.tidx = P->upload(I.tidx);
        M.lt = P->upload(I.lt);
        M.pidx = P->upload(I.pidx);
        M.lp = P->upload(I.lp);
        const double hc = T.lv[l + 1].len;
        M.ph_up = P->upload(shift_table(M.grid, kc[m], hc, -1.0));  // parent - child
        M.ph_dn = P->upload(shift_table(M.grid, kc[m], hc, +1.0));  // child - parent
        // bands of parent theta rows for the separable interpolation: at most
        // kUpBandOut outputs and kUpBandEntries staged child-row entries a band
        const int npp = M.nph;
        std::vector<int> rows;
        auto band_rows = [&](int t0, int R) {
          rows.clear();
          for (int t = t0; t < std::min(M.nth, t0 + R); ++t)
            for (int i = 0; i < 3; ++i) rows.push_back(I.tidx[3 * t + i]);
          std::sort(rows.begin(), rows.end());
          rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
        };
        auto worst_band = [&](int R) {
          int worst = 0;
          for (int t0 = 0; t0 < M.nth; t0 += R) {
            band_rows(t0, R);
            worst = std::max(worst, static_cast<int>(rows.size()));
          }
          return worst;
        };
        int R = std::max(1, std::min(M.nth, kUpBandOut / npp));
        while (R > 1 && worst_band(R) * npp > kUpBandEntries) --R;
        if (R * npp <= kUpBandOut && worst_band(R) * npp <= kUpBandEntries) {
          M.up_rows = R;
          M.up_nband = (M.nth + R - 1) / R;
          std::vector<int> rptr(M.up_nband + 1, 0), rlist, tpos(3 * static_cast<size_t>(M.nth));
          for (int bi = 0; bi < M.up_nband; ++bi) {
            band_rows(bi * R, R);
            for (int t = bi * R; t < std::min(M.nth, (bi + 1) * R); ++t)
              for (int i = 0; i < 3; ++i)
                tpos[3 * t + i] =
                    static_cast<int>(std::lower_bound(rows.begin(), rows.end(), I.tidx[3 * t + i]) - rows.begin());
            rlist.insert(rlist.end(), rows.begin(), rows.end());
            rptr[bi + 1] = static_cast<int>(rlist.size());
            M.up_band_max = std::max(M.up_band_max, static_cast<int>(rows.size()));
          }
          M.up_row_ptr = P->upload(rptr);
          M.up_row = P->upload(rlist);
          M.up_tpos = P->upload(tpos);
        }
        // bands of kUpColBand parent rows for the register-separable kernel
        if (worst_band(kUpColBand) <= kUpColRows) {
          M.up4_nband = (M.nth + kUpColBand - 1) / kUpColBand;
          std::vector<int> rptr(M.up4_nband + 1, 0), rlist, tpos(3 * static_cast<size_t>(M.nth));
          for (int bi = 0; bi < M.up4_nband; ++bi) {
            band_rows(bi * kUpColBand, kUpColBand);
            for (int t = bi * kUpColBand; t < std::min(M.nth, (bi + 1) * kUpColBand); ++t)
              for (int i = 0; i < 3; ++i)
                tpos[3 * t + i] =
                    static_cast<int>(std::lower_bound(rows.begin(), rows.end(), I.tidx[3 * t + i]) - rows.begin());
            rlist.insert(rlist.end(), rows.begin(), rows.end());
            rptr[bi + 1] = static_cast<int>(rlist.size());
          }
          M.up4_row_ptr = P->upload(rptr);
          M.up4_row = P->upload(rlist);
          M.up4_tpos = P->upload(tpos);
        }
      }
      if (l > 2) {
        // transposed interpolation: child direction <- (parent direction, weight)
        const MediumLevel& Pm = P->ml[m][l - 1];
        const Interp& I = Pm.interp;
        std::vector<int> cnt(M.K + 1, 0);
        for (int kp = 0; kp < Pm.K; ++kp) {
          const int t = kp / Pm.nph, p = kp % Pm.nph;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) cnt[I.tidx[3 * t + i] * M.nph + I.pidx[3 * p + j] + 1]++;
        }
        for (int kk = 0; kk < M.K; ++kk) cnt[kk + 1] += cnt[kk];
        std::vector<int> fill(cnt.begin(), cnt.end() - 1), kps(cnt[M.K]);
        std::vector<double> ws(cnt[M.K]);
        for (int kp = 0; kp < Pm.K; ++kp) {
          const int t = kp / Pm.nph, p = kp % Pm.nph;
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
              const int c = I.tidx[3 * t + i] * M.nph + I.pidx[3 * p + j];
              kps[fill[c]] = kp;
              ws[fill[c]] = I.lt[3 * t + i] * I.lp[3 * p + j];
              fill[c]++;
            }
        }
        M.tr_ptr = P->upload(cnt);
        M.tr_kp = P->upload(kps);
        M.tr_w = P->upload(ws);
        // separable transposes of the two 1-D stencils
        auto transpose1d = [&](const std::vector<int>& idx, const std::vector<double>& w, int nsrc, int ndst,
                               int*& d_ptr, int*& d_src, double*& d_w) {
          std::vector<int> ptr(ndst + 1, 0), src;
          std::vector<double> wt;
          for (int q = 0; q < nsrc; ++q)
            for (int i = 0; i < 3; ++i) ptr[idx[3 * q + i] + 1]++;
          for (int d = 0; d < ndst; ++d) ptr[d + 1] += ptr[d];
          src.resize(ptr[ndst]);
          wt.resize(ptr[ndst]);
          std::vector<int> f(ptr.begin(), ptr.end() - 1);
          for (int q = 0; q < nsrc; ++q)
            for (int i = 0; i < 3; ++i) {
              const int d = idx[3 * q + i];
              src[f[d]] = q;
              wt[f[d]] = w[3 * q + i];
              f[d]++;
            }
          d_ptr = P->upload(ptr);
          d_src = P->upload(src);
          d_w = P->upload(wt);
        };
        transpose1d(I.tidx, I.lt, Pm.nth, M.nth, M.thT_ptr, M.thT_src, M.thT_w);
        transpose1d(I.pidx, I.lp, Pm.nph, M.nph, M.phT_ptr, M.phT_src, M.phT_w);
      }
      // transfer factors over the offsets this level uses (Code/AlgoMLFMM.h:192-295)
      {
        std::vector<char> used(343, 0);
        for (int e : T.lv[l].far_off) used[e] = 1;
        std::vector<int> off2vec(343, -1);
        M.vec_off.clear();
        for (int e = 0; e < 343; ++e)
          if (used[e]) {
            off2vec[e] = static_cast<int>(M.vec_off.size());
            M.vec_off.push_back(e);
          }
        M.nvec = static_cast<int>(M.vec_off.size());
        M.off2vec = P->upload(off2vec);
        if (m == 0) {  // the offset -> row map depends on the level's lists only, not on the medium
          std::vector<int> fv(T.lv[l].far_off.size());
          for (size_t e = 0; e < fv.size(); ++e) fv[e] = off2vec[T.lv[l].far_off[e]];
          P->lv[l].far_vec = P->upload(fv);
          // merged lists of box pairs (2g, 2g+1)
          const Level& Lv = T.lv[l];
          const int B = Lv.size(), G = (B + 1) / 2;
          std::vector<int> pptr(G + 1, 0), psrc;
          std::vector<int2> pvec;
          for (int g = 0; g < G; ++g) {
            const int b0 = 2 * g, b1 = std::min(2 * g + 1, B - 1);
            int e0 = Lv.far_ptr[b0], e1 = b1 != b0 ? Lv.far_ptr[b1] : 0;
            const int f0 = Lv.far_ptr[b0 + 1], f1 = b1 != b0 ? Lv.far_ptr[b1 + 1] : 0;
            while (e0 < f0 || e1 < f1) {
              const int s0 = e0 < f0 ? Lv.far_idx[e0] : INT32_MAX, s1 = e1 < f1 ? Lv.far_idx[e1] : INT32_MAX;
              const int src = std::min(s0, s1);
              int2 v = make_int2(-1, -1);
              if (s0 == src) v.x = fv[e0++];
              if (s1 == src) v.y = fv[e1++];
              psrc.push_back(src);
              pvec.push_back(v);
            }
            pptr[g + 1] = static_cast<int>(psrc.size());
          }
          P->lv[l].pair_ptr = P->upload(pptr);
          P->lv[l].pair_src = P->upload(psrc);
          P->lv[l].pair_vec = P->upload(pvec);
          // merged lists of box groups (8q .. 8q+7)
          const int G8 = (B + 7) / 8;
          std::vector<int> gptr(G8 + 1, 0), gsrc;
          std::vector<int4> gcode;
          for (int q = 0; q < G8; ++q) {
            const int nb = std::min(8, B - 8 * q);
            int cur[8], end[8];
            for (int j = 0; j < nb; ++j) {
              cur[j] = Lv.far_ptr[8 * q + j];
              end[j] = Lv.far_ptr[8 * q + j + 1];
              for (int e = cur[j] + 1; e < end[j]; ++e)
                if (Lv.far_idx[e] <= Lv.far_idx[e - 1]) throw std::runtime_error("interaction list not ascending");
            }
            for (;;) {
              int src = INT32_MAX;
              for (int j = 0; j < nb; ++j)
                if (cur[j] < end[j]) src = std::min(src, Lv.far_idx[cur[j]]);
              if (src == INT32_MAX) break;
              unsigned w[4] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu};
              for (int j = 0; j < nb; ++j)
                if (cur[j] < end[j] && Lv.far_idx[cur[j]] == src) {
                  const int code = fv[cur[j]++];
                  if (code < 0 || code > 32767) throw std::runtime_error("transfer-factor row out of 16-bit range");
                  const int sh = 16 * (j & 1);
                  w[j >> 1] = (w[j >> 1] & ~(0xffffu << sh)) | (static_cast<unsigned>(code) << sh);
                }
              gsrc.push_back(src);
              gcode.push_back(make_int4(static_cast<int>(w[0]), static_cast<int>(w[1]), static_cast<int>(w[2]),
                                        static_cast<int>(w[3])));
            }
            gptr[q + 1] = static_cast<int>(gsrc.size());
          }
          P->lv[l].grp_ptr = P->upload(gptr);
          P->lv[l].grp_src = P->upload(gsrc);
          P->lv[l].grp_code = P->upload(gcode);
        }
        std::vector<double> rhat;
        std::vector<int> hoff, hL;
        std::vector<double2> h2all;
        P->tf_inputs(m, l, rhat, hoff, hL, h2all);
        M.tfw = P->alloc<double2>(static_cast<size_t>(std::max(M.nvec, 1)) * M.K);
        launch_transfer(*P, m, l, rhat, hoff, hL, h2all, true, M.tfw, s, true);
      }
    }
  }
  // leaf data
  {
    const Level& Lf = T.lv[L];
    P->d_leaf_ptr = P->upload(T.leaf_ptr);
    P->max_leaf_rwgs = 0;
    for (size_t b = 0; b + 1 < T.leaf_ptr.size(); ++b)
      P->max_leaf_rwgs = std::max(P->max_leaf_rwgs, T.leaf_ptr[b + 1] - T.leaf_ptr[b]);
    P->d_leaf_rwg = P->upload(T.leaf_rwg);
    P->d_rwg_leafbox = P->upload(T.rwg_leaf);
    P->d_leaf_center = P->upload(Lf.center);
    for (int m = 0; m < 2; ++m) {
      const int K = P->ml[m][L].K;
      P->d_Vs[m] = P->alloc<double2>(static_cast<size_t>(P->N) * 3 * K);
      P->d_Vf[m] = P->alloc<double2>(static_cast<size_t>(P->N) * 3 * K);
      launch_patterns(*P, m, s);
    }
  }
  // near field
  {
    std::vector<double> q(4 * static_cast<size_t>(P->quad.n));
    P->d_near_sptr = P->upload(P->h_near_sptr);
    P->d_near_src = P->upload(P->h_near_src);
    P->d_near_zoff = P->upload(P->h_near_zoff);
    P->d_near_z = P->alloc<double2>(3 * static_cast<size_t>(std::max<long long>(P->near_pairs, 1)));
    launch_near(*P, s);
    if (P->same_triangle_k == 1) {
      // the K entries of RWG pairs sharing a triangle, with the reference's
      // arithmetic on the host, written over the device kernel's
      std::vector<long long> pos;
      std::vector<int> tgt, src;
      same_triangle_pairs(P->rwg, P->tree, P->h_near_sptr, P->h_near_src, P->h_near_zoff, pos, tgt, src);
      std::vector<cplx> z12;
      same_triangle_z12(P->mesh, P->rwg, P->quad, P->k1, P->k2, tgt, src, z12);
      const long long n = static_cast<long long>(pos.size());
      P->same_triangle_pairs = n;
      if (n > 0) {
        std::vector<double2> zv(z12.size());
        for (size_t i = 0; i < z12.size(); ++i) zv[i] = make_double2(z12[i].real(), z12[i].imag());
        launch_near_z12_scatter(P->d_near_z, P->upload(pos), P->upload(zv), n, s);
      }
    }
  }
  P->d_x = P->alloc<double2>(2 * static_cast<size_t>(P->N));
  P->d_w = P->alloc<double2>(2 * static_cast<size_t>(P->N));
  P->d_status = P->alloc<int>(1);
  MLFMA_CUDA(cudaMemsetAsync(P->d_status, 0, sizeof(int), s));
  MLFMA_CUDA(cudaHostAlloc(&P->h_status, sizeof(int), cudaHostAllocDefault));
  *P->h_status = 0;
  // complex64 copies of the operator's tables and its workspaces
  if (P->precision == 1) {
    auto copy32 = [&](const double2* src, size_t n) {
      float2* d = P->alloc<float2>(n);
      to_c64(src, d, n, s);
      return d;
    };
    for (int m = 0; m < 2; ++m) {
      const size_t np = static_cast<size_t>(P->N) * 3 * P->ml[m][L].K;
      P->d_Vs32[m] = copy32(P->d_Vs[m], np);
      P->d_Vf32[m] = copy32(P->d_Vf[m], np);
      for (int l = 2; l <= L; ++l) {
        MediumLevel& M = P->ml[m][l];
        const size_t nb = static_cast<size_t>(P->lv[l].B) * 6 * M.K;
        M.S32 = P->alloc<float2>(nb);
        M.Bm32 = P->alloc<float2>(nb);
        M.tfw32 = copy32(M.tfw, static_cast<size_t>(std::max(M.nvec, 1)) * M.K);
        if (l < L) {
          M.ph_up32 = copy32(M.ph_up, 8 * static_cast<size_t>(M.K));
          M.ph_dn32 = copy32(M.ph_dn, 8 * static_cast<size_t>(M.K));
        }
      }
    }
  }
  // complex64 copy of the near field: the flexible GMRES preconditioner's
  // products (any plan) and the mixed operator's near rows
  {
    const size_t nz = 3 * static_cast<size_t>(std::max<long long>(P->near_pairs, 1));
    P->d_near_z32 = P->alloc<float2>(nz);
    to_c64(P->d_near_z, P->d_near_z32, nz, s);
  }
  MLFMA_CUDA(cudaStreamSynchronize(s));
  P->setup_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (P->verbose) {
    std::fprintf(stderr, "mlfma: N=%d maxLevel=%d near pairs=%lld device bytes=%.3e setup %.3f s\n", P->N, L,
                 P->near_pairs, static_cast<double>(P->bytes), P->setup_seconds);
  }
  return P;
}

// Inputs of the transfer-factor kernel for (medium, level): per used offset,
// the unit vector, h2_l(|k R|) for l <= min(L, ceil(|k R|)) (Code/AlgoMLFMM.h:252-267).
void Plan::tf_inputs(int m, int l, std::vector<double>& rhat, std::vector<int>& hoff, std::vector<int>& hL,
                     std::vector<double2>& h2all) const {
  const MediumLevel& M = ml[m][l];
  const cplx kw = m == 0 ? k1 : k2;
  const double len = tree.lv[l].len;
  rhat.clear();
  hoff.clear();
  hL.clear();
  h2all.clear();
  std::vector<cplx> h2;
  for (int e : M.vec_off) {
    int dx, dy, dz;
    decode_offset(e, dx, dy, dz);
    double r[3] = {dx * len, dy * len, dz * len};
    const double Rpq = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (double& v : r) v /= Rpq;
    const cplx kR = kw * Rpq;
    const int Lt = std::min(M.L, static_cast<int>(std::ceil(std::abs(kR))));
    if (tf_complex_argument)
      hankel2_array_complex(Lt, kR, h2);  // not the reference: see PlanParams::tf_complex_argument
    else
      hankel2_array(Lt, std::abs(kR), h2);
    rhat.insert(rhat.end(), r, r + 3);
    hoff.push_back(static_cast<int>(h2all.size()));
    hL.push_back(Lt);
    for (const cplx& v : h2) h2all.push_back(make_double2(v.real(), v.imag()));
  }
}

}  // namespace mlfma
