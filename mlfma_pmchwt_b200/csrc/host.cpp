// Host-side setup: mesh, RWGs, octree, grids, interpolation, special
// functions, quadrature. See host.hpp.
#include "host.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <unordered_map>

namespace mlfma {

// ---------------------------------------------------------------- mesh ----

void mesh_derive(Mesh& m) {
  const size_t nf = m.face_id.size();
  m.area.assign(nf, 0.0);
  m.normal.assign(3 * nf, 0.0);
  for (size_t f = 0; f < nf; ++f) {
    const double* a = &m.xyz[3 * m.face_v[3 * f]];
    const double* b = &m.xyz[3 * m.face_v[3 * f + 1]];
    const double* c = &m.xyz[3 * m.face_v[3 * f + 2]];
    const double ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const double cr[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2],
                          ab[0] * ac[1] - ab[1] * ac[0]};
    const double nrm = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    // Code/NASReader.cpp:24-37: area = |AB x AC| / 2.
    m.area[f] = nrm / 2.0;
    // Code/NASReader.cpp:39-58: unit normal from vertex order, components
    // below 1e-6 in magnitude set to zero (not renormalised).
    double n[3] = {cr[0], cr[1], cr[2]};
    if (nrm > 0) {
      n[0] /= nrm;
      n[1] /= nrm;
      n[2] /= nrm;
    }
    for (int i = 0; i < 3; ++i) {
      if (std::abs(n[i]) < 1e-6) n[i] = 0.0;
      m.normal[3 * f + i] = n[i];
    }
  }
}

bool mesh_from_arrays(int np, const int* pid, const double* xyz, int nf, const int* fid,
                      const int* fpts, Mesh& m, std::string& err) {
  if (np <= 0 || nf <= 0 || !pid || !xyz || !fid || !fpts) {
    err = "mesh: empty or null arrays";
    return false;
  }
  m.point_id.assign(pid, pid + np);
  m.xyz.assign(xyz, xyz + 3 * static_cast<size_t>(np));
  m.face_id.assign(fid, fid + nf);
  m.face_v.resize(3 * static_cast<size_t>(nf));
  std::unordered_map<int, int> index;
  index.reserve(static_cast<size_t>(np) * 2);
  for (int i = 0; i < np; ++i) {
    // Code/NASReader.cpp:114-118 binds a vertex id to the LAST point with that id.
    index[pid[i]] = i;
  }
  for (int f = 0; f < nf; ++f)
    for (int k = 0; k < 3; ++k) {
      auto it = index.find(fpts[3 * f + k]);
      if (it == index.end()) {
        err = "mesh: face " + std::to_string(fid[f]) + " references missing point " +
              std::to_string(fpts[3 * f + k]);
        return false;
      }
      m.face_v[3 * f + k] = it->second;
    }
  mesh_derive(m);
  return true;
}

// Reads GRID* (with its '*' continuation line carrying the same id and z) and
// CTRIA3 records, the dialect of Code/NASReader.cpp:60-144.
bool read_nas(const std::string& path, Mesh& m, std::string& err) {
  std::ifstream in(path);
  if (!in.is_open()) {
    err = "cannot open NAS file: " + path;
    return false;
  }
  std::vector<int> pid, fid, fpts;
  std::vector<double> xyz;
  std::string line;
  bool pending = false;
  int cur_id = 0;
  double cx = 0, cy = 0;
  while (std::getline(in, line)) {
    if (line.compare(0, 5, "GRID*") == 0) {
      std::istringstream ss(line.substr(5));
      if (!(ss >> cur_id >> cx >> cy)) {
        err = "invalid GRID* record: " + line;
        return false;
      }
      pending = true;
    } else if (pending && !line.empty() && line[0] == '*') {
      std::istringstream ss(line.substr(1));
      int cid;
      double cz;
      if (!(ss >> cid >> cz)) {
        err = "invalid GRID* continuation: " + line;
        return false;
      }
      if (cid != cur_id) {
        err = "GRID* continuation id mismatch";
        return false;
      }
      pid.push_back(cur_id);
      xyz.push_back(cx);
      xyz.push_back(cy);
      xyz.push_back(cz);
      pending = false;
    } else if (line.compare(0, 6, "CTRIA3") == 0) {
      std::istringstream ss(line.substr(6));
      int f, prop, a, b, c;
      if (!(ss >> f >> prop >> a >> b >> c)) {
        err = "invalid CTRIA3 record: " + line;
        return false;
      }
      fid.push_back(f);
      fpts.push_back(a);
      fpts.push_back(b);
      fpts.push_back(c);
    }
  }
  if (pending) {
    err = "unfinished GRID* record at end of file";
    return false;
  }
  return mesh_from_arrays(static_cast<int>(pid.size()), pid.data(), xyz.data(),
                          static_cast<int>(fid.size()), fid.data(), fpts.data(), m, err);
}

// ----------------------------------------------------------------- RWG ----

bool build_rwgs(const Mesh& m, Rwg& r, std::string& err) {
  // Code/RWGGenerator.cpp:41-53: edges keyed by (min id, max id) in ascending
  // order; each edge lists the faces containing it in face (file) order via
  // the face's edges (v1,v2), (v2,v3), (v3,v1).
  std::map<std::pair<int, int>, std::vector<int>> edges;
  const int nf = static_cast<int>(m.face_id.size());
  for (int f = 0; f < nf; ++f) {
    const int ids[3] = {m.point_id[m.face_v[3 * f]], m.point_id[m.face_v[3 * f + 1]],
                        m.point_id[m.face_v[3 * f + 2]]};
    for (int j = 0; j < 3; ++j) {
      int a = ids[j], b = ids[(j + 1) % 3];
      if (a > b) std::swap(a, b);
      edges[{a, b}].push_back(f);
    }
  }
  std::unordered_map<int, int> pindex;
  for (size_t i = 0; i < m.point_id.size(); ++i) pindex[m.point_id[i]] = static_cast<int>(i);
  r = Rwg();
  for (const auto& e : edges) {
    // Only edges shared by exactly two faces carry an RWG (:62); the first
    // face is T+, the second T- (:66-69).
    if (e.second.size() != 2) continue;
    const int fp = e.second[0], fn = e.second[1];
    // Code/RWGGenerator.cpp:73-76: commonEdgeVertex1/2 are the LAST points
    // carrying the two ids (same binding rule as the face vertices).
    const int pa = pindex.at(e.first.first), pb = pindex.at(e.first.second);
    auto free_vertex = [&](int f) {
      for (int k = 0; k < 3; ++k) {
        const int v = m.face_v[3 * f + k];
        const int id = m.point_id[v];
        if (id != e.first.first && id != e.first.second) return v;
      }
      return -1;
    };
    const int vp = free_vertex(fp), vn = free_vertex(fn);
    if (vp < 0 || vn < 0) {
      err = "degenerate face: free vertex not found";
      return false;
    }
    const double* A = &m.xyz[3 * pa];
    const double* B = &m.xyz[3 * pb];
    const double d0 = A[0] - B[0], d1 = A[1] - B[1], d2 = A[2] - B[2];
    r.fpos.push_back(fp);
    r.fneg.push_back(fn);
    r.free_pos.push_back(vp);
    r.free_neg.push_back(vn);
    r.ea.push_back(pa);
    r.eb.push_back(pb);
    r.len.push_back(std::sqrt(d0 * d0 + d1 * d1 + d2 * d2));   // :83 CalcDistance
    r.mid.push_back((A[0] + B[0]) / 2.0);                      // :84-89
    r.mid.push_back((A[1] + B[1]) / 2.0);
    r.mid.push_back((A[2] + B[2]) / 2.0);
  }
  r.N = static_cast<int>(r.len.size());
  if (r.N == 0) {
    err = "mesh has no interior edges (no RWG functions)";
    return false;
  }
  return true;
}

// -------------------------------------------------------------- octree ----

namespace {
uint64_t spread3(uint32_t x) {  // interleave with two zero bits (21-bit input)
  uint64_t v = x & 0x1fffff;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton(int x, int y, int z) {
  return spread3(static_cast<uint32_t>(x)) | (spread3(static_cast<uint32_t>(y)) << 1) |
         (spread3(static_cast<uint32_t>(z)) << 2);
}
}  // namespace

void build_tree(const Rwg& r, double leaf_target, Tree& t) {
  // Code/OCTree.cpp:161-242: bounding box of the RWG edge midpoints, root
  // edge 1.001 x the largest extent, maxLevel = clamp(ceil(log2(root/leaf)), 2, 15),
  // then a cube of leaf_target * 2^maxLevel centred on the box.
  double lo[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                  std::numeric_limits<double>::max()};
  double hi[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
                  std::numeric_limits<double>::lowest()};
  for (int i = 0; i < r.N; ++i)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], r.mid[3 * i + a]);
      hi[a] = std::max(hi[a], r.mid[3 * i + a]);
    }
  double root = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2])) * 1.001;
  double ratio = root / leaf_target;
  if (ratio < 1.0) ratio = 1.0;
  int maxL = static_cast<int>(std::ceil(std::log2(ratio)));
  maxL = std::max(2, std::min(maxL, 15));
  root = leaf_target * (1 << maxL);
  const double c[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), 0.5 * (lo[2] + hi[2])};
  t.maxLevel = maxL;
  t.rootLen = root;
  for (int a = 0; a < 3; ++a) t.gmin[a] = c[a] - 0.5 * root;
  t.leafLen = root / (1 << maxL);
  t.lv.assign(maxL + 1, Level());

  // Leaves (Code/OCTree.cpp:244-307): truncating division of the midpoint
  // offset by the leaf edge, clamped to the grid.
  const int maxIdx = (1 << maxL) - 1;
  std::vector<uint64_t> rcode(r.N);
  std::vector<std::array<int, 3>> rij(r.N);
  for (int i = 0; i < r.N; ++i) {
    int ij[3];
    for (int a = 0; a < 3; ++a) {
      ij[a] = static_cast<int>((r.mid[3 * i + a] - t.gmin[a]) / t.leafLen);
      ij[a] = std::max(0, std::min(ij[a], maxIdx));
    }
    rij[i] = {ij[0], ij[1], ij[2]};
    rcode[i] = morton(ij[0], ij[1], ij[2]);
  }
  {
    Level& L = t.lv[maxL];
    L.level = maxL;
    L.len = t.leafLen;
    std::vector<uint64_t> codes(rcode);
    std::sort(codes.begin(), codes.end());
    codes.erase(std::unique(codes.begin(), codes.end()), codes.end());
    L.code = codes;
  }
  for (int l = maxL - 1; l >= 0; --l) {
    Level& L = t.lv[l];
    L.level = l;
    L.len = t.lv[l + 1].len * 2.0;
    for (uint64_t cc : t.lv[l + 1].code) {
      const uint64_t p = cc >> 3;
      if (L.code.empty() || L.code.back() != p) L.code.push_back(p);  // sorted input
    }
  }
  for (int l = 0; l <= maxL; ++l) {
    Level& L = t.lv[l];
    const int B = L.size();
    L.ix.resize(B);
    L.iy.resize(B);
    L.iz.resize(B);
    L.center.resize(3 * B);
    for (int b = 0; b < B; ++b) {
      // decode Morton
      int v[3] = {0, 0, 0};
      const uint64_t cd = L.code[b];
      for (int bit = 0; bit < 21; ++bit)
        for (int a = 0; a < 3; ++a) v[a] |= static_cast<int>((cd >> (3 * bit + a)) & 1ULL) << bit;
      L.ix[b] = v[0];
      L.iy[b] = v[1];
      L.iz[b] = v[2];
      for (int a = 0; a < 3; ++a) L.center[3 * b + a] = t.gmin[a] + (v[a] + 0.5) * L.len;
    }
  }
  // parent / children links (children of a parent are contiguous in Morton order)
  for (int l = 0; l <= maxL; ++l) {
    Level& L = t.lv[l];
    const int B = L.size();
    L.parent.assign(B, -1);
    if (l > 0) {
      const Level& P = t.lv[l - 1];
      for (int b = 0; b < B; ++b)
        L.parent[b] = static_cast<int>(std::lower_bound(P.code.begin(), P.code.end(), L.code[b] >> 3) -
                                       P.code.begin());
    }
    if (l < maxL) {
      const Level& C = t.lv[l + 1];
      L.child_begin.assign(B + 1, 0);
      int ci = 0;
      for (int b = 0; b < B; ++b) {
        L.child_begin[b] = ci;
        while (ci < C.size() && (C.code[ci] >> 3) == L.code[b]) ++ci;
      }
      L.child_begin[B] = ci;
    }
  }
  // RWG -> leaf, leaf RWG lists in ascending RWG id (insertion order of
  // Code/OCTree.cpp:304).
  {
    const Level& Lf = t.lv[maxL];
    t.rwg_leaf.resize(r.N);
    std::vector<int> cnt(Lf.size() + 1, 0);
    for (int i = 0; i < r.N; ++i) {
      t.rwg_leaf[i] = static_cast<int>(std::lower_bound(Lf.code.begin(), Lf.code.end(), rcode[i]) -
                                       Lf.code.begin());
      cnt[t.rwg_leaf[i] + 1]++;
    }
    for (int b = 0; b < Lf.size(); ++b) cnt[b + 1] += cnt[b];
    t.leaf_ptr = cnt;
    t.leaf_rwg.resize(r.N);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int i = 0; i < r.N; ++i) t.leaf_rwg[fill[t.rwg_leaf[i]]++] = i;
  }
  // Near lists (Code/OCTree.cpp:385-426) and interaction lists
  // (:428-488): children of the parent's neighbourhood (parent included)
  // that are not within one box of the target.
  for (int l = 0; l <= maxL; ++l) {
    Level& L = t.lv[l];
    const int B = L.size();
    std::unordered_map<uint64_t, int> idx;
    idx.reserve(2 * static_cast<size_t>(B));
    for (int b = 0; b < B; ++b) idx[L.code[b]] = b;
    const int grid = 1 << l;
    L.near_ptr.assign(B + 1, 0);
    L.near_idx.clear();
    for (int b = 0; b < B; ++b) {
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            if (!dx && !dy && !dz) continue;
            const int x = L.ix[b] + dx, y = L.iy[b] + dy, z = L.iz[b] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= grid || y >= grid || z >= grid) continue;
            auto it = idx.find(morton(x, y, z));
            if (it != idx.end()) L.near_idx.push_back(it->second);
          }
      L.near_ptr[b + 1] = static_cast<int>(L.near_idx.size());
    }
    L.far_ptr.assign(B + 1, 0);
    L.far_idx.clear();
    L.far_off.clear();
    if (l >= 2) {
      const Level& P = t.lv[l - 1];
      const int pgrid = 1 << (l - 1);
      std::vector<int> cand;
      for (int b = 0; b < B; ++b) {
        cand.clear();
        const int p = L.parent[b];
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
              const int px = P.ix[p] + dx, py = P.iy[p] + dy, pz = P.iz[p] + dz;
              if (px < 0 || py < 0 || pz < 0 || px >= pgrid || py >= pgrid || pz >= pgrid) continue;
              for (int o = 0; o < 8; ++o) {
                const int x = 2 * px + (o & 1), y = 2 * py + ((o >> 1) & 1), z = 2 * pz + ((o >> 2) & 1);
                auto it = idx.find(morton(x, y, z));
                if (it == idx.end() || it->second == b) continue;
                const int ddx = L.ix[b] - x, ddy = L.iy[b] - y, ddz = L.iz[b] - z;
                if (std::max(std::abs(ddx), std::max(std::abs(ddy), std::abs(ddz))) <= 1) continue;
                cand.push_back(it->second);
              }
            }
        std::sort(cand.begin(), cand.end());
        for (int s : cand) {
          L.far_idx.push_back(s);
          L.far_off.push_back(encode_offset(L.ix[b] - L.ix[s], L.iy[b] - L.iy[s], L.iz[b] - L.iz[s]));
        }
        L.far_ptr[b + 1] = static_cast<int>(L.far_idx.size());
      }
    }
  }
}

// --------------------------------------------------- special functions ----

double legendre_p(int l, double x) {
  if (l < 0) l = -l - 1;
  if (l == 0) return 1.0;
  double pm1 = 1.0, p = x;
  for (int n = 1; n < l; ++n) {
    const double pn1 = ((2.0 * n + 1.0) * x * p - n * pm1) / (n + 1.0);
    pm1 = p;
    p = pn1;
  }
  return p;
}

double legendre_dp(int l, double x) {
  if (l < 0) l = -l - 1;
  if (l == 0) return 0.0;
  // dP_l/dx = sum of (2k+1) P_k over k = l-1, l-3, ...
  double deriv = 0.0;
  double pm1 = 1.0, p = x;
  if (((l - 1) & 1) == 0) deriv += 1.0;
  if (l - 1 >= 1 && ((l - 2) & 1) == 0) deriv += 3.0 * x;
  for (int k = 1; k + 1 <= l - 1; ++k) {
    const double pk1 = ((2.0 * k + 1.0) * x * p - k * pm1) / (k + 1.0);
    pm1 = p;
    p = pk1;
    const int kk = k + 1;
    if (((l - 1 - kk) & 1) == 0) deriv += (2.0 * kk + 1.0) * p;
  }
  return deriv;
}

double sph_j(int n, double x) {
  if (x == 0.0) return n == 0 ? 1.0 : 0.0;
  const double ax = std::fabs(x);
  double result;
  if (ax < 1e-3 * (n + 1) || ax < 1e-8) {
    double pref = 1.0;
    for (int k = 1; k <= n; ++k) pref *= ax / (2.0 * k + 1.0);
    double term = 1.0, sum = 1.0;
    const double h = -0.5 * ax * ax;
    for (int k = 1; k < 60; ++k) {
      term *= h / (k * (2.0 * n + 2.0 * k + 1.0));
      sum += term;
      if (std::fabs(term) < 1e-18 * std::fabs(sum)) break;
    }
    result = pref * sum;
  } else {
    const double s = std::sin(ax), c = std::cos(ax);
    const double j0 = s / ax;
    if (n == 0) return j0;
    const double j1 = s / (ax * ax) - c / ax;
    if (n <= ax) {  // upward recurrence is stable while n < x
      double jm = j0, j = j1;
      for (int k = 1; k < n; ++k) {
        const double jn = (2.0 * k + 1.0) / ax * j - jm;
        jm = j;
        j = jn;
      }
      result = j;
    } else {  // Miller's backward recurrence
      const int start = n + 20 + static_cast<int>(std::sqrt(40.0 * (n + ax)));
      double fp = 0.0, f = 1e-280, fn_keep = 0.0, f0 = 0.0, f1 = 0.0;
      for (int k = start; k >= 1; --k) {
        const double fm = (2.0 * k + 1.0) / ax * f - fp;
        fp = f;
        f = fm;
        if (std::fabs(f) > 1e250) {
          f *= 1e-250;
          fp *= 1e-250;
          fn_keep *= 1e-250;
          f1 *= 1e-250;
        }
        if (k - 1 == n) fn_keep = f;
        if (k - 1 == 1) f1 = f;
        if (k - 1 == 0) f0 = f;
      }
      const double scale = (std::fabs(j0) >= std::fabs(j1)) ? j0 / f0 : j1 / f1;
      result = fn_keep * scale;
    }
  }
  return (x < 0 && (n & 1)) ? -result : result;
}

double sph_y(int n, double x) {
  if (x <= 0.0) return -std::numeric_limits<double>::infinity();
  const double s = std::sin(x), c = std::cos(x);
  const double y0 = -c / x;
  if (n == 0) return y0;
  double ym = y0, y = -c / (x * x) - s / x;
  for (int k = 1; k < n; ++k) {
    const double yn = (2.0 * k + 1.0) / x * y - ym;
    ym = y;
    y = yn;
  }
  return y;
}

// h2_l(x) = j_l(x) - i y_l(x), l = 0..L (Code/Bessel.h:18-47).
void hankel2_array(int L, double x, std::vector<cplx>& h2) {
  h2.resize(L + 1);
  for (int l = 0; l <= L; ++l) h2[l] = cplx(sph_j(l, x), -sph_y(l, x));
}

void hankel2_array_complex(int L, cplx z, std::vector<cplx>& h2) {
  h2.resize(L + 1);
  const cplx I(0.0, 1.0);
  const cplx e = std::exp(-I * z);
  h2[0] = I * e / z;
  if (L >= 1) h2[1] = e * (I / (z * z) - 1.0 / z);
  for (int l = 1; l < L; ++l) h2[l + 1] = (2.0 * l + 1.0) / z * h2[l] - h2[l - 1];
}

// Code/OverloadAlgo.h:254-288: Newton on P_n from cos(pi (i+0.75)/(n+0.5)),
// |dx| < 1e-10, at most 100 steps; nodes stored as -root / +root.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double r = std::cos(kPi * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      const double dx = legendre_p(n, r) / legendre_dp(n, r);
      r -= dx;
      if (std::abs(dx) < 1e-10) break;
    }
    x[i] = -r;
    x[n - i - 1] = r;
    const double dp = legendre_dp(n, r);
    const double wt = 2.0 / ((1 - r * r) * dp * dp);
    w[i] = wt;
    w[n - i - 1] = wt;
  }
}

// ------------------------------------------------------- angular grids ----

Grid build_grid(double kabs, double box_len) {
  Grid g;
  // Code/AlgoMLFMM.h:34-39: L = ceil(kD + 6 (kD)^(1/3)), D = sqrt(3) * box edge.
  const double D = std::sqrt(3.0) * box_len;
  g.L = static_cast<int>(std::ceil(kabs * D + 6.0 * std::cbrt(kabs * D)));
  g.nth = g.L;           // theta count = L (:62)
  g.nph = 2 * g.L;       // phi count = 2L (:81)
  g.K = g.nth * g.nph;
  std::vector<double> xg;
  gauss_legendre(g.nth, xg, g.wth);
  g.theta.resize(g.nth);
  for (int j = 0; j < g.nth; ++j) g.theta[j] = std::acos(xg[g.nth - 1 - j]);  // :71-79
  g.wph = kPi / g.L;
  g.phi.resize(g.nph);
  for (int j = 0; j < g.nph; ++j) g.phi[j] = j * g.wph + 0.5 * g.wph;         // :81-89
  g.khat.resize(3 * static_cast<size_t>(g.K));
  for (int t = 0; t < g.nth; ++t)
    for (int p = 0; p < g.nph; ++p) {
      const size_t k = static_cast<size_t>(t) * g.nph + p;
      g.khat[3 * k] = std::sin(g.theta[t]) * std::cos(g.phi[p]);
      g.khat[3 * k + 1] = std::sin(g.theta[t]) * std::sin(g.phi[p]);
      g.khat[3 * k + 2] = std::cos(g.theta[t]);
    }
  return g;
}

namespace {
// Code/AlgoMLFMM.h:141-189: nearest node by bisection (early exit when within
// 1e-12), then its two neighbours, wrapping around the ends (periodic).
std::array<int, 3> interp_pos(double target, const std::vector<double>& arr) {
  const int n = static_cast<int>(arr.size());
  if (n < 3) return {-1, -1, -1};
  const bool asc = (arr[1] - arr[0]) > 0;
  int lo = 0, hi = n - 1, mid = 0;
  while (lo <= hi) {
    mid = (lo + hi) / 2;
    if (std::abs(arr[mid] - target) < 1e-12) break;
    if (asc) {
      if (arr[mid] > target) hi = mid - 1; else lo = mid + 1;
    } else {
      if (arr[mid] > target) lo = mid + 1; else hi = mid - 1;
    }
  }
  int cl = mid;
  if (mid > 0 && std::abs(arr[mid - 1] - target) < std::abs(arr[cl] - target)) cl = mid - 1;
  if (mid < n - 1 && std::abs(arr[mid + 1] - target) < std::abs(arr[cl] - target)) cl = mid + 1;
  int prev, next;
  if (asc) {
    if (cl == 0) { prev = n - 1; next = 1; }
    else if (cl == n - 1) { prev = cl - 1; next = 0; }
    else { prev = cl - 1; next = cl + 1; }
  } else {
    if (cl == 0) { prev = 1; next = n - 1; }
    else if (cl == n - 1) { prev = 0; next = cl - 1; }
    else { prev = cl + 1; next = cl - 1; }
  }
  return {prev, cl, next};
}
double lagrange(double x0, double x1, double x2, double x3) {
  return ((x0 - x2) * (x0 - x3)) / ((x1 - x2) * (x1 - x3));
}
}  // namespace

Interp build_interp(const Grid& parent, const Grid& child) {
  Interp it;
  it.tidx.resize(3 * parent.nth);
  it.lt.resize(3 * parent.nth);
  it.pidx.resize(3 * parent.nph);
  it.lp.resize(3 * parent.nph);
  for (int t = 0; t < parent.nth; ++t) {
    const double x0 = parent.theta[t];
    const auto id = interp_pos(x0, child.theta);
    const double v0 = child.theta[id[0]], v1 = child.theta[id[1]], v2 = child.theta[id[2]];
    for (int a = 0; a < 3; ++a) it.tidx[3 * t + a] = id[a];
    it.lt[3 * t] = lagrange(x0, v0, v1, v2);
    it.lt[3 * t + 1] = lagrange(x0, v1, v0, v2);
    it.lt[3 * t + 2] = lagrange(x0, v2, v0, v1);
  }
  for (int p = 0; p < parent.nph; ++p) {
    const double x0 = parent.phi[p];
    const auto id = interp_pos(x0, child.phi);
    const double v0 = child.phi[id[0]], v1 = child.phi[id[1]], v2 = child.phi[id[2]];
    for (int a = 0; a < 3; ++a) it.pidx[3 * p + a] = id[a];
    it.lp[3 * p] = lagrange(x0, v0, v1, v2);
    it.lp[3 * p + 1] = lagrange(x0, v1, v0, v2);
    it.lp[3 * p + 2] = lagrange(x0, v2, v0, v1);
  }
  return it;
}

// ---------------------------------------------------------- quadrature ----

namespace {
// Dunavant (1985) symmetric triangle rules with the digits the reference
// tabulates (Code/GaussPoints.cpp:11-284); orbit expansion in the same
// order: centroid; (a,b,b),(b,a,b),(b,b,a); (a,b,c),(a,c,b),(b,a,c),(b,c,a),(c,a,b),(c,b,a).
struct Rule {
  std::vector<double> l1, l2, l3, w;
  void centroid(double c, double wt) { l1.push_back(c); l2.push_back(c); l3.push_back(c); w.push_back(wt); }
  void orbit3(double a, double b, double wt) {
    const double p[3][3] = {{a, b, b}, {b, a, b}, {b, b, a}};
    for (auto& q : p) { l1.push_back(q[0]); l2.push_back(q[1]); l3.push_back(q[2]); w.push_back(wt); }
  }
  void orbit6(double a, double b, double c, double wt) {
    const double p[6][3] = {{a, b, c}, {a, c, b}, {b, a, c}, {b, c, a}, {c, a, b}, {c, b, a}};
    for (auto& q : p) { l1.push_back(q[0]); l2.push_back(q[1]); l3.push_back(q[2]); w.push_back(wt); }
  }
};
const Rule& rule(int n, bool& ok) {
  static std::map<int, Rule> rules = [] {
    std::map<int, Rule> r;
    r[1].centroid(0.333333333333, 0.5);
    r[3].orbit3(0.666666666666667, 0.166666666666667, 0.1666666666666665);
    r[4].centroid(0.333333333333, -0.281250000000000);
    r[4].orbit3(0.6, 0.2, 0.2604166666666665);
    r[6].orbit3(0.108103018168070, 0.445948490915965, 0.111690794839006);
    r[6].orbit3(0.816847572980459, 0.091576213509771, 0.054975871827661);
    r[7].centroid(0.333333333333333, 0.112500000000000);
    r[7].orbit3(0.059715871789770, 0.470142064105115, 0.066197076394253);
    r[7].orbit3(0.797426985353087, 0.101286507323456, 0.0629695902724135);
    r[12].orbit3(0.501426509658179, 0.249286745170910, 0.0583931378631895);
    r[12].orbit3(0.873821971016996, 0.063089014491502, 0.0254224531851035);
    r[12].orbit6(0.053145049844817, 0.310352451033785, 0.636502499121399, 0.041425537809187);
    r[13].centroid(0.333333333333333, -0.074785044733841);
    r[13].orbit3(0.479308067841920, 0.260345966079040, 0.087807628716604);
    r[13].orbit3(0.869739794195568, 0.065130102902216, 0.026673617804419);
    r[13].orbit6(0.048690315425316, 0.312865496004874, 0.638444188569810, 0.0385568804451285);
    r[16].centroid(0.333333333333333, 0.0721578038388935);
    r[16].orbit3(0.081414823414554, 0.459292588292723, 0.0475458171336425);
    r[16].orbit3(0.658861384496480, 0.170569307751760, 0.051608685267359);
    r[16].orbit3(0.898905543365938, 0.050547228317031, 0.016229248811599);
    r[16].orbit6(0.008394777409958, 0.263112829634638, 0.728492392955404, 0.0136151570872175);
    return r;
  }();
  auto it = rules.find(n);
  ok = it != rules.end();
  return ok ? it->second : rules.begin()->second;
}
}  // namespace

bool quad_rule(int n, Quad& q) {
  bool ok = false;
  const Rule& r = rule(n, ok);
  if (!ok) return false;
  q.n = static_cast<int>(r.w.size());
  q.l1 = r.l1.data();
  q.l2 = r.l2.data();
  q.l3 = r.l3.data();
  q.w = r.w.data();
  return true;
}

}  // namespace mlfma
