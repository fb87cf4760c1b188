// Near-field K entries of RWG pairs that share a triangle, evaluated on the
// host with the reference's own arithmetic.
//
// For a field point on its own source triangle, the reference computes the
// point's height above the triangle as D = n.(r - v_i) (Code/Operator.h:
// 582-587). That is zero in exact arithmetic but rounding noise in floating
// point; where the noise exceeds 10 eps0 the 1/R^3 integral takes its 1/|D|
// branch (Code/Operator.h:637-652) and leaves a residue in the K term that is
// set by the last bits of every operation on the way, atan and log included.
// The device near-field kernel evaluates these terms at the exact height 0.
// To reproduce the reference's entries bit for bit instead (plan parameter
// same_triangle_k = 1), this file evaluates the whole K operator of each such
// pair (Code/Operator.h:883-1046, singK :325-707) with std::complex<double>
// in the reference's order of operations, using the host C library's
// exp/log/atan and separately rounded multiplies and adds (this file is built
// with -ffp-contract=off, as the reference's own build never fuses). The
// helper semantics it mirrors are Code/OverloadAlgo.h:18-215 (dot, cross,
// norm: left-to-right sums of componentwise products).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <thread>
#include <vector>

#include "near_same_triangle.hpp"

namespace mlfma {
namespace {

using cd = std::complex<double>;
const cd kJ(0.0, 1.0);  // Code/PhyConstant.h:11

struct V3 {
  double a[3];
  double operator[](int i) const { return a[i]; }
  double& operator[](int i) { return a[i]; }
};

inline V3 vsub(const double* u, const double* v) { return {{u[0] - v[0], u[1] - v[1], u[2] - v[2]}}; }
inline V3 vsub(const V3& u, const V3& v) { return vsub(u.a, v.a); }
inline V3 vmul(const double* u, double c) { return {{u[0] * c, u[1] * c, u[2] * c}}; }
inline V3 vdiv(const V3& u, double c) { return {{u[0] / c, u[1] / c, u[2] / c}}; }
inline double vdot(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }
inline double vdot(const V3& u, const V3& v) { return vdot(u.a, v.a); }
inline double vnorm(const V3& u) { return std::sqrt(vdot(u, u)); }
inline V3 vcross(const double* u, const double* v) {
  return {{u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]}};
}

struct Face {
  const double* v[3];
  const double* n;
  double area;
  int id;
};

struct Geometry {
  const Mesh& m;
  const Rwg& r;
  const Quad& q;
  Face face(int f) const {
    Face t;
    for (int a = 0; a < 3; ++a) t.v[a] = &m.xyz[3 * static_cast<size_t>(m.face_v[3 * f + a])];
    t.n = &m.normal[3 * static_cast<size_t>(f)];
    t.area = m.area[f];
    t.id = m.face_id[f];
    return t;
  }
  const double* point(int p) const { return &m.xyz[3 * static_cast<size_t>(p)]; }
  V3 qpoint(int i, const Face& t) const {
    V3 o;
    for (int a = 0; a < 3; ++a) o[a] = q.l1[i] * t.v[0][a] + q.l2[i] * t.v[1][a] + q.l3[i] * t.v[2][a];
    return o;
  }
};

// The analytic part of the coincident-triangle K integral for field triangle
// F and source triangle S (the same face), Code/Operator.h:325-707.
cd sing_k(const Geometry& g, const Face& F, const double* freeF, double recAf, const Face& S, const double* freeS,
          double recAs, cd k) {
  const double* n = S.n;
  V3 rhoV[3];
  for (int i = 0; i < 3; ++i) {
    const double K = vdot(n, S.v[i]);
    const V3 np = vmul(n, K);
    rhoV[i] = vsub(S.v[i], np.a);
  }
  // edge unit vectors l_i (vertex i to i+1) and outward in-plane normals u_i
  V3 ll[3], u[3];
  for (int i = 0; i < 3; ++i) {
    const V3 d = vsub(rhoV[(i + 1) % 3], rhoV[i]);
    const double len = vnorm(d);
    ll[i] = vdiv(d, len);
    u[i] = vcross(ll[i].a, n);
  }
  cd alok(0.0, 0.0);
  for (int p = 0; p < g.q.n; ++p) {
    const V3 fp = g.qpoint(p, F);
    const double wF = g.q.w[p];
    const double K = vdot(n, fp.a);
    const V3 rho = vsub(fp, vmul(n, K));
    double Lpl[3], Lmn[3], Pnul[3], Ppl[3], Pmn[3], D[3], Rnul[3], Rpl[3], Rmn[3];
    V3 Pnv[3];
    for (int i = 0; i < 3; ++i) {
      const V3 de = vsub(rhoV[(i + 1) % 3], rho);  // edge end vertex - rho
      const V3 ds = vsub(rhoV[i], rho);            // edge start vertex - rho
      Lpl[i] = vdot(de, ll[i]);
      Lmn[i] = vdot(ds, ll[i]);
    }
    for (int i = 0; i < 3; ++i) Pnul[i] = std::abs(vdot(vsub(rhoV[(i + 1) % 3], rho), u[i]));
    for (int i = 0; i < 3; ++i) {
      Ppl[i] = vnorm(vsub(rhoV[(i + 1) % 3], rho));
      Pmn[i] = vnorm(vsub(rhoV[i], rho));
    }
    for (int i = 0; i < 3; ++i) {
      if (Pnul[i] < 50 * kEps0) {
        Pnv[i] = {{0.0, 0.0, 0.0}};
      } else {
        const V3 a = vsub(rhoV[(i + 1) % 3], rho);
        const V3 b = vmul(ll[i].a, Lpl[i]);
        Pnv[i] = vdiv(vsub(a, b), Pnul[i]);
      }
    }
    for (int i = 0; i < 3; ++i) D[i] = vdot(n, vsub(fp.a, S.v[i]).a);
    for (int i = 0; i < 3; ++i) Rnul[i] = std::sqrt(std::pow(Pnul[i], 2) + std::pow(D[i], 2));
    for (int i = 0; i < 3; ++i) Rpl[i] = std::sqrt(std::pow(Ppl[i], 2) + std::pow(D[i], 2));
    for (int i = 0; i < 3; ++i) Rmn[i] = std::sqrt(std::pow(Pmn[i], 2) + std::pow(D[i], 2));

    auto logs = [&](int i, double& lp, double& lm) {
      lp = (Rpl[i] + Lpl[i]) < 50 * kEps0 ? 0.0 : std::log(Rpl[i] + Lpl[i]);
      lm = (Rmn[i] + Lmn[i]) < 50 * kEps0 ? 0.0 : std::log(Rmn[i] + Lmn[i]);
    };
    V3 Iv1 = {{0.0, 0.0, 0.0}}, Iv3 = {{0.0, 0.0, 0.0}};
    double Is1 = 0.0, Is3 = 0.0;
    // vector part of the 1/R integral
    for (int i = 0; i < 3; ++i) {
      double lp, lm;
      logs(i, lp, lm);
      const double c1 = 0.5 * (std::pow(Rnul[i], 2) * (lp - lm) + Rpl[i] * Lpl[i] - Rmn[i] * Lmn[i]);
      const V3 t = vmul(u[i].a, c1);
      for (int a = 0; a < 3; ++a) Iv1[a] = Iv1[a] + t[a];
    }
    // scalar part of the 1/R integral
    for (int i = 0; i < 3; ++i) {
      double lp, lm;
      logs(i, lp, lm);
      const double aD = std::abs(D[i]);
      const double atp = (std::pow(Rnul[i], 2) + aD * Rpl[i]) < 50 * kEps0
                             ? 0.0
                             : std::atan((Pnul[i] * Lpl[i]) / (std::pow(Rnul[i], 2) + aD * Rpl[i]));
      const double atm = (std::pow(Rnul[i], 2) + aD * Rmn[i]) < 50 * kEps0
                             ? 0.0
                             : std::atan((Pnul[i] * Lmn[i]) / (std::pow(Rnul[i], 2) + aD * Rmn[i]));
      Is1 = Is1 + vdot(Pnv[i], u[i]) * (Pnul[i] * (lp - lm) - aD * (atp - atm));
    }
    // vector part of the 1/R^3 integral
    for (int i = 0; i < 3; ++i) {
      double lp, lm;
      logs(i, lp, lm);
      const double c1 = lp - lm;
      const V3 t = vmul(u[i].a, c1);
      for (int a = 0; a < 3; ++a) Iv3[a] = Iv3[a] - t[a];
    }
    // scalar part of the 1/R^3 integral; the last branch resets the sum
    for (int i = 0; i < 3; ++i) {
      const double aD = std::abs(D[i]);
      if (aD >= 10.0 * kEps0) {
        const double atp = std::atan((Pnul[i] * Lpl[i]) / (std::pow(Rnul[i], 2) + aD * Rpl[i]));
        const double atm = std::atan((Pnul[i] * Lmn[i]) / (std::pow(Rnul[i], 2) + aD * Rmn[i]));
        Is3 = Is3 + vdot(Pnv[i], u[i]) * ((1.0 / aD) * (atp - atm));
      } else if (aD < 10.0 * kEps0 && Pnul[i] >= 10.0 * kEps0) {
        Is3 = Is3 - vdot(Pnv[i], u[i]) * (Lpl[i] / (Pnul[i] * Rpl[i]) - Lmn[i] / (Pnul[i] * Rmn[i]));
      } else {
        Is3 = 0.0;
      }
    }
    // Galerkin testing with the field RWG
    const V3 RWGf = vmul(vsub(fp.a, freeF).a, recAf);
    const V3 Riv = vsub(fp.a, freeS);
    const double K1 = vdot(n, freeS);
    const V3 rho0N = vsub(freeS, vmul(n, K1).a);
    const V3 pv1 = vsub(rho, rho0N);
    const cd konst1 = k * k * 0.5;
    const cd konst2 = konst1 * Is1;
    cd Ikon[3];
    for (int a = 0; a < 3; ++a) {
      const cd v2 = Iv1[a] * konst1;
      const cd v3 = pv1[a] * konst2;
      const cd v4 = v2 + v3;
      const cd ik1 = v4 * recAs;
      const double v5 = pv1[a] * Is3;
      const double v6 = Iv3[a] + v5;
      const double ik3 = v6 * recAs;
      Ikon[a] = ik3 + ik1;
    }
    const cd kr[3] = {Riv[1] * Ikon[2] - Riv[2] * Ikon[1], Riv[2] * Ikon[0] - Riv[0] * Ikon[2],
                      Riv[0] * Ikon[1] - Riv[1] * Ikon[0]};
    const cd dK = RWGf[0] * kr[0] + RWGf[1] * kr[1] + RWGf[2] * kr[2];
    alok += wF * 2.0 * F.area * dK;
  }
  return alok;
}

// K operator of one RWG pair at wavenumber k (Code/Operator.h:883-1046).
cd k_operator(const Geometry& g, int fld, int src, cd k) {
  cd Z(0.0, 0.0);
  const double lF = g.r.len[fld], lS = g.r.len[src];
  for (int fi = 0; fi < 2; ++fi) {  // 0 = T-, 1 = T+
    const Face F = g.face(fi == 0 ? g.r.fneg[fld] : g.r.fpos[fld]);
    const double* freeF = g.point(fi == 0 ? g.r.free_neg[fld] : g.r.free_pos[fld]);
    const double recAf = 1.0 / (2.0 * F.area);
    for (int sj = 0; sj < 2; ++sj) {
      const Face S = g.face(sj == 0 ? g.r.fneg[src] : g.r.fpos[src]);
      const double* freeS = g.point(sj == 0 ? g.r.free_neg[src] : g.r.free_pos[src]);
      const double recAs = 1.0 / (2.0 * S.area);
      const bool same = F.id == S.id;
      cd alok1(0.0, 0.0);
      for (int i = 0; i < g.q.n; ++i) {
        const V3 fp = g.qpoint(i, F);
        const double wF = g.q.w[i];
        for (int j = 0; j < g.q.n; ++j) {
          const V3 sp = g.qpoint(j, S);
          const double wS = g.q.w[j];
          const V3 Rv = vsub(fp, sp);
          const double R = std::sqrt(Rv[0] * Rv[0] + Rv[1] * Rv[1] + Rv[2] * Rv[2]);
          cd G;
          if (!same) {
            G = (std::exp(-kJ * k * R) / (R * R * R)) * (1.0 + kJ * k * R);
          } else if (R < kEps0) {
            G = cd(0.0, 0.0);
          } else {
            G = (std::exp(-kJ * k * R) / (R * R * R)) * (1.0 + kJ * k * R) - 1.0 / (R * R * R) -
                0.5 * (k * k) * (1.0 / R);
          }
          const V3 pF = vsub(fp.a, freeF);
          const V3 pS = vsub(sp.a, freeS);
          const V3 cr = vcross(Rv.a, pS.a);
          const cd contrib = wF * wS * G * vdot(pF, cr);
          alok1 += contrib;
        }
      }
      if (same) alok1 += sing_k(g, F, freeF, recAf, S, freeS, recAs, k);
      const double sF = (fi == 0) ? -1.0 : 1.0;
      const double sS = (sj == 0) ? -1.0 : 1.0;
      Z += sF * sS * (lF * lS) / (4.0 * kPi) * alok1;
    }
  }
  return Z;
}

bool share_a_face(const Rwg& r, int a, int b) {
  return r.fpos[a] == r.fpos[b] || r.fpos[a] == r.fneg[b] || r.fneg[a] == r.fpos[b] || r.fneg[a] == r.fneg[b];
}

}  // namespace

void same_triangle_pairs(const Rwg& r, const Tree& t, const std::vector<int>& near_sptr,
                         const std::vector<int>& near_src, const std::vector<long long>& near_zoff,
                         std::vector<long long>& pos, std::vector<int>& tgt, std::vector<int>& src) {
  pos.clear();
  tgt.clear();
  src.clear();
  const int B = static_cast<int>(near_sptr.size()) - 1;
  for (int b = 0; b < B; ++b) {
    const int ns = near_sptr[b + 1] - near_sptr[b];
    for (int ti = t.leaf_ptr[b]; ti < t.leaf_ptr[b + 1]; ++ti) {
      const int tr = t.leaf_rwg[ti];
      for (int si = 0; si < ns; ++si) {
        const int sr = near_src[near_sptr[b] + si];
        if (!share_a_face(r, tr, sr)) continue;
        pos.push_back(near_zoff[b] + static_cast<long long>(ti - t.leaf_ptr[b]) * ns + si);
        tgt.push_back(tr);
        src.push_back(sr);
      }
    }
  }
}

void same_triangle_z12(const Mesh& m, const Rwg& r, const Quad& q, cplx k1, cplx k2, const std::vector<int>& tgt,
                       const std::vector<int>& src, std::vector<cplx>& z12) {
  const Geometry g{m, r, q};
  const size_t n = tgt.size();
  z12.assign(n, cplx(0.0, 0.0));
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nth = static_cast<unsigned>(std::min<size_t>(hw, std::max<size_t>(1, n / 64)));
  std::atomic<size_t> next{0};
  auto work = [&] {
    for (;;) {
      const size_t i0 = next.fetch_add(256);
      if (i0 >= n) return;
      const size_t i1 = std::min(n, i0 + 256);
      for (size_t i = i0; i < i1; ++i) {
        const cd ZK1 = k_operator(g, tgt[i], src[i], k1);
        const cd ZK2 = k_operator(g, tgt[i], src[i], k2);
        z12[i] = -(ZK1 + ZK2);  // Code/Zmartix.h:612
      }
    }
  };
  std::vector<std::thread> pool;
  for (unsigned i = 1; i < nth; ++i) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}

}  // namespace mlfma
