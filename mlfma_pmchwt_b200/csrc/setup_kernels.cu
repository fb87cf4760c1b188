// Operator setup on the GPU, FP64:
//  * leaf radiation / receive patterns (Code/ProcessFMM.h:17-146, 217-233),
//  * transfer factors (Code/AlgoMLFMM.h:192-295),
//  * near-field PMCHWT entries from the RWG L and K operators with the
//    analytic extraction of the 1/R and 1/R^3 parts on coincident triangles
//    (Code/Operator.h:10-1046, assembled as Code/Zmartix.h:541-643).
#include <algorithm>
#include "cplx.cuh"
#include "plan.hpp"

namespace mlfma {

namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kEps0D = 2.2204e-16;

struct QuadArg {
  int n;
  double l1[16], l2[16], l3[16], w[16];
};

QuadArg quad_arg(const Quad& q) {
  QuadArg a{};
  a.n = q.n;
  for (int i = 0; i < q.n; ++i) {
    a.l1[i] = q.l1[i];
    a.l2[i] = q.l2[i];
    a.l3[i] = q.l3[i];
    a.w[i] = q.w[i];
  }
  return a;
}

struct GeomArg {
  const double* xyz;
  const int* face_v;
  const int* face_id;
  const double* face_area;
  const double* face_normal;
  const int* fpos;
  const int* fneg;
  const int* vpos;
  const int* vneg;
  const double* len;
};

__host__ __device__ __forceinline__ void load3(const double* p, double* o) {
  o[0] = p[0];
  o[1] = p[1];
  o[2] = p[2];
}

__host__ __device__ __forceinline__ void qpoint(const QuadArg& q, int i, const double* a, const double* b,
                                       const double* c, double* r) {
  r[0] = q.l1[i] * a[0] + q.l2[i] * b[0] + q.l3[i] * c[0];
  r[1] = q.l1[i] * a[1] + q.l2[i] * b[1] + q.l3[i] * c[1];
  r[2] = q.l1[i] * a[2] + q.l2[i] * b[2] + q.l3[i] * c[2];
}

// ------------------------------------------------------------ patterns ----
// One thread per (RWG in leaf order, leaf direction). Vs = sum over the 7
// (or n) points of T+ minus T- of w l e^{-j k khat.(c - r)} (r - v_free);
// Vf = sum of w l e^{-j k khat.(r - c)} (-(khat x (khat x (r - v_free)))).
__global__ void patterns_kernel(GeomArg g, QuadArg q, const int* __restrict__ leaf_rwg,
                                const int* __restrict__ rwg_leaf_box, const double* __restrict__ box_center,
                                const double* __restrict__ khat, int K, int N, double2 k,
                                double2* __restrict__ Vs, double2* __restrict__ Vf) {
  const int kk = blockIdx.y * blockDim.x + threadIdx.x;
  const int r = blockIdx.x;
  if (kk >= K || r >= N) return;
  const int id = leaf_rwg[r];
  const int b = rwg_leaf_box[id];
  const double ctr[3] = {box_center[3 * b], box_center[3 * b + 1], box_center[3 * b + 2]};
  const double kp[3] = {khat[kk], khat[K + kk], khat[2 * K + kk]};
  const double l = g.len[id];
  double tp[3][3], tn[3][3], fp[3], fn[3];
  const int Fp = g.fpos[id], Fn = g.fneg[id];
  for (int a = 0; a < 3; ++a) {
    load3(&g.xyz[3 * g.face_v[3 * Fp + a]], tp[a]);
    load3(&g.xyz[3 * g.face_v[3 * Fn + a]], tn[a]);
  }
  load3(&g.xyz[3 * g.vpos[id]], fp);
  load3(&g.xyz[3 * g.vneg[id]], fn);
  double2 s[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
  double2 f[3] = {c2(0, 0), c2(0, 0), c2(0, 0)};
  for (int i = 0; i < q.n; ++i) {
    const double w = q.w[i] * l;
    for (int side = 0; side < 2; ++side) {
      double rq[3];
      qpoint(q, i, side ? tn[0] : tp[0], side ? tn[1] : tp[1], side ? tn[2] : tp[2], rq);
      const double* fv = side ? fn : fp;
      const double pf[3] = {rq[0] - fv[0], rq[1] - fv[1], rq[2] - fv[2]};
      // radiation: p = c - r
      const double ps[3] = {ctr[0] - rq[0], ctr[1] - rq[1], ctr[2] - rq[2]};
      const double2 es = cexp_mjkt(k, ps[0] * kp[0] + ps[1] * kp[1] + ps[2] * kp[2]);
      // receive: p = r - c
      const double pr[3] = {rq[0] - ctr[0], rq[1] - ctr[1], rq[2] - ctr[2]};
      const double2 er = cexp_mjkt(k, pr[0] * kp[0] + pr[1] * kp[1] + pr[2] * kp[2]);
      const double t1[3] = {kp[1] * pf[2] - kp[2] * pf[1], kp[2] * pf[0] - kp[0] * pf[2],
                            kp[0] * pf[1] - kp[1] * pf[0]};
      const double t2[3] = {kp[1] * t1[2] - kp[2] * t1[1], kp[2] * t1[0] - kp[0] * t1[2],
                            kp[0] * t1[1] - kp[1] * t1[0]};
      const double2 ws = cscale(es, w), wr = cscale(er, w);
      const double sg = side ? -1.0 : 1.0;
      for (int c = 0; c < 3; ++c) {
        s[c] = cfmas(sg, cscale(ws, pf[c]), s[c]);
        f[c] = cfmas(sg, cscale(wr, -t2[c]), f[c]);
      }
    }
  }
  for (int c = 0; c < 3; ++c) {
    Vs[(static_cast<size_t>(r) * 3 + c) * K + kk] = s[c];
    Vf[(static_cast<size_t>(r) * 3 + c) * K + kk] = f[c];
  }
}

// ------------------------------------------------------- transfer factors ----
// One thread per (vector, direction): sum_{l<=L'} (-j)^l (2l+1) h2_l(|kR|) P_l(Rhat.khat),
// P_l by the three-term recurrence; optionally times the quadrature weight
// w_theta(t) * dphi.
__global__ void transfer_kernel(const double* __restrict__ rhat, const int* __restrict__ hoff,
                                const int* __restrict__ hL, const double2* __restrict__ h2,
                                const double* __restrict__ khat, const double* __restrict__ wth,
                                double wph, int nph, int K, int nvec, int weighted,
                                double2* __restrict__ out) {
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (kk >= K || v >= nvec) return;
  const double x = rhat[3 * v] * khat[kk] + rhat[3 * v + 1] * khat[K + kk] + rhat[3 * v + 2] * khat[2 * K + kk];
  const int L = hL[v];
  const double2* h = h2 + hoff[v];
  double2 sum = c2(0.0, 0.0);
  double pm1 = 1.0, p = x;
  for (int l = 0; l <= L; ++l) {
    double pl;
    if (l == 0) pl = 1.0;
    else if (l == 1) pl = x;
    else {
      const int n = l - 1;
      const double pn1 = ((2.0 * n + 1.0) * x * p - n * pm1) / (n + 1.0);
      pm1 = p;
      p = pn1;
      pl = p;
    }
    double2 t = h[l];
    switch (l & 3) {  // (-j)^l * h2_l
      case 1: t = c2(t.y, -t.x); break;
      case 2: t = c2(-t.x, -t.y); break;
      case 3: t = c2(-t.y, t.x); break;
      default: break;
    }
    sum = cadd(sum, cscale(cscale(t, 2.0 * l + 1.0), pl));
  }
  if (weighted) sum = cscale(sum, wth[kk / nph] * wph);
  out[static_cast<size_t>(v) * K + kk] = sum;
}

// ------------------------------------------------------------ near field ----

struct Tri {
  double v[3][3];
  double area;
  double n[3];
  int id;
};

__host__ __device__ __forceinline__ void load_tri(const GeomArg& g, int f, Tri& t) {
  for (int a = 0; a < 3; ++a) load3(&g.xyz[3 * g.face_v[3 * f + a]], t.v[a]);
  t.area = g.face_area[f];
  load3(&g.face_normal[3 * f], t.n);
  t.id = g.face_id[f];
}

__host__ __device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__host__ __device__ __forceinline__ double norm3(const double* a) { return sqrt(dot3(a, a)); }
__host__ __device__ __forceinline__ void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Analytic source-triangle integrals of 1/R (vector Iv1, scalar Is1) and of
// the 1/R^3 kernel (vector Iv3, scalar Is3) seen from field point r, over the
// source triangle S projected on its plane (Code/Operator.h:10-323 singL and
// :325-707 singK share this geometry).
struct SingGeom {
  double rho[3];     // field point projected on the source plane
  double Iv1[3], Is1, Iv3[3], Is3;
};

// in_plane: r is a point of S itself (the same-triangle term), so its height
// above the source plane is exactly zero. The reference computes that height
// as n.(r - v_i), whose roundoff (~1e-15 for coordinates of order 1) can
// exceed its 10 eps0 threshold; it then takes the 1/|D| branch of the 1/R^3
// integral, whose ~1e15-sized result should cancel in the K term (exactly
// zero for a flat triangle) but leaves a residue set by the last bits of
// atan. Using D = 0 there evaluates the reference's formulas at the exact
// height: the same result wherever the reference stays below its threshold.
__host__ __device__ void sing_geometry(const Tri& S, const double* r, SingGeom& o, bool in_plane) {
  const double* nS = S.n;
  double rho_v[3][3];
  for (int i = 0; i < 3; ++i) {
    const double K = dot3(nS, S.v[i]);
    for (int a = 0; a < 3; ++a) rho_v[i][a] = S.v[i][a] - nS[a] * K;
  }
  double ll[3][3], u[3][3];
  for (int i = 0; i < 3; ++i) {
    const double* from = rho_v[i];
    const double* to = rho_v[(i + 1) % 3];
    double d[3] = {to[0] - from[0], to[1] - from[1], to[2] - from[2]};
    const double nn = norm3(d);
    for (int a = 0; a < 3; ++a) ll[i][a] = d[a] / nn;
    cross3(ll[i], nS, u[i]);
  }
  const double K = dot3(nS, r);
  for (int a = 0; a < 3; ++a) o.rho[a] = r[a] - nS[a] * K;
  const double* rho = o.rho;
  double Lpl[3], Lmn[3], Pnul[3], Ppl[3], Pmn[3], Pv[3][3], D[3];
  for (int i = 0; i < 3; ++i) {
    const double* pe = rho_v[(i + 1) % 3];   // end vertex of edge i
    const double* ps = rho_v[i];             // start vertex of edge i
    const double de[3] = {pe[0] - rho[0], pe[1] - rho[1], pe[2] - rho[2]};
    const double ds[3] = {ps[0] - rho[0], ps[1] - rho[1], ps[2] - rho[2]};
    Lpl[i] = dot3(de, ll[i]);
    Lmn[i] = dot3(ds, ll[i]);
    Pnul[i] = fabs(dot3(de, u[i]));
    Ppl[i] = norm3(de);
    Pmn[i] = norm3(ds);
    if (Pnul[i] < 50 * kEps0D) {
      Pv[i][0] = Pv[i][1] = Pv[i][2] = 0.0;
    } else {
      for (int a = 0; a < 3; ++a) Pv[i][a] = (de[a] - ll[i][a] * Lpl[i]) / Pnul[i];
    }
    const double dv[3] = {r[0] - S.v[i][0], r[1] - S.v[i][1], r[2] - S.v[i][2]};
    D[i] = in_plane ? 0.0 : dot3(nS, dv);
  }
  for (int a = 0; a < 3; ++a) {
    o.Iv1[a] = 0.0;
    o.Iv3[a] = 0.0;
  }
  o.Is1 = 0.0;
  o.Is3 = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double Rnul = sqrt(Pnul[i] * Pnul[i] + D[i] * D[i]);
    const double Rpl = sqrt(Ppl[i] * Ppl[i] + D[i] * D[i]);
    const double Rmn = sqrt(Pmn[i] * Pmn[i] + D[i] * D[i]);
    const double LOGpl = (Rpl + Lpl[i]) < 50 * kEps0D ? 0.0 : log(Rpl + Lpl[i]);
    const double LOGmn = (Rmn + Lmn[i]) < 50 * kEps0D ? 0.0 : log(Rmn + Lmn[i]);
    const double aD = fabs(D[i]);
    const double c1 = 0.5 * (Rnul * Rnul * (LOGpl - LOGmn) + Rpl * Lpl[i] - Rmn * Lmn[i]);
    for (int a = 0; a < 3; ++a) o.Iv1[a] += u[i][a] * c1;
    const double den_pl = Rnul * Rnul + aD * Rpl, den_mn = Rnul * Rnul + aD * Rmn;
    const double ATpl = den_pl < 50 * kEps0D ? 0.0 : atan((Pnul[i] * Lpl[i]) / den_pl);
    const double ATmn = den_mn < 50 * kEps0D ? 0.0 : atan((Pnul[i] * Lmn[i]) / den_mn);
    const double pu = dot3(Pv[i], u[i]);
    o.Is1 += pu * (Pnul[i] * (LOGpl - LOGmn) - aD * (ATpl - ATmn));
    for (int a = 0; a < 3; ++a) o.Iv3[a] -= u[i][a] * (LOGpl - LOGmn);
    // 1/R^3 scalar term (Code/Operator.h:637-652); the last branch resets
    // the running sum, as the reference does.
    if (aD >= 10.0 * kEps0D) {
      const double a1 = atan((Pnul[i] * Lpl[i]) / den_pl);
      const double a2 = atan((Pnul[i] * Lmn[i]) / den_mn);
      o.Is3 += pu * ((1.0 / aD) * (a1 - a2));
    } else if (Pnul[i] >= 10.0 * kEps0D) {
      o.Is3 -= pu * (Lpl[i] / (Pnul[i] * Rpl) - Lmn[i] / (Pnul[i] * Rmn));
    } else {
      o.Is3 = 0.0;
    }
  }
}

// The four PMCHWT operator values for one RWG pair:
// out[0] = L(k1), out[1] = L(k2), out[2] = K(k1), out[3] = K(k2).
__host__ __device__ void rwg_pair_ops(const GeomArg& g, const QuadArg& q, int fld, int src, double2 k1,
                             double2 k2, double2 out[4]) {
  const double2 ks[2] = {k1, k2};
  for (int i = 0; i < 4; ++i) out[i] = c2(0.0, 0.0);
  const double lF = g.len[fld], lS = g.len[src];
  for (int fi = 0; fi < 2; ++fi) {  // 0 = T-, 1 = T+
    Tri F;
    load_tri(g, fi == 0 ? g.fneg[fld] : g.fpos[fld], F);
    double vF[3];
    load3(&g.xyz[3 * (fi == 0 ? g.vneg[fld] : g.vpos[fld])], vF);
    const double recAf = 1.0 / (2.0 * F.area);
    for (int sj = 0; sj < 2; ++sj) {
      Tri S;
      load_tri(g, sj == 0 ? g.fneg[src] : g.fpos[src], S);
      double vS[3];
      load3(&g.xyz[3 * (sj == 0 ? g.vneg[src] : g.vpos[src])], vS);
      const double recAs = 1.0 / (2.0 * S.area);
      const bool same = F.id == S.id;
      double2 aL[2] = {c2(0, 0), c2(0, 0)}, aK[2] = {c2(0, 0), c2(0, 0)};
      for (int p = 0; p < q.n; ++p) {
        double rF[3];
        qpoint(q, p, F.v[0], F.v[1], F.v[2], rF);
        const double wF = q.w[p];
        const double pF[3] = {rF[0] - vF[0], rF[1] - vF[1], rF[2] - vF[2]};
        const double RWGf[3] = {pF[0] * recAf, pF[1] * recAf, pF[2] * recAf};
        for (int qq = 0; qq < q.n; ++qq) {
          double rS[3];
          qpoint(q, qq, S.v[0], S.v[1], S.v[2], rS);
          const double wS = q.w[qq];
          const double Rv[3] = {rF[0] - rS[0], rF[1] - rS[1], rF[2] - rS[2]};
          const double R = sqrt(Rv[0] * Rv[0] + Rv[1] * Rv[1] + Rv[2] * Rv[2]);
          const double pS[3] = {rS[0] - vS[0], rS[1] - vS[1], rS[2] - vS[2]};
          const double RWGs[3] = {pS[0] * recAs, pS[1] * recAs, pS[2] * recAs};
          double cr[3];
          cross3(Rv, pS, cr);
          const double fdot = dot3(RWGf, RWGs);
          const double kdot = dot3(pF, cr);
          for (int m = 0; m < 2; ++m) {
            const double2 k = ks[m];
            double2 GL, GK;
            if (!same) {
              const double2 e = cexp_mjkt(k, R);
              GL = cscale(e, 1.0 / R);
              // e / R^3 * (1 + j k R)
              GK = cmul(cscale(e, 1.0 / (R * R * R)), c2(1.0 - k.y * R, k.x * R));
            } else if (R < kEps0D) {
              GL = c2(k.y, -k.x);  // -j k
              GK = c2(0.0, 0.0);
            } else {
              const double2 e = cexp_mjkt(k, R);
              GL = csub(cscale(e, 1.0 / R), c2(1.0 / R, 0.0));
              const double2 k2v = cmul(k, k);
              GK = cmul(cscale(e, 1.0 / (R * R * R)), c2(1.0 - k.y * R, k.x * R));
              GK = csub(GK, c2(1.0 / (R * R * R), 0.0));
              GK = csub(GK, cscale(k2v, 0.5 * (1.0 / R)));
            }
            // L: j k wF wS 4 AF AS (G RWGf.RWGs - G / (k^2 AF AS))
            const double2 jk = cmulj(k);
            const double2 ik2 = cdiv(c2(1.0, 0.0), cmul(k, k));
            const double2 br = csub(cscale(GL, fdot), cscale(cmul(ik2, GL), 1.0 / (F.area * S.area)));
            aL[m] = cadd(aL[m], cmul(cscale(jk, wF * wS * 4.0 * F.area * S.area), br));
            // K: wF wS G (pF . (Rvec x pS))
            aK[m] = cadd(aK[m], cscale(GK, wF * wS * kdot));
          }
        }
      }
      if (same) {
        // Analytic parts over the source triangle for each field point.
        double rho0N[3];
        {
          const double K = dot3(S.n, vS);
          for (int a = 0; a < 3; ++a) rho0N[a] = vS[a] - S.n[a] * K;
        }
        for (int p = 0; p < q.n; ++p) {
          double rF[3];
          qpoint(q, p, F.v[0], F.v[1], F.v[2], rF);
          const double wF = q.w[p];
          SingGeom sg;
          sing_geometry(S, rF, sg, true);
          const double RWGf[3] = {(rF[0] - vF[0]) * recAf, (rF[1] - vF[1]) * recAf, (rF[2] - vF[2]) * recAf};
          const double pv1[3] = {sg.rho[0] - rho0N[0], sg.rho[1] - rho0N[1], sg.rho[2] - rho0N[2]};
          // singL (Code/Operator.h:301-321)
          double Ikon[3];
          for (int a = 0; a < 3; ++a) Ikon[a] = (sg.Iv1[a] + pv1[a] * sg.Is1) * recAs;
          const double dL = dot3(RWGf, Ikon);
          // singK (Code/Operator.h:655-704)
          const double Riv[3] = {rF[0] - vS[0], rF[1] - vS[1], rF[2] - vS[2]};
          double I3[3];
          for (int a = 0; a < 3; ++a) I3[a] = (sg.Iv3[a] + pv1[a] * sg.Is3) * recAs;
          for (int m = 0; m < 2; ++m) {
            const double2 k = ks[m];
            const double2 ik2 = cdiv(c2(1.0, 0.0), cmul(k, k));
            const double2 brL = csub(c2(dL, 0.0), cscale(ik2, (1.0 / (F.area * S.area)) * sg.Is1));
            aL[m] = cadd(aL[m], cmul(cscale(cmulj(k), wF * 2.0 * F.area), brL));
            const double2 konst1 = cscale(cmul(k, k), 0.5);
            const double2 konst2 = cscale(konst1, sg.Is1);
            double2 Ik[3];
            for (int a = 0; a < 3; ++a) {
              const double2 v1 = cadd(cscale(konst1, sg.Iv1[a]), cscale(konst2, pv1[a]));
              Ik[a] = cadd(c2(I3[a], 0.0), cscale(v1, recAs));
            }
            // Rivec x Ikon (real x complex)
            const double2 kr0 = csub(cscale(Ik[2], Riv[1]), cscale(Ik[1], Riv[2]));
            const double2 kr1 = csub(cscale(Ik[0], Riv[2]), cscale(Ik[2], Riv[0]));
            const double2 kr2 = csub(cscale(Ik[1], Riv[0]), cscale(Ik[0], Riv[1]));
            const double2 dK = cadd(cadd(cscale(kr0, RWGf[0]), cscale(kr1, RWGf[1])), cscale(kr2, RWGf[2]));
            aK[m] = cadd(aK[m], cscale(dK, wF * 2.0 * F.area));
          }
        }
      }
      const double sgn = (fi == 0 ? -1.0 : 1.0) * (sj == 0 ? -1.0 : 1.0);
      const double scl = (lF * lS) / (4.0 * kPiD) * sgn;
      for (int m = 0; m < 2; ++m) {
        out[m] = cadd(out[m], cscale(aL[m], scl));
        out[2 + m] = cadd(out[2 + m], cscale(aK[m], scl));
      }
    }
  }
}

// One block per leaf box; threads loop over the box's (target, source) pairs.
__global__ void near_kernel(GeomArg g, QuadArg q, const int* __restrict__ leaf_ptr,
                            const int* __restrict__ leaf_rwg, const int* __restrict__ sptr,
                            const int* __restrict__ src, const long long* __restrict__ zoff,
                            double2 k1, double2 k2, double2 etai, double2* __restrict__ Z) {
  const int b = blockIdx.x;
  const int nt = leaf_ptr[b + 1] - leaf_ptr[b];
  const int ns = sptr[b + 1] - sptr[b];
  const long long base = zoff[b];
  const double2 ietai = cdiv(c2(1.0, 0.0), etai);
  for (int e = threadIdx.x; e < nt * ns; e += blockDim.x) {
    const int t = leaf_rwg[leaf_ptr[b] + e / ns];
    const int s = src[sptr[b] + e % ns];
    double2 op[4];
    rwg_pair_ops(g, q, t, s, k1, k2, op);
    const double2 z11 = cadd(op[0], cmul(etai, op[1]));
    const double2 z12 = cneg(cadd(op[2], op[3]));
    const double2 z22 = cadd(op[0], cmul(ietai, op[1]));
    double2* zp = Z + 3 * (base + e);
    zp[0] = z11;
    zp[1] = z12;
    zp[2] = z22;
  }
}

GeomArg geom_arg(const Plan& P) {
  return GeomArg{P.d_xyz,      P.d_face_v,   P.d_face_id,  P.d_face_area, P.d_face_normal,
                 P.d_rwg_fpos, P.d_rwg_fneg, P.d_rwg_vpos, P.d_rwg_vneg,  P.d_rwg_len};
}

}  // namespace

namespace {
__global__ void to_c64_kernel(const double2* __restrict__ src, float2* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    dst[i] = make_float2(static_cast<float>(src[i].x), static_cast<float>(src[i].y));
}
}  // namespace

void to_c64(const double2* src, float2* dst, size_t n, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
  to_c64_kernel<<<std::max(blocks, 1), 256, 0, s>>>(src, dst, n);
  MLFMA_CUDA(cudaGetLastError());
}

void launch_patterns(Plan& P, int medium, cudaStream_t s) {
  const MediumLevel& M = P.ml[medium][P.maxL];
  const DevLevel& L = P.lv[P.maxL];
  (void)L;
  const cplx k = medium == 0 ? P.k1 : P.k2;
  dim3 block(128), grid(P.N, (M.K + 127) / 128);
  // box of each RWG and the leaf centres
  static_assert(sizeof(double2) == 2 * sizeof(double), "layout");
  patterns_kernel<<<grid, block, 0, s>>>(geom_arg(P), quad_arg(P.quad), P.d_leaf_rwg, P.d_rwg_leafbox,
                                         P.d_leaf_center, M.khat, M.K, P.N, c2(k.real(), k.imag()),
                                         P.d_Vs[medium], P.d_Vf[medium]);
  MLFMA_CUDA(cudaGetLastError());
}

void launch_transfer(Plan& P, int medium, int level, const std::vector<double>& rhat,
                     const std::vector<int>& hoff, const std::vector<int>& hL,
                     const std::vector<double2>& h2, bool weighted, double2* out, cudaStream_t s, bool in_heap) {
  const MediumLevel& M = P.ml[medium][level];
  const int nvec = static_cast<int>(hL.size());
  if (nvec == 0) return;
  // one device block for the five inputs, each part 256-byte aligned
  auto part = [](size_t bytes) { return (bytes + 255) & ~size_t(255); };
  const size_t b_rhat = part(rhat.size() * sizeof(double)), b_hoff = part(hoff.size() * sizeof(int)),
               b_hL = part(hL.size() * sizeof(int)), b_h2 = part(h2.size() * sizeof(double2));
  const size_t total = b_rhat + b_hoff + b_hL + b_h2 + part(M.grid.wth.size() * sizeof(double));
  char* blk = nullptr;
  if (in_heap)
    blk = P.alloc<char>(total);
  else
    MLFMA_CUDA(cudaMalloc(&blk, total));
  struct Owned {
    char* p;
    ~Owned() {
      if (p) cudaFree(p);
    }
  } owned{in_heap ? nullptr : blk};
  double* d_rhat = reinterpret_cast<double*>(blk);
  int* d_hoff = reinterpret_cast<int*>(blk + b_rhat);
  int* d_hL = reinterpret_cast<int*>(blk + b_rhat + b_hoff);
  double2* d_h2 = reinterpret_cast<double2*>(blk + b_rhat + b_hoff + b_hL);
  double* d_wth = reinterpret_cast<double*>(blk + b_rhat + b_hoff + b_hL + b_h2);
  MLFMA_CUDA(cudaMemcpyAsync(d_rhat, rhat.data(), rhat.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(d_hoff, hoff.data(), hoff.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(d_hL, hL.data(), hL.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(d_h2, h2.data(), h2.size() * sizeof(double2), cudaMemcpyHostToDevice, s));
  MLFMA_CUDA(cudaMemcpyAsync(d_wth, M.grid.wth.data(), M.grid.wth.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s));
  dim3 block(128), grid((M.K + 127) / 128, nvec);
  transfer_kernel<<<grid, block, 0, s>>>(d_rhat, d_hoff, d_hL, d_h2, M.khat, d_wth, M.grid.wph, M.nph,
                                         M.K, nvec, weighted ? 1 : 0, out);
  MLFMA_CUDA(cudaGetLastError());
  MLFMA_CUDA(cudaStreamSynchronize(s));
}

__global__ void near_z12_scatter_kernel(double2* __restrict__ Z, const long long* __restrict__ pos,
                                        const double2* __restrict__ z12, long long n) {
  const long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (i < n) Z[3 * pos[i] + 1] = z12[i];
}

void launch_near_z12_scatter(double2* Z, const long long* pos, const double2* z12, long long n, cudaStream_t s) {
  if (n <= 0) return;
  near_z12_scatter_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(Z, pos, z12, n);
  MLFMA_CUDA(cudaGetLastError());
}

void launch_near(Plan& P, cudaStream_t s) {
  const int B = P.lv[P.maxL].B;
  near_kernel<<<B, 128, 0, s>>>(geom_arg(P), quad_arg(P.quad), P.d_leaf_ptr, P.d_leaf_rwg, P.d_near_sptr,
                                P.d_near_src, P.d_near_zoff, c2(P.k1.real(), P.k1.imag()),
                                c2(P.k2.real(), P.k2.imag()), c2(P.etai.real(), P.etai.imag()),
                                P.d_near_z);
  MLFMA_CUDA(cudaGetLastError());
}

}  // namespace mlfma
