// First-generation Brenner bond-order potential and its first-order adjoint
// (mdtk/potentials/manybody/Brenner/Brenner.cxx), evaluated from either end of
// a bond with the same Sink routing as the REBO term (mdg_rebo.cuh).
//
// E = sum_{i<j} [V_R(ij) - Bbar_ij V_A(ij)],  Bbar = (B_ij + B_ji)/2 + F_ij/2,
// B_ij = D_ij^-delta,  D_ij = 1 + sum_k G(cos theta_jik) f_ik exp(alpha ...) + H_ij(N^H, N^C).
// Unlike REBO, the coordination numbers are re-summed over the neighbours each
// time (Brenner.cxx:259-315) and N_conj is linear in its two sums.
#pragma once

#include "mdg_rebo.cuh"
#include "mdg_step.cuh"

namespace mdg {

// Brenner::setupPotential1/2 (Brenner.cxx:498-611), A / eV.
struct BrennerParams {
  double Re[2][2], De[2][2], beta[2][2], S[2][2], delta[2][2];
  double alpha[2][2][2];
  double ao, co, d0, GHH;
};

inline void set_brenner_params(BrennerParams& p, int set)
{
  const int C = kC, H = kH;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) p.alpha[a][b][c] = 0.0;
  if (set != 2) {
    // Brenner::setupPotential1 (Brenner.cxx:498-556)
    p.Re[C][C] = 1.315; p.Re[H][H] = 0.74144; p.Re[C][H] = p.Re[H][C] = 1.1199;
    p.De[C][C] = 6.325; p.De[H][H] = 4.7509; p.De[C][H] = p.De[H][C] = 3.6422;
    p.beta[C][C] = 1.5; p.beta[H][H] = 1.9436; p.beta[C][H] = p.beta[H][C] = 1.9583;
    p.S[C][C] = 1.29; p.S[H][H] = 2.3432; p.S[C][H] = p.S[H][C] = 1.7386;
    p.delta[C][C] = 0.80469; p.delta[H][H] = 0.80469; p.delta[C][H] = p.delta[H][C] = 0.0;
    p.alpha[H][H][H] = p.alpha[H][H][C] = p.alpha[H][C][H] = p.alpha[H][C][C] = p.alpha[C][H][H] = 3.0;
    p.ao = 0.011304; p.co = 19.0; p.d0 = 2.5; p.GHH = 4.0;
  } else {
    // Brenner::setupPotential2 (Brenner.cxx:558-611)
    p.Re[C][C] = 1.39; p.Re[H][H] = 0.74144; p.Re[C][H] = p.Re[H][C] = 1.1199;
    p.De[C][C] = 6.0; p.De[H][H] = 4.7509; p.De[C][H] = p.De[H][C] = 3.6422;
    p.beta[C][C] = 2.1; p.beta[H][H] = 1.9436; p.beta[C][H] = p.beta[H][C] = 1.9583;
    p.S[C][C] = 1.22; p.S[H][H] = 2.3432; p.S[C][H] = p.S[H][C] = 1.69077;
    p.delta[C][C] = 0.5; p.delta[H][H] = 0.5; p.delta[C][H] = p.delta[H][C] = 0.0;
    p.alpha[H][H][H] = p.alpha[H][H][C] = p.alpha[H][C][H] = p.alpha[H][C][C] = p.alpha[C][H][H] = 4.0;
    p.ao = 0.00020813; p.co = 330.0; p.d0 = 3.5; p.GHH = 12.33;
  }
}

// H_CC / H_CH bicubic and F tricubic cells (Brenner/cubici.hpp:39-175).
struct BrennerTables {
  double H[2][4][4][3][16];     // [CC/CH][h][c][f/dH/dC][term]
  double F[4][4][5][4][64];     // [i][j][k][f/di/dj/dk][term]
};

// FuncH_*: zero for h >= 4 or c >= 4 (no integer shortcut in the Brenner tables).
MDG_HD void h_eval(const BrennerTables& T, int fam, double h, double c, double& v, double& dh, double& dc,
                   unsigned int* status)
{
  v = dh = dc = 0.0;
  if (!(h >= 0 && c >= 0)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (h >= 4 || c >= 4) return;
  const double* cell = T.H[fam][(int)h][(int)c][0];
  v = poly2(cell, h, c, 0);
  dh = poly2(cell + 16, h, c, 1);
  dc = poly2(cell + 32, h, c, 2);
}

// FuncF: zero for i >= 4 or j >= 4; k clamped to 4 (Brenner/cubici.hpp:134-177).
MDG_HD void f_eval(const BrennerTables& T, double i, double j, double k, double* out, unsigned int* status)
{
  out[0] = out[1] = out[2] = out[3] = 0.0;
  if (!(i >= 0 && j >= 0 && k >= 1)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (i >= 4 || j >= 4) return;
  if (k > 4) k = 4;
  const double* cell = T.F[(int)i][(int)j][(int)k][0];
  out[0] = poly3(cell, i, j, k, 0);
  out[1] = poly3(cell + 64, i, j, k, 1);
  out[2] = poly3(cell + 128, i, j, k, 2);
  out[3] = poly3(cell + 192, i, j, k, 3);
}

struct Brenner {
  const BrennerParams& P;
  const BrennerTables& T;
  const BondList& B;
  unsigned int* status;

  MDG_HD int type(int i) const { return (int)B.nco[i].w; }

  // Nt / NH / NC of the pair c -> o: the cutoff sum over c's neighbours other
  // than o (which: 0 all, 1 H, 2 C), with V * df along each of those bonds
  // (Brenner::Nt/NH/NC, Brenner.cxx:259-315).
  template <class S>
  MDG_HD double Nsum(int c, int o, int which, double V, S& sink) const
  {
    double N = 0.0;
    const int nb = B.nb[c];
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o) continue;
      if (which) {
        int tk = type(k);
        if (which == 1 && tk != kH) continue;
        if (which == 2 && tk != kC) continue;
      }
      double4 u = B.bu[q];
      N += u.w;
      if (V != 0.0) {
        double df = B.bd[q].x;
        if (df != 0.0) sink.cbond(c, s, v3(u.x, u.y, u.z) * (V * df));
      }
    }
    return N;
  }

  // Nt of the pair k -> c seen from k (third shell of N_conj): the value only;
  // its gradient goes through the W coefficients of c's slot for k.
  MDG_HD double Nt_value(int k, int c) const
  {
    double N = 0.0;
    const int nb = B.nb[k];
    for (int s = 0; s < nb; s++) {
      const int q = k * B.mb + s;
      if (B.bj[q] == c) continue;
      N += B.bu[q].w;
    }
    return N;
  }

  // G (Brenner::G / dGdCT, Brenner.cxx:229-257)
  template <class S>
  MDG_HD double G(int c, int o, const PairG& p, int s_k, V3 bk_rv, double bk_r, V3 bk_u, double V, S& sink) const
  {
    if (type(c) != kC) return P.GHH;
    double e1 = dot(p.rv, bk_rv);
    double e2 = p.r * bk_r;
    double cost = e1 / e2;
    if (!(cost >= -1.0 - 1e-7 && cost <= 1.0 + 1e-7)) *status |= ST_COS_RANGE;
    if (cost < -1.0) cost = -1.0;
    if (cost > 1.0) cost = 1.0;
    if (V != 0.0) {
      double Vc = 2.0 * P.ao * SQR(P.co) * (1.0 + cost) / SQR(SQR(P.d0) + SQR(1.0 + cost)) * V;
      if (Vc != 0.0) {
        double e2s = SQR(e2);
        V3 dpa = (bk_rv * e2 - p.u * (bk_r * e1)) / e2s;
        V3 dpb = (p.rv * e2 - bk_u * (p.r * e1)) / e2s;
        sink.pair(c, o, dpa * Vc);
        sink.cbond(c, s_k, dpb * Vc);
      }
    }
    return P.ao * (1.0 + SQR(P.co) / SQR(P.d0) - SQR(P.co) / (SQR(P.d0) + SQR(1.0 + cost)));
  }

  // H_co (Brenner::HN, Brenner.cxx:415-446)
  template <class S>
  MDG_HD double HN(int c, int o, double V, S& sink) const
  {
    if (type(c) != kC) return 0.0;
    const int fam = type(o) == kC ? 0 : 1;
    Sink dummy;
    double nh = Nsum(c, o, 1, 0.0, dummy);
    double nc = Nsum(c, o, 2, 0.0, dummy);
    double v, dh, dc;
    h_eval(T, fam, nh, nc, v, dh, dc, status);
    if (V != 0.0) {
      Nsum(c, o, 1, dh * V, sink);
      Nsum(c, o, 2, dc * V, sink);
    }
    return v;
  }

  // D_co (Brenner::D, Brenner.cxx:184-214); V = 0 for the value pass.
  template <class S>
  MDG_HD double D(int c, int o, const PairG& p, double V, S& sink) const
  {
    double Dij = 1.0;
    const int nb = B.nb[c];
    const int tc = type(c), to = type(o);
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o) continue;
      double4 rv = B.brv[q], u = B.bu[q];
      const V3 brv = v3(rv.x, rv.y, rv.z), bu3 = v3(u.x, u.y, u.z);
      const int tk = type(k);
      const double al = P.alpha[tc][to][tk];
      double ex = 1.0;
      if (al != 0.0) ex = exp(al * ((p.r - P.Re[tc][to]) - (rv.w - P.Re[tc][tk])));
      if (ex == 0.0) continue;
      Sink dummy;
      double gv = G(c, o, p, s, brv, rv.w, bu3, 0.0, dummy);
      double fv = u.w;
      if (V != 0.0) {
        G(c, o, p, s, brv, rv.w, bu3, fv * ex * V, sink);
        double df = B.bd[q].x;
        if (df != 0.0) sink.cbond(c, s, bu3 * ((gv * ex * V) * df));
        if (al != 0.0) {
          double Vx = gv * fv * V;
          if (Vx != 0.0) {
            double dert = ex * al;
            sink.pair(c, o, p.u * (dert * Vx));
            sink.cbond(c, s, bu3 * (-dert * Vx));
          }
        }
      }
      Dij += gv * fv * ex;
    }
    Dij += HN(c, o, V, sink);
    return Dij;
  }

  // B_co = D^-delta (Brenner::B, Brenner.cxx:216-227)
  template <class S>
  MDG_HD double Bterm(int c, int o, const PairG& p, double V, S& sink) const
  {
    Sink dummy;
    double DVal = D(c, o, p, 0.0, dummy);
    const double dl = P.delta[type(c)][type(c)];
    if (V != 0.0) {
      double Der = -dl * pow(DVal, -dl - 1.0);
      D(c, o, p, Der * V, sink);
    }
    return pow(DVal, -dl);
  }

  // N_conj (Brenner::Nconj, Brenner.cxx:353-413): 1 + sum_k f_ck F(N_kc) + sum_l f_ol F(N_lo).
  MDG_HD double Fsw(double x) const
  {
    if (x <= 2.0) return 1.0;
    if (x >= 3.0) return 0.0;
    return (1.0 + cos(kPi * (x - 2.0))) / 2.0;
  }
  MDG_HD double dFsw(double x) const
  {
    if (x <= 2.0) return 0.0;
    if (x >= 3.0) return 0.0;
    return (-kPi * sin(kPi * (x - 2.0))) / 2.0;
  }
  template <class S>
  MDG_HD double nconj_side(int c, int o, double& acc, double V, S& sink) const
  {
    const int nb = B.nb[c];
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o || type(k) != kC) continue;
      double4 u = B.bu[q];
      double f = u.w;
      double x = Nt_value(k, c);
      double Fx = Fsw(x);
      if (V != 0.0) {
        double df = B.bd[q].x;
        if (df != 0.0) sink.cbond(c, s, v3(u.x, u.y, u.z) * ((Fx * V) * df));
        double w = f * dFsw(x) * V;
        if (w != 0.0) sink.wt(c, s, w);
      }
      acc += f * Fx;
    }
    return acc;
  }
  template <class S>
  MDG_HD double nconj(int i, int j, double V, S& sink) const
  {
    double N = 1.0;
    nconj_side(i, j, N, V, sink);
    nconj_side(j, i, N, V, sink);
    return N;
  }

  // F_ij/2 term (Brenner::FN, Brenner.cxx:448-472), C-C only.
  template <class S>
  MDG_HD double FN(int i, int j, double V, S& sink) const
  {
    if (type(i) != kC || type(j) != kC) return 0.0;
    Sink dummy;
    double Nti = Nsum(i, j, 0, 0.0, dummy);
    double Ntj = Nsum(j, i, 0, 0.0, dummy);
    double Nc = nconj(i, j, 0.0, dummy);
    double F[4];
    f_eval(T, Nti, Ntj, Nc, F, status);
    if (V != 0.0) {
      Nsum(i, j, 0, F[1] * V, sink);
      Nsum(j, i, 0, F[2] * V, sink);
      nconj(i, j, F[3] * V, sink);
    }
    return F[0];
  }

  // Bbar (Brenner::Baver, Brenner.cxx:143-154)
  template <class S>
  MDG_HD double baver(int i, int j, const PairG& p, double V, S& sink) const
  {
    const PairG q = pair_reverse(p);
    return (Bterm(i, j, p, V / 2.0, sink) + Bterm(j, i, q, V / 2.0, sink)) / 2.0 + (FN(i, j, V / 2.0, sink) / 2.0);
  }

  // V_R, V_A (Brenner::VR_Exp / VA_Exp, Brenner.cxx:70-141): f * a exp(-b (r - Re)).
  template <class S>
  MDG_HD double Vexp(int i, int j, const PairG& p, bool attractive, double V, S& sink) const
  {
    double f = p.f;
    if (f == 0.0) return 0.0;
    const int ti = type(i), tj = type(j);
    const double De = P.De[ti][tj], Sv = P.S[ti][tj], be = P.beta[ti][tj], Re = P.Re[ti][tj];
    double a, b;
    if (!attractive) {
      a = De / (Sv - 1.0);
      b = sqrt(2.0 * Sv) * be;
    } else {
      a = De * Sv / (Sv - 1.0);
      b = sqrt(2.0 / Sv) * be;
    }
    double val = a * exp(-b * (p.r - Re));
    if (V != 0.0) {
      double der = val * (-b);
      sink.pair(i, j, p.u * (der * f * V));
      if (p.df != 0.0) sink.pair(i, j, p.u * ((val * V) * p.df));
    }
    return f * val;
  }

  // One Brenner bond i < j (Brenner::operator(), Brenner.cxx:31-61).
  template <class S>
  MDG_HD double bond(int i, int j, const PairG& p, S& sink) const
  {
    Sink dummy;
    double vav = Vexp(i, j, p, true, 0.0, dummy);
    double E = Vexp(i, j, p, false, 1.0, sink);
    if (vav != 0.0) {
      double bav = baver(i, j, p, -vav, sink);
      E += -bav * Vexp(i, j, p, true, -bav, sink);
    }
    return E;
  }
};

}  // namespace mdg

namespace mdg {

// Brenner for every bond of atom a, accumulated on top of what the REBO /
// torsion kernel left in a's slots (that kernel zeroes them first).
MDG_HD void brenner_atom(const Brenner& R, ForceOut& O, int a)
{
  const BondList& B = R.B;
  Sink sink;
  sink.a = a;
  sink.g = v3(0, 0, 0);
  sink.A = O.A + (long)a * O.mb * 3;
  sink.W = O.W + (long)a * O.mb;
  double e = 0.0;
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int q = a * B.mb + s;
    const int b = B.bj[q];
    PairG p = pair_from_slot(B, q);
    int lo = a, hi = b;
    if (b < a) { lo = b; hi = a; p = pair_reverse(p); }
    double E = R.bond(lo, hi, p, sink);
    if (a == lo) e += E;
  }
  double4 g = O.gown[a];
  O.gown[a] = make_double4(g.x + sink.g.x, g.y + sink.g.y, g.z + sink.g.z, 0.0);
  O.e_rebo[a] += e;
}

}  // namespace mdg
