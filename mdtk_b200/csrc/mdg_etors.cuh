// AIREBO torsion term (ETors, mdtk/potentials/manybody/AIREBO/AIREBO_ETors.cxx).
//
// E = sum_{i<j, C-C} sum_{k in N(i)\{i,j}} sum_{l in N(j)\{i,j,k}}
//       w_ki w_ij w_jl [ (256/405) eps_kl ((1 + cos w)/2)^5 - eps_kl/10 ]
// with cos w = -CosDihedral and the |sin theta| >= 0.1 filters
// (AIREBO_ETors.cxx:32-115).  The reference's derivative of V_tors omits the
// factor 5 of the fifth power (AIREBO_ETors.cxx:110); forces here follow the
// reference exactly, so they are not the exact gradient of this energy.
#pragma once

#include "mdg_rebo.cuh"

namespace mdg {

template <class S>
MDG_HD double etors_bond(const Rebo& R, const TorsParams& TP, int i, int j, const PairG& p, S& sink)
{
  if (R.type(i) != kC || R.type(j) != kC) return 0.0;
  const BondList& B = R.B;
  const V3 a = p.rv;
  const double wij = p.f;
  double E = 0.0;
  const int nbi = B.nb[i], nbj = B.nb[j];
  for (int si = 0; si < nbi; si++) {
    const int qi = i * B.mb + si;
    const int k = B.bj[qi];
    if (k == j) continue;
    double4 rk = B.brv[qi], uk = B.bu[qi];
    const V3 b = v3(rk.x, rk.y, rk.z);  // x_i - x_k
    const double wki = uk.w;
    for (int sj = 0; sj < nbj; sj++) {
      const int qj = j * B.mb + sj;
      const int l = B.bj[qj];
      if (l == i || l == k) continue;
      double sin_ki = sqrt(norm2(cross(a, -b))) / (p.r * rk.w);
      if (fabs(sin_ki) < 0.1) continue;
      double4 rl = B.brv[qj], ul = B.bu[qj];
      const V3 c = v3(rl.x, rl.y, rl.z);  // x_j - x_l
      double sin_jl = sqrt(norm2(cross(a, c))) / (p.r * rl.w);
      if (fabs(sin_jl) < 0.1) continue;
      const double wjl = ul.w;
      const double eps = TP.eps[R.type(k)][R.type(l)];
      V3 u = cross(-a, b);
      V3 w = cross(a, c);
      double e1 = dot(u, w);
      double uu = norm2(u), ww = norm2(w);
      double e2 = sqrt(uu) * sqrt(ww);
      double cosd = (e2 == 0.0) ? 0.0 : e1 / e2;
      if (cosd < -1.0) cosd = -1.0;
      if (cosd > 1.0) cosd = 1.0;
      double cdh = -cosd;
      double val = (256.0 / 405.0) * eps * pow(0.5 * (1.0 + cdh), 5.0) - 0.1 * eps;
      double V = wki * wij * wjl;  // seed of Vtors (AIREBO_ETors.cxx:78)
      if (val != 0.0) {
        double der = (256.0 / 405.0) * eps * pow(0.5 * (1.0 + cdh), 5.0 - 1.0) * 0.5;
        double Vd = -1.0 * der * V;
        if (Vd != 0.0 && e2 != 0.0) {
          double cr = e1 / e2;
          V3 U = w / e2 - u * (cr / uu);
          V3 Wv = u / e2 - w * (cr / ww);
          sink.pair(i, j, (cross(U, b) + cross(c, Wv)) * Vd);
          sink.cbond(i, si, cross(a, U) * Vd);
          sink.cbond(j, sj, cross(Wv, a) * Vd);
        }
      }
      // ki.f / ij.f / jl.f seeds (AIREBO_ETors.cxx:80-85)
      double dfk = B.bd[qi].x, dfl = B.bd[qj].x;
      if (dfk != 0.0) sink.cbond(i, si, v3(uk.x, uk.y, uk.z) * ((wij * wjl * val) * dfk));
      if (p.df != 0.0) sink.pair(i, j, p.u * ((wki * wjl * val) * p.df));
      if (dfl != 0.0) sink.cbond(j, sj, v3(ul.x, ul.y, ul.z) * ((wki * wij * val) * dfl));
      E += wki * wij * wjl * val;
    }
  }
  return E;
}

}  // namespace mdg
