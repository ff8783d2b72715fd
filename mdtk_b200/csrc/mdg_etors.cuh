// AIREBO torsion term (ETors, mdtk/potentials/manybody/AIREBO/AIREBO_ETors.cxx).
//
// E = sum_{i<j, C-C} sum_{k in N(i)\{i,j}} sum_{l in N(j)\{i,j,k}}
//       w_ki w_ij w_jl [ (256/405) eps_kl ((1 + cos w)/2)^5 - eps_kl/10 ]
// with cos w = -CosDihedral and the |sin theta| >= 0.1 filters
// (AIREBO_ETors.cxx:32-115).  The reference's derivative of V_tors omits the
// factor 5 of the fifth power (AIREBO_ETors.cxx:110); forces here follow the
// reference exactly, so they are not the exact gradient of this energy.
//
// On the adjoint path (an ADJ sink of duals whose position tangents are u)
// two corrections are routed (the second only when the sink asks for J^T u):
//  - value only: the missing 4/5 of the angle term, so the values of the
//    accumulated gradient are the exact gradient of the energy (the loss's
//    energy term needs it);
//  - tangent only: the reference's term is G = der(cdh) W grad(cdh) +
//    val(cdh) grad(W) = grad(val W) - 4 der W grad(cdh), whose Jacobian is
//    not symmetric; the adjoint needs J^T u while duals give J u, and
//    J^T u - J u = -4 der [grad(W) (grad(cdh).u) - grad(cdh) (grad(W).u)],
//    where grad(cdh).u and grad(W).u are the tangents of cdh and W.
#pragma once

#include "mdg_rebo.cuh"

namespace mdg {

template <class Real, class TB, class S>
MDG_HD Real etors_bond(const ReboT<Real, TB>& R, const TorsParams& TP, int i, int j, const PairGT<Real>& p,
                        S& sink)
{
  if (R.type(i) != kC || R.type(j) != kC) return 0.0;
  const auto& B = R.B;
  const V3T<Real> a = p.rv;
  const Real wij = p.f;
  Real E = 0.0;
  const int nbi = B.nb[i], nbj = B.nb[j];
  for (int si = 0; si < nbi; si++) {
    const int qi = i * B.mb + si;
    const int k = B.bj[qi];
    if (k == j) continue;
    const auto rk = B.brv[qi], uk = B.bu[qi];
    const V3T<Real> b = xyz<Real>(rk);  // x_i - x_k
    const Real wki = uk.w;
    for (int sj = 0; sj < nbj; sj++) {
      const int qj = j * B.mb + sj;
      const int l = B.bj[qj];
      if (l == i || l == k) continue;
      Real sin_ki = sqrt(norm2(cross(a, -b))) / (p.r * rk.w);
      if (fabs(sin_ki) < 0.1) continue;
      const auto rl = B.brv[qj], ul = B.bu[qj];
      const V3T<Real> c = xyz<Real>(rl);  // x_j - x_l
      Real sin_jl = sqrt(norm2(cross(a, c))) / (p.r * rl.w);
      if (fabs(sin_jl) < 0.1) continue;
      const Real wjl = ul.w;
      const Real eps = TP.eps[R.type(k)][R.type(l)];
      V3T<Real> u = cross(-a, b);
      V3T<Real> w = cross(a, c);
      Real e1 = dot(u, w);
      Real uu = norm2(u), ww = norm2(w);
      Real e2 = sqrt(uu) * sqrt(ww);
      Real cosd = (e2 == 0.0) ? 0.0 : e1 / e2;
      if (cosd < -1.0) cosd = -1.0;
      if (cosd > 1.0) cosd = 1.0;
      Real cdh = -cosd;
      // ((1 + cdh)/2)^5 and ^4 by multiplication (the reference's pow, equal to rounding)
      const Real hx = 0.5 * (1.0 + cdh);
      const Real hx2 = hx * hx, hx4 = hx2 * hx2;
      Real val = (256.0 / 405.0) * eps * (hx4 * hx) - 0.1 * eps;
      Real V = wki * wij * wjl;  // seed of Vtors (AIREBO_ETors.cxx:78)
      if (val != 0.0) {
        Real der = (256.0 / 405.0) * eps * hx4 * 0.5;
        Real Vd = -1.0 * der * V;
        if (Vd != 0.0 && e2 != 0.0) {
          const Real ie2 = Real(1.0) / e2;
          Real cr = e1 * ie2;
          V3T<Real> U = w * ie2 - u * (cr / uu);
          V3T<Real> Wv = u * ie2 - w * (cr / ww);
          sink.pair(i, j, (cross(U, b) + cross(c, Wv)) * Vd);
          sink.cbond(i, si, cross(a, U) * Vd);
          sink.cbond(j, sj, cross(Wv, a) * Vd);
          if constexpr (S::kAdj) {
            // The crosses are d cos(omega) (cdh = -cos(omega)), taken at their
            // values.  Value: -4 der W d cos(omega), the missing 4/5 of the
            // angle term; tangent: -4 der (grad(W).u) d cos(omega).
            const Real k = sink.jt ? V * (-4.0 * mdg::val(der)) : Real(-4.0 * mdg::val(der) * mdg::val(V));
            sink.pair(i, j, values_of(cross(U, b) + cross(c, Wv)) * k);
            sink.cbond(i, si, values_of(cross(a, U)) * k);
            sink.cbond(j, sj, values_of(cross(Wv, a)) * k);
          }
        }
      }
      // ki.f / ij.f / jl.f seeds (AIREBO_ETors.cxx:80-85)
      Real dfk = B.bd[qi].x, dfl = B.bd[qj].x;
      if (dfk != 0.0) sink.cbond(i, si, xyz<Real>(uk) * ((wij * wjl * val) * dfk));
      if (p.df != 0.0) sink.pair(i, j, p.u * ((wki * wjl * val) * p.df));
      if (dfl != 0.0) sink.cbond(j, sj, xyz<Real>(ul) * ((wki * wij * val) * dfl));
      if constexpr (S::kAdj) {
        // -4 der grad(W) (grad(cdh).u): tangent only
        if (sink.jt && e2 != 0.0) {
          const Real der = (256.0 / 405.0) * eps * hx4 * 0.5;
          const Real kw = Real(0.0, -4.0 * mdg::val(der) * cdh.d);
          if (dfk != 0.0) sink.cbond(i, si, values_of(xyz<Real>(uk) * (wij * wjl * dfk)) * kw);
          if (p.df != 0.0) sink.pair(i, j, values_of(p.u * (wki * wjl * p.df)) * kw);
          if (dfl != 0.0) sink.cbond(j, sj, values_of(xyz<Real>(ul) * (wki * wij * dfl)) * kw);
        }
      }
      E += wki * wij * wjl * val;
    }
  }
  return E;
}

}  // namespace mdg
