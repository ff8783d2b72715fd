// REBO bond-order term (second-generation REBO as used by AIREBO) and its
// first-order adjoint, evaluated from either end of a bond.
//
// Reference: mdtk/potentials/manybody/AIREBO/REBO.cxx.  The reference
// evaluates every term twice (a value pass, then a pass seeded with V that
// scatters V * d(term)/dx into Atom::grad).  Here each bond (i, j), i < j, is
// evaluated in the reference's operation order by BOTH of its end atoms; a
// Sink keeps only the gradient pieces that belong to the evaluating atom:
//   - dE/d(x_p - x_q) of the pair vector i-j itself -> the evaluating atom,
//   - dE/d(x_c - x_k) of a bond c-k of one end c -> the evaluating atom when
//     it is c (and -that, for atom k, into the per-bond slot A[c][slot]),
//   - third-shell coefficients (dfThem over k's switching bonds, reached
//     through N_ki in N_conj) -> W[c][slot], resolved later by a gather.
// No atom ever writes another atom's accumulator, so the force sum is
// deterministic without atomics.
#pragma once

#include "mdg_common.cuh"
#include "mdg_spline.cuh"

namespace mdg {

// Per-step bond list of the REBO range (pairs with |r| <= R2 of the pair),
// ascending partner index, atom-major [a * mb + s].
// W is the stored scalar: double, or dual on the adjoint path (values and
// their tangents along the position direction of that pass).
template <class W>
struct BondListT {
  typedef typename Q4T<W>::T Q4;
  int n, mb;
  const int* nb;        // bond count per atom
  const int* bj;        // partner index
  const int* brev;      // slot of this atom in the partner's list
  const Q4* brv;        // x_a - x_partner, w = |r|
  const Q4* bu;         // unit vector (x_a - x_partner)/|r|, w = f (R cutoff)
  const Q4* bd;         // x = df/dr, y = f' (Rprime cutoff), z = df'/dr
  const Q4* nco;        // per atom: Nt, NC, NH (sums of f over the bonds), w = type
};
typedef BondListT<double> BondList;

// A pair vector as AtomsPair holds it (AtomsPair.hpp:35-160): rv = x_1 - x_2.
// Real is the arithmetic type (double, or f32 on the mixed-precision path).
template <class Real>
struct PairGT {
  V3T<Real> rv, u;    // vector and unit vector
  Real r, f, df;      // length and REBO cosine cutoff (R cutoffs of the pair types)
  typename Wide<Real>::T rd;  // the length in the wide type (the pair terms V_R, V_A use it on every path)
  Real ralt;          // r_alter (b*_ij uses R1 of the pair, AIREBO_LJ.cxx:196-198)
  int alter;
};
typedef PairGT<double> PairG;

template <class Real>
MDG_HD PairGT<Real> pair_reverse(const PairGT<Real>& p)
{
  PairGT<Real> q = p;
  q.rv = -p.rv;
  q.u = -p.u;
  return q;
}

// Gradient routing for one evaluating atom.  Contributions arrive in the
// arithmetic type and are accumulated in its wide type (double; dual on the
// adjoint path).  ADJ marks the accumulating sink of the adjoint path: terms
// then also record the derivatives of their energy with respect to the
// differentiated parameters (par) and apply the corrections that turn the
// forward Jacobian product of a non-gradient force into its transpose.
template <class Real, bool ADJ = false>
struct SinkT {
  typedef typename Wide<Real>::T Wd;
  static constexpr bool kAdj = ADJ;
  int a;           // evaluating atom
  V3T<Wd> g;       // dE/dx_a accumulated here
  Wd* A;           // [mb*3] this atom's bond slots: gradient owed to each partner
  Wd* W;           // [mb]   third-shell coefficients of this atom's bond slots
  Wd* dp;          // [kNParam] energy derivatives by parameter (ADJ only)
  int jt;          // ADJ: 1 = tangents give J^T u (adjoint), 0 = J u (tangent-linear)
  // d(energy)/d(parameter k), recorded by the lower-index end (the end that
  // owns the term's energy)
  MDG_HD void par(int lo, int k, Wd v)
  {
    if (ADJ && a == lo) dp[k] += v;
  }
  MDG_HD void pair(int p, int q, V3T<Real> v)
  {
    if (p == a) g += to_d(v);
    else if (q == a) g -= to_d(v);
  }
  MDG_HD void cbond(int c, int s, V3T<Real> v)
  {
    if (c == a) {
      const V3T<Wd> d = to_d(v);
      g += d;
      A[3 * s + 0] -= d.x;
      A[3 * s + 1] -= d.y;
      A[3 * s + 2] -= d.z;
    }
  }
  MDG_HD void wt(int c, int s, Real w)
  {
    if (c == a) W[s] += dbl(w);
  }
};
typedef SinkT<double> Sink;

// Both ends of a bond (lo, hi) at once: contributions are routed to each
// end's record exactly as two single-end Sinks would route them (the same
// additions in the same order), so one evaluation of the bond replaces two.
// (Compiled into a different kernel, the arithmetic upstream may contract
// multiply-adds differently, so the two modes agree to rounding.)
template <class Real>
struct PairSinkT {
  static constexpr bool kAdj = false;
  MDG_HD void par(int, int, double) {}
  int a, b;          // lo, hi
  V3 ga, gb;
  double *Aa, *Wa, *Ab, *Wb;
  MDG_HD void pair(int p, int q, V3T<Real> v)
  {
    const V3 d = to_d(v);
    if (p == a) ga += d;
    else if (q == a) ga -= d;
    if (p == b) gb += d;
    else if (q == b) gb -= d;
  }
  MDG_HD void cbond(int c, int s, V3T<Real> v)
  {
    const V3 d = to_d(v);
    if (c == a) {
      ga += d;
      Aa[3 * s + 0] -= d.x;
      Aa[3 * s + 1] -= d.y;
      Aa[3 * s + 2] -= d.z;
    } else if (c == b) {
      gb += d;
      Ab[3 * s + 0] -= d.x;
      Ab[3 * s + 1] -= d.y;
      Ab[3 * s + 2] -= d.z;
    }
  }
  MDG_HD void wt(int c, int s, Real w)
  {
    if (c == a) Wa[s] += dbl(w);
    else if (c == b) Wb[s] += dbl(w);
  }
};

// One end of a bond (lo, hi) evaluated on its own lane: the bond-slot
// pieces and third-shell coefficients of this end's atom (me) go to its
// record, the pieces along the pair vector itself to both ends' own
// gradients (glo, ghi; the two lanes' sums are added at the end).  pair_on
// off: pair-vector pieces dropped (a term both lanes evaluate whose pair
// pieces one lane keeps).
template <class Real>
struct EndSinkT {
  static constexpr bool kAdj = false;
  MDG_HD void par(int, int, double) {}
  int me, lo, hi;
  bool pair_on;
  V3 glo, ghi;
  double *A, *W;     // this end's record
  MDG_HD void pair(int p, int q, V3T<Real> v)
  {
    if (!pair_on) return;
    const V3 d = to_d(v);
    if (p == lo) glo += d;
    else if (q == lo) glo -= d;
    if (p == hi) ghi += d;
    else if (q == hi) ghi -= d;
  }
  MDG_HD void cbond(int c, int s, V3T<Real> v)
  {
    if (c != me) return;
    const V3 d = to_d(v);
    if (me == lo) glo += d;
    else ghi += d;
    A[3 * s + 0] -= d.x;
    A[3 * s + 1] -= d.y;
    A[3 * s + 2] -= d.z;
  }
  MDG_HD void wt(int c, int s, Real w)
  {
    if (c == me) W[s] += dbl(w);
  }
};

template <class Real, class TB>
struct ReboT {
  typedef typename Wide<Real>::T Wd;
  const ReboParams& P;
  const TB& T;
  const BondListT<Wd>& B;
  unsigned int* status;

  MDG_HD int type(int i) const { return (int)val(B.nco[i].w); }
  MDG_HD double R2(int ti, int tj) const { return P.R[ti][tj][1]; }

  // ---- coordination numbers (REBO::Nt/NH/NC, REBO.cxx:423-502) ----
  // which: 0 = all neighbours (Nt), 1 = H only (NH), 2 = C only (NC).
  MDG_HD Real Nval(int c, int o, const PairGT<Real>& p, int which) const
  {
    const auto n = B.nco[c];
    Real N = which == 0 ? n.x : (which == 1 ? n.z : n.y);
    int to = type(o);
    bool sub = (which == 0) || (which == 1 && to == kH) || (which == 2 && to == kC);
    if (sub && p.r < R2(type(c), to)) N -= p.f;
    if (!(N > -n_neg_tol(N))) *status |= ST_N_NEGATIVE;
    if (N < 0) N = 0;
    return N;
  }

  // dfThem (REBO.cxx:409-421): V * df_ck along every switching-region bond
  // c-k (k != o) of the chosen neighbour class.
  template <class S>
  MDG_HD void dfthem(int c, int o, Real V, int which, S& sink) const
  {
    if (V == 0.0) return;
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
      Real df = B.bd[q].x;
      if (df != 0.0) {
        const auto u = B.bu[q];
        sink.cbond(c, s, xyz<Real>(u) * (V * df));
      }
    }
  }

  // ---- angular term G (REBO::G, REBO.cxx:280-326) ----
  // Returns G; with V != 0 routes V * dG to the pair c-o, the bond c-k and
  // (carbon centre) through N_co to c's switching bonds.  Sp = S'(N_co) and
  // SpDer = dS'(N_co) of a carbon centre are the same for every k, so the
  // callers evaluate them once per pass (SpDer only when V may be nonzero).
  template <class S>
  MDG_HD Real G(int c, int o, const PairGT<Real>& p, int s_k, V3T<Real> bk_rv, Real bk_r, V3T<Real> bk_u, Real Sp,
                  Real SpDer, Real V, S& sink) const
  {
    Real e1 = dot(p.rv, bk_rv);
    Real e2 = p.r * bk_r;
    Real cost = e1 / e2;
    if (!(cost >= -1.0 - 1e-7 && cost <= 1.0 + 1e-7)) *status |= ST_COS_RANGE;
    if (cost < -1.0) cost = -1.0;
    if (cost > 1.0) cost = 1.0;
    Real Vc = 0.0, val;
    if (type(c) == kC) {
      Real g1 = g_eval(T.G[0], cost, 0);
      Real g2 = g_eval(T.G[1], cost, 0);
      if (V != 0.0) {
        Real g1d = g_eval(T.G[0], cost, 1);
        Real g2d = g_eval(T.G[1], cost, 1);
        if (g2d != 0.0 || g1d != 0.0) Vc = g2d * V + g1d * Sp * V + (-g2d * Sp * V);
        if ((g2 != 0.0 || g1 != 0.0) && SpDer != 0.0) dfthem(c, o, g1 * SpDer * V + (-g2 * SpDer * V), 0, sink);
      }
      val = g2 + Sp * (g1 - g2);
    } else {
      if (V != 0.0) {
        Real ghd = g_eval(T.G[2], cost, 1);
        if (ghd != 0.0) Vc = ghd * V;
      }
      val = g_eval(T.G[2], cost, 0);
    }
    if (Vc != 0.0) {
      // d cos(theta_ock) / d(x_c - x_o) and d/d(x_c - x_k) (FGeneral.hpp:152-178)
      const Real ie2s = Real(1.0) / SQR(e2);
      V3T<Real> dpa = (bk_rv * e2 - p.u * (bk_r * e1)) * ie2s;
      V3T<Real> dpb = (p.rv * e2 - bk_u * (p.r * e1)) * ie2s;
      sink.pair(c, o, dpa * Vc);
      sink.cbond(c, s_k, dpb * Vc);
    }
    return val;
  }

  // ExpTerm (REBO.cxx:213-233): 1 unless the centre is H.
  MDG_HD Real expterm(int c, int o, const PairGT<Real>& p, int k, Real bk_r) const
  {
    if (type(c) != kH) return 1.0;
    int tc = type(c), to = type(o), tk = type(k);
    Real rij = p.alter ? p.ralt : p.r;
    return exp(4.0 * ((P.rho[tc][tk] - bk_r) - (P.rho[tc][to] - rij)));
  }

  // D_co = 1 + sum_k G f_ck lambda + P_co (REBO::D, REBO.cxx:235-265), value.
  MDG_HD Real D_value(int c, int o, const PairGT<Real>& p) const
  {
    SinkT<Real> dummy;
    Real Dij = 1.0;
    Real Nco = Nval(c, o, p, 0);
    const Real Sp = type(c) == kC ? Sprime(Nco, P.Ntot[0], P.Ntot[1]) : Real(0.0);
    const int nb = B.nb[c];
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o) continue;
      const auto rv = B.brv[q];
      const auto u = B.bu[q];
      Real ex = expterm(c, o, p, k, rv.w);
      if (ex != 0.0) {
        Real gv = G(c, o, p, s, xyz<Real>(rv), rv.w, xyz<Real>(u), Sp, Real(0.0), 0.0, dummy);
        Dij += gv * u.w * ex;
      }
    }
    Dij += P_term(c, o, p, 0.0, dummy);
    return Dij;
  }

  // D_co gradient pass with seed V.
  template <class S>
  MDG_HD void D_grad(int c, int o, const PairGT<Real>& p, Real V, S& sink) const
  {
    Real Nco = Nval(c, o, p, 0);
    const bool ccen = type(c) == kC;
    const Real Sp = ccen ? Sprime(Nco, P.Ntot[0], P.Ntot[1]) : Real(0.0);
    const Real SpDer = ccen ? dSprime(Nco, P.Ntot[0], P.Ntot[1]) : Real(0.0);
    const int nb = B.nb[c];
    const bool hcen = type(c) == kH;
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o) continue;
      const auto rv = B.brv[q];
      const auto u = B.bu[q];
      V3T<Real> brv = xyz<Real>(rv), bu3 = xyz<Real>(u);
      Real ex = expterm(c, o, p, k, rv.w);
      if (ex == 0.0) continue;
      // one evaluation: the value G returns does not depend on the seed
      Real fv = u.w;
      Real gv = G(c, o, p, s, brv, rv.w, bu3, Sp, SpDer, fv * ex * V, sink);
      Real df = B.bd[q].x;
      if (df != 0.0) sink.cbond(c, s, bu3 * ((gv * ex * V) * df));
      if (hcen) {
        Real Vx = gv * fv * V;
        if (Vx != 0.0) {
          Real dert = ex * 4.0;
          sink.pair(c, o, p.u * (dert * Vx));
          sink.cbond(c, s, bu3 * (-dert * Vx));
        }
      }
    }
    P_term(c, o, p, V, sink);
  }

  // P_co (REBO::P, REBO.cxx:626-657): bicubic in (N^H, N^C) for a carbon centre.
  template <class S>
  MDG_HD Real P_term(int c, int o, const PairGT<Real>& p, Real V, S& sink) const
  {
    if (type(c) != kC) return 0.0;
    int fam = type(o) == kC ? 0 : 1;
    Real nh = Nval(c, o, p, 1);
    Real nc = Nval(c, o, p, 2);
    if (V == 0.0) return p_value(T, fam, nh, nc);
    Real v, dh, dc;
    p_eval(T, fam, nh, nc, v, dh, dc, status);
    dfthem(c, o, dh * V, 1, sink);
    dfthem(c, o, dc * V, 2, sink);
    return v;
  }

  // p^{sigma pi}_co = D^-1/2 (REBO::p_sigma_pi, REBO.cxx:267-278); the
  // reference's pow(D, -1/2) and pow(D, -3/2) as 1/sqrt(D) and its cube
  // (equal to rounding, a fraction of pow's instructions).
  template <class S>
  MDG_HD Real p_sigma_pi(int c, int o, const PairGT<Real>& p, Real V, S& sink) const
  {
    Real DVal = D_value(c, o, p);
    const Real ir = Real(1.0) / sqrt(DVal);
    if (V != 0.0) {
      Real Der = -0.5 * (ir * ir * ir);
      D_grad(c, o, p, Der * V, sink);
    }
    return ir;
  }

  // N_conj halves (REBO::NconjSum1/2, REBO.cxx:540-606): sum over C
  // neighbours k of c (k != o) of f_ck * S'(N_kc).
  MDG_HD Real nconj_sum(int c, int o) const
  {
    Real sum = 0.0;
    const int nb = B.nb[c];
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o || type(k) != kC) continue;
      Real f = B.bu[q].w;
      Real N = Nk_excl(k, B.brv[q].w, f, c);
      sum += f * Sprime(N, P.Ntot[0], P.Ntot[1]);
    }
    return sum;
  }

  // N_kc = Nt_k - f_kc (the pair k-c seen from k), clamped at 0.
  MDG_HD Real Nk_excl(int k, Real r, Real f, int c) const
  {
    Real N = B.nco[k].x;
    if (r < R2(type(k), type(c))) N -= f;
    if (!(N > -n_neg_tol(N))) *status |= ST_N_NEGATIVE;
    if (N < 0) N = 0;
    return N;
  }

  template <class S>
  MDG_HD void nconj_sum_grad(int c, int o, Real V, S& sink) const
  {
    const int nb = B.nb[c];
    for (int s = 0; s < nb; s++) {
      const int q = c * B.mb + s;
      const int k = B.bj[q];
      if (k == o || type(k) != kC) continue;
      const auto u = B.bu[q];
      Real f = u.w;
      Real N = Nk_excl(k, B.brv[q].w, f, c);
      Real Sp = Sprime(N, P.Ntot[0], P.Ntot[1]);
      Real df = B.bd[q].x;
      if (df != 0.0) sink.cbond(c, s, xyz<Real>(u) * ((Sp * V) * df));
      Real w = f * dSprime(N, P.Ntot[0], P.Ntot[1]) * V;
      if (w != 0.0) sink.wt(c, s, w);
    }
  }

  // N_conj = 1 + sum1^2 + sum2^2 (REBO::Nconj, REBO.cxx:608-624).
  MDG_HD Real nconj(int i, int j, Real& s1, Real& s2) const
  {
    s1 = nconj_sum(i, j);
    s2 = nconj_sum(j, i);
    Real N = 1.0;
    N += SQR(s1);
    N += SQR(s2);
    return N;
  }
  template <class S>
  MDG_HD void nconj_grad(int i, int j, Real s1, Real s2, Real V, S& sink) const
  {
    if (V == 0.0) return;
    if (s1 != 0.0) nconj_sum_grad(i, j, 2.0 * s1 * V, sink);
    if (s2 != 0.0) nconj_sum_grad(j, i, 2.0 * s2 * V, sink);
  }

  // ---- dihedral sum (REBO::pi_dh_sum, REBO.cxx:716-759) ----
  template <class S>
  MDG_HD Real dh_sum(int i, int j, const PairGT<Real>& p, Real V, S& sink) const
  {
    Real tsum = 0.0;
    const int nbi = B.nb[i], nbj = B.nb[j];
    const V3T<Real> a = p.rv;
    for (int si = 0; si < nbi; si++) {
      const int qi = i * B.mb + si;
      const int k = B.bj[qi];
      if (k == j) continue;
      const auto rk = B.brv[qi];
      const V3T<Real> b = xyz<Real>(rk);  // x_i - x_k
      for (int sj = 0; sj < nbj; sj++) {
        const int qj = j * B.mb + sj;
        const int l = B.bj[qj];
        if (l == i) continue;
        if (k == l) continue;
        Real sin_ik = sqrt(norm2(cross(a, -b))) / (p.r * rk.w);
        if (fabs(sin_ik) < 0.1) continue;
        const auto rl = B.brv[qj];
        const V3T<Real> cc = xyz<Real>(rl);  // x_j - x_l
        Real sin_jl = sqrt(norm2(cross(a, -cc))) / (p.r * rl.w);
        if (fabs(sin_jl) < 0.1) continue;
        int ti = type(i), tk = type(k), tj = type(j), tl = type(l);
        Real fik = Sprime(Real(rk.w), P.Rp[ti][tk][0], P.Rp[ti][tk][1]);
        Real fjl = Sprime(Real(rl.w), P.Rp[tj][tl][0], P.Rp[tj][tl][1]);
        // cos of the dihedral (FGeneral::CosDihedral, FGeneral.hpp:197-305)
        V3T<Real> u = cross(-a, b);
        V3T<Real> w = cross(a, cc);
        Real e1 = dot(u, w);
        Real uu = norm2(u), ww = norm2(w);
        Real e21 = sqrt(uu), e22 = sqrt(ww);
        Real e2 = e21 * e22;
        Real cosd = (e2 == 0.0) ? 0.0 : e1 / e2;
        if (cosd < -1.0) cosd = -1.0;
        if (cosd > 1.0) cosd = 1.0;
        Real cdh = -cosd;
        if (V != 0.0) {
          Real Vd = 2.0 * cdh * fik * fjl * V;
          if (Vd != 0.0 && e2 != 0.0) {
            const Real ie2 = Real(1.0) / e2;
            Real cr = e1 * ie2;
            V3T<Real> U = w * ie2 - u * (cr / uu);
            V3T<Real> Wv = u * ie2 - w * (cr / ww);
            V3T<Real> da = cross(U, b) + cross(cc, Wv);
            V3T<Real> db = cross(a, U);
            V3T<Real> dc = cross(Wv, a);
            sink.pair(i, j, da * Vd);
            sink.cbond(i, si, db * Vd);
            sink.cbond(j, sj, dc * Vd);
          }
          Real vk = (1.0 - SQR(cdh)) * fjl * V;
          if (vk != 0.0 && rk.w >= P.Rp[ti][tk][0] && rk.w <= P.Rp[ti][tk][1]) {
            const auto uk = B.bu[qi];
            sink.cbond(i, si, xyz<Real>(uk) * (dSprime(Real(rk.w), P.Rp[ti][tk][0], P.Rp[ti][tk][1]) * vk));
          }
          Real vl = (1.0 - SQR(cdh)) * fik * V;
          if (vl != 0.0 && rl.w >= P.Rp[tj][tl][0] && rl.w <= P.Rp[tj][tl][1]) {
            const auto ul = B.bu[qj];
            sink.cbond(j, sj, xyz<Real>(ul) * (dSprime(Real(rl.w), P.Rp[tj][tl][0], P.Rp[tj][tl][1]) * vl));
          }
        }
        tsum += (1.0 - SQR(cdh)) * fik * fjl;
      }
    }
    return tsum;
  }

  // ---- b_ij average (REBO::Baver, REBO.cxx:200-211) with seed V ----
  // i < j in the reference's loop order; p = pair i->j.
  template <class S>
  MDG_HD Real baver(int i, int j, const PairGT<Real>& p, Real V, S& sink) const
  {
    const PairGT<Real> q = pair_reverse(p);
    const Real half = V / 2.0;
    Real pij = p_sigma_pi(i, j, p, half, sink);
    Real pji = p_sigma_pi(j, i, q, half, sink);
    Real val = (pij + pji) / 2.0;

    const int ti = type(i), tj = type(j);
    // pi_rc (REBO.cxx:659-714): the H-C order evaluates as C-H with i and j swapped
    int ci = i, cj = j;
    const PairGT<Real>* pc = &p;
    const PairGT<Real>* qc = &q;
    if (ti == kH && tj == kC) { ci = j; cj = i; pc = &q; qc = &p; }
    const int tci = type(ci), tcj = type(cj);
    int fam = (tci == kC && tcj == kC) ? 0 : ((tci == kC && tcj == kH) ? 1 : 2);
    Real Nti = Nval(ci, cj, *pc, 0);
    Real Ntj = Nval(cj, ci, *qc, 0);
    Real s1, s2;
    Real Nconj = nconj(ci, cj, s1, s2);
    Real F[4];
    t_eval(T, fam, Nti, Ntj, Nconj, F, status);
    val += F[0];
    Real cNti = 0.0, cNtj = 0.0, cNconj = 0.0;
    if (V != 0.0) {
      cNti = F[1] * V;
      cNtj = F[2] * V;
      cNconj = F[3] * V;
    }
    // pi_dh (REBO.cxx:761-814): C-C only, T_ij nonzero only near (2,2,.)
    if (ti == kC && tj == kC) {
      // here (ci,cj) == (i,j)
      Real Tv[4];
      t_eval(T, 3, Nti, Ntj, Nconj, Tv, status);
      if (Tv[0] != 0.0) {
        Real ts = dh_sum(i, j, p, 0.0, sink);
        val += Tv[0] * ts;
        if (V != 0.0) {
          if (ts != 0.0) {
            Real Vt = ts * V;
            cNti += Tv[1] * Vt;
            cNtj += Tv[2] * Vt;
            cNconj += Tv[3] * Vt;
          }
          dh_sum(i, j, p, Tv[0] * V, sink);
        }
      }
    }
    if (V != 0.0) {
      dfthem(ci, cj, cNti, 0, sink);
      dfthem(cj, ci, cNtj, 0, sink);
      nconj_grad(ci, cj, s1, s2, cNconj, sink);
    }
    return val;
  }

  // ---- repulsive / attractive pair terms (REBO.cxx:134-198) ----
  // Return f*V_R and -f*V_A; with V != 0 route V * d/d(r_ij) to the pair.
  // Evaluated in the wide type (double, or dual on the adjoint path) from the
  // wide length on every path: their exponentials are the largest, most
  // cancelling terms of the bond energy, and a float length alone would put
  // ~alpha*r*eps_f of relative error into them.
  template <class S>
  MDG_HD Real VR(int i, int j, const PairGT<Real>& p, Real V, S& sink) const
  {
    const Real f = p.f;
    if (f == 0.0) return 0.0;
    int ti = type(i), tj = type(j);
    const Wd r = p.rd;
    const double Q = P.Q[ti][tj], A = P.A[ti][tj], al = P.alpha[ti][tj];
    const Wd t1 = A * exp(-al * r);
    const Wd val = (1 + Q / r) * t1;
    if (V != 0.0) {
      const Wd der = -t1 * (Q + al * r * r + al * r * Q) / (r * r);
      sink.pair(i, j, p.u * Real(der * dbl(f) * dbl(V)));
      if (p.df != 0.0) sink.pair(i, j, p.u * Real((val * dbl(V)) * dbl(p.df)));
    }
    return Real(dbl(f) * val);
  }
  // V_A's sum of exponentials and its radial derivative, evaluated once per
  // bond: the value seeds b-bar and the gradient pass reuses both.
  MDG_HD void VA_terms(int i, int j, const PairGT<Real>& p, Wd& val, Wd& der) const
  {
    int ti = type(i), tj = type(j);
    const Wd r = p.rd;
    const Wd t1 = P.B[0][ti][tj] * exp(-P.beta[0][ti][tj] * r);
    const Wd t2 = P.B[1][ti][tj] * exp(-P.beta[1][ti][tj] * r);
    const Wd t3 = P.B[2][ti][tj] * exp(-P.beta[2][ti][tj] * r);
    val = t1 + t2 + t3;
    der = (-P.beta[0][ti][tj]) * t1 + (-P.beta[1][ti][tj]) * t2 + (-P.beta[2][ti][tj]) * t3;
  }
  template <class S>
  MDG_HD Real VA_from(int i, int j, const PairGT<Real>& p, Wd val, Wd der, Real V, S& sink) const
  {
    const Real f = p.f;
    if (f == 0.0) return 0.0;
    if (V != 0.0) {
      sink.pair(i, j, p.u * Real(-der * dbl(f) * dbl(V)));
      if (p.df != 0.0) sink.pair(i, j, p.u * Real((-val * dbl(V)) * dbl(p.df)));
    }
    return Real(-dbl(f) * val);
  }
  template <class S>
  MDG_HD Real VA(int i, int j, const PairGT<Real>& p, Real V, S& sink) const
  {
    if (p.f == 0.0) return 0.0;
    Wd val, der;
    VA_terms(i, j, p, val, der);
    return VA_from(i, j, p, val, der, V, sink);
  }

  // One REBO bond i < j (REBO::operator(), REBO.cxx:43-59): returns its energy.
  template <class S>
  MDG_HD Real bond(int i, int j, const PairGT<Real>& p, S& sink) const
  {
    SinkT<Real> dummy;
    Wd va_val = 0.0, va_der = 0.0;
    if (p.f != 0.0) VA_terms(i, j, p, va_val, va_der);
    Real vav = VA_from(i, j, p, va_val, va_der, 0.0, dummy);
    Real E = VR(i, j, p, 1.0, sink);
    Real bav = 0.0;
    if (vav != 0.0) {
      bav = baver(i, j, p, vav, sink);
      E += bav * VA_from(i, j, p, va_val, va_der, bav, sink);
    }
    if constexpr (S::kAdj) {
      // derivatives of this bond's energy by the C-C pair parameters: V_R is
      // linear in A, V_A's first term in B1 (the bond order does not depend on
      // A, alpha, B1, beta1)
      if (type(i) == kC && type(j) == kC && p.f != 0.0) {
        const Wd r = p.rd, f = dbl(p.f);
        const double Q = P.Q[kC][kC], A = P.A[kC][kC], al = P.alpha[kC][kC];
        const double B1 = P.B[0][kC][kC], be1 = P.beta[0][kC][kC];
        const Wd eR = f * (1 + Q / r) * exp(-al * r);  // d(f V_R)/dA
        const Wd e1 = f * exp(-be1 * r);                 // -d(f V_A)/dB1
        sink.par(i, kParReboA, eR);
        sink.par(i, kParReboAlpha, -r * A * eR);
        sink.par(i, kParReboB1, -dbl(bav) * e1);
        sink.par(i, kParReboBeta1, dbl(bav) * r * B1 * e1);
      }
    }
    return E;
  }
};
typedef ReboT<double, ReboTables> Rebo;

// Pair record of bond slot q of atom c (the pair c -> partner).
template <class Real = double>
MDG_HD PairGT<Real> pair_from_slot(const BondListT<typename Wide<Real>::T>& B, int q)
{
  PairGT<Real> p;
  const auto rv = B.brv[q], u = B.bu[q], d = B.bd[q];
  p.rv = xyz<Real>(rv);
  p.u = xyz<Real>(u);
  p.r = rv.w;
  p.rd = rv.w;
  p.f = u.w;
  p.df = d.x;
  p.ralt = 0.0;
  p.alter = 0;
  return p;
}

}  // namespace mdg
