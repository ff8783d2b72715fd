// AIREBO intermolecular LJ term (mdtk/potentials/manybody/AIREBO/AIREBO_LJ.cxx):
// parameters, the bond-path connectivity table C_ij, and the per-pair term
// E_ij = C_ij * [1 - S(t_r) + S(t_r) S(t_b(b*_ij))] * f^LJ * 4 eps [(s/r)^12 - (s/r)^6]
// with its first-order adjoint.
#pragma once

#include "mdg_step.cuh"

namespace mdg {

inline void set_lj_chain(LJParams& p, int lj_cut_mode);

// AIREBO::setupPotential (AIREBO_LJ.cxx:219-287), A / eV.  lj_cut_mode 1
// replaces the cosine cutoff window by [3 sigma - 0.5, 3 sigma].
inline void set_lj_params(LJParams& p, int lj_cut_mode)
{
  const int C = kC, H = kH;
  p.sigma[C][C] = 3.40;
  p.sigma[H][H] = 2.65;
  p.sigma[C][H] = p.sigma[H][C] = 0.5 * (p.sigma[C][C] + p.sigma[H][H]);
  p.eps[C][C] = 0.00284;
  p.eps[H][H] = 0.00150;
  p.eps[C][H] = p.eps[H][C] = sqrt(p.eps[C][C] * p.eps[H][H]);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      p.RLJ[a][b][0] = p.sigma[a][b];
      p.RLJ[a][b][1] = p.sigma[a][b] * pow(2.0, 1.0 / 6.0);
    }
  p.R[C][C][0] = 5.0;
  p.R[H][H][0] = 4.0;
  p.R[C][H][0] = p.R[H][C][0] = 4.5;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) p.R[a][b][1] = p.R[a][b][0] + 0.5;
  if (lj_cut_mode == 1)
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) {
        p.R[a][b][1] = 3.0 * p.sigma[a][b];
        p.R[a][b][0] = p.R[a][b][1] - 0.5;
      }
  p.b[C][C][0] = 0.77;
  p.b[H][H][0] = 0.32;
  p.b[C][H][0] = p.b[H][C][0] = 0.75;
  p.b[C][C][1] = 0.81;
  p.b[H][H][1] = 0.42;
  p.b[C][H][1] = p.b[H][C][1] = 0.90;
  set_lj_chain(p, lj_cut_mode);
}

// Chain factors of the derived C-H / H-H parameters by sigma_CC and eps_CC
// (sigma_CH = (sigma_CC + sigma_HH)/2, eps_CH = sqrt(eps_CC eps_HH),
// AIREBO_LJ.cxx:229-247), and of the 3-sigma cutoff window.
inline void set_lj_chain(LJParams& p, int lj_cut_mode)
{
  const int C = kC, H = kH;
  p.dsig[C][C] = 1.0;
  p.dsig[C][H] = p.dsig[H][C] = 0.5;
  p.dsig[H][H] = 0.0;
  p.deps[C][C] = 1.0;
  p.deps[C][H] = p.deps[H][C] = p.eps[C][H] / (2.0 * p.eps[C][C]);
  p.deps[H][H] = 0.0;
  p.dcut = lj_cut_mode == 1 ? 3.0 : 0.0;
}

// Sets sigma_CC or eps_CC and re-derives what depends on them as
// AIREBO::setupPotential does (AIREBO_LJ.cxx:229-262).
inline void set_lj_cc(LJParams& p, int lj_cut_mode, double sigma_cc, double eps_cc)
{
  const int C = kC, H = kH;
  p.sigma[C][C] = sigma_cc;
  p.sigma[C][H] = p.sigma[H][C] = 0.5 * (p.sigma[C][C] + p.sigma[H][H]);
  p.eps[C][C] = eps_cc;
  p.eps[C][H] = p.eps[H][C] = sqrt(p.eps[C][C] * p.eps[H][H]);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      p.RLJ[a][b][0] = p.sigma[a][b];
      p.RLJ[a][b][1] = p.sigma[a][b] * pow(2.0, 1.0 / 6.0);
    }
  if (lj_cut_mode == 1)
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) {
        p.R[a][b][1] = 3.0 * p.sigma[a][b];
        p.R[a][b][0] = p.R[a][b][1] - 0.5;
      }
  set_lj_chain(p, lj_cut_mode);
}

// Connectivity table of atom i: every atom reachable over at most three REBO
// bonds with the largest product of bond cutoffs w and the path that gives
// it (AIREBO::fill_Cij, AIREBO_LJ.cxx:289-367), sorted by target.
// W: double, or dual on the adjoint path (the same entries, w with its tangent).
template <class W>
struct CijTableT {
  int cap;
  int* cnt;        // [n]
  int4* ent;       // [n * cap] x = target, y = path length, z = k, w = m
  W* w;            // [n * cap]
  unsigned long long* mask;  // [n] bit (target & 63) of every target: a clear bit means "no entry"
};
typedef CijTableT<double> CijTable;

// The middle bond k-m of a 3-bond connectivity path i-k-m-j belongs to
// neither end of the LJ pair; its gradient is returned with the pair's task
// (written by the lower-index end) and gathered later by k and m.
template <class W>
struct MidOutT {
  int k, sm, m, valid;  // sm = slot of m in k's bond list
  W c;                  // dE/dr of the bond k-m
};
typedef MidOutT<double> MidOut;

template <class W>
MDG_HD int bond_slot(const BondListT<W>& B, int c, int k)
{
  const int nb = B.nb[c];
  for (int s = 0; s < nb; s++)
    if (B.bj[c * B.mb + s] == k) return s;
  return -1;
}

// Builds atom i's table with the reference's enumeration order and tie rules:
// a 1-bond path replaces an equal-weight longer one, a 2-bond path an equal
// 3-bond one, a 3-bond path only a strictly smaller weight.
template <int CAPL>
MDG_HD void cij_build_atom(const BondList& B, CijTable& T, int i, unsigned int* status)
{
  int tgt[CAPL];
  int len[CAPL], pk[CAPL], pm[CAPL];
  double w[CAPL];
  int n = 0;
  bool over = false;
  const int cap = T.cap < CAPL ? T.cap : CAPL;
  auto upd = [&](int t, double nw, int L, int k, int m) {
    int idx = -1;
    for (int e = 0; e < n; e++)
      if (tgt[e] == t) { idx = e; break; }
    double cw = idx >= 0 ? w[idx] : 0.0;
    int cl = idx >= 0 ? len[idx] : 0;
    bool rep;
    if (L == 1) rep = nw > cw || (cw > 0.0 && nw == cw && cl > 1);
    else if (L == 2) rep = nw > cw || (cw > 0.0 && nw == cw && cl > 2);
    else rep = nw > cw;
    if (!rep) return;
    if (idx < 0) {
      if (n >= cap) { over = true; return; }
      idx = n++;
      tgt[idx] = t;
    }
    w[idx] = nw;
    len[idx] = L;
    pk[idx] = k;
    pm[idx] = m;
  };
  const int nb1 = B.nb[i];
  for (int s1 = 0; s1 < nb1; s1++) {
    const int q1 = i * B.mb + s1;
    const int k = B.bj[q1];
    const double f1 = B.bu[q1].w;
    upd(k, f1, 1, -1, -1);
    const int nb2 = B.nb[k];
    for (int s2 = 0; s2 < nb2; s2++) {
      const int q2 = k * B.mb + s2;
      const int m = B.bj[q2];
      const double f2 = B.bu[q2].w;
      upd(m, f1 * f2, 2, k, -1);
      const int nb3 = B.nb[m];
      for (int s3 = 0; s3 < nb3; s3++) {
        const int q3 = m * B.mb + s3;
        const int t = B.bj[q3];
        const double f3 = B.bu[q3].w;
        upd(t, f1 * f2 * f3, 3, k, m);
      }
    }
  }
  if (over) *status |= ST_CIJ_OVERFLOW;
  // insertion sort by target, then store
  for (int a = 1; a < n; a++) {
    int t = tgt[a], l = len[a], k = pk[a], m = pm[a];
    double ww = w[a];
    int b = a - 1;
    while (b >= 0 && tgt[b] > t) {
      tgt[b + 1] = tgt[b]; len[b + 1] = len[b]; pk[b + 1] = pk[b]; pm[b + 1] = pm[b]; w[b + 1] = w[b];
      b--;
    }
    tgt[b + 1] = t; len[b + 1] = l; pk[b + 1] = k; pm[b + 1] = m; w[b + 1] = ww;
  }
  unsigned long long mask = 0ull;
  for (int e = 0; e < n; e++) {
    T.ent[(long)i * T.cap + e] = make_int4(tgt[e], len[e], pk[e], pm[e]);
    T.w[(long)i * T.cap + e] = w[e];
    mask |= 1ull << (tgt[e] & 63);
  }
  T.cnt[i] = n;
  T.mask[i] = mask;
}

// Lookup of target j in the table of i (binary search).  Returns the entry
// index or -1.
template <class W>
MDG_HD int cij_search(const CijTableT<W>& T, int i, int j)
{
  int lo = 0, hi = T.cnt[i] - 1;
  const int4* e = T.ent + (long)i * T.cap;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int t = e[mid].x;
    if (t == j) return mid;
    if (t < j) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// The same, after the mask test: most LJ partners are beyond three bonds,
// and one mask load rules them out without the dependent loads of the search.
template <class W>
MDG_HD int cij_find(const CijTableT<W>& T, int i, int j)
{
  if (!((T.mask[i] >> (j & 63)) & 1ull)) return -1;
  return cij_search(T, i, j);
}

// S(t) switch (AIREBO::S / dS, AIREBO_LJ.cxx:116-156).
template <class Real>
MDG_HD Real Slj(Real arg, double amin, double amax)
{
  if (arg < amin) return 1.0;
  if (arg > amax) return 0.0;
  Real t = (arg - amin) / (amax - amin);
  return 1.0 - t * t * (3.0 - 2.0 * t);
}
template <class Real>
MDG_HD Real dSlj(Real arg, double amin, double amax)
{
  if (arg < amin) return 0.0;
  if (arg > amax) return 0.0;
  Real t = (arg - amin) / (amax - amin);
  return (-2.0 * t * (3.0 - 2.0 * t) + 2.0 * t * t) / (amax - amin);
}

// VLJ (AIREBO_LJ.cxx:158-189): f^LJ * 4 eps [(s/r)^12 - (s/r)^6]; with
// V != 0 routes V * d/dr to the pair i-j.  Returns f*Val in `lj`, Val in `val`.
// The powers of s/r are taken in double from the double length on every path
// (a float length would carry 12 x its rounding into (s/r)^12).
template <class Real, class S>
MDG_HD void vlj(const LJParams& P, int ti, int tj, int i, int j, const PairGT<Real>& pl, Real V, S& sink,
                typename Wide<Real>::T& lj, typename Wide<Real>::T& val)
{
  typedef typename Wide<Real>::T Wd;
  const Real fv = pl.f;
  lj = 0.0;
  val = 0.0;
  if (fv == 0.0) return;
  const Wd r = pl.rd;
  const Wd ir = Wd(1.0) / r;
  const double sigma = P.sigma[ti][tj], zeta = P.eps[ti][tj];
  const Wd sdr = sigma * ir;
  Wd s6 = sdr;
  for (int q = 2; q <= 6; q++) s6 *= sdr;
  const Wd s12 = s6 * s6;
  const Wd vd = 4.0 * zeta * (s12 - s6);
  val = vd;
  if (V != 0.0) {
    const Wd der = 4.0 * zeta * (-12.0 * s12 + 6.0 * s6) * ir;
    sink.pair(i, j, pl.u * Real(der * dbl(fv) * dbl(V)));
    if (pl.df != 0.0) sink.pair(i, j, pl.u * Real((vd * dbl(V)) * dbl(pl.df)));
  }
  lj = dbl(fv) * vd;
}

// Derivatives of one LJ pair energy E = C SrSb f vd by eps_CC and sigma_CC
// (adjoint path): E is linear in eps; sigma enters vd = 4 eps ((s/r)^12 -
// (s/r)^6), the S(t_r) window [sigma, 2^(1/6) sigma] (d Str / d sigma =
// -dS/dr r / sigma) and, in the 3-sigma mode, the cutoff window
// (d f / d sigma = -3 df/dr).
template <class Real, class S, class Wd>
MDG_HD void lj_par(const LJParams& P, int ti, int tj, int lo, const PairGT<Real>& pl, Wd C, Wd SrSb, Wd dSrSb_ds,
                   Wd vd, S& sink)
{
  const double fs = P.dsig[ti][tj], fe = P.deps[ti][tj];
  if (fs == 0.0 && fe == 0.0) return;
  const Wd r = pl.rd, f = dbl(pl.f), df = dbl(pl.df);
  const double sigma = P.sigma[ti][tj], eps = P.eps[ti][tj];
  const Wd sdr = sigma / r;
  Wd s6 = sdr;
  for (int q = 2; q <= 6; q++) s6 *= sdr;
  const Wd s12 = s6 * s6;
  const Wd dvd = 4.0 * eps * (12.0 * s12 - 6.0 * s6) / sigma;
  const Wd dLJ = f * dvd - P.dcut * df * vd;
  sink.par(lo, kParLJEps, fe * (C * SrSb * f * vd / eps));
  sink.par(lo, kParLJSigma, fs * (C * (SrSb * dLJ + f * vd * dSrSb_ds)));
}

template <class Real, class TB>
struct LJT {
  typedef typename Wide<Real>::T Wd;
  const LJParams& P;
  const ReboT<Real, TB>& R;
  const CijTableT<Wd>& T;

  // b*_ij: REBO's b_ij average for the pair with r_alter = R1 of REBO
  // (AIREBO::BijAsterix, AIREBO_LJ.cxx:191-202).
  template <class S>
  MDG_HD Real bstar(int i, int j, const PairGT<Real>& pl, Real V, S& sink) const
  {
    PairGT<Real> p = pl;
    const int ti = R.type(i), tj = R.type(j);
    cutoff(p.r, R.P.R[ti][tj][0], R.P.R[ti][tj][1], p.f, p.df);
    p.alter = 1;
    p.ralt = R.P.R[ti][tj][0];
    return R.baver(i, j, p, V, sink);
  }

  // One LJ pair i < j (the body of AIREBO::operator(), AIREBO_LJ.cxx:52-70).
  // pl: the pair i -> j with the LJ cosine cutoff in f/df.  Returns its
  // energy; the middle bond of a 3-bond path is recorded through `mid` when
  // non-null (the i end passes it).
  template <class S>
  MDG_HD Real pair(int i, int j, const PairGT<Real>& pl, S& sink, MidOutT<Wd>* mid, unsigned int* status) const
  {
    // connectivity (AIREBO::Cij, AIREBO_LJ.cxx:381-408)
    int e = cij_find(T, i, j);
    Wd w = 0.0;
    int4 path = make_int4(j, 0, -1, -1);
    if (e >= 0) {
      w = T.w[(long)i * T.cap + e];
      path = T.ent[(long)i * T.cap + e];
    }
    // C_ij, the switches and their products are per-pair scalars, kept in
    // double on every path: 1 - w and 1 - S(t_r) cancel to ~1e-3 here, which
    // float would turn into 1e-5 relative errors of the pair force.  Only b*
    // and the vectors handed to the sink use the arithmetic type.
    const Wd C = 1 - w;
    if (!(C > 0.0)) return 0.0;
    const int ti = R.type(i), tj = R.type(j);
    const Wd r = pl.rd;
    // StrStb value (AIREBO_LJ.cxx:79-114)
    const double rmin = P.RLJ[ti][tj][0], rmax = P.RLJ[ti][tj][1];
    const Wd Str = Slj(r, rmin, rmax);
    Wd Stb = 0.0, bij = 0.0, SrSb = 1.0;
    SinkT<Real> dummy;
    if (Str != 0.0) {
      bij = dbl(bstar(i, j, pl, Real(0.0), dummy));
      Stb = Slj(bij, P.b[ti][tj][0], P.b[ti][tj][1]);
      SrSb += Str * Stb - Str;
    }
    // VLJ with seed SrSb*C
    if (pl.f == 0.0) return 0.0;
    Wd LJv, val;
    vlj(P, ti, tj, i, j, pl, Real(SrSb * C), sink, LJv, val);
    if constexpr (S::kAdj) {
      const Wd dSrSb = (Str != 0.0) ? dSlj(r, rmin, rmax) * (r / P.sigma[ti][tj]) * (1.0 - Stb) : Wd(0.0);
      lj_par(P, ti, tj, i, pl, C, SrSb, dSrSb, val, sink);
    }
    // StrStb gradient with seed C*LJ
    const Wd V2 = C * LJv;
    if (Str != 0.0 && V2 != 0.0) {
      const Wd dStr = dSlj(r, rmin, rmax);
      if (dStr != 0.0) sink.pair(i, j, pl.u * Real(-dStr * V2));
      const Wd dStb = dSlj(bij, P.b[ti][tj][0], P.b[ti][tj][1]);
      if (dStr != 0.0 && Stb != 0.0) sink.pair(i, j, pl.u * Real(dStr * Stb * V2));
      if (dStb != 0.0) bstar(i, j, pl, Real(Str * dStb * V2), sink);
    }
    // Cij gradient with seed Vc3 = SrSb*LJ: -V * (product of the other cutoffs) * df
    const Wd Vc3 = SrSb * LJv;
    if (e >= 0 && Vc3 != 0.0 && path.y > 0) {
      const auto& B = R.B;
      if (path.y == 1) {
        int s = bond_slot(B, i, j);
        if (s >= 0) {
          const int q = i * B.mb + s;
          const Wd df = B.bd[q].x;
          if (df != 0.0) {
            const auto u = B.bu[q];
            sink.pair(i, j, xyz<Real>(u) * Real((-1.0 * Vc3) * df));
          }
        }
      } else {
        const int k = path.z, m = path.w;
        const int s1 = bond_slot(B, i, k);
        // the last bond of the path, seen from j
        const int last = (path.y == 2) ? k : m;
        const int sj = bond_slot(B, j, last);
        if (s1 < 0 || sj < 0) { *status |= ST_CIJ_OVERFLOW; return 0.0; }
        const int q1 = i * B.mb + s1, qj = j * B.mb + sj;
        const Wd f1 = B.bu[q1].w, fl = B.bu[qj].w;
        Wd fmid = 1.0, dfmid = 0.0;
        int sm = -1, qm = -1;
        if (path.y == 3) {
          sm = bond_slot(B, k, m);
          if (sm < 0) { *status |= ST_CIJ_OVERFLOW; return 0.0; }
          qm = k * B.mb + sm;
          fmid = B.bu[qm].w;
          dfmid = B.bd[qm].x;
        }
        // products in path order (AIREBO_LJ.cxx:396-402)
        const Wd m1 = (path.y == 2) ? 1.0 * fl : 1.0 * fmid * fl;
        const Wd ml = (path.y == 2) ? 1.0 * f1 : 1.0 * f1 * fmid;
        const Wd df1 = B.bd[q1].x, dfl = B.bd[qj].x;
        if (df1 != 0.0) {
          const auto u = B.bu[q1];
          sink.cbond(i, s1, xyz<Real>(u) * Real((-m1 * Vc3) * df1));
        }
        if (dfl != 0.0) {
          const auto u = B.bu[qj];
          sink.cbond(j, sj, xyz<Real>(u) * Real((-ml * Vc3) * dfl));
        }
        if (path.y == 3 && dfmid != 0.0 && mid) {
          const Wd mm = 1.0 * f1 * fl;
          mid->k = k;
          mid->sm = sm;
          mid->m = m;
          mid->valid = 1;
          mid->c = (-mm * Vc3) * dfmid;
        }
      }
    }
    return Real(SrSb * C * LJv);
  }
};

typedef LJT<double, ReboTables> LJ;

// Special LJ pairs (those needing b*_ij or a connectivity gradient) are
// evaluated one task per (atom, pair); each task writes its own record and a
// per-atom pass sums an atom's records in list order.  An atom's tasks take
// the contiguous range [off[a], off[a] + cnt[a]) of the task arrays and its
// records one contiguous range of the record pool; where those ranges lie depends on
// scheduling (one atomicAdd per block), the order within them does not; trec
// holds each task's record offset.
template <class W>
struct SpecialTasksT {
  int cap;          // special pairs per atom
  int task_cap;     // total tasks
  long rec_cap;     // total record doubles
  int* cnt;         // [n] special pairs of each atom (LJ-list order)
  int* part;        // [n * cap] partner of each
  int* off;         // [n] first task of each atom
  int2* flat;       // [task_cap] (atom, partner)
  long* trec;       // [task_cap] record offset of each task (-1: beyond rec_cap)
  W* rec;           // [rec_cap] per task: own gradient xyz, energy, A[nb][3], W[nb]
  int4* mid;        // [task_cap] middle-bond output (k, slot of m in k, m, valid)
  W* midc;          // [task_cap]
  W* dp;            // [task_cap * kNParam] energy derivatives by parameter (adjoint path only)
  // one evaluation per pair (the lower-index end's task writes both records):
  int* work;        // [task_cap] tasks whose owner is the lower index (-1: beyond task_cap)
  unsigned long long* ctr;  // work items, tasks, record doubles handed out this evaluation, at
                            // ctr[0], ctr[kCtrStride], ctr[2 kCtrStride] (one 128-byte line each)
};
constexpr int kCtrStride = 16;
typedef SpecialTasksT<double> SpecialTasks;

// Record size of a task owned by an atom with nb bonds.
MDG_HD int rec_size(int nb) { return 4 + 4 * nb; }

// Atom a's tasks [t0, t1), clipped to the task capacity.
template <class W>
MDG_HD void spc_range(const SpecialTasksT<W>& X, int a, int& t0, int& t1)
{
  t0 = X.off[a];
  const long e = (long)t0 + X.cnt[a];
  t1 = e < X.task_cap ? (int)e : X.task_cap;
}

// Number of tasks handed out by the last special-pair search, clipped.
template <class W>
MDG_HD int spc_total(const SpecialTasksT<W>& X)
{
  const unsigned long long t = X.ctr[kCtrStride];
  return t < (unsigned long long)X.task_cap ? (int)t : X.task_cap;
}

// Geometry of a pair lo -> hi (rv = x_lo - x_hi, r = |rv| as the FP64 path
// computes them) in the arithmetic type; on the adjoint path with the
// tangents of rv and r along the position tangents tan.
template <class Real>
MDG_HD PairGT<Real> pair_geom(V3 rv, double r, const double4* tan, int lo, int hi)
{
  PairGT<Real> p;
  if constexpr (IsDual<Real>::v) {
    const double4 tl = tan[lo], th = tan[hi];
    const V3 dv = v3(tl.x - th.x, tl.y - th.y, tl.z - th.z);
    const dual rr(r, (rv.x * dv.x + rv.y * dv.y + rv.z * dv.z) / r);
    p.rv = v3r<dual>(dual(rv.x, dv.x), dual(rv.y, dv.y), dual(rv.z, dv.z));
    p.r = rr;
    p.rd = rr;
    p.u = p.rv / rr;
  } else {
    p.rv = cvt3<Real>(rv);
    p.r = r;
    p.rd = r;
    p.u = cvt3<Real>(rv * (1.0 / r));
  }
  p.alter = 0;
  p.ralt = 0.0;
  return p;
}

// Class of one LJ pair seen from atom a: kind 0 (skip: beyond the cutoff or
// C = 0), 1 (plain: C = 1 and S(t_r) = 0, so E = VLJ) or 2 (special: needs
// b*_ij or a connectivity gradient); amask = T.mask[a].  The classification
// is made in double on every path (the adjoint path's pairs are the FP64
// path's), and the special-pair finder and the plain-pair kernels make it
// with the same expressions.
struct LJClass {
  int kind, lo, hi, tb;
  V3 rv;     // x_lo - x_hi
  double r;  // |rv| (kinds 1 and 2)
  double C;  // 1 - w_ij (kinds 1 and 2)
};

// w_ij of the pair (a, b) as a's own connectivity table holds it; amask =
// T.mask[a] (a clear bit for b proves w = 0 without the search).  The
// special-pair evaluation takes w from the lower index's table, whose
// product of bond cutoffs may differ from a's in rounding (the factors are
// multiplied in the reverse order); the class of the pair does not: it
// depends on w only through w == 0 (no path within three bonds: the bonds
// are symmetric) and w == 1 (a path whose cutoffs are all 1; a product with
// a factor below 1 never rounds up to 1), and both read the same from
// either end.  So each end classifies from its own table, which the atom's
// lanes share in L1.
template <class W>
MDG_HD double lj_w_own(const CijTableT<W>& T, int a, int b, unsigned long long amask)
{
  if (!((amask >> (b & 63)) & 1ull)) return 0.0;
  const int ei = cij_search(T, a, b);
  return ei >= 0 ? val(T.w[(long)a * T.cap + ei]) : 0.0;
}

// The pair at squared distance d2 may lie in the window where S(t_r) != 0
// and E_LJ takes b*_ij (when C > 0): r below the window's upper end
// 2^(1/6) sigma, with a relative margin of 1e-12 on r^2, so that rounding
// never puts a pair with S(t_r) != 0 outside.  A pair inside the margin is
// evaluated by the special-pair path, which computes S(t_r) itself (0 there).
MDG_HD bool lj_close(const LJParams& P, int ta, int tb, double d2)
{
  const double rmax = P.RLJ[ta][tb][1];
  return d2 < rmax * rmax * (1.0 + 1e-12);
}

// The class of a pair from its geometry and w: far = !lj_close.
MDG_HD int lj_kind(double w, bool close)
{
  if (!(1 - w > 0.0)) return 0;
  return (close || w != 0.0) ? 2 : 1;
}

template <class W>
MDG_HD LJClass lj_class(const LJParams& P, const CijTableT<W>& T, const State& St, int a, int b, V3 xa, int ta,
                        unsigned long long amask, bool known_far = false)
{
  LJClass c;
  const double4 pb = St.pos[b];
  c.tb = (int)pb.w;
  c.lo = a;
  c.hi = b;
  c.kind = 0;
  c.r = 0.0;
  c.C = 0.0;
  const Box box = box_of(St, a);
  if (a < b) c.rv = depos(box, xa, v3(pb.x, pb.y, pb.z));
  else { c.lo = b; c.hi = a; c.rv = depos(box, v3(pb.x, pb.y, pb.z), xa); }
  const double d2 = norm2(c.rv);
  const double R2 = P.R[ta][c.tb][1];
  if (d2 > R2 * R2) return c;
  const double w = lj_w_own(T, a, b, amask);
  c.C = 1 - w;  // exact for the plain pairs (w = 0); kind 2 takes C from the lower index's table
  if (!(c.C > 0.0)) return c;
  c.r = sqrt(d2);
  c.kind = lj_kind(w, !known_far && lj_close(P, ta, c.tb, d2));
  return c;
}

// One LJ pair seen from atom a: returns its lj_class kind; for plain pairs
// adds the own gradient and, at the lower end, the energy.  known_far: the
// pair is known to lie outside the S(t_r) window (the in-range filter's far
// list).
template <class Real, class S, class W>
MDG_HD int lj_plain_pair(const LJParams& P, const CijTableT<W>& T, const State& St, int a, int b, V3 xa, int ta,
                         unsigned long long amask, S& sink, W& e, const double4* tan = nullptr,
                         bool known_far = false)
{
  const LJClass c = lj_class(P, T, St, a, b, xa, ta, amask, known_far);
  if (c.kind != 1) return c.kind;
  // the pair term itself in the arithmetic type
  PairGT<Real> p = pair_geom<Real>(c.rv, c.r, tan, c.lo, c.hi);
  cutoff(p.r, P.R[ta][c.tb][0], P.R[ta][c.tb][1], p.f, p.df);
  W LJv, val;
  const int tlo = c.lo == a ? ta : c.tb, thi = c.lo == a ? c.tb : ta;
  vlj(P, tlo, thi, c.lo, c.hi, p, Real(1.0 * c.C), sink, LJv, val);
  if constexpr (S::kAdj) lj_par(P, tlo, thi, c.lo, p, W(c.C), W(1.0), W(0.0), val, sink);
  if (a == c.lo) e += 1.0 * c.C * LJv;
  return 1;
}

// Gradient owed to atom a by middle bonds k-m of connectivity paths (a as k
// or as m); the tasks of every bond partner lo of k are scanned in order.
template <class W>
MDG_HD V3T<W> mid_gather_atom(const BondListT<W>& B, const SpecialTasksT<W>& X, int a)
{
  V3T<W> g = v3r<W>(0.0, 0.0, 0.0);
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int lo = B.bj[a * B.mb + s];
    int t0, t1;
    spc_range(X, lo, t0, t1);
    for (int t = t0; t < t1; t++) {
      int4 e = X.mid[t];
      if (!e.w || e.x != a) continue;
      const auto u = B.bu[a * B.mb + e.y];
      g += v3r<W>(u.x, u.y, u.z) * X.midc[t];
    }
  }
  for (int s = 0; s < nb; s++) {
    const int k = B.bj[a * B.mb + s];
    const auto ua = B.bu[a * B.mb + s];
    const int nbk = B.nb[k];
    for (int q = 0; q < nbk; q++) {
      const int lo = B.bj[k * B.mb + q];
      int t0, t1;
      spc_range(X, lo, t0, t1);
      for (int t = t0; t < t1; t++) {
        int4 e = X.mid[t];
        if (!e.w || e.x != k || e.z != a) continue;
        g += v3r<W>(ua.x, ua.y, ua.z) * X.midc[t];
      }
    }
  }
  return g;
}

// Records one special task: the full pair term from end a with a private sink.
// ADJ: the adjoint path (duals with position tangents tan; the task's
// parameter derivatives go to Tk.dp).
template <bool ADJ = false, class Real, class TB>
MDG_HD void lj_special_task(const LJT<Real, TB>& X, const State& St, SpecialTasksT<typename Wide<Real>::T>& Tk, int t,
                            unsigned int* status, const double4* tan = nullptr)
{
  typedef typename Wide<Real>::T Wd;
  const int2 ap = Tk.flat[t];
  const int a = ap.x, b = ap.y;
  const int nba = X.R.B.nb[a];
  const long ro = Tk.trec[t];
  if (ro < 0) {  // beyond the record capacity (already flagged): no middle bond either
    Tk.mid[t] = make_int4(0, 0, 0, 0);
    return;
  }
  Wd* rec = Tk.rec + ro;
  SinkT<Real, ADJ> sink;
  sink.a = a;
  sink.g = v3r<Wd>(0.0, 0.0, 0.0);
  sink.A = rec + 4;
  sink.W = rec + 4 + 3 * nba;
  sink.dp = nullptr;
  sink.jt = 1;
  if constexpr (ADJ) {
    sink.dp = Tk.dp + (long)t * kNParam;
    for (int k = 0; k < kNParam; k++) sink.dp[k] = 0.0;
  }
  for (int s = 0; s < nba; s++) {
    sink.A[3 * s] = sink.A[3 * s + 1] = sink.A[3 * s + 2] = 0.0;
    sink.W[s] = 0.0;
  }
  const double4 pa = St.pos[a], pb = St.pos[b];
  int lo = a, hi = b;
  V3 rv;
  const Box& box = box_of(St, a);
  if (a < b) rv = depos(box, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z));
  else { lo = b; hi = a; rv = depos(box, v3(pb.x, pb.y, pb.z), v3(pa.x, pa.y, pa.z)); }
  const int tlo = (int)St.pos[lo].w, thi = (int)St.pos[hi].w;
  const double r = sqrt(norm2(rv));
  PairGT<Real> p = pair_geom<Real>(rv, r, tan, lo, hi);
  cutoff(p.r, X.P.R[tlo][thi][0], X.P.R[tlo][thi][1], p.f, p.df);
  MidOutT<Wd> mo;
  mo.valid = 0;
  const Real E = X.pair(lo, hi, p, sink, (a == lo) ? &mo : nullptr, status);
  rec[0] = sink.g.x;
  rec[1] = sink.g.y;
  rec[2] = sink.g.z;
  rec[3] = (a == lo) ? dbl(E) : Wd(0.0);
  Tk.mid[t] = make_int4(mo.k, mo.sm, mo.m, mo.valid);
  Tk.midc[t] = mo.valid ? mo.c : Wd(0.0);
}

// One special pair (a < b) from task t of a and task t2 of b, written into
// both records by a PairSink: the same additions as the two single-end tasks.
template <class Real, class TB>
MDG_HD void lj_special_pair_task(const LJT<Real, TB>& X, const State& St, SpecialTasks& Tk, int t, int t2,
                                 unsigned int* status)
{
  const int2 ap = Tk.flat[t];
  const int a = ap.x, b = ap.y;
  const long ro = Tk.trec[t], ro2 = Tk.trec[t2];
  if (ro < 0 || ro2 < 0) return;  // beyond the record capacity (already flagged)
  const int na = X.R.B.nb[a], nb = X.R.B.nb[b];
  double* ra = Tk.rec + ro;
  double* rb = Tk.rec + ro2;
  PairSinkT<Real> sink;
  sink.a = a;
  sink.b = b;
  sink.ga = v3(0, 0, 0);
  sink.gb = v3(0, 0, 0);
  sink.Aa = ra + 4;
  sink.Wa = ra + 4 + 3 * na;
  sink.Ab = rb + 4;
  sink.Wb = rb + 4 + 3 * nb;
  for (int q = 0; q < 4 * na; q++) sink.Aa[q] = 0.0;
  for (int q = 0; q < 4 * nb; q++) sink.Ab[q] = 0.0;
  const double4 pa = St.pos[a], pb = St.pos[b];
  const V3 rv = depos(box_of(St, a), v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z));
  const int ta = (int)pa.w, tb = (int)pb.w;
  const double r = sqrt(norm2(rv));
  PairGT<Real> p;
  p.rv = cvt3<Real>(rv);
  p.r = r;
  p.rd = r;
  p.u = cvt3<Real>(rv * (1.0 / r));
  cutoff(p.r, X.P.R[ta][tb][0], X.P.R[ta][tb][1], p.f, p.df);
  p.alter = 0;
  p.ralt = 0.0;
  MidOut mo;
  mo.valid = 0;
  const Real E = X.pair(a, b, p, sink, &mo, status);
  ra[0] = sink.ga.x;
  ra[1] = sink.ga.y;
  ra[2] = sink.ga.z;
  ra[3] = dbl(E);
  rb[0] = sink.gb.x;
  rb[1] = sink.gb.y;
  rb[2] = sink.gb.z;
  rb[3] = 0.0;
  Tk.mid[t] = make_int4(mo.k, mo.sm, mo.m, mo.valid);
  Tk.midc[t] = mo.valid ? mo.c : 0.0;
  Tk.mid[t2] = make_int4(0, 0, 0, 0);
  Tk.midc[t2] = 0.0;
}

// Sums atom a's special-task records (in list order) into its accumulators
// (and, on the adjoint path, the tasks' parameter derivatives).
template <class Wd>
MDG_HD void lj_reduce_atom(const BondListT<Wd>& B, const SpecialTasksT<Wd>& Tk, ForceOutT<Wd>& O, int a)
{
  const int nb = B.nb[a];
  const auto g0 = O.glj[a];
  V3T<Wd> g = v3r<Wd>(g0.x, g0.y, g0.z);
  Wd e = O.e_lj[a];
  Wd* A = O.A + (long)a * O.mb * 3;
  Wd* W = O.W + (long)a * O.mb;
  int t0, t1;
  spc_range(Tk, a, t0, t1);
  for (int t = t0; t < t1; t++) {
    const long ro = Tk.trec[t];
    if (ro < 0) continue;
    if (O.dp && Tk.dp)
      for (int k = 0; k < kNParam; k++) O.dp[(long)a * kNParam + k] += Tk.dp[(long)t * kNParam + k];
    const Wd* rec = Tk.rec + ro;
    g += v3r<Wd>(rec[0], rec[1], rec[2]);
    e += rec[3];
    for (int s = 0; s < nb; s++) {
      A[3 * s] += rec[4 + 3 * s];
      A[3 * s + 1] += rec[4 + 3 * s + 1];
      A[3 * s + 2] += rec[4 + 3 * s + 2];
      W[s] += rec[4 + 3 * nb + s];
    }
  }
  O.glj[a] = make_q4(g.x, g.y, g.z, Wd(0.0));
  O.e_lj[a] = e;
}

}  // namespace mdg
