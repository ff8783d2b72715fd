// CPU restatement of the MDTK hot-path energies (test infrastructure only;
// never linked into the product).
//
// Energy-only, templated on the scalar type T, independent of both the
// reference code and the product: splines are evaluated in their Hermite
// form from the reference's knot tables (the interpolants the reference's LU
// solves represent), coordination sums and connectivity are recomputed by
// brute force.  Instantiated on
//   double   -> energies, pinned against the compiled reference;
//   Dual<N>  -> exact directional derivatives (forward mode), to check the
//               hand-written adjoints of the reference and of the product;
//   Counted  -> algorithmic floating-point operation counts.
//
// Followed: REBO.cxx:32-814 (REBO), AIREBO_LJ.cxx:34-408 (LJ),
// AIREBO_ETors.cxx:32-115 (torsion), Brenner.cxx:31-472 (Brenner),
// AtomsPair.hpp:137-158 (cutoff), FGeneral.hpp:140-305 (angles),
// Atom.hpp:116-140 (minimum image), AIREBO/cubici.cxx and Brenner/cubici.cxx
// (tables), SplineAux/Spline2D/Spline3D/Spline5n (interpolation conditions).
#pragma once

#include <cmath>
#include <cstring>
#include <vector>

namespace rs {

// ------------------------------------------------------------ scalar types
inline double val(double x) { return x; }

template <int N>
struct Dual {
  double v;
  double d[N];
  Dual(double x = 0.0) : v(x) { for (int i = 0; i < N; i++) d[i] = 0.0; }
};
template <int N> inline double val(const Dual<N>& x) { return x.v; }
template <int N> inline Dual<N> operator+(Dual<N> a, const Dual<N>& b) { a.v += b.v; for (int i = 0; i < N; i++) a.d[i] += b.d[i]; return a; }
template <int N> inline Dual<N> operator-(Dual<N> a, const Dual<N>& b) { a.v -= b.v; for (int i = 0; i < N; i++) a.d[i] -= b.d[i]; return a; }
template <int N> inline Dual<N> operator-(Dual<N> a) { a.v = -a.v; for (int i = 0; i < N; i++) a.d[i] = -a.d[i]; return a; }
template <int N> inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) { Dual<N> r(a.v * b.v); for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int N> inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) { Dual<N> r(a.v / b.v); for (int i = 0; i < N; i++) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v); return r; }
template <int N> inline Dual<N> operator+(Dual<N> a, double b) { a.v += b; return a; }
template <int N> inline Dual<N> operator+(double b, Dual<N> a) { a.v += b; return a; }
template <int N> inline Dual<N> operator-(Dual<N> a, double b) { a.v -= b; return a; }
template <int N> inline Dual<N> operator-(double b, const Dual<N>& a) { return Dual<N>(b) - a; }
template <int N> inline Dual<N> operator*(Dual<N> a, double b) { a.v *= b; for (int i = 0; i < N; i++) a.d[i] *= b; return a; }
template <int N> inline Dual<N> operator*(double b, Dual<N> a) { return a * b; }
template <int N> inline Dual<N> operator/(Dual<N> a, double b) { a.v /= b; for (int i = 0; i < N; i++) a.d[i] /= b; return a; }
template <int N> inline Dual<N> operator/(double b, const Dual<N>& a) { return Dual<N>(b) / a; }
template <int N> inline Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N> inline Dual<N> exp(const Dual<N>& a) { Dual<N> r(std::exp(a.v)); for (int i = 0; i < N; i++) r.d[i] = r.v * a.d[i]; return r; }
template <int N> inline Dual<N> cos(const Dual<N>& a) { Dual<N> r(std::cos(a.v)); double s = -std::sin(a.v); for (int i = 0; i < N; i++) r.d[i] = s * a.d[i]; return r; }
template <int N> inline Dual<N> sqrt(const Dual<N>& a) { Dual<N> r(std::sqrt(a.v)); for (int i = 0; i < N; i++) r.d[i] = a.d[i] / (2.0 * r.v); return r; }
template <int N> inline Dual<N> pow(const Dual<N>& a, double p) { Dual<N> r(std::pow(a.v, p)); double g = p * std::pow(a.v, p - 1.0); for (int i = 0; i < N; i++) r.d[i] = g * a.d[i]; return r; }
template <int N> inline Dual<N> fabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }

// Operation counter: a double that tallies what is done to it.
struct OpTally {
  long add = 0, mul = 0, div = 0, sqrt_ = 0, exp_ = 0, cos_ = 0, pow_ = 0, cmp = 0;
};
// Two buckets: 0 = everything else, 1 = the REBO bond order b*_ij that the
// LJ term evaluates for close non-bonded pairs (AIREBO_LJ.cxx:191-202).
inline int& tally_bucket() { static int b = 0; return b; }
inline OpTally& tally() { static OpTally t[2]; return t[tally_bucket()]; }
struct Counted {
  double v;
  Counted(double x = 0.0) : v(x) {}
};
inline double val(const Counted& x) { return x.v; }
inline Counted operator+(Counted a, Counted b) { tally().add++; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { tally().add++; return Counted(a.v - b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted operator*(Counted a, Counted b) { tally().mul++; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { tally().div++; return Counted(a.v / b.v); }
inline Counted operator+(Counted a, double b) { tally().add++; return Counted(a.v + b); }
inline Counted operator+(double b, Counted a) { tally().add++; return Counted(a.v + b); }
inline Counted operator-(Counted a, double b) { tally().add++; return Counted(a.v - b); }
inline Counted operator-(double b, Counted a) { tally().add++; return Counted(b - a.v); }
inline Counted operator*(Counted a, double b) { tally().mul++; return Counted(a.v * b); }
inline Counted operator*(double b, Counted a) { tally().mul++; return Counted(a.v * b); }
inline Counted operator/(Counted a, double b) { tally().div++; return Counted(a.v / b); }
inline Counted operator/(double b, Counted a) { tally().div++; return Counted(b / a.v); }
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted exp(Counted a) { tally().exp_++; return Counted(std::exp(a.v)); }
inline Counted cos(Counted a) { tally().cos_++; return Counted(std::cos(a.v)); }
inline Counted sqrt(Counted a) { tally().sqrt_++; return Counted(std::sqrt(a.v)); }
inline Counted pow(Counted a, double p) { tally().pow_++; return Counted(std::pow(a.v, p)); }
inline Counted fabs(Counted a) { return Counted(std::fabs(a.v)); }

using std::cos;
using std::exp;
using std::fabs;
using std::pow;
using std::sqrt;

const double kPi = 3.14159265358979323846;

template <class T> struct V3 { T x, y, z; };
template <class T> V3<T> sub(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> neg(const V3<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T> T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(const V3<T>& a, const V3<T>& b)
{
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ------------------------------------------------------------ Hermite splines
// 1-D quintic Hermite on [x0, x1] from value, first and second derivative
// at both ends (the interpolation conditions of Spline5n, Spline5n.cxx:35-105).
template <class T>
T quintic(const T& x, double x0, double x1, const double v[2], const double d1[2], const double d2[2], int deriv)
{
  const double h = x1 - x0;
  T t = (x - x0) / h;
  T t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  if (!deriv) {
    T H0 = 1.0 - 10.0 * t3 + 15.0 * t4 - 6.0 * t5;
    T H1 = t - 6.0 * t3 + 8.0 * t4 - 3.0 * t5;
    T H2 = 0.5 * (t2 - 3.0 * t3 + 3.0 * t4 - t5);
    T H3 = 0.5 * (t3 - 2.0 * t4 + t5);
    T H4 = -4.0 * t3 + 7.0 * t4 - 3.0 * t5;
    T H5 = 10.0 * t3 - 15.0 * t4 + 6.0 * t5;
    return v[0] * H0 + (d1[0] * h) * H1 + (d2[0] * h * h) * H2 + (d2[1] * h * h) * H3 + (d1[1] * h) * H4 + v[1] * H5;
  }
  T H0 = -30.0 * t2 + 60.0 * t3 - 30.0 * t4;
  T H1 = 1.0 - 18.0 * t2 + 32.0 * t3 - 15.0 * t4;
  T H2 = 0.5 * (2.0 * t - 9.0 * t2 + 12.0 * t3 - 5.0 * t4);
  T H3 = 0.5 * (3.0 * t2 - 8.0 * t3 + 5.0 * t4);
  T H4 = -12.0 * t2 + 28.0 * t3 - 15.0 * t4;
  T H5 = 30.0 * t2 - 60.0 * t3 + 30.0 * t4;
  return (v[0] * H0 + (d1[0] * h) * H1 + (d2[0] * h * h) * H2 + (d2[1] * h * h) * H3 + (d1[1] * h) * H4 +
          v[1] * H5) / h;
}

// cubic Hermite basis on a unit cell: value bases H(a) and derivative bases D(a)
template <class T> T Hb(int a, const T& t) { return a == 0 ? (2.0 * t * t * t - 3.0 * t * t + 1.0) : (-2.0 * t * t * t + 3.0 * t * t); }
template <class T> T Db(int a, const T& t) { return a == 0 ? (t * t * t - 2.0 * t * t + t) : (t * t * t - t * t); }

// Tricubic Hermite on the unit cell at (i0, j0, k0) with corner values and
// first partials, all mixed partials zero (Spline3D.cxx:35-163).
template <class T>
T tricubic(const T& x, const T& y, const T& z, int i0, int j0, int k0, const double* F, const double* FI,
           const double* FJ, const double* FK, int ni, int nj, int nk)
{
  T tx = x - double(i0), ty = y - double(j0), tz = z - double(k0);
  T s = 0.0;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) {
        const int idx = ((i0 + a) * nj + (j0 + b)) * nk + (k0 + c);
        T hx = Hb(a, tx), hy = Hb(b, ty), hz = Hb(c, tz);
        if (F[idx] != 0.0) s += F[idx] * (hx * hy * hz);
        if (FI && FI[idx] != 0.0) s += FI[idx] * (Db(a, tx) * hy * hz);
        if (FJ && FJ[idx] != 0.0) s += FJ[idx] * (hx * Db(b, ty) * hz);
        if (FK && FK[idx] != 0.0) s += FK[idx] * (hx * hy * Db(c, tz));
      }
  (void)ni;
  return s;
}

template <class T>
T bicubic(const T& x, const T& y, int i0, int j0, const double* F, const double* FX, const double* FY, int nj)
{
  T tx = x - double(i0), ty = y - double(j0);
  T s = 0.0;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      const int idx = (i0 + a) * nj + (j0 + b);
      T hx = Hb(a, tx), hy = Hb(b, ty);
      if (F[idx] != 0.0) s += F[idx] * (hx * hy);
      if (FX && FX[idx] != 0.0) s += FX[idx] * (Db(a, tx) * hy);
      if (FY && FY[idx] != 0.0) s += FY[idx] * (hx * Db(b, ty));
    }
  return s;
}

// ------------------------------------------------------------ tables
struct Tables {
  // G(cos theta): knots x, y, y', y'' (AIREBO/cubici.cxx:42-102)
  double gc1[5][4], gc2[5][4], gh[4][4];
  // P_CC, P_CH corner values (AIREBO/cubici.cxx:117-290)
  double pcc[5][5], pch[5][5];
  // pi_rc CC/CH/HH and Tij: values and partials (AIREBO/cubici.cxx:292-536)
  double fv[4][5][5][16], fi[4][5][5][16], fj[4][5][5][16], fk[4][5][5][16];
  // Brenner H_CC / H_CH and F (Brenner/cubici.cxx:36-346), per parameter set
  double hcc[2][5][5], hch[2][5][5], hchdh[2][5][5], hchdc[2][5][5];
  double bf[2][5][5][6], bfi[2][5][5][6], bfj[2][5][5][6];
  Tables();
};

// ------------------------------------------------------------ parameters
struct Params {
  // REBO (REBO.cxx:857-938), A / eV
  double Q[2][2], alpha[2][2], A[2][2], B[3][2][2], beta[3][2][2], rho[2][2], R[2][2][2], Rp[2][2][2];
  // AIREBO LJ (AIREBO_LJ.cxx:219-287)
  double sigma[2][2], eps[2][2], RLJ[2][2][2], RL[2][2][2], bw[2][2][2];
  // torsion (AIREBO_ETors.cxx:125-133)
  double teps[2][2];
  // Brenner set 1/2 (Brenner.cxx:498-611)
  double bRe[2][2][2], bDe[2][2][2], bbeta[2][2][2], bS[2][2][2], bdelta[2][2][2], balpha[2][2][2][2];
  double bao[2], bco[2], bdo[2], bGHH[2];
  Params(int lj_cut_mode = 0);
};

struct System {
  int n;
  std::vector<int> t;        // 0 = C, 1 = H
  double L[3];
  int pbc[3];
};

}  // namespace rs
