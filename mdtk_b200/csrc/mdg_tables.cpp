// Host-side construction of the REBO and Brenner spline tables.
//
// The reference builds every correction spline at start-up by setting up the
// Hermite corner conditions of a monomial polynomial and solving them with an
// LU factorisation (Spline2D/Spline3D/Spline5n::init, mdtk/Spline2D.cxx:36-125,
// Spline3D.cxx:35-163, Spline5n.cxx:35-105; SplineMultiD::addEquations,
// SplineAux.cxx:63-93).  This file re-derives the same tables from the same
// knot data, in the same equation and term order, with LU partial pivoting in
// the same elimination order, so the coefficients agree bit for bit with the
// reference's own.  The knot data are the reference's published parameter
// tables (AIREBO/cubici.cxx:42-536, Brenner/cubici.cxx) and must be identical.
#include <cmath>
#include <cstring>
#include <vector>

#include "mdg_spline.cuh"
#include "mdg_tables.h"
#include "mdg_brenner.cuh"

namespace mdg {
namespace {

// ---- SplineMultiD term bookkeeping (SplineAux.hpp:125-206) ----
struct Term {
  int p[3];
  double mult;
};

// Terms of a dim-dimensional polynomial of the given order, x0 fastest.
std::vector<Term> make_terms(int dim, int order)
{
  std::vector<Term> t;
  int n = 1;
  for (int d = 0; d < dim; d++) n *= (order + 1);
  for (int q = 0; q < n; q++) {
    Term x;
    x.p[0] = x.p[1] = x.p[2] = 0;
    int r = q;
    for (int d = 0; d < dim; d++) { x.p[d] = r % (order + 1); r /= (order + 1); }
    x.mult = 1.0;
    t.push_back(x);
  }
  return t;
}

void differentiate(std::vector<Term>& t, int d)
{
  for (size_t i = 0; i < t.size(); i++) {
    t[i].mult *= t[i].p[d];
    t[i].p[d] -= 1;
  }
}

double intpow_host(double a, int n)
{
  switch (n) {
    case 0: return 1.0;
    case 1: return a;
    case 2: return a * a;
    case 3: return a * a * a;
    case 4: return a * a * a * a;
    case 5: return a * a * a * a * a;
    case 6: return a * a * a * a * a * a;
    default: {
      double v = 1.0;
      int an = n < 0 ? -n : n;
      for (int i = 1; i <= an; i++) v *= a;
      if (n < 0) v = 1.0 / v;
      return v;
    }
  }
}

// SplineTerm::woC (SplineAux.hpp:96-110): multiplier * prod intpow, 0 if multiplier is 0.
double woC(const Term& t, const double* x, int dim)
{
  if (t.mult == 0) return 0.0;
  double v = t.mult;
  for (int d = 0; d < dim; d++) v *= intpow_host(x[d], t.p[d]);
  return v;
}

// LU with partial pivoting (first row holding the largest |a_ij| in the
// column), row elimination, unit-lower forward and upper back substitution.
std::vector<double> lu_solve(std::vector<double> a, std::vector<double> b)
{
  const size_t n = b.size();
  std::vector<size_t> perm(n);
  for (size_t i = 0; i < n; i++) perm[i] = i;
  for (size_t j = 0; j + 1 < n; j++) {
    double amax = std::fabs(a[j * n + j]);
    size_t ip = j;
    for (size_t i = j + 1; i < n; i++) {
      double v = std::fabs(a[i * n + j]);
      if (v > amax) { amax = v; ip = i; }
    }
    if (ip != j) {
      for (size_t k = 0; k < n; k++) std::swap(a[j * n + k], a[ip * n + k]);
      std::swap(perm[j], perm[ip]);
    }
    double ajj = a[j * n + j];
    if (ajj != 0.0) {
      for (size_t i = j + 1; i < n; i++) {
        double f = a[i * n + j] / ajj;
        a[i * n + j] = f;
        for (size_t k = j + 1; k < n; k++) a[i * n + k] -= f * a[j * n + k];
      }
    }
  }
  std::vector<double> x(n);
  for (size_t i = 0; i < n; i++) x[i] = b[perm[i]];
  for (size_t i = 1; i < n; i++) {
    double t = x[i];
    for (size_t k = 0; k < i; k++) t -= a[i * n + k] * x[k];
    x[i] = t;
  }
  x[n - 1] = x[n - 1] / a[(n - 1) * n + (n - 1)];
  for (size_t ii = n - 1; ii-- > 0;) {
    double t = x[ii];
    for (size_t k = ii + 1; k < n; k++) t -= a[ii * n + k] * x[k];
    x[ii] = t / a[ii * n + ii];
  }
  return x;
}

// A solved polynomial: its c vector and the term list (value poly).
struct Poly {
  std::vector<Term> terms;
  std::vector<double> c;
};

// Coefficient multiplier*c of the value poly or of a derivative poly
// (derivative d: 0 none, 1..3 = d/dx0..), 0 when either factor is 0.
void emit(const Poly& P, int deriv, std::vector<double>& out)
{
  std::vector<Term> t = P.terms;
  if (deriv > 0) differentiate(t, deriv - 1);
  for (size_t i = 0; i < t.size(); i++) {
    double m = t[i].mult, c = P.c[i];
    out.push_back((m == 0.0 || c == 0.0) ? 0.0 : m * c);
  }
}

// Value of a solved polynomial exactly as SplineMultiD::operator() sums it.
double eval_poly(const Poly& P, int deriv, const double* x, int dim)
{
  std::vector<Term> t = P.terms;
  if (deriv > 0) differentiate(t, deriv - 1);
  double val = 0;
  for (size_t i = 0; i < t.size(); i++) {
    if (t[i].mult == 0.0 || P.c[i] == 0.0) continue;
    double v = t[i].mult * P.c[i];
    for (int d = 0; d < dim; d++) v *= intpow_host(x[d], t[i].p[d]);
    val += v;
  }
  return val;
}

// Spline5n::init (Spline5n.cxx:35-105): value, first and second derivative at both ends.
Poly quintic(const double x[2], const double v[2], const double dv[2], const double d2v[2])
{
  Poly P;
  P.terms = make_terms(1, 5);
  std::vector<Term> Fv = P.terms, Fd = P.terms, Fd2 = P.terms;
  differentiate(Fd, 0);
  differentiate(Fd2, 0);
  differentiate(Fd2, 0);
  std::vector<double> A, b;
  const std::vector<Term>* sets[3] = {&Fv, &Fd, &Fd2};
  const double* vals[3] = {v, dv, d2v};
  for (int s = 0; s < 3; s++)
    for (int i = 0; i < 2; i++) {
      double xv[1] = {x[i]};
      for (size_t j = 0; j < sets[s]->size(); j++) A.push_back(woC((*sets[s])[j], xv, 1));
      b.push_back(vals[s][i]);
    }
  P.c = lu_solve(A, b);
  return P;
}

// Spline2D::init (Spline2D.cxx:36-125): v, dv/dx, dv/dy at the 4 corners, d2v/dxdy = 0.
Poly bicubic(const double x[2], const double y[2], const double v[2][2], const double dx[2][2],
             const double dy[2][2])
{
  Poly P;
  P.terms = make_terms(2, 3);
  std::vector<Term> Fv = P.terms, Fx = P.terms, Fy = P.terms, Fxy = P.terms;
  differentiate(Fx, 0);
  differentiate(Fy, 1);
  differentiate(Fxy, 0);
  differentiate(Fxy, 1);
  std::vector<double> A, b;
  const std::vector<Term>* sets[4] = {&Fv, &Fx, &Fy, &Fxy};
  for (int s = 0; s < 4; s++)
    for (int i1 = 0; i1 < 2; i1++)
      for (int i2 = 0; i2 < 2; i2++) {
        double xv[2] = {x[i1], y[i2]};
        for (size_t j = 0; j < sets[s]->size(); j++) A.push_back(woC((*sets[s])[j], xv, 2));
        double f = 0.0;
        if (s == 0) f = v[i1][i2];
        else if (s == 1) f = dx[i1][i2];
        else if (s == 2) f = dy[i1][i2];
        b.push_back(f);
      }
  P.c = lu_solve(A, b);
  return P;
}

// Spline3D::init (Spline3D.cxx:35-163): v, three first partials, three mixed
// second partials (= 0) and the mixed third partial (= 0) at the 8 corners.
Poly tricubic(const double x[2], const double y[2], const double z[2], const double v[2][2][2],
              const double dx[2][2][2], const double dy[2][2][2], const double dz[2][2][2])
{
  Poly P;
  P.terms = make_terms(3, 3);
  std::vector<Term> F[8];
  for (int s = 0; s < 8; s++) F[s] = P.terms;
  differentiate(F[1], 0);
  differentiate(F[2], 1);
  differentiate(F[3], 2);
  differentiate(F[4], 0); differentiate(F[4], 1);
  differentiate(F[5], 0); differentiate(F[5], 2);
  differentiate(F[6], 1); differentiate(F[6], 2);
  differentiate(F[7], 0); differentiate(F[7], 1); differentiate(F[7], 2);
  std::vector<double> A, b;
  for (int s = 0; s < 8; s++)
    for (int i1 = 0; i1 < 2; i1++)
      for (int i2 = 0; i2 < 2; i2++)
        for (int i3 = 0; i3 < 2; i3++) {
          double xv[3] = {x[i1], y[i2], z[i3]};
          for (size_t j = 0; j < F[s].size(); j++) A.push_back(woC(F[s][j], xv, 3));
          double f = 0.0;
          if (s == 0) f = v[i1][i2][i3];
          else if (s == 1) f = dx[i1][i2][i3];
          else if (s == 2) f = dy[i1][i2][i3];
          else if (s == 3) f = dz[i1][i2][i3];
          b.push_back(f);
        }
  P.c = lu_solve(A, b);
  return P;
}

Poly zero_poly(int dim)
{
  Poly P;
  P.terms = make_terms(dim, 3);
  P.c.assign(P.terms.size(), 0.0);
  return P;
}

// ---- reference knot data ----

// G(cos theta) knots: x, y, dy, d2y (AIREBO/cubici.cxx:42-102).
struct GKnot { double x, y, dy, d2y; };
const GKnot kGC1[5] = {{-1.0, -0.010000, 0.104000, 0.000000},
                       {-2.0 / 3.0, 0.028207, 0.131443, 0.140229},
                       {-1.0 / 2.0, 0.052804, 0.170000, 0.370000},
                       {-1.0 / 3.0, 0.097321, 0.400000, 1.980000},
                       {1.0, 1.000000, 2.834570, 10.264700}};
const GKnot kGC2[5] = {{-1.0, -0.010000, 0.104000, 0.000000},
                       {-2.0 / 3.0, 0.028207, 0.131443, 0.140229},
                       {-1.0 / 2.0, 0.052804, 0.170000, 0.370000},
                       {-1.0 / 3.0, 0.097321, 0.400000, 1.980000},
                       {1.0, 8.000000, 20.243600, 43.9336000}};
const GKnot kGH[4] = {{-1.0, 11.235700, 0.000000, 115.115000},
                      {-5.0 / 6.0, 12.595300, 13.854300, 32.361800},
                      {-1.0 / 2.0, 16.811100, 8.641230, -25.061700},
                      {1.0, 19.991800, 0.333013, -0.474189}};

struct Knot2 { int i, j; double v; };
// P_CC and P_CH knot values (AIREBO/cubici.cxx:129-135, 216-225); all corner
// derivatives are zero in the parameter set the reference uses.
const Knot2 kPCC[] = {{2, 0, -0.000500}, {3, 0, 0.016125}, {1, 1, -0.010960},
                      {2, 1, 0.006326},  {0, 2, -0.027603}, {1, 2, 0.003180}};
const Knot2 kPCH[] = {{1, 0, 0.209337},  {2, 0, -0.064450}, {3, 0, -0.303928},
                      {0, 1, 0.010000},  {1, 1, -0.125123}, {2, 1, -0.298905},
                      {0, 2, -0.122042}, {1, 2, -0.300529}, {0, 3, -0.307585}};

// One step of building a pi_rc-type table (AIREBO/cubici.cxx:292-311):
// set value (both i,j orders), set a partial (both orders), or copy the value
// at k upward for both orders.
enum Op { SET_V, SET_DI, SET_DJ, SET_DK, FILL_UP };
struct TStep { Op op; int i, j, k; double v; };

// pi_rc_CC (AIREBO/cubici.cxx:420-458)
const TStep kPiCC[] = {
  {SET_V, 0, 0, 3, 0.004959}, {FILL_UP, 0, 0, 3, 0},
  {SET_V, 1, 0, 1, 0.021694}, {SET_V, 1, 0, 2, 0.004959}, {FILL_UP, 1, 0, 2, 0},
  {SET_V, 1, 1, 1, 0.052500}, {SET_V, 1, 1, 2, -0.002089}, {SET_V, 1, 1, 3, -0.008043},
  {FILL_UP, 1, 1, 3, 0},
  {SET_V, 2, 0, 1, 0.024699}, {SET_V, 2, 0, 2, -0.005971}, {SET_V, 2, 0, 3, 0.004959},
  {FILL_UP, 2, 0, 3, 0},
  {SET_V, 2, 1, 1, 0.004825}, {SET_DI, 2, 1, 1, -0.026250},
  {SET_V, 2, 1, 2, 0.015000},
  {SET_V, 2, 1, 3, -0.010000},
  {SET_V, 2, 1, 4, -0.011689}, {SET_DK, 2, 1, 4, -0.010022},
  {SET_V, 2, 1, 5, -0.013378}, {SET_DI, 2, 1, 5, -0.027188}, {SET_DK, 2, 1, 5, -0.010022},
  {SET_V, 2, 1, 6, -0.015067}, {SET_DI, 2, 1, 6, -0.027188},
  {SET_V, 2, 1, 7, -0.015067}, {SET_DI, 2, 1, 7, -0.027188},
  {FILL_UP, 2, 1, 7, 0},
  {SET_V, 2, 2, 1, 0.047225}, {SET_V, 2, 2, 2, 0.011000}, {SET_V, 2, 2, 3, 0.019853},
  {SET_V, 2, 2, 4, 0.016544}, {SET_DK, 2, 2, 4, -0.003309},
  {SET_V, 2, 2, 5, 0.013235}, {SET_DK, 2, 2, 5, -0.003309},
  {SET_V, 2, 2, 6, 0.009926}, {SET_DK, 2, 2, 6, -0.003309},
  {SET_V, 2, 2, 7, 0.006618}, {SET_DK, 2, 2, 7, -0.003309},
  {SET_V, 2, 2, 8, 0.003309}, {SET_DK, 2, 2, 8, -0.003309},
  {SET_V, 3, 0, 1, -0.099899}, {SET_V, 3, 0, 2, -0.099899}, {SET_V, 3, 0, 3, 0.004959},
  {FILL_UP, 3, 0, 3, 0},
  {SET_V, 3, 1, 2, -0.062418}, {SET_DJ, 3, 1, 2, 0.037545},
  {SET_V, 3, 1, 3, -0.062418}, {FILL_UP, 3, 1, 3, 0},
  {SET_V, 3, 2, 1, -0.022355},
  {SET_V, 3, 2, 2, -0.022355}, {SET_DJ, 3, 2, 2, 0.062418}, {FILL_UP, 3, 2, 2, 0},
};
// pi_rc_CH (AIREBO/cubici.cxx:478-491)
const TStep kPiCH[] = {
  {SET_V, 1, 1, 1, -0.050000}, {SET_V, 1, 1, 2, -0.050000}, {SET_V, 1, 1, 3, -0.300000},
  {SET_V, 1, 1, 4, -0.050000}, {FILL_UP, 1, 1, 4, 0},
  {SET_V, 2, 0, 5, -0.004524}, {FILL_UP, 2, 0, 5, 0},
  {SET_V, 2, 1, 2, -0.250000}, {SET_V, 2, 1, 3, -0.250000},
  {SET_V, 3, 1, 1, -0.100000}, {SET_V, 3, 1, 2, -0.125000}, {SET_V, 3, 1, 3, -0.125000},
  {SET_V, 3, 1, 4, -0.100000}, {FILL_UP, 3, 1, 4, 0},
};
// pi_rc_HH (AIREBO/cubici.cxx:510)
const TStep kPiHH[] = {{SET_V, 1, 1, 1, 0.124916}};
// Tij (AIREBO/cubici.cxx:529-531)
const TStep kTij[] = {{SET_V, 2, 2, 1, -0.035140}, {SET_V, 2, 2, 2, -0.004048}, {FILL_UP, 2, 2, 2, 0}};

struct Grid3 {
  double F[5][5][16], DI[5][5][16], DJ[5][5][16], DK[5][5][16];
};

void apply_steps(Grid3& g, const TStep* s, size_t n)
{
  std::memset(&g, 0, sizeof(g));
  for (size_t q = 0; q < n; q++) {
    const TStep& t = s[q];
    switch (t.op) {
      case SET_V: g.F[t.i][t.j][t.k] = g.F[t.j][t.i][t.k] = t.v; break;
      case SET_DI: g.DI[t.i][t.j][t.k] = g.DI[t.j][t.i][t.k] = t.v; break;
      case SET_DJ: g.DJ[t.i][t.j][t.k] = g.DJ[t.j][t.i][t.k] = t.v; break;
      case SET_DK: g.DK[t.i][t.j][t.k] = g.DK[t.j][t.i][t.k] = t.v; break;
      case FILL_UP:
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++)
            if ((i == t.i && j == t.j) || (i == t.j && j == t.i))
              for (int k = t.k + 1; k < 16; k++) g.F[i][j][k] = g.F[i][j][t.k];
        break;
    }
  }
}

// Cell polynomials for a 5x5x16 family: cells i,j < 4, k < 15 are solved
// (pi_rc_c1_COMMON_INC, AIREBO/cubici.cxx:333-391); the rest stay empty.
void build_family(const Grid3& g, Poly cells[5][5][16])
{
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 16; k++) cells[i][j][k] = zero_poly(3);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 15; k++) {
        double x[2] = {(double)i, (double)i + 1}, y[2] = {(double)j, (double)j + 1},
               z[2] = {(double)k, (double)k + 1};
        double v[2][2][2], dx[2][2][2], dy[2][2][2], dz[2][2][2];
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++) {
              v[a][b][c] = g.F[i + a][j + b][k + c];
              dx[a][b][c] = g.DI[i + a][j + b][k + c];
              dy[a][b][c] = g.DJ[i + a][j + b][k + c];
              dz[a][b][c] = g.DK[i + a][j + b][k + c];
            }
        cells[i][j][k] = tricubic(x, y, z, v, dx, dy, dz);
      }
}

void put_g(const GKnot* kn, int nknots, GSpline& gs, std::vector<double>& flat)
{
  std::memset(&gs, 0, sizeof(gs));
  gs.npieces = nknots - 1;
  for (int p = 0; p < 4; p++) {
    if (p < nknots - 1) {
      double x[2] = {kn[p].x, kn[p + 1].x}, v[2] = {kn[p].y, kn[p + 1].y},
             dv[2] = {kn[p].dy, kn[p + 1].dy}, d2v[2] = {kn[p].d2y, kn[p + 1].d2y};
      Poly P = quintic(x, v, dv, d2v);
      std::vector<double> f, df;
      emit(P, 0, f);
      emit(P, 1, df);
      gs.x1[p] = x[0];
      gs.x2[p] = x[1];
      flat.push_back(x[0]);
      flat.push_back(x[1]);
      for (int t = 0; t < 6; t++) { gs.f[p][t] = f[t]; flat.push_back(f[t]); }
      for (int t = 0; t < 6; t++) { gs.df[p][t] = df[t]; flat.push_back(df[t]); }
    } else {
      for (int q = 0; q < 14; q++) flat.push_back(0.0);
    }
  }
}

void put_p(const Knot2* kn, size_t nk, double P[4][4][3][16], double Pint[4][4][3],
           std::vector<double>& flat, std::vector<double>& flat_int)
{
  double H[5][5];
  std::memset(H, 0, sizeof(H));
  for (size_t q = 0; q < nk; q++) H[kn[q].i][kn[q].j] = kn[q].v;
  const double zero[2][2] = {{0, 0}, {0, 0}};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double x[2] = {(double)i, (double)i + 1}, y[2] = {(double)j, (double)j + 1};
      double z[2][2] = {{H[i][j], H[i][j + 1]}, {H[i + 1][j], H[i + 1][j + 1]}};
      Poly cell = bicubic(x, y, z, zero, zero);
      for (int d = 0; d < 3; d++) {
        std::vector<double> c;
        emit(cell, d, c);
        for (int t = 0; t < 16; t++) { P[i][j][d][t] = c[t]; flat.push_back(c[t]); }
      }
      // fill_intarg (AIREBO/cubici.cxx:104-115)
      double xv[2] = {(double)i, (double)j};
      for (int d = 0; d < 3; d++) Pint[i][j][d] = eval_poly(cell, d, xv, 2);
    }
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int d = 0; d < 3; d++) flat_int.push_back(Pint[i][j][d]);
}

void put_t(const TStep* steps, size_t ns, double T[5][5][16][4][64], double Tint[5][5][16][4],
           std::vector<double>& flat, std::vector<double>& flat_int)
{
  static Grid3 g;
  apply_steps(g, steps, ns);
  static Poly cells[5][5][16];
  build_family(g, cells);
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 16; k++) {
        for (int d = 0; d < 4; d++) {
          std::vector<double> c;
          emit(cells[i][j][k], d, c);
          for (int t = 0; t < 64; t++) { T[i][j][k][d][t] = c[t]; flat.push_back(c[t]); }
        }
        // fill_intarg (AIREBO/cubici.cxx:394-407)
        double xv[3] = {(double)i, (double)j, (double)k};
        for (int d = 0; d < 4; d++) Tint[i][j][k][d] = eval_poly(cells[i][j][k], d, xv, 3);
      }
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 16; k++)
        for (int d = 0; d < 4; d++) flat_int.push_back(Tint[i][j][k][d]);
}

// ---- Brenner tables (Brenner/cubici.cxx:36-346) ----
struct Knot2v { int i, j; double v; };
// H_CC knots, parameter sets 1 and 2 (Brenner/cubici.cxx:47-60)
const Knot2v kHCC[2][5] = {
  {{1, 1, -0.0175}, {2, 0, -0.0070}, {3, 0, 0.0119}, {1, 2, 0.0115}, {2, 1, 0.0118}},
  {{1, 1, -0.0226}, {2, 0, -0.0061}, {3, 0, 0.0173}, {1, 2, 0.0149}, {2, 1, 0.0160}}};
// H_CH knots and corner derivatives (Brenner/cubici.cxx:115-148)
const Knot2v kHCH[2][9] = {
  {{1, 0, -0.0760}, {2, 0, -0.2163}, {3, 0, -0.3375}, {0, 1, -0.1792}, {0, 2, -0.2407},
   {1, 1, -0.2477}, {2, 1, -0.3320}, {0, 3, -0.3323}, {1, 2, -0.3321}},
  {{1, 0, -0.0984}, {2, 0, -0.2878}, {3, 0, -0.4507}, {0, 1, -0.2479}, {0, 2, -0.3221},
   {1, 1, -0.3344}, {2, 1, -0.4438}, {0, 3, -0.4460}, {1, 2, -0.4449}}};
const Knot2v kHCHdH[2][2] = {{{2, 0, -0.13075}, {1, 1, -0.0764}}, {{2, 0, -0.17615}, {1, 1, -0.09795}}};
const Knot2v kHCHdC[2][2] = {{{0, 2, -0.07655}, {1, 1, -0.12805}}, {{0, 2, -0.09905}, {1, 1, -0.17325}}};

struct Knot3v { int i, j, k; double v; };
// F knots (value, symmetric in i, j), and its i/j derivatives (Brenner/cubici.cxx:205-278)
const Knot3v kFv[2][14] = {
  {{2, 3, 1, -0.0465}, {2, 3, 2, -0.0465}, {1, 2, 2, -0.0355}, {1, 2, 1, 0.0126}, {1, 3, 1, -0.1130},
   {1, 3, 2, -0.1130}, {0, 3, 1, -0.1220}, {0, 3, 2, -0.1220}, {0, 2, 2, -0.0445}, {0, 2, 1, 0.0320},
   {0, 1, 1, 0.1100}, {1, 1, 2, 0.0074}, {1, 1, 1, 0.1511}, {2, 2, 1, 0.0750}},
  {{2, 3, 1, -0.0363}, {2, 3, 2, -0.0363}, {1, 2, 2, -0.0243}, {1, 2, 1, 0.0120}, {1, 3, 1, -0.0903},
   {1, 3, 2, -0.0903}, {0, 3, 1, -0.0904}, {0, 3, 2, -0.0904}, {0, 2, 2, -0.0269}, {0, 2, 1, 0.0427},
   {0, 1, 1, 0.0996}, {1, 1, 2, 0.0108}, {1, 1, 1, 0.1264}, {2, 2, 1, 0.0605}}};
const Knot3v kFdI[2][8] = {
  {{2, 0, 1, -0.1160}, {2, 1, 1, -0.13205}, {2, 0, 2, -0.0610}, {1, 2, 2, 0.02225}, {1, 3, 2, 0.03775},
   {2, 3, 2, 0.0565}, {2, 3, 1, 0.0565}, {2, 1, 2, -0.0602}},
  {{2, 0, 1, -0.0950}, {2, 1, 1, -0.10835}, {2, 0, 2, -0.0452}, {1, 2, 2, 0.01345}, {1, 3, 2, 0.02705},
   {2, 3, 2, 0.04515}, {2, 3, 1, 0.04515}, {2, 1, 2, -0.05055}}};
const Knot3v kFdJ[2][8] = {
  {{0, 2, 1, -0.1160}, {1, 2, 1, -0.13205}, {0, 2, 2, -0.0610}, {2, 1, 2, 0.02225}, {3, 1, 2, 0.03775},
   {3, 2, 2, 0.0565}, {3, 2, 1, 0.0565}, {1, 2, 2, -0.0602}},
  {{0, 2, 1, -0.0950}, {1, 2, 1, -0.10835}, {0, 2, 2, -0.0452}, {2, 1, 2, 0.01345}, {3, 1, 2, 0.02705},
   {3, 2, 2, 0.04515}, {3, 2, 1, 0.04515}, {1, 2, 2, -0.05055}}};

void put_h(const double H[5][5], const double DH[5][5], const double DC[5][5], double out[4][4][3][16],
           std::vector<double>& flat)
{
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      double x[2] = {(double)i, (double)i + 1}, y[2] = {(double)j, (double)j + 1};
      double z[2][2] = {{H[i][j], H[i][j + 1]}, {H[i + 1][j], H[i + 1][j + 1]}};
      double dx[2][2] = {{DH[i][j], DH[i][j + 1]}, {DH[i + 1][j], DH[i + 1][j + 1]}};
      double dy[2][2] = {{DC[i][j], DC[i][j + 1]}, {DC[i + 1][j], DC[i + 1][j + 1]}};
      Poly cell = bicubic(x, y, z, dx, dy);
      for (int d = 0; d < 3; d++) {
        std::vector<double> c;
        emit(cell, d, c);
        for (int t = 0; t < 16; t++) { out[i][j][d][t] = c[t]; flat.push_back(c[t]); }
      }
    }
}

}  // namespace

void build_brenner_tables(int set, BrennerTables* tb, std::vector<double>* flat_out)
{
  const int ps = (set == 2) ? 1 : 0;
  std::vector<double> flat;
  double H[5][5], Z[5][5], DH[5][5], DC[5][5];
  std::memset(Z, 0, sizeof(Z));
  // H_CC: corner values only (Brenner/cubici.cxx:36-96)
  std::memset(H, 0, sizeof(H));
  for (int q = 0; q < 5; q++) H[kHCC[ps][q].i][kHCC[ps][q].j] = kHCC[ps][q].v;
  put_h(H, Z, Z, tb->H[0], flat);
  // H_CH with its corner derivatives (Brenner/cubici.cxx:98-183)
  std::memset(H, 0, sizeof(H));
  std::memset(DH, 0, sizeof(DH));
  std::memset(DC, 0, sizeof(DC));
  for (int q = 0; q < 9; q++) H[kHCH[ps][q].i][kHCH[ps][q].j] = kHCH[ps][q].v;
  for (int q = 0; q < 2; q++) DH[kHCHdH[ps][q].i][kHCHdH[ps][q].j] = kHCHdH[ps][q].v;
  for (int q = 0; q < 2; q++) DC[kHCHdC[ps][q].i][kHCHdC[ps][q].j] = kHCHdC[ps][q].v;
  put_h(H, DH, DC, tb->H[1], flat);
  // F: values symmetric in (i, j), k >= 3 copied from k = 2 (Brenner/cubici.cxx:186-346)
  static double F[5][5][6], FI[5][5][6], FJ[5][5][6];
  std::memset(F, 0, sizeof(F));
  std::memset(FI, 0, sizeof(FI));
  std::memset(FJ, 0, sizeof(FJ));
  for (int q = 0; q < 14; q++) {
    const Knot3v& k = kFv[ps][q];
    F[k.i][k.j][k.k] = F[k.j][k.i][k.k] = k.v;
  }
  for (int q = 0; q < 8; q++) FI[kFdI[ps][q].i][kFdI[ps][q].j][kFdI[ps][q].k] = kFdI[ps][q].v;
  for (int q = 0; q < 8; q++) FJ[kFdJ[ps][q].i][kFdJ[ps][q].j][kFdJ[ps][q].k] = kFdJ[ps][q].v;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 3; k < 6; k++) F[i][j][k] = F[i][j][2];
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 5; k++) {
        double x[2] = {(double)i, (double)i + 1}, y[2] = {(double)j, (double)j + 1},
               z[2] = {(double)k, (double)k + 1};
        double v[2][2][2], dx[2][2][2], dy[2][2][2], dz[2][2][2];
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++) {
              v[a][b][c] = F[i + a][j + b][k + c];
              dx[a][b][c] = FI[i + a][j + b][k + c];
              dy[a][b][c] = FJ[i + a][j + b][k + c];
              dz[a][b][c] = 0.0;
            }
        Poly cell = tricubic(x, y, z, v, dx, dy, dz);
        for (int d = 0; d < 4; d++) {
          std::vector<double> c;
          emit(cell, d, c);
          for (int t = 0; t < 64; t++) { tb->F[i][j][k][d][t] = c[t]; flat.push_back(c[t]); }
        }
      }
  if (flat_out) *flat_out = flat;
}

void build_rebo_tables(ReboTables* tb, std::vector<double>* flat_out)
{
  std::vector<double> flat, pint_cc, pint_ch, tint[4];
  put_g(kGC1, 5, tb->G[0], flat);
  put_g(kGC2, 5, tb->G[1], flat);
  put_g(kGH, 4, tb->G[2], flat);
  put_p(kPCC, sizeof(kPCC) / sizeof(kPCC[0]), tb->P[0], tb->Pint[0], flat, pint_cc);
  put_p(kPCH, sizeof(kPCH) / sizeof(kPCH[0]), tb->P[1], tb->Pint[1], flat, pint_ch);
  flat.insert(flat.end(), pint_cc.begin(), pint_cc.end());
  flat.insert(flat.end(), pint_ch.begin(), pint_ch.end());
  put_t(kPiCC, sizeof(kPiCC) / sizeof(kPiCC[0]), tb->T[0], tb->Tint[0], flat, tint[0]);
  put_t(kPiCH, sizeof(kPiCH) / sizeof(kPiCH[0]), tb->T[1], tb->Tint[1], flat, tint[1]);
  put_t(kPiHH, sizeof(kPiHH) / sizeof(kPiHH[0]), tb->T[2], tb->Tint[2], flat, tint[2]);
  put_t(kTij, sizeof(kTij) / sizeof(kTij[0]), tb->T[3], tb->Tint[3], flat, tint[3]);
  for (int f = 0; f < 4; f++) flat.insert(flat.end(), tint[f].begin(), tint[f].end());
  if (flat_out) *flat_out = flat;
}

// ---- FP32 local-basis tables (ReboTables32) ----
namespace {

long double binom(int n, int k)
{
  long double r = 1.0L;
  for (int q = 1; q <= k; q++) r = r * (n - k + q) / q;
  return r;
}

long double lpow(long double x, int n)
{
  long double r = 1.0L;
  for (int q = 0; q < n; q++) r *= x;
  return r;
}

// Taylor shift of sum_t c_t prod_d x_d^e_d(t) (the term enumeration of the
// FP64 tables, x0 fastest; `deriv` lowers the exponent of that coordinate as
// the derivative polynomials do) to local coordinates u_d = x_d - x0_d.
void shift_poly(const double* c, int nterms, int ndim, int deriv, const double* x0, float* out)
{
  long double acc[64];
  const int nout = ndim == 1 ? 6 : (ndim == 2 ? 16 : 64);
  for (int i = 0; i < nout; i++) acc[i] = 0.0L;
  for (int t = 0; t < nterms; t++) {
    if (c[t] == 0.0) continue;
    int e[3] = {0, 0, 0};
    if (ndim == 1) e[0] = t;
    else if (ndim == 2) { e[0] = t & 3; e[1] = t >> 2; }
    else { e[0] = t & 3; e[1] = (t >> 2) & 3; e[2] = t >> 4; }
    if (deriv) e[deriv - 1] -= 1;
    if (e[0] < 0 || e[1] < 0 || e[2] < 0) continue;
    for (int k0 = 0; k0 <= e[0]; k0++)
      for (int k1 = 0; k1 <= e[1]; k1++)
        for (int k2 = 0; k2 <= e[2]; k2++) {
          long double w = (long double)c[t] * binom(e[0], k0) * lpow(x0[0], e[0] - k0);
          if (ndim > 1) w *= binom(e[1], k1) * lpow(x0[1], e[1] - k1);
          if (ndim > 2) w *= binom(e[2], k2) * lpow(x0[2], e[2] - k2);
          const int idx = ndim == 1 ? k0 : (ndim == 2 ? k0 + 4 * k1 : k0 + 4 * k1 + 16 * k2);
          acc[idx] += w;
        }
  }
  for (int i = 0; i < nout; i++) out[i] = (float)acc[i];
}

}  // namespace

void build_rebo_tables32(const ReboTables& d, ReboTables32* f)
{
  std::memset(f, 0, sizeof(*f));
  for (int g = 0; g < 3; g++) {
    const GSpline& a = d.G[g];
    GSpline32& b = f->G[g];
    b.npieces = a.npieces;
    for (int p = 0; p < 4; p++) {
      b.x1[p] = (float)a.x1[p];
      b.x2[p] = (float)a.x2[p];
      if (p >= a.npieces) continue;
      // expand about the float-rounded knot, the point the device subtracts
      const double x0 = (double)b.x1[p];
      shift_poly(a.f[p], 6, 1, 0, &x0, b.f[p]);
      shift_poly(a.df[p], 6, 1, 1, &x0, b.df[p]);
    }
  }
  for (int fam = 0; fam < 2; fam++)
    for (int h = 0; h < 4; h++)
      for (int c = 0; c < 4; c++) {
        const double x0[2] = {(double)h, (double)c};
        for (int q = 0; q < 3; q++) {
          shift_poly(d.P[fam][h][c][q], 16, 2, q, x0, f->P[fam][h][c][q]);
          f->Pint[fam][h][c][q] = (float)d.Pint[fam][h][c][q];
        }
      }
  for (int fam = 0; fam < 4; fam++)
    for (int i = 0; i < 5; i++)
      for (int j = 0; j < 5; j++)
        for (int k = 0; k < 16; k++) {
          const double x0[3] = {(double)i, (double)j, (double)k};
          for (int q = 0; q < 4; q++) {
            shift_poly(d.T[fam][i][j][k][q], 64, 3, q, x0, f->T[fam][i][j][k][q]);
            f->Tint[fam][i][j][k][q] = (float)d.Tint[fam][i][j][k][q];
          }
        }
}

// The REBO and torsion parameters of the reference, shared by every entry
// point that evaluates them (the context path and the allocation-free one).
void fill_rebo_params(ReboParams& p)
{
  std::memset(&p, 0, sizeof(p));
  const int C = kC, H = kH;
  // REBO::setupPotential1 (REBO.cxx:857-938), converted to A / eV
  p.Q[C][C] = 0.313460; p.Q[C][H] = p.Q[H][C] = 0.340776; p.Q[H][H] = 0.370471;
  p.alpha[C][C] = 4.7465391; p.alpha[C][H] = p.alpha[H][C] = 4.1025498; p.alpha[H][H] = 3.5362986;
  p.A[C][C] = 10953.544; p.A[C][H] = p.A[H][C] = 149.94099; p.A[H][H] = 32.817356;
  p.B[0][C][C] = 12388.792; p.B[0][C][H] = p.B[0][H][C] = 32.355187; p.B[0][H][H] = 29.632593;
  p.B[1][C][C] = 17.567065;
  p.B[2][C][C] = 30.714932;
  p.beta[0][C][C] = 4.7204523; p.beta[0][C][H] = p.beta[0][H][C] = 1.4344581; p.beta[0][H][H] = 1.7158922;
  p.beta[1][C][C] = 1.4332132;
  p.beta[2][C][C] = 1.3826913;
  p.rho[C][H] = p.rho[H][C] = 1.09; p.rho[H][H] = 0.7415887;
  p.R[C][C][0] = 1.7; p.R[H][H][0] = 1.1; p.R[C][H][0] = p.R[H][C][0] = 1.3;
  p.R[C][C][1] = 2.0; p.R[H][H][1] = 1.7; p.R[C][H][1] = p.R[H][C][1] = 1.8;
  p.Rp[C][C][0] = 1.7; p.Rp[H][H][0] = 1.1; p.Rp[C][H][0] = p.Rp[H][C][0] = 1.3;
  p.Rp[C][C][1] = 2.0; p.Rp[H][H][1] = 1.7; p.Rp[C][H][1] = p.Rp[H][C][1] = 1.6;
  p.Ntot[0] = 2;
  p.Ntot[1] = 3;
}

void fill_tors_params(TorsParams& t)
{
  // ETors::setupPotential (AIREBO_ETors.cxx:125-133)
  t.eps[kC][kC] = 0.3079;
  t.eps[kH][kH] = 0.1250;
  t.eps[kC][kH] = t.eps[kH][kC] = 0.1787;
}

}  // namespace mdg
