// Spline evaluation for the REBO correction functions.
//
// The reference stores every spline cell as a monomial polynomial in absolute
// coordinates, solved from corner data at start-up (SplineMultiD,
// mdtk/SplineAux.hpp:133-241).  Its value is the sequential sum over terms in
// x0-fastest order of (multiplier*c) * x0^p0 * x1^p1 * x2^p2
// (SplineTerm::operator(), SplineAux.hpp:82-94; intpow, tools.hpp:107-133).
// The tables here hold multiplier*c per term; the sum is evaluated in the same
// order with explicitly rounded multiply/add (no FMA contraction), because the
// monomial sums cancel heavily (sum |terms| reaches ~3e6 in the pi_rc cells).
#pragma once

#include "mdg_common.cuh"

namespace mdg {

#if defined(__CUDA_ARCH__)
MDG_DEV double mul_rn(double a, double b) { return __dmul_rn(a, b); }
MDG_DEV double add_rn(double a, double b) { return __dadd_rn(a, b); }
#else
inline double mul_rn(double a, double b) { return a * b; }
inline double add_rn(double a, double b) { return a + b; }
#endif

// intpow for the small non-negative powers the splines use (tools.hpp:107-133),
// left-to-right products.
MDG_HD double ipow(double a, int n)
{
  double v;
  switch (n) {
    case 0: return 1.0;
    case 1: return a;
    case 2: return mul_rn(a, a);
    case 3: v = mul_rn(a, a); return mul_rn(v, a);
    case 4: v = mul_rn(a, a); v = mul_rn(v, a); return mul_rn(v, a);
    default: v = mul_rn(a, a); v = mul_rn(v, a); v = mul_rn(v, a); return mul_rn(v, a);
  }
}

// Piecewise quintic G(cos theta) (FuncG, AIREBO/cubici.hpp:42-107).
struct GSpline {
  int npieces;
  int pad;
  double x1[4];   // lower knot of each piece
  double x2[4];   // upper knot
  double f[4][6];
  double df[4][6];
};

// All REBO spline tables, device resident (layout mirrors the host builder).
struct ReboTables {
  GSpline G[3];                 // G_C1, G_C2, G_H
  double P[2][4][4][3][16];     // P_CC / P_CH: cell [h][c], poly f / dH / dC
  double Pint[2][4][4][3];      // exact-integer shortcut tables (fill_intarg)
  double T[4][5][5][16][4][64]; // pi_rc CC / CH / HH, Tij: cell [i][j][k], poly f/di/dj/dk
  double Tint[4][5][5][16][4];  // their exact-integer tables
};

// 1-D quintic piece: sum_t coef[t] * x^(t - d), d = 0 for the value poly and
// 1 for the derivative poly (whose term 0 is always zero).
MDG_HD double poly1(const double* c, double x, int deriv)
{
  double val = 0.0;
  for (int t = 0; t < 6; t++) {
    double ct = c[t];
    if (ct == 0.0) continue;
    val = add_rn(val, mul_rn(ct, ipow(x, t - deriv)));
  }
  return val;
}

// FuncG::operator() / dCosT: first piece whose upper knot is >= CosT.
MDG_HD double g_eval(const GSpline& g, double cost, int deriv)
{
  int p = 0;
  for (p = 0; p < g.npieces; p++)
    if (cost <= g.x2[p]) break;
  if (p >= g.npieces) p = g.npieces - 1;
  return poly1(deriv ? g.df[p] : g.f[p], cost, deriv);
}

// Bicubic cell polynomial; d = 0 value, 1 = d/dx0, 2 = d/dx1.
MDG_HD double poly2(const double* c, double x0, double x1, int d)
{
  double val = 0.0;
  for (int t = 0; t < 16; t++) {
    double ct = c[t];
    if (ct == 0.0) continue;
    int p0 = t & 3, p1 = t >> 2;
    if (d == 1) p0 -= 1;
    if (d == 2) p1 -= 1;
    double v = mul_rn(ct, ipow(x0, p0));
    v = mul_rn(v, ipow(x1, p1));
    val = add_rn(val, v);
  }
  return val;
}

// Tricubic cell polynomial; d = 0 value, 1..3 = d/dx0..d/dx2.
MDG_HD double poly3(const double* c, double x0, double x1, double x2, int d)
{
  double val = 0.0;
  for (int t = 0; t < 64; t++) {
    double ct = c[t];
    if (ct == 0.0) continue;
    int p0 = t & 3, p1 = (t >> 2) & 3, p2 = t >> 4;
    if (d == 1) p0 -= 1;
    if (d == 2) p1 -= 1;
    if (d == 3) p2 -= 1;
    double v = mul_rn(ct, ipow(x0, p0));
    v = mul_rn(v, ipow(x1, p1));
    v = mul_rn(v, ipow(x2, p2));
    val = add_rn(val, v);
  }
  return val;
}

// P_CC / P_CH (FuncP_*, AIREBO/cubici.hpp:207-298): value and both partials.
// Zero for h >= 4 or c >= 4; exact-integer arguments read the intarg tables.
MDG_HD void p_eval(const ReboTables& tb, int fam, double h, double c, double& v, double& dh, double& dc,
                   unsigned int* status)
{
  v = dh = dc = 0.0;
  if (!(h >= 0 && c >= 0)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (h >= 4 || c >= 4) return;
  int hi = (int)h, ci = (int)c;
  if ((double)hi == h && (double)ci == c) {
    v = tb.Pint[fam][hi][ci][0];
    dh = tb.Pint[fam][hi][ci][1];
    dc = tb.Pint[fam][hi][ci][2];
    return;
  }
  const double* cell = tb.P[fam][hi][ci][0];
  v = poly2(cell, h, c, 0);
  dh = poly2(cell + 16, h, c, 1);
  dc = poly2(cell + 32, h, c, 2);
}

MDG_HD double p_value(const ReboTables& tb, int fam, double h, double c)
{
  if (!(h >= 0 && c >= 0)) return 0.0;
  if (h >= 4 || c >= 4) return 0.0;
  int hi = (int)h, ci = (int)c;
  if ((double)hi == h && (double)ci == c) return tb.Pint[fam][hi][ci][0];
  return poly2(tb.P[fam][hi][ci][0], h, c, 0);
}

// pi_rc CC/CH/HH and Tij (Func_pi_rc, AIREBO/cubici.hpp:301-369): value and
// the three partials.  Zero for i >= 4 or j >= 4; k is clamped to 15 (cells
// [.][.][15] are empty, so the function is zero from Nconj = 15 on).
MDG_HD void t_eval(const ReboTables& tb, int fam, double i, double j, double k, double* out,
                   unsigned int* status)
{
  out[0] = out[1] = out[2] = out[3] = 0.0;
  if (!(i >= 0 && j >= 0 && k >= 1)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (i >= 4 || j >= 4) return;
  if (k > 15) k = 15;
  int ii = (int)i, jj = (int)j, kk = (int)k;
  if ((double)ii == i && (double)jj == j && (double)kk == k) {
    const double* t = tb.Tint[fam][ii][jj][kk];
    out[0] = t[0]; out[1] = t[1]; out[2] = t[2]; out[3] = t[3];
    return;
  }
  const double* cell = tb.T[fam][ii][jj][kk][0];
  out[0] = poly3(cell, i, j, k, 0);
  out[1] = poly3(cell + 64, i, j, k, 1);
  out[2] = poly3(cell + 128, i, j, k, 2);
  out[3] = poly3(cell + 192, i, j, k, 3);
}

MDG_HD double t_value(const ReboTables& tb, int fam, double i, double j, double k)
{
  if (!(i >= 0 && j >= 0 && k >= 1)) return 0.0;
  if (i >= 4 || j >= 4) return 0.0;
  if (k > 15) k = 15;
  int ii = (int)i, jj = (int)j, kk = (int)k;
  if ((double)ii == i && (double)jj == j && (double)kk == k) return tb.Tint[fam][ii][jj][kk][0];
  return poly3(tb.T[fam][ii][jj][kk][0], i, j, k, 0);
}

// ---------------------------------------------------------------------------
// Dual arguments (adjoint path).  Values and first-derivative outputs are the
// FP64 path's (the same cells, the same integer shortcut); tangents come from
// the derivatives of the cell polynomials.  At an exact-integer argument the
// second derivatives are taken from the cell the argument opens (the one the
// non-integer path uses just above it).

// d/dx of poly1(c, x, deriv)
MDG_HD double poly1_dx(const double* c, double x, int deriv)
{
  double v = 0.0;
  for (int t = 0; t < 6; t++) {
    const int p = t - deriv;
    if (c[t] == 0.0 || p < 1) continue;
    v += c[t] * p * ipow(x, p - 1);
  }
  return v;
}

MDG_HD dual g_eval(const GSpline& g, dual cost, int deriv)
{
  int p = 0;
  for (p = 0; p < g.npieces; p++)
    if (cost.v <= g.x2[p]) break;
  if (p >= g.npieces) p = g.npieces - 1;
  const double* c = deriv ? g.df[p] : g.f[p];
  return dual(poly1(c, cost.v, deriv), poly1_dx(c, cost.v, deriv) * cost.d);
}

// gradient of poly2(c, x0, x1, d) in (x0, x1)
MDG_HD void poly2_grad(const double* c, double x0, double x1, int d, double* g)
{
  g[0] = g[1] = 0.0;
  for (int t = 0; t < 16; t++) {
    const double ct = c[t];
    if (ct == 0.0) continue;
    int p0 = t & 3, p1 = t >> 2;
    if (d == 1) p0 -= 1;
    if (d == 2) p1 -= 1;
    if (p0 < 0 || p1 < 0) continue;
    if (p0 >= 1) g[0] += ct * p0 * ipow(x0, p0 - 1) * ipow(x1, p1);
    if (p1 >= 1) g[1] += ct * p1 * ipow(x0, p0) * ipow(x1, p1 - 1);
  }
}

MDG_HD void p_eval(const ReboTables& tb, int fam, dual h, dual c, dual& v, dual& dh, dual& dc, unsigned int* status)
{
  double vv, dhv, dcv;
  p_eval(tb, fam, h.v, c.v, vv, dhv, dcv, status);
  double a[2] = {0.0, 0.0}, b[2] = {0.0, 0.0};
  if (h.v >= 0 && c.v >= 0 && h.v < 4 && c.v < 4) {
    const double* cell = tb.P[fam][(int)h.v][(int)c.v][0];
    poly2_grad(cell + 16, h.v, c.v, 1, a);
    poly2_grad(cell + 32, h.v, c.v, 2, b);
  }
  v = dual(vv, dhv * h.d + dcv * c.d);
  dh = dual(dhv, a[0] * h.d + a[1] * c.d);
  dc = dual(dcv, b[0] * h.d + b[1] * c.d);
}

MDG_HD dual p_value(const ReboTables& tb, int fam, dual h, dual c)
{
  dual v, dh, dc;
  p_eval(tb, fam, h, c, v, dh, dc, nullptr);
  return v;
}

// gradient of poly3(c, x0, x1, x2, d) in (x0, x1, x2)
MDG_HD void poly3_grad(const double* c, double x0, double x1, double x2, int d, double* g)
{
  g[0] = g[1] = g[2] = 0.0;
  for (int t = 0; t < 64; t++) {
    const double ct = c[t];
    if (ct == 0.0) continue;
    int p0 = t & 3, p1 = (t >> 2) & 3, p2 = t >> 4;
    if (d == 1) p0 -= 1;
    if (d == 2) p1 -= 1;
    if (d == 3) p2 -= 1;
    if (p0 < 0 || p1 < 0 || p2 < 0) continue;
    const double a0 = ipow(x0, p0), a1 = ipow(x1, p1), a2 = ipow(x2, p2);
    if (p0 >= 1) g[0] += ct * p0 * ipow(x0, p0 - 1) * a1 * a2;
    if (p1 >= 1) g[1] += ct * p1 * a0 * ipow(x1, p1 - 1) * a2;
    if (p2 >= 1) g[2] += ct * p2 * a0 * a1 * ipow(x2, p2 - 1);
  }
}

MDG_HD void t_eval(const ReboTables& tb, int fam, dual i, dual j, dual k, dual* out, unsigned int* status)
{
  double o[4];
  t_eval(tb, fam, i.v, j.v, k.v, o, status);
  double kv = k.v, kd = k.d;
  if (kv > 15) { kv = 15; kd = 0.0; }
  double h[4][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  if (i.v >= 0 && j.v >= 0 && k.v >= 1 && i.v < 4 && j.v < 4) {
    const double* cell = tb.T[fam][(int)i.v][(int)j.v][(int)kv][0];
    for (int q = 1; q < 4; q++) poly3_grad(cell + 64 * q, i.v, j.v, kv, q, h[q]);
  }
  out[0] = dual(o[0], o[1] * i.d + o[2] * j.d + o[3] * kd);
  for (int q = 1; q < 4; q++) out[q] = dual(o[q], h[q][0] * i.d + h[q][1] * j.d + h[q][2] * kd);
}

MDG_HD dual t_value(const ReboTables& tb, int fam, dual i, dual j, dual k)
{
  dual o[4];
  t_eval(tb, fam, i, j, k, o, nullptr);
  return o[0];
}

// ---------------------------------------------------------------------------
// FP32 tables of the mixed-precision path.  The FP64 tables above keep the
// reference's monomials in absolute coordinates, whose terms cancel to ~1e-7
// of their magnitude (sum |terms| ~3e6 in the pi_rc cells): float cannot
// carry that.  Here every cell polynomial is re-expanded about the cell's
// lower corner (a Taylor shift done in long double on the host) and evaluated
// by Horner's rule in local coordinates u = x - corner, u in [0, 1) on the
// bicubic/tricubic grids.  The functions are the same polynomials; only the
// basis and the rounding differ.
struct GSpline32 {
  int npieces;
  int pad;
  float x1[4];    // expansion point of each piece (its lower knot)
  float x2[4];    // upper knots
  float f[4][6];  // value poly in u = x - x1, coefficient of u^t
  float df[4][6]; // derivative poly in u
};

struct ReboTables32 {
  GSpline32 G[3];
  float P[2][4][4][3][16];      // cell [h][c], poly f/dH/dC: d[a + 4b] u^a v^b
  float Pint[2][4][4][3];
  float T[4][5][5][16][4][64];  // cell [i][j][k], poly f/di/dj/dk: d[a + 4b + 16c] u^a v^b w^c
  float Tint[4][5][5][16][4];
};

MDG_HD float horner6(const float* c, float u)
{
  float v = c[5];
  for (int t = 4; t >= 0; t--) v = fmaf(v, u, c[t]);
  return v;
}
MDG_HD float horner4(const float* c, float u)
{
  return fmaf(fmaf(fmaf(c[3], u, c[2]), u, c[1]), u, c[0]);
}
MDG_HD float local2(const float* d, float u, float v)
{
  return horner4(d + 12, u) * v * v * v + horner4(d + 8, u) * v * v + horner4(d + 4, u) * v + horner4(d, u);
}
MDG_HD float local3(const float* d, float u, float v, float w)
{
  float r = 0.0f;
  for (int c = 3; c >= 0; c--) {
    const float* e = d + 16 * c;
    float s = fmaf(fmaf(fmaf(horner4(e + 12, u), v, horner4(e + 8, u)), v, horner4(e + 4, u)), v, horner4(e, u));
    r = fmaf(r, w, s);
  }
  return r;
}

MDG_HD f32 g_eval(const GSpline32& g, f32 cost, int deriv)
{
  int p = 0;
  for (p = 0; p < g.npieces; p++)
    if (cost.v <= g.x2[p]) break;
  if (p >= g.npieces) p = g.npieces - 1;
  return mkf(horner6(deriv ? g.df[p] : g.f[p], cost.v - g.x1[p]));
}

MDG_HD void p_eval(const ReboTables32& tb, int fam, f32 h, f32 c, f32& v, f32& dh, f32& dc, unsigned int* status)
{
  v = dh = dc = 0.0;
  if (!(h.v >= 0 && c.v >= 0)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (h.v >= 4 || c.v >= 4) return;
  int hi = (int)h.v, ci = (int)c.v;
  if ((float)hi == h.v && (float)ci == c.v) {
    v = tb.Pint[fam][hi][ci][0];
    dh = tb.Pint[fam][hi][ci][1];
    dc = tb.Pint[fam][hi][ci][2];
    return;
  }
  const float* cell = tb.P[fam][hi][ci][0];
  const float u = h.v - hi, w = c.v - ci;
  v = mkf(local2(cell, u, w));
  dh = mkf(local2(cell + 16, u, w));
  dc = mkf(local2(cell + 32, u, w));
}

MDG_HD f32 p_value(const ReboTables32& tb, int fam, f32 h, f32 c)
{
  if (!(h.v >= 0 && c.v >= 0)) return 0.0;
  if (h.v >= 4 || c.v >= 4) return 0.0;
  int hi = (int)h.v, ci = (int)c.v;
  if ((float)hi == h.v && (float)ci == c.v) return tb.Pint[fam][hi][ci][0];
  return mkf(local2(tb.P[fam][hi][ci][0], h.v - hi, c.v - ci));
}

MDG_HD void t_eval(const ReboTables32& tb, int fam, f32 i, f32 j, f32 k, f32* out, unsigned int* status)
{
  out[0] = out[1] = out[2] = out[3] = 0.0;
  if (!(i.v >= 0 && j.v >= 0 && k.v >= 1)) { if (status) *status |= ST_SPLINE_DOMAIN; return; }
  if (i.v >= 4 || j.v >= 4) return;
  float kc = k.v > 15 ? 15.0f : k.v;
  int ii = (int)i.v, jj = (int)j.v, kk = (int)kc;
  if ((float)ii == i.v && (float)jj == j.v && (float)kk == kc) {
    const float* t = tb.Tint[fam][ii][jj][kk];
    out[0] = t[0]; out[1] = t[1]; out[2] = t[2]; out[3] = t[3];
    return;
  }
  const float* cell = tb.T[fam][ii][jj][kk][0];
  const float u = i.v - ii, v = j.v - jj, w = kc - kk;
  out[0] = mkf(local3(cell, u, v, w));
  out[1] = mkf(local3(cell + 64, u, v, w));
  out[2] = mkf(local3(cell + 128, u, v, w));
  out[3] = mkf(local3(cell + 192, u, v, w));
}

MDG_HD f32 t_value(const ReboTables32& tb, int fam, f32 i, f32 j, f32 k)
{
  if (!(i.v >= 0 && j.v >= 0 && k.v >= 1)) return 0.0;
  if (i.v >= 4 || j.v >= 4) return 0.0;
  float kc = k.v > 15 ? 15.0f : k.v;
  int ii = (int)i.v, jj = (int)j.v, kk = (int)kc;
  if ((float)ii == i.v && (float)jj == j.v && (float)kk == kc) return tb.Tint[fam][ii][jj][kk][0];
  return mkf(local3(tb.T[fam][ii][jj][kk][0], i.v - ii, j.v - jj, kc - kk));
}

}  // namespace mdg
