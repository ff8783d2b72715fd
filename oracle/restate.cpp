// CPU restatement of the MDTK hot-path energies: implementation and C ABI
// (test infrastructure only; see restate.hpp).
#include "restate.hpp"

#include <algorithm>
#include <map>

namespace rs {

// ------------------------------------------------------------ tables
Tables::Tables()
{
  std::memset(this, 0, sizeof(*this));
  // G_C1, G_C2, G_H knots: x, y, y', y'' (AIREBO/cubici.cxx:52-56, 73-77, 94-97)
  const double c1[5][4] = {{-1.0, -0.010000, 0.104000, 0.000000}, {-2.0 / 3.0, 0.028207, 0.131443, 0.140229},
                           {-1.0 / 2.0, 0.052804, 0.170000, 0.370000}, {-1.0 / 3.0, 0.097321, 0.400000, 1.980000},
                           {1.0, 1.000000, 2.834570, 10.264700}};
  std::memcpy(gc1, c1, sizeof(c1));
  std::memcpy(gc2, c1, sizeof(c1));
  gc2[4][1] = 8.000000;
  gc2[4][2] = 20.243600;
  gc2[4][3] = 43.9336000;
  const double h[4][4] = {{-1.0, 11.235700, 0.000000, 115.115000}, {-5.0 / 6.0, 12.595300, 13.854300, 32.361800},
                          {-1.0 / 2.0, 16.811100, 8.641230, -25.061700}, {1.0, 19.991800, 0.333013, -0.474189}};
  std::memcpy(gh, h, sizeof(h));
  // P_CC (AIREBO/cubici.cxx:130-135), P_CH (217-225)
  pcc[2][0] = -0.000500; pcc[3][0] = 0.016125; pcc[1][1] = -0.010960;
  pcc[2][1] = 0.006326; pcc[0][2] = -0.027603; pcc[1][2] = 0.003180;
  pch[1][0] = 0.209337; pch[2][0] = -0.064450; pch[3][0] = -0.303928; pch[0][1] = 0.010000;
  pch[1][1] = -0.125123; pch[2][1] = -0.298905; pch[0][2] = -0.122042; pch[1][2] = -0.300529;
  pch[0][3] = -0.307585;
  // pi_rc / Tij families: value and partials set for both (i,j) orders, and
  // "fill up" copies the value at k to every larger k (AIREBO/cubici.cxx:292-311)
  auto V = [&](int f, int i, int j, int k, double v) { fv[f][i][j][k] = fv[f][j][i][k] = v; };
  auto DI = [&](int f, int i, int j, int k, double v) { fi[f][i][j][k] = fi[f][j][i][k] = v; };
  auto DJ = [&](int f, int i, int j, int k, double v) { fj[f][i][j][k] = fj[f][j][i][k] = v; };
  auto DK = [&](int f, int i, int j, int k, double v) { fk[f][i][j][k] = fk[f][j][i][k] = v; };
  auto UP = [&](int f, int i, int j, int k) {
    for (int kk = k + 1; kk < 16; kk++) { fv[f][i][j][kk] = fv[f][i][j][k]; fv[f][j][i][kk] = fv[f][j][i][k]; }
  };
  // CC (AIREBO/cubici.cxx:420-458)
  V(0, 0, 0, 3, 0.004959); UP(0, 0, 0, 3);
  V(0, 1, 0, 1, 0.021694); V(0, 1, 0, 2, 0.004959); UP(0, 1, 0, 2);
  V(0, 1, 1, 1, 0.052500); V(0, 1, 1, 2, -0.002089); V(0, 1, 1, 3, -0.008043); UP(0, 1, 1, 3);
  V(0, 2, 0, 1, 0.024699); V(0, 2, 0, 2, -0.005971); V(0, 2, 0, 3, 0.004959); UP(0, 2, 0, 3);
  V(0, 2, 1, 1, 0.004825); DI(0, 2, 1, 1, -0.026250);
  V(0, 2, 1, 2, 0.015000);
  V(0, 2, 1, 3, -0.010000);
  V(0, 2, 1, 4, -0.011689); DK(0, 2, 1, 4, -0.010022);
  V(0, 2, 1, 5, -0.013378); DI(0, 2, 1, 5, -0.027188); DK(0, 2, 1, 5, -0.010022);
  V(0, 2, 1, 6, -0.015067); DI(0, 2, 1, 6, -0.027188);
  V(0, 2, 1, 7, -0.015067); DI(0, 2, 1, 7, -0.027188); UP(0, 2, 1, 7);
  V(0, 2, 2, 1, 0.047225); V(0, 2, 2, 2, 0.011000); V(0, 2, 2, 3, 0.019853);
  V(0, 2, 2, 4, 0.016544); DK(0, 2, 2, 4, -0.003309);
  V(0, 2, 2, 5, 0.013235); DK(0, 2, 2, 5, -0.003309);
  V(0, 2, 2, 6, 0.009926); DK(0, 2, 2, 6, -0.003309);
  V(0, 2, 2, 7, 0.006618); DK(0, 2, 2, 7, -0.003309);
  V(0, 2, 2, 8, 0.003309); DK(0, 2, 2, 8, -0.003309);
  V(0, 3, 0, 1, -0.099899); V(0, 3, 0, 2, -0.099899); V(0, 3, 0, 3, 0.004959); UP(0, 3, 0, 3);
  V(0, 3, 1, 2, -0.062418); DJ(0, 3, 1, 2, 0.037545);
  V(0, 3, 1, 3, -0.062418); UP(0, 3, 1, 3);
  V(0, 3, 2, 1, -0.022355);
  V(0, 3, 2, 2, -0.022355); DJ(0, 3, 2, 2, 0.062418); UP(0, 3, 2, 2);
  // CH (AIREBO/cubici.cxx:478-491)
  V(1, 1, 1, 1, -0.050000); V(1, 1, 1, 2, -0.050000); V(1, 1, 1, 3, -0.300000);
  V(1, 1, 1, 4, -0.050000); UP(1, 1, 1, 4);
  V(1, 2, 0, 5, -0.004524); UP(1, 2, 0, 5);
  V(1, 2, 1, 2, -0.250000); V(1, 2, 1, 3, -0.250000);
  V(1, 3, 1, 1, -0.100000); V(1, 3, 1, 2, -0.125000); V(1, 3, 1, 3, -0.125000);
  V(1, 3, 1, 4, -0.100000); UP(1, 3, 1, 4);
  // HH (AIREBO/cubici.cxx:510)
  V(2, 1, 1, 1, 0.124916);
  // Tij (AIREBO/cubici.cxx:529-531)
  V(3, 2, 2, 1, -0.035140); V(3, 2, 2, 2, -0.004048); UP(3, 2, 2, 2);
  // Brenner H_CC (Brenner/cubici.cxx:47-60), H_CH (115-148), F (205-287)
  const double hccv[2][5] = {{-0.0175, -0.0070, 0.0119, 0.0115, 0.0118}, {-0.0226, -0.0061, 0.0173, 0.0149, 0.0160}};
  for (int s = 0; s < 2; s++) {
    hcc[s][1][1] = hccv[s][0]; hcc[s][2][0] = hccv[s][1]; hcc[s][3][0] = hccv[s][2];
    hcc[s][1][2] = hccv[s][3]; hcc[s][2][1] = hccv[s][4];
  }
  const double hchv[2][9] = {{-0.0760, -0.2163, -0.3375, -0.1792, -0.2407, -0.2477, -0.3320, -0.3323, -0.3321},
                             {-0.0984, -0.2878, -0.4507, -0.2479, -0.3221, -0.3344, -0.4438, -0.4460, -0.4449}};
  for (int s = 0; s < 2; s++) {
    hch[s][1][0] = hchv[s][0]; hch[s][2][0] = hchv[s][1]; hch[s][3][0] = hchv[s][2];
    hch[s][0][1] = hchv[s][3]; hch[s][0][2] = hchv[s][4]; hch[s][1][1] = hchv[s][5];
    hch[s][2][1] = hchv[s][6]; hch[s][0][3] = hchv[s][7]; hch[s][1][2] = hchv[s][8];
  }
  hchdh[0][2][0] = -0.13075; hchdh[0][1][1] = -0.0764; hchdc[0][0][2] = -0.07655; hchdc[0][1][1] = -0.12805;
  hchdh[1][2][0] = -0.17615; hchdh[1][1][1] = -0.09795; hchdc[1][0][2] = -0.09905; hchdc[1][1][1] = -0.17325;
  const double fvv[2][14] = {
    {-0.0465, -0.0465, -0.0355, 0.0126, -0.1130, -0.1130, -0.1220, -0.1220, -0.0445, 0.0320, 0.1100, 0.0074, 0.1511, 0.0750},
    {-0.0363, -0.0363, -0.0243, 0.0120, -0.0903, -0.0903, -0.0904, -0.0904, -0.0269, 0.0427, 0.0996, 0.0108, 0.1264, 0.0605}};
  const int fidx[14][3] = {{2, 3, 1}, {2, 3, 2}, {1, 2, 2}, {1, 2, 1}, {1, 3, 1}, {1, 3, 2}, {0, 3, 1},
                           {0, 3, 2}, {0, 2, 2}, {0, 2, 1}, {0, 1, 1}, {1, 1, 2}, {1, 1, 1}, {2, 2, 1}};
  const double fiv[2][8] = {{-0.1160, -0.13205, -0.0610, 0.02225, 0.03775, 0.0565, 0.0565, -0.0602},
                            {-0.0950, -0.10835, -0.0452, 0.01345, 0.02705, 0.04515, 0.04515, -0.05055}};
  const int fiidx[8][3] = {{2, 0, 1}, {2, 1, 1}, {2, 0, 2}, {1, 2, 2}, {1, 3, 2}, {2, 3, 2}, {2, 3, 1}, {2, 1, 2}};
  for (int s = 0; s < 2; s++) {
    for (int q = 0; q < 14; q++) {
      const int* ix = fidx[q];
      bf[s][ix[0]][ix[1]][ix[2]] = bf[s][ix[1]][ix[0]][ix[2]] = fvv[s][q];
    }
    for (int q = 0; q < 8; q++) {
      const int* ix = fiidx[q];
      bfi[s][ix[0]][ix[1]][ix[2]] = fiv[s][q];
      bfj[s][ix[1]][ix[0]][ix[2]] = fiv[s][q];  // dF/dj at (j, i) mirrors dF/di at (i, j)
    }
    for (int i = 0; i < 5; i++)
      for (int j = 0; j < 5; j++)
        for (int k = 3; k < 6; k++) bf[s][i][j][k] = bf[s][i][j][2];
  }
}

Params::Params(int lj_cut_mode)
{
  std::memset(this, 0, sizeof(*this));
  const int C = 0, H = 1;
  Q[C][C] = 0.313460; Q[C][H] = Q[H][C] = 0.340776; Q[H][H] = 0.370471;
  alpha[C][C] = 4.7465391; alpha[C][H] = alpha[H][C] = 4.1025498; alpha[H][H] = 3.5362986;
  A[C][C] = 10953.544; A[C][H] = A[H][C] = 149.94099; A[H][H] = 32.817356;
  B[0][C][C] = 12388.792; B[0][C][H] = B[0][H][C] = 32.355187; B[0][H][H] = 29.632593;
  B[1][C][C] = 17.567065; B[2][C][C] = 30.714932;
  beta[0][C][C] = 4.7204523; beta[0][C][H] = beta[0][H][C] = 1.4344581; beta[0][H][H] = 1.7158922;
  beta[1][C][C] = 1.4332132; beta[2][C][C] = 1.3826913;
  rho[C][H] = rho[H][C] = 1.09; rho[H][H] = 0.7415887;
  R[C][C][0] = 1.7; R[H][H][0] = 1.1; R[C][H][0] = R[H][C][0] = 1.3;
  R[C][C][1] = 2.0; R[H][H][1] = 1.7; R[C][H][1] = R[H][C][1] = 1.8;
  std::memcpy(Rp, R, sizeof(R));
  Rp[C][H][1] = Rp[H][C][1] = 1.6;
  sigma[C][C] = 3.40; sigma[H][H] = 2.65; sigma[C][H] = sigma[H][C] = 0.5 * (3.40 + 2.65);
  eps[C][C] = 0.00284; eps[H][H] = 0.00150; eps[C][H] = eps[H][C] = std::sqrt(0.00284 * 0.00150);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      RLJ[a][b][0] = sigma[a][b];
      RLJ[a][b][1] = sigma[a][b] * std::pow(2.0, 1.0 / 6.0);
    }
  RL[C][C][0] = 5.0; RL[H][H][0] = 4.0; RL[C][H][0] = RL[H][C][0] = 4.5;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) RL[a][b][1] = RL[a][b][0] + 0.5;
  if (lj_cut_mode == 1)
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) { RL[a][b][1] = 3.0 * sigma[a][b]; RL[a][b][0] = RL[a][b][1] - 0.5; }
  bw[C][C][0] = 0.77; bw[H][H][0] = 0.32; bw[C][H][0] = bw[H][C][0] = 0.75;
  bw[C][C][1] = 0.81; bw[H][H][1] = 0.42; bw[C][H][1] = bw[H][C][1] = 0.90;
  teps[C][C] = 0.3079; teps[H][H] = 0.1250; teps[C][H] = teps[H][C] = 0.1787;
  // Brenner sets
  const double Re_[2][3] = {{1.315, 0.74144, 1.1199}, {1.39, 0.74144, 1.1199}};
  const double De_[2][3] = {{6.325, 4.7509, 3.6422}, {6.0, 4.7509, 3.6422}};
  const double be_[2][3] = {{1.5, 1.9436, 1.9583}, {2.1, 1.9436, 1.9583}};
  const double S_[2][3] = {{1.29, 2.3432, 1.7386}, {1.22, 2.3432, 1.69077}};
  const double dl_[2] = {0.80469, 0.5};
  const double al_[2] = {3.0, 4.0};
  for (int s = 0; s < 2; s++) {
    bRe[s][C][C] = Re_[s][0]; bRe[s][H][H] = Re_[s][1]; bRe[s][C][H] = bRe[s][H][C] = Re_[s][2];
    bDe[s][C][C] = De_[s][0]; bDe[s][H][H] = De_[s][1]; bDe[s][C][H] = bDe[s][H][C] = De_[s][2];
    bbeta[s][C][C] = be_[s][0]; bbeta[s][H][H] = be_[s][1]; bbeta[s][C][H] = bbeta[s][H][C] = be_[s][2];
    bS[s][C][C] = S_[s][0]; bS[s][H][H] = S_[s][1]; bS[s][C][H] = bS[s][H][C] = S_[s][2];
    bdelta[s][C][C] = bdelta[s][H][H] = dl_[s];
    balpha[s][H][H][H] = balpha[s][H][H][C] = balpha[s][H][C][H] = balpha[s][H][C][C] = balpha[s][C][H][H] = al_[s];
  }
  bao[0] = 0.011304; bco[0] = 19.0; bdo[0] = 2.5; bGHH[0] = 4.0;
  bao[1] = 0.00020813; bco[1] = 330.0; bdo[1] = 3.5; bGHH[1] = 12.33;
}

const Tables& tables()
{
  static Tables t;
  return t;
}

// ------------------------------------------------------------ evaluation
template <class T>
struct Eval {
  const System& S;
  const std::vector<V3<T>>& x;
  const Params& P;
  const Tables& Tb;
  int bset;  // Brenner set index 0/1

  // bonded neighbours (REBO/Brenner cutoffs, |r|^2 <= R2^2), ascending, and
  // the LJ Verlet partners (|r| < 1.44 Rcut of the LJ term); found with plain
  // doubles so that the search itself is not counted
  std::vector<std::vector<int>> nb, ljl;
  // per directed bond: r and the cutoff f (computed once, as AtomsPair and
  // REBO::countNeighbours cache them); per atom: Nt, NH, NC over all bonds
  std::vector<std::vector<T>> br, bf;
  std::vector<T> Nt_, NH_, NC_;

  Eval(const System& s, const std::vector<V3<T>>& xx, const Params& p, int brenner_set, bool with_lj = false)
    : S(s), x(xx), P(p), Tb(tables()), bset(brenner_set == 2 ? 1 : 0)
  {
    nb.resize(S.n);
    ljl.resize(S.n);
    double rl = 0.0;
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) rl = std::max(rl, P.RL[a][b][1]);
    const double range2 = (1.44 * rl) * (1.44 * rl);
    for (int i = 0; i < S.n; i++)
      for (int j = 0; j < S.n; j++) {
        if (i == j) continue;
        double dd[3] = {val(x[i].x) - val(x[j].x), val(x[i].y) - val(x[j].y), val(x[i].z) - val(x[j].z)};
        for (int a = 0; a < 3; a++)
          if (S.pbc[a] && std::fabs(dd[a]) > S.L[a] * 0.5) dd[a] += dd[a] > 0 ? -S.L[a] : S.L[a];
        double r2 = dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2];
        double R2 = P.R[S.t[i]][S.t[j]][1];
        if (r2 <= R2 * R2) nb[i].push_back(j);
        if (with_lj && j > i && r2 < range2) ljl[i].push_back(j);
      }
    br.resize(S.n);
    bf.resize(S.n);
    Nt_.assign(S.n, T(0.0));
    NH_.assign(S.n, T(0.0));
    NC_.assign(S.n, T(0.0));
    for (int i = 0; i < S.n; i++)
      for (int j : nb[i]) {
        V3<T> v = d(i, j);
        T rr = sqrt(dot(v, v));
        T ff = fc(rr, P.R[S.t[i]][S.t[j]][0], P.R[S.t[i]][S.t[j]][1]);
        br[i].push_back(rr);
        bf[i].push_back(ff);
        Nt_[i] += ff;
        if (S.t[j] == 1) NH_[i] += ff;
        else NC_[i] += ff;
      }
  }

  int slot(int i, int j) const
  {
    for (size_t q = 0; q < nb[i].size(); q++)
      if (nb[i][q] == j) return (int)q;
    return -1;
  }

  // minimum image x_i - x_j (Atom.hpp:116-140, atoms wrapped into the box)
  V3<T> d(int i, int j) const
  {
    V3<T> r = sub(x[i], x[j]);
    T* c[3] = {&r.x, &r.y, &r.z};
    for (int a = 0; a < 3; a++)
      if (S.pbc[a] && std::fabs(val(*c[a])) > S.L[a] * 0.5) *c[a] = *c[a] + (val(*c[a]) > 0 ? -S.L[a] : S.L[a]);
    return r;
  }
  T r(int i, int j) const
  {
    int q = slot(i, j);
    if (q >= 0) return br[i][q];
    V3<T> v = d(i, j);
    return sqrt(dot(v, v));
  }

  // cosine cutoff (AtomsPair.hpp:148-157)
  static T fc(const T& rr, double R1, double R2)
  {
    if (val(rr) < R1) return T(1.0);
    if (val(rr) < R2) return (1.0 + cos(kPi * (rr - R1) / (R2 - R1))) / 2.0;
    return T(0.0);
  }
  T f(int i, int j) const
  {
    int q = slot(i, j);
    if (q >= 0) return bf[i][q];
    return fc(r(i, j), P.R[S.t[i]][S.t[j]][0], P.R[S.t[i]][S.t[j]][1]);
  }
  static T Sp(const T& a, double lo, double hi)
  {
    if (val(a) < lo) return T(1.0);
    if (val(a) > hi) return T(0.0);
    return (1.0 + cos(kPi * (a - lo) / (hi - lo))) / 2.0;
  }

  // coordination of i over its bonds except o, of a neighbour class: the
  // cached sum minus f_io (REBO::Nt/NH/NC, REBO.cxx:423-502)
  T N(int i, int o, int which) const
  {
    T s = which == 0 ? Nt_[i] : (which == 1 ? NH_[i] : NC_[i]);
    int q = slot(i, o);
    bool cls = which == 0 || (which == 1 && S.t[o] == 1) || (which == 2 && S.t[o] == 0);
    if (q >= 0 && cls) s = s - bf[i][q];
    if (val(s) < 0) s = T(0.0);
    return s;
  }
  // the Brenner form: a fresh sum over the other neighbours (Brenner.cxx:259-315)
  T Nloop(int i, int o, int which) const
  {
    T s = 0.0;
    for (size_t q = 0; q < nb[i].size(); q++) {
      int k = nb[i][q];
      if (k == o) continue;
      if (which == 1 && S.t[k] != 1) continue;
      if (which == 2 && S.t[k] != 0) continue;
      s += bf[i][q];
    }
    return s;
  }

  // ---- REBO splines ----
  T G(const double kn[][4], int npts, const T& c) const
  {
    int p = 0;
    for (p = 0; p < npts - 1; p++)
      if (val(c) <= kn[p + 1][0]) break;
    if (p >= npts - 1) p = npts - 2;
    double v[2] = {kn[p][1], kn[p + 1][1]}, d1[2] = {kn[p][2], kn[p + 1][2]}, d2[2] = {kn[p][3], kn[p + 1][3]};
    return quintic(c, kn[p][0], kn[p + 1][0], v, d1, d2, 0);
  }
  T Pspl(const double tab[5][5], const T& h, const T& c) const
  {
    if (val(h) >= 4 || val(c) >= 4) return T(0.0);
    return bicubic(h, c, (int)val(h), (int)val(c), &tab[0][0], nullptr, nullptr, 5);
  }
  T Fspl(int fam, const T& i, T j, T k) const
  {
    if (val(i) >= 4 || val(j) >= 4) return T(0.0);
    if (val(k) >= 15) return T(0.0);  // the k = 15 cells are empty (cubici.hpp:307)
    return tricubic(i, j, k, (int)val(i), (int)val(j), (int)val(k), &Tb.fv[fam][0][0][0], &Tb.fi[fam][0][0][0],
                    &Tb.fj[fam][0][0][0], &Tb.fk[fam][0][0][0], 5, 5, 16);
  }

  // ---- REBO b_ij (REBO.cxx:200-814); rij_alt = r used in H's exp term ----
  T p_sp(int i, int j, const T& rij_alt) const
  {
    const int ti = S.t[i], tj = S.t[j];
    T D = 1.0;
    V3<T> a = d(i, j);
    T rij = sqrt(dot(a, a));
    T Nij = N(i, j, 0);
    for (int k : nb[i]) {
      if (k == j) continue;
      const int tk = S.t[k];
      V3<T> b = d(i, k);
      T rik = sqrt(dot(b, b));
      T ex = 1.0;
      if (ti == 1) ex = exp(4.0 * ((P.rho[ti][tk] - rik) - (P.rho[ti][tj] - rij_alt)));
      T c = dot(a, b) / (rij * rik);
      if (val(c) < -1.0) c = T(-1.0);
      if (val(c) > 1.0) c = T(1.0);
      T g;
      if (ti == 0) {
        T s = Sp(Nij, 2.0, 3.0);
        T g1 = G(Tb.gc1, 5, c), g2 = G(Tb.gc2, 5, c);
        g = g2 + s * (g1 - g2);
      } else {
        g = G(Tb.gh, 4, c);
      }
      D = D + g * fc(rik, P.R[ti][tk][0], P.R[ti][tk][1]) * ex;
    }
    if (ti == 0) D = D + Pspl(tj == 0 ? Tb.pcc : Tb.pch, N(i, j, 1), N(i, j, 2));
    return pow(D, -0.5);
  }
  T nconj(int i, int j) const
  {
    T s1 = 0.0, s2 = 0.0;
    for (int k : nb[i])
      if (k != j && S.t[k] == 0) s1 += f(i, k) * Sp(N(k, i, 0), 2.0, 3.0);
    for (int l : nb[j])
      if (l != i && S.t[l] == 0) s2 += f(j, l) * Sp(N(l, j, 0), 2.0, 3.0);
    return 1.0 + s1 * s1 + s2 * s2;
  }
  T bbar(int i, int j, const T& rij_alt) const
  {
    T val_ = (p_sp(i, j, rij_alt) + p_sp(j, i, rij_alt)) / 2.0;
    const int ti = S.t[i], tj = S.t[j];
    int ci = i, cj = j;
    if (ti == 1 && tj == 0) { ci = j; cj = i; }
    const int tci = S.t[ci], tcj = S.t[cj];
    const int fam = (tci == 0 && tcj == 0) ? 0 : ((tci == 0 && tcj == 1) ? 1 : 2);
    T Nti = N(ci, cj, 0), Ntj = N(cj, ci, 0), Nc = nconj(ci, cj);
    val_ = val_ + Fspl(fam, Nti, Ntj, Nc);
    if (ti == 0 && tj == 0) {
      T Tv = Fspl(3, Nti, Ntj, Nc);
      if (val(Tv) != 0.0) {
        T sum = 0.0;
        V3<T> a = d(i, j);
        T rij = sqrt(dot(a, a));
        for (int k : nb[i]) {
          if (k == j) continue;
          for (int l : nb[j]) {
            if (l == i || l == k) continue;
            V3<T> b = d(i, k), c = d(j, l);
            T rik = sqrt(dot(b, b)), rjl = sqrt(dot(c, c));
            V3<T> ab = cross(a, neg(b)), ac = cross(a, neg(c));
            if (val(sqrt(dot(ab, ab)) / (rij * rik)) < 0.1) continue;
            if (val(sqrt(dot(ac, ac)) / (rij * rjl)) < 0.1) continue;
            T fik = Sp(rik, P.Rp[0][S.t[k]][0], P.Rp[0][S.t[k]][1]);
            T fjl = Sp(rjl, P.Rp[0][S.t[l]][0], P.Rp[0][S.t[l]][1]);
            V3<T> u = cross(neg(a), b), w = cross(a, c);
            T e2 = sqrt(dot(u, u)) * sqrt(dot(w, w));
            T cd = val(e2) == 0.0 ? T(0.0) : dot(u, w) / e2;
            if (val(cd) < -1.0) cd = T(-1.0);
            if (val(cd) > 1.0) cd = T(1.0);
            sum += (1.0 - cd * cd) * fik * fjl;
          }
        }
        val_ = val_ + Tv * sum;
      }
    }
    return val_;
  }

  // ---- energies ----
  T rebo() const
  {
    T E = 0.0;
    for (int i = 0; i < S.n; i++)
      for (int j : nb[i]) {
        if (j < i) continue;
        const int ti = S.t[i], tj = S.t[j];
        T rr = r(i, j), ff = f(i, j);
        if (val(ff) == 0.0) continue;
        T vr = ff * (1.0 + P.Q[ti][tj] / rr) * P.A[ti][tj] * exp(-P.alpha[ti][tj] * rr);
        T va = T(0.0);
        for (int q = 0; q < 3; q++)
          if (P.B[q][ti][tj] != 0.0) va = va + P.B[q][ti][tj] * exp(-P.beta[q][ti][tj] * rr);
        va = -ff * va;
        E += vr;
        if (val(va) != 0.0) E += bbar(i, j, rr) * va;
      }
    return E;
  }

  // largest product of REBO cutoffs over paths of 1..3 bonds (AIREBO_LJ.cxx:289-367)
  double wmax(int i, int j) const
  {
    double w = 0.0;
    for (int k : nb[i]) {
      double f1 = val(f(i, k));
      if (k == j) w = std::max(w, f1);
      for (int m : nb[k]) {
        double f2 = val(f(k, m));
        if (m == j) w = std::max(w, f1 * f2);
        for (int t : nb[m])
          if (t == j) w = std::max(w, f1 * f2 * val(f(m, t)));
      }
    }
    return w;
  }
  // the same with the arg-max path's cutoffs as T (so derivatives flow)
  T wpath(int i, int j, double wv) const
  {
    if (wv == 0.0) return T(0.0);
    for (int k : nb[i]) {
      if (k == j && val(f(i, k)) == wv) return f(i, k);
    }
    for (int k : nb[i])
      for (int m : nb[k])
        if (m == j && val(f(i, k)) * val(f(k, m)) == wv) return f(i, k) * f(k, m);
    for (int k : nb[i])
      for (int m : nb[k])
        for (int t : nb[m])
          if (t == j && val(f(i, k)) * val(f(k, m)) * val(f(m, t)) == wv) return f(i, k) * f(k, m) * f(m, t);
    return T(wv);
  }
  static T Slj(const T& a, double lo, double hi)
  {
    if (val(a) < lo) return T(1.0);
    if (val(a) > hi) return T(0.0);
    T t = (a - lo) / (hi - lo);
    return 1.0 - t * t * (3.0 - 2.0 * t);
  }
  T lj() const
  {
    T E = 0.0;
    for (int i = 0; i < S.n; i++)
      for (int j : ljl[i]) {
        const int ti = S.t[i], tj = S.t[j];
        V3<T> a = d(i, j);
        double r2 = val(dot(a, a));
        if (r2 > P.RL[ti][tj][1] * P.RL[ti][tj][1]) continue;
        double wv = wmax(i, j);
        T C = 1.0 - wpath(i, j, wv);
        if (!(val(C) > 0.0)) continue;
        T rr = sqrt(dot(a, a));
        T fl = fc(rr, P.RL[ti][tj][0], P.RL[ti][tj][1]);
        if (val(fl) == 0.0) continue;
        T Str = Slj(rr, P.RLJ[ti][tj][0], P.RLJ[ti][tj][1]);
        T SrSb = 1.0;
        if (val(Str) != 0.0) {
          tally_bucket() = 1;
          T b = bbar(i, j, T(P.R[ti][tj][0]));
          tally_bucket() = 0;
          SrSb = 1.0 - Str + Str * Slj(b, P.bw[ti][tj][0], P.bw[ti][tj][1]);
        }
        T s6 = pow(P.sigma[ti][tj] / rr, 6.0);
        E += SrSb * C * fl * 4.0 * P.eps[ti][tj] * (s6 * s6 - s6);
      }
    return E;
  }
  T tors() const
  {
    T E = 0.0;
    for (int i = 0; i < S.n; i++)
      for (int j : nb[i]) {
        if (j < i || S.t[i] != 0 || S.t[j] != 0) continue;
        V3<T> a = d(i, j);
        T rij = sqrt(dot(a, a));
        T wij = f(i, j);
        for (int k : nb[i]) {
          if (k == j) continue;
          for (int l : nb[j]) {
            if (l == i || l == k) continue;
            V3<T> b = d(i, k), c = d(j, l);
            T rik = sqrt(dot(b, b)), rjl = sqrt(dot(c, c));
            V3<T> ab = cross(a, neg(b)), ac = cross(a, c);
            if (val(sqrt(dot(ab, ab)) / (rij * rik)) < 0.1) continue;
            if (val(sqrt(dot(ac, ac)) / (rij * rjl)) < 0.1) continue;
            V3<T> u = cross(neg(a), b), w = cross(a, c);
            T e2 = sqrt(dot(u, u)) * sqrt(dot(w, w));
            T cd = val(e2) == 0.0 ? T(0.0) : dot(u, w) / e2;
            if (val(cd) < -1.0) cd = T(-1.0);
            if (val(cd) > 1.0) cd = T(1.0);
            const double ep = P.teps[S.t[k]][S.t[l]];
            T v = (256.0 / 405.0) * ep * pow(0.5 * (1.0 - cd), 5.0) - 0.1 * ep;
            E += f(i, k) * wij * f(j, l) * v;
          }
        }
      }
    return E;
  }

  // ---- Brenner (Brenner.cxx:31-472) ----
  T Hspl(int fam, const T& h, const T& c) const
  {
    if (val(h) >= 4 || val(c) >= 4) return T(0.0);
    const double* F = fam == 0 ? &Tb.hcc[bset][0][0] : &Tb.hch[bset][0][0];
    const double* FX = fam == 0 ? nullptr : &Tb.hchdh[bset][0][0];
    const double* FY = fam == 0 ? nullptr : &Tb.hchdc[bset][0][0];
    return bicubic(h, c, (int)val(h), (int)val(c), F, FX, FY, 5);
  }
  T bF(const T& i, const T& j, T k) const
  {
    if (val(i) >= 4 || val(j) >= 4) return T(0.0);
    int kk = (int)val(k);
    if (val(k) > 4) kk = 4;  // cubici.hpp:134-177: k clamped to 4, cell [.][.][4]
    T kc = val(k) > 4 ? T(4.0) : k;
    return tricubic(i, j, kc, (int)val(i), (int)val(j), kk, &Tb.bf[bset][0][0][0], &Tb.bfi[bset][0][0][0],
                    &Tb.bfj[bset][0][0][0], nullptr, 5, 5, 6);
  }
  T bB(int i, int j) const
  {
    const int ti = S.t[i], tj = S.t[j];
    T D = 1.0;
    V3<T> a = d(i, j);
    T rij = sqrt(dot(a, a));
    for (int k : nb[i]) {
      if (k == j) continue;
      const int tk = S.t[k];
      V3<T> b = d(i, k);
      T rik = sqrt(dot(b, b));
      const double al = P.balpha[bset][ti][tj][tk];
      T ex = 1.0;
      if (al != 0.0) ex = exp(al * ((rij - P.bRe[bset][ti][tj]) - (rik - P.bRe[bset][ti][tk])));
      T g;
      if (ti == 0) {
        T c = dot(a, b) / (rij * rik);
        if (val(c) < -1.0) c = T(-1.0);
        if (val(c) > 1.0) c = T(1.0);
        const double ao = P.bao[bset], co = P.bco[bset], d0 = P.bdo[bset];
        g = ao * (1.0 + co * co / (d0 * d0) - co * co / (d0 * d0 + (1.0 + c) * (1.0 + c)));
      } else {
        g = T(P.bGHH[bset]);
      }
      D = D + g * f(i, k) * ex;
    }
    if (ti == 0) D = D + Hspl(tj == 0 ? 0 : 1, Nloop(i, j, 1), Nloop(i, j, 2));
    return pow(D, -P.bdelta[bset][ti][ti]);
  }
  T bFN(int i, int j) const
  {
    if (S.t[i] != 0 || S.t[j] != 0) return T(0.0);
    T Nc = 1.0;
    for (int k : nb[i])
      if (k != j && S.t[k] == 0) {
        T xk = Nloop(k, i, 0);
        T Fx = val(xk) <= 2.0 ? T(1.0) : (val(xk) >= 3.0 ? T(0.0) : (1.0 + cos(kPi * (xk - 2.0))) / 2.0);
        Nc = Nc + f(i, k) * Fx;
      }
    for (int l : nb[j])
      if (l != i && S.t[l] == 0) {
        T xl = Nloop(l, j, 0);
        T Fx = val(xl) <= 2.0 ? T(1.0) : (val(xl) >= 3.0 ? T(0.0) : (1.0 + cos(kPi * (xl - 2.0))) / 2.0);
        Nc = Nc + f(j, l) * Fx;
      }
    return bF(Nloop(i, j, 0), Nloop(j, i, 0), Nc);
  }
  T brenner() const
  {
    T E = 0.0;
    for (int i = 0; i < S.n; i++)
      for (int j : nb[i]) {
        if (j < i) continue;
        const int ti = S.t[i], tj = S.t[j];
        T rr = r(i, j), ff = f(i, j);
        if (val(ff) == 0.0) continue;
        const double De = P.bDe[bset][ti][tj], Sv = P.bS[bset][ti][tj], be = P.bbeta[bset][ti][tj],
                     Re = P.bRe[bset][ti][tj];
        T vr = ff * (De / (Sv - 1.0)) * exp(-(std::sqrt(2.0 * Sv) * be) * (rr - Re));
        T va = ff * (De * Sv / (Sv - 1.0)) * exp(-(std::sqrt(2.0 / Sv) * be) * (rr - Re));
        T bb = (bB(i, j) + bB(j, i)) / 2.0 + bFN(i, j) / 2.0;
        E += vr - bb * va;
      }
    return E;
  }
};

}  // namespace rs

// ------------------------------------------------------------ C ABI
using namespace rs;

namespace {

System make_system(int n, const int* z, const double* box, const int* pbc)
{
  System s;
  s.n = n;
  s.t.resize(n);
  for (int i = 0; i < n; i++) s.t[i] = (z[i] == 6) ? 0 : 1;
  for (int a = 0; a < 3; a++) { s.L[a] = box[a]; s.pbc[a] = pbc[a]; }
  return s;
}

// wrapped positions (Atom::applyPBC), as the reference sees them
std::vector<double> wrapped(int n, const double* pos, const System& s)
{
  std::vector<double> p(pos, pos + 3 * n);
  for (int i = 0; i < n; i++)
    for (int a = 0; a < 3; a++)
      if (s.pbc[a]) {
        double& x = p[3 * i + a];
        while (x < 0) x += s.L[a];
        while (x >= s.L[a]) x -= s.L[a];
      }
  return p;
}

template <class T>
void terms(const Eval<T>& E, int potset, T out[4])
{
  out[0] = out[1] = out[2] = out[3] = T(0.0);
  if (potset & 1) out[0] = E.rebo();
  if (potset & 2) out[1] = E.lj();
  if (potset & 4) out[2] = E.tors();
  if (potset & 8) out[3] = E.brenner();
}

}  // namespace

extern "C" {

/* Energies (eV) of each selected term: out[0] REBO, [1] AIREBO LJ, [2] torsion,
 * [3] Brenner.  potset bits as the oracle: 1 REBO, 2 LJ, 4 torsion, 8 Brenner. */
int rs_energy(int potset, int brenner_set, int lj_cut_mode, int n, const int* z, const double* pos,
              const double* box, const int* pbc, double* out)
{
  System s = make_system(n, z, box, pbc);
  std::vector<double> p = wrapped(n, pos, s);
  std::vector<V3<double>> x(n);
  for (int i = 0; i < n; i++) x[i] = {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
  Params P(lj_cut_mode);
  Eval<double> E(s, x, P, brenner_set, (potset & 2) != 0);
  terms(E, potset, out);
  return 0;
}

/* Directional derivatives dE/de (eV per unit of the direction e, [n*3]) of
 * each term, by forward-mode dual numbers: out[4] as in rs_energy. */
int rs_energy_dir(int potset, int brenner_set, int lj_cut_mode, int n, const int* z, const double* pos,
                  const double* dir, const double* box, const int* pbc, double* out)
{
  System s = make_system(n, z, box, pbc);
  std::vector<double> p = wrapped(n, pos, s);
  typedef Dual<1> D1;
  std::vector<V3<D1>> x(n);
  for (int i = 0; i < n; i++) {
    D1 a(p[3 * i]), b(p[3 * i + 1]), c(p[3 * i + 2]);
    a.d[0] = dir[3 * i];
    b.d[0] = dir[3 * i + 1];
    c.d[0] = dir[3 * i + 2];
    x[i] = {a, b, c};
  }
  Params P(lj_cut_mode);
  Eval<D1> E(s, x, P, brenner_set, (potset & 2) != 0);
  D1 t[4];
  terms(E, potset, t);
  for (int q = 0; q < 4; q++) out[q] = t[q].d[0];
  return 0;
}

/* Operation counts of one energy evaluation of the selected terms:
 * out[0..7] = add/sub, mul, div, sqrt, exp, cos, pow, (unused) over the whole
 * evaluation; out[8..15] the same for the part spent in the LJ term's b*_ij. */
int rs_opcount(int potset, int brenner_set, int n, const int* z, const double* pos, const double* box,
               const int* pbc, long* out)
{
  System s = make_system(n, z, box, pbc);
  std::vector<double> p = wrapped(n, pos, s);
  std::vector<V3<Counted>> x(n);
  for (int i = 0; i < n; i++) x[i] = {Counted(p[3 * i]), Counted(p[3 * i + 1]), Counted(p[3 * i + 2])};
  Params P(0);
  for (int b = 1; b >= 0; b--) { tally_bucket() = b; tally() = OpTally(); }
  Eval<Counted> E(s, x, P, brenner_set, (potset & 2) != 0);
  Counted t[4];
  terms(E, potset, t);
  for (int b = 0; b < 2; b++) {
    tally_bucket() = 1;
    const OpTally c1 = tally();
    tally_bucket() = 0;
    const OpTally c = b == 0 ? tally() : c1;
    long* o = out + 8 * b;
    o[0] = c.add + (b == 0 ? c1.add : 0); o[1] = c.mul + (b == 0 ? c1.mul : 0);
    o[2] = c.div + (b == 0 ? c1.div : 0); o[3] = c.sqrt_ + (b == 0 ? c1.sqrt_ : 0);
    o[4] = c.exp_ + (b == 0 ? c1.exp_ : 0); o[5] = c.cos_ + (b == 0 ? c1.cos_ : 0);
    o[6] = c.pow_ + (b == 0 ? c1.pow_ : 0); o[7] = 0;
  }
  return 0;
}

}  // extern "C"
