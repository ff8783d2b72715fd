// Metal and ion potentials of the applications' potential set
// (applications/common.h:36-77), beside REBO/AIREBO:
//
// * FBZL (pairwise/FBZL.cxx:34-129): ZBL repulsion of the noble-gas ions
//   (Ar, Xe) with every element, cosine switch 5.0-5.5 A;
// * FLJ (pairwise/FLJ.cxx:34-343): hydrocarbon (H, C) - metal (Cu, Au)
//   pairs, ZBL below 1.2 A, a cubic joining it to Lennard-Jones on
//   [1.2, 1.9) A, Lennard-Jones (Lorentz-Berthelot mixing) with the cosine
//   switch 5.0-5.5 A beyond;
// * Ackland (manybody/Ackland/Ackland.cxx:30-457): the embedded-atom model of
//   Cu, Ag, Au: pair term (ZBL below 1.0 A, a cubic on [1.0, 1.4) A, knot
//   cubics beyond), density g (knot cubics, geometric mean between unlike
//   metals) and embedding F = -sqrt(rho).
//
// Every function works in the reference's CGS units and expressions; the
// kernels convert the results to eV and eV/Angstrom.  Hydrocarbon-silver
// pairs have no interaction (no potential handles them), as in the reference.
#pragma once

namespace mdg {

// species indices beyond kC = 0, kH = 1
constexpr int kCu = 2, kAg = 3, kAu = 4, kAr = 5, kXe = 6, kNSpec = 7;
constexpr double kECgs = 4.8e-10;  // elementary charge (consts.cxx:29)

MDG_HD bool spec_ch(int t) { return t <= 1; }
MDG_HD bool spec_metal(int t) { return t >= kCu && t <= kAu; }
MDG_HD bool spec_ion(int t) { return t >= kAr; }

struct MetalParams {
  double Z[kNSpec];                  // Atom::Z (esu), Atom.hpp:100-115
  double R0, R1;                     // FBZL / FLJ switch (cm)
  double sig[kNSpec][kNSpec];        // FLJ sigma (cm)
  double eps[kNSpec][kNSpec];        // FLJ epsilon (erg)
  double flj_x[2];                   // FLJ joining cubic interval (cm)
  double flj_v[kNSpec][kNSpec][4];   // its end values and slopes: v0, dv0, v1, dv1
  double rk[3][3][7], ak[3][3][7];   // Ackland pair knots (cm) and coefficients (erg/cm^3)
  double Rk[3][3][3], Ak[3][3][3];   // Ackland density knots and coefficients
  double ack_x[2];                   // Ackland joining cubic interval (cm)
  double ack_v[3][3][4];
  double rcut;                       // largest range of the three (cm)
};

// Ziegler-Biersack-Littmark universal screened Coulomb repulsion with the
// reference's screening length 0.88534 a0 / (ZA^0.23 + ZB^0.23), a0 =
// 0.53e-8 cm; value (erg) and d/dr (erg/cm).
MDG_HD double zbl(double ZA, double ZB, double r, double& der)
{
  const double AS = 8.8534e-1 * 0.53e-8 / (pow(ZA / kECgs, 0.23) + pow(ZB / kECgs, 0.23));
  const double Y = r / AS;
  const double e1 = exp(-3.1998 * Y), e2 = exp(-0.94229 * Y), e3 = exp(-0.4029 * Y), e4 = exp(-0.20162 * Y);
  const double s = 0.18175 * e1 + 0.50986 * e2 + 0.28022 * e3 + 0.02817 * e4;
  const double ds = 0.18175 * 3.1998 * e1 + 0.50986 * 0.94229 * e2 + 0.28022 * 0.4029 * e3 + 0.02817 * 0.20162 * e4;
  der = -ZA * ZB / (r * r) * s - ZA * ZB / (r * AS) * ds;
  return ZA * ZB / r * s;
}

// The cubic through (x0, v0, dv0) and (x1, v1, dv1) (mdtk/Spline.cxx: the
// same cubic, here in Hermite form).
MDG_HD double join_cubic(const double* x, const double* v, double r, double& der)
{
  const double h = x[1] - x[0], t = (r - x[0]) / h, t2 = t * t, t3 = t2 * t;
  der = (6.0 * t2 - 6.0 * t) / h * v[0] + (3.0 * t2 - 4.0 * t + 1.0) * v[1] + (6.0 * t - 6.0 * t2) / h * v[2] +
        (3.0 * t2 - 2.0 * t) * v[3];
  return (2.0 * t3 - 3.0 * t2 + 1.0) * v[0] + (t3 - 2.0 * t2 + t) * h * v[1] + (3.0 * t2 - 2.0 * t3) * v[2] +
         (t3 - t2) * h * v[3];
}

// FLJ's Lennard-Jones (FLJ::VLJ, FLJ.cxx:299-320) without the switch.
MDG_HD double flj_lj(const MetalParams& M, int a, int b, double r, double& der)
{
  const double s = M.sig[a][b] / r;
  double s6 = s;
  for (int k = 2; k <= 6; k++) s6 *= s;
  const double s12 = s6 * s6;
  der = 4.0 * M.eps[a][b] * (-12.0 * s12 / r + 6.0 * s6 / r);
  return 4.0 * M.eps[a][b] * (s12 - s6);
}

// Ackland's knot cubics of the pair term (Ackland::Phi beyond the joining
// cubic, Ackland.cxx:100-115).
MDG_HD double ack_knots(const MetalParams& M, int a, int b, bool same, double r, double& der)
{
  const int nk = same ? 6 : 3;
  double val = 0.0;
  der = 0.0;
  for (int k = 1; k <= nk; k++) {
    const double rt = M.rk[a][b][k] - r;
    if (rt <= 0) continue;
    val += M.ak[a][b][k] * rt * rt * rt;
    der += M.ak[a][b][k] * 3.0 * rt * rt * (-1.0);
  }
  return val;
}

// Ackland::PhiCap / dPhiCap (Ackland.cxx:120-160)
MDG_HD double ack_phicap(const MetalParams& M, int a, int b, double r, double& der)
{
  der = 0.0;
  if (r >= M.Rk[a][b][1]) return 0.0;
  double val = 0.0;
  for (int k = 1; k <= 2; k++) {
    const double rt = M.Rk[a][b][k] - r;
    if (rt <= 0) continue;
    val += M.Ak[a][b][k] * rt * rt * rt;
    der += M.Ak[a][b][k] * 3.0 * rt * rt * (-1.0);
  }
  return val;
}

// Ackland::g: the density one metal atom gives another (Ackland.cxx:162-206)
MDG_HD double ack_g(const MetalParams& M, int a, int b, double r, double& der)
{
  if (a != b) {
    double d1, d2;
    const double p1 = ack_phicap(M, a, a, r, d1), p2 = ack_phicap(M, b, b, r, d2);
    const double sq = sqrt(p1 * p2);
    der = (r < M.Rk[a][a][1] && r < M.Rk[b][b][1]) ? 0.5 / sq * (d1 * p2 + p1 * d2) : 0.0;
    return sq;
  }
  return ack_phicap(M, a, a, r, der);
}

// Ackland::Phi (Ackland.cxx:57-118)
MDG_HD double ack_phi(const MetalParams& M, int a, int b, double ZA, double ZB, double r, double& der)
{
  der = 0.0;
  if (r >= M.rk[a][b][1]) return 0.0;
  if (r < M.ack_x[0]) return zbl(ZA, ZB, r, der);
  if (r < M.ack_x[1]) return join_cubic(M.ack_x, M.ack_v[a][b], r, der);
  return ack_knots(M, a, b, a == b, r, der);
}

// Energy (erg) and d/dr (erg/cm) of the pair term between species ti and tj
// at r (cm), the embedding excluded; kind of pair by the handled element
// pairs of the three potentials.
MDG_HD double metal_pair(const MetalParams& M, int ti, int tj, double r, double& der)
{
  der = 0.0;
  if (spec_ion(ti) || spec_ion(tj)) {  // FBZL::operator(), FBZL.cxx:105-127
    if (r > M.R1) return 0.0;
    double f, df, d;
    cutoff(r, M.R0, M.R1, f, df);
    const double v = zbl(M.Z[ti], M.Z[tj], r, d);
    der = d * f + v * df;
    return v * f;
  }
  const bool flj = (spec_ch(ti) && (tj == kCu || tj == kAu)) || (spec_ch(tj) && (ti == kCu || ti == kAu));
  if (flj) {  // FLJ::operator() and FLJ::VLJ, FLJ.cxx:250-343
    if (r > M.R1) return 0.0;
    if (r < M.flj_x[0]) return zbl(M.Z[ti], M.Z[tj], r, der);
    if (r < M.flj_x[1]) return join_cubic(M.flj_x, M.flj_v[ti][tj], r, der);
    double f, df, d;
    cutoff(r, M.R0, M.R1, f, df);
    const double v = flj_lj(M, ti, tj, r, d);
    der = d * f + v * df;
    return f * v;
  }
  if (spec_metal(ti) && spec_metal(tj))
    return ack_phi(M, ti - kCu, tj - kCu, M.Z[ti], M.Z[tj], r, der);
  return 0.0;
}

}  // namespace mdg

namespace mdg {

// The three potentials' parameters as their constructors set them (CGS):
// FLJ.cxx:115-160 (Lorentz-Berthelot set; the disabled set at 61-113 is not
// used), Ackland.cxx:265-385; the joining cubics' end conditions as
// FLJ::fillR_concat_ (FLJ.cxx:171-250) and Ackland::fillR_concat_
// (Ackland.cxx:387-457) take them.
inline void make_metal_params(MetalParams& M)
{
  std::memset(&M, 0, sizeof(M));
  const double Ao = 1e-8, eV = 1.6021E-012, kb = 8.617343E-5 * eV, K = 1.0;
  const double e = kECgs;
  const double zz[kNSpec] = {6.0, 1.0, 29.0, 47.0, 79.0, 18.0, 54.0};
  for (int t = 0; t < kNSpec; t++) M.Z[t] = zz[t] * e;
  M.R0 = 5.0 * Ao;
  M.R1 = 5.5 * Ao;
  M.rcut = M.R1;
  // FLJ
  M.sig[kCu][kCu] = 3.05 * Ao;
  M.eps[kCu][kCu] = 0.165565 * eV;
  M.sig[kC][kC] = 3.4 * Ao;
  M.eps[kC][kC] = 0.002413 * eV;
  M.sig[kAu][kAu] = 2.569 * Ao;
  M.eps[kAu][kAu] = 0.408 * eV;
  M.sig[kH][kH] = 2.81 * Ao;
  M.eps[kH][kH] = 8.6 * K * kb;
  for (int m : {kCu, kAu})
    for (int h : {kC, kH}) {
      M.sig[m][h] = M.sig[h][m] = (M.sig[m][m] + M.sig[h][h]) / 2;
      M.eps[m][h] = M.eps[h][m] = std::sqrt(M.eps[m][m] * M.eps[h][h]);
    }
  M.flj_x[0] = 1.2 * Ao;
  M.flj_x[1] = 1.9 * Ao;
  for (int m : {kCu, kAu})
    for (int h : {kC, kH})
      for (int o = 0; o < 2; o++) {
        const int a = o ? m : h, b = o ? h : m;
        double* v = M.flj_v[a][b];
        v[0] = zbl(M.Z[a], M.Z[b], M.flj_x[0], v[1]);
        v[2] = flj_lj(M, a, b, M.flj_x[1], v[3]);
      }
  // Ackland (indexes Cu 0, Ag 1, Au 2)
  const int Cu = 0, Ag = 1, Au = 2;
  auto mixed = [&](int x, int y, double r1, double r2, double r3, double a1, double a2, double a3) {
    M.rk[x][y][1] = M.rk[y][x][1] = r1 * Ao;
    M.rk[x][y][2] = M.rk[y][x][2] = r2 * Ao;
    M.rk[x][y][3] = M.rk[y][x][3] = r3 * Ao;
    M.ak[x][y][1] = M.ak[y][x][1] = a1 * eV / (Ao * Ao * Ao);
    M.ak[x][y][2] = M.ak[y][x][2] = a2 * eV / (Ao * Ao * Ao);
    M.ak[x][y][3] = M.ak[y][x][3] = a3 * eV / (Ao * Ao * Ao);
  };
  mixed(Ag, Au, 4.40856, 3.46970, 3.00000, 0.003566503525, 1.015075326, 0.00000000);
  mixed(Cu, Au, 4.309816, 4.047479, 3.297946, -0.08554551660, 0.192835880, 0.75932286);
  mixed(Ag, Cu, 4.15800, 3.15700, 3.00000, 0.03533037752, 0.8518466353, 0.0000000000);
  auto same = [&](int x, double a, const double* akv, const double* Akv, const double* rkv, const double* Rkv) {
    for (int k = 1; k <= 6; k++) {
      M.ak[x][x][k] = akv[k - 1] * eV / (a * a * a);
      M.rk[x][x][k] = rkv[k - 1] * a;
    }
    for (int k = 1; k <= 2; k++) {
      M.Ak[x][x][k] = Akv[k - 1] * (eV * eV) / (a * a * a);
      M.Rk[x][x][k] = Rkv[k - 1] * a;
    }
  };
  {
    const double akv[6] = {61.73525861, -108.18467800, 57.00053948, -12.88796578, 39.16381901, 0.00000000};
    const double Akv[2] = {10.03718305, 17.06363299};
    const double rkv[6] = {1.225, 1.202, 1.154, 1.050, 0.866, 0.707};
    const double Rkv[2] = {1.225, 0.990};
    same(Cu, 3.615 * Ao, akv, Akv, rkv, Rkv);
  }
  {
    const double akv[6] = {20.368404, -102.36075, 94.31277, -6.220051, 31.080889, 175.56047};
    const double Akv[2] = {1.458761, 42.946555};
    const double rkv[6] = {1.2247449, 1.1547054, 1.1180065, 1.0000000, 0.8660254, 0.7071068};
    const double Rkv[2] = {1.2247449, 1.0000000};
    same(Ag, 4.086 * Ao, akv, Akv, rkv, Rkv);
  }
  {
    const double akv[6] = {29.059066, -153.14779, 148.17881, -22.20508, 72.71465, 199.26269};
    const double Akv[2] = {21.930125, 284.99631};
    const double rkv[6] = {1.2247449, 1.1547054, 1.1180065, 1.0000000, 0.8660254, 0.7071068};
    const double Rkv[2] = {1.1180065, 0.8660254};
    same(Au, 4.078 * Ao, akv, Akv, rkv, Rkv);
  }
  M.ack_x[0] = 1.0 * Ao;
  M.ack_x[1] = 1.4 * Ao;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double* v = M.ack_v[a][b];
      v[0] = zbl(M.Z[kCu + a], M.Z[kCu + b], M.ack_x[0], v[1]);
      v[2] = ack_knots(M, a, b, a == b, M.ack_x[1], v[3]);
    }
}

MDG_HD double warp_sum(double x)
{
#if defined(__CUDA_ARCH__)
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
#endif
  return x;
}

// The partners of atom i within the potentials' range, handed to the lanes
// 32 at a time: each lane tests one list entry, a ballot packs the ones in
// range into a per-warp queue in list order, and every full queue is
// processed with all lanes busy (two thirds of a Verlet list lie in its
// skin).  f(j, lane) is called once per queued partner; deterministic.
template <class F>
__device__ void for_partners(const State& S, const NList& L, int i, const V3& xi, const Box& box, double rcut_A,
                             bool metal_only, int* wq, F&& f)
{
  const int lane = threadIdx.x & 31;
  const int* nl = L.list + (long)i * L.cap;
  const int nn = L.cnt[i];
  int cnt = 0;  // queued, the same in every lane
  for (int base = 0; base < nn; base += 32) {
    const int q = base + lane;
    bool keep = false;
    int j = -1;
    if (q < nn) {
      j = nl[q];
      const double4 pj = S.pos[j];
      if (!metal_only || spec_metal((int)pj.w)) keep = norm2(depos(box, xi, v3(pj.x, pj.y, pj.z))) < rcut_A * rcut_A;
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    const int pos = cnt + __popc(m & ((1u << lane) - 1u));
    if (keep && pos < 32) wq[pos] = j;
    const int total = cnt + __popc(m);
    __syncwarp();
    if (total >= 32) {
      f(wq[lane]);
      __syncwarp();
      if (keep && pos >= 32) wq[pos - 32] = j;
      __syncwarp();
      cnt = total - 32;
    } else {
      cnt = total;
    }
  }
  if (lane < cnt) f(wq[lane]);
  __syncwarp();
}

// Embedding of each metal atom (Ackland::F and rho, Ackland.cxx:208-232):
// rho_i = sum of g over its metal partners, F_i = -sqrt(rho_i),
// fp_i = dF/drho = 0.5 / F_i (0 when rho_i = 0); em gets F_i in eV.  One
// warp per atom, a fixed butterfly for the sum.
__global__ void k_eam_rho(State S, NList L, const MetalParams* __restrict__ Mp, double* fp, double* em,
                          unsigned int* status)
{
  pdl_enter();
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= S.n) return;  // uniform per warp
  const double4 pi = S.pos[i];
  const int ti = (int)pi.w;
  if (!spec_metal(ti)) {
    if (lane == 0) {
      fp[i] = 0.0;
      em[i] = 0.0;
    }
    return;
  }
  const MetalParams& M = *Mp;
  const Box& box = box_of(S, i);
  const V3 xi = v3(pi.x, pi.y, pi.z);
  // (the density terms are cheap: the lanes take the list entries in turn;
  // queueing the partners in range, as the pair kernel does, cost more here)
  const int* nl = L.list + (long)i * L.cap;
  const int nn = L.cnt[i];
  double rho = 0.0;
  for (int q = lane; q < nn; q += 32) {
    const double4 pj = S.pos[nl[q]];
    const int tj = (int)pj.w;
    if (!spec_metal(tj)) continue;
    const double r = sqrt(norm2(depos(box, xi, v3(pj.x, pj.y, pj.z)))) * kAo;
    double d;
    rho += ack_g(M, ti - kCu, tj - kCu, r, d);
  }
  rho = warp_sum(rho);
  if (lane != 0) return;
  if (!(rho >= 0.0)) atomicOr(status, ST_NONFINITE);
  const double F = -sqrt(rho);
  fp[i] = rho != 0.0 ? 0.5 / F : 0.0;
  em[i] = F / kEv;
}

// Pair terms of every metal or ion pair of atom i (half of each pair's
// energy to each end) plus the embedding's pair derivative
// (fp_i + fp_j) dg/dr for metal pairs: gradient gm (eV/A) and energy em (eV)
// of atom i.  One warp per atom over the partners in range, a fixed
// butterfly for the sums (deterministic, no atomics).
__global__ void k_metal_pairs(State S, NList L, const MetalParams* __restrict__ Mp, const double* fp, double* em,
                              double4* gm)
{
  pdl_enter();
  __shared__ int qbuf[kThreads];
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= S.n) return;  // uniform per warp
  const MetalParams& M = *Mp;
  const double4 pi = S.pos[i];
  const int ti = (int)pi.w;
  const Box& box = box_of(S, i);
  const V3 xi = v3(pi.x, pi.y, pi.z);
  const double fpi = fp[i];
  double e = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
  for_partners(S, L, i, xi, box, M.rcut / kAo, false, qbuf + (threadIdx.x & ~31), [&](int j) {
    const double4 pj = S.pos[j];
    const int tj = (int)pj.w;
    const V3 d = depos(box, xi, v3(pj.x, pj.y, pj.z));
    const double rA = sqrt(norm2(d));
    const double r = rA * kAo;
    double der;
    const double v = metal_pair(M, ti, tj, r, der);
    if (spec_metal(ti) && spec_metal(tj)) {
      double dg;
      ack_g(M, ti - kCu, tj - kCu, r, dg);
      der += (fpi + fp[j]) * dg;
    }
    e += 0.5 * v;
    const double k = der * kAo / kEv / rA;  // d/dr in eV/A, along the unit vector
    gx += d.x * k;
    gy += d.y * k;
    gz += d.z * k;
  });
  e = warp_sum(e);
  gx = warp_sum(gx);
  gy = warp_sum(gy);
  gz = warp_sum(gz);
  if (lane != 0) return;
  em[i] = (spec_metal(ti) ? em[i] : 0.0) + e / kEv;
  gm[i] = make_double4(gx, gy, gz, 0.0);
}

}  // namespace mdg
