// Per-atom work items of one force evaluation and one velocity-Verlet step.
// Each function is the body of one thread of the matching kernel in
// mdg_api.cu; thread a only ever writes atom a's own outputs.
#pragma once

#include "mdg_common.cuh"
#include "mdg_rebo.cuh"
#include "mdg_etors.cuh"

namespace mdg {

// Verlet neighbour list (full lists, NeighbourList::Update semantics,
// mdtk/potentials/NeighbourList.cxx:73-106): partners of atom i at
// list[i * cap + s], s < cnt[i].
struct NList {
  int cap;
  int sorted;         // 1: ascending partner order (the reference's); 0: cell order (deterministic)
  int pairs;          // 0: every pair; 1: hydrocarbon pairs only (the REBO/AIREBO lists of a system
                      // with metal or ion atoms); 2: pairs with a metal or ion atom (their own list)
  int* cnt;
  int* list;
  double range2;      // ((1 + 0.44) * Rcutoff)^2
  double trigger;     // 0.44 * Rcutoff: rebuild when the two largest displacements exceed it
  double4* pos0;      // positions at the last build
};

// Cell grid of one list.  A batched context (many independent systems in
// one atom array) keeps one grid per system, laid out one after another:
// per-system dimensions, origin, cell size and first cell in snc/slo/scs.
struct Grid {
  int nc[3];
  double lo[3], cs[3];  // origin and cell size per axis
  int ncell;            // all systems together
  int brute;            // 1: O(N^2) scan (single system, a periodic axis has fewer than 3 cells)
  int* ccount;          // [ncell]
  int* cstart;          // [ncell + 1]
  int* ccursor;         // [ncell]
  int* catoms;          // [n]
  const int4* snc;      // [nsys] x, y, z = cells per axis, w = first cell (batched only)
  const double4* slo;   // [nsys] origin
  const double4* scs;   // [nsys] cell size
};

struct State {
  int n;
  Box box;              // the box of a single-system context
  const int* sys;       // [n] system of each atom in a batched context, else null
  const Box* boxes;     // [nsys] boxes of a batched context
  double4* pos;         // x, y, z, w = species index (0 C, 1 H)
  double4* vel;         // w unused
  double4* acc;         // an (Angstrom/fs^2)
  int4* image;          // PBC_count
  const unsigned char* fixed;
  double* mass;         // amu
};

// The periodic box atom a lives in.
// By value: a reference that may point at the kernel parameter S.box would
// make every thread copy the parameter to local memory.
MDG_HD Box box_of(const State& S, int a)
{
  Box b = S.box;  // loaded field by field: no pointer to the parameter is formed
  if (S.sys) b = S.boxes[S.sys[a]];
  return b;
}

// The cell grid of atom a's system.
struct GridView {
  int nc[3];
  double lo[3], cs[3];
  int base;
};
MDG_HD GridView grid_view(const Grid& g, const State& S, int a)
{
  GridView v;
  if (S.sys) {
    const int s = S.sys[a];
    const int4 n = g.snc[s];
    const double4 lo = g.slo[s], cs = g.scs[s];
    v.nc[0] = n.x; v.nc[1] = n.y; v.nc[2] = n.z;
    v.lo[0] = lo.x; v.lo[1] = lo.y; v.lo[2] = lo.z;
    v.cs[0] = cs.x; v.cs[1] = cs.y; v.cs[2] = cs.z;
    v.base = n.w;
  } else {
    for (int ax = 0; ax < 3; ax++) { v.nc[ax] = g.nc[ax]; v.lo[ax] = g.lo[ax]; v.cs[ax] = g.cs[ax]; }
    v.base = 0;
  }
  return v;
}

MDG_HD int cell_coord(const GridView& g, const Box& box, int ax, double x)
{
  int c = (int)floor((x - g.lo[ax]) / g.cs[ax]);
  if (box.pbc[ax]) {
    c %= g.nc[ax];
    if (c < 0) c += g.nc[ax];
  } else {
    if (c < 0) c = 0;
    if (c >= g.nc[ax]) c = g.nc[ax] - 1;
  }
  return c;
}

MDG_HD int cell_of(const Grid& g, const State& S, int a)
{
  const GridView v = grid_view(g, S, a);
  const Box& box = box_of(S, a);
  const double4 p = S.pos[a];
  int cx = cell_coord(v, box, 0, p.x), cy = cell_coord(v, box, 1, p.y), cz = cell_coord(v, box, 2, p.z);
  return v.base + (cz * v.nc[1] + cy) * v.nc[0] + cx;
}

// Insertion sort of a short int range (ascending).
MDG_HD void isort(int* v, int n)
{
  for (int a = 1; a < n; a++) {
    int x = v[a];
    int b = a - 1;
    while (b >= 0 && v[b] > x) { v[b + 1] = v[b]; b--; }
    v[b + 1] = x;
  }
}

// Build atom i's list from the cell grid (or by brute force); ascending order.
// A periodic axis with fewer than 3 cells (batched systems only) visits each
// of its cells once.
MDG_HD void nl_build_atom(const State& S, const Grid& g, NList& L, int i, unsigned int* status)
{
  const double4 pi = S.pos[i];
  const V3 xi = v3(pi.x, pi.y, pi.z);
  const Box& box = box_of(S, i);
  int cnt = 0;
  int* out = L.list + (long)i * L.cap;
  // FGeneral's handled pairs: REBO and AIREBO never see metal or ion atoms
  const bool ich = pi.w < 1.5;
  if (L.pairs == 1 && !ich) {
    L.cnt[i] = 0;
    L.pos0[i] = pi;
    return;
  }
  if (g.brute && !S.sys) {
    for (int j = 0; j < S.n; j++) {
      if (j == i) continue;
      double4 pj = S.pos[j];
      if (L.pairs && (L.pairs == 1 ? pj.w > 1.5 : (ich && pj.w < 1.5))) continue;
      V3 d = depos(box, xi, v3(pj.x, pj.y, pj.z));
      if (norm2(d) < L.range2) {
        if (cnt < L.cap) out[cnt] = j;
        cnt++;
      }
    }
  } else {
    const GridView v = grid_view(g, S, i);
    int c0[3], dlo[3], dhi[3];
    for (int ax = 0; ax < 3; ax++) {
      c0[ax] = cell_coord(v, box, ax, ax == 0 ? pi.x : (ax == 1 ? pi.y : pi.z));
      dlo[ax] = -1;
      dhi[ax] = 1;
      if (box.pbc[ax] && v.nc[ax] < 3) { dlo[ax] = 0; dhi[ax] = v.nc[ax] - 1; }
    }
    for (int dz = dlo[2]; dz <= dhi[2]; dz++) {
      int cz = c0[2] + dz;
      if (box.pbc[2]) cz = (cz + v.nc[2]) % v.nc[2];
      else if (cz < 0 || cz >= v.nc[2]) continue;
      for (int dy = dlo[1]; dy <= dhi[1]; dy++) {
        int cy = c0[1] + dy;
        if (box.pbc[1]) cy = (cy + v.nc[1]) % v.nc[1];
        else if (cy < 0 || cy >= v.nc[1]) continue;
        for (int dx = dlo[0]; dx <= dhi[0]; dx++) {
          int cx = c0[0] + dx;
          if (box.pbc[0]) cx = (cx + v.nc[0]) % v.nc[0];
          else if (cx < 0 || cx >= v.nc[0]) continue;
          int cell = v.base + (cz * v.nc[1] + cy) * v.nc[0] + cx;
          int b = g.cstart[cell], e = g.cstart[cell + 1];
          for (int q = b; q < e; q++) {
            int j = g.catoms[q];
            if (j == i) continue;
            double4 pj = S.pos[j];
            if (L.pairs && (L.pairs == 1 ? pj.w > 1.5 : (ich && pj.w < 1.5))) continue;
            V3 d = depos(box, xi, v3(pj.x, pj.y, pj.z));
            if (norm2(d) < L.range2) {
              if (cnt < L.cap) out[cnt] = j;
              cnt++;
            }
          }
        }
      }
    }
    if (L.sorted && cnt <= L.cap) isort(out, cnt);
  }
  if (cnt > L.cap) {
    *status |= ST_NL_OVERFLOW;
    cnt = L.cap;
  }
  L.cnt[i] = cnt;
  L.pos0[i] = pi;
}

// Squared displacement since the last build (minimum image).
MDG_HD double disp_atom(const State& S, const NList& L, int i)
{
  double4 p = S.pos[i], q = L.pos0[i];
  V3 d = depos(box_of(S, i), v3(p.x, p.y, p.z), v3(q.x, q.y, q.z));
  return sqrt(norm2(d));
}

// Mutable view of the bond list for the builder.
struct BondBuild {
  int n, mb;
  int* nb;
  int* bj;
  int* brev;
  double4* brv;
  double4* bu;
  double4* bd;
  double4* nco;
};

// Bonds of atom a from its REBO-range Verlet list (ascending, as the
// reference's NL order), with the REBO cutoffs of each pair
// (REBO::countNeighbours, REBO.cxx:328-393; AtomsPair, AtomsPair.hpp:137-158).
MDG_HD void bonds_atom(const State& S, const NList& L, const ReboParams& P, BondBuild& B, int a,
                       unsigned int* status)
{
  const double4 pa = S.pos[a];
  const int ta = (int)pa.w;
  const V3 xa = v3(pa.x, pa.y, pa.z);
  const int cnt = L.cnt[a];
  const int* lst = L.list + (long)a * L.cap;
  double Nt = 0.0, NC = 0.0, NH = 0.0;
  int nb = 0;
  for (int s = 0; s < cnt; s++) {
    const int j = lst[s];
    const double4 pj = S.pos[j];
    const int tj = (int)pj.w;
    V3 rv = depos(box_of(S, a), xa, v3(pj.x, pj.y, pj.z));
    double d2 = norm2(rv);
    const double R1 = P.R[ta][tj][0], R2 = P.R[ta][tj][1];
    if (d2 > R2 * R2) continue;
    double r = sqrt(d2);
    double f, df;
    cutoff(r, R1, R2, f, df);
    double Rp1 = P.Rp[ta][tj][0], Rp2 = P.Rp[ta][tj][1];
    double fp = Sprime(r, Rp1, Rp2), dfp = dSprime(r, Rp1, Rp2);
    if (!(r > R2)) {
      Nt += f;
      if (tj == kH) NH += f;
      if (tj == kC) NC += f;
    }
    if (nb < B.mb) {
      const int q = a * B.mb + nb;
      B.bj[q] = j;
      B.brv[q] = make_double4(rv.x, rv.y, rv.z, r);
      B.bu[q] = make_double4(rv.x / r, rv.y / r, rv.z / r, f);
      B.bd[q] = make_double4(df, fp, dfp, 0.0);
    }
    nb++;
  }
  if (nb > B.mb) {
    *status |= ST_BOND_OVERFLOW;
    nb = B.mb;
  }
  B.nb[a] = nb;
  B.nco[a] = make_double4(Nt, NC, NH, (double)ta);
}

// Slot of atom a in each partner's bond list.
MDG_HD void brev_atom(BondBuild& B, int a)
{
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int j = B.bj[a * B.mb + s];
    const int nbj = B.nb[j];
    int r = -1;
    for (int t = 0; t < nbj; t++)
      if (B.bj[j * B.mb + t] == a) { r = t; break; }
    B.brev[a * B.mb + s] = r;
  }
}

// Per-atom force-evaluation outputs (W: double, or dual on the adjoint path).
template <class Ws>
struct ForceOutT {
  typedef typename Q4T<Ws>::T Q4;
  int mb;
  Ws* A;            // [n * mb * 3] gradient owed to the partner of each bond slot
  Ws* W;            // [n * mb]     third-shell coefficients
  Q4* gown;         // [n] own gradient (REBO + torsion kernel)
  Q4* glj;          // [n] own gradient (LJ kernels)
  Ws* e_rebo;       // [n] per-atom energies (lower-index end of each bond)
  Ws* e_tors;
  Ws* e_lj;
  Ws* dp;           // [n * kNParam] energy derivatives by parameter (adjoint path only)
  int jt;           // adjoint path: 1 = J^T u, 0 = J u in the gradient's tangents
};
typedef ForceOutT<double> ForceOut;

// REBO (+ torsion) for every bond of atom a, evaluated as the reference's
// bond (min, max) and routed through a Sink for atom a.  ADJ: the adjoint
// path (duals; parameter derivatives into O.dp).
template <bool ADJ = false, class Real, class TB>
MDG_HD void rebo_atom(const ReboT<Real, TB>& R, const TorsParams& TP, int do_rebo, int do_tors,
                      ForceOutT<typename Wide<Real>::T>& O, int a)
{
  typedef typename Wide<Real>::T Wd;
  const auto& B = R.B;
  SinkT<Real, ADJ> sink;
  sink.a = a;
  sink.g = v3r<Wd>(0.0, 0.0, 0.0);
  sink.A = O.A + (long)a * O.mb * 3;
  sink.W = O.W + (long)a * O.mb;
  sink.dp = nullptr;
  sink.jt = 1;
  if constexpr (ADJ) {
    sink.jt = O.jt;
    sink.dp = O.dp + (long)a * kNParam;
    for (int k = 0; k < kNParam; k++) sink.dp[k] = 0.0;
  }
  for (int s = 0; s < O.mb * 3; s++) sink.A[s] = 0.0;
  for (int s = 0; s < O.mb; s++) sink.W[s] = 0.0;
  Wd er = 0.0, et = 0.0;
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int q = a * B.mb + s;
    const int b = B.bj[q];
    PairGT<Real> p = pair_from_slot<Real>(B, q);
    int lo = a, hi = b;
    if (b < a) { lo = b; hi = a; p = pair_reverse(p); }
    if (do_rebo) {
      Wd E = dbl(R.bond(lo, hi, p, sink));
      if (a == lo) er += E;
    }
    if (do_tors) {
      Wd E = dbl(etors_bond(R, TP, lo, hi, p, sink));
      if (a == lo) et += E;
    }
  }
  O.gown[a] = make_q4(sink.g.x, sink.g.y, sink.g.z, Wd(0.0));
  O.e_rebo[a] = er;
  O.e_tors[a] = et;
}

// REBO (+ torsion) as one task per directed bond slot (a, s): the bond
// (min, max) is evaluated in full and routed through a Sink for atom a into a
// private record [g(3), e_rebo, e_tors, A(3 nb_a), W(nb_a)].  The records of
// an atom's slots lie consecutively from rbase[a]; a per-atom reduction sums
// them in slot order.  Splitting an atom's bonds over threads shortens the
// longest serial chain from all of a carbon's bonds to one bond.
struct BondTasks {
  int cap;                  // queue capacity (n * mb)
  // 0: one task per directed slot; 1: one task per bond (slots to higher
  // partners); 2: per bond, the two ends' bond-order terms on a lane pair and
  // the torsion of each C-C bond as a task of its own
  int pairs;
  int tors;                 // torsion on (mode 2 gives C-C bonds a torsion record at each end)
  int* q;                   // slots a*mb+s: C-C bonds from the front, the rest from the back
  unsigned long long* ctr;  // [0] C-C tasks, [1] other tasks, [2] record doubles handed out
  long* rbase;              // [n] first record double of atom a (-1: over capacity, flagged)
  int* nrec;                // [n] records of atom a: its bond slots, then (mode 2) its C-C torsion records
  double* rec;
  long rec_cap;
};

MDG_HD int bond_rec_size(int nb) { return 5 + 4 * nb; }

template <class Real, class TB>
MDG_HD void rebo_task(const ReboT<Real, TB>& R, const TorsParams& TP, int do_rebo, int do_tors, double* rec, int a,
                      int s)
{
  const auto& B = R.B;
  const int nb = B.nb[a];
  SinkT<Real> sink;
  sink.a = a;
  sink.g = v3(0, 0, 0);
  sink.A = rec + 5;
  sink.W = rec + 5 + 3 * nb;
  for (int t = 0; t < 4 * nb; t++) sink.A[t] = 0.0;  // A and W are contiguous
  const int q = a * B.mb + s;
  const int b = B.bj[q];
  PairGT<Real> p = pair_from_slot<Real>(B, q);
  int lo = a, hi = b;
  if (b < a) { lo = b; hi = a; p = pair_reverse(p); }
  double er = 0.0, et = 0.0;
  if (do_rebo) {
    const Real E = R.bond(lo, hi, p, sink);
    if (a == lo) er = dbl(E);
  }
  if (do_tors) {
    const Real E = etors_bond(R, TP, lo, hi, p, sink);
    if (a == lo) et = dbl(E);
  }
  rec[0] = sink.g.x;
  rec[1] = sink.g.y;
  rec[2] = sink.g.z;
  rec[3] = er;
  rec[4] = et;
}

// REBO (+ torsion) of bond slot s of atom lo (partner hi > lo, slot sh in
// hi's list) into both ends' records.
template <class Real, class TB>
MDG_HD void rebo_pair_task(const ReboT<Real, TB>& R, const TorsParams& TP, int do_rebo, int do_tors, double* rlo,
                           double* rhi, int lo, int s, int hi)
{
  const auto& B = R.B;
  const int na = B.nb[lo], nb = B.nb[hi];
  PairSinkT<Real> sink;
  sink.a = lo;
  sink.b = hi;
  sink.ga = v3(0, 0, 0);
  sink.gb = v3(0, 0, 0);
  sink.Aa = rlo + 5;
  sink.Wa = rlo + 5 + 3 * na;
  sink.Ab = rhi + 5;
  sink.Wb = rhi + 5 + 3 * nb;
  for (int t = 0; t < 4 * na; t++) sink.Aa[t] = 0.0;
  for (int t = 0; t < 4 * nb; t++) sink.Ab[t] = 0.0;
  const PairGT<Real> p = pair_from_slot<Real>(B, lo * B.mb + s);
  double er = 0.0, et = 0.0;
  if (do_rebo) er = dbl(R.bond(lo, hi, p, sink));
  if (do_tors) et = dbl(etors_bond(R, TP, lo, hi, p, sink));
  rlo[0] = sink.ga.x;
  rlo[1] = sink.ga.y;
  rlo[2] = sink.ga.z;
  rlo[3] = er;
  rlo[4] = et;
  rhi[0] = sink.gb.x;
  rhi[1] = sink.gb.y;
  rhi[2] = sink.gb.z;
  rhi[3] = 0.0;
  rhi[4] = 0.0;
}

// Total dE/dx_a: own parts, what bond partners owe a, and the third-shell
// switching derivatives (dfThem through N_conj) resolved by gathering the
// coefficients of the bonds around a and around each switching partner.
template <class Ws>
MDG_HD V3T<Ws> gather_atom(const BondListT<Ws>& B, const ForceOutT<Ws>& O, int a, int with_lj,
                           const typename Q4T<Ws>::T* gextra)
{
  const auto g0 = O.gown[a];
  V3T<Ws> g = v3r<Ws>(g0.x, g0.y, g0.z);
  if (with_lj) {
    const auto g1 = O.glj[a];
    g += v3r<Ws>(g1.x, g1.y, g1.z);
  }
  if (gextra) {
    const auto g2 = gextra[a];
    g += v3r<Ws>(g2.x, g2.y, g2.z);
  }
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int q = a * B.mb + s;
    const int k = B.bj[q];
    const int r = B.brev[q];
    if (r < 0) continue;  // partner list truncated by an overflow (already flagged)
    const Ws* Ak = O.A + ((long)k * O.mb + r) * 3;
    g += v3r<Ws>(Ak[0], Ak[1], Ak[2]);
  }
  for (int s = 0; s < nb; s++) {
    const int q = a * B.mb + s;
    const Ws df = B.bd[q].x;
    if (df == 0.0) continue;
    const int m = B.bj[q];
    Ws wa = 0.0;
    for (int t = 0; t < nb; t++) {
      if (t == s) continue;
      const int qt = a * B.mb + t;
      if (B.brev[qt] < 0) continue;
      wa += O.W[(long)B.bj[qt] * O.mb + B.brev[qt]];
    }
    Ws wm = 0.0;
    const int nbm = B.nb[m];
    for (int t = 0; t < nbm; t++) {
      const int qt = m * B.mb + t;
      const int c = B.bj[qt];
      if (c == a || B.brev[qt] < 0) continue;
      wm += O.W[(long)c * O.mb + B.brev[qt]];
    }
    const auto u = B.bu[q];
    g += v3r<Ws>(u.x, u.y, u.z) * (df * (wa + wm));
  }
  return g;
}

// eq 1 (SimLoop.cxx:323-332): x += v dt + a dt^2 / 2 for free atoms.
MDG_HD void verlet_pos_atom(State& S, double dt, int i)
{
  if (S.fixed && S.fixed[i]) return;
  double4 p = S.pos[i], v = S.vel[i], ac = S.acc[i];
  p.x += v.x * dt + ac.x * dt * dt / 2.0;
  p.y += v.y * dt + ac.y * dt * dt / 2.0;
  p.z += v.z * dt + ac.z * dt * dt / 2.0;
  S.pos[i] = p;
}

// Atom::applyPBC (mdtk/Atom.cxx:94-126): shift into [0, L) and count images.
// The reference subtracts L one period at a time; a one-period move (the
// normal case) gives the same value here.  Larger jumps are shifted in one
// step, and a non-finite coordinate is reported instead of looping forever.
MDG_HD bool wrap1(double& x, int& im, double L)
{
  if (!isfinite(x)) return false;
  if (x < 0 || x >= L) {
    double nsh = floor(x / L);
    if (fabs(nsh) > 1e9) return false;
    x -= nsh * L;
    im += (int)nsh;
    for (int q = 0; q < 2 && x < 0; q++) { x += L; --im; }
    for (int q = 0; q < 2 && x >= L; q++) { x -= L; ++im; }
  }
  return true;
}

MDG_HD void wrap_atom(State& S, int i, unsigned int* status)
{
  double4 p = S.pos[i];
  int4 im = S.image[i];
  bool ok = true;
  const Box& box = box_of(S, i);
  if (box.pbc[0]) ok &= wrap1(p.x, im.x, box.L[0]);
  if (box.pbc[1]) ok &= wrap1(p.y, im.y, box.L[1]);
  if (box.pbc[2]) ok &= wrap1(p.z, im.z, box.L[2]);
  if (!ok && status) *status |= ST_NONFINITE;
  S.pos[i] = p;
  S.image[i] = im;
}

// Thermal bath and adaptive time step of the step body (SimLoop.cxx:280-287,
// 352-388, 394-416; the bath geometries of SimLoop.hpp:96-191).  Times in fs,
// lengths in Angstrom, the friction rate gamma in 1/fs.
struct StepDev {
  double dt;                      // fixed time step when d_dt is null
  const double* d_dt;             // per-system time step (adaptive dt) or null
  int tb_geom;                    // 0 none, 1 universe, 2 box, 3 sphere (SimLoop::TB_GEOM_*)
  double T0, gamma;               // bath temperature (K), friction rate
  double gp[5];                   // box: zMin, dBoundary, zMinOfFreeZone; sphere: cx, cy, cz, radius, zMinOfFreeZone
  const unsigned char* tb_apply;  // per atom Atom::apply_ThermalBath (null: every atom)
  const double* tb_T;             // per system: the bath temperature at the step start
  unsigned long long* vmax;       // per system: bits of the largest |v| (adaptive dt), or null
  const int* nlc0;                // list counts, FProxy::hasNeighbors (FProxy.hpp:99-105)
  const int* nlc1;                // (null when there is no second list)
  const int* nlc2;                // metal and ion pair list (null when there is none)
  double* ekin_pre;               // per atom M V_n^2 / 2 before the kick (SimLoop::energyKin at
                                  // doEnergyConservationCheck, SimLoop.cxx:337), or null
  double4* acc_ntb;               // per atom Atom::an_no_tb, updated in the bath branch only
  double* eb;                     // per atom running sum of Check::energyTransferredFromBath
                                  // (SimLoop.cxx:362-385); both null without a bath
  const int* stop;                // per system: reached simTimeFinal (SimLoop's loop condition),
                                  // steps of dt 0 leave it unchanged; or null
};

MDG_HD int sys_of(const State& S, int i) { return S.sys ? S.sys[i] : 0; }
MDG_HD double step_dt(const StepDev& P, const State& S, int i)
{
  if (!P.d_dt) return P.dt;
  const int s = sys_of(S, i);
  return (P.stop && P.stop[s]) ? 0.0 : P.d_dt[s];
}

// SimLoop::thermalBathShouldBeApplied (SimLoop.hpp:164-191) at atom i's
// current coordinates.
MDG_HD bool in_bath(const StepDev& P, const State& S, int i)
{
  if (!P.tb_geom || (P.tb_apply && !P.tb_apply[i])) return false;
  if (P.tb_geom == 1) return true;
  const double4 x = S.pos[i];
  if (P.tb_geom == 2) {
    const Box& b = box_of(S, i);
    const bool lateral = b.pbc[0] && b.pbc[1];
    return (x.z > P.gp[0]) ||
           (lateral && ((x.x < 0.0 + P.gp[1]) || (x.x > b.L[0] - P.gp[1]) || (x.y < 0.0 + P.gp[1]) ||
                        (x.y > b.L[1] - P.gp[1])) &&
            x.z > P.gp[2]);
  }
  const double dx = P.gp[0] - x.x, dy = P.gp[1] - x.y, dz = P.gp[2] - x.z;
  return x.z > P.gp[4] && sqrt(dx * dx + dy * dy + dz * dz) > P.gp[3];
}

// eq 2-4 (SimLoop.cxx:339-399) without the thermal bath: v += a_old dt/2,
// a = F/M, v += a dt/2; then applyPBC (SimLoop.cxx:401).
MDG_HD void verlet_vel_atom(State& S, V3 grad, double dt, int i, unsigned int* status)
{
  if (!(S.fixed && S.fixed[i])) {
    double4 v = S.vel[i], ac = S.acc[i];
    double m = S.mass[i];
    V3 vdt2 = v3(v.x + ac.x * dt / 2.0, v.y + ac.y * dt / 2.0, v.z + ac.z * dt / 2.0);
    V3 an = v3(-grad.x / m * kAccConv, -grad.y / m * kAccConv, -grad.z / m * kAccConv);
    S.acc[i] = make_double4(an.x, an.y, an.z, 0.0);
    S.vel[i] = make_double4(vdt2.x + an.x * dt / 2.0, vdt2.y + an.y * dt / 2.0, vdt2.z + an.z * dt / 2.0, 0.0);
  }
  wrap_atom(S, i, status);
}

// eq 2-4 with the thermal bath and the adaptive-dt maximum: a bath atom
// feels dF = -V M gamma (1 - sqrt(T0/T)) with T0/T clamped to [-5, 5] (0 when
// |T| < 1e-5), so a = F/M - gamma (1 - sqrt(T0/T)) v_n; |v_{n+1}| of free
// atoms with neighbours enters the system's maximum (SimLoop.cxx:352-398).
MDG_HD void verlet_vel_ext_atom(State& S, V3 grad, const StepDev& P, int i, unsigned int* status)
{
  if (!(S.fixed && S.fixed[i])) {
    const double dt = step_dt(P, S, i);
    double4 v = S.vel[i], ac = S.acc[i];
    double m = S.mass[i];
    V3 vdt2 = v3(v.x + ac.x * dt / 2.0, v.y + ac.y * dt / 2.0, v.z + ac.z * dt / 2.0);
    V3 an = v3(-grad.x / m * kAccConv, -grad.y / m * kAccConv, -grad.z / m * kAccConv);
    if (in_bath(P, S, i)) {
      const double T = P.tb_T[sys_of(S, i)];
      double r = (fabs(T) < 1e-5) ? 0.0 : P.T0 / T;
      if (r < -5.0) r = -5.0;
      if (r > 5.0) r = 5.0;
      const double k = P.gamma * (1.0 - sqrt(r));
      const V3 an_ntb = an;
      an = v3(an.x - v.x * k, an.y - v.y * k, an.z - v.z * k);
      if (P.eb) {
        // the kinetic energy the bath added this step: the half-kicks with
        // and without the bath term, each from its own previous acceleration
        const double4 ao = P.acc_ntb[i];
        P.acc_ntb[i] = make_double4(an_ntb.x, an_ntb.y, an_ntb.z, 0.0);
        const double h = dt / 2.0;
        const V3 w = v3(v.x + (ac.x * h + an.x * h), v.y + (ac.y * h + an.y * h), v.z + (ac.z * h + an.z * h));
        const V3 u = v3(v.x + (ao.x * h + an_ntb.x * h), v.y + (ao.y * h + an_ntb.y * h),
                        v.z + (ao.z * h + an_ntb.z * h));
        P.eb[i] += (m * (w.x * w.x + w.y * w.y + w.z * w.z) / 2.0 - m * (u.x * u.x + u.y * u.y + u.z * u.z) / 2.0) /
                   kAccConv;
      }
    }
    S.acc[i] = make_double4(an.x, an.y, an.z, 0.0);
    const V3 vn = v3(vdt2.x + an.x * dt / 2.0, vdt2.y + an.y * dt / 2.0, vdt2.z + an.z * dt / 2.0);
    S.vel[i] = make_double4(vn.x, vn.y, vn.z, 0.0);
#if defined(__CUDA_ARCH__)
    if (P.vmax && (P.nlc0[i] > 0 || (P.nlc1 && P.nlc1[i] > 0) || (P.nlc2 && P.nlc2[i] > 0))) {
      const double vm = sqrt(vn.x * vn.x + vn.y * vn.y + vn.z * vn.z);
      // non-negative doubles order like their bit patterns: the maximum does
      // not depend on the order of the atomics
      atomicMax(P.vmax + sys_of(S, i), (unsigned long long)__double_as_longlong(vm));
    }
#endif
  }
  wrap_atom(S, i, status);
}

}  // namespace mdg

