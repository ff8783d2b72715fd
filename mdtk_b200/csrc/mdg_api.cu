// mdg context, kernels and C ABI.
//
// One force evaluation (REBO [+ torsion] [+ AIREBO LJ]) on the device:
//   disp check -> (conditional) cell-list Verlet rebuild -> bond list ->
//   bond-order kernel (each bond from both ends) -> [LJ kernels] ->
//   gather (deterministic per-atom force sum) -> integration / energy.
// All launches go to one stream; list rebuilds are decided on the device, so
// a device-resident MD run needs no host round trip per step.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "mdg.h"
#include "mdg_step.cuh"
#include "mdg_tables.h"
#include "mdg_lj.cuh"
#include "mdg_brenner.cuh"

using namespace mdg;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
  g_err = msg;
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(MDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kThreads = 128;
constexpr int kRedBlocks = 120;
constexpr double kAo = 1e-8, kEv = 1.6021e-12, kFs = 1e-15;

inline int nblk(int n, int t = kThreads) { return (n + t - 1) / t; }
}  // namespace
#include "mdg_metal.cuh"
namespace {

// ---------------------------------------------------------------- kernels

// (t1, t2) <- the two largest of {t1, t2, u1, u2}, given t1 >= t2, u1 >= u2.
__device__ __forceinline__ void top2_merge(double& t1, double& t2, double u1, double u2)
{
  if (u1 >= t1) { t2 = fmax(t1, u2); t1 = u1; }
  else t2 = fmax(t2, u1);
}

// Start of a step: the position update x += v dt + a dt^2/2 (do_pos, eq 1
// of the step) and, per block, the two largest displacements since each
// list's last build (lists 0-2 and, as slot 3, the LJ list's near sublist;
// partials of slot l at part + 2 gridDim.x l).  The last block to finish (a
// counter, no waiting) reduces the partials of each slot to its rebuild flag:
// need[l] = force[l] || top1 + top2 > trigger (NeighbourList::MovedTooMuch,
// NeighbourList.cxx:109-133), then clears force[l].
constexpr int kNSlots = 4;
__global__ void k_step_start(State S, StepDev P, int do_pos, NList L0, NList L1, NList L2, NList L3, int mask,
                             double* part, int* need, int* force, unsigned int* done)
{
  pdl_enter();
  __shared__ double s1[kNSlots][kThreads / 32], s2[kNSlots][kThreads / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double d1[kNSlots] = {0.0, 0.0, 0.0, 0.0}, d2[kNSlots] = {0.0, 0.0, 0.0, 0.0};
  for (int a = i; a < S.n; a += gridDim.x * blockDim.x) {
    if (do_pos) verlet_pos_atom(S, step_dt(P, S, a), a);
#pragma unroll
    for (int l = 0; l < kNSlots; l++) {
      if (!((mask >> l) & 1)) continue;
      const double d = disp_atom(S, l == 0 ? L0 : (l == 1 ? L1 : (l == 2 ? L2 : L3)), a);
      if (d >= d1[l]) { d2[l] = d1[l]; d1[l] = d; }
      else if (d >= d2[l]) d2[l] = d;
    }
  }
#pragma unroll
  for (int l = 0; l < kNSlots; l++) {
    if (!((mask >> l) & 1)) continue;
    for (int o = 16; o > 0; o >>= 1) {
      const double u1 = __shfl_down_sync(0xffffffffu, d1[l], o), u2 = __shfl_down_sync(0xffffffffu, d2[l], o);
      top2_merge(d1[l], d2[l], u1, u2);
    }
    if (lane == 0) {
      s1[l][wid] = d1[l];
      s2[l][wid] = d2[l];
    }
  }
  __syncthreads();
  if (threadIdx.x < kNSlots && ((mask >> threadIdx.x) & 1)) {
    const int l = threadIdx.x;
    double t1 = 0.0, t2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) top2_merge(t1, t2, s1[l][w], s2[l][w]);
    part[2 * gridDim.x * l + 2 * blockIdx.x] = t1;
    part[2 * gridDim.x * l + 2 * blockIdx.x + 1] = t2;
  }
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // warp l: each lane keeps the two largest of a strided share of the
  // partials, then the lanes' pairs are merged by shuffles (the two largest
  // of a set do not depend on the order they are met in)
  if (wid < kNSlots && ((mask >> wid) & 1)) {
    const int l = wid;
    const double* pl = part + 2 * gridDim.x * l;
    double t1 = 0.0, t2 = 0.0;
    for (int q = lane; q < (int)gridDim.x; q += 32) top2_merge(t1, t2, __ldcg(pl + 2 * q), __ldcg(pl + 2 * q + 1));
    for (int o = 16; o > 0; o >>= 1) {
      const double u1 = __shfl_down_sync(0xffffffffu, t1, o), u2 = __shfl_down_sync(0xffffffffu, t2, o);
      top2_merge(t1, t2, u1, u2);
    }
    if (lane == 0) {
      const double trig = l == 0 ? L0.trigger : (l == 1 ? L1.trigger : (l == 2 ? L2.trigger : L3.trigger));
      need[l] = force[l] || (t1 + t2 > trig);
      force[l] = 0;
    }
  }
  if (threadIdx.x == 0) *done = 0u;
}

__global__ void k_cell_count(State S, Grid g, const int* need)
{
  pdl_enter();
  if (!*need) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S.n) atomicAdd(&g.ccount[cell_of(g, S, i)], 1);
}

// single-block exclusive scan of the cell counts
__global__ void k_cell_scan(Grid g, const int* need)
{
  pdl_enter();
  if (!*need) return;
  __shared__ int part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int chunk = (g.ncell + nt - 1) / nt;
  int b = t * chunk, e = min(g.ncell, b + chunk);
  int s = 0;
  for (int c = b; c < e; c++) s += g.ccount[c];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int acc = 0;
    for (int q = 0; q < nt; q++) { int v = part[q]; part[q] = acc; acc += v; }
    g.cstart[g.ncell] = acc;
  }
  __syncthreads();
  int acc = part[t];
  for (int c = b; c < e; c++) { g.cstart[c] = acc; acc += g.ccount[c]; }
}

__global__ void k_cell_fill(State S, Grid g, const int* need)
{
  pdl_enter();
  if (!*need) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  int c = cell_of(g, S, i);
  int slot = atomicAdd(&g.ccursor[c], 1);
  g.catoms[g.cstart[c] + slot] = i;
}

// ascending atom order inside each cell (the fill order is racy); the cell's
// count and fill cursor, used up by now, go back to zero for the next build
__global__ void k_cell_sort(Grid g, const int* need)
{
  pdl_enter();
  if (!*need) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.ncell) return;
  int b = g.cstart[c], e = g.cstart[c + 1];
  isort(g.catoms + b, e - b);
  g.ccount[c] = 0;
  g.ccursor[c] = 0;
}

__global__ void k_nl_build(State S, Grid g, NList L, const int* need, unsigned int* status)
{
  pdl_enter();
  if (!*need) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < S.n) nl_build_atom(S, g, L, i, status);
}

__global__ void k_bonds(State S, NList L, ReboParams P, BondBuild B, BondTasks K, unsigned int* status)
{
  pdl_enter();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a == 0 && K.ctr) K.ctr[0] = K.ctr[1] = K.ctr[2] = 0;
  if (a < S.n) bonds_atom(S, L, P, B, a, status);
}

// Exclusive offset of this lane's v within a block handed out to the warp by
// one atomicAdd on *ctr.  All 32 lanes must call it.
__device__ unsigned long long warp_alloc(unsigned long long v, unsigned long long* ctr)
{
  const int lane = threadIdx.x & 31;
  unsigned long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  unsigned long long base = 0;
  if (lane == 31 && x) base = atomicAdd(ctr, x);
  base = __shfl_sync(0xffffffffu, base, 31);
  return base + x - v;
}

// Reverse slots, then the REBO bond tasks of each atom: record space and the
// task queue (C-C bonds, which carry the torsion and dihedral terms, first).
// Positions in the queue and the record pool depend on scheduling; the values
// written to each slot's record do not.
__global__ void k_brev(BondBuild B, BondTasks K, unsigned int* status)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = a < B.n;
  int nb = 0, ncc = 0;
  if (ok) {
    brev_atom(B, a);
    if (K.ctr) {
      nb = B.nb[a];
      if ((int)B.nco[a].w == kC)
        for (int s = 0; s < nb; s++) ncc += ((int)B.nco[B.bj[a * B.mb + s]].w == kC);
    }
  }
  if (!K.ctr) return;  // uniform over the launch
  // records: one per bond slot, then (split mode with torsion) one per C-C bond
  const int nrec = nb + ((K.pairs == 2 && K.tors) ? ncc : 0);
  const unsigned long long need = ok ? (unsigned long long)nrec * bond_rec_size(nb) : 0ull;
  const unsigned long long rb = warp_alloc(need, &K.ctr[2]);
  // queued slots: all (one task per directed slot) or those to higher
  // partners (one task per bond)
  int mcc = 0, mot = 0;
  if (ok)
    for (int s = 0; s < nb; s++) {
      const int j = B.bj[a * B.mb + s];
      if (K.pairs && j < a) continue;
      if (ncc && (int)B.nco[j].w == kC) mcc++;
      else mot++;
    }
  const unsigned long long i0 = warp_alloc(mcc, &K.ctr[0]);
  const unsigned long long i1 = warp_alloc(mot, &K.ctr[1]);
  if (!ok) return;
  if ((long)(rb + need) > K.rec_cap) {
    K.rbase[a] = -1;
    atomicOr(status, ST_RECORD_OVERFLOW);
  } else {
    K.rbase[a] = (long)rb;
  }
  K.nrec[a] = nrec;
  int f = (int)i0, b = (int)i1;
  for (int s = 0; s < nb; s++) {
    const int j = B.bj[a * B.mb + s];
    if (K.pairs && j < a) continue;
    const bool cc = ncc && (int)B.nco[j].w == kC;
    if (cc) K.q[f++] = a * B.mb + s;
    else K.q[K.cap - 1 - (b++)] = a * B.mb + s;
  }
}

__global__ void k_rebo(const ReboParams* P, const ReboTables* T, BondList B, TorsParams TP, int do_rebo,
                       int do_tors, ForceOut O, unsigned int* status)
{
  pdl_enter();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.n) return;
  Rebo R{*P, *T, B, status};
  rebo_atom(R, TP, do_rebo, do_tors, O, a);
}

// Task index of this thread in a grid-stride loop over a queue whose front
// holds the heaviest tasks (C-C bonds): consecutive warps of tasks go to
// consecutive blocks (warp w of block b takes task warp w * gridDim.x + b),
// so the heavy front of the queue is spread one warp per block over every SM
// instead of filling the first few blocks (and SMs).  A permutation of
// 0 .. gridDim.x * blockDim.x - 1.
__device__ __forceinline__ long spread_task_index()
{
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  return ((long)w * gridDim.x + blockIdx.x) * 32 + lane;
}

// REBO + torsion, one thread per directed bond slot, over a grid sized to the
// resident capacity of the GPU (grid-stride over the queue).
template <class Real, class TB>
__global__ void __launch_bounds__(128) k_rebo_task(const ReboParams* P, const TB* T, BondList B, TorsParams TP,
                                                   int do_rebo, int do_tors, BondTasks K, unsigned int* status)
{
  pdl_enter();
  const long n0 = (long)K.ctr[0], nt = n0 + (long)K.ctr[1];
  ReboT<Real, TB> R{*P, *T, B, status};
  for (long t = spread_task_index(); t < nt; t += (long)gridDim.x * blockDim.x) {
    const int q = t < n0 ? K.q[t] : K.q[K.cap - 1 - (t - n0)];
    const int a = q / B.mb, s = q - a * B.mb;
    const long rb = K.rbase[a];
    if (rb < 0) continue;
    rebo_task(R, TP, do_rebo, do_tors, K.rec + rb + (long)s * bond_rec_size(B.nb[a]), a, s);
  }
}

// REBO + torsion, one thread per bond (both ends' records), grid-stride.
template <class Real, class TB>
__global__ void __launch_bounds__(128) k_rebo_pair_task(const ReboParams* P, const TB* T, BondList B, TorsParams TP,
                                                        int do_rebo, int do_tors, BondTasks K,
                                                        unsigned int* status)
{
  pdl_enter();
  const long n0 = (long)K.ctr[0], nt = n0 + (long)K.ctr[1];
  ReboT<Real, TB> R{*P, *T, B, status};
  for (long t = spread_task_index(); t < nt; t += (long)gridDim.x * blockDim.x) {
    const int q = t < n0 ? K.q[t] : K.q[K.cap - 1 - (t - n0)];
    const int lo = q / B.mb, s = q - lo * B.mb;
    const int hi = B.bj[q], sh = B.brev[q];
    const long rl = K.rbase[lo], rh = K.rbase[hi];
    if (rl < 0 || rh < 0 || sh < 0) continue;  // already flagged
    rebo_pair_task(R, TP, do_rebo, do_tors, K.rec + rl + (long)s * bond_rec_size(B.nb[lo]),
                   K.rec + rh + (long)sh * bond_rec_size(B.nb[hi]), lo, s, hi);
  }
}

// The other lane's value of a lane pair (mask pm).
__device__ __forceinline__ double pair_swap(double v, unsigned pm) { return __shfl_xor_sync(pm, v, 1); }
__device__ __forceinline__ f32 pair_swap(f32 v, unsigned pm)
{
  f32 r;
  r.v = __shfl_xor_sync(pm, v.v, 1);
  return r;
}

// b-bar of bond (i, j), i < j, p = i -> j (REBO::Baver, REBO.cxx:200-211)
// split over the lane pair of the bond: lane e evaluates p^{sigma pi} of its
// own end (i for e = 0, j for e = 1) with its gradient, its half of N^conj
// and its end's third-shell terms; the two lanes trade p^{sigma pi} and the
// N^conj halves by shuffles and both evaluate pi^rc (and pi^dh, whose
// pair-vector pieces lane 0 keeps).  Every term is the one the whole-bond
// evaluation computes, in the same order within each end's record.
template <class Real, class TB>
__device__ Real baver_end(const ReboT<Real, TB>& R, int e, int i, int j, const PairGT<Real>& p, Real V,
                          EndSinkT<Real>& sink, unsigned pm)
{
  const PairGT<Real> q = pair_reverse(p);
  const Real half = V / 2.0;
  // one call on both lanes with this lane's end selected (branching on e
  // would make the warp run the two ends one after the other)
  const Real pmine = R.p_sigma_pi(e ? j : i, e ? i : j, e ? q : p, half, sink);
  const Real pother = pair_swap(pmine, pm);
  const Real pij = e == 0 ? pmine : pother, pji = e == 0 ? pother : pmine;
  Real val = (pij + pji) / 2.0;
  const int ti = R.type(i), tj = R.type(j);
  // pi_rc (REBO.cxx:659-714): the H-C order evaluates as C-H with i and j swapped
  int ci = i, cj = j;
  const PairGT<Real>* pc = &p;
  const PairGT<Real>* qc = &q;
  if (ti == kH && tj == kC) { ci = j; cj = i; pc = &q; qc = &p; }
  const int tci = R.type(ci), tcj = R.type(cj);
  const int fam = (tci == kC && tcj == kC) ? 0 : ((tci == kC && tcj == kH) ? 1 : 2);
  const Real Nti = R.Nval(ci, cj, *pc, 0);
  const Real Ntj = R.Nval(cj, ci, *qc, 0);
  const int me = e == 0 ? i : j;
  const bool is_ci = me == ci;
  const Real smine = R.nconj_sum(me, is_ci ? cj : ci);
  const Real sother = pair_swap(smine, pm);
  const Real s1 = is_ci ? smine : sother, s2 = is_ci ? sother : smine;
  Real Nconj = 1.0;
  Nconj += SQR(s1);
  Nconj += SQR(s2);
  Real F[4];
  t_eval(R.T, fam, Nti, Ntj, Nconj, F, R.status);
  val += F[0];
  Real cNti = 0.0, cNtj = 0.0, cNconj = 0.0;
  if (V != 0.0) {
    cNti = F[1] * V;
    cNtj = F[2] * V;
    cNconj = F[3] * V;
  }
  // pi_dh (REBO.cxx:761-814): C-C only, T_ij nonzero only near (2,2,.)
  if (ti == kC && tj == kC) {
    Real Tv[4];
    t_eval(R.T, 3, Nti, Ntj, Nconj, Tv, R.status);
    if (Tv[0] != 0.0) {
      const Real ts = R.dh_sum(i, j, p, 0.0, sink);
      val += Tv[0] * ts;
      if (V != 0.0) {
        if (ts != 0.0) {
          const Real Vt = ts * V;
          cNti += Tv[1] * Vt;
          cNtj += Tv[2] * Vt;
          cNconj += Tv[3] * Vt;
        }
        const bool on = sink.pair_on;
        sink.pair_on = e == 0;
        R.dh_sum(i, j, p, Tv[0] * V, sink);
        sink.pair_on = on;
      }
    }
  }
  if (V != 0.0) {
    const int oc = is_ci ? cj : ci;  // the other end
    R.dfthem(me, oc, is_ci ? cNti : cNtj, 0, sink);
    // REBO::Nconj's gradient (nconj_grad): each end its own half
    const Real sm = is_ci ? s1 : s2;
    if (cNconj != 0.0 && sm != 0.0) R.nconj_sum_grad(me, oc, 2.0 * sm * cNconj, sink);
  }
  return val;
}

// REBO of bond slot s of atom lo (partner hi) on a lane pair: lane e
// writes the record of its end (lo for e = 0, hi for e = 1); lane 0 adds
// V_R, the bond energy and V_A's pair pieces.  The torsion of the bond is
// a separate task.
template <class Real, class TB>
__device__ void rebo_end_task(const ReboT<Real, TB>& R, int do_rebo, double* rec, int e, int lo, int s, int hi)
{
  const auto& B = R.B;
  const unsigned pm = 3u << ((threadIdx.x & 31) & ~1);
  const int me = e ? hi : lo;
  const int nbm = B.nb[me];
  EndSinkT<Real> sink;
  sink.me = me;
  sink.lo = lo;
  sink.hi = hi;
  sink.pair_on = true;
  sink.glo = v3(0, 0, 0);
  sink.ghi = v3(0, 0, 0);
  sink.A = rec + 5;
  sink.W = rec + 5 + 3 * nbm;
  for (int t = 0; t < 4 * nbm; t++) sink.A[t] = 0.0;  // A and W are contiguous
  const PairGT<Real> p = pair_from_slot<Real>(B, lo * B.mb + s);
  double er = 0.0;
  if (do_rebo) {
    // REBO::operator() for one bond (REBO.cxx:43-59), as ReboT::bond does
    // V_R and V_A's pair pieces from lane 0 (lane 1 takes the values only)
    SinkT<Real> dummy;
    double va_val = 0.0, va_der = 0.0;
    if (p.f != 0.0) R.VA_terms(lo, hi, p, va_val, va_der);
    const Real vav = R.VA_from(lo, hi, p, va_val, va_der, 0.0, dummy);
    Real E = R.VR(lo, hi, p, e == 0 ? 1.0 : 0.0, sink);
    if (vav != 0.0) {
      const Real bav = baver_end(R, e, lo, hi, p, vav, sink, pm);
      E += bav * R.VA_from(lo, hi, p, va_val, va_der, e == 0 ? bav : Real(0.0), sink);
    }
    er = dbl(E);
  }
  // each end's own gradient: its lane's pieces plus the other lane's pair-vector pieces
  const double ox = __shfl_xor_sync(pm, e ? sink.glo.x : sink.ghi.x, 1);
  const double oy = __shfl_xor_sync(pm, e ? sink.glo.y : sink.ghi.y, 1);
  const double oz = __shfl_xor_sync(pm, e ? sink.glo.z : sink.ghi.z, 1);
  const V3 g = e ? sink.ghi : sink.glo;
  rec[0] = g.x + ox;
  rec[1] = g.y + oy;
  rec[2] = g.z + oz;
  rec[3] = e ? 0.0 : er;
  rec[4] = 0.0;
}

// Torsion of C-C bond slot s of atom lo (partner hi, slot sh in hi's list)
// into the two ends' torsion records (ETors::operator(), AIREBO_ETors.cxx:32-115).
template <class Real, class TB>
__device__ void rebo_tors_task(const ReboT<Real, TB>& R, const TorsParams& TP, double* rlo, double* rhi, int lo,
                               int s, int hi)
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
  const double et = dbl(etors_bond(R, TP, lo, hi, p, sink));
  rlo[0] = sink.ga.x;
  rlo[1] = sink.ga.y;
  rlo[2] = sink.ga.z;
  rlo[3] = 0.0;
  rlo[4] = et;
  rhi[0] = sink.gb.x;
  rhi[1] = sink.gb.y;
  rhi[2] = sink.gb.z;
  rhi[3] = 0.0;
  rhi[4] = 0.0;
}

// Index of slot s among atom a's C-C bond slots (its torsion record).
__device__ __forceinline__ int cc_index(const BondList& B, int a, int s)
{
  int k = 0;
  for (int t = 0; t < s; t++) k += ((int)B.nco[B.bj[a * B.mb + t]].w == kC);
  return k;
}

// REBO by bond ends on lane pairs, torsion by C-C bond: the work items are
// [0, 2 n0) the ends of the C-C bonds, [2 n0, 2 n0 + ntor) their torsions,
// then (from an even index) the ends of the other bonds; lanes 2m and 2m+1
// always hold items t and t^1, the two ends of one bond.
template <class Real, class TB>
__global__ void __launch_bounds__(128) k_rebo_split_task(const ReboParams* P, const TB* T, BondList B, TorsParams TP,
                                                         int do_rebo, int do_tors, BondTasks K, unsigned int* status)
{
  pdl_enter();
  const long n0 = (long)K.ctr[0], n1 = (long)K.ctr[1];
  const long ntor = do_tors ? n0 : 0;
  const long base1 = (2 * n0 + ntor + 1) & ~1L;
  const long total = base1 + 2 * n1;
  ReboT<Real, TB> R{*P, *T, B, status};
  // rounds alternate direction: a thread whose round-0 item was heavy (the
  // queue's front) takes one of the last, lightest items next, or none
  const long stride = (long)gridDim.x * blockDim.x, t0 = spread_task_index();
  for (long r = 0; r * stride < total; r++) {
    const long t = r * stride + ((r & 1) ? stride - 1 - t0 : t0);
    if (t >= total) continue;  // the same for both lanes of a pair (total is even)
    const bool cc_end = t < 2 * n0, tors = !cc_end && t < 2 * n0 + ntor;
    if (!cc_end && !tors && t < base1) continue;  // the padding item (its lane has no partner work)
    const long b = cc_end ? (t >> 1) : (tors ? t - 2 * n0 : ((t - base1) >> 1));
    const int q = (cc_end || tors) ? K.q[b] : K.q[K.cap - 1 - b];
    const int lo = q / B.mb, s = q - lo * B.mb;
    const int hi = B.bj[q], sh = B.brev[q];
    const long rl = K.rbase[lo], rh = K.rbase[hi];
    if (rl < 0 || rh < 0 || sh < 0) continue;  // already flagged (the same for both lanes of a pair)
    const int rsl = bond_rec_size(B.nb[lo]), rsh = bond_rec_size(B.nb[hi]);
    if (tors) {
      rebo_tors_task(R, TP, K.rec + rl + (long)(B.nb[lo] + cc_index(B, lo, s)) * rsl,
                     K.rec + rh + (long)(B.nb[hi] + cc_index(B, hi, sh)) * rsh, lo, s, hi);
    } else {
      const int e = (int)(t & 1);
      double* rec = e ? K.rec + rh + (long)sh * rsh : K.rec + rl + (long)s * rsl;
      rebo_end_task(R, do_rebo, rec, e, lo, s, hi);
    }
  }
}

// Per-atom sums of the bond-task records (REBO + torsion) and the special LJ
// records, a group of G lanes per atom.  Lane l owns elements l, l+G, ... of
//   [g_own(3), e_rebo, e_tors, g_lj(3), e_lj, A(3 nb), W(nb)]
// and adds each element's terms left to right: the atom's REBO slots in slot
// order, then its LJ tasks in task order.  Without REBO tasks the REBO-side
// elements keep what the per-atom kernels wrote; g_lj and e_lj start from the
// plain-pair kernel's values.
template <int G>
__global__ void k_bond_reduce(BondList B, BondTasks K, int rebo_tasks, SpecialTasks Tk, int with_lj, ForceOut O)
{
  pdl_enter();
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gid / G, l = gid - (gid / G) * G;
  if (a >= B.n) return;
  const int nb = B.nb[a];
  const int nel = 9 + 4 * nb;
  const long rb = rebo_tasks ? K.rbase[a] : -1;
  const int nrec = rebo_tasks ? K.nrec[a] : 0;
  const int rs = bond_rec_size(nb);
  int t0 = 0, t1 = 0;
  if (with_lj) spc_range(Tk, a, t0, t1);
  // the LJ pass over REBO sums already in place: an atom without special
  // pair records keeps every element as it is
  if (!rebo_tasks && with_lj && t1 <= t0) return;
  // an atom's special-pair records are handed out as one block, rec_size(nb)
  // doubles apart: when its first and last lie so (none beyond the pool),
  // every element reads them by stride instead of through trec
  long lbase = -1;
  const int lrs = rec_size(nb);
  if (with_lj && t1 > t0) {
    const long f = Tk.trec[t0], z = Tk.trec[t1 - 1];
    if (f >= 0 && z == f + (long)(t1 - 1 - t0) * lrs) lbase = f;
  }
  for (int e = l; e < nel; e += G) {
    int roff = -1, loff = -1;
    double* dst;
    if (e < 3) { roff = e; dst = reinterpret_cast<double*>(O.gown + a) + e; }
    else if (e == 3) { roff = 3; dst = O.e_rebo + a; }
    else if (e == 4) { roff = 4; dst = O.e_tors + a; }
    else if (e < 8) { loff = e - 5; dst = reinterpret_cast<double*>(O.glj + a) + (e - 5); }
    else if (e == 8) { loff = 3; dst = O.e_lj + a; }
    else {
      const int k = e - 9;
      roff = 5 + k;
      loff = 4 + k;
      dst = k < 3 * nb ? O.A + (long)a * O.mb * 3 + k : O.W + (long)a * O.mb + (k - 3 * nb);
    }
    if (!rebo_tasks) roff = -1;
    if (!with_lj) loff = -1;
    if (roff < 0 && loff < 0) continue;
    double acc = roff >= 0 ? 0.0 : *dst;
    if (roff >= 0 && rb >= 0)
      for (int s = 0; s < nrec; s++) acc += K.rec[rb + (long)s * rs + roff];
    if (loff >= 0 && lbase >= 0) {
      const double* r = Tk.rec + lbase + loff;
      for (int t = 0; t < t1 - t0; t++) acc += r[(long)t * lrs];
    } else if (loff >= 0) {
      int t = t0;
      for (; t + 3 < t1; t += 4) {
        const long r0 = Tk.trec[t], r1 = Tk.trec[t + 1], r2 = Tk.trec[t + 2], r3 = Tk.trec[t + 3];
        const double v0 = r0 >= 0 ? Tk.rec[r0 + loff] : 0.0;
        const double v1 = r1 >= 0 ? Tk.rec[r1 + loff] : 0.0;
        const double v2 = r2 >= 0 ? Tk.rec[r2 + loff] : 0.0;
        const double v3_ = r3 >= 0 ? Tk.rec[r3 + loff] : 0.0;
        if (r0 >= 0) acc += v0;
        if (r1 >= 0) acc += v1;
        if (r2 >= 0) acc += v2;
        if (r3 >= 0) acc += v3_;
      }
      for (; t < t1; t++) {
        const long r0 = Tk.trec[t];
        if (r0 >= 0) acc += Tk.rec[r0 + loff];
      }
    }
    *dst = acc;
  }
}

__global__ void k_brenner(const BrennerParams* P, const BrennerTables* T, BondList B, ForceOut O,
                          unsigned int* status)
{
  pdl_enter();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.n) return;
  Brenner R{*P, *T, B, status};
  brenner_atom(R, O, a);
}

constexpr int kCijLocal = 128;  // per-thread connectivity table capacity

// Also zeroes the special-pair counters that the special-pair finder after it
// hands ranges out of.
__global__ void k_cij(BondList B, CijTable T, unsigned long long* spc_ctr, unsigned int* status)
{
  pdl_enter();
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a == 0 && spc_ctr) spc_ctr[0] = spc_ctr[kCtrStride] = spc_ctr[2 * kCtrStride] = 0ull;
  if (a < B.n) cij_build_atom<kCijLocal>(B, T, a, status);
}

// The LJ list's near sublist: the entries within R2 + kLjNearSkin of the
// atom, in list order, one warp per atom (the filter's loop with a wider
// radius), and the positions it was taken at.  Rebuilt when the LJ list is
// (need[1]) or when the two largest displacements since the last near build
// exceed kLjNearSkin (need[3]); returns at once otherwise.  Every pair within
// R2 is in it: such a pair was within R2 + (its two displacements) <=
// R2 + kLjNearSkin at the near build, and in the LJ list.  The filter reads
// this sublist (about 0.3 of the LJ list) in place of the whole list; its
// order is the list's, so the in-range lists, and every sum over them, are
// the same.  A fixed grid of warps strides over the atoms, so the launch
// that finds no flag set costs a few blocks, not one per four atoms.
constexpr double kLjNearSkin = 0.5;  // Angstrom
__global__ void __launch_bounds__(kThreads) k_lj_near(LJParams P, State S, NList L, NList T, const int* need,
                                                      unsigned int* status)
{
  pdl_enter();
  if (!need[1] && !need[3]) return;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < S.n; a += nw) {  // whole warps
    const double4 pa = S.pos[a];
    const V3 xa = v3(pa.x, pa.y, pa.z);
    const int ta = (int)pa.w;
    const Box box = box_of(S, a);
    const int cnt = L.cnt[a];
    const int* lst = L.list + (long)a * L.cap;
    int* out = T.list + (long)a * T.cap;
    const unsigned below = (1u << lane) - 1u;
    int k = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int s = base + lane;
      bool in = false;
      int b = -1;
      if (s < cnt) {
        b = lst[s];
        const double4 pb = S.pos[b];
        const double R = P.R[ta][(int)pb.w][1] + kLjNearSkin;
        const V3 rv = depos(box, xa, v3(pb.x, pb.y, pb.z));
        in = norm2(rv) <= R * R * (1.0 + 1e-12);
      }
      const unsigned m = __ballot_sync(0xffffffffu, in);
      if (in) out[k + __popc(m & below)] = b;
      k += __popc(m);
    }
    if (lane == 0) {
      T.cnt[a] = k;
      T.pos0[a] = pa;
    }
  }
}

// LJ pairs inside their cutoff, one warp per atom: the atom's LJ list is
// read 32 entries at a time and the entries within the pair's cutoff R2 are
// appended, in list order, to the atom's far list (front of its in-range
// row, count far_cnt[a]) or, inside the S(t_r) window, its close list (back of
// the row, growing down; count close_cnt[a]); together about a quarter of
// the list.  It needs only positions and the list, so it runs concurrently
// with the bond and connectivity kernels; its few registers let many warps
// hide the position gathers.
__global__ void __launch_bounds__(kThreads) k_lj_filter(LJParams P, State S, NList L, int* inr, int* far_cnt,
                                                        int* close_cnt)
{
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < S.n; a += nw) {  // whole warps
    const double4 pa = S.pos[a];
    const V3 xa = v3(pa.x, pa.y, pa.z);
    const int ta = (int)pa.w;
    const Box box = box_of(S, a);
    const int cnt = L.cnt[a];
    const int* lst = L.list + (long)a * L.cap;
    int* out = inr + (long)a * L.cap;
    int* top = out + L.cap - 1;
    const unsigned below = (1u << lane) - 1u;
    int kf = 0, kc = 0;
    for (int base = 0; base < cnt; base += 32) {
      const int s = base + lane;
      bool in = false, close = false;
      int b = -1;
      if (s < cnt) {
        b = lst[s];
        const double4 pb = S.pos[b];
        const int tb = (int)pb.w;
        const double R2 = P.R[ta][tb][1];
        const V3 rv = depos(box, xa, v3(pb.x, pb.y, pb.z));
        const double d2 = norm2(rv);
        in = !(d2 > R2 * R2);
        close = in && lj_close(P, ta, tb, d2);  // lj_class's test, on the same d2
      }
      const unsigned mf = __ballot_sync(0xffffffffu, in && !close);
      const unsigned mc = __ballot_sync(0xffffffffu, close);
      if (in && !close) out[kf + __popc(mf & below)] = b;
      if (close) top[-(kc + __popc(mc & below))] = b;
      kf += __popc(mf);
      kc += __popc(mc);
    }
    if (lane == 0) {
      far_cnt[a] = kf;
      close_cnt[a] = kc;
    }
  }
}

// Exclusive offsets of this thread's v[0..2] within ranges handed out to the
// block by one atomicAdd per counter (ctr[0], ctr[kCtrStride],
// ctr[2 kCtrStride]).  Every thread of the block (blockDim.x == NT) calls it.
template <int NT>
__device__ void block_alloc3(const unsigned long long v[3], unsigned long long* ctr, unsigned long long out[3])
{
  __shared__ unsigned long long ws[3][NT / 32];
  __shared__ unsigned long long base[3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long x[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    x[k] = v[k];
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(0xffffffffu, x[k], o);
      if (lane >= o) x[k] += t;
    }
    if (lane == 31) ws[k][wid] = x[k];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int k = threadIdx.x;
    unsigned long long run = 0;
    for (int w = 0; w < NT / 32; w++) {
      const unsigned long long t = ws[k][w];
      ws[k][w] = run;
      run += t;
    }
    base[k] = run ? atomicAdd(ctr + k * kCtrStride, run) : 0ull;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 3; k++) out[k] = base[k] + ws[k][wid] + x[k] - v[k];
}

// The LJ pairs of each atom, kLjGroup lanes per atom: the plain pairs of its
// far list are evaluated here, and its special pairs (lj_class kind 2: the
// close pairs with C > 0, then the far pairs with 0 < w < 1, each in list
// order) are made into tasks for the special-pair kernels.  The filter has
// already split the in-range pairs by the S(t_r) window, so a close pair
// needs only its w (no positions).  w is looked up in the atom's own
// connectivity table, and only for the pairs its mask admits.  The atom's
// tasks, records and (with `pairs`) the work items of the pairs it owns as
// the lower index take ranges handed out per block.
constexpr int kLjGroup = 16;     // lanes per atom (a divisor of 32): ~30 in-range partners
constexpr int kLjThreads = 128;  // 8 atoms per block
constexpr int kReduceLanes = 8;
template <class Real>
__device__ __forceinline__ void lj_pairs_block(const LJParams& P, const CijTable& T, const State& S, int lcap,
                                               const int* inr, const int* far_cnt, const int* close_cnt,
                                               const int* nbonds, const ForceOut& O, const SpecialTasks& Tk,
                                               int pairs, unsigned int* status, int gid)
{
  const int lane = threadIdx.x & 31, gl = lane % kLjGroup, gbase = lane - gl;
  const bool live = gid < S.n;  // every thread stays for the block's allocation
  const int a = live ? gid : S.n - 1;
  const double4 pa = S.pos[a];
  const V3 xa = v3(pa.x, pa.y, pa.z);
  const int ta = (int)pa.w;
  const int nc = live ? close_cnt[a] : 0;
  const int nf = live ? far_cnt[a] : 0;
  const unsigned long long amask = T.mask[a];
  const int* row = inr + (long)a * lcap;
  int* part = Tk.part + (long)a * Tk.cap;
  const unsigned gmask = (kLjGroup == 32) ? 0xffffffffu : (((1u << kLjGroup) - 1u) << gbase);
  const unsigned below = ((1u << lane) - 1u) & gmask;
  int nsp = 0, nhi = 0;
  // appends this lane's b (when special) to the atom's special list
  auto note = [&](bool special, int b) {
    const unsigned m = __ballot_sync(0xffffffffu, special);
    const int pos = nsp + __popc(m & below);
    const bool keep = special && pos < Tk.cap;
    if (keep) part[pos] = b;
    nhi += __popc(__ballot_sync(0xffffffffu, keep && b > a) & gmask);
    nsp += __popc(m & gmask);
  };
  // the warp's longest lists bound its loops
  int wc = nc, wf = nf;
  for (int o = 16; o > 0; o >>= 1) {
    wc = max(wc, __shfl_xor_sync(0xffffffffu, wc, o));
    wf = max(wf, __shfl_xor_sync(0xffffffffu, wf, o));
  }
  for (int base = 0; base < wc; base += kLjGroup) {
    const int s = base + gl;
    int b = -1;
    bool sp = false;
    if (s < nc) {
      b = row[lcap - 1 - s];
      sp = lj_kind(lj_w_own(T, a, b, amask), true) == 2;
    }
    note(sp, b);
  }
  SinkT<Real> sk;
  sk.a = a;
  sk.g = v3(0, 0, 0);
  sk.A = nullptr;
  sk.W = nullptr;
  double e = 0.0;
  for (int base = 0; base < wf; base += kLjGroup) {
    const int s = base + gl;
    int b = -1, kind = 0;
    if (s < nf) {
      b = row[s];
      kind = lj_plain_pair<Real>(P, T, S, a, b, xa, ta, amask, sk, e, nullptr, true);
    }
    note(kind == 2, b);
  }
  double gx = sk.g.x, gy = sk.g.y, gz = sk.g.z;
  for (int o = kLjGroup / 2; o > 0; o >>= 1) {
    gx += __shfl_xor_sync(0xffffffffu, gx, o);
    gy += __shfl_xor_sync(0xffffffffu, gy, o);
    gz += __shfl_xor_sync(0xffffffffu, gz, o);
    e += __shfl_xor_sync(0xffffffffu, e, o);
  }
  if (nsp > Tk.cap) {
    if (live && gl == 0) atomicOr(status, ST_RECORD_OVERFLOW);
    nsp = Tk.cap;
  }
  const int rs = rec_size(live ? nbonds[a] : 0);
  const bool lead = live && gl == 0;
  unsigned long long v[3] = {lead && pairs ? (unsigned long long)nhi : 0ull, lead ? (unsigned long long)nsp : 0ull,
                             lead ? (unsigned long long)nsp * rs : 0ull};
  unsigned long long r[3];
  block_alloc3<kLjThreads>(v, Tk.ctr, r);  // also orders this block's part[] writes before the reads below
  // every lane of the group holds its leader's offsets
  const long wb = (long)__shfl_sync(0xffffffffu, r[0], gbase);
  const long o = (long)__shfl_sync(0xffffffffu, r[1], gbase);
  const long ro = (long)__shfl_sync(0xffffffffu, r[2], gbase);
  if (!live) return;
  if (gl == 0) {
    O.glj[a] = make_double4(gx, gy, gz, 0.0);
    O.e_lj[a] = e;
    Tk.cnt[a] = nsp;
    if (o + nsp > Tk.task_cap) atomicOr(status, ST_RECORD_OVERFLOW);
    Tk.off[a] = o < Tk.task_cap ? (int)o : Tk.task_cap;
  }
  for (int k = gl; k < nsp; k += kLjGroup) {
    const long t = o + k;
    if (t >= Tk.task_cap) break;
    Tk.flat[t] = make_int2(a, part[k]);
    const long rt = ro + (long)k * rs;
    if (rt + rs <= Tk.rec_cap) Tk.trec[t] = rt;
    else { Tk.trec[t] = -1; atomicOr(status, ST_RECORD_OVERFLOW); }
  }
  if (!pairs) return;  // uniform over the launch
  // the pairs this atom owns (b > a), in list order, as work items; a task
  // beyond the capacity leaves a -1 in its place
  int k = 0;
  for (int q0 = 0; q0 < nsp; q0 += kLjGroup) {
    const int qq = q0 + gl;
    const bool own = qq < nsp && part[qq] > a;
    const unsigned m = __ballot_sync(gmask, own);
    const long w = wb + k + __popc(m & below);
    if (own && w < Tk.task_cap) Tk.work[w] = (o + qq < Tk.task_cap) ? (int)(o + qq) : -1;
    k += __popc(m);
  }
}

template <class Real>
__global__ void __launch_bounds__(kLjThreads, 7) k_lj_pairs(LJParams P, CijTable T, State S, int lcap, const int* inr,
                                                         const int* far_cnt, const int* close_cnt,
                                                         const int* nbonds, ForceOut O, SpecialTasks Tk, int pairs,
                                                         unsigned int* status)
{
  pdl_enter();
  lj_pairs_block<Real>(P, T, S, lcap, inr, far_cnt, close_cnt, nbonds, O, Tk, pairs, status,
                       (blockIdx.x * blockDim.x + threadIdx.x) / kLjGroup);
}

// Special LJ pairs, one thread per (atom, pair) task.
template <class Real, class TB>
__global__ void k_lj_special(const ReboParams* P, const TB* Tb, LJParams LP, BondList B, CijTable T, State S,
                             SpecialTasks Tk, unsigned int* status)
{
  pdl_enter();
  const int total = spc_total(Tk);
  ReboT<Real, TB> R{*P, *Tb, B, status};
  LJT<Real, TB> X{LP, R, T};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x)
    lj_special_task(X, S, Tk, t, status);
}

// Special LJ pairs, one thread per pair (both ends' records): the work item
// is the lower-index end's task; the partner's task of the same pair is found
// by a linear search of the partner's special list.  The loop runs whole
// warps (w0 is uniform over a warp) and the lanes meet again after the
// search, so the pair terms that follow run with the warp converged.
template <class Real, class TB>
__global__ void k_lj_special_pair(const ReboParams* P, const TB* Tb, LJParams LP, BondList B, CijTable T, State S,
                                  SpecialTasks Tk, unsigned int* status)
{
  pdl_enter();
  const long total = (long)min(Tk.ctr[0], (unsigned long long)Tk.task_cap);
  ReboT<Real, TB> R{*P, *Tb, B, status};
  LJT<Real, TB> X{LP, R, T};
  const int lane = threadIdx.x & 31;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long w0 = (long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); w0 < total; w0 += stride) {
    const long w = w0 + lane;
    const int t = w < total ? Tk.work[w] : -1;  // -1: none, or beyond the task capacity (already flagged)
    int t2 = -1;
    if (t >= 0) {
      const int2 ab = Tk.flat[t];
      int u0, u1;
      spc_range(Tk, ab.y, u0, u1);
      const int* pb = Tk.part + (long)ab.y * Tk.cap;
      for (int u = 0; u < u1 - u0; u++)
        if (pb[u] == ab.x) { t2 = u0 + u; break; }
      if (t2 < 0) atomicOr(status, ST_RECORD_OVERFLOW);
    }
    __syncwarp();
    if (t2 >= 0) lj_special_pair_task(X, S, Tk, t, t2, status);
  }
}

// The gather split over kGatherLanes lanes per atom: lane l takes the bond
// slots l, l + kGatherLanes, ... of both the bond-record gather and the LJ
// middle-bond gather (the same terms as gather_atom + mid_gather_atom); lane 0
// adds the atom's own gradients.  The lanes' sums are combined by a fixed
// butterfly, so every lane holds the same, deterministic total.
constexpr int kGatherLanes = 4;
__device__ V3 gather_lanes(const BondList& B, const ForceOut& O, const SpecialTasks& X, int a, int with_lj,
                           const double4* gextra, int l)
{
  V3 g = v3(0.0, 0.0, 0.0);
  if (l == 0) {
    const double4 g0 = O.gown[a];
    g = v3(g0.x, g0.y, g0.z);
    if (with_lj) {
      const double4 g1 = O.glj[a];
      g += v3(g1.x, g1.y, g1.z);
    }
    if (gextra) {
      const double4 g2 = gextra[a];
      g += v3(g2.x, g2.y, g2.z);
    }
  }
  const int nb = B.nb[a];
  for (int s = l; s < nb; s += kGatherLanes) {
    const int q = a * B.mb + s;
    const int k = B.bj[q];
    const int r = B.brev[q];
    if (r >= 0) {  // (a partner list truncated by an overflow is already flagged)
      const double* Ak = O.A + ((long)k * O.mb + r) * 3;
      g += v3(Ak[0], Ak[1], Ak[2]);
    }
    const double df = B.bd[q].x;
    if (df != 0.0) {
      double wa = 0.0;
      for (int t = 0; t < nb; t++) {
        if (t == s) continue;
        const int qt = a * B.mb + t;
        if (B.brev[qt] < 0) continue;
        wa += O.W[(long)B.bj[qt] * O.mb + B.brev[qt]];
      }
      double wm = 0.0;
      const int nbm = B.nb[k];
      for (int t = 0; t < nbm; t++) {
        const int qt = k * B.mb + t;
        const int cc = B.bj[qt];
        if (cc == a || B.brev[qt] < 0) continue;
        wm += O.W[(long)cc * O.mb + B.brev[qt]];
      }
      const double4 u = B.bu[q];
      g += v3(u.x, u.y, u.z) * (df * (wa + wm));
    }
    if (with_lj) {
      // middle-bond terms of the LJ special pairs (mid_gather_atom)
      int t0, t1;
      spc_range(X, k, t0, t1);
      for (int t = t0; t < t1; t++) {
        const int4 e = X.mid[t];
        if (!e.w || e.x != a) continue;
        const double4 u = B.bu[a * B.mb + e.y];
        g += v3(u.x, u.y, u.z) * X.midc[t];
      }
      const double4 ua = B.bu[q];
      const int nbk = B.nb[k];
      for (int qq = 0; qq < nbk; qq++) {
        const int lo = B.bj[k * B.mb + qq];
        int u0, u1;
        spc_range(X, lo, u0, u1);
        for (int t = u0; t < u1; t++) {
          const int4 e = X.mid[t];
          if (!e.w || e.x != k || e.z != a) continue;
          g += v3(ua.x, ua.y, ua.z) * X.midc[t];
        }
      }
    }
  }
#pragma unroll
  for (int o = kGatherLanes / 2; o > 0; o >>= 1) {
    g.x += __shfl_xor_sync(0xffffffffu, g.x, o);
    g.y += __shfl_xor_sync(0xffffffffu, g.y, o);
    g.z += __shfl_xor_sync(0xffffffffu, g.z, o);
  }
  return g;
}

__global__ void k_gather(BondList B, ForceOut O, int with_lj, SpecialTasks Tk, double4* grad, const double4* gm)
{
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = t / kGatherLanes, l = t % kGatherLanes;
  if (__all_sync(0xffffffffu, a >= B.n)) return;  // whole warps
  const int aa = a < B.n ? a : B.n - 1;
  const V3 g = gather_lanes(B, O, Tk, aa, with_lj, gm, l);
  if (a < B.n && l == 0) grad[a] = make_double4(g.x, g.y, g.z, 0.0);
}

// The gather and the end of a step in one pass (eq 2-4 and applyPBC): the
// gather reads bond records and unit vectors, never positions, so each atom's
// velocity, acceleration and wrap follow its own gradient at once (on the
// atom's first lane).
__global__ void k_gather_vv(BondList B, ForceOut O, int with_lj, SpecialTasks Tk, double4* grad, State S, StepDev P,
                            double* ekin, const double4* gm, unsigned int* status)
{
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = t / kGatherLanes, l = t % kGatherLanes;
  if (__all_sync(0xffffffffu, a >= B.n)) return;  // whole warps
  const int aa = a < B.n ? a : B.n - 1;
  const V3 g = gather_lanes(B, O, Tk, aa, with_lj, gm, l);
  if (a >= B.n || l != 0) return;
  grad[a] = make_double4(g.x, g.y, g.z, 0.0);
  if (P.ekin_pre) {
    const double4 v0 = S.vel[a];
    P.ekin_pre[a] = S.mass[a] * (v0.x * v0.x + v0.y * v0.y + v0.z * v0.z) / 2.0 / kAccConv;
  }
  verlet_vel_ext_atom(S, g, P, a, status);
  const double4 v = S.vel[a];
  ekin[a] = S.mass[a] * (v.x * v.x + v.y * v.y + v.z * v.z) / 2.0 / kAccConv;
}

// Bath temperature at the start of a step (SimLoop::actualTemperatureOfThermalBath,
// SimLoop.cxx:526-546): per system, the kinetic energy and count of the free
// atoms inside the bath.  Grid (blocks per system, systems); partials
// [system][block][2], summed in a fixed order by k_bath_final.
__global__ void k_bath_partial(State S, StepDev P, const int64_t* first, double* part)
{
  pdl_enter();
  __shared__ double se[kThreads], sn[kThreads];
  const int sy = blockIdx.y;
  const long b = first ? first[sy] : 0, e = first ? first[sy + 1] : S.n;
  double ek = 0.0, cnt = 0.0;
  for (long i = b + blockIdx.x * (long)blockDim.x + threadIdx.x; i < e; i += (long)gridDim.x * blockDim.x) {
    if (S.fixed && S.fixed[i]) continue;
    if (!in_bath(P, S, (int)i)) continue;
    const double4 v = S.vel[i];
    ek += S.mass[i] * (v.x * v.x + v.y * v.y + v.z * v.z) / 2.0 / kAccConv;
    cnt += 1.0;
  }
  se[threadIdx.x] = ek;
  sn[threadIdx.x] = cnt;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      se[threadIdx.x] += se[threadIdx.x + w];
      sn[threadIdx.x] += sn[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * ((long)sy * gridDim.x + blockIdx.x)] = se[0];
    part[2 * ((long)sy * gridDim.x + blockIdx.x) + 1] = sn[0];
  }
}
__global__ void k_bath_final(const double* part, int nblk_sys, int nsys, double* T)
{
  pdl_enter();
  const int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= nsys) return;
  double ek = 0.0, cnt = 0.0;
  for (int q = 0; q < nblk_sys; q++) {
    ek += part[2 * ((long)sy * nblk_sys + q)];
    cnt += part[2 * ((long)sy * nblk_sys + q) + 1];
  }
  T[sy] = cnt == 0.0 ? 0.0 : ek / (3.0 / 2.0 * 8.617343e-5 * cnt);  // kb in eV/K (mdtk/consts.cxx:32)
}

// End of a step with adaptive dt (SimLoop.cxx:405-416): the simulated time
// advances by the step's dt, then dt = 0.05 timeaccel / v_max clamped to
// [1e-5, 0.5] fs (0.5 fs without a moving atom).
__global__ void k_dt_update(int nsys, unsigned long long* vmax, double* dt, double* dt_prev, double* time,
                            double timeaccel, int* stop, double time_final)
{
  pdl_enter();
  const int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy >= nsys) return;
  if (stop && stop[sy]) {  // finished: time and dt stay as the last step left them
    vmax[sy] = 0ull;
    return;
  }
  const double vm = __longlong_as_double((long long)vmax[sy]);
  const double dt_max = 0.5, dt_min = 1e-5;
  double d = vm != 0.0 ? 0.05 * timeaccel / vm : dt_max;
  if (d > dt_max) d = dt_max;
  if (d < dt_min) d = dt_min;
  time[sy] += dt[sy];
  dt_prev[sy] = dt[sy];
  dt[sy] = d;
  vmax[sy] = 0ull;
  // the loop runs while simTime < simTimeFinal (SimLoop.cxx:252)
  if (stop && !(time[sy] < time_final)) stop[sy] = 1;
}

// Systems already at or past simTimeFinal take no step.
__global__ void k_stop_init(int nsys, const double* time, int* stop, double time_final)
{
  pdl_enter();
  const int sy = blockIdx.x * blockDim.x + threadIdx.x;
  if (sy < nsys) stop[sy] = !(time[sy] < time_final);
}

// Host-step layout conversion: io = [pos (n*3) | vel (n*3)] in the caller's
// units; the species in pos.w is kept.
__global__ void k_state_unpack(State S, const double* io, double ul, double uv)
{
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const double* p = io + 3 * (long)i;
  const double* v = io + 3 * ((long)S.n + i);
  S.pos[i] = make_double4(p[0] * ul, p[1] * ul, p[2] * ul, S.pos[i].w);
  S.vel[i] = make_double4(v[0] * uv, v[1] * uv, v[2] * uv, 0.0);
}
__global__ void k_state_pack(State S, double* io, double ul, double uv)
{
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const double4 p = S.pos[i], v = S.vel[i];
  double* po = io + 3 * (long)i;
  double* vo = io + 3 * ((long)S.n + i);
  po[0] = p.x / ul; po[1] = p.y / ul; po[2] = p.z / ul;
  vo[0] = v.x / uv; vo[1] = v.y / uv; vo[2] = v.z / uv;
}

// initial accelerations (SimLoop.cxx:305-321)
// (and Atom::an_no_tb, Check::energyTransferredFromBath = 0, SimLoop.cxx:1137)
__global__ void k_init_acc(State S, const double4* grad, double4* acc_ntb, double* eb)
{
  pdl_enter();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  if (eb) eb[i] = 0.0;
  if (S.fixed && S.fixed[i]) return;
  double m = S.mass[i];
  double4 g = grad[i];
  S.acc[i] = make_double4(-g.x / m * kAccConv, -g.y / m * kAccConv, -g.z / m * kAccConv, 0.0);
  if (acc_ntb) acc_ntb[i] = S.acc[i];
}

__global__ void k_ekin(State S, double* ekin)
{
  pdl_enter();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  double4 v = S.vel[i];
  ekin[i] = S.mass[i] * (v.x * v.x + v.y * v.y + v.z * v.z) / 2.0 / kAccConv;
}

// Deterministic sums of up to 4 per-atom arrays: fixed grid, fixed order.
struct RedArgs {
  const double* a[5];
  int slot[5];  // output slot of each array (the metal energies join another slot or take their own)
  int narr, nout, n;
};
__global__ void k_reduce_partial(RedArgs R, double* part)
{
  pdl_enter();
  __shared__ double sh[kThreads];
  int which = blockIdx.y;
  const double* x = R.a[which];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R.n; i += gridDim.x * blockDim.x) s += x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[which * gridDim.x + blockIdx.x] = sh[0];
}
// out[w] = sum of the partials of the arrays of slot w (in array order)
__global__ void k_reduce_final(const double* part, int nparts, RedArgs R, double* out, int slot_stride, int slot,
                               unsigned int* status)
{
  pdl_enter();
  int w = threadIdx.x;
  if (w >= R.nout) return;
  double s = 0.0;
  for (int k = 0; k < R.narr; k++) {
    if (R.slot[k] != w) continue;
    double t = 0.0;
    for (int q = 0; q < nparts; q++) t += part[k * nparts + q];
    s = (k == w) ? t : s + t;
  }
  out[slot * slot_stride + w] = s;
  if (!isfinite(s)) atomicOr(status, ST_NONFINITE);
}

// Per-system energy sums of a batched context: one block per system; each
// thread sums a strided share of the system's atoms, then a fixed tree
// (deterministic).  out[4 s + {0,1,2,3}] = REBO, LJ, torsion, kinetic.
__global__ void k_sys_energy(const int64_t* first, int64_t n, const double* er, const double* el, const double* et,
                             const double* ek, const double* em, double* out, unsigned int* status)
{
  pdl_enter();
  __shared__ double sh[4][kThreads];
  const int sy = blockIdx.x;
  // a single-system context has no offsets array: its one system is [0, n)
  const int64_t b = first ? first[sy] : 0, e = first ? first[sy + 1] : n;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
    acc[0] += er[i];
    acc[1] += el[i];
    acc[2] += et[i];
    if (em) acc[2] += em[i];  // metal and ion energies join the torsion slot in the totals
    acc[3] += ek[i];
  }
  for (int q = 0; q < 4; q++) sh[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int q = 0; q < 4; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 4) {
    const double v = sh[threadIdx.x][0];
    out[4 * sy + threadIdx.x] = v;
    if (!isfinite(v)) atomicOr(status, ST_NONFINITE);
  }
}

__global__ void k_finite(const double4* g, int n, unsigned int* status)
{
  pdl_enter();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 v = g[i];
  if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) atomicOr(status, ST_NONFINITE);
}

// FMA-throughput probes for the roofline denominators (no peak for the FP64
// and FP32 CUDA-core pipes is recorded elsewhere): each thread runs 8
// independent dependent-FMA chains, so the pipes stay full.
__global__ void k_peak_fp64(double* out, int iters, double a, double b)
{
  double x[8];
  for (int q = 0; q < 8; q++) x[q] = threadIdx.x * 1e-9 + q;
  for (int it = 0; it < iters; it++)
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = fma(x[q], a, b);
  double s = 0;
  for (int q = 0; q < 8; q++) s += x[q];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
__global__ void k_peak_fp32(float* out, int iters, float a, float b)
{
  float x[8];
  for (int q = 0; q < 8; q++) x[q] = threadIdx.x * 1e-6f + q;
  for (int it = 0; it < iters; it++)
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = fmaf(x[q], a, b);
  float s = 0;
  for (int q = 0; q < 8; q++) s += x[q];
  if (s == 12345.678f) out[0] = s;
}

template <class T>
T* dalloc(size_t count)
{
  void* p = nullptr;
  if (count == 0) count = 1;
  if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
  return (T*)p;
}

}  // namespace

// ---------------------------------------------------------------- context

namespace {
struct AdjWs;  // adjoint-path buffers (mdg_adjoint.cuh)
}

struct mdg_ctx {
  mdg_params prm;
  ReboParams rp;
  TorsParams tp;
  LJParams ljp;
  ReboTables* d_tables = nullptr;
  ReboTables32* d_tables32 = nullptr;  // FP32-mixed path only
  ReboParams* d_rp = nullptr;
  BrennerTables* d_btables = nullptr;
  BrennerParams* d_bp = nullptr;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  int64_t launches = 0;

  int n = 0;
  Box box;
  // batched context: nsys independent systems, atoms [first[s], first[s+1])
  int nsys = 1;
  std::vector<int64_t> h_first;
  std::vector<Box> h_boxes;
  std::vector<int> h_sys;
  int* d_sys = nullptr;
  Box* d_boxes = nullptr;
  int64_t* d_first = nullptr;
  int4* d_snc[3] = {nullptr, nullptr, nullptr};
  double4* d_slo[3] = {nullptr, nullptr, nullptr};
  double4* d_scs[3] = {nullptr, nullptr, nullptr};
  double unit_len = 1.0, unit_vel = 1.0, unit_e = 1.0, unit_grad = 1.0;

  // state
  double4 *pos = nullptr, *vel = nullptr, *acc = nullptr, *grad = nullptr;
  int4* image = nullptr;
  unsigned char* fixed = nullptr;
  double* mass = nullptr;
  bool acc_valid = false;

  // lists: 0 = REBO range, 1 = LJ range
  NList nl[3];             // 0 REBO range, 1 AIREBO LJ range, 2 metal and ion pairs
  NList ljt;               // the LJ list's near sublist (entries within R2 + kLjNearSkin; flag slot 3)
  Grid grid[3];
  int* d_need = nullptr;   // [4]: lists 0-2, the LJ near sublist
  int* d_force = nullptr;  // [4]
  unsigned int* d_disp_done = nullptr;  // blocks of step_start finished (back to 0 by the last)
  double* d_part = nullptr;
  double rcut[3] = {0, 0, 0};
  bool has_list[3] = {false, false, false};
  // metal and ion potentials (FBZL, FLJ, Ackland)
  MetalParams* d_metal = nullptr;
  double* d_fp = nullptr;     // [n] dF/drho of the embedding
  double* d_em = nullptr;     // [n] metal and ion energies per atom
  double4* d_gm = nullptr;    // [n] their gradient

  // bonds
  int mb = 16;
  BondBuild bb;
  ForceOut fo;
  double* e_kin = nullptr;
  double* d_red_part = nullptr;
  double* d_energy = nullptr;   // [4] rebo, lj, tors, kin of the last evaluation
  double* d_elog = nullptr;     // per-step energy log [cap * 4]
  double* h_elog = nullptr;     // its pinned host copy
  int64_t h_elog_cap = 0;
  int64_t elog_cap = 0;

  CijTable cij;
  SpecialTasks spc;
  BondTasks bt;
  int rebo_task_blocks = 0;   // resident capacity of the REBO task kernel (blocks)
  int rebo_grid = 0;          // blocks it is launched with (the autotuner's choice; 0 = capacity)
  // REBO tasks on a second stream, concurrent with the LJ chain (which does
  // not read their records until the reduction): fork/join by events, also
  // inside a captured step
  // and the LJ distance filter on a third, concurrently with the bond and
  // connectivity kernels
  bool overlap = false;
  cudaStream_t side = nullptr, side2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fork2 = nullptr, ev_join2 = nullptr;
  int* lj_inr = nullptr;      // [n * LJ list cap] in-range LJ partners of the step: far from the front, close from the back
  int* lj_inr_cnt = nullptr;  // [2n] far counts, close counts
  bool tuned = false;        // the autotuner ran for this system
  float tune_ms[3] = {0, 0, 0};  // its timings of one force evaluation per task mode

  unsigned int* d_status = nullptr;
  int special_blocks = 0;
  int warp_blocks = 0;        // resident blocks of the warp-per-atom LJ list kernels (grid-stride over atoms)

  // one MD step captured as a CUDA graph (replayed when no per-step energies are wanted)
  cudaGraphExec_t step_graph = nullptr;
  double graph_dt = 0.0;
  int graph_cfg = -1;           // step_cfg the graph was captured with
  bool pdl = true;              // programmatic dependent launches (mdg_set_dependent_launch)
  int step_cfg = 0;             // bumped when the thermal bath or the dt mode changes

  // thermal bath (SimLoop::thermalBath*, SimLoop.hpp:96-191) and adaptive dt
  // (SimLoop.cxx:405-416); internal units (K, 1/fs, Angstrom)
  int tb_geom = 0;
  double tb_T0 = 0.0, tb_gamma = 1e13 * 1e-15;  // ThermalBathCommon defaults (1e13 / s)
  double tb_gp[5] = {0, 0, 0, 0, 0};
  unsigned char* d_tb_apply = nullptr;  // [n] Atom::apply_ThermalBath (null: every atom)
  double* d_tb_T = nullptr;             // [nsys] bath temperature at the step start
  double* d_tb_part = nullptr;          // [2 * kBathBlocks (+ nsys)] partial sums
  bool adaptive = false;
  double timeaccel = 1.0;               // SimLoop::timeaccel (1 Angstrom)
  double dt0 = 0.5;                     // starting time step of the adaptive mode (fs)
  double* d_dt = nullptr;               // [nsys] current time step (adaptive dt)
  double* d_time = nullptr;             // [nsys] simulated time since the mode was set
  unsigned long long* d_vmax = nullptr; // [nsys] bits of the step's largest |v|
  double* d_dt_prev = nullptr;          // [nsys] the step just taken (SimLoop::dt_prev)
  cudaStream_t graph_stream = nullptr;
  int graph_launches = 0;

  // SimLoop bookkeeping kept for the checkpoint and trajectory files
  // (SimLoopSaver, SimLoop::saveToStreamXVA): the iteration counter, the time
  // of fixed-dt steps (adaptive steps keep theirs on the device), the Check
  // record's inputs
  uint64_t iteration = 0;               // SimLoop::iteration
  double time_s = 0.0;                  // SimLoop::simTime (s) of fixed-dt steps
  double dt_s = 1e-20, dt_prev_s = 1e-20;  // SimLoop::dt, dt_prev (s) of fixed-dt steps
  double time_final_s = 4e-12;          // SimLoop::simTimeFinal (SimLoop.cxx:48)
  bool stepped = false;                 // a step ran since the state was set or loaded
  bool e0_dev = false;                  // Check::initialEnergy is d_e0 (else chk_e0)
  double chk_e0 = 1.0, chk_eb0 = 0.0;   // Check::initialEnergy, energyTransferredFromBath (erg) of a load
  bool chk_loaded = false;              // a loaded Check record stands until the next step
  double chk_net[3] = {0, 0, 0}, chk_cur = 1.0, chk_T = 0.0;
  double run_t0 = 0.0;                  // wall clock at the first step (SimLoop::CPUTimeUsed_total's start)
  bool stop_final = false;              // adaptive systems stop at simTimeFinal
  int* d_stop = nullptr;                // [nsys] a system reached simTimeFinal
  struct SnapState* snap = nullptr;     // device SnapshotList capture (mdtrajsim)
  double* d_e0 = nullptr;               // [nsys * 4] rebo, lj, tors, kin at the first step
  double* d_ekin_pre = nullptr;         // [n] M V_n^2 / 2 before the last kick
  double4* acc_ntb = nullptr;           // [n] Atom::an_no_tb (with a bath)
  double* d_eb = nullptr;               // [n] energy the bath gave each atom (with a bath)
  std::vector<int32_t> h_z;             // atomic numbers as loaded
  std::vector<unsigned char> h_fixed, h_tb_apply, h_tags;  // Atom::fixed, apply_ThermalBath, tag bits
  struct IoState* io = nullptr;         // snapshot slots, writer thread, output schedule

  // profiling: event pairs bracketing each launch while enabled
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<std::string, size_t>> prof_recs;  // name, index of the start event
  // host staging for mdg_step_host
  double4* h_stage = nullptr;
  double* d_io = nullptr;       // [6 n] the host step's pos and vel in the caller's [n*3] layout
  std::vector<int> h_type;
  AdjWs* adj = nullptr;       // adjoint path, allocated on first use

  State S() const
  {
    State s;
    s.n = n;
    s.box = box;
    s.sys = nsys > 1 ? d_sys : nullptr;
    s.boxes = nsys > 1 ? d_boxes : nullptr;
    s.pos = pos;
    s.vel = vel;
    s.acc = acc;
    s.image = image;
    s.fixed = fixed;
    s.mass = mass;
    return s;
  }
  BondList BL() const
  {
    BondList b;
    b.n = n;
    b.mb = mb;
    b.nb = bb.nb;
    b.bj = bb.bj;
    b.brev = bb.brev;
    b.brv = bb.brv;
    b.bu = bb.bu;
    b.bd = bb.bd;
    b.nco = bb.nco;
    return b;
  }
};

namespace {

cudaEvent_t pool_event(mdg_ctx* c)
{
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[c->ev_used++];
}

void prof_begin(mdg_ctx* c, const char* name)
{
  if (!c->prof) return;
  size_t i = c->ev_used;
  cudaEventRecord(pool_event(c), c->stream);
  c->prof_recs.push_back(std::make_pair(std::string(name), i));
}

void prof_end(mdg_ctx* c)
{
  if (!c->prof) return;
  cudaEventRecord(pool_event(c), c->stream);
}

int launch_check(mdg_ctx* c)
{
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return MDG_OK;
}

int status_to_code(unsigned int st, std::string& msg)
{
  if (st == 0) return MDG_OK;
  msg = "device status:";
  int code = MDG_OK;
  auto add = [&](unsigned int bit, int c, const char* m) {
    if (st & bit) { msg += std::string(" ") + m; if (code == MDG_OK) code = c; }
  };
  add(ST_NONFINITE, MDG_ERR_NONFINITE, "non-finite energy or force;");
  add(ST_NL_OVERFLOW, MDG_ERR_NL_OVERFLOW, "Verlet list capacity exceeded;");
  add(ST_BOND_OVERFLOW, MDG_ERR_BOND_OVERFLOW, "bond capacity exceeded;");
  add(ST_COS_RANGE, MDG_ERR_COS_RANGE, "cos(theta) out of range;");
  add(ST_N_NEGATIVE, MDG_ERR_N_NEGATIVE, "negative coordination;");
  add(ST_SPLINE_DOMAIN, MDG_ERR_SPLINE_DOMAIN, "spline argument out of domain;");
  add(ST_CIJ_OVERFLOW, MDG_ERR_CAPACITY, "connectivity table capacity exceeded;");
  add(ST_RECORD_OVERFLOW, MDG_ERR_CAPACITY, "bond or connectivity record capacity exceeded;");
  add(ST_CELL_OVERFLOW, MDG_ERR_CAPACITY, "cell grid capacity exceeded;");
  add(ST_SNAP_OVERFLOW, MDG_ERR_CAPACITY, "snapshot list capacity exceeded;");
  return code;
}

void adj_free(mdg_ctx* c);
void io_release(mdg_ctx* c);
void io_free(mdg_ctx* c);
void snap_free(mdg_ctx* c);
int snap_capture(mdg_ctx* c);

void free_system(mdg_ctx* c)
{
  io_release(c);
  adj_free(c);
  {
    void* st[] = {c->d_tb_apply, c->d_tb_T, c->d_tb_part, c->d_dt, c->d_time, c->d_vmax, c->d_dt_prev,
                  c->d_e0, c->d_ekin_pre, c->acc_ntb, c->d_eb, c->d_stop};
    for (void* p : st)
      if (p) cudaFree(p);
    c->d_tb_apply = nullptr;
    c->d_tb_T = c->d_tb_part = c->d_dt = c->d_time = c->d_dt_prev = nullptr;
    c->d_e0 = c->d_ekin_pre = c->d_eb = nullptr;
    c->acc_ntb = nullptr;
    c->d_stop = nullptr;
    snap_free(c);
    c->d_vmax = nullptr;
    c->h_z.clear();
    c->h_fixed.clear();
    c->h_tb_apply.clear();
    c->h_tags.clear();
  }
  void* ptrs[] = {c->pos, c->vel, c->acc, c->grad, c->image, c->fixed, c->mass,
                  c->bb.nb, c->bb.bj, c->bb.brev, c->bb.brv, c->bb.bu, c->bb.bd, c->bb.nco,
                  c->fo.A, c->fo.W, c->fo.gown, c->fo.glj, c->fo.e_rebo, c->fo.e_tors, c->fo.e_lj,
                  c->e_kin, c->d_part, c->d_red_part, c->d_elog};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int l = 0; l < 3; l++) {
    void* q[] = {c->nl[l].cnt, c->nl[l].list, c->nl[l].pos0, c->grid[l].ccount, c->grid[l].cstart,
                 c->grid[l].ccursor, c->grid[l].catoms};
    for (void* p : q)
      if (p) cudaFree(p);
    std::memset(&c->nl[l], 0, sizeof(NList));
    std::memset(&c->grid[l], 0, sizeof(Grid));
    c->has_list[l] = false;
  }
  void* lq[] = {c->cij.cnt, c->cij.ent, c->cij.w, c->cij.mask, c->spc.cnt, c->spc.part, c->spc.off,
                c->spc.flat, c->spc.trec, c->spc.rec, c->spc.mid, c->spc.midc, c->spc.work,
                c->spc.ctr, c->lj_inr, c->lj_inr_cnt, c->ljt.cnt, c->ljt.list, c->ljt.pos0};
  std::memset(&c->ljt, 0, sizeof(NList));
  c->lj_inr = nullptr;
  c->lj_inr_cnt = nullptr;
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
  for (void* p : lq)
    if (p) cudaFree(p);
  std::memset(&c->cij, 0, sizeof(c->cij));
  std::memset(&c->spc, 0, sizeof(c->spc));
  void* sq[] = {c->d_sys, c->d_boxes, c->d_first, c->d_snc[0], c->d_snc[1], c->d_snc[2], c->d_slo[0], c->d_slo[1],
                c->d_slo[2], c->d_scs[0], c->d_scs[1], c->d_scs[2], c->d_fp, c->d_em, c->d_gm};
  for (void* p : sq)
    if (p) cudaFree(p);
  c->d_sys = nullptr;
  c->d_boxes = nullptr;
  c->d_first = nullptr;
  for (int l = 0; l < 3; l++) { c->d_snc[l] = nullptr; c->d_slo[l] = nullptr; c->d_scs[l] = nullptr; }
  c->d_fp = c->d_em = nullptr;
  c->d_gm = nullptr;
  c->nsys = 1;
  c->tuned = false;
  c->overlap = false;
  c->rebo_grid = 0;
  c->h_first.clear();
  c->h_boxes.clear();
  c->h_sys.clear();
  void* bq[] = {c->bt.q, c->bt.ctr, c->bt.rbase, c->bt.nrec, c->bt.rec};
  for (void* p : bq)
    if (p) cudaFree(p);
  std::memset(&c->bt, 0, sizeof(c->bt));
  if (c->h_stage) cudaFreeHost(c->h_stage);
  c->h_stage = nullptr;
  if (c->h_elog) cudaFreeHost(c->h_elog);
  c->h_elog = nullptr;
  c->h_elog_cap = 0;
  if (c->d_io) cudaFree(c->d_io);
  c->d_io = nullptr;
  c->pos = c->vel = c->acc = c->grad = nullptr;
  c->image = nullptr;
  c->fixed = nullptr;
  c->mass = nullptr;
  std::memset(&c->bb, 0, sizeof(c->bb));
  std::memset(&c->fo, 0, sizeof(c->fo));
  c->e_kin = c->d_part = c->d_red_part = c->d_elog = nullptr;
  c->elog_cap = 0;
  c->n = 0;
}

// Cell grid for a list of the given range over the current box.
int setup_grid(mdg_ctx* c, int l, const std::vector<double>& hpos)
{
  Grid& g = c->grid[l];
  double range = std::sqrt(c->nl[l].range2);
  g.brute = 0;
  for (int ax = 0; ax < 3; ax++) {
    if (c->box.pbc[ax]) {
      int nc = (int)std::floor(c->box.L[ax] / range);
      if (nc < 3) { g.brute = 1; nc = 1; }
      g.nc[ax] = nc;
      g.lo[ax] = 0.0;
      g.cs[ax] = c->box.L[ax] / nc;
    } else {
      double lo = 1e300, hi = -1e300;
      for (int i = 0; i < c->n; i++) {
        lo = std::fmin(lo, hpos[3 * i + ax]);
        hi = std::fmax(hi, hpos[3 * i + ax]);
      }
      lo -= 2 * range;
      hi += 2 * range;
      int nc = (int)std::floor((hi - lo) / range);
      if (nc < 1) nc = 1;
      if (nc > 1024) nc = 1024;
      g.nc[ax] = nc;
      g.lo[ax] = lo;
      g.cs[ax] = (hi - lo) / nc;
    }
  }
  if (g.brute) { g.nc[0] = g.nc[1] = g.nc[2] = 1; }
  long nc = (long)g.nc[0] * g.nc[1] * g.nc[2];
  if (nc > (1L << 26)) return fail(MDG_ERR_ARG, "cell grid too large");
  g.ncell = (int)nc;
  g.ccount = dalloc<int>(nc);
  g.cstart = dalloc<int>(nc + 1);
  g.ccursor = dalloc<int>(nc);
  g.catoms = dalloc<int>(c->n);
  if (!g.ccount || !g.cstart || !g.ccursor || !g.catoms) return fail(MDG_ERR_CUDA, "cudaMalloc (cell grid)");
  // counts and cursors start at zero; each build's sort returns them there
  CK(cudaMemset(g.ccount, 0, (size_t)nc * sizeof(int)));
  CK(cudaMemset(g.ccursor, 0, (size_t)nc * sizeof(int)));
  return MDG_OK;
}

// One cell grid per system of a batched context, laid out one after another
// (non-periodic axes span the system's atoms at set-up plus two ranges, as
// in the single-system grid; a periodic axis may have 1 or 2 cells).
int setup_grid_batch(mdg_ctx* c, int l, const std::vector<double>& hpos)
{
  Grid& g = c->grid[l];
  const double range = std::sqrt(c->nl[l].range2);
  g.brute = 0;
  g.nc[0] = g.nc[1] = g.nc[2] = 1;
  std::vector<int4> snc(c->nsys);
  std::vector<double4> slo(c->nsys), scs(c->nsys);
  long total = 0;
  for (int sy = 0; sy < c->nsys; sy++) {
    const Box& b = c->h_boxes[sy];
    int nc[3];
    double lo[3], cs[3];
    for (int ax = 0; ax < 3; ax++) {
      if (b.pbc[ax]) {
        nc[ax] = std::max(1, (int)std::floor(b.L[ax] / range));
        lo[ax] = 0.0;
        cs[ax] = b.L[ax] / nc[ax];
      } else {
        double mn = 1e300, mx = -1e300;
        for (int64_t i = c->h_first[sy]; i < c->h_first[sy + 1]; i++) {
          mn = std::fmin(mn, hpos[3 * i + ax]);
          mx = std::fmax(mx, hpos[3 * i + ax]);
        }
        mn -= 2 * range;
        mx += 2 * range;
        nc[ax] = std::min(1024, std::max(1, (int)std::floor((mx - mn) / range)));
        lo[ax] = mn;
        cs[ax] = (mx - mn) / nc[ax];
      }
    }
    snc[sy] = make_int4(nc[0], nc[1], nc[2], (int)total);
    slo[sy] = make_double4(lo[0], lo[1], lo[2], 0.0);
    scs[sy] = make_double4(cs[0], cs[1], cs[2], 0.0);
    total += (long)nc[0] * nc[1] * nc[2];
    if (total > (1L << 26)) return fail(MDG_ERR_ARG, "cell grids too large");
  }
  g.ncell = (int)total;
  g.ccount = dalloc<int>(total);
  g.cstart = dalloc<int>(total + 1);
  g.ccursor = dalloc<int>(total);
  g.catoms = dalloc<int>(c->n);
  c->d_snc[l] = dalloc<int4>(c->nsys);
  c->d_slo[l] = dalloc<double4>(c->nsys);
  c->d_scs[l] = dalloc<double4>(c->nsys);
  if (!g.ccount || !g.cstart || !g.ccursor || !g.catoms || !c->d_snc[l] || !c->d_slo[l] || !c->d_scs[l])
    return fail(MDG_ERR_CUDA, "cudaMalloc (cell grids)");
  CK(cudaMemset(g.ccount, 0, (size_t)total * sizeof(int)));
  CK(cudaMemset(g.ccursor, 0, (size_t)total * sizeof(int)));
  CK(cudaMemcpy(c->d_snc[l], snc.data(), c->nsys * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_slo[l], slo.data(), c->nsys * sizeof(double4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_scs[l], scs.data(), c->nsys * sizeof(double4), cudaMemcpyHostToDevice));
  g.snc = c->d_snc[l];
  g.slo = c->d_slo[l];
  g.scs = c->d_scs[l];
  return MDG_OK;
}

// Every launch goes through LAUNCH: it counts the launch and, when
// profiling is on, brackets it with CUDA events on the launch stream.
void prof_begin(mdg_ctx* c, const char* name);
void prof_end(mdg_ctx* c);
// With pdl set, the launch carries the programmatic stream-serialisation
// attribute: the kernel's blocks may be scheduled while the grid before it
// drains, and wait in pdl_enter() (their first statement) for its completion.
template <typename... P, typename... A>
inline void launch_kernel(bool pdl, cudaStream_t st, void (*k)(P...), dim3 grid, dim3 block, A&&... args)
{
  cudaLaunchAttribute at;
  at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at.val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = &at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}
#define LAUNCH(c, NAME, KERNEL, GRID, BLOCK, ...)                           \
  do {                                                                      \
    prof_begin(c, NAME);                                                    \
    launch_kernel((c)->pdl, (c)->stream, KERNEL, GRID, BLOCK, __VA_ARGS__); \
    prof_end(c);                                                            \
    (c)->launches++;                                                        \
  } while (0)
// The same on another stream (never while profiling: the events are on c->stream).
#define LAUNCH_ON(c, STREAM, NAME, KERNEL, GRID, BLOCK, ...)               \
  do {                                                                      \
    prof_begin(c, NAME);                                                    \
    launch_kernel((c)->pdl, (STREAM), KERNEL, GRID, BLOCK, __VA_ARGS__);    \
    prof_end(c);                                                            \
    (c)->launches++;                                                        \
  } while (0)

// The displacement partials of both lists (after the step's position update
// when a step is given; before it, the bath temperature) in one pass over
// the atoms.
constexpr int kDispParts = 592;  // 4 blocks per SM of a B200: at most one atom per thread on the liquid
constexpr int kMetalListCap = 320;  // metal / ion list partners per atom (fcc Cu holds ~180 within 7.92 A)
constexpr int kBathBlocks = 120;
int step_start(mdg_ctx* c, const StepDev* step)
{
  State S = c->S();
  const int mask = (c->has_list[0] ? 1 : 0) | (c->has_list[1] ? 2 | 8 : 0) | (c->has_list[2] ? 4 : 0);
  if (step && step->tb_geom) {
    const int bps = std::max(1, kBathBlocks / c->nsys);
    LAUNCH(c, "bath_temp_partial", k_bath_partial, dim3(bps, c->nsys), kThreads, S, *step,
           c->nsys > 1 ? c->d_first : nullptr, c->d_tb_part);
    LAUNCH(c, "bath_temp_final", k_bath_final, nblk(c->nsys), kThreads, c->d_tb_part, bps, c->nsys, c->d_tb_T);
  }
  StepDev none;
  std::memset(&none, 0, sizeof(none));
  LAUNCH(c, step ? "verlet_pos_disp" : "nl_disp", k_step_start, kDispParts, kThreads, S,
         step ? *step : none, step ? 1 : 0, c->nl[0], c->nl[1], c->nl[2], c->ljt, mask, c->d_part, c->d_need, c->d_force,
         c->d_disp_done);
  return MDG_OK;
}

// Cell-list rebuild of list l on stream st when step_start's flag for it is
// set (each kernel returns at once otherwise); each list has its own flag
// and grid, so the lists can be rebuilt on different streams.
int rebuild_list(mdg_ctx* c, int l, cudaStream_t st)
{
  if (!c->has_list[l]) return MDG_OK;
  State S = c->S();
  NList& L = c->nl[l];
  Grid& g = c->grid[l];
  int* need = c->d_need + l;
  if (!g.brute) {
    LAUNCH_ON(c, st, "nl_cell_count", k_cell_count, nblk(c->n), kThreads, S, g, need);
    LAUNCH_ON(c, st, "nl_cell_scan", k_cell_scan, 1, 1024, g, need);
    LAUNCH_ON(c, st, "nl_cell_fill", k_cell_fill, nblk(c->n), kThreads, S, g, need);
    LAUNCH_ON(c, st, "nl_cell_sort", k_cell_sort, nblk(g.ncell), kThreads, g, need);
  }
  LAUNCH_ON(c, st, l == 0 ? "nl_build_rebo" : (l == 1 ? "nl_build_lj" : "nl_build_metal"), k_nl_build, nblk(c->n),
            kThreads, S, g, L, need, c->d_status);
  if (l == 1)
    LAUNCH_ON(c, st, "nl_build_lj_near", k_lj_near, std::min(nblk(c->n * 32), c->warp_blocks), kThreads, c->ljp, S,
              L, c->ljt, c->d_need, c->d_status);
  return MDG_OK;
}

int rebuild_lists(mdg_ctx* c, const StepDev* step = nullptr)
{
  int rc = step_start(c, step);
  if (!rc) rc = rebuild_list(c, 0, c->stream);
  if (!rc) rc = rebuild_list(c, 1, c->stream);
  if (!rc) rc = rebuild_list(c, 2, c->stream);
  if (rc) return rc;
  return launch_check(c);
}

// One force evaluation at the current positions; leaves dE/dx in c->grad and
// per-atom energies in c->fo.  With a step, the evaluation is the body of a
// velocity-Verlet step: the position update comes first (fused with the
// displacement check) and the velocity update last (fused with the gather),
// with the thermal bath and the adaptive dt when they are on.
int evaluate(mdg_ctx* c, const StepDev* step = nullptr)
{
  State S = c->S();
  const int pot = c->prm.potentials;
  const bool rebo = pot & MDG_POT_REBO, tors = pot & MDG_POT_ETORS, lj = pot & MDG_POT_AIREBO_LJ;
  const bool tasks = c->bt.ctr != nullptr;
  const bool ovl = tasks && lj && c->overlap && !c->prof && c->side;
  int rc;
  if (step && c->snap) {
    // CustomSimLoop::doBeforeIteration's snapshots (mdtrajsim/main.cpp:59-80)
    rc = snap_capture(c);
    if (rc) return rc;
  }
  if (ovl) {
    // the LJ list's check/rebuild and the in-range filter (positions and the
    // LJ list only) on the third stream, beside the REBO list and the bonds
    rc = step_start(c, step);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev_fork2, c->stream));
    CK(cudaStreamWaitEvent(c->side2, c->ev_fork2, 0));
    rc = rebuild_list(c, 1, c->side2);
    if (rc) return rc;
    LAUNCH_ON(c, c->side2, "lj_filter", k_lj_filter, std::min(nblk(c->n * 32), c->warp_blocks), kThreads, c->ljp, S,
              c->ljt, c->lj_inr, c->lj_inr_cnt, c->lj_inr_cnt + c->n);
    CK(cudaEventRecord(c->ev_join2, c->side2));
    rc = rebuild_list(c, 0, c->stream);
    if (rc) return rc;
  } else {
    rc = rebuild_lists(c, step);
    if (rc) return rc;
    if (lj)
      LAUNCH(c, "lj_filter", k_lj_filter, std::min(nblk(c->n * 32), c->warp_blocks), kThreads, c->ljp, S, c->ljt,
             c->lj_inr, c->lj_inr_cnt, c->lj_inr_cnt + c->n);
  }
  LAUNCH(c, "bonds", k_bonds, nblk(c->n), kThreads, S, c->nl[0], c->rp, c->bb, c->bt, c->d_status);
  BondList B = c->BL();
  const bool f32p = c->prm.precision == MDG_PREC_FP32_MIXED;
  cudaStream_t rs = c->stream;
  if (ovl) {
    // the reverse slots, the REBO bond tasks and the reduction of their
    // records on the second stream: none of the LJ kernels reads them
    CK(cudaEventRecord(c->ev_fork, c->stream));
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    rs = c->side;
  }
  LAUNCH_ON(c, rs, "bonds_rev", k_brev, nblk(c->n), kThreads, c->bb, c->bt, c->d_status);
  if (tasks) {
    const int ir = rebo ? 1 : 0, it = tors ? 1 : 0;
    const int grid = c->rebo_grid > 0 ? c->rebo_grid : c->rebo_task_blocks;
    if (f32p && c->bt.pairs == 2) {
      auto kern = k_rebo_split_task<f32, ReboTables32>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables32, B, c->tp, ir, it, c->bt,
                c->d_status);
    } else if (c->bt.pairs == 2) {
      auto kern = k_rebo_split_task<double, ReboTables>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables, B, c->tp, ir, it, c->bt,
                c->d_status);
    } else if (f32p && c->bt.pairs) {
      auto kern = k_rebo_pair_task<f32, ReboTables32>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables32, B, c->tp, ir, it, c->bt,
                c->d_status);
    } else if (f32p) {
      auto kern = k_rebo_task<f32, ReboTables32>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables32, B, c->tp, ir, it, c->bt,
                c->d_status);
    } else if (c->bt.pairs) {
      auto kern = k_rebo_pair_task<double, ReboTables>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables, B, c->tp, ir, it, c->bt,
                c->d_status);
    } else {
      auto kern = k_rebo_task<double, ReboTables>;
      LAUNCH_ON(c, rs, "rebo_tors", kern, grid, kThreads, c->d_rp, c->d_tables, B, c->tp, ir, it, c->bt,
                c->d_status);
    }
  }
  else
    LAUNCH(c, "rebo_tors", k_rebo, nblk(c->n), kThreads, c->d_rp, c->d_tables, B, c->tp, rebo ? 1 : 0,
           tors ? 1 : 0, c->fo, c->d_status);
  if (ovl) {
    // the REBO half of the record sums; the LJ half adds to it after the join
    // (the same additions in the same order as one combined pass)
    LAUNCH_ON(c, rs, "bond_reduce", k_bond_reduce<kReduceLanes>, nblk(c->n * kReduceLanes), kThreads, B, c->bt, 1,
              c->spc, 0, c->fo);
    CK(cudaEventRecord(c->ev_join, c->side));
  }
  if (pot & MDG_POT_BRENNER)
    LAUNCH(c, "brenner", k_brenner, nblk(c->n), kThreads, c->d_bp, c->d_btables, B, c->fo, c->d_status);
  if (lj) {
    LAUNCH(c, "cij_table", k_cij, nblk(c->n), kThreads, B, c->cij, c->spc.ctr, c->d_status);
    if (ovl) CK(cudaStreamWaitEvent(c->stream, c->ev_join2, 0));
    const int pairs = (c->bt.ctr && c->bt.pairs) ? 1 : 0;
    const int lgrid = nblk(c->n * kLjGroup, kLjThreads);
    if (f32p)
      LAUNCH(c, "lj_pairs", k_lj_pairs<f32>, lgrid, kLjThreads, c->ljp, c->cij, S, c->nl[1].cap, c->lj_inr,
             c->lj_inr_cnt, c->lj_inr_cnt + c->n, c->bb.nb, c->fo, c->spc, pairs, c->d_status);
    else
      LAUNCH(c, "lj_pairs", k_lj_pairs<double>, lgrid, kLjThreads, c->ljp, c->cij, S, c->nl[1].cap, c->lj_inr,
             c->lj_inr_cnt, c->lj_inr_cnt + c->n, c->bb.nb, c->fo, c->spc, pairs, c->d_status);
    // b*_ij of close non-bonded pairs stays FP64 in the mixed mode too: the
    // S(t_b) window (0.04 wide for C-C) multiplies an error of b* by up to
    // 1/0.04^2 in the pair force, beyond what float b* can carry.
    if (pairs) {
      auto kern = k_lj_special_pair<double, ReboTables>;
      LAUNCH(c, "lj_special", kern, c->special_blocks, kThreads, c->d_rp, c->d_tables, c->ljp, B, c->cij, S,
             c->spc, c->d_status);
    } else {
      auto kern = k_lj_special<double, ReboTables>;
      LAUNCH(c, "lj_special", kern, c->special_blocks, kThreads, c->d_rp, c->d_tables, c->ljp, B, c->cij, S,
             c->spc, c->d_status);
    }
  }
  if (ovl) {
    CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    LAUNCH(c, "lj_reduce", k_bond_reduce<kReduceLanes>, nblk(c->n * kReduceLanes), kThreads, B, c->bt, 0, c->spc,
           1, c->fo);
  } else if (tasks || lj) {
    LAUNCH(c, "bond_reduce", k_bond_reduce<kReduceLanes>, nblk(c->n * kReduceLanes), kThreads, B, c->bt,
           tasks ? 1 : 0, c->spc, lj ? 1 : 0, c->fo);
  }
  if (c->has_list[2]) {
    LAUNCH(c, "eam_density", k_eam_rho, nblk(c->n * 32), kThreads, S, c->nl[2], c->d_metal, c->d_fp, c->d_em,
           c->d_status);
    LAUNCH(c, "metal_pairs", k_metal_pairs, nblk(c->n * 32), kThreads, S, c->nl[2], c->d_metal, c->d_fp, c->d_em,
           c->d_gm);
  }
  if (step) {
    LAUNCH(c, "gather_verlet_vel", k_gather_vv, nblk(c->n * kGatherLanes), kThreads, B, c->fo, lj ? 1 : 0, c->spc, c->grad, S,
           *step, c->e_kin, c->d_gm, c->d_status);
    if (step->vmax)
      LAUNCH(c, "dt_update", k_dt_update, nblk(c->nsys), kThreads, c->nsys, c->d_vmax, c->d_dt, c->d_dt_prev, c->d_time,
             c->timeaccel, c->stop_final ? c->d_stop : nullptr, c->time_final_s / kFs);
  }
  else
    LAUNCH(c, "gather", k_gather, nblk(c->n * kGatherLanes), kThreads, B, c->fo, lj ? 1 : 0, c->spc, c->grad, c->d_gm);
  return launch_check(c);
}

// Sums of rebo, lj, tors (, kin) into slots 0-3; the metal and ion energies
// join the torsion slot, or take slot 3 of their own (split_metal, no kin).
int reduce_energies(mdg_ctx* c, double* out_dev, int slot_stride, int slot, bool with_kin, bool split_metal = false)
{
  RedArgs R;
  R.a[0] = c->fo.e_rebo;
  R.a[1] = c->fo.e_lj;
  R.a[2] = c->fo.e_tors;
  R.a[3] = c->e_kin;
  for (int k = 0; k < 5; k++) R.slot[k] = k;
  R.narr = with_kin ? 4 : 3;
  R.nout = R.narr;
  if (c->has_list[2]) {
    R.a[R.narr] = c->d_em;
    R.slot[R.narr] = split_metal && !with_kin ? 3 : 2;
    R.narr++;
    if (split_metal && !with_kin) R.nout = 4;
  }
  R.n = c->n;
  LAUNCH(c, "energy_partial", k_reduce_partial, dim3(kRedBlocks, R.narr), kThreads, R, c->d_red_part);
  LAUNCH(c, "energy_final", k_reduce_final, 1, 32, c->d_red_part, kRedBlocks, R, out_dev, slot_stride, slot,
         c->d_status);
  return launch_check(c);
}

int read_status(mdg_ctx* c)
{
  unsigned int st = 0;
  CK(cudaMemcpyAsync(&st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st) {
    unsigned int z = 0;
    CK(cudaMemcpy(c->d_status, &z, sizeof(z), cudaMemcpyHostToDevice));
    std::string msg;
    int code = status_to_code(st, msg);
    return fail(code, msg);
  }
  return MDG_OK;
}

}  // namespace

#include "mdg_adjoint.cuh"

// Lets the library's other translation units report through mdg_last_error().
__attribute__((visibility("hidden"))) void mdg_set_last_error_internal(const char* msg) { g_err = msg; }

// ---------------------------------------------------------------- C ABI

extern "C" {

void mdg_default_params(mdg_params* p)
{
  std::memset(p, 0, sizeof(*p));
  p->potentials = MDG_POT_REBO;
  p->brenner_set = 1;
  p->precision = MDG_PREC_FP64;
  p->units = MDG_UNITS_AEVFS;
  p->nl_skin = 0.3;
}

const char* mdg_last_error(void) { return g_err.c_str(); }

int mdg_create(const mdg_params* p, mdg_ctx** out)
{
  if (!p || !out) return fail(MDG_ERR_ARG, "null argument");
  *out = nullptr;
  if ((p->potentials & MDG_POT_AIREBO_LJ) && !(p->potentials & MDG_POT_REBO))
    return fail(MDG_ERR_ARG, "the AIREBO LJ term needs REBO (AIREBO_LJ.cxx:204-212)");
  if ((p->potentials & MDG_POT_BRENNER) && (p->potentials & (MDG_POT_REBO | MDG_POT_AIREBO_LJ)))
    return fail(MDG_ERR_ARG, "choose one bond-order potential: Brenner or REBO (the LJ term uses REBO)");
  if ((p->potentials & MDG_POT_BRENNER) && p->brenner_set != 1 && p->brenner_set != 2)
    return fail(MDG_ERR_ARG, "Brenner parameter set must be 1 or 2");
  if (!(p->potentials & (MDG_POT_REBO | MDG_POT_BRENNER | MDG_POT_ETORS)))
    return fail(MDG_ERR_ARG, "no potential selected");
  if (p->precision != MDG_PREC_FP64 && p->precision != MDG_PREC_FP32_MIXED)
    return fail(MDG_ERR_ARG, "unknown precision mode");
  if (p->precision == MDG_PREC_FP32_MIXED && (p->potentials & MDG_POT_BRENNER))
    return fail(MDG_ERR_ARG, "the FP32-mixed mode covers REBO, the LJ term and torsion; Brenner is FP64 only");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(MDG_ERR_CUDA, "no CUDA device");
  CK(cudaSetDevice(p->device));
  mdg_ctx* c = new mdg_ctx();
  c->prm = *p;
  if (c->prm.cap_bonds <= 0) c->prm.cap_bonds = 16;
  if (c->prm.bond_rec_avg <= 0) c->prm.bond_rec_avg = 256;
  if (c->prm.cap_rebo_list <= 0) c->prm.cap_rebo_list = 64;
  if (c->prm.cap_lj_list <= 0) c->prm.cap_lj_list = 512;
  if (c->prm.cap_cij <= 0) c->prm.cap_cij = 128;
  if (c->prm.cap_special <= 0) c->prm.cap_special = 64;
  if (c->prm.special_avg <= 0) c->prm.special_avg = 48;
  c->mb = c->prm.cap_bonds;
  fill_rebo_params(c->rp);
  fill_tors_params(c->tp);
  set_lj_params(c->ljp, c->prm.lj_cut_mode);
  if (p->units == MDG_UNITS_CGS) {
    c->unit_len = 1.0 / kAo;          // cm -> A
    c->unit_vel = kFs / kAo;          // cm/s -> A/fs
    c->unit_e = kEv;                  // eV -> erg
    c->unit_grad = kEv / kAo;         // eV/A -> erg/cm
  }
  ReboTables* h = new ReboTables();
  build_rebo_tables(h, nullptr);
  c->d_tables = dalloc<ReboTables>(1);
  c->d_rp = dalloc<ReboParams>(1);
  if (!c->d_tables || !c->d_rp) { delete h; mdg_destroy(c); return fail(MDG_ERR_CUDA, "cudaMalloc (tables)"); }
  cudaMemcpy(c->d_tables, h, sizeof(ReboTables), cudaMemcpyHostToDevice);
  cudaMemcpy(c->d_rp, &c->rp, sizeof(ReboParams), cudaMemcpyHostToDevice);
  if (p->precision == MDG_PREC_FP32_MIXED) {
    ReboTables32* h32 = new ReboTables32();
    build_rebo_tables32(*h, h32);
    c->d_tables32 = dalloc<ReboTables32>(1);
    if (!c->d_tables32) { delete h; delete h32; mdg_destroy(c); return fail(MDG_ERR_CUDA, "cudaMalloc (tables)"); }
    cudaMemcpy(c->d_tables32, h32, sizeof(ReboTables32), cudaMemcpyHostToDevice);
    delete h32;
  }
  delete h;
  if (p->potentials & MDG_POT_BRENNER) {
    BrennerTables* bt = new BrennerTables();
    BrennerParams bp;
    build_brenner_tables(p->brenner_set, bt, nullptr);
    set_brenner_params(bp, p->brenner_set);
    c->d_btables = dalloc<BrennerTables>(1);
    c->d_bp = dalloc<BrennerParams>(1);
    if (!c->d_btables || !c->d_bp) { delete bt; mdg_destroy(c); return fail(MDG_ERR_CUDA, "cudaMalloc (Brenner)"); }
    cudaMemcpy(c->d_btables, bt, sizeof(BrennerTables), cudaMemcpyHostToDevice);
    cudaMemcpy(c->d_bp, &bp, sizeof(BrennerParams), cudaMemcpyHostToDevice);
    delete bt;
  }
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->side2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork2, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join2, cudaEventDisableTiming) != cudaSuccess) {
    mdg_destroy(c);
    return fail(MDG_ERR_CUDA, "cudaStreamCreate / cudaEventCreate");
  }
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    mdg_destroy(c);
    return fail(MDG_ERR_CUDA, "cudaStreamCreate");
  }
  c->stream = c->own_stream;
  c->d_status = dalloc<unsigned int>(1);
  c->d_need = dalloc<int>(4);
  c->d_force = dalloc<int>(4);
  c->d_disp_done = dalloc<unsigned int>(1);
  c->d_energy = dalloc<double>(8);
  if (!c->d_status || !c->d_need || !c->d_force || !c->d_disp_done || !c->d_energy) {
    mdg_destroy(c);
    return fail(MDG_ERR_CUDA, "cudaMalloc");
  }
  cudaMemset(c->d_status, 0, sizeof(unsigned int));
  cudaMemset(c->d_need, 0, 4 * sizeof(int));
  cudaMemset(c->d_force, 0, 4 * sizeof(int));
  cudaMemset(c->d_disp_done, 0, sizeof(unsigned int));
  if (cudaGetLastError() != cudaSuccess) { mdg_destroy(c); return fail(MDG_ERR_CUDA, "setup copies failed"); }
  *out = c;
  return MDG_OK;
}

int mdg_destroy(mdg_ctx* c)
{
  if (!c) return MDG_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  io_free(c);
  free_system(c);
  void* ptrs[] = {c->d_tables, c->d_tables32, c->d_rp, c->d_btables, c->d_bp, c->d_status, c->d_need, c->d_force, c->d_energy,
                  c->d_metal, c->d_disp_done};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->ev_fork2) cudaEventDestroy(c->ev_fork2);
  if (c->ev_join2) cudaEventDestroy(c->ev_join2);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->side2) cudaStreamDestroy(c->side2);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return MDG_OK;
}

int mdg_set_stream(mdg_ctx* c, void* stream)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return MDG_OK;
}

// Per-atom bath bookkeeping (Atom::an_no_tb and the energy the bath gave
// each atom, SimLoop.cxx:362-385), allocated with the first bath; an_no_tb
// starts as the current an.
static int ensure_bath_acct(mdg_ctx* c)
{
  if (!c->n || c->acc_ntb) return MDG_OK;
  c->acc_ntb = dalloc<double4>(c->n);
  c->d_eb = dalloc<double>(c->n);
  if (!c->acc_ntb || !c->d_eb) return fail(MDG_ERR_CUDA, "cudaMalloc (bath bookkeeping)");
  CK(cudaMemcpyAsync(c->acc_ntb, c->acc, c->n * sizeof(double4), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_eb, 0, c->n * sizeof(double), c->stream));
  c->step_cfg++;
  return MDG_OK;
}

// Loads nsys independent systems (atoms [first[s], first[s+1]) with box
// box[3s..3s+2] and periodicity pbc[3s..3s+2]); nsys = 1 is the ordinary
// single-system context.
static int set_systems(mdg_ctx* c, int nsys, const int64_t* first, const int32_t* z, const double* pos,
                       const double* vel, const double* box, const int32_t* pbc, const uint8_t* fixed)
{
  if (!c || nsys <= 0 || !first || !z || !pos || !box || !pbc) return fail(MDG_ERR_ARG, "bad argument");
  if (first[0] != 0) return fail(MDG_ERR_ARG, "first[0] must be 0");
  for (int sy = 0; sy < nsys; sy++)
    if (!(first[sy + 1] > first[sy])) return fail(MDG_ERR_ARG, "every system needs at least one atom");
  if (first[nsys] > (1LL << 30)) return fail(MDG_ERR_ARG, "too many atoms");
  const int n = (int)first[nsys];
  free_system(c);
  c->n = n;
  c->nsys = nsys;
  c->h_first.assign(first, first + nsys + 1);
  c->h_boxes.resize(nsys);
  c->h_sys.resize(n);
  for (int sy = 0; sy < nsys; sy++) {
    Box& b = c->h_boxes[sy];
    for (int a = 0; a < 3; a++) {
      b.pbc[a] = pbc[3 * sy + a] ? 1 : 0;
      b.L[a] = b.pbc[a] ? box[3 * sy + a] * c->unit_len : 0.0;
      if (b.pbc[a] && !(b.L[a] > 0)) return fail(MDG_ERR_ARG, "periodic axis with non-positive period");
    }
    for (int64_t i = first[sy]; i < first[sy + 1]; i++) c->h_sys[i] = sy;
  }
  c->box = c->h_boxes[0];
  // host-side packing: species, wrap (Atom::applyPBC), masses (Atom.hpp:104-105)
  std::vector<double4> hp(n), hv(n), ha(n);
  std::vector<int4> him(n);
  std::vector<double> hm(n), hpos(3 * (size_t)n);
  std::vector<unsigned char> hf(n, 0);
  c->h_type.assign(n, 0);
  const bool metal = c->prm.potentials & MDG_POT_METAL;
  int nonch = 0;
  // Atom::setAttributesByElementID (Atom.hpp:100-115): masses in amu by species
  const double mass_of[kNSpec] = {12.0, 1.0, 63.546, 107.868, 196.967, 39.948, 131.293};
  for (int i = 0; i < n; i++) {
    int t;
    switch (z[i]) {
      case 6: t = kC; break;
      case 1: t = kH; break;
      case 29: t = kCu; break;
      case 47: t = kAg; break;
      case 79: t = kAu; break;
      case 18: t = kAr; break;
      case 54: t = kXe; break;
      default: return fail(MDG_ERR_ARG, "unknown element (H, C, Cu, Ag, Au, Ar, Xe are on this path)");
    }
    if (t > kH) {
      if (!metal) return fail(MDG_ERR_ARG, "Cu, Ag, Au, Ar and Xe need MDG_POT_METAL (REBO::e2i handles only H and C)");
      nonch++;
    }
    double x[3];
    int im[3] = {0, 0, 0};
    const Box& bx = c->h_boxes[c->h_sys[i]];
    for (int a = 0; a < 3; a++) {
      x[a] = pos[3 * i + a] * c->unit_len;
      if (!std::isfinite(x[a])) return fail(MDG_ERR_NONFINITE, "non-finite coordinate");
      if (bx.pbc[a] && !wrap1(x[a], im[a], bx.L[a])) return fail(MDG_ERR_ARG, "coordinate too far outside the box");
      hpos[3 * i + a] = x[a];
    }
    hp[i] = make_double4(x[0], x[1], x[2], (double)t);
    c->h_type[i] = t;
    hf[i] = (fixed && fixed[i]) ? 1 : 0;
    if (vel && !hf[i])
      hv[i] = make_double4(vel[3 * i] * c->unit_vel, vel[3 * i + 1] * c->unit_vel, vel[3 * i + 2] * c->unit_vel, 0.0);
    else
      hv[i] = make_double4(0, 0, 0, 0);
    ha[i] = make_double4(0, 0, 0, 0);
    him[i] = make_int4(im[0], im[1], im[2], 0);
    hm[i] = mass_of[t];
  }
  // minimum image needs every period above twice the largest cutoff
  // (SimLoop.cxx:239-245, AtomsArray::checkMIC)
  double rmax = (c->prm.potentials & MDG_POT_AIREBO_LJ) ? c->ljp.R[0][0][1] : 2.0;
  if (metal && nonch) rmax = std::fmax(rmax, 5.5);  // FBZL / FLJ (Rcutoff 5.5 A, applications/common.h:46-49)
  for (const Box& bx : c->h_boxes)
    for (int a = 0; a < 3; a++)
      if (bx.pbc[a] && !(bx.L[a] > 2.0 * rmax))
        return fail(MDG_ERR_ARG, "Rcutoff is too large for given PBC (AtomsArray::checkMIC)");
  if (nsys > 1) {
    c->d_sys = dalloc<int>(n);
    c->d_boxes = dalloc<Box>(nsys);
    c->d_first = dalloc<int64_t>(nsys + 1);
    if (!c->d_sys || !c->d_boxes || !c->d_first) return fail(MDG_ERR_CUDA, "cudaMalloc (systems)");
    CK(cudaMemcpy(c->d_sys, c->h_sys.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_boxes, c->h_boxes.data(), nsys * sizeof(Box), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_first, first, (nsys + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
  }
  c->pos = dalloc<double4>(n);
  c->vel = dalloc<double4>(n);
  c->acc = dalloc<double4>(n);
  c->grad = dalloc<double4>(n);
  c->image = dalloc<int4>(n);
  c->fixed = dalloc<unsigned char>(n);
  c->mass = dalloc<double>(n);
  if (!c->pos || !c->vel || !c->acc || !c->grad || !c->image || !c->fixed || !c->mass)
    return fail(MDG_ERR_CUDA, "cudaMalloc (state)");
  CK(cudaMemcpy(c->pos, hp.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->vel, hv.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->acc, ha.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->image, him.data(), n * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->fixed, hf.data(), n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->mass, hm.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  c->acc_valid = false;

  // neighbour lists (NeighbourList::Update range (1+0.44) Rcut, NeighbourList.cxx:65)
  const bool with_lj = c->prm.potentials & MDG_POT_AIREBO_LJ;
  c->rcut[0] = 2.0;  // REBO::getRcutoff = max R2 (REBO.hpp:147)
  c->rcut[1] = with_lj ? std::fmax(std::fmax(c->ljp.R[0][0][1], c->ljp.R[0][1][1]), c->ljp.R[1][1][1]) : 0.0;
  c->has_list[0] = true;
  c->has_list[1] = with_lj;
  c->has_list[2] = metal && nonch > 0;
  c->rcut[2] = 5.5;  // FBZL, FLJ 5.5 A; Ackland's own ranges are below it
  for (int l = 0; l < 3; l++) {
    if (!c->has_list[l]) continue;
    NList& L = c->nl[l];
    double range = c->prm.nl_skin_mode == 0 ? (1.0 + 0.44) * c->rcut[l] : c->rcut[l] + c->prm.nl_skin;
    L.range2 = range * range;
    L.trigger = c->prm.nl_skin_mode == 0 ? 0.44 * c->rcut[l] : c->prm.nl_skin;
    L.cap = (l == 0) ? c->prm.cap_rebo_list : (l == 1 ? c->prm.cap_lj_list : kMetalListCap);
    // The REBO list keeps the reference's ascending order (it fixes the bond
    // slot order, hence every bond-order sum).  The LJ list only orders pair
    // sums, so it stays in (deterministic) cell order and skips the sort.
    L.sorted = (l == 0) ? 1 : 0;
    // with metal or ion atoms present, REBO and AIREBO see hydrocarbon pairs
    // only, the metal list every other pair (FGeneral's handled pairs)
    L.pairs = (l == 2) ? 2 : (nonch ? 1 : 0);
    L.cnt = dalloc<int>(n);
    L.list = dalloc<int>((size_t)n * L.cap);
    L.pos0 = dalloc<double4>(n);
    if (!L.cnt || !L.list || !L.pos0) return fail(MDG_ERR_CUDA, "cudaMalloc (neighbour list)");
    if (l == 1) {
      c->lj_inr = dalloc<int>((size_t)n * L.cap);
      c->lj_inr_cnt = dalloc<int>(2 * (size_t)n);  // far counts, then close counts
      NList& T = c->ljt;
      T.cap = L.cap;
      T.sorted = L.sorted;
      T.pairs = L.pairs;
      T.range2 = 0.0;  // per pair: (R2 + kLjNearSkin)^2
      T.trigger = kLjNearSkin;
      T.cnt = dalloc<int>(n);
      T.list = dalloc<int>((size_t)n * T.cap);
      T.pos0 = dalloc<double4>(n);
      if (!c->lj_inr || !c->lj_inr_cnt || !T.cnt || !T.list || !T.pos0)
        return fail(MDG_ERR_CUDA, "cudaMalloc (LJ in-range lists)");
    }
    int rc = nsys > 1 ? setup_grid_batch(c, l, hpos) : setup_grid(c, l, hpos);
    if (rc) return rc;
  }
  int one[4] = {1, 1, 1, 1};
  CK(cudaMemcpy(c->d_force, one, sizeof(one), cudaMemcpyHostToDevice));
  c->d_part = dalloc<double>(2 * 4 * kDispParts);
  if (c->has_list[2]) {
    if (!c->d_metal) {
      MetalParams hmp;
      make_metal_params(hmp);
      c->d_metal = dalloc<MetalParams>(1);
      if (!c->d_metal) return fail(MDG_ERR_CUDA, "cudaMalloc (metal parameters)");
      CK(cudaMemcpy(c->d_metal, &hmp, sizeof(hmp), cudaMemcpyHostToDevice));
    }
    c->d_fp = dalloc<double>(n);
    c->d_em = dalloc<double>(n);
    c->d_gm = dalloc<double4>(n);
    if (!c->d_fp || !c->d_em || !c->d_gm) return fail(MDG_ERR_CUDA, "cudaMalloc (metal forces)");
    CK(cudaMemset(c->d_em, 0, n * sizeof(double)));
  }

  // bonds and force outputs
  const int mb = c->mb;
  c->bb.n = n;
  c->bb.mb = mb;
  c->bb.nb = dalloc<int>(n);
  c->bb.bj = dalloc<int>((size_t)n * mb);
  c->bb.brev = dalloc<int>((size_t)n * mb);
  c->bb.brv = dalloc<double4>((size_t)n * mb);
  c->bb.bu = dalloc<double4>((size_t)n * mb);
  c->bb.bd = dalloc<double4>((size_t)n * mb);
  c->bb.nco = dalloc<double4>(n);
  c->fo.mb = mb;
  c->fo.A = dalloc<double>((size_t)n * mb * 3);
  c->fo.W = dalloc<double>((size_t)n * mb);
  c->fo.gown = dalloc<double4>(n);
  c->fo.glj = dalloc<double4>(n);
  c->fo.e_rebo = dalloc<double>(n);
  c->fo.e_tors = dalloc<double>(n);
  c->fo.e_lj = dalloc<double>(n);
  c->e_kin = dalloc<double>(n);
  c->d_red_part = dalloc<double>(5 * kRedBlocks);
  if (!c->bb.nb || !c->bb.bj || !c->bb.brev || !c->bb.brv || !c->bb.bu || !c->bb.bd || !c->bb.nco || !c->fo.A ||
      !c->fo.W || !c->fo.gown || !c->fo.glj || !c->fo.e_rebo || !c->fo.e_tors || !c->fo.e_lj || !c->e_kin ||
      !c->d_red_part)
    return fail(MDG_ERR_CUDA, "cudaMalloc (bonds)");
  CK(cudaMemset(c->fo.glj, 0, n * sizeof(double4)));
  CK(cudaMemset(c->fo.e_lj, 0, n * sizeof(double)));
  if (c->prm.potentials & (MDG_POT_REBO | MDG_POT_ETORS) && !(c->prm.potentials & MDG_POT_BRENNER)) {
    BondTasks& K = c->bt;
    K.cap = n * mb;
    K.pairs = c->prm.task_mode >= 2 ? c->prm.task_mode - 1 : 0;
    K.tors = (c->prm.potentials & MDG_POT_ETORS) ? 1 : 0;
    K.rec_cap = (long)n * c->prm.bond_rec_avg;
    K.q = dalloc<int>((size_t)K.cap);
    K.ctr = dalloc<unsigned long long>(4);
    K.rbase = dalloc<long>(n);
    K.nrec = dalloc<int>(n);
    K.rec = dalloc<double>((size_t)K.rec_cap);
    if (!K.q || !K.ctr || !K.rbase || !K.nrec || !K.rec) return fail(MDG_ERR_CUDA, "cudaMalloc (bond tasks)");
    CK(cudaMemset(K.ctr, 0, 4 * sizeof(unsigned long long)));
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (c->prm.precision == MDG_PREC_FP32_MIXED)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rebo_task<f32, ReboTables32>, kThreads, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rebo_task<double, ReboTables>, kThreads, 0);
    c->rebo_task_blocks = sms * (per > 0 ? per : 1);
  }
  if (with_lj) {
    if (c->prm.cap_cij > kCijLocal) c->prm.cap_cij = kCijLocal;
    c->cij.cap = c->prm.cap_cij;
    c->cij.cnt = dalloc<int>(n);
    c->cij.ent = dalloc<int4>((size_t)n * c->cij.cap);
    c->cij.w = dalloc<double>((size_t)n * c->cij.cap);
    c->cij.mask = dalloc<unsigned long long>(n);
    SpecialTasks& X = c->spc;
    X.cap = c->prm.cap_special;
    X.task_cap = (int)std::min<long>((long)n * c->prm.special_avg, 1L << 30);
    X.rec_cap = (long)X.task_cap * rec_size(6);
    X.cnt = dalloc<int>(n);
    X.part = dalloc<int>((size_t)n * X.cap);
    X.off = dalloc<int>(n);
    X.flat = dalloc<int2>(X.task_cap);
    X.trec = dalloc<long>(X.task_cap);
    X.rec = dalloc<double>(X.rec_cap);
    X.mid = dalloc<int4>(X.task_cap);
    X.midc = dalloc<double>(X.task_cap);
    X.work = dalloc<int>(X.task_cap);
    X.ctr = dalloc<unsigned long long>(3 * kCtrStride);
    if (!X.work || !X.ctr) return fail(MDG_ERR_CUDA, "cudaMalloc (LJ work list)");
    CK(cudaMemset(X.ctr, 0, 3 * kCtrStride * sizeof(unsigned long long)));
    if (!c->cij.cnt || !c->cij.ent || !c->cij.w || !c->cij.mask || !X.cnt || !X.part || !X.off || !X.flat ||
        !X.trec || !X.rec || !X.mid || !X.midc)
      return fail(MDG_ERR_CUDA, "cudaMalloc (LJ)");
    CK(cudaMemset(X.cnt, 0, n * sizeof(int)));
    CK(cudaMemset(X.off, 0, n * sizeof(int)));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    c->special_blocks = sms * 8;
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_lj_filter, kThreads, 0);
    c->warp_blocks = sms * (per > 0 ? per : 1);
  }
  if (cudaHostAlloc((void**)&c->h_stage, 2 * (size_t)n * sizeof(double4), cudaHostAllocDefault) != cudaSuccess)
    return fail(MDG_ERR_CUDA, "cudaHostAlloc (staging)");
  c->d_io = dalloc<double>(6 * (size_t)n);
  if (!c->d_io) return fail(MDG_ERR_CUDA, "cudaMalloc (host-step staging)");
  // per-system step state: bath temperature, adaptive dt, time, v_max
  c->d_tb_T = dalloc<double>(nsys);
  c->d_tb_part = dalloc<double>(2 * (size_t)std::max(kBathBlocks, nsys));
  c->d_dt = dalloc<double>(nsys);
  c->d_dt_prev = dalloc<double>(nsys);
  c->d_time = dalloc<double>(nsys);
  c->d_vmax = dalloc<unsigned long long>(nsys);
  c->d_e0 = dalloc<double>(4 * (size_t)nsys);
  c->d_ekin_pre = dalloc<double>(n);
  c->d_stop = dalloc<int>(nsys);
  if (!c->d_tb_T || !c->d_tb_part || !c->d_dt || !c->d_dt_prev || !c->d_time || !c->d_vmax || !c->d_e0 ||
      !c->d_ekin_pre || !c->d_stop)
    return fail(MDG_ERR_CUDA, "cudaMalloc (step state)");
  CK(cudaMemset(c->d_stop, 0, nsys * sizeof(int)));
  CK(cudaMemset(c->d_ekin_pre, 0, n * sizeof(double)));
  CK(cudaMemset(c->d_e0, 0, 4 * (size_t)nsys * sizeof(double)));
  c->h_z.assign(z, z + n);
  c->h_fixed = hf;
  c->h_tags.assign(n, 0);
  c->iteration = 0;
  c->time_s = 0.0;
  c->dt_s = c->dt_prev_s = 1e-20;
  c->stepped = c->e0_dev = c->chk_loaded = false;
  c->chk_e0 = 1.0;
  c->chk_eb0 = 0.0;
  c->chk_net[0] = c->chk_net[1] = c->chk_net[2] = 0.0;  // Check::Check (SimLoop.cxx:1280-1286)
  c->chk_cur = 1.0;
  c->chk_T = 0.0;
  c->run_t0 = 0.0;
  {
    std::vector<double> dt0((size_t)nsys, c->dt0);
    CK(cudaMemcpy(c->d_dt, dt0.data(), nsys * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_dt_prev, dt0.data(), nsys * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->d_time, 0, nsys * sizeof(double)));
    CK(cudaMemset(c->d_vmax, 0, nsys * sizeof(unsigned long long)));
    CK(cudaMemset(c->d_tb_T, 0, nsys * sizeof(double)));
  }
  if (c->tb_geom) {
    int rc = ensure_bath_acct(c);
    if (rc) return rc;
  }
  c->step_cfg++;
  CK(cudaDeviceSynchronize());
  return MDG_OK;
}

int mdg_set_system(mdg_ctx* c, int n, const int32_t* z, const double* pos, const double* vel,
                   const double box[3], const int32_t pbc[3], const uint8_t* fixed)
{
  if (n <= 0) return fail(MDG_ERR_ARG, "bad argument");
  const int64_t first[2] = {0, n};
  return set_systems(c, 1, first, z, pos, vel, box, pbc, fixed);
}

int mdg_set_batch(mdg_ctx* c, int nsys, const int64_t* first, const int32_t* z, const double* pos,
                  const double* vel, const double* box, const int32_t* pbc, const uint8_t* fixed)
{
  return set_systems(c, nsys, first, z, pos, vel, box, pbc, fixed);
}

int mdg_set_positions(mdg_ctx* c, const double* pos)
{
  return mdg_set_state(c, pos, nullptr);
}

int mdg_set_state(mdg_ctx* c, const double* pos, const double* vel)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  const int n = c->n;
  std::vector<double4> hp(n), hv;
  std::vector<int4> him(n);
  std::vector<double4> old(n);
  CK(cudaMemcpyAsync(old.data(), c->pos, n * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(him.data(), c->image, n * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; i++) {
    double x[3];
    int im[3] = {him[i].x, him[i].y, him[i].z};
    for (int a = 0; a < 3; a++) {
      x[a] = pos[3 * i + a] * c->unit_len;
      if (!std::isfinite(x[a])) return fail(MDG_ERR_NONFINITE, "non-finite coordinate");
      const Box& bx = c->h_boxes[c->h_sys[i]];
      if (bx.pbc[a] && !wrap1(x[a], im[a], bx.L[a])) return fail(MDG_ERR_ARG, "coordinate too far outside the box");
    }
    hp[i] = make_double4(x[0], x[1], x[2], old[i].w);
    him[i] = make_int4(im[0], im[1], im[2], 0);
  }
  CK(cudaMemcpyAsync(c->pos, hp.data(), n * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->image, him.data(), n * sizeof(int4), cudaMemcpyHostToDevice, c->stream));
  if (vel) {
    hv.resize(n);
    for (int i = 0; i < n; i++)
      hv[i] = make_double4(vel[3 * i] * c->unit_vel, vel[3 * i + 1] * c->unit_vel, vel[3 * i + 2] * c->unit_vel, 0.0);
    CK(cudaMemcpyAsync(c->vel, hv.data(), n * sizeof(double4), cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->acc_valid = false;
  return MDG_OK;
}

int mdg_compute(mdg_ctx* c, double* e_total, double* e_terms, double* grad)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  int rc = evaluate(c);
  if (rc) return rc;
  rc = reduce_energies(c, c->d_energy, 0, 0, false, true);
  if (rc) return rc;
  LAUNCH(c, "finite_check", k_finite, nblk(c->n), kThreads, c->grad, c->n, c->d_status);
  double he[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(he, c->d_energy, (c->has_list[2] ? 4 : 3) * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  std::vector<double4> hg;
  if (grad) {
    hg.resize(c->n);
    CK(cudaMemcpyAsync(hg.data(), c->grad, c->n * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  }
  rc = read_status(c);
  if (rc) return rc;
  double E = (he[0] + he[1]) + he[2];
  if (c->has_list[2]) E += he[3];
  if (e_total) *e_total = E * c->unit_e;
  if (e_terms) {
    e_terms[0] = he[0] * c->unit_e;
    e_terms[1] = he[1] * c->unit_e;
    e_terms[2] = he[2] * c->unit_e;
    e_terms[3] = he[3] * c->unit_e;  // FBZL + FLJ + Ackland
  }
  if (grad)
    for (int i = 0; i < c->n; i++) {
      grad[3 * i] += hg[i].x * c->unit_grad;
      grad[3 * i + 1] += hg[i].y * c->unit_grad;
      grad[3 * i + 2] += hg[i].z * c->unit_grad;
    }
  return MDG_OK;
}

int mdg_nl_update(mdg_ctx* c, int force, int32_t* rebuilt)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (force) {
    static const int one[4] = {1, 1, 1, 1};
    CK(cudaMemcpyAsync(c->d_force, one, sizeof(one), cudaMemcpyHostToDevice, c->stream));
  }
  int rc = rebuild_lists(c);
  if (rc) return rc;
  int need[3] = {0, 0, 0};
  CK(cudaMemcpyAsync(need, c->d_need, sizeof(need), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  if (rebuilt)
    for (int l = 0; l < 3; l++) rebuilt[l] = (c->has_list[l] && need[l]) ? 1 : 0;
  return MDG_OK;
}

int mdg_nl_pairs(mdg_ctx* c, int list_id, int32_t* pairs, int64_t cap, int64_t* count)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (list_id < 0 || list_id > 1 || !c->has_list[list_id]) return fail(MDG_ERR_ARG, "no such list");
  int rc = rebuild_lists(c);
  if (rc) return rc;
  const NList& L = c->nl[list_id];
  std::vector<int> cnt(c->n), lst((size_t)c->n * L.cap);
  CK(cudaMemcpyAsync(cnt.data(), L.cnt, c->n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(lst.data(), L.list, lst.size() * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  std::vector<std::pair<int, int>> out;
  for (int i = 0; i < c->n; i++)
    for (int s = 0; s < cnt[i]; s++) {
      int j = lst[(size_t)i * L.cap + s];
      if (j > i) out.push_back(std::make_pair(i, j));
    }
  std::sort(out.begin(), out.end());
  if (count) *count = (int64_t)out.size();
  if (pairs)
    for (int64_t q = 0; q < (int64_t)out.size() && q < cap; q++) {
      pairs[2 * q] = out[q].first;
      pairs[2 * q + 1] = out[q].second;
    }
  return MDG_OK;
}

// The autotuner: with task_mode 0, on the first run of a system, times one
// force evaluation (after one untimed evaluation; best of three) in each
// configuration of the REBO work and keeps the fastest:
//   - the split: one task per directed bond, or one per bond (both route the
//     same terms into the same records, equal to rounding);
//   - with the LJ term, where the REBO tasks run: in order before the LJ
//     chain with the grid at the kernel's resident capacity, or on the second
//     stream concurrently with the LJ chain with 1, 2 or all resident blocks
//     per SM (fewer blocks leave the SMs' registers to the LJ kernels).
// The choice changes only the speed; results are bitwise the same for a
// given split.
// Time one force evaluation as the steps run it: captured into a CUDA graph
// (stream overlap and dependent launches included) and replayed four times
// back to back per sample; the best of three samples, per evaluation.
static int time_eval_graph(mdg_ctx* c, cudaEvent_t e0, cudaEvent_t e1, float* best)
{
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  const int64_t l0 = c->launches;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = evaluate(c);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  c->launches = l0;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
  *best = 1e30f;
  ce = cudaGraphLaunch(ge, c->stream);
  for (int r = 0; r < 3 && ce == cudaSuccess; r++) {
    cudaEventRecord(e0, c->stream);
    for (int k = 0; k < 4 && ce == cudaSuccess; k++) ce = cudaGraphLaunch(ge, c->stream);
    cudaEventRecord(e1, c->stream);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    *best = std::min(*best, 0.25f * ms);
  }
  cudaGraphExecDestroy(ge);
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("graph replay: ") + cudaGetErrorString(ce));
  return MDG_OK;
}

static int autotune(mdg_ctx* c)
{
  if (c->tuned || !c->bt.ctr) return MDG_OK;
  c->tuned = true;
  const bool lj = c->prm.potentials & MDG_POT_AIREBO_LJ;
  // a fixed task mode (task_mode 1 or 2) keeps its split; the launch
  // configuration, which never changes results, is still chosen
  if (c->prm.task_mode != 0 && !lj) return MDG_OK;
  const int mode0 = c->prm.task_mode ? c->prm.task_mode - 1 : 0;
  const int mode1 = c->prm.task_mode ? c->prm.task_mode : 3;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  struct Cfg { bool overlap; int grid; };
  std::vector<Cfg> cfgs = {{false, c->rebo_task_blocks}};
  if (lj)
    for (int per : {1, 2})
      if (sms * per < c->rebo_task_blocks) cfgs.push_back({true, sms * per});
  if (lj) cfgs.push_back({true, c->rebo_task_blocks});
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best_all = 1e30f;
  int best_mode = mode0;
  Cfg best_cfg = cfgs[0];
  for (int mode = mode0; mode < mode1; mode++) {
    c->bt.pairs = mode;
    c->tune_ms[mode] = 1e30f;
    for (const Cfg& g : cfgs) {
      c->overlap = g.overlap;
      c->rebo_grid = g.grid;
      int rc = evaluate(c);
      if (rc) return rc;
      float best = 1e30f;
      if (!c->prof) {
        rc = time_eval_graph(c, e0, e1, &best);
        if (rc) return rc;
      } else {
        for (int r = 0; r < 3; r++) {
          CK(cudaEventRecord(e0, c->stream));
          rc = evaluate(c);
          if (rc) return rc;
          CK(cudaEventRecord(e1, c->stream));
          CK(cudaEventSynchronize(e1));
          float ms = 0.0f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          best = std::min(best, ms);
        }
      }
      c->tune_ms[mode] = std::min(c->tune_ms[mode], best);
      if (best < best_all) {
        best_all = best;
        best_mode = mode;
        best_cfg = g;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->bt.pairs = best_mode;
  c->overlap = best_cfg.overlap;
  c->rebo_grid = best_cfg.grid;
  return read_status(c);
}

// The captured step (position update, forces, velocity update) for time
// step dtf on the context's stream, captured again when either changes.
// The step descriptor of the context's current configuration (fixed dt dtf,
// or the device's per-system dt when adaptive; the thermal bath when set).
static StepDev step_dev(mdg_ctx* c, double dtf)
{
  StepDev P;
  std::memset(&P, 0, sizeof(P));
  P.dt = dtf;
  P.d_dt = c->adaptive ? c->d_dt : nullptr;
  P.tb_geom = c->tb_geom;
  P.T0 = c->tb_T0;
  P.gamma = c->tb_gamma;
  for (int k = 0; k < 5; k++) P.gp[k] = c->tb_gp[k];
  P.tb_apply = c->d_tb_apply;
  P.tb_T = c->d_tb_T;
  P.vmax = c->adaptive ? c->d_vmax : nullptr;
  P.nlc0 = c->nl[0].cnt;
  P.nlc1 = c->has_list[1] ? c->nl[1].cnt : nullptr;
  P.nlc2 = c->has_list[2] ? c->nl[2].cnt : nullptr;
  P.ekin_pre = c->d_ekin_pre;
  P.acc_ntb = c->tb_geom ? c->acc_ntb : nullptr;
  P.eb = c->tb_geom ? c->d_eb : nullptr;
  P.stop = (c->adaptive && c->stop_final) ? c->d_stop : nullptr;
  return P;
}

static int ensure_step_graph(mdg_ctx* c, double dtf)
{
  if (c->step_graph && c->graph_dt == dtf && c->graph_stream == c->stream && c->graph_cfg == c->step_cfg)
    return MDG_OK;
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
  cudaGraph_t g = nullptr;
  int64_t l0 = c->launches;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  const StepDev sd = step_dev(c, dtf);
  int rc = evaluate(c, &sd);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
  c->graph_launches = (int)(c->launches - l0);
  c->launches = l0;
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&c->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
  c->graph_dt = dtf;
  c->graph_stream = c->stream;
  c->graph_cfg = c->step_cfg;
  return MDG_OK;
}

int sys_energies(mdg_ctx* c, double* out_dev);
// checkpoint and trajectory output around the steps (defined with the file formats)
int io_run_start(mdg_ctx* c, double dtf, bool fresh);
int io_before_step(mdg_ctx* c);
int io_after_step(mdg_ctx* c);
int io_run_end(mdg_ctx* c);

// The first step's accelerations, and at iteration 0 the Check record's
// initial energy and the bath's energy count (SimLoop.cxx:305-321, 1133-1137).
static int init_first_step(mdg_ctx* c)
{
  if (c->acc_valid) return MDG_OK;
  int rc = evaluate(c);
  if (rc) return rc;
  State S = c->S();
  const bool first = c->iteration == 0;
  LAUNCH(c, "init_acc", k_init_acc, nblk(c->n), kThreads, S, c->grad, c->acc_ntb, first ? c->d_eb : nullptr);
  if (first) {
    LAUNCH(c, "ekin", k_ekin, nblk(c->n), kThreads, S, c->e_kin);
    // one system: the grid-wide reduction (the per-system kernel is one block per system)
    rc = c->nsys == 1 ? reduce_energies(c, c->d_e0, 0, 0, true) : sys_energies(c, c->d_e0);
    if (rc) return rc;
    c->e0_dev = true;
    c->chk_eb0 = 0.0;
  }
  c->acc_valid = true;
  return MDG_OK;
}

// Per-step potential and total energies from the pinned log of the last run.
static void fill_energy_log(mdg_ctx* c, int nsteps, double* epot, double* etot)
{
  const double* h = c->h_elog;
  for (int s = 0; s < nsteps; s++) {
    double ep = (h[4 * s] + h[4 * s + 1]) + h[4 * s + 2];
    if (epot) epot[s] = ep * c->unit_e;
    if (etot) etot[s] = (ep + h[4 * s + 3]) * c->unit_e;
  }
}

// fresh: a new SimLoop::execute (dt_prev = dt); else the continuation of
// the previous call's loop
static int run_steps(mdg_ctx* c, int nsteps, double dt, double* epot, double* etot, bool fresh,
                     bool defer_log = false)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (nsteps < 0) return fail(MDG_ERR_ARG, "negative step count");
  const double dtf = (c->prm.units == MDG_UNITS_CGS) ? dt / kFs : dt;
  // the split is chosen before the initial forces, so that they come from
  // the split every step uses
  int rc = autotune(c);
  if (rc) return rc;
  rc = init_first_step(c);
  if (rc) return rc;
  rc = io_run_start(c, dtf, fresh);
  if (rc) return rc;
  const bool log = epot || etot;
  if (log && c->elog_cap < (int64_t)nsteps * 4) {
    if (c->d_elog) cudaFree(c->d_elog);
    c->d_elog = dalloc<double>((size_t)nsteps * 4);
    if (!c->d_elog) return fail(MDG_ERR_CUDA, "cudaMalloc (energy log)");
    c->elog_cap = (int64_t)nsteps * 4;
  }
  // Unless profiling, a step is replayed from a CUDA graph: same kernels,
  // same arguments, no host launch cost; the per-step energy sums (when
  // asked for) follow each replay.
  const bool graph = !c->prof && nsteps > 0;
  if (graph) {
    rc = ensure_step_graph(c, dtf);
    if (rc) return rc;
  }
  for (int s = 0; s < nsteps; s++) {
    rc = io_before_step(c);  // scheduled state and trajectory files (SimLoop.cxx:263-277)
    if (rc) return rc;
    if (graph) {
      CK(cudaGraphLaunch(c->step_graph, c->stream));
      c->launches += c->graph_launches;
    } else {
      const StepDev sd = step_dev(c, dtf);
      rc = evaluate(c, &sd);  // position update, forces, velocity update
      if (rc) return rc;
    }
    rc = io_after_step(c);
    if (rc) return rc;
    if (log) {
      rc = reduce_energies(c, c->d_elog, 4, s, true);
      if (rc) return rc;
    }
  }
  rc = io_run_end(c);
  if (rc) return rc;
  if (log) {
    if (c->h_elog_cap < (int64_t)nsteps * 4) {
      if (c->h_elog) cudaFreeHost(c->h_elog);
      c->h_elog = nullptr;
      if (cudaHostAlloc((void**)&c->h_elog, (size_t)nsteps * 4 * sizeof(double), cudaHostAllocDefault) != cudaSuccess)
        return fail(MDG_ERR_CUDA, "cudaHostAlloc (energy log)");
      c->h_elog_cap = (int64_t)nsteps * 4;
    }
    CK(cudaMemcpyAsync(c->h_elog, c->d_elog, (size_t)nsteps * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    if (defer_log) return MDG_OK;  // the caller synchronises, then calls fill_energy_log
    rc = read_status(c);
    if (rc) return rc;
    fill_energy_log(c, nsteps, epot, etot);
    return MDG_OK;
  }
  return launch_check(c);
}

int mdg_run(mdg_ctx* c, int nsteps, double dt, double* epot, double* etot)
{
  return run_steps(c, nsteps, dt, epot, etot, true);
}

int sys_energies(mdg_ctx* c, double* out_dev)
{
  LAUNCH(c, "sys_energy", k_sys_energy, c->nsys, kThreads, c->d_first ? c->d_first : nullptr, (int64_t)c->n, c->fo.e_rebo,
         c->fo.e_lj, c->fo.e_tors, c->e_kin, c->has_list[2] ? c->d_em : nullptr, out_dev, c->d_status);
  return launch_check(c);
}

int mdg_batch_run(mdg_ctx* c, int nsteps, double dt, double* epot, double* etot)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (c->nsys < 2 || !c->d_first) return fail(MDG_ERR_STATE, "not a batched context (mdg_set_batch)");
  if (nsteps < 0) return fail(MDG_ERR_ARG, "negative step count");
  if (!epot && !etot) return mdg_run(c, nsteps, dt, nullptr, nullptr);
  const double dtf = (c->prm.units == MDG_UNITS_CGS) ? dt / kFs : dt;
  int rc = autotune(c);
  if (rc) return rc;
  rc = init_first_step(c);
  if (rc) return rc;
  rc = io_run_start(c, dtf, true);
  if (rc) return rc;
  const int64_t need = (int64_t)nsteps * c->nsys * 4;
  if (c->elog_cap < need) {
    if (c->d_elog) cudaFree(c->d_elog);
    c->d_elog = dalloc<double>((size_t)need);
    if (!c->d_elog) return fail(MDG_ERR_CUDA, "cudaMalloc (energy log)");
    c->elog_cap = need;
  }
  for (int s = 0; s < nsteps; s++) {
    rc = io_before_step(c);
    if (rc) return rc;
    const StepDev sd = step_dev(c, dtf);
    rc = evaluate(c, &sd);  // position update, forces, velocity update
    if (rc) return rc;
    rc = io_after_step(c);
    if (rc) return rc;
    rc = sys_energies(c, c->d_elog + (int64_t)s * c->nsys * 4);
    if (rc) return rc;
  }
  rc = io_run_end(c);
  if (rc) return rc;
  std::vector<double> h((size_t)need);
  CK(cudaMemcpyAsync(h.data(), c->d_elog, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  for (int64_t q = 0; q < (int64_t)nsteps * c->nsys; q++) {
    const double ep = (h[4 * q] + h[4 * q + 1]) + h[4 * q + 2];
    if (epot) epot[q] = ep * c->unit_e;
    if (etot) etot[q] = (ep + h[4 * q + 3]) * c->unit_e;
  }
  return MDG_OK;
}

int mdg_batch_energies(mdg_ctx* c, double* e_sys)
{
  if (!c || !c->n || !e_sys) return fail(MDG_ERR_ARG, "bad argument");
  if (c->nsys < 2 || !c->d_first) return fail(MDG_ERR_STATE, "not a batched context (mdg_set_batch)");
  int rc = evaluate(c);
  if (rc) return rc;
  State S = c->S();
  LAUNCH(c, "ekin", k_ekin, nblk(c->n), kThreads, S, c->e_kin);
  if (c->elog_cap < (int64_t)c->nsys * 4) {
    if (c->d_elog) cudaFree(c->d_elog);
    c->d_elog = dalloc<double>((size_t)c->nsys * 4);
    if (!c->d_elog) return fail(MDG_ERR_CUDA, "cudaMalloc (energy log)");
    c->elog_cap = (int64_t)c->nsys * 4;
  }
  rc = sys_energies(c, c->d_elog);
  if (rc) return rc;
  std::vector<double> h((size_t)c->nsys * 4);
  CK(cudaMemcpyAsync(h.data(), c->d_elog, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  for (size_t q = 0; q < h.size(); q++) e_sys[q] = h[q] * c->unit_e;
  return MDG_OK;
}

int mdg_set_thermal_bath(mdg_ctx* c, int geom, double T0, double gamma, const double* params, const uint8_t* apply)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  if (geom < MDG_TB_NONE || geom > MDG_TB_SPHERE) return fail(MDG_ERR_ARG, "unknown thermal bath geometry");
  if (geom != MDG_TB_NONE) {
    if (!(T0 >= 0.0) || !(gamma >= 0.0) || !std::isfinite(T0) || !std::isfinite(gamma))
      return fail(MDG_ERR_ARG, "bath temperature and friction rate must be finite and non-negative");
    if ((geom == MDG_TB_BOX || geom == MDG_TB_SPHERE) && !params) return fail(MDG_ERR_ARG, "null bath geometry");
    if (apply && !c->n) return fail(MDG_ERR_STATE, "per-atom bath flags need a loaded system");
    // the geometries' own REQUIREs (SimLoop.hpp:140, 166): a box bath needs
    // lateral periodicity, a sphere bath none
    for (const Box& b : c->h_boxes) {
      if (geom == MDG_TB_BOX && !(b.pbc[0] && b.pbc[1]))
        return fail(MDG_ERR_ARG, "a box thermal bath needs periodic x and y (ThermalBathGeomBox)");
      if (geom == MDG_TB_SPHERE && (b.pbc[0] || b.pbc[1] || b.pbc[2]))
        return fail(MDG_ERR_ARG, "a sphere thermal bath needs an open box (ThermalBathGeomSphere)");
    }
  }
  const double tconv = (c->prm.units == MDG_UNITS_CGS) ? kFs : 1.0;  // 1/(time unit) -> 1/fs
  c->tb_geom = geom;
  c->tb_T0 = T0;
  c->tb_gamma = gamma * tconv;
  for (int k = 0; k < 5; k++) c->tb_gp[k] = 0.0;
  if (geom == MDG_TB_BOX)
    for (int k = 0; k < 3; k++) c->tb_gp[k] = params[k] * c->unit_len;
  if (geom == MDG_TB_SPHERE)
    for (int k = 0; k < 5; k++) c->tb_gp[k] = params[k] * c->unit_len;
  if (c->d_tb_apply) cudaFree(c->d_tb_apply);
  c->d_tb_apply = nullptr;
  c->h_tb_apply.clear();
  if (apply) {
    c->d_tb_apply = dalloc<unsigned char>(c->n);
    if (!c->d_tb_apply) return fail(MDG_ERR_CUDA, "cudaMalloc (bath flags)");
    CK(cudaMemcpy(c->d_tb_apply, apply, c->n, cudaMemcpyHostToDevice));
    c->h_tb_apply.assign(apply, apply + c->n);
  }
  if (geom != MDG_TB_NONE) {
    int rc = ensure_bath_acct(c);
    if (rc) return rc;
  }
  c->step_cfg++;
  return MDG_OK;
}

int mdg_set_adaptive_dt(mdg_ctx* c, int on, double timeaccel, double dt0)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  const double tconv = (c->prm.units == MDG_UNITS_CGS) ? 1.0 / kFs : 1.0;  // time unit -> fs
  if (on && !(timeaccel > 0.0 && dt0 > 0.0 && std::isfinite(timeaccel) && std::isfinite(dt0)))
    return fail(MDG_ERR_ARG, "timeaccel and the starting dt must be finite and positive");
  c->adaptive = on != 0;
  if (on) {
    c->timeaccel = timeaccel * c->unit_len;
    c->dt0 = std::min(std::max(dt0 * tconv, 1e-5), 0.5);
    if (c->n) {
      std::vector<double> d((size_t)c->nsys, c->dt0);
      CK(cudaMemcpyAsync(c->d_dt, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(c->d_dt_prev, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemsetAsync(c->d_time, 0, c->nsys * sizeof(double), c->stream));
      CK(cudaMemsetAsync(c->d_vmax, 0, c->nsys * sizeof(unsigned long long), c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  }
  c->step_cfg++;
  return MDG_OK;
}

int mdg_get_time(mdg_ctx* c, double* sim_time, double* dt)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  std::vector<double> t((size_t)c->nsys), d((size_t)c->nsys);
  CK(cudaMemcpyAsync(t.data(), c->d_time, t.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(d.data(), c->d_dt, d.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  int rc = read_status(c);
  if (rc) return rc;
  const double tconv = (c->prm.units == MDG_UNITS_CGS) ? kFs : 1.0;  // fs -> time unit
  for (int s = 0; s < c->nsys; s++) {
    if (sim_time) sim_time[s] = t[s] * tconv;
    if (dt) dt[s] = d[s] * tconv;
  }
  return MDG_OK;
}

int mdg_tuned_launch(mdg_ctx* c, int* overlap, int* rebo_blocks)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  if (overlap) *overlap = c->overlap ? 1 : 0;
  if (rebo_blocks) *rebo_blocks = c->rebo_grid > 0 ? c->rebo_grid : c->rebo_task_blocks;
  return MDG_OK;
}

int mdg_set_dependent_launch(mdg_ctx* c, int on)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  c->pdl = on != 0;
  c->step_cfg++;  // recapture the step graph with the new launch attribute
  return MDG_OK;
}

int mdg_task_mode(mdg_ctx* c, int* mode, float* ms_directed, float* ms_per_bond, float* ms_split)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  if (mode) *mode = c->bt.pairs + 1;
  if (ms_directed) *ms_directed = c->tune_ms[0];
  if (ms_per_bond) *ms_per_bond = c->tune_ms[1];
  if (ms_split) *ms_split = c->tune_ms[2];
  return MDG_OK;
}

int mdg_sync(mdg_ctx* c)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  return read_status(c);
}

int mdg_get_state(mdg_ctx* c, double* pos, double* vel, int32_t* image)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  const int n = c->n;
  std::vector<double4> hp(n), hv(n);
  std::vector<int4> him(n);
  CK(cudaMemcpyAsync(hp.data(), c->pos, n * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(hv.data(), c->vel, n * sizeof(double4), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(him.data(), c->image, n * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  int rc = read_status(c);
  if (rc) return rc;
  for (int i = 0; i < n; i++) {
    if (pos) { pos[3*i] = hp[i].x / c->unit_len; pos[3*i+1] = hp[i].y / c->unit_len; pos[3*i+2] = hp[i].z / c->unit_len; }
    if (vel) { vel[3*i] = hv[i].x / c->unit_vel; vel[3*i+1] = hv[i].y / c->unit_vel; vel[3*i+2] = hv[i].z / c->unit_vel; }
    if (image) { image[3*i] = him[i].x; image[3*i+1] = him[i].y; image[3*i+2] = him[i].z; }
  }
  return MDG_OK;
}

int64_t mdg_launch_count(mdg_ctx* c) { return c ? c->launches : 0; }

int mdg_set_profiling(mdg_ctx* c, int on)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  c->prof = on != 0;
  c->prof_recs.clear();
  c->ev_used = 0;
  return MDG_OK;
}

int mdg_profile_read(mdg_ctx* c, int max, char* names, double* ms, int64_t* counts, int* nout)
{
  if (!c || !nout) return fail(MDG_ERR_ARG, "null argument");
  CK(cudaStreamSynchronize(c->stream));
  std::vector<std::string> keys;
  std::vector<double> tot;
  std::vector<int64_t> cnt;
  for (auto& r : c->prof_recs) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->ev_pool[r.second], c->ev_pool[r.second + 1]));
    size_t k = 0;
    while (k < keys.size() && keys[k] != r.first) k++;
    if (k == keys.size()) { keys.push_back(r.first); tot.push_back(0.0); cnt.push_back(0); }
    tot[k] += t;
    cnt[k] += 1;
  }
  int n = (int)keys.size();
  *nout = n;
  for (int k = 0; k < n && k < max; k++) {
    if (names) {
      std::strncpy(names + 32 * k, keys[k].c_str(), 31);
      names[32 * k + 31] = 0;
    }
    if (ms) ms[k] = tot[k];
    if (counts) counts[k] = cnt[k];
  }
  c->prof_recs.clear();
  c->ev_used = 0;
  return MDG_OK;
}

int mdg_step_host(mdg_ctx* c, int nsteps, double dt, double* pos, double* vel, double* epot, double* etot)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (!pos || !vel) return fail(MDG_ERR_ARG, "null state buffer");
  const int n = c->n;
  // the caller's [n*3] arrays move as they are (one copy each way; DMA
  // straight from and to them when they are pinned) and are converted to and
  // from the device layout by kernels
  double* io = c->d_io;
  CK(cudaMemcpyAsync(io, pos, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(io + 3 * (size_t)n, vel, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  State S = c->S();
  LAUNCH(c, "state_unpack", k_state_unpack, nblk(n), kThreads, S, io, c->unit_len, c->unit_vel);
  // one synchronisation for the whole call: the energy log, the state and
  // the status come back together
  int rc = run_steps(c, nsteps, dt, epot, etot, true, true);
  if (rc) return rc;
  LAUNCH(c, "state_pack", k_state_pack, nblk(n), kThreads, S, io, c->unit_len, c->unit_vel);
  CK(cudaMemcpyAsync(pos, io, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(vel, io + 3 * (size_t)n, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  if (epot || etot) fill_energy_log(c, nsteps, epot, etot);
  return MDG_OK;
}

int mdg_pipe_peak(int device, int fp32, double* tflops)
{
  if (!tflops) return fail(MDG_ERR_ARG, "null argument");
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  void* buf = nullptr;
  CK(cudaMalloc(&buf, 64));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0.0;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0);
    if (fp32) k_peak_fp32<<<blocks, threads>>>((float*)buf, iters, 0.999999f, 1e-7f);
    else k_peak_fp64<<<blocks, threads>>>((double*)buf, iters, 0.999999999, 1e-12);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    if (rep > 0) best = std::fmax(best, flops / (t * 1e-3) / 1e12);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  CK(cudaGetLastError());
  *tflops = best;
  return MDG_OK;
}

// The floor of a step of `phases` dependent phases with no work in them, two
// ways: phases empty kernels of a graph, each a programmatic dependent launch
// (how the step runs), and one cooperative kernel with a grid-wide barrier
// between phases (a persistent fused step).  Both over two blocks per SM.
__global__ void k_floor_phase()
{
  pdl_enter();
}

__global__ void k_floor_coop(int phases)
{
  cooperative_groups::grid_group g = cooperative_groups::this_grid();
  for (int p = 0; p < phases; p++) g.sync();
}

#if defined(MDG_TIMELINE)
// The timeline build's stamps (see pdl_enter): reset before a step, read
// after it; slot = the source line of a kernel's pdl_enter() in this file.
int mdg_timeline_reset(void)
{
  static unsigned long long hi[kTimelineSlots], lo[kTimelineSlots];
  for (int i = 0; i < kTimelineSlots; i++) { hi[i] = ~0ull; lo[i] = 0ull; }
  if (cudaMemcpyToSymbol(g_tl_start, hi, sizeof(hi)) != cudaSuccess ||
      cudaMemcpyToSymbol(g_tl_wait, hi, sizeof(hi)) != cudaSuccess ||
      cudaMemcpyToSymbol(g_tl_end, lo, sizeof(lo)) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
    return fail(MDG_ERR_CUDA, "timeline reset");
  return MDG_OK;
}
int mdg_timeline_read(uint64_t* start, uint64_t* wait, uint64_t* end, int slots)
{
  if (slots < kTimelineSlots) return fail(MDG_ERR_ARG, "timeline arrays hold kTimelineSlots entries");
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpyFromSymbol(start, g_tl_start, kTimelineSlots * 8) != cudaSuccess ||
      cudaMemcpyFromSymbol(wait, g_tl_wait, kTimelineSlots * 8) != cudaSuccess ||
      cudaMemcpyFromSymbol(end, g_tl_end, kTimelineSlots * 8) != cudaSuccess)
    return fail(MDG_ERR_CUDA, "timeline read");
  return MDG_OK;
}
#endif

int mdg_launch_floor(int device, int phases, double* graph_us, double* coop_us)
{
  if (!graph_us || !coop_us || phases < 1 || phases > 1000) return fail(MDG_ERR_ARG, "bad argument");
  CK(cudaSetDevice(device));
  int sms = 0, coop = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop) return fail(MDG_ERR_CUDA, "no cooperative launch on this device");
  const int blocks = 2 * sms, threads = 128, reps = 200;
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  // the graph of dependent launches
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.stream = st;
  cudaLaunchAttribute at;
  at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &at;
  cfg.numAttrs = 1;
  for (int p = 0; p < phases; p++) cudaLaunchKernelEx(&cfg, k_floor_phase);
  cudaError_t ce = cudaStreamEndCapture(st, &g);
  if (ce == cudaSuccess) ce = cudaGraphInstantiate(&ge, g, 0);
  if (g) cudaGraphDestroy(g);
  double best_graph = 1e30, best_coop = 1e30;
  for (int rep = 0; rep < 3 && ce == cudaSuccess; rep++) {
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && ce == cudaSuccess; r++) ce = cudaGraphLaunch(ge, st);
    cudaEventRecord(e1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    best_graph = std::min(best_graph, 1e3 * ms / reps);
  }
  if (ge) cudaGraphExecDestroy(ge);
  // the cooperative kernel, launched back to back
  int ph = phases;
  void* args[] = {&ph};
  for (int rep = 0; rep < 3 && ce == cudaSuccess; rep++) {
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps && ce == cudaSuccess; r++)
      ce = cudaLaunchCooperativeKernel((const void*)k_floor_coop, dim3(blocks), dim3(threads), args, 0, st);
    cudaEventRecord(e1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
    float ms = 0.0f;
    if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
    best_coop = std::min(best_coop, 1e3 * ms / reps);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("launch floor: ") + cudaGetErrorString(ce));
  *graph_us = best_graph;
  *coop_us = best_coop;
  return MDG_OK;
}

int64_t mdg_debug_brenner_tables(int set, double* out, int64_t cap)
{
  BrennerTables* h = new BrennerTables();
  std::vector<double> flat;
  build_brenner_tables(set, h, &flat);
  delete h;
  for (int64_t i = 0; i < (int64_t)flat.size() && i < cap; i++) out[i] = flat[i];
  return (int64_t)flat.size();
}

int64_t mdg_debug_rebo_tables(double* out, int64_t cap)
{
  ReboTables* h = new ReboTables();
  std::vector<double> flat;
  build_rebo_tables(h, &flat);
  delete h;
  for (int64_t i = 0; i < (int64_t)flat.size() && i < cap; i++) out[i] = flat[i];
  return (int64_t)flat.size();
}

int mdg_debug_spline(int precision, int kind, int fam, int n, const double* args, double* out)
{
  if (!args || !out || n < 0 || kind < 0 || kind > 2) return fail(MDG_ERR_ARG, "bad spline query");
  if ((kind == 0 && (fam < 0 || fam > 2)) || (kind == 1 && (fam < 0 || fam > 1)) ||
      (kind == 2 && (fam < 0 || fam > 3)))
    return fail(MDG_ERR_ARG, "bad spline family");
  ReboTables* d = new ReboTables();
  build_rebo_tables(d, nullptr);
  ReboTables32* f = nullptr;
  if (precision == MDG_PREC_FP32_MIXED) {
    f = new ReboTables32();
    build_rebo_tables32(*d, f);
  }
  unsigned int st = 0;
  for (int q = 0; q < n; q++) {
    if (kind == 0) {
      if (f) {
        out[2 * q] = dbl(g_eval(f->G[fam], f32(args[q]), 0));
        out[2 * q + 1] = dbl(g_eval(f->G[fam], f32(args[q]), 1));
      } else {
        out[2 * q] = g_eval(d->G[fam], args[q], 0);
        out[2 * q + 1] = g_eval(d->G[fam], args[q], 1);
      }
    } else if (kind == 1) {
      if (f) {
        f32 v, dh, dc;
        p_eval(*f, fam, f32(args[2 * q]), f32(args[2 * q + 1]), v, dh, dc, &st);
        out[3 * q] = dbl(v); out[3 * q + 1] = dbl(dh); out[3 * q + 2] = dbl(dc);
      } else {
        p_eval(*d, fam, args[2 * q], args[2 * q + 1], out[3 * q], out[3 * q + 1], out[3 * q + 2], &st);
      }
    } else {
      if (f) {
        f32 r[4];
        t_eval(*f, fam, f32(args[3 * q]), f32(args[3 * q + 1]), f32(args[3 * q + 2]), r, &st);
        for (int t = 0; t < 4; t++) out[4 * q + t] = dbl(r[t]);
      } else {
        t_eval(*d, fam, args[3 * q], args[3 * q + 1], args[3 * q + 2], out + 4 * q, &st);
      }
    }
  }
  delete d;
  delete f;
  return MDG_OK;
}

}  // extern "C"

#include "mdg_io.cuh"
