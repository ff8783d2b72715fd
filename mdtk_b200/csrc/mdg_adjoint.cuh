// Adjoint of a velocity-Verlet trajectory under REBO (+ AIREBO LJ)
// (+ torsion): gradients of a loss of the final state with respect to the
// initial positions and velocities and to the C-C pair parameters
// (eps_CC, sigma_CC of the LJ term; A, B1, alpha, beta1 of REBO's V_R/V_A).
// The reference has no adjoint; the forward map it differentiates is the
// reference's step (SimLoop.cxx:323-399, fixed dt) with the reference's
// forces.
//
// Part of mdg_api.cu's translation unit (it uses the context internals);
// included once, after them.
//
// Discrete adjoint.  A step is
//   x' = x + v dt + a dt^2/2,   a' = -c g(x')/m,   v' = v + (a + a') dt/2
// (g the gradient the force kernels accumulate, c = kAccConv).  With the
// adjoints (X', V', A') of (x', v', a'):
//   At = A' + V' dt/2,  Xt = X' - c J^T (At/m)   (J = dg/dx at x')
//   X = Xt,  V = V' + Xt dt,  A = V' dt/2 + Xt dt^2/2
//   theta_bar += -c d/dtheta [ (At/m) . g(x') ]
// Fixed atoms keep x, v, a: X = Xt, V = V', A = A'.  At step 0, a_0 = -c
// g(x_0)/m adds -c J^T (A_0/m) to X_0 and its parameter term.
//
// The Jacobian products come from one forward-mode pass of the force kernels
// on duals: positions carry the tangent u = At/m, so the tangent of every
// gradient component is (J u), and the tangents of the energy's parameter
// derivatives are d/dtheta (u . g).  REBO and LJ forces are gradients of
// their energies, so J is symmetric there and J u = J^T u; the reference's
// torsion force is not (mdg_etors.cuh routes the transpose correction).  The
// b*_ij of an LJ pair with a hydrogen centre follows the reference's r_alter
// gradient (REBO.cxx:224-233), which is not a gradient either; for systems
// with hydrogen that term's product is the forward one.  Pure carbon (the
// adjoint's target systems) is exact.
//
// Checkpointed recomputation: the forward run keeps the state every
// `checkpoint_every` steps; the backward run recomputes one segment at a time
// from its checkpoint (keeping that segment's positions) and walks it
// backwards, so memory is O(n (steps/every + every)).
#pragma once

namespace {

// Device buffers of the adjoint path (dual copies of the force-evaluation
// intermediates, the adjoint state, the checkpoints).
struct AdjWs {
  int n = 0, mb = 0, ccap = 0, tcap = 0;
  long rcap = 0;
  // dual bond list and force outputs
  dual4 *brv = nullptr, *bu = nullptr, *bd = nullptr, *nco = nullptr;
  dual *A = nullptr, *W = nullptr, *er = nullptr, *et = nullptr, *el = nullptr, *dp = nullptr;
  dual4 *gown = nullptr, *glj = nullptr, *g = nullptr;
  dual* cw = nullptr;                 // connectivity weights
  dual *trec = nullptr, *tmidc = nullptr, *tdp = nullptr;  // special-pair task records
  int4* tmid = nullptr;
  double4* tan = nullptr;             // position tangents of the dual pass
  // adjoint state and parameter gradient
  double4 *lx = nullptr, *lv = nullptr, *la = nullptr;
  double* theta = nullptr;            // [kNParam] accumulated parameter gradient
  double* dpar = nullptr;             // [2 * kNParam] last pass: sums of dE/dtheta (value, tangent)
  // forward record
  bool have_fwd = false;
  int nsteps = 0, every = 0, ncp = 0, cp_cap = 0;
  double dt = 0.0;
  double4 *cp_pos = nullptr, *cp_vel = nullptr, *cp_acc = nullptr;  // [cp_cap * n]
  int4* cp_img = nullptr;
  double4* seg_pos = nullptr;         // [every * n]
  int seg_cap = 0;
  double4 *fin_pos = nullptr, *fin_vel = nullptr, *fin_acc = nullptr;
  int4* fin_img = nullptr;
};

struct DualBonds {
  dual4 *brv, *bu, *bd, *nco;
};

// Bond list with tangents: the FP64 path's bonds (same slots, same lengths),
// rebuilt on duals whose positions carry tan.
__global__ void k_adj_bonds(State S, const double4* tan, ReboParams P, BondList B, DualBonds D)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= S.n) return;
  const double4 pa = S.pos[a], ua = tan[a];
  const int ta = (int)pa.w;
  const V3 xa = v3(pa.x, pa.y, pa.z);
  dual Nt = 0.0, NC = 0.0, NH = 0.0;
  const int nb = B.nb[a];
  for (int s = 0; s < nb; s++) {
    const int q = a * B.mb + s;
    const int j = B.bj[q];
    const double4 pj = S.pos[j], uj = tan[j];
    const int tj = (int)pj.w;
    const V3 rv = depos(box_of(S, a), xa, v3(pj.x, pj.y, pj.z));
    const double r0 = sqrt(norm2(rv));
    const V3 dv = v3(ua.x - uj.x, ua.y - uj.y, ua.z - uj.z);
    const dual r(r0, (rv.x * dv.x + rv.y * dv.y + rv.z * dv.z) / r0);
    const dual x(rv.x, dv.x), y(rv.y, dv.y), z(rv.z, dv.z);
    dual f, df;
    cutoff(r, P.R[ta][tj][0], P.R[ta][tj][1], f, df);
    const dual fp = Sprime(r, P.Rp[ta][tj][0], P.Rp[ta][tj][1]);
    const dual dfp = dSprime(r, P.Rp[ta][tj][0], P.Rp[ta][tj][1]);
    if (!(r0 > P.R[ta][tj][1])) {
      Nt += f;
      if (tj == kH) NH += f;
      if (tj == kC) NC += f;
    }
    D.brv[q] = make_dual4(x, y, z, r);
    D.bu[q] = make_dual4(x / r, y / r, z / r, f);
    D.bd[q] = make_dual4(df, fp, dfp, 0.0);
  }
  D.nco[a] = make_dual4(Nt, NC, NH, dual((double)ta));
}

__global__ void k_adj_rebo(const ReboParams* P, const ReboTables* T, BondListT<dual> B, TorsParams TP, int do_rebo,
                           int do_tors, ForceOutT<dual> O, unsigned int* status)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.n) return;
  ReboT<dual, ReboTables> R{*P, *T, B, status};
  rebo_atom<true>(R, TP, do_rebo, do_tors, O, a);
}

// Connectivity weights with tangents along the FP64 table's arg-max paths
// (the products in the order cij_build_atom forms them).
__global__ void k_adj_cij(BondListT<dual> B, CijTable T, dual* w)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.n) return;
  auto fb = [&](int c, int o) -> dual {
    const int s = bond_slot(B, c, o);
    return s >= 0 ? B.bu[c * B.mb + s].w : dual(0.0);
  };
  const int cnt = T.cnt[a];
  for (int e = 0; e < cnt; e++) {
    const int4 en = T.ent[(long)a * T.cap + e];
    dual v;
    if (en.y == 1) v = fb(a, en.x);
    else if (en.y == 2) v = fb(a, en.z) * fb(en.z, en.x);
    else v = fb(a, en.z) * fb(en.z, en.w) * fb(en.w, en.x);
    w[(long)a * T.cap + e] = v;
  }
}

// Plain LJ pairs (the FP64 path's classification), one thread per atom; the
// REBO kernel has already zeroed and filled this atom's parameter slots.
__global__ void k_adj_lj_plain(LJParams P, CijTableT<dual> T, State S, NList L, const double4* tan,
                               ForceOutT<dual> O)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= S.n) return;
  const double4 pa = S.pos[a];
  const V3 xa = v3(pa.x, pa.y, pa.z);
  const int ta = (int)pa.w;
  SinkT<dual, true> sk;
  sk.a = a;
  sk.g = v3r<dual>(0.0, 0.0, 0.0);
  sk.A = nullptr;
  sk.W = nullptr;
  sk.dp = O.dp + (long)a * kNParam;
  sk.jt = 1;
  dual e = 0.0;
  const int cnt = L.cnt[a];
  const int* lst = L.list + (long)a * L.cap;
  const unsigned long long amask = T.mask[a];
  for (int s = 0; s < cnt; s++) lj_plain_pair<dual>(P, T, S, a, lst[s], xa, ta, amask, sk, e, tan);
  O.glj[a] = make_dual4(sk.g.x, sk.g.y, sk.g.z, 0.0);
  O.e_lj[a] = e;
}

__global__ void k_adj_lj_special(const ReboParams* P, const ReboTables* Tb, LJParams LP, BondListT<dual> B,
                                 CijTableT<dual> T, State S, SpecialTasksT<dual> Tk, const double4* tan,
                                 unsigned int* status)
{
  pdl_enter();
  const int total = spc_total(Tk);
  ReboT<dual, ReboTables> R{*P, *Tb, B, status};
  LJT<dual, ReboTables> X{LP, R, T};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x)
    lj_special_task<true>(X, S, Tk, t, status, tan);
}

__global__ void k_adj_lj_reduce(BondListT<dual> B, SpecialTasksT<dual> Tk, ForceOutT<dual> O)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < B.n) lj_reduce_atom(B, Tk, O, a);
}

__global__ void k_adj_gather(BondListT<dual> B, ForceOutT<dual> O, int with_lj, SpecialTasksT<dual> Tk, dual4* g)
{
  pdl_enter();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.n) return;
  V3T<dual> gg = gather_atom(B, O, a, with_lj, (const dual4*)nullptr);
  if (with_lj) gg += mid_gather_atom(B, Tk, a);
  g[a] = make_dual4(gg.x, gg.y, gg.z, 0.0);
}

// Direction of the Jacobian product: u = (A' + V' dt/2)/m (mode 0, a step) or
// A_0/m (mode 1, the initial accelerations); 0 for fixed atoms.
__global__ void k_adj_dir(State S, const double4* lv, const double4* la, double dt, int mode, double4* tan)
{
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  if (S.fixed && S.fixed[i]) { tan[i] = make_double4(0.0, 0.0, 0.0, 0.0); return; }
  const double m = S.mass[i];
  const double4 a = la[i];
  double4 u = a;
  if (mode == 0) {
    const double4 v = lv[i];
    u = make_double4(a.x + v.x * dt / 2.0, a.y + v.y * dt / 2.0, a.z + v.z * dt / 2.0, 0.0);
  }
  tan[i] = make_double4(u.x / m, u.y / m, u.z / m, 0.0);
}

// Adjoint update after the product q = J^T u (the tangents of g):
// Xt = X' + seed_e g_exact - c q, then the step's transposed update (mode 0)
// or X_0 = Xt (mode 1).
__global__ void k_adj_update(State S, const dual4* g, double4* lx, double4* lv, double4* la, double dt, int mode,
                             double seed_e)
{
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const dual4 gi = g[i];
  const double4 x = lx[i];
  const double c = kAccConv;
  const double4 xt = make_double4(x.x + seed_e * gi.x.v - c * gi.x.d, x.y + seed_e * gi.y.v - c * gi.y.d,
                                  x.z + seed_e * gi.z.v - c * gi.z.d, 0.0);
  lx[i] = xt;
  if (mode != 0 || (S.fixed && S.fixed[i])) return;
  const double4 v = lv[i];
  lv[i] = make_double4(v.x + xt.x * dt, v.y + xt.y * dt, v.z + xt.z * dt, 0.0);
  la[i] = make_double4(v.x * dt / 2.0 + xt.x * dt * dt / 2.0, v.y * dt / 2.0 + xt.y * dt * dt / 2.0,
                       v.z * dt / 2.0 + xt.z * dt * dt / 2.0, 0.0);
}

// Per-parameter sums over atoms of dE/dtheta (value and tangent), one block
// per parameter in a fixed order; theta += scale_t * tangent + scale_v * value.
__global__ void k_adj_par(const dual* dp, int n, double scale_t, double scale_v, double* theta, double* last)
{
  pdl_enter();
  __shared__ double sv[128], sd[128];
  const int k = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const dual x = dp[(long)i * kNParam + k];
    a += x.v;
    b += x.d;
  }
  sv[threadIdx.x] = a;
  sd[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sv[threadIdx.x] += sv[threadIdx.x + w];
      sd[threadIdx.x] += sd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    theta[k] += scale_t * sd[0] + scale_v * sv[0];
    last[k] = sv[0];
    last[kNParam + k] = sd[0];
  }
}

template <class T>
bool adj_realloc(T*& p, size_t count)
{
  if (p) cudaFree(p);
  p = dalloc<T>(count);
  return p != nullptr;
}

void adj_free(mdg_ctx* c)
{
  AdjWs* w = c->adj;
  if (!w) return;
  void* ptrs[] = {w->brv, w->bu, w->bd, w->nco, w->A, w->W, w->er, w->et, w->el, w->dp, w->gown, w->glj, w->g,
                  w->cw, w->trec, w->tmidc, w->tdp, w->tmid, w->tan, w->lx, w->lv, w->la, w->theta, w->dpar,
                  w->cp_pos, w->cp_vel, w->cp_acc, w->cp_img, w->seg_pos, w->fin_pos, w->fin_vel, w->fin_acc,
                  w->fin_img};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete w;
  c->adj = nullptr;
}

// The adjoint needs an FP64 single-system REBO-family context in A/eV/fs.
int adj_check(mdg_ctx* c)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (c->prm.precision != MDG_PREC_FP64) return fail(MDG_ERR_ARG, "the adjoint runs on FP64 contexts");
  if (c->prm.potentials & MDG_POT_BRENNER) return fail(MDG_ERR_ARG, "the adjoint covers REBO, the LJ term and torsion");
  if (c->has_list[2]) return fail(MDG_ERR_ARG, "the adjoint covers hydrocarbons (no metal or ion atoms)");
  if (c->nsys > 1) return fail(MDG_ERR_ARG, "the adjoint runs on single-system contexts");
  if (c->prm.units != MDG_UNITS_AEVFS) return fail(MDG_ERR_ARG, "the adjoint works in Angstrom / eV / fs units");
  if (c->tb_geom || c->adaptive)
    return fail(MDG_ERR_ARG, "the adjoint differentiates fixed-dt steps without a thermal bath");
  return MDG_OK;
}

// Allocates (or re-sizes) the dual buffers for the loaded system.
int adj_ensure(mdg_ctx* c)
{
  if (!c->adj) c->adj = new AdjWs();
  AdjWs* w = c->adj;
  const int n = c->n, mb = c->mb;
  const bool lj = c->prm.potentials & MDG_POT_AIREBO_LJ;
  const int ccap = lj ? c->cij.cap : 0, tcap = lj ? c->spc.task_cap : 0;
  const long rcap = lj ? c->spc.rec_cap : 0;
  if (w->n == n && w->mb == mb && w->ccap == ccap && w->tcap == tcap && w->rcap == rcap) return MDG_OK;
  bool ok = adj_realloc(w->brv, (size_t)n * mb) && adj_realloc(w->bu, (size_t)n * mb) &&
            adj_realloc(w->bd, (size_t)n * mb) && adj_realloc(w->nco, (size_t)n) &&
            adj_realloc(w->A, (size_t)n * mb * 3) && adj_realloc(w->W, (size_t)n * mb) &&
            adj_realloc(w->er, (size_t)n) && adj_realloc(w->et, (size_t)n) && adj_realloc(w->el, (size_t)n) &&
            adj_realloc(w->dp, (size_t)n * kNParam) && adj_realloc(w->gown, (size_t)n) &&
            adj_realloc(w->glj, (size_t)n) && adj_realloc(w->g, (size_t)n) &&
            adj_realloc(w->cw, (size_t)n * (ccap > 0 ? ccap : 1)) &&
            adj_realloc(w->trec, (size_t)(rcap > 0 ? rcap : 1)) && adj_realloc(w->tmidc, (size_t)(tcap > 0 ? tcap : 1)) &&
            adj_realloc(w->tdp, (size_t)(tcap > 0 ? tcap : 1) * kNParam) &&
            adj_realloc(w->tmid, (size_t)(tcap > 0 ? tcap : 1)) && adj_realloc(w->tan, (size_t)n) &&
            adj_realloc(w->lx, (size_t)n) && adj_realloc(w->lv, (size_t)n) && adj_realloc(w->la, (size_t)n) &&
            adj_realloc(w->theta, kNParam) && adj_realloc(w->dpar, 2 * kNParam) &&
            adj_realloc(w->fin_pos, (size_t)n) && adj_realloc(w->fin_vel, (size_t)n) &&
            adj_realloc(w->fin_acc, (size_t)n) && adj_realloc(w->fin_img, (size_t)n);
  if (!ok) return fail(MDG_ERR_CUDA, "cudaMalloc (adjoint buffers)");
  // the glj of a context without the LJ term stays zero; no task holds a
  // middle bond before the first pass
  CK(cudaMemsetAsync(w->glj, 0, sizeof(dual4) * n, c->stream));
  CK(cudaMemsetAsync(w->tmid, 0, sizeof(int4) * (tcap > 0 ? tcap : 1), c->stream));
  w->n = n;
  w->mb = mb;
  w->ccap = ccap;
  w->tcap = tcap;
  w->rcap = rcap;
  w->have_fwd = false;
  w->cp_cap = 0;
  w->seg_cap = 0;
  return MDG_OK;
}

// One dual pass at the current positions (after evaluate(c) built the lists,
// the bond list, the connectivity table and the special-pair tasks there):
// w->g gets the gradient (values: the exact gradient of the energy) with
// tangents J^T tan (transpose = 1) or J tan (0); w->dp the per-atom
// dE/dtheta with tangents d/dtheta(tan . g).
int adj_dual_pass(mdg_ctx* c, int transpose = 1)
{
  AdjWs* w = c->adj;
  const int n = c->n;
  const int pot = c->prm.potentials;
  const bool rebo = pot & MDG_POT_REBO, tors = pot & MDG_POT_ETORS, lj = pot & MDG_POT_AIREBO_LJ;
  State S = c->S();
  BondList B = c->BL();
  DualBonds D{w->brv, w->bu, w->bd, w->nco};
  LAUNCH(c, "adj_bonds", k_adj_bonds, nblk(n), kThreads, S, w->tan, c->rp, B, D);
  BondListT<dual> DB;
  DB.n = n;
  DB.mb = c->mb;
  DB.nb = B.nb;
  DB.bj = B.bj;
  DB.brev = B.brev;
  DB.brv = w->brv;
  DB.bu = w->bu;
  DB.bd = w->bd;
  DB.nco = w->nco;
  ForceOutT<dual> O;
  O.mb = c->mb;
  O.A = w->A;
  O.W = w->W;
  O.gown = w->gown;
  O.glj = w->glj;
  O.e_rebo = w->er;
  O.e_tors = w->et;
  O.e_lj = w->el;
  O.dp = w->dp;
  O.jt = transpose;
  LAUNCH(c, "adj_rebo_tors", k_adj_rebo, nblk(n), kThreads, c->d_rp, c->d_tables, DB, c->tp, rebo ? 1 : 0,
         tors ? 1 : 0, O, c->d_status);
  SpecialTasksT<dual> Tk;
  std::memset(&Tk, 0, sizeof(Tk));
  if (lj) {
    CijTableT<dual> DT;
    DT.cap = c->cij.cap;
    DT.cnt = c->cij.cnt;
    DT.ent = c->cij.ent;
    DT.w = w->cw;
    DT.mask = c->cij.mask;
    LAUNCH(c, "adj_cij", k_adj_cij, nblk(n), kThreads, DB, c->cij, w->cw);
    LAUNCH(c, "adj_lj_plain", k_adj_lj_plain, nblk(n), kThreads, c->ljp, DT, S, c->nl[1], w->tan, O);
    const SpecialTasks& P = c->spc;
    Tk.cap = P.cap;
    Tk.task_cap = P.task_cap;
    Tk.rec_cap = P.rec_cap;
    Tk.cnt = P.cnt;
    Tk.part = P.part;
    Tk.off = P.off;
    Tk.flat = P.flat;
    Tk.trec = P.trec;
    Tk.ctr = P.ctr;
    Tk.rec = w->trec;
    Tk.mid = w->tmid;
    Tk.midc = w->tmidc;
    Tk.dp = w->tdp;
    LAUNCH(c, "adj_lj_special", k_adj_lj_special, c->special_blocks, kThreads, c->d_rp, c->d_tables, c->ljp, DB, DT,
           S, Tk, w->tan, c->d_status);
    LAUNCH(c, "adj_lj_reduce", k_adj_lj_reduce, nblk(n), kThreads, DB, Tk, O);
  }
  LAUNCH(c, "adj_gather", k_adj_gather, nblk(n), kThreads, DB, O, lj ? 1 : 0, Tk, w->g);
  return launch_check(c);
}

// Positions <- p (device), then a full FP64 evaluation there.
int adj_eval_at(mdg_ctx* c, const double4* p)
{
  if (p != c->pos) CK(cudaMemcpyAsync(c->pos, p, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice, c->stream));
  return evaluate(c);
}

int adj_step(mdg_ctx* c, double dt)
{
  StepDev sd;
  std::memset(&sd, 0, sizeof(sd));
  sd.dt = dt;
  sd.nlc0 = c->nl[0].cnt;
  return evaluate(c, &sd);  // position update, forces, velocity update (mdg_run's step, fixed dt)
}

template <class T>
int d2d(mdg_ctx* c, T* dst, const T* src, size_t count)
{
  CK(cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToDevice, c->stream));
  return MDG_OK;
}

int adj_save(mdg_ctx* c, int k)
{
  AdjWs* w = c->adj;
  const size_t n = c->n, o = (size_t)k * n;
  int rc = d2d(c, w->cp_pos + o, c->pos, n);
  if (!rc) rc = d2d(c, w->cp_vel + o, c->vel, n);
  if (!rc) rc = d2d(c, w->cp_acc + o, c->acc, n);
  if (!rc) rc = d2d(c, w->cp_img + o, c->image, n);
  return rc;
}

int adj_restore(mdg_ctx* c, const double4* p, const double4* v, const double4* a, const int4* im)
{
  const size_t n = c->n;
  int rc = d2d(c, c->pos, p, n);
  if (!rc) rc = d2d(c, c->vel, v, n);
  if (!rc) rc = d2d(c, c->acc, a, n);
  if (!rc) rc = d2d(c, c->image, im, n);
  c->acc_valid = true;
  return rc;
}

// Sums of the last pass's dE/dtheta into theta (scale_t on the tangents,
// scale_v on the values).
int adj_params(mdg_ctx* c, double scale_t, double scale_v)
{
  AdjWs* w = c->adj;
  LAUNCH(c, "adj_params", k_adj_par, kNParam, 128, w->dp, c->n, scale_t, scale_v, w->theta, w->dpar);
  return launch_check(c);
}

}  // namespace

extern "C" {

int mdg_set_param(mdg_ctx* c, int id, double value)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  if (id < 0 || id >= MDG_NPARAM) return fail(MDG_ERR_ARG, "unknown parameter id");
  if (!(std::isfinite(value) && value > 0.0)) return fail(MDG_ERR_ARG, "parameters must be finite and positive");
  if (id == MDG_PARAM_LJ_SIGMA_CC && c->prm.lj_cut_mode == 1 && c->n)
    return fail(MDG_ERR_STATE, "in the 3-sigma cutoff mode sigma_CC sets the LJ list range: set it before "
                               "mdg_set_system");
  const double v = value;
  switch (id) {
    case MDG_PARAM_LJ_EPS_CC: set_lj_cc(c->ljp, c->prm.lj_cut_mode, c->ljp.sigma[kC][kC], v); break;
    case MDG_PARAM_LJ_SIGMA_CC: set_lj_cc(c->ljp, c->prm.lj_cut_mode, v, c->ljp.eps[kC][kC]); break;
    case MDG_PARAM_REBO_A_CC: c->rp.A[kC][kC] = v; break;
    case MDG_PARAM_REBO_B1_CC: c->rp.B[0][kC][kC] = v; break;
    case MDG_PARAM_REBO_ALPHA_CC: c->rp.alpha[kC][kC] = v; break;
    case MDG_PARAM_REBO_BETA1_CC: c->rp.beta[0][kC][kC] = v; break;
  }
  CK(cudaMemcpyAsync(c->d_rp, &c->rp, sizeof(ReboParams), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // forces changed: the captured step (kernel arguments hold the LJ
  // parameters) and the stored accelerations are stale
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  c->step_graph = nullptr;
  c->acc_valid = false;
  if (c->adj) c->adj->have_fwd = false;
  return MDG_OK;
}

int mdg_get_param(mdg_ctx* c, int id, double* value)
{
  if (!c || !value) return fail(MDG_ERR_ARG, "null argument");
  switch (id) {
    case MDG_PARAM_LJ_EPS_CC: *value = c->ljp.eps[kC][kC]; break;
    case MDG_PARAM_LJ_SIGMA_CC: *value = c->ljp.sigma[kC][kC]; break;
    case MDG_PARAM_REBO_A_CC: *value = c->rp.A[kC][kC]; break;
    case MDG_PARAM_REBO_B1_CC: *value = c->rp.B[0][kC][kC]; break;
    case MDG_PARAM_REBO_ALPHA_CC: *value = c->rp.alpha[kC][kC]; break;
    case MDG_PARAM_REBO_BETA1_CC: *value = c->rp.beta[0][kC][kC]; break;
    default: return fail(MDG_ERR_ARG, "unknown parameter id");
  }
  return MDG_OK;
}

int mdg_force_product(mdg_ctx* c, const double* u, int transpose, double* ju, double* grad, double* de_dparam,
                      double* dprod_dparam)
{
  int rc = adj_check(c);
  if (rc) return rc;
  if (!u) return fail(MDG_ERR_ARG, "null direction");
  rc = evaluate(c);
  if (rc) return rc;
  rc = adj_ensure(c);
  if (rc) return rc;
  AdjWs* w = c->adj;
  const int n = c->n;
  std::vector<double4> h(n);
  for (int i = 0; i < n; i++) h[i] = make_double4(u[3 * i], u[3 * i + 1], u[3 * i + 2], 0.0);
  CK(cudaMemcpyAsync(w->tan, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, c->stream));
  rc = adj_dual_pass(c, transpose ? 1 : 0);
  if (rc) return rc;
  CK(cudaMemsetAsync(w->theta, 0, sizeof(double) * kNParam, c->stream));
  rc = adj_params(c, 0.0, 0.0);
  if (rc) return rc;
  std::vector<dual4> g(n);
  double dp[2 * kNParam];
  CK(cudaMemcpyAsync(g.data(), w->g, sizeof(dual4) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(dp, w->dpar, sizeof(dp), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  for (int i = 0; i < n; i++) {
    if (ju) { ju[3 * i] = g[i].x.d; ju[3 * i + 1] = g[i].y.d; ju[3 * i + 2] = g[i].z.d; }
    if (grad) { grad[3 * i] = g[i].x.v; grad[3 * i + 1] = g[i].y.v; grad[3 * i + 2] = g[i].z.v; }
  }
  for (int k = 0; k < kNParam; k++) {
    if (de_dparam) de_dparam[k] = dp[k];
    if (dprod_dparam) dprod_dparam[k] = dp[kNParam + k];
  }
  return MDG_OK;
}

int mdg_adjoint_forward(mdg_ctx* c, int nsteps, double dt, int every, double* pos, double* vel, double* epot)
{
  int rc = adj_check(c);
  if (rc) return rc;
  if (nsteps < 1 || every < 1) return fail(MDG_ERR_ARG, "nsteps and checkpoint_every must be positive");
  if (!(dt > 0.0)) return fail(MDG_ERR_ARG, "dt must be positive");
  rc = evaluate(c);  // sizes the special-pair tables before the dual buffers
  if (rc) return rc;
  rc = adj_ensure(c);
  if (rc) return rc;
  AdjWs* w = c->adj;
  const int n = c->n;
  const int ncp = (nsteps + every - 1) / every;  // checkpoints at steps 0, every, 2 every, ... < nsteps
  if (w->cp_cap < ncp) {
    if (!(adj_realloc(w->cp_pos, (size_t)ncp * n) && adj_realloc(w->cp_vel, (size_t)ncp * n) &&
          adj_realloc(w->cp_acc, (size_t)ncp * n) && adj_realloc(w->cp_img, (size_t)ncp * n)))
      return fail(MDG_ERR_CUDA, "cudaMalloc (checkpoints)");
    w->cp_cap = ncp;
  }
  if (w->seg_cap < every) {
    if (!adj_realloc(w->seg_pos, (size_t)every * n)) return fail(MDG_ERR_CUDA, "cudaMalloc (segment)");
    w->seg_cap = every;
  }
  // a_0 = A(x_0): the accelerations are a function of the initial positions
  State S = c->S();
  LAUNCH(c, "init_acc", k_init_acc, nblk(n), kThreads, S, c->grad, nullptr, nullptr);
  c->acc_valid = true;
  rc = adj_save(c, 0);
  for (int s = 1; s <= nsteps && !rc; s++) {
    rc = adj_step(c, dt);
    if (!rc && s % every == 0 && s < nsteps) rc = adj_save(c, s / every);
  }
  if (rc) return rc;
  rc = reduce_energies(c, c->d_energy, 0, 0, true);
  if (rc) return rc;
  rc = d2d(c, w->fin_pos, c->pos, n);
  if (!rc) rc = d2d(c, w->fin_vel, c->vel, n);
  if (!rc) rc = d2d(c, w->fin_acc, c->acc, n);
  if (!rc) rc = d2d(c, w->fin_img, c->image, n);
  if (rc) return rc;
  double e[4];
  CK(cudaMemcpyAsync(e, c->d_energy, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  w->have_fwd = true;
  w->nsteps = nsteps;
  w->every = every;
  w->ncp = ncp;
  w->dt = dt;
  if (epot) *epot = (e[0] + e[1]) + e[2];
  if (pos || vel) {
    std::vector<double> p((size_t)n * 3), v((size_t)n * 3);
    std::vector<int32_t> im((size_t)n * 3);
    rc = mdg_get_state(c, p.data(), v.data(), im.data());
    if (rc) return rc;
    for (int i = 0; i < n; i++)
      for (int a = 0; a < 3; a++) {
        const double L = c->box.pbc[a] ? c->box.L[a] : 0.0;
        if (pos) pos[3 * i + a] = p[3 * i + a] + im[3 * i + a] * L;
        if (vel) vel[3 * i + a] = v[3 * i + a];
      }
  }
  return MDG_OK;
}

int mdg_adjoint_backward(mdg_ctx* c, const double* seed_pos, const double* seed_vel, double seed_epot,
                         double* grad_params, double* grad_pos0, double* grad_vel0)
{
  int rc = adj_check(c);
  if (rc) return rc;
  AdjWs* w = c->adj;
  if (!w || !w->have_fwd) return fail(MDG_ERR_STATE, "mdg_adjoint_backward needs a preceding mdg_adjoint_forward");
  const int n = c->n, N = w->nsteps, C = w->every;
  const double dt = w->dt;
  std::vector<double4> h(n);
  for (int i = 0; i < n; i++)
    h[i] = seed_pos ? make_double4(seed_pos[3 * i], seed_pos[3 * i + 1], seed_pos[3 * i + 2], 0.0)
                    : make_double4(0.0, 0.0, 0.0, 0.0);
  CK(cudaMemcpyAsync(w->lx, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, c->stream));
  for (int i = 0; i < n; i++)
    h[i] = seed_vel ? make_double4(seed_vel[3 * i], seed_vel[3 * i + 1], seed_vel[3 * i + 2], 0.0)
                    : make_double4(0.0, 0.0, 0.0, 0.0);
  CK(cudaMemcpyAsync(w->lv, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));  // h is reused below
  CK(cudaMemsetAsync(w->la, 0, sizeof(double4) * n, c->stream));
  CK(cudaMemsetAsync(w->theta, 0, sizeof(double) * kNParam, c->stream));
  State S = c->S();
  const double cacc = kAccConv;
  // segments from the last to the first: [s0, s1] with s0 = k C
  for (int k = w->ncp - 1; k >= 0 && !rc; k--) {
    const int s0 = k * C, s1 = std::min(N, s0 + C);
    const size_t o = (size_t)k * n;
    rc = adj_restore(c, w->cp_pos + o, w->cp_vel + o, w->cp_acc + o, w->cp_img + o);
    for (int s = s0 + 1; s <= s1 && !rc; s++) {
      rc = adj_step(c, dt);
      if (!rc) rc = d2d(c, w->seg_pos + (size_t)(s - s0 - 1) * n, c->pos, (size_t)n);
    }
    for (int s = s1; s > s0 && !rc; s--) {
      // step s-1 -> s, products at x_s
      rc = adj_eval_at(c, w->seg_pos + (size_t)(s - s0 - 1) * n);
      if (rc) break;
      LAUNCH(c, "adj_dir", k_adj_dir, nblk(n), kThreads, S, w->lv, w->la, dt, 0, w->tan);
      rc = adj_dual_pass(c);
      if (rc) break;
      const double se = (s == N) ? seed_epot : 0.0;
      LAUNCH(c, "adj_update", k_adj_update, nblk(n), kThreads, S, w->g, w->lx, w->lv, w->la, dt, 0, se);
      rc = adj_params(c, -cacc, se);
    }
  }
  if (rc) return rc;
  // a_0 = A(x_0)
  rc = adj_eval_at(c, w->cp_pos);
  if (rc) return rc;
  LAUNCH(c, "adj_dir", k_adj_dir, nblk(n), kThreads, S, w->lv, w->la, dt, 1, w->tan);
  rc = adj_dual_pass(c);
  if (rc) return rc;
  LAUNCH(c, "adj_update", k_adj_update, nblk(n), kThreads, S, w->g, w->lx, w->lv, w->la, dt, 1, 0.0);
  rc = adj_params(c, -cacc, 0.0);
  if (rc) return rc;
  // leave the context at the forward run's final state
  rc = adj_restore(c, w->fin_pos, w->fin_vel, w->fin_acc, w->fin_img);
  if (rc) return rc;
  rc = evaluate(c);
  if (rc) return rc;
  double th[kNParam];
  CK(cudaMemcpyAsync(th, w->theta, sizeof(th), cudaMemcpyDeviceToHost, c->stream));
  if (grad_pos0) {
    CK(cudaMemcpyAsync(h.data(), w->lx, sizeof(double4) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < n; i++) {
      grad_pos0[3 * i] = h[i].x;
      grad_pos0[3 * i + 1] = h[i].y;
      grad_pos0[3 * i + 2] = h[i].z;
    }
  }
  if (grad_vel0) {
    CK(cudaMemcpyAsync(h.data(), w->lv, sizeof(double4) * n, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < n; i++) {
      grad_vel0[3 * i] = h[i].x;
      grad_vel0[3 * i + 1] = h[i].y;
      grad_vel0[3 * i + 2] = h[i].z;
    }
  }
  rc = read_status(c);
  if (rc) return rc;
  if (grad_params)
    for (int k = 0; k < kNParam; k++) grad_params[k] = th[k];
  return MDG_OK;
}

}  // extern "C"
