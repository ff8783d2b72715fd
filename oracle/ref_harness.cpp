/*
 * Oracle harness: a C ABI over the reference MDTK library compiled from its
 * own sources (test infrastructure only; loaded by tests/ and by bench.py's
 * CPU-baseline leg, never by the product).
 *
 * It drives the unmodified reference code:
 *   - potential stacks built as applications/common.h:36-77 does
 *     (REBO, REBO+AIREBO-LJ+ETors, Brenner set 1/2);
 *   - FProxy::operator() for energy and gradient (mdtk/potentials/FProxy.cxx:46-61);
 *   - NeighbourList::Update for the pair sets (mdtk/potentials/NeighbourList.cxx:32-107);
 *   - SimLoop::execute with dt fixed through the reference's own
 *     doBeforeIteration hook (mdtk/SimLoop.hpp:46, SimLoop.cxx:254) and file
 *     output off (SimLoop.hpp:49).
 * Units at this ABI: Angstrom, eV, fs, amu-free (masses are the reference's:
 * C 12 amu, H 1 amu, mdtk/Atom.hpp:104-105).  Conversions use the reference's
 * own constants (mdtk/consts.cxx:28-36).
 */
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <sstream>
#include <iostream>
#include <map>
#include <set>
#include <sys/time.h>
#include <unistd.h>

#include <mdtk/SimLoop.hpp>
#include <mdtk/SimLoopSaver.hpp>
#include <mdtk/SnapshotList.hpp>
#include <climits>
#include <sys/stat.h>
#include <mdtk/potentials/manybody/AIREBO/REBO.hpp>
#include <mdtk/potentials/manybody/AIREBO/AIREBO_LJ.hpp>
#include <mdtk/potentials/manybody/AIREBO/AIREBO_ETors.hpp>
#include <mdtk/potentials/manybody/Brenner/Brenner.hpp>
#include <mdtk/potentials/pairwise/FBZL.hpp>
#include <mdtk/potentials/pairwise/FLJ.hpp>
#include <mdtk/potentials/manybody/Ackland/Ackland.hpp>

using namespace mdtk;

namespace {

std::string g_last_error;

enum { POT_REBO = 1, POT_AIREBO_LJ = 2, POT_ETORS = 4, POT_BRENNER = 8, POT_METAL = 16, POT_GPU = 64 };

// Test support for the drop-in GPU classes (mdtk_b200/mdtk/GpuPotentials.hpp):
// the library that binds them (oracle/shim_harness.cpp) installs a factory
// here, and ref_create with POT_GPU builds its potential stack from it, in
// place of the reference's own classes, so that the unmodified FProxy and
// SimLoop drive the GPU path.  The factory adds the potentials to fpot and
// returns their names (comma-separated).
typedef const char* (*ref_gpu_factory_fn)(int potset, int brenner_set, int lj_cut_mode, mdtk::FProxy* fpot);
ref_gpu_factory_fn g_gpu_factory = 0;

double wall_now()
{
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

class FixedDtLoop : public SimLoop
{
public:
  Float fixed_dt;
  Float ekin_before;
  bool adaptive;  // leave dt to SimLoop's own adaptation (SimLoop.cxx:405-416)
  int max_iter;   // adaptive runs stop after this many iterations
  std::vector<double> epot_log, etot_log, t_log, dt_log;
  // mdtrajsim's CustomSimLoop (applications/mdtrajsim/main.cpp:36-90): its
  // SnapshotList and its doBeforeIteration, restated here because the
  // application's own potential set (applications/common.h:36-77) carries
  // metal potentials outside this path
  bool trajsim;
  SnapshotList snapshotList;
  FixedDtLoop()
    : SimLoop(), fixed_dt(0.5 * fs), ekin_before(0.0), adaptive(false), max_iter(0), trajsim(false), snapshotList()
  {
  }
  bool isItTimeToSave(Float interval)
  {
    return (simTime == 0.0 || int(simTime / interval) != int((simTime - dt_prev) / interval));
  }
  void trajsimBeforeIteration()
  {
    if (simTime < 2.0 * ps) simTimeSaveTrajInterval = 1.0 * ps;
    else simTimeSaveTrajInterval = 5.0 * ps;
    if (simTime < 2.0 * ps) {
      if (isItTimeToSave(5e-16 * 5 * 4)) snapshotList.getSnapshot(*this);
    } else {
      if (simTime < 4.0 * ps) {
        if (isItTimeToSave(5e-16 * 25 * 4)) snapshotList.getSnapshot(*this);
      } else {
        if (isItTimeToSave(5e-16 * 50 * 4)) snapshotList.getSnapshot(*this);
      }
    }
    if (iteration % iterationFlushStateInterval == 0 && iteration != 0) snapshotList.writestate();
  }
  virtual void doBeforeIteration()
  {
    if (trajsim) trajsimBeforeIteration();
    t_log.push_back(wall_now());
    if (!adaptive) dt = fixed_dt;
    dt_log.push_back(dt / fs);
    ekin_before = energyKin();
  }
  virtual void doAfterIteration()
  {
    // check.currentEnergy = Epot(x_{n+1}) + Ekin(v_n) (SimLoop.cxx:337 precedes :392)
    Float epot = check.currentEnergy - ekin_before;
    epot_log.push_back(epot / eV);
    etot_log.push_back((epot + energyKin()) / eV);
    if (adaptive && (int)epot_log.size() >= max_iter) breakSimLoop = true;
  }
};

struct RefCtx
{
  FixedDtLoop loop;
  int potset;
  int brenner_set;
  int lj_cut_mode;
  bool adaptive;
  bool keep_time;  // ref_run continues simTime and iteration (a resumed state)
  std::string out_dir;          // ref_run writes SimLoop's own files here (empty: none)
  long flush_interval;          // SimLoop::iterationFlushStateInterval for out_dir runs
  double traj_interval_fs;      // SimLoop::simTimeSaveTrajInterval for out_dir runs
  double dt0_fs;
  std::vector<std::string> names;
  REBO* rebo;
  AIREBO* lj;
  ETors* etors;
  Brenner* brenner;
  bool nl_ready;
  RefCtx() : potset(0), brenner_set(1), lj_cut_mode(0), adaptive(false), keep_time(false), flush_interval(1000000), traj_interval_fs(0.0), dt0_fs(0.5), rebo(0), lj(0), etors(0),
             brenner(0), nl_ready(false) {}
};

ElementID el_from_z(int z)
{
  switch (z) {
    case 1: return H_EL;
    case 6: return C_EL;
    case 29: return Cu_EL;
    case 47: return Ag_EL;
    case 79: return Au_EL;
    case 18: return Ar_EL;
    case 54: return Xe_EL;
  }
  throw Exception("unknown element (H, C, Cu, Ag, Au, Ar, Xe are on this path)");
}

int z_from_el(ElementID e)
{
  switch (e) {
    case H_EL: return 1;
    case C_EL: return 6;
    case Cu_EL: return 29;
    case Ag_EL: return 47;
    case Au_EL: return 79;
    case Ar_EL: return 18;
    case Xe_EL: return 54;
    default: return -1;
  }
}

void ensure_nl(RefCtx* c)
{
  if (c->nl_ready) return;
  c->loop.atoms.prepareForSimulatation();
  c->loop.fpot.NL_init(c->loop.atoms);
  c->loop.fpot.NL_UpdateIfNeeded(c->loop.atoms);
  c->nl_ready = true;
}

FGeneral* pot_at(RefCtx* c, int index)
{
  if (index < 0 || index >= (int)c->loop.fpot.potentials.size()) return 0;
  return c->loop.fpot.potentials[index];
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_last_error.c_str(); }

int ref_set_gpu_factory(ref_gpu_factory_fn f)
{
  g_gpu_factory = f;
  return 0;
}

void ref_set_verbose(int on) { yaatk::verboseTrace = (on != 0); }

/* potset: bitmask of REBO(1) | AIREBO_LJ(2) | ETORS(4) | BRENNER(8).
 * The AIREBO LJ term needs REBO (it holds a reference to it, AIREBO_LJ.cxx:204-212).
 * lj_cut_mode 0 = the reference's cosine cutoff (AIREBO_LJ.cxx:249-262);
 * lj_cut_mode 1 = cutoff at 3*sigma_CC/3*sigma_CH/3*sigma_HH with a 0.5 A switch. */
void* ref_create(int potset, int brenner_set, int lj_cut_mode)
{
  try {
    yaatk::verboseTrace = false;
    RefCtx* c = new RefCtx();
    c->potset = potset;
    c->brenner_set = brenner_set;
    c->lj_cut_mode = lj_cut_mode;
    c->loop.preventFileOutput = true;
    if (potset & POT_GPU) {
      if (!g_gpu_factory) throw Exception("no GPU potential factory installed");
      const char* names = g_gpu_factory(potset & ~POT_GPU, brenner_set, lj_cut_mode, &c->loop.fpot);
      if (!names) throw Exception("GPU potential factory failed");
      c->names.push_back(names);
      return c;
    }
    if (potset & POT_METAL) {
      // the ion and metal-hydrocarbon pair potentials first, as
      // setupPotentials adds them (applications/common.h:45-50)
      c->loop.fpot.addPotential(new FBZL(Rcutoff(5.0 * Ao, 5.5 * Ao)));
      c->names.push_back("FBZL");
      c->loop.fpot.addPotential(new FLJ(Rcutoff(5.0 * Ao, 5.5 * Ao)));
      c->names.push_back("FLJ");
    }
    if (potset & POT_REBO) {
      c->rebo = new REBO();
      c->loop.fpot.addPotential(c->rebo);
      c->names.push_back("REBO");
    }
    if (potset & POT_AIREBO_LJ) {
      if (!c->rebo) throw Exception("AIREBO LJ needs REBO");
      c->lj = new AIREBO(c->rebo);
      if (lj_cut_mode == 1) {
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++) {
            c->lj->R_[a][b][0] = 3.0 * c->lj->sigma_[a][b] - 0.5 * Ao;
            c->lj->R_[a][b][1] = 3.0 * c->lj->sigma_[a][b];
          }
        c->lj->nl.Rcutoff = c->lj->getRcutoff();
      }
      c->loop.fpot.addPotential(c->lj);
      c->names.push_back("AIREBO_LJ");
    }
    if (potset & POT_ETORS) {
      c->etors = new ETors();
      c->loop.fpot.addPotential(c->etors);
      c->names.push_back("ETors");
    }
    if (potset & POT_BRENNER) {
      c->brenner = new Brenner(brenner_set == 2 ? Brenner::POTENTIAL2 : Brenner::POTENTIAL1);
      c->loop.fpot.addPotential(c->brenner);
      c->names.push_back("Brenner");
    }
    if (potset & POT_METAL) {
      c->loop.fpot.addPotential(new Ackland());  // applications/common.h:62-63
      c->names.push_back("Ackland");
    }
    return c;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return 0;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return 0;
  }
}

void ref_destroy(void* h) { delete (RefCtx*)h; }

int ref_num_potentials(void* h) { return (int)((RefCtx*)h)->loop.fpot.potentials.size(); }

/* box[a] is the period along axis a in Angstrom; pbc_on[a] = 0 means NO_PBC on
 * that axis (mdtk/consts.cxx:40).  Positions in Angstrom, velocities in A/fs. */
int ref_set_atoms(void* h, int n, const int* z, const double* pos, const double* vel,
                  const double* box, const int* pbc_on, const unsigned char* fixed)
{
  RefCtx* c = (RefCtx*)h;
  try {
    c->loop.atoms.clear();
    c->loop.atoms.reserve(n);
    const Float vconv = Ao / fs;
    for (int i = 0; i < n; i++) {
      Atom a(el_from_z(z[i]),
             Vector3D(pos[3 * i] * Ao, pos[3 * i + 1] * Ao, pos[3 * i + 2] * Ao),
             vel ? Vector3D(vel[3 * i] * vconv, vel[3 * i + 1] * vconv, vel[3 * i + 2] * vconv)
                 : Vector3D(0, 0, 0));
      c->loop.atoms.push_back(a);
      if (fixed && fixed[i]) c->loop.atoms.back().fix();
    }
    Vector3D pbc(pbc_on[0] ? box[0] * Ao : NO_PBC.x,
                 pbc_on[1] ? box[1] * Ao : NO_PBC.y,
                 pbc_on[2] ? box[2] * Ao : NO_PBC.z);
    c->loop.atoms.PBC(pbc);
    c->nl_ready = false;
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* Energy (eV) and dE/dx (eV/A) through FProxy::operator().  e_terms[p] gets
 * each potential's energy and, when grad_terms is non-null, grad_terms[p*3n..]
 * its own gradient; grad gets the total.  Positions are read after the
 * reference's prepareForSimulatation wrap (applyPBC). */
int ref_compute(void* h, double* e_total, double* e_terms, double* grad, double* grad_terms)
{
  RefCtx* c = (RefCtx*)h;
  try {
    ensure_nl(c);
    AtomsArray& at = c->loop.atoms;
    const size_t n = at.size();
    const Float gconv = Ao / eV;
    Float etot = 0.0;
    for (size_t i = 0; i < n; i++) at[i].grad = Vector3D(0, 0, 0);
    std::vector<Vector3D> total(n, Vector3D(0, 0, 0));
    for (size_t p = 0; p < c->loop.fpot.potentials.size(); p++) {
      for (size_t i = 0; i < n; i++) at[i].grad = Vector3D(0, 0, 0);
      Float e = (*c->loop.fpot.potentials[p])(at);
      etot += e;
      if (e_terms) e_terms[p] = e / eV;
      for (size_t i = 0; i < n; i++) {
        total[i] += at[i].grad;
        if (grad_terms) {
          grad_terms[p * 3 * n + 3 * i + 0] = at[i].grad.x * gconv;
          grad_terms[p * 3 * n + 3 * i + 1] = at[i].grad.y * gconv;
          grad_terms[p * 3 * n + 3 * i + 2] = at[i].grad.z * gconv;
        }
      }
    }
    if (e_total) *e_total = etot / eV;
    if (grad)
      for (size_t i = 0; i < n; i++) {
        grad[3 * i + 0] = total[i].x * gconv;
        grad[3 * i + 1] = total[i].y * gconv;
        grad[3 * i + 2] = total[i].z * gconv;
      }
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* Energy through FProxy::operator() exactly (one summed value, as SimLoop sees it). */
int ref_energy_proxy(void* h, double* e_total, double* grad)
{
  RefCtx* c = (RefCtx*)h;
  try {
    ensure_nl(c);
    AtomsArray& at = c->loop.atoms;
    Float e = c->loop.fpot(at);
    if (e_total) *e_total = e / eV;
    if (grad)
      for (size_t i = 0; i < at.size(); i++) {
        grad[3 * i + 0] = at[i].grad.x * Ao / eV;
        grad[3 * i + 1] = at[i].grad.y * Ao / eV;
        grad[3 * i + 2] = at[i].grad.z * Ao / eV;
      }
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* Neighbour-list pairs (i<j) of potential `index` after a fresh build.
 * Writes up to cap pairs as (i, j) int32; returns the total count. */
long ref_nl_pairs(void* h, int index, int* pairs, long cap)
{
  RefCtx* c = (RefCtx*)h;
  try {
    ensure_nl(c);
    FGeneral* p = pot_at(c, index);
    if (!p) { g_last_error = "bad potential index"; return -1; }
    AtomsArray& at = c->loop.atoms;
    long cnt = 0;
    for (size_t i = 0; i < at.size(); i++) {
      AtomRefsContainer& l = p->nl.nl[i];
      for (size_t q = 0; q < l.size(); q++) {
        size_t j = l[q]->globalIndex;
        if (j <= i) continue;
        if (cnt < cap) { pairs[2 * cnt] = (int)i; pairs[2 * cnt + 1] = (int)j; }
        cnt++;
      }
    }
    return cnt;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* SimLoop's thermal bath (SimLoop.hpp:96-191): geom 0 none, 1 universe,
 * 2 box (params zMin, dBoundary, zMinOfFreeZone), 3 sphere (params cx, cy, cz,
 * radius, zMinOfFreeZone); lengths in Angstrom, T0 in K, gamma in 1/s;
 * flags: NULL or per-atom Atom::apply_ThermalBath (after ref_set_atoms). */
int ref_set_bath(void* h, int geom, double T0, double gamma, const double* params, const unsigned char* flags)
{
  RefCtx* c = (RefCtx*)h;
  SimLoop& L = c->loop;
  L.thermalBathGeomType = (SimLoop::TB_GEOM_TYPE)geom;
  L.thermalBathCommon.To = T0;
  L.thermalBathCommon.gamma = gamma;
  if (geom == 2) {
    L.thermalBathGeomBox.zMin = params[0] * Ao;
    L.thermalBathGeomBox.dBoundary = params[1] * Ao;
    L.thermalBathGeomBox.zMinOfFreeZone = params[2] * Ao;
  }
  if (geom == 3) {
    L.thermalBathGeomSphere.center = Vector3D(params[0] * Ao, params[1] * Ao, params[2] * Ao);
    L.thermalBathGeomSphere.radius = params[3] * Ao;
    L.thermalBathGeomSphere.zMinOfFreeZone = params[4] * Ao;
  }
  if (flags)
    for (size_t i = 0; i < L.atoms.size(); i++) L.atoms[i].apply_ThermalBath = flags[i] != 0;
  return 0;
}

/* Leave dt to SimLoop's adaptation (SimLoop.cxx:405-416) in ref_run, starting
 * from dt0 (fs), with timeaccel in Angstrom; off = the fixed dt of ref_run. */
int ref_set_adaptive(void* h, int on, double timeaccel, double dt0)
{
  RefCtx* c = (RefCtx*)h;
  c->adaptive = on != 0;
  c->dt0_fs = dt0;
  c->loop.timeaccel = timeaccel * Ao;
  return 0;
}

/* Per-iteration dt (fs) of the last ref_run. */
int ref_last_run_dts(void* h, double* out, int cap)
{
  FixedDtLoop& L = ((RefCtx*)h)->loop;
  int n = (int)L.dt_log.size();
  for (int i = 0; i < n && i < cap; i++) out[i] = L.dt_log[i];
  return n;
}

/* Override one C-C pair parameter (Angstrom / eV) of the potentials in place,
 * re-deriving what AIREBO::setupPotential derives from it
 * (AIREBO_LJ.cxx:229-262): id 0 = AIREBO zeta_[C][C], 1 = AIREBO
 * sigma_[C][C], 2 = REBO A_[C][C], 3 = REBO B_[0][C][C], 4 = REBO
 * alpha_[C][C], 5 = REBO beta_[0][C][C].  Test support for finite
 * differences of the reference with respect to its parameters. */
int ref_set_param(void* h, int id, double value)
{
  RefCtx* c = (RefCtx*)h;
  const int C = 0, H = 1;  // REBO::C, REBO::H (REBO.hpp:157-158)
  if (id <= 1 && !c->lj) { g_last_error = "no AIREBO LJ term"; return -1; }
  if (id >= 2 && !c->rebo) { g_last_error = "no REBO term"; return -1; }
  switch (id) {
    case 0:
    case 1: {
      AIREBO* a = c->lj;
      if (id == 0) a->zeta_[C][C] = value * eV;
      else a->sigma_[C][C] = value * Ao;
      a->sigma_[C][H] = 0.5 * (a->sigma_[C][C] + a->sigma_[H][H]);
      a->sigma_[H][C] = a->sigma_[C][H];
      a->zeta_[C][H] = sqrt(a->zeta_[C][C] * a->zeta_[H][H]);
      a->zeta_[H][C] = a->zeta_[C][H];
      for (int x = 0; x < 2; x++)
        for (int y = 0; y < 2; y++) {
          a->RLJ_[x][y][0] = a->sigma_[x][y];
          a->RLJ_[x][y][1] = a->sigma_[x][y] * pow(2.0, 1.0 / 6.0);
          if (c->lj_cut_mode == 1) {
            a->R_[x][y][0] = 3.0 * a->sigma_[x][y] - 0.5 * Ao;
            a->R_[x][y][1] = 3.0 * a->sigma_[x][y];
          }
        }
      if (c->lj_cut_mode == 1) {
        a->nl.Rcutoff = a->getRcutoff();
        c->nl_ready = false;
      }
      break;
    }
    case 2: c->rebo->A_[C][C] = value * eV; break;
    case 3: c->rebo->B_[0][C][C] = value * eV; break;
    case 4: c->rebo->alpha_[C][C] = value / Ao; break;
    case 5: c->rebo->beta_[0][C][C] = value / Ao; break;
    default: g_last_error = "unknown parameter id"; return -1;
  }
  return 0;
}

double ref_rcutoff(void* h, int index)
{
  FGeneral* p = pot_at((RefCtx*)h, index);
  return p ? p->getRcutoff() / Ao : -1.0;
}

/* Unmodified SimLoop::execute for nsteps steps of fixed dt (fs).  Returns the
 * final wrapped positions (A), velocities (A/fs), image counters, and per-step
 * potential and total energies (eV) with E_{n+1} = Epot(x_{n+1}) + Ekin(v_{n+1}). */
int ref_run(void* h, int nsteps, double dt_fs, double* pos, double* vel, int* image,
            double* epot_steps, double* etot_steps, double* e0)
{
  RefCtx* c = (RefCtx*)h;
  try {
    FixedDtLoop& L = c->loop;
    L.fixed_dt = dt_fs * fs;
    L.dt = L.fixed_dt;
    if (!c->keep_time) {
      L.simTime = 0.0;
      L.iteration = 0;
    }
    L.simTimeFinal = L.simTime + dt_fs * fs * (nsteps - 0.5);
    L.adaptive = c->adaptive;
    if (c->adaptive) {
      L.dt = c->dt0_fs * fs;
      L.simTimeFinal = 1e9 * ps;
      L.max_iter = nsteps;
      L.breakSimLoop = false;
    }
    L.simTimeSaveTrajInterval = 1e9 * ps;
    L.iterationFlushStateInterval = 1000000;
    char cwd[4096] = {0};
    const bool out = !c->out_dir.empty();
    if (out) {
      // SimLoop writes into the working directory (SimLoop.cxx:807-845, 1084-1092)
      if (!getcwd(cwd, sizeof(cwd)) || chdir(c->out_dir.c_str()) != 0) {
        g_last_error = "cannot enter " + c->out_dir;
        return -1;
      }
      L.preventFileOutput = false;
      L.iterationFlushStateInterval = c->flush_interval;
      if (c->traj_interval_fs > 0) L.simTimeSaveTrajInterval = c->traj_interval_fs * fs;
    }
    L.epot_log.clear();
    L.etot_log.clear();
    L.t_log.clear();
    L.dt_log.clear();
    double t_start = wall_now();
    int rc = L.execute();
    if (out) {
      L.preventFileOutput = true;
      if (chdir(cwd) != 0) { g_last_error = "cannot return to the working directory"; return -1; }
    }
    L.t_log.insert(L.t_log.begin(), t_start);
    L.t_log.push_back(wall_now());
    if (rc != 0) { g_last_error = "SimLoop::execute failed"; return -1; }
    if ((int)L.epot_log.size() != nsteps) {
      std::ostringstream os;
      os << "ran " << L.epot_log.size() << " steps instead of " << nsteps;
      g_last_error = os.str();
      return -1;
    }
    if (e0) *e0 = L.check.initialEnergy / eV;
    AtomsArray& at = L.atoms;
    const Float vconv = fs / Ao;
    for (size_t i = 0; i < at.size(); i++) {
      if (pos) { pos[3*i] = at[i].coords.x / Ao; pos[3*i+1] = at[i].coords.y / Ao; pos[3*i+2] = at[i].coords.z / Ao; }
      if (vel) { vel[3*i] = at[i].V.x * vconv; vel[3*i+1] = at[i].V.y * vconv; vel[3*i+2] = at[i].V.z * vconv; }
      if (image) { image[3*i] = at[i].PBC_count.x; image[3*i+1] = at[i].PBC_count.y; image[3*i+2] = at[i].PBC_count.z; }
    }
    for (int s = 0; s < nsteps; s++) {
      if (epot_steps) epot_steps[s] = L.epot_log[s];
      if (etot_steps) etot_steps[s] = L.etot_log[s];
    }
    c->nl_ready = true;
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // extern "C"

extern "C" {
/* Wall-clock stamps (s) of the last ref_run: [0] = entry to SimLoop::execute,
 * [1 + s] = start of iteration s (doBeforeIteration), [nsteps + 1] = return.
 * The list build and the initial energy evaluation happen between [0] and
 * the end of iteration 0.  Returns the number of stamps. */
int ref_last_run_times(void* h, double* out, int cap)
{
  RefCtx* c = (RefCtx*)h;
  int n = (int)c->loop.t_log.size();
  for (int i = 0; i < n && i < cap; i++) out[i] = c->loop.t_log[i];
  return n;
}
}  // extern "C"

/* ---- spline tables, in the layout the product builds its own copy in ----
 * Every stored coefficient is multiplier*c of one SplineTerm (the first factor
 * SplineTerm::operator() forms, mdtk/SplineAux.hpp:82-94), zero when either is
 * zero, in the SplineMultiD term order (x0 fastest, SplineAux.hpp:179-206). */

static void put_multi(const SplineMultiD& s, std::vector<double>& out, size_t nterms)
{
  for (size_t t = 0; t < nterms; t++) {
    if (t < s.terms.size()) {
      const SplineTerm& tt = s.terms[t];
      out.push_back((tt.multiplier == 0.0 || tt.c == 0.0) ? 0.0 : tt.multiplier * tt.c);
    } else out.push_back(0.0);
  }
}

static void put_G(const FuncG& g, std::vector<double>& out)
{
  // 4 pieces x (x1, x2, f[6], df[6])
  for (int p = 0; p < 4; p++) {
    if (p < g.splineCount) {
      out.push_back(g.spline[p].x_[0]);
      out.push_back(g.spline[p].x_[1]);
      put_multi(g.spline[p].f, out, 6);
      put_multi(g.spline[p].dfdx, out, 6);
    } else {
      for (int q = 0; q < 14; q++) out.push_back(0.0);
    }
  }
}

template <class FP>
static void put_P(const FP& f, std::vector<double>& out)
{
  for (int h = 0; h < 4; h++)
    for (int c = 0; c < 4; c++) {
      put_multi(f.spline[h][c].f, out, 16);
      put_multi(f.spline[h][c].dfdx, out, 16);
      put_multi(f.spline[h][c].dfdy, out, 16);
    }
}

template <class FP>
static void put_P_intarg(const FP& f, std::vector<double>& out)
{
  for (int h = 0; h < 4; h++)
    for (int c = 0; c < 4; c++) {
      out.push_back(f.intarg[h][c]);
      out.push_back(f.dH_intarg[h][c]);
      out.push_back(f.dC_intarg[h][c]);
    }
}

static void put_T(const Func_pi_rc& f, std::vector<double>& out)
{
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 16; k++) {
        put_multi(f.spline[i][j][k].f, out, 64);
        put_multi(f.spline[i][j][k].dfdx, out, 64);
        put_multi(f.spline[i][j][k].dfdy, out, 64);
        put_multi(f.spline[i][j][k].dfdz, out, 64);
      }
}

static void put_T_intarg(const Func_pi_rc& f, std::vector<double>& out)
{
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      for (int k = 0; k < 16; k++) {
        out.push_back(f.intarg[i][j][k]);
        out.push_back(f.di_intarg[i][j][k]);
        out.push_back(f.dj_intarg[i][j][k]);
        out.push_back(f.dk_intarg[i][j][k]);
      }
}

extern "C" {

/* which: 0 = REBO tables (G_C1, G_C2, G_H, P_CC, P_CH, P intarg CC/CH,
 *            pi_rc CC/CH/HH, Tij, their intarg tables);
 *        1 = Brenner tables of the given parameter set (H_CC, H_CH, F).
 * Returns the number of doubles (writes at most cap). */
long ref_tables(int which, int brenner_set, double* out, long cap)
{
  try {
    yaatk::verboseTrace = false;
    std::vector<double> v;
    if (which == 0) {
      REBO r;
      put_G(r.funcG_C1, v);
      put_G(r.funcG_C2, v);
      put_G(r.funcG_H, v);
      put_P(r.funcP_CC, v);
      put_P(r.funcP_CH, v);
      put_P_intarg(r.funcP_CC, v);
      put_P_intarg(r.funcP_CH, v);
      put_T(r.func_pi_rc_CC, v);
      put_T(r.func_pi_rc_CH, v);
      put_T(r.func_pi_rc_HH, v);
      put_T(r.func_Tij, v);
      put_T_intarg(r.func_pi_rc_CC, v);
      put_T_intarg(r.func_pi_rc_CH, v);
      put_T_intarg(r.func_pi_rc_HH, v);
      put_T_intarg(r.func_Tij, v);
    } else {
      Brenner b(brenner_set == 2 ? Brenner::POTENTIAL2 : Brenner::POTENTIAL1);
      for (int h = 0; h < 4; h++)
        for (int c = 0; c < 4; c++) {
          put_multi(b.funcH_CC.spline[h][c].f, v, 16);
          put_multi(b.funcH_CC.spline[h][c].dfdx, v, 16);
          put_multi(b.funcH_CC.spline[h][c].dfdy, v, 16);
        }
      for (int h = 0; h < 4; h++)
        for (int c = 0; c < 4; c++) {
          put_multi(b.funcH_CH.spline[h][c].f, v, 16);
          put_multi(b.funcH_CH.spline[h][c].dfdx, v, 16);
          put_multi(b.funcH_CH.spline[h][c].dfdy, v, 16);
        }
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
          for (int k = 0; k < 5; k++) {
            put_multi(b.funcF.spline[i][j][k].f, v, 64);
            put_multi(b.funcF.spline[i][j][k].dfdx, v, 64);
            put_multi(b.funcF.spline[i][j][k].dfdy, v, 64);
            put_multi(b.funcF.spline[i][j][k].dfdz, v, 64);
          }
    }
    for (long i = 0; i < (long)v.size() && i < cap; i++) out[i] = v[i];
    return (long)v.size();
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* Spline function values through the reference's own evaluators, for
 * known-answer checks: fn 0..2 = G_C1/G_C2/G_H(x0) value, 3..5 their dCosT;
 * 10/11/12 = P_CC value/dH/dC(x0,x1); 13/14/15 = P_CH;
 * 20+4f+d = pi_rc CC(f=0)/CH(1)/HH(2)/Tij(3), d = value/di/dj/dk at (x0,x1,x2). */
int ref_spline_eval(int fn, int n, const double* x, double* out)
{
  try {
    static REBO* r = 0;
    yaatk::verboseTrace = false;
    if (!r) r = new REBO();
    for (int q = 0; q < n; q++) {
      const double* a = x + 3 * q;
      double v = 0.0;
      if (fn == 0) v = r->funcG_C1(a[0]);
      else if (fn == 1) v = r->funcG_C2(a[0]);
      else if (fn == 2) v = r->funcG_H(a[0]);
      else if (fn == 3) v = r->funcG_C1.dCosT(a[0]);
      else if (fn == 4) v = r->funcG_C2.dCosT(a[0]);
      else if (fn == 5) v = r->funcG_H.dCosT(a[0]);
      else if (fn == 10) v = r->funcP_CC(a[0], a[1]);
      else if (fn == 11) v = r->funcP_CC.dH(a[0], a[1]);
      else if (fn == 12) v = r->funcP_CC.dC(a[0], a[1]);
      else if (fn == 13) v = r->funcP_CH(a[0], a[1]);
      else if (fn == 14) v = r->funcP_CH.dH(a[0], a[1]);
      else if (fn == 15) v = r->funcP_CH.dC(a[0], a[1]);
      else if (fn >= 20 && fn < 36) {
        int f = (fn - 20) / 4, d = (fn - 20) % 4;
        const Func_pi_rc* F = f == 0 ? (const Func_pi_rc*)&r->func_pi_rc_CC
                            : f == 1 ? (const Func_pi_rc*)&r->func_pi_rc_CH
                            : f == 2 ? (const Func_pi_rc*)&r->func_pi_rc_HH
                                     : (const Func_pi_rc*)&r->func_Tij;
        if (d == 0) v = (*F)(a[0], a[1], a[2]);
        else if (d == 1) v = F->di(a[0], a[1], a[2]);
        else if (d == 2) v = F->dj(a[0], a[1], a[2]);
        else v = F->dk(a[0], a[1], a[2]);
      } else { g_last_error = "bad spline id"; return -1; }
      out[q] = v;
    }
    return 0;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // extern "C"

extern "C" {
/* Compression of the reference's file streams: 0 plain, 1 ".gz" (zlib,
 * yaatk's gzip_internal), 2 ".xz" (the xz program).  yaatk picks its first
 * working method at start-up (yaatk.cxx:50); this overrides it. */
int ref_set_zip(int mode)
{
  if (mode == 0) yaatk::Stream::zipInvokeInfoGlobal = yaatk::Stream::ZipInvokeInfo("nozip", "");
  else if (mode == 1) yaatk::Stream::zipInvokeInfoGlobal = yaatk::Stream::ZipInvokeInfo("gzip_internal", ".gz");
  else if (mode == 2) yaatk::Stream::zipInvokeInfoGlobal = yaatk::Stream::ZipInvokeInfo("xz", ".xz");
  else return -1;
  return 0;
}

/* SimLoopSaver::write(id) of the current state (SimLoopSaver.cxx:118-231). */
int ref_write_state(void* h, const char* id)
{
  RefCtx* c = (RefCtx*)h;
  try {
    mdtk::SimLoopSaver saver(c->loop);
    return saver.write(id);
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* SimLoop::saveToStreamXVA into path (SimLoop.cxx:680-748), through the same
 * yaatk text stream writetrajXVA uses. */
int ref_write_xva(void* h, const char* path)
{
  RefCtx* c = (RefCtx*)h;
  try {
    c->loop.preventFileOutput = false;
    {
      yaatk::text_ofstream fo(path);
      c->loop.saveToStreamXVA(fo);
      fo.close();
    }
    c->loop.preventFileOutput = true;
    return 0;
  } catch (std::exception& e) {
    c->loop.preventFileOutput = true;
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    c->loop.preventFileOutput = true;
    g_last_error = e.what();
    return -1;
  }
}

/* SimLoopSaver::load(id) into an emptied atom array with SimLoop::iteration
 * = iteration (SimLoopSaver::loadIteration, SimLoopSaver.cxx:849-854);
 * later ref_run calls continue its time and iteration.  Returns the
 * LOADED_* bits or -1. */
int ref_load_state(void* h, const char* id, unsigned long iteration)
{
  RefCtx* c = (RefCtx*)h;
  try {
    c->loop.atoms.clear();
    mdtk::SimLoopSaver saver(c->loop);
    int got = saver.load(id);
    c->loop.iteration = iteration;
    c->nl_ready = false;
    c->keep_time = true;
    return got;
  } catch (std::exception& e) {
    g_last_error = e.what();
    return -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    return -1;
  }
}

/* Number of atoms, then per-atom state in Angstrom / (A/fs) / (A/fs^2):
 * coords, V, an, PBC_count, Atom::fixed, apply_ThermalBath, tag bits; any
 * NULL is skipped. */
int ref_atom_count(void* h) { return (int)((RefCtx*)h)->loop.atoms.size(); }

int ref_get_atoms(void* h, double* pos, double* vel, double* acc, int* image, unsigned char* fixed,
                  unsigned char* tb_apply, unsigned char* tags, int* z)
{
  RefCtx* c = (RefCtx*)h;
  AtomsArray& at = c->loop.atoms;
  const Float vconv = fs / Ao, aconv = fs * fs / Ao;
  for (size_t i = 0; i < at.size(); i++) {
    const Atom& a = at[i];
    if (pos) { pos[3*i] = a.coords.x / Ao; pos[3*i+1] = a.coords.y / Ao; pos[3*i+2] = a.coords.z / Ao; }
    if (vel) { vel[3*i] = a.V.x * vconv; vel[3*i+1] = a.V.y * vconv; vel[3*i+2] = a.V.z * vconv; }
    if (acc) { acc[3*i] = a.an.x * aconv; acc[3*i+1] = a.an.y * aconv; acc[3*i+2] = a.an.z * aconv; }
    if (image) { image[3*i] = a.PBC_count.x; image[3*i+1] = a.PBC_count.y; image[3*i+2] = a.PBC_count.z; }
    if (fixed) fixed[i] = a.isFixed() ? 1 : 0;
    if (tb_apply) tb_apply[i] = a.apply_ThermalBath ? 1 : 0;
    if (tags) {
      unsigned char t = 0;
      const unsigned bits[6] = {ATOMTAG_TARGET, ATOMTAG_PROJECTILE, ATOMTAG_SUBSTRATE, ATOMTAG_MONOMER,
                                ATOMTAG_CLUSTER, ATOMTAG_FULLERENE};
      for (int k = 0; k < 6; k++) if (a.hasTag(bits[k])) t |= (unsigned char)bits[k];
      tags[i] = t;
    }
    if (z) z[i] = z_from_el(a.ID);
  }
  return 0;
}

/* Per-atom tag bits (Atom::tag). */
int ref_set_tags(void* h, const unsigned char* tags)
{
  RefCtx* c = (RefCtx*)h;
  AtomsArray& at = c->loop.atoms;
  const unsigned bits[6] = {ATOMTAG_TARGET, ATOMTAG_PROJECTILE, ATOMTAG_SUBSTRATE, ATOMTAG_MONOMER,
                            ATOMTAG_CLUSTER, ATOMTAG_FULLERENE};
  for (size_t i = 0; i < at.size(); i++)
    for (int k = 0; k < 6; k++) {
      if (tags[i] & bits[k]) at[i].tag(bits[k]);
      else at[i].untag(bits[k]);
    }
  return 0;
}

/* SimLoop scalars: [0] simTime (fs), [1] dt (fs), [2] dt_prev (fs),
 * [3] iteration, [4] bath geometry, [5] To (K), [6] gamma (1/s),
 * [7..11] geometry parameters (A), [12..14] box (A, 0 = open axis),
 * [15..21] Check: netForce (eV/A x3), initialEnergy, currentEnergy,
 * energyTransferredFromBath (eV), currentTemperature (K). */
int ref_get_loop(void* h, double* out)
{
  RefCtx* c = (RefCtx*)h;
  FixedDtLoop& L = c->loop;
  out[0] = L.simTime / fs;
  out[1] = L.dt / fs;
  out[2] = L.dt_prev / fs;
  out[3] = (double)L.iteration;
  out[4] = (double)L.thermalBathGeomType;
  out[5] = L.thermalBathCommon.To;
  out[6] = L.thermalBathCommon.gamma;
  for (int k = 7; k < 12; k++) out[k] = 0.0;
  if (L.thermalBathGeomType == SimLoop::TB_GEOM_BOX) {
    out[7] = L.thermalBathGeomBox.zMin / Ao;
    out[8] = L.thermalBathGeomBox.dBoundary / Ao;
    out[9] = L.thermalBathGeomBox.zMinOfFreeZone / Ao;
  }
  if (L.thermalBathGeomType == SimLoop::TB_GEOM_SPHERE) {
    out[7] = L.thermalBathGeomSphere.center.x / Ao;
    out[8] = L.thermalBathGeomSphere.center.y / Ao;
    out[9] = L.thermalBathGeomSphere.center.z / Ao;
    out[10] = L.thermalBathGeomSphere.radius / Ao;
    out[11] = L.thermalBathGeomSphere.zMinOfFreeZone / Ao;
  }
  const Vector3D pbc = L.atoms.PBC();
  out[12] = pbc.x != NO_PBC.x ? pbc.x / Ao : 0.0;
  out[13] = pbc.y != NO_PBC.y ? pbc.y / Ao : 0.0;
  out[14] = pbc.z != NO_PBC.z ? pbc.z / Ao : 0.0;
  out[15] = L.check.netForce.x * Ao / eV;
  out[16] = L.check.netForce.y * Ao / eV;
  out[17] = L.check.netForce.z * Ao / eV;
  out[18] = L.check.initialEnergy / eV;
  out[19] = L.check.currentEnergy / eV;
  out[20] = L.check.energyTransferredFromBath / eV;
  out[21] = L.check.currentTemperature;
  return 0;
}
}  // extern "C"

extern "C" {
/* Let ref_run write SimLoop's own state and XVA files into dir (NULL: none),
 * with iterationFlushStateInterval = flush_interval and
 * simTimeSaveTrajInterval = traj_interval_fs (fs; 0 keeps it out of reach). */
int ref_set_output(void* h, const char* dir, long flush_interval, double traj_interval_fs)
{
  RefCtx* c = (RefCtx*)h;
  c->out_dir = dir ? dir : "";
  c->flush_interval = flush_interval > 0 ? flush_interval : 1000000;
  c->traj_interval_fs = traj_interval_fs;
  return 0;
}
}  // extern "C"

extern "C" {
/* mdtrajsim's impact-sequence mode (applications/mdtrajsim/main.cpp:295-345)
 * with its runTraj (main.cpp:113-180), on this harness's potential set:
 * load the base state, and for each (x, y) of ionpos.bin from impact
 * `start` on, in workdir/%08d: place the last atom (the projectile) there,
 * record ionpos_used.bin/.txt, write the state, run SimLoop (adaptive dt)
 * to the base's simTimeFinal with CustomSimLoop's snapshots and intervals,
 * write the final state, snapshots.conf and completed.ok, and keep only the
 * last state.  Files go through yaatk's streams (compression as ref_set_zip).
 * Directory changes do not redirect the standard streams (yaatk::ChDir's
 * stdout.txt/stderr.txt logs are not made). */
int ref_impact_sequence(int potset, const char* base_id, const char* ionpos_path, const char* workdir, int start)
{
  char cwd[4096] = {0};
  if (!getcwd(cwd, sizeof(cwd))) { g_last_error = "getcwd"; return -1; }
  RefCtx* base = (RefCtx*)ref_create(potset, 1, 0);
  if (!base) return -1;
  int rc = 0;
  try {
    mdtk::SimLoopSaver mds(base->loop);
    int got = mds.load(base_id);
    REQUIRE(got & mdtk::SimLoopSaver::LOADED_R);
    double bombX, bombY;
    yaatk::binary_ifstream ionpos_bin(ionpos_path);
    int recordLength = ionpos_bin.getDataLength();
    REQUIRE(recordLength % (sizeof(bombX) + sizeof(bombY)) == 0);
    int impactCount = recordLength / (sizeof(bombX) + sizeof(bombY));
    for (int impact = 0; impact < impactCount; ++impact) {
      YAATK_BIN_READ(ionpos_bin, bombX);
      YAATK_BIN_READ(ionpos_bin, bombY);
      Atom& projectile = base->loop.atoms.back();
      projectile.coords.x = bombX;
      projectile.coords.y = bombY;
      if (impact < start) continue;
      char name[64];
      sprintf(name, "%08d", impact);
      const std::string dir = std::string(workdir) + "/" + name;
      ::mkdir(dir.c_str(), 0755);
      if (chdir(dir.c_str()) != 0) throw Exception("cannot enter " + dir);
      if (yaatk::exists("completed.ok") || yaatk::exists("completed.error")) {
        if (chdir(cwd) != 0) throw Exception("chdir");
        continue;
      }
      {
        yaatk::binary_ofstream ionpos_used_bin("ionpos_used.bin");
        yaatk::text_ofstream ionpos_used_txt("ionpos_used.txt");
        YAATK_BIN_WRITE(ionpos_used_bin, bombX);
        YAATK_BIN_WRITE(ionpos_used_bin, bombY);
        ionpos_used_txt << bombX << " " << bombY << "\n";
        ionpos_used_bin.close();
        ionpos_used_txt.close();
      }
      base->loop.simTimeSaveTrajInterval = 1e6 * ps;
      mds.write();
      {
        // runTraj
        RefCtx* t = (RefCtx*)ref_create(potset, 1, 0);
        if (!t) throw Exception(g_last_error);
        try {
          mdtk::SimLoopSaver tm(t->loop);
          if (tm.listIterations().size() > 0) tm.loadIterationLatest();
          if (yaatk::exists("snapshots.conf")) t->loop.snapshotList.loadstate();
          t->loop.iterationFlushStateInterval = 1000;
          t->loop.trajsim = true;
          t->loop.adaptive = true;
          t->loop.max_iter = INT_MAX;
          t->loop.preventFileOutput = false;
          t->loop.execute();
          tm.write();
          t->loop.snapshotList.writestate();
          if (t->loop.simTime >= t->loop.simTimeFinal) {
            yaatk::text_ofstream fo2("completed.ok");
            fo2.close();
            tm.removeIterations();
          }
        } catch (...) {
          delete t;
          throw;
        }
        delete t;
      }
      mds.removeIterations(false, true);
      if (chdir(cwd) != 0) throw Exception("chdir");
    }
    ionpos_bin.close();
  } catch (std::exception& e) {
    g_last_error = e.what();
    rc = -1;
    if (chdir(cwd) != 0) rc = -1;
  } catch (yaatk::Exception& e) {
    g_last_error = e.what();
    rc = -1;
    if (chdir(cwd) != 0) rc = -1;
  }
  delete base;
  return rc;
}
}  // extern "C"

extern "C" {
/* SimLoop::simTime, simTimeFinal and dt (fs), e.g. of a base state to write. */
int ref_set_time(void* h, double time_fs, double time_final_fs, double dt_fs)
{
  RefCtx* c = (RefCtx*)h;
  c->loop.simTime = time_fs * fs;
  c->loop.simTimeFinal = time_final_fs * fs;
  c->loop.dt = dt_fs * fs;
  c->loop.dt_prev = dt_fs * fs;
  return 0;
}
}  // extern "C"
