/*
 * mdg: B200-native MDTK hot path (REBO / Brenner bond-order forces, AIREBO
 * Lennard-Jones and torsion terms, Verlet neighbour lists, velocity Verlet)
 * behind a plain C ABI.
 *
 * Every entry point returns an int status (MDG_OK = 0, negative = error) and
 * never throws; mdg_last_error() returns the message of the last failure on
 * the calling thread.  Contexts are independent; a context is used by one
 * host thread at a time.
 *
 * The entry points replace the reference's potential interface
 * (mdtk/potentials/FGeneral.hpp:54-114, aggregated by FProxy,
 * mdtk/potentials/FProxy.hpp:31-112) and the SimLoop step body
 * (mdtk/SimLoop.cxx:252-445); each declaration names the reference function
 * it stands in for.
 */
#ifndef MDG_H
#define MDG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdg_ctx mdg_ctx;

/* ---- status codes ---- */
#define MDG_OK 0
#define MDG_ERR_ARG (-1)            /* bad argument (replaces REQUIRE on inputs) */
#define MDG_ERR_CUDA (-2)           /* CUDA runtime failure or no device */
#define MDG_ERR_NL_OVERFLOW (-3)    /* a Verlet list exceeded its capacity */
#define MDG_ERR_BOND_OVERFLOW (-4)  /* an atom has more REBO bonds than the bond capacity */
#define MDG_ERR_COS_RANGE (-5)      /* cos(theta) outside [-1-1e-7, 1+1e-7] (FGeneral.hpp:147) */
#define MDG_ERR_N_NEGATIVE (-6)     /* coordination below -1e-15 (REBO.cxx:434) */
#define MDG_ERR_NONFINITE (-7)      /* non-finite energy or force */
#define MDG_ERR_CAPACITY (-8)       /* connectivity / special-pair / record capacity exceeded */
#define MDG_ERR_SPLINE_DOMAIN (-9)  /* spline argument out of its domain (cubici.hpp:90,211,305) */
#define MDG_ERR_STATE (-10)         /* call out of order (e.g. compute before set_system) */
#define MDG_ERR_TIMEOUT (-11)       /* a bounded device wait gave up */
#define MDG_ERR_IO (-12)            /* a checkpoint or trajectory file could not be read or written */

/* ---- potential selection (bitmask) ---- */
#define MDG_POT_REBO 1        /* REBO (AIREBO/REBO.cxx) */
#define MDG_POT_AIREBO_LJ 2   /* AIREBO LJ term (AIREBO/AIREBO_LJ.cxx); needs MDG_POT_REBO */
#define MDG_POT_ETORS 4       /* AIREBO torsion (AIREBO/AIREBO_ETors.cxx) */
#define MDG_POT_BRENNER 8     /* first-generation Brenner (Brenner/Brenner.cxx) */
#define MDG_POT_METAL 16      /* the metal and ion potentials of applications/common.h:36-77:
                                 FBZL (pairwise/FBZL.cxx: Ar, Xe ions with every element),
                                 FLJ (pairwise/FLJ.cxx: H, C with Cu, Au) and Ackland
                                 (manybody/Ackland/Ackland.cxx: Cu, Ag, Au); needed for any
                                 atom other than H and C */
#define MDG_POT_AIREBO (MDG_POT_REBO | MDG_POT_AIREBO_LJ | MDG_POT_ETORS)

/* ---- units at this ABI ---- */
#define MDG_UNITS_AEVFS 0  /* Angstrom, Angstrom/fs, eV, eV/Angstrom, fs */
#define MDG_UNITS_CGS 1    /* cm, cm/s, erg, erg/cm, s (the reference's units) */

/* ---- precision ---- */
#define MDG_PREC_FP64 0        /* everything in FP64 */
#define MDG_PREC_FP32_MIXED 1  /* FP32 bond-order / LJ arithmetic, FP64 accumulation and integration */

typedef struct mdg_params {
  int potentials;     /* MDG_POT_* bitmask */
  int brenner_set;    /* Brenner parameter set 1 or 2 (Brenner::POTENTIAL1/2); Brenner excludes
                         REBO and the LJ term in one context (the LJ term is built on REBO) */
  int precision;      /* MDG_PREC_* */
  int units;          /* MDG_UNITS_* */
  int lj_cut_mode;    /* 0: reference cosine cutoff 5.0-5.5/4.5-5.0/4.0-4.5 A; 1: 3 sigma */
  int nl_skin_mode;   /* 0: list range 1.44 Rcut, rebuild at 0.44 Rcut (NeighbourList.cxx:29);
                         1: list range Rcut + nl_skin, rebuild at nl_skin */
  double nl_skin;     /* absolute skin in Angstrom for nl_skin_mode 1 */
  int cap_rebo_list;  /* Verlet-list capacities (partners per atom); 0 = default */
  int cap_lj_list;
  int cap_bonds;      /* REBO bonds per atom; 0 = default (16) */
  int cap_cij;        /* connectivity targets per atom; 0 = default */
  int cap_special;    /* LJ pairs per atom that need b*_ij or a connectivity gradient;
                         0 = default (64) */
  int special_avg;    /* capacity of those pairs over the whole system, per atom on average;
                         0 = default (48) */
  int device;         /* CUDA device ordinal */
  int bond_rec_avg;   /* capacity of the per-bond REBO records over the whole system, doubles per
                         atom on average (a bond slot of an atom with b bonds takes 5 + 4b, and in
                         the lane-pair split each C-C bond adds a torsion record of that size);
                         0 = default (256: five bonds per atom in every split) */
  int task_mode;      /* REBO work split: 1 = one task per directed bond (both ends evaluate each
                         bond, shortest critical path), 2 = one task per bond writing both ends'
                         records (half the work), 3 = per bond on a pair of lanes, each lane the
                         bond-order terms of one end, and the torsion of each C-C bond a task of
                         its own (a bond's serial chain about halved); 0 = timed once per system
                         on the first mdg_run (the autotuner) and the fastest kept.  All route the
                         same terms into the same records; results agree to rounding (the kernels
                         may contract multiply-adds differently and mode 3 adds an end's pieces in
                         two sums).  With the LJ term the launch configuration (stream overlap,
                         REBO grid) is timed on the first mdg_run in every mode; it never changes
                         results. */
} mdg_params;

/* Fill *p with the defaults: REBO only, FP64, Angstrom/eV/fs, reference cutoffs and skin. */
void mdg_default_params(mdg_params* p);

/* Create a context (replaces constructing the potentials: REBO::REBO
 * REBO.cxx:816-854, AIREBO::AIREBO AIREBO_LJ.cxx:204-212, ETors::ETors
 * AIREBO_ETors.cxx:117-122, Brenner::Brenner Brenner.cxx:474-496; the spline
 * tables are built once on the host and uploaded). */
int mdg_create(const mdg_params* p, mdg_ctx** out);

/* Free every device and host resource of the context (FProxy::freePotentials,
 * FProxy.hpp:49-53). */
int mdg_destroy(mdg_ctx* ctx);

/* Message of the last error on this thread (yaatk::Exception::what). */
const char* mdg_last_error(void);

/* Launch all work on this CUDA stream (cudaStream_t passed as void*; NULL =
 * the context's own stream). */
int mdg_set_stream(mdg_ctx* ctx, void* stream);

/* Elements (z): H 1, C 6 (REBO, AIREBO, Brenner); Cu 29, Ag 47, Au 79 and
 * the ions Ar 18, Xe 54 (MDG_POT_METAL).  REBO and AIREBO see hydrocarbon
 * pairs only; the metal potentials every pair with a metal or ion atom.
 * mdg_compute's e_terms[3] is the metal and ion energy. */

/* Load an atom set (AtomsArray with its PBC, AtomsContainer.hpp:31-104, plus
 * AtomsArray::prepareForSimulatation AtomsContainer.cxx:107-123: positions are
 * wrapped into the box on periodic axes and image counters start at 0).
 * z: atomic numbers (1 = H, 6 = C); pos, vel: [n*3]; box: periods;
 * pbc[a] != 0 marks a periodic axis; fixed: NULL or [n] flags (Atom::fix).
 * Neighbour lists are built on the next evaluation (FGeneral::NL_init). */
int mdg_set_system(mdg_ctx* ctx, int n, const int32_t* z, const double* pos, const double* vel,
                   const double box[3], const int32_t pbc[3], const uint8_t* fixed);

/* Replace positions (same atoms, same order).  Lists are rebuilt only when
 * the displacement criterion fires (NeighbourList::MovedTooMuch,
 * NeighbourList.cxx:109-133). */
int mdg_set_positions(mdg_ctx* ctx, const double* pos);

/* Verlet-list maintenance at the current positions (FGeneral::NL_init,
 * NL_checkRequestUpdate and NL_UpdateIfNeeded, FGeneral.hpp:71-91, over
 * NeighbourList::Update / MovedTooMuch, NeighbourList.cxx:32-133).  force = 0:
 * each list is rebuilt when the two largest displacements since its last
 * build exceed its trigger (0.44 Rcut, or the absolute skin); force != 0:
 * every list is rebuilt.  Displacements are measured on the device from the
 * positions themselves, so FGeneral::incDisplacement has no counterpart.
 * rebuilt: NULL or [3], set to 1 for each list (0 REBO/Brenner/torsion,
 * 1 AIREBO LJ, 2 metal) that was rebuilt, else 0.  mdg_compute and mdg_run
 * perform the same check on their own. */
int mdg_nl_update(mdg_ctx* ctx, int force, int32_t* rebuilt);

/* Energy and gradient of the configured potentials at the current positions
 * (FProxy::operator(), FProxy.cxx:46-61).  e_total: total energy; e_terms
 * (NULL or [4]): REBO or Brenner, AIREBO LJ, torsion, 0; grad (NULL or [n*3]):
 * dE/dx is ADDED into it, as each potential adds into Atom::grad. */
int mdg_compute(mdg_ctx* ctx, double* e_total, double* e_terms, double* grad);

/* Sorted (i < j) pairs of a Verlet list after the last build: list_id 0 =
 * REBO/Brenner/torsion list, 1 = AIREBO LJ list (NeighbourList::nl,
 * NeighbourList.hpp:41-83).  Writes min(count, cap) pairs as int32 (i, j);
 * *count gets the total. */
int mdg_nl_pairs(mdg_ctx* ctx, int list_id, int32_t* pairs, int64_t cap, int64_t* count);

/* Advance nsteps velocity-Verlet steps of fixed dt entirely on the device
 * (SimLoop::executeMain step body, SimLoop.cxx:252-445, with dt fixed, no
 * thermal bath).  epot/etot: NULL or [nsteps] per-step potential / total
 * energies E(x_{n+1}, v_{n+1}).  Asynchronous on the context stream unless an
 * energy array or a status check needs the host: pass NULL arrays and call
 * mdg_sync() to collect the status. */
int mdg_run(mdg_ctx* ctx, int nsteps, double dt, double* epot, double* etot);

/* Wait for the context stream and report any device-side status. */
int mdg_sync(mdg_ctx* ctx);

/* Copy the state back (SimLoop atoms: coords, V, PBC_count).  Any NULL is skipped. */
int mdg_get_state(mdg_ctx* ctx, double* pos, double* vel, int32_t* image);

/* Replace positions and velocities of the loaded atoms (same order) from
 * host memory; used by drivers that keep the state on the host. */
int mdg_set_state(mdg_ctx* ctx, const double* pos, const double* vel);

/* Advance nsteps steps from a host-held state (pos, vel [n*3], updated in
 * place with the final state; epot/etot as in mdg_run): the state is copied to
 * the device, stepped there, and copied back.  This is SimLoop::execute on
 * caller-owned AtomsArray data (SimLoop.cxx:141-206) for drivers that keep
 * the atoms on the host between calls. */
int mdg_step_host(mdg_ctx* ctx, int nsteps, double dt, double* pos, double* vel, double* epot, double* etot);

/* Number of kernels this context has launched so far. */
int64_t mdg_launch_count(mdg_ctx* ctx);

/* Per-kernel timing: while on, every launch is bracketed by CUDA events on
 * the launch stream.  mdg_profile_read waits for the stream and returns, for
 * up to max kernel names (32-byte NUL-terminated slots in names), the summed
 * milliseconds and launch counts since profiling was switched on or last
 * read; *nout gets the number of distinct kernels.  No reference counterpart
 * (the reference times whole runs with procmon, mdtk/procmon.hpp:99-131). */
int mdg_set_profiling(mdg_ctx* ctx, int on);
int mdg_profile_read(mdg_ctx* ctx, int max, char* names, double* ms, int64_t* counts, int* nout);

/* Measured FMA throughput of the FP64 (fp32 = 0) or FP32 (fp32 = 1) CUDA-core
 * pipe of a device in TFLOP/s (2 flops per FMA): the roofline denominator for
 * the bond-order kernels.  No reference counterpart. */
int mdg_pipe_peak(int device, int fp32, double* tflops);

/* The floor of one step of `phases` dependent phases that do no work, on
 * `device`, two ways: a CUDA graph of `phases` empty kernels, each a
 * programmatic dependent launch (how mdg_run's steps are launched), and one
 * cooperative kernel with a grid-wide barrier between its phases (a
 * persistent fused step); both over two blocks per SM, microseconds per step
 * (best of three 200-step samples).  A diagnostic with no reference
 * counterpart: it bounds what fusing a step's kernels could save. */
int mdg_launch_floor(int device, int phases, double* graph_us, double* coop_us);

/* ---- Parameters and the adjoint ----
 * The adjoint differentiates a velocity-Verlet trajectory (the step of
 * mdg_run) with respect to the initial positions and velocities and to the
 * C-C pair parameters below; derived C-H / H-H parameters follow them as
 * AIREBO::setupPotential derives them (AIREBO_LJ.cxx:229-247).  No
 * counterpart in the reference (which has no gradients of trajectories);
 * the parameters are those of REBO::setupPotential1 (REBO.cxx:859-938) and
 * AIREBO::setupPotential (AIREBO_LJ.cxx:229-236), in Angstrom / eV. */
#define MDG_PARAM_LJ_EPS_CC 0      /* AIREBO zeta_[C][C] (eV) */
#define MDG_PARAM_LJ_SIGMA_CC 1    /* AIREBO sigma_[C][C] (Angstrom) */
#define MDG_PARAM_REBO_A_CC 2      /* REBO A_[C][C] (eV) */
#define MDG_PARAM_REBO_B1_CC 3     /* REBO B_[0][C][C] (eV) */
#define MDG_PARAM_REBO_ALPHA_CC 4  /* REBO alpha_[C][C] (1/Angstrom) */
#define MDG_PARAM_REBO_BETA1_CC 5  /* REBO beta_[0][C][C] (1/Angstrom) */
#define MDG_NPARAM 6

/* Set / read one parameter (Angstrom / eV).  Setting invalidates the stored
 * accelerations and the captured step.  In the 3-sigma cutoff mode sigma_CC
 * also sets the LJ list range and must be set before mdg_set_system. */
int mdg_set_param(mdg_ctx* ctx, int id, double value);
int mdg_get_param(mdg_ctx* ctx, int id, double* value);

/* Products of the force field's derivatives at the current positions, for a
 * direction u [n*3]: ju = J^T u (transpose != 0, what the adjoint uses) or
 * J u (transpose = 0, the tangent-linear product) with J = d(grad)/dx the
 * Jacobian of the gradient mdg_compute returns; grad = the exact gradient of
 * the energy (it differs from mdg_compute's only by the reference's torsion
 * derivative, AIREBO_ETors.cxx:110), de_dparam [MDG_NPARAM] = dE/dtheta and
 * dprod_dparam [MDG_NPARAM] = d(u . grad)/dtheta.  Any output may be NULL.
 * FP64 single-system REBO (+LJ) (+torsion) contexts in Angstrom/eV/fs. */
int mdg_force_product(mdg_ctx* ctx, const double* u, int transpose, double* ju, double* grad, double* de_dparam,
                      double* dprod_dparam);

/* Forward run of the adjoint: nsteps velocity-Verlet steps of dt from the
 * current state (the accelerations are recomputed from the positions first),
 * keeping the state every checkpoint_every steps on the device.  Outputs (any
 * may be NULL): pos [n*3] final positions UNWRAPPED (box position plus image
 * count times the period), vel [n*3], epot = E_pot(x_N).  The context ends at
 * the final state. */
int mdg_adjoint_forward(mdg_ctx* ctx, int nsteps, double dt, int checkpoint_every, double* pos, double* vel,
                        double* epot);

/* Backward run for a loss L(x_N, v_N, E_pot(x_N)) of the last forward run:
 * seeds dL/dx_N [n*3] and dL/dv_N [n*3] (NULL = zero) and dL/dE_pot.
 * Outputs (any may be NULL): grad_params [MDG_NPARAM] = dL/dtheta,
 * grad_pos0 = dL/dx_0, grad_vel0 = dL/dv_0.  Each segment between
 * checkpoints is recomputed from its checkpoint; the context ends at the
 * forward run's final state. */
int mdg_adjoint_backward(mdg_ctx* ctx, const double* seed_pos, const double* seed_vel, double seed_epot,
                         double* grad_params, double* grad_pos0, double* grad_vel0);

/* REBO energy and gradient (plus the torsion term when with_torsion != 0)
 * for callers that cannot allocate device memory: hosts whose device memory
 * is all owned by their own allocator, which forbids driver allocations by
 * plugins, and time-critical loops that cannot afford the device-wide
 * synchronisation cudaMalloc/cudaFree imply.  Nothing is allocated: every
 * intermediate lives in a fixed static device array (about 11 MiB, held by
 * every GPU that loads the library until the process exits), so n is limited
 * to 4096 atoms; larger n is rejected with MDG_ERR_ARG.  pos (n*3, Angstrom),
 * z (n atomic numbers), energy (2 doubles: REBO, torsion, eV) and grad (n*3,
 * eV/Angstrom, overwritten) are DEVICE pointers owned by the caller; box and
 * pbc are host arrays.  Work runs on `stream` (cudaStream_t as void*; NULL =
 * legacy default stream) and the call waits for it to report the status.
 * The first call on a device sets that device up with synchronous copies, so
 * make it before any stream capture.  Calls share the one scratch array:
 * calls that overlap on the GPU race.  No counterpart in the reference. */
int mdg_rebo_compute_noalloc(int n, const double* pos, const int32_t* z, const double box[3], const int32_t pbc[3],
                             int with_torsion, double* energy, double* grad, void* stream);

/* The REBO task mode in use (1 directed, 2 per bond, 3 per bond on lane
 * pairs) and, when the autotuner ran, its timings of one force evaluation in
 * each mode (ms; 0 otherwise).  No reference counterpart. */
int mdg_task_mode(mdg_ctx* ctx, int* mode, float* ms_directed, float* ms_per_bond, float* ms_split);

/* ---- Thermal bath and adaptive time step ----
 * The SimLoop step's thermal bath (SimLoop.cxx:352-388, geometries
 * SimLoop.hpp:96-191) and adaptive dt (SimLoop.cxx:405-416), both off by
 * default.  A free atom inside the bath (and flagged, Atom::apply_ThermalBath)
 * feels dF = -V M gamma (1 - sqrt(T0/T)), T the bath's temperature at the
 * start of the step (SimLoop::actualTemperatureOfThermalBath).  Batched
 * contexts keep one bath temperature, dt and time per system. */
#define MDG_TB_NONE 0
#define MDG_TB_UNIVERSE 1  /* every atom (TB_GEOM_UNIVERSE) */
#define MDG_TB_BOX 2       /* ThermalBathGeomBox: params zMin, dBoundary, zMinOfFreeZone; needs periodic x, y */
#define MDG_TB_SPHERE 3    /* ThermalBathGeomSphere: params cx, cy, cz, radius, zMinOfFreeZone; open box */

/* T0 in K; gamma in 1/(time unit) (the reference's default is 1e13 / s);
 * params in length units; apply: NULL (every atom) or [n] flags. */
int mdg_set_thermal_bath(mdg_ctx* ctx, int geom, double T0, double gamma, const double* params, const uint8_t* apply);

/* Adaptive dt: after each step dt = 0.05 timeaccel / v_max (v_max over free
 * atoms with neighbours), clamped to [1e-20, 5e-16] s; dt0 starts it.  While
 * on, the dt argument of mdg_run / mdg_batch_run is ignored.  Setting it
 * restarts the simulated time. */
int mdg_set_adaptive_dt(mdg_ctx* ctx, int on, double timeaccel, double dt0);

/* Simulated time and current dt per system ([nsys] each; time counts the
 * adaptive steps since mdg_set_adaptive_dt). */
int mdg_get_time(mdg_ctx* ctx, double* sim_time, double* dt);

/* ---- Checkpoint and trajectory files ----
 * SimLoopSaver's state files (SimLoopSaver.cxx:118-231 write, 275-625 load):
 * "<id>.z", ".r", ".v", ".pbc_rect", ".pbc_rect.count", ".pbc_rect.enabled",
 * ".a", ".indices", ".tag.*", ".thermal_bath.*", ".time", ".check", raw
 * host-order records in the reference's CGS units; and the XVA text frames of
 * SimLoop::saveToStreamXVA (SimLoop.cxx:680-748).  Files are written from a
 * device snapshot by a writer thread while the steps go on; compression as
 * yaatk::Stream (plain, .gz, .xz; reading also finds .bz2). */
#define MDG_ZIP_NONE 0
#define MDG_ZIP_GZIP 1  /* "<file>.gz" (yaatk's gzip_internal) */
#define MDG_ZIP_XZ 2    /* "<file>.xz" through the xz program (yaatk's first choice) */

/* SimLoopSaver::LOADED_* bits returned by mdg_load_state (SimLoopSaver.hpp:56-71) */
#define MDG_LOADED_Z 1
#define MDG_LOADED_R 2
#define MDG_LOADED_V 4
#define MDG_LOADED_PBC_RECT 8
#define MDG_LOADED_PBC_COUNT 16
#define MDG_LOADED_PBC_ENABLED 32
#define MDG_LOADED_A 64

/* Per-atom tag bits (Atom::tag, ATOMTAG_TARGET .. ATOMTAG_FULLERENE = bits
 * 1..6, Atom.hpp:84-90) written to and read from the ".tag.*" files; NULL
 * clears them.  They do not change the dynamics. */
int mdg_set_atom_tags(mdg_ctx* ctx, const uint8_t* tags);
int mdg_get_atom_tags(mdg_ctx* ctx, uint8_t* tags);

/* SimLoopSaver::write(id) for system sys (0 for a single-system context):
 * returns when the files are written.  The Check record holds the net force
 * at the current positions, the kinetic energy before the last kick plus the
 * potential energy, the initial energy of iteration 0 and the energy the
 * bath has given (SimLoop.cxx:337-385, 1133-1153). */
int mdg_write_state(mdg_ctx* ctx, int sys, const char* id, int zip);

/* SimLoop::saveToStreamXVA of system sys into path (+ the compression's
 * extension); returns when the file is written. */
int mdg_write_xva(mdg_ctx* ctx, int sys, const char* path, int zip);

/* SimLoopSaver::loadIteration: SimLoopSaver::load(id) into this context (it
 * replaces the loaded system; one system) and SimLoop::iteration = iteration.
 * Needs the Z numbers and positions; the other files are optional, as in the
 * reference.  A loaded ".a" is kept (no new initial accelerations) unless
 * iteration is 0.  *loaded (may be NULL) gets the MDG_LOADED_* bits. */
int mdg_load_state(mdg_ctx* ctx, const char* id, uint64_t iteration, int* loaded);

/* SimLoop::executeMain's output inside mdg_run / mdg_batch_run
 * (SimLoop.cxx:263-277): at the top of each iteration, the state files
 * "<dir>/md%010lu" (SimLoopSaver::generateId) every flush_interval
 * iterations except iteration 0 (0 = never), and an XVA frame
 * "<dir>/mde%010lu.xva" at iteration 0 and whenever the simulated time has
 * crossed a multiple of traj_interval (time units; 0 = never).  Batched
 * contexts write system s under "<dir>/sys%05d".  dir NULL stops the output.
 * With adaptive dt and traj_interval > 0 each step reads its time back. */
int mdg_set_output(mdg_ctx* ctx, const char* dir, int64_t flush_interval, double traj_interval, int zip);

/* Wait for the files queued so far; reports the first write error. */
int mdg_flush_output(mdg_ctx* ctx);

/* SimLoop::iteration: steps taken since the system was loaded (or the
 * iteration given to mdg_load_state). */
int mdg_get_iteration(mdg_ctx* ctx, uint64_t* iteration);

/* Number of atoms loaded (AtomsArray::size), 0 before a system is set. */
int mdg_atom_count(mdg_ctx* ctx, int* n);

/* SimLoop::simTimeFinal as stored in the ".time" file (time units; default 4 ps). */
int mdg_set_time_final(mdg_ctx* ctx, double time_final);

/* Per-system simulated time and dt (time units, [nsys] each; the adaptive
 * step's state, SimLoop::simTime and dt of a loaded base state); dt_prev = dt. */
int mdg_set_time(mdg_ctx* ctx, const double* sim_time, const double* dt);

/* PBC_count of every atom ([n*3]; the wrapped positions stay). */
int mdg_set_images(mdg_ctx* ctx, const int32_t* image);

/* SimLoop's loop condition simTime < simTimeFinal (SimLoop.cxx:252) per
 * system, with adaptive dt: a system that reached simTimeFinal takes no more
 * steps (its later steps have dt 0 and leave it unchanged; its time, dt and
 * dt_prev stay as its last step left them) and, with output on, gets its
 * final state files (executeMain's closing writestate) at the iteration it
 * ended on. */
int mdg_set_stop_at_time_final(mdg_ctx* ctx, int on);

/* Steps (graph-replayed, checked every 16 steps) until every system reached
 * simTimeFinal or max_steps were taken; *steps gets the steps taken,
 * *finished 1 when every system is done.  Waits for the queued files. */
int mdg_run_until_final(mdg_ctx* ctx, int64_t max_steps, int64_t* steps, int* finished);

/* Output directory of each system of a batched context ([nsys] names,
 * created if missing; NULL restores "<dir>/sys%05d"). */
int mdg_set_output_dirs(mdg_ctx* ctx, const char* const* dirs);

/* The XVA interval as a table: interval[k] while simTime < until[k] (time
 * units, up to 4 entries; mdtrajsim's CustomSimLoop uses 1 ps below 2 ps,
 * then 5 ps, mdtrajsim/main.cpp:59-60).  Call after mdg_set_output. */
int mdg_set_traj_schedule(mdg_ctx* ctx, int n, const double* until, const double* interval);

/* ---- SnapshotList (SnapshotList.hpp:38-205) ----
 * mdtrajsim's snapshots of the projectile and cluster atoms (tag bits 2 and
 * 5), taken on the device at the top of each iteration whenever simTime has
 * crossed a multiple of the current interval (CustomSimLoop::isItTimeToSave,
 * mdtrajsim/main.cpp:52-80: 10 fs below 2 ps, 50 fs below 4 ps, then 100 fs);
 * records are float coordinates and velocities in CGS and the PBC counters,
 * as SnapshotList::AtomSnapshot.  Needs the adaptive time step (snapshots
 * follow simTime); capacity = snapshots kept per system (exceeding it is an
 * MDG_ERR_CAPACITY status).  With output on, "snapshots.conf" is written in
 * each system's directory every flush_interval iterations. */
int mdg_snapshots_enable(mdg_ctx* ctx, int on, int capacity);
int mdg_snapshots_set_schedule(mdg_ctx* ctx, int n, const double* until, const double* interval);
int mdg_snapshots_count(mdg_ctx* ctx, int sys, int* nshots, int* natoms);
/* times [nshots] (time units), indices [natoms] (atomsSelectedForSaving),
 * pbc_count/pos/vel [nshots * natoms * 3]; any NULL is skipped. */
int mdg_snapshots_get(mdg_ctx* ctx, int sys, double* times, uint32_t* indices, int32_t* pbc_count, float* pos,
                      float* vel);
/* SnapshotList::writestate ("snapshots.conf" layout) or, text != 0, saveInText. */
int mdg_snapshots_write(mdg_ctx* ctx, int sys, const char* path, int zip, int text);
/* SnapshotList::loadstate: earlier snapshots of system sys (same selection). */
int mdg_snapshots_load(mdg_ctx* ctx, int sys, const char* path);

/* The launch configuration the autotuner chose (with the LJ term): overlap = 1
 * when the REBO tasks run on a second stream concurrently with the LJ
 * kernels, rebo_blocks = the REBO task kernel's grid.  No reference
 * counterpart. */
int mdg_tuned_launch(mdg_ctx* ctx, int* overlap, int* rebo_blocks);

/* Programmatic dependent launch of the step's kernels (default on): each
 * kernel may be scheduled while the one before it on its stream drains and
 * waits on the device for that kernel's completion before its first read, so
 * results are those of ordinary launches; on = 0 launches them ordinarily.
 * No reference counterpart. */
int mdg_set_dependent_launch(mdg_ctx* ctx, int on);

/* ---- Batched systems ----
 * Many independent systems of uneven size in one context (the reference runs
 * impacts one after another, mdtrajsim/main.cpp:295-345): atoms of system s
 * are [first[s], first[s+1]) of the concatenated arrays, its box and
 * periodicity are box[3s..3s+2] and pbc[3s..3s+2].  Every kernel of a step
 * covers all systems in one launch; lists, bonds and forces never cross
 * systems.  mdg_compute, mdg_run, mdg_get_state/mdg_set_state work on the
 * concatenated arrays; the energies below are per system. */
int mdg_set_batch(mdg_ctx* ctx, int nsys, const int64_t* first, const int32_t* z, const double* pos,
                  const double* vel, const double* box, const int32_t* pbc, const uint8_t* fixed);

/* Per-system energies at the current state: e_sys[4 s + {0,1,2,3}] = REBO,
 * LJ, torsion, kinetic. */
int mdg_batch_energies(mdg_ctx* ctx, double* e_sys);

/* mdg_run for a batched context with per-system energies: epot/etot
 * [nsteps * nsys] (step-major), either may be NULL. */
int mdg_batch_run(mdg_ctx* ctx, int nsteps, double dt, double* epot, double* etot);

/* Test hook: the REBO spline tables the library built on the host, flattened
 * in the oracle's export order; returns the number of doubles (writes at most
 * cap).  Host only; needs no device. */
int64_t mdg_debug_rebo_tables(double* out, int64_t cap);

/* Test hook: the Brenner tables of parameter set 1 or 2 (H_CC, H_CH, F), in
 * the oracle's export order.  Host only. */
int64_t mdg_debug_brenner_tables(int set, double* out, int64_t cap);

/* Host evaluation of one REBO spline family in the given precision's tables
 * (test support): kind 0 = G (fam 0..2 = G_C1, G_C2, G_H; args cos theta;
 * out value, d/dcos), 1 = P (fam 0..1 = CC, CH; args (N^H, N^C); out value,
 * d/dN^H, d/dN^C), 2 = pi_rc / T_ij (fam 0..3 = CC, CH, HH, Tij; args
 * (N_ij, N_ji, N_conj); out value and the three partials). */
int mdg_debug_spline(int precision, int kind, int fam, int n, const double* args, double* out);

#ifdef __cplusplus
}
#endif

#endif /* MDG_H */
