// Checkpoint and trajectory files, written from device snapshots:
//
// * the state files of SimLoopSaver (SimLoopSaver.cxx:118-231 write,
//   275-625 load): one file per attribute, "<id>.<attribute>", raw
//   little-endian records in the reference's CGS units, optionally compressed
//   (yaatk::Stream: plain, .gz, .xz, .bz2);
// * the XVA text frames of SimLoop::saveToStreamXVA (SimLoop.cxx:680-748),
//   "mde<iteration %010>.xva";
// * SimLoop::executeMain's output schedule (SimLoop.cxx:263-277): state files
//   every iterationFlushStateInterval iterations, an XVA frame whenever the
//   simulated time crosses a multiple of simTimeSaveTrajInterval.
//
// A snapshot is one kernel on the context stream that converts the device
// state into a staging slot in CGS units, then one DMA copy on a separate
// stream into pinned host memory.  A writer thread waits for the copy,
// formats, compresses and writes the files while the steps go on.  Two slots:
// a third snapshot waits until the first slot's files are written.
//
// Included at the end of mdg_api.cu (it uses the context's internals).

#include <zlib.h>
#include <sys/stat.h>

#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <deque>
#include <mutex>
#include <thread>

namespace {

// CGS conversions of the internal units, written as the reference forms them
constexpr double kCgsLen = kAo;                 // Angstrom -> cm
constexpr double kCgsVel = kAo / kFs;           // Angstrom/fs -> cm/s (Ao/fs)
constexpr double kCgsAcc = kAo / (kFs * kFs);   // Angstrom/fs^2 -> cm/s^2
constexpr double kCgsForce = kEv / kAo;         // eV/Angstrom -> erg/cm
constexpr double kKbErg = 8.617343E-5 * kEv;    // kb (consts.cxx:32), erg/K
constexpr double kNoPbcCm = 10000.0 * kAo;      // NO_PBC_L (consts.hpp:96)
// ElementID (consts.hpp:46-55) by atomic number and back
inline int element_id(int z)
{
  switch (z) {
    case 1: return 1;
    case 6: return 12;
    case 29: return 64;
    case 47: return 108;
    case 79: return 197;
    case 18: return 40;
    case 54: return 131;
  }
  return -1;
}
inline int z_of_element(int e)
{
  for (int z : {1, 6, 29, 47, 79, 18, 54})
    if (element_id(z) == e) return z;
  return -1;
}
constexpr int kHdr = 7;                         // per-system header doubles of a snapshot

// Byte offsets of one snapshot (same layout on the device and the host).
struct SnapLayout {
  size_t r, v, a, f, img, ekp, ep, eb, hdr, bytes;
};

SnapLayout snap_layout(int64_t n, int nsys)
{
  SnapLayout L;
  size_t o = 0;
  auto take = [&](size_t b) { size_t at = o; o += (b + 255) & ~size_t(255); return at; };
  L.r = take(24 * n);
  L.v = take(24 * n);
  L.a = take(24 * n);
  L.f = take(24 * n);
  L.img = take(12 * n);
  L.ekp = take(8 * n);
  L.ep = take(8 * n);
  L.eb = take(8 * n);
  L.hdr = take(8 * (size_t)kHdr * nsys);
  L.bytes = o;
  return L;
}

// -------------------------------------------------------------------------
// files: plain or compressed as yaatk::Stream does (Stream::zipMe / unZipMe,
// yaatk.cxx:200-330): .gz through zlib (its "gzip_internal"), .xz and .bz2
// through the xz and bzip2 programs

const char* zip_ext(int zip) { return zip == MDG_ZIP_GZIP ? ".gz" : zip == MDG_ZIP_XZ ? ".xz" : ""; }

bool safe_for_shell(const std::string& p) { return p.find('\'') == std::string::npos; }

bool file_exists(const std::string& p)
{
  struct stat st;
  return ::stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

// Writes len bytes to path + the compression's extension; other compressed
// copies of the same file are removed so that a reader finds this one.
bool write_blob(const std::string& path, const void* data, size_t len, int zip, std::string& err)
{
  for (const char* e : {"", ".gz", ".xz", ".bz2"}) std::remove((path + e).c_str());
  const std::string name = path + zip_ext(zip);
  if (zip == MDG_ZIP_GZIP) {
    gzFile g = gzopen(name.c_str(), "wb");
    if (!g) { err = "cannot open " + name; return false; }
    size_t done = 0;
    while (done < len) {
      const unsigned chunk = (unsigned)std::min<size_t>(len - done, 1u << 30);
      const int w = gzwrite(g, (const char*)data + done, chunk);
      if (w <= 0) { gzclose(g); err = "gzwrite failed on " + name; return false; }
      done += (size_t)w;
    }
    if (gzclose(g) != Z_OK) { err = "gzclose failed on " + name; return false; }
    return true;
  }
  FILE* f = nullptr;
  if (zip == MDG_ZIP_XZ) {
    if (!safe_for_shell(name)) { err = "file name with a quote: " + name; return false; }
    f = popen(("xz -c > '" + name + "'").c_str(), "w");
  } else {
    f = std::fopen(name.c_str(), "wb");
  }
  if (!f) { err = "cannot open " + name; return false; }
  const bool ok = len == 0 || std::fwrite(data, 1, len, f) == len;
  const int st = (zip == MDG_ZIP_XZ) ? pclose(f) : std::fclose(f);
  if (!ok || st != 0) { err = "write failed on " + name; return false; }
  return true;
}

// Reads path as yaatk::Stream finds it (Stream::guessZipTypeByPresence,
// yaatk.cxx:160-177): the plain file, else .xz, .bz2, .gz.  Returns 1 and the
// bytes, 0 when no copy exists, -1 on a read error.
int read_blob(const std::string& path, std::string& out, std::string& err)
{
  out.clear();
  char buf[1 << 16];
  if (file_exists(path)) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path; return -1; }
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, k);
    std::fclose(f);
    return 1;
  }
  for (const char* prog : {"xz", "bzip2"}) {
    const std::string name = path + (prog[0] == 'x' ? ".xz" : ".bz2");
    if (!file_exists(name)) continue;
    if (!safe_for_shell(name)) { err = "file name with a quote: " + name; return -1; }
    FILE* f = popen((std::string(prog) + " -dc '" + name + "'").c_str(), "r");
    if (!f) { err = "cannot run " + std::string(prog); return -1; }
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, k);
    if (pclose(f) != 0) { err = std::string(prog) + " failed on " + name; return -1; }
    return 1;
  }
  const std::string gz = path + ".gz";
  if (file_exists(gz)) {
    gzFile g = gzopen(gz.c_str(), "rb");
    if (!g) { err = "cannot open " + gz; return -1; }
    int k;
    while ((k = gzread(g, buf, sizeof(buf))) > 0) out.append(buf, (size_t)k);
    const bool bad = k < 0;
    gzclose(g);
    if (bad) { err = "gzread failed on " + gz; return -1; }
    return 1;
  }
  return 0;
}

// host-order binary records, as YAATK_BIN_WRITE writes them
struct Rec {
  std::string b;
  template <typename T> void put(T v) { b.append((const char*)&v, sizeof(T)); }
};

}  // namespace

// -------------------------------------------------------------------------
// snapshot kernels

// Per atom: coords, V, an, -grad in CGS, PBC_count, and the Check inputs
// (kinetic energy before the last kick, potential energy, bath energy) in erg.
__global__ void k_snap_pack(State S, const double4* grad, const double* er, const double* el, const double* et,
                            const double* em, const double* ekp, const double* eb, char* out, SnapLayout L)
{
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  double* r = (double*)(out + L.r) + 3 * (size_t)i;
  double* v = (double*)(out + L.v) + 3 * (size_t)i;
  double* a = (double*)(out + L.a) + 3 * (size_t)i;
  double* f = (double*)(out + L.f) + 3 * (size_t)i;
  int* im = (int*)(out + L.img) + 3 * (size_t)i;
  const double4 p = S.pos[i], u = S.vel[i], ac = S.acc[i], g = grad[i];
  const int4 m = S.image[i];
  r[0] = p.x * kCgsLen; r[1] = p.y * kCgsLen; r[2] = p.z * kCgsLen;
  v[0] = u.x * kCgsVel; v[1] = u.y * kCgsVel; v[2] = u.z * kCgsVel;
  a[0] = ac.x * kCgsAcc; a[1] = ac.y * kCgsAcc; a[2] = ac.z * kCgsAcc;
  f[0] = -g.x * kCgsForce; f[1] = -g.y * kCgsForce; f[2] = -g.z * kCgsForce;
  im[0] = m.x; im[1] = m.y; im[2] = m.z;
  ((double*)(out + L.ekp))[i] = ekp[i] * kEv;
  ((double*)(out + L.ep))[i] = (((er[i] + el[i]) + et[i]) + (em ? em[i] : 0.0)) * kEv;
  ((double*)(out + L.eb))[i] = eb ? eb[i] * kEv : 0.0;
}

// Per system: time, dt, dt_prev of adaptive steps (s) and the first step's
// energies (eV: REBO, LJ, torsion, kinetic).
__global__ void k_snap_header(int nsys, const double* time, const double* dt, const double* dt_prev, const double* e0,
                              char* out, SnapLayout L)
{
  pdl_enter();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  double* h = (double*)(out + L.hdr) + kHdr * (size_t)s;
  h[0] = time[s] * kFs;
  h[1] = dt[s] * kFs;
  h[2] = dt_prev[s] * kFs;
  for (int k = 0; k < 4; k++) h[3 + k] = e0[4 * s + k];
}

// -------------------------------------------------------------------------
// writer

namespace {

enum { kJobState = 0, kJobXva = 1 };

struct IoJob {
  int slot = 0, kind = kJobState, zip = MDG_ZIP_NONE, sys = 0;
  std::string path;            // the state's id, or the XVA file
  int64_t first = 0, count = 0;
  uint64_t iteration = 0;
  bool adaptive = false;       // time from the snapshot header
  double time_s = 0, dt_s = 0, dt_prev_s = 0, time_final_s = 0, cpu_s = 0;
  bool stepped = false, e0_dev = false;
  double chk_e0 = 1.0, chk_eb0 = 0.0, chk_net[3] = {0, 0, 0}, chk_cur = 1.0, chk_T = 0.0;
  Box box;
  int tb_geom = 0;
  double tb_T0 = 0, tb_gamma_s = 0, tb_gp_cm[5] = {0, 0, 0, 0, 0};
  std::vector<int32_t> z;
  std::vector<unsigned char> fixed, tb_apply, tags;
};

struct SnapSlot {
  char* d = nullptr;
  char* h = nullptr;
  size_t bytes = 0;
  cudaEvent_t copied = nullptr, packed = nullptr;
  int users = 0;               // jobs that still read this slot
};

}  // namespace

struct IoState {
  int device = 0;
  cudaStream_t stream = nullptr;
  SnapSlot slot[2];
  SnapLayout lay{};
  int next = 0;
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<IoJob> q;
  int active = 0;              // jobs queued or being written
  bool stop = false;
  std::string err;             // first writer error, reported by the next call
  // schedule (SimLoop::iterationFlushStateInterval, simTimeSaveTrajInterval)
  bool on = false;
  std::string dir;
  std::vector<std::string> dirs;  // per-system directories (batched contexts), else dir/sys%05d
  int64_t flush_interval = 0;
  int ntraj = 0;                  // XVA interval table: traj_int[k] while simTime < traj_until[k] (s)
  double traj_until[4] = {0, 0, 0, 0}, traj_int[4] = {0, 0, 0, 0};
  std::vector<char> fin;          // per system: its final state is written
  int zip = MDG_ZIP_NONE;
  double* h_time = nullptr;    // pinned [3 nsys]: time, dt_prev, stop flag of adaptive steps
  int h_time_cap = 0;
  std::chrono::steady_clock::time_point t_run;  // start of the current mdg_run
  double cpu_prev_s = 0.0;     // run time of the earlier runs (SimLoop::CPUTimeUsed_prev)
};

namespace {

// The Check record of one system (SimLoop::Check, SimLoop.cxx:1280-1300):
// netForce sums the forces of the current positions over every atom,
// currentEnergy is the kinetic energy before the last kick plus the potential
// energy, currentTemperature that kinetic energy over the free atoms
// (SimLoop::temperatureWithoutFixed), both as doEnergyConservationCheck
// leaves them (SimLoop.cxx:337, 1150-1153).
struct CheckRec {
  double net[3], e0, cur, eb, T;
};

CheckRec job_check(const IoJob& J, const char* h, const SnapLayout& L)
{
  CheckRec C;
  const double* f = (const double*)(h + L.f) + 3 * J.first;
  const double* ekp = (const double*)(h + L.ekp) + J.first;
  const double* ep = (const double*)(h + L.ep) + J.first;
  const double* eb = (const double*)(h + L.eb) + J.first;
  double ebs = 0.0;
  for (int64_t i = 0; i < J.count; i++) ebs += eb[i];
  C.eb = J.chk_eb0 + ebs;
  if (J.e0_dev) {
    const double* e0 = (const double*)(h + L.hdr) + kHdr * (size_t)J.sys + 3;
    C.e0 = (((e0[0] + e0[1]) + e0[2]) + e0[3]) * kEv;
  } else {
    C.e0 = J.chk_e0;
  }
  if (J.stepped) {
    C.net[0] = C.net[1] = C.net[2] = 0.0;
    double ek = 0.0, ekf = 0.0, epot = 0.0;
    int64_t nf = 0;
    for (int64_t i = 0; i < J.count; i++) {
      C.net[0] += f[3 * i];
      C.net[1] += f[3 * i + 1];
      C.net[2] += f[3 * i + 2];
      ek += ekp[i];
      epot += ep[i];
      if (!J.fixed[i]) { ekf += ekp[i]; nf++; }
    }
    C.cur = ek + epot;
    C.T = nf ? ekf / (3.0 / 2.0 * kKbErg * nf) : 0.0;
  } else {
    for (int k = 0; k < 3; k++) C.net[k] = J.chk_net[k];
    C.cur = J.chk_cur;
    C.T = J.chk_T;
  }
  return C;
}

void job_times(const IoJob& J, const char* h, const SnapLayout& L, double& t, double& dt, double& dtp)
{
  if (J.adaptive) {
    const double* hd = (const double*)(h + L.hdr) + kHdr * (size_t)J.sys;
    t = hd[0]; dt = hd[1]; dtp = hd[2];
  } else {
    t = J.time_s; dt = J.dt_s; dtp = J.dt_prev_s;
  }
}

// SimLoopSaver::write(id) (SimLoopSaver.cxx:118-231) for one system.
bool write_state_files(const IoJob& J, const char* h, const SnapLayout& L, std::string& err)
{
  const int64_t n = J.count, f0 = J.first;
  const double* r = (const double*)(h + L.r) + 3 * f0;
  const double* v = (const double*)(h + L.v) + 3 * f0;
  const double* a = (const double*)(h + L.a) + 3 * f0;
  const int* im = (const int*)(h + L.img) + 3 * f0;
  const std::string& id = J.path;
  auto put = [&](const char* attr, const std::string& b) { return write_blob(id + attr, b.data(), b.size(), J.zip, err); };
  Rec z, pr, cnt, en, idx;
  for (int64_t i = 0; i < n; i++) {
    z.put<uint8_t>((uint8_t)element_id(J.z[i]));
    for (int k = 0; k < 3; k++) cnt.put<int32_t>(im[3 * i + k]);
    for (int k = 0; k < 3; k++) en.put<uint8_t>(J.box.pbc[k] ? 1 : 0);
    idx.put<uint32_t>((uint32_t)i);  // Atom::globalIndex (AtomsContainer.cxx:114)
  }
  for (int k = 0; k < 3; k++) pr.put<double>(J.box.pbc[k] ? J.box.L[k] * kCgsLen : kNoPbcCm);
  if (!put(".z", z.b)) return false;
  if (!put(".r", std::string((const char*)r, 24 * n))) return false;
  if (!put(".v", std::string((const char*)v, 24 * n))) return false;
  if (!put(".pbc_rect", pr.b)) return false;
  if (!put(".pbc_rect.count", cnt.b)) return false;
  if (!put(".pbc_rect.enabled", en.b)) return false;
  if (!put(".a", std::string((const char*)a, 24 * n))) return false;
  if (!put(".indices", idx.b)) return false;
  {
    // Atom::apply_ThermalBath, Atom::fixed and the tag bits (Atom.hpp:84-90)
    Rec tb, fx, t[6];
    for (int64_t i = 0; i < n; i++) {
      tb.put<uint8_t>(J.tb_apply.empty() ? 1 : (J.tb_apply[i] ? 1 : 0));
      fx.put<uint8_t>(J.fixed[i] ? 1 : 0);
      for (int k = 0; k < 6; k++) t[k].put<uint8_t>((J.tags[i] >> (k + 1)) & 1);
    }
    static const char* names[6] = {".tag.target", ".tag.projectile", ".tag.substrate",
                                   ".tag.monomer", ".tag.cluster", ".tag.fullerene"};
    if (!put(".tag.thermal_bath_applicable", tb.b) || !put(".tag.fixed", fx.b)) return false;
    for (int k = 0; k < 6; k++)
      if (!put(names[k], t[k].b)) return false;
  }
  // bath files of the other geometries stay from an earlier write unless removed
  for (const char* g : {".thermal_bath.common", ".thermal_bath.univserse", ".thermal_bath.box", ".thermal_bath.sphere"})
    for (const char* e : {"", ".gz", ".xz", ".bz2"}) std::remove((id + g + e).c_str());
  if (J.tb_geom != MDG_TB_NONE) {
    Rec cm;
    cm.put<double>(J.tb_T0);
    cm.put<double>(J.tb_gamma_s);
    if (!put(".thermal_bath.common", cm.b)) return false;
    Rec g;
    // the universe geometry's file name keeps the reference's spelling
    // (SimLoopSaver.cxx:149), which its loader looks for
    const char* gname = J.tb_geom == MDG_TB_UNIVERSE ? ".thermal_bath.univserse"
                        : J.tb_geom == MDG_TB_BOX    ? ".thermal_bath.box"
                                                     : ".thermal_bath.sphere";
    const int np = J.tb_geom == MDG_TB_UNIVERSE ? 0 : J.tb_geom == MDG_TB_BOX ? 3 : 5;
    for (int k = 0; k < np; k++) g.put<double>(J.tb_gp_cm[k]);
    if (!put(gname, g.b)) return false;
  }
  double t, dt, dtp;
  job_times(J, h, L, t, dt, dtp);
  Rec tm;
  tm.put<double>(t);
  tm.put<double>(J.time_final_s);
  tm.put<double>(dt);
  tm.put<double>(dtp);
  if (!put(".time", tm.b)) return false;
  const CheckRec C = job_check(J, h, L);
  Rec ck;
  ck.put<uint8_t>(1);  // Check::checkForce (SimLoop.cxx:66)
  for (int k = 0; k < 3; k++) ck.put<double>(C.net[k]);
  ck.put<uint8_t>(1);  // Check::checkEnergy (SimLoop.cxx:65)
  ck.put<double>(C.e0);
  ck.put<double>(C.cur);
  ck.put<double>(C.eb);
  ck.put<double>(C.T);
  return put(".check", ck.b);
}

// printf conversions equal to the ostream settings the reference uses:
// default float field with precision 6 = %g, fixed with precision 2 = %.2f,
// scientific with FLOAT_PRECISION (config.cxx:29) = %.10e
void appendf(std::string& s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void appendf(std::string& s, const char* fmt, ...)
{
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  const int k = vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (k > 0) s.append(buf, std::min<int>(k, (int)sizeof(buf) - 1));
}

// SimLoop::saveToStreamXVA (SimLoop.cxx:680-748) for one system.
bool write_xva_file(const IoJob& J, const char* h, const SnapLayout& L, std::string& err)
{
  const int64_t n = J.count, f0 = J.first;
  const double* r = (const double*)(h + L.r) + 3 * f0;
  const double* v = (const double*)(h + L.v) + 3 * f0;
  const int* im = (const int*)(h + L.img) + 3 * f0;
  double vs = 0.0;
  for (int64_t i = 0; i < n; i++) {
    vs += std::fabs(v[3 * i]);
    vs += std::fabs(v[3 * i + 1]);
    vs += std::fabs(v[3 * i + 2]);
  }
  vs /= (3.0 * n);
  if (std::fabs(vs) < 1e-30) vs = 1e-30;
  vs = std::pow(10.0, std::ceil(std::log10(std::fabs(vs))) - 2);
  const double ds = kAo;
  std::string s;
  s.reserve((size_t)n * 64 + 512);
  appendf(s, "%g\n%g\n%d\n", vs, ds, (int)n);
  // the atom lines, formatted by several threads over contiguous ranges and
  // joined in order
  const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(8, n / 4096));
  std::vector<std::string> part(nt);
  auto fmt = [&](int t) {
    const int64_t b = n * t / nt, e = n * (t + 1) / nt;
    std::string& q = part[t];
    q.reserve((size_t)(e - b) * 64);
    for (int64_t i = b; i < e; i++) {
      appendf(q, "%.2f %.2f %.2f\n", v[3 * i] / vs, v[3 * i + 1] / vs, v[3 * i + 2] / vs);
      appendf(q, "%.2f %.2f %.2f\n", r[3 * i] / ds, r[3 * i + 1] / ds, r[3 * i + 2] / ds);
      appendf(q, "%d %d %d\n", im[3 * i], im[3 * i + 1], im[3 * i + 2]);
    }
  };
  if (nt == 1) {
    fmt(0);
  } else {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(fmt, t);
    fmt(0);
    for (auto& x : th) x.join();
  }
  for (const std::string& q : part) s += q;
  const CheckRec C = job_check(J, h, L);
  double t, dt, dtp;
  job_times(J, h, L, t, dt, dtp);
  // Check::saveToStream in text mode: one value per line, a Vector3D as
  // "x y z " (Vector3D.cxx:343-348), bools as 1
  appendf(s, "1\n%.10e %.10e %.10e \n1\n", C.net[0], C.net[1], C.net[2]);
  appendf(s, "%.10e\n%.10e\n%.10e\n%.10e\n", C.e0, C.cur, C.eb, C.T);
  appendf(s, "%.10e\n%.10e\n%lu\n%.10e\n", t, dt, (unsigned long)J.iteration, J.cpu_s);
  return write_blob(J.path, s.data(), s.size(), J.zip, err);
}

void writer_loop(IoState* io)
{
  cudaSetDevice(io->device);
  for (;;) {
    IoJob J;
    {
      std::unique_lock<std::mutex> lk(io->mu);
      io->cv.wait(lk, [&] { return io->stop || !io->q.empty(); });
      if (io->q.empty()) return;
      J = std::move(io->q.front());
      io->q.pop_front();
    }
    SnapSlot& S = io->slot[J.slot];
    std::string err;
    const cudaError_t ce = cudaEventSynchronize(S.copied);
    bool ok = ce == cudaSuccess;
    if (!ok) err = std::string("snapshot copy: ") + cudaGetErrorString(ce);
    if (ok) ok = (J.kind == kJobState) ? write_state_files(J, S.h, io->lay, err) : write_xva_file(J, S.h, io->lay, err);
    {
      std::lock_guard<std::mutex> lk(io->mu);
      if (!ok && io->err.empty()) io->err = err;
      S.users--;
      io->active--;
    }
    io->cv.notify_all();
  }
}

double wall_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// -------------------------------------------------------------------------
// host side: writer, slots, snapshots

static int io_get(mdg_ctx* c, IoState** out)
{
  if (!c->io) {
    IoState* io = new IoState();
    io->device = c->prm.device;
    if (cudaStreamCreateWithFlags(&io->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete io;
      return fail(MDG_ERR_CUDA, "cudaStreamCreate (snapshot copies)");
    }
    io->th = std::thread(writer_loop, io);
    c->io = io;
  }
  *out = c->io;
  return MDG_OK;
}

// Waits until every queued file is written; returns (and clears) the first
// writer error.
static int io_wait(mdg_ctx* c)
{
  if (!c->io) return MDG_OK;
  IoState* io = c->io;
  std::string err;
  {
    std::unique_lock<std::mutex> lk(io->mu);
    io->cv.wait(lk, [&] { return io->active == 0; });
    err.swap(io->err);
  }
  if (!err.empty()) return fail(MDG_ERR_IO, err);
  return MDG_OK;
}

static void io_free_slots(IoState* io)
{
  for (SnapSlot& S : io->slot) {
    if (S.d) cudaFree(S.d);
    if (S.h) cudaFreeHost(S.h);
    if (S.copied) cudaEventDestroy(S.copied);
    if (S.packed) cudaEventDestroy(S.packed);
    S = SnapSlot();
  }
}

namespace {  // declared beside free_system

// The system's arrays are about to change size: finish the files, drop the slots.
void io_release(mdg_ctx* c)
{
  if (!c->io) return;
  io_wait(c);
  io_free_slots(c->io);
}

void io_free(mdg_ctx* c)
{
  if (!c->io) return;
  IoState* io = c->io;
  io_wait(c);
  {
    std::lock_guard<std::mutex> lk(io->mu);
    io->stop = true;
  }
  io->cv.notify_all();
  if (io->th.joinable()) io->th.join();
  io_free_slots(io);
  if (io->h_time) cudaFreeHost(io->h_time);
  if (io->stream) cudaStreamDestroy(io->stream);
  delete io;
  c->io = nullptr;
}

}  // namespace

// Packs the state into the next free slot and starts its copy to the host;
// returns the slot.  The caller queues the slot's jobs with io_push.
static int io_snapshot(mdg_ctx* c, int* slot_out)
{
  IoState* io = nullptr;
  int rc = io_get(c, &io);
  if (rc) return rc;
  const SnapLayout L = snap_layout(c->n, c->nsys);
  const int k = io->next;
  SnapSlot& S = io->slot[k];
  {
    std::unique_lock<std::mutex> lk(io->mu);
    io->cv.wait(lk, [&] { return S.users == 0; });
  }
  if (S.bytes != L.bytes) {
    if (S.d) cudaFree(S.d);
    if (S.h) cudaFreeHost(S.h);
    S.d = nullptr;
    S.h = nullptr;
    S.bytes = 0;
    if (cudaMalloc(&S.d, L.bytes) != cudaSuccess) return fail(MDG_ERR_CUDA, "cudaMalloc (snapshot)");
    if (cudaHostAlloc((void**)&S.h, L.bytes, cudaHostAllocDefault) != cudaSuccess)
      return fail(MDG_ERR_CUDA, "cudaHostAlloc (snapshot)");
    if (!S.copied) CK(cudaEventCreateWithFlags(&S.copied, cudaEventDisableTiming));
    if (!S.packed) CK(cudaEventCreateWithFlags(&S.packed, cudaEventDisableTiming));
    S.bytes = L.bytes;
  }
  io->lay = L;
  State St = c->S();
  LAUNCH(c, "snap_pack", k_snap_pack, nblk(c->n), kThreads, St, c->grad, c->fo.e_rebo, c->fo.e_lj, c->fo.e_tors,
         c->has_list[2] ? c->d_em : nullptr, c->d_ekin_pre, c->tb_geom ? c->d_eb : nullptr, S.d, L);
  LAUNCH(c, "snap_header", k_snap_header, nblk(c->nsys), kThreads, c->nsys, c->d_time, c->d_dt, c->d_dt_prev,
         c->d_e0, S.d, L);
  CK(cudaEventRecord(S.packed, c->stream));
  CK(cudaStreamWaitEvent(io->stream, S.packed, 0));
  CK(cudaMemcpyAsync(S.h, S.d, L.bytes, cudaMemcpyDeviceToHost, io->stream));
  CK(cudaEventRecord(S.copied, io->stream));
  io->next ^= 1;
  *slot_out = k;
  return launch_check(c);
}

// A job for system sys of the snapshot in slot, with the context's
// bookkeeping as it stands now.
static IoJob io_job(mdg_ctx* c, int slot, int kind, int sys, const std::string& path, int zip)
{
  IoJob J;
  J.slot = slot;
  J.kind = kind;
  J.sys = sys;
  J.path = path;
  J.zip = zip;
  J.first = c->nsys > 1 ? c->h_first[sys] : 0;
  J.count = c->nsys > 1 ? c->h_first[sys + 1] - c->h_first[sys] : c->n;
  J.iteration = c->iteration;
  J.adaptive = c->adaptive;
  J.time_s = c->time_s;
  J.dt_s = c->dt_s;
  J.dt_prev_s = c->dt_prev_s;
  J.time_final_s = c->time_final_s;
  J.cpu_s = c->run_t0 > 0.0 ? wall_s() - c->run_t0 : 0.0;
  J.stepped = c->stepped;
  // SimLoop writes at the top of an iteration, before iteration 0 sets the
  // initial energy (SimLoop.cxx:263-277 precede 305-308)
  J.e0_dev = c->e0_dev && c->iteration != 0;
  J.chk_e0 = c->chk_e0;
  J.chk_eb0 = c->chk_eb0;
  for (int k = 0; k < 3; k++) J.chk_net[k] = c->chk_net[k];
  J.chk_cur = c->chk_cur;
  J.chk_T = c->chk_T;
  J.box = c->h_boxes[sys];
  J.tb_geom = c->tb_geom;
  J.tb_T0 = c->tb_T0;
  J.tb_gamma_s = c->tb_gamma / kFs;
  for (int k = 0; k < 5; k++) J.tb_gp_cm[k] = c->tb_gp[k] * kCgsLen;
  const size_t b = (size_t)J.first, e = b + (size_t)J.count;
  J.z.assign(c->h_z.begin() + b, c->h_z.begin() + e);
  J.fixed.assign(c->h_fixed.begin() + b, c->h_fixed.begin() + e);
  J.tags.assign(c->h_tags.begin() + b, c->h_tags.begin() + e);
  if (!c->h_tb_apply.empty()) J.tb_apply.assign(c->h_tb_apply.begin() + b, c->h_tb_apply.begin() + e);
  return J;
}

static void io_push(mdg_ctx* c, std::vector<IoJob>& jobs)
{
  IoState* io = c->io;
  {
    std::lock_guard<std::mutex> lk(io->mu);
    for (IoJob& J : jobs) {
      io->slot[J.slot].users++;
      io->active++;
      io->q.push_back(std::move(J));
    }
  }
  io->cv.notify_all();
}

static std::string sys_dir(mdg_ctx* c, int sys)
{
  if ((int)c->io->dirs.size() == c->nsys) return c->io->dirs[sys];
  if (c->nsys == 1) return c->io->dir;
  char b[32];
  std::snprintf(b, sizeof(b), "/sys%05d", sys);
  return c->io->dir + b;
}

// -------------------------------------------------------------------------
// SimLoop::executeMain's bookkeeping and output schedule around the steps

int io_run_start(mdg_ctx* c, double dtf, bool fresh)
{
  if (c->run_t0 <= 0.0) c->run_t0 = wall_s();
  // executeMain takes dt_prev = dt before its loop (SimLoop.cxx:249)
  if (!fresh) {
  } else if (c->adaptive) {
    CK(cudaMemcpyAsync(c->d_dt_prev, c->d_dt, c->nsys * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (c->stop_final)
      LAUNCH(c, "stop_init", k_stop_init, nblk(c->nsys), kThreads, c->nsys, c->d_time, c->d_stop,
             c->time_final_s / kFs);
  } else {
    c->dt_s = dtf * kFs;
    c->dt_prev_s = c->dt_s;
  }
  if (c->io && c->io->on) {
    std::lock_guard<std::mutex> lk(c->io->mu);
    if (!c->io->err.empty()) {
      std::string e;
      e.swap(c->io->err);
      return fail(MDG_ERR_IO, e);
    }
  }
  return MDG_OK;
}

// The top of an iteration (SimLoop.cxx:263-277): the state files every
// iterationFlushStateInterval iterations but the first, an XVA frame at the
// first iteration and whenever simTime has crossed a multiple of
// simTimeSaveTrajInterval during the last step.
namespace {
int snap_write(mdg_ctx* c, int sys, const std::string& path, int zip, bool text);
}

static double traj_interval(const IoState* io, double t)
{
  for (int k = 0; k < io->ntraj; k++)
    if (t < io->traj_until[k]) return io->traj_int[k];
  return io->traj_int[io->ntraj - 1];
}

// Per-system time, dt_prev and stop flag of adaptive steps, read back.
static int io_read_times(mdg_ctx* c)
{
  IoState* io = c->io;
  if (io->h_time_cap < c->nsys) {
    if (io->h_time) cudaFreeHost(io->h_time);
    io->h_time = nullptr;
    if (cudaHostAlloc((void**)&io->h_time, 3 * c->nsys * sizeof(double), cudaHostAllocDefault) != cudaSuccess)
      return fail(MDG_ERR_CUDA, "cudaHostAlloc (time readback)");
    io->h_time_cap = c->nsys;
  }
  CK(cudaMemcpyAsync(io->h_time, c->d_time, c->nsys * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(io->h_time + c->nsys, c->d_dt_prev, c->nsys * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  std::vector<int> st((size_t)c->nsys, 0);
  if (c->stop_final)
    CK(cudaMemcpyAsync(st.data(), c->d_stop, c->nsys * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < c->nsys; s++) io->h_time[2 * c->nsys + s] = st[s];
  return MDG_OK;
}

// Systems that reached simTimeFinal since the last look get executeMain's
// closing state files (SimLoop.cxx:460-464) at the iteration they ended on.
static int io_finalize(mdg_ctx* c, std::vector<IoJob>& jobs, int& slot)
{
  IoState* io = c->io;
  if (!c->stop_final || !c->adaptive) return MDG_OK;
  io->fin.resize(c->nsys, 0);
  char name[64];
  for (int s = 0; s < c->nsys; s++) {
    if (!io->h_time[2 * c->nsys + s] || io->fin[s]) continue;
    if (slot < 0) {
      int rc = io_snapshot(c, &slot);
      if (rc) return rc;
    }
    std::snprintf(name, sizeof(name), "/md%010lu", (unsigned long)c->iteration);
    jobs.push_back(io_job(c, slot, kJobState, s, sys_dir(c, s) + name, io->zip));
    io->fin[s] = 1;
  }
  return MDG_OK;
}

// The top of an iteration (SimLoop.cxx:263-277, with CustomSimLoop's
// doBeforeIteration before it, mdtrajsim/main.cpp:59-85): the snapshot list
// and the state files every iterationFlushStateInterval iterations but the
// first, an XVA frame at the first iteration and whenever simTime has crossed
// a multiple of simTimeSaveTrajInterval during the last step.  Systems that
// reached simTimeFinal write nothing more.
int io_before_step(mdg_ctx* c)
{
  if (!c->io || !c->io->on) return MDG_OK;
  IoState* io = c->io;
  const uint64_t it = c->iteration;
  const bool flush = io->flush_interval > 0 && it % (uint64_t)io->flush_interval == 0 && it != 0;
  const bool readback = c->adaptive && (io->ntraj > 0 || c->stop_final);
  if (readback) {
    int rc = io_read_times(c);
    if (rc) return rc;
  }
  auto stopped = [&](int s) { return readback && io->h_time[2 * c->nsys + s] != 0.0; };
  std::vector<IoJob> jobs;
  int slot = -1;
  int rc = io_finalize(c, jobs, slot);
  if (rc) return rc;
  std::vector<char> xva((size_t)c->nsys, 0);
  bool any = false;
  for (int s = 0; s < c->nsys; s++) {
    if (stopped(s)) continue;
    if (io->ntraj > 0) {
      const double t = c->adaptive ? io->h_time[s] * kFs : c->time_s;
      const double dtp = c->adaptive ? io->h_time[c->nsys + s] * kFs : c->dt_prev_s;
      const double I = traj_interval(io, t);
      xva[s] = it == 0 || t == 0.0 || (long long)(t / I) != (long long)((t - dtp) / I);
    }
    any = any || xva[s] || flush;
  }
  if (flush && c->snap) {
    // CustomSimLoop writes its snapshot list at the same iterations
    for (int s = 0; s < c->nsys; s++) {
      if (stopped(s)) continue;
      rc = snap_write(c, s, sys_dir(c, s) + "/snapshots.conf", io->zip, false);
      if (rc) return rc;
    }
  }
  if (any && slot < 0) {
    rc = io_snapshot(c, &slot);
    if (rc) return rc;
  }
  char name[64];
  for (int s = 0; s < c->nsys && any; s++) {
    if (stopped(s)) continue;
    if (flush) {
      std::snprintf(name, sizeof(name), "/md%010lu", (unsigned long)it);  // SimLoopSaver::generateId
      jobs.push_back(io_job(c, slot, kJobState, s, sys_dir(c, s) + name, io->zip));
    }
    if (xva[s]) {
      std::snprintf(name, sizeof(name), "/mde%010lu.xva", (unsigned long)it);  // SimLoop::writetrajXVA
      jobs.push_back(io_job(c, slot, kJobXva, s, sys_dir(c, s) + name, io->zip));
    }
  }
  if (!jobs.empty()) io_push(c, jobs);
  return MDG_OK;
}

// After the last step of a run: final states of systems that just ended.
int io_run_end(mdg_ctx* c)
{
  if (!c->io || !c->io->on || !c->adaptive || !c->stop_final) return MDG_OK;
  int rc = io_read_times(c);
  if (rc) return rc;
  std::vector<IoJob> jobs;
  int slot = -1;
  rc = io_finalize(c, jobs, slot);
  if (rc) return rc;
  if (!jobs.empty()) io_push(c, jobs);
  return MDG_OK;
}

// The end of an iteration: simTime += dt, dt_prev = dt, iteration + 1
// (SimLoop.cxx:403-405, 443); adaptive steps keep their time on the device.
int io_after_step(mdg_ctx* c)
{
  c->iteration++;
  c->stepped = true;
  if (!c->adaptive) {
    c->time_s += c->dt_s;
    c->dt_prev_s = c->dt_s;
  }
  return MDG_OK;
}

// -------------------------------------------------------------------------
// C ABI

static int check_sys(mdg_ctx* c, int sys)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (sys < 0 || sys >= c->nsys) return fail(MDG_ERR_ARG, "system index out of range");
  return MDG_OK;
}

static int check_zip(int zip)
{
  if (zip < MDG_ZIP_NONE || zip > MDG_ZIP_XZ) return fail(MDG_ERR_ARG, "unknown compression");
  return MDG_OK;
}

int mdg_set_atom_tags(mdg_ctx* c, const uint8_t* tags)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  int rc = io_wait(c);
  if (rc) return rc;
  if (tags) c->h_tags.assign(tags, tags + c->n);
  else c->h_tags.assign(c->n, 0);
  return MDG_OK;
}

int mdg_get_atom_tags(mdg_ctx* c, uint8_t* tags)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (!tags) return fail(MDG_ERR_ARG, "null argument");
  std::memcpy(tags, c->h_tags.data(), c->n);
  return MDG_OK;
}

static int write_now(mdg_ctx* c, int kind, int sys, const char* path, int zip)
{
  int rc = check_sys(c, sys);
  if (!rc) rc = check_zip(zip);
  if (rc) return rc;
  if (!path || !*path) return fail(MDG_ERR_ARG, "empty file name");
  int slot = 0;
  rc = io_snapshot(c, &slot);
  if (rc) return rc;
  std::vector<IoJob> jobs;
  jobs.push_back(io_job(c, slot, kind, sys, path, zip));
  io_push(c, jobs);
  return io_wait(c);
}

int mdg_write_state(mdg_ctx* c, int sys, const char* id, int zip)
{
  return write_now(c, kJobState, sys, id, zip);
}

int mdg_write_xva(mdg_ctx* c, int sys, const char* path, int zip)
{
  return write_now(c, kJobXva, sys, path, zip);
}

int mdg_set_output(mdg_ctx* c, const char* dir, int64_t flush_interval, double traj_interval, int zip)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  int rc = check_zip(zip);
  if (rc) return rc;
  IoState* io = nullptr;
  if (!dir) {
    if (c->io) c->io->on = false;
    return io_wait(c);
  }
  if (flush_interval < 0 || !(traj_interval >= 0.0) || !std::isfinite(traj_interval))
    return fail(MDG_ERR_ARG, "negative output interval");
  if (!c->n) return fail(MDG_ERR_STATE, "no system loaded");
  rc = io_get(c, &io);
  if (rc) return rc;
  rc = io_wait(c);
  if (rc) return rc;
  io->dir = dir;
  while (io->dir.size() > 1 && io->dir.back() == '/') io->dir.pop_back();
  ::mkdir(io->dir.c_str(), 0755);
  if ((int)io->dirs.size() != c->nsys) io->dirs.clear();
  for (int s = 0; s < c->nsys; s++) ::mkdir(sys_dir(c, s).c_str(), 0755);
  io->flush_interval = flush_interval;
  io->ntraj = traj_interval > 0.0 ? 1 : 0;
  io->traj_until[0] = HUGE_VAL;
  io->traj_int[0] = (c->prm.units == MDG_UNITS_CGS) ? traj_interval : traj_interval * kFs;
  io->zip = zip;
  io->fin.assign(c->nsys, 0);
  io->on = true;
  return MDG_OK;
}

int mdg_flush_output(mdg_ctx* c)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  return io_wait(c);
}

int mdg_get_iteration(mdg_ctx* c, uint64_t* iteration)
{
  if (!c || !iteration) return fail(MDG_ERR_ARG, "null argument");
  *iteration = c->iteration;
  return MDG_OK;
}

int mdg_atom_count(mdg_ctx* c, int* n)
{
  if (!c || !n) return fail(MDG_ERR_ARG, "null argument");
  *n = c->n;
  return MDG_OK;
}

int mdg_set_time_final(mdg_ctx* c, double time_final)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  c->time_final_s = (c->prm.units == MDG_UNITS_CGS) ? time_final : time_final * kFs;
  return MDG_OK;
}

// SimLoopSaver::load(id) with SimLoop::iteration = iteration
// (SimLoopSaver.cxx:275-625, 849-854): replaces the context's system.
int mdg_load_state(mdg_ctx* c, const char* id_c, uint64_t iteration, int* loaded)
{
  if (!c || !id_c || !*id_c) return fail(MDG_ERR_ARG, "null argument");
  int rc = io_wait(c);
  if (rc) return rc;
  const std::string id = id_c;
  std::string err, b;
  int got = 0;
  auto rd = [&](const char* attr) -> int {
    const int k = read_blob(id + attr, b, err);
    if (k < 0) fail(MDG_ERR_IO, err);
    return k;
  };
  // Z numbers and positions fix the atom count (prepareForAttributeReading)
  int k = rd(".z");
  if (k < 0) return MDG_ERR_IO;
  if (k == 0 || b.empty()) return fail(MDG_ERR_ARG, "cannot read Z numbers of " + id);
  const int64_t n = (int64_t)b.size();
  if (n > (1LL << 30)) return fail(MDG_ERR_ARG, "too many atoms");
  std::vector<int32_t> z(n);
  for (int64_t i = 0; i < n; i++) {
    z[i] = z_of_element((uint8_t)b[i]);
    if (z[i] < 0) return fail(MDG_ERR_ARG, "unknown element in " + id + ".z");
  }
  got |= MDG_LOADED_Z;
  auto sized = [&](const char* attr, size_t rec) -> int {
    const int q = rd(attr);
    if (q <= 0) return q;
    if (b.size() != rec * (size_t)n) {
      fail(MDG_ERR_ARG, id + attr + ": size does not match the atom count");
      return -2;
    }
    return 1;
  };
  std::vector<double> r(3 * n), v(3 * n, 0.0), a(3 * n, 0.0);
  k = sized(".r", 24);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k == 0) return fail(MDG_ERR_ARG, "cannot read positions of " + id);
  std::memcpy(r.data(), b.data(), b.size());
  got |= MDG_LOADED_R;
  k = sized(".v", 24);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) { std::memcpy(v.data(), b.data(), b.size()); got |= MDG_LOADED_V; }
  double pr[3] = {kNoPbcCm, kNoPbcCm, kNoPbcCm};
  k = rd(".pbc_rect");
  if (k < 0) return MDG_ERR_IO;
  if (k) {
    if (b.size() != 24) return fail(MDG_ERR_ARG, id + ".pbc_rect: not one vector");
    std::memcpy(pr, b.data(), 24);
    got |= MDG_LOADED_PBC_RECT;
  }
  std::vector<int32_t> img(3 * n, 0);
  k = sized(".pbc_rect.count", 12);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) { std::memcpy(img.data(), b.data(), b.size()); got |= MDG_LOADED_PBC_COUNT; }
  int32_t pbc[3];
  for (int q = 0; q < 3; q++) pbc[q] = pr[q] != kNoPbcCm;
  k = sized(".pbc_rect.enabled", 3);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) {
    // per-atom periodicity: one system here, so every atom must agree
    for (int q = 0; q < 3; q++) pbc[q] = b[q] != 0;
    for (int64_t i = 0; i < n; i++)
      for (int q = 0; q < 3; q++)
        if ((b[3 * i + q] != 0) != (pbc[q] != 0))
          return fail(MDG_ERR_ARG, id + ".pbc_rect.enabled: atoms with different periodicity");
    got |= MDG_LOADED_PBC_ENABLED;
  }
  k = sized(".a", 24);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) { std::memcpy(a.data(), b.data(), b.size()); got |= MDG_LOADED_A; }
  std::vector<unsigned char> fixed(n, 0), tba(n, 1), tags(n, 0);
  k = sized(".tag.fixed", 1);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) for (int64_t i = 0; i < n; i++) fixed[i] = b[i] != 0;
  k = sized(".tag.thermal_bath_applicable", 1);
  if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
  if (k) for (int64_t i = 0; i < n; i++) tba[i] = b[i] != 0;
  static const char* names[6] = {".tag.target", ".tag.projectile", ".tag.substrate",
                                 ".tag.monomer", ".tag.cluster", ".tag.fullerene"};
  for (int t = 0; t < 6; t++) {
    k = sized(names[t], 1);
    if (k < 0) return k == -2 ? MDG_ERR_ARG : MDG_ERR_IO;
    if (k) for (int64_t i = 0; i < n; i++) if (b[i]) tags[i] |= (unsigned char)(1u << (t + 1));
  }
  // thermal bath (geometry NONE unless a geometry file is present)
  int geom = MDG_TB_NONE;
  double T0 = 0.0, gamma_s = 1e13, gp[5] = {0, 0, 0, 0, 0};
  k = rd(".thermal_bath.common");
  if (k < 0) return MDG_ERR_IO;
  if (k) {
    if (b.size() != 16) return fail(MDG_ERR_ARG, id + ".thermal_bath.common: wrong size");
    std::memcpy(&T0, b.data(), 8);
    std::memcpy(&gamma_s, b.data() + 8, 8);
  }
  struct { const char* f; int g; size_t np; } geoms[3] = {
      {".thermal_bath.univserse", MDG_TB_UNIVERSE, 0}, {".thermal_bath.box", MDG_TB_BOX, 3},
      {".thermal_bath.sphere", MDG_TB_SPHERE, 5}};
  for (auto& G : geoms) {
    k = rd(G.f);
    if (k < 0) return MDG_ERR_IO;
    if (!k) continue;
    if (b.size() != 8 * G.np) return fail(MDG_ERR_ARG, id + G.f + ": wrong size");
    std::memcpy(gp, b.data(), b.size());
    geom = G.g;
  }
  double tm[4];
  k = rd(".time");
  if (k < 0) return MDG_ERR_IO;
  const bool have_time = k != 0;
  if (have_time) {
    if (b.size() != 32) return fail(MDG_ERR_ARG, id + ".time: wrong size");
    std::memcpy(tm, b.data(), 32);
  }
  k = rd(".check");
  if (k < 0) return MDG_ERR_IO;
  const bool have_check = k != 0;
  double ck[7] = {0, 0, 0, 1.0, 1.0, 0.0, 0.0};
  if (have_check) {
    if (b.size() != 58) return fail(MDG_ERR_ARG, id + ".check: wrong size");
    std::memcpy(ck, b.data() + 1, 24);
    std::memcpy(ck + 3, b.data() + 26, 32);
  }

  // the system, in internal units
  std::vector<double> pos(3 * n), vel(3 * n);
  double box[3];
  for (int q = 0; q < 3; q++) box[q] = pr[q] / kCgsLen;
  for (int64_t q = 0; q < 3 * n; q++) {
    pos[q] = r[q] / kCgsLen;
    vel[q] = v[q] / kCgsVel;
    // a coordinate just below the period in cm can round to the period in
    // Angstrom: keep it inside [0, L) without changing its image counter
    if (pbc[q % 3] && pos[q] >= box[q % 3]) pos[q] = std::nextafter(box[q % 3], 0.0);
  }
  const int64_t first[2] = {0, n};
  const double ul = c->unit_len, uv = c->unit_vel;
  c->unit_len = c->unit_vel = 1.0;
  rc = set_systems(c, 1, first, z.data(), pos.data(), vel.data(), box, pbc, fixed.data());
  c->unit_len = ul;
  c->unit_vel = uv;
  if (rc) return rc;
  {
    std::vector<int4> him(n);
    for (int64_t i = 0; i < n; i++) him[i] = make_int4(img[3 * i], img[3 * i + 1], img[3 * i + 2], 0);
    CK(cudaMemcpy(c->image, him.data(), n * sizeof(int4), cudaMemcpyHostToDevice));
  }
  if ((got & MDG_LOADED_A) && iteration != 0) {
    // SimLoop computes an only at iteration 0 (SimLoop.cxx:305-321)
    std::vector<double4> ha(n);
    for (int64_t i = 0; i < n; i++)
      ha[i] = fixed[i] ? make_double4(0, 0, 0, 0)
                       : make_double4(a[3 * i] / kCgsAcc, a[3 * i + 1] / kCgsAcc, a[3 * i + 2] / kCgsAcc, 0.0);
    CK(cudaMemcpy(c->acc, ha.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
    c->acc_valid = true;
  }
  // bath
  bool all_on = true;
  for (int64_t i = 0; i < n; i++) all_on = all_on && tba[i];
  if (c->d_tb_apply) cudaFree(c->d_tb_apply);
  c->d_tb_apply = nullptr;
  c->h_tb_apply.clear();
  if (!all_on) {
    c->d_tb_apply = dalloc<unsigned char>(n);
    if (!c->d_tb_apply) return fail(MDG_ERR_CUDA, "cudaMalloc (bath flags)");
    CK(cudaMemcpy(c->d_tb_apply, tba.data(), n, cudaMemcpyHostToDevice));
    c->h_tb_apply = tba;
  }
  c->tb_geom = geom;
  c->tb_T0 = T0;
  c->tb_gamma = gamma_s * kFs;
  for (int q = 0; q < 5; q++) c->tb_gp[q] = gp[q] / kCgsLen;
  if (geom != MDG_TB_NONE) {
    rc = ensure_bath_acct(c);
    if (rc) return rc;
    // loaded atoms start with Atom::an_no_tb = 0 (Atom.cxx:41)
    CK(cudaMemset(c->acc_ntb, 0, n * sizeof(double4)));
  }
  c->step_cfg++;
  // time, iteration, Check
  c->iteration = iteration;
  if (have_time) {
    c->time_s = tm[0];
    c->time_final_s = tm[1];
    c->dt_s = tm[2];
    c->dt_prev_s = tm[3];
    if (c->adaptive) {
      const double t = tm[0] / kFs, d = std::min(std::max(tm[2] / kFs, 1e-5), 0.5), dp = tm[3] / kFs;
      CK(cudaMemcpy(c->d_time, &t, sizeof(double), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(c->d_dt, &d, sizeof(double), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(c->d_dt_prev, &dp, sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  for (int q = 0; q < 3; q++) c->chk_net[q] = ck[q];
  c->chk_e0 = ck[3];
  c->chk_cur = ck[4];
  c->chk_eb0 = ck[5];
  c->chk_T = ck[6];
  c->h_tags = tags;
  c->run_t0 = 0.0;
  if (loaded) *loaded = got;
  return MDG_OK;
}

// -------------------------------------------------------------------------
// SnapshotList (SnapshotList.hpp:38-205) captured on the device: at the top
// of every iteration, for each system whose simTime has crossed a multiple
// of the current interval (CustomSimLoop::isItTimeToSave and its interval
// table, mdtrajsim/main.cpp:52-80), the PBC counters, coordinates and
// velocities of the atoms tagged projectile or cluster
// (SnapshotList::initSelectedAtomList) go into a per-system device list, as
// floats in CGS like SnapshotList::AtomSnapshot.  Both kernels run inside the
// captured step graph: no host round trip per step.

struct SnapRec {        // SnapshotList::AtomSnapshot: 36 bytes, no padding
  int32_t pc[3];
  float p[3];
  float v[3];
};
static_assert(sizeof(SnapRec) == 36, "AtomSnapshot layout");

struct SnapDev {
  int nsel = 0, nsys = 0, cap = 0, nsched = 0;
  const int* sel = nullptr;      // [nsel] selected atoms (context indices), grouped by system
  const int* sel_sys = nullptr;  // [nsel] their systems
  int* cnt = nullptr;            // [nsys] snapshots taken
  double* t = nullptr;           // [nsys * cap] their simTime (s)
  SnapRec* rec = nullptr;        // [cap * nsel]
  double until[4], interval[4];  // interval while simTime < until (s)
};

struct SnapState {
  SnapDev D;
  std::vector<int64_t> off;      // [nsys + 1] each system's selected atoms in sel
  std::vector<uint32_t> local;   // [nsel] index within its system (atomsSelectedForSaving)
  void* mem = nullptr;
};

MDG_HD bool snap_due(const SnapDev& D, double t, double dtp)
{
  double I = D.interval[D.nsched - 1];
  for (int k = 0; k < D.nsched; k++)
    if (t < D.until[k]) { I = D.interval[k]; break; }
  return t == 0.0 || (long long)(t / I) != (long long)((t - dtp) / I);
}

// k-th snapshot of system s is due now (and not already taken at this time,
// SnapshotList::getSnapshot's alreadyAccounted)
MDG_HD int snap_slot(const SnapDev& D, int s, const double* time, const double* dt_prev, const int* stop)
{
  if (stop && stop[s]) return -1;
  const double t = time[s] * kFs, dtp = dt_prev[s] * kFs;
  if (!snap_due(D, t, dtp)) return -1;
  const int k = D.cnt[s];
  if (k > 0 && D.t[(size_t)s * D.cap + k - 1] == t) return -1;
  return k;
}

__global__ void k_snap_atoms(State S, SnapDev D, const double* time, const double* dt_prev, const int* stop)
{
  pdl_enter();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.nsel) return;
  const int s = D.sel_sys[j];
  const int k = snap_slot(D, s, time, dt_prev, stop);
  if (k < 0 || k >= D.cap) return;
  const int a = D.sel[j];
  const double4 p = S.pos[a], u = S.vel[a];
  const int4 m = S.image[a];
  SnapRec r;
  r.pc[0] = m.x; r.pc[1] = m.y; r.pc[2] = m.z;
  r.p[0] = (float)(p.x * kCgsLen); r.p[1] = (float)(p.y * kCgsLen); r.p[2] = (float)(p.z * kCgsLen);
  r.v[0] = (float)(u.x * kCgsVel); r.v[1] = (float)(u.y * kCgsVel); r.v[2] = (float)(u.z * kCgsVel);
  D.rec[(size_t)k * D.nsel + j] = r;
}

// after k_snap_atoms (which reads the counts): record the time, count it
__global__ void k_snap_commit(SnapDev D, const double* time, const double* dt_prev, const int* stop,
                              unsigned int* status)
{
  pdl_enter();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= D.nsys) return;
  const int k = snap_slot(D, s, time, dt_prev, stop);
  if (k < 0) return;
  if (k >= D.cap) { atomicOr(status, ST_SNAP_OVERFLOW); return; }
  D.t[(size_t)s * D.cap + k] = time[s] * kFs;
  D.cnt[s] = k + 1;
}

namespace {  // declared beside free_system

void snap_free(mdg_ctx* c)
{
  if (!c->snap) return;
  if (c->snap->mem) cudaFree(c->snap->mem);
  delete c->snap;
  c->snap = nullptr;
}

int snap_capture(mdg_ctx* c)
{
  SnapState* Z = c->snap;
  if (!Z) return MDG_OK;
  const int* stop = c->stop_final ? c->d_stop : nullptr;
  State S = c->S();
  if (Z->D.nsel > 0)
    LAUNCH(c, "snap_atoms", k_snap_atoms, nblk(Z->D.nsel), kThreads, S, Z->D, c->d_time, c->d_dt_prev, stop);
  LAUNCH(c, "snap_commit", k_snap_commit, nblk(c->nsys), kThreads, Z->D, c->d_time, c->d_dt_prev, stop,
         c->d_status);
  return MDG_OK;
}

// Host copy of system sys's snapshots: times (s) and records [nshots][natoms].
int snap_fetch(mdg_ctx* c, int sys, std::vector<double>& t, std::vector<SnapRec>& rec, int& natoms)
{
  SnapState* Z = c->snap;
  int cnt = 0;
  CK(cudaMemcpyAsync(&cnt, Z->D.cnt + sys, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  natoms = (int)(Z->off[sys + 1] - Z->off[sys]);
  t.resize(cnt);
  rec.resize((size_t)cnt * natoms);
  if (cnt) CK(cudaMemcpy(t.data(), Z->D.t + (size_t)sys * Z->D.cap, cnt * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<SnapRec> all((size_t)cnt * Z->D.nsel);
  if (cnt && Z->D.nsel)
    CK(cudaMemcpy(all.data(), Z->D.rec, all.size() * sizeof(SnapRec), cudaMemcpyDeviceToHost));
  for (int k = 0; k < cnt; k++)
    for (int j = 0; j < natoms; j++) rec[(size_t)k * natoms + j] = all[(size_t)k * Z->D.nsel + Z->off[sys] + j];
  return MDG_OK;
}

// SnapshotList::writestate (binary "snapshots.conf") or saveInText.
int snap_write(mdg_ctx* c, int sys, const std::string& path, int zip, bool text)
{
  std::vector<double> t;
  std::vector<SnapRec> rec;
  int na = 0;
  int rc = snap_fetch(c, sys, t, rec, na);
  if (rc) return rc;
  const uint32_t* loc = c->snap->local.data() + c->snap->off[sys];
  std::string err;
  if (!text) {
    Rec b;
    b.put<uint32_t>((uint32_t)na);
    for (int j = 0; j < na; j++) b.put<uint32_t>(loc[j]);
    b.put<uint32_t>((uint32_t)t.size());
    for (size_t k = 0; k < t.size(); k++) {
      b.put<double>(t[k]);
      b.put<uint32_t>((uint32_t)na);
      b.b.append((const char*)(rec.data() + k * na), sizeof(SnapRec) * na);
    }
    if (!write_blob(path, b.b.data(), b.b.size(), zip, err)) return fail(MDG_ERR_IO, err);
    return MDG_OK;
  }
  // saveInText: default ostream formatting (%g)
  std::string s;
  for (int j = 0; j < na; j++) appendf(s, "%u ", loc[j]);
  s += "\n";
  for (size_t k = 0; k < t.size(); k++) {
    appendf(s, "%g\n", t[k]);
    for (int j = 0; j < na; j++) {
      const SnapRec& r = rec[k * na + j];
      appendf(s, "%d %d %d \n%g %g %g \n%g %g %g \n", r.pc[0], r.pc[1], r.pc[2], (double)r.p[0], (double)r.p[1],
              (double)r.p[2], (double)r.v[0], (double)r.v[1], (double)r.v[2]);
    }
  }
  if (!write_blob(path, s.data(), s.size(), zip, err)) return fail(MDG_ERR_IO, err);
  return MDG_OK;
}

}  // namespace

// -------------------------------------------------------------------------
// C ABI: snapshots, simTimeFinal, per-system output

int mdg_snapshots_enable(mdg_ctx* c, int on, int capacity)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  snap_free(c);
  c->step_cfg++;
  if (!on) return MDG_OK;
  if (!c->adaptive) return fail(MDG_ERR_STATE, "snapshots follow simTime: enable the adaptive time step first");
  if (capacity <= 0 || capacity > (1 << 24)) return fail(MDG_ERR_ARG, "snapshot capacity out of range");
  SnapState* Z = new SnapState();
  Z->off.assign(c->nsys + 1, 0);
  std::vector<int> sel, sys;
  for (int s = 0; s < c->nsys; s++) {
    const int64_t b = c->nsys > 1 ? c->h_first[s] : 0, e = c->nsys > 1 ? c->h_first[s + 1] : c->n;
    for (int64_t i = b; i < e; i++)
      if (c->h_tags[i] & ((1u << 2) | (1u << 5))) {  // ATOMTAG_PROJECTILE | ATOMTAG_CLUSTER
        sel.push_back((int)i);
        sys.push_back(s);
        Z->local.push_back((uint32_t)(i - b));
      }
    Z->off[s + 1] = (int64_t)sel.size();
  }
  SnapDev& D = Z->D;
  D.nsel = (int)sel.size();
  D.nsys = c->nsys;
  D.cap = capacity;
  // CustomSimLoop's intervals (mdtrajsim/main.cpp:62-80), in its own expressions
  D.nsched = 3;
  D.until[0] = 2.0 * 1e-12;
  D.until[1] = 4.0 * 1e-12;
  D.until[2] = HUGE_VAL;
  D.interval[0] = 5e-16 * 5 * 4;
  D.interval[1] = 5e-16 * 25 * 4;
  D.interval[2] = 5e-16 * 50 * 4;
  const size_t b_sel = 2 * sizeof(int) * (size_t)D.nsel, b_cnt = sizeof(int) * (size_t)c->nsys,
               b_t = sizeof(double) * (size_t)c->nsys * capacity, b_rec = sizeof(SnapRec) * (size_t)capacity * D.nsel;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* m = nullptr;
  if (cudaMalloc((void**)&m, up(b_sel) + up(b_cnt) + up(b_t) + up(b_rec) + 256) != cudaSuccess) {
    delete Z;
    return fail(MDG_ERR_CUDA, "cudaMalloc (snapshots)");
  }
  Z->mem = m;
  int* dsel = (int*)m;
  D.sel = dsel;
  D.sel_sys = dsel + D.nsel;
  D.cnt = (int*)(m + up(b_sel));
  D.t = (double*)(m + up(b_sel) + up(b_cnt));
  D.rec = (SnapRec*)(m + up(b_sel) + up(b_cnt) + up(b_t));
  c->snap = Z;
  if (D.nsel) {
    CK(cudaMemcpy(dsel, sel.data(), D.nsel * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dsel + D.nsel, sys.data(), D.nsel * sizeof(int), cudaMemcpyHostToDevice));
  }
  CK(cudaMemset(D.cnt, 0, b_cnt));
  return MDG_OK;
}

int mdg_snapshots_set_schedule(mdg_ctx* c, int n, const double* until, const double* interval)
{
  if (!c || !c->snap) return fail(MDG_ERR_STATE, "snapshots are not enabled");
  if (n < 1 || n > 4 || !until || !interval) return fail(MDG_ERR_ARG, "1 to 4 schedule entries");
  const double tc = (c->prm.units == MDG_UNITS_CGS) ? 1.0 : kFs;  // time unit -> s
  for (int k = 0; k < n; k++) {
    if (!(interval[k] > 0.0)) return fail(MDG_ERR_ARG, "snapshot intervals must be positive");
    c->snap->D.until[k] = until[k] * tc;
    c->snap->D.interval[k] = interval[k] * tc;
  }
  c->snap->D.nsched = n;
  c->step_cfg++;
  return MDG_OK;
}

int mdg_snapshots_count(mdg_ctx* c, int sys, int* nshots, int* natoms)
{
  int rc = check_sys(c, sys);
  if (rc) return rc;
  if (!c->snap) return fail(MDG_ERR_STATE, "snapshots are not enabled");
  int cnt = 0;
  CK(cudaMemcpyAsync(&cnt, c->snap->D.cnt + sys, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  rc = read_status(c);
  if (rc) return rc;
  if (nshots) *nshots = cnt;
  if (natoms) *natoms = (int)(c->snap->off[sys + 1] - c->snap->off[sys]);
  return MDG_OK;
}

int mdg_snapshots_get(mdg_ctx* c, int sys, double* times, uint32_t* indices, int32_t* pbc_count, float* pos,
                      float* vel)
{
  int rc = check_sys(c, sys);
  if (rc) return rc;
  if (!c->snap) return fail(MDG_ERR_STATE, "snapshots are not enabled");
  std::vector<double> t;
  std::vector<SnapRec> rec;
  int na = 0;
  rc = snap_fetch(c, sys, t, rec, na);
  if (rc) return rc;
  const double tc = (c->prm.units == MDG_UNITS_CGS) ? 1.0 : 1.0 / kFs;
  for (size_t k = 0; k < t.size(); k++)
    if (times) times[k] = t[k] * tc;
  if (indices)
    for (int j = 0; j < na; j++) indices[j] = c->snap->local[c->snap->off[sys] + j];
  for (size_t q = 0; q < rec.size(); q++)
    for (int a = 0; a < 3; a++) {
      if (pbc_count) pbc_count[3 * q + a] = rec[q].pc[a];
      if (pos) pos[3 * q + a] = rec[q].p[a];
      if (vel) vel[3 * q + a] = rec[q].v[a];
    }
  return MDG_OK;
}

int mdg_snapshots_write(mdg_ctx* c, int sys, const char* path, int zip, int text)
{
  int rc = check_sys(c, sys);
  if (!rc) rc = check_zip(zip);
  if (rc) return rc;
  if (!c->snap) return fail(MDG_ERR_STATE, "snapshots are not enabled");
  if (!path || !*path) return fail(MDG_ERR_ARG, "empty file name");
  return snap_write(c, sys, path, zip, text != 0);
}

// SnapshotList::loadstate: earlier snapshots of system sys, so that a resumed
// trajectory appends to them.
int mdg_snapshots_load(mdg_ctx* c, int sys, const char* path)
{
  int rc = check_sys(c, sys);
  if (rc) return rc;
  if (!c->snap) return fail(MDG_ERR_STATE, "snapshots are not enabled");
  std::string b, err;
  const int k = read_blob(path, b, err);
  if (k < 0) return fail(MDG_ERR_IO, err);
  if (k == 0) return fail(MDG_ERR_ARG, std::string("no snapshot list ") + path);
  SnapState* Z = c->snap;
  const int na = (int)(Z->off[sys + 1] - Z->off[sys]);
  size_t o = 0;
  auto get = [&](void* dst, size_t n) {
    if (o + n > b.size()) return false;
    std::memcpy(dst, b.data() + o, n);
    o += n;
    return true;
  };
  uint32_t nsel = 0, nshots = 0;
  if (!get(&nsel, 4) || (int)nsel != na) return fail(MDG_ERR_ARG, "snapshot list: selected atoms differ");
  for (int j = 0; j < na; j++) {
    uint32_t v = 0;
    if (!get(&v, 4) || v != Z->local[Z->off[sys] + j]) return fail(MDG_ERR_ARG, "snapshot list: selected atoms differ");
  }
  if (!get(&nshots, 4)) return fail(MDG_ERR_ARG, "snapshot list: truncated");
  if ((int)nshots > Z->D.cap) return fail(MDG_ERR_CAPACITY, "snapshot list larger than the capacity");
  std::vector<double> t(nshots);
  std::vector<SnapRec> all((size_t)nshots * Z->D.nsel);
  if (nshots && Z->D.nsel)
    CK(cudaMemcpy(all.data(), Z->D.rec, all.size() * sizeof(SnapRec), cudaMemcpyDeviceToHost));
  for (uint32_t q = 0; q < nshots; q++) {
    uint32_t sz = 0;
    if (!get(&t[q], 8) || !get(&sz, 4) || (int)sz != na) return fail(MDG_ERR_ARG, "snapshot list: truncated");
    for (int j = 0; j < na; j++)
      if (!get(&all[(size_t)q * Z->D.nsel + Z->off[sys] + j], sizeof(SnapRec)))
        return fail(MDG_ERR_ARG, "snapshot list: truncated");
  }
  if (nshots && Z->D.nsel)
    CK(cudaMemcpy(Z->D.rec, all.data(), all.size() * sizeof(SnapRec), cudaMemcpyHostToDevice));
  if (nshots) CK(cudaMemcpy(Z->D.t + (size_t)sys * Z->D.cap, t.data(), nshots * sizeof(double), cudaMemcpyHostToDevice));
  const int cnt = (int)nshots;
  CK(cudaMemcpy(Z->D.cnt + sys, &cnt, sizeof(int), cudaMemcpyHostToDevice));
  return MDG_OK;
}

int mdg_set_stop_at_time_final(mdg_ctx* c, int on)
{
  if (!c) return fail(MDG_ERR_ARG, "null context");
  c->stop_final = on != 0;
  if (c->n && c->d_stop) CK(cudaMemset(c->d_stop, 0, c->nsys * sizeof(int)));
  c->step_cfg++;
  return MDG_OK;
}

int mdg_run_until_final(mdg_ctx* c, int64_t max_steps, int64_t* steps, int* finished)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (!c->adaptive || !c->stop_final)
    return fail(MDG_ERR_STATE, "needs the adaptive time step and mdg_set_stop_at_time_final");
  int64_t done = 0;
  int all = 0;
  std::vector<int> st((size_t)c->nsys);
  while (done < max_steps) {
    const int chunk = (int)std::min<int64_t>(16, max_steps - done);
    int rc = run_steps(c, chunk, 0.5, nullptr, nullptr, done == 0);
    if (rc) return rc;
    done += chunk;
    CK(cudaMemcpyAsync(st.data(), c->d_stop, c->nsys * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    rc = read_status(c);
    if (rc) return rc;
    all = 1;
    for (int v : st) all = all && v;
    if (all) break;
  }
  if (steps) *steps = done;
  if (finished) *finished = all;
  return io_wait(c);
}

int mdg_set_time(mdg_ctx* c, const double* sim_time, const double* dt)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (!sim_time || !dt) return fail(MDG_ERR_ARG, "null argument");
  const double tc = (c->prm.units == MDG_UNITS_CGS) ? 1.0 / kFs : 1.0;  // time unit -> fs
  std::vector<double> t(c->nsys), d(c->nsys);
  for (int s = 0; s < c->nsys; s++) {
    if (!(dt[s] > 0.0) || !std::isfinite(sim_time[s])) return fail(MDG_ERR_ARG, "bad time or dt");
    t[s] = sim_time[s] * tc;
    d[s] = std::min(std::max(dt[s] * tc, 1e-5), 0.5);
  }
  CK(cudaMemcpy(c->d_time, t.data(), c->nsys * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_dt, d.data(), c->nsys * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_dt_prev, d.data(), c->nsys * sizeof(double), cudaMemcpyHostToDevice));
  c->time_s = t[0] * kFs;
  c->dt_s = c->dt_prev_s = d[0] * kFs;
  return MDG_OK;
}

int mdg_set_output_dirs(mdg_ctx* c, const char* const* dirs)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  IoState* io = nullptr;
  int rc = io_get(c, &io);
  if (!rc) rc = io_wait(c);
  if (rc) return rc;
  io->dirs.clear();
  if (!dirs) return MDG_OK;
  for (int s = 0; s < c->nsys; s++) {
    if (!dirs[s] || !*dirs[s]) return fail(MDG_ERR_ARG, "empty directory name");
    io->dirs.push_back(dirs[s]);
    ::mkdir(dirs[s], 0755);
  }
  return MDG_OK;
}

int mdg_set_traj_schedule(mdg_ctx* c, int n, const double* until, const double* interval)
{
  if (!c || !c->io || !c->io->on) return fail(MDG_ERR_STATE, "call mdg_set_output first");
  if (n < 0 || n > 4 || (n && (!until || !interval))) return fail(MDG_ERR_ARG, "0 to 4 schedule entries");
  const double tc = (c->prm.units == MDG_UNITS_CGS) ? 1.0 : kFs;
  for (int k = 0; k < n; k++) {
    if (!(interval[k] > 0.0)) return fail(MDG_ERR_ARG, "trajectory intervals must be positive");
    c->io->traj_until[k] = until[k] * tc;
    c->io->traj_int[k] = interval[k] * tc;
  }
  c->io->ntraj = n;
  return MDG_OK;
}

int mdg_set_images(mdg_ctx* c, const int32_t* image)
{
  if (!c || !c->n) return fail(MDG_ERR_STATE, "no system loaded");
  if (!image) return fail(MDG_ERR_ARG, "null argument");
  std::vector<int4> h(c->n);
  for (int i = 0; i < c->n; i++) h[i] = make_int4(image[3 * i], image[3 * i + 1], image[3 * i + 2], 0);
  CK(cudaMemcpy(c->image, h.data(), c->n * sizeof(int4), cudaMemcpyHostToDevice));
  return MDG_OK;
}
