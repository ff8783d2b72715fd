// REBO (+ torsion) energy and gradient without any device allocation.
//
// Some callers cannot call cudaMalloc: a host framework that owns every byte
// of device memory through its own allocator and forbids driver allocations
// by its plugins, or a time-critical loop where the implicit device-wide
// synchronisation of cudaMalloc/cudaFree would break the step budget.  This
// entry point serves them: the caller passes device buffers for the inputs
// and outputs, and every intermediate (neighbour list, bond list, per-bond
// accumulators, per-atom energies, status word) lives in one file-scope
// static device array of fixed size, kNoAllocMaxAtoms atoms' worth.  Every
// GPU that loads the library keeps that array (and the spline tables) until
// the process exits.
//
// The kernels are the same per-atom work items the context path uses
// (mdg_step.cuh); only where their buffers live differs.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "mdg.h"
#include "mdg_step.cuh"
#include "mdg_tables.h"

using namespace mdg;

namespace {

constexpr int kNoAllocMaxAtoms = 4096;
constexpr int kMB = 16;        // bond slots per atom
constexpr int kNLCap = 64;     // REBO-range Verlet partners per atom
constexpr int kMaxDevices = 64;

// Byte layout of the scratch array (offsets are 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t N = kNoAllocMaxAtoms;
constexpr size_t OFF_POS = 0;
constexpr size_t OFF_NLCNT = align256(OFF_POS + N * sizeof(double4));
constexpr size_t OFF_NL = align256(OFF_NLCNT + N * sizeof(int));
constexpr size_t OFF_NLPOS0 = align256(OFF_NL + N * kNLCap * sizeof(int));
constexpr size_t OFF_NB = align256(OFF_NLPOS0 + N * sizeof(double4));
constexpr size_t OFF_BJ = align256(OFF_NB + N * sizeof(int));
constexpr size_t OFF_BREV = align256(OFF_BJ + N * kMB * sizeof(int));
constexpr size_t OFF_BRV = align256(OFF_BREV + N * kMB * sizeof(int));
constexpr size_t OFF_BU = align256(OFF_BRV + N * kMB * sizeof(double4));
constexpr size_t OFF_BD = align256(OFF_BU + N * kMB * sizeof(double4));
constexpr size_t OFF_NCO = align256(OFF_BD + N * kMB * sizeof(double4));
constexpr size_t OFF_A = align256(OFF_NCO + N * sizeof(double4));
constexpr size_t OFF_W = align256(OFF_A + N * kMB * 3 * sizeof(double));
constexpr size_t OFF_GOWN = align256(OFF_W + N * kMB * sizeof(double));
constexpr size_t OFF_EREBO = align256(OFF_GOWN + N * sizeof(double4));
constexpr size_t OFF_ETORS = align256(OFF_EREBO + N * sizeof(double));
constexpr size_t OFF_ELJ = align256(OFF_ETORS + N * sizeof(double));
constexpr size_t OFF_STATUS = align256(OFF_ELJ + N * sizeof(double));
constexpr size_t kScratchBytes = align256(OFF_STATUS + sizeof(unsigned int));
static_assert(kScratchBytes < 12u * 1024u * 1024u, "no-alloc scratch above its stated 12 MiB bound");

// The scratch array, its spline tables and parameters: static device memory.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ ReboTables g_noalloc_tables;
static __device__ ReboParams g_noalloc_params;

struct DeviceSetup {
  bool ready = false;
  unsigned char* scratch = nullptr;
  ReboTables* tables = nullptr;
  ReboParams* params = nullptr;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

// status bit of this file: an atomic number other than 1 or 6
constexpr unsigned int ST_NA_ELEMENT = 1u << 20;

}  // namespace

// Defined in mdg_api.cu: makes the message visible through mdg_last_error().
void mdg_set_last_error_internal(const char* msg);

namespace {

int na_fail(int code, const std::string& msg)
{
  mdg_set_last_error_internal(msg.c_str());
  return code;
}

// Once per device, with that device current: resolve the device addresses of
// the static arrays (their host-side names are only stand-ins) and upload the
// spline tables and parameters.
int na_setup(int dev, DeviceSetup** out)
{
  if (dev < 0 || dev >= kMaxDevices) return na_fail(MDG_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (!s.ready) {
    cudaError_t e = cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void**)&s.tables, g_noalloc_tables);
    if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    e = cudaGetSymbolAddress((void**)&s.params, g_noalloc_params);
    if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    static ReboTables host_tables;  // host copy, built once per process
    static bool built = false;
    if (!built) {
      build_rebo_tables(&host_tables, nullptr);
      built = true;
    }
    ReboParams hp;
    fill_rebo_params(hp);
    e = cudaMemcpyToSymbol(g_noalloc_tables, &host_tables, sizeof(ReboTables));
    if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaMemcpyToSymbol: ") + cudaGetErrorString(e));
    e = cudaMemcpyToSymbol(g_noalloc_params, &hp, sizeof(ReboParams));
    if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaMemcpyToSymbol: ") + cudaGetErrorString(e));
    s.ready = true;
  }
  *out = &s;
  return MDG_OK;
}

struct NaView {
  State S;
  NList L;
  Grid G;
  BondBuild BB;
  BondList B;
  ForceOut O;
  unsigned int* status;
};

NaView na_view(unsigned char* base, int n, const Box& box)
{
  NaView v;
  std::memset(&v, 0, sizeof(v));
  v.S.n = n;
  v.S.box = box;
  v.S.pos = (double4*)(base + OFF_POS);
  v.L.cap = kNLCap;
  v.L.cnt = (int*)(base + OFF_NLCNT);
  v.L.list = (int*)(base + OFF_NL);
  v.L.pos0 = (double4*)(base + OFF_NLPOS0);
  const double range = (1.0 + 0.44) * 2.0;  // NeighbourList range of REBO (Rcutoff 2.0 A)
  v.L.range2 = range * range;
  v.G.brute = 1;
  v.BB.n = n;
  v.BB.mb = kMB;
  v.BB.nb = (int*)(base + OFF_NB);
  v.BB.bj = (int*)(base + OFF_BJ);
  v.BB.brev = (int*)(base + OFF_BREV);
  v.BB.brv = (double4*)(base + OFF_BRV);
  v.BB.bu = (double4*)(base + OFF_BU);
  v.BB.bd = (double4*)(base + OFF_BD);
  v.BB.nco = (double4*)(base + OFF_NCO);
  v.B.n = n;
  v.B.mb = kMB;
  v.B.nb = v.BB.nb;
  v.B.bj = v.BB.bj;
  v.B.brev = v.BB.brev;
  v.B.brv = v.BB.brv;
  v.B.bu = v.BB.bu;
  v.B.bd = v.BB.bd;
  v.B.nco = v.BB.nco;
  v.O.mb = kMB;
  v.O.A = (double*)(base + OFF_A);
  v.O.W = (double*)(base + OFF_W);
  v.O.gown = (double4*)(base + OFF_GOWN);
  v.O.glj = nullptr;
  v.O.e_rebo = (double*)(base + OFF_EREBO);
  v.O.e_tors = (double*)(base + OFF_ETORS);
  v.O.e_lj = (double*)(base + OFF_ELJ);
  v.status = (unsigned int*)(base + OFF_STATUS);
  return v;
}

// Positions into the scratch (wrapped into the box, Atom::applyPBC) with the
// species index in w; unknown elements are reported through the status word.
__global__ void k_na_pack(NaView v, const double* pos, const int32_t* z)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.S.n) return;
  double x[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  int im[3] = {0, 0, 0};
  bool ok = true;
  for (int a = 0; a < 3; a++) {
    if (!isfinite(x[a])) ok = false;
    else if (v.S.box.pbc[a]) ok &= wrap1(x[a], im[a], v.S.box.L[a]);
  }
  if (!ok) atomicOr(v.status, ST_NONFINITE);
  int t = kC;
  if (z[i] == 1) t = kH;
  else if (z[i] != 6) atomicOr(v.status, ST_NA_ELEMENT);
  v.S.pos[i] = make_double4(x[0], x[1], x[2], (double)t);
}

__global__ void k_na_nl(NaView v)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < v.S.n) nl_build_atom(v.S, v.G, v.L, i, v.status);
}

__global__ void k_na_bonds(NaView v, const ReboParams* P)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < v.S.n) bonds_atom(v.S, v.L, *P, v.BB, a, v.status);
}

__global__ void k_na_brev(NaView v)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a < v.S.n) brev_atom(v.BB, a);
}

__global__ void k_na_rebo(NaView v, const ReboParams* P, const ReboTables* T, TorsParams TP, int do_tors)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= v.S.n) return;
  Rebo R{*P, *T, v.B, v.status};
  rebo_atom(R, TP, 1, do_tors, v.O, a);
}

__global__ void k_na_gather(NaView v, double* grad)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= v.S.n) return;
  V3 g = gather_atom(v.B, v.O, a, 0, nullptr);
  if (!isfinite(g.x) || !isfinite(g.y) || !isfinite(g.z)) atomicOr(v.status, ST_NONFINITE);
  grad[3 * a] = g.x;
  grad[3 * a + 1] = g.y;
  grad[3 * a + 2] = g.z;
}

// Deterministic energy sums (one block, fixed order).
__global__ void k_na_energy(NaView v, double* energy)
{
  __shared__ double sr[256], st[256];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < v.S.n; i += blockDim.x) {
    a += v.O.e_rebo[i];
    b += v.O.e_tors[i];
  }
  sr[threadIdx.x] = a;
  st[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sr[threadIdx.x] += sr[threadIdx.x + w];
      st[threadIdx.x] += st[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    energy[0] = sr[0];
    energy[1] = st[0];
    if (!isfinite(sr[0]) || !isfinite(st[0])) atomicOr(v.status, ST_NONFINITE);
  }
}

}  // namespace

extern "C" {

// See include/mdg.h.  The first call on a device performs that device's
// set-up (symbol addresses, table upload with synchronous copies), so it should
// come before any stream capture.  All calls share one scratch array: calls
// that overlap on the GPU (other streams, other host threads) race.
int mdg_rebo_compute_noalloc(int n, const double* pos, const int32_t* z, const double box[3], const int32_t pbc[3],
                             int with_torsion, double* energy, double* grad, void* stream)
{
  if (n <= 0 || n > kNoAllocMaxAtoms)
    return na_fail(MDG_ERR_ARG, "mdg_rebo_compute_noalloc: n must be in [1, 4096] (its static scratch holds "
                                "4096 atoms)");
  if (!pos || !z || !box || !pbc || !energy || !grad) return na_fail(MDG_ERR_ARG, "null argument");
  Box bx;
  for (int a = 0; a < 3; a++) {
    bx.pbc[a] = pbc[a] ? 1 : 0;
    bx.L[a] = bx.pbc[a] ? box[a] : 0.0;
    if (bx.pbc[a] && !(bx.L[a] > 4.0))
      return na_fail(MDG_ERR_ARG, "Rcutoff is too large for given PBC (AtomsArray::checkMIC)");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  DeviceSetup* s = nullptr;
  int rc = na_setup(dev, &s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  NaView v = na_view(s->scratch, n, bx);
  // the status word is the only scratch that must start at zero
  e = cudaMemsetAsync(v.status, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  TorsParams tp;
  fill_tors_params(tp);
  const int T = 128, B = (n + T - 1) / T;
  k_na_pack<<<B, T, 0, st>>>(v, pos, z);
  k_na_nl<<<B, T, 0, st>>>(v);
  k_na_bonds<<<B, T, 0, st>>>(v, s->params);
  k_na_brev<<<B, T, 0, st>>>(v);
  k_na_rebo<<<B, T, 0, st>>>(v, s->params, s->tables, tp, with_torsion ? 1 : 0);
  k_na_gather<<<B, T, 0, st>>>(v, grad);
  k_na_energy<<<1, 256, 0, st>>>(v, energy);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  unsigned int status = 0;
  e = cudaMemcpyAsync(&status, v.status, sizeof(status), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return na_fail(MDG_ERR_CUDA, std::string("status read: ") + cudaGetErrorString(e));
  if (status & ST_NA_ELEMENT) return na_fail(MDG_ERR_ARG, "unknown element (only H = 1 and C = 6)");
  if (status & ST_SPLINE_DOMAIN) return na_fail(MDG_ERR_SPLINE_DOMAIN, "spline argument out of its domain");
  if (status & ST_NONFINITE) return na_fail(MDG_ERR_NONFINITE, "non-finite position, energy or force");
  if (status & ST_NL_OVERFLOW) return na_fail(MDG_ERR_NL_OVERFLOW, "more than 64 list partners for an atom");
  if (status & ST_BOND_OVERFLOW) return na_fail(MDG_ERR_BOND_OVERFLOW, "more than 16 bonds for an atom");
  if (status & ST_COS_RANGE) return na_fail(MDG_ERR_COS_RANGE, "cos(theta) out of range");
  if (status & ST_N_NEGATIVE) return na_fail(MDG_ERR_N_NEGATIVE, "negative coordination");
  return MDG_OK;
}

}  // extern "C"
