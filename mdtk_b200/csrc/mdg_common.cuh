// Shared definitions for the mdg kernels: vector type, species, parameters,
// cutoff functions, status flags.
//
// Internal units: Angstrom, eV, fs, amu.  The reference works in CGS
// (mdtk/consts.cxx:28-36); conversion happens only at the C ABI edge.
#pragma once
#include <type_traits>

#include <stdint.h>
#include <math.h>

#if !defined(__CUDACC__)
#include <vector_types.h>
#include <vector_functions.h>
#endif

#if defined(__CUDACC__)
#define MDG_HD __host__ __device__ __forceinline__
#define MDG_DEV __device__ __forceinline__
#else
#define MDG_HD inline
#define MDG_DEV inline
#endif

namespace mdg {

constexpr double kPi = 3.14159265358979323846;  // M_PI
// 1 eV/(Angstrom*amu) in Angstrom/fs^2, from the reference's eV and amu
// (mdtk/consts.cxx:28-31): 1.6021e-12 erg / (1e-8 cm * 1.6605655e-24 g) * 1e8 / 1e30
constexpr double kAccConv = 1.6021e-12 / 1.6605655e-24 * 1e16 / 1e30;

constexpr int kC = 0;  // species index of carbon (REBO::C, REBO.hpp:157)
constexpr int kH = 1;  // species index of hydrogen (REBO::H, REBO.hpp:158)

// Status bits written by kernels (never a trap): the host turns them into
// MDG_ERR_* codes.  Mirrors the reference's REQUIRE checks on the path.
enum StatusBits : unsigned int {
  ST_NL_OVERFLOW = 1u << 0,     // a Verlet list exceeded its capacity
  ST_BOND_OVERFLOW = 1u << 1,   // more bonds than the per-atom bond capacity
  ST_COS_RANGE = 1u << 2,       // CosTheta outside [-1-1e-7, 1+1e-7] (FGeneral.hpp:147)
  ST_N_NEGATIVE = 1u << 3,      // coordination below -1e-15 (REBO.cxx:434,462,489)
  ST_NONFINITE = 1u << 4,       // NaN/Inf energy or force
  ST_CIJ_OVERFLOW = 1u << 5,    // connectivity table capacity exceeded
  ST_RECORD_OVERFLOW = 1u << 7, // bond-task or special-pair record capacity exceeded
  ST_SPLINE_DOMAIN = 1u << 8,   // spline argument outside its domain (cubici.hpp:90,211,305)
  ST_CELL_OVERFLOW = 1u << 9,   // cell grid capacity exceeded
  ST_SNAP_OVERFLOW = 1u << 10,  // snapshot list capacity exceeded
};

#if defined(__CUDACC__)
// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialisation attribute may be scheduled while the grid before it on
// the stream is still draining; the first statement of every such kernel is
// this call, which waits until that grid has completed and its memory writes
// are visible (griddepcontrol.wait, a no-op for a kernel launched without the
// attribute), and then lets the next grid be scheduled in turn.  Completion
// is thereby transitive along the stream, as with ordinary launches.
#if !defined(MDG_TIMELINE)
__device__ __forceinline__ void pdl_enter()
{
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#else
// The timeline build (python -m mdtk_b200.build --timeline, a separate
// library): pdl_enter() also stamps, per kernel (keyed by the source line of
// its pdl_enter() call), the global timer when the first block started, when
// it passed the wait, and when the last warp left (a destructor on every
// return path).  Atomics on 8192-entry arrays; read back by
// mdg_timeline_read.  Never in the product library.
constexpr int kTimelineSlots = 8192;
__device__ unsigned long long g_tl_start[kTimelineSlots];
__device__ unsigned long long g_tl_wait[kTimelineSlots];
__device__ unsigned long long g_tl_end[kTimelineSlots];
__device__ __forceinline__ unsigned long long tl_now()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
struct TimelineStamp {
  int id;
  __device__ __forceinline__ explicit TimelineStamp(int line) : id(line % kTimelineSlots)
  {
    if (threadIdx.x == 0) atomicMin(&g_tl_start[id], tl_now());
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0) atomicMin(&g_tl_wait[id], tl_now());
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  }
  __device__ __forceinline__ ~TimelineStamp()
  {
    if ((threadIdx.x & 31) == 0) atomicMax(&g_tl_end[id], tl_now());
  }
};
#define pdl_enter() TimelineStamp mdg_timeline_stamp_(__LINE__)
#endif
#endif

// FP32 scalar of the mixed-precision path: float arithmetic; double operands
// (parameters, literals, loads from the FP64 bond list) convert to float
// implicitly, conversion back to double is explicit (dbl()).
struct f32 {
  float v;
  f32() = default;
  MDG_HD f32(double x) : v((float)x) {}
  MDG_HD explicit operator double() const { return (double)v; }
  // Math functions as hidden friends: found only through an f32 argument, so
  // they never hide the double functions for FP64 code in this namespace.
  friend MDG_HD f32 exp(f32 a) { f32 r; r.v = expf(a.v); return r; }
  friend MDG_HD f32 sqrt(f32 a) { f32 r; r.v = sqrtf(a.v); return r; }
  friend MDG_HD f32 cos(f32 a) { f32 r; r.v = cosf(a.v); return r; }
  friend MDG_HD f32 sin(f32 a) { f32 r; r.v = sinf(a.v); return r; }
  friend MDG_HD f32 fabs(f32 a) { f32 r; r.v = fabsf(a.v); return r; }
  friend MDG_HD f32 pow(f32 a, f32 b) { f32 r; r.v = powf(a.v, b.v); return r; }
};
MDG_HD f32 mkf(float x) { f32 r; r.v = x; return r; }
MDG_HD f32 operator+(f32 a, f32 b) { return mkf(a.v + b.v); }
MDG_HD f32 operator-(f32 a, f32 b) { return mkf(a.v - b.v); }
MDG_HD f32 operator*(f32 a, f32 b) { return mkf(a.v * b.v); }
MDG_HD f32 operator/(f32 a, f32 b) { return mkf(a.v / b.v); }
MDG_HD f32 operator-(f32 a) { return mkf(-a.v); }
MDG_HD f32& operator+=(f32& a, f32 b) { a.v += b.v; return a; }
MDG_HD f32& operator-=(f32& a, f32 b) { a.v -= b.v; return a; }
MDG_HD f32& operator*=(f32& a, f32 b) { a.v *= b.v; return a; }
MDG_HD bool operator<(f32 a, f32 b) { return a.v < b.v; }
MDG_HD bool operator>(f32 a, f32 b) { return a.v > b.v; }
MDG_HD bool operator<=(f32 a, f32 b) { return a.v <= b.v; }
MDG_HD bool operator>=(f32 a, f32 b) { return a.v >= b.v; }
MDG_HD bool operator==(f32 a, f32 b) { return a.v == b.v; }
MDG_HD bool operator!=(f32 a, f32 b) { return a.v != b.v; }
MDG_HD double dbl(double x) { return x; }
// Slack of the reference's coordination check N > -1e-15 (REBO.cxx:434): in
// float, N = N_t - f rounds to about -5e-7 where it is 0.
MDG_HD double n_neg_tol(double) { return 1e-15; }
MDG_HD double n_neg_tol(f32) { return 1e-5; }
MDG_HD double dbl(f32 x) { return (double)x.v; }

// Forward-mode dual number (value, tangent) of the adjoint path: the force
// code run on duals whose position tangents are u gives, in the tangent of
// every output, its derivative along u (the tangent of the gradient is the
// Jacobian product J u).  Ordering compares values; equality compares value
// and tangent, so a "skip when zero" test never drops a nonzero tangent.
struct dual {
  double v, d;
  dual() = default;
  MDG_HD dual(double x) : v(x), d(0.0) {}
  MDG_HD dual(double x, double t) : v(x), d(t) {}
  friend MDG_HD dual exp(dual a) { const double e = exp(a.v); return dual(e, e * a.d); }
  friend MDG_HD dual sqrt(dual a) { const double s = sqrt(a.v); return dual(s, a.d / (2.0 * s)); }
  friend MDG_HD dual cos(dual a) { return dual(cos(a.v), -sin(a.v) * a.d); }
  friend MDG_HD dual sin(dual a) { return dual(sin(a.v), cos(a.v) * a.d); }
  friend MDG_HD dual fabs(dual a) { return a.v < 0 ? dual(-a.v, -a.d) : a; }
  friend MDG_HD dual pow(dual a, double b) { return dual(pow(a.v, b), b * pow(a.v, b - 1.0) * a.d); }
};
MDG_HD dual operator+(dual a, dual b) { return dual(a.v + b.v, a.d + b.d); }
MDG_HD dual operator-(dual a, dual b) { return dual(a.v - b.v, a.d - b.d); }
MDG_HD dual operator*(dual a, dual b) { return dual(a.v * b.v, a.d * b.v + a.v * b.d); }
MDG_HD dual operator/(dual a, dual b) { const double q = a.v / b.v; return dual(q, (a.d - q * b.d) / b.v); }
MDG_HD dual operator-(dual a) { return dual(-a.v, -a.d); }
MDG_HD dual& operator+=(dual& a, dual b) { a.v += b.v; a.d += b.d; return a; }
MDG_HD dual& operator-=(dual& a, dual b) { a.v -= b.v; a.d -= b.d; return a; }
MDG_HD dual& operator*=(dual& a, dual b) { a = a * b; return a; }
MDG_HD bool operator<(dual a, dual b) { return a.v < b.v; }
MDG_HD bool operator>(dual a, dual b) { return a.v > b.v; }
MDG_HD bool operator<=(dual a, dual b) { return a.v <= b.v; }
MDG_HD bool operator>=(dual a, dual b) { return a.v >= b.v; }
MDG_HD bool operator==(dual a, dual b) { return a.v == b.v && a.d == b.d; }
MDG_HD bool operator!=(dual a, dual b) { return !(a == b); }
MDG_HD dual dbl(dual x) { return x; }
MDG_HD double n_neg_tol(dual) { return 1e-15; }
// value of a scalar (for indices and types stored in floating-point fields)
MDG_HD double val(double x) { return x; }
MDG_HD double val(dual x) { return x.v; }

// A dual vector's values with zero tangents.
template <class Real>
MDG_HD Real value_only(Real x) { return Real(val(x)); }

// The wide type of an arithmetic type: what its results are stored and
// accumulated in (double for the FP64 and FP32-mixed paths, dual on the
// adjoint path).
template <class Real> struct Wide { typedef double T; };
template <> struct Wide<dual> { typedef dual T; };

template <class T> struct IsDual { static constexpr bool v = false; };
template <> struct IsDual<dual> { static constexpr bool v = true; };

// Four wide scalars (x, y, z, w) of a stored record: double4 on the FP64 and
// mixed paths.
struct dual4 {
  dual x, y, z, w;
};
template <class W> struct Q4T { typedef double4 T; };
template <> struct Q4T<dual> { typedef dual4 T; };
MDG_HD dual4 make_dual4(dual x, dual y, dual z, dual w) { dual4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
MDG_HD double4 make_q4(double x, double y, double z, double w) { return make_double4(x, y, z, w); }
MDG_HD dual4 make_q4(dual x, dual y, dual z, dual w) { return make_dual4(x, y, z, w); }

template <class T> struct Id { typedef T type; };

template <class Real>
struct V3T {
  Real x, y, z;
};
typedef V3T<double> V3;
MDG_HD V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
template <class Real>
MDG_HD V3T<Real> v3r(Real x, Real y, Real z) { V3T<Real> r; r.x = x; r.y = y; r.z = z; return r; }
// xyz of a double4 in the arithmetic type Real
template <class Real>
MDG_HD V3T<Real> xyz(double4 q) { return v3r<Real>(Real(q.x), Real(q.y), Real(q.z)); }
template <class Real>
MDG_HD V3T<Real> xyz(const dual4& q) { return v3r<Real>(Real(q.x), Real(q.y), Real(q.z)); }
template <class Real>
MDG_HD V3T<Real> cvt3(V3 a) { return v3r<Real>(Real(a.x), Real(a.y), Real(a.z)); }
template <class Real>
MDG_HD V3T<typename Wide<Real>::T> to_d(V3T<Real> a)
{
  return v3r<typename Wide<Real>::T>(dbl(a.x), dbl(a.y), dbl(a.z));
}
template <class Real>
MDG_HD V3T<Real> operator+(V3T<Real> a, V3T<Real> b) { return v3r<Real>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class Real>
MDG_HD V3T<Real> operator-(V3T<Real> a, V3T<Real> b) { return v3r<Real>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class Real>
MDG_HD V3T<Real> operator-(V3T<Real> a) { return v3r<Real>(-a.x, -a.y, -a.z); }
template <class Real>
MDG_HD V3T<Real> operator*(V3T<Real> a, typename Id<Real>::type s) { return v3r<Real>(a.x * s, a.y * s, a.z * s); }
template <class Real>
MDG_HD V3T<Real> operator*(typename Id<Real>::type s, V3T<Real> a) { return v3r<Real>(a.x * s, a.y * s, a.z * s); }
template <class Real>
MDG_HD V3T<Real> operator/(V3T<Real> a, typename Id<Real>::type s) { return v3r<Real>(a.x / s, a.y / s, a.z / s); }
template <class Real>
MDG_HD void operator+=(V3T<Real>& a, V3T<Real> b) { a.x += b.x; a.y += b.y; a.z += b.z; }
template <class Real>
MDG_HD void operator-=(V3T<Real>& a, V3T<Real> b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
// same evaluation order as mdtk Vector3D scalarmul/vectormul (Vector3D.hpp:272-282)
template <class Real>
MDG_HD Real dot(V3T<Real> a, V3T<Real> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class Real>
MDG_HD V3T<Real> cross(V3T<Real> a, V3T<Real> b)
{
  return v3r<Real>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class Real>
MDG_HD Real norm2(V3T<Real> a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// Squared length in double with every product and sum rounded on its own (no
// FMA contraction): a distance computed in two kernels is then the same
// number, so a cutoff f_ij subtracted from a coordination sum N_i cancels it
// exactly (the reference's check N > -1e-15, REBO.cxx:434), and it equals the
// reference's own x*x + y*y + z*z.
MDG_HD double norm2(V3 a)
{
#if defined(__CUDA_ARCH__)
  return __dadd_rn(__dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)), __dmul_rn(a.z, a.z));
#else
  return a.x * a.x + a.y * a.y + a.z * a.z;
#endif
}
template <class Real>
MDG_HD Real SQR(Real x) { return x * x; }
template <class Real>
MDG_HD V3T<Real> values_of(V3T<Real> a) { return v3r<Real>(value_only(a.x), value_only(a.y), value_only(a.z)); }

// Parameters the adjoint differentiates (their order in gradients), the
// C-C pair parameters of the LJ term (AIREBO_LJ.cxx:229-247) and of REBO's
// V_R / V_A (REBO.cxx:859-938).
enum ParamId : int {
  kParLJEps = 0,      // epsilon_CC (AIREBO's zeta_)
  kParLJSigma = 1,    // sigma_CC
  kParReboA = 2,      // A_CC
  kParReboB1 = 3,     // B1_CC
  kParReboAlpha = 4,  // alpha_CC
  kParReboBeta1 = 5,  // beta1_CC
  kNParam = 6
};

// Periodic box: only uniform per-axis periodicity (every atom shares the
// array's PBC, as AtomsArray::PBC sets it, mdtk/AtomsContainer.cxx:43-54).
struct Box {
  double L[3];
  int pbc[3];
};

// Minimum-image displacement a1 - a2 for atoms wrapped into [0, L) on
// periodic axes: one shift by L when |r| > L/2 (depos, mdtk/Atom.hpp:116-140,
// the equal-PBC branch).
MDG_HD double depos1(double r, double L, int p)
{
  if (p && fabs(r) > L * 0.5) r += (r > 0) ? (-L) : (L);
  return r;
}
MDG_HD V3 depos(const Box& b, V3 a1, V3 a2)
{
  return v3(depos1(a1.x - a2.x, b.L[0], b.pbc[0]),
            depos1(a1.y - a2.y, b.L[1], b.pbc[1]),
            depos1(a1.z - a2.z, b.L[2], b.pbc[2]));
}

// Cosine cutoff of AtomsPair (AtomsPair.hpp:137-158): f = 1 below R1,
// (1 + cos(pi (r-R1)/(R2-R1)))/2 on [R1, R2), 0 beyond; df = df/dr.
template <class Real>
MDG_HD void cutoff(Real r, double R1, double R2, Real& f, Real& df)
{
  if (r < R1) { f = 1.0; df = 0.0; return; }
  if (r < R2) {
    if constexpr (std::is_same<Real, double>::value) {
      double sn, cs;
      sincos(kPi * (r - R1) / (R2 - R1), &sn, &cs);
      f = (1.0 + cs) / 2.0;
      df = (-(kPi / (R2 - R1)) * sn) / 2.0;
    } else {
      f = (1.0 + cos(kPi * (r - R1) / (R2 - R1))) / 2.0;
      df = (-(kPi / (R2 - R1)) * sin(kPi * (r - R1) / (R2 - R1))) / 2.0;
    }
    return;
  }
  f = 0.0;
  df = 0.0;
}

// Sprime / dSprime (REBO.cxx:67-106): 1 below min, 0 above max, cosine between.
template <class Real>
MDG_HD Real Sprime(Real arg, double amin, double amax)
{
  if (arg < amin) return 1.0;
  if (arg > amax) return 0.0;
  return (1.0 + cos(kPi * (arg - amin) / (amax - amin))) / 2.0;
}
template <class Real>
MDG_HD Real dSprime(Real arg, double amin, double amax)
{
  if (arg < amin) return 0.0;
  if (arg > amax) return 0.0;
  return (-(kPi / (amax - amin)) * sin(kPi * (arg - amin) / (amax - amin))) / 2.0;
}

// REBO parameter set (REBO::setupPotential1, REBO.cxx:857-938) in A / eV.
struct ReboParams {
  double Q[2][2], alpha[2][2], A[2][2];
  double B[3][2][2], beta[3][2][2];
  double rho[2][2];
  double R[2][2][2];      // R[a][b][0] = R1, [1] = R2 (cosine cutoff f)
  double Rp[2][2][2];     // Rprime (fprime of the dihedral term)
  double Ntot[2];         // Sprime window of N for G_C and Nconj
};

// AIREBO LJ parameters (AIREBO::setupPotential, AIREBO_LJ.cxx:219-287).
struct LJParams {
  double sigma[2][2], eps[2][2];
  double RLJ[2][2][2];    // S(t_r) window: [sigma, 2^(1/6) sigma]
  double R[2][2][2];      // LJ cosine cutoff window
  double b[2][2][2];      // S(t_b) window on b*_ij
  // chain factors of the adjoint's parameters: d sigma_ab / d sigma_CC,
  // d eps_ab / d eps_CC (sigma_CH is the mean, eps_CH the geometric mean),
  // and d R_ab / d sigma_ab of the cutoff window (3 in the 3-sigma mode)
  double dsig[2][2], deps[2][2];
  double dcut;
};

// ETors parameters (ETors::setupPotential, AIREBO_ETors.cxx:125-133).
struct TorsParams {
  double eps[2][2];
};

}  // namespace mdg
