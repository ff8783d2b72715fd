// Shared definitions for the mdg kernels: vector type, species, parameters,
// cutoff functions, status flags.
//
// Internal units: Angstrom, eV, fs, amu.  The reference works in CGS
// (mdtk/consts.cxx:28-36); conversion happens only at the C ABI edge.
#pragma once

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
};

struct V3 {
  double x, y, z;
};
MDG_HD V3 v3(double x, double y, double z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
MDG_HD V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
MDG_HD V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
MDG_HD V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
MDG_HD V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
MDG_HD V3 operator*(double s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }
MDG_HD V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
MDG_HD void operator+=(V3& a, V3 b) { a.x += b.x; a.y += b.y; a.z += b.z; }
MDG_HD void operator-=(V3& a, V3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
// same evaluation order as mdtk Vector3D scalarmul/vectormul (Vector3D.hpp:272-282)
MDG_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MDG_HD V3 cross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
MDG_HD double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
MDG_HD double SQR(double x) { return x * x; }

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
MDG_HD void cutoff(double r, double R1, double R2, double& f, double& df)
{
  if (r < R1) { f = 1.0; df = 0.0; return; }
  if (r < R2) {
    f = (1.0 + cos(kPi * (r - R1) / (R2 - R1))) / 2.0;
    df = (-(kPi / (R2 - R1)) * sin(kPi * (r - R1) / (R2 - R1))) / 2.0;
    return;
  }
  f = 0.0;
  df = 0.0;
}

// Sprime / dSprime (REBO.cxx:67-106): 1 below min, 0 above max, cosine between.
MDG_HD double Sprime(double arg, double amin, double amax)
{
  if (arg < amin) return 1.0;
  if (arg > amax) return 0.0;
  return (1.0 + cos(kPi * (arg - amin) / (amax - amin))) / 2.0;
}
MDG_HD double dSprime(double arg, double amin, double amax)
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
};

// ETors parameters (ETors::setupPotential, AIREBO_ETors.cxx:125-133).
struct TorsParams {
  double eps[2][2];
};

}  // namespace mdg
