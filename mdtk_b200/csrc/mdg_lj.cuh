// AIREBO intermolecular LJ term (mdtk/potentials/manybody/AIREBO/AIREBO_LJ.cxx):
// parameters and per-pair device code.
#pragma once

#include "mdg_rebo.cuh"

namespace mdg {

// AIREBO::setupPotential (AIREBO_LJ.cxx:219-287), A / eV.  lj_cut_mode 1
// replaces the cosine cutoff window by [3 sigma - 0.5, 3 sigma].
inline void set_lj_params(LJParams& p, int lj_cut_mode)
{
  const int C = kC, H = kH;
  p.sigma[C][C] = 3.40;
  p.sigma[H][H] = 2.65;
  p.sigma[C][H] = p.sigma[H][C] = 0.5 * (p.sigma[C][C] + p.sigma[H][H]);
  p.eps[C][C] = 0.00284;
  p.eps[H][H] = 0.00150;
  p.eps[C][H] = p.eps[H][C] = sqrt(p.eps[C][C] * p.eps[H][H]);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      p.RLJ[a][b][0] = p.sigma[a][b];
      p.RLJ[a][b][1] = p.sigma[a][b] * pow(2.0, 1.0 / 6.0);
    }
  p.R[C][C][0] = 5.0;
  p.R[H][H][0] = 4.0;
  p.R[C][H][0] = p.R[H][C][0] = 4.5;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) p.R[a][b][1] = p.R[a][b][0] + 0.5;
  if (lj_cut_mode == 1)
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++) {
        p.R[a][b][1] = 3.0 * p.sigma[a][b];
        p.R[a][b][0] = p.R[a][b][1] - 0.5;
      }
  p.b[C][C][0] = 0.77;
  p.b[H][H][0] = 0.32;
  p.b[C][H][0] = p.b[H][C][0] = 0.75;
  p.b[C][C][1] = 0.81;
  p.b[H][H][1] = 0.42;
  p.b[C][H][1] = p.b[H][C][1] = 0.90;
}

}  // namespace mdg

#if defined(__CUDACC__)
namespace mdg {
struct LJState {
  int n = 0;
};
inline void lj_free(LJState& s) { s.n = 0; }
inline int lj_alloc(LJState& s, int n, int, int, int) { s.n = n; return 0; }
inline int lj_evaluate(LJState&, const State&, const NList&, const BondList&, const ReboParams*, const ReboTables*,
                       const LJParams&, const ForceOut&, cudaStream_t, unsigned int*, int64_t*, const double4**)
{
  return -1;
}
}  // namespace mdg
#endif
