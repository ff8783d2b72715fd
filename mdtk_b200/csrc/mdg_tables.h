// Host builders of the spline tables (see mdg_tables.cpp).
#pragma once

#include <vector>

#include "mdg_spline.cuh"

namespace mdg {

// Fills the device-layout REBO tables; when flat_out is given, also returns
// the tables flattened in the oracle's export order (for the bitwise check).
void build_rebo_tables(ReboTables* tb, std::vector<double>* flat_out);

// FP32 tables of the mixed-precision path: the same cell polynomials
// re-expanded about each cell's lower corner, rounded to float.
void build_rebo_tables32(const ReboTables& d, ReboTables32* f);

// REBO::setupPotential1 (REBO.cxx:857-938) and ETors::setupPotential
// (AIREBO_ETors.cxx:125-133) parameters, Angstrom / eV.
void fill_rebo_params(ReboParams& p);
void fill_tors_params(TorsParams& t);

struct BrennerTables;
// Brenner H_CC / H_CH / F tables of parameter set 1 or 2, same layout rules.
void build_brenner_tables(int set, BrennerTables* tb, std::vector<double>* flat_out);

}  // namespace mdg
