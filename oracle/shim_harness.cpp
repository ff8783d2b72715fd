/*
 * Oracle-side binding of the drop-in GPU potentials (test infrastructure only;
 * loaded by tests/, never by the product).
 *
 * mdtk_b200/mdtk/GpuPotentials.hpp holds the classes a maintainer adds to
 * MDTK: GpuREBO, GpuAIREBO, GpuETors and GpuBrenner, FManybody potentials
 * over the mdg C ABI.  This file compiles them against the reference's own
 * headers and installs a factory in the oracle harness (ref_harness.cpp), so
 * that a harness context created with POT_GPU holds them in its FProxy in
 * place of REBO, AIREBO, ETors or Brenner, and the reference's unmodified
 * FProxy::operator() and SimLoop::execute drive the GPU path.
 *
 * The potential stack is built in the reference's order
 * (applications/common.h:60-71): REBO, AIREBO (LJ), ETors, or Brenner.
 */
#include <string>

#include <mdtk/potentials/FProxy.hpp>

#include "../mdtk_b200/mdtk/GpuPotentials.hpp"

using namespace mdtk;

typedef const char* (*shim_factory_fn)(int potset, int brenner_set, int lj_cut_mode, FProxy* fpot);
extern "C" int ref_set_gpu_factory(shim_factory_fn f);

namespace {

// the harness's potential-set bits (ref_harness.cpp)
enum { POT_REBO = 1, POT_AIREBO_LJ = 2, POT_ETORS = 4, POT_BRENNER = 8 };

std::string g_names, g_error;

const char* make_stack(int potset, int brenner_set, int lj_cut_mode, FProxy* fpot)
{
  try {
    int flags = 0;
    if (potset & POT_REBO) flags |= MDG_POT_REBO;
    if (potset & POT_AIREBO_LJ) flags |= MDG_POT_AIREBO_LJ;
    if (potset & POT_ETORS) flags |= MDG_POT_ETORS;
    if (potset & POT_BRENNER) flags |= MDG_POT_BRENNER;
    if (potset & ~(POT_REBO | POT_AIREBO_LJ | POT_ETORS | POT_BRENNER)) {
      g_error = "the GPU classes cover REBO, AIREBO, ETors and Brenner";
      return 0;
    }
    GpuStack* s = new GpuStack(flags, brenner_set, lj_cut_mode);
    s->attach();  // held while the terms are added
    g_names.clear();
    if (potset & POT_REBO) {
      fpot->addPotential(new GpuREBO(s));
      g_names += "GpuREBO,";
    }
    if (potset & POT_AIREBO_LJ) {
      fpot->addPotential(new GpuAIREBO(s));
      g_names += "GpuAIREBO,";
    }
    if (potset & POT_ETORS) {
      fpot->addPotential(new GpuETors(s));
      g_names += "GpuETors,";
    }
    if (potset & POT_BRENNER) {
      fpot->addPotential(new GpuBrenner(s));
      g_names += "GpuBrenner,";
    }
    s->detach();
    if (!g_names.empty()) g_names.erase(g_names.size() - 1);
    return g_names.c_str();
  } catch (yaatk::Exception& e) {
    g_error = e.what();
    return 0;
  }
}

}  // namespace

extern "C" {

int shim_install() { return ref_set_gpu_factory(&make_stack); }

const char* shim_last_error() { return g_error.c_str(); }

}
