/*
 * Drop-in MDTK potentials evaluated on the GPU through the mdg C ABI
 * (include/mdg.h, library mdtk_b200/libmdg.so).
 *
 * GpuREBO, GpuAIREBO, GpuETors and GpuBrenner are mdtk::FManybody classes
 * (mdtk/potentials/manybody/FManybody.hpp:33-45) that stand in for REBO
 * (mdtk/potentials/manybody/AIREBO/REBO.hpp), AIREBO (AIREBO_LJ.hpp), ETors
 * (AIREBO_ETors.hpp) and Brenner (Brenner/Brenner.hpp) inside an unchanged
 * FProxy / SimLoop:
 *
 *   GpuStack* s = new GpuStack(MDG_POT_AIREBO);       // one device context
 *   loop.fpot.addPotential(new GpuREBO(s));            // applications/common.h:60-71
 *   loop.fpot.addPotential(new GpuAIREBO(s));
 *   loop.fpot.addPotential(new GpuETors(s));
 *
 * The reference's AIREBO reads its REBO instance's lists and bond orders
 * (AIREBO_LJ.cxx:196-212, 299-344); here the terms of a stack share one
 * device context that evaluates them together.  FProxy::operator() zeroes
 * Atom::grad and calls its potentials in order (FProxy.cxx:46-61): the first
 * term called at new positions evaluates the whole stack on the device and
 * adds the stack's gradient into Atom::grad; the stack's other terms then
 * return their own energies and add nothing.  A term called a second time
 * before its siblings starts a new evaluation.  So the terms of one stack
 * are used together, in one FProxy, as the reference uses REBO with AIREBO.
 *
 * Neighbour lists live on the device: NL_init loads the atoms and builds the
 * lists, NL_checkRequestUpdate loads the current positions and rebuilds the
 * lists whose displacement check (NeighbourList::MovedTooMuch,
 * NeighbourList.cxx:109-133) fires (mdg_nl_update); the device measures the
 * displacements from the positions, so incDisplacement has nothing to do.
 * After each device build a term copies its list into its NeighbourList, so
 * FGeneral::NL and FProxy::hasNeighbors (SimLoop.cxx:394-398) see the
 * reference's lists.  Errors come back as yaatk::Exception,
 * the reference's own (REQUIRE), which SimLoop::execute catches
 * (SimLoop.cxx:176-205).
 *
 * Units are MDTK's own (CGS: cm, erg), set through MDG_UNITS_CGS.  Elements
 * are H and C, as for the classes they replace.  The header is C++98, like the
 * code it is added to.
 */
#ifndef MDTK_GPU_POTENTIALS_HPP
#define MDTK_GPU_POTENTIALS_HPP

#include <cstring>
#include <vector>

#include <yaatk/Exception.hpp>
#include <mdtk/potentials/manybody/FManybody.hpp>

#include "mdg.h"

namespace mdtk
{

class GpuStack
{
public:
  // the stack's terms and their slots in mdg_compute's e_terms
  enum Term { TERM_REBO = 0, TERM_LJ = 1, TERM_TORS = 2, TERM_BRENNER = 3 };

  // potentials: MDG_POT_* flags of the whole stack (REBO or Brenner among
  // them); brenner_set: 1 or 2 (Brenner::POTENTIAL1 / POTENTIAL2,
  // Brenner.cxx:498-611); lj_cut_mode: mdg_params::lj_cut_mode
  explicit GpuStack(int potentials, int brenner_set = 1, int lj_cut_mode = 0)
    : ctx_(0), refs_(0), lj_cut_mode_(lj_cut_mode), served_(0), n_(0), loaded_(false), evaluated_(false),
      grad_pending_(false)
  {
    mdg_params p;
    mdg_default_params(&p);
    p.potentials = potentials;
    p.brenner_set = brenner_set;
    p.lj_cut_mode = lj_cut_mode;
    p.units = MDG_UNITS_CGS;
    if (mdg_create(&p, &ctx_) != MDG_OK) throw yaatk::Exception(mdg_last_error());
    for (int t = 0; t < 4; t++) eterms_[t] = 0.0;
    for (int l = 0; l < 3; l++) builds_[l] = 0;
  }

  // the device context (for the C ABI's other entry points)
  mdg_ctx* context() { return ctx_; }

  void attach() { refs_++; }
  // FProxy::freePotentials deletes each term; the last one frees the stack
  void detach()
  {
    if (--refs_ == 0) delete this;
  }

  // cutoffs of the classes replaced: the largest R2 of their pair types
  // (REBO.hpp:147 and Brenner.hpp:107, C-C 2.0 A; ETors is a REBO;
  // AIREBO_LJ.hpp:88, C-C 5.5 A, AIREBO_LJ.cxx:249-262, or 3 sigma_CC =
  // 10.2 A in the 3-sigma mode)
  Float rcutoff(Term t) const
  {
    if (t == TERM_LJ) return (lj_cut_mode_ == 1 ? 3.0 * 3.4 : 5.5) * Ao;
    return 2.0 * Ao;
  }

  // NL_init: load the atoms and build every list
  void nl_init(AtomsArray& atoms)
  {
    load(atoms, true);
    int32_t rebuilt[3];
    check(mdg_nl_update(ctx_, 1, rebuilt));
    for (int l = 0; l < 3; l++) builds_[l]++;
  }

  // NL_checkRequestUpdate / NL_UpdateIfNeeded: load the current positions
  // and rebuild the lists whose displacement check fires
  void nl_update(AtomsArray& atoms)
  {
    load(atoms, false);
    int32_t rebuilt[3] = {0, 0, 0};
    check(mdg_nl_update(ctx_, 0, rebuilt));
    for (int l = 0; l < 3; l++) builds_[l] += rebuilt[l];
  }

  // how many times list l (0: REBO / Brenner / torsion, 1: AIREBO LJ) was built
  unsigned long builds(int l) const { return builds_[l]; }

  // the device's list l as the reference's NeighbourList holds it:
  // nl[i] = the partners of atom i in ascending order (NeighbourList.cxx:73-106
  // pushes them so), so that FGeneral::NL and FProxy::hasNeighbors read
  // what they read from the reference's own lists
  void export_list(AtomsArray& atoms, int l, std::vector<AtomRefsContainer>& nl)
  {
    int64_t cnt = 0;
    check(mdg_nl_pairs(ctx_, l, 0, 0, &cnt));
    std::vector<int32_t> pairs(2 * (size_t)cnt + 2);
    check(mdg_nl_pairs(ctx_, l, &pairs[0], cnt, &cnt));
    nl.resize(atoms.size());
    for (size_t i = 0; i < nl.size(); i++) nl[i].clear();
    for (int64_t q = 0; q < cnt; q++) {
      const int32_t i = pairs[2 * q], j = pairs[2 * q + 1];
      nl[i].push_back(&atoms[j]);
      nl[j].push_back(&atoms[i]);
    }
  }

  // FGeneral::operator() of term t
  Float energy(AtomsArray& atoms, Term t)
  {
    pack(atoms);
    const unsigned bit = 1u << t;
    const bool same = evaluated_ && pos_.size() == at_eval_.size() &&
                      std::memcmp(&pos_[0], &at_eval_[0], pos_.size() * sizeof(double)) == 0;
    if (!same || (served_ & bit)) {
      load(atoms, false);
      grad_.assign(pos_.size(), 0.0);
      double e = 0.0;
      check(mdg_compute(ctx_, &e, eterms_, &grad_[0]));
      at_eval_ = pos_;
      evaluated_ = true;
      served_ = 0;
      grad_pending_ = true;
    }
    served_ |= bit;
    if (grad_pending_) {
      for (size_t i = 0; i < atoms.size(); i++)
        atoms[i].grad += Vector3D(grad_[3 * i], grad_[3 * i + 1], grad_[3 * i + 2]);
      grad_pending_ = false;
    }
    return eterms_[t == TERM_BRENNER ? 0 : (int)t];
  }

private:
  ~GpuStack() { mdg_destroy(ctx_); }
  GpuStack(const GpuStack&);
  GpuStack& operator=(const GpuStack&);

  static void check(int rc)
  {
    if (rc != MDG_OK) throw yaatk::Exception(mdg_last_error());
  }

  void pack(AtomsArray& atoms)
  {
    pos_.resize(3 * atoms.size());
    for (size_t i = 0; i < atoms.size(); i++) {
      pos_[3 * i] = atoms[i].coords.x;
      pos_[3 * i + 1] = atoms[i].coords.y;
      pos_[3 * i + 2] = atoms[i].coords.z;
    }
  }

  // the atom set on the device: loaded whole when it is new (or on NL_init),
  // otherwise only positions that changed since the last upload
  void load(AtomsArray& atoms, bool whole)
  {
    pack(atoms);
    if (whole || !loaded_ || atoms.size() != n_) {
      const size_t n = atoms.size();
      std::vector<int32_t> z(n);
      std::vector<uint8_t> fixed(n);
      for (size_t i = 0; i < n; i++) {
        if (atoms[i].ID == H_EL) z[i] = 1;
        else if (atoms[i].ID == C_EL) z[i] = 6;
        else throw yaatk::Exception("GPU potentials handle H and C only");
        fixed[i] = atoms[i].isFixed() ? 1 : 0;
      }
      const Vector3D L = atoms.PBC();
      const double box[3] = {L.x, L.y, L.z};
      const int32_t pbc[3] = {L.x != NO_PBC.x, L.y != NO_PBC.y, L.z != NO_PBC.z};
      check(mdg_set_system(ctx_, (int)n, &z[0], &pos_[0], 0, box, pbc, &fixed[0]));
      n_ = n;
      loaded_ = true;
      evaluated_ = false;
    } else if (pos_ != uploaded_) {
      check(mdg_set_positions(ctx_, &pos_[0]));
    } else {
      return;
    }
    uploaded_ = pos_;
  }

  mdg_ctx* ctx_;
  int refs_;
  int lj_cut_mode_;
  unsigned served_;   // terms that have returned their energy since the last evaluation
  size_t n_;
  bool loaded_, evaluated_, grad_pending_;
  std::vector<double> pos_, uploaded_, at_eval_, grad_;
  double eterms_[4];
  unsigned long builds_[3];
};

// One term of a GpuStack, with FGeneral's interface (FGeneral.hpp:54-114).
class GpuTerm : public FManybody
{
public:
  GpuTerm(GpuStack* stack, GpuStack::Term term) : FManybody(), stack_(stack), term_(term), seen_(0)
  {
    stack_->attach();
    handledElements.insert(H_EL);
    handledElements.insert(C_EL);
    nl.Rcutoff = getRcutoff();
  }
  virtual ~GpuTerm() { stack_->detach(); }

  GpuStack* stack() { return stack_; }

  Float operator()(AtomsArray& atoms) { return stack_->energy(atoms, term_); }
  Float getRcutoff() const { return stack_->rcutoff(term_); }

  // FProxy::NL_init and NL_checkRequestUpdate call these on every potential
  // in order (FProxy.hpp:59-71); the stack's first term (REBO or Brenner)
  // does the device work and every term then copies its own list out when
  // the device rebuilt it.  nl.ListUpdateRequested stays false, so
  // FProxy::NL_UpdateIfNeeded never runs the CPU list build on these terms.
  void NL_init(AtomsArray& atoms)
  {
    nl.init(atoms);
    nl.ListUpdateRequested = false;
    if (first()) stack_->nl_init(atoms);
    refresh(atoms);
  }
  void NL_checkRequestUpdate(AtomsArray& atoms)
  {
    if (first()) stack_->nl_update(atoms);
    refresh(atoms);
    nl.ListUpdateRequested = false;
  }
  void NL_UpdateIfNeeded(AtomsArray& atoms) { NL_checkRequestUpdate(atoms); }
  // the device measures displacements from the positions themselves
  void incDisplacement(Atom&, Vector3D) {}

private:
  bool first() const { return term_ == GpuStack::TERM_REBO || term_ == GpuStack::TERM_BRENNER; }
  int list_id() const { return term_ == GpuStack::TERM_LJ ? 1 : 0; }
  void refresh(AtomsArray& atoms)
  {
    const unsigned long b = stack_->builds(list_id());
    if (b != seen_) {
      stack_->export_list(atoms, list_id(), nl.nl);
      seen_ = b;
    }
  }
  GpuStack* stack_;
  GpuStack::Term term_;
  unsigned long seen_;  // the stack's build count of this term's list when nl.nl was copied
};

// REBO (AIREBO/REBO.hpp) on the device
class GpuREBO : public GpuTerm
{
public:
  explicit GpuREBO(GpuStack* s) : GpuTerm(s, GpuStack::TERM_REBO) {}
};

// AIREBO's intermolecular LJ term (AIREBO/AIREBO_LJ.hpp) on the device
class GpuAIREBO : public GpuTerm
{
public:
  explicit GpuAIREBO(GpuStack* s) : GpuTerm(s, GpuStack::TERM_LJ) {}
};

// AIREBO's torsion term (AIREBO/AIREBO_ETors.hpp) on the device
class GpuETors : public GpuTerm
{
public:
  explicit GpuETors(GpuStack* s) : GpuTerm(s, GpuStack::TERM_TORS) {}
};

// first-generation Brenner (Brenner/Brenner.hpp) on the device
class GpuBrenner : public GpuTerm
{
public:
  explicit GpuBrenner(GpuStack* s) : GpuTerm(s, GpuStack::TERM_BRENNER) {}
};

}  // namespace mdtk

#endif
