// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Stand-in for the KMC library's header (the reference's extern/KMC
// submodule, which is empty in the reference tree), so that the reference's
// own src/crosslink.cpp compiles into the checker.  Written from the call
// sites in src/crosslink.cpp (Crosslink::SinglyKMC, :57-127) alone: the
// names and signatures it uses, nothing of the library's implementation.
// The checker places crosslinks doubly bound with zero unbinding rate and no
// diffusion, so binding -- the only path that would run this class -- never
// runs: every member is an inert stub, and whichRodBindSD reports failure.
#ifndef SCREF_KMC_STUB_HPP
#define SCREF_KMC_STUB_HPP

#include <vector>

class LookupTable {};

template <class T>
class KMC {
 public:
  KMC(const double * /*pos*/, int /*n_neighbors*/, double /*delta*/, LookupTable * /*lut*/) {}
  void SetPBCs(int /*n_dim*/, int /*n_periodic*/, const double * /*unit_cell*/) {}
  template <class L, class F, class B>
  void LUCalcTotProbsSD(L /*neighbors*/, F & /*filter*/, int /*bound_oid*/,
                        B & /*bind_factors*/) {}
  double getTotProb() const { return 0.0; }
  int whichRodBindSD(double &bind_lambda, double /*roll*/) {
    bind_lambda = 0.0;
    return -1;
  }
};

#endif
