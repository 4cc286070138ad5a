// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// Stand-in for the KMC library's choice helper, written from its call sites
// in the reference's src/crosslink.cpp (:89, :147, :152): given the
// probabilities of two events in one step and a uniform roll, the index of
// the event that happens (0 or 1), or -1 for neither.  With the zero
// unbinding rates the checker uses, both probabilities are 0 and no event
// happens, whatever the rule for nonzero ones.
#ifndef SCREF_KMC_CHOOSE_STUB_HPP
#define SCREF_KMC_CHOOSE_STUB_HPP

inline int choose_kmc_double(double p0, double p1, double roll) {
  if (roll < p0) return 0;
  if (roll < p0 + p1) return 1;
  return -1;
}

#endif
