// simcore_host.hpp -- C++ host classes over the C ABI of simcore_gpu.h.
//
// The reference drives its filament step through three classes
// (src/simulation.cpp:37-62, :84-95):
//   Simulation::RunSimulation -- per step ZeroForces, Interact, Integrate,
//                                Statistics, WriteOutputs;
//   InteractionManager::Interact -- the pair path
//                                (include/simcore/interaction_manager.hpp:72);
//   FilamentSpecies::UpdatePositions -- the integrator
//                                (include/simcore/species_base.hpp:29).
// These classes keep those names and roles, and each hot method is one call
// into libsimcore_b200 (every array lives on the GPU).  A Simulation owns one
// context (sc_ctx); its InteractionManager and FilamentSpecies are views of
// it.  Errors of the C ABI (sc_status) are thrown as simcore_b200::Error,
// carrying the context's message; nothing here exits, as the reference's
// Logger::Error does.
//
// Header only; link with libsimcore_b200.so.
#ifndef SIMCORE_HOST_HPP
#define SIMCORE_HOST_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "simcore_gpu.h"

namespace simcore_b200 {

class Error : public std::runtime_error {
 public:
  Error(sc_status code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
  sc_status code() const { return code_; }

 private:
  sc_status code_;
};

inline void check(sc_status s, const sc_ctx *ctx, const char *what) {
  if (s != SC_OK)
    throw Error(s, std::string(what) + ": " + (ctx ? sc_last_error(ctx) : "no context"));
}

// System parameters the step reads (the reference's system_parameters that
// matter on this path).
struct SystemParameters {
  int n_dim = 3;
  double system_radius = 100;
  double delta = 1e-4;
  double wca_eps = 1, wca_sig = 1, f_cutoff = 2000;
  bool stoch_flag = true, interaction_flag = true, like_like_interactions = true;
  uint32_t seed = 0;
  sc_precision precision = SC_PREC_FP64;
  int device = 0;
};

// InteractionManager: the pair path of one Simulation's context.
class InteractionManager {
 public:
  explicit InteractionManager(sc_ctx *ctx = nullptr) : ctx_(ctx) {}
  // InteractionManager::Interact: rebuild check, pair forces and torques
  // into the bond accumulators (src/interaction_manager.cpp:63-95).
  void Interact() { check(sc_interact(ctx_), ctx_, "Interact"); }
  // Bond::force_ / torque_ after the last Interact, 3 per bond.
  void GetBondForces(std::vector<double> &force, std::vector<double> &torque) const {
    sc_counters c = counters();
    force.resize(3 * (size_t)c.n_bonds);
    torque.resize(3 * (size_t)c.n_bonds);
    check(sc_get_bond_forces(ctx_, force.data(), torque.data()), ctx_, "GetBondForces");
  }
  // The candidate pair list (global bond ids), in the reference's order.
  std::vector<int32_t> GetPairs() const {
    int64_t n = 0;
    check(sc_get_pairs(ctx_, nullptr, 0, &n), ctx_, "GetPairs");
    std::vector<int32_t> p(2 * (size_t)n);
    check(sc_get_pairs(ctx_, p.data(), n, &n), ctx_, "GetPairs");
    return p;
  }
  int64_t GetNRebuilds() const { return counters().n_rebuilds; }

 private:
  sc_counters counters() const {
    sc_counters c;
    check(sc_get_counters(ctx_, &c), ctx_, "counters");
    return c;
  }
  sc_ctx *ctx_;
};

// FilamentSpecies: every filament of one Simulation's context.
class FilamentSpecies {
 public:
  explicit FilamentSpecies(sc_ctx *ctx = nullptr) : ctx_(ctx) {}
  // FilamentSpecies::UpdatePositions: one integrator (half) step of every
  // filament, toggling the midstep (src/filament_species.cpp:59-85).
  void UpdatePositions() { check(sc_update_positions(ctx_), ctx_, "UpdatePositions"); }
  int64_t GetNMembers() const { return counters().n_filaments; }
  int64_t GetNSites() const { return counters().n_sites; }
  int64_t GetNBonds() const { return counters().n_bonds; }
  // Site positions, 3 per site, filaments back to back.
  std::vector<double> GetSitePositions() const {
    std::vector<double> xyz(3 * (size_t)GetNSites());
    check(sc_get_sites(ctx_, xyz.data()), ctx_, "GetSitePositions");
    return xyz;
  }
  void SetSitePositions(const std::vector<double> &xyz) {
    check(sc_set_sites(ctx_, xyz.data()), ctx_, "SetSitePositions");
  }

 private:
  sc_counters counters() const {
    sc_counters c;
    check(sc_get_counters(ctx_, &c), ctx_, "counters");
    return c;
  }
  sc_ctx *ctx_;
};

// Simulation: one system (or a batch of independent ones) on one GPU.
class Simulation {
 public:
  Simulation() = default;
  Simulation(const Simulation &) = delete;
  Simulation &operator=(const Simulation &) = delete;
  ~Simulation() {
    if (ctx_) sc_destroy(ctx_);
  }

  // Simulation::InitSimulation with the filaments in place
  // (src/simulation.cpp:139-173): space, interaction engine, species, and the
  // forced pair-list update that ends the insertion.
  void InitSimulation(const SystemParameters &p, const std::vector<sc_filament_params> &filaments,
                      const std::vector<double> &site_xyz) {
    sc_system_desc d = {};
    d.n_dim = p.n_dim;
    d.system_radius = p.system_radius;
    d.delta = p.delta;
    d.wca_eps = p.wca_eps;
    d.wca_sig = p.wca_sig;
    d.f_cutoff = p.f_cutoff;
    d.stoch_flag = p.stoch_flag ? 1 : 0;
    d.interaction_flag = p.interaction_flag ? 1 : 0;
    d.like_like_interactions = p.like_like_interactions ? 1 : 0;
    d.seed = p.seed;
    d.precision = p.precision;
    d.device = p.device;
    if (ctx_) sc_destroy(ctx_);
    ctx_ = nullptr;
    check(sc_create(&d, &ctx_), nullptr, "InitSimulation");
    check(sc_add_filaments(ctx_, (int)filaments.size(), filaments.data(), site_xyz.data(),
                           (int64_t)(site_xyz.size() / 3)),
          ctx_, "InitSimulation");
    ix_mgr_ = InteractionManager(ctx_);
    species_ = FilamentSpecies(ctx_);
    i_step_ = 0;
  }

  // The step loop of Simulation::RunSimulation (src/simulation.cpp:37-62)
  // for n steps: ZeroForces (folded into Interact on the GPU), Interact,
  // Integrate.  With per_step_hook null the steps run back to back as one
  // captured graph per call (sc_step_graph); otherwise host-driven, the hook
  // called after every step (where the reference runs Statistics and
  // WriteOutputs).
  template <class Hook>
  void RunSimulation(int n_steps, Hook per_step_hook) {
    for (int i = 0; i < n_steps; ++i) {
      ++i_step_;
      Interact();
      Integrate();
      per_step_hook(*this);
    }
  }
  void RunSimulation(int n_steps) {
    check(sc_step_graph(ctx_, n_steps), ctx_, "RunSimulation");
    i_step_ += n_steps;
  }

  // Simulation::Interact and Simulation::Integrate (src/simulation.cpp:84-95).
  void Interact() { ix_mgr_.Interact(); }
  void Integrate() { species_.UpdatePositions(); }

  InteractionManager &GetInteractionManager() { return ix_mgr_; }
  FilamentSpecies &GetFilamentSpecies() { return species_; }
  long GetIStep() const { return i_step_; }
  double GetTime(double delta) const { return i_step_ * 0.5 * delta; }
  sc_ctx *context() { return ctx_; }

 private:
  sc_ctx *ctx_ = nullptr;
  InteractionManager ix_mgr_;
  FilamentSpecies species_;
  long i_step_ = 0;
};

}  // namespace simcore_b200

#endif
