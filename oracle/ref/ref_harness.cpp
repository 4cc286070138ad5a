// ORACLE / TEST INFRASTRUCTURE ONLY -- built into oracle/_ref/libscref.so
// together with the reference's own, unmodified hot-path sources (object,
// site, bond, mesh, filament, cell, cell_list, minimum_distance,
// linear_algebra, rng, space, logger, cpu_time), compiled where they lie.
//
// The reference's InteractionManager, FilamentSpecies and Simulation sources
// cannot be compiled here (they pull in yaml-cpp, the unvendored KMC
// submodule and FFTW), so this file restates just the parts of them that the
// Brownian-dynamics step runs, with the reference's own classes doing all the
// arithmetic:
//   - Simulation::RunSimulation step body      src/simulation.cpp:37-62
//   - InteractionManager::InitInteractions     src/interaction_manager.cpp:37-56
//   - InteractionManager::Interact             src/interaction_manager.cpp:63-95
//   - CheckUpdateObjects / CheckUpdateInteractions / GetDrMax / ZeroDrTot
//                                              src/interaction_manager.cpp:262-321
//   - UpdateInteractions / UpdatePairInteractions
//                                              src/interaction_manager.cpp:211-231
//   - ProcessPairInteraction                   src/interaction_manager.cpp:323-397
//   - CalculatePairInteractions (OpenMP chunks, culling)
//                                              src/interaction_manager.cpp:448-498
//   - ApplyPairInteractions                    src/interaction_manager.cpp:500-517
//   - FilamentSpecies::UpdatePositions         src/filament_species.cpp:59-85
//   - Species::GetDrMax / ZeroDrTot / ZeroForces  include/simcore/species.hpp:105-127,198-203
//   - Simulation::InsertSpecies tail           src/simulation.cpp:399-404
//   - CrosslinkManager::UpdateCrosslinks -> CrosslinkSpecies::UpdatePositions
//     for doubly-bound crosslinks that neither unbind nor move
//                                              src/crosslink_manager.cpp:64-70,
//                                              src/crosslink_species.cpp:218-258
// The reference's own Crosslink and Anchor classes (src/crosslink.cpp,
// src/anchor.cpp, compiled with a stand-in for the absent KMC headers) place
// the crosslinks and compute and apply every tether force.
// Insertion itself is replaced by loading a given configuration into each
// filament (Mesh::GetSite(i)->SetPosition, then UpdateBondPositions and
// UpdatePrevPositions, src/mesh.cpp:24,324,175), after which every Philox
// stream is rewound so that dynamics starts at draw 0 in every code.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

// White-box access to the reference's private per-filament solver state
// (tensions_, ...) and to CellList's static configuration, in this
// translation unit only.  Layout is unaffected.
#define private public
#define protected public
#include "simcore/cell_list.hpp"
#include "simcore/crosslink.hpp"
#include "simcore/filament.hpp"
#include "simcore/minimum_distance.hpp"
#include "simcore/potential_manager.hpp"
#include "simcore/space.hpp"
#undef private
#undef protected

bool early_exit = false;  // defined by the reference in simulation_manager.cpp

extern "C" void scshim_set_global_seed(uint32_t seed);
extern "C" void scshim_rewind_all(void);
extern "C" void scshim_set_noise_layout(uint32_t key1, int n_sites, int n_dim);

extern "C" {
typedef struct {
  int n_dim;              // 2 or 3; every dimension periodic
  double system_radius;   // R, the cube (square) has side 2R
  double delta;
  double wca_eps;
  double wca_sig;
  double f_cutoff;
  int stoch_flag;
  int interaction_flag;
  int like_like_interactions;
  unsigned int seed;      // Philox key word 0 for every filament stream
  int n_threads;          // OpenMP threads, 0 = library default
} scref_system;

typedef struct {
  double length;
  double persistence_length;
  double diameter;
  double min_bond_length;
  double friction_ratio;
} scref_filament;
}

namespace {

struct RefSim {
  system_parameters params;
  Space space;
  space_struct *sp = nullptr;
  std::vector<filament_parameters> fparams;
  std::vector<Filament> members;
  bool midstep = true;  // FilamentSpecies::midstep_ (filament_species.hpp:9)

  CellList clist;
  PotentialManager potentials;
  MinimumDistance mindist;
  std::vector<Interaction> pair_interactions;
  std::vector<Object *> interactors;
  double dr_update = 0;
  int i_update = 0;
  int n_objs = -1;
  long n_rebuilds = 0;
  int i_step = 0;
  bool overlap = false;
  double stress[9] = {0};
  int n_thermo = 0;
  std::vector<double> thermo_rec;  // i_step, pressure tensor (9), pressure, volume
  std::unordered_map<const Object *, int> bond_gid;
  // FilamentSpecies analyses (scref_analysis_*): mse2e_, mse2e2_, n_samples_,
  // n_bins_, theta_histogram_ (src/filament_species.cpp:366-456)
  double mse2e = 0, mse2e2 = 0;
  long an_samples = 0;
  int n_bins = 0;
  std::vector<std::vector<int>> theta_histogram;
  // diffusion analysis (scref_diffusion_*): SpherocylinderSpecies' time-
  // origin averaged MSD and orientation correlation, on filament averages
  int dif_interval = 0, dif_time = 0;
  std::vector<double> pos0, u0, msd, msd_err, vcf, vcf_err;
  // doubly-bound crosslinks (scref_add_crosslinks)
  crosslink_parameters xparams;
  std::vector<Crosslink> xlinks;
  std::vector<int> site_fil, site_local;  // per global site: filament, index in it
  int n_threads = 0;
  int n_sites_total = 0;
  int n_bonds_total = 0;

  // ---- restated Species<Filament> helpers (species.hpp) -------------------
  double GetDrMax() {  // species.hpp:105-120 and interaction_manager.cpp:299-312
    double max_dr = 0;
    for (auto &f : members) {
      double dr = f.GetDrTot();
      if (dr > max_dr) max_dr = dr;
    }
    if (max_dr > 10000) throw std::runtime_error("Unphysical result");
    return max_dr;
  }
  void ZeroDrTot() {
    for (auto &f : members) f.ZeroDrTot();
  }
  void ZeroForces() {
    for (auto &f : members) f.ZeroForce();
  }
  int CountSpecies() {
    int c = 0;
    for (auto &f : members) c += f.GetCount();
    return c;
  }
  bool CheckSpeciesInteractorUpdate() {  // species.hpp:556-563
    bool result = false;
    for (auto &f : members)
      if (f.CheckInteractorUpdate()) result = true;
    return result;
  }

  // ---- restated InteractionManager pieces ---------------------------------
  void UpdateInteractors() {
    interactors.clear();
    for (auto &f : members) f.GetInteractors(interactors);
  }
  void UpdatePairInteractions() {
    if (!params.interaction_flag) return;
    pair_interactions.clear();
    clist.RenewObjectsCells(interactors);
    clist.MakePairs(pair_interactions);
  }
  void UpdateInteractions() {
    i_update = 0;
    n_rebuilds++;
    UpdatePairInteractions();
    ZeroDrTot();
  }
  void ForceUpdate() {
    UpdateInteractors();
    UpdateInteractions();
  }
  void CheckUpdateObjects() {
    if (params.static_particle_number) return;
    bool ix_update = CheckSpeciesInteractorUpdate();
    int obj_count = CountSpecies();
    if (obj_count != n_objs || ix_update) {
      n_objs = obj_count;
      ForceUpdate();
    }
  }
  void CheckUpdateInteractions() {
    double dr_max = GetDrMax();
    if (dr_max > dr_update) UpdateInteractions();
  }
  void ProcessPairInteraction(Interaction *ix) {
    Object *obj1 = ix->obj1;
    Object *obj2 = ix->obj2;
    if (obj1->GetOID() == obj2->GetOID()) {
      fprintf(stderr, "scref: self interaction\n");
      exit(1);
    }
    if (!params.like_like_interactions && obj1->GetSID() == obj2->GetSID()) {
      ix->no_interaction = true;
      return;
    }
    if (obj1->GetMeshID() > 0 && obj1->GetMeshID() == obj2->GetMeshID()) {
      if (obj1->HasNeighbor(obj2->GetOID())) {
        ix->no_interaction = true;
        return;
      }
    }
    mindist.ObjectObject(*ix);
    if (ix->dr_mag2 < 0.25 * SQR(obj1->GetDiameter() + obj2->GetDiameter()))
      overlap = true;
    if (ix->dr_mag2 > potentials.GetRCut2()) return;
    potentials.CalcPotential(*ix);
  }
  void CalculatePairInteractions() {
#ifdef _OPENMP
    int max_threads = omp_get_max_threads();
    typedef std::vector<Interaction>::iterator it_t;
    std::vector<std::pair<it_t, it_t>> chunks;
    chunks.reserve(max_threads);
    size_t chunk_size = pair_interactions.size() / max_threads;
    auto cur = pair_interactions.begin();
    for (int i = 0; i < max_threads - 1; ++i) {
      auto last = cur;
      std::advance(cur, chunk_size);
      chunks.push_back(std::make_pair(last, cur));
    }
    chunks.push_back(std::make_pair(cur, pair_interactions.end()));
#pragma omp parallel for
    for (int i = 0; i < max_threads; ++i) {
      for (auto ix = chunks[i].first; ix != chunks[i].second; ++ix) {
        ProcessPairInteraction(&*ix);
        cross_product(ix->contact1, ix->force, ix->t1, 3);
        cross_product(ix->contact2, ix->force, ix->t2, 3);
      }
    }
#else
    for (auto ix = pair_interactions.begin(); ix != pair_interactions.end();
         ++ix) {
      ProcessPairInteraction(&*ix);
      cross_product(ix->contact1, ix->force, ix->t1, 3);
      cross_product(ix->contact2, ix->force, ix->t2, 3);
    }
#endif
    if (i_update == 0) {
      pair_interactions.erase(
          std::remove_if(pair_interactions.begin(), pair_interactions.end(),
                         [](Interaction x) { return x.no_interaction; }),
          pair_interactions.end());
    }
  }
  void ApplyPairInteractions() {
    int n_dim = params.n_dim;
    for (auto ix = pair_interactions.begin(); ix != pair_interactions.end();
         ++ix) {
      Object *obj1 = ix->obj1;
      Object *obj2 = ix->obj2;
      obj1->AddForce(ix->force);
      obj2->SubForce(ix->force);
      obj1->AddTorque(ix->t1);
      obj2->SubTorque(ix->t2);
      obj1->AddPotential(ix->pote);
      obj2->AddPotential(ix->pote);
      for (int i = 0; i < n_dim; ++i)
        for (int j = 0; j < n_dim; ++j)
          stress[n_dim * i + j] += ix->stress[n_dim * i + j];
    }
  }
  // CrosslinkManager::UpdateCrosslinks (src/crosslink_manager.cpp:64-70) ->
  // CrosslinkSpecies::UpdatePositions (src/crosslink_species.cpp:218-238):
  // on even steps UpdateBoundCrosslinks (forces of every bound crosslink,
  // applied in member order, then anchor motion and binding, :241-258);
  // on odd steps the stored anchor forces are applied again.  The crosslinks
  // are doubly bound with zero unbinding rate, no diffusion and no free
  // crosslinks in solution, so binding changes nothing.
  void UpdateCrosslinks() {
    if (xlinks.empty()) return;
    if (i_step % 2 == 0) {
      for (auto &x : xlinks) x.UpdateCrosslinkForces();
      for (auto &x : xlinks) x.ApplyTetherForces();
      for (auto &x : xlinks) x.UpdateCrosslinkPositions();
    } else {
      for (auto &x : xlinks) x.ApplyTetherForces();
    }
  }
  void Interact() {
    if (!params.interaction_flag) return;  // no interactions, no boundaries
    CheckUpdateObjects();
    UpdateCrosslinks();
    CheckUpdateInteractions();
    CalculatePairInteractions();
    ApplyPairInteractions();
    i_update++;
  }
  // FilamentSpecies::UpdatePositions (filament_species.cpp:59-85)
  void UpdatePositions() {
#ifdef _OPENMP
    int max_threads = omp_get_max_threads();
    typedef std::vector<Filament>::iterator it_t;
    std::vector<std::pair<it_t, it_t>> chunks;
    chunks.reserve(max_threads);
    size_t chunk_size = members.size() / max_threads;
    auto cur = members.begin();
    for (int i = 0; i < max_threads - 1; ++i) {
      auto last = cur;
      std::advance(cur, chunk_size);
      chunks.push_back(std::make_pair(last, cur));
    }
    chunks.push_back(std::make_pair(cur, members.end()));
    bool ms = midstep;
#pragma omp parallel for
    for (int i = 0; i < max_threads; ++i)
      for (auto it = chunks[i].first; it != chunks[i].second; ++it)
        it->UpdatePosition(ms);
#else
    for (auto &f : members) f.UpdatePosition(midstep);
#endif
    midstep = !midstep;
  }
  // InteractionManager::CalculatePressure (src/interaction_manager.cpp:535-559)
  // into a record, with the Space's own volume and the interactor count the
  // restated CheckUpdateObjects keeps.
  void CalculatePressure() {
    int n_dim = params.n_dim;
    double pressure_tensor[9] = {0};
    double inv_V = 1.0 / sp->volume;
    for (int i = 0; i < n_dim; ++i) {
      for (int j = 0; j < n_dim; ++j) {
        if (i == j) pressure_tensor[n_dim * i + j] += n_objs * inv_V;
        pressure_tensor[n_dim * i + j] += stress[n_dim * i + j] * inv_V / n_thermo;
      }
    }
    double pressure = 0;
    for (int i = 0; i < n_dim; ++i) pressure += pressure_tensor[n_dim * i + i];
    pressure /= n_dim;
    std::fill(stress, stress + 9, 0);
    thermo_rec.push_back((double)i_step);
    for (int i = 0; i < 9; ++i) thermo_rec.push_back(pressure_tensor[i]);
    thermo_rec.push_back(pressure);
    thermo_rec.push_back(sp->volume);
  }
  void Step() {  // simulation.cpp:37-62 (outputs and graphics off)
    ++i_step;
    params.i_step = i_step;
    ZeroForces();
    Interact();
    UpdatePositions();
    // Simulation::Statistics (src/simulation.cpp:108-114)
    if (n_thermo > 0 && i_step % n_thermo == 0 && i_step > 0) CalculatePressure();
  }
};

RefSim *g_active = nullptr;  // the reference keeps static state: one at a time

}  // namespace

extern "C" {

void *scref_create(const scref_system *sys, int n_fil,
                   const scref_filament *fils, const double *site_xyz,
                   int n_sites_given) {
  if (g_active) return nullptr;
  if (!sys || n_fil <= 0 || !fils || !site_xyz) return nullptr;
  RefSim *s = new RefSim();
  s->n_threads = sys->n_threads;
#ifdef _OPENMP
  if (sys->n_threads > 0) omp_set_num_threads(sys->n_threads);
#endif
  system_parameters &p = s->params;
  p.n_dim = sys->n_dim;
  p.n_periodic = sys->n_dim;
  p.boundary = 0;
  p.system_radius = sys->system_radius;
  p.delta = sys->delta;
  p.wca_eps = sys->wca_eps;
  p.wca_sig = sys->wca_sig;
  p.f_cutoff = sys->f_cutoff;
  p.stoch_flag = sys->stoch_flag != 0;
  p.interaction_flag = sys->interaction_flag != 0;
  p.like_like_interactions = sys->like_like_interactions != 0;
  p.potential = "wca";
  p.n_steps = 1 << 30;

  // Simulation::InitSimulation: space, static object parameters.
  s->space.Init(&p);
  s->sp = s->space.GetStruct();
  Object::SetParams(&p);
  Object::SetSpace(s->sp);
  Object::SetNDim(p.n_dim);
  Object::SetDelta(p.delta);

  // Fresh static cell-list configuration for this run.
  CellList::_min_cell_length_ = -1;
  CellList::_n_dim_ = -1;
  CellList::_n_periodic_ = -1;

  // Species parameters, one struct per filament (per-filament persistence
  // lengths need their own filament_parameters).
  s->fparams.resize(n_fil);
  for (int i = 0; i < n_fil; ++i) {
    filament_parameters &fp = s->fparams[i];
    fp.num = n_fil;
    fp.length = fils[i].length;
    fp.persistence_length = fils[i].persistence_length;
    fp.diameter = fils[i].diameter;
    fp.min_bond_length = fils[i].min_bond_length;
    fp.friction_ratio = fils[i].friction_ratio;
    fp.insertion_type = "random";
  }
  // Simulation::InitSpecies: spec length = 1.5*min_bond_length vs diameter.
  {
    double spec_length = 1.5 * fils[0].min_bond_length;
    double spec_d = fils[0].diameter;
    spec_length = (spec_d > spec_length ? spec_d : spec_length);
    CellList::SetMinCellLength(spec_length);
  }
  // InteractionManager::InitInteractions (no crosslinks: rcutoff 0).
  CellList::SetMinCellLength(0.0);
  s->potentials.InitPotentials(&p);
  CellList::SetMinCellLength(sqrt(s->potentials.GetRCut2()));
  CellList::Init(p.n_dim, p.n_periodic, p.system_radius);
  // CellList::BuildCellList (src/cell_list.cpp:66-74) minus its redundant
  // full-shell neighbour pass, which only serves insertion's overlap checks
  // (not run here) and is replaced by the half-shell pass of
  // ResetNeighbors below anyway; the final cell structure is the same.
  s->clist.AllocateCells();
  s->clist.LabelCells();
  s->clist.ClearCellObjects();
  s->dr_update = 0.25 * CellList::GetCellLength() * CellList::GetCellLength();
  MinimumDistance::Init(s->sp, 2 * s->dr_update);

  // Members: filament i is seeded with i, so its Philox key is (seed, i).
  scshim_set_global_seed(sys->seed);
  s->members.reserve(n_fil);
  int site_cursor = 0;
  for (int i = 0; i < n_fil; ++i) {
    s->members.emplace_back((unsigned long)i);
    Filament &f = s->members.back();
    f.SetSID(species_id::filament);
    f.Init(&s->fparams[i]);
    int ns = f.n_sites_;
    if (site_cursor + ns > n_sites_given) {
      delete s;
      return nullptr;
    }
    for (int j = 0; j < ns; ++j) {
      double r[3] = {0, 0, 0};
      for (int d = 0; d < p.n_dim; ++d) r[d] = site_xyz[3 * (site_cursor + j) + d];
      f.GetSite(j)->SetPosition(r);
    }
    f.UpdateBondPositions();
    f.UpdatePrevPositions();
    f.CalculateAngles();
    site_cursor += ns;
  }
  if (site_cursor != n_sites_given) {
    delete s;
    return nullptr;
  }
  s->n_sites_total = site_cursor;
  for (int i = 0; i < n_fil; ++i)
    for (int j = 0; j < s->members[i].n_sites_; ++j) {
      s->site_fil.push_back(i);
      s->site_local.push_back(j);
    }

  // Simulation::InsertSpecies tail: half-shell neighbours, then a forced
  // update that bins every bond and zeroes the displacement trackers.
  s->clist.ResetNeighbors();
  s->pair_interactions.clear();
  s->interactors.clear();
  s->clist.ClearCellObjects();
  if (p.interaction_flag) s->CheckUpdateObjects();
  s->n_rebuilds = 0;  // count rebuilds triggered during dynamics only

  int gid = 0;
  for (auto &f : s->members)
    for (int b = 0; b < f.n_bonds_; ++b) s->bond_gid[f.GetBond(b)] = gid++;
  s->n_bonds_total = gid;

  // Filament i draws its noise from stream (seed, i); sites and bonds own
  // streams of their own keyed by other values.  Only the filament streams
  // are declared noise streams (key1 = i, n_sites of filament i).
  for (int i = 0; i < n_fil; ++i)
    scshim_set_noise_layout((uint32_t)i, s->members[i].n_sites_, p.n_dim);
  scshim_rewind_all();
  g_active = s;
  return s;
}

void scref_destroy(void *h) {
  RefSim *s = (RefSim *)h;
  if (!s) return;
  s->clist.Clear();
  delete s;
  if (g_active == s) g_active = nullptr;
}

int scref_n_sites(void *h) { return ((RefSim *)h)->n_sites_total; }
int scref_n_bonds(void *h) { return ((RefSim *)h)->n_bonds_total; }
int scref_n_cells_1d(void *) { return CellList::_n_cells_1d_; }
double scref_cell_length(void *) { return CellList::_cell_length_; }
double scref_dr_update(void *h) { return ((RefSim *)h)->dr_update; }
long scref_n_rebuilds(void *h) { return ((RefSim *)h)->n_rebuilds; }
int scref_i_step(void *h) { return ((RefSim *)h)->i_step; }

// Runs n reference steps (i_steps); returns the wall time of the loop in s,
// or -1 if the reference raised its "Unphysical result" error.
double scref_step(void *h, int n) {
  RefSim *s = (RefSim *)h;
  auto t0 = std::chrono::steady_clock::now();
  try {
    for (int i = 0; i < n; ++i) s->Step();
  } catch (const std::runtime_error &) {
    return -1.0;
  }
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

void scref_get_sites(void *h, double *xyz) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int j = 0; j < f.n_sites_; ++j, ++c) {
      const double *r = f.GetSite(j)->GetPosition();
      for (int d = 0; d < 3; ++d) xyz[3 * c + d] = r[d];
    }
}

void scref_get_prev_sites(void *h, double *xyz) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int j = 0; j < f.n_sites_; ++j, ++c) {
      const double *r = f.GetSite(j)->GetPrevPosition();
      for (int d = 0; d < 3; ++d) xyz[3 * c + d] = r[d];
    }
}

void scref_get_site_forces(void *h, double *fo) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int j = 0; j < f.n_sites_; ++j, ++c) {
      const double *v = f.GetSite(j)->GetForce();
      for (int d = 0; d < 3; ++d) fo[3 * c + d] = v[d];
    }
}

void scref_get_random_forces(void *h, double *fo) {
  RefSim *s = (RefSim *)h;
  int n_dim = s->params.n_dim;
  int c = 0;
  for (auto &f : s->members)
    for (int j = 0; j < f.n_sites_; ++j, ++c) {
      const double *v = f.GetSite(j)->GetRandomForce();
      for (int d = 0; d < 3; ++d) fo[3 * c + d] = d < n_dim ? v[d] : 0.0;
    }
}

void scref_get_bond_ft(void *h, double *fo, double *to) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int b = 0; b < f.n_bonds_; ++b, ++c) {
      const double *v = f.GetBond(b)->GetForce();
      const double *t = f.GetBond(b)->GetTorque();
      for (int d = 0; d < 3; ++d) {
        fo[3 * c + d] = v[d];
        to[3 * c + d] = t[d];
      }
    }
}

void scref_get_tensions(void *h, double *tens) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int b = 0; b < f.n_bonds_; ++b, ++c) tens[c] = f.tensions_[b];
}

void scref_get_bond_geom(void *h, double *pos, double *spos, double *u,
                         double *len) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int b = 0; b < f.n_bonds_; ++b, ++c) {
      Bond *bd = f.GetBond(b);
      for (int d = 0; d < 3; ++d) {
        pos[3 * c + d] = bd->GetPosition()[d];
        spos[3 * c + d] = bd->GetScaledPosition()[d];
        u[3 * c + d] = bd->GetOrientation()[d];
      }
      len[c] = bd->GetLength();
    }
}

void scref_get_filament_state(void *h, int *normalize_switch,
                              int *n_normalize) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members) {
    normalize_switch[c] = f.normalize_switch_ ? 1 : 0;
    n_normalize[c] = f.n_normalize_;
    ++c;
  }
}

void scref_get_frictions(void *h, double *gpar, double *gperp, double *spar,
                         double *sperp) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members) {
    gpar[c] = f.friction_par_;
    gperp[c] = f.friction_perp_;
    spar[c] = f.rand_sigma_par_;
    sperp[c] = f.rand_sigma_perp_;
    ++c;
  }
}

// Current pair list (after the culling that follows a rebuild) as pairs of
// global bond indices in list order.  Returns the number of pairs; writes at
// most cap of them.
long scref_get_pairs(void *h, int *out, long cap) {
  RefSim *s = (RefSim *)h;
  long n = (long)s->pair_interactions.size();
  for (long i = 0; i < n && i < cap; ++i) {
    out[2 * i] = s->bond_gid[s->pair_interactions[i].obj1];
    out[2 * i + 1] = s->bond_gid[s->pair_interactions[i].obj2];
  }
  return n;
}

// Cell coordinates (x, y, z) that CellList::FindCellCoords gives each bond
// from its current scaled position.
void scref_get_bond_cells(void *h, int *xyz) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int b = 0; b < f.n_bonds_; ++b, ++c) {
      int x, y, z;
      std::tie(x, y, z) = s->clist.FindCellCoords(*f.GetBond(b));
      xyz[3 * c] = x;
      xyz[3 * c + 1] = y;
      xyz[3 * c + 2] = z;
    }
}

// Thermo records every n_thermo steps from now on (0: none).
void scref_set_thermo(void *h, int n_thermo) {
  RefSim *s = (RefSim *)h;
  s->n_thermo = n_thermo;
  s->thermo_rec.clear();
}

// The records since the last call (at most max): i_step, pressure tensor
// (9), pressure and volume each.  Returns how many were written.
long scref_thermo_records(void *h, long max, long *i_step, double *tensor, double *pressure,
                          double *volume) {
  RefSim *s = (RefSim *)h;
  long n = (long)s->thermo_rec.size() / 12;
  if (n > max) n = max;
  for (long k = 0; k < n; ++k) {
    const double *q = s->thermo_rec.data() + 12 * k;
    i_step[k] = (long)q[0];
    for (int i = 0; i < 9; ++i) tensor[9 * k + i] = q[1 + i];
    pressure[k] = q[10];
    volume[k] = q[11];
  }
  s->thermo_rec.clear();
  return n;
}

// InteractionManager::stress_ as accumulated since the last pressure.
void scref_get_stress(void *h, double *out) {
  RefSim *s = (RefSim *)h;
  for (int i = 0; i < 9; ++i) out[i] = s->stress[i];
}

// Object::GetPotentialEnergy of every filament (its bonds' pair potentials,
// added by Filament::ApplyInteractionForces during the last step).
void scref_get_potential_energy(void *h, double *pote) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members) pote[c++] = f.GetPotentialEnergy();
}

// One spec frame of the filament species appended to the file at path: the
// member count, then each filament's own Filament::WriteSpec
// (Species::WriteSpecs, include/simcore/species.hpp:229-235, restated;
// src/filament.cpp:1314-1319, src/mesh.cpp:482-492).  Returns 0 on success.
int scref_write_spec_frame(void *h, const char *path) {
  RefSim *s = (RefSim *)h;
  std::fstream out(path, std::ios::out | std::ios::binary | std::ios::app);
  if (!out.is_open()) return -1;
  int size = (int)s->members.size();
  out.write(reinterpret_cast<char *>(&size), sizeof(int));
  for (auto &m : s->members) m.WriteSpec(out);
  return out.good() ? 0 : -1;
}

// One posit frame likewise: the member count and each filament's own
// Filament::WritePosit (Species::WritePosits, include/simcore/species.hpp:
// 221-227, restated; src/filament.cpp:1347-1361).
int scref_write_posit_frame(void *h, const char *path) {
  RefSim *s = (RefSim *)h;
  std::fstream out(path, std::ios::out | std::ios::binary | std::ios::app);
  if (!out.is_open()) return -1;
  int size = (int)s->members.size();
  out.write(reinterpret_cast<char *>(&size), sizeof(int));
  for (auto &m : s->members) m.WritePosit(out);
  return out.good() ? 0 : -1;
}

// The global order of FilamentSpecies::RunGlobalOrderAnalysis
// (src/filament_species.cpp:487-517, restated) on freshly zeroed
// accumulators, as its first sample: every filament's own
// Filament::GetPolarOrder / GetNematicOrder (src/filament.cpp:488-516) added,
// then both divided by the member count.
void scref_global_order(void *h, double *polar, double *nematic) {
  RefSim *s = (RefSim *)h;
  std::fill(polar, polar + 3, 0.0);
  std::fill(nematic, nematic + 9, 0.0);
  for (auto &m : s->members) {
    m.GetPolarOrder(polar);
    m.GetNematicOrder(nematic);
  }
  const int n_members = (int)s->members.size();
  for (int i = 0; i < 3; ++i) polar[i] /= n_members;
  for (int i = 0; i < 9; ++i) nematic[i] /= n_members;
}

// Per-site accumulated squared displacement since the last rebuild.
void scref_get_dr_tot(void *h, double *dr) {
  RefSim *s = (RefSim *)h;
  int c = 0;
  for (auto &f : s->members)
    for (int j = 0; j < f.n_sites_; ++j, ++c) dr[c] = f.GetSite(j)->dr_tot_;
}

// Doubly-bound crosslinks between global sites site_a[k] and site_b[k],
// made and attached by the reference's own code: Crosslink::Init with
// crosslink parameters of zero unbinding rates, no diffusion or walking,
// end pausing on, the given spring constants and rest length; each anchor
// AttachObjLambda'd to the bond whose tail is its site (lambda 0), or, for a
// filament's last site, to the last bond at its head (lambda = its length);
// then SetDoubly.  Once, before the first step.  Returns 0, or -1 on a bad
// site index or a repeated call.
int scref_add_crosslinks(void *h, int n, const int *site_a, const int *site_b, double k_spring,
                         double k_spring_compress, double rest_length) {
  RefSim *s = (RefSim *)h;
  if (!s || n < 0 || !s->xlinks.empty()) return -1;
  crosslink_parameters &xp = s->xparams;
  xp.num = n;
  xp.k_spring = k_spring;
  xp.k_spring_compress = k_spring_compress;
  xp.rest_length = rest_length;
  xp.static_flag = false;
  xp.k_on_s = xp.k_on_d = 0;
  xp.k_off_s = xp.k_off_d = 0;
  xp.diffusion_s = xp.diffusion_d = 0;
  xp.velocity_s = xp.velocity_d = 0;
  xp.end_pausing = true;
  xp.concentration = 0;
  const int ns = (int)s->site_fil.size();
  for (int q = 0; q < n; ++q)
    if (site_a[q] < 0 || site_a[q] >= ns || site_b[q] < 0 || site_b[q] >= ns) return -1;
  s->xlinks.reserve(n);
  for (int q = 0; q < n; ++q) {
    s->xlinks.emplace_back((unsigned long)(1000003u + (unsigned)q));
    Crosslink &x = s->xlinks.back();
    x.Init(&xp);
    const int sites[2] = {site_a[q], site_b[q]};
    for (int a = 0; a < 2; ++a) {
      Filament &f = s->members[s->site_fil[sites[a]]];
      const int j = s->site_local[sites[a]];
      Bond *b = j < f.n_bonds_ ? f.GetBond(j) : f.GetBond(f.n_bonds_ - 1);
      const double lambda = j < f.n_bonds_ ? 0.0 : b->GetLength();
      x.anchors_[a].AttachObjLambda(b, lambda);
    }
    x.SetDoubly();
  }
  return 0;
}

// FilamentSpecies::RunMse2eAnalysis and RunThetaAnalysis (src/filament_species.
// cpp:569-610) over the members, as the reference runs them after a step:
// head-to-tail distance from the current sites, joint cosines from
// Filament::GetThetas (the cosines CalculateAngles took at the start of the
// last step's integration).  The histogram is sized at the first sample as
// InitThetaAnalysis sizes it (:417-456), with n_bins bins.
void scref_analysis_sample(void *h, int n_bins) {
  RefSim *s = (RefSim *)h;
  const int nd = s->params.n_dim;
  if (s->theta_histogram.empty()) {
    s->n_bins = n_bins;
    const int nbonds = s->members.back().GetNBonds();
    s->theta_histogram.assign(nbonds - 1, std::vector<int>(n_bins, 0));
  }
  for (auto it = s->members.begin(); it != s->members.end(); ++it) {
    double const *const head_pos = it->GetHeadPosition();
    double const *const tail_pos = it->GetTailPosition();
    double mse2e_temp = 0.0;
    for (int i = 0; i < nd; ++i) {
      double temp = (head_pos[i] - tail_pos[i]);
      mse2e_temp += temp * temp;
    }
    s->mse2e += mse2e_temp;
    s->mse2e2 += mse2e_temp * mse2e_temp;
  }
  s->an_samples++;
  for (auto it = s->members.begin(); it != s->members.end(); ++it) {
    std::vector<double> const *const thetas = it->GetThetas();
    for (int i = 0; i < (it->GetNBonds() - 1); ++i) {
      int bin_number = (int)floor((1 + (*thetas)[i]) * (s->n_bins / 2));
      if (bin_number == s->n_bins) bin_number = s->n_bins - 1;
      else if (bin_number == -1) bin_number = 0;
      s->theta_histogram[i][bin_number]++;
    }
  }
}

// FilamentSpecies::FinalizeMse2eAnalysis (src/filament_species.cpp:686-698)
// on copies of the sums, and the histogram (joints x bins).
void scref_analysis_results(void *h, double *mean, double *err, long *n_samples, int *n_joints,
                            long *hist) {
  RefSim *s = (RefSim *)h;
  const int num = (int)s->members.size();
  double m = s->mse2e, m2 = s->mse2e2;
  m /= s->an_samples * num;
  m2 /= s->an_samples * num;
  if (mean) *mean = m;
  if (err) *err = sqrt((m2 - m * m) / (num * s->an_samples));
  if (n_samples) *n_samples = s->an_samples;
  if (n_joints) *n_joints = (int)s->theta_histogram.size();
  if (hist)
    for (size_t j = 0; j < s->theta_histogram.size(); ++j)
      for (int b = 0; b < s->n_bins; ++b) hist[j * s->n_bins + b] = s->theta_histogram[j][b];
}

// The reference's diffusion analysis (SpherocylinderSpecies::
// InitDiffusionAnalysis, DiffusionAnalysis, UpdateInitPositions, CalculateMSD,
// CalculateVCF, FinalizeDiffusionAnalysis; src/spherocylinder_species.cpp:
// 30-134) applied to the filaments' average positions and orientations
// (Filament::UpdateAvgPosition, src/filament.cpp:953-968, which every
// UpdatePosition runs): a time-origin average over windows of `interval`
// samples, each window's points weighted by the inverse variance over the
// members.
void scref_diffusion_init(void *h, int interval) {
  RefSim *s = (RefSim *)h;
  const int n = (int)s->members.size(), nd = s->params.n_dim;
  s->dif_interval = interval;
  s->dif_time = 0;
  s->pos0.assign((size_t)n * nd, 0.0);
  s->u0.assign((size_t)n * nd, 0.0);
  s->msd.assign(interval, 0.0);
  s->msd_err.assign(interval, 0.0);
  s->vcf.assign(interval, 0.0);
  s->vcf_err.assign(interval, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < nd; ++j) {
      s->pos0[(size_t)i * nd + j] = s->members[i].GetPosition()[j];
      s->u0[(size_t)i * nd + j] = s->members[i].GetOrientation()[j];
    }
}

void scref_diffusion_sample(void *h) {
  RefSim *s = (RefSim *)h;
  const int n = (int)s->members.size(), nd = s->params.n_dim;
  {  // CalculateMSD
    double avg_sqr_dist = 0.0, avg_sqr_dist_sqr = 0.0;
    for (int i = 0; i < n; ++i) {
      double sqr_diff = 0;
      double const *const position = s->members[i].GetPosition();
      for (int j = 0; j < nd; ++j) {
        double r_diff = position[j] - s->pos0[(size_t)i * nd + j];
        sqr_diff += SQR(r_diff);
      }
      avg_sqr_dist += sqr_diff;
      avg_sqr_dist_sqr += SQR(sqr_diff);
    }
    avg_sqr_dist /= n;
    avg_sqr_dist_sqr /= n;
    double stdev2 = avg_sqr_dist_sqr - SQR(avg_sqr_dist);
    s->msd[s->dif_time] += avg_sqr_dist / stdev2;
    s->msd_err[s->dif_time] += 1.0 / stdev2;
  }
  {  // CalculateVCF
    double avg_udotu0 = 0.0, avg_udotu0_sqr = 0.0;
    for (int i = 0; i < n; ++i) {
      double udotu0 = 0.0;
      double const *const orientation = s->members[i].GetOrientation();
      for (int j = 0; j < nd; ++j) udotu0 += orientation[j] * s->u0[(size_t)i * nd + j];
      avg_udotu0 += udotu0;
      avg_udotu0_sqr += udotu0 * udotu0;
    }
    avg_udotu0 /= n;
    avg_udotu0_sqr /= n;
    double stdev2 = avg_udotu0_sqr - SQR(avg_udotu0);
    s->vcf[s->dif_time] += avg_udotu0 / stdev2;
    s->vcf_err[s->dif_time] += 1.0 / stdev2;
  }
  if (++s->dif_time == s->dif_interval) {  // UpdateInitPositions
    s->dif_time = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < nd; ++j) {
        s->pos0[(size_t)i * nd + j] = s->members[i].GetPosition()[j];
        s->u0[(size_t)i * nd + j] = s->members[i].GetOrientation()[j];
      }
  }
}

// FinalizeDiffusionAnalysis' quotients (on copies): msd, its error, vcf and
// its error per window point.
void scref_diffusion_results(void *h, double *msd, double *msd_err, double *vcf,
                             double *vcf_err) {
  RefSim *s = (RefSim *)h;
  const int n = (int)s->members.size();
  for (int t = 0; t < s->dif_interval; ++t) {
    msd[t] = s->msd[t] / s->msd_err[t];
    vcf[t] = s->vcf[t] / s->vcf_err[t];
    msd_err[t] = 1.0 / sqrt(n * s->msd_err[t]);
    vcf_err[t] = 1.0 / sqrt(n * s->vcf_err[t]);
  }
}

// Crosslink::force_ of every crosslink (the tether force on anchor 0).
void scref_get_crosslink_forces(void *h, double *out) {
  RefSim *s = (RefSim *)h;
  for (size_t q = 0; q < s->xlinks.size(); ++q)
    for (int d = 0; d < 3; ++d) out[3 * q + d] = s->xlinks[q].force_[d];
}

}  // extern "C"
