// Drives the C++ host classes of include/simcore_host.hpp (Simulation,
// InteractionManager, FilamentSpecies) the way the reference's step loop
// does, for tests/test_host_classes.py.
//
//   host_classes_run <input> <output> <n_host_steps> <n_graph_steps>
//
// input: int32 n_dim, n_fil, n_sites, precision; float64 system_radius,
// delta, seed; per filament float64 length, persistence_length, diameter,
// min_bond_length, friction_ratio; float64 sites (n_sites x 3).
// output: float64 sites after the steps (n_sites x 3), then the bond forces
// and torques of the last Interact (n_bonds x 3 each), then int64 rebuild
// count.  Exit status 0, or 1 with the error on stderr.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "simcore_host.hpp"

using simcore_b200::Simulation;

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s input output n_host_steps n_graph_steps\n", argv[0]);
    return 2;
  }
  try {
    std::FILE *in = std::fopen(argv[1], "rb");
    if (!in) throw std::runtime_error("cannot open input");
    int hdr[4];
    double sysv[3];
    if (std::fread(hdr, sizeof(int), 4, in) != 4 || std::fread(sysv, sizeof(double), 3, in) != 3)
      throw std::runtime_error("short input");
    simcore_b200::SystemParameters p;
    p.n_dim = hdr[0];
    p.precision = hdr[3] ? SC_PREC_MIXED : SC_PREC_FP64;
    p.system_radius = sysv[0];
    p.delta = sysv[1];
    p.seed = (uint32_t)sysv[2];
    std::vector<sc_filament_params> fils(hdr[1]);
    for (auto &f : fils) {
      double v[5];
      if (std::fread(v, sizeof(double), 5, in) != 5) throw std::runtime_error("short input");
      f.length = v[0];
      f.persistence_length = v[1];
      f.diameter = v[2];
      f.min_bond_length = v[3];
      f.friction_ratio = v[4];
    }
    std::vector<double> sites(3 * (size_t)hdr[2]);
    if (std::fread(sites.data(), sizeof(double), sites.size(), in) != sites.size())
      throw std::runtime_error("short input");
    std::fclose(in);

    Simulation sim;
    sim.InitSimulation(p, fils, sites);
    long interacts = 0;
    sim.RunSimulation(std::atoi(argv[3]), [&](Simulation &) { ++interacts; });
    sim.RunSimulation(std::atoi(argv[4]));
    sim.Interact();  // the forces of the next step's Interact
    std::vector<double> xyz = sim.GetFilamentSpecies().GetSitePositions(), f, t;
    sim.GetInteractionManager().GetBondForces(f, t);
    const int64_t rebuilds = sim.GetInteractionManager().GetNRebuilds();
    std::FILE *out = std::fopen(argv[2], "wb");
    if (!out) throw std::runtime_error("cannot open output");
    std::fwrite(xyz.data(), sizeof(double), xyz.size(), out);
    std::fwrite(f.data(), sizeof(double), f.size(), out);
    std::fwrite(t.data(), sizeof(double), t.size(), out);
    std::fwrite(&rebuilds, sizeof(int64_t), 1, out);
    std::fclose(out);
    if (interacts != std::atoi(argv[3])) throw std::runtime_error("step hook count");
  } catch (const std::exception &e) {
    std::fprintf(stderr, "host_classes_run: %s\n", e.what());
    return 1;
  }
  return 0;
}
