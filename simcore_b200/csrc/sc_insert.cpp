// Random filament insertion with overlap rejection, on the host.
//
// Produces initial configurations with the distributions of simcore's
// random insertion: Mesh::InitRandomBond (reference src/mesh.cpp:244-258:
// isotropic first bond, centre uniform in (-(R-d), R-d)^n_dim, tail at
// centre - L/2 u), Filament::InsertFilament and GenerateProbableOrientation
// (src/filament.cpp:225-249, 350-383: each further bond drawn from
// P(theta) ~ exp((lp/l) cos theta) relative to the previous one, with the
// large-stiffness approximation above lp = 100), and overlap rejection of
// InteractionManager::CheckOverlap (src/interaction_manager.cpp:561-571,
// 390: reject a filament if any of its bonds comes closer than the mean
// diameter to an already accepted bond).  Randomness is Philox4x32-10 keyed
// by (seed, 0xC0FFEE), so a configuration is a pure function of its seed.
// Both the GPU path and the CPU reference load the same configuration.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "sc_host_philox.h"
#include "simcore_gpu.h"

namespace {

struct Stream {
  uint32_t k0, k1;
  uint64_t k = 0;
  double uniform() { return sc_host_philox_uniform(k0, k1, k++); }
};

double dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Rotate v so that its local z axis maps onto unit vector w
// (the reference's rotate_vector_relative, src/linear_algebra.cpp:222-251).
void rotate_relative(int n_dim, double *v, const double *w) {
  double vx = v[0], vy = v[1], vz = v[2];
  double phi = std::atan2(w[1], w[0]);
  if (n_dim == 3) {
    double theta = std::acos(w[2] > 1 ? 1 : (w[2] < -1 ? -1 : w[2]));
    v[0] = vx * std::cos(theta) * std::cos(phi) - vy * std::sin(phi) +
           vz * std::cos(phi) * std::sin(theta);
    v[1] = vx * std::cos(theta) * std::sin(phi) + vy * std::cos(phi) +
           vz * std::sin(theta) * std::sin(phi);
    v[2] = vz * std::cos(theta) - vx * std::sin(theta);
  } else {
    v[0] = vx * std::cos(phi) - vy * std::sin(phi);
    v[1] = vx * std::sin(phi) + vy * std::cos(phi);
    v[2] = 0;
  }
}

// Minimum squared distance between two segments (centres c, unit axes u,
// half lengths h) in a periodic box of side L (every dimension periodic).
double seg_dist2(int n_dim, const double *c1, const double *u1, double h1,
                 const double *c2, const double *u2, double h2, double L) {
  double dr[3] = {0, 0, 0};
  for (int i = 0; i < n_dim; ++i) {
    double d = c2[i] - c1[i];
    d -= L * std::nearbyint(d / L);
    dr[i] = d;
  }
  double a = dot3(dr, u1), b = dot3(dr, u2), c = dot3(u1, u2);
  double den = 1.0 - c * c, lam, mu;
  if (den < 1e-12) {
    lam = 0.5 * a;
    mu = -0.5 * b;
  } else {
    lam = (a - c * b) / den;
    mu = (-b + c * a) / den;
  }
  auto clamp = [](double x, double h) { return x > h ? h : (x < -h ? -h : x); };
  // Clamp one parameter, re-project the other, clamp again (both orders).
  double best = 1e300;
  for (int pass = 0; pass < 3; ++pass) {
    double l2, m2;
    if (pass == 0) {
      l2 = clamp(lam, h1);
      m2 = clamp(-b + l2 * c, h2);
      l2 = clamp(a + m2 * c, h1);
    } else if (pass == 1) {
      m2 = clamp(mu, h2);
      l2 = clamp(a + m2 * c, h1);
      m2 = clamp(-b + l2 * c, h2);
    } else {
      l2 = clamp(lam, h1);
      m2 = clamp(mu, h2);
    }
    double r2 = 0;
    for (int i = 0; i < 3; ++i) {
      double d = dr[i] - l2 * u1[i] + m2 * u2[i];
      r2 += d * d;
    }
    if (r2 < best) best = r2;
  }
  return best;
}

struct Grid {
  int n1d, n_dim;
  double L, cell;
  std::vector<std::vector<int>> cells;
  Grid(int n_dim_, double L_, double min_cell) : n_dim(n_dim_), L(L_) {
    n1d = (int)std::floor(L / min_cell);
    if (n1d < 3) n1d = 3;
    if (n1d > (n_dim == 3 ? 400 : 8000)) n1d = (n_dim == 3 ? 400 : 8000);
    cell = L / n1d;
    size_t nc = (size_t)n1d * n1d * (n_dim == 3 ? n1d : 1);
    cells.resize(nc);
  }
  int coord(double x) const {
    double s = x / L + 0.5;
    s -= std::floor(s);
    int c = (int)(s * n1d);
    return c >= n1d ? n1d - 1 : c;
  }
  size_t index(int x, int y, int z) const {
    return ((size_t)x * n1d + y) * (n_dim == 3 ? n1d : 1) + z;
  }
};

}  // namespace

// One insertion attempt of a filament of nb bonds (length `length`,
// persistence length lp) drawn from the stream (k0, k1) at position k:
// site positions (3 (nb + 1)), bond centres and unit axes (3 nb each).
// Returns the stream position after the attempt's draws; the number of draws
// depends only on the insertion type, n_dim and nb.
uint64_t sc_insert_candidate(int n_dim, double system_radius, double diameter,
                             int insertion_type, int nb, double length, double lp,
                             uint32_t k0, uint32_t k1, uint64_t k, double *pos, double *cen,
                             double *axis) {
  Stream rng{k0, k1, k};
  const double l = length / nb;
  std::memset(pos, 0, sizeof(double) * 3 * (nb + 1));
  std::memset(cen, 0, sizeof(double) * 3 * nb);
  std::memset(axis, 0, sizeof(double) * 3 * nb);
  double u[3] = {0, 0, 0}, p[3] = {0, 0, 0};
  if (insertion_type == SC_INSERT_RANDOM) {
    // RNG::RandomUnitVector (src/rng.cpp:34-49)
    double w = 1.0;
    if (n_dim == 3) {
      double z = 2.0 * rng.uniform() - 1.0;
      w = std::sqrt(1 - z * z);
      u[2] = z;
    }
    double t = 2.0 * M_PI * rng.uniform();
    u[0] = w * std::cos(t);
    u[1] = w * std::sin(t);
  } else {
    // Filament::InsertFirstBond, random_nematic / random_polar
    // (src/filament.cpp:195-202): along +-z (+-y in 2D), straight.
    u[n_dim - 1] = insertion_type == SC_INSERT_RANDOM_POLAR
                       ? 1.0
                       : (rng.uniform() > 0.5 ? 1.0 : -1.0);
  }
  // RNG::RandomCoordinate, box/none (src/rng.cpp:50-66)
  for (int i = 0; i < n_dim; ++i) p[i] = (2.0 * rng.uniform() - 1.0) * (system_radius - diameter);
  for (int i = 0; i < n_dim; ++i) p[i] -= 0.5 * u[i] * length;
  for (int i = 0; i < 3; ++i) pos[i] = p[i];
  for (int b = 0; b < nb; ++b) {
    if (b > 0 && insertion_type == SC_INSERT_RANDOM) {
      // Filament::GenerateProbableOrientation
      double kk = lp / l, theta;
      if (lp == 0) {
        theta = rng.uniform() * M_PI;
      } else if (lp < 100) {
        theta = std::acos(std::log(std::exp(-kk) + 2.0 * rng.uniform() * std::sinh(kk)) / kk);
      } else {
        theta = std::acos((std::log(2.0 * rng.uniform()) - std::log(2.0) + kk) / kk);
      }
      double nu[3] = {0, 0, 0};
      if (n_dim == 2) {
        theta = (rng.uniform() < 0.5 ? -1 : 1) * theta;
        nu[0] = std::cos(theta);
        nu[1] = std::sin(theta);
      } else {
        double phi = rng.uniform() * 2.0 * M_PI;
        nu[0] = std::sin(theta) * std::cos(phi);
        nu[1] = std::sin(theta) * std::sin(phi);
        nu[2] = std::cos(theta);
      }
      rotate_relative(n_dim, nu, u);
      double m = std::sqrt(dot3(nu, nu));
      for (int i = 0; i < 3; ++i) u[i] = nu[i] / m;
    }
    for (int i = 0; i < n_dim; ++i) pos[3 * (b + 1) + i] = pos[3 * b + i] + l * u[i];
    for (int i = 0; i < n_dim; ++i) {
      cen[3 * b + i] = pos[3 * b + i] + 0.5 * l * u[i];
      axis[3 * b + i] = u[i];
    }
  }
  return rng.k;
}

extern "C" int sc_insert_filaments(int n_dim, double system_radius,
                                   uint64_t seed, int n_fil,
                                   const int *n_bonds, const double *length,
                                   const double *persistence_length,
                                   double diameter, int insertion_type,
                                   int max_attempts, double *site_xyz) {
  if ((n_dim != 2 && n_dim != 3) || n_fil <= 0 || !n_bonds || !length ||
      !persistence_length || !site_xyz || system_radius <= diameter ||
      insertion_type < SC_INSERT_RANDOM || insertion_type > SC_INSERT_RANDOM_POLAR)
    return SC_ERR_INVALID_ARG;
  const double L = 2.0 * system_radius;
  double max_bond = 0;
  for (int f = 0; f < n_fil; ++f) {
    if (n_bonds[f] < 2) return SC_ERR_INVALID_ARG;
    max_bond = std::fmax(max_bond, length[f] / n_bonds[f]);
  }
  // Two bonds can touch only if their centres are within max_bond + d.
  Grid grid(n_dim, L, max_bond + diameter);
  std::vector<double> bc, bu;  // accepted bond centres and axes
  std::vector<double> bh;      // half lengths
  Stream rng{(uint32_t)seed ^ (uint32_t)(seed >> 32), 0xC0FFEEu, 0};
  // Longest filaments first (a stable order, so equal lengths keep theirs):
  // they find room while the box is empty; each filament's sites still go
  // to its own place in site_xyz.
  std::vector<size_t> site_at(n_fil + 1, 0);
  for (int f = 0; f < n_fil; ++f) site_at[f + 1] = site_at[f] + n_bonds[f] + 1;
  std::vector<int> order(n_fil);
  for (int f = 0; f < n_fil; ++f) order[f] = f;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return length[a] > length[b]; });
  std::vector<double> pos, cen, axis;
  for (int oi = 0; oi < n_fil; ++oi) {
    const int f = order[oi];
    const size_t site_cursor = site_at[f];
    const int nb = n_bonds[f];
    const double l = length[f] / nb, lp = persistence_length[f];
    bool placed = false;
    for (int attempt = 0; attempt < max_attempts && !placed; ++attempt) {
      pos.resize(3 * (nb + 1));
      cen.resize(3 * nb);
      axis.resize(3 * nb);
      rng.k = sc_insert_candidate(n_dim, system_radius, diameter, insertion_type, nb, length[f],
                                  persistence_length[f], rng.k0, rng.k1, rng.k, pos.data(),
                                  cen.data(), axis.data());
      // Overlap test against accepted bonds.
      bool overlap = false;
      for (int b = 0; b < nb && !overlap; ++b) {
        const double *c = &cen[3 * b];
        int cx = grid.coord(c[0]), cy = grid.coord(c[1]),
            cz = n_dim == 3 ? grid.coord(c[2]) : 0;
        int zr = n_dim == 3 ? 1 : 0;
        for (int dx = -1; dx <= 1 && !overlap; ++dx)
          for (int dy = -1; dy <= 1 && !overlap; ++dy)
            for (int dz = -zr; dz <= zr && !overlap; ++dz) {
              int x = (cx + dx + grid.n1d) % grid.n1d;
              int y = (cy + dy + grid.n1d) % grid.n1d;
              int z = n_dim == 3 ? (cz + dz + grid.n1d) % grid.n1d : 0;
              for (int o : grid.cells[grid.index(x, y, z)]) {
                double d2 = seg_dist2(n_dim, c, &axis[3 * b], 0.5 * l, &bc[3 * o],
                                      &bu[3 * o], bh[o], L);
                if (d2 < diameter * diameter) {
                  overlap = true;
                  break;
                }
              }
            }
      }
      if (overlap) continue;
      for (int b = 0; b < nb; ++b) {
        int id = (int)bh.size();
        for (int i = 0; i < 3; ++i) {
          bc.push_back(cen[3 * b + i]);
          bu.push_back(axis[3 * b + i]);
        }
        bh.push_back(0.5 * l);
        const double *c = &cen[3 * b];
        grid.cells[grid.index(grid.coord(c[0]), grid.coord(c[1]),
                              n_dim == 3 ? grid.coord(c[2]) : 0)]
            .push_back(id);
      }
      std::memcpy(site_xyz + 3 * site_cursor, pos.data(),
                  sizeof(double) * 3 * (nb + 1));
      placed = true;
    }
    if (!placed) return SC_ERR_INSERTION;
  }
  return SC_OK;
}
