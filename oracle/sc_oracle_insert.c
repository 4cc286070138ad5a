/* ORACLE / TEST INFRASTRUCTURE ONLY -- see sc_oracle.h.
 *
 * Random filament insertion with overlap rejection, restated in plain C from
 * the reference:
 *   - first bond: RNG::RandomUnitVector (src/rng.cpp:34-49) for random
 *     insertion, or along +-z (+-y in 2D) for random_nematic / random_polar
 *     (Filament::InsertFirstBond, src/filament.cpp:192-222);
 *   - centre: RNG::RandomCoordinate of a periodic box, uniform in
 *     (-(R - d), R - d) per dimension (src/rng.cpp:50-66), tail at
 *     centre - L/2 u (Mesh::InitRandomBond, src/mesh.cpp:244-258);
 *   - further bonds: Filament::GenerateProbableOrientation
 *     (src/filament.cpp:350-383) relative to the previous bond, rotated by
 *     rotate_vector_relative (src/linear_algebra.cpp:222-251);
 *   - rejection: InteractionManager::CheckOverlap (src/interaction_manager.cpp:
 *     561-571, 390): a filament is redrawn while any of its bonds comes
 *     closer than the diameter to an accepted bond.
 * The reference draws from GSL; like the thermal noise, insertion draws here
 * come from the shared Philox4x32-10 stream: key (seed low ^ seed high,
 * 0xC0FFEE), k-th uniform = word (k & 3) of philox(counter (k >> 2, k >> 34,
 * 0, 0)), mapped to (word + 0.5) 2^-32.  Filaments are placed longest first
 * (a stable order), each at its own place in the output.  The same stream and
 * order drive the library's insertion, so both give one configuration for one
 * seed; tests/test_oracle.py checks that they agree bit for bit. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sc_oracle.h"
#include "sc_philox.h"

#define INS_PI 3.14159265358979323846 /* M_PI */

typedef struct {
  uint32_t k0, k1;
  uint64_t k;
} ins_stream;

static double ins_uniform(ins_stream *s) {
  const uint64_t k = s->k++;
  const uint32_t ctr[4] = {(uint32_t)(k >> 2), (uint32_t)(k >> 34), 0u, 0u};
  const uint32_t key[2] = {s->k0, s->k1};
  uint32_t w[4];
  sc_philox4x32_10(ctr, key, w);
  return ((double)w[k & 3u] + 0.5) * 2.3283064365386963e-10;
}

static double ins_dot3(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* rotate_vector_relative (src/linear_algebra.cpp:222-251): v's local z axis
 * onto the unit vector w. */
static void ins_rotate(int n_dim, double *v, const double *w) {
  const double vx = v[0], vy = v[1], vz = v[2];
  const double phi = atan2(w[1], w[0]);
  if (n_dim == 3) {
    const double theta = acos(w[2] > 1 ? 1 : (w[2] < -1 ? -1 : w[2]));
    v[0] = vx * cos(theta) * cos(phi) - vy * sin(phi) + vz * cos(phi) * sin(theta);
    v[1] = vx * cos(theta) * sin(phi) + vy * cos(phi) + vz * sin(theta) * sin(phi);
    v[2] = vz * cos(theta) - vx * sin(theta);
  } else {
    v[0] = vx * cos(phi) - vy * sin(phi);
    v[1] = vx * sin(phi) + vy * cos(phi);
    v[2] = 0;
  }
}

static double ins_clamp(double x, double h) { return x > h ? h : (x < -h ? -h : x); }

/* Squared minimum distance of two segments (centres c, unit axes u, half
 * lengths h) under the periodic minimum image of a box of side L: the
 * unconstrained closest points (MinimumDistance::Sphero's parallel case at
 * 1 - c^2 < 1e-12), then the end clamps tried both ways. */
static double ins_seg_dist2(int n_dim, const double *c1, const double *u1, double h1,
                            const double *c2, const double *u2, double h2, double L) {
  double dr[3] = {0, 0, 0};
  int i, pass;
  for (i = 0; i < n_dim; ++i) {
    double d = c2[i] - c1[i];
    d -= L * nearbyint(d / L);
    dr[i] = d;
  }
  const double a = ins_dot3(dr, u1), b = ins_dot3(dr, u2), c = ins_dot3(u1, u2);
  const double den = 1.0 - c * c;
  double lam, mu, best = 1e300;
  if (den < 1e-12) {
    lam = 0.5 * a;
    mu = -0.5 * b;
  } else {
    lam = (a - c * b) / den;
    mu = (-b + c * a) / den;
  }
  for (pass = 0; pass < 3; ++pass) {
    double l2, m2, r2 = 0;
    if (pass == 0) {
      l2 = ins_clamp(lam, h1);
      m2 = ins_clamp(-b + l2 * c, h2);
      l2 = ins_clamp(a + m2 * c, h1);
    } else if (pass == 1) {
      m2 = ins_clamp(mu, h2);
      l2 = ins_clamp(a + m2 * c, h1);
      m2 = ins_clamp(-b + l2 * c, h2);
    } else {
      l2 = ins_clamp(lam, h1);
      m2 = ins_clamp(mu, h2);
    }
    for (i = 0; i < 3; ++i) {
      const double d = dr[i] - l2 * u1[i] + m2 * u2[i];
      r2 += d * d;
    }
    if (r2 < best) best = r2;
  }
  return best;
}

/* Accepted bonds in a periodic grid of cells of at least max bond + d, each
 * cell a linked list. */
typedef struct {
  int n_dim, n1d;
  double L;
  int *head;             /* per cell: last bond added, -1 */
  int *next;             /* per bond */
  double *c, *u, *h;     /* per bond: centre (3), axis (3), half length */
  int n, cap;
} ins_grid;

static int ins_coord(const ins_grid *g, double x) {
  double s = x / g->L + 0.5;
  int c;
  s -= floor(s);
  c = (int)(s * g->n1d);
  return c >= g->n1d ? g->n1d - 1 : c;
}

static size_t ins_cell(const ins_grid *g, int x, int y, int z) {
  return ((size_t)x * g->n1d + y) * (g->n_dim == 3 ? g->n1d : 1) + z;
}

static const double *ins_len_key;
static int ins_longer_first(const void *pa, const void *pb) {
  const int a = *(const int *)pa, b = *(const int *)pb;
  if (ins_len_key[a] > ins_len_key[b]) return -1;
  if (ins_len_key[a] < ins_len_key[b]) return 1;
  return a < b ? -1 : (a > b ? 1 : 0); /* equal lengths keep their order */
}

int sco_insert_filaments(int n_dim, double system_radius, uint64_t seed, int n_fil,
                         const int *n_bonds, const double *length,
                         const double *persistence_length, double diameter,
                         int insertion_type, int max_attempts, double *site_xyz) {
  const double L = 2.0 * system_radius;
  double max_bond = 0;
  int f, oi, rc = 0;
  size_t nc, total_bonds = 0;
  ins_grid g;
  ins_stream rng;
  int *order;
  size_t *site_at;
  double *pos = NULL, *cen = NULL, *axis = NULL;
  if ((n_dim != 2 && n_dim != 3) || n_fil <= 0 || !n_bonds || !length ||
      !persistence_length || !site_xyz || system_radius <= diameter || insertion_type < 0 ||
      insertion_type > 2)
    return 1; /* invalid argument */
  for (f = 0; f < n_fil; ++f) {
    if (n_bonds[f] < 2) return 1;
    max_bond = fmax(max_bond, length[f] / n_bonds[f]);
    total_bonds += (size_t)n_bonds[f];
  }
  memset(&g, 0, sizeof(g));
  g.n_dim = n_dim;
  g.L = L;
  g.n1d = (int)floor(L / (max_bond + diameter));
  if (g.n1d < 3) g.n1d = 3;
  if (g.n1d > (n_dim == 3 ? 400 : 8000)) g.n1d = n_dim == 3 ? 400 : 8000;
  nc = (size_t)g.n1d * g.n1d * (n_dim == 3 ? g.n1d : 1);
  g.head = (int *)malloc(sizeof(int) * nc);
  g.next = (int *)malloc(sizeof(int) * total_bonds);
  g.c = (double *)malloc(sizeof(double) * 3 * total_bonds);
  g.u = (double *)malloc(sizeof(double) * 3 * total_bonds);
  g.h = (double *)malloc(sizeof(double) * total_bonds);
  order = (int *)malloc(sizeof(int) * n_fil);
  site_at = (size_t *)malloc(sizeof(size_t) * (n_fil + 1));
  memset(g.head, 0xff, sizeof(int) * nc);
  rng.k0 = (uint32_t)seed ^ (uint32_t)(seed >> 32);
  rng.k1 = 0xC0FFEEu;
  rng.k = 0;
  site_at[0] = 0;
  for (f = 0; f < n_fil; ++f) {
    site_at[f + 1] = site_at[f] + n_bonds[f] + 1;
    order[f] = f;
  }
  ins_len_key = length;
  qsort(order, n_fil, sizeof(int), ins_longer_first);
  for (oi = 0; oi < n_fil && rc == 0; ++oi) {
    const int fi = order[oi], nb = n_bonds[fi];
    const double l = length[fi] / nb, lp = persistence_length[fi];
    int attempt, placed = 0, b, i;
    pos = (double *)realloc(pos, sizeof(double) * 3 * (nb + 1));
    cen = (double *)realloc(cen, sizeof(double) * 3 * nb);
    axis = (double *)realloc(axis, sizeof(double) * 3 * nb);
    for (attempt = 0; attempt < max_attempts && !placed; ++attempt) {
      double u[3] = {0, 0, 0}, p[3] = {0, 0, 0};
      int overlap = 0;
      memset(pos, 0, sizeof(double) * 3 * (nb + 1));
      memset(cen, 0, sizeof(double) * 3 * nb);
      memset(axis, 0, sizeof(double) * 3 * nb);
      if (insertion_type == 0) {
        double w = 1.0, t;
        if (n_dim == 3) {
          const double z = 2.0 * ins_uniform(&rng) - 1.0;
          w = sqrt(1 - z * z);
          u[2] = z;
        }
        t = 2.0 * INS_PI * ins_uniform(&rng);
        u[0] = w * cos(t);
        u[1] = w * sin(t);
      } else {
        u[n_dim - 1] = insertion_type == 2 ? 1.0 : (ins_uniform(&rng) > 0.5 ? 1.0 : -1.0);
      }
      for (i = 0; i < n_dim; ++i) p[i] = (2.0 * ins_uniform(&rng) - 1.0) * (system_radius - diameter);
      for (i = 0; i < n_dim; ++i) p[i] -= 0.5 * u[i] * length[fi];
      for (i = 0; i < 3; ++i) pos[i] = p[i];
      for (b = 0; b < nb; ++b) {
        if (b > 0 && insertion_type == 0) {
          const double k = lp / l;
          double theta, nu[3] = {0, 0, 0}, m;
          if (lp == 0) {
            theta = ins_uniform(&rng) * INS_PI;
          } else if (lp < 100) {
            theta = acos(log(exp(-k) + 2.0 * ins_uniform(&rng) * sinh(k)) / k);
          } else {
            theta = acos((log(2.0 * ins_uniform(&rng)) - log(2.0) + k) / k);
          }
          if (n_dim == 2) {
            theta = (ins_uniform(&rng) < 0.5 ? -1 : 1) * theta;
            nu[0] = cos(theta);
            nu[1] = sin(theta);
          } else {
            const double phi = ins_uniform(&rng) * 2.0 * INS_PI;
            nu[0] = sin(theta) * cos(phi);
            nu[1] = sin(theta) * sin(phi);
            nu[2] = cos(theta);
          }
          ins_rotate(n_dim, nu, u);
          m = sqrt(ins_dot3(nu, nu));
          for (i = 0; i < 3; ++i) u[i] = nu[i] / m;
        }
        for (i = 0; i < n_dim; ++i) pos[3 * (b + 1) + i] = pos[3 * b + i] + l * u[i];
        for (i = 0; i < n_dim; ++i) {
          cen[3 * b + i] = pos[3 * b + i] + 0.5 * l * u[i];
          axis[3 * b + i] = u[i];
        }
      }
      for (b = 0; b < nb && !overlap; ++b) {
        const double *c = &cen[3 * b];
        const int cx = ins_coord(&g, c[0]), cy = ins_coord(&g, c[1]);
        const int cz = n_dim == 3 ? ins_coord(&g, c[2]) : 0, zr = n_dim == 3 ? 1 : 0;
        int dx, dy, dz;
        for (dx = -1; dx <= 1 && !overlap; ++dx)
          for (dy = -1; dy <= 1 && !overlap; ++dy)
            for (dz = -zr; dz <= zr && !overlap; ++dz) {
              const int x = (cx + dx + g.n1d) % g.n1d, y = (cy + dy + g.n1d) % g.n1d;
              const int z = n_dim == 3 ? (cz + dz + g.n1d) % g.n1d : 0;
              int o;
              for (o = g.head[ins_cell(&g, x, y, z)]; o >= 0 && !overlap; o = g.next[o])
                if (ins_seg_dist2(n_dim, c, &axis[3 * b], 0.5 * l, &g.c[3 * o], &g.u[3 * o],
                                  g.h[o], L) < diameter * diameter)
                  overlap = 1;
            }
      }
      if (overlap) continue;
      for (b = 0; b < nb; ++b) {
        const int id = g.n++;
        const double *c = &cen[3 * b];
        size_t cell;
        for (i = 0; i < 3; ++i) {
          g.c[3 * id + i] = cen[3 * b + i];
          g.u[3 * id + i] = axis[3 * b + i];
        }
        g.h[id] = 0.5 * l;
        cell = ins_cell(&g, ins_coord(&g, c[0]), ins_coord(&g, c[1]),
                        n_dim == 3 ? ins_coord(&g, c[2]) : 0);
        g.next[id] = g.head[cell];
        g.head[cell] = id;
      }
      memcpy(site_xyz + 3 * site_at[fi], pos, sizeof(double) * 3 * (nb + 1));
      placed = 1;
    }
    if (!placed) rc = 8; /* the attempt budget ran out */
  }
  free(pos);
  free(cen);
  free(axis);
  free(order);
  free(site_at);
  free(g.head);
  free(g.next);
  free(g.c);
  free(g.u);
  free(g.h);
  return rc;
}
