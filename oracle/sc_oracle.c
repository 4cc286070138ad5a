/* ORACLE / TEST INFRASTRUCTURE ONLY -- see sc_oracle.h.
 *
 * Plain-C restatement of the reference's Brownian-dynamics step.  Every
 * floating-point expression keeps the reference's operand order and
 * association so that, compiled without FMA contraction, the results are
 * bit-identical to the reference's own code.  Citations are to the
 * reference sources (src/..., include/simcore/...). */
#include "sc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "sc_philox.h"

/* include/simcore/macros.hpp */
#define SQR(x) ((x) * (x))
#define NINT(x) ((x) < 0.0 ? (int)((x)-0.5) : (int)((x) + 0.5))
#define ABS(x) ((x) < 0 ? -(x) : (x))
#define SIGN(a, b) ((b) >= 0.0 ? fabs(a) : -fabs(a))
#define SIGNOF(x) ((x) >= 0.0 ? 1 : -1)
#define SMALL 1.0e-12 /* src/minimum_distance.cpp:3 */

struct sco_sim {
  int n_dim;
  double R;
  double h[9], hinv[9];
  double delta;
  double eps, sig, fcut, rcut2, c12, c6;
  int stoch, interaction, like_like;
  uint32_t seed;
  /* cell list */
  int n1d;
  double cl, dr_update;
  int n_cells;
  int *nbr;      /* n_cells * 13 neighbour cell indices (half shell) */
  int *n_nbr;    /* per cell */
  int *cell_start, *cell_count, *cell_items; /* bonds per cell, insertion order */
  /* filaments */
  int nf, ns, nb, max_ns;
  int *fs_off, *fb_off;
  double *fl, *flp, *fd, *gpar, *gperp, *spar, *sperp, *fdrmesh;
  int *fswitch, *fnnorm, *fmid;
  uint64_t *fdraw; /* noisy midsteps taken, per filament */
  /* sites */
  double *r, *rp, *fr, *F, *tn, *u, *dz, *dt;
  /* bonds */
  double *bp, *bs, *bu, *bl, *bF, *bT, *tens;
  /* pairs: obj1, obj2 (global bond ids), persistent force, scratch */
  long np, pcap;
  int *pa, *pb;
  double *pf;
  /* per pair, beside the force: the dr its stress used and its potential
   * (Interaction::dr / stress / pote, kept like the force until re-evaluated) */
  double *pdr, *ppote;
  /* thermo: InteractionManager::stress_ and the pressure records
   * (src/interaction_manager.cpp:500-517, 535-559) */
  double stress[9];
  double *bpote; /* per bond: Object::p_energy_ after ApplyPairInteractions */
  int n_thermo;
  long n_rec, rec_cap;
  double *rec; /* per record: i_step, pressure tensor (9), pressure, volume */
  /* mesh lambdas (Bond::mesh_lambda_, Mesh::true_length_): the summed
   * current lengths of the bonds before each bond, and of a filament's
   * bonds; the nominal length of each filament (Mesh::length_) */
  double *bml, *ftl, *fL;
  /* doubly-bound crosslinks: anchor 2k+a of link k is bound at mesh lambda
   * xM[2k+a] of filament xfil[2k+a] and sits on bond xbond[2k+a] (set again
   * from xM at every recomputation) */
  int nx;
  int *xbond, *xfil, xerr;
  double *xM;
  double xk, xkc, xrest;
  double *xc; /* 6 per anchor: the anchor's force_ and torque_ */
  double *xF; /* 3 per link: Crosslink::force_ */
  /* control */
  int i_update;
  long n_rebuilds;
  int i_step;
  int species_midstep;
  /* scratch for one filament */
  double *w_cos, *w_gl, *w_gd, *w_gu, *w_dt, *w_db, *w_ginv, *w_keff, *w_hd,
      *w_hu, *w_hl, *w_gam;
};

/* ---- src/linear_algebra.cpp --------------------------------------------- */

static double dot_product(int n, const double *a, const double *b) { /* :3-9 */
  double mag = 0.0;
  int i;
  for (i = 0; i < n; ++i) mag += a[i] * b[i];
  return mag;
}

static void cross3(const double *a, const double *b, double *c) { /* :13-24 */
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

static void normalize_vector(double *a, int n) { /* :26-35 */
  double mag = 0.0;
  int i;
  for (i = 0; i < n; ++i) mag += a[i] * a[i];
  mag = sqrt(mag);
  for (i = 0; i < n; ++i) a[i] /= mag;
}

static void invert_sym_2d(const double *a, double *b) { /* :40-47 */
  double inv_det = a[0] * a[3] - a[1] * a[1];
  inv_det = 1.0 / inv_det;
  b[0] = a[3] * inv_det;
  b[3] = a[0] * inv_det;
  b[2] = b[1] = -a[1] * inv_det;
}

static void invert_sym_3d(const double *a, double *b) { /* :52-64 */
  double inv_det = a[0] * (a[4] * a[8] - a[5] * a[7]) -
                   a[1] * (a[3] * a[8] - a[5] * a[6]) +
                   a[2] * (a[3] * a[7] - a[4] * a[6]);
  inv_det = 1.0 / inv_det;
  b[0] = inv_det * (a[4] * a[8] - a[5] * a[7]);
  b[4] = inv_det * (a[0] * a[8] - a[2] * a[6]);
  b[8] = inv_det * (a[0] * a[4] - a[1] * a[3]);
  b[1] = b[3] = -inv_det * (a[3] * a[8] - a[5] * a[6]);
  b[2] = b[6] = inv_det * (a[3] * a[7] - a[4] * a[6]);
  b[5] = b[7] = -inv_det * (a[0] * a[7] - a[1] * a[6]);
}

/* periodic_boundary_conditions :100-117 (n_periodic == n_dim) */
static void periodic_bc(int n, const double *hinv, const double *r, double *s) {
  int i, j;
  for (i = 0; i < n; ++i) {
    s[i] = 0.0;
    for (j = 0; j < n; ++j) s[i] += hinv[n * i + j] * r[j];
    s[i] -= NINT(s[i]);
  }
}

/* tridiagonal_solver :164-197 (Thomas, no pivoting, in place) */
static void thomas(double *a, double *b, double *c, double *d, int n) {
  int i;
  (void)b;
  n--;
  c[0] /= b[0];
  d[0] /= b[0];
  for (i = 1; i < n; ++i) {
    c[i] /= b[i] - a[i - 1] * c[i - 1];
    d[i] = (d[i] - a[i - 1] * d[i - 1]) / (b[i] - a[i - 1] * c[i - 1]);
  }
  d[n] = (d[n] - a[n - 1] * d[n - 1]) / (b[n] - a[n - 1] * c[n - 1]);
  for (i = n; i-- > 0;) d[i] -= c[i] * d[i + 1];
}

/* ---- geometry of bonds and sites ------------------------------------------ */

#define V3(p, i) ((p) + 3 * (size_t)(i))

/* Bond::ReInit (src/bond.cpp:22-37) + Object::UpdatePeriodic (src/object.cpp:202-210) */
static void bond_reinit(sco_sim *s, int b, int site1) {
  const double *r1 = V3(s->r, site1), *r2 = V3(s->r, site1 + 1);
  double *o = V3(s->bu, b), *pos = V3(s->bp, b), *sp = V3(s->bs, b);
  double len = 0;
  int i, n = s->n_dim;
  for (i = 0; i < n; ++i) {
    o[i] = r2[i] - r1[i];
    len += o[i] * o[i];
  }
  len = sqrt(len);
  for (i = 0; i < n; ++i) {
    pos[i] = r1[i] + 0.5 * o[i];
    o[i] /= len;
  }
  s->bl[b] = len;
  periodic_bc(n, s->hinv, pos, sp);
}

/* Mesh::UpdateBondPositions + UpdateSiteOrientations (src/mesh.cpp:168-173, 324-334) */
static void update_bond_positions(sco_sim *s, int f) {
  int s0 = s->fs_off[f], b0 = s->fb_off[f];
  int nbf = s->fb_off[f + 1] - b0, i, d;
  double true_length = 0;
  for (i = 0; i < nbf; ++i) {
    bond_reinit(s, b0 + i, s0 + i);
    s->bml[b0 + i] = true_length;  /* Bond::SetMeshLambda (src/mesh.cpp:324-330) */
    true_length += s->bl[b0 + i];
  }
  s->ftl[f] = true_length;
  for (i = 0; i < nbf; ++i)
    for (d = 0; d < s->n_dim; ++d) V3(s->u, s0 + i)[d] = V3(s->bu, b0 + i)[d];
  for (d = 0; d < s->n_dim; ++d)
    V3(s->u, s0 + nbf)[d] = V3(s->bu, b0 + nbf - 1)[d];
}

/* Site::CalcTangent (src/site.cpp:88-102): end sites copy their single bond's
 * orientation, interior sites normalise the sum of the incoming and outgoing
 * bond orientations. */
static void calc_tangents(sco_sim *s, int f) {
  int s0 = s->fs_off[f], b0 = s->fb_off[f];
  int n = s->fs_off[f + 1] - s0, j, i;
  for (j = 0; j < n; ++j) {
    double *t = V3(s->tn, s0 + j);
    if (j == 0 || j == n - 1) {
      const double *uu = V3(s->bu, b0 + (j == 0 ? 0 : n - 2));
      t[0] = uu[0];
      t[1] = uu[1];
      t[2] = uu[2];
    } else {
      const double *u1 = V3(s->bu, b0 + j - 1), *u2 = V3(s->bu, b0 + j);
      for (i = 0; i < s->n_dim; ++i) t[i] = u1[i] + u2[i];
      normalize_vector(t, s->n_dim);
    }
  }
}

/* ---- minimum distance and potentials -------------------------------------- */

/* MinimumDistance::Sphero (src/minimum_distance.cpp:202-344) */
static void sphero(const sco_sim *s, const double *s_1, const double *u_1,
                   double length_1, const double *s_2, const double *u_2,
                   double length_2, double *r_min, double *r_min_mag2,
                   double *contact_1, double *contact_2) {
  int n = s->n_dim, i, j;
  double dr[3], ds[3];
  double half_length_1 = 0.5 * length_1;
  double half_length_2 = 0.5 * length_2;
  double dr_dot_u_1, dr_dot_u_2, u_1_dot_u_2, lambda, mu, denom, lambda_mag,
      mu_mag;
  for (i = 0; i < n; ++i) {
    ds[i] = s_2[i] - s_1[i];
    ds[i] -= NINT(ds[i]);
  }
  for (i = 0; i < n; ++i) {
    dr[i] = 0.0;
    for (j = 0; j < n; ++j) dr[i] += s->h[n * i + j] * ds[j];
  }
  dr_dot_u_1 = dr_dot_u_2 = u_1_dot_u_2 = 0.0;
  for (i = 0; i < n; ++i) {
    dr_dot_u_1 += dr[i] * u_1[i];
    dr_dot_u_2 += dr[i] * u_2[i];
    u_1_dot_u_2 += u_1[i] * u_2[i];
  }
  denom = 1.0 - SQR(u_1_dot_u_2);
  if (denom < SMALL) {
    lambda = dr_dot_u_1 / 2.0;
    mu = -dr_dot_u_2 / 2.0;
  } else {
    lambda = (dr_dot_u_1 - u_1_dot_u_2 * dr_dot_u_2) / denom;
    mu = (-dr_dot_u_2 + u_1_dot_u_2 * dr_dot_u_1) / denom;
  }
  lambda_mag = ABS(lambda);
  mu_mag = ABS(mu);
  if (lambda_mag > half_length_1 && mu_mag > half_length_2) {
    double lambda_a, lambda_b, mu_a, mu_b, r_min_mag2_a, r_min_mag2_b;
    double r_min_a[3], r_min_b[3];
    lambda_a = SIGN(half_length_1, lambda);
    mu_a = -dr_dot_u_2 + lambda_a * u_1_dot_u_2;
    mu_mag = ABS(mu_a);
    if (mu_mag > half_length_2) mu_a = SIGN(half_length_2, mu_a);
    r_min_mag2_a = 0.0;
    for (i = 0; i < n; ++i) {
      r_min_a[i] = dr[i] - lambda_a * u_1[i] + mu_a * u_2[i];
      r_min_mag2_a += SQR(r_min_a[i]);
    }
    mu_b = SIGN(half_length_2, mu);
    lambda_b = dr_dot_u_1 + mu_b * u_1_dot_u_2;
    lambda_mag = ABS(lambda_b);
    if (lambda_mag > half_length_1) lambda_b = SIGN(half_length_1, lambda_b);
    r_min_mag2_b = 0.0;
    for (i = 0; i < n; ++i) {
      r_min_b[i] = dr[i] - lambda_b * u_1[i] + mu_b * u_2[i];
      r_min_mag2_b += SQR(r_min_b[i]);
    }
    if (r_min_mag2_a < r_min_mag2_b) {
      lambda = lambda_a;
      mu = mu_a;
      *r_min_mag2 = r_min_mag2_a;
      for (i = 0; i < n; ++i) r_min[i] = r_min_a[i];
    } else {
      lambda = lambda_b;
      mu = mu_b;
      *r_min_mag2 = r_min_mag2_b;
      for (i = 0; i < n; ++i) r_min[i] = r_min_b[i];
    }
  } else if (lambda_mag > half_length_1) {
    lambda = SIGN(half_length_1, lambda);
    mu = -dr_dot_u_2 + lambda * u_1_dot_u_2;
    mu_mag = ABS(mu);
    if (mu_mag > half_length_2) mu = SIGN(half_length_2, mu);
    *r_min_mag2 = 0.0;
    for (i = 0; i < n; ++i) {
      r_min[i] = dr[i] - lambda * u_1[i] + mu * u_2[i];
      *r_min_mag2 += SQR(r_min[i]);
    }
  } else if (mu_mag > half_length_2) {
    mu = SIGN(half_length_2, mu);
    lambda = dr_dot_u_1 + mu * u_1_dot_u_2;
    lambda_mag = ABS(lambda);
    if (lambda_mag > half_length_1) lambda = SIGN(half_length_1, lambda);
    *r_min_mag2 = 0.0;
    for (i = 0; i < n; ++i) {
      r_min[i] = dr[i] - lambda * u_1[i] + mu * u_2[i];
      *r_min_mag2 += SQR(r_min[i]);
    }
  } else {
    *r_min_mag2 = 0.0;
    for (i = 0; i < n; ++i) {
      r_min[i] = dr[i] - lambda * u_1[i] + mu * u_2[i];
      *r_min_mag2 += SQR(r_min[i]);
    }
  }
  for (i = 0; i < n; ++i) {
    contact_1[i] = lambda * u_1[i];
    contact_2[i] = mu * u_2[i];
  }
}

/* Force on obj1 of one candidate pair, following
 * InteractionManager::ProcessPairInteraction (src/interaction_manager.cpp:375-396),
 * MinimumDistance::ObjectObject (src/minimum_distance.cpp:20-66),
 * PotentialManager::CalcPotential (include/simcore/potential_manager.hpp:41-52),
 * WCAPotential::CalcPotential (include/simcore/wca_potential.hpp:14-32) and
 * MaxForcePotential::CalcPotential (include/simcore/max_force_potential.hpp:11-40).
 * force[] holds the pair's force from its last in-range evaluation since the
 * list was built (the reference never clears it) and is overwritten only when
 * a potential is evaluated, and so are the dr its stress was computed from
 * (rdr; the contact difference in the max-force case) and its potential
 * (rpote; 0 in the max-force case).  t1 = contact1 x force,
 * t2 = contact2 x force (src/interaction_manager.cpp:469-470). */
static void pair_force(const sco_sim *s, int b1, int b2, double *force,
                       double *t1, double *t2, double *rdr, double *rpote) {
  double dr[3] = {0, 0, 0}, c1[3] = {0, 0, 0}, c2[3] = {0, 0, 0}, dr_mag2 = 0;
  int n = s->n_dim, i;
  sphero(s, V3(s->bs, b1), V3(s->bu, b1), s->bl[b1], V3(s->bs, b2),
         V3(s->bu, b2), s->bl[b2], dr, &dr_mag2, c1, c2);
  if (!(dr_mag2 > s->rcut2)) {
    if (dr_mag2 < 1e-12) {
      double rmag = 0.0, rinv;
      if (c1[0] || c1[1] || c1[2])
        for (i = 0; i < n; ++i) dr[i] = c1[i] - c2[i];
      for (i = 0; i < n; ++i) rmag += dr[i] * dr[i];
      rmag = sqrt(rmag);
      if (!(rmag < 1e-12)) {
        rinv = 1.0 / (rmag);
        for (i = 0; i < n; ++i) force[i] = s->fcut * dr[i] * rinv;
        for (i = 0; i < n; ++i) rdr[i] = dr[i];
        *rpote = 0;
      }
    } else {
      double rmag = sqrt(dr_mag2);
      double rinv = 1.0 / (rmag);
      double rinv2 = rinv * rinv;
      double r6 = rinv2 * rinv2 * rinv2;
      double ffac = -(12.0 * s->c12 * r6 - 6.0 * s->c6) * r6 * rinv;
      if (ABS(ffac) > s->fcut) ffac = SIGNOF(ffac) * s->fcut;
      for (i = 0; i < n; ++i) force[i] = ffac * dr[i] * rinv;
      for (i = 0; i < n; ++i) rdr[i] = dr[i];
      *rpote = r6 * (s->c12 * r6 - s->c6) + s->eps;
    }
  }
  cross3(c1, force, t1);
  cross3(c2, force, t2);
}

/* ---- cell list (src/cell_list.cpp, src/cell.cpp) --------------------------- */

static int cell_index(const sco_sim *s, int x, int y, int z) {
  int third = (s->n_dim == 3 ? s->n1d : 1);
  return (x * s->n1d + y) * third + z;
}

/* CellList::AssignCellNeighbors(false) (src/cell_list.cpp:206-262) */
static void build_neighbors(sco_sim *s) {
  int n1d = s->n1d, third = (s->n_dim == 3 ? n1d : 1);
  int x, y, z, zp, yp, xp;
  for (z = 0; z < third; ++z)
    for (y = 0; y < n1d; ++y)
      for (x = 0; x < n1d; ++x) {
        int c = cell_index(s, x, y, z), cnt = 0;
        int z_begin = z, z_end = (s->n_dim == 3 ? z + 2 : z + 1);
        for (zp = z_begin; zp < z_end; ++zp) {
          int nz = zp;
          if ((nz < 0 || nz == n1d) && s->n_dim >= 3)
            nz = (nz < 0 ? n1d - 1 : 0);
          else if (nz < 0 || nz == n1d)
            continue;
          for (yp = (zp > z ? y - 1 : y); yp < y + 2; ++yp) {
            int ny = yp;
            if ((ny < 0 || ny == n1d) && s->n_dim >= 2)
              ny = (ny < 0 ? n1d - 1 : 0);
            else if (ny < 0 || ny == n1d)
              continue;
            for (xp = (yp > y || zp > z ? x - 1 : x + 1); xp < x + 2; ++xp) {
              int nx = xp;
              if (nx < 0 || nx == n1d) nx = (nx < 0 ? n1d - 1 : 0);
              if (nx == x && ny == y && nz == z) continue;
              s->nbr[13 * (size_t)c + cnt++] = cell_index(s, nx, ny, nz);
            }
          }
        }
        s->n_nbr[c] = cnt;
      }
}

/* CellList::FindCellCoords (src/cell_list.cpp:139-157) */
static void find_cell_coords(const sco_sim *s, const double *spos, int *xyz) {
  int n1d = s->n1d;
  double x = spos[0] + 0.5;
  int xc = (int)floor(n1d * x), yc, zc = 0;
  double y;
  if (xc == n1d) xc -= 1;
  y = spos[1] + 0.5;
  yc = (int)floor(n1d * y);
  if (yc == n1d) yc -= 1;
  if (s->n_dim == 3) {
    double z = spos[2] + 0.5;
    zc = (int)floor(n1d * z);
    if (zc == n1d) zc -= 1;
  }
  xyz[0] = xc;
  xyz[1] = yc;
  xyz[2] = zc;
}

static int filament_of_bond(const sco_sim *s, int b) {
  int lo = 0, hi = s->nf - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (s->fb_off[mid] <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

/* Exclusion of ProcessPairInteraction (src/interaction_manager.cpp:341-367):
 * without like-like interactions every filament pair is excluded; bonds of
 * one filament that share a site (Bond::HasNeighbor, src/bond.cpp:118-121)
 * are excluded. */
static int excluded(const sco_sim *s, int b1, int b2) {
  int f1, f2;
  if (!s->like_like) return 1;
  f1 = filament_of_bond(s, b1);
  f2 = filament_of_bond(s, b2);
  if (f1 == f2 && abs(b1 - b2) <= 1) return 1;
  return 0;
}

static void push_pair(sco_sim *s, int a, int b) {
  if (excluded(s, a, b)) return;
  if (s->np == s->pcap) {
    s->pcap = s->pcap ? 2 * s->pcap : 1024;
    s->pa = (int *)realloc(s->pa, sizeof(int) * s->pcap);
    s->pb = (int *)realloc(s->pb, sizeof(int) * s->pcap);
    s->pf = (double *)realloc(s->pf, sizeof(double) * 3 * s->pcap);
    s->pdr = (double *)realloc(s->pdr, sizeof(double) * 3 * s->pcap);
    s->ppote = (double *)realloc(s->ppote, sizeof(double) * s->pcap);
  }
  s->pa[s->np] = a;
  s->pb[s->np] = b;
  s->pf[3 * s->np] = s->pf[3 * s->np + 1] = s->pf[3 * s->np + 2] = 0.0;
  s->pdr[3 * s->np] = s->pdr[3 * s->np + 1] = s->pdr[3 * s->np + 2] = 0.0;
  s->ppote[s->np] = 0.0;
  s->np++;
}

/* InteractionManager::UpdatePairInteractions (src/interaction_manager.cpp:219-231):
 * bin every bond by its scaled position (CellList::AssignObjectsCells), then
 * CellList::MakePairs -> Cell::MakePairs (src/cell.cpp:14-22): per cell in
 * x-major order, first the pairs inside the cell (MakePairsSelf :60-70),
 * then with each half-shell neighbour (MakePairsCell :43-58).  Pairs that
 * can never interact are dropped here; the reference culls the same pairs,
 * stably, at the end of the first evaluation after the rebuild
 * (src/interaction_manager.cpp:485-497). */
static void rebuild_pairs(sco_sim *s) {
  int b, c, i, j, k;
  memset(s->cell_count, 0, sizeof(int) * s->n_cells);
  for (b = 0; b < s->nb; ++b) {
    int xyz[3];
    find_cell_coords(s, V3(s->bs, b), xyz);
    s->cell_count[cell_index(s, xyz[0], xyz[1], xyz[2])]++;
  }
  s->cell_start[0] = 0;
  for (c = 1; c < s->n_cells; ++c)
    s->cell_start[c] = s->cell_start[c - 1] + s->cell_count[c - 1];
  memset(s->cell_count, 0, sizeof(int) * s->n_cells);
  for (b = 0; b < s->nb; ++b) {
    int xyz[3], cc;
    find_cell_coords(s, V3(s->bs, b), xyz);
    cc = cell_index(s, xyz[0], xyz[1], xyz[2]);
    s->cell_items[s->cell_start[cc] + s->cell_count[cc]++] = b;
  }
  s->np = 0;
  for (c = 0; c < s->n_cells; ++c) {
    int m = s->cell_count[c];
    const int *it = s->cell_items + s->cell_start[c];
    if (m == 0) continue;
    for (i = 0; i < m - 1; ++i)
      for (j = i + 1; j < m; ++j) push_pair(s, it[i], it[j]);
    for (k = 0; k < s->n_nbr[c]; ++k) {
      int cn = s->nbr[13 * (size_t)c + k], mn = s->cell_count[cn];
      const int *itn = s->cell_items + s->cell_start[cn];
      for (i = 0; i < m; ++i)
        for (j = 0; j < mn; ++j) push_pair(s, it[i], itn[j]);
    }
  }
}

/* UpdateInteractions + ZeroDrTot (src/interaction_manager.cpp:211-217, 316-321;
 * src/mesh.cpp:546-551; src/object.cpp:278-281) */
static void update_interactions(sco_sim *s) {
  int f, j;
  s->i_update = 0;
  s->n_rebuilds++;
  if (s->interaction) rebuild_pairs(s);
  for (f = 0; f < s->nf; ++f) s->fdrmesh[f] = 0;
  for (j = 0; j < s->ns; ++j) {
    memcpy(V3(s->dz, j), V3(s->r, j), 3 * sizeof(double));
    s->dt[j] = 0;
  }
}

/* GetDrMax with Mesh::UpdateDrTot / Object::UpdateDrTot
 * (src/interaction_manager.cpp:299-312, include/simcore/species.hpp:105-120,
 * src/mesh.cpp:533-556, src/object.cpp:282-292).  Mesh::UpdateDrTot calls
 * site->UpdateDrTot() and then site->GetDrTot(), which accumulates once
 * more, so every query adds the squared displacement twice, as two
 * separate sums.  Returns -1 on the reference's "Unphysical result" error. */
static double get_dr_max(sco_sim *s) {
  double max_dr = 0;
  int f, j, i, twice;
  for (f = 0; f < s->nf; ++f) {
    if (!s->fmid[f]) {
      for (j = s->fs_off[f]; j < s->fs_off[f + 1]; ++j) {
        for (twice = 0; twice < 2; ++twice)
          for (i = 0; i < s->n_dim; ++i) {
            double dr = V3(s->r, j)[i] - V3(s->dz, j)[i];
            s->dt[j] += dr * dr;
          }
        if (s->dt[j] > s->fdrmesh[f]) s->fdrmesh[f] = s->dt[j];
      }
    }
    if (s->fdrmesh[f] > max_dr) max_dr = s->fdrmesh[f];
  }
  if (max_dr > 10000) return -1.0;
  return max_dr;
}

/* ---- static crosslinks (config E) ----------------------------------------- */

/* Anchor::UpdateAnchorPositionToMesh (src/anchor.cpp:45-68) of a bound,
 * non-static anchor with end pausing: Anchor::CheckMesh (:180-201) clamps its
 * mesh lambda to [0, true length]; Mesh::GetBondAtLambda (src/mesh.cpp:
 * 667-675) picks a bond from the nominal bond length; Anchor::CalcBondLambda
 * (:70-111) measures the lambda from that bond's mesh lambda and moves once
 * to a neighbouring bond when it falls outside; Anchor::
 * UpdateAnchorPositionToBond (:236-249) and Object::UpdatePeriodic place it.
 * Returns the anchor's scaled position, orientation, bond length and lambda;
 * its bond is recorded in xbond. */
static void anchor_state(sco_sim *s, int anchor, double *sp, double *u, double *len,
                         double *lambda) {
  const int f = s->xfil[anchor], b0 = s->fb_off[f], nbf = s->fb_off[f + 1] - b0;
  double M = s->xM[anchor], ap[3] = {0, 0, 0}, bl, lam;
  int k, i, n = s->n_dim;
  if (M < 0) M = 0;
  else if (M > s->ftl[f]) M = s->ftl[f];
  s->xM[anchor] = M;
  if (M < 0) k = 0;
  else if (M >= s->fL[f]) k = nbf - 1;
  else k = (int)floor(M / s->fl[f]);
  /* M / l can round up to the bond count just below the nominal length,
   * where the reference would index past its bonds: kept on the last. */
  if (k > nbf - 1) k = nbf - 1;
  if (k < 0) k = 0;
  lam = M - s->bml[b0 + k];
  bl = s->bl[b0 + k];
  if (lam < 0) {
    if (k > 0) {
      --k;
      lam = M - s->bml[b0 + k];
      bl = s->bl[b0 + k];
    } else {
      lam = 0;
    }
  } else if (lam > bl) {
    if (k < nbf - 1) {
      ++k;
      lam = M - s->bml[b0 + k];
      bl = s->bl[b0 + k];
    } else {
      lam = bl;
    }
  }
  if (lam < -1e-6 || lam > bl + 1e-6) s->xerr = 1; /* the reference stops here */
  s->xbond[anchor] = b0 + k;
  for (i = 0; i < 3; ++i) u[i] = V3(s->bu, b0 + k)[i];
  for (i = 0; i < n; ++i) ap[i] = V3(s->bp, b0 + k)[i] - (0.5 * bl - lam) * u[i];
  *len = bl;
  *lambda = lam;
  periodic_bc(n, s->hinv, ap, sp);
}

/* Crosslink::CalculateTetherForces (src/crosslink.cpp:247-275) with
 * MinimumDistance::PointPoint (src/minimum_distance.cpp:71-101), then the
 * torque of Anchor::ApplyAnchorForces (src/anchor.cpp:132-146). */
static void tether_forces(sco_sim *s) {
  int k, i, a, n = s->n_dim;
  for (k = 0; k < s->nx; ++k) {
    double sp[2][3] = {{0}}, u[2][3] = {{0}}, len[2], lam[2];
    double ds[3] = {0, 0, 0}, dr[3] = {0, 0, 0}, dr2 = 0, f[3] = {0, 0, 0};
    double length, stretch, tf;
    int j;
    for (a = 0; a < 2; ++a) anchor_state(s, 2 * k + a, sp[a], u[a], &len[a], &lam[a]);
    for (i = 0; i < n; ++i) {
      ds[i] = sp[1][i] - sp[0][i];
      ds[i] -= NINT(ds[i]);
    }
    for (i = 0; i < n; ++i) {
      dr[i] = 0.0;
      for (j = 0; j < n; ++j) dr[i] += s->h[n * i + j] * ds[j];
    }
    for (i = 0; i < n; ++i) dr2 += dr[i] * dr[i];
    length = sqrt(dr2);
    stretch = length - s->xrest;
    tf = (s->xkc >= 0 && stretch < 0) ? s->xkc * stretch : s->xk * stretch;
    for (i = 0; i < n; ++i) f[i] = tf * (dr[i] / length);
    memcpy(s->xF + 3 * k, f, sizeof(f));
    for (a = 0; a < 2; ++a) {
      double *c = s->xc + 6 * (size_t)(2 * k + a);
      double dl[3] = {0, 0, 0};
      c[0] = c[1] = c[2] = 0.0;
      for (i = 0; i < n; ++i) c[i] = a == 0 ? c[i] + f[i] : c[i] - f[i];
      for (i = 0; i < n; ++i) dl[i] = (lam[a] - 0.5 * len[a]) * u[a][i];
      cross3(dl, c, c + 3);
    }
  }
}

/* CrosslinkSpecies::UpdatePositions (src/crosslink_species.cpp:218-238):
 * even i_steps recompute the tether forces, every i_step applies the stored
 * anchor forces and torques in link order (ApplyCrosslinkTetherForces
 * :260-266, Anchor::ApplyAnchorForces). */
static void crosslink_update(sco_sim *s) {
  int k, i;
  if (s->i_step % 2 == 0) tether_forces(s);
  for (k = 0; k < 2 * s->nx; ++k) {
    const double *c = s->xc + 6 * (size_t)k;
    const int b = s->xbond[k];
    for (i = 0; i < s->n_dim; ++i) V3(s->bF, b)[i] += c[i];
    for (i = 0; i < 3; ++i) V3(s->bT, b)[i] += c[3 + i];
  }
}

/* CalculatePairInteractions + ApplyPairInteractions
 * (src/interaction_manager.cpp:448-517), serial. */
static void pair_interactions(sco_sim *s, double *bF, double *bT, int commit) {
  long p;
  int i;
  for (p = 0; p < s->np; ++p) {
    int a = s->pa[p], b = s->pb[p], n = s->n_dim, j;
    double force[3], t1[3], t2[3], rdr[3], rpote = s->ppote[p];
    memcpy(force, s->pf + 3 * p, sizeof(force));
    memcpy(rdr, s->pdr + 3 * p, sizeof(rdr));
    pair_force(s, a, b, force, t1, t2, rdr, &rpote);
    if (commit) {
      memcpy(s->pf + 3 * p, force, sizeof(force));
      memcpy(s->pdr + 3 * p, rdr, sizeof(rdr));
      s->ppote[p] = rpote;
    }
    for (i = 0; i < s->n_dim; ++i) {
      V3(bF, a)[i] += force[i];
      V3(bF, b)[i] -= force[i];
    }
    for (i = 0; i < 3; ++i) {
      V3(bT, a)[i] += t1[i];
      V3(bT, b)[i] -= t2[i];
    }
    if (commit) {
      /* obj1/obj2->AddPotential(pote); stress_ += ix->stress, where
       * ix->stress[n i + j] = -dr[i] * force[j] (wca_potential.hpp:26-28) */
      s->bpote[a] += rpote;
      s->bpote[b] += rpote;
      for (i = 0; i < n; ++i)
        for (j = 0; j < n; ++j) s->stress[n * i + j] += -rdr[i] * force[j];
    }
  }
}

/* ---- the filament integrator (src/filament.cpp) ---------------------------- */

/* Filament::UpdatePosition (src/filament.cpp:394-404) for one filament:
 * ApplyInteractionForces (:992-1048), then Integrate (:410-428). */
static void filament_update(sco_sim *s, int f, int midstep) {
  const int nd = s->n_dim;
  const int s0 = s->fs_off[f], b0 = s->fb_off[f];
  const int n = s->fs_off[f + 1] - s0; /* n_sites */
  const double l = s->fl[f], kappa = s->flp[f];
  const double gpar = s->gpar[f], gperp = s->gperp[f];
  double *cosv = s->w_cos, *gl = s->w_gl, *gd = s->w_gd, *gu = s->w_gu;
  double *dtm = s->w_dt, *dbm = s->w_db, *ginv = s->w_ginv, *keff = s->w_keff;
  double *hd = s->w_hd, *hu = s->w_hu, *hl = s->w_hl, *gam = s->w_gam;
  double *T = s->tens + b0;
  int i, j, k;
#define SU(j) V3(s->u, s0 + (j))
#define SR(j) V3(s->r, s0 + (j))
#define SRP(j) V3(s->rp, s0 + (j))
#define SF(j) V3(s->F, s0 + (j))
#define SFR(j) V3(s->fr, s0 + (j))
#define ST(j) V3(s->tn, s0 + (j))

  s->fmid[f] = midstep;

  /* ApplyInteractionForces: bond force/torque -> forces on its two sites. */
  {
    double linv = 1.0 / l;
    for (i = 0; i < n - 1; ++i) {
      const double *fb = V3(s->bF, b0 + i), *tb = V3(s->bT, b0 + i);
      const double *uu = SU(i);
      double pt[3], sf[3], fdr[3] = {0, 0, 0}, mag;
      cross3(uu, tb, pt);
      for (k = 0; k < nd; ++k) {
        pt[k] *= linv;
        sf[k] = 0.5 * fb[k];
      }
      for (k = 0; k < nd; ++k) SF(i)[k] += sf[k];
      for (k = 0; k < nd; ++k) SF(i)[k] += pt[k];
      for (k = 0; k < nd; ++k) pt[k] *= -1;
      for (k = 0; k < nd; ++k) SF(i + 1)[k] += sf[k];
      for (k = 0; k < nd; ++k) SF(i + 1)[k] += pt[k];
      /* driving from the bond centre with driving_factor 0 */
      mag = 0.5 * 0.0 * l;
      for (k = 0; k < nd; ++k) fdr[k] = mag * uu[k];
      for (k = 0; k < nd; ++k) SF(i)[k] += fdr[k];
      for (k = 0; k < nd; ++k) SF(i + 1)[k] += fdr[k];
    }
  }

  /* CalculateAngles (:430-437), CalculateTangents (:439-443) */
  for (i = 0; i < n - 2; ++i) cosv[i] = dot_product(nd, SU(i), SU(i + 1));
  calc_tangents(s, f);

  if (midstep) {
    if (s->stoch) {
      /* ConstructUnprojectedRandomForces (:518-548) */
      for (j = 0; j < n; ++j) {
        const double *ut = ST(j);
        double xi[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
        for (i = 0; i < nd; ++i)
          xi[i] = sc_philox_noise(s->seed, (uint32_t)f, s->fdraw[f], (uint32_t)j, i) - 0.5;
        if (nd == 2) {
          xt[0] = SQR(ut[0]) * xi[0] + ut[0] * ut[1] * xi[1];
          xt[1] = SQR(ut[1]) * xi[1] + ut[0] * ut[1] * xi[0];
        } else {
          xt[0] = SQR(ut[0]) * xi[0] + ut[0] * ut[1] * xi[1] +
                  ut[0] * ut[2] * xi[2];
          xt[1] = SQR(ut[1]) * xi[1] + ut[0] * ut[1] * xi[0] +
                  ut[1] * ut[2] * xi[2];
          xt[2] = SQR(ut[2]) * xi[2] + ut[0] * ut[2] * xi[0] +
                  ut[1] * ut[2] * xi[1];
        }
        for (i = 0; i < nd; ++i)
          SFR(j)[i] = s->sperp[f] * xi[i] + (s->spar[f] - s->sperp[f]) * xt[i];
      }
      s->fdraw[f]++; /* one noisy midstep of this filament */
      /* GeometricallyProjectRandomForces (:550-599) */
      for (j = 0; j < n - 1; ++j) {
        double tmp[3];
        for (i = 0; i < nd; ++i) tmp[i] = SFR(j + 1)[i] - SFR(j)[i];
        T[j] = dot_product(nd, tmp, SU(j));
        gd[j] = 2;
        if (j > 0) {
          gu[j - 1] = -cosv[j - 1];
          gl[j - 1] = -cosv[j - 1];
        }
      }
      thomas(gl, gd, gu, T, n - 1);
      {
        double fp[3];
        for (i = 0; i < nd; ++i) fp[i] = SFR(0)[i] + T[0] * SU(0)[i];
        for (i = 0; i < nd; ++i) SFR(0)[i] = fp[i];
        for (i = 0; i < nd; ++i)
          fp[i] = SFR(n - 1)[i] - T[n - 2] * SU(n - 2)[i];
        for (i = 0; i < nd; ++i) SFR(n - 1)[i] = fp[i];
        for (j = 1; j < n - 1; ++j) {
          for (i = 0; i < nd; ++i)
            fp[i] = SFR(j)[i] + T[j] * SU(j)[i] - T[j - 1] * SU(j - 1)[i];
          for (i = 0; i < nd; ++i) SFR(j)[i] = fp[i];
        }
      }
    }
    /* Mesh::UpdatePrevPositions (src/mesh.cpp:175-182) */
    for (j = 0; j < n; ++j)
      for (i = 0; i < nd; ++i) SRP(j)[i] = SR(j)[i];
  }

  /* AddRandomForces (:601-606) */
  if (s->stoch)
    for (j = 0; j < n; ++j)
      for (i = 0; i < nd; ++i) SF(j)[i] += SFR(j)[i];

  /* CalculateBendingForces (:608-776) */
  {
    double det_g;
    dtm[0] = 1;
    dtm[1] = 2;
    dbm[n] = 1;
    dbm[n - 1] = 2;
    for (i = 2; i < n; ++i) {
      dtm[i] = 2 * dtm[i - 1] - SQR(-cosv[i - 2]) * dtm[i - 2];
      dbm[n - i] = 2 * dbm[n - i + 1] - SQR(-cosv[n - i - 1]) * dbm[n - i + 2];
    }
    det_g = dtm[n - 1];
    for (i = 0; i < n - 2; ++i)
      ginv[i] = cosv[i] * dtm[i] * dbm[i + 3] / det_g;
    for (i = 0; i < n - 2; ++i) keff[i] = (kappa + l * ginv[i]) / SQR(l);
    for (k = 0; k < n; ++k) {
      double fs[3] = {0, 0, 0};
      if (nd == 2) {
        if (k > 1) {
          const double *u1 = SU(k - 2), *u2 = SU(k - 1);
          fs[0] += keff[k - 2] * ((1 - SQR(u2[0])) * u1[0] - u2[0] * u2[1] * u1[1]);
          fs[1] += keff[k - 2] * ((1 - SQR(u2[1])) * u1[1] - u2[0] * u2[1] * u1[0]);
        }
        if (k > 0 && k < n - 1) {
          const double *u1 = SU(k - 1), *u2 = SU(k);
          fs[0] += keff[k - 1] *
                   ((1 - SQR(u1[0])) * u2[0] - u1[0] * u1[1] * u2[1] -
                    ((1 - SQR(u2[0])) * u1[0] - u2[0] * u2[1] * u1[1]));
          fs[1] += keff[k - 1] *
                   ((1 - SQR(u1[1])) * u2[1] - u1[0] * u1[1] * u2[0] -
                    ((1 - SQR(u2[1])) * u1[1] - u2[0] * u2[1] * u1[0]));
        }
        if (k < n - 2) {
          const double *u1 = SU(k), *u2 = SU(k + 1);
          fs[0] -= keff[k] * ((1 - SQR(u1[0])) * u2[0] - u1[0] * u1[1] * u2[1]);
          fs[1] -= keff[k] * ((1 - SQR(u1[1])) * u2[1] - u1[0] * u1[1] * u2[0]);
        }
      } else {
        if (k > 1) {
          const double *u1 = SU(k - 2), *u2 = SU(k - 1);
          fs[0] += keff[k - 2] * ((1 - SQR(u2[0])) * u1[0] -
                                  u2[0] * u2[1] * u1[1] - u2[0] * u2[2] * u1[2]);
          fs[1] += keff[k - 2] * ((1 - SQR(u2[1])) * u1[1] -
                                  u2[1] * u2[0] * u1[0] - u2[1] * u2[2] * u1[2]);
          fs[2] += keff[k - 2] * ((1 - SQR(u2[2])) * u1[2] -
                                  u2[2] * u2[0] * u1[0] - u2[2] * u2[1] * u1[1]);
        }
        if (k > 0 && k < n - 1) {
          const double *u1 = SU(k - 1), *u2 = SU(k);
          fs[0] += keff[k - 1] *
                   ((1 - SQR(u1[0])) * u2[0] - u1[0] * u1[1] * u2[1] -
                    u1[0] * u1[2] * u2[2] -
                    ((1 - SQR(u2[0])) * u1[0] - u2[0] * u2[1] * u1[1] -
                     u2[0] * u2[2] * u1[2]));
          fs[1] += keff[k - 1] *
                   ((1 - SQR(u1[1])) * u2[1] - u1[1] * u1[0] * u2[0] -
                    u1[1] * u1[2] * u2[2] -
                    ((1 - SQR(u2[1])) * u1[1] - u2[1] * u2[0] * u1[0] -
                     u2[1] * u2[2] * u1[2]));
          fs[2] += keff[k - 1] *
                   ((1 - SQR(u1[2])) * u2[2] - u1[2] * u1[0] * u2[0] -
                    u1[2] * u1[1] * u2[1] -
                    ((1 - SQR(u2[2])) * u1[2] - u2[2] * u2[0] * u1[0] -
                     u2[1] * u2[2] * u1[1]));
        }
        if (k < n - 2) {
          const double *u1 = SU(k), *u2 = SU(k + 1);
          fs[0] -= keff[k] * ((1 - SQR(u1[0])) * u2[0] - u1[0] * u1[1] * u2[1] -
                              u1[0] * u1[2] * u2[2]);
          fs[1] -= keff[k] * ((1 - SQR(u1[1])) * u2[1] - u1[1] * u1[0] * u2[0] -
                              u1[1] * u1[2] * u2[2]);
          fs[2] -= keff[k] * ((1 - SQR(u1[2])) * u2[2] - u1[2] * u1[0] * u2[0] -
                              u1[2] * u1[1] * u2[1]);
        }
      }
      for (i = 0; i < nd; ++i) SF(k)[i] += fs[i];
    }
  }

  /* CalculateTensions (:778-838) */
  for (j = 0; j < n; ++j) {
    const double *ut = ST(j);
    int gi = 0, a, b;
    for (a = 0; a < nd; ++a)
      for (b = 0; b < nd; ++b) {
        gam[9 * j + gi] = 1.0 / gpar * (ut[a] * ut[b]) +
                          1.0 / gperp * ((a == b ? 1 : 0) - ut[a] * ut[b]);
        gi++;
      }
  }
  for (j = 0; j < n - 1; ++j) {
    const double *f1 = SF(j), *f2 = SF(j + 1), *u2 = SU(j);
    const double *ut1 = ST(j), *ut2 = ST(j + 1);
    const double *g1 = gam + 9 * j, *g2 = gam + 9 * (j + 1);
    double fdiff[3], ta, tb, d1, d2;
    for (i = 0; i < nd; ++i) {
      ta = g1[nd * i] * f1[0] + g1[nd * i + 1] * f1[1];
      if (nd == 3) ta += g1[nd * i + 2] * f1[2];
      tb = g2[nd * i] * f2[0] + g2[nd * i + 1] * f2[1];
      if (nd == 3) tb += g2[nd * i + 2] * f2[2];
      fdiff[i] = tb - ta;
    }
    T[j] = dot_product(nd, u2, fdiff);
    d1 = dot_product(nd, ut1, u2);
    d2 = dot_product(nd, ut2, u2);
    hd[j] = 2.0 / gperp + (1.0 / gpar - 1.0 / gperp) * (SQR(d1) + SQR(d2));
    if (j > 0) {
      const double *u1 = SU(j - 1);
      hu[j - 1] = -1.0 / gperp * dot_product(nd, u2, u1) -
                  (1.0 / gpar - 1.0 / gperp) *
                      (dot_product(nd, ut1, u1) * dot_product(nd, ut1, u2));
      hl[j - 1] = hu[j - 1];
    }
  }
  thomas(hl, hd, hu, T, n - 1);

  /* UpdateSitePositions (:840-927) with CheckBondLengths (:934-951) */
  {
    double dl = (midstep ? 0.5 * s->delta : s->delta);
    double fs[3], ft[3], rn[3], rd[3], um;
    int renorm = 0;
    for (i = 0; i < nd; ++i) fs[i] = T[0] * SU(0)[i];
    for (i = 0; i < nd; ++i) SF(0)[i] += fs[i];
    for (i = 0; i < nd; ++i) fs[i] = -T[n - 2] * SU(n - 2)[i];
    for (i = 0; i < nd; ++i) SF(n - 1)[i] += fs[i];
    for (j = 1; j < n - 1; ++j) {
      for (i = 0; i < nd; ++i) fs[i] = T[j] * SU(j)[i] - T[j - 1] * SU(j - 1)[i];
      for (i = 0; i < nd; ++i) SF(j)[i] += fs[i];
    }
    for (j = 0; j < n; ++j) {
      const double *g = gam + 9 * j, *fsite = SF(j), *rprev = SRP(j);
      for (i = 0; i < nd; ++i) {
        ft[i] = g[nd * i] * fsite[0] + g[nd * i + 1] * fsite[1];
        if (nd == 3) ft[i] += g[nd * i + 2] * fsite[2];
        rn[i] = rprev[i] + dl * ft[i];
      }
      for (i = 0; i < nd; ++i) SR(j)[i] = rn[i];
    }
    for (j = 0; j < n - 1; ++j) {
      um = 0.0;
      for (i = 0; i < nd; ++i) {
        rd[i] = SR(j + 1)[i] - SR(j)[i];
        um += SQR(rd[i]);
      }
      um = sqrt(um);
      for (i = 0; i < nd; ++i) rd[i] /= um;
      for (i = 0; i < nd; ++i) SU(j)[i] = rd[i];
    }
    for (i = 0; i < nd; ++i) SU(n - 1)[i] = SU(n - 2)[i];
    for (j = 1; j < n; ++j) {
      double a = 0.0, err;
      for (i = 0; i < nd; ++i) {
        double temp = SR(j)[i] - SR(j - 1)[i];
        a += temp * temp;
      }
      a = sqrt(a);
      err = ABS(l - a) / l;
      if (err > 1e-3) renorm = 1;
    }
    if (renorm) {
      s->fswitch[f] = !s->fswitch[f];
      s->fnnorm[f] = 0;
      if (s->fswitch[f]) {
        for (j = 1; j < n; ++j) {
          for (i = 0; i < nd; ++i) rd[i] = SR(j - 1)[i] + l * SU(j - 1)[i];
          for (i = 0; i < nd; ++i) SR(j)[i] = rd[i];
        }
      } else {
        for (j = n - 1; j > 0; --j) {
          for (i = 0; i < nd; ++i) rd[i] = SR(j)[i] - l * SU(j - 1)[i];
          for (i = 0; i < nd; ++i) SR(j - 1)[i] = rd[i];
        }
      }
    }
    s->fnnorm[f]++;
  }
  update_bond_positions(s, f);
#undef SU
#undef SR
#undef SRP
#undef SF
#undef SFR
#undef ST
}

/* ---- public interface ------------------------------------------------------ */

int sco_filament_n_bonds(const sco_filament *f) {
  /* Filament::SetParameters / InitFilamentLength (src/filament.cpp:73-83,
   * 104-147) for static lengths: max bond length 1.5 * min_bond_length,
   * at least two bonds, length clamped to [max(5, 2*mbl), 500]. */
  double max_bond_length = 1.5 * f->min_bond_length;
  double min_length = 5, max_length = 500, length = f->length;
  int n_bonds;
  if (min_length < 2 * f->min_bond_length) min_length = 2 * f->min_bond_length;
  if (max_length < min_length) max_length = min_length;
  if (length > max_length)
    length = max_length;
  else if (length < min_length)
    length = min_length;
  n_bonds = (int)floor(length / max_bond_length);
  n_bonds = (n_bonds == 1 ? 2 : n_bonds);
  return n_bonds;
}

static void *xcalloc(size_t n, size_t sz) {
  void *p = calloc(n ? n : 1, sz);
  return p;
}

sco_sim *sco_create(const sco_system *sys, int n_fil, const sco_filament *fils,
                    const double *site_xyz, int n_sites) {
  sco_sim *s;
  int f, j, nd, max_ns = 0;
  double min_len, spec_length;
  if (!sys || n_fil <= 0 || !fils || !site_xyz) return NULL;
  if (sys->n_dim != 2 && sys->n_dim != 3) return NULL;
  s = (sco_sim *)xcalloc(1, sizeof(sco_sim));
  nd = s->n_dim = sys->n_dim;
  s->R = sys->system_radius;
  s->delta = sys->delta;
  s->eps = sys->wca_eps;
  s->sig = sys->wca_sig;
  s->fcut = sys->f_cutoff;
  s->stoch = sys->stoch_flag != 0;
  s->interaction = sys->interaction_flag != 0;
  s->like_like = sys->like_like_interactions != 0;
  s->seed = sys->seed;
  s->species_midstep = 1;

  /* Space::InitUnitCell / CalculateUnitCellQuantities (src/space.cpp:85-138) */
  {
    int a, b;
    double hh = 2.0 * s->R;
    for (a = 0; a < 9; ++a) s->h[a] = s->hinv[a] = 0;
    for (a = 0; a < nd; ++a)
      for (b = 0; b < nd; ++b) s->h[a * nd + b] = (a == b ? 1 : 0) * hh;
    s->h[nd * nd - 1] = hh;
    if (nd == 2) invert_sym_2d(s->h, s->hinv);
    else invert_sym_3d(s->h, s->hinv);
  }
  /* WCAPotential::Init (include/simcore/wca_potential.hpp:34-48) */
  {
    double rcut = pow(2.0, 1.0 / 6.0) * s->sig;
    s->rcut2 = rcut * rcut;
    s->c12 = 4.0 * s->eps * pow(s->sig, 12.0);
    s->c6 = 4.0 * s->eps * pow(s->sig, 6.0);
  }
  /* Cell size: SetMinCellLength calls of Simulation::InitSpecies
   * (src/simulation.cpp:248-251) and InteractionManager::InitInteractions
   * (src/interaction_manager.cpp:46-48), then CellList::Init
   * (src/cell_list.cpp:17-64). */
  min_len = -1;
  spec_length = 1.5 * fils[0].min_bond_length;
  if (fils[0].diameter > spec_length) spec_length = fils[0].diameter;
  if (spec_length > min_len) min_len = spec_length;
  if (0.0 > min_len) min_len = 0.0;
  if (sqrt(s->rcut2) > min_len) min_len = sqrt(s->rcut2);
  s->n1d = (int)floor(2 * s->R / min_len);
  if (s->n1d <= 3) s->n1d = 3;
  s->cl = (double)2 * s->R / s->n1d;
  s->dr_update = 0.25 * s->cl * s->cl;
  s->n_cells = s->n1d * s->n1d * (nd == 3 ? s->n1d : 1);
  s->nbr = (int *)xcalloc((size_t)s->n_cells * 13, sizeof(int));
  s->n_nbr = (int *)xcalloc(s->n_cells, sizeof(int));
  s->cell_start = (int *)xcalloc(s->n_cells, sizeof(int));
  s->cell_count = (int *)xcalloc(s->n_cells, sizeof(int));
  build_neighbors(s);

  /* filaments */
  s->nf = n_fil;
  s->fs_off = (int *)xcalloc(n_fil + 1, sizeof(int));
  s->fb_off = (int *)xcalloc(n_fil + 1, sizeof(int));
  for (f = 0; f < n_fil; ++f) {
    int nb = sco_filament_n_bonds(&fils[f]);
    s->fb_off[f + 1] = s->fb_off[f] + nb;
    s->fs_off[f + 1] = s->fs_off[f] + nb + 1;
    if (nb + 1 > max_ns) max_ns = nb + 1;
  }
  if (s->fs_off[n_fil] != n_sites) {
    free(s->nbr); free(s->n_nbr); free(s->cell_start); free(s->cell_count);
    free(s->fs_off); free(s->fb_off); free(s);
    return NULL;
  }
  s->ns = n_sites;
  s->nb = s->fb_off[n_fil];
  s->max_ns = max_ns;
  s->cell_items = (int *)xcalloc(s->nb, sizeof(int));
#define ALLOCD(p, n) p = (double *)xcalloc((size_t)(n), sizeof(double))
  ALLOCD(s->fl, n_fil); ALLOCD(s->flp, n_fil); ALLOCD(s->fd, n_fil);
  ALLOCD(s->gpar, n_fil); ALLOCD(s->gperp, n_fil); ALLOCD(s->spar, n_fil);
  ALLOCD(s->sperp, n_fil); ALLOCD(s->fdrmesh, n_fil);
  s->fswitch = (int *)xcalloc(n_fil, sizeof(int));
  s->fnnorm = (int *)xcalloc(n_fil, sizeof(int));
  s->fmid = (int *)xcalloc(n_fil, sizeof(int));
  s->fdraw = (uint64_t *)xcalloc(n_fil, sizeof(uint64_t));
  ALLOCD(s->r, 3 * n_sites); ALLOCD(s->rp, 3 * n_sites); ALLOCD(s->fr, 3 * n_sites);
  ALLOCD(s->F, 3 * n_sites); ALLOCD(s->tn, 3 * n_sites); ALLOCD(s->u, 3 * n_sites);
  ALLOCD(s->dz, 3 * n_sites); ALLOCD(s->dt, n_sites);
  ALLOCD(s->bp, 3 * s->nb); ALLOCD(s->bs, 3 * s->nb); ALLOCD(s->bu, 3 * s->nb);
  ALLOCD(s->bl, s->nb); ALLOCD(s->bF, 3 * s->nb); ALLOCD(s->bT, 3 * s->nb);
  ALLOCD(s->bml, s->nb); ALLOCD(s->ftl, n_fil); ALLOCD(s->fL, n_fil);
  ALLOCD(s->tens, s->nb); ALLOCD(s->bpote, s->nb);
  ALLOCD(s->w_cos, max_ns); ALLOCD(s->w_gl, max_ns); ALLOCD(s->w_gd, max_ns);
  ALLOCD(s->w_gu, max_ns); ALLOCD(s->w_dt, max_ns + 1); ALLOCD(s->w_db, max_ns + 1);
  ALLOCD(s->w_ginv, max_ns); ALLOCD(s->w_keff, max_ns); ALLOCD(s->w_hd, max_ns);
  ALLOCD(s->w_hu, max_ns); ALLOCD(s->w_hl, max_ns); ALLOCD(s->w_gam, 9 * max_ns);
#undef ALLOCD
  for (f = 0; f < n_fil; ++f) {
    int nb = s->fb_off[f + 1] - s->fb_off[f], ns = nb + 1;
    double length = fils[f].length, logLD;
    double min_length = 5, max_length = 500;
    if (min_length < 2 * fils[f].min_bond_length)
      min_length = 2 * fils[f].min_bond_length;
    if (max_length < min_length) max_length = min_length;
    if (length > max_length) length = max_length;
    else if (length < min_length) length = min_length;
    s->fl[f] = length / nb; /* bond_length_ = length_ / n_bonds_ */
    s->fL[f] = length;      /* length_ */
    s->flp[f] = fils[f].persistence_length;
    s->fd[f] = fils[f].diameter;
    /* Filament::SetDiffusion (src/filament.cpp:320-348) */
    logLD = log(length / fils[f].diameter);
    s->gperp[f] = 4.0 * length / (3.0 * ns * logLD);
    s->gpar[f] = s->gperp[f] / fils[f].friction_ratio;
    s->sperp[f] = sqrt(24.0 * s->gperp[f] / s->delta);
    s->spar[f] = sqrt(24.0 * s->gpar[f] / s->delta);
    s->fswitch[f] = 1; /* normalize_switch_ = true (include/simcore/filament.hpp:18) */
    s->fnnorm[f] = 0;
    s->fmid[f] = 1;    /* Mesh::midstep_ = true (include/simcore/mesh.hpp:17) */
  }
  sco_set_sites(s, site_xyz);
  /* Simulation::InsertSpecies tail: forced update = rebuild + ZeroDrTot */
  update_interactions(s);
  s->n_rebuilds = 0;
  (void)j;
  return s;
}

void sco_set_sites(sco_sim *s, const double *xyz) {
  int f, j, d;
  for (j = 0; j < s->ns; ++j)
    for (d = 0; d < 3; ++d) {
      double v = d < s->n_dim ? xyz[3 * j + d] : 0.0;
      V3(s->r, j)[d] = v;
      V3(s->rp, j)[d] = v;
    }
  for (f = 0; f < s->nf; ++f) update_bond_positions(s, f);
}

void sco_destroy(sco_sim *s) {
  if (!s) return;
  free(s->nbr); free(s->n_nbr); free(s->cell_start); free(s->cell_count);
  free(s->cell_items); free(s->fs_off); free(s->fb_off);
  free(s->fl); free(s->flp); free(s->fd); free(s->gpar); free(s->gperp);
  free(s->spar); free(s->sperp); free(s->fdrmesh); free(s->fswitch);
  free(s->fnnorm); free(s->fmid); free(s->fdraw);
  free(s->r); free(s->rp); free(s->fr); free(s->F); free(s->tn); free(s->u);
  free(s->dz); free(s->dt); free(s->bp); free(s->bs); free(s->bu); free(s->bl);
  free(s->bF); free(s->bT); free(s->tens);
  free(s->xbond); free(s->xfil); free(s->xM); free(s->xc); free(s->xF);
  free(s->bml); free(s->ftl); free(s->fL);
  free(s->pa); free(s->pb); free(s->pf); free(s->pdr); free(s->ppote);
  free(s->bpote); free(s->rec);
  free(s->w_cos); free(s->w_gl); free(s->w_gd); free(s->w_gu); free(s->w_dt);
  free(s->w_db); free(s->w_ginv); free(s->w_keff); free(s->w_hd); free(s->w_hu);
  free(s->w_hl); free(s->w_gam);
  free(s);
}

int sco_n_sites(const sco_sim *s) { return s->ns; }
int sco_n_bonds(const sco_sim *s) { return s->nb; }
int sco_n_cells_1d(const sco_sim *s) { return s->n1d; }
double sco_cell_length(const sco_sim *s) { return s->cl; }
double sco_dr_update(const sco_sim *s) { return s->dr_update; }
long sco_n_rebuilds(const sco_sim *s) { return s->n_rebuilds; }
int sco_i_step(const sco_sim *s) { return s->i_step; }

/* InteractionManager::CalculatePressure (src/interaction_manager.cpp:535-559)
 * for the periodic box of Space::CalculateVolume (src/space.cpp:252-264,
 * boundary 0): n_objs = the bond count (Mesh::GetCount, src/mesh.cpp:399).
 * Appends the record OutputManager::WriteThermo writes. */
static void calculate_pressure(sco_sim *s) {
  const int n = s->n_dim;
  const double side = 2 * s->R;
  const double volume = n == 2 ? side * side : side * side * side;
  const double inv_V = 1.0 / volume;
  double P[9] = {0}, pressure = 0;
  int i, j;
  for (i = 0; i < n; ++i)
    for (j = 0; j < n; ++j) {
      if (i == j) P[n * i + j] += s->nb * inv_V;
      P[n * i + j] += s->stress[n * i + j] * inv_V / s->n_thermo;
    }
  for (i = 0; i < n; ++i) pressure += P[n * i + i];
  pressure /= n;
  memset(s->stress, 0, sizeof(s->stress));
  if (s->n_rec == s->rec_cap) {
    s->rec_cap = s->rec_cap ? 2 * s->rec_cap : 64;
    s->rec = (double *)realloc(s->rec, sizeof(double) * 12 * (size_t)s->rec_cap);
  }
  {
    double *q = s->rec + 12 * s->n_rec++;
    q[0] = (double)s->i_step;
    memcpy(q + 1, P, sizeof(P));
    q[10] = pressure;
    q[11] = volume;
  }
}

/* Simulation::RunSimulation body (src/simulation.cpp:37-62): ZeroForces,
 * Interact, Integrate.  Interact follows src/interaction_manager.cpp:63-95. */
int sco_step(sco_sim *s, int nsteps) {
  int it, f;
  for (it = 0; it < nsteps; ++it) {
    s->i_step++;
    memset(s->F, 0, sizeof(double) * 3 * s->ns);
    memset(s->bF, 0, sizeof(double) * 3 * s->nb);
    memset(s->bT, 0, sizeof(double) * 3 * s->nb);
    memset(s->bpote, 0, sizeof(double) * s->nb);
    if (s->interaction) {
      double dr_max;
      if (s->nx) crosslink_update(s); /* src/interaction_manager.cpp:70 */
      dr_max = get_dr_max(s);
      if (dr_max < 0) return -1;
      if (dr_max > s->dr_update) update_interactions(s);
      pair_interactions(s, s->bF, s->bT, 1);
      s->i_update++;
    }
    for (f = 0; f < s->nf; ++f) filament_update(s, f, s->species_midstep);
    s->species_midstep = !s->species_midstep;
    /* Simulation::Statistics (src/simulation.cpp:108-114) */
    if (s->n_thermo > 0 && s->i_step % s->n_thermo == 0) calculate_pressure(s);
  }
  return 0;
}

void sco_set_thermo(sco_sim *s, int n_thermo) {
  s->n_thermo = n_thermo;
  s->n_rec = 0;
}

/* Pressure records since the last call (at most max): i_step, pressure
 * tensor (9, n_dim x n_dim packed), pressure and volume each. */
long sco_thermo_records(sco_sim *s, long max, long *i_step, double *tensor, double *pressure,
                        double *volume) {
  long k, n = s->n_rec < max ? s->n_rec : max;
  for (k = 0; k < n; ++k) {
    const double *q = s->rec + 12 * k;
    i_step[k] = (long)q[0];
    memcpy(tensor + 9 * k, q + 1, 9 * sizeof(double));
    pressure[k] = q[10];
    volume[k] = q[11];
  }
  s->n_rec = 0;
  return n;
}

void sco_get_stress(const sco_sim *s, double *stress) {
  memcpy(stress, s->stress, sizeof(s->stress));
}

/* Object::GetPotentialEnergy of each filament after the last step: the sum,
 * in bond order, of its bonds' potentials (Filament::ApplyInteractionForces,
 * src/filament.cpp:1007), each the sum of its pairs' in list order. */
void sco_get_potential_energy(const sco_sim *s, double *pote) {
  int f, i;
  for (f = 0; f < s->nf; ++f) {
    double e = 0;
    for (i = s->fb_off[f]; i < s->fb_off[f + 1]; ++i) e += s->bpote[i];
    pote[f] = e;
  }
}

int sco_add_crosslinks(sco_sim *s, int n, const int *site_a, const int *site_b,
                       double k_spring, double k_spring_compress, double rest_length) {
  int k, a;
  if (s->nx || n <= 0) return -1;
  s->xbond = (int *)xcalloc(2 * (size_t)n, sizeof(int));
  s->xfil = (int *)xcalloc(2 * (size_t)n, sizeof(int));
  s->xM = (double *)xcalloc(2 * (size_t)n, sizeof(double));
  s->xc = (double *)xcalloc(12 * (size_t)n, sizeof(double));
  s->xF = (double *)xcalloc(3 * (size_t)n, sizeof(double));
  /* Anchor::AttachObjLambda (src/anchor.cpp:284-316): on the bond whose tail
   * is the site at lambda 0, or for a filament's last site on its last bond
   * at lambda = that bond's length; the anchor's mesh lambda is the bond's
   * plus lambda. */
  for (k = 0; k < n; ++k)
    for (a = 0; a < 2; ++a) {
      const int site = a == 0 ? site_a[k] : site_b[k];
      int f = 0, b;
      double lambda;
      if (site < 0 || site >= s->ns) return -1;
      while (s->fs_off[f + 1] <= site) ++f;
      if (site - s->fs_off[f] < s->fb_off[f + 1] - s->fb_off[f]) {
        b = site - f;
        lambda = 0.0;
      } else {
        b = site - f - 1;
        lambda = s->bl[b];
      }
      s->xbond[2 * k + a] = b;
      s->xfil[2 * k + a] = f;
      s->xM[2 * k + a] = s->bml[b] + lambda;
    }
  s->nx = n;
  s->xk = k_spring;
  s->xkc = k_spring_compress;
  s->xrest = rest_length;
  return 0;
}

void sco_get_crosslink_forces(const sco_sim *s, double *f) {
  memcpy(f, s->xF, sizeof(double) * 3 * (size_t)s->nx);
}

void sco_pair_forces(sco_sim *s, double *f, double *t) {
  memset(f, 0, sizeof(double) * 3 * s->nb);
  memset(t, 0, sizeof(double) * 3 * s->nb);
  pair_interactions(s, f, t, 0);
}

void sco_get_sites(const sco_sim *s, double *xyz) {
  memcpy(xyz, s->r, sizeof(double) * 3 * s->ns);
}
void sco_get_prev_sites(const sco_sim *s, double *xyz) {
  memcpy(xyz, s->rp, sizeof(double) * 3 * s->ns);
}
void sco_get_site_forces(const sco_sim *s, double *f) {
  memcpy(f, s->F, sizeof(double) * 3 * s->ns);
}
void sco_get_random_forces(const sco_sim *s, double *f) {
  memcpy(f, s->fr, sizeof(double) * 3 * s->ns);
}
void sco_get_bond_ft(const sco_sim *s, double *f, double *t) {
  memcpy(f, s->bF, sizeof(double) * 3 * s->nb);
  memcpy(t, s->bT, sizeof(double) * 3 * s->nb);
}
void sco_get_tensions(const sco_sim *s, double *t) {
  memcpy(t, s->tens, sizeof(double) * s->nb);
}
void sco_get_bond_geom(const sco_sim *s, double *pos, double *spos, double *u,
                       double *len) {
  memcpy(pos, s->bp, sizeof(double) * 3 * s->nb);
  memcpy(spos, s->bs, sizeof(double) * 3 * s->nb);
  memcpy(u, s->bu, sizeof(double) * 3 * s->nb);
  memcpy(len, s->bl, sizeof(double) * s->nb);
}
void sco_get_filament_state(const sco_sim *s, int *sw, int *nn) {
  memcpy(sw, s->fswitch, sizeof(int) * s->nf);
  memcpy(nn, s->fnnorm, sizeof(int) * s->nf);
}
void sco_get_frictions(const sco_sim *s, double *gpar, double *gperp,
                       double *spar, double *sperp) {
  memcpy(gpar, s->gpar, sizeof(double) * s->nf);
  memcpy(gperp, s->gperp, sizeof(double) * s->nf);
  memcpy(spar, s->spar, sizeof(double) * s->nf);
  memcpy(sperp, s->sperp, sizeof(double) * s->nf);
}
long sco_get_pairs(const sco_sim *s, int *out, long cap) {
  long p;
  for (p = 0; p < s->np && p < cap; ++p) {
    out[2 * p] = s->pa[p];
    out[2 * p + 1] = s->pb[p];
  }
  return s->np;
}
void sco_get_bond_cells(const sco_sim *s, int *xyz) {
  int b;
  for (b = 0; b < s->nb; ++b) find_cell_coords(s, V3(s->bs, b), xyz + 3 * b);
}
void sco_get_dr_tot(const sco_sim *s, double *dr) {
  memcpy(dr, s->dt, sizeof(double) * s->ns);
}

void sco_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  sc_philox4x32_10(ctr, key, out);
}

int sco_segment_force(const sco_system *sys, const double *a1, const double *a2,
                      const double *b1, const double *b2, double *force) {
  /* Two one-bond "filaments" are not allowed (at least two bonds), so build
   * the pair geometry directly with the oracle's own routines. */
  sco_sim s;
  double sa[3], sb[3], ua[3], ub[3], pa[3], pb[3], la = 0, lb = 0, t1[3], t2[3];
  double f[3] = {0, 0, 0};
  int i, n = sys->n_dim;
  memset(&s, 0, sizeof(s));
  s.n_dim = n;
  {
    double hh = 2.0 * sys->system_radius;
    int a, b;
    for (a = 0; a < n; ++a)
      for (b = 0; b < n; ++b) s.h[a * n + b] = (a == b ? 1 : 0) * hh;
    s.h[n * n - 1] = hh;
    if (n == 2) invert_sym_2d(s.h, s.hinv);
    else invert_sym_3d(s.h, s.hinv);
  }
  {
    double rcut = pow(2.0, 1.0 / 6.0) * sys->wca_sig;
    s.rcut2 = rcut * rcut;
    s.c12 = 4.0 * sys->wca_eps * pow(sys->wca_sig, 12.0);
    s.c6 = 4.0 * sys->wca_eps * pow(sys->wca_sig, 6.0);
    s.fcut = sys->f_cutoff;
  }
  for (i = 0; i < 3; ++i) ua[i] = ub[i] = pa[i] = pb[i] = sa[i] = sb[i] = 0;
  for (i = 0; i < n; ++i) {
    ua[i] = a2[i] - a1[i];
    la += ua[i] * ua[i];
    ub[i] = b2[i] - b1[i];
    lb += ub[i] * ub[i];
  }
  la = sqrt(la);
  lb = sqrt(lb);
  for (i = 0; i < n; ++i) {
    pa[i] = a1[i] + 0.5 * ua[i];
    pb[i] = b1[i] + 0.5 * ub[i];
    ua[i] /= la;
    ub[i] /= lb;
  }
  periodic_bc(n, s.hinv, pa, sa);
  periodic_bc(n, s.hinv, pb, sb);
  {
    double dr[3] = {0, 0, 0}, c1[3] = {0, 0, 0}, c2[3] = {0, 0, 0}, d2 = 0;
    sphero(&s, sa, ua, la, sb, ub, lb, dr, &d2, c1, c2);
    (void)t1;
    (void)t2;
    if (d2 > s.rcut2) {
      for (i = 0; i < 3; ++i) force[i] = 0;
      return 0;
    }
  }
  /* reuse the pair path with a private two-bond geometry table */
  {
    double bs[6], bu[6], bl[2];
    for (i = 0; i < 3; ++i) {
      bs[i] = sa[i];
      bs[3 + i] = sb[i];
      bu[i] = ua[i];
      bu[3 + i] = ub[i];
    }
    bl[0] = la;
    bl[1] = lb;
    s.bs = bs;
    s.bu = bu;
    s.bl = bl;
    double rdr[3] = {0, 0, 0}, rpote = 0;
    pair_force(&s, 0, 1, f, t1, t2, rdr, &rpote);
  }
  for (i = 0; i < 3; ++i) force[i] = f[i];
  return 1;
}
