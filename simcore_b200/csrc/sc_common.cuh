// Shared device-side definitions of the B200 filament step.
//
// Every kernel translation unit is compiled with --fmad=false: the FP64
// stages reproduce the reference's scalar, contraction-free arithmetic
// operation by operation, which makes them bit-identical to it.  FP32 code
// that wants fused multiply-adds asks for them explicitly (__fmaf_rn).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sc_host_philox.h"

namespace sc {

// The reference's macros (include/simcore/macros.hpp).
__device__ __forceinline__ int nint(double x) {
  return x < 0.0 ? (int)(x - 0.5) : (int)(x + 0.5);
}
__device__ __forceinline__ double dabs(double x) { return x < 0 ? -x : x; }
__device__ __forceinline__ double sign_of(double a, double b) {  // SIGN(a, b)
  return b >= 0.0 ? fabs(a) : -fabs(a);
}
__device__ __forceinline__ int signof(double x) { return x >= 0.0 ? 1 : -1; }

// Programmatic dependent launch (sm_90 and later).  A kernel launched with
// programmatic stream serialization may begin while the kernel before it in
// the stream is still finishing.  grid_dep_sync() blocks the calling thread
// until that kernel, and so every kernel before it, has completed with its
// writes visible, then lets the next kernel in the stream launch: its blocks
// take SM slots as this kernel's retire, and run their own loads of older
// data before they wait in turn.  Every kernel of the step and rebuild
// sequences calls it before its first access to data the kernel just before
// it writes (or reads, for data it writes itself); in a kernel launched
// without the attribute it returns at once.
__device__ __forceinline__ void grid_dep_sync() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Status bits set by kernels; the host maps them to sc_status codes.
enum : unsigned {
  ST_NAN = 1u,            // non-finite position or force
  ST_LIST_OVERFLOW = 2u,  // pair list did not fit
  ST_UNPHYSICAL = 4u,     // accumulated displacement above 10000
  ST_BAD_CELL = 8u,       // cell index out of range (non-finite position)
  ST_BAD_INPUT = 16u,     // caller's device data out of range (site offsets)
  ST_TETHER = 32u         // a crosslink anchor left the bonds it can sit on
};

// Bond geometry for the FP64 pair stage: the reference's Bond state after
// Bond::ReInit (scaled position, unit orientation, length).  64 bytes.
struct __align__(16) BondGeomF64 {
  double s[3];
  double u[3];
  double len;
  double pad;
};

// Bond geometry for the mixed-precision pair stage.  The scaled position is
// stored as 32-bit fixed point q = round(s * 2^32) (s in [-1/2, 1/2]): the
// periodic minimum image of a separation is then the wrapping int32
// difference, exact, with 2^-32 box-length resolution.  32 bytes.
struct __align__(16) BondGeomF32 {
  int32_t q[3];
  float hl;      // half length
  float u[3];
  float pad;
};

// Constants shared by every system of a context (kernel parameter).
struct SysConst {
  int n_dim;
  int n_cells;        // cells of all systems together
  double delta;
  double rcut2;
  double c12, c6, fcut;
  float rcut2f, c12f, c6f, fcutf;
  int stoch;
  int like_like;
  double xk, xkc, xrest;  // crosslink tether: k_spring, k_spring_compress, rest_length
  double eps;             // WCA epsilon (the potential's shift)
  float epsf;
  int thermo;             // pair virial and potential records kept
  float npx_s2;           // mixed: |u1 x u2|^2 below which a side-by-side pair is FP64
};

// One independent periodic system (a replica) of a context: its box, cell
// grid, rebuild threshold and noise key, and where its sites, bonds, cells
// and pairs lie in the context's arrays.  A single-system context has one.
struct ReplicaConst {
  double h[9];        // unit cell (box side 2R on the diagonal), n_dim stride
  double hinv[9];     // its inverse, as the reference computes it
  float hf[9];        // h in FP32 (mixed pair stage)
  int n1d;            // cells per dimension
  int third;          // n1d in 3D, 1 in 2D
  int n_cells;        // n1d^n_dim
  int cell0;          // first cell in the context's cell arrays
  double dr_update;   // rebuild threshold 0.25 cell_length^2
  uint32_t seed;      // Philox key word 0 of this system's noise
  int f0, nf;         // filaments
  int s0, ns;         // sites
  int b0, nb;         // bonds
  int p0, pcap;       // pair segment [p0, p0 + pcap), slots [2 p0, 2 (p0 + pcap))
};

// Per-filament constants of the integrator.  The reciprocals are the
// reference's own quotients (1.0 / friction_par_, 2.0 / friction_perp_, ...,
// src/filament.cpp:783-830, 992-996), evaluated once on the host with the
// same IEEE operations, so every use sees the bits the reference computes
// inline.  112 bytes.
struct FilConst {
  double l, linv, kappa, l2;                   // bond length, 1/l, lp, l*l
  double igpar, igperp, two_igperp, m1_igperp; // 1/g_par, 1/g_perp, 2/g_perp, -1/g_perp
  double dgam;                                 // 1/g_par - 1/g_perp
  double spar, sperp;                          // sqrt(24 g / delta)
  int site0, n;                                // first site, number of sites
  int rep, f_local;                            // system, index within it (noise key)
  int pad0, pad1;
};

// Launch-invariant device pointers of one context.
struct DevState {
  // systems (replicas)
  int nrep;
  const ReplicaConst *rep;  // nrep
  const int *bond_rep;      // nb: system of every bond (null: all in system 0)
  int *due;                 // nrep: pair list rebuilt in the current rebuild pass
  int *np_rep;              // nrep: pairs in each system's segment
  long long *rep_rebuilds;  // nrep: rebuilds per system
  // filaments
  int nf, ns, nb;
  const FilConst *fil;     // nf
  int *f_switch, *f_nnorm;
  const int *site_fil;     // ns
  const int *site_jn;      // ns: site index in its filament | filament sites << 16
  const int *bond_fil;     // nb
  // integrator blocks (filaments longer than a warp): runs of whole filaments
  const int *blk_site0;    // per block: first site
  const int *blk_f0;       // per block: first filament
  const int *blk_nf;       // per block: filament count
  const int *blk_ns;       // per block: site count
  int blk_maxf;            // most filaments in one block (shared-memory size)
  // Equal filaments of blk_uni_n sites, blk_uni_fpb to a block, every block
  // but the last full, sites numbered filament by filament from 0: blocks
  // and sites then find their filaments by arithmetic (0: read the tables).
  int blk_uni_n, blk_uni_fpb;
  // integrator warp groups (filaments of at most 32 sites): runs of whole
  // filaments, one lane per site
  int n_wg;
  const int *wg_site0;     // per group: first site
  const int *wg_f0;        // per group: first filament
  const int *wg_ns;        // per group: site count
  // sites (SoA, 3 components each)
  double *r[3], *rp[3], *fr[3], *dz[3];
  double *dt;
  // bonds
  double *ub[3];           // FP64 orientation of every bond (Bond::orientation_)
  double *bF[3], *bT[3];   // FP64 accumulators (unfused path)
  BondGeomF64 *g64[2];     // double-buffered geometry
  BondGeomF32 *g32[2];
  // pairs
  int *pa, *pb;
  double *pf64;            // stored force per pair, 4 per pair (x, y, z, pad)
  float *pf32;
  int *e_off;              // nb: first slot of each bond's pair entries
  int *e_cnt;              // nb: its number of entries
  int *e_ent;              // entries (pair << 1 | role), sorted by pair per bond
  int *pos1, *pos2;        // slot of each pair's obj1 / obj2 entry
  double *cf64;            // per slot, 8 values: signed force (3), torque (3), pad (2)
  float *cf32;
  // thermo (kept while SysConst::thermo is set): per pair the dr its stress
  // was computed from and its potential, stored with the force
  double *pv64;            // 4 per pair: dr (3), pote
  float *pv32;
  double *th_part;         // per system, th_gx partial virials of 9
  unsigned *th_ticket;     // per system: blocks done in the current launch
  double *th_acc;          // per system: accumulated virial (9)
  long long *th_istep;     // per system: steps accumulated (the reference's i_step)
  long long *th_nrec;      // per system: records written
  double *th_rec;          // ring of th_cap records per system: i_step, tensor (9), pressure, volume
  int th_cap, th_gx, th_n;
  // static crosslinks (harmonic tethers between two bonds)
  int nx;                  // links
  const int *xl_fil;       // 2 per link: filament of each anchor
  double *xl_M;            // 2 per link: mesh lambda of each anchor (Anchor::mesh_lambda_)
  double *xl_c;            // 8 per anchor: force (3), torque (3), its bond, pad
  double *xl_F;            // 4 per link: tether force (Crosslink::force_), pad
  const int *xb_off;       // nb+1 CSR of anchors per bond
  const int *xb_ent;       // anchor ids (2 link + a), ascending per bond: an anchor is
                           // listed on the bond it was attached to and on both of its
                           // neighbours, and counts on the one it sits on
  double *bml;             // nb: mesh lambda of every bond (Bond::mesh_lambda_)
  double *ftl;             // nf: summed current bond lengths (Mesh::true_length_)
  const double *fil_L;     // nf: nominal filament length (Mesh::length_)
  // capture (optional)
  double *cap_F[3];
  double *cap_T;
  // status / control (device-resident so captured graphs need no host state)
  unsigned *status;
  unsigned long long *dr_max_bits;  // nrep: displacement maximum per system
  unsigned long long *mcount;  // midsteps that drew noise (Philox draw offset)
  long long *n_rebuilds;       // rebuild passes (any system)
  int *loop_count;             // remaining BD steps of a graph launch
  int pcap_total;              // pair slots of all segments
};

__device__ __forceinline__ int rep_of_bond(const DevState &d, int b) {
  return d.bond_rep ? d.bond_rep[b] : 0;
}

}  // namespace sc
