// Host-side launchers of the device kernels (sc_kernels.cu).  Each returns
// the number of kernels it launched.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "sc_common.cuh"

namespace sc {

// Bond geometry of the current sites (Bond::ReInit) into record buffer buf;
// write_ub also sets the FP64 bond orientations (loading positions), which
// the FP64 scratch record of mixed precision must leave alone.
void launch_init_geometry(const SysConst &k, const DevState &d, int buf,
                          int prec, cudaStream_t st, bool write_ub = true);
int scan_temp_ints(long long n);
// Analyses per system: end-to-end sums and joint-angle histograms
// (accumulated), polar and nematic order (12 doubles per system).
int launch_analysis_sample(const SysConst &k, const DevState &d, int n_bins, int max_joints,
                           double *acc, int *hist, cudaStream_t st);
int launch_global_order(const SysConst &k, const DevState &d, double *out, cudaStream_t st);
// Diffusion analysis: one sample at window point t of every system's MSD and
// orientation correlation, from the filament averages avg; restart replaces
// the origins pos0 / u0 with the current averages.
int launch_diffusion_sample(const SysConst &k, const DevState &d, const double *avg,
                            double *pos0, double *u0, double *acc, int t, int interval,
                            int restart, cudaStream_t st);
// Diffusion origins (average position and orientation, 3 each per filament)
// from the filament averages.
int launch_aos_to_origins(int nf, const double *avg, double *pos0, double *u0,
                          cudaStream_t st);
// Per filament average position, its scaled image and average orientation
// (9 doubles each).
int launch_filament_averages(const SysConst &k, const DevState &d, double *out, cudaStream_t st);
// Interleaved x, y, z triples into positions and previous positions.
int launch_aos_to_soa(int n, int nd, const double *aos, const DevState &d, cudaStream_t st);
// Component arrays into interleaved triples.
template <class T>
int launch_soa_to_aos(int n, const T *x, const T *y, const T *z, double *aos, cudaStream_t st);
// With occ, also one bit per element (set where it is non-zero), 32 to a word.
int launch_exclusive_scan(const int *in, int *out, long long n, int *tmp,
                          cudaStream_t st, unsigned *occ = nullptr);
int launch_bin_count(const SysConst &k, const DevState &d, int *key,
                     int *cell_count, cudaStream_t st);
int launch_bond_cells(const SysConst &k, const DevState &d, int *xyz,
                      cudaStream_t st);
// The rebuild pass covers the systems flagged in d.due; bonds of other
// systems are skipped and keep their lists.
int launch_bin_scatter(const DevState &d, const int *key, const int *cell_start,
                       int *cell_count, int *sorted, cudaStream_t st);
// occ: the cell scan's occupancy bits (null: look every neighbour cell up).
int launch_cell_sort_count(const SysConst &k, const DevState &d, const int *key,
                           int *sorted, const int *cell_start, int *pair_count,
                           cudaStream_t st, const unsigned *occ = nullptr);
// Emits the pairs into the systems' segments and records each system's count.
int launch_pair_emit(const SysConst &k, const DevState &d, const int *key,
                     const int *sorted, const int *cell_start,
                     const int *pair_off, int *deg, int prec,
                     cudaStream_t st, const unsigned *occ = nullptr);
// Per-bond entry lists; deg_off is the exclusive scan of deg over all bonds.
int launch_csr(const DevState &d, int *deg, const int *deg_off, cudaStream_t st);
// Scratch of a context's rebuild (sc_rebuild.cu).  Sizes: key, tmp, skey,
// sval, pair_count, deg: nb; gcount: n_groups; gstart: n_groups + 1;
// pair_off, deg_off: nb + 1; range: n_cells; occ: n_groups words;
// scan_tmp: scan_temp_ints(max(n_groups, nb)).  gcount, deg, range and occ
// start zeroed.
struct RebuildBufs {
  int n_groups;        // groups of 32 cells: n_cells / 32 (each system's cells
                       // start at a multiple of 32)
  uint32_t *key;       // cell key of every bond, bond order (n_cells: not rebuilt)
  int *gcount;         // bonds per group (zero between rebuilds)
  int *gstart;         // first sorted entry of each group
  int *tmp;            // bonds by group, any order inside a group
  uint32_t *skey;      // sorted cell keys
  int *sval;           // sorted bond ids
  int2 *range;         // per cell: [start, end) in the sorted order
  unsigned *occ;       // per cell: occupied in the last rebuild of its system
  // Per sorted entry: the pairs of the cell it heads (0 elsewhere), then per
  // bond its pair entries; one array of 2 nb, scanned as one into 2 nb + 1
  // offsets (pair_count = counts, deg = counts + nb; pair_off = offsets,
  // deg_off = offsets + nb, shifted by the pair total, which cancels in
  // every use).
  int *pair_count, *pair_off;
  int *deg, *deg_off;
  int *scan_tmp;
  // Candidate pairs (a, b, head entry, -), each cell head's at
  // cand_start[entry], in the reference's order; cand_cap = the pair slots of
  // all segments.
  int4 *cand;
  int cand_cap;
  int *cand_n;         // slots taken in the current rebuild
  int *cand_start;     // per sorted entry
};
// The whole rebuild of the systems flagged in d.due; returns the kernels
// launched.  first_in_graph: the first kernel opens a captured conditional
// body (launched without the programmatic-dependence attribute).
int launch_rebuild(const SysConst &k, const DevState &d, const RebuildBufs &rb, int prec,
                   cudaStream_t st, bool first_in_graph);
// Graph loop control: the head sets the WHILE condition h and, with
// `decide`, the first step's rebuild decision (IF condition h_if); the tail
// ends a BD step and decides the next step's rebuild.
int launch_loop_head(const DevState &d, cudaGraphConditionalHandle h,
                     cudaGraphConditionalHandle h_if, int decide, cudaStream_t st);
int launch_loop_tail(const DevState &d, int stoch, cudaGraphConditionalHandle h,
                     cudaGraphConditionalHandle h_if, int decide, cudaStream_t st);
int launch_advance_mcount(const DevState &d, cudaStream_t st);
int launch_zero_dr(const DevState &d, cudaStream_t st);
// Grid sized for `expected` pairs (one system) or every slot (several); the
// kernel strides over the actual pairs.  block: threads per block, 128 or 256
// (the autotuner's choice).
// npx (mixed only): nearly parallel pairs are evaluated in FP64 from the
// sites, in place.  The kernel loads the pair list and slot indices before
// it waits on the kernel launched just before it (programmatic dependent
// launch): that kernel must not write them -- the last kernel of a rebuild
// does not -- or the launch must be made without the overlap (PdlOff).
int launch_pairs(const SysConst &k, const DevState &d, int rbuf, int prec,
                 int expected, cudaStream_t st, bool npx = false, int block = 256);
// Crosslink tethers of an even step into the per-anchor contributions.
int launch_tether(const SysConst &k, const DevState &d, cudaStream_t st);
// Thermo: one step's pair virial per system, the pressure record every
// th_n steps (grid th_gx x systems).
int launch_thermo(const SysConst &k, const DevState &d, int prec, cudaStream_t st);
// Potential energy of every filament from the pair records.
int launch_potential(const DevState &d, int prec, double *out, cudaStream_t st);
int launch_bond_sum(const SysConst &k, const DevState &d, int prec, cudaStream_t st);
size_t integrate_smem_bytes(int C, int max_filaments);
void prepare_integrate(int C);
// fast: the contraction/reciprocal variant (mixed precision only).
// fuse (fast mixed only): the integrator evaluates the pairs itself, in place
// of the pair stage (launch_pairs is then not launched for the step).
int launch_integrate(const SysConst &k, const DevState &d, int nblocks, int C,
                     int midstep, int rbuf, int interaction, int capture,
                     int prec, bool fast, cudaStream_t st, bool fuse = false);
void prepare_integrate_fast(int C);
int launch_integrate_fast(const SysConst &k, const DevState &d, int nblocks, int C,
                          int midstep, int rbuf, int interaction, int capture,
                          cudaStream_t st, bool fuse);

}  // namespace sc
