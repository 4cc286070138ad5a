// Cell-list helpers shared by the rebuild pipelines (sc_kernels.cu for the
// caller-scratch entry point, sc_rebuild.cu for contexts): bond cells,
// exclusion rule, half-shell neighbours (CellList + Cell, src/cell_list.cpp,
// src/cell.cpp, src/interaction_manager.cpp).
#pragma once

#include "sc_common.cuh"
#include "sc_step.cuh"

namespace sc {

// CellList::FindCellCoords (src/cell_list.cpp:139-157) on the bond's scaled
// position, recomputed exactly from its sites; the cell index within the
// bond's system.
template <int ND>
__device__ __forceinline__ int bond_cell(const DevState &d, const ReplicaConst &R, int b,
                                         int *xyz) {
  int f = d.bond_fil[b];
  int site = b + f;
  double r1[3], r2[3], s[3], u[3], len;
  for (int i = 0; i < 3; ++i) {
    r1[i] = d.r[i][site];
    r2[i] = d.r[i][site + 1];
  }
  bond_from_sites<ND>(R.hinv, r1, r2, s, u, len);
  int c[3] = {0, 0, 0};
  bool bad = false;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    double x = s[i] + 0.5;
    double fl = floor(R.n1d * x);
    int cc = (fl >= 0.0 && fl <= (double)R.n1d) ? (int)fl : -1;
    if (cc == R.n1d) cc -= 1;
    if (cc < 0) {
      bad = true;
      cc = 0;
    }
    c[i] = cc;
  }
  if (bad) atomicOr(d.status, ST_BAD_CELL);
  xyz[0] = c[0];
  xyz[1] = c[1];
  xyz[2] = c[2];
  return (c[0] * R.n1d + c[1]) * R.third + c[2];
}

// Pairs that ProcessPairInteraction marks no_interaction and the first
// evaluation after a rebuild culls (src/interaction_manager.cpp:341-367,
// 485-497): all pairs without like-like interactions, and bonds of one
// filament that share a site (Bond::HasNeighbor, src/bond.cpp:118-121).
__device__ __forceinline__ bool pair_excluded(const SysConst &k,
                                              const DevState &d, int a, int b) {
  if (!k.like_like) return true;
  // Adjacent indices first: the filaments are read only for those.
  const int diff = a - b;
  if (diff > 1 || diff < -1) return false;
  return d.bond_fil[a] == d.bond_fil[b];
}

// Half-shell neighbour cells of (x, y, z) in the order of
// CellList::AssignCellNeighbors(false) (src/cell_list.cpp:206-262), as
// indices within the system, without compaction: entry kk (a compile-time
// index) is the kk-th candidate of its loops -- (x+1, y, z); (x-1..x+1,
// y+1, z); then, in 3D, (x-1..x+1, y-1..y+1, z+1), x fastest -- with
// periodic wrap, and bit kk of the returned mask says it is kept (it is not
// the cell itself, which wrap can give on small grids).  Visiting the set
// bits in order visits the reference's neighbour list in its order, with
// every index in registers.
__device__ __forceinline__ unsigned half_shell_fixed(const SysConst &k, const ReplicaConst &R,
                                                     int x, int y, int z, int out[13]) {
  const int n1d = R.n1d;
  unsigned mask = 0;
#pragma unroll
  for (int kk = 0; kk < 13; ++kk) {
    const int dz = kk < 4 ? 0 : 1;
    const int dy = kk == 0 ? 0 : (kk < 4 ? 1 : (kk - 4) / 3 - 1);
    const int dx = kk == 0 ? 1 : (kk < 4 ? kk - 2 : (kk - 4) % 3 - 1);
    int nx = x + dx, ny = y + dy, nz = z + dz;
    if (nx < 0) nx = n1d - 1;
    else if (nx == n1d) nx = 0;
    if (ny < 0) ny = n1d - 1;
    else if (ny == n1d) ny = 0;
    if (nz == n1d) nz = 0;
    out[kk] = (nx * n1d + ny) * R.third + nz;
    const bool keep = (kk < 4 || k.n_dim == 3) && !(nx == x && ny == y && nz == z);
    mask |= keep ? (1u << kk) : 0u;
  }
  return mask;
}

__device__ __forceinline__ void cell_coords(const ReplicaConst &R, int c, int &x, int &y,
                                            int &z) {
  z = c % R.third;
  int t = c / R.third;
  y = t % R.n1d;
  x = t / R.n1d;
}

// Whether cell c holds a bond, from the occupancy bits the cell scan wrote
// (a small array that stays in cache, unlike the cell offsets); without
// them, every cell is looked up.
__device__ __forceinline__ bool cell_occupied(const unsigned *occ, int c) {
  return !occ || ((occ[c >> 5] >> (c & 31)) & 1u);
}

// Pairs of rebuilt system r: the span of its cells' offsets.  A list longer
// than its segment sets the overflow bit (the count is kept so the host can
// size the segment).
__device__ __forceinline__ void rep_pairs(const DevState &d, int r, const int *cell_start,
                                          const int *pair_off) {
  if (!d.due[r]) return;
  const ReplicaConst &R = d.rep[r];
  const int np = pair_off[cell_start[R.cell0 + R.n_cells]] - pair_off[cell_start[R.cell0]];
  d.np_rep[r] = np;
  if (np > R.pcap) atomicOr(d.status, ST_LIST_OVERFLOW);
}

// System of pair slot p (the segment that holds it).
__device__ __forceinline__ int rep_of_pair(const DevState &d, int p) {
  int lo = 0, hi = d.nrep - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d.rep[mid].p0 <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Slot p holds a current pair of its system.
__device__ __forceinline__ bool pair_live(const DevState &d, int p, int &r) {
  r = rep_of_pair(d, p);
  const ReplicaConst &R = d.rep[r];
  const int local = p - R.p0;
  return local < R.pcap && local < d.np_rep[r];
}

}  // namespace sc
