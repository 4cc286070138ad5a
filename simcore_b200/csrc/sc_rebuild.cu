// Pair-list rebuild of a context (InteractionManager::UpdateInteractions,
// src/interaction_manager.cpp:211-231, over CellList::MakePairs,
// src/cell_list.cpp:139-199, and Cell::MakePairs, src/cell.cpp:14-70).
//
// The bonds of the rebuilt systems are sorted by cell with a two-level
// (most-significant-digit first) radix sort on the cell key: a counting pass
// on the high digits -- the group of 32 consecutive cells, one occupancy word
// -- and then, inside every group, each bond's rank by (cell, bond id).  The
// ranking keeps every cell's bonds in bond order, the order in which
// Cell::AddObj appends them.  The counting pass scans one counter per group
// (n_cells / 32 of them), not the cell grid; cell ranges and occupancy bits
// are written where cells start and end in the sorted order.
//
//   k_rb_keys      ZeroDrTot and the rebuild counters; cell key of every
//                  bond, group counts; clears the occupancy words and the
//                  per-bond entry counts of the rebuilt systems
//   (scan)         group offsets
//   k_rb_scatter   bonds into their groups (counts back to zero)
//   k_rb_rank      stable order inside each group; cell ranges and bits
//   k_rb_count     each cell's pairs in the reference's order, as candidates
//                  (one reservation per block), their count at the cell's
//                  head entry, per-bond entry counts
//   (scan)         pair offsets and entry offsets, one scan of both
//   k_rb_place     candidates to their list slots, stored forces zeroed,
//                  per-bond entries (pair << 1 | role)
//   k_rb_csr_sort  entries in pair order, slots of both roles, ranges
#include <cuda_runtime.h>

#include "sc_cells.cuh"
#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_launch.h"

namespace sc {

// Bonds of the rebuilt systems: cell key (system's first cell + cell within
// it) and warp-aggregated group counts; others get the sentinel n_cells.
// Clears the occupancy words of the rebuilt systems (each system's cells
// start at a multiple of 32: a word, a group, belongs to one system).
template <int ND>
__global__ void __launch_bounds__(256) k_rb_keys(SysConst k, DevState d, RebuildBufs rb) {
  grid_dep_sync();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  // InteractionManager::ZeroDrTot (src/interaction_manager.cpp:316-321) for
  // the rebuilt systems, and the rebuild counters (nothing in the rebuild
  // reads or moves the sites).
  if (tid == 0) {
    *d.n_rebuilds += 1;
    *rb.cand_n = 0;
  }
  for (int r = tid; r < d.nrep; r += nthreads) {
    if (!d.due[r]) continue;
    d.dr_max_bits[r] = 0ull;
    d.rep_rebuilds[r] += 1;
  }
  for (int i = tid; i < d.ns; i += nthreads) {
    // (One system is always due when its rebuild runs: no lookup.)
    if (d.nrep > 1 && !d.due[d.fil[d.site_fil[i]].rep]) continue;
    d.dz[0][i] = d.r[0][i];
    d.dz[1][i] = d.r[1][i];
    d.dz[2][i] = d.r[2][i];
    d.dt[i] = 0.0;
  }
  for (int r = 0; r < d.nrep; ++r) {
    if (!d.due[r]) continue;
    const ReplicaConst &R = d.rep[r];
    const int w0 = R.cell0 >> 5, w1 = (R.cell0 + R.n_cells + 31) >> 5;
    for (int w = w0 + tid; w < w1; w += nthreads) rb.occ[w] = 0u;
  }
  const int b = tid;
  bool in = false;
  int g = 0;
  if (b < d.nb) {
    uint32_t c = (uint32_t)k.n_cells;
    const int r = rep_of_bond(d, b);
    if (d.due[r]) {
      rb.deg[b] = 0;
      const ReplicaConst &R = d.rep[r];
      int xyz[3];
      c = (uint32_t)(R.cell0 + bond_cell<ND>(d, R, b, xyz));
      in = true;
      g = (int)(c >> 5);
    }
    rb.key[b] = c;
  }
  const unsigned mask = __ballot_sync(0xffffffffu, in);
  if (in) {
    const unsigned peers = __match_any_sync(mask, g);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&rb.gcount[g], __popc(peers));
  }
}

// Each rebuilt bond into its group's range of the scanned offsets (any
// order inside the group); decrements the counts back to zero, ready for
// the next rebuild.
__global__ void k_rb_scatter(DevState d, RebuildBufs rb) {
  grid_dep_sync();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb || !d.due[rep_of_bond(d, b)]) return;
  const int g = (int)(rb.key[b] >> 5);
  const int slot = atomicSub(&rb.gcount[g], 1) - 1;
  rb.tmp[rb.gstart[g] + slot] = b;
}

// Sorted position of every rebuilt bond: its group's first entry plus the
// number of bonds of the group that come before it by (cell, bond id).  The
// first of a cell writes the cell's start and occupancy bit, the last its
// end.
__global__ void k_rb_rank(DevState d, RebuildBufs rb) {
  grid_dep_sync();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= rb.gstart[rb.n_groups]) return;
  const int b = rb.tmp[q];
  const uint32_t c = rb.key[b];
  const int g = (int)(c >> 5);
  const int s = rb.gstart[g], e = rb.gstart[g + 1];
  int rank = 0;
  bool first = true, last = true;
  for (int j = s; j < e; ++j) {
    const int bj = rb.tmp[j];
    const uint32_t cj = rb.key[bj];
    rank += (cj < c || (cj == c && bj < b)) ? 1 : 0;
    if (cj == c) {
      first = first && !(bj < b);
      last = last && !(bj > b);
    }
  }
  const int pos = s + rank;
  rb.skey[pos] = c;
  rb.sval[pos] = b;
  if (first) {
    rb.range[c].x = pos;
    atomicOr(&rb.occ[c >> 5], 1u << (c & 31));
  }
  if (last) rb.range[c].y = pos + 1;
}

__device__ __forceinline__ bool occupied(const unsigned *occ, int c) {
  return (occ[c >> 5] >> (c & 31)) & 1u;
}

// Sorted span [lo, hi) of system R's bonds: its groups' entries.
__device__ __forceinline__ int sys_lo(const RebuildBufs &rb, const ReplicaConst &R) {
  return rb.gstart[R.cell0 >> 5];
}
__device__ __forceinline__ int sys_hi(const RebuildBufs &rb, const ReplicaConst &R) {
  return rb.gstart[(R.cell0 + R.n_cells + 31) >> 5];
}

// The cell whose head is sorted entry q: its m members, its half-shell
// neighbours (context cell indices; -1 where the wrap gives the cell itself
// or, in 2D, a third dimension) and their sorted ranges (empty where
// unoccupied), and the mask of non-empty neighbours.
struct CellHead {
  int c, m;
  const int *it;
  int nbr[13], s0[13], s1[13];
  unsigned busy;
};

__device__ __forceinline__ void cell_head(const SysConst &k, const RebuildBufs &rb,
                                          const ReplicaConst &R, int q, int c, CellHead &h) {
  h.c = c;
  h.m = rb.range[c].y - q;
  h.it = rb.sval + q;
  int x, y, z;
  cell_coords(R, c - R.cell0, x, y, z);
  const unsigned keep = half_shell_fixed(k, R, x, y, z, h.nbr);
  h.busy = 0;
#pragma unroll
  for (int kk = 0; kk < 13; ++kk) {  // all ranges loaded together
    h.s0[kk] = h.s1[kk] = 0;
    h.nbr[kk] += R.cell0;
    if ((keep >> kk) & 1u) {
      if (occupied(rb.occ, h.nbr[kk])) {
        const int2 g = rb.range[h.nbr[kk]];
        h.s0[kk] = g.x;
        h.s1[kk] = g.y;
        h.busy |= 1u << kk;
      }
    } else {
      h.nbr[kk] = -1;  // matches no cell key
    }
  }
}

// Calls f(a, b) for the cell's pairs in the reference's list order
// (Cell::MakePairs, src/cell.cpp:14-22): pairs inside the cell, then with
// each half-shell neighbour in order, less those pair_excluded drops.  Only
// the non-empty neighbours are visited (a warp steps through as many as its
// busiest lane has, not all 13).
template <class F>
__device__ __forceinline__ void cell_pairs_visit(const SysConst &k, const DevState &d,
                                                 const RebuildBufs &rb, const CellHead &h,
                                                 F &&f) {
  const int m = h.m;
  for (int i = 0; i < m - 1; ++i)
    for (int j = i + 1; j < m; ++j) {
      const int a = h.it[i], b = h.it[j];
      if (!pair_excluded(k, d, a, b)) f(a, b);
    }
  unsigned busy = h.busy;
  while (busy) {
    const int kk = __ffs(busy) - 1;
    busy &= busy - 1;
    int lo = 0, hi = 0;
#pragma unroll
    for (int q2 = 0; q2 < 13; ++q2)
      if (q2 == kk) {
        lo = h.s0[q2];
        hi = h.s1[q2];
      }
    for (int i = 0; i < m; ++i)
      for (int j = lo; j < hi; ++j) {
        const int a = h.it[i], b = rb.sval[j];
        if (!pair_excluded(k, d, a, b)) f(a, b);
      }
  }
}

// Each cell's pairs, found once: the head entry of a cell collects them (the
// first kHeadBuf in shared memory, all again in the rare longer case), takes
// a run of candidate slots from one reservation per block, and writes them
// there in order; it records their count (0 at the other entries) and adds
// each pair to both bonds' entry counts.  Candidates past cand_cap are
// dropped: their system's list then outgrows its segment, which k_rb_place
// reports.
constexpr int kCountBlock = 128;
constexpr int kHeadBuf = 8;

__global__ void __launch_bounds__(kCountBlock) k_rb_count(SysConst k, DevState d, RebuildBufs rb) {
  __shared__ int2 sbuf[kCountBlock][kHeadBuf];
  __shared__ int swarp[kCountBlock / 32];
  grid_dep_sync();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = threadIdx.x, lane = t & 31;
  int cnt = 0;
  const ReplicaConst *R = nullptr;
  int c = 0;
  if (q < d.nb && q < rb.gstart[rb.n_groups] && k.like_like) {
    c = (int)rb.skey[q];
    if (q == 0 || (int)rb.skey[q - 1] != c) {
      R = &d.rep[d.nrep > 1 ? rep_of_bond(d, rb.sval[q]) : 0];
      CellHead h;
      cell_head(k, rb, *R, q, c, h);
      cell_pairs_visit(k, d, rb, h, [&](int a, int b) {
        if (cnt < kHeadBuf) sbuf[t][cnt] = make_int2(a, b);
        atomicAdd(&rb.deg[a], 1);
        atomicAdd(&rb.deg[b], 1);
        ++cnt;
      });
    }
  }
  // The block's candidate slots: a scan of the counts, one atomic.
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) swarp[t >> 5] = incl;
  __syncthreads();
  if (t == 0) {
    int run = 0;
#pragma unroll
    for (int w = 0; w < kCountBlock / 32; ++w) {
      const int v = swarp[w];
      swarp[w] = run;
      run += v;
    }
    const int base = run > 0 ? atomicAdd(rb.cand_n, run) : 0;
#pragma unroll
    for (int w = 0; w < kCountBlock / 32; ++w) swarp[w] += base;
  }
  __syncthreads();
  const int t0 = swarp[t >> 5] + incl - cnt;
  if (cnt > 0 && cnt <= kHeadBuf) {
    for (int i = 0; i < cnt; ++i)
      if (t0 + i < rb.cand_cap) rb.cand[t0 + i] = make_int4(sbuf[t][i].x, sbuf[t][i].y, q, 0);
  } else if (cnt > kHeadBuf) {
    CellHead h;
    cell_head(k, rb, *R, q, c, h);
    int i = 0;
    cell_pairs_visit(k, d, rb, h, [&](int a, int b) {
      if (t0 + i < rb.cand_cap) rb.cand[t0 + i] = make_int4(a, b, q, 0);
      ++i;
    });
  }
  if (q < d.nb) {
    rb.pair_count[q] = cnt;
    rb.cand_start[q] = t0;
  }
}

// First entry slot of bond b (rebuilt system R): its system's slots start at
// 2 p0, its bonds' entries follow in bond order.
__device__ __forceinline__ int entry_first(const RebuildBufs &rb, const ReplicaConst &R, int b) {
  return 2 * R.p0 + (rb.deg_off[b] - rb.deg_off[R.b0]);
}

// Every candidate to its slot -- its cell's scanned offset in its system's
// pair segment plus its place among the cell's candidates (slots past the
// segment are not written) -- with the new pair's stored force (and virial
// record) zeroed and both of its per-bond entries (pair << 1 | role; role 0
// = obj1, 1 = obj2) in any order, the entry counts going back to zero.  A
// system whose list outgrew its segment gets no entries: its step stops on
// the overflow bit and is redone.  Threads u < nrep record their system's
// pair count (the count is kept so the host can size the segment).
__global__ void k_rb_place(DevState d, RebuildBufs rb, int prec) {
  grid_dep_sync();
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < d.nrep && d.due[u]) {
    const ReplicaConst &R = d.rep[u];
    const int np = rb.pair_off[sys_hi(rb, R)] - rb.pair_off[sys_lo(rb, R)];
    d.np_rep[u] = np;
    if (np > R.pcap) atomicOr(d.status, ST_LIST_OVERFLOW);
  }
  if (u >= min(*rb.cand_n, rb.cand_cap)) return;
  const int4 e = rb.cand[u];
  const int q = e.z;
  const ReplicaConst &R = d.rep[d.nrep > 1 ? rep_of_bond(d, e.x) : 0];
  const int lo = rb.pair_off[sys_lo(rb, R)];
  const bool fits = rb.pair_off[sys_hi(rb, R)] - lo <= R.pcap;
  const int p = rb.pair_off[q] - lo + (u - rb.cand_start[q]);
  if (p < R.pcap) {
    const int g = R.p0 + p;
    d.pa[g] = e.x;
    d.pb[g] = e.y;
    if (prec == 0) {
      double2 *st = reinterpret_cast<double2 *>(d.pf64) + 2 * (size_t)g;
      st[0] = make_double2(0.0, 0.0);
      st[1] = make_double2(0.0, 0.0);
      if (d.pv64) {  // a new Interaction's stress and potential are 0
        double2 *v = reinterpret_cast<double2 *>(d.pv64) + 2 * (size_t)g;
        v[0] = make_double2(0.0, 0.0);
        v[1] = make_double2(0.0, 0.0);
      }
    } else {
      reinterpret_cast<float4 *>(d.pf32)[g] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (d.pv32) reinterpret_cast<float4 *>(d.pv32)[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (fits) {
      const int sa = atomicSub(&rb.deg[e.x], 1) - 1;
      const int sb = atomicSub(&rb.deg[e.y], 1) - 1;
      d.e_ent[entry_first(rb, R, e.x) + sa] = g << 1;
      d.e_ent[entry_first(rb, R, e.y) + sb] = (g << 1) | 1;
    }
  }
}

// Each bond's entries sorted by pair index -- the order in which the
// reference's serial ApplyPairInteractions adds them to the bond -- in
// registers up to kRegEntries of them; the slot of each (pair, role)
// entry; the bond's entry range.
constexpr int kRegEntries = 16;

__global__ void k_rb_csr_sort(DevState d, RebuildBufs rb) {
  grid_dep_sync();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  const int r = rep_of_bond(d, b);
  if (!d.due[r]) return;
  const ReplicaConst &R = d.rep[r];
  if (d.np_rep[r] > R.pcap) return;  // outgrew its segment: no entries
  const int e0 = entry_first(rb, R, b), n = rb.deg_off[b + 1] - rb.deg_off[b];
  d.e_off[b] = e0;
  d.e_cnt[b] = n;
  int *e = d.e_ent + e0;
  if (n <= kRegEntries) {
    int v[kRegEntries];
#pragma unroll
    for (int i = 0; i < kRegEntries; ++i) v[i] = i < n ? e[i] : 0x7fffffff;
    // Odd-even transposition sort: kRegEntries rounds sort kRegEntries keys.
#pragma unroll
    for (int round = 0; round < kRegEntries; ++round) {
#pragma unroll
      for (int i = round & 1; i + 1 < kRegEntries; i += 2) {
        const int lo = min(v[i], v[i + 1]), hi = max(v[i], v[i + 1]);
        v[i] = lo;
        v[i + 1] = hi;
      }
    }
#pragma unroll
    for (int i = 0; i < kRegEntries; ++i) {
      if (i < n) {
        e[i] = v[i];
        if (v[i] & 1) d.pos2[v[i] >> 1] = e0 + i;
        else d.pos1[v[i] >> 1] = e0 + i;
      }
    }
    return;
  }
  for (int i = 1; i < n; ++i) {
    const int v = e[i];
    int j = i - 1;
    while (j >= 0 && e[j] > v) {
      e[j + 1] = e[j];
      --j;
    }
    e[j + 1] = v;
  }
  for (int i = 0; i < n; ++i) {
    const int ent = e[i];
    if (ent & 1) d.pos2[ent >> 1] = e0 + i;
    else d.pos1[ent >> 1] = e0 + i;
  }
}


int launch_rebuild(const SysConst &k, const DevState &d, const RebuildBufs &rb, int prec,
                   cudaStream_t st, bool first_in_graph) {
  int launched = 0;
  const int nb = d.nb > 0 ? d.nb : 1;
  const int g256 = (nb + 255) / 256;
  if (first_in_graph) {
    // Captured, the first kernel starts the conditional body: no kernel
    // before it to overlap.
    PdlOff off;
    if (k.n_dim == 3) launch_pdl(k_rb_keys<3>, dim3(g256), dim3(256), 0, st, k, d, rb);
    else launch_pdl(k_rb_keys<2>, dim3(g256), dim3(256), 0, st, k, d, rb);
  } else {
    if (k.n_dim == 3) launch_pdl(k_rb_keys<3>, dim3(g256), dim3(256), 0, st, k, d, rb);
    else launch_pdl(k_rb_keys<2>, dim3(g256), dim3(256), 0, st, k, d, rb);
  }
  ++launched;
  launched += launch_exclusive_scan(rb.gcount, rb.gstart, rb.n_groups, rb.scan_tmp, st);
  launch_pdl(k_rb_scatter, dim3(g256), dim3(256), 0, st, d, rb);
  launch_pdl(k_rb_rank, dim3(g256), dim3(256), 0, st, d, rb);
  const int gc = (nb + kCountBlock - 1) / kCountBlock;
  launch_pdl(k_rb_count, dim3(gc), dim3(kCountBlock), 0, st, k, d, rb);
  // pair_count and deg are one array of 2 nb (pair_off and deg_off alike).
  launched += 3 + launch_exclusive_scan(rb.pair_count, rb.pair_off, 2LL * d.nb, rb.scan_tmp, st);
  const int cap = rb.cand_cap > d.nrep ? rb.cand_cap : d.nrep;
  launch_pdl(k_rb_place, dim3((cap + 255) / 256), dim3(256), 0, st, d, rb, prec);
  launch_pdl(k_rb_csr_sort, dim3(g256), dim3(256), 0, st, d, rb);
  return launched + 2;
}

}  // namespace sc
