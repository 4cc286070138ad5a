// Device kernels of the B200 filament step.  Compiled with --fmad=false
// (see sc_common.cuh).
//
//   cell list      k_bin_count, k_bin_scatter, k_cell_sort, k_cell_count,
//                  k_pair_emit   (CellList + Cell, src/cell_list.cpp,
//                                 src/cell.cpp)
//   pair CSR       k_csr_fill, k_csr_sort (per-bond pair entries in list
//                  order, for the reference's serial scatter order)
//   pair forces    k_pairs       (InteractionManager::CalculatePairInteractions
//                                 + ApplyPairInteractions)
//   integrator     k_integrate   (Filament::UpdatePosition for every
//                                 filament; FUSED also runs the pair stage)
//   utilities      exclusive scan, geometry init, displacement reset.
#include <cuda_runtime.h>

#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_pair.cuh"

namespace sc {

// ---------------------------------------------------------------------------
// Bond geometry from two sites: Bond::ReInit (src/bond.cpp:22-37) followed by
// Object::UpdatePeriodic / periodic_boundary_conditions
// (src/object.cpp:202-210, src/linear_algebra.cpp:100-117).
template <int ND>
__device__ __forceinline__ void bond_from_sites(const SysConst &k,
                                                const double *r1,
                                                const double *r2, double s[3],
                                                double u[3], double &len) {
  double pos[3] = {0, 0, 0};
  u[0] = u[1] = u[2] = 0.0;
  s[0] = s[1] = s[2] = 0.0;
  len = 0;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    u[i] = r2[i] - r1[i];
    len += u[i] * u[i];
  }
  len = sqrt(len);
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    pos[i] = r1[i] + 0.5 * u[i];
    u[i] /= len;
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    s[i] = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) s[i] += k.hinv[ND * i + j] * pos[j];
    s[i] -= nint(s[i]);
  }
}

__device__ __forceinline__ int32_t to_fixed(double s) {
  // s in [-1/2, 1/2]: round(s * 2^32) wraps into int32 (1/2 and -1/2 map to
  // the same point of the periodic box).
  long long q = __double2ll_rn(s * 4294967296.0);
  return (int32_t)(uint32_t)(unsigned long long)q;
}

template <int ND>
__device__ __forceinline__ void store_geom(const DevState &d, int buf, int b,
                                           const double s[3],
                                           const double u[3], double len,
                                           int prec) {
  if (prec == 0) {
    BondGeomF64 g;
    g.s[0] = s[0];
    g.s[1] = s[1];
    g.s[2] = s[2];
    g.u[0] = u[0];
    g.u[1] = u[1];
    g.u[2] = u[2];
    g.len = len;
    g.pad = 0.0;
    d.g64[buf][b] = g;
  } else {
    BondGeomF32 g;
    g.q[0] = to_fixed(s[0]);
    g.q[1] = to_fixed(s[1]);
    g.q[2] = ND == 3 ? to_fixed(s[2]) : 0;
    g.hl = (float)(0.5 * len);
    g.u[0] = (float)u[0];
    g.u[1] = (float)u[1];
    g.u[2] = (float)u[2];
    g.pad = 0.f;
    d.g32[buf][b] = g;
  }
}

template <int ND>
__global__ void k_init_geometry(SysConst k, DevState d, int buf, int prec) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  int f = d.bond_fil[b];
  int site = b + f;  // filament f's bond j joins its sites j and j+1
  double r1[3], r2[3], s[3], u[3], len;
  for (int i = 0; i < 3; ++i) {
    r1[i] = d.r[i][site];
    r2[i] = d.r[i][site + 1];
  }
  bond_from_sites<ND>(k, r1, r2, s, u, len);
  store_geom<ND>(d, buf, b, s, u, len, prec);
}

// ---------------------------------------------------------------------------
// Cell list.

// CellList::FindCellCoords (src/cell_list.cpp:139-157) on the bond's scaled
// position, recomputed exactly from its sites.
template <int ND>
__device__ __forceinline__ int bond_cell(const SysConst &k, const DevState &d,
                                         int b, int *xyz) {
  int f = d.bond_fil[b];
  int site = b + f;
  double r1[3], r2[3], s[3], u[3], len;
  for (int i = 0; i < 3; ++i) {
    r1[i] = d.r[i][site];
    r2[i] = d.r[i][site + 1];
  }
  bond_from_sites<ND>(k, r1, r2, s, u, len);
  int c[3] = {0, 0, 0};
  bool bad = false;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    double x = s[i] + 0.5;
    double fl = floor(k.n1d * x);
    int cc = (fl >= 0.0 && fl <= (double)k.n1d) ? (int)fl : -1;
    if (cc == k.n1d) cc -= 1;
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
  return (c[0] * k.n1d + c[1]) * k.third + c[2];
}

template <int ND>
__global__ void k_bond_cells(SysConst k, DevState d, int *xyz) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  bond_cell<ND>(k, d, b, xyz + 3 * (size_t)b);
}

template <int ND>
__global__ void k_bin_count(SysConst k, DevState d, int *key, int *cell_count) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = b < d.nb;
  int c = -1;
  if (active) {
    int xyz[3];
    c = bond_cell<ND>(k, d, b, xyz);
    key[b] = c;
  }
  // Warp-aggregated increment: one atomic per distinct cell in the warp.
  unsigned mask = __ballot_sync(0xffffffffu, active);
  if (active) {
    unsigned peers = __match_any_sync(mask, c);
    int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(&cell_count[c], __popc(peers));
  }
}

// Places each bond into its cell's range; decrements the counts back to
// zero so the count array is ready for the next rebuild without clearing.
__global__ void k_bin_scatter(int nb, const int *key, const int *cell_start,
                              int *cell_count, int *sorted) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int c = key[b];
  int slot = atomicSub(&cell_count[c], 1) - 1;
  sorted[cell_start[c] + slot] = b;
}

// Half-shell neighbour cells of (x, y, z) in the order of
// CellList::AssignCellNeighbors(false) (src/cell_list.cpp:206-262).
__device__ __forceinline__ int half_shell(const SysConst &k, int x, int y,
                                          int z, int *out) {
  int n1d = k.n1d, cnt = 0;
  int z_end = (k.n_dim == 3 ? z + 2 : z + 1);
  for (int zp = z; zp < z_end; ++zp) {
    int nz = zp;
    if (nz == n1d) nz = 0;
    for (int yp = (zp > z ? y - 1 : y); yp < y + 2; ++yp) {
      int ny = yp;
      if (ny < 0) ny = n1d - 1;
      else if (ny == n1d) ny = 0;
      for (int xp = (yp > y || zp > z ? x - 1 : x + 1); xp < x + 2; ++xp) {
        int nx = xp;
        if (nx < 0) nx = n1d - 1;
        else if (nx == n1d) nx = 0;
        if (nx == x && ny == y && nz == z) continue;
        out[cnt++] = (nx * n1d + ny) * k.third + nz;
      }
    }
  }
  return cnt;
}

// Pairs that ProcessPairInteraction marks no_interaction and the first
// evaluation after a rebuild culls (src/interaction_manager.cpp:341-367,
// 485-497): all pairs without like-like interactions, and bonds of one
// filament that share a site (Bond::HasNeighbor, src/bond.cpp:118-121).
__device__ __forceinline__ bool pair_excluded(const SysConst &k,
                                              const DevState &d, int a, int b) {
  if (!k.like_like) return true;
  if (d.bond_fil[a] == d.bond_fil[b]) {
    int diff = a - b;
    if (diff <= 1 && diff >= -1) return true;
  }
  return false;
}

__device__ __forceinline__ void cell_coords(const SysConst &k, int c, int &x,
                                            int &y, int &z) {
  z = c % k.third;
  int t = c / k.third;
  y = t % k.n1d;
  x = t / k.n1d;
}

// One thread per cell head (first entry of a cell in the sorted order):
// restores insertion order inside the cell (bond order, as Cell::AddObj
// appends in interactor order).
__global__ void k_cell_sort(int nb, const int *key, int *sorted,
                            const int *cell_start) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  int c = key[sorted[q]];
  if (cell_start[c] != q) return;
  int m = cell_start[c + 1] - q;
  int *it = sorted + q;
  for (int i = 1; i < m; ++i) {  // insertion sort (cells are small)
    int v = it[i], j = i - 1;
    while (j >= 0 && it[j] > v) {
      it[j + 1] = it[j];
      --j;
    }
    it[j + 1] = v;
  }
}

// One thread per cell head: number of kept pairs the cell contributes.
__global__ void k_cell_count(SysConst k, DevState d, int nb, const int *key,
                             const int *sorted, const int *cell_start,
                             int *pair_count) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  int c = key[sorted[q]];
  if (cell_start[c] != q) {
    pair_count[q] = 0;
    return;
  }
  int m = cell_start[c + 1] - q;
  const int *it = sorted + q;
  long long cnt = 0;
  for (int i = 0; i < m - 1; ++i)
    for (int j = i + 1; j < m; ++j) cnt += !pair_excluded(k, d, it[i], it[j]);
  int x, y, z, nbr[13];
  cell_coords(k, c, x, y, z);
  int nn = half_shell(k, x, y, z, nbr);
  for (int kk = 0; kk < nn; ++kk) {
    int cn = nbr[kk];
    int s0 = cell_start[cn], s1 = cell_start[cn + 1];
    for (int i = 0; i < m; ++i)
      for (int j = s0; j < s1; ++j) cnt += !pair_excluded(k, d, it[i], sorted[j]);
  }
  pair_count[q] = cnt > 0x3fffffff ? 0x3fffffff : (int)cnt;
}

// Writes each cell's pairs at its offset in the reference's list order
// (Cell::MakePairs, src/cell.cpp:14-22): pairs inside the cell, then with
// each half-shell neighbour; clears each new pair's stored force and counts
// per-bond pair entries for the CSR.
__global__ void k_pair_emit(SysConst k, DevState d, int nb, const int *key,
                            const int *sorted, const int *cell_start,
                            const int *pair_off, int cap, int *deg, int prec) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  int c = key[sorted[q]];
  if (cell_start[c] != q) return;
  int m = cell_start[c + 1] - q;
  const int *it = sorted + q;
  int p = pair_off[q];
  int x, y, z, nbr[13];
  cell_coords(k, c, x, y, z);
  int nn = half_shell(k, x, y, z, nbr);
  auto emit = [&](int a, int b) {
    if (pair_excluded(k, d, a, b)) return;
    if (p < cap) {
      d.pa[p] = a;
      d.pb[p] = b;
      if (prec == 0) {
        d.pf64[3 * (size_t)p] = 0.0;
        d.pf64[3 * (size_t)p + 1] = 0.0;
        d.pf64[3 * (size_t)p + 2] = 0.0;
      } else {
        d.pf32[3 * (size_t)p] = 0.f;
        d.pf32[3 * (size_t)p + 1] = 0.f;
        d.pf32[3 * (size_t)p + 2] = 0.f;
      }
      atomicAdd(&deg[a], 1);
      atomicAdd(&deg[b], 1);
    }
    ++p;
  };
  for (int i = 0; i < m - 1; ++i)
    for (int j = i + 1; j < m; ++j) emit(it[i], it[j]);
  for (int kk = 0; kk < nn; ++kk) {
    int cn = nbr[kk];
    int s0 = cell_start[cn], s1 = cell_start[cn + 1];
    for (int i = 0; i < m; ++i)
      for (int j = s0; j < s1; ++j) emit(it[i], sorted[j]);
  }
}

// Entries (pair << 1 | role) of every bond; role 0 = obj1, 1 = obj2.  The
// degree array is decremented back to zero.
__global__ void k_csr_fill(DevState d, int np, int *deg) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  int a = d.pa[p], b = d.pb[p];
  int sa = atomicSub(&deg[a], 1) - 1;
  int sb = atomicSub(&deg[b], 1) - 1;
  d.e_ent[d.e_off[a] + sa] = p << 1;
  d.e_ent[d.e_off[b] + sb] = (p << 1) | 1;
}

// Sorts each bond's entries by pair index = the order in which the
// reference's serial ApplyPairInteractions adds them to the bond.
__global__ void k_csr_sort(DevState d) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  int e0 = d.e_off[b], e1 = d.e_off[b + 1];
  int *e = d.e_ent;
  for (int i = e0 + 1; i < e1; ++i) {
    int v = e[i], j = i - 1;
    while (j >= e0 && e[j] > v) {
      e[j + 1] = e[j];
      --j;
    }
    e[j + 1] = v;
  }
}

// InteractionManager::ZeroDrTot (src/interaction_manager.cpp:316-321).
__global__ void k_zero_dr(DevState d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *d.dr_max_bits = 0ull;
  if (i >= d.ns) return;
  d.dz[0][i] = d.r[0][i];
  d.dz[1][i] = d.r[1][i];
  d.dz[2][i] = d.r[2][i];
  d.dt[i] = 0.0;
}

// ---------------------------------------------------------------------------
// Exclusive scan of int32 (n elements, out has n+1 entries, out[n] = total).

constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int *tmp, int &total) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) tmp[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < (SCAN_BLOCK / 32) ? tmp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < (SCAN_BLOCK / 32)) tmp[lane] = s;
  }
  __syncthreads();
  total = tmp[SCAN_BLOCK / 32 - 1];
  int excl = x - v + (w > 0 ? tmp[w - 1] : 0);
  __syncthreads();
  return excl;
}

__global__ void k_scan_tiles(const int *in, int *out, int n, int *tile_sums) {
  __shared__ int tmp[SCAN_BLOCK / 32];
  int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS], sum = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    v[i] = (base + i < n) ? in[base + i] : 0;
    sum += v[i];
  }
  int total;
  int run = block_exclusive_scan(sum, tmp, total);
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile sums in place; total -> *out_total.
__global__ void k_scan_sums(int *sums, int n, int *out_total) {
  __shared__ int tmp[SCAN_BLOCK / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += SCAN_BLOCK) {
    int i = base + threadIdx.x;
    int v = i < n ? sums[i] : 0;
    int total;
    int e = block_exclusive_scan(v, tmp, total);
    if (i < n) sums[i] = e + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *out_total = carry;
}

__global__ void k_scan_add(int *out, int n, const int *tile_sums) {
  int base = blockIdx.x * SCAN_TILE;
  int add = tile_sums[blockIdx.x];
  for (int i = threadIdx.x; i < SCAN_TILE; i += SCAN_BLOCK)
    if (base + i < n) out[base + i] += add;
}

// ---------------------------------------------------------------------------
// Pair stage of one bond: loops over the bond's pairs in list order and sums
// +F / -F and +t1 / -t2 as ApplyPairInteractions does
// (src/interaction_manager.cpp:500-517).  A pair whose potential is not
// evaluated this step keeps its force from the last evaluation since the
// list was built (the reference's Interaction records are never cleared,
// src/minimum_distance.cpp:31-34 resets only dr and the contacts).  Only the
// obj1 side stores a new force; both sides reach the same in-range verdict
// bit for bit, so no side reads a force the other is writing.

__device__ __forceinline__ void cross3(const double *a, const double *b,
                                       double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

template <int ND>
__device__ __forceinline__ void bond_pairs_f64(const SysConst &k,
                                               const DevState &d, int b,
                                               int rbuf, double F[3],
                                               double T[3]) {
  F[0] = F[1] = F[2] = 0.0;
  T[0] = T[1] = T[2] = 0.0;
  const BondGeomF64 *geo = d.g64[rbuf];
  const BondGeomF64 self = geo[b];
  const int e1 = d.e_off[b + 1];
  for (int e = d.e_off[b]; e < e1; ++e) {
    int ent = d.e_ent[e];
    int p = ent >> 1, role = ent & 1;
    int other = role ? d.pa[p] : d.pb[p];
    const BondGeomF64 o = geo[other];
    PairGeom<double> g;
    if (role == 0) sphero_f64<ND>(k, self, o, g);
    else sphero_f64<ND>(k, o, self, g);
    double force[3] = {0.0, 0.0, 0.0};
    double *stale = d.pf64 + 3 * (size_t)p;
    if (wca_f64<ND>(k, g, force)) {
      if (role == 0) {
        stale[0] = force[0];
        stale[1] = force[1];
        stale[2] = force[2];
      }
    } else {
      force[0] = stale[0];
      force[1] = stale[1];
      force[2] = stale[2];
    }
    double t[3];
    cross3(role ? g.c2 : g.c1, force, t);
    if (role == 0) {
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += force[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) T[i] += t[i];
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] -= force[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) T[i] -= t[i];
    }
  }
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float x) {
  float y = x - comp;
  float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

template <int ND>
__device__ __forceinline__ void bond_pairs_f32(const SysConst &k,
                                               const DevState &d, int b,
                                               int rbuf, double F[3],
                                               double T[3]) {
  float sF[3] = {0.f, 0.f, 0.f}, cF[3] = {0.f, 0.f, 0.f};
  float sT[3] = {0.f, 0.f, 0.f}, cT[3] = {0.f, 0.f, 0.f};
  const BondGeomF32 *geo = d.g32[rbuf];
  const BondGeomF32 self = geo[b];
  const int e1 = d.e_off[b + 1];
  for (int e = d.e_off[b]; e < e1; ++e) {
    int ent = d.e_ent[e];
    int p = ent >> 1, role = ent & 1;
    int other = role ? d.pa[p] : d.pb[p];
    const BondGeomF32 o = geo[other];
    PairGeom<float> g;
    if (role == 0) sphero_f32<ND>(k, self, o, g);
    else sphero_f32<ND>(k, o, self, g);
    float force[3] = {0.f, 0.f, 0.f};
    float *stale = d.pf32 + 3 * (size_t)p;
    if (wca_f32<ND>(k, g, force)) {
      if (role == 0) {
        stale[0] = force[0];
        stale[1] = force[1];
        stale[2] = force[2];
      }
    } else {
      force[0] = stale[0];
      force[1] = stale[1];
      force[2] = stale[2];
    }
    const float *c = role ? g.c2 : g.c1;
    float t[3] = {c[1] * force[2] - c[2] * force[1],
                  c[2] * force[0] - c[0] * force[2],
                  c[0] * force[1] - c[1] * force[0]};
    float sgn = role ? -1.f : 1.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) kahan_add(sF[i], cF[i], sgn * force[i]);
#pragma unroll
    for (int i = 0; i < 3; ++i) kahan_add(sT[i], cT[i], sgn * t[i]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    F[i] = (double)sF[i] - (double)cF[i];
    T[i] = (double)sT[i] - (double)cT[i];
  }
}

template <int ND, int PREC>
__global__ void k_pairs(SysConst k, DevState d, int rbuf) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  double F[3], T[3];
  if (PREC == 0) bond_pairs_f64<ND>(k, d, b, rbuf, F, T);
  else bond_pairs_f32<ND>(k, d, b, rbuf, F, T);
  for (int i = 0; i < 3; ++i) {
    d.bF[i][b] = F[i];
    d.bT[i][b] = T[i];
  }
}

// ---------------------------------------------------------------------------
// Integrator.  A block holds a run of whole filaments, one thread per site,
// filaments back to back.  Per-site work runs in parallel; the sequential
// recurrences of one filament (Thomas solves, metric determinants,
// renormalisation) run on its first thread, in the reference's order.

// Thomas algorithm of the reference's tridiagonal_solver
// (src/linear_algebra.cpp:164-197); n unknowns, in place.
__device__ __forceinline__ void thomas(double *a, const double *b, double *c,
                                       double *d, int n) {
  n--;
  c[0] /= b[0];
  d[0] /= b[0];
  for (int i = 1; i < n; ++i) {
    c[i] /= b[i] - a[i - 1] * c[i - 1];
    d[i] = (d[i] - a[i - 1] * d[i - 1]) / (b[i] - a[i - 1] * c[i - 1]);
  }
  d[n] = (d[n] - a[n - 1] * d[n - 1]) / (b[n] - a[n - 1] * c[n - 1]);
  for (int i = n; i-- > 0;) d[i] -= c[i] * d[i + 1];
}

template <int ND>
__device__ __forceinline__ double dotn(const double *a, const double *b) {
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) m += a[i] * b[i];
  return m;
}

template <int ND, int PREC, bool FUSED>
__global__ void __launch_bounds__(256)
    k_integrate(SysConst k, DevState d, int midstep, unsigned long long mcount,
                int rbuf, int interaction, int capture) {
  extern __shared__ double smem[];
  const int C = blockDim.x;
  double *sr = smem;            // positions            3C
  double *su = sr + 3 * C;      // site orientations    3C
  double *stn = su + 3 * C;     // tangents             3C
  double *sfr = stn + 3 * C;    // random forces        3C
  double *sbF = sfr + 3 * C;    // bond forces / gamma.F 3C
  double *sbT = sbF + 3 * C;    // bond torques         3C
  double *scos = sbT + 3 * C;   // cos(theta)           C
  double *sT = scos + C;        // rhs / tensions       C
  double *sa = sT + C;          // lower diagonal       C
  double *sb = sa + C;          // diagonal             C
  double *sc = sb + C;          // upper diagonal       C
  double *skeff = sc + C;       // k_eff                C
  double *sdt = skeff + C;      // det_t                2C
  double *sdb = sdt + 2 * C;    // det_b                2C
  int *sflag = (int *)(sdb + 2 * C);
  __shared__ double s_drmax[32];

#define V(arr, slot, comp) arr[(comp) * C + (slot)]

  const int blk = blockIdx.x;
  const int t = threadIdx.x;
  const int s0 = d.blk_site0[blk];
  const int count = d.blk_site0[blk + 1] - s0;
  const bool active = t < count;
  const int g = s0 + t;
  int f = 0, n = 0, j = -1, base = 0, dbase = 0, lf = 0;
  if (active) {
    f = d.site_fil[g];
    int fs0 = d.f_site_off[f];
    n = d.f_site_off[f + 1] - fs0;
    j = g - fs0;
    base = t - j;
    lf = f - d.blk_f0[blk];
    dbase = base + lf;
  }
  if (t < C) sflag[t] = 0;
  const int b = g - f;  // this thread's bond (valid when j < n-1)
  const bool has_bond = active && j < n - 1;
  double l = 0, linv = 0, kappa = 0, gpar = 1, gperp = 1, spar = 0, sperp = 0;
  if (active) {
    l = d.f_l[f];
    linv = d.f_linv[f];
    kappa = d.f_kappa[f];
    gpar = d.f_gpar[f];
    gperp = d.f_gperp[f];
    spar = d.f_spar[f];
    sperp = d.f_sperp[f];
  }

  // ---- P0: positions, orientations, bond forces --------------------------
  double r[3] = {0, 0, 0};
  if (active) {
    r[0] = d.r[0][g];
    r[1] = d.r[1][g];
    r[2] = d.r[2][g];
    V(sr, t, 0) = r[0];
    V(sr, t, 1) = r[1];
    V(sr, t, 2) = r[2];
  }
  double bF[3] = {0, 0, 0}, bT[3] = {0, 0, 0};
  if (has_bond && interaction) {
    if (FUSED) {
      if (PREC == 0) bond_pairs_f64<ND>(k, d, b, rbuf, bF, bT);
      else bond_pairs_f32<ND>(k, d, b, rbuf, bF, bT);
    } else {
      for (int i = 0; i < 3; ++i) {
        bF[i] = d.bF[i][b];
        bT[i] = d.bT[i][b];
      }
    }
  }
  if (has_bond) {
    for (int i = 0; i < 3; ++i) {
      V(sbF, t, i) = bF[i];
      V(sbT, t, i) = bT[i];
    }
  }
  __syncthreads();
  // Site orientation = orientation of its bond (Mesh::UpdateSiteOrientations,
  // src/mesh.cpp:168-173), recomputed as Bond::ReInit does.
  double u[3] = {0, 0, 0};
  if (has_bond) {
    double r2[3] = {V(sr, t + 1, 0), V(sr, t + 1, 1), V(sr, t + 1, 2)};
    double len = 0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      u[i] = r2[i] - r[i];
      len += u[i] * u[i];
    }
    len = sqrt(len);
#pragma unroll
    for (int i = 0; i < ND; ++i) u[i] /= len;
    for (int i = 0; i < 3; ++i) V(su, t, i) = u[i];
  }
  __syncthreads();
  if (active && j == n - 1) {
    for (int i = 0; i < 3; ++i) {
      u[i] = V(su, t - 1, i);
      V(su, t, i) = u[i];
    }
  }
  __syncthreads();

  // ---- P1: ApplyInteractionForces (src/filament.cpp:992-1048) -------------
  double F[3] = {0.0, 0.0, 0.0};
  if (active) {
    const double mag = 0.5 * 0.0 * l;  // driving_factor 0, from bond centre
    if (j >= 1) {  // this site is site i+1 of bond i = j-1
      double up[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
      double fb[3] = {V(sbF, t - 1, 0), V(sbF, t - 1, 1), V(sbF, t - 1, 2)};
      double tb[3] = {V(sbT, t - 1, 0), V(sbT, t - 1, 1), V(sbT, t - 1, 2)};
      double pt[3], sf[3];
      cross3(up, tb, pt);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        pt[i] *= linv;
        sf[i] = 0.5 * fb[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) pt[i] *= -1;
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += sf[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += pt[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += mag * up[i];
    }
    if (j <= n - 2) {  // site i of bond i = j
      double pt[3], sf[3];
      cross3(u, bT, pt);  // bF/bT hold this thread's bond
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        pt[i] *= linv;
        sf[i] = 0.5 * bF[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += sf[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += pt[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += mag * u[i];
    }
  }
  // CalculateAngles (:430-437), CalculateTangents (:439-443, Site::CalcTangent)
  double tn[3] = {0, 0, 0};
  if (active) {
    if (j < n - 2) {
      double un[3] = {V(su, t + 1, 0), V(su, t + 1, 1), V(su, t + 1, 2)};
      scos[t] = dotn<ND>(u, un);
    }
    if (j == 0 || j == n - 1) {
      tn[0] = u[0];
      tn[1] = u[1];
      tn[2] = u[2];
    } else {
      double mag = 0.0;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        tn[i] = V(su, t - 1, i) + u[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) mag += tn[i] * tn[i];
      mag = sqrt(mag);
#pragma unroll
      for (int i = 0; i < ND; ++i) tn[i] /= mag;
    }
    for (int i = 0; i < 3; ++i) V(stn, t, i) = tn[i];
  }
  __syncthreads();

  // ---- P2: random forces, projection, previous positions -----------------
  double fr[3] = {0, 0, 0}, rp[3] = {0, 0, 0};
  if (midstep) {
    if (active) rp[0] = r[0], rp[1] = r[1], rp[2] = r[2];
    if (k.stoch) {
      if (active) {  // ConstructUnprojectedRandomForces (:518-548)
        double xi[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
        unsigned long long k0 = (mcount * (unsigned long long)n + j) * ND;
#pragma unroll
        for (int i = 0; i < ND; ++i)
          xi[i] = sc_host_philox_uniform(k.seed, (uint32_t)f, k0 + i) - 0.5;
        if (ND == 2) {
          xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1];
          xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0];
        } else {
          xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1] +
                  tn[0] * tn[2] * xi[2];
          xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0] +
                  tn[1] * tn[2] * xi[2];
          xt[2] = tn[2] * tn[2] * xi[2] + tn[0] * tn[2] * xi[0] +
                  tn[1] * tn[2] * xi[1];
        }
#pragma unroll
        for (int i = 0; i < ND; ++i) fr[i] = sperp * xi[i] + (spar - sperp) * xt[i];
        for (int i = 0; i < 3; ++i) V(sfr, t, i) = fr[i];
      }
      __syncthreads();
      // GeometricallyProjectRandomForces (:550-599)
      if (has_bond) {
        double tmp[3];
#pragma unroll
        for (int i = 0; i < ND; ++i) tmp[i] = V(sfr, t + 1, i) - fr[i];
        sT[t] = dotn<ND>(tmp, u);
        sb[t] = 2;
        if (j > 0) {
          sc[t - 1] = -scos[t - 1];
          sa[t - 1] = -scos[t - 1];
        }
      }
      __syncthreads();
      if (active && j == 0) thomas(sa + t, sb + t, sc + t, sT + t, n - 1);
      __syncthreads();
      if (active) {
        double fp[3];
        if (j == 0) {
#pragma unroll
          for (int i = 0; i < ND; ++i) fp[i] = fr[i] + sT[t] * u[i];
        } else if (j == n - 1) {
#pragma unroll
          for (int i = 0; i < ND; ++i) fp[i] = fr[i] - sT[t - 1] * V(su, t - 1, i);
        } else {
#pragma unroll
          for (int i = 0; i < ND; ++i)
            fp[i] = fr[i] + sT[t] * u[i] - sT[t - 1] * V(su, t - 1, i);
        }
#pragma unroll
        for (int i = 0; i < ND; ++i) fr[i] = fp[i];
      }
    }
  } else if (active) {
    rp[0] = d.rp[0][g];
    rp[1] = d.rp[1][g];
    rp[2] = d.rp[2][g];
    if (k.stoch) {
      fr[0] = d.fr[0][g];
      fr[1] = d.fr[1][g];
      fr[2] = d.fr[2][g];
    }
  }
  // AddRandomForces (:601-606)
  if (active && k.stoch) {
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fr[i];
  }

  // ---- P3: bending and metric forces (:608-776) ---------------------------
  if (active && j == 0) {
    double *dt = sdt + dbase;
    dt[0] = 1;
    dt[1] = 2;
    for (int i = 2; i < n; ++i)
      dt[i] = 2 * dt[i - 1] - (-scos[t + i - 2]) * (-scos[t + i - 2]) * dt[i - 2];
  }
  if (active && j == 1) {
    double *db = sdb + dbase;  // the filament's det_b[0]
    db[n] = 1;
    db[n - 1] = 2;
    const int tb0 = t - 1;  // slot of the filament's first site
    for (int i = 2; i < n; ++i)
      db[n - i] = 2 * db[n - i + 1] -
                  (-scos[tb0 + n - i - 1]) * (-scos[tb0 + n - i - 1]) * db[n - i + 2];
  }
  __syncthreads();
  if (active && j < n - 2) {
    const double det_g = sdt[dbase + n - 1];
    double ginv = scos[t] * sdt[dbase + j] * sdb[dbase + j + 3] / det_g;
    skeff[t] = (kappa + l * ginv) / (l * l);
  }
  __syncthreads();
  if (active) {
    double fs[3] = {0, 0, 0};
    const int kk = j;
    if (ND == 2) {
      if (kk > 1) {
        double u1[3] = {V(su, t - 2, 0), V(su, t - 2, 1), 0};
        double u2[3] = {V(su, t - 1, 0), V(su, t - 1, 1), 0};
        double ke = skeff[t - 2];
        fs[0] += ke * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]);
        fs[1] += ke * ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]);
      }
      if (kk > 0 && kk < n - 1) {
        double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), 0};
        double u2[3] = {u[0], u[1], 0};
        double ke = skeff[t - 1];
        fs[0] += ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]));
        fs[1] += ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0] -
                       ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]));
      }
      if (kk < n - 2) {
        double u1[3] = {u[0], u[1], 0};
        double u2[3] = {V(su, t + 1, 0), V(su, t + 1, 1), 0};
        double ke = skeff[t];
        fs[0] -= ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1]);
        fs[1] -= ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0]);
      }
    } else {
      if (kk > 1) {
        double u1[3] = {V(su, t - 2, 0), V(su, t - 2, 1), V(su, t - 2, 2)};
        double u2[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
        double ke = skeff[t - 2];
        fs[0] += ke * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                       u2[0] * u2[2] * u1[2]);
        fs[1] += ke * ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                       u2[1] * u2[2] * u1[2]);
        fs[2] += ke * ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                       u2[2] * u2[1] * u1[1]);
      }
      if (kk > 0 && kk < n - 1) {
        double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
        const double *u2 = u;
        double ke = skeff[t - 1];
        fs[0] += ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       u1[0] * u1[2] * u2[2] -
                       ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                        u2[0] * u2[2] * u1[2]));
        fs[1] += ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[1] * u1[0] * u2[0] -
                       u1[1] * u1[2] * u2[2] -
                       ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                        u2[1] * u2[2] * u1[2]));
        fs[2] += ke * ((1 - u1[2] * u1[2]) * u2[2] - u1[2] * u1[0] * u2[0] -
                       u1[2] * u1[1] * u2[1] -
                       ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                        u2[1] * u2[2] * u1[1]));
      }
      if (kk < n - 2) {
        const double *u1 = u;
        double u2[3] = {V(su, t + 1, 0), V(su, t + 1, 1), V(su, t + 1, 2)};
        double ke = skeff[t];
        fs[0] -= ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       u1[0] * u1[2] * u2[2]);
        fs[1] -= ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[1] * u1[0] * u2[0] -
                       u1[1] * u1[2] * u2[2]);
        fs[2] -= ke * ((1 - u1[2] * u1[2]) * u2[2] - u1[2] * u1[0] * u2[0] -
                       u1[2] * u1[1] * u2[1]);
      }
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
  }

  // ---- P4: tensions (:778-838) --------------------------------------------
  double gam[9];
  if (active) {
    int gi = 0;
#pragma unroll
    for (int a = 0; a < ND; ++a)
#pragma unroll
      for (int c = 0; c < ND; ++c) {
        gam[gi] = 1.0 / gpar * (tn[a] * tn[c]) +
                  1.0 / gperp * ((a == c ? 1 : 0) - tn[a] * tn[c]);
        gi++;
      }
    // gamma^-1 F of this site: "temp_a" of row j and "temp_b" of row j-1.
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double v = gam[ND * i] * F[0] + gam[ND * i + 1] * F[1];
      if (ND == 3) v += gam[ND * i + 2] * F[2];
      V(sbF, t, i) = v;
    }
  }
  __syncthreads();
  if (has_bond) {
    double fdiff[3];
#pragma unroll
    for (int i = 0; i < ND; ++i) fdiff[i] = V(sbF, t + 1, i) - V(sbF, t, i);
    sT[t] = dotn<ND>(u, fdiff);
    double tn2[3] = {V(stn, t + 1, 0), V(stn, t + 1, 1), V(stn, t + 1, 2)};
    double d1 = dotn<ND>(tn, u);
    double d2 = dotn<ND>(tn2, u);
    sb[t] = 2.0 / gperp + (1.0 / gpar - 1.0 / gperp) * (d1 * d1 + d2 * d2);
    if (j > 0) {
      double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
      double hu = -1.0 / gperp * dotn<ND>(u, u1) -
                  (1.0 / gpar - 1.0 / gperp) * (dotn<ND>(tn, u1) * dotn<ND>(tn, u));
      sc[t - 1] = hu;
      sa[t - 1] = hu;
    }
  }
  __syncthreads();
  if (active && j == 0) thomas(sa + t, sb + t, sc + t, sT + t, n - 1);
  __syncthreads();

  // ---- P5: UpdateSitePositions (:840-927), CheckBondLengths (:934-951) ----
  if (active) {
    double fs[3];
    if (j == 0) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = sT[t] * u[i];
    } else if (j == n - 1) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = -sT[t - 1] * V(su, t - 1, i);
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = sT[t] * u[i] - sT[t - 1] * V(su, t - 1, i);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
    const double dl = (midstep ? 0.5 * k.delta : k.delta);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double ft = gam[ND * i] * F[0] + gam[ND * i + 1] * F[1];
      if (ND == 3) ft += gam[ND * i + 2] * F[2];
      r[i] = rp[i] + dl * ft;
    }
  }
  __syncthreads();  // everyone is done reading su / sr of the old state
  if (active) {
    for (int i = 0; i < 3; ++i) V(sr, t, i) = r[i];
  }
  __syncthreads();
  if (has_bond) {
    double rd[3], um = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rd[i] = V(sr, t + 1, i) - r[i];
      um += rd[i] * rd[i];
    }
    um = sqrt(um);
#pragma unroll
    for (int i = 0; i < ND; ++i) V(su, t, i) = rd[i] / um;
  }
  if (active && j >= 1) {
    double a = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double temp = r[i] - V(sr, t - 1, i);
      a += temp * temp;
    }
    a = sqrt(a);
    double err = dabs(l - a) / l;
    if (err > 1e-3) sflag[lf] = 1;
  }
  __syncthreads();
  if (active && j == 0) {
    int sw = d.f_switch[f], nn = d.f_nnorm[f];
    if (sflag[lf]) {
      sw = !sw;
      nn = 0;
      if (sw) {
        for (int jj = 1; jj < n; ++jj)
#pragma unroll
          for (int i = 0; i < ND; ++i)
            V(sr, t + jj, i) = V(sr, t + jj - 1, i) + l * V(su, t + jj - 1, i);
      } else {
        for (int jj = n - 1; jj > 0; --jj)
#pragma unroll
          for (int i = 0; i < ND; ++i)
            V(sr, t + jj - 1, i) = V(sr, t + jj, i) - l * V(su, t + jj - 1, i);
      }
    }
    nn++;
    d.f_switch[f] = sw;
    d.f_nnorm[f] = nn;
  }
  __syncthreads();

  // ---- P6: bond geometry (Mesh::UpdateBondPositions), state write-back ----
  double my_dr = 0.0;
  if (active) {
    for (int i = 0; i < 3; ++i) r[i] = V(sr, t, i);
    if (has_bond) {
      double r2[3] = {V(sr, t + 1, 0), V(sr, t + 1, 1), V(sr, t + 1, 2)};
      double s[3], ub[3], len;
      bond_from_sites<ND>(k, r, r2, s, ub, len);
      store_geom<ND>(d, 1 - rbuf, b, s, ub, len, PREC);
    }
    d.r[0][g] = r[0];
    d.r[1][g] = r[1];
    d.r[2][g] = r[2];
    if (midstep) {
      d.rp[0][g] = rp[0];
      d.rp[1][g] = rp[1];
      d.rp[2][g] = rp[2];
      if (k.stoch) {
        d.fr[0][g] = fr[0];
        d.fr[1][g] = fr[1];
        d.fr[2][g] = fr[2];
      }
    }
    bool bad = false;
#pragma unroll
    for (int i = 0; i < ND; ++i) bad |= !isfinite(r[i]);
    if (bad) atomicOr(d.status, ST_NAN);
    if (capture) {
      for (int i = 0; i < 3; ++i) d.cap_F[i][g] = F[i];
      if (has_bond) d.cap_T[b] = sT[t];
    }
    // Displacement tracking for the next query (Mesh::UpdateDrTot runs on
    // the filaments whose last update was a full step; each query adds the
    // squared displacement twice, src/mesh.cpp:538-541, src/object.cpp:
    // 282-292).
    if (!midstep && interaction) {
      double acc = d.dt[g];
      for (int twice = 0; twice < 2; ++twice)
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          double dr = r[i] - d.dz[i][g];
          acc += dr * dr;
        }
      d.dt[g] = acc;
      my_dr = acc;
    }
  }
  if (!midstep && interaction) {
    // Block max, then one atomic per block on the IEEE bits (non-negative).
    double v = my_dr;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((t & 31) == 0) s_drmax[t >> 5] = v;
    __syncthreads();
    if (t < 32) {
      v = (t < (C + 31) / 32) ? s_drmax[t] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
      if (t == 0) {
        if (!(v <= 1e300)) atomicOr(d.status, ST_NAN);
        atomicMax(d.dr_max_bits, (unsigned long long)__double_as_longlong(v));
      }
    }
  }
#undef V
}

// ---------------------------------------------------------------------------
// Host launchers.

static inline int cdiv(long long a, int b) { return (int)((a + b - 1) / b); }

void launch_init_geometry(const SysConst &k, const DevState &d, int buf,
                          int prec, cudaStream_t st) {
  if (d.nb == 0) return;
  if (k.n_dim == 3) k_init_geometry<3><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, buf, prec);
  else k_init_geometry<2><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, buf, prec);
}

int scan_temp_ints(long long n) { return cdiv(n, SCAN_TILE) + 1; }

// Exclusive scan in[0..n) -> out[0..n], out[n] = total.  tmp holds
// scan_temp_ints(n) ints.  Returns launches issued.
int launch_exclusive_scan(const int *in, int *out, long long n, int *tmp,
                          cudaStream_t st) {
  int tiles = cdiv(n, SCAN_TILE);
  if (tiles == 0) tiles = 1;
  k_scan_tiles<<<tiles, SCAN_BLOCK, 0, st>>>(in, out, (int)n, tmp);
  k_scan_sums<<<1, SCAN_BLOCK, 0, st>>>(tmp, tiles, out + n);
  k_scan_add<<<tiles, SCAN_BLOCK, 0, st>>>(out, (int)n, tmp);
  return 3;
}

int launch_bin_count(const SysConst &k, const DevState &d, int *key,
                     int *cell_count, cudaStream_t st) {
  if (k.n_dim == 3) k_bin_count<3><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, key, cell_count);
  else k_bin_count<2><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, key, cell_count);
  return 1;
}

int launch_bond_cells(const SysConst &k, const DevState &d, int *xyz,
                      cudaStream_t st) {
  if (k.n_dim == 3) k_bond_cells<3><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, xyz);
  else k_bond_cells<2><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, xyz);
  return 1;
}

int launch_bin_scatter(int nb, const int *key, const int *cell_start,
                       int *cell_count, int *sorted, cudaStream_t st) {
  k_bin_scatter<<<cdiv(nb, 256), 256, 0, st>>>(nb, key, cell_start, cell_count, sorted);
  return 1;
}

int launch_cell_sort_count(const SysConst &k, const DevState &d, const int *key,
                           int *sorted, const int *cell_start, int *pair_count,
                           cudaStream_t st) {
  k_cell_sort<<<cdiv(d.nb, 128), 128, 0, st>>>(d.nb, key, sorted, cell_start);
  k_cell_count<<<cdiv(d.nb, 128), 128, 0, st>>>(k, d, d.nb, key, sorted,
                                                cell_start, pair_count);
  return 2;
}

int launch_pair_emit(const SysConst &k, const DevState &d, const int *key,
                     const int *sorted, const int *cell_start,
                     const int *pair_off, int cap, int *deg, int prec,
                     cudaStream_t st) {
  k_pair_emit<<<cdiv(d.nb, 128), 128, 0, st>>>(k, d, d.nb, key, sorted, cell_start,
                                               pair_off, cap, deg, prec);
  return 1;
}

int launch_csr(const DevState &d, int np, int *deg, cudaStream_t st) {
  int n = 0;
  if (np > 0) {
    k_csr_fill<<<cdiv(np, 256), 256, 0, st>>>(d, np, deg);
    ++n;
  }
  k_csr_sort<<<cdiv(d.nb, 256), 256, 0, st>>>(d);
  return n + 1;
}

int launch_zero_dr(const DevState &d, cudaStream_t st) {
  k_zero_dr<<<cdiv(d.ns > 0 ? d.ns : 1, 256), 256, 0, st>>>(d);
  return 1;
}

int launch_pairs(const SysConst &k, const DevState &d, int rbuf, int prec,
                 cudaStream_t st) {
  int grid = cdiv(d.nb, 128);
  if (k.n_dim == 3) {
    if (prec == 0) k_pairs<3, 0><<<grid, 128, 0, st>>>(k, d, rbuf);
    else k_pairs<3, 1><<<grid, 128, 0, st>>>(k, d, rbuf);
  } else {
    if (prec == 0) k_pairs<2, 0><<<grid, 128, 0, st>>>(k, d, rbuf);
    else k_pairs<2, 1><<<grid, 128, 0, st>>>(k, d, rbuf);
  }
  return 1;
}

size_t integrate_smem_bytes(int C) {
  return sizeof(double) * 28 * (size_t)C + sizeof(int) * (size_t)C;
}

template <int ND, int PREC, bool FUSED>
static void set_attr(size_t smem) {
  cudaFuncSetAttribute(k_integrate<ND, PREC, FUSED>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

void prepare_integrate(int C) {
  size_t smem = integrate_smem_bytes(C);
  set_attr<3, 0, false>(smem);
  set_attr<3, 0, true>(smem);
  set_attr<3, 1, false>(smem);
  set_attr<3, 1, true>(smem);
  set_attr<2, 0, false>(smem);
  set_attr<2, 0, true>(smem);
  set_attr<2, 1, false>(smem);
  set_attr<2, 1, true>(smem);
}

int launch_integrate(const SysConst &k, const DevState &d, int nblocks, int C,
                     int midstep, unsigned long long mcount, int rbuf,
                     int interaction, int capture, int prec, bool fused,
                     cudaStream_t st) {
  size_t smem = integrate_smem_bytes(C);
#define SC_LAUNCH(ND, P, FU)                                                   \
  k_integrate<ND, P, FU><<<nblocks, C, smem, st>>>(k, d, midstep, mcount, rbuf, \
                                                    interaction, capture)
  if (k.n_dim == 3) {
    if (prec == 0) {
      if (fused) SC_LAUNCH(3, 0, true); else SC_LAUNCH(3, 0, false);
    } else {
      if (fused) SC_LAUNCH(3, 1, true); else SC_LAUNCH(3, 1, false);
    }
  } else {
    if (prec == 0) {
      if (fused) SC_LAUNCH(2, 0, true); else SC_LAUNCH(2, 0, false);
    } else {
      if (fused) SC_LAUNCH(2, 1, true); else SC_LAUNCH(2, 1, false);
    }
  }
#undef SC_LAUNCH
  return 1;
}

}  // namespace sc
