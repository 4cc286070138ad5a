// Device kernels of the B200 filament step.  Compiled with --fmad=false
// (see sc_common.cuh).
//
//   cell list      k_bin_count, k_bin_scatter, k_cell_sort_count,
//                  k_pair_emit   (CellList + Cell, src/cell_list.cpp,
//                                 src/cell.cpp)
//   pair CSR       k_csr_offsets, k_csr_fill, k_csr_sort_pos (per-bond pair
//                  entries in list order, for the reference's serial
//                  scatter order)
//   pair forces    k_pair_eval   (InteractionManager::CalculatePairInteractions,
//                                 one thread per pair, signed per-bond slots)
//                                (mixed: nearly parallel pairs in FP64)
//                  k_bond_sum    (ApplyPairInteractions into bond accumulators)
//   thermo         k_thermo, k_potential (pair virial and pressure records,
//                                 per-filament potential energy)
//   integrator     k_integrate   (Filament::UpdatePosition for every
//                                 filament; sums each bond's pair slots first)
//   utilities      exclusive scan, geometry init, displacement reset.
#include <cuda_runtime.h>

#include <cstdlib>

#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_launch.h"
#include "sc_cells.cuh"
#include "sc_pair.cuh"
#include "sc_step.cuh"
#include "sc_step_warp.cuh"

namespace sc {

template <int ND>
__global__ void k_init_geometry(SysConst k, DevState d, int buf, int prec, int write_ub) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  int f = d.bond_fil[b];
  int site = b + f;  // filament f's bond j joins its sites j and j+1
  double r1[3], r2[3], s[3], u[3], len;
  for (int i = 0; i < 3; ++i) {
    r1[i] = d.r[i][site];
    r2[i] = d.r[i][site + 1];
  }
  bond_from_sites<ND>(d.rep[rep_of_bond(d, b)].hinv, r1, r2, s, u, len);
  store_geom<ND>(d, buf, b, s, u, len, prec);
  if (write_ub) {
    d.ub[0][b] = u[0];
    d.ub[1][b] = u[1];
    d.ub[2][b] = u[2];
  }
}

// ---------------------------------------------------------------------------
// Cell list.

template <int ND>
__global__ void k_bond_cells(SysConst k, DevState d, int *xyz) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  bond_cell<ND>(d, d.rep[rep_of_bond(d, b)], b, xyz + 3 * (size_t)b);
}

// Bonds of the systems whose list is rebuilt in this pass: global cell key
// and cell counts.
template <int ND>
__global__ void k_bin_count(SysConst k, DevState d, int *key, int *cell_count) {
  grid_dep_sync();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = b < d.nb;
  int c = -1;
  if (active) {
    const int r = rep_of_bond(d, b);
    if (d.due[r]) {
      const ReplicaConst &R = d.rep[r];
      int xyz[3];
      c = R.cell0 + bond_cell<ND>(d, R, b, xyz);
      key[b] = c;
    } else {
      active = false;
    }
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
__global__ void k_bin_scatter(DevState d, const int *key, const int *cell_start,
                              int *cell_count, int *sorted) {
  grid_dep_sync();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb || !d.due[rep_of_bond(d, b)]) return;
  int c = key[b];
  int slot = atomicSub(&cell_count[c], 1) - 1;
  sorted[cell_start[c] + slot] = b;
}

// One thread per cell head (first entry of a cell in the sorted order):
// restores insertion order inside its cell (bond order, as Cell::AddObj
// appends in interactor order), then counts the pairs the cell contributes
// (zero for every other entry, so that the scan over all bonds sees only
// heads).  The sorted order holds the bonds of the systems rebuilt in this
// pass, cell_start[n_cells] of them.  A pair is dropped only between
// adjacent bonds of one filament, or always without like-like interactions
// (pair_excluded), so a half-shell neighbour cell contributes m * m_nbr
// pairs less one for each of the cell's bonds whose filament neighbour
// (b - 1 or b + 1) lies in it -- told by that bond's cell key.  No thread
// reads another cell's members, which their heads are sorting meanwhile.
__global__ void k_cell_sort_count(SysConst k, DevState d, int nb, const int *key, int *sorted,
                                  const int *cell_start, int *pair_count, const unsigned *occ) {
  grid_dep_sync();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nb) return;
  if (q >= cell_start[k.n_cells]) {
    pair_count[q] = 0;
    return;
  }
  // Any entry of a cell names a member of it, also while its head sorts.
  const int c = key[sorted[q]];
  if (cell_start[c] != q) {
    pair_count[q] = 0;
    return;
  }
  const int m = cell_start[c + 1] - q;
  int *it = sorted + q;
  for (int i = 1; i < m; ++i) {  // insertion sort (cells are small)
    int v = it[i], j = i - 1;
    while (j >= 0 && it[j] > v) {
      it[j + 1] = it[j];
      --j;
    }
    it[j + 1] = v;
  }
  if (!k.like_like) {
    pair_count[q] = 0;
    return;
  }
  const ReplicaConst &R = d.rep[rep_of_bond(d, it[0])];
  int x, y, z, nbr[13];
  cell_coords(R, c - R.cell0, x, y, z);
  const unsigned keep = half_shell_fixed(k, R, x, y, z, nbr);
  long long cnt = (long long)m * (m - 1) / 2;
#pragma unroll
  for (int kk = 0; kk < 13; ++kk) {  // all ranges loaded together
    nbr[kk] += R.cell0;
    if ((keep >> kk) & 1u) {
      if (cell_occupied(occ, nbr[kk]))
        cnt += (long long)m * (cell_start[nbr[kk] + 1] - cell_start[nbr[kk]]);
    } else {
      nbr[kk] = -1;  // matches no cell key
    }
  }
  for (int i = 0; i < m; ++i) {
    const int a = it[i], fa = d.bond_fil[a];
    if (a + 1 < nb && d.bond_fil[a + 1] == fa) {
      const int ka = key[a + 1];
      if (ka == c) --cnt;  // each adjacent pair inside the cell, once
#pragma unroll
      for (int kk = 0; kk < 13; ++kk) cnt -= ka == nbr[kk];
    }
    if (a > 0 && d.bond_fil[a - 1] == fa) {
      const int ka = key[a - 1];
#pragma unroll
      for (int kk = 0; kk < 13; ++kk) cnt -= ka == nbr[kk];
    }
  }
  pair_count[q] = cnt > 0x3fffffff ? 0x3fffffff : (int)cnt;
}

// Writes each cell's pairs at its offset in its system's pair segment, in the
// reference's list order (Cell::MakePairs, src/cell.cpp:14-22): pairs inside
// the cell, then with each half-shell neighbour; clears each new pair's
// stored force and counts per-bond pair entries for the CSR.
__global__ void k_pair_emit(SysConst k, DevState d, int nb, const int *key,
                            const int *sorted, const int *cell_start,
                            const int *pair_off, int *deg, int prec, const unsigned *occ) {
  grid_dep_sync();
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < d.nrep) rep_pairs(d, q, cell_start, pair_off);
  if (q >= cell_start[k.n_cells]) return;
  int c = key[sorted[q]];
  if (cell_start[c] != q) return;
  const ReplicaConst &R = d.rep[rep_of_bond(d, sorted[q])];
  int m = cell_start[c + 1] - q;
  const int *it = sorted + q;
  // Offset within the system: its pairs start at its first cell's head.
  int p = pair_off[q] - pair_off[cell_start[R.cell0]];
  int x, y, z, nbr[13];
  cell_coords(R, c - R.cell0, x, y, z);
  const unsigned keep = half_shell_fixed(k, R, x, y, z, nbr);
  auto emit = [&](int a, int b) {
    if (pair_excluded(k, d, a, b)) return;
    if (p < R.pcap) {
      const int g = R.p0 + p;
      d.pa[g] = a;
      d.pb[g] = b;
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
      atomicAdd(&deg[a], 1);
      atomicAdd(&deg[b], 1);
    }
    ++p;
  };
  for (int i = 0; i < m - 1; ++i)
    for (int j = i + 1; j < m; ++j) emit(it[i], it[j]);
  int s0[13], s1[13];
#pragma unroll
  for (int kk = 0; kk < 13; ++kk) {  // all ranges loaded together
    s0[kk] = s1[kk] = 0;
    const int cn = R.cell0 + nbr[kk];
    if (((keep >> kk) & 1u) && cell_occupied(occ, cn)) {
      s0[kk] = cell_start[cn];
      s1[kk] = cell_start[cn + 1];
    }
  }
#pragma unroll
  for (int kk = 0; kk < 13; ++kk)
    for (int i = 0; i < m; ++i)
      for (int j = s0[kk]; j < s1[kk]; ++j) emit(it[i], sorted[j]);
}

// Per-bond entry ranges of the rebuilt systems, inside their slot segments,
// from the exclusive scan of the degrees over all bonds.
__global__ void k_csr_offsets(DevState d, const int *deg_off, const int *deg) {
  grid_dep_sync();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  const int r = rep_of_bond(d, b);
  if (!d.due[r]) return;
  const ReplicaConst &R = d.rep[r];
  d.e_off[b] = 2 * R.p0 + (deg_off[b] - deg_off[R.b0]);
  d.e_cnt[b] = deg[b];
}

// Entries (pair << 1 | role) of every bond of the rebuilt systems; role 0 =
// obj1, 1 = obj2.  The degree array is decremented back to zero.
__global__ void k_csr_fill(DevState d, int *deg) {
  grid_dep_sync();
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= d.pcap_total) return;
  int r;
  if (!pair_live(d, p, r) || !d.due[r]) return;
  int a = d.pa[p], b = d.pb[p];
  int sa = atomicSub(&deg[a], 1) - 1;
  int sb = atomicSub(&deg[b], 1) - 1;
  d.e_ent[d.e_off[a] + sa] = p << 1;
  d.e_ent[d.e_off[b] + sb] = (p << 1) | 1;
}

// Sorts each bond's entries by pair index = the order in which the
// reference's serial ApplyPairInteractions adds them to the bond, then
// records the slot of each (pair, role) entry.
__global__ void k_csr_sort_pos(DevState d) {
  grid_dep_sync();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb || !d.due[rep_of_bond(d, b)]) return;
  int e0 = d.e_off[b], e1 = e0 + d.e_cnt[b];
  int *e = d.e_ent;
  for (int i = e0 + 1; i < e1; ++i) {
    int v = e[i], j = i - 1;
    while (j >= e0 && e[j] > v) {
      e[j + 1] = e[j];
      --j;
    }
    e[j + 1] = v;
  }
  for (int i = e0; i < e1; ++i) {
    const int ent = e[i];
    if (ent & 1) d.pos2[ent >> 1] = i;
    else d.pos1[ent >> 1] = i;
  }
}

// InteractionManager::ZeroDrTot (src/interaction_manager.cpp:316-321) for
// the systems rebuilt in this pass.
__global__ void k_zero_dr(DevState d) {
  grid_dep_sync();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *d.n_rebuilds += 1;
  if (i < d.nrep && d.due[i]) {
    d.dr_max_bits[i] = 0ull;
    d.rep_rebuilds[i] += 1;
  }
  if (i >= d.ns) return;
  if (!d.due[d.fil[d.site_fil[i]].rep]) return;
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

// Sum of each tile of SCAN_TILE elements.
template <bool VEC>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const int *in, int n, int *tile_sums) {
  grid_dep_sync();
  __shared__ int red[SCAN_BLOCK / 32];
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int sum = 0;
  if (VEC && base + SCAN_ITEMS <= n) {
    const int4 a = reinterpret_cast<const int4 *>(in + base)[0];
    const int4 b = reinterpret_cast<const int4 *>(in + base)[1];
    sum = a.x + a.y + a.z + a.w + b.x + b.y + b.z + b.w;
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) sum += (base + i < n) ? in[base + i] : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < SCAN_BLOCK / 32; ++w) t += red[w];
    tile_sums[blockIdx.x] = t;
  }
}

// Exclusive scan of each tile, offset by the sum of the tiles before it,
// which every block adds up for itself (no block waits on another); the
// last tile's block writes the total to out[n].  With occ, also one bit per
// element: set where the element is non-zero (the occupied cells).
template <bool VEC>
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_down(const int *in, int *out, int n,
                                                         const int *tile_sums, unsigned *occ) {
  grid_dep_sync();
  __shared__ int tmp[SCAN_BLOCK / 32];
  __shared__ int red[SCAN_BLOCK / 32];
  // Sum of the earlier tiles: independent loads, then a block reduction.
  int p0 = 0, p1 = 0, p2 = 0, p3 = 0;
  const int nt = (int)blockIdx.x;
  int t = threadIdx.x;
  for (; t + 3 * SCAN_BLOCK < nt; t += 4 * SCAN_BLOCK) {
    p0 += tile_sums[t];
    p1 += tile_sums[t + SCAN_BLOCK];
    p2 += tile_sums[t + 2 * SCAN_BLOCK];
    p3 += tile_sums[t + 3 * SCAN_BLOCK];
  }
  for (; t < nt; t += SCAN_BLOCK) p0 += tile_sums[t];
  int pre = (p0 + p1) + (p2 + p3);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pre += __shfl_xor_sync(0xffffffffu, pre, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pre;
  const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS], sum = 0;
  const bool full = base + SCAN_ITEMS <= n;
  if (VEC && full) {
    const int4 a = reinterpret_cast<const int4 *>(in + base)[0];
    const int4 b = reinterpret_cast<const int4 *>(in + base)[1];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) v[i] = (base + i < n) ? in[base + i] : 0;
  }
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) sum += v[i];
  int total;
  int run = block_exclusive_scan(sum, tmp, total);  // synchronises: red[] is complete
  int offset = 0;
#pragma unroll
  for (int w = 0; w < SCAN_BLOCK / 32; ++w) offset += red[w];
  run += offset;
  int r[SCAN_ITEMS];
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; ++i) {
    r[i] = run;
    run += v[i];
  }
  if (VEC && full) {
    reinterpret_cast<int4 *>(out + base)[0] = make_int4(r[0], r[1], r[2], r[3]);
    reinterpret_cast<int4 *>(out + base)[1] = make_int4(r[4], r[5], r[6], r[7]);
  } else {
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
      if (base + i < n) out[base + i] = r[i];
  }
  if (occ) {  // four threads' 8 elements make one 32-bit word
    unsigned m = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) m |= (v[i] != 0 ? 1u : 0u) << i;
    const int sh = (threadIdx.x & 3) * 8;
    unsigned w = m << sh;
    w |= __shfl_down_sync(0xffffffffu, w, 2);
    w |= __shfl_down_sync(0xffffffffu, w, 1);
    const int word = (blockIdx.x * SCAN_TILE) / 32 + (threadIdx.x >> 2);
    if ((threadIdx.x & 3) == 0 && word * 32 < n) occ[word] = w;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = offset + total;
}

// ---------------------------------------------------------------------------
// Pair stage.  One thread per candidate pair evaluates it once
// (ProcessPairInteraction + the torque cross products of
// CalculatePairInteractions, src/interaction_manager.cpp:323-397, 466-471)
// and writes its signed contributions -- (+F, +t1) for obj1, (-F, -t2) for
// obj2 -- into the two per-bond slots the pair owns.  Every bond's slots are
// sorted by pair index, so summing them in slot order repeats the
// reference's serial scatter ApplyPairInteractions
// (src/interaction_manager.cpp:500-517) operation for operation; x - y and
// x + (-y) are the same IEEE operation.
//
// A pair whose potential is not evaluated this step keeps the force of its
// last evaluation since the list was built: the reference never clears an
// Interaction's force (src/minimum_distance.cpp:31-34 resets only dr and the
// contacts), and the pair's thread owns that stored force.

// A bond's FP64 geometry recomputed from its sites, with the operations of
// Bond::ReInit (src/bond.cpp:22-37) -- what the FP64 path's geometry holds.
template <int ND>
__device__ __forceinline__ void bond_geom_from_sites(const DevState &d, const ReplicaConst &R,
                                                     int b, BondGeomF64 &G) {
  const int site = b + d.bond_fil[b];
  double r1[3], r2[3];
  for (int i = 0; i < 3; ++i) {
    r1[i] = d.r[i][site];
    r2[i] = d.r[i][site + 1];
  }
  bond_from_sites<ND>(R.hinv, r1, r2, G.s, G.u, G.len);
  G.pad = 0.0;
}

// Nearly parallel contacts of the mixed pair stage, which FP32 cannot
// evaluate: segments within 0.18 degrees of parallel (FP32 |u1 x u2|^2,
// accurate where 1 - (u1 . u2)^2 is rounding alone, above 0 and below 1e-5)
// that lie side by side -- their projections on A's axis overlap, or nearly
// -- and near enough to interact, or that carry a stored force.  Side by
// side, the closest points can be anywhere along the overlap, and which end
// the reference picks hangs on orientation bits FP32 does not hold; such
// pairs are evaluated in FP64, from the sites (pair_eval_fp64_sites).
// Nearly parallel segments that do not overlap (the next-nearest bonds of a
// straight filament) meet at a unique pair of facing ends, which FP32 finds.
// Exactly parallel FP32 orientations take the parallel branch in both
// precisions (their FP64 1 - c^2 is below the reference's 1e-12).
template <int ND>
__device__ __forceinline__ bool near_parallel(const SysConst &k, const float *hf,
                                              const BondGeomF32 &A, const BondGeomF32 &B,
                                              const float4 &st) {
  // Cheap rejection first, with the operations sphero_f32 repeats (so they
  // are shared): for unit vectors 1 - (u1 . u2)^2 = |u1 x u2|^2, and the two
  // FP32 evaluations differ by less than 2e-6 here, so no pair the exact
  // test below flags is rejected.
  float c = 0.f;
#pragma unroll
  for (int i = 0; i < ND; ++i) c = __fmaf_rn(A.u[i], B.u[i], c);
  if (!(__fmaf_rn(-c, c, 1.0f) < k.npx_s2 + 2e-6f)) return false;
  float s2;
  const float cz = __fmaf_rn(A.u[0], B.u[1], -A.u[1] * B.u[0]);
  if (ND == 3) {
    const float cx = __fmaf_rn(A.u[1], B.u[2], -A.u[2] * B.u[1]);
    const float cy = __fmaf_rn(A.u[2], B.u[0], -A.u[0] * B.u[2]);
    s2 = __fmaf_rn(cx, cx, __fmaf_rn(cy, cy, cz * cz));
  } else {
    s2 = cz * cz;
  }
  if (!(s2 > 0.f && s2 < k.npx_s2)) return false;
  float dr[3] = {0.f, 0.f, 0.f}, a1 = 0.f, r2 = 0.f;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const int32_t dq = (int32_t)((uint32_t)B.q[j] - (uint32_t)A.q[j]);
      acc = __fmaf_rn(hf[ND * i + j], (float)dq * 2.3283064365386963e-10f, acc);
    }
    dr[i] = acc;
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    a1 = __fmaf_rn(dr[i], A.u[i], a1);
    r2 = __fmaf_rn(dr[i], dr[i], r2);
  }
  if (fabsf(a1) > A.hl + B.hl + 0.25f) return false;  // end to end: facing ends
  const bool loaded = st.x != 0.f || st.y != 0.f || st.z != 0.f;
  return loaded || r2 - a1 * a1 < 1.5f * k.rcut2f;
}

// A nearly parallel pair of the mixed pair stage, evaluated as the FP64 path
// evaluates it -- from both bonds' FP64 sites, which both paths share -- and
// written as the pair stage writes every pair (its two slots, its stored
// force, its virial record).
template <int ND>
__device__ __forceinline__ void pair_eval_fp64_sites(const SysConst &k, const DevState &d,
                                                  const ReplicaConst &R, int p) {
  const int a = d.pa[p], b = d.pb[p];
  BondGeomF64 A64, B64;
  bond_geom_from_sites<ND>(d, R, a, A64);
  bond_geom_from_sites<ND>(d, R, b, B64);
  PairGeom<double> g;
  sphero_f64<ND>(R.h, A64, B64, g);
  float4 *stale = reinterpret_cast<float4 *>(d.pf32) + (size_t)p;
  const float4 st = *stale;
  double f[3] = {st.x, st.y, st.z}, rec[4];
  if (wca_f64<ND>(k, g, f, k.thermo ? rec : nullptr)) {
    if (ND == 2) f[2] = st.z;
    *stale = make_float4((float)f[0], (float)f[1], (float)f[2], 0.f);
    if (k.thermo)
      reinterpret_cast<float4 *>(d.pv32)[p] =
          make_float4((float)rec[0], (float)rec[1], (float)rec[2], (float)rec[3]);
  }
  double t1[3], t2[3];
  cross3(g.c1, f, t1);
  cross3(g.c2, f, t2);
  float4 *c1 = reinterpret_cast<float4 *>(d.cf32) + 2 * (size_t)d.pos1[p];
  float4 *c2 = reinterpret_cast<float4 *>(d.cf32) + 2 * (size_t)d.pos2[p];
  c1[0] = make_float4((float)f[0], (float)f[1], (float)f[2], (float)t1[0]);
  c1[1] = make_float4((float)t1[1], (float)t1[2], 0.f, 0.f);
  c2[0] = make_float4(-(float)f[0], -(float)f[1], -(float)f[2], -(float)t2[0]);
  c2[1] = make_float4(-(float)t2[1], -(float)t2[2], 0.f, 0.f);
}

// What the FP64 evaluation of one nearly parallel pair reads and writes,
// passed by value so that the evaluation can be a separate function.
struct NearParallelArgs {
  const double *r0, *r1, *r2;
  const int *bond_fil, *pa, *pb, *pos1, *pos2;
  float *pf32, *pv32, *cf32;
  const ReplicaConst *R;
  double rcut2, c12, c6, fcut, eps;
  int thermo;
};

// One nearly parallel pair of the mixed pair stage, evaluated from the FP64
// sites (pair_eval_fp64_sites) by the thread that met it.  Not inlined: the
// FP64 evaluation's registers and spills stay in this function, which runs
// for a few pairs in ten thousand, and the FP32 path of k_pair_eval keeps its
// register budget.
template <int ND>
__device__ __noinline__ void eval_near_parallel(NearParallelArgs a, int p) {
  SysConst k;
  k.rcut2 = a.rcut2;
  k.c12 = a.c12;
  k.c6 = a.c6;
  k.fcut = a.fcut;
  k.eps = a.eps;
  k.thermo = a.thermo;
  DevState d;
  d.r[0] = const_cast<double *>(a.r0);
  d.r[1] = const_cast<double *>(a.r1);
  d.r[2] = const_cast<double *>(a.r2);
  d.bond_fil = a.bond_fil;
  d.pa = const_cast<int *>(a.pa);
  d.pb = const_cast<int *>(a.pb);
  d.pos1 = const_cast<int *>(a.pos1);
  d.pos2 = const_cast<int *>(a.pos2);
  d.pf32 = a.pf32;
  d.pv32 = a.pv32;
  d.cf32 = a.cf32;
  pair_eval_fp64_sites<ND>(k, d, *a.R, p);
}

// Pair slot indices, written by the rebuild: a pair kernel may load them
// before it waits for the kernel just before it (which never writes them).
struct PairIdx {
  int a, b, s1, s2;
};
__device__ __forceinline__ PairIdx pair_idx(const DevState &d, int p) {
  return PairIdx{d.pa[p], d.pb[p], d.pos1[p], d.pos2[p]};
}

// One pair of the pair stage.  Mixed with NPX: returns false, having
// written nothing, for a nearly parallel pair, which the caller evaluates in
// FP64 (eval_near_parallel) outside its loop over pairs.
template <int ND, int PREC, bool NPX>
__device__ __forceinline__ bool pair_eval_one(const SysConst &k, const DevState &d,
                                              const ReplicaConst &R, int rbuf, int p,
                                              const PairIdx &ix) {
  const int a = ix.a, b = ix.b;
  const int s1 = ix.s1, s2 = ix.s2;
  if (PREC == 0) {
    const BondGeomF64 A = d.g64[rbuf][a], B = d.g64[rbuf][b];
    double2 *stale = reinterpret_cast<double2 *>(d.pf64) + 2 * (size_t)p;
    const double2 st0 = stale[0], st1 = stale[1];
    PairGeom<double> g;
    sphero_f64<ND>(R.h, A, B, g);
    double force[3], rec[4];
    if (!wca_f64<ND>(k, g, force, k.thermo ? rec : nullptr)) {
      force[0] = st0.x;
      force[1] = st0.y;
      force[2] = st1.x;
    } else {
      if (ND == 2) force[2] = st1.x;
      stale[0] = make_double2(force[0], force[1]);
      stale[1] = make_double2(force[2], 0.0);
      if (k.thermo) {
        double2 *v = reinterpret_cast<double2 *>(d.pv64) + 2 * (size_t)p;
        v[0] = make_double2(rec[0], rec[1]);
        v[1] = make_double2(rec[2], rec[3]);
      }
    }
    double t1[3], t2[3];
    cross3(g.c1, force, t1);
    cross3(g.c2, force, t2);
    double2 *c1 = reinterpret_cast<double2 *>(d.cf64) + 4 * (size_t)s1;
    double2 *c2 = reinterpret_cast<double2 *>(d.cf64) + 4 * (size_t)s2;
    c1[0] = make_double2(force[0], force[1]);
    c1[1] = make_double2(force[2], t1[0]);
    c1[2] = make_double2(t1[1], t1[2]);
    c2[0] = make_double2(-force[0], -force[1]);
    c2[1] = make_double2(-force[2], -t2[0]);
    c2[2] = make_double2(-t2[1], -t2[2]);
    return true;
  } else {
    const BondGeomF32 A = d.g32[rbuf][a], B = d.g32[rbuf][b];
    float4 *stale = reinterpret_cast<float4 *>(d.pf32) + (size_t)p;
    const float4 st = *stale;
    if (NPX && near_parallel<ND>(k, R.hf, A, B, st)) return false;
    float force[3], rec[4], t1[3], t2[3];
    const bool set = pair_force_f32<ND>(k, R.hf, A, B, st, force, t1, t2,
                                        k.thermo ? rec : nullptr);
    if (set) {
      *stale = make_float4(force[0], force[1], force[2], 0.f);
      if (k.thermo)
        reinterpret_cast<float4 *>(d.pv32)[p] = make_float4(rec[0], rec[1], rec[2], rec[3]);
    }
    float4 *c1 = reinterpret_cast<float4 *>(d.cf32) + 2 * (size_t)s1;
    float4 *c2 = reinterpret_cast<float4 *>(d.cf32) + 2 * (size_t)s2;
    c1[0] = make_float4(force[0], force[1], force[2], t1[0]);
    c1[1] = make_float4(t1[1], t1[2], 0.f, 0.f);
    c2[0] = make_float4(-force[0], -force[1], -force[2], -t2[0]);
    c2[1] = make_float4(-t2[1], -t2[2], 0.f, 0.f);
    return true;
  }
}

// A nearly parallel pair of the mixed pair stage, in FP64 from the sites.
template <int ND>
__device__ __forceinline__ void near_parallel_fp64(const SysConst &k, const DevState &d,
                                                   const ReplicaConst &R, int p) {
  NearParallelArgs na;
  na.r0 = d.r[0];
  na.r1 = d.r[1];
  na.r2 = d.r[2];
  na.bond_fil = d.bond_fil;
  na.pa = d.pa;
  na.pb = d.pb;
  na.pos1 = d.pos1;
  na.pos2 = d.pos2;
  na.pf32 = d.pf32;
  na.pv32 = d.pv32;
  na.cf32 = d.cf32;
  na.R = &R;
  na.rcut2 = k.rcut2;
  na.c12 = k.c12;
  na.c6 = k.c6;
  na.fcut = k.fcut;
  na.eps = k.eps;
  na.thermo = k.thermo;
  eval_near_parallel<ND>(na, p);
}

// Grid-stride over the pair slots, so a captured launch stays correct
// whatever length the lists grow to between captures.  A single system's
// list is the prefix of its segment; with several systems every slot checks
// that it holds a current pair of its system.
// NPX (mixed only): nearly parallel pairs are evaluated in FP64
// (eval_near_parallel) by the thread that meets them.
// The list and its slot indices date from the last rebuild, whose kernels
// completed before the kernel just before this one waited (every kernel
// waits before it lets the next one start): they are loaded before the
// wait; the bond geometry, which that kernel may be writing, after it.
template <int ND, int PREC, bool NPX, int BLOCK>
__global__ void __launch_bounds__(BLOCK, NPX ? 1024 / BLOCK : 1)
    k_pair_eval(SysConst k, DevState d, int rbuf) {
  if (d.nrep == 1) {
    const ReplicaConst &R = d.rep[0];
    const int np = min(d.np_rep[0], R.pcap);
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    PairIdx ix = {0, 0, 0, 0};
    if (p < np) ix = pair_idx(d, p);
    grid_dep_sync();
    // The grid covers the list (it is sized for it), so a thread has one
    // pair: a nearly parallel one is evaluated in FP64 after the FP32 work,
    // out of any loop.  Pairs past the grid (a list that grew after the
    // launch was sized) are handled by the loop below.
    const int stride = gridDim.x * blockDim.x;
    int flagged = -1;
    if (p < np && !pair_eval_one<ND, PREC, NPX>(k, d, R, rbuf, p, ix)) flagged = p;
    for (p += stride; p < np; p += stride)
      if (!pair_eval_one<ND, PREC, NPX>(k, d, R, rbuf, p, pair_idx(d, p)))
        if (NPX) near_parallel_fp64<ND>(k, d, R, p);
    if (NPX && flagged >= 0) near_parallel_fp64<ND>(k, d, R, flagged);
    return;
  }
  grid_dep_sync();
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < d.pcap_total;
       p += gridDim.x * blockDim.x) {
    int r;
    if (pair_live(d, p, r) && !pair_eval_one<ND, PREC, NPX>(k, d, d.rep[r], rbuf, p, pair_idx(d, p)))
      if (NPX) near_parallel_fp64<ND>(k, d, d.rep[r], p);
  }
}

// Bond force/torque accumulators (Bond::force_ / torque_ after Interact),
// for sc_interact and the getters.
template <int ND, int PREC>
__global__ void k_bond_sum(DevState d) {
  grid_dep_sync();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nb) return;
  double F[3], T[3];
  bond_pair_sum<ND, PREC>(d, b, d.e_off[b], d.e_off[b] + d.e_cnt[b], F, T);
  for (int i = 0; i < 3; ++i) {
    d.bF[i][b] = F[i];
    d.bT[i][b] = T[i];
  }
}

// Crosslink tethers, recomputed on even steps (CrosslinkSpecies::
// UpdateBoundCrosslinks, src/crosslink_species.cpp:218-258), one thread per
// link.  Each anchor is placed on its bond re-initialised from the current
// sites (Bond::ReInit, src/bond.cpp:22-37, then Anchor::
// UpdateAnchorPositionToBond, src/anchor.cpp:236-249, and
// periodic_boundary_conditions); the tether follows Crosslink::
// CalculateTetherForces (src/crosslink.cpp:247-275) with MinimumDistance::
// PointPoint (src/minimum_distance.cpp:71-101); each anchor's force and its
// torque (lambda - l/2) u x f are stored as Anchor::ApplyAnchorForces
// (src/anchor.cpp:132-146) computes them, for re-use on the odd step.
// Mesh::UpdateBondPositions' mesh lambdas (src/mesh.cpp:324-330): one thread
// per filament sums its bonds' current lengths in order, each bond taking
// the sum before it, and records the total (Mesh::true_length_).  The
// lengths are Bond::ReInit's (src/bond.cpp:22-37), from the sites.
template <int ND>
__global__ void k_mesh_lambda(DevState d) {
  grid_dep_sync();
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int s0 = d.fil[f].site0, nbf = d.fil[f].n - 1, b0 = s0 - f;
  double true_length = 0.0;
  double r1[3], r2[3];
#pragma unroll
  for (int i = 0; i < ND; ++i) r1[i] = d.r[i][s0];
  for (int q = 0; q < nbf; ++q) {
    double l = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      r2[i] = d.r[i][s0 + q + 1];
      const double u = r2[i] - r1[i];
      l += u * u;
    }
    l = sqrt(l);
    d.bml[b0 + q] = true_length;
    true_length += l;
#pragma unroll
    for (int i = 0; i < ND; ++i) r1[i] = r2[i];
  }
  d.ftl[f] = true_length;
}

// Bond::ReInit of bond b from its sites (src/bond.cpp:22-37): unwrapped
// centre, unit orientation, length.
template <int ND>
__device__ __forceinline__ double bond_reinit(const DevState &d, int b, double pos[3],
                                              double u[3]) {
  const int s1 = b + d.bond_fil[b];
  double l = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) pos[i] = u[i] = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    u[i] = d.r[i][s1 + 1] - d.r[i][s1];
    l += u[i] * u[i];
  }
  l = sqrt(l);
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    pos[i] = d.r[i][s1] + 0.5 * u[i];
    u[i] /= l;
  }
  return l;
}

// Crosslink tethers, recomputed on even steps (CrosslinkSpecies::
// UpdateBoundCrosslinks, src/crosslink_species.cpp:218-258), one thread per
// link, after k_mesh_lambda.  Each anchor follows its mesh lambda as the
// reference's Anchor::UpdateAnchorPositionToMesh (src/anchor.cpp:45-68)
// does for a bound anchor with end pausing: CheckMesh (:180-201) clamps the
// mesh lambda to [0, true length]; Mesh::GetBondAtLambda (src/mesh.cpp:
// 667-675) picks a bond from the nominal bond length; CalcBondLambda
// (:70-111) measures lambda from that bond's mesh lambda and moves once to
// a neighbouring bond when lambda falls outside it; UpdateAnchorPositionToBond
// (:236-249) places the anchor, then periodic_boundary_conditions.  The
// tether follows Crosslink::CalculateTetherForces (src/crosslink.cpp:
// 247-275) with MinimumDistance::PointPoint (src/minimum_distance.cpp:
// 71-101); each anchor's force, torque and bond are stored as Anchor::
// ApplyAnchorForces (src/anchor.cpp:132-146) uses them, for re-use on the
// odd step.  An anchor that leaves the bonds it is listed on, or whose lambda
// ends outside its bond (where the reference stops with an error), sets
// ST_TETHER.
template <int ND>
__global__ void k_tether(SysConst k, DevState d) {
  grid_dep_sync();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= d.nx) return;
  if (*d.status & ST_LIST_OVERFLOW) return;  // the step stopped at its rebuild
  double sp[2][3], ua[2][3], len[2], lam[2];
  int bond[2];
  int rep = 0;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int A = 2 * x + a;
    const int f = d.xl_fil[A];
    const FilConst &fc = d.fil[f];
    const int nbf = fc.n - 1, b0 = fc.site0 - f;
    rep = fc.rep;  // both anchors lie in one system (checked when the links are added)
    const double tl = d.ftl[f];
    double M = d.xl_M[A];
    if (M < 0) M = 0;
    else if (M > tl) M = tl;
    d.xl_M[A] = M;
    int kb;
    if (M < 0) kb = 0;
    else if (M >= d.fil_L[f]) kb = nbf - 1;
    else kb = (int)floor(M / fc.l);
    // (M / l can round up to the bond count just below the nominal length,
    // where the reference would index past its bonds: kept on the last.)
    kb = min(max(kb, 0), nbf - 1);
    double pos[3], u[3];
    double bl = bond_reinit<ND>(d, b0 + kb, pos, u);
    double lm = M - d.bml[b0 + kb];
    if (lm < 0) {
      if (kb > 0) {
        --kb;
        bl = bond_reinit<ND>(d, b0 + kb, pos, u);
        lm = M - d.bml[b0 + kb];
      } else {
        lm = 0;
      }
    } else if (lm > bl) {
      if (kb < nbf - 1) {
        ++kb;
        bl = bond_reinit<ND>(d, b0 + kb, pos, u);
        lm = M - d.bml[b0 + kb];
      } else {
        lm = bl;
      }
    }
    bool listed = false;
    for (int e = d.xb_off[b0 + kb]; e < d.xb_off[b0 + kb + 1]; ++e) listed |= d.xb_ent[e] == A;
    if (lm < -1e-6 || lm > bl + 1e-6 || !listed) atomicOr(d.status, ST_TETHER);
    bond[a] = b0 + kb;
    len[a] = bl;
    lam[a] = lm;
    double ap[3] = {0, 0, 0};
#pragma unroll
    for (int i = 0; i < 3; ++i) ua[a][i] = u[i];
#pragma unroll
    for (int i = 0; i < ND; ++i) ap[i] = pos[i] - (0.5 * bl - lm) * u[i];
    const ReplicaConst &R = d.rep[rep];
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double v = 0.0;
#pragma unroll
      for (int j = 0; j < ND; ++j) v += R.hinv[ND * i + j] * ap[j];
      sp[a][i] = v - nint(v);
    }
  }
  const ReplicaConst &Rx = d.rep[rep];
  double dr[3] = {0, 0, 0}, dr2 = 0.0, f[3] = {0, 0, 0};
  double ds[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    ds[i] = sp[1][i] - sp[0][i];
    ds[i] -= nint(ds[i]);
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    double v = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) v += Rx.h[ND * i + j] * ds[j];
    dr[i] = v;
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) dr2 += dr[i] * dr[i];
  const double length = sqrt(dr2);
  const double stretch = length - k.xrest;
  const double tf = (k.xkc >= 0 && stretch < 0) ? k.xkc * stretch : k.xk * stretch;
#pragma unroll
  for (int i = 0; i < ND; ++i) f[i] = tf * (dr[i] / length);
  reinterpret_cast<double4 *>(d.xl_F)[x] = make_double4(f[0], f[1], f[2], 0.0);
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    double c[3] = {0.0, 0.0, 0.0}, dl[3] = {0.0, 0.0, 0.0}, t[3];
#pragma unroll
    for (int i = 0; i < ND; ++i) c[i] = a == 0 ? c[i] + f[i] : c[i] - f[i];
#pragma unroll
    for (int i = 0; i < ND; ++i) dl[i] = (lam[a] - 0.5 * len[a]) * ua[a][i];
    cross3(dl, c, t);
    double4 *o = reinterpret_cast<double4 *>(d.xl_c) + 2 * (size_t)(2 * x + a);
    o[0] = make_double4(c[0], c[1], c[2], t[0]);
    o[1] = make_double4(t[1], t[2], (double)bond[a], 0.0);
  }
}

// Host transfers: x, y, z triples <-> component arrays.
__global__ void k_aos_to_soa(int n, int nd, const double *aos, DevState d) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double v = c < nd ? aos[3 * (size_t)i + c] : 0.0;
    d.r[c][i] = v;
    d.rp[c][i] = v;
  }
}

// Filament averages (9 per filament) -> diffusion origins: average position
// (3) and average orientation (3) per filament.
__global__ void k_avg_to_origins(int nf, const double *avg, double *pos0, double *u0) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  for (int j = 0; j < 3; ++j) {
    pos0[3 * (size_t)f + j] = avg[9 * (size_t)f + j];
    u0[3 * (size_t)f + j] = avg[9 * (size_t)f + 6 + j];
  }
}

template <class T>
__global__ void k_soa_to_aos(int n, const T *x, const T *y, const T *z, double *aos) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  aos[3 * (size_t)i] = (double)x[i];
  aos[3 * (size_t)i + 1] = (double)y[i];
  aos[3 * (size_t)i + 2] = (double)z[i];
}

// Per filament: average site position, its scaled (periodic) image and the
// normalised average site orientation, 9 doubles, in the reference's
// summation order (Mesh::GetAvgPosition / GetAvgOrientation,
// src/mesh.cpp:581-608, then Object::UpdatePeriodic).  Site orientations are
// their bonds' (the last site's is the last bond's).
template <int ND>
__global__ void k_filament_averages(SysConst k, DevState d, double *out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const FilConst &fc = d.fil[f];
  double ap[3] = {0.0, 0.0, 0.0}, au[3] = {0.0, 0.0, 0.0};
  const int b0 = fc.site0 - f;
  for (int j = 0; j < fc.n; ++j) {
    const int b = b0 + (j < fc.n - 1 ? j : fc.n - 2);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      ap[i] += d.r[i][fc.site0 + j];
      au[i] += d.ub[i][b];
    }
  }
  double mag = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) mag += au[i] * au[i];
  mag = sqrt(mag);
#pragma unroll
  for (int i = 0; i < ND; ++i) au[i] /= mag;
#pragma unroll
  for (int i = 0; i < ND; ++i) ap[i] /= fc.n;
  const ReplicaConst &R = d.rep[fc.rep];
  double s[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < ND; ++i) {
#pragma unroll
    for (int j = 0; j < ND; ++j) s[i] += R.hinv[ND * i + j] * ap[j];
    s[i] -= nint(s[i]);
  }
  double *o = out + 9 * (size_t)f;
  for (int i = 0; i < 3; ++i) {
    o[i] = ap[i];
    o[3 + i] = s[i];
    o[6 + i] = au[i];
  }
}

// ---------------------------------------------------------------------------
// Filament analyses, one block per system, deterministic reduction order.

// Block sum of v (blockDim.x == 256) into thread 0.
__device__ __forceinline__ double block_sum256(double v, double *tmp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < 8; ++w) t += tmp[w];
  __syncthreads();
  return t;
}

// FilamentSpecies::RunMse2eAnalysis (src/filament_species.cpp:569-592):
// |head - tail|^2 and its square, summed over a system's filaments into
// acc[2 r]; and RunThetaAnalysis (:594-610): the histogram of each joint's
// cos(theta) = u_i . u_{i+1} into hist[(r max_joints + i) n_bins + bin].
template <int ND>
__global__ void __launch_bounds__(256) k_analysis_sample(DevState d, int n_bins, int max_joints,
                                                         double *acc, int *hist) {
  __shared__ double tmp[8];
  const int r = blockIdx.x;
  const ReplicaConst &R = d.rep[r];
  double m = 0.0, m2 = 0.0;
  for (int f = R.f0 + threadIdx.x; f < R.f0 + R.nf; f += blockDim.x) {
    const FilConst &fc = d.fil[f];
    const int tail = fc.site0, head = fc.site0 + fc.n - 1;
    double e = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      const double t = d.r[i][head] - d.r[i][tail];
      e += t * t;
    }
    m += e;
    m2 += e * e;
    const int b0 = fc.site0 - f;
    for (int j = 0; j < fc.n - 2 && j < max_joints; ++j) {
      double c = 0.0;
#pragma unroll
      for (int i = 0; i < ND; ++i) c += d.ub[i][b0 + j] * d.ub[i][b0 + j + 1];
      int bin = (int)floor((1 + c) * (n_bins / 2));
      if (bin >= n_bins) bin = n_bins - 1;
      if (bin < 0) bin = 0;
      atomicAdd(&hist[((size_t)r * max_joints + j) * n_bins + bin], 1);
    }
  }
  m = block_sum256(m, tmp);
  m2 = block_sum256(m2, tmp);
  if (threadIdx.x == 0) {
    acc[2 * r] += m;
    acc[2 * r + 1] += m2;
  }
}

// The reference's diffusion analysis (SpherocylinderSpecies::CalculateMSD,
// CalculateVCF, UpdateInitPositions; src/spherocylinder_species.cpp:62-121)
// on the filaments' average positions and orientations (avg, 9 per filament
// from k_filament_averages: Filament::UpdateAvgPosition), one block per
// system: the mean over its filaments of |r - r0|^2 and of u . u0 and their
// second moments, each weighted by the inverse variance into window point t
// of acc (per system: msd, msd weight, vcf, vcf weight, each `interval`
// long); when the window closes (restart) the current averages become the
// new origins (pos0, u0: 3 each per filament).
template <int ND>
__global__ void __launch_bounds__(256) k_diffusion_sample(DevState d, const double *avg,
                                                          double *pos0, double *u0,
                                                          double *acc, int t, int interval,
                                                          int restart) {
  __shared__ double tmp[8];
  const int r = blockIdx.x;
  const ReplicaConst &R = d.rep[r];
  double q[4] = {0.0, 0.0, 0.0, 0.0};
  for (int f = R.f0 + threadIdx.x; f < R.f0 + R.nf; f += blockDim.x) {
    const double *a = avg + 9 * (size_t)f;
    double sqr_diff = 0.0, udotu0 = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const double r_diff = a[j] - pos0[3 * (size_t)f + j];
      sqr_diff += r_diff * r_diff;
    }
#pragma unroll
    for (int j = 0; j < ND; ++j) udotu0 += a[6 + j] * u0[3 * (size_t)f + j];
    q[0] += sqr_diff;
    q[1] += sqr_diff * sqr_diff;
    q[2] += udotu0;
    q[3] += udotu0 * udotu0;
  }
  for (int k2 = 0; k2 < 4; ++k2) q[k2] = block_sum256(q[k2], tmp);
  if (threadIdx.x == 0) {
    double *o = acc + 4 * (size_t)interval * r;
    const double n = R.nf;
    const double m = q[0] / n, m2 = q[1] / n, v = q[2] / n, v2 = q[3] / n;
    const double s_msd = m2 - m * m, s_vcf = v2 - v * v;
    o[t] += m / s_msd;
    o[interval + t] += 1.0 / s_msd;
    o[2 * interval + t] += v / s_vcf;
    o[3 * interval + t] += 1.0 / s_vcf;
  }
  if (restart)  // each thread replaces only the origins it read
    for (int f = R.f0 + threadIdx.x; f < R.f0 + R.nf; f += blockDim.x)
      for (int j = 0; j < 3; ++j) {
        pos0[3 * (size_t)f + j] = avg[9 * (size_t)f + j];
        u0[3 * (size_t)f + j] = avg[9 * (size_t)f + 6 + j];
      }
}

// FilamentSpecies::RunGlobalOrderAnalysis (src/filament_species.cpp:486-535)
// with Filament::GetPolarOrder / GetNematicOrder (src/filament.cpp:488-516):
// per system, the mean over filaments of the mean bond orientation (3) and
// of the bond nematic tensor 2 u u - I (9, n_dim stride 3).
template <int ND>
__global__ void __launch_bounds__(256) k_global_order(DevState d, double *out) {
  __shared__ double tmp[8];
  const int r = blockIdx.x;
  const ReplicaConst &R = d.rep[r];
  double acc[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) acc[q] = 0.0;
  for (int f = R.f0 + threadIdx.x; f < R.f0 + R.nf; f += blockDim.x) {
    const FilConst &fc = d.fil[f];
    const int b0 = fc.site0 - f, nbf = fc.n - 1;
    double p[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < nbf; ++j) {
      double u[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        u[i] = d.ub[i][b0 + j];
        p[i] += u[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i)
#pragma unroll
        for (int k2 = 0; k2 < ND; ++k2)
          acc[3 + 3 * i + k2] += (i == k2 ? 2 * u[i] * u[k2] - 1 : 2 * u[i] * u[k2]) / nbf;
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) acc[i] += p[i] / nbf;
  }
  double *o = out + 12 * (size_t)r;
  for (int q = 0; q < 12; ++q) {
    const double t = block_sum256(acc[q], tmp);
    if (threadIdx.x == 0) o[q] = t / R.nf;
  }
}

// ---------------------------------------------------------------------------
// Host launchers.

static inline int cdiv(long long a, int b) { return (int)((a + b - 1) / b); }

// Programmatic dependent launch: on unless SIMCORE_PDL=0; PdlOff switches it
// off for the launches of its thread while it lives.
static bool pdl_default() {
  const char *v = std::getenv("SIMCORE_PDL");
  return !(v && v[0] == '0');
}
static thread_local bool t_pdl_off = false;
bool pdl_enabled() {
  static const bool on = pdl_default();
  return on && !t_pdl_off;
}
PdlOff::PdlOff() : prev(t_pdl_off) { t_pdl_off = true; }
PdlOff::~PdlOff() { t_pdl_off = prev; }

void launch_init_geometry(const SysConst &k, const DevState &d, int buf,
                          int prec, cudaStream_t st, bool write_ub) {
  if (d.nb == 0) return;
  const int w = write_ub ? 1 : 0;
  if (k.n_dim == 3) k_init_geometry<3><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, buf, prec, w);
  else k_init_geometry<2><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, buf, prec, w);
}

int scan_temp_ints(long long n) { return cdiv(n, SCAN_TILE) + 1; }

int launch_analysis_sample(const SysConst &k, const DevState &d, int n_bins, int max_joints,
                           double *acc, int *hist, cudaStream_t st) {
  if (k.n_dim == 3) k_analysis_sample<3><<<d.nrep, 256, 0, st>>>(d, n_bins, max_joints, acc, hist);
  else k_analysis_sample<2><<<d.nrep, 256, 0, st>>>(d, n_bins, max_joints, acc, hist);
  return 1;
}

int launch_aos_to_origins(int nf, const double *avg, double *pos0, double *u0,
                          cudaStream_t st) {
  k_avg_to_origins<<<cdiv(nf, 256), 256, 0, st>>>(nf, avg, pos0, u0);
  return 1;
}

int launch_diffusion_sample(const SysConst &k, const DevState &d, const double *avg,
                            double *pos0, double *u0, double *acc, int t, int interval,
                            int restart, cudaStream_t st) {
  if (k.n_dim == 3)
    k_diffusion_sample<3><<<d.nrep, 256, 0, st>>>(d, avg, pos0, u0, acc, t, interval, restart);
  else
    k_diffusion_sample<2><<<d.nrep, 256, 0, st>>>(d, avg, pos0, u0, acc, t, interval, restart);
  return 1;
}

int launch_global_order(const SysConst &k, const DevState &d, double *out, cudaStream_t st) {
  if (k.n_dim == 3) k_global_order<3><<<d.nrep, 256, 0, st>>>(d, out);
  else k_global_order<2><<<d.nrep, 256, 0, st>>>(d, out);
  return 1;
}

int launch_filament_averages(const SysConst &k, const DevState &d, double *out, cudaStream_t st) {
  if (d.nf <= 0) return 0;
  if (k.n_dim == 3) k_filament_averages<3><<<cdiv(d.nf, 128), 128, 0, st>>>(k, d, out);
  else k_filament_averages<2><<<cdiv(d.nf, 128), 128, 0, st>>>(k, d, out);
  return 1;
}

int launch_aos_to_soa(int n, int nd, const double *aos, const DevState &d, cudaStream_t st) {
  if (n <= 0) return 0;
  k_aos_to_soa<<<cdiv(n, 256), 256, 0, st>>>(n, nd, aos, d);
  return 1;
}

template <class T>
int launch_soa_to_aos(int n, const T *x, const T *y, const T *z, double *aos, cudaStream_t st) {
  if (n <= 0) return 0;
  k_soa_to_aos<T><<<cdiv(n, 256), 256, 0, st>>>(n, x, y, z, aos);
  return 1;
}
template int launch_soa_to_aos<double>(int, const double *, const double *, const double *,
                                       double *, cudaStream_t);

// Exclusive scan in[0..n) -> out[0..n], out[n] = total.  tmp holds
// scan_temp_ints(n) ints.  Returns launches issued.
int launch_exclusive_scan(const int *in, int *out, long long n, int *tmp, cudaStream_t st,
                          unsigned *occ) {
  int tiles = cdiv(n, SCAN_TILE);
  if (tiles == 0) tiles = 1;
  const bool vec = (((uintptr_t)in | (uintptr_t)out) & 15u) == 0;
  if (vec) {
    launch_pdl(k_scan_reduce<true>, dim3(tiles), dim3(SCAN_BLOCK), 0, st, in, (int)n, tmp);
    launch_pdl(k_scan_down<true>, dim3(tiles), dim3(SCAN_BLOCK), 0, st, in, out, (int)n, tmp, occ);
  } else {
    launch_pdl(k_scan_reduce<false>, dim3(tiles), dim3(SCAN_BLOCK), 0, st, in, (int)n, tmp);
    launch_pdl(k_scan_down<false>, dim3(tiles), dim3(SCAN_BLOCK), 0, st, in, out, (int)n, tmp, occ);
  }
  return 2;
}

int launch_bin_count(const SysConst &k, const DevState &d, int *key,
                     int *cell_count, cudaStream_t st) {
  if (k.n_dim == 3) launch_pdl(k_bin_count<3>, dim3(cdiv(d.nb, 256)), dim3(256), 0, st, k, d, key, cell_count);
  else launch_pdl(k_bin_count<2>, dim3(cdiv(d.nb, 256)), dim3(256), 0, st, k, d, key, cell_count);
  return 1;
}

int launch_bond_cells(const SysConst &k, const DevState &d, int *xyz,
                      cudaStream_t st) {
  if (k.n_dim == 3) k_bond_cells<3><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, xyz);
  else k_bond_cells<2><<<cdiv(d.nb, 256), 256, 0, st>>>(k, d, xyz);
  return 1;
}

int launch_bin_scatter(const DevState &d, const int *key, const int *cell_start,
                       int *cell_count, int *sorted, cudaStream_t st) {
  launch_pdl(k_bin_scatter, dim3(cdiv(d.nb, 256)), dim3(256), 0, st, d, key, cell_start, cell_count, sorted);
  return 1;
}

int launch_cell_sort_count(const SysConst &k, const DevState &d, const int *key,
                           int *sorted, const int *cell_start, int *pair_count,
                           cudaStream_t st, const unsigned *occ) {
  launch_pdl(k_cell_sort_count, dim3(cdiv(d.nb, 128)), dim3(128), 0, st, k, d, d.nb, key, sorted, cell_start,
                                                     pair_count, occ);
  return 1;
}

int launch_pair_emit(const SysConst &k, const DevState &d, const int *key,
                     const int *sorted, const int *cell_start,
                     const int *pair_off, int *deg, int prec,
                     cudaStream_t st, const unsigned *occ) {
  launch_pdl(k_pair_emit, dim3(cdiv(d.nb, 128)), dim3(128), 0, st, k, d, d.nb, key, sorted, cell_start,
                                               pair_off, deg, prec, occ);
  return 1;
}

int launch_csr(const DevState &d, int *deg, const int *deg_off, cudaStream_t st) {
  launch_pdl(k_csr_offsets, dim3(cdiv(d.nb, 256)), dim3(256), 0, st, d, deg_off, deg);
  launch_pdl(k_csr_fill, dim3(cdiv(d.pcap_total > 0 ? d.pcap_total : 1, 256)), dim3(256), 0, st, d, deg);
  launch_pdl(k_csr_sort_pos, dim3(cdiv(d.nb, 256)), dim3(256), 0, st, d);
  return 3;
}

// ---------------------------------------------------------------------------
// Device-side control of captured step graphs.

// Interact's rebuild check on the device for the next BD step of a graph
// loop (CheckUpdateInteractions + GetDrMax, src/interaction_manager.cpp:
// 284-312, include/simcore/species.hpp:114-118), one block: each system is
// due when its displacement maximum (reduced on the device by the last full
// step) is above its threshold; above 10000 the reference throws, here the
// status word records it and no rebuild runs.  Sets the rebuild node's
// condition h_if.
__device__ void decide_systems(const DevState &d, cudaGraphConditionalHandle h_if) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < d.nrep; r += blockDim.x) {
    const double dr = __longlong_as_double((long long)d.dr_max_bits[r]);
    int due = 0;
    if (dr > 10000.0 || !(dr == dr)) atomicOr(d.status, ST_UNPHYSICAL);
    else due = dr > d.rep[r].dr_update ? 1 : 0;
    d.due[r] = due;
    if (due) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h_if, any ? 1u : 0u);
}

// Start of a graph loop: the loop condition and the first step's rebuild
// decision.
__global__ void k_loop_head(DevState d, cudaGraphConditionalHandle h,
                            cudaGraphConditionalHandle h_if, int decide) {
  if (decide) decide_systems(d, h_if);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, *d.loop_count > 0 ? 1u : 0u);
}

// End of one BD step (midstep + full step) of a graph loop: advances the
// noise counter, decrements the remaining count and decides the next step's
// rebuild.  A recorded error stops the loop.  A step whose rebuild
// overflowed its list did nothing past the rebuild: it stays counted as
// remaining, so the host can grow the list, redo the rebuild and resume
// with it.
__global__ void k_loop_tail(DevState d, int stoch, cudaGraphConditionalHandle h,
                            cudaGraphConditionalHandle h_if, int decide) {
  const unsigned status = *d.status;  // the same word for every thread
  if (status & ST_LIST_OVERFLOW) {
    if (threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
    return;
  }
  if (threadIdx.x == 0) {
    if (stoch) *d.mcount += 1ull;
    int left = *d.loop_count - 1;
    if (status != 0u) left = 0;
    *d.loop_count = left;
    cudaGraphSetConditional(h, left > 0 ? 1u : 0u);
  }
  if (decide) decide_systems(d, h_if);
}

__global__ void k_advance_mcount(DevState d) {
  grid_dep_sync();
  *d.mcount += 1ull;
}

int launch_loop_head(const DevState &d, cudaGraphConditionalHandle h,
                     cudaGraphConditionalHandle h_if, int decide, cudaStream_t st) {
  k_loop_head<<<1, 256, 0, st>>>(d, h, h_if, decide);
  return 1;
}

int launch_loop_tail(const DevState &d, int stoch, cudaGraphConditionalHandle h,
                     cudaGraphConditionalHandle h_if, int decide, cudaStream_t st) {
  k_loop_tail<<<1, 256, 0, st>>>(d, stoch, h, h_if, decide);
  return 1;
}

int launch_advance_mcount(const DevState &d, cudaStream_t st) {
  launch_pdl(k_advance_mcount, dim3(1), dim3(1), 0, st, d);
  return 1;
}

int launch_zero_dr(const DevState &d, cudaStream_t st) {
  const int n = d.ns > d.nrep ? d.ns : d.nrep;
  launch_pdl(k_zero_dr, dim3(cdiv(n > 0 ? n : 1, 256)), dim3(256), 0, st, d);
  return 1;
}

template <int BLOCK>
static void launch_pairs_block(const SysConst &k, const DevState &d, int rbuf, int prec, int grid,
                               cudaStream_t st, bool npx) {
  if (k.n_dim == 3) {
    if (prec == 0) launch_pdl(k_pair_eval<3, 0, false, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
    else if (!npx) launch_pdl(k_pair_eval<3, 1, false, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
    else launch_pdl(k_pair_eval<3, 1, true, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
  } else {
    if (prec == 0) launch_pdl(k_pair_eval<2, 0, false, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
    else if (!npx) launch_pdl(k_pair_eval<2, 1, false, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
    else launch_pdl(k_pair_eval<2, 1, true, BLOCK>, dim3(grid), dim3(BLOCK), 0, st, k, d, rbuf);
  }
}

int launch_pairs(const SysConst &k, const DevState &d, int rbuf, int prec,
                 int expected, cudaStream_t st, bool npx, int block) {
  if (d.nrep > 1) expected = d.pcap_total;
  npx = npx && prec != 0;
  if (block == 128)
    launch_pairs_block<128>(k, d, rbuf, prec, cdiv(expected > 0 ? expected : 1, 128), st, npx);
  else
    launch_pairs_block<256>(k, d, rbuf, prec, cdiv(expected > 0 ? expected : 1, 256), st, npx);
  return 1;
}

// ---------------------------------------------------------------------------
// Thermo.  One launch per step after the pair stage, while thermo is on.
// Every live pair's stress -dr x F from its record (the values of its last
// evaluation, like its force: src/minimum_distance.cpp:31-34 resets neither)
// is summed per system -- ApplyPairInteractions' stress_ += ix->stress
// (src/interaction_manager.cpp:511-516) -- and, every th_n steps,
// CalculatePressure (src/interaction_manager.cpp:535-559) turns the sum into
// the pressure tensor and pressure of the periodic box (volume (2R)^d,
// src/space.cpp:252-264; n_objs = the system's bond count, src/mesh.cpp:399)
// and resets it.  Grid (th_gx, systems): each block sums a fixed stride of
// its system's pairs and reduces in a fixed order; the last block of a
// system (ticket counter, no waiting) adds the block sums in block order.
// The sum order differs from the reference's serial one, so the result
// agrees to rounding, and is the same on every run.
template <int ND, int PREC>
__global__ void __launch_bounds__(256) k_thermo(SysConst k, DevState d) {
  grid_dep_sync();
  if (*d.status & ST_LIST_OVERFLOW) return;  // the step stopped at its rebuild
  const int r = blockIdx.y;
  const ReplicaConst &R = d.rep[r];
  const int np = min(d.np_rep[r], R.pcap);
  double s[ND * ND];
#pragma unroll
  for (int c = 0; c < ND * ND; ++c) s[c] = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
    const size_t p = (size_t)R.p0 + q;
    double F[3], dr[3];
    if (PREC == 0) {
      const double2 *f = reinterpret_cast<const double2 *>(d.pf64) + 2 * p;
      const double2 *v = reinterpret_cast<const double2 *>(d.pv64) + 2 * p;
      const double2 f0 = f[0], f1 = f[1], v0 = v[0], v1 = v[1];
      F[0] = f0.x;
      F[1] = f0.y;
      F[2] = f1.x;
      dr[0] = v0.x;
      dr[1] = v0.y;
      dr[2] = v1.x;
    } else {
      const float4 f = reinterpret_cast<const float4 *>(d.pf32)[p];
      const float4 v = reinterpret_cast<const float4 *>(d.pv32)[p];
      F[0] = f.x;
      F[1] = f.y;
      F[2] = f.z;
      dr[0] = v.x;
      dr[1] = v.y;
      dr[2] = v.z;
    }
#pragma unroll
    for (int i = 0; i < ND; ++i)
#pragma unroll
      for (int j = 0; j < ND; ++j) s[ND * i + j] += -dr[i] * F[j];
  }
  __shared__ double red[8][ND * ND];
  __shared__ int last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < ND * ND; ++c) {
    double v = s[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double *part = d.th_part + ((size_t)r * gridDim.x + blockIdx.x) * 9;
    for (int c = 0; c < ND * ND; ++c) {
      double v = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][c];
      part[c] = v;
    }
    __threadfence();
    last = atomicAdd(&d.th_ticket[r], 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  const volatile double *part = d.th_part + (size_t)r * gridDim.x * 9;
  double *acc = d.th_acc + 9 * (size_t)r;
  for (int c = 0; c < ND * ND; ++c) {
    double v = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) v += part[(size_t)b * 9 + c];
    acc[c] += v;
  }
  d.th_ticket[r] = 0u;
  const long long istep = ++d.th_istep[r];
  if (d.th_n <= 0 || istep % d.th_n != 0) return;
  const double side = R.h[0];
  const double volume = ND == 2 ? side * side : side * side * side;
  const double inv_V = 1.0 / volume;
  double P[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < ND; ++i)
    for (int j = 0; j < ND; ++j) {
      if (i == j) P[ND * i + j] += R.nb * inv_V;
      P[ND * i + j] += acc[ND * i + j] * inv_V / d.th_n;
    }
  double pressure = 0;
  for (int i = 0; i < ND; ++i) pressure += P[ND * i + i];
  pressure /= ND;
  for (int c = 0; c < 9; ++c) acc[c] = 0.0;
  const long long n = d.th_nrec[r]++;
  double *rec = d.th_rec + ((size_t)(n % d.th_cap) * d.nrep + r) * 12;
  rec[0] = (double)istep;
  for (int c = 0; c < 9; ++c) rec[1 + c] = P[c];
  rec[10] = pressure;
  rec[11] = volume;
}

// Object::GetPotentialEnergy of every filament after the last pair stage:
// Filament::ApplyInteractionForces adds its bonds' potentials in bond order
// (src/filament.cpp:1007), each bond's the potentials of its pairs in list
// order (obj1/obj2->AddPotential, src/interaction_manager.cpp:509-510) --
// the order of its entries, which are sorted by pair.
template <int PREC>
__global__ void k_potential(DevState d, double *out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const FilConst fc = d.fil[f];
  const int b0 = fc.site0 - f;
  double e = 0.0;
  for (int i = 0; i < fc.n - 1; ++i) {
    const int b = b0 + i;
    double bp = 0.0;
    for (int q = d.e_off[b], q1 = q + d.e_cnt[b]; q < q1; ++q) {
      const size_t p = (size_t)(d.e_ent[q] >> 1);
      bp += PREC == 0 ? d.pv64[4 * p + 3] : (double)d.pv32[4 * p + 3];
    }
    e += bp;
  }
  out[f] = e;
}

int launch_thermo(const SysConst &k, const DevState &d, int prec, cudaStream_t st) {
  const dim3 grid(d.th_gx, d.nrep);
  if (k.n_dim == 3) {
    if (prec == 0) launch_pdl(k_thermo<3, 0>, dim3(grid), dim3(256), 0, st, k, d);
    else launch_pdl(k_thermo<3, 1>, dim3(grid), dim3(256), 0, st, k, d);
  } else {
    if (prec == 0) launch_pdl(k_thermo<2, 0>, dim3(grid), dim3(256), 0, st, k, d);
    else launch_pdl(k_thermo<2, 1>, dim3(grid), dim3(256), 0, st, k, d);
  }
  return 1;
}

int launch_potential(const DevState &d, int prec, double *out, cudaStream_t st) {
  if (prec == 0) k_potential<0><<<cdiv(d.nf, 128), 128, 0, st>>>(d, out);
  else k_potential<1><<<cdiv(d.nf, 128), 128, 0, st>>>(d, out);
  return 1;
}

int launch_tether(const SysConst &k, const DevState &d, cudaStream_t st) {
  if (d.nx == 0) return 0;
  if (k.n_dim == 3) {
    launch_pdl(k_mesh_lambda<3>, dim3(cdiv(d.nf, 128)), dim3(128), 0, st, d);
    launch_pdl(k_tether<3>, dim3(cdiv(d.nx, 128)), dim3(128), 0, st, k, d);
  } else {
    launch_pdl(k_mesh_lambda<2>, dim3(cdiv(d.nf, 128)), dim3(128), 0, st, d);
    launch_pdl(k_tether<2>, dim3(cdiv(d.nx, 128)), dim3(128), 0, st, k, d);
  }
  return 2;
}

int launch_bond_sum(const SysConst &k, const DevState &d, int prec, cudaStream_t st) {
  int grid = cdiv(d.nb, 256);
  if (k.n_dim == 3) {
    if (prec == 0) launch_pdl(k_bond_sum<3, 0>, dim3(grid), dim3(256), 0, st, d);
    else launch_pdl(k_bond_sum<3, 1>, dim3(grid), dim3(256), 0, st, d);
  } else {
    if (prec == 0) launch_pdl(k_bond_sum<2, 0>, dim3(grid), dim3(256), 0, st, d);
    else launch_pdl(k_bond_sum<2, 1>, dim3(grid), dim3(256), 0, st, d);
  }
  return 1;
}

size_t integrate_smem_bytes(int C, int max_filaments) {
  // (shared by both integrator units)
  return sizeof(double) * integrate_smem_doubles(C) + sizeof(int) * (size_t)(C / 2) +
         sizeof(FilConst) * (size_t)max_filaments;
}

template <int ND, int PREC, int MAXC>
static void set_attr(size_t smem) {
  cudaFuncSetAttribute(k_integrate<ND, PREC, false, MAXC>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(k_integrate<ND, PREC, false, MAXC, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

void prepare_integrate(int C) {
  size_t smem = integrate_smem_bytes(C, C / 2);
  if (C <= 128) {
    set_attr<3, 0, 128>(smem);
    set_attr<3, 1, 128>(smem);
    set_attr<2, 0, 128>(smem);
    set_attr<2, 1, 128>(smem);
  } else if (C <= 192) {
    set_attr<3, 0, 192>(smem);
    set_attr<3, 1, 192>(smem);
    set_attr<2, 0, 192>(smem);
    set_attr<2, 1, 192>(smem);
  } else if (C <= 256) {
    set_attr<3, 0, 256>(smem);
    set_attr<3, 1, 256>(smem);
    set_attr<2, 0, 256>(smem);
    set_attr<2, 1, 256>(smem);
  } else {
    set_attr<3, 0, 512>(smem);
    set_attr<3, 1, 512>(smem);
    set_attr<2, 0, 512>(smem);
    set_attr<2, 1, 512>(smem);
  }
  prepare_integrate_fast(C);
}

int launch_integrate(const SysConst &k, const DevState &d, int nblocks, int C,
                     int midstep, int rbuf, int interaction, int capture,
                     int prec, bool fast, cudaStream_t st, bool fuse) {
  if (fast && prec == 1)
    return launch_integrate_fast(k, d, nblocks, C, midstep, rbuf, interaction, capture, st,
                                 fuse && interaction);
  int launched = 0;
  if (d.n_wg > 0) {
    const int grid = cdiv(d.n_wg, kIntWarps);
#define SC_INTEGRATE_WARP(ND, P)                                              \
  launch_pdl(k_integrate_warp<ND, P, false>, dim3(grid), dim3(kIntWarps * 32), 0, st, k, d, midstep, rbuf, \
                                                                  interaction, capture)
    if (k.n_dim == 3) {
      if (prec == 0) SC_INTEGRATE_WARP(3, 0); else SC_INTEGRATE_WARP(3, 1);
    } else {
      if (prec == 0) SC_INTEGRATE_WARP(2, 0); else SC_INTEGRATE_WARP(2, 1);
    }
#undef SC_INTEGRATE_WARP
    ++launched;
  }
  if (nblocks == 0) return launched;
  size_t smem = integrate_smem_bytes(C, d.blk_maxf);
#define SC_INTEGRATE(ND, P, MC)                                                                  \
  ((C == MC) ? launch_pdl(k_integrate<ND, P, false, MC, false, true>, dim3(nblocks), dim3(C), smem, \
                          st, k, d, midstep, rbuf, interaction, capture)                        \
             : launch_pdl(k_integrate<ND, P, false, MC>, dim3(nblocks), dim3(C), smem, st, k, d,  \
                          midstep, rbuf, interaction, capture))
  if (C <= 128) {
    if (k.n_dim == 3) {
      if (prec == 0) SC_INTEGRATE(3, 0, 128); else SC_INTEGRATE(3, 1, 128);
    } else {
      if (prec == 0) SC_INTEGRATE(2, 0, 128); else SC_INTEGRATE(2, 1, 128);
    }
  } else if (C <= 192) {
    if (k.n_dim == 3) {
      if (prec == 0) SC_INTEGRATE(3, 0, 192); else SC_INTEGRATE(3, 1, 192);
    } else {
      if (prec == 0) SC_INTEGRATE(2, 0, 192); else SC_INTEGRATE(2, 1, 192);
    }
  } else if (C <= 256) {
    if (k.n_dim == 3) {
      if (prec == 0) SC_INTEGRATE(3, 0, 256); else SC_INTEGRATE(3, 1, 256);
    } else {
      if (prec == 0) SC_INTEGRATE(2, 0, 256); else SC_INTEGRATE(2, 1, 256);
    }
  } else {
    if (k.n_dim == 3) {
      if (prec == 0) SC_INTEGRATE(3, 0, 512); else SC_INTEGRATE(3, 1, 512);
    } else {
      if (prec == 0) SC_INTEGRATE(2, 0, 512); else SC_INTEGRATE(2, 1, 512);
    }
  }
#undef SC_INTEGRATE
  return launched + 1;
}

}  // namespace sc
