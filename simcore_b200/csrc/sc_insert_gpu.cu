// Random insertion with overlap rejection, the overlap tests on the GPU
// (sc_insert_filaments_gpu).  Same result as the host insertion
// (sc_insert_filaments) for the same arguments, bit for bit.
//
// The host insertion places filaments one after another (longest first):
// each attempt draws a candidate from one Philox stream and is redrawn while
// any of its bonds comes closer than the diameter to an accepted bond
// (InteractionManager::CheckOverlap, src/interaction_manager.cpp:561-571).
// An attempt's draws depend only on its filament, so the stream position of
// every attempt is known once the outcomes of the earlier ones are.  The
// batched version guesses that the next B filaments all succeed at their
// next attempt: the host draws those B candidates at their stream positions
// (the same code as the host insertion), and the GPU tests every candidate
// bond against the accepted bonds and against the bonds of every earlier
// candidate of the batch.  The first candidate m that overlaps anything
// (an earlier candidate counts, since before m all are accepted) is where
// the guess fails: candidates 0..m-1 are accepted, exactly as the sequential
// loop accepts them, and m's filament retries from the stream position after
// its failed attempt.  The batch grows while guesses hold and shrinks when
// they fail early.
//
// Compiled with --fmad=false, like the host code, so the squared distances
// compared with the diameter are the host's bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "sc_host_philox.h"
#include "simcore_gpu.h"

uint64_t sc_insert_candidate(int n_dim, double system_radius, double diameter,
                             int insertion_type, int nb, double length, double lp,
                             uint32_t k0, uint32_t k1, uint64_t k, double *pos, double *cen,
                             double *axis);

namespace {

struct GridDims {
  int n_dim, n1d;
  double L;
};

__device__ __forceinline__ int ins_coord(const GridDims &g, double x) {
  double s = x / g.L + 0.5;
  s -= floor(s);
  const int c = (int)(s * g.n1d);
  return c >= g.n1d ? g.n1d - 1 : c;
}

__device__ __forceinline__ int ins_cell(const GridDims &g, const double *c) {
  const int x = ins_coord(g, c[0]), y = ins_coord(g, c[1]);
  const int z = g.n_dim == 3 ? ins_coord(g, c[2]) : 0;
  return (x * g.n1d + y) * (g.n_dim == 3 ? g.n1d : 1) + z;
}

__device__ __forceinline__ double ins_clamp(double x, double h) {
  return x > h ? h : (x < -h ? -h : x);
}

// The host insertion's segment distance (seg_dist2), operation for operation.
__device__ double ins_seg_dist2(int n_dim, const double *c1, const double *u1, double h1,
                                const double *c2, const double *u2, double h2, double L) {
  double dr[3] = {0, 0, 0};
  for (int i = 0; i < n_dim; ++i) {
    double d = c2[i] - c1[i];
    d -= L * rint(d / L);
    dr[i] = d;
  }
  const double a = dr[0] * u1[0] + dr[1] * u1[1] + dr[2] * u1[2];
  const double b = dr[0] * u2[0] + dr[1] * u2[1] + dr[2] * u2[2];
  const double c = u1[0] * u2[0] + u1[1] * u2[1] + u1[2] * u2[2];
  const double den = 1.0 - c * c;
  double lam, mu;
  if (den < 1e-12) {
    lam = 0.5 * a;
    mu = -0.5 * b;
  } else {
    lam = (a - c * b) / den;
    mu = (-b + c * a) / den;
  }
  double best = 1e300;
  for (int pass = 0; pass < 3; ++pass) {
    double l2, m2;
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
    double r2 = 0;
    for (int i = 0; i < 3; ++i) {
      const double d = dr[i] - l2 * u1[i] + m2 * u2[i];
      r2 += d * d;
    }
    if (r2 < best) best = r2;
  }
  return best;
}

// Bonds in a grid of cells of at least (longest bond + diameter): per cell
// a linked list (head per cell, next per bond); per bond centre, axis, half
// length and its candidate (batch bonds) .
struct BondSet {
  int *head, *next, *owner;
  double *c, *u, *h;
};

// Batch bonds into the batch grid.
__global__ void k_ins_bin(GridDims g, BondSet s, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cell = ins_cell(g, s.c + 3 * (size_t)i);
  s.next[i] = atomicExch(&s.head[cell], i);
}

// Every batch bond against the accepted bonds and the bonds of earlier
// candidates: the smallest candidate with an overlap goes to *first_bad.
__global__ void k_ins_check(GridDims g, BondSet acc, BondSet bat, int n, double d2max,
                            int *first_bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int m = bat.owner[i];
  if (m >= *(volatile int *)first_bad) return;  // a smaller one failed already
  const double *c = bat.c + 3 * (size_t)i, *u = bat.u + 3 * (size_t)i;
  const double h = bat.h[i];
  const int cx = ins_coord(g, c[0]), cy = ins_coord(g, c[1]);
  const int cz = g.n_dim == 3 ? ins_coord(g, c[2]) : 0, zr = g.n_dim == 3 ? 1 : 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -zr; dz <= zr; ++dz) {
        const int x = (cx + dx + g.n1d) % g.n1d, y = (cy + dy + g.n1d) % g.n1d;
        const int z = g.n_dim == 3 ? (cz + dz + g.n1d) % g.n1d : 0;
        const int cell = (x * g.n1d + y) * (g.n_dim == 3 ? g.n1d : 1) + z;
        for (int o = acc.head[cell]; o >= 0; o = acc.next[o])
          if (ins_seg_dist2(g.n_dim, c, u, h, acc.c + 3 * (size_t)o, acc.u + 3 * (size_t)o,
                            acc.h[o], g.L) < d2max) {
            atomicMin(first_bad, m);
            return;
          }
        for (int o = bat.head[cell]; o >= 0; o = bat.next[o])
          if (bat.owner[o] < m &&
              ins_seg_dist2(g.n_dim, c, u, h, bat.c + 3 * (size_t)o, bat.u + 3 * (size_t)o,
                            bat.h[o], g.L) < d2max) {
            atomicMin(first_bad, m);
            return;
          }
      }
}

// The accepted candidates' bonds (those of candidates below first_bad) join
// the accepted set; every batch bond leaves the batch grid.
__global__ void k_ins_accept(GridDims g, BondSet acc, BondSet bat, int n, int n_acc,
                             const int *first_bad, int *accepted_bonds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *c = bat.c + 3 * (size_t)i;
  bat.head[ins_cell(g, c)] = -1;
  if (bat.owner[i] >= *first_bad) return;
  // Batch bonds of accepted candidates come first, in order: i is the index.
  const int id = n_acc + i;
  for (int k = 0; k < 3; ++k) {
    acc.c[3 * (size_t)id + k] = c[k];
    acc.u[3 * (size_t)id + k] = bat.u[3 * (size_t)i + k];
  }
  acc.h[id] = bat.h[i];
  acc.next[id] = atomicExch(&acc.head[ins_cell(g, c)], id);
  atomicAdd(accepted_bonds, 1);
}

struct DeviceBuffers {
  std::vector<void *> ptrs;
  ~DeviceBuffers() {
    for (void *p : ptrs) cudaFree(p);
  }
  template <class T>
  bool alloc(T **p, size_t n) {
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    ptrs.push_back(q);
    *p = (T *)q;
    return true;
  }
};

}  // namespace

extern "C" int sc_insert_filaments_gpu(int device, int n_dim, double system_radius,
                                       uint64_t seed, int n_fil, const int *n_bonds,
                                       const double *length, const double *persistence_length,
                                       double diameter, int insertion_type, int max_attempts,
                                       double *site_xyz) {
  if ((n_dim != 2 && n_dim != 3) || n_fil <= 0 || !n_bonds || !length ||
      !persistence_length || !site_xyz || system_radius <= diameter ||
      insertion_type < SC_INSERT_RANDOM || insertion_type > SC_INSERT_RANDOM_POLAR)
    return SC_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return SC_ERR_NO_DEVICE;
  }
  const double L = 2.0 * system_radius;
  double max_bond = 0;
  size_t total_bonds = 0;
  int max_nb = 0;
  for (int f = 0; f < n_fil; ++f) {
    if (n_bonds[f] < 2) return SC_ERR_INVALID_ARG;
    max_bond = std::fmax(max_bond, length[f] / n_bonds[f]);
    total_bonds += (size_t)n_bonds[f];
    max_nb = std::max(max_nb, n_bonds[f]);
  }
  if (total_bonds >= (1u << 30)) return SC_ERR_INVALID_ARG;
  // The host insertion's grid (its Grid: cells of at least max bond + d).
  GridDims g;
  g.n_dim = n_dim;
  g.L = L;
  g.n1d = (int)std::floor(L / (max_bond + diameter));
  if (g.n1d < 3) g.n1d = 3;
  if (g.n1d > (n_dim == 3 ? 400 : 8000)) g.n1d = n_dim == 3 ? 400 : 8000;
  const size_t n_cells = (size_t)g.n1d * g.n1d * (n_dim == 3 ? g.n1d : 1);

  // Batches hold at most kMaxBatch candidates and kMaxBatchBonds bonds.
  const int kMaxBatch = 8192;
  const size_t kMaxBatchBonds = std::max<size_t>((size_t)1 << 18, (size_t)max_nb);
  DeviceBuffers mem;
  BondSet acc, bat;
  int *first_bad = nullptr, *accepted_bonds = nullptr;
  if (!mem.alloc(&acc.head, n_cells) || !mem.alloc(&acc.next, total_bonds) ||
      !mem.alloc(&acc.c, 3 * total_bonds) || !mem.alloc(&acc.u, 3 * total_bonds) ||
      !mem.alloc(&acc.h, total_bonds) || !mem.alloc(&bat.head, n_cells) ||
      !mem.alloc(&bat.next, kMaxBatchBonds) || !mem.alloc(&bat.owner, kMaxBatchBonds) ||
      !mem.alloc(&bat.c, 3 * kMaxBatchBonds) || !mem.alloc(&bat.u, 3 * kMaxBatchBonds) ||
      !mem.alloc(&bat.h, kMaxBatchBonds) || !mem.alloc(&first_bad, 1) ||
      !mem.alloc(&accepted_bonds, 1))
    return SC_ERR_OOM;
  acc.owner = nullptr;
  cudaStream_t st = 0;
  if (cudaMemsetAsync(acc.head, 0xff, sizeof(int) * n_cells, st) != cudaSuccess ||
      cudaMemsetAsync(bat.head, 0xff, sizeof(int) * n_cells, st) != cudaSuccess) {
    cudaGetLastError();
    return SC_ERR_CUDA;
  }

  // The host insertion's order, stream and site layout.
  std::vector<size_t> site_at(n_fil + 1, 0);
  for (int f = 0; f < n_fil; ++f) site_at[f + 1] = site_at[f] + n_bonds[f] + 1;
  std::vector<int> order(n_fil);
  for (int f = 0; f < n_fil; ++f) order[f] = f;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return length[a] > length[b]; });
  const uint32_t k0 = (uint32_t)seed ^ (uint32_t)(seed >> 32), k1 = 0xC0FFEEu;
  uint64_t kpos = 0;

  std::vector<double> pos, hc, hu, hh;  // batch: sites, bond centres, axes, half lengths
  std::vector<int> howner;
  std::vector<size_t> cand_site;        // per candidate: offset of its sites in pos
  std::vector<uint64_t> cand_end;       // per candidate: stream position after it
  int batch = 64, oi = 0, attempts_here = 0, n_acc = 0;
  while (oi < n_fil) {
    // Candidates of filaments order[oi], order[oi + 1], ..., each its next
    // attempt, at the stream positions they take if all before succeed.
    pos.clear();
    hc.clear();
    hu.clear();
    hh.clear();
    howner.clear();
    cand_site.clear();
    cand_end.clear();
    uint64_t k = kpos;
    int m = 0;
    for (; m < batch && oi + m < n_fil; ++m) {
      const int f = order[oi + m], nb = n_bonds[f];
      if (hh.size() + nb > kMaxBatchBonds) break;
      const size_t p0 = pos.size(), b0 = hh.size();
      pos.resize(p0 + 3 * (nb + 1));
      hc.resize(3 * (b0 + nb));
      hu.resize(3 * (b0 + nb));
      k = sc_insert_candidate(n_dim, system_radius, diameter, insertion_type, nb, length[f],
                              persistence_length[f], k0, k1, k, pos.data() + p0,
                              hc.data() + 3 * b0, hu.data() + 3 * b0);
      const double half = 0.5 * (length[f] / nb);
      for (int b = 0; b < nb; ++b) {
        hh.push_back(half);
        howner.push_back(m);
      }
      cand_site.push_back(p0);
      cand_end.push_back(k);
    }
    const int n_cand = m, nbat = (int)hh.size();
    const int big = 0x7fffffff;
    cudaError_t e = cudaSuccess;
    e = cudaMemcpyAsync(bat.c, hc.data(), sizeof(double) * hc.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(bat.u, hu.data(), sizeof(double) * hu.size(), cudaMemcpyHostToDevice,
                          st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(bat.h, hh.data(), sizeof(double) * hh.size(), cudaMemcpyHostToDevice,
                          st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(bat.owner, howner.data(), sizeof(int) * howner.size(),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(first_bad, &big, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return SC_ERR_CUDA;
    }
    const int grid = (nbat + 255) / 256;
    k_ins_bin<<<grid, 256, 0, st>>>(g, bat, nbat);
    k_ins_check<<<grid, 256, 0, st>>>(g, acc, bat, nbat, diameter * diameter, first_bad);
    k_ins_accept<<<grid, 256, 0, st>>>(g, acc, bat, nbat, n_acc, first_bad, accepted_bonds);
    int bad = big;
    e = cudaMemcpyAsync(&bad, first_bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return SC_ERR_CUDA;
    }
    const int n_ok = std::min(bad, n_cand);
    for (int q = 0; q < n_ok; ++q) {
      const int f = order[oi + q];
      std::memcpy(site_xyz + 3 * site_at[f], pos.data() + cand_site[q],
                  sizeof(double) * 3 * (n_bonds[f] + 1));
      n_acc += n_bonds[f];
    }
    if (n_ok > 0) attempts_here = 0;
    if (n_ok < n_cand) {
      // Candidate n_ok failed: its filament retries after its failed attempt.
      kpos = cand_end[n_ok];
      if (++attempts_here >= max_attempts) return SC_ERR_INSERTION;
      batch = std::max(16, n_ok > batch / 2 ? batch : batch / 2);
    } else {
      kpos = cand_end[n_cand - 1];
      batch = std::min(kMaxBatch, 2 * batch);
    }
    oi += n_ok;
  }
  return SC_OK;
}
