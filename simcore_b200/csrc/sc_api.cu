// C ABI of the B200 filament step (include/simcore_gpu.h): context,
// device memory, rebuild orchestration and the step loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_launch.h"
#include "simcore_gpu.h"

using sc::DevState;
using sc::SysConst;

struct sc_ctx {
  sc_system_desc desc{};
  int nd = 3;
  int prec = 0;
  SysConst k{};
  DevState d{};
  cudaStream_t st = nullptr;
  std::string err;
  std::vector<void *> allocs;  // every device allocation, freed at destroy

  // host mirrors
  int nf = 0, ns = 0, nb = 0;
  std::vector<int> site_off;
  std::vector<int> bond_fil;
  std::vector<int> fil_rep;        // system of each filament
  // per filament, for output files: diameter, length, bond length, lp
  std::vector<double> fil_diam, fil_len, fil_bl, fil_lp;

  // analyses (sc_analysis_*): device accumulators
  struct Analysis {
    int n_bins = 0, max_joints = 0;
    long long n_samples = 0;
    double *acc = nullptr;     // 2 per system
    int *hist = nullptr;       // nrep x max_joints x n_bins
    double *order = nullptr;   // 12 per system
  } an;

  // diffusion analysis (sc_diffusion_*): window of `interval` samples, the
  // next sample's point, origins and per-system sums (4 x interval each)
  struct Diffusion {
    int interval = 0, t = 0;
    long long n_samples = 0;
    double *avg = nullptr, *pos0 = nullptr, *u0 = nullptr, *acc = nullptr;
  } dif;

  // reference-format output (sc_output_*): one spec and one posit file per
  // system, frames snapshotted on the device and copied on out_st
  struct Output {
    bool open = false;
    int n_steps = 0, n_posit = 0, n_spec = 0;
    std::vector<FILE *> spec, posit;   // per system (null when not written)
    cudaStream_t out_st = nullptr;
    cudaEvent_t taken = nullptr, copied = nullptr;
    double *d_snap = nullptr;          // positions (3 ns) then averages (9 nf)
    double *h_snap = nullptr;          // pinned copy
    bool pending_spec = false, pending_posit = false;
  } out;
  bool loaded = false;

  // systems (replicas): host copy of the device table
  std::vector<sc::ReplicaConst> reps;
  std::vector<int> np_rep;         // pairs per system (last read back)

  // cell list and pair list storage
  int *key = nullptr, *cell_count = nullptr, *cell_start = nullptr;
  unsigned *cell_occ = nullptr;  // one bit per cell: occupied in the last rebuild
  int *sorted = nullptr, *pair_count = nullptr, *pair_off = nullptr;
  int *deg = nullptr, *deg_off = nullptr, *scan_tmp = nullptr, *cells_xyz = nullptr;
  double *stage = nullptr;         // interleaved host-transfer staging, 3 * max(ns, nb)
  long long np = 0, pcap = 0;      // pairs and slots of all systems

  // integrator blocks
  int nblocks = 0, C = 128;
  int warp_sites = 32;             // longest filament for the warp-synchronous kernel
  int block_sites = 0;             // sites per block of the block kernel (0: 128, 256 or 512)

  // control state
  long long i_step = 0, n_rebuilds = 0, launches = 0;
  int midstep = 1;                 // FilamentSpecies::midstep_
  unsigned long long mcount = 0;   // midsteps that drew noise
  int rbuf = 0;                    // geometry buffer read by the next pair stage
  int capture = 0;
  bool fast = true;                // mixed precision: contraction/reciprocal integrator
  bool pairs_ready = false;        // pair contributions of the next update exist

  // pinned readback slots
  struct Readback {
    unsigned long long dr_bits;
    unsigned status;
    int total;
  } *hb = nullptr;
  unsigned long long *h_dr = nullptr;  // per system displacement maxima
  int *h_np = nullptr;                 // per system pair counts
  int *h_due = nullptr;                // per system rebuild flags

  // CUDA graph: a WHILE loop of BD steps (sc_step_graph)
  cudaGraphExec_t graph_exec = nullptr;
  int graph_rbuf = -1;             // geometry buffer parity the graph was built for
  int *h_loop = nullptr;           // pinned loop count

  // optional per-launch timing of the step kernel (host-driven path)
  long long rebuild_kernels = 0;    // kernels in one rebuild sequence
  bool timing = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double timed_ms = 0.0;
  long long timed_launches = 0;
  cudaEvent_t gev0 = nullptr, gev1 = nullptr;  // around each graph launch
  double graph_ms = 0.0;
  bool graph_fused = false;  // the captured steps evaluate their pairs in the integrator
  long long n_regrowths = 0;  // pair lists grown after an overflowing rebuild
  // Mixed: nearly parallel pairs evaluated from the FP64 sites by a one-block
  // kernel after each pair stage (on by default; sc_set_exact_near_parallel).
  bool npx = true;
  // The last step fused its pair evaluation into the integrator, so the
  // per-bond slots do not hold it yet (materialize_slots writes them).
  bool slots_stale = false;
  bool fuse_pairs = false;  // sc_set_fused_pairs

  // thermo (sc_set_thermo): records are produced on the device every th_n
  // steps and pulled into th_host (and the open .thermo files)
  long long th_i0 = 0;            // i_step when the records started
  long long th_pulled = 0;        // records copied to the host
  std::vector<double> th_host;    // pulled, not yet returned: per record nrep x 12
  std::vector<FILE *> th_files;   // per system, while a .thermo file is open
};

namespace {

sc_status fail(sc_ctx *c, sc_status code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess)                                                \
      return fail(c, SC_ERR_CUDA, "%s: %s (%s:%d)", #call,                \
                  cudaGetErrorString(e_), __FILE__, __LINE__);            \
  } while (0)

#define CKS(expr)                     \
  do {                                \
    sc_status s_ = (expr);            \
    if (s_ != SC_OK) return s_;       \
  } while (0)

template <class T>
sc_status dalloc(sc_ctx *c, T **p, size_t n) {
  void *q = nullptr;
  size_t bytes = sizeof(T) * (n ? n : 1);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SC_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", bytes,
                cudaGetErrorString(e));
  }
  c->allocs.push_back(q);
  *p = (T *)q;
  return SC_OK;
}

void dfree(sc_ctx *c, void *p) {
  if (!p) return;
  auto it = std::find(c->allocs.begin(), c->allocs.end(), p);
  if (it != c->allocs.end()) c->allocs.erase(it);
  cudaFree(p);
}

// The reference's symmetric 2x2 / 3x3 inverses (src/linear_algebra.cpp:40-64),
// so that h^-1 has the same bits as the reference's unit_cell_inv.
void invert_sym_2d(const double *a, double *b) {
  double inv_det = a[0] * a[3] - a[1] * a[1];
  inv_det = 1.0 / inv_det;
  b[0] = a[3] * inv_det;
  b[3] = a[0] * inv_det;
  b[2] = b[1] = -a[1] * inv_det;
}

void invert_sym_3d(const double *a, double *b) {
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

// Filament::InitFilamentLength for static lengths (src/filament.cpp:104-147).
void filament_length(const sc_filament_params &p, double *length, int *n_bonds) {
  double max_bond_length = 1.5 * p.min_bond_length;
  double min_length = 5, max_length = 500, L = p.length;
  if (min_length < 2 * p.min_bond_length) min_length = 2 * p.min_bond_length;
  if (max_length < min_length) max_length = min_length;
  if (L > max_length) L = max_length;
  else if (L < min_length) L = min_length;
  int nb = (int)std::floor(L / max_bond_length);
  nb = (nb == 1 ? 2 : nb);
  *length = L;
  *n_bonds = nb;
}

sc_status check_status(sc_ctx *c) {
  unsigned s = c->hb->status;
  if (s & sc::ST_NAN) return fail(c, SC_ERR_NAN, "non-finite position or displacement");
  if (s & sc::ST_BAD_CELL) return fail(c, SC_ERR_NAN, "bond outside the cell grid (non-finite position)");
  if (s & sc::ST_LIST_OVERFLOW) return fail(c, SC_ERR_LIST_OVERFLOW, "pair list overflow");
  if (s & sc::ST_TETHER)
    return fail(c, SC_ERR_UNPHYSICAL, "a crosslink anchor moved off the bonds around its site");
  return SC_OK;
}

// Reads the status word and every system's displacement maximum.
sc_status readback(sc_ctx *c) {
  if (c->d.nrep > 0)
    CK(cudaMemcpyAsync(c->h_dr, c->d.dr_max_bits, sizeof(unsigned long long) * c->d.nrep,
                       cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&c->hb->status, c->d.status, sizeof(unsigned),
                     cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return check_status(c);
}

constexpr int kThermoMaxBlocks = 296;  // two per SM

void drop_graph(sc_ctx *c) {
  if (c->graph_exec) {
    cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
  }
  c->graph_rbuf = -1;
}

// Copies the system table to the device (segments or layout changed).
sc_status upload_reps(sc_ctx *c) {
  const int nrep = (int)c->reps.size();
  if (!c->d.rep) {
    sc::ReplicaConst *q = nullptr;
    CKS(dalloc(c, &q, nrep));
    c->d.rep = q;
  }
  CK(cudaMemcpyAsync(const_cast<sc::ReplicaConst *>(c->d.rep), c->reps.data(),
                     sizeof(sc::ReplicaConst) * nrep, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->d.pcap_total = (int)c->pcap;
  // Thermo blocks per system: one per 2,048 slots of the largest segment.
  int maxcap = 0;
  for (const auto &R : c->reps) maxcap = std::max(maxcap, R.pcap);
  c->d.th_gx = std::max(1, std::min(kThermoMaxBlocks, (maxcap + 2047) / 2048));
  drop_graph(c);  // kernel parameters changed
  return SC_OK;
}

// The pair-list arrays of a context (DevState's pair members).
struct PairStore {
  int *pa = nullptr, *pb = nullptr, *pos1 = nullptr, *pos2 = nullptr, *e_ent = nullptr;
  double *pf64 = nullptr, *cf64 = nullptr, *pv64 = nullptr;
  float *pf32 = nullptr, *cf32 = nullptr, *pv32 = nullptr;
};

void free_store(sc_ctx *c, PairStore &q) {
  for (void *p : {(void *)q.pa, (void *)q.pb, (void *)q.pos1, (void *)q.pos2, (void *)q.pf64,
                  (void *)q.pf32, (void *)q.cf64, (void *)q.cf32, (void *)q.e_ent,
                  (void *)q.pv64, (void *)q.pv32})
    dfree(c, p);
  q = PairStore{};
}

PairStore current_store(const sc_ctx *c) {
  const DevState &d = c->d;
  PairStore q;
  q.pa = d.pa;
  q.pb = d.pb;
  q.pos1 = d.pos1;
  q.pos2 = d.pos2;
  q.e_ent = d.e_ent;
  q.pf64 = d.pf64;
  q.cf64 = d.cf64;
  q.pv64 = d.pv64;
  q.pf32 = d.pf32;
  q.cf32 = d.cf32;
  q.pv32 = d.pv32;
  return q;
}

// Frees the context's pair arrays and puts q's in their place.
void install_store(sc_ctx *c, const PairStore &q) {
  PairStore old = current_store(c);
  free_store(c, old);
  DevState &d = c->d;
  d.pa = q.pa;
  d.pb = q.pb;
  d.pos1 = q.pos1;
  d.pos2 = q.pos2;
  d.e_ent = q.e_ent;
  d.pf64 = q.pf64;
  d.cf64 = q.cf64;
  d.pv64 = q.pv64;
  d.pf32 = q.pf32;
  d.cf32 = q.cf32;
  d.pv32 = q.pv32;
}

// New pair arrays for `total` slots, with the context's precision and
// options: slot indices and slots zeroed (a slot index names a valid slot
// until a rebuild or a restore fills it), virial records zeroed (a pair not
// evaluated since the list was built has stress and potential 0).  Either
// every array is allocated, or none is (the context is left as it was).
sc_status alloc_store(sc_ctx *c, long long total, PairStore &q) {
  q = PairStore{};
  const size_t n = (size_t)(total > 0 ? total : 1);
  auto all = [&]() -> sc_status {
    CKS(dalloc(c, &q.pa, n));
    CKS(dalloc(c, &q.pb, n));
    CKS(dalloc(c, &q.pos1, n));
    CKS(dalloc(c, &q.pos2, n));
    CKS(dalloc(c, &q.e_ent, 2 * n));
    CK(cudaMemsetAsync(q.pos1, 0, sizeof(int) * n, c->st));
    CK(cudaMemsetAsync(q.pos2, 0, sizeof(int) * n, c->st));
    if (c->prec == 0) {
      CKS(dalloc(c, &q.pf64, 4 * n));
      CKS(dalloc(c, &q.cf64, 16 * n));
      CK(cudaMemsetAsync(q.cf64, 0, sizeof(double) * 16 * n, c->st));
      if (c->k.thermo) {
        CKS(dalloc(c, &q.pv64, 4 * n));
        CK(cudaMemsetAsync(q.pv64, 0, sizeof(double) * 4 * n, c->st));
      }
    } else {
      CKS(dalloc(c, &q.pf32, 4 * n));
      CKS(dalloc(c, &q.cf32, 16 * n));
      CK(cudaMemsetAsync(q.cf32, 0, sizeof(float) * 16 * n, c->st));
      if (c->k.thermo) {
        CKS(dalloc(c, &q.pv32, 4 * n));
        CK(cudaMemsetAsync(q.pv32, 0, sizeof(float) * 4 * n, c->st));
      }
    }
    return SC_OK;
  };
  const sc_status s = all();
  if (s != SC_OK) free_store(c, q);
  return s;
}

// Pair storage for segments of the given capacities, one per system, back
// to back; previous contents are discarded.  Stored pair forces are padded
// to 4 values and per-bond slots to 8, so every write is a 16-byte store.
// The new arrays are allocated before the old ones are freed: a failed
// allocation leaves the context's storage and segments as they were.
sc_status layout_pairs(sc_ctx *c, const std::vector<long long> &caps) {
  long long total = 0;
  for (long long x : caps) total += x;
  if (total >= (1ll << 30)) return fail(c, SC_ERR_LIST_OVERFLOW, "pair lists of %lld slots too large", total);
  PairStore q;
  CKS(alloc_store(c, total, q));
  install_store(c, q);
  long long p0 = 0;
  for (size_t r = 0; r < caps.size(); ++r) {
    c->reps[r].p0 = (int)p0;
    c->reps[r].pcap = (int)caps[r];
    p0 += caps[r];
  }
  c->pcap = total;
  return upload_reps(c);
}

// One system only: grows its segment to at least `need` pairs, keeping the
// current list (pairs, their stored forces and the per-bond entries).  A
// failed allocation leaves the current list in place.
sc_status ensure_pair_capacity(sc_ctx *c, long long need) {
  if (need <= c->pcap) return SC_OK;
  if (c->reps.size() != 1)
    return fail(c, SC_ERR_LIST_OVERFLOW, "a system's pair list outgrew its segment");
  long long cap = std::max<long long>(need + need / 2, 1024);
  if (cap >= (1ll << 30)) return fail(c, SC_ERR_LIST_OVERFLOW, "pair list of %lld pairs too large", need);
  const DevState &old = c->d;
  const long long keep = std::min<long long>(c->np, c->pcap);
  PairStore q;
  CKS(alloc_store(c, cap, q));
  if (keep > 0) {
    auto cp = [&](void *dst, const void *src, size_t bytes) {
      return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->st);
    };
    CK(cp(q.pa, old.pa, sizeof(int) * keep));
    CK(cp(q.pb, old.pb, sizeof(int) * keep));
    CK(cp(q.pos1, old.pos1, sizeof(int) * keep));
    CK(cp(q.pos2, old.pos2, sizeof(int) * keep));
    if (c->prec == 0) {
      CK(cp(q.pf64, old.pf64, sizeof(double) * 4 * keep));
      CK(cp(q.cf64, old.cf64, sizeof(double) * 16 * keep));
    } else {
      CK(cp(q.pf32, old.pf32, sizeof(float) * 4 * keep));
      CK(cp(q.cf32, old.cf32, sizeof(float) * 16 * keep));
    }
    CK(cp(q.e_ent, old.e_ent, sizeof(int) * 2 * keep));
    if (q.pv64 && old.pv64) CK(cp(q.pv64, old.pv64, sizeof(double) * 4 * keep));
    if (q.pv32 && old.pv32) CK(cp(q.pv32, old.pv32, sizeof(float) * 4 * keep));
  }
  CK(cudaStreamSynchronize(c->st));
  install_store(c, q);
  c->reps[0].p0 = 0;
  c->reps[0].pcap = (int)cap;
  c->pcap = cap;
  return upload_reps(c);
}

// Pair counts of every system (device values); c->np is their total.
sc_status sync_pair_count(sc_ctx *c) {
  const int nrep = c->d.nrep;
  CK(cudaMemcpyAsync(c->h_np, c->d.np_rep, sizeof(int) * nrep, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->np = 0;
  for (int r = 0; r < nrep; ++r) {
    c->np_rep[r] = c->h_np[r];
    c->np += std::min(c->h_np[r], c->reps[r].pcap);
  }
  return SC_OK;
}

// InteractionManager::UpdateInteractions (src/interaction_manager.cpp:211-231)
// for the systems flagged in d.due: bin their bonds, emit their half-shell
// pair lists in the reference's order into their segments, build their
// per-bond pair entries, zero their displacement trackers.  Device work only
// (capturable); a list longer than its segment sets the overflow bit.
void rebuild_enqueue(sc_ctx *c, bool first_in_graph = false) {
  const SysConst &k = c->k;
  const long long before = c->launches;
  const DevState &d = c->d;
  if (c->desc.interaction_flag) {
    if (first_in_graph) {
      // Captured, the rebuild's first kernel starts the conditional body:
      // no kernel before it to overlap.
      sc::PdlOff off;
      c->launches += sc::launch_bin_count(k, d, c->key, c->cell_count, c->st);
    } else {
      c->launches += sc::launch_bin_count(k, d, c->key, c->cell_count, c->st);
    }
    c->launches += sc::launch_exclusive_scan(c->cell_count, c->cell_start, k.n_cells,
                                             c->scan_tmp, c->st, c->cell_occ);
    c->launches += sc::launch_bin_scatter(d, c->key, c->cell_start, c->cell_count, c->sorted,
                                          c->st);
    c->launches += sc::launch_cell_sort_count(k, d, c->key, c->sorted, c->cell_start,
                                              c->pair_count, c->st, c->cell_occ);
    c->launches += sc::launch_exclusive_scan(c->pair_count, c->pair_off, c->nb,
                                             c->scan_tmp, c->st);
    c->launches += sc::launch_pair_emit(k, d, c->key, c->sorted, c->cell_start,
                                        c->pair_off, c->deg, c->prec, c->st, c->cell_occ);
    c->launches += sc::launch_exclusive_scan(c->deg, c->deg_off, c->nb, c->scan_tmp, c->st);
    c->launches += sc::launch_csr(d, c->deg, c->deg_off, c->st);
  }
  c->launches += sc::launch_zero_dr(d, c->st);
  c->rebuild_kernels = c->launches - before;
}

// Host-driven rebuild of the systems flagged in d.due, then a check that
// every list fitted.  One system grows its segment and rebuilds again
// (binning is a pure function of the positions, so the second pass gives the
// same list); with several systems an overflow is reported, unless
// allow_overflow (the initial pass, whose caller sizes the segments).
sc_status grow_after_overflow(sc_ctx *c);

sc_status rebuild(sc_ctx *c, bool allow_overflow = false) {
  for (int attempt = 0; attempt < 3; ++attempt) {
    rebuild_enqueue(c);
    CK(cudaGetLastError());
    if (!c->desc.interaction_flag) return SC_OK;
    CK(cudaMemcpyAsync(&c->hb->status, c->d.status, sizeof(unsigned),
                       cudaMemcpyDeviceToHost, c->st));
    CKS(sync_pair_count(c));
    if (!(c->hb->status & sc::ST_LIST_OVERFLOW)) return SC_OK;
    unsigned clear = c->hb->status & ~sc::ST_LIST_OVERFLOW;
    CK(cudaMemcpyAsync(c->d.status, &clear, sizeof(unsigned), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (allow_overflow) return SC_OK;
    if (c->reps.size() != 1)
      return fail(c, SC_ERR_LIST_OVERFLOW, "a system's pair list outgrew its segment");
    CKS(grow_after_overflow(c));
  }
  return fail(c, SC_ERR_LIST_OVERFLOW, "pair list kept overflowing");
}

// A rebuild of the single system overflowed its list (the overflow bit
// already cleared): grow the list to the full count and take that pass back
// out of the rebuild counters, since the pass is redone.
sc_status grow_after_overflow(sc_ctx *c) {
  const int want = c->np_rep[0];
  c->np = 0;  // the overflowed list is incomplete: nothing to keep
  CKS(ensure_pair_capacity(c, (long long)want));
  long long cnt[2] = {0, 0};
  CK(cudaMemcpyAsync(&cnt[0], c->d.n_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&cnt[1], c->d.rep_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  cnt[0] -= 1;
  cnt[1] -= 1;
  CK(cudaMemcpyAsync(c->d.n_rebuilds, &cnt[0], sizeof(long long), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d.rep_rebuilds, &cnt[1], sizeof(long long), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->n_regrowths++;
  return SC_OK;
}

// Flags every system and rebuilds (the forced update after insertion).
sc_status rebuild_all(sc_ctx *c) {
  const int nrep = c->d.nrep;
  for (int r = 0; r < nrep; ++r) c->h_due[r] = 1;
  CK(cudaMemcpyAsync(c->d.due, c->h_due, sizeof(int) * nrep, cudaMemcpyHostToDevice, c->st));
  return rebuild(c, true);
}

// Interact's rebuild check (CheckUpdateInteractions + GetDrMax,
// src/interaction_manager.cpp:284-312, include/simcore/species.hpp:105-120),
// per system.  Only a query after a full step can see a grown displacement,
// so the device maxima are read back only then.
sc_status maybe_rebuild(sc_ctx *c) {
  if (!c->desc.interaction_flag) return SC_OK;
  if (!c->midstep) return SC_OK;  // previous update was a midstep: unchanged
  if (c->i_step <= 1) return SC_OK;
  CKS(readback(c));
  const int nrep = c->d.nrep;
  bool any = false;
  for (int r = 0; r < nrep; ++r) {
    double dr_max;
    std::memcpy(&dr_max, &c->h_dr[r], sizeof(double));
    if (dr_max > 10000)
      return fail(c, SC_ERR_UNPHYSICAL, "Unphysical result: dr_max %g (system %d)", dr_max, r);
    c->h_due[r] = dr_max > c->reps[r].dr_update ? 1 : 0;
    any = any || c->h_due[r];
  }
  if (!any) return SC_OK;
  CK(cudaMemcpyAsync(c->d.due, c->h_due, sizeof(int) * nrep, cudaMemcpyHostToDevice, c->st));
  return rebuild(c);
}

// Integrator work units over the filaments in order: runs of whole
// filaments of at most warp_sites sites each go to the warp-synchronous
// kernel (one lane per site, at most 32 sites per group); longer filaments go
// to the block kernel (runs of whole filaments up to C sites per block).
sc_status layout_integrator(sc_ctx *c) {
  const std::vector<int> &off = c->site_off;
  const int n = c->nf;
  std::vector<int> blk_site0, blk_f0, blk_nf, blk_ns, wg_site0, wg_f0, wg_ns;
  int max_long = 0;
  auto short_fil = [&](int f) { return off[f + 1] - off[f] <= c->warp_sites; };
  for (int f = 0; f < n; ++f)
    if (!short_fil(f)) max_long = std::max(max_long, off[f + 1] - off[f]);
  c->C = c->block_sites > 0 ? c->block_sites
                            : (max_long <= 128 ? 128 : max_long <= 256 ? 256 : 512);
  if (max_long > c->C)
    return fail(c, SC_ERR_INVALID_ARG, "a %d-site filament does not fit %d-site blocks", max_long,
                c->C);
  // A work unit never mixes systems (its displacement maximum is one
  // system's).
  auto same = [&](int f, int f0) { return c->fil_rep.empty() || c->fil_rep[f] == c->fil_rep[f0]; };
  int f = 0;
  while (f < n) {
    const int s0 = off[f], f0 = f;
    if (short_fil(f)) {
      while (f < n && short_fil(f) && same(f, f0) && off[f + 1] - s0 <= 32) ++f;
      wg_site0.push_back(s0);
      wg_f0.push_back(f0);
      wg_ns.push_back(off[f] - s0);
    } else {
      while (f < n && !short_fil(f) && same(f, f0) && off[f + 1] - s0 <= c->C) ++f;
      blk_site0.push_back(s0);
      blk_f0.push_back(f0);
      blk_nf.push_back(f - f0);
      blk_ns.push_back(off[f] - s0);
    }
  }
  for (const int *q : {c->d.blk_site0, c->d.blk_f0, c->d.blk_nf, c->d.blk_ns, c->d.wg_site0,
                       c->d.wg_f0, c->d.wg_ns})
    dfree(c, const_cast<int *>(q));
  auto up = [&](const int **dst, const std::vector<int> &v) -> sc_status {
    int *q = nullptr;
    CKS(dalloc(c, &q, v.size()));
    if (!v.empty())
      CK(cudaMemcpyAsync(q, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice, c->st));
    *dst = q;
    return SC_OK;
  };
  DevState &d = c->d;
  CKS(up(&d.blk_site0, blk_site0));
  CKS(up(&d.blk_f0, blk_f0));
  CKS(up(&d.blk_nf, blk_nf));
  CKS(up(&d.blk_ns, blk_ns));
  CKS(up(&d.wg_site0, wg_site0));
  CKS(up(&d.wg_f0, wg_f0));
  CKS(up(&d.wg_ns, wg_ns));
  CK(cudaStreamSynchronize(c->st));
  c->nblocks = (int)blk_f0.size();
  d.n_wg = (int)wg_f0.size();
  sc::prepare_integrate(c->C);
  drop_graph(c);
  return SC_OK;
}

// Records CUDA events around one launch when kernel timing is on.
template <class F>
sc_status timed(sc_ctx *c, F launch) {
  if (c->timing) CK(cudaEventRecord(c->ev0, c->st));
  c->launches += launch();
  if (c->timing) {
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->timed_ms += ms;
    c->timed_launches += 1;
  }
  return SC_OK;
}

// Crosslinks of Interact (src/interaction_manager.cpp:70): on even steps the
// tethers are recomputed; odd steps re-use the stored anchor contributions.
void tether_if_due(sc_ctx *c) {
  if (c->desc.interaction_flag && c->d.nx && c->i_step % 2 == 0)
    c->launches += sc::launch_tether(c->k, c->d, c->st);
}

// ---- thermo ----------------------------------------------------------------

// Records the device has produced by step i (one every th_n steps since th_i0).
long long thermo_total(const sc_ctx *c, long long i) {
  const long long n = c->d.th_n;
  return n > 0 ? i / n - c->th_i0 / n : 0;
}

// One record of every system as OutputManager::WriteThermo writes it
// (include/simcore/output_manager.hpp:169-183): unit cell (9), pressure
// tensor (9), pressure, volume.
void thermo_write(sc_ctx *c, const double *rec) {
  for (size_t r = 0; r < c->th_files.size(); ++r) {
    FILE *f = c->th_files[r];
    if (!f) continue;
    const double *q = rec + 12 * r;
    std::fwrite(c->reps[r].h, sizeof(double), 9, f);
    std::fwrite(q + 1, sizeof(double), 11, f);
  }
}

// Copies the records produced so far from the device ring to th_host (and
// the open files).
sc_status thermo_pull(sc_ctx *c) {
  if (c->d.th_n <= 0 || !c->d.th_rec) return SC_OK;
  const long long tot = thermo_total(c, c->i_step);
  if (tot <= c->th_pulled) return SC_OK;
  const size_t per = 12 * (size_t)c->d.nrep;
  std::vector<double> ring(per * (size_t)c->d.th_cap);
  CK(cudaMemcpyAsync(ring.data(), c->d.th_rec, sizeof(double) * ring.size(),
                     cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (long long k = c->th_pulled; k < tot; ++k) {
    const double *rec = ring.data() + per * (size_t)(k % c->d.th_cap);
    c->th_host.insert(c->th_host.end(), rec, rec + per);
    thermo_write(c, rec);
  }
  c->th_pulled = tot;
  return SC_OK;
}

// Room in the device ring for the records of the next n steps: pulls the
// pending ones, and grows the ring when n steps alone would overrun it.
sc_status thermo_reserve(sc_ctx *c, long long n) {
  if (!c->k.thermo) return SC_OK;
  const long long after = thermo_total(c, c->i_step + n);
  if (after - c->th_pulled <= c->d.th_cap) return SC_OK;
  CKS(thermo_pull(c));
  const long long need = after - c->th_pulled;
  if (need <= c->d.th_cap) return SC_OK;
  // Everything produced is pulled: the ring holds nothing live.
  const long long cap = need + need / 2;
  if (cap > (1ll << 24)) return fail(c, SC_ERR_INVALID_ARG, "%lld thermo records in one run", need);
  double *ring = nullptr;
  CKS(dalloc(c, &ring, 12 * (size_t)c->d.nrep * cap));
  dfree(c, c->d.th_rec);
  c->d.th_rec = ring;
  c->d.th_cap = (int)cap;
  drop_graph(c);
  return SC_OK;
}

// With sc_set_fused_pairs, the fast mixed step evaluates the pairs inside the
// integrator (each bond its own pairs, bit for bit the pair stage's forces)
// and launches no pair stage.  Not with thermo (whose records the pair stage
// writes), nor with the FP64 evaluation of nearly parallel pairs; the split
// interface (sc_interact, then sc_update_positions) keeps the separate pair
// stage.
bool fused_pairs(const sc_ctx *c) {
  return c->fuse_pairs && c->desc.interaction_flag && c->prec == 1 && c->fast &&
         !c->k.thermo && !c->npx;
}

// The pair stage of one step, then the step's thermo accumulation.
sc_status pair_stage(sc_ctx *c) {
  CKS(timed(c, [&] {
    return sc::launch_pairs(c->k, c->d, c->rbuf, c->prec, (int)c->np, c->st, c->npx);
  }));
  c->slots_stale = false;
  if (c->k.thermo) c->launches += sc::launch_thermo(c->k, c->d, c->prec, c->st);
  return SC_OK;
}

sc_status step_once(sc_ctx *c) {
  CKS(thermo_reserve(c, 1));
  c->i_step++;
  tether_if_due(c);
  CKS(maybe_rebuild(c));
  const int interaction = c->desc.interaction_flag ? 1 : 0;
  const bool fuse = fused_pairs(c);
  if (interaction && !fuse) CKS(pair_stage(c));
  CKS(timed(c, [&] {
    return sc::launch_integrate(c->k, c->d, c->nblocks, c->C, c->midstep, c->rbuf,
                                interaction, c->capture, c->prec, c->fast, c->st, fuse);
  }));
  if (c->midstep && c->desc.stoch_flag)
    c->launches += sc::launch_advance_mcount(c->d, c->st);
  CK(cudaGetLastError());
  c->pairs_ready = false;
  if (fuse) c->slots_stale = true;
  if (c->midstep && c->desc.stoch_flag) c->mcount++;
  c->midstep = !c->midstep;
  c->rbuf = 1 - c->rbuf;
  return SC_OK;
}

// The slots of the last fused step, written by the pair stage run again on
// that step's geometry: the buffer the step read (1 - rbuf), which nothing
// writes before the next step (sc_set_sites fills the other one).  With the
// same pair list, geometry and stored forces, every pair in range gets the
// bits the step computed and every other pair re-reads its unchanged stored
// force, so the slots are those a separate pair stage would have left.
sc_status materialize_slots(sc_ctx *c) {
  if (!c->slots_stale) return SC_OK;
  c->launches += sc::launch_pairs(c->k, c->d, 1 - c->rbuf, c->prec, (int)c->np, c->st, false);
  CK(cudaGetLastError());
  c->slots_stale = false;
  return SC_OK;
}

template <class T>
sc_status copy_soa3(sc_ctx *c, T *const *src, int n, double *xyz) {
  // Interleave on the device, then one copy into the caller's buffer (at
  // full link speed when that buffer is pinned).
  c->launches += sc::launch_soa_to_aos(n, src[0], src[1], src[2], c->stage, c->st);
  CK(cudaMemcpyAsync(xyz, c->stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

template <class T>
void put(FILE *f, const T &v) {
  std::fwrite(&v, sizeof(T), 1, f);
}

// Writes the frame whose copy has completed.
sc_status output_flush(sc_ctx *c) {
  sc_ctx::Output &o = c->out;
  if (!o.pending_spec && !o.pending_posit) return SC_OK;
  CK(cudaEventSynchronize(o.copied));
  const double *pos = o.h_snap;
  const double *avg = o.h_snap + 3 * (size_t)c->ns;
  for (size_t r = 0; r < c->reps.size(); ++r) {
    const sc::ReplicaConst &R = c->reps[r];
    if (o.pending_spec && o.spec[r]) {
      FILE *f = o.spec[r];
      put(f, (int32_t)R.nf);
      for (int fi = R.f0; fi < R.f0 + R.nf; ++fi) {
        const int n = c->site_off[fi + 1] - c->site_off[fi];
        put(f, c->fil_diam[fi]);
        put(f, c->fil_len[fi]);
        put(f, c->fil_bl[fi]);
        put(f, (int32_t)n);
        std::fwrite(pos + 3 * (size_t)c->site_off[fi], sizeof(double), 3 * (size_t)n, f);
        put(f, c->fil_lp[fi]);          // bending_stiffness_ = persistence length
        put(f, (unsigned char)0);       // poly_state::grow
      }
    }
    if (o.pending_posit && o.posit[r]) {
      FILE *f = o.posit[r];
      put(f, (int32_t)R.nf);
      for (int fi = R.f0; fi < R.f0 + R.nf; ++fi) {
        std::fwrite(avg + 9 * (size_t)fi, sizeof(double), 9, f);  // pos, scaled pos, u
        put(f, c->fil_diam[fi]);
        put(f, c->fil_len[fi]);
      }
    }
  }
  o.pending_spec = o.pending_posit = false;
  return SC_OK;
}
}  // namespace

extern "C" {

int sc_filament_n_bonds(const sc_filament_params *p) {
  if (!p) return -1;
  double L;
  int nb;
  filament_length(*p, &L, &nb);
  return nb;
}

sc_status sc_create(const sc_system_desc *desc, sc_ctx **out) {
  if (!desc || !out) return SC_ERR_INVALID_ARG;
  *out = nullptr;
  if (desc->n_dim != 2 && desc->n_dim != 3) return SC_ERR_INVALID_ARG;
  if (!(desc->system_radius > 0) || !(desc->delta > 0) || !(desc->wca_sig > 0))
    return SC_ERR_INVALID_ARG;
  if (desc->precision != SC_PREC_FP64 && desc->precision != SC_PREC_MIXED)
    return SC_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return SC_ERR_NO_DEVICE;
  }
  if (desc->device < 0 || desc->device >= ndev) return SC_ERR_INVALID_ARG;
  sc_ctx *c = new sc_ctx();
  c->desc = *desc;
  c->nd = desc->n_dim;
  c->prec = desc->precision;
  if (cudaSetDevice(desc->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaHostAlloc((void **)&c->hb, sizeof(sc_ctx::Readback), cudaHostAllocDefault) !=
          cudaSuccess) {
    cudaGetLastError();
    delete c;
    return SC_ERR_CUDA;
  }
  SysConst &k = c->k;
  std::memset(&k, 0, sizeof(k));
  k.n_dim = c->nd;
  k.delta = desc->delta;
  // WCAPotential::Init (include/simcore/wca_potential.hpp:34-48)
  double rcut = std::pow(2.0, 1.0 / 6.0) * desc->wca_sig;
  k.rcut2 = rcut * rcut;
  k.c12 = 4.0 * desc->wca_eps * std::pow(desc->wca_sig, 12.0);
  k.c6 = 4.0 * desc->wca_eps * std::pow(desc->wca_sig, 6.0);
  k.fcut = desc->f_cutoff;
  k.rcut2f = (float)k.rcut2;
  k.c12f = (float)k.c12;
  k.c6f = (float)k.c6;
  k.fcutf = (float)k.fcut;
  k.eps = desc->wca_eps;
  k.epsf = (float)desc->wca_eps;
  k.stoch = desc->stoch_flag ? 1 : 0;
  k.like_like = desc->like_like_interactions ? 1 : 0;
  CK(cudaMalloc((void **)&c->d.status, sizeof(unsigned)));
  c->allocs.push_back(c->d.status);
  CK(cudaMalloc((void **)&c->d.mcount, sizeof(unsigned long long)));
  c->allocs.push_back(c->d.mcount);
  CK(cudaMalloc((void **)&c->d.n_rebuilds, sizeof(long long)));
  c->allocs.push_back(c->d.n_rebuilds);
  CK(cudaMalloc((void **)&c->d.loop_count, sizeof(int)));
  c->allocs.push_back(c->d.loop_count);
  CK(cudaMemsetAsync(c->d.status, 0, sizeof(unsigned), c->st));
  CK(cudaMemsetAsync(c->d.mcount, 0, sizeof(unsigned long long), c->st));
  CK(cudaMemsetAsync(c->d.n_rebuilds, 0, sizeof(long long), c->st));
  CK(cudaMemsetAsync(c->d.loop_count, 0, sizeof(int), c->st));
  if (cudaHostAlloc((void **)&c->h_loop, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SC_ERR_CUDA, "pinned allocation failed");
  }
  *out = c;
  return SC_OK;
}

sc_status sc_destroy(sc_ctx *c) {
  if (!c) return SC_ERR_INVALID_ARG;
  cudaSetDevice(c->desc.device);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->out.open) sc_output_close(c);
  if (!c->th_files.empty()) {
    thermo_pull(c);
    for (FILE *f : c->th_files)
      if (f) std::fclose(f);
    c->th_files.clear();
  }
  drop_graph(c);
  for (void *p : c->allocs) cudaFree(p);
  if (c->hb) cudaFreeHost(c->hb);
  if (c->h_loop) cudaFreeHost(c->h_loop);
  for (void *h : {(void *)c->h_dr, (void *)c->h_np, (void *)c->h_due})
    if (h) cudaFreeHost(h);
  if (c->gev0) cudaEventDestroy(c->gev0);
  if (c->gev1) cudaEventDestroy(c->gev1);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->st) cudaStreamDestroy(c->st);
  cudaGetLastError();
  delete c;
  return SC_OK;
}

const char *sc_last_error(const sc_ctx *c) { return c ? c->err.c_str() : "null context"; }

// Loads nrep independent systems: system r has radius[r], noise key seed[r]
// and nfil[r] filaments, which come next in p and site_xyz.  A single-system
// context is the case nrep = 1.
static sc_status add_systems(sc_ctx *c, int nrep, const double *radius, const uint32_t *seed,
                             const int32_t *nfil, int n, const sc_filament_params *p,
                             const double *site_xyz, int64_t n_sites_total) {
  if (!c) return SC_ERR_INVALID_ARG;
  if (c->loaded) return fail(c, SC_ERR_INVALID_ARG, "filaments already added");
  if (n <= 0 || !p || !site_xyz) return fail(c, SC_ERR_INVALID_ARG, "bad filament arrays");
  if (nrep <= 0 || !radius || !seed || !nfil)
    return fail(c, SC_ERR_INVALID_ARG, "bad system arrays");
  {
    long long tot = 0;
    for (int r = 0; r < nrep; ++r) {
      if (nfil[r] <= 0) return fail(c, SC_ERR_INVALID_ARG, "system %d has no filaments", r);
      if (!(radius[r] > 0) || !std::isfinite(radius[r]))
        return fail(c, SC_ERR_INVALID_ARG, "system %d: bad radius", r);
      tot += nfil[r];
    }
    if (tot != n)
      return fail(c, SC_ERR_INVALID_ARG, "filament counts of the systems sum to %lld, not %d",
                  tot, n);
  }
  CK(cudaSetDevice(c->desc.device));
  const double mbl = p[0].min_bond_length, dia = p[0].diameter;
  std::vector<double> len(n);
  std::vector<int> nbf(n);
  long long ns = 0;
  int max_ns = 0;
  for (int f = 0; f < n; ++f) {
    if (!(p[f].length > 0) || !(p[f].diameter > 0) || !(p[f].min_bond_length > 0) ||
        !(p[f].friction_ratio > 0) || !(p[f].persistence_length >= 0) ||
        !std::isfinite(p[f].diameter) || !std::isfinite(p[f].min_bond_length) ||
        !std::isfinite(p[f].friction_ratio) || !std::isfinite(p[f].persistence_length))
      return fail(c, SC_ERR_INVALID_ARG, "filament %d: bad parameters", f);
    if (p[f].min_bond_length != mbl || p[f].diameter != dia)
      return fail(c, SC_ERR_INVALID_ARG,
                  "filament %d: min_bond_length and diameter are species-wide", f);
    filament_length(p[f], &len[f], &nbf[f]);
    c->fil_diam.push_back(p[f].diameter);
    c->fil_len.push_back(len[f]);
    c->fil_bl.push_back(len[f] / nbf[f]);
    c->fil_lp.push_back(p[f].persistence_length);
    ns += nbf[f] + 1;
    max_ns = std::max(max_ns, nbf[f] + 1);
  }
  if (ns != n_sites_total)
    return fail(c, SC_ERR_INVALID_ARG, "n_sites_total %lld != %lld implied by the lengths",
                (long long)n_sites_total, ns);
  if (max_ns > 512)
    return fail(c, SC_ERR_INVALID_ARG, "filaments longer than 511 bonds are not supported");
  if (ns > (1ll << 30)) return fail(c, SC_ERR_INVALID_ARG, "too many sites");
  const int nsi = (int)ns, nbi = nsi - n;
  c->nf = n;
  c->ns = nsi;
  c->nb = nbi;

  // Per-filament constants: Filament::SetParameters / InitFilamentLength /
  // SetDiffusion (src/filament.cpp:6-84, 104-170, 320-348).
  std::vector<int> site_off(n + 1, 0);
  std::vector<sc::FilConst> fil(n);
  for (int f = 0; f < n; ++f) {
    site_off[f + 1] = site_off[f] + nbf[f] + 1;
    const int nsf = nbf[f] + 1;
    sc::FilConst &q = fil[f];
    q.l = len[f] / nbf[f];
    q.linv = 1.0 / q.l;
    q.kappa = p[f].persistence_length;
    q.l2 = q.l * q.l;
    double logLD = std::log(len[f] / p[f].diameter);
    double gperp = 4.0 * len[f] / (3.0 * nsf * logLD);
    double gpar = gperp / p[f].friction_ratio;
    q.igpar = 1.0 / gpar;
    q.igperp = 1.0 / gperp;
    q.two_igperp = 2.0 / gperp;
    q.m1_igperp = -1.0 / gperp;
    q.dgam = 1.0 / gpar - 1.0 / gperp;
    q.sperp = std::sqrt(24.0 * gperp / c->desc.delta);
    q.spar = std::sqrt(24.0 * gpar / c->desc.delta);
    q.site0 = site_off[f];
    q.n = nsf;
  }
  c->site_off = site_off;
  std::vector<int> fil_rep(n);
  {
    int f = 0;
    for (int r = 0; r < nrep; ++r)
      for (int i = 0; i < nfil[r]; ++i, ++f) {
        fil[f].rep = r;
        fil[f].f_local = i;
        fil_rep[f] = r;
      }
  }
  std::vector<int> site_fil(nsi), site_jn(nsi), bond_fil(nbi);
  for (int f = 0; f < n; ++f) {
    for (int s = site_off[f]; s < site_off[f + 1]; ++s) {
      site_fil[s] = f;
      site_jn[s] = (s - site_off[f]) | (site_off[f + 1] - site_off[f]) << 16;
    }
    for (int b = site_off[f] - f; b < site_off[f + 1] - f - 1; ++b) bond_fil[b] = f;
  }
  c->bond_fil = bond_fil;
  DevState &d = c->d;
  d.nf = n;
  d.ns = nsi;
  d.nb = nbi;
  auto up = [&](auto **dst, const auto &vec) -> sc_status {
    using T = typename std::remove_reference<decltype(vec)>::type::value_type;
    T *q = nullptr;
    CKS(dalloc(c, &q, vec.size()));
    CK(cudaMemcpyAsync(q, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice,
                       c->st));
    *dst = q;
    return SC_OK;
  };
  int *tmp_i = nullptr;
  {
    sc::FilConst *q = nullptr;
    CKS(up(&q, fil));
    d.fil = q;
  }
  std::vector<int> sw(n, 1), nn(n, 0);
  CKS(up(&d.f_switch, sw));
  CKS(up(&d.f_nnorm, nn));
  CKS(up(&tmp_i, site_fil)); d.site_fil = tmp_i;
  CKS(up(&tmp_i, site_jn)); d.site_jn = tmp_i;
  CKS(up(&tmp_i, bond_fil)); d.bond_fil = tmp_i;
  d.bond_rep = nullptr;  // one system: every bond in system 0
  if (nrep > 1) {
    std::vector<int> bond_rep(nbi);
    for (int b = 0; b < nbi; ++b) bond_rep[b] = fil_rep[bond_fil[b]];
    CKS(up(&tmp_i, bond_rep));
    d.bond_rep = tmp_i;
  }
  c->fil_rep = fil_rep;
  c->warp_sites = 32;

  // Sites: positions (z = 0 in 2D); previous positions = positions as after
  // Mesh::UpdatePrevPositions; no stored noise yet.
  std::vector<double> comp(nsi);
  for (int i = 0; i < 3; ++i) {
    for (int s = 0; s < nsi; ++s) comp[s] = i < c->nd ? site_xyz[3 * (size_t)s + i] : 0.0;
    CKS(up(&d.r[i], comp));
    CKS(up(&d.rp[i], comp));
    CKS(dalloc(c, &d.fr[i], nsi));
    CK(cudaMemsetAsync(d.fr[i], 0, sizeof(double) * nsi, c->st));
    CKS(dalloc(c, &d.dz[i], nsi));
    CKS(dalloc(c, &d.cap_F[i], nsi));
    CK(cudaMemsetAsync(d.cap_F[i], 0, sizeof(double) * nsi, c->st));
    CKS(dalloc(c, &d.ub[i], nbi));
    CKS(dalloc(c, &d.bF[i], nbi));
    CKS(dalloc(c, &d.bT[i], nbi));
    CK(cudaMemsetAsync(d.bF[i], 0, sizeof(double) * nbi, c->st));
    CK(cudaMemsetAsync(d.bT[i], 0, sizeof(double) * nbi, c->st));
  }
  CKS(dalloc(c, &d.dt, nsi));
  CKS(dalloc(c, &d.cap_T, nbi));
  CK(cudaMemsetAsync(d.cap_T, 0, sizeof(double) * nbi, c->st));
  for (int b = 0; b < 2; ++b) {
    CKS(dalloc(c, &d.g64[b], nbi));
    CKS(dalloc(c, &d.g32[b], nbi));
  }

  // Systems: Space::InitUnitCell / CalculateUnitCellQuantities
  // (src/space.cpp:85-138); cell lists: SetMinCellLength calls of
  // Simulation::InitSpecies (src/simulation.cpp:248-251) and
  // InteractionManager::InitInteractions (src/interaction_manager.cpp:46-48),
  // CellList::Init (src/cell_list.cpp:17-64).
  SysConst &k = c->k;
  c->reps.assign(nrep, sc::ReplicaConst{});
  long long cells = 0;
  {
    int f = 0;
    for (int r = 0; r < nrep; ++r) {
      sc::ReplicaConst &R = c->reps[r];
      std::memset(&R, 0, sizeof(R));
      const double hh = 2.0 * radius[r];
      for (int a = 0; a < c->nd; ++a)
        for (int b = 0; b < c->nd; ++b) R.h[a * c->nd + b] = (a == b ? 1 : 0) * hh;
      R.h[c->nd * c->nd - 1] = hh;
      if (c->nd == 2) invert_sym_2d(R.h, R.hinv);
      else invert_sym_3d(R.h, R.hinv);
      for (int i = 0; i < 9; ++i) R.hf[i] = (float)R.h[i];
      double min_len = -1, spec_length = 1.5 * mbl;
      if (dia > spec_length) spec_length = dia;
      if (spec_length > min_len) min_len = spec_length;
      if (0.0 > min_len) min_len = 0.0;
      if (std::sqrt(k.rcut2) > min_len) min_len = std::sqrt(k.rcut2);
      // Cells a side, bounded while still a double so that no integer below
      // can overflow: at most 1024 in 3D, 32768 in 2D (2^30 cells).
      const double per_side = 2 * radius[r] / min_len;
      if (!std::isfinite(per_side) || !(per_side < (c->nd == 3 ? 1025.0 : 32769.0)))
        return fail(c, SC_ERR_INVALID_ARG,
                    "system %d: a cell grid of %g cells a side is too large", r, per_side);
      int n1d = (int)std::floor(per_side);
      if (n1d <= 3) n1d = 3;
      const long long ncell = (long long)n1d * n1d * (c->nd == 3 ? n1d : 1);
      R.n1d = n1d;
      R.third = c->nd == 3 ? n1d : 1;
      R.n_cells = (int)std::min<long long>(ncell, 1ll << 30);
      R.cell0 = (int)std::min<long long>(cells, 1ll << 30);
      cells += ncell;
      const double cl = (double)2 * radius[r] / n1d;
      R.dr_update = 0.25 * cl * cl;
      R.seed = seed[r];
      R.f0 = f;
      R.nf = nfil[r];
      R.s0 = site_off[f];
      R.ns = site_off[f + nfil[r]] - site_off[f];
      R.b0 = R.s0 - f;
      R.nb = R.ns - nfil[r];
      f += nfil[r];
    }
  }
  if (cells > (1ll << 30))
    return fail(c, SC_ERR_INVALID_ARG, "cell grids of %lld cells too large", cells);
  k.n_cells = (int)cells;
  d.nrep = nrep;
  CKS(upload_reps(c));  // every kernel below reads the system table
  CKS(layout_integrator(c));
  auto dzero = [&](auto **dst, size_t count) -> sc_status {
    CKS(dalloc(c, dst, count));
    CK(cudaMemsetAsync(*dst, 0, sizeof(**dst) * (count ? count : 1), c->st));
    return SC_OK;
  };
  CKS(dzero(&d.dr_max_bits, nrep));
  CKS(dzero(&d.due, nrep));
  CKS(dzero(&d.np_rep, nrep));
  CKS(dzero(&d.rep_rebuilds, nrep));
  for (void **h : {(void **)&c->h_dr, (void **)&c->h_np, (void **)&c->h_due})
    if (cudaHostAlloc(h, sizeof(unsigned long long) * nrep, cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      return fail(c, SC_ERR_OOM, "pinned allocation failed");
    }
  c->np_rep.assign(nrep, 0);
  CKS(dalloc(c, &c->key, nbi));
  CKS(dzero(&c->cell_count, (size_t)k.n_cells));
  CKS(dalloc(c, &c->cell_start, (size_t)k.n_cells + 1));
  CKS(dalloc(c, &c->cell_occ, (size_t)k.n_cells / 32 + 1));
  CKS(dalloc(c, &c->sorted, nbi));
  CKS(dalloc(c, &c->pair_count, nbi));
  CKS(dzero(&c->pair_off, (size_t)nbi + 1));
  CKS(dzero(&c->deg, nbi));
  CKS(dzero(&c->deg_off, (size_t)nbi + 1));
  CKS(dzero(&d.e_off, nbi));
  CKS(dzero(&d.e_cnt, nbi));
  CKS(dalloc(c, &c->scan_tmp,
             (size_t)std::max(sc::scan_temp_ints(k.n_cells), sc::scan_temp_ints(nbi))));
  CKS(dalloc(c, &c->cells_xyz, 3 * (size_t)nbi));
  CKS(dalloc(c, &c->stage, 3 * (size_t)std::max(nsi, nbi)));

  sc::launch_init_geometry(c->k, d, 0, c->prec, c->st);
  if (c->prec != 0) sc::launch_init_geometry(c->k, d, 0, 0, c->st, false);
  c->rbuf = 0;
  // Simulation::InsertSpecies tail: forced update (rebuild + ZeroDrTot) of
  // every system, into pair segments sized until every list fits with
  // headroom for growth during captured runs (no resizing inside a graph).
  std::vector<long long> want(nrep);
  for (int r = 0; r < nrep; ++r) want[r] = std::max<long long>(c->reps[r].nb, 1024);
  for (int attempt = 0;; ++attempt) {
    CKS(layout_pairs(c, want));
    CKS(rebuild_all(c));
    c->slots_stale = false;
    bool ok = true;
    for (int r = 0; r < nrep; ++r) {
      const long long need = (long long)c->np_rep[r] + c->np_rep[r] / 2 + 1024;
      if (need > want[r]) {
        want[r] = need;
        ok = false;
      }
    }
    if (ok) break;
    if (attempt == 3) return fail(c, SC_ERR_LIST_OVERFLOW, "pair lists kept overflowing");
  }
  CK(cudaMemsetAsync(c->d.n_rebuilds, 0, sizeof(long long), c->st));
  CK(cudaMemsetAsync(c->d.rep_rebuilds, 0, sizeof(long long) * nrep, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->loaded = true;
  c->i_step = 0;
  c->midstep = 1;
  c->mcount = 0;
  return SC_OK;
}

sc_status sc_add_filaments(sc_ctx *c, int n, const sc_filament_params *p,
                           const double *site_xyz, int64_t n_sites_total) {
  if (!c) return SC_ERR_INVALID_ARG;
  const double radius = c->desc.system_radius;
  const uint32_t seed = c->desc.seed;
  const int32_t nf = n;
  return add_systems(c, 1, &radius, &seed, &nf, n, p, site_xyz, n_sites_total);
}

sc_status sc_add_replicas(sc_ctx *c, int n_replicas, const double *system_radius,
                          const uint32_t *seed, const int32_t *n_filaments, int n,
                          const sc_filament_params *p, const double *site_xyz,
                          int64_t n_sites_total) {
  return add_systems(c, n_replicas, system_radius, seed, n_filaments, n, p, site_xyz,
                     n_sites_total);
}

sc_status sc_interact(sc_ctx *c) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  // ZeroForces + Interact of the next step.
  CKS(thermo_reserve(c, 1));
  c->i_step++;
  tether_if_due(c);
  CKS(maybe_rebuild(c));
  if (c->desc.interaction_flag) CKS(pair_stage(c));
  CK(cudaGetLastError());
  c->pairs_ready = true;
  return SC_OK;
}

sc_status sc_update_positions(sc_ctx *c) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  if (!c->pairs_ready) return fail(c, SC_ERR_INVALID_ARG, "sc_update_positions needs sc_interact first");
  CKS(timed(c, [&] {
    return sc::launch_integrate(c->k, c->d, c->nblocks, c->C, c->midstep, c->rbuf,
                                c->desc.interaction_flag ? 1 : 0, c->capture, c->prec,
                                c->fast, c->st);
  }));
  if (c->midstep && c->desc.stoch_flag)
    c->launches += sc::launch_advance_mcount(c->d, c->st);
  CK(cudaGetLastError());
  if (c->midstep && c->desc.stoch_flag) c->mcount++;
  c->midstep = !c->midstep;
  c->rbuf = 1 - c->rbuf;
  c->pairs_ready = false;
  return SC_OK;
}

sc_status sc_step(sc_ctx *c, int n) {
  if (!c || !c->loaded || n < 0) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  for (int i = 0; i < n; ++i) CKS(step_once(c));
  return SC_OK;
}

// Captures one graph: WHILE (loop_count > 0) { decide -> IF(rebuild) ->
// midstep -> full step -> tail }.  Built for the current geometry-buffer
// parity; every BD step returns the parity to where it started.
static sc_status build_graph(sc_ctx *c) {
  drop_graph(c);
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h_loop;
  CK(cudaGraphConditionalHandleCreate(&h_loop, g, 0, 0));
  // head kernel: sets the loop condition
  CK(cudaStreamBeginCaptureToGraph(c->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  sc::launch_loop_head(c->d, h_loop, c->st);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, nullptr, &deps, &ndeps));
  std::vector<cudaGraphNode_t> head(deps, deps + ndeps);
  CK(cudaStreamEndCapture(c->st, &g));
  // WHILE node
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = h_loop;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  CK(cudaGraphAddNode(&wnode, g, head.data(), head.size(), &wp));
  cudaGraph_t body = wp.conditional.phGraph_out[0];
  const int interaction = c->desc.interaction_flag ? 1 : 0;
  std::vector<cudaGraphNode_t> tail;
  if (interaction) {
    cudaGraphConditionalHandle h_if;
    CK(cudaGraphConditionalHandleCreate(&h_if, body, 0, 0));
    CK(cudaStreamBeginCaptureToGraph(c->st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    sc::launch_decide(c->k, c->d, h_if, c->st);
    CK(cudaStreamGetCaptureInfo(c->st, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> dec(deps, deps + ndeps);
    CK(cudaStreamEndCapture(c->st, &body));
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h_if;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, body, dec.data(), dec.size(), &ip));
    cudaGraph_t rb = ip.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(c->st, rb, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    long long launches = c->launches;
    rebuild_enqueue(c, true);
    c->launches = launches;
    CK(cudaStreamEndCapture(c->st, &rb));
    tail.push_back(inode);
  }
  CK(cudaStreamBeginCaptureToGraph(c->st, body, tail.empty() ? nullptr : tail.data(), nullptr,
                                   tail.size(), cudaStreamCaptureModeRelaxed));
  const bool fuse = fused_pairs(c);
  c->graph_fused = fuse;
  for (int half = 0; half < 2; ++half) {
    const int rb = half == 0 ? c->rbuf : 1 - c->rbuf;
    // The body's first kernel follows the conditional rebuild node (or the
    // body's start), not a kernel: it is launched without the programmatic
    // attribute.
    // The second half is the even (full) step: crosslink tethers first.
    if (half == 1 && interaction) sc::launch_tether(c->k, c->d, c->st);
    if (interaction && !fuse) {
      if (half == 0) {
        sc::PdlOff off;
        sc::launch_pairs(c->k, c->d, rb, c->prec, (int)(c->np + c->np / 8), c->st, c->npx);
      } else {
        sc::launch_pairs(c->k, c->d, rb, c->prec, (int)(c->np + c->np / 8), c->st, c->npx);
      }
    }
    if (interaction && c->k.thermo) sc::launch_thermo(c->k, c->d, c->prec, c->st);
    if (half == 0 && (!interaction || fuse)) {
      sc::PdlOff off;
      sc::launch_integrate(c->k, c->d, c->nblocks, c->C, 1, rb, interaction, c->capture, c->prec,
                           c->fast, c->st, fuse);
    } else {
      sc::launch_integrate(c->k, c->d, c->nblocks, c->C, half == 0 ? 1 : 0, rb, interaction,
                           c->capture, c->prec, c->fast, c->st, fuse);
    }
  }
  sc::launch_loop_tail(c->d, c->desc.stoch_flag ? 1 : 0, h_loop, c->st);
  CK(cudaStreamEndCapture(c->st, &body));
  CK(cudaGetLastError());
  cudaError_t e = cudaGraphInstantiate(&c->graph_exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->graph_exec = nullptr;
    return fail(c, SC_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  }
  c->graph_rbuf = c->rbuf;
  return SC_OK;
}

sc_status sc_step_graph(sc_ctx *c, int n) {
  if (!c || !c->loaded || n < 0) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  // Align to a midstep with the host-driven loop, then run whole BD steps.
  if (!c->midstep && n > 0) {
    CKS(step_once(c));
    --n;
  }
  int bd = n / 2;
  if (bd > 0) {
    CKS(thermo_reserve(c, 2 * (long long)bd));
    // The list must have room to grow by half before a captured run.
    CKS(sync_pair_count(c));
    if (c->reps.size() == 1 && c->np + c->np / 2 > c->pcap)
      CKS(ensure_pair_capacity(c, c->np + c->np / 2));
    if (!c->gev0) {
      CK(cudaEventCreate(&c->gev0));
      CK(cudaEventCreate(&c->gev1));
    }
    c->graph_ms = 0.0;
    // A rebuild whose list outgrows its segment stops the run at that BD
    // step, with nothing past the rebuild done; the list then grows, the
    // rebuild is redone host-side and the run resumes with that step.
    for (int attempt = 0; bd > 0; ++attempt) {
      if (attempt == 8) return fail(c, SC_ERR_LIST_OVERFLOW, "pair list kept overflowing inside captured runs");
      if (!c->graph_exec || c->graph_rbuf != c->rbuf) CKS(build_graph(c));
      *c->h_loop = bd;
      CK(cudaMemcpyAsync(c->d.loop_count, c->h_loop, sizeof(int), cudaMemcpyHostToDevice, c->st));
      long long nr0 = 0, nr1 = 0;
      CK(cudaMemcpyAsync(&nr0, c->d.n_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
      CK(cudaEventRecord(c->gev0, c->st));
      CK(cudaGraphLaunch(c->graph_exec, c->st));
      CK(cudaEventRecord(c->gev1, c->st));
      CK(cudaMemcpyAsync(&nr1, c->d.n_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
      CK(cudaMemcpyAsync(c->h_loop, c->d.loop_count, sizeof(int), cudaMemcpyDeviceToHost, c->st));
      c->pairs_ready = false;
      CK(cudaMemcpyAsync(&c->hb->status, c->d.status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                         c->st));
      CK(cudaStreamSynchronize(c->st));
      const unsigned st = c->hb->status;
      const bool overflow = (st & sc::ST_LIST_OVERFLOW) != 0u;
      // BD steps completed: all of them, or those before the stopped one.
      const int done = overflow ? bd - *c->h_loop : bd;
      if (c->graph_fused && done > 0) c->slots_stale = true;
      c->i_step += 2 * (long long)done;
      if (c->desc.stoch_flag) c->mcount += done;
      {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->gev0, c->gev1));
        c->graph_ms += ms;
      }
      // Kernels the graph ran: loop head, per BD step decide + the two
      // tether kernels (mesh lambdas, anchor forces) + 2 steps + tail (the
      // stopped step's too), per rebuild the captured sequence.  A step is
      // its pair kernel (unless fused; near-parallel pairs are evaluated in
      // place), thermo and one or two integrator kernels.
      const int int_l = (c->d.n_wg > 0 ? 1 : 0) + (c->nblocks > 0 ? 1 : 0);
      const long long per_bd =
          c->desc.interaction_flag
              ? 2 + (c->d.nx ? 2 : 0) +
                    2 * ((c->graph_fused ? 0 : 1) + int_l + (c->k.thermo ? 1 : 0))
              : 1 + 2 * int_l;
      c->launches += 1 + (long long)(done + (overflow ? 1 : 0)) * per_bd +
                     (nr1 - nr0) * c->rebuild_kernels;
      bd -= done;
      if (!overflow) {
        CKS(readback(c));
        break;
      }
      if (st & ~sc::ST_LIST_OVERFLOW) {
        CKS(readback(c));  // reports the other error
        return fail(c, SC_ERR_LIST_OVERFLOW, "pair list overflow inside a captured run");
      }
      if (c->reps.size() != 1)
        return fail(c, SC_ERR_LIST_OVERFLOW, "a system's pair list outgrew its segment inside a captured run");
      const unsigned clear = 0u;
      CK(cudaMemcpyAsync(c->d.status, &clear, sizeof(unsigned), cudaMemcpyHostToDevice, c->st));
      CKS(sync_pair_count(c));
      CKS(grow_after_overflow(c));
      // The stopped step's due flag is still set: redo its rebuild, with
      // headroom for the rest of the run.
      CKS(rebuild(c));
      if (c->np + c->np / 2 > c->pcap) CKS(ensure_pair_capacity(c, c->np + c->np / 2));
    }
    unsigned st = c->hb->status;
    if (st & sc::ST_UNPHYSICAL) return fail(c, SC_ERR_UNPHYSICAL, "Unphysical result");
  }
  if (n % 2) CKS(step_once(c));
  return SC_OK;
}

sc_status sc_synchronize(sc_ctx *c) {
  if (!c) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  CKS(readback(c));
  return SC_OK;
}

sc_status sc_get_sites(sc_ctx *c, double *xyz) {
  if (!c || !c->loaded || !xyz) return SC_ERR_INVALID_ARG;
  return copy_soa3(c, c->d.r, c->ns, xyz);
}

sc_status sc_get_prev_sites(sc_ctx *c, double *xyz) {
  if (!c || !c->loaded || !xyz) return SC_ERR_INVALID_ARG;
  return copy_soa3(c, c->d.rp, c->ns, xyz);
}

sc_status sc_get_random_forces(sc_ctx *c, double *f) {
  if (!c || !c->loaded || !f) return SC_ERR_INVALID_ARG;
  return copy_soa3(c, c->d.fr, c->ns, f);
}

sc_status sc_set_sites(sc_ctx *c, const double *xyz) {
  if (!c || !c->loaded || !xyz) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  // One copy of the caller's x, y, z triples, split into the component
  // arrays of positions and previous positions on the device.
  CK(cudaMemcpyAsync(c->stage, xyz, sizeof(double) * 3 * (size_t)c->ns, cudaMemcpyHostToDevice,
                     c->st));
  c->launches += sc::launch_aos_to_soa(c->ns, c->nd, c->stage, c->d, c->st);
  sc::launch_init_geometry(c->k, c->d, c->rbuf, c->prec, c->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_get_bond_forces(sc_ctx *c, double *f, double *t) {
  if (!c || !c->loaded || !f || !t) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  // Bond accumulators of the last pair evaluation (Bond::force_/torque_
  // after Interact), summed from its per-bond slots.
  if (c->desc.interaction_flag) {
    CKS(materialize_slots(c));
    c->launches += sc::launch_bond_sum(c->k, c->d, c->prec, c->st);
  } else {
    for (int i = 0; i < 3; ++i) {
      CK(cudaMemsetAsync(c->d.bF[i], 0, sizeof(double) * c->nb, c->st));
      CK(cudaMemsetAsync(c->d.bT[i], 0, sizeof(double) * c->nb, c->st));
    }
  }
  CK(cudaGetLastError());
  CKS(copy_soa3(c, c->d.bF, c->nb, f));
  return copy_soa3(c, c->d.bT, c->nb, t);
}

sc_status sc_set_integrator_layout(sc_ctx *c, int warp_max_sites, int block_sites) {
  if (!c || !c->loaded || warp_max_sites < 0 || warp_max_sites > 32) return SC_ERR_INVALID_ARG;
  if (block_sites != 0 && (block_sites < 32 || block_sites > 512 || block_sites % 32))
    return fail(c, SC_ERR_INVALID_ARG, "block_sites must be 0 or a multiple of 32 in [32, 512]");
  CK(cudaSetDevice(c->desc.device));
  const int ow = c->warp_sites, ob = c->block_sites;
  c->warp_sites = warp_max_sites;
  c->block_sites = block_sites;
  sc_status st = layout_integrator(c);
  if (st != SC_OK) {
    c->warp_sites = ow;
    c->block_sites = ob;
    layout_integrator(c);
  }
  return st;
}

// Integrator autotuner.  Candidate layouts (warp kernel or not, block size)
// are timed on the context's own state: the arrays the integrator writes are
// saved first and restored afterwards, so the simulation is unchanged.  The
// fastest layout is applied and, with a cache file, recorded per shape (device,
// precision, filament count and site range) so later contexts skip the timing.
sc_status sc_autotune(sc_ctx *c, const char *cache_path, int *warp_sites_out,
                      int *block_sites_out) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, c->desc.device));
  int min_n = 1 << 30, max_n = 0;
  for (int f = 0; f < c->nf; ++f) {
    const int nn = c->site_off[f + 1] - c->site_off[f];
    min_n = std::min(min_n, nn);
    max_n = std::max(max_n, nn);
  }
  char key[512];
  const bool fuse = fused_pairs(c);
  std::snprintf(key, sizeof(key), "v2|%s|sm%d|nd%d|prec%d|fast%d|fuse%d|nf%d|ns%d|n%d-%d",
                prop.name, prop.multiProcessorCount, c->nd, c->prec,
                (c->prec == 1 && c->fast) ? 1 : 0, fuse ? 1 : 0, c->nf, c->ns, min_n, max_n);
  auto finish = [&](int w, int b) -> sc_status {
    if (warp_sites_out) *warp_sites_out = w;
    if (block_sites_out) *block_sites_out = b;
    return SC_OK;
  };
  if (cache_path) {
    if (FILE *fp = std::fopen(cache_path, "r")) {
      char line[768];
      int w = -1, b = -1;
      while (std::fgets(line, sizeof(line), fp)) {
        char *tab = std::strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        int ww, bb;
        if (std::strcmp(line, key) == 0 && std::sscanf(tab + 1, "%d %d", &ww, &bb) == 2) {
          w = ww;
          b = bb;
        }
      }
      std::fclose(fp);
      if (w >= 0) {
        CKS(sc_set_integrator_layout(c, w, b));
        return finish(w, b);
      }
    }
  }
  // Candidates: every block size that holds the longest block-kernel
  // filament, with and without the warp kernel for filaments of <= 32 sites.
  std::vector<std::pair<int, int>> cand;
  for (int w : {32, 0}) {
    if (w == 32 && min_n > 32) continue;
    const int longest = w == 32 ? (max_n > 32 ? max_n : 0) : max_n;
    if (longest == 0) {
      cand.push_back({w, 0});
      continue;
    }
    for (int bsz : {64, 96, 128, 160, 192, 256, 512})
      if (bsz >= longest && (bsz < 512 || longest > 256)) cand.push_back({w, bsz});
  }
  // Save what the integrator writes.
  const int wbuf = 1 - c->rbuf;
  std::vector<std::pair<void *, size_t>> regions;
  for (int i = 0; i < 3; ++i) {
    regions.push_back({c->d.r[i], sizeof(double) * c->ns});
    regions.push_back({c->d.rp[i], sizeof(double) * c->ns});
    regions.push_back({c->d.fr[i], sizeof(double) * c->ns});
    regions.push_back({c->d.ub[i], sizeof(double) * c->nb});
  }
  regions.push_back({c->d.dt, sizeof(double) * c->ns});
  regions.push_back({c->d.f_switch, sizeof(int) * c->nf});
  regions.push_back({c->d.f_nnorm, sizeof(int) * c->nf});
  if (c->prec == 0) regions.push_back({c->d.g64[wbuf], sizeof(sc::BondGeomF64) * c->nb});
  else regions.push_back({c->d.g32[wbuf], sizeof(sc::BondGeomF32) * c->nb});
  regions.push_back({c->d.dr_max_bits, sizeof(unsigned long long) * c->d.nrep});
  regions.push_back({c->d.status, sizeof(unsigned)});
  if (fuse) regions.push_back({c->d.pf32, sizeof(float) * 4 * c->d.pcap_total});
  size_t total = 0;
  for (auto &r : regions) total += (r.second + 255) & ~(size_t)255;
  char *save = nullptr;
  CKS(dalloc(c, &save, total));
  auto copy_all = [&](bool to_save) -> sc_status {
    size_t off = 0;
    for (auto &r : regions) {
      void *dst = to_save ? (void *)(save + off) : r.first;
      const void *src = to_save ? (const void *)r.first : (const void *)(save + off);
      CK(cudaMemcpyAsync(dst, src, r.second, cudaMemcpyDeviceToDevice, c->st));
      off += (r.second + 255) & ~(size_t)255;
    }
    return SC_OK;
  };
  CKS(copy_all(true));
  const int ow = c->warp_sites, ob = c->block_sites;
  const int interaction = c->desc.interaction_flag ? 1 : 0;
  float best = 1e30f;
  std::pair<int, int> best_lay{ow, ob};
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  sc_status st = SC_OK;
  for (auto lay : cand) {
    c->warp_sites = lay.first;
    c->block_sites = lay.second;
    st = layout_integrator(c);
    if (st != SC_OK) break;
    for (int it = 0; it < 2; ++it)
      sc::launch_integrate(c->k, c->d, c->nblocks, c->C, 1 - it, c->rbuf, interaction, 0,
                           c->prec, c->fast, c->st, fuse);
    cudaEventRecord(e0, c->st);
    for (int it = 0; it < 8; ++it)
      sc::launch_integrate(c->k, c->d, c->nblocks, c->C, 1 - (it & 1), c->rbuf, interaction, 0,
                           c->prec, c->fast, c->st, fuse);
    cudaEventRecord(e1, c->st);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      st = fail(c, SC_ERR_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) {
      best = ms;
      best_lay = lay;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CKS(copy_all(false));
  CK(cudaStreamSynchronize(c->st));
  dfree(c, save);
  CKS(st);
  c->warp_sites = best_lay.first;
  c->block_sites = best_lay.second;
  CKS(layout_integrator(c));
  if (cache_path) {
    if (FILE *fp = std::fopen(cache_path, "a")) {
      std::fprintf(fp, "%s\t%d %d %.2f\n", key, best_lay.first, best_lay.second,
                   1000.0 * best / 8);
      std::fclose(fp);
    }
  }
  return finish(best_lay.first, best_lay.second);
}

// ---------------------------------------------------------------------------
// Checkpoint / restore: every piece of state a later step reads, so that a
// restored context continues bit for bit.

namespace {
struct CkptHeader {
  char magic[8];       // "SCB200CK"
  int32_t version, nd, prec, nrep, nf, ns, nb, nx;
  int32_t midstep, rbuf, stoch, pad;
  int64_t i_step;
  uint64_t mcount;
  int64_t n_rebuilds;
  int64_t payload_bytes;  // everything after the header
  uint64_t payload_hash;  // payload_hash() of those bytes
};
constexpr int32_t kCkptVersion = 2;

// 64-bit FNV-1a over 8-byte words (then the tail bytes): any change to a
// checkpoint's payload changes it, in one host pass at memory speed.
uint64_t payload_hash(const char *p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h = (h ^ w) * 1099511628211ull;
  }
  for (; i < n; ++i) h = (h ^ (unsigned char)p[i]) * 1099511628211ull;
  return h;
}

// Device regions of a checkpoint, in file order.  Pair-list regions are
// sized for P pair slots (recorded per system first); the pointers are the
// context's own, valid when P is its current capacity.  Index regions carry
// their kind, for the range checks of a restore.
enum RegionKind { RK_DATA, RK_NP, RK_EOFF, RK_ECNT, RK_PA, RK_PB, RK_POS1, RK_POS2, RK_EENT };
struct Region {
  void *ptr;
  size_t bytes;
  RegionKind kind = RK_DATA;
};

std::vector<Region> state_regions(sc_ctx *c, long long pcap = -1) {
  std::vector<Region> v;
  const DevState &d = c->d;
  const size_t ns = c->ns, nb = c->nb, nf = c->nf, nrep = c->d.nrep;
  for (int i = 0; i < 3; ++i) v.push_back({d.r[i], sizeof(double) * ns});
  for (int i = 0; i < 3; ++i) v.push_back({d.rp[i], sizeof(double) * ns});
  for (int i = 0; i < 3; ++i) v.push_back({d.fr[i], sizeof(double) * ns});
  for (int i = 0; i < 3; ++i) v.push_back({d.dz[i], sizeof(double) * ns});
  v.push_back({d.dt, sizeof(double) * ns});
  v.push_back({d.f_switch, sizeof(int) * nf});
  v.push_back({d.f_nnorm, sizeof(int) * nf});
  v.push_back({d.dr_max_bits, sizeof(unsigned long long) * nrep});
  v.push_back({d.np_rep, sizeof(int) * nrep, RK_NP});
  v.push_back({d.rep_rebuilds, sizeof(long long) * nrep});
  v.push_back({d.e_off, sizeof(int) * nb, RK_EOFF});
  v.push_back({d.e_cnt, sizeof(int) * nb, RK_ECNT});
  // Bond orientations and the geometry the next pair stage reads, as the
  // integrator wrote them (the fast integrator's bits differ from a
  // re-derivation).
  for (int i = 0; i < 3; ++i) v.push_back({d.ub[i], sizeof(double) * nb});
  if (c->prec == 0) v.push_back({d.g64[c->rbuf], sizeof(sc::BondGeomF64) * nb});
  else v.push_back({d.g32[c->rbuf], sizeof(sc::BondGeomF32) * nb});
  const size_t P = (size_t)(pcap >= 0 ? pcap : c->pcap);
  v.push_back({d.pa, sizeof(int) * P, RK_PA});
  v.push_back({d.pb, sizeof(int) * P, RK_PB});
  v.push_back({d.pos1, sizeof(int) * P, RK_POS1});  // where each pair writes its two
  v.push_back({d.pos2, sizeof(int) * P, RK_POS2});  // contributions
  v.push_back({d.e_ent, sizeof(int) * 2 * P, RK_EENT});
  if (c->prec == 0) {
    v.push_back({d.pf64, sizeof(double) * 4 * P});
    v.push_back({d.cf64, sizeof(double) * 16 * P});
  } else {
    v.push_back({d.pf32, sizeof(float) * 4 * P});
    v.push_back({d.cf32, sizeof(float) * 16 * P});
  }
  if (d.nx) {
    v.push_back({d.xl_c, sizeof(double) * 16 * (size_t)d.nx});
    v.push_back({d.xl_F, sizeof(double) * 4 * (size_t)d.nx});
    v.push_back({d.xl_M, sizeof(double) * 2 * (size_t)d.nx});
  }
  if (c->k.thermo) {  // pair virial records and the running virial sums
    if (c->prec == 0) v.push_back({d.pv64, sizeof(double) * 4 * P});
    else v.push_back({d.pv32, sizeof(float) * 4 * P});
    v.push_back({d.th_acc, sizeof(double) * 9 * nrep});
    v.push_back({d.th_istep, sizeof(long long) * nrep});
  }
  return v;
}
}  // namespace

sc_status sc_checkpoint(sc_ctx *c, void *buf, size_t cap, size_t *size) {
  if (!c || !c->loaded || !size) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  const int nrep = c->d.nrep;
  auto regions = state_regions(c);
  size_t need = sizeof(CkptHeader) + sizeof(int32_t) * nrep;
  for (auto &r : regions) need += r.bytes;
  *size = need;
  if (!buf) return SC_OK;
  if (cap < need) return fail(c, SC_ERR_INVALID_ARG, "checkpoint needs %zu bytes", need);
  CKS(materialize_slots(c));
  CKS(readback(c));
  long long nr = 0;
  CK(cudaMemcpyAsync(&nr, c->d.n_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "SCB200CK", 8);
  h.version = kCkptVersion;
  h.nd = c->nd;
  h.prec = c->prec;
  h.nrep = nrep;
  h.nf = c->nf;
  h.ns = c->ns;
  h.nb = c->nb;
  h.nx = c->d.nx;
  h.midstep = c->midstep;
  h.rbuf = c->rbuf;
  h.stoch = c->desc.stoch_flag;
  h.i_step = c->i_step;
  h.mcount = c->mcount;
  h.n_rebuilds = nr;
  h.payload_bytes = (int64_t)(need - sizeof(h));
  char *out = (char *)buf + sizeof(h);
  for (int r = 0; r < nrep; ++r) {
    const int32_t pc = c->reps[r].pcap;
    std::memcpy(out, &pc, sizeof(pc));
    out += sizeof(pc);
  }
  for (auto &r : regions) {
    CK(cudaMemcpyAsync(out, r.ptr, r.bytes, cudaMemcpyDeviceToHost, c->st));
    out += r.bytes;
  }
  CK(cudaStreamSynchronize(c->st));
  h.payload_hash = payload_hash((const char *)buf + sizeof(h), need - sizeof(h));
  std::memcpy(buf, &h, sizeof(h));
  return SC_OK;
}

// The index ranges of a checkpoint's pair lists, checked on the host before
// anything is uploaded, so that no blob can send a later launch outside its
// arrays: system r's live pairs join two of its bonds and write two of its
// slots, and every entry of its bonds names one of its live pairs.
sc_status check_pair_indices(sc_ctx *c, const std::vector<long long> &caps,
                             const std::vector<Region> &regions, const char *payload) {
  const int32_t *ix[RK_EENT + 1] = {};
  for (const Region &r : regions) {
    if (r.kind != RK_DATA) ix[r.kind] = (const int32_t *)payload;
    payload += r.bytes;
  }
  const int32_t *np = ix[RK_NP], *e_off = ix[RK_EOFF], *e_cnt = ix[RK_ECNT];
  const int32_t *pa = ix[RK_PA], *pb = ix[RK_PB], *pos1 = ix[RK_POS1], *pos2 = ix[RK_POS2];
  const int32_t *e_ent = ix[RK_EENT];
  long long p0 = 0;
  for (size_t r = 0; r < caps.size(); ++r) {
    const sc::ReplicaConst &R = c->reps[r];
    const long long n = np[r], cap = caps[r], s0 = 2 * p0, s1 = 2 * (p0 + cap);
    if (n < 0 || n > cap)
      return fail(c, SC_ERR_INVALID_ARG, "checkpoint: system %zu holds %lld pairs", r, n);
    for (long long p = p0; p < p0 + n; ++p)
      if (pa[p] < R.b0 || pa[p] >= R.b0 + R.nb || pb[p] < R.b0 || pb[p] >= R.b0 + R.nb ||
          pos1[p] < s0 || pos1[p] >= s1 || pos2[p] < s0 || pos2[p] >= s1)
        return fail(c, SC_ERR_INVALID_ARG, "checkpoint: pair %lld out of range", p);
    for (long long b = R.b0; b < R.b0 + R.nb; ++b) {
      const long long e0 = e_off[b], ec = e_cnt[b];
      if (ec < 0 || e0 < s0 || e0 + ec > s1)
        return fail(c, SC_ERR_INVALID_ARG, "checkpoint: bond %lld entries out of range", b);
      for (long long e = e0; e < e0 + ec; ++e)
        if (e_ent[e] < 0 || (e_ent[e] >> 1) < p0 || (e_ent[e] >> 1) >= p0 + n)
          return fail(c, SC_ERR_INVALID_ARG, "checkpoint: entry %lld out of range", e);
    }
    p0 += cap;
  }
  return SC_OK;
}

sc_status sc_restore(sc_ctx *c, const void *buf, size_t size) {
  if (!c || !c->loaded || !buf) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  CkptHeader h;
  if (size < sizeof(h)) return fail(c, SC_ERR_INVALID_ARG, "checkpoint truncated");
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, "SCB200CK", 8) != 0 || h.version != kCkptVersion)
    return fail(c, SC_ERR_INVALID_ARG, "not a checkpoint of this library (version %d)",
                kCkptVersion);
  if (h.nd != c->nd || h.prec != c->prec || h.nrep != c->d.nrep || h.nf != c->nf ||
      h.ns != c->ns || h.nb != c->nb || h.nx != c->d.nx)
    return fail(c, SC_ERR_INVALID_ARG, "checkpoint of a different system shape");
  if (h.payload_bytes < 0 || size - sizeof(h) < (size_t)h.payload_bytes)
    return fail(c, SC_ERR_INVALID_ARG, "checkpoint truncated");
  const char *payload = (const char *)buf + sizeof(h);
  if (payload_hash(payload, (size_t)h.payload_bytes) != h.payload_hash)
    return fail(c, SC_ERR_INVALID_ARG, "checkpoint corrupted (payload hash differs)");
  if ((h.rbuf != 0 && h.rbuf != 1) || (h.midstep != 0 && h.midstep != 1))
    return fail(c, SC_ERR_INVALID_ARG, "checkpoint: bad step state");
  // Everything is checked before the context changes.
  const int nrep = h.nrep;
  const char *in = payload;
  if ((size_t)h.payload_bytes < sizeof(int32_t) * nrep)
    return fail(c, SC_ERR_INVALID_ARG, "checkpoint truncated");
  std::vector<long long> caps(nrep);
  long long total = 0;
  for (int r = 0; r < nrep; ++r) {
    int32_t pc;
    std::memcpy(&pc, in, sizeof(pc));
    in += sizeof(pc);
    if (pc < 1) return fail(c, SC_ERR_INVALID_ARG, "checkpoint: system %d has %d pair slots", r, pc);
    caps[r] = pc;
    total += pc;
  }
  if (total >= (1ll << 30)) return fail(c, SC_ERR_INVALID_ARG, "checkpoint: %lld pair slots", total);
  {
    const auto sized = state_regions(c, total);
    size_t need = sizeof(int32_t) * nrep;
    for (auto &r : sized) need += r.bytes;
    if ((size_t)h.payload_bytes < need) return fail(c, SC_ERR_INVALID_ARG, "checkpoint truncated");
    CKS(check_pair_indices(c, caps, sized, in));
  }
  // The checkpoint's segments; a failed allocation leaves the context as it
  // was.  Then rbuf selects the geometry buffer the checkpoint fills.
  CKS(layout_pairs(c, caps));
  c->rbuf = h.rbuf;
  auto regions = state_regions(c);
  for (auto &r : regions) {
    CK(cudaMemcpyAsync(r.ptr, in, r.bytes, cudaMemcpyHostToDevice, c->st));
    in += r.bytes;
  }
  const long long nr = h.n_rebuilds;
  CK(cudaMemcpyAsync(c->d.n_rebuilds, &nr, sizeof(long long), cudaMemcpyHostToDevice, c->st));
  const unsigned long long mc = h.mcount;
  CK(cudaMemcpyAsync(c->d.mcount, &mc, sizeof(mc), cudaMemcpyHostToDevice, c->st));
  const unsigned zero = 0;
  CK(cudaMemcpyAsync(c->d.status, &zero, sizeof(zero), cudaMemcpyHostToDevice, c->st));
  c->i_step = h.i_step;
  c->mcount = h.mcount;
  c->midstep = h.midstep;
  c->pairs_ready = false;
  c->slots_stale = false;  // the checkpoint's slots hold its last evaluation
  if (c->k.thermo) {  // records restart from the restored step
    CK(cudaMemsetAsync(c->d.th_nrec, 0, sizeof(long long) * c->d.nrep, c->st));
    CK(cudaMemsetAsync(c->d.th_ticket, 0, sizeof(unsigned) * c->d.nrep, c->st));
    c->th_i0 = c->i_step;
    c->th_pulled = 0;
    c->th_host.clear();
  }
  // The FP64 record of mixed precision serves only the geometry getter.
  if (c->prec != 0) sc::launch_init_geometry(c->k, c->d, 0, 0, c->st, false);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  CKS(sync_pair_count(c));
  drop_graph(c);
  return SC_OK;
}

sc_status sc_set_noise_key(sc_ctx *c, int replica, uint32_t seed) {
  if (!c || !c->loaded || replica < -1 || replica >= c->d.nrep) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  for (int r = 0; r < c->d.nrep; ++r)
    if (replica < 0 || r == replica) c->reps[r].seed = seed;
  return upload_reps(c);
}

// ---------------------------------------------------------------------------
// Reference-format output files: the filament species' spec and posit files
// (SpeciesBase::InitSpecFile / InitPositFile, src/species_base.cpp:13-70;
// Species::WriteSpecs / WritePosits, include/simcore/species.hpp:221-233;
// Mesh::WriteSpec, src/mesh.cpp:482-492; Filament::WriteSpec / WritePosit,
// src/filament.cpp:1314-1361), at the cadence of OutputManager::WriteOutputs
// (include/simcore/output_manager.hpp:112-127).


sc_status sc_output_open(sc_ctx *c, const char *run_name, const char *species_name, int n_steps,
                         int n_posit, int n_spec) {
  if (!c || !c->loaded || !run_name || !species_name || n_steps < 0 || n_posit < 0 ||
      n_spec < 0)
    return SC_ERR_INVALID_ARG;
  if (c->out.open) return fail(c, SC_ERR_INVALID_ARG, "output already open");
  CK(cudaSetDevice(c->desc.device));
  sc_ctx::Output &o = c->out;
  o.n_steps = n_steps;
  o.n_posit = n_posit;
  o.n_spec = n_spec;
  const size_t nrep = c->reps.size();
  o.spec.assign(nrep, nullptr);
  o.posit.assign(nrep, nullptr);
  for (size_t r = 0; r < nrep; ++r) {
    std::string run = run_name;
    if (nrep > 1) {
      char sfx[32];
      std::snprintf(sfx, sizeof(sfx), "_r%03zu", r);
      run += sfx;
    }
    const std::string base = run + "_filament_" + species_name;
    for (int kind = 0; kind < 2; ++kind) {
      const int cadence = kind == 0 ? n_spec : n_posit;
      if (cadence <= 0) continue;
      const std::string name = base + (kind == 0 ? ".spec" : ".posit");
      FILE *f = std::fopen(name.c_str(), "wb");
      if (!f) return fail(c, SC_ERR_INVALID_ARG, "cannot open %s", name.c_str());
      put(f, (int32_t)n_steps);
      put(f, (int32_t)cadence);
      put(f, c->desc.delta);
      (kind == 0 ? o.spec : o.posit)[r] = f;
    }
  }
  const size_t doubles = 3 * (size_t)c->ns + 9 * (size_t)c->nf;
  CKS(dalloc(c, &o.d_snap, doubles));
  if (cudaHostAlloc((void **)&o.h_snap, sizeof(double) * doubles, cudaHostAllocDefault) !=
      cudaSuccess) {
    cudaGetLastError();
    return fail(c, SC_ERR_OOM, "pinned allocation failed");
  }
  CK(cudaStreamCreateWithFlags(&o.out_st, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&o.taken, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&o.copied, cudaEventDisableTiming));
  o.open = true;
  return SC_OK;
}

sc_status sc_output_write(sc_ctx *c) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  sc_ctx::Output &o = c->out;
  if (!o.open) return fail(c, SC_ERR_INVALID_ARG, "output not open");
  CK(cudaSetDevice(c->desc.device));
  const bool spec = o.n_spec > 0 && c->i_step % o.n_spec == 0;
  const bool posit = o.n_posit > 0 && c->i_step % o.n_posit == 0;
  if (!spec && !posit) return SC_OK;
  CKS(output_flush(c));  // the previous frame, whose copy overlapped the steps since
  // Snapshot on the simulation stream, copy on the output stream.
  if (spec)
    c->launches += sc::launch_soa_to_aos(c->ns, c->d.r[0], c->d.r[1], c->d.r[2], o.d_snap, c->st);
  if (posit)
    c->launches += sc::launch_filament_averages(c->k, c->d, o.d_snap + 3 * (size_t)c->ns, c->st);
  CK(cudaGetLastError());
  CK(cudaEventRecord(o.taken, c->st));
  CK(cudaStreamWaitEvent(o.out_st, o.taken, 0));
  if (spec)
    CK(cudaMemcpyAsync(o.h_snap, o.d_snap, sizeof(double) * 3 * (size_t)c->ns,
                       cudaMemcpyDeviceToHost, o.out_st));
  if (posit)
    CK(cudaMemcpyAsync(o.h_snap + 3 * (size_t)c->ns, o.d_snap + 3 * (size_t)c->ns,
                       sizeof(double) * 9 * (size_t)c->nf, cudaMemcpyDeviceToHost, o.out_st));
  CK(cudaEventRecord(o.copied, o.out_st));
  o.pending_spec = spec;
  o.pending_posit = posit;
  return SC_OK;
}

sc_status sc_output_close(sc_ctx *c) {
  if (!c) return SC_ERR_INVALID_ARG;
  sc_ctx::Output &o = c->out;
  if (!o.open) return SC_OK;
  cudaSetDevice(c->desc.device);
  sc_status st = output_flush(c);
  for (FILE *f : o.spec)
    if (f) std::fclose(f);
  for (FILE *f : o.posit)
    if (f) std::fclose(f);
  o.spec.clear();
  o.posit.clear();
  if (o.out_st) cudaStreamSynchronize(o.out_st);
  if (o.h_snap) cudaFreeHost(o.h_snap);
  if (o.d_snap) dfree(c, o.d_snap);
  if (o.taken) cudaEventDestroy(o.taken);
  if (o.copied) cudaEventDestroy(o.copied);
  if (o.out_st) cudaStreamDestroy(o.out_st);
  o = sc_ctx::Output{};
  return st;
}

// ---------------------------------------------------------------------------
// Filament analyses on the device (FilamentSpecies::RunAnalysis family).

sc_status sc_analysis_sample(sc_ctx *c, int n_bins) {
  if (!c || !c->loaded || n_bins < 1) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  sc_ctx::Analysis &a = c->an;
  if (a.n_bins && a.n_bins != n_bins)
    return fail(c, SC_ERR_INVALID_ARG, "histogram bins changed between samples");
  if (!a.acc) {
    int maxn = 0;
    for (int f = 0; f < c->nf; ++f) maxn = std::max(maxn, c->site_off[f + 1] - c->site_off[f]);
    a.n_bins = n_bins;
    a.max_joints = std::max(1, maxn - 2);
    const size_t nrep = c->reps.size();
    CKS(dalloc(c, &a.acc, 2 * nrep));
    CK(cudaMemsetAsync(a.acc, 0, sizeof(double) * 2 * nrep, c->st));
    CKS(dalloc(c, &a.hist, nrep * a.max_joints * (size_t)n_bins));
    CK(cudaMemsetAsync(a.hist, 0, sizeof(int) * nrep * a.max_joints * (size_t)n_bins, c->st));
  }
  c->launches += sc::launch_analysis_sample(c->k, c->d, a.n_bins, a.max_joints, a.acc, a.hist, c->st);
  CK(cudaGetLastError());
  a.n_samples++;
  return SC_OK;
}

sc_status sc_analysis_results(sc_ctx *c, double *mse2e, double *mse2e_err, int64_t *n_samples,
                              int32_t *max_joints, int64_t *theta_hist) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  sc_ctx::Analysis &a = c->an;
  const int nrep = (int)c->reps.size();
  if (n_samples) *n_samples = a.n_samples;
  if (max_joints) *max_joints = a.max_joints;
  if (!a.acc || a.n_samples == 0) return SC_OK;
  std::vector<double> acc(2 * (size_t)nrep);
  CK(cudaMemcpyAsync(acc.data(), a.acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, c->st));
  std::vector<int> hist((size_t)nrep * a.max_joints * a.n_bins);
  CK(cudaMemcpyAsync(hist.data(), a.hist, sizeof(int) * hist.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  // FilamentSpecies::FinalizeMse2eAnalysis (src/filament_species.cpp:686-698).
  for (int r = 0; r < nrep; ++r) {
    const double num = c->reps[r].nf, ns = (double)a.n_samples;
    const double m = acc[2 * r] / (ns * num), m2 = acc[2 * r + 1] / (ns * num);
    if (mse2e) mse2e[r] = m;
    if (mse2e_err) mse2e_err[r] = std::sqrt((m2 - m * m) / (num * ns));
  }
  if (theta_hist)
    for (size_t i = 0; i < hist.size(); ++i) theta_hist[i] = hist[i];
  return SC_OK;
}

sc_status sc_diffusion_init(sc_ctx *c, int interval) {
  if (!c || !c->loaded || interval < 1) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  sc_ctx::Diffusion &a = c->dif;
  const size_t nrep = c->reps.size();
  if (!a.avg) {
    CKS(dalloc(c, &a.avg, 9 * (size_t)c->nf));
    CKS(dalloc(c, &a.pos0, 3 * (size_t)c->nf));
    CKS(dalloc(c, &a.u0, 3 * (size_t)c->nf));
  }
  if (a.interval != interval) {
    dfree(c, a.acc);
    a.acc = nullptr;
    CKS(dalloc(c, &a.acc, 4 * nrep * (size_t)interval));
  }
  CK(cudaMemsetAsync(a.acc, 0, sizeof(double) * 4 * nrep * interval, c->st));
  a.interval = interval;
  a.t = 0;
  a.n_samples = 0;
  // SpherocylinderSpecies::UpdateInitPositions: the current averages.
  c->launches += sc::launch_filament_averages(c->k, c->d, a.avg, c->st);
  c->launches += sc::launch_aos_to_origins(c->nf, a.avg, a.pos0, a.u0, c->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_diffusion_sample(sc_ctx *c) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  sc_ctx::Diffusion &a = c->dif;
  if (!a.acc) return fail(c, SC_ERR_INVALID_ARG, "sc_diffusion_sample needs sc_diffusion_init");
  CK(cudaSetDevice(c->desc.device));
  const int restart = a.t + 1 == a.interval ? 1 : 0;
  c->launches += sc::launch_filament_averages(c->k, c->d, a.avg, c->st);
  c->launches += sc::launch_diffusion_sample(c->k, c->d, a.avg, a.pos0, a.u0, a.acc, a.t,
                                             a.interval, restart, c->st);
  CK(cudaGetLastError());
  a.t = restart ? 0 : a.t + 1;
  a.n_samples++;
  return SC_OK;
}

sc_status sc_diffusion_results(sc_ctx *c, double *msd, double *msd_err, double *vcf,
                               double *vcf_err) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  sc_ctx::Diffusion &a = c->dif;
  if (!a.acc) return fail(c, SC_ERR_INVALID_ARG, "sc_diffusion_results needs sc_diffusion_init");
  CK(cudaSetDevice(c->desc.device));
  const int nrep = (int)c->reps.size(), T = a.interval;
  std::vector<double> acc(4 * (size_t)nrep * T);
  CK(cudaMemcpyAsync(acc.data(), a.acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  // SpherocylinderSpecies::FinalizeDiffusionAnalysis
  // (src/spherocylinder_species.cpp:125-134).
  for (int r = 0; r < nrep; ++r) {
    const double *o = acc.data() + 4 * (size_t)T * r;
    const double n = c->reps[r].nf;
    for (int t = 0; t < T; ++t) {
      const size_t i = (size_t)r * T + t;
      if (msd) msd[i] = o[t] / o[T + t];
      if (vcf) vcf[i] = o[2 * T + t] / o[3 * T + t];
      if (msd_err) msd_err[i] = 1.0 / std::sqrt(n * o[T + t]);
      if (vcf_err) vcf_err[i] = 1.0 / std::sqrt(n * o[3 * T + t]);
    }
  }
  return SC_OK;
}

sc_status sc_global_order(sc_ctx *c, double *polar, double *nematic) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  sc_ctx::Analysis &a = c->an;
  const int nrep = (int)c->reps.size();
  if (!a.order) CKS(dalloc(c, &a.order, 12 * (size_t)nrep));
  c->launches += sc::launch_global_order(c->k, c->d, a.order, c->st);
  CK(cudaGetLastError());
  std::vector<double> o(12 * (size_t)nrep);
  CK(cudaMemcpyAsync(o.data(), a.order, sizeof(double) * o.size(), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int r = 0; r < nrep; ++r) {
    for (int i = 0; i < 3; ++i)
      if (polar) polar[3 * (size_t)r + i] = o[12 * (size_t)r + i];
    for (int i = 0; i < 9; ++i)
      if (nematic) nematic[9 * (size_t)r + i] = o[12 * (size_t)r + 3 + i];
  }
  return SC_OK;
}

sc_status sc_add_crosslinks(sc_ctx *c, int n, const int32_t *site_a, const int32_t *site_b,
                            double k_spring, double k_spring_compress, double rest_length) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  if (c->d.nx) return fail(c, SC_ERR_INVALID_ARG, "crosslinks already added");
  if (c->i_step != 0) return fail(c, SC_ERR_INVALID_ARG, "crosslinks must be added before the first step");
  if (n <= 0 || !site_a || !site_b) return fail(c, SC_ERR_INVALID_ARG, "bad crosslink arrays");
  if (!(k_spring >= 0) || !(rest_length >= 0))
    return fail(c, SC_ERR_INVALID_ARG, "bad spring constants");
  CK(cudaSetDevice(c->desc.device));
  // Anchor::AttachObjLambda (src/anchor.cpp:284-316): an anchor on site j of
  // a filament is bound to bond j at lambda 0, one on the last site to the
  // last bond at lambda = its length; its mesh lambda is the bond's (the
  // summed lengths of the bonds before it, Mesh::UpdateBondPositions,
  // src/mesh.cpp:324-330) plus lambda.  The lengths are Bond::ReInit's, from
  // the loaded sites.
  std::vector<double> xyz(3 * (size_t)c->ns);
  CKS(copy_soa3(c, c->d.r, c->ns, xyz.data()));
  std::vector<double> blen(c->nb), bml(c->nb);
  for (int f = 0; f < c->nf; ++f) {
    double true_length = 0.0;
    for (int s0 = c->site_off[f]; s0 < c->site_off[f + 1] - 1; ++s0) {
      double l = 0.0;
      for (int i = 0; i < c->nd; ++i) {
        const double u = xyz[3 * (size_t)(s0 + 1) + i] - xyz[3 * (size_t)s0 + i];
        l += u * u;
      }
      const int b = s0 - f;
      blen[b] = std::sqrt(l);
      bml[b] = true_length;
      true_length += blen[b];
    }
  }
  std::vector<int> bond(2 * (size_t)n), xfil(2 * (size_t)n);
  std::vector<double> xM(2 * (size_t)n);
  for (int x = 0; x < n; ++x)
    for (int a = 0; a < 2; ++a) {
      const int site = a == 0 ? site_a[x] : site_b[x];
      if (site < 0 || site >= c->ns)
        return fail(c, SC_ERR_INVALID_ARG, "crosslink %d: site %d out of range", x, site);
      const int f = (int)(std::upper_bound(c->site_off.begin(), c->site_off.end(), site) -
                          c->site_off.begin()) - 1;
      const bool last = site == c->site_off[f + 1] - 1;
      const int b = last ? site - f - 1 : site - f;
      const size_t A = 2 * (size_t)x + a;
      bond[A] = b;
      xfil[A] = f;
      xM[A] = bml[b] + (last ? blen[b] : 0.0);
      if (a == 1 && c->fil_rep[f] != c->fil_rep[xfil[A - 1]])
        return fail(c, SC_ERR_INVALID_ARG, "crosslink %d joins two systems", x);
    }
  // Per-bond anchor lists, ascending anchor id (link order, anchor 0 first):
  // each anchor on its bond and that bond's neighbours in the filament, the
  // bonds it can move to as the filament's bonds stretch.
  auto first_bond = [&](int f) { return c->site_off[f] - f; };
  auto last_bond = [&](int f) { return c->site_off[f + 1] - f - 2; };
  std::vector<int> off(c->nb + 1, 0), ent;
  for (int A = 0; A < 2 * n; ++A)
    for (int b = std::max(bond[A] - 1, first_bond(xfil[A]));
         b <= std::min(bond[A] + 1, last_bond(xfil[A])); ++b)
      off[b + 1]++;
  for (int b = 0; b < c->nb; ++b) off[b + 1] += off[b];
  ent.resize(off[c->nb]);
  {
    std::vector<int> fill(off.begin(), off.end() - 1);
    for (int A = 0; A < 2 * n; ++A)
      for (int b = std::max(bond[A] - 1, first_bond(xfil[A]));
           b <= std::min(bond[A] + 1, last_bond(xfil[A])); ++b)
        ent[fill[b]++] = A;
  }
  auto up = [&](auto **dst, const auto &v) -> sc_status {
    using T = typename std::remove_reference<decltype(v)>::type::value_type;
    T *q = nullptr;
    CKS(dalloc(c, &q, v.size()));
    CK(cudaMemcpyAsync(q, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, c->st));
    *dst = q;
    return SC_OK;
  };
  int *qi = nullptr;
  double *qd = nullptr;
  CKS(up(&qi, xfil)); c->d.xl_fil = qi;
  CKS(up(&qi, off)); c->d.xb_off = qi;
  CKS(up(&qi, ent)); c->d.xb_ent = qi;
  CKS(up(&qd, xM)); c->d.xl_M = qd;
  CKS(up(&qd, c->fil_len)); c->d.fil_L = qd;
  CKS(dalloc(c, &c->d.bml, (size_t)c->nb));
  CKS(dalloc(c, &c->d.ftl, (size_t)c->nf));
  // Anchor records: zero force and torque on the attach bond.
  std::vector<double> rec(16 * (size_t)n, 0.0);
  for (int A = 0; A < 2 * n; ++A) rec[8 * (size_t)A + 6] = (double)bond[A];
  CKS(up(&qd, rec)); c->d.xl_c = qd;
  CKS(dalloc(c, &c->d.xl_F, 4 * (size_t)n));
  CK(cudaMemsetAsync(c->d.xl_F, 0, sizeof(double) * 4 * (size_t)n, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->k.xk = k_spring;
  c->k.xkc = k_spring_compress;
  c->k.xrest = rest_length;
  c->d.nx = n;
  drop_graph(c);  // kernel parameters changed
  return SC_OK;
}

sc_status sc_get_crosslink_forces(sc_ctx *c, double *f) {
  if (!c || !c->loaded || !f) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  if (c->d.nx == 0) return SC_OK;
  std::vector<double> tmp(4 * (size_t)c->d.nx);
  CK(cudaMemcpyAsync(tmp.data(), c->d.xl_F, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int x = 0; x < c->d.nx; ++x)
    for (int i = 0; i < 3; ++i) f[3 * (size_t)x + i] = tmp[4 * (size_t)x + i];
  return SC_OK;
}

sc_status sc_get_bond_geometry(sc_ctx *c, double *pos, double *spos, double *u,
                               double *len) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  // FP64 geometry of the current positions (buffer 0 of the FP64 records is
  // scratch in mixed precision; in FP64 the read buffer already holds it).
  int buf = c->prec == 0 ? c->rbuf : 0;
  if (c->prec != 0) sc::launch_init_geometry(c->k, c->d, 0, 0, c->st, false);
  std::vector<sc::BondGeomF64> g(c->nb);
  CK(cudaMemcpyAsync(g.data(), c->d.g64[buf], sizeof(sc::BondGeomF64) * c->nb,
                     cudaMemcpyDeviceToHost, c->st));
  std::vector<double> r(3 * (size_t)c->ns);
  CK(cudaStreamSynchronize(c->st));
  CKS(copy_soa3(c, c->d.r, c->ns, r.data()));
  for (int b = 0; b < c->nb; ++b) {
    const int f = c->bond_fil[b];
    const double *r1 = &r[3 * (size_t)(b + f)];
    if (pos) {
      double o[3] = {0, 0, 0};
      for (int i = 0; i < c->nd; ++i) o[i] = r1[3 + i] - r1[i];
      for (int i = 0; i < 3; ++i) pos[3 * (size_t)b + i] = i < c->nd ? r1[i] + 0.5 * o[i] : 0.0;
    }
    for (int i = 0; i < 3; ++i) {
      if (spos) spos[3 * (size_t)b + i] = g[b].s[i];
      if (u) u[3 * (size_t)b + i] = g[b].u[i];
    }
    if (len) len[b] = g[b].len;
  }
  return SC_OK;
}

sc_status sc_set_fast_integrator(sc_ctx *c, int on) {
  if (!c) return SC_ERR_INVALID_ARG;
  if (c->fast != (on != 0)) drop_graph(c);
  c->fast = on != 0;
  return SC_OK;
}

sc_status sc_set_capture(sc_ctx *c, int on) {
  if (!c) return SC_ERR_INVALID_ARG;
  if (c->capture != (on ? 1 : 0)) drop_graph(c);
  c->capture = on ? 1 : 0;
  return SC_OK;
}

sc_status sc_get_site_forces(sc_ctx *c, double *f) {
  if (!c || !c->loaded || !f) return SC_ERR_INVALID_ARG;
  return copy_soa3(c, c->d.cap_F, c->ns, f);
}

sc_status sc_get_tensions(sc_ctx *c, double *t) {
  if (!c || !c->loaded || !t) return SC_ERR_INVALID_ARG;
  CK(cudaMemcpyAsync(t, c->d.cap_T, sizeof(double) * c->nb, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_get_filament_state(sc_ctx *c, int *sw, int *nn) {
  if (!c || !c->loaded || !sw || !nn) return SC_ERR_INVALID_ARG;
  CK(cudaMemcpyAsync(sw, c->d.f_switch, sizeof(int) * c->nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(nn, c->d.f_nnorm, sizeof(int) * c->nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_get_dr_tot(sc_ctx *c, double *dr) {
  if (!c || !c->loaded || !dr) return SC_ERR_INVALID_ARG;
  CK(cudaMemcpyAsync(dr, c->d.dt, sizeof(double) * c->ns, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_get_pairs(sc_ctx *c, int32_t *pairs, int64_t cap, int64_t *n_pairs) {
  if (!c || !c->loaded || !n_pairs) return SC_ERR_INVALID_ARG;
  CKS(sync_pair_count(c));
  *n_pairs = c->np;
  long long out = 0;
  for (size_t r = 0; r < c->reps.size() && pairs && out < cap; ++r) {
    const long long m = std::min<long long>(std::min(c->np_rep[r], c->reps[r].pcap), cap - out);
    if (m <= 0) continue;
    std::vector<int> a(m), b(m);
    const int p0 = c->reps[r].p0;
    CK(cudaMemcpyAsync(a.data(), c->d.pa + p0, sizeof(int) * m, cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(b.data(), c->d.pb + p0, sizeof(int) * m, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (long long i = 0; i < m; ++i, ++out) {
      pairs[2 * out] = a[i];
      pairs[2 * out + 1] = b[i];
    }
  }
  return SC_OK;
}

// ---- thermo ----------------------------------------------------------------

sc_status sc_set_thermo(sc_ctx *c, int n_thermo) {
  if (!c || !c->loaded || n_thermo < 0) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  DevState &d = c->d;
  const int nrep = d.nrep;
  if (c->k.thermo) CKS(thermo_pull(c));
  if (n_thermo == 0) {
    for (FILE *f : c->th_files)
      if (f) std::fclose(f);
    c->th_files.clear();
    c->k.thermo = 0;
    d.th_n = 0;
    drop_graph(c);
    return SC_OK;
  }
  if (!c->desc.interaction_flag)
    return fail(c, SC_ERR_INVALID_ARG, "thermo needs pair interactions");
  if (!d.th_part) {
    CKS(dalloc(c, &d.th_part, (size_t)nrep * kThermoMaxBlocks * 9));
    CKS(dalloc(c, &d.th_ticket, nrep));
    CKS(dalloc(c, &d.th_acc, 9 * (size_t)nrep));
    CKS(dalloc(c, &d.th_istep, nrep));
    CKS(dalloc(c, &d.th_nrec, nrep));
    d.th_cap = 256;
    CKS(dalloc(c, &d.th_rec, 12 * (size_t)nrep * d.th_cap));
  }
  if (!(c->prec == 0 ? (void *)d.pv64 : (void *)d.pv32)) {
    // Per-pair virial records, zeroed (a pair not evaluated since the list
    // was built has stress and potential 0).
    const size_t n = (size_t)(c->pcap > 0 ? c->pcap : 1);
    if (c->prec == 0) {
      CKS(dalloc(c, &d.pv64, 4 * n));
      CK(cudaMemsetAsync(d.pv64, 0, sizeof(double) * 4 * n, c->st));
    } else {
      CKS(dalloc(c, &d.pv32, 4 * n));
      CK(cudaMemsetAsync(d.pv32, 0, sizeof(float) * 4 * n, c->st));
    }
  }
  std::vector<long long> ist(nrep, c->i_step);
  CK(cudaMemsetAsync(d.th_ticket, 0, sizeof(unsigned) * nrep, c->st));
  CK(cudaMemsetAsync(d.th_acc, 0, sizeof(double) * 9 * nrep, c->st));
  CK(cudaMemsetAsync(d.th_nrec, 0, sizeof(long long) * nrep, c->st));
  CK(cudaMemcpyAsync(d.th_istep, ist.data(), sizeof(long long) * nrep, cudaMemcpyHostToDevice,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  c->th_i0 = c->i_step;
  c->th_pulled = 0;
  d.th_n = n_thermo;
  c->k.thermo = 1;
  drop_graph(c);
  return SC_OK;
}

sc_status sc_thermo_open(sc_ctx *c, const char *run_name, int n_steps) {
  if (!c || !c->loaded || !run_name || n_steps < 0) return SC_ERR_INVALID_ARG;
  if (!c->k.thermo) return fail(c, SC_ERR_INVALID_ARG, "thermo is off");
  if (!c->th_files.empty()) return fail(c, SC_ERR_INVALID_ARG, "thermo file already open");
  CK(cudaSetDevice(c->desc.device));
  CKS(thermo_pull(c));  // records taken before the file opened stay out of it
  const size_t nrep = c->reps.size();
  c->th_files.assign(nrep, nullptr);
  for (size_t r = 0; r < nrep; ++r) {
    std::string name = run_name;
    if (nrep > 1) {
      char sfx[32];
      std::snprintf(sfx, sizeof(sfx), "_r%03zu", r);
      name += sfx;
    }
    name += ".thermo";
    FILE *f = std::fopen(name.c_str(), "wb");
    if (!f) return fail(c, SC_ERR_INVALID_ARG, "cannot open %s", name.c_str());
    // OutputManager::InitThermo (include/simcore/output_manager.hpp:156-168)
    put(f, (int32_t)n_steps);
    put(f, (int32_t)c->d.th_n);
    put(f, c->desc.delta);
    put(f, (int32_t)c->nd);
    c->th_files[r] = f;
  }
  return SC_OK;
}

sc_status sc_get_thermo(sc_ctx *c, int max_records, int *n_records, int64_t *i_step,
                        double *tensor, double *pressure, double *volume) {
  if (!c || !c->loaded || max_records < 0 || !n_records) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  CKS(thermo_pull(c));
  const size_t nrep = c->reps.size(), per = 12 * nrep;
  const size_t n = std::min(c->th_host.size() / per, (size_t)max_records);
  for (size_t k = 0; k < n; ++k)
    for (size_t r = 0; r < nrep; ++r) {
      const double *q = c->th_host.data() + per * k + 12 * r;
      if (i_step && r == 0) i_step[k] = (int64_t)q[0];
      if (tensor) std::memcpy(tensor + 9 * (k * nrep + r), q + 1, sizeof(double) * 9);
      if (pressure) pressure[k * nrep + r] = q[10];
      if (volume) volume[k * nrep + r] = q[11];
    }
  c->th_host.erase(c->th_host.begin(), c->th_host.begin() + per * n);
  *n_records = (int)n;
  return SC_OK;
}

sc_status sc_get_potential_energy(sc_ctx *c, double *pote) {
  if (!c || !c->loaded || !pote) return SC_ERR_INVALID_ARG;
  if (!c->k.thermo) return fail(c, SC_ERR_INVALID_ARG, "potential energies need thermo on");
  CK(cudaSetDevice(c->desc.device));
  c->launches += sc::launch_potential(c->d, c->prec, c->stage, c->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(pote, c->stage, sizeof(double) * c->nf, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_set_exact_near_parallel(sc_ctx *c, int on) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  if (c->prec == 0 || c->npx == (on != 0)) return SC_OK;
  CK(cudaSetDevice(c->desc.device));
  c->npx = on != 0;
  CK(cudaStreamSynchronize(c->st));
  drop_graph(c);
  return SC_OK;
}

sc_status sc_set_fused_pairs(sc_ctx *c, int on) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  if (c->fuse_pairs == (on != 0)) return SC_OK;
  CK(cudaSetDevice(c->desc.device));
  CK(cudaStreamSynchronize(c->st));
  c->fuse_pairs = on != 0;
  drop_graph(c);
  return SC_OK;
}

sc_status sc_get_replica_counters(sc_ctx *c, int64_t *n_rebuilds, int64_t *n_pairs) {
  if (!c || !c->loaded) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  const int nrep = c->d.nrep;
  CKS(sync_pair_count(c));
  if (n_rebuilds) {
    std::vector<long long> v(nrep);
    CK(cudaMemcpyAsync(v.data(), c->d.rep_rebuilds, sizeof(long long) * nrep,
                       cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int r = 0; r < nrep; ++r) n_rebuilds[r] = v[r];
  }
  if (n_pairs)
    for (int r = 0; r < nrep; ++r) n_pairs[r] = std::min(c->np_rep[r], c->reps[r].pcap);
  return SC_OK;
}

sc_status sc_get_bond_cells(sc_ctx *c, int32_t *xyz) {
  if (!c || !c->loaded || !xyz) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  c->launches += sc::launch_bond_cells(c->k, c->d, c->cells_xyz, c->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(xyz, c->cells_xyz, sizeof(int) * 3 * (size_t)c->nb,
                     cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return SC_OK;
}

sc_status sc_get_counters(sc_ctx *c, sc_counters *o) {
  if (!c || !o) return SC_ERR_INVALID_ARG;
  std::memset(o, 0, sizeof(*o));
  if (c->loaded) {
    long long nr = 0;
    CK(cudaMemcpyAsync(&nr, c->d.n_rebuilds, sizeof(long long), cudaMemcpyDeviceToHost, c->st));
    CKS(sync_pair_count(c));
    c->n_rebuilds = nr;
  }
  o->i_step = c->i_step;
  o->n_rebuilds = c->n_rebuilds;
  o->n_pairs = c->np;
  o->pair_capacity = c->pcap;
  o->n_filaments = c->nf;
  o->n_sites = c->ns;
  o->n_bonds = c->nb;
  if (!c->reps.empty()) {  // system 0's cell grid
    o->n_cells_1d = c->reps[0].n1d;
    o->cell_length = c->reps[0].h[0] / c->reps[0].n1d;
    o->dr_update = c->reps[0].dr_update;
  }
  o->n_replicas = (int32_t)c->reps.size();
  o->n_list_regrowths = c->n_regrowths;
  o->kernel_launches = c->launches;
  return SC_OK;
}

void *sc_get_stream(sc_ctx *c) { return c ? (void *)c->st : nullptr; }

sc_status sc_set_kernel_timing(sc_ctx *c, int on) {
  if (!c) return SC_ERR_INVALID_ARG;
  if (on && !c->ev0) {
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
  }
  c->timing = on != 0;
  c->timed_ms = 0.0;
  c->timed_launches = 0;
  return SC_OK;
}

sc_status sc_get_graph_time(sc_ctx *c, double *ms) {
  if (!c || !ms) return SC_ERR_INVALID_ARG;
  *ms = c->graph_ms;
  return SC_OK;
}

sc_status sc_get_kernel_timing(sc_ctx *c, double *total_ms, int64_t *launches) {
  if (!c || !total_ms || !launches) return SC_ERR_INVALID_ARG;
  *total_ms = c->timed_ms;
  *launches = c->timed_launches;
  return SC_OK;
}

}  // extern "C"
