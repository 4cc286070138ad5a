// Host side of the C ABI (include/simcore_gpu.h), shared by its
// implementation files: the context (sc_ctx), error and allocation helpers,
// and the orchestration every entry point uses -- pair storage, rebuilds,
// the reference step, thermo records.
//
//   sc_api.cu        context, systems and filaments, step, state access
//   sc_graph.cu      the captured step loop (sc_step_graph)
//   sc_autotune.cu   integrator layout and its autotuner
//   sc_state.cu      checkpoint / restore, noise keys
//   sc_output.cu     reference-format spec/posit files, thermo records
//   sc_analysis.cu   filament analyses, diffusion, order parameters
//   sc_xlinks.cu     static crosslinks
#pragma once

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
  sc::RebuildBufs rb = {};         // the rebuild's sort, cell ranges and offsets
  int *cells_xyz = nullptr;
  double *stage = nullptr;         // interleaved host-transfer staging, 3 * max(ns, nb)
  long long np = 0, pcap = 0;      // pairs and slots of all systems

  // integrator blocks
  int nblocks = 0, C = 128;
  int warp_sites = 32;             // longest filament for the warp-synchronous kernel
  int block_sites = 0;             // sites per block of the block kernel (0: 128, 256 or 512)
  int pair_block = 256;            // threads per block of the pair kernel (128 or 256)

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
    long long rebuilds[2];  // rebuild counter before and after a graph launch
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

namespace scapi {

// Error of the call: the message is kept in the context (sc_last_error).
sc_status fail(sc_ctx *c, sc_status code, const char *fmt, ...);

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

// The pair-list arrays of a context (DevState's pair members).
struct PairStore {
  int *pa = nullptr, *pb = nullptr, *pos1 = nullptr, *pos2 = nullptr, *e_ent = nullptr;
  double *pf64 = nullptr, *cf64 = nullptr, *pv64 = nullptr;
  float *pf32 = nullptr, *cf32 = nullptr, *pv32 = nullptr;
  int4 *cand = nullptr;  // the rebuild's candidate pairs, one per slot
  long long cap = 0;     // slots
};

void dfree(sc_ctx *c, void *p);
// The reference's symmetric inverses (src/linear_algebra.cpp:40-64).
void invert_sym_2d(const double *a, double *b);
void invert_sym_3d(const double *a, double *b);
// Filament::InitFilamentLength for static lengths (src/filament.cpp:104-147).
void filament_length(const sc_filament_params &p, double *length, int *n_bonds);
// Status word -> sc_status; readback copies it (and the displacement maxima).
sc_status check_status(sc_ctx *c);
sc_status readback(sc_ctx *c);
void drop_graph(sc_ctx *c);
sc_status upload_reps(sc_ctx *c);
// Pair storage (lists, slots, stored forces) of all systems.
void free_store(sc_ctx *c, PairStore &q);
PairStore current_store(const sc_ctx *c);
void install_store(sc_ctx *c, const PairStore &q);
sc_status alloc_store(sc_ctx *c, long long total, PairStore &q);
sc_status layout_pairs(sc_ctx *c, const std::vector<long long> &caps);
sc_status ensure_pair_capacity(sc_ctx *c, long long need);
sc_status sync_pair_count(sc_ctx *c);
// Pair-list rebuild (InteractionManager::UpdateInteractions).
void rebuild_enqueue(sc_ctx *c, bool first_in_graph = false);
sc_status rebuild(sc_ctx *c, bool allow_overflow = false);
sc_status grow_after_overflow(sc_ctx *c);
sc_status rebuild_all(sc_ctx *c);
sc_status maybe_rebuild(sc_ctx *c);
sc_status layout_integrator(sc_ctx *c);
void tether_if_due(sc_ctx *c);
// Thermo records on the device and their pull to the host.
long long thermo_total(const sc_ctx *c, long long i);
void thermo_write(sc_ctx *c, const double *rec);
sc_status thermo_pull(sc_ctx *c);
sc_status thermo_reserve(sc_ctx *c, long long n);
// The reference step (Interact + Integrate) and its pieces.
bool fused_pairs(const sc_ctx *c);
sc_status pair_stage(sc_ctx *c);
sc_status step_once(sc_ctx *c);
sc_status materialize_slots(sc_ctx *c);
sc_status output_flush(sc_ctx *c);

// Blocks of the thermo kernel per system.
constexpr int kThermoMaxBlocks = 296;  // two per SM

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

}  // namespace scapi
