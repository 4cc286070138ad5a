// Pair forces without any device allocation (sc_pair_forces_noalloc).
//
// Some callers cannot call cudaMalloc: a host application whose device
// memory is owned by its own pool or caching allocator, which must not be
// grown or fragmented behind its back, or one that runs under a fixed
// device-memory budget reserved at start-up (a solver embedded in a larger
// simulation code, a real-time controller).  This entry point serves them:
// it evaluates the WCA bond forces and torques of one configuration held in
// the caller's device buffers, using only a fixed scratch area that is part
// of the library image.  It reads one size back and synchronises the
// stream, so it is called outside stream capture.
//
// The scratch is one file-scope __device__ array (g_noalloc_scratch below,
// SC_NOALLOC_SCRATCH_BYTES = 8.5 MiB).  Every GPU that loads the library
// holds it until the process exits.  All calls on a device share it and it
// keeps the last call's contents, so every call clears what must start at
// zero; calls whose GPU work overlaps (several host threads, or several
// streams) race on it and must be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "sc_common.cuh"
#include "sc_kernels.h"
#include "sc_launch.h"
#include "simcore_gpu.h"

namespace {

using sc::DevState;
using sc::SysConst;

// Limits of the static scratch.
constexpr int kMaxBonds = SC_NOALLOC_MAX_BONDS;
constexpr int kMaxFilaments = SC_NOALLOC_MAX_BONDS;
constexpr int kMaxSites = kMaxBonds + kMaxFilaments;
constexpr int kMaxCells = SC_NOALLOC_MAX_CELLS;
constexpr int kMaxPairs = SC_NOALLOC_MAX_PAIRS;

// Byte layout of the scratch area: each region 256-byte aligned.
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
  size_t r, key, cell_count, cell_start, sorted, pair_count, pair_off, deg, deg_off, e_off,
      e_cnt, scan_tmp, bond_fil, ub, g64, pa, pb, pos1, pos2, pf, cf, e_ent, bF, bT, status,
      counters, rep, sys, total;
};

constexpr int kScanTmp = (kMaxCells > kMaxBonds ? kMaxCells : kMaxBonds) / 2048 + 2;

constexpr Layout make_layout() {
  Layout L{};
  size_t o = 0;
  L.r = o;          o = align256(o + sizeof(double) * 3 * kMaxSites);
  L.key = o;        o = align256(o + sizeof(int) * kMaxBonds);
  L.cell_count = o; o = align256(o + sizeof(int) * kMaxCells);
  L.cell_start = o; o = align256(o + sizeof(int) * (kMaxCells + 1));
  L.sorted = o;     o = align256(o + sizeof(int) * kMaxBonds);
  L.pair_count = o; o = align256(o + sizeof(int) * kMaxBonds);
  L.pair_off = o;   o = align256(o + sizeof(int) * (kMaxBonds + 1));
  L.deg = o;        o = align256(o + sizeof(int) * kMaxBonds);
  L.deg_off = o;    o = align256(o + sizeof(int) * (kMaxBonds + 1));
  L.e_off = o;      o = align256(o + sizeof(int) * kMaxBonds);
  L.e_cnt = o;      o = align256(o + sizeof(int) * kMaxBonds);
  L.scan_tmp = o;   o = align256(o + sizeof(int) * kScanTmp);
  L.bond_fil = o;   o = align256(o + sizeof(int) * kMaxBonds);
  L.ub = o;         o = align256(o + sizeof(double) * 3 * kMaxBonds);
  L.g64 = o;        o = align256(o + sizeof(sc::BondGeomF64) * kMaxBonds);
  L.pa = o;         o = align256(o + sizeof(int) * kMaxPairs);
  L.pb = o;         o = align256(o + sizeof(int) * kMaxPairs);
  L.pos1 = o;       o = align256(o + sizeof(int) * kMaxPairs);
  L.pos2 = o;       o = align256(o + sizeof(int) * kMaxPairs);
  L.pf = o;         o = align256(o + sizeof(double) * 4 * kMaxPairs);
  L.cf = o;         o = align256(o + sizeof(double) * 16 * kMaxPairs);
  L.e_ent = o;      o = align256(o + sizeof(int) * 2 * kMaxPairs);
  L.bF = o;         o = align256(o + sizeof(double) * 3 * kMaxBonds);
  L.bT = o;         o = align256(o + sizeof(double) * 3 * kMaxBonds);
  L.status = o;     o = align256(o + sizeof(unsigned));
  L.counters = o;   o = align256(o + sizeof(unsigned long long) * 4);
  L.rep = o;        o = align256(o + sizeof(sc::ReplicaConst));
  L.sys = o;        o = align256(o + sizeof(int) * 4);
  L.total = o;
  return L;
}

constexpr Layout kLayout = make_layout();
static_assert(kLayout.total == SC_NOALLOC_SCRATCH_BYTES,
              "SC_NOALLOC_SCRATCH_BYTES must state the scratch size");

}  // namespace

// The scratch area itself (device memory of the library image).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kLayout.total];

namespace {

// Device address of g_noalloc_scratch, looked up with cudaGetSymbolAddress
// once per device and CUDA context (with that device current) and cached.
// In host code the symbol name is only a host-side stand-in, never a device
// address.  The cache is keyed on the context's unique id (cuCtxGetId, never
// reused within a process), so a context created after cudaDeviceReset, or
// another context made current on the same device, gets its own lookup.  The
// first call on a device (and after a reset) does the lookup, which may load
// the library's device code: make that call before any stream capture.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mtx;
struct ScratchAddr {
  unsigned long long ctx_id;  // 0: not looked up
  unsigned char *ptr;
};
ScratchAddr g_addr[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// Unique id of the calling thread's current context; false when there is
// none yet (the runtime makes its primary context current on first use).
bool current_context_id(unsigned long long *id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {  // (under g_addr_mtx)
    looked_up = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)f;
    cudaGetLastError();
  }
  if (!get_current || !get_id) return false;
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return get_id(ctx, id) == CUDA_SUCCESS && *id != 0;
}

sc_status scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return SC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_addr_mtx);
  unsigned long long id = 0;
  const bool have_id = current_context_id(&id);
  ScratchAddr &a = g_addr[dev];
  if (!have_id || a.ctx_id != id || !a.ptr) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return SC_ERR_CUDA;
    }
    // The lookup made the device's primary context current if none was.
    unsigned long long after = 0;
    a.ptr = (unsigned char *)p;
    a.ctx_id = current_context_id(&after) ? after : 0;
  }
  *out = a.ptr;
  return SC_OK;
}

// The reference's symmetric inverses (src/linear_algebra.cpp:40-64).
void inv2(const double *a, double *b) {
  double inv_det = a[0] * a[3] - a[1] * a[1];
  inv_det = 1.0 / inv_det;
  b[0] = a[3] * inv_det;
  b[3] = a[0] * inv_det;
  b[2] = b[1] = -a[1] * inv_det;
}

void inv3(const double *a, double *b) {
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

// AoS caller positions -> SoA scratch; bond -> filament map from offsets.
// The offsets must rise from 0 by at least 2 sites a filament (the last one,
// ns, is checked on the host); then filament i's bonds s0 - i .. s1 - i - 2
// lie in [0, nb).  Offsets that break this set ST_BAD_INPUT, and every write
// stays inside the bond range whatever they hold.
__global__ void k_noalloc_unpack(int nf, int ns, const int32_t *site_off,
                                 const double *xyz, int n_dim, DevState d, int *bond_fil) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ns) {
    for (int c = 0; c < 3; ++c) d.r[c][i] = c < n_dim ? xyz[3 * (size_t)i + c] : 0.0;
  }
  if (i < nf) {
    const int s0 = site_off[i], s1 = site_off[i + 1];
    if ((i == 0 && s0 != 0) || s0 < 0 || s1 > ns || s1 - s0 < 2) atomicOr(d.status, sc::ST_BAD_INPUT);
    const int b0 = max(s0 - i, 0), b1 = min(s1 - i - 1, d.nb);
    for (int b = b0; b < b1; ++b) bond_fil[b] = i;
  }
}

// Bond accumulators (SoA scratch) -> caller's AoS outputs.
__global__ void k_noalloc_pack(int nb, DevState d, double *f, double *t) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  for (int c = 0; c < 3; ++c) {
    f[3 * (size_t)b + c] = d.bF[c][b];
    t[3 * (size_t)b + c] = d.bT[c][b];
  }
}

#define NA_CK(call)                                      \
  do {                                                   \
    if ((call) != cudaSuccess) {                         \
      cudaGetLastError();                                \
      return SC_ERR_CUDA;                                \
    }                                                    \
  } while (0)

}  // namespace

extern "C" sc_status sc_pair_forces_noalloc(const sc_system_desc *desc,
                                            const sc_filament_params *species,
                                            int n_filaments, const int32_t *d_site_offsets,
                                            const double *d_site_xyz, double *d_bond_force,
                                            double *d_bond_torque, void *stream) {
  if (!desc || !species || !d_site_offsets || !d_site_xyz || !d_bond_force ||
      !d_bond_torque)
    return SC_ERR_INVALID_ARG;
  if (desc->n_dim != 2 && desc->n_dim != 3) return SC_ERR_INVALID_ARG;
  if (!(desc->system_radius > 0) || !std::isfinite(desc->system_radius) ||
      !(desc->wca_sig > 0) || !std::isfinite(desc->wca_sig))
    return SC_ERR_INVALID_ARG;
  if (!(species->min_bond_length > 0) || !std::isfinite(species->min_bond_length) ||
      !(species->diameter > 0) || !std::isfinite(species->diameter))
    return SC_ERR_INVALID_ARG;
  if (n_filaments <= 0 || n_filaments > kMaxFilaments) return SC_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  unsigned char *base = nullptr;
  sc_status s = scratch_address(dev, &base);
  if (s != SC_OK) return s;

  // Sizes: the last site offset (one 4-byte read of the caller's array).
  int32_t ns32 = 0;
  NA_CK(cudaMemcpyAsync(&ns32, d_site_offsets + n_filaments, sizeof(int32_t),
                        cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  const int ns = ns32, nb = ns32 - n_filaments;
  if (ns <= 0 || nb <= 0 || ns > kMaxSites || nb > kMaxBonds) return SC_ERR_INVALID_ARG;

  // System constants, as sc_create and sc_add_filaments derive them.
  SysConst k;
  std::memset(&k, 0, sizeof(k));
  const int nd = desc->n_dim;
  k.n_dim = nd;
  sc::ReplicaConst R;
  std::memset(&R, 0, sizeof(R));
  const double hh = 2.0 * desc->system_radius;
  for (int a = 0; a < nd; ++a)
    for (int b = 0; b < nd; ++b) R.h[a * nd + b] = (a == b ? 1 : 0) * hh;
  R.h[nd * nd - 1] = hh;
  if (nd == 2) inv2(R.h, R.hinv);
  else inv3(R.h, R.hinv);
  for (int i = 0; i < 9; ++i) R.hf[i] = (float)R.h[i];
  k.delta = desc->delta;
  const double rcut = std::pow(2.0, 1.0 / 6.0) * desc->wca_sig;
  k.rcut2 = rcut * rcut;
  k.c12 = 4.0 * desc->wca_eps * std::pow(desc->wca_sig, 12.0);
  k.c6 = 4.0 * desc->wca_eps * std::pow(desc->wca_sig, 6.0);
  k.fcut = desc->f_cutoff;
  k.like_like = desc->like_like_interactions ? 1 : 0;
  {
    double min_len = -1, spec_length = 1.5 * species->min_bond_length;
    if (species->diameter > spec_length) spec_length = species->diameter;
    if (spec_length > min_len) min_len = spec_length;
    if (0.0 > min_len) min_len = 0.0;
    if (std::sqrt(k.rcut2) > min_len) min_len = std::sqrt(k.rcut2);
    // The cell count is bounded while it is still a double: at most
    // floor(cbrt(SC_NOALLOC_MAX_CELLS)) = 50 cells a side in 3D,
    // floor(sqrt(SC_NOALLOC_MAX_CELLS)) = 362 in 2D, so no integer below
    // can overflow or wrap.
    const double per_side = 2 * desc->system_radius / min_len;
    const double max_side =
        std::floor(nd == 3 ? std::cbrt((double)kMaxCells) : std::sqrt((double)kMaxCells));
    if (!std::isfinite(per_side) || !(per_side < max_side + 1.0)) return SC_ERR_INVALID_ARG;
    int n1d = (int)std::floor(per_side);
    if (n1d <= 3) n1d = 3;
    const long long ncell = (long long)n1d * n1d * (nd == 3 ? n1d : 1);
    if (ncell > kMaxCells) return SC_ERR_INVALID_ARG;
    R.n1d = n1d;
    R.third = nd == 3 ? n1d : 1;
    R.n_cells = (int)ncell;
    k.n_cells = (int)ncell;
  }
  R.seed = desc->seed;
  R.nf = n_filaments;
  R.ns = ns;
  R.nb = nb;
  R.pcap = kMaxPairs;

  // Device views into the scratch area.
  const Layout &L = kLayout;
  DevState d;
  std::memset(&d, 0, sizeof(d));
  d.nf = n_filaments;
  d.ns = ns;
  d.nb = nb;
  double *r = (double *)(base + L.r);
  for (int c = 0; c < 3; ++c) d.r[c] = r + (size_t)c * kMaxSites;
  d.bond_fil = (const int *)(base + L.bond_fil);
  double *ub = (double *)(base + L.ub);
  for (int c = 0; c < 3; ++c) d.ub[c] = ub + (size_t)c * kMaxBonds;
  d.g64[0] = d.g64[1] = (sc::BondGeomF64 *)(base + L.g64);
  d.pa = (int *)(base + L.pa);
  d.pb = (int *)(base + L.pb);
  d.pos1 = (int *)(base + L.pos1);
  d.pos2 = (int *)(base + L.pos2);
  d.pf64 = (double *)(base + L.pf);
  d.cf64 = (double *)(base + L.cf);
  d.e_off = (int *)(base + L.e_off);
  d.e_cnt = (int *)(base + L.e_cnt);
  d.e_ent = (int *)(base + L.e_ent);
  d.nrep = 1;
  d.rep = (const sc::ReplicaConst *)(base + L.rep);
  d.bond_rep = nullptr;
  int *sys = (int *)(base + L.sys);
  d.due = sys;
  d.np_rep = sys + 1;
  d.pcap_total = kMaxPairs;
  double *bF = (double *)(base + L.bF), *bT = (double *)(base + L.bT);
  for (int c = 0; c < 3; ++c) {
    d.bF[c] = bF + (size_t)c * kMaxBonds;
    d.bT[c] = bT + (size_t)c * kMaxBonds;
  }
  d.status = (unsigned *)(base + L.status);
  unsigned long long *ctr = (unsigned long long *)(base + L.counters);
  d.dr_max_bits = ctr;
  d.mcount = ctr + 1;
  d.n_rebuilds = (long long *)(ctr + 2);
  d.rep_rebuilds = (long long *)(ctr + 3);
  int *key = (int *)(base + L.key), *cell_count = (int *)(base + L.cell_count);
  int *cell_start = (int *)(base + L.cell_start), *sorted = (int *)(base + L.sorted);
  int *pair_count = (int *)(base + L.pair_count), *pair_off = (int *)(base + L.pair_off);
  int *deg = (int *)(base + L.deg), *scan_tmp = (int *)(base + L.scan_tmp);
  int *deg_off = (int *)(base + L.deg_off);

  // What must start at zero: the cell and degree counters (the previous
  // call may have stopped early), the status word and the counters.
  NA_CK(cudaMemsetAsync(cell_count, 0, sizeof(int) * (size_t)k.n_cells, st));
  NA_CK(cudaMemsetAsync(deg, 0, sizeof(int) * (size_t)nb, st));
  NA_CK(cudaMemsetAsync(d.status, 0, sizeof(unsigned), st));
  NA_CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * 4, st));
  // The system table and its rebuild flag (a pageable copy: staged before
  // the call returns).
  const int sys_init[4] = {1, 0, 0, 0};
  NA_CK(cudaMemcpyAsync(base + L.rep, &R, sizeof(R), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(sys, sys_init, sizeof(sys_init), cudaMemcpyHostToDevice, st));

  const int grid = (ns > n_filaments ? ns : n_filaments) / 256 + 1;
  k_noalloc_unpack<<<grid, 256, 0, st>>>(n_filaments, ns, d_site_offsets, d_site_xyz, nd, d,
                                         (int *)(base + L.bond_fil));
  sc::launch_init_geometry(k, d, 0, 0, st);
  // Pair list of a rebuild (InteractionManager::UpdatePairInteractions) and
  // one evaluation with fresh Interaction records, as the first Interact
  // after the reference's insertion computes.
  sc::launch_bin_count(k, d, key, cell_count, st);
  sc::launch_exclusive_scan(cell_count, cell_start, k.n_cells, scan_tmp, st);
  sc::launch_bin_scatter(d, key, cell_start, cell_count, sorted, st);
  sc::launch_cell_sort_count(k, d, key, sorted, cell_start, pair_count, st);
  sc::launch_exclusive_scan(pair_count, pair_off, nb, scan_tmp, st);
  sc::launch_pair_emit(k, d, key, sorted, cell_start, pair_off, deg, 0, st);
  sc::launch_exclusive_scan(deg, deg_off, nb, scan_tmp, st);
  sc::launch_csr(d, deg, deg_off, st);
  {
    // The pair kernel reads its slot indices before it waits on the kernel
    // before it, which here writes them: launched without the overlap.
    sc::PdlOff off;
    sc::launch_pairs(k, d, 0, 0, kMaxPairs, st);
  }
  sc::launch_bond_sum(k, d, 0, st);
  k_noalloc_pack<<<nb / 256 + 1, 256, 0, st>>>(nb, d, d_bond_force, d_bond_torque);
  NA_CK(cudaGetLastError());

  unsigned status = 0;
  NA_CK(cudaMemcpyAsync(&status, d.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  if (status & sc::ST_BAD_INPUT) return SC_ERR_INVALID_ARG;
  if (status & sc::ST_LIST_OVERFLOW) return SC_ERR_LIST_OVERFLOW;
  if (status) return SC_ERR_NAN;
  return SC_OK;
}
