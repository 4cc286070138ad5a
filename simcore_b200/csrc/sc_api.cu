// C ABI of the B200 filament step (include/simcore_gpu.h): context, systems
// and filaments, the reference step, state access.  The shared helpers of
// sc_context.h are defined here.
#include "sc_context.h"

namespace scapi {

sc_status fail(sc_ctx *c, sc_status code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
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

void free_store(sc_ctx *c, PairStore &q) {
  for (void *p : {(void *)q.pa, (void *)q.pb, (void *)q.pos1, (void *)q.pos2, (void *)q.pf64,
                  (void *)q.pf32, (void *)q.cf64, (void *)q.cf32, (void *)q.e_ent,
                  (void *)q.pv64, (void *)q.pv32, (void *)q.cand})
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
  q.cand = c->rb.cand;
  q.cap = c->rb.cand_cap;
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
  c->rb.cand = q.cand;
  c->rb.cand_cap = (int)q.cap;
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
    CKS(dalloc(c, &q.cand, n));
    q.cap = (long long)n;
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
void rebuild_enqueue(sc_ctx *c, bool first_in_graph) {
  const long long before = c->launches;
  const DevState &d = c->d;
  if (c->desc.interaction_flag)
    c->launches += sc::launch_rebuild(c->k, d, c->rb, c->prec, c->st, first_in_graph);
  else
    c->launches += sc::launch_zero_dr(d, c->st);
  c->rebuild_kernels = c->launches - before;
}

// Host-driven rebuild of the systems flagged in d.due, then a check that
// every list fitted.  One system grows its segment and rebuilds again
// (binning is a pure function of the positions, so the second pass gives the
// same list); with several systems an overflow is reported, unless
// allow_overflow (the initial pass, whose caller sizes the segments).

sc_status rebuild(sc_ctx *c, bool allow_overflow) {
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
  d.blk_maxf = 0;
  for (int v : blk_nf) d.blk_maxf = std::max(d.blk_maxf, v);
  // Equal filaments in equal blocks covering every filament: the kernel
  // indexes them by arithmetic.
  d.blk_uni_n = d.blk_uni_fpb = 0;
  if (!blk_f0.empty() && n > 0) {
    const int nn = off[1] - off[0], fpb = blk_nf[0];
    bool uni = nn > 0 && fpb > 0 && (long long)blk_f0.size() == ((long long)n + fpb - 1) / fpb;
    for (int q = 0; uni && q <= n; ++q) uni = off[q] == (long long)q * nn;
    for (size_t i = 0; uni && i < blk_f0.size(); ++i) {
      const long long f0 = (long long)i * fpb;
      uni = blk_f0[i] == f0 && blk_nf[i] == std::min<long long>(fpb, n - f0) &&
            blk_site0[i] == f0 * nn && blk_ns[i] == (long long)blk_nf[i] * nn;
    }
    if (uni) {
      d.blk_uni_n = nn;
      d.blk_uni_fpb = fpb;
    }
  }
  d.n_wg = (int)wg_f0.size();
  sc::prepare_integrate(c->C);
  drop_graph(c);
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
    return sc::launch_pairs(c->k, c->d, c->rbuf, c->prec, (int)c->np, c->st, c->npx,
                            c->pair_block);
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
  c->launches += sc::launch_pairs(c->k, c->d, 1 - c->rbuf, c->prec, (int)c->np, c->st, false,
                                 c->pair_block);
  CK(cudaGetLastError());
  c->slots_stale = false;
  return SC_OK;
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

}  // namespace scapi

using namespace scapi;

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
  k.npx_s2 = 1e-5f;
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
      cells += (ncell + 31) & ~31ll;  // every system's cells start at a multiple of 32
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
  {
    sc::RebuildBufs &rb = c->rb;
    rb.n_groups = (int)(k.n_cells / 32);
    CKS(dalloc(c, &rb.key, nbi));
    CKS(dzero(&rb.gcount, (size_t)rb.n_groups));
    CKS(dalloc(c, &rb.gstart, (size_t)rb.n_groups + 1));
    CKS(dalloc(c, &rb.tmp, nbi));
    CKS(dalloc(c, &rb.skey, nbi));
    CKS(dalloc(c, &rb.sval, nbi));
    CKS(dzero(&rb.range, (size_t)k.n_cells));
    CKS(dzero(&rb.occ, (size_t)rb.n_groups));
    CKS(dzero(&rb.pair_count, 2 * (size_t)nbi));
    rb.deg = rb.pair_count + nbi;
    CKS(dzero(&rb.pair_off, 2 * (size_t)nbi + 1));
    rb.deg_off = rb.pair_off + nbi;
    CKS(dalloc(c, &rb.scan_tmp,
               (size_t)std::max(sc::scan_temp_ints(rb.n_groups), sc::scan_temp_ints(2 * nbi))));
    CKS(dzero(&rb.cand_n, 1));
    CKS(dalloc(c, &rb.cand_start, nbi));
  }
  CKS(dzero(&d.e_off, nbi));
  CKS(dzero(&d.e_cnt, nbi));
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

sc_status sc_set_near_parallel_threshold(sc_ctx *c, double s2) {
  if (!c || !c->loaded || !(s2 >= 0.0) || !(s2 <= 1.0)) return SC_ERR_INVALID_ARG;
  CK(cudaSetDevice(c->desc.device));
  CK(cudaStreamSynchronize(c->st));
  c->k.npx_s2 = (float)s2;
  drop_graph(c);
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
