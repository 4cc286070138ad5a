// Checkpoint / restore of a context and its noise keys.
#include "sc_context.h"

using namespace scapi;

extern "C" {

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

}  // extern "C"
