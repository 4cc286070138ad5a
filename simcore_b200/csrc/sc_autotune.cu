// Integrator work layout (warp kernel for short filaments, block size of the
// block kernel) and its autotuner, cached per shape.
#include "sc_context.h"

using namespace scapi;

extern "C" {

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

// Autotuner.  Candidate integrator layouts (warp kernel or not, block size)
// and pair-kernel block sizes (128 or 256 threads) are timed on the
// context's own state: the arrays they write are saved first and restored
// afterwards, so the simulation is unchanged.  The fastest choices are
// applied and, with a cache file, recorded per shape (device, precision,
// filament count and site range) so later contexts skip the timing.
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
  std::snprintf(key, sizeof(key), "v3|%s|sm%d|nd%d|prec%d|fast%d|fuse%d|nf%d|ns%d|n%d-%d",
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
      int w = -1, b = -1, pb = 256;
      while (std::fgets(line, sizeof(line), fp)) {
        char *tab = std::strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        int ww, bb, pp;
        float ms;
        if (std::strcmp(line, key) == 0 &&
            std::sscanf(tab + 1, "%d %d %f %d", &ww, &bb, &ms, &pp) == 4) {
          w = ww;
          b = bb;
          pb = pp == 128 ? 128 : 256;
        }
      }
      std::fclose(fp);
      if (w >= 0) {
        CKS(sc_set_integrator_layout(c, w, b));
        c->pair_block = pb;
        drop_graph(c);
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
  // The pair kernel's timing rewrites the per-bond slots, stored forces and
  // virial records from the current geometry: save those too.
  const bool tune_pairs = c->desc.interaction_flag && !fuse && c->np > 0;
  if (tune_pairs) {
    const size_t np = (size_t)c->d.pcap_total;
    if (c->prec == 0) {
      regions.push_back({c->d.cf64, sizeof(double) * 16 * np});
      if (!fuse) regions.push_back({c->d.pf64, sizeof(double) * 4 * np});
      if (c->d.pv64) regions.push_back({c->d.pv64, sizeof(double) * 4 * np});
    } else {
      regions.push_back({c->d.cf32, sizeof(float) * 16 * np});
      regions.push_back({c->d.pf32, sizeof(float) * 4 * np});
      if (c->d.pv32) regions.push_back({c->d.pv32, sizeof(float) * 4 * np});
    }
  }
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
  // Pair kernel: threads per block, timed on the current geometry.
  int best_pb = c->pair_block;
  if (st == SC_OK && tune_pairs) {
    float best_p = 1e30f;
    for (int pb : {256, 128}) {
      for (int it = 0; it < 2; ++it)
        sc::launch_pairs(c->k, c->d, c->rbuf, c->prec, (int)c->np, c->st, c->npx, pb);
      cudaEventRecord(e0, c->st);
      for (int it = 0; it < 8; ++it)
        sc::launch_pairs(c->k, c->d, c->rbuf, c->prec, (int)c->np, c->st, c->npx, pb);
      cudaEventRecord(e1, c->st);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = fail(c, SC_ERR_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_p) {
        best_p = ms;
        best_pb = pb;
      }
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
  c->pair_block = best_pb;
  CKS(layout_integrator(c));
  if (cache_path) {
    if (FILE *fp = std::fopen(cache_path, "a")) {
      std::fprintf(fp, "%s\t%d %d %.2f %d\n", key, best_lay.first, best_lay.second,
                   1000.0 * best / 8, best_pb);
      std::fclose(fp);
    }
  }
  return finish(best_lay.first, best_lay.second);
}

}  // extern "C"
