// Filament analyses on the device: end-to-end distance and joint-angle
// statistics, centre-of-mass diffusion, orientational order.
#include "sc_context.h"

using namespace scapi;

extern "C" {

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

}  // extern "C"
