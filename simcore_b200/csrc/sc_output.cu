// Reference-format output files and thermo records of a context.
#include "sc_context.h"

using namespace scapi;

extern "C" {

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

}  // extern "C"
