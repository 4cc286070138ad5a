// sc_step_graph: the reference step loop captured as one CUDA graph, a WHILE
// loop of Brownian-dynamics steps with device-decided rebuilds.
#include "sc_context.h"

using namespace scapi;

extern "C" {

// Captures one graph: head (loop condition, first rebuild decision) ->
// WHILE (loop_count > 0) { IF(rebuild) -> midstep -> full step -> tail (next
// rebuild decision) }.  Built for the current geometry-buffer parity; every
// BD step returns the parity to where it started.
static sc_status build_graph(sc_ctx *c) {
  drop_graph(c);
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  const int interaction = c->desc.interaction_flag ? 1 : 0;
  cudaGraphConditionalHandle h_loop, h_if = 0;
  CK(cudaGraphConditionalHandleCreate(&h_loop, g, 0, 0));
  // The rebuild condition is set by the head and by every tail (the decision
  // for the step after), so it belongs to the outer graph, like the loop's.
  if (interaction) CK(cudaGraphConditionalHandleCreate(&h_if, g, 0, 0));
  // head kernel: sets the loop condition and decides the first rebuild
  CK(cudaStreamBeginCaptureToGraph(c->st, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  sc::launch_loop_head(c->d, h_loop, h_if, interaction, c->st);
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
  std::vector<cudaGraphNode_t> tail;
  if (interaction) {
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h_if;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    CK(cudaGraphAddNode(&inode, body, nullptr, 0, &ip));
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
        sc::launch_pairs(c->k, c->d, rb, c->prec, (int)(c->np + c->np / 8), c->st, c->npx,
                         c->pair_block);
      } else {
        sc::launch_pairs(c->k, c->d, rb, c->prec, (int)(c->np + c->np / 8), c->st, c->npx,
                         c->pair_block);
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
  sc::launch_loop_tail(c->d, c->desc.stoch_flag ? 1 : 0, h_loop, h_if, interaction, c->st);
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
      // Every readback goes to pinned memory: one synchronisation per launch.
      CK(cudaMemcpyAsync(&c->hb->rebuilds[0], c->d.n_rebuilds, sizeof(long long),
                         cudaMemcpyDeviceToHost, c->st));
      CK(cudaEventRecord(c->gev0, c->st));
      CK(cudaGraphLaunch(c->graph_exec, c->st));
      CK(cudaEventRecord(c->gev1, c->st));
      CK(cudaMemcpyAsync(&c->hb->rebuilds[1], c->d.n_rebuilds, sizeof(long long),
                         cudaMemcpyDeviceToHost, c->st));
      CK(cudaMemcpyAsync(c->h_loop, c->d.loop_count, sizeof(int), cudaMemcpyDeviceToHost, c->st));
      c->pairs_ready = false;
      CK(cudaMemcpyAsync(&c->hb->status, c->d.status, sizeof(unsigned), cudaMemcpyDeviceToHost,
                         c->st));
      if (c->d.nrep > 0)  // the displacement maxima too (readback's copies)
        CK(cudaMemcpyAsync(c->h_dr, c->d.dr_max_bits, sizeof(unsigned long long) * c->d.nrep,
                           cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      const unsigned st = c->hb->status;
      const long long nr0 = c->hb->rebuilds[0], nr1 = c->hb->rebuilds[1];
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
      // Kernels the graph ran: loop head, per BD step the two tether
      // kernels (mesh lambdas, anchor forces) + 2 steps + tail (the stopped
      // step's too), per rebuild the captured sequence.  A step is its pair
      // kernel (unless fused; near-parallel pairs are evaluated in place),
      // thermo and one or two integrator kernels.
      const int int_l = (c->d.n_wg > 0 ? 1 : 0) + (c->nblocks > 0 ? 1 : 0);
      const long long per_bd =
          c->desc.interaction_flag
              ? 1 + (c->d.nx ? 2 : 0) +
                    2 * ((c->graph_fused ? 0 : 1) + int_l + (c->k.thermo ? 1 : 0))
              : 1 + 2 * int_l;
      c->launches += 1 + (long long)(done + (overflow ? 1 : 0)) * per_bd +
                     (nr1 - nr0) * c->rebuild_kernels;
      bd -= done;
      if (!overflow) {
        CKS(check_status(c));  // status and maxima were read with the counters
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

}  // extern "C"
