// Static crosslinks (doubly bound tethers) of a context.
#include "sc_context.h"

using namespace scapi;

extern "C" {

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

}  // extern "C"
