// Warp-synchronous integrator for filaments of at most 32 sites.
//
// A warp holds a group of whole filaments, one lane per site, filaments back
// to back.  Values of neighbouring sites move by register shuffles; the
// sequential recurrences of a filament (metric determinants, the two Thomas
// solves, renormalisation) run on one lane of the filament over a small
// per-warp shared-memory area, fenced by __syncwarp only.  No block-wide
// barrier exists, so a warp waiting on its recurrences holds up no other
// warp.  The arithmetic and its order are those of k_integrate (sc_step.cuh),
// so the exact variant stays bit-identical to the reference
// (src/filament.cpp:394-951, 992-1048).
#pragma once

#include "sc_step.cuh"

namespace sc {

constexpr int kIntWarps = 4;        // warps per block
constexpr int kIntMinBlocks = 5;    // resident blocks per SM the registers must allow
constexpr int kIntWarpDoubles = 480;  // shared doubles per warp

__device__ __forceinline__ double shfl_prev(double v, int dist) {
  return __shfl_up_sync(0xffffffffu, v, dist);
}
__device__ __forceinline__ double shfl_next(double v, int dist) {
  return __shfl_down_sync(0xffffffffu, v, dist);
}

// FUSE (fast mixed step only): each bond evaluates its own pairs
// (bond_pair_eval_sum) instead of summing the pair stage's slots.
template <int ND, int PREC, bool FAST, bool FUSE = false>
__global__ void __launch_bounds__(kIntWarps * 32, kIntMinBlocks)
    k_integrate_warp(SysConst k, DevState d, int midstep, int rbuf, int interaction,
                     int capture) {
  __shared__ double s_all[kIntWarps][kIntWarpDoubles];
  const unsigned FULL = 0xffffffffu;
  const int t = threadIdx.x & 31;
  const int w = blockIdx.x * kIntWarps + (threadIdx.x >> 5);
  if (w >= d.n_wg) return;  // whole warps only: nothing below synchronises the block
  // Without a pair stage in between (fused pairs, or no interactions) the
  // kernel before this one may be the previous integrator step, whose
  // writes every load below reads: wait for it first.
  if (FUSE || !interaction) grid_dep_sync();
  double *sm = s_all[threadIdx.x >> 5];
  double *scos = sm;         // cos(theta) of joint j at lane j      32
  double *sa = sm + 32;      // Thomas lower diagonal                 32
  double *sb = sm + 64;      // diagonal                              32
  double *sc = sm + 96;      // upper diagonal                        32
  double *sd = sm + 128;     // right-hand side / solution            32
  double *sdt = sm + 160;    // det_t, per filament at base + lf      64
  double *sdb = sm + 224;    // det_b                                 64
  double *srr = sm + 288;    // renormalisation: positions            3 x 32
  double *suu = sm + 384;    // renormalisation: bond orientations    3 x 32

  const int s0 = d.wg_site0[w];
  const int count = d.wg_ns[w];
  const int f0 = d.wg_f0[w];
  const bool active = t < count;
  const int g = s0 + (active ? t : 0);  // loads use a valid site on every lane
  const int f = d.site_fil[g];
  const int jn = d.site_jn[g];
  const int n = active ? jn >> 16 : 0;
  const int j = active ? jn & 0xffff : -1;
  const int base = t - j;    // lane of the filament's first site
  const int lf = f - f0;     // filament within the warp
  const int b = g - f;       // this lane's bond (valid when j < n-1)
  const bool has_bond = active && j < n - 1;
  const int bq = has_bond ? b : (b > 0 ? b - 1 : 0);  // a valid bond for loads
  const FilConst &fc = d.fil[f];
  const unsigned long long mcount = *d.mcount;
  // An overflowed rebuild of this step stops it before the first store
  // (read here, tested after the loads are issued).
  const bool overflowed = (*d.status & ST_LIST_OVERFLOW) != 0u;

  // ---- every global read of the step, issued together ---------------------
  double r[3] = {0, 0, 0}, u[3] = {0, 0, 0};
#pragma unroll
  for (int i = 0; i < ND; ++i) r[i] = d.r[i][g];
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i] = d.ub[i][bq];
  double fr[3] = {0, 0, 0}, rp[3] = {0, 0, 0}, dz[3] = {0, 0, 0}, dtot = 0.0;
  if (!midstep) {  // the midstep's positions and projected noise; rebuild origin
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rp[i] = d.rp[i][g];
      if (k.stoch) fr[i] = d.fr[i][g];
      if (interaction) dz[i] = d.dz[i][g];
    }
    if (interaction) dtot = d.dt[g];
  }
  int e0 = 0, e1 = 0;  // the bond's pair slots (written by the rebuild)
  if (!FUSE && has_bond && interaction) {
    e0 = d.e_off[b];
    e1 = e0 + d.e_cnt[b];
  }
  // Everything above is the previous integrator step's or older; the pair
  // stage just before this kernel writes the bond slots read below.
  grid_dep_sync();
  double bF[3] = {0, 0, 0}, bT[3] = {0, 0, 0};
  if (has_bond && interaction) {
    // (The fused evaluation follows the pair list only when the rebuild of
    // this step completed it.)
    if (FUSE) {
      if (!overflowed) bond_pair_eval_sum<ND>(k, d, d.rep[fc.rep].hf, rbuf, b, bF, bT);
    } else {
      bond_pair_sum<ND, PREC>(d, b, e0, e1, bF, bT);
    }
  }
  if (!has_bond) u[0] = u[1] = u[2] = 0.0;
  double xi[3] = {0, 0, 0};
  float xif[3] = {0.f, 0.f, 0.f};  // fast: the mixed step's FP32 noise
  if (midstep && k.stoch) {  // uniforms of ConstructUnprojectedRandomForces
    uint32_t wv[4];
    sc_host_philox4x32_10((uint32_t)j, (uint32_t)mcount, (uint32_t)(mcount >> 32), 0u,
                          d.rep[fc.rep].seed, (uint32_t)fc.f_local, wv);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      if (FAST) xif[i] = centered_uniform_f(wv[i]);
      else xi[i] = centered_uniform(wv[i]);
    }
  }
  if (overflowed) return;  // the whole warp: the bit is uniform
  if (active && midstep) {  // Mesh::UpdatePrevPositions (src/mesh.cpp:175-182)
#pragma unroll
    for (int i = 0; i < 3; ++i) d.rp[i][g] = r[i];
  }
  if (midstep) {
#pragma unroll
    for (int i = 0; i < 3; ++i) rp[i] = r[i];
  }
  double um[3], bFm[3], bTm[3];  // bond j-1, held by lane t-1
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    um[i] = shfl_prev(u[i], 1);
    bFm[i] = shfl_prev(bF[i], 1);
    bTm[i] = shfl_prev(bT[i], 1);
  }
  if (active && j == n - 1) {  // the last site copies the last bond's
    u[0] = um[0];
    u[1] = um[1];
    u[2] = um[2];
  }

  // ---- ApplyInteractionForces (src/filament.cpp:992-1048) -----------------
  double F[3] = {0.0, 0.0, 0.0};
  if (active) {
    const double mag = 0.5 * 0.0 * fc.l;  // driving_factor 0
    if (j >= 1) {
      double pt[3], sf[3];
      cross3(um, bTm, pt);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        pt[i] *= fc.linv;
        sf[i] = 0.5 * bFm[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) pt[i] *= -1;
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += sf[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += pt[i];
      if (!FAST) {
#pragma unroll
        for (int i = 0; i < ND; ++i) F[i] += mag * um[i];
      }
    }
    if (j <= n - 2) {
      double pt[3], sf[3];
      cross3(u, bT, pt);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        pt[i] *= fc.linv;
        sf[i] = 0.5 * bF[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += sf[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += pt[i];
      if (!FAST) {
#pragma unroll
        for (int i = 0; i < ND; ++i) F[i] += mag * u[i];
      }
    }
  }
  // CalculateAngles (:430-437), CalculateTangents (:439-443)
  double un[3];  // orientation of site j+1
#pragma unroll
  for (int i = 0; i < 3; ++i) un[i] = shfl_next(u[i], 1);
  double cs = 0.0;
  if (active && j < n - 2) cs = dotn<ND>(u, un);
  scos[t] = cs;
  double tn[3] = {0, 0, 0};
  if (active) {
    if (j == 0 || j == n - 1) {
      tn[0] = u[0];
      tn[1] = u[1];
      tn[2] = u[2];
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) tn[i] = um[i] + u[i];
      normalize<ND, FAST>(tn);
    }
  }

  // ---- random forces and their projection (midsteps, :518-599) ------------
  if (FAST && midstep && k.stoch) {
    // The mixed step: noise, projection and its solve in FP32 over the
    // Thomas arrays' first halves (as in k_integrate), the result in FP64.
    float *fa = reinterpret_cast<float *>(sa), *fb = reinterpret_cast<float *>(sb);
    float *fcm = reinterpret_cast<float *>(sc), *fd = reinterpret_cast<float *>(sd);
    float frf[3] = {0.f, 0.f, 0.f};
    const float uf[3] = {(float)u[0], (float)u[1], (float)u[2]};
    if (active) {
      float tnf[3] = {0.f, 0.f, 0.f}, txi = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        tnf[i] = (float)tn[i];
        txi = fmaf(tnf[i], xif[i], txi);
      }
      const float sperp = (float)fc.sperp, dsp = (float)(fc.spar - fc.sperp);
#pragma unroll
      for (int i = 0; i < ND; ++i) frf[i] = fmaf(sperp, xif[i], dsp * txi * tnf[i]);
    }
    float frn[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) frn[i] = __shfl_down_sync(0xffffffffu, frf[i], 1);
    if (has_bond) {
      float rhs = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) rhs = fmaf(frn[i] - frf[i], uf[i], rhs);
      fd[t] = rhs;
      fb[t] = 2.f;
      if (j < n - 2) {
        fcm[t] = -(float)cs;
        fa[t] = -(float)cs;
      }
    }
    __syncwarp();
    if (active && j == 0) thomas_fast(fa + t, fb + t, fcm + t, fd + t, n - 1);
    __syncwarp();
    if (active) {
      const float tt = j < n - 1 ? fd[t] : 0.f, tp = j > 0 ? fd[t - 1] : 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        const float up = j > 0 ? (float)um[i] : 0.f;
        fr[i] = (double)fmaf(tt, uf[i], fmaf(-tp, up, frf[i]));
      }
      d.fr[0][g] = fr[0];  // re-used by the full step
      d.fr[1][g] = fr[1];
      d.fr[2][g] = fr[2];
    }
  } else if (midstep && k.stoch) {
    if (active) {
      double xt[3] = {0, 0, 0};
      if (FAST) {
        const double txi = dotn<ND>(tn, xi);
#pragma unroll
        for (int i = 0; i < ND; ++i) xt[i] = txi * tn[i];
      } else if (ND == 2) {
        xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1];
        xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0];
      } else {
        xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1] + tn[0] * tn[2] * xi[2];
        xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0] + tn[1] * tn[2] * xi[2];
        xt[2] = tn[2] * tn[2] * xi[2] + tn[0] * tn[2] * xi[0] + tn[1] * tn[2] * xi[1];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) fr[i] = fc.sperp * xi[i] + (fc.spar - fc.sperp) * xt[i];
    }
    double frn[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) frn[i] = shfl_next(fr[i], 1);
    if (has_bond) {
      double tmp[3];
#pragma unroll
      for (int i = 0; i < ND; ++i) tmp[i] = frn[i] - fr[i];
      sd[t] = dotn<ND>(tmp, u);
      sb[t] = 2;
      if (j < n - 2) {
        sc[t] = -cs;
        sa[t] = -cs;
      }
    }
    __syncwarp();
    if (active && j == 0) solve_tridiag<FAST>(sa + t, sb + t, sc + t, sd + t, n - 1);
    __syncwarp();
    if (active) {
      double fp[3];
      if (j == 0) {
        const double T0 = sd[t];
#pragma unroll
        for (int i = 0; i < ND; ++i) fp[i] = fr[i] + T0 * u[i];
      } else if (j == n - 1) {
        const double Tm = sd[t - 1];
#pragma unroll
        for (int i = 0; i < ND; ++i) fp[i] = fr[i] - Tm * um[i];
      } else {
        const double T0 = sd[t], Tm = sd[t - 1];
#pragma unroll
        for (int i = 0; i < ND; ++i) fp[i] = fr[i] + T0 * u[i] - Tm * um[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) fr[i] = fp[i];
      d.fr[0][g] = fr[0];  // re-used by the full step
      d.fr[1][g] = fr[1];
      d.fr[2][g] = fr[2];
    }
  }
  // AddRandomForces (:601-606)
  if (active && k.stoch) {
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fr[i];
  }

  // ---- bending and metric forces (:608-776) -------------------------------
  __syncwarp();
  if (active && j <= 1) {
    // Lane j = 0: det_t forward; lane j = 1: det_b backward (same stream of
    // instructions, mirrored indices).
    const bool fwd = j == 0;
    double *dst = (fwd ? sdt : sdb) + base + lf;
    const double *cz = scos + base;
    double x0 = 1.0, x1 = 2.0;
    dst[fwd ? 0 : n] = x0;
    dst[fwd ? 1 : n - 1] = x1;
    for (int i = 2; i < n; ++i) {
      const double c = cz[fwd ? i - 2 : n - i - 1];
      const double x2 = 2 * x1 - (-c) * (-c) * x0;
      dst[fwd ? i : n - i] = x2;
      x0 = x1;
      x1 = x2;
    }
  }
  __syncwarp();
  double ke = 0.0;
  if (active && j < n - 2) {
    const int dbase = base + lf;
    const double det_g = sdt[dbase + n - 1];
    if (FAST) {
      const double ginv = cs * sdt[dbase + j] * sdb[dbase + j + 3] * recip_nr(det_g);
      ke = (fc.kappa + fc.l * ginv) * recip_nr(fc.l2);
    } else {
      const double ginv = cs * sdt[dbase + j] * sdb[dbase + j + 3] / det_g;
      ke = (fc.kappa + fc.l * ginv) / fc.l2;
    }
  }
  const double kem1 = shfl_prev(ke, 1), kem2 = shfl_prev(ke, 2);
  const double csm1 = shfl_prev(cs, 1), csm2 = shfl_prev(cs, 2);
  double umm[3];  // orientation of site j-2
#pragma unroll
  for (int i = 0; i < 3; ++i) umm[i] = shfl_prev(u[i], 2);
  if (active && FAST) {
    // (I - u2 u2^T) u1 = u1 - (u1 . u2) u2, with the cosines of CalculateAngles
    double fs[3] = {0, 0, 0};
    if (j > 1) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] += kem2 * (umm[i] - csm2 * um[i]);
    }
    if (j > 0 && j < n - 1) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] += kem1 * ((u[i] - csm1 * um[i]) - (um[i] - csm1 * u[i]));
    }
    if (j < n - 2) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] -= ke * (un[i] - cs * u[i]);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
  } else if (active) {
    double fs[3] = {0, 0, 0};
    if (ND == 2) {
      if (j > 1) {
        const double *u1 = umm, *u2 = um;
        fs[0] += kem2 * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]);
        fs[1] += kem2 * ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]);
      }
      if (j > 0 && j < n - 1) {
        const double *u1 = um, *u2 = u;
        fs[0] += kem1 * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                         ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]));
        fs[1] += kem1 * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0] -
                         ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]));
      }
      if (j < n - 2) {
        const double *u1 = u, *u2 = un;
        fs[0] -= ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1]);
        fs[1] -= ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0]);
      }
    } else {
      if (j > 1) {
        const double *u1 = umm, *u2 = um;
        fs[0] += kem2 * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                         u2[0] * u2[2] * u1[2]);
        fs[1] += kem2 * ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                         u2[1] * u2[2] * u1[2]);
        fs[2] += kem2 * ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                         u2[2] * u2[1] * u1[1]);
      }
      if (j > 0 && j < n - 1) {
        const double *u1 = um, *u2 = u;
        fs[0] += kem1 * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                         u1[0] * u1[2] * u2[2] -
                         ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                          u2[0] * u2[2] * u1[2]));
        fs[1] += kem1 * ((1 - u1[1] * u1[1]) * u2[1] - u1[1] * u1[0] * u2[0] -
                         u1[1] * u1[2] * u2[2] -
                         ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                          u2[1] * u2[2] * u1[2]));
        fs[2] += kem1 * ((1 - u1[2] * u1[2]) * u2[2] - u1[2] * u1[0] * u2[0] -
                         u1[2] * u1[1] * u2[1] -
                         ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                          u2[1] * u2[2] * u1[1]));
      }
      if (j < n - 2) {
        const double *u1 = u, *u2 = un;
        fs[0] -= ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       u1[0] * u1[2] * u2[2]);
        fs[1] -= ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[1] * u1[0] * u2[0] -
                       u1[1] * u1[2] * u2[2]);
        fs[2] -= ke * ((1 - u1[2] * u1[2]) * u2[2] - u1[2] * u1[0] * u2[0] -
                       u1[2] * u1[1] * u2[1]);
      }
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
  }

  // ---- tensions (:778-838) ------------------------------------------------
  // gamma^-1 = (1/gpar) t t + (1/gperp)(I - t t)
  auto gam = [&](int a, int c) -> double {
    return fc.igpar * (tn[a] * tn[c]) + fc.igperp * ((a == c ? 1 : 0) - tn[a] * tn[c]);
  };
  auto gamma_inv_F = [&](double out[3]) {
    if (FAST) {
      const double tF = dotn<ND>(tn, F);
#pragma unroll
      for (int i = 0; i < ND; ++i) out[i] = fc.igperp * F[i] + fc.dgam * tF * tn[i];
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        double v = gam(i, 0) * F[0] + gam(i, 1) * F[1];
        if (ND == 3) v += gam(i, 2) * F[2];
        out[i] = v;
      }
    }
  };
  double gF[3] = {0, 0, 0};
  if (active) gamma_inv_F(gF);
  double gFn[3], tnn[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    gFn[i] = shfl_next(gF[i], 1);
    tnn[i] = shfl_next(tn[i], 1);
  }
  if (has_bond) {
    double fdiff[3];
#pragma unroll
    for (int i = 0; i < ND; ++i) fdiff[i] = gFn[i] - gF[i];
    sd[t] = dotn<ND>(u, fdiff);
    const double d1 = dotn<ND>(tn, u);
    const double d2 = dotn<ND>(tnn, u);
    sb[t] = fc.two_igperp + fc.dgam * (d1 * d1 + d2 * d2);
    if (j > 0) {
      const double hu = fc.m1_igperp * dotn<ND>(u, um) -
                        fc.dgam * (dotn<ND>(tn, um) * dotn<ND>(tn, u));
      sc[t - 1] = hu;
      sa[t - 1] = hu;
    }
  }
  __syncwarp();
  if (active && j == 0) solve_tridiag<FAST>(sa + t, sb + t, sc + t, sd + t, n - 1);
  __syncwarp();

  // ---- UpdateSitePositions (:840-927), CheckBondLengths (:934-951) --------
  double T0 = 0.0;
  if (active) {
    double fs[3];
    if (j == 0) {
      T0 = sd[t];
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = T0 * u[i];
    } else if (j == n - 1) {
      const double Tm = sd[t - 1];
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = -Tm * um[i];
    } else {
      T0 = sd[t];
      const double Tm = sd[t - 1];
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = T0 * u[i] - Tm * um[i];
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
    const double dl = (midstep ? 0.5 * k.delta : k.delta);
    double ft[3] = {0, 0, 0};
    gamma_inv_F(ft);
#pragma unroll
    for (int i = 0; i < ND; ++i) r[i] = rp[i] + dl * ft[i];
  }
  double rn[3], rm[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    rn[i] = shfl_next(r[i], 1);
    rm[i] = shfl_prev(r[i], 1);
  }
  double rd[3] = {0, 0, 0}, um_len = 0.0;
  if (has_bond) {
#pragma unroll
    for (int i = 0; i < ND; ++i) rd[i] = rn[i] - r[i];
    um_len = normalize<ND, FAST>(rd);
  }
  bool bad_len = false;
  if (active && j >= 1) {
    double a = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      const double temp = r[i] - rm[i];
      a += temp * temp;
    }
    if (FAST) {
      const double lo = fc.l * (1.0 - 1e-3), hi = fc.l * (1.0 + 1e-3);
      bad_len = a < lo * lo || a > hi * hi;
    } else {
      a = sqrt(a);
      const double err = dabs(fc.l - a) / fc.l;
      bad_len = err > 1e-3;
    }
  }
  const unsigned bad_lanes = __ballot_sync(FULL, bad_len);
  const unsigned fil_lanes =
      active ? (unsigned)((((unsigned long long)1 << n) - 1ull) << base) : 0u;
  const bool renorm = (bad_lanes & fil_lanes) != 0u;
  int sw = 0;
  if (active && j == 0) {
    sw = d.f_switch[f];
    int nnorm = d.f_nnorm[f];
    if (renorm) {
      sw = !sw;
      nnorm = 0;
    }
    nnorm++;
    d.f_switch[f] = sw;
    d.f_nnorm[f] = nnorm;
  }
  if (__any_sync(FULL, renorm)) {
    // Re-place the sites along the new bond orientations, tail to head or
    // head to tail (the sequential loops of CheckBondLengths).
    if (active) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        srr[32 * i + t] = r[i];
        suu[32 * i + t] = rd[i];
      }
    }
    __syncwarp();
    if (active && j == 0 && renorm) {
      const double l = fc.l;
      if (sw) {
        for (int jj = 1; jj < n; ++jj)
#pragma unroll
          for (int i = 0; i < ND; ++i)
            srr[32 * i + t + jj] = srr[32 * i + t + jj - 1] + l * suu[32 * i + t + jj - 1];
      } else {
        for (int jj = n - 1; jj > 0; --jj)
#pragma unroll
          for (int i = 0; i < ND; ++i)
            srr[32 * i + t + jj - 1] = srr[32 * i + t + jj] - l * suu[32 * i + t + jj - 1];
      }
    }
    __syncwarp();
    if (active && renorm) {
#pragma unroll
      for (int i = 0; i < 3; ++i) r[i] = srr[32 * i + t];
    }
  }

  // ---- bond geometry (Mesh::UpdateBondPositions), state write-back --------
  double r2[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) r2[i] = shfl_next(r[i], 1);
  double my_dr = 0.0;
  if (active) {
    if (has_bond) {
      // Bond::ReInit on the final sites; without renormalisation it repeats
      // the orientation just computed (same operands, same operations).
      double s[3] = {0, 0, 0}, ub[3] = {0, 0, 0}, len, pos[3] = {0, 0, 0}, o[3] = {0, 0, 0};
      if (renorm) {
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          o[i] = r2[i] - r[i];
          ub[i] = o[i];
        }
        len = normalize<ND, FAST>(ub);
      } else {
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          o[i] = r2[i] - r[i];
          ub[i] = rd[i];
        }
        len = um_len;
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) pos[i] = r[i] + 0.5 * o[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        s[i] = 0.0;
#pragma unroll
        for (int jj = 0; jj < ND; ++jj) s[i] += d.rep[fc.rep].hinv[ND * i + jj] * pos[jj];
        s[i] -= nint(s[i]);
      }
      store_geom<ND>(d, 1 - rbuf, b, s, ub, len, PREC);
      d.ub[0][b] = ub[0];
      d.ub[1][b] = ub[1];
      d.ub[2][b] = ub[2];
    }
    d.r[0][g] = r[0];
    d.r[1][g] = r[1];
    d.r[2][g] = r[2];
    bool nan = false;
#pragma unroll
    for (int i = 0; i < ND; ++i) nan |= !isfinite(r[i]);
    if (nan) atomicOr(d.status, ST_NAN);
    if (capture) {
      for (int i = 0; i < 3; ++i) d.cap_F[i][g] = F[i];
      if (has_bond) d.cap_T[b] = T0;
    }
    // Displacement tracking for the next rebuild check: each query adds the
    // squared displacement twice (src/mesh.cpp:538-541, src/object.cpp:282-292).
    if (!midstep && interaction) {
      double acc = dtot;
      for (int twice = 0; twice < 2; ++twice)
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          const double dr = r[i] - dz[i];
          acc += dr * dr;
        }
      d.dt[g] = acc;
      my_dr = acc;
    }
  }
  if (!midstep && interaction) {
    double v = my_dr;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    if (t == 0) {
      if (!(v <= 1e300)) atomicOr(d.status, ST_NAN);
      // Non-negative doubles order as their bit patterns; most warps see a
      // larger maximum already and skip the atomic.
      const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
      unsigned long long *slot = &d.dr_max_bits[fc.rep];
      if (bits > *(volatile unsigned long long *)slot) atomicMax(slot, bits);
    }
  }
}

}  // namespace sc
