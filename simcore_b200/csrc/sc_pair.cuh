// Segment-segment minimum distance and WCA pair force, FP64 (bit-exact) and
// FP32 (mixed) variants.
//
// FP64: MinimumDistance::Sphero (reference src/minimum_distance.cpp:202-344),
// WCAPotential::CalcPotential (include/simcore/wca_potential.hpp:14-32),
// MaxForcePotential::CalcPotential (include/simcore/max_force_potential.hpp:
// 11-40), dispatched as PotentialManager::CalcPotential
// (include/simcore/potential_manager.hpp:41-52), with the range test of
// InteractionManager::ProcessPairInteraction (src/interaction_manager.cpp:394).
// Expressions keep the reference's operand order; the unit is compiled with
// --fmad=false, so results are bit-identical.
//
// FP32: the same algorithm in single precision from fixed-point scaled
// positions (BondGeomF32), for the mixed-precision step.
#pragma once

#include "sc_common.cuh"

namespace sc {

// Result of one pair evaluation for obj1 = a, obj2 = b.
template <typename T>
struct PairGeom {
  T dr[3];
  T dr_mag2;
  T c1[3], c2[3];
};

template <int ND>
__device__ __forceinline__ void sphero_f64(const double *h,
                                           const BondGeomF64 &A,
                                           const BondGeomF64 &B,
                                           PairGeom<double> &g) {
  double dr[3], ds[3];
  const double half_length_1 = 0.5 * A.len;
  const double half_length_2 = 0.5 * B.len;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    ds[i] = B.s[i] - A.s[i];
    ds[i] -= nint(ds[i]);
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    dr[i] = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) dr[i] += h[ND * i + j] * ds[j];
  }
  double dr_dot_u_1 = 0.0, dr_dot_u_2 = 0.0, u_1_dot_u_2 = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    dr_dot_u_1 += dr[i] * A.u[i];
    dr_dot_u_2 += dr[i] * B.u[i];
    u_1_dot_u_2 += A.u[i] * B.u[i];
  }
  double lambda, mu;
  const double denom = 1.0 - u_1_dot_u_2 * u_1_dot_u_2;
  if (denom < 1.0e-12) {
    lambda = dr_dot_u_1 / 2.0;
    mu = -dr_dot_u_2 / 2.0;
  } else {
    lambda = (dr_dot_u_1 - u_1_dot_u_2 * dr_dot_u_2) / denom;
    mu = (-dr_dot_u_2 + u_1_dot_u_2 * dr_dot_u_1) / denom;
  }
  double lambda_mag = dabs(lambda);
  double mu_mag = dabs(mu);
  double r2 = 0.0;
  if (lambda_mag > half_length_1 && mu_mag > half_length_2) {
    double lambda_a = sign_of(half_length_1, lambda);
    double mu_a = -dr_dot_u_2 + lambda_a * u_1_dot_u_2;
    mu_mag = dabs(mu_a);
    if (mu_mag > half_length_2) mu_a = sign_of(half_length_2, mu_a);
    double ra[3], rb[3], r2a = 0.0, r2b = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      ra[i] = dr[i] - lambda_a * A.u[i] + mu_a * B.u[i];
      r2a += ra[i] * ra[i];
    }
    double mu_b = sign_of(half_length_2, mu);
    double lambda_b = dr_dot_u_1 + mu_b * u_1_dot_u_2;
    lambda_mag = dabs(lambda_b);
    if (lambda_mag > half_length_1) lambda_b = sign_of(half_length_1, lambda_b);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      rb[i] = dr[i] - lambda_b * A.u[i] + mu_b * B.u[i];
      r2b += rb[i] * rb[i];
    }
    if (r2a < r2b) {
      lambda = lambda_a;
      mu = mu_a;
      r2 = r2a;
#pragma unroll
      for (int i = 0; i < ND; ++i) g.dr[i] = ra[i];
    } else {
      lambda = lambda_b;
      mu = mu_b;
      r2 = r2b;
#pragma unroll
      for (int i = 0; i < ND; ++i) g.dr[i] = rb[i];
    }
  } else {
    if (lambda_mag > half_length_1) {
      lambda = sign_of(half_length_1, lambda);
      mu = -dr_dot_u_2 + lambda * u_1_dot_u_2;
      mu_mag = dabs(mu);
      if (mu_mag > half_length_2) mu = sign_of(half_length_2, mu);
    } else if (mu_mag > half_length_2) {
      mu = sign_of(half_length_2, mu);
      lambda = dr_dot_u_1 + mu * u_1_dot_u_2;
      lambda_mag = dabs(lambda);
      if (lambda_mag > half_length_1) lambda = sign_of(half_length_1, lambda);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      g.dr[i] = dr[i] - lambda * A.u[i] + mu * B.u[i];
      r2 += g.dr[i] * g.dr[i];
    }
  }
  g.dr_mag2 = r2;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    g.c1[i] = lambda * A.u[i];
    g.c2[i] = mu * B.u[i];
  }
#pragma unroll
  for (int i = ND; i < 3; ++i) g.dr[i] = g.c1[i] = g.c2[i] = 0.0;
}

// Evaluates the pair's potential if it is in range.  Returns true and
// writes force when a potential set the force; returns false when the
// reference leaves the pair's previous force in place (out of range, or
// the max-force fallback finds no direction).  When rec is given, a true
// return also writes the dr the pair's stress uses (the contact difference
// in the max-force case) and the potential (0 there) into rec[0..3]
// (Interaction::dr, pote; include/simcore/wca_potential.hpp:26-31,
// include/simcore/max_force_potential.hpp:15-39).
template <int ND>
__device__ __forceinline__ bool wca_f64(const SysConst &k, PairGeom<double> &g,
                                        double force[3], double *rec = nullptr) {
  if (g.dr_mag2 > k.rcut2) return false;
  if (g.dr_mag2 < 1e-12) {
    double dr[3] = {g.dr[0], g.dr[1], g.dr[2]};
    if (g.c1[0] || g.c1[1] || g.c1[2]) {
#pragma unroll
      for (int i = 0; i < ND; ++i) dr[i] = g.c1[i] - g.c2[i];
    }
    double rmag = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) rmag += dr[i] * dr[i];
    rmag = sqrt(rmag);
    if (rmag < 1e-12) return false;
    double rinv = 1.0 / (rmag);
#pragma unroll
    for (int i = 0; i < ND; ++i) force[i] = k.fcut * dr[i] * rinv;
    if (rec) {
      for (int i = 0; i < 3; ++i) rec[i] = i < ND ? dr[i] : 0.0;
      rec[3] = 0.0;
    }
    return true;
  }
  double rmag = sqrt(g.dr_mag2);
  double rinv = 1.0 / (rmag);
  double rinv2 = rinv * rinv;
  double r6 = rinv2 * rinv2 * rinv2;
  double ffac = -(12.0 * k.c12 * r6 - 6.0 * k.c6) * r6 * rinv;
  if (dabs(ffac) > k.fcut) ffac = signof(ffac) * k.fcut;
#pragma unroll
  for (int i = 0; i < ND; ++i) force[i] = ffac * g.dr[i] * rinv;
  if (rec) {
    for (int i = 0; i < 3; ++i) rec[i] = i < ND ? g.dr[i] : 0.0;
    rec[3] = r6 * (k.c12 * r6 - k.c6) + k.eps;
  }
  return true;
}

// ---- FP32 variant --------------------------------------------------------

__device__ __forceinline__ float fsign_of(float a, float b) {
  return b >= 0.0f ? fabsf(a) : -fabsf(a);
}

template <int ND>
__device__ __forceinline__ void sphero_f32(const float *hf,
                                           const BondGeomF32 &A,
                                           const BondGeomF32 &B,
                                           PairGeom<float> &g) {
  float ds[3], dr[3];
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    // Wrapping difference of fixed-point coordinates = minimum image.
    int32_t d = (int32_t)((uint32_t)B.q[i] - (uint32_t)A.q[i]);
    ds[i] = (float)d * 2.3283064365386963e-10f;
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < ND; ++j) acc = __fmaf_rn(hf[ND * i + j], ds[j], acc);
    dr[i] = acc;
  }
  float a1 = 0.f, a2 = 0.f, c = 0.f;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    a1 = __fmaf_rn(dr[i], A.u[i], a1);
    a2 = __fmaf_rn(dr[i], B.u[i], a2);
    c = __fmaf_rn(A.u[i], B.u[i], c);
  }
  const float h1 = A.hl, h2 = B.hl;
  float lambda, mu;
  const float denom = __fmaf_rn(-c, c, 1.0f);
  if (denom < 1.0e-12f) {
    lambda = 0.5f * a1;
    mu = -0.5f * a2;
  } else {
    float inv = 1.0f / denom;
    lambda = __fmaf_rn(-c, a2, a1) * inv;
    mu = __fmaf_rn(c, a1, -a2) * inv;
  }
  float lm = fabsf(lambda), mm = fabsf(mu), r2 = 0.f;
  if (lm > h1 && mm > h2) {
    float la = fsign_of(h1, lambda);
    float ma = __fmaf_rn(la, c, -a2);
    if (fabsf(ma) > h2) ma = fsign_of(h2, ma);
    float mb = fsign_of(h2, mu);
    float lb = __fmaf_rn(mb, c, a1);
    if (fabsf(lb) > h1) lb = fsign_of(h1, lb);
    float ra[3], rb[3], r2a = 0.f, r2b = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      ra[i] = __fmaf_rn(ma, B.u[i], __fmaf_rn(-la, A.u[i], dr[i]));
      r2a = __fmaf_rn(ra[i], ra[i], r2a);
      rb[i] = __fmaf_rn(mb, B.u[i], __fmaf_rn(-lb, A.u[i], dr[i]));
      r2b = __fmaf_rn(rb[i], rb[i], r2b);
    }
    if (r2a < r2b) {
      lambda = la;
      mu = ma;
      r2 = r2a;
#pragma unroll
      for (int i = 0; i < ND; ++i) g.dr[i] = ra[i];
    } else {
      lambda = lb;
      mu = mb;
      r2 = r2b;
#pragma unroll
      for (int i = 0; i < ND; ++i) g.dr[i] = rb[i];
    }
  } else {
    if (lm > h1) {
      lambda = fsign_of(h1, lambda);
      mu = __fmaf_rn(lambda, c, -a2);
      if (fabsf(mu) > h2) mu = fsign_of(h2, mu);
    } else if (mm > h2) {
      mu = fsign_of(h2, mu);
      lambda = __fmaf_rn(mu, c, a1);
      if (fabsf(lambda) > h1) lambda = fsign_of(h1, lambda);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      g.dr[i] = __fmaf_rn(mu, B.u[i], __fmaf_rn(-lambda, A.u[i], dr[i]));
      r2 = __fmaf_rn(g.dr[i], g.dr[i], r2);
    }
  }
  g.dr_mag2 = r2;
  // Explicit roundings here and below: no unit's contraction setting can
  // fuse these products into a later sum, so every unit computes one bits.
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    g.c1[i] = __fmul_rn(lambda, A.u[i]);
    g.c2[i] = __fmul_rn(mu, B.u[i]);
  }
#pragma unroll
  for (int i = ND; i < 3; ++i) g.dr[i] = g.c1[i] = g.c2[i] = 0.0f;
}

template <int ND>
__device__ __forceinline__ bool wca_f32(const SysConst &k, PairGeom<float> &g,
                                        float force[3], float *rec = nullptr) {
  if (g.dr_mag2 > k.rcut2f) return false;
  if (g.dr_mag2 < 1e-12f) {
    float dr[3] = {g.dr[0], g.dr[1], g.dr[2]};
    if (g.c1[0] != 0.f || g.c1[1] != 0.f || g.c1[2] != 0.f) {
#pragma unroll
      for (int i = 0; i < ND; ++i) dr[i] = g.c1[i] - g.c2[i];
    }
    float rm2 = 0.f;
#pragma unroll
    for (int i = 0; i < ND; ++i) rm2 = __fmaf_rn(dr[i], dr[i], rm2);
    float rmag = sqrtf(rm2);
    if (rmag < 1e-12f) return false;
    float s = k.fcutf / rmag;
#pragma unroll
    for (int i = 0; i < ND; ++i) force[i] = __fmul_rn(s, dr[i]);
    if (rec) {
      for (int i = 0; i < 3; ++i) rec[i] = i < ND ? dr[i] : 0.f;
      rec[3] = 0.f;
    }
    return true;
  }
  float rinv = rsqrtf(g.dr_mag2);
  float rinv2 = rinv * rinv;
  float r6 = rinv2 * rinv2 * rinv2;
  float ffac = -__fmaf_rn(12.0f * k.c12f, r6, -6.0f * k.c6f) * r6 * rinv;
  if (fabsf(ffac) > k.fcutf) ffac = (ffac >= 0.0f ? k.fcutf : -k.fcutf);
  float s = ffac * rinv;
#pragma unroll
  for (int i = 0; i < ND; ++i) force[i] = __fmul_rn(s, g.dr[i]);
  if (rec) {
    for (int i = 0; i < 3; ++i) rec[i] = i < ND ? g.dr[i] : 0.f;
    rec[3] = __fadd_rn(__fmul_rn(__fmaf_rn(k.c12f, r6, -k.c6f), r6), k.epsf);
  }
  return true;
}

// One pair of the mixed-precision pair stage: ProcessPairInteraction and the
// two torque cross products of InteractionManager::CalculatePairInteractions
// (src/interaction_manager.cpp:448-481).  Out of range, the force is the
// pair's stored one (st); in 2D the stored z component stays.  Returns
// whether the force was computed (and is to be stored).  The pair stage and
// the fused integrator both call this, and its products are explicitly
// rounded, so the two give the same bits.
template <int ND>
__device__ __forceinline__ bool pair_force_f32(const SysConst &k, const float *hf,
                                               const BondGeomF32 &A, const BondGeomF32 &B,
                                               const float4 &st, float force[3], float t1[3],
                                               float t2[3], float *rec = nullptr) {
  PairGeom<float> g;
  sphero_f32<ND>(hf, A, B, g);
  const bool set = wca_f32<ND>(k, g, force, rec);
  if (!set) {
    force[0] = st.x;
    force[1] = st.y;
    force[2] = st.z;
  } else if (ND == 2) {
    force[2] = st.z;
  }
  t1[0] = __fsub_rn(__fmul_rn(g.c1[1], force[2]), __fmul_rn(g.c1[2], force[1]));
  t1[1] = __fsub_rn(__fmul_rn(g.c1[2], force[0]), __fmul_rn(g.c1[0], force[2]));
  t1[2] = __fsub_rn(__fmul_rn(g.c1[0], force[1]), __fmul_rn(g.c1[1], force[0]));
  t2[0] = __fsub_rn(__fmul_rn(g.c2[1], force[2]), __fmul_rn(g.c2[2], force[1]));
  t2[1] = __fsub_rn(__fmul_rn(g.c2[2], force[0]), __fmul_rn(g.c2[0], force[2]));
  t2[2] = __fsub_rn(__fmul_rn(g.c2[0], force[1]), __fmul_rn(g.c2[1], force[0]));
  return set;
}

}  // namespace sc
