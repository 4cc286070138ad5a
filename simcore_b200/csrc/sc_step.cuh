// Integrator of the filament step and the device helpers it shares with the
// rest of the pipeline, as a header compiled by two units:
//   sc_kernels.cu      (--fmad=false): FAST = false, the reference's exact
//                      arithmetic, bit-identical to it;
//   sc_kernels_fast.cu (--fmad=true):  FAST = true, the same algorithm with
//                      contraction, one reciprocal per shared denominator and
//                      rsqrt normalisation (mixed precision only).
#pragma once

#include "sc_common.cuh"
#include "sc_pair.cuh"

namespace sc {

// ---------------------------------------------------------------------------
// Bond geometry from two sites: Bond::ReInit (src/bond.cpp:22-37) followed by
// Object::UpdatePeriodic / periodic_boundary_conditions
// (src/object.cpp:202-210, src/linear_algebra.cpp:100-117).
template <int ND>
__device__ __forceinline__ void bond_from_sites(const double *hinv,
                                                const double *r1,
                                                const double *r2, double s[3],
                                                double u[3], double &len) {
  double pos[3] = {0, 0, 0};
  u[0] = u[1] = u[2] = 0.0;
  s[0] = s[1] = s[2] = 0.0;
  len = 0;
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    u[i] = r2[i] - r1[i];
    len += u[i] * u[i];
  }
  len = sqrt(len);
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    pos[i] = r1[i] + 0.5 * u[i];
    u[i] /= len;
  }
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    s[i] = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) s[i] += hinv[ND * i + j] * pos[j];
    s[i] -= nint(s[i]);
  }
}

__device__ __forceinline__ int32_t to_fixed(double s) {
  // s in [-1/2, 1/2]: round(s * 2^32) wraps into int32 (1/2 and -1/2 map to
  // the same point of the periodic box).
  long long q = __double2ll_rn(s * 4294967296.0);
  return (int32_t)(uint32_t)(unsigned long long)q;
}

template <int ND>
__device__ __forceinline__ void store_geom(const DevState &d, int buf, int b,
                                           const double s[3],
                                           const double u[3], double len,
                                           int prec) {
  if (prec == 0) {
    BondGeomF64 g;
    g.s[0] = s[0];
    g.s[1] = s[1];
    g.s[2] = s[2];
    g.u[0] = u[0];
    g.u[1] = u[1];
    g.u[2] = u[2];
    g.len = len;
    g.pad = 0.0;
    d.g64[buf][b] = g;
  } else {
    BondGeomF32 g;
    g.q[0] = to_fixed(s[0]);
    g.q[1] = to_fixed(s[1]);
    g.q[2] = ND == 3 ? to_fixed(s[2]) : 0;
    g.hl = (float)(0.5 * len);
    g.u[0] = (float)u[0];
    g.u[1] = (float)u[1];
    g.u[2] = (float)u[2];
    g.pad = 0.f;
    d.g32[buf][b] = g;
  }
}

__device__ __forceinline__ void cross3(const double *a, const double *b,
                                       double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ void kahan_add(float &sum, float &comp, float x) {
  float y = x - comp;
  float t = sum + y;
  comp = (t - sum) - y;
  sum = t;
}

// Sum of one bond's crosslink anchor contributions in link order, as
// CrosslinkSpecies::ApplyCrosslinkTetherForces adds them to Bond::force_ /
// torque_ before the pair path (src/crosslink_species.cpp:260-266,
// src/anchor.cpp:132-146): ND force components, 3 torque components.  Of
// the anchors listed on the bond, those that sit on it count.
template <int ND>
__device__ __forceinline__ void bond_xlink_sum(const DevState &d, int b, double F[3],
                                               double T[3]) {
  const int e0 = d.xb_off[b], e1 = d.xb_off[b + 1];
  for (int e = e0; e < e1; ++e) {
    const double2 *c = reinterpret_cast<const double2 *>(d.xl_c) + 4 * (size_t)d.xb_ent[e];
    if ((int)c[3].x != b) continue;
    const double2 v0 = c[0], v1 = c[1], v2 = c[2];
    F[0] += v0.x;
    F[1] += v0.y;
    if (ND == 3) F[2] += v1.x;
    T[0] += v1.y;
    T[1] += v2.x;
    T[2] += v2.y;
  }
}

// Bond::force_ / torque_ after Interact: crosslink anchors first, then the
// bond's pair contributions in slot (= pair) order.  FP64 sums as the
// reference accumulates them; in mixed precision FP32 sums with Kahan
// compensation, added to the FP64 crosslink sum.  A pair slot is 8 values: force (3), torque (3),
// padding (2).  [e0, e1) is the bond's slot range (e_off, e_off + e_cnt),
// which the integrators load before they wait for the pair stage: the
// rebuild wrote it, before the pair stage ran.
template <int ND, int PREC>
__device__ __forceinline__ void bond_pair_sum(const DevState &d, int b, int e0, int e1,
                                              double F[3], double T[3]) {
  F[0] = F[1] = F[2] = 0.0;
  T[0] = T[1] = T[2] = 0.0;
  if (d.nx) bond_xlink_sum<ND>(d, b, F, T);
  if (PREC == 0) {
    const double2 *c = reinterpret_cast<const double2 *>(d.cf64) + 4 * (size_t)e0;
#pragma unroll 2
    for (int e = e0; e < e1; ++e, c += 4) {
      const double2 v0 = c[0], v1 = c[1], v2 = c[2];
      F[0] += v0.x;
      F[1] += v0.y;
      if (ND == 3) F[2] += v1.x;
      T[0] += v1.y;
      T[1] += v2.x;
      T[2] += v2.y;
    }
  } else {
    float sF[3] = {0.f, 0.f, 0.f}, cF[3] = {0.f, 0.f, 0.f};
    float sT[3] = {0.f, 0.f, 0.f}, cT[3] = {0.f, 0.f, 0.f};
    const float4 *c = reinterpret_cast<const float4 *>(d.cf32) + 2 * (size_t)e0;
#pragma unroll 4
    for (int e = e0; e < e1; ++e, c += 2) {
      const float4 v0 = c[0], v1 = c[1];
      kahan_add(sF[0], cF[0], v0.x);
      kahan_add(sF[1], cF[1], v0.y);
      if (ND == 3) kahan_add(sF[2], cF[2], v0.z);
      kahan_add(sT[0], cT[0], v0.w);
      kahan_add(sT[1], cT[1], v1.x);
      kahan_add(sT[2], cT[2], v1.y);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      F[i] += (double)sF[i] - (double)cF[i];
      T[i] += (double)sT[i] - (double)cT[i];
    }
  }
}

// Bond::force_ / torque_ of the mixed step with the pair stage fused in.
// The bond evaluates each of its pairs itself (pair_force_f32 on both bonds'
// FP32 geometry of this step), in entry (= slot) order, and adds its side of
// the force and torque exactly as bond_pair_sum adds the slots the pair stage
// would have written: the same values in the same order, so the same bits.
// Both bonds of a pair evaluate it.  The first (role 0) stores the force, and
// only when it was computed; the second reads the stored force only when it
// was not, so no bond reads a value that another is writing for this step.
template <int ND>
__device__ __forceinline__ void bond_pair_eval_sum(const SysConst &k, const DevState &d,
                                                   const float *hf, int rbuf, int b,
                                                   double F[3], double T[3]) {
  const int e0 = d.e_off[b], e1 = e0 + d.e_cnt[b];
  F[0] = F[1] = F[2] = 0.0;
  T[0] = T[1] = T[2] = 0.0;
  if (d.nx) bond_xlink_sum<ND>(d, b, F, T);
  float sF[3] = {0.f, 0.f, 0.f}, cF[3] = {0.f, 0.f, 0.f};
  float sT[3] = {0.f, 0.f, 0.f}, cT[3] = {0.f, 0.f, 0.f};
  for (int e = e0; e < e1; ++e) {
    const int ent = d.e_ent[e], p = ent >> 1;
    const BondGeomF32 A = d.g32[rbuf][d.pa[p]], B = d.g32[rbuf][d.pb[p]];
    float4 *stale = reinterpret_cast<float4 *>(d.pf32) + (size_t)p;
    float f[3], t1[3], t2[3], v[6];
    const bool set = pair_force_f32<ND>(k, hf, A, B, *stale, f, t1, t2);
    if (ent & 1) {
      v[0] = -f[0];
      v[1] = -f[1];
      v[2] = -f[2];
      v[3] = -t2[0];
      v[4] = -t2[1];
      v[5] = -t2[2];
    } else {
      if (set) *stale = make_float4(f[0], f[1], f[2], 0.f);
      v[0] = f[0];
      v[1] = f[1];
      v[2] = f[2];
      v[3] = t1[0];
      v[4] = t1[1];
      v[5] = t1[2];
    }
    kahan_add(sF[0], cF[0], v[0]);
    kahan_add(sF[1], cF[1], v[1]);
    if (ND == 3) kahan_add(sF[2], cF[2], v[2]);
    kahan_add(sT[0], cT[0], v[3]);
    kahan_add(sT[1], cT[1], v[4]);
    kahan_add(sT[2], cT[2], v[5]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    F[i] += (double)sF[i] - (double)cF[i];
    T[i] += (double)sT[i] - (double)cT[i];
  }
}

// ---------------------------------------------------------------------------
// Integrator.  A block holds a run of whole filaments, one thread per site,
// filaments back to back.  Per-site work runs in parallel; the sequential
// recurrences of one filament (metric determinants, Thomas solves,
// renormalisation) run on one dedicated lane per filament (lane lf for
// filament lf of the block, lane C/2 + lf for the backward determinant), so
// a block's serial work occupies one or two warps instead of every warp.

// Thomas algorithm of the reference's tridiagonal_solver
// (src/linear_algebra.cpp:164-197); n unknowns, in place.  The previous
// row's c and d stay in registers (same values, same operations as reading
// them back).
__device__ __forceinline__ void thomas(double *a, const double *b, double *c,
                                       double *d, int n) {
  n--;
  double cp = c[0] / b[0];
  double dp = d[0] / b[0];
  c[0] = cp;
  d[0] = dp;
  for (int i = 1; i < n; ++i) {
    const double am = a[i - 1], bi = b[i];
    const double cn = c[i] / (bi - am * cp);
    const double dn = (d[i] - am * dp) / (bi - am * cp);
    c[i] = cn;
    d[i] = dn;
    cp = cn;
    dp = dn;
  }
  dp = (d[n] - a[n - 1] * dp) / (b[n] - a[n - 1] * cp);
  d[n] = dp;
  for (int i = n; i-- > 0;) {
    dp = d[i] - c[i] * dp;
    d[i] = dp;
  }
}

// 1/x for the fast integrator: from the hardware's FP64 approximate
// reciprocal y of x (PTX rcp.approx.ftz.f64), one step of the third-order
// iteration y <- y (1 + e + e^2) with e = 1 - x y, the truncated series of
// y / (1 - e) (Muller et al., Handbook of Floating-Point Arithmetic, 2nd
// ed., sec. 4.7).  The seed's relative error is below 2^-19 (measured
// 9.9e-7), so the step leaves e^3 < 2^-57 before the final rounding: within
// an ulp of 1/x, from three dependent FMAs after one approximation and no
// FP32 round trip (conversions are slow on this part).  For normal |x|,
// which the diagonals, determinants and lengths it serves are.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double recip_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

// x^-1/2 for the fast integrator, the same way: the hardware's approximate
// inverse square root y (PTX rsqrt.approx.ftz.f64), e = 1 - x y^2, and
// y (1 - e)^-1/2 by its series to the second order, y (1 + e/2 + 3e^2/8):
// relative error about 5e^3/16 before the final rounding (seed error below
// 2^-19, measured 9.2e-7; the result within an ulp of 1/sqrt(x)).
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y * y, 1.0);
  return fma(y, e * fma(e, 0.375, 0.5), y);
}

// ((double)w + 0.5) * 2^-32 - 0.5 for a 32-bit Philox word w, the noise's
// uniform on (-1/2, 1/2).  w + 1/2 is formed exactly from bits -- 2^51 + w +
// 1/2 is the double with exponent 51 and mantissa 2w + 1 -- instead of by an
// integer-to-double conversion; the product with 2^-32 is exact, so the
// result has the same bits as the expression above.
__device__ __forceinline__ double centered_uniform(uint32_t w) {
  const double h =
      __longlong_as_double(0x4320000000000000ll | (((long long)w << 1) | 1ll)) - 2251799813685248.0;
  return h * 2.3283064365386963e-10 - 0.5;
}

// The same uniform in FP32 from the word's top 23 bits, (m + 1/2) 2^-23 -
// 1/2 with m = w >> 9, exact (m from its bits, as above): the mixed step's
// noise, within 2^-24 of the FP64 one.
__device__ __forceinline__ float centered_uniform_f(uint32_t w) {
  const float m = __uint_as_float(0x4B000000u | (w >> 9)) - 8388608.0f;
  return fmaf(m + 0.5f, 1.1920928955078125e-7f, -0.5f);
}

__device__ __forceinline__ double recip_t(double x) { return recip_nr(x); }
__device__ __forceinline__ float recip_t(float x) { return rcp_approx(x); }

// FAST: one reciprocal per row instead of two divisions (FP64: recip_nr;
// FP32: the approximate reciprocal, within an ulp).
template <class T>
__device__ __forceinline__ void thomas_fast(T *a, const T *b, T *c, T *d, int n) {
  n--;
  T r = recip_t(b[0]);
  T cp = c[0] * r;
  T dp = d[0] * r;
  c[0] = cp;
  d[0] = dp;
  for (int i = 1; i < n; ++i) {
    const T am = a[i - 1];
    r = recip_t(b[i] - am * cp);
    const T cn = c[i] * r;
    const T dn = (d[i] - am * dp) * r;
    c[i] = cn;
    d[i] = dn;
    cp = cn;
    dp = dn;
  }
  dp = (d[n] - a[n - 1] * dp) * recip_t(b[n] - a[n - 1] * cp);
  d[n] = dp;
  for (int i = n; i-- > 0;) {
    dp = d[i] - c[i] * dp;
    d[i] = dp;
  }
}

template <bool FAST>
__device__ __forceinline__ void solve_tridiag(double *a, const double *b, double *c,
                                              double *d, int n) {
  if (FAST) thomas_fast(a, b, c, d, n);
  else thomas(a, b, c, d, n);
}

// Two-sided ("twisted") elimination of one tridiagonal system of n rows for
// the fast integrator (van der Vorst, "Large tridiagonal and block
// tridiagonal linear systems on vector and parallel computers", Parallel
// Computing 5:45-54, 1987): a pair of lanes of one warp, the top lane
// eliminating rows 0..m-1 downwards and the bottom lane rows n-1..m+1
// upwards, meet at row m = n/2, then substitute back outwards.  Half the
// sequential depth of thomas_fast, the same layout (row r: lower coefficient
// a[r-1], diagonal b[r], upper c[r], right-hand side d[r]); the solution
// ends in d.  Both lanes of the pair (lanes 2k, 2k+1) call it, and both run
// one instruction stream: P[r] is the coupling to the row eliminated before
// (a[r-1] going down, c[r] going up), Q[r] the one towards row m, which the
// elimination overwrites with its reduced value.
template <class T>
__device__ __forceinline__ void thomas_twisted(T *a, const T *b, T *c, T *d, int n, bool top) {
  const unsigned pair = 3u << ((threadIdx.x & 31) & 30);
  const int m = n >> 1;
  const int steps = top ? m : n - 1 - m;
  const int dir = top ? 1 : -1;
  const int r0 = top ? 0 : n - 1;
  const T *P = top ? a - 1 : c;
  T *Q = top ? c : a - 1;
  T u = 0, v = 0;  // reduced (Q, d) of the last row eliminated
  // Each row's coefficients are loaded before the stores of the row before
  // (they never overlap), so only the elimination's own chain is serial.
  // The first row has no coupling (pc = 0 leaves b and d as they are).
  int r = r0;
  T pc = 0, bb = 0, qq = 0, dd = 0;
  if (steps > 0) {
    bb = b[r];
    qq = Q[r];
    dd = d[r];
  }
  for (int st = 0; st < steps; ++st) {
    const int rn = r + dir;
    T pcn = 0, bbn = 0, qqn = 0, ddn = 0;
    if (st + 1 < steps) {
      pcn = P[rn];
      bbn = b[rn];
      qqn = Q[rn];
      ddn = d[rn];
    }
    const T ri = recip_t(bb - pc * u);
    u = qq * ri;
    v = (dd - pc * v) * ri;
    Q[r] = u;
    d[r] = v;
    r = rn;
    pc = pcn;
    bb = bbn;
    qq = qqn;
    dd = ddn;
  }
  const T u2 = __shfl_xor_sync(pair, u, 1), v2 = __shfl_xor_sync(pair, v, 1);
  const T tu = top ? u : u2, tv = top ? v : v2;  // row m-1: c', d'
  const T bu = top ? u2 : u, bv = top ? v2 : v;  // row m+1: a', d'
  T num = d[m], den = b[m];
  if (m >= 1) {
    num -= a[m - 1] * tv;
    den -= a[m - 1] * tu;
  }
  if (m + 1 <= n - 1) {
    num -= c[m] * bv;
    den -= c[m] * bu;
  }
  T x = num * recip_t(den);
  __syncwarp(pair);  // both lanes have read row m
  if (top) d[m] = x;
  r = m - dir;
  T qb = 0, db = 0;
  if (steps > 0) {
    qb = Q[r];
    db = d[r];
  }
  for (int st = 0; st < steps; ++st) {
    const int rn = r - dir;
    T qn = 0, dn = 0;
    if (st + 1 < steps) {
      qn = Q[rn];
      dn = d[rn];
    }
    x = db - qb * x;
    d[r] = x;
    r = rn;
    qb = qn;
    db = dn;
  }
}

// Metric determinants of filament q of a block (CalculateBendingForces,
// src/filament.cpp:627-660): det_t forward and det_b backward, each on its
// own lane; filament q's values start at slot (first site) + q.
__device__ __forceinline__ void det_forward(double *sdt, const double *scos, const FilConst &f,
                                            int s0, int q) {
  const int fb0 = f.site0 - s0, nn = f.n;
  double *dt = sdt + fb0 + q;
  const double *cs = scos + fb0;
  // The two previous values are carried in registers and each cosine is
  // loaded a row ahead: the recurrence's chain holds no memory access.
  double d2 = 1, d1 = 2;
  dt[0] = d2;
  dt[1] = d1;
  double m = nn > 2 ? -cs[0] : 0.0;
  for (int i = 2; i < nn; ++i) {
    const double mn = i + 1 < nn ? -cs[i - 1] : 0.0;
    const double dn = 2 * d1 - m * m * d2;
    dt[i] = dn;
    d2 = d1;
    d1 = dn;
    m = mn;
  }
}
__device__ __forceinline__ void det_backward(double *sdb, const double *scos, const FilConst &f,
                                             int s0, int q) {
  const int fb0 = f.site0 - s0, nn = f.n;
  double *db = sdb + fb0 + q;
  const double *cs = scos + fb0;
  double d2 = 1, d1 = 2;
  db[nn] = d2;
  db[nn - 1] = d1;
  double m = nn > 2 ? -cs[nn - 3] : 0.0;
  for (int i = 2; i < nn; ++i) {
    const double mn = i + 1 < nn ? -cs[nn - i - 2] : 0.0;
    const double dn = 2 * d1 - m * m * d2;
    db[nn - i] = dn;
    d2 = d1;
    d1 = dn;
    m = mn;
  }
}

// v /= |v| over ND components.  Exact: the reference's normalize_vector
// (src/linear_algebra.cpp:26-35).  FAST: one rsqrt and ND products.
template <int ND, bool FAST>
__device__ __forceinline__ double normalize(double *v) {
  double mag = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) mag += v[i] * v[i];
  if (FAST) {
    double inv = rsqrt_nr(mag);
#pragma unroll
    for (int i = 0; i < ND; ++i) v[i] *= inv;
    return mag * inv;
  }
  mag = sqrt(mag);
#pragma unroll
  for (int i = 0; i < ND; ++i) v[i] /= mag;
  return mag;
}

template <int ND>
__device__ __forceinline__ double dotn(const double *a, const double *b) {
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < ND; ++i) m += a[i] * b[i];
  return m;
}

// Shared-memory words of one integrator block of C sites (the doubles; C/2
// renormalisation flags and the block's filament constants follow).
__host__ __device__ constexpr size_t integrate_smem_doubles(int C) {
  return 28 * (size_t)C;
}

// 8-byte asynchronous global -> shared copy (cp.async), completed by
// cp_async_wait_all() in the same thread.
__device__ __forceinline__ void cp_async8(double *smem_dst, const double *gsrc) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// MAXC: largest block (sites) the instantiation is launched with; blocks
// per SM requested so that the register budget leaves room for several
// blocks in flight.
// Block-wide parallel cyclic reduction (Hockney, J. ACM 12:95-113, 1965;
// Hockney & Jesshope, "Parallel Computers 2", 1988, sec. 5.4) of every
// filament's tridiagonal system of the block at once, for the fast
// integrator's blocks of long filaments: the rows laid out as solve_tridiag
// takes them (row i of a filament at slot first + i: lower coefficient in
// a[slot - 1], diagonal b, upper c, right-hand side d).  Each row thread
// eliminates the unknowns s rows away on both sides (s = 1, 2, 4, ... below
// max_rows), exchanging rows through the same arrays; a coupling that
// reaches past its filament's rows is zero at every step, so it is skipped.
// Every thread of the block calls it (max_rows is uniform); the solution
// ends in d.  O(log n) steps instead of the O(n) sequential elimination,
// with other rounding (the exact integrator keeps the reference's Thomas).
__device__ __forceinline__ void pcr_block(double *a, double *b, double *c, double *d, bool row,
                                          int t, int first, int last, int max_rows) {
  double lo = 0.0, dg = 1.0, up = 0.0, rhs = 0.0;
  if (row) {
    lo = t > first ? a[t - 1] : 0.0;
    dg = b[t];
    up = t < last ? c[t] : 0.0;
    rhs = d[t];
  }
  for (int s = 1; s < max_rows; s <<= 1) {
    __syncthreads();  // every read of the previous values is done
    if (row) {
      a[t] = lo;
      b[t] = dg;
      c[t] = up;
      d[t] = rhs;
    }
    __syncthreads();
    if (row) {
      const bool has_m = t - s >= first, has_p = t + s <= last;
      double al = 0.0, ga = 0.0, ndg = dg, nrhs = rhs, nlo = 0.0, nup = 0.0;
      if (has_m) {
        al = -lo * recip_nr(b[t - s]);
        ndg = fma(al, c[t - s], ndg);
        nrhs = fma(al, d[t - s], nrhs);
        nlo = al * a[t - s];
      }
      if (has_p) {
        ga = -up * recip_nr(b[t + s]);
        ndg = fma(ga, a[t + s], ndg);
        nrhs = fma(ga, d[t + s], nrhs);
        nup = ga * c[t + s];
      }
      lo = nlo;
      up = nup;
      dg = ndg;
      rhs = nrhs;
    }
  }
  __syncthreads();
  if (row) d[t] = rhs * recip_nr(dg);
}

// Rows of the longest system (bonds of the longest filament) above which the
// fast 256- and 512-site integrators solve by pcr_block instead of Thomas
// lanes.
constexpr int kPcrMinRows = 32;

template <int MAXC, bool FAST>
struct IntegrateBounds {
  // The exact variant spills below 96 registers; the fast one fits 80, which
  // also holds 4 blocks of 192 sites per SM (2 waves of 17-filament blocks
  // for 20,000 11-site filaments on 148 SMs).
  static constexpr int min_blocks =
      MAXC <= 128 ? (FAST ? 6 : 5) : MAXC <= 192 ? (FAST ? 4 : 3) : MAXC <= 256 ? 2 : 1;
};

// FUSE (fast mixed step only): each bond evaluates its own pairs
// (bond_pair_eval_sum) instead of summing the pair stage's slots.
// FIXC: launched with exactly MAXC threads, so every shared-memory offset is
// a compile-time constant.
template <int ND, int PREC, bool FAST, int MAXC, bool FUSE = false, bool FIXC = false>
__global__ void __launch_bounds__(MAXC, IntegrateBounds<MAXC, FAST>::min_blocks)
    k_integrate(SysConst k, DevState d, int midstep, int rbuf, int interaction,
                int capture) {
  extern __shared__ double smem[];
  const int C = FIXC ? MAXC : (int)blockDim.x;
  double *su = smem;            // site orientations    3C
  double *stn = su + 3 * C;     // tangents             3C
  double *sfr = stn + 3 * C;    // random forces; bond torques in P0-P1  3C
  double *sbF = sfr + 3 * C;    // bond forces, then gamma^-1 F          3C
  double *scos = sbF + 3 * C;   // cos(theta)           C
  double *sT = scos + C;        // rhs / tensions       C
  double *sa = sT + C;          // lower diagonal       C
  double *sb = sa + C;          // diagonal             C
  double *sc = sb + C;          // upper diagonal       C
  double *skeff = sc + C;       // k_eff                C
  double *srp = skeff + C;      // full step: prefetched previous positions 3C
  double *sfp = srp + 3 * C;    // full step: prefetched projected noise     3C
  // New positions (P5 on) take the slots of the previous positions: each
  // thread reads its own previous position before it writes its new one.
  double *sr = srp;             // positions            3C
  // Midstep random forces (P2), read by the projection rows only, before
  // the determinants are written over them.
  double *sfn = sfp;            // 3C
  // The metric determinants (P3): in a midstep in the prefetch area, which
  // only full steps use, so that they are computed alongside the
  // random-force solve; in a full step in the Thomas arrays (sT, sa, sb,
  // sc), free between the two solves' uses.
  double *sdt = midstep ? srp : sT;  // det_t     2C
  double *sdb = sdt + 2 * C;         // det_b     2C
  double *sdz = sfp + 3 * C;    // full step: prefetched rebuild origin (3C), tracker (C)
  int *sflag = (int *)(sdz + 4 * C);            // C/2 renormalisation flags
  FilConst *sfil = (FilConst *)(sflag + C / 2); // the block's filaments

#define V(arr, slot, comp) arr[(comp) * C + (slot)]

  const int blk = blockIdx.x;
  const int t = threadIdx.x;
  // Without a pair stage in between (fused pairs, or no interactions) the
  // kernel before this one may be the previous integrator step, whose
  // writes every load below reads: wait for it first.
  if (FUSE || !interaction) grid_dep_sync();
  // A rebuild of this step whose list outgrew its segment stops the step
  // before its first store (uniform over the grid: nothing in this kernel
  // sets that bit), so the host can grow the list and redo the step.
  const bool overflowed = (*d.status & ST_LIST_OVERFLOW) != 0u;
  const unsigned long long mcount = *d.mcount;
  const int un = d.blk_uni_n;
  int s0, count, f0, nfb;
  if (un > 0) {  // equal filaments: the block's range without a table load
    f0 = blk * d.blk_uni_fpb;
    nfb = min(d.blk_uni_fpb, d.nf - f0);
    s0 = f0 * un;
    count = nfb * un;
  } else {
    s0 = d.blk_site0[blk];
    count = d.blk_ns[blk];
    f0 = d.blk_f0[blk];
    nfb = d.blk_nf[blk];
  }
  __shared__ double s_hinv[9];  // the block's system (blocks never mix systems)
  __shared__ uint32_t s_seed;
  // Every global load the step needs is issued here, before the first
  // barrier: the filament constants, the renormalisation state and the
  // block's system constants, below the site state.
  int pre_sw = 0, pre_nn = 0;
  if (t < nfb) {
    sfil[t] = d.fil[f0 + t];
    sflag[t] = 0;
    pre_sw = d.f_switch[f0 + t];
    pre_nn = d.f_nnorm[f0 + t];
  }
  if (t < 10) {
    const ReplicaConst &Rb = d.rep[d.nrep == 1 ? 0 : d.fil[f0].rep];
    if (t < 9) s_hinv[t] = Rb.hinv[t];
    else s_seed = Rb.seed;
  }
  const bool active = t < count;
  const int g = s0 + t;
  // The site's place in its filament comes from site_jn, so every load of
  // P0 is issued here, alongside the staging of the filament constants,
  // rather than after the barrier.
  int f = 0, lf = 0, jn = 0;
  if (active && un > 0) {
    lf = t / un;
    jn = (t - lf * un) | un << 16;
    f = f0 + lf;
  } else if (active) {
    f = d.site_fil[g];
    jn = d.site_jn[g];
    lf = f - f0;
  }
  const int n = active ? jn >> 16 : 0;
  const int j = active ? jn & 0xffff : -1;
  const int base = t - j;            // slot of the filament's first site
  const int b = g - f;               // this thread's bond (valid when j < n-1)
  const bool has_bond = active && j < n - 1;

  // ---- P0: positions, orientations, bond forces --------------------------
  double r[3] = {0, 0, 0}, u[3] = {0, 0, 0};
  double bF[3] = {0, 0, 0}, bT[3] = {0, 0, 0};
  int fsw = 0;  // the filament's renormalisation direction before this step
  if (active) {
    fsw = d.f_switch[f];
    r[0] = d.r[0][g];
    r[1] = d.r[1][g];
    r[2] = d.r[2][g];
    if (!midstep) {
      // The full step needs the midstep's positions and projected noise
      // later; fetch them now, in the background.
      for (int i = 0; i < ND; ++i) cp_async8(&V(srp, t, i), &d.rp[i][g]);
      if (k.stoch)
        for (int i = 0; i < ND; ++i) cp_async8(&V(sfp, t, i), &d.fr[i][g]);
      if (interaction) {  // the displacement tracker's inputs, read last
        for (int i = 0; i < ND; ++i) cp_async8(&V(sdz, t, i), &d.dz[i][g]);
        cp_async8(&V(sdz, t, 3), &d.dt[g]);
      }
      cp_async_commit();
    }
  }
  int e0 = 0, e1 = 0;  // the bond's pair slots
  if (has_bond) {
    // Site orientation = orientation of its bond as Bond::ReInit left it
    // (Mesh::UpdateSiteOrientations, src/mesh.cpp:168-173).
    u[0] = d.ub[0][b];
    u[1] = d.ub[1][b];
    u[2] = d.ub[2][b];
    if (!FUSE && interaction) {
      e0 = d.e_off[b];
      e1 = e0 + d.e_cnt[b];
    }
  }
  // Everything above is the previous integrator step's or older; the pair
  // stage just before this kernel writes the bond slots read below.
  grid_dep_sync();
  if (overflowed) {  // uniform over the grid
    cp_async_wait_all();  // no copy into this block's shared memory outlives it
    return;
  }
  if (has_bond && interaction) {
    if (FUSE)
      bond_pair_eval_sum<ND>(k, d, d.rep[d.nrep == 1 ? 0 : d.fil[f].rep].hf, rbuf, b, bF, bT);
    else
      bond_pair_sum<ND, PREC>(d, b, e0, e1, bF, bT);
  }
  if (active && midstep) {  // Mesh::UpdatePrevPositions (src/mesh.cpp:175-182)
    d.rp[0][g] = r[0];
    d.rp[1][g] = r[1];
    d.rp[2][g] = r[2];
  }
  if (has_bond) {
    for (int i = 0; i < 3; ++i) {
      V(su, t, i) = u[i];
      V(sbF, t, i) = bF[i];
      V(sfr, t, i) = bT[i];
    }
  }
  __syncthreads();  // the staged filament constants and the bond values
  const FilConst &fc = sfil[active ? lf : 0];  // read from shared memory on use
  // Fast 256-site blocks with a long filament solve by parallel cyclic
  // reduction (uniform over the block).
  int max_rows = 0;
  if (FAST && MAXC > 128)
    for (int q = 0; q < nfb; ++q) max_rows = max(max_rows, sfil[q].n - 1);
  const bool pcr = FAST && MAXC > 128 && max_rows > kPcrMinRows;
  // Sequential solves: the exact step keeps the reference's Thomas order on
  // one lane per filament; the fast step solves from both ends on lanes
  // 2q, 2q+1.
  auto solve_rows = [&](int lane_t) {
    if (FAST) {
      if (lane_t < 2 * nfb) {
        const FilConst &f = sfil[lane_t >> 1];
        const int fb0 = f.site0 - s0;
        thomas_twisted(sa + fb0, sb + fb0, sc + fb0, sT + fb0, f.n - 1, (lane_t & 1) == 0);
      }
    } else if (lane_t < nfb) {
      const int fb0 = sfil[lane_t].site0 - s0;
      solve_tridiag<FAST>(sa + fb0, sb + fb0, sc + fb0, sT + fb0, sfil[lane_t].n - 1);
    }
  };
  // Midstep determinants on warps the random-force solve leaves idle: lanes
  // from g_dt (forward) and g_db (backward), when three warp-aligned groups
  // fit in the block.
  const int g_dt = ((FAST ? 2 * nfb : nfb) + 31) & ~31;
  const int g_db = g_dt + ((nfb + 31) & ~31);
  const bool dets_early = g_db + nfb <= C;
  if (active && j == n - 1) {
    for (int i = 0; i < 3; ++i) u[i] = V(su, t - 1, i);
  }

  // ---- P1: ApplyInteractionForces (src/filament.cpp:992-1048) -------------
  double F[3] = {0.0, 0.0, 0.0};
  if (active) {
    const double mag = 0.5 * 0.0 * fc.l;  // driving_factor 0, from bond centre
    if (j >= 1) {  // this site is site i+1 of bond i = j-1
      double up[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
      double fb[3] = {V(sbF, t - 1, 0), V(sbF, t - 1, 1), V(sbF, t - 1, 2)};
      double tb[3] = {V(sfr, t - 1, 0), V(sfr, t - 1, 1), V(sfr, t - 1, 2)};
      double pt[3], sf[3];
      cross3(up, tb, pt);
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        pt[i] *= fc.linv;
        sf[i] = 0.5 * fb[i];
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) pt[i] *= -1;
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += sf[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += pt[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += mag * up[i];
    }
    if (j <= n - 2) {  // site i of bond i = j (bF/bT hold this bond)
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
#pragma unroll
      for (int i = 0; i < ND; ++i) F[i] += mag * u[i];
    }
  }
  // CalculateAngles (:430-437), CalculateTangents (:439-443, Site::CalcTangent)
  double tn[3] = {0, 0, 0};
  if (active) {
    if (j < n - 2) {
      double un[3] = {V(su, t + 1, 0), V(su, t + 1, 1), V(su, t + 1, 2)};
      scos[t] = dotn<ND>(u, un);
    }
    if (j == 0 || j == n - 1) {
      tn[0] = u[0];
      tn[1] = u[1];
      tn[2] = u[2];
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) tn[i] = V(su, t - 1, i) + u[i];
      normalize<ND, FAST>(tn);
    }
    for (int i = 0; i < 3; ++i) V(stn, t, i) = tn[i];
  }
  if (active && j == n - 1) {
    for (int i = 0; i < 3; ++i) V(su, t, i) = u[i];
  }
  // A noisy midstep writes its random forces to the prefetch area (unused in
  // midsteps), not over the bond torques P1 reads, and nothing before its
  // next barrier reads what P1 wrote: only other steps need a barrier here.
  if (!(midstep && k.stoch)) __syncthreads();

  // ---- P2: random forces, projection, previous positions -----------------
  double fr[3] = {0, 0, 0};
  if (midstep && k.stoch && FAST && !pcr) {
    // The mixed step draws, projects and applies its noise in FP32 (its
    // precision contract keeps only the tension solve, the bending forces
    // that feed it and the positions in FP64): the same Philox words, the
    // uniforms to 2^-24, the projection system solved from both ends in FP32
    // over the Thomas arrays' first halves, the projected force added in
    // FP64.
    float *ffn = reinterpret_cast<float *>(sfn);  // 3 x C floats
    float *fT = reinterpret_cast<float *>(sT), *fa = reinterpret_cast<float *>(sa);
    float *fb = reinterpret_cast<float *>(sb), *fcm = reinterpret_cast<float *>(sc);
    float frf[3] = {0.f, 0.f, 0.f};
    const float uf[3] = {(float)u[0], (float)u[1], (float)u[2]};
    if (active) {  // ConstructUnprojectedRandomForces (:518-548)
      uint32_t w[4];
      sc_host_philox4x32_10((uint32_t)j, (uint32_t)mcount, (uint32_t)(mcount >> 32), 0u,
                            s_seed, (uint32_t)fc.f_local, w);
      float xi[3] = {0.f, 0.f, 0.f}, tnf[3] = {0.f, 0.f, 0.f}, txi = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        xi[i] = centered_uniform_f(w[i]);
        tnf[i] = (float)tn[i];
        txi = fmaf(tnf[i], xi[i], txi);
      }
      const float sperp = (float)fc.sperp, dsp = (float)(fc.spar - fc.sperp);
#pragma unroll
      for (int i = 0; i < ND; ++i) frf[i] = fmaf(sperp, xi[i], dsp * txi * tnf[i]);
#pragma unroll
      for (int i = 0; i < ND; ++i) ffn[i * C + t] = frf[i];
    }
    __syncthreads();
    if (has_bond) {  // GeometricallyProjectRandomForces (:550-599)
      float rhs = 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) rhs = fmaf(ffn[i * C + t + 1] - frf[i], uf[i], rhs);
      fT[t] = rhs;
      fb[t] = 2.f;
      if (j > 0) {
        fcm[t - 1] = -(float)scos[t - 1];
        fa[t - 1] = -(float)scos[t - 1];
      }
    }
    __syncthreads();
    if (t < 2 * nfb) {
      const FilConst &f = sfil[t >> 1];
      const int fb0 = f.site0 - s0;
      thomas_twisted(fa + fb0, fb + fb0, fcm + fb0, fT + fb0, f.n - 1, (t & 1) == 0);
    }
    if (dets_early) {  // the determinants, on lanes of other warps meanwhile
      if (t >= g_dt && t - g_dt < nfb) det_forward(sdt, scos, sfil[t - g_dt], s0, t - g_dt);
      else if (t >= g_db && t - g_db < nfb) det_backward(sdb, scos, sfil[t - g_db], s0, t - g_db);
    }
    __syncthreads();
    if (active) {
      const float tt = j < n - 1 ? fT[t] : 0.f, tp = j > 0 ? fT[t - 1] : 0.f;
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        const float up = j > 0 ? (float)V(su, t - 1, i) : 0.f;
        fr[i] = (double)fmaf(tt, uf[i], fmaf(-tp, up, frf[i]));
      }
      d.fr[0][g] = fr[0];  // the projected noise, reused by the full step
      d.fr[1][g] = fr[1];
      d.fr[2][g] = fr[2];
    }
  } else if (midstep) {
    if (k.stoch) {
      if (active) {  // ConstructUnprojectedRandomForces (:518-548)
        uint32_t w[4];
        sc_host_philox4x32_10((uint32_t)j, (uint32_t)mcount, (uint32_t)(mcount >> 32), 0u,
                              s_seed, (uint32_t)fc.f_local, w);
        double xi[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
#pragma unroll
        for (int i = 0; i < ND; ++i)
          xi[i] = centered_uniform(w[i]);
        if (FAST) {
          // (t t^T) xi = (t . xi) t
          const double txi = dotn<ND>(tn, xi);
#pragma unroll
          for (int i = 0; i < ND; ++i) xt[i] = txi * tn[i];
        } else if (ND == 2) {
          xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1];
          xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0];
        } else {
          xt[0] = tn[0] * tn[0] * xi[0] + tn[0] * tn[1] * xi[1] +
                  tn[0] * tn[2] * xi[2];
          xt[1] = tn[1] * tn[1] * xi[1] + tn[0] * tn[1] * xi[0] +
                  tn[1] * tn[2] * xi[2];
          xt[2] = tn[2] * tn[2] * xi[2] + tn[0] * tn[2] * xi[0] +
                  tn[1] * tn[2] * xi[1];
        }
#pragma unroll
        for (int i = 0; i < ND; ++i)
          fr[i] = fc.sperp * xi[i] + (fc.spar - fc.sperp) * xt[i];
        for (int i = 0; i < 3; ++i) V(sfn, t, i) = fr[i];
      }
      __syncthreads();
      // GeometricallyProjectRandomForces (:550-599)
      if (has_bond) {
        double tmp[3];
#pragma unroll
        for (int i = 0; i < ND; ++i) tmp[i] = V(sfn, t + 1, i) - fr[i];
        sT[t] = dotn<ND>(tmp, u);
        sb[t] = 2;
        if (j > 0) {
          sc[t - 1] = -scos[t - 1];
          sa[t - 1] = -scos[t - 1];
        }
      }
      __syncthreads();
      if (pcr) {
        pcr_block(sa, sb, sc, sT, has_bond, t, base, base + n - 2, max_rows);
      } else {
        solve_rows(t);
        if (dets_early) {  // the determinants, on lanes of other warps meanwhile
          if (t >= g_dt && t - g_dt < nfb) det_forward(sdt, scos, sfil[t - g_dt], s0, t - g_dt);
          else if (t >= g_db && t - g_db < nfb) det_backward(sdb, scos, sfil[t - g_db], s0, t - g_db);
        }
      }
      __syncthreads();
      if (active) {
        double fp[3];
        if (j == 0) {
#pragma unroll
          for (int i = 0; i < ND; ++i) fp[i] = fr[i] + sT[t] * u[i];
        } else if (j == n - 1) {
#pragma unroll
          for (int i = 0; i < ND; ++i) fp[i] = fr[i] - sT[t - 1] * V(su, t - 1, i);
        } else {
#pragma unroll
          for (int i = 0; i < ND; ++i)
            fp[i] = fr[i] + sT[t] * u[i] - sT[t - 1] * V(su, t - 1, i);
        }
#pragma unroll
        for (int i = 0; i < ND; ++i) fr[i] = fp[i];
        d.fr[0][g] = fr[0];  // the projected noise, reused by the full step
        d.fr[1][g] = fr[1];
        d.fr[2][g] = fr[2];
      }
    }
  } else if (active) {
    cp_async_wait_all();
    if (k.stoch)
      for (int i = 0; i < ND; ++i) fr[i] = V(sfp, t, i);
  }
  // AddRandomForces (:601-606)
  if (active && k.stoch) {
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fr[i];
  }

  // ---- P3: bending and metric forces (:608-776) ---------------------------
  // (The determinants do not share memory with the projection's solution,
  // which every thread has just read.)
  if (!(dets_early && midstep && k.stoch && !pcr)) {
    if (t < nfb) det_forward(sdt, scos, sfil[t], s0, t);
    else if (t >= C / 2 && t - C / 2 < nfb) det_backward(sdb, scos, sfil[t - C / 2], s0, t - C / 2);
    __syncthreads();
  }
  if (!FAST && active && j < n - 2) {
    const int dbase = base + lf;
    const double det_g = sdt[dbase + n - 1];
    double ginv = scos[t] * sdt[dbase + j] * sdb[dbase + j + 3] / det_g;
    skeff[t] = (fc.kappa + fc.l * ginv) / fc.l2;
  }
  if (!FAST) __syncthreads();
  if (active && FAST) {
    // Each site forms the k_eff of the (up to) three joints its stencil
    // uses from the determinants and cosines, instead of reading them from
    // a barrier later.
    const int dbase = base + lf;
    const double rdet = recip_nr(sdt[dbase + n - 1]), rl2 = recip_nr(fc.l2);
    auto keff_at = [&](int jj) {
      const double ginv = scos[base + jj] * sdt[dbase + jj] * sdb[dbase + jj + 3] * rdet;
      return (fc.kappa + fc.l * ginv) * rl2;
    };
    // (I - u2 u2^T) u1 = u1 - (u1 . u2) u2 with the cosines of
    // CalculateAngles: the reference's three stencil terms in vector form.
    double fs[3] = {0, 0, 0};
    const int kk = j;
    if (kk > 1) {
      const double ke = keff_at(j - 2), c = scos[t - 2];
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] += ke * (V(su, t - 2, i) - c * V(su, t - 1, i));
    }
    if (kk > 0 && kk < n - 1) {
      const double ke = keff_at(j - 1), c = scos[t - 1];
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        const double um = V(su, t - 1, i);
        fs[i] += ke * ((u[i] - c * um) - (um - c * u[i]));
      }
    }
    if (kk < n - 2) {
      const double ke = keff_at(j), c = scos[t];
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] -= ke * (V(su, t + 1, i) - c * u[i]);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
  } else if (active) {
    double fs[3] = {0, 0, 0};
    const int kk = j;
    if (ND == 2) {
      if (kk > 1) {
        double u1[3] = {V(su, t - 2, 0), V(su, t - 2, 1), 0};
        double u2[3] = {V(su, t - 1, 0), V(su, t - 1, 1), 0};
        double ke = skeff[t - 2];
        fs[0] += ke * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]);
        fs[1] += ke * ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]);
      }
      if (kk > 0 && kk < n - 1) {
        double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), 0};
        double u2[3] = {u[0], u[1], 0};
        double ke = skeff[t - 1];
        fs[0] += ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1]));
        fs[1] += ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0] -
                       ((1 - u2[1] * u2[1]) * u1[1] - u2[0] * u2[1] * u1[0]));
      }
      if (kk < n - 2) {
        double u1[3] = {u[0], u[1], 0};
        double u2[3] = {V(su, t + 1, 0), V(su, t + 1, 1), 0};
        double ke = skeff[t];
        fs[0] -= ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1]);
        fs[1] -= ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[0] * u1[1] * u2[0]);
      }
    } else {
      if (kk > 1) {
        double u1[3] = {V(su, t - 2, 0), V(su, t - 2, 1), V(su, t - 2, 2)};
        double u2[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
        double ke = skeff[t - 2];
        fs[0] += ke * ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                       u2[0] * u2[2] * u1[2]);
        fs[1] += ke * ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                       u2[1] * u2[2] * u1[2]);
        fs[2] += ke * ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                       u2[2] * u2[1] * u1[1]);
      }
      if (kk > 0 && kk < n - 1) {
        double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
        const double *u2 = u;
        double ke = skeff[t - 1];
        fs[0] += ke * ((1 - u1[0] * u1[0]) * u2[0] - u1[0] * u1[1] * u2[1] -
                       u1[0] * u1[2] * u2[2] -
                       ((1 - u2[0] * u2[0]) * u1[0] - u2[0] * u2[1] * u1[1] -
                        u2[0] * u2[2] * u1[2]));
        fs[1] += ke * ((1 - u1[1] * u1[1]) * u2[1] - u1[1] * u1[0] * u2[0] -
                       u1[1] * u1[2] * u2[2] -
                       ((1 - u2[1] * u2[1]) * u1[1] - u2[1] * u2[0] * u1[0] -
                        u2[1] * u2[2] * u1[2]));
        fs[2] += ke * ((1 - u1[2] * u1[2]) * u2[2] - u1[2] * u1[0] * u2[0] -
                       u1[2] * u1[1] * u2[1] -
                       ((1 - u2[2] * u2[2]) * u1[2] - u2[2] * u2[0] * u1[0] -
                        u2[1] * u2[2] * u1[1]));
      }
      if (kk < n - 2) {
        const double *u1 = u;
        double u2[3] = {V(su, t + 1, 0), V(su, t + 1, 1), V(su, t + 1, 2)};
        double ke = skeff[t];
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

  // ---- P4: tensions (:778-838) --------------------------------------------
  // gamma^-1 = (1/gpar) t t + (1/gperp)(I - t t); the reciprocals are the
  // reference's own quotients 1.0 / friction, computed once per filament.
  auto gam = [&](int a, int c) -> double {
    return fc.igpar * (tn[a] * tn[c]) + fc.igperp * ((a == c ? 1 : 0) - tn[a] * tn[c]);
  };
  // FAST: gamma^-1 F = F / g_perp + (1/g_par - 1/g_perp) (t . F) t
  auto gamF = [&](int i, const double *Fv, double tF) -> double {
    return fc.igperp * Fv[i] + fc.dgam * tF * tn[i];
  };
  if (active) {
    // gamma^-1 F of this site: "temp_a" of row j and "temp_b" of row j-1.
    const double tF = FAST ? dotn<ND>(tn, F) : 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double v;
      if (FAST) {
        v = gamF(i, F, tF);
      } else {
        v = gam(i, 0) * F[0] + gam(i, 1) * F[1];
        if (ND == 3) v += gam(i, 2) * F[2];
      }
      V(sbF, t, i) = v;
    }
  }
  __syncthreads();
  if (has_bond) {
    double fdiff[3];
#pragma unroll
    for (int i = 0; i < ND; ++i) fdiff[i] = V(sbF, t + 1, i) - V(sbF, t, i);
    sT[t] = dotn<ND>(u, fdiff);
    double tn2[3] = {V(stn, t + 1, 0), V(stn, t + 1, 1), V(stn, t + 1, 2)};
    double d1 = dotn<ND>(tn, u);
    double d2 = dotn<ND>(tn2, u);
    sb[t] = fc.two_igperp + fc.dgam * (d1 * d1 + d2 * d2);
    if (j > 0) {
      double u1[3] = {V(su, t - 1, 0), V(su, t - 1, 1), V(su, t - 1, 2)};
      double hu = fc.m1_igperp * dotn<ND>(u, u1) -
                  fc.dgam * (dotn<ND>(tn, u1) * dotn<ND>(tn, u));
      sc[t - 1] = hu;
      sa[t - 1] = hu;
    }
  }
  __syncthreads();
  if (pcr) pcr_block(sa, sb, sc, sT, has_bond, t, base, base + n - 2, max_rows);
  else solve_rows(t);
  __syncthreads();

  // ---- P5: UpdateSitePositions (:840-927), CheckBondLengths (:934-951) ----
  if (active) {
    double fs[3];
    if (j == 0) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = sT[t] * u[i];
    } else if (j == n - 1) {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = -sT[t - 1] * V(su, t - 1, i);
    } else {
#pragma unroll
      for (int i = 0; i < ND; ++i) fs[i] = sT[t] * u[i] - sT[t - 1] * V(su, t - 1, i);
    }
#pragma unroll
    for (int i = 0; i < ND; ++i) F[i] += fs[i];
    const double dl = (midstep ? 0.5 * k.delta : k.delta);
    double rp[3] = {r[0], r[1], r[2]};  // midstep: the previous positions are these
    if (!midstep)
      for (int i = 0; i < ND; ++i) rp[i] = V(srp, t, i);
    const double tF = FAST ? dotn<ND>(tn, F) : 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double ft;
      if (FAST) {
        ft = gamF(i, F, tF);
      } else {
        ft = gam(i, 0) * F[0] + gam(i, 1) * F[1];
        if (ND == 3) ft += gam(i, 2) * F[2];
      }
      r[i] = rp[i] + dl * ft;
    }
    for (int i = 0; i < 3; ++i) V(sr, t, i) = r[i];
  }
  __syncthreads();
  double rd[3] = {0, 0, 0}, um = 0.0;
  if (has_bond) {
#pragma unroll
    for (int i = 0; i < ND; ++i) rd[i] = V(sr, t + 1, i) - r[i];
    um = normalize<ND, FAST>(rd);
#pragma unroll
    for (int i = 0; i < ND; ++i) V(su, t, i) = rd[i];
  }
  bool stretched = false;
  if (active && j >= 1) {
    double a = 0.0;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double temp = r[i] - V(sr, t - 1, i);
      a += temp * temp;
    }
    if (FAST) {
      // |l - |dr|| / l > 1e-3 without the root and the quotient
      const double lo = fc.l * (1.0 - 1e-3), hi = fc.l * (1.0 + 1e-3);
      stretched = a < lo * lo || a > hi * hi;
    } else {
      a = sqrt(a);
      double err = dabs(fc.l - a) / fc.l;
      stretched = err > 1e-3;
    }
    if (stretched) sflag[lf] = 1;
  }
  // Positions change below only in a block with a filament to renormalise.
  __syncthreads_or(stretched);
  if (t < nfb) {
    const int fg = f0 + t;
    int sw = pre_sw, nnorm = pre_nn;
    if (sflag[t]) {
      sw = !sw;
      nnorm = 0;
    }
    nnorm++;
    d.f_switch[fg] = sw;
    d.f_nnorm[fg] = nnorm;
  }
  // The renormalised filament is rebuilt from one end along the bond
  // orientations just computed: from its first site when the switch turns
  // on, else from its last.  Every site runs the chain from that end itself
  // (the same operations in the same order as one sweep over the filament),
  // keeping its own position and its bond's far end, so no site waits for
  // another's result.
  const bool renorm = active && sflag[lf] != 0;
  double rnext[3] = {0, 0, 0};
  if (renorm) {
    const double l = fc.l;
    if (!fsw) {
      double a[3] = {V(sr, base, 0), V(sr, base, 1), V(sr, base, 2)};
      for (int jj = 1; jj <= j; ++jj)
#pragma unroll
        for (int i = 0; i < ND; ++i) a[i] = a[i] + l * V(su, base + jj - 1, i);
      r[0] = a[0];
      r[1] = a[1];
      r[2] = a[2];
      if (j < n - 1) {
        rnext[0] = a[0];
        rnext[1] = a[1];
        rnext[2] = a[2];
#pragma unroll
        for (int i = 0; i < ND; ++i) rnext[i] = a[i] + l * V(su, t, i);
      }
    } else {
      double a[3] = {V(sr, base + n - 1, 0), V(sr, base + n - 1, 1), V(sr, base + n - 1, 2)};
      for (int jj = n - 1; jj > j; --jj) {
        rnext[0] = a[0];
        rnext[1] = a[1];
        rnext[2] = a[2];
#pragma unroll
        for (int i = 0; i < ND; ++i) a[i] = a[i] - l * V(su, base + jj - 1, i);
      }
      r[0] = a[0];
      r[1] = a[1];
      r[2] = a[2];
    }
  }

  // ---- P6: bond geometry (Mesh::UpdateBondPositions), state write-back ----
  double my_dr = 0.0;
  if (active) {
    if (has_bond) {
      // Bond::ReInit on the final sites.  Without renormalisation it repeats
      // the orientation just computed (same operands, same operations).
      double r2[3];
      for (int i = 0; i < 3; ++i) r2[i] = renorm ? rnext[i] : V(sr, t + 1, i);
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
        len = um;
      }
#pragma unroll
      for (int i = 0; i < ND; ++i) pos[i] = r[i] + 0.5 * o[i];
#pragma unroll
      for (int i = 0; i < ND; ++i) {
        s[i] = 0.0;
#pragma unroll
        for (int jj = 0; jj < ND; ++jj) s[i] += s_hinv[ND * i + jj] * pos[jj];
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
    bool bad = false;
#pragma unroll
    for (int i = 0; i < ND; ++i) bad |= !isfinite(r[i]);
    if (bad) atomicOr(d.status, ST_NAN);
    if (capture) {
      for (int i = 0; i < 3; ++i) d.cap_F[i][g] = F[i];
      if (has_bond) d.cap_T[b] = sT[t];
    }
    // Displacement tracking for the next query (Mesh::UpdateDrTot runs on
    // the filaments whose last update was a full step; each query adds the
    // squared displacement twice, src/mesh.cpp:538-541, src/object.cpp:
    // 282-292).
    if (!midstep && interaction) {
      double acc = V(sdz, t, 3);
      for (int twice = 0; twice < 2; ++twice)
#pragma unroll
        for (int i = 0; i < ND; ++i) {
          double dr = r[i] - V(sdz, t, i);
          acc += dr * dr;
        }
      d.dt[g] = acc;
      my_dr = acc;
    }
  }
  if (!midstep && interaction) {
    // Warp max, then one atomic per warp on the IEEE bits (non-negative),
    // with no barrier.
    double v = my_dr;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((t & 31) == 0 && v != 0.0) {
      if (!(v <= 1e300)) atomicOr(d.status, ST_NAN);
      atomicMax(&d.dr_max_bits[sfil[0].rep], (unsigned long long)__double_as_longlong(v));
    }
  }
#undef V
}


}  // namespace sc
