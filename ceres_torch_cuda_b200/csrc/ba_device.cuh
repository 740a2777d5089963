// Device helpers for the Schur bundle-adjustment kernels (sm_100a).
//
// Everything here is per-thread register math: the Snavely projection with
// its analytic Jacobian, the robust losses and the Ceres corrector, small
// symmetric inverses, and the warp/block reductions the kernels share.
#pragma once

#include <cuda_runtime.h>
#include <cuda/atomic>
#include <math.h>
#include <stdint.h>

#include "../../include/ceres_b200.h"

namespace cb200 {

constexpr double kEps64 = 2.220446049250313080847e-16;   // float64 machine epsilon
constexpr double kTiny64 = 2.2250738585072013831e-308;   // smallest normal float64
constexpr float kEps32 = 1.1920928955078125e-7f;          // float32 machine epsilon
constexpr int kRec = 24;                                   // Jacobian scalars per slot

template <typename T> struct Eps;
template <> struct Eps<double> { static __host__ __device__ __forceinline__ double v() { return kEps64; } };
template <> struct Eps<float> { static __host__ __device__ __forceinline__ double v() { return (double)kEps32; } };

// ------------------------------------------------------------------------------------
// Robust losses (ceres-torch losses.py:21-133): rho(s), rho'(s), rho''(s)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double softplus(double x) {
  // torch.nn.functional.softplus with beta 1 and threshold 20
  return x > 20.0 ? x : log1p(exp(x));
}

// The divisions of the formulas are written as products with one reciprocal each
// (a float64 division is a long instruction sequence on the critical path of the
// evaluator); the results differ from the quotient forms by an ulp or two.
__device__ inline void loss_base(int kind, double a, double b, double s, double& r0, double& r1, double& r2) {
  switch (kind) {
    case CERES_B200_LOSS_HUBER: {
      const double b2 = a * a;
      if (s <= b2) { r0 = s; r1 = 1.0; r2 = 0.0; }
      else {
        const double sq = sqrt(fmax(s, kTiny64));
        const double isq = 1.0 / sq;
        r0 = 2.0 * a * sq - b2;
        r1 = a * isq;
        r2 = -0.5 * a * isq / s;
      }
      return;
    }
    case CERES_B200_LOSS_SOFTLONE: {
      const double b2 = a * a;
      const double ib2 = 1.0 / b2;
      const double z = 1.0 + s * ib2;
      const double sz = sqrt(z);
      const double isz = 1.0 / sz;
      r0 = 2.0 * b2 * (sz - 1.0);
      r1 = isz;
      r2 = -0.5 * ib2 * isz * isz * isz;
      return;
    }
    case CERES_B200_LOSS_CAUCHY: {
      const double b2 = a * a;
      const double ib2 = 1.0 / b2;
      const double z = 1.0 + s * ib2;
      const double iz = 1.0 / z;
      r0 = b2 * log(z);
      r1 = iz;
      r2 = -ib2 * iz * iz;
      return;
    }
    case CERES_B200_LOSS_ARCTAN: {
      const double ia = 1.0 / a;
      const double z = s * ia;
      const double den = 1.0 + z * z;
      const double iden = 1.0 / den;
      r0 = a * atan(z);
      r1 = iden;
      r2 = -2.0 * z * ia * iden * iden;
      return;
    }
    case CERES_B200_LOSS_TOLERANT: {
      const double z = (s - a) / b;
      const double c = b * softplus(-a / b);
      r0 = b * softplus(z) - c;
      r1 = 1.0 / (1.0 + exp(-z));
      r2 = r1 * (1.0 - r1) / b;
      return;
    }
    case CERES_B200_LOSS_TUKEY: {
      const double a2 = a * a;
      const double ia2 = 1.0 / a2;
      const double z = s * ia2;
      const double inner = 1.0 - z;
      if (s <= a2) {
        r0 = (a2 * (1.0 / 3.0)) * (1.0 - inner * inner * inner);
        r1 = inner * inner;
        r2 = -2.0 * inner * ia2;
      } else {
        r0 = a2 * (1.0 / 3.0); r1 = 0.0; r2 = 0.0;
      }
      return;
    }
    default:
      r0 = s; r1 = 1.0; r2 = 0.0;
      return;
  }
}

struct LossSpec {
  int kind; double a, b, scale;
  int inner; double ia, ib, iscale;
};

__device__ __forceinline__ LossSpec loss_spec(const ceres_b200_ba_t& ba) {
  return LossSpec{ba.loss_kind, ba.loss_a, ba.loss_b, ba.loss_scale,
                  ba.inner_loss_kind, ba.inner_a, ba.inner_b, ba.inner_scale};
}

__device__ inline void loss_eval(const LossSpec& L, double s, double& r0, double& r1, double& r2) {
  if (L.inner >= 0) {  // ComposedLoss(outer, inner): losses.py:125-133
    double g0, g1, g2, f0, f1, f2;
    loss_base(L.inner, L.ia, L.ib, s, g0, g1, g2);
    g0 *= L.iscale; g1 *= L.iscale; g2 *= L.iscale;
    loss_base(L.kind, L.a, L.b, g0, f0, f1, f2);
    r0 = f0; r1 = f1 * g1; r2 = f2 * g1 * g1 + f1 * g2;
  } else {
    loss_base(L.kind, L.a, L.b, s, r0, r1, r2);
  }
  r0 *= L.scale; r1 *= L.scale; r2 *= L.scale;  // ScaledLoss: losses.py:113-122
}

// ------------------------------------------------------------------------------------
// Snavely reprojection with its analytic Jacobian
// ------------------------------------------------------------------------------------
// Residual r = f d (xp, yp) - obs with p = R(aa) X + t, xp = -p0/p2, yp = -p1/p2,
// d = 1 + r2 (k1 + k2 r2) (examples/simple_bundle_adjuster.py:73-79). The rotation
// goes through the unit quaternion of rotation.py:104-110 (small-angle branch
// k = 0.5 - theta^2/48 when theta <= eps), normalised (rotation.py:68-69), and
// applied as X + w uv + u x uv with uv = 2 u x X (rotation.py:211-214). The
// derivative follows the same chain, including the normalisation, so it equals
// what autograd produces on the reference (costs.py:31-44), up to rounding.
// Residual (float64) and Jacobian rows in J: float64, or float32 for the float32
// Jacobian store, whose entries carry float32 rounding anyway.
template <typename J>
struct ProjT {
  double r[2];
  J jc[2][9];
  J jp[2][3];
};
using Proj = ProjT<double>;

template <typename V>
__device__ __forceinline__ void cross3(const V a[3], const V b[3], V o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// The camera-only part of the projection: the unit quaternion (w, u) of the
// angle-axis aa and, for the Jacobian, its derivative dqn = d(w, u)/d(aa) (4 x 3),
// including the normalisation. It depends on the 3 rotation parameters alone, so
// the kernels compute it once per camera (k_camera_frames) and every observation of
// the camera reads it back.
struct CamRot {
  double w;
  double u[3];
  double dqn[4][3];
};

template <bool kJac>
__device__ __forceinline__ void camera_rotation(const double aa[3], CamRot& R) {
  const double th2 = aa[0] * aa[0] + aa[1] * aa[1] + aa[2] * aa[2];
  const double theta = sqrt(th2);
  const double half = theta * 0.5;
  const bool small = theta <= kEps64;
  double sh, ch;
  sincos(half, &sh, &ch);
  // one reciprocal per divisor, reused below (a float64 division is a long
  // instruction sequence; the products differ from the quotients by at most an ulp)
  const double inv_theta = small ? 1.0 : 1.0 / theta;
  const double k = small ? 0.5 - theta * theta * (1.0 / 48.0) : sh * inv_theta;
  double q[4] = {ch, k * aa[0], k * aa[1], k * aa[2]};
  double qn2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  double n = sqrt(qn2);
  const bool clamped = n < kTiny64;
  if (clamped) n = kTiny64;
  const double inv_n = 1.0 / n;
  R.w = q[0] * inv_n;
  R.u[0] = q[1] * inv_n;
  R.u[1] = q[2] * inv_n;
  R.u[2] = q[3] * inv_n;
  if (!kJac) return;

  // d q_raw / d aa  (4 x 3)
  double dth[3];
  if (theta > 0.0) {
    const double it = small ? 1.0 / theta : inv_theta;
    dth[0] = aa[0] * it; dth[1] = aa[1] * it; dth[2] = aa[2] * it;
  } else {
    dth[0] = dth[1] = dth[2] = 0.0;  // torch.linalg.norm's subgradient at 0
  }
  const double dk_dth = small ? -(2.0 * theta) * (1.0 / 48.0) : (ch * 0.5 * theta - sh) * (inv_theta * inv_theta);
  double dq[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    dq[0][j] = -sh * 0.5 * dth[j];
    const double dkj = dk_dth * dth[j];
#pragma unroll
    for (int i = 0; i < 3; ++i) dq[1 + i][j] = (i == j ? k : 0.0) + aa[i] * dkj;
  }
  // normalisation: dqn = (dq - qn (qn . dq)) / n
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    if (clamped) {
#pragma unroll
      for (int i = 0; i < 4; ++i) R.dqn[i][j] = dq[i][j] * inv_n;
    } else {
      const double qn_dot = (R.w * dq[0][j] + R.u[0] * dq[1][j] + R.u[1] * dq[2][j] + R.u[2] * dq[3][j]);
      R.dqn[0][j] = (dq[0][j] - R.w * qn_dot) * inv_n;
#pragma unroll
      for (int i = 0; i < 3; ++i) R.dqn[1 + i][j] = (dq[1 + i][j] - R.u[i] * qn_dot) * inv_n;
    }
  }
}

// The observation part: residual (and Jacobian) of point X seen by a camera with
// rotation R and parameters tail = cam[3..8] (translation, f, k1, k2). The residual
// is float64; the Jacobian is computed in J from the float64 intermediates.
template <bool kJac, typename J = double>
__device__ __forceinline__ void snavely_project(const CamRot& R, const double tail[6], const double X[3], double ox,
                                                double oy, ProjT<J>& o) {
  const double w = R.w;
  const double* u = R.u;
  double c1[3];
  cross3(u, X, c1);
  const double uv[3] = {c1[0] * 2.0, c1[1] * 2.0, c1[2] * 2.0};
  double c2[3];
  cross3(u, uv, c2);
  double p[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) p[i] = (X[i] + w * uv[i] + c2[i]) + tail[i];
  const double inv_p2 = 1.0 / p[2];
  const double xp = -p[0] * inv_p2;
  const double yp = -p[1] * inv_p2;
  const double r2 = xp * xp + yp * yp;
  const double k1 = tail[4], k2 = tail[5], f = tail[3];
  const double dist = 1.0 + r2 * (k1 + k2 * r2);
  const double fd = f * dist;
  o.r[0] = fd * xp - ox;
  o.r[1] = fd * yp - oy;
  if constexpr (kJac) {
    const J wj = (J)w;
    const J uj[3] = {(J)u[0], (J)u[1], (J)u[2]};
    const J Xj[3] = {(J)X[0], (J)X[1], (J)X[2]};
    const J uvj[3] = {(J)uv[0], (J)uv[1], (J)uv[2]};
    // dp/daa: d(X + w uv + u x uv) = dw uv + w duv + du x uv + u x duv, duv = 2 du x X
    J dpa[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const J du[3] = {(J)R.dqn[1][j], (J)R.dqn[2][j], (J)R.dqn[3][j]};
      J t1[3];
      cross3(du, Xj, t1);
      const J duv[3] = {(J)2 * t1[0], (J)2 * t1[1], (J)2 * t1[2]};
      J t2[3], t3[3];
      cross3(du, uvj, t2);
      cross3(uj, duv, t3);
      const J dw = (J)R.dqn[0][j];
#pragma unroll
      for (int i = 0; i < 3; ++i) dpa[i][j] = dw * uvj[i] + wj * duv[i] + t2[i] + t3[i];
    }
    // dp/dX = I + 2 w [u]x + 2 [u]x^2, [u]x^2 = u u^T - (u.u) I
    const J uu = uj[0] * uj[0] + uj[1] * uj[1] + uj[2] * uj[2];
    J M[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) M[i][j] = (J)2 * uj[i] * uj[j] + (i == j ? (J)1 - (J)2 * uu : (J)0);
    M[0][1] -= (J)2 * wj * uj[2]; M[0][2] += (J)2 * wj * uj[1];
    M[1][0] += (J)2 * wj * uj[2]; M[1][2] -= (J)2 * wj * uj[0];
    M[2][0] -= (J)2 * wj * uj[1]; M[2][1] += (J)2 * wj * uj[0];

    // projection
    const J ip = (J)inv_p2, xq = (J)xp, yq = (J)yp, r2q = (J)r2, fq = (J)f, k1q = (J)k1, k2q = (J)k2;
    const J distq = (J)dist;
    const J dxp[3] = {-ip, (J)0, -xq * ip};
    const J dyp[3] = {(J)0, -ip, -yq * ip};
    const J g = k1q + (J)2 * k2q * r2q;
    const J dd_dx = (J)2 * xq * g, dd_dy = (J)2 * yq * g;
    const J A00 = fq * (distq + xq * dd_dx), A01 = fq * xq * dd_dy;
    const J A10 = fq * yq * dd_dx, A11 = fq * (distq + yq * dd_dy);
    J Dp[2][3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      Dp[0][m] = A00 * dxp[m] + A01 * dyp[m];
      Dp[1][m] = A10 * dxp[m] + A11 * dyp[m];
    }
#pragma unroll
    for (int rrow = 0; rrow < 2; ++rrow) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        o.jc[rrow][j] = Dp[rrow][0] * dpa[0][j] + Dp[rrow][1] * dpa[1][j] + Dp[rrow][2] * dpa[2][j];
        o.jc[rrow][3 + j] = Dp[rrow][j];
        o.jp[rrow][j] = Dp[rrow][0] * M[0][j] + Dp[rrow][1] * M[1][j] + Dp[rrow][2] * M[2][j];
      }
    }
    o.jc[0][6] = distq * xq; o.jc[1][6] = distq * yq;
    o.jc[0][7] = fq * r2q * xq; o.jc[1][7] = fq * r2q * yq;
    o.jc[0][8] = fq * r2q * r2q * xq; o.jc[1][8] = fq * r2q * r2q * yq;
  }
}

template <bool kJac>
__device__ __forceinline__ void snavely(const double* __restrict__ cam, const double X[3], double ox, double oy,
                                        Proj& o) {
  const double aa[3] = {cam[0], cam[1], cam[2]};
  CamRot R;
  camera_rotation<kJac>(aa, R);
  const double tail[6] = {cam[3], cam[4], cam[5], cam[6], cam[7], cam[8]};
  snavely_project<kJac>(R, tail, X, ox, oy, o);
}

// Camera frame record: 24 float64 per camera, [0] w, [1..3] u, [4..15] dqn (row-major
// 4 x 3), [16..21] cam[3..8], [22..23] zero.
constexpr int kFrame = 24;

template <bool kJac>
__device__ __forceinline__ void frame_store(double* __restrict__ f, const CamRot& R, const double* __restrict__ cam) {
  f[0] = R.w; f[1] = R.u[0]; f[2] = R.u[1]; f[3] = R.u[2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) f[4 + 3 * i + j] = kJac ? R.dqn[i][j] : 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) f[16 + i] = cam[3 + i];
  f[22] = 0.0; f[23] = 0.0;
}

// Ceres corrector (losses.py:158-193) applied in place. Returns 0.5 rho0.
template <bool kJac, typename J = double>
__device__ __forceinline__ double robustify(const LossSpec& L, ProjT<J>& o, unsigned& err) {
  const double s = o.r[0] * o.r[0] + o.r[1] * o.r[1];
  double r0, r1, r2;
  loss_eval(L, s, r0, r1, r2);
  const double sqrt_rho1 = sqrt(fmax(r1, 0.0));
  double rscale = sqrt_rho1, alpha_s = 0.0;
  if (s > 0.0 && r2 > 0.0) {
    if (r1 <= 0.0) err |= CERES_B200_DEVERR_LOSS;
    // alpha = 1 - sqrt(1 + 2 s rho''/rho'); 1 - alpha is that square root
    const double root = sqrt(1.0 + 2.0 * s * r2 / r1);
    const double alpha = 1.0 - root;
    rscale = sqrt_rho1 / root;
    alpha_s = alpha / s;
  }
  if (kJac) {
    const J sq = (J)sqrt_rho1;
    if (alpha_s == 0.0) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
#pragma unroll
        for (int j = 0; j < 9; ++j) o.jc[i][j] *= sq;
#pragma unroll
        for (int j = 0; j < 3; ++j) o.jp[i][j] *= sq;
      }
    } else {
      const J as = (J)alpha_s, ra = (J)o.r[0], rb = (J)o.r[1];
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const J rTj = ra * o.jc[0][j] + rb * o.jc[1][j];
        o.jc[0][j] = sq * (o.jc[0][j] - as * ra * rTj);
        o.jc[1][j] = sq * (o.jc[1][j] - as * rb * rTj);
      }
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const J rTj = ra * o.jp[0][j] + rb * o.jp[1][j];
        o.jp[0][j] = sq * (o.jp[0][j] - as * ra * rTj);
        o.jp[1][j] = sq * (o.jp[1][j] - as * rb * rTj);
      }
    }
  }
  o.r[0] *= rscale;
  o.r[1] *= rscale;
  return 0.5 * r0;
}

// ------------------------------------------------------------------------------------
// Jacobian record I/O (24 scalars per slot)
// ------------------------------------------------------------------------------------
template <typename T> struct Rec { T v[kRec]; };

// 256-bit global loads (sm_100): a record is 3 (float32) or 6 (float64) aligned
// 32-byte sectors, one load each, half the load instructions and L1 wavefronts of
// 128-bit loads. The store must be 32-byte aligned (the entry points check it).
// kCross: through L2 only (data written by other CTAs of the same launch).
template <bool kCross = false>
__device__ __forceinline__ void ld256(const float* p, float* v) {
  if constexpr (kCross)
    asm volatile("ld.global.cg.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p) : "memory");
  else
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}
template <bool kCross = false>
__device__ __forceinline__ void ld256(const double* p, double* v) {
  if constexpr (kCross)
    asm volatile("ld.global.cg.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p) : "memory");
  else
    asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}

// A camera frame with 256-bit loads: 6 (with the rotation derivative) or 3 instead of
// 11 / 5 128-bit loads per observation; frames start on 32-byte boundaries (kFrame
// float64 per camera from a 256-byte aligned base).
template <bool kJac>
__device__ __forceinline__ void frame_load_wide(const double* __restrict__ f, CamRot& R, double tail[6]) {
  double a[4];
  ld256(f, a);
  R.w = a[0]; R.u[0] = a[1]; R.u[1] = a[2]; R.u[2] = a[3];
  if (kJac) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double b[4];
      ld256(f + 4 + 4 * k, b);
#pragma unroll
      for (int m = 0; m < 4; ++m) R.dqn[(4 * k + m) / 3][(4 * k + m) % 3] = b[m];
    }
  }
  double c[4], d[4];
  ld256(f + 16, c);
  ld256(f + 20, d);
  tail[0] = c[0]; tail[1] = c[1]; tail[2] = c[2]; tail[3] = c[3]; tail[4] = d[0]; tail[5] = d[1];
}

// 128-bit loads of a float32 record (6 per record). The camera-major gather of
// k_camera_reduce, whose lanes read scattered records, runs faster with these
// (0.43 instead of 0.50 ms on the 6.0M-observation problem).
__device__ __forceinline__ void load_rec128(const float* __restrict__ base, size_t slot, float v[kRec]) {
  const float4* p = reinterpret_cast<const float4*>(base + slot * kRec);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const float4 t = __ldg(p + i);
    v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
  }
}

template <bool kCross = false, typename T>
__device__ __forceinline__ void load_rec(const T* __restrict__ base, size_t slot, T v[kRec]) {
  constexpr int kPer = 32 / (int)sizeof(T);
#pragma unroll
  for (int i = 0; i < kRec / kPer; ++i) ld256<kCross>(base + slot * kRec + kPer * i, v + kPer * i);
}
// point rows only (the last 6 scalars)
__device__ __forceinline__ void load_rec_jp(const float* __restrict__ base, size_t slot, float v[6]) {
  const float2* p = reinterpret_cast<const float2*>(base + slot * kRec + 18);
#pragma unroll
  for (int i = 0; i < 3; ++i) { const float2 t = __ldg(p + i); v[2 * i] = t.x; v[2 * i + 1] = t.y; }
}
__device__ __forceinline__ void load_rec_jp(const double* __restrict__ base, size_t slot, double v[6]) {
  const double2* p = reinterpret_cast<const double2*>(base + slot * kRec + 18);
#pragma unroll
  for (int i = 0; i < 3; ++i) { const double2 t = __ldg(p + i); v[2 * i] = t.x; v[2 * i + 1] = t.y; }
}
__device__ __forceinline__ void st256(float* p, const float* v) {
  asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]),
               "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]) : "memory");
}
__device__ __forceinline__ void st256(double* p, const double* v) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
               : "memory");
}

// record layout: camera rows jc[0][0..8], jc[1][0..8], then point rows jp[0][0..2], jp[1][0..2]
template <typename T, typename J>
__device__ __forceinline__ void store_rec(T* __restrict__ base, size_t slot, const ProjT<J>& o) {
  T v[kRec];
#pragma unroll
  for (int j = 0; j < 9; ++j) { v[j] = (T)o.jc[0][j]; v[9 + j] = (T)o.jc[1][j]; }
#pragma unroll
  for (int j = 0; j < 3; ++j) { v[18 + j] = (T)o.jp[0][j]; v[21 + j] = (T)o.jp[1][j]; }
  constexpr int kPer = 32 / (int)sizeof(T);
#pragma unroll
  for (int i = 0; i < kRec / kPer; ++i) st256(base + slot * kRec + kPer * i, v + kPer * i);
}

// symmetric 3x3 stored as (00, 01, 02, 11, 12, 22)
template <typename T>
__device__ __forceinline__ void sym3_mul(const T m[6], const double x[3], double y[3]) {
  y[0] = (double)m[0] * x[0] + (double)m[1] * x[1] + (double)m[2] * x[2];
  y[1] = (double)m[1] * x[0] + (double)m[3] * x[1] + (double)m[4] * x[2];
  y[2] = (double)m[2] * x[0] + (double)m[4] * x[1] + (double)m[5] * x[2];
}

// Inverse of a symmetric 3x3 (float64). Cholesky when positive definite;
// otherwise the adjugate formula (an LU-equivalent solve for a nonsingular
// block, as torch.linalg.solve would give).
__device__ inline void sym3_inverse(const double a[6], double inv[6]) {
  const double l00sq = a[0];
  bool pd = l00sq > 0.0;
  if (pd) {
    const double l00 = sqrt(l00sq);
    const double l10 = a[1] / l00, l20 = a[2] / l00;
    const double l11sq = a[3] - l10 * l10;
    pd = l11sq > 0.0;
    if (pd) {
      const double l11 = sqrt(l11sq);
      const double l21 = (a[4] - l20 * l10) / l11;
      const double l22sq = a[5] - l20 * l20 - l21 * l21;
      pd = l22sq > 0.0;
      if (pd) {
        const double l22 = sqrt(l22sq);
        // L^-1 (lower)
        const double i00 = 1.0 / l00, i11 = 1.0 / l11, i22 = 1.0 / l22;
        const double i10 = -l10 * i00 * i11;
        const double i21 = -l21 * i11 * i22;
        const double i20 = -(l20 * i00 + l21 * i10) * i22;
        // A^-1 = L^-T L^-1
        inv[0] = i00 * i00 + i10 * i10 + i20 * i20;
        inv[1] = i10 * i11 + i20 * i21;
        inv[2] = i20 * i22;
        inv[3] = i11 * i11 + i21 * i21;
        inv[4] = i21 * i22;
        inv[5] = i22 * i22;
        return;
      }
    }
  }
  const double c00 = a[3] * a[5] - a[4] * a[4];
  const double c01 = a[2] * a[4] - a[1] * a[5];
  const double c02 = a[1] * a[4] - a[2] * a[3];
  const double c11 = a[0] * a[5] - a[2] * a[2];
  const double c12 = a[1] * a[2] - a[0] * a[4];
  const double c22 = a[0] * a[3] - a[1] * a[1];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  const double id = 1.0 / det;
  inv[0] = c00 * id; inv[1] = c01 * id; inv[2] = c02 * id;
  inv[3] = c11 * id; inv[4] = c12 * id; inv[5] = c22 * id;
}

// Inverse of a 9x9 block (float64, row-major, full storage). Cholesky when
// positive definite, Gauss-Jordan with partial pivoting otherwise
// (linear.py:1169-1174: cholesky, else a plain solve of the block).
__device__ inline void block9_inverse(double A[81], double inv[81]) {
  double L[81];
  bool pd = true;
#pragma unroll 1
  for (int j = 0; j < 9 && pd; ++j) {
    double d = A[j * 9 + j];
    for (int k = 0; k < j; ++k) d -= L[j * 9 + k] * L[j * 9 + k];
    if (!(d > 0.0)) { pd = false; break; }
    const double ljj = sqrt(d);
    L[j * 9 + j] = ljj;
    for (int i = j + 1; i < 9; ++i) {
      double s = A[i * 9 + j];
      for (int k = 0; k < j; ++k) s -= L[i * 9 + k] * L[j * 9 + k];
      L[i * 9 + j] = s / ljj;
    }
  }
  if (pd) {
    // solve L L^T X = I column by column
#pragma unroll 1
    for (int c = 0; c < 9; ++c) {
      double y[9];
      for (int i = 0; i < 9; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k) s -= L[i * 9 + k] * y[k];
        y[i] = s / L[i * 9 + i];
      }
      for (int i = 8; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < 9; ++k) s -= L[k * 9 + i] * inv[k * 9 + c];
        inv[i * 9 + c] = s / L[i * 9 + i];
      }
    }
    return;
  }
  // Gauss-Jordan with partial pivoting on [A | I]
  for (int i = 0; i < 81; ++i) inv[i] = (i % 10 == 0) ? 1.0 : 0.0;
#pragma unroll 1
  for (int c = 0; c < 9; ++c) {
    int piv = c;
    double best = fabs(A[c * 9 + c]);
    for (int r = c + 1; r < 9; ++r) {
      const double v = fabs(A[r * 9 + c]);
      if (v > best) { best = v; piv = r; }
    }
    if (piv != c) {
      for (int k = 0; k < 9; ++k) {
        double t = A[c * 9 + k]; A[c * 9 + k] = A[piv * 9 + k]; A[piv * 9 + k] = t;
        t = inv[c * 9 + k]; inv[c * 9 + k] = inv[piv * 9 + k]; inv[piv * 9 + k] = t;
      }
    }
    const double d = 1.0 / A[c * 9 + c];
    for (int k = 0; k < 9; ++k) { A[c * 9 + k] *= d; inv[c * 9 + k] *= d; }
    for (int r = 0; r < 9; ++r) {
      if (r == c) continue;
      const double fct = A[r * 9 + c];
      if (fct == 0.0) continue;
      for (int k = 0; k < 9; ++k) { A[r * 9 + k] -= fct * A[c * 9 + k]; inv[r * 9 + k] -= fct * inv[c * 9 + k]; }
    }
  }
}

// Slices in "snake" order: round r of the grid-stride walk runs forward on even
// rounds and backward on odd ones, so with slices sorted by length every warp
// gets a mix of long and short tracks.
// Balanced slice schedule: CTA b owns one slice of every round of gridDim.x slices
// (snake order over the CTAs, so the CTAs' totals agree to a few per cent although the
// slices are sorted by length) and its warps pull them in that order, longest first,
// from a shared-memory counter (zero when the CTA starts). Returns -1 when done.
__device__ __forceinline__ int next_cta_slice(int* counter, int num_slices) {
  int i = 0;
  if ((threadIdx.x & 31) == 0) i = atomicAdd(counter, 1);
  i = __shfl_sync(0xffffffffu, i, 0);
  const long long s = (long long)i * gridDim.x + ((i & 1) ? (int)gridDim.x - 1 - (int)blockIdx.x : (int)blockIdx.x);
  return s < num_slices ? (int)s : -1;
}

// Longest-first dynamic schedule over the whole grid: slices are sorted by length
// (descending), so warps taking them in index order from one global counter follow the
// LPT rule, and no CTA slot idles behind the slowest warp of its CTA. The counter is
// reset by the fold that follows (k_slice_fold). Returns -1 when no slice is left.
__device__ __forceinline__ int next_global_slice(unsigned* counter, int num_slices) {
  int i = 0;
  if ((threadIdx.x & 31) == 0) i = (int)atomicAdd(counter, 1u);
  i = __shfl_sync(0xffffffffu, i, 0);
  return i < num_slices ? i : -1;
}

__device__ __forceinline__ int snake_slice(int r, int gw, int nw) {
  return r * nw + ((r & 1) ? nw - 1 - gw : gw);
}

// ------------------------------------------------------------------------------------
// Reductions
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide reduction of NV values (sum, or max where is_max bit set). Result
// valid in thread 0. smem must hold NV * (blockDim.x / 32) doubles.
template <int NV>
__device__ __forceinline__ void block_reduce(double v[NV], unsigned is_max_mask, double* smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = ((is_max_mask >> i) & 1u) ? warp_max(v[i]) : warp_sum(v[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) smem[i * nw + wid] = v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double acc = smem[i * nw];
      for (int w = 1; w < nw; ++w) acc = ((is_max_mask >> i) & 1u) ? fmax(acc, smem[i * nw + w]) : acc + smem[i * nw + w];
      v[i] = acc;
    }
  }
  __syncthreads();
}

// Deterministic grid reduction: each CTA's thread 0 posts NV partials; the last CTA
// to arrive folds them (thread t takes partials t, t + blockDim, ...; then a fixed
// block reduction) and writes stats[out_idx[i]]. counter returns to zero afterwards.
// smem must hold NV * (blockDim.x / 32) doubles.
template <int NV>
__device__ __forceinline__ void grid_finish(const double v[NV], unsigned is_max_mask, double* partials,
                                            unsigned* counter, double* stats, const int out_idx[NV],
                                            double* smem) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partials[(size_t)blockIdx.x * NV + i] = v[i];
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      const double x = __ldcg(&partials[(size_t)b * NV + i]);
      acc[i] = ((is_max_mask >> i) & 1u) ? fmax(acc[i], x) : acc[i] + x;
    }
  }
  block_reduce<NV>(acc, is_max_mask, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) stats[out_idx[i]] = acc[i];
    *counter = 0u;
    __threadfence();
  }
}

// ------------------------------------------------------------------------------------
// Grid barrier for the cooperative persistent PCG. Every wait is bounded: after
// kSpinLimit polls the CTA records CERES_B200_DEVERR_BARRIER in *flag and the
// barrier reports failure so that all CTAs leave the kernel.
// ------------------------------------------------------------------------------------
constexpr unsigned kSpinLimit = 1u << 24;

struct GridBarrier {
  unsigned* count;
  unsigned* generation;
  unsigned* flag;
  unsigned limit = kSpinLimit;  // polls before the wait gives up
};

__device__ __forceinline__ bool grid_sync(const GridBarrier& gb) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    // the CTA's writes (ordered before thread 0 by the bar.sync) are released at device scope
    cuda::atomic_thread_fence(cuda::memory_order_release, cuda::thread_scope_device);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(*gb.generation);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(*gb.count);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> flg(*gb.flag);
    const unsigned my_gen = gen.load(cuda::memory_order_acquire);
    int good = 1;
    if (flg.load(cuda::memory_order_relaxed) != 0u) {
      good = 0;
    } else {
      const unsigned arrived = cnt.fetch_add(1u, cuda::memory_order_acq_rel);
      if (arrived == gridDim.x - 1) {
        cnt.store(0u, cuda::memory_order_relaxed);
        gen.fetch_add(1u, cuda::memory_order_release);
      } else {
        unsigned spins = 0;
        while (gen.load(cuda::memory_order_acquire) == my_gen) {
          if (flg.load(cuda::memory_order_relaxed) != 0u) { good = 0; break; }
          if (++spins > gb.limit) {
            flg.fetch_or(CERES_B200_DEVERR_BARRIER, cuda::memory_order_relaxed);
            good = 0;
            break;
          }
          if (spins > 64) __nanosleep(64);
        }
      }
    }
    cuda::atomic_thread_fence(cuda::memory_order_acquire, cuda::thread_scope_device);
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Loads of data another CTA wrote in this launch go around L1 (L1 is not
// coherent across SMs).
template <typename T> __device__ __forceinline__ T ld_cross(const T* p) { return __ldcg(p); }

}  // namespace cb200
