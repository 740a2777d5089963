// Batched bundle adjustment: many independent problems in one persistent launch.
//
// Every CTA pulls whole problems from a work counter and runs the complete
// Levenberg-Marquardt solve of one problem at a time: the same evaluation, Schur
// assembly, implicit-Schur PCG and step arithmetic as the single-problem kernels of
// ba_kernels.cu, at CTA scope (warps walk the problem's slices, __syncthreads instead
// of grid barriers), and the trust-region decisions of ceres-torch's solver.py:35-357
// (LM radius rule solver.py:805-820, step quality solver.py:823-861, convergence
// tests solver.py:320-336 and :1169-1175) on the device. There is no host round
// trip between iterations and no spin-wait anywhere: a CTA only synchronises with
// itself.
//
// Data written during the launch (Jacobian store, residuals, vectors) is read with
// plain loads, never through the read-only path.
#include <cstdio>

#include "ba_device.cuh"

using namespace cb200;

namespace {

constexpr int kBR = CERES_B200_BATCH_RESULT;
constexpr int kBT = CERES_B200_BATCH_TRACE;
constexpr int kMaxWarps = 16;
constexpr int kBatchStall = 20;  // float32 PCG: iterations without a 1% residual drop before it stops

__device__ __forceinline__ int tri9b(int j, int l) { return j * 9 - (j * (j - 1)) / 2 + (l - j); }

// Jacobian record loads through the coherent path (the store is rewritten in-launch).
__device__ __forceinline__ void rec_load(const float* base, size_t slot, float v[kRec]) {
  const float4* p = reinterpret_cast<const float4*>(base + slot * kRec);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const float4 t = p[i];
    v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
  }
}
__device__ __forceinline__ void rec_load(const double* base, size_t slot, double v[kRec]) {
  const double2* p = reinterpret_cast<const double2*>(base + slot * kRec);
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const double2 t = p[i];
    v[2 * i] = t.x; v[2 * i + 1] = t.y;
  }
}

// Reduce NV values over the CTA and hand the result to every thread.
template <int NV>
__device__ __forceinline__ void cta_allreduce(double v[NV], unsigned max_mask, double* red, double* bcast) {
  block_reduce<NV>(v, max_mask, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) bcast[i] = v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = bcast[i];
  __syncthreads();
}

struct Prob {
  int b;
  int nc, cam0;  // cameras [cam0, cam0 + nc)
  int ns, s0;    // slices [s0, s0 + ns); sorted points 32 * s0 ...
};

struct Smem {
  double* red;    // [8 * kMaxWarps]
  double* bcast;  // [8]
  void* ps;       // [9 * max_cameras] T: the PCG direction
  void* ys;       // [9 * max_cameras] T: the product accumulator
  double* y64;    // [9 * max_cameras]: float64 product accumulator (refinement)
};

// ------------------------------------------------------------------------------------
// camera frames of cams (nc x 9) into frames
// ------------------------------------------------------------------------------------
template <bool kJac>
__device__ void cta_frames(const double* cams, double* frames, int nc) {
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    const double* cam = cams + 9 * (size_t)c;
    const double aa[3] = {cam[0], cam[1], cam[2]};
    CamRot R;
    camera_rotation<kJac>(aa, R);
    frame_store<kJac>(frames + kFrame * (size_t)c, R, cam);
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------
// evaluation at B.cameras / B.points: residuals, Jacobian records, point sums, cost
// ------------------------------------------------------------------------------------
template <typename T>
__device__ double cta_evaluate(const ceres_b200_batch_t& B, const LossSpec& L, const Prob& P, const Smem& S,
                               unsigned& err) {
  cta_frames<true>(B.cameras + 9 * (size_t)P.cam0, B.frames + kFrame * (size_t)P.cam0, P.nc);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T* jac = reinterpret_cast<T*>(B.jac);
  const double* frames = B.frames + kFrame * (size_t)P.cam0;
  double cost = 0.0;
  for (int s = P.s0 + w; s < P.s0 + P.ns; s += nw) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s];
    const double X[3] = {B.points[3 * (size_t)q], B.points[3 * (size_t)q + 1], B.points[3 * (size_t)q + 2]};
    const bool pconst = B.pt_const[q] != 0;
    double W[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0};
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k + lane;
      const int c = B.slot_cam[slot];
      if (c < 0) continue;
      const double2 ob = reinterpret_cast<const double2*>(B.slot_obs)[slot];
      Proj o;
      CamRot R;
      double tail[6];
      frame_load<true>(frames + kFrame * (size_t)c, R, tail);
      snavely_project<true>(R, tail, X, ob.x, ob.y, o);
      cost += robustify<true>(L, o, err);
      reinterpret_cast<double2*>(B.res)[slot] = make_double2(o.r[0], o.r[1]);
      if (B.cam_const[P.cam0 + c]) {
#pragma unroll
        for (int j = 0; j < 9; ++j) o.jc[0][j] = o.jc[1][j] = 0.0;
      }
      if (pconst) {
#pragma unroll
        for (int j = 0; j < 3; ++j) o.jp[0][j] = o.jp[1][j] = 0.0;
      }
      store_rec(jac, slot, o);
      double a[3], bb[3];
#pragma unroll
      for (int m = 0; m < 3; ++m) { a[m] = (double)(T)o.jp[0][m]; bb[m] = (double)(T)o.jp[1][m]; }
      W[0] += a[0] * a[0] + bb[0] * bb[0];
      W[1] += a[0] * a[1] + bb[0] * bb[1];
      W[2] += a[0] * a[2] + bb[0] * bb[2];
      W[3] += a[1] * a[1] + bb[1] * bb[1];
      W[4] += a[1] * a[2] + bb[1] * bb[2];
      W[5] += a[2] * a[2] + bb[2] * bb[2];
#pragma unroll
      for (int m = 0; m < 3; ++m) g[m] += a[m] * o.r[0] + bb[m] * o.r[1];
    }
    double* pr = B.point_raw + 9 * (size_t)q;
#pragma unroll
    for (int i = 0; i < 6; ++i) pr[i] = W[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) pr[6 + i] = g[i];
  }
  double v[1] = {cost};
  cta_allreduce<1>(v, 0u, S.red, S.bcast);
  return v[0];
}

// ------------------------------------------------------------------------------------
// Schur assembly for a radius: point blocks, camera sums, camera finish.
// Returns the gradient stats {gmax, gsq} over point and camera columns.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cta_point_assemble(const ceres_b200_batch_t& B, const Prob& P, double inv_radius, double& gmax,
                                   double& gsq) {
  T* winv = reinterpret_cast<T*>(B.winv);
  const double mn = B.min_lm_diagonal, mx = B.max_lm_diagonal;
  const int q0 = 32 * P.s0, np = 32 * P.ns;
  for (int ql = threadIdx.x; ql < np; ql += blockDim.x) {
    const int q = q0 + ql;
    const double* pr = B.point_raw + 9 * (size_t)q;
    double W[6], g[3];
#pragma unroll
    for (int i = 0; i < 6; ++i) W[i] = pr[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] = pr[6 + i];
    double inv[6] = {0, 0, 0, 0, 0, 0};
    double wga[3] = {0, 0, 0};
    if (!B.pt_const[q]) {
      const int dg[3] = {0, 3, 5};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double col = B.jacobi_scaling ? W[dg[i]] : 1.0;
        W[dg[i]] += fmin(fmax(col, mn), mx) * inv_radius;
        gmax = fmax(gmax, fabs(g[i]));
        gsq += g[i] * g[i];
      }
      sym3_inverse(W, inv);
      const double ga[3] = {-g[0], -g[1], -g[2]};
      sym3_mul(inv, ga, wga);
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) winv[6 * (size_t)q + i] = (T)inv[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) B.winv_ga[3 * (size_t)q + i] = wga[i];
  }
}

// One of three passes over a camera's observations (a warp per camera); each pass
// keeps a third of the 72 float64 sums in registers: pass 0 the Schur-block rows 0-2,
// pass 1 rows 3-8, pass 2 the column sums, gradient and reduced rhs.
template <typename T, int kPass>
__device__ void warp_camera_pass(const ceres_b200_batch_t& B, int cg, int cl, double* acc_out) {
  constexpr int kN = kPass == 0 ? 24 : (kPass == 1 ? 21 : 27);
  constexpr int kOff = kPass == 0 ? 0 : (kPass == 1 ? 24 : 45);
  constexpr int j0 = kPass == 0 ? 0 : 3, j1 = kPass == 0 ? 3 : 9;
  const int lane = threadIdx.x & 31;
  const T* jac = reinterpret_cast<const T*>(B.jac);
  const T* winv = reinterpret_cast<const T*>(B.winv);
  double acc[kN];
#pragma unroll
  for (int i = 0; i < kN; ++i) acc[i] = 0.0;
  const int e0 = B.cam_offsets[cg], e1 = B.cam_offsets[cg + 1];
  for (int e = e0 + lane; e < e1; e += 32) {
    const int2 ent = reinterpret_cast<const int2*>(B.cam_entries)[e];
    const size_t slot = (size_t)ent.x;
    const int q = ent.y;
    T rv[kRec];
    rec_load(jac, slot, rv);
    double wi[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) wi[i] = (double)winv[6 * (size_t)q + i];
    double jp0[3], jp1[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) { jp0[m] = rv[18 + m]; jp1[m] = rv[21 + m]; }
    double P0[3], P1[3];
    sym3_mul(wi, jp0, P0);
    sym3_mul(wi, jp1, P1);
    if constexpr (kPass < 2) {
      const double B00 = P0[0] * jp0[0] + P0[1] * jp0[1] + P0[2] * jp0[2];
      const double B01 = P0[0] * jp1[0] + P0[1] * jp1[1] + P0[2] * jp1[2];
      const double B11 = P1[0] * jp1[0] + P1[1] * jp1[1] + P1[2] * jp1[2];
      const double M00 = 1.0 - B00, M01 = -B01, M11 = 1.0 - B11;
      double K0[9], K1[9];
#pragma unroll
      for (int l = 0; l < 9; ++l) {
        const double c0 = rv[l], c1 = rv[9 + l];
        K0[l] = M00 * c0 + M01 * c1;
        K1[l] = M01 * c0 + M11 * c1;
      }
#pragma unroll
      for (int j = j0; j < j1; ++j)
#pragma unroll
        for (int l = j; l < 9; ++l) acc[tri9b(j, l) - kOff] += (double)rv[j] * K0[l] + (double)rv[9 + j] * K1[l];
      if (B.has_duplicate_cameras) {
        // other observations of the same point in this camera: -Jc_i^T P_i Jp_k^T Jc_k
        const int sidx = q >> 5, ln = q & 31;
        const int len = B.slice_len[sidx];
        const size_t sb = (size_t)B.slice_base[sidx];
        for (int k = 0; k < len; ++k) {
          const size_t slot2 = sb + 32 * (size_t)k + ln;
          if (slot2 == slot || B.slot_cam[slot2] != cl) continue;
          T rk[kRec];
          rec_load(jac, slot2, rk);
          const double C00 = P0[0] * rk[18] + P0[1] * rk[19] + P0[2] * rk[20];
          const double C01 = P0[0] * rk[21] + P0[1] * rk[22] + P0[2] * rk[23];
          const double C10 = P1[0] * rk[18] + P1[1] * rk[19] + P1[2] * rk[20];
          const double C11 = P1[0] * rk[21] + P1[1] * rk[22] + P1[2] * rk[23];
#pragma unroll
          for (int j = j0; j < j1; ++j) {
            const double t0 = (double)rv[j] * C00 + (double)rv[9 + j] * C10;
            const double t1 = (double)rv[j] * C01 + (double)rv[9 + j] * C11;
#pragma unroll
            for (int l = j; l < 9; ++l) acc[tri9b(j, l) - kOff] -= t0 * (double)rk[l] + t1 * (double)rk[9 + l];
          }
        }
      }
    } else {
      const double2 r = reinterpret_cast<const double2*>(B.res)[slot];
      const double wg[3] = {B.winv_ga[3 * (size_t)q], B.winv_ga[3 * (size_t)q + 1], B.winv_ga[3 * (size_t)q + 2]};
      const double a0 = jp0[0] * wg[0] + jp0[1] * wg[1] + jp0[2] * wg[2];
      const double a1 = jp1[0] * wg[0] + jp1[1] * wg[1] + jp1[2] * wg[2];
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const double c0 = rv[j], c1 = rv[9 + j];
        acc[j] += c0 * c0 + c1 * c1;
        acc[9 + j] += c0 * r.x + c1 * r.y;
        acc[18 + j] += c0 * (r.x + a0) + c1 * (r.y + a1);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kN; ++i) {
    const double v = warp_sum(acc[i]);
    if (lane == 0) acc_out[kOff + i] = v;
  }
}

// The damping, rhs, gradient stats and preconditioner block of camera cg from its 72
// sums (the warp version of k_camera_finish).
template <typename T>
__device__ void warp_camera_finish(const ceres_b200_batch_t& B, int cg, double inv_radius, double& gmax,
                                   double& gsq) {
  constexpr unsigned kFull = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const double* sacc = B.cam_acc + (size_t)cg * 72;
  T* pre = reinterpret_cast<T*>(B.precond) + 81 * (size_t)cg;
  double* dc = B.cam_diag + 9 * (size_t)cg;
  double* rh = B.rhs + 9 * (size_t)cg;
  const double mn = B.min_lm_diagonal, mx = B.max_lm_diagonal;
  if (B.cam_const[cg]) {
    if (lane < 9) { dc[lane] = 0.0; rh[lane] = 0.0; }
    for (int i = lane; i < 81; i += 32) pre[i] = (T)((i % 10 == 0) ? 1.0 : 0.0);
    return;
  }
  const int i = lane < 9 ? lane : 8;
  const double col = B.jacobi_scaling ? sacc[45 + i] : 1.0;
  const double di = fmin(fmax(col, mn), mx) * inv_radius;
  if (lane < 9) {
    dc[i] = di;
    rh[i] = -sacc[63 + i];
    const double gi = sacc[54 + i];
    gmax = fmax(gmax, fabs(gi));
    gsq += gi * gi;
  }
  double a[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) a[l] = sacc[l < i ? tri9b(l, i) : tri9b(i, l)] + (l == i ? di : 0.0);
  if (B.preconditioner == CERES_B200_PRECOND_SCHUR_JACOBI) {
    double Lr[9];
    bool pd = true;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      double Lj[9];
#pragma unroll
      for (int k = 0; k < j; ++k) Lj[k] = __shfl_sync(kFull, Lr[k], j);
      double d = __shfl_sync(kFull, a[j], j);
#pragma unroll
      for (int k = 0; k < j; ++k) d -= Lj[k] * Lj[k];
      if (!(d > 0.0)) { pd = false; break; }
      const double ljj = sqrt(d);
      double sj = a[j];
#pragma unroll
      for (int k = 0; k < j; ++k) sj -= Lr[k] * Lj[k];
      Lr[j] = (i == j) ? ljj : sj / ljj;
    }
    if (pd) {
      double Lf[45];
#pragma unroll
      for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int k = 0; k <= r; ++k) Lf[r * (r + 1) / 2 + k] = __shfl_sync(kFull, Lr[k], r);
      double y[9], x[9];
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        double sv = (r == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < r; ++k) sv -= Lf[r * (r + 1) / 2 + k] * y[k];
        y[r] = sv / Lf[r * (r + 1) / 2 + r];
      }
#pragma unroll
      for (int r = 8; r >= 0; --r) {
        double sv = y[r];
#pragma unroll
        for (int k = r + 1; k < 9; ++k) sv -= Lf[k * (k + 1) / 2 + r] * x[k];
        x[r] = sv / Lf[r * (r + 1) / 2 + r];
      }
      if (lane < 9) {
#pragma unroll
        for (int r = 0; r < 9; ++r) pre[r * 9 + lane] = (T)x[r];
      }
    } else if (lane == 0) {
      double Sm[81], inv[81];
      for (int j = 0; j < 9; ++j) {
        const double dj = fmin(fmax(B.jacobi_scaling ? sacc[45 + j] : 1.0, mn), mx) * inv_radius;
        for (int l = j; l < 9; ++l) {
          const double v = sacc[tri9b(j, l)] + (j == l ? dj : 0.0);
          Sm[j * 9 + l] = v;
          Sm[l * 9 + j] = v;
        }
      }
      block9_inverse(Sm, inv);
      for (int k = 0; k < 81; ++k) pre[k] = (T)inv[k];
    }
  } else if (lane < 9) {
    double sii = 0.0;
#pragma unroll
    for (int l = 0; l < 9; ++l) sii = (l == i) ? a[l] : sii;
    const double v = (B.preconditioner == CERES_B200_PRECOND_JACOBI) ? 1.0 / fmax(sii, Eps<T>::v()) : 1.0;
#pragma unroll
    for (int l = 0; l < 9; ++l) pre[i * 9 + l] = (T)(l == i ? v : 0.0);
  }
}

template <typename T>
__device__ void cta_assemble(const ceres_b200_batch_t& B, const Prob& P, double radius, const Smem& S,
                             double& gmax, double& gnorm) {
  const double inv_radius = 1.0 / fmax(radius, kEps64);
  double gp = 0.0, gsp = 0.0;
  cta_point_assemble<T>(B, P, inv_radius, gp, gsp);
  __syncthreads();
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double gc = 0.0, gsc = 0.0;
  for (int cl = w; cl < P.nc; cl += nw) {
    const int cg = P.cam0 + cl;
    double* acc = B.cam_acc + (size_t)cg * 72;
    if (!B.cam_const[cg]) {
      warp_camera_pass<T, 0>(B, cg, cl, acc);
      warp_camera_pass<T, 1>(B, cg, cl, acc);
      warp_camera_pass<T, 2>(B, cg, cl, acc);
    }
    __syncwarp();
    warp_camera_finish<T>(B, cg, inv_radius, gc, gsc);
  }
  double v[4] = {gp, gsp, gc, gsc};
  cta_allreduce<4>(v, 0x5u, S.red, S.bcast);
  gmax = fmax(v[0], v[2]);
  gnorm = sqrt(v[1] + v[3]);
}

// ------------------------------------------------------------------------------------
// Implicit Schur product over the problem's slices (the point-major walk of
// matvec_slices): y = (J_c^T J_c - H_cp W^-1 H_pc) p into shared memory, A the
// accumulation type (T, or double for the refinement residual).
// ------------------------------------------------------------------------------------
template <typename T, typename TP, typename A>
__device__ void cta_schur_product(const ceres_b200_batch_t& B, const Prob& P, const TP* ps, A* ys) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const T* jac = reinterpret_cast<const T*>(B.jac);
  const T* winv = reinterpret_cast<const T*>(B.winv);
  for (int s = P.s0 + w; s < P.s0 + P.ns; s += nw) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s] + lane;
    A t0 = 0, t1 = 0, t2 = 0;
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = max(B.slot_cam[slot], 0);  // padding slots: zero Jacobians, camera 0 as the address
      T rv[kRec];
      rec_load(jac, slot, rv);
      const TP* pc = ps + 9 * (size_t)c;
      A u0 = 0, u1 = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) { u0 += (A)rv[j] * (A)pc[j]; u1 += (A)rv[9 + j] * (A)pc[j]; }
      t0 += (A)rv[18] * u0 + (A)rv[21] * u1;
      t1 += (A)rv[19] * u0 + (A)rv[22] * u1;
      t2 += (A)rv[20] * u0 + (A)rv[23] * u1;
    }
    const T* wi = winv + 6 * (size_t)q;
    const A w0 = (A)wi[0], w1 = (A)wi[1], w2 = (A)wi[2], w3 = (A)wi[3], w4 = (A)wi[4], w5 = (A)wi[5];
    const A s0 = w0 * t0 + w1 * t1 + w2 * t2;
    const A s1 = w1 * t0 + w3 * t1 + w4 * t2;
    const A s2 = w2 * t0 + w4 * t1 + w5 * t2;
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = B.slot_cam[slot];
      if (c < 0) continue;
      T rv[kRec];
      rec_load(jac, slot, rv);
      const TP* pc = ps + 9 * (size_t)c;
      A u0 = 0, u1 = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) { u0 += (A)rv[j] * (A)pc[j]; u1 += (A)rv[9 + j] * (A)pc[j]; }
      const A v0 = u0 - ((A)rv[18] * s0 + (A)rv[19] * s1 + (A)rv[20] * s2);
      const A v1 = u1 - ((A)rv[21] * s0 + (A)rv[22] * s1 + (A)rv[23] * s2);
      A* yc = ys + 9 * (size_t)c;
#pragma unroll
      for (int j = 0; j < 9; ++j) atomicAdd(yc + j, (A)rv[j] * v0 + (A)rv[9 + j] * v1);
    }
  }
}

template <typename T>
__device__ __forceinline__ void precond_apply_b(const T* M, const double* r, double* z) {
  double rr[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) rr[j] = r[j];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) s += (double)M[i * 9 + j] * rr[j];
    z[i] = s;
  }
}

struct PcgOut {
  int iterations;
  bool success;
  double rnorm, rhs_norm;
};

// PCG (linear.py:1216-1256) on S x = rhs for one problem: x0 = 0, stop when
// |r| <= tol * max(|rhs| or *norm_ref, eps) after min_it; float64 vectors, the product
// in T. accumulate: x_out += x, else x_out = x.
template <typename T>
__device__ PcgOut cta_pcg(const ceres_b200_batch_t& B, const Prob& P, const Smem& S, const double* rhs,
                          double* x_out, bool accumulate, int min_it, int max_it, double tol, double norm_ref,
                          int stall_window) {
  const size_t N = 9 * (size_t)B.cam_off[B.num_problems];
  const int n = 9 * P.nc;
  const size_t o = 9 * (size_t)P.cam0;
  double* X = B.pcg + o;
  double* R = B.pcg + N + o;
  double* Z = B.pcg + 2 * N + o;
  double* Pv = B.pcg + 3 * N + o;
  double* AP = B.pcg + 4 * N + o;
  const T* Minv = reinterpret_cast<const T*>(B.precond) + 81 * (size_t)P.cam0;
  const double* D = B.cam_diag + o;
  T* ps = reinterpret_cast<T*>(S.ps);
  T* ys = reinterpret_cast<T*>(S.ys);
  const double eps = Eps<T>::v();

  for (int j = threadIdx.x; j < n; j += blockDim.x) { X[j] = 0.0; R[j] = rhs[j]; }
  __syncthreads();
  for (int c = threadIdx.x; c < P.nc; c += blockDim.x) precond_apply_b(Minv + 81 * (size_t)c, R + 9 * c, Z + 9 * c);
  __syncthreads();
  double v3[3] = {0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    v3[0] += R[j] * Z[j];
    v3[1] += R[j] * R[j];
    v3[2] += rhs[j] * rhs[j];
  }
  cta_allreduce<3>(v3, 0u, S.red, S.bcast);
  double rz_old = v3[0];
  double rnorm = sqrt(v3[1]);
  const double rhs_norm = fmax(norm_ref >= 0.0 ? norm_ref : sqrt(v3[2]), eps);
  PcgOut out{0, false, rnorm, rhs_norm};
  double rbest = rnorm, beta = 0.0;
  int last_improvement = 0;
  if (min_it <= 0 && rnorm <= tol * rhs_norm) {
    out.success = true;
  } else {
    for (int k = 0; k < max_it; ++k) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double pv = (k == 0) ? Z[j] : Z[j] + beta * Pv[j];
        Pv[j] = pv;
        ps[j] = (T)pv;
        ys[j] = (T)0;
      }
      __syncthreads();
      cta_schur_product<T, T, T>(B, P, ps, ys);
      __syncthreads();
      double v1[1] = {0.0};
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double y = (double)ys[j] + D[j] * Pv[j];
        AP[j] = y;
        v1[0] += Pv[j] * y;
      }
      cta_allreduce<1>(v1, 0u, S.red, S.bcast);
      const double denom = v1[0];
      if (fabs(denom) <= eps) {
        out.success = rnorm <= tol * rhs_norm;
        break;
      }
      const double alpha = rz_old / denom;
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        X[j] += alpha * Pv[j];
        R[j] -= alpha * AP[j];
      }
      __syncthreads();
      for (int c = threadIdx.x; c < P.nc; c += blockDim.x)
        precond_apply_b(Minv + 81 * (size_t)c, R + 9 * c, Z + 9 * c);
      __syncthreads();
      double v2[2] = {0.0, 0.0};
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        v2[0] += R[j] * Z[j];
        v2[1] += R[j] * R[j];
      }
      cta_allreduce<2>(v2, 0u, S.red, S.bcast);
      const double rz_new = v2[0];
      rnorm = sqrt(v2[1]);
      out.iterations = k + 1;
      if (out.iterations >= min_it && rnorm <= tol * rhs_norm) {
        out.success = true;
        break;
      }
      if (fabs(rz_old) <= eps) break;
      if (stall_window > 0) {
        if (rnorm < 0.99 * rbest) { rbest = rnorm; last_improvement = out.iterations; }
        else if (out.iterations - last_improvement >= stall_window) break;
      }
      beta = rz_new / rz_old;
      rz_old = rz_new;
    }
  }
  out.rnorm = rnorm;
  for (int j = threadIdx.x; j < n; j += blockDim.x) x_out[j] = accumulate ? x_out[j] + X[j] : X[j];
  __syncthreads();
  return out;
}

// The camera step: PCG with float64 refinement passes for the float32 store (the same
// sequence as the single-problem entry point). Returns the PCG iterations.
template <typename T>
__device__ int cta_linear_solve(const ceres_b200_batch_t& B, const Prob& P, const Smem& S) {
  const size_t N = 9 * (size_t)B.cam_off[B.num_problems];
  const size_t o = 9 * (size_t)P.cam0;
  const int n = 9 * P.nc;
  double* step = B.step_cameras + o;
  const double* rhs = B.rhs + o;
  const bool refine = B.max_refinements > 0 && sizeof(T) == sizeof(float);
  const PcgOut first = cta_pcg<T>(B, P, S, rhs, step, false, B.min_linear_solver_iterations,
                                  B.max_linear_solver_iterations, B.eta, -1.0, refine ? kBatchStall : 0);
  int iterations = first.iterations;
  if (refine && !first.success) {
    // float64 refinement: r64 = rhs - S step with float64 accumulation, then a float32
    // solve of S dx = r64 (tolerance relative to the original |rhs|) added to the step
    double* r64 = B.pcg + 5 * N + o;
    for (int it = 0; it < B.max_refinements; ++it) {
      for (int j = threadIdx.x; j < n; j += blockDim.x) S.y64[j] = 0.0;
      __syncthreads();
      cta_schur_product<T, double, double>(B, P, step, S.y64);
      __syncthreads();
      for (int j = threadIdx.x; j < n; j += blockDim.x) r64[j] = rhs[j] - (S.y64[j] + B.cam_diag[o + j] * step[j]);
      __syncthreads();
      const PcgOut corr = cta_pcg<T>(B, P, S, r64, step, true, 0, B.max_linear_solver_iterations, B.eta,
                                     first.rhs_norm, kBatchStall);
      iterations += corr.iterations;
    }
  }
  return iterations;
}

// ------------------------------------------------------------------------------------
// Step: candidate cameras, point back-substitution, model decrease, candidate cost
// (ceres_b200_ba_step at CTA scope). Outputs {cand cost, model, |dp|^2 + |dc|^2,
// non-finite count, |x + step|^2}.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cta_step(const ceres_b200_batch_t& B, const LossSpec& L, const Prob& P, const Smem& S,
                         unsigned& err, double out[5]) {
  const size_t o = 9 * (size_t)P.cam0;
  const int n = 9 * P.nc;
  double sq = 0.0, nonfinite = 0.0, state = 0.0, cand = 0.0, model = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const int c = P.cam0 + j / 9;
    double d = B.cam_const[c] ? 0.0 : B.step_cameras[o + j];
    if (!B.cam_const[c]) {
      if (!isfinite(d)) nonfinite += 1.0;
      sq += d * d;
    }
    B.step_cameras[o + j] = d;
    const double xc = B.cameras[o + j] + d;
    B.cand_cameras[o + j] = xc;
    state += xc * xc;
  }
  __syncthreads();
  cta_frames<false>(B.cand_cameras + o, B.frames + kFrame * (size_t)P.cam0, P.nc);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const T* jac = reinterpret_cast<const T*>(B.jac);
  const T* winv = reinterpret_cast<const T*>(B.winv);
  const double* frames = B.frames + kFrame * (size_t)P.cam0;
  const double* dcv = B.step_cameras + o;
  for (int s = P.s0 + w; s < P.s0 + P.ns; s += nw) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s] + lane;
    double t[3] = {0, 0, 0};
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = max(B.slot_cam[slot], 0);
      T rv[kRec];
      rec_load(jac, slot, rv);
      const double* dc = dcv + 9 * (size_t)c;
      double u0 = 0.0, u1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) { u0 += (double)rv[j] * dc[j]; u1 += (double)rv[9 + j] * dc[j]; }
#pragma unroll
      for (int m = 0; m < 3; ++m) t[m] += (double)rv[18 + m] * u0 + (double)rv[21 + m] * u1;
    }
    double dp[3] = {0, 0, 0};
    if (!B.pt_const[q]) {
      double wi[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) wi[i] = (double)winv[6 * (size_t)q + i];
      double wt[3];
      sym3_mul(wi, t, wt);
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        dp[m] = B.winv_ga[3 * (size_t)q + m] - wt[m];
        if (!isfinite(dp[m])) nonfinite += 1.0;
        sq += dp[m] * dp[m];
      }
    }
    double Xc[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      B.step_points[3 * (size_t)q + m] = dp[m];
      Xc[m] = B.points[3 * (size_t)q + m] + dp[m];
      B.cand_points[3 * (size_t)q + m] = Xc[m];
      state += Xc[m] * Xc[m];
    }
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = B.slot_cam[slot];
      if (c < 0) continue;
      T rv[kRec];
      rec_load(jac, slot, rv);
      const double2 r = reinterpret_cast<const double2*>(B.res)[slot];
      const double* dc = dcv + 9 * (size_t)c;
      double j0 = 0.0, j1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) { j0 += (double)rv[j] * dc[j]; j1 += (double)rv[9 + j] * dc[j]; }
#pragma unroll
      for (int m = 0; m < 3; ++m) { j0 += (double)rv[18 + m] * dp[m]; j1 += (double)rv[21 + m] * dp[m]; }
      const double a0 = r.x + j0, a1 = r.y + j1;
      model += 0.5 * (r.x * r.x + r.y * r.y) - 0.5 * (a0 * a0 + a1 * a1);
      const double2 ob = reinterpret_cast<const double2*>(B.slot_obs)[slot];
      Proj pj;
      CamRot R;
      double tail[6];
      frame_load<false>(frames + kFrame * (size_t)c, R, tail);
      snavely_project<false>(R, tail, Xc, ob.x, ob.y, pj);
      cand += robustify<false>(L, pj, err);
    }
  }
  double v[5] = {cand, model, sq, nonfinite, state};
  cta_allreduce<5>(v, 0u, S.red, S.bcast);
#pragma unroll
  for (int i = 0; i < 5; ++i) out[i] = v[i];
}

// candidate -> current for one problem's cameras and points
__device__ void cta_accept(const ceres_b200_batch_t& B, const Prob& P) {
  const size_t o = 9 * (size_t)P.cam0;
  for (int j = threadIdx.x; j < 9 * P.nc; j += blockDim.x) B.cameras[o + j] = B.cand_cameras[o + j];
  const size_t po = 3 * 32 * (size_t)P.s0;
  for (int j = threadIdx.x; j < 3 * 32 * P.ns; j += blockDim.x) B.points[po + j] = B.cand_points[po + j];
  __syncthreads();
}

// ------------------------------------------------------------------------------------
// The trust-region solve of one problem (the host loop of engine.run_lm, monotonic
// steps): scalars live in registers of every thread (all threads compute the same
// values from broadcast reductions), thread 0 writes the records.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cta_solve(const ceres_b200_batch_t& B, const Prob& P, const Smem& S) {
  const LossSpec L{B.loss_kind, B.loss_a, B.loss_b, B.loss_scale, B.inner_loss_kind, B.inner_a, B.inner_b,
                   B.inner_scale};
  double* res = B.result + (size_t)P.b * kBR;
  double* trace = B.trace + (size_t)P.b * B.max_trace * kBT;
  const bool lead = threadIdx.x == 0;
  unsigned err = 0;
  int records = 0, successful = 0, unsuccessful = 0, jac_evals = 0, res_evals = 0, linear_solves = 0;
  int term = CERES_B200_TERM_NO_CONVERGENCE, msg = CERES_B200_MSG_MAX_ITERATIONS;

  auto record = [&](double cost, double change, double gmax, double gnorm, double step_norm, double rho,
                    double radius, int lin, int flags) {
    if (lead && records < B.max_trace) {
      double* t = trace + (size_t)records * kBT;
      t[CERES_B200_BT_COST] = cost;
      t[CERES_B200_BT_COST_CHANGE] = change;
      t[CERES_B200_BT_GMAX] = gmax;
      t[CERES_B200_BT_GNORM] = gnorm;
      t[CERES_B200_BT_STEP_NORM] = step_norm;
      t[CERES_B200_BT_RHO] = rho;
      t[CERES_B200_BT_RADIUS] = radius;
      t[CERES_B200_BT_LINEAR_ITERATIONS] = (double)lin;
      t[CERES_B200_BT_FLAGS] = (double)flags;
      t[9] = 0.0;
    }
    ++records;
  };

  double radius = B.initial_radius;
  double decrease_factor = 2.0;
  double cost = cta_evaluate<T>(B, L, P, S, err);
  double gmax, gnorm;
  cta_assemble<T>(B, P, radius, S, gmax, gnorm);
  ++jac_evals;
  const double initial_cost = cost;
  double best_cost = cost;
  // _StepEvaluator with max_nonmonotonic = 0 (solver.py:823-861)
  double current_cost = cost, reference_cost = cost, candidate_cost_h = cost, minimum_cost = cost;
  double acc_reference = 0.0, acc_candidate = 0.0;
  int nonmonotonic = 0;
  bool need_assemble = false;
  bool previous_set = false;
  double previous_cost = 0.0;
  int consecutive_invalid = 0;
  bool done = false;

  // iteration 0
  record(cost, 0.0, gmax, gnorm, 0.0, 0.0, radius, 0, 3);
  if (gmax <= B.gradient_tolerance) {
    term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_GRADIENT; done = true;
  } else if (B.max_num_iterations == 0) {
    term = CERES_B200_TERM_NO_CONVERGENCE; msg = CERES_B200_MSG_MAX_ITERATIONS; done = true;
  }
  for (int iteration = 1; !done && iteration <= B.max_num_iterations; ++iteration) {
    if (need_assemble) {
      double gm, gn;  // the gradient stats of a re-assembly are not reported (the host loop keeps the old ones)
      cta_assemble<T>(B, P, radius, S, gm, gn);
      need_assemble = false;
    }
    ++jac_evals;
    const int lin = P.nc > 0 ? cta_linear_solve<T>(B, P, S) : 1;
    ++linear_solves;
    double st[5];
    cta_step<T>(B, L, P, S, err, st);
    if (st[3] > 0.0) {  // non-finite step
      ++consecutive_invalid;
      radius = radius / decrease_factor;
      decrease_factor *= 2.0;
      need_assemble = true;
      ++unsuccessful;
      if (consecutive_invalid >= B.max_consecutive_invalid_steps) {
        term = CERES_B200_TERM_FAILURE; msg = CERES_B200_MSG_INVALID_STEPS;
        break;
      }
      record(cost, 0.0, gmax, gnorm, 0.0, 0.0, radius, lin, 0);
      continue;
    }
    ++res_evals;
    const double cand_cost = st[0];
    const double model_decrease = fmax(st[1], 0.0);
    const bool step_is_valid = model_decrease > 0.0;
    double rho = 0.0;
    if (step_is_valid) {
      const double relative = (current_cost - cand_cost) / model_decrease;
      const double historical = (reference_cost - cand_cost) / (acc_reference + model_decrease);
      rho = fmax(relative, historical);
    }
    const bool accepted = step_is_valid && rho > B.min_relative_decrease;
    const double step_norm = sqrt(st[2]);
    int flags = step_is_valid ? 1 : 0;
    if (accepted) {
      consecutive_invalid = 0;
      ++successful;
      // step_accepted (max_nonmonotonic = 0)
      current_cost = cand_cost;
      acc_candidate += model_decrease;
      acc_reference += model_decrease;
      if (cand_cost < minimum_cost) {
        minimum_cost = cand_cost; nonmonotonic = 0; candidate_cost_h = cand_cost; acc_candidate = 0.0;
      } else {
        ++nonmonotonic;
        if (cand_cost > candidate_cost_h) { candidate_cost_h = cand_cost; acc_candidate = 0.0; }
      }
      if (nonmonotonic == 0) { reference_cost = candidate_cost_h; acc_reference = acc_candidate; }
      cta_accept(B, P);
      if (cand_cost < best_cost) best_cost = cand_cost;
      else flags |= (cand_cost > best_cost) ? 4 : 0;
      const double tmp = 2.0 * rho - 1.0;
      radius = fmin(B.max_radius, radius / fmax(1.0 / 3.0, 1.0 - tmp * tmp * tmp));
      decrease_factor = 2.0;
      flags |= 2;
    } else {
      ++unsuccessful;
      radius = radius / decrease_factor;
      decrease_factor *= 2.0;
      need_assemble = true;
    }
    record(cost, cost - cand_cost, gmax, gnorm, step_norm, rho, radius, lin, flags);
    if (accepted) {
      const double state_norm = sqrt(st[4]);
      if (step_norm <= B.parameter_tolerance * (state_norm + B.parameter_tolerance)) {
        term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_PARAMETER;
        break;
      }
      if (previous_set && fabs(previous_cost - cand_cost) <= B.function_tolerance * fmax(previous_cost, 1.0)) {
        term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_FUNCTION;
        break;
      }
      previous_cost = cand_cost;
      previous_set = true;
      cost = cta_evaluate<T>(B, L, P, S, err);
      cta_assemble<T>(B, P, radius, S, gmax, gnorm);
      ++jac_evals;
      if (gmax <= B.gradient_tolerance) {
        term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_GRADIENT;
        best_cost = cost;
        break;
      }
    }
    if (radius <= B.min_radius) {
      term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_MIN_RADIUS;
      break;
    }
  }
  // err: OR over the threads
  const unsigned any_err = __syncthreads_or(err);
  if (lead) {
    res[CERES_B200_BR_INITIAL_COST] = initial_cost;
    res[CERES_B200_BR_FINAL_COST] = best_cost;
    res[CERES_B200_BR_RECORDS] = (double)records;
    res[CERES_B200_BR_TERMINATION] = (double)term;
    res[CERES_B200_BR_MESSAGE] = (double)msg;
    res[CERES_B200_BR_SUCCESSFUL] = (double)successful;
    res[CERES_B200_BR_UNSUCCESSFUL] = (double)unsuccessful;
    res[CERES_B200_BR_JACOBIAN_EVALS] = (double)jac_evals;
    res[CERES_B200_BR_RESIDUAL_EVALS] = (double)res_evals;
    res[CERES_B200_BR_LINEAR_SOLVES] = (double)linear_solves;
    res[CERES_B200_BR_ERROR] = (double)any_err;
    res[CERES_B200_BR_FINAL_GMAX] = gmax;
  }
  __syncthreads();
}

template <typename T, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_batch_solve(ceres_b200_batch_t B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[8 * kMaxWarps];
  __shared__ double bcast[8];
  __shared__ int next;
  const size_t vec = (size_t)((9 * B.max_cameras + 3) & ~3);
  Smem S;
  S.red = red;
  S.bcast = bcast;
  S.y64 = reinterpret_cast<double*>(smem_raw);
  S.ps = smem_raw + (sizeof(T) == sizeof(float) ? vec * sizeof(double) : 0);
  S.ys = reinterpret_cast<unsigned char*>(S.ps) + vec * sizeof(T);
  for (;;) {
    if (threadIdx.x == 0) next = (int)atomicAdd(B.queue, 1u);
    __syncthreads();
    const int b = next;
    __syncthreads();
    if (b >= B.num_problems) break;
    Prob P;
    P.b = b;
    P.cam0 = B.cam_off[b];
    P.nc = B.cam_off[b + 1] - P.cam0;
    P.s0 = B.slice_off[b];
    P.ns = B.slice_off[b + 1] - P.s0;
    cta_solve<T>(B, P, S);
  }
}

using BatchKernel = void (*)(ceres_b200_batch_t);

// The compiled (threads per CTA, resident CTAs per SM) shapes; the CTA count per SM
// sets the register cap (65536 / (threads * ctas)).
template <typename T>
BatchKernel batch_kernel(int threads, int ctas) {
  if (threads == 128 && ctas <= 2) return k_batch_solve<T, 128, 1>;
  if (threads == 128 && ctas == 4) return k_batch_solve<T, 128, 4>;
  if (threads == 256 && ctas <= 1) return k_batch_solve<T, 256, 1>;
  if (threads == 256 && ctas == 2) return k_batch_solve<T, 256, 2>;
  if (threads == 512 && ctas <= 1) return k_batch_solve<T, 512, 1>;
  return nullptr;
}

}  // namespace

extern "C" {

int ceres_b200_batch_struct_bytes(void) { return (int)sizeof(ceres_b200_batch_t); }

int ceres_b200_batch_solve(const ceres_b200_batch_t* batch, int threads_per_cta, int ctas_per_sm, void* stream) {
  if (!batch || batch->num_problems < 0) return CERES_B200_EINVAL;
  if (batch->num_problems == 0) return CERES_B200_OK;
  const ceres_b200_batch_t& B = *batch;
  if (!B.cam_off || !B.slice_off || !B.slice_base || !B.slice_len || !B.slot_cam || !B.slot_obs || !B.cam_offsets ||
      !B.cam_entries || !B.cam_const || !B.pt_const || !B.cameras || !B.points || !B.cand_cameras ||
      !B.cand_points || !B.jac || !B.res || !B.point_raw || !B.winv || !B.winv_ga || !B.step_points ||
      !B.cam_diag || !B.precond || !B.rhs || !B.step_cameras || !B.cam_acc || !B.frames || !B.pcg || !B.result ||
      !B.trace || !B.queue)
    return CERES_B200_EINVAL;
  if (B.precision != CERES_B200_FP32 && B.precision != CERES_B200_FP64) return CERES_B200_EINVAL;
  if (B.max_cameras < 0 || B.max_trace < 1 || B.max_num_iterations < 0) return CERES_B200_EINVAL;
  if (B.preconditioner < CERES_B200_PRECOND_IDENTITY || B.preconditioner > CERES_B200_PRECOND_SCHUR_JACOBI)
    return CERES_B200_EINVAL;
  const int threads = threads_per_cta == 0 ? 256 : threads_per_cta;
  const int ctas = ctas_per_sm == 0 ? 1 : ctas_per_sm;
  const bool f32 = B.precision == CERES_B200_FP32;
  BatchKernel kern = f32 ? batch_kernel<float>(threads, ctas) : batch_kernel<double>(threads, ctas);
  if (!kern) return CERES_B200_EINVAL;
  const size_t vec = (size_t)((9 * B.max_cameras + 3) & ~3);
  const size_t smem = f32 ? vec * (sizeof(double) + 2 * sizeof(float)) : vec * 2 * sizeof(double);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CERES_B200_ECUDA;
  int sms = 0, optin = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return CERES_B200_ECUDA;
  if (smem + 8 * 1024 > (size_t)optin) return CERES_B200_ETOOBIG;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return CERES_B200_ESMEM;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
    return CERES_B200_ESMEM;
  long long grid = (long long)sms * per_sm;
  if (grid > B.num_problems) grid = B.num_problems;
  kern<<<(int)grid, threads, smem, (cudaStream_t)stream>>>(B);
  return cudaGetLastError() == cudaSuccess ? CERES_B200_OK : CERES_B200_ECUDA;
}

}  // extern "C"
