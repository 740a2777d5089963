// Batched bundle adjustment: many independent problems in one persistent launch.
//
// Every thread-block cluster (1 to 16 CTAs) pulls whole problems from a work counter
// and runs the complete Levenberg-Marquardt solve of one problem at a time: the same
// evaluation, Schur assembly, implicit-Schur PCG and step arithmetic as the
// single-problem kernels of ba_kernels.cu, spread over the cluster's CTAs, and the
// trust-region decisions of ceres-torch's solver.py:35-357 (LM radius rule
// solver.py:805-820, step quality solver.py:823-861, convergence tests
// solver.py:320-336 and :1169-1175) on the device. There is no host round trip
// between iterations and no spin-wait: CTAs synchronise through the hardware cluster
// barrier only, and reductions read the other CTAs' partial sums from distributed
// shared memory in rank order, so every CTA of a cluster computes bit-identical
// scalars and takes the same branches.
//
// Ownership inside a cluster: slices (points) go to cluster warps round robin and
// stay with them for the whole solve, camera ranges go to CTAs (PCG vectors, camera
// steps, frames, accepted parameters), and the camera sums go to cluster warps.
// Data written by one CTA and read by another (frames, camera vectors, the Jacobian
// records in the camera-major pass) is read with ld.global.cg, so a stale line in
// another SM's L1 is never used; data written and read by the same CTA uses plain
// loads (never the read-only path: everything here is rewritten in-launch).
#include <cooperative_groups.h>

#include <cstdio>

#include "ba_device.cuh"

using namespace cb200;
namespace cgp = cooperative_groups;

namespace {

constexpr int kBR = CERES_B200_BATCH_RESULT;
constexpr int kBT = CERES_B200_BATCH_TRACE;
constexpr int kMaxWarps = 16;
constexpr int kBatchStall = 20;  // float32 PCG: iterations without a 1% residual drop before it stops

__device__ __forceinline__ int tri9b(int j, int l) { return j * 9 - (j * (j - 1)) / 2 + (l - j); }

template <typename V>
__device__ __forceinline__ V ldx(const V* p) { return __ldcg(p); }  // cross-CTA data

// Jacobian record loads; kCross: through L2 only.
template <bool kCross, typename T>
__device__ __forceinline__ void rec_load(const T* base, size_t slot, T v[kRec]) {
  load_rec<kCross>(base, slot, v);
}

struct Ctx {
  int rank, G;   // CTA rank in the cluster, cluster size
  int ct, CT;    // cluster-wide thread index and count
  int cw, CW;    // cluster-wide warp index and count
};

__device__ __forceinline__ void csync() { cgp::this_cluster().sync(); }

template <typename V>
__device__ __forceinline__ V* remote(V* p, int rank) {
  return cgp::this_cluster().map_shared_rank(p, rank);
}

struct Prob {
  int b;
  int nc, cam0;  // cameras [cam0, cam0 + nc)
  int ns, s0;    // slices [s0, s0 + ns); sorted points 32 * s0 ...
  int c0, c1;    // this CTA's camera range (local indices)
};

struct Smem {
  double* red;    // [8 * kMaxWarps]
  double* part;   // [8]: this CTA's partial sums for cluster reductions
  double* ps;     // [9 * max_cameras]: the PCG direction (all cameras)
  double* ys;     // [9 * max_cameras]: this CTA's product accumulator
  double* y64;    // the refinement's product accumulator (the same memory as ys: the
                  // refinement runs between PCG solves)
};

// Reduce NV values over the cluster (sum, or max where max_mask has the bit) and hand
// the result to every thread; every CTA folds the CTA partials in rank order.
template <int NV>
__device__ __forceinline__ void cl_allreduce(double v[NV], unsigned max_mask, const Ctx& X, const Smem& S) {
  block_reduce<NV>(v, max_mask, S.red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) S.part[i] = v[i];
  }
  csync();
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = ((max_mask >> i) & 1u) ? -INFINITY : 0.0;
  for (int r = 0; r < X.G; ++r) {
    const double* pr = remote(S.part, r);
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = ((max_mask >> i) & 1u) ? fmax(v[i], pr[i]) : v[i] + pr[i];
  }
  csync();
}

// ------------------------------------------------------------------------------------
// camera frames of this CTA's cameras; the cluster barrier publishes them
// ------------------------------------------------------------------------------------
template <bool kJac>
__device__ void cl_frames(const double* cams, double* frames, const Prob& P) {
  for (int c = P.c0 + threadIdx.x; c < P.c1; c += blockDim.x) {
    const double* cam = cams + 9 * (size_t)c;
    double cv[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) cv[i] = cam[i];
    const double aa[3] = {cv[0], cv[1], cv[2]};
    CamRot R;
    camera_rotation<kJac>(aa, R);
    frame_store<kJac>(frames + kFrame * (size_t)c, R, cv);
  }
  csync();
}

__device__ __forceinline__ void frame_load_x(const double* f, CamRot& R, double tail[6], bool jac) {
  const double2* f2 = reinterpret_cast<const double2*>(f);
  double2 v = __ldcg(f2);
  R.w = v.x; R.u[0] = v.y;
  v = __ldcg(f2 + 1);
  R.u[1] = v.x; R.u[2] = v.y;
  if (jac) {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      v = __ldcg(f2 + 2 + i);
      R.dqn[(2 * i) / 3][(2 * i) % 3] = v.x;
      R.dqn[(2 * i + 1) / 3][(2 * i + 1) % 3] = v.y;
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    v = __ldcg(f2 + 8 + i);
    tail[2 * i] = v.x;
    tail[2 * i + 1] = v.y;
  }
}

// ------------------------------------------------------------------------------------
// evaluation at B.cameras / B.points: residuals, Jacobian records, point sums, cost
// ------------------------------------------------------------------------------------
template <typename T>
__device__ double cl_evaluate(const ceres_b200_batch_t& B, const LossSpec& L, const Prob& P, const Ctx& X,
                              const Smem& S, unsigned& err) {
  cl_frames<true>(B.cameras + 9 * (size_t)P.cam0, B.frames + kFrame * (size_t)P.cam0, P);
  const int lane = threadIdx.x & 31;
  T* jac = reinterpret_cast<T*>(B.jac);
  const double* frames = B.frames + kFrame * (size_t)P.cam0;
  double cost = 0.0;
  for (int s = P.s0 + X.cw; s < P.s0 + P.ns; s += X.CW) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s];
    const double Xp[3] = {B.points[3 * (size_t)q], B.points[3 * (size_t)q + 1], B.points[3 * (size_t)q + 2]};
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
      frame_load_x(frames + kFrame * (size_t)c, R, tail, true);
      snavely_project<true>(R, tail, Xp, ob.x, ob.y, o);
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
  cl_allreduce<1>(v, 0u, X, S);
  return v[0];
}

// ------------------------------------------------------------------------------------
// Schur assembly for a radius: point blocks (own slices), camera sums and finish
// (cameras by cluster warp). Returns gmax and the gradient norm.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cl_point_assemble(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, double inv_radius,
                                  double& gmax, double& gsq) {
  T* winv = reinterpret_cast<T*>(B.winv);
  const double mn = B.min_lm_diagonal, mx = B.max_lm_diagonal;
  const int lane = threadIdx.x & 31;
  for (int s = P.s0 + X.cw; s < P.s0 + P.ns; s += X.CW) {
    const int q = s * 32 + lane;
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
// pass 1 rows 3-8, pass 2 the column sums, gradient and reduced rhs. The records,
// point blocks and residuals come from other CTAs' slices: read through L2.
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
    rec_load<true>(jac, slot, rv);
    double wi[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) wi[i] = (double)ldx(winv + 6 * (size_t)q + i);
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
          rec_load<true>(jac, slot2, rk);
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
      const double2 r = __ldcg(reinterpret_cast<const double2*>(B.res) + slot);
      const double wg[3] = {ldx(B.winv_ga + 3 * (size_t)q), ldx(B.winv_ga + 3 * (size_t)q + 1),
                            ldx(B.winv_ga + 3 * (size_t)q + 2)};
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
  double* pre = reinterpret_cast<double*>(B.precond) + 81 * (size_t)cg;  // float64 in both precisions
  double* dc = B.cam_diag + 9 * (size_t)cg;
  double* rh = B.rhs + 9 * (size_t)cg;
  const double mn = B.min_lm_diagonal, mx = B.max_lm_diagonal;
  if (B.cam_const[cg]) {
    if (lane < 9) { dc[lane] = 0.0; rh[lane] = 0.0; }
    for (int i = lane; i < 81; i += 32) pre[i] = (i % 10 == 0) ? 1.0 : 0.0;
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
        for (int r = 0; r < 9; ++r) pre[r * 9 + lane] = x[r];
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
      for (int k = 0; k < 81; ++k) pre[k] = inv[k];
    }
  } else if (lane < 9) {
    double sii = 0.0;
#pragma unroll
    for (int l = 0; l < 9; ++l) sii = (l == i) ? a[l] : sii;
    const double v = (B.preconditioner == CERES_B200_PRECOND_JACOBI) ? 1.0 / fmax(sii, kEps64) : 1.0;
#pragma unroll
    for (int l = 0; l < 9; ++l) pre[i * 9 + l] = l == i ? v : 0.0;
  }
}

template <typename T>
__device__ void cl_assemble(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, double radius, const Smem& S,
                            double& gmax, double& gnorm) {
  const double inv_radius = 1.0 / fmax(radius, kEps64);
  double gp = 0.0, gsp = 0.0;
  cl_point_assemble<T>(B, P, X, inv_radius, gp, gsp);
  csync();  // point blocks of every CTA before the camera sums read them
  double gc = 0.0, gsc = 0.0;
  for (int cl = X.cw; cl < P.nc; cl += X.CW) {
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
  cl_allreduce<4>(v, 0x5u, X, S);  // also publishes the camera blocks
  gmax = fmax(v[0], v[2]);
  gnorm = sqrt(v[1] + v[3]);
}

// ------------------------------------------------------------------------------------
// Implicit Schur product y = (J_c^T J_c - H_cp W^-1 H_pc) p of one problem in two passes
// with no atomics, so every sum has a fixed order whatever the cluster shape:
//   point pass  (the problem's slices over the cluster's warps, lane = point):
//                 s_q = W_q^-1 sum_k Jp_k^T (Jc_k p_c(k)), into B.step_points (scratch
//                 during the linear solve; the step overwrites it afterwards);
//   cluster barrier;
//   camera pass (the problem's cameras over the cluster's warps, lane = observation):
//                 y_c = sum_e Jc_e^T (Jc_e p_c - Jp_e s_q(e)), the lane sums added by a
//                 butterfly, written to ys of the CTA that owns camera c (distributed
//                 shared memory, one writer per element).
// The caller's cluster barrier publishes ys. kCrossP: p is a global float64 vector
// written by other CTAs (otherwise this CTA's shared-memory copy).
// ------------------------------------------------------------------------------------
template <typename T, typename TP, bool kCrossP>
__device__ void cl_schur_product(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, const TP* ps, double* ys) {
  const int lane = threadIdx.x & 31;
  const T* jac = reinterpret_cast<const T*>(B.jac);
  const T* winv = reinterpret_cast<const T*>(B.winv);
  double* sv = B.step_points;
  for (int s = P.s0 + X.cw; s < P.s0 + P.ns; s += X.CW) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s] + lane;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = max(B.slot_cam[slot], 0);  // padding slots: zero Jacobians, camera 0 as the address
      T rv[kRec];
      rec_load<false>(jac, slot, rv);
      const TP* pc = ps + 9 * (size_t)c;
      double u0 = 0.0, u1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const double pj = kCrossP ? (double)ldx(pc + j) : (double)pc[j];
        u0 += (double)rv[j] * pj;
        u1 += (double)rv[9 + j] * pj;
      }
      t0 += (double)rv[18] * u0 + (double)rv[21] * u1;
      t1 += (double)rv[19] * u0 + (double)rv[22] * u1;
      t2 += (double)rv[20] * u0 + (double)rv[23] * u1;
    }
    const T* wi = winv + 6 * (size_t)q;
    const double w0 = wi[0], w1 = wi[1], w2 = wi[2], w3 = wi[3], w4 = wi[4], w5 = wi[5];
    sv[3 * (size_t)q] = w0 * t0 + w1 * t1 + w2 * t2;
    sv[3 * (size_t)q + 1] = w1 * t0 + w3 * t1 + w4 * t2;
    sv[3 * (size_t)q + 2] = w2 * t0 + w4 * t1 + w5 * t2;
  }
  csync();  // every point's s_q
  const int per = (P.nc + X.G - 1) / X.G;  // cameras per CTA (Prob::c0 = rank * per)
  for (int cl = X.cw; cl < P.nc; cl += X.CW) {
    const int cg = P.cam0 + cl;
    const TP* pcp = ps + 9 * (size_t)cl;
    double pc[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) pc[j] = kCrossP ? (double)ldx(pcp + j) : (double)pcp[j];
    double y[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) y[j] = 0.0;
    const int e1 = B.cam_offsets[cg + 1];
    for (int e = B.cam_offsets[cg] + lane; e < e1; e += 32) {
      const int2 ent = reinterpret_cast<const int2*>(B.cam_entries)[e];
      T rv[kRec];
      rec_load<true>(jac, (size_t)ent.x, rv);
      const double* sq = sv + 3 * (size_t)ent.y;
      const double s0 = ldx(sq), s1 = ldx(sq + 1), s2 = ldx(sq + 2);
      double u0 = 0.0, u1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        u0 += (double)rv[j] * pc[j];
        u1 += (double)rv[9 + j] * pc[j];
      }
      const double v0 = u0 - ((double)rv[18] * s0 + (double)rv[19] * s1 + (double)rv[20] * s2);
      const double v1 = u1 - ((double)rv[21] * s0 + (double)rv[22] * s1 + (double)rv[23] * s2);
#pragma unroll
      for (int j = 0; j < 9; ++j) y[j] += (double)rv[j] * v0 + (double)rv[9 + j] * v1;
    }
    double mine = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const double w = warp_sum(y[j]);
      mine = (lane == j) ? w : mine;
    }
    if (lane < 9) remote(ys, cl / per)[9 * (size_t)cl + lane] = mine;
  }
}

__device__ __forceinline__ void precond_apply_b(const double* M, const double* r, double* z) {
  double rr[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) rr[j] = r[j];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) s += ldx(M + i * 9 + j) * rr[j];
    z[i] = s;
  }
}

struct PcgOut {
  int iterations;
  bool success;
  double rnorm, rhs_norm;
};

// PCG (linear.py:1216-1256) on S x = rhs for one problem: x0 = 0, stop when
// |r| <= tol * max(|rhs| or norm_ref, eps) after min_it; float64 vectors (each CTA
// owns the entries of its camera range), the product in T over each CTA's slices,
// folded across the cluster by the owner. accumulate: x_out += x, else x_out = x.
template <typename T>
__device__ PcgOut cl_pcg(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, const Smem& S, const double* rhs,
                         double* x_out, bool accumulate, int min_it, int max_it, double tol, double norm_ref,
                         int stall_window) {
  const size_t N = 9 * (size_t)B.cam_off[B.num_problems];
  const int n = 9 * P.nc;
  const int j0 = 9 * P.c0, j1 = 9 * P.c1;
  const size_t o = 9 * (size_t)P.cam0;
  double* Xv = B.pcg + o;
  double* R = B.pcg + N + o;
  double* Z = B.pcg + 2 * N + o;
  double* Pb[2] = {B.pcg + 3 * N + o, B.pcg + 4 * N + o};
  double* AP = B.pcg + 5 * N + o;
  const double* Minv = reinterpret_cast<const double*>(B.precond) + 81 * (size_t)P.cam0;
  const double* D = B.cam_diag + o;
  // the products stream the store in T and compute in float64 (float32 arithmetic adds
  // errors of 1e-7 |U| |p| per product that swamp the small eigenvalues of S once the
  // LM damping has decayed, and costs the same time)
  double* ps = S.ps;
  double* ys = S.ys;
  const double eps = kEps64;  // float64 vectors and arithmetic in both precisions

  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) { Xv[j] = 0.0; R[j] = ldx(rhs + j); }
  __syncthreads();
  for (int c = P.c0 + threadIdx.x; c < P.c1; c += blockDim.x)
    precond_apply_b(Minv + 81 * (size_t)c, R + 9 * c, Z + 9 * c);
  __syncthreads();
  double v3[3] = {0.0, 0.0, 0.0};
  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const double rhsj = ldx(rhs + j);
    v3[0] += R[j] * Z[j];
    v3[1] += R[j] * R[j];
    v3[2] += rhsj * rhsj;
  }
  cl_allreduce<3>(v3, 0u, X, S);  // also publishes Z
  double rz_old = v3[0];
  double rnorm = sqrt(v3[1]);
  const double rhs_norm = fmax(norm_ref >= 0.0 ? norm_ref : sqrt(v3[2]), eps);
  PcgOut out{0, false, rnorm, rhs_norm};
  double rbest = rnorm, beta = 0.0;
  int last_improvement = 0, cur = 0;
  if (min_it <= 0 && rnorm <= tol * rhs_norm) {
    out.success = true;
  } else {
    for (int k = 0; k < max_it; ++k) {
      const int nxt = k == 0 ? 0 : cur ^ 1;
      const double* Pold = Pb[cur];
      double* Pnew = Pb[nxt];
      // every CTA builds the whole direction in shared memory; the owner stores its part
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double pv = (k == 0) ? ldx(Z + j) : ldx(Z + j) + beta * ldx(Pold + j);
        ps[j] = pv;
        if (j >= j0 && j < j1) Pnew[j] = pv;
      }
      cur = nxt;
      __syncthreads();
      cl_schur_product<T, double, false>(B, P, X, ps, ys);
      csync();  // this CTA's cameras' products are complete
      double v1[1] = {0.0};
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double y = ys[j] + ldx(D + j) * Pnew[j];
        AP[j] = y;
        v1[0] += Pnew[j] * y;
      }
      cl_allreduce<1>(v1, 0u, X, S);
      const double denom = v1[0];
      if (fabs(denom) <= eps) {
        out.success = rnorm <= tol * rhs_norm;
        break;
      }
      const double alpha = rz_old / denom;
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        Xv[j] += alpha * Pnew[j];
        R[j] -= alpha * AP[j];
      }
      __syncthreads();
      for (int c = P.c0 + threadIdx.x; c < P.c1; c += blockDim.x)
        precond_apply_b(Minv + 81 * (size_t)c, R + 9 * c, Z + 9 * c);
      __syncthreads();
      double v2[2] = {0.0, 0.0};
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        v2[0] += R[j] * Z[j];
        v2[1] += R[j] * R[j];
      }
      cl_allreduce<2>(v2, 0u, X, S);  // also publishes Z and the new direction
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
  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) x_out[j] = accumulate ? x_out[j] + Xv[j] : Xv[j];
  csync();  // the solution is published
  return out;
}

// The camera step: PCG with float64 refinement passes for the float32 store (the same
// sequence as the single-problem entry point). Returns the PCG iterations.
template <typename T>
__device__ int cl_linear_solve(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, const Smem& S) {
  const size_t N = 9 * (size_t)B.cam_off[B.num_problems];
  const size_t o = 9 * (size_t)P.cam0;
  const int j0 = 9 * P.c0, j1 = 9 * P.c1;
  double* step = B.step_cameras + o;
  const double* rhs = B.rhs + o;
  const bool refine = B.max_refinements > 0 && sizeof(T) == sizeof(float);
  const PcgOut first = cl_pcg<T>(B, P, X, S, rhs, step, false, B.min_linear_solver_iterations,
                                 B.max_linear_solver_iterations, B.eta, -1.0, refine ? kBatchStall : 0);
  int iterations = first.iterations;
  if (refine && !first.success) {
    // float64 refinement: r64 = rhs - S step with float64 accumulation, then a float32
    // solve of S dx = r64 (tolerance relative to the original |rhs|) added to the step
    double* r64 = B.pcg + 6 * N + o;
    for (int it = 0; it < B.max_refinements; ++it) {
      cl_schur_product<T, double, true>(B, P, X, step, S.y64);
      csync();
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        r64[j] = ldx(rhs + j) - (S.y64[j] + ldx(B.cam_diag + o + j) * step[j]);
      }
      csync();
      const PcgOut corr = cl_pcg<T>(B, P, X, S, r64, step, true, 0, B.max_linear_solver_iterations, B.eta,
                                    first.rhs_norm, kBatchStall);
      iterations += corr.iterations;
    }
  }
  return iterations;
}

// ------------------------------------------------------------------------------------
// Step: candidate cameras (own range), point back-substitution, model decrease and
// candidate cost (own slices). Outputs {cand cost, model, |step|^2, non-finite,
// |x + step|^2} over the cluster.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cl_step(const ceres_b200_batch_t& B, const LossSpec& L, const Prob& P, const Ctx& X,
                        const Smem& S, unsigned& err, double out[5]) {
  const size_t o = 9 * (size_t)P.cam0;
  double sq = 0.0, nonfinite = 0.0, state = 0.0, cand = 0.0, model = 0.0;
  for (int j = 9 * P.c0 + threadIdx.x; j < 9 * P.c1; j += blockDim.x) {
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
  cl_frames<false>(B.cand_cameras + o, B.frames + kFrame * (size_t)P.cam0, P);  // ends with a cluster barrier
  const int lane = threadIdx.x & 31;
  const T* jac = reinterpret_cast<const T*>(B.jac);
  const T* winv = reinterpret_cast<const T*>(B.winv);
  const double* frames = B.frames + kFrame * (size_t)P.cam0;
  const double* dcv = B.step_cameras + o;
  for (int s = P.s0 + X.cw; s < P.s0 + P.ns; s += X.CW) {
    const int q = s * 32 + lane;
    const int len = B.slice_len[s];
    const size_t base = (size_t)B.slice_base[s] + lane;
    double t[3] = {0, 0, 0};
    double sa = 0.0;  // sum_o r_o.a_o + 0.5 |a_o|^2 with a_o = Jc_o dc
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k;
      const int c = B.slot_cam[slot];
      T rv[kRec];
      rec_load<false>(jac, slot, rv);
      double2 r = reinterpret_cast<const double2*>(B.res)[slot];
      if (c < 0) r = make_double2(0.0, 0.0);  // padding: zero Jacobian, camera 0 as the address
      const double* dc = dcv + 9 * (size_t)max(c, 0);
      double u0 = 0.0, u1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        const double dj = ldx(dc + j);
        u0 += (double)rv[j] * dj;
        u1 += (double)rv[9 + j] * dj;
      }
#pragma unroll
      for (int m = 0; m < 3; ++m) t[m] += (double)rv[18 + m] * u0 + (double)rv[21 + m] * u1;
      sa += r.x * u0 + r.y * u1 + 0.5 * (u0 * u0 + u1 * u1);
    }
    // model decrease of the track: -sa - dp.(g + t) - 0.5 dp^T V dp, with V and g the
    // point sums of the evaluation (the per-observation form expanded, so the records
    // are read once)
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
      const double* pr = B.point_raw + 9 * (size_t)q;
      double V[6], Vdp[3];
#pragma unroll
      for (int i = 0; i < 6; ++i) V[i] = pr[i];
      sym3_mul(V, dp, Vdp);
#pragma unroll
      for (int m = 0; m < 3; ++m) model -= dp[m] * (pr[6 + m] + t[m] + 0.5 * Vdp[m]);
    }
    model -= sa;
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
      const double2 ob = reinterpret_cast<const double2*>(B.slot_obs)[slot];
      Proj pj;
      CamRot R;
      double tail[6];
      frame_load_x(frames + kFrame * (size_t)c, R, tail, false);
      snavely_project<false>(R, tail, Xc, ob.x, ob.y, pj);
      cand += robustify<false>(L, pj, err);
    }
  }
  double v[5] = {cand, model, sq, nonfinite, state};
  cl_allreduce<5>(v, 0u, X, S);
#pragma unroll
  for (int i = 0; i < 5; ++i) out[i] = v[i];
}

// candidate -> current: this CTA's camera range and its own slices' points
__device__ void cl_accept(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X) {
  const size_t o = 9 * (size_t)P.cam0;
  for (int j = 9 * P.c0 + threadIdx.x; j < 9 * P.c1; j += blockDim.x) B.cameras[o + j] = B.cand_cameras[o + j];
  const int lane = threadIdx.x & 31;
  for (int s = P.s0 + X.cw; s < P.s0 + P.ns; s += X.CW) {
    const size_t q = (size_t)s * 32 + lane;
#pragma unroll
    for (int m = 0; m < 3; ++m) B.points[3 * q + m] = B.cand_points[3 * q + m];
  }
  csync();
}

// ------------------------------------------------------------------------------------
// The trust-region solve of one problem (the host loop of engine.run_lm, monotonic
// steps). Every thread of every CTA of the cluster holds the same scalars (computed
// from cluster reductions); thread 0 of rank 0 writes the records.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ void cl_solve(const ceres_b200_batch_t& B, const Prob& P, const Ctx& X, const Smem& S) {
  const LossSpec L{B.loss_kind, B.loss_a, B.loss_b, B.loss_scale, B.inner_loss_kind, B.inner_a, B.inner_b,
                   B.inner_scale};
  double* res = B.result + (size_t)P.b * kBR;
  double* trace = B.trace + (size_t)P.b * B.max_trace * kBT;
  const bool lead = threadIdx.x == 0 && X.rank == 0;
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
  double cost = cl_evaluate<T>(B, L, P, X, S, err);
  double gmax, gnorm;
  cl_assemble<T>(B, P, X, radius, S, gmax, gnorm);
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

  record(cost, 0.0, gmax, gnorm, 0.0, 0.0, radius, 0, 3);  // iteration 0
  if (gmax <= B.gradient_tolerance) {
    term = CERES_B200_TERM_CONVERGENCE; msg = CERES_B200_MSG_GRADIENT; done = true;
  } else if (B.max_num_iterations == 0) {
    term = CERES_B200_TERM_NO_CONVERGENCE; msg = CERES_B200_MSG_MAX_ITERATIONS; done = true;
  }
  for (int iteration = 1; !done && iteration <= B.max_num_iterations; ++iteration) {
    if (need_assemble) {
      double gm, gn;  // the host loop keeps the gradient stats of the last evaluation
      cl_assemble<T>(B, P, X, radius, S, gm, gn);
      need_assemble = false;
    }
    ++jac_evals;
    const int lin = cl_linear_solve<T>(B, P, X, S);
    ++linear_solves;
    double st[5];
    cl_step<T>(B, L, P, X, S, err, st);
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
      cl_accept(B, P, X);
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
      cost = cl_evaluate<T>(B, L, P, X, S, err);
      cl_assemble<T>(B, P, X, radius, S, gmax, gnorm);
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
  double ev[1] = {(double)__syncthreads_or(err)};
  cl_allreduce<1>(ev, 1u, X, S);
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
    res[CERES_B200_BR_ERROR] = ev[0];
    res[CERES_B200_BR_FINAL_GMAX] = gmax;
  }
}

template <typename T, int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_batch_solve(ceres_b200_batch_t B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[8 * kMaxWarps];
  __shared__ double part[8];
  __shared__ int next;
  const cgp::cluster_group cluster = cgp::this_cluster();
  Ctx X;
  X.rank = (int)cluster.block_rank();
  X.G = (int)cluster.num_blocks();
  X.ct = X.rank * blockDim.x + threadIdx.x;
  X.CT = X.G * blockDim.x;
  X.cw = X.rank * (blockDim.x >> 5) + (threadIdx.x >> 5);
  X.CW = X.G * (blockDim.x >> 5);
  const size_t vec = (size_t)((9 * B.max_cameras + 3) & ~3);
  Smem S;
  S.red = red;
  S.part = part;
  S.ps = reinterpret_cast<double*>(smem_raw);
  S.ys = S.ps + vec;
  S.y64 = S.ys;
  for (;;) {
    if (X.rank == 0 && threadIdx.x == 0) next = (int)atomicAdd(B.queue, 1u);
    csync();
    const int b = *remote(&next, 0);
    csync();
    if (b >= B.num_problems) break;
    Prob P;
    P.b = b;
    P.cam0 = B.cam_off[b];
    P.nc = B.cam_off[b + 1] - P.cam0;
    P.s0 = B.slice_off[b];
    P.ns = B.slice_off[b + 1] - P.s0;
    const int per = (P.nc + X.G - 1) / X.G;
    P.c0 = min(P.nc, X.rank * per);
    P.c1 = min(P.nc, P.c0 + per);
    cl_solve<T>(B, P, X, S);
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

int ceres_b200_batch_solve(const ceres_b200_batch_t* batch, int threads_per_cta, int ctas_per_sm, int cluster_size,
                           void* stream) {
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
  if ((reinterpret_cast<uintptr_t>(B.jac) & 31) != 0) return CERES_B200_EINVAL;  // 256-bit record loads
  if (B.max_cameras < 0 || B.max_trace < 1 || B.max_num_iterations < 0) return CERES_B200_EINVAL;
  if (B.preconditioner < CERES_B200_PRECOND_IDENTITY || B.preconditioner > CERES_B200_PRECOND_SCHUR_JACOBI)
    return CERES_B200_EINVAL;
  const int G = cluster_size == 0 ? 1 : cluster_size;
  if (G != 1 && G != 2 && G != 4 && G != 8 && G != 16) return CERES_B200_EINVAL;
  const int threads = threads_per_cta == 0 ? 256 : threads_per_cta;
  const int ctas = ctas_per_sm == 0 ? 1 : ctas_per_sm;
  const bool f32 = B.precision == CERES_B200_FP32;
  BatchKernel kern = f32 ? batch_kernel<float>(threads, ctas) : batch_kernel<double>(threads, ctas);
  if (!kern) return CERES_B200_EINVAL;
  const size_t vec = (size_t)((9 * B.max_cameras + 3) & ~3);
  const size_t smem = vec * 2 * sizeof(double);
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
  if (G > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return CERES_B200_ECOOP;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)G;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = (cudaStream_t)stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3((unsigned)G);
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) return CERES_B200_ECOOP;
  long long n = clusters;
  if (n > B.num_problems) n = B.num_problems;
  cfg.gridDim = dim3((unsigned)(n * G));
  if (cudaLaunchKernelEx(&cfg, kern, B) != cudaSuccess) return CERES_B200_ECUDA;
  return cudaGetLastError() == cudaSuccess ? CERES_B200_OK : CERES_B200_ECUDA;
}

}  // extern "C"
