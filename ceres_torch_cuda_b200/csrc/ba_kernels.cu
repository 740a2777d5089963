// Schur-complement bundle-adjustment kernels for B200 (sm_100a) and their C ABI.
//
// Data layout (see include/ceres_b200.h): observations in a sliced-ELL store
// where warp w owns slices of 32 points (lane = point, sorted by track length)
// and walks their observations slot by slot; Jacobians are 24-scalar records
// (96 B in FP32, 192 B in FP64) read with 128-bit loads. Every kernel is
// bandwidth-bound; all reductions are deterministic (fixed CTA count, fixed
// fold order) so a solve is bit-reproducible on one device.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <mutex>

#include "ba_device.cuh"

using namespace cb200;

namespace {

// kernels launched by this library since load (reported by ceres_b200_launch_count)
unsigned long long g_launches = 0;

// CERES_B200_TRACE=1 in the environment prints each host-side step to stderr.
bool trace_on() {
  static int on = -1;
  if (on < 0) {
    const char* v = getenv("CERES_B200_TRACE");
    on = (v && v[0] == '1') ? 1 : 0;
  }
  return on == 1;
}
#define CB_TRACE(...)                        \
  do {                                       \
    if (trace_on()) {                        \
      fprintf(stderr, "[ceres_b200] " __VA_ARGS__); \
      fprintf(stderr, "\n");                 \
      fflush(stderr);                        \
    }                                        \
  } while (0)
inline void count_launch(int n = 1) { __atomic_fetch_add(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }

// counters[] slots
constexpr int kCtrEval = 0, kCtrPoint = 1, kCtrCamera = 2, kCtrStep = 3, kCtrCamStep = 4;
constexpr int kCtrSliceEval = 5, kCtrSliceStep = 6;  // dynamic slice counters (zero between launches)

template <int NV> struct StatIdx { int idx[NV]; };  // stats entries a kernel argument names
constexpr int kCtrBarCount = 8, kCtrBarGen = 9, kCtrBarFlag = 10, kCtrError = 12;

constexpr int kWarpBlock = 256;  // threads per CTA of the slice-walking kernels
// Resident CTAs per SM the evaluator and the step kernel are compiled for: a register
// cap that trades a few spilled registers for twice (evaluator with Jacobian: 128
// registers, 2 CTAs) or 1.5 times (step: 80 registers, 3 CTAs) the warps in flight;
// both kernels wait on chains of dependent float64 operations, so more warps hide more
// of that latency (measured on the 6.0M-observation problem: evaluator 0.62 -> 0.42 ms,
// step 0.49 -> 0.45 ms).
#ifndef CERES_B200_EVAL_MIN_BLOCKS
#define CERES_B200_EVAL_MIN_BLOCKS 2
#endif
#ifndef CERES_B200_EVAL_NOJAC_MIN_BLOCKS
#define CERES_B200_EVAL_NOJAC_MIN_BLOCKS 3
#endif
#ifndef CERES_B200_STEP_MIN_BLOCKS
#define CERES_B200_STEP_MIN_BLOCKS 3
#endif

struct DevInfo {
  int sms = 0;
  int max_smem_optin = 0;
};

DevInfo device_info() {
  static DevInfo cache[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cache[dev].sms > 0) return cache[dev];
  DevInfo d;
  cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (dev >= 0 && dev < 64) cache[dev] = d;
  return d;
}

inline int slice_grid(const ceres_b200_ba_t& ba, const DevInfo& d) {
  const int warps = kWarpBlock / 32;
  int g = (ba.num_slices + warps - 1) / warps;
  const int cap = d.sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return g;
}

// scratch layout: per-CTA reduction partials of the slice and camera kernels,
// one auxiliary stats row, then the PCG area.
constexpr size_t kRedSlots = 8;  // doubles per CTA

inline size_t red_area_bytes(const ceres_b200_ba_t& ba, const DevInfo& d) {
  int g = slice_grid(ba, d);
  if (ba.num_cameras > g) g = ba.num_cameras;
  if (g < 64) g = 64;
  return ((size_t)g * kRedSlots * sizeof(double) + 255) & ~(size_t)255;
}

// Camera frames (kFrame float64 per camera) follow the reduction area in the scratch.
inline size_t frames_bytes(const ceres_b200_ba_t& ba) {
  return ((size_t)(ba.num_cameras > 0 ? ba.num_cameras : 1) * kFrame * sizeof(double) + 255) & ~(size_t)255;
}

// Per-slice partial sums of the evaluation and step kernels (5 float64 per slice)
// follow the frames.
inline size_t slice_part_bytes(const ceres_b200_ba_t& ba) {
  return ((size_t)(ba.num_slices > 0 ? ba.num_slices : 1) * 5 * sizeof(double) + 255) & ~(size_t)255;
}

// Grid of the dynamically scheduled slice kernels: the CTAs resident at once (the
// kernels' register caps fix that count), at most slice_grid.
inline int resident_slice_grid(const ceres_b200_ba_t& ba, const DevInfo& d, int ctas_per_sm) {
  const int g = d.sms * ctas_per_sm;
  const int sg = slice_grid(ba, d);
  return g < sg ? g : sg;
}

}  // namespace

// ======================================================================================
// Evaluation: residual, Jacobian, corrector
// ======================================================================================
// Camera frames (the per-camera rotation part of the projection, see CamRot) of
// cams[nc][9] into frames[nc][kFrame]; one thread per camera.
template <bool kJac>
__global__ void k_camera_frames(const double* __restrict__ cams, double* __restrict__ frames, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double* cam = cams + 9 * (size_t)c;
  const double aa[3] = {cam[0], cam[1], cam[2]};
  CamRot R;
  camera_rotation<kJac>(aa, R);
  frame_store<kJac>(frames + kFrame * (size_t)c, R, cam);
}

// kFrames: the cameras' rotation parts come from frames[nc][kFrame] (k_camera_frames
// of ba.cameras), and the slices follow the dynamic longest-first schedule with per-slice
// cost partials in slice_part (scratch); otherwise (the allocation-free entry, no
// scratch) every observation computes its camera's rotation and the CTAs take fixed
// slice sets (next_cta_slice) with per-CTA partials.
// Staging each lane's next two frames and observations into shared memory with cp.async
// (as the camera reduction does) ran slower here, 0.56 instead of 0.50 ms on the
// 6.0M-observation problem: the kernel is bound by its L1 data path (62% busy; 78% with
// the staging's copies and shared-memory reads), not by the latency of the gathers.
template <typename T, bool kJac, bool kFrames>
__global__ void __launch_bounds__(kWarpBlock, kJac ? CERES_B200_EVAL_MIN_BLOCKS : CERES_B200_EVAL_NOJAC_MIN_BLOCKS)
k_evaluate(ceres_b200_ba_t ba, double* partials, const double* __restrict__ frames, double* __restrict__ slice_part) {
  constexpr bool kDyn = kFrames;
  __shared__ double red[kWarpBlock / 32];
  const LossSpec L = loss_spec(ba);
  const int lane = threadIdx.x & 31;
  double cost = 0.0;
  unsigned err = 0;
  T* __restrict__ jac = reinterpret_cast<T*>(ba.jac);
  __shared__ int slice_counter;
  if (!kDyn) {
    if (threadIdx.x == 0) slice_counter = 0;
    __syncthreads();
  }
  auto next = [&]() -> int {
    return kDyn ? next_global_slice(&ba.counters[kCtrSliceEval], ba.num_slices)
                : next_cta_slice(&slice_counter, ba.num_slices);
  };
  for (int s = next(); s >= 0; s = next()) {
    double cs = 0.0;  // this lane's cost in slice s
    const int q = s * 32 + lane;
    const int len = ba.slice_len[s];
    const size_t base = (size_t)ba.slice_base[s];
    const double X[3] = {ba.points[3 * (size_t)q], ba.points[3 * (size_t)q + 1], ba.points[3 * (size_t)q + 2]};
    const bool pconst = ba.pt_const[q] != 0;
    // point sums J_p^T J_p (6) and J_p^T r (3) of this lane's track, from the stored
    // (precision-T) Jacobian, so the point side of the Schur system needs no pass over
    // the observations
    double W[6] = {0, 0, 0, 0, 0, 0}, g[3] = {0, 0, 0};
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k + lane;
      const int c = ba.slot_cam[slot];
      if (c < 0) continue;
      const double2 ob = reinterpret_cast<const double2*>(ba.slot_obs)[slot];
      // Jacobian in float64, rounded to T when stored: a Jacobian computed in float32
      // arithmetic (errors of ~1e-6 instead of the 6e-8 of rounding) made the mixed
      // LM solves of the 6.0M-observation problem take 1.3x the iterations
      Proj o;
      CamRot R;
      double tail[6];
      if (kFrames) {
        frame_load_wide<kJac>(frames + kFrame * (size_t)c, R, tail);
      } else {
        const double* cam = ba.cameras + 9 * (size_t)c;
        const double aa[3] = {cam[0], cam[1], cam[2]};
        camera_rotation<kJac>(aa, R);
#pragma unroll
        for (int i = 0; i < 6; ++i) tail[i] = cam[3 + i];
      }
      snavely_project<kJac>(R, tail, X, ob.x, ob.y, o);
      cs += robustify<kJac>(L, o, err);
      reinterpret_cast<double2*>(ba.res)[slot] = make_double2(o.r[0], o.r[1]);
      if (kJac) {
        if (ba.cam_const[c]) {
#pragma unroll
          for (int j = 0; j < 9; ++j) o.jc[0][j] = o.jc[1][j] = 0.0;
        }
        if (pconst) {
#pragma unroll
          for (int j = 0; j < 3; ++j) o.jp[0][j] = o.jp[1][j] = 0.0;
        }
        store_rec(jac, slot, o);
        // the camera-major copy, when the caller keeps one (the camera-side passes then
        // stream it in camera order instead of gathering records by slot)
        if (ba.cm_jac != nullptr) store_rec(reinterpret_cast<T*>(ba.cm_jac), (size_t)ba.slot_pos[slot], o);
        double a[3], b[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) { a[m] = (double)(T)o.jp[0][m]; b[m] = (double)(T)o.jp[1][m]; }
        W[0] += a[0] * a[0] + b[0] * b[0];
        W[1] += a[0] * a[1] + b[0] * b[1];
        W[2] += a[0] * a[2] + b[0] * b[2];
        W[3] += a[1] * a[1] + b[1] * b[1];
        W[4] += a[1] * a[2] + b[1] * b[2];
        W[5] += a[2] * a[2] + b[2] * b[2];
        // the gradient J_p^T r from the float64 Jacobian before rounding: with the float32
        // store, a gradient summed from rounded values moves the point where the step
        // vanishes along weakly determined directions (a point's depth)
#pragma unroll
        for (int m = 0; m < 3; ++m) g[m] += o.jp[0][m] * o.r[0] + o.jp[1][m] * o.r[1];
      }
    }
    if (kJac) {
      double* pr = ba.point_raw + 9 * (size_t)q;
#pragma unroll
      for (int i = 0; i < 6; ++i) pr[i] = W[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) pr[6 + i] = g[i];
    }
    if (kDyn) {
      const double w = warp_sum(cs);
      if (lane == 0) slice_part[s] = w;
    } else {
      cost += cs;
    }
  }
  if (err) atomicOr(&ba.counters[kCtrError], err);
  if (!kDyn) {  // with kDyn the sum is k_slice_fold's
    const int out[1] = {CERES_B200_STAT_COST};
    double v[1] = {cost};
    block_reduce<1>(v, 0u, red);
    grid_finish<1>(v, 0u, partials, &ba.counters[kCtrEval], ba.stats, out, red);
  }
}

// Deterministic sums of the dynamically scheduled slice kernels: the warp that took
// slice s wrote its NV sums (fixed lane order) to part[v * num_slices + s]; CTA b folds
// the fixed range of slices [b * chunk, (b + 1) * chunk) and the last CTA folds the CTA
// partials in CTA order (grid_finish), so the result does not depend on which warp took
// which slice. Runs after the slice kernel on the same stream and resets its counter.
template <int NV>
__global__ void __launch_bounds__(256) k_slice_fold(const double* __restrict__ part, int num_slices, int chunk,
                                                    double* partials, unsigned* ticket, unsigned* slice_counter,
                                                    double* stats, StatIdx<NV> out) {
  __shared__ double red[NV * 8];
  if (blockIdx.x == 0 && threadIdx.x == 0) *slice_counter = 0u;
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = 0.0;
  const int s0 = blockIdx.x * chunk, s1 = min(num_slices, s0 + chunk);
  for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] += part[(size_t)i * num_slices + s];
  }
  block_reduce<NV>(v, 0u, red);
  grid_finish<NV>(v, 0u, partials, ticket, stats, out.idx, red);
}

// The fold of the per-slice partials that follows a dynamically scheduled slice kernel.
template <int NV>
static void launch_slice_fold(const ceres_b200_ba_t& ba, const DevInfo& d, const double* part, double* partials,
                       int ticket_ctr, int slice_ctr, StatIdx<NV> out, cudaStream_t st) {
  int grid = (ba.num_slices + 255) / 256;
  if (grid > d.sms) grid = d.sms;
  if (grid < 1) grid = 1;
  const int chunk = (ba.num_slices + grid - 1) / grid;
  k_slice_fold<NV><<<grid, 256, 0, st>>>(part, ba.num_slices, chunk > 0 ? chunk : 1, partials, &ba.counters[ticket_ctr],
                                        &ba.counters[slice_ctr], ba.stats, out);
}

// ======================================================================================
// Point side: W_p = J_p^T J_p + D_p, its inverse, W^-1 g_a, point gradient
// ======================================================================================
template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_point_assemble(ceres_b200_ba_t ba, double inv_radius, double mn,
                                                               double mx, int jacobi_scaling, double* partials) {
  __shared__ double red[2 * (kWarpBlock / 32)];
  T* __restrict__ winv = reinterpret_cast<T*>(ba.winv);
  double gmax = 0.0, gsq = 0.0;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ba.num_points; q += gridDim.x * blockDim.x) {
    const double* pr = ba.point_raw + 9 * (size_t)q;
    double W[6], g[3];
#pragma unroll
    for (int i = 0; i < 6; ++i) W[i] = pr[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) g[i] = pr[6 + i];
    double inv[6] = {0, 0, 0, 0, 0, 0};
    double wga[3] = {0, 0, 0};
    if (!ba.pt_const[q]) {
      const int dg[3] = {0, 3, 5};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double col = jacobi_scaling ? W[dg[i]] : 1.0;
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
    for (int i = 0; i < 3; ++i) ba.winv_ga[3 * (size_t)q + i] = wga[i];
  }
  double v[2] = {gmax, gsq};
  block_reduce<2>(v, 1u, red);
  const int out[2] = {CERES_B200_STAT_GMAX_P, CERES_B200_STAT_GSQ_P};
  grid_finish<2>(v, 1u, partials, &ba.counters[kCtrPoint], ba.stats, out, red);
}

// ======================================================================================
// Camera side: one CTA per camera. Reduces J_c^T (I - J_p W^-1 J_p^T) J_c (the
// Schur diagonal block before damping), the camera column sums, the gradient and
// the reduced rhs over the camera's observations, then forms the preconditioner.
// ======================================================================================
constexpr int kCamBlock = 128;
constexpr int kCamAcc = 45 + 9 + 9 + 9;  // V (upper), colsum, g, h

__device__ __forceinline__ int tri9(int j, int l) {  // upper-triangle index, j <= l
  return j * 9 - (j * (j - 1)) / 2 + (l - j);
}

// The camera sums are float64 in both precisions. With the float32 store, float32
// accumulators (168 registers, three CTAs per SM: 0.34 instead of 0.42 ms on the
// 6.0M-observation problem) made the SCHUR_JACOBI blocks inaccurate enough to change
// PCG iteration counts: the mixed LM solves then took 71-176 iterations to the target
// (median 89, 9 runs) instead of 77-94 (median 90).

// One entry of a camera's observation list with the data its update reads.
template <typename T>
struct CamObs {
  int2 ent;  // (slot, sorted point)
  T rv[kRec];
  double2 r;
  T wi[6];
  double wg[3];
};

// Register path (float64 store): the record comes from the camera-major copy when there
// is one (entry e: consecutive threads read consecutive records), else from its slot;
// residual and point blocks are gathered by slot and point.
template <typename T>
__device__ __forceinline__ void cam_obs_load(const ceres_b200_ba_t& ba, const T* __restrict__ jac,
                                             const T* __restrict__ cm, const T* __restrict__ winv, int e, int2 ent,
                                             CamObs<T>& o) {
  o.ent = ent;
  if (cm != nullptr) load_rec(cm, (size_t)e, o.rv);
  else if constexpr (sizeof(T) == 4) load_rec128(jac, (size_t)ent.x, o.rv);
  else load_rec(jac, (size_t)ent.x, o.rv);
  o.r = reinterpret_cast<const double2*>(ba.res)[ent.x];
#pragma unroll
  for (int i = 0; i < 6; ++i) o.wi[i] = winv[6 * (size_t)ent.y + i];
#pragma unroll
  for (int i = 0; i < 3; ++i) o.wg[i] = ba.winv_ga[3 * (size_t)ent.y + i];
}

// Asynchronous staging of the camera reduction's inputs (cp.async, 16- and 8-byte
// copies). Each thread stages the observations it will reduce itself, kStages chunks
// ahead, into its own column of a structure-of-arrays stage (conflict-free reads);
// it only waits for its own copies (cp.async.wait_group), so no CTA barrier is needed.
// A stage is refilled after the thread has consumed the values it read from it.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The float32 store is staged; the float64 store's records (192 bytes) are loaded into
// registers just before use: staged through shared memory they ran slower (0.62 instead
// of 0.50 ms on the 6.0M-observation problem with two stages).
template <typename T>
struct CamStage {
  static constexpr bool kStaged = sizeof(T) == 4;
  static constexpr int kRecV = kRec * (int)sizeof(T) / 16;  // 16-byte pieces of a record
  static constexpr int kWiV = 6 * (int)sizeof(T) / 8;        // 8-byte pieces of W^-1
  static constexpr int kStages = 4;
  // per thread: record, residual, W^-1, W^-1 g, entry
  static constexpr size_t kStageBytes = (size_t)kCamBlock * (16 * kRecV + 16 + 8 * kWiV + 24 + 8);
  static constexpr size_t kBytes = kStaged ? kStages * kStageBytes : 0;
  static constexpr size_t kRes = (size_t)16 * kRecV * kCamBlock;
  static constexpr size_t kWi = kRes + (size_t)16 * kCamBlock;
  static constexpr size_t kWg = kWi + (size_t)8 * kWiV * kCamBlock;
  static constexpr size_t kEnt = kWg + (size_t)24 * kCamBlock;
};

// The record comes from the camera-major copy when there is one (entry e: consecutive
// threads read consecutive records), else from its slot; residual and point blocks are
// gathered by slot and point.
template <typename T>
__device__ __forceinline__ void cam_stage_issue(const ceres_b200_ba_t& ba, const T* __restrict__ jac,
                                                const T* __restrict__ cm, const T* __restrict__ winv, int e,
                                                int2 ent, char* stage) {
  using D = CamStage<T>;
  const int t = threadIdx.x;
  const uint4* rs = reinterpret_cast<const uint4*>(cm != nullptr ? cm + (size_t)e * kRec : jac + (size_t)ent.x * kRec);
  uint4* rd = reinterpret_cast<uint4*>(stage);
#pragma unroll
  for (int i = 0; i < D::kRecV; ++i) cp_async16(rd + i * kCamBlock + t, rs + i);
  cp_async16(reinterpret_cast<double2*>(stage + D::kRes) + t, reinterpret_cast<const double2*>(ba.res) + ent.x);
  const uint2* ws = reinterpret_cast<const uint2*>(winv + 6 * (size_t)ent.y);
  uint2* wd = reinterpret_cast<uint2*>(stage + D::kWi);
#pragma unroll
  for (int i = 0; i < D::kWiV; ++i) cp_async8(wd + i * kCamBlock + t, ws + i);
  double* gd = reinterpret_cast<double*>(stage + D::kWg);
#pragma unroll
  for (int i = 0; i < 3; ++i) cp_async8(gd + i * kCamBlock + t, ba.winv_ga + 3 * (size_t)ent.y + i);
  reinterpret_cast<int2*>(stage + D::kEnt)[t] = ent;
}

template <typename T>
__device__ __forceinline__ void cam_stage_read(const char* stage, CamObs<T>& o) {
  using D = CamStage<T>;
  const int t = threadIdx.x;
  const uint4* rd = reinterpret_cast<const uint4*>(stage);
#pragma unroll
  for (int i = 0; i < D::kRecV; ++i) {
    const uint4 v = rd[i * kCamBlock + t];
    if constexpr (sizeof(T) == 4) {
      o.rv[4 * i] = __uint_as_float(v.x); o.rv[4 * i + 1] = __uint_as_float(v.y);
      o.rv[4 * i + 2] = __uint_as_float(v.z); o.rv[4 * i + 3] = __uint_as_float(v.w);
    } else {
      o.rv[2 * i] = __hiloint2double((int)v.y, (int)v.x);
      o.rv[2 * i + 1] = __hiloint2double((int)v.w, (int)v.z);
    }
  }
  o.r = reinterpret_cast<const double2*>(stage + D::kRes)[t];
  const uint2* wd = reinterpret_cast<const uint2*>(stage + D::kWi);
#pragma unroll
  for (int i = 0; i < D::kWiV; ++i) {
    const uint2 v = wd[i * kCamBlock + t];
    if constexpr (sizeof(T) == 4) {
      o.wi[2 * i] = __uint_as_float(v.x); o.wi[2 * i + 1] = __uint_as_float(v.y);
    } else {
      o.wi[i] = __hiloint2double((int)v.y, (int)v.x);
    }
  }
  const double* gd = reinterpret_cast<const double*>(stage + D::kWg);
#pragma unroll
  for (int i = 0; i < 3; ++i) o.wg[i] = gd[i * kCamBlock + t];
  o.ent = reinterpret_cast<const int2*>(stage + D::kEnt)[t];
}

// Warp sums of 72 values, scattered over the lanes (recursive halving): at the xor
// distances 16, 8, 4, 2, 1 each lane keeps one half of its values and adds the partner's
// copy of that half, so it ends with the sums of (at most) 3 indices, 36 b4 + 18 b3 +
// 9 b2 + 5 b1 + 3 b0 + k (b: the lane's bits; k < 3, 3 b0 + k < 5, index within the
// group of 9 below 9), each added over the same xor tree as warp_sum, so the sums are
// warp_sum's bit for bit, in about half the instructions.
__device__ __forceinline__ void warp_reduce_scatter72(double (&v)[72], int lane) {
  constexpr unsigned kFull = 0xffffffffu;
  {
    const bool hi = (lane & 16) != 0;
#pragma unroll
    for (int j = 0; j < 36; ++j) {
      const double keep = hi ? v[j + 36] : v[j], send = hi ? v[j] : v[j + 36];
      v[j] = keep + __shfl_xor_sync(kFull, send, 16);
    }
  }
  {
    const bool hi = (lane & 8) != 0;
#pragma unroll
    for (int j = 0; j < 18; ++j) {
      const double keep = hi ? v[j + 18] : v[j], send = hi ? v[j] : v[j + 18];
      v[j] = keep + __shfl_xor_sync(kFull, send, 8);
    }
  }
  {
    const bool hi = (lane & 4) != 0;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
      const double keep = hi ? v[j + 9] : v[j], send = hi ? v[j] : v[j + 9];
      v[j] = keep + __shfl_xor_sync(kFull, send, 4);
    }
  }
  v[9] = 0.0;  // 9 values: padded to 10
  {
    const bool hi = (lane & 2) != 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const double keep = hi ? v[j + 5] : v[j], send = hi ? v[j] : v[j + 5];
      v[j] = keep + __shfl_xor_sync(kFull, send, 2);
    }
  }
  v[5] = 0.0;  // 5 values: padded to 6
  {
    const bool hi = (lane & 1) != 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double keep = hi ? v[j + 3] : v[j], send = hi ? v[j] : v[j + 3];
      v[j] = keep + __shfl_xor_sync(kFull, send, 1);
    }
  }
}

// Phase 1: one CTA per camera reduces the 72 sums over the camera's observations
// into acc_out[c][72] (float64). kHbb: the camera block is the Hbb block sum Jc^T Jc
// (M = I below) instead of the Schur block; the base of SCHUR_POWER_SERIES_EXPANSION.
// Thread t reduces the camera's entries t, t + 128, ...; with the float32 store their
// inputs arrive through the cp.async stages (CamStage), kStages observations ahead.
// (Cutting the camera-major list into equal ranges, one resident CTA each, with
// per-camera segment sums folded afterwards, ran slower: 0.42 instead of 0.39 ms mixed
// and 0.64 instead of 0.55 ms float64 for the assembly of the 6.0M-observation problem.)
template <typename T, bool kDup, bool kHbb = false>
__global__ void __launch_bounds__(kCamBlock) k_camera_reduce(ceres_b200_ba_t ba, double* __restrict__ acc_out) {
  using A = double;
  using D = CamStage<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double sred[kCamAcc * (kCamBlock / 32)];
  const int c = blockIdx.x;
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ cm = reinterpret_cast<const T*>(ba.cm_jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  const int e0 = ba.cam_offsets[c], e1 = ba.cam_offsets[c + 1];
  {
    A av[54];      // Schur block (upper triangle, 45), column sums (9)
    double ag[18]; // gradient (9), reduced rhs (9)
#pragma unroll
    for (int i = 0; i < 54; ++i) av[i] = (A)0;
#pragma unroll
    for (int i = 0; i < 18; ++i) ag[i] = 0.0;
    const bool cconst = ba.cam_const[c] != 0;
    if (!cconst) {
      const int2* __restrict__ ents = reinterpret_cast<const int2*>(ba.cam_entries);
      const int stride = blockDim.x;
      const int first = e0 + threadIdx.x;
      char* stages = reinterpret_cast<char*>(smem_raw);
      int en_i = first, st = 0;
      int2 en_next = make_int2(0, 0), en2 = make_int2(0, 0);
      if constexpr (D::kStaged) {
#pragma unroll
        for (int k = 0; k < D::kStages; ++k) {
          const int e = first + k * stride;
          if (e < e1) cam_stage_issue<T>(ba, jac, cm, winv, e, ents[e], stages + k * D::kStageBytes);
          cp_async_commit();
        }
        en_i = first + D::kStages * stride;                  // the next entry to stage
        en_next = en_i < e1 ? ents[en_i] : make_int2(0, 0);  // its (slot, point), read one chunk early
      } else {
        // entries are read two observations ahead, so each observation waits for one
        // gather (its data) instead of two (entry, then data)
        en_next = first < e1 ? ents[first] : make_int2(0, 0);
        en2 = first + stride < e1 ? ents[first + stride] : make_int2(0, 0);
      }
      for (int e = first; e < e1; e += stride) {
        CamObs<T> cur;
        if constexpr (D::kStaged) {
          cp_async_wait<D::kStages - 1>();
          cam_stage_read<T>(stages + st * D::kStageBytes, cur);
        } else {
          cam_obs_load<T>(ba, jac, cm, winv, e, en_next, cur);
          en_next = en2;
          en2 = e + 2 * stride < e1 ? ents[e + 2 * stride] : make_int2(0, 0);
        }
        const size_t slot = (size_t)cur.ent.x;
        const int q = cur.ent.y;
        const T* rv = cur.rv;
        const double2 r = cur.r;
        A wi[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) wi[i] = (A)cur.wi[i];
        const double* wg = cur.wg;
        A jp0[3], jp1[3];
#pragma unroll
        for (int m = 0; m < 3; ++m) { jp0[m] = (A)rv[18 + m]; jp1[m] = (A)rv[21 + m]; }
        // P = Jp W^-1 (2x3); B = P Jp^T (2x2); a = Jp W^-1 g_a
        A P0[3], P1[3];
        P0[0] = wi[0] * jp0[0] + wi[1] * jp0[1] + wi[2] * jp0[2];
        P0[1] = wi[1] * jp0[0] + wi[3] * jp0[1] + wi[4] * jp0[2];
        P0[2] = wi[2] * jp0[0] + wi[4] * jp0[1] + wi[5] * jp0[2];
        P1[0] = wi[0] * jp1[0] + wi[1] * jp1[1] + wi[2] * jp1[2];
        P1[1] = wi[1] * jp1[0] + wi[3] * jp1[1] + wi[4] * jp1[2];
        P1[2] = wi[2] * jp1[0] + wi[4] * jp1[1] + wi[5] * jp1[2];
        const A B00 = P0[0] * jp0[0] + P0[1] * jp0[1] + P0[2] * jp0[2];
        const A B01 = P0[0] * jp1[0] + P0[1] * jp1[1] + P0[2] * jp1[2];
        const A B11 = P1[0] * jp1[0] + P1[1] * jp1[1] + P1[2] * jp1[2];
        const double a0 = (double)rv[18] * wg[0] + (double)rv[19] * wg[1] + (double)rv[20] * wg[2];
        const double a1 = (double)rv[21] * wg[0] + (double)rv[22] * wg[1] + (double)rv[23] * wg[2];
        const A M00 = kHbb ? (A)1 : (A)1 - B00, M01 = kHbb ? (A)0 : -B01, M11 = kHbb ? (A)1 : (A)1 - B11;
        A K0[9], K1[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) {
          const A c0 = (A)rv[j], c1 = (A)rv[9 + j];
          K0[j] = M00 * c0 + M01 * c1;
          K1[j] = M01 * c0 + M11 * c1;
          av[45 + j] += c0 * c0 + c1 * c1;
          const double d0 = (double)rv[j], d1 = (double)rv[9 + j];
          ag[j] += d0 * r.x + d1 * r.y;
          ag[9 + j] += d0 * (r.x + a0) + d1 * (r.y + a1);
        }
#pragma unroll
        for (int j = 0; j < 9; ++j)
#pragma unroll
          for (int l = j; l < 9; ++l) av[tri9(j, l)] += (A)rv[j] * K0[l] + (A)rv[9 + j] * K1[l];

        if (kDup && !kHbb) {
          // other observations of the same point in this camera: -Jc_i^T P_i Jp_k^T Jc_k
          const int sidx = q >> 5, ln = q & 31;
          const int len = ba.slice_len[sidx];
          const size_t sb = (size_t)ba.slice_base[sidx];
          for (int k = 0; k < len; ++k) {
            const size_t slot2 = sb + 32 * (size_t)k + ln;
            if (slot2 == slot || ba.slot_cam[slot2] != c) continue;
            T rk[kRec];
            load_rec(jac, slot2, rk);
            const A C00 = P0[0] * (A)rk[18] + P0[1] * (A)rk[19] + P0[2] * (A)rk[20];
            const A C01 = P0[0] * (A)rk[21] + P0[1] * (A)rk[22] + P0[2] * (A)rk[23];
            const A C10 = P1[0] * (A)rk[18] + P1[1] * (A)rk[19] + P1[2] * (A)rk[20];
            const A C11 = P1[0] * (A)rk[21] + P1[1] * (A)rk[22] + P1[2] * (A)rk[23];
#pragma unroll
            for (int j = 0; j < 9; ++j) {
              const A t0 = (A)rv[j] * C00 + (A)rv[9 + j] * C10;
              const A t1 = (A)rv[j] * C01 + (A)rv[9 + j] * C11;
#pragma unroll
              for (int l = j; l < 9; ++l) av[tri9(j, l)] -= t0 * (A)rk[l] + t1 * (A)rk[9 + l];
            }
          }
        }
        if constexpr (D::kStaged) {
          // refill this stage with the observation kStages chunks ahead (its values are consumed)
          if (en_i < e1) cam_stage_issue<T>(ba, jac, cm, winv, en_i, en_next, stages + st * D::kStageBytes);
          cp_async_commit();
          en_i += stride;
          en_next = en_i < e1 ? ents[en_i] : make_int2(0, 0);
          st = st + 1 == D::kStages ? 0 : st + 1;
        }
      }
      if constexpr (D::kStaged) cp_async_wait<0>();
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    {
      double v[72];
#pragma unroll
      for (int i = 0; i < 54; ++i) v[i] = (double)av[i];
#pragma unroll
      for (int i = 0; i < 18; ++i) v[54 + i] = ag[i];
      warp_reduce_scatter72(v, lane);
      const int base = 36 * ((lane >> 4) & 1) + 18 * ((lane >> 3) & 1) + 9 * ((lane >> 2) & 1);
      const int l0 = 5 * ((lane >> 1) & 1), s0 = 3 * (lane & 1);
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (s0 + k < 5 && l0 + s0 + k < 9) sred[(base + l0 + s0 + k) * nw + wid] = v[k];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kCamAcc; i += blockDim.x) {
      double sum = 0.0;
      for (int w = 0; w < nw; ++w) sum += sred[i * nw + w];
      acc_out[(size_t)c * kCamAcc + i] = sum;
    }
  }
}

// Phase 2: one warp per camera forms the damping, the reduced rhs, the gradient stats
// and the preconditioner block from the 72 sums. Lane i < 9 holds row i of the
// damped Schur block S; the SCHUR_JACOBI inverse is the Cholesky factorisation and
// the two triangular solves of block9_inverse, spread over the lanes (row i of L on
// lane i, column c of the inverse on lane c) with the same operation order, so it
// gives block9_inverse's result. A block that is not positive definite goes to
// block9_inverse's pivoted Gauss-Jordan on lane 0 (linear.py:1156-1182 falls back
// from Cholesky to a general solve the same way).
constexpr int kFinishWarps = 4;  // cameras per CTA

template <typename T>
__global__ void __launch_bounds__(32 * kFinishWarps) k_camera_finish(ceres_b200_ba_t ba, const double* __restrict__ acc_in,
                                                                     double inv_radius, double mn, double mx,
                                                                     int jacobi_scaling, int precond, double* partials,
                                                                     double* __restrict__ pre_out) {
  constexpr unsigned kFull = 0xffffffffu;
  __shared__ double sred2[2 * kFinishWarps];
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kFinishWarps + (threadIdx.x >> 5);
  double gmax = 0.0, gsq = 0.0;
  if (c < ba.num_cameras) {  // uniform in the warp
    const double* sacc = acc_in + (size_t)c * kCamAcc;
    double* __restrict__ pre = pre_out + 81 * (size_t)c;
    double* dc = ba.cam_diag + 9 * (size_t)c;
    double* rh = ba.rhs + 9 * (size_t)c;
    if (ba.cam_const[c]) {
      if (lane < 9) { dc[lane] = 0.0; rh[lane] = 0.0; }
      for (int i = lane; i < 81; i += 32) pre[i] = (i % 10 == 0) ? 1.0 : 0.0;
    } else {
      const int i = lane < 9 ? lane : 8;  // lanes 9..31 shadow row 8 and store nothing
      const double col = jacobi_scaling ? sacc[45 + i] : 1.0;
      const double di = fmin(fmax(col, mn), mx) * inv_radius;
      if (lane < 9) {
        dc[i] = di;
        rh[i] = -sacc[63 + i];
        const double gi = sacc[54 + i];
        gmax = fabs(gi);
        gsq = gi * gi;
      }
      double a[9];  // row i of S = V + D
#pragma unroll
      for (int l = 0; l < 9; ++l) a[l] = sacc[l < i ? tri9(l, i) : tri9(i, l)] + (l == i ? di : 0.0);
      if (precond == CERES_B200_PRECOND_SCHUR_JACOBI) {
        double Lr[9];  // row i of L (entries 0..i)
        bool pd = true;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
          double Lj[9];
#pragma unroll
          for (int k = 0; k < j; ++k) Lj[k] = __shfl_sync(kFull, Lr[k], j);
          double d = __shfl_sync(kFull, a[j], j);
#pragma unroll
          for (int k = 0; k < j; ++k) d -= Lj[k] * Lj[k];
          if (!(d > 0.0)) { pd = false; break; }  // every lane computed the same d
          const double ljj = sqrt(d);
          double sj = a[j];
#pragma unroll
          for (int k = 0; k < j; ++k) sj -= Lr[k] * Lj[k];
          Lr[j] = (i == j) ? ljj : sj / ljj;
        }
        if (pd) {
          double Lf[45];  // packed lower triangle of L: row r, column k at r (r + 1) / 2 + k
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
          double S[81], inv[81];
          for (int j = 0; j < 9; ++j) {
            const double dj = fmin(fmax(jacobi_scaling ? sacc[45 + j] : 1.0, mn), mx) * inv_radius;
            for (int l = j; l < 9; ++l) {
              const double v = sacc[tri9(j, l)] + (j == l ? dj : 0.0);
              S[j * 9 + l] = v;
              S[l * 9 + j] = v;
            }
          }
          block9_inverse(S, inv);
          for (int k = 0; k < 81; ++k) pre[k] = inv[k];
        }
      } else if (lane < 9) {
        double sii = 0.0;
#pragma unroll
        for (int l = 0; l < 9; ++l) sii = (l == i) ? a[l] : sii;
        const double v = (precond == CERES_B200_PRECOND_JACOBI) ? 1.0 / fmax(sii, kEps64) : 1.0;
#pragma unroll
        for (int l = 0; l < 9; ++l) pre[i * 9 + l] = l == i ? v : 0.0;
      }
    }
  }
  double v[2] = {gmax, gsq};
  block_reduce<2>(v, 1u, sred2);
  const int out[2] = {CERES_B200_STAT_GMAX_C, CERES_B200_STAT_GSQ_C};
  grid_finish<2>(v, 1u, partials, &ba.counters[kCtrCamera], ba.stats, out, sred2);
}

// ======================================================================================
// Implicit Schur product S p = (U + D) p - H_cp W^-1 H_pc p in two passes that need no
// atomics and give the same sums whatever the schedule:
//   point pass  (point-major store, lane = point, a warp per slice):
//                 s_q = W_q^-1 sum_k Jp_k^T (Jc_k p_c(k))
//   camera pass (camera-major copy, a warp per camera work item):
//                 y_item = sum over the item's entries of Jc^T (Jc p_c - Jp s_q)
//               summed across the warp by a fixed shuffle tree; a camera's items are then
//               added in item order (fold_items).
// kE: the eliminated term E p = H_cp W^-1 H_pc p only, y = sum Jc^T Jp s_q (the
// SCHUR_POWER_SERIES_EXPANSION series multiplies by E).
// ======================================================================================
// Observations processed per step of a lane's walk: their loads are all issued before
// any is used, so a warp keeps two records in flight per lane.
constexpr int kUnroll = 2;

template <typename T, typename TP, typename A, bool kCrossP>
__device__ __forceinline__ void camera_product(const T* rv, const TP* __restrict__ pc, A& u0, A& u1) {
  u0 = 0;
  u1 = 0;
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    const A pj = kCrossP ? (A)ld_cross(pc + j) : (A)pc[j];
    u0 += (A)rv[j] * pj;
    u1 += (A)rv[9 + j] * pj;
  }
}

// Point pass of slice s: sv[q] = W_q^-1 t_q with t_q = sum_k Jp_k^T (Jc_k p_c(k)) (float64).
template <typename T, typename TP, typename A, bool kCrossP>
__device__ __forceinline__ void point_pass_slice(const ceres_b200_ba_t& ba, const TP* __restrict__ pvec,
                                                 double* __restrict__ sv, int s, int lane) {
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  const int q = s * 32 + lane;
  const int len = ba.slice_len[s];
  const size_t base = (size_t)ba.slice_base[s] + lane;
  // padding slots hold zero Jacobians and camera -1; they are read like any slot
  // (camera 0 stands in for the address) and add nothing
  A t0 = 0, t1 = 0, t2 = 0;
  int k = 0;
  for (; k + kUnroll <= len; k += kUnroll) {
    int c[kUnroll];
    T rv[kUnroll][kRec];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const size_t slot = base + 32 * (size_t)(k + u);
      c[u] = ba.slot_cam[slot];
      load_rec(jac, slot, rv[u]);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      A u0, u1;
      camera_product<T, TP, A, kCrossP>(rv[u], pvec + 9 * (size_t)max(c[u], 0), u0, u1);
      t0 += (A)rv[u][18] * u0 + (A)rv[u][21] * u1;
      t1 += (A)rv[u][19] * u0 + (A)rv[u][22] * u1;
      t2 += (A)rv[u][20] * u0 + (A)rv[u][23] * u1;
    }
  }
  for (; k < len; ++k) {
    const size_t slot = base + 32 * (size_t)k;
    const int c = ba.slot_cam[slot];
    T rv[kRec];
    load_rec(jac, slot, rv);
    A u0, u1;
    camera_product<T, TP, A, kCrossP>(rv, pvec + 9 * (size_t)max(c, 0), u0, u1);
    t0 += (A)rv[18] * u0 + (A)rv[21] * u1;
    t1 += (A)rv[19] * u0 + (A)rv[22] * u1;
    t2 += (A)rv[20] * u0 + (A)rv[23] * u1;
  }
  const T* wi = winv + 6 * (size_t)q;
  const A w0 = (A)wi[0], w1 = (A)wi[1], w2 = (A)wi[2], w3 = (A)wi[3], w4 = (A)wi[4], w5 = (A)wi[5];
  double* o = sv + 3 * (size_t)q;
  o[0] = (double)(w0 * t0 + w1 * t1 + w2 * t2);
  o[1] = (double)(w1 * t0 + w3 * t1 + w4 * t2);
  o[2] = (double)(w2 * t0 + w4 * t1 + w5 * t2);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_any(double v) { return warp_sum(v); }
__device__ __forceinline__ float warp_sum_any(float v) { return warp_sum_f(v); }

// Camera pass of work item `item` (camera c, entries e0..e1-1 of the camera-major copy):
// y = sum_e Jc_e^T (Jc_e p_c - Jp_e s_q(e)) (kE: Jc_e^T Jp_e s_q(e)). Lane l takes
// entries e0 + l, e0 + l + 32, ...; the 32 lane sums are added by a butterfly whose
// pairwise additions commute, so every lane ends with the same bits. sv was written by
// other CTAs of the same launch (read through L2).
template <typename T, typename TP, typename A, bool kCrossP, bool kE>
__device__ __forceinline__ int camera_pass_item(const ceres_b200_ba_t& ba, const TP* __restrict__ pvec,
                                                const double* __restrict__ sv, int item, int lane, A y[9]) {
  const int2 it = reinterpret_cast<const int2*>(ba.items)[item];
  const int c = it.x, e0 = it.y;
  // the item ends where the camera's next item starts, or with the camera's entries
  const int e1 = item + 1 < ba.cam_items[c + 1] ? reinterpret_cast<const int2*>(ba.items)[item + 1].y
                                                : ba.cam_offsets[c + 1];
  const T* __restrict__ cm = reinterpret_cast<const T*>(ba.cm_jac);
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const int2* __restrict__ ents = reinterpret_cast<const int2*>(ba.cam_entries);
  // the record of entry e: streamed from the camera-major copy, or gathered by slot
  auto load = [&](int e, T rv[kRec], int& q) {
    const int2 en = ents[e];
    q = en.y;
    if (cm != nullptr) load_rec(cm, (size_t)e, rv);
    else if constexpr (sizeof(T) == 4) load_rec128(jac, (size_t)en.x, rv);
    else load_rec(jac, (size_t)en.x, rv);
  };
  A pc[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) {
    pc[j] = 0;
    if (!kE) pc[j] = kCrossP ? (A)ld_cross(pvec + 9 * (size_t)c + j) : (A)pvec[9 * (size_t)c + j];
    y[j] = 0;
  }
  auto one = [&](const T* rv, int q) {
    const double* sq = sv + 3 * (size_t)q;
    const A s0 = (A)ld_cross(sq), s1 = (A)ld_cross(sq + 1), s2 = (A)ld_cross(sq + 2);
    A v0 = (A)rv[18] * s0 + (A)rv[19] * s1 + (A)rv[20] * s2;
    A v1 = (A)rv[21] * s0 + (A)rv[22] * s1 + (A)rv[23] * s2;
    if constexpr (!kE) {
      A u0 = 0, u1 = 0;
#pragma unroll
      for (int j = 0; j < 9; ++j) {
        u0 += (A)rv[j] * pc[j];
        u1 += (A)rv[9 + j] * pc[j];
      }
      v0 = u0 - v0;
      v1 = u1 - v1;
    }
#pragma unroll
    for (int j = 0; j < 9; ++j) y[j] += (A)rv[j] * v0 + (A)rv[9 + j] * v1;
  };
  int e = e0 + lane;
  for (; e + 32 * (kUnroll - 1) < e1; e += 32 * kUnroll) {
    T rv[kUnroll][kRec];
    int q[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) load(e + 32 * u, rv[u], q[u]);
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) one(rv[u], q[u]);
  }
  for (; e < e1; e += 32) {
    T rv[kRec];
    int q;
    load(e, rv, q);
    one(rv, q);
  }
#pragma unroll
  for (int j = 0; j < 9; ++j) y[j] = warp_sum_any(y[j]);
  return c;
}

// The camera pass over a range of warps: warp gw of nw takes items gw, gw + nw, ... and
// writes each item's 9 sums (float64) to part[item]. Returns this thread's share of
// sum_items dot_p_c . y_item (lane 0 only; 0 elsewhere) when dot_p is set.
template <typename T, typename TP, typename A, bool kCrossP, bool kE>
__device__ __forceinline__ double camera_pass(const ceres_b200_ba_t& ba, const TP* __restrict__ pvec,
                                              const double* __restrict__ sv, double* __restrict__ part,
                                              const double* __restrict__ dot_p, int gw, int nw) {
  const int lane = threadIdx.x & 31;
  double dot = 0.0;
  for (int i = gw; i < ba.num_items; i += nw) {
    A y[9];
    const int c = camera_pass_item<T, TP, A, kCrossP, kE>(ba, pvec, sv, i, lane, y);
    double mine = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) mine = (lane == j) ? (double)y[j] : mine;
    if (lane < 9) part[9 * (size_t)i + lane] = mine;
    if (dot_p != nullptr && lane == 0) {
      double d = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) d += ld_cross(dot_p + 9 * (size_t)c + j) * (double)y[j];
      dot += d;
    }
  }
  return dot;
}

// out[j] for camera entries j in [j0, j1): the camera's item sums in item order, plus
// D V when add_diag. Returns this thread's share of sum_j V_j out_j.
__device__ __forceinline__ double fold_items(const ceres_b200_ba_t& ba, const double* __restrict__ part,
                                             const double* __restrict__ V, double* __restrict__ out, int j0, int j1,
                                             bool add_diag) {
  double dot = 0.0;
  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const int c = j / 9, m = j - 9 * c;
    double y = 0.0;
    const int i1 = ba.cam_items[c + 1];
    for (int i = ba.cam_items[c]; i < i1; ++i) y += ld_cross(part + 9 * (size_t)i + m);
    const double vj = ld_cross(V + j);
    if (add_diag) y += ba.cam_diag[j] * vj;
    out[j] = y;
    dot += vj * y;
  }
  return dot;
}

// y = S x for the test entry point: the same two passes in float64 arithmetic, one
// launch each, then the fold.
template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_point_pass64(ceres_b200_ba_t ba, const double* __restrict__ x,
                                                             double* __restrict__ sv) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = gw; s < ba.num_slices; s += nw) point_pass_slice<T, double, double, true>(ba, x, sv, s, lane);
}

template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_camera_pass64(ceres_b200_ba_t ba, const double* __restrict__ x,
                                                              const double* __restrict__ sv, double* __restrict__ part) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  (void)camera_pass<T, double, double, true, false>(ba, x, sv, part, nullptr, gw, nw);
}

__global__ void k_fold_items(ceres_b200_ba_t ba, const double* __restrict__ part, const double* __restrict__ x,
                             double* __restrict__ y) {
  const int n = 9 * ba.num_cameras;
  const int j0 = blockIdx.x * blockDim.x;
  const int j1 = min(n, j0 + (int)blockDim.x);
  (void)fold_items(ba, part, x, y, j0, j1, true);
}

// ======================================================================================
// Cooperative persistent PCG (linear.py:1216-1256) on the reduced camera system, with
// the float64 refinement of the float32 store in the same launch.
// ======================================================================================
// Device view of ceres_b200_clusters_t (the visibility-cluster preconditioner).
struct ClusterArgs {
  int num_components, num_pairs, max_dim, tridiagonal;
  const int2* pairs;
  const int2* entries;
  const int* cam_comp;
  const int* cam_pos;
  const int* cam_cluster;
  const int* comp_cams;
  const int* comp_cam_off;
  const long long* comp_base;
  const long long* comp_piv;
  double* inv;
  double* piv;
  unsigned* flags;
};

struct PcgArgs {
  const double* rhs;   // [n] right-hand side (float64)
  double* x_out;       // [n] solution (float64)
  int min_iterations, max_iterations;
  double tolerance, eps;
  int n;               // 9 * num_cameras
  int cams_per_cta;
  int smem_vectors;    // 1: a copy of p in shared memory for the product
  double* sv;          // [num_points][3] point-pass results s_q
  double* item_part;   // [num_items][9] camera-pass item sums
  double* part_b;      // [G]
  double* part_c;      // [G][2]
  double* r64;         // [n] refinement right-hand side rhs - S x
  int stall_window;    // > 0: stop when |r| has not dropped below 0.99 of its best for this many iterations
  int max_refinements; // float32 store: float64 refinement passes after a solve that missed the tolerance
  // SCHUR_POWER_SERIES_EXPANSION (linear.py:59-67, :482-497, :745-756)
  int precond_series;      // z = sum_i (B E)^i B r with B = ba.precond (inverted damped Hbb blocks)
  int init_series;         // x0 = the series applied to rhs with B = init_blocks
  const double* init_blocks; // [nc][81]
  int series_terms;        // max_num_spse_iterations (>= 1)
  double series_tol;       // spse_tolerance
  double* part_s;          // [G][2] partials of the series norms and of |r|^2
  // CLUSTER_JACOBI / CLUSTER_TRIDIAGONAL: z = M^-1 r with the component inverses of cl
  int cluster;
  ClusterArgs cl;
};

constexpr int kPcgBlock = 512;
constexpr int kStallWindow = 20;  // float32 PCG: iterations without a 1% residual drop before it stops

__device__ __forceinline__ void precond_apply(const double* __restrict__ Minv, const double* __restrict__ r,
                                              double* __restrict__ z, int c) {
  const double* M = Minv + 81 * (size_t)c;
  const double* rc = r + 9 * (size_t)c;
  double rr[9];
#pragma unroll
  for (int j = 0; j < 9; ++j) rr[j] = (double)rc[j];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 9; ++j) s += M[i * 9 + j] * rr[j];
    z[9 * (size_t)c + i] = s;
  }
}

// z_j = (M^-1 r)_j for the entries j in [j0, j1) (whole cameras): one warp per entry,
// the lanes over the columns of the camera's component (a fixed shuffle tree sums them,
// so the result does not depend on the schedule). r is complete in global memory (a
// grid barrier precedes the call). Cameras outside every component get z = 0.
__device__ __forceinline__ void cluster_apply(const ClusterArgs& cl, const double* __restrict__ r,
                                              double* __restrict__ z, int j0, int j1) {
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int j = j0 + (threadIdx.x >> 5); j < j1; j += nwarps) {
    const int c = j / 9, m = j - 9 * c;
    const int comp = cl.cam_comp[c];
    double acc = 0.0;
    if (comp >= 0) {
      const int cam0 = cl.comp_cam_off[comp];
      const int dim = 9 * (cl.comp_cam_off[comp + 1] - cam0);
      const double* __restrict__ row = cl.inv + cl.comp_base[comp] + (size_t)(9 * cl.cam_pos[c] + m) * dim;
      for (int col = lane; col < dim; col += 32) {
        const int k = col / 9;
        acc += row[col] * ld_cross(r + 9 * (size_t)cl.comp_cams[cam0 + k] + (col - 9 * k));
      }
      acc = warp_sum(acc);
    }
    if (lane == 0) z[j] = acc;
  }
}

// Sum of the G per-CTA partials part[g * stride + off] (NV values), computed by the
// whole CTA (thread g loads partial g) and broadcast to every thread. Every CTA
// folds the same values in the same order, so all CTAs agree bit for bit.
template <int NV>
__device__ __forceinline__ void cta_sum_partials(const double* part, int G, int stride, double out[NV],
                                                 double* red, double* bcast) {
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = 0.0;
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] += ld_cross(part + (size_t)g * stride + i);
  }
  block_reduce<NV>(v, 0u, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) bcast[i] = v[i];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) out[i] = bcast[i];
  __syncthreads();
}

// Product kinds of the persistent PCG: S and E in the store's precision T, S in
// float64 arithmetic (the float32 store's refinement residual)
enum { kProdS = 0, kProdE = 1, kProdS64 = 2 };

template <typename T>
__global__ void __launch_bounds__(kPcgBlock, 1) k_pcg(ceres_b200_ba_t ba, PcgArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[2 * (kPcgBlock / 32)];
  __shared__ double bcast[4];
  __shared__ int slice_counter;
  const int n = a.n;
  double* ps = reinterpret_cast<double*>(smem_raw);
  // PCG state vectors are float64 in both precisions, and so is the arithmetic of the
  // products S p and E p: they stream the Jacobian store in T (half the bytes when T is
  // float) and compute in float64. Float32 arithmetic would cost the same time (the
  // passes are bound by the store's bytes) but adds errors of 1e-7 |U| |p| to each
  // product, which swamp the small eigenvalues of S once the LM damping has decayed:
  // the steps then stop converging in the weakly determined directions and the solve
  // ends above the float64 minimum.
  double* __restrict__ X = reinterpret_cast<double*>(ba.pcg_x);
  double* __restrict__ R = reinterpret_cast<double*>(ba.pcg_r);
  double* __restrict__ Z = reinterpret_cast<double*>(ba.pcg_z);
  double* __restrict__ Pbuf = reinterpret_cast<double*>(ba.pcg_p);
  double* __restrict__ AP = reinterpret_cast<double*>(ba.pcg_ap);
  const double* __restrict__ Minv = reinterpret_cast<const double*>(ba.precond);
  const GridBarrier gb{&ba.counters[kCtrBarCount], &ba.counters[kCtrBarGen], &ba.counters[kCtrBarFlag], kSpinLimit};
  const int G = gridDim.x;
  const int c0 = blockIdx.x * a.cams_per_cta;
  const int c1 = min(ba.num_cameras, c0 + a.cams_per_cta);
  const int j0 = 9 * c0, j1 = 9 * max(c0, c1);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (G * blockDim.x) >> 5;

  // point pass of this CTA's slices (the balanced CTA schedule of next_cta_slice) with p
  // from ps (shared memory, T) or V (global memory, float64)
  auto point_pass = [&](const double* V, int kind) {
    if (threadIdx.x == 0) slice_counter = 0;
    __syncthreads();
    for (int s = next_cta_slice(&slice_counter, ba.num_slices); s >= 0; s = next_cta_slice(&slice_counter, ba.num_slices)) {
      if (kind != kProdS64 && a.smem_vectors) point_pass_slice<T, double, double, false>(ba, ps, a.sv, s, lane);
      else point_pass_slice<T, double, double, true>(ba, V, a.sv, s, lane);
    }
  };
  // camera pass over the grid's warps; returns this thread's share of
  // sum_items V_c . y_item (when with_dot)
  auto camera_pass_all = [&](const double* V, int kind, bool with_dot) -> double {
    const double* dp = with_dot ? V : nullptr;
    if (kind == kProdE) {
      if (a.smem_vectors) return camera_pass<T, double, double, false, true>(ba, ps, a.sv, a.item_part, dp, gw, nw);
      return camera_pass<T, double, double, true, true>(ba, V, a.sv, a.item_part, dp, gw, nw);
    }
    if (kind != kProdS64 && a.smem_vectors)
      return camera_pass<T, double, double, false, false>(ba, ps, a.sv, a.item_part, dp, gw, nw);
    return camera_pass<T, double, double, true, false>(ba, V, a.sv, a.item_part, dp, gw, nw);
  };
  // p (complete in global memory, read through L2) into shared memory as T
  auto stage_p = [&](const double* V) {
    if (a.smem_vectors)
      for (int j = threadIdx.x; j < n; j += blockDim.x) ps[j] = ld_cross(V + j);
    __syncthreads();
  };

  // ---- out[j0..j1) = (S V) (kinds S, S64) or (E V) of this CTA's cameras; V complete in
  // global memory on entry (a grid barrier precedes the call). Two grid barriers.
  auto product = [&](const double* V, double* out, int kind) -> bool {
    if (kind != kProdS64) stage_p(V);
    point_pass(V, kind);
    if (!grid_sync(gb)) return false;
    (void)camera_pass_all(V, kind, false);
    if (!grid_sync(gb)) return false;
    (void)fold_items(ba, a.item_part, V, out, j0, j1, kind != kProdE);
    __syncthreads();
    return true;
  };
  // ---- the power series (linear.py:59-67): out = sum_i (B E)^i B in over this CTA's
  // cameras; term and w are scratch vectors (term is read by every CTA).
  auto series = [&](const double* B, const double* in, double* out, double* term, double* w) -> bool {
    __syncthreads();
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) precond_apply(B, in, out, c);
    __syncthreads();
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) term[j] = out[j];
    for (int it = 1; it < a.series_terms; ++it) {
      if (!grid_sync(gb)) return false;
      if (!product(term, w, kProdE)) return false;
      for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) precond_apply(B, w, term, c);
      __syncthreads();
      double v[2] = {0.0, 0.0};
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double t = term[j], o = out[j];
        v[0] += t * t;
        v[1] += o * o;
      }
      block_reduce<2>(v, 0u, red);
      if (threadIdx.x == 0) { a.part_s[2 * blockIdx.x] = v[0]; a.part_s[2 * blockIdx.x + 1] = v[1]; }
      if (!grid_sync(gb)) return false;
      double t2[2];
      cta_sum_partials<2>(a.part_s, G, 2, t2, red, bcast);
      if (sqrt(t2[0]) <= a.series_tol * fmax(sqrt(t2[1]), 1.0)) break;  // same decision on every CTA
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) out[j] += term[j];
    }
    __syncthreads();
    return true;
  };

  // ---- one PCG solve of S X = b (X, R, Z, P, AP: the state vectors). x0 = 0, or the
  // series applied to b (init); stop when |r| <= tolerance * max(|b|, eps) (norm_ref in
  // place of |b| when it is >= 0) after min_it iterations. Returns false when a grid
  // barrier failed.
  struct CgOut {
    int iterations;
    bool success;
    double rnorm, rhs_norm;
  };
  auto cg = [&](const double* b, bool init, double norm_ref, int min_it, CgOut& o) -> bool {
    double rz_old, rr;
    // init: x = x0, r = b - S x0, z = M^-1 r, p = z (written at the first phase A)
    {
      double rz = 0.0, rr0 = 0.0;
      if (init) {
        if (!series(a.init_blocks, b, X, Pbuf + n, AP)) return false;
        if (!grid_sync(gb)) return false;
        if (!product(X, Z, kProdS)) return false;
        for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) R[j] = b[j] - Z[j];
      } else {
        for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
          X[j] = 0.0;
          R[j] = b[j];
        }
      }
      __syncthreads();
      if (a.precond_series) {
        if (!series(Minv, R, Z, Pbuf + n, AP)) return false;
      } else if (a.cluster) {
        if (!grid_sync(gb)) return false;  // r of every camera
        cluster_apply(a.cl, R, Z, j0, j1);
      } else {
        for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) precond_apply(Minv, R, Z, c);
      }
      __syncthreads();
      double bb = 0.0;
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
        const double r = R[j], z = Z[j];
        rz += r * z;
        rr0 += r * r;
        bb += b[j] * b[j];
      }
      // r.z, r.r and the float64 |b|^2 in one grid reduction
      double v[2] = {rz, rr0};
      block_reduce<2>(v, 0u, red);
      double vb[1] = {bb};
      block_reduce<1>(vb, 0u, red);
      if (threadIdx.x == 0) {
        a.part_c[2 * blockIdx.x] = v[0];
        a.part_c[2 * blockIdx.x + 1] = v[1];
        a.part_b[blockIdx.x] = vb[0];
      }
    }
    if (!grid_sync(gb)) return false;
    {
      double t2[2], t1[1];
      cta_sum_partials<2>(a.part_c, G, 2, t2, red, bcast);
      cta_sum_partials<1>(a.part_b, G, 1, t1, red, bcast);
      rz_old = t2[0];
      rr = t2[1];
      o.rhs_norm = fmax(norm_ref >= 0.0 ? norm_ref : sqrt(t1[0]), a.eps);
    }
    int iterations = 0;
    bool success = false;
    double rnorm = sqrt(rr);
    double rbest = rnorm;
    int last_improvement = 0;
    double beta = 0.0;
    int cur = 0;
    if (!(min_it <= 0 && rnorm <= a.tolerance * o.rhs_norm)) {
      for (int k = 0; k < a.max_iterations; ++k) {
        // ---- phase A: p = z + beta p_old (all cameras, redundantly per CTA: every CTA's
        // point pass reads any camera); point pass
        const int nxt = k == 0 ? 0 : cur ^ 1;
        double* Pold = Pbuf + (size_t)cur * n;
        double* Pnew = Pbuf + (size_t)nxt * n;
        if (a.smem_vectors) {
#pragma unroll 4
          for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double pv = (k == 0) ? ld_cross(Z + j) : ld_cross(Z + j) + beta * ld_cross(Pold + j);
            ps[j] = pv;
            if (j >= j0 && j < j1) Pnew[j] = pv;
          }
          __syncthreads();
        } else {
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) Pnew[j] = (k == 0) ? Z[j] : Z[j] + beta * Pold[j];
          if (!grid_sync(gb)) return false;
        }
        point_pass(Pnew, kProdS);
        cur = nxt;
        if (!grid_sync(gb)) return false;
        // ---- phase B: camera pass; p.Ap = sum_items p_c . y_item + sum_j D_j p_j^2
        {
          double v[1] = {camera_pass_all(Pnew, kProdS, true)};
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            const double pj = Pnew[j];
            v[0] += ba.cam_diag[j] * pj * pj;
          }
          block_reduce<1>(v, 0u, red);
          if (threadIdx.x == 0) a.part_b[blockIdx.x] = v[0];
        }
        if (!grid_sync(gb)) return false;
        double denom;
        {
          double t1[1];
          cta_sum_partials<1>(a.part_b, G, 1, t1, red, bcast);
          denom = t1[0];
        }
        if (fabs(denom) <= a.eps) {
          success = rnorm <= a.tolerance * o.rhs_norm;
          break;
        }
        const double alpha = rz_old / denom;
        // Ap of this CTA's cameras: their item sums in item order, plus D p
        (void)fold_items(ba, a.item_part, Pnew, AP, j0, j1, true);
        __syncthreads();
        if (a.precond_series) {
          // the reference's order: x, r; test |r|; only then z = M^-1 r (a series costs
          // up to series_terms - 1 products)
          double v[1] = {0.0};
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            X[j] = X[j] + alpha * Pnew[j];
            const double rj = R[j] - alpha * AP[j];
            R[j] = rj;
            v[0] += rj * rj;
          }
          block_reduce<1>(v, 0u, red);
          if (threadIdx.x == 0) a.part_s[2 * blockIdx.x] = v[0];
          if (!grid_sync(gb)) return false;
          double t[2];
          cta_sum_partials<1>(a.part_s, G, 2, t, red, bcast);
          rr = t[0];
          rnorm = sqrt(rr);
          iterations = k + 1;
          if (iterations >= min_it && rnorm <= a.tolerance * o.rhs_norm) {
            success = true;
            break;
          }
          if (!series(Minv, R, Z, Pbuf + (size_t)(cur ^ 1) * n, AP)) return false;
          double v2[1] = {0.0};
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) v2[0] += R[j] * Z[j];
          block_reduce<1>(v2, 0u, red);
          if (threadIdx.x == 0) a.part_c[2 * blockIdx.x] = v2[0];
          if (!grid_sync(gb)) return false;
          double t2[1];
          cta_sum_partials<1>(a.part_c, G, 2, t2, red, bcast);
          const double rz_new = t2[0];
          if (fabs(rz_old) <= a.eps) break;
          if (a.stall_window > 0) {
            if (rnorm < 0.99 * rbest) { rbest = rnorm; last_improvement = iterations; }
            else if (iterations - last_improvement >= a.stall_window) break;
          }
          beta = rz_new / rz_old;
          rz_old = rz_new;
          continue;
        }
        // ---- phase C: x += alpha p ; r -= alpha Ap ; z = M^-1 r ; partial r.z, r.r
        {
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            X[j] = X[j] + alpha * Pnew[j];
            R[j] = R[j] - alpha * AP[j];
          }
          if (a.cluster) {
            if (!grid_sync(gb)) return false;  // r of every camera
            cluster_apply(a.cl, R, Z, j0, j1);
          } else {
            __syncthreads();
            for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) precond_apply(Minv, R, Z, c);
          }
          __syncthreads();
          double v[2] = {0.0, 0.0};
          for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
            const double r = R[j];
            v[0] += r * Z[j];
            v[1] += r * r;
          }
          block_reduce<2>(v, 0u, red);
          if (threadIdx.x == 0) { a.part_c[2 * blockIdx.x] = v[0]; a.part_c[2 * blockIdx.x + 1] = v[1]; }
        }
        if (!grid_sync(gb)) return false;
        double rz_new;
        {
          double t2[2];
          cta_sum_partials<2>(a.part_c, G, 2, t2, red, bcast);
          rz_new = t2[0];
          rr = t2[1];
        }
        rnorm = sqrt(rr);
        iterations = k + 1;
        if (iterations >= min_it && rnorm <= a.tolerance * o.rhs_norm) {
          success = true;
          break;
        }
        if (fabs(rz_old) <= a.eps) break;
        if (a.stall_window > 0) {
          // float32 products: the recurrence residual stops shrinking at the rounding floor;
          // the float64 refinement then judges the iterate by its true residual
          if (rnorm < 0.99 * rbest) { rbest = rnorm; last_improvement = iterations; }
          else if (iterations - last_improvement >= a.stall_window) break;
        }
        beta = rz_new / rz_old;
        rz_old = rz_new;
      }
    } else {
      success = true;
    }
    o.iterations = iterations;
    o.success = success;
    o.rnorm = rnorm;
    return true;
  };

  // The solve, then (float32 store) the float64 refinement: r64 = rhs - S x with float64
  // arithmetic; while |r64| is above the tolerance (relative to the original |rhs|),
  // solve S dx = r64 in float32 from zero (no series start point) and add dx. With
  // eta-size tolerances the first solve normally meets the tolerance and no refinement
  // runs; it matters when the float32 recurrence stalled at its rounding floor. One call
  // site of cg, so that it is inlined.
  CgOut o0{0, false, 0.0, 0.0};
  int refine_iterations = 0;
  double refine_rnorm = -1.0;
  const bool refine = sizeof(T) == sizeof(float) && a.max_refinements > 0;
  for (int pass = 0;; ++pass) {
    CgOut oc;
    if (!cg(pass == 0 ? a.rhs : a.r64, pass == 0 && a.init_series != 0, pass == 0 ? -1.0 : o0.rhs_norm,
            pass == 0 ? a.min_iterations : 0, oc))
      return;
    if (pass == 0) {
      o0 = oc;
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) a.x_out[j] = X[j];
      if (!refine || o0.success) break;
    } else {
      refine_iterations += oc.iterations;
      for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) a.x_out[j] += X[j];
    }
    if (!grid_sync(gb)) return;  // x_out complete
    if (!product(a.x_out, AP, kProdS64)) return;
    double v[1] = {0.0};
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      const double r = a.rhs[j] - AP[j];
      a.r64[j] = r;
      v[0] += r * r;
    }
    block_reduce<1>(v, 0u, red);
    if (threadIdx.x == 0) a.part_b[blockIdx.x] = v[0];
    if (!grid_sync(gb)) return;
    double t1[1];
    cta_sum_partials<1>(a.part_b, G, 1, t1, red, bcast);
    refine_rnorm = sqrt(t1[0]);
    if (pass == a.max_refinements || refine_rnorm <= a.tolerance * o0.rhs_norm) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ba.stats[CERES_B200_STAT_PCG_ITERS] = (double)(o0.iterations + refine_iterations);
    ba.stats[CERES_B200_STAT_PCG_SUCCESS] = o0.success ? 1.0 : 0.0;
    ba.stats[CERES_B200_STAT_PCG_RNORM] = o0.rnorm;
    ba.stats[CERES_B200_STAT_RHS_NORM] = o0.rhs_norm;
    ba.stats[CERES_B200_STAT_REFINE_RNORM] = refine_rnorm;
  }
}

// ======================================================================================
// Step: candidate cameras, then point back-substitution + model decrease + candidate cost
// ======================================================================================
__global__ void k_camera_step(ceres_b200_ba_t ba, double* partials) {
  __shared__ double red[3 * 8];
  double sq = 0.0, nonfinite = 0.0, state = 0.0;
  const int n = 9 * ba.num_cameras;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int c = j / 9;
    double d = ba.cam_const[c] ? 0.0 : ba.step_cameras[j];
    if (!ba.cam_const[c]) {
      if (!isfinite(d)) nonfinite += 1.0;
      sq += d * d;
    }
    ba.step_cameras[j] = d;
    const double xc = ba.cameras[j] + d;
    ba.cand_cameras[j] = xc;
    state += xc * xc;
  }
  double v[3] = {sq, nonfinite, state};
  block_reduce<3>(v, 0u, red);
  const int out[3] = {CERES_B200_STAT_STEP_SQ_C, CERES_B200_STAT_NONFINITE, CERES_B200_STAT_CAND_STATE_SQ_C};
  grid_finish<3>(v, 0u, partials, &ba.counters[kCtrCamStep], ba.stats, out, red);
}

// The model decrease sum_o 0.5|r_o|^2 - 0.5|r_o + Jc_o dc + Jp_o dp|^2 of a point's
// track is expanded as -sum_o (r_o.a_o + 0.5|a_o|^2) - dp.(g + t) - 0.5 dp^T V dp with
// a_o = Jc_o dc, t = sum_o Jp_o^T a_o, and V = sum_o Jp_o^T Jp_o, g = sum_o Jp_o^T r_o
// the point sums of the evaluation (point_raw). The first pass over the track reads the
// Jacobian records and residuals once; the second pass (candidate cost) reads only the
// observations and the candidate camera frames.
// Slices follow the dynamic longest-first schedule; the five sums go through per-slice
// partials (slice_part[5][num_slices], folded by k_slice_fold) so the result does not
// depend on the schedule.
template <typename T>
__global__ void __launch_bounds__(kWarpBlock, CERES_B200_STEP_MIN_BLOCKS) k_step(ceres_b200_ba_t ba, const double* __restrict__ frames,
                                                                               double* __restrict__ slice_part) {
  const LossSpec L = loss_spec(ba);
  const int lane = threadIdx.x & 31;
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  unsigned err = 0;
  for (int s = next_global_slice(&ba.counters[kCtrSliceStep], ba.num_slices); s >= 0;
       s = next_global_slice(&ba.counters[kCtrSliceStep], ba.num_slices)) {
    double cand = 0.0, model = 0.0, sq = 0.0, nonfinite = 0.0, state = 0.0;  // this lane, slice s
    const int q = s * 32 + lane;
    const int len = ba.slice_len[s];
    const size_t base = (size_t)ba.slice_base[s];
    double t[3] = {0, 0, 0};
    double sa = 0.0;  // sum_o r_o.a_o + 0.5 |a_o|^2
    // padding slots have zero Jacobians: read them with camera 0 as the address and a
    // zero residual
    int k = 0;
    for (; k + 2 <= len; k += 2) {
      int c[2];
      T rv[2][kRec];
      double2 r[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const size_t slot = base + 32 * (size_t)(k + u) + lane;
        c[u] = ba.slot_cam[slot];
        load_rec(jac, slot, rv[u]);
        r[u] = reinterpret_cast<const double2*>(ba.res)[slot];
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (c[u] < 0) r[u] = make_double2(0.0, 0.0);
        const double* dc = ba.step_cameras + 9 * (size_t)max(c[u], 0);
        double u0 = 0.0, u1 = 0.0;
#pragma unroll
        for (int j = 0; j < 9; ++j) { u0 += (double)rv[u][j] * dc[j]; u1 += (double)rv[u][9 + j] * dc[j]; }
#pragma unroll
        for (int m = 0; m < 3; ++m) t[m] += (double)rv[u][18 + m] * u0 + (double)rv[u][21 + m] * u1;
        sa += r[u].x * u0 + r[u].y * u1 + 0.5 * (u0 * u0 + u1 * u1);
      }
    }
    for (; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k + lane;
      const int c = ba.slot_cam[slot];
      T rv[kRec];
      load_rec(jac, slot, rv);
      double2 r = reinterpret_cast<const double2*>(ba.res)[slot];
      if (c < 0) r = make_double2(0.0, 0.0);
      const double* dc = ba.step_cameras + 9 * (size_t)max(c, 0);
      double u0 = 0.0, u1 = 0.0;
#pragma unroll
      for (int j = 0; j < 9; ++j) { u0 += (double)rv[j] * dc[j]; u1 += (double)rv[9 + j] * dc[j]; }
#pragma unroll
      for (int m = 0; m < 3; ++m) t[m] += (double)rv[18 + m] * u0 + (double)rv[21 + m] * u1;
      sa += r.x * u0 + r.y * u1 + 0.5 * (u0 * u0 + u1 * u1);
    }
    double dp[3] = {0, 0, 0};
    const bool pconst = ba.pt_const[q] != 0;
    if (!pconst) {
      double wi[6];
#pragma unroll
      for (int i = 0; i < 6; ++i) wi[i] = (double)winv[6 * (size_t)q + i];
      double wt[3];
      sym3_mul(wi, t, wt);
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        dp[m] = ba.winv_ga[3 * (size_t)q + m] - wt[m];
        if (!isfinite(dp[m])) nonfinite += 1.0;
        sq += dp[m] * dp[m];
      }
      const double* pr = ba.point_raw + 9 * (size_t)q;
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
      ba.step_points[3 * (size_t)q + m] = dp[m];
      Xc[m] = ba.points[3 * (size_t)q + m] + dp[m];
      ba.cand_points[3 * (size_t)q + m] = Xc[m];
      state += Xc[m] * Xc[m];
    }
    for (int k = 0; k < len; ++k) {
      const size_t slot = base + 32 * (size_t)k + lane;
      const int c = ba.slot_cam[slot];
      if (c < 0) continue;
      const double2 ob = reinterpret_cast<const double2*>(ba.slot_obs)[slot];
      Proj o;
      CamRot R;
      double tail[6];
      frame_load_wide<false>(frames + kFrame * (size_t)c, R, tail);  // frames of the candidate cameras
      snavely_project<false>(R, tail, Xc, ob.x, ob.y, o);
      cand += robustify<false>(L, o, err);
    }
    const double v[5] = {cand, model, sq, nonfinite, state};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const double w = warp_sum(v[i]);
      if (lane == 0) slice_part[(size_t)i * ba.num_slices + s] = w;
    }
  }
  if (err) atomicOr(&ba.counters[kCtrError], err);
  // the sums: k_slice_fold; the camera step kernel's non-finite count is added
  // afterwards (k_add_nonfinite)
}

__global__ void k_add_nonfinite(double* stats, const double* cam_nonfinite) {
  stats[CERES_B200_STAT_NONFINITE] += *cam_nonfinite;
}

__global__ void k_copy_error(ceres_b200_ba_t ba) {
  ba.stats[CERES_B200_STAT_ERROR] = (double)(ba.counters[kCtrError] | ba.counters[kCtrBarFlag]);
}

// ======================================================================================
// Explicit reduced camera matrix and its dense Cholesky solve (the DENSE_SCHUR /
// SPARSE_SCHUR route: linear.py:667-699, solver.py:788-795). S is float64 [n][n],
// n = 9 num_cameras, zeroed by the caller.
// ======================================================================================
template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_schur_explicit(ceres_b200_ba_t ba, double* S, int n) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  for (int r_ = 0; r_ * nw < ba.num_slices; ++r_) {
    const int s = snake_slice(r_, gw, nw);
    if (s >= ba.num_slices) continue;
    const int q = s * 32 + lane;
    const int len = ba.slice_len[s];
    const size_t base = (size_t)ba.slice_base[s];
    double wi[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) wi[i] = (double)winv[6 * (size_t)q + i];
    for (int i = 0; i < len; ++i) {
      const size_t si = base + 32 * (size_t)i + lane;
      const int ci = ba.slot_cam[si];
      if (ci < 0 || ba.cam_const[ci]) continue;
      T ri[kRec];
      load_rec(jac, si, ri);
      const double jp0[3] = {(double)ri[18], (double)ri[19], (double)ri[20]};
      const double jp1[3] = {(double)ri[21], (double)ri[22], (double)ri[23]};
      double P0[3], P1[3];
      sym3_mul(wi, jp0, P0);
      sym3_mul(wi, jp1, P1);
      for (int k = 0; k < len; ++k) {
        const size_t sk = base + 32 * (size_t)k + lane;
        const int ck = ba.slot_cam[sk];
        if (ck < 0 || ba.cam_const[ck]) continue;
        T rk[kRec];
        load_rec(jac, sk, rk);
        const double C00 = P0[0] * rk[18] + P0[1] * rk[19] + P0[2] * rk[20];
        const double C01 = P0[0] * rk[21] + P0[1] * rk[22] + P0[2] * rk[23];
        const double C10 = P1[0] * rk[18] + P1[1] * rk[19] + P1[2] * rk[20];
        const double C11 = P1[0] * rk[21] + P1[1] * rk[22] + P1[2] * rk[23];
        const double d = (i == k) ? 1.0 : 0.0;
        const double M00 = d - C00, M01 = -C01, M10 = -C10, M11 = d - C11;
        for (int a = 0; a < 9; ++a) {
          const double t0 = (double)ri[a] * M00 + (double)ri[9 + a] * M10;
          const double t1 = (double)ri[a] * M01 + (double)ri[9 + a] * M11;
          double* row = S + (size_t)(9 * ci + a) * n + 9 * (size_t)ck;
#pragma unroll
          for (int b = 0; b < 9; ++b) atomicAdd(row + b, t0 * (double)rk[b] + t1 * (double)rk[9 + b]);
        }
      }
    }
  }
}

// The explicit S in a fixed order: one warp per listed block (a, b), a <= b, summing the
// block's contributions (slot i, slot j, point q) in list order (points ascending):
// -G_i W_q^-1 G_j^T, G = Jc^T Jp of one observation, plus Jc_i^T Jc_i when i == j (the
// diagonal blocks list every observation of the camera with itself and every ordered
// pair of its observations of one point). Float64 arithmetic on the store; lane l
// holds entries l, l + 32, l + 64 of the block; G, W^-1 G and Jc go through the warp's
// shared memory. A diagonal block is written from its upper triangle. k_dense_diag
// then adds the damping.
template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_schur_ordered(ceres_b200_ba_t ba, double* S, int n) {
  __shared__ double sg[kWarpBlock / 32][4][27];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  double* Ga = sg[wid][0];
  double* Gb = sg[wid][1];
  double* Ha = sg[wid][2];
  double* Ja = sg[wid][3];
  const int gi = lane / 3, gk = lane - 3 * (lane / 3);
  const int c0 = gk == 0 ? 0 : (gk == 1 ? 1 : 2);  // column gk of the packed symmetric 3 x 3
  const int c1 = gk == 0 ? 1 : (gk == 1 ? 3 : 4);
  const int c2 = gk == 0 ? 2 : (gk == 1 ? 4 : 5);
  for (long long bi = gw; bi < ba.num_schur_blocks; bi += nw) {
    const int a = ba.schur_blocks[2 * bi], b = ba.schur_blocks[2 * bi + 1];
    double acc[3] = {0.0, 0.0, 0.0};
    const long long e1 = ba.schur_block_start[bi + 1];
    for (long long ci = ba.schur_block_start[bi]; ci < e1; ++ci) {
      const int sa = ba.schur_contrib[3 * ci], sb = ba.schur_contrib[3 * ci + 1], q = ba.schur_contrib[3 * ci + 2];
      const bool self = sa == sb;
      const T* ra = jac + (size_t)kRec * (size_t)sa;
      if (lane < 27) {
        const T* rb = jac + (size_t)kRec * (size_t)sb;
        Ga[lane] = (double)ra[gi] * (double)ra[18 + gk] + (double)ra[9 + gi] * (double)ra[21 + gk];
        Gb[lane] = (double)rb[gi] * (double)rb[18 + gk] + (double)rb[9 + gi] * (double)rb[21 + gk];
      }
      if (self && lane < 18) Ja[lane] = (double)ra[lane];
      __syncwarp();
      if (lane < 27) {
        const T* w = winv + 6 * (size_t)q;
        Ha[lane] = Ga[3 * gi] * (double)w[c0] + Ga[3 * gi + 1] * (double)w[c1] + Ga[3 * gi + 2] * (double)w[c2];
      }
      __syncwarp();
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int idx = lane + 32 * m;
        if (idx < 81) {
          const int i = idx / 9, j = idx - 9 * (idx / 9);
          const double jj = self ? Ja[i] * Ja[j] + Ja[9 + i] * Ja[9 + j] : 0.0;
          acc[m] += jj - (Ha[3 * i] * Gb[3 * j] + Ha[3 * i + 1] * Gb[3 * j + 1] + Ha[3 * i + 2] * Gb[3 * j + 2]);
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int idx = lane + 32 * m;
      if (idx >= 81) continue;
      const int i = idx / 9, j = idx - 9 * (idx / 9);
      if (a == b && i > j) continue;
      S[(size_t)(9 * a + i) * n + 9 * b + j] = acc[m];
      S[(size_t)(9 * b + j) * n + 9 * a + i] = acc[m];
    }
  }
}

__global__ void k_dense_diag(ceres_b200_ba_t ba, double* S, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int c = j / 9;
    if (ba.cam_const[c]) S[(size_t)j * n + j] = 1.0;
    else S[(size_t)j * n + j] += ba.cam_diag[j];
  }
}

constexpr int kCholSmemMax = 160;  // n * n doubles fit in one CTA's shared memory

// One-CTA Cholesky solve of S x = rhs in shared memory (n <= kCholSmemMax).
__global__ void __launch_bounds__(1024) k_chol_smem(const double* __restrict__ S, const double* __restrict__ rhs,
                                                    double* __restrict__ x, int n, unsigned* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* A = reinterpret_cast<double*>(smem_raw);
  double* y = A + (size_t)n * n;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  for (int i = threadIdx.x; i < n * n; i += blockDim.x) A[i] = S[i];
  for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = rhs[i];
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x == 0) {
      const double d = A[j * n + j];
      if (!(d > 0.0)) bad = 1;
      A[j * n + j] = sqrt(fmax(d, kTiny64));
    }
    __syncthreads();
    const double ljj = A[j * n + j];
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[i * n + j] /= ljj;
    __syncthreads();
    const int m = n - j - 1;
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
      const int i = j + 1 + t / m, k = j + 1 + t % m;
      if (k <= i) A[i * n + k] -= A[i * n + j] * A[k * n + j];
    }
    __syncthreads();
  }
  // forward L y = b, backward L^T x = y (one warp, column-oriented)
  if (threadIdx.x < 32) {
    for (int j = 0; j < n; ++j) {
      const double yj = y[j] / A[j * n + j];
      __syncwarp();
      if (threadIdx.x == 0) y[j] = yj;
      for (int i = j + 1 + threadIdx.x; i < n; i += 32) y[i] -= A[i * n + j] * yj;
      __syncwarp();
    }
    for (int j = n - 1; j >= 0; --j) {
      double s = 0.0;
      for (int i = j + 1 + threadIdx.x; i < n; i += 32) s += A[i * n + j] * y[i];
      s = warp_sum(s);
      if (threadIdx.x == 0) y[j] = (y[j] - s) / A[j * n + j];
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = y[i];
  if (threadIdx.x == 0 && bad) atomicOr(err, 4u);
}

// Cooperative right-looking Cholesky in global memory for larger n; the lower
// triangle of A is overwritten by L. Every barrier wait is bounded.
__global__ void __launch_bounds__(512) k_chol_global(double* A, int n, GridBarrier gb, unsigned* err) {
  for (int j = 0; j < n; ++j) {
    if (blockIdx.x == 0) {
      __shared__ double ljj;
      if (threadIdx.x == 0) {
        const double d = A[(size_t)j * n + j];
        if (!(d > 0.0)) atomicOr(err, 4u);
        ljj = sqrt(fmax(d, kTiny64));
        A[(size_t)j * n + j] = ljj;
      }
      __syncthreads();
      for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)i * n + j] /= ljj;
    }
    if (!grid_sync(gb)) return;
    const size_t m = (size_t)(n - j - 1);
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < m * m; t += (size_t)gridDim.x * blockDim.x) {
      const int i = j + 1 + (int)(t / m), k = j + 1 + (int)(t % m);
      if (k <= i) A[(size_t)i * n + k] -= A[(size_t)i * n + j] * A[(size_t)k * n + j];
    }
    if (!grid_sync(gb)) return;
  }
}

__global__ void __launch_bounds__(1024) k_tri_solve(const double* __restrict__ Lm, const double* __restrict__ rhs,
                                                    double* __restrict__ x, int n) {
  // x holds y during the forward pass; column-oriented updates by the whole CTA
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = rhs[i];
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    __shared__ double yj;
    if (threadIdx.x == 0) { yj = x[j] / Lm[(size_t)j * n + j]; x[j] = yj; }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) x[i] -= Lm[(size_t)i * n + j] * yj;
    __syncthreads();
  }
  __shared__ double red[32];
  for (int j = n - 1; j >= 0; --j) {
    double v[1] = {0.0};
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) v[0] += Lm[(size_t)i * n + j] * x[i];
    block_reduce<1>(v, 0u, red);
    if (threadIdx.x == 0) x[j] = (x[j] - v[0]) / Lm[(size_t)j * n + j];
    __syncthreads();
  }
}

// Column j (= row j: the inverse is symmetric) of (L L^T)^-1 from the Cholesky factor L
// in the lower triangle of Lm, one CTA per column: L y = e_j (entries above j stay 0),
// then L^T x = y. The camera covariance of the reduced camera system.
__global__ void __launch_bounds__(256) k_chol_inverse(const double* __restrict__ Lm, int n, double* __restrict__ out) {
  __shared__ double yj;
  __shared__ double red[8];
  const int col = blockIdx.x;
  double* x = out + (size_t)col * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (i == col) ? 1.0 : 0.0;
  __syncthreads();
  for (int j = col; j < n; ++j) {
    if (threadIdx.x == 0) {
      yj = x[j] / Lm[(size_t)j * n + j];
      x[j] = yj;
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) x[i] -= Lm[(size_t)i * n + j] * yj;
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {
    double v[1] = {0.0};
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) v[0] += Lm[(size_t)i * n + j] * x[i];
    block_reduce<1>(v, 0u, red);
    if (threadIdx.x == 0) x[j] = (x[j] - v[0]) / Lm[(size_t)j * n + j];
    __syncthreads();
  }
}

// Bounded-wait check: two CTAs meet at a grid barrier (the barrier of the persistent
// PCG), except that CTA absent_cta returns at once. The waiting CTA gives up after
// gb.limit polls, records CERES_B200_DEVERR_BARRIER in *gb.flag and returns.
__global__ void k_barrier_probe(GridBarrier gb, int absent_cta) {
  if ((int)blockIdx.x == absent_cta) return;
  (void)grid_sync(gb);
}

// ======================================================================================
// Visibility-cluster preconditioner (linear.py:1032-1085): S kept on the cluster block
// pairs, one dense matrix per component, inverted by the symmetric sweep operator.
// ======================================================================================
// One warp per kept pair (a, b), a <= b, writes the 9 x 9 block S_ab and its transpose
// into the component's matrix. A diagonal block is camera_assemble's damped Schur block
// (V_a from its camera sums, plus D_a): the block SCHUR_JACOBI inverts. An off-diagonal
// block is -sum over the points q seen by both cameras of G_a,q W_q^-1 G_b,q^T, with
// G_c,q = sum of Jc^T Jp over camera c's observations of q (float64 arithmetic on the
// store); the shared points are taken in point order, so the block does not depend on
// the schedule. Lane l holds entries l, l + 32, l + 64 of the block (row-major); the
// 9 x 3 products go through the warp's shared memory. With pass 1 (the rebuild after a
// kept matrix that was not positive definite) the blocks between different clusters
// are halved (linear.py:1059-1072).
constexpr int kClusterWarps = kWarpBlock / 32;

template <typename T>
__global__ void __launch_bounds__(kWarpBlock) k_cluster_assemble(ceres_b200_ba_t ba, ClusterArgs cl,
                                                                 const double* __restrict__ cam_acc, int pass) {
  if (pass == 1 && *reinterpret_cast<volatile unsigned*>(cl.flags) == 0u) return;
  __shared__ double sg[kClusterWarps][3][27];  // G_a, G_b, G_a W^-1 of the current point
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const T* __restrict__ jac = reinterpret_cast<const T*>(ba.jac);
  const T* __restrict__ winv = reinterpret_cast<const T*>(ba.winv);
  const int2* __restrict__ ents = cl.entries;
  double* Ga = sg[wid][0];
  double* Gb = sg[wid][1];
  double* Ha = sg[wid][2];
  const int gi = lane / 3, gk = lane - 3 * (lane / 3);  // lane < 27: G entry (row gi, column gk)
  // G[gi][gk] over the observations [e0, e1) of one camera and one point
  auto group_g = [&](int e0, int e1) -> double {
    double g = 0.0;
    if (lane < 27) {
      for (int e = e0; e < e1; ++e) {
        const T* rv = jac + (size_t)kRec * (size_t)ents[e].x;
        g += (double)rv[gi] * (double)rv[18 + gk] + (double)rv[9 + gi] * (double)rv[21 + gk];
      }
    }
    return g;
  };
  for (int pi = gw; pi < cl.num_pairs; pi += nw) {
    const int2 pr = cl.pairs[pi];
    const int a = pr.x, b = pr.y;
    const int comp = cl.cam_comp[a];
    if (comp < 0 || cl.cam_comp[b] != comp) continue;  // uniform in the warp
    double acc[3] = {0.0, 0.0, 0.0};
    if (a != b) {
      const int ea0 = ba.cam_offsets[a], ea1 = ba.cam_offsets[a + 1];
      const int eb0 = ba.cam_offsets[b], eb1 = ba.cam_offsets[b + 1];
      for (int base = ea0; base < ea1; base += 32) {
        // lane: the entry base + lane; the first entry of a point group looks the point
        // up in b's list (sorted by point lane)
        const int e = base + lane;
        int q = -1, lo = eb1;
        bool hit = false;
        if (e < ea1) {
          q = ents[e].y;
          if (e == ea0 || ents[e - 1].y != q) {
            int l = eb0, h = eb1;
            while (l < h) {
              const int mid = (l + h) >> 1;
              if (ents[mid].y < q) l = mid + 1;
              else h = mid;
            }
            lo = l;
            hit = lo < eb1 && ents[lo].y == q;
          }
        }
        unsigned mask = __ballot_sync(0xffffffffu, hit);
        while (mask) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1;
          const int qs = __shfl_sync(0xffffffffu, q, src);
          const int ga = __shfl_sync(0xffffffffu, e, src);
          const int gb = __shfl_sync(0xffffffffu, lo, src);
          int ga1 = ga + 1, gb1 = gb + 1;
          while (ga1 < ea1 && ents[ga1].y == qs) ++ga1;
          while (gb1 < eb1 && ents[gb1].y == qs) ++gb1;
          const double va = group_g(ga, ga1), vb = group_g(gb, gb1);
          if (lane < 27) { Ga[lane] = va; Gb[lane] = vb; }
          __syncwarp();
          if (lane < 27) {  // (G_a W^-1)[gi][gk], W^-1 symmetric (6 values)
            const T* w = winv + 6 * (size_t)qs;
            const int c0 = gk == 0 ? 0 : (gk == 1 ? 1 : 2);
            const int c1 = gk == 0 ? 1 : (gk == 1 ? 3 : 4);
            const int c2 = gk == 0 ? 2 : (gk == 1 ? 4 : 5);
            Ha[lane] = Ga[3 * gi] * (double)w[c0] + Ga[3 * gi + 1] * (double)w[c1] + Ga[3 * gi + 2] * (double)w[c2];
          }
          __syncwarp();
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const int idx = lane + 32 * m;
            if (idx < 81) {
              const int i = idx / 9, j = idx - 9 * (idx / 9);
              acc[m] -= Ha[3 * i] * Gb[3 * j] + Ha[3 * i + 1] * Gb[3 * j + 1] + Ha[3 * i + 2] * Gb[3 * j + 2];
            }
          }
          __syncwarp();
        }
      }
    }
    const int dim = 9 * (cl.comp_cam_off[comp + 1] - cl.comp_cam_off[comp]);
    double* __restrict__ M = cl.inv + cl.comp_base[comp];
    const int pa = cl.cam_pos[a], pb = cl.cam_pos[b];
    const double scale = (pass == 1 && cl.tridiagonal && cl.cam_cluster[a] != cl.cam_cluster[b]) ? 0.5 : 1.0;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int idx = lane + 32 * m;
      if (idx >= 81) continue;
      const int i = idx / 9, j = idx - 9 * (idx / 9);
      double v = acc[m];
      if (a == b) {
        if (i > j) continue;  // from the upper triangle of the camera sums: exactly symmetric
        v = cam_acc[(size_t)a * kCamAcc + tri9(i, j)] + (i == j ? ba.cam_diag[9 * (size_t)a + i] : 0.0);
      }
      v *= scale;
      M[(size_t)(9 * pa + i) * dim + 9 * pb + j] = v;
      M[(size_t)(9 * pb + j) * dim + 9 * pa + i] = v;
    }
  }
}

// Zero the component matrices (pass 1: only when the first matrix was not positive definite).
__global__ void k_cluster_zero(ClusterArgs cl, long long num_elements, int pass) {
  if (pass == 1 && *reinterpret_cast<volatile unsigned*>(cl.flags) == 0u) return;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < num_elements;
       e += (long long)gridDim.x * blockDim.x)
    cl.inv[e] = 0.0;
}

// In-place inversion of every component matrix by the symmetric sweep operator, all
// components at once, in blocks of kSweepBlock pivots. Sweeping the pivot set K of a
// symmetric A = [[A11, A12], [A21, A22]] (1 = K):
//   A11 <- -A11^-1,  A12 <- A11^-1 A12,  A21 <- A21 A11^-1,  A22 <- A22 - A21 A11^-1 A12;
// sweeping every pivot once leaves -A^-1 (the epilogue negates it). Per block, three
// phases with a grid barrier after each:
//   1. the block's rows are copied (P = A[K, :]); the CTA of each component inverts A11
//      (taken from P: the current Schur complement) by the single-pivot sweep in shared
//      memory, whose pivots are A's LDL^T pivots: all positive exactly when A is positive
//      definite (the test torch.linalg.cholesky makes, linear.py:1141-1145); a
//      non-positive one sets flags[pass], a zero or non-finite one flags[2];
//   2. W = A11^-1 P (kSweepBlock x dim);
//   3. every element in 32 x 32 tiles: A22 -= P^T W (A21 = P^T by symmetry), A12 = W,
//      A21 = W^T, A11 = -A11^-1; the tile's P and W columns staged in shared memory.
// A tile may go to a different CTA in each block, so A is read with ld.global.cg (L1 is
// not coherent across SMs).
// Pass 1 runs only when pass 0 found its matrix not positive definite.
constexpr int kSweepBlock = 32;
constexpr int kSweepTile = 32;

__global__ void __launch_bounds__(256) k_cluster_sweep(ClusterArgs cl, GridBarrier gb, int pass) {
  if (pass == 1 && *reinterpret_cast<volatile unsigned*>(cl.flags) == 0u) return;
  __shared__ double sa[kSweepBlock][kSweepBlock + 1];
  __shared__ double spi[kSweepBlock][kSweepTile];  // P[:, I]
  __shared__ double swi[kSweepBlock][kSweepTile];  // W[:, I]
  __shared__ double swj[kSweepBlock][kSweepTile];  // W[:, J]
  __shared__ double sd;
  const int tid = threadIdx.x;
  const long long gtid = blockIdx.x * (long long)blockDim.x + tid;
  const long long gthreads = (long long)gridDim.x * blockDim.x;
  const int nblocks = (cl.max_dim + kSweepBlock - 1) / kSweepBlock;
  for (int kb = 0; kb < nblocks; ++kb) {
    const int k0 = kb * kSweepBlock;
    // ---- phase 1: P = A[K, :]; A11^-1 per component (component c on CTA c mod grid)
    for (int c = 0; c < cl.num_components; ++c) {
      const int dim = 9 * (cl.comp_cam_off[c + 1] - cl.comp_cam_off[c]);
      if (dim <= k0) continue;
      const int bk = min(kSweepBlock, dim - k0);
      const double* A = cl.inv + cl.comp_base[c];
      double* P = cl.piv + cl.comp_piv[c];
      const long long n = (long long)bk * dim;
      for (long long e = gtid; e < n; e += gthreads) {
        const int k = (int)(e / dim), j = (int)(e - (long long)k * dim);
        P[e] = ld_cross(A + (size_t)(k0 + k) * dim + j);
      }
    }
    for (int c = blockIdx.x; c < cl.num_components; c += gridDim.x) {
      const int dim = 9 * (cl.comp_cam_off[c + 1] - cl.comp_cam_off[c]);
      if (dim <= k0) continue;
      const int bk = min(kSweepBlock, dim - k0);
      const double* A = cl.inv + cl.comp_base[c];
      double* Ainv = cl.piv + cl.comp_piv[c] + 2 * (size_t)kSweepBlock * dim;
      for (int e = tid; e < bk * bk; e += blockDim.x) {
        const int i = e / bk, j = e - (e / bk) * bk;
        sa[i][j] = ld_cross(A + (size_t)(k0 + i) * dim + k0 + j);
      }
      __syncthreads();
      for (int k = 0; k < bk; ++k) {
        if (tid == 0) {
          const double d = sa[k][k];
          sd = d;
          if (!(d > 0.0)) atomicOr(cl.flags + pass, 1u);
          if (d == 0.0 || !isfinite(d)) atomicOr(cl.flags + 2, 1u);
        }
        __syncthreads();
        const double rd = 1.0 / sd;
        // the single-pivot sweep of k; every element read before any thread writes (256
        // threads x 4 >= 32 x 32 elements)
        double v[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int e = tid + 256 * m;
          v[m] = 0.0;
          if (e < bk * bk) {
            const int i = e / bk, j = e - (e / bk) * bk;
            if (i == k) v[m] = (j == k) ? -rd : sa[k][j] * rd;
            else if (j == k) v[m] = sa[i][k] * rd;
            else v[m] = sa[i][j] - sa[i][k] * sa[k][j] * rd;
          }
        }
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int e = tid + 256 * m;
          if (e < bk * bk) sa[e / bk][e - (e / bk) * bk] = v[m];
        }
        __syncthreads();
      }
      for (int e = tid; e < bk * bk; e += blockDim.x) Ainv[e] = -sa[e / bk][e - (e / bk) * bk];  // +A11^-1
      __syncthreads();
    }
    if (!grid_sync(gb)) return;
    // ---- phase 2: W = A11^-1 P
    for (int c = 0; c < cl.num_components; ++c) {
      const int dim = 9 * (cl.comp_cam_off[c + 1] - cl.comp_cam_off[c]);
      if (dim <= k0) continue;
      const int bk = min(kSweepBlock, dim - k0);
      const double* P = cl.piv + cl.comp_piv[c];
      double* W = cl.piv + cl.comp_piv[c] + (size_t)kSweepBlock * dim;
      const double* Ainv = cl.piv + cl.comp_piv[c] + 2 * (size_t)kSweepBlock * dim;
      const long long n = (long long)bk * dim;
      for (long long e = gtid; e < n; e += gthreads) {
        const int k = (int)(e / dim), j = (int)(e - (long long)k * dim);
        double w = 0.0;
        for (int m = 0; m < bk; ++m) w += ld_cross(Ainv + k * bk + m) * ld_cross(P + (size_t)m * dim + j);
        W[e] = w;
      }
    }
    if (!grid_sync(gb)) return;
    // ---- phase 3: the tiles (a global tile index over the components, CTA-strided)
    long long tile_base = 0;
    const int ty = tid / 16, tx = tid - 16 * (tid / 16);  // 16 x 16 threads, 2 x 2 elements each
    for (int c = 0; c < cl.num_components; ++c) {
      const int dim = 9 * (cl.comp_cam_off[c + 1] - cl.comp_cam_off[c]);
      if (dim <= k0) continue;
      const int bk = min(kSweepBlock, dim - k0);
      const int nt = (dim + kSweepTile - 1) / kSweepTile;
      const long long ntiles = (long long)nt * nt;
      double* A = cl.inv + cl.comp_base[c];
      const double* P = cl.piv + cl.comp_piv[c];
      const double* W = cl.piv + cl.comp_piv[c] + (size_t)kSweepBlock * dim;
      const double* Ainv = cl.piv + cl.comp_piv[c] + 2 * (size_t)kSweepBlock * dim;
      long long t = ((blockIdx.x - tile_base) % gridDim.x + gridDim.x) % gridDim.x;
      for (; t < ntiles; t += gridDim.x) {
        const int i0 = (int)(t / nt) * kSweepTile, j0 = (int)(t % nt) * kSweepTile;
        for (int e = tid; e < bk * kSweepTile; e += blockDim.x) {
          const int k = e / kSweepTile, l = e - (e / kSweepTile) * kSweepTile;
          const bool ri = i0 + l < dim, rj = j0 + l < dim;
          spi[k][l] = ri ? ld_cross(P + (size_t)k * dim + i0 + l) : 0.0;
          swi[k][l] = ri ? ld_cross(W + (size_t)k * dim + i0 + l) : 0.0;
          swj[k][l] = rj ? ld_cross(W + (size_t)k * dim + j0 + l) : 0.0;
        }
        __syncthreads();
        double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
        for (int k = 0; k < bk; ++k) {
          const double pa0 = spi[k][2 * ty], pa1 = spi[k][2 * ty + 1];
          const double wb0 = swj[k][2 * tx], wb1 = swj[k][2 * tx + 1];
          acc[0][0] += pa0 * wb0;
          acc[0][1] += pa0 * wb1;
          acc[1][0] += pa1 * wb0;
          acc[1][1] += pa1 * wb1;
        }
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          const int i = i0 + 2 * ty + a;
          if (i >= dim) continue;
          const bool ik = i >= k0 && i < k0 + bk;
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const int j = j0 + 2 * tx + b;
            if (j >= dim) continue;
            const bool jk = j >= k0 && j < k0 + bk;
            double* out = A + (size_t)i * dim + j;
            if (ik && jk) *out = -ld_cross(Ainv + (i - k0) * bk + (j - k0));
            else if (ik) *out = swj[i - k0][2 * tx + b];
            else if (jk) *out = swi[j - k0][2 * ty + a];
            else *out = ld_cross(out) - acc[a][b];
          }
        }
        __syncthreads();
      }
      tile_base += ntiles;
    }
    if (!grid_sync(gb)) return;
  }
  for (int c = 0; c < cl.num_components; ++c) {
    const int dim = 9 * (cl.comp_cam_off[c + 1] - cl.comp_cam_off[c]);
    double* M = cl.inv + cl.comp_base[c];
    const long long n2 = (long long)dim * dim;
    for (long long e = gtid; e < n2; e += gthreads) M[e] = -ld_cross(M + e);
  }
}

// ======================================================================================
// C ABI
// ======================================================================================
namespace {

bool valid(const ceres_b200_ba_t* ba) {
  if (!ba) return false;
  if (ba->num_cameras < 0 || ba->num_points < 0 || ba->num_slices < 0 || ba->num_slots < 0) return false;
  if (ba->num_points != 32 * ba->num_slices) return false;
  if (ba->precision != CERES_B200_FP64 && ba->precision != CERES_B200_FP32) return false;
  if (!ba->counters || !ba->stats) return false;
  if (ba->num_slices > 0 && (!ba->slice_base || !ba->slice_len || !ba->slot_cam || !ba->slot_obs || !ba->jac ||
                             !ba->res || !ba->cameras || !ba->points || !ba->pt_const))
    return false;
  if (ba->num_cameras > 0 && (!ba->cam_offsets || !ba->cam_const || !ba->cam_diag || !ba->rhs || !ba->precond))
    return false;
  if ((reinterpret_cast<uintptr_t>(ba->jac) & 31) != 0) return false;  // 256-bit record loads
  // the camera reduction's cp.async copies: 16-byte residual pairs, 8-byte W^-1 pieces
  if ((reinterpret_cast<uintptr_t>(ba->res) & 15) != 0 || (reinterpret_cast<uintptr_t>(ba->winv) & 7) != 0 ||
      (reinterpret_cast<uintptr_t>(ba->winv_ga) & 7) != 0)
    return false;
  if (ba->num_observations > 0) {
    if (!ba->cam_entries || !ba->cam_items || !ba->items || ba->num_items <= 0) return false;
    if (ba->cm_jac && (!ba->slot_pos || (reinterpret_cast<uintptr_t>(ba->cm_jac) & 31) != 0)) return false;
  }
  if (ba->num_items < 0) return false;
  return true;
}

// The cluster struct against the problem: pointers present, sizes consistent. The index
// arrays themselves are the host builder's (clustering.py) and are not re-checked here.
bool valid_clusters(const ceres_b200_ba_t& ba, const ceres_b200_clusters_t* cl) {
  if (!cl) return false;
  if (cl->num_components < 1 || cl->num_pairs < cl->num_components || cl->max_dim < 9 || cl->max_dim % 9 != 0)
    return false;
  if (cl->max_dim > 16384 || cl->max_dim > 9 * ba.num_cameras || cl->num_elements < 81) return false;
  if (!cl->pairs || !cl->entries || !cl->cam_comp || !cl->cam_pos || !cl->cam_cluster || !cl->comp_cams ||
      !cl->comp_cam_off || !cl->comp_base || !cl->comp_piv || !cl->inv || !cl->piv || !cl->flags)
    return false;
  return true;
}

ClusterArgs cluster_args(const ceres_b200_clusters_t& c) {
  ClusterArgs a;
  a.num_components = c.num_components;
  a.num_pairs = c.num_pairs;
  a.max_dim = c.max_dim;
  a.tridiagonal = c.tridiagonal;
  a.pairs = reinterpret_cast<const int2*>(c.pairs);
  a.entries = reinterpret_cast<const int2*>(c.entries);
  a.cam_comp = c.cam_comp;
  a.cam_pos = c.cam_pos;
  a.cam_cluster = c.cam_cluster;
  a.comp_cams = c.comp_cams;
  a.comp_cam_off = c.comp_cam_off;
  a.comp_base = reinterpret_cast<const long long*>(c.comp_base);
  a.comp_piv = reinterpret_cast<const long long*>(c.comp_piv);
  a.inv = c.inv;
  a.piv = c.piv;
  a.flags = c.flags;
  return a;
}

int check_launch() {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "ceres_b200: CUDA error %s\n", cudaGetErrorString(e));
    return CERES_B200_ECUDA;
  }
  return CERES_B200_OK;
}

struct PcgLayout {
  int grid = 0;
  int cams_per_cta = 0;
  int smem_vectors = 0;
  size_t dyn_smem = 0;
  size_t frames = 0, aux = 0, cam_acc = 0, sv = 0, item_part = 0, part_b = 0, part_c = 0, r64 = 0, spse_base = 0,
         part_s = 0, slice_part = 0, total = 0;
};

template <typename T>
int pcg_layout(const ceres_b200_ba_t& ba, PcgLayout& L) {
  const DevInfo d = device_info();
  const int n = 9 * ba.num_cameras;
  auto kern = k_pcg<T>;
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return CERES_B200_ECUDA;
  // shared memory: a float64 copy of p for the products' camera gathers
  const size_t vec_bytes = ((size_t)n * sizeof(double) + 15) & ~(size_t)15;
  L.smem_vectors = (vec_bytes + fa.sharedSizeBytes + 1024 <= (size_t)d.max_smem_optin) ? 1 : 0;
  L.dyn_smem = L.smem_vectors ? vec_bytes : 0;
  if (L.dyn_smem > 48 * 1024) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.dyn_smem) != cudaSuccess)
      return CERES_B200_ESMEM;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPcgBlock, L.dyn_smem) != cudaSuccess || per_sm < 1)
    return CERES_B200_ECOOP;
  L.grid = d.sms * per_sm;
  const int needed_for_cams = ba.num_cameras > 0 ? ba.num_cameras : 1;
  L.cams_per_cta = (needed_for_cams + L.grid - 1) / L.grid;
  size_t off = red_area_bytes(ba, d);
  L.frames = off;
  off += frames_bytes(ba);
  L.slice_part = off;
  off += slice_part_bytes(ba);
  L.aux = off;
  off += 256;
  L.cam_acc = off;
  off += ((size_t)(ba.num_cameras > 0 ? ba.num_cameras : 1) * kCamAcc * sizeof(double) + 255) & ~(size_t)255;
  L.sv = off;
  off += ((size_t)(ba.num_points > 0 ? ba.num_points : 1) * 3 * sizeof(double) + 255) & ~(size_t)255;
  L.item_part = off;
  off += ((size_t)(ba.num_items > 0 ? ba.num_items : 1) * 9 * sizeof(double) + 255) & ~(size_t)255;
  L.part_b = off;
  off += (size_t)L.grid * sizeof(double);
  L.part_c = off;
  off += (size_t)L.grid * 2 * sizeof(double);
  L.part_s = off;
  off += (size_t)L.grid * 2 * sizeof(double);
  off = (off + 255) & ~(size_t)255;
  L.r64 = off;
  off += (size_t)n * sizeof(double);
  off = (off + 255) & ~(size_t)255;
  L.spse_base = off;
  off += (size_t)(ba.num_cameras > 0 ? ba.num_cameras : 1) * 81 * sizeof(double);
  L.total = (off + 255) & ~(size_t)255;
  return CERES_B200_OK;
}

int scratch_bytes_impl(const ceres_b200_ba_t& ba, size_t& bytes) {
  PcgLayout L;
  const int rc = ba.precision == CERES_B200_FP32 ? pcg_layout<float>(ba, L) : pcg_layout<double>(ba, L);
  if (rc) return rc;
  bytes = L.total;
  return CERES_B200_OK;
}

// Series options of one PCG launch (SCHUR_POWER_SERIES_EXPANSION / SPSE initial point).
struct SeriesOpts {
  int precond = 0, init = 0, terms = 1;
  double tol = 0.0;
  const double* init_blocks = nullptr;
};

template <typename T>
int launch_pcg(const ceres_b200_ba_t& ba, int min_it, int max_it, double tol, int max_ref, cudaStream_t st,
               const PcgLayout& L, char* scratch, const SeriesOpts& so, const ClusterArgs* cl = nullptr) {
  PcgArgs a;
  a.cluster = cl != nullptr ? 1 : 0;
  if (cl != nullptr) a.cl = *cl;
  a.precond_series = so.precond;
  a.init_series = so.init;
  a.init_blocks = so.init_blocks;
  a.series_terms = so.terms;
  a.series_tol = so.tol;
  a.part_s = reinterpret_cast<double*>(scratch + L.part_s);
  a.rhs = ba.rhs;
  a.x_out = ba.step_cameras;
  a.min_iterations = min_it;
  a.max_iterations = max_it;
  a.tolerance = tol;
  a.eps = kEps64;  // the PCG vectors and arithmetic are float64 in both precisions
  a.n = 9 * ba.num_cameras;
  a.cams_per_cta = L.cams_per_cta;
  a.smem_vectors = L.smem_vectors;
  a.sv = reinterpret_cast<double*>(scratch + L.sv);
  a.item_part = reinterpret_cast<double*>(scratch + L.item_part);
  a.part_b = reinterpret_cast<double*>(scratch + L.part_b);
  a.part_c = reinterpret_cast<double*>(scratch + L.part_c);
  a.r64 = reinterpret_cast<double*>(scratch + L.r64);
  // float32 store: float64 refinement passes inside the launch, and the float32
  // recurrence stops at its rounding floor so that the refinement can take over
  a.max_refinements = sizeof(T) == sizeof(float) ? max_ref : 0;
  a.stall_window = a.max_refinements > 0 ? kStallWindow : 0;
  // barrier words start at zero for every launch
  CB_TRACE("pcg: memset barrier words");
  if (cudaMemsetAsync(&ba.counters[kCtrBarCount], 0, 3 * sizeof(uint32_t), st) != cudaSuccess) return CERES_B200_ECUDA;
  ceres_b200_ba_t bcopy = ba;
  void* args[] = {&bcopy, &a};
  count_launch();
  CB_TRACE("pcg: cooperative launch grid=%d block=%d smem=%zu n=%d cams/cta=%d smem_vectors=%d", L.grid, kPcgBlock,
           L.dyn_smem, a.n, a.cams_per_cta, a.smem_vectors);
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_pcg<T>, dim3(L.grid), dim3(kPcgBlock), args,
                                                    L.dyn_smem, st);
  if (e != cudaSuccess) {
    fprintf(stderr, "ceres_b200: cooperative PCG launch failed: %s\n", cudaGetErrorString(e));
    return CERES_B200_ECOOP;
  }
  CB_TRACE("pcg: launched (%s)", trace_on() ? cudaGetErrorString(cudaStreamSynchronize(st)) : "");
  return CERES_B200_OK;
}

// y = S x in float64 arithmetic from the stored Jacobian (precision T): the point pass,
// the camera pass and the fold of the persistent PCG as three launches. The y = S x
// test entry point.
template <typename T>
int matvec64(const ceres_b200_ba_t& ba, const double* x, double* y, cudaStream_t st) {
  const DevInfo d = device_info();
  const int n = 9 * ba.num_cameras;
  PcgLayout L;
  int rc = pcg_layout<T>(ba, L);
  if (rc) return rc;
  if (!ba.scratch || (size_t)ba.scratch_bytes < L.total) return CERES_B200_EINVAL;
  char* scratch = reinterpret_cast<char*>(ba.scratch);
  double* sv = reinterpret_cast<double*>(scratch + L.sv);
  double* part = reinterpret_cast<double*>(scratch + L.item_part);
  if (ba.num_slices > 0) {
    count_launch();
    k_point_pass64<T><<<slice_grid(ba, d), kWarpBlock, 0, st>>>(ba, x, sv);
  }
  if (ba.num_items > 0) {
    int g = (ba.num_items * 32 + kWarpBlock - 1) / kWarpBlock;
    if (g > 8 * d.sms) g = 8 * d.sms;
    count_launch();
    k_camera_pass64<T><<<g, kWarpBlock, 0, st>>>(ba, x, sv, part);
  }
  count_launch();
  k_fold_items<<<(n + 255) / 256 > 0 ? (n + 255) / 256 : 1, 256, 0, st>>>(ba, part, x, y);
  return check_launch();
}

// Camera side of the assembly. pc: the preconditioner whose blocks go to ba.precond
// (SCHUR_POWER_SERIES: the inverted damped Hbb blocks); FLAG_SPSE_BASE: the Hbb
// blocks for the SPSE initial point as well, into the scratch. Each block set is one
// reduction over the camera-major lists; the damping, rhs and gradient stats come
// out of every reduction alike.
template <typename T, bool kDup, bool kHbb = false>
int launch_camera_reduce(const ceres_b200_ba_t& ba, double* acc, cudaStream_t st) {
  const size_t smem = CamStage<T>::kBytes;
  if (cudaFuncSetAttribute(k_camera_reduce<T, kDup, kHbb>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return CERES_B200_ESMEM;
  k_camera_reduce<T, kDup, kHbb><<<ba.num_cameras, kCamBlock, smem, st>>>(ba, acc);
  return CERES_B200_OK;
}

template <typename T>
int camera_assemble_impl(const ceres_b200_ba_t& ba, const PcgLayout& L, char* scratch, double inv_radius,
                         double mn, double mx, int jacobi_scaling, int pc, int flags, cudaStream_t st) {
  double* partials = reinterpret_cast<double*>(scratch);
  double* acc = reinterpret_cast<double*>(scratch + L.cam_acc);
  const int nc = ba.num_cameras;
  const int fgrid = (nc + kFinishWarps - 1) / kFinishWarps;
  double* pre = reinterpret_cast<double*>(ba.precond);
  const bool spse = pc == CERES_B200_PRECOND_SCHUR_POWER_SERIES;
  count_launch(2);
  int rc = spse ? launch_camera_reduce<T, false, true>(ba, acc, st)
                : (ba.has_duplicate_cameras ? launch_camera_reduce<T, true>(ba, acc, st)
                                            : launch_camera_reduce<T, false>(ba, acc, st));
  if (rc) return rc;
  k_camera_finish<T><<<fgrid, 32 * kFinishWarps, 0, st>>>(ba, acc, inv_radius, mn, mx, jacobi_scaling,
                                                         spse ? CERES_B200_PRECOND_SCHUR_JACOBI : pc, partials, pre);
  if ((flags & CERES_B200_PRECOND_FLAG_SPSE_BASE) && !spse) {
    count_launch(2);
    rc = launch_camera_reduce<T, false, true>(ba, acc, st);
    if (rc) return rc;
    k_camera_finish<T><<<fgrid, 32 * kFinishWarps, 0, st>>>(ba, acc, inv_radius, mn, mx, jacobi_scaling,
                                                           CERES_B200_PRECOND_SCHUR_JACOBI, partials,
                                                           reinterpret_cast<double*>(scratch + L.spse_base));
  }
  return CERES_B200_OK;
}

template <typename T>
int pcg_impl(const ceres_b200_ba_t& ba, int precond, int min_it, int max_it, double tol, int max_ref, cudaStream_t st,
             int series_terms = 1, double series_tol = 0.0, int series_init = 0, const ClusterArgs* cl = nullptr) {
  PcgLayout L;
  CB_TRACE("pcg: layout");
  int rc = pcg_layout<T>(ba, L);
  CB_TRACE("pcg: layout rc=%d grid=%d total=%zu scratch=%lld", rc, L.grid, L.total, (long long)ba.scratch_bytes);
  if (rc) return rc;
  if (!ba.scratch || (size_t)ba.scratch_bytes < L.total) return CERES_B200_EINVAL;
  char* scratch = reinterpret_cast<char*>(ba.scratch);
  const int n = 9 * ba.num_cameras;
  if (n == 0) return CERES_B200_OK;
  SeriesOpts so;
  so.precond = precond == CERES_B200_PRECOND_SCHUR_POWER_SERIES ? 1 : 0;
  so.terms = series_terms;
  so.tol = series_tol;
  so.init = series_init ? 1 : 0;
  so.init_blocks = so.precond ? reinterpret_cast<const double*>(ba.precond)
                              : reinterpret_cast<const double*>(scratch + L.spse_base);
  rc = launch_pcg<T>(ba, min_it, max_it, tol, max_ref, st, L, scratch, so, cl);
  if (rc) return rc;
  count_launch();
  k_copy_error<<<1, 1, 0, st>>>(ba);
  return check_launch();
}

}  // namespace

extern "C" {

int ceres_b200_abi_version(void) { return CERES_B200_ABI_VERSION; }

uint64_t ceres_b200_launch_count(void) { return (uint64_t)__atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int ceres_b200_ba_struct_bytes(void) { return (int)sizeof(ceres_b200_ba_t); }

int ceres_b200_scratch_bytes(const ceres_b200_ba_t* ba, int64_t* bytes_out) {
  if (!ba || !bytes_out) return CERES_B200_EINVAL;
  size_t b = 0;
  const int rc = scratch_bytes_impl(*ba, b);
  if (rc) return rc;
  *bytes_out = (int64_t)b;
  return CERES_B200_OK;
}

int ceres_b200_ba_evaluate(const ceres_b200_ba_t* ba, int with_jacobian, void* stream) {
  if (!valid(ba) || !ba->scratch || (with_jacobian && !ba->point_raw)) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  const size_t red = red_area_bytes(*ba, d);
  if (ba->scratch_bytes < 0 || (size_t)ba->scratch_bytes < red + frames_bytes(*ba) + slice_part_bytes(*ba))
    return CERES_B200_EINVAL;
  const int grid = resident_slice_grid(*ba, d, with_jacobian ? CERES_B200_EVAL_MIN_BLOCKS : CERES_B200_EVAL_NOJAC_MIN_BLOCKS);
  double* partials = reinterpret_cast<double*>(ba->scratch);
  double* frames = reinterpret_cast<double*>(reinterpret_cast<char*>(ba->scratch) + red);
  double* slice_part = reinterpret_cast<double*>(reinterpret_cast<char*>(ba->scratch) + red + frames_bytes(*ba));
  const int nc = ba->num_cameras;
  if (nc > 0) {
    count_launch();
    if (with_jacobian) k_camera_frames<true><<<(nc + 127) / 128, 128, 0, st>>>(ba->cameras, frames, nc);
    else k_camera_frames<false><<<(nc + 127) / 128, 128, 0, st>>>(ba->cameras, frames, nc);
  }
  count_launch(2);
  if (ba->precision == CERES_B200_FP32) {
    if (with_jacobian) k_evaluate<float, true, true><<<grid, kWarpBlock, 0, st>>>(*ba, partials, frames, slice_part);
    else k_evaluate<float, false, true><<<grid, kWarpBlock, 0, st>>>(*ba, partials, frames, slice_part);
  } else {
    if (with_jacobian) k_evaluate<double, true, true><<<grid, kWarpBlock, 0, st>>>(*ba, partials, frames, slice_part);
    else k_evaluate<double, false, true><<<grid, kWarpBlock, 0, st>>>(*ba, partials, frames, slice_part);
  }
  launch_slice_fold<1>(*ba, d, slice_part, partials, kCtrEval, kCtrSliceEval, StatIdx<1>{{CERES_B200_STAT_COST}}, st);
  count_launch();
  k_copy_error<<<1, 1, 0, st>>>(*ba);
  return check_launch();
}

}  // extern "C"

// --------------------------------------------------------------------------------------
// Evaluation without caller-provided scratch (ceres_b200_ba_evaluate_noalloc)
// --------------------------------------------------------------------------------------
namespace {

// Per-CTA cost partials of the evaluator for callers that cannot hand us a scratch
// buffer. It lives in the library image: every GPU that loads the library holds these
// 256 KB until the process exits. All calls on a device share it.
constexpr int kNoAllocPartials = 32768;  // float64 slots: one per evaluation CTA
static __device__ __align__(256) double g_noalloc_partials[kNoAllocPartials];

// Identity of the calling thread's current CUDA context (0 when it cannot be read),
// through the driver entry points the runtime hands out, so the library needs no link
// against the driver library.
unsigned long long current_context_id() {
  typedef CUresult (*GetCurrentFn)(CUcontext*);
  typedef CUresult (*GetIdFn)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<GetCurrentFn>(f1);
      get_id = reinterpret_cast<GetIdFn>(f2);
    }
    looked_up = true;
  }
  if (!get_current || !get_id) return 0ull;
  CUcontext ctx = nullptr;
  unsigned long long id = 0ull;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, &id) != CUDA_SUCCESS) return 0ull;
  return id;
}

// Device address of g_noalloc_partials, looked up with the device current the first
// time a context of that device calls (the symbol's host-side name is only a stand-in,
// so kernels are given this address). The cache remembers the context it was taken in:
// after a device reset the device gets a new context, the module is loaded again and
// the address is looked up again.
double* noalloc_partials(int device, int* rc) {
  static std::mutex mu;
  static double* addr[64] = {nullptr};
  static unsigned long long ctx_of[64] = {0ull};
  *rc = CERES_B200_OK;
  if (device < 0 || device >= 64) {
    *rc = CERES_B200_EINVAL;
    return nullptr;
  }
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(mu);
  if (addr[device] == nullptr || ctx == 0ull || ctx_of[device] != ctx) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
    if (e != cudaSuccess || ptr == nullptr) {
      fprintf(stderr, "ceres_b200: cudaGetSymbolAddress for the static evaluation scratch failed: %s\n",
              cudaGetErrorString(e));
      *rc = CERES_B200_ECUDA;
      return nullptr;
    }
    addr[device] = static_cast<double*>(ptr);
    ctx_of[device] = ctx;
  }
  return addr[device];
}

}  // namespace

extern "C" {

int ceres_b200_ba_evaluate_noalloc(const ceres_b200_ba_t* ba, int with_jacobian, void* stream) {
  if (!valid(ba) || (with_jacobian && !ba->point_raw)) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return CERES_B200_ECUDA;
  const DevInfo d = device_info();
  const int grid = slice_grid(*ba, d);
  if (grid > kNoAllocPartials) {
    fprintf(stderr,
            "ceres_b200: ceres_b200_ba_evaluate_noalloc needs %d reduction slots, above its static capacity of %d\n",
            grid, kNoAllocPartials);
    return CERES_B200_ETOOBIG;
  }
  int rc = CERES_B200_OK;
  double* partials = noalloc_partials(dev, &rc);
  if (rc) return rc;
  // every CTA writes its own slot before the last one folds them, so the shared array
  // needs no clearing between calls; the ticket counter is the caller's (counters[])
  // no scratch for camera frames here: each observation computes its camera's rotation
  // (the same arithmetic as the frames, so the results are those of ceres_b200_ba_evaluate)
  if (ba->precision == CERES_B200_FP32) {
    if (with_jacobian) { count_launch(); k_evaluate<float, true, false><<<grid, kWarpBlock, 0, st>>>(*ba, partials, nullptr, nullptr); }
    else { count_launch(); k_evaluate<float, false, false><<<grid, kWarpBlock, 0, st>>>(*ba, partials, nullptr, nullptr); }
  } else {
    if (with_jacobian) { count_launch(); k_evaluate<double, true, false><<<grid, kWarpBlock, 0, st>>>(*ba, partials, nullptr, nullptr); }
    else { count_launch(); k_evaluate<double, false, false><<<grid, kWarpBlock, 0, st>>>(*ba, partials, nullptr, nullptr); }
  }
  count_launch();
  k_copy_error<<<1, 1, 0, st>>>(*ba);
  return check_launch();
}

int ceres_b200_ba_point_assemble(const ceres_b200_ba_t* ba, double radius, double min_diagonal, double max_diagonal,
                                 int jacobi_scaling, void* stream) {
  if (!valid(ba) || !ba->scratch || !ba->winv || !ba->winv_ga || !ba->point_raw) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  const double inv_radius = 1.0 / fmax(radius, kEps64);
  double* partials = reinterpret_cast<double*>(ba->scratch);
  int grid = (ba->num_points + kWarpBlock - 1) / kWarpBlock;
  if (grid > d.sms * 8) grid = d.sms * 8;
  if (grid < 1) grid = 1;
  count_launch();
  if (ba->precision == CERES_B200_FP32)
    k_point_assemble<float><<<grid, kWarpBlock, 0, st>>>(*ba, inv_radius, min_diagonal, max_diagonal, jacobi_scaling,
                                                         partials);
  else
    k_point_assemble<double><<<grid, kWarpBlock, 0, st>>>(*ba, inv_radius, min_diagonal, max_diagonal, jacobi_scaling,
                                                          partials);
  return check_launch();
}

int ceres_b200_ba_camera_assemble(const ceres_b200_ba_t* ba, double radius, double min_diagonal, double max_diagonal,
                                  int jacobi_scaling, int preconditioner, void* stream) {
  if (!valid(ba) || !ba->scratch) return CERES_B200_EINVAL;
  const int flags = preconditioner & ~0xff;
  int pc = preconditioner & 0xff;
  if (pc < CERES_B200_PRECOND_IDENTITY || pc > CERES_B200_PRECOND_CLUSTER) return CERES_B200_EINVAL;
  if (pc == CERES_B200_PRECOND_CLUSTER) pc = CERES_B200_PRECOND_IDENTITY;  // built by cluster_factor
  if ((flags & ~CERES_B200_PRECOND_FLAG_SPSE_BASE) != 0) return CERES_B200_EINVAL;
  if (ba->num_cameras == 0) return CERES_B200_OK;
  PcgLayout L;
  const int lrc = ba->precision == CERES_B200_FP32 ? pcg_layout<float>(*ba, L) : pcg_layout<double>(*ba, L);
  if (lrc) return lrc;
  if ((size_t)ba->scratch_bytes < L.total) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const double inv_radius = 1.0 / fmax(radius, kEps64);
  char* scratch = reinterpret_cast<char*>(ba->scratch);
  const int rc = ba->precision == CERES_B200_FP32
                     ? camera_assemble_impl<float>(*ba, L, scratch, inv_radius, min_diagonal, max_diagonal,
                                                   jacobi_scaling, pc, flags, st)
                     : camera_assemble_impl<double>(*ba, L, scratch, inv_radius, min_diagonal, max_diagonal,
                                                    jacobi_scaling, pc, flags, st);
  if (rc) return rc;
  return check_launch();
}

int ceres_b200_ba_pcg(const ceres_b200_ba_t* ba, int preconditioner, int min_iterations, int max_iterations,
                      double tolerance, int max_refinements, void* stream) {
  if (!valid(ba) || max_iterations < 0 || min_iterations < 0 || max_refinements < 0) return CERES_B200_EINVAL;
  if (!ba->pcg_x || !ba->pcg_r || !ba->pcg_z || !ba->pcg_p || !ba->pcg_ap || !ba->step_cameras) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (ba->precision == CERES_B200_FP32)
    return pcg_impl<float>(*ba, preconditioner, min_iterations, max_iterations, tolerance, max_refinements, st);
  return pcg_impl<double>(*ba, preconditioner, min_iterations, max_iterations, tolerance, max_refinements, st);
}

int ceres_b200_ba_pcg_spse(const ceres_b200_ba_t* ba, int preconditioner, int min_iterations, int max_iterations,
                           double tolerance, int max_refinements, int spse_terms, double spse_tolerance, int spse_init,
                           void* stream) {
  if (!valid(ba) || max_iterations < 0 || min_iterations < 0 || max_refinements < 0) return CERES_B200_EINVAL;
  if (!ba->pcg_x || !ba->pcg_r || !ba->pcg_z || !ba->pcg_p || !ba->pcg_ap || !ba->step_cameras) return CERES_B200_EINVAL;
  if (preconditioner < CERES_B200_PRECOND_IDENTITY || preconditioner > CERES_B200_PRECOND_SCHUR_POWER_SERIES)
    return CERES_B200_EINVAL;
  const bool uses = preconditioner == CERES_B200_PRECOND_SCHUR_POWER_SERIES || spse_init != 0;
  if (uses && (spse_terms < 1 || !(spse_tolerance >= 0.0))) return CERES_B200_EINVAL;
  if (!uses) spse_terms = 1;
  cudaStream_t st = (cudaStream_t)stream;
  if (ba->precision == CERES_B200_FP32)
    return pcg_impl<float>(*ba, preconditioner, min_iterations, max_iterations, tolerance, max_refinements, st,
                           spse_terms, spse_tolerance, spse_init);
  return pcg_impl<double>(*ba, preconditioner, min_iterations, max_iterations, tolerance, max_refinements, st,
                          spse_terms, spse_tolerance, spse_init);
}

int ceres_b200_ba_schur_matvec(const ceres_b200_ba_t* ba, const double* x, double* y, void* stream) {
  if (!valid(ba) || !x || !y) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = 9 * ba->num_cameras;
  if (n == 0) return CERES_B200_OK;
  if (ba->precision == CERES_B200_FP32) return matvec64<float>(*ba, x, y, st);
  return matvec64<double>(*ba, x, y, st);
}

int ceres_b200_ba_step(const ceres_b200_ba_t* ba, void* stream) {
  if (!valid(ba) || !ba->scratch || !ba->cand_cameras || !ba->cand_points || !ba->step_points) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  double* partials = reinterpret_cast<double*>(ba->scratch);
  // camera candidates; their non-finite count goes to a scratch double
  const int n = 9 * ba->num_cameras;
  const int cgrid = n > 0 ? ((n + 255) / 256 < 64 ? (n + 255) / 256 : 64) : 1;
  PcgLayout L;
  const int lrc = ba->precision == CERES_B200_FP32 ? pcg_layout<float>(*ba, L) : pcg_layout<double>(*ba, L);
  if (lrc) return lrc;
  if ((size_t)ba->scratch_bytes < L.total) return CERES_B200_EINVAL;
  ceres_b200_ba_t b2 = *ba;
  double* cam_stats = reinterpret_cast<double*>(reinterpret_cast<char*>(ba->scratch) + L.aux);
  b2.stats = cam_stats;
  count_launch();
  k_camera_step<<<cgrid, 256, 0, st>>>(b2, partials);
  double* frames = reinterpret_cast<double*>(reinterpret_cast<char*>(ba->scratch) + L.frames);
  const int nc = ba->num_cameras;
  if (nc > 0) {
    count_launch();
    k_camera_frames<false><<<(nc + 127) / 128, 128, 0, st>>>(ba->cand_cameras, frames, nc);
  }
  const int grid = resident_slice_grid(*ba, d, CERES_B200_STEP_MIN_BLOCKS);
  double* slice_part = reinterpret_cast<double*>(reinterpret_cast<char*>(ba->scratch) + L.slice_part);
  count_launch(2);
  if (ba->precision == CERES_B200_FP32) k_step<float><<<grid, kWarpBlock, 0, st>>>(*ba, frames, slice_part);
  else k_step<double><<<grid, kWarpBlock, 0, st>>>(*ba, frames, slice_part);
  launch_slice_fold<5>(*ba, d, slice_part, partials, kCtrStep, kCtrSliceStep,
                       StatIdx<5>{{CERES_B200_STAT_CAND_COST, CERES_B200_STAT_MODEL, CERES_B200_STAT_STEP_SQ_P,
                                   CERES_B200_STAT_NONFINITE, CERES_B200_STAT_CAND_STATE_SQ_P}},
                       st);
  // STEP_SQ_C and the camera non-finite count into the shared stats
  count_launch();
  k_add_nonfinite<<<1, 1, 0, st>>>(ba->stats, cam_stats + CERES_B200_STAT_NONFINITE);
  cudaMemcpyAsync(ba->stats + CERES_B200_STAT_STEP_SQ_C, cam_stats + CERES_B200_STAT_STEP_SQ_C, sizeof(double),
                  cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(ba->stats + CERES_B200_STAT_CAND_STATE_SQ_C, cam_stats + CERES_B200_STAT_CAND_STATE_SQ_C,
                  sizeof(double), cudaMemcpyDeviceToDevice, st);
  count_launch();
  k_copy_error<<<1, 1, 0, st>>>(*ba);
  return check_launch();
}

int ceres_b200_dense_cholesky_solve(double* H, const double* rhs, double* x, int64_t n64, uint32_t* flags,
                                    void* stream) {
  if (!H || !rhs || !x || !flags || n64 < 0 || n64 > (int64_t)1 << 30) return CERES_B200_EINVAL;
  const int n = (int)n64;
  if (n == 0) return CERES_B200_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  if (n <= kCholSmemMax) {
    const size_t smem = ((size_t)n * n + n) * sizeof(double);
    if (cudaFuncSetAttribute(k_chol_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return CERES_B200_ESMEM;
    count_launch();
    k_chol_smem<<<1, 1024, smem, st>>>(H, rhs, x, n, flags + 3);
    return check_launch();
  }
  if (cudaMemsetAsync(flags, 0, 3 * sizeof(uint32_t), st) != cudaSuccess) return CERES_B200_ECUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chol_global, 512, 0) != cudaSuccess || per_sm < 1)
    return CERES_B200_ECOOP;
  GridBarrier gb{flags, flags + 1, flags + 2};
  unsigned* errp = flags + 3;
  int nn = n;
  void* args[] = {&H, &nn, &gb, &errp};
  count_launch();
  if (cudaLaunchCooperativeKernel((const void*)k_chol_global, dim3(d.sms * per_sm), dim3(512), args, 0, st) !=
      cudaSuccess)
    return CERES_B200_ECOOP;
  count_launch();
  k_tri_solve<<<1, 1024, 0, st>>>(H, rhs, x, n);
  return check_launch();
}

int ceres_b200_dense_schur_bytes(const ceres_b200_ba_t* ba, int64_t* bytes_out) {
  if (!ba || !bytes_out || ba->num_cameras < 0) return CERES_B200_EINVAL;
  const int64_t n = 9 * (int64_t)ba->num_cameras;
  *bytes_out = n * n * (int64_t)sizeof(double);
  return CERES_B200_OK;
}

namespace {
// The explicit S (undamped; k_dense_diag adds the damping): in the listed fixed order when
// the struct carries the contribution list, else with float64 atomics.
int assemble_explicit_schur(const ceres_b200_ba_t& ba, double* S, int n, cudaStream_t st) {
  const DevInfo d = device_info();
  if (ba.schur_blocks != nullptr) {
    if (!ba.schur_block_start || !ba.schur_contrib || ba.num_schur_blocks < 0) return CERES_B200_EINVAL;
    if (ba.num_schur_blocks > 0) {
      long long grid = (ba.num_schur_blocks * 32 + kWarpBlock - 1) / kWarpBlock;
      if (grid > 16LL * d.sms) grid = 16LL * d.sms;
      count_launch();
      if (ba.precision == CERES_B200_FP32)
        k_schur_ordered<float><<<(unsigned)grid, kWarpBlock, 0, st>>>(ba, S, n);
      else
        k_schur_ordered<double><<<(unsigned)grid, kWarpBlock, 0, st>>>(ba, S, n);
    }
    return CERES_B200_OK;
  }
  if (ba.num_slices > 0) {
    count_launch();
    if (ba.precision == CERES_B200_FP32)
      k_schur_explicit<float><<<slice_grid(ba, d), kWarpBlock, 0, st>>>(ba, S, n);
    else
      k_schur_explicit<double><<<slice_grid(ba, d), kWarpBlock, 0, st>>>(ba, S, n);
  }
  return CERES_B200_OK;
}
}  // namespace

int ceres_b200_ba_dense_schur_solve(const ceres_b200_ba_t* ba, double* work, void* stream) {
  if (!valid(ba) || !ba->step_cameras) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = 9 * ba->num_cameras;
  if (n == 0) return CERES_B200_OK;
  if (!work) return CERES_B200_EINVAL;
  const DevInfo d = device_info();
  if (cudaMemsetAsync(work, 0, (size_t)n * n * sizeof(double), st) != cudaSuccess) return CERES_B200_ECUDA;
  const int arc = assemble_explicit_schur(*ba, work, n, st);
  if (arc) return arc;
  count_launch();
  k_dense_diag<<<(n + 255) / 256, 256, 0, st>>>(*ba, work, n);
  if (n <= kCholSmemMax) {
    const size_t smem = ((size_t)n * n + n) * sizeof(double);
    if (cudaFuncSetAttribute(k_chol_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return CERES_B200_ESMEM;
    count_launch();
    k_chol_smem<<<1, 1024, smem, st>>>(work, ba->rhs, ba->step_cameras, n, &ba->counters[kCtrError]);
  } else {
    if (cudaMemsetAsync(&ba->counters[kCtrBarCount], 0, 3 * sizeof(uint32_t), st) != cudaSuccess)
      return CERES_B200_ECUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chol_global, 512, 0) != cudaSuccess || per_sm < 1)
      return CERES_B200_ECOOP;
    GridBarrier gb{&ba->counters[kCtrBarCount], &ba->counters[kCtrBarGen], &ba->counters[kCtrBarFlag]};
    unsigned* errp = &ba->counters[kCtrError];
    int nn = n;
    void* args[] = {&work, &nn, &gb, &errp};
    count_launch();
    if (cudaLaunchCooperativeKernel((const void*)k_chol_global, dim3(d.sms * per_sm), dim3(512), args, 0, st) !=
        cudaSuccess)
      return CERES_B200_ECOOP;
    count_launch();
    k_tri_solve<<<1, 1024, 0, st>>>(work, ba->rhs, ba->step_cameras, n);
  }
  count_launch();
  k_copy_error<<<1, 1, 0, st>>>(*ba);
  return check_launch();
}

int ceres_b200_clusters_struct_bytes(void) { return (int)sizeof(ceres_b200_clusters_t); }

int ceres_b200_ba_cluster_factor(const ceres_b200_ba_t* ba, const ceres_b200_clusters_t* cl, void* stream) {
  if (!valid(ba) || !valid_clusters(*ba, cl) || !ba->scratch) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  const ClusterArgs c = cluster_args(*cl);
  // the camera sums of the last camera_assemble, in the scratch
  PcgLayout L;
  const int lrc = ba->precision == CERES_B200_FP32 ? pcg_layout<float>(*ba, L) : pcg_layout<double>(*ba, L);
  if (lrc) return lrc;
  if ((size_t)ba->scratch_bytes < L.total) return CERES_B200_EINVAL;
  const double* cam_acc = reinterpret_cast<const double*>(reinterpret_cast<const char*>(ba->scratch) + L.cam_acc);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cluster_sweep, 256, 0) != cudaSuccess || per_sm < 1)
    return CERES_B200_ECOOP;
  const int sweep_grid = d.sms * (per_sm < 4 ? per_sm : 4);
  int pair_grid = (cl->num_pairs * 32 + kWarpBlock - 1) / kWarpBlock;
  if (pair_grid > 16 * d.sms) pair_grid = 16 * d.sms;
  int zero_grid = (int)((cl->num_elements + 255) / 256);
  if (zero_grid > 8 * d.sms) zero_grid = 8 * d.sms;
  if (cudaMemsetAsync(cl->flags, 0, 8 * sizeof(uint32_t), st) != cudaSuccess) return CERES_B200_ECUDA;
  for (int pass = 0; pass < (cl->tridiagonal ? 2 : 1); ++pass) {
    ClusterArgs cp = c;
    int pp = pass;
    GridBarrier gb{cl->flags + 3, cl->flags + 4, cl->flags + 5};
    long long ne = cl->num_elements;
    count_launch(2);
    k_cluster_zero<<<zero_grid, 256, 0, st>>>(c, ne, pass);
    if (ba->precision == CERES_B200_FP32)
      k_cluster_assemble<float><<<pair_grid, kWarpBlock, 0, st>>>(*ba, c, cam_acc, pass);
    else
      k_cluster_assemble<double><<<pair_grid, kWarpBlock, 0, st>>>(*ba, c, cam_acc, pass);
    void* args[] = {&cp, &gb, &pp};
    count_launch();
    if (cudaLaunchCooperativeKernel((const void*)k_cluster_sweep, dim3(sweep_grid), dim3(256), args, 0, st) !=
        cudaSuccess)
      return CERES_B200_ECOOP;
  }
  return check_launch();
}

int ceres_b200_ba_pcg_cluster(const ceres_b200_ba_t* ba, const ceres_b200_clusters_t* cl, int min_iterations,
                              int max_iterations, double tolerance, int max_refinements, void* stream) {
  if (!valid(ba) || !valid_clusters(*ba, cl) || max_iterations < 0 || min_iterations < 0 || max_refinements < 0)
    return CERES_B200_EINVAL;
  if (!ba->pcg_x || !ba->pcg_r || !ba->pcg_z || !ba->pcg_p || !ba->pcg_ap || !ba->step_cameras) return CERES_B200_EINVAL;
  const ClusterArgs c = cluster_args(*cl);
  cudaStream_t st = (cudaStream_t)stream;
  if (ba->precision == CERES_B200_FP32)
    return pcg_impl<float>(*ba, CERES_B200_PRECOND_CLUSTER, min_iterations, max_iterations, tolerance,
                           max_refinements, st, 1, 0.0, 0, &c);
  return pcg_impl<double>(*ba, CERES_B200_PRECOND_CLUSTER, min_iterations, max_iterations, tolerance,
                          max_refinements, st, 1, 0.0, 0, &c);
}

int ceres_b200_debug_barrier_timeout(uint32_t* words, uint32_t spin_limit, void* stream) {
  if (!words || spin_limit == 0u) return CERES_B200_EINVAL;
  GridBarrier gb{words, words + 1, words + 2};
  gb.limit = spin_limit < kSpinLimit ? spin_limit : kSpinLimit;
  count_launch();
  k_barrier_probe<<<2, 32, 0, (cudaStream_t)stream>>>(gb, 1);
  return check_launch();
}

int ceres_b200_ba_schur_matrix(const ceres_b200_ba_t* ba, double* S, void* stream) {
  if (!valid(ba) || (ba->num_cameras > 0 && !S)) return CERES_B200_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  const int n = 9 * ba->num_cameras;
  if (n == 0) return CERES_B200_OK;
  const DevInfo d = device_info();
  if (cudaMemsetAsync(S, 0, (size_t)n * n * sizeof(double), st) != cudaSuccess) return CERES_B200_ECUDA;
  const int arc = assemble_explicit_schur(*ba, S, n, st);
  if (arc) return arc;
  count_launch();
  k_dense_diag<<<(n + 255) / 256, 256, 0, st>>>(*ba, S, n);
  return check_launch();
}

int ceres_b200_dense_spd_inverse(double* A, double* inv, int64_t n64, uint32_t* flags, void* stream) {
  if (!A || !inv || !flags || n64 < 0 || n64 > (1 << 15)) return CERES_B200_EINVAL;
  const int n = (int)n64;
  if (n == 0) return CERES_B200_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const DevInfo d = device_info();
  if (cudaMemsetAsync(flags, 0, 3 * sizeof(uint32_t), st) != cudaSuccess) return CERES_B200_ECUDA;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_chol_global, 512, 0) != cudaSuccess || per_sm < 1)
    return CERES_B200_ECOOP;
  GridBarrier gb{flags, flags + 1, flags + 2};
  unsigned* errp = flags + 3;
  int nn = n;
  void* args[] = {&A, &nn, &gb, &errp};
  count_launch();
  if (cudaLaunchCooperativeKernel((const void*)k_chol_global, dim3(d.sms * per_sm), dim3(512), args, 0, st) !=
      cudaSuccess)
    return CERES_B200_ECOOP;
  count_launch();
  k_chol_inverse<<<n, 256, 0, st>>>(A, n, inv);
  return check_launch();
}

}  // extern "C"
