// Stepper with the learned surrogate: one BD step is three phases over the live
// slots instead of the fused persistent kernel, because the surrogate is a
// batched tensor-core GEMM chain over every trusted trajectory at once.
//
//   sur_begin_kernel  reaction test and escape/return (step_begin); every exact force
//                     term for poses outside the trust region, the terms the surrogate
//                     does not replace for the others; features of the trusted poses,
//                     packed as BF16 rows of the MLP's input
//   MLP ensemble      every member on the trusted rows (bd_mlp.cu)
//   sur_end_kernel    the surrogate's terms for trusted poses whose ensemble agrees,
//                     the exact kernels for them elsewhere; then the move,
//                     overlap test, bridge and step count (step_move, step_end);
//                     ended trajectories are replaced from the pending pool
//
// No reference counterpart (the surrogate is the engine's own addition); the
// exact parts are the same device functions as the fused stepper, and the noise
// is the same keyed Philox stream, so a trajectory differs from its exact twin
// only through the surrogate's force error.
#pragma once

#include <cuda_bf16.h>

#include "bd_kernels.cuh"

namespace bd {

constexpr int kSurIn = 13, kSurInPad = 32, kSurOut = 6;

constexpr int kSurEnv = 32;  // radial envelope table entries

struct DevSurrogate {
  double r_scale, rbf_centre[5], rbf_width;
  double out_scale[kSurOut];
  double r_min, r_max, threshold, force_floor;
  double env_r0, env_r1;       // envelope table range (env_r1 <= env_r0: no envelope)
  double env_log[kSurEnv];     // log of the force size at kSurEnv evenly spaced radii
  unsigned terms;              // force terms (group_forces bits) the surrogate replaces
};

// Outputs are normalised by out_scale and by a radial envelope: the RMS force
// size of the training targets as a function of |c|, interpolated linearly in
// its log between table entries (clamped at the ends), so that the network sees
// targets of similar size at every distance.
__device__ __forceinline__ double sur_envelope(const DevSurrogate& Q, double r) {
  if (!(Q.env_r1 > Q.env_r0)) return 1.0;
  double u = (r - Q.env_r0) / (Q.env_r1 - Q.env_r0) * (kSurEnv - 1);
  u = fmin(fmax(u, 0.0), (double)(kSurEnv - 1));
  const int i = min((int)u, kSurEnv - 2);
  const double t = u - i;
  return exp((1.0 - t) * Q.env_log[i] + t * Q.env_log[i + 1]);
}

// Per-slot scratch of one BD step.
struct SurBuf {
  double* F;       // 3 * cap
  double* T;       // 3 * cap
  int8_t* mode;    // 0: no step this time, 1: exact forces complete, 2: trusted (surrogate pending),
                   // 3: the pose did not move since the last step, F and T are its complete forces
  int8_t* fresh;   // per slot: F and T hold the complete forces of the slot's current pose (cleared
                   // at the start of every launch, whose compaction moves slots)
  int* row;        // trusted: row of the MLP input
  __nv_bfloat16* X;  // cap x kSurInPad packed features
  const float* mean;    // cap x kSurOut (ensemble mean, scaled outputs)
  const float* spread;  // cap x kSurOut
  int* n_rows;          // device count of trusted rows this step
  unsigned long long* ctr;  // [0] surrogate evaluations, [1] exact fallbacks
};

// warp_forces with a per-lane choice of force terms.
template <typename FT, bool TORQUE>
__device__ __forceinline__ void warp_forces_terms(const DevSystem& S, const double c[3], const double R[9], bool need,
                                                  unsigned terms, double F[3], double T[3], int lane, Counts& cnt) {
  const unsigned FULL = 0xffffffffu;
  unsigned m = __ballot_sync(FULL, need);
  while (m) {
    const int j = __ffs(m) - 1;
    m &= m - 1;
    double cj[3], Rj[9];
#pragma unroll
    for (int k = 0; k < 3; ++k) cj[k] = __shfl_sync(FULL, c[k], j);
#pragma unroll
    for (int k = 0; k < 9; ++k) Rj[k] = __shfl_sync(FULL, R[k], j);
    const unsigned tj = __shfl_sync(FULL, terms, j);
    double f[3], t[3], e;
    group_forces<FT, 32, TORQUE, false>(S, cj, Rj, lane, FULL, PosFromPose{Rj, cj}, f, t, e, cnt,
                                        RecView{nullptr, nullptr}, tj);
    if (lane == j) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = f[k];
        T[k] = t[k];
      }
    }
  }
}

__device__ __forceinline__ void record_end(const DevSim& P, const Traj& tr, int st, Tally& tl) {
  P.out_status[tr.id] = (int8_t)st;
  P.out_steps[tr.id] = tr.steps;
  P.out_returns[tr.id] = tr.rets;
  tl.reacted += st == ST_REACTED;
  tl.escaped += st == ST_ESCAPED;
  tl.maxsteps += st == ST_MAXSTEPS;
}

template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 2) sur_begin_kernel(DevSystem S, DevSim P, SlotBuf B,
                                                           const int* __restrict__ n_live, SurBuf U, DevSurrogate Q) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, n_warps = (gridDim.x * blockDim.x) >> 5;
  const int live = *n_live;
  Tally tl{};
  unsigned long long n_sur = 0;
  for (int base = warp * 32; base < live; base += n_warps * 32) {
    const int slot = base + lane;
    const bool own = slot < live;
    Traj tr{};
    tr.status = ST_EMPTY;
    if (own) load_slot(B, slot, tr);
    const bool run = own && tr.status == ST_RUNNING;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, r = 0;
    int st = ST_EMPTY;
    const int rets0 = tr.rets;
    if (run) st = step_begin(S, P, traj_key(P, tr.id), (uint32_t)tr.steps, tr, R, r, tl);
    const bool need = run && st == ST_RUNNING;
    // a step rejected by the overlap test left the pose unchanged: its forces are reused
    const bool reuse = need && tr.rets == rets0 && U.fresh[slot];
    const bool trusted = need && !reuse && r >= Q.r_min && r <= Q.r_max;
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    warp_forces_terms<FT, TORQUE>(S, tr.c, R, need && !reuse, trusted ? (15u & ~Q.terms) : 15u, F, T, lane, tl.cnt);
    if (run && st != ST_RUNNING) {
      tr.status = st;
      record_end(P, tr, st, tl);
    }
    // rows of the trusted poses: one atomic per warp
    const unsigned tm = __ballot_sync(FULL, trusted);
    int row0 = 0;
    if (tm) {
      if (lane == __ffs(tm) - 1) row0 = atomicAdd(U.n_rows, __popc(tm));
      row0 = __shfl_sync(FULL, row0, __ffs(tm) - 1);
    }
    if (trusted) {
      const int row = row0 + __popc(tm & ((1u << lane) - 1u));
      U.row[slot] = row;
      n_sur += 1;
      // features: c / r_scale, |c| / r_scale, q with w >= 0, radial basis values of |c|
      float f[kSurIn];
      const double sg = tr.q[0] < 0 ? -1.0 : 1.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) f[k] = (float)(tr.c[k] / Q.r_scale);
      f[3] = (float)(r / Q.r_scale);
#pragma unroll
      for (int k = 0; k < 4; ++k) f[4 + k] = (float)(sg * tr.q[k]);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const double d = (r - Q.rbf_centre[k]) / Q.rbf_width;
        f[8 + k] = (float)exp(-0.5 * d * d);
      }
      __nv_bfloat16* x = U.X + (size_t)row * kSurInPad;
#pragma unroll
      for (int k = 0; k < kSurInPad; ++k) x[k] = __float2bfloat16_rn(k < kSurIn ? f[k] : 0.f);
    }
    if (own) {
      store_slot(B, slot, tr);
      if (!reuse) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          U.F[3 * slot + k] = F[k];
          U.T[3 * slot + k] = T[k];
        }
      }
      U.mode[slot] = (int8_t)(need ? (reuse ? 3 : trusted ? 2 : 1) : 0);
    }
  }
  flush_tally(P, tl, true);
  n_sur = gsumu<32>((unsigned)n_sur, FULL);
  if (lane == 0 && n_sur) atomicAdd(U.ctr, n_sur);
}

template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 2) sur_end_kernel(DevSystem S, DevSim P, SlotBuf B,
                                                         const int* __restrict__ n_live, SurBuf U, DevSurrogate Q) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, n_warps = (gridDim.x * blockDim.x) >> 5;
  const int live = *n_live;
  Tally tl{};
  unsigned n_fb = 0;
  for (int base = warp * 32; base < live; base += n_warps * 32) {
    const int slot = base + lane;
    const bool own = slot < live;
    Traj tr{};
    tr.status = ST_EMPTY;
    if (own) load_slot(B, slot, tr);
    const int mode = own ? (int)U.mode[slot] : 0;
    const bool need = mode != 0;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, r = 0;
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    bool fallback = false;
    if (need) {
      quat_to_rot(tr.q, R);
      r = norm3(tr.c[0], tr.c[1], tr.c[2]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = U.F[3 * slot + k];
        T[k] = U.T[3 * slot + k];
      }
      if (mode == 2) {
        const float* mu = U.mean + (size_t)U.row[slot] * kSurOut;
        const float* sp = U.spread + (size_t)U.row[slot] * kSurOut;
        const double env = sur_envelope(Q, r);
        double fs[3], ts[3], s2 = 0, f2 = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          fs[k] = (double)mu[k] * Q.out_scale[k] * env;
          ts[k] = (double)mu[3 + k] * Q.out_scale[3 + k] * env;
          const double e = (double)sp[k] * Q.out_scale[k] * env;
          s2 += e * e;
          f2 += fs[k] * fs[k];
        }
        const double size = fmax(sqrt(f2), Q.force_floor * env);
        fallback = !(sqrt(s2) <= Q.threshold * size);  // NaN spreads fall back too
        if (!fallback) {
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            F[k] += fs[k];
            if (TORQUE) T[k] += ts[k];
          }
        }
      }
    }
    // the surrogate's terms, exact, where the ensemble disagrees
    double Fx[3] = {0, 0, 0}, Tx[3] = {0, 0, 0};
    warp_forces_terms<FT, TORQUE>(S, tr.c, R, fallback, Q.terms, Fx, Tx, lane, tl.cnt);
    if (fallback) {
      n_fb += 1;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] += Fx[k];
        T[k] += Tx[k];
      }
    }
    const Keyed key = traj_key(P, tr.id);
    const uint32_t s = (uint32_t)tr.steps;
    double cn[3] = {0, 0, 0}, qn[4] = {1, 0, 0, 0}, dt = 0;
    bool ok = true;
    if (need) ok = step_move<FT>(S, P, key, s, tr, R, r, F, T, cn, qn, dt);
    int st = tr.status;
    if (need && !ok) {
      tl.nonfinite += 1;
      st = ST_ERROR;
    }
    const bool ovl = warp_overlap(S, cn, need && ok && P.overlap, lane, RecView{nullptr, nullptr});
    if (need && ok) st = step_end(S, P, key, s, tr, R, cn, qn, !ovl, dt, tl);
    if (need && st != ST_RUNNING) {
      tr.status = st;
      record_end(P, tr, st, tl);
    }
    bool dead = !own;
    warp_refill(P, tr, dead, lane);
    if (own) {
      store_slot(B, slot, tr);
      // rejected and still running: the next step starts from the same pose with these forces
      const bool keep = need && ok && ovl && st == ST_RUNNING;
      if (keep && mode != 3) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          U.F[3 * slot + k] = F[k];
          U.T[3 * slot + k] = T[k];
        }
      }
      U.fresh[slot] = (int8_t)keep;
    }
  }
  flush_tally(P, tl, true);
  n_fb = gsumu<32>(n_fb, FULL);
  if (lane == 0 && n_fb) atomicAdd(U.ctr + 1, (unsigned long long)n_fb);
}

__global__ void zero_int_kernel(int* p) { *p = 0; }

}  // namespace bd
