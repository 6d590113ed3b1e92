// Split stepper: one BD step as three kernels instead of one fused persistent kernel.
//
//   split_begin_kernel  reaction test and escape/return (step_begin), the forces on the
//                       ligand atoms (grid, far-field, contact), and the list of poses whose
//                       receptor atoms can reach the ligand Born grid
//   split_rev_kernel    Born direction 2 of the listed poses, one warp per pose
//   split_end_kernel    the rest of the step (step_move, overlap test, step_end, statistics)
//                       and the refill of ended trajectories from the pending pool
//
// Near contact Born direction 2 is most of a step's work, and it is bound by the latency of
// its grid gathers.  In the fused kernel it shares the per-trajectory state's registers
// (128 per thread: 16 warps per SM); here it runs in a kernel capped at 64 registers, so
// twice as many warps hide the gather latency.  Candidates (receptor atoms inside the
// ligand's Born box, in the ligand frame) go to a per-warp buffer in shared memory and are
// drained in whole groups of 32, entry i by lane i mod 32, in the order of the fused
// kernel's ring: every lane sums the same terms in the same order, so the forces, and so
// the trajectories, are those of the fused stepper.  The same keyed Philox stream drives
// both (gpu_batch_simulator.py:783-1254 is the step being split).
#pragma once

#include "bd_kernels.cuh"

namespace bd {

constexpr int kSplitBuf = 128;  // candidate entries per warp (whole groups of 32 are drained)

// Per-slot scratch of one BD step.
struct SplitBuf {
  double* F;       // 3 * cap: forces on the ligand atoms; the step's total force once complete
  double* T;       // 3 * cap
  double* rv;      // 6 * cap: Born direction 2 sums r (ligand frame) and u, from the sweep
  double* rprev;   // cap: |c| at the end of the previous step (statistics)
  int8_t* mode;    // 0: no step; 1: F, T to be used as they are; 2: reused (complete);
                   // 3: F, T plus the Born direction 2 sums in rv
  int8_t* fresh;   // F, T hold the complete forces of the slot's current pose
  int* list;       // slots listed for the sweep this step
  int* cnt;        // [0] list length, [1] sweep cursor (both cleared before every step)
};

// Forces on the ligand atoms of every lane with `need`, the warp sweeping one pose at a time.
template <typename FT, bool TORQUE>
__device__ __forceinline__ void warp_forces_ligand(const DevSystem& S, const double c[3], const double R[9],
                                                   bool need, double F[3], double T[3], int lane, Counts& cnt,
                                                   const RecView& v) {
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
    double f[3], t[3], e;
    group_forces<FT, 32, TORQUE, false, PosFromPose, false>(S, cj, Rj, lane, FULL, PosFromPose{Rj, cj}, f, t, e,
                                                           cnt, v);
    if (lane == j) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = f[k];
        T[k] = t[k];
      }
    }
  }
}

template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 2) split_begin_kernel(DevSystem S, DevSim P, SlotBuf B,
                                                             const int* __restrict__ n_live, SplitBuf U) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, n_warps = (gridDim.x * blockDim.x) >> 5;
  const int live = *n_live;
  Tally tl{};
  for (int base = warp * 32; base < live; base += n_warps * 32) {
    const int slot = base + lane;
    const bool own = slot < live;
    Traj tr{};
    tr.status = ST_EMPTY;
    if (own) load_slot(B, slot, tr);
    const bool run = own && tr.status == ST_RUNNING;
    const uint32_t s = (uint32_t)tr.steps;
    if (run && P.stats) U.rprev[slot] = norm3(tr.c[0], tr.c[1], tr.c[2]);
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, r = 0;
    int st = ST_EMPTY;
    const int rets0 = tr.rets;
    if (run) {
      st = step_begin(S, P, traj_key(P, tr.id), s, tr, R, r, tl);
      if (P.stats && st == ST_REACTED) stats_encounter(P, tr, s, false);
    }
    const bool need = run && st == ST_RUNNING;
    // a step rejected by the overlap test left the pose unchanged: its forces are reused
    const bool reuse = need && tr.rets == rets0 && U.fresh[slot];
    const bool eval = need && !reuse;
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    warp_forces_ligand<FT, TORQUE>(S, tr.c, R, eval, F, T, lane, tl.cnt, RecView{nullptr, nullptr});
    const bool rev = eval && S.born_rev && r - S.rec_max_r < S.lig_born_rho;
    const unsigned rm = __ballot_sync(FULL, rev);
    if (rm) {
      int at = 0;
      if (lane == __ffs(rm) - 1) at = atomicAdd(U.cnt, __popc(rm));
      at = __shfl_sync(FULL, at, __ffs(rm) - 1);
      if (rev) U.list[at + __popc(rm & ((1u << lane) - 1u))] = slot;
    }
    if (run && st != ST_RUNNING) {
      tr.status = st;
      P.out_status[tr.id] = (int8_t)st;
      P.out_steps[tr.id] = tr.steps;
      P.out_returns[tr.id] = tr.rets;
      tl.reacted += st == ST_REACTED;
      tl.escaped += st == ST_ESCAPED;
      tl.maxsteps += st == ST_MAXSTEPS;
    }
    if (own) {
      store_slot(B, slot, tr);
      if (eval) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          U.F[3 * slot + k] = F[k];
          U.T[3 * slot + k] = T[k];
        }
      }
      U.mode[slot] = (int8_t)(need ? (reuse ? 2 : rev ? 3 : 1) : 0);
    }
  }
  flush_tally(P, tl, true);
}

// Born direction 2 of one pose by a whole warp (the same terms and order as warp_reverse_born):
// receptor chunks culled against the ligand Born grid's margin box in the ligand frame, in-box
// atoms gathered into `buf` and drained 32 at a time.  Adds this lane's share of the sums to
// r (ligand frame) and u; the caller reduces over the warp.
template <typename FT, bool TORQUE>
__device__ __forceinline__ void lean_reverse_born(const DevSystem& S, const SlotBuf& B, int slot, int lane,
                                                  typename Vec4<FT>::type* buf, double r[3], double u[3],
                                                  unsigned& nr) {
  using V4 = typename Vec4<FT>::type;
  const unsigned FULL = 0xffffffffu;
  const DevGrid& g = S.lig_born;
  FT Rt[9], cx, cy, cz;
  {
    const double q[4] = {B.q[slot], B.q[B.cap + slot], B.q[2 * B.cap + slot], B.q[3 * B.cap + slot]};
    double R[9];
    quat_to_rot(q, R);
#pragma unroll
    for (int k = 0; k < 9; ++k) Rt[k] = (FT)R[k];
    cx = (FT)B.c[slot];
    cy = (FT)B.c[B.cap + slot];
    cz = (FT)B.c[2 * B.cap + slot];
  }
  const FT lox = (FT)g.lox, loy = (FT)g.loy, loz = (FT)g.loz, hix = (FT)g.hix, hiy = (FT)g.hiy, hiz = (FT)g.hiz;
  using AT = typename Vec4<FT>::type;
  const AT* atoms;
  const AT* spheres;
  if constexpr (sizeof(FT) == 4) {
    atoms = S.rec_f;
    spheres = S.chunks_f;
  } else {
    atoms = S.rec;
    spheres = S.chunks;
  }
  FT rs0 = 0, rs1 = 0, rs2 = 0;
  int k0 = 0, head = 0;
  unsigned hits = 0;
  bool done = false;
  for (;;) {
    // gather until the buffer has no room for another chunk, or every chunk is done
    while (head <= kSplitBuf - 32) {
      if (!hits) {
        if (k0 >= S.n_chunks) {
          done = true;
          break;
        }
        const int k = k0 + lane;
        bool hit = false;
        if (k < S.n_chunks) {
          const AT sp = spheres[k];
          const FT d0 = (FT)sp.x - cx, d1 = (FT)sp.y - cy, d2 = (FT)sp.z - cz;
          const FT l0 = Rt[0] * d0 + Rt[3] * d1 + Rt[6] * d2;
          const FT l1 = Rt[1] * d0 + Rt[4] * d1 + Rt[7] * d2;
          const FT l2 = Rt[2] * d0 + Rt[5] * d1 + Rt[8] * d2;
          const FT ex = fmax(fmax(lox - l0, l0 - hix), (FT)0);
          const FT ey = fmax(fmax(loy - l1, l1 - hiy), (FT)0);
          const FT ez = fmax(fmax(loz - l2, l2 - hiz), (FT)0);
          // the radius is inflated against rounding; the extra margin covers FP32 geometry
          const FT lim = (FT)sp.w + (sizeof(FT) == 4 ? (FT)1e-3 : (FT)1e-9);
          hit = ex * ex + ey * ey + ez * ez < lim * lim;
        }
        hits = __ballot_sync(FULL, hit);
        k0 += 32;
        continue;
      }
      const int kk = k0 - 32 + __ffs(hits) - 1;
      hits &= hits - 1;
      const int idx = kk * BD_CHUNK + lane;
      const AT at = atoms[idx];
      FT l0 = 0, l1 = 0, l2 = 0;
      bool cand = false;
      if (fabs(at.w) >= (FT)1e-9) {
        const FT d0 = (FT)at.x - cx, d1 = (FT)at.y - cy, d2 = (FT)at.z - cz;
        l0 = Rt[0] * d0 + Rt[3] * d1 + Rt[6] * d2;
        l1 = Rt[1] * d0 + Rt[4] * d1 + Rt[7] * d2;
        l2 = Rt[2] * d0 + Rt[5] * d1 + Rt[8] * d2;
        cand = l0 > lox && l0 < hix && l1 > loy && l1 < hiy && l2 > loz && l2 < hiz;
        if constexpr (sizeof(FT) == 4) {
          // within 1e-3 A of a face the FP64 box test decides (the set of atoms is the FP64 one)
          const float m = fminf(fminf(fminf(l0 - lox, hix - l0), fminf(l1 - loy, hiy - l1)),
                                fminf(l2 - loz, hiz - l2));
          if (fabsf(m) < 1e-3f) {
            const double q[4] = {B.q[slot], B.q[B.cap + slot], B.q[2 * B.cap + slot], B.q[3 * B.cap + slot]};
            double R[9];
            quat_to_rot(q, R);
            const double4 a64 = S.rec[idx];
            const double e0 = a64.x - B.c[slot], e1 = a64.y - B.c[B.cap + slot], e2 = a64.z - B.c[2 * B.cap + slot];
            cand = in_box(g, R[0] * e0 + R[3] * e1 + R[6] * e2, R[1] * e0 + R[4] * e1 + R[7] * e2,
                          R[2] * e0 + R[5] * e1 + R[8] * e2);
          }
        }
      }
      const unsigned m = __ballot_sync(FULL, cand);
      if (cand) buf[head + __popc(m & ((1u << lane) - 1u))] = Vec4<FT>::make(l0, l1, l2, (FT)at.w);
      head += __popc(m);
    }
    __syncwarp();
    // drain whole groups of 32 (everything once the chunks are done): entry e by lane e mod 32
    const int n_drain = done ? head : (head & ~31);
    const FT alpha = (FT)S.alpha;
#pragma unroll 1
    for (int e = lane; e < n_drain; e += 32) {
      const V4 v = buf[e];
      const StencilOut<FT, 1> st = stencil<FT, 1, FT>(g, v.x, v.y, v.z);
      const FT cf = -alpha * v.w * v.w;
      const FT g0 = cf * st.gx[0], g1 = cf * st.gy[0], g2 = cf * st.gz[0];
      rs0 += g0;
      rs1 += g1;
      rs2 += g2;
      if (TORQUE) {
        const double x = (double)v.x, y = (double)v.y, z = (double)v.z;
        u[0] += y * (double)g2 - z * (double)g1;
        u[1] += z * (double)g0 - x * (double)g2;
        u[2] += x * (double)g1 - y * (double)g0;
      }
      nr += 1;
    }
    if (done) break;
    // the remainder (fewer than 32 entries) moves to the front of the buffer
    __syncwarp();
    const int rem = head - n_drain;
    V4 keep{};
    if (lane < rem) keep = buf[n_drain + lane];
    __syncwarp();
    if (lane < rem) buf[lane] = keep;
    __syncwarp();
    head = rem;
  }
  __syncwarp();  // the buffer is reused by the next pose
  r[0] += (double)rs0;
  r[1] += (double)rs1;
  r[2] += (double)rs2;
}

template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 4) split_rev_kernel(DevSystem S, SlotBuf B, SplitBuf U,
                                                           unsigned long long* ctr) {
  using V4 = typename Vec4<FT>::type;
  __shared__ V4 bufs[8][kSplitBuf];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int n = U.cnt[0];
  unsigned nr = 0;
  for (;;) {
    int j = 0;
    if (lane == 0) j = atomicAdd(U.cnt + 1, 1);
    j = __shfl_sync(FULL, j, 0);
    if (j >= n) break;
    const int slot = U.list[j];
    double r[3] = {0, 0, 0}, u[3] = {0, 0, 0};
    lean_reverse_born<FT, TORQUE>(S, B, slot, lane, bufs[threadIdx.x >> 5], r, u, nr);
    r[0] = gsum<32>(r[0], FULL);
    r[1] = gsum<32>(r[1], FULL);
    r[2] = gsum<32>(r[2], FULL);
    if (TORQUE) {
      u[0] = gsum<32>(u[0], FULL);
      u[1] = gsum<32>(u[1], FULL);
      u[2] = gsum<32>(u[2], FULL);
    }
    if (lane < 3) U.rv[6 * slot + lane] = r[lane];
    else if (lane < 6) U.rv[6 * slot + lane] = u[lane - 3];
  }
  nr = gsumu<32>(nr, FULL);
  if (lane == 0 && nr) atomicAdd(ctr + C_REV_EVALS, (unsigned long long)nr);
}

template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 2) split_end_kernel(DevSystem S, DevSim P, SlotBuf B,
                                                           const int* __restrict__ n_live, SplitBuf U) {
  const BlockShared sh = block_shared_begin(S, P);
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, n_warps = (gridDim.x * blockDim.x) >> 5;
  const int live = *n_live;
  Tally tl{};
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
    if (need) {
      quat_to_rot(tr.q, R);
      r = norm3(tr.c[0], tr.c[1], tr.c[2]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = U.F[3 * slot + k];
        T[k] = U.T[3 * slot + k];
      }
      if (mode == 3) {
        // the reverse-Born force on the receptor, rotated to the lab frame, acts on the ligand
        // with the opposite sign
        const double* rv = U.rv + 6 * slot;
#pragma unroll
        for (int k = 0; k < 3; ++k) F[k] = F[k] - (R[3 * k] * rv[0] + R[3 * k + 1] * rv[1] + R[3 * k + 2] * rv[2]);
        if (TORQUE) {
#pragma unroll
          for (int k = 0; k < 3; ++k)
            T[k] = T[k] - (R[3 * k] * rv[3] + R[3 * k + 1] * rv[4] + R[3 * k + 2] * rv[5]);
        }
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
    const bool ovl = warp_overlap(S, cn, need && ok && P.overlap, lane, sh.v);
    if (need && ok) {
      const double c0[3] = {tr.c[0], tr.c[1], tr.c[2]};
      st = step_end(S, P, key, s, tr, R, cn, qn, !ovl, dt, tl);
      if (P.stats) {
        stats_step(S, P, tr, s, U.rprev[slot], dt, c0, R, sh.stats);
        trace_step(P, tr, s, F, dt);
        if (st == ST_REACTED) stats_encounter(P, tr, s, true);
      }
    }
    if (need && st != ST_RUNNING) {
      tr.status = st;
      P.out_status[tr.id] = (int8_t)st;
      P.out_steps[tr.id] = tr.steps;
      P.out_returns[tr.id] = tr.rets;
      tl.reacted += st == ST_REACTED;
      tl.escaped += st == ST_ESCAPED;
      tl.maxsteps += st == ST_MAXSTEPS;
    }
    bool dead = !own;
    warp_refill(P, tr, dead, lane);
    if (own) {
      store_slot(B, slot, tr);
      // rejected and still running: the next step starts from the same pose with these forces
      const bool keep = need && ok && ovl && st == ST_RUNNING;
      if (keep && mode != 2) {
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
  stats_block_end(P, sh.stats);
}

}  // namespace bd
