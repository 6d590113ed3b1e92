// Heterogeneous batch: trajectories of several receptor-ligand systems (each
// with its own grids, atoms, reaction pairs and run parameters) share one slot
// pool and one persistent launch.  The trajectory index space is the
// concatenation of the systems' ranges; a slot stores the global index, and the
// system is found by a binary search over the prefix sums.  Every per-system
// quantity is read from device tables of DevSystem / DevSim, so the step itself
// is the same device code as the single-system warp stepper.  No reference
// counterpart (the reference runs one system per process).
#pragma once

#include "bd_kernels.cuh"

namespace bd {

struct MultiTab {
  const DevSystem* sys;     // n_sys systems
  const DevSim* sim;        // n_sys run parameters (ctr: the shared counters)
  const long long* base;    // n_sys + 1: first global index of each system, then the total
  int n_sys;
  long long total;
  unsigned long long* ctr;  // shared counters: pending cursor over global indices, slot cursor, tallies
};

// System of global trajectory index g (the last s with base[s] <= g).
__device__ __forceinline__ int sys_of(const MultiTab& T, long long g) {
  int lo = 0, hi = T.n_sys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (T.base[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// warp_forces where every lane's trajectory may belong to another system.
template <typename FT, bool TORQUE>
__device__ __forceinline__ void warp_forces_multi(const MultiTab& T, int sys, const double c[3], const double R[9],
                                                  bool need, double F[3], double Tq[3], int lane, Counts& cnt) {
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
    const int sj = __shfl_sync(FULL, sys, j);
    double f[3], t[3], e;
    group_forces<FT, 32, TORQUE, false>(T.sys[sj], cj, Rj, lane, FULL, PosFromPose{Rj, cj}, f, t, e, cnt);
    if (lane == j) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = f[k];
        Tq[k] = t[k];
      }
    }
  }
}

__device__ __forceinline__ bool warp_overlap_multi(const MultiTab& T, int sys, const double cn[3], bool need,
                                                   int lane) {
  const unsigned FULL = 0xffffffffu;
  unsigned m = __ballot_sync(FULL, need);
  bool mine = false;
  while (m) {
    const int j = __ffs(m) - 1;
    m &= m - 1;
    double cj[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cj[k] = __shfl_sync(FULL, cn[k], j);
    const int sj = __shfl_sync(FULL, sys, j);
    const bool hit = overlap_any<32>(T.sys[sj], cj, lane, FULL, RecView{nullptr, nullptr});
    if (lane == j) mine = hit;
  }
  return mine;
}

// Lanes whose trajectory ended take the next global indices (one atomic per warp).
__device__ __forceinline__ void multi_refill(const MultiTab& T, Traj& tr, int& sys, bool& dead, int lane) {
  const unsigned FULL = 0xffffffffu;
  const bool want = !dead && tr.status != ST_RUNNING;
  const unsigned wm = __ballot_sync(FULL, want);
  if (!wm) return;
  const int leader = __ffs(wm) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(T.ctr + C_PENDING, (unsigned long long)__popc(wm));
  base = __shfl_sync(FULL, base, leader);
  if (want) {
    const long long g = (long long)(base + __popc(wm & ((1u << lane) - 1u)));
    if (g >= T.total) {
      tr.status = ST_EMPTY;
      dead = true;
    } else {
      sys = sys_of(T, g);
      start_trajectory(T.sim[sys], (int)(g - T.base[sys]), tr);
    }
  }
}

__global__ void init_slots_multi_kernel(MultiTab T, SlotBuf B, int n_slots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots) return;
  const int s = sys_of(T, i);
  Traj tr;
  start_trajectory(T.sim[s], (int)(i - T.base[s]), tr);
  tr.id = i;  // slots hold global indices
  store_slot(B, i, tr);
}

// The warp-cooperative persistent stepper over a heterogeneous pool (statistics
// and receptor staging are off in this mode).
template <typename FT, bool TORQUE>
__global__ void __launch_bounds__(256, 2) step_kernel_multi(MultiTab T, SlotBuf B, const int* __restrict__ n_live,
                                                            int K) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int live = *n_live;
  Tally tl{};
  for (;;) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(T.ctr + C_SLOT_CURSOR, 32ull);
    b = __shfl_sync(FULL, b, 0);
    if (b >= (unsigned long long)live) break;
    const int slot = (int)b + lane;
    const bool own = slot < live;
    Traj tr{};
    tr.status = ST_EMPTY;
    int sys = 0;
    if (own) {
      load_slot(B, slot, tr);
      sys = sys_of(T, tr.id);
      tr.id = (int)(tr.id - T.base[sys]);
    }
    bool dead = !own;
    double F[3] = {0, 0, 0}, Tq[3] = {0, 0, 0};
    bool fresh = false;  // F, Tq are the forces at the current pose (kept over rejected steps)
    for (int k = 0; k < K; ++k) {
      multi_refill(T, tr, sys, dead, lane);
      if (__all_sync(FULL, dead)) break;
      const DevSim& P = T.sim[sys];
      const DevSystem& S = T.sys[sys];
      const Keyed key = traj_key(P, tr.id);
      const uint32_t s = (uint32_t)tr.steps;
      double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, r = 0;
      int st = ST_EMPTY;
      if (!dead) {
        const int rets0 = tr.rets;
        st = step_begin(S, P, key, s, tr, R, r, tl);
        if (tr.rets != rets0) fresh = false;
      }
      const bool need_f = !dead && st == ST_RUNNING;
      warp_forces_multi<FT, TORQUE>(T, sys, tr.c, R, need_f && !fresh, F, Tq, lane, tl.cnt);
      double cn[3] = {0, 0, 0}, qn[4] = {1, 0, 0, 0}, dt = 0;
      bool ok = true;
      if (need_f) ok = step_move<FT>(S, P, key, s, tr, R, r, F, Tq, cn, qn, dt);
      if (need_f && !ok) {
        tl.nonfinite += 1;
        st = ST_ERROR;
      }
      const bool ovl = warp_overlap_multi(T, sys, cn, need_f && ok && P.overlap, lane);
      fresh = need_f && ok && ovl;
      if (need_f && ok) st = step_end(S, P, key, s, tr, R, cn, qn, !ovl, dt, tl);
      if (st != ST_RUNNING) fresh = false;
      if (!dead && st != ST_RUNNING) {
        tr.status = st;
        P.out_status[tr.id] = (int8_t)st;
        P.out_steps[tr.id] = tr.steps;
        P.out_returns[tr.id] = tr.rets;
        tl.reacted += st == ST_REACTED;
        tl.escaped += st == ST_ESCAPED;
        tl.maxsteps += st == ST_MAXSTEPS;
      }
    }
    multi_refill(T, tr, sys, dead, lane);
    if (own) {
      tr.id = (int)(T.base[sys] + tr.id);
      store_slot(B, slot, tr);
    }
  }
  flush_tally(T.sim[0], tl, true);  // every table entry's ctr is the shared counter array
}

}  // namespace bd
