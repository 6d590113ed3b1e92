// Kernels of the batched BD engine: fused per-trajectory forces, the persistent
// K-step stepper with refill from the pending pool, and slot compaction.
#pragma once

#include "bd_device.cuh"

namespace bd {

template <int G>
__device__ __forceinline__ double gsum(double v, unsigned m) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o, G);
  return v;
}

template <int G>
__device__ __forceinline__ unsigned gsumu(unsigned v, unsigned m) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o, G);
  return v;
}

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (G == 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
  }
}

struct Counts {
  unsigned grid, rev, ff;
};

// FP32 copy of the receptor table staged in shared memory by the stepper
// kernels (null members: read the FP64 table from global memory).  Tests on it
// only prune: they keep every atom within the FP64 test's reach plus a margin
// far above the FP32 rounding of coordinates of tens of Angstrom, and the FP64
// test then decides, so results do not depend on which path ran.
struct RecView {
  const float4* rec;
  const float4* chunks;
};
constexpr float kPruneMargin = 1e-3f;  // A

// Bit j set: receptor chunk k0 + j has a bounding sphere within `reach` of c.
// Lane j of the group tests chunk k0 + j; the mask is the same on every lane.
template <int G>
__device__ __forceinline__ unsigned chunk_hits(const DevSystem& S, const RecView& v, const double c[3], double reach,
                                               int k0, int lane, unsigned gm) {
  const int k = k0 + lane;
  bool hit = false;
  if (k < S.n_chunks) {
    if (v.chunks) {
      const float4 sp = v.chunks[k];
      const float dx = sp.x - (float)c[0], dy = sp.y - (float)c[1], dz = sp.z - (float)c[2];
      const float lim = (float)reach + sp.w + kPruneMargin;
      hit = dx * dx + dy * dy + dz * dz < lim * lim;
    } else {
      const double4 sp = S.chunks[k];
      const double dx = sp.x - c[0], dy = sp.y - c[1], dz = sp.z - c[2];
      const double lim = reach + sp.w;
      hit = dx * dx + dy * dy + dz * dz < lim * lim;
    }
  }
  if constexpr (G == 1) {
    return hit ? 1u : 0u;
  } else {
    unsigned m = __ballot_sync(gm, hit);
    if constexpr (G < 32) m = (m >> ((threadIdx.x & 31u) & ~(unsigned)(G - 1))) & ((1u << G) - 1u);
    return m;
  }
}

// Lab-frame offset ro = x - c and lab position x of ligand atom i.
struct PosFromPose {
  const double* R;
  const double* c;
  __device__ __forceinline__ void operator()(int, const double4& a, double ro[3], double x[3]) const {
    ro[0] = R[0] * a.x + R[1] * a.y + R[2] * a.z;
    ro[1] = R[3] * a.x + R[4] * a.y + R[5] * a.z;
    ro[2] = R[6] * a.x + R[7] * a.y + R[8] * a.z;
    x[0] = c[0] + ro[0];
    x[1] = c[1] + ro[1];
    x[2] = c[2] + ro[2];
  }
};

struct PosFromAtoms {
  const double* p;  // this trajectory's (n_lig, 3) lab positions
  const double* c;
  __device__ __forceinline__ void operator()(int i, const double4&, double ro[3], double x[3]) const {
    x[0] = p[3 * i];
    x[1] = p[3 * i + 1];
    x[2] = p[3 * i + 2];
    ro[0] = x[0] - c[0];
    ro[1] = x[1] - c[1];
    ro[2] = x[2] - c[2];
  }
};

// Reverse Born (direction 2) of one trajectory by a whole warp.  Receptor
// chunks are culled against the ligand Born grid's margin box in the ligand
// frame; the in-box atoms of the surviving chunks are queued in a per-warp ring
// in shared memory and interpolated 32 at a time, so the stencil runs on full
// warps however sparsely a chunk overlaps the box.
// Geometry is in FT: FP64 in the FP64 engine; FP32 in mixed precision, where a
// box decision within 1e-3 A of a face (far above the FP32 rotation error for
// coordinates of hundreds of A) is taken again in FP64, so the set of
// contributing atoms is exactly the FP64 one in both modes.
// Blocks have at most 256 threads (every caller's launch bound): 8 rings.
constexpr int kRevRing = 64;  // > 31 pending + 32 new candidates

template <typename T>
struct Vec4;
template <>
struct Vec4<float> {
  using type = float4;
  static __device__ __forceinline__ float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};
template <>
struct Vec4<double> {
  using type = double4;
  static __device__ __forceinline__ double4 make(double a, double b, double c, double d) {
    return make_double4(a, b, c, d);
  }
};

template <typename FT, bool TORQUE>
__device__ __forceinline__ void warp_reverse_born(const DevSystem& S, const double c[3], const double R[9], int lane,
                                                  double r[3], double u[3], unsigned& nr) {
  using V4 = typename Vec4<FT>::type;
  __shared__ V4 rings[8][kRevRing];
  V4* ring = rings[threadIdx.x >> 5];
  const unsigned FULL = 0xffffffffu;
  const DevGrid& g = S.lig_born;
  const FT alpha = (FT)S.alpha;
  const FT Rt[9] = {(FT)R[0], (FT)R[1], (FT)R[2], (FT)R[3], (FT)R[4], (FT)R[5], (FT)R[6], (FT)R[7], (FT)R[8]};
  const FT lox = (FT)g.lox, loy = (FT)g.loy, loz = (FT)g.loz, hix = (FT)g.hix, hiy = (FT)g.hiy, hiz = (FT)g.hiz;
  unsigned head = 0, tail = 0;  // warp-uniform ring cursors
  FT rs0 = 0, rs1 = 0, rs2 = 0;  // per-lane sums in FT (at most a few dozen terms per lane)
  auto drain = [&](unsigned count) {
    if ((unsigned)lane < count) {
      const V4 e = ring[(tail + lane) % kRevRing];
      const StencilOut<FT, 1> st = stencil<FT, 1, FT>(g, e.x, e.y, e.z);
      const FT qr = (FT)e.w;
      const FT cf = -alpha * qr * qr;
      const FT g0 = cf * st.gx[0], g1 = cf * st.gy[0], g2 = cf * st.gz[0];
      rs0 += g0;
      rs1 += g1;
      rs2 += g2;
      if (TORQUE) {
        const double x = (double)e.x, y = (double)e.y, z = (double)e.z;
        u[0] += y * (double)g2 - z * (double)g1;
        u[1] += z * (double)g0 - x * (double)g2;
        u[2] += x * (double)g1 - y * (double)g0;
      }
      nr += 1;
    }
    tail += count;
  };
  // Atom rows of the sweep: the FP32 table in mixed precision (offsets from an
  // FP32 centre are good to ~1e-5 A, far inside the 1e-3 A re-check band).
  using AT = typename Vec4<FT>::type;
  const AT* atoms = nullptr;
  if constexpr (sizeof(FT) == 4) atoms = S.rec_f;
  else atoms = S.rec;
  const FT cx = (FT)c[0], cy = (FT)c[1], cz = (FT)c[2];
  // one hit chunk: lane = atom; in-box atoms go to the ring in lane order
  auto gather = [&](const AT& at, int idx) {
    FT l0 = 0, l1 = 0, l2 = 0;
    bool cand = false;
    if (fabs(at.w) >= (FT)1e-9) {
      FT d0, d1, d2;
      if constexpr (sizeof(FT) == 4) {
        d0 = at.x - cx;
        d1 = at.y - cy;
        d2 = at.z - cz;
      } else {
        d0 = at.x - c[0];
        d1 = at.y - c[1];
        d2 = at.z - c[2];
      }
      l0 = Rt[0] * d0 + Rt[3] * d1 + Rt[6] * d2;
      l1 = Rt[1] * d0 + Rt[4] * d1 + Rt[7] * d2;
      l2 = Rt[2] * d0 + Rt[5] * d1 + Rt[8] * d2;
      cand = l0 > lox && l0 < hix && l1 > loy && l1 < hiy && l2 > loz && l2 < hiz;
      if constexpr (sizeof(FT) == 4) {
        const float m = fminf(fminf(fminf(l0 - lox, hix - l0), fminf(l1 - loy, hiy - l1)),
                              fminf(l2 - loz, hiz - l2));
        if (fabsf(m) < 1e-3f) {
          const double4 a64 = S.rec[idx];
          const double e0 = a64.x - c[0], e1 = a64.y - c[1], e2 = a64.z - c[2];
          cand = in_box(g, R[0] * e0 + R[3] * e1 + R[6] * e2, R[1] * e0 + R[4] * e1 + R[7] * e2,
                        R[2] * e0 + R[5] * e1 + R[8] * e2);
        }
      }
    }
    const unsigned m = __ballot_sync(FULL, cand);
    if (cand) ring[(head + __popc(m & ((1u << lane) - 1u))) % kRevRing] = Vec4<FT>::make(l0, l1, l2, (FT)at.w);
    head += __popc(m);
    if (head - tail >= 32) {
      __syncwarp();
      drain(32);
      __syncwarp();
    }
  };
  for (int k0 = 0; k0 < S.n_chunks; k0 += 32) {
    const int k = k0 + lane;
    bool hit = false;
    if (k < S.n_chunks) {
      FT d0, d1, d2, rad;
      if constexpr (sizeof(FT) == 4) {  // FP32 centres: ~1e-5 A off, inside the 1e-3 A margin below
        const float4 sp = S.chunks_f[k];
        d0 = sp.x - cx;
        d1 = sp.y - cy;
        d2 = sp.z - cz;
        rad = sp.w;
      } else {
        const double4 sp = S.chunks[k];
        d0 = sp.x - c[0];
        d1 = sp.y - c[1];
        d2 = sp.z - c[2];
        rad = sp.w;
      }
      const FT l0 = Rt[0] * d0 + Rt[3] * d1 + Rt[6] * d2;
      const FT l1 = Rt[1] * d0 + Rt[4] * d1 + Rt[7] * d2;
      const FT l2 = Rt[2] * d0 + Rt[5] * d1 + Rt[8] * d2;
      const FT ex = fmax(fmax(lox - l0, l0 - hix), (FT)0);
      const FT ey = fmax(fmax(loy - l1, l1 - hiy), (FT)0);
      const FT ez = fmax(fmax(loz - l2, l2 - hiz), (FT)0);
      // the radius is inflated against rounding; the extra margin covers FP32 geometry
      const FT lim = rad + (sizeof(FT) == 4 ? (FT)1e-3 : (FT)1e-9);
      hit = ex * ex + ey * ey + ez * ez < lim * lim;
    }
    unsigned hits = __ballot_sync(FULL, hit);
    if (!hits) continue;
    // software-pipelined: the next hit chunk's atoms load while this one is tested
    int kk = k0 + __ffs(hits) - 1;
    hits &= hits - 1;
    AT at = atoms[kk * BD_CHUNK + lane];
    for (;;) {
      const int kn = hits ? k0 + __ffs(hits) - 1 : -1;
      hits &= hits - 1;
      AT an = at;
      if (kn >= 0) an = atoms[kn * BD_CHUNK + lane];
      gather(at, kk * BD_CHUNK + lane);
      kk = kn;
      if (kn < 0) break;
      at = an;
    }
  }
  __syncwarp();
  drain(head - tail);
  __syncwarp();  // the ring is reused by the next call
  r[0] += (double)rs0;
  r[1] += (double)rs1;
  r[2] += (double)rs2;
}

template <int G>
__device__ __forceinline__ double gmax(double v, unsigned m) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(m, v, o, G));
  return v;
}

constexpr double kWcaCut = 1.122462;  // the WCA cutoff in units of sigma (2^(1/6) to 7 digits)

// WCA contact forces of one pose (gpu_batch_engine.py:474-529): every ligand atom
// against every receptor atom, charged or not, with sigma = r_lig + r_rec and
// force eps (12 (sigma/r)^12 - 6 (sigma/r)^6) / r^2 along (x_lig - x_rec) / r for
// r < 1.122462 sigma, where r = sqrt(max(r^2, 1e-6)) and the r^2 divisor is the
// unclamped one, as the reference computes them.  Only receptor chunks whose
// bounding spheres come within the largest pair cutoff of the ligand's bounding
// sphere about c are read.  Lanes own ligand atoms and read each hit chunk's
// receptor atoms together (same address on every lane).  Adds this lane's share
// of the force, and of the torque about c, to f / t.
template <int G, bool TORQUE, class PosFn>
__device__ void group_contact(const DevSystem& S, const double c[3], int lane, unsigned gm, const PosFn& pos,
                              double f[3], double t[3]) {
  const int nl = S.n_lig;
  double ext2 = 0;
  for (int i = lane; i < nl; i += G) {
    double ro[3], x[3];
    pos(i, S.lig[i], ro, x);
    ext2 = fmax(ext2, ro[0] * ro[0] + ro[1] * ro[1] + ro[2] * ro[2]);
  }
  if constexpr (G > 1) ext2 = gmax<G>(ext2, gm);
  const double reach = sqrt(ext2) * (1 + 1e-12) + S.wca_cut + 1e-6;
  for (int k0 = 0; k0 < S.n_chunks; k0 += G) {
    unsigned hits = chunk_hits<G>(S, RecView{nullptr, nullptr}, c, reach, k0, lane, gm);
    while (hits) {
      const int k = k0 + __ffs(hits) - 1;
      hits &= hits - 1;
      const double4* ra = S.rec + (size_t)k * BD_CHUNK;
      const double* rr = S.rec_rad + (size_t)k * BD_CHUNK;
      for (int i = lane; i < nl; i += G) {
        double ro[3], x[3];
        pos(i, S.lig[i], ro, x);
        const double rl = S.lig_rad[i];
        double g0 = 0, g1 = 0, g2 = 0;
        for (int a = 0; a < BD_CHUNK; ++a) {
          const double4 at = ra[a];
          const double d0 = x[0] - at.x, d1 = x[1] - at.y, d2 = x[2] - at.z;
          const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
          const double r = sqrt(fmax(r2, 1e-6));
          const double sig = rl + rr[a];
          if (!(r < kWcaCut * sig)) continue;
          const double sr = sig / r, sr2 = sr * sr, sr6 = sr2 * sr2 * sr2, sr12 = sr6 * sr6;
          const double fm = S.wca_eps * (12.0 * sr12 - 6.0 * sr6) / r2;
          g0 += fm * d0 / r;
          g1 += fm * d1 / r;
          g2 += fm * d2 / r;
        }
        f[0] += g0;
        f[1] += g1;
        f[2] += g2;
        if (TORQUE) {
          t[0] += ro[1] * g2 - ro[2] * g1;
          t[1] += ro[2] * g0 - ro[0] * g2;
          t[2] += ro[0] * g1 - ro[1] * g0;
        }
      }
    }
  }
}

// Net force, torque (about c) and energy on the ligand of one trajectory,
// computed cooperatively by the G lanes of a group.  Follows
// GPUBatchForceEngine.__call__ (pystarc/forces/gpu_batch_engine.py:531-605):
// elec grid (finest containing grid) or Yukawa multipole far-field, Born
// direction 1 on the receptor Born grid, Born direction 2 on the ligand Born
// grid at the receptor atoms with the force negated, and the WCA contact forces
// when they are on.  Every lane returns the same totals.
// REV = false compiles the function without Born direction 2 (the split stepper sweeps it in a
// kernel of its own).
template <typename FT, int G, bool TORQUE, bool ENERGY, class PosFn, bool REV = true>
__device__ void group_forces(const DevSystem& S, const double c[3], const double R[9], int lane, unsigned gm,
                             const PosFn& pos, double F[3], double T[3], double& E, Counts& cnt,
                             const RecView& v = RecView{nullptr, nullptr}, unsigned terms = 15u) {
  double f0 = 0, f1 = 0, f2 = 0, t0 = 0, t1 = 0, t2 = 0, e = 0;
  const bool t_grid = terms & 1u, t_ff = terms & 2u, t_rev = terms & 4u;
  unsigned ng = 0, nf = 0, nr = 0;
  const int nl = S.n_lig;
  for (int i = lane; i < nl; i += G) {
    const double4 a = S.lig[i];
    if (fabs(a.w) < 1e-9) continue;
    double ro[3], x[3];
    pos(i, a, ro, x);
    const FT q = (FT)a.w;
    FT fa0 = 0, fa1 = 0, fa2 = 0, ea = 0;
    int gi = -1;
    for (int k = 0; k < S.n_elec; ++k)
      if (in_box(S.elec[k], x[0], x[1], x[2])) {
        gi = k;
        break;
      }
    const bool bin = S.has_born && in_box(S.born, x[0], x[1], x[2]);
    const FT cb = (FT)S.alpha * q * q;
    if (gi == 0 && bin && S.paired) {
      if (!t_grid) continue;
      const StencilOut<FT, 2> s = stencil<FT, 2>(S.pair, x[0], x[1], x[2]);
      fa0 = -q * s.gx[0] - cb * s.gx[1];
      fa1 = -q * s.gy[0] - cb * s.gy[1];
      fa2 = -q * s.gz[0] - cb * s.gz[1];
      if (ENERGY) ea = q * s.phi[0] + cb * s.phi[1];
      ng += 2;
    } else {
      if (gi >= 0) {
        if (t_grid) {
        const StencilOut<FT, 1> s = stencil<FT, 1>(S.elec[gi], x[0], x[1], x[2]);
        fa0 = -q * s.gx[0];
        fa1 = -q * s.gy[0];
        fa2 = -q * s.gz[0];
        if (ENERGY) ea = q * s.phi[0];
        ng += 1;
        }
      } else if (S.has_yukawa && t_ff) {
        FT ff[3], ef;
        farfield<FT>(S, x[0], x[1], x[2], q, ff, ef);
        fa0 = ff[0];
        fa1 = ff[1];
        fa2 = ff[2];
        if (ENERGY) ea = ef;
        nf += 1;
      }
      if (bin && t_grid) {
        const StencilOut<FT, 1> s = stencil<FT, 1>(S.born, x[0], x[1], x[2]);
        fa0 -= cb * s.gx[0];
        fa1 -= cb * s.gy[0];
        fa2 -= cb * s.gz[0];
        if (ENERGY) ea += cb * s.phi[0];
        ng += 1;
      }
    }
    f0 += (double)fa0;
    f1 += (double)fa1;
    f2 += (double)fa2;
    if (ENERGY) e += (double)ea;
    if (TORQUE) {
      t0 += ro[1] * (double)fa2 - ro[2] * (double)fa1;
      t1 += ro[2] * (double)fa0 - ro[0] * (double)fa2;
      t2 += ro[0] * (double)fa1 - ro[1] * (double)fa0;
    }
  }
  // WCA contact forces, for centroids within the activation radius (gpu_batch_engine.py:488-490)
  if ((terms & 8u) && S.wca && norm3(c[0], c[1], c[2]) < S.wca_act) {
    double wf[3] = {f0, f1, f2}, wt[3] = {t0, t1, t2};
    group_contact<G, TORQUE>(S, c, lane, gm, pos, wf, wt);
    f0 = wf[0];
    f1 = wf[1];
    f2 = wf[2];
    t0 = wt[0];
    t1 = wt[1];
    t2 = wt[2];
  }
  // Born direction 2: ligand Born grid at the receptor atoms, in the ligand frame.
  // Lanes test G receptor chunks at a time against the box's circumsphere, then
  // sweep the hit chunks' atoms together.
  double r0 = 0, r1 = 0, r2 = 0, u0 = 0, u1 = 0, u2 = 0;
  if constexpr (!REV) {
  } else if constexpr (G == 32) {
    if (t_rev && S.born_rev && norm3(c[0], c[1], c[2]) - S.rec_max_r < S.lig_born_rho) {
      double rr[3] = {0, 0, 0}, uu[3] = {0, 0, 0};
      warp_reverse_born<FT, TORQUE>(S, c, R, lane, rr, uu, nr);
      r0 = rr[0];
      r1 = rr[1];
      r2 = rr[2];
      u0 = uu[0];
      u1 = uu[1];
      u2 = uu[2];
    }
  } else if (t_rev && S.born_rev) {
    const double rho = S.lig_born_rho;
    if (norm3(c[0], c[1], c[2]) - S.rec_max_r < rho) {
      const double rho2 = rho * rho;
      const float cf0 = (float)c[0], cf1 = (float)c[1], cf2 = (float)c[2];
      const float rho_f = (float)rho + kPruneMargin, rho_f2 = rho_f * rho_f;
      for (int k0 = 0; k0 < S.n_chunks; k0 += G) {
       unsigned hits = chunk_hits<G>(S, v, c, rho, k0, lane, gm);
       while (hits) {
        const int k = k0 + __ffs(hits) - 1;
        hits &= hits - 1;
        for (int a = lane; a < BD_CHUNK; a += G) {
          if (v.rec) {
            const float4 af = v.rec[k * BD_CHUNK + a];
            const float e0 = af.x - cf0, e1 = af.y - cf1, e2 = af.z - cf2;
            if (e0 * e0 + e1 * e1 + e2 * e2 >= rho_f2) continue;
          }
          const double4 at = S.rec[k * BD_CHUNK + a];
          if (fabs(at.w) < 1e-9) continue;
          const double d0 = at.x - c[0], d1 = at.y - c[1], d2 = at.z - c[2];
          if (d0 * d0 + d1 * d1 + d2 * d2 >= rho2) continue;
          const double l0 = R[0] * d0 + R[3] * d1 + R[6] * d2;
          const double l1 = R[1] * d0 + R[4] * d1 + R[7] * d2;
          const double l2 = R[2] * d0 + R[5] * d1 + R[8] * d2;
          if (!in_box(S.lig_born, l0, l1, l2)) continue;
          const StencilOut<FT, 1> s = stencil<FT, 1>(S.lig_born, l0, l1, l2);
          const FT qr = (FT)at.w;
          const FT cf = -(FT)S.alpha * qr * qr;
          const FT g0 = cf * s.gx[0], g1 = cf * s.gy[0], g2 = cf * s.gz[0];
          r0 += (double)g0;
          r1 += (double)g1;
          r2 += (double)g2;
          if (TORQUE) {
            u0 += l1 * (double)g2 - l2 * (double)g1;
            u1 += l2 * (double)g0 - l0 * (double)g2;
            u2 += l0 * (double)g1 - l1 * (double)g0;
          }
          nr += 1;
        }
       }
      }
    }
  }
  if (G > 1) {
    f0 = gsum<G>(f0, gm);
    f1 = gsum<G>(f1, gm);
    f2 = gsum<G>(f2, gm);
    if (ENERGY) e = gsum<G>(e, gm);
    if (TORQUE) {
      t0 = gsum<G>(t0, gm);
      t1 = gsum<G>(t1, gm);
      t2 = gsum<G>(t2, gm);
    }
    if (REV && S.born_rev) {
      r0 = gsum<G>(r0, gm);
      r1 = gsum<G>(r1, gm);
      r2 = gsum<G>(r2, gm);
      if (TORQUE) {
        u0 = gsum<G>(u0, gm);
        u1 = gsum<G>(u1, gm);
        u2 = gsum<G>(u2, gm);
      }
    }
  }
  // Reverse-Born force on the receptor, rotated to the lab frame, acts on the ligand with the opposite sign.
  F[0] = f0 - (R[0] * r0 + R[1] * r1 + R[2] * r2);
  F[1] = f1 - (R[3] * r0 + R[4] * r1 + R[5] * r2);
  F[2] = f2 - (R[6] * r0 + R[7] * r1 + R[8] * r2);
  if (TORQUE) {
    T[0] = t0 - (R[0] * u0 + R[1] * u1 + R[2] * u2);
    T[1] = t1 - (R[3] * u0 + R[4] * u1 + R[5] * u2);
    T[2] = t2 - (R[6] * u0 + R[7] * u1 + R[8] * u2);
  } else {
    T[0] = T[1] = T[2] = 0.0;
  }
  E = e;
  cnt.grid += ng;
  cnt.rev += nr;
  cnt.ff += nf;
}

// Parity kernel: one group per pose.  pose = centroid + quaternion (w,x,y,z) or rotation matrix.
template <typename FT, int G, bool TORQUE>
__global__ void __launch_bounds__(256) eval_pose_kernel(DevSystem S, long long n, const double* __restrict__ cen,
                                                        const double* __restrict__ rot, int rot_is_matrix,
                                                        double* __restrict__ F, double* __restrict__ T,
                                                        double* __restrict__ E, unsigned long long* ctr) {
  const int lane = threadIdx.x & (G - 1);
  const unsigned gm = group_mask<G>();
  const long long groups = (long long)gridDim.x * (blockDim.x / G);
  Counts cnt{0, 0, 0};
  for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G; t < n; t += groups) {
    double c[3] = {cen[3 * t], cen[3 * t + 1], cen[3 * t + 2]};
    double R[9];
    if (rot_is_matrix) {
#pragma unroll
      for (int k = 0; k < 9; ++k) R[k] = rot[9 * t + k];
    } else {
      double q[4] = {rot[4 * t], rot[4 * t + 1], rot[4 * t + 2], rot[4 * t + 3]};
      quat_to_rot(q, R);
    }
    double f[3], tq[3], e;
    group_forces<FT, G, TORQUE, true>(S, c, R, lane, gm, PosFromPose{R, c}, f, tq, e, cnt, RecView{nullptr, nullptr},
                                      S.terms);
    if (lane == 0) {
      F[3 * t] = f[0];
      F[3 * t + 1] = f[1];
      F[3 * t + 2] = f[2];
      T[3 * t] = tq[0];
      T[3 * t + 1] = tq[1];
      T[3 * t + 2] = tq[2];
      E[t] = e;
    }
  }
  if (ctr) {
    const unsigned g = gsumu<32>(cnt.grid, 0xffffffffu), r = gsumu<32>(cnt.rev, 0xffffffffu),
                   f = gsumu<32>(cnt.ff, 0xffffffffu);
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(ctr + C_GRID_EVALS, (unsigned long long)g);
      atomicAdd(ctr + C_REV_EVALS, (unsigned long long)r);
      atomicAdd(ctr + C_FF_EVALS, (unsigned long long)f);
    }
  }
}

// Parity kernel with explicit lab atom positions (the reference __call__ signature).
template <typename FT, int G, bool TORQUE>
__global__ void __launch_bounds__(256) eval_atoms_kernel(DevSystem S, long long n, const double* __restrict__ pos,
                                                         const double* __restrict__ Rm,
                                                         const double* __restrict__ cen, double* __restrict__ F,
                                                         double* __restrict__ T, double* __restrict__ E) {
  const int lane = threadIdx.x & (G - 1);
  const unsigned gm = group_mask<G>();
  const long long groups = (long long)gridDim.x * (blockDim.x / G);
  Counts cnt{0, 0, 0};
  for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / G; t < n; t += groups) {
    double c[3] = {cen[3 * t], cen[3 * t + 1], cen[3 * t + 2]};
    double R[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = Rm[9 * t + k];
    double f[3], tq[3], e;
    group_forces<FT, G, TORQUE, true>(S, c, R, lane, gm, PosFromAtoms{pos + (long long)t * S.n_lig * 3, c}, f,
                                      tq, e, cnt, RecView{nullptr, nullptr}, S.terms);
    if (lane == 0) {
      F[3 * t] = f[0];
      F[3 * t + 1] = f[1];
      F[3 * t + 2] = f[2];
      T[3 * t] = tq[0];
      T[3 * t + 1] = tq[1];
      T[3 * t + 2] = tq[2];
      E[t] = e;
    }
  }
}

// ----------------------------------------------------------------------------
// Stepper
// ----------------------------------------------------------------------------
struct Traj {
  double c[3], q[4];
  int id, steps, rets, status;
  int state;  // state-machine reaction state
};

struct Tally {
  unsigned long long steps;
  unsigned reacted, escaped, maxsteps, returns, overlap, bridge, nonfinite;
  Counts cnt;
};

__device__ __forceinline__ void flush_tally(const DevSim& P, Tally tl, bool owner);

__device__ __forceinline__ Keyed traj_key(const DevSim& P, int id) {
  const unsigned long long g = (unsigned long long)(P.id_offset + id);
  return Keyed{P.k0, P.k1, (uint32_t)(g & 0xffffffffull), (uint32_t)(g >> 32)};
}

__device__ __forceinline__ void start_trajectory(const DevSim& P, int id, Traj& tr) {
  const Keyed key = traj_key(P, id);
  const W4 a = key.w(INIT_STEP, SUB_INIT_DIR), b = key.w(INIT_STEP, SUB_INIT_DIR + 1);
  double v0, v1, v2, spare;
  box_muller(u53(a.a, a.b), u53(a.c, a.d), v0, v1);
  box_muller(u53(b.a, b.b), u53(b.c, b.d), v2, spare);
  const double n = norm3(v0, v1, v2);
  tr.c[0] = v0 / n * P.r_b;
  tr.c[1] = v1 / n * P.r_b;
  tr.c[2] = v2 / n * P.r_b;
  const W4 qa = key.w(INIT_STEP, SUB_INIT_Q), qb = key.w(INIT_STEP, SUB_INIT_Q + 1);
  shoemake(u53(qa.a, qa.b), u53(qa.c, qa.d), u53(qb.a, qb.b), tr.q);
  tr.id = id;
  tr.steps = 0;
  tr.rets = 0;
  tr.status = ST_RUNNING;
  tr.state = 0;
  if (P.stats) {
#pragma unroll
    for (int k = 0; k < 3; ++k) P.st.start_c[3 * id + k] = tr.c[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) P.st.start_q[4 * id + k] = tr.q[k];
  }
}

// Adaptive dt (pystarc/simulation/gpu_batch_simulator.py:961-1067).
// rc >= 0: state-machine mode, rc the distance to the nearest reaction surface reachable
// from the current state (1e30 if none): where 12 sqrt(2 D_t dt) exceeds it, dt drops to
// rc^2 / (288 D_t), floored at min_core_rxn_dt (gpu_batch_simulator.py:1005-1060).
__device__ __forceinline__ double adaptive_dt(const DevSim& P, double r, double rc = -1.0) {
  const double D_t = P.D_t;
  const double dt_pair = (0.1 * 0.1 / 2.0) * r * r / D_t;
  double dt_force = dt_pair;
  if (P.adt_has_force) {
    const double lam = P.adt_debye;
    const double expf_ = exp(-r / lam);
    const double Fr0 = P.adt_V0 * expf_ * (1.0 / (r * r) + 1.0 / (r * lam));
    const double Fr1 = -P.adt_V0 * expf_ / (lam * lam) - 2.0 * Fr0 / r;
    const double DFr1 = fabs(D_t * Fr1);
    if (DFr1 > 1e-15 && r < 3.0 * lam) dt_force = 0.01 / DFr1;
  }
  const double dist_b = fmax(r - P.r_b, 1e-3), dist_esc = fmax(P.r_esc - r, 1e-3);
  const double de = fmin(dist_b, dist_esc);
  const double dt_edge = de * de / (18.0 * D_t);
  double dt = (r > 1.1 * P.r_b) ? fmin(fmin(dt_force, dt_edge), dt_pair) : fmin(dt_force, dt_pair);
  if (rc >= 0.0 && 12.0 * sqrt(2.0 * D_t * dt) > rc) {
    const double crit = rc * rc / (288.0 * D_t);
    dt = fmin(dt, P.min_core_rxn_dt > 0 ? fmax(crit, P.min_core_rxn_dt) : crit);
  }
  if (P.max_dt > 0) dt = fmin(dt, P.max_dt);
  if (P.min_core_dt > 0) dt = fmax(dt, P.min_core_dt);
  return dt;
}

// Relative translational diffusion D_t - (2/3) tr M12(r) with the Zuk et al. (2014)
// three-regime RPY coupling M12 = kBT/eta (tt_I I + tt_uu r^ r^T), whose trace is
// kBT/eta (3 tt_I + tt_uu), clamped at 1e-12 (hydrodynamics/rotne_prager.py:67-124, :177-200).
template <typename FT>
__device__ __forceinline__ double zuk_diffusion(const DevSim& P, double rd) {
  if (rd < 1e-10) return fmax(P.D_t, 1e-12);  // M12 = 0 at coincident centres
  const FT pi = (FT)3.14159265358979323846;
  const FT r = (FT)rd, a = (FT)P.zuk_a, b = (FT)P.zuk_b;
  const FT r2 = r * r, r3 = r2 * r;
  FT tI, tuu;
  if (r > a + b) {  // far field
    const FT den = (FT)8 * pi * r, s2 = a * a + b * b;
    tI = ((FT)1 + s2 / ((FT)3 * r2)) / den;
    tuu = ((FT)1 - s2 / r2) / den;
  } else if (r > fabs(a - b)) {  // partial overlap
    const FT am2 = (a - b) * (a - b), den = (FT)192 * pi * a * b * r3, w = am2 + (FT)3 * r2;
    tI = ((FT)16 * r3 * (a + b) - w * w) / den;
    tuu = (FT)3 * (am2 - r2) * (am2 - r2) / den;
  } else {  // one sphere inside the other: self-mobility of the larger
    tI = (FT)1 / ((FT)6 * pi * fmax(a, b));
    tuu = 0;
  }
  const FT tr = (FT)P.zuk_kTeta * ((FT)3 * tI + tuu);
  return fmax(P.D_t - (2.0 / 3.0) * (double)tr, 1e-12);
}

// Relative translational diffusion with HI.  Reference GPU mode: far-field RPY along
// the line of centres, mu = 0.243, clamp 1e-6 (gpu_batch_simulator.py:741-751,
// :1074-1084); Zuk mode: zuk_diffusion.
template <typename FT>
__device__ __forceinline__ double hi_diffusion(const DevSim& P, double r) {
  if (!P.use_hi) return P.D_t;
  if (P.hi_mode == 1) return zuk_diffusion<FT>(P, r);
  const FT rm1 = (FT)1 / (FT)fmax(r, 0.01);
  const FT rm3 = rm1 * rm1 * rm1;
  const FT Df = (FT)P.hi_Df;
  const FT Di = (FT)-2 * Df * ((FT)2 * rm1 - ((FT)4 / (FT)3) * (FT)P.hi_a2 * rm3) / (FT)(8.0 * 3.14159265358979323846);
  const FT D = Df * (FT)P.hi_ainv + Di;
  return (double)(D > (FT)1e-6 ? D : (FT)1e-6);
}

// Overlap rejection test: is the new centroid within 1.5 A of any receptor atom
// (gpu_batch_simulator.py:1106-1128)?  Chunks whose bounding sphere is farther
// than 1.5 A are skipped; the answer is exact.  With the occupancy grid built, one lane
// answers alone from the cell holding c (overlap_cells); the answer is the same.
__device__ __forceinline__ bool overlap_cells(const DevSystem& S, const double c[3]);

template <int G>
__device__ __forceinline__ bool overlap_any(const DevSystem& S, const double c[3], int lane, unsigned gm,
                                            const RecView& v = RecView{nullptr, nullptr}) {
  if (S.ov_cell) return overlap_cells(S, c);
  bool any = false;
  if (norm3(c[0], c[1], c[2]) < S.rec_max_r + 1.5) {
    const float cf0 = (float)c[0], cf1 = (float)c[1], cf2 = (float)c[2];
    const float lim_f = 1.5f + kPruneMargin, lim_f2 = lim_f * lim_f;
    for (int k0 = 0; k0 < S.n_chunks && !any; k0 += G) {
      unsigned hits = chunk_hits<G>(S, v, c, 1.5, k0, lane, gm);
      bool hit = false;
      while (hits) {
        const int k = k0 + __ffs(hits) - 1;
        hits &= hits - 1;
        for (int a = lane; a < BD_CHUNK; a += G) {
          if (v.rec) {
            const float4 af = v.rec[k * BD_CHUNK + a];
            const float e0 = af.x - cf0, e1 = af.y - cf1, e2 = af.z - cf2;
            if (e0 * e0 + e1 * e1 + e2 * e2 >= lim_f2) continue;
          }
          const double4 at = S.rec[k * BD_CHUNK + a];
          if (norm3(c[0] - at.x, c[1] - at.y, c[2] - at.z) < 1.5) hit = true;
        }
      }
      any = G > 1 ? __any_sync(gm, hit) : hit;
    }
  }
  return any;
}

// ----------------------------------------------------------------------------
// Overlap occupancy grid.  The reference rejects a move when the new centroid lies within
// 1.5 A of any receptor atom (gpu_batch_simulator.py:770-781, 1102-1128).  Cells of
// kOvCell A over the receptor's box (widened by 1.5 A + one cell) are classified once:
// EMPTY when every atom is at least 1.5 A + kOvEps from the whole cell, FULL when some atom
// is within 1.5 A - kOvEps of all of it, MIXED otherwise with the list of atoms that come
// within 1.5 A + kOvEps of it.  A query reads the cell word and, for a MIXED cell, tests
// the listed atoms with the reference's distance (the same norm3 < 1.5 as the sweep).  The
// margins are far above the rounding of the cell index and of the distance, so the answer
// equals the sweep's for every centroid; outside the box no atom is within 1.5 A.
// ----------------------------------------------------------------------------
constexpr double kOvCell = 0.5;   // cell edge (A)
constexpr double kOvEps = 1e-9;   // classification margin (A)
constexpr double kOvBin = 2.0;    // atom bins of the build (A)
constexpr double kOvR = 1.5;      // the reference's overlap distance (A)

__device__ __forceinline__ bool overlap_cells(const DevSystem& S, const double c[3]) {
  const double u0 = (c[0] - S.ov_o[0]) * S.ov_inv_h, u1 = (c[1] - S.ov_o[1]) * S.ov_inv_h,
               u2 = (c[2] - S.ov_o[2]) * S.ov_inv_h;
  // outside the box (or NaN): no atom within 1.5 A
  if (!(u0 >= 0.0 && u0 < (double)S.ov_n[0] && u1 >= 0.0 && u1 < (double)S.ov_n[1] && u2 >= 0.0 &&
        u2 < (double)S.ov_n[2]))
    return false;
  const long cell = ((long)(int)u0 * S.ov_n[1] + (int)u1) * S.ov_n[2] + (int)u2;
  const uint32_t w = __ldg(S.ov_cell + cell);
  if (w == 0u) return false;
  if (w == 0xffffffffu) return true;
  const int off = (int)(w >> 8), cnt = (int)(w & 255u);
  for (int t = 0; t < cnt; ++t) {
    const double4 a = S.rec[__ldg(S.ov_list + off + t)];
    if (norm3(c[0] - a.x, c[1] - a.y, c[2] - a.z) < kOvR) return true;
  }
  return false;
}

struct OvGeom {
  double o[3];   // grid origin (cell and bin lattices share it)
  int n[3];      // cells per axis
  int nb[3];     // bins per axis
};

// Nearest and farthest distance from atom a to cell (i, j, k).
__device__ __forceinline__ void ov_cell_dist(const OvGeom& G, int i, int j, int k, const double4& a, double& dn,
                                             double& df) {
  const int ix[3] = {i, j, k};
  const double x[3] = {a.x, a.y, a.z};
  double n2 = 0, f2 = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lo = G.o[d] + ix[d] * kOvCell, hi = lo + kOvCell;
    const double e = fmax(fmax(lo - x[d], x[d] - hi), 0.0);
    const double f = fmax(fabs(x[d] - lo), fabs(x[d] - hi));
    n2 += e * e;
    f2 += f * f;
  }
  dn = sqrt(n2);
  df = sqrt(f2);
}

// One thread per cell.  Pass 1 (list == NULL): class (0 empty, 1 full, 2 mixed) and the
// number of listed atoms.  Pass 2: the atoms of each mixed cell, in bin order, at the offset
// held in its cell word.
__global__ void ov_cells_kernel(const double4* __restrict__ rec, const int* __restrict__ bin_start,
                                const int* __restrict__ bin_atoms, OvGeom G, uint8_t* __restrict__ cls,
                                int* __restrict__ cnt, const uint32_t* __restrict__ word, int* __restrict__ list) {
  const long n_cells = (long)G.n[0] * G.n[1] * G.n[2];
  for (long cell = (long)blockIdx.x * blockDim.x + threadIdx.x; cell < n_cells; cell += (long)gridDim.x * blockDim.x) {
    const int i = (int)(cell / ((long)G.n[1] * G.n[2])), j = (int)((cell / G.n[2]) % G.n[1]), k = (int)(cell % G.n[2]);
    if (list && (word[cell] == 0u || word[cell] == 0xffffffffu)) continue;
    const int ix[3] = {i, j, k};
    int b0[3], b1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double lo = ix[d] * kOvCell - (kOvR + kOvEps), hi = (ix[d] + 1) * kOvCell + (kOvR + kOvEps);
      b0[d] = max(0, (int)floor(lo / kOvBin));
      b1[d] = min(G.nb[d] - 1, (int)floor(hi / kOvBin));
    }
    bool full = false;
    int m = 0;
    int at = list ? (int)(word[cell] >> 8) : 0;
    for (int bx = b0[0]; bx <= b1[0] && !full; ++bx)
      for (int by = b0[1]; by <= b1[1] && !full; ++by)
        for (int bz = b0[2]; bz <= b1[2] && !full; ++bz) {
          const int b = (bx * G.nb[1] + by) * G.nb[2] + bz;
          for (int t = bin_start[b]; t < bin_start[b + 1]; ++t) {
            const int a = bin_atoms[t];
            double dn, df;
            ov_cell_dist(G, i, j, k, rec[a], dn, df);
            if (!list && df < kOvR - kOvEps) {
              full = true;
              break;
            }
            if (dn < kOvR + kOvEps) {
              if (list) list[at++] = a;
              ++m;
            }
          }
        }
    if (!list) {
      cls[cell] = full ? 1 : (m ? 2 : 0);
      cnt[cell] = full ? 0 : m;
    }
  }
}

__global__ void eval_overlap_kernel(DevSystem S, long long n, const double* __restrict__ cen, int8_t* __restrict__ out) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double c[3] = {cen[3 * t], cen[3 * t + 1], cen[3 * t + 2]};
    out[t] = (int8_t)overlap_any<1>(S, c, 0, 1u);
  }
}

__device__ __forceinline__ double pair_distance(const DevSystem& S, const double c[3], const double R[9], int p) {
  const double* b = S.rx_body[p];
  const double lx = R[0] * b[0] + R[1] * b[1] + R[2] * b[2] + c[0] - S.rx_rec[p][0];
  const double ly = R[3] * b[0] + R[4] * b[1] + R[5] * b[2] + c[1] - S.rx_rec[p][1];
  const double lz = R[6] * b[0] + R[7] * b[1] + R[8] * b[2] + c[2] - S.rx_rec[p][2];
  return norm3(lx, ly, lz);
}

// Terminal flag of state k; k = -1 (an unlabelled state) reads the last entry, as the
// reference's state arrays index.
__device__ __forceinline__ bool sm_terminal(const DevSystem& S, int k) {
  const int i = k < 0 ? k + S.n_states : k;
  return i >= 0 && i < 64 && ((S.terminal >> i) & 1ull);
}

// Distance above the nearest reaction surface reachable from the current state
// (pose c, R), 1e30 if no reaction leaves it (gpu_batch_simulator.py:1018-1033).
__device__ __forceinline__ double sm_rxn_coord(const DevSystem& S, const Traj& tr, const double R[9]) {
  double rc = 1.0e30;
  for (int p = 0; p < S.n_pairs; ++p)
    if (S.rx_before[p] == tr.state) rc = fmin(rc, fmax(pair_distance(S, tr.c, R, p) - S.rx_cut[p], 0.0));
  return rc;
}

// Discrete reaction test and escape/return at the start of a step
// (gpu_batch_simulator.py:818-911).  Returns ST_RUNNING if the trajectory
// goes on to the force evaluation; sets R = R(q) and r = |c| of that pose.
// State-machine mode: the lowest-numbered reaction whose source state is the
// trajectory's and whose pair is within its cutoff fires; the trajectory moves
// to the reaction's destination state and has reacted if that state is terminal.
// A trajectory that fired skips the escape test of this step (:880).
__device__ __forceinline__ int step_begin(const DevSystem& S, const DevSim& P, const Keyed& key, uint32_t s, Traj& tr,
                                          double R[9], double& r, Tally& tl) {
  quat_to_rot(tr.q, R);
  bool fired = false;
  if (S.sm) {
    for (int p = 0; p < S.n_pairs; ++p)
      if (S.rx_before[p] == tr.state && pair_distance(S, tr.c, R, p) < S.rx_cut[p]) {
        tr.state = S.rx_after[p];
        atomicAdd(P.ctr + C_SM_DISCRETE + p, 1ull);
        if (sm_terminal(S, tr.state)) return ST_REACTED;
        fired = true;
        break;
      }
  } else if (S.n_pairs > 0) {
    int nsat = 0;
    for (int p = 0; p < S.n_pairs; ++p) nsat += pair_distance(S, tr.c, R, p) < S.rx_cut[p];
    if (nsat >= S.n_needed) return ST_REACTED;
  }
  r = norm3(tr.c[0], tr.c[1], tr.c[2]);
  if (r >= P.r_esc && !fired) {
    const W4 w = key.w(s, SUB_ESCAPE);
    if (u53(w.a, w.b) < P.return_prob) {
      tr.c[0] = tr.c[0] / r * P.r_b;
      tr.c[1] = tr.c[1] / r * P.r_b;
      tr.c[2] = tr.c[2] / r * P.r_b;
      const W4 qa = key.w(s, SUB_RETURN_Q), qb = key.w(s, SUB_RETURN_Q + 1);
      shoemake(u53(qa.a, qa.b), u53(qa.c, qa.d), u53(qb.a, qb.b), tr.q);
      quat_to_rot(tr.q, R);
      tr.rets += 1;
      tl.returns += 1;
      r = norm3(tr.c[0], tr.c[1], tr.c[2]);
    } else {
      return ST_ESCAPED;
    }
  }
  return ST_RUNNING;
}

// Adaptive dt, D(r), Ermak-McCammon translation and the body-frame rotation
// (gpu_batch_simulator.py:961-1101).  Writes the proposed pose; false if it is not finite.
template <typename FT>
__device__ __forceinline__ bool step_move(const DevSystem& S, const DevSim& P, const Keyed& key, uint32_t s,
                                          const Traj& tr, const double R[9], double r, const double F[3],
                                          const double T[3], double cn[3], double qn[4], double& dt) {
  dt = adaptive_dt(P, r, S.sm ? sm_rxn_coord(S, tr, R) : -1.0);
  const double D = hi_diffusion<FT>(P, r);
  double xt[3], xr[3];
  {
    const W4 a = key.w(s, SUB_NORMALS), b = key.w(s, SUB_NORMALS + 1), c = key.w(s, SUB_NORMALS + 2);
    box_muller(u53(a.a, a.b), u53(a.c, a.d), xt[0], xt[1]);
    box_muller(u53(b.a, b.b), u53(b.c, b.d), xt[2], xr[0]);
    box_muller(u53(c.a, c.b), u53(c.c, c.d), xr[1], xr[2]);
  }
  const double sig_t = sqrt(2.0 * D * dt), ddt = D * dt;
#pragma unroll
  for (int k = 0; k < 3; ++k) cn[k] = tr.c[k] + (ddt * F[k] + sig_t * xt[k]);
#pragma unroll
  for (int k = 0; k < 4; ++k) qn[k] = tr.q[k];
  const double sig_r = sqrt(2.0 * P.D_r * dt), rdt = P.D_r * dt;
  rotate_quat(qn, rdt * T[0] + sig_r * xr[0], rdt * T[1] + sig_r * xr[1], rdt * T[2] + sig_r * xr[2]);
  return isfinite(cn[0]) && isfinite(cn[1]) && isfinite(cn[2]) && isfinite(qn[0]);
}

// Overlap outcome, Brownian bridge, step count (gpu_batch_simulator.py:1102-1254).
// R is the rotation at the old pose tr.c; the pose moves to (cn, qn) if `moved`.
__device__ __forceinline__ int step_end(const DevSystem& S, const DevSim& P, const Keyed& key, uint32_t s, Traj& tr,
                                        const double R[9], const double cn[3], const double qn[4], bool moved,
                                        double dt, Tally& tl) {
  const double c0[3] = {tr.c[0], tr.c[1], tr.c[2]};
  if (moved) {
    tr.c[0] = cn[0];
    tr.c[1] = cn[1];
    tr.c[2] = cn[2];
    tr.q[0] = qn[0];
    tr.q[1] = qn[1];
    tr.q[2] = qn[2];
    tr.q[3] = qn[3];
  } else {
    tl.overlap += 1;
  }
  int st = ST_RUNNING;
  if (S.n_pairs > 0) {
    double Rn[9];
    if (moved) {
      quat_to_rot(tr.q, Rn);
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) Rn[k] = R[k];
    }
    int fired = 0, first = -1;
    for (int p = 0; p < S.n_pairs; ++p) {
      const double d0 = pair_distance(S, c0, R, p), d1 = pair_distance(S, tr.c, Rn, p);
      const double x0 = d0 - S.rx_cut[p], x1 = d1 - S.rx_cut[p];
      double pc = 0.0;
      if (x0 > 0 && x1 > 0) pc = exp(-x0 * x1 / fmax(S.rx_deff[p] * dt, 1e-30));
      const W4 w = key.w(s, SUB_BRIDGE + (uint32_t)(p >> 1));
      const double u = (p & 1) ? u53(w.c, w.d) : u53(w.a, w.b);
      const bool f = (u < pc) || (d1 < S.rx_cut[p]);
      fired += f;
      if (f && first < 0 && S.rx_before[p] == tr.state) first = p;
    }
    if (S.sm) {
      // the lowest-numbered reaction from the current state whose pair fired (:1185-1234)
      if (first >= 0) {
        tr.state = S.rx_after[first];
        atomicAdd(P.ctr + C_SM_BRIDGE + first, 1ull);
        if (sm_terminal(S, tr.state)) {
          st = ST_REACTED;
          tl.bridge += 1;
        }
      }
    } else if (fired >= S.n_needed) {
      st = ST_REACTED;
      tl.bridge += 1;
    }
  }
  tr.steps += 1;
  tl.steps += 1;
  if (st == ST_RUNNING && tr.steps >= P.max_steps) st = ST_MAXSTEPS;
  return st;
}

// numpy.searchsorted(edges, x) - 1 (side "left"), clipped to [0, n-1]; edges has n+1 entries.
__device__ __forceinline__ int hist_bin(const double* e, int n, double x) {
  int lo = 0, hi = n + 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (e[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  const int b = lo - 1;
  return b < 0 ? 0 : (b > n - 1 ? n - 1 : b);
}

// Statistics of one completed step (gpu_batch_simulator.py:1255-1317): closest
// approach, accumulated time, radial / angular / transition histograms,
// milestone crossings between r_prev (end of the previous step) and now, and
// pair contacts at the force-evaluation pose (c0, R).  `sh` is the block's
// shared-memory histogram (SH_* layout).
__device__ __forceinline__ void stats_step(const DevSystem& S, const DevSim& P, const Traj& tr, uint32_t s,
                                           double r_prev, double dt, const double c0[3], const double R[9],
                                           unsigned* sh) {
  const DevStats& st = P.st;
  const int id = tr.id;
  const double cur = norm3(tr.c[0], tr.c[1], tr.c[2]);
  if (cur < st.min_dist[id]) {
    st.min_dist[id] = cur;
    st.step_at_min[id] = (int)s;
#pragma unroll
    for (int k = 0; k < 3; ++k) st.nm_c[3 * id + k] = tr.c[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) st.nm_q[4 * id + k] = tr.q[k];
  }
  st.total_time[id] += dt;
  atomicAdd(sh + SH_RAD + hist_bin(st.rad_edges, ST_RAD_BINS, cur), 1u);
  const double PI = 3.14159265358979323846;
  const double rs = fmax(cur, 1e-30);
  const double th = acos(fmin(fmax(tr.c[2] / rs, -1.0), 1.0));
  const double ph = atan2(tr.c[1], tr.c[0]) + PI;
  int ti = (int)(th / PI * ST_THETA), pi = (int)(ph / (2 * PI) * ST_PHI);
  ti = ti < 0 ? 0 : (ti > ST_THETA - 1 ? ST_THETA - 1 : ti);
  pi = pi < 0 ? 0 : (pi > ST_PHI - 1 ? ST_PHI - 1 : pi);
  atomicAdd(sh + SH_ANG + ti * ST_PHI + pi, 1u);
  for (int m = 0; m < ST_MILESTONES; ++m) {
    const double mr = st.ms_radii[m];
    if (r_prev < mr && cur >= mr) atomicAdd(sh + SH_MS_OUT + m, 1u);
    if (r_prev >= mr && cur < mr) atomicAdd(sh + SH_MS_IN + m, 1u);
  }
  atomicAdd(sh + SH_TRANS + hist_bin(st.trans_edges, ST_TRANS, r_prev) * ST_TRANS +
                hist_bin(st.trans_edges, ST_TRANS, cur),
            1u);
  for (int p = 0; p < S.n_pairs; ++p)
    if (pair_distance(S, c0, R, p) < S.rx_cut[p]) atomicAdd(sh + SH_CONTACT + p, 1u);
}

// Path and energy rows of one completed step s (gpu_batch_simulator.py:1319-1340):
// [id, s, x, y, z, q0, q1, q2] after the step and [id, s, fx, fy, fz, dt] of the step.
__device__ __forceinline__ void trace_step(const DevSim& P, const Traj& tr, uint32_t s, const double F[3],
                                           double dt) {
  if (P.trace_cap <= 0 || (s % (uint32_t)P.save_interval) != 0u) return;
  const unsigned long long i = atomicAdd(P.ctr + C_TRACE, 1ull);
  if (i >= (unsigned long long)P.trace_cap) return;
  double* p = P.trace_path + 8 * i;
  p[0] = (double)tr.id;
  p[1] = (double)s;
  p[2] = tr.c[0];
  p[3] = tr.c[1];
  p[4] = tr.c[2];
  p[5] = tr.q[0];
  p[6] = tr.q[1];
  p[7] = tr.q[2];
  double* e = P.trace_energy + 6 * i;
  e[0] = (double)tr.id;
  e[1] = (double)s;
  e[2] = F[0];
  e[3] = F[1];
  e[4] = F[2];
  e[5] = dt;
}

// Pose at reaction; `bridge` marks a reaction found by the Brownian bridge.
__device__ __forceinline__ void stats_encounter(const DevSim& P, const Traj& tr, uint32_t s, bool bridge) {
  const DevStats& st = P.st;
#pragma unroll
  for (int k = 0; k < 3; ++k) st.enc_c[3 * tr.id + k] = tr.c[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) st.enc_q[4 * tr.id + k] = tr.q[k];
  st.enc_step[tr.id] = (int)s;
  st.bridge[tr.id] = bridge ? 1 : 0;
}

__device__ __forceinline__ void stats_block_begin(const DevSim& P, unsigned* sh) {
  if (!P.stats) return;
  for (int i = threadIdx.x; i < SH_NUM; i += blockDim.x) sh[i] = 0u;
  __syncthreads();
}

// Dynamic shared memory of a stepper block, in this order: the FP32 receptor
// atoms (n_rec_pad float4) and chunk spheres (n_chunks float4) when
// S.rec_in_smem, then the statistics histograms (SH_NUM words) when P.stats.
// The host sizes every stepper launch for exactly this layout.
struct BlockShared {
  RecView v;
  unsigned* stats;
};

__device__ __forceinline__ BlockShared block_shared_begin(const DevSystem& S, const DevSim& P) {
  extern __shared__ float4 sh_dyn[];
  BlockShared b{RecView{nullptr, nullptr}, reinterpret_cast<unsigned*>(sh_dyn)};
  if (S.rec_in_smem) {
    const int nr = S.n_rec_pad, n = nr + S.n_chunks;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sh_dyn[i] = i < nr ? S.rec_f[i] : S.chunks_f[i - nr];
    b.v = RecView{sh_dyn, sh_dyn + nr};
    b.stats = reinterpret_cast<unsigned*>(sh_dyn + n);
    __syncthreads();
  }
  stats_block_begin(P, b.stats);
  return b;
}

__device__ __forceinline__ void stats_block_end(const DevSim& P, const unsigned* sh) {
  if (!P.stats) return;
  __syncthreads();
  for (int i = threadIdx.x; i < SH_NUM; i += blockDim.x)
    if (sh[i]) atomicAdd(P.st.hist + i, (unsigned long long)sh[i]);
}

// One BD step of one trajectory by the G lanes of its group, in the
// reference's order (gpu_batch_simulator.py:783-1254): discrete reaction test,
// escape/return, forces, adaptive dt, D(r), translation, rotation, overlap
// rejection, Brownian bridge, step count.  Returns the new status.
template <typename FT, int G, bool TORQUE>
__device__ __forceinline__ int bd_step(const DevSystem& S, const DevSim& P, Traj& tr, int lane, unsigned gm,
                                       Tally& tl, unsigned* sh, const RecView& v) {
  const Keyed key = traj_key(P, tr.id);
  const uint32_t s = (uint32_t)tr.steps;
  const double r_prev = P.stats ? norm3(tr.c[0], tr.c[1], tr.c[2]) : 0.0;
  double R[9], r;
  const int st0 = step_begin(S, P, key, s, tr, R, r, tl);
  if (st0 != ST_RUNNING) {
    if (P.stats && st0 == ST_REACTED && lane == 0) stats_encounter(P, tr, s, false);
    return st0;
  }
  double F[3], T[3], E;
  group_forces<FT, G, TORQUE, false>(S, tr.c, R, lane, gm, PosFromPose{R, tr.c}, F, T, E, tl.cnt, v);
  double cn[3], qn[4], dt;
  if (!step_move<FT>(S, P, key, s, tr, R, r, F, T, cn, qn, dt)) {
    tl.nonfinite += 1;
    return ST_ERROR;
  }
  const bool moved = !(P.overlap && overlap_any<G>(S, cn, lane, gm, v));
  const double c0[3] = {tr.c[0], tr.c[1], tr.c[2]};
  const int st = step_end(S, P, key, s, tr, R, cn, qn, moved, dt, tl);
  if (P.stats && lane == 0) {
    stats_step(S, P, tr, s, r_prev, dt, c0, R, sh);
    trace_step(P, tr, s, F, dt);
    if (st == ST_REACTED) stats_encounter(P, tr, s, true);
  }
  return st;
}

__device__ __forceinline__ void load_slot(const SlotBuf& B, int s, Traj& tr) {
  tr.c[0] = B.c[s];
  tr.c[1] = B.c[B.cap + s];
  tr.c[2] = B.c[2 * B.cap + s];
#pragma unroll
  for (int k = 0; k < 4; ++k) tr.q[k] = B.q[k * B.cap + s];
  tr.id = B.traj[s];
  tr.steps = B.steps[s];
  tr.rets = B.rets[s];
  tr.status = B.status[s];
  tr.state = B.state[s];
}

__device__ __forceinline__ void store_slot(const SlotBuf& B, int s, const Traj& tr) {
  B.c[s] = tr.c[0];
  B.c[B.cap + s] = tr.c[1];
  B.c[2 * B.cap + s] = tr.c[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) B.q[k * B.cap + s] = tr.q[k];
  B.traj[s] = tr.id;
  B.steps[s] = tr.steps;
  B.rets[s] = tr.rets;
  B.status[s] = (int8_t)tr.status;
  B.state[s] = (int8_t)tr.state;
}

template <int G>
__device__ __forceinline__ int group_fetch(unsigned long long* p, int lane, unsigned gm) {
  unsigned long long v = 0;
  if (lane == 0) v = atomicAdd(p, 1ull);
  v = __shfl_sync(gm, v, 0, G);
  return v > 0x7fffffffull ? 0x7fffffff : (int)v;
}

// Window copy of a grid (DevGrid::win): entry n holds nodes n .. n + 4/ch - 1 of
// node n's z row, all `ch` channels of each, zero past the end of the row.
__global__ void window_kernel(const float* __restrict__ d, float4* __restrict__ w, long n_nodes, int nz, int ch) {
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < n_nodes; n += (long)gridDim.x * blockDim.x) {
    const int z = (int)(n % nz);
    float v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int node = k / ch, c = k % ch;
      v[k] = z + node < nz ? d[(n + node) * ch + c] : 0.f;
    }
    w[n] = make_float4(v[0], v[1], v[2], v[3]);
  }
}

// Cube copy of a one-channel grid (DevGrid::cube): entry n = (x, y, z) holds the 2x2x2 block
// v(x + i, y + j, z + k) at 4i + 2j + k, zero past the grid's faces.
__global__ void cube_kernel(const float* __restrict__ d, float* __restrict__ cube, int nx, int ny, int nz) {
  const long n_nodes = (long)nx * ny * nz;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < n_nodes; n += (long)gridDim.x * blockDim.x) {
    const int z = (int)(n % nz), y = (int)((n / nz) % ny), x = (int)(n / ((long)ny * nz));
    float v[8];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k)
          v[4 * i + 2 * j + k] =
              (x + i < nx && y + j < ny && z + k < nz) ? d[((long)(x + i) * ny + (y + j)) * nz + (z + k)] : 0.f;
    float4* o = reinterpret_cast<float4*>(cube + 8 * n);
    o[0] = make_float4(v[0], v[1], v[2], v[3]);
    o[1] = make_float4(v[4], v[5], v[6], v[7]);
  }
}

// The xy records of a one-channel grid (DevGrid::xy): per node, for each cell half in x and y,
// the extra x plane's four nodes and the extra y row's four nodes of the stencil (nodes off the
// grid read as 0; stencils never reach them, every stencil position lies in the margin box).
__global__ void xy_kernel(const float* __restrict__ d, float* __restrict__ xy, int nx, int ny, int nz) {
  const long n_nodes = (long)nx * ny * nz;
  auto at = [&](int x, int y, int z) -> float {
    return (x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz) ? d[((long)x * ny + y) * nz + z] : 0.f;
  };
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < n_nodes; n += (long)gridDim.x * blockDim.x) {
    const int z = (int)(n % nz), y = (int)((n / nz) % ny), x = (int)(n / ((long)ny * nz));
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int ex = a ? x + 2 : x - 1, ey = b ? y + 2 : y - 1;
        float v[8];
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            v[2 * j + k] = at(ex, y + j, z + k);
            v[4 + 2 * j + k] = at(x + j, ey, z + k);
          }
        float4* o = reinterpret_cast<float4*>(xy + 8 * (4 * n + 2 * a + b));
        o[0] = make_float4(v[0], v[1], v[2], v[3]);
        o[1] = make_float4(v[4], v[5], v[6], v[7]);
      }
  }
}

// z-edge records of a one-channel grid (DevGrid::ztex); nodes off the grid read as 0.
__global__ void zedge_kernel(const float* __restrict__ d, float4* __restrict__ out, int nx, int ny, int nz) {
  const long n_nodes = (long)nx * ny * nz;
  auto at = [&](int x, int y, int z) -> float {
    return (x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz) ? d[((long)x * ny + y) * nz + z] : 0.f;
  };
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < n_nodes; n += (long)gridDim.x * blockDim.x) {
    const int z = (int)(n % nz), y = (int)((n / nz) % ny), x = (int)(n / ((long)ny * nz));
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int ez = c ? z + 2 : z - 1;
      out[2 * n + c] = make_float4(at(x, y, ez), at(x, y + 1, ez), at(x + 1, y, ez), at(x + 1, y + 1, ez));
    }
  }
}

// D(r) of the stepper at n distances (parity entry point bd_sim_hi_diffusion).
template <typename FT>
__global__ void hi_diffusion_kernel(DevSim P, int n, const double* __restrict__ r, double* __restrict__ D) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) D[i] = hi_diffusion<FT>(P, r[i]);
}

// Fill `n_slots` slots with the first trajectories of the pending pool.
__global__ void init_slots_kernel(DevSim P, SlotBuf B, int n_slots) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  Traj tr;
  start_trajectory(P, s, tr);
  store_slot(B, s, tr);
}

// Persistent stepper: groups take live slots from a dynamic cursor, advance
// each by K steps with its state in registers, start a pending trajectory
// whenever theirs ends, and write the slot back.  Slots whose trajectory ended
// with the pool empty are left EMPTY for the compaction.
template <typename FT, int G, bool TORQUE>
__global__ void __launch_bounds__(256) step_kernel(DevSystem S, DevSim P, SlotBuf B, const int* __restrict__ n_live,
                                                   int K) {
  const BlockShared sh = block_shared_begin(S, P);
  const int lane = threadIdx.x & (G - 1);
  const unsigned gm = group_mask<G>();
  const int live = *n_live;
  Tally tl{};
  for (;;) {
    const int slot = group_fetch<G>(P.ctr + C_SLOT_CURSOR, lane, gm);
    if (slot >= live) break;
    Traj tr;
    load_slot(B, slot, tr);
    // A slot always leaves a launch RUNNING or EMPTY: an ended trajectory is
    // replaced right away, even after the launch's last step, so the compaction
    // only ever drops slots whose replacement found the pool empty.
    for (int k = 0; k < K && tr.status != ST_EMPTY; ++k) {
      if (tr.status != ST_RUNNING) {
        const int id = group_fetch<G>(P.ctr + C_PENDING, lane, gm);
        if (id >= P.n_traj) {
          tr.status = ST_EMPTY;
          break;
        }
        start_trajectory(P, id, tr);
      }
      const int st = bd_step<FT, G, TORQUE>(S, P, tr, lane, gm, tl, sh.stats, sh.v);
      if (st != ST_RUNNING) {
        tr.status = st;
        if (lane == 0) {
          P.out_status[tr.id] = (int8_t)st;
          P.out_steps[tr.id] = tr.steps;
          P.out_returns[tr.id] = tr.rets;
        }
        tl.reacted += st == ST_REACTED;
        tl.escaped += st == ST_ESCAPED;
        tl.maxsteps += st == ST_MAXSTEPS;
        const int id = group_fetch<G>(P.ctr + C_PENDING, lane, gm);
        if (id >= P.n_traj) {
          tr.status = ST_EMPTY;
        } else {
          start_trajectory(P, id, tr);
        }
      }
    }
    if (lane == 0) store_slot(B, slot, tr);
  }
  // Only lane 0 of each group counts scalar events.
  flush_tally(P, tl, lane == 0);
  stats_block_end(P, sh.stats);
}

// All forces of the lanes with `need`, one trajectory at a time, the whole warp
// sweeping that trajectory's ligand atoms and receptor chunks.
template <typename FT, bool TORQUE>
__device__ __forceinline__ void warp_forces(const DevSystem& S, const double c[3], const double R[9], bool need,
                                            double F[3], double T[3], int lane, Counts& cnt, const RecView& v) {
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
    group_forces<FT, 32, TORQUE, false>(S, cj, Rj, lane, FULL, PosFromPose{Rj, cj}, f, t, e, cnt, v);
    if (lane == j) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        F[k] = f[k];
        T[k] = t[k];
      }
    }
  }
}

// Overlap test of every lane with `need`, the warp sweeping the receptor chunks together.
__device__ __forceinline__ bool warp_overlap(const DevSystem& S, const double cn[3], bool need, int lane,
                                             const RecView& v) {
  // with the occupancy grid every lane answers for its own centroid
  if (S.ov_cell) return need && overlap_cells(S, cn);
  const unsigned FULL = 0xffffffffu;
  unsigned m = __ballot_sync(FULL, need);
  bool mine = false;
  while (m) {
    const int j = __ffs(m) - 1;
    m &= m - 1;
    double cj[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cj[k] = __shfl_sync(FULL, cn[k], j);
    const bool hit = overlap_any<32>(S, cj, lane, FULL, v);
    if (lane == j) mine = hit;
  }
  return mine;
}

// Lanes whose trajectory ended (and that are not out of work) take the next
// pending ids, one atomic per warp; a lane that finds the pool empty goes EMPTY.
__device__ __forceinline__ void warp_refill(const DevSim& P, Traj& tr, bool& dead, int lane) {
  const unsigned FULL = 0xffffffffu;
  const bool want = !dead && tr.status != ST_RUNNING;
  const unsigned wm = __ballot_sync(FULL, want);
  if (!wm) return;
  const int leader = __ffs(wm) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(P.ctr + C_PENDING, (unsigned long long)__popc(wm));
  base = __shfl_sync(FULL, base, leader);
  if (want) {
    const unsigned long long id = base + __popc(wm & ((1u << lane) - 1u));
    if (id >= (unsigned long long)P.n_traj) {
      tr.status = ST_EMPTY;
      dead = true;
    } else {
      start_trajectory(P, (int)id, tr);
    }
  }
}

// Warp-cooperative persistent stepper.  Each lane owns one live slot and does
// that trajectory's per-step scalar work (reaction test, escape/return, dt,
// noise, pose update, bridge) with no redundancy; the warp then sweeps the
// force and overlap loops one trajectory at a time, so those loops run with
// all 32 lanes on the same trajectory instead of diverging groups.
// MINB = minimum resident 256-thread blocks per SM requested from the register
// allocator (1: no cap; 2: at most 128 registers per thread).
template <typename FT, bool TORQUE, int MINB>
__global__ void __launch_bounds__(256, MINB) step_kernel_warp(DevSystem S, DevSim P, SlotBuf B,
                                                              const int* __restrict__ n_live, int K) {
  const BlockShared sh = block_shared_begin(S, P);
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int live = *n_live;
  Tally tl{};
  for (;;) {
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(P.ctr + C_SLOT_CURSOR, 32ull);
    b = __shfl_sync(FULL, b, 0);
    if (b >= (unsigned long long)live) break;
    const int slot = (int)b + lane;
    const bool own = slot < live;
    Traj tr{};
    tr.status = ST_EMPTY;
    if (own) load_slot(B, slot, tr);
    bool dead = !own;
    // F, T hold the forces at the lane's current pose while `fresh`: a step that the
    // overlap test rejected leaves the pose, and so the forces, unchanged, and the next
    // step reuses them instead of evaluating the same pose again
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    bool fresh = false;
    for (int k = 0; k < K; ++k) {
      warp_refill(P, tr, dead, lane);
      if (__all_sync(FULL, dead)) break;
      const Keyed key = traj_key(P, tr.id);
      const uint32_t s = (uint32_t)tr.steps;
      double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, r = 0;
      const double r_prev = P.stats ? norm3(tr.c[0], tr.c[1], tr.c[2]) : 0.0;
      int st = ST_EMPTY;
      if (!dead) {
        const int rets0 = tr.rets;
        st = step_begin(S, P, key, s, tr, R, r, tl);
        if (tr.rets != rets0) fresh = false;  // returned to the b-sphere: a new pose
        if (P.stats && st == ST_REACTED) stats_encounter(P, tr, s, false);
      }
      const bool need_f = !dead && st == ST_RUNNING;
      warp_forces<FT, TORQUE>(S, tr.c, R, need_f && !fresh, F, T, lane, tl.cnt, sh.v);
      double cn[3] = {0, 0, 0}, qn[4] = {1, 0, 0, 0}, dt = 0;
      bool ok = true;
      if (need_f) ok = step_move<FT>(S, P, key, s, tr, R, r, F, T, cn, qn, dt);
      if (need_f && !ok) {
        tl.nonfinite += 1;
        st = ST_ERROR;
      }
      const bool ovl = warp_overlap(S, cn, need_f && ok && P.overlap, lane, sh.v);
      fresh = need_f && ok && ovl;
      if (need_f && ok) {
        const double c0[3] = {tr.c[0], tr.c[1], tr.c[2]};
        st = step_end(S, P, key, s, tr, R, cn, qn, !ovl, dt, tl);
        if (P.stats) {
          stats_step(S, P, tr, s, r_prev, dt, c0, R, sh.stats);
          trace_step(P, tr, s, F, dt);
          if (st == ST_REACTED) stats_encounter(P, tr, s, true);
        }
      }
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
    // a slot leaves the launch RUNNING or EMPTY (ended trajectories are replaced now)
    warp_refill(P, tr, dead, lane);
    if (own) store_slot(B, slot, tr);
  }
  flush_tally(P, tl, true);
  stats_block_end(P, sh.stats);
}

// Sum the per-thread tallies of a warp and add them to the device counters.
// Threads that do not own scalar events pass owner = false.
__device__ __forceinline__ void flush_tally(const DevSim& P, Tally tl, bool owner) {
  if (!owner) {
    tl.steps = 0;
    tl.reacted = tl.escaped = tl.maxsteps = tl.returns = tl.overlap = tl.bridge = tl.nonfinite = 0;
  }
  __syncwarp();
  const unsigned long long st64 = [&] {
    unsigned long long v = tl.steps;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }();
  const unsigned vals[10] = {tl.reacted, tl.escaped, tl.maxsteps, tl.returns, tl.overlap, tl.bridge,
                             tl.nonfinite, tl.cnt.grid, tl.cnt.rev, tl.cnt.ff};
  unsigned red[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) red[i] = gsumu<32>(vals[i], 0xffffffffu);
  if ((threadIdx.x & 31) == 0) {
    const int idx[10] = {C_REACTED, C_ESCAPED, C_MAXSTEPS, C_RETURNS, C_OVERLAP, C_BRIDGE, C_NONFINITE,
                         C_GRID_EVALS, C_REV_EVALS, C_FF_EVALS};
    if (st64) atomicAdd(P.ctr + C_STEPS, st64);
#pragma unroll
    for (int i = 0; i < 10; ++i)
      if (red[i]) atomicAdd(P.ctr + idx[i], (unsigned long long)red[i]);
  }
}

// Move live slots of `src` (status RUNNING) densely into `dst`; the order is
// irrelevant because every draw is keyed by trajectory id and step.
__global__ void compact_kernel(SlotBuf src, SlotBuf dst, const int* __restrict__ n_live_src,
                               unsigned long long* ctr) {
  const int n = *n_live_src;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const bool alive = src.status[s] == ST_RUNNING;
    const unsigned m = __ballot_sync(__activemask(), alive);
    if (!alive) continue;
    const int leader = __ffs(m) - 1;
    const int lane = threadIdx.x & 31;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(ctr + C_LIVE_NEXT, (unsigned long long)__popc(m));
    base = __shfl_sync(m, base, leader);
    const int d = (int)base + __popc(m & ((1u << lane) - 1u));
    Traj tr;
    load_slot(src, s, tr);
    store_slot(dst, d, tr);
  }
}

// Publish the compacted count and reset the cursors for the next launch.
__global__ void finish_compact_kernel(int* n_live_dst, unsigned long long* ctr) {
  *n_live_dst = (int)ctr[C_LIVE_NEXT];
  ctr[C_LIVE_NEXT] = 0;
  ctr[C_SLOT_CURSOR] = 0;
}

}  // namespace bd
