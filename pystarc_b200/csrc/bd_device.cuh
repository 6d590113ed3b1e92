// Device-side building blocks of the batched rigid-body BD engine (sm_100a).
//
// Conventions follow the reference's batched stepper and force engine:
//   quaternions (w,x,y,z), R(q) as pystarc/simulation/gpu_batch_simulator.py:1611-1629,
//   q <- normalize(q (x) dq(omega)) as :1631-1660,
//   grids C-ordered (nx,ny,nz), z fastest, index i*ny*nz + j*nz + k
//   (pystarc/forces/electrostatic/grid_force.py:144), strict in-grid box
//   [origin + 3 sp, origin + (n-4) sp] (pystarc/forces/gpu_batch_engine.py:268-273).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define BD_MAX_ELEC 4
#define BD_MAX_PAIRS 16
#define BD_CHUNK 32

namespace bd {

enum : int { ST_RUNNING = 0, ST_REACTED = 1, ST_ESCAPED = 2, ST_MAXSTEPS = 3, ST_EMPTY = 4, ST_ERROR = 5 };

// Tally slots (unsigned long long counters on the device).
enum : int {
  C_PENDING = 0,    // next trajectory id to start (the pending pool cursor)
  C_REACTED,
  C_ESCAPED,
  C_MAXSTEPS,
  C_STEPS,          // trajectory-steps (reference total_steps)
  C_RETURNS,        // escape -> return events
  C_OVERLAP,        // overlap rejections
  C_BRIDGE,         // reactions found by the Brownian bridge
  C_GRID_EVALS,     // (atom, grid) stencil evaluations, forward direction
  C_REV_EVALS,      // receptor-atom stencil evaluations, reverse Born
  C_FF_EVALS,       // far-field atom evaluations
  C_NONFINITE,      // steps that produced a non-finite pose (trajectory stopped)
  C_SLOT_CURSOR,    // dynamic slot cursor of the current launch
  C_LIVE_NEXT,      // live-slot count being built by the compaction
  C_TRACE,          // path/energy trace rows claimed (may exceed the capacity)
  C_SM_DISCRETE,    // BD_MAX_PAIRS counters: state-machine reactions fired by the discrete test
  C_SM_BRIDGE = C_SM_DISCRETE + BD_MAX_PAIRS,  // BD_MAX_PAIRS counters: fired by the Brownian bridge
  C_NUM = C_SM_BRIDGE + BD_MAX_PAIRS
};

struct DevGrid {
  const float* data;  // FP32 values; `ch` interleaved channels per node
  const float4* win;  // optional: entry n = nodes n .. n + 4/ch - 1 of node n's z row, all channels
  const float* cube;  // optional (ch = 1): 8 floats per node n = (x, y, z), the 2x2x2 block
                      // v(x + i, y + j, z + k) at 4i + 2j + k, 32-byte aligned (one sector)
  const float* xy;    // optional (with cube): per node n = (x, y, z), four 8-float records, record
                      // 2a + b for the extra x plane ex = (a ? x + 2 : x - 1) and the extra y row
                      // ey = (b ? y + 2 : y - 1): v(ex, y + j, z + k) at 2j + k, v(x + i, ey, z + k)
                      // at 4 + 2i + k
  cudaTextureObject_t xytex;  // optional: a float4 texture view of xy (record r = elements 2r, 2r + 1)
  cudaTextureObject_t ptex;   // optional (ch = 2): a float2 texture view of data (element = node)
  cudaTextureObject_t ztex;  // optional (with cube): per node n = (x, y, z), two float4 records
                             // read through the texture path, record 2n + c for the extra z node
                             // ez = (c ? z + 2 : z - 1): v(x, y, ez), v(x, y + 1, ez),
                             // v(x + 1, y, ez), v(x + 1, y + 1, ez)
  int nx, ny, nz, ch;
  double ox, oy, oz;
  double isx, isy, isz;  // 1/spacing
  double lox, loy, loz, hix, hiy, hiz;  // strict margin box
  float oxf, oyf, ozf, isxf, isyf, iszf;  // FP32 origin and 1/spacing (the FP32-position stencil)
};

struct DevSystem {
  // ligand (body frame = about the ligand centroid)
  int n_lig;
  const double4* lig;  // x,y,z,q (FP64)
  // receptor atoms in spatial chunks of BD_CHUNK (padded with copies of the last atom, q = 0)
  int n_rec_pad, n_chunks;
  const double4* rec;     // x,y,z,q
  const double4* chunks;  // centre xyz, radius
  const float4* rec_f;    // FP32 copies for the shared-memory pre-tests (radius not inflated)
  const float4* chunks_f;
  int rec_in_smem;        // stepper kernels stage rec_f / chunks_f in shared memory
  unsigned terms;         // BD_TERM_* summed by the evaluation kernels (the stepper sums all)
  double rec_max_r;
  // overlap occupancy grid (BD_LAYOUT_OVERLAP_GRID; ov_cell = NULL: not built).  Cell words:
  // 0 no receptor atom within 1.5 A of any point of the cell, 0xffffffff every point within
  // 1.5 A of some atom, else (offset << 8 | count): the atoms (indices into rec) that may be
  const uint32_t* ov_cell;
  const int* ov_list;
  double ov_o[3], ov_inv_h;
  int ov_n[3];
  // grids
  int n_elec;
  DevGrid elec[BD_MAX_ELEC];
  int has_born;
  DevGrid born;
  int paired;        // elec[0] and born share a lattice; `pair` holds both (ch = 2)
  DevGrid pair;
  int born_rev;      // reverse Born active
  DevGrid lig_born;
  double lig_born_rho;  // circumradius of the ligand Born box about the ligand origin
  // far field (receptor at the origin)
  int has_yukawa, use_dip, use_quad;
  double V_factor, inv_debye, inv_fpe;
  double dip[3], quad[9];
  double alpha;
  // WCA contact term (wca = 0: off): epsilon, centroid activation radius, largest pair cutoff
  int wca;
  double wca_eps, wca_act, wca_cut;
  const double* rec_rad;  // n_rec_pad, receptor table order (padding -1e300: never within a cutoff)
  const double* lig_rad;  // n_lig
  // reaction pairs (flattened)
  int n_pairs, n_needed;
  double rx_rec[BD_MAX_PAIRS][3];
  double rx_body[BD_MAX_PAIRS][3];
  double rx_cut[BD_MAX_PAIRS];
  double rx_deff[BD_MAX_PAIRS];
  // state-machine reactions (sm = 1): reaction p is pair p and fires only from state rx_before[p]
  int sm, n_states;
  int rx_before[BD_MAX_PAIRS], rx_after[BD_MAX_PAIRS];
  unsigned long long terminal;  // bit k: state k has no reaction leaving it
};

// Per-step statistics of the reference's stepper (gpu_batch_simulator.py:577-620,
// :1255-1317), kept on the device.  Histogram sizes are the reference's.
enum : int { ST_RAD_BINS = 200, ST_THETA = 36, ST_PHI = 72, ST_MILESTONES = 11, ST_TRANS = 50 };
enum : int {
  SH_RAD = 0,
  SH_ANG = SH_RAD + ST_RAD_BINS,
  SH_MS_OUT = SH_ANG + ST_THETA * ST_PHI,
  SH_MS_IN = SH_MS_OUT + ST_MILESTONES,
  SH_TRANS = SH_MS_IN + ST_MILESTONES,
  SH_CONTACT = SH_TRANS + ST_TRANS * ST_TRANS,
  SH_NUM = SH_CONTACT + BD_MAX_PAIRS
};

struct DevStats {
  // per trajectory (local id)
  double* start_c;   // 3n
  double* start_q;   // 4n
  double* min_dist;  // n (initialised to 1e30)
  int* step_at_min;  // n
  double* nm_c;      // 3n, pose at the closest approach
  double* nm_q;      // 4n
  double* total_time;  // n
  int8_t* bridge;    // n, reaction found by the Brownian bridge
  double* enc_c;     // 3n, pose at reaction
  double* enc_q;     // 4n
  int* enc_step;     // n
  // histograms (SH_* layout) and the bin edges they use
  unsigned long long* hist;
  const double* rad_edges;    // ST_RAD_BINS + 1
  const double* trans_edges;  // ST_TRANS + 1
  const double* ms_radii;     // ST_MILESTONES
};

struct DevSim {
  long long n_traj;
  long long id_offset;  // global id of local trajectory 0
  uint32_t k0, k1;  // seed words
  double r_b, r_esc, return_prob;
  int max_steps;
  double max_dt, min_core_dt, min_core_rxn_dt;
  int use_hi, overlap;
  double D_t, D_r;
  double adt_V0, adt_inv_debye, adt_debye;
  int adt_has_force;
  double hi_Df, hi_ainv, hi_a2;
  int hi_mode;                 // BD_HI_REFERENCE_GPU or BD_HI_ZUK
  double zuk_a, zuk_b, zuk_kTeta;  // hydrodynamic radii and kBT/eta of the Zuk coupling
  unsigned long long* ctr;
  int8_t* out_status;
  int* out_steps;
  int* out_returns;
  DevStats st;
  int stats;  // collect DevStats (needs SH_NUM * 4 B of dynamic shared memory per block)
  // path / energy traces (with stats): rows of 8 and 6 doubles every save_interval steps
  int save_interval;
  long long trace_cap;
  double* trace_path;
  double* trace_energy;
};

struct SlotBuf {
  double* c;    // 3 * cap (x block, y block, z block)
  double* q;    // 4 * cap
  int* traj;
  int* steps;
  int* rets;
  int8_t* status;
  int8_t* state;  // state-machine reaction state (0 = the first state)
  int cap;
};

// ----------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11) and the draws built from it
// ----------------------------------------------------------------------------
struct W4 { uint32_t a, b, c, d; };

__device__ __forceinline__ W4 philox10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                       uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return {c0, c1, c2, c3};
}

__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ void box_muller(double u1, double u2, double& n0, double& n1) {
  const double rad = sqrt(-2.0 * log(1.0 - u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  n0 = rad * c;
  n1 = rad * s;
}

enum : uint32_t { SUB_ESCAPE = 0, SUB_NORMALS = 1, SUB_RETURN_Q = 4, SUB_BRIDGE = 6 };
enum : uint32_t { INIT_STEP = 0xFFFFFFFFu, SUB_INIT_DIR = 0, SUB_INIT_Q = 2 };

struct Keyed {
  uint32_t k0, k1, t0, t1;
  __device__ __forceinline__ W4 w(uint32_t step, uint32_t sub) const { return philox10(step, sub, t0, t1, k0, k1); }
};

// ----------------------------------------------------------------------------
// Small vector helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ double norm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

__device__ __forceinline__ void quat_to_rot(const double q[4], double R[9]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z);
  R[1] = 2 * (x * y - w * z);
  R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);
  R[4] = 1 - 2 * (x * x + z * z);
  R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);
  R[7] = 2 * (y * z + w * x);
  R[8] = 1 - 2 * (x * x + y * y);
}

__device__ __forceinline__ void shoemake(double u0, double u1, double u2, double q[4]) {
  const double a = sqrt(1 - u0), b = sqrt(u0);
  double s1, c1, s2, c2;
  sincospi(2.0 * u1, &s1, &c1);
  sincospi(2.0 * u2, &s2, &c2);
  q[0] = a * s1;
  q[1] = a * c1;
  q[2] = b * s2;
  q[3] = b * c2;
}

// q <- normalize(q (x) dq(omega)); omega applied in the body frame.
__device__ __forceinline__ void rotate_quat(double q[4], double o0, double o1, double o2) {
  const double angle = norm3(o0, o1, o2);
  double a0 = 0, a1 = 0, a2 = 0;
  if (angle > 1e-10) {
    a0 = o0 / angle;
    a1 = o1 / angle;
    a2 = o2 / angle;
  }
  double sh, ch;
  sincos(angle * 0.5, &sh, &ch);
  const double w2 = ch, x2 = a0 * sh, y2 = a1 * sh, z2 = a2 * sh;
  const double w1 = q[0], x1 = q[1], y1 = q[2], z1 = q[3];
  double n0 = w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2;
  double n1 = w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2;
  double n2 = w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2;
  double n3 = w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2;
  const double nn = sqrt(n0 * n0 + n1 * n1 + n2 * n2 + n3 * n3);
  q[0] = n0 / nn;
  q[1] = n1 / nn;
  q[2] = n2 / nn;
  q[3] = n3 / nn;
}

// ----------------------------------------------------------------------------
// Grid stencil.
//
// The reference's gradient is (I(x+h) - I(x-h)) / (2h), h = sp/2, with I the
// trilinear interpolant, per axis and at the centre point's other two
// coordinates (gpu_batch_engine.py:111-114).  Because I is linear in the node
// values, each axis term equals a weighted sum of ADJACENT-node differences:
// with c = floor(u), s = u - c, the two probes share the fraction |s - 1/2|
// and straddle one extra node e = c-1 (s < 1/2) or c+2 (s >= 1/2), so
//     D = (1 - a) (v[c+1] - v[c]) + a * De,   a = |s - 1/2|,
// De = v[c] - v[c-1] or v[c+2] - v[c+1], summed with the centre's bilinear
// weights on the other axes.  This reads 20 distinct nodes (centre cube + one
// extra node per cube edge line) instead of the reference's 7 x 8 = 56, and
// the differences avoid cancelling the large common offset in FP32.
// ----------------------------------------------------------------------------
template <typename FT, int CH>
struct StencilOut {
  FT phi[CH], gx[CH], gy[CH], gz[CH];
};

__device__ __forceinline__ bool in_box(const DevGrid& g, double x, double y, double z) {
  return x > g.lox && x < g.hix && y > g.loy && y < g.hiy && z > g.loz && z < g.hiz;
}

template <int CH>
__device__ __forceinline__ void ld(const float* p, float v[CH]) {
  if constexpr (CH == 1) {
    v[0] = __ldg(p);
  } else {
    const float2 t = __ldg(reinterpret_cast<const float2*>(p));
    v[0] = t.x;
    v[1] = t.y;
  }
}

// One 32-byte read-only load (a whole sector) of eight floats; p is 32-byte aligned.
__device__ __forceinline__ void ld8(const float* p, float v[8]) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
      : "l"(p));
}

// floor(u) as a value and as an int, for 0 <= u < 2^23 (float) or 2^52 (double):
// adding 2^23 (2^52) with round-down leaves exactly floor(u) in the low mantissa
// bits, so the cell index needs no float-to-int conversion.  Every stencil
// position is inside its grid's margin box, so u >= 3.
__device__ __forceinline__ void floor_split(float u, float& f, int& c) {
  const float t = __fadd_rd(u, 8388608.0f);
  c = __float_as_int(t) - 0x4B000000;
  f = t - 8388608.0f;
}
__device__ __forceinline__ void floor_split(double u, double& f, int& c) {
  const double t = __dadd_rd(u, 4503599627370496.0);
  c = (int)(__double_as_longlong(t) - 0x4330000000000000ll);
  f = t - 4503599627370496.0;
}

// PT is the type of the position and of the cell/fraction arithmetic: double
// everywhere except the mixed-precision reverse-Born sweep, which hands in FP32
// ligand-frame coordinates (the interpolant is continuous, so an FP32 position
// only moves the result by its own rounding).
template <typename FT, int CH, typename PT = double>
__device__ __forceinline__ StencilOut<FT, CH> stencil(const DevGrid& g, PT x, PT y, PT z) {
  PT ox, oy, oz, isx, isy, isz;
  if constexpr (sizeof(PT) == 4) {  // the host-rounded FP32 copies: no conversion per evaluation
    ox = g.oxf;
    oy = g.oyf;
    oz = g.ozf;
    isx = g.isxf;
    isy = g.isyf;
    isz = g.iszf;
  } else {
    ox = g.ox;
    oy = g.oy;
    oz = g.oz;
    isx = g.isx;
    isy = g.isy;
    isz = g.isz;
  }
  const PT ux = (x - ox) * isx, uy = (y - oy) * isy, uz = (z - oz) * isz;
  PT fx, fy, fz;
  int cx, cy, cz;
  floor_split(ux, fx, cx);
  floor_split(uy, fy, cy);
  floor_split(uz, fz, cz);
  const PT sxd = ux - fx, syd = uy - fy, szd = uz - fz;
  const PT half = (PT)0.5;
  const bool lx = sxd < half, ly = syd < half, lz = szd < half;
  const int ex = lx ? cx - 1 : cx + 2, ey = ly ? cy - 1 : cy + 2;
  const FT sx = (FT)sxd, sy = (FT)syd, sz = (FT)szd;
  const FT ax = (FT)(lx ? half - sxd : sxd - half);
  const FT ay = (FT)(ly ? half - syd : syd - half);
  const FT az = (FT)(lz ? half - szd : szd - half);
  // node indices fit in int: grids are limited to 2^30 nodes of at most two channels
  const int nz = g.nz, syz = g.ny * g.nz;
  const float* d = g.data;
  // centre rows (cx+i, cy+j): three z nodes starting at zb
  const int zb = lz ? cz - 1 : cz;
  const int zc = lz ? 1 : 0;  // position of node cz inside the three-node run
  const int ze = lz ? 0 : 2;  // position of the extra z node
  float r[2][2][3][CH], xe[2][2][CH], ye[2][2][CH];
  if (CH == 1 && g.cube) {
    // cube copy: the centre block, the x-extra face, the y-extra and z-extra edges in four loads
    // (three with the xy records: the x face and the y edge of this cell half come in one)
    const float* cb = g.cube;
    const long node = (long)(cx * g.ny + cy) * nz + cz;
    float c8[8], z8[8];
    ld8(cb + 8 * node, c8);
    if (g.ztex) {
      const float4 zr = tex1Dfetch<float4>(g.ztex, (int)(2 * node + (lz ? 0 : 1)));
      z8[0] = zr.x;
      z8[2] = zr.y;
      z8[4] = zr.z;
      z8[6] = zr.w;
    } else {
      ld8(cb + 8 * ((long)(cx * g.ny + cy) * nz + (lz ? cz - 1 : cz + 2)), z8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        r[i][j][zc][0] = c8[4 * i + 2 * j];
        r[i][j][zc + 1][0] = c8[4 * i + 2 * j + 1];
        r[i][j][ze][0] = z8[4 * i + 2 * j];
      }
    if (g.xy) {
      float e8[8];
      const long rec = 4 * node + 2 * (lx ? 0 : 1) + (ly ? 0 : 1);
      if (g.xytex) {
        const float4 a = tex1Dfetch<float4>(g.xytex, (int)(2 * rec)), b = tex1Dfetch<float4>(g.xytex, (int)(2 * rec + 1));
        e8[0] = a.x;
        e8[1] = a.y;
        e8[2] = a.z;
        e8[3] = a.w;
        e8[4] = b.x;
        e8[5] = b.y;
        e8[6] = b.z;
        e8[7] = b.w;
      } else {
        ld8(g.xy + 8 * rec, e8);
      }
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          xe[j][k][0] = e8[2 * j + k];
          ye[j][k][0] = e8[4 + 2 * j + k];
        }
    } else {
      float y8[8];
      const float4 xf = __ldg(reinterpret_cast<const float4*>(cb + 8 * (long)((ex * g.ny + cy) * nz + cz)));
      ld8(cb + 8 * (long)((cx * g.ny + ey) * nz + cz), y8);
      xe[0][0][0] = xf.x;
      xe[0][1][0] = xf.y;
      xe[1][0][0] = xf.z;
      xe[1][1][0] = xf.w;
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        ye[i][0][0] = y8[4 * i];
        ye[i][1][0] = y8[4 * i + 1];
      }
    }
  } else if (g.win) {
    // window copy: one 16-byte load per z run (two for a 3-node run of two channels)
    const float4* w = g.win;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n = (cx + i) * syz + (cy + j) * nz + zb;
        const float4 t = __ldg(w + n);
        if constexpr (CH == 1) {
          r[i][j][0][0] = t.x;
          r[i][j][1][0] = t.y;
          r[i][j][2][0] = t.z;
        } else {
          const float4 u = __ldg(w + n + 2);
          r[i][j][0][0] = t.x;
          r[i][j][0][1] = t.y;
          r[i][j][1][0] = t.z;
          r[i][j][1][1] = t.w;
          r[i][j][2][0] = u.x;
          r[i][j][2][1] = u.y;
        }
      }
    float4 tx[2], ty[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) tx[j] = __ldg(w + (ex * syz + (cy + j) * nz + cz));
#pragma unroll
    for (int i = 0; i < 2; ++i) ty[i] = __ldg(w + ((cx + i) * syz + ey * nz + cz));
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if constexpr (CH == 1) {
        xe[j][0][0] = tx[j].x;
        xe[j][1][0] = tx[j].y;
        ye[j][0][0] = ty[j].x;
        ye[j][1][0] = ty[j].y;
      } else {
        xe[j][0][0] = tx[j].x;
        xe[j][0][1] = tx[j].y;
        xe[j][1][0] = tx[j].z;
        xe[j][1][1] = tx[j].w;
        ye[j][0][0] = ty[j].x;
        ye[j][0][1] = ty[j].y;
        ye[j][1][0] = ty[j].z;
        ye[j][1][1] = ty[j].w;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int base = ((cx + i) * syz + (cy + j) * nz + zb) * CH;
#pragma unroll
        for (int k = 0; k < 3; ++k) ld<CH>(d + base + k * CH, r[i][j][k]);
      }
    if (CH == 2 && g.ptex) {
      // the eight extra nodes through the texture path, the twelve centre-row nodes above through LSU
      auto tx = [&](int node, float v[CH]) {
        const float2 t = tex1Dfetch<float2>(g.ptex, node);
        v[0] = t.x;
        v[CH - 1] = t.y;
      };
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int n = ex * syz + (cy + j) * nz + cz;
        tx(n, xe[j][0]);
        tx(n + 1, xe[j][1]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int n = (cx + i) * syz + ey * nz + cz;
        tx(n, ye[i][0]);
        tx(n + 1, ye[i][1]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int base = (ex * syz + (cy + j) * nz + cz) * CH;
        ld<CH>(d + base, xe[j][0]);
        ld<CH>(d + base + CH, xe[j][1]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int base = ((cx + i) * syz + ey * nz + cz) * CH;
        ld<CH>(d + base, ye[i][0]);
        ld<CH>(d + base + CH, ye[i][1]);
      }
    }
  }
  const FT wx[2] = {(FT)1 - sx, sx}, wy[2] = {(FT)1 - sy, sy}, wz[2] = {(FT)1 - sz, sz};
  StencilOut<FT, CH> o;
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    FT v[2][2][2], zx[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        v[i][j][0] = (FT)r[i][j][zc][c];
        v[i][j][1] = (FT)r[i][j][zc + 1][c];
        zx[i][j] = (FT)r[i][j][ze][c];
      }
    FT phi = 0, Dx = 0, Dy = 0, Dz = 0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int k = 0; k < 2; ++k) phi += wx[i] * wy[j] * wz[k] * v[i][j][k];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const FT d0 = v[1][j][k] - v[0][j][k];
        const FT e = (FT)xe[j][k][c];
        const FT de = lx ? (v[0][j][k] - e) : (e - v[1][j][k]);
        Dx += wy[j] * wz[k] * (((FT)1 - ax) * d0 + ax * de);
      }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const FT d0 = v[i][1][k] - v[i][0][k];
        const FT e = (FT)ye[i][k][c];
        const FT de = ly ? (v[i][0][k] - e) : (e - v[i][1][k]);
        Dy += wx[i] * wz[k] * (((FT)1 - ay) * d0 + ay * de);
      }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const FT d0 = v[i][j][1] - v[i][j][0];
        const FT e = zx[i][j];
        const FT de = lz ? (v[i][j][0] - e) : (e - v[i][j][1]);
        Dz += wx[i] * wy[j] * (((FT)1 - az) * d0 + az * de);
      }
    o.phi[c] = phi;
    o.gx[c] = Dx * (FT)g.isx;
    o.gy[c] = Dy * (FT)g.isy;
    o.gz[c] = Dz * (FT)g.isz;
  }
  return o;
}

// ----------------------------------------------------------------------------
// Yukawa multipole far-field for one ligand atom (gpu_batch_engine.py:393-472):
// monopole + dipole + quadrupole, radial derivative only, r clamped at 1 A.
// ----------------------------------------------------------------------------
template <typename FT>
__device__ __forceinline__ void farfield(const DevSystem& S, double xd, double yd, double zd, FT q, FT f[3],
                                         FT& e) {
  const FT x = (FT)xd, y = (FT)yd, z = (FT)zd;
  const FT r = sqrt(x * x + y * y + z * z);
  const FT sr = r > (FT)1 ? r : (FT)1;
  const FT inv = (FT)1 / sr;
  const FT il = (FT)S.inv_debye;
  const FT ex = exp(-sr * il);
  const FT rx = x * inv, ry = y * inv, rz = z * inv;
  const FT Vf = (FT)S.V_factor;
  FT phi = Vf * ex * inv;
  FT dphi = Vf * ex * (-inv * inv - inv * il);
  if (S.use_dip) {
    const FT pr = rx * (FT)S.dip[0] + ry * (FT)S.dip[1] + rz * (FT)S.dip[2];
    const FT ifpe = (FT)S.inv_fpe;
    phi += pr * ifpe * inv * inv * ((FT)1 + sr * il) * ex;
    dphi += pr * ifpe * ex * ((FT)-2 * inv * inv * inv - (FT)2 * inv * inv * il - inv * il * il);
  }
  if (S.use_quad) {
    const FT qx = (FT)S.quad[0] * rx + (FT)S.quad[1] * ry + (FT)S.quad[2] * rz;
    const FT qy = (FT)S.quad[3] * rx + (FT)S.quad[4] * ry + (FT)S.quad[5] * rz;
    const FT qz = (FT)S.quad[6] * rx + (FT)S.quad[7] * ry + (FT)S.quad[8] * rz;
    const FT rQr = rx * qx + ry * qy + rz * qz;
    const FT ifpe = (FT)S.inv_fpe;
    const FT i2 = inv * inv, i3 = i2 * inv;
    phi += rQr * ifpe * i3 * ((FT)1 + sr * il + sr * sr * il * il * ((FT)1 / (FT)3)) * ex;
    dphi += rQr * ifpe * ex *
            ((FT)-3 * i3 * inv - (FT)3 * i3 * il - i2 * il * il - inv * il * il * il * ((FT)1 / (FT)3));
  }
  const FT c = -q * dphi;
  f[0] = c * rx;
  f[1] = c * ry;
  f[2] = c * rz;
  e = q * phi;
}

}  // namespace bd
