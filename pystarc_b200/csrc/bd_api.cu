// C ABI of the batched BD engine: handle, uploads, force evaluation and the stepper.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "bd_kernels.cuh"
#include "bd_nvtx.cuh"
#include "bd_multi.cuh"
#include "bd_surrogate.cuh"
#include "bd_split.cuh"
#include "pystarc_b200.h"

// surrogate MLP (bd_mlp.cu)
int bd_internal_mlp_shape(const BdMlp* m, int* in_dim, int* in_pad, int* out_dim);
int bd_internal_mlp_prepare(BdMlp* m, int rows);
int bd_internal_mlp_ensemble_rows(BdMlp* m, int rows, const int* n_dev, const void* Xpacked, float* mean,
                                  float* spread, cudaStream_t s);
const char* bd_internal_mlp_error(const BdMlp* m);

using namespace bd;

namespace {

const double kEps0 = 0.000142;
const double kPi = 3.14159265358979323846;

struct GridHost {
  std::vector<float> data;
  int n[3];
  double o[3], sp[3];
};

std::string g_create_error;

}  // namespace

struct BdHandle {
  int device = 0;
  int n_sm = 148;
  std::string err;
  cudaStream_t own = nullptr;
  // host-side inputs
  std::vector<double> lig;  // x,y,z,q
  std::vector<double> rec;  // x,y,z,q
  std::vector<double> rec_rad, lig_rad;  // WCA contact radii (empty: term off)
  int sm_n = 0, sm_states = 0;  // state-machine reactions (bd_set_reaction_states; 0: off)
  int sm_before[BD_MAX_PAIRS] = {}, sm_after[BD_MAX_PAIRS] = {};
  unsigned long long sm_terminal = 0;
  double wca_eps = 0.0, wca_act = -1.0;
  std::vector<GridHost> grids[3];
  BdForceParams fp{};
  bool fp_set = false;
  int n_pairs = 0, n_needed = 1;
  double rx_rec[BD_MAX_PAIRS][3], rx_body[BD_MAX_PAIRS][3], rx_cut[BD_MAX_PAIRS], rx_deff[BD_MAX_PAIRS];
  bool dirty = true;
  // device system
  DevSystem S{};
  std::vector<void*> sys_allocs;
  std::vector<cudaTextureObject_t> sys_tex;  // texture views of system buffers
  // stepper
  bool sim_ready = false;
  BdSimParams sp{};
  DevSim P{};
  SlotBuf buf[2]{};
  int* d_live = nullptr;  // [2]
  int cur = 0;
  unsigned long long* d_ctr = nullptr;
  std::vector<void*> sim_allocs;
  int group = 8, block = 128;
  bool launch_user = false;
  int layout = BD_LAYOUT_DEFAULT;
  unsigned terms = BD_TERM_ALL;
  // learned surrogate (bd_sim_set_surrogate): the model, its constants, per-slot scratch
  BdMlp* sur = nullptr;
  DevSurrogate sur_q{};
  SurBuf sur_buf{};
  int sur_cap = 0;
  // split stepper (BD_GROUP_SPLIT): per-slot scratch of one step
  SplitBuf split_buf{};
  int split_cap = 0;
  unsigned long long* sur_ctr_host_base = nullptr;
  // graphs: [cur][steps] cache
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_K = -1, graph_G = -1, graph_B = -1, graph_prec = -1, graph_torque = -1;
};

namespace {

int fail(BdHandle* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  else g_create_error = buf;
  return code;
}

#define CK(h, x)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess)                                                                         \
      return fail(h, e_ == cudaErrorMemoryAllocation ? BD_ERR_OOM : BD_ERR_CUDA, "%s: %s (%s:%d)", #x, \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                                      \
  } while (0)

int dev_alloc(BdHandle* h, std::vector<void*>& list, void** p, size_t bytes) {
  CK(h, cudaMalloc(p, bytes ? bytes : 16));
  list.push_back(*p);
  return BD_OK;
}

void free_list(std::vector<void*>& list) {
  for (void* p : list) cudaFree(p);
  list.clear();
}

void free_tex(std::vector<cudaTextureObject_t>& list) {
  for (cudaTextureObject_t t : list) cudaDestroyTextureObject(t);
  list.clear();
}

// Receptor atoms order[b, e) split at the median of their widest axis until every
// group holds at most BD_CHUNK atoms; the left part of each split is a whole number
// of chunks, so only the last chunk can be partial.  The chunks are compact
// (median-split boxes), which keeps their bounding spheres small for the culls.
void kd_chunks(const std::vector<double>& rec, std::vector<int>& order, int b, int e) {
  const int n = e - b;
  if (n <= BD_CHUNK) return;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = b; i < e; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], rec[4 * order[i] + k]);
      hi[k] = std::max(hi[k], rec[4 * order[i] + k]);
    }
  int ax = 0;
  for (int k = 1; k < 3; ++k)
    if (hi[k] - lo[k] > hi[ax] - lo[ax]) ax = k;
  const int left = ((n + BD_CHUNK - 1) / BD_CHUNK / 2) * BD_CHUNK;
  std::nth_element(order.begin() + b, order.begin() + b + left, order.begin() + e, [&](int x, int y) {
    const double u = rec[4 * x + ax], v = rec[4 * y + ax];
    return u < v || (u == v && x < y);
  });
  kd_chunks(rec, order, b, b + left);
  kd_chunks(rec, order, b + left, e);
}

void grid_to_dev(const GridHost& g, const float* dptr, int ch, DevGrid& d) {
  d.data = dptr;
  d.nx = g.n[0];
  d.ny = g.n[1];
  d.nz = g.n[2];
  d.ch = ch;
  d.ox = g.o[0];
  d.oy = g.o[1];
  d.oz = g.o[2];
  d.isx = 1.0 / g.sp[0];
  d.isy = 1.0 / g.sp[1];
  d.isz = 1.0 / g.sp[2];
  const double m = 3.0;
  d.lox = g.o[0] + m * g.sp[0];
  d.loy = g.o[1] + m * g.sp[1];
  d.loz = g.o[2] + m * g.sp[2];
  d.hix = g.o[0] + ((double)g.n[0] - 1 - m) * g.sp[0];
  d.hiy = g.o[1] + ((double)g.n[1] - 1 - m) * g.sp[1];
  d.hiz = g.o[2] + ((double)g.n[2] - 1 - m) * g.sp[2];
  d.oxf = (float)d.ox;
  d.oyf = (float)d.oy;
  d.ozf = (float)d.oz;
  d.isxf = (float)d.isx;
  d.isyf = (float)d.isy;
  d.iszf = (float)d.isz;
}

int upload_floats(BdHandle* h, const float* src, size_t n, const float** out) {
  void* p = nullptr;
  int rc = dev_alloc(h, h->sys_allocs, &p, n * sizeof(float));
  if (rc) return rc;
  CK(h, cudaMemcpy(p, src, n * sizeof(float), cudaMemcpyHostToDevice));
  *out = (const float*)p;
  return BD_OK;
}

// Window copy of an uploaded grid for the vector stencil loads (DevGrid::win).
int add_window(BdHandle* h, DevGrid& g) {
  const long n = (long)g.nx * g.ny * g.nz;
  void* p = nullptr;
  int rc = dev_alloc(h, h->sys_allocs, &p, (size_t)n * sizeof(float4));
  if (rc) return rc;
  window_kernel<<<h->n_sm * 8, 256>>>(g.data, (float4*)p, n, g.nz, g.ch);
  CK(h, cudaGetLastError());
  g.win = (const float4*)p;
  return BD_OK;
}

// Cube copy of an uploaded one-channel grid for the four-load stencil (DevGrid::cube).
int add_cube(BdHandle* h, DevGrid& g) {
  const long n = (long)g.nx * g.ny * g.nz;
  void* p = nullptr;
  int rc = dev_alloc(h, h->sys_allocs, &p, (size_t)n * 8 * sizeof(float));
  if (rc) return rc;
  cube_kernel<<<h->n_sm * 8, 256>>>(g.data, (float*)p, g.nx, g.ny, g.nz);
  CK(h, cudaGetLastError());
  g.cube = (const float*)p;
  return BD_OK;
}

// Overlap occupancy grid over the first nr atoms of the receptor table ra (x, y, z, q per
// atom, already on the device as S.rec): classified on the device in two passes around a
// host prefix sum.  Leaves S.ov_cell NULL (the chunk sweep) when the grid would exceed
// BD_OVERLAP_MAX_CELLS cells or its lists the 24-bit offsets.
int build_overlap_grid(BdHandle* h, DevSystem& S, const std::vector<double>& ra, int nr) {
  OvGeom G{};
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int a = 0; a < nr; ++a)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], ra[4 * a + d]);
      hi[d] = std::max(hi[d], ra[4 * a + d]);
    }
  long long cells = 1;
  for (int d = 0; d < 3; ++d) {
    G.o[d] = lo[d] - (kOvR + kOvCell);
    G.n[d] = (int)std::ceil((hi[d] + kOvR + kOvCell - G.o[d]) / kOvCell);
    G.nb[d] = (int)std::ceil(G.n[d] * kOvCell / kOvBin);
    cells *= G.n[d];
  }
  if (cells > BD_OVERLAP_MAX_CELLS) return BD_OK;
  // atoms binned on the kOvBin lattice (CSR, atoms in table order within a bin)
  const int nbins = G.nb[0] * G.nb[1] * G.nb[2];
  std::vector<int> bin_of(nr), start(nbins + 1, 0), atoms(nr);
  for (int a = 0; a < nr; ++a) {
    int b[3];
    for (int d = 0; d < 3; ++d) b[d] = std::min(G.nb[d] - 1, std::max(0, (int)std::floor((ra[4 * a + d] - G.o[d]) / kOvBin)));
    bin_of[a] = (b[0] * G.nb[1] + b[1]) * G.nb[2] + b[2];
    ++start[bin_of[a] + 1];
  }
  for (int b = 0; b < nbins; ++b) start[b + 1] += start[b];
  {
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int a = 0; a < nr; ++a) atoms[fill[bin_of[a]]++] = a;
  }
  // build-only buffers, freed on every way out
  struct Tmp {
    void* p = nullptr;
    ~Tmp() {
      if (p) cudaFree(p);
    }
  } t_start, t_atoms, t_cnt, t_cls;
  if (cudaMalloc(&t_start.p, start.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&t_atoms.p, std::max<size_t>(1, atoms.size()) * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&t_cnt.p, (size_t)cells * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&t_cls.p, (size_t)cells) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, BD_ERR_CUDA, "out of device memory for the overlap grid (%lld cells)", cells);
  }
  int* d_start = (int*)t_start.p;
  int* d_atoms = (int*)t_atoms.p;
  int* d_cnt = (int*)t_cnt.p;
  uint8_t* d_cls = (uint8_t*)t_cls.p;
  int* d_list = nullptr;
  uint32_t* d_word = nullptr;
  CK(h, cudaMemcpy(d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(d_atoms, atoms.data(), atoms.size() * sizeof(int), cudaMemcpyHostToDevice));
  const int blocks = h->n_sm * 8;
  ov_cells_kernel<<<blocks, 256>>>(S.rec, d_start, d_atoms, G, d_cls, d_cnt, nullptr, nullptr);
  CK(h, cudaGetLastError());
  std::vector<uint8_t> cls((size_t)cells);
  std::vector<int> cnt((size_t)cells);
  CK(h, cudaMemcpy(cls.data(), d_cls, cls.size(), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(cnt.data(), d_cnt, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> word((size_t)cells);
  long long total = 0;
  for (long long c = 0; c < cells; ++c) {
    if (cls[c] == 0) {
      word[c] = 0u;
    } else if (cls[c] == 1) {
      word[c] = 0xffffffffu;
    } else {
      if (cnt[c] > 255 || total + cnt[c] >= (1ll << 24) - 1) return BD_OK;  // does not fit the encoding: keep the sweep
      word[c] = ((uint32_t)total << 8) | (uint32_t)cnt[c];
      total += cnt[c];
    }
  }
  void* p;
  int rc = dev_alloc(h, h->sys_allocs, &p, (size_t)cells * sizeof(uint32_t));
  if (rc) return rc;
  d_word = (uint32_t*)p;
  CK(h, cudaMemcpy(d_word, word.data(), word.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
  rc = dev_alloc(h, h->sys_allocs, &p, (size_t)std::max(1ll, total) * sizeof(int));
  if (rc) return rc;
  d_list = (int*)p;
  ov_cells_kernel<<<blocks, 256>>>(S.rec, d_start, d_atoms, G, nullptr, nullptr, d_word, d_list);
  CK(h, cudaGetLastError());
  CK(h, cudaDeviceSynchronize());
  S.ov_cell = d_word;
  S.ov_list = d_list;
  for (int d = 0; d < 3; ++d) {
    S.ov_o[d] = G.o[d];
    S.ov_n[d] = G.n[d];
  }
  S.ov_inv_h = 1.0 / kOvCell;
  return BD_OK;
}

// A float4 texture view of n float4 elements at p (linear memory, point sampling).
int float4_texture(BdHandle* h, void* p, size_t n, cudaTextureObject_t* out) {
  cudaResourceDesc res{};
  res.resType = cudaResourceTypeLinear;
  res.res.linear.devPtr = p;
  res.res.linear.desc = cudaCreateChannelDesc<float4>();
  res.res.linear.sizeInBytes = n * sizeof(float4);
  cudaTextureDesc td{};
  td.readMode = cudaReadModeElementType;
  td.filterMode = cudaFilterModePoint;
  td.addressMode[0] = cudaAddressModeClamp;
  cudaTextureObject_t t = 0;
  CK(h, cudaCreateTextureObject(&t, &res, &td, nullptr));
  h->sys_tex.push_back(t);
  *out = t;
  return BD_OK;
}

// A float2 texture view of n float2 elements at p (linear memory, point sampling).
int float2_texture(BdHandle* h, void* p, size_t n, cudaTextureObject_t* out) {
  cudaResourceDesc res{};
  res.resType = cudaResourceTypeLinear;
  res.res.linear.devPtr = p;
  res.res.linear.desc = cudaCreateChannelDesc<float2>();
  res.res.linear.sizeInBytes = n * sizeof(float2);
  cudaTextureDesc td{};
  td.readMode = cudaReadModeElementType;
  td.filterMode = cudaFilterModePoint;
  td.addressMode[0] = cudaAddressModeClamp;
  cudaTextureObject_t t = 0;
  CK(h, cudaCreateTextureObject(&t, &res, &td, nullptr));
  h->sys_tex.push_back(t);
  *out = t;
  return BD_OK;
}

// xy records of a grid that has its cube copy (DevGrid::xy), and their texture view when asked.
int add_xy(BdHandle* h, DevGrid& g, bool tex) {
  const long n = (long)g.nx * g.ny * g.nz;
  void* p = nullptr;
  int rc = dev_alloc(h, h->sys_allocs, &p, (size_t)n * 32 * sizeof(float));
  if (rc) return rc;
  xy_kernel<<<h->n_sm * 8, 256>>>(g.data, (float*)p, g.nx, g.ny, g.nz);
  CK(h, cudaGetLastError());
  g.xy = (const float*)p;
  // linear textures address at most 2^27 elements
  if (tex && (double)n * 8.0 <= (double)(1 << 27)) return float4_texture(h, p, (size_t)n * 8, &g.xytex);
  return BD_OK;
}

// z-edge records of a grid that has its cube copy, read through the texture path (DevGrid::ztex).
int add_ztex(BdHandle* h, DevGrid& g) {
  const long n = (long)g.nx * g.ny * g.nz;
  void* p = nullptr;
  int rc = dev_alloc(h, h->sys_allocs, &p, (size_t)n * 2 * sizeof(float4));
  if (rc) return rc;
  zedge_kernel<<<h->n_sm * 8, 256>>>(g.data, (float4*)p, g.nx, g.ny, g.nz);
  CK(h, cudaGetLastError());
  return float4_texture(h, p, (size_t)n * 2, &g.ztex);
}

bool same_lattice(const GridHost& a, const GridHost& b) {
  for (int i = 0; i < 3; ++i)
    if (a.n[i] != b.n[i] || a.o[i] != b.o[i] || a.sp[i] != b.sp[i]) return false;
  return true;
}

// Build the device-side system: grid selection rules, uploads, receptor chunks.
int finalize(BdHandle* h) {
  if (!h->dirty) return BD_OK;
  CK(h, cudaSetDevice(h->device));
  CK(h, cudaDeviceSynchronize());
  free_tex(h->sys_tex);
  free_list(h->sys_allocs);
  DevSystem S{};
  if (h->lig.empty()) return fail(h, BD_ERR_STATE, "ligand not set");
  const BdForceParams& fp = h->fp;
  // far field (gpu_batch_engine.py:162-175)
  const double eps_s = fp.sdie * kEps0;
  S.V_factor = eps_s > 0 ? fp.receptor_charge / (4.0 * kPi * eps_s) : 0.0;
  S.has_yukawa = std::fabs(fp.receptor_charge) > 1e-9 && fp.debye_length > 0;
  S.inv_debye = fp.debye_length > 0 ? 1.0 / fp.debye_length : 0.0;
  S.alpha = fp.alpha;
  if (fp.use_multipole) {
    double pn = 0, qn = 0;
    for (int i = 0; i < 3; ++i) pn += fp.dipole[i] * fp.dipole[i];
    for (int i = 0; i < 9; ++i) qn += fp.quadrupole[i] * fp.quadrupole[i];
    S.use_dip = std::sqrt(pn) > 1e-9;
    S.use_quad = std::sqrt(qn) > 1e-9;
    for (int i = 0; i < 3; ++i) S.dip[i] = fp.dipole[i];
    for (int i = 0; i < 9; ++i) S.quad[i] = fp.quadrupole[i];
    S.inv_fpe = 1.0 / fp.four_pi_eps;
  }
  // grids: finest first (stable on the x spacing), reference dropping rules
  std::vector<GridHost> el = h->grids[BD_GRID_ELEC], bo = h->grids[BD_GRID_BORN], lb = h->grids[BD_GRID_LIG_BORN];
  auto finer = [](const GridHost& a, const GridHost& b) { return a.sp[0] < b.sp[0]; };
  std::stable_sort(el.begin(), el.end(), finer);
  std::stable_sort(bo.begin(), bo.end(), finer);
  std::stable_sort(lb.begin(), lb.end(), finer);
  if (S.has_yukawa && el.size() > 1) el.resize(1);
  if (bo.size() > 1) bo.resize(1);
  if (lb.size() > 1) lb.resize(1);
  if (el.size() > BD_MAX_ELEC) return fail(h, BD_ERR_ARG, "at most %d electrostatic grids", BD_MAX_ELEC);
  S.n_elec = (int)el.size();
  for (int k = 0; k < S.n_elec; ++k) {
    const float* p;
    int rc = upload_floats(h, el[k].data.data(), el[k].data.size(), &p);
    if (rc) return rc;
    grid_to_dev(el[k], p, 1, S.elec[k]);
  }
  S.has_born = !bo.empty();
  if (S.has_born) {
    const float* p;
    int rc = upload_floats(h, bo[0].data.data(), bo[0].data.size(), &p);
    if (rc) return rc;
    grid_to_dev(bo[0], p, 1, S.born);
    if (S.n_elec > 0 && same_lattice(el[0], bo[0])) {
      std::vector<float> il(2 * el[0].data.size());
      for (size_t i = 0; i < el[0].data.size(); ++i) {
        il[2 * i] = el[0].data[i];
        il[2 * i + 1] = bo[0].data[i];
      }
      rc = upload_floats(h, il.data(), il.size(), &p);
      if (rc) return rc;
      grid_to_dev(el[0], p, 2, S.pair);
      S.paired = 1;
      // linear textures address at most 2^27 elements
      if ((h->layout & BD_LAYOUT_PTEX_2) && el[0].data.size() <= (size_t)(1 << 27))
        if ((rc = float2_texture(h, (void*)p, el[0].data.size(), &S.pair.ptex))) return rc;
    }
  }
  if (h->layout & BD_LAYOUT_WINDOWS_1) {
    // a paired lattice is read through the pair copy only: its single-channel grids need no window
    for (int k = S.paired ? 1 : 0; k < S.n_elec; ++k)
      if (int rc = add_window(h, S.elec[k])) return rc;
    if (S.has_born && !S.paired)
      if (int rc = add_window(h, S.born)) return rc;
  }
  if (S.paired && (h->layout & BD_LAYOUT_WINDOWS_2))
    if (int rc = add_window(h, S.pair)) return rc;
  // ligand
  const int nl = (int)(h->lig.size() / 4);
  S.n_lig = nl;
  {
    void* p;
    int rc = dev_alloc(h, h->sys_allocs, &p, h->lig.size() * sizeof(double));
    if (rc) return rc;
    CK(h, cudaMemcpy(p, h->lig.data(), h->lig.size() * sizeof(double), cudaMemcpyHostToDevice));
    S.lig = (const double4*)p;
  }
  // receptor: spatial (k-d median split) order, chunks of BD_CHUNK with bounding spheres
  const int nr = (int)(h->rec.size() / 4);
  if (nr > 0) {
    double rmax = 0;
    for (int i = 0; i < nr; ++i)
      rmax = std::max(rmax, std::sqrt(h->rec[4 * i] * h->rec[4 * i] + h->rec[4 * i + 1] * h->rec[4 * i + 1] +
                                      h->rec[4 * i + 2] * h->rec[4 * i + 2]));
    std::vector<int> order(nr);
    std::iota(order.begin(), order.end(), 0);
    kd_chunks(h->rec, order, 0, nr);
    const int nc = (nr + BD_CHUNK - 1) / BD_CHUNK;
    std::vector<double> ra(4 * (size_t)nc * BD_CHUNK), cs(4 * (size_t)nc);
    for (int j = 0; j < nc * BD_CHUNK; ++j) {
      const int src = order[std::min(j, nr - 1)];
      for (int k = 0; k < 3; ++k) ra[4 * j + k] = h->rec[4 * src + k];
      ra[4 * j + 3] = j < nr ? h->rec[4 * src + 3] : 0.0;
    }
    for (int c = 0; c < nc; ++c) {
      double m[3] = {0, 0, 0};
      for (int a = 0; a < BD_CHUNK; ++a)
        for (int k = 0; k < 3; ++k) m[k] += ra[4 * (c * BD_CHUNK + a) + k] / BD_CHUNK;
      double r = 0;
      for (int a = 0; a < BD_CHUNK; ++a) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
          const double d = ra[4 * (c * BD_CHUNK + a) + k] - m[k];
          d2 += d * d;
        }
        r = std::max(r, std::sqrt(d2));
      }
      for (int k = 0; k < 3; ++k) cs[4 * c + k] = m[k];
      cs[4 * c + 3] = r * (1 + 1e-12) + 1e-9;  // conservative against rounding
    }
    void* p;
    int rc = dev_alloc(h, h->sys_allocs, &p, ra.size() * sizeof(double));
    if (rc) return rc;
    CK(h, cudaMemcpy(p, ra.data(), ra.size() * sizeof(double), cudaMemcpyHostToDevice));
    S.rec = (const double4*)p;
    rc = dev_alloc(h, h->sys_allocs, &p, cs.size() * sizeof(double));
    if (rc) return rc;
    CK(h, cudaMemcpy(p, cs.data(), cs.size() * sizeof(double), cudaMemcpyHostToDevice));
    S.chunks = (const double4*)p;
    S.n_chunks = nc;
    S.n_rec_pad = nc * BD_CHUNK;
    S.rec_max_r = rmax * (1 + 1e-12) + 1e-9;
    // FP32 copies for the stepper's shared-memory pre-tests (same order and chunking)
    std::vector<float> rf(ra.size()), cf(cs.size());
    for (size_t i = 0; i < ra.size(); ++i) rf[i] = (float)ra[i];
    for (size_t i = 0; i < cs.size(); ++i) cf[i] = (float)cs[i];
    rc = dev_alloc(h, h->sys_allocs, &p, rf.size() * sizeof(float));
    if (rc) return rc;
    CK(h, cudaMemcpy(p, rf.data(), rf.size() * sizeof(float), cudaMemcpyHostToDevice));
    S.rec_f = (const float4*)p;
    rc = dev_alloc(h, h->sys_allocs, &p, cf.size() * sizeof(float));
    if (rc) return rc;
    CK(h, cudaMemcpy(p, cf.data(), cf.size() * sizeof(float), cudaMemcpyHostToDevice));
    S.chunks_f = (const float4*)p;
    S.rec_in_smem = (h->layout & BD_LAYOUT_STAGE_RECEPTOR) &&
                    (size_t)(S.n_rec_pad + nc) * sizeof(float4) <= BD_STAGE_MAX_BYTES;
    if (h->layout & BD_LAYOUT_OVERLAP_GRID) {
      if ((rc = build_overlap_grid(h, S, ra, nr))) return rc;
    }
    // WCA radii in the same order; padding entries never come within a cutoff
    if (!h->rec_rad.empty()) {
      if (h->rec_rad.size() != (size_t)nr || h->lig_rad.size() != (size_t)nl)
        return fail(h, BD_ERR_ARG, "contact radii (%zu receptor, %zu ligand) do not match the atoms (%d, %d)",
                    h->rec_rad.size(), h->lig_rad.size(), nr, nl);
      std::vector<double> rd((size_t)nc * BD_CHUNK, -1e300);
      for (int j = 0; j < nr; ++j) rd[j] = h->rec_rad[order[j]];
      rc = dev_alloc(h, h->sys_allocs, &p, rd.size() * sizeof(double));
      if (rc) return rc;
      CK(h, cudaMemcpy(p, rd.data(), rd.size() * sizeof(double), cudaMemcpyHostToDevice));
      S.rec_rad = (const double*)p;
      rc = dev_alloc(h, h->sys_allocs, &p, h->lig_rad.size() * sizeof(double));
      if (rc) return rc;
      CK(h, cudaMemcpy(p, h->lig_rad.data(), h->lig_rad.size() * sizeof(double), cudaMemcpyHostToDevice));
      S.lig_rad = (const double*)p;
      const double mr = *std::max_element(h->rec_rad.begin(), h->rec_rad.end()),
                   ml = *std::max_element(h->lig_rad.begin(), h->lig_rad.end());
      S.wca = 1;
      S.wca_eps = h->wca_eps;
      // activation radius 2.5 x the largest sigma (gpu_batch_engine.py:241-242)
      S.wca_act = h->wca_act >= 0 ? h->wca_act : (mr + ml) * 2.5;
      S.wca_cut = std::max(0.0, kWcaCut * (mr + ml)) * (1 + 1e-12);
    }
  }
  if (!h->rec_rad.empty() && nr == 0) return fail(h, BD_ERR_ARG, "contact forces need the receptor atoms");
  // Born direction 2 needs the ligand Born grid, receptor atoms and alpha > 1e-12 (gpu_batch_engine.py:583-590)
  if (!lb.empty() && nr > 0 && fp.alpha > 1e-12) {
    const float* p;
    int rc = upload_floats(h, lb[0].data.data(), lb[0].data.size(), &p);
    if (rc) return rc;
    grid_to_dev(lb[0], p, 1, S.lig_born);
    if (h->layout & BD_LAYOUT_WINDOWS_1)
      if ((rc = add_window(h, S.lig_born))) return rc;
    if ((h->layout & BD_LAYOUT_CUBES_1) &&
        (double)S.lig_born.nx * S.lig_born.ny * S.lig_born.nz * 32.0 <= (double)BD_CUBE_MAX_BYTES)
      if ((rc = add_cube(h, S.lig_born))) return rc;
    if ((h->layout & BD_LAYOUT_XY_1) && S.lig_born.cube &&
        (double)S.lig_born.nx * S.lig_born.ny * S.lig_born.nz * 128.0 <= (double)BD_XY_MAX_BYTES)
      if ((rc = add_xy(h, S.lig_born, h->layout & BD_LAYOUT_XYTEX_1))) return rc;
    // linear textures address at most 2^27 elements
    if ((h->layout & BD_LAYOUT_ZTEX_1) && S.lig_born.cube &&
        (double)S.lig_born.nx * S.lig_born.ny * S.lig_born.nz * 2.0 <= (double)(1 << 27))
      if ((rc = add_ztex(h, S.lig_born))) return rc;
    S.born_rev = 1;
    const DevGrid& g = S.lig_born;
    const double mx = std::max(std::fabs(g.lox), std::fabs(g.hix)), my = std::max(std::fabs(g.loy), std::fabs(g.hiy)),
                 mz = std::max(std::fabs(g.loz), std::fabs(g.hiz));
    S.lig_born_rho = std::sqrt(mx * mx + my * my + mz * mz) * (1 + 1e-12) + 1e-9;
  }
  // reactions
  S.n_pairs = h->n_pairs;
  S.n_needed = h->n_needed;
  for (int p = 0; p < h->n_pairs; ++p) {
    for (int k = 0; k < 3; ++k) {
      S.rx_rec[p][k] = h->rx_rec[p][k];
      S.rx_body[p][k] = h->rx_body[p][k];
    }
    S.rx_cut[p] = h->rx_cut[p];
    S.rx_deff[p] = h->rx_deff[p];
  }
  if (h->sm_n > 0) {
    if (h->sm_n != h->n_pairs)
      return fail(h, BD_ERR_ARG, "state-machine reactions: %d reactions but %d reaction pairs (one pair each)",
                  h->sm_n, h->n_pairs);
    S.sm = 1;
    S.n_states = h->sm_states;
    S.terminal = h->sm_terminal;
    for (int p = 0; p < h->sm_n; ++p) {
      S.rx_before[p] = h->sm_before[p];
      S.rx_after[p] = h->sm_after[p];
    }
  }
  CK(h, cudaDeviceSynchronize());  // window copies are built on the legacy stream
  S.terms = h->terms;
  h->S = S;
  h->dirty = false;
  h->graph_K = -1;  // system changed: rebuild graphs
  return BD_OK;
}

// Stream arguments follow CUDA: NULL is the legacy default stream.  The handle's own
// stream is only used to capture the stepper's CUDA graphs.
cudaStream_t pick(BdHandle*, void* s) { return (cudaStream_t)s; }

// ---------------------------------------------------------------------------
// Kernel dispatch over (precision, group size, torque)
// ---------------------------------------------------------------------------
template <typename FT, int G, bool TQ>
struct K {
  static void* pose() { return (void*)&eval_pose_kernel<FT, G, TQ>; }
  static void* atoms() { return (void*)&eval_atoms_kernel<FT, G, TQ>; }
  static void* step() { return (void*)&step_kernel<FT, G, TQ>; }
};

template <typename FT, bool TQ>
void* pick_g(int G, int which) {
  if (G == BD_GROUP_SPLIT) {
    // the stepper's last phase sizes the slot pool; the parity kernels use a full-warp group
    if (which == 2) return (void*)&split_end_kernel<FT, TQ>;
    G = 32;
  }
  if (G == BD_GROUP_WARP || G == BD_GROUP_WARP_CAPPED) {
    // warp-cooperative stepper; the parity kernels use a full-warp group (same sweep code)
    if (which == 2)
      return G == BD_GROUP_WARP ? (void*)&step_kernel_warp<FT, TQ, 1> : (void*)&step_kernel_warp<FT, TQ, 2>;
    G = 32;
  }
  switch (G) {
#define BD_CASE(g)                                                  \
  case g:                                                           \
    return which == 0 ? K<FT, g, TQ>::pose() : which == 1 ? K<FT, g, TQ>::atoms() : K<FT, g, TQ>::step();
    BD_CASE(1)
    BD_CASE(4)
    BD_CASE(8)
    BD_CASE(16)
    BD_CASE(32)
#undef BD_CASE
  }
  return nullptr;
}

void* kernel_for(int prec, int G, int torque, int which) {
  const bool tq = torque == BD_TORQUE_CENTROID;
  if (prec == BD_PREC_FP64) return tq ? pick_g<double, true>(G, which) : pick_g<double, false>(G, which);
  return tq ? pick_g<float, true>(G, which) : pick_g<float, false>(G, which);
}

bool valid_group(int g) {
  return g == 1 || g == 4 || g == 8 || g == 16 || g == 32 || g == BD_GROUP_WARP || g == BD_GROUP_WARP_CAPPED ||
         g == BD_GROUP_SPLIT;
}

// Lanes that hold one trajectory's state (the warp-cooperative modes keep one per lane).
int lanes_per_traj(int g) {
  return (g == BD_GROUP_WARP || g == BD_GROUP_WARP_CAPPED || g == BD_GROUP_SPLIT) ? 1 : g;
}

// Tiny ligands with nothing to sweep: one lane per trajectory does everything.
// Otherwise the warp-cooperative mode.  The autotuner can override either.
int default_group(int n_lig_charged, bool sweeps_receptor) {
  if (!sweeps_receptor && n_lig_charged <= 2) return 1;
  return BD_GROUP_WARP;
}

int n_charged(const BdHandle* h) {
  int n = 0;
  for (size_t i = 0; i < h->lig.size() / 4; ++i) n += std::fabs(h->lig[4 * i + 3]) >= 1e-9;
  return n;
}

// Run constants of the stepper from the caller's parameters (pointers left null).
void sim_constants(const BdSimParams* p, const DevSystem& S, DevSim& P) {
  P = DevSim{};
  P.n_traj = p->n_traj;
  P.id_offset = p->id_offset;
  P.k0 = (uint32_t)(p->seed & 0xffffffffull);
  P.k1 = (uint32_t)(p->seed >> 32);
  P.r_b = p->r_start;
  P.r_esc = p->r_escape;
  P.return_prob = p->return_prob;
  P.max_steps = p->max_steps;
  P.max_dt = p->max_dt;
  P.min_core_dt = p->min_core_dt;
  P.min_core_rxn_dt = p->min_core_rxn_dt;
  P.use_hi = p->use_hi;
  P.overlap = p->overlap && S.n_chunks > 0;
  P.D_t = p->D_t;
  P.D_r = p->D_r;
  // adaptive dt force criterion: dielectric hard-coded to 78 (gpu_batch_simulator.py:622-629)
  P.adt_V0 = p->q_rec_total * p->q_lig_total / (4.0 * kPi * (78.0 * kEps0));
  P.adt_has_force = std::fabs(P.adt_V0) > 1e-9;
  P.adt_debye = p->adt_debye;
  P.adt_inv_debye = 1.0 / p->adt_debye;
  // HI constants, mu = 0.243 hard-coded (gpu_batch_simulator.py:741-751)
  P.hi_Df = 1.0 / 0.243;
  if (p->use_hi) {
    const double a0 = p->r_hydro_rec, a1 = p->r_hydro_lig;
    P.hi_a2 = 0.5 * (a0 * a0 + a1 * a1);
    P.hi_ainv = (P.hi_Df / (6.0 * kPi * a0) + P.hi_Df / (6.0 * kPi * a1)) / P.hi_Df;
  }
  // Zuk RPY coupling (hydrodynamics/rotne_prager.py:67-124)
  P.hi_mode = p->hi_mode;
  P.zuk_a = p->r_hydro_rec;
  P.zuk_b = p->r_hydro_lig;
  P.zuk_kTeta = p->hi_kT_eta;
}

// Launch group for a run with overlap rejection on or off: the autotuned or user
// choice, else the default for this system.
int launch_group_for(const BdHandle* h, int overlap) {
  if (h->launch_user) return h->group;
  const bool sweeps = h->S.born_rev || (overlap && !h->rec.empty());
  const int g = default_group(n_charged(h), sweeps);
  if (g != BD_GROUP_WARP) return g;
  // measured on the aged protein-ligand pool: the split step is fastest in mixed precision when
  // there is a reverse-Born sweep; otherwise the fused kernel with registers capped at 128
  return (h->S.born_rev && h->sp.precision == BD_PREC_MIXED) ? BD_GROUP_SPLIT : BD_GROUP_WARP_CAPPED;
}

int launch_group(const BdHandle* h) { return launch_group_for(h, h->sp.overlap); }

int eval_grid_blocks(BdHandle* h, long long n, int G, int block) {
  const long long groups = (n + 0);
  const long long per_block = block / G;
  long long blocks = (groups + per_block - 1) / per_block;
  blocks = std::min<long long>(blocks, (long long)h->n_sm * 64);
  return (int)std::max<long long>(blocks, 1);
}

int persistent_blocks(BdHandle* h, void* fn, int block, size_t smem = 0) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  return per_sm * h->n_sm;
}

// Dynamic shared memory of a stepper launch (block_shared_begin's layout): the
// staged FP32 receptor table, then the block's statistics histograms.  Raises the
// kernel's dynamic shared-memory limit to match, so occupancy queries and launches
// agree.
size_t stepper_smem(const DevSystem& S, const DevSim& P, void* fn) {
  size_t b = S.rec_in_smem ? (size_t)(S.n_rec_pad + S.n_chunks) * sizeof(float4) : 0;
  if (P.stats) b += (size_t)SH_NUM * sizeof(unsigned);
  if (fn) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b);
  return b;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* bd_version(void) { return "pystarc_b200 0.1.0 (sm_100a)"; }

int bd_create(int device, BdHandle** out) {
  if (!out) return fail(nullptr, BD_ERR_ARG, "out is NULL");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(nullptr, BD_ERR_CUDA, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
  if (device < 0 || device >= n) return fail(nullptr, BD_ERR_ARG, "device %d out of range (%d devices)", device, n);
  BdHandle* h = new BdHandle();
  h->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    fail(nullptr, BD_ERR_CUDA, "device setup: %s", cudaGetErrorString(e));
    delete h;
    return BD_ERR_CUDA;
  }
  *out = h;
  return BD_OK;
}

int bd_destroy(BdHandle* h) {
  if (!h) return BD_OK;
  cudaSetDevice(h->device);
  cudaDeviceSynchronize();
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  free_tex(h->sys_tex);
  free_list(h->sys_allocs);
  free_list(h->sim_allocs);
  if (h->own) cudaStreamDestroy(h->own);
  delete h;
  return BD_OK;
}

int bd_last_error(const BdHandle* h, char* buf, int len) {
  if (!buf || len <= 0) return BD_ERR_ARG;
  const std::string& s = h ? h->err : g_create_error;
  snprintf(buf, (size_t)len, "%s", s.c_str());
  return BD_OK;
}

int bd_set_ligand(BdHandle* h, int n, const double* xyz, const double* q) {
  if (!h || n <= 0 || !xyz || !q) return fail(h, BD_ERR_ARG, "bd_set_ligand: bad arguments");
  h->lig.assign(4 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) h->lig[4 * i + k] = xyz[3 * i + k];
    h->lig[4 * i + 3] = q[i];
    for (int k = 0; k < 4; ++k)
      if (!std::isfinite(h->lig[4 * i + k])) return fail(h, BD_ERR_NAN, "ligand atom %d is not finite", i);
  }
  h->dirty = true;
  return BD_OK;
}

int bd_set_receptor(BdHandle* h, int n, const double* xyz, const double* q) {
  if (!h || n < 0 || (n > 0 && (!xyz || !q))) return fail(h, BD_ERR_ARG, "bd_set_receptor: bad arguments");
  h->rec.assign(4 * (size_t)n, 0.0);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) h->rec[4 * i + k] = xyz[3 * i + k];
    h->rec[4 * i + 3] = q[i];
    for (int k = 0; k < 4; ++k)
      if (!std::isfinite(h->rec[4 * i + k])) return fail(h, BD_ERR_NAN, "receptor atom %d is not finite", i);
  }
  h->dirty = true;
  return BD_OK;
}

int bd_add_grid(BdHandle* h, int kind, const float* data, int nx, int ny, int nz, const double* origin,
                const double* spacing) {
  if (!h) return BD_ERR_ARG;
  if (kind < 0 || kind > 2 || !data || !origin || !spacing) return fail(h, BD_ERR_ARG, "bd_add_grid: bad arguments");
  if (nx < 8 || ny < 8 || nz < 8) return fail(h, BD_ERR_ARG, "grid %dx%dx%d: each axis needs >= 8 nodes", nx, ny, nz);
  if ((long long)nx * ny * nz > (1ll << 31) / 2) return fail(h, BD_ERR_ARG, "grid too large");
  GridHost g;
  g.n[0] = nx;
  g.n[1] = ny;
  g.n[2] = nz;
  for (int k = 0; k < 3; ++k) {
    g.o[k] = origin[k];
    g.sp[k] = spacing[k];
    if (!(spacing[k] > 0) || !std::isfinite(origin[k])) return fail(h, BD_ERR_ARG, "bad grid origin/spacing");
  }
  const size_t n = (size_t)nx * ny * nz;
  g.data.assign(data, data + n);
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(g.data[i])) return fail(h, BD_ERR_NAN, "grid value %zu is not finite", i);
  h->grids[kind].push_back(std::move(g));
  h->dirty = true;
  return BD_OK;
}

int bd_clear_grids(BdHandle* h) {
  if (!h) return BD_ERR_ARG;
  for (auto& v : h->grids) v.clear();
  h->dirty = true;
  return BD_OK;
}

int bd_set_force_params(BdHandle* h, const BdForceParams* p) {
  if (!h || !p) return fail(h, BD_ERR_ARG, "bd_set_force_params: NULL");
  if (p->use_multipole && !(p->four_pi_eps > 0)) return fail(h, BD_ERR_ARG, "four_pi_eps must be > 0");
  h->fp = *p;
  h->fp_set = true;
  h->dirty = true;
  return BD_OK;
}

int bd_set_reactions(BdHandle* h, int n_pairs, const double* rec_xyz, const double* lig_xyz, const double* cut,
                     const double* d_eff, int n_needed) {
  if (!h) return BD_ERR_ARG;
  if (n_pairs < 0 || n_pairs > BD_MAX_PAIRS) return fail(h, BD_ERR_ARG, "n_pairs must be in [0, %d]", BD_MAX_PAIRS);
  if (n_pairs > 0 && (!rec_xyz || !lig_xyz || !cut || !d_eff)) return fail(h, BD_ERR_ARG, "bd_set_reactions: NULL");
  h->n_pairs = n_pairs;
  h->n_needed = n_needed;
  for (int p = 0; p < n_pairs; ++p) {
    for (int k = 0; k < 3; ++k) {
      h->rx_rec[p][k] = rec_xyz[3 * p + k];
      h->rx_body[p][k] = lig_xyz[3 * p + k];
    }
    h->rx_cut[p] = cut[p];
    h->rx_deff[p] = d_eff[p];
  }
  h->dirty = true;
  return BD_OK;
}

int bd_eval_forces(BdHandle* h, int64_t n, const double* cen, const double* rot, int rot_is_matrix, double* F,
                   double* T, double* E, int prec, int torque, void* stream) {
  bd::NvtxRange nvtx("bd_eval_forces");
  if (!h) return BD_ERR_ARG;
  if (n < 0 || (n > 0 && (!cen || !rot || !F || !T || !E))) return fail(h, BD_ERR_ARG, "bd_eval_forces: bad arguments");
  if (prec != BD_PREC_FP64 && prec != BD_PREC_MIXED) return fail(h, BD_ERR_ARG, "bad precision %d", prec);
  if (torque != BD_TORQUE_ZERO && torque != BD_TORQUE_CENTROID) return fail(h, BD_ERR_ARG, "bad torque mode %d", torque);
  int rc = finalize(h);
  if (rc) return rc;
  if (n == 0) return BD_OK;
  const int G = launch_group(h);
  const int block = 128;
  void* fn = kernel_for(prec, G, torque, 0);
  unsigned long long* ctr = nullptr;
  long long nn = n;
  int rim = rot_is_matrix;
  void* args[] = {&h->S, &nn, &cen, &rot, &rim, &F, &T, &E, &ctr};
  CK(h, cudaLaunchKernel(fn, dim3(eval_grid_blocks(h, n, G, block)), dim3(block), args, 0, pick(h, stream)));
  return BD_OK;
}

int bd_eval_forces_atoms(BdHandle* h, int64_t n, const double* pos, const double* R, const double* cen, double* F,
                         double* T, double* E, int prec, int torque, void* stream) {
  bd::NvtxRange nvtx("bd_eval_forces_atoms");
  if (!h) return BD_ERR_ARG;
  if (n < 0 || (n > 0 && (!pos || !R || !cen || !F || !T || !E)))
    return fail(h, BD_ERR_ARG, "bd_eval_forces_atoms: bad arguments");
  if (prec != BD_PREC_FP64 && prec != BD_PREC_MIXED) return fail(h, BD_ERR_ARG, "bad precision %d", prec);
  if (torque != BD_TORQUE_ZERO && torque != BD_TORQUE_CENTROID) return fail(h, BD_ERR_ARG, "bad torque mode %d", torque);
  int rc = finalize(h);
  if (rc) return rc;
  if (n == 0) return BD_OK;
  const int G = launch_group(h);
  const int block = 128;
  void* fn = kernel_for(prec, G, torque, 1);
  long long nn = n;
  void* args[] = {&h->S, &nn, &pos, &R, &cen, &F, &T, &E};
  CK(h, cudaLaunchKernel(fn, dim3(eval_grid_blocks(h, n, G, block)), dim3(block), args, 0, pick(h, stream)));
  return BD_OK;
}

int bd_eval_overlap(BdHandle* h, int64_t n, const double* cen, int8_t* out, void* stream) {
  bd::NvtxRange nvtx("bd_eval_overlap");
  if (!h) return BD_ERR_ARG;
  if (n < 0 || (n > 0 && (!cen || !out))) return fail(h, BD_ERR_ARG, "bd_eval_overlap: bad arguments");
  int rc = finalize(h);
  if (rc) return rc;
  if (n == 0) return BD_OK;
  const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)h->n_sm * 16);
  eval_overlap_kernel<<<blocks, 256, 0, pick(h, stream)>>>(h->S, (long long)n, cen, out);
  CK(h, cudaGetLastError());
  return BD_OK;
}

int bd_set_launch(BdHandle* h, int group, int block) {
  if (!h) return BD_ERR_ARG;
  if (group && !valid_group(group)) return fail(h, BD_ERR_ARG, "group must be 1, 4, 8, 16, 32, 64 or 65 (warp-cooperative) or 66 (split)");
  if (block && (block % 32 || block < 32 || block > 256)) return fail(h, BD_ERR_ARG, "block must be 32..256, x32");
  if (group) h->group = group;
  if (block) h->block = block;
  h->launch_user = group != 0 || h->launch_user;
  h->graph_K = -1;
  return BD_OK;
}

int bd_set_layout(BdHandle* h, int flags) {
  if (!h) return BD_ERR_ARG;
  const int all = BD_LAYOUT_STAGE_RECEPTOR | BD_LAYOUT_WINDOWS_1 | BD_LAYOUT_WINDOWS_2 | BD_LAYOUT_CUBES_1 |
                  BD_LAYOUT_OVERLAP_GRID | BD_LAYOUT_XY_1 | BD_LAYOUT_ZTEX_1 | BD_LAYOUT_XYTEX_1 | BD_LAYOUT_PTEX_2;
  if (flags & ~all) return fail(h, BD_ERR_ARG, "unknown layout flags 0x%x", flags & ~all);
  if (flags != h->layout) {
    h->layout = flags;
    h->dirty = true;  // rebuilt by the next configure or evaluation
  }
  return BD_OK;
}

int bd_sim_set_surrogate(BdHandle* h, BdMlp* m, const BdSurrogateParams* p) {
  if (!h) return BD_ERR_ARG;
  h->graph_K = -1;  // the step sequence changes
  if (!m) {
    h->sur = nullptr;
    return BD_OK;
  }
  if (!p) return fail(h, BD_ERR_ARG, "bd_sim_set_surrogate: params are NULL");
  int in_dim, in_pad, out_dim;
  bd_internal_mlp_shape(m, &in_dim, &in_pad, &out_dim);
  if (in_dim != kSurIn || in_pad != kSurInPad || out_dim != kSurOut)
    return fail(h, BD_ERR_ARG, "the surrogate needs %d inputs and %d outputs (got %d, %d)", kSurIn, kSurOut, in_dim,
                out_dim);
  if (!(p->r_scale > 0) || !(p->rbf_width > 0) || !(p->threshold >= 0) || !(p->r_max >= p->r_min))
    return fail(h, BD_ERR_ARG, "bd_sim_set_surrogate: bad feature or trust-region constants");
  const int terms = p->terms ? p->terms : (BD_TERM_FARFIELD | BD_TERM_REV_BORN);
  if (terms & ~(BD_TERM_GRID | BD_TERM_FARFIELD | BD_TERM_REV_BORN))
    return fail(h, BD_ERR_ARG, "bd_sim_set_surrogate: terms %d outside grid | far-field | reverse Born", p->terms);
  DevSurrogate& q = h->sur_q;
  q.terms = (unsigned)terms;
  q.r_scale = p->r_scale;
  for (int k = 0; k < 5; ++k) q.rbf_centre[k] = p->rbf_centre[k];
  q.rbf_width = p->rbf_width;
  for (int k = 0; k < kSurOut; ++k) q.out_scale[k] = p->out_scale[k];
  q.r_min = p->r_min;
  q.r_max = p->r_max;
  q.threshold = p->threshold;
  q.force_floor = p->force_floor;
  q.env_r0 = p->env_r0;
  q.env_r1 = p->env_r1;
  for (int k = 0; k < kSurEnv; ++k) {
    if (!std::isfinite(p->env_log[k])) return fail(h, BD_ERR_ARG, "envelope entry %d is not finite", k);
    q.env_log[k] = p->env_log[k];
  }
  h->sur = m;
  return BD_OK;
}

int bd_sim_surrogate_counters(BdHandle* h, uint64_t* out) {
  if (!h || !out) return BD_ERR_ARG;
  out[0] = out[1] = 0;
  if (!h->sur || !h->sur_buf.ctr || !h->sur_cap) return BD_OK;
  CK(h, cudaDeviceSynchronize());
  CK(h, cudaMemcpy(out, h->sur_buf.ctr, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return BD_OK;
}

int bd_set_reaction_states(BdHandle* h, int n_pairs, const int32_t* state_before, const int32_t* state_after,
                           int n_states, const uint8_t* terminal) {
  if (!h) return BD_ERR_ARG;
  if (n_pairs < 0 || n_pairs > BD_MAX_PAIRS) return fail(h, BD_ERR_ARG, "n_pairs must be in [0, %d]", BD_MAX_PAIRS);
  if (n_pairs > 0 && (!state_before || !state_after || !terminal || n_states < 1 || n_states > 64))
    return fail(h, BD_ERR_ARG, "bd_set_reaction_states: bad arguments (1 <= n_states <= 64)");
  unsigned long long term = 0;
  for (int p = 0; p < n_pairs; ++p) {
    if (state_before[p] < -1 || state_before[p] >= n_states || state_after[p] < -1 || state_after[p] >= n_states)
      return fail(h, BD_ERR_ARG, "reaction %d: state index out of [-1, %d)", p, n_states);
    h->sm_before[p] = state_before[p];
    h->sm_after[p] = state_after[p];
  }
  for (int k = 0; k < n_states && n_pairs > 0; ++k)
    if (terminal[k]) term |= 1ull << k;
  h->sm_n = n_pairs;
  h->sm_states = n_pairs > 0 ? n_states : 0;
  h->sm_terminal = term;
  h->dirty = true;
  return BD_OK;
}

int bd_set_contact(BdHandle* h, int n_rec, const double* rec_radii, int n_lig, const double* lig_radii, double eps,
                   double activation) {
  if (!h) return BD_ERR_ARG;
  if (n_rec < 0 || n_lig < 0 || (n_rec > 0 && (!rec_radii || !lig_radii || n_lig == 0)))
    return fail(h, BD_ERR_ARG, "bd_set_contact: bad arguments");
  if (!std::isfinite(eps) || !std::isfinite(activation)) return fail(h, BD_ERR_NAN, "contact eps/activation not finite");
  h->rec_rad.clear();
  h->lig_rad.clear();
  if (n_rec > 0) {
    h->rec_rad.assign(rec_radii, rec_radii + n_rec);
    h->lig_rad.assign(lig_radii, lig_radii + n_lig);
    for (double r : h->rec_rad)
      if (!std::isfinite(r)) return fail(h, BD_ERR_NAN, "receptor radius is not finite");
    for (double r : h->lig_rad)
      if (!std::isfinite(r)) return fail(h, BD_ERR_NAN, "ligand radius is not finite");
  }
  h->wca_eps = eps;
  h->wca_act = activation;
  h->dirty = true;
  return BD_OK;
}

int bd_set_terms(BdHandle* h, int terms) {
  if (!h) return BD_ERR_ARG;
  if (terms < 0 || terms > BD_TERM_ALL) return fail(h, BD_ERR_ARG, "terms must be a mask of BD_TERM_* bits");
  h->terms = (unsigned)terms;
  h->S.terms = (unsigned)terms;  // evaluation kernels take S by value at launch
  return BD_OK;
}

int bd_get_layout(BdHandle* h, int* flags) {
  if (!h || !flags) return BD_ERR_ARG;
  *flags = h->layout;
  return BD_OK;
}

int bd_get_launch(BdHandle* h, int* group, int* block, int* grid) {
  if (!h) return BD_ERR_ARG;
  const int G = launch_group(h);
  if (group) *group = G;
  if (block) *block = h->block;
  if (grid) {
    void* fn = kernel_for(h->sp.precision, G, h->sp.torque_mode, 2);
    *grid = fn ? persistent_blocks(h, fn, h->block, stepper_smem(h->S, h->P, fn)) : 0;
  }
  return BD_OK;
}

int bd_sim_configure(BdHandle* h, const BdSimParams* p) {
  bd::NvtxRange nvtx("bd_sim_configure");
  if (!h || !p) return fail(h, BD_ERR_ARG, "bd_sim_configure: NULL");
  if (p->n_traj <= 0 || p->n_traj > 0x7ffffff0ll) return fail(h, BD_ERR_ARG, "n_traj out of range");
  if (p->id_offset < 0) return fail(h, BD_ERR_ARG, "id_offset must be >= 0");
  if (!(p->r_escape > p->r_start) || !(p->r_start > 0)) return fail(h, BD_ERR_ARG, "need 0 < r_start < r_escape");
  if (!(p->D_t > 0) || !(p->D_r >= 0)) return fail(h, BD_ERR_ARG, "diffusion coefficients must be positive");
  if (p->max_steps <= 0) return fail(h, BD_ERR_ARG, "max_steps must be positive");
  if (p->precision != BD_PREC_FP64 && p->precision != BD_PREC_MIXED) return fail(h, BD_ERR_ARG, "bad precision");
  if (p->torque_mode != BD_TORQUE_ZERO && p->torque_mode != BD_TORQUE_CENTROID) return fail(h, BD_ERR_ARG, "bad torque");
  if (p->use_hi && !(p->r_hydro_rec > 0 && p->r_hydro_lig > 0)) return fail(h, BD_ERR_ARG, "HI needs hydro radii");
  if (p->hi_mode != BD_HI_REFERENCE_GPU && p->hi_mode != BD_HI_ZUK) return fail(h, BD_ERR_ARG, "bad hi_mode");
  if (p->use_hi && p->hi_mode == BD_HI_ZUK && !(p->hi_kT_eta > 0))
    return fail(h, BD_ERR_ARG, "BD_HI_ZUK needs hi_kT_eta > 0");
  if (p->trace_capacity < 0 || (p->stats && p->trace_capacity > 0 && p->save_interval <= 0))
    return fail(h, BD_ERR_ARG, "traces need trace_capacity >= 0 and save_interval > 0");
  int rc = finalize(h);
  if (rc) return rc;
  CK(h, cudaSetDevice(h->device));
  CK(h, cudaDeviceSynchronize());
  free_list(h->sim_allocs);
  h->sim_ready = false;
  h->sur_cap = 0;
  h->sur_buf = SurBuf{};
  h->split_cap = 0;
  h->split_buf = SplitBuf{};
  h->sp = *p;
  // live-slot capacity
  const int G = launch_group(h);
  void* fn = kernel_for(p->precision, G, p->torque_mode, 2);
  DevSim probe{};
  probe.stats = p->stats;
  const long long resident =
      (long long)persistent_blocks(h, fn, h->block, stepper_smem(h->S, probe, fn)) * (h->block / lanes_per_traj(G));
  long long cap = p->slots > 0 ? p->slots : std::max<long long>(65536, 8 * resident);
  cap = std::min<long long>(cap, p->n_traj);
  const int C = (int)cap;
  for (int b = 0; b < 2; ++b) {
    SlotBuf& B = h->buf[b];
    void* q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, 3 * (size_t)C * sizeof(double)))) return rc;
    B.c = (double*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, 4 * (size_t)C * sizeof(double)))) return rc;
    B.q = (double*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(int)))) return rc;
    B.traj = (int*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(int)))) return rc;
    B.steps = (int*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(int)))) return rc;
    B.rets = (int*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
    B.status = (int8_t*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
    B.state = (int8_t*)q;
    B.cap = C;
  }
  void* q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 2 * sizeof(int)))) return rc;
  h->d_live = (int*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, C_NUM * sizeof(unsigned long long)))) return rc;
  h->d_ctr = (unsigned long long*)q;
  DevSim& P = h->P;
  sim_constants(p, h->S, P);
  P.ctr = h->d_ctr;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)p->n_traj))) return rc;
  P.out_status = (int8_t*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)p->n_traj * sizeof(int)))) return rc;
  P.out_steps = (int*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)p->n_traj * sizeof(int)))) return rc;
  P.out_returns = (int*)q;
  if (p->stats) {
    const size_t n = (size_t)p->n_traj;
    DevStats& st = P.st;
    auto dbl = [&](double** out, size_t k) {
      void* v;
      int r = dev_alloc(h, h->sim_allocs, &v, k * sizeof(double));
      *out = (double*)v;
      return r;
    };
    if ((rc = dbl(&st.start_c, 3 * n)) || (rc = dbl(&st.start_q, 4 * n)) || (rc = dbl(&st.min_dist, n)) ||
        (rc = dbl(&st.nm_c, 3 * n)) || (rc = dbl(&st.nm_q, 4 * n)) || (rc = dbl(&st.total_time, n)) ||
        (rc = dbl(&st.enc_c, 3 * n)) || (rc = dbl(&st.enc_q, 4 * n)))
      return rc;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, n * sizeof(int)))) return rc;
    st.step_at_min = (int*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, n * sizeof(int)))) return rc;
    st.enc_step = (int*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, n))) return rc;
    st.bridge = (int8_t*)q;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, SH_NUM * sizeof(unsigned long long)))) return rc;
    st.hist = (unsigned long long*)q;
    // bin edges as numpy.linspace builds them: start + i * (stop - start) / (num - 1), last = stop
    std::vector<double> edges(ST_RAD_BINS + 1 + ST_TRANS + 1 + ST_MILESTONES);
    const double top = p->r_escape * 1.2;
    for (int i = 0; i <= ST_RAD_BINS; ++i) edges[i] = i * (top / ST_RAD_BINS);
    edges[ST_RAD_BINS] = top;
    double* te = edges.data() + ST_RAD_BINS + 1;
    for (int i = 0; i <= ST_TRANS; ++i) te[i] = i * (top / ST_TRANS);
    te[ST_TRANS] = top;
    double* mr = te + ST_TRANS + 1;
    const double dm = (p->r_escape - p->r_start) / (ST_MILESTONES - 1);
    for (int i = 0; i < ST_MILESTONES; ++i) mr[i] = i * dm + p->r_start;
    mr[ST_MILESTONES - 1] = p->r_escape;
    if ((rc = dev_alloc(h, h->sim_allocs, &q, edges.size() * sizeof(double)))) return rc;
    CK(h, cudaMemcpy(q, edges.data(), edges.size() * sizeof(double), cudaMemcpyHostToDevice));
    st.rad_edges = (const double*)q;
    st.trans_edges = st.rad_edges + ST_RAD_BINS + 1;
    st.ms_radii = st.trans_edges + ST_TRANS + 1;
    P.stats = 1;
    if (p->trace_capacity > 0) {
      if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)p->trace_capacity * 8 * sizeof(double)))) return rc;
      P.trace_path = (double*)q;
      if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)p->trace_capacity * 6 * sizeof(double)))) return rc;
      P.trace_energy = (double*)q;
      P.trace_cap = p->trace_capacity;
      P.save_interval = p->save_interval;
    }
  }
  h->sim_ready = true;
  h->graph_K = -1;
  return BD_OK;
}

int bd_sim_reset(BdHandle* h, void* stream) {
  bd::NvtxRange nvtx("bd_sim_reset");
  if (!h) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "bd_sim_reset before bd_sim_configure");
  int rc = finalize(h);
  if (rc) return rc;
  cudaStream_t s = pick(h, stream);
  const int C = h->buf[0].cap;
  CK(h, cudaMemsetAsync(h->d_ctr, 0, C_NUM * sizeof(unsigned long long), s));
  CK(h, cudaMemsetAsync(h->P.out_status, 0, (size_t)h->P.n_traj, s));
  CK(h, cudaMemsetAsync(h->P.out_steps, 0, (size_t)h->P.n_traj * sizeof(int), s));
  CK(h, cudaMemsetAsync(h->P.out_returns, 0, (size_t)h->P.n_traj * sizeof(int), s));
  if (h->P.stats) {
    const DevStats& st = h->P.st;
    const size_t n = (size_t)h->P.n_traj;
    CK(h, cudaMemsetAsync(st.hist, 0, SH_NUM * sizeof(unsigned long long), s));
    CK(h, cudaMemsetAsync(st.total_time, 0, n * sizeof(double), s));
    CK(h, cudaMemsetAsync(st.step_at_min, 0, n * sizeof(int), s));
    CK(h, cudaMemsetAsync(st.enc_step, 0, n * sizeof(int), s));
    CK(h, cudaMemsetAsync(st.bridge, 0, n, s));
    CK(h, cudaMemsetAsync(st.nm_c, 0, 3 * n * sizeof(double), s));
    CK(h, cudaMemsetAsync(st.nm_q, 0, 4 * n * sizeof(double), s));
    CK(h, cudaMemsetAsync(st.enc_c, 0, 3 * n * sizeof(double), s));
    CK(h, cudaMemsetAsync(st.enc_q, 0, 4 * n * sizeof(double), s));
    const std::vector<double> far(n, 1e30);  // the reference starts min_dist at 1e30
    CK(h, cudaMemcpyAsync(st.min_dist, far.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(h, cudaStreamSynchronize(s));
  }
  init_slots_kernel<<<(C + 255) / 256, 256, 0, s>>>(h->P, h->buf[0], C);
  CK(h, cudaGetLastError());
  const unsigned long long started = (unsigned long long)C;
  CK(h, cudaMemcpyAsync(h->d_ctr + C_PENDING, &started, sizeof started, cudaMemcpyHostToDevice, s));
  CK(h, cudaMemcpyAsync(h->d_live, &C, sizeof C, cudaMemcpyHostToDevice, s));
  CK(h, cudaStreamSynchronize(s));
  h->cur = 0;
  return BD_OK;
}

namespace {

// One stepper launch plus the compaction into the other slot buffer.  `fn`,
// `smem` and `blocks` are fixed before stream capture starts.
int enqueue_launch(BdHandle* h, int K, cudaStream_t s, int cur, void* fn, size_t smem, int blocks) {
  SlotBuf src = h->buf[cur], dst = h->buf[1 - cur];
  const int* live = h->d_live + cur;
  int* live_dst = h->d_live + (1 - cur);
  void* args[] = {&h->S, &h->P, &src, &live, &K};
  CK(h, cudaLaunchKernel(fn, dim3(blocks), dim3(h->block), args, smem, s));
  compact_kernel<<<h->n_sm * 4, 256, 0, s>>>(src, dst, live, h->d_ctr);
  CK(h, cudaGetLastError());
  finish_compact_kernel<<<1, 1, 0, s>>>(live_dst, h->d_ctr);
  CK(h, cudaGetLastError());
  return BD_OK;
}

// Scratch of the surrogate stepper for the configured capacity (outside any capture).
int ensure_surrogate_buffers(BdHandle* h) {
  const int C = h->buf[0].cap;
  if (h->sur_cap == C) return BD_OK;
  SurBuf& U = h->sur_buf;
  void* q;
  int rc;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 3 * (size_t)C * sizeof(double)))) return rc;
  U.F = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 3 * (size_t)C * sizeof(double)))) return rc;
  U.T = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
  U.mode = (int8_t*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
  U.fresh = (int8_t*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(int)))) return rc;
  U.row = (int*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * kSurInPad * 2))) return rc;
  U.X = (__nv_bfloat16*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * kSurOut * sizeof(float)))) return rc;
  U.mean = (const float*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * kSurOut * sizeof(float)))) return rc;
  U.spread = (const float*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, sizeof(int)))) return rc;
  U.n_rows = (int*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 2 * sizeof(unsigned long long)))) return rc;
  U.ctr = (unsigned long long*)q;
  CK(h, cudaMemset(U.X, 0, (size_t)C * kSurInPad * 2));
  CK(h, cudaMemset(U.ctr, 0, 2 * sizeof(unsigned long long)));
  if ((rc = bd_internal_mlp_prepare(h->sur, C))) return fail(h, rc, "surrogate: %s", bd_internal_mlp_error(h->sur));
  h->sur_cap = C;
  return BD_OK;
}

extern "C++" {
template <typename FT, bool TQ>
int enqueue_surrogate_step(BdHandle* h, cudaStream_t s, int cur, int blocks) {
  SlotBuf B = h->buf[cur];
  const int* live = h->d_live + cur;
  SurBuf U = h->sur_buf;
  zero_int_kernel<<<1, 1, 0, s>>>(U.n_rows);
  sur_begin_kernel<FT, TQ><<<blocks, 256, 0, s>>>(h->S, h->P, B, live, U, h->sur_q);
  CK(h, cudaGetLastError());
  int rc = bd_internal_mlp_ensemble_rows(h->sur, h->sur_cap, U.n_rows, U.X, (float*)U.mean, (float*)U.spread, s);
  if (rc) return fail(h, rc, "surrogate: %s", bd_internal_mlp_error(h->sur));
  sur_end_kernel<FT, TQ><<<blocks, 256, 0, s>>>(h->S, h->P, B, live, U, h->sur_q);
  CK(h, cudaGetLastError());
  return BD_OK;
}
}  // extern "C++"

// K surrogate BD steps on buffer `cur`, then the compaction into the other buffer.
int enqueue_surrogate_launch(BdHandle* h, int K, cudaStream_t s, int cur, int blocks) {
  const bool tq = h->sp.torque_mode == BD_TORQUE_CENTROID, f64 = h->sp.precision == BD_PREC_FP64;
  // forces kept over rejected steps are per slot: the compaction between launches moves slots
  CK(h, cudaMemsetAsync(h->sur_buf.fresh, 0, (size_t)h->sur_cap, s));
  for (int k = 0; k < K; ++k) {
    int rc = f64 ? (tq ? enqueue_surrogate_step<double, true>(h, s, cur, blocks)
                       : enqueue_surrogate_step<double, false>(h, s, cur, blocks))
                 : (tq ? enqueue_surrogate_step<float, true>(h, s, cur, blocks)
                       : enqueue_surrogate_step<float, false>(h, s, cur, blocks));
    if (rc) return rc;
  }
  SlotBuf src = h->buf[cur], dst = h->buf[1 - cur];
  compact_kernel<<<h->n_sm * 4, 256, 0, s>>>(src, dst, h->d_live + cur, h->d_ctr);
  CK(h, cudaGetLastError());
  finish_compact_kernel<<<1, 1, 0, s>>>(h->d_live + (1 - cur), h->d_ctr);
  CK(h, cudaGetLastError());
  return BD_OK;
}

int surrogate_blocks(BdHandle* h) {
  const bool tq = h->sp.torque_mode == BD_TORQUE_CENTROID, f64 = h->sp.precision == BD_PREC_FP64;
  void* fa = f64 ? (tq ? (void*)&sur_begin_kernel<double, true> : (void*)&sur_begin_kernel<double, false>)
                 : (tq ? (void*)&sur_begin_kernel<float, true> : (void*)&sur_begin_kernel<float, false>);
  return persistent_blocks(h, fa, 256);
}

// Scratch of the split stepper for the configured capacity (outside any capture).
int ensure_split_buffers(BdHandle* h) {
  const int C = h->buf[0].cap;
  if (h->split_cap == C) return BD_OK;
  SplitBuf& U = h->split_buf;
  void* q;
  int rc;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 3 * (size_t)C * sizeof(double)))) return rc;
  U.F = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 3 * (size_t)C * sizeof(double)))) return rc;
  U.T = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 6 * (size_t)C * sizeof(double)))) return rc;
  U.rv = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(double)))) return rc;
  U.rprev = (double*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
  U.mode = (int8_t*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C))) return rc;
  U.fresh = (int8_t*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, (size_t)C * sizeof(int)))) return rc;
  U.list = (int*)q;
  if ((rc = dev_alloc(h, h->sim_allocs, &q, 2 * sizeof(int)))) return rc;
  U.cnt = (int*)q;
  h->split_cap = C;
  return BD_OK;
}

struct SplitKernels {
  void *begin, *rev, *end;
};

extern "C++" {
template <typename FT, bool TQ>
SplitKernels split_kernels_t() {
  return {(void*)&split_begin_kernel<FT, TQ>, (void*)&split_rev_kernel<FT, TQ>, (void*)&split_end_kernel<FT, TQ>};
}
}  // extern "C++"

SplitKernels split_kernels(int prec, int torque) {
  const bool tq = torque == BD_TORQUE_CENTROID;
  if (prec == BD_PREC_FP64) return tq ? split_kernels_t<double, true>() : split_kernels_t<double, false>();
  return tq ? split_kernels_t<float, true>() : split_kernels_t<float, false>();
}

// K split steps on buffer `cur` (three kernels each), then the compaction into the other buffer.
int enqueue_split_launch(BdHandle* h, int K, cudaStream_t s, int cur) {
  const SplitKernels kn = split_kernels(h->sp.precision, h->sp.torque_mode);
  const size_t smem = stepper_smem(h->S, h->P, kn.end);
  const int b_begin = persistent_blocks(h, kn.begin, 256), b_rev = persistent_blocks(h, kn.rev, 256),
            b_end = persistent_blocks(h, kn.end, 256, smem);
  SlotBuf src = h->buf[cur], dst = h->buf[1 - cur];
  const int* live = h->d_live + cur;
  SplitBuf U = h->split_buf;
  unsigned long long* ctr = h->d_ctr;
  // forces kept over rejected steps are per slot: the compaction between launches moves slots
  CK(h, cudaMemsetAsync(U.fresh, 0, (size_t)h->split_cap, s));
  for (int k = 0; k < K; ++k) {
    CK(h, cudaMemsetAsync(U.cnt, 0, 2 * sizeof(int), s));
    void* a_args[] = {&h->S, &h->P, &src, &live, &U};
    CK(h, cudaLaunchKernel(kn.begin, dim3(b_begin), dim3(256), a_args, 0, s));
    void* r_args[] = {&h->S, &src, &U, &ctr};
    CK(h, cudaLaunchKernel(kn.rev, dim3(b_rev), dim3(256), r_args, 0, s));
    void* e_args[] = {&h->S, &h->P, &src, &live, &U};
    CK(h, cudaLaunchKernel(kn.end, dim3(b_end), dim3(256), e_args, smem, s));
  }
  compact_kernel<<<h->n_sm * 4, 256, 0, s>>>(src, dst, live, h->d_ctr);
  CK(h, cudaGetLastError());
  finish_compact_kernel<<<1, 1, 0, s>>>(h->d_live + (1 - cur), h->d_ctr);
  CK(h, cudaGetLastError());
  return BD_OK;
}

int build_graphs(BdHandle* h, int K) {
  const int G = launch_group(h);
  if (h->graph_K == K && h->graph_G == G && h->graph_B == h->block && h->graph_prec == h->sp.precision &&
      h->graph_torque == h->sp.torque_mode)
    return BD_OK;
  for (auto& g : h->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  void* fn = kernel_for(h->sp.precision, G, h->sp.torque_mode, 2);
  const size_t smem = stepper_smem(h->S, h->P, fn);
  const int blocks = persistent_blocks(h, fn, h->block, smem);
  const int sblocks = h->sur ? surrogate_blocks(h) : 0;
  if (h->sur) {
    int rc = ensure_surrogate_buffers(h);
    if (rc) return rc;
  }
  const bool split = !h->sur && G == BD_GROUP_SPLIT;
  if (split) {
    int rc = ensure_split_buffers(h);
    if (rc) return rc;
  }
  for (int c = 0; c < 2; ++c) {
    cudaGraph_t graph;
    CK(h, cudaStreamBeginCapture(h->own, cudaStreamCaptureModeThreadLocal));
    int rc = h->sur ? enqueue_surrogate_launch(h, K, h->own, c, sblocks)
             : split ? enqueue_split_launch(h, K, h->own, c)
                     : enqueue_launch(h, K, h->own, c, fn, smem, blocks);
    cudaError_t e = cudaStreamEndCapture(h->own, &graph);
    if (rc) return rc;
    CK(h, e);
    e = cudaGraphInstantiate(&h->graph[c], graph, 0);
    cudaGraphDestroy(graph);
    CK(h, e);
  }
  h->graph_K = K;
  h->graph_G = G;
  h->graph_B = h->block;
  h->graph_prec = h->sp.precision;
  h->graph_torque = h->sp.torque_mode;
  return BD_OK;
}

}  // namespace

int bd_sim_run(BdHandle* h, int n_launch, int K, void* stream) {
  bd::NvtxRange nvtx("bd_sim_run");
  if (!h) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "bd_sim_run before bd_sim_configure");
  if (n_launch < 0 || K <= 0) return fail(h, BD_ERR_ARG, "bd_sim_run: n_launch >= 0 and steps > 0 needed");
  if (h->dirty) return fail(h, BD_ERR_STATE, "system changed after bd_sim_reset; reset again");
  if (h->sur && h->P.stats) return fail(h, BD_ERR_STATE, "per-step statistics are not collected by the surrogate stepper");
  int rc = build_graphs(h, K);
  if (rc) return rc;
  cudaStream_t s = pick(h, stream);
  for (int i = 0; i < n_launch; ++i) {
    CK(h, cudaGraphLaunch(h->graph[h->cur], s));
    h->cur = 1 - h->cur;
  }
  return BD_OK;
}

int bd_sim_counters(BdHandle* h, uint64_t* out, int n, void* stream) {
  if (!h || !out) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  unsigned long long c[C_NUM];
  cudaStream_t s = pick(h, stream);
  CK(h, cudaMemcpyAsync(c, h->d_ctr, sizeof c, cudaMemcpyDeviceToHost, s));
  CK(h, cudaStreamSynchronize(s));
  const int m = std::min(n, (int)BD_CTR_NUM);
  for (int i = 0; i < m; ++i) out[i] = c[i];
  if (m > 0) out[0] = std::min<unsigned long long>(c[C_PENDING], (unsigned long long)h->P.n_traj);
  return BD_OK;
}

int bd_sim_outcomes(BdHandle* h, int8_t* status, int32_t* steps, int32_t* rets) {
  if (!h) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  const size_t n = (size_t)h->P.n_traj;
  if (status) CK(h, cudaMemcpy(status, h->P.out_status, n, cudaMemcpyDeviceToHost));
  if (steps) CK(h, cudaMemcpy(steps, h->P.out_steps, n * sizeof(int), cudaMemcpyDeviceToHost));
  if (rets) CK(h, cudaMemcpy(rets, h->P.out_returns, n * sizeof(int), cudaMemcpyDeviceToHost));
  return BD_OK;
}

int bd_sim_stats(BdHandle* h, const BdStatsOut* o) {
  if (!h || !o) return fail(h, BD_ERR_ARG, "bd_sim_stats: NULL");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  if (!h->P.stats) return fail(h, BD_ERR_STATE, "statistics were not requested (BdSimParams.stats = 0)");
  CK(h, cudaDeviceSynchronize());
  const DevStats& st = h->P.st;
  const size_t n = (size_t)h->P.n_traj;
  auto get = [&](void* dst, const void* src, size_t bytes) -> int {
    if (dst) CK(h, cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return BD_OK;
  };
  int rc = 0;
  if ((rc = get(o->start_pos, st.start_c, 3 * n * 8)) || (rc = get(o->start_q, st.start_q, 4 * n * 8)) ||
      (rc = get(o->min_dist, st.min_dist, n * 8)) || (rc = get(o->near_miss_pos, st.nm_c, 3 * n * 8)) ||
      (rc = get(o->near_miss_q, st.nm_q, 4 * n * 8)) || (rc = get(o->total_time, st.total_time, n * 8)) ||
      (rc = get(o->encounter_pos, st.enc_c, 3 * n * 8)) || (rc = get(o->encounter_q, st.enc_q, 4 * n * 8)) ||
      (rc = get(o->step_at_min, st.step_at_min, n * 4)) || (rc = get(o->encounter_step, st.enc_step, n * 4)) ||
      (rc = get(o->bridge, st.bridge, n)))
    return rc;
  std::vector<unsigned long long> hist(SH_NUM);
  CK(h, cudaMemcpy(hist.data(), st.hist, SH_NUM * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  auto put = [&](uint64_t* dst, int off, int cnt) {
    if (dst)
      for (int i = 0; i < cnt; ++i) dst[i] = hist[off + i];
  };
  put(o->radial, SH_RAD, ST_RAD_BINS);
  put(o->angular, SH_ANG, ST_THETA * ST_PHI);
  put(o->milestone_out, SH_MS_OUT, ST_MILESTONES);
  put(o->milestone_in, SH_MS_IN, ST_MILESTONES);
  put(o->transition, SH_TRANS, ST_TRANS * ST_TRANS);
  put(o->contact, SH_CONTACT, h->S.n_pairs);
  if ((rc = get(o->radial_edges, st.rad_edges, (ST_RAD_BINS + 1) * 8)) ||
      (rc = get(o->transition_edges, st.trans_edges, (ST_TRANS + 1) * 8)) ||
      (rc = get(o->milestone_radii, st.ms_radii, ST_MILESTONES * 8)))
    return rc;
  return BD_OK;
}

int bd_sim_live(BdHandle* h, int32_t* n_live) {
  if (!h || !n_live) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  CK(h, cudaMemcpy(n_live, h->d_live + h->cur, sizeof(int), cudaMemcpyDeviceToHost));
  return BD_OK;
}

int bd_sim_traces(BdHandle* h, double* path, double* energy, int64_t cap, int64_t* n_rows, int64_t* n_dropped) {
  if (!h || !n_rows || !n_dropped || cap < 0) return fail(h, BD_ERR_ARG, "bd_sim_traces: bad arguments");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  *n_rows = 0;
  *n_dropped = 0;
  if (!h->P.stats || h->P.trace_cap <= 0) return BD_OK;
  CK(h, cudaSetDevice(h->device));
  CK(h, cudaDeviceSynchronize());
  unsigned long long claimed = 0;
  CK(h, cudaMemcpy(&claimed, h->d_ctr + C_TRACE, sizeof claimed, cudaMemcpyDeviceToHost));
  const long long kept = std::min<long long>((long long)claimed, h->P.trace_cap);
  const long long n = std::min<long long>(kept, cap);
  if (path && n > 0) CK(h, cudaMemcpy(path, h->P.trace_path, (size_t)n * 8 * sizeof(double), cudaMemcpyDeviceToHost));
  if (energy && n > 0)
    CK(h, cudaMemcpy(energy, h->P.trace_energy, (size_t)n * 6 * sizeof(double), cudaMemcpyDeviceToHost));
  *n_rows = n;
  *n_dropped = (long long)claimed - kept;
  return BD_OK;
}

int bd_sim_hi_diffusion(BdHandle* h, int n, const double* r, double* D) {
  if (!h || (n > 0 && (!r || !D)) || n < 0) return fail(h, BD_ERR_ARG, "bd_sim_hi_diffusion: bad arguments");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  if (n == 0) return BD_OK;
  CK(h, cudaSetDevice(h->device));
  std::vector<void*> tmp;
  void *dr, *dD;
  int rc;
  if ((rc = dev_alloc(h, tmp, &dr, (size_t)n * sizeof(double))) || (rc = dev_alloc(h, tmp, &dD, (size_t)n * sizeof(double)))) {
    free_list(tmp);
    return rc;
  }
  cudaError_t e = cudaMemcpy(dr, r, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (h->sp.precision == BD_PREC_FP64)
      hi_diffusion_kernel<double><<<(n + 255) / 256, 256>>>(h->P, n, (const double*)dr, (double*)dD);
    else
      hi_diffusion_kernel<float><<<(n + 255) / 256, 256>>>(h->P, n, (const double*)dr, (double*)dD);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(D, dD, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  free_list(tmp);
  CK(h, e);
  return BD_OK;
}

int bd_sim_capacity(BdHandle* h, int32_t* cap) {
  if (!h || !cap) return BD_ERR_ARG;
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  *cap = h->buf[0].cap;
  return BD_OK;
}

int bd_sim_reaction_fires(BdHandle* h, uint64_t* discrete, uint64_t* bridge, int n) {
  if (!h || n < 0 || n > BD_MAX_PAIRS || (n > 0 && (!discrete || !bridge)))
    return fail(h, BD_ERR_ARG, "bd_sim_reaction_fires: bad arguments");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  unsigned long long ctr[C_NUM];
  CK(h, cudaMemcpy(ctr, h->d_ctr, sizeof ctr, cudaMemcpyDeviceToHost));
  for (int p = 0; p < n; ++p) {
    discrete[p] = ctr[C_SM_DISCRETE + p];
    bridge[p] = ctr[C_SM_BRIDGE + p];
  }
  return BD_OK;
}

int bd_sim_get_states(BdHandle* h, int8_t* state) {
  if (!h || !state) return fail(h, BD_ERR_ARG, "bd_sim_get_states: NULL");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  const SlotBuf& B = h->buf[h->cur];
  CK(h, cudaMemcpy(state, B.state, (size_t)B.cap, cudaMemcpyDeviceToHost));
  return BD_OK;
}

int bd_sim_set_states(BdHandle* h, const int8_t* state) {
  if (!h || !state) return fail(h, BD_ERR_ARG, "bd_sim_set_states: NULL");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  const SlotBuf& B = h->buf[h->cur];
  CK(h, cudaMemcpy(B.state, state, (size_t)B.cap, cudaMemcpyHostToDevice));
  return BD_OK;
}

int bd_sim_snapshot(BdHandle* h, double* c, double* q, int32_t* traj, int32_t* steps, int32_t* rets, int8_t* status,
                    int32_t* n_live, uint64_t* counters) {
  if (!h || !c || !q || !traj || !steps || !rets || !status || !n_live || !counters)
    return fail(h, BD_ERR_ARG, "bd_sim_snapshot: NULL");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  CK(h, cudaDeviceSynchronize());
  const SlotBuf& B = h->buf[h->cur];
  const size_t C = (size_t)B.cap;
  CK(h, cudaMemcpy(c, B.c, 3 * C * sizeof(double), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(q, B.q, 4 * C * sizeof(double), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(traj, B.traj, C * sizeof(int), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(steps, B.steps, C * sizeof(int), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(rets, B.rets, C * sizeof(int), cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(status, B.status, C, cudaMemcpyDeviceToHost));
  CK(h, cudaMemcpy(n_live, h->d_live + h->cur, sizeof(int), cudaMemcpyDeviceToHost));
  unsigned long long ctr[C_NUM];
  CK(h, cudaMemcpy(ctr, h->d_ctr, sizeof ctr, cudaMemcpyDeviceToHost));
  for (int i = 0; i < BD_CTR_NUM; ++i) counters[i] = ctr[i];
  return BD_OK;
}

int bd_sim_restore(BdHandle* h, const double* c, const double* q, const int32_t* traj, const int32_t* steps,
                   const int32_t* rets, const int8_t* status, int32_t n_live, const uint64_t* counters,
                   const int8_t* out_status, const int32_t* out_steps, const int32_t* out_returns) {
  if (!h || !c || !q || !traj || !steps || !rets || !status || !counters || !out_status || !out_steps || !out_returns)
    return fail(h, BD_ERR_ARG, "bd_sim_restore: NULL");
  if (!h->sim_ready) return fail(h, BD_ERR_STATE, "no simulation configured");
  int rc = finalize(h);
  if (rc) return rc;
  const SlotBuf& B = h->buf[0];
  const size_t C = (size_t)B.cap;
  if (n_live < 0 || (size_t)n_live > C) return fail(h, BD_ERR_ARG, "n_live out of range");
  CK(h, cudaDeviceSynchronize());
  CK(h, cudaMemcpy(B.c, c, 3 * C * sizeof(double), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(B.q, q, 4 * C * sizeof(double), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(B.traj, traj, C * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(B.steps, steps, C * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(B.rets, rets, C * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(B.status, status, C, cudaMemcpyHostToDevice));
  unsigned long long ctr[C_NUM] = {0};
  for (int i = 0; i < BD_CTR_NUM; ++i) ctr[i] = counters[i];
  ctr[C_SLOT_CURSOR] = 0;
  ctr[C_LIVE_NEXT] = 0;
  CK(h, cudaMemcpy(h->d_ctr, ctr, sizeof ctr, cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->d_live, &n_live, sizeof(int), cudaMemcpyHostToDevice));
  const size_t n = (size_t)h->P.n_traj;
  CK(h, cudaMemcpy(h->P.out_status, out_status, n, cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->P.out_steps, out_steps, n * sizeof(int), cudaMemcpyHostToDevice));
  CK(h, cudaMemcpy(h->P.out_returns, out_returns, n * sizeof(int), cudaMemcpyHostToDevice));
  h->cur = 0;
  return BD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free run, called by bd_sim_run_noalloc (bd_noalloc.cu) with the
// address of its static device scratch array.  Nothing here allocates device
// memory: the live-slot pool, live counts and counters are carved from
// `scratch`; per-trajectory outputs and the final counters go to caller arrays.
// ---------------------------------------------------------------------------
namespace {

unsigned char* carve(unsigned char*& p, size_t bytes) {
  unsigned char* out = p;
  p += (bytes + 255) & ~(size_t)255;
  return out;
}

}  // namespace

int bd_internal_device(const BdHandle* h) { return h ? h->device : -1; }

int bd_internal_fail(BdHandle* h, int code, const char* msg) { return fail(h, code, "%s", msg); }

int bd_internal_run_noalloc(BdHandle* h, const BdSimParams* p, unsigned char* scratch, size_t scratch_bytes,
                            int max_slots, int8_t* out_status, int32_t* out_steps, int32_t* out_returns,
                            uint64_t* counters, int K, int max_launches, cudaStream_t s) {
  if (!h) return BD_ERR_ARG;
  if (!p || !out_status || !out_steps || !out_returns || !counters)
    return fail(h, BD_ERR_ARG, "bd_sim_run_noalloc: NULL argument");
  if (p->n_traj <= 0 || p->n_traj > 0x7ffffff0ll) return fail(h, BD_ERR_ARG, "n_traj out of range");
  if (p->id_offset < 0) return fail(h, BD_ERR_ARG, "id_offset must be >= 0");
  if (!(p->r_escape > p->r_start) || !(p->r_start > 0)) return fail(h, BD_ERR_ARG, "need 0 < r_start < r_escape");
  if (!(p->D_t > 0) || !(p->D_r >= 0)) return fail(h, BD_ERR_ARG, "diffusion coefficients must be positive");
  if (p->max_steps <= 0) return fail(h, BD_ERR_ARG, "max_steps must be positive");
  if (p->precision != BD_PREC_FP64 && p->precision != BD_PREC_MIXED) return fail(h, BD_ERR_ARG, "bad precision");
  if (p->torque_mode != BD_TORQUE_ZERO && p->torque_mode != BD_TORQUE_CENTROID) return fail(h, BD_ERR_ARG, "bad torque");
  if (p->use_hi && !(p->r_hydro_rec > 0 && p->r_hydro_lig > 0)) return fail(h, BD_ERR_ARG, "HI needs hydro radii");
  if (p->hi_mode != BD_HI_REFERENCE_GPU && p->hi_mode != BD_HI_ZUK) return fail(h, BD_ERR_ARG, "bad hi_mode");
  if (p->use_hi && p->hi_mode == BD_HI_ZUK && !(p->hi_kT_eta > 0))
    return fail(h, BD_ERR_ARG, "BD_HI_ZUK needs hi_kT_eta > 0");
  if (K <= 0 || max_launches <= 0) return fail(h, BD_ERR_ARG, "steps_per_launch and max_launches must be > 0");
  if (p->slots > max_slots)
    return fail(h, BD_ERR_ARG, "bd_sim_run_noalloc: %d slots requested, the static scratch holds at most %d",
                p->slots, max_slots);
  if (h->dirty)
    return fail(h, BD_ERR_STATE,
                "bd_sim_run_noalloc: the system is not on the device yet; its upload allocates, so call "
                "bd_sim_configure or an evaluation once before");
  if (h->sur)
    return fail(h, BD_ERR_STATE,
                "bd_sim_run_noalloc runs the exact-force stepper only; remove the surrogate "
                "(bd_sim_set_surrogate with NULL) first");
  CK(h, cudaSetDevice(h->device));
  const int C = (int)std::min<long long>(p->slots > 0 ? p->slots : max_slots, p->n_traj);
  // scratch layout: two slot buffers, two live counts, the counters
  unsigned char* cur_p = scratch;
  SlotBuf B[2];
  for (int b = 0; b < 2; ++b) {
    B[b].c = (double*)carve(cur_p, 3 * (size_t)C * sizeof(double));
    B[b].q = (double*)carve(cur_p, 4 * (size_t)C * sizeof(double));
    B[b].traj = (int*)carve(cur_p, (size_t)C * sizeof(int));
    B[b].steps = (int*)carve(cur_p, (size_t)C * sizeof(int));
    B[b].rets = (int*)carve(cur_p, (size_t)C * sizeof(int));
    B[b].status = (int8_t*)carve(cur_p, (size_t)C);
    B[b].state = (int8_t*)carve(cur_p, (size_t)C);
    B[b].cap = C;
  }
  int* live = (int*)carve(cur_p, 2 * sizeof(int));
  unsigned long long* ctr = (unsigned long long*)carve(cur_p, C_NUM * sizeof(unsigned long long));
  if ((size_t)(cur_p - scratch) > scratch_bytes) return fail(h, BD_ERR_ARG, "scratch layout exceeds the array");
  DevSim P{};
  sim_constants(p, h->S, P);
  P.ctr = ctr;
  P.out_status = out_status;
  P.out_steps = out_steps;
  P.out_returns = out_returns;
  // the array keeps the previous call's contents: zero the counters and the outputs
  CK(h, cudaMemsetAsync(ctr, 0, C_NUM * sizeof(unsigned long long), s));
  CK(h, cudaMemsetAsync(out_status, 0, (size_t)p->n_traj, s));
  CK(h, cudaMemsetAsync(out_steps, 0, (size_t)p->n_traj * sizeof(int), s));
  CK(h, cudaMemsetAsync(out_returns, 0, (size_t)p->n_traj * sizeof(int), s));
  init_slots_kernel<<<(C + 255) / 256, 256, 0, s>>>(P, B[0], C);
  CK(h, cudaGetLastError());
  unsigned long long started = (unsigned long long)C;
  int c_live = C;
  CK(h, cudaMemcpyAsync(ctr + C_PENDING, &started, sizeof started, cudaMemcpyHostToDevice, s));
  CK(h, cudaMemcpyAsync(live, &c_live, sizeof c_live, cudaMemcpyHostToDevice, s));
  CK(h, cudaStreamSynchronize(s));
  int G = launch_group_for(h, p->overlap);
  if (G == BD_GROUP_SPLIT) G = BD_GROUP_WARP_CAPPED;  // the split stepper's scratch would need allocating
  void* fn = kernel_for(p->precision, G, p->torque_mode, 2);
  const size_t smem = stepper_smem(h->S, P, fn);
  const int blocks = persistent_blocks(h, fn, h->block, smem);
  int cur = 0;
  for (int launch = 0; launch < max_launches; ++launch) {
    SlotBuf src = B[cur], dst = B[1 - cur];
    const int* lsrc = live + cur;
    int* ldst = live + (1 - cur);
    int KK = K;
    void* args[] = {&h->S, &P, &src, &lsrc, &KK};
    CK(h, cudaLaunchKernel(fn, dim3(blocks), dim3(h->block), args, smem, s));
    compact_kernel<<<h->n_sm * 4, 256, 0, s>>>(src, dst, lsrc, ctr);
    CK(h, cudaGetLastError());
    finish_compact_kernel<<<1, 1, 0, s>>>(ldst, ctr);
    CK(h, cudaGetLastError());
    cur = 1 - cur;
    if ((launch & 3) == 3 || launch == max_launches - 1) {
      unsigned long long c[C_NUM];
      int n_live = 0;
      CK(h, cudaMemcpyAsync(c, ctr, sizeof c, cudaMemcpyDeviceToHost, s));
      CK(h, cudaMemcpyAsync(&n_live, live + cur, sizeof n_live, cudaMemcpyDeviceToHost, s));
      CK(h, cudaStreamSynchronize(s));
      if (n_live == 0 && c[C_PENDING] >= (unsigned long long)p->n_traj) break;
    }
  }
  unsigned long long c[C_NUM];
  CK(h, cudaMemcpyAsync(c, ctr, sizeof c, cudaMemcpyDeviceToHost, s));
  CK(h, cudaStreamSynchronize(s));
  c[C_PENDING] = std::min<unsigned long long>(c[C_PENDING], (unsigned long long)p->n_traj);  // trajectories started
  CK(h, cudaMemcpyAsync(counters, c, BD_CTR_NUM * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  CK(h, cudaStreamSynchronize(s));
  return BD_OK;
}

// ===========================================================================
// Heterogeneous batch (bd_multi_*): several configured handles in one pool.
// ===========================================================================
struct BdMulti {
  int device = 0, n_sm = 148;
  std::vector<BdHandle*> hs;
  int precision = BD_PREC_MIXED, torque = BD_TORQUE_ZERO;
  MultiTab T{};
  SlotBuf buf[2]{};
  int* d_live = nullptr;
  int cap = 0, cur = 0, blocks = 0;
  std::vector<void*> allocs;
  cudaStream_t own = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_K = -1;
  std::string err;
};

namespace {

int mfail(BdMulti* m, int code, const char* fmt, ...) {
  char b[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(b, sizeof b, fmt, ap);
  va_end(ap);
  if (m) m->err = b;
  return code;
}

#define MCK(m, x)                                                                                      \
  do {                                                                                                 \
    cudaError_t e_ = (x);                                                                              \
    if (e_ != cudaSuccess)                                                                             \
      return mfail(m, e_ == cudaErrorMemoryAllocation ? BD_ERR_OOM : BD_ERR_CUDA, "%s: %s (%s:%d)", #x, \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                                        \
  } while (0)

int malloc_multi(BdMulti* m, void** p, size_t bytes) {
  MCK(m, cudaMalloc(p, bytes ? bytes : 16));
  m->allocs.push_back(*p);
  return BD_OK;
}

void* multi_kernel(int prec, int torque) {
  const bool tq = torque == BD_TORQUE_CENTROID;
  if (prec == BD_PREC_FP64) return tq ? (void*)&step_kernel_multi<double, true> : (void*)&step_kernel_multi<double, false>;
  return tq ? (void*)&step_kernel_multi<float, true> : (void*)&step_kernel_multi<float, false>;
}

int multi_graphs(BdMulti* m, int K) {
  if (m->graph_K == K) return BD_OK;
  for (auto& g : m->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  void* fn = multi_kernel(m->precision, m->torque);
  for (int c = 0; c < 2; ++c) {
    cudaGraph_t graph;
    MCK(m, cudaStreamBeginCapture(m->own, cudaStreamCaptureModeThreadLocal));
    SlotBuf src = m->buf[c], dst = m->buf[1 - c];
    const int* live = m->d_live + c;
    int KK = K;
    MultiTab T = m->T;
    void* args[] = {&T, &src, &live, &KK};
    cudaError_t e = cudaLaunchKernel(fn, dim3(m->blocks), dim3(256), args, 0, m->own);
    if (e == cudaSuccess) {
      compact_kernel<<<m->n_sm * 4, 256, 0, m->own>>>(src, dst, live, m->T.ctr);
      finish_compact_kernel<<<1, 1, 0, m->own>>>(m->d_live + (1 - c), m->T.ctr);
      e = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamEndCapture(m->own, &graph);
    MCK(m, e);
    MCK(m, e2);
    e = cudaGraphInstantiate(&m->graph[c], graph, 0);
    cudaGraphDestroy(graph);
    MCK(m, e);
  }
  m->graph_K = K;
  return BD_OK;
}

}  // namespace

extern "C" {

int bd_multi_create(BdHandle* const* handles, int n, BdMulti** out) {
  if (!out) return BD_ERR_ARG;
  *out = nullptr;
  if (!handles || n < 1 || n > 1024) return BD_ERR_ARG;
  BdMulti* m = new BdMulti();
  auto bail = [&](int rc) {
    for (void* p : m->allocs) cudaFree(p);
    if (m->own) cudaStreamDestroy(m->own);
    g_create_error = m->err;
    delete m;
    return rc;
  };
  m->device = handles[0] ? handles[0]->device : 0;
  std::vector<DevSystem> sys(n);
  std::vector<DevSim> sim(n);
  std::vector<long long> base(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    BdHandle* h = handles[i];
    if (!h || !h->sim_ready || h->dirty)
      return bail(mfail(m, BD_ERR_STATE, "handle %d is not configured (bd_sim_configure after its last change)", i));
    if (h->device != m->device) return bail(mfail(m, BD_ERR_ARG, "handle %d is on another device", i));
    if (i == 0) {
      m->precision = h->sp.precision;
      m->torque = h->sp.torque_mode;
    } else if (h->sp.precision != m->precision || h->sp.torque_mode != m->torque) {
      return bail(mfail(m, BD_ERR_ARG, "handle %d: every system needs the same precision and torque mode", i));
    }
    if (h->sur) return bail(mfail(m, BD_ERR_ARG, "handle %d has a surrogate; the batch runs the exact kernels", i));
    sys[i] = h->S;
    sys[i].rec_in_smem = 0;
    sim[i] = h->P;
    sim[i].stats = 0;
    base[i + 1] = base[i] + h->P.n_traj;
  }
  if (base[n] > 0x7fffffffll) return bail(mfail(m, BD_ERR_ARG, "more than 2^31 - 1 trajectories in the batch"));
  if (cudaSetDevice(m->device) != cudaSuccess) return bail(mfail(m, BD_ERR_CUDA, "cudaSetDevice failed"));
  cudaDeviceGetAttribute(&m->n_sm, cudaDevAttrMultiProcessorCount, m->device);
  void* p;
  int rc;
  if ((rc = malloc_multi(m, &p, C_NUM * sizeof(unsigned long long)))) return bail(rc);
  unsigned long long* ctr = (unsigned long long*)p;
  for (auto& q : sim) q.ctr = ctr;
  if ((rc = malloc_multi(m, &p, n * sizeof(DevSystem)))) return bail(rc);
  if (cudaMemcpy(p, sys.data(), n * sizeof(DevSystem), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(mfail(m, BD_ERR_CUDA, "upload of the system table failed"));
  m->T.sys = (const DevSystem*)p;
  if ((rc = malloc_multi(m, &p, n * sizeof(DevSim)))) return bail(rc);
  if (cudaMemcpy(p, sim.data(), n * sizeof(DevSim), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(mfail(m, BD_ERR_CUDA, "upload of the run-parameter table failed"));
  m->T.sim = (const DevSim*)p;
  if ((rc = malloc_multi(m, &p, (n + 1) * sizeof(long long)))) return bail(rc);
  if (cudaMemcpy(p, base.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(mfail(m, BD_ERR_CUDA, "upload of the index table failed"));
  m->T.base = (const long long*)p;
  m->T.n_sys = n;
  m->T.total = base[n];
  m->T.ctr = ctr;
  m->hs.assign(handles, handles + n);
  // slot pool: eight resident waves, at least 65536, at most every trajectory
  void* fn = multi_kernel(m->precision, m->torque);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  m->blocks = per_sm * m->n_sm;
  const long long cap = std::min<long long>(base[n], std::max<long long>(65536, 8ll * m->blocks * 256));
  m->cap = (int)cap;
  for (int b = 0; b < 2; ++b) {
    SlotBuf& B = m->buf[b];
    if ((rc = malloc_multi(m, &p, 3 * (size_t)cap * sizeof(double)))) return bail(rc);
    B.c = (double*)p;
    if ((rc = malloc_multi(m, &p, 4 * (size_t)cap * sizeof(double)))) return bail(rc);
    B.q = (double*)p;
    if ((rc = malloc_multi(m, &p, (size_t)cap * sizeof(int)))) return bail(rc);
    B.traj = (int*)p;
    if ((rc = malloc_multi(m, &p, (size_t)cap * sizeof(int)))) return bail(rc);
    B.steps = (int*)p;
    if ((rc = malloc_multi(m, &p, (size_t)cap * sizeof(int)))) return bail(rc);
    B.rets = (int*)p;
    if ((rc = malloc_multi(m, &p, (size_t)cap))) return bail(rc);
    B.status = (int8_t*)p;
    if ((rc = malloc_multi(m, &p, (size_t)cap))) return bail(rc);
    B.state = (int8_t*)p;
    B.cap = (int)cap;
  }
  if ((rc = malloc_multi(m, &p, 2 * sizeof(int)))) return bail(rc);
  m->d_live = (int*)p;
  if (cudaStreamCreateWithFlags(&m->own, cudaStreamNonBlocking) != cudaSuccess)
    return bail(mfail(m, BD_ERR_CUDA, "stream creation failed"));
  *out = m;
  return BD_OK;
}

int bd_multi_destroy(BdMulti* m) {
  if (!m) return BD_OK;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  for (auto& g : m->graph)
    if (g) cudaGraphExecDestroy(g);
  for (void* p : m->allocs) cudaFree(p);
  if (m->own) cudaStreamDestroy(m->own);
  delete m;
  return BD_OK;
}

int bd_multi_last_error(const BdMulti* m, char* buf, int len) {
  if (!buf || len <= 0) return BD_ERR_ARG;
  snprintf(buf, (size_t)len, "%s", m ? m->err.c_str() : g_create_error.c_str());
  return BD_OK;
}

int bd_multi_reset(BdMulti* m, void* stream) {
  bd::NvtxRange nvtx("bd_multi_reset");
  if (!m) return BD_ERR_ARG;
  MCK(m, cudaSetDevice(m->device));
  cudaStream_t s = (cudaStream_t)stream;
  MCK(m, cudaMemsetAsync(m->T.ctr, 0, C_NUM * sizeof(unsigned long long), s));
  for (BdHandle* h : m->hs) {
    const size_t n = (size_t)h->P.n_traj;
    MCK(m, cudaMemsetAsync(h->P.out_status, 0, n, s));
    MCK(m, cudaMemsetAsync(h->P.out_steps, 0, n * sizeof(int), s));
    MCK(m, cudaMemsetAsync(h->P.out_returns, 0, n * sizeof(int), s));
  }
  init_slots_multi_kernel<<<(m->cap + 255) / 256, 256, 0, s>>>(m->T, m->buf[0], m->cap);
  MCK(m, cudaGetLastError());
  const unsigned long long started = (unsigned long long)m->cap;
  const int live[2] = {m->cap, 0};
  MCK(m, cudaMemcpyAsync(m->T.ctr + C_PENDING, &started, sizeof started, cudaMemcpyHostToDevice, s));
  MCK(m, cudaMemcpyAsync(m->d_live, live, sizeof live, cudaMemcpyHostToDevice, s));
  MCK(m, cudaStreamSynchronize(s));
  m->cur = 0;
  return BD_OK;
}

int bd_multi_run(BdMulti* m, int n_launch, int K, void* stream) {
  bd::NvtxRange nvtx("bd_multi_run");
  if (!m) return BD_ERR_ARG;
  if (n_launch < 0 || K <= 0) return mfail(m, BD_ERR_ARG, "bd_multi_run: n_launch >= 0 and steps > 0 needed");
  MCK(m, cudaSetDevice(m->device));
  int rc = multi_graphs(m, K);
  if (rc) return rc;
  for (int i = 0; i < n_launch; ++i) {
    MCK(m, cudaGraphLaunch(m->graph[m->cur], (cudaStream_t)stream));
    m->cur = 1 - m->cur;
  }
  return BD_OK;
}

int bd_multi_counters(BdMulti* m, uint64_t* out, int n, void* stream) {
  if (!m || !out) return BD_ERR_ARG;
  unsigned long long c[C_NUM];
  cudaStream_t s = (cudaStream_t)stream;
  MCK(m, cudaMemcpyAsync(c, m->T.ctr, sizeof c, cudaMemcpyDeviceToHost, s));
  MCK(m, cudaStreamSynchronize(s));
  const int k = std::min(n, (int)BD_CTR_NUM);
  for (int i = 0; i < k; ++i) out[i] = c[i];
  if (k > 0) out[0] = std::min<unsigned long long>(c[C_PENDING], (unsigned long long)m->T.total);
  return BD_OK;
}

int bd_multi_live(BdMulti* m, int32_t* n_live) {
  if (!m || !n_live) return BD_ERR_ARG;
  MCK(m, cudaDeviceSynchronize());
  MCK(m, cudaMemcpy(n_live, m->d_live + m->cur, sizeof(int), cudaMemcpyDeviceToHost));
  return BD_OK;
}

}  // extern "C"
