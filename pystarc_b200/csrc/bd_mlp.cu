// Surrogate MLP ensemble: training and inference on the tensor cores.
//
// No reference counterpart: this is the engine's learned part.  A member maps
// in_dim inputs through n_hidden SiLU layers of width `hidden` to out_dim
// outputs.  Weights and activations are BF16, every product accumulates in
// FP32 (mma.sync m16n8k16), biases, pre-activations, master weights, Adam
// moments and the loss are FP32.
//
// Training data flow for one member and a batch of n rows (n a multiple of 32):
//   forward   Z_l = A_{l-1} W_l^T + b_l, A_l = SiLU(Z_l)   (Z_l FP32; A_l BF16 in both
//             row-major [n][h] and transposed [h][n] order)
//   loss      L = mean((Y - T)^2) over rows and real outputs; dY = 2 (Y - T) / (n out_dim)
//   backward  dW_l = dZ_l^T A_{l-1} (split over the batch, reduced in a fixed order),
//             db_l = column sums of dZ_l, dA_{l-1} = dZ_l W_l,
//             dZ_{l-1} = dA_{l-1} * SiLU'(Z_{l-1})
//   update    Adam on the FP32 masters, then fresh BF16 copies W_l and W_l^T.
// Every GEMM has the form C = A B^T with both operands K-contiguous in memory,
// which is why activations and gradients are also kept transposed.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "bd_nvtx.cuh"
#include "pystarc_b200.h"

typedef __nv_bfloat16 bf16;

namespace {

constexpr int kBK = 32;        // K step of a GEMM tile
constexpr int kMaxLayers = 9;  // n_hidden <= 8, plus the output layer
constexpr int kChunkRows = 65536;  // inference processes this many rows at a time

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// GEMM C[M][N] = A[M][K] B[N][K]^T (+ epilogue), BF16 in, FP32 accumulate.
// K and N are multiples of 32, lda/ldb multiples of 8; M is arbitrary.
// ---------------------------------------------------------------------------
enum { EPI_HIDDEN_FWD = 0, EPI_OUT_FWD = 1, EPI_HIDDEN_BWD = 2, EPI_PARTIAL = 3 };

struct GemmArgs {
  int M, N, K;
  const bf16* A;
  int lda;
  const bf16* B;
  int ldb;
  int k_per_split;  // multiple of kBK; gridDim.z splits cover K
  const float* bias;
  int n_real;  // EPI_OUT_FWD: columns stored
  float* C;    // Z (hidden fwd, optional), Y (out fwd) or split partials
  int ldc;
  long long split_stride;
  bf16* O;  // BF16 row-major result (activation or dZ), optional
  int ldo;
  bf16* Ot;  // BF16 transposed result [N][ldot], optional
  int ldot;
  const float* Zin;  // pre-activations for the SiLU derivative
  int ldz;
  const int* m_dev;  // optional device row count: rows >= *m_dev are skipped
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], const unsigned b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
// z * sigmoid(z) with sigmoid(z) = (1 + tanh(z / 2)) / 2 on the hardware tanh (relative error
// ~2^-11, below the BF16 rounding the result goes through next)
__device__ __forceinline__ float silu_fast(float z) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * z));
  return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

template <int BM, int BN, int WM, int WN, int EPI>
__global__ void __launch_bounds__(256) gemm_nt(GemmArgs g) {
  static_assert(WM * WN == 8, "8 warps");
  constexpr int TM = BM / WM, TN = BN / WN;  // warp tile
  constexpr int MT = TM / 16, NT = TN / 8;
  constexpr int LDS = kBK + 8;  // padded smem row (bank-conflict free 32-bit fragment loads)
  __shared__ __align__(16) bf16 As[2][BM][LDS];
  __shared__ __align__(16) bf16 Bs[2][BN][LDS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp / WN) * TM, wn0 = (warp % WN) * TN;
  const int gq = lane >> 2, tq = lane & 3;
  const int n0 = blockIdx.x * BN;
  const int M = g.m_dev ? min(g.M, *g.m_dev) : g.M;
  const int kb = blockIdx.z * g.k_per_split, ke = min(g.K, kb + g.k_per_split);
  // row tiles are shared out over gridDim.y blocks (block-uniform loop: barriers stay whole)
  for (int m0 = blockIdx.y * BM; m0 < M; m0 += gridDim.y * BM) {
    float acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;

    auto load = [&](int st, int k) {
      for (int c = tid; c < BM * (kBK / 8); c += 256) {
        const int r = c / (kBK / 8), kc = (c % (kBK / 8)) * 8;
        const int row = m0 + r;
        const bool ok = row < M;
        cp_async16(&As[st][r][kc], g.A + (size_t)(ok ? row : 0) * g.lda + k + kc, ok ? 16 : 0);
      }
      for (int c = tid; c < BN * (kBK / 8); c += 256) {
        const int r = c / (kBK / 8), kc = (c % (kBK / 8)) * 8;
        const int row = n0 + r;
        const bool ok = row < g.N;
        cp_async16(&Bs[st][r][kc], g.B + (size_t)(ok ? row : 0) * g.ldb + k + kc, ok ? 16 : 0);
      }
      cp_async_commit();
    };

    int st = 0;
    if (kb < ke) load(0, kb);
    for (int k = kb; k < ke; k += kBK) {
      if (k + kBK < ke) {
        load(st ^ 1, k + kBK);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kBK; kk += 16) {
        unsigned a[MT][4], b[NT][2];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          const int r = wm0 + i * 16 + gq;
          a[i][0] = *reinterpret_cast<const unsigned*>(&As[st][r][kk + 2 * tq]);
          a[i][1] = *reinterpret_cast<const unsigned*>(&As[st][r + 8][kk + 2 * tq]);
          a[i][2] = *reinterpret_cast<const unsigned*>(&As[st][r][kk + 2 * tq + 8]);
          a[i][3] = *reinterpret_cast<const unsigned*>(&As[st][r + 8][kk + 2 * tq + 8]);
        }
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int c = wn0 + j * 8 + gq;
          b[j][0] = *reinterpret_cast<const unsigned*>(&Bs[st][c][kk + 2 * tq]);
          b[j][1] = *reinterpret_cast<const unsigned*>(&Bs[st][c][kk + 2 * tq + 8]);
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], a[i], b[j]);
      }
      __syncthreads();
      st ^= 1;
    }

    // epilogue: acc[i][j][h*2 + e] is row wm0 + i*16 + gq + 8h, column wn0 + j*8 + 2tq + e
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = m0 + wm0 + i * 16 + gq + 8 * h;
          const int c = n0 + wn0 + j * 8 + 2 * tq;
          if (r >= M || c >= g.N) continue;
          float v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
          if constexpr (EPI == EPI_PARTIAL) {
            float* p = g.C + blockIdx.z * g.split_stride + (size_t)r * g.ldc + c;
            p[0] = v0;
            p[1] = v1;
          } else if constexpr (EPI == EPI_OUT_FWD) {
            if (c < g.n_real) g.C[(size_t)r * g.ldc + c] = v0 + g.bias[c];
            if (c + 1 < g.n_real) g.C[(size_t)r * g.ldc + c + 1] = v1 + g.bias[c + 1];
          } else {
            float o0, o1;
            if constexpr (EPI == EPI_HIDDEN_FWD) {
              v0 += g.bias[c];
              v1 += g.bias[c + 1];
              if (g.C) {
                g.C[(size_t)r * g.ldc + c] = v0;
                g.C[(size_t)r * g.ldc + c + 1] = v1;
              }
              o0 = silu(v0);
              o1 = silu(v1);
            } else {  // EPI_HIDDEN_BWD: v = dA, output dZ
              o0 = v0 * silu_grad(g.Zin[(size_t)r * g.ldz + c]);
              o1 = v1 * silu_grad(g.Zin[(size_t)r * g.ldz + c + 1]);
            }
            const bf16 b0 = __float2bfloat16_rn(o0), b1 = __float2bfloat16_rn(o1);
            if (g.O) {
              __nv_bfloat162 pr;
              pr.x = b0;
              pr.y = b1;
              *reinterpret_cast<__nv_bfloat162*>(g.O + (size_t)r * g.ldo + c) = pr;
            }
            if (g.Ot) {
              g.Ot[(size_t)c * g.ldot + r] = b0;
              g.Ot[(size_t)(c + 1) * g.ldot + r] = b1;
            }
          }
        }
  }  // row tiles
}

// ---------------------------------------------------------------------------
// Small kernels
// ---------------------------------------------------------------------------

// FP32 rows (n x in_dim) -> BF16 rows padded to ld (zeros), optionally transposed [ld][ldt].
__global__ void pack_input_kernel(const float* __restrict__ X, int n, int in_dim, bf16* __restrict__ Xb, int ld,
                                  bf16* __restrict__ Xt, int ldt) {
  const long long total = (long long)n * ld;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / ld), c = (int)(i % ld);
    const bf16 v = __float2bfloat16_rn(c < in_dim ? X[(size_t)r * in_dim + c] : 0.f);
    Xb[i] = v;
    if (Xt) Xt[(size_t)c * ldt + r] = v;
  }
}

// dY = 2 (Y - T) / (n out_dim) as BF16 rows [n][ld] and transposed [ld][ldt]; per-block loss partials.
__global__ void loss_kernel(const float* __restrict__ Y, int ldy, const float* __restrict__ T, int n, int out_dim,
                            bf16* __restrict__ dY, int ld, bf16* __restrict__ dYt, int ldt,
                            float* __restrict__ partial) {
  __shared__ float red[256];
  const float scale = 2.0f / ((float)n * (float)out_dim);
  float s = 0.f;
  const long long total = (long long)n * ld;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / ld), c = (int)(i % ld);
    float d = 0.f;
    if (c < out_dim) {
      const float e = Y[(size_t)r * ldy + c] - T[(size_t)r * out_dim + c];
      s += e * e;
      d = scale * e;
    }
    const bf16 b = __float2bfloat16_rn(d);
    dY[i] = b;
    dYt[(size_t)c * ldt + r] = b;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// loss = sum(partials) / (n out_dim), in a fixed order.
// One warp: lane l sums partials l, l + 32, ... in order, then a fixed-order butterfly.
__global__ void loss_finish_kernel(const float* __restrict__ partial, int nb, float denom, float* __restrict__ loss,
                                   float* __restrict__ trace, const long long* __restrict__ step) {
  const int lane = threadIdx.x;
  if (lane >= 32 || blockIdx.x != 0) return;
  float s = 0.f;
  for (int i = lane; i < nb; i += 32) s += partial[i];
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
  if (lane == 0) {
    if (loss) *loss = s / denom;
    if (trace) trace[*step] = s / denom;
  }
}

// Weight gradient of one layer from split partials (summed in split order) and
// bias gradient as the row sums of dZ^T [out_pad][ldt] over the first n columns.
__global__ void grad_reduce_kernel(const float* __restrict__ part, int splits, long long split_stride, int ldp,
                                   int out_real, int in_real, float* __restrict__ gW) {
  const int total = out_real * in_real;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int o = i / in_real, c = i % in_real;
    float s = 0.f;
    for (int z = 0; z < splits; ++z) s += part[z * split_stride + (size_t)o * ldp + c];
    gW[i] = s;
  }
}

// Bias gradient: one 256-thread block per output row o sums dZ^T[o][0..n) (n and ldt
// multiples of 8): thread t adds the 8-element vectors t, t + 256, ... in order, then a
// fixed-order butterfly per warp and the eight warp sums in order.
__global__ void __launch_bounds__(256) bias_grad_kernel(const bf16* __restrict__ dZt, int ldt, int n, int out_real,
                                                        float* __restrict__ gb) {
  __shared__ float ws[8];
  const int o = blockIdx.x, tid = threadIdx.x, lane = tid & 31;
  if (o >= out_real) return;
  const uint4* row = reinterpret_cast<const uint4*>(dZt + (size_t)o * ldt);
  float s = 0.f;
  for (int v = tid; v < n / 8; v += 256) {
    const uint4 u = __ldg(row + v);
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[k]));
      s += f.x + f.y;
    }
  }
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
  if (lane == 0) ws[tid >> 5] = s;
  __syncthreads();
  if (tid == 0) {
    float t = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += ws[k];
    gb[o] = t;
  }
}

// Random training batch: row i of the batch is data row hash(seed, step, i) mod n_data.
__global__ void gather_batch_kernel(const float* __restrict__ X, const float* __restrict__ T, long long n_data,
                                    int in_dim, int out_dim, int batch, unsigned long long seed,
                                    const long long* __restrict__ step, float* __restrict__ Xb,
                                    float* __restrict__ Tb) {
  const long long st = *step;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
    unsigned long long z = seed ^ ((unsigned long long)st << 24) ^ (unsigned long long)i;
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const long long r = (long long)(z % (unsigned long long)n_data);
    for (int k = 0; k < in_dim; ++k) Xb[(size_t)i * in_dim + k] = X[r * in_dim + k];
    for (int k = 0; k < out_dim; ++k) Tb[(size_t)i * out_dim + k] = T[r * out_dim + k];
  }
}

__global__ void step_increment_kernel(long long* step) { *step += 1; }

struct LayerGeom {
  int in_real[kMaxLayers], out_real[kMaxLayers], in_pad[kMaxLayers], out_pad[kMaxLayers];
  long long w_off[kMaxLayers], b_off[kMaxLayers];  // into the FP32 parameter vector
  long long wb_off[kMaxLayers];                     // into the padded BF16 W / W^T buffers
  int n_layers;
};

// ---------------------------------------------------------------------------
// Inference on the 5th-generation tensor cores (tcgen05).  One CTA of 128
// threads runs every layer of one member on 128 rows: the activation tile
// (128 x K, BF16) and the layer's weights (N x K, BF16) sit in shared memory in
// the canonical K-major no-swizzle layout (8-row x 16-byte core matrices; K
// chunks 128 B apart, 8-row groups SBO apart), one elected thread issues the
// 128 x N x 16 MMAs into a TMEM accumulator of N FP32 columns, and the four
// warps read their 32 TMEM lanes back (tcgen05.ld 32x32b) for the epilogue:
// bias + SiLU into the next activation tile, or bias into the FP32 outputs.
// Hidden widths up to 256; the input and output are padded to 32.
// ---------------------------------------------------------------------------
constexpr int kTcRows = 128;
constexpr int kTcK = 256;                        // widest K held in the activation tile
constexpr int kTcSboA = kTcK / 8 * 128;          // bytes between 8-row groups of the activation tile
constexpr int kTcBytesA = kTcRows * kTcK * 2;    // 64 KB
constexpr int kTcBytesB = 256 * kTcK * 2;        // 128 KB
constexpr int kTcSmem = kTcBytesA + kTcBytesB + 64;  // + two mbarriers and the TMEM address
constexpr int kTcMaxMembers = 8;

struct TcArgs {
  const bf16* X;  // n x 32 packed BF16 input rows
  int n;
  const int* n_dev;  // optional device row count
  const bf16* Wc[kTcMaxMembers];  // per member: each layer's weights as the canonical shared-memory image
  const float* P[kTcMaxMembers];  // FP32 parameter vectors (biases)
  LayerGeom L;
  float* Y;  // per member: rows x ldy, members y_stride apart (member0's block first)
  int ldy;
  long long y_stride;
  int member0;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (row, k) in a canonical K-major no-swizzle tile.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int sbo) {
  return (uint32_t)((row >> 3) * sbo + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (sm100): start, leading and stride byte offsets
// (>> 4), version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  // bounded: a wait that never completes returns false instead of hanging the GPU
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Thread 0: stream layer l's weight image (already in the canonical layout) into the B tile.
__device__ __forceinline__ void load_weights_async(const TcArgs& a, int member, int l, unsigned char* Bs,
                                                   uint32_t bar) {
  const LayerGeom& L = a.L;
  const uint32_t bytes = (uint32_t)(L.out_pad[l] * L.in_pad[l] * 2);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  const unsigned char* src = reinterpret_cast<const unsigned char*>(a.Wc[member] + L.wb_off[l]);
  for (uint32_t off = 0; off < bytes; off += 32768u)
    bulk_g2s(smem_u32(Bs) + off, src + off, min(32768u, bytes - off), bar);
}

__global__ void __launch_bounds__(512, 1) mlp_forward_tc_kernel(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char* As = tc_smem;
  unsigned char* Bs = tc_smem + kTcBytesA;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tc_smem + kTcBytesA + kTcBytesB);  // [0] MMA done, [1] weights in
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(tc_smem + kTcBytesA + kTcBytesB + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int member = a.member0 + blockIdx.y;
  const int n = a.n_dev ? min(a.n, *a.n_dev) : a.n;
  const int r0 = blockIdx.x * kTcRows;
  if (r0 >= n) return;  // whole block, before any allocation
  const LayerGeom& L = a.L;
  int width = 32;  // columns of TMEM used
  for (int l = 0; l < L.n_layers; ++l) width = max(width, L.out_pad[l]);
  const uint32_t ncols = width <= 32 ? 32 : width <= 64 ? 64 : width <= 128 ? 128 : 256;
  const uint32_t bar_mma = smem_u32(bar), bar_w = smem_u32(bar + 1);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_mma), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_w), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    load_weights_async(a, member, 0, Bs, bar_w);
  }
  // input rows: 32 BF16 (four 16-byte chunks) per row; rows past n are zero
  for (int c = tid; c < kTcRows * 4; c += blockDim.x) {
    const int r = c >> 2, kc = c & 3;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (r0 + r < n) v = *reinterpret_cast<const uint4*>(a.X + (size_t)(r0 + r) * 32 + kc * 8);
    *reinterpret_cast<uint4*>(As + kmajor_off(r, kc * 8, kTcSboA)) = v;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_slot;
  bool ok = true;
  // epilogue split: warp w reads TMEM lanes 32 (w % 4) .. + 31 and every fourth 32-column chunk
  const int quarter = warp & 3, colgroup = warp >> 2;
  const int row = quarter * 32 + lane;
  for (int l = 0; l < L.n_layers; ++l) {
    const int N = L.out_pad[l], K = L.in_pad[l], sbo_b = K / 8 * 128;
    if (tid == 0) {
      ok = mbar_wait(bar_w, (uint32_t)(l & 1)) && ok;  // this layer's weights are in
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t idesc = umma_idesc_bf16(kTcRows, N);
      for (int j = 0; j < K / 16; ++j) {
        const uint64_t ad = umma_desc(smem_u32(As) + j * 256, 128, kTcSboA);
        const uint64_t bd = umma_desc(smem_u32(Bs) + j * 256, 128, sbo_b);
        const uint32_t acc = j > 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_mma)
                   : "memory");
    }
    ok = mbar_wait(bar_mma, (uint32_t)(l & 1)) && ok;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // the B tile is free again: the next layer's weights stream in during this epilogue
    if (tid == 0 && l + 1 < L.n_layers) load_weights_async(a, member, l + 1, Bs, bar_w);
    const float* bias = a.P[member] + L.b_off[l];
    const bool last = l + 1 == L.n_layers;
    for (int c0 = 32 * colgroup; c0 < N; c0 += 128) {
      uint32_t v[32];
      const uint32_t addr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (last) {
        if (r0 + row < n) {
          float* y = a.Y + blockIdx.y * a.y_stride + (size_t)(r0 + row) * a.ldy;
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            const int c = c0 + k;
            if (c < L.out_real[l]) y[c] = ok ? __uint_as_float(v[k]) + bias[c] : __int_as_float(0x7fc00000);
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t pk[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int c = c0 + q * 8 + 2 * e;
            const float z0 = __uint_as_float(v[q * 8 + 2 * e]) + bias[c];
            const float z1 = __uint_as_float(v[q * 8 + 2 * e + 1]) + bias[c + 1];
            __nv_bfloat162 h2 = __floats2bfloat162_rn(silu_fast(z0), silu_fast(z1));
            pk[e] = *reinterpret_cast<uint32_t*>(&h2);
          }
          *reinterpret_cast<uint4*>(As + kmajor_off(row, c0 + q * 8, kTcSboA)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}


// ---------------------------------------------------------------------------
// The training GEMMs on tcgen05: C[M][N] = A[M][K] B[N][K]^T with the fused epilogues of gemm_nt.
// One CTA of 128 threads per 128-row tile (looping over its share of the tiles) and BN columns
// (BN <= 256, a multiple of 16): K is staged 64 at a time into kGtStages shared-memory buffers in
// the canonical K-major no-swizzle layout by cp.async (rows past M read as zero).  The first
// kGtStages - 1 chunks load up front; one elected thread issues each chunk's 128 x BN x 16 MMAs
// into a TMEM accumulator as soon as it is in and commits them to the buffer's mbarrier, and the
// chunk kGtStages - 1 ahead then loads into the buffer the previous chunk's MMAs release.  The four
// warps read their 32 TMEM lanes (rows) back with tcgen05.ld for the epilogue.  Split-K
// (gridDim.z) writes partials for a fixed-order reduction, as gemm_nt does.
// ---------------------------------------------------------------------------
constexpr int kGtKc = 64;                  // K per staged chunk
constexpr int kGtStages = 4;               // staged chunks in flight
constexpr int kGtSbo = kGtKc / 8 * 128;    // bytes between 8-row groups of a chunk
constexpr int kGtBytesA = 128 * kGtKc * 2;  // 16 KB
__host__ __device__ constexpr int gt_stage_bytes(int BN) { return kGtBytesA + BN * kGtKc * 2; }
// stages + kGtStages mbarriers + the TMEM address
__host__ __device__ constexpr int gt_smem_bytes(int BN) { return kGtStages * gt_stage_bytes(BN) + 8 * kGtStages + 16; }

template <int EPI>
__global__ void __launch_bounds__(128, 1) gemm_nt_tc(GemmArgs g, int BN) {
  extern __shared__ __align__(1024) unsigned char gt_smem[];
  // stage st: A tile at st * stage bytes, B tile right after it
  const int sb = gt_stage_bytes(BN);
  auto As = [&](int st) { return gt_smem + st * sb; };
  auto Bs = [&](int st) { return gt_smem + st * sb + kGtBytesA; };
  uint64_t* bar = reinterpret_cast<uint64_t*>(gt_smem + kGtStages * sb);
  uint32_t* taddr_slot = reinterpret_cast<uint32_t*>(gt_smem + kGtStages * sb + 8 * kGtStages);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n0 = blockIdx.x * BN;
  const int M = g.m_dev ? min(g.M, *g.m_dev) : g.M;
  const int kb = blockIdx.z * g.k_per_split, ke = min(g.K, kb + g.k_per_split);
  if (blockIdx.y * 128 >= M || kb >= ke) return;  // whole block, before any allocation
  const int nb = min(BN, g.N - n0);  // columns of this block (a multiple of 16)
  const uint32_t ncols = nb <= 32 ? 32 : nb <= 64 ? 64 : nb <= 128 ? 128 : 256;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int st = 0; st < kGtStages; ++st)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar + st)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_slot;
  const uint32_t idesc = umma_idesc_bf16(128, nb);
  uint32_t phase[kGtStages] = {};
  bool pending[kGtStages] = {};
  bool ok = true;
  auto wait_stage = [&](int st) {
    if (pending[st]) {
      ok = mbar_wait(smem_u32(bar + st), phase[st]) && ok;
      phase[st] ^= 1u;
      pending[st] = false;
    }
  };
  const int nk = (ke - kb + kGtKc - 1) / kGtKc;
  for (int m0 = blockIdx.y * 128; m0 < M; m0 += gridDim.y * 128) {
    // chunk kc of this tile into buffer kc % kGtStages (whose MMAs, if any, are waited for first)
    auto load_chunk = [&](int kc) {
      const int st = kc % kGtStages, k = kb + kc * kGtKc, nch = min(kGtKc, ke - k) / 8;
      wait_stage(st);
      for (int c = tid; c < 128 * nch; c += 128) {
        const int r = c / nch, kk = (c % nch) * 8;
        const bool in = m0 + r < M;
        cp_async16(As(st) + kmajor_off(r, kk, kGtSbo), g.A + (size_t)(in ? m0 + r : 0) * g.lda + k + kk, in ? 16 : 0);
      }
      for (int c = tid; c < nb * nch; c += 128) {
        const int r = c / nch, kk = (c % nch) * 8;
        cp_async16(Bs(st) + kmajor_off(r, kk, kGtSbo), g.B + (size_t)(n0 + r) * g.ldb + k + kk, 16);
      }
    };
    // every thread commits one cp.async group per chunk slot (empty past the last chunk), so
    // "all but the newest kGtStages - 2 groups done" means "chunk kc is in"
#pragma unroll 1
    for (int kc = 0; kc < kGtStages - 1; ++kc) {
      if (kc < nk) load_chunk(kc);
      cp_async_commit();
    }
#pragma unroll 1
    for (int kc = 0; kc < nk; ++kc) {
      const int st = kc % kGtStages, klen = min(kGtKc, ke - (kb + kc * kGtKc));
      cp_async_wait<kGtStages - 2>();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        for (int j = 0; j < klen / 16; ++j) {
          const uint64_t ad = umma_desc(smem_u32(As(st)) + j * 256, 128, kGtSbo);
          const uint64_t bd = umma_desc(smem_u32(Bs(st)) + j * 256, 128, kGtSbo);
          const uint32_t acc = (kc > 0 || j > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(bar + st))
                     : "memory");
      }
      pending[st] = true;
      // the chunk kGtStages - 1 ahead goes into the buffer of chunk kc - 1 once its MMAs are done
      if (kc + kGtStages - 1 < nk) load_chunk(kc + kGtStages - 1);
      cp_async_commit();
    }
    cp_async_wait<0>();
#pragma unroll
    for (int st = 0; st < kGtStages; ++st) wait_stage(st);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: thread = row m0 + 32 warp + lane, 32 columns per TMEM load
    const int r = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < nb; c0 += 32) {
      uint32_t v[32];
      const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(addr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // rows past M store nothing, but their lanes stay for the transposed store's shuffles
      const bool valid = r < M;
      const int cw = min(32, nb - c0);  // columns of this load that exist (32 or 16)
      const int cb = n0 + c0;           // first column
      float f[32];
#pragma unroll
      for (int e = 0; e < 32; ++e) f[e] = ok ? __uint_as_float(v[e]) : __int_as_float(0x7fc00000);
      if (!valid && !(EPI == EPI_HIDDEN_FWD || EPI == EPI_HIDDEN_BWD)) continue;
      if constexpr (EPI == EPI_PARTIAL) {
        float* p = g.C + blockIdx.z * g.split_stride + (size_t)r * g.ldc + cb;
#pragma unroll
        for (int e = 0; e < 32; e += 4)
          if (e < cw) *reinterpret_cast<float4*>(p + e) = make_float4(f[e], f[e + 1], f[e + 2], f[e + 3]);
      } else if constexpr (EPI == EPI_OUT_FWD) {
#pragma unroll
        for (int e = 0; e < 32; ++e)
          if (e < cw && cb + e < g.n_real) g.C[(size_t)r * g.ldc + cb + e] = f[e] + g.bias[cb + e];
      } else {
        uint32_t pk[16];
#pragma unroll
        for (int e = 0; e < 32; e += 2) {
          float o0, o1;
          if constexpr (EPI == EPI_HIDDEN_FWD) {
            f[e] += g.bias[cb + e];
            f[e + 1] += g.bias[cb + e + 1];
            o0 = silu(f[e]);
            o1 = silu(f[e + 1]);
          } else {  // EPI_HIDDEN_BWD: f = dA, output dZ; Z read two columns at a time
            float z0 = 0.f, z1 = 0.f;
            if (valid && e < cw) {
              const float2 z = *reinterpret_cast<const float2*>(g.Zin + (size_t)r * g.ldz + cb + e);
              z0 = z.x;
              z1 = z.y;
            }
            o0 = e < cw ? f[e] * silu_grad(z0) : 0.f;
            o1 = e < cw ? f[e + 1] * silu_grad(z1) : 0.f;
          }
          __nv_bfloat162 h2 = __floats2bfloat162_rn(o0, o1);
          pk[e / 2] = *reinterpret_cast<uint32_t*>(&h2);
        }
        if (valid && EPI == EPI_HIDDEN_FWD && g.C) {
          float* z = g.C + (size_t)r * g.ldc + cb;
#pragma unroll
          for (int e = 0; e < 32; e += 4)
            if (e < cw) *reinterpret_cast<float4*>(z + e) = make_float4(f[e], f[e + 1], f[e + 2], f[e + 3]);
        }
        if (valid && g.O) {
          bf16* o = g.O + (size_t)r * g.ldo + cb;
#pragma unroll
          for (int e = 0; e < 32; e += 8)
            if (e < cw) *reinterpret_cast<uint4*>(o + e) = make_uint4(pk[e / 2], pk[e / 2 + 1], pk[e / 2 + 2], pk[e / 2 + 3]);
        }
        if (g.Ot) {
          // transposed copy, two rows per 4-byte store: the lane pair (2k, 2k+1) holds rows r, r + 1;
          // for columns (e, e + 1) the even lane stores column e of both rows, the odd lane column e + 1
          // (M is even wherever a transposed copy is kept, so both rows of a pair are valid or neither)
          const bool odd = lane & 1;
          const int r0 = r & ~1;
#pragma unroll
          for (int e = 0; e < 32; e += 2) {
            const uint32_t w = pk[e / 2];  // columns e (low half) and e + 1 (high half) of this row
            const uint32_t send = odd ? (w & 0xffffu) : (w >> 16);
            const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 1);
            const uint32_t out = odd ? (recv | (w & 0xffff0000u)) : ((w & 0xffffu) | (recv << 16));
            if (valid && e < cw)
              *reinterpret_cast<uint32_t*>(g.Ot + (size_t)(cb + e + (odd ? 1 : 0)) * g.ldot + r0) = out;
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // every lane is read before the next tile's MMAs overwrite the accumulator
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// Adam on the FP32 parameters, then the padded BF16 copies W [out_pad][in_pad] and W^T [in_pad][out_pad].
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m1,
                            float* __restrict__ m2, long long n_params, float lr, float b1, float b2, float eps,
                            const long long* __restrict__ t_prev, LayerGeom L, bf16* __restrict__ Wb,
                            bf16* __restrict__ Wt, bf16* __restrict__ Wc) {
  // bias corrections of step t = t_prev + 1
  const double t = (double)(*t_prev + 1);
  const float c1 = (float)(1.0 - pow((double)b1, t)), c2 = (float)(1.0 - pow((double)b2, t));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_params;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float w = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    p[i] = w;
    for (int l = 0; l < L.n_layers; ++l) {
      if (i >= L.w_off[l] && i < L.b_off[l]) {
        const int k = (int)(i - L.w_off[l]);
        const int o = k / L.in_real[l], c = k % L.in_real[l];
        const bf16 v = __float2bfloat16_rn(w);
        Wb[L.wb_off[l] + (size_t)o * L.in_pad[l] + c] = v;
        Wt[L.wb_off[l] + (size_t)c * L.out_pad[l] + o] = v;
        Wc[L.wb_off[l] + kmajor_off(o, c, L.in_pad[l] / 8 * 128) / 2] = v;
      }
    }
  }
}

// BF16 copies of every weight from the FP32 parameters (after set/initialise).
__global__ void refresh_kernel(const float* __restrict__ p, long long n_params, LayerGeom L, bf16* __restrict__ Wb,
                               bf16* __restrict__ Wt, bf16* __restrict__ Wc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_params;
       i += (long long)gridDim.x * blockDim.x) {
    for (int l = 0; l < L.n_layers; ++l) {
      if (i >= L.w_off[l] && i < L.b_off[l]) {
        const int k = (int)(i - L.w_off[l]);
        const int o = k / L.in_real[l], c = k % L.in_real[l];
        const bf16 v = __float2bfloat16_rn(p[i]);
        Wb[L.wb_off[l] + (size_t)o * L.in_pad[l] + c] = v;
        Wt[L.wb_off[l] + (size_t)c * L.out_pad[l] + o] = v;
        Wc[L.wb_off[l] + kmajor_off(o, c, L.in_pad[l] / 8 * 128) / 2] = v;
      }
    }
  }
}

// Ensemble mean and spread (RMS deviation of the members from the mean), per output.
__global__ void ensemble_kernel(const float* __restrict__ Ys, int members, long long stride, int n, int out_dim,
                                float* __restrict__ mean, float* __restrict__ spread, const int* __restrict__ n_dev) {
  if (n_dev) n = min(n, *n_dev);
  const long long total = (long long)n * out_dim;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int m = 0; m < members; ++m) s += Ys[m * stride + i];
    const float mu = s / (float)members;
    float d = 0.f;
    for (int m = 0; m < members; ++m) {
      const float e = Ys[m * stride + i] - mu;
      d += e * e;
    }
    mean[i] = mu;
    if (spread) spread[i] = sqrtf(d / (float)members);
  }
}

}  // namespace

// ===========================================================================
struct BdMlp {
  int device = 0;
  BdMlpDesc d{};
  std::string err;
  LayerGeom L{};
  long long n_params = 0, wb_size = 0;
  int n_sm = 148;
  struct Member {
    float *p = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr;
    bf16 *Wb = nullptr, *Wt = nullptr, *Wc = nullptr;  // W, W^T, and W as canonical tcgen05 tiles
    long long* step = nullptr;  // device: Adam steps taken
  };
  // graph of one training step (bd_mlp_train), rebuilt when its arguments change
  cudaGraphExec_t train_graph = nullptr;
  int tg_member = -1, tg_batch = 0;
  const float *tg_X = nullptr, *tg_T = nullptr;
  long long tg_n = 0;
  float tg_lr = 0.f;
  unsigned long long tg_seed = 0;
  float* tg_trace = nullptr;
  float *Xbatch = nullptr, *Tbatch = nullptr;
  int batch_cap = 0;
  long long* data_step = nullptr;  // device: batches drawn by bd_mlp_train
  std::vector<Member> mem;
  std::vector<void*> allocs;  // everything, freed at destroy
  // training scratch (sized for `train_cap` rows)
  int train_cap = 0;
  std::vector<void*> train_allocs;
  bf16 *Xb = nullptr, *Xt = nullptr, *dY = nullptr, *dYt = nullptr;
  std::vector<float*> Z;
  std::vector<bf16*> A, At, dZ, dZt;
  float *Y = nullptr, *part = nullptr, *loss_part = nullptr, *loss_tmp = nullptr;
  long long part_stride = 0;
  int inference = 1;  // 1: tcgen05 kernel when the shape allows, 0: mma.sync GEMM chain
  int gemm_tc = 1;    // GEMMs of training and of the GEMM chain: 1 tcgen05 (gemm_nt_tc), 0 mma.sync
  bool gt_attr = false;
  bool tc_attr = false;
  // inference scratch (infer_cap rows)
  int infer_cap = 0;
  std::vector<void*> infer_allocs;
  bf16 *act[2] = {nullptr, nullptr}, *Xi = nullptr;
  float* Ys = nullptr;
};

namespace {

int mfail(BdMlp* m, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (m) m->err = buf;
  return code;
}

#define MCK(m, x)                                                                                       \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess)                                                                              \
      return mfail(m, e_ == cudaErrorMemoryAllocation ? BD_ERR_OOM : BD_ERR_CUDA, "%s: %s (%s:%d)", #x, \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                                         \
  } while (0)

int malloc_into(BdMlp* m, std::vector<void*>& list, void** p, size_t bytes) {
  MCK(m, cudaMalloc(p, bytes));
  list.push_back(*p);
  MCK(m, cudaMemset(*p, 0, bytes));
  return BD_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

int grid_for(BdMlp* m, long long n) { return (int)std::min<long long>((n + 255) / 256, (long long)m->n_sm * 16); }

template <int BM, int BN, int WM, int WN, int EPI>
int launch_gemm(BdMlp* m, const GemmArgs& g, int splits, cudaStream_t s) {
  const int nx = (g.N + BN - 1) / BN, tiles = (g.M + BM - 1) / BM;
  // enough blocks for two per SM; each loops over its share of the row tiles
  const int ny = std::max(1, std::min(tiles, (2 * m->n_sm + nx * splits - 1) / (nx * splits)));
  dim3 grid(nx, ny, splits);
  gemm_nt<BM, BN, WM, WN, EPI><<<grid, 256, 0, s>>>(g);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

template <int EPI>
int launch_gemm_tc(BdMlp* m, const GemmArgs& g, int splits, cudaStream_t s) {
  if (!m->gt_attr) {
    const int mx = gt_smem_bytes(256);
    MCK(m, cudaFuncSetAttribute(gemm_nt_tc<EPI_HIDDEN_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    MCK(m, cudaFuncSetAttribute(gemm_nt_tc<EPI_OUT_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    MCK(m, cudaFuncSetAttribute(gemm_nt_tc<EPI_HIDDEN_BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    MCK(m, cudaFuncSetAttribute(gemm_nt_tc<EPI_PARTIAL>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx));
    m->gt_attr = true;
  }
  // the widest column tile (256, 128 or 64) whose CTAs still cover every SM; 64-wide tiles fit
  // two CTAs per SM (96 KB of shared memory, 64 TMEM columns each)
  const int tiles = (g.M + 127) / 128;
  int BN = std::min(g.N, 256);
  while (BN > 64 && ((g.N + BN - 1) / BN) * tiles * splits < m->n_sm) BN = std::max(64, (BN / 2 + 15) / 16 * 16);
  const int nx = (g.N + BN - 1) / BN, per_sm = BN <= 64 ? 2 : 1;
  const int ny = std::max(1, std::min(tiles, (per_sm * m->n_sm + nx * splits - 1) / (nx * splits)));
  dim3 grid(nx, ny, splits);
  gemm_nt_tc<EPI><<<grid, 128, gt_smem_bytes(BN), s>>>(g, BN);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

// C = A B^T: tcgen05 (N a multiple of 16, K of 32), else mma.sync with the tile picked from N
// (hidden widths use 128-wide tiles).
template <int EPI>
int gemm(BdMlp* m, const GemmArgs& g, int splits, cudaStream_t s) {
  if (m->gemm_tc && g.N % 16 == 0 && g.K % 32 == 0 && g.k_per_split % 32 == 0)
    return launch_gemm_tc<EPI>(m, g, splits, s);
  if (g.N >= 128) return launch_gemm<128, 128, 2, 4, EPI>(m, g, splits, s);
  return launch_gemm<128, 32, 4, 2, EPI>(m, g, splits, s);
}

int ensure_train(BdMlp* m, int n) {
  if (n <= m->train_cap) return BD_OK;
  if (m->train_graph) {  // it holds the old buffers
    cudaGraphExecDestroy(m->train_graph);
    m->train_graph = nullptr;
  }
  for (void* p : m->train_allocs) cudaFree(p);
  m->train_allocs.clear();
  m->Z.assign(m->L.n_layers, nullptr);
  m->A.assign(m->L.n_layers, nullptr);
  m->At.assign(m->L.n_layers, nullptr);
  m->dZ.assign(m->L.n_layers, nullptr);
  m->dZt.assign(m->L.n_layers, nullptr);
  const LayerGeom& L = m->L;
  void* p;
  int rc;
  auto get = [&](size_t bytes) -> void* {
    p = nullptr;
    rc = malloc_into(m, m->train_allocs, &p, bytes);
    return p;
  };
  m->Xb = (bf16*)get((size_t)n * L.in_pad[0] * 2);
  if (rc) return rc;
  m->Xt = (bf16*)get((size_t)n * L.in_pad[0] * 2);
  if (rc) return rc;
  const int nl = L.n_layers;
  for (int l = 0; l + 1 < nl; ++l) {  // hidden layers
    const int h = L.out_pad[l];
    if (!(m->Z[l] = (float*)get((size_t)n * h * 4))) return rc;
    if (!(m->A[l] = (bf16*)get((size_t)n * h * 2))) return rc;
    if (!(m->At[l] = (bf16*)get((size_t)n * h * 2))) return rc;
    if (!(m->dZ[l] = (bf16*)get((size_t)n * h * 2))) return rc;
    if (!(m->dZt[l] = (bf16*)get((size_t)n * h * 2))) return rc;
  }
  const int op = L.out_pad[nl - 1];
  if (!(m->Y = (float*)get((size_t)n * op * 4))) return rc;
  if (!(m->dY = (bf16*)get((size_t)n * op * 2))) return rc;
  if (!(m->dYt = (bf16*)get((size_t)n * op * 2))) return rc;
  int maxw = 0;
  for (int l = 0; l < nl; ++l) maxw = std::max(maxw, L.out_pad[l] * L.in_pad[l]);
  m->part_stride = maxw;
  if (!(m->part = (float*)get((size_t)64 * maxw * 4))) return rc;
  if (!(m->loss_part = (float*)get((size_t)m->n_sm * 16 * 4))) return rc;
  if (!(m->loss_tmp = (float*)get(4))) return rc;
  m->train_cap = n;
  return BD_OK;
}

// Inference buffers for `rows` rows at a time (at least kChunkRows).
int ensure_infer(BdMlp* m, int rows = kChunkRows) {
  rows = std::max(rows, kChunkRows);
  if (rows <= m->infer_cap) return BD_OK;
  MCK(m, cudaDeviceSynchronize());
  for (void* q : m->infer_allocs) cudaFree(q);
  m->infer_allocs.clear();
  m->infer_cap = 0;
  const LayerGeom& L = m->L;
  int wmax = L.in_pad[0];
  for (int l = 0; l < L.n_layers; ++l) wmax = std::max(wmax, L.out_pad[l]);
  void* p;
  int rc;
  if ((rc = malloc_into(m, m->infer_allocs, &p, (size_t)rows * L.in_pad[0] * 2))) return rc;
  m->Xi = (bf16*)p;
  for (int k = 0; k < 2; ++k) {
    if ((rc = malloc_into(m, m->infer_allocs, &p, (size_t)rows * wmax * 2))) return rc;
    m->act[k] = (bf16*)p;
  }
  if ((rc = malloc_into(m, m->infer_allocs, &p, (size_t)m->d.n_members * rows * m->d.out_dim * 4))) return rc;
  m->Ys = (float*)p;
  m->infer_cap = rows;
  return BD_OK;
}

// Forward of one member on packed BF16 rows Xb [n][in_pad]; writes Y [n][ldy] (FP32, real outputs).
// Training mode keeps Z, A and A^T of every hidden layer.
int forward(BdMlp* m, int member, int n, const bf16* Xb, float* Y, int ldy, bool train, cudaStream_t s,
            const int* n_dev = nullptr) {
  const LayerGeom& L = m->L;
  const BdMlp::Member& w = m->mem[member];
  const bf16* in = Xb;
  int ld_in = L.in_pad[0];
  for (int l = 0; l < L.n_layers; ++l) {
    GemmArgs g{};
    g.M = n;
    g.N = L.out_pad[l];
    g.K = L.in_pad[l];
    g.A = in;
    g.lda = ld_in;
    g.B = w.Wb + L.wb_off[l];
    g.ldb = L.in_pad[l];
    g.k_per_split = g.K;
    g.bias = w.p + L.b_off[l];
    g.m_dev = n_dev;
    int rc;
    if (l + 1 < L.n_layers) {
      bf16* out = train ? m->A[l] : m->act[l & 1];
      g.C = train ? m->Z[l] : nullptr;
      g.ldc = g.N;
      g.O = out;
      g.ldo = g.N;
      g.Ot = train ? m->At[l] : nullptr;
      g.ldot = n;
      if ((rc = gemm<EPI_HIDDEN_FWD>(m, g, 1, s))) return rc;
      in = out;
      ld_in = g.N;
    } else {
      g.C = Y;
      g.ldc = ldy;
      g.n_real = L.out_real[l];
      if ((rc = gemm<EPI_OUT_FWD>(m, g, 1, s))) return rc;
    }
  }
  return BD_OK;
}

bool tc_eligible(const BdMlp* m) {
  if (m->inference != 1 || m->L.in_pad[0] != 32 || m->d.hidden > kTcK) return false;
  for (int l = 0; l < m->L.n_layers; ++l)
    if (m->L.out_pad[l] > 256 || m->L.in_pad[l] > kTcK) return false;
  return true;
}

// Members [member0, member0 + count) on packed rows Xp (n x 32 BF16): Y block of member k at
// Y + k * y_stride, rows ldy apart.  tcgen05 kernel, one CTA per (128-row tile, member).
int forward_tc(BdMlp* m, int member0, int count, int n, const bf16* Xp, float* Y, int ldy, long long y_stride,
               cudaStream_t s, const int* n_dev = nullptr) {
  if (!m->tc_attr) {
    MCK(m, cudaFuncSetAttribute(mlp_forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
    m->tc_attr = true;
  }
  TcArgs a{};
  a.X = Xp;
  a.n = n;
  a.n_dev = n_dev;
  // the kernel indexes the tables by member0 + blockIdx.y
  TcArgs b = a;
  for (int k = 0; k < count; ++k) {
    b.Wc[member0 + k] = m->mem[member0 + k].Wc;
    b.P[member0 + k] = m->mem[member0 + k].p;
  }
  b.L = m->L;
  b.Y = Y;
  b.ldy = ldy;
  b.y_stride = y_stride;
  b.member0 = member0;
  dim3 grid((n + kTcRows - 1) / kTcRows, count);
  if (grid.x == 0) return BD_OK;
  mlp_forward_tc_kernel<<<grid, 512, kTcSmem, s>>>(b);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

// Loss and gradient of one member on n rows (n % 32 == 0) into the member's grad buffer.
int backward(BdMlp* m, int member, int n, const float* X, const float* T, float* loss, cudaStream_t s,
             float* trace = nullptr) {
  const LayerGeom& L = m->L;
  BdMlp::Member& w = m->mem[member];
  int rc;
  if ((rc = ensure_train(m, n))) return rc;
  pack_input_kernel<<<grid_for(m, (long long)n * L.in_pad[0]), 256, 0, s>>>(X, n, m->d.in_dim, m->Xb, L.in_pad[0],
                                                                             m->Xt, n);
  MCK(m, cudaGetLastError());
  const int nl = L.n_layers, op = L.out_pad[nl - 1];
  if ((rc = forward(m, member, n, m->Xb, m->Y, op, true, s))) return rc;
  const int nb = grid_for(m, (long long)n * op);
  loss_kernel<<<nb, 256, 0, s>>>(m->Y, op, T, n, m->d.out_dim, m->dY, op, m->dYt, n, m->loss_part);
  MCK(m, cudaGetLastError());
  loss_finish_kernel<<<1, 32, 0, s>>>(m->loss_part, nb, (float)n * (float)m->d.out_dim, loss ? loss : m->loss_tmp,
                                     trace, trace ? m->data_step : nullptr);
  MCK(m, cudaGetLastError());
  // split-K of the weight gradients: 512 rows per split (16 at batch 8192) keep every SM busy
  // while halving the partials that grad_reduce_kernel reads back
  const int splits = std::max(1, std::min(64, n / 512));
  const int kps = round_up((n + splits - 1) / splits, kBK);
  for (int l = nl - 1; l >= 0; --l) {
    const bf16* dZ = l == nl - 1 ? m->dY : m->dZ[l];
    const bf16* dZt = l == nl - 1 ? m->dYt : m->dZt[l];
    const bf16* Ain_t = l == 0 ? m->Xt : m->At[l - 1];
    // dW_l = dZ_l^T A_{l-1}: M = out_pad, N = in_pad, K = n
    GemmArgs g{};
    g.M = L.out_pad[l];
    g.N = L.in_pad[l];
    g.K = n;
    g.A = dZt;
    g.lda = n;
    g.B = Ain_t;
    g.ldb = n;
    g.k_per_split = kps;
    g.C = m->part;
    g.ldc = L.in_pad[l];
    g.split_stride = m->part_stride;
    const int used = (n + kps - 1) / kps;
    if ((rc = gemm<EPI_PARTIAL>(m, g, used, s))) return rc;
    const int tot = L.out_real[l] * L.in_real[l];
    grad_reduce_kernel<<<grid_for(m, tot), 256, 0, s>>>(m->part, used, m->part_stride, L.in_pad[l], L.out_real[l],
                                                         L.in_real[l], w.grad + L.w_off[l]);
    MCK(m, cudaGetLastError());
    bias_grad_kernel<<<L.out_real[l], 256, 0, s>>>(dZt, n, n, L.out_real[l], w.grad + L.b_off[l]);
    MCK(m, cudaGetLastError());
    if (l == 0) break;
    // dZ_{l-1} = (dZ_l W_l) * SiLU'(Z_{l-1}): M = n, N = in_pad (hidden), K = out_pad
    GemmArgs b{};
    b.M = n;
    b.N = L.in_pad[l];
    b.K = L.out_pad[l];
    b.A = dZ;
    b.lda = L.out_pad[l];
    b.B = w.Wt + L.wb_off[l];
    b.ldb = L.out_pad[l];
    b.k_per_split = b.K;
    b.Zin = m->Z[l - 1];
    b.ldz = L.in_pad[l];
    b.O = m->dZ[l - 1];
    b.ldo = L.in_pad[l];
    b.Ot = m->dZt[l - 1];
    b.ldot = n;
    if ((rc = gemm<EPI_HIDDEN_BWD>(m, b, 1, s))) return rc;
  }
  return BD_OK;
}

int check_member(BdMlp* m, int member) {
  if (!m) return BD_ERR_ARG;
  if (member < 0 || member >= m->d.n_members) return mfail(m, BD_ERR_ARG, "member %d out of range", member);
  MCK(m, cudaSetDevice(m->device));
  return BD_OK;
}

}  // namespace

// Ensemble inference for the stepper (same translation unit boundary as the C ABI).
int bd_internal_mlp_ensemble(BdMlp* m, int64_t n, const float* X, float* mean, float* spread, cudaStream_t s) {
  int rc;
  if ((rc = ensure_infer(m))) return rc;
  const LayerGeom& L = m->L;
  const int od = m->d.out_dim;
  for (int64_t r0 = 0; r0 < n; r0 += kChunkRows) {
    const int rows = (int)std::min<int64_t>(kChunkRows, n - r0);
    pack_input_kernel<<<grid_for(m, (long long)rows * L.in_pad[0]), 256, 0, s>>>(
        X + r0 * m->d.in_dim, rows, m->d.in_dim, m->Xi, L.in_pad[0], nullptr, 0);
    MCK(m, cudaGetLastError());
    if (tc_eligible(m)) {
      if ((rc = forward_tc(m, 0, m->d.n_members, rows, m->Xi, m->Ys, od, (long long)m->infer_cap * od, s))) return rc;
    } else {
      for (int k = 0; k < m->d.n_members; ++k)
        if ((rc = forward(m, k, rows, m->Xi, m->Ys + (size_t)k * m->infer_cap * od, od, false, s))) return rc;
    }
    ensemble_kernel<<<grid_for(m, (long long)rows * od), 256, 0, s>>>(
        m->Ys, m->d.n_members, (long long)m->infer_cap * od, rows, od, mean + r0 * od,
        spread ? spread + r0 * od : nullptr, nullptr);
    MCK(m, cudaGetLastError());
  }
  return BD_OK;
}

int adam_update(BdMlp* m, int member, float lr, cudaStream_t s) {
  BdMlp::Member& w = m->mem[member];
  adam_kernel<<<grid_for(m, m->n_params), 256, 0, s>>>(w.p, w.grad, w.m1, w.m2, m->n_params, lr, 0.9f, 0.999f, 1e-8f,
                                                        w.step, m->L, w.Wb, w.Wt, w.Wc);
  MCK(m, cudaGetLastError());
  step_increment_kernel<<<1, 1, 0, s>>>(w.step);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

// One training step on a random batch of device-resident data: gather, forward,
// loss, backward, Adam.  Enqueued once under stream capture and replayed.
int enqueue_train_step(BdMlp* m, int member, long long n_data, const float* X, const float* T, int batch, float lr,
                       unsigned long long seed, float* trace, cudaStream_t s) {
  gather_batch_kernel<<<grid_for(m, batch), 256, 0, s>>>(X, T, n_data, m->d.in_dim, m->d.out_dim, batch, seed,
                                                         m->data_step, m->Xbatch, m->Tbatch);
  MCK(m, cudaGetLastError());
  int rc = backward(m, member, batch, m->Xbatch, m->Tbatch, nullptr, s, trace);
  if (rc) return rc;
  if ((rc = adam_update(m, member, lr, s))) return rc;
  step_increment_kernel<<<1, 1, 0, s>>>(m->data_step);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

// The stepper's view: shape checks, buffers for `rows` rows (before any graph
// capture), and the ensemble on packed BF16 feature rows whose count is on the device.
int bd_internal_mlp_shape(const BdMlp* m, int* in_dim, int* in_pad, int* out_dim) {
  *in_dim = m->d.in_dim;
  *in_pad = m->L.in_pad[0];
  *out_dim = m->d.out_dim;
  return BD_OK;
}

int bd_internal_mlp_prepare(BdMlp* m, int rows) {
  MCK(m, cudaSetDevice(m->device));
  return ensure_infer(m, rows);
}

int bd_internal_mlp_ensemble_rows(BdMlp* m, int rows, const int* n_dev, const void* Xpacked, float* mean,
                                  float* spread, cudaStream_t s) {
  if (rows > m->infer_cap) return mfail(m, BD_ERR_STATE, "inference buffers hold %d rows, %d asked", m->infer_cap, rows);
  const int od = m->d.out_dim;
  int rc;
  if (tc_eligible(m)) {
    if ((rc = forward_tc(m, 0, m->d.n_members, rows, (const bf16*)Xpacked, m->Ys, od, (long long)m->infer_cap * od,
                         s, n_dev)))
      return rc;
  } else {
    for (int k = 0; k < m->d.n_members; ++k)
      if ((rc = forward(m, k, rows, (const bf16*)Xpacked, m->Ys + (size_t)k * m->infer_cap * od, od, false, s,
                        n_dev)))
        return rc;
  }
  ensemble_kernel<<<grid_for(m, (long long)rows * od), 256, 0, s>>>(m->Ys, m->d.n_members, (long long)m->infer_cap * od,
                                                                     rows, od, mean, spread, n_dev);
  MCK(m, cudaGetLastError());
  return BD_OK;
}

const char* bd_internal_mlp_error(const BdMlp* m) { return m->err.c_str(); }

extern "C" {

int bd_mlp_create(int device, const BdMlpDesc* d, BdMlp** out) {
  if (!out || !d) return BD_ERR_ARG;
  *out = nullptr;
  if (d->n_members < 1 || d->n_members > 8 || d->in_dim < 1 || d->in_dim > 32 || d->hidden < 128 ||
      d->hidden % 128 || d->hidden > 512 || d->n_hidden < 1 || d->n_hidden > kMaxLayers - 1 || d->out_dim < 1 ||
      d->out_dim > 32)
    return BD_ERR_ARG;
  BdMlp* m = new BdMlp();
  m->device = device;
  m->d = *d;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete m;
    return BD_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&m->n_sm, cudaDevAttrMultiProcessorCount, device);
  LayerGeom& L = m->L;
  L.n_layers = d->n_hidden + 1;
  long long off = 0, woff = 0;
  for (int l = 0; l < L.n_layers; ++l) {
    L.in_real[l] = l == 0 ? d->in_dim : d->hidden;
    L.out_real[l] = l + 1 == L.n_layers ? d->out_dim : d->hidden;
    L.in_pad[l] = round_up(L.in_real[l], 32);
    L.out_pad[l] = round_up(L.out_real[l], 32);
    L.w_off[l] = off;
    off += (long long)L.out_real[l] * L.in_real[l];
    L.b_off[l] = off;
    off += L.out_real[l];
    L.wb_off[l] = woff;
    woff += (long long)L.out_pad[l] * L.in_pad[l];
  }
  m->n_params = off;
  m->wb_size = woff;
  m->mem.resize(d->n_members);
  uint64_t seed = d->seed;
  std::vector<float> init(off);
  for (int k = 0; k < d->n_members; ++k) {
    BdMlp::Member& w = m->mem[k];
    void* p;
    int rc = 0;
    if ((rc = malloc_into(m, m->allocs, &p, off * 4))) goto fail;
    w.p = (float*)p;
    if ((rc = malloc_into(m, m->allocs, &p, off * 4))) goto fail;
    w.m1 = (float*)p;
    if ((rc = malloc_into(m, m->allocs, &p, off * 4))) goto fail;
    w.m2 = (float*)p;
    if ((rc = malloc_into(m, m->allocs, &p, off * 4))) goto fail;
    w.grad = (float*)p;
    if ((rc = malloc_into(m, m->allocs, &p, woff * 2))) goto fail;
    w.Wb = (bf16*)p;
    if ((rc = malloc_into(m, m->allocs, &p, woff * 2))) goto fail;
    w.Wt = (bf16*)p;
    if ((rc = malloc_into(m, m->allocs, &p, woff * 2))) goto fail;
    w.Wc = (bf16*)p;
    if ((rc = malloc_into(m, m->allocs, &p, sizeof(long long)))) goto fail;
    w.step = (long long*)p;
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases, member by member
    for (int l = 0; l < L.n_layers; ++l) {
      const float bound = 1.0f / std::sqrt((float)L.in_real[l]);
      for (long long i = L.w_off[l]; i < L.b_off[l] + L.out_real[l]; ++i) {
        const double u = (double)(splitmix(seed) >> 11) * (1.0 / 9007199254740992.0);
        init[i] = (float)((2.0 * u - 1.0) * bound);
      }
    }
    if (cudaMemcpy(w.p, init.data(), off * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = BD_ERR_CUDA;
      goto fail;
    }
    refresh_kernel<<<grid_for(m, off), 256>>>(w.p, off, L, w.Wb, w.Wt, w.Wc);
    continue;
  fail:
    for (void* q : m->allocs) cudaFree(q);
    delete m;
    return rc;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    for (void* q : m->allocs) cudaFree(q);
    delete m;
    return BD_ERR_CUDA;
  }
  *out = m;
  return BD_OK;
}

int bd_mlp_destroy(BdMlp* m) {
  if (!m) return BD_OK;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  if (m->train_graph) cudaGraphExecDestroy(m->train_graph);
  for (void* p : m->train_allocs) cudaFree(p);
  for (void* p : m->infer_allocs) cudaFree(p);
  for (void* p : m->allocs) cudaFree(p);
  delete m;
  return BD_OK;
}

int bd_mlp_last_error(const BdMlp* m, char* buf, int len) {
  if (!buf || len <= 0) return BD_ERR_ARG;
  snprintf(buf, (size_t)len, "%s", m ? m->err.c_str() : "no MLP");
  return BD_OK;
}

int bd_mlp_n_params(const BdMlp* m, int64_t* n) {
  if (!m || !n) return BD_ERR_ARG;
  *n = m->n_params;
  return BD_OK;
}

int bd_mlp_get_params(BdMlp* m, int member, float* params) {
  int rc = check_member(m, member);
  if (rc) return rc;
  if (!params) return mfail(m, BD_ERR_ARG, "params is NULL");
  MCK(m, cudaDeviceSynchronize());
  MCK(m, cudaMemcpy(params, m->mem[member].p, m->n_params * 4, cudaMemcpyDeviceToHost));
  return BD_OK;
}

int bd_mlp_set_params(BdMlp* m, int member, const float* params) {
  int rc = check_member(m, member);
  if (rc) return rc;
  if (!params) return mfail(m, BD_ERR_ARG, "params is NULL");
  BdMlp::Member& w = m->mem[member];
  MCK(m, cudaDeviceSynchronize());
  MCK(m, cudaMemcpy(w.p, params, m->n_params * 4, cudaMemcpyHostToDevice));
  MCK(m, cudaMemset(w.m1, 0, m->n_params * 4));
  MCK(m, cudaMemset(w.m2, 0, m->n_params * 4));
  MCK(m, cudaMemset(w.step, 0, sizeof(long long)));
  refresh_kernel<<<grid_for(m, m->n_params), 256>>>(w.p, m->n_params, m->L, w.Wb, w.Wt, w.Wc);
  MCK(m, cudaGetLastError());
  MCK(m, cudaDeviceSynchronize());
  return BD_OK;
}

int bd_mlp_forward(BdMlp* m, int member, int64_t n, const float* X, float* Y, void* stream) {
  bd::NvtxRange nvtx("bd_mlp_forward");
  int rc = check_member(m, member);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!X || !Y))) return mfail(m, BD_ERR_ARG, "bd_mlp_forward: bad arguments");
  if ((rc = ensure_infer(m))) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  for (int64_t r0 = 0; r0 < n; r0 += kChunkRows) {
    const int rows = (int)std::min<int64_t>(kChunkRows, n - r0);
    pack_input_kernel<<<grid_for(m, (long long)rows * m->L.in_pad[0]), 256, 0, s>>>(
        X + r0 * m->d.in_dim, rows, m->d.in_dim, m->Xi, m->L.in_pad[0], nullptr, 0);
    MCK(m, cudaGetLastError());
    if (tc_eligible(m)) {
      if ((rc = forward_tc(m, member, 1, rows, m->Xi, Y + r0 * m->d.out_dim, m->d.out_dim, 0, s))) return rc;
    } else if ((rc = forward(m, member, rows, m->Xi, Y + r0 * m->d.out_dim, m->d.out_dim, false, s))) {
      return rc;
    }
  }
  return BD_OK;
}

int bd_mlp_grad(BdMlp* m, int member, int n, const float* X, const float* T, float* grad, float* loss, void* stream) {
  int rc = check_member(m, member);
  if (rc) return rc;
  if (n <= 0 || n % 32 || !X || !T) return mfail(m, BD_ERR_ARG, "bd_mlp_grad: n must be a positive multiple of 32");
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = backward(m, member, n, X, T, loss, s))) return rc;
  if (grad) MCK(m, cudaMemcpyAsync(grad, m->mem[member].grad, m->n_params * 4, cudaMemcpyDeviceToDevice, s));
  return BD_OK;
}

int bd_mlp_train_step(BdMlp* m, int member, int n, const float* X, const float* T, float lr, float* loss,
                      void* stream) {
  int rc = check_member(m, member);
  if (rc) return rc;
  if (n <= 0 || n % 32 || !X || !T || !(lr > 0))
    return mfail(m, BD_ERR_ARG, "bd_mlp_train_step: n must be a positive multiple of 32 and lr > 0");
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = backward(m, member, n, X, T, loss, s))) return rc;
  return adam_update(m, member, lr, s);
}

int bd_mlp_train(BdMlp* m, int member, int64_t n_data, const float* X, const float* T, int batch, int steps,
                 float lr, uint64_t seed, float* loss_trace, void* stream) {
  bd::NvtxRange nvtx("bd_mlp_train");
  int rc = check_member(m, member);
  if (rc) return rc;
  if (n_data <= 0 || !X || !T || batch <= 0 || batch % 32 || steps < 0 || !(lr > 0))
    return mfail(m, BD_ERR_ARG, "bd_mlp_train: need data, a batch that is a positive multiple of 32, lr > 0");
  cudaStream_t s = (cudaStream_t)stream;
  if ((rc = ensure_train(m, batch))) return rc;
  if (batch > m->batch_cap) {
    void* p;
    MCK(m, cudaDeviceSynchronize());
    if ((rc = malloc_into(m, m->allocs, &p, (size_t)batch * m->d.in_dim * 4))) return rc;
    m->Xbatch = (float*)p;
    if ((rc = malloc_into(m, m->allocs, &p, (size_t)batch * m->d.out_dim * 4))) return rc;
    m->Tbatch = (float*)p;
    m->batch_cap = batch;
    if (m->train_graph) {
      cudaGraphExecDestroy(m->train_graph);
      m->train_graph = nullptr;
    }
  }
  if (!m->data_step) {
    void* p;
    if ((rc = malloc_into(m, m->allocs, &p, sizeof(long long)))) return rc;
    m->data_step = (long long*)p;
  }
  // the loss trace is indexed by batches drawn since this call began
  MCK(m, cudaMemsetAsync(m->data_step, 0, sizeof(long long), s));
  if (!m->train_graph || m->tg_member != member || m->tg_batch != batch || m->tg_X != X || m->tg_T != T ||
      m->tg_n != n_data || m->tg_lr != lr || m->tg_seed != seed || m->tg_trace != loss_trace) {
    if (m->train_graph) {
      cudaGraphExecDestroy(m->train_graph);
      m->train_graph = nullptr;
    }
    cudaStream_t cs;
    MCK(m, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
      cudaStreamDestroy(cs);
      MCK(m, e);
    }
    rc = enqueue_train_step(m, member, n_data, X, T, batch, lr, seed ^ ((unsigned long long)member << 56), loss_trace,
                            cs);
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc) return rc;
    MCK(m, e);
    e = cudaGraphInstantiate(&m->train_graph, g, 0);
    cudaGraphDestroy(g);
    MCK(m, e);
    m->tg_member = member;
    m->tg_batch = batch;
    m->tg_X = X;
    m->tg_T = T;
    m->tg_n = n_data;
    m->tg_lr = lr;
    m->tg_seed = seed;
    m->tg_trace = loss_trace;
  }
  for (int i = 0; i < steps; ++i) MCK(m, cudaGraphLaunch(m->train_graph, s));
  return BD_OK;
}

int bd_mlp_set_inference(BdMlp* m, int mode) {
  if (!m) return BD_ERR_ARG;
  if (mode != 0 && mode != 1) return mfail(m, BD_ERR_ARG, "inference mode must be 0 (mma.sync) or 1 (tcgen05)");
  m->inference = mode;
  return BD_OK;
}

int bd_mlp_set_gemm(BdMlp* m, int mode) {
  if (!m) return BD_ERR_ARG;
  if (mode != 0 && mode != 1) return mfail(m, BD_ERR_ARG, "GEMM mode must be 0 (mma.sync) or 1 (tcgen05)");
  if (mode != m->gemm_tc && m->train_graph) {  // the captured training step holds the old kernels
    cudaGraphExecDestroy(m->train_graph);
    m->train_graph = nullptr;
    m->tg_member = -1;
  }
  m->gemm_tc = mode;
  return BD_OK;
}

int bd_mlp_ensemble(BdMlp* m, int64_t n, const float* X, float* mean, float* spread, void* stream) {
  bd::NvtxRange nvtx("bd_mlp_ensemble");
  if (!m) return BD_ERR_ARG;
  MCK(m, cudaSetDevice(m->device));
  if (n < 0 || (n > 0 && (!X || !mean))) return mfail(m, BD_ERR_ARG, "bd_mlp_ensemble: bad arguments");
  return bd_internal_mlp_ensemble(m, n, X, mean, spread, (cudaStream_t)stream);
}

}  // extern "C"
