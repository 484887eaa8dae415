// mlp.cu — the learned read-cost model behind the SMEM scheduler (include/hfm.h,
// hfm_mlp_*): per-read features, a 258 -> 128 -> 128 -> 3 ReLU MLP with its forward and
// backward passes on the tensor cores (BF16 operands, FP32 accumulation,
// mma.sync.m16n8k16), Adam, and the binning of reads by predicted cost.
//
// Features of read q (length L): x[f] = 256 * c_f / V - 1 for the 256 4-mers f over ACGT
// (c_f occurrences, V = 4-mers without an ambiguity code; all 0 when V == 0), x[256] =
// (log2(L + 1) - 10) / 4, x[257] = (L - 3 - V) / (L - 3), the share of 4-mers holding an
// ambiguity code (0 when L < 4), x[258..271] = 0 (padding to the MMA K step).  Outputs predict
// log1p of the exact kernel's per-read work log: Occ touches, MemHits, positions.
//
// One CTA owns a tile of 128 reads; each of its 8 warps owns 16 rows and computes all 128
// hidden units of its rows, so activations never cross warps in the forward pass.  The
// weights (W1 70 KB, W2 34 KB as BF16) sit in shared memory next to the activation tiles.
// Training CTAs write per-tile gradient partials, reduced in a fixed order (the result does
// not depend on scheduling), then one Adam step updates the FP32 master weights and their
// BF16 copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "hfm_internal.h"

namespace hfm {
namespace mlp {

constexpr int IN = 258, INP = HFM_MLP_IN_PAD, HID = HFM_MLP_HIDDEN, OUT = HFM_MLP_OUT;
constexpr int TILE = 128, THREADS = 256;
constexpr int XS = 280;   // shared row stride (bf16) of 272-wide tiles: conflict-free fragment loads
constexpr int HS = 136;   // shared row stride (bf16) of 128-wide tiles
constexpr int P_W1 = 0, P_B1 = P_W1 + HID * INP, P_W2 = P_B1 + HID, P_B2 = P_W2 + HID * HID,
              P_W3 = P_B2 + HID, P_B3 = P_W3 + OUT * HID, NPARAM = P_B3 + OUT;
static_assert(NPARAM == HFM_MLP_NPARAM, "parameter layout");

// shared memory map (bytes)
constexpr int SZ_X = TILE * XS * 2;          // 71,680
constexpr int SZ_H = TILE * HS * 2;          // 34,816
constexpr int OFF_A = 0;                     // W1; training: H2 then dH1, and dH2
constexpr int OFF_B = OFF_A + SZ_X;          // X tile; inference: H2
constexpr int OFF_C = OFF_B + SZ_X;          // H1
constexpr int OFF_D = OFF_C + SZ_H;          // W2
constexpr int OFF_E = OFF_D + SZ_H;          // fp32: W3[3][128], b1, b2, b3, dY[128][3], scratch
constexpr int E_W3 = 0, E_B1 = E_W3 + OUT * HID, E_B2 = E_B1 + HID, E_B3 = E_B2 + HID, E_DY = E_B3 + 4,
              E_RED = E_DY + TILE * OUT, E_END = E_RED + THREADS;
constexpr int SMEM_BYTES = OFF_E + E_END * 4;
static_assert(2 * SZ_H <= SZ_X, "H2 and dH2 share the W1 region");
static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");

__device__ __forceinline__ float bf2f(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }
__device__ __forceinline__ uint16_t f2bf(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) { return (uint32_t)lo | ((uint32_t)hi << 16); }

__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// acc[nt] (16 x 8 tile nt of this warp) += A[16 x K] * B[K x 8*NT].  la(r, k) returns the
// BF16 pair {A[r][k], A[r][k+1]}, lb(k, n) the pair {B[k][n], B[k+1][n]} (k even).
// Fragment layout of m16n8k16: lane = 4*g + t; a0 = A[g][2t..], a1 = A[g+8][2t..],
// a2 = A[g][2t+8..], a3 = A[g+8][2t+8..]; b0 = B[2t..][g], b1 = B[2t+8..][g];
// c0,c1 = C[g][2t, 2t+1], c2,c3 = C[g+8][2t, 2t+1].
template <int NT, class LA, class LB>
__device__ __forceinline__ void warp_gemm(float (&acc)[NT][4], int K, LA la, LB lb) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t a0 = la(g, k0 + 2 * t), a1 = la(g + 8, k0 + 2 * t);
    uint32_t a2 = la(g, k0 + 2 * t + 8), a3 = la(g + 8, k0 + 2 * t + 8);
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      uint32_t b0 = lb(k0 + 2 * t, nt * 8 + g), b1 = lb(k0 + 2 * t + 8, nt * 8 + g);
      mma_bf16(acc[nt], a0, a1, a2, a3, b0, b1);
    }
  }
}

template <int NT>
__device__ __forceinline__ void zero(float (&acc)[NT][4]) {
#pragma unroll
  for (int i = 0; i < NT; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
}

struct Params {
  const uint16_t* w1h; const uint16_t* w2h; const uint16_t* w3h;   // BF16 copies
  const float* master;                                             // biases read from here
};

__device__ void load_weights(const Params& P, unsigned char* sm, bool with_w1) {
  uint16_t* sW1 = (uint16_t*)(sm + OFF_A);
  uint16_t* sW2 = (uint16_t*)(sm + OFF_D);
  float* sE = (float*)(sm + OFF_E);
  if (with_w1)
    for (int k = threadIdx.x; k < HID * (INP / 8); k += THREADS) {
      int r = k / (INP / 8), c = k % (INP / 8);
      reinterpret_cast<uint4*>(sW1 + r * XS)[c] = reinterpret_cast<const uint4*>(P.w1h + r * INP)[c];
    }
  for (int k = threadIdx.x; k < HID * (HID / 8); k += THREADS) {
    int r = k / (HID / 8), c = k % (HID / 8);
    reinterpret_cast<uint4*>(sW2 + r * HS)[c] = reinterpret_cast<const uint4*>(P.w2h + r * HID)[c];
  }
  for (int k = threadIdx.x; k < OUT * HID; k += THREADS) sE[E_W3 + k] = bf2f(P.w3h[k]);
  for (int k = threadIdx.x; k < HID; k += THREADS) {
    sE[E_B1 + k] = P.master[P_B1 + k];
    sE[E_B2 + k] = P.master[P_B2 + k];
  }
  if (threadIdx.x < OUT) sE[E_B3 + threadIdx.x] = P.master[P_B3 + threadIdx.x];
}

// X rows of tile `tile` (row ids from `rows`, or consecutive) into the X region; rows past
// n are zero.
__device__ void load_x(unsigned char* sm, const uint16_t* X, const uint32_t* rows, uint32_t n, uint32_t tile) {
  uint16_t* sX = (uint16_t*)(sm + OFF_B);
  for (int k = threadIdx.x; k < TILE * (INP / 8); k += THREADS) {
    int r = k / (INP / 8), c = k % (INP / 8);
    uint32_t b = tile * TILE + r;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (b < n) {
      uint32_t row = rows ? rows[b] : b;
      v = reinterpret_cast<const uint4*>(X + (size_t)row * INP)[c];
    }
    reinterpret_cast<uint4*>(sX + r * XS)[c] = v;
  }
}

// H = relu(A * W^T + bias) for this warp's 16 rows, BF16 into H (stride HS).
template <int NT>
__device__ __forceinline__ void dense_relu(const float (&acc)[NT][4], const float* bias, uint16_t* H, int rb) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
    int col = nt * 8 + 2 * t;
    float b0 = bias[col], b1 = bias[col + 1];
    *reinterpret_cast<uint32_t*>(H + (rb + g) * HS + col) =
        pack2(f2bf(fmaxf(acc[nt][0] + b0, 0.f)), f2bf(fmaxf(acc[nt][1] + b1, 0.f)));
    *reinterpret_cast<uint32_t*>(H + (rb + g + 8) * HS + col) =
        pack2(f2bf(fmaxf(acc[nt][2] + b0, 0.f)), f2bf(fmaxf(acc[nt][3] + b1, 0.f)));
  }
}

// Forward pass of this warp's 16 rows: X (OFF_B) -> H1 (OFF_C) -> H2 (h2) ; returns nothing,
// Y computed by the caller from H2.
__device__ __forceinline__ void forward_rows(unsigned char* sm, uint16_t* sH2, int rb) {
  const uint16_t* sX = (const uint16_t*)(sm + OFF_B);
  const uint16_t* sW1 = (const uint16_t*)(sm + OFF_A);
  const uint16_t* sW2 = (const uint16_t*)(sm + OFF_D);
  uint16_t* sH1 = (uint16_t*)(sm + OFF_C);
  const float* sE = (const float*)(sm + OFF_E);
  float acc[HID / 8][4];
  zero(acc);
  warp_gemm<HID / 8>(acc, INP,
      [&](int r, int k) { return *reinterpret_cast<const uint32_t*>(sX + (rb + r) * XS + k); },
      [&](int k, int n) { return *reinterpret_cast<const uint32_t*>(sW1 + n * XS + k); });
  dense_relu(acc, sE + E_B1, sH1, rb);
  __syncwarp();
  zero(acc);
  warp_gemm<HID / 8>(acc, HID,
      [&](int r, int k) { return *reinterpret_cast<const uint32_t*>(sH1 + (rb + r) * HS + k); },
      [&](int k, int n) { return *reinterpret_cast<const uint32_t*>(sW2 + n * HS + k); });
  __syncwarp();   // in inference H2 overwrites this warp's own X rows
  dense_relu(acc, sE + E_B2, sH2, rb);
  __syncwarp();
}

// Y[b][o] of this warp's rows (fp32 CUDA-core dot products of the BF16 H2 row and W3).
__device__ __forceinline__ float out_dot(const uint16_t* sH2, const float* sE, int b, int o) {
  float s = sE[E_B3 + o];
  const uint16_t* h = sH2 + b * HS;
  const float* w = sE + E_W3 + o * HID;
  for (int j = 0; j < HID; j++) s = fmaf(bf2f(h[j]), w[j], s);
  return s;
}

// Inference: persistent over tiles; Y[row][3].
__global__ void __launch_bounds__(THREADS, 1) k_mlp_forward(Params P, const uint16_t* __restrict__ X, uint32_t n,
                                                            float* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char sm[];
  load_weights(P, sm, true);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, rb = w * 16;
  uint32_t ntiles = (n + TILE - 1) / TILE;
  uint16_t* sH2 = (uint16_t*)(sm + OFF_B);
  const float* sE = (const float*)(sm + OFF_E);
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    __syncthreads();                 // previous tile's H2 reads done before X is replaced
    load_x(sm, X, nullptr, n, tile);
    __syncthreads();
    forward_rows(sm, sH2, rb);
    for (int k = lane; k < 16 * OUT; k += 32) {
      int r = k / OUT, o = k % OUT;
      uint32_t b = tile * TILE + rb + r;
      if (b < n) Y[(size_t)b * OUT + o] = out_dot(sH2, sE, rb + r, o);
    }
  }
}

// Training tile: forward, MSE loss against T (rows[b] indexes X and T), backward; writes
// this tile's gradient partial gpart[tile][NPARAM] and loss partial lpart[tile].
// inv = 1 / (rows in the whole batch * OUT): the loss is the batch mean.
__global__ void __launch_bounds__(THREADS, 1) k_mlp_train_tile(Params P, const uint16_t* __restrict__ X,
                                                               const float* __restrict__ T,
                                                               const uint32_t* __restrict__ rows, uint32_t n,
                                                               float inv, float* __restrict__ gpart,
                                                               float* __restrict__ lpart) {
  extern __shared__ __align__(16) unsigned char sm[];
  const uint32_t tile = blockIdx.x;
  load_weights(P, sm, true);
  load_x(sm, X, rows, n, tile);
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, rb = w * 16;
  const int g = lane >> 2, t = lane & 3;
  uint16_t* sH2 = (uint16_t*)(sm + OFF_A);            // W1 is dead once layer 1 is done ...
  uint16_t* sdH2 = (uint16_t*)(sm + OFF_A + SZ_H);
  uint16_t* sdH1 = (uint16_t*)(sm + OFF_A);           // ... and H2 once dH2 exists
  const uint16_t* sX = (const uint16_t*)(sm + OFF_B);
  const uint16_t* sH1 = (const uint16_t*)(sm + OFF_C);
  const uint16_t* sW2 = (const uint16_t*)(sm + OFF_D);
  float* sE = (float*)(sm + OFF_E);
  float* gp = gpart + (size_t)tile * NPARAM;

  // forward (layer 1 reads W1 from the region H2 will take: all warps finish it first)
  {
    const uint16_t* sW1 = (const uint16_t*)(sm + OFF_A);
    uint16_t* h1 = (uint16_t*)(sm + OFF_C);
    float acc[HID / 8][4];
    zero(acc);
    warp_gemm<HID / 8>(acc, INP,
        [&](int r, int k) { return *reinterpret_cast<const uint32_t*>(sX + (rb + r) * XS + k); },
        [&](int k, int n2) { return *reinterpret_cast<const uint32_t*>(sW1 + n2 * XS + k); });
    dense_relu(acc, sE + E_B1, h1, rb);
    __syncthreads();
    zero(acc);
    warp_gemm<HID / 8>(acc, HID,
        [&](int r, int k) { return *reinterpret_cast<const uint32_t*>(sH1 + (rb + r) * HS + k); },
        [&](int k, int n2) { return *reinterpret_cast<const uint32_t*>(sW2 + n2 * HS + k); });
    dense_relu(acc, sE + E_B2, sH2, rb);
  }
  __syncwarp();
  // outputs, loss and dY (rows past n contribute nothing)
  float lsum = 0.f;
  for (int k = lane; k < 16 * OUT; k += 32) {
    int r = k / OUT, o = k % OUT;
    uint32_t b = tile * TILE + rb + r;
    float dy = 0.f;
    if (b < n) {
      float y = out_dot(sH2, sE, rb + r, o);
      float d = y - T[(size_t)rows[b] * OUT + o];
      lsum += d * d;
      dy = 2.f * d * inv;
    }
    sE[E_DY + (rb + r) * OUT + o] = dy;
  }
  sE[E_RED + threadIdx.x] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int k = 0; k < THREADS; k++) s += sE[E_RED + k];
    lpart[tile] = s;
  }
  // dW3[o][j] = sum_b dY[b][o] H2[b][j]; db3
  for (int k = threadIdx.x; k < OUT * HID; k += THREADS) {
    int o = k / HID, j = k % HID;
    float s = 0.f;
    for (int b = 0; b < TILE; b++) s = fmaf(sE[E_DY + b * OUT + o], bf2f(sH2[b * HS + j]), s);
    gp[P_W3 + k] = s;
  }
  if (threadIdx.x < OUT) {
    float s = 0.f;
    for (int b = 0; b < TILE; b++) s += sE[E_DY + b * OUT + threadIdx.x];
    gp[P_B3 + threadIdx.x] = s;
  }
  // dH2 = (dY W3) * [H2 > 0]
  for (int k = threadIdx.x; k < TILE * HID; k += THREADS) {
    int b = k / HID, j = k % HID;
    float h = bf2f(sH2[b * HS + j]);
    float s = 0.f;
    if (h > 0.f)
      for (int o = 0; o < OUT; o++) s = fmaf(sE[E_DY + b * OUT + o], sE[E_W3 + o * HID + j], s);
    sdH2[b * HS + j] = f2bf(s);
  }
  __syncthreads();
  // dW2[j][i] = sum_b dH2[b][j] H1[b][i] (this warp: j in rb..rb+15); db2
  {
    float acc[HID / 8][4];
    zero(acc);
    warp_gemm<HID / 8>(acc, TILE,
        [&](int r, int k) { return pack2(sdH2[k * HS + rb + r], sdH2[(k + 1) * HS + rb + r]); },
        [&](int k, int n2) { return pack2(sH1[k * HS + n2], sH1[(k + 1) * HS + n2]); });
#pragma unroll
    for (int nt = 0; nt < HID / 8; nt++) {
      int col = nt * 8 + 2 * t;
      gp[P_W2 + (rb + g) * HID + col] = acc[nt][0];
      gp[P_W2 + (rb + g) * HID + col + 1] = acc[nt][1];
      gp[P_W2 + (rb + g + 8) * HID + col] = acc[nt][2];
      gp[P_W2 + (rb + g + 8) * HID + col + 1] = acc[nt][3];
    }
  }
  if (threadIdx.x < HID) {
    float s = 0.f;
    for (int b = 0; b < TILE; b++) s += bf2f(sdH2[b * HS + threadIdx.x]);
    gp[P_B2 + threadIdx.x] = s;
  }
  // dH1 = (dH2 W2) * [H1 > 0] for this warp's rows, into the H2 region
  {
    float acc[HID / 8][4];
    zero(acc);
    warp_gemm<HID / 8>(acc, HID,
        [&](int r, int k) { return *reinterpret_cast<const uint32_t*>(sdH2 + (rb + r) * HS + k); },
        [&](int k, int n2) { return pack2(sW2[k * HS + n2], sW2[(k + 1) * HS + n2]); });
#pragma unroll
    for (int nt = 0; nt < HID / 8; nt++) {
      int col = nt * 8 + 2 * t;
      const uint16_t* h0 = sH1 + (rb + g) * HS + col;
      const uint16_t* h8 = sH1 + (rb + g + 8) * HS + col;
      *reinterpret_cast<uint32_t*>(sdH1 + (rb + g) * HS + col) =
          pack2(f2bf(bf2f(h0[0]) > 0.f ? acc[nt][0] : 0.f), f2bf(bf2f(h0[1]) > 0.f ? acc[nt][1] : 0.f));
      *reinterpret_cast<uint32_t*>(sdH1 + (rb + g + 8) * HS + col) =
          pack2(f2bf(bf2f(h8[0]) > 0.f ? acc[nt][2] : 0.f), f2bf(bf2f(h8[1]) > 0.f ? acc[nt][3] : 0.f));
    }
  }
  __syncthreads();
  // dW1[j][f] = sum_b dH1[b][j] X[b][f] in two halves of 136 columns; db1
  for (int half = 0; half < 2; half++) {
    const int n0 = half * (INP / 2);
    float acc[INP / 16][4];
    zero(acc);
    warp_gemm<INP / 16>(acc, TILE,
        [&](int r, int k) { return pack2(sdH1[k * HS + rb + r], sdH1[(k + 1) * HS + rb + r]); },
        [&](int k, int n2) { return pack2(sX[k * XS + n0 + n2], sX[(k + 1) * XS + n0 + n2]); });
#pragma unroll
    for (int nt = 0; nt < INP / 16; nt++) {
      int col = n0 + nt * 8 + 2 * t;
      gp[P_W1 + (rb + g) * INP + col] = acc[nt][0];
      gp[P_W1 + (rb + g) * INP + col + 1] = acc[nt][1];
      gp[P_W1 + (rb + g + 8) * INP + col] = acc[nt][2];
      gp[P_W1 + (rb + g + 8) * INP + col + 1] = acc[nt][3];
    }
  }
  if (threadIdx.x < HID) {
    float s = 0.f;
    for (int b = 0; b < TILE; b++) s += bf2f(sdH1[b * HS + threadIdx.x]);
    gp[P_B1 + threadIdx.x] = s;
  }
}

// grad[p] = sum over tiles of gpart[tile][p], tiles in order.
__global__ void k_reduce_tiles(const float* __restrict__ gpart, uint32_t ntiles, float* __restrict__ grad,
                               const float* __restrict__ lpart, double* __restrict__ loss_acc) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NPARAM) {
    float s = 0.f;
    for (uint32_t k = 0; k < ntiles; k++) s += gpart[(size_t)k * NPARAM + p];
    grad[p] = s;
  }
  if (p == 0 && loss_acc) {
    double s = 0.0;
    for (uint32_t k = 0; k < ntiles; k++) s += lpart[k];
    *loss_acc += s;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; refreshes the BF16 copies.
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, float lr, float b1, float b2, float eps, float c1, float c2,
                       uint16_t* __restrict__ w1h, uint16_t* __restrict__ w2h, uint16_t* __restrict__ w3h) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  float g = grad[p];
  float mm = b1 * m[p] + (1.f - b1) * g;
  float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm; v[p] = vv;
  float x = w[p] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[p] = x;
  if (p < P_B1) w1h[p - P_W1] = f2bf(x);
  else if (p >= P_W2 && p < P_B2) w2h[p - P_W2] = f2bf(x);
  else if (p >= P_W3 && p < P_B3) w3h[p - P_W3] = f2bf(x);
}

__global__ void k_to_bf16(const float* __restrict__ w, uint16_t* __restrict__ w1h, uint16_t* __restrict__ w2h,
                          uint16_t* __restrict__ w3h) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  if (p < P_B1) w1h[p - P_W1] = f2bf(w[p]);
  else if (p >= P_W2 && p < P_B2) w2h[p - P_W2] = f2bf(w[p]);
  else if (p >= P_W3 && p < P_B3) w3h[p - P_W3] = f2bf(w[p]);
}

// One warp per read: 4-mer histogram in shared memory, then the feature row.
constexpr int FEAT_WARPS = 8;
__global__ void __launch_bounds__(FEAT_WARPS * 32) k_features(const uint8_t* __restrict__ q,
                                                              const uint64_t* __restrict__ qoff, uint32_t nq,
                                                              uint16_t* __restrict__ X) {
  __shared__ uint32_t hist[FEAT_WARPS][256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* hw = hist[w];
  for (uint32_t i = blockIdx.x * FEAT_WARPS + w; i < nq; i += gridDim.x * FEAT_WARPS) {
    for (int k = lane; k < 256; k += 32) hw[k] = 0;
    __syncwarp();
    uint64_t o = qoff[i];
    uint32_t len = (uint32_t)(qoff[i + 1] - o);
    uint32_t valid = 0;
    for (uint32_t p = lane; p + 3 < len; p += 32) {
      uint32_t c0 = q[o + p] - 1u, c1 = q[o + p + 1] - 1u, c2 = q[o + p + 2] - 1u, c3 = q[o + p + 3] - 1u;
      if ((c0 | c1 | c2 | c3) < 4u) {
        atomicAdd(hw + ((c0 << 6) | (c1 << 4) | (c2 << 2) | c3), 1u);
        valid++;
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) valid += __shfl_xor_sync(0xFFFFFFFFu, valid, d);
    __syncwarp();
    uint16_t* xr = X + (size_t)i * INP;
    for (int k = lane; k < INP / 2; k += 32) {
      float f[2];
      for (int e = 0; e < 2; e++) {
        int c = 2 * k + e;
        if (c < 256) f[e] = valid ? (float)(256u * hw[c]) / (float)valid - 1.f : 0.f;
        else if (c == 256) f[e] = (log2f((float)len + 1.f) - 10.f) * 0.25f;
        else if (c == 257) f[e] = len >= 4 ? (float)(len - 3 - valid) / (float)(len - 3) : 0.f;
        else f[e] = 0.f;
      }
      reinterpret_cast<uint32_t*>(xr)[k] = pack2(f2bf(f[0]), f2bf(f[1]));
    }
    __syncwarp();
  }
}

// ---- scheduling: reads binned by predicted cost, costliest first --------------------------
constexpr int NBINS = 4096;
constexpr float BIN_SCALE = NBINS / 24.f;   // log1p(touches) in [0, 24)

__device__ __forceinline__ uint32_t sched_bin(const float* y, float warp_hits_min_log) {
  // bin 0: routed to the warp-per-read kernel; then descending predicted touches
  if (y[1] >= warp_hits_min_log) return 0;
  float c = fminf(fmaxf(y[0] * BIN_SCALE, 0.f), (float)(NBINS - 2));
  return (uint32_t)(NBINS - 1) - (uint32_t)c;
}

__global__ void k_bin_hist(const float* __restrict__ y, uint32_t n, float wl, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[NBINS];
  for (int k = threadIdx.x; k < NBINS; k += blockDim.x) h[k] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(h + sched_bin(y + (size_t)i * OUT, wl), 1u);
  __syncthreads();
  for (int k = threadIdx.x; k < NBINS; k += blockDim.x)
    if (h[k]) atomicAdd(hist + k, h[k]);
}

// exclusive scan of the bins (one block of 1024 threads, 4 bins each)
__global__ void k_bin_scan(uint32_t* __restrict__ hist, uint32_t* __restrict__ n_warp) {
  __shared__ uint32_t s[1024];
  int t = threadIdx.x;
  uint32_t v[4], sum = 0;
  for (int e = 0; e < 4; e++) { v[e] = hist[4 * t + e]; sum += v[e]; }
  s[t] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    uint32_t x = t >= d ? s[t - d] : 0;
    __syncthreads();
    s[t] += x;
    __syncthreads();
  }
  uint32_t base = s[t] - sum;
  if (t == 0) *n_warp = v[0];
  for (int e = 0; e < 4; e++) { hist[4 * t + e] = base; base += v[e]; }
}

__global__ void k_bin_scatter(const float* __restrict__ y, uint32_t n, float wl, uint32_t* __restrict__ cursor,
                              uint32_t* __restrict__ order) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  order[atomicAdd(cursor + sched_bin(y + (size_t)i * OUT, wl), 1u)] = i;
}

}  // namespace mlp
}  // namespace hfm

// =====================================================================================
// C ABI
// =====================================================================================
using namespace hfm;
using namespace hfm::mlp;

#define MCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess) return set_error(HFM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

struct hfm_mlp {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  uint16_t *w1h = nullptr, *w2h = nullptr, *w3h = nullptr;
  uint64_t step = 0;
  // grow-only scratch
  float* gpart = nullptr; size_t gpart_cap = 0;
  float* lpart = nullptr; size_t lpart_cap = 0;
  uint32_t* perm = nullptr; size_t perm_cap = 0;
  uint16_t* x = nullptr; size_t x_cap = 0;
  uint32_t* bins = nullptr;
  double* loss_acc = nullptr;
};

namespace {

int grow(void** p, size_t* cap, size_t bytes) {
  if (*cap >= bytes) return HFM_OK;
  if (*p) cudaFree(*p);
  *p = nullptr; *cap = 0;
  if (cudaMalloc(p, bytes) != cudaSuccess) { cudaGetLastError(); return set_error(HFM_E_OOM, "MLP scratch allocation failed"); }
  *cap = bytes;
  return HFM_OK;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) { cudaGetDevice(&prev); if (prev != d) cudaSetDevice(d); }
  ~DevGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

Params params_of(const hfm_mlp* m) { return Params{m->w1h, m->w2h, m->w3h, m->w}; }

int sync(hfm_mlp* m) {
  MCK(cudaGetLastError());
  MCK(cudaStreamSynchronize(m->stream));
  return HFM_OK;
}

// one batch: forward + backward over `n` rows listed in rows (device), into m->grad
int batch_grad(hfm_mlp* m, const uint16_t* X, const float* T, const uint32_t* rows, uint32_t n, double* loss_acc) {
  uint32_t ntiles = (n + TILE - 1) / TILE;
  int rc;
  if ((rc = grow((void**)&m->gpart, &m->gpart_cap, (size_t)ntiles * NPARAM * 4))) return rc;
  if ((rc = grow((void**)&m->lpart, &m->lpart_cap, (size_t)ntiles * 4))) return rc;
  k_mlp_train_tile<<<ntiles, THREADS, SMEM_BYTES, m->stream>>>(params_of(m), X, T, rows, n, 1.f / ((float)n * OUT),
                                                               m->gpart, m->lpart);
  k_reduce_tiles<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->gpart, ntiles, m->grad, m->lpart,
                                                              loss_acc);
  MCK(cudaGetLastError());
  return HFM_OK;
}

int identity_rows(hfm_mlp* m, uint32_t n) {
  int rc;
  if ((rc = grow((void**)&m->perm, &m->perm_cap, (size_t)n * 4 + 4))) return rc;
  std::vector<uint32_t> id(n);
  for (uint32_t i = 0; i < n; i++) id[i] = i;
  if (n) MCK(cudaMemcpyAsync(m->perm, id.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
  return sync(m);
}

}  // namespace

extern "C" {

int hfm_mlp_create(int device, uint64_t seed, hfm_mlp** out) {
  if (!out) return set_error(HFM_E_ARG, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  MCK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_error(HFM_E_ARG, "no such CUDA device");
  DevGuard dg(device);
  hfm_mlp* m = new hfm_mlp();
  m->device = device;
  auto fail = [&](int rc) { hfm_mlp_free(m); return rc; };
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(set_error(HFM_E_CUDA, "stream"));
  cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device);
  size_t f = (size_t)NPARAM * 4;
  if (cudaMalloc(&m->w, f) || cudaMalloc(&m->m, f) || cudaMalloc(&m->v, f) || cudaMalloc(&m->grad, f) ||
      cudaMalloc(&m->w1h, (size_t)HID * INP * 2) || cudaMalloc(&m->w2h, (size_t)HID * HID * 2) ||
      cudaMalloc(&m->w3h, (size_t)OUT * HID * 2) || cudaMalloc(&m->bins, (size_t)NBINS * 4 + 16) ||
      cudaMalloc(&m->loss_acc, 8)) {
    cudaGetLastError();
    return fail(set_error(HFM_E_OOM, "MLP allocation failed"));
  }
  if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) ||
      cudaFuncSetAttribute(k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES)) {
    cudaGetLastError();
    return fail(set_error(HFM_E_CUDA, "shared memory opt-in failed"));
  }
  // He-uniform weights (bound sqrt(6 / fan_in)), zero biases, from a splitmix64 stream
  std::vector<float> w(NPARAM, 0.f);
  uint64_t s = seed;
  auto uni = [&](float a) { return (float)((double)(splitmix(s) >> 11) * 0x1.0p-53 * 2.0 - 1.0) * a; };
  for (int j = 0; j < HID; j++) for (int c = 0; c < IN; c++) w[P_W1 + j * INP + c] = uni(std::sqrt(6.f / IN));
  for (int j = 0; j < HID * HID; j++) w[P_W2 + j] = uni(std::sqrt(6.f / HID));
  for (int j = 0; j < OUT * HID; j++) w[P_W3 + j] = uni(std::sqrt(6.f / HID));
  int rc = hfm_mlp_set_params(m, w.data());
  if (rc) return fail(rc);
  *out = m;
  return HFM_OK;
}

void hfm_mlp_free(hfm_mlp* m) {
  if (!m) return;
  DevGuard dg(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (void* p : {(void*)m->w, (void*)m->m, (void*)m->v, (void*)m->grad, (void*)m->w1h, (void*)m->w2h,
                  (void*)m->w3h, (void*)m->gpart, (void*)m->lpart, (void*)m->perm, (void*)m->x, (void*)m->bins,
                  (void*)m->loss_acc})
    if (p) cudaFree(p);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

int hfm_mlp_set_params(hfm_mlp* m, const float* params) {
  if (!m || !params) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  MCK(cudaMemcpyAsync(m->w, params, (size_t)NPARAM * 4, cudaMemcpyHostToDevice, m->stream));
  MCK(cudaMemsetAsync(m->m, 0, (size_t)NPARAM * 4, m->stream));
  MCK(cudaMemsetAsync(m->v, 0, (size_t)NPARAM * 4, m->stream));
  m->step = 0;
  k_to_bf16<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->w, m->w1h, m->w2h, m->w3h);
  return sync(m);
}

int hfm_mlp_get_params(hfm_mlp* m, float* params) {
  if (!m || !params) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  MCK(cudaMemcpyAsync(params, m->w, (size_t)NPARAM * 4, cudaMemcpyDeviceToHost, m->stream));
  return sync(m);
}

void* hfm_mlp_stream(hfm_mlp* m) { return m ? (void*)m->stream : nullptr; }

int hfm_mlp_features(hfm_mlp* m, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, uint16_t* d_x) {
  if (!m || (nq && (!d_q_off || !d_x))) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  if (nq) {
    unsigned grid = (unsigned)std::min<uint64_t>((nq + FEAT_WARPS - 1) / FEAT_WARPS, (uint64_t)m->num_sms * 8);
    k_features<<<grid, FEAT_WARPS * 32, 0, m->stream>>>(d_q, d_q_off, nq, d_x);
  }
  return sync(m);
}

int hfm_mlp_forward(hfm_mlp* m, const uint16_t* d_x, uint32_t n, float* d_y) {
  if (!m || (n && (!d_x || !d_y))) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  if (n) {
    uint32_t ntiles = (n + TILE - 1) / TILE;
    unsigned grid = (unsigned)std::min<uint32_t>(ntiles, (uint32_t)m->num_sms);
    k_mlp_forward<<<grid, THREADS, SMEM_BYTES, m->stream>>>(params_of(m), d_x, n, d_y);
  }
  return sync(m);
}

int hfm_mlp_predict(hfm_mlp* m, const uint8_t* d_q, const uint64_t* d_q_off, uint32_t nq, float* d_y) {
  if (!m || (nq && (!d_q_off || !d_y))) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  if (!nq) return HFM_OK;
  int rc;
  if ((rc = grow((void**)&m->x, &m->x_cap, (size_t)nq * INP * 2))) return rc;
  unsigned fgrid = (unsigned)std::min<uint64_t>((nq + FEAT_WARPS - 1) / FEAT_WARPS, (uint64_t)m->num_sms * 8);
  k_features<<<fgrid, FEAT_WARPS * 32, 0, m->stream>>>(d_q, d_q_off, nq, m->x);
  uint32_t ntiles = (nq + TILE - 1) / TILE;
  k_mlp_forward<<<std::min<uint32_t>(ntiles, (uint32_t)m->num_sms), THREADS, SMEM_BYTES, m->stream>>>(
      params_of(m), m->x, nq, d_y);
  return sync(m);
}

int hfm_mlp_grad(hfm_mlp* m, const uint16_t* d_x, const float* d_t, uint32_t n, float* d_grad, float* loss) {
  if (!m || !d_grad || (n && (!d_x || !d_t))) return set_error(HFM_E_ARG, "NULL argument");
  if (n == 0) return set_error(HFM_E_ARG, "empty batch");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  int rc;
  if ((rc = identity_rows(m, n))) return rc;
  MCK(cudaMemsetAsync(m->loss_acc, 0, 8, m->stream));
  if ((rc = batch_grad(m, d_x, d_t, m->perm, n, m->loss_acc))) return rc;
  MCK(cudaMemcpyAsync(d_grad, m->grad, (size_t)NPARAM * 4, cudaMemcpyDeviceToDevice, m->stream));
  double l = 0;
  MCK(cudaMemcpyAsync(&l, m->loss_acc, 8, cudaMemcpyDeviceToHost, m->stream));
  if ((rc = sync(m))) return rc;
  if (loss) *loss = (float)(l / ((double)n * OUT));
  return HFM_OK;
}

int hfm_mlp_train(hfm_mlp* m, const uint16_t* d_x, const float* d_t, uint32_t n, uint32_t epochs, uint32_t batch,
                  float lr, uint64_t seed, float* loss_per_epoch) {
  if (!m || (n && (!d_x || !d_t))) return set_error(HFM_E_ARG, "NULL argument");
  if (n == 0 || batch == 0) return set_error(HFM_E_ARG, "empty training set or batch");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  int rc;
  if ((rc = grow((void**)&m->perm, &m->perm_cap, (size_t)n * 4 + 4))) return rc;
  std::vector<uint32_t> perm(n);
  uint64_t s = seed;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (uint32_t e = 0; e < epochs; e++) {
    for (uint32_t i = 0; i < n; i++) perm[i] = i;
    for (uint32_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[splitmix(s) % (i + 1)]);   // Fisher-Yates
    MCK(cudaMemcpyAsync(m->perm, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, m->stream));
    MCK(cudaMemsetAsync(m->loss_acc, 0, 8, m->stream));
    for (uint32_t a = 0; a < n; a += batch) {
      uint32_t nb = std::min(batch, n - a);
      if ((rc = batch_grad(m, d_x, d_t, m->perm + a, nb, m->loss_acc))) return rc;
      m->step++;
      float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
      k_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->w, m->m, m->v, m->grad, lr, b1, b2, eps, c1, c2,
                                                          m->w1h, m->w2h, m->w3h);
    }
    double l = 0;
    MCK(cudaMemcpyAsync(&l, m->loss_acc, 8, cudaMemcpyDeviceToHost, m->stream));
    if ((rc = sync(m))) return rc;
    if (loss_per_epoch) loss_per_epoch[e] = (float)(l / ((double)n * OUT));
  }
  return sync(m);
}

int hfm_mlp_schedule(hfm_mlp* m, const float* d_y, uint32_t nq, float warp_min_hits, uint32_t* d_order,
                     uint32_t* n_warp) {
  if (!m || !n_warp || (nq && (!d_y || !d_order))) return set_error(HFM_E_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(m->mu);
  DevGuard dg(m->device);
  *n_warp = 0;
  if (!nq) return HFM_OK;
  float wl = warp_min_hits > 0.f ? std::log1p(warp_min_hits) : INFINITY;
  MCK(cudaMemsetAsync(m->bins, 0, (size_t)NBINS * 4 + 16, m->stream));
  unsigned grid = (unsigned)std::min<uint64_t>((nq + 255) / 256, (uint64_t)m->num_sms * 2);
  k_bin_hist<<<grid, 256, 0, m->stream>>>(d_y, nq, wl, m->bins);
  k_bin_scan<<<1, 1024, 0, m->stream>>>(m->bins, m->bins + NBINS);
  k_bin_scatter<<<(nq + 255) / 256, 256, 0, m->stream>>>(d_y, nq, wl, m->bins, d_order);
  uint32_t nw = 0;
  MCK(cudaMemcpyAsync(&nw, m->bins + NBINS, 4, cudaMemcpyDeviceToHost, m->stream));
  int rc = sync(m);
  if (rc) return rc;
  *n_warp = nw;
  return HFM_OK;
}

}  // extern "C"
