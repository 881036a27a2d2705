// The wave-speed network of the learned path: a 35 -> 128 -> 128 -> 128 -> 6
// MLP with SiLU, BF16 weights and activations, FP32 accumulation, run on the
// tcgen05 tensor cores of sm_100a.
//
//   k_wavenet        inference fused with its input features: per tile of 128
//                    cells, the standardized moments (FP64, M2CS4_35 of the
//                    realized state) are rounded to BF16 straight into the
//                    shared-memory A tile, four MMA chains run with the
//                    accumulator in TMEM, each epilogue (bias + SiLU + BF16)
//                    writes the next A tile, and the six predicted
//                    standardized extreme speeds go to the seed buffer.
//   k_wavenet_train  forward and backward of a training batch: the same
//                    forward, the loss gradient, the data gradients
//                    dH = dZ W and the weight gradients dW = dZ^T H (the
//                    activation tiles read transposed through MN-major
//                    descriptors), accumulated in TMEM over the tiles a CTA
//                    takes; per-CTA partial gradients go to global memory.
//   k_wavenet_adam   reduce the partials, Adam update of the FP32 parameters.
//   k_wavenet_pack   FP32 parameters -> the BF16 weight image (the swizzled
//                    shared-memory layout, so one bulk copy loads it).
//   k_wavenet_features  the input tiles of a training set (same features as
//                    k_wavenet computes inline).
//
// One CTA of 128 threads per tile of 128 cells: thread t owns row (cell) t,
// which is TMEM lane t of every accumulator, so each epilogue is row-local.
// Thread 0 issues the MMAs and commits them to an mbarrier; every wait is
// bounded (umma::mbar_wait) and a timeout sets the error word instead of
// hanging.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "hyq_cell.cuh"
#include "hyq_step.cuh"
#include "hyq_umma.cuh"
#include "../../include/hyqmom.h"

namespace hyqk {

using namespace umma;

// ------------------------------------------------------------ geometry
constexpr int NIN = 35, NH = 128, NOUT = 6;
constexpr int KIN = 64;    // padded input width: one 128-byte swizzle chunk
constexpr int NOUTP = 16;  // padded output width (UMMA N >= 16 at M = 128)
constexpr int TILE = 128;  // cells per tile (UMMA M)

// FP32 parameter vector (the C-ABI order): W1 b1 W2 b2 W3 b3 W4 b4, W row-major out x in
constexpr int P_W1 = 0, P_B1 = P_W1 + NH * NIN, P_W2 = P_B1 + NH, P_B2 = P_W2 + NH * NH, P_W3 = P_B2 + NH,
              P_B3 = P_W3 + NH * NH, P_W4 = P_B3 + NH, P_B4 = P_W4 + NOUT * NH, NPARAM = P_B4 + NOUT;
static_assert(NPARAM == HYQ_NET_PARAMS, "parameter count");

// BF16 weight image (bytes): W1 [128 x 64], W2, W3 [128 x 128], W4 [16 x 128]
// in SW128 layout, then the FP32 biases b1, b2, b3 (128 each) and b4 (16).
constexpr int IMG_W1 = 0, IMG_W2 = IMG_W1 + NH * 128, IMG_W3 = IMG_W2 + 2 * NH * 128, IMG_W4 = IMG_W3 + 2 * NH * 128,
              IMG_B = IMG_W4 + 2 * NOUTP * 128, IMG_BYTES = IMG_B + (3 * NH + NOUTP) * 4;
static_assert(IMG_W4 % 1024 == 0 && IMG_B % 16 == 0 && IMG_BYTES % 16 == 0, "image alignment");
constexpr int IMG_ALIGNED = (IMG_BYTES + 1023) / 1024 * 1024;

constexpr uint32_t TILE_X_BYTES = TILE * 128;        // one input tile [128 x 64] BF16
constexpr uint32_t TILE_H_BYTES = 2 * TILE * 128;    // one hidden tile [128 x 128] BF16

// error word values
constexpr int NET_ERR_WAIT = 1;

// SiLU through the logistic function written as 0.5 (1 + tanh(z / 2)), with
// the hardware tanh approximation (one MUFU operation; its error is far below
// the BF16 rounding of the activations).  Inference and training use the same
// function.
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sigmoid(float z) { return 0.5f + 0.5f * tanh_approx(0.5f * z); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigmoid(z);
  return s * (1.0f + z * (1.0f - s));
}

// The network input of one cell: its 35 standardized moments (M2CS4_35 of
// the moments at stride st), as BF16 in the 64-wide padded row.
__device__ __forceinline__ void cell_features(const double* M, long long st, bool valid, uint32_t (&packed)[32]) {
  double S[35];
  if (valid) {
    double C[35];
    hyq::raw_to_central_r(M, st, C);
    hyq::central_to_std(C, S);
  } else {
#pragma unroll
    for (int q = 0; q < 35; ++q) S[q] = 0.0;
  }
#pragma unroll
  for (int q = 0; q < 32; ++q) {
    const int a = 2 * q, b = 2 * q + 1;
    const float fa = a < NIN ? (float)S[a] : 0.0f;
    const float fb = b < NIN ? (float)S[b] : 0.0f;
    packed[q] = pack_bf16(fa, fb);
  }
}

// Row r of an SW128 tile of 128 rows from 8 * n packed BF16 pairs.
template <int NUNITS>
__device__ __forceinline__ void store_row_sw128(unsigned char* tile, int r, const uint32_t* packed) {
#pragma unroll
  for (int u = 0; u < NUNITS; ++u) {
    uint4 v = make_uint4(packed[4 * u], packed[4 * u + 1], packed[4 * u + 2], packed[4 * u + 3]);
    *reinterpret_cast<uint4*>(tile + sw128_unit(TILE, r, u)) = v;
  }
}

// K-major SW128 operand descriptors for K step kk (16 elements) of a matrix of
// R rows stored as 64-wide chunks
__device__ __forceinline__ uint64_t kdesc(uint32_t base, int R, int kk) {
  return sdesc(base + uint32_t((kk >> 2) * R * 128 + (kk & 3) * 32), 16, 1024, LAYOUT_SW128);
}
// MN-major SW128 operand (MN along the stored row, K along the rows) for K
// step kk (16 rows) of a matrix with R stored rows
__device__ __forceinline__ uint64_t mdesc(uint32_t base, int R, int kk) {
  return sdesc(base + uint32_t(kk * 2048), uint32_t(R * 128), 1024, LAYOUT_SW128);
}

// D (TMEM) = A (K-major, R_a rows) * B^T (K-major, N rows), K = 16 * nk
__device__ __forceinline__ void mma_kk(uint32_t tmem, uint32_t a, int Ra, uint32_t b, int Rb, int nk, int N, uint32_t acc0) {
  const uint32_t id = idesc_bf16(128, N, false, false);
  for (int kk = 0; kk < nk; ++kk) mma_bf16(tmem, kdesc(a, Ra, kk), kdesc(b, Rb, kk), id, (kk > 0) ? 1u : acc0);
}

// Epilogue of a hidden layer for this thread's row: z = acc + b, h = SiLU(z)
// to the SW128 tile `out` (BF16); with DS, SiLU'(z) to ds[0..127] (BF16).
template <bool DS>
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem_row, const float* bias, unsigned char* out, int r, __nv_bfloat16* ds) {
#pragma unroll 1
  for (int j = 0; j < 4; ++j) {
    float v[32];
    tmem_ld32(tmem_row + 32 * j, v);
    uint32_t hp[16], dp[16];
#pragma unroll
    for (int i = 0; i < 32; i += 2) {
      const float z0 = v[i] + bias[32 * j + i], z1 = v[i + 1] + bias[32 * j + i + 1];
      hp[i / 2] = pack_bf16(silu(z0), silu(z1));
      if (DS) dp[i / 2] = pack_bf16(dsilu(z0), dsilu(z1));
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int u = 4 * j + q;
      *reinterpret_cast<uint4*>(out + sw128_unit(TILE, r, u)) = make_uint4(hp[4 * q], hp[4 * q + 1], hp[4 * q + 2], hp[4 * q + 3]);
      if (DS) *reinterpret_cast<uint4*>(ds + 8 * u) = make_uint4(dp[4 * q], dp[4 * q + 1], dp[4 * q + 2], dp[4 * q + 3]);
    }
  }
}

__device__ __forceinline__ unsigned char* align1024(unsigned char* p) {
  return reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// ------------------------------------------------------------ inference
// One CTA runs INF_GROUPS independent tile pipelines of 128 threads (4 warps)
// each, so that one group's features and epilogues overlap another's MMAs:
// group g owns an activation tile (the input in its first chunk), TMEM
// columns [128 g, 128 g + 128) and an mbarrier, and synchronises on named
// barrier 1 + g.  Shared memory: weight image | INF_GROUPS activation tiles |
// barriers and the TMEM address.
constexpr int INF_GROUPS = 4;
constexpr int INF_THREADS = 128 * INF_GROUPS;
constexpr int INF_ACT = IMG_ALIGNED, INF_BAR = INF_ACT + INF_GROUPS * TILE_H_BYTES, INF_SMEM = INF_BAR + 64 + 2048;

__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory"); }
// named-barrier AND of `pred` over the group
__device__ __forceinline__ bool group_and(int g, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(1 + g)
      : "memory");
  return r != 0;
}

// Mr: moments (stride N) of cells [c0, c1); seeds: [6][N] FP32.  clk (may be
// NULL): the step's loop predicate.
__global__ void __launch_bounds__(INF_THREADS, 1) k_wavenet(const double* __restrict__ Mr, long long N, long long c0, long long c1,
                                                           const unsigned char* __restrict__ image, float* __restrict__ seeds,
                                                           double tmax, long long nnmax, const DevClock* clk, int* err) {
  if (clk && !((clk->t < tmax) && (clk->nn < nnmax))) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  const int tid = threadIdx.x, g = tid >> 7, r = tid & 127, warp = tid >> 5;
  unsigned char* act = sm + INF_ACT + g * TILE_H_BYTES;
  const float* bias = reinterpret_cast<const float*>(sm + IMG_B);
  const uint32_t s_img = smem_u32(sm), s_act = smem_u32(act);
  const uint32_t bar_w = smem_u32(sm + INF_BAR), bar_m = bar_w + 8 * (1 + g), slot = bar_w + 8 * (1 + INF_GROUPS);
  if (tid == 0) {
    for (int q = 0; q <= INF_GROUPS; ++q) mbar_init(bar_w + 8 * q, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar_w, IMG_BYTES);
    bulk_g2s(s_img, image, IMG_BYTES, bar_w);
  }
  if (warp == 0) tmem_alloc(slot, 128 * INF_GROUPS);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + INF_BAR + 8 * (1 + INF_GROUPS)) + uint32_t(128 * g);
  const uint32_t trow = tmem + (uint32_t((warp & 3) * 32) << 16);
  bool ok = __syncthreads_and(mbar_wait(bar_w, 0)) != 0;
  uint32_t phase = 0;
  const long long ntiles = (c1 - c0 + TILE - 1) / TILE;
  for (long long t = (long long)blockIdx.x * INF_GROUPS + g; t < ntiles && ok; t += (long long)gridDim.x * INF_GROUPS) {
    const long long c = c0 + t * TILE + r;
    const bool valid = c < c1;
    {
      uint32_t packed[32];
      cell_features(Mr + (valid ? c : c0), N, valid, packed);
      store_row_sw128<8>(act, r, packed);
    }
    // layers 1..3: A = act (K-major), B = W_l, D = the group's TMEM columns
#pragma unroll 1
    for (int l = 0; l < 4; ++l) {
      fence_proxy_async();
      fence_before();
      group_sync(g);
      if (r == 0) {
        fence_after();
        if (l < 3) {
          const uint32_t w = s_img + (l == 0 ? IMG_W1 : (l == 1 ? IMG_W2 : IMG_W3));
          mma_kk(tmem, s_act, TILE, w, NH, l == 0 ? KIN / 16 : NH / 16, NH, 0u);
        } else {
          mma_kk(tmem, s_act, TILE, s_img + IMG_W4, NOUTP, NH / 16, NOUTP, 0u);  // layer 4: N = 16
        }
        mma_commit(bar_m);
      }
      ok = group_and(g, ok && mbar_wait(bar_m, phase));
      phase ^= 1u;
      fence_after();
      if (l < 3) hidden_epilogue<false>(trow, bias + NH * l, act, r, nullptr);
    }
    float y[16];
    tmem_ld16(trow, y);
    if (valid) {
#pragma unroll
      for (int q = 0; q < NOUT; ++q) seeds[(long long)q * N + c] = y[q] + bias[3 * NH + q];
    }
    fence_before();
    group_sync(g);
  }
  if (!ok && r == 0 && err) atomicExch(err, NET_ERR_WAIT);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem - uint32_t(128 * g), 128 * INF_GROUPS);
}

// ------------------------------------------------------------ training
// Shared memory: image | X tile | hidden tiles A, B, C | output-gradient
// tile D | barriers.  TMEM (512 columns): [0,128) the layer accumulator and
// the data gradients, [128,256) dW2, [256,384) dW3, [384,448) dW1,
// [448,464) dW4^T.
constexpr int TR_X = IMG_ALIGNED, TR_A = TR_X + TILE_X_BYTES, TR_B = TR_A + TILE_H_BYTES, TR_C = TR_B + TILE_H_BYTES,
              TR_D = TR_C + TILE_H_BYTES, TR_BAR = TR_D + 4096, TR_SMEM = TR_BAR + 64 + 2048;
constexpr uint32_t T_S = 0, T_W2 = 128, T_W3 = 256, T_W1 = 384, T_W4 = 448;

// dZ = dH * SiLU'(z) for this row from the TMEM data gradient; BF16 into the
// SW128 tile `out`; column sums go to db (one float per column, this thread's
// share added by the caller)
__device__ __forceinline__ void grad_epilogue(uint32_t tmem_row, const __nv_bfloat16* ds, unsigned char* out, int r, bool valid) {
#pragma unroll 1
  for (int j = 0; j < 4; ++j) {
    float v[32];
    tmem_ld32(tmem_row + 32 * j, v);
    uint32_t gp[16];
#pragma unroll
    for (int i = 0; i < 32; i += 2) {
      const float d0 = valid ? v[i] * __bfloat162float(ds[32 * j + i]) : 0.0f;
      const float d1 = valid ? v[i + 1] * __bfloat162float(ds[32 * j + i + 1]) : 0.0f;
      gp[i / 2] = pack_bf16(d0, d1);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int u = 4 * j + q;
      *reinterpret_cast<uint4*>(out + sw128_unit(TILE, r, u)) = make_uint4(gp[4 * q], gp[4 * q + 1], gp[4 * q + 2], gp[4 * q + 3]);
    }
  }
}

// Column sum over the 128 rows of an SW128 gradient tile (column = thread).
__device__ __forceinline__ float column_sum(const unsigned char* tile, int col) {
  float s = 0.0f;
#pragma unroll 4
  for (int r = 0; r < TILE; ++r) s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(tile + sw128_elem(TILE, r, col)));
  return s;
}

// X: training inputs, ntiles tiles of [128 x 64] BF16 in SW128 layout; T:
// targets [ntiles * 128][8] FP32 (6 used); n valid rows; order: the tile
// order of this batch (ntiles_batch entries).  dscale = 2 / (rows * 6), the
// mean-square loss gradient factor.  ds_scratch: per-CTA SiLU' rows
// [gridDim][3][128][128] BF16.  partial: per-CTA gradients [gridDim][NPARAM].
// loss: sum of squared errors of the batch (atomic).
__global__ void __launch_bounds__(128, 1) k_wavenet_train(const unsigned char* __restrict__ image, const unsigned char* __restrict__ X,
                                                         const float* __restrict__ T, long long n, const int* __restrict__ order,
                                                         int ntiles_batch, float dscale, __nv_bfloat16* ds_scratch, float* partial,
                                                         float* loss, int* err) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = align1024(smem_raw);
  unsigned char *xs = sm + TR_X, *ta = sm + TR_A, *tb = sm + TR_B, *tc = sm + TR_C, *td = sm + TR_D;
  const float* bias = reinterpret_cast<const float*>(sm + IMG_B);
  const uint32_t s_img = smem_u32(sm), s_x = smem_u32(xs), s_a = smem_u32(ta), s_b = smem_u32(tb), s_c = smem_u32(tc), s_d = smem_u32(td);
  const uint32_t bar_w = smem_u32(sm + TR_BAR), bar_m = bar_w + 8, bar_x = bar_w + 16, slot = bar_w + 24;
  const int tid = threadIdx.x, warp = tid >> 5;
  __nv_bfloat16* dsl = ds_scratch + ((size_t)blockIdx.x * 3 * TILE + tid) * NH;  // this row's SiLU' for layer l: dsl + l * TILE * NH
  if (tid == 0) {
    mbar_init(bar_w, 1);
    mbar_init(bar_m, 1);
    mbar_init(bar_x, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_expect_tx(bar_w, IMG_BYTES);
    bulk_g2s(s_img, image, IMG_BYTES, bar_w);
  }
  if (warp == 0) tmem_alloc(slot, 512);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + TR_BAR + 24);
  const uint32_t lane_off = uint32_t(warp * 32) << 16;
  bool ok = __syncthreads_and(mbar_wait(bar_w, 0)) != 0;
  uint32_t ph_m = 0, ph_x = 0;
  float db1 = 0.f, db2 = 0.f, db3 = 0.f, db4 = 0.f, sse = 0.f;
  bool first = true;
  auto mma_sync = [&]() {
    ok = __syncthreads_and(ok && mbar_wait(bar_m, ph_m)) != 0;
    ph_m ^= 1u;
    fence_after();
  };
  auto to_mma = [&]() {
    fence_proxy_async();
    fence_before();
    __syncthreads();
  };
  for (int it = blockIdx.x; it < ntiles_batch && ok; it += gridDim.x) {
    const int tile = order[it];
    const long long row = (long long)tile * TILE + tid;
    const bool valid = row < n;
    if (tid == 0) {
      mbar_expect_tx(bar_x, TILE_X_BYTES);
      bulk_g2s(s_x, X + (size_t)tile * TILE_X_BYTES, TILE_X_BYTES, bar_x);
    }
    ok = __syncthreads_and(ok && mbar_wait(bar_x, ph_x)) != 0;
    ph_x ^= 1u;
    // ---- forward
    unsigned char* hbuf[3] = {ta, tb, tc};
    const uint32_t hs[3] = {s_a, s_b, s_c};
#pragma unroll 1
    for (int l = 0; l < 3; ++l) {
      if (l > 0) to_mma(); else { fence_before(); __syncthreads(); }
      if (tid == 0) {
        fence_after();
        const uint32_t w = s_img + (l == 0 ? IMG_W1 : (l == 1 ? IMG_W2 : IMG_W3));
        mma_kk(tmem + T_S, l == 0 ? s_x : hs[l - 1], TILE, w, NH, l == 0 ? KIN / 16 : NH / 16, NH, 0u);
        mma_commit(bar_m);
      }
      mma_sync();
      hidden_epilogue<true>(tmem + T_S + lane_off, bias + NH * l, hbuf[l], tid, dsl + (size_t)l * TILE * NH);
    }
    to_mma();
    if (tid == 0) {
      fence_after();
      mma_kk(tmem + T_S, s_c, TILE, s_img + IMG_W4, NOUTP, NH / 16, NOUTP, 0u);
      mma_commit(bar_m);
    }
    mma_sync();
    // ---- loss gradient of the output layer -> D (SW32, 16 wide)
    {
      float y[16];
      tmem_ld16(tmem + T_S + lane_off, y);
      float g[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) g[q] = 0.0f;
      if (valid) {
#pragma unroll
        for (int q = 0; q < NOUT; ++q) {
          const float e = y[q] + bias[3 * NH + q] - T[row * 8 + q];
          sse += e * e;
          g[q] = dscale * e;
        }
      }
      uint32_t gp[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) gp[q] = pack_bf16(g[2 * q], g[2 * q + 1]);
      *reinterpret_cast<uint4*>(td + sw32_unit(tid, 0)) = make_uint4(gp[0], gp[1], gp[2], gp[3]);
      *reinterpret_cast<uint4*>(td + sw32_unit(tid, 1)) = make_uint4(gp[4], gp[5], gp[6], gp[7]);
    }
    to_mma();
    if (tid < NOUTP) {
      float s = 0.0f;
      for (int r = 0; r < TILE; ++r) s += __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(td + sw32_elem(r, tid)));
      db4 += s;
    }
    // ---- layer 4: dW4^T += H3^T dZ4 ; dH3 = dZ4 W4
    if (tid == 0) {
      fence_after();
      const uint32_t id_w = idesc_bf16(128, NOUTP, true, true);
      for (int kk = 0; kk < TILE / 16; ++kk)
        mma_bf16(tmem + T_W4, mdesc(s_c, TILE, kk), sdesc(s_d + uint32_t(kk * 512), 512, 256, LAYOUT_SW32), id_w,
                 (first && kk == 0) ? 0u : 1u);
      const uint32_t id_h = idesc_bf16(128, NH, false, true);
      mma_bf16(tmem + T_S, sdesc(s_d, 16, 256, LAYOUT_SW32), sdesc(s_img + IMG_W4, NOUTP * 128, 1024, LAYOUT_SW128), id_h, 0u);
      mma_commit(bar_m);
    }
    mma_sync();
    // ---- layers 3, 2, 1
    // dZ_l = dH_l * SiLU'(z_l) into the tile that held H_l; then
    // dW_l += dZ_l^T H_(l-1) and (l > 1) dH_(l-1) = dZ_l W_l
#pragma unroll 1
    for (int l = 2; l >= 0; --l) {
      grad_epilogue(tmem + T_S + lane_off, dsl + (size_t)l * TILE * NH, hbuf[l], tid, valid);
      to_mma();
      {
        const float s = column_sum(hbuf[l], tid);
        if (l == 2) db3 += s; else if (l == 1) db2 += s; else db1 += s;
      }
      if (tid == 0) {
        fence_after();
        const uint32_t acc_col = l == 2 ? T_W3 : (l == 1 ? T_W2 : T_W1);
        const uint32_t prev = l == 0 ? s_x : hs[l - 1];
        const int nin = l == 0 ? KIN : NH;
        const uint32_t id_w = idesc_bf16(128, nin, true, true);
        for (int kk = 0; kk < TILE / 16; ++kk)
          mma_bf16(tmem + acc_col, mdesc(hs[l], TILE, kk), mdesc(prev, TILE, kk), id_w, (first && kk == 0) ? 0u : 1u);
        if (l > 0) {
          const uint32_t id_h = idesc_bf16(128, NH, false, true);
          const uint32_t w = s_img + (l == 1 ? IMG_W2 : IMG_W3);
          for (int kk = 0; kk < NH / 16; ++kk) mma_bf16(tmem + T_S, kdesc(hs[l], TILE, kk), mdesc(w, NH, kk), id_h, kk > 0 ? 1u : 0u);
        }
        mma_commit(bar_m);
      }
      mma_sync();
    }
    first = false;
    fence_before();
    __syncthreads();
  }
  // ---- per-CTA partial gradients
  float* out = partial + (size_t)blockIdx.x * NPARAM;
  if (first) {
    // no tile taken: zero partials
    for (int i = tid; i < NPARAM; i += 128) out[i] = 0.0f;
  } else if (ok) {
    const int o = tid;  // TMEM lane = output feature (dW1..dW3) or input feature (dW4^T)
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      float v[32];
      tmem_ld32(tmem + T_W2 + lane_off + 32 * j, v);
      for (int i = 0; i < 32; ++i) out[P_W2 + o * NH + 32 * j + i] = v[i];
      tmem_ld32(tmem + T_W3 + lane_off + 32 * j, v);
      for (int i = 0; i < 32; ++i) out[P_W3 + o * NH + 32 * j + i] = v[i];
    }
#pragma unroll 1
    for (int j = 0; j < 2; ++j) {
      float v[32];
      tmem_ld32(tmem + T_W1 + lane_off + 32 * j, v);
      for (int i = 0; i < 32; ++i)
        if (32 * j + i < NIN) out[P_W1 + o * NIN + 32 * j + i] = v[i];
    }
    {
      float v[16];
      tmem_ld16(tmem + T_W4 + lane_off, v);
      for (int q = 0; q < NOUT; ++q) out[P_W4 + q * NH + o] = v[q];
    }
    out[P_B1 + o] = db1;
    out[P_B2 + o] = db2;
    out[P_B3 + o] = db3;
    if (o < NOUT) out[P_B4 + o] = db4;
  }
  // squared error of the batch
  float s = sse;
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  if ((tid & 31) == 0) atomicAdd(loss, s);
  if (!ok && tid == 0 && err) atomicExch(err, NET_ERR_WAIT);
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// Sum of the per-CTA partial gradients and one Adam step on the FP32
// parameters (bias-corrected, step count `step` >= 1).
__global__ void k_wavenet_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ partial,
                               int nparts, float lr, float b1, float b2, float eps, float wd, int step, float* gout) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  float g = 0.0f;
  for (int p = 0; p < nparts; ++p) g += partial[(size_t)p * NPARAM + i];
  if (gout) gout[i] = g;
  if (lr == 0.0f) return;
  const float mi = b1 * m[i] + (1.0f - b1) * g;
  const float vi = b2 * v[i] + (1.0f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, (float)step)), vh = vi / (1.0f - powf(b2, (float)step));
  w[i] = w[i] - lr * (mh / (sqrtf(vh) + eps) + wd * w[i]);
}

// FP32 parameters -> the BF16 weight image.
__global__ void k_wavenet_pack(const float* __restrict__ w, unsigned char* __restrict__ image) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  auto put = [&](int base, int R, int r, int k, float x) {
    *reinterpret_cast<__nv_bfloat16*>(image + base + sw128_elem(R, r, k)) = __float2bfloat16_rn(x);
  };
  // W1 [128 x 64] (inputs 35..63 zero)
  if (i < NH * KIN) {
    const int r = i / KIN, k = i % KIN;
    put(IMG_W1, NH, r, k, k < NIN ? w[P_W1 + r * NIN + k] : 0.0f);
  }
  if (i < NH * NH) {
    const int r = i / NH, k = i % NH;
    put(IMG_W2, NH, r, k, w[P_W2 + r * NH + k]);
    put(IMG_W3, NH, r, k, w[P_W3 + r * NH + k]);
  }
  if (i < NOUTP * NH) {
    const int r = i / NH, k = i % NH;
    put(IMG_W4, NOUTP, r, k, r < NOUT ? w[P_W4 + r * NH + k] : 0.0f);
  }
  float* b = reinterpret_cast<float*>(image + IMG_B);
  if (i < NH) {
    b[i] = w[P_B1 + i];
    b[NH + i] = w[P_B2 + i];
    b[2 * NH + i] = w[P_B3 + i];
  }
  if (i < NOUTP) b[3 * NH + i] = i < NOUT ? w[P_B4 + i] : 0.0f;
}

// Training inputs: the features of n cells (moments at stride n) as tiles.
__global__ void __launch_bounds__(128) k_wavenet_features(const double* __restrict__ M, long long n, unsigned char* __restrict__ X) {
  const long long c = (long long)blockIdx.x * TILE + threadIdx.x;
  const bool valid = c < n;
  uint32_t packed[32];
  cell_features(M + (valid ? c : 0), n, valid, packed);
  store_row_sw128<8>(X + (size_t)blockIdx.x * TILE_X_BYTES, threadIdx.x, packed);
}

}  // namespace hyqk (kernels)

namespace hyqk {

int net_grid() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// The kernels' shared memory above the 48 KB default (set on the current
// device; cheap to repeat).
cudaError_t net_set_smem() {
  cudaError_t e = cudaFuncSetAttribute(k_wavenet, cudaFuncAttributeMaxDynamicSharedMemorySize, INF_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_wavenet_train, cudaFuncAttributeMaxDynamicSharedMemorySize, TR_SMEM);
  return e;
}

void launch_wavespeed_seeds(const StepConst& sc, const double* Mr, const WaveNet* net, float* seeds, const DevClock* clk, cudaStream_t s,
                            long long c0, long long c1) {
  const long long ntiles = (c1 - c0 + TILE - 1) / TILE;
  const long long need = (ntiles + INF_GROUPS - 1) / INF_GROUPS;
  const int g = (int)(need < net_grid() ? need : net_grid());
  k_wavenet<<<g, INF_THREADS, INF_SMEM, s>>>(Mr, sc.N, c0, c1, net->image, seeds, sc.tmax, sc.nnmax, clk, net->err);
}

}  // namespace hyqk

// ------------------------------------------------------------ C-ABI
using namespace hyqk;

namespace {
int net_cuda_fail(cudaError_t e, const char* what) {
  return report_error(HYQ_ECUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}
#define NET_LAUNCH_CHECK(what)                                  \
  do {                                                          \
    cudaError_t e_ = cudaGetLastError();                        \
    if (e_ != cudaSuccess) return net_cuda_fail(e_, what);      \
  } while (0)
}  // namespace

extern "C" {

int64_t hyq_net_image_bytes(void) { return IMG_BYTES; }
int64_t hyq_net_tile_bytes(void) { return TILE_X_BYTES; }
int64_t hyq_net_scratch_bytes(int32_t nparts) { return (int64_t)nparts * 3 * TILE * NH * 2; }

int hyq_net_pack(const float* w, void* image, void* stream) {
  if (!w || !image) return report_error(HYQ_EINVAL, "null argument");
  k_wavenet_pack<<<(NH * NH + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, (unsigned char*)image);
  NET_LAUNCH_CHECK("k_wavenet_pack");
  return HYQ_OK;
}

int hyq_net_features(const double* M, int64_t n, void* X, void* stream) {
  if (!M || !X || n <= 0) return report_error(HYQ_EINVAL, "bad argument");
  const long long ntiles = (n + TILE - 1) / TILE;
  k_wavenet_features<<<(unsigned)ntiles, TILE, 0, (cudaStream_t)stream>>>(M, n, (unsigned char*)X);
  NET_LAUNCH_CHECK("k_wavenet_features");
  return HYQ_OK;
}

int hyq_net_forward(const void* image, const double* M, int64_t n, float* out, int32_t* err, void* stream) {
  if (!image || !M || !out || !err || n <= 0) return report_error(HYQ_EINVAL, "bad argument");
  cudaError_t e = net_set_smem();
  if (e != cudaSuccess) return net_cuda_fail(e, "cudaFuncSetAttribute");
  const long long ntiles = (n + TILE - 1) / TILE;
  const long long need = (ntiles + INF_GROUPS - 1) / INF_GROUPS;
  const int g = (int)(need < net_grid() ? need : net_grid());
  k_wavenet<<<g, INF_THREADS, INF_SMEM, (cudaStream_t)stream>>>(M, n, 0, n, (const unsigned char*)image, out, 0.0, 0, nullptr, (int*)err);
  NET_LAUNCH_CHECK("k_wavenet");
  return HYQ_OK;
}

int hyq_net_train_batch(const void* image, const void* X, const float* T, int64_t n, const int32_t* order, int32_t ntiles,
                        float dscale, void* ds_scratch, float* partial, int32_t nparts, float* loss, int32_t* err, void* stream) {
  if (!image || !X || !T || !order || !ds_scratch || !partial || !loss || !err || n <= 0 || ntiles <= 0 || nparts <= 0)
    return report_error(HYQ_EINVAL, "bad argument");
  cudaError_t e = net_set_smem();
  if (e != cudaSuccess) return net_cuda_fail(e, "cudaFuncSetAttribute");
  k_wavenet_train<<<nparts, 128, TR_SMEM, (cudaStream_t)stream>>>((const unsigned char*)image, (const unsigned char*)X, T, n, order, ntiles,
                                                                  dscale, (__nv_bfloat16*)ds_scratch, partial, loss, (int*)err);
  NET_LAUNCH_CHECK("k_wavenet_train");
  return HYQ_OK;
}

int hyq_net_adam(float* w, float* m, float* v, const float* partial, int32_t nparts, float lr, float beta1, float beta2, float eps,
                 float wd, int32_t step, float* gout, void* stream) {
  if (!w || !m || !v || !partial || nparts <= 0 || step < 1) return report_error(HYQ_EINVAL, "bad argument");
  k_wavenet_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(w, m, v, partial, nparts, lr, beta1, beta2, eps, wd, step, gout);
  NET_LAUNCH_CHECK("k_wavenet_adam");
  return HYQ_OK;
}

}  // extern "C"
