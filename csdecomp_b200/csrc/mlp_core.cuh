// mlp_core.cuh -- device code of the surrogate MLP shared by the bank's own
// kernels (mlp.cu) and the batched EI-ZO scoring stage (batch.cu): operand
// tile loads and the fused three-layer forward of one 128-row tile.
#pragma once
#include <cuda_bf16.h>

#include "umma.cuh"

namespace csd {
namespace mlp {

using bf16 = __nv_bfloat16;
constexpr int kH = 256;     // hidden width
constexpr int kIn = 16;     // padded input width
constexpr int kKC = 64;     // K chunk of the streamed operand
constexpr int kThreads = 256;

// parameter offsets within one net (floats)
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kH, kParams = oB4 + 1;
// bf16 weight copies within one net: W1 [256][16], W2, W3 [out][in], W2t, W3t [in][out]
constexpr int qW1 = 0, qW2 = qW1 + kH * kIn, qW3 = qW2 + kH * kH, qW2t = qW3 + kH * kH, qW3t = qW2t + kH * kH,
              kBf = qW3t + kH * kH;

// Copies rows [r0, r0 + R) x k [k0, k0 + KC) of a K-major bf16 matrix (row
// stride ld elements, `rows` x `K` valid) into an R x KC K-major tile; zero
// outside. ld, K and k0 are multiples of 8 and the base 16-byte aligned.
__device__ __forceinline__ void load_tile(const bf16* __restrict__ src, int ld, int rows, int K, int r0, int k0,
                                          int R, int KC, char* tile) {
  const int pieces = R * (KC >> 3);
  for (int idx = threadIdx.x; idx < pieces; idx += blockDim.x) {
    const int r8 = idx & 7, chunk = (idx >> 3) % (KC >> 3), rg = idx / KC;
    const int row = rg * 8 + r8, k = chunk * 8;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (r0 + row < rows && k0 + k < K) v = *reinterpret_cast<const uint4*>(src + (size_t)(r0 + row) * ld + k0 + k);
    *reinterpret_cast<uint4*>(tile + umma::tile_offset(row, k, KC)) = v;
  }
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// --------------------------------------------------------- fused forward
// One group = rows of one net's input. Inputs are f32 rows of `dim`
// coordinates (scaled by in_scale, zero padded to 16) or, for training, bf16
// rows already padded (xb).
struct FwdGroup {
  const float* x;   // [rows][dim] f32, or null when xb is used
  const bf16* xb;   // [rows][16] bf16
  int rows, dim, net;
  float* logits;    // [rows]
  // training outputs (optional): transposed bf16 copies, leading dimension ld_t
  bf16 *xt, *h1t, *h2t, *h3t;
  int ld_t;
};

struct FwdArgs {
  const FwdGroup* groups;
  const bf16* wb;      // bf16 weights, kBf per net
  const float* params; // f32 parameters, kParams per net (biases, w4, b4)
  float in_scale;
  int* status;
};

constexpr size_t kFwdX = 128 * kIn * 2;           // 4 KB
constexpr size_t kFwdH = 128 * kH * 2;            // 64 KB
constexpr size_t kFwdStage = (size_t)kH * kKC * 2;  // 32 KB
constexpr size_t kFwdSmem = kFwdX + kFwdH + 2 * kFwdStage + 1024;

// Epilogue of a hidden layer: relu(acc + b) -> bf16 into the next layer's
// operand tile (and the transposed copy when training).
__device__ __forceinline__ void hidden_epilogue(uint32_t tmem, const float* bias, char* hs, bf16* ht, int ld_t,
                                                int row0, int rows) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = 32 * (warp & 3) + lane;
  const int c0 = (warp >> 2) * (kH / 2);
  for (int j = c0; j < c0 + kH / 2; j += 16) {
    float v[16];
    umma::tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)j, v);
    uint32_t p[8];
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
      const float a = fmaxf(v[i] + bias[j + i], 0.f), b = fmaxf(v[i + 1] + bias[j + i + 1], 0.f);
      p[i >> 1] = pack2(a, b);
      v[i] = a;
      v[i + 1] = b;
    }
    *reinterpret_cast<uint4*>(hs + umma::tile_offset(r, j, kH)) = make_uint4(p[0], p[1], p[2], p[3]);
    *reinterpret_cast<uint4*>(hs + umma::tile_offset(r, j + 8, kH)) = make_uint4(p[4], p[5], p[6], p[7]);
    if (ht && row0 + r < rows) {
#pragma unroll
      for (int i = 0; i < 16; ++i) ht[(size_t)(j + i) * ld_t + row0 + r] = __float2bfloat16_rn(v[i]);
    }
  }
}

// MMAs of one hidden layer (K = 256) with the weight matrix streamed in
// four 64-wide chunks through the two stages. `uses` counts each stage's
// commits over the kernel (barrier phase parity). Returns false on a
// barrier timeout.
__device__ __forceinline__ bool hidden_layer(uint32_t tmem, const bf16* W, char* hs, char* stages, uint64_t* bars,
                                             int* uses) {
  const uint32_t idesc = umma::instr_desc_bf16(128, kH);
  bool ok = true;
  for (int c = 0; c < kH / kKC; ++c) {
    const int st = c & 1;
    char* sb = stages + st * kFwdStage;
    if (uses[st] > 0) ok = umma::bar_wait(&bars[st], (uses[st] - 1) & 1);
    if (!__syncthreads_and(ok)) return false;
    load_tile(W, kH, kH, kH, 0, c * kKC, kH, kKC, sb);
    umma::fence_smem_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      for (int s = 0; s < kKC / 16; ++s)
        umma::mma_bf16(tmem, umma::tile_desc(umma::smem_u32(hs), c * (kKC / 16) + s, kH),
                       umma::tile_desc(umma::smem_u32(sb), s, kKC), idesc, (c > 0 || s > 0) ? 1u : 0u);
      umma::commit(&bars[st]);
    }
    uses[st] += 1;
  }
  // the last commit covers every MMA of the layer; drain the other stage's phase too
  ok = umma::bar_wait(&bars[1], (uses[1] - 1) & 1) && umma::bar_wait(&bars[0], (uses[0] - 1) & 1);
  ok = __syncthreads_and(ok);
  umma::fence_after_sync();
  return ok;
}

static __device__ void forward_tile(const FwdArgs& a, const FwdGroup& G, int row0, char* smem, uint64_t* bars,
                             uint32_t tmem) {
  char* xs = smem;
  char* hs = xs + kFwdX;
  char* stages = hs + kFwdH;
  const bf16* wb = a.wb + (size_t)G.net * kBf;
  const float* pr = a.params + (size_t)G.net * kParams;
  // input tile (128 x 16) and W1 (256 x 16), K-major, KC = 16
  for (int idx = threadIdx.x; idx < 128 * 2; idx += blockDim.x) {
    const int r = idx >> 1, half = idx & 1, row = row0 + r;
    uint32_t p[4] = {0, 0, 0, 0};
    if (row < G.rows) {
      if (G.xb) {
        uint4 v = *reinterpret_cast<const uint4*>(G.xb + (size_t)row * kIn + half * 8);
        p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
      } else {
        float f[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int k = half * 8 + i;
          f[i] = k < G.dim ? G.x[(size_t)row * G.dim + k] * a.in_scale : 0.f;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) p[i] = pack2(f[2 * i], f[2 * i + 1]);
      }
    }
    *reinterpret_cast<uint4*>(xs + umma::tile_offset(r, half * 8, kIn)) = make_uint4(p[0], p[1], p[2], p[3]);
    if (G.xt && row < G.rows) {
      const bf16* hv = reinterpret_cast<const bf16*>(p);
#pragma unroll
      for (int i = 0; i < 8; ++i) G.xt[(size_t)(half * 8 + i) * G.ld_t + row] = hv[i];
    }
  }
  load_tile(wb + qW1, kIn, kH, kIn, 0, 0, kH, kIn, stages);
  umma::fence_smem_async();
  __syncthreads();
  int uses[2] = {0, 0};
  // layer 1: one K step
  if (threadIdx.x == 0) {
    umma::fence_after_sync();
    umma::mma_bf16(tmem, umma::tile_desc(umma::smem_u32(xs), 0, kIn), umma::tile_desc(umma::smem_u32(stages), 0, kIn),
                   umma::instr_desc_bf16(128, kH), 0u);
    umma::commit(&bars[0]);
  }
  uses[0] = 1;
  bool ok = __syncthreads_and(umma::bar_wait(&bars[0], 0));
  umma::fence_after_sync();
  if (ok) hidden_epilogue(tmem, pr + oB1, hs, G.h1t, G.ld_t, row0, G.rows);
  umma::fence_before_sync();
  umma::fence_smem_async();
  __syncthreads();
  // layers 2 and 3
  ok = ok && hidden_layer(tmem, wb + qW2, hs, stages, bars, uses);
  if (ok) hidden_epilogue(tmem, pr + oB2, hs, G.h2t, G.ld_t, row0, G.rows);
  umma::fence_before_sync();
  umma::fence_smem_async();
  __syncthreads();
  ok = ok && hidden_layer(tmem, wb + qW3, hs, stages, bars, uses);
  if (!ok) {
    if (threadIdx.x == 0 && a.status) atomicExch(a.status, 1);
    return;
  }
  // layer 3 epilogue: h3 = relu(acc + b3); logit = h3 . w4 + b4 (the two warps of a lane quadrant add halves)
  __shared__ float part[128];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = 32 * (warp & 3) + lane;
  const int c0 = (warp >> 2) * (kH / 2);
  float acc = 0.f;
  for (int j = c0; j < c0 + kH / 2; j += 16) {
    float v[16];
    umma::tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)j, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float h = fmaxf(v[i] + pr[oB3 + j + i], 0.f);
      const float hb = __bfloat162float(__float2bfloat16_rn(h));
      acc = fmaf(hb, pr[oW4 + j + i], acc);
      if (G.h3t && row0 + r < G.rows) G.h3t[(size_t)(j + i) * G.ld_t + row0 + r] = __float2bfloat16_rn(h);
    }
  }
  if (warp >= 4) part[r] = acc;
  __syncthreads();
  if (warp < 4 && row0 + r < G.rows) G.logits[row0 + r] = acc + part[r] + pr[oB4];
  umma::fence_before_sync();
  __syncthreads();
}

}  // namespace mlp
}  // namespace csd
