// mlp.cu -- the collision-likelihood surrogate: a bank of BF16 MLPs
// (in -> 256 -> 256 -> 256 -> 1, ReLU, FP32 accumulate), one per plant, with
// hand-written tcgen05 forward and backward kernels and an Adam trainer.
//
// Tensor-core work (umma.cuh):
//   * mlp_forward_kernel: one CTA per 128 rows of one net; the three hidden
//     layers are chained through shared memory (the epilogue of layer l
//     writes relu(acc + b) as bf16 straight into the K-major operand tile of
//     layer l + 1), weights stream in 64-wide K chunks through a double
//     buffer, the accumulator (128 x 256 f32) lives in TMEM. The 256 -> 1
//     output is a dot product in the last epilogue.
//   * gemm_kernel<NT>: grouped D = A * B^T (both K-major bf16 in global
//     memory) for the backward pass, with epilogues that store f32, or apply
//     the ReLU mask and store bf16 row-major and transposed.
// CUDA-core kernels: the output-layer gradient, bias reductions, Adam.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include <cuda_bf16.h>

#include "csd_internal.h"
#include "mlp_core.cuh"

namespace csd {
namespace mlp {

// ------------------------------------------------------------------ GEMM
enum Epi { kEpiF32 = 0, kEpiReluGrad = 1 };

struct GemmArgs {
  const bf16* A;
  long long a_group;
  int lda;
  const bf16* B;
  long long b_group;
  int ldb;
  int M, N, K;
  int epi;
  float* D;  // kEpiF32: D[m][n]
  long long d_group;
  int ldd;
  const bf16* mask_t;  // kEpiReluGrad: value kept where mask_t[n][m] > 0
  long long mt_group;
  int ldmt;
  bf16* out;  // [m][n], optional
  long long o_group;
  int ldo;
  bf16* out_t;  // [n][m], optional
  long long ot_group;
  int ldot;
  int* status;
};

template <int NT>
__global__ void __launch_bounds__(kThreads) gemm_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  constexpr int kA = 128 * kKC * 2, kB = NT * kKC * 2, kStage = kA + kB;
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_base;
  constexpr uint32_t kCols = NT < 32 ? 32 : NT;
  const int grp = blockIdx.z, m0 = blockIdx.x * 128, n0 = blockIdx.y * NT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bf16* A = g.A + grp * g.a_group;
  const bf16* B = g.B + grp * g.b_group;
  if (warp == 0) {
    umma::tmem_alloc(&tmem_base, kCols);
    umma::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    umma::bar_init(&bars[0], 1);
    umma::bar_init(&bars[1], 1);
    umma::bar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = umma::instr_desc_bf16(128, NT);
  const int nchunks = (g.K + kKC - 1) / kKC;
  bool ok = true;
  for (int c = 0; c < nchunks && ok; ++c) {
    const int st = c & 1;
    char* sa = smem + st * kStage;
    char* sb = sa + kA;
    if (c >= 2) ok = umma::bar_wait(&bars[st], ((c - 2) >> 1) & 1);
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    load_tile(A, g.lda, g.M, g.K, m0, c * kKC, 128, kKC, sa);
    load_tile(B, g.ldb, g.N, g.K, n0, c * kKC, NT, kKC, sb);
    umma::fence_smem_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      const int steps = min(kKC, g.K - c * kKC + 15) >> 4;
      for (int s = 0; s < steps; ++s)
        umma::mma_bf16(tmem, umma::tile_desc(umma::smem_u32(sa), s, kKC), umma::tile_desc(umma::smem_u32(sb), s, kKC),
                       idesc, (c > 0 || s > 0) ? 1u : 0u);
      umma::commit(&bars[st]);
    }
  }
  if (ok && nchunks > 0) ok = umma::bar_wait(&bars[(nchunks - 1) & 1], ((nchunks - 1) >> 1) & 1);
  if (nchunks > 1 && ok) ok = umma::bar_wait(&bars[(nchunks - 2) & 1], ((nchunks - 2) >> 1) & 1);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0 && g.status) atomicExch(g.status, 1);
  } else {
    umma::fence_after_sync();
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31; warps w and w + 4 split the columns
    const int row = m0 + 32 * (warp & 3) + lane;
    constexpr int kSplit = NT >= 32 ? 2 : 1;
    const int cpw = NT / kSplit;
    if (warp < 4 * kSplit) {
      for (int j0 = (warp >> 2) * cpw; j0 < (warp >> 2) * cpw + cpw; j0 += 16) {
        float v[16];
        umma::tmem_ld16(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)j0, v);
        if (row < g.M) {
          if (g.epi == kEpiF32) {
            float* d = g.D + grp * g.d_group + (size_t)row * g.ldd;
#pragma unroll
            for (int i = 0; i < 16; ++i)
              if (n0 + j0 + i < g.N) d[n0 + j0 + i] = v[i];
          } else {
            const bf16* mt = g.mask_t + grp * g.mt_group;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int n = n0 + j0 + i;
              if (n < g.N) {
                const float keep = __bfloat162float(mt[(size_t)n * g.ldmt + row]) > 0.f ? 1.f : 0.f;
                const bf16 h = __float2bfloat16_rn(v[i] * keep);
                if (g.out) g.out[grp * g.o_group + (size_t)row * g.ldo + n] = h;
                if (g.out_t) g.out_t[grp * g.ot_group + (size_t)n * g.ldot + row] = h;
              }
            }
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kCols);
}

template <int NT>
size_t gemm_smem() {
  return 2 * (size_t)(128 * kKC * 2 + NT * kKC * 2) + 1024;
}

template <int NT>
csd_status_t launch_gemm(const GemmArgs& g, int groups, cudaStream_t st) {
  CSD_CHECK(g.lda % 8 == 0 && g.ldb % 8 == 0 && g.K % 8 == 0 && g.a_group % 8 == 0 && g.b_group % 8 == 0,
            CSD_ERR_INVALID, "GEMM operands need 16-byte aligned rows");
  static std::atomic<bool> attr[64] = {};  // per device: limit raised (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr[dev]) {
    CSD_CUDA_TRY(raise_smem_limit(gemm_kernel<NT>, (int)gemm_smem<NT>()));
    if (dev < 64) attr[dev] = true;
  }
  dim3 grid((g.M + 127) / 128, (g.N + NT - 1) / NT, groups);
  gemm_kernel<NT><<<grid, kThreads, gemm_smem<NT>(), st>>>(g);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

// grid: (tiles, groups); tiles past a group's rows exit at once
__global__ void __launch_bounds__(kThreads) mlp_forward_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_base;
  const FwdGroup G = a.groups[blockIdx.y];
  const int row0 = blockIdx.x * 128;
  if (row0 >= G.rows) return;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    umma::tmem_alloc(&tmem_base, kH);
    umma::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    umma::bar_init(&bars[0], 1);
    umma::bar_init(&bars[1], 1);
    umma::bar_fence_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  forward_tile(a, G, row0, smem, bars, tmem_base);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem_base, kH);
}

csd_status_t launch_forward(const FwdArgs& a, int groups, int max_rows, cudaStream_t st) {
  static std::atomic<bool> attr[64] = {};  // per device: limit raised (any thread)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr[dev]) {
    CSD_CUDA_TRY(raise_smem_limit(mlp_forward_kernel, (int)kFwdSmem));
    if (dev < 64) attr[dev] = true;
  }
  if (groups <= 0 || max_rows <= 0) return CSD_OK;
  dim3 grid((max_rows + 127) / 128, groups);
  mlp_forward_kernel<<<grid, kThreads, kFwdSmem, st>>>(a);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

// ------------------------------------------------------- CUDA-core kernels
// dlogit = (sigmoid(z) - y) / B and the BCE-with-logits loss; block per net.
__global__ void dlogit_kernel(const float* __restrict__ logits, const uint8_t* __restrict__ y, int B,
                              float* __restrict__ dlogit, float* __restrict__ loss) {
  __shared__ float red[32];
  const int net = blockIdx.x;
  float l = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const float z = logits[(size_t)net * B + b], t = y[(size_t)net * B + b] ? 1.f : 0.f;
    const float sg = 1.f / (1.f + expf(-z));
    dlogit[(size_t)net * B + b] = (sg - t) / (float)B;
    l += fmaxf(z, 0.f) - z * t + log1pf(expf(-fabsf(z)));
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    loss[net] = t / (float)B;
  }
}

// Output layer: dW4[i] = sum_b dlogit[b] h3[b][i], db4 = sum_b dlogit[b],
// dz3[b][i] = bf16(dlogit[b] w4[i] [h3 > 0]) row-major and transposed.
// Block per (net, 32 columns); 32 x 32 tiles transposed through shared memory.
__global__ void out_backward_kernel(const bf16* __restrict__ h3t, const float* __restrict__ dlogit,
                                    const float* __restrict__ params, int B, float* __restrict__ grads,
                                    bf16* __restrict__ dz3, bf16* __restrict__ dz3t) {
  __shared__ bf16 tile[32][33];
  __shared__ float dw[32][33];
  const int net = blockIdx.y, i0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, nty = blockDim.x >> 5;
  const bf16* H = h3t + (size_t)net * kH * B;
  const float* dl = dlogit + (size_t)net * B;
  const float* pr = params + (size_t)net * kParams;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int b0 = 0; b0 < B; b0 += 32) {
    // rows i = i0 + ty + k * nty, columns b = b0 + tx (coalesced over b)
    for (int ii = ty; ii < 32; ii += nty) {
      const int i = i0 + ii, b = b0 + tx;
      float v = 0.f;
      if (b < B) {
        const float h = __bfloat162float(H[(size_t)i * B + b]);
        acc[ii / nty] = fmaf(dl[b], h, acc[ii / nty]);
        v = h > 0.f ? dl[b] * pr[oW4 + i] : 0.f;
        dz3t[(size_t)net * kH * B + (size_t)i * B + b] = __float2bfloat16_rn(v);
      }
      tile[ii][tx] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    for (int bb = ty; bb < 32; bb += nty) {
      const int b = b0 + bb;
      if (b < B) dz3[(size_t)net * B * kH + (size_t)b * kH + i0 + tx] = tile[tx][bb];
    }
    __syncthreads();
  }
  for (int k = 0; k < 4; ++k) {
    const int ii = ty + k * nty;
    if (ii < 32) {
      float v = acc[k];
      for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (tx == 0) dw[ii][0] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) grads[(size_t)net * kParams + oW4 + i0 + threadIdx.x] = dw[threadIdx.x][0];
  if (blockIdx.x == 0 && threadIdx.x < 32) {
    float v = 0.f;
    for (int b = threadIdx.x; b < B; b += 32) v += dl[b];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) grads[(size_t)net * kParams + oB4] = v;
  }
}

// bias gradient: g[net][o] = sum_b dzt[net][o][b]; warp per (net, o)
__global__ void bias_grad_kernel(const bf16* __restrict__ dzt, int B, int nets, float* __restrict__ grads, int off) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nets * kH) return;
  const int net = w / kH, o = w % kH;
  const bf16* row = dzt + (size_t)net * kH * B + (size_t)o * B;
  float v = 0.f;
  for (int b = lane; b < B; b += 32) v += __bfloat162float(row[b]);
  for (int s = 16; s; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  if (lane == 0) grads[(size_t)net * kParams + off + o] = v;
}

// bf16 weight copies (and the transposed W2, W3) from the f32 parameters
__global__ void weights_bf16_kernel(const float* __restrict__ params, int nets, bf16* __restrict__ wb) {
  const long long total = (long long)nets * (kH * kIn + 2 * kH * kH);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int net = (int)(t / (kH * kIn + 2 * kH * kH));
    const int e = (int)(t % (kH * kIn + 2 * kH * kH));
    const float* pr = params + (size_t)net * kParams;
    bf16* w = wb + (size_t)net * kBf;
    if (e < kH * kIn) {
      w[qW1 + e] = __float2bfloat16_rn(pr[oW1 + e]);
    } else if (e < kH * kIn + kH * kH) {
      const int f = e - kH * kIn, o = f / kH, i = f % kH;
      const bf16 v = __float2bfloat16_rn(pr[oW2 + f]);
      w[qW2 + f] = v;
      w[qW2t + i * kH + o] = v;
    } else {
      const int f = e - kH * kIn - kH * kH, o = f / kH, i = f % kH;
      const bf16 v = __float2bfloat16_rn(pr[oW3 + f]);
      w[qW3 + f] = v;
      w[qW3t + i * kH + o] = v;
    }
  }
}

// Adam (Kingma & Ba 2015) with bias correction; t is the 1-based step.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// f32 rows [n][dim] -> bf16 rows [n][16] scaled and zero padded
__global__ void to_bf16_rows_kernel(const float* __restrict__ x, long long n, int dim, float scale,
                                    bf16* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * kIn; t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / kIn;
    const int k = (int)(t % kIn);
    out[t] = __float2bfloat16_rn(k < dim ? x[r * dim + k] * scale : 0.f);
  }
}

}  // namespace mlp
}  // namespace csd

// ------------------------------------------------------------------ handle
struct csd_mlp_s {
  int device = 0;
  int nets = 0;
  std::vector<int> dims;
  float in_scale = 1.f;
  long long step = 0;
  csd::DevBuf params, grads, m, v, wb, groups, status;
  // training buffers (batch B)
  int batch = 0;
  csd::DevBuf xb, y, logits, dlogit, loss, xt, h1t, h2t, h3t, dz3, dz3t, dz2, dz2t, dz1t;
};

namespace csd {
namespace mlp {

static csd_status_t ensure_batch(csd_mlp_s* h, int B) {
  if (h->batch == B) return CSD_OK;
  const size_t n = (size_t)h->nets, b = (size_t)B;
  csd_status_t s;
  if ((s = h->xb.reserve(n * b * kIn * 2)) || (s = h->y.reserve(n * b)) || (s = h->logits.reserve(n * b * 4)) ||
      (s = h->dlogit.reserve(n * b * 4)) || (s = h->loss.reserve(n * 4)) || (s = h->xt.reserve(n * kIn * b * 2)) ||
      (s = h->h1t.reserve(n * kH * b * 2)) || (s = h->h2t.reserve(n * kH * b * 2)) ||
      (s = h->h3t.reserve(n * kH * b * 2)) || (s = h->dz3.reserve(n * b * kH * 2)) ||
      (s = h->dz3t.reserve(n * kH * b * 2)) || (s = h->dz2.reserve(n * b * kH * 2)) ||
      (s = h->dz2t.reserve(n * kH * b * 2)) || (s = h->dz1t.reserve(n * kH * b * 2)))
    return s;
  h->batch = B;
  return CSD_OK;
}

// forward (training outputs) + backward into h->grads for the batch in h->xb / h->y
static csd_status_t forward_backward(csd_mlp_s* h, int B, cudaStream_t st) {
  const int n = h->nets;
  std::vector<FwdGroup> gs(n);
  for (int i = 0; i < n; ++i) {
    FwdGroup& G = gs[i];
    G = FwdGroup{};
    G.xb = h->xb.as<bf16>() + (size_t)i * B * kIn;
    G.rows = B;
    G.dim = h->dims[i];
    G.net = i;
    G.logits = h->logits.as<float>() + (size_t)i * B;
    G.xt = h->xt.as<bf16>() + (size_t)i * kIn * B;
    G.h1t = h->h1t.as<bf16>() + (size_t)i * kH * B;
    G.h2t = h->h2t.as<bf16>() + (size_t)i * kH * B;
    G.h3t = h->h3t.as<bf16>() + (size_t)i * kH * B;
    G.ld_t = B;
  }
  csd_status_t s;
  if ((s = h->groups.reserve(gs.size() * sizeof(FwdGroup)))) return s;
  CSD_CUDA_TRY(cudaMemcpyAsync(h->groups.ptr, gs.data(), gs.size() * sizeof(FwdGroup), cudaMemcpyHostToDevice, st));
  FwdArgs fa{h->groups.as<FwdGroup>(), h->wb.as<bf16>(), h->params.as<float>(), h->in_scale, h->status.as<int>()};
  if ((s = launch_forward(fa, n, B, st))) return s;
  dlogit_kernel<<<n, 256, 0, st>>>(h->logits.as<float>(), h->y.as<uint8_t>(), B, h->dlogit.as<float>(),
                                   h->loss.as<float>());
  out_backward_kernel<<<dim3(kH / 32, n), 256, 0, st>>>(h->h3t.as<bf16>(), h->dlogit.as<float>(),
                                                         h->params.as<float>(), B, h->grads.as<float>(),
                                                         h->dz3.as<bf16>(), h->dz3t.as<bf16>());
  CSD_CUDA_TRY(cudaGetLastError());
  const long long hb = (long long)kH * B, bh = (long long)B * kH;
  float* gr = h->grads.as<float>();
  const int bias_blocks = (n * kH * 32 + 255) / 256;
  // layer 3
  GemmArgs g{};
  g.status = h->status.as<int>();
  g.A = h->dz3t.as<bf16>(); g.a_group = hb; g.lda = B;
  g.B = h->h2t.as<bf16>(); g.b_group = hb; g.ldb = B;
  g.M = kH; g.N = kH; g.K = B; g.epi = kEpiF32;
  g.D = gr + oW3; g.d_group = kParams; g.ldd = kH;
  if ((s = launch_gemm<256>(g, n, st))) return s;
  bias_grad_kernel<<<bias_blocks, 256, 0, st>>>(h->dz3t.as<bf16>(), B, n, gr, oB3);
  g = GemmArgs{};
  g.status = h->status.as<int>();
  g.A = h->dz3.as<bf16>(); g.a_group = bh; g.lda = kH;
  g.B = h->wb.as<bf16>() + qW3t; g.b_group = kBf; g.ldb = kH;
  g.M = B; g.N = kH; g.K = kH; g.epi = kEpiReluGrad;
  g.mask_t = h->h2t.as<bf16>(); g.mt_group = hb; g.ldmt = B;
  g.out = h->dz2.as<bf16>(); g.o_group = bh; g.ldo = kH;
  g.out_t = h->dz2t.as<bf16>(); g.ot_group = hb; g.ldot = B;
  if ((s = launch_gemm<256>(g, n, st))) return s;
  // layer 2
  g = GemmArgs{};
  g.status = h->status.as<int>();
  g.A = h->dz2t.as<bf16>(); g.a_group = hb; g.lda = B;
  g.B = h->h1t.as<bf16>(); g.b_group = hb; g.ldb = B;
  g.M = kH; g.N = kH; g.K = B; g.epi = kEpiF32;
  g.D = gr + oW2; g.d_group = kParams; g.ldd = kH;
  if ((s = launch_gemm<256>(g, n, st))) return s;
  bias_grad_kernel<<<bias_blocks, 256, 0, st>>>(h->dz2t.as<bf16>(), B, n, gr, oB2);
  g = GemmArgs{};
  g.status = h->status.as<int>();
  g.A = h->dz2.as<bf16>(); g.a_group = bh; g.lda = kH;
  g.B = h->wb.as<bf16>() + qW2t; g.b_group = kBf; g.ldb = kH;
  g.M = B; g.N = kH; g.K = kH; g.epi = kEpiReluGrad;
  g.mask_t = h->h1t.as<bf16>(); g.mt_group = hb; g.ldmt = B;
  g.out_t = h->dz1t.as<bf16>(); g.ot_group = hb; g.ldot = B;
  if ((s = launch_gemm<256>(g, n, st))) return s;
  // layer 1
  g = GemmArgs{};
  g.status = h->status.as<int>();
  g.A = h->dz1t.as<bf16>(); g.a_group = hb; g.lda = B;
  g.B = h->xt.as<bf16>(); g.b_group = (long long)kIn * B; g.ldb = B;
  g.M = kH; g.N = kIn; g.K = B; g.epi = kEpiF32;
  g.D = gr + oW1; g.d_group = kParams; g.ldd = kIn;
  if ((s = launch_gemm<16>(g, n, st))) return s;
  bias_grad_kernel<<<bias_blocks, 256, 0, st>>>(h->dz1t.as<bf16>(), B, n, gr, oB1);
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

static csd_status_t refresh_bf16(csd_mlp_s* h, cudaStream_t st) {
  weights_bf16_kernel<<<1024, 256, 0, st>>>(h->params.as<float>(), h->nets, h->wb.as<bf16>());
  CSD_CUDA_TRY(cudaGetLastError());
  return CSD_OK;
}

static csd_status_t check_status(csd_mlp_s* h, cudaStream_t st) {
  int v = 0;
  CSD_CUDA_TRY(cudaMemcpyAsync(&v, h->status.ptr, 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  if (v) {
    set_error("a tensor-core barrier wait timed out in the surrogate kernels");
    return CSD_ERR_CUDA;
  }
  return CSD_OK;
}

struct DeviceScope {
  int cur = 0, dev = 0;
  explicit DeviceScope(int d) : dev(d) {
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
  }
  ~DeviceScope() {
    if (cur != dev) cudaSetDevice(cur);
  }
};

}  // namespace mlp
}  // namespace csd

using namespace csd;
using namespace csd::mlp;

namespace csd {
MlpView mlp_view(csd_mlp_t h) {
  return MlpView{h->wb.ptr, h->params.as<float>(), h->in_scale, h->nets, h->dims.data(), h->device};
}
}  // namespace csd

extern "C" {

int32_t csd_mlp_num_params(void) { return kParams; }

csd_status_t csd_mlp_create(int32_t nets, const int32_t* dims, float in_scale, uint64_t seed, csd_mlp_t* out) {
  CSD_CHECK(nets > 0 && dims && out, CSD_ERR_INVALID, "bad MLP arguments");
  *out = nullptr;
  for (int i = 0; i < nets; ++i)
    CSD_CHECK(dims[i] >= 1 && dims[i] <= kIn, CSD_ERR_DIMENSION, "MLP input dimension must be in [1, 16]");
  std::unique_ptr<csd_mlp_s> h(new csd_mlp_s());
  cudaGetDevice(&h->device);
  h->nets = nets;
  h->dims.assign(dims, dims + nets);
  h->in_scale = in_scale;
  const size_t P = (size_t)nets * kParams;
  csd_status_t s;
  if ((s = h->params.reserve(P * 4)) || (s = h->grads.reserve(P * 4)) || (s = h->m.reserve(P * 4)) ||
      (s = h->v.reserve(P * 4)) || (s = h->wb.reserve((size_t)nets * kBf * 2)) || (s = h->status.reserve(16)))
    return s;
  // He-uniform initialisation from a seeded 64-bit LCG (Knuth's MMIX constants); biases zero.
  std::vector<float> p(P, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((st >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f;
  };
  for (int n = 0; n < nets; ++n) {
    float* q = p.data() + (size_t)n * kParams;
    const float a1 = std::sqrt(6.f / dims[n]), a = std::sqrt(6.f / kH);
    for (int o = 0; o < kH; ++o)
      for (int i = 0; i < kIn; ++i) q[oW1 + o * kIn + i] = i < dims[n] ? a1 * uni() : 0.f;
    for (int e = 0; e < kH * kH; ++e) q[oW2 + e] = a * uni();
    for (int e = 0; e < kH * kH; ++e) q[oW3 + e] = a * uni();
    for (int e = 0; e < kH; ++e) q[oW4 + e] = std::sqrt(3.f / kH) * uni();
  }
  CSD_CUDA_TRY(cudaMemcpy(h->params.ptr, p.data(), P * 4, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMemset(h->m.ptr, 0, P * 4));
  CSD_CUDA_TRY(cudaMemset(h->v.ptr, 0, P * 4));
  CSD_CUDA_TRY(cudaMemset(h->grads.ptr, 0, P * 4));
  CSD_CUDA_TRY(cudaMemset(h->status.ptr, 0, 16));
  if ((s = refresh_bf16(h.get(), 0))) return s;
  CSD_CUDA_TRY(cudaDeviceSynchronize());
  *out = h.release();
  return CSD_OK;
}

csd_status_t csd_mlp_destroy(csd_mlp_t h) {
  if (!h) return CSD_OK;
  DeviceScope ds(h->device);
  delete h;
  return CSD_OK;
}

csd_status_t csd_mlp_get_params(csd_mlp_t h, float* params) {
  CSD_CHECK(h && params, CSD_ERR_INVALID, "null argument");
  DeviceScope ds(h->device);
  CSD_CUDA_TRY(cudaMemcpy(params, h->params.ptr, (size_t)h->nets * kParams * 4, cudaMemcpyDeviceToHost));
  return CSD_OK;
}

csd_status_t csd_mlp_set_params(csd_mlp_t h, const float* params) {
  CSD_CHECK(h && params, CSD_ERR_INVALID, "null argument");
  DeviceScope ds(h->device);
  CSD_CUDA_TRY(cudaMemcpy(h->params.ptr, params, (size_t)h->nets * kParams * 4, cudaMemcpyHostToDevice));
  csd_status_t s = refresh_bf16(h, 0);
  if (s) return s;
  CSD_CUDA_TRY(cudaDeviceSynchronize());
  return CSD_OK;
}

csd_status_t csd_mlp_infer(csd_mlp_t h, int32_t groups, const int32_t* net, const int32_t* rows, const float* x,
                           float* logits, int32_t flags, void* stream) {
  CSD_CHECK(h && groups >= 0 && (groups == 0 || (net && rows && x && logits)), CSD_ERR_INVALID, "null argument");
  DeviceScope ds(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<FwdGroup> gs(groups);
  size_t total_x = 0, total_r = 0;
  int max_rows = 0;
  for (int i = 0; i < groups; ++i) {
    CSD_CHECK(net[i] >= 0 && net[i] < h->nets && rows[i] >= 0, CSD_ERR_INVALID, "bad net index or row count");
    total_x += (size_t)rows[i] * h->dims[net[i]];
    total_r += rows[i];
    max_rows = std::max(max_rows, (int)rows[i]);
  }
  const bool dev = (flags & CSD_PTR_DEVICE) != 0;
  DevBuf dx, dl;
  const float* xd = x;
  float* ld = logits;
  csd_status_t s;
  if (!dev) {
    if ((s = dx.reserve(total_x * 4 + 16)) || (s = dl.reserve(total_r * 4 + 16))) return s;
    CSD_CUDA_TRY(cudaMemcpyAsync(dx.ptr, x, total_x * 4, cudaMemcpyHostToDevice, st));
    xd = dx.as<float>();
    ld = dl.as<float>();
  }
  size_t ox = 0, orow = 0;
  for (int i = 0; i < groups; ++i) {
    gs[i] = FwdGroup{};
    gs[i].x = xd + ox;
    gs[i].rows = rows[i];
    gs[i].dim = h->dims[net[i]];
    gs[i].net = net[i];
    gs[i].logits = ld + orow;
    ox += (size_t)rows[i] * gs[i].dim;
    orow += rows[i];
  }
  DevBuf dg;
  if ((s = dg.reserve(gs.size() * sizeof(FwdGroup) + 16))) return s;
  CSD_CUDA_TRY(cudaMemcpyAsync(dg.ptr, gs.data(), gs.size() * sizeof(FwdGroup), cudaMemcpyHostToDevice, st));
  FwdArgs fa{dg.as<FwdGroup>(), h->wb.as<bf16>(), h->params.as<float>(), h->in_scale, h->status.as<int>()};
  if ((s = launch_forward(fa, groups, max_rows, st))) return s;
  if (!dev) CSD_CUDA_TRY(cudaMemcpyAsync(logits, ld, total_r * 4, cudaMemcpyDeviceToHost, st));
  return check_status(h, st);
}

csd_status_t csd_mlp_gradients(csd_mlp_t h, const float* x, const uint8_t* y, int32_t batch, float* grads,
                               float* loss) {
  CSD_CHECK(h && x && y && grads && batch > 0 && batch % 32 == 0, CSD_ERR_INVALID,
            "gradients need host x, y, grads and a batch that is a multiple of 32");
  DeviceScope ds(h->device);
  csd_status_t s;
  if ((s = ensure_batch(h, batch))) return s;
  size_t off = 0;
  DevBuf dx;
  size_t total = 0;
  for (int i = 0; i < h->nets; ++i) total += (size_t)batch * h->dims[i];
  if ((s = dx.reserve(total * 4))) return s;
  CSD_CUDA_TRY(cudaMemcpy(dx.ptr, x, total * 4, cudaMemcpyHostToDevice));
  for (int i = 0; i < h->nets; ++i) {
    to_bf16_rows_kernel<<<256, 256>>>(dx.as<float>() + off, batch, h->dims[i], h->in_scale,
                                      h->xb.as<bf16>() + (size_t)i * batch * kIn);
    off += (size_t)batch * h->dims[i];
  }
  CSD_CUDA_TRY(cudaMemcpy(h->y.ptr, y, (size_t)h->nets * batch, cudaMemcpyHostToDevice));
  if ((s = forward_backward(h, batch, 0))) return s;
  if ((s = check_status(h, 0))) return s;
  CSD_CUDA_TRY(cudaMemcpy(grads, h->grads.ptr, (size_t)h->nets * kParams * 4, cudaMemcpyDeviceToHost));
  if (loss) CSD_CUDA_TRY(cudaMemcpy(loss, h->loss.ptr, (size_t)h->nets * 4, cudaMemcpyDeviceToHost));
  return CSD_OK;
}

csd_status_t csd_mlp_train(csd_mlp_t h, const float* x, const uint8_t* y, int32_t n, int32_t batch, int32_t steps,
                           float lr, float* loss_history, void* stream) {
  CSD_CHECK(h && x && y && n > 0 && batch > 0 && batch % 32 == 0 && n % batch == 0 && steps >= 0, CSD_ERR_INVALID,
            "training needs device x [nets][n][dim], y [nets][n], a batch that is a multiple of 32 dividing n");
  DeviceScope ds(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  csd_status_t s;
  if ((s = ensure_batch(h, batch))) return s;
  // the whole dataset as bf16 rows, then per step copy one contiguous batch per net
  DevBuf xall;
  if ((s = xall.reserve((size_t)h->nets * n * kIn * 2))) return s;
  size_t off = 0;
  for (int i = 0; i < h->nets; ++i) {
    to_bf16_rows_kernel<<<1024, 256, 0, st>>>(x + off, n, h->dims[i], h->in_scale,
                                              xall.as<bf16>() + (size_t)i * n * kIn);
    off += (size_t)n * h->dims[i];
  }
  CSD_CUDA_TRY(cudaGetLastError());
  const long long P = (long long)h->nets * kParams;
  std::vector<float> lh(h->nets);
  for (int t = 0; t < steps; ++t) {
    const int start = (int)(((long long)t * batch) % n);
    for (int i = 0; i < h->nets; ++i) {
      CSD_CUDA_TRY(cudaMemcpyAsync(h->xb.as<bf16>() + (size_t)i * batch * kIn, xall.as<bf16>() + ((size_t)i * n + start) * kIn,
                                   (size_t)batch * kIn * 2, cudaMemcpyDeviceToDevice, st));
      CSD_CUDA_TRY(cudaMemcpyAsync(h->y.as<uint8_t>() + (size_t)i * batch, y + (size_t)i * n + start, batch,
                                   cudaMemcpyDeviceToDevice, st));
    }
    if ((s = forward_backward(h, batch, st))) return s;
    h->step += 1;
    const float c1 = 1.f - std::pow(0.9f, (float)h->step), c2 = 1.f - std::pow(0.999f, (float)h->step);
    adam_kernel<<<2048, 256, 0, st>>>(h->params.as<float>(), h->grads.as<float>(), h->m.as<float>(), h->v.as<float>(),
                                      P, lr, 0.9f, 0.999f, 1e-8f, c1, c2);
    if ((s = refresh_bf16(h, st))) return s;
    if (loss_history) {
      CSD_CUDA_TRY(cudaMemcpyAsync(lh.data(), h->loss.ptr, (size_t)h->nets * 4, cudaMemcpyDeviceToHost, st));
      CSD_CUDA_TRY(cudaStreamSynchronize(st));
      double m = 0;
      for (float v : lh) m += v;
      loss_history[t] = (float)(m / h->nets);
    }
  }
  return check_status(h, st);
}

csd_status_t csd_mlp_gemm_test(const uint16_t* A, const uint16_t* B, int32_t M, int32_t N, int32_t K, float* D) {
  CSD_CHECK(A && B && D && M > 0 && (N == 16 || N == 256) && K > 0 && K % 8 == 0, CSD_ERR_INVALID,
            "gemm test: N must be 16 or 256, K a multiple of 8");
  DevBuf da, db, dd, st;
  csd_status_t s;
  if ((s = da.reserve((size_t)M * K * 2)) || (s = db.reserve((size_t)N * K * 2)) || (s = dd.reserve((size_t)M * N * 4)) ||
      (s = st.reserve(16)))
    return s;
  CSD_CUDA_TRY(cudaMemcpy(da.ptr, A, (size_t)M * K * 2, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMemcpy(db.ptr, B, (size_t)N * K * 2, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMemset(st.ptr, 0, 16));
  GemmArgs g{};
  g.A = da.as<bf16>(); g.lda = K;
  g.B = db.as<bf16>(); g.ldb = K;
  g.M = M; g.N = N; g.K = K; g.epi = kEpiF32;
  g.D = dd.as<float>(); g.ldd = N;
  g.status = st.as<int>();
  s = N == 16 ? launch_gemm<16>(g, 1, 0) : launch_gemm<256>(g, 1, 0);
  if (s) return s;
  CSD_CUDA_TRY(cudaDeviceSynchronize());
  int v = 0;
  CSD_CUDA_TRY(cudaMemcpy(&v, st.ptr, 4, cudaMemcpyDeviceToHost));
  CSD_CHECK(v == 0, CSD_ERR_CUDA, "tensor-core barrier wait timed out");
  CSD_CUDA_TRY(cudaMemcpy(D, dd.ptr, (size_t)M * N * 4, cudaMemcpyDeviceToHost));
  return CSD_OK;
}

}  // extern "C"
