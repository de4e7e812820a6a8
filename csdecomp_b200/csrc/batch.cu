// batch.cu -- many EI-ZO inflations advancing together (no counterpart in the
// reference, which inflates one edge per executeEizo call,
// csdecomp/src/planning/cuda_edge_inflation_zero_order.cu:94-339).
//
// Every active slot (one inflation: its own plant, segment and domain) runs
// the same iteration k at the same time. The unadaptive sample count M_k
// depends only on k and the shared options, so every slot draws the same N_k.
// One iteration is five persistent kernels over (slot, chunk) work items:
//   sample -> check -> compact (+ the admissibility decision, on the device)
//   -> bisect -> faces
// plus a counter bump; the sequence is captured once as a CUDA graph and
// replayed, and the host reads one active-slot count per iteration. Each slot
// runs exactly the arithmetic of the single-inflation path (csd_inflator_*),
// so it produces the same region bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "eizo_core.cuh"
#include "mlp_core.cuh"
#include "sampler_core.cuh"

namespace csd {

struct SlotState {
  int plant;          // index into the batch's plant array
  int dim;
  int domain_faces;
  int nf;             // faces of the region so far
  int done;           // finished: admissible, iteration limit, or error
  int iters;          // iterations executed
  int K;              // collisions kept for this iteration's bisection
  int status;         // 2: face capacity exceeded
  long long a_off;    // floats: region A [capacity][dim]
  long long pr_off;   // floats: region as face-pair rows [capacity / 2 + 1][pair_stride(dim)]
  long long b_off;    // floats: region b [capacity]
  long long seg_off;  // floats: line start [dim], line end [dim]
  long long smp_off;  // floats: samples [n_max][dim]
  long long col_off;  // floats: collision points / projections [num_particles][dim] each
  long long dist_off; // floats: distances [num_particles]
  long long flag_off; // bytes: verdicts [n_max]
  long long configs;  // configurations checked: samples + bisection points
  EizoCounters cnt;
  // surrogate mode: sorted-order checking of this iteration's samples
  int pos;            // sorted positions checked so far
  int need;           // more positions must be checked
  int coll;           // colliding samples found
  int m_chk;          // checked samples among the first M
  int m_coll;         // colliding samples among the first M
  int ord;            // 1: checks this iteration's samples in surrogate order; 0: in sample order, all of them
  int k;              // the slot's iteration (slots refilled during a call run different iterations)
  int harvested;      // finished and listed for the host by the step kernel
};

static_assert(sizeof(SlotState) == 152, "slot record size is part of the transfer accounting");

struct BatchIter {    // device-side iteration state
  int k;              // current iteration
  int active;         // slots still running, counted by the faces kernel
  int last_active;    // the count of the iteration that just finished
  int num_act;        // length of the active-slot list of iteration k
  int max_nf8;        // most faces of an active slot with dim <= 8
  int max_nf16;       // most faces of an active slot with dim > 8
  int sample_next;    // work queues of the sampler, check and bisection launches: items claimed past the
  int check_next;     // first one per block (each zeroed before every launch that uses it)
  int bisect_next;
  int num_ord;        // active slots still checking in surrogate order (surrogate mode)
  int n_act;          // largest N_k of the active slots (work-item sizing)
  int num_fin;        // slots that finished in the last iteration, listed in BatchArgs::fin
};

struct BatchArgs {
  SlotState* slots;
  const DevPlant* plants;
  int num_slots;
  int n_max;          // max over k of N_k (buffer stride)
  int max_iters;
  int num_particles;
  int mixing;
  int bisection;
  int max_faces;
  int capacity;
  int cfg_max;        // largest check work item (configurations)
  int part_max;       // largest bisection work item (particles)
  float margin;
  uint32_t k0, k1;    // Philox key (seed)
  const int* n_tab;   // N_k
  const int* m_tab;   // M_k
  const float* thr_tab;  // (1 - tau) * eps * M_k
  float* fpool;
  uint8_t* bpool;
  BatchIter* it;
  int* act;           // active-slot list of iteration k (slot indices, ascending)
  int* fin;           // slots that finished in the last iteration (the host harvests and refills them)
  // surrogate mode (mlp_wb null: off)
  const void* mlp_wb;
  const float* mlp_params;
  float mlp_scale;
  float stop_logit;   // keep checking a decided-inadmissible slot while the next score is at least this
  float* scores;      // [slot][n_max] logits
  int* order;         // [slot][n_max] sample indices, most likely colliding first
  int rounds;         // check rounds per iteration
  int round_base;     // positions of the first round; round r ends at base * (2^(r+1) - 1)
  int* status;        // tensor-core barrier timeout
};

// Sorted positions [round_begin, round_end) checked in round r (the last round runs to N).
static __device__ __forceinline__ int round_end(const BatchArgs& a, int r, int N) {
  if (r >= a.rounds - 1) return N;
  const long long e = (long long)a.round_base * ((2ll << r) - 1);
  return e < N ? (int)e : N;
}
static __device__ __forceinline__ int round_begin(const BatchArgs& a, int r, int N) {
  return r == 0 ? 0 : round_end(a, r - 1, N);
}

// Work-item size for `total` units over the grid: about four items per
// block, a multiple of the block's warps, at most `cap`.
static __device__ __forceinline__ int item_size(int64_t total, int cap, int nw) {
  int64_t c = total / (4 * (int64_t)gridDim.x);
  c = c < nw ? nw : c > cap ? cap : c;
  return (int)(c / nw) * nw;
}

// Work queue of a launch: block b starts with item b; whenever a block has
// finished an item it claims the next unclaimed one from `counter` (zeroed
// before the launch), so blocks that drew costly items (large regions, big
// plants) do not hold up a launch while others idle. Block-uniform result.
static __device__ __forceinline__ int claim_item(int* counter) {
  __shared__ int next;
  if (threadIdx.x == 0) next = gridDim.x + atomicAdd(counter, 1);
  __syncthreads();
  const int it = next;
  __syncthreads();  // every thread has read `next` before thread 0 writes it again
  return it;
}

// Staging buffer of a sampler variant with MINB resident blocks per SM: the
// largest that MINB blocks (with their static shared memory) fit in the SM.
template <int MINB>
struct SampleStage {
  static constexpr size_t bytes = (MINB == 1 ? 200 : MINB == 2 ? 104 : 68) * size_t(1024);
  static_assert(MINB * (bytes + 5120) <= 227 * 1024, "MINB staging buffers fit one SM");
};

// ------------------------------------------------------------------ kernels
// Chains of the active slots in work items (slot, chunk of chains), handed
// out by the work queue it->sample_next (a slot's cost grows with its faces
// and dimension, so fixed ranges of items would leave blocks idle). A block
// stages each new slot's face-pair rows in shared memory when they fit its
// buffer (else the chains read them from global memory, through L1) and runs
// the chains with G lanes each: G from the total chain count (8 when the
// batch is full, up to 32 in the tail), widened so that no lane holds more
// than KP face pairs. Each chain's draws and output row follow from its index
// alone and its arithmetic does not depend on G, so neither the order in
// which blocks take items nor the variant changes a sample.
template <int KP, int MINB>
__global__ void __launch_bounds__(256, MINB) batch_sample_kernel(BatchArgs a) {
  extern __shared__ __align__(16) float smf[];  // the face loop reads 16-byte vectors
  __shared__ GroupScratch gsa[kMaxWideGroups];
  const int N = a.it->n_act;  // items per slot are sized by the largest active N_k
  const int64_t total = (int64_t)a.it->num_act * N;
  const int G0 = group_width(total, (int64_t)gridDim.x * (blockDim.x >> 5));
  int64_t c = total / (16 * (int64_t)gridDim.x);
  c = c < 32 ? 32 : c > 1024 ? 1024 : c;
  const int chunk = (int)(c / 32) * 32;
  const int ips = (N + chunk - 1) / chunk;
  const int items = a.it->num_act * ips;  // at most slots * N / 32
  constexpr int stage_floats = (int)(SampleStage<MINB>::bytes / sizeof(float));
  int staged = -1;
  for (int it = blockIdx.x; it < items;) {
    const int slot = a.act[it / ips], first = (int)(it % ips) * chunk;
    const SlotState& S = a.slots[slot];
    const int Ns = a.n_tab[S.k];
    if (first >= Ns) {  // past this slot's chains (uniform across the block)
      it = claim_item(&a.it->sample_next);
      continue;
    }
    const int last = min(Ns, first + chunk);
    const int dim = S.dim, P = (S.nf + 1) >> 1, rs = pair_stride(dim);
    const float* rows = a.fpool + S.pr_off;
    const float* ls = a.fpool + S.seg_off;
    float* out = a.fpool + S.smp_off;
    const int G = pair_group_width(G0, P, KP);  // the batch refuses capacities that need more than 256 lanes
    const bool fits = P * rs <= stage_floats;
    if (fits && staged != slot) {
      __syncthreads();  // the previous slot's chains are done with the buffer
      stage_pairs(rows, P, rs, smf);
      __syncthreads();
      staged = slot;
    }
    // separate calls for the staged and the global rows, so that the staged face loop reads shared memory
    // with shared-memory loads (a pointer that may be either would make every load a generic one)
    if (fits) {
      if (dim <= 8)
        sample_region<8, KP>(G, smf, P, dim, ls, first, last, a.mixing, a.k0, a.k1, 0u, out, gsa);
      else
        sample_region<16, KP>(G, smf, P, dim, ls, first, last, a.mixing, a.k0, a.k1, 0u, out, gsa);
    } else {
      if (dim <= 8)
        sample_region<8, KP>(G, rows, P, dim, ls, first, last, a.mixing, a.k0, a.k1, 0u, out, gsa);
      else
        sample_region<16, KP>(G, rows, P, dim, ls, first, last, a.mixing, a.k0, a.k1, 0u, out, gsa);
    }
    it = claim_item(&a.it->sample_next);
  }
}

// Block per slot (slots slot0, slot0 + 1, ...): the face-pair rows of the
// domain (start slacks at the slot's segment start).
__global__ void batch_init_rows_kernel(BatchArgs a, int slot0) {
  const int slot = slot0 + (int)blockIdx.x;
  if (slot >= a.num_slots) return;
  const SlotState& S = a.slots[slot];
  put_faces(a.fpool + S.a_off, a.fpool + S.b_off, S.nf, S.dim, a.fpool + S.seg_off, a.fpool + S.pr_off, threadIdx.x,
            blockDim.x);
}

// Loads plant `pi` into the block's shared DevPlant and stages its statics.
template <bool SM>
static __device__ bool block_plant(const BatchArgs& a, int pi, DevPlant* sp, int* cur, float4* smem4, uint64_t* bar) {
  if (*cur == pi) return true;
  __syncthreads();
  if (threadIdx.x == 0) {
    *sp = a.plants[pi];
    *cur = pi;
  }
  __syncthreads();
  if (SM) return stage_statics(*sp, smem4, bar);
  return true;
}

template <bool SM>
static __device__ __forceinline__ WarpCtx<SM> batch_ctx(const DevPlant& p, float4* smem4, int static_floats) {
  WarpCtx<SM> w;
  const int warp = threadIdx.x >> 5;
  w.ok = true;
  w.stat = SM ? smem4 : p.statics;
  w.aabb = SM ? smem4 + 4 * p.num_static : p.aabb;
  float* wbase = reinterpret_cast<float*>(smem4) + (SM ? static_floats : 0);
  w.X = wbase + warp * warp_floats(p);
  w.qs = w.X + p.num_slots * 12;
  w.q1 = w.qs + kMaxDim;
  w.q2 = w.q1 + kMaxDim;
  w.pose = w.q2 + kMaxDim;
  return w;
}

// Work item = (active slot, chunk of configurations), sized so that the grid
// gets about four items per block whether 256 slots or one are active; items
// are handed out by the work queue it->check_next (plants differ in cost).
template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) batch_check_kernel(BatchArgs a, int static_floats) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  __shared__ DevPlant sp;
  __shared__ int cur;
  if (threadIdx.x == 0) cur = -1;
  __syncthreads();
  const int N = a.it->n_act;  // items per slot are sized by the largest active N_k
  const int na = a.it->num_act;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int c = item_size((int64_t)na * N, a.cfg_max, nw);
  const int ips = (N + c - 1) / c;
  const int items = na * ips;
  const VoxArgs none{nullptr, 0, 0.f, nullptr, nullptr, 0};
  for (int it = blockIdx.x; it < items; it = claim_item(&a.it->check_next)) {
    const int slot = a.act[it / ips], first = (it % ips) * c;
    const SlotState& S = a.slots[slot];
    const int Ns = a.n_tab[S.k];
    if (first >= Ns) continue;  // uniform across the block
    if (!block_plant<SM>(a, S.plant, &sp, &cur, smem4, &bar)) return;
    const WarpCtx<SM> w = batch_ctx<SM>(sp, smem4, static_floats);
    const float* smp = a.fpool + S.smp_off;
    uint8_t* flags = a.bpool + S.flag_off;
    const int last = std::min(Ns, first + c);
    for (int i = first + warp; i < last; i += nw) {
      if (lane < sp.dim) w.qs[lane] = smp[(int64_t)i * sp.dim + lane];
      __syncwarp();
      fk_warp(sp, w.qs, w.X, lane);
      const bool hit = check_config(sp, w.stat, w.aabb, w.X, w.pose, lane, none);
      if (lane == 0) flags[i] = hit ? 0 : 1;
    }
  }
}

// Block per slot: ordered compaction, first-M count, admissibility decision.
__global__ void __launch_bounds__(1024) batch_compact_kernel(BatchArgs a) {
  SlotState& S = a.slots[blockIdx.x];
  if (S.done) return;
  const int k = S.k;
  const int N = a.n_tab[k], M = a.m_tab[k];
  if (S.status == 2) {  // the previous faces kernel ran out of capacity
    if (threadIdx.x == 0) S.done = 1;
    return;
  }
  compact_block(a.bpool + S.flag_off, a.fpool + S.smp_off, N, M, a.num_particles, S.dim, a.fpool + S.col_off,
                &S.cnt);
  if (threadIdx.x == 0) {
    S.configs += N;
    if ((float)S.cnt.first_m <= a.thr_tab[k]) {
      S.done = 1;
      S.iters = k + 1;
      S.K = 0;
    } else {
      S.K = (int)std::min<uint32_t>(S.cnt.total, (uint32_t)a.num_particles);
      S.configs += (long long)S.K * a.bisection;
    }
  }
}

template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) batch_bisect_kernel(BatchArgs a, int static_floats) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  __shared__ DevPlant sp;
  __shared__ int cur;
  if (threadIdx.x == 0) cur = -1;
  __syncthreads();
  const int na = a.it->num_act;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int c = item_size((int64_t)na * a.num_particles, a.part_max, nw);
  const int ips = (a.num_particles + c - 1) / c;
  const int items = na * ips;
  const VoxArgs none{nullptr, 0, 0.f, nullptr, nullptr, 0};
  // work queue it->bisect_next: `for` advances through claim_item on every path, `continue` included
  for (int it = blockIdx.x; it < items; it = claim_item(&a.it->bisect_next)) {
    const int slot = a.act[it / ips], first = (it % ips) * c;
    const SlotState& S = a.slots[slot];
    if (S.done || first >= S.K) continue;  // uniform across the block
    if (!block_plant<SM>(a, S.plant, &sp, &cur, smem4, &bar)) return;
    const WarpCtx<SM> w = batch_ctx<SM>(sp, smem4, static_floats);
    const float* ls = a.fpool + S.seg_off;
    const int last = std::min(S.K, first + c);
    for (int i = first + warp; i < last; i += nw)
      bisect_particle<SM>(sp, w, i, S.dim, a.bisection, ls, ls + S.dim, none, a.fpool + S.col_off,
                          a.fpool + S.col_off + (int64_t)a.num_particles * S.dim, a.fpool + S.dist_off, lane);
  }
}

// Block per slot: greedy faces, iteration bookkeeping, active-slot count.
__global__ void __launch_bounds__(1024) batch_faces_kernel(BatchArgs a) {
  SlotState& S = a.slots[blockIdx.x];
  const int k = S.k;
  if (!S.done) {
    const float* ls = a.fpool + S.seg_off;
    faces_block(S.K, S.dim, a.max_faces, a.capacity, a.margin, ls, ls + S.dim, a.fpool + S.col_off,
                a.fpool + S.col_off + (int64_t)a.num_particles * S.dim, a.fpool + S.dist_off, a.fpool + S.a_off,
                a.fpool + S.b_off, &S.nf, &S.cnt, a.fpool + S.pr_off);
    if (threadIdx.x == 0) {
      S.iters = k + 1;
      S.status = S.cnt.status;
      if (k + 1 >= a.max_iters) S.done = 1;
    }
  }
  if (threadIdx.x == 0 && !S.done) atomicAdd(&a.it->active, 1);
}

// One block: advances k and rebuilds the active-slot list (ascending).
__global__ void __launch_bounds__(1024) batch_step_kernel(BatchArgs a) {
  __shared__ int warp_n[32];
  __shared__ int base, mf8, mf16, nord, nmax, nfin;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) {
    base = 0;
    mf8 = 0;
    mf16 = 0;
    nord = 0;
    nmax = 0;
    nfin = 0;
  }
  __syncthreads();
  for (int s0 = 0; s0 < a.num_slots; s0 += blockDim.x) {
    const int s = s0 + tid;
    const bool act = s < a.num_slots && !a.slots[s].done;
    if (act) {
      SlotState& S = a.slots[s];
      S.k += 1;  // the slot finished its iteration and runs the next
      atomicMax(S.dim <= 8 ? &mf8 : &mf16, S.nf);
      atomicMax(&nmax, a.n_tab[min(S.k, a.max_iters - 1)]);
      if (S.ord) atomicAdd(&nord, 1);
    } else if (s < a.num_slots && !a.slots[s].harvested) {
      a.slots[s].harvested = 1;
      a.fin[atomicAdd(&nfin, 1)] = s;  // finished this iteration: the host collects it
    }
    const unsigned m = __ballot_sync(0xffffffffu, act);
    if (lane == 0) warp_n[warp] = __popc(m);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += warp_n[w];
    if (act) a.act[off + __popc(m & ((1u << lane) - 1u))] = s;
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < nw; ++w) base += warp_n[w];
    __syncthreads();
  }
  if (tid == 0) {
    BatchIter* it = a.it;
    it->last_active = it->active;
    it->active = 0;
    it->k += 1;
    it->num_act = base;
    it->max_nf8 = mf8;
    it->max_nf16 = mf16;
    it->num_ord = nord;
    it->n_act = nmax;
    it->num_fin = nfin;
  }
}

// ---------------------------------------------------------- surrogate mode
// Logits of the active slots' samples: one CTA per (128-sample tile, active
// slot), the slot's plant indexing its net (fused tensor-core forward).
__global__ void __launch_bounds__(mlp::kThreads) batch_score_kernel(BatchArgs a) {
  extern __shared__ __align__(1024) char smem_raw[];
  char* smem = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_base;
  if ((int)blockIdx.y >= a.it->num_act) return;
  const int slot = a.act[blockIdx.y];
  const SlotState& S = a.slots[slot];
  const int N = a.n_tab[S.k];
  const int row0 = blockIdx.x * 128;
  if (row0 >= N) return;
  if (!S.ord) return;  // this slot checks in sample order: no scores needed
  mlp::FwdGroup G{};
  G.x = a.fpool + S.smp_off;
  G.rows = N;
  G.dim = S.dim;
  G.net = S.plant;
  G.logits = a.scores + (size_t)slot * a.n_max;
  const mlp::FwdArgs fa{nullptr, reinterpret_cast<const mlp::bf16*>(a.mlp_wb), a.mlp_params, a.mlp_scale, a.status};
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    umma::tmem_alloc(&tmem_base, mlp::kH);
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
  mlp::forward_tile(fa, G, row0, smem, bars, tmem_base);
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem_base, mlp::kH);
}

constexpr int kSortMax = 16384;  // samples per iteration the sort handles (shared-memory keys)

// Block per active slot: bitonic sort of (descending logit, index) keys in
// shared memory; writes the order and resets the slot's round counters.
__global__ void __launch_bounds__(1024) batch_sort_kernel(BatchArgs a) {
  extern __shared__ unsigned long long keys[];
  if ((int)blockIdx.x >= a.it->num_act) return;
  const int slot = a.act[blockIdx.x];
  const int N = a.n_tab[a.slots[slot].k];
  int* ord = a.order + (size_t)slot * a.n_max;
  uint8_t* flags = a.bpool + a.slots[slot].flag_off;
  const bool sorted = a.slots[slot].ord != 0;  // uniform across the block
  if (!sorted)
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      ord[i] = i;
      flags[i] = 2;  // unchecked this iteration
    }
  int P = 1;
  while (P < N) P <<= 1;
  if (!sorted) P = 0;
  const float* sc = a.scores + (size_t)slot * a.n_max;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    unsigned long long key = ~0ull;
    if (i < N) {
      uint32_t u = __float_as_uint(sc[i]);
      u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);  // order-preserving for finite floats
      key = ((unsigned long long)(~u) << 32) | (uint32_t)i;
    }
    keys[i] = key;
  }
  __syncthreads();
  for (int kk = 2; kk <= P; kk <<= 1)
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long x = keys[i], y = keys[ixj];
          if ((x > y) == ((i & kk) == 0)) {
            keys[i] = y;
            keys[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  if (sorted)
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      ord[i] = (int)(keys[i] & 0xffffffffu);
      flags[i] = 2;  // unchecked this iteration
    }
  if (threadIdx.x == 0) {
    SlotState& S = a.slots[slot];
    S.pos = 0;
    S.need = 1;
    S.coll = 0;
    S.m_chk = 0;
    S.m_coll = 0;
  }
}

// Round r of the sorted check: the positions of round r of every slot that
// still needs checking, in (slot, chunk) items from the work queue as
// batch_check_kernel.
template <bool SM>
__global__ void __launch_bounds__(32 * kWarpsPerBlock, 3) batch_check_sorted_kernel(BatchArgs a, int static_floats,
                                                                                   int r) {
  extern __shared__ float4 smem4[];
  __shared__ uint64_t bar;
  __shared__ DevPlant sp;
  __shared__ int cur;
  if (threadIdx.x == 0) cur = -1;
  __syncthreads();
  const int N = a.it->n_act;  // items are sized by the largest active N_k
  const int beg = round_begin(a, r, N), end = round_end(a, r, N), cnt = end - beg;
  if (cnt <= 0) return;
  const int na = a.it->num_act;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int c = item_size((int64_t)na * cnt, a.cfg_max, nw);
  const int ips = (cnt + c - 1) / c;
  const int items = na * ips;
  const VoxArgs none{nullptr, 0, 0.f, nullptr, nullptr, 0};
  // work queue it->check_next: `for` advances through claim_item on every path, `continue` included
  for (int it = blockIdx.x; it < items; it = claim_item(&a.it->check_next)) {
    const int slot = a.act[it / ips];
    const SlotState& S = a.slots[slot];
    const int Ns = a.n_tab[S.k], end_s = round_end(a, r, Ns), first = round_begin(a, r, Ns) + (it % ips) * c;
    if (S.done || !S.need || first >= end_s) continue;  // uniform across the block
    if (!block_plant<SM>(a, S.plant, &sp, &cur, smem4, &bar)) return;
    const WarpCtx<SM> w = batch_ctx<SM>(sp, smem4, static_floats);
    const float* smp = a.fpool + S.smp_off;
    const int* ord = a.order + (size_t)slot * a.n_max;
    uint8_t* flags = a.bpool + S.flag_off;
    const int last = min(end_s, first + c);
    for (int p = first + warp; p < last; p += nw) {
      const int i = ord[p];
      if (lane < sp.dim) w.qs[lane] = smp[(int64_t)i * sp.dim + lane];
      __syncwarp();
      fk_warp(sp, w.qs, w.X, lane);
      const bool hit = check_config(sp, w.stat, w.aabb, w.X, w.pose, lane, none);
      if (lane == 0) flags[i] = hit ? 0 : 1;
    }
  }
}

// Block per slot after round r: counts what the round found and decides
// whether the slot needs the next round. Undecided (first-M collisions within
// the threshold, first-M samples left): continue. Decided inadmissible:
// continue while fewer than num_particles collisions are known, positions
// remain and the next position's logit is at least stop_logit. Decided
// admissible (all first-M samples checked): stop.
__global__ void __launch_bounds__(256) batch_tally_kernel(BatchArgs a, int r) {
  __shared__ int red[3][8];
  SlotState& S = a.slots[blockIdx.x];
  if (S.done || !S.need) return;
  const int k = S.k, N = a.n_tab[k], M = a.m_tab[k];
  const int beg = round_begin(a, r, N), end = round_end(a, r, N);
  const int* ord = a.order + (size_t)blockIdx.x * a.n_max;
  const uint8_t* flags = a.bpool + S.flag_off;
  int coll = 0, mchk = 0, mcoll = 0;
  for (int p = beg + threadIdx.x; p < end; p += blockDim.x) {
    const int i = ord[p];
    const int c = flags[i] == 0;
    coll += c;
    mchk += i < M;
    mcoll += c && i < M;
  }
  for (int o = 16; o; o >>= 1) {
    coll += __shfl_xor_sync(0xffffffffu, coll, o);
    mchk += __shfl_xor_sync(0xffffffffu, mchk, o);
    mcoll += __shfl_xor_sync(0xffffffffu, mcoll, o);
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][warp] = coll;
    red[1][warp] = mchk;
    red[2][warp] = mcoll;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      coll += red[0][w];
      mchk += red[1][w];
      mcoll += red[2][w];
    }
    S.coll += coll;
    S.m_chk += mchk;
    S.m_coll += mcoll;
    S.pos = end;
    int need;
    if (!S.ord)
      need = end < N;  // sample order: every sample, as the batched form
    else if ((float)S.m_coll > a.thr_tab[k])
      need = S.coll < a.num_particles && end < N &&
             a.scores[(size_t)blockIdx.x * a.n_max + ord[end]] >= a.stop_logit;
    else
      need = S.m_chk < M;
    S.need = need;
  }
}

// Block per slot: ordered compaction (by sample index, as the plain form) of
// the colliding samples among those checked, the admissibility decision and
// the particle count. If no colliding sample was left unchecked, the
// particles are exactly the plain form's.
__global__ void __launch_bounds__(1024) batch_compact_sorted_kernel(BatchArgs a) {
  __shared__ int warp_n[32];
  __shared__ int base;
  SlotState& S = a.slots[blockIdx.x];
  if (S.done) return;
  if (S.status == 2) {
    if (threadIdx.x == 0) S.done = 1;
    return;
  }
  const int k = S.k, N = a.n_tab[k];
  const int dim = S.dim;
  const uint8_t* flags = a.bpool + S.flag_off;
  const float* smp = a.fpool + S.smp_off;
  float* cols = a.fpool + S.col_off;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int i0 = 0; i0 < N; i0 += blockDim.x) {
    const int i = i0 + tid;
    const bool c = i < N && flags[i] == 0;
    const unsigned m = __ballot_sync(0xffffffffu, c);
    if (lane == 0) warp_n[warp] = __popc(m);
    __syncthreads();
    int off = base;
    for (int w = 0; w < warp; ++w) off += warp_n[w];
    const int rank = off + __popc(m & ((1u << lane) - 1u));
    if (c && rank < a.num_particles)
      for (int d = 0; d < dim; ++d) cols[(size_t)rank * dim + d] = smp[(size_t)i * dim + d];
    __syncthreads();
    if (tid == 0)
      for (int w = 0; w < nw; ++w) base += warp_n[w];
    __syncthreads();
  }
  if (tid == 0) {
    // ordering that left fewer than 1/8 of the samples unchecked is not worth its
    // scoring, sort and rounds: the slot checks in sample order from now on
    if (S.ord && 8ll * (N - S.pos) < (long long)N) S.ord = 0;
    S.configs += S.pos;
    S.cnt.total = (uint32_t)base;
    S.cnt.first_m = (uint32_t)S.m_coll;
    if ((float)S.m_coll <= a.thr_tab[k]) {
      S.done = 1;
      S.iters = k + 1;
      S.K = 0;
    } else {
      S.K = min(base, a.num_particles);
      S.configs += (long long)S.K * a.bisection;
    }
  }
}

// Sampler variants the autotuner chooses from: KP face pairs per lane at
// most (register-held slacks; wider groups for larger regions) and MINB
// resident blocks per SM (register cap and staging buffer). Every variant
// yields the same samples.
using SampleFn = void (*)(BatchArgs);
struct SampleVariant {
  SampleFn fn;
  int kp, minb;
  size_t smem;   // staging buffer (SampleStage<minb>::bytes)
  int f8, f16;   // faces staged for dim <= 8 / <= 16
};
#define CSD_SAMPLE_VARIANT(KP, MINB)                                                                 \
  {                                                                                                  \
    batch_sample_kernel<KP, MINB>, KP, MINB, SampleStage<MINB>::bytes,                               \
        2 * (int)(SampleStage<MINB>::bytes / (pair_stride(8) * sizeof(float))),                      \
        2 * (int)(SampleStage<MINB>::bytes / (pair_stride(16) * sizeof(float)))                      \
  }
static const SampleVariant kSampleVariants[] = {
    CSD_SAMPLE_VARIANT(8, 1), CSD_SAMPLE_VARIANT(8, 2), CSD_SAMPLE_VARIANT(8, 3),
    CSD_SAMPLE_VARIANT(16, 1), CSD_SAMPLE_VARIANT(16, 2),
};
#undef CSD_SAMPLE_VARIANT
// Smallest KP of the variants: a region of up to 2 * 256 * kMinKP faces fits
// every variant's widest group.
constexpr int kMinKP = 8;
static_assert(2 * 256 * kMinKP >= kMaxRegionFaces, "every variant samples the largest region");
constexpr int kNumSampleVariants = (int)(sizeof(kSampleVariants) / sizeof(kSampleVariants[0]));
// Largest check work item (configurations) the autotuner chooses from.
constexpr int kCheckItemCaps[] = {8, 16, 32, 128, 512};
constexpr int kNumCheckVariants = (int)(sizeof(kCheckItemCaps) / sizeof(kCheckItemCaps[0]));
// profiled stages: sample, score, sort, check, compact, bisect, faces, step
constexpr int kStages = 8;

}  // namespace csd

// --------------------------------------------------------------------- handle
struct csd_batch_s {
  int device = 0;
  std::vector<csd_plant_t> plants;
  csd_eizo_options_t opt{};
  int max_slots = 0, capacity = 0, n_max = 0, max_dim = 0;
  bool sm = true;
  int static_floats = 0;
  size_t check_smem = 0;
  int check_grid = 0, bisect_grid = 0;
  int cfg_max = 128, part_max = 8;  // bisection: one particle per warp per item (every block busy)
  int sample_variant = 0;     // tuned (or set) variant
  int large_variant = 1;      // variant chosen once a slot's faces exceeded the tuned variant's staging
  int run_variant = 0;        // variant of the current iterations
  bool switch_large = true;   // false after csd_batch_set_shapes: run exactly the set variant
  int sample_grid[csd::kNumSampleVariants] = {};
  int tune_iters = 0;                               // iterations of the next inflate to tune on
  double tune_ms[csd::kNumSampleVariants + csd::kNumCheckVariants] = {};
  int tuned_iters = 0;
  // large regions: the first time a region outgrows the tuned variant's staging, the next
  // iteration times every sampler variant on its own inputs (kept until the next autotune)
  bool large_pending = false, large_tuned = false;
  double large_ms[csd::kNumSampleVariants] = {};
  std::vector<int> n_tab, m_tab;
  std::vector<float> thr_tab;
  csd::DevBuf plants_dev, slots_dev, tabs, fpool, bpool, iter, act, fin;
  // surrogate mode
  csd_mlp_t mlp = nullptr;
  float stop_logit = 0.f;
  int rounds = 3, round_base = 1024;
  csd::DevBuf scores, order, status;
  std::vector<long long> job_configs;  // configurations checked per inflation of the last call
  std::vector<int> act_host;
  cudaGraphExec_t graph = nullptr;
  int graph_slots = -1, graph_cfg = -1, graph_variant = -1;
  int graph_kernels = 0;        // kernel nodes of the captured iteration
  long long launches = 0;       // kernels launched by the last inflate
  const void* graph_mlp = nullptr;
  cudaStream_t graph_stream = nullptr;
  csd::BatchIter* host_iter = nullptr;
  bool profile = false;         // launch stage by stage with events instead of the graph
  cudaEvent_t ev[csd::kStages + 1] = {};
  double stage_ms[csd::kStages] = {};
  std::vector<float> iter_ms;   // profiling mode: [iteration][kStages] of the last inflate
  std::vector<int> iter_active; // slots active at the start of each iteration
  std::vector<int> iter_variant;  // sampler variant each iteration ran
  std::vector<int> iter_faces;    // most faces of an active slot when each iteration started
  double sample_flop = 0.0;     // profiling mode: sampler FLOPs of the last inflate ((2 d + 4) F per chain step)
  ~csd_batch_s() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (graph) cudaGraphExecDestroy(graph);
    if (graph_stream) cudaStreamDestroy(graph_stream);
    if (host_iter) cudaFreeHost(host_iter);
  }
};

using namespace csd;

namespace {

// Floats of one slot's face-pair rows, and of all its buffers (a multiple of
// 4, so every slot's rows start 16-byte aligned): pair rows, A, b, segment,
// samples, collision points and projections, distances.
size_t pair_floats(const csd_batch_s* h) {
  return ((size_t)h->capacity / 2 + 1) * (size_t)pair_stride(h->max_dim);
}
size_t slot_floats(const csd_batch_s* h) {
  const size_t D = (size_t)h->max_dim, np = h->opt.num_particles, cap = (size_t)h->capacity;
  const size_t f = pair_floats(h) + cap * D + cap + 2 * D + (size_t)h->n_max * D + 2 * np * D + np;
  return (f + 3) & ~size_t(3);
}

// Sampler variant for regions of up to nf8 (dim <= 8) and nf16 faces: the
// fastest by tuning time among those whose staging buffer holds them, else
// the one with the most room (faces beyond it are read from global memory).
int variant_for(const csd_batch_s* h, int nf8, int nf16) {
  const double* ms = h->large_tuned ? h->large_ms : h->tune_ms;
  int best = -1;
  for (int v = 0; v < kNumSampleVariants; ++v) {
    const SampleVariant& cv = kSampleVariants[v];
    if (cv.f8 >= nf8 && cv.f16 >= nf16 && (best < 0 || ms[v] < ms[best])) best = v;
  }
  if (best >= 0) return best;
  best = 0;
  for (int v = 1; v < kNumSampleVariants; ++v) {
    const SampleVariant &cv = kSampleVariants[v], &bv = kSampleVariants[best];
    const bool roomier = cv.f16 > bv.f16 || (cv.f16 == bv.f16 && cv.f8 > bv.f8);
    const bool same = cv.f16 == bv.f16 && cv.f8 == bv.f8;
    if (roomier || (same && ms[v] < ms[best])) best = v;
  }
  return best;
}

// One iteration's launches on stream s. ev (kStages + 1 events) brackets the
// stages for the profiling mode; skip_sample leaves out the sampler (the
// autotuner has just run it).
// Returns the number of kernels launched.
int launch_iteration(csd_batch_s* h, int num_slots, const BatchArgs& a, cudaStream_t s, cudaEvent_t* ev,
                     bool skip_sample = false) {
  if (!skip_sample) cudaMemsetAsync(&a.it->sample_next, 0, sizeof(int), s);  // the sampler's work queue
  if (ev) cudaEventRecord(ev[0], s);
  if (!skip_sample)
    kSampleVariants[h->run_variant].fn<<<h->sample_grid[h->run_variant], 256, kSampleVariants[h->run_variant].smem,
                                         s>>>(a);
  if (ev) cudaEventRecord(ev[1], s);
  if (a.mlp_wb) {
    batch_score_kernel<<<dim3((h->n_max + 127) / 128, num_slots), mlp::kThreads, mlp::kFwdSmem, s>>>(a);
    if (ev) cudaEventRecord(ev[2], s);
    batch_sort_kernel<<<num_slots, 1024, kSortMax * sizeof(unsigned long long), s>>>(a);
    if (ev) cudaEventRecord(ev[3], s);
    for (int r = 0; r < a.rounds; ++r) {
      cudaMemsetAsync(&a.it->check_next, 0, sizeof(int), s);
      if (h->sm)
        batch_check_sorted_kernel<true><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, h->static_floats,
                                                                                                  r);
      else
        batch_check_sorted_kernel<false><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, 0, r);
      batch_tally_kernel<<<num_slots, 256, 0, s>>>(a, r);
    }
    if (ev) cudaEventRecord(ev[4], s);
    batch_compact_sorted_kernel<<<num_slots, 1024, 0, s>>>(a);
  } else {
    if (ev) cudaEventRecord(ev[2], s);
    if (ev) cudaEventRecord(ev[3], s);
    cudaMemsetAsync(&a.it->check_next, 0, sizeof(int), s);
    if (h->sm)
      batch_check_kernel<true><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, h->static_floats);
    else
      batch_check_kernel<false><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, 0);
    if (ev) cudaEventRecord(ev[4], s);
    batch_compact_kernel<<<num_slots, 1024, 0, s>>>(a);
  }
  if (ev) cudaEventRecord(ev[5], s);
  cudaMemsetAsync(&a.it->bisect_next, 0, sizeof(int), s);
  if (h->sm)
    batch_bisect_kernel<true><<<h->bisect_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, h->static_floats);
  else
    batch_bisect_kernel<false><<<h->bisect_grid, 32 * kWarpsPerBlock, h->check_smem, s>>>(a, 0);
  if (ev) cudaEventRecord(ev[6], s);
  batch_faces_kernel<<<num_slots, 1024, 0, s>>>(a);
  if (ev) cudaEventRecord(ev[7], s);
  batch_step_kernel<<<1, 1024, 0, s>>>(a);
  if (ev) cudaEventRecord(ev[8], s);
  // sampler; score, sort, (check + tally) per round, compaction | check, compaction; bisect, faces, step
  return (skip_sample ? 0 : 1) + (a.mlp_wb ? 3 + 2 * a.rounds : 2) + 3;
}

csd_status_t build_graph(csd_batch_s* h, int num_slots, const BatchArgs& a) {
  if (h->graph && h->graph_slots == num_slots && h->graph_cfg == a.cfg_max && h->graph_variant == h->run_variant &&
      h->graph_mlp == a.mlp_wb)
    return CSD_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaStream_t s = h->graph_stream;
  cudaGraph_t g = nullptr;
  CSD_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  h->graph_kernels = launch_iteration(h, num_slots, a, s, nullptr);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess) {
    set_error(std::string("graph capture failed: ") + cudaGetErrorString(e));
    return CSD_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    set_error(std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    return CSD_ERR_CUDA;
  }
  h->graph_slots = num_slots;
  h->graph_cfg = a.cfg_max;
  h->graph_variant = h->run_variant;
  h->graph_mlp = a.mlp_wb;
  return CSD_OK;
}

}  // namespace

extern "C" {

csd_status_t csd_batch_create(const csd_plant_t* plants, int32_t num_plants, int32_t max_slots,
                              const csd_eizo_options_t* o, int32_t face_capacity, csd_batch_t* out) {
  CSD_CHECK(plants && num_plants > 0 && max_slots > 0 && o && out && face_capacity > 0, CSD_ERR_INVALID,
            "bad batch arguments");
  CSD_CHECK(face_capacity <= kMaxRegionFaces, CSD_ERR_CAPACITY,
            "face capacity above " + std::to_string(kMaxRegionFaces) + " (the sampler's largest region)");
  *out = nullptr;
  CSD_CHECK(o->num_particles >= 1 && o->max_iterations >= 1, CSD_ERR_INVALID,
            "num_particles and max_iterations must be positive");
  CSD_CHECK(o->tau > 0.f && o->tau < 1.f && o->epsilon > 0.f && o->delta > 0.f, CSD_ERR_INVALID,
            "bad epsilon/delta/tau");
  std::unique_ptr<csd_batch_s> h(new csd_batch_s());
  h->device = plants[0]->device;
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, h->device};
  h->opt = *o;
  h->max_slots = max_slots;
  h->capacity = face_capacity;
  int max_static = 0, max_wf = 0;
  std::vector<DevPlant> dps;
  for (int i = 0; i < num_plants; ++i) {
    CSD_CHECK(plants[i] && plants[i]->device == h->device, CSD_ERR_INVALID, "plants must live on one device");
    h->plants.push_back(plants[i]);
    dps.push_back(plants[i]->dp);
    CSD_CHECK(plants[i]->dp.dim >= 1 && plants[i]->dp.dim <= kMaxDim, CSD_ERR_DIMENSION, "plant dimension must be in [1, 16]");
    h->max_dim = std::max(h->max_dim, plants[i]->dp.dim);
    max_static = std::max(max_static, plants[i]->dp.static_bytes);
    max_wf = std::max(max_wf, warp_floats(plants[i]->dp));
  }
  // iteration tables (cuda_edge_inflation_zero_order.cu:113-119)
  for (uint32_t k = 0; k < o->max_iterations; ++k) {
    float delta_k = (float)(6 * o->delta / (M_PI * M_PI * (k + 1) * (k + 1)));
    uint32_t M = csd_num_samples_unadaptive(o->epsilon, delta_k, o->tau);
    h->m_tab.push_back((int)M);
    h->n_tab.push_back((int)std::max(M, o->num_particles));
    h->thr_tab.push_back((1 - o->tau) * o->epsilon * M);
  }
  h->n_max = *std::max_element(h->n_tab.begin(), h->n_tab.end());
  // the stage kernels number their work items (slot, 8 or more configurations) with 32-bit integers
  CSD_CHECK((int64_t)max_slots * (h->n_max / 8 + 1) + (1 << 20) < (int64_t)INT32_MAX, CSD_ERR_CAPACITY,
            "too many slots times samples per iteration");
  h->sm = max_static <= kStaticSmemLimit;
  h->static_floats = h->sm ? max_static / 4 : 0;
  h->check_smem = (size_t)max_wf * sizeof(float) * kWarpsPerBlock + (h->sm ? (size_t)max_static : 0);
  csd_status_t s;
  int g1 = 0, g2 = 0;
  int g3 = 0;
  if (h->sm) {
    if ((s = grid_for(batch_check_kernel<true>, h->check_smem, 1ll << 40, &g1, kWarpsPerBlock))) return s;
    if ((s = grid_for(batch_bisect_kernel<true>, h->check_smem, 1ll << 40, &g2, kWarpsPerBlock))) return s;
    if ((s = grid_for(batch_check_sorted_kernel<true>, h->check_smem, 1ll << 40, &g3, kWarpsPerBlock))) return s;
  } else {
    if ((s = grid_for(batch_check_kernel<false>, h->check_smem, 1ll << 40, &g1, kWarpsPerBlock))) return s;
    if ((s = grid_for(batch_bisect_kernel<false>, h->check_smem, 1ll << 40, &g2, kWarpsPerBlock))) return s;
    if ((s = grid_for(batch_check_sorted_kernel<false>, h->check_smem, 1ll << 40, &g3, kWarpsPerBlock))) return s;
  }
  h->check_grid = g1;
  h->bisect_grid = g2;
  for (int v = 0; v < kNumSampleVariants; ++v) {
    CSD_CUDA_TRY(raise_smem_limit(kSampleVariants[v].fn, (int)kSampleVariants[v].smem));
    int per_sm = 0;
    CSD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kSampleVariants[v].fn, 256,
                                                             kSampleVariants[v].smem));
    h->sample_grid[v] = device_sm_count() * std::max(1, per_sm);
  }
  // buffers
  const size_t per_slot_f = slot_floats(h.get());
  if ((s = h->plants_dev.reserve(dps.size() * sizeof(DevPlant))) || (s = h->slots_dev.reserve(max_slots * sizeof(SlotState))) ||
      (s = h->tabs.reserve(h->n_tab.size() * 12 + 64)) || (s = h->fpool.reserve(per_slot_f * max_slots * 4 + 256)) ||
      (s = h->bpool.reserve((size_t)h->n_max * max_slots + 256)) || (s = h->iter.reserve(sizeof(BatchIter))) ||
      (s = h->act.reserve((size_t)max_slots * 4)) || (s = h->fin.reserve((size_t)max_slots * 4)) ||
      (s = h->status.reserve(16)))
    return s;
  CSD_CUDA_TRY(cudaMemcpy(h->plants_dev.ptr, dps.data(), dps.size() * sizeof(DevPlant), cudaMemcpyHostToDevice));
  int* t = h->tabs.as<int>();
  const size_t K = h->n_tab.size();
  CSD_CUDA_TRY(cudaMemcpy(t, h->n_tab.data(), K * 4, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMemcpy(t + K, h->m_tab.data(), K * 4, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaMemcpy(t + 2 * K, h->thr_tab.data(), K * 4, cudaMemcpyHostToDevice));
  CSD_CUDA_TRY(cudaStreamCreateWithFlags(&h->graph_stream, cudaStreamNonBlocking));
  CSD_CUDA_TRY(cudaMallocHost((void**)&h->host_iter, sizeof(BatchIter)));
  *out = h.release();
  return CSD_OK;
}

csd_status_t csd_batch_destroy(csd_batch_t h) {
  if (!h) return CSD_OK;
  int cur = 0, dev = h->device;
  cudaGetDevice(&cur);
  if (cur != dev) cudaSetDevice(dev);
  delete h;
  if (cur != dev) cudaSetDevice(cur);
  return CSD_OK;
}

csd_status_t csd_batch_inflate(csd_batch_t h, int32_t n, const int32_t* slot_plant, const float* starts,
                               const float* ends, const float* domain_A, const float* domain_b,
                               const int32_t* domain_face_offsets, float* A_out, float* b_out, int32_t* num_faces,
                               int32_t* num_iterations, float* device_ms) {
  CSD_CHECK(h && n >= 0, CSD_ERR_INVALID, "bad inflation count");
  if (n == 0) return CSD_OK;
  CSD_CHECK(slot_plant && starts && ends && domain_A && domain_b && domain_face_offsets && A_out && b_out && num_faces,
            CSD_ERR_INVALID, "null argument");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, h->device};
  const size_t D = (size_t)h->max_dim, np = h->opt.num_particles, cap = (size_t)h->capacity;
  const size_t per_slot_f = slot_floats(h);
  const int ns = std::min<int>(n, h->max_slots);  // slots in use; inflations past them wait for a free slot
  // every inflation's inputs are checked before any work starts
  std::vector<size_t> q_off(n), a_row(n), out_off(n);
  size_t qoff = 0, arow = 0, ooff = 0;
  for (int i = 0; i < n; ++i) {
    const int pi = slot_plant[i];
    CSD_CHECK(pi >= 0 && pi < (int)h->plants.size(), CSD_ERR_INVALID, "slot plant index out of range");
    const int d = h->plants[pi]->dp.dim;
    const int f0 = domain_face_offsets[i], f1 = domain_face_offsets[i + 1];
    CSD_CHECK(f0 >= 0 && f1 >= f0, CSD_ERR_INVALID, "bad domain face offsets");
    CSD_CHECK(f1 - f0 <= 0.9 * h->capacity, CSD_ERR_CAPACITY, "domain uses almost all of the face capacity");
    // the segment must lie in the domain (CudaEdgeInflator::inflateEdge asserts it)
    for (int sidx = 0; sidx < 2; ++sidx) {
      const float* x = (sidx ? ends : starts) + qoff;
      for (int f = 0; f < f1 - f0; ++f) {
        float ax = 0.f;
        for (int k = 0; k < d; ++k) ax += domain_A[arow + (size_t)f * d + k] * x[k];
        if (!(ax <= domain_b[f0 + f] + 1e-9f)) {
          set_error("inflation " + std::to_string(i) + ": line segment endpoints must lie in the domain");
          return CSD_ERR_NOT_CONTAINED;
        }
      }
    }
    q_off[i] = qoff;
    a_row[i] = arow;
    out_off[i] = ooff;
    qoff += d;
    arow += (size_t)(f1 - f0) * d;
    ooff += cap * d;
  }
  cudaStream_t st = h->graph_stream;
  // the record of slot `slot` starting inflation `job`, and the upload of that inflation's domain and segment
  auto record = [&](int slot, int job) {
    SlotState S{};
    S.plant = slot_plant[job];
    S.dim = h->plants[S.plant]->dp.dim;
    S.domain_faces = domain_face_offsets[job + 1] - domain_face_offsets[job];
    S.nf = S.domain_faces;
    S.ord = 1;
    const long long base = (long long)(per_slot_f * slot);
    S.pr_off = base;  // 16-byte aligned: per_slot_f is a multiple of 4 floats
    S.a_off = S.pr_off + (long long)pair_floats(h);
    S.b_off = S.a_off + (long long)(cap * D);
    S.seg_off = S.b_off + (long long)cap;
    S.smp_off = S.seg_off + (long long)(2 * D);
    S.col_off = S.smp_off + (long long)((size_t)h->n_max * D);
    S.dist_off = S.col_off + (long long)(2 * np * D);
    S.flag_off = (long long)h->n_max * slot;
    return S;
  };
  auto upload = [&](const SlotState& S, int job) -> csd_status_t {
    const int d = S.dim, F = S.nf;
    float* fp = h->fpool.as<float>();
    CSD_CUDA_TRY(cudaMemcpyAsync(fp + S.a_off, domain_A + a_row[job], (size_t)F * d * 4, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(fp + S.b_off, domain_b + domain_face_offsets[job], (size_t)F * 4,
                                 cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(fp + S.seg_off, starts + q_off[job], d * 4, cudaMemcpyHostToDevice, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(fp + S.seg_off + d, ends + q_off[job], d * 4, cudaMemcpyHostToDevice, st));
    return CSD_OK;
  };
  std::vector<SlotState> slots(ns);
  std::vector<int> slot_job(ns);
  csd_status_t s;
  for (int i = 0; i < ns; ++i) {
    slots[i] = record(i, i);
    slot_job[i] = i;
    if ((s = upload(slots[i], i))) return s;
  }
  int next_job = ns;
  CSD_CUDA_TRY(cudaMemcpyAsync(h->slots_dev.ptr, slots.data(), ns * sizeof(SlotState), cudaMemcpyHostToDevice, st));
  BatchIter zero{};
  zero.num_act = ns;
  zero.n_act = h->n_tab[0];
  *h->host_iter = zero;
  CSD_CUDA_TRY(cudaMemcpyAsync(h->iter.ptr, h->host_iter, sizeof(BatchIter), cudaMemcpyHostToDevice, st));
  h->act_host.resize(ns);
  for (int i = 0; i < ns; ++i) h->act_host[i] = i;
  CSD_CUDA_TRY(cudaMemcpyAsync(h->act.ptr, h->act_host.data(), (size_t)ns * 4, cudaMemcpyHostToDevice, st));
  BatchArgs a{};
  a.slots = h->slots_dev.as<SlotState>();
  a.plants = h->plants_dev.as<DevPlant>();
  a.num_slots = ns;
  a.n_max = h->n_max;
  a.max_iters = (int)h->opt.max_iterations;
  a.num_particles = (int)h->opt.num_particles;
  a.mixing = (int)h->opt.mixing_steps;
  a.bisection = (int)h->opt.bisection_steps;
  a.max_faces = (int)h->opt.max_hyperplanes_per_iteration;
  a.capacity = h->capacity;
  a.margin = h->opt.configuration_margin;
  a.k0 = (uint32_t)h->opt.seed;
  a.k1 = (uint32_t)(h->opt.seed >> 32);
  const size_t K = h->n_tab.size();
  a.n_tab = h->tabs.as<int>();
  a.m_tab = h->tabs.as<int>() + K;
  a.thr_tab = reinterpret_cast<const float*>(h->tabs.as<int>() + 2 * K);
  a.fpool = h->fpool.as<float>();
  a.bpool = h->bpool.as<uint8_t>();
  a.it = h->iter.as<BatchIter>();
  a.act = h->act.as<int>();
  a.fin = h->fin.as<int>();
  a.cfg_max = h->cfg_max;
  a.part_max = h->part_max;
  if (h->mlp) {
    const MlpView mv = mlp_view(h->mlp);
    a.mlp_wb = mv.wb;
    a.mlp_params = mv.params;
    a.mlp_scale = mv.in_scale;
    a.stop_logit = h->stop_logit;
    a.scores = h->scores.as<float>();
    a.order = h->order.as<int>();
    a.rounds = h->rounds;
    a.round_base = h->round_base;
  }
  a.status = h->status.as<int>();
  CSD_CUDA_TRY(cudaMemsetAsync(h->status.ptr, 0, 16, st));
  batch_init_rows_kernel<<<ns, 256, 0, st>>>(a, 0);
  h->launches = 1;
  CSD_CUDA_TRY(cudaGetLastError());
  h->run_variant = h->sample_variant;
  if ((s = build_graph(h, ns, a))) return s;
  // collected results: a finished slot's region, iteration count and configurations go to its inflation
  h->job_configs.assign(n, 0);
  std::vector<char> done_job(n, 0);
  auto harvest = [&](int slot, const SlotState& S) -> csd_status_t {
    const int job = slot_job[slot];
    if (job < 0 || done_job[job]) return CSD_OK;
    if (S.status == 2) {
      set_error("Max face count exceeded in inflation " + std::to_string(job));
      return CSD_ERR_CAPACITY;
    }
    num_faces[job] = S.nf;
    if (num_iterations) num_iterations[job] = S.iters;
    h->job_configs[job] = S.configs;
    CSD_CUDA_TRY(cudaMemcpyAsync(A_out + out_off[job], h->fpool.as<float>() + S.a_off, (size_t)S.nf * S.dim * 4,
                                 cudaMemcpyDeviceToHost, st));
    CSD_CUDA_TRY(cudaMemcpyAsync(b_out + (size_t)job * cap, h->fpool.as<float>() + S.b_off, (size_t)S.nf * 4,
                                 cudaMemcpyDeviceToHost, st));
    done_job[job] = 1;
    slot_job[slot] = -1;
    return CSD_OK;
  };
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (device_ms) {
    CSD_CUDA_TRY(cudaEventCreate(&ev0));
    CSD_CUDA_TRY(cudaEventCreate(&ev1));
    CSD_CUDA_TRY(cudaEventRecord(ev0, st));
  }
  h->iter_ms.clear();
  h->iter_active.clear();
  h->iter_variant.clear();
  h->iter_faces.clear();
  h->sample_flop = 0.0;
  std::vector<SlotState> prof_slots;
  if (h->profile) prof_slots = slots;  // the records as uploaded: faces of the domain
  std::vector<int> fin;
  int active_now = ns;
  for (;;) {
    if (h->large_pending && h->tune_iters == 0) {
      // regions outgrew the tuned variant's staging for the first time: every sampler variant
      // on this iteration's inputs (the stage is idempotent), then the rest of the iteration;
      // the fastest samples the large regions from here on
      h->large_pending = false;
      std::vector<cudaEvent_t> tev(2 * kNumSampleVariants);
      for (cudaEvent_t& e : tev) CSD_CUDA_TRY(cudaEventCreate(&e));
      for (int v = 0; v < kNumSampleVariants; ++v) {
        cudaMemsetAsync(&a.it->sample_next, 0, sizeof(int), st);
        cudaEventRecord(tev[2 * v], st);
        kSampleVariants[v].fn<<<h->sample_grid[v], 256, kSampleVariants[v].smem, st>>>(a);
        cudaEventRecord(tev[2 * v + 1], st);
        ++h->launches;
      }
      h->launches += launch_iteration(h, ns, a, st, nullptr, true);
      CSD_CUDA_TRY(cudaGetLastError());
      CSD_CUDA_TRY(cudaStreamSynchronize(st));
      int best = 0;
      for (int v = 0; v < kNumSampleVariants; ++v) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, tev[2 * v], tev[2 * v + 1]);
        h->large_ms[v] = ms;
        if (ms < h->large_ms[best]) best = v;
      }
      for (cudaEvent_t& e : tev) cudaEventDestroy(e);
      h->large_tuned = true;
      h->large_variant = best;
      h->run_variant = best;
      if ((s = build_graph(h, ns, a))) return s;
      if (h->profile)
        CSD_CUDA_TRY(cudaMemcpyAsync(prof_slots.data(), h->slots_dev.ptr, ns * sizeof(SlotState),
                                     cudaMemcpyDeviceToHost, st));
    } else if (h->tune_iters > 0) {
      // every sampler variant and check item size on this iteration's inputs
      // (both stages are idempotent: a rerun writes the same samples and
      // verdicts), then the rest of the iteration as usual
      if (!h->ev[0])
        for (cudaEvent_t& e : h->ev) CSD_CUDA_TRY(cudaEventCreate(&e));
      std::vector<cudaEvent_t> tev(2 * (kNumSampleVariants + kNumCheckVariants));
      for (cudaEvent_t& e : tev) CSD_CUDA_TRY(cudaEventCreate(&e));
      int j = 0;
      for (int v = 0; v < kNumSampleVariants; ++v, ++j) {
        cudaMemsetAsync(&a.it->sample_next, 0, sizeof(int), st);
        cudaEventRecord(tev[2 * j], st);
        kSampleVariants[v].fn<<<h->sample_grid[v], 256, kSampleVariants[v].smem, st>>>(a);
        cudaEventRecord(tev[2 * j + 1], st);
        ++h->launches;
      }
      for (int c = 0; c < kNumCheckVariants && !a.mlp_wb; ++c, ++j) {
        BatchArgs ac = a;
        ac.cfg_max = kCheckItemCaps[c];
        cudaMemsetAsync(&a.it->check_next, 0, sizeof(int), st);
        cudaEventRecord(tev[2 * j], st);
        if (h->sm)
          batch_check_kernel<true><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, st>>>(ac, h->static_floats);
        else
          batch_check_kernel<false><<<h->check_grid, 32 * kWarpsPerBlock, h->check_smem, st>>>(ac, 0);
        cudaEventRecord(tev[2 * j + 1], st);
        ++h->launches;
      }
      h->launches += launch_iteration(h, ns, a, st, nullptr, true);
      CSD_CUDA_TRY(cudaGetLastError());
      CSD_CUDA_TRY(cudaStreamSynchronize(st));
      for (int q = 0; q < j; ++q) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, tev[2 * q], tev[2 * q + 1]);
        h->tune_ms[q] += ms;
      }
      for (cudaEvent_t& e : tev) cudaEventDestroy(e);
      ++h->tuned_iters;
      if (--h->tune_iters == 0) {
        int bs = 0, bc = 0;
        for (int v = 1; v < kNumSampleVariants; ++v)
          if (h->tune_ms[v] < h->tune_ms[bs]) bs = v;
        for (int c = 1; c < kNumCheckVariants; ++c)
          if (h->tune_ms[kNumSampleVariants + c] < h->tune_ms[kNumSampleVariants + bc]) bc = c;
        h->sample_variant = bs;
        h->run_variant = bs;
        // reported until a region outgrows bs's staging: the variant that would take over then
        h->large_variant = variant_for(h, kSampleVariants[bs].f8 + 1, kSampleVariants[bs].f16 + 1);
        if (!a.mlp_wb) h->cfg_max = kCheckItemCaps[bc];
        a.cfg_max = h->cfg_max;
        h->graph_slots = -1;  // recapture with the chosen shapes
        if ((s = build_graph(h, ns, a))) return s;
      }
    } else if (h->profile) {
      h->launches += launch_iteration(h, ns, a, st, h->ev);
      CSD_CUDA_TRY(cudaGetLastError());
      CSD_CUDA_TRY(cudaEventSynchronize(h->ev[kStages]));
      for (int j = 0; j < kStages; ++j) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev[j], h->ev[j + 1]);
        h->stage_ms[j] += ms;
        h->iter_ms.push_back(ms);
      }
      h->iter_active.push_back(active_now);
      h->iter_variant.push_back(h->run_variant);
      // sampler work of this iteration, from the records before it ran
      int most = 0;
      for (const SlotState& S : prof_slots)
        if (!S.done) {
          h->sample_flop += (double)h->n_tab[S.k] * h->opt.mixing_steps * (2.0 * S.dim + 4.0) * S.nf;
          most = std::max(most, S.nf);
        }
      h->iter_faces.push_back(most);
      CSD_CUDA_TRY(cudaMemcpyAsync(prof_slots.data(), h->slots_dev.ptr, ns * sizeof(SlotState),
                                   cudaMemcpyDeviceToHost, st));
    } else {
      CSD_CUDA_TRY(cudaGraphLaunch(h->graph, st));
      h->launches += h->graph_kernels;
    }
    CSD_CUDA_TRY(cudaMemcpyAsync(h->host_iter, h->iter.ptr, sizeof(BatchIter), cudaMemcpyDeviceToHost, st));
    CSD_CUDA_TRY(cudaStreamSynchronize(st));
    active_now = h->host_iter->last_active;
    // slots that finished: collect their inflations and start queued ones in them
    const int nfin = h->host_iter->num_fin;
    if (nfin > 0 && next_job < n) {
      fin.resize(nfin);
      CSD_CUDA_TRY(cudaMemcpyAsync(fin.data(), h->fin.ptr, (size_t)nfin * 4, cudaMemcpyDeviceToHost, st));
      CSD_CUDA_TRY(cudaStreamSynchronize(st));
      std::sort(fin.begin(), fin.end());
      std::vector<int> refilled;
      for (int slot : fin) {
        SlotState S{};
        CSD_CUDA_TRY(cudaMemcpyAsync(&S, h->slots_dev.as<SlotState>() + slot, sizeof(SlotState),
                                     cudaMemcpyDeviceToHost, st));
        CSD_CUDA_TRY(cudaStreamSynchronize(st));
        if ((s = harvest(slot, S))) return s;
        if (next_job >= n) continue;
        const int job = next_job++;
        slots[slot] = record(slot, job);
        slot_job[slot] = job;
        if ((s = upload(slots[slot], job))) return s;
        CSD_CUDA_TRY(cudaMemcpyAsync(h->slots_dev.as<SlotState>() + slot, &slots[slot], sizeof(SlotState),
                                     cudaMemcpyHostToDevice, st));
        batch_init_rows_kernel<<<1, 256, 0, st>>>(a, slot);
        ++h->launches;
        refilled.push_back(slot);
      }
      if (!refilled.empty()) {
        // append the refilled slots to the next iteration's active list
        const int na = h->host_iter->num_act;
        CSD_CUDA_TRY(cudaMemcpyAsync(h->act.as<int>() + na, refilled.data(), refilled.size() * 4,
                                     cudaMemcpyHostToDevice, st));
        h->host_iter->num_act = na + (int)refilled.size();
        h->host_iter->n_act = std::max(h->host_iter->n_act, h->n_tab[0]);
        CSD_CUDA_TRY(cudaMemcpyAsync(h->iter.ptr, h->host_iter, sizeof(BatchIter), cudaMemcpyHostToDevice, st));
        CSD_CUDA_TRY(cudaStreamSynchronize(st));
        active_now += (int)refilled.size();
        if (h->profile)
          for (int slot : refilled) prof_slots[slot] = slots[slot];
      }
    }
    if (active_now == 0) break;
    // surrogate mode: once no active slot checks in surrogate order, the remaining
    // iterations run the batched form's graph (no scoring, sorting or rounds; the
    // same checks as a slot checking in sample order)
    if (a.mlp_wb && h->host_iter->num_ord == 0 && next_job >= n && h->tune_iters == 0) {
      a.mlp_wb = nullptr;
      if ((s = build_graph(h, ns, a))) return s;
    }
    // a slot's region outgrew the staging buffer of the running variant: the first time, time
    // every variant on the next iteration; after that, continue with the fastest variant (by
    // those times) that stages it (identical samples; the graph is captured again)
    if (h->switch_large && h->tune_iters == 0 && !h->large_pending) {
      const SampleVariant& rv = kSampleVariants[h->run_variant];
      if (h->host_iter->max_nf8 > rv.f8 || h->host_iter->max_nf16 > rv.f16) {
        if (!h->large_tuned) {
          h->large_pending = true;
          continue;
        }
        const int v = variant_for(h, h->host_iter->max_nf8, h->host_iter->max_nf16);
        if (v != h->run_variant) {
          h->run_variant = v;
          h->large_variant = v;
          if ((s = build_graph(h, ns, a))) return s;
        }
      }
    }
  }
  if (device_ms) {
    CSD_CUDA_TRY(cudaEventRecord(ev1, st));
    CSD_CUDA_TRY(cudaEventSynchronize(ev1));
    cudaEventElapsedTime(device_ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
  }
  CSD_CUDA_TRY(cudaMemcpyAsync(slots.data(), h->slots_dev.ptr, ns * sizeof(SlotState), cudaMemcpyDeviceToHost, st));
  int kstat = 0;
  CSD_CUDA_TRY(cudaMemcpyAsync(&kstat, h->status.ptr, 4, cudaMemcpyDeviceToHost, st));
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  if (kstat) {
    set_error("a tensor-core barrier wait timed out in the scoring stage");
    return CSD_ERR_CUDA;
  }
  for (csd_plant_t pl : h->plants)
    if ((s = plant_status(pl, st))) return s;
  for (int i = 0; i < ns; ++i)
    if ((s = harvest(i, slots[i]))) return s;
  CSD_CUDA_TRY(cudaStreamSynchronize(st));
  for (int j = 0; j < n; ++j)
    if (!done_job[j]) {
      set_error("inflation " + std::to_string(j) + " was not completed");
      return CSD_ERR_CUDA;
    }
  return CSD_OK;
}

csd_status_t csd_batch_set_profiling(csd_batch_t h, int32_t enable) {
  CSD_CHECK(h, CSD_ERR_INVALID, "null batch");
  if (enable && !h->ev[0]) {
    for (cudaEvent_t& e : h->ev) CSD_CUDA_TRY(cudaEventCreate(&e));
  }
  h->profile = enable != 0;
  for (double& x : h->stage_ms) x = 0.0;
  return CSD_OK;
}

csd_status_t csd_batch_stage_ms(csd_batch_t h, float* ms) {
  CSD_CHECK(h && ms, CSD_ERR_INVALID, "null argument");
  for (int j = 0; j < kStages; ++j) ms[j] = (float)h->stage_ms[j];
  return CSD_OK;
}

csd_status_t csd_batch_autotune(csd_batch_t h, int32_t iterations) {
  CSD_CHECK(h && iterations >= 0, CSD_ERR_INVALID, "bad autotune arguments");
  h->tune_iters = iterations;
  h->tuned_iters = 0;
  for (double& x : h->tune_ms) x = 0.0;
  h->large_tuned = false;
  h->large_pending = false;
  for (double& x : h->large_ms) x = 0.0;
  return CSD_OK;
}

csd_status_t csd_batch_set_surrogate(csd_batch_t h, csd_mlp_t mlp, float stop_probability) {
  CSD_CHECK(h, CSD_ERR_INVALID, "null batch");
  if (!mlp) {
    h->mlp = nullptr;
    return CSD_OK;
  }
  CSD_CHECK(stop_probability > 0.f && stop_probability < 1.f, CSD_ERR_INVALID, "stop probability must be in (0, 1)");
  const MlpView mv = mlp_view(mlp);
  CSD_CHECK(mv.device == h->device, CSD_ERR_INVALID, "surrogate and batch must live on one device");
  CSD_CHECK(mv.nets == (int)h->plants.size(), CSD_ERR_INVALID, "the surrogate needs one net per plant of the batch");
  for (int i = 0; i < mv.nets; ++i)
    CSD_CHECK(mv.dims[i] == h->plants[i]->dp.dim, CSD_ERR_DIMENSION, "net " + std::to_string(i) +
                                                                         " does not match its plant's dimension");
  CSD_CHECK(h->n_max <= kSortMax, CSD_ERR_CAPACITY, "more samples per iteration than the surrogate sort handles");
  int cur = 0;
  cudaGetDevice(&cur);
  if (cur != h->device) cudaSetDevice(h->device);
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, h->device};
  csd_status_t s;
  if ((s = h->scores.reserve((size_t)h->max_slots * h->n_max * 4)) ||
      (s = h->order.reserve((size_t)h->max_slots * h->n_max * 4)))
    return s;
  CSD_CUDA_TRY(raise_smem_limit(batch_score_kernel, (int)mlp::kFwdSmem));
  CSD_CUDA_TRY(raise_smem_limit(batch_sort_kernel, (int)(kSortMax * sizeof(unsigned long long))));
  h->mlp = mlp;
  h->stop_logit = std::log(stop_probability / (1.f - stop_probability));
  return CSD_OK;
}

csd_status_t csd_batch_set_surrogate_rounds(csd_batch_t h, int32_t rounds, int32_t first_round) {
  CSD_CHECK(h && rounds >= 1 && rounds <= 8 && first_round >= 32, CSD_ERR_INVALID,
            "rounds must be in [1, 8] and the first round at least 32 samples");
  h->rounds = rounds;
  h->round_base = first_round;
  h->graph_slots = -1;
  return CSD_OK;
}

csd_status_t csd_batch_set_shapes(csd_batch_t h, int32_t sample_variant, int32_t check_item_cap) {
  CSD_CHECK(h && sample_variant >= 0 && sample_variant < kNumSampleVariants && check_item_cap >= 8 &&
                check_item_cap % 8 == 0,
            CSD_ERR_INVALID, "bad shapes: sampler variant out of range, or check item cap not a positive multiple of 8");
  h->sample_variant = sample_variant;
  h->run_variant = sample_variant;
  h->switch_large = false;
  h->cfg_max = check_item_cap;
  return CSD_OK;
}

csd_status_t csd_batch_sample_variants(csd_batch_t h, int32_t* tuned, int32_t* large, int32_t* last_run) {
  CSD_CHECK(h, CSD_ERR_INVALID, "null batch");
  if (tuned) *tuned = h->sample_variant;
  if (large) *large = h->switch_large ? h->large_variant : h->sample_variant;
  if (last_run) *last_run = h->run_variant;
  return CSD_OK;
}

void csd_batch_shape_counts(int32_t* num_sample_variants, int32_t* num_check_caps) {
  if (num_sample_variants) *num_sample_variants = kNumSampleVariants;
  if (num_check_caps) *num_check_caps = kNumCheckVariants;
}

csd_status_t csd_batch_tuning(csd_batch_t h, int32_t* sample_variant, int32_t* check_item_cap, float* variant_ms,
                              int32_t* num_variants) {
  CSD_CHECK(h, CSD_ERR_INVALID, "null batch");
  if (sample_variant) *sample_variant = h->sample_variant;
  if (check_item_cap) *check_item_cap = h->cfg_max;
  if (num_variants) *num_variants = kNumSampleVariants + kNumCheckVariants;
  if (variant_ms)
    for (int q = 0; q < kNumSampleVariants + kNumCheckVariants; ++q) variant_ms[q] = (float)h->tune_ms[q];
  return CSD_OK;
}

csd_status_t csd_batch_last_launches(csd_batch_t h, int64_t* launches) {
  CSD_CHECK(h && launches, CSD_ERR_INVALID, "null argument");
  *launches = h->launches;
  return CSD_OK;
}

csd_status_t csd_batch_sample_flops(csd_batch_t h, double* flops) {
  CSD_CHECK(h && flops, CSD_ERR_INVALID, "null argument");
  *flops = h->sample_flop;
  return CSD_OK;
}

csd_status_t csd_batch_iteration_profile(csd_batch_t h, int32_t cap, float* stage_ms, int32_t* active,
                                         int32_t* count) {
  CSD_CHECK(h && count && (cap == 0 || (stage_ms && active)), CSD_ERR_INVALID, "null argument");
  const int n = (int)h->iter_active.size();
  *count = n;
  for (int i = 0; i < std::min(n, (int)cap); ++i) {
    active[i] = h->iter_active[i];
    for (int j = 0; j < kStages; ++j) stage_ms[i * kStages + j] = h->iter_ms[(size_t)i * kStages + j];
  }
  return CSD_OK;
}

csd_status_t csd_batch_iteration_variants(csd_batch_t h, int32_t cap, int32_t* variant, int32_t* max_faces,
                                          int32_t* count) {
  CSD_CHECK(h && count && (cap == 0 || (variant && max_faces)), CSD_ERR_INVALID, "null argument");
  const int n = (int)h->iter_variant.size();
  *count = n;
  for (int i = 0; i < std::min(n, (int)cap); ++i) {
    variant[i] = h->iter_variant[i];
    max_faces[i] = h->iter_faces[i];
  }
  return CSD_OK;
}

csd_status_t csd_batch_configs_checked(csd_batch_t h, int32_t n, int64_t* configs) {
  CSD_CHECK(h && configs && n >= 0 && n <= (int)h->job_configs.size(), CSD_ERR_INVALID,
            "count exceeds the inflations of the last call");
  for (int i = 0; i < n; ++i) configs[i] = h->job_configs[i];
  return CSD_OK;
}

}  // extern "C"
