// g1_mlp.cuh -- tcgen05 tile MLP for sm_100a: 128 rows (envs) per CTA, BF16
// operands in shared memory, FP32 accumulators in tensor memory.
//
// One CTA evaluates a chain of dense layers y = act(x W^T + b) for the 128
// rows of its tile.  The activation tile (the A operand) is written by the
// CTA's threads into shared memory; the weights stream from global memory
// (L2-resident, shared by every CTA) through a ring of kStages shared-memory
// stages with cp.async.bulk + mbarrier transaction counts; one elected
// thread issues tcgen05.mma (M = 128, N <= 256 per instruction, K = 16) into
// a tensor-memory accumulator; every warp of the CTA then reads its lane
// quarter of the accumulator with tcgen05.ld, adds the bias, applies the
// activation and writes the next layer's A tile as BF16.
//
// Shared-memory operand layout (UMMA "no swizzle", K-major): 8x8 BF16 core
// matrices of 128 contiguous bytes, stored [K/8][rows/8][8][8].  For a tile
// of R rows the leading byte offset (next core matrix along K) is R*16 and
// the stride byte offset (next 8-row group) is 128.  Weights are packed on
// the host in the same layout per K-chunk (g1sim_b200/policy.py), so one
// chunk is one contiguous bulk copy.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

namespace g1b::tc {

constexpr int kRows = 128;          // rows of every MMA / TMEM lanes used
constexpr int kStageBytes = 16384;  // one weight chunk
constexpr int kStages = 3;          // weight ring depth
constexpr int kTmemCols = 512;      // whole tensor memory of the SM (one CTA per SM)

enum Act : int { kNone = 0, kElu = 1, kSilu = 2 };

struct Layer {
  int K, N, KC, act;  // padded K, padded N, K columns per streamed chunk, activation
};

// --------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for the phase of `parity` to complete, for at most ~kWaitNs.  Returns
// false (and the caller raises the CTA's abort flag) if it gave up.
constexpr uint64_t kWaitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  while (!mbar_try(bar, parity))
    if (globaltimer() - t0 > kWaitNs) return false;
  return true;
}
// Bulk global -> shared copy completing on an mbarrier (no multicast).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor-memory allocation: executed by one whole warp.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// Arrive on `bar` once every tcgen05.mma issued so far by this thread is complete.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape);
// the wait is part of the same statement so no use can move above it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------- tile layout
// Byte offset of element (row, k) in a [K/8][R/8][8][8] BF16 tile.
template <int R = kRows>
__host__ __device__ constexpr uint32_t tile_off(int row, int k) {
  return (uint32_t)(((k >> 3) * (R >> 3) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
// Store 8 consecutive K values of one row (16 bytes) of a BF16 tile.
__device__ __forceinline__ void st_row8(uint8_t* tile, int row, int k8, const float* v) {
  uint4 w;
  w.x = pack_bf16x2(v[0], v[1]);
  w.y = pack_bf16x2(v[2], v[3]);
  w.z = pack_bf16x2(v[4], v[5]);
  w.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + tile_off(row, k8)) = w;
}

__device__ __forceinline__ float activate(float x, int act) {
  if (act == kElu) return x > 0.0f ? x : expm1f(x);
  if (act == kSilu) return x / (1.0f + expf(-x));
  return x;
}

// ------------------------------------------------------ network chain
// Net supplies `static constexpr int kL` and `static constexpr Layer layer[kL]`;
// consecutive layers of one network have K(l + 1) = N(l), and a pass may
// hold several networks back to back (their weights stream as one sequence).
template <class Net>
struct Chain {
  static constexpr int kL = Net::kL;
  static consteval int chunks(int l) { return Net::layer[l].K / Net::layer[l].KC; }
  static consteval uint32_t chunk_bytes(int l) { return (uint32_t)(Net::layer[l].N * Net::layer[l].KC * 2); }
  static consteval int first_chunk(int l) {
    int c = 0;
    for (int i = 0; i < l; ++i) c += chunks(i);
    return c;
  }
  static constexpr int kChunks = first_chunk(kL);
  static consteval uint32_t weight_off(int l) {
    uint32_t b = 0;
    for (int i = 0; i < l; ++i) b += chunk_bytes(i) * chunks(i);
    return b;
  }
  static constexpr uint32_t kWeightBytes = weight_off(kL);
  static consteval int bias_off(int l) {
    int b = 0;
    for (int i = 0; i < l; ++i) b += Net::layer[i].N;
    return b;
  }
  static constexpr int kBiasFloats = bias_off(kL);
  static consteval int layer_of_chunk(int c) {
    int l = 0;
    while (l + 1 < kL && c >= first_chunk(l + 1)) ++l;
    return l;
  }
  static consteval int max_k() {
    int m = 0;
    for (int i = 0; i < kL; ++i) m = Net::layer[i].K > m ? Net::layer[i].K : m;
    for (int i = 0; i < kL; ++i) m = Net::layer[i].N > m ? Net::layer[i].N : m;
    return m;
  }
  static constexpr uint32_t kActBytes = (uint32_t)(kRows * max_k() * 2);

  static consteval bool valid() {
    for (int i = 0; i < kL; ++i) {
      const Layer& L = Net::layer[i];
      if (L.K % 16 || L.KC % 16 || L.K % L.KC || L.N % 16 || L.N < 16 || L.N > kTmemCols) return false;
      if (L.N > 256 && L.N % 256) return false;
      if (L.N * L.KC * 2 > kStageBytes) return false;
    }
    return true;
  }
};

// Per-CTA pipeline state.  Every thread holds a copy; the chunk counters
// advance only in the issuing thread (thread 0), the accumulator phase in
// all threads (each waits on every layer's completion).
struct Pipe {
  uint32_t act;      // shared address of the A tile
  uint32_t stage;    // shared address of stage 0
  uint32_t bar;      // shared address of the barriers: full[kStages], empty[kStages], acc
  uint32_t tmem;     // tensor-memory base address
  uint32_t loaded;   // chunks whose copy was issued (thread 0)
  uint32_t issued;   // chunks whose MMAs were issued (thread 0)
  uint32_t base;     // global index of chunk 0 of the current pass (thread 0)
  uint32_t acc_n;    // accumulator completions waited for (all threads)
  __device__ uint32_t full(int s) const { return bar + 8u * s; }
  __device__ uint32_t empty(int s) const { return bar + 8u * (kStages + s); }
  __device__ uint32_t accb() const { return bar + 8u * (2 * kStages); }
};
constexpr int kBarriers = 2 * kStages + 1;

// Barrier initialisation (one thread), before the CTA's first barrier sync.
__device__ __forceinline__ void pipe_init(const Pipe& p) {
  for (int s = 0; s < kStages; ++s) {
    mbar_init(p.full(s), 1);
    mbar_init(p.empty(s), 1);
  }
  mbar_init(p.accb(), 1);
  mbar_fence_init();
}

template <class Net>
struct Runner {
  using C = Chain<Net>;
  static_assert(C::valid(), "layer shapes must fit the UMMA / staging constraints");

  // Offset and size of pass chunk c, from compile-time layer data.
  template <int L = 0>
  static __device__ __forceinline__ void chunk_info(int c, uint32_t& off, uint32_t& bytes) {
    if constexpr (L < C::kL) {
      constexpr int f = C::first_chunk(L), nc = C::chunks(L);
      constexpr uint32_t b = C::chunk_bytes(L), wo = C::weight_off(L);
      if (c < f + nc || L + 1 == C::kL) {
        off = wo + (uint32_t)(c - f) * b;
        bytes = b;
        return;
      }
      chunk_info<L + 1>(c, off, bytes);
    }
  }
  // Issue the copy of pass chunk c (thread 0).  Returns false on a timeout.
  static __device__ bool load(Pipe& p, const uint8_t* blob, int c) {
    const uint32_t g = p.loaded;
    const int s = (int)(g % kStages);
    if (g >= (uint32_t)kStages && !mbar_wait(p.empty(s), ((g / kStages) - 1) & 1)) return false;
    uint32_t off = 0, bytes = 0;
    chunk_info(c, off, bytes);
    mbar_expect_tx(p.full(s), bytes);
    bulk_g2s(p.stage + (uint32_t)s * kStageBytes, blob + off, bytes, p.full(s));
    ++p.loaded;
    return true;
  }
  // Start a pass over the whole chain: prefetch the first kStages chunks.
  static __device__ bool begin(Pipe& p, const uint8_t* blob) {
    if (threadIdx.x != 0) return true;
    p.base = p.loaded;
    for (int c = 0; c < kStages && c < C::kChunks; ++c)
      if (!load(p, blob, c)) return false;
    return true;
  }
  // Issue the MMAs of layer L (thread 0); its accumulator occupies TMEM
  // columns [0, N).  The A tile must be complete and fenced.
  template <int L>
  static __device__ bool issue(Pipe& p, const uint8_t* blob) {
    if (threadIdx.x != 0) return true;
    constexpr Layer Ly = Net::layer[L];
    constexpr uint32_t lbo_a = kRows * 16, lbo_b = (uint32_t)Ly.N * 16;
    constexpr int nmma = Ly.N > 256 ? Ly.N / 256 : 1;
    constexpr uint32_t id = idesc_bf16(kRows, Ly.N > 256 ? 256 : Ly.N);
    constexpr int ksteps = Ly.KC / 16;
    tc_fence_after();
    for (int c = 0; c < C::chunks(L); ++c) {
      const uint32_t g = p.issued;
      const int s = (int)(g % kStages);
      if (!mbar_wait(p.full(s), (g / kStages) & 1)) return false;
      const uint32_t bstage = p.stage + (uint32_t)s * kStageBytes;
#pragma unroll
      for (int j = 0; j < ksteps; ++j) {
        const int kk = c * ksteps + j;  // K step of 16 within the layer
        const uint64_t ad = sdesc(p.act + (uint32_t)kk * 2 * lbo_a, lbo_a, 128);
#pragma unroll
        for (int h = 0; h < nmma; ++h) {
          const uint64_t bd = sdesc(bstage + (uint32_t)j * 2 * lbo_b + (uint32_t)h * 32 * 128, lbo_b, 128);
          mma_bf16(p.tmem + (uint32_t)(h * 256), ad, bd, id, kk > 0 ? 1u : 0u);
        }
      }
      mma_commit(p.empty(s));
      ++p.issued;
      // keep kStages - 1 chunks in flight behind the one just issued
      while (p.loaded < p.issued + (uint32_t)kStages - 1 && (int)(p.loaded - p.base) < C::kChunks)
        if (!load(p, blob, (int)(p.loaded - p.base))) return false;
    }
    mma_commit(p.accb());
    return true;
  }
  // Every thread: wait for layer completion, then make TMEM reads safe.
  static __device__ bool wait_acc(Pipe& p) {
    const bool ok = mbar_wait(p.accb(), p.acc_n & 1);
    ++p.acc_n;
    tc_fence_after();
    return ok;
  }
  // Every thread: bias + activation of layer l's accumulator into the A tile
  // of layer l+1.  Warp w reads TMEM lanes 32*(w%4).. and the column half w/4
  // (kThreads = 256) or all columns (kThreads = 128).
  template <int L, int kThreads>
  static __device__ void epilogue(const Pipe& p, uint8_t* act_tile, const float* bias) {
    constexpr Layer Ly = Net::layer[L];
    const int warp = threadIdx.x >> 5, q = warp & 3;
    const int row = q * 32 + (threadIdx.x & 31);
    constexpr int kHalves = kThreads / 128;
    constexpr int span = Ly.N / kHalves;
    static_assert(span % 16 == 0, "epilogue columns come in groups of 16");
    const int c0 = (warp >> 2) * span;
    const uint32_t lane_base = p.tmem + ((uint32_t)(q * 32) << 16);
    for (int c = c0; c < c0 + span; c += 16) {
      float v[16];
      tmem_ld16(lane_base + (uint32_t)c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = activate(v[i] + __ldg(bias + c + i), Ly.act);
      st_row8(act_tile, row, c, v);
      st_row8(act_tile, row, c + 8, v + 8);
    }
  }
};

// Every thread: publish generic shared stores of the A tile to the tensor
// core and order this thread's TMEM reads before the next MMA; follow with
// a CTA barrier.
__device__ __forceinline__ void tile_written() {
  fence_async_smem();
  tc_fence_before();
}

}  // namespace g1b::tc
