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
constexpr int kStages = 4;          // weight ring depth = loader threads
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
// The thread sleeps until the phase completes or kTrySuspendNs pass, so that a
// waiting warp takes no issue slots from the warps that compute (the callers'
// loops still give up after kWaitNs).
constexpr uint32_t kTrySuspendNs = 1000000u;
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(kTrySuspendNs)
      : "memory");
  return ok != 0;
}
// Non-blocking test of the same condition.
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
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
// Bulk global -> shared copy into this CTA only, completing on an mbarrier.
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

// 32 consecutive FP32 columns of this thread's TMEM lane, one wait.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
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

// Hidden activations.  The result is rounded to BF16 (8 significant bits)
// for the next layer, so the hardware exponential (ex2.approx, relative
// error ~2^-22) is far inside that rounding.
__device__ __forceinline__ float activate(float x, int act) {
  if (act == kElu) return x > 0.0f ? x : __expf(x) - 1.0f;
  if (act == kSilu) return __fdividef(x, 1.0f + __expf(-x));
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

// Per-CTA pipeline state.  Every thread holds a copy.  Weight copies are
// issued by kStages loader threads (lane 0 of warps 0..kStages-1), loader j
// owning ring stage j and therefore the chunks g = j (mod kStages) of the
// global chunk sequence.  Bulk copies issued by one thread complete one after
// another (about 0.3 us each on B200 whatever their size up to 64 KB, measured),
// while copies of different threads overlap; four issuers keep the stream
// near the L2 -> SM rate.  Thread 0 (loader 0) also issues the MMAs.
// Loaders issue their next copy whenever they wait anyway (for a chunk to
// land or for a layer to finish) and its stage has been released by the MMAs
// of the chunk kStages earlier.
struct Pipe {
  uint32_t act;      // shared address of the A tile
  uint32_t stage;    // shared address of stage 0
  uint32_t bar;      // shared address of the barriers: full[kStages], empty[kStages], acc
  uint32_t tmem;     // tensor-memory base address
  uint32_t loaded;   // loader: global index of the next chunk it copies
  uint32_t issued;   // thread 0: chunks whose MMAs were issued
  uint32_t base;     // global index of chunk 0 of the current pass
  uint32_t passes;   // passes begun
  uint32_t acc_n;    // accumulator completions waited for (all threads)
  __device__ uint32_t full(int s) const { return bar + 8u * s; }
  __device__ uint32_t empty(int s) const { return bar + 8u * (kStages + s); }
  __device__ uint32_t accb() const { return bar + 8u * (2 * kStages); }
};
constexpr int kBarriers = 2 * kStages + 1;

// Loader index of this thread (lane 0 of warps 0..kStages-1), or -1.
__device__ __forceinline__ int loader_id() {
  return ((threadIdx.x & 31) == 0 && (threadIdx.x >> 5) < kStages) ? (int)(threadIdx.x >> 5) : -1;
}

// Every thread, before its first use of the pipe; thread 0 also initialises
// the barriers (before the CTA's first barrier sync).
__device__ __forceinline__ void pipe_init(Pipe& p) {
  const int j = loader_id();
  p.loaded = j >= 0 ? (uint32_t)j : 0u;
  p.issued = p.base = p.passes = p.acc_n = 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(p.full(s), 1);
      mbar_init(p.empty(s), 1);
    }
    mbar_init(p.accb(), 1);
    mbar_fence_init();
  }
}

template <class Net>
struct Runner {
  using C = Chain<Net>;
  static_assert(C::valid(), "layer shapes must fit the UMMA / staging constraints");
  static_assert(C::kChunks % kStages == 0, "loader j owns the chunks j (mod kStages) of every pass");

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
  // Loader threads: issue this loader's next copy of the pass if its stage
  // has been released (non-blocking).
  static __device__ __forceinline__ void service(Pipe& p, const uint8_t* blob) {
    const int j = loader_id();
    if (j < 0) return;
    const uint32_t g = p.loaded;
    const int c = (int)(g - p.base);
    if (c >= C::kChunks) return;
    if (g >= (uint32_t)kStages && !mbar_test(p.empty(j), ((g / kStages) - 1) & 1)) return;
    uint32_t off = 0, bytes = 0;
    chunk_info(c, off, bytes);
    mbar_expect_tx(p.full(j), bytes);
    bulk_g2s(p.stage + (uint32_t)j * kStageBytes, blob + off, bytes, p.full(j));
    p.loaded += kStages;
  }
  // Every thread: start a pass over the whole chain (loaders copy their
  // first chunk; every stage is free between passes).
  static __device__ bool begin(Pipe& p, const uint8_t* blob) {
    p.base = p.passes * (uint32_t)C::kChunks;
    ++p.passes;
    service(p, blob);
    return true;
  }
  // Thread 0: wait until chunk g has landed, serving its own loads meanwhile.
  static __device__ bool wait_chunk(Pipe& p, const uint8_t* blob, uint32_t g) {
    const int s = (int)(g % kStages);
    const uint32_t par = (g / kStages) & 1;
    if (mbar_test(p.full(s), par)) return true;
    const uint64_t t0 = globaltimer();
    for (;;) {
      service(p, blob);
      if (mbar_test(p.full(s), par)) return true;
      if (globaltimer() - t0 > kWaitNs) return false;
    }
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
      if (!wait_chunk(p, blob, g)) return false;
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
      service(p, blob);
    }
    mma_commit(p.accb());
    return true;
  }
  // Every thread: wait for the layer's accumulator (loaders keep copying
  // meanwhile, and once more when it completes since the layer's MMAs have
  // then released every stage), then make TMEM reads safe.
  static __device__ bool wait_acc(Pipe& p, const uint8_t* blob) {
    const uint32_t par = p.acc_n & 1;
    ++p.acc_n;
    bool ok = true;
    if (!mbar_test(p.accb(), par)) {
      const uint64_t t0 = globaltimer();
      for (;;) {
        service(p, blob);
        if (mbar_test(p.accb(), par)) break;
        if (globaltimer() - t0 > kWaitNs) {
          ok = false;
          break;
        }
      }
    }
    service(p, blob);
    tc_fence_after();
    return ok;
  }
  // After an abort: loaders wait (bounded) for their last copy, thread 0 for
  // its last MMAs, so nothing writes the CTA's memory once it has left.
  static __device__ void drain(const Pipe& p) {
    const int j = loader_id();
    if (j >= 0 && p.loaded >= (uint32_t)kStages) {
      const uint32_t g = p.loaded - kStages;
      mbar_wait(p.full(j), (g / kStages) & 1);
    }
    if (threadIdx.x == 0 && p.issued > 0) {
      const uint32_t g = p.issued - 1;
      mbar_wait(p.empty((int)(g % kStages)), (g / kStages) & 1);
    }
  }
  // bias + activation of 32 accumulator columns, stored as BF16 at (row, c..c+31)
  template <int kAct>
  static __device__ __forceinline__ void finish32(const float (&r)[32], const float* bias, uint8_t* act_tile,
                                                  int row, int c) {
    float v[32];
    const float4* b4 = reinterpret_cast<const float4*>(bias);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float4 b = __ldg(b4 + i);
      v[4 * i + 0] = activate(r[4 * i + 0] + b.x, kAct);
      v[4 * i + 1] = activate(r[4 * i + 1] + b.y, kAct);
      v[4 * i + 2] = activate(r[4 * i + 2] + b.z, kAct);
      v[4 * i + 3] = activate(r[4 * i + 3] + b.w, kAct);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) st_row8(act_tile, row, c + 8 * i, v + 8 * i);
  }
  // Every thread: bias + activation of layer L's accumulator into the A tile
  // of layer L+1.  Warp w reads TMEM lanes 32*(w%4).. and the column half w/4
  // (kThreads = 256) or all columns (kThreads = 128).  bias: 16-byte aligned.
  template <int L, int kThreads>
  static __device__ void epilogue(const Pipe& p, uint8_t* act_tile, const float* bias) {
    constexpr Layer Ly = Net::layer[L];
    const int warp = threadIdx.x >> 5, q = warp & 3;
    const int row = q * 32 + (threadIdx.x & 31);
    constexpr int kHalves = kThreads / 128;
    constexpr int span = Ly.N / kHalves;
    static_assert(span % 32 == 0, "epilogue columns come in groups of 32");
    const int c0 = (warp >> 2) * span;
    const uint32_t lane_base = p.tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
    for (int c = c0; c < c0 + span; c += 32) {
      float v[32];
      tmem_ld32(lane_base + (uint32_t)c, v);
      finish32<Ly.act>(v, bias + c, act_tile, row, c);
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
