// g1_gemm.cuh -- BF16 tcgen05 GEMM for the dynamics-surrogate training
// (included by g1_kernels.cu inside namespace g1b, after g1_mlp.cuh).
//
//   C[M x N] (= or +=) A[M x K] . B[N x K]^T (+ bias[N])
// A and B are BF16, row-major with K contiguous (leading dimensions lda,
// ldb in elements); C is FP32 row-major (ldc).  One CTA (128 threads) owns
// a 128 MT x Nt tile of C (MT = 1 or 2 row tiles, Nt = min(N, 256), an MMA's N) and a K range of its
// split: 64-wide K chunks are copied global -> shared with 16-byte cp.async
// into the UMMA 128-byte-swizzle K-major layout (kGemmStages-deep ring), thread 0 issues
// tcgen05.mma (M 128, K 16) into a tensor-memory accumulator, and the four
// warps read their 32 lanes back for the epilogue.  With several K splits
// the partial tiles are added into C with atomics (C zeroed by the caller).
//
// Constraints (checked by the host launcher): M % 128 == 0, N % 16 == 0,
// N % Nt == 0, K % (64 * splits) == 0, lda / ldb multiples of 8.

constexpr int kGemmKC = 64;  // K columns per chunk
constexpr int kGemmMaxN = 256;
constexpr uint32_t kGemmABytes = 128 * kGemmKC * 2;        // 16 KB
constexpr uint32_t kGemmBBytes = kGemmMaxN * kGemmKC * 2;  // 32 KB
// MT row tiles of 128 per CTA share each B chunk (MT = 2 halves the weight
// traffic per row, the bound of this kernel); the ring holds 192 KB.
template <int MT>
__host__ __device__ constexpr uint32_t gemm_stage_bytes() { return MT * kGemmABytes + kGemmBBytes; }
template <int MT>
__host__ __device__ constexpr int gemm_stages() { return MT == 2 ? 3 : 4; }
template <int MT>
__host__ __device__ constexpr size_t gemm_smem() {
  return gemm_stages<MT>() * (size_t)gemm_stage_bytes<MT>() + 1024;  // + alignment slack
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy K chunk [k0, k0 + 64) of rows [r0, r0 + rows) of a row-major BF16
// matrix into shared memory at dst (1024-byte aligned) in the UMMA K-major
// 128-byte-swizzle layout: each row's 64 values are one 128-byte line, eight
// lines form a 1024-byte atom, and the 16-byte piece j of row r sits at piece
// position j ^ (r % 8) of its line (bank-conflict-free for the tensor core).
__device__ __forceinline__ void gemm_load_tile(uint32_t dst, const __nv_bfloat16* X, int ld, int r0, int rows,
                                               int k0) {
  const int pieces = rows * (kGemmKC / 8);
  for (int p = threadIdx.x; p < pieces; p += 128) {
    const int r = p >> 3, j = p & 7;
    const __nv_bfloat16* src = X + (size_t)(r0 + r) * ld + k0 + j * 8;
    const uint32_t off = (uint32_t)(r >> 3) * 1024u + (uint32_t)(r & 7) * 128u + (uint32_t)((j ^ (r & 7)) * 16);
    cp_async16(dst + off, src);
  }
}
// Shared-memory descriptor of such a tile, K step kk (16 values = 32 bytes
// along the line): swizzle mode 128B (2), stride between 8-row atoms 1024 B.
__device__ __forceinline__ uint64_t gemm_desc_sw128(uint32_t tile, int kk) {
  const uint32_t a = tile + (uint32_t)kk * 32u;
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

template <bool kAtomic, int MT>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                        const __nv_bfloat16* __restrict__ B, int ldb, float* C,
                                                        int ldc, const float* __restrict__ bias, int Nt, int Ks,
                                                        int* err) {
  constexpr int kGemmStages = gemm_stages<MT>();
  constexpr uint32_t kGemmStage = gemm_stage_bytes<MT>();
  constexpr uint32_t kBOff = MT * kGemmABytes;
  constexpr uint32_t kCols = 256 * MT;
  extern __shared__ __align__(1024) uint8_t gsm[];
  __shared__ uint64_t bars[kGemmStages + 1];  // mma done per stage, accumulator
  __shared__ uint32_t tslot;
  const int m0 = blockIdx.x * 128 * MT, n0 = blockIdx.y * Nt, kbeg = blockIdx.z * Ks;
  const int nchunks = Ks / kGemmKC;
  const uint32_t sbase = (tc::smem_u32(gsm) + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
  const uint32_t bacc = tc::smem_u32(&bars[kGemmStages]);
  if (threadIdx.x == 0) {
    for (int i = 0; i <= kGemmStages; ++i) tc::mbar_init(tc::smem_u32(&bars[i]), 1);
    tc::mbar_fence_init();
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tslot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t idesc = tc::idesc_bf16(128, Nt);
  bool ok = true;

  // prologue: chunks 0 .. kGemmStages - 2 (one commit group each, empty groups past the end)
  for (int i = 0; i < kGemmStages - 1; ++i) {
    if (i < nchunks) {
      const uint32_t st = sbase + (uint32_t)i * kGemmStage;
      gemm_load_tile(st, A, lda, m0, 128 * MT, kbeg + i * kGemmKC);
      gemm_load_tile(st + kBOff, B, ldb, n0, Nt, kbeg + i * kGemmKC);
    }
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    const int s = c % kGemmStages;
    cp_async_wait<kGemmStages - 2>();  // this thread's copies of chunk c have landed
    tc::fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::tc_fence_after();
      const uint32_t st = sbase + (uint32_t)s * kGemmStage;
#pragma unroll
      for (int j = 0; j < kGemmKC / 16; ++j)
#pragma unroll
        for (int t = 0; t < MT; ++t)
          tc::mma_bf16(tmem + (uint32_t)(t * 256), gemm_desc_sw128(st + (uint32_t)t * kGemmABytes, j),
                       gemm_desc_sw128(st + kBOff, j), idesc, (c > 0 || j > 0) ? 1u : 0u);
      tc::mma_commit(tc::smem_u32(&bars[s]));
      if (c + 1 == nchunks) tc::mma_commit(bacc);
    }
    // refill the stage read by chunk c - 1 with chunk c + kGemmStages - 1
    const int nx = c + kGemmStages - 1;
    if (nx < nchunks) {
      const int sp = nx % kGemmStages;
      if (c >= 1 && !tc::mbar_wait(tc::smem_u32(&bars[sp]), ((c - 1) / kGemmStages) & 1)) ok = false;
      const uint32_t st = sbase + (uint32_t)sp * kGemmStage;
      gemm_load_tile(st, A, lda, m0, 128 * MT, kbeg + nx * kGemmKC);
      gemm_load_tile(st + kBOff, B, ldb, n0, Nt, kbeg + nx * kGemmKC);
    }
    cp_async_commit();
  }
  if (!tc::mbar_wait(bacc, 0)) ok = false;
  tc::tc_fence_after();
  // epilogue: warp w holds rows 32 w .. 32 w + 31 of each 128-row subtile
  for (int t = 0; t < MT; ++t) {
    const int row = m0 + t * 128 + (int)threadIdx.x;
    const uint32_t lane_base = tmem + (uint32_t)(t * 256) + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
    float* crow = C + (size_t)row * ldc + n0;
    for (int c = 0; c < Nt; c += 32) {
      float v[32];
      tc::tmem_ld32(lane_base + (uint32_t)c, v);
      if (bias && blockIdx.z == 0) {
        const int nb = Nt - c < 32 ? Nt - c : 32;  // the bias holds exactly N floats
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (i < nb) v[i] += __ldg(bias + n0 + c + i);
      }
      if (c + 32 > Nt) {  // Nt = 16 or 48 ...: partial last group
        for (int i = 0; i < Nt - c; ++i) {
          if (kAtomic)
            atomicAdd(crow + c + i, v[i]);
          else
            crow[c + i] = v[i];
        }
      } else if (kAtomic) {
#pragma unroll
        for (int i = 0; i < 32; ++i) atomicAdd(crow + c + i, v[i]);
      } else {
#pragma unroll
        for (int i = 0; i < 32; i += 4)
          *reinterpret_cast<float4*>(crow + c + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
    }
  }
  if (!ok) atomicExch(err, 1);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}
