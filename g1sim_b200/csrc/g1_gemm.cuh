// g1_gemm.cuh -- BF16 tcgen05 GEMM for the dynamics-surrogate training
// (included by g1_kernels.cu inside namespace g1b, after g1_mlp.cuh).
//
//   C[M x N] (= or +=) A[M x K] . B[N x K]^T (+ bias[N])
// A and B are BF16, row-major with K contiguous (leading dimensions lda,
// ldb in elements); C is FP32 row-major (ldc).  One CTA (128 threads) owns
// a 128 x Nt tile of C (Nt = min(N, 256), an MMA's N) and a K range of its
// split: 64-wide K chunks are copied global -> shared with 16-byte cp.async
// into the UMMA no-swizzle K-major layout (two stages), thread 0 issues
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
constexpr uint32_t kGemmStage = kGemmABytes + kGemmBBytes;
constexpr size_t kGemmSmem = 2 * (size_t)kGemmStage;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy K chunk [k0, k0 + 64) of rows [r0, r0 + rows) of a row-major BF16
// matrix into a [8][rows/8][8][8] tile at shared address dst.
__device__ __forceinline__ void gemm_load_tile(uint32_t dst, const __nv_bfloat16* X, int ld, int r0, int rows,
                                               int k0) {
  const int pieces = rows * (kGemmKC / 8);
  for (int p = threadIdx.x; p < pieces; p += 128) {
    const int r = p >> 3, k8 = (p & 7) * 8;
    const __nv_bfloat16* src = X + (size_t)(r0 + r) * ld + k0 + k8;
    const uint32_t off = (uint32_t)((k8 >> 3) * (rows >> 3) + (r >> 3)) * 128u + (uint32_t)(r & 7) * 16u;
    cp_async16(dst + off, src);
  }
}

template <bool kAtomic>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                        const __nv_bfloat16* __restrict__ B, int ldb, float* C,
                                                        int ldc, const float* __restrict__ bias, int Nt, int Ks,
                                                        int* err) {
  extern __shared__ __align__(128) uint8_t gsm[];
  __shared__ uint64_t bars[3];  // mma done per stage, accumulator
  __shared__ uint32_t tslot;
  const int m0 = blockIdx.x * 128, n0 = blockIdx.y * Nt, kbeg = blockIdx.z * Ks;
  const int nchunks = Ks / kGemmKC;
  const uint32_t sbase = tc::smem_u32(gsm);
  const uint32_t bar0 = tc::smem_u32(&bars[0]), bar1 = tc::smem_u32(&bars[1]), bacc = tc::smem_u32(&bars[2]);
  if (threadIdx.x == 0) {
    tc::mbar_init(bar0, 1);
    tc::mbar_init(bar1, 1);
    tc::mbar_init(bacc, 1);
    tc::mbar_fence_init();
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tslot)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t idesc = tc::idesc_bf16(128, Nt);
  const uint32_t lbo_a = 128 * 16, lbo_b = (uint32_t)Nt * 16;
  bool ok = true;

  gemm_load_tile(sbase, A, lda, m0, 128, kbeg);
  gemm_load_tile(sbase + kGemmABytes, B, ldb, n0, Nt, kbeg);
  cp_async_commit();
  for (int c = 0; c < nchunks; ++c) {
    const int s = c & 1;
    if (c + 1 < nchunks) {
      const int s1 = (c + 1) & 1;
      // the stage was last read by the MMAs of chunk c - 1
      if (c >= 1 && !tc::mbar_wait(s1 ? bar1 : bar0, ((c - 1) >> 1) & 1)) ok = false;
      const uint32_t st = sbase + (uint32_t)s1 * kGemmStage;
      gemm_load_tile(st, A, lda, m0, 128, kbeg + (c + 1) * kGemmKC);
      gemm_load_tile(st + kGemmABytes, B, ldb, n0, Nt, kbeg + (c + 1) * kGemmKC);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    tc::fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::tc_fence_after();
      const uint32_t st = sbase + (uint32_t)s * kGemmStage;
#pragma unroll
      for (int j = 0; j < kGemmKC / 16; ++j) {
        const uint64_t ad = tc::sdesc(st + (uint32_t)j * 2 * lbo_a, lbo_a, 128);
        const uint64_t bd = tc::sdesc(st + kGemmABytes + (uint32_t)j * 2 * lbo_b, lbo_b, 128);
        tc::mma_bf16(tmem, ad, bd, idesc, (c > 0 || j > 0) ? 1u : 0u);
      }
      tc::mma_commit(s ? bar1 : bar0);
      if (c + 1 == nchunks) tc::mma_commit(bacc);
    }
  }
  if (!tc::mbar_wait(bacc, 0)) ok = false;
  tc::tc_fence_after();
  // epilogue: warp w holds rows 32 w .. 32 w + 31 of the tile
  const int row = m0 + (int)threadIdx.x;
  const uint32_t lane_base = tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
  float* crow = C + (size_t)row * ldc + n0;
  for (int c = 0; c < Nt; c += 32) {
    float v[32];
    tc::tmem_ld32(lane_base + (uint32_t)c, v);
    if (bias && blockIdx.z == 0) {
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] += __ldg(bias + n0 + c + i);
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
      for (int i = 0; i < 32; i += 4) *reinterpret_cast<float4*>(crow + c + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    }
  }
  if (!ok) atomicExch(err, 1);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}
