// g1_gemm.cuh -- persistent BF16 tcgen05 GEMM with TMA operand loads and
// TMA-stored fused epilogues, for the dynamics surrogate (included by
// g1_surrogate.cu inside namespace g1b, after g1_mlp.cuh).
//
//   C[M x N] = A[M x K] . B[N x K]^T, A and B BF16 row-major with K
//   contiguous, FP32 accumulation in tensor memory, and one of four
//   epilogues (GemmMode):
//     kGemmStore    C (FP32) = acc (+ bias)
//     kGemmAtomic   C (FP32) += acc (+ bias once): K split over CTAs
//                   (stream-K), C cleared by the caller
//     kGemmSilu     z = acc + bias; Z (FP16, nullable) = z,
//                   H (BF16) = silu(z), Ht (BF16, transposed [N][M], nullable)
//     kGemmSiluBwd  g = acc * silu'(Zin) (Zin FP16); H (BF16) = g, Ht = g
//                   transposed (nullable), db[N] += column sums of g (nullable)
// With GemmArgs::mn the operands are instead A[K x M] and B[K x N], both
// row-major (C = A^T . B, the weight gradient dW = dZ^T . H from the
// activations as the forward and backward layers store them, with no
// transposed copies): the TMA boxes are 64 K rows x 64 columns and the MMAs
// read them as MN-major tiles.  A row tile may then extend past M (the boxes
// beyond it are zero-filled and the atomic epilogue skips those rows).
// The pre-activation Z is kept in FP16 (11 significant bits, eight times
// finer than the BF16 activations; |z| clamped to 65000, where silu' is
// 0 or 1) only for the SiLU derivative of the backward pass.
//
// One CTA per SM walks its work units (GemmSched): tiles of 128 rows x Nt
// columns (Nt = min(N, 256)), blockIdx.x, + gridDim.x, ..., row tiles
// outermost so that the column tiles of one row block run close together and
// read its A rows from L2; in the atomic mode an equal share of (tile,
// K chunk) pairs per CTA.  Warp roles:
//   warp 0   (one lane) TMA producer: for every 64-wide K chunk of a tile,
//            waits until the MMAs have released the stage, then copies the
//            A chunk (128 x 64) and the B chunk (Nt x 64) with
//            cp.async.bulk.tensor (tensor maps over this GPU's memory, each
//            copy into this CTA only) into the ring (EpiCfg::kStages stages of the
//            widest tile, more for narrower ones); the copies
//            complete on the stage's `full` mbarrier (transaction bytes);
//   warp 1   (one lane) MMA issuer: per chunk waits on `full`, issues four
//            tcgen05.mma (M 128, N Nt, K 16) into one of two tensor-memory
//            accumulators and commits them to the stage's `empty` barrier;
//            after a tile's last chunk commits to the accumulator's `full`
//            barrier, and before a tile waits until the epilogue has
//            drained that accumulator (its `empty` barrier, one arrival per
//            epilogue warp);
//   warps 2.. epilogue (EpiCfg::kWarps: 8 or 12, i.e. 2 or 3 per TMEM lane
//            quarter; warp w may access lanes 32 (w % 4) .. + 31, i.e. 32
//            rows of the tile), sharing the tile's 32-column groups:
//            tcgen05.ld, the mode's arithmetic, then the 32 x 32 results go
//            to the warp's staging buffer in shared memory in the layout of
//            the output's tensor map and one lane stores them with
//            cp.async.bulk.tensor (whole lines to global memory instead of
//            one row per lane).  Several warps per SM sub-partition hide
//            each other's latencies, and the MMAs of the next tile run on
//            the other accumulator meanwhile.  The backward mode's
//            pre-activation Z comes in the same way, ahead of its step (TMA
//            load into the staging buffer, per-warp mbarriers).  The bias of
//            the warp's columns is staged once per tile.
// Operand tiles land in the UMMA K-major 128-byte-swizzle layout (each row's
// 64 values one 128-byte line, eight lines a 1024-byte atom, 16-byte piece j
// of row r at piece j ^ (r % 8)), the tensor map's SWIZZLE_128B.  Staging
// layouts: FP32 32 x 32 boxes with SWIZZLE_128B (row r, piece j at
// j ^ (r % 8)), BF16 32 x 32 boxes (64-byte rows) with SWIZZLE_64B (piece j
// at j ^ ((r / 2) % 4)), the transposed BF16 boxes unswizzled: each is
// conflict-free for the lane-per-row writes.  A column group narrower than
// 32 (N % 32 == 16) is written with plain stores instead, so that no box
// reaches into a neighbouring tile.
//
// Every wait is bounded (tc::kWaitNs).  A wait that gives up raises the
// CTA's abort flag and the kernel's error flag; every role then stops
// issuing work, the producer waits (bounded) until the copies it issued have
// landed, the MMA lane until the MMAs it issued are complete, the epilogue
// until its loads and stores have finished, and the tensor memory is
// released.
//
// Constraints (checked by the host launcher): M % 128 == 0, N % 16 == 0,
// N % Nt == 0, K % 64 == 0, lda / ldb / ldh / ldt multiples of 8,
// ldc / ldz of 4, 16-byte aligned operands.

constexpr int kGemmKC = 64;  // K columns per chunk (one 128-byte swizzle line)
constexpr int kGemmMaxN = 256;
constexpr int kGemmMaxStages = 4;
constexpr uint32_t kGemmABytes = 128 * kGemmKC * 2;        // 16 KB
constexpr uint32_t kGemmBBytes = kGemmMaxN * kGemmKC * 2;  // 32 KB
constexpr uint32_t kGemmStageBytes = kGemmABytes + kGemmBBytes;
constexpr uint32_t kGemmAccCols = 256;  // one accumulator; two of them fill the 512 TMEM columns
constexpr uint32_t kEpiBiasBytes = 512;  // per epilogue warp: the bias of its columns of a tile
constexpr int kGemmMaxEpiWarps = 12;
constexpr int kGemmMaxRing = 8;  // ring stages at most (narrow tiles)

// Per mode: operand ring depth, epilogue warps (a multiple of four: 2 or 3
// per TMEM lane quarter, so 2 or 3 per SM sub-partition to hide each other's
// latencies) and each warp's staging layout (byte offsets of its FP32 / FP16
// box F, BF16 box H and transposed BF16 box T; FBoxes boxes alternate in F).
//   store    3 stages, 8 warps: two 4 KB FP32 boxes
//   atomic   4 stages (its epilogue adds straight into C and stages nothing,
//            and its operands both stream from DRAM), 8 warps
//   silu     3 stages, 12 warps: FP16 Z 2 KB, H 2 KB, T 2 KB
//   silu_bwd 3 stages, 12 warps: one FP16 Z input box 2 KB, H 2 KB, T 2 KB
template <int kMode>
struct EpiCfg {
  static constexpr int kStages = kMode == 1 ? 4 : 3;
  static constexpr int kWarps = kMode >= 2 ? 12 : 8;
  static constexpr uint32_t kF = 0, kH = 2048, kT = 4096;
  static constexpr uint32_t kBytes = kMode == 1 ? 0u : (kMode == 0 ? 8192u : 6144u);
  static constexpr int kFBoxes = kMode == 0 ? 2 : 1;  // store mode: FP32 boxes alternating in F
  static constexpr int kZBoxes = 1;                    // backward: FP16 Z boxes in flight in F
  static constexpr int kThreads = 64 + 32 * kWarps;
  static_assert(kMode != 3 || kF + 2048u * kZBoxes <= kH, "the Z boxes must fit below H");
  static_assert(kMode != 0 || kFBoxes * 4096u <= kBytes, "the FP32 boxes must fit the staging");
};
template <int kMode>
__host__ __device__ constexpr size_t gemm_smem() {
  return EpiCfg<kMode>::kStages * (size_t)kGemmStageBytes +
         EpiCfg<kMode>::kWarps * (size_t)(EpiCfg<kMode>::kBytes + kEpiBiasBytes) + 1024;
}

enum GemmMode : int { kGemmStore = 0, kGemmAtomic = 1, kGemmSilu = 2, kGemmSiluBwd = 3 };

struct GemmArgs {
  int ntm, ntn, nk;  // row tiles, column tiles, 64-wide K chunks
  int Nt;                    // columns per tile
  float* C;  // store / atomic: C
  int ldc;
  const float* bias;  // [N], nullable (store, atomic, silu)
  __nv_bfloat16* H;   // silu: silu(z); silu_bwd: g
  int ldh;
  __nv_bfloat16* Ht;  // transposed copy [N][ldt], nullable
  int ldt;
  __half* Z;  // silu: the pre-activation out (nullable); silu_bwd: in
  int ldz;
  float* db;  // silu_bwd: column sums, nullable
  int M;      // rows of C: the atomic epilogue adds no row at or beyond M (a partial last row tile)
  int mn;     // 1: A given as [K][M] and B as [K][N], row-major (MN-major operands, C += A^T B)
  int* err;
};

// The output tensor maps (a map the mode does not use holds a valid dummy).
struct GemmOutMaps {
  CUtensorMap f;  // store: C, FP32 [M][N] box 32 x 32, SWIZZLE_128B; silu / silu_bwd: Z, FP16, SWIZZLE_64B
  CUtensorMap h;  // BF16 [M][N] box 32 x 32, SWIZZLE_64B: H
  CUtensorMap t;  // BF16 [N][M] box 32 x 32, no swizzle: Ht
};

// SiLU and its derivative.  Both results are rounded to BF16 (8 significant
// bits) before they are used, so the hardware exponential and division
// (relative errors ~2^-21) sit far inside that rounding; for z < -87 the
// denominator overflows to infinity and both return 0.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Shared-memory descriptor of a swizzled K-major tile at K step kk (16
// values = 32 bytes along the line): layout SWIZZLE_128B (2), stride between
// 8-row atoms 1024 B, version 1.
__device__ __forceinline__ uint64_t gemm_desc_sw128(uint32_t tile, int kk) {
  const uint32_t a = tile + (uint32_t)kk * 32u;
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// Shared-memory descriptor of an MN-major tile (SWIZZLE_128B) at K step kk:
// each TMA box is 64 K rows of 64 M (or N) values (128 B per row, 8 KB per
// box), so the 8-row atoms of one box are 1024 B apart (stride offset) and
// the boxes, i.e. the 64-wide blocks along M or N, 8 KB apart (leading
// offset); a K step of 16 rows starts 2048 B further on.
__device__ __forceinline__ uint64_t gemm_desc_mn128(uint32_t tile, int kk) {
  const uint32_t a = tile + (uint32_t)kk * 2048u;
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)(8192u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

// 2-D tiled TMA load of the box at (x, y) (x the inner coordinate, a
// multiple of 16 bytes) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// 2-D tiled TMA store of a staged box to (x, y) >= 0, in the bulk group of
// the issuing thread.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// No committed group of this thread still reading shared memory / at most the last one.
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
// Every committed group of this thread complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void gemm_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Bounded wait that also gives up as soon as another role raised the abort flag.
__device__ __forceinline__ bool gemm_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  if (tc::mbar_try(bar, parity)) return true;
  const uint64_t t0 = tc::globaltimer();
  while (!tc::mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (tc::globaltimer() - t0 > tc::kWaitNs) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// One unit of a CTA's work: K chunks [k0, k0 + nk) of output tile (m, n).
struct GemmWork {
  int m, n, k0, nk;
};
// The CTA's sequence of work units (the producer, the MMA lane and the
// epilogue walk the same one).  Atomic mode (split K): with fewer tiles than
// CTAs, cpt = G / tiles CTAs per tile, each a contiguous share of the tile's
// K chunks (the same shares for every tile); otherwise (stream-K) the CTA's
// contiguous share [b T / G, (b + 1) T / G) of the T = tiles x K-chunks
// (tile, chunk) pairs, cut at tile boundaries.  Either way every SM gets
// (nearly) the same number of chunks whatever the tile count; partial tiles
// meet in C through the atomic adds.  Other modes: whole tiles blockIdx.x,
// + gridDim.x, ...
template <int kMode>
struct GemmSched {
  int pos, end;
  __device__ explicit GemmSched(const GemmArgs& g) {
    if (kMode == kGemmAtomic) {
      const int ntiles = g.ntm * g.ntn, G = (int)gridDim.x;
      if (ntiles < G) {
        // every tile gets cpt CTAs and the same split of its K chunks, so the
        // CTAs that read one operand chunk for different tiles (the column
        // tiles of a row block, the row tiles of a column block) fetch it at
        // the same time and all but the first find it in L2
        const int cpt = G / ntiles, b = (int)blockIdx.x;
        const int t = b / cpt, s = b - t * cpt;
        const int k0 = (int)((long long)g.nk * s / cpt), k1 = (int)((long long)g.nk * (s + 1) / cpt);
        pos = t * g.nk + k0;
        end = b < cpt * ntiles ? t * g.nk + k1 : pos;  // the G - cpt * ntiles spare CTAs idle
      } else {
        const long long T = (long long)ntiles * g.nk;
        pos = (int)(T * blockIdx.x / gridDim.x);
        end = (int)(T * (blockIdx.x + 1) / gridDim.x);
      }
    } else {
      pos = (int)blockIdx.x;
      end = g.ntm * g.ntn;
    }
  }
  __device__ bool next(const GemmArgs& g, GemmWork& w) {
    if (pos >= end) return false;
    if (kMode == kGemmAtomic) {
      const int t = pos / g.nk, k0 = pos - t * g.nk;
      const int nk = g.nk - k0 < end - pos ? g.nk - k0 : end - pos;
      w = {t / g.ntn, t % g.ntn, k0, nk};
      pos += nk;
    } else {
      w = {pos / g.ntn, pos % g.ntn, 0, g.nk};
      pos += (int)gridDim.x;
    }
    return true;
  }
};

// ------------------------------------------------------------ epilogue
// Staging writes of one lane's row r (0..31) of a 32 x 32 box.
// FP32 box, SWIZZLE_128B: 128-byte rows, 16-byte piece j at j ^ (r % 8).
__device__ __forceinline__ void stage_f32(uint8_t* box, int r, const float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 8; ++j)
    *reinterpret_cast<float4*>(box + r * 128 + ((j ^ (r & 7)) << 4)) =
        make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
}
__device__ __forceinline__ void unstage_f32(const uint8_t* box, int r, float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const float4 q = *reinterpret_cast<const float4*>(box + r * 128 + ((j ^ (r & 7)) << 4));
    v[4 * j] = q.x;
    v[4 * j + 1] = q.y;
    v[4 * j + 2] = q.z;
    v[4 * j + 3] = q.w;
  }
}
// BF16 box, SWIZZLE_64B: 64-byte rows, 16-byte piece j (8 values) at j ^ ((r / 2) % 4).
__device__ __forceinline__ void stage_bf16(uint8_t* box, int r, const float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    uint4 w;
    w.x = tc::pack_bf16x2(v[8 * j], v[8 * j + 1]);
    w.y = tc::pack_bf16x2(v[8 * j + 2], v[8 * j + 3]);
    w.z = tc::pack_bf16x2(v[8 * j + 4], v[8 * j + 5]);
    w.w = tc::pack_bf16x2(v[8 * j + 6], v[8 * j + 7]);
    *reinterpret_cast<uint4*>(box + r * 64 + ((j ^ ((r >> 1) & 3)) << 4)) = w;
  }
}
// FP16 box, SWIZZLE_64B, as the BF16 one (the pre-activation Z).
__device__ __forceinline__ void stage_f16(uint8_t* box, int r, const float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const __half2 h = __floats2half2_rn(fminf(fmaxf(v[8 * j + 2 * i], -65000.0f), 65000.0f),
                                          fminf(fmaxf(v[8 * j + 2 * i + 1], -65000.0f), 65000.0f));
      w[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    *reinterpret_cast<uint4*>(box + r * 64 + ((j ^ ((r >> 1) & 3)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}
__device__ __forceinline__ void unstage_f16(const uint8_t* box, int r, float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint4 q = *reinterpret_cast<const uint4*>(box + r * 64 + ((j ^ ((r >> 1) & 3)) << 4));
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[i]));
      v[8 * j + 2 * i] = f.x;
      v[8 * j + 2 * i + 1] = f.y;
    }
  }
}
// Transposed BF16 box, no swizzle: element (column i, row r) at i * 64 + 2 r.
__device__ __forceinline__ void stage_bf16_t(uint8_t* box, int r, const float (&v)[32]) {
  __nv_bfloat16* b = reinterpret_cast<__nv_bfloat16*>(box);
#pragma unroll
  for (int i = 0; i < 32; ++i) b[i * 32 + r] = __float2bfloat16_rn(v[i]);
}

// Plain stores of a narrow group (nb < 32 columns) or of the atomic mode:
// FP32 row to C (store, atomic add), BF16 row to H and its transpose to Ht.
template <bool kAtomic>
__device__ __forceinline__ void direct_f32(float* crow, const float (&v)[32], int nb) {
  if (nb == 32) {
#pragma unroll
    for (int i = 0; i < 32; i += 4) {
      const float4 q = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      if (kAtomic)
        atomicAdd(reinterpret_cast<float4*>(crow + i), q);
      else
        *reinterpret_cast<float4*>(crow + i) = q;
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    if (i >= nb) continue;
    if (kAtomic)
      atomicAdd(crow + i, v[i]);
    else
      crow[i] = v[i];
  }
}
__device__ __forceinline__ void direct_f16(__half* zrow, const float (&v)[32], int nb) {
#pragma unroll
  for (int i = 0; i < 32; ++i)
    if (i < nb) zrow[i] = __float2half_rn(fminf(fmaxf(v[i], -65000.0f), 65000.0f));
}
__device__ __forceinline__ void direct_bf16(const GemmArgs& g, const float (&v)[32], int row, int col, int nb) {
  __nv_bfloat16* h = g.H + (size_t)row * g.ldh + col;
#pragma unroll
  for (int i = 0; i < 32; ++i)
    if (i < nb) h[i] = __float2bfloat16_rn(v[i]);
  if (g.Ht) {
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (i < nb) g.Ht[(size_t)(col + i) * g.ldt + row] = __float2bfloat16_rn(v[i]);
  }
}

// Column sums over the warp's 32 rows (lane = row) into db[col .. col + nb):
// recursive halving across the lanes, five shuffle levels (16 + 8 + 4 + 2 +
// 1 exchanges), after which lane l holds the sum of column l.
__device__ __forceinline__ void column_sums(float* db, const float (&v)[32], int col, int nb) {
  const int lane = threadIdx.x & 31;
  float w[16];
  {
    const bool hi = lane & 16;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float send = hi ? v[i] : v[i + 16];
      w[i] = (hi ? v[i + 16] : v[i]) + __shfl_xor_sync(0xffffffffu, send, 16);
    }
  }
#pragma unroll
  for (int off = 8; off >= 1; off >>= 1) {
    const bool hi = lane & off;
#pragma unroll
    for (int i = 0; i < off; ++i) {
      const float send = hi ? w[i] : w[i + off];
      w[i] = (hi ? w[i + off] : w[i]) + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  if (lane < nb) atomicAdd(db + col + lane, w[0]);
}

// The epilogue role (warps 2 .. 2 + kWarps - 1).  Warp w owns TMEM lane
// quarter w % 4 (rows 32 (w % 4) .. + 31 of the tile) and, of the tile's
// 32-column groups, those g with g % P == (w - 2) / 4 (P = kWarps / 4).  mf / mh
// / mt: the output maps (kernel parameters, so their generic addresses stay
// valid for TMA).
template <int kMode>
__device__ __forceinline__ bool gemm_epilogue(const GemmArgs& g, const CUtensorMap* mf, const CUtensorMap* mh,
                                              const CUtensorMap* mt, uint32_t tmem, uint8_t* ep0, uint32_t ebase0,
                                              uint64_t* zbar, uint64_t* accf, uint64_t* acce, int ntiles,
                                              volatile int* abort_v) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3;   // TMEM lane quarter = the warp's 32 rows of the tile
  const int ew = warp - 2;  // staging area and mbarrier of this warp
  using E = EpiCfg<kMode>;
  constexpr int P = E::kWarps / 4;                  // warps per lane quarter
  constexpr int ZB = E::kZBoxes;                   // backward: Z boxes in flight
  const int par = ew >> 2;  // the warp's column groups: par, par + P, ...
  uint8_t* const ep = ep0 + (size_t)ew * E::kBytes;
  const uint32_t es = ebase0 + (uint32_t)ew * E::kBytes;
  float* const sbias = reinterpret_cast<float*>(ep0 + (size_t)E::kWarps * E::kBytes + ew * kEpiBiasBytes);
  const uint32_t zb0 = tc::smem_u32(&zbar[2 * ew]);  // Z box k: slot k % ZB, barrier zb0 + 8 (k % ZB)
  const bool st_f = kMode == kGemmStore;                      // FP32 C
  const bool st_z = kMode == kGemmSilu && g.Z != nullptr;      // FP16 Z
  const bool st_h = kMode == kGemmSilu || kMode == kGemmSiluBwd;
  const bool st_t = st_h && g.Ht != nullptr;
  const bool has_bias = g.bias != nullptr && kMode != kGemmSiluBwd;
  const int ngroups = (g.Nt + 31) / 32;
  const int spw = (ngroups - par + P - 1) / P;  // this warp's groups per tile
  // steps of the backward mode's Z prefetch (whole tiles blockIdx.x, + gridDim.x, ...)
  const int my_tiles = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int nsteps = my_tiles * spw;
  bool ok = true;
  int zi = 0, zw = 0;  // backward: Z boxes issued, waited for
  // backward: TMA load of the Z box of step k (this warp's rows and group)
  auto z_issue = [&](int k) {
    if (lane == 0) {
      const int t = (int)blockIdx.x + (k / spw) * (int)gridDim.x;
      const uint32_t zb = zb0 + 8u * (uint32_t)(k % ZB);
      tc::fence_async_smem();
      tc::mbar_expect_tx(zb, 2048);
      tma_load_2d(es + E::kF + 2048u * (uint32_t)(k % ZB), mf, (t % g.ntn) * g.Nt + (P * (k % spw) + par) * 32,
                  (t / g.ntn) * 128 + q * 32, zb);
    }
    ++zi;
  };
  if (kMode == kGemmSiluBwd)
    for (int kk = 0; kk < ZB && kk < nsteps; ++kk) z_issue(kk);
  int k = 0, j = 0;
  GemmSched<kMode> sched(g);
  GemmWork tl;
  for (; ok && sched.next(g, tl); ++j) {
    const int b = j & 1;
    const bool add_bias = has_bias && tl.k0 == 0;  // atomic mode: the unit holding K chunk 0
    if (add_bias) {  // this warp's bias values of the tile
      __syncwarp();
      for (int s = 0; s < spw; ++s) {
        const int c = (P * s + par) * 32 + lane;
        sbias[s * 32 + lane] = c < g.Nt ? __ldg(g.bias + tl.n * g.Nt + c) : 0.0f;  // exactly N floats
      }
      __syncwarp();
    }
    // every wait of the epilogue is warp-uniform (the warp's tcgen05.ld are .sync.aligned)
    if (!__all_sync(0xffffffffu, gemm_wait(tc::smem_u32(&accf[b]), ((uint32_t)j >> 1) & 1, abort_v))) {
      ok = false;
      break;
    }
    tc::tc_fence_after();
    const int row0 = tl.m * 128 + q * 32, row = row0 + lane;
    const uint32_t taddr = tmem + (uint32_t)b * kGemmAccCols + ((uint32_t)(q * 32) << 16);
    for (int s = 0; s < spw; ++s, ++k) {
      const int c = (P * s + par) * 32;
      const int nb = g.Nt - c < 32 ? g.Nt - c : 32;
      const int col = tl.n * g.Nt + c;
      float v[32];
      tc::tmem_ld32(taddr + (uint32_t)c, v);
      if (kMode == kGemmSiluBwd) {
        if (!__all_sync(0xffffffffu, gemm_wait(zb0 + 8u * (uint32_t)(k % ZB), (uint32_t)(k / ZB) & 1, abort_v))) {
          ok = false;
          break;
        }
        ++zw;
        float z[32];
        unstage_f16(ep + E::kF + 2048 * (k % ZB), lane, z);
        __syncwarp();  // every lane has read the box: the next one may land in its place
        if (k + ZB < nsteps) z_issue(k + ZB);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] *= silu_grad(z[i]);
        if (g.db) column_sums(g.db, v, col, nb);
      } else if (add_bias) {
        const float4* bq = reinterpret_cast<const float4*>(sbias + s * 32);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const float4 bb = bq[i];  // same address in every lane: a broadcast
          v[4 * i] += bb.x;
          v[4 * i + 1] += bb.y;
          v[4 * i + 2] += bb.z;
          v[4 * i + 3] += bb.w;
        }
      }
      if constexpr (kMode == kGemmAtomic) {
        if (row < g.M) direct_f32<true>(g.C + (size_t)row * g.ldc + col, v, nb);
      } else {
        float hv[32];  // the BF16 output's values
#pragma unroll
        for (int i = 0; i < 32; ++i) hv[i] = kMode == kGemmSilu ? silu(v[i]) : v[i];
        if (nb < 32) {  // narrow group: plain stores
          if (st_f) direct_f32<false>(g.C + (size_t)row * g.ldc + col, v, nb);
          if (st_z) direct_f16(g.Z + (size_t)row * g.ldz + col, v, nb);
          if (st_h) direct_bf16(g, hv, row, col, nb);
          continue;
        }
        // the store mode alternates two FP32 boxes (its H and T slots are free): the stores of
        // step k - 2 have read this one; the other modes' single slot: those of step k - 1
        const uint32_t fofs = 4096u * (uint32_t)(k % E::kFBoxes);
        if (lane == 0) {
          if (kMode == kGemmStore)
            bulk_wait_read1();
          else
            bulk_wait_read0();
        }
        __syncwarp();
        if (st_f) stage_f32(ep + E::kF + fofs, lane, v);
        if (st_z) stage_f16(ep + E::kF, lane, v);
        if (st_h) stage_bf16(ep + E::kH, lane, hv);
        if (st_t) stage_bf16_t(ep + E::kT, lane, hv);
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) {
          if (st_f || st_z) tma_store_2d(mf, col, row0, es + E::kF + fofs);
          if (st_h) tma_store_2d(mh, col, row0, es + E::kH);
          if (st_t) tma_store_2d(mt, row0, col, es + E::kT);
          bulk_commit();
        }
      }
    }
    if (!ok) break;
    tc::tc_fence_before();
    __syncwarp();
    if (lane == 0) gemm_arrive(tc::smem_u32(&acce[b]));
  }
  // the Z boxes issued and not waited for have landed, the stores have completed
  for (; zw < zi; ++zw)
    if (!tc::mbar_wait(zb0 + 8u * (uint32_t)(zw % ZB), (uint32_t)(zw / ZB) & 1)) ok = false;
  if (lane == 0) bulk_wait_all();
  __syncwarp();
  return ok;
}

// ---------------------------------------------------------------- kernel
template <int kMode>
__global__ void __launch_bounds__(EpiCfg<kMode>::kThreads, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ GemmOutMaps om, GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t gsm[];
  // The ring holds EpiCfg::kStages stages of the widest tile (Nt = 256); a
  // narrower tile (the output layer's Nt = 64) packs more, smaller stages
  // into the same bytes, so more of its operand stream is in flight.
  constexpr uint32_t kRingBytes = (uint32_t)EpiCfg<kMode>::kStages * kGemmStageBytes;
  const uint32_t stage_bytes = kGemmABytes + (uint32_t)g.Nt * kGemmKC * 2;  // a multiple of 2 KB
  const uint32_t nst = kRingBytes / stage_bytes < (uint32_t)kGemmMaxRing ? kRingBytes / stage_bytes
                                                                         : (uint32_t)kGemmMaxRing;
  __shared__ uint64_t full[kGemmMaxRing], empty[kGemmMaxRing], accf[2], acce[2], drain, zbar[2 * kGemmMaxEpiWarps];
  __shared__ uint32_t tslot;
  __shared__ int abort_flag;
  volatile int* abort_v = &abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t base0 = tc::smem_u32(gsm);
  const uint32_t sbase = (base0 + 1023u) & ~1023u;  // swizzle atoms need 1024-byte alignment
  const uint32_t ebase0 = sbase + kRingBytes;  // epilogue staging
  const int ntiles = g.ntm * g.ntn;
  const uint32_t btx = (uint32_t)g.Nt * kGemmKC * 2;  // B bytes per chunk
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < nst; ++s) {
      tc::mbar_init(tc::smem_u32(&full[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(tc::smem_u32(&accf[b]), 1);
      tc::mbar_init(tc::smem_u32(&acce[b]), EpiCfg<kMode>::kWarps);
    }
    for (int w = 0; w < 2 * EpiCfg<kMode>::kWarps; ++w) tc::mbar_init(tc::smem_u32(&zbar[w]), 1);
    tc::mbar_init(tc::smem_u32(&drain), 1);
    abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), 2 * kGemmAccCols);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tslot;
  bool ok = true;
  // Launched as a programmatic dependent of the previous kernel on the stream:
  // the setup above may overlap that kernel's last CTAs; nothing below reads
  // or writes global memory before it has completed and its writes are
  // visible.  Our own dependents may be scheduled from now on (they wait the
  // same way).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
      uint32_t it = 0;  // chunks issued by this CTA
      GemmSched<kMode> sched(g);
      GemmWork w;
      while (ok && sched.next(g, w)) {
        for (int c = 0; c < w.nk; ++c) {
          const int s = (int)(it % nst);
          const uint32_t r = it / nst;
          if (r > 0 && !gemm_wait(tc::smem_u32(&empty[s]), (r - 1) & 1, abort_v)) {
            ok = false;
            break;
          }
          const uint32_t st = sbase + (uint32_t)s * stage_bytes;
          const uint32_t bar = tc::smem_u32(&full[s]);
          const int kx = (w.k0 + c) * kGemmKC;
          tc::mbar_expect_tx(bar, kGemmABytes + btx);
          if (g.mn) {  // 64-column boxes of the row-major [K][M] and [K][N] operands
            tma_load_2d(st, &tmA, w.m * 128, kx, bar);
            tma_load_2d(st + 8192u, &tmA, w.m * 128 + 64, kx, bar);  // beyond M: zero fill
            for (int b = 0; b < g.Nt / 64; ++b)
              tma_load_2d(st + kGemmABytes + 8192u * (uint32_t)b, &tmB, w.n * g.Nt + 64 * b, kx, bar);
          } else {
            tma_load_2d(st, &tmA, kx, w.m * 128, bar);
            tma_load_2d(st + kGemmABytes, &tmB, kx, w.n * g.Nt, bar);
          }
          ++it;
        }
      }
      // every copy issued has landed before the CTA may exit
      for (uint32_t s = 0; s < nst; ++s) {
        const uint32_t n_s = it > s ? (it - s - 1) / nst + 1 : 0;
        if (n_s > 0 && !tc::mbar_wait(tc::smem_u32(&full[s]), (n_s - 1) & 1)) ok = false;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer
      // bits 15 and 16: A and B MN-major
      const uint32_t idesc = tc::idesc_bf16(128, g.Nt) | (g.mn ? (3u << 15) : 0u);
      uint32_t it = 0;
      int j = 0;  // work units of this CTA
      GemmSched<kMode> sched(g);
      GemmWork w;
      for (; ok && sched.next(g, w); ++j) {
        const int b = j & 1;
        const uint32_t u = (uint32_t)j >> 1;
        if (u > 0 && !gemm_wait(tc::smem_u32(&acce[b]), (u - 1) & 1, abort_v)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t d = tmem + (uint32_t)b * kGemmAccCols;
        for (int c = 0; c < w.nk; ++c, ++it) {
          const int s = (int)(it % nst);
          const uint32_t r = it / nst;
          if (!gemm_wait(tc::smem_u32(&full[s]), r & 1, abort_v)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t st = sbase + (uint32_t)s * stage_bytes;
#pragma unroll
          for (int kk = 0; kk < kGemmKC / 16; ++kk) {
            const uint64_t ad = g.mn ? gemm_desc_mn128(st, kk) : gemm_desc_sw128(st, kk);
            const uint64_t bd = g.mn ? gemm_desc_mn128(st + kGemmABytes, kk) : gemm_desc_sw128(st + kGemmABytes, kk);
            tc::mma_bf16(d, ad, bd, idesc, (c > 0 || kk > 0) ? 1u : 0u);
          }
          tc::mma_commit(tc::smem_u32(&empty[s]));
        }
        if (!ok) break;
        tc::mma_commit(tc::smem_u32(&accf[b]));
      }
      // every MMA issued is complete before the tensor memory is released
      tc::mma_commit(tc::smem_u32(&drain));
      if (!tc::mbar_wait(tc::smem_u32(&drain), 0)) ok = false;
    }
  } else {
    ok = gemm_epilogue<kMode>(g, &om.f, &om.h, &om.t, tmem, gsm + (ebase0 - base0), ebase0, zbar, accf, acce, ntiles,
                              abort_v);
  }
  if (!ok) {
    *abort_v = 1;
    atomicExch(g.err, 1);
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 0) tc::tmem_dealloc(tmem, 2 * kGemmAccCols);
}
