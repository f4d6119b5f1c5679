// g1_surrogate.cu -- the learned dynamics surrogate's kernels and their
// C-ABI: the tcgen05 BF16 GEMM (g1_gemm.cuh) and the element-wise forward,
// backward, loss, Adam, feature and integration kernels (g1_surrogate.cuh).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "g1_host.h"
#include "g1_mlp.cuh"
#include "g1_surfeat.cuh"

namespace g1b {
#include "g1_gemm.cuh"
#include "g1_surrogate.cuh"
__device__ int g_gemm_error = 0;
}  // namespace g1b

using namespace g1b;

// Tensor map of a row-major [rows x cols] matrix (leading dimension ld
// elements of esize bytes) read or written in boxes of box_cols x box_rows.
static int gemm_map(CUtensorMap* map, const void* base, CUtensorMapDataType type, int esize, int rows, int cols,
                    int ld, int box_cols, int box_rows, CUtensorMapSwizzle swz) {
  static std::atomic<void*> fn{nullptr};
  void* f = fn.load();
  if (!f) {
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return fail("gemm: cuTensorMapEncodeTiled is not available");
    fn.store(f);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * (cuuint64_t)esize};
  const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f)(
      map, type, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : failf("gemm: tensor map encoding failed (CUresult %d)", (int)r);
}
static int map_bf16_operand(CUtensorMap* m, const void* p, int rows, int cols, int ld, int box_rows) {
  return gemm_map(m, p, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, rows, cols, ld, kGemmKC, box_rows,
                  CU_TENSOR_MAP_SWIZZLE_128B);
}

// Shape checks, tensor maps and the persistent launch of gemm_kernel<kMode>
// (one CTA per SM, at most one per tile).  mn: A is [K][M] and B [K][N]
// (row-major, C = A^T B), loaded in 64 x 64 boxes as MN-major tiles.
template <int kMode>
static int gemm_run(const char* what, int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                    GemmArgs g, cudaStream_t st, bool clear_c = false, bool mn = false) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B) return failf("%s: invalid arguments", what);
  const int Nt = N <= kGemmMaxN ? N : kGemmMaxN;
  if (mn) {
    if (M % 16 || N % 64 || N % Nt || K % kGemmKC)
      return failf("%s: needs M %% 16 == 0, N %% 64 == 0 (and N %% 256 == 0 above 256), K %% 64 == 0", what);
    if (lda % 8 || ldb % 8 || lda < M || ldb < N || (((uintptr_t)A | (uintptr_t)B) & 15))
      return failf("%s: lda >= M, ldb >= N, both multiples of 8, 16-byte aligned operands", what);
  } else {
    if (M % 128 || N % 16 || N % Nt || K % kGemmKC)
      return failf("%s: needs M %% 128 == 0, N %% 16 == 0 (and N %% 256 == 0 above 256), K %% 64 == 0", what);
    if (lda % 8 || ldb % 8 || lda < K || ldb < K || (((uintptr_t)A | (uintptr_t)B) & 15))
      return failf("%s: lda, ldb multiples of 8 and >= K, 16-byte aligned operands", what);
  }
  if (g.Ht && (g.ldt % 8 || ((uintptr_t)g.Ht & 15)))
    return failf("%s: the transposed output needs ldt %% 8 == 0 and 16-byte alignment", what);
  CUtensorMap ma, mb;
  GemmOutMaps om;
  memset(&om, 0, sizeof(om));
  if (mn) {
    if (gemm_map(&ma, A, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, K, M, lda, 64, kGemmKC, CU_TENSOR_MAP_SWIZZLE_128B) ||
        gemm_map(&mb, B, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, K, N, ldb, 64, kGemmKC, CU_TENSOR_MAP_SWIZZLE_128B))
      return -1;
  } else if (map_bf16_operand(&ma, A, M, K, lda, 128) || map_bf16_operand(&mb, B, N, K, ldb, Nt)) {
    return -1;
  }
  // the f map: FP32 C (store), or the FP16 pre-activation (silu out, silu_bwd in)
  if (kMode == kGemmStore &&
      gemm_map(&om.f, g.C, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, M, N, g.ldc, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B))
    return -1;
  if ((kMode == kGemmSilu || kMode == kGemmSiluBwd) && g.Z &&
      gemm_map(&om.f, g.Z, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, M, N, g.ldz, 32, 32, CU_TENSOR_MAP_SWIZZLE_64B))
    return -1;
  if (g.H && gemm_map(&om.h, g.H, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, M, N, g.ldh, 32, 32,
                      CU_TENSOR_MAP_SWIZZLE_64B))
    return -1;
  if (g.Ht && gemm_map(&om.t, g.Ht, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, N, M, g.ldt, 32, 32,
                       CU_TENSOR_MAP_SWIZZLE_NONE))
    return -1;
  cudaError_t e = cudaGetSymbolAddress((void**)&g.err, g_gemm_error);
  if (e != cudaSuccess) return cuda_fail(e, "gemm: error flag");
  if (clear_c && (e = cudaMemset2DAsync(g.C, (size_t)g.ldc * 4, 0, (size_t)N * 4, M, st)) != cudaSuccess)
    return cuda_fail(e, "gemm: clear C");
  g.ntm = (M + 127) / 128;
  g.M = M;
  g.mn = mn ? 1 : 0;
  g.ntn = N / Nt;
  g.nk = K / kGemmKC;
  g.Nt = Nt;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // work items: whole tiles, or (atomic, stream-K) (tile, K chunk) pairs shared evenly by the CTAs
  const long long units = (long long)g.ntm * g.ntn * (kMode == kGemmAtomic ? g.nk : 1);
  if (units > INT32_MAX) return failf("%s: problem too large", what);
  const int grid = units < sms ? (int)units : sms;
  if ((e = prepare<20, kMode>(gemm_kernel<kMode>, gemm_smem<kMode>())) != cudaSuccess)
    return cuda_fail(e, "gemm: attributes");
  // programmatic dependent launch: this kernel's setup may overlap the previous kernel's tail
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3(grid);
  lc.blockDim = dim3(EpiCfg<kMode>::kThreads);
  lc.dynamicSmemBytes = gemm_smem<kMode>();
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  e = cudaLaunchKernelEx(&lc, gemm_kernel<kMode>, ma, mb, om, g);
  if (e != cudaSuccess) return cuda_fail(e, "gemm_kernel");
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, "gemm_kernel");
}

extern "C" {

// ------------------------------------------------- surrogate kernels
int g1b_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                  const float* bias, int splits, void* stream) {
  if (!C || ldc < N || ldc % 4 || ((uintptr_t)C & 15))
    return fail("gemm_bf16: C needs ldc >= N, ldc % 4 == 0, 16-byte alignment");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GemmArgs g{};
  g.C = C;
  g.ldc = ldc;
  g.bias = bias;
  if (splits > 1) return gemm_run<kGemmAtomic>("gemm_bf16", M, N, K, A, lda, B, ldb, g, st, true);
  return gemm_run<kGemmStore>("gemm_bf16", M, N, K, A, lda, B, ldb, g, st);
}

int g1b_gemm_bf16_acc(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                      void* stream) {
  if (!C || ldc < N || ldc % 4 || ((uintptr_t)C & 15))
    return fail("gemm_bf16_acc: C needs ldc >= N, ldc % 4 == 0, 16-byte alignment");
  GemmArgs g{};
  g.C = C;
  g.ldc = ldc;
  return gemm_run<kGemmAtomic>("gemm_bf16_acc", M, N, K, A, lda, B, ldb, g, static_cast<cudaStream_t>(stream));
}

int g1b_gemm_bf16_atb_acc(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                          void* stream) {
  if (!C || ldc < N || ldc % 4 || ((uintptr_t)C & 15))
    return fail("gemm_bf16_atb_acc: C needs ldc >= N, ldc % 4 == 0, 16-byte alignment");
  GemmArgs g{};
  g.C = C;
  g.ldc = ldc;
  return gemm_run<kGemmAtomic>("gemm_bf16_atb_acc", M, N, K, A, lda, B, ldb, g, static_cast<cudaStream_t>(stream),
                               false, true);
}

int g1b_sur_linear_silu(int M, int N, int K, const void* A, int lda, const void* W, int ldw, const float* bias,
                        void* Z, int ldz, void* H, int ldh, void* Ht, int ldt, void* stream) {
  if (!H || ldh < N || ldh % 8 || ((uintptr_t)H & 15))
    return fail("sur_linear_silu: H needs ldh >= N, ldh % 8 == 0, 16-byte alignment");
  if (Z && (ldz < N || ldz % 8 || ((uintptr_t)Z & 15)))
    return fail("sur_linear_silu: Z needs ldz >= N, ldz % 8 == 0, 16-byte alignment");
  if (Ht && ldt < M) return fail("sur_linear_silu: Ht needs ldt >= M");
  GemmArgs g{};
  g.Z = static_cast<__half*>(Z);
  g.ldz = ldz;
  g.bias = bias;
  g.H = static_cast<__nv_bfloat16*>(H);
  g.ldh = ldh;
  g.Ht = static_cast<__nv_bfloat16*>(Ht);
  g.ldt = ldt;
  return gemm_run<kGemmSilu>("sur_linear_silu", M, N, K, A, lda, W, ldw, g, static_cast<cudaStream_t>(stream));
}

int g1b_sur_linear_silu_bwd(int M, int N, int K, const void* dZ, int ldd, const void* W, int ldw, const void* Z,
                            int ldz, void* dH, int ldh, void* dHt, int ldt, float* db, void* stream) {
  if (!Z || ldz < N || ldz % 8 || ((uintptr_t)Z & 15))
    return fail("sur_linear_silu_bwd: Z needs ldz >= N, ldz % 8 == 0, 16-byte alignment");
  if (!dH || ldh < N || ldh % 8 || ((uintptr_t)dH & 15))
    return fail("sur_linear_silu_bwd: dH needs ldh >= N, ldh % 8 == 0, 16-byte alignment");
  if (dHt && ldt < M) return fail("sur_linear_silu_bwd: dHt needs ldt >= M");
  if (dH == dZ) return fail("sur_linear_silu_bwd: dH must not alias dZ");
  GemmArgs g{};
  g.H = static_cast<__nv_bfloat16*>(dH);
  g.ldh = ldh;
  g.Ht = static_cast<__nv_bfloat16*>(dHt);
  g.ldt = ldt;
  g.Z = const_cast<__half*>(static_cast<const __half*>(Z));
  g.ldz = ldz;
  g.db = db;
  return gemm_run<kGemmSiluBwd>("sur_linear_silu_bwd", M, N, K, dZ, ldd, W, ldw, g, static_cast<cudaStream_t>(stream));
}

int g1b_gemm_status(int* code) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_gemm_error, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "gemm_status");
  const int zero = 0;
  e = cudaMemcpyToSymbol(g_gemm_error, &zero, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "gemm_status");
  if (code) *code = v;
  return 0;
}

static int grid_1d(size_t n, int block) {
  const size_t g = (n + block - 1) / block;
  return (int)(g < 148 * 16 ? g : 148 * 16);
}

int g1b_sur_loss(int B, int D, const float* Y, const float* T, const float* w, void* dY, void* dYt, float* db,
                 float* loss, void* stream) {
  if (B <= 0 || D <= 0 || !Y || !T || !w || !dY || !db || !loss) return fail("sur_loss: invalid arguments");
  if (D % 8 || kLossThreads % D) return fail("sur_loss: D must divide 256 and be a multiple of 8");
  const int blocks = (B + kLossRows - 1) / kLossRows;
  sur_loss_kernel<<<blocks, kLossThreads, (size_t)kLossRows * (D + 2) * 2, static_cast<cudaStream_t>(stream)>>>(
      B, D, Y, T, w, static_cast<__nv_bfloat16*>(dY), static_cast<__nv_bfloat16*>(dYt), db, loss);
  return launched("sur_loss_kernel");
}

int g1b_sur_adam_cast(int nl, const g1b_sur_layer* layers, const int* step, const float* lr, float b1, float b2,
                      float eps, void* stream) {
  if (nl <= 0 || nl > kSurMaxLayers || !layers || !step || !lr) return fail("sur_adam_cast: invalid arguments");
  SurOpt o{};
  long long tiles = 0, biases = 0;
  for (int i = 0; i < nl; ++i) {
    const g1b_sur_layer& L = layers[i];
    if (!L.W || !L.b || !L.mW || !L.vW || !L.mb || !L.vb || !L.gW || !L.gb || !L.Wb || !L.Wt || L.rows <= 0 ||
        L.cols <= 0 || (long long)L.rows * L.cols > INT32_MAX)
      return fail("sur_adam_cast: invalid layer");
    o.l[i] = {L.W, L.b, L.mW, L.vW, L.mb, L.vb, L.gW, L.gb, static_cast<__nv_bfloat16*>(L.Wb),
              static_cast<__nv_bfloat16*>(L.Wt), L.rows, L.cols};
    o.tile0[i] = (int)tiles;
    tiles += (long long)((L.rows + kAdamRows - 1) / kAdamRows) * ((L.cols + kAdamCols - 1) / kAdamCols);
    biases += L.rows;
  }
  const long long blocks = tiles + (biases + kAdamThreads - 1) / kAdamThreads;
  if (blocks > INT32_MAX) return fail("sur_adam_cast: too many parameters");
  o.tile0[nl] = (int)tiles;
  o.nl = nl;
  o.step = step;
  o.lr = lr;
  o.b1 = b1;
  o.b2 = b2;
  o.eps = eps;
  sur_adam_cast_kernel<<<(unsigned)blocks, kAdamThreads, 0, static_cast<cudaStream_t>(stream)>>>(o);
  return launched("sur_adam_cast_kernel");
}

int g1b_sur_cast(int rows, int cols, const float* W, void* Wb, void* Wt, void* stream) {
  if (rows <= 0 || cols <= 0 || !W || !Wb || !Wt) return fail("sur_cast: invalid arguments");
  sur_cast_kernel<<<grid_1d((size_t)rows * cols, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, W, static_cast<__nv_bfloat16*>(Wb), static_cast<__nv_bfloat16*>(Wt));
  return launched("sur_cast_kernel");
}

int g1b_sur_features(int n, const float* qpos, const float* qvel, const float* anchor, const float* ctrl,
                     const float* mu, const float* dmass, const float* mean, const float* istd, void* X, void* Xt,
                     float* F, void* stream) {
  if (n <= 0 || !qpos || !qvel || !anchor || !ctrl || !mean || !istd || !X)
    return fail("sur_features: invalid arguments");
  sur_features_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      n, qpos, qvel, anchor, ctrl, mu, dmass, mean, istd, static_cast<__nv_bfloat16*>(X),
      static_cast<__nv_bfloat16*>(Xt), F);
  return launched("sur_features_kernel");
}

int g1b_sur_features_vjp(int n, const float* qpos, const float* qvel, const float* anchor, const float* istd,
                         const float* dX, int ld, float* qpos_b, float* qvel_b, float* anchor_b, float* ctrl_b,
                         void* stream) {
  if (n <= 0 || !qpos || !qvel || !anchor || !istd || !dX || ld < kSurFeat || !qpos_b || !qvel_b || !ctrl_b)
    return fail("sur_features_vjp: invalid arguments");
  sur_feat_vjp_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      n, qpos, qvel, anchor, istd, dX, ld, qpos_b, qvel_b, anchor_b, ctrl_b);
  return launched("sur_feat_vjp_kernel");
}

int g1b_sur_integrate(int n, const float* Y, int ldy, const float* omean, const float* ostd, float dt, float* qpos,
                      float* qvel, void* stream) {
  if (n <= 0 || !Y || ldy < kNV || !omean || !ostd || !qpos || !qvel) return fail("sur_integrate: invalid arguments");
  sur_integrate_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(n, Y, ldy, omean, ostd, dt,
                                                                                       qpos, qvel);
  return launched("sur_integrate_kernel");
}

int g1b_sur_integrate_vjp(int n, const float* qpos, const float* qvel, const float* Y, int ldy, const float* omean,
                          const float* ostd, float dt, float* lam_qpos, float* lam_qvel, float* dY, int ldd,
                          void* stream) {
  if (n <= 0 || !qpos || !qvel || !Y || ldy < kNV || !omean || !ostd || !lam_qpos || !lam_qvel || !dY || ldd < kNV)
    return fail("sur_integrate_vjp: invalid arguments");
  sur_integrate_vjp_kernel<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      n, qpos, qvel, Y, ldy, omean, ostd, dt, lam_qpos, lam_qvel, dY, ldd);
  return launched("sur_integrate_vjp_kernel");
}

int g1b_sur_seed(int total, const float* dY, void* dZ, void* stream) {
  if (total <= 0 || !dY || !dZ) return fail("sur_seed: invalid arguments");
  sur_seed_kernel<<<grid_1d((size_t)total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      total, dY, static_cast<__nv_bfloat16*>(dZ));
  return launched("sur_seed_kernel");
}

}  // extern "C"
