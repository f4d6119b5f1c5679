// g1_surrogate.cu -- the learned dynamics surrogate's kernels and their
// C-ABI: the tcgen05 BF16 GEMM (g1_gemm.cuh) and the element-wise forward,
// backward, loss, Adam, feature and integration kernels (g1_surrogate.cuh).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "g1_host.h"
#include "g1_mlp.cuh"
#include "g1_surfeat.cuh"

namespace g1b {
#include "g1_gemm.cuh"
#include "g1_surrogate.cuh"
__device__ int g_gemm_error = 0;
}  // namespace g1b

using namespace g1b;

extern "C" {

// ------------------------------------------------- surrogate kernels
int g1b_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                  const float* bias, int splits, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !C) return fail("gemm_bf16: invalid arguments");
  if (splits < 1) splits = 1;
  const int Nt = N <= kGemmMaxN ? N : kGemmMaxN;
  if (M % 128 || N % 16 || N % Nt || K % (kGemmKC * splits))
    return fail("gemm_bf16: needs M % 128 == 0, N % 16 == 0 (and N % 256 == 0 above 256), K % (64 splits) == 0");
  if (lda % 8 || ldb % 8 || ldc % 4 || (((uintptr_t)A | (uintptr_t)B) & 15) || (((uintptr_t)C) & 15))
    return fail("gemm_bf16: lda, ldb multiples of 8, ldc of 4, 16-byte aligned pointers");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int MT = M % 256 == 0 ? 2 : 1;  // two row tiles per CTA share each weight chunk
  const dim3 grid(M / (128 * MT), N / Nt, splits);
  int* err = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&err, g_gemm_error);
  if (e != cudaSuccess) return cuda_fail(e, "gemm_bf16: error flag");
  const __nv_bfloat16* a = static_cast<const __nv_bfloat16*>(A);
  const __nv_bfloat16* b = static_cast<const __nv_bfloat16*>(B);
  if (splits > 1) {
    e = cudaMemset2DAsync(C, (size_t)ldc * 4, 0, (size_t)N * 4, M, st);
    if (e != cudaSuccess) return cuda_fail(e, "gemm_bf16: clear C");
  }
#define G1_GEMM_LAUNCH(AT, M_T, KEY)                                                              \
  do {                                                                                           \
    if ((e = prepare<20, KEY>(gemm_bf16_kernel<AT, M_T>, gemm_smem<M_T>())) != cudaSuccess)      \
      return cuda_fail(e, "gemm_bf16: attributes");                                              \
    gemm_bf16_kernel<AT, M_T><<<grid, 128, gemm_smem<M_T>(), st>>>(a, lda, b, ldb, C, ldc, bias, Nt, \
                                                                  K / splits, err);              \
  } while (0)
  if (splits > 1) {
    if (MT == 2) G1_GEMM_LAUNCH(true, 2, 3); else G1_GEMM_LAUNCH(true, 1, 1);
  } else {
    if (MT == 2) G1_GEMM_LAUNCH(false, 2, 2); else G1_GEMM_LAUNCH(false, 1, 0);
  }
#undef G1_GEMM_LAUNCH
  e = cudaGetLastError();
  return e == cudaSuccess ? 0 : cuda_fail(e, "gemm_bf16_kernel");
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

int g1b_sur_act(int B, int D, const float* Z, void* H, void* Ht, void* stream) {
  if (B <= 0 || D <= 0 || !Z || !H) return fail("sur_act: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_act_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, Z, static_cast<__nv_bfloat16*>(H), static_cast<__nv_bfloat16*>(Ht));
  return launched("sur_act_kernel");
}

int g1b_sur_act_bwd(int B, int D, const float* dH, const float* Z, void* dZ, void* dZt, float* db, void* stream) {
  if (B <= 0 || D <= 0 || !dH || !Z || !dZ || !dZt || !db) return fail("sur_act_bwd: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_act_bwd_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, dH, Z, static_cast<__nv_bfloat16*>(dZ), static_cast<__nv_bfloat16*>(dZt), db);
  return launched("sur_act_bwd_kernel");
}

int g1b_sur_loss(int B, int D, const float* Y, const float* T, const float* w, void* dY, void* dYt, float* db,
                 float* loss, void* stream) {
  if (B <= 0 || D <= 0 || !Y || !T || !w || !dY || !dYt || !db || !loss) return fail("sur_loss: invalid arguments");
  const dim3 grid((D + 31) / 32, (B + 31) / 32), block(32, 8);
  sur_loss_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      B, D, Y, T, w, static_cast<__nv_bfloat16*>(dY), static_cast<__nv_bfloat16*>(dYt), db, loss);
  return launched("sur_loss_kernel");
}

int g1b_sur_adam(int n, float* p, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                 int step, void* stream) {
  if (n <= 0 || !p || !g || !m || !v || step < 1) return fail("sur_adam: invalid arguments");
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  sur_adam_kernel<<<grid_1d((size_t)n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, p, g, m, v, lr, b1, b2,
                                                                                         eps, c1, c2);
  return launched("sur_adam_kernel");
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
