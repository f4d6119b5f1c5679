// g1_surrogate.cuh -- kernels of the learned one-step dynamics surrogate
// (included by g1_kernels.cu inside namespace g1b, after g1_gemm.cuh).
//
// The surrogate is an MLP 128 -> 512 -> 512 -> 512 -> 512 -> 64 with SiLU on
// the hidden layers, over a normalised feature vector of the state and the
// PD targets, predicting the normalised generalised acceleration of the step
// (the state delta is dt * qacc for qvel, and qpos follows by the step's own
// semi-implicit Euler).  Its matrix products run on gemm_bf16_kernel
// (tcgen05); the element-wise parts of the forward and backward passes, the
// loss, Adam and the feature extraction are the kernels below.

constexpr int kSurIn = 128;    // padded input features (109 used)
constexpr int kSurOut = 64;    // padded outputs (35 used: qacc)
constexpr int kSurFeat = 109;  // q 29, qd 29, z 1, rot6 6, v body 3, w body 3, contact flags 8, targets 29, 1

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// The element-wise kernels below work on 32 x 32 tiles (block 32 x 8): rows
// r0..r0+31 of the batch and columns c0..c0+31, reading and writing the
// row-major arrays along columns and the transposed copies along rows
// through a shared-memory tile, so both sides are coalesced.

// H = SiLU(Z) (BF16, [B][D]) and its transpose Ht ([D][B], nullable).
__global__ void sur_act_kernel(int B, int D, const float* __restrict__ Z, __nv_bfloat16* H, __nv_bfloat16* Ht) {
  __shared__ __nv_bfloat16 t[32][34];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < B && c < D) {
      const size_t i = (size_t)r * D + c;
      const __nv_bfloat16 h = __float2bfloat16_rn(silu(Z[i]));
      H[i] = h;
      t[k][threadIdx.x] = h;
    }
  }
  if (!Ht) return;
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < B && c < D) Ht[(size_t)c * B + r] = t[threadIdx.x][k];
  }
}

// dZ = dH * SiLU'(Z): BF16 [B][D] and transposed [D][B]; db[c] += column sums.
__global__ void sur_act_bwd_kernel(int B, int D, const float* __restrict__ dH, const float* __restrict__ Z,
                                   __nv_bfloat16* dZ, __nv_bfloat16* dZt, float* db) {
  __shared__ __nv_bfloat16 t[32][34];
  __shared__ float red[8][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  float acc = 0.0f;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < B && c < D) {
      const size_t i = (size_t)r * D + c;
      const float g = dH[i] * silu_grad(Z[i]);
      acc += g;
      const __nv_bfloat16 gb = __float2bfloat16_rn(g);
      dZ[i] = gb;
      t[k][threadIdx.x] = gb;
    }
  }
  red[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < B && c < D) dZt[(size_t)c * B + r] = t[threadIdx.x][k];
  }
  if (threadIdx.y == 0 && c0 + threadIdx.x < D) {
    float s = 0.0f;
    for (int k = 0; k < 8; ++k) s += red[k][threadIdx.x];
    atomicAdd(db + c0 + threadIdx.x, s);
  }
}

// Weighted MSE over the output columns: loss += sum_r sum_c w[c] (Y - T)^2 / B;
// dY = 2 w[c] (Y - T) / B as BF16 [B][D] and transposed [D][B]; db += sums.
__global__ void sur_loss_kernel(int B, int D, const float* __restrict__ Y, const float* __restrict__ T,
                                const float* __restrict__ w, __nv_bfloat16* dY, __nv_bfloat16* dYt, float* db,
                                float* loss) {
  __shared__ __nv_bfloat16 t[32][34];
  __shared__ float red[2][8][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int c = c0 + threadIdx.x;
  const float wc = c < D ? w[c] : 0.0f;
  float acc = 0.0f, l = 0.0f;
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int r = r0 + k;
    if (r < B && c < D) {
      const size_t i = (size_t)r * D + c;
      const float e = Y[i] - T[i];
      l += wc * e * e;
      const float g = 2.0f * wc * e / (float)B;
      acc += g;
      const __nv_bfloat16 gb = __float2bfloat16_rn(g);
      dY[i] = gb;
      t[k][threadIdx.x] = gb;
    }
  }
  red[0][threadIdx.y][threadIdx.x] = acc;
  red[1][threadIdx.y][threadIdx.x] = l;
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += 8) {
    const int cc = c0 + k, r = r0 + threadIdx.x;
    if (r < B && cc < D) dYt[(size_t)cc * B + r] = t[threadIdx.x][k];
  }
  if (threadIdx.y == 0) {
    float s = 0.0f, ls = 0.0f;
    for (int k = 0; k < 8; ++k) {
      s += red[0][k][threadIdx.x];
      ls += red[1][k][threadIdx.x];
    }
    if (c < D) atomicAdd(db + c, s);
    // one loss atomic per block (warp sum), not one per column
    for (int o = 16; o > 0; o >>= 1) ls += __shfl_xor_sync(0xffffffffu, ls, o);
    if (threadIdx.x == 0) atomicAdd(loss, ls / (float)B);
  }
}

// Adam (Kingma & Ba 2015) with bias correction, in place on FP32 p, m, v.
__global__ void sur_adam_kernel(int n, float* p, const float* __restrict__ g, float* m, float* v, float lr, float b1,
                                float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// W [rows][cols] FP32 -> BF16 copy and BF16 transpose [cols][rows].
__global__ void sur_cast_kernel(int rows, int cols, const float* __restrict__ W, __nv_bfloat16* Wb,
                                __nv_bfloat16* Wt) {
  const int n = rows * cols;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = i / cols, c = i % cols;
    const __nv_bfloat16 h = __float2bfloat16_rn(W[i]);
    Wb[i] = h;
    Wt[(size_t)c * rows + r] = h;
  }
}

// Feature vector of env e (raw, before normalisation): joint angles and
// rates, base height, the first two columns of the base rotation, base
// linear and angular velocity in the body frame, contact flags (normal force
// > 0 per sphere), PD targets, and a constant 1.
__device__ __forceinline__ void sur_features_raw(const float* qpos, const float* qvel, const float* ctrl,
                                                 const float* cf, size_t n, int e, float* f) {
  int k = 0;
  for (int j = 0; j < 29; ++j) f[k++] = qpos[(size_t)(7 + j) * n + e];
  for (int j = 0; j < 29; ++j) f[k++] = qvel[(size_t)(6 + j) * n + e];
  f[k++] = qpos[2 * n + e];
  const float qw = qpos[3 * n + e], qx = qpos[4 * n + e], qy = qpos[5 * n + e], qz = qpos[6 * n + e];
  const float R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz),     2 * (qx * qz + qw * qy),
                      2 * (qx * qy + qw * qz),     1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx),
                      2 * (qx * qz - qw * qy),     2 * (qy * qz + qw * qx),     1 - 2 * (qx * qx + qy * qy)};
  f[k++] = R[0];
  f[k++] = R[3];
  f[k++] = R[6];
  f[k++] = R[1];
  f[k++] = R[4];
  f[k++] = R[7];
  const float vw[3] = {qvel[e], qvel[n + e], qvel[2 * n + e]};
  for (int i = 0; i < 3; ++i) f[k++] = R[i] * vw[0] + R[3 + i] * vw[1] + R[6 + i] * vw[2];  // R^T v
  for (int i = 0; i < 3; ++i) f[k++] = qvel[(size_t)(3 + i) * n + e];
  for (int i = 0; i < 8; ++i) f[k++] = cf ? (cf[(size_t)i * n + e] > 0.0f ? 1.0f : 0.0f) : 0.0f;
  for (int j = 0; j < 29; ++j) f[k++] = ctrl[(size_t)j * n + e];
  f[k++] = 1.0f;
}

// X[e][:] = BF16((f - mean) * istd), padded with zeros to 128; Xt the
// transpose (nullable); raw features to F (FP32 [n][128], nullable).
__global__ void sur_features_kernel(int n, const float* qpos, const float* qvel, const float* ctrl, const float* cf,
                                    const float* __restrict__ mean, const float* __restrict__ istd,
                                    __nv_bfloat16* X, __nv_bfloat16* Xt, float* F) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float f[kSurFeat];
  sur_features_raw(qpos, qvel, ctrl, cf, (size_t)n, e, f);
  for (int k = 0; k < kSurIn; ++k) {
    const float raw = k < kSurFeat ? f[k] : 0.0f;
    if (F) F[(size_t)e * kSurIn + k] = raw;
    const float x = k < kSurFeat ? (raw - mean[k]) * istd[k] : 0.0f;
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    X[(size_t)e * kSurIn + k] = h;
    if (Xt) Xt[(size_t)k * n + e] = h;
  }
}

// One surrogate step in place: qacc = Y[e][0:35] * ostd + omean, then the
// step's semi-implicit Euler (qvel += dt qacc; qpos from the new qvel, the
// base quaternion by q (x) exp(w dt / 2)).  Anchors are left free.
__global__ void sur_integrate_kernel(int n, const float* __restrict__ Y, int ldy, const float* __restrict__ omean,
                                     const float* __restrict__ ostd, float dt, float* qpos, float* qvel) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const size_t sn = (size_t)n;
  for (int i = 0; i < kNV; ++i) {
    const float a = Y[(size_t)e * ldy + i] * ostd[i] + omean[i];
    qvel[i * sn + e] += dt * a;
  }
  for (int i = 0; i < 3; ++i) qpos[i * sn + e] += dt * qvel[i * sn + e];
  const float wx = qvel[3 * sn + e], wy = qvel[4 * sn + e], wz = qvel[5 * sn + e];
  const float wn = sqrtf(wx * wx + wy * wy + wz * wz);
  const float ang = wn * dt;
  if (ang >= 1e-12f) {
    const float s = sinf(0.5f * ang) / wn, c = cosf(0.5f * ang);
    const float dx = s * wx, dy = s * wy, dz = s * wz;
    const float aw = qpos[3 * sn + e], ax = qpos[4 * sn + e], ay = qpos[5 * sn + e], az = qpos[6 * sn + e];
    float rw = aw * c - ax * dx - ay * dy - az * dz;
    float rx = aw * dx + ax * c + ay * dz - az * dy;
    float ry = aw * dy - ax * dz + ay * c + az * dx;
    float rz = aw * dz + ax * dy - ay * dx + az * c;
    const float inv = 1.0f / sqrtf(rw * rw + rx * rx + ry * ry + rz * rz);
    qpos[3 * sn + e] = rw * inv;
    qpos[4 * sn + e] = rx * inv;
    qpos[5 * sn + e] = ry * inv;
    qpos[6 * sn + e] = rz * inv;
  }
  for (int h = 0; h < 29; ++h) qpos[(7 + h) * sn + e] += dt * qvel[(6 + h) * sn + e];
}
