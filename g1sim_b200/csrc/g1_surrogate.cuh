// g1_surrogate.cuh -- kernels of the learned one-step dynamics surrogate
// (included by g1_surrogate.cu inside namespace g1b, after g1_gemm.cuh).
//
// The surrogate is an MLP 192 -> 512 -> 512 -> 512 -> 512 -> 64 with SiLU on
// the hidden layers, over a normalised feature vector of the state and the
// PD targets (g1_surfeat.cuh), predicting the normalised generalised
// acceleration of the step (the state delta is dt * qacc for qvel, and qpos
// follows by the step's own semi-implicit Euler).  The feature and update
// kernels also have their vector-Jacobian products, so that a loss can be
// differentiated through a surrogate rollout.  Its matrix products run on gemm_kernel
// (tcgen05); the element-wise parts of the forward and backward passes, the
// loss, Adam and the feature extraction are the kernels below.

using sur::kSurFeat;
using sur::kSurIn;
constexpr int kSurOut = 64;  // padded outputs (35 used: qacc)

// silu and silu_grad: g1_gemm.cuh (its fused epilogues use them too).

// Weighted MSE over the output columns: loss += sum_r sum_c w[c] (Y - T)^2 / B;
// dY = 2 w[c] (Y - T) / B as BF16 [B][D] and transposed [D][B]; db[c] += the
// column sums of the FP32 gradient.  One block per 128 rows, D dividing the
// 256 threads so that each thread keeps one column: the row-major arrays are
// read and written column-fastest (coalesced), the gradient tile is staged in
// shared memory ([128][D + 2], conflict-free both ways) for the transposed
// copy, and each block adds one partial sum per column and one loss term.
constexpr int kLossRows = 128, kLossThreads = 256;
__global__ void __launch_bounds__(kLossThreads) sur_loss_kernel(int B, int D, const float* __restrict__ Y,
                                                                const float* __restrict__ T,
                                                                const float* __restrict__ w, __nv_bfloat16* dY,
                                                                __nv_bfloat16* dYt, float* db, float* loss) {
  extern __shared__ __nv_bfloat16 tile[];  // [kLossRows][D + 2]
  __shared__ float red[kLossThreads];
  __shared__ float lred[kLossThreads / 32];
  const int r0 = blockIdx.x * kLossRows;
  const int rows = B - r0 < kLossRows ? B - r0 : kLossRows;
  const int ld = D + 2;
  // the thread's column is fixed (D divides the block) and its rows step by
  // kLossThreads / D: row r_t, r_t + rpp, ...
  const int c = threadIdx.x % D, r_t = threadIdx.x / D, rpp = kLossThreads / D;
  const float wc = w[c];
  float acc = 0.0f, l = 0.0f;
  // eight rows' loads in flight per thread before their arithmetic
  for (int rb = r_t; rb < rows; rb += 8 * rpp) {
    float e[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = rb + u * rpp;
      const size_t gi = (size_t)(r0 + r) * D + c;
      e[u] = r < rows ? Y[gi] - T[gi] : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int r = rb + u * rpp;
      if (r >= rows) continue;
      l += wc * e[u] * e[u];
      const float g = 2.0f * wc * e[u] / (float)B;
      acc += g;
      const __nv_bfloat16 gb = __float2bfloat16_rn(g);
      dY[(size_t)(r0 + r) * D + c] = gb;
      if (dYt) tile[r * ld + c] = gb;
    }
  }
  red[threadIdx.x] = acc;
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) lred[threadIdx.x >> 5] = l;
  __syncthreads();
  // transposed copy (dYt nullable), eight consecutive rows of one column
  // (16 bytes) per store where a full, 16-byte aligned group of eight rows exists
  const bool vec = (B & 7) == 0 && (reinterpret_cast<uintptr_t>(dYt) & 15) == 0;
  const int groups = vec ? rows / 8 : 0;
  const int tail = dYt ? rows - 8 * groups : 0;
  for (int i = threadIdx.x; dYt && i < D * groups; i += kLossThreads) {
    const int cc = i / groups, r = (i - cc * groups) * 8;
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = tile[(r + u) * ld + cc];
    *reinterpret_cast<uint4*>(dYt + (size_t)cc * B + r0 + r) = *reinterpret_cast<const uint4*>(v);
  }
  for (int i = threadIdx.x; i < D * tail; i += kLossThreads) {
    const int cc = i / tail, r = 8 * groups + i % tail;
    dYt[(size_t)cc * B + r0 + r] = tile[r * ld + cc];
  }
  if (threadIdx.x < D) {
    float sum = 0.0f;
    for (int k = threadIdx.x; k < kLossThreads; k += D) sum += red[k];
    atomicAdd(db + threadIdx.x, sum);
  }
  if (threadIdx.x == 0) {
    float ls = 0.0f;
    for (int k = 0; k < kLossThreads / 32; ++k) ls += lred[k];
    atomicAdd(loss, ls / (float)B);
  }
}

// The optimiser step of every layer in one launch: Adam on the FP32
// weights and biases (moments m, v; bias corrections 1 - b1^t, 1 - b2^t for
// the step count t and the learning rate read from device memory, so that a
// captured CUDA graph of the training step replays with the current ones),
// then the BF16 copy and BF16 transpose of each updated weight that the
// GEMMs read.  Each block of kAdamThreads owns one kAdamRows x kAdamCols
// tile of one layer's weight (row-major reads and writes, one 128-byte
// line per warp instruction) and writes the tile's transpose from shared
// memory as 16-byte runs of eight rows; the blocks after the last tile
// update the biases, one entry per thread, the layers' biases in order.
constexpr int kAdamRows = 32, kAdamCols = 64, kAdamThreads = 256;
static_assert(kAdamCols * (kAdamRows / 8) == kAdamThreads && kAdamCols == 64 && kAdamThreads == 256,
              "a warp's entries: 8 rows x 2 x 32 columns; one column's eight-row run per thread");
struct SurLayerOpt {
  float *W, *b, *mW, *vW, *mb, *vb;
  const float *gW, *gb;
  __nv_bfloat16 *Wb, *Wt;
  int rows, cols;
};
constexpr int kSurMaxLayers = 8;
struct SurOpt {
  SurLayerOpt l[kSurMaxLayers];
  int tile0[kSurMaxLayers + 1];  // first block of each layer's tiles; tile0[nl]: the first bias block
  int nl;
  const int* step;
  const float* lr;
  float b1, b2, eps;
};

__device__ __forceinline__ float adam_update(float& p, float& m, float& v, float g, float lr, float b1, float b2,
                                             float eps, float c1, float c2) {
  const float mi = b1 * m + (1.0f - b1) * g;
  const float vi = b2 * v + (1.0f - b2) * g * g;
  m = mi;
  v = vi;
  p -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  return p;
}

__global__ void __launch_bounds__(kAdamThreads) sur_adam_cast_kernel(SurOpt o) {
  // the tile transposed: 34 values (17 words) per column, so the warps'
  // column-wise writes fall in distinct banks
  __shared__ __align__(16) __nv_bfloat16 tr[kAdamCols][kAdamRows + 2];
  const float t = (float)*o.step, lr = *o.lr;
  const float c1 = 1.0f - powf(o.b1, t), c2 = 1.0f - powf(o.b2, t);
  const int blk = blockIdx.x;
  if (blk >= o.tile0[o.nl]) {
    int k = (blk - o.tile0[o.nl]) * kAdamThreads + threadIdx.x;
    for (int L = 0; L < o.nl; ++L) {
      const SurLayerOpt& q = o.l[L];
      if (k < q.rows) {
        adam_update(q.b[k], q.mb[k], q.vb[k], q.gb[k], lr, o.b1, o.b2, o.eps, c1, c2);
        break;
      }
      k -= q.rows;
    }
    return;
  }
  int L = 0;
  while (blk >= o.tile0[L + 1]) ++L;
  const SurLayerOpt& q = o.l[L];
  const int tcols = (q.cols + kAdamCols - 1) / kAdamCols;
  const int r0 = ((blk - o.tile0[L]) / tcols) * kAdamRows, c0 = ((blk - o.tile0[L]) % tcols) * kAdamCols;
  // entry e of this thread: row warp + 8 (e / 2), column lane + 32 (e % 2); every
  // load is issued before the first store (the stores could alias the loads
  // of a later entry, so the compiler would not hoist them by itself)
  constexpr int kPer = kAdamRows * kAdamCols / kAdamThreads;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float w[kPer], m[kPer], v[kPer], gr[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int r = r0 + warp + 8 * (e >> 1), c = c0 + lane + 32 * (e & 1);
    const bool in = r < q.rows && c < q.cols;
    const size_t k = in ? (size_t)r * q.cols + c : 0;
    w[e] = in ? q.W[k] : 0.0f;
    m[e] = in ? q.mW[k] : 0.0f;
    v[e] = in ? q.vW[k] : 0.0f;
    gr[e] = in ? q.gW[k] : 0.0f;
  }
#pragma unroll
  for (int e = 0; e < kPer; ++e) {
    const int rr = warp + 8 * (e >> 1), cc = lane + 32 * (e & 1), r = r0 + rr, c = c0 + cc;
    __nv_bfloat16 h = __float2bfloat16_rn(0.0f);
    if (r < q.rows && c < q.cols) {
      const size_t k = (size_t)r * q.cols + c;
      h = __float2bfloat16_rn(adam_update(w[e], m[e], v[e], gr[e], lr, o.b1, o.b2, o.eps, c1, c2));
      q.W[k] = w[e];
      q.mW[k] = m[e];
      q.vW[k] = v[e];
      q.Wb[k] = h;
    }
    tr[cc][rr] = h;
  }
  __syncthreads();
  const bool vec = r0 + kAdamRows <= q.rows && c0 + kAdamCols <= q.cols && (q.rows & 7) == 0 &&
                   (reinterpret_cast<uintptr_t>(q.Wt) & 15) == 0;
  if (vec) {  // thread: one column, eight rows
    const int cc = threadIdx.x >> 2, j = threadIdx.x & 3;
    const uint32_t* w = reinterpret_cast<const uint32_t*>(&tr[cc][8 * j]);
    *reinterpret_cast<uint4*>(q.Wt + (size_t)(c0 + cc) * q.rows + r0 + 8 * j) = make_uint4(w[0], w[1], w[2], w[3]);
  } else {
    for (int i = threadIdx.x; i < kAdamRows * kAdamCols; i += kAdamThreads) {
      const int cc = i / kAdamRows, rr = i % kAdamRows;
      if (r0 + rr < q.rows && c0 + cc < q.cols) q.Wt[(size_t)(c0 + cc) * q.rows + r0 + rr] = tr[cc][rr];
    }
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

// One env's state and targets as seen by the feature and update functions:
// the 87 state entries (qpos, qvel, anchors) over the SoA arrays.
struct SoAState {
  float* qpos;
  float* qvel;
  const float* anchor;
  size_t n;
  int e;
  __device__ __forceinline__ float get(int k) const {
    return k < kNQ ? qpos[(size_t)k * n + e]
                   : (k < kNQ + kNV ? qvel[(size_t)(k - kNQ) * n + e] : anchor[(size_t)(k - kNQ - kNV) * n + e]);
  }
  __device__ __forceinline__ void put(int k, float v) {
    if (k < kNQ)
      qpos[(size_t)k * n + e] = v;
    else if (k < kNQ + kNV)
      qvel[(size_t)(k - kNQ) * n + e] = v;
  }
};
struct SoACol {
  const float* p;
  size_t n;
  int e;
  __device__ __forceinline__ float get(int k) const { return p[(size_t)k * n + e]; }
};
// accumulating column of a SoA array (adjoints)
struct SoAAdd {
  float* p;
  size_t n;
  int e;
  __device__ __forceinline__ void add(int k, float v) { p[(size_t)k * n + e] += v; }
};
// adjoint of the 87 state entries over (qpos, qvel, anchor) SoA arrays; the
// anchors' adjoint is dropped when anchor is null
struct SoAStateAdd {
  float* qpos;
  float* qvel;
  float* anchor;
  size_t n;
  int e;
  __device__ __forceinline__ void add(int k, float v) {
    if (k < kNQ)
      qpos[(size_t)k * n + e] += v;
    else if (k < kNQ + kNV)
      qvel[(size_t)(k - kNQ) * n + e] += v;
    else if (anchor)
      anchor[(size_t)(k - kNQ - kNV) * n + e] += v;
  }
  __device__ __forceinline__ float get(int k) const {
    return k < kNQ ? qpos[(size_t)k * n + e] : qvel[(size_t)(k - kNQ) * n + e];
  }
  __device__ __forceinline__ void put(int k, float v) {
    if (k < kNQ)
      qpos[(size_t)k * n + e] = v;
    else if (k < kNQ + kNV)
      qvel[(size_t)(k - kNQ) * n + e] = v;
  }
};

// X[e][:] = BF16((f - mean) * istd), padded with zeros to kSurIn; Xt the
// transpose (nullable); raw features to F (FP32 [n][kSurIn], nullable).
// mu, dmass: per-env friction and base-mass offset (nullable: 1, 0).
__global__ void sur_features_kernel(int n, const float* qpos, const float* qvel, const float* anchor, const float* ctrl,
                                    const float* mu, const float* dmass, const float* __restrict__ mean,
                                    const float* __restrict__ istd, __nv_bfloat16* X, __nv_bfloat16* Xt, float* F) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float f[kSurFeat];
  const SoAState x{const_cast<float*>(qpos), const_cast<float*>(qvel), anchor, (size_t)n, e};
  sur::features<float>(x, SoACol{ctrl, (size_t)n, e}, mu ? mu[e] : (float)g1m_contact_mu, dmass ? dmass[e] : 0.0f, f);
  for (int k = 0; k < kSurIn; ++k) {
    const float raw = k < kSurFeat ? f[k] : 0.0f;
    if (F) F[(size_t)e * kSurIn + k] = raw;
    const float xv = k < kSurFeat ? (raw - mean[k]) * istd[k] : 0.0f;
    const __nv_bfloat16 h = __float2bfloat16_rn(xv);
    X[(size_t)e * kSurIn + k] = h;
    if (Xt) Xt[(size_t)k * n + e] = h;
  }
}

// Adjoint of the features: dX [n][ld] is the adjoint of the normalised
// inputs; the state adjoints (qpos_b [36][n], qvel_b [35][n], anchor_b
// [16][n] nullable) and the targets' (ctrl_b [29][n]) are accumulated.
__global__ void sur_feat_vjp_kernel(int n, const float* qpos, const float* qvel, const float* anchor,
                                    const float* __restrict__ istd, const float* __restrict__ dX, int ld,
                                    float* qpos_b, float* qvel_b, float* anchor_b, float* ctrl_b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float fb[kSurFeat];
  for (int k = 0; k < kSurFeat; ++k) fb[k] = dX[(size_t)e * ld + k] * istd[k];
  const SoAState x{const_cast<float*>(qpos), const_cast<float*>(qvel), anchor, (size_t)n, e};
  SoAStateAdd xb{qpos_b, qvel_b, anchor_b, (size_t)n, e};
  SoAAdd ub{ctrl_b, (size_t)n, e};
  sur::features_vjp<float>(x, fb, xb, ub);
}

// One surrogate step in place: qacc = Y[e][0:35] * ostd + omean, then the
// step's semi-implicit Euler (g1_surfeat.cuh).  Anchors are not touched.
__global__ void sur_integrate_kernel(int n, const float* __restrict__ Y, int ldy, const float* __restrict__ omean,
                                     const float* __restrict__ ostd, float dt, float* qpos, float* qvel) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float a[kNV];
  for (int i = 0; i < kNV; ++i) a[i] = Y[(size_t)e * ldy + i] * ostd[i] + omean[i];
  SoAState x{qpos, qvel, nullptr, (size_t)n, e};
  sur::integrate<float>(x, a, dt);
}

// Reverse of sur_integrate at the state before the update (qpos, qvel):
// lam_qpos [36][n], lam_qvel [35][n] hold the adjoint of the updated state
// and are replaced by the adjoint of the state through the update; dY
// [n][ldd] (FP32) gets the adjoint of the normalised network output (zero
// past the 35 used columns).
__global__ void sur_integrate_vjp_kernel(int n, const float* qpos, const float* qvel, const float* __restrict__ Y,
                                         int ldy, const float* __restrict__ omean, const float* __restrict__ ostd,
                                         float dt, float* lam_qpos, float* lam_qvel, float* dY, int ldd) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float a[kNV], ab[kNV];
  for (int i = 0; i < kNV; ++i) a[i] = Y[(size_t)e * ldy + i] * ostd[i] + omean[i];
  const SoAState x{const_cast<float*>(qpos), const_cast<float*>(qvel), nullptr, (size_t)n, e};
  SoAStateAdd lam{lam_qpos, lam_qvel, nullptr, (size_t)n, e};
  sur::integrate_vjp<float>(x, a, dt, lam, ab);
  for (int i = 0; i < ldd; ++i) dY[(size_t)e * ldd + i] = i < kNV ? ab[i] * ostd[i] : 0.0f;
}

// BF16 copy of an FP32 [B][D] adjoint (the seed of the network's input
// gradient chain).
__global__ void sur_seed_kernel(int total, const float* __restrict__ dY, __nv_bfloat16* dZ) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x)
    dZ[i] = __float2bfloat16_rn(dY[i]);
}
