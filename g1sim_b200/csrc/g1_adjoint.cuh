// g1_adjoint.cuh -- gradient of a horizon loss through the G1 step
// (included by g1_kernels.cu inside namespace g1b).
//
// Problem (one env per row, H steps of one substep each):
//   x_{t+1} = step(x_t, u_t, kp_scale, kd_scale),  x = (qpos 36, qvel 35, anchor 16)
//   L = sum_{t=1..H} (z_t - z_ref)^2 + w_track * |q_t - u_{t-1}|^2
// with z the base height qpos[2] and q the 29 joint angles qpos[7:36].
// Outputs L, dL/du_t (H x 29), dL/dkp_scale, dL/dkd_scale and dL/dx_0.
//
// Reverse sweep with checkpoints: the forward rollout keeps x_t every C
// steps; the backward sweep recomputes each segment of C states from its
// checkpoint and walks it backwards with the adjoint state
//   lambda_t = (dx_{t+1}/dx_t)^T lambda_{t+1} + dL/dx_t.
// The vector-Jacobian product of one step is assembled from forward-mode
// tangents: the step runs on Dual<R, 4> numbers seeded with 4 of the 118
// input directions (state 87, targets 29, two gain scales) and the output
// tangents are contracted with lambda_{t+1}; 30 threads per env cover the
// 118 directions in parallel.  Exact to rounding (the derivative of the
// step as computed, the branch taken at each switch).
//
// Scratch (caller-provided, R = float or double), SoA [slot][nenv]:
//   checkpoints (ceil(H / C) + 1) x 87, segment C x 87, lambda 87, G 120.

constexpr int kAdjState = 87;   // qpos 36, qvel 35, anchor 16
constexpr int kAdjDirs = 118;   // state 87, targets 29, kp_scale, kd_scale
constexpr int kAdjK = 4;        // tangent directions per thread
constexpr int kAdjBlocks = (kAdjDirs + kAdjK - 1) / kAdjK;
constexpr int kAdjG = kAdjBlocks * kAdjK;

template <class R>
struct AdjArgs {
  int n, H, C, S;  // envs, horizon, checkpoint interval, segments
  tg::CfgT<R> cfg;
  const R *qpos0, *qvel0, *anchor0, *targets, *kp, *kd;
  R z_ref, w_track;
  R *loss, *gtar, *gkp, *gkd, *gq0, *gv0;
  R *ck, *seg, *lam, *G;
};

template <class R>
__host__ __device__ inline size_t adj_scratch_count(int n, int H, int C) {
  const int S = (H + C - 1) / C;
  return (size_t)n * ((size_t)(S + 1) * kAdjState + (size_t)C * kAdjState + kAdjState + kAdjG);
}

template <class T>
__device__ __forceinline__ void adj_load(T* x, const typename tg::Real<T>::type* base, int n, int e) {
#pragma unroll 1
  for (int i = 0; i < kAdjState; ++i) x[i] = T(base[(size_t)i * n + e]);
}
template <class R>
__device__ __forceinline__ void adj_store(const R* x, R* base, int n, int e) {
#pragma unroll 1
  for (int i = 0; i < kAdjState; ++i) base[(size_t)i * n + e] = x[i];
}
// dL/dx_t of the terms at x_t (t >= 1), added into g; u: targets of step t-1
template <class R>
__device__ __forceinline__ void adj_loss_grad(const R* x, const R* u_prev, int n, int e, R z_ref, R w, R* g) {
  g[2] += R(2) * (x[2] - z_ref);
#pragma unroll 1
  for (int j = 0; j < tg::kNU; ++j) g[7 + j] += R(2) * w * (x[7 + j] - u_prev[(size_t)j * n + e]);
}

// Forward rollout: loss, checkpoints, lambda_H; zero the gain gradients.
template <class R>
__global__ void __launch_bounds__(128) adj_forward_kernel(AdjArgs<R> a) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  const int n = a.n;
  R x[kAdjState], u[tg::kNU];
  tg::Work<R> w;
#pragma unroll 1
  for (int i = 0; i < 36; ++i) x[i] = a.qpos0[(size_t)i * n + e];
#pragma unroll 1
  for (int i = 0; i < 35; ++i) x[36 + i] = a.qvel0[(size_t)i * n + e];
#pragma unroll 1
  for (int i = 0; i < 16; ++i) x[71 + i] = a.anchor0[(size_t)i * n + e];
  const R kp = a.kp ? a.kp[e] : R(1), kd = a.kd ? a.kd[e] : R(1);
  R loss = R(0);
#pragma unroll 1
  for (int t = 0; t < a.H; ++t) {
    if (t % a.C == 0) adj_store(x, a.ck + (size_t)(t / a.C) * kAdjState * n, n, e);
    const R* ut = a.targets + (size_t)t * tg::kNU * n;
#pragma unroll 1
    for (int j = 0; j < tg::kNU; ++j) u[j] = ut[(size_t)j * n + e];
    tg::step<R>(a.cfg, x, x + 36, x + 71, u, kp, kd, R(1), R(0), w);
    R l = (x[2] - a.z_ref) * (x[2] - a.z_ref), tr = R(0);
#pragma unroll 1
    for (int j = 0; j < tg::kNU; ++j) tr += (x[7 + j] - u[j]) * (x[7 + j] - u[j]);
    loss += l + a.w_track * tr;
  }
  adj_store(x, a.ck + (size_t)a.S * kAdjState * n, n, e);
  a.loss[e] = loss;
  R g[kAdjState];
#pragma unroll 1
  for (int i = 0; i < kAdjState; ++i) g[i] = R(0);
  adj_loss_grad(x, a.targets + (size_t)(a.H - 1) * tg::kNU * n, n, e, a.z_ref, a.w_track, g);
  adj_store(g, a.lam, n, e);
  if (a.gkp) a.gkp[e] = R(0);
  if (a.gkd) a.gkd[e] = R(0);
}

// Recompute the states of segment s from its checkpoint into seg[0..len).
template <class R>
__global__ void __launch_bounds__(128) adj_segment_kernel(AdjArgs<R> a, int s) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  const int n = a.n, t0 = s * a.C;
  const int len = a.H - t0 < a.C ? a.H - t0 : a.C;
  R x[kAdjState], u[tg::kNU];
  tg::Work<R> w;
  adj_load(x, a.ck + (size_t)s * kAdjState * n, n, e);
  const R kp = a.kp ? a.kp[e] : R(1), kd = a.kd ? a.kd[e] : R(1);
#pragma unroll 1
  for (int i = 0; i < len; ++i) {
    adj_store(x, a.seg + (size_t)i * kAdjState * n, n, e);
    if (i + 1 == len) break;
    const R* ut = a.targets + (size_t)(t0 + i) * tg::kNU * n;
#pragma unroll 1
    for (int j = 0; j < tg::kNU; ++j) u[j] = ut[(size_t)j * n + e];
    tg::step<R>(a.cfg, x, x + 36, x + 71, u, kp, kd, R(1), R(0), w);
  }
}

// G[d] = lambda_{t+1} . d x_{t+1} / d(input d) for this thread's kAdjK
// directions d = blockIdx.y * kAdjK + k, at state seg[i] = x_t.
template <class R>
__global__ void __launch_bounds__(64) adj_vjp_kernel(AdjArgs<R> a, int t, int i) {
  using D = tg::Dual<R, kAdjK>;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  const int n = a.n, d0 = blockIdx.y * kAdjK;
  D x[kAdjState], u[tg::kNU];
  tg::Work<D> w;
  adj_load(x, a.seg + (size_t)i * kAdjState * n, n, e);
  const R* ut = a.targets + (size_t)t * tg::kNU * n;
#pragma unroll 1
  for (int j = 0; j < tg::kNU; ++j) u[j] = D(ut[(size_t)j * n + e]);
  D kp(a.kp ? a.kp[e] : R(1)), kd(a.kd ? a.kd[e] : R(1));
#pragma unroll
  for (int k = 0; k < kAdjK; ++k) {
    const int d = d0 + k;
    if (d < kAdjState)
      x[d].d[k] = R(1);
    else if (d < kAdjState + tg::kNU)
      u[d - kAdjState].d[k] = R(1);
    else if (d == kAdjState + tg::kNU)
      kp.d[k] = R(1);
    else if (d == kAdjState + tg::kNU + 1)
      kd.d[k] = R(1);
  }
  tg::step<D>(a.cfg, x, x + 36, x + 71, u, kp, kd, R(1), R(0), w);
  R g[kAdjK];
#pragma unroll
  for (int k = 0; k < kAdjK; ++k) g[k] = R(0);
#pragma unroll 1
  for (int s = 0; s < kAdjState; ++s) {
    const R l = a.lam[(size_t)s * n + e];
#pragma unroll
    for (int k = 0; k < kAdjK; ++k) g[k] += l * x[s].d[k];
  }
#pragma unroll
  for (int k = 0; k < kAdjK; ++k) a.G[(size_t)(d0 + k) * n + e] = g[k];
}

// lambda_t, dL/du_t and the gain gradients from G; t = t0 + i of segment s.
template <class R>
__global__ void __launch_bounds__(128) adj_accum_kernel(AdjArgs<R> a, int t, int i, int s) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.n) return;
  const int n = a.n, t0 = s * a.C;
  const int len = a.H - t0 < a.C ? a.H - t0 : a.C;
  R g[kAdjState], x[kAdjState];
#pragma unroll 1
  for (int k = 0; k < kAdjState; ++k) g[k] = a.G[(size_t)k * n + e];
  // dL/du_t = G_u - 2 w (q_{t+1} - u_t)
  const R* x1 = (i + 1 < len) ? a.seg + (size_t)(i + 1) * kAdjState * n : a.ck + (size_t)(s + 1) * kAdjState * n;
  const R* ut = a.targets + (size_t)t * tg::kNU * n;
  R* gt = a.gtar + (size_t)t * tg::kNU * n;
#pragma unroll 1
  for (int j = 0; j < tg::kNU; ++j) {
    const R q1 = x1[(size_t)(7 + j) * n + e];
    gt[(size_t)j * n + e] = a.G[(size_t)(kAdjState + j) * n + e] - R(2) * a.w_track * (q1 - ut[(size_t)j * n + e]);
  }
  if (a.gkp) a.gkp[e] += a.G[(size_t)(kAdjState + tg::kNU) * n + e];
  if (a.gkd) a.gkd[e] += a.G[(size_t)(kAdjState + tg::kNU + 1) * n + e];
  if (t >= 1) {
    adj_load(x, a.seg + (size_t)i * kAdjState * n, n, e);
    adj_loss_grad(x, a.targets + (size_t)(t - 1) * tg::kNU * n, n, e, a.z_ref, a.w_track, g);
  } else {
    if (a.gq0)
      for (int k = 0; k < 36; ++k) a.gq0[(size_t)k * n + e] = g[k];
    if (a.gv0)
      for (int k = 0; k < 35; ++k) a.gv0[(size_t)k * n + e] = g[36 + k];
  }
  adj_store(g, a.lam, n, e);
}

// The whole sweep on one stream.
template <class R>
cudaError_t adj_launch(const AdjArgs<R>& a, cudaStream_t st) {
  const dim3 b128(128), g128((a.n + 127) / 128);
  adj_forward_kernel<R><<<g128, b128, 0, st>>>(a);
  for (int s = a.S - 1; s >= 0; --s) {
    adj_segment_kernel<R><<<g128, b128, 0, st>>>(a, s);
    const int t0 = s * a.C;
    const int len = a.H - t0 < a.C ? a.H - t0 : a.C;
    for (int i = len - 1; i >= 0; --i) {
      adj_vjp_kernel<R><<<dim3((a.n + 63) / 64, kAdjBlocks), dim3(64), 0, st>>>(a, t0 + i, i);
      adj_accum_kernel<R><<<g128, b128, 0, st>>>(a, t0 + i, i, s);
    }
  }
  return cudaGetLastError();
}
