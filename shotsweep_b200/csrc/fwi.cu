// Full-waveform inversion by L-BFGS, batched over models, on the device.
//
// The iteration of the reference's FWI (archive/toy/slopes/fwi.py:130-164)
// for many independent models at once: the gradient (the library's adjoint
// kernel, summed over shots) is preconditioned by a mute of the top rows and a
// separable Gaussian smoothing (fwi.py:142-143, slopes.py:20-26); the
// direction comes from the two-loop recursion over the last `mem` (s, y)
// pairs (fwi.py:130-136), capped to 50 m/s on the first step and replaced by
// scaled steepest descent when it is not a descent direction (fwi.py:150-151);
// trial models are clipped to [lo, hi] (fwi.py:154); accepted steps push their
// (s, y) pair when s.y > 1e-12 (fwi.py:160-161).  One CTA per model; dot
// products accumulate in float64, as the reference's NumPy does.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/shotsweep.h"
#include "internal.h"

namespace {

using ss_internal::fail;

constexpr int kThreads = 256;
constexpr int kMaxRadius = 32;

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w];
  __syncthreads();
  return s;
}

__device__ float block_max(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float s = 0.f;
  for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s = fmaxf(s, red[w]);
  __syncthreads();
  return s;
}

struct PrecondParams {
  const float* grads;   // [B][S][nz][nx]
  int S, nz, nx, radius, mute_rows;
  float kernel[2 * kMaxRadius + 1];
  float* out;           // [B][nz][nx]
};

// out = mute * smooth_x(smooth_z(mute * sum_s grads)), edge padding (slopes.py:20-26)
__global__ void __launch_bounds__(kThreads) precond_kernel(const PrecondParams P) {
  extern __shared__ float sm[];
  const int n = P.nz * P.nx;
  float* a = sm;
  float* b = sm + n;
  const int m = blockIdx.x;
  auto mute = [&](int z) { return fminf(fmaxf((z - 1) / 3.f, 0.f), 1.f); };   // fwi.py:142
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < P.S; ++k) s += P.grads[(static_cast<size_t>(m) * P.S + k) * n + i];
    a[i] = s * mute(i / P.nx);
  }
  __syncthreads();
  const int r = P.radius;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {   // along z
    const int z = i / P.nx, x = i - z * P.nx;
    float acc = 0.f;
    for (int j = 0; j <= 2 * r; ++j) acc += P.kernel[j] * a[min(max(z + j - r, 0), P.nz - 1) * P.nx + x];
    b[i] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {   // along x
    const int z = i / P.nx, x = i - z * P.nx;
    float acc = 0.f;
    for (int j = 0; j <= 2 * r; ++j) acc += P.kernel[j] * b[z * P.nx + min(max(x + j - r, 0), P.nx - 1)];
    P.out[static_cast<size_t>(m) * n + i] = acc * mute(z);
  }
}

// J[m] = 0.5 sum (sim - obs)^2 over the model's traces
__global__ void __launch_bounds__(kThreads) misfit_kernel(const float* __restrict__ sim, const float* __restrict__ obs,
                                                          int64_t per, double* __restrict__ J) {
  __shared__ double red[kThreads / 32];
  const int m = blockIdx.x;
  const float* s = sim + static_cast<size_t>(m) * per;
  const float* o = obs + static_cast<size_t>(m) * per;
  double acc = 0;
  for (int64_t i = threadIdx.x; i < per; i += blockDim.x) {
    const double d = static_cast<double>(s[i]) - o[i];
    acc += d * d;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) J[m] = 0.5 * acc;
}

struct LbfgsParams {
  const float* g;       // [B][n]
  const float* S;       // [B][mem][n]
  const float* Y;
  int* count;           // [B] pairs held (reset to 0 on a steepest-descent restart)
  const int* next;      // [B] slot of the next pair
  const int* active;    // [B]
  int n, mem;
  float cap;
  float* d;             // [B][n] out
  double* gd;           // [B] out: g . d
};

__global__ void __launch_bounds__(kThreads) lbfgs_direction_kernel(const LbfgsParams P) {
  __shared__ double red[kThreads / 32];
  __shared__ float redf[kThreads / 32];
  __shared__ double alpha[16], rho[16];
  const int m = blockIdx.x;
  if (!P.active[m]) return;
  const int n = P.n;
  const float* g = P.g + static_cast<size_t>(m) * n;
  float* q = P.d + static_cast<size_t>(m) * n;
  const int cnt = P.count[m], nx = P.next[m];
  auto slot = [&](int j) { return ((nx - cnt + j) % P.mem + P.mem) % P.mem; };   // j = 0 oldest .. cnt-1 newest
  auto Sv = [&](int j) { return P.S + (static_cast<size_t>(m) * P.mem + slot(j)) * n; };
  auto Yv = [&](int j) { return P.Y + (static_cast<size_t>(m) * P.mem + slot(j)) * n; };
  for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = g[i];
  __syncthreads();
  for (int j = cnt - 1; j >= 0; --j) {   // newest first (fwi.py:132-133)
    const float *s = Sv(j), *y = Yv(j);
    double ys = 0, sq = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      ys += static_cast<double>(y[i]) * s[i];
      sq += static_cast<double>(s[i]) * q[i];
    }
    ys = block_sum(ys, red);
    sq = block_sum(sq, red);
    const double r = 1.0 / ys, a = r * sq;
    if (threadIdx.x == 0) {
      rho[j] = r;
      alpha[j] = a;
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = static_cast<float>(q[i] - a * y[i]);
    __syncthreads();
  }
  if (cnt > 0) {   // initial Hessian scaling s.y / y.y of the newest pair (fwi.py:134)
    const float *s = Sv(cnt - 1), *y = Yv(cnt - 1);
    double sy = 0, yy = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      sy += static_cast<double>(s[i]) * y[i];
      yy += static_cast<double>(y[i]) * y[i];
    }
    sy = block_sum(sy, red);
    yy = block_sum(yy, red);
    const double sc = sy / yy;
    for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = static_cast<float>(q[i] * sc);
    __syncthreads();
  }
  for (int j = 0; j < cnt; ++j) {        // oldest first (fwi.py:135)
    const float *s = Sv(j), *y = Yv(j);
    double yq = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) yq += static_cast<double>(y[i]) * q[i];
    yq = block_sum(yq, red);
    const double b = rho[j] * yq, a = alpha[j];
    for (int i = threadIdx.x; i < n; i += blockDim.x) q[i] = static_cast<float>(q[i] + s[i] * (a - b));
    __syncthreads();
  }
  // d = -q; capped first step; steepest descent when not a descent direction (fwi.py:136,150-151)
  float mx = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmaxf(mx, fabsf(q[i]));
  mx = block_max(mx, redf);
  const float f = cnt == 0 ? -P.cap / (mx + 1e-30f) : -1.f;
  double dg = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    q[i] *= f;
    dg += static_cast<double>(q[i]) * g[i];
  }
  dg = block_sum(dg, red);
  if (dg >= 0) {
    float gm = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) gm = fmaxf(gm, fabsf(g[i]));
    gm = block_max(gm, redf);
    const float h = -P.cap / (gm + 1e-30f);
    dg = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      q[i] = g[i] * h;
      dg += static_cast<double>(q[i]) * g[i];
    }
    dg = block_sum(dg, red);
    if (threadIdx.x == 0) P.count[m] = 0;
  }
  if (threadIdx.x == 0) P.gd[m] = dg;
}

// vt = clip(v + step[m] d, lo, hi) for models with mask[m]
__global__ void trial_kernel(const float* __restrict__ v, const float* __restrict__ d, const float* __restrict__ step,
                             const int* __restrict__ mask, int B, int n, float lo, float hi, float* __restrict__ vt) {
  const int64_t total = static_cast<int64_t>(B) * n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int m = static_cast<int>(i / n);
    if (mask[m]) vt[i] = fminf(fmaxf(v[i] + step[m] * d[i], lo), hi);
  }
}

// For accepted models: push (vt - v, gn - g) when s.y > 1e-12, then v = vt, g = gn.
__global__ void __launch_bounds__(kThreads) lbfgs_push_kernel(float* __restrict__ v, const float* __restrict__ vt,
                                                              float* __restrict__ g, const float* __restrict__ gn,
                                                              float* __restrict__ S, float* __restrict__ Y,
                                                              int* __restrict__ count, int* __restrict__ next,
                                                              const int* __restrict__ accept, int n, int mem) {
  __shared__ double red[kThreads / 32];
  const int m = blockIdx.x;
  if (!accept[m]) return;
  const size_t base = static_cast<size_t>(m) * n;
  float* s = S + (static_cast<size_t>(m) * mem + next[m]) * n;
  float* y = Y + (static_cast<size_t>(m) * mem + next[m]) * n;
  double sy = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float si = vt[base + i] - v[base + i], yi = gn[base + i] - g[base + i];
    s[i] = si;
    y[i] = yi;
    sy += static_cast<double>(si) * yi;
  }
  sy = block_sum(sy, red);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    v[base + i] = vt[base + i];
    g[base + i] = gn[base + i];
  }
  if (threadIdx.x == 0 && sy > 1e-12) {
    next[m] = (next[m] + 1) % mem;
    count[m] = min(count[m] + 1, mem);
  }
}

int grid_for_f(long long total) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
}

}  // namespace

extern "C" {

int32_t ss_fwi_precondition(const float* grads, int32_t B, int32_t S, int32_t nz, int32_t nx, float smooth, float* out,
                            void* stream) {
  ss_internal::clear_error();
  if (!grads || !out || B < 0 || S < 1 || nz < 1 || nx < 1 || !(smooth >= 0.f)) return fail(SS_ERR_INVALID, "bad arguments");
  if (B == 0) return SS_OK;
  PrecondParams P{};
  P.grads = grads;
  P.S = S;
  P.nz = nz;
  P.nx = nx;
  P.out = out;
  if (smooth > 0.f) {   // slopes.py:21-22: radius int(3 s) + 1, normalised exp(-x^2 / 2s^2)
    P.radius = static_cast<int>(3 * smooth) + 1;
    if (P.radius > kMaxRadius) return fail(SS_ERR_UNSUPPORTED, "smoothing radius above 32 cells");
    std::vector<double> k(2 * P.radius + 1);
    double sum = 0;
    for (int j = -P.radius; j <= P.radius; ++j) sum += (k[j + P.radius] = std::exp(-0.5 * (j / static_cast<double>(smooth)) * (j / static_cast<double>(smooth))));
    for (int j = 0; j <= 2 * P.radius; ++j) P.kernel[j] = static_cast<float>(k[j] / sum);
  } else {
    P.radius = 0;
    P.kernel[0] = 1.f;
  }
  const size_t smem = 2 * static_cast<size_t>(nz) * nx * sizeof(float);
  if (smem > 200 * 1024) return fail(SS_ERR_UNSUPPORTED, "model too large for the preconditioner");
  if (smem > 48 * 1024)
    SS_TRY_CUDA(cudaFuncSetAttribute(precond_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  precond_kernel<<<B, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(P);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_fwi_misfit(const float* sim, const float* obs, int32_t B, int64_t per_model, double* J, void* stream) {
  ss_internal::clear_error();
  if (!sim || !obs || !J || B < 0 || per_model < 1) return fail(SS_ERR_INVALID, "bad arguments");
  if (B == 0) return SS_OK;
  misfit_kernel<<<B, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(sim, obs, per_model, J);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_lbfgs_direction(const float* g, const float* S, const float* Y, int32_t* count, const int32_t* next,
                           const int32_t* active, int32_t B, int32_t n, int32_t mem, float cap, float* d, double* gd,
                           void* stream) {
  ss_internal::clear_error();
  if (!g || !S || !Y || !count || !next || !active || !d || !gd || B < 0 || n < 1 || mem < 1 || mem > 16 || !(cap > 0.f))
    return fail(SS_ERR_INVALID, "bad arguments");
  if (B == 0) return SS_OK;
  LbfgsParams P{g, S, Y, count, next, active, n, mem, cap, d, gd};
  lbfgs_direction_kernel<<<B, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(P);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_fwi_trial(const float* v, const float* d, const float* step, const int32_t* mask, int32_t B, int32_t n,
                     float lo, float hi, float* vt, void* stream) {
  ss_internal::clear_error();
  if (!v || !d || !step || !mask || !vt || B < 0 || n < 1 || !(lo < hi)) return fail(SS_ERR_INVALID, "bad arguments");
  if (B == 0) return SS_OK;
  trial_kernel<<<grid_for_f(static_cast<long long>(B) * n), 256, 0, static_cast<cudaStream_t>(stream)>>>(v, d, step, mask,
                                                                                                     B, n, lo, hi, vt);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_lbfgs_push(float* v, const float* vt, float* g, const float* gn, float* S, float* Y, int32_t* count,
                      int32_t* next, const int32_t* accept, int32_t B, int32_t n, int32_t mem, void* stream) {
  ss_internal::clear_error();
  if (!v || !vt || !g || !gn || !S || !Y || !count || !next || !accept || B < 0 || n < 1 || mem < 1 || mem > 16)
    return fail(SS_ERR_INVALID, "bad arguments");
  if (B == 0) return SS_OK;
  lbfgs_push_kernel<<<B, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(v, vt, g, gn, S, Y, count, next, accept, n, mem);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

}  // extern "C"
