// After the images: the per-model steps ShotSweep runs around the RTM images
// before training (openfwi/2_process.py, openfwi/physics/background.py,
// openfwi/3_train.py), as device kernels.
//
//   ss_surface_velocity  first-arrival onsets, short-offset line fits and their
//                        quality checks (background.py:19-83), one CTA per model
//   ss_backgrounds       slow / medium / fast laterally constant backgrounds
//                        (background.py:97-99)
//   ss_image_cache       zero the top rows, scale by the 99th percentile of |img|
//                        per model, clip to +-4, binary16 (2_process.py:206-210)
//   ss_signed_log1p_f16  sign(g) log1p(|g|) as binary16 (3_train.py:157)
//   ss_f16_scaled        binary16 inputs / scale in float32 (3_train.py:198)
//   ss_velocity_targets  (v - 3000) / 1500 and the clipped reference velocity
//                        (3_train.py:158,188-189)
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/shotsweep.h"
#include "internal.h"

namespace {

using ss_internal::fail;

int grid_for(long long total) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
}

// ----------------------------------------------------------------------------
// Image cache: exact order statistics by radix selection on the bit patterns
// of |img| (non-negative floats order like their bits), then numpy's linear
// interpolation in float32.
// ----------------------------------------------------------------------------
constexpr int kCacheThreads = 512;

struct CacheParams {
  const float* img;
  int n_images, nz, nx, zero_rows;
  long long prev, next;   // order statistics to interpolate (0-based, ascending)
  float gamma;            // float32 weight, as numpy computes it for float32 data
  float clip;
  uint16_t* out;
  float* scale;
  int* status;
};

__device__ __forceinline__ uint32_t abs_bits(const CacheParams& P, const float* im, long long i, int per_image) {
  const int z = static_cast<int>((i % per_image) / P.nx);
  if (z < P.zero_rows) return 0u;
  return __float_as_uint(im[i]) & 0x7fffffffu;
}

// k-th smallest (0-based) of the model's |values|, as bits.
__device__ uint32_t radix_select(const CacheParams& P, const float* im, long long n, long long k, uint32_t* hist,
                                 uint32_t* shared_word) {
  const int per_image = P.nz * P.nx;
  uint32_t prefix = 0, mask = 0;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t v = abs_bits(P, im, i, per_image);
      if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long acc = 0;
      int b = 0;
      for (; b < 256; ++b) {
        if (acc + hist[b] > k) break;
        acc += hist[b];
      }
      shared_word[0] = static_cast<uint32_t>(b);
      shared_word[1] = static_cast<uint32_t>(acc);   // values below this bucket (fits: n < 2^32)
    }
    __syncthreads();
    const uint32_t b = shared_word[0];
    k -= shared_word[1];
    prefix |= b << shift;
    mask |= 0xffu << shift;
    __syncthreads();
  }
  return prefix;
}

__global__ void __launch_bounds__(kCacheThreads) image_cache_kernel(const CacheParams P) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t word[4];
  __shared__ int bad;
  const int m = blockIdx.x;
  const int per_image = P.nz * P.nx;
  const long long n = static_cast<long long>(P.n_images) * per_image;
  const float* im = P.img + static_cast<size_t>(m) * n;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    if (!isfinite(im[i])) bad = 1;
  __syncthreads();
  if (bad) {   // 2_process raises on non-finite images; nothing is written for this model
    if (threadIdx.x == 0) {
      P.status[m] = SS_ERR_NONFINITE;
      P.scale[m] = NAN;
    }
    return;
  }
  const uint32_t lo_bits = radix_select(P, im, n, P.prev, hist, word);
  uint32_t hi_bits = lo_bits;
  if (P.next != P.prev) {
    // the next order statistic: lo again if it repeats, else the smallest value above it
    if (threadIdx.x == 0) {
      word[2] = 0;
      word[3] = 0xffffffffu;
    }
    __syncthreads();
    unsigned int le = 0, above = 0xffffffffu;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t v = abs_bits(P, im, i, per_image);
      if (v <= lo_bits) ++le;
      else above = min(above, v);
    }
    atomicAdd(&word[2], le);
    atomicMin(&word[3], above);
    __syncthreads();
    hi_bits = static_cast<long long>(word[2]) > P.next ? lo_bits : word[3];
  }
  // numpy _lerp in float32: a + (b - a) * t, or b - (b - a) * (1 - t) for t >= 0.5
  const float a = __uint_as_float(lo_bits), b = __uint_as_float(hi_bits);
  const float d = __fsub_rn(b, a);
  const float s = P.gamma >= 0.5f ? __fsub_rn(b, __fmul_rn(d, __fsub_rn(1.f, P.gamma)))
                                  : __fadd_rn(a, __fmul_rn(d, P.gamma));
  if (threadIdx.x == 0) {
    P.scale[m] = s;
    P.status[m] = (s > 0.f) ? SS_OK : SS_ERR_INVALID;
  }
  if (!(s > 0.f)) return;
  uint16_t* o = P.out + static_cast<size_t>(m) * n;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const int z = static_cast<int>((i % per_image) / P.nx);
    const float v = z < P.zero_rows ? 0.f : im[i];
    const float r = fminf(fmaxf(__fdiv_rn(v, s), -P.clip), P.clip);
    o[i] = __half_as_ushort(__float2half_rn(r));
  }
}

// ----------------------------------------------------------------------------
// Surface velocity from first-arrival onsets (background.py:19-83)
// ----------------------------------------------------------------------------
constexpr int kSurfThreads = 384;
constexpr int kMaxTraces = 3 * 1024;   // shared memory: 56 bytes per trace

struct SurfParams {
  const float* gathers;
  int n_shots, nt, nx;
  double src_x[SS_MAX_SHOTS];
  double dx, dt, frac;
  ss_surface_estimate* out;
};

// Least-squares line t = a + s h through n points (np.polyfit(h, t, 1)):
// returns s and the RMS residual.
__device__ void fit_line(const double* h, const double* t, int n, double* slope, double* rmse) {
  double hm = 0, tm = 0;
  for (int i = 0; i < n; ++i) {
    hm += h[i];
    tm += t[i];
  }
  hm /= n;
  tm /= n;
  double sxy = 0, sxx = 0;
  for (int i = 0; i < n; ++i) {
    sxy += (h[i] - hm) * (t[i] - tm);
    sxx += (h[i] - hm) * (h[i] - hm);
  }
  const double s = sxy / sxx, a = tm - s * hm;
  double rr = 0;
  for (int i = 0; i < n; ++i) {
    const double r = t[i] - (a + s * h[i]);
    rr += r * r;
  }
  *slope = s;
  *rmse = sqrt(rr / n);
}

// Median of v[0..n) (sorted in place, n small).
__device__ double median_small(double* v, int n) {
  for (int i = 1; i < n; ++i) {
    const double x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
  return (n & 1) ? v[n / 2] : (v[n / 2 - 1] + v[n / 2]) * 0.5;
}

__global__ void __launch_bounds__(kSurfThreads) surface_kernel(const SurfParams P) {
  extern __shared__ unsigned char smem[];
  const int m = blockIdx.x;
  const int n_tr = P.n_shots * P.nx;
  int* arrival = reinterpret_cast<int*>(smem);                       // onset sample, -1: zero trace
  double* work = reinterpret_cast<double*>(smem + ((n_tr * sizeof(int) + 15) & ~size_t(15)));
  __shared__ int nonfinite;
  if (threadIdx.x == 0) nonfinite = 0;
  __syncthreads();
  const float* g = P.gathers + static_cast<size_t>(m) * P.n_shots * P.nt * P.nx;
  // one thread per trace: its peak |amplitude|, then the first sample above frac x peak
  for (int tr = threadIdx.x; tr < n_tr; tr += blockDim.x) {
    const int s = tr / P.nx, r = tr - s * P.nx;
    const float* col = g + static_cast<size_t>(s) * P.nt * P.nx + r;
    float peak = 0.f;
    bool finite = true;
    for (int t = 0; t < P.nt; ++t) {
      const float v = col[static_cast<size_t>(t) * P.nx];
      finite = finite && isfinite(v);
      peak = fmaxf(peak, fabsf(v));
    }
    if (!finite) nonfinite = 1;
    int on = -1;
    if (peak > 0.f) {
      const double thr = P.frac * static_cast<double>(peak);
      for (int t = 0; t < P.nt; ++t)
        if (static_cast<double>(fabsf(col[static_cast<size_t>(t) * P.nx])) > thr) {
          on = t;
          break;
        }
    }
    arrival[tr] = on;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  ss_surface_estimate e{};
  e.far_offset_velocity = NAN;
  if (nonfinite) {
    e.status = SS_SURF_NONFINITE;
    P.out[m] = e;
    return;
  }
  // picks at 10-250 m offset: (offset, time, shot); distinct offsets ascending
  double* off = work;                 // [n_tr]
  double* tim = work + n_tr;          // [n_tr]
  double* dist = work + 2 * n_tr;     // [n_tr] distinct offsets
  double* med = work + 3 * n_tr;      // [n_tr] median time per distinct offset
  double* tmp = work + 4 * n_tr;      // [n_tr] scratch
  double* tmp2 = work + 5 * n_tr;     // [n_tr] scratch
  int* shot = reinterpret_cast<int*>(work + 6 * n_tr);
  int n = 0;
  for (int tr = 0; tr < n_tr; ++tr) {
    const int s = tr / P.nx, r = tr - s * P.nx;
    const double h = fabs(r * P.dx - P.src_x[s]);
    if (h >= 10.0 && h <= 250.0 && arrival[tr] >= 0) {
      off[n] = h;
      tim[n] = arrival[tr] * P.dt;
      shot[n] = s;
      ++n;
    }
  }
  if (n == 0) {
    e.status = SS_SURF_NO_ONSETS;
    P.out[m] = e;
    return;
  }
  int nd = 0;
  for (int i = 0; i < n; ++i) {
    bool seen = false;
    for (int j = 0; j < nd; ++j) seen = seen || dist[j] == off[i];
    if (!seen) {
      int j = nd++;
      while (j > 0 && dist[j - 1] > off[i]) {
        dist[j] = dist[j - 1];
        --j;
      }
      dist[j] = off[i];
    }
  }
  for (int d = 0; d < nd; ++d) {
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (off[i] == dist[d]) tmp[k++] = tim[i];
    med[d] = median_small(tmp, k);
  }
  // distinct offsets in [lo, hi] -> contiguous range of dist (ascending)
  auto range = [&](double lo, double hi, int* a) {
    int b = 0;
    *a = nd;
    for (int d = 0; d < nd; ++d)
      if (dist[d] >= lo && dist[d] <= hi) {
        if (*a == nd) *a = d;
        ++b;
      }
    return b;
  };
  int a_near;
  const int n_near = range(10.0, 60.0, &a_near);
  if (n_near != 6) {
    e.status = SS_SURF_FEW_NEAR;
    P.out[m] = e;
    return;
  }
  double slope, rmse;
  fit_line(dist + a_near, med + a_near, n_near, &slope, &rmse);
  if (slope <= 0 || !(1.0 / slope >= 1400.0 && 1.0 / slope <= 4600.0)) {
    e.status = SS_SURF_SLOPE;
    P.out[m] = e;
    return;
  }
  int a1, a2;
  const int n1 = range(10.0, 40.0, &a1), n2 = range(30.0, 60.0, &a2);
  double early, late, unused;
  fit_line(dist + a1, med + a1, n1, &early, &unused);
  fit_line(dist + a2, med + a2, n2, &late, &unused);
  const double curvature = fabs(early - late) / slope;
  double shot_slopes[SS_MAX_SHOTS];
  int n_shot_slopes = 0;
  for (int s = 0; s < P.n_shots; ++s) {
    int k = 0;
    for (int i = 0; i < n; ++i)
      if (shot[i] == s && off[i] >= 10.0 && off[i] <= 60.0) {
        tmp[k] = off[i];
        tmp2[k] = tim[i];
        ++k;
      }
    int distinct = 0;
    for (int i = 0; i < k; ++i) {
      bool seen = false;
      for (int j = 0; j < i; ++j) seen = seen || tmp[j] == tmp[i];
      distinct += seen ? 0 : 1;
    }
    if (distinct >= 4) {
      double sl, rm;
      fit_line(tmp, tmp2, k, &sl, &rm);
      shot_slopes[n_shot_slopes++] = sl;
    }
  }
  if (n_shot_slopes < 3) {
    e.status = SS_SURF_FEW_SHOTS;
    P.out[m] = e;
    return;
  }
  double mean = 0;
  for (int i = 0; i < n_shot_slopes; ++i) mean += shot_slopes[i];
  mean /= n_shot_slopes;
  double var = 0;
  for (int i = 0; i < n_shot_slopes; ++i) var += (shot_slopes[i] - mean) * (shot_slopes[i] - mean);
  const double spread = sqrt(var / n_shot_slopes) / slope;
  e.fit_rmse_ms = rmse * 1000.0;
  e.short_offset_curvature = curvature;
  e.shot_slope_spread = spread;
  if (rmse > 0.002 || curvature > 0.15 || spread > 0.15) {
    e.status = SS_SURF_UNRELIABLE;
    P.out[m] = e;
    return;
  }
  int af;
  const int nf = range(120.0, 250.0, &af);
  double far_slope = slope;
  if (nf >= 4) fit_line(dist + af, med + af, nf, &far_slope, &unused);
  e.far_offset_velocity = far_slope > 0 ? 1.0 / far_slope : NAN;
  const double refraction = fmax(0.0, 1.0 - far_slope / slope);
  e.confidence = 1.0 / (1.0 + rmse / P.dt + curvature / 0.15 + spread / 0.15 + refraction);
  e.velocity = fmin(fmax(1.0 / slope, 1500.0), 4500.0);
  e.possible_refraction = refraction > 0.15 ? 1 : 0;
  e.status = SS_SURF_OK;
  P.out[m] = e;
}

// ----------------------------------------------------------------------------
// Backgrounds and training inputs
// ----------------------------------------------------------------------------
__global__ void backgrounds_kernel(const double* __restrict__ v_surface, const double* __restrict__ trend,
                                   const double* __restrict__ rhos, int n_models, int n_rhos, int nz, int nx,
                                   float* __restrict__ out) {
  const long long total = static_cast<long long>(n_models) * n_rhos * nz * nx;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int z = static_cast<int>((i / nx) % nz);
    const long long mk = i / (static_cast<long long>(nz) * nx);
    const int k = static_cast<int>(mk % n_rhos);
    const long long m = mk / n_rhos;
    const double v = v_surface[m] + rhos[k] * trend[z];
    out[i] = static_cast<float>(fmin(fmax(v, 1500.0), 4500.0));
  }
}

__global__ void signed_log1p_kernel(const float* __restrict__ g, long long n, uint16_t* __restrict__ out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float v = g[i];
    const float l = log1pf(fabsf(v));
    const float r = v > 0.f ? l : (v < 0.f ? -l : 0.f);
    out[i] = __half_as_ushort(__float2half_rn(r));
  }
}

__global__ void f16_scaled_kernel(const uint16_t* __restrict__ in, long long n, float scale, float* __restrict__ out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    out[i] = __fdiv_rn(__half2float(__ushort_as_half(in[i])), scale);
}

__global__ void targets_kernel(const float* __restrict__ vel, long long n, float* __restrict__ y) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    y[i] = (vel[i] - 3000.f) / 1500.f;
}

__global__ void vref_kernel(const float* __restrict__ v1, const float* __restrict__ trend, int n_models, int nz,
                            int nx, float* __restrict__ out) {
  const long long total = static_cast<long long>(n_models) * nz * nx;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int z = static_cast<int>((i / nx) % nz);
    const long long m = i / (static_cast<long long>(nz) * nx);
    const float v = v1[m] + trend[z];
    out[i] = fminf(fmaxf((v - 3000.f) / 1500.f, -1.f), 1.f);
  }
}

}  // namespace

extern "C" {

int32_t ss_image_cache(const float* img, int32_t n_models, int32_t n_images, int32_t nz, int32_t nx,
                       int32_t zero_rows, double q, float clip, uint16_t* out, float* scale, int32_t* status,
                       void* stream) {
  ss_internal::clear_error();
  if (!img || !out || !scale || !status || n_models < 0 || n_images < 1 || nz < 1 || nx < 1 || zero_rows < 0)
    return fail(SS_ERR_INVALID, "bad arguments");
  if (!(q >= 0.0 && q <= 100.0)) return fail(SS_ERR_INVALID, "percentile must lie in [0, 100]");
  if (!(clip > 0.f)) return fail(SS_ERR_INVALID, "clip must be positive");
  const long long n = static_cast<long long>(n_images) * nz * nx;
  if (n >= (1LL << 31)) return fail(SS_ERR_UNSUPPORTED, "more than 2^31 values per model");
  if (n_models == 0) return SS_OK;
  // numpy's 'linear' percentile of float32 data: the virtual index
  // n*q + (1 - q) - 1 and its fractional part are float32 operations.
  const float qf = static_cast<float>(q / 100.0);
  const float t1 = static_cast<float>(n) * qf;
  const float t3 = 1.0f + (-qf);
  const float vi = (t1 + t3) - 1.0f;
  const float fl = std::floor(vi);
  CacheParams P{};
  P.img = img;
  P.n_images = n_images;
  P.nz = nz;
  P.nx = nx;
  P.zero_rows = std::min(zero_rows, nz);
  P.prev = std::min<long long>(std::max<long long>(static_cast<long long>(fl), 0), n - 1);
  P.next = std::min<long long>(P.prev + 1, n - 1);
  P.gamma = vi - fl;
  P.clip = clip;
  P.out = out;
  P.scale = scale;
  P.status = status;
  image_cache_kernel<<<n_models, kCacheThreads, 0, static_cast<cudaStream_t>(stream)>>>(P);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_surface_velocity(const float* gathers, int32_t n_models, int32_t n_shots, int32_t nt, int32_t nx,
                            const double* src_x, double dx, double dt, double frac, ss_surface_estimate* out,
                            void* stream) {
  ss_internal::clear_error();
  if (!gathers || !src_x || !out || n_models < 0 || n_shots < 1 || n_shots > SS_MAX_SHOTS || nt < 1 || nx < 1)
    return fail(SS_ERR_INVALID, "bad arguments");
  if (!(frac > 0.0 && frac < 1.0)) return fail(SS_ERR_INVALID, "onset threshold frac must lie between zero and one");
  if (!(dx > 0.0) || !(dt > 0.0)) return fail(SS_ERR_INVALID, "dx and dt must be positive");
  const int n_tr = n_shots * nx;
  if (n_tr > kMaxTraces) return fail(SS_ERR_UNSUPPORTED, "too many traces per model");
  if (n_models == 0) return SS_OK;
  SurfParams P{};
  P.gathers = gathers;
  P.n_shots = n_shots;
  P.nt = nt;
  P.nx = nx;
  for (int s = 0; s < n_shots; ++s) P.src_x[s] = src_x[s];
  P.dx = dx;
  P.dt = dt;
  P.frac = frac;
  P.out = out;
  const size_t smem = ((n_tr * sizeof(int) + 15) & ~size_t(15)) + 6 * static_cast<size_t>(n_tr) * sizeof(double) +
                      static_cast<size_t>(n_tr) * sizeof(int);
  if (smem > 48 * 1024)
    SS_TRY_CUDA(cudaFuncSetAttribute(surface_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  surface_kernel<<<n_models, kSurfThreads, smem, static_cast<cudaStream_t>(stream)>>>(P);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_backgrounds(const double* v_surface, const double* trend, const double* rhos, int32_t n_models,
                       int32_t n_rhos, int32_t nz, int32_t nx, float* out, void* stream) {
  ss_internal::clear_error();
  if (!v_surface || !trend || !rhos || !out || n_models < 0 || n_rhos < 1 || nz < 1 || nx < 1)
    return fail(SS_ERR_INVALID, "bad arguments");
  const long long total = static_cast<long long>(n_models) * n_rhos * nz * nx;
  if (total == 0) return SS_OK;
  backgrounds_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(v_surface, trend, rhos, n_models,
                                                                                    n_rhos, nz, nx, out);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_signed_log1p_f16(const float* g, int64_t n, uint16_t* out, void* stream) {
  ss_internal::clear_error();
  if (!g || !out || n < 0) return fail(SS_ERR_INVALID, "bad arguments");
  if (n == 0) return SS_OK;
  signed_log1p_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(g, n, out);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_f16_scaled(const uint16_t* in, int64_t n, float scale, float* out, void* stream) {
  ss_internal::clear_error();
  if (!in || !out || n < 0) return fail(SS_ERR_INVALID, "bad arguments");
  if (!std::isfinite(scale) || !(scale > 0.f))
    return fail(SS_ERR_INVALID, "Gather normalization scale must be finite and positive");
  if (n == 0) return SS_OK;
  f16_scaled_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, n, scale, out);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_velocity_targets(const float* vel, int64_t n, float* y, const float* v_surface, const float* trend,
                            int32_t n_models, int32_t nz, int32_t nx, float* vref, void* stream) {
  ss_internal::clear_error();
  if (n < 0 || (n > 0 && (!vel || !y))) return fail(SS_ERR_INVALID, "bad arguments");
  if (vref && (!v_surface || !trend || n_models < 0 || nz < 1 || nx < 1)) return fail(SS_ERR_INVALID, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n > 0) targets_kernel<<<grid_for(n), 256, 0, st>>>(vel, n, y);
  const long long total = static_cast<long long>(n_models) * nz * nx;
  if (vref && total > 0) vref_kernel<<<grid_for(total), 256, 0, st>>>(v_surface, trend, n_models, nz, nx, vref);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

}  // extern "C"
