// libshotsweep: B200 (sm_100a) kernels for ShotSweep's physics hot path.
//
// One velocity model x one shot is a "solve".  Each solve runs on a thread-block
// cluster of C CTAs (C = 3 for the 150x150 padded OpenFWI grid); the padded grid
// is cut into C horizontal bands, one per CTA.  Each thread keeps a 5 x 4 tile
// of both time levels in registers for the whole time loop; shared memory holds
// the current level of the band for the neighbouring tiles' stencils, and the
// tile's per-cell coefficients sit in tensor memory (TMEM), read row by row
// with tcgen05.ld, which leaves the registers to the wavefields.
// Neighbouring bands push their two edge rows into each other's halo rows every
// step through distributed shared memory (st.async counted on mbarriers).
//
// Arithmetic (reference: openfwi/physics/gpu.py)
//   forward   p[t+1] = p[t-1] + kappa*(p[t]-p[t-1]) + sigma*S(p[t])  (+ source)
//   adjoint   th[t]  = th[t+2] + kappa*(th[t+1]-th[t+2]) + sigma*S(th[t+1]) (+ sigma*res)
// with S the 9-point 4th-order Laplacian times 12*dx^2, kappa = 2A and
// sigma = c2*A/12 masked to the interior (zero on the 2-cell border).  The
// forward is the reference update (2p1 - B p0 + c2 L) A (gpu.py:111-115)
// rewritten with A*B = 2A - 1 (true for A = 1/(1+a), B = 1-a).  The adjoint is
// the reference adjoint mu = 2A m1 + lap^T(c2 A m1) - A B m2 (gpu.py:179)
// after the diagonal change of variable th = sigma*mu, which gives it the same
// form as the forward; the gradient becomes g*2v(dt/dx)^2 = 2/v * sum_t th*S(p)
// and mu at the source is th/sigma there (gpu.py:181-187).
//
// Instead of the reference's checkpoint-and-recompute (gpu.py:131,169-176) the
// forward stores S(p[t]) of every step to a per-cluster history in HBM
// (coalesced 16-byte stores from every thread) and the adjoint streams it
// back in reverse with TMA bulk copies (cp.async.bulk), two steps ahead.  This trades 2x4 bytes of HBM traffic per cell
// and step for the 16 flops per cell and step that a recompute would cost.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/shotsweep.h"
#include "internal.h"

namespace {

// Tile height H (rows of the band per thread) and the CTA size it allows: the
// register file holds 65,536 registers per SM and a CTA runs alone on its SM,
// so H x 4 cells at two time levels plus accumulators leave 168 registers per
// thread at H = 5 (384 threads), 128 at H = 4 (512), 102 at H = 3 (640).
constexpr int kDefaultRows = 5;
__host__ __device__ constexpr int max_threads_for(int H) { return H <= 3 ? 640 : H == 4 ? 512 : H == 5 ? 384 : 320; }
constexpr int kMinRows = 3, kMaxRows = 6;
constexpr int kMaxCluster = 16;
// Adjoint history slabs in shared memory (prefetch depth: slabs - 1): four on
// the OpenFWI fast path (timed 0.7 % faster than three), three for every other
// grid and for uneven batches, whose large grids need the shared memory for
// their bands.
constexpr int kStagesFast = 4;
constexpr int kStagesGeneric = 3;
constexpr int kFastRS = 156;               // shared row stride of the 150-column padded OpenFWI grid
constexpr size_t kMaxSmem = 227 * 1024;
// The fixed-geometry kernels allocate kCoefCols of an SM's 512 tensor-memory
// columns per CTA.  At least 60 KB of shared memory per CTA keeps three or
// fewer of them on one SM (228 KB), so every allocation is served at once and
// no CTA waits for columns held by a CTA that waits for it.
constexpr size_t kTcMinSmem = 60 * 1024;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;   // 2 s per bounded wait

thread_local std::string g_last_error;

// NVTX range around an entry point (header-only NVTX: free unless a profiler is attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define SS_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(SS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

// ----------------------------------------------------------------------------
// PTX helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster_u32(uint32_t addr, int v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Tensor memory (TMEM) holds the per-cell coefficients of the fixed-geometry
// kernels: warp w may reach lanes 32*(w%4) .. +31 only, so thread (w, l) owns
// lane 32*(w%4) + l and columns 8H*(w/4) + 8k .. +7 for tile row k: kappa
// (4 cells), then -sigma (4 cells).
constexpr uint32_t kCoefCols = 128;         // a power of two >= 8H x warp groups
__device__ __forceinline__ void tmem_alloc_warp(uint32_t dst_smem, uint32_t ncols) {   // one whole warp
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr, uint32_t ncols) {   // the allocating warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 8 consecutive 32-bit columns of this thread's lane (whole warp, converged).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
               "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// Starts loading 8 columns; the registers are valid after tmem_wait_ld on them.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
               : "r"(taddr)
               : "memory");
}
// Completes this thread's TMEM loads; the operands order every later use of v after it.
__device__ __forceinline__ void tmem_wait_ld(float (&v)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]), "+f"(v[6]), "+f"(v[7])
               :
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after kWaitLimitNs, records SS_ERR_TIMEOUT and
// returns, so that every thread still reaches every barrier of the kernel.
__device__ __forceinline__ void mbar_wait_bounded(uint32_t bar, uint32_t parity, int* err,
                                                  unsigned long long limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) {
      atomicExch(err, static_cast<int>(SS_ERR_TIMEOUT));
      return;
    }
  }
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_all() { asm volatile("fence.proxy.async;" ::: "memory"); }


// Normalised depth into the absorbing layer (gpu.py:85-87).
__device__ __forceinline__ double layer_depth(int i, int n, int pad) {
  const int d = max(max(pad - i, i - (n - 1 - pad)), 0);
  return static_cast<double>(d) / pad;
}

// ----------------------------------------------------------------------------
// Fused per-solve kernel
// ----------------------------------------------------------------------------
// One model (one background row) of an uneven batch, as the kernel reads it:
// its grid, its band plan for the launch's cluster size, and where its data
// lie in the packed arrays.  Built on the host by the batch planner.
struct BatchItemDev {
  int nz, nx, nt, pad, nzp, nxp, src_row, n_shots;
  int ncg, nseg, bh, nact;            // column groups, tile rows per band, band rows, active threads
  int shot_cols[SS_MAX_SHOTS];
  long long vel_off;                  // floats: [nz][nx] velocities
  long long obs_off;                  // floats: [n_shots][nt][nx] observations (images) or gathers (forward)
  long long out_off;                  // floats: [n_shots][nz][nx] img / illum / grad
  double damp_k;                      // damping constant of this pad
  float vmute;                        // mute velocity; <= 0: no mute
  int reserved;
};

// The current solve's geometry inside a batch launch (registers).
struct SolveGeo {
  int nz, nx, nt, pad, nzp, nxp, src_row, ncg, nseg, bh, nact, rs, sw;
};

struct KParams {
  int nz, nx, nt, pad, nzp, nxp, n_shots, src_row;
  int shot_cols[SS_MAX_SHOTS];
  double dtdx2, damp_k, amp_ref;
  float dx, dt;
  int ncg, nseg, bh, C, rs, sw, nact;
  int nxs;         // trace row stride of the per-slot scratch (nx rounded up to 4)
  int n_solves;
  const float* vel;
  const float* wav;
  long long wav_stride;   // floats between consecutive models' wavelets; 0: one wavelet for all
  const float* obs;
  const float* vmute;
  float t_mute;
  float* gathers;  // forward mode output [solve][nt][nx]
  float* trace;    // per-slot scratch [nt][nx]
  float* illum;
  float* grad;     // output, or per-slot scratch [nz][nx]
  int grad_per_slot;
  float* img;
  float* gpad;     // per-slot scratch [nzp][nxp]
  float* hist;     // per-slot [nt][C][bh*sw]
  float* ckpt;
  int ckpt_interval, n_ckpt;
  float eps;
  int laplacian;
  int* err;
  // segment mode (checkpointed adjoint): levels [seg_start, seg_start + seg_steps)
  int seg_start, seg_steps, seg_index, hist_steps;
  float* theta;        // [solve][2][nzp][nxp]: in (th[e+1], th[e+2]), out (th[s], th[s+1])
  float* gacc;         // [solve][nzp][nxp]: += -sum_t th*S over the segment
  float* illum_acc;    // [solve][nz][nx]: += sum_t S^2 over the segment
  float* src_acc_io;   // [solve]: += sum_t th(source cell) * w[t]
  const float* res_in; // [solve][nt][nx]: adjoint source (the gathers' cotangent)
  // uneven batch: per-item geometry, the longest-first solve list, its counter
  const BatchItemDev* items;
  const int* order;    // [n_solves] item << 4 | shot
  int* counter;        // next entry of order; zero at launch
  size_t hist_slot, trace_slot, gpad_slot, grad_slot;   // per-slot scratch (floats)
};

struct Smem {
  float* f[2];
  float* stg0;     // kStages history slabs of bh x sw, consecutive (the adjoint's prefetch ring)
  float* wav;
  float* red;
  float* res0;     // kStages residual rows of nxs, consecutive
  float* dummy;    // zero tile for lanes without cells: (H + 4) rows of RS, then H rows of sw
  uint64_t* bar;
};

__device__ __forceinline__ float mute_weight(int t, int r, int shot_col, float dx, float dt, float vm, float t_mute) {
  // gpu.py:146-150 in float32: h/v_mute + t_mute, 30 ms cosine ramp.
  const float h = fabsf(static_cast<float>(r) * dx - static_cast<float>(shot_col) * dx);
  const float tt = static_cast<float>(t) * dt;
  const float t0 = h / vm + t_mute;
  const float ramp = fminf(fmaxf((tt - t0) / 0.03f, 0.f), 1.f);
  // before and after the ramp the weight is exactly 0 and 1 (as the reference's float64 value); the cosine
  // is needed only inside it
  if (ramp <= 0.f) return 0.f;
  if (ramp >= 1.f) return 1.f;
  return 0.5f - 0.5f * cosf(3.14159265358979323846f * ramp);
}

// Fold the padded gradient onto the model edges (gpu.py:56-67, 185-187) and,
// for images, normalise by illumination and Laplacian-filter (gpu.py:206-209).
// Called by every thread of the cluster; gp holds this slot's padded gradient.
template <int MODE>
__device__ __forceinline__ void epilogue(const KParams& P, Smem& S, float* gp, float* go, const float* il, float* im,
                                         const int nz, const int nx, const int pad, const int nzp, const int nxp,
                                         int rank, int tid, int nthr) {
    // ---- fold the padding onto the edge cells (gpu.py:56-67, 185-187) ----
    {
      const int zlo = 2, zhi = nzp - 2, xlo = 2, xhi = nxp - 2;
      auto G = [&](int i, int j) -> float { return gp[static_cast<size_t>(i) * nxp + j]; };
      const int gthr = rank * nthr + tid, gstride = P.C * nthr;
      for (int o = gthr; o < nz * nx; o += gstride) {
        const int z = o / nx, x = o - z * nx;
        const bool zc = (z == 0 || z == nz - 1), xc = (x == 0 || x == nx - 1);
        if (zc && xc) continue;   // corners: one warp each below
        const int i = pad + z, j = pad + x;
        float val = G(i, j);
        if (z == 0)
          for (int ii = zlo; ii < pad; ++ii) val += G(ii, j);
        if (z == nz - 1)
          for (int ii = pad + nz; ii < zhi; ++ii) val += G(ii, j);
        if (x == 0)
          for (int jj = xlo; jj < pad; ++jj) val += G(i, jj);
        if (x == nx - 1)
          for (int jj = pad + nx; jj < xhi; ++jj) val += G(i, jj);
        go[o] = val;
      }
      const int warp = tid >> 5, lane = tid & 31, n_warps = nthr >> 5;
      for (int corner = warp; rank == 0 && corner < 4; corner += n_warps) {
        const int z = (corner & 1) ? nz - 1 : 0, x = (corner & 2) ? nx - 1 : 0;
        const int i = pad + z, j = pad + x;
        const int i0 = z == 0 ? zlo : pad + nz, i1 = z == 0 ? pad : zhi;
        const int j0 = x == 0 ? xlo : pad + nx, j1 = x == 0 ? pad : xhi;
        float val = 0.f;
        for (int ii = i0 + lane; ii < i1; ii += 32) val += G(ii, j);   // strip above/below
        for (int jj = j0 + lane; jj < j1; jj += 32) val += G(i, jj);   // strip left/right
        const int bw = j1 - j0, bn = (i1 - i0) * bw;
        for (int q = lane; q < bn; q += 32) val += G(i0 + q / bw, j0 + q % bw);   // corner block
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) val += __shfl_xor_sync(0xffffffffu, val, off);
        if (lane == 0) go[z * nx + x] = G(i, j) + val;
      }
    }
    if (MODE == SS_MODE_IMAGES) {
      __threadfence();
      cluster_sync();
      // ---- image epilogue (gpu.py:206-209) --------------------------------
      float mx = -INFINITY;
      for (int o = tid; o < nz * nx; o += nthr) mx = fmaxf(mx, il[o]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if ((tid & 31) == 0) S.red[tid >> 5] = mx;
      __syncthreads();
      if (tid < 32) {
        float w = tid < (nthr + 31) / 32 ? S.red[tid] : -INFINITY;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, off));
        if (tid == 0) S.red[0] = w;
      }
      __syncthreads();
      const float emax = P.eps * S.red[0];
      float* pre = gp;   // reuse the padded-gradient scratch for the unfiltered image
      const int gthr = rank * nthr + tid, gstride = P.C * nthr;
      for (int o = gthr; o < nz * nx; o += gstride) {
        const float den = fmaxf(il[o] + emax, 1.17549435e-38f);
        pre[o] = -go[o] / den;
      }
      if (P.laplacian) {
        __threadfence();
        cluster_sync();
        for (int o = gthr; o < nz * nx; o += gstride) {
          const int z = o / nx, x = o - z * nx;
          auto I = [&](int zz, int xx) -> float {
            zz = min(max(zz, 0), nz - 1);
            xx = min(max(xx, 0), nx - 1);
            return pre[zz * nx + xx];
          };
          const float c = I(z, x);
          const float lz = -I(z - 2, x) + 16.f * I(z - 1, x) - 30.f * c + 16.f * I(z + 1, x) - I(z + 2, x);
          const float lx = -I(z, x - 2) + 16.f * I(z, x - 1) - 30.f * c + 16.f * I(z, x + 1) - I(z, x + 2);
          im[o] = -((lz + lx) / 12.f);
        }
      } else {
        for (int o = gthr; o < nz * nx; o += gstride) im[o] = pre[o];
      }
    }
}

// Negated 9-point stencil, -S, of the four cells of one row (S = 12 dx^2 x the
// 4th-order Laplacian of gpu.py:33-37).  r0..r4 are the rows -2..+2 of the
// thread's four columns; lf / rt are the two columns left / right of them.
// Pairs (columns 0-1, 2-3) go through the packed FP32x2 pipe.
__device__ __forceinline__ void neg_stencil(const float4& r0, const float4& r1, const float4& r2, const float4& r3,
                                            const float4& r4, const float2& lf, const float2& rt, float2& lo,
                                            float2& hi) {
  const float2 zn_lo = __fadd2_rn(make_float2(r1.x, r1.y), make_float2(r3.x, r3.y));
  const float2 zn_hi = __fadd2_rn(make_float2(r1.z, r1.w), make_float2(r3.z, r3.w));
  const float2 zf_lo = __fadd2_rn(make_float2(r0.x, r0.y), make_float2(r4.x, r4.y));
  const float2 zf_hi = __fadd2_rn(make_float2(r0.z, r0.w), make_float2(r4.z, r4.w));
  const float2 xn_lo = make_float2(lf.y + r2.y, r2.x + r2.z);
  const float2 xn_hi = make_float2(r2.y + r2.w, r2.z + rt.x);
  const float2 xf_lo = make_float2(lf.x + r2.z, lf.y + r2.w);
  const float2 xf_hi = make_float2(r2.x + rt.x, r2.y + rt.y);
  const float2 m16 = make_float2(-16.f, -16.f), p60 = make_float2(60.f, 60.f);
  lo = __ffma2_rn(p60, make_float2(r2.x, r2.y), __ffma2_rn(m16, __fadd2_rn(zn_lo, xn_lo), __fadd2_rn(zf_lo, xf_lo)));
  hi = __ffma2_rn(p60, make_float2(r2.z, r2.w), __ffma2_rn(m16, __fadd2_rn(zn_hi, xn_hi), __fadd2_rn(zf_hi, xf_hi)));
}

// new = old2 + kappa*(old1 - old2) - nsig*(-S), for a pair of cells.
__device__ __forceinline__ float2 leapfrog(float2 kap, float2 nsig, float2 old1, float2 old2, float2 sneg) {
  const float2 d = __ffma2_rn(make_float2(-1.f, -1.f), old2, old1);
  return __ffma2_rn(nsig, sneg, __ffma2_rn(kap, d, old2));
}

// Predicated global store (no branch in the row loop), streaming (.cs): the
// history is read back only after the whole forward sweep.
__device__ __forceinline__ void st_global_v4_if(bool p, float* addr, float4 v) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t@q st.global.cs.v4.f32 [%0], {%1, %2, %3, %4};\n\t}" ::"l"(addr),
      "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(static_cast<uint32_t>(p))
      : "memory");
}

// Predicated form: no branch (and no divergence bookkeeping) in the row loop.
__device__ __forceinline__ void st_async_v4_if(bool p, uint32_t addr, float4 v, uint32_t bar) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %6, 0;\n\t"
      "@q st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];\n\t}" ::"r"(addr),
      "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(bar), "r"(static_cast<uint32_t>(p))
      : "memory");
}


// Coefficients of tile row k: ck0, ck1 (kappa) and cs0, cs1 (-sigma), each
// for two cells; from registers, or (TC) loaded from tensor memory at the
// row.  (Loading the next row one row ahead keeps 8 more registers live and
// measured slower.)
#define SS_COEF_ROW(k) \
          float2 ck0, ck1, cs0, cs1; \
          if constexpr (TC) { \
            float cfr[8]; \
            tmem_ld8(tc_base + 8u * (k), cfr); \
            tmem_wait_ld(cfr); \
            ck0 = make_float2(cfr[0], cfr[1]); \
            ck1 = make_float2(cfr[2], cfr[3]); \
            cs0 = make_float2(cfr[4], cfr[5]); \
            cs1 = make_float2(cfr[6], cfr[7]); \
          } else { \
            ck0 = kap[k][0]; \
            ck1 = kap[k][1]; \
            cs0 = nsig[k][0]; \
            cs1 = nsig[k][1]; \
          }

// Body of one tile row k (a compile-time constant after unrolling) inside
// solve_kernel's step; written once, expanded with
// (SPECIAL) and without the source / receiver terms.  The row's two x-halo
// pairs lf / rt come from the enclosing loop, which loads them one row ahead
// (1.2 % faster than loading them at the row).
#define SS_TILE_ROW(k, SPECIAL) \
          const float4 rm2 = k >= 2 ? as4(O1[k - 2]) : (k == 0 ? h0 : h1); \
          const float4 rm1 = k >= 1 ? as4(O1[k - 1]) : h1; \
          const float4 rc = as4(O1[k]); \
          const float4 rp1 = k + 1 < H ? as4(O1[k + 1]) : h2; \
          const float4 rp2 = k + 2 < H ? as4(O1[k + 2]) : (k + 2 == H ? h2 : h3); \
          float2 s_lo, s_hi; \
          neg_stencil(rm2, rm1, rc, rp1, rp2, lf, rt, s_lo, s_hi); \
          const float2 n_lo = leapfrog(ck0, cs0, O1[k][0], O2[k][0], s_lo); \
          const float2 n_hi = leapfrog(ck1, cs1, O1[k][1], O2[k][1], s_hi); \
          float4 nw = make_float4(n_lo.x, n_lo.y, n_hi.x, n_hi.y); \
          if (fwd) { \
            if (SPECIAL) {  /* injection after damping (gpu.py:113-114): + w at the source cell */ \
              if (k == src_k) { \
                nw.x = fmaf(1.f, am0, nw.x); \
                nw.y = fmaf(1.f, am1, nw.y); \
                nw.z = fmaf(1.f, am2, nw.z); \
                nw.w = fmaf(1.f, am3, nw.w); \
              } \
            } \
          } else { \
            if (SPECIAL) {  /* residual injection th += sigma*res (gpu.py:180), res loaded once per step; */ \
              /* a branch on the one receiver row (per-row selects on every row measured 1.3 % slower) */ \
              if (k == rec_k) { \
                nw.x = fmaf(-cs0.x, rv0, nw.x); \
                nw.y = fmaf(-cs0.y, rv1, nw.y); \
                nw.z = fmaf(-cs1.x, rv2, nw.z); \
                nw.w = fmaf(-cs1.y, rv3, nw.w); \
              } \
            } \
          } \
          if (k < 2) \
            st_async_v4_if(push_up, up_addr + (cur ^ 1) * field_bytes + 4u * (k * RS), nw, up_bar + 8u * (cur ^ 1)); \
          if (k >= H - 2) \
            st_async_v4_if(push_dn, dn_addr + (cur ^ 1) * field_bytes + 4u * ((k - (H - 2)) * RS), nw, \
                           dn_bar + 8u * (cur ^ 1)); \
          O2[k][0] = make_float2(nw.x, nw.y); \
          O2[k][1] = make_float2(nw.z, nw.w); \
          *reinterpret_cast<float4*>(yc + k * RS) = nw; \
          if (fwd) { \
            if (ADJ) { \
              st_global_v4_if(active, stg + k * SW, make_float4(s_lo.x, s_lo.y, s_hi.x, s_hi.y)); \
              acc[k][0] = __ffma2_rn(s_lo, s_lo, acc[k][0]); \
              acc[k][1] = __ffma2_rn(s_hi, s_hi, acc[k][1]); \
            } \
          } else { \
            const float4 h = *reinterpret_cast<const float4*>(hl + k * SW); \
            acc[k][0] = __ffma2_rn(O2[k][0], make_float2(h.x, h.y), acc[k][0]); \
            acc[k][1] = __ffma2_rn(O2[k][1], make_float2(h.z, h.w), acc[k][1]); \
          }

// FAST: the OpenFWI geometry (nx = 70, pad = 40), whose strides are
// compile-time constants; otherwise they come from the parameters.
//
// Each thread owns an H x 4 tile of cells and keeps both of its time levels
// (old1 = t, old2 = t-1) in registers; shared memory carries only what the
// neighbouring tiles read (the full field of the current level, ping-pong
// buffered).  The time loop is unrolled by two so that the two register
// arrays swap roles without moves.
template <int MODE, bool FAST, bool BATCH, int H>
__global__ void __launch_bounds__(max_threads_for(H), 1) solve_kernel(const KParams P) {
  constexpr bool ADJ = MODE != SS_MODE_FORWARD;
  constexpr int kStages = (FAST && !BATCH) ? kStagesFast : kStagesGeneric;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // Geometry: compile-time constants on the fast path, parameter-bank reads
  // on the generic path (macros, so that it keeps no registers for them), and
  // the current solve's values in an uneven batch (BATCH).
  SolveGeo gs{};
#define RS (FAST ? kFastRS : BATCH ? gs.rs : P.rs)        /* shared row stride (floats) */
#define NX (FAST ? 70 : BATCH ? gs.nx : P.nx)             /* receivers per shot */
#define PAD (FAST ? 40 : BATCH ? gs.pad : P.pad)
#define SW (FAST ? kFastRS - 8 : BATCH ? gs.sw : P.sw)    /* history row width */
#define NXS (FAST ? 72 : P.nxs)                           /* padded trace row */
#define GNZ (BATCH ? gs.nz : P.nz)
#define GNT (BATCH ? gs.nt : P.nt)
#define GNZP (BATCH ? gs.nzp : P.nzp)
#define GNXP (BATCH ? gs.nxp : P.nxp)
#define GBH (BATCH ? gs.bh : P.bh)
#define GNCG (BATCH ? gs.ncg : P.ncg)
#define GNSEG (BATCH ? gs.nseg : P.nseg)
#define GNACT (BATCH ? gs.nact : P.nact)

  // The fixed-geometry instantiations keep the per-cell coefficients in
  // tensor memory (freeing 8H registers per thread); the uneven batch keeps
  // them in registers.  Thread (w, l) owns TMEM lane 32*(w%4) + l and the
  // 8H columns from 8H*(w/4): kappa (4 cells), then -sigma (4 cells) per
  // tile row; at most kCoefCols columns for every H <= 5.
  constexpr bool TC = !BATCH && H <= 5;
  constexpr uint32_t kColsPerWarp = 8u * H;
  static_assert(!TC || kColsPerWarp * ((max_threads_for(H) / 32 + 3) / 4) <= kCoefCols, "TMEM columns");
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  // A 1-D grid of 1-D clusters: the CTA's rank in its cluster and the
  // cluster index follow from blockIdx, which the compiler knows is uniform.
  const int rank = static_cast<int>(blockIdx.x % P.C);
  const int slot = static_cast<int>(blockIdx.x / P.C);
  const int n_slots = static_cast<int>(gridDim.x / P.C);

  // ---- shared-memory carve-up (identical in every CTA of the cluster) ----
  // Fixed geometry: fields, history slabs, then the rest.  Uneven batch:
  // barriers, wavelet, reduction words and receiver rows first, at fixed
  // offsets; the fields, slabs and zero tile of each solve after them.
  Smem S;
  size_t field_floats = static_cast<size_t>(P.bh + 4) * RS;
  size_t stage_floats = ADJ ? static_cast<size_t>(P.bh) * SW : 0;
  float* solve_smem = nullptr;   // BATCH: start of the per-solve part
  if (!BATCH) {
    float* base = reinterpret_cast<float*>(smem_raw);
    S.f[0] = base;
    S.f[1] = base + field_floats;
    S.stg0 = base + 2 * field_floats;
    S.wav = base + 2 * field_floats + kStages * stage_floats;
    S.red = S.wav + ((P.nt + 31) & ~31);
    S.res0 = S.red + 32;
    S.dummy = S.res0 + kStages * NXS;
    S.bar = reinterpret_cast<uint64_t*>(S.dummy + (H + 4) * RS + H * SW);   // [0,kStages) history, then 2 halos
    {   // self-check: the layout (barriers and the TMEM address word last) must fit the launch's allocation;
        // every CTA of the cluster computes the same sizes, so all of them return together
      uint32_t dyn = 0;
      asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
      const size_t end = reinterpret_cast<const unsigned char*>(S.bar + kStages + 3) - smem_raw;
      if (end > dyn) {
        if (tid == 0) atomicExch(P.err, static_cast<int>(SS_ERR_UNSUPPORTED));
        return;
      }
    }
  } else {
    S.bar = reinterpret_cast<uint64_t*>(smem_raw);
    static_assert((kStages + 2) * sizeof(uint64_t) <= 16 * sizeof(float), "barriers overrun the wavelet");
    S.wav = reinterpret_cast<float*>(smem_raw) + 16;   // 64-byte aligned after the barriers
    S.red = S.wav + ((P.nt + 31) & ~31);
    S.res0 = S.red + 32;
    solve_smem = S.res0 + kStages * NXS;
  }
  for (int i = tid; i < P.nt; i += nthr) S.wav[i] = P.wav[i];
  if (tid == 0) {
    for (int b = 0; b < kStages + 2; ++b) mbar_init(smem_u32(&S.bar[b]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // kCoefCols TMEM columns, allocated by warp 0; the address lands in the
  // word after the barriers.  The planner keeps at most three CTAs of this
  // kernel on an SM, so the allocation never waits on another CTA.
  if (TC && tid < 32) tmem_alloc_warp(smem_u32(&S.bar[kStages + 2]), kCoefCols);
  if (TC) tmem_fence_before();
  const uint32_t hist_bar0 = smem_u32(&S.bar[0]);
  const uint32_t halo_bar0 = smem_u32(&S.bar[kStages]);
  uint32_t hist_phase = 0, halo_phase = 0;   // parity of the next wait, one bit per buffer
  auto stage_buf = [&](int b) { return S.stg0 + b * stage_floats; };
  auto res_buf = [&](int b) { return S.res0 + b * NXS; };
  int* const next_solve = reinterpret_cast<int*>(S.red) + 31;   // BATCH: the cluster's next entry of P.order

  constexpr bool SEG = MODE == SS_MODE_SEGMENT;
  const size_t hist_step_fixed = static_cast<size_t>(P.C) * P.bh * SW;
  const size_t trace_slot = BATCH ? P.trace_slot : static_cast<size_t>(P.nt) * NXS;

  cluster_sync();   // barriers initialised and wavelet staged everywhere
  uint32_t tc_base = 0;   // this thread's TMEM lane and first coefficient column
  if (TC) {
    tmem_fence_after();
    const uint32_t warp = static_cast<uint32_t>(tid >> 5);
    tc_base = *reinterpret_cast<const uint32_t*>(&S.bar[kStages + 2]) + ((32u * (warp & 3u)) << 16) +
              kColsPerWarp * (warp >> 2);
  }

  for (int it = slot;; it += n_slots) {
    // ---- next solve: round robin, or (uneven batch) the next entry of the
    // longest-first list, taken by rank 0 and broadcast through DSMEM ------
    int solve, b, s;
    if (BATCH) {
      if (rank == 0 && tid == 0) {
        const int j = atomicAdd(P.counter, 1);
        for (int r = 0; r < P.C; ++r) st_cluster_u32(mapa(smem_u32(next_solve), r), j);
      }
      cluster_sync();
      const int j = *next_solve;
      if (j >= P.n_solves) break;
      solve = P.order[j];
      b = solve >> 4;
      s = solve & 15;
      const BatchItemDev& item = P.items[b];
      gs.nz = item.nz;
      gs.nx = item.nx;
      gs.nt = item.nt;
      gs.pad = item.pad;
      gs.nzp = item.nzp;
      gs.nxp = item.nxp;
      gs.src_row = item.src_row;
      gs.ncg = item.ncg;
      gs.nseg = item.nseg;
      gs.bh = item.bh;
      gs.nact = item.nact;
      gs.rs = 4 * item.ncg + 8;
      gs.sw = 4 * item.ncg;
      // per-solve part of shared memory
      field_floats = static_cast<size_t>(gs.bh + 4) * gs.rs;
      stage_floats = ADJ ? static_cast<size_t>(gs.bh) * gs.sw : 0;
      S.f[0] = solve_smem;
      S.f[1] = solve_smem + field_floats;
      S.stg0 = solve_smem + 2 * field_floats;
      S.dummy = S.stg0 + kStages * stage_floats;
      {   // self-check: this solve's part of shared memory must fit the launch's allocation
        uint32_t dyn = 0;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        const size_t end = reinterpret_cast<const unsigned char*>(S.dummy + (H + 4) * gs.rs + H * gs.sw) - smem_raw;
        if (end > dyn || gs.nact > nthr) {
          if (tid == 0) atomicExch(P.err, static_cast<int>(SS_ERR_UNSUPPORTED));
          continue;   // uniform across the cluster: every CTA sees the same solve and sizes
        }
      }
    } else {
      if (it >= P.n_solves) break;
      solve = it;
      b = solve / P.n_shots;
      s = solve - b * P.n_shots;
    }
    const float* v = BATCH ? P.vel + P.items[b].vel_off : P.vel + static_cast<size_t>(b) * P.nz * NX;
    const int shot_col = BATCH ? P.items[b].shot_cols[s] : P.shot_cols[s];
    const int src_c = PAD + shot_col;
    // offsets of this solve's [nz][nx] outputs and [nt][nx] traces
    const size_t out_off = BATCH ? static_cast<size_t>(P.items[b].out_off) + static_cast<size_t>(s) * GNZ * NX
                                 : static_cast<size_t>(solve) * P.nz * NX;
    const size_t trc_off = BATCH ? static_cast<size_t>(P.items[b].obs_off) + static_cast<size_t>(s) * GNT * NX
                                 : static_cast<size_t>(solve) * P.nt * NX;
    const double damp_k = BATCH ? P.items[b].damp_k : P.damp_k;
    const float v_mute = BATCH ? P.items[b].vmute : (P.vmute ? P.vmute[b] : 0.f);
    const bool muted = BATCH ? v_mute > 0.f : P.vmute != nullptr;

    // ---- this thread's tile -----------------------------------------------
    // Warp-aligned mapping: the first nseg*ncg_main threads cover column
    // groups [0, ncg_main) with one tile row per warp; the remaining column
    // groups of every tile row are packed after them.
    const bool active = tid < GNACT;
    const int ncg_main = (GNCG / 32) * 32, ncg_rem = GNCG - ncg_main;
    int cg = 0, seg = 0;
    if (active) {
      if (tid < GNSEG * ncg_main) {
        seg = tid / ncg_main;
        cg = tid - seg * ncg_main;
      } else {
        const int u = tid - GNSEG * ncg_main;
        seg = u / ncg_rem;
        cg = ncg_main + (u - seg * ncg_rem);
      }
    }
    const int row0 = 2 + rank * GBH;                // first padded row of the band
    const int myrow = row0 + seg * H;               // first padded row of this thread
    const int col0 = 2 + 4 * cg;                    // first padded column
    const int o0 = 4 * cg + 4;                      // shared-memory column offset of col0
    const int lr0 = seg * H;                        // shared row of tile row -2
    const int src_r = PAD + (BATCH ? gs.src_row : P.src_row);   // padded row of sources and receivers
    const int rec_rank = (src_r - 2) / GBH;

    // Halo exchange: the two edge rows of a band are pushed into the
    // neighbour's halo rows with st.async, which counts the bytes on the
    // neighbour's halo mbarrier of that buffer; readers of halo rows wait on it.
    const bool edge_up = active && seg == 0 && rank > 0;
    const bool edge_dn = active && seg == GNSEG - 1 && rank < P.C - 1;
    const uint32_t field_bytes = static_cast<uint32_t>(field_floats * sizeof(float));
    const uint32_t up_addr = edge_up ? mapa(smem_u32(S.f[0] + (GBH + 2) * RS + o0), rank - 1) : 0u;
    const uint32_t up_bar = edge_up ? mapa(halo_bar0, rank - 1) : 0u;
    const uint32_t dn_addr = edge_dn ? mapa(smem_u32(S.f[0] + o0), rank + 1) : 0u;
    const uint32_t dn_bar = edge_dn ? mapa(halo_bar0, rank + 1) : 0u;
    const uint32_t halo_bytes = 32u * GNCG * ((rank > 0 ? 1u : 0u) + (rank < P.C - 1 ? 1u : 0u));
    const int rec_k = (active && src_r >= myrow && src_r < myrow + H) ? src_r - myrow : -1;
    // Warp-uniform forms of per-thread conditions of the step (votes, which
    // the compiler knows are uniform): the branches they guard need no
    // reconvergence in the warps that skip them.
    const bool warp_edge = __any_sync(0xffffffffu, edge_up || edge_dn);
    const bool warp0 = __any_sync(0xffffffffu, tid == 0);
    const bool warp_recv = __any_sync(0xffffffffu, tid < NX);

    const uint32_t stage_bytes = static_cast<uint32_t>(static_cast<size_t>(GBH) * SW * sizeof(float));
    const size_t hist_slot = BATCH ? P.hist_slot : static_cast<size_t>(P.hist_steps) * hist_step_fixed;
    const int lvl_lo = SEG ? P.seg_start : 0;                  // first level of the time range
    const int n_steps = SEG ? P.seg_steps : GNT;                // steps of each sweep
    const int lvl_hi = lvl_lo + n_steps - 1;
    const size_t hist_step = BATCH ? static_cast<size_t>(P.C) * GBH * SW : hist_step_fixed;
    float* const hist_mine = ADJ ? P.hist + static_cast<size_t>(slot) * hist_slot + static_cast<size_t>(rank) * GBH * SW
                                 : nullptr;

    // ---- per-cell coefficients ----------------------------------------
    // kappa = 2A and -sigma = -(c2 A)/12 of every cell: in tensor memory
    // (TC; the source cell's -sigma also stays in a register for the
    // gradient's source term) or in registers.
    int src_k = -1, src_m = 0;
    if (active && src_r >= myrow && src_r < myrow + H && src_c >= col0 && src_c < col0 + 4) {
      src_k = src_r - myrow;
      src_m = src_c - col0;
    }
    float nsig_src = 0.f;
    float2 kap[H][2], nsig[H][2], acc[H][2], A[H][2], B[H][2];
#pragma unroll
    for (int k = 0; k < H; ++k) {
      float kvs[4], svs[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int r = myrow + k, c = col0 + m;
        float kv = 0.f, sv = 0.f;
        if (active && r < GNZP - 2 && c < GNXP - 2) {
          const double dz = layer_depth(r, GNZP, PAD), dxl = layer_depth(c, GNXP, PAD);
          const float Ad = static_cast<float>(1.0 / (1.0 + damp_k * (dz * dz + dxl * dxl)));
          const int vz = min(max(r - PAD, 0), GNZ - 1), vx = min(max(c - PAD, 0), NX - 1);
          const double vp = v[vz * NX + vx];
          const float c2 = static_cast<float>(vp * vp * P.dtdx2);
          kv = 2.f * Ad;
          sv = -((c2 * Ad) / 12.f);
        }
        kvs[m] = kv;
        svs[m] = sv;
        if (TC && k == src_k && m == src_m) nsig_src = sv;
      }
      if (TC) {
        const float cf[8] = {kvs[0], kvs[1], kvs[2], kvs[3], svs[0], svs[1], svs[2], svs[3]};
        tmem_st8(tc_base + 8u * k, cf);
      } else {
        kap[k][0] = make_float2(kvs[0], kvs[1]);
        kap[k][1] = make_float2(kvs[2], kvs[3]);
        nsig[k][0] = make_float2(svs[0], svs[1]);
        nsig[k][1] = make_float2(svs[2], svs[3]);
      }
      acc[k][0] = acc[k][1] = A[k][0] = A[k][1] = B[k][0] = B[k][1] = make_float2(0.f, 0.f);
    }
    if (TC) tmem_wait_st();
    // Halo rows are pushed inside the row loop.  Injections and the source
    // term are needed only by warps that hold a receiver (or source) cell:
    // the step branches once on this warp-uniform flag into a row loop with
    // that work and one without it, instead of testing it on every row.
    const bool warp_special = __any_sync(0xffffffffu, src_k >= 0 || rec_k >= 0);
    const double v_src = v[(src_r - PAD) * NX + shot_col];
    const float amp = static_cast<float>((v_src / P.amp_ref) * (v_src / P.amp_ref));

    const int tstride = (MODE == SS_MODE_FORWARD) ? NX : NXS;
    float src_acc = 0.f;   // sum_t th(source cell) * w[t]
    float* trace = (MODE == SS_MODE_FORWARD) ? P.gathers + trc_off : P.trace + static_cast<size_t>(slot) * trace_slot;

    // ---- this model's wavelet (one per model: forward and gradient modes),
    // both shared fields zeroed.  Every thread has passed the previous
    // solve's last step barrier, after which nothing reads the staged
    // wavelet; the cluster barrier below orders the new samples before the
    // first step.
    if ((MODE == SS_MODE_FORWARD || MODE == SS_MODE_GRADIENT) && !BATCH && P.wav_stride) {
      const float* wm = P.wav + static_cast<size_t>(b) * P.wav_stride;
      for (int i = tid; i < P.nt; i += nthr) S.wav[i] = wm[i];
    }
    for (size_t i = tid; i < field_floats / 2; i += nthr) {
      reinterpret_cast<float2*>(S.f[0])[i] = make_float2(0.f, 0.f);
      reinterpret_cast<float2*>(S.f[1])[i] = make_float2(0.f, 0.f);
    }
    #pragma unroll 1
    for (int i = tid; i < (H + 4) * RS + H * SW; i += nthr) S.dummy[i] = 0.f;
    cluster_sync();

    // One leapfrog step of the tile.  O1 = own cells at level t (old1), O2 =
    // own cells at t-1 (old2), overwritten with level t+1.  step = index in
    // the loop (0-based), lvl = time index t, cur = step & 1.
    // FWD: source injection, receivers, history of -S (images/gradient).
    // !FWD (adjoint): residual injection, source term, gradient correlation.
    auto tile_step = [&](float2(&O1)[H][2], float2(&O2)[H][2], const int step, const int lvl, const int cur,
                         const bool fwd) {
      const float* X = cur ? S.f[1] : S.f[0];
      float* Y = cur ? S.f[0] : S.f[1];
      const bool more = step + 1 < n_steps;
      const int bi = lvl % kStages;
      if (warp0 && more && tid == 0) {
        if (halo_bytes) mbar_expect_tx(halo_bar0 + 8u * (cur ^ 1), halo_bytes);
        if (!fwd && lvl - (kStages - 1) >= lvl_lo) {   // history slab (and residual row) kStages-1 steps ahead
          const int tn = lvl - (kStages - 1), bn = tn % kStages;
          const uint32_t bar = hist_bar0 + 8u * bn;
          const bool res_here = rank == rec_rank;
          const uint32_t res_bytes = static_cast<uint32_t>(NXS * sizeof(float));
          mbar_expect_tx(bar, stage_bytes + (res_here ? res_bytes : 0u));
          bulk_load(smem_u32(stage_buf(bn)), hist_mine + static_cast<size_t>(tn - lvl_lo) * hist_step, stage_bytes,
                    bar);
          if (res_here) bulk_load(smem_u32(res_buf(bn)), trace + static_cast<size_t>(tn) * NXS, res_bytes, bar);
        }
      }
      if (!BATCH && MODE == SS_MODE_FORWARD && fwd && P.ckpt != nullptr && lvl % P.ckpt_interval == 0) {
        float* ck = P.ckpt + ((static_cast<size_t>(solve) * P.n_ckpt + lvl / P.ckpt_interval) * 2) * P.nzp * P.nxp;
#pragma unroll
        for (int k = 0; k < H; ++k) {
          const int r = myrow + k;
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int c = col0 + m;
            if (active && r < P.nzp - 2 && c < P.nxp - 2) {   // per-thread test inside the uniform branch
              const float2 o2 = O2[k][m >> 1], o1 = O1[k][m >> 1];
              ck[static_cast<size_t>(r) * P.nxp + c] = (m & 1) ? o2.y : o2.x;
              ck[static_cast<size_t>(P.nzp) * P.nxp + static_cast<size_t>(r) * P.nxp + c] = (m & 1) ? o1.y : o1.x;
            }
          }
        }
      }
      // A halo barrier completes one phase per step after the first; every
      // thread follows the phases, and every thread of a warp that holds an
      // edge tile waits (the other lanes would wait for their warp anyway).
      if (warp_edge && step > 0) mbar_wait_bounded(halo_bar0 + 8u * cur, (halo_phase >> cur) & 1u, P.err);
      if (step > 0) halo_phase ^= 1u << cur;
      if (!fwd) {
        mbar_wait_bounded(hist_bar0 + 8u * bi, (hist_phase >> bi) & 1u, P.err);
        hist_phase ^= 1u << bi;
      }
      const bool push_up = more && edge_up, push_dn = more && edge_dn;
      if (!SEG && fwd && rank == rec_rank && step > 0 && warp_recv) {
        // receivers at every model column (gpu.py:134): the level recorded at
        // the previous step is now the read-only field X; one coalesced row
        // straight to global memory per step (a shared ring flushed in bursts
        // held up this CTA, which paces the cluster, every ring-full of steps)
        #pragma unroll 1
        for (int r = tid; r < NX; r += nthr)
          trace[static_cast<size_t>(lvl - 1) * tstride + r] = X[(src_r - row0 + 2) * RS + PAD + r + 2];
      }
      {
        // Lanes without a tile run the same code on a private zero tile
        // (zero coefficients keep it zero), so the loop needs no branch.
        const float wt = fwd ? S.wav[lvl] * amp : S.wav[lvl];
        const float* xc = active ? X + lr0 * RS + o0 : S.dummy;      // tile row -2
        float* yc = active ? Y + (lr0 + 2) * RS + o0 : S.dummy + 2 * RS;   // tile row 0
        const float4 h0 = *reinterpret_cast<const float4*>(xc);
        const float4 h1 = *reinterpret_cast<const float4*>(xc + RS);
        const float4 h2 = *reinterpret_cast<const float4*>(xc + (H + 2) * RS);
        const float4 h3 = *reinterpret_cast<const float4*>(xc + (H + 3) * RS);
        float* const dstg = S.dummy + (H + 4) * RS;
        // forward of an adjoint mode: -S of this step straight to the band's history slab in HBM
        float* stg = (fwd && ADJ) ? hist_mine + static_cast<size_t>(lvl - lvl_lo) * hist_step + lr0 * SW + 4 * cg
                                  : nullptr;
        const float* hl = fwd ? nullptr : (active ? stage_buf(bi) + lr0 * SW + 4 * cg : dstg);
        auto as4 = [](const float2(&r)[2]) { return make_float4(r[0].x, r[0].y, r[1].x, r[1].y); };
        // Every warp computes its rows top-down (a second, bottom-up copy of the
        // row loop for the warps on the lower band edge, so that their halo push
        // left earlier, measured 3.1 % slower: the doubled step code missed the
        // instruction cache).  The source and receiver terms are compiled into
        // the rows of the first branch only (one warp-uniform branch per step
        // instead of one per row).
        // Adjoint, receiver warps: this step's residual at the tile's four
        // columns (zero off the receiver columns), read once for all rows.
        // Forward: this step's source amount at each of the tile's columns.
        float rv0 = 0.f, rv1 = 0.f, rv2 = 0.f, rv3 = 0.f;
        float am0 = 0.f, am1 = 0.f, am2 = 0.f, am3 = 0.f;
        if (warp_special) {
          if (fwd) {
            am0 = (src_m == 0) ? wt : 0.f;
            am1 = (src_m == 1) ? wt : 0.f;
            am2 = (src_m == 2) ? wt : 0.f;
            am3 = (src_m == 3) ? wt : 0.f;
          }
          if (!fwd) {
            const float* rs = res_buf(bi);
            const int rr = col0 - PAD;
            rv0 = (rr >= 0 && rr < NX) ? rs[min(max(rr, 0), NX - 1)] : 0.f;
            rv1 = (rr + 1 >= 0 && rr + 1 < NX) ? rs[min(max(rr + 1, 0), NX - 1)] : 0.f;
            rv2 = (rr + 2 >= 0 && rr + 2 < NX) ? rs[min(max(rr + 2, 0), NX - 1)] : 0.f;
            rv3 = (rr + 3 >= 0 && rr + 3 < NX) ? rs[min(max(rr + 3, 0), NX - 1)] : 0.f;
          }
          {
            float2 lfn = *reinterpret_cast<const float2*>(xc + 2 * RS - 2);
            float2 rtn = *reinterpret_cast<const float2*>(xc + 2 * RS + 4);
#pragma unroll
            for (int k = 0; k < H; ++k) {
              const float2 lf = lfn, rt = rtn;
              if (k + 1 < H) {
                lfn = *reinterpret_cast<const float2*>(xc + (k + 3) * RS - 2);
                rtn = *reinterpret_cast<const float2*>(xc + (k + 3) * RS + 4);
              }
              SS_COEF_ROW(k)
              SS_TILE_ROW(k, true)
            }
          }
          // Adjoint: source-strength term (gpu.py:182) from the source cell's new
          // value, read back from the field this thread just wrote, once per step
          // (in the row loop it cost every row of the receiver warps, which pace
          // the cluster).
          if (!fwd && src_k >= 0) src_acc = fmaf(yc[src_k * RS + src_m], wt, src_acc);
        } else {
          {
            float2 lfn = *reinterpret_cast<const float2*>(xc + 2 * RS - 2);
            float2 rtn = *reinterpret_cast<const float2*>(xc + 2 * RS + 4);
#pragma unroll
            for (int k = 0; k < H; ++k) {
              const float2 lf = lfn, rt = rtn;
              if (k + 1 < H) {
                lfn = *reinterpret_cast<const float2*>(xc + (k + 3) * RS - 2);
                rtn = *reinterpret_cast<const float2*>(xc + (k + 3) * RS + 4);
              }
              SS_COEF_ROW(k)
              SS_TILE_ROW(k, false)
            }
          }
        }
      }
      __syncthreads();
      if (!SEG && fwd && rank == rec_rank && lvl == GNT - 1) {
        // the last level, recorded after the final barrier; the barrier after
        // it publishes every recorded row to the CTA's residual pass
        #pragma unroll 1
        for (int r = tid; r < NX; r += nthr)
          trace[static_cast<size_t>(lvl) * tstride + r] = Y[(src_r - row0 + 2) * RS + PAD + r + 2];
        __syncthreads();
      }
    };

    // Segment mode: the sweep starts from stored fields (a forward checkpoint,
    // or the carried adjoint state) instead of zero; shared field f[0] gets the
    // current level for the whole band and its halo rows straight from them.
    auto load_state = [&](const float* cur_lvl, const float* prev_lvl) {
#pragma unroll 1
      for (int i = tid; i < (P.bh + 4) * RS; i += nthr) {
        const int r = row0 - 2 + i / RS, c = i % RS - 2;
        S.f[0][i] = (r >= 0 && r < P.nzp - 2 && c >= 0 && c < P.nxp - 2) ? cur_lvl[static_cast<size_t>(r) * P.nxp + c] : 0.f;
      }
#pragma unroll
      for (int k = 0; k < H; ++k) {
        float a[4], p[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int r = myrow + k, c = col0 + m;
          const bool in = active && r < P.nzp - 2 && c < P.nxp - 2;
          a[m] = in ? cur_lvl[static_cast<size_t>(r) * P.nxp + c] : 0.f;
          p[m] = in ? prev_lvl[static_cast<size_t>(r) * P.nxp + c] : 0.f;
        }
        A[k][0] = make_float2(a[0], a[1]);
        A[k][1] = make_float2(a[2], a[3]);
        B[k][0] = make_float2(p[0], p[1]);
        B[k][1] = make_float2(p[2], p[3]);
      }
    };
    if (SEG) {
      const size_t fld = static_cast<size_t>(P.nzp) * P.nxp;
      const float* ck = P.ckpt + (static_cast<size_t>(solve) * P.n_ckpt + P.seg_index) * 2 * fld;
      load_state(ck + fld, ck);   // (p[s], p[s-1])
      cluster_sync();
    }

    // ================= forward: t = lvl_lo .. lvl_hi ======================
    {
      int i = 0;
      for (; i + 1 < n_steps; i += 2) {
        tile_step(A, B, i, lvl_lo + i, 0, true);
        tile_step(B, A, i + 1, lvl_lo + i + 1, 1, true);
      }
      if (i < n_steps) tile_step(A, B, i, lvl_lo + i, 0, true);
    }

    if (MODE == SS_MODE_FORWARD) continue;

    // ---- forward epilogue: illumination = sum_t (S/12)^2 on model cells --
    fence_proxy_async_all();   // every thread's history stores, before the adjoint's bulk loads read them
    {
      float* il = P.illum + out_off;
#pragma unroll
      for (int k = 0; k < H; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int z = myrow + k - PAD, x = col0 + m - PAD;
          const float a = (m & 1) ? acc[k][m >> 1].y : acc[k][m >> 1].x;
          if (active && z >= 0 && z < GNZ && x >= 0 && x < NX) {
            if (SEG)
              P.illum_acc[static_cast<size_t>(solve) * P.nz * NX + z * NX + x] += a;
            else
              il[z * NX + x] = a * (1.f / 144.f);
          }
        }
#pragma unroll
      for (int k = 0; k < H; ++k)
        acc[k][0] = acc[k][1] = A[k][0] = A[k][1] = B[k][0] = B[k][1] = make_float2(0.f, 0.f);
    }
    // ---- residual (sim - obs) * mute, in place over the trace ------------
    // the receiver CTA's recorded rows, visible to every CTA of the cluster
    cluster_sync();
    if (SEG && rank == rec_rank) {   // segment mode: the adjoint source is given
      const float* rg = P.res_in + static_cast<size_t>(solve) * P.nt * NX;
#pragma unroll 1
      for (int i = tid; i < n_steps * NX; i += nthr) {
        const int t = lvl_lo + i / NX, r = i % NX;
        trace[t * NXS + r] = rg[static_cast<size_t>(t) * NX + r];
      }
      fence_proxy_async_all();
      __syncthreads();
    } else if (!SEG) {
      // every CTA of the cluster takes a contiguous share of the receiver CTA's
      // trace (one CTA alone kept the others waiting at the next cluster
      // barrier); the fence and that barrier publish the rows to the receiver
      // CTA's bulk copies.  (Segment mode has no observations: its adjoint
      // source comes in res_in and only the receiver CTA copies it, above.)
      const float* ob = P.obs + trc_off;
      const float vm = v_mute;
      const int total = GNT * NX, share = (total + P.C - 1) / P.C;
      const int i1 = min(total, (rank + 1) * share);
      for (int i = rank * share + tid; i < i1; i += nthr) {
        const int t = i / NX, r = i - t * NX;
        const float o = ob[i];
        if (!isfinite(o)) atomicExch(P.err, static_cast<int>(SS_ERR_NONFINITE));
        float res = trace[t * NXS + r] - o;
        if (muted) res *= mute_weight(t, r, shot_col, P.dx, P.dt, vm, P.t_mute);
        trace[t * NXS + r] = res;
      }
      fence_proxy_async_all();   // these rows are read back by bulk copies
      __syncthreads();
    }

    // ================= adjoint: t = lvl_hi .. lvl_lo ======================
    for (size_t i = tid; i < field_floats / 2; i += nthr) {
      reinterpret_cast<float2*>(S.f[0])[i] = make_float2(0.f, 0.f);
      reinterpret_cast<float2*>(S.f[1])[i] = make_float2(0.f, 0.f);
    }
    float* th_io = SEG ? P.theta + static_cast<size_t>(solve) * 2 * P.nzp * P.nxp : nullptr;
    if (SEG) {
      __syncthreads();   // the zeroing above and load_state map threads to f[0] differently
      load_state(th_io, th_io + static_cast<size_t>(P.nzp) * P.nxp);   // (th[e+1], th[e+2])
    }
    cluster_sync();
    if (tid == 0) {   // history slabs and residual rows of the first kStages-1 adjoint steps
      for (int tn = lvl_hi; tn >= lvl_lo && tn > lvl_hi - (kStages - 1); --tn) {
        const int bn = tn % kStages;
        const uint32_t bar = hist_bar0 + 8u * bn;
        const bool res_here = rank == rec_rank;
        const uint32_t res_bytes = static_cast<uint32_t>(NXS * sizeof(float));
        mbar_expect_tx(bar, stage_bytes + (res_here ? res_bytes : 0u));
        bulk_load(smem_u32(stage_buf(bn)), hist_mine + static_cast<size_t>(tn - lvl_lo) * hist_step, stage_bytes,
                  bar);
        if (res_here) bulk_load(smem_u32(res_buf(bn)), trace + static_cast<size_t>(tn) * NXS, res_bytes, bar);
      }
    }
    {
      int i = 0;
      for (; i + 1 < n_steps; i += 2) {
        tile_step(A, B, i, lvl_hi - i, 0, false);
        tile_step(B, A, i + 1, lvl_hi - 1 - i, 1, false);
      }
      if (i < n_steps) tile_step(A, B, i, lvl_hi - i, 0, false);
    }
    if (SEG) {
      // carry the adjoint state (th[s], th[s+1]) and the accumulators to the next segment
      const size_t fld = static_cast<size_t>(P.nzp) * P.nxp;
      float* g = P.gacc + static_cast<size_t>(solve) * fld;
#pragma unroll
      for (int k = 0; k < H; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int r = myrow + k, c = col0 + m;
          if (active && r < P.nzp - 2 && c < P.nxp - 2) {
            const size_t o = static_cast<size_t>(r) * P.nxp + c;
            const float a = (m & 1) ? A[k][m >> 1].y : A[k][m >> 1].x;
            const float bv = (m & 1) ? B[k][m >> 1].y : B[k][m >> 1].x;
            th_io[o] = (n_steps & 1) ? bv : a;          // newest level, th[s]
            th_io[fld + o] = (n_steps & 1) ? a : bv;    // th[s+1]
            g[o] += (m & 1) ? acc[k][m >> 1].y : acc[k][m >> 1].x;
          }
        }
      if (src_k >= 0) P.src_acc_io[solve] += src_acc;
      __threadfence();
      cluster_sync();
      continue;
    }

    // ---- padded gradient 2/v * sum_t th*S(p), plus the source term -------
    // acc holds -sum_t th*S (the history holds -S); nsig = -sigma.
    float* gp = P.gpad + static_cast<size_t>(slot) * (BATCH ? P.gpad_slot : static_cast<size_t>(P.nzp) * P.nxp);
    if (active) {
#pragma unroll
      for (int k = 0; k < H; ++k)
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const int r = myrow + k, c = col0 + m;
          if (r < GNZP - 2 && c < GNXP - 2) {
            const int vz = min(max(r - PAD, 0), GNZ - 1), vx = min(max(c - PAD, 0), NX - 1);
            const float vp = v[vz * NX + vx];
            const float a = (m & 1) ? acc[k][m >> 1].y : acc[k][m >> 1].x;
            float gval = -2.f * a / vp;
            if (k == src_k && m == src_m) {
              const float deriv = static_cast<float>(2.0 * v_src / (P.amp_ref * P.amp_ref));
              const float ns = TC ? nsig_src : ((m & 1) ? nsig[k][m >> 1].y : nsig[k][m >> 1].x);
              gval += src_acc * deriv / -ns;
            }
            gp[static_cast<size_t>(r) * GNXP + c] = gval;
          }
        }
    }
    __threadfence();
    cluster_sync();
    {
      float* go = P.grad_per_slot ? P.grad + static_cast<size_t>(slot) * (BATCH ? P.grad_slot : static_cast<size_t>(P.nz) * P.nx)
                                  : P.grad + out_off;
      epilogue<MODE>(P, S, gp, go, P.illum + out_off, P.img + out_off, GNZ, NX, PAD, GNZP, GNXP, rank, tid, nthr);
    }
    __threadfence();
    cluster_sync();   // scratch of this slot is free for the next solve
  }
  if (TC) tmem_fence_before();
  cluster_sync();     // no CTA leaves while a neighbour may still write its shared memory
  if (TC && tid < 32) {
    tmem_fence_after();
    tmem_dealloc_warp(*reinterpret_cast<const uint32_t*>(&S.bar[kStages + 2]), kCoefCols);
  }
}

#undef RS
#undef NX
#undef PAD
#undef SW
#undef NXS
#undef GNZ
#undef GNT
#undef GNZP
#undef GNXP
#undef GBH
#undef GNCG
#undef GNSEG
#undef GNACT

// ----------------------------------------------------------------------------
// Small helper kernels (module-level functions of the reference)
// ----------------------------------------------------------------------------
template <typename T>
__global__ void lap_kernel(const T* __restrict__ p, T* __restrict__ out, long long batch, int n0, int n1) {
  const long long total = batch * n0 * n1;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx % n1);
    const int i = static_cast<int>((idx / n1) % n0);
    T val = T(0);
    if (i >= 2 && i < n0 - 2 && j >= 2 && j < n1 - 2) {
      const T* q = p + idx;
      const T c = q[0];
      const T z = -q[-2 * n1] + T(16) * q[-n1] - T(30) * c + T(16) * q[n1] - q[2 * n1];
      const T x = -q[-2] + T(16) * q[-1] - T(30) * c + T(16) * q[1] - q[2];
      val = (z + x) / T(12);
    }
    out[idx] = val;
  }
}

template <typename T>
__global__ void lap_adjoint_kernel(const T* __restrict__ p, T* __restrict__ out, long long batch, int n0, int n1) {
  // Gather form of the scatter in gpu.py:40-53: out = S(M p)/12, M = interior mask.
  const long long total = batch * n0 * n1;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx % n1);
    const int i = static_cast<int>((idx / n1) % n0);
    auto q = [&](int di, int dj) -> T {
      const int ii = i + di, jj = j + dj;
      if (ii < 2 || ii >= n0 - 2 || jj < 2 || jj >= n1 - 2) return T(0);
      return p[idx + static_cast<long long>(di) * n1 + dj] / T(12);
    };
    T val = -T(60) * q(0, 0);
    val += -q(-2, 0) + T(16) * q(-1, 0) + T(16) * q(1, 0) - q(2, 0);
    val += -q(0, -2) + T(16) * q(0, -1) + T(16) * q(0, 1) - q(0, 2);
    out[idx] = val;
  }
}

template <typename T>
__global__ void fold_kernel(const T* __restrict__ g, T* __restrict__ out, long long batch, int nz, int nx, int pad) {
  const int nzp = nz + 2 * pad, nxp = nx + 2 * pad;
  const long long total = batch * nz * nx;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(idx % nx);
    const int z = static_cast<int>((idx / nx) % nz);
    const T* G = g + (idx / (static_cast<long long>(nz) * nx)) * nzp * nxp;
    auto at = [&](int i, int j) -> T { return G[static_cast<long long>(i) * nxp + j]; };
    const int i = pad + z, j = pad + x;
    T val = at(i, j);
    const int zi0 = z == 0 ? 0 : (z == nz - 1 ? pad + nz : -1), zi1 = z == 0 ? pad : nzp;
    const int xj0 = x == 0 ? 0 : (x == nx - 1 ? pad + nx : -1), xj1 = x == 0 ? pad : nxp;
    if (zi0 >= 0)
      for (int ii = zi0; ii < zi1; ++ii) val += at(ii, j);
    if (xj0 >= 0)
      for (int jj = xj0; jj < xj1; ++jj) val += at(i, jj);
    if (zi0 >= 0 && xj0 >= 0)
      for (int ii = zi0; ii < zi1; ++ii)
        for (int jj = xj0; jj < xj1; ++jj) val += at(ii, jj);
    out[idx] = val;
  }
}

__global__ void mute_kernel(float* __restrict__ out, const float* __restrict__ vmute, int n_models, int n_shots, int nt,
                            int nx, KParams P) {
  const long long total = static_cast<long long>(n_models) * n_shots * nt * nx;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(idx % nx);
    const int t = static_cast<int>((idx / nx) % nt);
    const int s = static_cast<int>((idx / (static_cast<long long>(nx) * nt)) % n_shots);
    const int b = static_cast<int>(idx / (static_cast<long long>(nx) * nt * n_shots));
    out[idx] = mute_weight(t, r, P.shot_cols[s], P.dx, P.dt, vmute[b], P.t_mute);
  }
}

__global__ void c2_kernel(const float* __restrict__ vel, float* __restrict__ out, int n_models, int nz, int nx, int pad,
                          double dtdx2) {
  const int nzp = nz + 2 * pad, nxp = nx + 2 * pad;
  const long long total = static_cast<long long>(n_models) * nzp * nxp;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(idx % nxp);
    const int i = static_cast<int>((idx / nxp) % nzp);
    const long long b = idx / (static_cast<long long>(nzp) * nxp);
    const int vz = min(max(i - pad, 0), nz - 1), vx = min(max(j - pad, 0), nx - 1);
    const double vp = vel[b * nz * nx + vz * nx + vx];
    out[idx] = static_cast<float>(vp * vp * dtdx2);
  }
}

// Gradient from the segment accumulators: g_pad = -2 gacc / v on interior
// cells plus the source-strength term, folded onto the model edges
// (gpu.py:56-67, 185-187); illumination = sum S^2 / 144.
__global__ void finish_kernel(KParams P, const float* __restrict__ gacc, const float* __restrict__ src_acc,
                              const float* __restrict__ illum_acc, float* __restrict__ grad, float* __restrict__ illum) {
  const long long total = static_cast<long long>(P.n_solves) * P.nz * P.nx;
  const int nzp = P.nzp, nxp = P.nxp, pad = P.pad;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(idx % P.nx);
    const int z = static_cast<int>((idx / P.nx) % P.nz);
    const int solve = static_cast<int>(idx / (static_cast<long long>(P.nz) * P.nx));
    const int b = solve / P.n_shots, s = solve - b * P.n_shots;
    const float* v = P.vel + static_cast<size_t>(b) * P.nz * P.nx;
    const float* G = gacc + static_cast<size_t>(solve) * nzp * nxp;
    auto at = [&](int i, int j) -> float {
      if (i < 2 || i >= nzp - 2 || j < 2 || j >= nxp - 2) return 0.f;
      const int vz = min(max(i - pad, 0), P.nz - 1), vx = min(max(j - pad, 0), P.nx - 1);
      return -2.f * G[static_cast<size_t>(i) * nxp + j] / v[vz * P.nx + vx];
    };
    const int i = pad + z, j = pad + x;
    float val = at(i, j);
    const int zi0 = z == 0 ? 0 : (z == P.nz - 1 ? pad + P.nz : -1), zi1 = z == 0 ? pad : nzp;
    const int xj0 = x == 0 ? 0 : (x == P.nx - 1 ? pad + P.nx : -1), xj1 = x == 0 ? pad : nxp;
    if (zi0 >= 0)
      for (int ii = zi0; ii < zi1; ++ii) val += at(ii, j);
    if (xj0 >= 0)
      for (int jj = xj0; jj < xj1; ++jj) val += at(i, jj);
    if (zi0 >= 0 && xj0 >= 0)
      for (int ii = zi0; ii < zi1; ++ii)
        for (int jj = xj0; jj < xj1; ++jj) val += at(ii, jj);
    if (z == P.src_row && x == P.shot_cols[s]) {   // source-strength derivative (gpu.py:182,187)
      const double vs = v[P.src_row * P.nx + x];
      const double dz = layer_depth(i, nzp, pad), dxl = layer_depth(j, nxp, pad);
      const float Ad = static_cast<float>(1.0 / (1.0 + P.damp_k * (dz * dz + dxl * dxl)));
      const float c2 = static_cast<float>(vs * vs * P.dtdx2);
      const float sigma = (c2 * Ad) / 12.f;
      const float deriv = static_cast<float>(2.0 * vs / (P.amp_ref * P.amp_ref));
      val += src_acc[solve] * deriv / sigma;
    }
    grad[idx] = val;
    illum[idx] = illum_acc[idx] * (1.f / 144.f);
  }
}

// Failure-detection probe: the solve kernel's bounded mbarrier wait on a
// barrier that nothing arrives on.  It must give up after `limit_ns`, record
// SS_ERR_TIMEOUT and return, leaving the context usable.
__global__ void wait_probe_kernel(int* status, unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(smem_u32(&bar), 1);
  __syncthreads();
  mbar_wait_bounded(smem_u32(&bar), 0u, status, limit_ns);
}

// FP32 throughput probe: 8 independent FMA chains per thread, scalar or
// packed FP32x2, for the roofline denominator of the stencil kernels.
template <bool PACKED>
__global__ void __launch_bounds__(256) fp32_probe_kernel(float* out, int iters) {
  float2 a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = make_float2(threadIdx.x * 1e-3f + j, j * 0.5f);
  const float2 m = make_float2(0.999999f, 0.999998f), c = make_float2(1e-6f, 2e-6f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (PACKED) {
        a[j] = __ffma2_rn(a[j], m, c);
      } else {
        a[j].x = fmaf(a[j].x, m.x, c.x);
        a[j].y = fmaf(a[j].y, m.y, c.y);
      }
    }
  }
  float acc = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) acc += a[j].x + a[j].y;
  if (acc == 12345.678f) out[0] = acc;   // keeps the chains live; practically never stores
}

// ----------------------------------------------------------------------------
// Host side: plans, workspace, launches
// ----------------------------------------------------------------------------
struct Plan {
  int nzp, nxp, ncg, nseg, bh, C, rs, sw, threads, H;
  bool fast;
  size_t smem;
  int max_clusters;
  int slots;
};

int check_geometry(const ss_geometry* g) {
  if (!g) return fail(SS_ERR_INVALID, "geometry pointer is NULL");
  if (g->nz < 1 || g->nx < 1 || g->nt < 1) return fail(SS_ERR_INVALID, "nz, nx and nt must be positive");
  if (g->pad < 2) return fail(SS_ERR_INVALID, "pad must be >= 2");
  if (g->n_shots < 1 || g->n_shots > SS_MAX_SHOTS) return fail(SS_ERR_INVALID, "n_shots must lie in 1..16");
  if (g->src_row < 0 || g->src_row >= g->nz) return fail(SS_ERR_INVALID, "src_row outside the model");
  for (int s = 0; s < g->n_shots; ++s)
    if (g->shot_cols[s] < 0 || g->shot_cols[s] >= g->nx) return fail(SS_ERR_INVALID, "shot column outside the model");
  if (!(g->dx > 0.0) || !(g->dt > 0.0) || !(g->r_coef > 0.0) || !(g->r_coef < 1.0) || !(g->vmax_damping > 0.0) ||
      !(g->amp_ref > 0.0))
    return fail(SS_ERR_INVALID, "dx, dt, vmax_damping and amp_ref must be positive and 0 < r_coef < 1");
  return SS_OK;
}

using SolveFn = void (*)(KParams);

// The OpenFWI geometry (nx = 70, pad = 40) gets an instantiation with
// compile-time strides; every other geometry takes them from KParams.
bool fast_geometry(int nx, int pad) { return nx == 70 && pad == 40; }

// Tile heights with fixed-geometry instantiations, and with batch ones.
bool fixed_rows_ok(int H) { return H == 4 || H == 5; }
bool batch_rows_ok(int H) { return H >= 4 && H <= 6; }

template <int H>
SolveFn kernel_for_rows(int mode, bool fast) {
  switch (mode) {
    case SS_MODE_FORWARD:
      return fast ? solve_kernel<SS_MODE_FORWARD, true, false, H> : solve_kernel<SS_MODE_FORWARD, false, false, H>;
    case SS_MODE_GRADIENT:
      return fast ? solve_kernel<SS_MODE_GRADIENT, true, false, H> : solve_kernel<SS_MODE_GRADIENT, false, false, H>;
    case SS_MODE_SEGMENT:
      return fast ? solve_kernel<SS_MODE_SEGMENT, true, false, H> : solve_kernel<SS_MODE_SEGMENT, false, false, H>;
    default: return fast ? solve_kernel<SS_MODE_IMAGES, true, false, H> : solve_kernel<SS_MODE_IMAGES, false, false, H>;
  }
}
SolveFn kernel_for(int mode, bool fast, int H) {
  return H == 4 ? kernel_for_rows<4>(mode, fast) : kernel_for_rows<5>(mode, fast);
}

// Uneven batches: one generic instantiation per mode and tile height, geometry per solve.
template <int H>
SolveFn batch_kernel_rows(int mode) {
  switch (mode) {
    case SS_MODE_FORWARD: return solve_kernel<SS_MODE_FORWARD, false, true, H>;
    case SS_MODE_GRADIENT: return solve_kernel<SS_MODE_GRADIENT, false, true, H>;
    default: return solve_kernel<SS_MODE_IMAGES, false, true, H>;
  }
}
SolveFn batch_kernel_for(int mode, int H) {
  return H == 4 ? batch_kernel_rows<4>(mode) : H == 6 ? batch_kernel_rows<6>(mode) : batch_kernel_rows<5>(mode);
}

// Tile height of fixed-geometry plans per mode (0: the default), set by a
// caller's tuner through ss_set_rows_per_thread.
std::atomic<int> g_rows_pref[4] = {{0}, {0}, {0}, {0}};
int rows_for_mode(int mode) {
  const int r = (mode >= 0 && mode < 4) ? g_rows_pref[mode].load() : 0;
  return fixed_rows_ok(r) ? r : kDefaultRows;
}

size_t smem_bytes(int bh, int rs, int sw, int nt, int nxs, bool adj, int H, bool fast) {
  const int slabs = fast ? kStagesFast : kStagesGeneric;   // what solve_kernel<.., fast, false, ..> lays out
  const size_t field = static_cast<size_t>(bh + 4) * rs;
  const size_t stage = adj ? static_cast<size_t>(bh) * sw : 0;
  return (2 * field + slabs * stage + ((nt + 31) & ~31) + 32 +
          slabs * static_cast<size_t>(nxs) + (H + 4) * static_cast<size_t>(rs) +
          H * static_cast<size_t>(sw)) *
             sizeof(float) +
         (slabs + 3) * sizeof(uint64_t);   // barriers, then the TMEM address word
}

// The band plan of a geometry: cluster size, band height, threads and shared
// memory (arithmetic only; make_plan adds what the device can hold at once).
int plan_shape(const ss_geometry* g, int mode, Plan* p) {
  const int H = rows_for_mode(mode);
  p->H = H;
  const bool adj = mode != SS_MODE_FORWARD;
  p->nzp = g->nz + 2 * g->pad;
  p->nxp = g->nx + 2 * g->pad;
  p->ncg = (p->nxp - 4 + 3) / 4;
  p->rs = 4 * p->ncg + 8;
  p->sw = 4 * p->ncg;
  const int nrows = p->nzp - 4;
  const int max_nseg = max_threads_for(H) / p->ncg;
  if (max_nseg < 1) return fail(SS_ERR_UNSUPPORTED, "model too wide for one band of threads");
  bool ok = false;
  for (int C = std::max(1, (nrows + max_nseg * H - 1) / (max_nseg * H)); C <= kMaxCluster; ++C) {
    const int nseg = (nrows + C * H - 1) / (C * H);
    if (C > 1 && nseg < 1) break;
    const int bh = nseg * H;
    if (C > 1 && bh < 2) continue;
    const size_t sm = smem_bytes(bh, p->rs, p->sw, g->nt, (g->nx + 3) & ~3, adj, H, fast_geometry(g->nx, g->pad));
    if (sm <= kMaxSmem) {
      p->C = C;
      p->nseg = nseg;
      p->bh = bh;
      p->smem = sm;
      ok = true;
      break;
    }
  }
  if (!ok) return fail(SS_ERR_UNSUPPORTED, "no cluster plan fits shared memory for this grid");
  p->threads = ((p->ncg * p->nseg + 31) / 32) * 32;
  p->smem = std::max(p->smem, kTcMinSmem);
  p->fast = fast_geometry(g->nx, g->pad);
  p->max_clusters = 0;
  p->slots = 1;
  return SS_OK;
}

int make_plan(const ss_geometry* g, int mode, int n_solves, Plan* p) {
  int rc = plan_shape(g, mode, p);
  if (rc) return rc;
  const void* fn = reinterpret_cast<const void*>(kernel_for(mode, p->fast, p->H));
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p->smem));
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  if (p->C > 8) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("non-portable cluster: ") + cudaGetErrorString(e));
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p->C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(p->C, 1, 1);
  cfg.blockDim = dim3(p->threads, 1, 1);
  cfg.dynamicSmemBytes = p->smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int nclusters = 0;
  e = cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaOccupancyMaxActiveClusters: ") + cudaGetErrorString(e));
  if (nclusters < 1) return fail(SS_ERR_UNSUPPORTED, "no cluster of this plan fits on the device");
  p->max_clusters = nclusters;
  p->slots = std::max(1, std::min(nclusters, n_solves));
  return SS_OK;
}

inline size_t align_up(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct WsLayout {
  size_t err, hist, trace, gpad, grad, total;
};

WsLayout ws_layout(const ss_geometry* g, const Plan& p, int mode, int hist_steps = -1) {
  if (hist_steps < 0) hist_steps = g->nt;
  WsLayout w{};
  size_t off = 0;
  w.err = off;
  off = align_up(off + 256);
  if (mode != SS_MODE_FORWARD) {
    w.hist = off;
    off = align_up(off + static_cast<size_t>(p.slots) * hist_steps * p.C * p.bh * p.sw * sizeof(float));
    w.trace = off;
    off = align_up(off + static_cast<size_t>(p.slots) * g->nt * ((g->nx + 3) & ~3) * sizeof(float));
    w.gpad = off;
    off = align_up(off + static_cast<size_t>(p.slots) * std::max(p.nzp * p.nxp, g->nz * g->nx) * sizeof(float));
    w.grad = off;
    off = align_up(off + static_cast<size_t>(p.slots) * g->nz * g->nx * sizeof(float));
  }
  w.total = off;
  return w;
}

// The most solves in flight whose scratch fits `bytes` (0: not even one).
// The layout grows monotonically with the slots (each region is 256-byte
// aligned, so the growth per slot varies by a few bytes): binary search.
int slots_for_bytes(const ss_geometry* g, Plan p, int mode, size_t bytes) {
  auto total = [&](int n) {
    p.slots = n;
    return ws_layout(g, p, mode).total;
  };
  if (total(1) > bytes) return 0;
  constexpr int kCap = 1 << 24;
  if (total(kCap) <= bytes) return kCap;   // forward mode: no per-slot scratch
  int lo = 1, hi = kCap;                    // total(lo) <= bytes < total(hi)
  while (hi - lo > 1) {
    const int mid = lo + (hi - lo) / 2;
    if (total(mid) <= bytes) lo = mid;
    else hi = mid;
  }
  return lo;
}

KParams base_params(const ss_geometry* g, const Plan& p, int n_models) {
  KParams k{};
  k.nz = g->nz;
  k.nx = g->nx;
  k.nt = g->nt;
  k.pad = g->pad;
  k.nzp = p.nzp;
  k.nxp = p.nxp;
  k.n_shots = g->n_shots;
  k.src_row = g->src_row;
  for (int s = 0; s < SS_MAX_SHOTS; ++s) k.shot_cols[s] = s < g->n_shots ? g->shot_cols[s] : 0;
  const double dtdx = g->dt / g->dx;
  k.dtdx2 = dtdx * dtdx;
  k.damp_k = 3.0 * g->vmax_damping / (2.0 * g->pad * g->dx) * std::log(1.0 / g->r_coef) * g->dt / 2.0;
  k.amp_ref = g->amp_ref;
  k.dx = static_cast<float>(g->dx);
  k.dt = static_cast<float>(g->dt);
  k.ncg = p.ncg;
  k.nseg = p.nseg;
  k.bh = p.bh;
  k.C = p.C;
  k.rs = p.rs;
  k.sw = p.sw;
  k.nact = p.ncg * p.nseg;
  k.nxs = (g->nx + 3) & ~3;
  k.n_solves = n_models * g->n_shots;
  k.hist_steps = g->nt;
  return k;
}

int launch(const Plan& p, int mode, const KParams& k, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = p.C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(p.C * p.slots, 1, 1);
  cfg.blockDim = dim3(p.threads, 1, 1);
  cfg.dynamicSmemBytes = p.smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel_for(mode, p.fast, p.H), k);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaLaunchKernelEx: ") + cudaGetErrorString(e));
  return SS_OK;
}

int run_adjoint(int mode, const ss_geometry* g, int n_models, const float* vel, const float* wavelet, const float* obs,
                const float* v_mute, float t_mute, float eps, int laplacian, float* img, float* illum, float* grad,
                void* ws, size_t ws_bytes, void* stream, long long wav_stride = 0) {
  NvtxRange range(mode == SS_MODE_IMAGES ? "ss_images" : "ss_gradient");
  g_last_error.clear();
  int rc = check_geometry(g);
  if (rc) return rc;
  if (n_models < 1) return fail(SS_ERR_INVALID, "n_models must be positive");
  if (!vel || !wavelet || !obs || !illum) return fail(SS_ERR_INVALID, "vel, wavelet, obs and illum are required");
  if (mode == SS_MODE_GRADIENT && !grad) return fail(SS_ERR_INVALID, "grad output is required");
  if (mode == SS_MODE_IMAGES && !img) return fail(SS_ERR_INVALID, "img output is required");
  if (!(eps > 0.f) && mode == SS_MODE_IMAGES) return fail(SS_ERR_INVALID, "illumination regularization eps must be positive");
  Plan p;
  rc = make_plan(g, mode, n_models * g->n_shots, &p);
  if (rc) return rc;
  // A workspace smaller than the full plan's keeps fewer solves in flight.
  p.slots = std::min(p.slots, slots_for_bytes(g, p, mode, ws ? ws_bytes : 0));
  if (p.slots < 1) return fail(SS_ERR_WORKSPACE, "workspace missing or too small for one solve in flight");
  const WsLayout L = ws_layout(g, p, mode);
  unsigned char* w = static_cast<unsigned char*>(ws);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SS_CUDA(cudaMemsetAsync(w + L.err, 0, 256, st));
  KParams k = base_params(g, p, n_models);
  k.vel = vel;
  k.wav = wavelet;
  k.wav_stride = wav_stride;
  k.obs = obs;
  k.vmute = v_mute;
  k.t_mute = t_mute;
  k.trace = reinterpret_cast<float*>(w + L.trace);
  k.illum = illum;
  k.grad_per_slot = grad == nullptr;
  k.grad = grad ? grad : reinterpret_cast<float*>(w + L.grad);
  k.img = img;
  k.gpad = reinterpret_cast<float*>(w + L.gpad);
  k.hist = reinterpret_cast<float*>(w + L.hist);
  k.eps = eps;
  k.laplacian = laplacian;
  k.err = reinterpret_cast<int*>(w + L.err);
  k.ckpt_interval = 1;
  return launch(p, mode, k, st);
}

int grid_for(long long total) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
}

// ----------------------------------------------------------------------------
// Allocation-free images: scratch in a file-scope device array
// ----------------------------------------------------------------------------
// Some callers cannot allocate device memory when they call us: a plugin
// host that hands out only input/output buffers, a framework whose caching
// allocator owns all device memory, or a process that must not allocate
// after start-up.  ss_images_noalloc serves them with the images kernel and
// a fixed 32 MiB scratch array that every GPU loading this library holds
// until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void* g_noalloc_address[64] = {};   // device address of g_noalloc_scratch, per device index

// Device address of the scratch array on the current device.  The first call
// on a device looks it up with cudaGetSymbolAddress (the host-side name of the
// array is only a stand-in, not a device address) and caches it.
int noalloc_scratch(void** out) {
  int dev = 0;
  SS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS_ERR_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (g_noalloc_address[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(SS_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_noalloc_address[dev] = p;
  }
  *out = g_noalloc_address[dev];
  return SS_OK;
}

// ----------------------------------------------------------------------------
// Uneven batches: planner (host) and runner
// ----------------------------------------------------------------------------
// A plan is one contiguous blob, identical in host and device memory:
// BatchPlanHeader, then BatchItemDev[n_items], then int order[n_solves]
// (per class, solves longest-first).  The header carries the launch shapes.
constexpr uint64_t kPlanMagic = 0x3430504853535342ull;   // "BSSSHP04"
constexpr int kMaxClasses = 32;   // (cluster size, tile height) pairs of one plan

struct BatchClassHost {
  int C, H, min_C, threads, slots, smem, stream, n_solves, order_begin, nt_max, nxs, bh_max, counter;
  int max_clusters, idle_sms;   // co-resident clusters alone on the GPU, and the SMs they leave idle
  size_t hist_slot, trace_slot, gpad_slot, grad_slot;   // floats per slot
  size_t ws_off;                                        // bytes: this class's scratch in the workspace
  double cell_steps;
};

struct BatchPlanHeader {
  uint64_t magic;
  int32_t mode, n_items, n_solves, n_classes, max_nt, concurrent;
  int64_t total_bytes, ws_bytes, items_off, order_off;
  double dtdx2, amp_ref, dx, dt;
  BatchClassHost cls[kMaxClasses];
};

// Shared memory of a batch launch: the fixed part (barriers, wavelet,
// reduction words, residual rows) and one solve's part
// (two fields, the history slabs, the zero tile).
size_t batch_fixed_smem(int nt_max, int nxs) {
  return (16 + static_cast<size_t>((nt_max + 31) & ~31) + 32 + static_cast<size_t>(kStagesGeneric) * nxs) *
         sizeof(float);
}
size_t batch_solve_smem(int bh, int ncg, bool adj, int H) {
  const size_t rs = 4 * static_cast<size_t>(ncg) + 8, sw = 4 * static_cast<size_t>(ncg);
  return (2 * (bh + 4) * rs + (adj ? kStagesGeneric * bh * sw : 0) + (H + 4) * rs + H * sw) * sizeof(float);
}

int item_ncg(const ss_batch_item& it) { return (it.nx + 2 * it.pad - 4 + 3) / 4; }

struct ItemShape {
  int nseg, bh, nact;
};
// Band shape of one item at cluster size C and tile height H; nact >
// max_threads_for(H) means it does not fit.
ItemShape item_shape(const ss_batch_item& it, int C, int H) {
  const int nrows = it.nz + 2 * it.pad - 4;
  const int ncg = item_ncg(it);
  ItemShape s;
  s.nseg = (nrows + C * H - 1) / (C * H);
  s.bh = s.nseg * H;
  s.nact = ncg * s.nseg;
  return s;
}
bool item_fits(const ss_batch_item& it, int C, bool adj, int H = kDefaultRows) {
  const ItemShape s = item_shape(it, C, H);
  const int ncg = item_ncg(it);
  return s.nact <= max_threads_for(H) &&
         batch_fixed_smem(it.nt, (it.nx + 3) & ~3) + batch_solve_smem(s.bh, ncg, adj, H) <= kMaxSmem;
}

struct DeviceStreams {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_stream_mutex;
DeviceStreams g_streams[64];

// The library's second stream and its fork/join events on the current device,
// created once (plan time, so that runs under stream capture create nothing).
int device_streams(DeviceStreams** out) {
  int dev = 0;
  SS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS_ERR_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lock(g_stream_mutex);
  DeviceStreams& d = g_streams[dev];
  if (!d.side) {
    SS_CUDA(cudaStreamCreateWithFlags(&d.side, cudaStreamNonBlocking));
    SS_CUDA(cudaEventCreateWithFlags(&d.fork, cudaEventDisableTiming));
    SS_CUDA(cudaEventCreateWithFlags(&d.join, cudaEventDisableTiming));
  }
  *out = &d;
  return SS_OK;
}

// Dynamic shared memory limit of a batch instantiation on the current
// device, raised (never lowered) as plans need more; a run whose plan set it
// already makes no attribute call.
std::mutex g_attr_mutex;
int g_batch_smem[64][3][kMaxRows + 1] = {};
int ensure_batch_smem(int mode, int H, int bytes) {
  int dev = 0;
  SS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS_ERR_UNSUPPORTED, "device index beyond 63");
  if (!batch_rows_ok(H)) return fail(SS_ERR_INVALID, "rows per thread of a batch class must lie in 4..6");
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  int& cur = g_batch_smem[dev][mode][H];
  if (bytes <= cur) return SS_OK;
  const void* fn = reinterpret_cast<const void*>(batch_kernel_for(mode, H));
  SS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  SS_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cur = bytes;
  return SS_OK;
}

int check_item(const ss_batch_item& it, int i) {
  const std::string at = "item " + std::to_string(i) + ": ";
  if (it.nz < 1 || it.nx < 1 || it.nt < 1) return fail(SS_ERR_INVALID, at + "nz, nx and nt must be positive");
  if (it.pad < 2) return fail(SS_ERR_INVALID, at + "pad must be >= 2");
  if (it.n_shots < 1 || it.n_shots > SS_MAX_SHOTS) return fail(SS_ERR_INVALID, at + "n_shots must lie in 1..16");
  if (it.src_row < 0 || it.src_row >= it.nz) return fail(SS_ERR_INVALID, at + "src_row outside the model");
  for (int s = 0; s < it.n_shots; ++s)
    if (it.shot_cols[s] < 0 || it.shot_cols[s] >= it.nx) return fail(SS_ERR_INVALID, at + "shot column outside the model");
  if (it.vel_offset < 0 || it.obs_offset < 0 || it.out_offset < 0) return fail(SS_ERR_INVALID, at + "negative offset");
  return SS_OK;
}

int batch_plan(const ss_physics* phys, int mode, const ss_batch_item* items, int n_items, const int* cluster_by_class,
               int concurrent, void* plan, size_t* plan_bytes, size_t* ws_bytes) {
  if (!phys || !items || n_items < 1 || !plan_bytes || !ws_bytes) return fail(SS_ERR_INVALID, "bad arguments");
  if (mode != SS_MODE_FORWARD && mode != SS_MODE_GRADIENT && mode != SS_MODE_IMAGES)
    return fail(SS_ERR_INVALID, "mode must be forward, gradient or images");
  if (!(phys->dx > 0.0) || !(phys->dt > 0.0) || !(phys->r_coef > 0.0) || !(phys->r_coef < 1.0) ||
      !(phys->vmax_damping > 0.0) || !(phys->amp_ref > 0.0))
    return fail(SS_ERR_INVALID, "dx, dt, vmax_damping and amp_ref must be positive and 0 < r_coef < 1");
  const bool adj = mode != SS_MODE_FORWARD;
  // ---- size class of every item: its smallest fitting cluster at the
  // default tile height; the caller's table maps a size class to a cluster
  // size (bits 0-7) and a tile height (bits 8-15, 0: the default) -----------
  std::vector<int> cl(n_items), rows(n_items), min_c(n_items);
  long long n_solves = 0;
  int max_nt = 0;
  for (int i = 0; i < n_items; ++i) {
    const int rc = check_item(items[i], i);
    if (rc) return rc;
    int C = 1;
    while (C <= kMaxCluster && !item_fits(items[i], C, adj)) ++C;
    if (C > kMaxCluster) return fail(SS_ERR_UNSUPPORTED, "item " + std::to_string(i) + ": no cluster plan fits this grid");
    min_c[i] = C;
    int use = C, H = kDefaultRows;
    if (cluster_by_class && cluster_by_class[C] > 0) {
      use = std::min(kMaxCluster, std::max(C, cluster_by_class[C] & 0xff));
      const int hr = (cluster_by_class[C] >> 8) & 0xff;
      if (hr) {
        if (!batch_rows_ok(hr)) return fail(SS_ERR_INVALID, "rows per thread of a batch class must lie in 4..6");
        H = hr;
      }
    }
    while (use <= kMaxCluster && !item_fits(items[i], use, adj, H)) ++use;   // a tile height may need more CTAs
    if (use > kMaxCluster)
      return fail(SS_ERR_UNSUPPORTED, "item " + std::to_string(i) + ": no cluster plan fits at this tile height");
    cl[i] = use;
    rows[i] = H;
    n_solves += items[i].n_shots;
    max_nt = std::max(max_nt, items[i].nt);
  }
  if (n_solves > (1LL << 27) || n_items > (1 << 27)) return fail(SS_ERR_INVALID, "too many items");
  // ---- classes by cluster size; a class whose combined shared memory does
  // not fit moves its largest items one cluster size up ---------------------
  BatchPlanHeader h{};
  // members[H][C]: the items launched at cluster size C and tile height H
  std::vector<std::vector<std::vector<int>>> members(kMaxRows + 1, std::vector<std::vector<int>>(kMaxCluster + 1));
  for (int i = 0; i < n_items; ++i) members[rows[i]][cl[i]].push_back(i);
  for (int H = kMinRows; H <= kMaxRows; ++H)
    for (int C = 1; C <= kMaxCluster; ++C) {
      for (;;) {
        auto& m = members[H][C];
        if (m.empty()) break;
        int nt_max = 0, nxs = 0;
        size_t solve_part = 0;
        for (int i : m) {
          nt_max = std::max(nt_max, items[i].nt);
          nxs = std::max(nxs, (items[i].nx + 3) & ~3);
          const ItemShape s = item_shape(items[i], C, H);
          solve_part = std::max(solve_part, batch_solve_smem(s.bh, item_ncg(items[i]), adj, H));
        }
        if (batch_fixed_smem(nt_max, nxs) + solve_part <= kMaxSmem) break;
        if (C == kMaxCluster) return fail(SS_ERR_UNSUPPORTED, "no cluster plan fits the batch's shared memory");
        std::vector<int> keep;
        for (int i : m) {
          const ItemShape s = item_shape(items[i], C, H);
          if (batch_solve_smem(s.bh, item_ncg(items[i]), adj, H) == solve_part)
            members[H][C + 1].push_back(i);
          else
            keep.push_back(i);
        }
        if (keep.size() == m.size()) return fail(SS_ERR_UNSUPPORTED, "batch planner made no progress");
        m.swap(keep);
      }
    }
  // ---- launch shape, solve order and scratch of every class -------------
  struct Cls {
    int C, H;
    std::vector<int> items;
    double work;
  };
  std::vector<Cls> cls;
  for (int H = kMinRows; H <= kMaxRows; ++H)
    for (int C = 1; C <= kMaxCluster; ++C)
      if (!members[H][C].empty()) {
        double work = 0;
        for (int i : members[H][C]) work += static_cast<double>(items[i].nt) * items[i].n_shots * C;
        cls.push_back({C, H, members[H][C], work});
      }
  if (cls.size() > static_cast<size_t>(kMaxClasses)) return fail(SS_ERR_UNSUPPORTED, "more than 32 batch classes");
  // Heaviest class first: it starts on the whole GPU; lighter ones fill tails.
  std::stable_sort(cls.begin(), cls.end(), [](const Cls& a, const Cls& b) { return a.work > b.work; });
  h.magic = kPlanMagic;
  h.mode = mode;
  h.n_items = n_items;
  h.n_solves = static_cast<int32_t>(n_solves);
  h.n_classes = static_cast<int32_t>(cls.size());
  h.max_nt = max_nt;
  h.concurrent = std::min(std::max(concurrent, 0), 2);
  const double dtdx = phys->dt / phys->dx;
  h.dtdx2 = dtdx * dtdx;
  h.amp_ref = phys->amp_ref;
  h.dx = phys->dx;
  h.dt = phys->dt;
  h.items_off = static_cast<int64_t>(align_up(sizeof(BatchPlanHeader)));
  h.order_off = static_cast<int64_t>(align_up(h.items_off + sizeof(BatchItemDev) * static_cast<size_t>(n_items)));
  h.total_bytes = static_cast<int64_t>(align_up(h.order_off + sizeof(int) * static_cast<size_t>(n_solves)));

  std::vector<int> order;
  order.reserve(n_solves);
  size_t region[2] = {0, 0};
  for (size_t c = 0; c < cls.size(); ++c) {
    BatchClassHost& k = h.cls[c];
    const int C = cls[c].C, H = cls[c].H;
    const void* fn = reinterpret_cast<const void*>(batch_kernel_for(mode, H));
    k.C = C;
    k.H = H;
    k.min_C = kMaxCluster;
    k.counter = static_cast<int>(c);
    int max_nact = 0;
    size_t solve_part = 0;
    k.nt_max = 0;
    k.nxs = 0;
    k.bh_max = 0;
    k.cell_steps = 0;
    for (int i : cls[c].items) {
      const ss_batch_item& it = items[i];
      const ItemShape s = item_shape(it, C, H);
      const int ncg = item_ncg(it);
      k.min_C = std::min(k.min_C, min_c[i]);
      max_nact = std::max(max_nact, s.nact);
      solve_part = std::max(solve_part, batch_solve_smem(s.bh, ncg, adj, H));
      k.nt_max = std::max(k.nt_max, it.nt);
      k.nxs = std::max(k.nxs, (it.nx + 3) & ~3);
      k.bh_max = std::max(k.bh_max, s.bh);
      const size_t nzp = it.nz + 2 * it.pad, nxp = it.nx + 2 * it.pad;
      k.hist_slot = std::max(k.hist_slot, static_cast<size_t>(it.nt) * C * s.bh * 4 * ncg);
      k.gpad_slot = std::max(k.gpad_slot, nzp * nxp);
      k.grad_slot = std::max(k.grad_slot, static_cast<size_t>(it.nz) * it.nx);
      k.cell_steps += static_cast<double>(nzp) * nxp * it.nt * it.n_shots;
    }
    k.trace_slot = static_cast<size_t>(k.nt_max) * k.nxs;
    k.threads = ((max_nact + 31) / 32) * 32;
    k.smem = static_cast<int>(batch_fixed_smem(k.nt_max, k.nxs) + solve_part);
    // solves longest-first
    const int begin = static_cast<int>(order.size());
    for (int i : cls[c].items)
      for (int s = 0; s < items[i].n_shots; ++s) order.push_back(i << 4 | s);
    std::stable_sort(order.begin() + begin, order.end(),
                     [&](int a, int b) { return items[a >> 4].nt > items[b >> 4].nt; });
    k.order_begin = begin;
    k.n_solves = static_cast<int>(order.size()) - begin;
    // persistent clusters: as many as fit on the device at once
    int rc = ensure_batch_smem(mode, H, k.smem);
    if (rc) return rc;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(k.threads, 1, 1);
    cfg.dynamicSmemBytes = k.smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg);
    if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaOccupancyMaxActiveClusters: ") + cudaGetErrorString(e));
    if (nclusters < 1) return fail(SS_ERR_UNSUPPORTED, "no cluster of a batch class fits on the device");
    k.slots = std::max(1, std::min(nclusters, k.n_solves));
    k.max_clusters = nclusters;
    int per_sm = 1, n_sm = 0, dev = 0;
    SS_CUDA(cudaGetDevice(&dev));
    SS_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    SS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, k.threads, k.smem));
    k.idle_sms = n_sm - (nclusters * C + std::max(per_sm, 1) - 1) / std::max(per_sm, 1);
  }
  // ---- streams and launch order -------------------------------------------
  // 0: one stream, heaviest class first.  1: heaviest first, alternating
  // between two streams, so that a class's tail overlaps the next class.
  // 2: classes whose clusters leave many SMs idle (large clusters pack GPCs
  // badly) go first on stream 0, largest cluster first; the rest, on
  // stream 1, fill the SMs they leave.
  const int n_cls = static_cast<int>(cls.size());
  std::vector<BatchClassHost> sorted(h.cls, h.cls + n_cls);
  if (h.concurrent == 2) {
    int n_sm = 0, dev = 0;
    SS_CUDA(cudaGetDevice(&dev));
    SS_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
    std::vector<BatchClassHost> big, rest;
    for (const auto& k : sorted) (k.idle_sms * 10 >= n_sm ? big : rest).push_back(k);
    auto by_c = [](const BatchClassHost& a, const BatchClassHost& b) { return a.C > b.C; };
    std::stable_sort(big.begin(), big.end(), by_c);
    std::stable_sort(rest.begin(), rest.end(), by_c);
    if (big.empty() || rest.empty()) {
      h.concurrent = 1;
    } else {
      for (auto& k : big) k.stream = 0;
      for (auto& k : rest) k.stream = 1;
      sorted = big;
      sorted.insert(sorted.end(), rest.begin(), rest.end());
    }
  }
  if (h.concurrent != 2)
    for (int c = 0; c < n_cls; ++c) sorted[c].stream = h.concurrent ? (c & 1) : 0;
  for (int c = 0; c < n_cls; ++c) {
    BatchClassHost& k = sorted[c];
    k.counter = c;
    size_t bytes = 0;
    if (adj)
      bytes = align_up(k.slots * k.hist_slot * sizeof(float)) + align_up(k.slots * k.trace_slot * sizeof(float)) +
              align_up(k.slots * k.gpad_slot * sizeof(float)) + align_up(k.slots * k.grad_slot * sizeof(float));
    region[k.stream] = std::max(region[k.stream], bytes);
    h.cls[c] = k;
  }
  // workspace: status word and class counters, then one scratch region per stream
  for (int c = 0; c < n_cls; ++c) h.cls[c].ws_off = 256 + (h.cls[c].stream ? region[0] : 0);
  h.ws_bytes = static_cast<int64_t>(256 + region[0] + region[1]);
  *plan_bytes = static_cast<size_t>(h.total_bytes);
  *ws_bytes = static_cast<size_t>(h.ws_bytes);
  DeviceStreams* ds = nullptr;
  int rc = device_streams(&ds);
  if (rc) return rc;
  if (!plan) return SS_OK;
  unsigned char* out = static_cast<unsigned char*>(plan);
  std::memset(out, 0, static_cast<size_t>(h.total_bytes));
  std::memcpy(out, &h, sizeof(h));
  BatchItemDev* dv = reinterpret_cast<BatchItemDev*>(out + h.items_off);
  for (int i = 0; i < n_items; ++i) {
    const ss_batch_item& it = items[i];
    BatchItemDev d{};
    d.nz = it.nz;
    d.nx = it.nx;
    d.nt = it.nt;
    d.pad = it.pad;
    d.nzp = it.nz + 2 * it.pad;
    d.nxp = it.nx + 2 * it.pad;
    d.src_row = it.src_row;
    d.n_shots = it.n_shots;
    d.ncg = item_ncg(it);
    for (int q = 0; q < SS_MAX_SHOTS; ++q) d.shot_cols[q] = q < it.n_shots ? it.shot_cols[q] : 0;
    d.vel_off = it.vel_offset;
    d.obs_off = it.obs_offset;
    d.out_off = it.out_offset;
    d.damp_k = 3.0 * phys->vmax_damping / (2.0 * it.pad * phys->dx) * std::log(1.0 / phys->r_coef) * phys->dt / 2.0;
    d.vmute = it.v_mute;
    dv[i] = d;
  }
  for (size_t c = 0; c < cls.size(); ++c)   // band shape at the class's cluster size and tile height
    for (int i : cls[c].items) {
      const ItemShape s = item_shape(items[i], cls[c].C, cls[c].H);
      dv[i].nseg = s.nseg;
      dv[i].bh = s.bh;
      dv[i].nact = s.nact;
    }
  std::memcpy(out + h.order_off, order.data(), sizeof(int) * order.size());
  return SS_OK;
}

int batch_run(const void* plan, const void* plan_dev, const float* vel, const float* wavelet, const float* obs,
              float t_mute, float eps, int laplacian, float* gathers, float* img, float* illum, float* grad, void* ws,
              size_t ws_bytes, void* stream) {
  NvtxRange range("ss_batch_run");
  if (!plan || !plan_dev) return fail(SS_ERR_INVALID, "plan and its device copy are required");
  BatchPlanHeader h;
  std::memcpy(&h, plan, sizeof(h));
  if (h.magic != kPlanMagic) return fail(SS_ERR_INVALID, "not a batch plan");
  const int mode = h.mode;
  if (!vel || !wavelet) return fail(SS_ERR_INVALID, "vel and wavelet are required");
  if (mode == SS_MODE_FORWARD && !gathers) return fail(SS_ERR_INVALID, "gathers output is required");
  if (mode != SS_MODE_FORWARD && (!obs || !illum)) return fail(SS_ERR_INVALID, "obs and illum are required");
  if (mode == SS_MODE_GRADIENT && !grad) return fail(SS_ERR_INVALID, "grad output is required");
  if (mode == SS_MODE_IMAGES && !img) return fail(SS_ERR_INVALID, "img output is required");
  if (mode == SS_MODE_IMAGES && !(eps > 0.f)) return fail(SS_ERR_INVALID, "illumination regularization eps must be positive");
  if (!ws || ws_bytes < static_cast<size_t>(h.ws_bytes)) return fail(SS_ERR_WORKSPACE, "workspace missing or too small");
  DeviceStreams* ds = nullptr;
  int rc = device_streams(&ds);
  if (rc) return rc;
  unsigned char* w = static_cast<unsigned char*>(ws);
  const unsigned char* pd = static_cast<const unsigned char*>(plan_dev);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SS_CUDA(cudaMemsetAsync(w, 0, 256, st));
  bool two = false;
  for (int c = 0; c < h.n_classes; ++c) {
    rc = ensure_batch_smem(mode, h.cls[c].H, h.cls[c].smem);
    if (rc) return rc;
    two = two || h.cls[c].stream == 1;
  }
  if (two) {
    SS_CUDA(cudaEventRecord(ds->fork, st));
    SS_CUDA(cudaStreamWaitEvent(ds->side, ds->fork, 0));
  }
  for (int c = 0; c < h.n_classes; ++c) {
    const BatchClassHost& k = h.cls[c];
    KParams p{};
    p.C = k.C;
    p.nt = k.nt_max;
    p.nxs = k.nxs;
    p.bh = k.bh_max;
    p.n_solves = k.n_solves;
    p.items = reinterpret_cast<const BatchItemDev*>(pd + h.items_off);
    p.order = reinterpret_cast<const int*>(pd + h.order_off) + k.order_begin;
    p.counter = reinterpret_cast<int*>(w + 64) + k.counter;
    p.dtdx2 = h.dtdx2;
    p.amp_ref = h.amp_ref;
    p.dx = static_cast<float>(h.dx);
    p.dt = static_cast<float>(h.dt);
    p.vel = vel;
    p.wav = wavelet;
    p.obs = obs;
    p.t_mute = t_mute;
    p.gathers = gathers;
    p.illum = illum;
    p.img = img;
    p.eps = eps;
    p.laplacian = laplacian;
    p.err = reinterpret_cast<int*>(w);
    p.ckpt_interval = 1;
    p.hist_slot = k.hist_slot;
    p.trace_slot = k.trace_slot;
    p.gpad_slot = k.gpad_slot;
    p.grad_slot = k.grad_slot;
    if (mode != SS_MODE_FORWARD) {
      unsigned char* r = w + k.ws_off;
      p.hist = reinterpret_cast<float*>(r);
      r += align_up(k.slots * k.hist_slot * sizeof(float));
      p.trace = reinterpret_cast<float*>(r);
      r += align_up(k.slots * k.trace_slot * sizeof(float));
      p.gpad = reinterpret_cast<float*>(r);
      r += align_up(k.slots * k.gpad_slot * sizeof(float));
      p.grad_per_slot = grad == nullptr;
      p.grad = grad ? grad : reinterpret_cast<float*>(r);
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = k.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(k.C * k.slots, 1, 1);
    cfg.blockDim = dim3(k.threads, 1, 1);
    cfg.dynamicSmemBytes = k.smem;
    cfg.stream = k.stream ? ds->side : st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, batch_kernel_for(mode, k.H), p);
    if (e != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaLaunchKernelEx: ") + cudaGetErrorString(e));
  }
  if (two) {
    SS_CUDA(cudaEventRecord(ds->join, ds->side));
    SS_CUDA(cudaStreamWaitEvent(st, ds->join, 0));
  }
  return SS_OK;
}

}  // namespace

namespace ss_internal {
int fail(int code, const std::string& msg) { return ::fail(code, msg); }
void clear_error() { g_last_error.clear(); }
}  // namespace ss_internal

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* ss_version(void) { return "shotsweep-b200 0.1.0 (sm_100a)"; }

const char* ss_last_error(void) { return g_last_error.c_str(); }

size_t ss_workspace_bytes(const ss_geometry* geom, int32_t n_models, int32_t mode) {
  if (check_geometry(geom) || n_models < 1 || mode < 0 || mode > 2) return 0;
  Plan p;
  if (make_plan(geom, mode, n_models * geom->n_shots, &p)) return 0;
  return ws_layout(geom, p, mode).total;
}

int32_t ss_workspace_slots(const ss_geometry* geom, int32_t mode, size_t bytes) {
  if (check_geometry(geom) || mode < 0 || mode > 2) return 0;
  Plan p;
  if (plan_shape(geom, mode, &p)) return 0;
  return slots_for_bytes(geom, p, mode, bytes);
}

int32_t ss_set_rows_per_thread(int32_t mode, int32_t rows) {
  g_last_error.clear();
  if (mode < 0 || mode > 3) return fail(SS_ERR_INVALID, "mode must lie in 0..3");
  if (rows != 0 && !fixed_rows_ok(rows)) return fail(SS_ERR_INVALID, "rows per thread must be 4 or 5 (0: default)");
  g_rows_pref[mode].store(rows);
  return SS_OK;
}

size_t ss_workspace_bytes_slots(const ss_geometry* geom, int32_t mode, int32_t slots) {
  if (check_geometry(geom) || slots < 1 || mode < 0 || mode > 2) return 0;
  Plan p;
  if (plan_shape(geom, mode, &p)) return 0;
  p.slots = slots;
  return ws_layout(geom, p, mode).total;
}

int32_t ss_workspace_status(const void* workspace, void* stream) {
  g_last_error.clear();
  if (!workspace) return fail(SS_ERR_WORKSPACE, "workspace is NULL");
  int flag = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SS_CUDA(cudaMemcpyAsync(&flag, workspace, sizeof(int), cudaMemcpyDeviceToHost, st));
  SS_CUDA(cudaStreamSynchronize(st));
  if (flag == SS_ERR_NONFINITE) return fail(flag, "observations must be finite");
  if (flag != 0) return fail(flag, "a device-side bounded wait ran out (history copy did not complete)");
  return SS_OK;
}

int32_t ss_plan_info(const ss_geometry* geom, int32_t n_models, int32_t mode, int64_t out[8]) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (!out || n_models < 1) return fail(SS_ERR_INVALID, "bad arguments");
  Plan p;
  rc = make_plan(geom, mode, n_models * geom->n_shots, &p);
  if (rc) return rc;
  out[0] = p.C;
  out[1] = p.threads;
  out[2] = static_cast<int64_t>(p.smem);
  out[3] = p.bh;
  out[4] = p.ncg;
  out[5] = p.H;
  out[6] = p.max_clusters;
  out[7] = p.slots;
  return SS_OK;
}

static int run_forward(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                       float* gathers, float* ckpt, int32_t ckpt_interval, void* workspace, size_t workspace_bytes,
                       void* stream, long long wav_stride) {
  NvtxRange range("ss_forward");
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (n_models < 1) return fail(SS_ERR_INVALID, "n_models must be positive");
  if (!vel || !wavelet || !gathers) return fail(SS_ERR_INVALID, "vel, wavelet and gathers are required");
  if (ckpt && ckpt_interval < 1) return fail(SS_ERR_INVALID, "ckpt_interval must be positive");
  Plan p;
  rc = make_plan(geom, SS_MODE_FORWARD, n_models * geom->n_shots, &p);
  if (rc) return rc;
  const WsLayout L = ws_layout(geom, p, SS_MODE_FORWARD);
  if (!workspace || workspace_bytes < L.total) return fail(SS_ERR_WORKSPACE, "workspace missing or too small");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SS_CUDA(cudaMemsetAsync(workspace, 0, 256, st));
  KParams k = base_params(geom, p, n_models);
  k.vel = vel;
  k.wav = wavelet;
  k.wav_stride = wav_stride;
  k.gathers = gathers;
  k.ckpt = ckpt;
  k.ckpt_interval = ckpt ? ckpt_interval : 1;
  k.n_ckpt = ckpt ? (geom->nt + ckpt_interval - 1) / ckpt_interval : 0;
  k.err = static_cast<int*>(workspace);
  return launch(p, SS_MODE_FORWARD, k, st);
}

int32_t ss_forward(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet, float* gathers,
                   float* ckpt, int32_t ckpt_interval, void* workspace, size_t workspace_bytes, void* stream) {
  return run_forward(geom, n_models, vel, wavelet, gathers, ckpt, ckpt_interval, workspace, workspace_bytes, stream, 0);
}

int32_t ss_forward_wavelets(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelets,
                            float* gathers, void* workspace, size_t workspace_bytes, void* stream) {
  if (!geom) return check_geometry(geom);
  return run_forward(geom, n_models, vel, wavelets, gathers, nullptr, 1, workspace, workspace_bytes, stream, geom->nt);
}

int32_t ss_gradient(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                    const float* obs, const float* v_mute, float t_mute, float* grad, float* illum, void* workspace,
                    size_t workspace_bytes, void* stream) {
  return run_adjoint(SS_MODE_GRADIENT, geom, n_models, vel, wavelet, obs, v_mute, t_mute, 1.f, 0, nullptr, illum,
                     grad, workspace, workspace_bytes, stream);
}

int32_t ss_gradient_wavelets(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelets,
                             const float* obs, const float* v_mute, float t_mute, float* grad, float* illum,
                             void* workspace, size_t workspace_bytes, void* stream) {
  if (!geom) return check_geometry(geom);
  return run_adjoint(SS_MODE_GRADIENT, geom, n_models, vel, wavelets, obs, v_mute, t_mute, 1.f, 0, nullptr, illum,
                     grad, workspace, workspace_bytes, stream, geom->nt);
}

int32_t ss_images(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet, const float* obs,
                  const float* v_mute, float t_mute, float eps, int32_t laplacian, float* img, float* illum,
                  float* grad, void* workspace, size_t workspace_bytes, void* stream) {
  return run_adjoint(SS_MODE_IMAGES, geom, n_models, vel, wavelet, obs, v_mute, t_mute, eps, laplacian, img, illum,
                     grad, workspace, workspace_bytes, stream);
}

#define SS_ELEMENTWISE(NAME, T, KERNEL)                                                                  \
  int32_t NAME(const T* p, T* out, int64_t batch, int32_t n0, int32_t n1, void* stream) {               \
    g_last_error.clear();                                                                               \
    if (!p || !out || batch < 0 || n0 < 1 || n1 < 1) return fail(SS_ERR_INVALID, "bad arguments");      \
    const long long total = static_cast<long long>(batch) * n0 * n1;                                    \
    if (total == 0) return SS_OK;                                                                        \
    KERNEL<T><<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(p, out, batch, n0, n1);   \
    SS_CUDA(cudaGetLastError());                                                                        \
    return SS_OK;                                                                                        \
  }
SS_ELEMENTWISE(ss_lap_f32, float, lap_kernel)
SS_ELEMENTWISE(ss_lap_f64, double, lap_kernel)
SS_ELEMENTWISE(ss_lap_adjoint_f32, float, lap_adjoint_kernel)
SS_ELEMENTWISE(ss_lap_adjoint_f64, double, lap_adjoint_kernel)
#undef SS_ELEMENTWISE

#define SS_FOLD(NAME, T)                                                                                      \
  int32_t NAME(const T* g, T* out, int64_t batch, int32_t nz, int32_t nx, int32_t pad, void* stream) {       \
    g_last_error.clear();                                                                                    \
    if (!g || !out || batch < 0 || nz < 1 || nx < 1 || pad < 0) return fail(SS_ERR_INVALID, "bad arguments"); \
    const long long total = static_cast<long long>(batch) * nz * nx;                                         \
    if (total == 0) return SS_OK;                                                                             \
    fold_kernel<T><<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(g, out, batch, nz, nx, pad); \
    SS_CUDA(cudaGetLastError());                                                                             \
    return SS_OK;                                                                                             \
  }
SS_FOLD(ss_fold_edge_padding_f32, float)
SS_FOLD(ss_fold_edge_padding_f64, double)
#undef SS_FOLD

int32_t ss_mute_weights(const ss_geometry* geom, int32_t n_models, const float* v_mute, float t_mute, float* out,
                        void* stream) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (!v_mute || !out || n_models < 0) return fail(SS_ERR_INVALID, "bad arguments");
  const long long total = static_cast<long long>(n_models) * geom->n_shots * geom->nt * geom->nx;
  if (total == 0) return SS_OK;
  KParams k{};
  for (int s = 0; s < SS_MAX_SHOTS; ++s) k.shot_cols[s] = s < geom->n_shots ? geom->shot_cols[s] : 0;
  k.dx = static_cast<float>(geom->dx);
  k.dt = static_cast<float>(geom->dt);
  k.t_mute = t_mute;
  mute_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(out, v_mute, n_models, geom->n_shots,
                                                                              geom->nt, geom->nx, k);
  SS_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_images_noalloc(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                          const float* obs, const float* v_mute, float t_mute, float eps, int32_t laplacian,
                          float* img, float* illum, float* grad, void* stream) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (n_models < 1) return fail(SS_ERR_INVALID, "n_models must be positive");
  if (!vel || !wavelet || !obs || !illum || !img) return fail(SS_ERR_INVALID, "vel, wavelet, obs, img and illum are required");
  if (!(eps > 0.f)) return fail(SS_ERR_INVALID, "illumination regularization eps must be positive");
  {
    // the call ends by waiting for its own work, which a stream capture cannot record
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    SS_CUDA(cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs));
    if (cs != cudaStreamCaptureStatusNone)
      return fail(SS_ERR_UNSUPPORTED, "ss_images_noalloc waits for its work and cannot be captured into a CUDA graph");
  }
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  Plan p;
  rc = make_plan(geom, SS_MODE_IMAGES, n_models * geom->n_shots, &p);
  if (rc) return rc;
  // As many solves in flight as their scratch fits in the fixed array.
  const int fit = slots_for_bytes(geom, p, SS_MODE_IMAGES, kNoAllocScratchBytes);
  if (fit < 1) {
    p.slots = 1;
    return fail(SS_ERR_UNSUPPORTED, "one solve of this geometry needs " +
                                        std::to_string(ws_layout(geom, p, SS_MODE_IMAGES).total) +
                                        " bytes of scratch, more than the 33554432-byte allocation-free array; "
                                        "use ss_images with a workspace");
  }
  p.slots = std::min(p.slots, fit);
  const WsLayout L = ws_layout(geom, p, SS_MODE_IMAGES);
  unsigned char* w = static_cast<unsigned char*>(scratch);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The array keeps the previous call's contents; only the status word must
  // start at zero (every other scratch byte is written before it is read).
  SS_CUDA(cudaMemsetAsync(w + L.err, 0, 256, st));
  KParams k = base_params(geom, p, n_models);
  k.vel = vel;
  k.wav = wavelet;
  k.obs = obs;
  k.vmute = v_mute;
  k.t_mute = t_mute;
  k.trace = reinterpret_cast<float*>(w + L.trace);
  k.illum = illum;
  k.grad_per_slot = grad == nullptr;
  k.grad = grad ? grad : reinterpret_cast<float*>(w + L.grad);
  k.img = img;
  k.gpad = reinterpret_cast<float*>(w + L.gpad);
  k.hist = reinterpret_cast<float*>(w + L.hist);
  k.eps = eps;
  k.laplacian = laplacian;
  k.err = reinterpret_cast<int*>(w + L.err);
  k.ckpt_interval = 1;
  rc = launch(p, SS_MODE_IMAGES, k, st);
  if (rc) return rc;
  // No workspace to read a status from later: wait here and report it.
  int flag = 0;
  SS_CUDA(cudaMemcpyAsync(&flag, w + L.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SS_CUDA(cudaStreamSynchronize(st));
  if (flag == SS_ERR_NONFINITE) return fail(flag, "observations must be finite");
  if (flag != 0) return fail(flag, "a device-side bounded wait ran out (history copy did not complete)");
  return SS_OK;
}

size_t ss_segment_workspace_bytes(const ss_geometry* geom, int32_t n_models, int32_t ckpt_interval) {
  if (check_geometry(geom) || n_models < 1 || ckpt_interval < 1) return 0;
  Plan p;
  if (make_plan(geom, SS_MODE_SEGMENT, n_models * geom->n_shots, &p)) return 0;
  return ws_layout(geom, p, SS_MODE_SEGMENT, std::min(ckpt_interval, geom->nt)).total;
}

int32_t ss_adjoint_segment(const ss_geometry* geom, int32_t n_models, const float* vel, const float* wavelet,
                           const float* ckpt, int32_t ckpt_interval, int32_t seg_index, const float* res,
                           float* theta, float* gacc, float* illum_acc, float* src_acc, void* workspace,
                           size_t workspace_bytes, void* stream) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (n_models < 1 || ckpt_interval < 1) return fail(SS_ERR_INVALID, "n_models and ckpt_interval must be positive");
  const int n_ck = (geom->nt + ckpt_interval - 1) / ckpt_interval;
  if (seg_index < 0 || seg_index >= n_ck) return fail(SS_ERR_INVALID, "segment index outside the checkpoints");
  if (!vel || !wavelet || !ckpt || !res || !theta || !gacc || !illum_acc || !src_acc)
    return fail(SS_ERR_INVALID, "every array argument is required");
  Plan p;
  rc = make_plan(geom, SS_MODE_SEGMENT, n_models * geom->n_shots, &p);
  if (rc) return rc;
  const int K = std::min(ckpt_interval, geom->nt);
  const WsLayout L = ws_layout(geom, p, SS_MODE_SEGMENT, K);
  if (!workspace || workspace_bytes < L.total) return fail(SS_ERR_WORKSPACE, "workspace missing or too small");
  unsigned char* w = static_cast<unsigned char*>(workspace);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SS_CUDA(cudaMemsetAsync(w + L.err, 0, 256, st));
  KParams k = base_params(geom, p, n_models);
  k.vel = vel;
  k.wav = wavelet;
  k.trace = reinterpret_cast<float*>(w + L.trace);
  k.gpad = reinterpret_cast<float*>(w + L.gpad);
  k.grad = reinterpret_cast<float*>(w + L.grad);
  k.grad_per_slot = 1;
  k.hist = reinterpret_cast<float*>(w + L.hist);
  k.hist_steps = K;
  k.err = reinterpret_cast<int*>(w + L.err);
  k.ckpt = const_cast<float*>(ckpt);
  k.ckpt_interval = ckpt_interval;
  k.n_ckpt = n_ck;
  k.seg_index = seg_index;
  k.seg_start = seg_index * ckpt_interval;
  k.seg_steps = std::min(ckpt_interval, geom->nt - k.seg_start);
  k.theta = theta;
  k.gacc = gacc;
  k.illum_acc = illum_acc;
  k.src_acc_io = src_acc;
  k.res_in = res;
  k.eps = 1.f;
  return launch(p, SS_MODE_SEGMENT, k, st);
}

int32_t ss_gradient_finish(const ss_geometry* geom, int32_t n_models, const float* vel, const float* gacc,
                           const float* src_acc, const float* illum_acc, float* grad, float* illum, void* stream) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (n_models < 1 || !vel || !gacc || !src_acc || !illum_acc || !grad || !illum)
    return fail(SS_ERR_INVALID, "bad arguments");
  Plan p{};
  p.nzp = geom->nz + 2 * geom->pad;
  p.nxp = geom->nx + 2 * geom->pad;
  KParams k = base_params(geom, p, n_models);
  k.vel = vel;
  const long long total = static_cast<long long>(n_models) * geom->n_shots * geom->nz * geom->nx;
  finish_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(k, gacc, src_acc, illum_acc, grad,
                                                                              illum);
  SS_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_wait_probe(int32_t* status, double limit_ms, void* stream) {
  g_last_error.clear();
  if (!status || !(limit_ms > 0.0) || limit_ms > 10000.0) return fail(SS_ERR_INVALID, "bad arguments");
  wait_probe_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(
      status, static_cast<unsigned long long>(limit_ms * 1e6));
  SS_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_fp32_probe(float* out, int32_t blocks, int32_t iters, int32_t packed, double* flops, void* stream) {
  g_last_error.clear();
  if (!out || blocks < 1 || iters < 1 || !flops) return fail(SS_ERR_INVALID, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (packed)
    fp32_probe_kernel<true><<<blocks, 256, 0, st>>>(out, iters);
  else
    fp32_probe_kernel<false><<<blocks, 256, 0, st>>>(out, iters);
  SS_CUDA(cudaGetLastError());
  *flops = 2.0 * 16.0 * static_cast<double>(iters) * 256.0 * blocks;   // 16 FMAs per thread per iteration
  return SS_OK;
}

int32_t ss_c2_field(const ss_geometry* geom, int32_t n_models, const float* vel, float* out, void* stream) {
  g_last_error.clear();
  int rc = check_geometry(geom);
  if (rc) return rc;
  if (!vel || !out || n_models < 0) return fail(SS_ERR_INVALID, "bad arguments");
  const long long total = static_cast<long long>(n_models) * (geom->nz + 2 * geom->pad) * (geom->nx + 2 * geom->pad);
  if (total == 0) return SS_OK;
  const double dtdx = geom->dt / geom->dx;
  c2_kernel<<<grid_for(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(vel, out, n_models, geom->nz, geom->nx,
                                                                           geom->pad, dtdx * dtdx);
  SS_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_batch_plan(const ss_physics* phys, int32_t mode, const ss_batch_item* items, int32_t n_items,
                      const int32_t* cluster_by_class, int32_t concurrent, void* plan, size_t* plan_bytes,
                      size_t* workspace_bytes) {
  g_last_error.clear();
  return batch_plan(phys, mode, items, n_items, cluster_by_class, concurrent, plan, plan_bytes, workspace_bytes);
}

int32_t ss_batch_min_cluster(const ss_batch_item* item, int32_t mode) {
  g_last_error.clear();
  if (!item) return fail(SS_ERR_INVALID, "item is NULL");
  int rc = check_item(*item, 0);
  if (rc) return rc;
  for (int C = 1; C <= kMaxCluster; ++C)
    if (item_fits(*item, C, mode != SS_MODE_FORWARD)) return C;
  return fail(SS_ERR_UNSUPPORTED, "no cluster plan fits this grid");
}

int32_t ss_batch_min_cluster_rows(const ss_batch_item* item, int32_t mode, int32_t rows) {
  g_last_error.clear();
  if (!item) return fail(SS_ERR_INVALID, "item is NULL");
  if (!batch_rows_ok(rows)) return fail(SS_ERR_INVALID, "rows per thread of a batch class must lie in 4..6");
  int rc = check_item(*item, 0);
  if (rc) return rc;
  for (int C = 1; C <= kMaxCluster; ++C)
    if (item_fits(*item, C, mode != SS_MODE_FORWARD, rows)) return C;
  return fail(SS_ERR_UNSUPPORTED, "no cluster plan fits this grid at this tile height");
}

int32_t ss_batch_classes(const void* plan, ss_batch_class_info* out, int32_t max_classes, int32_t* n_classes) {
  g_last_error.clear();
  if (!plan || !n_classes || (max_classes > 0 && !out)) return fail(SS_ERR_INVALID, "bad arguments");
  BatchPlanHeader h;
  std::memcpy(&h, plan, sizeof(h));
  if (h.magic != kPlanMagic) return fail(SS_ERR_INVALID, "not a batch plan");
  *n_classes = h.n_classes;
  for (int c = 0; c < std::min<int>(h.n_classes, max_classes); ++c) {
    const BatchClassHost& k = h.cls[c];
    ss_batch_class_info& o = out[c];
    o.min_cluster = k.min_C;
    o.cluster = k.C;
    o.n_solves = k.n_solves;
    o.threads = k.threads;
    o.smem_bytes = k.smem;
    o.slots = k.slots;
    o.stream = k.stream;
    o.rows_per_thread = k.H;
    o.cell_steps = k.cell_steps;
  }
  return SS_OK;
}

int32_t ss_batch_run(const void* plan, const void* plan_device, const float* vel, const float* wavelet,
                     const float* obs, float t_mute, float eps, int32_t laplacian, float* gathers, float* img,
                     float* illum, float* grad, void* workspace, size_t workspace_bytes, void* stream) {
  g_last_error.clear();
  return batch_run(plan, plan_device, vel, wavelet, obs, t_mute, eps, laplacian, gathers, img, illum, grad, workspace,
                   workspace_bytes, stream);
}

}  // extern "C"
