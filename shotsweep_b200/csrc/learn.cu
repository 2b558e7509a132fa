// Tensor-core kernels of the learned velocity proposal: a BF16 x BF16 -> F32
// GEMM on the 5th-generation tensor cores (TMA tile loads with 128-byte
// swizzling into a 4-stage shared-memory ring, tcgen05.mma issued by one
// thread, the 128 x N accumulator in tensor memory, fused epilogues), and the
// convolution plumbing around it (im2col / col2im, transposes, activation
// derivatives, bias gradients, the output head, L1 loss, Adam).
//
// GEMM convention: C[M][N] = A[M][K] . B[N][K]^T, both operands K-major
// (row-major with K innermost), as every convolution here is laid out:
//   forward   Y[pixels][Cout]   = cols[pixels][K] . W[Cout][K]^T
//   backward  dW[Cout][K]       = dYt[Cout][pixels] . colsT[K][pixels]^T   (split over pixels)
//             dcols[pixels][K]  = dY[pixels][Cout] . Wt[K][Cout]^T
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/shotsweep.h"
#include "internal.h"
#include "sm100.cuh"

namespace {

using ss_internal::fail;
using bf16 = __nv_bfloat16;

constexpr int kStagesG = 4;            // shared-memory ring depth
constexpr int kBM = 128;               // rows per CTA tile (one tcgen05 M=128 MMA)
constexpr int kBK = 64;                // K per stage: 64 BF16 = one 128-byte swizzled row
constexpr int kGemmThreads = 192;      // warp 0: TMA, warp 1: TMEM + MMA, warps 2-5: epilogue

struct GemmArgs {
  int M, N, K;
  int k_tiles, k_tiles_per_split;
  void* c;
  long long ldc;
  const float* bias;
  float slope;
  int* err;
  int stages;   // ring slots in use (1..kStagesG): no more than the K steps of a CTA, so that short-K
                // GEMMs take less shared memory and several CTAs share an SM (one's epilogue overlaps
                // another's loads and MMAs)
};

template <int BN>
constexpr size_t gemm_smem_bytes(int stages = kStagesG) {
  return 1024 + static_cast<size_t>(stages) * (kBM * 128 + BN * 128) + (2 * kStagesG + 1) * 8 + 16;
}

// AMN / BMN: operand stored K-outer (A[k][m], B[k][n]) and read in place
// through MN-major descriptors, two (A) or BN/64 (B) 64 x 64 boxes per stage.
// TMAC (BF16 epilogue only): C leaves through TMA tile stores (map tc: boxes
// of 32 x 32, 64-byte swizzle) instead of per-thread stores.
template <int BN, int EPI, bool AMN, bool BMN, bool TMAC>
__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb,
                     const __grid_constant__ CUtensorMap tc, const GemmArgs g) {
  using namespace sm100;
  constexpr uint32_t A_BYTES = kBM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int ns = g.stages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + ns * STAGE);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * kStagesG + 1);
  const uint32_t sbase = smem_u32(base);
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[kStagesG + s]); };
  const uint32_t acc_bar = smem_u32(&bars[2 * kStagesG]);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  const int kt0 = blockIdx.z * g.k_tiles_per_split;
  const int nk = min(kt0 + g.k_tiles_per_split, g.k_tiles) - kt0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesG; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    mbar_init(acc_bar, 1);
    fence_mbar_init();
  }
  if (warp == 1) tmem_alloc(smem_u32(tslot), TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = *tslot;

  if (warp == 0 && lane == 0) {
    // ---- producer: A and B tiles of each K step into the ring ----------
    for (int i = 0; i < nk; ++i) {
      const int s = i % ns;
      if (i >= ns && !mbar_wait(empty(s), ((i / ns) - 1) & 1, g.err, 1)) break;
      mbar_expect_tx(full(s), STAGE);
      const int kc = (kt0 + i) * kBK;
      const uint32_t sa = sbase + s * STAGE, sb = sa + A_BYTES;
      if (AMN) {
#pragma unroll
        for (int j = 0; j < kBM / 64; ++j) tma_load_2d(sa + j * 8192, &ta, m0 + 64 * j, kc, full(s));
      } else {
        tma_load_2d(sa, &ta, kc, m0, full(s));
      }
      if (BMN) {
#pragma unroll
        for (int j = 0; j < BN / 64; ++j) tma_load_2d(sb + j * 8192, &tb, n0 + 64 * j, kc, full(s));
      } else {
        tma_load_2d(sb, &tb, kc, n0, full(s));
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: four K=16 MMAs per stage, the stage freed on completion
    constexpr uint32_t idesc = idesc_bf16_f32(kBM, BN, AMN, BMN);
    constexpr uint32_t a_step = AMN ? 2048 >> 4 : 32 >> 4, b_step = BMN ? 2048 >> 4 : 32 >> 4;   // per K=16
    for (int i = 0; i < nk; ++i) {
      const int s = i % ns;
      if (!mbar_wait(full(s), (i / ns) & 1, g.err, 2)) break;
      tc_fence_after();
      const uint32_t sa = sbase + s * STAGE, sb = sa + A_BYTES;
      const uint64_t da = AMN ? desc_sw128_mnmajor(sa, 8192) : desc_sw128_kmajor(sa);
      const uint64_t db = BMN ? desc_sw128_mnmajor(sb, 8192) : desc_sw128_kmajor(sb);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk)
        mma_bf16(taddr, da + a_step * kk, db + b_step * kk, idesc, (i > 0 || kk > 0) ? 1u : 0u);
      mma_commit(empty(s));
    }
    mma_commit(acc_bar);
  } else if (warp >= 2) {
    // ---- epilogue: warp w owns TMEM lanes 32*(w%4) .. +31 (rows of the tile).
    // Each 32-column slab goes TMEM -> registers (one row per thread) -> a
    // padded 32 x 33 shared slab -> registers (8 threads per row, 4 columns
    // each), so every store instruction covers 4 whole rows of 32 columns.
    // The ring is free once the accumulator barrier completes (every load was
    // consumed by an MMA that has finished), so the slabs live in stage 0.
    mbar_wait(acc_bar, 0, g.err, 3);
    tc_fence_after();
    const int q = warp & 3;
    if constexpr (TMAC) {
      // Two 2 KB BF16 slabs per warp in stage 0 (1024-byte aligned), alternated
      // so that a slab's previous store has read it before it is rewritten.
      // Row r (this lane) holds 32 columns = four 16-byte chunks; chunk j sits
      // at chunk j ^ ((r >> 1) & 3) of the row, the 64-byte swizzle the map
      // uses, which also spreads the warp's writes over all banks.
      const uint32_t slab0 = sbase + static_cast<uint32_t>(q) * 4096u;
      int k = 0;
#pragma unroll 1
      for (int c = 0; c < BN && n0 + c < g.N; c += 32, ++k) {
        float v[32];
        tmem_ld32(taddr + (static_cast<uint32_t>(q * 32) << 16) + c, v);
        uint32_t pk[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          float x0 = v[2 * j], x1 = v[2 * j + 1];
          if (g.bias) {
            const int col = n0 + c + 2 * j;
            x0 += col < g.N ? g.bias[col] : 0.f;
            x1 += col + 1 < g.N ? g.bias[col + 1] : 0.f;
          }
          x0 = x0 > 0.f ? x0 : g.slope * x0;
          x1 = x1 > 0.f ? x1 : g.slope * x1;
          const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
          pk[j] = *reinterpret_cast<const uint32_t*>(&h);
        }
        const uint32_t slab = slab0 + static_cast<uint32_t>(k & 1) * 2048u;
        if (lane == 0) bulk_wait_read<1>();   // the store issued from this slab two slabs ago has read it
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint32_t a =
              slab + static_cast<uint32_t>(lane) * 64u + static_cast<uint32_t>((j ^ ((lane >> 1) & 3)) * 16);
          asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(a), "r"(pk[4 * j]), "r"(pk[4 * j + 1]),
                       "r"(pk[4 * j + 2]), "r"(pk[4 * j + 3])
                       : "memory");
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          tma_store_2d(&tc, slab, n0 + c, m0 + q * 32);
          bulk_commit();
        }
      }
      if (lane == 0) bulk_wait_all();
      __syncwarp();
    } else {
    float* slab = reinterpret_cast<float*>(base) + q * (32 * 33);
    const int rsub = lane >> 3, c4 = (lane & 7) * 4;
    const bool vec = g.ldc % 4 == 0;
#pragma unroll 1
    for (int c = 0; c < BN && n0 + c < g.N; c += 32) {
      float v[32];
      tmem_ld32(taddr + (static_cast<uint32_t>(q * 32) << 16) + c, v);
#pragma unroll
      for (int j = 0; j < 32; ++j) slab[lane * 33 + j] = v[j];
      __syncwarp();
      const int col = n0 + c + c4;
      float bj[4] = {0.f, 0.f, 0.f, 0.f};
      if ((EPI == SS_EPI_BIAS_LRELU_BF16 || EPI == SS_EPI_BIAS_F32) && g.bias) {
#pragma unroll
        for (int j = 0; j < 4; ++j) bj[j] = col + j < g.N ? g.bias[col + j] : 0.f;
      }
#pragma unroll
      for (int pass = 0; pass < 8; ++pass) {
        const int r = pass * 4 + rsub;
        const int row = m0 + q * 32 + r;
        float x[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          x[j] = slab[r * 33 + c4 + j] + bj[j];
          if (EPI == SS_EPI_BIAS_LRELU_BF16) x[j] = x[j] > 0.f ? x[j] : g.slope * x[j];
        }
        if (row >= g.M) continue;
        const long long off = static_cast<long long>(row) * g.ldc + col;
        if (vec && col + 4 <= g.N) {
          if (EPI == SS_EPI_BIAS_LRELU_BF16) {
            __align__(8) bf16 o[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) o[j] = __float2bfloat16_rn(x[j]);
            *reinterpret_cast<uint2*>(static_cast<bf16*>(g.c) + off) = *reinterpret_cast<const uint2*>(o);
          } else {
            float4* dst = reinterpret_cast<float4*>(static_cast<float*>(g.c) + off);
            const float4 q4 = make_float4(x[0], x[1], x[2], x[3]);
            if (EPI == SS_EPI_F32_ADD)
              atomicAdd(dst, q4);
            else
              *dst = q4;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (col + j >= g.N) break;
            if (EPI == SS_EPI_BIAS_LRELU_BF16)
              static_cast<bf16*>(g.c)[off + j] = __float2bfloat16_rn(x[j]);
            else if (EPI == SS_EPI_F32_ADD)
              atomicAdd(static_cast<float*>(g.c) + off + j, x[j]);
            else
              static_cast<float*>(g.c)[off + j] = x[j];
          }
        }
      }
      __syncwarp();
    }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    tmem_dealloc(taddr, TMEM_COLS);
  }
}

// ---- host: tensor maps ------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// BF16 output matrix [rows][ld] (first `cols` columns) as TMA store tiles of
// 32 x 32 with the 64-byte swizzle (the epilogue's slab layout).
int make_tmap_store(CUtensorMap* map, void* ptr, long long cols, long long rows, long long ld) {
  auto fn = encode_fn();
  if (!fn) return fail(SS_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * 2)};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")");
  return SS_OK;
}

// K-major BF16 matrix [rows][ld] (K = first `k` columns) as TMA tiles of 64 x box_rows.
int make_tmap(CUtensorMap* map, const void* ptr, long long k, long long rows, long long ld, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return fail(SS_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) != 0) return fail(SS_ERR_INVALID, "GEMM operands must be 16-byte aligned");
  if ((ld * 2) % 16 != 0) return fail(SS_ERR_INVALID, "GEMM operand row strides must be multiples of 8 elements");
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * 2)};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SS_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(r) + ")");
  return SS_OK;
}

template <int BN, int EPI, bool AMN, bool BMN, bool TMAC = false>
int launch_gemm_t(const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc, const GemmArgs& g, int splits,
                  cudaStream_t st) {
  auto kern = gemm_bf16_kernel<BN, EPI, AMN, BMN, TMAC>;
  constexpr size_t smem = gemm_smem_bytes<BN>();   // the attribute allows the full ring
  const size_t smem_run = gemm_smem_bytes<BN>(g.stages);
  // the attribute is per device: set once on each device that launches this instantiation
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  SS_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS_ERR_UNSUPPORTED, "device index beyond 63");
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!done[dev]) {
      SS_TRY_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
      done[dev] = true;
    }
  }
  dim3 grid((g.N + BN - 1) / BN, (g.M + kBM - 1) / kBM, splits);
  kern<<<grid, kGemmThreads, smem_run, st>>>(ta, tb, tc, g);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

// tc: the output's store map when `tmac` (BF16 epilogue with a stride TMA can describe), else unused.
template <int BN, bool AMN, bool BMN>
int launch_gemm_epi(int epi, bool tmac, const CUtensorMap& ta, const CUtensorMap& tb, const CUtensorMap& tc,
                    const GemmArgs& g, int splits, cudaStream_t st) {
  switch (epi) {
    case SS_EPI_F32: return launch_gemm_t<BN, SS_EPI_F32, AMN, BMN>(ta, tb, tc, g, splits, st);
    case SS_EPI_F32_ADD: return launch_gemm_t<BN, SS_EPI_F32_ADD, AMN, BMN>(ta, tb, tc, g, splits, st);
    case SS_EPI_BIAS_LRELU_BF16:
      if (tmac) return launch_gemm_t<BN, SS_EPI_BIAS_LRELU_BF16, AMN, BMN, true>(ta, tb, tc, g, splits, st);
      return launch_gemm_t<BN, SS_EPI_BIAS_LRELU_BF16, AMN, BMN>(ta, tb, tc, g, splits, st);
    default: return launch_gemm_t<BN, SS_EPI_BIAS_F32, AMN, BMN>(ta, tb, tc, g, splits, st);
  }
}

// layout bit 0: A stored K-outer; bit 1: B stored K-outer (layouts 0, 2 and 3).
// An MN-major B needs whole 64-column boxes, so its tiles are at least 64 wide.
template <int BN>
int launch_gemm_bn(int layout, int epi, bool tmac, const CUtensorMap& ta, const CUtensorMap& tb,
                   const CUtensorMap& tc, const GemmArgs& g, int splits, cudaStream_t st) {
  if constexpr (BN >= 64) {
    if (layout == 3) return launch_gemm_epi<BN, true, true>(epi, tmac, ta, tb, tc, g, splits, st);
    if (layout == 2) return launch_gemm_epi<BN, false, true>(epi, tmac, ta, tb, tc, g, splits, st);
  }
  return launch_gemm_epi<BN, false, false>(epi, tmac, ta, tb, tc, g, splits, st);
}


// ---- convolution plumbing ----------------------------------------------------
// Activations are NHWC BF16.  A convolution layer reads its input through an
// optional nearest-neighbour upsampling by `up` (the decoder's x2 steps) and
// has im2col column index k = (kh * KW + kw) * Cin + c.
struct ConvGeom {
  int B, Hin, Win, Cin, KH, KW, sh, sw, ph, pw, up, Hout, Wout;
};

__device__ __forceinline__ int64_t conv_src(const ConvGeom& g, int64_t m, int k) {
  const int c = k % g.Cin, kk = k / g.Cin, kw = kk % g.KW, kh = kk / g.KW;
  const int ox = static_cast<int>(m % g.Wout);
  const int64_t t = m / g.Wout;
  const int oy = static_cast<int>(t % g.Hout);
  const int b = static_cast<int>(t / g.Hout);
  const int uy = oy * g.sh - g.ph + kh, ux = ox * g.sw - g.pw + kw;
  if (uy < 0 || ux < 0 || uy >= g.Hin * g.up || ux >= g.Win * g.up) return -1;
  return ((static_cast<int64_t>(b) * g.Hin + uy / g.up) * g.Win + ux / g.up) * g.Cin + c;
}

__global__ void im2col_kernel(const bf16* __restrict__ x, ConvGeom g, int K, int Kc, bf16* __restrict__ cols) {
  const int64_t M = static_cast<int64_t>(g.B) * g.Hout * g.Wout;
  const int64_t total = M * Kc;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int k = static_cast<int>(i % Kc);
    const int64_t m = i / Kc;
    const int64_t src = k < K ? conv_src(g, m, k) : -1;
    cols[i] = src >= 0 ? x[src] : __float2bfloat16_rn(0.f);
  }
}

// 8 channels (16 bytes) per thread where Cin % 8 == 0 (then K == Kc).
__global__ void im2col_vec8_kernel(const bf16* __restrict__ x, ConvGeom g, bf16* __restrict__ cols) {
  const int chunks = g.Cin / 8, taps = g.KH * g.KW;
  const int64_t M = static_cast<int64_t>(g.B) * g.Hout * g.Wout;
  const int64_t total = M * taps * chunks;
  const int64_t K = static_cast<int64_t>(taps) * g.Cin;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int ch = static_cast<int>(i % chunks);
    const int64_t mt = i / chunks;
    const int tap = static_cast<int>(mt % taps);
    const int64_t m = mt / taps;
    const int64_t src = conv_src(g, m, tap * g.Cin + ch * 8);
    uint4 v = make_uint4(0, 0, 0, 0);
    if (src >= 0) v = *reinterpret_cast<const uint4*>(x + src);
    *reinterpret_cast<uint4*>(cols + m * K + tap * g.Cin + ch * 8) = v;
  }
}

// Columns of small-K layers (K <= 64, Kc % 8 == 0; the first encoder layer,
// whose 5 input channels rule out 16-byte gathers): each thread gathers one
// pixel's row, tap by tap (runs of Cin contiguous inputs), into shared memory;
// the CTA then writes its 256 consecutive rows with coalesced 16-byte stores.
constexpr int kRowThreads = 256;
__global__ void __launch_bounds__(kRowThreads) im2col_rows_kernel(const bf16* __restrict__ x, ConvGeom g, int K, int Kc,
                                                                  bf16* __restrict__ cols) {
  extern __shared__ __align__(16) unsigned char rows_raw[];
  bf16* rows = reinterpret_cast<bf16*>(rows_raw);   // [kRowThreads][Kc]
  const int64_t M = static_cast<int64_t>(g.B) * g.Hout * g.Wout;
  for (int64_t m0 = static_cast<int64_t>(blockIdx.x) * kRowThreads; m0 < M;
       m0 += static_cast<int64_t>(gridDim.x) * kRowThreads) {
    const int64_t m = m0 + threadIdx.x;
    bf16* row = rows + threadIdx.x * Kc;
    if (m < M) {
      const int ox = static_cast<int>(m % g.Wout);
      const int64_t t = m / g.Wout;
      const int oy = static_cast<int>(t % g.Hout);
      const int b = static_cast<int>(t / g.Hout);
      for (int kh = 0; kh < g.KH; ++kh)
        for (int kw = 0; kw < g.KW; ++kw) {
          const int uy = oy * g.sh - g.ph + kh, ux = ox * g.sw - g.pw + kw;
          const bool in = uy >= 0 && ux >= 0 && uy < g.Hin * g.up && ux < g.Win * g.up;
          const bf16* src = in ? x + ((static_cast<int64_t>(b) * g.Hin + uy / g.up) * g.Win + ux / g.up) * g.Cin : x;
          bf16* dst = row + (kh * g.KW + kw) * g.Cin;
          for (int c = 0; c < g.Cin; ++c) dst[c] = in ? src[c] : __float2bfloat16_rn(0.f);
        }
      for (int k = K; k < Kc; ++k) row[k] = __float2bfloat16_rn(0.f);
    }
    __syncthreads();
    const int64_t n_rows = M - m0 < kRowThreads ? M - m0 : static_cast<int64_t>(kRowThreads);
    const int64_t n16 = n_rows * Kc / 8;   // 16-byte words of this CTA's rows
    uint4* out = reinterpret_cast<uint4*>(cols + m0 * Kc);
    const uint4* in16 = reinterpret_cast<const uint4*>(rows);
    for (int64_t i = threadIdx.x; i < n16; i += kRowThreads) out[i] = in16[i];
    __syncthreads();
  }
}


// BF16 column gradients back onto the input, 8 channels per thread (16-byte
// loads and stores), times the leaky-ReLU derivative of the layer below.
// The tap geometry (KH, KW, strides, upsampling) is a template parameter for
// the network's layer families (0: read at run time), so the stride tests and
// divisions of the tap loops fold to constants; the per-thread index work
// otherwise bounds a gather this short.  Indices are 32-bit (the host checks
// the element count); Cin / 8 is a power of two (c8_shift).
template <int KH_, int KW_, int SH_, int SW_, int UP_>
__global__ void __launch_bounds__(256) col2im16_lrelu_kernel(const bf16* __restrict__ dcols, ConvGeom g, int Kc,
                                                             const bf16* __restrict__ y, float slope,
                                                             bf16* __restrict__ dpre, int64_t ldp, int total,
                                                             int c8_shift) {
  const int KH = KH_ ? KH_ : g.KH, KW = KW_ ? KW_ : g.KW, SH = SH_ ? SH_ : g.sh, SW = SW_ ? SW_ : g.sw;
  const int UP = UP_ ? UP_ : g.up;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int pix = i >> c8_shift;
    const int c = (i - (pix << c8_shift)) * 8;
    const int ix = pix % g.Win, t = pix / g.Win;
    const int iy = t % g.Hin, b = t / g.Hin;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int dy = 0; dy < UP; ++dy)
#pragma unroll
      for (int kh = 0; kh < KH; ++kh) {
        const int ty = iy * UP + dy + g.ph - kh;
        if (ty < 0 || ty % SH) continue;
        const int oy = ty / SH;
        if (oy >= g.Hout) continue;
        const bf16* rowp = dcols + (static_cast<int64_t>(b) * g.Hout + oy) * g.Wout * Kc + kh * KW * g.Cin + c;
#pragma unroll
        for (int dx = 0; dx < UP; ++dx)
#pragma unroll
          for (int kw = 0; kw < KW; ++kw) {
            const int tx = ix * UP + dx + g.pw - kw;
            if (tx < 0 || tx % SW) continue;
            const int ox = tx / SW;
            if (ox >= g.Wout) continue;
            const uint4 d = *reinterpret_cast<const uint4*>(rowp + static_cast<int64_t>(ox) * Kc + kw * g.Cin);
            const uint32_t w[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              acc[2 * j] += __uint_as_float(w[j] << 16);
              acc[2 * j + 1] += __uint_as_float(w[j] & 0xffff0000u);
            }
          }
      }
    const uint4 yv = *reinterpret_cast<const uint4*>(y + static_cast<int64_t>(pix) * g.Cin + c);
    const uint32_t yw[4] = {yv.x, yv.y, yv.z, yv.w};
    __align__(16) bf16 o[8];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float y0 = __uint_as_float(yw[j] << 16), y1 = __uint_as_float(yw[j] & 0xffff0000u);
      o[2 * j] = __float2bfloat16_rn(y0 > 0.f ? acc[2 * j] : slope * acc[2 * j]);
      o[2 * j + 1] = __float2bfloat16_rn(y1 > 0.f ? acc[2 * j + 1] : slope * acc[2 * j + 1]);
    }
    bf16* dst = dpre + static_cast<int64_t>(pix) * ldp + c;
    if ((ldp & 7) == 0 && (reinterpret_cast<uintptr_t>(dpre) & 15) == 0) {
      *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(o);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) dst[j] = o[j];
    }
  }
}

// im2col in 16-byte chunks (Cin % 8 == 0, Kc == K, Cin / 8 a power of two):
// 2^lanes_shift consecutive threads share one output pixel, whose coordinates
// they work out once, and write its column row chunk by chunk (a warp's
// stores cover whole rows); a chunk costs a shift, the tap split (a constant
// KW) and one 16-byte load and store.  32-bit indices (checked on the host).
template <int KW_, int UP_>
__global__ void __launch_bounds__(256) im2col_px_kernel(const bf16* __restrict__ x, ConvGeom g, int M, int chunks,
                                                        int c8_shift, int lanes_shift, bf16* __restrict__ cols) {
  const int KW = KW_ ? KW_ : g.KW, UP = UP_ ? UP_ : g.up;
  const int lanes = 1 << lanes_shift;
  const int sub = threadIdx.x & (lanes - 1);
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) >> lanes_shift;
  const int ngroups = (gridDim.x * blockDim.x) >> lanes_shift;
  const int Hup = g.Hin * UP, Wup = g.Win * UP;
  for (int m = group; m < M; m += ngroups) {
    const int ox = m % g.Wout, t = m / g.Wout;
    const int oy = t % g.Hout, b = t / g.Hout;
    const int uy0 = oy * g.sh - g.ph, ux0 = ox * g.sw - g.pw;
    const bf16* xb = x + static_cast<int64_t>(b) * g.Hin * g.Win * g.Cin;
    bf16* dst = cols + static_cast<int64_t>(m) * (chunks * 8);
    for (int j = sub; j < chunks; j += lanes) {
      const int tap = j >> c8_shift, c8 = j - (tap << c8_shift);
      const int kh = tap / KW, kw = tap - kh * KW;
      const int uy = uy0 + kh, ux = ux0 + kw;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (uy >= 0 && ux >= 0 && uy < Hup && ux < Wup)
        v = *reinterpret_cast<const uint4*>(xb + (static_cast<int64_t>(uy / UP) * g.Win + ux / UP) * g.Cin + c8 * 8);
      *reinterpret_cast<uint4*>(dst + j * 8) = v;
    }
  }
}

// db[c] += sum over rows of dpre[row][c]
__global__ void bias_grad_kernel(const bf16* __restrict__ dpre, int64_t ld, int64_t M, int C, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float acc = 0.f;
  for (int64_t m = blockIdx.y; m < M; m += gridDim.y) acc += __bfloat162float(dpre[m * ld + c]);
  atomicAdd(db + c, acc);
}

// Column sums with 16-byte loads (C % 8 == 0, ld % 8 == 0, aligned base): a
// CTA sums a slab of rows; L threads span a row's column groups of 8, R = 256
// / L rows are read at once (four loads in flight per thread), and the R
// partial sums of each column meet in shared memory, summed by 256 threads in
// parallel, before one atomic per column and CTA.
__global__ void __launch_bounds__(256) bias_grad_v8_kernel(const bf16* __restrict__ dpre, int64_t ld, int64_t M,
                                                           int C, int64_t rows_per_cta, float* __restrict__ db) {
  __shared__ float red[256 * 8];
  const int G = C >> 3, L = G < 256 ? G : 256, R = 256 / L;
  const int t = threadIdx.x, cgi = t % L, rr = t / L;
  const int64_t r0 = blockIdx.x * rows_per_cta;
  const int64_t r1 = r0 + rows_per_cta < M ? r0 + rows_per_cta : M;
  for (int cg0 = blockIdx.y * L; cg0 < G; cg0 += gridDim.y * L) {
    const int cg = cg0 + cgi;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (rr < R && cg < G) {
#pragma unroll 4
      for (int64_t r = r0 + rr; r < r1; r += R) {
        const uint4 v = *reinterpret_cast<const uint4*>(dpre + r * ld + cg * 8);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[2 * j] += __uint_as_float(w[j] << 16);
          acc[2 * j + 1] += __uint_as_float(w[j] & 0xffff0000u);
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) red[t * 8 + j] = acc[j];
    __syncthreads();
    for (int q = t; q < L * 8; q += 256) {   // q = column group within the pass x 8 + column
      const int qc = q >> 3, j = q & 7;
      if (cg0 + qc >= G) continue;
      float sum = 0.f;
      for (int p = 0; p < R; ++p) sum += red[(p * L + qc) * 8 + j];
      atomicAdd(db + (cg0 + qc) * 8 + j, sum);
    }
    __syncthreads();
  }
}

// Output head: crop rows/cols [off, off+n) of x [B][H][W][C], 3x3 convolution
// with zero padding, bias, tanh (the reference decoder's head on the cropped map).
struct HeadGeom {
  int B, H, W, C, off, n;
};

__global__ void head_forward_kernel(const bf16* __restrict__ x, HeadGeom g, const float* __restrict__ w,
                                    const float* __restrict__ bias_dev, float* __restrict__ out) {
  const float bias = *bias_dev;
  const int64_t total = static_cast<int64_t>(g.B) * g.n * g.n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int xo = static_cast<int>(i % g.n), yo = static_cast<int>((i / g.n) % g.n);
    const int b = static_cast<int>(i / (static_cast<int64_t>(g.n) * g.n));
    float acc = bias;
    for (int kh = 0; kh < 3; ++kh) {
      const int yy = yo + kh - 1;
      if (yy < 0 || yy >= g.n) continue;
      for (int kw = 0; kw < 3; ++kw) {
        const int xx = xo + kw - 1;
        if (xx < 0 || xx >= g.n) continue;
        const bf16* px = x + ((static_cast<int64_t>(b) * g.H + yy + g.off) * g.W + xx + g.off) * g.C;
        const float* wk = w + (kh * 3 + kw) * g.C;
        for (int c = 0; c < g.C; ++c) acc = fmaf(__bfloat162float(px[c]), wk[c], acc);
      }
    }
    out[i] = tanhf(acc);
  }
}

// L1 loss of tanh outputs: loss_sum += sum |p - t|; dpre = sign(p - t) / n * (1 - p^2).
__global__ void l1_tanh_kernel(const float* __restrict__ p, const float* __restrict__ t, int64_t n, float inv_n,
                               float* __restrict__ loss_sum, float* __restrict__ dpre) {
  float acc = 0.f;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float d = p[i] - t[i];
    acc += fabsf(d);
    const float sg = d > 0.f ? 1.f : (d < 0.f ? -1.f : 0.f);
    dpre[i] = sg * inv_n * (1.f - p[i] * p[i]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, acc);
}

// Head backward: weight / bias gradients (dw [9][C] += ..., db += ...) and the
// input gradient on the uncropped map times the leaky-ReLU derivative of x.
__global__ void head_wgrad_kernel(const bf16* __restrict__ x, HeadGeom g, const float* __restrict__ dpre,
                                  float* __restrict__ dw, float* __restrict__ db) {
  // one thread per (tap, channel); blocks split the pixels
  const int j = threadIdx.x;               // tap * C + c, blockDim.x = 9 * C
  const int tap = j / g.C, c = j % g.C, kh = tap / 3, kw = tap % 3;
  const int total = g.B * g.n * g.n;       // checked < 2^31 on the host
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(i0 + per, total);
  float acc = 0.f, accb = 0.f;
  int xo = i0 % g.n, yo = (i0 / g.n) % g.n, b = i0 / (g.n * g.n);
  for (int i = i0; i < i1; ++i) {
    const float d = dpre[i];
    if (j == 0) accb += d;
    const int yy = yo + kh - 1, xx = xo + kw - 1;
    if (yy >= 0 && yy < g.n && xx >= 0 && xx < g.n)
      acc = fmaf(d, __bfloat162float(x[((static_cast<int64_t>(b) * g.H + yy + g.off) * g.W + xx + g.off) * g.C + c]),
                 acc);
    if (++xo == g.n) {   // next position (x fastest, then y, then the model)
      xo = 0;
      if (++yo == g.n) {
        yo = 0;
        ++b;
      }
    }
  }
  atomicAdd(dw + j, acc);
  if (j == 0) atomicAdd(db, accb);
}

__global__ void head_dgrad_kernel(const bf16* __restrict__ x, HeadGeom g, const float* __restrict__ dpre,
                                  const float* __restrict__ w, float slope, bf16* __restrict__ dpre_x) {
  const int64_t total = static_cast<int64_t>(g.B) * g.H * g.W * g.C;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i % g.C);
    const int64_t pix = i / g.C;
    const int X = static_cast<int>(pix % g.W), Y = static_cast<int>((pix / g.W) % g.H);
    const int b = static_cast<int>(pix / (static_cast<int64_t>(g.W) * g.H));
    const int yy = Y - g.off, xx = X - g.off;
    float acc = 0.f;
    if (yy >= 0 && yy < g.n && xx >= 0 && xx < g.n)
      for (int kh = 0; kh < 3; ++kh) {
        const int yo = yy - kh + 1;
        if (yo < 0 || yo >= g.n) continue;
        for (int kw = 0; kw < 3; ++kw) {
          const int xo = xx - kw + 1;
          if (xo < 0 || xo >= g.n) continue;
          acc = fmaf(dpre[(static_cast<int64_t>(b) * g.n + yo) * g.n + xo], w[(kh * 3 + kw) * g.C + c], acc);
        }
      }
    const float yv = __bfloat162float(x[i]);
    dpre_x[i] = __float2bfloat16_rn(yv > 0.f ? acc : slope * acc);
  }
}

// Output head with 8-channel (16-byte) input loads and the 3 x 3 x C weights
// in shared memory; one thread per output pixel (C % 8 == 0, C <= 64).
__global__ void __launch_bounds__(256) head_forward_v8_kernel(const bf16* __restrict__ x, HeadGeom g,
                                                              const float* __restrict__ w,
                                                              const float* __restrict__ bias_dev,
                                                              float* __restrict__ out) {
  __shared__ float ws[9 * 64];
  for (int i = threadIdx.x; i < 9 * g.C; i += blockDim.x) ws[i] = w[i];
  __syncthreads();
  const float bias = *bias_dev;
  const int64_t total = static_cast<int64_t>(g.B) * g.n * g.n;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int xo = static_cast<int>(i % g.n), yo = static_cast<int>((i / g.n) % g.n);
    const int b = static_cast<int>(i / (static_cast<int64_t>(g.n) * g.n));
    float acc = bias;
    for (int kh = 0; kh < 3; ++kh) {
      const int yy = yo + kh - 1;
      if (yy < 0 || yy >= g.n) continue;
      for (int kw = 0; kw < 3; ++kw) {
        const int xx = xo + kw - 1;
        if (xx < 0 || xx >= g.n) continue;
        const uint4* px =
            reinterpret_cast<const uint4*>(x + ((static_cast<int64_t>(b) * g.H + yy + g.off) * g.W + xx + g.off) * g.C);
        const float* wk = ws + (kh * 3 + kw) * g.C;
        for (int q = 0; q < g.C / 8; ++q) {
          const uint4 v = px[q];
          const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float2 f = __bfloat1622float2(h[j]);
            acc = fmaf(f.x, wk[8 * q + 2 * j], acc);
            acc = fmaf(f.y, wk[8 * q + 2 * j + 1], acc);
          }
        }
      }
    }
    out[i] = tanhf(acc);
  }
}

// Head weight and bias gradients: dw[tap][c] = sum_p dpre[p] x[p + tap][c],
// db = sum_p dpre[p].  Thread (pixel lane, 8-channel group) accumulates the
// 9 x 8 products of its pixels in registers; lanes reduce with shuffles, warps
// through shared memory, and each CTA adds its 9 x C sums with one atomic each.
template <int CG>   // channel groups of 8: C = 8 * CG
__global__ void __launch_bounds__(256) head_wgrad_v8_kernel(const bf16* __restrict__ x, HeadGeom g,
                                                            const float* __restrict__ dpre, float* __restrict__ dw,
                                                            float* __restrict__ db) {
  constexpr int kLanes = 256 / CG;   // pixel lanes per CTA
  __shared__ float red[8][CG][72];
  __shared__ float redb[8];
  const int cg = threadIdx.x % CG, pl = threadIdx.x / CG;
  const int total = g.B * g.n * g.n;   // checked < 2^31 on the host
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int p0 = blockIdx.x * per, p1 = min(p0 + per, total);
  float acc[72];
#pragma unroll
  for (int j = 0; j < 72; ++j) acc[j] = 0.f;
  float accb = 0.f;
  for (int p = p0 + pl; p < p1; p += kLanes) {
    const float d = dpre[p];
    accb += d;
    const int xo = p % g.n, yo = (p / g.n) % g.n, b = p / (g.n * g.n);
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int yy = yo + tap / 3 - 1, xx = xo + tap % 3 - 1;
      if (yy < 0 || yy >= g.n || xx < 0 || xx >= g.n) continue;
      const uint4 v = *reinterpret_cast<const uint4*>(
          x + ((static_cast<int64_t>(b) * g.H + yy + g.off) * g.W + xx + g.off) * g.C + 8 * cg);
      const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 f = __bfloat1622float2(h[j]);
        acc[tap * 8 + 2 * j] = fmaf(d, f.x, acc[tap * 8 + 2 * j]);
        acc[tap * 8 + 2 * j + 1] = fmaf(d, f.y, acc[tap * 8 + 2 * j + 1]);
      }
    }
  }
  // lanes of one channel group within a warp: reduce over pixel lanes
#pragma unroll
  for (int j = 0; j < 72; ++j)
    for (int o = CG; o < 32; o <<= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  for (int o = 1; o < 32; o <<= 1) accb += __shfl_xor_sync(0xffffffffu, accb, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane < CG)
#pragma unroll
    for (int j = 0; j < 72; ++j) red[warp][lane][j] = acc[j];
  if (lane == 0) redb[warp] = accb / CG;   // every channel group added the same dpre values
  __syncthreads();
  for (int o = threadIdx.x; o < 9 * 8 * CG; o += blockDim.x) {
    const int tap = o / (8 * CG), c = o % (8 * CG);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += red[k][c / 8][tap * 8 + c % 8];
    atomicAdd(dw + o, s);
  }
  if (threadIdx.x == 0) {
    float s = 0.f;
    for (int k = 0; k < 8; ++k) s += redb[k];
    atomicAdd(db, s);
  }
}

// Head input gradient times the leaky-ReLU derivative of x, 8 channels per
// thread (16-byte loads and stores), weights in shared memory.
__global__ void __launch_bounds__(256) head_dgrad_v8_kernel(const bf16* __restrict__ x, HeadGeom g,
                                                            const float* __restrict__ dpre,
                                                            const float* __restrict__ w, float slope,
                                                            bf16* __restrict__ dpre_x) {
  __shared__ float ws[9 * 64];
  for (int i = threadIdx.x; i < 9 * g.C; i += blockDim.x) ws[i] = w[i];
  __syncthreads();
  const int cgs = g.C / 8;
  const int64_t total = static_cast<int64_t>(g.B) * g.H * g.W * cgs;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int c0 = static_cast<int>(i % cgs) * 8;
    const int64_t pix = i / cgs;
    const int X = static_cast<int>(pix % g.W), Y = static_cast<int>((pix / g.W) % g.H);
    const int b = static_cast<int>(pix / (static_cast<int64_t>(g.W) * g.H));
    const int yy = Y - g.off, xx = X - g.off;
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (yy >= 0 && yy < g.n && xx >= 0 && xx < g.n)
      for (int kh = 0; kh < 3; ++kh) {
        const int yo = yy - kh + 1;
        if (yo < 0 || yo >= g.n) continue;
        for (int kw = 0; kw < 3; ++kw) {
          const int xo = xx - kw + 1;
          if (xo < 0 || xo >= g.n) continue;
          const float d = dpre[(static_cast<int64_t>(b) * g.n + yo) * g.n + xo];
          const float* wk = ws + (kh * 3 + kw) * g.C + c0;
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[j] = fmaf(d, wk[j], acc[j]);
        }
      }
    const uint4 yv = *reinterpret_cast<const uint4*>(x + pix * g.C + c0);
    const __nv_bfloat162* yh = reinterpret_cast<const __nv_bfloat162*>(&yv);
    uint4 o;
    __nv_bfloat162* oh = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float2 f = __bfloat1622float2(yh[j]);
      const float a0 = f.x > 0.f ? acc[2 * j] : slope * acc[2 * j];
      const float a1 = f.y > 0.f ? acc[2 * j + 1] : slope * acc[2 * j + 1];
      oh[j] = __floats2bfloat162_rn(a0, a1);
    }
    *reinterpret_cast<uint4*>(dpre_x + pix * g.C + c0) = o;
  }
}

// AdamW (decoupled weight decay), then the BF16 copy used by the GEMMs.
__global__ void step_inc_kernel(int* step) { *step += 1; }

// lr and the step count live in device memory, so that a captured training
// step replays with the current values.
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                             float* __restrict__ v, int64_t n, const float* __restrict__ lr_dev, float b1, float b2,
                             float eps, float wd, const int* __restrict__ step, bf16* __restrict__ p16) {
  const float lr = *lr_dev;
  const float c1 = 1.f - powf(b1, static_cast<float>(*step)), c2 = 1.f - powf(b2, static_cast<float>(*step));
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] * (1.f - lr * wd);
    pi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (p16) p16[i] = __float2bfloat16_rn(pi);
  }
}

// Network input: stored float16 gathers [n][S][T][X] of the samples ids[0..B)
// as BF16 NHWC [B][T][X][S] divided by the normalisation scale.
// One thread per (model, t, x) pixel: its S <= 8 samples come from S planes
// of the stored gathers (each plane read coalesced across the warp); a
// block's 256 x S outputs leave through shared memory as 16-byte stores.
// 32-bit pixel indices (the host checks the count).
__global__ void __launch_bounds__(256) gathers_nhwc_px_kernel(const uint16_t* __restrict__ stored,
                                                              const int* __restrict__ ids, int S, int T, int X,
                                                              float scale, bf16* __restrict__ out, int total_px) {
  __shared__ __align__(16) bf16 buf[256 * 8];
  const int64_t plane = static_cast<int64_t>(T) * X;
  for (int p0 = blockIdx.x * 256; p0 < total_px; p0 += gridDim.x * 256) {
    const int p = p0 + threadIdx.x;
    if (p < total_px) {
      const int x = p % X, bt = p / X;
      const int t = bt % T, b = bt / T;
      const uint16_t* src = stored + static_cast<int64_t>(ids[b]) * S * plane + static_cast<int64_t>(t) * X + x;
      for (int s = 0; s < S; ++s)
        buf[threadIdx.x * S + s] =
            __float2bfloat16_rn(__fdiv_rn(__half2float(__ushort_as_half(src[s * plane])), scale));
    }
    __syncthreads();
    const int n = min(256, total_px - p0) * S;   // this block's outputs, from a 16-byte aligned start
    bf16* dst = out + static_cast<int64_t>(p0) * S;
    for (int j = threadIdx.x; j < n / 8; j += 256)
      reinterpret_cast<uint4*>(dst)[j] = reinterpret_cast<const uint4*>(buf)[j];
    for (int j = (n / 8) * 8 + threadIdx.x; j < n; j += 256) dst[j] = buf[j];
    __syncthreads();
  }
}

__global__ void gathers_nhwc_kernel(const uint16_t* __restrict__ stored, const int* __restrict__ ids, int B, int S,
                                    int T, int X, float scale, bf16* __restrict__ out) {
  const int64_t total = static_cast<int64_t>(B) * T * X * S;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int s = static_cast<int>(i % S);
    const int64_t tx = i / S;
    const int x = static_cast<int>(tx % X);
    const int64_t bt = tx / X;
    const int t = static_cast<int>(bt % T);
    const int b = static_cast<int>(bt / T);
    const int64_t src = ((static_cast<int64_t>(ids[b]) * S + s) * T + t) * X + x;
    const float v = __fdiv_rn(__half2float(__ushort_as_half(stored[src])), scale);
    out[i] = __float2bfloat16_rn(v);
  }
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const int* __restrict__ ids, int B, int64_t row,
                                   float* __restrict__ out) {
  const int64_t total = static_cast<int64_t>(B) * row;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = src[static_cast<int64_t>(ids[i / row]) * row + i % row];
}

int grid_for_l(long long total) {
  return static_cast<int>(std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 32)));
}

ConvGeom conv_geom(const int32_t* d) {
  ConvGeom g{d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], d[10], 0, 0};
  g.Hout = (g.Hin * g.up + 2 * g.ph - g.KH) / g.sh + 1;
  g.Wout = (g.Win * g.up + 2 * g.pw - g.KW) / g.sw + 1;
  return g;
}
}  // namespace

extern "C" {

int32_t ss_gemm_bf16_layout(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N,
                            int32_t K, int32_t layout, int32_t epi, void* C, int64_t ldc, const float* bias,
                            float slope, int32_t splits, int32_t* err, void* stream) {
  ss_internal::clear_error();
  if (layout != 0 && layout != 2 && layout != 3) return fail(SS_ERR_INVALID, "GEMM operand layout must be 0, 2 or 3");
  const bool amn = layout & 1, bmn = layout & 2;
  if (!A || !B || !C || !err || M < 1 || N < 1 || K < 1 || lda < (amn ? M : K) || ldb < (bmn ? N : K) || ldc < N)
    return fail(SS_ERR_INVALID, "bad GEMM arguments");
  if (epi < SS_EPI_F32 || epi > SS_EPI_BIAS_F32) return fail(SS_ERR_INVALID, "unknown GEMM epilogue");
  const int k_tiles = (K + kBK - 1) / kBK;
  // tile width: the smallest of 32 / 64 / 128 covering N, 256 for wide outputs with enough row tiles
  int bn = N <= 32 && !bmn ? 32 : N <= 64 ? 64 : 128;
  const int m_tiles = (M + kBM - 1) / kBM;
  if (N >= 256 && m_tiles * ((N + 255) / 256) >= 148 && k_tiles > 2) bn = 256;   // short K: 128-wide tiles, 4 CTAs per SM
  const int tiles = m_tiles * ((N + bn - 1) / bn);
  if (splits <= 0) {   // split the K loop only where the output is accumulated, to fill the GPU
    splits = 1;
    if (epi == SS_EPI_F32_ADD)
      splits = std::max(1, std::min(k_tiles / 4, (2 * 148 + tiles - 1) / tiles));
  }
  if (splits > 1 && epi != SS_EPI_F32_ADD) return fail(SS_ERR_INVALID, "split-K needs the accumulating epilogue");
  splits = std::min(splits, k_tiles);
  const int per = (k_tiles + splits - 1) / splits;
  splits = (k_tiles + per - 1) / per;   // every split gets at least one K tile
  // K-major operands: boxes of 64 K x the tile's rows; MN-major: boxes of 64 x 64 (M/N innermost)
  CUtensorMap ta, tb;
  int rc = amn ? make_tmap(&ta, A, M, K, lda, 64) : make_tmap(&ta, A, K, M, lda, kBM);
  if (rc) return rc;
  rc = bmn ? make_tmap(&tb, B, N, K, ldb, 64) : make_tmap(&tb, B, K, N, ldb, bn);
  if (rc) return rc;
  // ring depth: no deeper than the CTA's K steps, and the deepest ring with which two CTAs share an SM
  // (4 slots for tiles up to 64 wide, 3 for 128, 2 for 256: one CTA's epilogue then overlaps the other's
  // loads and MMAs); two slots for split-K (weight-gradient) CTAs, so that three share an SM.  Each choice
  // timed faster than one CTA per SM with four slots.
  const int fit2 = bn >= 256 ? 2 : bn >= 128 ? 3 : kStagesG;
  const int stages = std::min(epi == SS_EPI_F32_ADD ? 2 : fit2, per);
  GemmArgs g{M, N, K, k_tiles, per, C, ldc, bias, slope, err, stages};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // BF16 outputs of one- or two-step K loops (epilogue-bound: the input-gradient GEMMs) leave through tile
  // stores where TMA can address their rows (16-byte aligned base and stride); with longer K loops the
  // per-thread stores timed faster inside the training step
  CUtensorMap tc;
  std::memset(&tc, 0, sizeof(tc));
  const bool tmac = epi == SS_EPI_BIAS_LRELU_BF16 && per <= 2 && ldc % 8 == 0 &&
                    (reinterpret_cast<uintptr_t>(C) & 15) == 0;
  if (tmac) {
    rc = make_tmap_store(&tc, C, N, M, ldc);
    if (rc) return rc;
  }
  switch (bn) {
    case 32: return launch_gemm_bn<32>(layout, epi, tmac, ta, tb, tc, g, splits, st);
    case 64: return launch_gemm_bn<64>(layout, epi, tmac, ta, tb, tc, g, splits, st);
    case 128: return launch_gemm_bn<128>(layout, epi, tmac, ta, tb, tc, g, splits, st);
    default: return launch_gemm_bn<256>(layout, epi, tmac, ta, tb, tc, g, splits, st);
  }
}

int32_t ss_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                     int32_t epi, void* C, int64_t ldc, const float* bias, float slope, int32_t splits, int32_t* err,
                     void* stream) {
  return ss_gemm_bf16_layout(A, lda, B, ldb, M, N, K, 0, epi, C, ldc, bias, slope, splits, err, stream);
}

// conv: {B, Hin, Win, Cin, KH, KW, sh, sw, ph, pw, up}; the output size follows.
int32_t ss_im2col_bf16(const void* x, const int32_t* conv, int32_t Kc, void* cols, void* stream) {
  ss_internal::clear_error();
  if (!x || !conv || !cols) return fail(SS_ERR_INVALID, "bad arguments");
  const ConvGeom g = conv_geom(conv);
  const int K = g.KH * g.KW * g.Cin;
  if (g.Hout < 1 || g.Wout < 1 || g.up < 1 || g.sh < 1 || g.sw < 1 || Kc < K) return fail(SS_ERR_INVALID, "bad convolution");
  const long long M = static_cast<long long>(g.B) * g.Hout * g.Wout;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (g.Cin % 8 == 0 && Kc == K && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
           (reinterpret_cast<uintptr_t>(cols) & 15) == 0 && (g.Cin & (g.Cin - 1)) == 0 && M * K / 8 < (1LL << 31) &&
           static_cast<long long>(g.B) * g.Hin * g.Win * g.Cin < (1LL << 31)) {
    int c8_shift = 0;
    while ((8 << c8_shift) < g.Cin) ++c8_shift;
    const int chunks = K / 8;
    int lanes_shift = 0;
    while ((1 << lanes_shift) < chunks && lanes_shift < 5) ++lanes_shift;
    const int grid = static_cast<int>(std::max<long long>(1, std::min<long long>(
        (M * (1LL << lanes_shift) + 255) / 256, 148LL * 32)));
    const bf16* xx = static_cast<const bf16*>(x);
    bf16* cc = static_cast<bf16*>(cols);
    const int m = static_cast<int>(M);
    if (g.KW == 1 && g.up == 1)
      im2col_px_kernel<1, 1><<<grid, 256, 0, st>>>(xx, g, m, chunks, c8_shift, lanes_shift, cc);
    else if (g.KW == 3 && g.up == 1)
      im2col_px_kernel<3, 1><<<grid, 256, 0, st>>>(xx, g, m, chunks, c8_shift, lanes_shift, cc);
    else if (g.KW == 3 && g.up == 2)
      im2col_px_kernel<3, 2><<<grid, 256, 0, st>>>(xx, g, m, chunks, c8_shift, lanes_shift, cc);
    else
      im2col_px_kernel<0, 0><<<grid, 256, 0, st>>>(xx, g, m, chunks, c8_shift, lanes_shift, cc);
  } else if (g.Cin % 8 == 0 && Kc == K && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
             (reinterpret_cast<uintptr_t>(cols) & 15) == 0)
    im2col_vec8_kernel<<<grid_for_l(M * K / 8), 256, 0, st>>>(static_cast<const bf16*>(x), g, static_cast<bf16*>(cols));
  else if (Kc % 8 == 0 && Kc <= 96 && (reinterpret_cast<uintptr_t>(cols) & 15) == 0)
    im2col_rows_kernel<<<static_cast<int>(std::min<long long>((M + kRowThreads - 1) / kRowThreads, 148LL * 8)),
                         kRowThreads, kRowThreads * Kc * sizeof(bf16), st>>>(static_cast<const bf16*>(x), g, K, Kc,
                                                                             static_cast<bf16*>(cols));
  else
    im2col_kernel<<<grid_for_l(M * Kc), 256, 0, st>>>(static_cast<const bf16*>(x), g, K, Kc, static_cast<bf16*>(cols));
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_col2im16_lrelu_bf16(const void* dcols, const int32_t* conv, int32_t Kc, const void* y, float slope,
                               void* dpre, int64_t ldp, void* stream) {
  ss_internal::clear_error();
  if (!dcols || !conv || !y || !dpre) return fail(SS_ERR_INVALID, "bad arguments");
  const ConvGeom g = conv_geom(conv);
  if (g.B < 1 || g.Hin < 1 || g.Win < 1 || g.Cin < 1 || g.Hout < 1 || g.Wout < 1 || g.sh < 1 || g.sw < 1 || g.up < 1)
    return fail(SS_ERR_INVALID, "bad convolution geometry");
  if (ldp < g.Cin) return fail(SS_ERR_INVALID, "ldp < channels");
  if (g.Cin % 8 || Kc % 8 || Kc < g.KH * g.KW * g.Cin || (reinterpret_cast<uintptr_t>(dcols) & 15) ||
      (reinterpret_cast<uintptr_t>(y) & 15))
    return fail(SS_ERR_UNSUPPORTED, "BF16 column gradients need Cin % 8 == 0, Kc % 8 == 0 and 16-byte aligned buffers");
  const long long total = static_cast<long long>(g.B) * g.Hin * g.Win * (g.Cin / 8);
  if (total >= (1LL << 31)) return fail(SS_ERR_UNSUPPORTED, "too many input elements for one launch");
  int c8_shift = 0;
  while ((8 << c8_shift) < g.Cin) ++c8_shift;
  if ((8 << c8_shift) != g.Cin) return fail(SS_ERR_UNSUPPORTED, "BF16 column gradients need Cin / 8 a power of two");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int grid = grid_for_l(total);
  const bf16* dc = static_cast<const bf16*>(dcols);
  const bf16* yy = static_cast<const bf16*>(y);
  bf16* dp = static_cast<bf16*>(dpre);
  const int n = static_cast<int>(total);
  auto is = [&](int kh, int kw, int sh, int sw, int up) {
    return g.KH == kh && g.KW == kw && g.sh == sh && g.sw == sw && g.up == up;
  };
  if (is(4, 1, 2, 1, 1))
    col2im16_lrelu_kernel<4, 1, 2, 1, 1><<<grid, 256, 0, st>>>(dc, g, Kc, yy, slope, dp, ldp, n, c8_shift);
  else if (is(3, 3, 2, 2, 1))
    col2im16_lrelu_kernel<3, 3, 2, 2, 1><<<grid, 256, 0, st>>>(dc, g, Kc, yy, slope, dp, ldp, n, c8_shift);
  else if (is(3, 3, 1, 1, 2))
    col2im16_lrelu_kernel<3, 3, 1, 1, 2><<<grid, 256, 0, st>>>(dc, g, Kc, yy, slope, dp, ldp, n, c8_shift);
  else if (is(1, 1, 1, 1, 1))
    col2im16_lrelu_kernel<1, 1, 1, 1, 1><<<grid, 256, 0, st>>>(dc, g, Kc, yy, slope, dp, ldp, n, c8_shift);
  else
    col2im16_lrelu_kernel<0, 0, 0, 0, 0><<<grid, 256, 0, st>>>(dc, g, Kc, yy, slope, dp, ldp, n, c8_shift);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_bias_grad_bf16(const void* dpre, int64_t ld, int64_t M, int32_t C, float* db, void* stream) {
  ss_internal::clear_error();
  if (!dpre || !db || M < 1 || C < 1 || ld < C) return fail(SS_ERR_INVALID, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (C % 8 == 0 && ld % 8 == 0 && (reinterpret_cast<uintptr_t>(dpre) & 15) == 0) {
    // column passes of 256 groups across grid.y; row slabs of at least 32 rows across grid.x
    const int G = C / 8, passes = (G + 255) / 256;
    const long long ctas = std::max(1LL, std::min((static_cast<long long>(M) + 31) / 32, 148LL * 4 / passes + 1));
    const long long rows = (M + ctas - 1) / ctas;
    bias_grad_v8_kernel<<<dim3(static_cast<unsigned>((M + rows - 1) / rows), passes), 256, 0, st>>>(
        static_cast<const bf16*>(dpre), ld, M, C, rows, db);
  } else {
    dim3 grid((C + 127) / 128, static_cast<unsigned>(std::min<long long>(M, 512)));
    bias_grad_kernel<<<grid, 128, 0, st>>>(static_cast<const bf16*>(dpre), ld, M, C, db);
  }
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

// The 16-byte head kernels: channels a multiple of 8 (at most 64), 16-byte aligned map.
static bool head_v8_ok(const void* x, const HeadGeom& g) {
  return g.C % 8 == 0 && g.C <= 64 && (reinterpret_cast<uintptr_t>(x) & 15) == 0;
}

// head: {B, H, W, C, off, n}
int32_t ss_head_forward(const void* x, const int32_t* head, const float* w, const float* bias, float* out, void* stream) {
  ss_internal::clear_error();
  if (!x || !head || !w || !bias || !out) return fail(SS_ERR_INVALID, "bad arguments");
  const HeadGeom g{head[0], head[1], head[2], head[3], head[4], head[5]};
  if (g.off < 0 || g.off + g.n > g.H || g.off + g.n > g.W) return fail(SS_ERR_INVALID, "crop outside the map");
  const long long total = static_cast<long long>(g.B) * g.n * g.n;
  if (head_v8_ok(x, g))
    head_forward_v8_kernel<<<grid_for_l(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const bf16*>(x), g, w, bias, out);
  else
    head_forward_kernel<<<grid_for_l(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const bf16*>(x),
                                                                                         g, w, bias, out);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_head_backward(const void* x, const int32_t* head, const float* w, const float* dpre, float slope, float* dw,
                         float* db, void* dpre_x, void* stream) {
  ss_internal::clear_error();
  if (!x || !head || !w || !dpre || !dw || !db || !dpre_x) return fail(SS_ERR_INVALID, "bad arguments");
  const HeadGeom g{head[0], head[1], head[2], head[3], head[4], head[5]};
  if (9 * g.C > 1024) return fail(SS_ERR_UNSUPPORTED, "head with more than 113 channels");
  if (static_cast<long long>(g.B) * g.n * g.n >= (1LL << 31)) return fail(SS_ERR_UNSUPPORTED, "head output beyond 2^31 values");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long total = static_cast<long long>(g.B) * g.H * g.W * g.C;
  if (head_v8_ok(x, g) && (reinterpret_cast<uintptr_t>(dpre_x) & 15) == 0 && g.C == 32) {
    head_wgrad_v8_kernel<4><<<592, 256, 0, st>>>(static_cast<const bf16*>(x), g, dpre, dw, db);
    head_dgrad_v8_kernel<<<grid_for_l(total / 8), 256, 0, st>>>(static_cast<const bf16*>(x), g, dpre, w, slope,
                                                                 static_cast<bf16*>(dpre_x));
  } else {
    head_wgrad_kernel<<<296, 9 * g.C, 0, st>>>(static_cast<const bf16*>(x), g, dpre, dw, db);
    head_dgrad_kernel<<<grid_for_l(total), 256, 0, st>>>(static_cast<const bf16*>(x), g, dpre, w, slope,
                                                          static_cast<bf16*>(dpre_x));
  }
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_l1_tanh_loss(const float* pred, const float* target, int64_t n, float* loss_sum, float* dpre, void* stream) {
  ss_internal::clear_error();
  if (!pred || !target || !loss_sum || !dpre || n < 1) return fail(SS_ERR_INVALID, "bad arguments");
  l1_tanh_kernel<<<grid_for_l(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(pred, target, n, 1.f / n, loss_sum, dpre);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_adamw(float* p, const float* grad, float* m, float* v, int64_t n, const float* lr, float b1, float b2,
                 float eps, float wd, int32_t* step, void* p_bf16, void* stream) {
  ss_internal::clear_error();
  if (!p || !grad || !m || !v || !lr || !step || n < 1) return fail(SS_ERR_INVALID, "bad arguments");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  step_inc_kernel<<<1, 1, 0, st>>>(step);
  adamw_kernel<<<grid_for_l(n), 256, 0, st>>>(p, grad, m, v, n, lr, b1, b2, eps, wd, step, static_cast<bf16*>(p_bf16));
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_gather_rows_f32(const float* src, const int32_t* ids, int32_t B, int64_t row, float* out, void* stream) {
  ss_internal::clear_error();
  if (!src || !ids || !out || B < 1 || row < 1) return fail(SS_ERR_INVALID, "bad arguments");
  const long long total = static_cast<long long>(B) * row;
  gather_rows_kernel<<<grid_for_l(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(src, ids, B, row, out);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

int32_t ss_gathers_nhwc_bf16(const uint16_t* stored, const int32_t* ids, int32_t B, int32_t S, int32_t T, int32_t X,
                             float scale, void* out, void* stream) {
  ss_internal::clear_error();
  if (!stored || !ids || !out || B < 1 || S < 1 || T < 1 || X < 1) return fail(SS_ERR_INVALID, "bad arguments");
  if (!std::isfinite(scale) || !(scale > 0.f)) return fail(SS_ERR_INVALID, "Gather normalization scale must be finite and positive");
  const long long total = static_cast<long long>(B) * S * T * X;
  const long long px = static_cast<long long>(B) * T * X;
  if (S <= 8 && px < (1LL << 31) && (reinterpret_cast<uintptr_t>(out) & 15) == 0) {
    const int grid = static_cast<int>(std::min<long long>((px + 255) / 256, 148LL * 8));
    gathers_nhwc_px_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        stored, ids, S, T, X, scale, static_cast<bf16*>(out), static_cast<int>(px));
    SS_TRY_CUDA(cudaGetLastError());
    return SS_OK;
  }
  gathers_nhwc_kernel<<<grid_for_l(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(stored, ids, B, S, T, X, scale,
                                                                                       static_cast<bf16*>(out));
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

}  // extern "C"
