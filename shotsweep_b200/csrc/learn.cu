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
};

template <int BN>
constexpr size_t gemm_smem_bytes() {
  return 1024 + kStagesG * (kBM * 128 + BN * 128) + (2 * kStagesG + 1) * 8 + 16;
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    gemm_bf16_kernel(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, const GemmArgs g) {
  using namespace sm100;
  constexpr uint32_t A_BYTES = kBM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStagesG * STAGE);
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
      const int s = i % kStagesG;
      if (i >= kStagesG && !mbar_wait(empty(s), ((i / kStagesG) - 1) & 1, g.err, 1)) break;
      mbar_expect_tx(full(s), STAGE);
      tma_load_2d(sbase + s * STAGE, &ta, (kt0 + i) * kBK, m0, full(s));
      tma_load_2d(sbase + s * STAGE + A_BYTES, &tb, (kt0 + i) * kBK, n0, full(s));
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: four K=16 MMAs per stage, the stage freed on completion
    constexpr uint32_t idesc = idesc_bf16_f32(kBM, BN);
    for (int i = 0; i < nk; ++i) {
      const int s = i % kStagesG;
      if (!mbar_wait(full(s), (i / kStagesG) & 1, g.err, 2)) break;
      tc_fence_after();
      const uint64_t da = desc_sw128_kmajor(sbase + s * STAGE);
      const uint64_t db = desc_sw128_kmajor(sbase + s * STAGE + A_BYTES);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk)
        mma_bf16(taddr, da + 2 * kk, db + 2 * kk, idesc, (i > 0 || kk > 0) ? 1u : 0u);
      mma_commit(empty(s));
    }
    mma_commit(acc_bar);
  } else if (warp >= 2) {
    // ---- epilogue: warp w reads TMEM lanes 32*(w%4) .. +31, one row each --
    mbar_wait(acc_bar, 0, g.err, 3);
    tc_fence_after();
    const int q = warp & 3;
    const int row = m0 + q * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tmem_ld16(taddr + (static_cast<uint32_t>(q * 32) << 16) + c, v);
      if (row >= g.M) continue;
      const long long off = static_cast<long long>(row) * g.ldc;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int col = n0 + c + j;
        if (col >= g.N) break;
        float x = v[j];
        if (EPI == SS_EPI_F32) {
          static_cast<float*>(g.c)[off + col] = x;
        } else if (EPI == SS_EPI_F32_ADD) {
          atomicAdd(static_cast<float*>(g.c) + off + col, x);
        } else if (EPI == SS_EPI_BIAS_LRELU_BF16) {
          x += g.bias ? g.bias[col] : 0.f;
          x = x > 0.f ? x : g.slope * x;
          static_cast<bf16*>(g.c)[off + col] = __float2bfloat16_rn(x);
        } else {   // SS_EPI_BIAS_F32
          static_cast<float*>(g.c)[off + col] = x + (g.bias ? g.bias[col] : 0.f);
        }
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

template <int BN, int EPI>
int launch_gemm_t(const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, int splits, cudaStream_t st) {
  auto kern = gemm_bf16_kernel<BN, EPI>;
  constexpr size_t smem = gemm_smem_bytes<BN>();
  static std::once_flag once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(once, [&] {
    attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  });
  if (attr_err != cudaSuccess) return fail(SS_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(attr_err));
  dim3 grid((g.N + BN - 1) / BN, (g.M + kBM - 1) / kBM, splits);
  kern<<<grid, kGemmThreads, smem, st>>>(ta, tb, g);
  SS_TRY_CUDA(cudaGetLastError());
  return SS_OK;
}

template <int BN>
int launch_gemm_bn(int epi, const CUtensorMap& ta, const CUtensorMap& tb, const GemmArgs& g, int splits,
                   cudaStream_t st) {
  switch (epi) {
    case SS_EPI_F32: return launch_gemm_t<BN, SS_EPI_F32>(ta, tb, g, splits, st);
    case SS_EPI_F32_ADD: return launch_gemm_t<BN, SS_EPI_F32_ADD>(ta, tb, g, splits, st);
    case SS_EPI_BIAS_LRELU_BF16: return launch_gemm_t<BN, SS_EPI_BIAS_LRELU_BF16>(ta, tb, g, splits, st);
    default: return launch_gemm_t<BN, SS_EPI_BIAS_F32>(ta, tb, g, splits, st);
  }
}

}  // namespace

extern "C" {

int32_t ss_gemm_bf16(const void* A, int64_t lda, const void* B, int64_t ldb, int32_t M, int32_t N, int32_t K,
                     int32_t epi, void* C, int64_t ldc, const float* bias, float slope, int32_t splits, int32_t* err,
                     void* stream) {
  ss_internal::clear_error();
  if (!A || !B || !C || !err || M < 1 || N < 1 || K < 1 || lda < K || ldb < K || ldc < N)
    return fail(SS_ERR_INVALID, "bad GEMM arguments");
  if (epi < SS_EPI_F32 || epi > SS_EPI_BIAS_F32) return fail(SS_ERR_INVALID, "unknown GEMM epilogue");
  const int k_tiles = (K + kBK - 1) / kBK;
  // tile width: the smallest of 32 / 64 / 128 covering N, 256 for wide outputs with enough row tiles
  int bn = N <= 32 ? 32 : N <= 64 ? 64 : 128;
  const int m_tiles = (M + kBM - 1) / kBM;
  if (N >= 256 && m_tiles * ((N + 255) / 256) >= 148) bn = 256;
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
  CUtensorMap ta, tb;
  int rc = make_tmap(&ta, A, K, M, lda, kBM);
  if (rc) return rc;
  rc = make_tmap(&tb, B, K, N, ldb, bn);
  if (rc) return rc;
  GemmArgs g{M, N, K, k_tiles, per, C, ldc, bias, slope, err};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (bn) {
    case 32: return launch_gemm_bn<32>(epi, ta, tb, g, splits, st);
    case 64: return launch_gemm_bn<64>(epi, ta, tb, g, splits, st);
    case 128: return launch_gemm_bn<128>(epi, ta, tb, g, splits, st);
    default: return launch_gemm_bn<256>(epi, ta, tb, g, splits, st);
  }
}

}  // extern "C"
