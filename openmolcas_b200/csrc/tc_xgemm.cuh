// Half-transform of the exchange build, X_J = L_J C, on the tcgen05 tensor
// cores with split-BF16 operands (three products Lhi Chi + Lhi Clo + Llo Chi,
// FP32 accumulation in tensor memory).  The epilogue writes X_J straight into
// the split, K-major operand of the exchange kernel (tc_syrk.cuh):
// XThi/XTlo[a][J*r + k] = split(X_J[a][k]).
//
// Operands, both K-major and staged by TMA with 128-byte swizzle into a
// 2-stage ring:
//   A = the dense split square L_J (rows J*ld + a, the K index b contiguous;
//       L_J is symmetric, so row a is column a)
//   B = C^T (rows k < r, the K index b contiguous: C column-major with
//       leading dimension ld); rows r..NB-1 of the box read as zero
// One CTA per (128-row tile of a, vector J, 256-column tile of k); M = 128,
// N = the column tile rounded up to a multiple of 16 (<= 256).  Warp roles
// and the bounded waits follow tc_syrk3_kernel.
#pragma once
#include <cuda_bf16.h>

#include "tc_syrk.cuh"

namespace mg {

constexpr int kXgStages = 2;
constexpr int kXgMaxN = 256;
constexpr int kXgAStage = 2 * kTcTileBytes;                 // Lhi, Llo: 128 x 64 BF16 each
constexpr int kXgBTile = kXgMaxN * kTcBK * 2;               // up to 256 x 64 BF16
constexpr int kXgStageBytes = kXgAStage + 2 * kXgBTile;     // + Chi, Clo
constexpr int kXgSmem = kXgStages * kXgStageBytes + 1024;

__host__ __device__ constexpr uint32_t tc_idesc_m128(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void tc_mma_n(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

// grid (ld / 128, nb, ceil(r / 256)); ld (rows of a square, K extent) a
// multiple of 128; XT row length kpad; bbox = rows of the C boxes of the
// tensor maps (the transaction size of a stage; rows beyond r read as zero).
__global__ void __launch_bounds__(128, 1)
    tc_xgemm3_kernel(const __grid_constant__ CUtensorMap map_lhi, const __grid_constant__ CUtensorMap map_llo,
                     const __grid_constant__ CUtensorMap map_chi, const __grid_constant__ CUtensorMap map_clo,
                     int ld, int r, int bbox, int kpad, __nv_bfloat16* __restrict__ xthi,
                     __nv_bfloat16* __restrict__ xtlo, int* __restrict__ err) {
  extern __shared__ uint8_t tc_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kXgStages], empty_bar[kXgStages], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  uint8_t* smem = (uint8_t*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * kTcTile, J = blockIdx.y;
  const int noff = blockIdx.z * kXgMaxN;
  const int nbn = min(kXgMaxN, (r - noff + 15) / 16 * 16);
  const int nk = ld / kTcBK;
  const uint32_t idesc = tc_idesc_m128(nbn);
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < kXgStages; ++s) {
      tc_mbar_init(tc_smem_addr(&full_bar[s]), 1);
      tc_mbar_init(tc_smem_addr(&empty_bar[s]), 1);
    }
    tc_mbar_init(tc_smem_addr(&done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&tmem_base)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  volatile int* abort = &abort_flag;
  const uint32_t btile = (uint32_t)bbox * kTcBK * 2;
  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    const uint32_t bytes = 2 * kTcTileBytes + 2 * btile;
    for (int s = 0; s < nk; ++s) {
      const int st = s % kXgStages;
      const uint32_t ph = (s / kXgStages) & 1;
      if (s >= kXgStages && !tc_mbar_wait(tc_smem_addr(&empty_bar[st]), ph ^ 1, abort)) break;
      uint8_t* base = smem + st * kXgStageBytes;
      const uint32_t fb = tc_smem_addr(&full_bar[st]);
      tc_mbar_expect_tx(fb, bytes);
      const int kx = s * kTcBK;
      tc_tma_load(tc_smem_addr(base), &map_lhi, fb, kx, J * ld + row0);
      tc_tma_load(tc_smem_addr(base + kTcTileBytes), &map_llo, fb, kx, J * ld + row0);
      tc_tma_load(tc_smem_addr(base + kXgAStage), &map_chi, fb, kx, noff);
      tc_tma_load(tc_smem_addr(base + kXgAStage + kXgBTile), &map_clo, fb, kx, noff);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int s = 0; s < nk; ++s) {
      const int st = s % kXgStages;
      const uint32_t ph = (s / kXgStages) & 1;
      if (!tc_mbar_wait(tc_smem_addr(&full_bar[st]), ph, abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint8_t* base = smem + st * kXgStageBytes;
      const uint64_t ahi = tc_desc_sw128(tc_smem_addr(base));
      const uint64_t alo = tc_desc_sw128(tc_smem_addr(base + kTcTileBytes));
      const uint64_t bhi = tc_desc_sw128(tc_smem_addr(base + kXgAStage));
      const uint64_t blo = tc_desc_sw128(tc_smem_addr(base + kXgAStage + kXgBTile));
#pragma unroll
      for (int kk = 0; kk < kTcBK / 16; ++kk) {
        const uint64_t o = 2 * kk;
        tc_mma_n(tmem, ahi + o, bhi + o, idesc, (s > 0 || kk > 0) ? 1u : 0u);
        tc_mma_n(tmem, ahi + o, blo + o, idesc, 1u);
        tc_mma_n(tmem, alo + o, bhi + o, idesc, 1u);
      }
      tc_commit(tc_smem_addr(&empty_bar[st]));
    }
    tc_commit(tc_smem_addr(&done_bar));
  }
  __syncwarp();
  // ---- epilogue: row a = row0 + 32 warp + lane, columns k < r -> split X^T
  int never = 0;
  const bool ok = tc_mbar_wait(tc_smem_addr(&done_bar), 0, (volatile int*)&never) && !*abort;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // The accumulator goes through shared memory (the pipeline ring is idle once
  // done_bar has fired): each warp moves its 32 TMEM lanes to rows of a
  // staging tile, then whole warps write rows of X^T with coalesced stores.
  float* stage = reinterpret_cast<float*>(smem);
  const int sp = nbn | 1;  // odd row stride: the 32 lanes of a warp hit distinct banks
  if (ok) {
#pragma unroll 1
    for (int cb = 0; cb * 32 < nbn; ++cb) {
      uint32_t v[32];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float* srow = stage + (size_t)(warp * 32 + lane) * sp + cb * 32;
#pragma unroll
      for (int jj = 0; jj < 32; ++jj)
        if (cb * 32 + jj < nbn) srow[jj] = __uint_as_float(v[jj]);
    }
  }
  __syncthreads();
  if (ok) {
    const int ncol = min(nbn, r - noff);
    for (int rho = warp; rho < kTcTile; rho += 4) {
      const size_t base = (size_t)(row0 + rho) * kpad + (size_t)J * r + noff;
      const float* srow = stage + (size_t)rho * sp;
      for (int k = lane; k < ncol; k += 32) {
        const float x = srow[k];
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        xthi[base + k] = h;
        xtlo[base + k] = __float2bfloat16_rn(x - __bfloat162float(h));
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
  }
}

}  // namespace mg
