// Exchange build K += X X^T on the 5th-generation tensor cores (tcgen05),
// with X split into two BF16 pieces (X = Xhi + Xlo) and three products
// Xhi Xhi^T + Xhi Xlo^T + Xlo Xhi^T accumulated in FP32 in tensor memory.
//
// Operands are K-major (row a of X^T holds the K index contiguous), staged
// by TMA with 128-byte swizzle into a 3-stage shared-memory ring:
//   warp 0 lane 0  TMA producer (cp.async.bulk.tensor, mbarrier complete_tx)
//   warp 1 lane 0  MMA issuer (tcgen05.mma kind::f16, M = N = 128, K = 16),
//                  tcgen05.commit releases a stage / signals the accumulator
//   warp 2         allocates and frees 128 TMEM columns
//   warps 0-3      epilogue: tcgen05.ld 32 lanes x 32 columns per warp, FP64
//                  atomic add into K (split-K CTAs share an output tile)
// Only output tiles on or below the diagonal are computed (K is symmetric;
// the caller mirrors the lower triangle).  Every mbarrier wait is bounded: a
// wait that runs out sets *err, the CTA stops issuing work and still frees
// its tensor memory.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mg {

constexpr int kTcTile = 128;           // output tile edge (rows of X^T per operand tile)
constexpr int kTcBK = 64;              // K elements per stage (128 bytes of BF16)
constexpr int kTcStages = 3;
constexpr int kTcTileBytes = kTcTile * kTcBK * 2;  // 16 KB
constexpr int kTcStageBytes = 4 * kTcTileBytes;   // Ahi, Alo, Bhi, Blo
constexpr int kTcSmem = kTcStages * kTcStageBytes + 1024;  // + alignment slack
constexpr long long kTcWaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tc_mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false when it ran out or
// another role of the CTA already gave up.
__device__ __forceinline__ bool tc_mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
  for (long long i = 0; i < kTcWaitLimit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if (*abort) return false;
  }
  *abort = 1;
  return false;
}

__device__ __forceinline__ void tc_tma_load(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"((uint64_t)map), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms of
// 1024 bytes stacked along M/N (stride byte offset 1024), Blackwell version 1.
__device__ __forceinline__ uint64_t tc_desc_sw128(uint32_t addr) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
  d |= (uint64_t)1 << 46;              // descriptor version
  d |= (uint64_t)2 << 61;              // SWIZZLE_128B
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = N = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// grid.x: lower-triangle output tiles (ti >= tj) of an ld x ld result,
// grid.y: split of the K range.  K (column-major, leading dimension n) +=
// lower tiles of Xhi Xhi^T + Xhi Xlo^T + Xlo Xhi^T.  ld is a multiple of 128,
// kdim of 64 * gridDim.y.
__global__ void __launch_bounds__(128, 1)
    tc_syrk3_kernel(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo, int n,
                    int kdim, double* __restrict__ K, int* __restrict__ err) {
  extern __shared__ uint8_t tc_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kTcStages], empty_bar[kTcStages], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  uint8_t* smem = (uint8_t*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // tile (ti, tj), ti >= tj, from the triangular index
  const int x = blockIdx.x;
  int ti = (int)((sqrtf(8.0f * x + 1.0f) - 1.0f) * 0.5f);
  while ((ti + 1) * (ti + 2) / 2 <= x) ++ti;
  while (ti * (ti + 1) / 2 > x) --ti;
  const int tj = x - ti * (ti + 1) / 2;
  const bool diag = ti == tj;
  const int kpart = kdim / gridDim.y;
  const int k0 = blockIdx.y * kpart;
  const int nk = kpart / kTcBK;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < kTcStages; ++s) {
      tc_mbar_init(tc_smem_addr(&full_bar[s]), 1);
      tc_mbar_init(tc_smem_addr(&empty_bar[s]), 1);
    }
    tc_mbar_init(tc_smem_addr(&done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  volatile int* abort = &abort_flag;
  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    const uint32_t bytes = diag ? 2 * kTcTileBytes : 4 * kTcTileBytes;
    for (int s = 0; s < nk; ++s) {
      const int st = s % kTcStages;
      const uint32_t ph = (s / kTcStages) & 1;
      if (s >= kTcStages && !tc_mbar_wait(tc_smem_addr(&empty_bar[st]), ph ^ 1, abort)) break;
      uint8_t* base = smem + st * kTcStageBytes;
      const uint32_t fb = tc_smem_addr(&full_bar[st]);
      tc_mbar_expect_tx(fb, bytes);
      const int kx = k0 + s * kTcBK;
      tc_tma_load(tc_smem_addr(base), &map_hi, fb, kx, ti * kTcTile);
      tc_tma_load(tc_smem_addr(base + kTcTileBytes), &map_lo, fb, kx, ti * kTcTile);
      if (!diag) {
        tc_tma_load(tc_smem_addr(base + 2 * kTcTileBytes), &map_hi, fb, kx, tj * kTcTile);
        tc_tma_load(tc_smem_addr(base + 3 * kTcTileBytes), &map_lo, fb, kx, tj * kTcTile);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int s = 0; s < nk; ++s) {
      const int st = s % kTcStages;
      const uint32_t ph = (s / kTcStages) & 1;
      if (!tc_mbar_wait(tc_smem_addr(&full_bar[st]), ph, abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint8_t* base = smem + st * kTcStageBytes;
      const uint64_t ahi = tc_desc_sw128(tc_smem_addr(base));
      const uint64_t alo = tc_desc_sw128(tc_smem_addr(base + kTcTileBytes));
      const uint64_t bhi = diag ? ahi : tc_desc_sw128(tc_smem_addr(base + 2 * kTcTileBytes));
      const uint64_t blo = diag ? alo : tc_desc_sw128(tc_smem_addr(base + 3 * kTcTileBytes));
#pragma unroll
      for (int kk = 0; kk < kTcBK / 16; ++kk) {
        const uint64_t o = 2 * kk;  // 32 bytes along K, in 16-byte units
        tc_mma(tmem, ahi + o, bhi + o, (s > 0 || kk > 0) ? 1u : 0u);
        tc_mma(tmem, ahi + o, blo + o, 1u);
        tc_mma(tmem, alo + o, bhi + o, 1u);
      }
      tc_commit(tc_smem_addr(&empty_bar[st]));
    }
    tc_commit(tc_smem_addr(&done_bar));
  }
  __syncwarp();
  // ---- epilogue: lane quarter `warp` of the accumulator.  The MMA issuer
  // always commits done_bar, so this wait also drains MMAs still in flight
  // after an abort (it does not give up early on the abort flag).
  int never = 0;
  const bool ok = tc_mbar_wait(tc_smem_addr(&done_bar), 0, (volatile int*)&never) && !*abort;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int row = ti * kTcTile + warp * 32 + lane;
#pragma unroll 1
    for (int cb = 0; cb < kTcTile / 32; ++cb) {
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
      if (row < n) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = tj * kTcTile + cb * 32 + j;
          if (col < n) atomicAdd(&K[(size_t)row + (size_t)n * col], (double)__uint_as_float(v[j]));
        }
      }
    }
  } else if (threadIdx.x == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 2) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
}

}  // namespace mg
