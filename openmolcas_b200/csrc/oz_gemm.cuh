// Exact-integer sliced GEMMs on the tcgen05 tensor cores (kind::i8), the
// engine of the mixed-precision exchange build.
//
// Scheme (Ozaki-style splitting).  Every row i of an operand is scaled by a
// power of two 2^-e_i (e_i = frexp exponent of the row's largest |x|, so
// y = x 2^-e_i lies in (-1, 1)) and cut into s 8-bit slices:
//   y = 2^-7 S_0 + sum_{p>=1} 2^-(7+8p) U_p + tail,  |tail| < 2^-(7+8(s-1)),
//   S_0 = floor(128 y) in [-128, 127] (signed), U_p in [0, 255] (unsigned)
// (each remainder after a floor lies in [0, 1)).  A product of two sliced
// operands is then
//   (A B^T)_ij = 2^(e_i + f_j) sum_d 2^-(14+8d) sum_{p+q=d} (A_p B_q^T)_ij
// truncated to d <= s-1.  Each (A_p B_q^T) runs on the tensor cores in 8-bit
// integers with exact INT32 accumulation in tensor memory (one accumulator
// per diagonal d); accumulators are read out and combined in FP64 after at
// most kOzKChunk products per element (4096 * 6 * 255^2 < 2^31), so the only
// roundings are the FP64 combination and the truncated tail.
//
// Operand layout in HBM (blocked): slice p of a matrix of R rows and K
// 8-bit columns is stored as tiles of BR rows x 32 bytes (one MMA K step),
// each tile contiguous (BR * 32 bytes), tiles ordered K step fastest, then
// row tile:  byte (row, k) at ((row / BR) (K / 32) + k / 32) BR 32 +
// (row % BR) 32 + k % 32  (oz_blk_off).  BR = 128 for A operands, Nt for the
// B operand of the half-transform.  A TMA box is then one contiguous run of
// memory (whole cache lines), not BR separate 32-byte pieces.
//
// One CTA of 192 threads per SM:
//   warp 4 lane 0   TMA producer: per K step of 32, the slices 0..d1-1 of the
//                   A tile (128 rows) and of the B tile (Nt rows), 32-byte
//                   swizzle, into a ring of stages guarded by mbarriers
//   warp 5          allocates the 512 TMEM columns; lane 0 issues the MMAs
//                   (M = 128, N = Nt, K = 32), releases stages with
//                   tcgen05.commit and signals a full set of accumulators
//   warps 0-3       epilogue: TMEM lanes 32w..32w+31, combine the diagonals
//                   in FP64, scale, write (half-transform) or accumulate into
//                   a CTA-private FP64 tile (exchange product)
// The diagonals of one output tile are computed in passes of at most nd
// accumulators (nd * acc_stride <= 512 TMEM columns); a pass loads only the
// slices it needs.  The half-transform picks its column tile so that all s
// diagonals fit (one pass: the epilogue writes X once and records every row's
// largest |X| for the slicing that follows); the exchange product runs its
// 128 x 128 tiles in passes of 4 diagonals into CTA-private FP64 tiles.  Every mbarrier wait is bounded: a wait that runs out sets
// *err, the CTA stops issuing work, waits (bounded) for its own loads and
// MMAs in flight and still frees its tensor memory.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tc_common.cuh"

namespace mg {

constexpr int kOzThreads = 192;
constexpr int kOzMaxStages = 8;
constexpr int kOzMaxSlices = 8;
constexpr int kOzKChunk = 4096;  // K elements between accumulator read-outs
constexpr int kOzABytes = 128 * 32;
// dynamic shared memory of every launch of the kernels (the attribute is set
// once per device to this size; stages are planned within it)
constexpr int kOzSmemLimit = 221 * 1024;

// 2^k for -1022 <= k <= 1023
__device__ __forceinline__ double oz_pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }
// 2^e for any int e (outside the normal range through ldexp)
__device__ __forceinline__ double oz_pow2e(int e) { return (e >= -1022 && e <= 1023) ? oz_pow2(e) : ldexp(1.0, e); }

// Exact int32 -> double on the FP64 adder: the double with high word
// 0x43380000 and low word x + 2^31 is 1.5 2^52 + 2^31 + x; subtracting that
// offset leaves x exactly.
__device__ __forceinline__ double oz_i2d(uint32_t v) {
  return __hiloint2double(0x43380000, (int)(v ^ 0x80000000u)) - 6755401588539392.0;
}

// byte offset of element (row, k) of one blocked slice (K columns, tiles of
// br rows x 32 bytes)
__host__ __device__ __forceinline__ size_t oz_blk_off(long long row, long long k, long long kdim, int br) {
  return ((size_t)(row / br) * (size_t)(kdim >> 5) + (size_t)(k >> 5)) * (size_t)(br * 32) + (size_t)(row % br) * 32 +
         (size_t)(k & 31);
}

struct OzArgs {
  int s;           // slices
  int nd;          // accumulators per pass
  int acc_stride;  // TMEM columns per accumulator
  int Nt;          // rows of a B tile (MMA N)
  int stages, stage_bytes;
  int b_bytes;     // shared-memory stride of one B slice tile (multiple of 1024)
  int nitems;
  int* err;
  // half-transform X_J = L_J C (SYRK == false): items (row tile, vector, column tile)
  int nrt, nJ, nnt;
  int ld;          // rows (and K extent) of one vector's square
  int n;           // valid rows / columns (nbf)
  int r;           // columns of C
  const int* eA;   // row exponents of the L slices, [J * ld + a]
  const double* fB;  // column scale factors of C, 2^f_k
  double* X;       // X[(J * r + k) * xld + a] (FP64, column-major)
  int xld;
  unsigned long long* xmax;  // per row a: bits of the largest |X| written (atomicMax)
  // exchange product K += X X^T (SYRK == true): items (lower tile, block, sub-chunk)
  int ntile, nblk, nsub;
  int kblk;        // K extent of one block (multiple of 32)
  int ksub;        // K elements of a sub-chunk (multiple of 32)
  const int* eX;   // row exponents of the X slices, [blk * ld + a]
  double* P;       // CTA-private FP64 tiles, 128 x 128 per CTA (column-major)
  double* K;       // column-major n x n (lower triangle accumulated)
};

// One unit of tensor-core work: an output tile, a K range, one pass of diagonals.
struct OzUnit {
  int rowA, rowB;  // first row of the A and B tiles in their tensor maps
  int k0, nk;      // K range [k0, k0 + 32 nk)
  int d0, d1;      // diagonals [d0, d1)
  bool same;       // B tile == A tile (diagonal tile of the exchange product)
  // epilogue context
  int t0, t1, J, nt;  // X: row tile, (unused), vector, column tile; SYRK: ti, tj, block
  bool first;      // first unit of this output tile (write instead of add)
  bool last;       // last unit of this output tile in this CTA
};

__device__ __forceinline__ void oz_tile_ij(int x, int& ti, int& tj) {
  ti = (int)((sqrtf(8.0f * x + 1.0f) - 1.0f) * 0.5f);
  while ((ti + 1) * (ti + 2) / 2 <= x) ++ti;
  while (ti * (ti + 1) / 2 > x) --ti;
  tj = x - ti * (ti + 1) / 2;
}

// Enumerate this CTA's units in a fixed order (every role walks the same list).
template <bool SYRK, typename F>
__device__ __forceinline__ void oz_for_units(const OzArgs& a, F&& f) {
  const int npass = (a.s + a.nd - 1) / a.nd;
  if (!SYRK) {
    const int nsubk = (a.ld + kOzKChunk - 1) / kOzKChunk;
    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
      const int nt = item % a.nnt, r1 = item / a.nnt, J = r1 % a.nJ, rt = r1 / a.nJ;
      for (int sk = 0; sk < nsubk; ++sk)
        for (int g = 0; g < npass; ++g) {
          OzUnit u;
          u.rowA = J * a.ld + rt * 128;
          u.rowB = nt * a.Nt;
          u.k0 = sk * kOzKChunk;
          u.nk = (min(a.ld, u.k0 + kOzKChunk) - u.k0) / 32;
          u.d0 = g * a.nd;
          u.d1 = min(a.s, u.d0 + a.nd);
          u.same = false;
          u.t0 = rt; u.t1 = 0; u.J = J; u.nt = nt;
          u.first = sk == 0 && g == 0;
          u.last = sk == nsubk - 1 && g == npass - 1;
          if (!f(u)) return;
        }
    }
  } else {
    // items in (block, sub-chunk, tile) order, strided over the CTAs: the
    // CTAs that run at the same time take the tiles of one or two K
    // sub-chunks, whose slices stay in L2 while they are read; every item is
    // a complete segment (its passes add into the CTA-private tile, then the
    // tile is added into K)
    for (int item = blockIdx.x; item < a.nitems; item += gridDim.x) {
      const int tile = item % a.ntile, r1 = item / a.ntile, sub = r1 % a.nsub, blk = r1 / a.nsub;
      int ti, tj;
      oz_tile_ij(tile, ti, tj);
      const int kb0 = sub * a.ksub;
      const int kb1 = min(a.kblk, kb0 + a.ksub);
      if (kb1 <= kb0) {  // the planner never makes an empty sub-chunk; every role stops here alike
        if (threadIdx.x == 0) atomicExch(a.err, 2);
        return;
      }
      // the highest diagonals first: the later pass then needs only the
      // slices of its own (low) diagonals
      for (int g = 0; g < npass; ++g) {
        OzUnit u;
        u.rowA = ti * 128;
        u.rowB = tj * 128;
        u.k0 = blk * a.kblk + kb0;
        u.nk = (kb1 - kb0) / 32;
        u.d1 = a.s - g * a.nd;
        u.d0 = max(0, u.d1 - a.nd);
        u.same = ti == tj;
        u.t0 = ti; u.t1 = tj; u.J = blk; u.nt = 0;
        u.first = g == 0;
        u.last = g == npass - 1;
        if (!f(u)) return;
      }
    }
  }
}

// The MMAs of diagonals [D0, D1) for one K step of 32, unrolled: the slice
// p of A and q of B are descriptor offsets (p * 4096 and q * bst bytes, in
// 16-byte units), id[] the four signedness variants of the instruction
// descriptor, (p == 0 ? 2 : 0) + (q == 0 ? 1 : 0); the first product of
// every accumulator overwrites it at the first K step of a unit.
template <int D0, int D1>
__device__ __forceinline__ void oz_issue(uint32_t tmem, int acc_stride, uint64_t da, uint64_t db, uint32_t bst,
                                         const uint32_t (&id)[4], bool first) {
#pragma unroll
  for (int d = D0; d < D1; ++d) {
    const uint32_t acc = tmem + (uint32_t)((d - D0) * acc_stride);
#pragma unroll
    for (int p = 0; p <= d; ++p) {
      const int q = d - p;
      tc_mma_i8(acc, da + (uint64_t)(p * (kOzABytes >> 4)), db + (uint64_t)q * bst,
                id[(p == 0 ? 2 : 0) + (q == 0 ? 1 : 0)], (first && p == 0) ? 0u : 1u);
    }
  }
}

// Accumulators per pass: all NS diagonals for the half-transform (its column
// tile is chosen so that they fit), 4 of 128 columns for the exchange product.
template <bool SYRK, int NS>
struct OzPass {
  static constexpr int nd = SYRK ? (NS < 4 ? NS : 4) : NS;
};

template <bool SYRK, int NS>
__global__ void __launch_bounds__(kOzThreads, 1)
    oz_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const OzArgs a) {
  constexpr int ND = OzPass<SYRK, NS>::nd;
  if (a.s != NS || a.nd != ND) {  // launched with another plan: nothing has started yet
    if (threadIdx.x == 0) atomicExch(a.err, 3);
    return;
  }
  extern __shared__ uint8_t oz_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kOzMaxStages], empty_bar[kOzMaxStages], accf_bar, acce_bar;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  uint8_t* smem = (uint8_t*)(((uintptr_t)oz_smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int* abort = &abort_flag;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (int s = 0; s < a.stages; ++s) {
      tc_mbar_init(tc_smem_addr(&full_bar[s]), 1);
      tc_mbar_init(tc_smem_addr(&empty_bar[s]), 1);
    }
    tc_mbar_init(tc_smem_addr(&accf_bar), 1);
    tc_mbar_init(tc_smem_addr(&acce_bar), 4);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(&tmem_base)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const int S = a.stages;
  if (warp == 4) {
    if (lane == 0) {
      // ---- TMA producer
      int it = 0;
      oz_for_units<SYRK>(a, [&](const OzUnit& u) -> bool {
        const int nsl = u.d1;  // slices 0..d1-1 of both operands
        const uint32_t bytes = nsl * (kOzABytes + (u.same ? 0 : 32 * a.Nt));
        for (int kk = 0; kk < u.nk; ++kk, ++it) {
          const int st = it % S;
          const uint32_t ph = (it / S) & 1;
          if (it >= S && !tc_mbar_wait(tc_smem_addr(&empty_bar[st]), ph ^ 1, abort)) return false;
          uint8_t* base = smem + (size_t)st * a.stage_bytes;
          const uint32_t fb = tc_smem_addr(&full_bar[st]);
          tc_mbar_expect_tx(fb, bytes);
          // blocked operands: (32-byte K step, row tile) addresses one contiguous box
          const int ks = (u.k0 >> 5) + kk;
          for (int p = 0; p < nsl; ++p)
            tc_tma_load5(tc_smem_addr(base + p * kOzABytes), &mapA, fb, 0, 0, ks, u.rowA >> 7, p);
          if (!u.same)
            for (int q = 0; q < nsl; ++q)
              tc_tma_load5(tc_smem_addr(base + a.s * kOzABytes + q * a.b_bytes), &mapB, fb, 0, 0, ks, u.rowB / a.Nt,
                           q);
        }
        return true;
      });
      // do not leave while loads of this CTA are still landing: wait (bounded)
      // for the last ring's worth of stages to fill
      int never = 0;
      for (int k = (it > S ? it - S : 0); k < it; ++k)
        tc_mbar_wait(tc_smem_addr(&full_bar[k % S]), (k / S) & 1, (volatile int*)&never);
    }
  } else if (warp == 5) {
    if (lane == 0) {
      // ---- MMA issuer
      const uint32_t id[4] = {tc_idesc_i8(a.Nt, false, false), tc_idesc_i8(a.Nt, false, true),
                              tc_idesc_i8(a.Nt, true, false), tc_idesc_i8(a.Nt, true, true)};
      int it = 0, un = 0;
      oz_for_units<SYRK>(a, [&](const OzUnit& u) -> bool {
        // the accumulators must have been read out by the epilogue
        if (un > 0 && !tc_mbar_wait(tc_smem_addr(&acce_bar), (un - 1) & 1, abort)) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        bool ok = true;
        for (int kk = 0; kk < u.nk; ++kk, ++it) {
          const int st = it % S;
          const uint32_t ph = (it / S) & 1;
          if (!tc_mbar_wait(tc_smem_addr(&full_bar[st]), ph, abort)) { ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          uint8_t* base = smem + (size_t)st * a.stage_bytes;
          const uint32_t abase = tc_smem_addr(base);
          const uint32_t bbase = u.same ? abase : tc_smem_addr(base + a.s * kOzABytes);
          const uint32_t bst = (u.same ? kOzABytes : a.b_bytes) >> 4;
          const uint64_t da = tc_desc_sw32(abase), db = tc_desc_sw32(bbase);
          // at most two passes: diagonals [NS - ND, NS), then [0, NS - ND)
          constexpr int DH = NS - ND;
          if (u.d1 == NS) oz_issue<DH, NS>(tmem, a.acc_stride, da, db, bst, id, kk == 0);
          else oz_issue<0, DH>(tmem, a.acc_stride, da, db, bst, id, kk == 0);
          tc_commit(tc_smem_addr(&empty_bar[st]));
        }
        // accumulators complete (also after a failure, so the epilogue's wait drains the MMAs in flight)
        tc_commit(tc_smem_addr(&accf_bar));
        ++un;
        return ok;
      });
    }
  } else {
    // ---- epilogue, warps 0-3: row 32 warp + lane of the output tile
    const int row = warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    int un = 0;
    oz_for_units<SYRK>(a, [&](const OzUnit& u) -> bool {
      int never = 0;
      bool ok = tc_mbar_wait(tc_smem_addr(&accf_bar), un & 1, (volatile int*)&never) && !*abort;
      ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld below needs the whole warp
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        const int ncol = SYRK ? 128 : a.Nt;
        double rmax = 0.0;
        // row scale factor of this thread's output row (power of two)
        const int arow = u.t0 * 128 + row;
        const double fa = SYRK ? oz_pow2e(a.eX[u.J * a.ld + arow]) : (arow < a.n ? oz_pow2e(a.eA[u.J * a.ld + arow]) : 0.0);
        for (int c0 = 0; c0 < ncol; c0 += 16) {
          double sum[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) sum[i] = 0.0;
          {
            // every accumulator's 16 columns in flight at once, one wait
            uint32_t v[ND][16];
            const int nacc = u.d1 - u.d0;
#pragma unroll
            for (int j = 0; j < ND; ++j)
              if (j < nacc) tc_ld16_async(tl + (uint32_t)(j * a.acc_stride + c0), v[j]);
            tc_ld_wait();
#pragma unroll
            for (int j = 0; j < ND; ++j)
              if (j < nacc) {
                tc_ld_bind(v[j]);
                const double w = oz_pow2(-14 - 8 * (u.d0 + j));
#pragma unroll
                for (int i = 0; i < 16; ++i) sum[i] = fma(oz_i2d(v[j][i]), w, sum[i]);
              }
          }
          // (the scaling by powers of two is exact; the warp's 32 rows of one
          // column are consecutive in X and in the tile)
          if (!SYRK) {
            if (arow < a.n) {
              double* xc = a.X + (size_t)u.J * a.r * a.xld + arow;
#pragma unroll
              for (int i = 0; i < 16; ++i) {
                const int k = u.nt * a.Nt + c0 + i;
                if (k < a.r) {
                  const double val = sum[i] * fa * a.fB[k];
                  double* xp = xc + (size_t)k * a.xld;
                  *xp = u.first ? val : *xp + val;
                  rmax = fmax(rmax, fabs(val));
                }
              }
            }
          } else {
            const int* eb = a.eX + u.J * a.ld + u.t1 * 128 + c0;
            double* pc = a.P + (size_t)blockIdx.x * 128 * 128 + (size_t)c0 * 128 + row;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const double val = sum[i] * fa * oz_pow2e(eb[i]);
              pc[i * 128] = u.first ? val : pc[i * 128] + val;
            }
          }
        }
        if (!SYRK && u.last && rmax > 0.0)  // (a single pass: the values written are final)
          atomicMax(a.xmax + u.t0 * 128 + row, (unsigned long long)__double_as_longlong(rmax));
        if (SYRK && u.last) {
          // this CTA's share of the tile is complete: add it into K
          const double* pc = a.P + (size_t)blockIdx.x * 128 * 128 + row;
          if (arow < a.n)
            for (int c = 0; c < 128; ++c) {
              const int bcol = u.t1 * 128 + c;
              if (bcol < a.n) atomicAdd(&a.K[(size_t)arow + (size_t)a.n * bcol], pc[c * 128]);
            }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) tc_mbar_arrive(tc_smem_addr(&acce_bar));
      ++un;
      if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
      return ok;
    });
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (*abort && threadIdx.x == 0) atomicExch(a.err, 1);
  if (warp == 5) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

}  // namespace mg
