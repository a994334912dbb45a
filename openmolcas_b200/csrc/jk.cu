// Coulomb / exchange matrices from Cholesky vectors (the CHO_LK_SCF build,
// fock_util/cho_lk_scf.F90:14) on the GPU.
//
//   D = C C^T (C: nbf x r, the Cholesky/orbital factor of the density, as
//   ChoSCF_Drv passes it, scf/choscf_drv.F90:115-116)
//   J_ab = sum_J L_ab,J V_J,  V_J = sum_cd L_cd,J D_cd     (cho_lk_scf.F90:442-449)
//   K_ab = sum_J sum_k X_J[a,k] X_J[b,k],  X_J = L_J C      (cho_lk_scf.F90:507-830)
//
// Mixed path: the FP64 vectors are cut into 8-bit slices per row (oz_gemm.cuh
// gives the scheme; s slices for the half-transform, sk for the exchange
// product, whose error dominates) and both exchange GEMMs run on the tcgen05
// tensor cores in 8-bit integers with exact INT32 accumulation: per block of
// vectors, a slicing kernel unpacks the rs-packed L_J into sliced dense
// squares (and forms the Coulomb contractions V_J on the way), the
// half-transform X_J = L_J C writes X in FP64, X is sliced per row over the
// block, and the exchange product K += X X^T runs over groups of blocks
// (lower-triangle tiles, CTA-private FP64 tiles, FP64 atomics into K).  J
// is FP64 throughout.
//
// FP64 path ("plain FP64 GPU path"): vectors in FP64, per block of vectors
// the rs-packed L_J are unpacked to dense symmetric nbf x nbf matrices, the
// half-transform is one strided-batched DGEMM and K accumulates by DSYRK.
// LK screening is not applied (dense tensor work is cheaper on the GPU than
// the screening bookkeeping); the result equals the unscreened reference.
#include <cublas_v2.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "kern_common.cuh"
#include "mg_internal.h"
#include "oz_gemm.cuh"

namespace mg {

// dw[t] = w_t D[a_t, b_t], w = 2 for a != b (both triangles), 1 on the diagonal
__global__ void k_pack_density(const int* __restrict__ rs_a, const int* __restrict__ rs_b, int64_t nrs,
                               const double* __restrict__ D, int n, double* __restrict__ dw) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  const int a = rs_a[t], b = rs_b[t];
  dw[t] = (a == b ? 1.0 : 2.0) * D[(size_t)a * n + b];
}

// J[a,b] = J[b,a] = jrs[t]
__global__ void k_unpack_sym(const int* __restrict__ rs_a, const int* __restrict__ rs_b, int64_t nrs,
                             const double* __restrict__ v, int n, double* __restrict__ M) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  const int a = rs_a[t], b = rs_b[t];
  M[(size_t)a * n + b] = v[t];
  M[(size_t)b * n + a] = v[t];
}

// Lsq[J][a][b] = Lsq[J][b][a] = L[t + nrs*J] for a block of nb vectors
__global__ void k_unpack_block(const int* __restrict__ rs_a, const int* __restrict__ rs_b, int64_t nrs,
                               const double* __restrict__ L, int nb, int n, double* __restrict__ Lsq) {
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= nrs * nb) return;
  const int64_t t = o % nrs;
  const int64_t J = o / nrs;
  const int a = rs_a[t], b = rs_b[t];
  const double v = L[t + nrs * J];
  double* M = Lsq + (size_t)J * n * n;
  M[(size_t)a * n + b] = v;
  M[(size_t)b * n + a] = v;
}

__global__ void k_symmetrize_lower(double* __restrict__ K, int n) {
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)n * n) return;
  const int i = (int)(o % n), j = (int)(o / n);
  if (i > j) K[(size_t)i * n + j] = K[(size_t)j * n + i];  // column-major lower -> full
}

static inline unsigned nb256(int64_t n) { return (unsigned)((n + 255) / 256); }

// F += J - factxi K (CHO_LK_SCF's FLT update)
__global__ void k_fock_acc(double* __restrict__ F, const double* __restrict__ J, const double* __restrict__ K,
                           double factxi, int64_t n) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) F[t] += J[t] - factxi * K[t];
}

int fock_accumulate(double* F, const double* J, const double* K, double factxi, int64_t n, cudaStream_t st) {
  k_fock_acc<<<nb256(n), 256, 0, st>>>(F, J, K, factxi, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : MG_ERR_CUDA;
}

struct JkWork {
  int* d_rs_a = nullptr;
  int* d_rs_b = nullptr;
  int64_t nrs = 0;
};

int jk_fp64(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block) {
  return jk_fp64_batch(h, 1, &d_C, &r, &d_J, &d_K, st, block);
}

// FP64 J/K of k densities: every block of vectors is unpacked once, each
// density runs its DGEMVs, half-transform and DSYRK on the squares.
int jk_fp64_batch(Handle* h, int k, const double* const* Cs, const int* rs_, double* const* Js, double* const* Ks,
                  cudaStream_t st, int block) {
  ChoState* c = h->cho;
  const int64_t nrs = cho_nrs(c);
  const int M = cho_nvec(c);
  const int n = h->nbf;
  if (k < 1) { h->err = "FP64 J/K: no density"; return MG_ERR_ARG; }
  int rmax = 0;
  for (int d = 0; d < k; ++d) {
    if (!Cs[d] || !Js[d] || !Ks[d] || rs_[d] < 1) { h->err = "FP64 J/K: a density of the batch has no factor or outputs"; return MG_ERR_ARG; }
    rmax = std::max(rmax, rs_[d]);
  }
  cublasHandle_t cb = cho_cublas(c);
  cublasSetStream(cb, st);
  const int* d_ra = cho_rs_a_dev(c);
  const int* d_rb = cho_rs_b_dev(c);
  // scratch: dw (k nrs), jrs (k nrs), V (block), D (n*n), Lsq (block*n*n), X (n * block * rmax)
  const size_t need = sizeof(double) * ((size_t)nrs * 2 * k + block + (size_t)n * n + (size_t)block * n * n +
                                        (size_t)n * block * rmax);
  double* ws = (double*)ws_get(h, need, st);
  if (!ws) { h->err = "jk workspace allocation failed"; return MG_ERR_MEMORY; }
  double* dw = ws;
  double* jrs = dw + (size_t)nrs * k;
  double* V = jrs + (size_t)nrs * k;
  double* D = V + block;
  double* Lsq = D + (size_t)n * n;
  double* X = Lsq + (size_t)block * n * n;
  const double one = 1.0, zero = 0.0;
  for (int d = 0; d < k; ++d) {
    // D = C C^T  (C column-major n x r); D symmetric so layout-agnostic
    cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, rs_[d], &one, Cs[d], n, Cs[d], n, &zero, D, n);
    k_pack_density<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, D, n, dw + (size_t)d * nrs);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaMemsetAsync(Ks[d], 0, sizeof(double) * n * n, st);
    cudaMemsetAsync(Js[d], 0, sizeof(double) * n * n, st);  // AO pairs without rows stay zero
  }
  cudaMemsetAsync(jrs, 0, sizeof(double) * nrs * k, st);
  // AO pairs without rows (screened-out shell pairs) stay zero in every square
  cudaMemsetAsync(Lsq, 0, sizeof(double) * block * n * n, st);
  for (int J0 = 0; J0 < M; J0 += block) {
    const int nb = std::min(block, M - J0);
    // vectors J0.. may straddle storage blocks: gather into a contiguous view
    const double* Lb = cho_vec_ptr(c, J0, nb, st, h);
    if (!Lb) { h->err = "vector block gather failed"; return MG_ERR_MEMORY; }
    k_unpack_block<<<nb256(nrs * nb), 256, 0, st>>>(d_ra, d_rb, nrs, Lb, nb, n, Lsq);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    for (int d = 0; d < k; ++d) {
      // Coulomb: V = L_b^T dw ; jrs += L_b V
      cublasDgemv(cb, CUBLAS_OP_T, (int)nrs, nb, &one, Lb, (int)nrs, dw + (size_t)d * nrs, 1, &zero, V, 1);
      cublasDgemv(cb, CUBLAS_OP_N, (int)nrs, nb, &one, Lb, (int)nrs, V, 1, &one, jrs + (size_t)d * nrs, 1);
      // Exchange: X_J = Lsq_J C (n x r each), K += X X^T
      cublasDgemmStridedBatched(cb, CUBLAS_OP_N, CUBLAS_OP_N, n, rs_[d], n, &one, Lsq, n, (long long)n * n, Cs[d], n,
                                0, &zero, X, n, (long long)n * rs_[d], nb);
      cublasDsyrk(cb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, n, nb * rs_[d], &one, X, n, &one, Ks[d], n);
    }
  }
  for (int d = 0; d < k; ++d) {
    k_unpack_sym<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, jrs + (size_t)d * nrs, n, Js[d]);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_symmetrize_lower<<<nb256((int64_t)n * n), 256, 0, st>>>(Ks[d], n);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : MG_ERR_CUDA;
}

// ------------------------------------------------------------ mixed path
// Slicing of one value x of a row with exponent e (y = x 2^-e in (-1, 1))
// into S 8-bit pieces (oz_gemm.cuh): y as the S-byte two's-complement
// fixed-point integer Y = floor(y 2^(8S-1)), its lowest byte rounded to
// nearest where that does not carry out of the byte; slice p is byte S-1-p
// of Y (S_0 the signed top byte, U_p unsigned), so every slice but the last
// is the floor digit and the dropped tail is below one unit of the last.
struct OzScale {
  double lo, hi;  // 2^(8S-1-e) as two factors, each a normal double
};

template <int S>
__device__ __forceinline__ OzScale oz_scale(int e) {
  const int k = 8 * S - 1 - e, k1 = k >> 1;  // e in [-1073, 1024]: both halves in range
  return {oz_pow2(k1), oz_pow2(k - k1)};
}

template <int S>
__device__ __forceinline__ long long oz_fixed(double x, OzScale sc) {
  const double z = (x * sc.lo) * sc.hi;  // exact power-of-two scaling, |z| < 2^(8S-1)
  long long y;
  double frac;
  if (S <= 6) {
    // |z| < 2^47: adding 1.5 2^52 rounded down leaves floor(z) in the low
    // mantissa bits (the unit in the last place is 1 there), on the adder
    constexpr double kM = 6755399441055744.0;  // 1.5 2^52
    const double t = __dadd_rd(z, kM);
    y = (__double_as_longlong(t) & ((1ll << 52) - 1)) - (1ll << 51);
    frac = z - (t - kM);  // both differences exact
  } else {
    y = __double2ll_rd(z);
    frac = z - (double)y;  // exact: z is integral beyond 2^52
  }
  if (frac >= 0.5 && (y & 255) != 255) ++y;
  return y;
}

// slice p of 8 consecutive values: out[p] holds their bytes S-1-p
template <int S>
__device__ __forceinline__ void oz_pack8(const long long (&y)[8], uint2 (&out)[S]) {
#pragma unroll
  for (int p = 0; p < S; ++p) {
    const int sh = 8 * (S - 1 - p);
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      lo |= (uint32_t)((y[u] >> sh) & 255) << (8 * u);
      hi |= (uint32_t)((y[4 + u] >> sh) & 255) << (8 * u);
    }
    out[p] = make_uint2(lo, hi);
  }
}

// f(std::integral_constant<int, s>) for s = 2..kOzMaxSlices
template <typename F>
static bool oz_with_slices(int s, F&& f) {
  switch (s) {
    case 2: f(std::integral_constant<int, 2>{}); return true;
    case 3: f(std::integral_constant<int, 3>{}); return true;
    case 4: f(std::integral_constant<int, 4>{}); return true;
    case 5: f(std::integral_constant<int, 5>{}); return true;
    case 6: f(std::integral_constant<int, 6>{}); return true;
    case 7: f(std::integral_constant<int, 7>{}); return true;
    case 8: f(std::integral_constant<int, 8>{}); return true;
  }
  return false;
}
static_assert(kOzMaxSlices == 8, "oz_with_slices covers 2..8 slices");

__device__ __forceinline__ int oz_exponent(double m) {
  int e = 0;
  if (m > 0.0) frexp(m, &e);
  return e;
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Row exponents of the square Cholesky vectors, computed once per
// decomposition: one warp per row (J, a) gathers L_J[a, 0..n) from the
// rs-packed FP64 vectors through the inverse rs table and stores the frexp
// exponent of its largest |element| (0 for a zero row and for a >= n).
__global__ void k_oz_lexp(const int* __restrict__ inv, int n, int64_t nrs, const double* __restrict__ L, int nb,
                          int ld, short* __restrict__ eL) {
  const int lane = threadIdx.x & 31;
  const int64_t row = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= (int64_t)nb * ld) return;
  const int J = (int)(row / ld), a = (int)(row - (int64_t)J * ld);
  const double* LJ = L + nrs * J;
  double m = 0.0;
  if (a < n)
    for (int b = lane; b < n; b += 32) {
      const int t = inv[(size_t)a * n + b];  // -1: not stored (zero)
      if (t >= 0) m = fmax(m, fabs(LJ[t]));
    }
  m = warp_max(m);
  if (lane == 0) eL[row] = (short)max(-32000, oz_exponent(m));
}

// L slicing in blocks: one CTA per (256 AOs b, 16 AOs a0..a0+15, vector J).
// Thread t owns b = c0 + t and loads L_J[a0..a0+16, b] straight from the
// rs-packed vector, the rs index worked out from the shells of a and b (pair
// (I, J') with I > J' stores a-fastest, I < J' the mirror, I = J' a
// triangle, plf_cho_diag.F90:60-72), all 16 loads in flight at once.  L_J is
// symmetric, so these are also row b, columns a0..a0+15: 16 consecutive K
// bytes of row b of every slice, cut with row b's cached exponent, packed in
// registers and written with one 16-byte store per slice (the blocked layout
// of oz_blk_off).  The grid covers all ld columns a, so the K padding
// a >= n is written as zeros (as are the rows b >= n).
// sh_off[ns + 1]: first AO of every shell (sh_off[ns] = n); ao_sh[n]: the
// shell of every AO.
constexpr int kOzChunk = 256;   // AOs b per CTA (= threads)
constexpr int kOzRows = 16;     // AOs a per CTA

template <int S>
__global__ void __launch_bounds__(kOzChunk) k_oz_slice_l_blocks(const int64_t* __restrict__ sp_first,
                                                                const int* __restrict__ sh_off,
                                                                const int* __restrict__ ao_sh, int n, int64_t nrs,
                                                                const double* __restrict__ L, int ld, int64_t slice,
                                                                const short* __restrict__ eL,
                                                                const double* __restrict__ D,
                                                                uint8_t* __restrict__ LS, int* __restrict__ eA,
                                                                double* __restrict__ V) {
  __shared__ int rI[kOzRows], rla[kOzRows], rnA[kOzRows];  // shell of a, index in it, its width
  __shared__ double red[kOzChunk / 32];
  const int c0 = blockIdx.x * kOzChunk;
  const int a0 = blockIdx.y * kOzRows;
  const int J = blockIdx.z;
  const int nr = max(0, min(kOzRows, n - a0));
  if ((int)threadIdx.x < nr) {
    const int r = threadIdx.x, a = a0 + r;
    const int I = ao_sh[a], aa = sh_off[I];
    rI[r] = I;
    rla[r] = a - aa;
    rnA[r] = sh_off[I + 1] - aa;
  }
  __syncthreads();
  const double* LJ = L + nrs * J;
  const int b = c0 + threadIdx.x;
  double x[kOzRows];
  if (b < n) {
    // rs indices fit in 32 bits (nrs < 2^31 for n < 65536)
    const int Jp = ao_sh[b], bb = sh_off[Jp], nB = sh_off[Jp + 1] - bb, lb = b - bb, trib = Jp * (Jp + 1) / 2;
#pragma unroll
    for (int r = 0; r < kOzRows; ++r) {
      x[r] = 0.0;
      if (r < nr) {
        // one load for every lane (the lanes of a warp may lie on either side of I)
        const int I = rI[r], la = rla[r];
        const int pair = Jp < I ? I * (I + 1) / 2 + Jp : trib + I;
        const int hi = la >= lb ? la : lb, lo = la >= lb ? lb : la;
        const int off = Jp < I ? la + rnA[r] * lb : (Jp > I ? lb + nB * la : hi * (hi + 1) / 2 + lo);
        const int base = (int)__ldg(sp_first + pair);  // -1: a shell pair without rows (screened out)
        x[r] = base >= 0 ? __ldg(LJ + base + off) : 0.0;
      }
    }
  } else {
#pragma unroll
    for (int r = 0; r < kOzRows; ++r) x[r] = 0.0;
  }
  // cut, and the Coulomb contraction V_J = sum_ab L_J[a, b] D[a, b] over the
  // lower triangle (off-diagonal elements twice: L_J and D are symmetric)
  double v = 0.0;
  if (b < ld) {
    const int64_t row = (int64_t)J * ld + b;
    const int e = eL[row];
    if (blockIdx.y == 0) eA[row] = e;
    const OzScale sc = oz_scale<S>(e);
    uint32_t w[S][kOzRows / 4];  // slice p, rows 4 g .. 4 g + 3 (one byte each)
#pragma unroll
    for (int g = 0; g < kOzRows / 4; ++g) {
      uint32_t lo[4], hi[4];  // the two words of Y for the four rows
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int r = 4 * g + k, a = a0 + r;
        if (r < nr && b <= a) v = fma(b < a ? 2.0 * x[r] : x[r], __ldg(D + (size_t)a * n + b), v);
        const long long y = oz_fixed<S>(x[r], sc);
        lo[k] = (uint32_t)y;
        hi[k] = (uint32_t)((unsigned long long)y >> 32);
      }
      // byte S-1-p of the four Y into one word: two byte permutes take the
      // byte from rows (0, 1) and (2, 3), a third joins the halves
#pragma unroll
      for (int p = 0; p < S; ++p) {
        const int bi = S - 1 - p, kb = bi & 3;
        const uint32_t sel = (uint32_t)(((4 + kb) << 4) | kb);
        const uint32_t s01 = bi >= 4 ? __byte_perm(hi[0], hi[1], sel) : __byte_perm(lo[0], lo[1], sel);
        const uint32_t s23 = bi >= 4 ? __byte_perm(hi[2], hi[3], sel) : __byte_perm(lo[2], lo[3], sel);
        w[p][g] = __byte_perm(s01, s23, 0x5410);
      }
    }
    uint8_t* dst = LS + oz_blk_off(row, a0, ld, 128);  // a0 % 16 == 0: 16 bytes of one 32-byte chunk
#pragma unroll
    for (int p = 0; p < S; ++p)
      *reinterpret_cast<uint4*>(dst + p * slice) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
  }
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w8 = 0; w8 < kOzChunk / 32; ++w8) t += red[w8];
    atomicAdd(&V[J], t);
  }
}

// C (n x r, column-major FP64) -> slices CS[q] of the npad x ld matrix C^T,
// blocked in tiles of Nt rows (rows k >= r and columns b >= n zero), column
// scale factors fC[k] = 2^e_k.  One warp per column k.
template <int S>
__global__ void k_oz_slice_c(const double* __restrict__ C, int n, int r, int npad, int ld, int Nt,
                             uint8_t* __restrict__ CS, double* __restrict__ fC) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (k >= npad) return;
  const double* ck = C + (size_t)n * k;
  double m = 0.0;
  if (k < r)
    for (int b = lane; b < n; b += 32) m = fmax(m, fabs(ck[b]));
  const int e = oz_exponent(warp_max(m));
  if (lane == 0) fC[k] = oz_pow2e(e);
  const OzScale sc = oz_scale<S>(e);
  const size_t slice = (size_t)npad * ld;
  for (int b0 = 8 * lane; b0 < ld; b0 += 256) {
    uint8_t* out = CS + oz_blk_off(k, b0, ld, Nt);
    long long y[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int b = b0 + u;
      y[u] = oz_fixed<S>((k < r && b < n) ? ck[b] : 0.0, sc);
    }
    uint2 w[S];
    oz_pack8<S>(y, w);
#pragma unroll
    for (int q = 0; q < S; ++q) *reinterpret_cast<uint2*>(out + q * slice) = w[q];
  }
}

// X (FP64, column-major: element (a, c) at X[c * xld + a], columns
// [0, kx)) -> slices of XS (ld rows x xs_row columns, blocked in 128-row
// tiles) at columns col0 + c (zero beyond kx and for rows a >= n), with the
// row exponent of xmax[a] (the largest |X| of the row, recorded by the
// half-transform), stored in eX[a].  One thread per (row a, 32-column
// chunk): consecutive threads take consecutive rows, so that a warp reads
// 256 consecutive bytes per column and writes 1 KB per slice.
template <int S>
__global__ void k_oz_slice_x(const double* __restrict__ X, int64_t xld, int n, int kx, int ld, int kblk,
                             int64_t xs_row, int64_t col0, const unsigned long long* __restrict__ xmax,
                             uint8_t* __restrict__ XS, int* __restrict__ eX) {
  const int nch = kblk / 32;
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)ld * nch) return;
  const int ri = (int)(o & 127);
  const int64_t r2 = o >> 7;
  const int ch = (int)(r2 % nch), tile = (int)(r2 / nch);
  const int a = tile * 128 + ri;
  const int e = a < n ? oz_exponent(__longlong_as_double((long long)xmax[a])) : 0;
  if (ch == 0) eX[a] = e;
  const OzScale sc = oz_scale<S>(e);
  uint2 w[4][S];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    long long y[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int c = 32 * ch + 8 * g + u;
      y[u] = oz_fixed<S>((a < n && c < kx) ? X[(size_t)c * xld + a] : 0.0, sc);
    }
    oz_pack8<S>(y, w[g]);
  }
  const size_t slice = (size_t)ld * xs_row;
  uint8_t* out = XS + oz_blk_off(a, col0 + 32 * ch, xs_row, 128);
#pragma unroll
  for (int q = 0; q < S; ++q) {
    uint4* d = reinterpret_cast<uint4*>(out + q * slice);
    d[0] = make_uint4(w[0][q].x, w[0][q].y, w[1][q].x, w[1][q].y);
    d[1] = make_uint4(w[2][q].x, w[2][q].y, w[3][q].x, w[3][q].y);
  }
}

// xmax[a] = bits of max_c |X[c * xld + a]| (for the self-test, where X is given)
__global__ void k_row_absmax(const double* __restrict__ X, int64_t xld, int n, int kx,
                             unsigned long long* __restrict__ xmax) {
  const int a = blockIdx.x;
  double m = 0.0;
  if (a < n)
    for (int c = threadIdx.x; c < kx; c += blockDim.x) m = fmax(m, fabs(X[(size_t)c * xld + a]));
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(xmax + a, (unsigned long long)__double_as_longlong(m));
}

// jrs[t] += sum_J L[t, J] V[J] over one block of nb FP64 vectors
__global__ void k_jacc64(const double* __restrict__ L, int64_t nrs, int nb, const double* __restrict__ V,
                         double* __restrict__ jrs) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  double s = 0.0;
  for (int J = 0; J < nb; ++J) s = fma(L[t + nrs * J], V[J], s);
  jrs[t] += s;
}

// Coulomb contractions of a batch's further densities (the first one's are
// formed by the L unpacking): V[d nb + J] = sum_t L[t, J] dw_d[t] for
// d = 1 .. kd, dw_d = dws + (d - 1) nrs the packed weighted density
// (k_pack_density).  One CTA per vector J, each vector element read once.
constexpr int kJkMaxDens = 8;

__global__ void __launch_bounds__(256) k_vmulti(const double* __restrict__ L, int64_t nrs, int nb, int kd,
                                                const double* __restrict__ dws, double* __restrict__ V) {
  __shared__ double red[kJkMaxDens][8];
  const int J = blockIdx.x;
  const double* LJ = L + nrs * J;
  double acc[kJkMaxDens - 1];
#pragma unroll
  for (int d = 0; d < kJkMaxDens - 1; ++d) acc[d] = 0.0;
  for (int64_t t = threadIdx.x; t < nrs; t += blockDim.x) {
    const double x = __ldg(LJ + t);
#pragma unroll
    for (int d = 0; d < kJkMaxDens - 1; ++d)
      if (d < kd) acc[d] = fma(x, __ldg(dws + (size_t)d * nrs + t), acc[d]);
  }
#pragma unroll
  for (int d = 0; d < kJkMaxDens - 1; ++d) {
    const double v = warp_sum(acc[d]);
    if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < kd) {
    double v = 0.0;
    for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
    V[(size_t)(threadIdx.x + 1) * nb + J] = v;
  }
}

// jrs_d[t] += sum_J L[t, J] V[d nb + J] for the k densities of a batch,
// each vector element read once (k_jacc64 for one density)
__global__ void k_jacc_multi(const double* __restrict__ L, int64_t nrs, int nv, int nb, int k,
                             const double* __restrict__ V, double* __restrict__ jrs) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  double acc[kJkMaxDens];
#pragma unroll
  for (int d = 0; d < kJkMaxDens; ++d) acc[d] = 0.0;
  for (int J = 0; J < nv; ++J) {
    const double x = L[t + nrs * J];
#pragma unroll
    for (int d = 0; d < kJkMaxDens; ++d)
      if (d < k) acc[d] = fma(x, V[(size_t)d * nb + J], acc[d]);
  }
#pragma unroll
  for (int d = 0; d < kJkMaxDens; ++d)
    if (d < k) jrs[(size_t)d * nrs + t] += acc[d];
}

// inv[a*n + b] = inv[b*n + a] = t for every rs pair t (the caller fills inv
// with -1 first: AO pairs of shell pairs without rows keep it)
__global__ void k_rs_inverse(const int* __restrict__ rs_a, const int* __restrict__ rs_b, int64_t nrs, int n,
                             int* __restrict__ inv) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  const int a = rs_a[t], b = rs_b[t];
  inv[(size_t)a * n + b] = (int)t;
  inv[(size_t)b * n + a] = (int)t;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on the driver library).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// 8-bit tensor map over s blocked slices of a rows x kx matrix (layout of
// oz_blk_off: tiles of br rows x 32 bytes, each contiguous), as a 5D tensor
// (32 bytes, br rows, kx / 32 K steps, rows / br row tiles, s slices); a box
// is one tile, placed in shared memory with the 32-byte swizzle.
static bool make_slice_map(CUtensorMap* m, const uint8_t* base, int64_t kx, int64_t rows, int s, int br) {
  auto enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15) || kx % 32 || br < 8 || br > 256 || br % 8 || rows % br) return false;
  cuuint64_t gdim[5] = {32u, (cuuint64_t)br, (cuuint64_t)(kx / 32), (cuuint64_t)(rows / br), (cuuint64_t)s};
  cuuint64_t gstr[4] = {32u, (cuuint64_t)br * 32, (cuuint64_t)(kx * br), (cuuint64_t)(kx * rows)};
  cuuint32_t box[5] = {32u, (cuuint32_t)br, 1u, 1u, 1u}, es[5] = {1, 1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, (void*)base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static inline int rup(int x, int m) { return (x + m - 1) / m * m; }

// Column tiles of the half-transform: the widest multiple of 16 (<= 256)
// whose s accumulators fit the 512 TMEM columns (one pass per tile), then
// spread evenly over the r columns.
static void oz_col_tiles(int r, int s, int& nnt, int& Nt) {
  const int nmax = std::min(256, (512 / s) / 16 * 16);
  nnt = (r + nmax - 1) / nmax;
  Nt = rup((r + nnt - 1) / nnt, 16);
}

// Pass plan of one kind of output tile: accumulators of acc_stride TMEM
// columns, at most 512 columns; shared-memory ring of the slices 0..s-1.
static void oz_plan(OzArgs& a, int s, int Nt) {
  a.s = s;
  a.Nt = Nt;
  a.acc_stride = Nt;
  a.nd = std::min(s, 512 / a.acc_stride);
  a.b_bytes = rup(32 * Nt, 1024);
  a.stage_bytes = s * (kOzABytes + a.b_bytes);
  a.stages = std::min(kOzMaxStages, (kOzSmemLimit - 1024) / a.stage_bytes);
}

// Row exponents of the handle's Cholesky vectors for squares of ld rows
// (computed once per decomposition, cached in the Cholesky state).
static const short* oz_row_exponents(Handle* h, const int* inv, int ld, cudaStream_t st) {
  ChoState* c = h->cho;
  if (const short* e = cho_lexp(c, ld)) return e;
  const int M = cho_nvec(c), n = h->nbf, vb = cho_vec_block();
  const int64_t nrs = cho_nrs(c);
  short* e = nullptr;
  if (dev_malloc(&e, sizeof(short) * (size_t)M * ld) != cudaSuccess) return nullptr;
  for (int J0 = 0; J0 < M; J0 += vb) {
    const int nv = std::min(vb, M - J0);
    const double* L = cho_vec_ptr(c, J0, nv, st, h);
    const int64_t rows = (int64_t)nv * ld;
    k_oz_lexp<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(inv, n, nrs, L, nv, ld, e + (size_t)J0 * ld);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) {
      cudaFree(e);
      return nullptr;
    }
  }
  cho_set_lexp(c, e, ld);
  return e;
}

// Per-density state of a mixed J/K batch.
struct OzDens {
  const double* C;
  int r;
  double* J;
  double* K;
  int nnt, Nt, npad, kx, kblk, nsub, ksub;
  int64_t xs_row;
  double* jrs;           // Coulomb in rs layout
  double* dw;            // packed weighted density (densities after the first)
  uint8_t* CS;           // slices of C
  double* fC;            // column scale factors of C
  uint8_t* XS;           // slices of X for one group of blocks
  int* eX;               // their row exponents
  CUtensorMap map_c, map_x;
  OzArgs ax, ak;
};

int jk_mixed(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block, int s,
             int sk) {
  return jk_mixed_batch(h, 1, &d_C, &r, &d_J, &d_K, st, block, s, sk);
}

// J/K of k densities over one pass of the vectors: every block of vectors is
// unpacked and sliced once (with the first density's Coulomb contraction
// fused), the further densities' contractions take one more read of the
// block (k_vmulti), J accumulates for all densities in one read
// (k_jacc_multi), and each density runs its half-transform, X slicing and
// exchange product on the shared slices.
int jk_mixed_batch(Handle* h, int k, const double* const* Cs, const int* rs_, double* const* Js, double* const* Ks,
                   cudaStream_t st, int block, int s, int sk) {
  ChoState* c = h->cho;
  const int64_t nrs = cho_nrs(c);
  const int M = cho_nvec(c);
  const int n = h->nbf;
  if (s < 2 || s > kOzMaxSlices || sk < 2 || sk > kOzMaxSlices) {
    h->err = "mixed J/K: slices must be 2..8";
    return MG_ERR_ARG;
  }
  if (k < 1 || k > kJkMaxDens) {
    h->err = "mixed J/K: 1..8 densities per batch";
    return MG_ERR_ARG;
  }
  if (const cudaError_t e = cudaGetLastError(); e != cudaSuccess) {
    h->err = std::string("mixed J/K: error pending from earlier work: ") + cudaGetErrorString(e);
    return MG_ERR_CUDA;
  }
  const int ld = rup(n, 128);
  // vectors per block: one block's K extent of the exchange product, nb r
  const int nb = std::min(block, M);
  const int nblocks = (M + nb - 1) / nb;
  const int G = std::min(16, nblocks);  // blocks per exchange-product group
  const int ntile = (ld / 128) * (ld / 128 + 1) / 2;
  std::vector<OzDens> dd(k);
  int kxmax = 0;
  for (int d = 0; d < k; ++d) {
    OzDens& q = dd[d];
    q.C = Cs[d];
    q.r = rs_[d];
    q.J = Js[d];
    q.K = Ks[d];
    if (!q.C || !q.J || !q.K || q.r < 1) {
      h->err = "mixed J/K: a density of the batch has no factor or outputs";
      return MG_ERR_ARG;
    }
    oz_col_tiles(q.r, s, q.nnt, q.Nt);
    q.npad = q.nnt * q.Nt;
    q.kx = nb * q.r;
    q.kblk = rup(q.kx, 32);
    q.nsub = (q.kblk + kOzKChunk - 1) / kOzKChunk;
    q.ksub = rup((q.kblk + q.nsub - 1) / q.nsub, 32);
    q.xs_row = (int64_t)G * q.kblk;
    kxmax = std::max(kxmax, q.kx);
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  cublasHandle_t cb = cho_cublas(c);
  cublasSetStream(cb, st);
  const int* d_ra = cho_rs_a_dev(c);
  const int* d_rb = cho_rs_b_dev(c);
  const size_t nn = (size_t)n * n;
  const int ns = (int)h->sh.size();
  // one term per take() below (each rounded up to 256 bytes)
  size_t need = 8 * ((size_t)nb * k + 2 * nn) + 4 * nn + (size_t)s * nb * ld * ld + 4 * (size_t)nb * ld +
                8 * (size_t)ld * kxmax + 8 * (size_t)ld + 8 * (size_t)nsm * 128 * 128 + sizeof(int) +
                4 * (size_t)(ns + 1 + n) + 11 * 256;
  for (const OzDens& q : dd)
    need += 16 * (size_t)nrs + (size_t)s * q.npad * ld + 8 * (size_t)q.npad + (size_t)sk * ld * q.xs_row +
            4 * (size_t)G * ld + 6 * 256;
  char* ws = (char*)ws_get(h, need, st);
  if (!ws) { h->err = "jk workspace allocation failed"; return MG_ERR_MEMORY; }
  char* const ws_end = ws + need;
  auto take = [&](size_t bytes) { char* p = ws; ws += (bytes + 255) & ~(size_t)255; return (void*)p; };
  double* V = (double*)take(8 * (size_t)nb * k);  // V[d nb + J]
  double* D = (double*)take(8 * nn);               // D of the first density (its contraction is fused)
  double* Dt = (double*)take(8 * nn);              // D of a further density, while it is packed
  int* inv = (int*)take(4 * nn);
  uint8_t* LS = (uint8_t*)take((size_t)s * nb * ld * ld);
  int* eA = (int*)take(4 * (size_t)nb * ld);
  double* Xf = (double*)take(8 * (size_t)ld * kxmax);  // column-major, ld rows
  unsigned long long* xmax = (unsigned long long*)take(8 * (size_t)ld);
  double* P = (double*)take(8 * (size_t)nsm * 128 * 128);
  int* d_err = (int*)take(sizeof(int));
  int* sh_off = (int*)take(4 * (size_t)(ns + 1 + n));
  int* ao_sh = sh_off + ns + 1;
  double* jrs_all = (double*)take(8 * (size_t)nrs * k);  // jrs of density d at d nrs
  double* dws = (double*)take(8 * (size_t)nrs * std::max(1, k - 1));
  for (int d = 0; d < k; ++d) {
    OzDens& q = dd[d];
    q.jrs = jrs_all + (size_t)d * nrs;
    q.dw = d > 0 ? dws + (size_t)(d - 1) * nrs : nullptr;
    q.CS = (uint8_t*)take((size_t)s * q.npad * ld);
    q.fC = (double*)take(8 * (size_t)q.npad);
    q.XS = (uint8_t*)take((size_t)sk * ld * q.xs_row);
    q.eX = (int*)take(4 * (size_t)G * ld);
  }
  if (ws > ws_end) { h->err = "mixed J/K: workspace layout exceeds its size"; return MG_ERR_CUDA; }
  // every launch is checked at once, so that an error names its kernel
  auto launched = [&](const char* what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return true;
    h->err = std::string("mixed J/K: ") + what + ": " + cudaGetErrorString(e);
    return false;
  };
  std::vector<int> hoff(ns + 1 + n);
  for (int i = 0; i < ns; ++i) {
    hoff[i] = h->sh[i].off;
    for (int a = h->sh[i].off; a < h->sh[i].off + h->sh[i].nc * h->sh[i].ncomp; ++a) hoff[ns + 1 + a] = i;
  }
  hoff[ns] = n;
  if (const cudaError_t e = cudaMemcpyAsync(sh_off, hoff.data(), 4 * (size_t)(ns + 1 + n), cudaMemcpyHostToDevice, st);
      e != cudaSuccess) {
    h->err = std::string("mixed J/K: shell table upload: ") + cudaGetErrorString(e);
    return MG_ERR_CUDA;
  }
  CUtensorMap map_l;
  if (!make_slice_map(&map_l, LS, ld, (int64_t)nb * ld, s, 128)) {
    h->err = "tensor maps for the exchange GEMMs could not be encoded";
    return MG_ERR_CUDA;
  }
  for (OzDens& q : dd)
    if (!make_slice_map(&q.map_c, q.CS, ld, q.npad, s, q.Nt) || !make_slice_map(&q.map_x, q.XS, q.xs_row, ld, sk, 128)) {
      h->err = "tensor maps for the exchange GEMMs could not be encoded";
      return MG_ERR_CUDA;
    }
  bool attr = true;
  oz_with_slices(s, [&](auto S) { attr &= smem_attr_once((const void*)oz_gemm_kernel<false, decltype(S)::value>, kOzSmemLimit); });
  oz_with_slices(sk, [&](auto S) { attr &= smem_attr_once((const void*)oz_gemm_kernel<true, decltype(S)::value>, kOzSmemLimit); });
  if (!attr) {
    h->err = "exchange GEMMs: shared-memory limit could not be raised";
    return MG_ERR_CUDA;
  }
  for (OzDens& q : dd) {
    OzArgs& ax = q.ax;
    OzArgs& ak = q.ak;
    ax = OzArgs{};
    ak = OzArgs{};
    oz_plan(ax, s, q.Nt);
    oz_plan(ak, sk, 128);
    if (ax.stages < 2 || ak.stages < 2) { h->err = "mixed J/K: slice tiles do not fit in shared memory"; return MG_ERR_ARG; }
    ax.err = ak.err = d_err;
    ax.nrt = ld / 128; ax.nnt = q.nnt; ax.ld = ld; ax.n = n; ax.r = q.r; ax.eA = eA; ax.fB = q.fC; ax.X = Xf;
    ax.xld = ld; ax.xmax = xmax;
    ak.ld = ld; ak.n = n; ak.ntile = ntile; ak.nsub = q.nsub; ak.kblk = q.kblk; ak.ksub = q.ksub; ak.eX = q.eX;
    ak.P = P; ak.K = q.K;
  }
  const double one = 1.0, zero = 0.0;
  if (cudaMemsetAsync(d_err, 0, sizeof(int), st) != cudaSuccess ||
      cudaMemsetAsync(jrs_all, 0, 8 * nrs * k, st) != cudaSuccess) {
    h->err = std::string("mixed J/K: clearing buffers: ") + cudaGetErrorString(cudaGetLastError());
    return MG_ERR_CUDA;
  }
  for (int d = 0; d < k; ++d) {
    OzDens& q = dd[d];
    if (cudaMemsetAsync(q.K, 0, 8 * nn, st) != cudaSuccess) {
      h->err = std::string("mixed J/K: clearing K: ") + cudaGetErrorString(cudaGetLastError());
      return MG_ERR_CUDA;
    }
    // D = C C^T: the first density's is read by the L unpacking, the others are packed over rs
    double* Dd = d == 0 ? D : Dt;
    if (const cublasStatus_t bs = cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, q.r, &one, q.C, n, q.C, n, &zero, Dd, n);
        bs != CUBLAS_STATUS_SUCCESS) {
      h->err = "mixed J/K: density product (cublasDgemm) failed, status " + std::to_string((int)bs);
      return MG_ERR_CUDA;
    }
    if (d > 0) {
      k_pack_density<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, Dt, n, q.dw);
      if (!launched("k_pack_density")) return MG_ERR_CUDA;
    }
  }
  if (const cudaError_t e = cudaGetLastError(); e != cudaSuccess) {
    h->err = std::string("mixed J/K: after the density products: ") + cudaGetErrorString(e);
    return MG_ERR_CUDA;
  }
  cudaMemsetAsync(inv, 0xFF, 4 * nn, st);
  k_rs_inverse<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, n, inv);
  if (!launched("k_rs_inverse")) return MG_ERR_CUDA;
  const short* eL = oz_row_exponents(h, inv, ld, st);
  if (!eL) { h->err = "mixed J/K: row exponents could not be stored"; return MG_ERR_MEMORY; }
  for (OzDens& q : dd) {
    oz_with_slices(s, [&](auto S) {
      k_oz_slice_c<decltype(S)::value><<<(q.npad + 7) / 8, 256, 0, st>>>(q.C, n, q.r, q.npad, ld, q.Nt, q.CS, q.fC);
    });
    if (!launched("k_oz_slice_c")) return MG_ERR_CUDA;
  }
  for (int g0 = 0; g0 < nblocks; g0 += G) {
    const int gn = std::min(G, nblocks - g0);
    for (int bi = 0; bi < gn; ++bi) {
      const int J0 = (g0 + bi) * nb;
      const int nv = std::min(nb, M - J0);
      const double* Lb = cho_vec_ptr(c, J0, nv, st, h);
      if (!Lb) { h->err = "vector block straddles storage blocks"; return MG_ERR_ARG; }
      cudaMemsetAsync(V, 0, 8 * (size_t)nb, st);
      oz_with_slices(s, [&](auto S) {
        k_oz_slice_l_blocks<decltype(S)::value>
            <<<dim3((ld + kOzChunk - 1) / kOzChunk, ld / kOzRows, nv), kOzChunk, 0, st>>>(
                cho_sp_first_dev(c), sh_off, ao_sh, n, nrs, Lb, ld, (int64_t)nb * ld * ld, eL + (size_t)J0 * ld, D,
                LS, eA, V);
      });
      if (!launched("k_oz_slice_l_blocks")) return MG_ERR_CUDA;
      if (k == 1) {
        k_jacc64<<<nb256(nrs), 256, 0, st>>>(Lb, nrs, nv, V, dd[0].jrs);
        if (!launched("k_jacc64")) return MG_ERR_CUDA;
      } else {
        k_vmulti<<<nv, 256, 0, st>>>(Lb, nrs, nb, k - 1, dws, V);
        if (!launched("k_vmulti")) return MG_ERR_CUDA;
        k_jacc_multi<<<nb256(nrs), 256, 0, st>>>(Lb, nrs, nv, nb, k, V, jrs_all);
        if (!launched("k_jacc_multi")) return MG_ERR_CUDA;
      }
      for (OzDens& q : dd) {
        // a short last block: clear the columns of the missing vectors
        if (nv < nb) cudaMemsetAsync(Xf, 0, 8 * (size_t)ld * q.kx, st);
        cudaMemsetAsync(xmax, 0, 8 * (size_t)ld, st);
        // X_J = L_J C for the block (the slice map covers nb vectors; nv <= nb of them are used)
        OzArgs& ax = q.ax;
        ax.nJ = nv;
        ax.nitems = ax.nrt * nv * q.nnt;
        const int gx = std::min(ax.nitems, nsm);
        oz_with_slices(s, [&](auto S) {
          oz_gemm_kernel<false, decltype(S)::value><<<gx, kOzThreads, ax.stages * ax.stage_bytes + 1024, st>>>(
              map_l, q.map_c, ax);
        });
        if (!launched("oz_gemm_kernel<false>")) return MG_ERR_CUDA;
        oz_with_slices(sk, [&](auto S) {
          k_oz_slice_x<decltype(S)::value><<<nb256((int64_t)ld * (q.kblk / 32)), 256, 0, st>>>(
              Xf, ld, n, q.kx, ld, q.kblk, q.xs_row, (int64_t)bi * q.kblk, xmax, q.XS, q.eX + (size_t)bi * ld);
        });
        if (!launched("k_oz_slice_x")) return MG_ERR_CUDA;
      }
    }
    // K += X X^T over the group (lower tiles), per density
    for (OzDens& q : dd) {
      OzArgs& ak = q.ak;
      ak.nblk = gn;
      ak.nitems = ntile * gn * q.nsub;
      const int gk = std::min(ak.nitems, nsm);
      oz_with_slices(sk, [&](auto S) {
        oz_gemm_kernel<true, decltype(S)::value><<<gk, kOzThreads, ak.stages * ak.stage_bytes + 1024, st>>>(
            q.map_x, q.map_x, ak);
      });
      if (!launched("oz_gemm_kernel<true>")) return MG_ERR_CUDA;
    }
  }
  for (OzDens& q : dd) {
    k_symmetrize_lower<<<nb256((int64_t)nn), 256, 0, st>>>(q.K, n);
    if (!launched("k_symmetrize_lower")) return MG_ERR_CUDA;
    cudaMemsetAsync(q.J, 0, 8 * nn, st);  // AO pairs without rows
    k_unpack_sym<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, q.jrs, n, q.J);
    if (!launched("k_unpack_sym")) return MG_ERR_CUDA;
  }
  if (const cudaError_t e = cudaGetLastError(); e != cudaSuccess) {
    h->err = std::string("mixed J/K: ") + cudaGetErrorString(e);
    return MG_ERR_CUDA;
  }
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (const cudaError_t e = cudaStreamSynchronize(st); e != cudaSuccess) {
    h->err = std::string("mixed J/K: ") + cudaGetErrorString(e);
    return MG_ERR_CUDA;
  }
  if (herr) {
    h->err = "exchange GEMMs: a pipeline wait ran out (result incomplete)";
    return MG_ERR_CUDA;
  }
  return 0;
}

// The sliced engine on given dense matrices (verification of the kernels
// used by jk_mixed): X = A B (A: ld x ld, B: ld x r, X: ld x r, all
// column-major) and K = X X^T (lower triangle, column-major ld x ld).
int oz_selftest(Handle* h, int ld, int r, int s, const double* d_A, const double* d_B, double* d_X, double* d_K,
                uint8_t* d_slices, int* d_exps, cudaStream_t st) {
  if (ld < 128 || ld % 128 || r < 1 || s < 2 || s > kOzMaxSlices) return MG_ERR_ARG;
  int nnt, Nt;
  oz_col_tiles(r, s, nnt, Nt);
  const int npad = nnt * Nt;
  const int kblk = rup(r, 32);
  const int nsub = (kblk + kOzKChunk - 1) / kOzKChunk;
  const int ksub = rup((kblk + nsub - 1) / nsub, 32);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const size_t need = (size_t)s * ld * ld + 4 * (size_t)ld + (size_t)s * npad * ld + 8 * (size_t)npad +
                      (size_t)s * ld * kblk + 4 * (size_t)ld + 16 * (size_t)ld + 8 * (size_t)nsm * 128 * 128 +
                      18 * 256;
  char* ws = (char*)ws_get(h, need, st);
  if (!ws) return MG_ERR_MEMORY;
  auto take = [&](size_t bytes) { char* p = ws; ws += (bytes + 255) & ~(size_t)255; return (void*)p; };
  uint8_t* LS = (uint8_t*)take((size_t)s * ld * ld);
  int* eA = (int*)take(4 * (size_t)ld);
  uint8_t* CS = (uint8_t*)take((size_t)s * npad * ld);
  double* fC = (double*)take(8 * (size_t)npad);
  uint8_t* XS = (uint8_t*)take((size_t)s * ld * kblk);
  int* eX = (int*)take(4 * (size_t)ld);
  unsigned long long* amax = (unsigned long long*)take(8 * (size_t)ld);
  unsigned long long* xmax = (unsigned long long*)take(8 * (size_t)ld);
  double* P = (double*)take(8 * (size_t)nsm * 128 * 128);
  int* d_err = (int*)take(sizeof(int));
  CUtensorMap map_l, map_c, map_x;
  if (!make_slice_map(&map_l, LS, ld, ld, s, 128) || !make_slice_map(&map_c, CS, ld, npad, s, Nt) ||
      !make_slice_map(&map_x, XS, kblk, ld, s, 128))
    return MG_ERR_CUDA;
  OzArgs ax{}, ak{};
  oz_plan(ax, s, Nt);
  oz_plan(ak, s, 128);
  bool attr = true;
  oz_with_slices(s, [&](auto S) {
    attr &= smem_attr_once((const void*)oz_gemm_kernel<false, decltype(S)::value>, kOzSmemLimit) &&
            smem_attr_once((const void*)oz_gemm_kernel<true, decltype(S)::value>, kOzSmemLimit);
  });
  if (!attr) return MG_ERR_CUDA;
  ax.err = ak.err = d_err;
  ax.nrt = ld / 128; ax.nnt = nnt; ax.ld = ld; ax.n = ld; ax.r = r; ax.eA = eA; ax.fB = fC; ax.X = d_X; ax.xld = ld;
  ax.xmax = xmax; ax.nJ = 1; ax.nitems = ax.nrt * nnt;
  ak.ld = ld; ak.n = ld; ak.ntile = (ld / 128) * (ld / 128 + 1) / 2; ak.nsub = nsub; ak.kblk = kblk; ak.ksub = ksub;
  ak.eX = eX; ak.P = P; ak.K = d_K; ak.nblk = 1; ak.nitems = ak.ntile * nsub;
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  cudaMemsetAsync(d_K, 0, 8 * (size_t)ld * ld, st);
  cudaMemsetAsync(amax, 0, 8 * (size_t)ld, st);
  cudaMemsetAsync(xmax, 0, 8 * (size_t)ld, st);
  k_row_absmax<<<ld, 256, 0, st>>>(d_A, ld, ld, ld, amax);
  oz_with_slices(s, [&](auto S) {
    k_oz_slice_x<decltype(S)::value><<<nb256((int64_t)ld * (ld / 32)), 256, 0, st>>>(d_A, ld, ld, ld, ld, ld, ld, 0,
                                                                                    amax, LS, eA);
  });
  if (d_slices) cudaMemcpyAsync(d_slices, LS, (size_t)s * ld * ld, cudaMemcpyDeviceToDevice, st);
  if (d_exps) cudaMemcpyAsync(d_exps, eA, 4 * (size_t)ld, cudaMemcpyDeviceToDevice, st);
  oz_with_slices(s, [&](auto S) {
    k_oz_slice_c<decltype(S)::value><<<(npad + 7) / 8, 256, 0, st>>>(d_B, ld, r, npad, ld, Nt, CS, fC);
  });
  oz_with_slices(s, [&](auto S) {
    oz_gemm_kernel<false, decltype(S)::value>
        <<<std::min(ax.nitems, nsm), kOzThreads, ax.stages * ax.stage_bytes + 1024, st>>>(map_l, map_c, ax);
  });
  oz_with_slices(s, [&](auto S) {
    k_oz_slice_x<decltype(S)::value><<<nb256((int64_t)ld * (kblk / 32)), 256, 0, st>>>(d_X, ld, ld, r, ld, kblk, kblk,
                                                                                      0, xmax, XS, eX);
  });
  oz_with_slices(s, [&](auto S) {
    oz_gemm_kernel<true, decltype(S)::value>
        <<<std::min(ak.nitems, nsm), kOzThreads, ak.stages * ak.stage_bytes + 1024, st>>>(map_x, map_x, ak);
  });
  g_launches.fetch_add(6, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return MG_ERR_CUDA;
  return herr ? MG_ERR_CUDA : 0;
}

}  // namespace mg
