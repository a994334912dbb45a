// Coulomb / exchange matrices from Cholesky vectors (the CHO_LK_SCF build,
// fock_util/cho_lk_scf.F90:14) on the GPU.
//
//   D = C C^T (C: nbf x r, the Cholesky/orbital factor of the density, as
//   ChoSCF_Drv passes it, scf/choscf_drv.F90:115-116)
//   J_ab = sum_J L_ab,J V_J,  V_J = sum_cd L_cd,J D_cd     (cho_lk_scf.F90:442-449)
//   K_ab = sum_J sum_k X_J[a,k] X_J[b,k],  X_J = L_J C      (cho_lk_scf.F90:507-830)
//
// Mixed path: the FP64 vectors are cut into s 8-bit slices per row
// (oz_gemm.cuh gives the scheme) and both exchange GEMMs run on the tcgen05
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
  ChoState* c = h->cho;
  const int64_t nrs = cho_nrs(c);
  const int M = cho_nvec(c);
  const int n = h->nbf;
  cublasHandle_t cb = cho_cublas(c);
  cublasSetStream(cb, st);
  const int* d_ra = cho_rs_a_dev(c);
  const int* d_rb = cho_rs_b_dev(c);
  // scratch: dw (nrs), V (block), jrs (nrs), D (n*n), Lsq (block*n*n), X (n * block * r)
  const size_t need = sizeof(double) * ((size_t)nrs * 2 + block + (size_t)n * n + (size_t)block * n * n +
                                        (size_t)n * block * r);
  double* ws = (double*)ws_get(h, need, st);
  if (!ws) { h->err = "jk workspace allocation failed"; return MG_ERR_MEMORY; }
  double* dw = ws;
  double* jrs = dw + nrs;
  double* V = jrs + nrs;
  double* D = V + block;
  double* Lsq = D + (size_t)n * n;
  double* X = Lsq + (size_t)block * n * n;
  const double one = 1.0, zero = 0.0;
  // D = C C^T  (C column-major n x r); D symmetric so layout-agnostic
  cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, r, &one, d_C, n, d_C, n, &zero, D, n);
  k_pack_density<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, D, n, dw);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaMemsetAsync(jrs, 0, sizeof(double) * nrs, st);
  cudaMemsetAsync(d_K, 0, sizeof(double) * n * n, st);
  for (int J0 = 0; J0 < M; J0 += block) {
    const int nb = std::min(block, M - J0);
    // vectors J0.. may straddle storage blocks: gather into a contiguous view
    const double* Lb = cho_vec_ptr(c, J0, nb, st, h);
    if (!Lb) { h->err = "vector block gather failed"; return MG_ERR_MEMORY; }
    // Coulomb: V = L_b^T dw ; jrs += L_b V
    cublasDgemv(cb, CUBLAS_OP_T, (int)nrs, nb, &one, Lb, (int)nrs, dw, 1, &zero, V, 1);
    cublasDgemv(cb, CUBLAS_OP_N, (int)nrs, nb, &one, Lb, (int)nrs, V, 1, &one, jrs, 1);
    // Exchange: X_J = Lsq_J C (n x r each), K += X X^T
    k_unpack_block<<<nb256(nrs * nb), 256, 0, st>>>(d_ra, d_rb, nrs, Lb, nb, n, Lsq);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cublasDgemmStridedBatched(cb, CUBLAS_OP_N, CUBLAS_OP_N, n, r, n, &one, Lsq, n, (long long)n * n, d_C, n, 0, &zero,
                              X, n, (long long)n * r, nb);
    cublasDsyrk(cb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, n, nb * r, &one, X, n, &one, d_K, n);
  }
  k_unpack_sym<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, jrs, n, d_J);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_symmetrize_lower<<<nb256((int64_t)n * n), 256, 0, st>>>(d_K, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? 0 : MG_ERR_CUDA;
}

// ------------------------------------------------------------ mixed path
// Slicing of one value y in (-1, 1) into s 8-bit pieces (oz_gemm.cuh):
// byte p of the result, S_0 signed, U_p (p >= 1) unsigned.  Every slice but
// the last is a floor (remainder in [0, 1)); the last one is rounded to
// nearest (clamped to 255), so the dropped tail has no systematic sign.
__device__ __forceinline__ void oz_cut(double y, int s, uint32_t (&w)[2 * kOzMaxSlices], int u) {
  const int word = u >> 2, sh = 8 * (u & 3);
  double t = floor(y * 128.0);
  y = y * 128.0 - t;
  // a tiny negative y (|128 y| < 2^-53) leaves 1 - |128 y|, which rounds to
  // exactly 1: carry it back (the value is then 0 to within 2^-53 of the row
  // maximum) so that every later slice stays within [0, 255]
  if (y >= 1.0) {
    t += 1.0;
    y -= 1.0;
  }
  w[word] |= ((uint32_t)(int)t & 255u) << sh;
  for (int p = 1; p < s; ++p) {
    t = p + 1 < s ? floor(y * 256.0) : fmin(floor(fma(y, 256.0, 0.5)), 255.0);
    w[2 * p + word] |= ((uint32_t)(int)t & 255u) << sh;
    y = y * 256.0 - t;
  }
}

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
    for (int b = lane; b < n; b += 32) m = fmax(m, fabs(LJ[inv[(size_t)a * n + b]]));
  m = warp_max(m);
  if (lane == 0) eL[row] = (short)max(-32000, oz_exponent(m));
}

// One thread per 8 consecutive columns of a row (J, a) of a block of nb
// vectors (slice p starts at LS + p * slice, the stride of the tensor map
// over a full block): gathers L_J[a, b0..b0+8) from the rs-packed FP64
// vectors through the inverse rs table, writes the s slices
// LS[p][J*ld + a][b0..b0+8) (zero beyond n) with the cached row exponent
// eL[J*ld + a] (copied to eA for the epilogue), and adds
// sum_b L_J[a,b] D[a,b] to V[J] (the Coulomb contraction
// V_J = sum_cd L_cd,J D_cd over the full square).
__global__ void k_oz_slice_l(const int* __restrict__ inv, int n, int64_t nrs, const double* __restrict__ L, int nb,
                             int ld, int s, int64_t slice, const short* __restrict__ eL, const double* __restrict__ D,
                             uint8_t* __restrict__ LS, int* __restrict__ eA, double* __restrict__ V) {
  const int per_row = ld / 8;
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = o < (int64_t)nb * ld * per_row;
  const int64_t row = live ? o / per_row : 0;
  const int b0 = live ? 8 * (int)(o - row * per_row) : 0;
  const int J = (int)(row / ld), a = (int)(row - (int64_t)J * ld);
  const int e = eL[row];
  double v = 0.0;
  if (live) {
    const double* LJ = L + nrs * J;
    uint32_t w[2 * kOzMaxSlices];
#pragma unroll
    for (int k = 0; k < 2 * kOzMaxSlices; ++k) w[k] = 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int b = b0 + u;
      double x = 0.0;
      if (a < n && b < n) {
        x = LJ[inv[(size_t)a * n + b]];
        v = fma(x, D[(size_t)a * n + b], v);
      }
      oz_cut(ldexp(x, -e), s, w, u);
    }
    uint8_t* out = LS + (size_t)row * ld + b0;
    for (int p = 0; p < s; ++p) *reinterpret_cast<uint2*>(out + p * slice) = make_uint2(w[2 * p], w[2 * p + 1]);
    if (b0 == 0) eA[row] = e;
  }
  // V[J]: a warp covers one row when ld / 8 >= 32 (ld is a multiple of 128), so
  // reduce over the warp and add once
  v = warp_sum(v);
  if (live && (threadIdx.x & 31) == 0 && a < n) atomicAdd(&V[J], v);
}

// C (n x r, column-major FP64) -> slices CS[q][k][0..ld) for k < npad
// (rows k >= r and columns b >= n zero), column exponents fC[k].  One warp
// per column k.
__global__ void k_oz_slice_c(const double* __restrict__ C, int n, int r, int npad, int ld, int s,
                             uint8_t* __restrict__ CS, int* __restrict__ fC) {
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (k >= npad) return;
  const double* ck = C + (size_t)n * k;
  double m = 0.0;
  if (k < r)
    for (int b = lane; b < n; b += 32) m = fmax(m, fabs(ck[b]));
  const int e = oz_exponent(warp_max(m));
  if (lane == 0) fC[k] = e;
  uint8_t* out = CS + (size_t)k * ld;
  const size_t slice = (size_t)npad * ld;
  for (int b0 = 8 * lane; b0 < ld; b0 += 256) {
    uint32_t w[2 * kOzMaxSlices];
#pragma unroll
    for (int q = 0; q < 2 * kOzMaxSlices; ++q) w[q] = 0;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int b = b0 + u;
      oz_cut(ldexp((k < r && b < n) ? ck[b] : 0.0, -e), s, w, u);
    }
    for (int q = 0; q < s; ++q) *reinterpret_cast<uint2*>(out + q * slice + b0) = make_uint2(w[2 * q], w[2 * q + 1]);
  }
}

// One thread per 8 consecutive columns of a row a of X (FP64, row stride
// xrow, columns [0, kx)): slices XS[p][a][col0 + c0 .. +8) (zero beyond kx and
// for rows a >= n) with the row exponent of xmax[a] (the largest |X| of the
// row, recorded by the half-transform), stored in eX[a].
__global__ void k_oz_slice_x(const double* __restrict__ X, int64_t xrow, int n, int kx, int ld, int kblk, int s,
                             int64_t xs_row, int64_t col0, const unsigned long long* __restrict__ xmax,
                             uint8_t* __restrict__ XS, int* __restrict__ eX) {
  const int per_row = kblk / 8;
  const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)ld * per_row) return;
  const int a = (int)(o / per_row), c0 = 8 * (int)(o - (int64_t)a * per_row);
  const int e = a < n ? oz_exponent(__longlong_as_double((long long)xmax[a])) : 0;
  if (c0 == 0) eX[a] = e;
  const double* xa = X + (size_t)a * xrow;
  uint32_t w[2 * kOzMaxSlices];
#pragma unroll
  for (int q = 0; q < 2 * kOzMaxSlices; ++q) w[q] = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int c = c0 + u;
    oz_cut(ldexp((a < n && c < kx) ? xa[c] : 0.0, -e), s, w, u);
  }
  const size_t slice = (size_t)ld * xs_row;
  uint8_t* out = XS + (size_t)a * xs_row + col0 + c0;
  for (int q = 0; q < s; ++q) *reinterpret_cast<uint2*>(out + q * slice) = make_uint2(w[2 * q], w[2 * q + 1]);
}

// xmax[a] = bits of max_c |X[a][c]| (for the self-test, where X is given)
__global__ void k_row_absmax(const double* __restrict__ X, int64_t xrow, int n, int kx,
                             unsigned long long* __restrict__ xmax) {
  const int a = blockIdx.x;
  double m = 0.0;
  if (a < n)
    for (int c = threadIdx.x; c < kx; c += blockDim.x) m = fmax(m, fabs(X[(size_t)a * xrow + c]));
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

// inv[a*n + b] = inv[b*n + a] = t for every rs pair t
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

// 3D 8-bit tensor map over slices [s][rows][kx] (kx contiguous), boxes of
// 32 bytes x box_rows x 1 slice, 32-byte swizzle.
static bool make_slice_map(CUtensorMap* m, const uint8_t* base, int64_t kx, int64_t rows, int s, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15) || kx % 32 || box_rows < 1 || box_rows > 256) return false;
  cuuint64_t gdim[3] = {(cuuint64_t)kx, (cuuint64_t)rows, (cuuint64_t)s};
  cuuint64_t gstr[2] = {(cuuint64_t)kx, (cuuint64_t)(kx * rows)};
  cuuint32_t box[3] = {32u, (cuuint32_t)box_rows, 1u}, es[3] = {1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, (void*)base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
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
  }
  cho_set_lexp(c, e, ld);
  return e;
}

int jk_mixed(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block, int s) {
  ChoState* c = h->cho;
  const int64_t nrs = cho_nrs(c);
  const int M = cho_nvec(c);
  const int n = h->nbf;
  if (s < 2 || s > kOzMaxSlices) { h->err = "mixed J/K: slices must be 2..8"; return MG_ERR_ARG; }
  const int ld = rup(n, 128);
  int nnt, Nt;
  oz_col_tiles(r, s, nnt, Nt);
  const int npad = nnt * Nt;
  // vectors per block: one block's K extent of the exchange product, nb r
  const int nb = std::min(block, M);
  const int kx = nb * r;
  const int kblk = rup(kx, 32);
  const int nsub = (kblk + kOzKChunk - 1) / kOzKChunk;
  const int ksub = rup((kblk + nsub - 1) / nsub, 32);
  const int nblocks = (M + nb - 1) / nb;
  const int G = std::min(16, nblocks);  // blocks per exchange-product group
  const int ntile = (ld / 128) * (ld / 128 + 1) / 2;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  cublasHandle_t cb = cho_cublas(c);
  cublasSetStream(cb, st);
  const int* d_ra = cho_rs_a_dev(c);
  const int* d_rb = cho_rs_b_dev(c);
  const size_t nn = (size_t)n * n;
  const int64_t xs_row = (int64_t)G * kblk;
  size_t need = 8 * (nrs + (size_t)nb + nn) + 4 * nn + (size_t)s * npad * ld + 4 * (size_t)npad +
                (size_t)s * nb * ld * ld + 4 * (size_t)nb * ld + 8 * (size_t)n * kx + 8 * (size_t)ld +
                (size_t)s * ld * xs_row + 4 * (size_t)G * ld + 8 * (size_t)nsm * 128 * 128 + 17 * 256;
  char* ws = (char*)ws_get(h, need, st);
  if (!ws) { h->err = "jk workspace allocation failed"; return MG_ERR_MEMORY; }
  auto take = [&](size_t bytes) { char* p = ws; ws += (bytes + 255) & ~(size_t)255; return (void*)p; };
  double* jrs = (double*)take(8 * nrs);
  double* V = (double*)take(8 * (size_t)nb);
  double* D = (double*)take(8 * nn);
  int* inv = (int*)take(4 * nn);
  uint8_t* CS = (uint8_t*)take((size_t)s * npad * ld);
  int* fC = (int*)take(4 * (size_t)npad);
  uint8_t* LS = (uint8_t*)take((size_t)s * nb * ld * ld);
  int* eA = (int*)take(4 * (size_t)nb * ld);
  double* Xf = (double*)take(8 * (size_t)n * kx);
  unsigned long long* xmax = (unsigned long long*)take(8 * (size_t)ld);
  uint8_t* XS = (uint8_t*)take((size_t)s * ld * xs_row);
  int* eX = (int*)take(4 * (size_t)G * ld);
  double* P = (double*)take(8 * (size_t)nsm * 128 * 128);
  int* d_err = (int*)take(sizeof(int));
  CUtensorMap map_l, map_c, map_x;
  if (!make_slice_map(&map_l, LS, ld, (int64_t)nb * ld, s, 128) || !make_slice_map(&map_c, CS, ld, npad, s, Nt) ||
      !make_slice_map(&map_x, XS, xs_row, ld, s, 128)) {
    h->err = "tensor maps for the exchange GEMMs could not be encoded";
    return MG_ERR_CUDA;
  }
  OzArgs ax{}, ak{};
  oz_plan(ax, s, Nt);
  oz_plan(ak, s, 128);
  if (ax.stages < 2 || ak.stages < 2) { h->err = "mixed J/K: slice tiles do not fit in shared memory"; return MG_ERR_ARG; }
  if (!smem_attr_once((const void*)oz_gemm_kernel<false>, kOzSmemLimit) ||
      !smem_attr_once((const void*)oz_gemm_kernel<true>, kOzSmemLimit)) {
    h->err = "exchange GEMMs: shared-memory limit could not be raised";
    return MG_ERR_CUDA;
  }
  ax.err = ak.err = d_err;
  ax.nrt = ld / 128; ax.nnt = nnt; ax.ld = ld; ax.n = n; ax.r = r; ax.eA = eA; ax.eB = fC; ax.X = Xf; ax.xrow = kx;
  ax.xmax = xmax;
  ak.ld = ld; ak.n = n; ak.ntile = ntile; ak.nsub = nsub; ak.kblk = kblk; ak.ksub = ksub; ak.eX = eX; ak.P = P;
  ak.K = d_K;
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  const double one = 1.0, zero = 0.0;
  cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, r, &one, d_C, n, d_C, n, &zero, D, n);
  cudaMemsetAsync(jrs, 0, 8 * nrs, st);
  cudaMemsetAsync(d_K, 0, 8 * nn, st);
  k_rs_inverse<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, n, inv);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const short* eL = oz_row_exponents(h, inv, ld, st);
  if (!eL) { h->err = "mixed J/K: row exponents could not be stored"; return MG_ERR_MEMORY; }
  k_oz_slice_c<<<(npad + 7) / 8, 256, 0, st>>>(d_C, n, r, npad, ld, s, CS, fC);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  for (int g0 = 0; g0 < nblocks; g0 += G) {
    const int gn = std::min(G, nblocks - g0);
    for (int bi = 0; bi < gn; ++bi) {
      const int J0 = (g0 + bi) * nb;
      const int nv = std::min(nb, M - J0);
      const double* Lb = cho_vec_ptr(c, J0, nv, st, h);
      if (!Lb) { h->err = "vector block straddles storage blocks"; return MG_ERR_ARG; }
      // a short last block: clear the columns of the missing vectors
      if (nv < nb) cudaMemsetAsync(Xf, 0, 8 * (size_t)n * kx, st);
      cudaMemsetAsync(V, 0, 8 * (size_t)nb, st);
      cudaMemsetAsync(xmax, 0, 8 * (size_t)ld, st);
      const int64_t nthr = (int64_t)nv * ld * (ld / 8);
      k_oz_slice_l<<<nb256(nthr), 256, 0, st>>>(inv, n, nrs, Lb, nv, ld, s, (int64_t)nb * ld * ld,
                                               eL + (size_t)J0 * ld, D, LS, eA, V);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      k_jacc64<<<nb256(nrs), 256, 0, st>>>(Lb, nrs, nv, V, jrs);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      // X_J = L_J C for the block (the slice map covers nb vectors; nv <= nb of them are used)
      ax.nJ = nv;
      ax.nitems = ax.nrt * nv * nnt;
      const int gx = std::min(ax.nitems, nsm);
      oz_gemm_kernel<false><<<gx, kOzThreads, ax.stages * ax.stage_bytes + 1024, st>>>(map_l, map_c, ax);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      k_oz_slice_x<<<nb256((int64_t)ld * (kblk / 8)), 256, 0, st>>>(Xf, kx, n, kx, ld, kblk, s, xs_row,
                                                                   (int64_t)bi * kblk, xmax, XS, eX + (size_t)bi * ld);
      g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    // K += X X^T over the group (lower tiles)
    ak.nblk = gn;
    ak.nitems = ntile * gn * nsub;
    const int gk = std::min(ak.nitems, nsm);
    oz_gemm_kernel<true><<<gk, kOzThreads, ak.stages * ak.stage_bytes + 1024, st>>>(map_x, map_x, ak);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  k_symmetrize_lower<<<nb256((int64_t)nn), 256, 0, st>>>(d_K, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_unpack_sym<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, jrs, n, d_J);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) { h->err = "mixed J/K: launch failed"; return MG_ERR_CUDA; }
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { h->err = "mixed J/K: device error"; return MG_ERR_CUDA; }
  if (herr) {
    h->err = "exchange GEMMs: a pipeline wait ran out (result incomplete)";
    return MG_ERR_CUDA;
  }
  return 0;
}

// The sliced engine on given dense matrices (verification of the kernels
// used by jk_mixed): X = A B^T (A: ld x ld, B: r x ld, both row-major; X
// row-major ld x r) and K = X X^T (lower triangle, column-major ld x ld).
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
  const size_t need = (size_t)s * ld * ld + 4 * (size_t)ld + (size_t)s * npad * ld + 4 * (size_t)npad +
                      (size_t)s * ld * kblk + 4 * (size_t)ld + 16 * (size_t)ld + 8 * (size_t)nsm * 128 * 128 +
                      18 * 256;
  char* ws = (char*)ws_get(h, need, st);
  if (!ws) return MG_ERR_MEMORY;
  auto take = [&](size_t bytes) { char* p = ws; ws += (bytes + 255) & ~(size_t)255; return (void*)p; };
  uint8_t* LS = (uint8_t*)take((size_t)s * ld * ld);
  int* eA = (int*)take(4 * (size_t)ld);
  uint8_t* CS = (uint8_t*)take((size_t)s * npad * ld);
  int* fC = (int*)take(4 * (size_t)npad);
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
  if (!smem_attr_once((const void*)oz_gemm_kernel<false>, kOzSmemLimit) ||
      !smem_attr_once((const void*)oz_gemm_kernel<true>, kOzSmemLimit))
    return MG_ERR_CUDA;
  ax.err = ak.err = d_err;
  ax.nrt = ld / 128; ax.nnt = nnt; ax.ld = ld; ax.n = ld; ax.r = r; ax.eA = eA; ax.eB = fC; ax.X = d_X; ax.xrow = r;
  ax.xmax = xmax; ax.nJ = 1; ax.nitems = ax.nrt * nnt;
  ak.ld = ld; ak.n = ld; ak.ntile = (ld / 128) * (ld / 128 + 1) / 2; ak.nsub = nsub; ak.kblk = kblk; ak.ksub = ksub;
  ak.eX = eX; ak.P = P; ak.K = d_K; ak.nblk = 1; ak.nitems = ak.ntile * nsub;
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  cudaMemsetAsync(d_K, 0, 8 * (size_t)ld * ld, st);
  cudaMemsetAsync(amax, 0, 8 * (size_t)ld, st);
  cudaMemsetAsync(xmax, 0, 8 * (size_t)ld, st);
  k_row_absmax<<<ld, 256, 0, st>>>(d_A, ld, ld, ld, amax);
  k_oz_slice_x<<<nb256((int64_t)ld * (ld / 8)), 256, 0, st>>>(d_A, ld, ld, ld, ld, ld, s, ld, 0, amax, LS, eA);
  if (d_slices) cudaMemcpyAsync(d_slices, LS, (size_t)s * ld * ld, cudaMemcpyDeviceToDevice, st);
  if (d_exps) cudaMemcpyAsync(d_exps, eA, 4 * (size_t)ld, cudaMemcpyDeviceToDevice, st);
  k_oz_slice_c<<<(npad + 7) / 8, 256, 0, st>>>(d_B, ld, r, npad, ld, s, CS, fC);
  oz_gemm_kernel<false><<<std::min(ax.nitems, nsm), kOzThreads, ax.stages * ax.stage_bytes + 1024, st>>>(map_l, map_c,
                                                                                                       ax);
  k_oz_slice_x<<<nb256((int64_t)ld * (kblk / 8)), 256, 0, st>>>(d_X, r, ld, r, ld, kblk, s, kblk, 0, xmax, XS, eX);
  oz_gemm_kernel<true><<<std::min(ak.nitems, nsm), kOzThreads, ak.stages * ak.stage_bytes + 1024, st>>>(map_x, map_x,
                                                                                                      ak);
  g_launches.fetch_add(6, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return MG_ERR_CUDA;
  return herr ? MG_ERR_CUDA : 0;
}

}  // namespace mg
