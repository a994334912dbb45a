// Coulomb / exchange matrices from Cholesky vectors (the CHO_LK_SCF build,
// fock_util/cho_lk_scf.F90:14) on the GPU.
//
//   D = C C^T (C: nbf x r, the Cholesky/orbital factor of the density, as
//   ChoSCF_Drv passes it, scf/choscf_drv.F90:115-116)
//   J_ab = sum_J L_ab,J V_J,  V_J = sum_cd L_cd,J D_cd     (cho_lk_scf.F90:442-449)
//   K_ab = sum_J sum_k X_J[a,k] X_J[b,k],  X_J = L_J C      (cho_lk_scf.F90:507-830)
//
// Mixed path: vectors stored FP32; per block of vectors the rs-packed L_J
// are unpacked into dense split BF16 squares (hi + lo, hi = bf16(x),
// lo = bf16(x - hi)); both exchange GEMMs are hand-written tcgen05 kernels
// with 3 BF16 products (hi*hi + hi*lo + lo*hi) into FP32 tensor memory, fed
// by TMA: the half-transform X_J = L_J C (tc_xgemm.cuh) writes the split,
// K-major X^T directly, and K += X X^T (tc_syrk.cuh: lower-triangle tiles,
// FP32 over one block's nb*r terms, FP64 atomic accumulation) keeps the
// accumulation error from growing with the number of vectors.  J uses FP32
// loads with FP64 accumulation.
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
#include "tc_syrk.cuh"
#include "tc_xgemm.cuh"

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
// split x -> (hi, lo) BF16
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// inv[a*n + b] = inv[b*n + a] = t for every rs pair t (entries outside the
// reduced set stay -1)
__global__ void k_rs_inverse(const int* __restrict__ rs_a, const int* __restrict__ rs_b, int64_t nrs, int n,
                             int* __restrict__ inv) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  const int a = rs_a[t], b = rs_b[t];
  inv[(size_t)a * n + b] = (int)t;
  inv[(size_t)b * n + a] = (int)t;
}

// Dense split squares Lhi/Llo[J][a][b] (leading dimension ld, padding zero)
// written row by row, two columns per thread (coalesced 4-byte stores); the
// packed value is gathered through the inverse rs table.
__global__ void k_unpack_dense_split(const int* __restrict__ inv, int n, int64_t nrs, const float* __restrict__ L,
                                     int nb, int ld, __nv_bfloat162* __restrict__ Lhi,
                                     __nv_bfloat162* __restrict__ Llo) {
  const int64_t half = ld / 2;
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)nb * ld * half) return;
  const int b2 = (int)(o % half);
  const int64_t r1 = o / half;
  const int a = (int)(r1 % ld);
  const int J = (int)(r1 / ld);
  float v[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int b = 2 * b2 + u;
    float x = 0.0f;
    if (a < n && b < n) {
      const int t = inv[(size_t)a * n + b];
      if (t >= 0) x = L[t + nrs * J];
    }
    v[u] = x;
  }
  __nv_bfloat16 h0, l0, h1, l1;
  split_bf16(v[0], h0, l0);
  split_bf16(v[1], h1, l1);
  Lhi[o] = __halves2bfloat162(h0, h1);
  Llo[o] = __halves2bfloat162(l0, l1);
}

// C (n x r, column-major FP64) -> split BF16 with leading dimension ld (padding zero)
__global__ void k_split_c(const double* __restrict__ C, int n, int r, int ld, __nv_bfloat16* __restrict__ hi,
                          __nv_bfloat16* __restrict__ lo) {
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)ld * r) return;
  const int a = (int)(o % ld), k = (int)(o / ld);
  __nv_bfloat16 h = __float2bfloat16_rn(0.0f), l = h;
  if (a < n) split_bf16((float)C[a + (size_t)n * k], h, l);
  hi[o] = h;
  lo[o] = l;
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

// 2D BF16 tensor map over rows x kpad (K contiguous), 64 x box_rows boxes, 128-byte swizzle.
static bool make_operand_map(CUtensorMap* m, const __nv_bfloat16* base, int rows, int kpad, int box_rows = kTcTile) {
  auto enc = tensor_map_encoder();
  if (!enc || ((uintptr_t)base & 15) || (kpad * 2) % 16 || box_rows < 1 || box_rows > 256) return false;
  cuuint64_t gdim[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
  cuuint64_t gstr[1] = {(cuuint64_t)kpad * 2};
  cuuint32_t box[2] = {(cuuint32_t)kTcBK, (cuuint32_t)box_rows}, es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// V[J] += sum_t L[t,J] dw[t] over one row chunk (FP32 loads, FP64 accumulation);
// grid (vectors, row chunks); V must be zeroed first
__global__ void k_jvec(const float* __restrict__ L, int64_t nrs, const double* __restrict__ dw, double* __restrict__ V) {
  const int J = blockIdx.x;
  const float* l = L + nrs * J;
  const int64_t chunk = (nrs + gridDim.y - 1) / gridDim.y;
  const int64_t t0 = chunk * blockIdx.y, t1 = min(nrs, t0 + chunk);
  double s = 0.0;
  for (int64_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) s = fma((double)l[t], dw[t], s);
  __shared__ double red[32];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) atomicAdd(&V[J], s);
  }
}

// jrs[t] += sum_J L[t,J] V[J]
__global__ void k_jacc(const float* __restrict__ L, int64_t nrs, int nb, const double* __restrict__ V,
                       double* __restrict__ jrs) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  double s = 0.0;
  for (int J = 0; J < nb; ++J) s = fma((double)L[t + nrs * J], V[J], s);
  jrs[t] += s;
}


int jk_mixed(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block) {
  ChoState* c = h->cho;
  const int64_t nrs = cho_nrs(c);
  const int M = cho_nvec(c);
  const int n = h->nbf;
  // rows of the squares and of X^T padded to the 128-row tensor-core tile (padding zero)
  const int ld = (n + 127) / 128 * 128;
  if (!cho_vec_ptr32(c, 0, 1)) {
    int rc = cho_make_fp32(c, st);
    if (rc) { h->err = "FP32 vector copy failed"; return rc; }
  }
  cublasHandle_t cb = cho_cublas(c);
  cublasSetStream(cb, st);
  const int* d_ra = cho_rs_a_dev(c);
  const int* d_rb = cho_rs_b_dev(c);
  const size_t nn = (size_t)n * n, ll = (size_t)ld * ld;
  // exchange product: K range split so that the lower-triangle tiles x splits cover the SMs
  const int ntile = (ld / kTcTile) * (ld / kTcTile + 1) / 2;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  const int nsplit = std::max(1, std::min(8, (nsm + ntile - 1) / ntile));
  const int kq = kTcBK * nsplit;
  const int kpad = (block * r + kq - 1) / kq * kq;
  const size_t xt = (size_t)ld * kpad;
  const int bbox = r <= kXgMaxN ? (r + 15) / 16 * 16 : kXgMaxN;  // rows of a C box
  size_t need = 8 * ((size_t)2 * nrs + block + nn) + 2 * (2 * (size_t)ld * r) + 2 * (2 * (size_t)block * ll) +
                2 * (2 * xt) + 4 * nn + 16 * 256;
  char* ws = (char*)ws_get(h, need, st);
  if (!ws) { h->err = "jk workspace allocation failed"; return MG_ERR_MEMORY; }
  auto take = [&](size_t bytes) { char* p = ws; ws += (bytes + 255) & ~(size_t)255; return (void*)p; };
  double* dw = (double*)take(8 * nrs);
  double* jrs = (double*)take(8 * nrs);
  double* V = (double*)take(8 * block);
  double* D = (double*)take(8 * nn);
  __nv_bfloat16* Chi = (__nv_bfloat16*)take(2 * (size_t)ld * r);
  __nv_bfloat16* Clo = (__nv_bfloat16*)take(2 * (size_t)ld * r);
  __nv_bfloat16* Lhi = (__nv_bfloat16*)take(2 * (size_t)block * ll);
  __nv_bfloat16* Llo = (__nv_bfloat16*)take(2 * (size_t)block * ll);
  __nv_bfloat16* XThi = (__nv_bfloat16*)take(2 * xt);
  __nv_bfloat16* XTlo = (__nv_bfloat16*)take(2 * xt);
  int* d_err = (int*)take(sizeof(int));
  int* inv = (int*)take(4 * nn);
  CUtensorMap map_hi, map_lo, map_lhi, map_llo, map_chi, map_clo;
  if (!make_operand_map(&map_hi, XThi, ld, kpad) || !make_operand_map(&map_lo, XTlo, ld, kpad) ||
      !make_operand_map(&map_lhi, Lhi, block * ld, ld) || !make_operand_map(&map_llo, Llo, block * ld, ld) ||
      !make_operand_map(&map_chi, Chi, r, ld, bbox) || !make_operand_map(&map_clo, Clo, r, ld, bbox)) {
    h->err = "tensor maps for the exchange GEMMs could not be encoded";
    return MG_ERR_CUDA;
  }
  if (!smem_attr_once((const void*)tc_syrk3_kernel, kTcSmem) ||
      !smem_attr_once((const void*)tc_xgemm3_kernel, kXgSmem)) {
    h->err = "exchange GEMMs: shared-memory limit could not be raised";
    return MG_ERR_CUDA;
  }
  cudaMemsetAsync(d_err, 0, sizeof(int), st);
  const double one = 1.0, zero = 0.0;
  cublasDgemm(cb, CUBLAS_OP_N, CUBLAS_OP_T, n, n, r, &one, d_C, n, d_C, n, &zero, D, n);
  k_pack_density<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, D, n, dw);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_split_c<<<nb256((int64_t)ld * r), 256, 0, st>>>(d_C, n, r, ld, Chi, Clo);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaMemsetAsync(jrs, 0, 8 * nrs, st);
  cudaMemsetAsync(d_K, 0, 8 * nn, st);
  cudaMemsetAsync(XThi, 0, 2 * xt, st);  // columns beyond nb*r stay zero
  cudaMemsetAsync(XTlo, 0, 2 * xt, st);
  cudaMemsetAsync(inv, 0xFF, 4 * nn, st);
  k_rs_inverse<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, n, inv);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  const unsigned jchunks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(64, nrs / 8192));
  for (int J0 = 0; J0 < M; J0 += block) {
    const int nb = std::min(block, M - J0);
    const float* Lb = cho_vec_ptr32(c, J0, nb);
    if (!Lb) { h->err = "vector block straddles storage blocks"; return MG_ERR_ARG; }
    // Coulomb
    cudaMemsetAsync(V, 0, 8 * nb, st);
    k_jvec<<<dim3(nb, jchunks), 256, 0, st>>>(Lb, nrs, dw, V);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_jacc<<<nb256(nrs), 256, 0, st>>>(Lb, nrs, nb, V, jrs);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    // Exchange: split squares of the block, X_J = L_J C written as split X^T (tcgen05),
    // then K += X X^T (tcgen05; 3 products into one FP32 accumulator per tile, FP64
    // atomic add into K).  A short last block leaves stale X^T columns of the previous
    // block beyond nb*r: clear them first.
    k_unpack_dense_split<<<nb256((int64_t)nb * ld * (ld / 2)), 256, 0, st>>>(
        inv, n, nrs, Lb, nb, ld, (__nv_bfloat162*)Lhi, (__nv_bfloat162*)Llo);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (nb < block && J0 > 0) {
      cudaMemsetAsync(XThi, 0, 2 * xt, st);
      cudaMemsetAsync(XTlo, 0, 2 * xt, st);
    }
    tc_xgemm3_kernel<<<dim3(ld / kTcTile, nb, (r + kXgMaxN - 1) / kXgMaxN), 128, kXgSmem, st>>>(
        map_lhi, map_llo, map_chi, map_clo, ld, r, bbox, kpad, XThi, XTlo, d_err);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    tc_syrk3_kernel<<<dim3(ntile, nsplit), 128, kTcSmem, st>>>(map_hi, map_lo, n, kpad, d_K, d_err);
    g_launches.fetch_add(1, std::memory_order_relaxed);
  }
  k_symmetrize_lower<<<nb256((int64_t)nn), 256, 0, st>>>(d_K, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  k_unpack_sym<<<nb256(nrs), 256, 0, st>>>(d_ra, d_rb, nrs, jrs, n, d_J);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (cudaGetLastError() != cudaSuccess) return MG_ERR_CUDA;
  int herr = 0;
  cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) return MG_ERR_CUDA;
  if (herr) {
    h->err = "exchange GEMMs: a pipeline wait ran out (result incomplete)";
    return MG_ERR_CUDA;
  }
  return 0;
}

}  // namespace mg
