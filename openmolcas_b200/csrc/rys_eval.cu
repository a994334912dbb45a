// Device evaluation of the Rys root/weight table for arbitrary arguments
// (mg_rys_roots): the same table lookup the ERI and gradient kernels use,
// exposed for unit tests against the reference's own table values.
#include <cuda_runtime.h>

#include "kern_common.cuh"

namespace mg {

template <int N>
__global__ void k_rys_eval(RysArgs ra, const double* __restrict__ T, int64_t n, double* __restrict__ x,
                           double* __restrict__ w) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xr[N], wr[N];
  rys_all<N>(ra, T[i], xr, wr);
#pragma unroll
  for (int r = 0; r < N; ++r) {
    x[i * N + r] = xr[r];
    w[i * N + r] = wr[r];
  }
}

int rys_eval(Handle* h, int nrys, int64_t n, const double* d_T, double* d_x, double* d_w) {
  RysArgs ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  const unsigned nb = (unsigned)((n + 255) / 256);
  switch (nrys) {
#define MG_RYS_CASE(N) \
  case N: k_rys_eval<N><<<nb, 256>>>(ra, d_T, n, d_x, d_w); break;
    MG_RYS_CASE(1) MG_RYS_CASE(2) MG_RYS_CASE(3) MG_RYS_CASE(4) MG_RYS_CASE(5)
    MG_RYS_CASE(6) MG_RYS_CASE(7) MG_RYS_CASE(8) MG_RYS_CASE(9)
#undef MG_RYS_CASE
    default: return MG_ERR_ARG;
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? 0 : MG_ERR_CUDA;
}

}  // namespace mg
