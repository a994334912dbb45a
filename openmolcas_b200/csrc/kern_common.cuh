// Device helpers shared by the Rys-quadrature kernels (ERIs and gradient).
#pragma once
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "mg_internal.h"

namespace mg {

// Raise the dynamic shared-memory limit of kernel `fn` on the current device.
// The attribute belongs to a (kernel, device) pair, so it is set once per
// device, under a lock (threads may make their first calls together).
inline bool smem_attr_once(const void* fn, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return true;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) return false;
  done.insert({fn, dev});
  return true;
}

// Rys root/weight table: per-order metadata and the device coefficient pool.
struct RysArgs {
  RysMeta m[MG_MAX_RYS];
  const double* tab;
};

// Threads of one work group synchronise on their own named barrier (id 1 + group).
__device__ __forceinline__ void gsync(int g, int tpq) {
  if (tpq == 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(tpq) : "memory");
}

__device__ __forceinline__ int d_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int d_ncomp(int l) { return l >= 2 ? 2 * l + 1 : d_ncart(l); }
__device__ __forceinline__ int d_ccum(int l) { return l * (l + 1) * (l + 2) / 6; }
__device__ __forceinline__ int d_sph_off(int l) { return l == 0 ? 0 : l == 1 ? 1 : l == 2 ? 10 : 40; }
__device__ __forceinline__ int ev2(int x) { return (x + 1) & ~1; }

// Division by a run-time divisor n through a multiply-high:
// q = floor(o * ceil(2^32 / n) / 2^32), exact for o < 2^32 / n (the host
// planner checks every loop extent against that bound); n = 1 uses the mask.
struct FDiv {
  unsigned m, k, n;
};
__device__ __forceinline__ FDiv fdiv(unsigned n) {
  FDiv f;
  f.n = n;
  f.m = n == 1 ? 0u : 0xFFFFFFFFu / n + 1u;
  f.k = n == 1 ? 0xFFFFFFFFu : 0u;
  return f;
}
__device__ __forceinline__ unsigned fq(unsigned o, const FDiv& f) { return __umulhi(o, f.m) + (o & f.k); }

// one Rys root/weight of order N at T (table or asymptotic)
template <int N>
__device__ __forceinline__ void rys_one(const RysArgs& ra, double T, int r, double& x, double& w) {
  const RysMeta& m = ra.m[N - 1];
  if (T >= m.tmax) {
    const double ai = 1.0 / T;
    x = m.hx[r] * ai;
    w = m.hw[r] * sqrt(ai);
  } else {
    int k = (int)(T * m.invh);
    k = k < m.K ? k : m.K - 1;
    const double s = 2.0 * (T - k * m.h) * m.invh - 1.0;
    const double* c = ra.tab + m.off + (size_t)k * (2 * N * 8);
    const double* cx = c + r * 8;
    const double* cw = c + (N + r) * 8;
    double ax = __ldg(cx + 7), aw = __ldg(cw + 7);
#pragma unroll
    for (int j = 6; j >= 0; --j) {
      ax = fma(ax, s, __ldg(cx + j));
      aw = fma(aw, s, __ldg(cw + j));
    }
    x = ax;
    w = aw;
  }
}

// all N Rys roots/weights of order N at T (one table interval shared by the roots)
template <int N>
__device__ __forceinline__ void rys_all(const RysArgs& ra, double T, double* x, double* w) {
  const RysMeta& m = ra.m[N - 1];
  if (T >= m.tmax) {
    const double ai = 1.0 / T, si = sqrt(ai);
#pragma unroll
    for (int r = 0; r < N; ++r) {
      x[r] = m.hx[r] * ai;
      w[r] = m.hw[r] * si;
    }
  } else {
    int k = (int)(T * m.invh);
    k = k < m.K ? k : m.K - 1;
    const double s = 2.0 * (T - k * m.h) * m.invh - 1.0;
    const double* c = ra.tab + m.off + (size_t)k * (2 * N * 8);
#pragma unroll
    for (int q = 0; q < 2 * N; ++q) {
      const double* cq = c + q * 8;
      double acc = __ldg(cq + 7);
#pragma unroll
      for (int j = 6; j >= 0; --j) acc = fma(acc, s, __ldg(cq + j));
      if (q < N) x[q] = acc;
      else w[q - N] = acc;
    }
  }
}

// Cartesian exponents of the components of one shell in C3 order (compile-time).
template <int L>
struct CartExp {
  static constexpr int n = (L + 1) * (L + 2) / 2;
  int e[n > 0 ? n : 1][3];
  constexpr CartExp() : e() {
    int k = 0;
    for (int lx = L; lx >= 0; --lx)
      for (int ly = L - lx; ly >= 0; --ly) {
        e[k][0] = lx;
        e[k][1] = ly;
        e[k][2] = L - lx - ly;
        ++k;
      }
  }
};

}  // namespace mg
