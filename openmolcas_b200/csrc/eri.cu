// FP64 Rys-quadrature ERIs: launch planning and the class launcher.  The
// kernel (stages, reference anchors) is in eri_kernel.cuh; its instantiations
// are in eri_k_lo.cu and eri_k_hi.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <vector>

#include "eri_kernel.cuh"

namespace mg {

EriFn eri_kernel_pick_lo(int nab, int ncd);
EriFn eri_kernel_pick_hi(int nab, int ncd);
EriFn eri_kernel_pick(int nab, int ncd) {
  return nab <= 3 ? eri_kernel_pick_lo(nab, ncd) : eri_kernel_pick_hi(nab, ncd);
}

// Cartesian exponent table of the kernel (l = 0..7, C3 order, packed as
// lx | ly << 8 | lz << 16), built at compile time into a file-scope device
// array: the launcher only looks its address up, so an ERI launch never
// allocates device memory.
struct EriCartTable {
  int v[2 * kETabD];
  constexpr EriCartTable() : v() {
    int k = 0;
    for (int l = 0; l <= 7; ++l)
      for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) v[k++] = lx | (ly << 8) | ((l - lx - ly) << 16);
  }
};
static_assert(sizeof(EriCartTable) == sizeof(double) * kETabD, "exponent table size");
static __device__ __align__(16) const EriCartTable g_eri_cart_table{};

// Device address of the table on `device` (looked up once per device, with
// that device current; cudaGetSymbolAddress does not allocate).
static const double* eri_tables(int device) {
  static const double* tab[64] = {nullptr};
  static std::mutex mu;
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!tab[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_eri_cart_table) != cudaSuccess) return nullptr;
    tab[device] = (const double*)p;
  }
  return tab[device];
}

static inline size_t ev2s(size_t x) { return (x + 1) & ~(size_t)1; }

// Launch plan of one class: tpq threads per work item (a group), 512/tpq
// groups per CTA, primitive quartets in tiles of PAB bra x PCD ket pairs.
// Per-group shared memory (doubles), the kernel's layout:
//   hdr 2 | acc | Cab | Ccd | Ft (bounded by ne + nf ints) | max( X + cf + I + E, HRR temp )
static size_t eri_group_smem(int nab, int ncd, const ClassStats& cs, int pab, int pcd) {
  const int NR = (nab + ncd) / 2 + 1, NI = nab + 1, NJ = ncd + 1;
  const size_t gst = (size_t)(3 * NR * NI * NJ) | 1, cfs = NR * 10 + 1;
  const size_t nt = (size_t)pab * pcd;
  const size_t tile = ev2s((size_t)cs.max_nij * pcd * cs.max_nef) + ev2s(nt * cfs) + nt * gst +
                      nt * (size_t)(cs.max_nef | 1);
  return 2 + ev2s(cs.max_acc) + ev2s(cs.max_cab) + ev2s(cs.max_ccd) + ev2s((cs.max_ne + cs.max_nf + 1) / 2) +
         std::max(tile, ev2s(cs.max_tmp));
}

// tpq0: the first group size tried (0: from the widest stage); order: the tile
// dimension shrunk first when it does not fit (0 ket primitives, 1 bra; + 2:
// the tile starts from 64 x 16 primitive pairs instead of 32 x 8)
ClassPlan eri_plan(int nab, int ncd, const ClassStats& cs, int tpq0, int order) {
  const int NR = (nab + ncd) / 2 + 1;
  ClassPlan pl{0, 0, 0, 0, 0};
  const size_t budget = (227 * 1024) / 8 - kETabD;  // one CTA per SM
  const bool big = order >= 2;
  order %= 2;
  int pab = std::max(1, std::min(cs.max_npab, big ? 64 : 32));
  int pcd = std::max(1, std::min(cs.max_npcd, big ? 16 : 8));
  const int width = std::max({cs.max_acc, pab * pcd * cs.max_nef / 2, pab * pcd * NR * 3 * 8});
  // the kernel's multiply-high divisions are exact below 2^32: largest loop
  // extent x divisor of a tile a x c
  auto bound = [&](int a, int c) {
    const double nt = (double)a * c;
    return std::max({nt * cs.max_nef * nt, (double)cs.max_nij * c * cs.max_nef * cs.max_nef,
                     (double)cs.max_acc * cs.max_nef, (double)cs.max_tmp * cs.max_nf, (double)cs.max_tmp * cs.max_nc});
  };
  for (int tpq = tpq0 ? tpq0 : width <= 96 ? 64 : width <= 384 ? 128 : 256; tpq <= kEriThreads; tpq *= 2) {
    const int groups = kEriThreads / tpq;
    const size_t gbudget = (budget / groups) & ~(size_t)1;
    int a = pab, c = pcd;
    while ((eri_group_smem(nab, ncd, cs, a, c) > gbudget || bound(a, c) >= 4294967296.0) && (a > 1 || c > 1)) {
      if (order == 1 && a > 1) a = (a + 1) / 2;
      else if (c > 1) c = (c + 1) / 2;
      else a = (a + 1) / 2;
    }
    if (eri_group_smem(nab, ncd, cs, a, c) <= gbudget) {
      pl.tpq = tpq;
      pl.PAB = a;
      pl.PCD = c;
      pl.gsm = (int)eri_group_smem(nab, ncd, cs, a, c);
      pl.smem = 8 * ((size_t)pl.gsm * groups + kETabD);
      if (bound(a, c) >= 4294967296.0) pl.PAB = 0;
      return pl;
    }
  }
  return pl;  // PAB == 0: does not fit
}

int eri_launch_class(Handle* h, const EriItem* d_items, int nitems, int nab, int ncd, const ClassPlan& pl, double* out,
                     int* d_counter, cudaStream_t st) {
  EriFn k = eri_kernel_pick(nab, ncd);
  const double* tab = eri_tables(h->device);
  if (!k || !tab) return 2;
  RysArgs ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  const int groups = kEriThreads / pl.tpq;
  int per_sm = 0, nsm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kEriThreads, pl.smem);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
  if (per_sm < 1) return 3;
  const long long want = (nitems + groups - 1) / groups;
  const int nblk = (int)std::min<long long>(want, (long long)per_sm * nsm);
  EriArgs a{d_items, nitems, h->d_pairs, h->d_prim, h->tot_np, h->d_coef, h->d_hrr, tab, out, d_counter,
            pl.tpq, pl.gsm, pl.PAB, pl.PCD};
  k<<<nblk, kEriThreads, pl.smem, st>>>(a, ra);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // namespace mg
