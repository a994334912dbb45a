// FP64 Rys-quadrature ERIs over contracted shell quartets (sm_100a).
//
// One CTA per work item (bra pair, ket pair, range of contracted ijkl).
// Per chunk of NP primitive quartets:
//   1a  thread per primitive quartet: T, prefactor, Rys roots/weights
//       (table lookup), recursion coefficients (TERI teri.F90:51-57, ModU2,
//       vCff2D vcff2d.F90) -> shared memory
//   1b  thread per (quartet, root, xyz): 2D recursion (vRys2D vrys2d.F90)
//       in registers, weight*prefactor folded into z -> shared memory
//   2a  thread per (quartet, e, f): [e0|f0] = sum_r Ix Iy Iz  (RysEF)
//   2b  thread per (ijkl, e, f): contraction with the general-contraction
//       coefficient products (Cntrct), accumulated in shared memory
// then HRR + real-spherical transform with the per-pair matrices
// (HrrMtrx/TnsCtl, hrrmtrx.F90, tnsctl.F90) and the store in the layout of
// Eval_IJKL's AOInt(nijkl, iCmp1..4) (twoel_nosym.F90:372).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "mg_internal.h"

namespace mg {

struct RysArgs {
  RysMeta m[MG_MAX_RYS];
  const double* tab;
};

// Cartesian exponents in C3 order (index_functions.F90 C3_Ind3), l = 0..7
__constant__ unsigned char c_cart[120][3];

static void init_cart_table() {
  static bool done = false;
  if (done) return;
  unsigned char t[120][3];
  int k = 0;
  for (int l = 0; l <= 7; ++l)
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) {
        t[k][0] = lx; t[k][1] = ly; t[k][2] = l - lx - ly;
        ++k;
      }
  cudaMemcpyToSymbol(c_cart, t, sizeof(t));
  done = true;
}

template <int N>
__device__ __forceinline__ void rys_rw(const RysArgs& ra, double T, double* x, double* w) {
  const RysMeta& m = ra.m[N - 1];
  if (T >= m.tmax) {
    const double ai = 1.0 / T, si = sqrt(ai);
#pragma unroll
    for (int i = 0; i < N; ++i) { x[i] = m.hx[i] * ai; w[i] = m.hw[i] * si; }
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
      if (q < N) x[q] = acc; else w[q - N] = acc;
    }
  }
}

template <int NAB, int NCD>
__global__ void __launch_bounds__(256) eri_kernel(const EriItem* __restrict__ items, const DPair* __restrict__ pairs,
                                                  const double* __restrict__ prim, int tot_np,
                                                  const double* __restrict__ coef, const double* __restrict__ hrr,
                                                  RysArgs ra, double* __restrict__ out, int NP) {
  constexpr int NR = (NAB + NCD) / 2 + 1;
  constexpr int NI = NAB + 1, NJ = NCD + 1;
  constexpr int G1 = NR * NI * NJ;  // one direction
  constexpr int NCF = 10;
  extern __shared__ double sm[];
  const EriItem it = items[blockIdx.x];
  const DPair& P = pairs[it.p];
  const DPair& Q = pairs[it.q];
  const int npab = P.np, npcd = Q.np;
  const int nij = P.nci * P.ncj;
  const int ne = P.ne, nf = Q.ne, nef = ne * nf;
  const int nc = it.c1 - it.c0;
  const int eoff = P.emin * (P.emin + 1) * (P.emin + 2) / 6;
  const int foff = Q.emin * (Q.emin + 1) * (Q.emin + 2) / 6;
  double* acc = sm;                       // nc * nef
  double* cf = acc + nc * nef;            // NP * NR * NCF
  double* G = cf + NP * NR * NCF;         // NP * 3 * G1
  double* E = G + NP * 3 * G1;            // NP * nef (also HRR temp)
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int o = tid; o < nc * nef; o += nth) acc[o] = 0.0;
  const double Ap0 = P.Ap[0], Ap1 = P.Ap[1], Ap2 = P.Ap[2];
  const double Cp0 = Q.Ap[0], Cp1 = Q.Ap[1], Cp2 = Q.Ap[2];
  const long long ntot = (long long)npab * npcd;
  for (long long base = 0; base < ntot; base += NP) {
    const int nt = (int)min((long long)NP, ntot - base);
    __syncthreads();
    // ---- 1a: roots and recursion coefficients
    for (int t = tid; t < nt; t += nth) {
      const long long tg = base + t;
      const int pcd = (int)(tg / npab), pab = (int)(tg - (long long)pcd * npab);
      const int ia = P.prim_off + pab, ic = Q.prim_off + pcd;
      const double zeta = prim[ia], eta = prim[ic];
      const double kab = prim[tot_np + ia], kcd = prim[tot_np + ic];
      const double px = prim[2 * tot_np + ia], py = prim[3 * tot_np + ia], pz = prim[4 * tot_np + ia];
      const double qx = prim[2 * tot_np + ic], qy = prim[3 * tot_np + ic], qz = prim[4 * tot_np + ic];
      const double ze = zeta + eta, zei = 1.0 / ze, rho = zeta * eta * zei;
      const double dx = px - qx, dy = py - qy, dz = pz - qz;
      const double T = rho * (dx * dx + dy * dy + dz * dz);
      const double fact = kab * kcd * sqrt(zei);
      double x[NR], w[NR];
      rys_rw<NR>(ra, T, x, w);
      const double zi = 1.0 / zeta, ei = 1.0 / eta;
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const double U2 = x[r] * zei;
        double* c = cf + (t * NR + r) * NCF;
        c[0] = 0.5 * U2;
        c[1] = 0.5 * (1.0 - U2 * eta) * zi;
        c[2] = 0.5 * (1.0 - U2 * zeta) * ei;
        c[3] = px - Ap0 - eta * U2 * dx;
        c[4] = py - Ap1 - eta * U2 * dy;
        c[5] = pz - Ap2 - eta * U2 * dz;
        c[6] = qx - Cp0 + zeta * U2 * dx;
        c[7] = qy - Cp1 + zeta * U2 * dy;
        c[8] = qz - Cp2 + zeta * U2 * dz;
        c[9] = w[r] * fact;
      }
    }
    __syncthreads();
    // ---- 1b: 2D recursion per (quartet, root, direction)
    for (int job = tid; job < nt * NR * 3; job += nth) {
      const int d = job % 3, tr = job / 3, r = tr % NR, t = tr / NR;
      const double* c = cf + (t * NR + r) * NCF;
      const double B00 = c[0], B10 = c[1], B01 = c[2], C00 = c[3 + d], D00 = c[6 + d];
      double I[NI][NJ];
      I[0][0] = d == 2 ? c[9] : 1.0;
      if (NI > 1) I[1][0] = C00 * I[0][0];
#pragma unroll
      for (int i = 1; i < NI - 1; ++i) I[i + 1][0] = C00 * I[i][0] + i * B10 * I[i - 1][0];
#pragma unroll
      for (int j = 0; j < NJ - 1; ++j) {
#pragma unroll
        for (int i = 0; i < NI; ++i) {
          double v = D00 * I[i][j];
          if (j > 0) v += j * B01 * I[i][j - 1];
          if (i > 0) v += i * B00 * I[i - 1][j];
          I[i][j + 1] = v;
        }
      }
      double* g = G + (t * 3 + d) * G1 + r * NI * NJ;
#pragma unroll
      for (int i = 0; i < NI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) g[i * NJ + j] = I[i][j];
    }
    __syncthreads();
    // ---- 2a: [e0|f0] per primitive quartet
    for (int job = tid; job < nt * nef; job += nth) {
      const int ef = job % nef, t = job / nef;
      const int ie = ef % ne, jf = ef / ne;
      const unsigned char* ce = c_cart[eoff + ie];
      const unsigned char* cfp = c_cart[foff + jf];
      const double* gx = G + (t * 3 + 0) * G1 + ce[0] * NJ + cfp[0];
      const double* gy = G + (t * 3 + 1) * G1 + ce[1] * NJ + cfp[1];
      const double* gz = G + (t * 3 + 2) * G1 + ce[2] * NJ + cfp[2];
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < NR; ++r) s = fma(gx[r * NI * NJ] * gy[r * NI * NJ], gz[r * NI * NJ], s);
      E[t * nef + ef] = s;
    }
    __syncthreads();
    // ---- 2b: contraction
    for (int o = tid; o < nc * nef; o += nth) {
      const int ijkl = it.c0 + o / nef, ef = o - (o / nef) * nef;
      const int kl = ijkl / nij, ij = ijkl - kl * nij;
      const double* ca = coef + P.coef_off + (size_t)ij * npab;
      const double* cc = coef + Q.coef_off + (size_t)kl * npcd;
      int pcd = (int)(base / npab), pab = (int)(base - (long long)pcd * npab);
      double s = 0.0;
      for (int t = 0; t < nt; ++t) {
        s = fma(__ldg(ca + pab) * __ldg(cc + pcd), E[t * nef + ef], s);
        if (++pab == npab) { pab = 0; ++pcd; }
      }
      acc[o] += s;
    }
  }
  __syncthreads();
  // ---- 3: HRR + spherical, bra then ket
  const int nsab = P.nsa * P.nsb, nscd = Q.nsa * Q.nsb;
  const double* Hab = hrr + P.hrr_off;
  const double* Hcd = hrr + Q.hrr_off;
  double* tmp = E;  // nc * nsab * nf
  for (int o = tid; o < nc * nsab * nf; o += nth) {
    const int jf = o % nf, r1 = o / nf, sab = r1 % nsab, cl = r1 / nsab;
    const double* a = acc + cl * nef + jf * ne;
    const double* hc = Hab + (size_t)sab * ne;
    double s = 0.0;
    for (int ie = 0; ie < ne; ++ie) s = fma(__ldg(hc + ie), a[ie], s);
    tmp[o] = s;
  }
  __syncthreads();
  const long long nijkl = (long long)nij * Q.nci * Q.ncj;
  for (int o = tid; o < nc * nsab * nscd; o += nth) {
    const int cl = o % nc, r1 = o / nc, sab = r1 % nsab, scd = r1 / nsab;
    const double* tp = tmp + ((size_t)cl * nsab + sab) * nf;
    const double* hc = Hcd + (size_t)scd * nf;
    double s = 0.0;
    for (int jf = 0; jf < nf; ++jf) s = fma(__ldg(hc + jf), tp[jf], s);
    out[it.out_off + (it.c0 + cl) + nijkl * (sab + (long long)nsab * scd)] = s;
  }
}

// ---------------------------------------------------------------- launch
using KernelFn = void (*)(const EriItem*, const DPair*, const double*, int, const double*, const double*, RysArgs,
                          double*, int);

template <int NAB, int NCD>
static KernelFn get_kernel() {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(eri_kernel<NAB, NCD>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  return eri_kernel<NAB, NCD>;
}

template <int NAB>
static KernelFn pick_ncd(int ncd) {
  switch (ncd) {
    case 0: return get_kernel<NAB, 0>();
    case 1: return get_kernel<NAB, 1>();
    case 2: return get_kernel<NAB, 2>();
    case 3: return get_kernel<NAB, 3>();
    case 4: return get_kernel<NAB, 4>();
    case 5: return get_kernel<NAB, 5>();
    case 6: return get_kernel<NAB, 6>();
  }
  return nullptr;
}

static KernelFn pick(int nab, int ncd) {
  switch (nab) {
    case 0: return pick_ncd<0>(ncd);
    case 1: return pick_ncd<1>(ncd);
    case 2: return pick_ncd<2>(ncd);
    case 3: return pick_ncd<3>(ncd);
    case 4: return pick_ncd<4>(ncd);
    case 5: return pick_ncd<5>(ncd);
    case 6: return pick_ncd<6>(ncd);
  }
  return nullptr;
}

// shared-memory plan for one class: NP primitive quartets per chunk and the
// dynamic shared-memory bytes (acc | cf | G | max(E, HRR temp)).
size_t eri_smem_plan(int nab, int ncd, int max_accd, int max_nef, int max_tmp, int& NP) {
  const int NR = (nab + ncd) / 2 + 1;
  const int G1 = NR * (nab + 1) * (ncd + 1);
  const size_t budget = 224 * 1024 / 8;  // doubles
  size_t total = 0;
  int np = 256;
  for (; np >= 1; --np) {
    total = (size_t)max_accd + (size_t)np * (NR * 10 + 3 * G1) + std::max((size_t)np * max_nef, (size_t)max_tmp);
    if (total <= budget) break;
  }
  if (np < 1) { NP = 0; return 0; }
  NP = np;
  return 8 * total;
}

int eri_launch_class(Handle* h, const EriItem* d_items, int nitems, int nab, int ncd, int NP, size_t smem, double* out,
                     cudaStream_t st) {
  init_cart_table();
  KernelFn k = pick(nab, ncd);
  if (!k) return 2;
  RysArgs ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  k<<<nitems, 256, smem, st>>>(d_items, h->d_pairs, h->d_prim, h->tot_np, h->d_coef, h->d_hrr, ra, out, NP);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // namespace mg
