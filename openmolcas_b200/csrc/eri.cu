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

// Threads of one quartet group synchronise on their own named barrier
// (id 1 + group); a group of 32 is one warp.
__device__ __forceinline__ void group_sync(int g, int tpq) {
  if (tpq == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(tpq) : "memory");
  }
}

template <int NAB, int NCD>
__global__ void __launch_bounds__(256, 3) eri_kernel(const EriItem* __restrict__ items, int nitems,
                                                  const DPair* __restrict__ pairs, const double* __restrict__ prim,
                                                  int tot_np, const double* __restrict__ coef,
                                                  const double* __restrict__ hrr, RysArgs ra, double* __restrict__ out,
                                                  int PAB, int PCD, int tpq, int gsm) {
  constexpr int NR = (NAB + NCD) / 2 + 1;
  constexpr int NI = NAB + 1, NJ = NCD + 1;
  constexpr int G1 = NR * NI * NJ;  // one direction
  constexpr int NCF = 10;
  extern __shared__ double smem_all[];
  const int g = threadIdx.x / tpq;
  const int item = blockIdx.x * (blockDim.x / tpq) + g;
  if (item >= nitems) return;  // whole group leaves; no other group waits on it
  double* sm = smem_all + (size_t)g * gsm;
  const EriItem it = items[item];
  const DPair& P = pairs[it.p];
  const DPair& Q = pairs[it.q];
  const int npab = P.np, npcd = Q.np;
  const int nij = P.nci * P.ncj;
  const int ne = P.ne, nf = Q.ne, nef = ne * nf;
  const int nklc = it.c1 - it.c0;  // ket contracted-pair range [c0, c1)
  const int nacc = nij * nklc * nef;
  const int eoff = P.emin * (P.emin + 1) * (P.emin + 2) / 6;
  const int foff = Q.emin * (Q.emin + 1) * (Q.emin + 2) / 6;
  const int NT = PAB * PCD;
  // shared layout: acc | Cab | Ccd | { X | cf | G | E }  (HRR temp reuses {})
  double* acc = sm;
  double* Cab = acc + nacc;
  double* Ccd = Cab + nij * npab;
  double* X = Ccd + nklc * npcd;
  double* cf = X + nij * PCD * nef;
  double* G = cf + NT * NR * NCF;
  double* E = G + NT * 3 * G1;
  const int tid = threadIdx.x - g * tpq, nth = tpq;
  for (int o = tid; o < nacc; o += nth) acc[o] = 0.0;
  for (int o = tid; o < nij * npab; o += nth) Cab[o] = coef[P.coef_off + o];
  for (int o = tid; o < nklc * npcd; o += nth) Ccd[o] = coef[Q.coef_off + (size_t)it.c0 * npcd + o];
  const double Ap0 = P.Ap[0], Ap1 = P.Ap[1], Ap2 = P.Ap[2];
  const double Cp0 = Q.Ap[0], Cp1 = Q.Ap[1], Cp2 = Q.Ap[2];
  for (int pcd0 = 0; pcd0 < npcd; pcd0 += PCD) {
    const int npc = min(PCD, npcd - pcd0);
    group_sync(g, tpq);
    for (int o = tid; o < nij * PCD * nef; o += nth) X[o] = 0.0;
    for (int pab0 = 0; pab0 < npab; pab0 += PAB) {
      const int npa = min(PAB, npab - pab0);
      const int nt = npa * npc;
      group_sync(g, tpq);
      // ---- 1a: roots and recursion coefficients (t = pa + npa * pc)
      for (int t = tid; t < nt; t += nth) {
        const int pc = t / npa, pa = t - pc * npa;
        const int ia = P.prim_off + pab0 + pa, ic = Q.prim_off + pcd0 + pc;
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
      group_sync(g, tpq);
      // ---- 1b: 2D recursion per (quartet, root, direction)
      if (NI * NJ > 1) {
        for (int job = tid; job < nt * NR * 3; job += nth) {
          const int d = job % 3, tr = job / 3, r = tr % NR, t = tr / NR;
          const double* c = cf + (t * NR + r) * NCF;
          const double B00 = c[0], B10 = c[1], B01 = c[2], C00 = c[3 + d], D00 = c[6 + d];
          // recursion written straight to shared memory (keeps registers low)
          double* gg = G + (t * 3 + d) * G1 + r * NI * NJ;
          gg[0] = d == 2 ? c[9] : 1.0;
          if (NI > 1) gg[NJ] = C00 * gg[0];
          for (int i = 1; i < NI - 1; ++i) gg[(i + 1) * NJ] = C00 * gg[i * NJ] + i * B10 * gg[(i - 1) * NJ];
          for (int j = 0; j < NJ - 1; ++j)
            for (int i = 0; i < NI; ++i) {
              double v = D00 * gg[i * NJ + j];
              if (j > 0) v += j * B01 * gg[i * NJ + j - 1];
              if (i > 0) v += i * B00 * gg[(i - 1) * NJ + j];
              gg[i * NJ + j + 1] = v;
            }
        }
        group_sync(g, tpq);
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
      } else {
        // (ss|ss): [00|00] = w * prefactor, no recursion
        for (int t = tid; t < nt; t += nth) E[t] = cf[t * NR * NCF + 9];
      }
      group_sync(g, tpq);
      // ---- 2b1: bra half-transform  X[ij][pc][ef] += sum_pa Cab[ij][pa] E[pa,pc][ef]
      for (int o = tid; o < nij * npc * nef; o += nth) {
        const int ef = o % nef, r1 = o / nef, pc = r1 % npc, ij = r1 / npc;
        const double* ca = Cab + ij * npab + pab0;
        const double* e = E + (size_t)pc * npa * nef + ef;
        double s = 0.0;
        for (int pa = 0; pa < npa; ++pa) s = fma(ca[pa], e[pa * nef], s);
        X[ef + nef * (pc + PCD * ij)] += s;
      }
    }
    group_sync(g, tpq);
    // ---- 2b2: ket half-transform  acc[ij][kl][ef] += sum_pc Ccd[kl][pc] X[ij][pc][ef]
    for (int o = tid; o < nacc; o += nth) {
      const int ef = o % nef, r1 = o / nef, ij = r1 % nij, klc = r1 / nij;
      const double* cc = Ccd + klc * npcd + pcd0;
      const double* xx = X + ef + nef * PCD * ij;
      double s = 0.0;
      for (int pc = 0; pc < npc; ++pc) s = fma(cc[pc], xx[nef * pc], s);
      acc[o] += s;
    }
  }
  group_sync(g, tpq);
  // ---- 3: HRR + spherical, bra then ket
  const int nc = nij * nklc;
  const int nsab = P.nsa * P.nsb, nscd = Q.nsa * Q.nsb;
  const double* Hab = hrr + P.hrr_off;
  const double* Hcd = hrr + Q.hrr_off;
  double* tmp = X;  // nc * nsab * nf
  for (int o = tid; o < nc * nsab * nf; o += nth) {
    const int jf = o % nf, r1 = o / nf, sab = r1 % nsab, cl = r1 / nsab;
    const double* a = acc + cl * nef + jf * ne;
    const double* hc = Hab + (size_t)sab * ne;
    double s = 0.0;
    for (int ie = 0; ie < ne; ++ie) s = fma(__ldg(hc + ie), a[ie], s);
    tmp[o] = s;
  }
  group_sync(g, tpq);
  const long long nijkl = (long long)nij * Q.nci * Q.ncj;
  const long long cbase = (long long)nij * it.c0;
  for (int o = tid; o < nc * nsab * nscd; o += nth) {
    const int cl = o % nc, r1 = o / nc, sab = r1 % nsab, scd = r1 / nsab;
    const double* tp = tmp + ((size_t)cl * nsab + sab) * nf;
    const double* hc = Hcd + (size_t)scd * nf;
    double s = 0.0;
    for (int jf = 0; jf < nf; ++jf) s = fma(__ldg(hc + jf), tp[jf], s);
    out[it.out_off + cbase + cl + nijkl * (sab + (long long)nsab * scd)] = s;
  }
}

// ---------------------------------------------------------------- launch
using KernelFn = void (*)(const EriItem*, int, const DPair*, const double*, int, const double*, const double*,
                          RysArgs, double*, int, int, int, int);

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

// Launch plan of one class.  tpq threads work on one quartet (a group);
// 256/tpq groups share a CTA.  Primitive quartets are processed in tiles of
// PAB bra x PCD ket primitive pairs.  Per-group shared memory (doubles):
//   acc (nij*nklc*nef) | Cab (nij*npab) | Ccd (nklc*npcd) |
//   max( X (nij*PCD*nef) + NT*(NR*10 + 3*G1 + nef),  HRR temp )


ClassPlan eri_plan(int nab, int ncd, const ClassStats& cs) {
  const int NR = (nab + ncd) / 2 + 1;
  const int G1 = NR * (nab + 1) * (ncd + 1);
  ClassPlan pl{0, 0, 0, 0, 0};
  auto need = [&](int pab, int pcd) {
    const size_t nt = (size_t)pab * pcd;
    const size_t tile = (size_t)cs.max_nij * pcd * cs.max_nef + nt * (NR * 10 + 3 * G1 + cs.max_nef);
    return (size_t)cs.max_acc + cs.max_cab + cs.max_ccd + std::max(tile, (size_t)cs.max_tmp);
  };
  // Shared-memory budget per CTA: 72 KB first (3 CTAs per SM), larger only
  // when the class needs it.
  const size_t budgets[3] = {72 * 1024 / 8, 112 * 1024 / 8, 224 * 1024 / 8};
  for (size_t budget : budgets) {
    int pab = std::max(1, std::min(cs.max_npab, 64));
    int pcd = std::max(1, std::min(cs.max_npcd, std::max(1, 256 / pab)));
    const int width = std::max({cs.max_acc, pab * pcd * cs.max_nef / 2, pab * pcd * NR * 3});
    int tpq = width <= 48 ? 32 : width <= 160 ? 64 : width <= 640 ? 128 : 256;
    for (; tpq <= 256; tpq *= 2) {
      const int groups = 256 / tpq;
      const size_t gbudget = budget / groups;
      int a = pab, c = pcd;
      while (need(a, c) > gbudget && (a > 1 || c > 1)) {
        if (c > 1) c = (c + 1) / 2;
        else a = (a + 1) / 2;
      }
      if (need(a, c) <= gbudget) {
        pl.tpq = tpq;
        pl.PAB = a;
        pl.PCD = c;
        pl.gsm = (int)((need(a, c) + 1) & ~(size_t)1);
        pl.smem = 8 * (size_t)pl.gsm * groups;
        return pl;
      }
    }
  }
  return pl;  // PAB == 0: does not fit
}

int eri_launch_class(Handle* h, const EriItem* d_items, int nitems, int nab, int ncd, const ClassPlan& pl, double* out,
                     cudaStream_t st) {
  init_cart_table();
  KernelFn k = pick(nab, ncd);
  if (!k) return 2;
  RysArgs ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  const int groups = 256 / pl.tpq;
  const int nblk = (nitems + groups - 1) / groups;
  k<<<nblk, 256, pl.smem, st>>>(d_items, nitems, h->d_pairs, h->d_prim, h->tot_np, h->d_coef, h->d_hrr, ra, out, pl.PAB,
                                pl.PCD, pl.tpq, pl.gsm);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

}  // namespace mg
