// FP64 Rys-quadrature ERIs over contracted shell quartets (sm_100a).
//
// Persistent kernel: one 512-thread CTA per SM; groups of tpq threads take
// work items (bra pair, ket pair, range of contracted kl) from a counter.
// Per tile of PAB x PCD primitive quartets:
//   1a  thread per (primitive quartet, root): T, prefactor, Rys root/weight
//       (table lookup), recursion coefficients (TERI teri.F90:51-57, ModU2,
//       vCff2D vcff2d.F90) -> shared memory
//   1b  NI-lane warp segment per (quartet, root, direction): 2D recursion
//       (vRys2D vrys2d.F90), lane e holds row I[e][0..NCD] in registers and
//       takes I[e-1][f] from its neighbour; weight * prefactor folded into z
//   2a  thread per (quartet, f, Cartesian shell of the bra range):
//       [e0|f0] = sum_r Ix Iy Iz  (RysEF), each shell's rows loaded once per
//       root; consecutive lanes on consecutive primitive quartets
//   2b  half-transforms with the general-contraction coefficients (Cntrct)
// then HRR + real-spherical transform with the per-pair matrices
// (HrrMtrx/TnsCtl, hrrmtrx.F90, tnsctl.F90) and the store in the layout of
// Eval_IJKL's AOInt(nijkl, iCmp1..4) (twoel_nosym.F90:372).
#pragma once
#include <cuda_runtime.h>

#include "kern_common.cuh"

namespace mg {

// Per-CTA table block: Cartesian exponents of l = 0..7 in C3 order
// (index_functions.F90 C3_Ind3) packed as x | y << 8 | z << 16.
constexpr int kETabD = 60;  // 120 ints

struct EriArgs {
  const EriItem* items;
  int nitems;
  const DPair* pairs;
  const double* prim;
  int tot_np;
  const double* coef;
  const double* hrr;
  const double* etab;
  double* out;
  int* counter;  // work-item counter of this launch (starts at 0)
  int tpq, gsm, PAB, PCD;
};
using EriFn = void (*)(EriArgs, RysArgs);
EriFn eri_kernel_pick(int nab, int ncd);
constexpr int kEriThreads = 512;

// [e0|f0] of one Cartesian shell L of the bra range for one primitive quartet
// and one ket component f: the L + 1 values of each direction's row are loaded
// once per root and reused across the NCL components of the shell.
// Ib: the quartet's 2D integrals [dir][root][f][e]; fxo/fyo/fzo: f * NI offsets.
template <int L, int NR, int RS, int DS>
__device__ __forceinline__ void ef_shell(const double* __restrict__ Ib, int fxo, int fyo, int fzo,
                                         double* __restrict__ out) {
  constexpr int NCL = (L + 1) * (L + 2) / 2;
  constexpr CartExp<L> ce{};
  double acc[NCL];
#pragma unroll
  for (int c = 0; c < NCL; ++c) acc[c] = 0.0;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const double* px = Ib + r * RS + fxo;
    const double* py = Ib + DS + r * RS + fyo;
    const double* pz = Ib + 2 * DS + r * RS + fzo;
    double X[L + 1], Y[L + 1], Z[L + 1];
#pragma unroll
    for (int k = 0; k <= L; ++k) {
      X[k] = px[k];
      Y[k] = py[k];
      Z[k] = pz[k];
    }
#pragma unroll
    for (int c = 0; c < NCL; ++c) acc[c] = fma(X[ce.e[c][0]] * Y[ce.e[c][1]], Z[ce.e[c][2]], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < NCL; ++c) out[c] = acc[c];
}

// Per-group shared layout (doubles, every region even):
//   hdr[2] | acc | Cab | Ccd | Ft (ints) | union{ HRR temp | X | tile: cf | I | E }
// I holds per primitive quartet [dir][root][f][e] (stride GST, odd); E per
// quartet [ef] (stride nef | 1).
template <int NAB, int NCD>
__global__ void __launch_bounds__(kEriThreads, 1) eri_kernel(const EriArgs a, const RysArgs ra) {
  constexpr int NR = (NAB + NCD) / 2 + 1;
  constexpr int NI = NAB + 1, NJ = NCD + 1;
  constexpr int RS = NJ * NI;           // one root of one direction
  constexpr int DS = NR * RS;           // one direction of one quartet
  constexpr int GST = (3 * DS) | 1;     // quartet stride (odd)
  constexpr int CFS = NR * 10 + 1;      // coefficient record per quartet (odd)
  extern __shared__ __align__(16) double smem_all[];
  for (int o = threadIdx.x; o < kETabD; o += blockDim.x) smem_all[o] = a.etab[o];
  __syncthreads();
  const int* cart = reinterpret_cast<const int*>(smem_all);
  const int tpq = a.tpq;
  const int g = threadIdx.x / tpq;
  const int tid = threadIdx.x - g * tpq;
  double* sm = smem_all + kETabD + (size_t)g * a.gsm;
  int* slot = reinterpret_cast<int*>(sm);
  const double* prim = a.prim;
  const int tot_np = a.tot_np;
  const int PAB = a.PAB, PCD = a.PCD, NT = PAB * PCD;
  for (;;) {
    if (tid == 0) *slot = atomicAdd(a.counter, 1);
    gsync(g, tpq);
    const int item = *slot;
    if (item >= a.nitems) break;
    const EriItem it = a.items[item];
    const DPair& P = a.pairs[it.p];
    const DPair& Q = a.pairs[it.q];
    const int npab = P.np, npcd = Q.np;
    const int nij = P.nci * P.ncj;
    const int ne = P.ne, nf = Q.ne, nef = ne * nf;
    const int Est = nef | 1;
    const int nklc = it.c1 - it.c0;  // ket contracted-pair range [c0, c1)
    const int nacc = nij * nklc * nef;
    double* acc = sm + 2;
    double* Cab = acc + ev2(nacc);
    double* Ccd = Cab + ev2(nij * npab);
    int* Ft = reinterpret_cast<int*>(Ccd + ev2(nklc * npcd));
    double* X = reinterpret_cast<double*>(Ft) + ev2((nf + 1) / 2);
    double* cf = X + ev2(nij * PCD * nef);
    double* I = cf + ev2(NT * CFS);
    double* E = I + NT * GST;
    for (int o = tid; o < nacc; o += tpq) acc[o] = 0.0;
    for (int o = tid; o < nij * npab; o += tpq) Cab[o] = a.coef[P.coef_off + o];
    for (int o = tid; o < nklc * npcd; o += tpq) Ccd[o] = a.coef[Q.coef_off + (size_t)it.c0 * npcd + o];
    {  // packed offsets of the Cartesian f components (f * NI per direction) into one root of I
      const int foff = d_ccum(Q.emin);
      for (int o = tid; o < nf; o += tpq) {
        const int v = cart[foff + o];
        Ft[o] = ((v & 255) * NI) | ((((v >> 8) & 255) * NI) << 8) | (((v >> 16) * NI) << 16);
      }
    }
    const double Ap0 = P.Ap[0], Ap1 = P.Ap[1], Ap2 = P.Ap[2];
    const double Cp0 = Q.Ap[0], Cp1 = Q.Ap[1], Cp2 = Q.Ap[2];
    for (int pcd0 = 0; pcd0 < npcd; pcd0 += PCD) {
      const int npc = min(PCD, npcd - pcd0);
      gsync(g, tpq);
      for (int o = tid; o < nij * PCD * nef; o += tpq) X[o] = 0.0;
      for (int pab0 = 0; pab0 < npab; pab0 += PAB) {
        const int npa = min(PAB, npab - pab0);
        const int nt = npa * npc;
        const FDiv fnpa = fdiv(npa);
        gsync(g, tpq);
        // ---- 1a: roots and recursion coefficients, one (quartet, root) per thread
        for (int job = tid; job < nt * NR; job += tpq) {
          const int t = job / NR, r = job - t * NR;
          const int pc = fq(t, fnpa), pa = t - pc * npa;
          const int ia = P.prim_off + pab0 + pa, ic = Q.prim_off + pcd0 + pc;
          const double zeta = prim[ia], eta = prim[ic];
          const double px = prim[2 * tot_np + ia], py = prim[3 * tot_np + ia], pz = prim[4 * tot_np + ia];
          const double qx = prim[2 * tot_np + ic], qy = prim[3 * tot_np + ic], qz = prim[4 * tot_np + ic];
          const double ze = zeta + eta, zei = 1.0 / ze, rho = zeta * eta * zei;
          const double dx = px - qx, dy = py - qy, dz = pz - qz;
          const double T = rho * (dx * dx + dy * dy + dz * dz);
          double x, w;
          rys_one<NR>(ra, T, r, x, w);
          const double fact = prim[tot_np + ia] * prim[tot_np + ic] * sqrt(zei);
          const double U2 = x * zei;
          double* c = cf + t * CFS + r * 10;
          c[0] = 0.5 * U2;
          c[1] = 0.5 * (1.0 - U2 * eta) * prim[7 * tot_np + ia];   // 1/zeta from the table
          c[2] = 0.5 * (1.0 - U2 * zeta) * prim[7 * tot_np + ic];
          c[3] = px - Ap0 - eta * U2 * dx;
          c[4] = py - Ap1 - eta * U2 * dy;
          c[5] = pz - Ap2 - eta * U2 * dz;
          c[6] = qx - Cp0 + zeta * U2 * dx;
          c[7] = qy - Cp1 + zeta * U2 * dy;
          c[8] = qz - Cp2 + zeta * U2 * dz;
          c[9] = w * fact;
        }
        gsync(g, tpq);
        if (NI * NJ > 1) {
          // ---- 1b: 2D recursion, one NI-lane warp segment per (quartet, root, direction)
          //      (32/NI jobs per warp): I[e][f+1] = D00 I[e][f] + f B01 I[e][f-1] + e B00 I[e-1][f]
          constexpr int JPW = 32 / NI;
          const int njobs = nt * NR * 3;
          const int lane = tid & 31;
          const int seg = lane / NI, e = lane - seg * NI;  // seg >= JPW: spare lanes
          const int lup = (lane + 31) & 31;
          for (int jb = (tid >> 5) * JPW; jb < njobs; jb += (tpq >> 5) * JPW) {  // warp-uniform trip count
            const bool valid = seg < JPW && jb + seg < njobs;
            const int job = min(jb + seg, njobs - 1);
            const int d = job % 3, tr = job / 3, t = tr / NR, r = tr - t * NR;
            const double* c = cf + t * CFS + r * 10;
            const double B00 = c[0], B10 = c[1], B01 = c[2], C00 = c[3 + d], D00 = c[6 + d];
            // column f = 0 by the recursion over e: I[i+1][0] = C00 I[i][0] + i B10 I[i-1][0]
            double gm1 = 0.0, g0 = d == 2 ? c[9] : 1.0;
            for (int i = 0; i < e; ++i) {
              const double gn = fma(i * B10, gm1, C00 * g0);
              gm1 = g0;
              g0 = gn;
            }
            double* Io = I + (size_t)t * GST + d * DS + r * RS + e;
            double L = g0, Lm = 0.0;
            if (valid) Io[0] = L;
#pragma unroll
            for (int j = 0; j < NJ - 1; ++j) {
              const double up = __shfl_sync(0xffffffffu, L, lup);  // I[e-1][j]
              double v = D00 * L;
              if (j > 0) v = fma(j * B01, Lm, v);
              if (e > 0) v = fma(e * B00, up, v);
              Lm = L;
              L = v;
              if (valid) Io[(j + 1) * NI] = v;
            }
          }
          gsync(g, tpq);
          // ---- 2a: [e0|f0] = sum_r Ix Iy Iz, one thread per (quartet, f, bra shell L);
          //      consecutive lanes on consecutive quartets
          {
            const int emin = P.emin, nsh = NAB - emin + 1;
            const int c0 = d_ccum(emin);
            const FDiv fnt = fdiv(nt), fnf = fdiv(nf);
            for (int w = tid; w < nt * nf * nsh; w += tpq) {
              const int u = fq(w, fnt), t = w - u * nt;
              const int s = fq(u, fnf), jf = u - s * nf;
              const int L = emin + s;
              const int pf = Ft[jf];
              const double* Ib = I + (size_t)t * GST;
              double* out = E + (size_t)t * Est + (size_t)ne * jf + (d_ccum(L) - c0);
              const int fxo = pf & 255, fyo = (pf >> 8) & 255, fzo = pf >> 16;
              switch (L) {
#define MG_EF_CASE(LL) \
  case LL:             \
    if (LL <= NAB) ef_shell<(LL <= NAB ? LL : 0), NR, RS, DS>(Ib, fxo, fyo, fzo, out); \
    break;
                MG_EF_CASE(0) MG_EF_CASE(1) MG_EF_CASE(2) MG_EF_CASE(3) MG_EF_CASE(4) MG_EF_CASE(5) MG_EF_CASE(6)
#undef MG_EF_CASE
              }
            }
          }
        } else {
          // (ss|ss): [00|00] = w * prefactor, no recursion
          for (int t = tid; t < nt; t += tpq) E[(size_t)t * Est] = cf[t * CFS + 9];
        }
        gsync(g, tpq);
        // ---- 2b1: bra half-transform  X[ij][pc][ef] += sum_pa Cab[ij][pa] E[pa,pc][ef];
        //      a thread makes 4 consecutive ij of one (pc, ef), each E load feeds 4 FMAs
        {
          const int nij4 = (nij + 3) >> 2;
          const FDiv fnef = fdiv(nef), fnpc = fdiv(npc);
          for (int o = tid; o < nij4 * npc * nef; o += tpq) {
            const int r1 = fq(o, fnef), ef = o - r1 * nef, q = fq(r1, fnpc), pc = r1 - q * npc;
            const int ij0 = 4 * q;
            const double* ca = Cab + ij0 * npab + pab0;
            const double* e = E + (size_t)pc * npa * Est + ef;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            for (int pa = 0; pa < npa; ++pa) {
              const double ev = e[(size_t)pa * Est];
              s0 = fma(ca[pa], ev, s0);
              if (ij0 + 1 < nij) s1 = fma(ca[npab + pa], ev, s1);
              if (ij0 + 2 < nij) s2 = fma(ca[2 * npab + pa], ev, s2);
              if (ij0 + 3 < nij) s3 = fma(ca[3 * npab + pa], ev, s3);
            }
            double* x = X + ef + nef * (pc + PCD * ij0);
            x[0] += s0;
            if (ij0 + 1 < nij) x[nef * PCD] += s1;
            if (ij0 + 2 < nij) x[2 * nef * PCD] += s2;
            if (ij0 + 3 < nij) x[3 * nef * PCD] += s3;
          }
        }
      }
      gsync(g, tpq);
      // ---- 2b2: ket half-transform  acc[kl][ij][ef] += sum_pc Ccd[kl][pc] X[ij][pc][ef];
      //      a thread makes 4 consecutive kl of one (ij, ef), each X load feeds 4 FMAs
      {
        const int nkl4 = (nklc + 3) >> 2;
        const FDiv fnef = fdiv(nef), fnij = fdiv(nij);
        for (int o = tid; o < nkl4 * nij * nef; o += tpq) {
          const int r1 = fq(o, fnef), ef = o - r1 * nef, q = fq(r1, fnij), ij = r1 - q * nij;
          const int kl0 = 4 * q;
          const double* cc = Ccd + kl0 * npcd + pcd0;
          const double* xx = X + ef + nef * PCD * ij;
          double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
          for (int pc = 0; pc < npc; ++pc) {
            const double xv = xx[nef * pc];
            s0 = fma(cc[pc], xv, s0);
            if (kl0 + 1 < nklc) s1 = fma(cc[npcd + pc], xv, s1);
            if (kl0 + 2 < nklc) s2 = fma(cc[2 * npcd + pc], xv, s2);
            if (kl0 + 3 < nklc) s3 = fma(cc[3 * npcd + pc], xv, s3);
          }
          double* ac = acc + (size_t)(kl0 * nij + ij) * nef + ef;
          ac[0] += s0;
          if (kl0 + 1 < nklc) ac[(size_t)nij * nef] += s1;
          if (kl0 + 2 < nklc) ac[(size_t)2 * nij * nef] += s2;
          if (kl0 + 3 < nklc) ac[(size_t)3 * nij * nef] += s3;
        }
      }
    }
    gsync(g, tpq);
    // ---- 3: HRR + spherical, bra then ket
    const int nc = nij * nklc;
    const int nsab = P.nsa * P.nsb, nscd = Q.nsa * Q.nsb;
    const double* Hab = a.hrr + P.hrr_off;
    const double* Hcd = a.hrr + Q.hrr_off;
    double* tmp = X;  // nc * nsab * nf
    {
      const FDiv fnf = fdiv(nf), fsab = fdiv(nsab);
      for (int o = tid; o < nc * nsab * nf; o += tpq) {
        const int r1 = fq(o, fnf), jf = o - r1 * nf, cl = fq(r1, fsab), sab = r1 - cl * nsab;
        const double* av = acc + cl * nef + jf * ne;
        const double* hc = Hab + (size_t)sab * ne;
        double s = 0.0;
        for (int ie = 0; ie < ne; ++ie) s = fma(__ldg(hc + ie), av[ie], s);
        tmp[o] = s;
      }
    }
    gsync(g, tpq);
    {
      const long long nijkl = (long long)nij * Q.nci * Q.ncj;
      const long long cbase = (long long)nij * it.c0;
      const FDiv fnc = fdiv(nc), fsab = fdiv(nsab);
      for (int o = tid; o < nc * nsab * nscd; o += tpq) {
        const int r1 = fq(o, fnc), cl = o - r1 * nc, scd = fq(r1, fsab), sab = r1 - scd * nsab;
        const double* tp = tmp + ((size_t)cl * nsab + sab) * nf;
        const double* hc = Hcd + (size_t)scd * nf;
        double s = 0.0;
        for (int jf = 0; jf < nf; ++jf) s = fma(__ldg(hc + jf), tp[jf], s);
        a.out[it.out_off + cbase + cl + nijkl * (sab + (long long)nsab * scd)] = s;
      }
    }
    gsync(g, tpq);
  }  // work items
}

template <int A, int B>
EriFn eri_fn() {
  if (!smem_attr_once((const void*)eri_kernel<A, B>, 227 * 1024)) return nullptr;
  return eri_kernel<A, B>;
}
template <int A>
EriFn eri_fn_b(int b) {
  switch (b) {
    case 0: return eri_fn<A, 0>();
    case 1: return eri_fn<A, 1>();
    case 2: return eri_fn<A, 2>();
    case 3: return eri_fn<A, 3>();
    case 4: return eri_fn<A, 4>();
    case 5: return eri_fn<A, 5>();
    case 6: return eri_fn<A, 6>();
  }
  return nullptr;
}

}  // namespace mg
