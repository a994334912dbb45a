// Two-electron nuclear gradient (FP64) -- the adjoint of the ERI kernel.
//
// Restates the reference path Drvg1 -> Eval_g1_ijkl -> TwoEl_g -> Rysg1
// (alaska/drvg1.F90:15, alaska_util/eval_g1_ijkl.F90:15, twoel_g.F90:15,
// rys_util/rysg1.F90:91-288):
//   * 2-PDM of a closed-shell determinant, PGet1 (integral_util/pget1.F90:
//     66-106): G_ijkl = D_ij D_kl - 1/4 (D_ik D_jl + D_il D_jk), built per
//     shell quartet from D in shared memory, back-transformed spherical ->
//     Cartesian (SphCr1/SphCr2, twoel_g.F90:328-340);
//   * de-contraction to each primitive quartet (Tcrtnc, twoel_g.F90:390);
//   * Rys roots for l_tot + 1 (nRys = (sum l + 3)/2, rysg1.F90:91), 2D
//     recursion, 2D-level HRR (HRR2Da/HRR2Db), derivative 2D integrals
//     2a I(a+1) - a I(a-1) (Rys2Dg), contraction with the 2-PDM (Assg1);
//   * translational invariance gives the fourth centre (Distg1), the
//     gradient is scaled by 1/2 (alaska.F90:236) and by the permutational
//     degeneracy of the unique quartet.
// Nothing is stored: integrals are recomputed primitive quartet by primitive
// quartet and contracted on the fly (the "hand-written adjoint").
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mg_internal.h"

namespace mg {

struct RysArgsG {
  RysMeta m[MG_MAX_RYS];
  const double* tab;
};


// Cartesian -> spherical matrices (column m, row Cartesian) for l = 0..3,
// C3 Cartesian order; offsets c_sph_off[l].
__constant__ double c_sph[1 + 9 + 30 + 70];
__constant__ int c_sph_off[4];
__constant__ unsigned char c_cartg[120][3];
// binomial coefficients C(n, k), n, k <= 8
__constant__ double c_binom[9][9];

static void init_grad_tables(const Handle* h) {
  static bool done = false;
  if (done) return;
  std::vector<double> s;
  int off[4];
  for (int l = 0; l <= 3; ++l) {
    off[l] = s.size();
    s.insert(s.end(), h->sph[l].begin(), h->sph[l].end());
  }
  cudaMemcpyToSymbol(c_sph, s.data(), sizeof(double) * s.size());
  cudaMemcpyToSymbol(c_sph_off, off, sizeof(off));
  unsigned char t[120][3];
  int k = 0;
  for (int l = 0; l <= 7; ++l)
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) {
        t[k][0] = lx; t[k][1] = ly; t[k][2] = l - lx - ly;
        ++k;
      }
  cudaMemcpyToSymbol(c_cartg, t, sizeof(t));
  double bn[9][9] = {};
  for (int n = 0; n <= 8; ++n) {
    bn[n][0] = 1.0;
    for (int k = 1; k <= n; ++k) bn[n][k] = bn[n][k - 1] * (n - k + 1) / k;
  }
  cudaMemcpyToSymbol(c_binom, bn, sizeof(bn));
  done = true;
}

__device__ __forceinline__ void gsync(int g, int tpq) {
  if (tpq == 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(tpq) : "memory");
}

__device__ __forceinline__ int d_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__device__ __forceinline__ int d_ncomp(int l) { return l >= 2 ? 2 * l + 1 : d_ncart(l); }
__device__ __forceinline__ int d_ccum(int l) { return l * (l + 1) * (l + 2) / 6; }

// one Rys root/weight of order N at T (table or asymptotic)
template <int N>
__device__ __forceinline__ void rys_one(const RysArgsG& ra, double T, int r, double& x, double& w) {
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

template <int NAB1, int NCD1>
__global__ void __launch_bounds__(256, 3) grad_kernel(const GradItem* __restrict__ items, int nitems,
                                                   const DPair* __restrict__ pairs, const double* __restrict__ prim,
                                                   int tot_np, const double* __restrict__ coef,
                                                   const double* __restrict__ Dm, int nbf, RysArgsG ra,
                                                   double* __restrict__ grad, int tpq, int gsm, int PAB, int PCD,
                                                   int RW) {
  constexpr int NR = (NAB1 + NCD1 + 1) / 2;
  constexpr int NI = NAB1 + 1, NJ = NCD1 + 1;
  extern __shared__ double smem_all[];
  const int g = threadIdx.x / tpq;
  const int item = blockIdx.x * (blockDim.x / tpq) + g;
  if (item >= nitems) return;
  const int tid = threadIdx.x - g * tpq;
  double* sm = smem_all + (size_t)g * gsm;
  const GradItem it = items[item];
  const DPair& P = pairs[it.p];
  const DPair& Q = pairs[it.q];
  const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
  const int nca = d_ncart(la), ncb = d_ncart(lb), ncc = d_ncart(lc), ncd = d_ncart(ld);
  const int nsa = d_ncomp(la), nsb = d_ncomp(lb), nsc = d_ncomp(lc), nsd = d_ncomp(ld);
  const int ncart4 = nca * ncb * ncc * ncd;
  const int nij = it.i1 - it.i0;   // bra contracted pairs [i0, i1)
  const int nklc = it.c1 - it.c0;  // ket contracted pairs [c0, c1)
  const int nc = nij * nklc;
  const bool multi = nc > 1;
  const int npab = P.np, npcd = Q.np;
  const int n1d = (la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
  const int nV = NI * (lc + 2) * (ld + 1);  // ket-transferred 2D integrals per job
  const int scr = NI * NJ + nV;             // G + V per job
  const int NT = PAB * PCD;
  const int CFT = NR * 10 + 4;  // per-quartet coefficient record
  // shared layout: Gam | Cab | Ccd | Y | union{ stage-0 temp | tile: cf, Gp, F, S }
  double* Gam = sm;                            // nc * ncart4, index il + nc * abcd
  double* Cab = Gam + nc * ncart4;             // nij * npab
  double* Ccd = Cab + nij * npab;              // nklc * npcd
  double* Y = Ccd + nklc * npcd;               // nij * PCD * ncart4 (multi only)
  double* U0 = Y + (multi ? nij * PCD * ncart4 : 0);
  double* Tmp = U0;                            // stage-0 temp (nc * ncart4)
  double* cf = U0;                             // NT * CFT
  double* Gp = cf + NT * CFT;                  // NT * ncart4 (multi only)
  double* F = Gp + (multi ? NT * ncart4 : 0);  // NT * RW * 12 * n1d  (RW roots per wave)
  double* S = F + NT * RW * 12 * n1d;          // NT * 3 * RW * scr
  for (int o = tid; o < nij * npab; o += tpq) Cab[o] = coef[P.coef_off + (size_t)it.i0 * npab + o];
  for (int o = tid; o < nklc * npcd; o += tpq) Ccd[o] = coef[Q.coef_off + (size_t)it.c0 * npcd + o];
  // ---- stage 0: contracted 2-PDM (PGet1), spherical, then -> Cartesian
  {
    const int nsp4 = nsa * nsb * nsc * nsd;
    for (int o = tid; o < nc * nsp4; o += tpq) {
      const int il = o % nc, r1 = o / nc;
      const int sa = r1 % nsa, r2 = r1 / nsa, sb = r2 % nsb, r3 = r2 / nsb, sc = r3 % nsc, sd = r3 / nsc;
      const int ij = it.i0 + il % nij, kl = it.c0 + il / nij;
      const int ki = ij % P.nci, kj = ij / P.nci, kk = kl % Q.nci, kq = kl / Q.nci;
      const int pa = P.ao_a + sa * P.nci + ki, pb = P.ao_b + sb * P.ncj + kj;
      const int pc = Q.ao_a + sc * Q.nci + kk, pd = Q.ao_b + sd * Q.ncj + kq;
      Tmp[o] = Dm[(size_t)pa * nbf + pb] * Dm[(size_t)pc * nbf + pd] -
               0.25 * (Dm[(size_t)pa * nbf + pc] * Dm[(size_t)pb * nbf + pd] +
                       Dm[(size_t)pa * nbf + pd] * Dm[(size_t)pb * nbf + pc]);
    }
    gsync(g, tpq);
    const double* Sd = c_sph + c_sph_off[ld];
    const double* Sc = c_sph + c_sph_off[lc];
    const double* Sb = c_sph + c_sph_off[lb];
    const double* Sa = c_sph + c_sph_off[la];
    {  // d: [il][sa][sb][sc][sd] -> [il][sa][sb][sc][cd]   (Tmp -> Gam)
      const int inner = nc * nsa * nsb * nsc;
      for (int o = tid; o < inner * ncd; o += tpq) {
        const int in = o % inner, cd = o / inner;
        double s = 0;
        for (int m = 0; m < nsd; ++m) s = fma(Sd[cd + ncd * m], Tmp[in + inner * m], s);
        Gam[o] = s;
      }
      gsync(g, tpq);
    }
    {  // c  (Gam -> Tmp)
      const int inner = nc * nsa * nsb;
      for (int o = tid; o < inner * ncc * ncd; o += tpq) {
        const int in = o % inner, r1 = o / inner, cc = r1 % ncc, cd = r1 / ncc;
        double s = 0;
        for (int m = 0; m < nsc; ++m) s = fma(Sc[cc + ncc * m], Gam[in + inner * (m + nsc * cd)], s);
        Tmp[o] = s;
      }
      gsync(g, tpq);
    }
    {  // b  (Tmp -> Gam)
      const int inner = nc * nsa;
      const int outer = ncc * ncd;
      for (int o = tid; o < inner * ncb * outer; o += tpq) {
        const int in = o % inner, r1 = o / inner, cb = r1 % ncb, ou = r1 / ncb;
        double s = 0;
        for (int m = 0; m < nsb; ++m) s = fma(Sb[cb + ncb * m], Tmp[in + inner * (m + nsb * ou)], s);
        Gam[o] = s;
      }
      gsync(g, tpq);
    }
    {  // a  (Gam -> Tmp -> Gam)
      const int outer = ncb * ncc * ncd;
      for (int o = tid; o < nc * nca * outer; o += tpq) {
        const int il = o % nc, r1 = o / nc, ca = r1 % nca, ou = r1 / nca;
        double s = 0;
        for (int m = 0; m < nsa; ++m) s = fma(Sa[ca + nca * m], Gam[il + nc * (m + nsa * ou)], s);
        Tmp[o] = s;
      }
      gsync(g, tpq);
      for (int o = tid; o < nc * ncart4; o += tpq) Gam[o] = Tmp[o];
      gsync(g, tpq);
    }
  }
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  const double A0 = P.A[0], A1 = P.A[1], A2 = P.A[2];
  const double C0 = Q.A[0], C1 = Q.A[1], C2 = Q.A[2];
  const double ABx[3] = {P.A[0] - P.B[0], P.A[1] - P.B[1], P.A[2] - P.B[2]};
  const double CDx[3] = {Q.A[0] - Q.B[0], Q.A[1] - Q.B[1], Q.A[2] - Q.B[2]};
  const int ca0 = d_ccum(la), cb0 = d_ccum(lb), cc0 = d_ccum(lc), cd0 = d_ccum(ld);
  for (int pcd0 = 0; pcd0 < npcd; pcd0 += PCD) {
    const int npc = min(PCD, npcd - pcd0);
    gsync(g, tpq);
    // ---- ket half-transform of the 2-PDM: Y[ij][pc][abcd] = sum_kl Ccd[kl][pc] Gam[ij,kl][abcd]
    if (multi) {
      for (int o = tid; o < nij * npc * ncart4; o += tpq) {
        const int ij = o % nij, r1 = o / nij, pc = r1 % npc, abcd = r1 / npc;
        double s = 0.0;
        for (int klc = 0; klc < nklc; ++klc) s = fma(Ccd[klc * npcd + pcd0 + pc], Gam[ij + nij * klc + nc * abcd], s);
        Y[ij + nij * (pc + PCD * abcd)] = s;
      }
    }
    for (int pab0 = 0; pab0 < npab; pab0 += PAB) {
      const int npa = min(PAB, npab - pab0);
      const int nt = npa * npc;
      gsync(g, tpq);
      // ---- (1) roots: one (quartet, root) per thread
      for (int job = tid; job < nt * NR; job += tpq) {
        const int r = job % NR, t = job / NR;
        const int pc = t / npa, pa = t - pc * npa;
        const int ia = P.prim_off + pab0 + pa, ic = Q.prim_off + pcd0 + pc;
        const double zeta = prim[ia], eta = prim[ic];
        const double px = prim[2 * tot_np + ia], py = prim[3 * tot_np + ia], pz = prim[4 * tot_np + ia];
        const double qx = prim[2 * tot_np + ic], qy = prim[3 * tot_np + ic], qz = prim[4 * tot_np + ic];
        const double ze = zeta + eta, zei = 1.0 / ze, rho = zeta * eta * zei;
        const double dx = px - qx, dy = py - qy, dz = pz - qz;
        const double T = rho * (dx * dx + dy * dy + dz * dz);
        const double fact = prim[tot_np + ia] * prim[tot_np + ic] * sqrt(zei);
        double x, w;
        rys_one<NR>(ra, T, r, x, w);
        const double U2 = x * zei;
        double* c = cf + t * CFT + r * 10;
        c[0] = 0.5 * U2;
        c[1] = 0.5 * (1.0 - U2 * eta) / zeta;
        c[2] = 0.5 * (1.0 - U2 * zeta) / eta;
        c[3] = px - A0 - eta * U2 * dx;
        c[4] = py - A1 - eta * U2 * dy;
        c[5] = pz - A2 - eta * U2 * dz;
        c[6] = qx - C0 + zeta * U2 * dx;
        c[7] = qy - C1 + zeta * U2 * dy;
        c[8] = qz - C2 + zeta * U2 * dz;
        c[9] = w * fact;
        if (r == 0) {
          double* e = cf + t * CFT + NR * 10;
          e[0] = 2.0 * prim[5 * tot_np + ia];         // 2 alpha
          e[1] = 2.0 * prim[6 * tot_np + ia];         // 2 beta
          e[2] = 2.0 * prim[5 * tot_np + ic];         // 2 gamma
          e[3] = Cab[pab0 + pa] * Ccd[pcd0 + pc];     // single-contraction coefficient
        }
      }
      // ---- (3) primitive 2-PDM (Tcrtnc) by the bra half-transform
      if (multi) {
        for (int o = tid; o < nt * ncart4; o += tpq) {
          const int abcd = o % ncart4, t = o / ncart4;
          const int pc = t / npa, pa = t - pc * npa;
          const double* y = Y + nij * (pc + PCD * abcd);
          double s = 0.0;
          for (int ij = 0; ij < nij; ++ij) s = fma(Cab[ij * npab + pab0 + pa], y[ij], s);
          Gp[t * ncart4 + abcd] = s;
        }
      }
      gsync(g, tpq);
      for (int r0 = 0; r0 < NR; r0 += RW) {
      const int nrw = min(RW, NR - r0);
      // ---- (2a) 2D recursion per (quartet, root, direction): G[e][f], e at A, f at C
      for (int job = tid; job < nt * nrw * 3; job += tpq) {
        const int d = job % 3, tr = job / 3, rl = tr % nrw, t = tr / nrw, r = r0 + rl;
        const double* c = cf + t * CFT + r * 10;
        const double B00 = c[0], B10 = c[1], B01 = c[2], C00 = c[3 + d], D00 = c[6 + d];
        double* G = S + (size_t)job * scr;
        G[0] = d == 2 ? c[9] : 1.0;
        if (NI > 1) G[NJ] = C00 * G[0];
        for (int i = 1; i < NI - 1; ++i) G[(i + 1) * NJ] = C00 * G[i * NJ] + i * B10 * G[(i - 1) * NJ];
        for (int j = 0; j < NJ - 1; ++j)
          for (int i = 0; i < NI; ++i) {
            double v = D00 * G[i * NJ + j];
            if (j > 0) v += j * B01 * G[i * NJ + j - 1];
            if (i > 0) v += i * B00 * G[(i - 1) * NJ + j];
            G[i * NJ + j + 1] = v;
          }
      }
      gsync(g, tpq);
      // ---- (2b) ket 2D-level HRR (HRR2Db): V[e][c][d] = sum_l C(d,l) CD^(d-l) G[e][c+l]
      for (int o = tid; o < nt * nrw * 3 * nV; o += tpq) {
        const int v = o % nV, job = o / nV, d = job % 3;
        const int e = v % NI, r1 = v / NI, cc = r1 % (lc + 2), dd = r1 / (lc + 2);
        double* Gj = S + (size_t)job * scr;
        double out = 0.0;
        if (cc + dd <= NCD1) {
          const double cdv = CDx[d];
          const double* gr = Gj + e * NJ + cc;
          double pl = 1.0;
          for (int l = dd; l >= 0; --l) {
            out = fma(c_binom[dd][l] * pl, gr[l], out);
            pl *= cdv;
          }
        }
        Gj[NI * NJ + v] = out;
      }
      gsync(g, tpq);
      // ---- (2c) bra 2D-level HRR (HRR2Da) folded into the derivative factors (Rys2Dg):
      //      U(a,b,c,d) = sum_k C(b,k) AB^(b-k) V[a+k][c][d];  F = U, 2a U(a+1) - a U(a-1), ...
      for (int o = tid; o < nt * nrw * 3 * n1d; o += tpq) {
        const int e1 = o % n1d, job = o / n1d, d = job % 3, t = job / 3 / nrw;
        const int a = e1 % (la + 1), r1 = e1 / (la + 1), b = r1 % (lb + 1), r2 = r1 / (lb + 1);
        const int cc = r2 % (lc + 1), dd = r2 / (lc + 1);
        const double* Vj = S + (size_t)job * scr + NI * NJ;
        const double ab = ABx[d];
        auto U = [&](int ua, int ub, int uc) {
          const double* V = Vj + uc * NI + dd * NI * (lc + 2);
          double sum = 0.0, pk = 1.0;
          for (int k = ub; k >= 0; --k) {
            sum = fma(c_binom[ub][k] * pk, V[ua + k], sum);
            pk *= ab;
          }
          return sum;
        };
        const double* e = cf + t * CFT + NR * 10;
        double* Fo = F + (size_t)job * 4 * n1d;
        Fo[e1] = U(a, b, cc);
        Fo[n1d + e1] = e[0] * U(a + 1, b, cc) - (a ? a * U(a - 1, b, cc) : 0.0);
        Fo[2 * n1d + e1] = e[1] * U(a, b + 1, cc) - (b ? b * U(a, b - 1, cc) : 0.0);
        Fo[3 * n1d + e1] = e[2] * U(a, b, cc + 1) - (cc ? cc * U(a, b, cc - 1) : 0.0);
      }
      gsync(g, tpq);
      // ---- (4) Assg1: sum over Cartesian components and roots
      for (int o = tid; o < nt * ncart4; o += tpq) {
        const int abcd = o % ncart4, t = o / ncart4;
        const double gm = multi ? Gp[t * ncart4 + abcd] : cf[t * CFT + NR * 10 + 3] * Gam[abcd];
        if (gm == 0.0) continue;
        const int ca = abcd % nca, r1 = abcd / nca, cb = r1 % ncb, r2 = r1 / ncb, cc = r2 % ncc, cd = r2 / ncc;
        const unsigned char* ea = c_cartg[ca0 + ca];
        const unsigned char* eb = c_cartg[cb0 + cb];
        const unsigned char* ec = c_cartg[cc0 + cc];
        const unsigned char* ed = c_cartg[cd0 + cd];
        int idx[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) idx[d] = ea[d] + (la + 1) * (eb[d] + (lb + 1) * (ec[d] + (lc + 1) * ed[d]));
        for (int rl = 0; rl < nrw; ++rl) {
          const double* Fb = F + (size_t)(t * nrw + rl) * 3 * 4 * n1d;
          const double* Fx = Fb + idx[0];
          const double* Fy = Fb + 4 * n1d + idx[1];
          const double* Fz = Fb + 8 * n1d + idx[2];
          const double X = Fx[0], Yv = Fy[0], Z = Fz[0];
          const double gyz = gm * Yv * Z, gxz = gm * X * Z, gxy = gm * X * Yv;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            acc[3 * k + 0] = fma(gyz, Fx[(k + 1) * n1d], acc[3 * k + 0]);
            acc[3 * k + 1] = fma(gxz, Fy[(k + 1) * n1d], acc[3 * k + 1]);
            acc[3 * k + 2] = fma(gxy, Fz[(k + 1) * n1d], acc[3 * k + 2]);
          }
        }
      }
      gsync(g, tpq);
      }  // root waves
    }
  }
  gsync(g, tpq);
  // ---- reduce over the group, distribute to atoms (Distg1)
  double* red = U0;  // tpq/32 * 9 doubles
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    double v = acc[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((tid & 31) == 0) red[(tid >> 5) * 9 + k] = v;
  }
  gsync(g, tpq);
  if (tid < 9) {
    double v = 0.0;
    for (int w = 0; w < tpq / 32; ++w) v += red[w * 9 + tid];
    v *= it.scale;
    const int X = tid / 3, d = tid % 3;
    const int atom = X == 0 ? P.atom_a : X == 1 ? P.atom_b : Q.atom_a;
    atomicAdd(&grad[3 * atom + d], v);
    atomicAdd(&grad[3 * Q.atom_b + d], -v);  // translational invariance
  }
}

// ------------------------------------------------------------------ launch
using GradFn = void (*)(const GradItem*, int, const DPair*, const double*, int, const double*, const double*, int,
                        RysArgsG, double*, int, int, int, int, int);

template <int A, int B>
static GradFn gk() {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(grad_kernel<A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr = true;
  }
  return grad_kernel<A, B>;
}
template <int A>
static GradFn gk_b(int b) {
  switch (b) {
    case 1: return gk<A, 1>();
    case 2: return gk<A, 2>();
    case 3: return gk<A, 3>();
    case 4: return gk<A, 4>();
    case 5: return gk<A, 5>();
    case 6: return gk<A, 6>();
    case 7: return gk<A, 7>();
  }
  return nullptr;
}
static GradFn pick_grad(int a, int b) {
  switch (a) {
    case 1: return gk_b<1>(b);
    case 2: return gk_b<2>(b);
    case 3: return gk_b<3>(b);
    case 4: return gk_b<4>(b);
    case 5: return gk_b<5>(b);
    case 6: return gk_b<6>(b);
    case 7: return gk_b<7>(b);
  }
  return nullptr;
}


// Per-group shared memory (doubles) of one work item with PAB x PCD tiles:
//   Gam + Cab + Ccd + Y + max(stage-0 temp, tile (cf + Gp + F + S per quartet))
static size_t grad_group_smem(const DPair& P, const DPair& Q, int nijc, int nklc, int pab, int pcd, int rw) {
  const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
  const int NI = la + lb + 2, NJ = lc + ld + 2;
  const int NR = (la + lb + lc + ld + 3) / 2;
  const size_t ncart4 = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  const size_t nsp4 = (size_t)ncomp(la) * ncomp(lb) * ncomp(lc) * ncomp(ld);
  const size_t n1d = (size_t)(la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
  const size_t scr = (size_t)NI * NJ + (size_t)NI * (lc + 2) * (ld + 1);
  const size_t nij = nijc, nc = nij * nklc;
  const bool multi = nc > 1;
  const size_t fixed = nc * ncart4 + nij * P.np + (size_t)nklc * Q.np + (multi ? nij * pcd * ncart4 : 0);
  const size_t nt = (size_t)pab * pcd;
  const size_t w = std::min<size_t>(rw, NR);
  const size_t tile = nt * ((size_t)NR * 10 + 4 + (multi ? ncart4 : 0) + w * 12 * n1d + 3 * w * scr);
  return fixed + std::max({nc * std::max(ncart4, nsp4), tile, (size_t)8 * 9});
}

static inline int c_nab1(int key) { return key / 8; }
static inline int c_ncd1(int key) { return key % 8; }

// Shared-memory target per CTA: ~3 CTAs per SM when the work item allows.
static const size_t kGradCtaBudget = 72 * 1024 / 8;
static const size_t kGradMaxBudget = 224 * 1024 / 8;

int grad_build(Handle* h, double cutint, GradPlan& plan) {
  const int ns = h->sh.size();
  std::vector<std::vector<GradItem>> byc(64);
  struct Mx { int npab = 0, npcd = 0; };
  std::vector<Mx> mx(64);
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      const int p = pair_id(i, j);
      const double tij = h->tmax[(size_t)i * ns + j];
      for (int k = 0; k <= i; ++k)
        for (int l = 0; l <= (k == i ? j : k); ++l) {
          if (tij * h->tmax[(size_t)k * ns + l] < cutint) continue;
          const int q = pair_id(k, l);
          const DPair &P = h->pairs[p], &Q = h->pairs[q];
          // all four on one atom: the gradient contribution vanishes
          if (P.atom_a == P.atom_b && P.atom_a == Q.atom_a && P.atom_a == Q.atom_b) continue;
          const int deg = (i == j ? 1 : 2) * (k == l ? 1 : 2) * (p == q ? 1 : 2);
          const int nkl = Q.nci * Q.ncj, nij = P.nci * P.ncj;
          // chunk the contracted block (kl first, then ij) only when one quartet tile
          // cannot fit at all: every chunk repeats the primitive-quartet work
          int ckl = nkl, cij = nij;
          while ((ckl > 1 || cij > 1) && grad_group_smem(P, Q, cij, ckl, 1, 1, 1) > kGradMaxBudget) {
            if (ckl > 1) ckl = (ckl + 1) / 2;
            else cij = (cij + 1) / 2;
          }
          if (grad_group_smem(P, Q, cij, ckl, 1, 1, 1) > kGradMaxBudget) {
            h->err = "gradient quartet does not fit in shared memory";
            return MG_ERR_ARG;
          }
          const int key = (P.la + P.lb + 1) * 8 + (Q.la + Q.lb + 1);
          Mx& m = mx[key];
          for (int i0 = 0; i0 < nij; i0 += cij)
            for (int c0 = 0; c0 < nkl; c0 += ckl) {
              GradItem it{p, q, c0, std::min(nkl, c0 + ckl), i0, std::min(nij, i0 + cij), 0.5 * deg};
              byc[key].push_back(it);
              m.npab = std::max(m.npab, P.np);
              m.npcd = std::max(m.npcd, Q.np);
            }
        }
    }
  plan.items.clear();
  plan.classes.clear();
  for (int key = 0; key < 64; ++key) {
    if (byc[key].empty()) continue;
    auto& v = byc[key];
    std::stable_sort(v.begin(), v.end(), [&](const GradItem& a, const GradItem& b) {
      return (long long)h->pairs[a.p].np * h->pairs[a.q].np > (long long)h->pairs[b.p].np * h->pairs[b.q].np;
    });
    // tile: largest PAB x PCD (<= 8 x 4 primitive quartets) whose worst item fits the CTA budget
    auto worst = [&](int a, int c, int rw) {
      size_t w = 0;
      for (const GradItem& it : v)
        w = std::max(w, grad_group_smem(h->pairs[it.p], h->pairs[it.q], it.i1 - it.i0, it.c1 - it.c0, a, c, rw));
      return w;
    };
    const int NRc = (c_nab1(key) + c_ncd1(key) + 1) / 2;
    const Mx& m = mx[key];
    // widest per-quartet stage of the class (threads that can work at once)
    size_t wmax = 0;
    for (const GradItem& it : v) {
      const DPair &P = h->pairs[it.p], &Q = h->pairs[it.q];
      const size_t n4 = (size_t)ncart(P.la) * ncart(P.lb) * ncart(Q.la) * ncart(Q.lb);
      const size_t nU = (size_t)(P.la + 2) * (P.lb + 2) * (Q.la + 2) * (Q.lb + 1);
      wmax = std::max({wmax, n4, (size_t)3 * NRc * nU});
    }
    GradClass c;
    c.tpq = 0;
    // try budgets (per CTA) and thread counts per quartet; 256 threads per CTA
    const size_t budgets[3] = {kGradCtaBudget, 112 * 1024 / 8, kGradMaxBudget};
    for (size_t cta : budgets) {
      for (int tpq = wmax <= 64 ? 64 : wmax <= 512 ? 128 : 256; tpq <= 256 && !c.tpq; tpq *= 2) {
        const int groups = 256 / tpq;
        const size_t gb = cta / groups;
        int pab = std::max(1, std::min(m.npab, 8)), pcd = std::max(1, std::min(m.npcd, 4)), rw = NRc;
        size_t need = worst(pab, pcd, rw);
        while (need > gb && (pab > 1 || pcd > 1 || rw > 1)) {
          if (pcd > 1) pcd = (pcd + 1) / 2;
          else if (pab > 1) pab = (pab + 1) / 2;
          else --rw;
          need = worst(pab, pcd, rw);
        }
        if (need <= gb) {
          c.tpq = tpq;
          c.groups = groups;
          c.gsm = (int)((need + 1) & ~(size_t)1);
          c.rw = rw;
          c.pab = pab;
          c.pcd = pcd;
        }
      }
      if (c.tpq) break;
    }
    if (!c.tpq) { h->err = "gradient class does not fit in shared memory"; return MG_ERR_ARG; }
    c.nab1 = key / 8;
    c.ncd1 = key % 8;
    c.begin = plan.items.size();
    c.count = v.size();
    plan.items.insert(plan.items.end(), v.begin(), v.end());
    plan.classes.push_back(c);
  }
  cudaFree(plan.d_items);
  plan.d_items = nullptr;
  if (!plan.items.empty()) {
    if (cudaMalloc(&plan.d_items, sizeof(GradItem) * plan.items.size()) != cudaSuccess) return MG_ERR_MEMORY;
    cudaMemcpy(plan.d_items, plan.items.data(), sizeof(GradItem) * plan.items.size(), cudaMemcpyHostToDevice);
  }
  plan.cutint = cutint;
  return 0;
}

int grad_run(Handle* h, const GradPlan& plan, const double* d_D, double* d_grad, cudaStream_t st) {
  init_grad_tables(h);
  RysArgsG ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * h->natom, st);
  for (const GradClass& c : plan.classes) {
    GradFn k = pick_grad(c.nab1, c.ncd1);
    if (!k) { h->err = "gradient class out of range"; return MG_ERR_ARG; }
    const int nblk = (c.count + c.groups - 1) / c.groups;
    k<<<nblk, c.tpq * c.groups, sizeof(double) * (size_t)c.gsm * c.groups, st>>>(
        plan.d_items + c.begin, c.count, h->d_pairs, h->d_prim, h->tot_np, h->d_coef, d_D, h->nbf, ra, d_grad, c.tpq,
        c.gsm, c.pab, c.pcd, c.rw);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) { h->err = "gradient kernel launch failed"; return MG_ERR_CUDA; }
  }
  return 0;
}

void grad_free(GradPlan* p) {
  if (!p) return;
  cudaFree(p->d_items);
  delete p;
}

// Algorithmic FP64 flop count of a gradient plan (FMA = 2): per primitive
// quartet the Rys roots (2 x 7 FMA per root and weight + 30), per root and
// direction the 2D recursion (4 NI NJ), 2D-level HRR (2 (lb+1) NI NJ +
// 2 (la+2)(lb+2) NJ ld) and derivative factors (8 n1d), the bra half of the
// primitive 2-PDM (2 nij ncart4 when nc > 1) and Assg1 (24 flops per
// Cartesian quartet and root); per work item the 2-PDM, its spherical ->
// Cartesian transform and the ket half of the de-contraction.
double grad_plan_flops(const Handle* h, const GradPlan& plan) {
  double f = 0;
  for (const GradItem& it : plan.items) {
    const DPair &P = h->pairs[it.p], &Q = h->pairs[it.q];
    const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
    const int NI = la + lb + 2, NJ = lc + ld + 2, NR = (la + lb + lc + ld + 3) / 2;
    const double ncart4 = (double)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    const double nsp4 = (double)ncomp(la) * ncomp(lb) * ncomp(lc) * ncomp(ld);
    const double n1d = (double)(la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
    const int nij = it.i1 - it.i0, nklc = it.c1 - it.c0, nc = nij * nklc;
    const double per_prim = NR * 28.0 + 30.0 +
                            3.0 * NR * (4.0 * NI * NJ + 2.0 * (lb + 1) * NI * NJ + 2.0 * (la + 2) * (lb + 2) * NJ * ld +
                                        8.0 * n1d) +
                            (nc > 1 ? 2.0 * nij * ncart4 : 0.0) + 24.0 * ncart4 * NR;
    const double per_item = nc * nsp4 * 8.0 + 2.0 * nc * ncart4 * 4.0 * std::max(ncomp(la), ncomp(ld)) +
                            (nc > 1 ? 2.0 * nc * ncart4 * Q.np : 0.0);
    f += per_prim * (double)P.np * Q.np + per_item;
  }
  return f;
}

}  // namespace mg
