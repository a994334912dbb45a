// Two-electron gradient kernel (FP64), one template instantiated per
// (la+lb+1, lc+ld+1) class; MINB (resident CTAs per SM) sets the threads per
// CTA and the register budget.  The algorithm and its reference anchors are
// described in grad.cu; the instantiations live in grad_k1.cu.
#pragma once
#include <cuda_runtime.h>

#include "kern_common.cuh"

namespace mg {

// Per-CTA table block (doubles), copied from global memory at kernel start:
// Cartesian -> spherical matrices for l = 0..3 (column m, row Cartesian) and
// the Cartesian exponents of l = 0..7 in C3 order packed as
// x | y << 8 | z << 16 (ints).
constexpr int kGTabSph = 0;
constexpr int kGTabCart = 110;  // 120 ints = 60 doubles
constexpr int kGTabD = 170;

struct GradArgs {
  const GradItem* items;
  int nitems;
  const DPair* pairs;
  const double* prim;
  int tot_np;
  const double* coef;
  const double* Dm;
  int nbf;
  const double* gtab;
  double* grad;
  double* scratch;       // per-group global slots: contracted 2-PDM + stage-0 temp
  long long scr_stride;  // doubles per slot
  int* counter;          // work-item counter of this launch (starts at 0)
  int tpq, gsm, PAB, PCD, RW;
  // 2-PDM of PGet1 (integral_util/pget1.F90:66-106):
  //   G = cq D(ab) D(cd) - xq [D(ac) D(bd) + D(ad) D(bc) + Ds(ac) Ds(bd) + Ds(ad) Ds(bc)]
  const double* Ds;  // spin density (open shell) or null
  double cq;         // CoulFac
  double xq;         // ExFac / 4
};

using GradFn = void (*)(GradArgs, RysArgs);
GradFn grad_kernel_m1(int nab1, int ncd1);

// Assg1 for one shell quartet class with la = LA, blocked over the Cartesian
// components of centre A: a thread takes all NCA components that share one
// (b, c, d) component and one primitive quartet, loads the LA + 1 interleaved
// 2D records (I, dA, dB, dC) per direction once and reuses them across the NCA
// components (component 0 is (LA, 0, 0), so the x records start LA before it).
template <int LA>
__device__ __forceinline__ void assg1_a_block(const double* __restrict__ F, const double* __restrict__ Gp,
                                              const int* __restrict__ IX, int nt, int nrest, int St, int Gs, int J4,
                                              int nrw, int tid, int tpq, double* acc) {
  constexpr int NCA = (LA + 1) * (LA + 2) / 2;
  constexpr CartExp<LA> ce{};
  const FDiv fnt = fdiv(nt);
  for (int w = tid; w < nt * nrest; w += tpq) {
    const int rest = fq(w, fnt), t = w - rest * nt;
    const int abcd0 = NCA * rest;
    double gm[NCA];
    bool any = false;
#pragma unroll
    for (int ca = 0; ca < NCA; ++ca) {
      gm[ca] = Gp[t * Gs + abcd0 + ca];
      any |= gm[ca] != 0.0;
    }
    if (!any) continue;
    const int pk = IX[abcd0];
    const int bx = 4 * ((pk & 255) - LA), by = J4 + 4 * ((pk >> 8) & 255), bz = 2 * J4 + 4 * (pk >> 16);
    const double* Fb = F + (size_t)t * St;
    for (int rl = 0; rl < nrw; ++rl, Fb += 3 * J4) {
      double2 X01[LA + 1], X23[LA + 1], Y01[LA + 1], Y23[LA + 1], Z01[LA + 1], Z23[LA + 1];
#pragma unroll
      for (int k = 0; k <= LA; ++k) {
        X01[k] = *reinterpret_cast<const double2*>(Fb + bx + 4 * k);
        X23[k] = *reinterpret_cast<const double2*>(Fb + bx + 4 * k + 2);
        Y01[k] = *reinterpret_cast<const double2*>(Fb + by + 4 * k);
        Y23[k] = *reinterpret_cast<const double2*>(Fb + by + 4 * k + 2);
        Z01[k] = *reinterpret_cast<const double2*>(Fb + bz + 4 * k);
        Z23[k] = *reinterpret_cast<const double2*>(Fb + bz + 4 * k + 2);
      }
#pragma unroll
      for (int ca = 0; ca < NCA; ++ca) {
        const int ax = ce.e[ca][0], ay = ce.e[ca][1], az = ce.e[ca][2];
        const double g = gm[ca];
        const double gyz = g * Y01[ay].x * Z01[az].x, gxz = g * X01[ax].x * Z01[az].x, gxy = g * X01[ax].x * Y01[ay].x;
        acc[0] = fma(gyz, X01[ax].y, acc[0]);
        acc[1] = fma(gxz, Y01[ay].y, acc[1]);
        acc[2] = fma(gxy, Z01[az].y, acc[2]);
        acc[3] = fma(gyz, X23[ax].x, acc[3]);
        acc[4] = fma(gxz, Y23[ay].x, acc[4]);
        acc[5] = fma(gxy, Z23[az].x, acc[5]);
        acc[6] = fma(gyz, X23[ax].y, acc[6]);
        acc[7] = fma(gxz, Y23[ay].y, acc[7]);
        acc[8] = fma(gxy, Z23[az].y, acc[8]);
      }
    }
  }
}

// Persistent kernel: each group of tpq threads takes work items from a
// counter until none are left.  The contracted Cartesian 2-PDM of an item
// (Gam[il][abcd]) and the stage-0 temporaries live in the group's global
// scratch slot (L2 resident); the per-tile data in shared memory.
// Per-group shared layout (doubles, every region starts on an even offset):
//   hdr[8] (AB, CD, item) | Cab | Ccd | Y | union{ reduction | tile: cf | Gp | F | S }
// F holds, per (quartet, root, direction), the 2D integral and its three
// centre derivatives interleaved: F[job * J4 + e1 * 4 + {0: I, 1: dA, 2: dB, 3: dC}],
// J4 = 4 n1d + 2: a job stride of 2 mod 4 doubles shifts each job's 16-byte
// records by an odd number of bank groups, so the jobs that a warp's lane
// segments store at once fall in different banks.
// Threads per CTA of a variant: 512 when one CTA fills the SM (128 registers
// per thread), 256 otherwise.
template <int MINB>
struct GradThreads {
  static constexpr int value = MINB == 1 ? 512 : 256;
};

template <int NAB1, int NCD1, int MINB>
__global__ void __launch_bounds__(GradThreads<MINB>::value, MINB) grad_kernel(const GradArgs a, const RysArgs ra) {
  constexpr int NR = (NAB1 + NCD1 + 1) / 2;
  constexpr int NI = NAB1 + 1, NJ = NCD1 + 1;
  extern __shared__ __align__(16) double smem_all[];
  double* tabs = smem_all;
  for (int o = threadIdx.x; o < kGTabD; o += blockDim.x) tabs[o] = a.gtab[o];
  __syncthreads();
  const int tpq = a.tpq;
  const int g = threadIdx.x / tpq;
  const int tid = threadIdx.x - g * tpq;
  double* sm = smem_all + kGTabD + (size_t)g * a.gsm;
  double* Gg = a.scratch + (size_t)(blockIdx.x * (blockDim.x / tpq) + g) * a.scr_stride;
  int* slot = reinterpret_cast<int*>(sm + 6);
  for (;;) {
  if (tid == 0) *slot = atomicAdd(a.counter, 1);
  gsync(g, tpq);
  const int item = *slot;
  if (item >= a.nitems) break;
  const int* cart = reinterpret_cast<const int*>(tabs + kGTabCart);
  const double* prim = a.prim;
  const int tot_np = a.tot_np;
  const GradItem it = a.items[item];
  const DPair& P = a.pairs[it.p];
  const DPair& Q = a.pairs[it.q];
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
  const int PAB = a.PAB, PCD = a.PCD, RW = a.RW;
  const int NT = PAB * PCD;
  const int CFT = NR * 10 + 5;  // per-quartet coefficient record (odd stride)
  double* hdr = sm;
  double* Cab = hdr + 8;                              // nij * npab
  double* Ccd = Cab + ev2(nij * npab);                // nklc * npcd
  double* Y = Ccd + ev2(nklc * npcd);                 // [ij][pc][abcd] (multi only)
  int* IX = reinterpret_cast<int*>(Y + (multi ? ev2(nij * PCD * ncart4) : 0));  // [abcd] packed 2D indices
  double* U0 = reinterpret_cast<double*>(IX) + ev2((ncart4 + 1) / 2);
  // padded strides: consecutive primitive quartets fall in different bank groups
  const int Gs = ncart4 | 1;                          // Gp row (odd)
  const int J4 = 4 * n1d + 2;                          // F record of one (root, direction) job
  const int St = 3 * RW * J4 + (RW & 1 ? 0 : 2);       // F block of one quartet (= 2 mod 4)
  double* cf = U0;                                    // NT * CFT
  double* Gp = cf + ev2(NT * CFT);                    // [t][abcd] primitive 2-PDM, row stride Gs
  double* F = Gp + ev2(NT * Gs);                      // [t][rl][dir][e1][4], job stride J4, quartet stride St
  double* Gam = Gg;                                   // [il][abcd] (global scratch)
  double* Tmp = Gg + ev2(nc * ncart4);                // stage-0 temp (global scratch)
  if (tid < 3) {
    hdr[tid] = P.A[tid] - P.B[tid];
    hdr[3 + tid] = Q.A[tid] - Q.B[tid];
  }
  for (int o = tid; o < nij * npab; o += tpq) Cab[o] = a.coef[P.coef_off + (size_t)it.i0 * npab + o];
  for (int o = tid; o < nklc * npcd; o += tpq) Ccd[o] = a.coef[Q.coef_off + (size_t)it.c0 * npcd + o];
  // ---- stage 0: contracted 2-PDM (PGet1), spherical, then -> Cartesian
  {
    const double* Dm = a.Dm;
    const size_t nbf = a.nbf;
    const int nsp4 = nsa * nsb * nsc * nsd;
    for (int o = tid; o < nc * nsp4; o += tpq) {
      const int il = o % nc, r1 = o / nc;
      const int sa = r1 % nsa, r2 = r1 / nsa, sb = r2 % nsb, r3 = r2 / nsb, sc = r3 % nsc, sd = r3 / nsc;
      const int ij = it.i0 + il % nij, kl = it.c0 + il / nij;
      const int ki = ij % P.nci, kj = ij / P.nci, kk = kl % Q.nci, kq = kl / Q.nci;
      const int pa = P.ao_a + sa * P.nci + ki, pb = P.ao_b + sb * P.ncj + kj;
      const int pc = Q.ao_a + sc * Q.nci + kk, pd = Q.ao_b + sd * Q.ncj + kq;
      // D is symmetric: index it with the fastest-varying AO (pa, then pb) as the
      // column so that neighbouring threads read neighbouring addresses
      double x = Dm[pc * nbf + pa] * Dm[pd * nbf + pb] + Dm[pd * nbf + pa] * Dm[pc * nbf + pb];
      if (a.Ds) x += a.Ds[pc * nbf + pa] * a.Ds[pd * nbf + pb] + a.Ds[pd * nbf + pa] * a.Ds[pc * nbf + pb];
      Tmp[o] = a.cq * Dm[pb * nbf + pa] * Dm[pd * nbf + pc] - a.xq * x;
    }
    gsync(g, tpq);
    const double* Sd = tabs + kGTabSph + d_sph_off(ld);
    const double* Sc = tabs + kGTabSph + d_sph_off(lc);
    const double* Sb = tabs + kGTabSph + d_sph_off(lb);
    const double* Sa = tabs + kGTabSph + d_sph_off(la);
    // one-index transforms, ping-ponging between the two scratch buffers; s and p
    // shells are Cartesian already (identity), so their passes are skipped
    double* cur = Tmp;
    double* nxt = Gam;
    if (ld >= 2) {  // d: [il][sa][sb][sc][sd] -> [il][sa][sb][sc][cd]
      const int inner = nc * nsa * nsb * nsc;
      for (int o = tid; o < inner * ncd; o += tpq) {
        const int in = o % inner, cd = o / inner;
        double s = 0;
        for (int m = 0; m < nsd; ++m) s = fma(Sd[cd + ncd * m], cur[in + inner * m], s);
        nxt[o] = s;
      }
      gsync(g, tpq);
      double* t = cur; cur = nxt; nxt = t;
    }
    if (lc >= 2) {  // c
      const int inner = nc * nsa * nsb;
      for (int o = tid; o < inner * ncc * ncd; o += tpq) {
        const int in = o % inner, r1 = o / inner, cc = r1 % ncc, cd = r1 / ncc;
        double s = 0;
        for (int m = 0; m < nsc; ++m) s = fma(Sc[cc + ncc * m], cur[in + inner * (m + nsc * cd)], s);
        nxt[o] = s;
      }
      gsync(g, tpq);
      double* t = cur; cur = nxt; nxt = t;
    }
    if (lb >= 2) {  // b
      const int inner = nc * nsa;
      const int outer = ncc * ncd;
      for (int o = tid; o < inner * ncb * outer; o += tpq) {
        const int in = o % inner, r1 = o / inner, cb = r1 % ncb, ou = r1 / ncb;
        double s = 0;
        for (int m = 0; m < nsb; ++m) s = fma(Sb[cb + ncb * m], cur[in + inner * (m + nsb * ou)], s);
        nxt[o] = s;
      }
      gsync(g, tpq);
      double* t = cur; cur = nxt; nxt = t;
    }
    if (la >= 2) {  // a
      const int outer = ncb * ncc * ncd;
      for (int o = tid; o < nc * nca * outer; o += tpq) {
        const int il = o % nc, r1 = o / nc, ca = r1 % nca, ou = r1 / nca;
        double s = 0;
        for (int m = 0; m < nsa; ++m) s = fma(Sa[ca + nca * m], cur[il + nc * (m + nsa * ou)], s);
        nxt[o] = s;
      }
      gsync(g, tpq);
      double* t = cur; cur = nxt; nxt = t;
    }
    for (int o = tid; o < nc * ncart4; o += tpq) {  // transpose to [il][abcd]
      const int il = o / ncart4, abcd = o - il * ncart4;
      nxt[o] = cur[il + nc * abcd];
    }
    Gam = nxt;
    gsync(g, tpq);
  }
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  const int ca0 = d_ccum(la), cb0 = d_ccum(lb), cc0 = d_ccum(lc), cd0 = d_ccum(ld);
  // packed 2D-integral offsets of every Cartesian quartet: x | y << 8 | z << 16
  {
    const FDiv fca = fdiv(nca), fcb = fdiv(ncb), fcc = fdiv(ncc);
    for (int abcd = tid; abcd < ncart4; abcd += tpq) {
      const int r1 = fq(abcd, fca), ca = abcd - r1 * nca;
      const int r2 = fq(r1, fcb), cb = r1 - r2 * ncb;
      const int cd = fq(r2, fcc), cc = r2 - cd * ncc;
      const int ea = cart[ca0 + ca], eb = cart[cb0 + cb], ec = cart[cc0 + cc], ed = cart[cd0 + cd];
      int pk = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int sh = 8 * d;
        pk |= (((ea >> sh) & 255) +
               (la + 1) * (((eb >> sh) & 255) + (lb + 1) * (((ec >> sh) & 255) + (lc + 1) * ((ed >> sh) & 255))))
              << sh;
      }
      IX[abcd] = pk;
    }
  }
  for (int pcd0 = 0; pcd0 < npcd; pcd0 += PCD) {
    const int npc = min(PCD, npcd - pcd0);
    gsync(g, tpq);
    // ---- ket half-transform of the 2-PDM: Y[ij][pc][abcd] = sum_kl Ccd[kl][pc] Gam[ij,kl][abcd];
    //      a thread makes 4 consecutive pc of one (ij, abcd), each Gam load feeds 4 FMAs
    if (multi) {
      const int npc4 = (npc + 3) >> 2;
      const FDiv f4 = fdiv(ncart4), fpc = fdiv(npc4);
      for (int o = tid; o < nij * npc4 * ncart4; o += tpq) {
        const int r1 = fq(o, f4), abcd = o - r1 * ncart4, ij = fq(r1, fpc), pc0 = 4 * (r1 - ij * npc4);
        const double* gm = Gam + (size_t)ij * ncart4 + abcd;
        const double* cc = Ccd + pcd0 + pc0;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int klc = 0; klc < nklc; ++klc) {
          const double gv = gm[(size_t)nij * klc * ncart4];
          const double* ck = cc + klc * npcd;
          s0 = fma(ck[0], gv, s0);
          if (pc0 + 1 < npc) s1 = fma(ck[1], gv, s1);
          if (pc0 + 2 < npc) s2 = fma(ck[2], gv, s2);
          if (pc0 + 3 < npc) s3 = fma(ck[3], gv, s3);
        }
        double* y = Y + abcd + ncart4 * (pc0 + PCD * ij);
        y[0] = s0;
        if (pc0 + 1 < npc) y[ncart4] = s1;
        if (pc0 + 2 < npc) y[2 * ncart4] = s2;
        if (pc0 + 3 < npc) y[3 * ncart4] = s3;
      }
    }
    for (int pab0 = 0; pab0 < npab; pab0 += PAB) {
      const int npa = min(PAB, npab - pab0);
      const int nt = npa * npc;
      const FDiv fnpa = fdiv(npa);
      gsync(g, tpq);
      // ---- (1) roots: one (primitive quartet, root) per thread
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
        double* c = cf + t * CFT + r * 10;
        c[0] = 0.5 * U2;
        c[1] = 0.5 * (1.0 - U2 * eta) * prim[7 * tot_np + ia];
        c[2] = 0.5 * (1.0 - U2 * zeta) * prim[7 * tot_np + ic];
        c[3] = px - P.A[0] - eta * U2 * dx;
        c[4] = py - P.A[1] - eta * U2 * dy;
        c[5] = pz - P.A[2] - eta * U2 * dz;
        c[6] = qx - Q.A[0] + zeta * U2 * dx;
        c[7] = qy - Q.A[1] + zeta * U2 * dy;
        c[8] = qz - Q.A[2] + zeta * U2 * dz;
        c[9] = w * fact;
        if (r == 0) {
          double* e = cf + t * CFT + NR * 10;
          e[0] = 2.0 * prim[5 * tot_np + ia];         // 2 alpha
          e[1] = 2.0 * prim[6 * tot_np + ia];         // 2 beta
          e[2] = 2.0 * prim[5 * tot_np + ic];         // 2 gamma
        }
      }
      // (no barrier: the primitive 2-PDM below reads neither the roots' records nor
      // anything they overwrite, so both stages share one phase)
      // ---- (3) primitive 2-PDM (Tcrtnc): bra half-transform of Y (a thread makes 4
      //      consecutive pa of one (pc, abcd), each Y load feeds 4 FMAs), or the single
      //      contraction coefficient times the contracted 2-PDM
      {
        const int npa4 = (npa + 3) >> 2;
        const FDiv f4 = fdiv(ncart4), fpa = fdiv(npa4);
        for (int o = tid; o < npa4 * npc * ncart4; o += tpq) {
          const int r1 = fq(o, f4), abcd = o - r1 * ncart4, pc = fq(r1, fpa), pa0 = 4 * (r1 - pc * npa4);
          double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
          if (multi) {
            const double* y = Y + abcd + ncart4 * pc;
            const double* ca = Cab + pab0 + pa0;
            for (int ij = 0; ij < nij; ++ij) {
              const double yv = y[(size_t)ncart4 * PCD * ij];
              const double* ci = ca + ij * npab;
              s0 = fma(ci[0], yv, s0);
              if (pa0 + 1 < npa) s1 = fma(ci[1], yv, s1);
              if (pa0 + 2 < npa) s2 = fma(ci[2], yv, s2);
              if (pa0 + 3 < npa) s3 = fma(ci[3], yv, s3);
            }
          } else {
            const double gv = Gam[abcd] * Ccd[pcd0 + pc];
            const double* ca = Cab + pab0 + pa0;
            s0 = ca[0] * gv;
            if (pa0 + 1 < npa) s1 = ca[1] * gv;
            if (pa0 + 2 < npa) s2 = ca[2] * gv;
            if (pa0 + 3 < npa) s3 = ca[3] * gv;
          }
          double* gp = Gp + (size_t)(pa0 + npa * pc) * Gs + abcd;
          gp[0] = s0;
          if (pa0 + 1 < npa) gp[Gs] = s1;
          if (pa0 + 2 < npa) gp[2 * Gs] = s2;
          if (pa0 + 3 < npa) gp[3 * Gs] = s3;
        }
      }
      gsync(g, tpq);
      for (int r0 = 0; r0 < NR; r0 += RW) {
        const int nrw = min(RW, NR - r0);
        const FDiv fnrw = fdiv(nrw);
        // ---- (2) one NI-lane segment of a warp per (quartet, root, direction) job (32/NI jobs
        //      per warp), all in registers:
        //      2D recursion: lane e holds the row G[e][0..NJ-1] and takes G[e-1][j] from its
        //        neighbour,  G[e][j+1] = D00 G[e][j] + j B01 G[e][j-1] + e B00 G[e-1][j];
        //      ket 2D-level HRR (HRR2Db) in the lane:  V[e][c][0] = G[e][c],
        //        V[e][c][d+1] = V[e][c+1][d] + CD V[e][c][d];
        //      bra 2D-level HRR (HRR2Da) across the lanes of the group (a shift along e):
        //        U(a,0) = V[a][c][d],  U(a,b+1) = U(a+1,b) + AB U(a,b);
        //      derivative factors (Rys2Dg): F = U, dA = 2alpha U(a+1,b) - a U(a-1,b),
        //        dB = 2beta U(a,b+1) - b U(a,b-1), dC = the same transfer of
        //        W[a] = 2gamma V[a][c+1][d] - c V[a][c-1][d]
        {
          constexpr int JPW = 32 / NI;  // jobs per warp
          const int njobs = nt * nrw * 3;
          const int lane = tid & 31;
          const int seg = lane / NI, e = lane - seg * NI;  // seg >= JPW: spare lanes
          const int lup = (lane + 31) & 31, ldn = (lane + 1) & 31;
          for (int jb = (tid >> 5) * JPW; jb < njobs; jb += (tpq >> 5) * JPW) {  // warp-uniform trip count
            const bool valid = seg < JPW && jb + seg < njobs;
            const int job = min(jb + seg, njobs - 1);
            const int d = job % 3, tr = job / 3, t = fq(tr, fnrw), rl = tr - t * nrw, r = r0 + rl;
            const double* c = cf + t * CFT + r * 10;
            const double B00 = c[0], B10 = c[1], B01 = c[2], C00 = c[3 + d], D00 = c[6 + d];
            // column 0 by the recursion over e: G[i+1][0] = C00 G[i][0] + i B10 G[i-1][0]
            double gm1 = 0.0, g0 = d == 2 ? c[9] : 1.0;
            for (int i = 0; i < e; ++i) {
              const double gn = fma(i * B10, gm1, C00 * g0);
              gm1 = g0;
              g0 = gn;
            }
            double L[NJ];
            L[0] = g0;
#pragma unroll
            for (int j = 0; j < NJ - 1; ++j) {
              const double up = __shfl_sync(0xffffffffu, L[j], lup);  // G[e-1][j]
              double v = D00 * L[j];
              if (j > 0) v = fma(j * B01, L[j > 0 ? j - 1 : 0], v);
              if (e > 0) v = fma(e * B00, up, v);
              L[j + 1] = v;
            }
            const double cdv = hdr[3 + d], abv = hdr[d];
            const double* ex = cf + t * CFT + NR * 10;
            const double e2a = ex[0], e2b = ex[1], e2c = ex[2];
            double2* Fo = reinterpret_cast<double2*>(F + (size_t)t * St + (size_t)(job - 3 * nrw * t) * J4);
            const bool wr = valid && e <= la;
#pragma unroll
            for (int m = 0; m < NJ; ++m) {  // ket level: L[c] = V[e][c][m]
              if (m > ld) break;
              if (m > 0) {
#pragma unroll
                for (int cc = 0; cc + m < NJ; ++cc) L[cc] = fma(cdv, L[cc], L[cc + 1]);
              }
#pragma unroll
              for (int cc = 0; cc + m + 1 < NJ; ++cc) {
                if (cc > lc) break;
                double u = L[cc];
                double w = e2c * L[cc + 1] - (cc > 0 ? cc * L[cc > 0 ? cc - 1 : 0] : 0.0);
                double uprev = 0.0;
                // U(e-1, 0) from the neighbour once; later levels by the transfer itself,
                // U(e-1, b+1) = U(e, b) + AB U(e-1, b), so each level needs two shuffles
                double ud = __shfl_sync(0xffffffffu, u, lup);
                const int ebase = (la + 1) * (lb + 1) * (cc + (lc + 1) * m);
#pragma unroll
                for (int b = 0; b < NI - 1; ++b) {
                  if (b > lb) break;
                  const double un = __shfl_sync(0xffffffffu, u, ldn);  // U(e+1, b)
                  const double wn = __shfl_sync(0xffffffffu, w, ldn);
                  const double unext = fma(abv, u, un);                       // U(e, b+1)
                  if (wr) {
                    double2 v01, v23;
                    v01.x = u;
                    v01.y = e2a * un - (e > 0 ? e * ud : 0.0);
                    v23.x = e2b * unext - (b > 0 ? b * uprev : 0.0);
                    v23.y = w;
                    const int e1 = e + (la + 1) * b + ebase;
                    Fo[2 * e1] = v01;
                    Fo[2 * e1 + 1] = v23;
                  }
                  ud = fma(abv, ud, u);  // U(e-1, b+1)
                  uprev = u;
                  u = unext;
                  w = fma(abv, w, wn);
                }
              }
            }
          }
        }
        gsync(g, tpq);
        // ---- (4) Assg1: sum over Cartesian components and roots; consecutive threads
        //      take consecutive primitive quartets of one Cartesian quartet (blocked over
        //      the components of centre A for la = 1, 2; over those of centre B when
        //      la = 0, which puts B first in the component order with unit stride)
        const int lblk = la > 0 ? la : lb;
        if (lblk == 1) {
          assg1_a_block<1>(F, Gp, IX, nt, ncart4 / 3, St, Gs, J4, nrw, tid, tpq, acc);
        } else if (lblk == 2) {
          assg1_a_block<2>(F, Gp, IX, nt, ncart4 / 6, St, Gs, J4, nrw, tid, tpq, acc);
        } else {
          const FDiv fnt = fdiv(nt);
          for (int w = tid; w < nt * ncart4; w += tpq) {
            const int abcd = fq(w, fnt), t = w - abcd * nt;
            const double gm = Gp[t * Gs + abcd];
            if (gm == 0.0) continue;
            const int pk = IX[abcd];
            const int i0 = 4 * (pk & 255), i1 = J4 + 4 * ((pk >> 8) & 255), i2 = 2 * J4 + 4 * (pk >> 16);
            const double* Fb = F + (size_t)t * St;
            for (int rl = 0; rl < nrw; ++rl, Fb += 3 * J4) {
              const double2 x01 = *reinterpret_cast<const double2*>(Fb + i0);
              const double2 x23 = *reinterpret_cast<const double2*>(Fb + i0 + 2);
              const double2 y01 = *reinterpret_cast<const double2*>(Fb + i1);
              const double2 y23 = *reinterpret_cast<const double2*>(Fb + i1 + 2);
              const double2 z01 = *reinterpret_cast<const double2*>(Fb + i2);
              const double2 z23 = *reinterpret_cast<const double2*>(Fb + i2 + 2);
              const double gyz = gm * y01.x * z01.x, gxz = gm * x01.x * z01.x, gxy = gm * x01.x * y01.x;
              acc[0] = fma(gyz, x01.y, acc[0]);
              acc[1] = fma(gxz, y01.y, acc[1]);
              acc[2] = fma(gxy, z01.y, acc[2]);
              acc[3] = fma(gyz, x23.x, acc[3]);
              acc[4] = fma(gxz, y23.x, acc[4]);
              acc[5] = fma(gxy, z23.x, acc[5]);
              acc[6] = fma(gyz, x23.y, acc[6]);
              acc[7] = fma(gxz, y23.y, acc[7]);
              acc[8] = fma(gxy, z23.y, acc[8]);
            }
          }
        }
        // the next wave overwrites F; after the last wave the next tile (or chunk, or the
        // final reduction) starts with its own barrier
        if (r0 + RW < NR) gsync(g, tpq);
      }  // root waves
    }
  }
  gsync(g, tpq);
  // ---- reduce over the group, distribute to atoms (Distg1)
  double* red = U0;  // tpq/32 * 9 doubles (<= 144)
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
    atomicAdd(&a.grad[3 * atom + d], v);
    atomicAdd(&a.grad[3 * Q.atom_b + d], -v);  // translational invariance
  }
  gsync(g, tpq);
  }  // work items
}

template <int MINB, int A, int B>
GradFn grad_fn() {
  if (!smem_attr_once((const void*)grad_kernel<A, B, MINB>, 227 * 1024)) return nullptr;
  return grad_kernel<A, B, MINB>;
}
template <int MINB, int A>
GradFn grad_fn_b(int b) {
  switch (b) {
    case 1: return grad_fn<MINB, A, 1>();
    case 2: return grad_fn<MINB, A, 2>();
    case 3: return grad_fn<MINB, A, 3>();
    case 4: return grad_fn<MINB, A, 4>();
    case 5: return grad_fn<MINB, A, 5>();
    case 6: return grad_fn<MINB, A, 6>();
    case 7: return grad_fn<MINB, A, 7>();
  }
  return nullptr;
}
template <int MINB>
GradFn grad_pick(int a, int b) {
  switch (a) {
    case 1: return grad_fn_b<MINB, 1>(b);
    case 2: return grad_fn_b<MINB, 2>(b);
    case 3: return grad_fn_b<MINB, 3>(b);
    case 4: return grad_fn_b<MINB, 4>(b);
    case 5: return grad_fn_b<MINB, 5>(b);
    case 6: return grad_fn_b<MINB, 6>(b);
    case 7: return grad_fn_b<MINB, 7>(b);
  }
  return nullptr;
}

}  // namespace mg
