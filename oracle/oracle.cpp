// ORACLE -- test infrastructure only.
//
// CPU FP64 restatement of OpenMolcas's two-electron hot path, used by the
// parity tests, by __graft_entry__.smoke() as the checker and by bench.py as
// the timed CPU baseline ("port").  Nothing in the product library links,
// loads or calls this file.
//
// What it restates (paths relative to the OpenMolcas tree):
//  * Rys roots/weights: evaluated from the project's own fitted table
//    (openmolcas_b200/rys/rys_table.bin), same quantity as
//    src/rys_util/vrysrw.F90:15 + rys22.F90:36-47 (x = t^2, asymptotic
//    Hermite rule above TMax).
//  * Shell-pair data: DoZeta (src/integral_util/dozeta.F90:36-52):
//    zeta = a+b, kappa = sqrt(2) pi^(5/4) exp(-ab/zeta |AB|^2)/zeta, P.
//  * TERI (src/rys_util/teri.F90:51-57), ModU2 (modu2.F90), vCff2D
//    (vcff2d.F90: B00, B10, B01, PAQP, QCPQ), vRys2D (vrys2d.F90: 2D
//    recursion), RysEF (rysef.F90:200-215: [e0|f0] = Fact sum_r Ix Iy Iz).
//  * Contraction with general contraction coefficients (cntrct.F90).
//  * HrrMtrx (src/integral_util/hrrmtrx.F90:61-100): HRR transfer to the
//    centre of higher l, folded with the real-spherical transform; CoorAC
//    choice as twoel_nosym.F90:262-271.
//  * Real_Sphere / Recurse / Ladder / NrmSph
//    (src/integral_util/real_spherical.F90:182-420), Condon-Shortley off
//    (gateway_util/rdctl_seward.F90:74 default CSPF=.false.).
//  * Output layout of Eval_IJKL/TwoEl_NoSym (twoel_nosym.F90:372):
//    AOInt(nijkl, iCmp1, iCmp2, iCmp3, iCmp4), contracted index fastest,
//    i fastest inside ijkl.
//  * Cholesky alg 4 (cholesky_util): Cho_SetPass (cho_setpass.F90:29-47),
//    Cho_GetInt (cho_getint.F90:38-140, MXSHPR), Cho_GetMaxShl
//    (cho_getmaxshl.F90), Cho_Qualify_2 (cho_qualify_2.F90; IALQUA = 2, the
//    default) and Cho_Qualify_1 (cho_qualify_1.F90:26-40), Cho_Dec_Qual
//    (cho_dec_qual.F90:57-83), CD_InCore_1p
//    (cd_incore_1p.F90:33-85), Cho_CompVec (cho_compvec.F90:40-120),
//    Cho_ChkDia_A4 (cho_chkdia_a4.F90:31-62), Cho_SetRed mode 1
//    (cho_setred.F90:72-100), Cho_SetDamp (cho_setdamp.F90).
//  * J/K from Cholesky vectors (fock_util/cho_lk_scf.F90:442-449 for J,
//    :507-830 for K), without LK screening.
//  * Two-electron gradient: Drvg1/TwoEl_g/Rysg1/Assg1
//    (alaska/drvg1.F90, alaska_util/twoel_g.F90, rys_util/rysg1.F90,
//    rys_util/rys2dg.F90, rys_util/assg1.F90) with the PGet1 2-PDM
//    (integral_util/pget1.F90:66-106) and the 1/2 of alaska.F90:236.
//  * Built a second time with -DOR_COUNT_FLOPS (_build/liboracle_count.so),
//    the same loops tally the FP64 operations they execute (or_flops).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <memory>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ------------------------------------------- FLOP tally (instrumented build)
// With -DOR_COUNT_FLOPS every FP64 add, subtract, multiply, divide and square
// root that the restated loops execute is tallied where it is written (a*b + c
// counts 2; a product with a loop index counts 1), per stage; the default
// build compiles the tally away.  Shell-pair data (make_pair) and the HRR
// matrices (hrr_mtrx) are basis set-up and are not counted.
enum FlopStage {
  FS_PRIM,      // per primitive quartet: zeta + eta, rho, |PQ|^2, T, prefactor
  FS_ROOTS,     // Rys roots and weights (table or asymptotic form)
  FS_RYS2D,     // vCff2D + vRys2D coefficients and recursion
  FS_RYSEF,     // [e0|f0] = Fact sum_r Ix Iy Iz
  FS_CONTRACT,  // contraction with the general-contraction coefficients
  FS_HRR,       // HRR + spherical transforms of the contracted block
  FS_TRANSFER,  // gradient: 2D-level HRR transfers (HRR2Da/HRR2Db)
  FS_ASSG1,     // gradient: derivative 2D factors, Assg1 products, Distg1
  FS_PDM,       // gradient: PGet1 2-PDM, spherical -> Cartesian, de-contraction
  FS_N
};
#ifdef OR_COUNT_FLOPS
thread_local double t_flops[FS_N];
double g_flops[FS_N];
std::mutex g_flops_mu;
#define OR_FLOPS(stage, n) (t_flops[stage] += (double)(n))
// move this thread's tally into the total (at the end of each shell quartet)
void flops_commit() {
  std::lock_guard<std::mutex> lk(g_flops_mu);
  for (int t = 0; t < FS_N; ++t) {
    g_flops[t] += t_flops[t];
    t_flops[t] = 0.0;
  }
}
#else
#define OR_FLOPS(stage, n) ((void)0)
inline void flops_commit() {}
#endif

// ----------------------------------------------------------------- Rys table
struct RysOrder {
  double h = 0, tmax = 0;
  int K = 0;
  std::vector<double> hx, hw, coef;  // coef[K][2n][D+1]
};
struct RysTable {
  int nmax = 0, D = 0;
  std::vector<RysOrder> ord;  // index n-1
} g_rys;

int load_rys(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  char magic[8];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "RYSTAB01", 8) != 0) { fclose(f); return 2; }
  int32_t hdr[2];
  if (fread(hdr, 4, 2, f) != 2) { fclose(f); return 3; }
  g_rys.nmax = hdr[0];
  g_rys.D = hdr[1];
  g_rys.ord.assign(g_rys.nmax, RysOrder());
  for (int n = 1; n <= g_rys.nmax; ++n) {
    double hd[2];
    int32_t K;
    if (fread(hd, 8, 2, f) != 2 || fread(&K, 4, 1, f) != 1) { fclose(f); return 4; }
    g_rys.ord[n - 1].h = hd[0];
    g_rys.ord[n - 1].tmax = hd[1];
    g_rys.ord[n - 1].K = K;
  }
  for (int n = 1; n <= g_rys.nmax; ++n) {
    auto& o = g_rys.ord[n - 1];
    o.hx.resize(n);
    o.hw.resize(n);
    if (fread(o.hx.data(), 8, n, f) != (size_t)n || fread(o.hw.data(), 8, n, f) != (size_t)n) { fclose(f); return 5; }
  }
  for (int n = 1; n <= g_rys.nmax; ++n) {
    auto& o = g_rys.ord[n - 1];
    size_t cnt = (size_t)o.K * 2 * n * (g_rys.D + 1);
    o.coef.resize(cnt);
    if (fread(o.coef.data(), 8, cnt, f) != cnt) { fclose(f); return 6; }
  }
  fclose(f);
  return 0;
}

// roots x_i = t_i^2 and weights w_i of order n at argument T
inline void rys_rw(int n, double T, double* x, double* w) {
  const RysOrder& o = g_rys.ord[n - 1];
  if (T >= o.tmax) {
    double ai = 1.0 / T, si = std::sqrt(ai);
    for (int i = 0; i < n; ++i) { x[i] = o.hx[i] * ai; w[i] = o.hw[i] * si; }
    OR_FLOPS(FS_ROOTS, 2 + 2 * n);
    return;
  }
  int k = (int)(T / o.h);
  if (k >= o.K) k = o.K - 1;
  double s = 2.0 * (T - k * o.h) / o.h - 1.0;
  OR_FLOPS(FS_ROOTS, 6);
  const int D = g_rys.D;
  const double* c = &o.coef[(size_t)k * 2 * n * (D + 1)];
  for (int q = 0; q < 2 * n; ++q) {
    const double* cq = c + q * (D + 1);
    double acc = cq[D];
    for (int j = D - 1; j >= 0; --j) acc = acc * s + cq[j];
    OR_FLOPS(FS_ROOTS, 2 * D);
    if (q < n) x[q] = acc; else w[q - n] = acc;
  }
}

// ---------------------------------------------------------- index helpers
inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
inline int ncart_cum(int l) { return l < 0 ? 0 : l * (l + 1) * (l + 2) / 6; }  // # Cartesians with angular < l ... (nTri3_Elem(l))
// C3_Ind3 (misc_util/index_functions.F90:59-63), 0-based
inline int c3ind(int lx, int ly, int lz) {
  int l = lx + ly + lz;
  return ncart_cum(l) + (ly + lz) * (ly + lz + 1) / 2 + lz;
}
// C_Ind3, 0-based within a given l
inline int cind(int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }
struct Cart { int x, y, z; };
std::vector<Cart> cart_list(int l) {  // canonical ordering of iCan for one l
  std::vector<Cart> v;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) v.push_back({lx, ly, l - lx - ly});
  return v;
}
double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}
double dblfac(int n) {  // (n)!! with (-1)!! = 1
  double r = 1;
  for (int i = n; i > 1; i -= 2) r *= i;
  return r;
}

// ---------------------------------------------- real spherical harmonics
// Restates Real_Sphere for one l: returns matrix S[cart][m'] (ncart x (2l+1)),
// columns ordered m = -l..l (real_spherical.F90: Recurse, Ladder, NrmSph).
std::vector<std::vector<double>> g_sph;  // per l: ncart*(2l+1), column-major
void build_sph(int lmax) {
  g_sph.assign(lmax + 1, {});
  // m=0 functions P_l by Recurse: P_n = (2n-1)/n z P_{n-1} - (n-1)/n r^2 P_{n-2}
  std::vector<std::vector<double>> P0(lmax + 1);
  for (int n = 0; n <= lmax; ++n) {
    P0[n].assign(ncart(n), 0.0);
    if (n == 0) { P0[0][0] = 1.0; continue; }
    double f1 = double(2 * n - 1) / n;
    int n1 = n - 1;
    for (int ix = n1; ix >= 0; --ix)
      for (int iy = n1 - ix; iy >= 0; --iy) {
        int iz = n1 - ix - iy;
        P0[n][cind(iy, iz + 1)] += f1 * P0[n1][cind(iy, iz)];
      }
    if (n >= 2) {
      double f2 = double(n - 1) / n;
      int n0 = n - 2;
      for (int ix = n0; ix >= 0; --ix)
        for (int iy = n0 - ix; iy >= 0; --iy) {
          int iz = n0 - ix - iy;
          double v = P0[n0][cind(iy, iz)];
          P0[n][cind(iy, iz)] -= f2 * v;          // x+2
          P0[n][cind(iy + 2, iz)] -= f2 * v;      // y+2
          P0[n][cind(iy, iz + 2)] -= f2 * v;      // z+2
        }
    }
  }
  for (int n = 0; n <= lmax; ++n) {
    int nc = ncart(n);
    // Pm[m+n][cart]
    std::vector<std::vector<double>> Pm(2 * n + 1, std::vector<double>(nc, 0.0));
    Pm[n] = P0[n];
    auto idx = [&](int ix, int iy, int iz) { (void)ix; return cind(iy, iz); };
    for (int m = 0; m <= n - 1; ++m) {
      int mp = m + 1, mm = -(m + 1);
      std::vector<double>& Pp = Pm[mp + n];
      std::vector<double>& Pn = Pm[mm + n];
      std::fill(Pp.begin(), Pp.end(), 0.0);
      std::fill(Pn.begin(), Pn.end(), 0.0);
      double fact = 1.0 / (2.0 * std::sqrt(double(n * (n + 1) - m * (m - 1))));
      const std::vector<double>& Pc = Pm[m + n];
      const std::vector<double>& Pcm = Pm[-m + n];
      for (int ix = n; ix >= 0; --ix)
        for (int iy = n - ix; iy >= 0; --iy) {
          int iz = n - ix - iy;
          double pm = Pc[idx(ix, iy, iz)];
          double pmm = Pcm[idx(ix, iy, iz)];
          if (iz >= 1) Pp[idx(ix + 1, iy, iz - 1)] += fact * iz * pm;
          if (ix >= 1) Pp[idx(ix - 1, iy, iz + 1)] -= fact * ix * pm;
          if (m != 0) {
            if (iz >= 1) Pp[idx(ix, iy + 1, iz - 1)] -= fact * iz * pmm;
            if (iy >= 1) Pp[idx(ix, iy - 1, iz + 1)] += fact * iy * pmm;
          }
          if (iz >= 1) Pn[idx(ix, iy + 1, iz - 1)] += fact * iz * pm;
          if (iy >= 1) Pn[idx(ix, iy - 1, iz + 1)] -= fact * iy * pm;
          if (m != 0) {
            if (iz >= 1) Pn[idx(ix + 1, iy, iz - 1)] += fact * iz * pmm;
            if (ix >= 1) Pn[idx(ix - 1, iy, iz + 1)] -= fact * ix * pmm;
          }
        }
    }
    // NrmSph: drop tiny entries, normalise with the double-factorial metric
    auto carts = cart_list(n);
    for (int m = -n; m <= n; ++m) {
      std::vector<double>& P = Pm[m + n];
      double rmax = 0;
      for (double v : P) rmax = std::max(rmax, std::fabs(v));
      for (double& v : P) if (std::fabs(v) < 1e-12 * rmax) v = 0.0;
      double tmp = 0;
      for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
          int ex = carts[i].x + carts[j].x, ey = carts[i].y + carts[j].y, ez = carts[i].z + carts[j].z;
          if ((ex & 1) || (ey & 1) || (ez & 1)) continue;
          tmp += P[i] * P[j] * dblfac(ex - 1) * dblfac(ey - 1) * dblfac(ez - 1);
        }
      double sc = 1.0 / std::sqrt(tmp);
      for (double& v : P) v *= sc;
    }
    g_sph[n].assign((size_t)nc * (2 * n + 1), 0.0);
    for (int m = -n; m <= n; ++m)
      for (int c = 0; c < nc; ++c) g_sph[n][c + (size_t)nc * (m + n)] = Pm[m + n][c];
  }
  // s and p shells are never transformed (gateway_util/rdctl_seward.F90:
  // 3863-3865, SPHE only from d on): p stays Cartesian x, y, z.
  if (lmax >= 1) {
    g_sph[1].assign(9, 0.0);
    for (int i = 0; i < 3; ++i) g_sph[1][i + 3 * i] = 1.0;
  }
}

// ------------------------------------------------------------------ basis
struct Shell {
  double A[3];
  int l, np, nc, atom, off;  // off = first spherical AO index
  std::vector<double> e, c;  // c[p + np*k]
};
struct Basis {
  std::vector<Shell> sh;
  int nbf = 0, natom = 0;
  std::vector<double> tmax;  // Schwarz sqrt(max|(ab|ab)|) per shell pair [i*nsh+j]
};

inline int nsph(int l) { return 2 * l + 1; }
inline bool eq3(const double* a, const double* b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

// HrrMtrx restated (hrrmtrx.F90): H[ipe][sa][sb] with e relative to emin block
std::vector<double> hrr_mtrx(int la, int lb, const double* A, const double* B, int& ne_out) {
  int lta = ncart(la), ltb = ncart(lb);
  int na = nsph(la), nb = nsph(lb);
  bool AeqB = eq3(A, B);
  int emin = AeqB ? la + lb : std::max(la, lb);
  int emax = la + lb;
  int ne = ncart_cum(emax + 1) - ncart_cum(emin);
  ne_out = ne;
  int joff = ncart_cum(emin);
  std::vector<double> H((size_t)ne * na * nb, 0.0);
  double AB[3];
  for (int i = 0; i < 3; ++i) AB[i] = (la >= lb) ? A[i] - B[i] : B[i] - A[i];
  auto pw = [](double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; };
  auto ca = cart_list(la), cb = cart_list(lb);
  const std::vector<double>& Sa = g_sph[la];
  const std::vector<double>& Sb = g_sph[lb];
  for (int sa = 0; sa < na; ++sa)
    for (int ipa = 0; ipa < lta; ++ipa) {
      double Ca = Sa[ipa + (size_t)lta * sa];
      if (Ca == 0.0) continue;
      int ix = ca[ipa].x, iy = ca[ipa].y, iz = ca[ipa].z;
      for (int sb = 0; sb < nb; ++sb)
        for (int ipb = 0; ipb < ltb; ++ipb) {
          double Cb = Sb[ipb + (size_t)ltb * sb];
          if (Cb == 0.0) continue;
          int jx = cb[ipb].x, jy = cb[ipb].y, jz = cb[ipb].z;
          // transfer onto the centre of higher l
          int bx = (la >= lb) ? ix : jx, by = (la >= lb) ? iy : jy, bz = (la >= lb) ? iz : jz;  // kept
          int tx = (la >= lb) ? jx : ix, ty = (la >= lb) ? jy : iy, tz = (la >= lb) ? jz : iz;  // transferred
          int lox = AeqB ? bx + tx : bx, loy = AeqB ? by + ty : by, loz = AeqB ? bz + tz : bz;
          for (int kx = lox; kx <= bx + tx; ++kx)
            for (int ky = loy; ky <= by + ty; ++ky)
              for (int kz = loz; kz <= bz + tz; ++kz) {
                int ipe = c3ind(kx, ky, kz) - joff;
                double f = pw(AB[0], bx + tx - kx) * binom(tx, kx - bx) * pw(AB[1], by + ty - ky) * binom(ty, ky - by) *
                           pw(AB[2], bz + tz - kz) * binom(tz, kz - bz);
                H[ipe + (size_t)ne * (sa + (size_t)na * sb)] += f * Ca * Cb;
              }
        }
    }
  return H;
}

const double kTwoP54 = std::sqrt(2.0) * std::pow(M_PI, 1.25);

struct PairData {
  int np;  // nalpha*nbeta, alpha fastest
  std::vector<double> zeta, kappa, P, alpha, beta;
};
PairData make_pair(const Shell& a, const Shell& b) {
  PairData d;
  d.np = a.np * b.np;
  double AB2 = 0;
  for (int i = 0; i < 3; ++i) AB2 += (a.A[i] - b.A[i]) * (a.A[i] - b.A[i]);
  d.zeta.resize(d.np); d.kappa.resize(d.np); d.P.resize(3 * d.np); d.alpha.resize(d.np); d.beta.resize(d.np);
  for (int jb = 0; jb < b.np; ++jb)
    for (int ia = 0; ia < a.np; ++ia) {
      int iz = ia + a.np * jb;
      double al = a.e[ia], be = b.e[jb], z = al + be, zi = 1.0 / z;
      d.zeta[iz] = z;
      d.alpha[iz] = al;
      d.beta[iz] = be;
      double k = kTwoP54 * std::exp(-al * be * AB2 * zi) * zi;
      if (k < 1e-99) k = 1e-99;
      d.kappa[iz] = k;
      for (int x = 0; x < 3; ++x) d.P[iz + d.np * x] = (al * a.A[x] + be * b.A[x]) * zi;
    }
  return d;
}

// 2D integrals I[r][i][j] for i<=imax (bra, at centre "A"), j<=jmax (ket at "C")
// restating vCff2D + vRys2D; z component carries the Rys weight.
struct TwoD {
  int nr, ni, nj;
  std::vector<double> v;  // [xyz][r][i][j]
  double& at(int c, int r, int i, int j) { return v[(((size_t)c * nr + r) * ni + i) * nj + j]; }
};
void rys2d(int nr, int imax, int jmax, double zeta, double eta, const double* P, const double* Q, const double* Ap,
           const double* Cp, const double* u2, const double* w, TwoD& G) {
  G.nr = nr; G.ni = imax + 1; G.nj = jmax + 1;
  G.v.assign((size_t)3 * nr * G.ni * G.nj, 0.0);
  double zi = 1.0 / zeta, ei = 1.0 / eta, ze = zeta + eta, zei = 1.0 / ze;
  OR_FLOPS(FS_RYS2D, 4);
  for (int r = 0; r < nr; ++r) {
    double U2 = u2[r] * zei;              // ModU2
    double B00 = 0.5 * U2;
    double B10 = 0.5 * (1.0 - U2 * eta) * zi;
    double B01 = 0.5 * (1.0 - U2 * zeta) * ei;
    OR_FLOPS(FS_RYS2D, 10);
    for (int c = 0; c < 3; ++c) {
      double PAQP = P[c] - Ap[c] + eta * U2 * (Q[c] - P[c]);
      double QCPQ = Q[c] - Cp[c] - zeta * U2 * (Q[c] - P[c]);
      OR_FLOPS(FS_RYS2D, 10);
      double I00 = (c == 2) ? w[r] : 1.0;
      G.at(c, r, 0, 0) = I00;
      if (imax >= 1) { G.at(c, r, 1, 0) = PAQP * I00; OR_FLOPS(FS_RYS2D, 1); }
      for (int i = 1; i < imax; ++i) {
        G.at(c, r, i + 1, 0) = PAQP * G.at(c, r, i, 0) + i * B10 * G.at(c, r, i - 1, 0);
        OR_FLOPS(FS_RYS2D, 4);
      }
      for (int j = 0; j < jmax; ++j)
        for (int i = 0; i <= imax; ++i) {
          double v = QCPQ * G.at(c, r, i, j);
          if (j >= 1) v += j * B01 * G.at(c, r, i, j - 1);
          if (i >= 1) v += i * B00 * G.at(c, r, i - 1, j);
          G.at(c, r, i, j + 1) = v;
          OR_FLOPS(FS_RYS2D, 1 + (j >= 1 ? 3 : 0) + (i >= 1 ? 3 : 0));
        }
    }
  }
}

// (AB|CD) contracted, spherical, reference layout [ijkl][a][b][c][d]
// absmode: use |contraction coefficients| and |[e0|f0]| -- the cancellation-free
// magnitude S of each integral, used to scale the FP64 parity bar.
void eri_quartet(const Basis& bs, int iS, int jS, int kS, int lS, double* out, bool absmode = false) {
  const Shell &a = bs.sh[iS], &b = bs.sh[jS], &c = bs.sh[kS], &d = bs.sh[lS];
  int la = a.l, lb = b.l, lc = c.l, ld = d.l;
  int nijkl = a.nc * b.nc * c.nc * d.nc;
  int na = nsph(la), nb = nsph(lb), nc = nsph(lc), nd = nsph(ld);
  size_t nout = (size_t)nijkl * na * nb * nc * nd;
  std::fill(out, out + nout, 0.0);
  bool AeqB = eq3(a.A, b.A), CeqD = eq3(c.A, d.A);
  int lsum = la + lb + lc + ld;
  // twoel_nosym.F90:136-137 zero-by-symmetry exits (all on one centre)
  if (AeqB && CeqD && eq3(a.A, c.A)) {
    if (lsum & 1) return;
    if (2 * std::max(std::max(la, lb), std::max(lc, ld)) > lsum) return;
  }
  const double* Ap = (la >= lb) ? a.A : b.A;
  const double* Cp = (lc >= ld) ? c.A : d.A;
  int emin = AeqB ? la + lb : std::max(la, lb), emax = la + lb;
  int fmin = CeqD ? lc + ld : std::max(lc, ld), fmax = lc + ld;
  int ne, nf;
  std::vector<double> Hab = hrr_mtrx(la, lb, a.A, b.A, ne);
  std::vector<double> Hcd = hrr_mtrx(lc, ld, c.A, d.A, nf);
  int eoff = ncart_cum(emin), foff = ncart_cum(fmin);
  std::vector<Cart> elist, flist;
  for (int l = emin; l <= emax; ++l) for (auto& q : cart_list(l)) elist.push_back(q);
  for (int l = fmin; l <= fmax; ++l) for (auto& q : cart_list(l)) flist.push_back(q);
  (void)eoff; (void)foff;
  int nr = lsum / 2 + 1;
  PairData pab = make_pair(a, b), pcd = make_pair(c, d);
  std::vector<double> acc((size_t)nijkl * ne * nf, 0.0);  // [ijkl][e][f]
  std::vector<double> ef((size_t)ne * nf);
  double x[16], w[16];
  TwoD G;
  for (int pq = 0; pq < pcd.np; ++pq) {
    int ic = pq % c.np, id = pq / c.np;
    double eta = pcd.zeta[pq];
    double Q[3] = {pcd.P[pq], pcd.P[pq + pcd.np], pcd.P[pq + 2 * pcd.np]};
    for (int pp = 0; pp < pab.np; ++pp) {
      int ia = pp % a.np, ib = pp / a.np;
      double zeta = pab.zeta[pp];
      double P[3] = {pab.P[pp], pab.P[pp + pab.np], pab.P[pp + 2 * pab.np]};
      double ze = zeta + eta, tmp = 1.0 / ze, rho = zeta * eta * tmp;
      double PQ2 = (P[0] - Q[0]) * (P[0] - Q[0]) + (P[1] - Q[1]) * (P[1] - Q[1]) + (P[2] - Q[2]) * (P[2] - Q[2]);
      double T = rho * PQ2;
      double Fact = pab.kappa[pp] * pcd.kappa[pq] * std::sqrt(tmp);
      OR_FLOPS(FS_PRIM, 16);
      rys_rw(nr, T, x, w);
      rys2d(nr, emax, fmax, zeta, eta, P, Q, Ap, Cp, x, w, G);
      for (int ie = 0; ie < ne; ++ie)
        for (int jf = 0; jf < nf; ++jf) {
          const Cart &E = elist[ie], &F = flist[jf];
          double s = 0;
          for (int r = 0; r < nr; ++r) s += G.at(0, r, E.x, F.x) * G.at(1, r, E.y, F.y) * G.at(2, r, E.z, F.z);
          ef[ie + (size_t)ne * jf] = absmode ? std::fabs(s * Fact) : s * Fact;
          OR_FLOPS(FS_RYSEF, 3 * nr + 1);
        }
      for (int l4 = 0; l4 < d.nc; ++l4)
        for (int k3 = 0; k3 < c.nc; ++k3) {
          double ccd = c.c[ic + c.np * k3] * d.c[id + d.np * l4];
          OR_FLOPS(FS_CONTRACT, 1);
          if (absmode) ccd = std::fabs(ccd);
          if (ccd == 0.0) continue;
          for (int j2 = 0; j2 < b.nc; ++j2)
            for (int i1 = 0; i1 < a.nc; ++i1) {
              double cf = a.c[ia + a.np * i1] * b.c[ib + b.np * j2] * ccd;
              OR_FLOPS(FS_CONTRACT, 2);
              if (absmode) cf = std::fabs(cf);
              if (cf == 0.0) continue;
              int ijkl = i1 + a.nc * (j2 + b.nc * (k3 + c.nc * l4));
              double* ac = &acc[(size_t)ijkl * ne * nf];
              for (size_t t = 0; t < (size_t)ne * nf; ++t) ac[t] += cf * ef[t];
              OR_FLOPS(FS_CONTRACT, 2 * ne * nf);
            }
        }
    }
  }
  // HRR + spherical (TnsCtl with HrrMtrx): bra then ket
  std::vector<double> tmpab((size_t)na * nb * nf);
  for (int ijkl = 0; ijkl < nijkl; ++ijkl) {
    const double* ac = &acc[(size_t)ijkl * ne * nf];
    std::fill(tmpab.begin(), tmpab.end(), 0.0);
    for (int jf = 0; jf < nf; ++jf)
      for (int sab = 0; sab < na * nb; ++sab) {
        double s = 0;
        for (int ie = 0; ie < ne; ++ie) s += (absmode ? std::fabs(Hab[ie + (size_t)ne * sab]) : Hab[ie + (size_t)ne * sab]) * ac[ie + (size_t)ne * jf];
        tmpab[sab + (size_t)na * nb * jf] = s;
        OR_FLOPS(FS_HRR, 2 * ne);
      }
    for (int scd = 0; scd < nc * nd; ++scd)
      for (int sab = 0; sab < na * nb; ++sab) {
        double s = 0;
        for (int jf = 0; jf < nf; ++jf) s += (absmode ? std::fabs(Hcd[jf + (size_t)nf * scd]) : Hcd[jf + (size_t)nf * scd]) * tmpab[sab + (size_t)na * nb * jf];
        out[ijkl + (size_t)nijkl * (sab + (size_t)na * nb * scd)] = s;
        OR_FLOPS(FS_HRR, 2 * nf);
      }
  }
  flops_commit();
}

// AO index of (shell, contracted k, spherical m): shells store functions
// as [k][m] with m fastest?  The reference orders basis functions of a shell
// by contracted function then component is NOT assumed here; we use the
// layout ao = off + m*nc + k  (component-major, as iSD4(7)/iAO offsets in
// the reference: for each component the nBas contracted functions follow).
inline int ao_index(const Shell& s, int k, int m) { return s.off + m * s.nc + k; }

struct RSList;
struct Handle {
  Basis bs;
  std::shared_ptr<RSList> rs;  // the rs list of the last decomposition (or of rs_compact); null: every pair
};

std::vector<int> quartet_dims(const Basis& bs, int i, int j, int k, int l) {
  return {bs.sh[i].nc * bs.sh[j].nc * bs.sh[k].nc * bs.sh[l].nc, nsph(bs.sh[i].l), nsph(bs.sh[j].l), nsph(bs.sh[k].l),
          nsph(bs.sh[l].l)};
}

size_t quartet_size(const Basis& bs, int i, int j, int k, int l) {
  auto d = quartet_dims(bs, i, j, k, l);
  return (size_t)d[0] * d[1] * d[2] * d[3] * d[4];
}

// scatter a quartet block into a full nbf^4 tensor (all 8 permutations)
void scatter_full(const Basis& bs, int iS, int jS, int kS, int lS, const double* blk, double* full) {
  const Shell &A = bs.sh[iS], &B = bs.sh[jS], &C = bs.sh[kS], &D = bs.sh[lS];
  size_t n = bs.nbf;
  int nijkl = A.nc * B.nc * C.nc * D.nc;
  int na = nsph(A.l), nb = nsph(B.l), nc = nsph(C.l), nd = nsph(D.l);
  for (int md = 0; md < nd; ++md)
    for (int mc = 0; mc < nc; ++mc)
      for (int mb = 0; mb < nb; ++mb)
        for (int ma = 0; ma < na; ++ma)
          for (int l4 = 0; l4 < D.nc; ++l4)
            for (int k3 = 0; k3 < C.nc; ++k3)
              for (int j2 = 0; j2 < B.nc; ++j2)
                for (int i1 = 0; i1 < A.nc; ++i1) {
                  int ijkl = i1 + A.nc * (j2 + B.nc * (k3 + C.nc * l4));
                  double v = blk[ijkl + (size_t)nijkl * (ma + na * (mb + nb * (mc + (size_t)nc * md)))];
                  size_t p = ao_index(A, i1, ma), q = ao_index(B, j2, mb), r = ao_index(C, k3, mc), s = ao_index(D, l4, md);
                  full[((p * n + q) * n + r) * n + s] = v;
                  full[((q * n + p) * n + r) * n + s] = v;
                  full[((p * n + q) * n + s) * n + r] = v;
                  full[((q * n + p) * n + s) * n + r] = v;
                  full[((r * n + s) * n + p) * n + q] = v;
                  full[((s * n + r) * n + p) * n + q] = v;
                  full[((r * n + s) * n + q) * n + p] = v;
                  full[((s * n + r) * n + q) * n + p] = v;
                }
}

// ------------------------------------------------------ Schwarz screening
void compute_tmax(Basis& bs) {
  int ns = bs.sh.size();
  bs.tmax.assign((size_t)ns * ns, 0.0);
  std::vector<std::pair<int, int>> prs;
  for (int i = 0; i < ns; ++i) for (int j = 0; j <= i; ++j) prs.push_back({i, j});
#pragma omp parallel for schedule(dynamic)
  for (size_t t = 0; t < prs.size(); ++t) {
    int i = prs[t].first, j = prs[t].second;
    std::vector<double> blk(quartet_size(bs, i, j, i, j));
    eri_quartet(bs, i, j, i, j, blk.data());
    auto dm = quartet_dims(bs, i, j, i, j);
    // diagonal elements (ab|ab): ijkl with k=i,l=j and (a,b)=(c,d)
    const Shell &A = bs.sh[i], &B = bs.sh[j];
    double mx = 0;
    for (int mb = 0; mb < dm[2]; ++mb)
      for (int ma = 0; ma < dm[1]; ++ma)
        for (int j2 = 0; j2 < B.nc; ++j2)
          for (int i1 = 0; i1 < A.nc; ++i1) {
            int ijkl = i1 + A.nc * (j2 + B.nc * (i1 + A.nc * j2));
            double v = blk[ijkl + (size_t)dm[0] * (ma + dm[1] * (mb + dm[2] * (ma + (size_t)dm[1] * mb)))];
            mx = std::max(mx, std::fabs(v));
          }
    bs.tmax[(size_t)i * ns + j] = bs.tmax[(size_t)j * ns + i] = std::sqrt(mx);
  }
}


// ------------------------------------------------------------- AO pairs
// Reduced-set ("rs") ordering of AO pairs a>=b used by the Cholesky code:
// shell pairs iS>=jS in iTri order; inside a pair with iS>jS the local index
// is a + nA*b (a fastest), inside iS==jS it is iTri(a,b), a>=b
// (cholesky_util/plf_cho_diag.F90:60-72).  a, b are local AO indices of the
// shells (component-major, contracted fastest).
struct RSList {
  std::vector<int> a, b, sp;      // global AO indices and shell pair id
  std::vector<int> sp_i, sp_j;    // shells of each pair
  std::vector<int> sp_first, sp_count;
};
// keep: the shell pairs that carry rows (null: all); the others keep their
// pair id with sp_first = -1 and no rows.
RSList make_rs(const Basis& bs, const std::vector<char>* keep = nullptr) {
  RSList R;
  int ns = bs.sh.size();
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      int id = R.sp_i.size();
      R.sp_i.push_back(i);
      R.sp_j.push_back(j);
      if (keep && !(*keep)[id]) {
        R.sp_first.push_back(-1);
        R.sp_count.push_back(0);
        continue;
      }
      R.sp_first.push_back(R.a.size());
      const Shell &A = bs.sh[i], &B = bs.sh[j];
      int nA = A.nc * nsph(A.l), nB = B.nc * nsph(B.l);
      if (i != j) {
        for (int lb = 0; lb < nB; ++lb)
          for (int la = 0; la < nA; ++la) { R.a.push_back(A.off + la); R.b.push_back(B.off + lb); R.sp.push_back(id); }
      } else {
        for (int la = 0; la < nA; ++la)
          for (int lb = 0; lb <= la; ++lb) { R.a.push_back(A.off + la); R.b.push_back(A.off + lb); R.sp.push_back(id); }
      }
      R.sp_count.push_back((int)R.a.size() - R.sp_first.back());
    }
  return R;
}

// element (p q | r s) out of a shell-quartet block; p in shell i, etc.
inline double blk_elem(const Basis& bs, const double* blk, int i, int j, int k, int l, int p, int q, int r, int s) {
  const Shell &A = bs.sh[i], &B = bs.sh[j], &C = bs.sh[k], &D = bs.sh[l];
  int lp = p - A.off, lq = q - B.off, lr = r - C.off, ls = s - D.off;
  int ma = lp / A.nc, ka = lp % A.nc, mb = lq / B.nc, kb = lq % B.nc;
  int mc = lr / C.nc, kc = lr % C.nc, md = ls / D.nc, kd = ls % D.nc;
  int nijkl = A.nc * B.nc * C.nc * D.nc;
  int ijkl = ka + A.nc * (kb + B.nc * (kc + C.nc * kd));
  int na = nsph(A.l), nb = nsph(B.l), nc = nsph(C.l);
  return blk[ijkl + (size_t)nijkl * (ma + na * (mb + (size_t)nb * (mc + (size_t)nc * md)))];
}

// columns (rs_row | ab_q) for all rows and the listed columns (all in one
// shell pair AB), restating CHO_MCA_CALCINT_1 + PLF_Cho
void cho_columns_sp(const Basis& bs, const RSList& R, const std::vector<char>& inred, const std::vector<int>& cols,
                    std::vector<double>& xint /* nrs x ncol */) {
  size_t nrs = R.a.size();
  int ncol = cols.size();
  xint.assign(nrs * ncol, 0.0);
  int spAB = R.sp[cols[0]];
  int iA = R.sp_i[spAB], iB = R.sp_j[spAB];
  int nsp = R.sp_i.size();
#pragma omp parallel for schedule(dynamic)
  for (int sp = 0; sp < nsp; ++sp) {
    bool any = false;
    for (int t = 0; t < R.sp_count[sp]; ++t) if (inred[R.sp_first[sp] + t]) { any = true; break; }
    if (!any) continue;
    int iC = R.sp_i[sp], iD = R.sp_j[sp];
    std::vector<double> blk(quartet_size(bs, iC, iD, iA, iB));
    eri_quartet(bs, iC, iD, iA, iB, blk.data());
    for (int t = 0; t < R.sp_count[sp]; ++t) {
      int rs = R.sp_first[sp] + t;
      if (!inred[rs]) continue;
      for (int q = 0; q < ncol; ++q) {
        int cq = cols[q];
        xint[rs + nrs * q] = blk_elem(bs, blk.data(), iC, iD, iA, iB, R.a[rs], R.b[rs], R.a[cq], R.b[cq]);
      }
    }
  }
}

// columns of qualified diagonals taken from several shell pairs (one
// Cho_MCA_CalcInt per shell pair, cho_getint.F90:118), in list order
void cho_columns(const Basis& bs, const RSList& R, const std::vector<char>& inred, const std::vector<int>& cols,
                 std::vector<double>& xint /* nrs x ncol */) {
  size_t nrs = R.a.size();
  xint.assign(nrs * cols.size(), 0.0);
  std::vector<char> done(cols.size(), 0);
  for (size_t c0 = 0; c0 < cols.size(); ++c0) {
    if (done[c0]) continue;
    std::vector<int> sub, pos;
    for (size_t c = c0; c < cols.size(); ++c)
      if (!done[c] && R.sp[cols[c]] == R.sp[cols[c0]]) { sub.push_back(cols[c]); pos.push_back((int)c); done[c] = 1; }
    std::vector<double> x;
    cho_columns_sp(bs, R, inred, sub, x);
    for (size_t q = 0; q < sub.size(); ++q)
      std::copy(x.begin() + nrs * q, x.begin() + nrs * (q + 1), xint.begin() + nrs * pos[q]);
  }
}

struct ChoCfg {
  double thrcom, span, damp1, damp2, thrneg, warneg, tooneg;
  int minqual, maxqual;
  int mxshpr = 1;  // max. shell pairs qualified per pass (1 for algorithm 4); 0 = no limit (algorithms 1-3)
  int ialqua = 2;  // qualification: 1 = Cho_Qualify_1 (in order up to MaxQual), 2 = Cho_Qualify_2 (the default)
};
double cho_default_damp(double thrcom) {  // cho_setdamp.F90
  if (thrcom > 9.99e-3) return 1e7;
  if (thrcom > 9.99e-4) return 1e6;
  if (thrcom > 9.99e-5) return 1e5;
  if (thrcom > 9.99e-6) return 1e4;
  if (thrcom > 9.99e-7) return 1e3;
  if (thrcom > 9.99e-8) return 1e2;
  if (thrcom > 9.99e-9) return 1e1;
  return 1.0;
}

// CD_InCore_1p restated; X n x n column-major, Vec n x mxvec; returns irc
int cd_incore_1p(std::vector<double>& X, int n, std::vector<double>& Vec, int mxvec, int& numcho, double thr,
                 double thrneg, double thrfail, std::vector<int>& iD) {
  numcho = 0;
  double acc = std::min(1e-12, thr * 1e-2);
  auto x = [&](int i, int j) -> double& { return X[i + (size_t)n * j]; };
  for (int pass = 0; pass < n; ++pass) {
    if (x(0, 0) < thrneg) {
      if (x(0, 0) < thrfail) return 101;
      for (int t = 0; t < n; ++t) { x(t, 0) = 0; x(0, t) = 0; }
    }
    double xmax = 0;
    int imax = -1;
    for (int i = 0; i < n; ++i) {
      if (x(i, i) < thrneg) {
        if (x(i, i) < thrfail) return 101;
        for (int t = 0; t < n; ++t) { x(t, i) = 0; x(i, t) = 0; }
      }
      if (x(i, i) > xmax + acc) { xmax = x(i, i); imax = i; }
    }
    if (xmax <= thr) return 0;
    double xfac = 1.0 / std::sqrt(std::fabs(xmax));
    if (numcho == mxvec) return 102;
    for (int j = 0; j < numcho; ++j) {
      double v = Vec[imax + (size_t)n * j];
      for (int t = 0; t < n; ++t) x(t, imax) -= v * Vec[t + (size_t)n * j];
    }
    x(imax, imax) = xmax;
    int k = numcho++;
    for (int i = 0; i < n; ++i) Vec[i + (size_t)n * k] = (x(i, i) == 0.0) ? 0.0 : xfac * x(i, imax);
    for (int i = 0; i < n; ++i) x(i, i) -= Vec[i + (size_t)n * k] * Vec[i + (size_t)n * k];
    x(imax, imax) = 0.0;
    iD.push_back(imax);
  }
  return 0;
}

struct ChoResult {
  std::vector<double> L;   // nrs x M (column-major), zero outside the pass's reduced set
  std::vector<int> piv;    // rs index of each vector
  std::vector<int> pass_of;
  int M = 0;
  int npass = 0;
  int irc = 0;
};

ChoResult cho_decompose(const Basis& bs, const ChoCfg& cfg, const std::vector<double>& diag0, const RSList& R) {
  ChoResult res;
  size_t nrs = R.a.size();
  std::vector<double> diag = diag0;
  // initial screening (cho_calcdiag.F90:255-300)
  double diamax = 0;
  for (double d : diag) diamax = std::max(diamax, std::fabs(d));
  double scrmax = diamax > 0 ? cfg.thrcom * cfg.thrcom / cfg.damp1 / diamax : 1e15;
  std::vector<char> inred(nrs, 0);
  for (size_t t = 0; t < nrs; ++t) {
    if (diag[t] < scrmax) diag[t] = 0.0; else inred[t] = 1;
  }
  int nsp = R.sp_i.size();
  std::vector<double> L;  // nrs x M
  int M = 0;
  for (int pass = 0; pass < (int)nrs + 1; ++pass) {
    // Cho_SetPass
    double dgmax = -1e15;
    for (size_t t = 0; t < nrs; ++t) if (inred[t]) dgmax = std::max(dgmax, std::fabs(diag[t]));
    if (dgmax < cfg.thrcom) break;
    double diamin = std::max(dgmax * cfg.span, cfg.thrcom);
    std::vector<double> diash(nsp, 0.0);
    for (size_t t = 0; t < nrs; ++t) if (inred[t]) diash[R.sp[t]] = std::max(diash[R.sp[t]], diag[t]);
    int npotsh = 0;
    for (int sp = 0; sp < nsp; ++sp) {
      if (!(diash[sp] > cfg.thrcom)) diash[sp] = 0.0; else ++npotsh;
    }
    // Cho_GetInt (cho_getint.F90:38-140): take shell pairs in order of their
    // largest diagonal (Cho_GetMaxShl zeroes the one it returns) and qualify
    // their columns (Cho_Qualify, IALQUA = 2: cho_qualify_2.F90) until
    // MinQual columns, MaxQual (FULL) or MXSHPR shell pairs
    const int mcount = cfg.mxshpr > 0 ? std::min(npotsh, cfg.mxshpr) : npotsh;
    std::vector<int> qual;
    bool dodeco = false, fail = false;
    for (int icount = 0; !dodeco && icount < mcount;) {
      ++icount;
      double smax = -1e9;
      int spab = -1;
      for (int sp = 0; sp < nsp; ++sp) if (diash[sp] > smax) { smax = diash[sp]; spab = sp; }
      diash[spab] = 0.0;
      if (smax == 0.0 || std::fabs(smax) < diamin) {
        if (icount == 1) { fail = true; break; }
        dodeco = !qual.empty();
        break;
      }
      const int maxq = cfg.maxqual - (int)qual.size();
      const size_t ioffq = qual.size();
      if (cfg.ialqua == 1) {  // cho_qualify_1.F90:26-40: in order, up to MAXQ
        for (int t = 0; t < R.sp_count[spab] && (int)(qual.size() - ioffq) < maxq; ++t) {
          int rs = R.sp_first[spab] + t;
          if (inred[rs] && diag[rs] >= diamin) qual.push_back(rs);
        }
      } else if (maxq == 1) {  // the largest >= DIAMIN (last one on ties)
        double xmax = diamin;
        int imax = -1;
        for (int t = 0; t < R.sp_count[spab]; ++t) {
          int rs = R.sp_first[spab] + t;
          if (inred[rs] && diag[rs] >= xmax) { xmax = diag[rs]; imax = rs; }
        }
        if (imax >= 0) qual.push_back(imax);
      } else if (maxq > 1) {  // in order; once MAXQ are taken, a larger one replaces the smallest
        for (int t = 0; t < R.sp_count[spab]; ++t) {
          int rs = R.sp_first[spab] + t;
          if (!inred[rs] || !(diag[rs] >= diamin)) continue;
          if ((int)(qual.size() - ioffq) < maxq) {
            qual.push_back(rs);
          } else {
            size_t kmin = ioffq;
            for (size_t k = ioffq + 1; k < qual.size(); ++k) if (diag[qual[k]] < diag[qual[kmin]]) kmin = k;
            if (diag[rs] > diag[qual[kmin]]) qual[kmin] = rs;
          }
        }
      }
      const int ncolab = (int)(qual.size() - ioffq);
      const bool full = (int)qual.size() == cfg.maxqual;
      if (ncolab > 0) {
        dodeco = full || (int)qual.size() >= cfg.minqual;
      } else {
        if (qual.empty()) { fail = true; break; }
        dodeco = true;
      }
    }
    if (fail || qual.empty()) { res.irc = 104; break; }
    int nq = qual.size();
    std::vector<double> xint;
    cho_columns(bs, R, inred, qual, xint);
    // Cho_Dec_Qual: Q = MQ - LQ LQ^T, pivoted CD of Q
    std::vector<double> Q((size_t)nq * nq);
    for (int c = 0; c < nq; ++c)
      for (int r = 0; r < nq; ++r) {
        double v = xint[qual[r] + nrs * c];
        for (int J = 0; J < M; ++J) v -= L[qual[r] + nrs * J] * L[qual[c] + nrs * J];
        Q[r + (size_t)nq * c] = v;
      }
    std::vector<double> qdiag(nq);
    for (int q = 0; q < nq; ++q) qdiag[q] = Q[q + (size_t)nq * q];
    double dmax = 0;  // Cho_P_MaxDX: largest diagonal in the reduced set
    for (size_t t = 0; t < nrs; ++t) if (inred[t]) dmax = std::max(dmax, diag[t]);
    double thr = std::max(cfg.thrcom, dmax * cfg.span);
    std::vector<double> Vec((size_t)nq * nq, 0.0);
    std::vector<int> iD;
    int nk = 0;
    int irc = cd_incore_1p(Q, nq, Vec, nq, nk, thr, -1e-13, -1e-8, iD);
    if (irc) { res.irc = 104; break; }
    // reorder to pivot order (cho_decom_a4.F90:120-170)
    std::vector<double> K((size_t)nk * nk);
    for (int i = 0; i < nk; ++i)
      for (int j = 0; j < nk; ++j) K[j + (size_t)nk * i] = Vec[iD[j] + (size_t)nq * i];
    std::vector<double> qd(nk);
    std::vector<int> qrs(nk);
    std::vector<double> X(nrs * (size_t)nk);
    for (int i = 0; i < nk; ++i) {
      qd[i] = qdiag[iD[i]];
      qrs[i] = qual[iD[i]];
      for (size_t t = 0; t < nrs; ++t) X[t + nrs * i] = inred[t] ? xint[t + nrs * iD[i]] : 0.0;
    }
    // Cho_Subtr: X -= L_prev LQ^T
    for (int i = 0; i < nk; ++i)
      for (int J = 0; J < M; ++J) {
        double lq = L[qrs[i] + nrs * J];
        if (lq == 0.0) continue;
        for (size_t t = 0; t < nrs; ++t) if (inred[t]) X[t + nrs * i] -= L[t + nrs * J] * lq;
      }
    // Cho_CompVec
    double qdmax = qd[0];
    for (int i = 0; i < nk; ++i) {
      double fac = 1.0 / std::sqrt(std::fabs(qd[i]));
      double* xi = &X[nrs * i];
      for (size_t t = 0; t < nrs; ++t) if (inred[t]) xi[t] *= fac;
      for (size_t t = 0; t < nrs; ++t) if (inred[t] && diag[t] == 0.0) xi[t] = 0.0;
      for (size_t t = 0; t < nrs; ++t) if (inred[t]) diag[t] -= xi[t] * xi[t];
      for (int j = i; j < nk; ++j) qd[j] -= K[j + (size_t)nk * i] * K[j + (size_t)nk * i];
      qd[i] = 0.0;
      diag[qrs[i]] = 0.0;  // Cho_P_ZeroDiag
      // Cho_ChkDia_A4
      for (size_t t = 0; t < nrs; ++t) {
        if (!inred[t]) continue;
        if (diag[t] < 0.0 && diag[t] < cfg.thrneg) {
          if (diag[t] < cfg.tooneg) { res.irc = 104; return res; }
          diag[t] = 0.0;
        }
      }
      for (size_t t = 0; t < nrs; ++t) {
        if (!inred[t]) continue;
        if (std::sqrt(std::fabs(diag[t]) * qdmax) * cfg.damp2 <= cfg.thrcom) diag[t] = 0.0;
      }
      for (int j = i + 1; j < nk; ++j) {
        double f = -K[j + (size_t)nk * i];
        double* xj = &X[nrs * j];
        for (size_t t = 0; t < nrs; ++t) if (inred[t]) xj[t] += f * xi[t];
      }
    }
    L.insert(L.end(), X.begin(), X.end());
    for (int i = 0; i < nk; ++i) { res.piv.push_back(qrs[i]); res.pass_of.push_back(pass); }
    M += nk;
    res.npass = pass + 1;
    // Cho_SetRed mode 1 (damped, negative diagonals excluded)
    double xm = 0;
    bool any = false;
    for (size_t t = 0; t < nrs; ++t) if (inred[t]) { xm = any ? std::max(xm, std::fabs(diag[t])) : std::fabs(diag[t]); any = true; }
    std::vector<char> nr(nrs, 0);
    if (xm > cfg.thrcom)
      for (size_t t = 0; t < nrs; ++t)
        if (inred[t] && diag[t] > 0.0 && std::sqrt(diag[t] * xm) * cfg.damp2 > cfg.thrcom) nr[t] = 1;
    inred.swap(nr);
  }
  res.L.swap(L);
  res.M = M;
  return res;
}

// ERI diagonal (ab|ab) over the rs list (CHO_CALCDIAG)
std::vector<double> eri_diag(const Basis& bs, const RSList& R) {
  std::vector<double> d(R.a.size());
  int nsp = R.sp_i.size();
#pragma omp parallel for schedule(dynamic)
  for (int sp = 0; sp < nsp; ++sp) {
    if (R.sp_count[sp] == 0) continue;  // a screened-out pair: no rows
    int i = R.sp_i[sp], j = R.sp_j[sp];
    std::vector<double> blk(quartet_size(bs, i, j, i, j));
    eri_quartet(bs, i, j, i, j, blk.data());
    for (int t = 0; t < R.sp_count[sp]; ++t) {
      int rs = R.sp_first[sp] + t;
      d[rs] = blk_elem(bs, blk.data(), i, j, i, j, R.a[rs], R.b[rs], R.a[rs], R.b[rs]);
    }
  }
  return d;
}

// --------------------------------------------------------------- gradient
// Cartesian 2-PDM for one shell quartet, primitive quartet loop with the
// derivative 2D integrals (Rysg1 + Rys2Dg + Assg1 + Distg1 restated).
void grad_quartet(const Basis& bs, int iS, int jS, int kS, int lS, const double* Dm, double scale, double* grad,
                  const double* Ds = nullptr, double coulfac = 1.0, double exfac = 1.0) {
  const Shell* S[4] = {&bs.sh[iS], &bs.sh[jS], &bs.sh[kS], &bs.sh[lS]};
  int l[4], ns[4], ncr[4], nc[4];
  for (int t = 0; t < 4; ++t) { l[t] = S[t]->l; ns[t] = nsph(l[t]); ncr[t] = ncart(l[t]); nc[t] = S[t]->nc; }
  size_t n = bs.nbf;
  // Gamma in contracted spherical form, [ijkl][a][b][c][d] (PGet1)
  int nijkl = nc[0] * nc[1] * nc[2] * nc[3];
  size_t nsp4 = (size_t)ns[0] * ns[1] * ns[2] * ns[3];
  std::vector<double> Gs((size_t)nijkl * nsp4);
  for (int md = 0; md < ns[3]; ++md) for (int mc = 0; mc < ns[2]; ++mc) for (int mb = 0; mb < ns[1]; ++mb) for (int ma = 0; ma < ns[0]; ++ma)
    for (int k4 = 0; k4 < nc[3]; ++k4) for (int k3 = 0; k3 < nc[2]; ++k3) for (int k2 = 0; k2 < nc[1]; ++k2) for (int k1 = 0; k1 < nc[0]; ++k1) {
      size_t p = ao_index(*S[0], k1, ma), q = ao_index(*S[1], k2, mb), r = ao_index(*S[2], k3, mc), s = ao_index(*S[3], k4, md);
      // CoulFac, ExFac and the spin density DSSO as in integral_util/pget1.F90:66-106
      double x = Dm[p * n + r] * Dm[q * n + s] + Dm[p * n + s] * Dm[q * n + r];
      if (Ds) x += Ds[p * n + r] * Ds[q * n + s] + Ds[p * n + s] * Ds[q * n + r];
      double g = coulfac * Dm[p * n + q] * Dm[r * n + s] - 0.25 * exfac * x;
      OR_FLOPS(FS_PDM, 8 + (Ds ? 4 : 0));
      int ijkl = k1 + nc[0] * (k2 + nc[1] * (k3 + nc[2] * k4));
      Gs[ijkl + (size_t)nijkl * (ma + ns[0] * (mb + (size_t)ns[1] * (mc + (size_t)ns[2] * md)))] = g;
    }
  // spherical -> Cartesian (SphCr1/SphCr2): Gc[ijkl][ca][cb][cc][cd]
  size_t ncr4 = (size_t)ncr[0] * ncr[1] * ncr[2] * ncr[3];
  std::vector<double> Gc((size_t)nijkl * ncr4, 0.0);
  for (int md = 0; md < ns[3]; ++md) for (int mc = 0; mc < ns[2]; ++mc) for (int mb = 0; mb < ns[1]; ++mb) for (int ma = 0; ma < ns[0]; ++ma)
    for (int cd = 0; cd < ncr[3]; ++cd) { double sd = g_sph[l[3]][cd + (size_t)ncr[3] * md]; if (sd == 0) continue;
    for (int cc = 0; cc < ncr[2]; ++cc) { double sc = g_sph[l[2]][cc + (size_t)ncr[2] * mc] * sd; OR_FLOPS(FS_PDM, 1); if (sc == 0) continue;
    for (int cb = 0; cb < ncr[1]; ++cb) { double sb = g_sph[l[1]][cb + (size_t)ncr[1] * mb] * sc; OR_FLOPS(FS_PDM, 1); if (sb == 0) continue;
    for (int ca = 0; ca < ncr[0]; ++ca) { double sa = g_sph[l[0]][ca + (size_t)ncr[0] * ma] * sb; OR_FLOPS(FS_PDM, 1); if (sa == 0) continue;
      size_t cidx = ca + ncr[0] * (cb + (size_t)ncr[1] * (cc + (size_t)ncr[2] * cd));
      size_t sidx = ma + ns[0] * (mb + (size_t)ns[1] * (mc + (size_t)ns[2] * md));
      for (int ijkl = 0; ijkl < nijkl; ++ijkl) Gc[ijkl + (size_t)nijkl * cidx] += sa * Gs[ijkl + (size_t)nijkl * sidx];
      OR_FLOPS(FS_PDM, 2 * nijkl);
    }}}}
  auto cl0 = cart_list(l[0]), cl1 = cart_list(l[1]), cl2 = cart_list(l[2]), cl3 = cart_list(l[3]);
  const double *A = S[0]->A, *B = S[1]->A, *C = S[2]->A, *D = S[3]->A;
  int emax = l[0] + l[1] + 1, fmax = l[2] + l[3] + 1;
  int nr = (l[0] + l[1] + l[2] + l[3] + 3) / 2;
  PairData pab = make_pair(*S[0], *S[1]), pcd = make_pair(*S[2], *S[3]);
  double AB[3], CD[3];
  for (int x = 0; x < 3; ++x) { AB[x] = A[x] - B[x]; CD[x] = C[x] - D[x]; }
  int na1 = l[0] + 2, nb1 = l[1] + 2, nc1 = l[2] + 2, nd1 = l[3] + 1;
  std::vector<double> Gp(ncr4);
  std::vector<double> H((size_t)3 * nr * na1 * nb1 * nc1 * nd1);
  auto h = [&](int c, int r, int a, int b, int cc, int d) -> double& {
    return H[(((((size_t)c * nr + r) * na1 + a) * nb1 + b) * nc1 + cc) * nd1 + d];
  };
  double x[16], w[16];
  TwoD G;
  double gq[9] = {0};
  for (int pq = 0; pq < pcd.np; ++pq) {
    int ic = pq % S[2]->np, id = pq / S[2]->np;
    double eta = pcd.zeta[pq], gam = pcd.alpha[pq];
    double Q[3] = {pcd.P[pq], pcd.P[pq + pcd.np], pcd.P[pq + 2 * pcd.np]};
    for (int pp = 0; pp < pab.np; ++pp) {
      int ia = pp % S[0]->np, ib = pp / S[0]->np;
      double zeta = pab.zeta[pp], alp = pab.alpha[pp], bet = pab.beta[pp];
      // de-contract Gamma (Tcrtnc)
      std::fill(Gp.begin(), Gp.end(), 0.0);
      bool nz = false;
      for (int k4 = 0; k4 < nc[3]; ++k4) for (int k3 = 0; k3 < nc[2]; ++k3) for (int k2 = 0; k2 < nc[1]; ++k2) for (int k1 = 0; k1 < nc[0]; ++k1) {
        double cf = S[0]->c[ia + S[0]->np * k1] * S[1]->c[ib + S[1]->np * k2] * S[2]->c[ic + S[2]->np * k3] * S[3]->c[id + S[3]->np * k4];
        OR_FLOPS(FS_PDM, 3);
        if (cf == 0.0) continue;
        nz = true;
        int ijkl = k1 + nc[0] * (k2 + nc[1] * (k3 + nc[2] * k4));
        for (size_t t = 0; t < ncr4; ++t) Gp[t] += cf * Gc[ijkl + (size_t)nijkl * t];
        OR_FLOPS(FS_PDM, 2 * ncr4);
      }
      if (!nz) continue;
      double P[3] = {pab.P[pp], pab.P[pp + pab.np], pab.P[pp + 2 * pab.np]};
      double ze = zeta + eta, tmp = 1.0 / ze, rho = zeta * eta * tmp;
      double PQ2 = (P[0] - Q[0]) * (P[0] - Q[0]) + (P[1] - Q[1]) * (P[1] - Q[1]) + (P[2] - Q[2]) * (P[2] - Q[2]);
      double T = rho * PQ2;
      double Fact = pab.kappa[pp] * pcd.kappa[pq] * std::sqrt(tmp);
      OR_FLOPS(FS_PRIM, 16);
      rys_rw(nr, T, x, w);
      rys2d(nr, emax, fmax, zeta, eta, P, Q, A, C, x, w, G);
      // 2D-level HRR (HRR2Da/HRR2Db): h(a,b,c,d) from G(e,f), e at A, f at C
      for (int c = 0; c < 3; ++c)
        for (int r = 0; r < nr; ++r) {
          // bra: I(a,b,f) with a+b<=emax
          std::vector<double> tb((size_t)(emax + 1) * nb1 * (fmax + 1), 0.0);
          auto TB = [&](int a, int b, int f) -> double& { return tb[((size_t)a * nb1 + b) * (fmax + 1) + f]; };
          for (int e = 0; e <= emax; ++e) for (int f = 0; f <= fmax; ++f) TB(e, 0, f) = G.at(c, r, e, f);
          for (int b = 1; b < nb1; ++b)
            for (int a = 0; a + b <= emax; ++a)
              for (int f = 0; f <= fmax; ++f) {
                TB(a, b, f) = TB(a + 1, b - 1, f) + AB[c] * TB(a, b - 1, f);
                OR_FLOPS(FS_TRANSFER, 2);
              }
          for (int a = 0; a < na1; ++a)
            for (int b = 0; b < nb1; ++b) {
              if (a + b > emax) continue;
              std::vector<double> tk((size_t)(fmax + 1) * nd1, 0.0);
              for (int f = 0; f <= fmax; ++f) tk[(size_t)f * nd1] = TB(a, b, f);
              for (int d = 1; d < nd1; ++d)
                for (int cc = 0; cc + d <= fmax; ++cc) {
                  tk[(size_t)cc * nd1 + d] = tk[(size_t)(cc + 1) * nd1 + d - 1] + CD[c] * tk[(size_t)cc * nd1 + d - 1];
                  OR_FLOPS(FS_TRANSFER, 2);
                }
              for (int cc = 0; cc < nc1; ++cc)
                for (int d = 0; d < nd1; ++d) if (cc + d <= fmax) h(c, r, a, b, cc, d) = tk[(size_t)cc * nd1 + d];
            }
        }
      // Assg1: sum over Cartesian components of Gamma x derivative products
      double ex[3] = {2 * alp, 2 * bet, 2 * gam};
      OR_FLOPS(FS_ASSG1, 3);
      for (int cd = 0; cd < ncr[3]; ++cd) for (int cc = 0; cc < ncr[2]; ++cc) for (int cb = 0; cb < ncr[1]; ++cb) for (int ca = 0; ca < ncr[0]; ++ca) {
        double g = Gp[ca + ncr[0] * (cb + (size_t)ncr[1] * (cc + (size_t)ncr[2] * cd))];
        if (g == 0.0) continue;
        int ai[3] = {cl0[ca].x, cl0[ca].y, cl0[ca].z}, bi[3] = {cl1[cb].x, cl1[cb].y, cl1[cb].z};
        int ci[3] = {cl2[cc].x, cl2[cc].y, cl2[cc].z}, di[3] = {cl3[cd].x, cl3[cd].y, cl3[cd].z};
        for (int r = 0; r < nr; ++r) {
          double v[3], dv[3][3];
          for (int c = 0; c < 3; ++c) {
            v[c] = h(c, r, ai[c], bi[c], ci[c], di[c]);
            dv[0][c] = ex[0] * h(c, r, ai[c] + 1, bi[c], ci[c], di[c]) - (ai[c] ? ai[c] * h(c, r, ai[c] - 1, bi[c], ci[c], di[c]) : 0.0);
            dv[1][c] = ex[1] * h(c, r, ai[c], bi[c] + 1, ci[c], di[c]) - (bi[c] ? bi[c] * h(c, r, ai[c], bi[c] - 1, ci[c], di[c]) : 0.0);
            dv[2][c] = ex[2] * h(c, r, ai[c], bi[c], ci[c] + 1, di[c]) - (ci[c] ? ci[c] * h(c, r, ai[c], bi[c], ci[c] - 1, di[c]) : 0.0);
            OR_FLOPS(FS_ASSG1, 6 + (ai[c] ? 1 : 0) + (bi[c] ? 1 : 0) + (ci[c] ? 1 : 0));
          }
          for (int X = 0; X < 3; ++X) {
            gq[3 * X + 0] += g * Fact * dv[X][0] * v[1] * v[2];
            gq[3 * X + 1] += g * Fact * v[0] * dv[X][1] * v[2];
            gq[3 * X + 2] += g * Fact * v[0] * v[1] * dv[X][2];
            OR_FLOPS(FS_ASSG1, 15);
          }
        }
      }
    }
  }
  // Distg1: translational invariance gives centre D
  int at[4] = {S[0]->atom, S[1]->atom, S[2]->atom, S[3]->atom};
  for (int c = 0; c < 3; ++c) {
    double gd = -(gq[c] + gq[3 + c] + gq[6 + c]);
    grad[3 * at[0] + c] += scale * gq[c];
    grad[3 * at[1] + c] += scale * gq[3 + c];
    grad[3 * at[2] + c] += scale * gq[6 + c];
    grad[3 * at[3] + c] += scale * gd;
    OR_FLOPS(FS_ASSG1, 10);
  }
  flops_commit();
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int or_load_rys(const char* path) { return load_rys(path); }

int or_rys_rw(int n, int npts, const double* T, double* x, double* w) {
  if (n < 1 || n > g_rys.nmax) return 1;
  for (int i = 0; i < npts; ++i) rys_rw(n, T[i], x + (size_t)i * n, w + (size_t)i * n);
  return 0;
}

int or_sph_matrix(int l, double* out) {  // ncart x (2l+1) column-major
  if ((int)g_sph.size() <= l) build_sph(std::max(l, 4));
  std::copy(g_sph[l].begin(), g_sph[l].end(), out);
  return 0;
}

// Basis: per shell centre xyz, l, nprim, ncontr, atom; exps concatenated;
// coefs concatenated (nprim x ncontr column-major per shell, normalised).
void* or_basis_create(int nshell, const double* xyz, const int* l, const int* np, const int* nc, const int* atom,
                      const double* exps, const double* coefs) {
  Handle* h = new Handle;
  int lmax = 0;
  size_t pe = 0, pc = 0;
  int off = 0, natom = 0;
  for (int s = 0; s < nshell; ++s) {
    Shell sh;
    for (int i = 0; i < 3; ++i) sh.A[i] = xyz[3 * s + i];
    sh.l = l[s]; sh.np = np[s]; sh.nc = nc[s]; sh.atom = atom[s];
    sh.e.assign(exps + pe, exps + pe + sh.np);
    sh.c.assign(coefs + pc, coefs + pc + (size_t)sh.np * sh.nc);
    pe += sh.np;
    pc += (size_t)sh.np * sh.nc;
    sh.off = off;
    off += sh.nc * nsph(sh.l);
    lmax = std::max(lmax, sh.l);
    natom = std::max(natom, sh.atom + 1);
    h->bs.sh.push_back(sh);
  }
  h->bs.nbf = off;
  h->bs.natom = natom;
  if ((int)g_sph.size() <= lmax + 1) build_sph(std::max(lmax + 1, 4));
  return h;
}
void or_basis_free(void* h) { delete (Handle*)h; }
int or_nbf(void* h) { return ((Handle*)h)->bs.nbf; }

int or_eri_quartet(void* h, int i, int j, int k, int l, double* out) {
  eri_quartet(((Handle*)h)->bs, i, j, k, l, out);
  return 0;
}
// cancellation-free magnitude of every integral of the block (same layout)
int or_eri_quartet_abs(void* h, int i, int j, int k, int l, double* out) {
  eri_quartet(((Handle*)h)->bs, i, j, k, l, out, true);
  return 0;
}

int or_schwarz(void* h, double* tmax) {
  Basis& bs = ((Handle*)h)->bs;
  if (bs.tmax.empty()) compute_tmax(bs);
  std::copy(bs.tmax.begin(), bs.tmax.end(), tmax);
  return 0;
}

// full ERI tensor (small systems only), Schwarz-screened at cutint
int or_eri_full(void* h, double cutint, double* full) {
  Basis& bs = ((Handle*)h)->bs;
  if (bs.tmax.empty()) compute_tmax(bs);
  int ns = bs.sh.size();
  size_t n = bs.nbf;
  std::fill(full, full + n * n * n * n, 0.0);
  std::vector<std::array<int, 4>> qs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= i; ++k)
        for (int l = 0; l <= (k == i ? j : k); ++l) {
          if (bs.tmax[(size_t)i * ns + j] * bs.tmax[(size_t)k * ns + l] < cutint) continue;
          qs.push_back({i, j, k, l});
        }
#pragma omp parallel for schedule(dynamic)
  for (size_t t = 0; t < qs.size(); ++t) {
    auto q = qs[t];
    std::vector<double> blk(quartet_size(bs, q[0], q[1], q[2], q[3]));
    eri_quartet(bs, q[0], q[1], q[2], q[3], blk.data());
    scatter_full(bs, q[0], q[1], q[2], q[3], blk.data(), full);
  }
  return 0;
}

// The rs list in use: the one of the handle's last decomposition (or of
// or_rs_compact), else every AO pair.
static RSList cur_rs(Handle* h) { return h->rs ? *h->rs : make_rs(h->bs); }

// Initial screening of the decomposition (cho_calcdiag.F90:255-300): elements
// with diag < ScrMax = ThrCom^2 / (Damp DiaMax) leave the reduced set; the
// vectors are stored over the shell pairs that keep at least one element.
static RSList screened_rs(const Basis& bs, double thrcom, double damp, std::vector<double>* diag_out) {
  RSList F = make_rs(bs);
  std::vector<double> d = eri_diag(bs, F);
  double dm = 0.0;
  for (double v : d) dm = std::max(dm, std::fabs(v));
  const double scrmax = dm > 0 ? thrcom * thrcom / damp / dm : 1e15;
  std::vector<char> keep(F.sp_i.size(), 0);
  for (size_t t = 0; t < d.size(); ++t)
    if (!(d[t] < scrmax)) keep[F.sp[t]] = 1;
  RSList R = make_rs(bs, &keep);
  if (diag_out) {
    diag_out->clear();
    for (size_t t = 0; t < d.size(); ++t)
      if (keep[F.sp[t]]) diag_out->push_back(d[t]);
  }
  return R;
}

// ERI diagonal over the rs list; returns nrs (fills a,b,sp if non-null)
int64_t or_rs_count(void* h) { return cur_rs((Handle*)h).a.size(); }
int or_rs_list(void* h, int* a, int* b, int* sp) {
  RSList R = cur_rs((Handle*)h);
  for (size_t t = 0; t < R.a.size(); ++t) { a[t] = R.a[t]; b[t] = R.b[t]; sp[t] = R.sp[t]; }
  return 0;
}
int or_eri_diag(void* h, double* d) {
  Basis& bs = ((Handle*)h)->bs;
  RSList R = cur_rs((Handle*)h);
  auto v = eri_diag(bs, R);
  std::copy(v.begin(), v.end(), d);
  return 0;
}
// the rs list a decomposition at thrcom would store its vectors over (no decomposition)
int or_rs_compact(void* h, double thrcom) {
  Handle* H = (Handle*)h;
  H->rs = std::make_shared<RSList>(screened_rs(H->bs, thrcom, cho_default_damp(thrcom), nullptr));
  return 0;
}

// Cholesky alg 4. Output: M, pivots[M] (rs index), pass[M], L (nrs x maxvec)
int or_cholesky_x(void* h, double thrcom, double span, int minqual, int maxqual, int mxshpr, int ialqua, int maxvec,
                  int* M_out, int* piv, int* pass_of, double* L, int* npass);
int or_cholesky(void* h, double thrcom, double span, int minqual, int maxqual, int maxvec, int* M_out, int* piv,
                int* pass_of, double* L, int* npass) {
  return or_cholesky_x(h, thrcom, span, minqual, maxqual, 1, 2, maxvec, M_out, piv, pass_of, L, npass);
}
// mxshpr: shell pairs qualified per pass (MXSHPR: 1 for algorithm 4,
// cho_inp.F90:709-715; 0 = no limit, algorithms 1-3); ialqua: qualification
// algorithm (IALQUA; 2 = the default, cho_inp.F90:156).  or_cholesky is (1, 2).
int or_cholesky_x(void* h, double thrcom, double span, int minqual, int maxqual, int mxshpr, int ialqua, int maxvec,
                  int* M_out, int* piv, int* pass_of, double* L, int* npass) {
  Basis& bs = ((Handle*)h)->bs;
  ChoCfg cfg;
  cfg.thrcom = thrcom; cfg.span = span; cfg.minqual = minqual; cfg.maxqual = maxqual; cfg.mxshpr = mxshpr;
  cfg.ialqua = ialqua;
  cfg.damp1 = cfg.damp2 = cho_default_damp(thrcom);
  cfg.thrneg = -1e-40; cfg.warneg = -1e-10; cfg.tooneg = -1e-8;
  std::vector<double> d;
  RSList R = screened_rs(bs, thrcom, cfg.damp1, &d);
  ((Handle*)h)->rs = std::make_shared<RSList>(R);
  ChoResult res = cho_decompose(bs, cfg, d, R);
  if (res.irc) return res.irc;
  if (res.M > maxvec) return 102;
  *M_out = res.M;
  *npass = res.npass;
  size_t nrs = R.a.size();
  for (int k = 0; k < res.M; ++k) {
    piv[k] = res.piv[k];
    pass_of[k] = res.pass_of[k];
    std::copy(res.L.begin() + nrs * k, res.L.begin() + nrs * (k + 1), L + nrs * k);
  }
  return 0;
}

// J, K (nbf x nbf) from vectors L (nrs x M) and density factor C (nbf x r,
// column-major): D = C C^T.  J_ab = sum_J L_ab,J V_J, V_J = sum_cd L_cd,J D_cd;
// K_ab = sum_J sum_k (L_J C)_ak (L_J C)_bk (CHO_LK_SCF without screening,
// cho_lk_scf.F90:442-449 and :507-830).  The loops are shaped like the DGEMV /
// DGEMM calls of the reference: vectors in batches, every inner loop a
// contiguous dot product (OpenMP SIMD), threads over rows.
static inline double dot_simd(const double* __restrict__ x, const double* __restrict__ y, int n) {
  double s = 0.0;
#pragma omp simd reduction(+ : s)
  for (int i = 0; i < n; ++i) s += x[i] * y[i];
  return s;
}

int or_cho_jk(void* h, const double* L, int M, const double* C, int r, double* J, double* K) {
  Basis& bs = ((Handle*)h)->bs;
  RSList R = cur_rs((Handle*)h);
  const size_t nrs = R.a.size();
  const int n = bs.nbf;
  std::vector<double> D((size_t)n * n, 0.0), Ct((size_t)n * r);
  for (int k = 0; k < r; ++k)
    for (int a = 0; a < n; ++a) Ct[(size_t)a * r + k] = C[a + (size_t)n * k];
#pragma omp parallel for schedule(static)
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < n; ++a) D[a + (size_t)n * b] = dot_simd(Ct.data() + (size_t)a * r, Ct.data() + (size_t)b * r, r);
  std::vector<double> Jrs(nrs, 0.0), Kl((size_t)n * n, 0.0);
  const int rp = (r + 7) / 8 * 8;  // C row-major, k contiguous, padded to 8
  std::vector<double> Cr((size_t)n * rp, 0.0);
  for (int b = 0; b < n; ++b)
    for (int k = 0; k < r; ++k) Cr[(size_t)b * rp + k] = C[b + (size_t)n * k];
  const int nvb = std::max(1, std::min(M, 16));  // vectors per batch
  const int np8 = (n + 7) / 8 * 8;
  std::vector<double> Lf((size_t)nvb * n * n), X((size_t)n * nvb * r), Xt((size_t)nvb * r * np8, 0.0), V(nvb);
  const int xr = nvb * r;
  for (int J0 = 0; J0 < M; J0 += nvb) {
    const int nb = std::min(nvb, M - J0);
    // unpack the batch's L_J into full symmetric squares; V_J (DGEMV)
#pragma omp parallel for schedule(static)
    for (int jb = 0; jb < nb; ++jb) {
      double* lf = Lf.data() + (size_t)jb * n * n;
      const double* l = L + nrs * (J0 + jb);
      double v = 0;
      for (size_t t = 0; t < nrs; ++t) {  // the stored (a >= b) half, column b contiguous in a
        const int a = R.a[t], b = R.b[t];
        lf[a + (size_t)n * b] = l[t];
        v += (a == b ? 1.0 : 2.0) * l[t] * D[a + (size_t)n * b];
      }
      V[jb] = v;
      for (int b0 = 0; b0 < n; b0 += 64)  // mirror into the upper half in 64 x 64 blocks
        for (int a0 = b0; a0 < n; a0 += 64)
          for (int b = b0; b < std::min(n, b0 + 64); ++b)
            for (int a = std::max(a0, b + 1); a < std::min(n, a0 + 64); ++a) lf[b + (size_t)n * a] = lf[a + (size_t)n * b];
    }
    // Coulomb accumulation (DGEMV): Jrs += L_batch V
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < (int64_t)nrs; ++t) {
      double s = 0;
      for (int jb = 0; jb < nb; ++jb) s += L[t + nrs * (J0 + jb)] * V[jb];
      Jrs[t] += s;
    }
    // half-transform X[a][jb*r + k] = sum_b L_J[b,a] C[b,k] (DGEMM; L_J symmetric):
    // 4 x 8 register blocks over (a, k), Cr = C row-major (k contiguous)
    const int na4 = (n + 3) / 4, nk8 = (r + 7) / 8;
#pragma omp parallel for schedule(static) collapse(3)
    for (int jb = 0; jb < nb; ++jb)
      for (int ab = 0; ab < na4; ++ab)
        for (int kb = 0; kb < nk8; ++kb) {
          const double* lf = Lf.data() + (size_t)jb * n * n;
          double acc[4][8] = {};
          int ai[4];
          for (int i = 0; i < 4; ++i) ai[i] = std::min(n - 1, 4 * ab + i);
          const int k0 = 8 * kb;
          for (int b = 0; b < n; ++b) {
            const double* cr = Cr.data() + (size_t)b * rp + k0;
#pragma GCC unroll 4
            for (int i = 0; i < 4; ++i) {
              const double l = lf[b + (size_t)n * ai[i]];
#pragma omp simd
              for (int j = 0; j < 8; ++j) acc[i][j] += l * cr[j];
            }
          }
          for (int i = 0; i < 4 && 4 * ab + i < n; ++i)
            for (int j = 0; j < 8 && k0 + j < r; ++j) X[(size_t)(4 * ab + i) * xr + (size_t)jb * r + k0 + j] = acc[i][j];
        }
    // exchange K[a,b] += sum_c X[a][c] X[b][c], b <= a (DSYRK): X transposed to
    // Xt[c][b] (b contiguous), then 4 x 8 register blocks over (a, b) as above
    const int kx = nb * r;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < kx; ++c)
      for (int b = 0; b < n; ++b) Xt[(size_t)c * np8 + b] = X[(size_t)b * xr + c];
    const int nb8 = (n + 7) / 8;
#pragma omp parallel for schedule(dynamic, 4) collapse(2)
    for (int ab = 0; ab < na4; ++ab)
      for (int bb = 0; bb < nb8; ++bb) {
        if (8 * bb > 4 * ab + 3) continue;
        int ai[4];
        for (int i = 0; i < 4; ++i) ai[i] = std::min(n - 1, 4 * ab + i);
        double acc[4][8] = {};
        for (int c = 0; c < kx; ++c) {
          const double* xt = Xt.data() + (size_t)c * np8 + 8 * bb;
#pragma GCC unroll 4
          for (int i = 0; i < 4; ++i) {
            const double x = X[(size_t)ai[i] * xr + c];
#pragma omp simd
            for (int j = 0; j < 8; ++j) acc[i][j] += x * xt[j];
          }
        }
        for (int i = 0; i < 4 && 4 * ab + i < n; ++i)
          for (int j = 0; j < 8 && 8 * bb + j <= 4 * ab + i; ++j) Kl[(size_t)(4 * ab + i) * n + 8 * bb + j] += acc[i][j];
      }
  }
  std::fill(J, J + (size_t)n * n, 0.0);
  for (size_t t = 0; t < nrs; ++t) {
    const int a = R.a[t], b = R.b[t];
    J[a + (size_t)n * b] = J[b + (size_t)n * a] = Jrs[t];
  }
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b) K[a + (size_t)n * b] = K[b + (size_t)n * a] = Kl[(size_t)a * n + b];
  return 0;
}

// dE/dR of E = 1/2 tr(DJ) - 1/4 tr(DK) with exact ERIs (Drvg1 path),
// D full nbf x nbf symmetric; grad[3*natom].  Quartets screened by
// tmax(ij) tmax(kl) < cutint.
int or_grad_sampled(void* h, const double* D, double cutint, int stride, double* grad, int64_t* nquartets);
static int grad_sampled_x(void* h, const double* D, const double* Ds, double coulfac, double exfac, double cutint,
                          int stride, double* grad, int64_t* nquartets);
int or_grad(void* h, const double* D, double cutint, double* grad) {
  return grad_sampled_x(h, D, nullptr, 1.0, 1.0, cutint, 1, grad, nullptr);
}
// the same with PGet1's full 2-PDM (integral_util/pget1.F90:66-106): spin
// density Ds (or null), CoulFac and ExFac
int or_grad_x(void* h, const double* D, const double* Ds, double coulfac, double exfac, double cutint, double* grad) {
  return grad_sampled_x(h, D, Ds, coulfac, exfac, cutint, 1, grad, nullptr);
}
// every stride-th unique quartet only (timing samples of the CPU baseline);
// *nquartets receives the total number of unique quartets after screening
int or_grad_sampled(void* h, const double* D, double cutint, int stride, double* grad, int64_t* nquartets) {
  return grad_sampled_x(h, D, nullptr, 1.0, 1.0, cutint, stride, grad, nquartets);
}
// the same starting at quartet `offset` (offset < stride): disjoint samples
static int g_sample_offset = 0;
int or_grad_sampled_at(void* h, const double* D, double cutint, int stride, int offset, double* grad,
                       int64_t* nquartets) {
  g_sample_offset = offset;
  const int rc = grad_sampled_x(h, D, nullptr, 1.0, 1.0, cutint, stride, grad, nquartets);
  g_sample_offset = 0;
  return rc;
}
static int grad_sampled_x(void* h, const double* D, const double* Ds, double coulfac, double exfac, double cutint,
                          int stride, double* grad, int64_t* nquartets) {
  Basis& bs = ((Handle*)h)->bs;
  if (bs.tmax.empty()) compute_tmax(bs);
  int ns = bs.sh.size();
  std::vector<std::array<int, 5>> qs;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j)
      for (int k = 0; k <= i; ++k)
        for (int l = 0; l <= (k == i ? j : k); ++l) {
          if (bs.tmax[(size_t)i * ns + j] * bs.tmax[(size_t)k * ns + l] < cutint) continue;
          int deg = (i == j ? 1 : 2) * (k == l ? 1 : 2) * ((i == k && j == l) ? 1 : 2);
          qs.push_back({i, j, k, l, deg});
        }
  if (nquartets) *nquartets = qs.size();
  if (stride > 1) {
    std::vector<std::array<int, 5>> sub;
    for (size_t t = g_sample_offset; t < qs.size(); t += stride) sub.push_back(qs[t]);
    qs.swap(sub);
  }
  int na = bs.natom;
  std::fill(grad, grad + 3 * na, 0.0);
#pragma omp parallel
  {
    std::vector<double> gl(3 * na, 0.0);
#pragma omp for schedule(dynamic)
    for (size_t t = 0; t < qs.size(); ++t) {
      auto q = qs[t];
      grad_quartet(bs, q[0], q[1], q[2], q[3], D, 0.5 * q[4], gl.data(), Ds, coulfac, exfac);
    }
#pragma omp critical
    for (int t = 0; t < 3 * na; ++t) grad[t] += gl[t];
  }
  return 0;
}

// Per-stage FP64 operation tally of the instrumented build (the FlopStage
// order: primitive set-up, roots, 2D recursion, RysEF, contraction, HRR +
// spherical, 2D transfers, Assg1 + Distg1, 2-PDM); returns the number of
// stages, or -1 in the default build.  reset != 0 clears the tally.
int or_flops(double* out, int reset) {
#ifdef OR_COUNT_FLOPS
  flops_commit();
  std::lock_guard<std::mutex> lk(g_flops_mu);
  for (int t = 0; t < FS_N; ++t) {
    out[t] = g_flops[t];
    if (reset) g_flops[t] = 0.0;
  }
  return FS_N;
#else
  (void)out;
  (void)reset;
  return -1;
#endif
}

int or_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
