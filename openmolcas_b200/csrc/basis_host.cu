// Host-side basis set-up for libmolgpu: Rys table, real-spherical matrices,
// canonical shell pairs (DoZeta data, contraction products, HRR matrices).
//
// Conventions follow OpenMolcas:
//  * DoZeta (integral_util/dozeta.F90:36-52): zeta = a + b,
//    kappa = sqrt(2) pi^(5/4) exp(-ab |AB|^2 / zeta) / zeta (floored at
//    1e-99), P = (a A + b B) / zeta; primitive pairs alpha-fastest.
//  * HrrMtrx (integral_util/hrrmtrx.F90:61-100): transfer onto the centre of
//    higher l with binomial (A-B)^k factors, folded with the
//    Cartesian->spherical matrix; e-range [max(la,lb), la+lb] (only la+lb
//    when A == B, twoel_nosym.F90:252-259).
//  * Real_Sphere (integral_util/real_spherical.F90:182-420): m = -l..l,
//    Condon-Shortley phase off; s and p shells stay Cartesian
//    (gateway_util/rdctl_seward.F90:3863-3865).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "mg_internal.h"

namespace mg {

static int cind(int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }
static double dfac(int n) {
  double r = 1;
  for (int i = n; i > 1; i -= 2) r *= i;
  return r;
}
static double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

int load_rys_table(Handle* h, const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) { h->err = std::string("cannot open Rys table ") + path; return 1; }
  char magic[8];
  int32_t hdr[2];
  bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "RYSTAB01", 8) == 0 && fread(hdr, 4, 2, f) == 2;
  if (!ok || hdr[0] < 1 || hdr[0] > MG_MAX_RYS || hdr[1] != 7) { fclose(f); h->err = "bad Rys table header"; return 2; }
  int nmax = hdr[0];
  h->rys_nmax = nmax;
  h->rys_degree = hdr[1];
  int off = 0;
  for (int n = 1; n <= nmax; ++n) {
    double hd[2];
    int32_t K;
    if (fread(hd, 8, 2, f) != 2 || fread(&K, 4, 1, f) != 1) { fclose(f); h->err = "bad Rys table"; return 3; }
    RysMeta& m = h->rys_meta[n - 1];
    m.h = hd[0];
    m.invh = 1.0 / hd[0];
    m.tmax = hd[1];
    m.K = K;
    m.off = off;
    off += K * 2 * n * (h->rys_degree + 1);
  }
  for (int n = 1; n <= nmax; ++n) {
    RysMeta& m = h->rys_meta[n - 1];
    if (fread(m.hx, 8, n, f) != (size_t)n || fread(m.hw, 8, n, f) != (size_t)n) { fclose(f); h->err = "bad Rys table"; return 4; }
  }
  std::vector<double> coef(off);
  if (fread(coef.data(), 8, off, f) != (size_t)off) { fclose(f); h->err = "truncated Rys table"; return 5; }
  fclose(f);
  if (dev_malloc(&h->d_rys, sizeof(double) * off) != cudaSuccess) { h->err = "cudaMalloc rys"; return 6; }
  cudaMemcpy(h->d_rys, coef.data(), sizeof(double) * off, cudaMemcpyHostToDevice);
  return 0;
}

void build_sph(Handle* h, int lmax) {
  std::vector<std::vector<double>> P0(lmax + 1);
  for (int n = 0; n <= lmax; ++n) {
    P0[n].assign(ncart(n), 0.0);
    if (n == 0) { P0[0][0] = 1.0; continue; }
    const double f1 = double(2 * n - 1) / n;
    for (int ix = n - 1; ix >= 0; --ix)
      for (int iy = n - 1 - ix; iy >= 0; --iy) P0[n][cind(iy, n - 1 - ix - iy + 1)] += f1 * P0[n - 1][cind(iy, n - 1 - ix - iy)];
    if (n >= 2) {
      const double f2 = double(n - 1) / n;
      for (int ix = n - 2; ix >= 0; --ix)
        for (int iy = n - 2 - ix; iy >= 0; --iy) {
          int iz = n - 2 - ix - iy;
          double v = P0[n - 2][cind(iy, iz)];
          P0[n][cind(iy, iz)] -= f2 * v;
          P0[n][cind(iy + 2, iz)] -= f2 * v;
          P0[n][cind(iy, iz + 2)] -= f2 * v;
        }
    }
  }
  for (int n = 0; n <= lmax; ++n) {
    const int nc = ncart(n);
    std::vector<std::vector<double>> Pm(2 * n + 1, std::vector<double>(nc, 0.0));
    Pm[n] = P0[n];
    for (int m = 0; m < n; ++m) {
      std::vector<double>& Pp = Pm[n + m + 1];
      std::vector<double>& Pn = Pm[n - m - 1];
      const std::vector<double> Pc = Pm[n + m], Pcm = Pm[n - m];
      const double fact = 1.0 / (2.0 * std::sqrt(double(n * (n + 1) - m * (m - 1))));
      for (int ix = n; ix >= 0; --ix)
        for (int iy = n - ix; iy >= 0; --iy) {
          const int iz = n - ix - iy;
          const double pm = Pc[cind(iy, iz)], pmm = Pcm[cind(iy, iz)];
          if (iz >= 1) Pp[cind(iy, iz - 1)] += fact * iz * pm;
          if (ix >= 1) Pp[cind(iy, iz + 1)] -= fact * ix * pm;
          if (m != 0) {
            if (iz >= 1) Pp[cind(iy + 1, iz - 1)] -= fact * iz * pmm;
            if (iy >= 1) Pp[cind(iy - 1, iz + 1)] += fact * iy * pmm;
          }
          if (iz >= 1) Pn[cind(iy + 1, iz - 1)] += fact * iz * pm;
          if (iy >= 1) Pn[cind(iy - 1, iz + 1)] -= fact * iy * pm;
          if (m != 0) {
            if (iz >= 1) Pn[cind(iy, iz - 1)] += fact * iz * pmm;
            if (ix >= 1) Pn[cind(iy, iz + 1)] -= fact * ix * pmm;
          }
        }
    }
    // normalise in the double-factorial metric of unnormalised Cartesians
    std::vector<int> cx, cy, cz;
    for (int lx = n; lx >= 0; --lx)
      for (int ly = n - lx; ly >= 0; --ly) { cx.push_back(lx); cy.push_back(ly); cz.push_back(n - lx - ly); }
    for (auto& P : Pm) {
      double rmax = 0;
      for (double v : P) rmax = std::max(rmax, std::fabs(v));
      for (double& v : P) if (std::fabs(v) < 1e-12 * rmax) v = 0.0;
      double t = 0;
      for (int i = 0; i < nc; ++i)
        for (int j = 0; j < nc; ++j) {
          int ex = cx[i] + cx[j], ey = cy[i] + cy[j], ez = cz[i] + cz[j];
          if ((ex | ey | ez) & 1) continue;
          t += P[i] * P[j] * dfac(ex - 1) * dfac(ey - 1) * dfac(ez - 1);
        }
      for (double& v : P) v /= std::sqrt(t);
    }
    const int nco = ncomp(n);
    h->sph[n].assign((size_t)nc * nco, 0.0);
    if (n <= 1) {
      for (int i = 0; i < nc; ++i) h->sph[n][i + (size_t)nc * i] = 1.0;
    } else {
      for (int m = 0; m < 2 * n + 1; ++m)
        for (int c = 0; c < nc; ++c) h->sph[n][c + (size_t)nc * m] = Pm[m][c];
    }
  }
}

std::vector<double> hrr_matrix(const Handle* h, int la, int lb, const double* A, const double* B, int& ne, int& emin) {
  const bool AeqB = A[0] == B[0] && A[1] == B[1] && A[2] == B[2];
  emin = AeqB ? la + lb : std::max(la, lb);
  const int emax = la + lb;
  ne = ncart_cum(emax + 1) - ncart_cum(emin);
  const int joff = ncart_cum(emin);
  const int lta = ncart(la), ltb = ncart(lb), na = ncomp(la), nb = ncomp(lb);
  std::vector<double> H((size_t)ne * na * nb, 0.0);
  double AB[3];
  for (int x = 0; x < 3; ++x) AB[x] = la >= lb ? A[x] - B[x] : B[x] - A[x];
  auto pw = [](double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; };
  auto carts = [](int l) {
    std::vector<int> v;
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) { v.push_back(lx); v.push_back(ly); v.push_back(l - lx - ly); }
    return v;
  };
  auto c3 = [](int x, int y, int z) { int l = x + y + z; return ncart_cum(l) + cind(y, z); };
  const std::vector<int> ca = carts(la), cb = carts(lb);
  const std::vector<double>& Sa = h->sph[la];
  const std::vector<double>& Sb = h->sph[lb];
  for (int sa = 0; sa < na; ++sa)
    for (int ia = 0; ia < lta; ++ia) {
      const double Ca = Sa[ia + (size_t)lta * sa];
      if (Ca == 0.0) continue;
      for (int sb = 0; sb < nb; ++sb)
        for (int ib = 0; ib < ltb; ++ib) {
          const double Cb = Sb[ib + (size_t)ltb * sb];
          if (Cb == 0.0) continue;
          const int* keep = la >= lb ? &ca[3 * ia] : &cb[3 * ib];
          const int* tran = la >= lb ? &cb[3 * ib] : &ca[3 * ia];
          int lo[3];
          for (int x = 0; x < 3; ++x) lo[x] = AeqB ? keep[x] + tran[x] : keep[x];
          for (int kx = lo[0]; kx <= keep[0] + tran[0]; ++kx)
            for (int ky = lo[1]; ky <= keep[1] + tran[1]; ++ky)
              for (int kz = lo[2]; kz <= keep[2] + tran[2]; ++kz) {
                const double f = pw(AB[0], keep[0] + tran[0] - kx) * binom(tran[0], kx - keep[0]) *
                                 pw(AB[1], keep[1] + tran[1] - ky) * binom(tran[1], ky - keep[1]) *
                                 pw(AB[2], keep[2] + tran[2] - kz) * binom(tran[2], kz - keep[2]);
                H[(c3(kx, ky, kz) - joff) + (size_t)ne * (sa + (size_t)na * sb)] += f * Ca * Cb;
              }
        }
    }
  return H;
}

// Primitive-pair prescreening (the role of Screen, integral_util/
// screen.F90:109-148): a primitive pair p of shell pair AB is dropped when
//   s_p * S / sqrt(zeta_p + zeta_min) * 1e3 < kPrimThr,
// s_p = kappa_p * max_ij |C_i(a) C_j(b)| * (1 + |AB| + zeta_p^-1/2)^(la+lb),
// S = max over all primitive pairs of s_q.  s_p s_q / sqrt(zeta+eta) bounds
// |[ab|cd]| of the primitive quartet (F_m <= 1, polynomial factors bounded
// generously), so every dropped contribution is below 1e-21.
static const double kPrimThr = 1e-18;

int setup_pairs(Handle* h) {
  const int ns = h->sh.size();
  const double twop54 = std::sqrt(2.0) * std::pow(M_PI, 1.25);
  h->pairs.clear();
  // pass 1: bounds
  struct PP { double s, z; };
  std::vector<std::vector<PP>> est(ns * (ns + 1) / 2);
  double Smax = 0, zmin = 1e300;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      const ShellH &a = h->sh[i], &b = h->sh[j];
      double AB2 = 0;
      for (int x = 0; x < 3; ++x) AB2 += (a.A[x] - b.A[x]) * (a.A[x] - b.A[x]);
      auto& v = est[pair_id(i, j)];
      for (int jb = 0; jb < b.np; ++jb)
        for (int ia = 0; ia < a.np; ++ia) {
          const double x = a.e[ia], y = b.e[jb], z = x + y;
          const double k = std::max(twop54 * std::exp(-x * y * AB2 / z) / z, 1e-99);
          double cm = 0;
          for (int kb = 0; kb < b.nc; ++kb)
            for (int ka = 0; ka < a.nc; ++ka) cm = std::max(cm, std::fabs(a.c[ia + a.np * ka] * b.c[jb + b.np * kb]));
          const double ang = std::pow(1.0 + std::sqrt(AB2) + 1.0 / std::sqrt(z), a.l + b.l);
          v.push_back({k * cm * ang, z});
          Smax = std::max(Smax, k * cm * ang);
          zmin = std::min(zmin, z);
        }
    }
  std::vector<double> zeta, kappa, px, py, pz, al, be, coef, hrr;
  long long kept = 0, total = 0;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      const ShellH &a = h->sh[i], &b = h->sh[j];
      const auto& v = est[pair_id(i, j)];
      std::vector<int> keep;
      int best = 0;
      for (int p = 0; p < (int)v.size(); ++p) {
        if (v[p].s > v[best].s) best = p;
        if (v[p].s * Smax / std::sqrt(v[p].z + zmin) * 1e3 >= kPrimThr) keep.push_back(p);
      }
      if (keep.empty()) keep.push_back(best);
      total += v.size();
      kept += keep.size();
      DPair d{};
      d.i = i; d.j = j; d.la = a.l; d.lb = b.l; d.na = a.np; d.nb = b.np; d.nci = a.nc; d.ncj = b.nc;
      d.np = keep.size();
      d.prim_off = zeta.size();
      d.coef_off = coef.size();
      d.nsa = ncomp(a.l); d.nsb = ncomp(b.l);
      d.aeqb = a.A[0] == b.A[0] && a.A[1] == b.A[1] && a.A[2] == b.A[2];
      for (int x = 0; x < 3; ++x) { d.A[x] = a.A[x]; d.B[x] = b.A[x]; d.Ap[x] = a.l >= b.l ? a.A[x] : b.A[x]; }
      d.atom_a = a.atom; d.atom_b = b.atom; d.ao_a = a.off; d.ao_b = b.off;
      double AB2 = 0;
      for (int x = 0; x < 3; ++x) AB2 += (a.A[x] - b.A[x]) * (a.A[x] - b.A[x]);
      for (int p : keep) {
        const int ia = p % a.np, jb = p / a.np;
        const double x = a.e[ia], y = b.e[jb], z = x + y, zi = 1.0 / z;
        double k = twop54 * std::exp(-x * y * AB2 * zi) * zi;
        if (k < 1e-99) k = 1e-99;
        zeta.push_back(z); kappa.push_back(k); al.push_back(x); be.push_back(y);
        px.push_back((x * a.A[0] + y * b.A[0]) * zi);
        py.push_back((x * a.A[1] + y * b.A[1]) * zi);
        pz.push_back((x * a.A[2] + y * b.A[2]) * zi);
      }
      for (int kb = 0; kb < b.nc; ++kb)
        for (int ka = 0; ka < a.nc; ++ka)
          for (int p : keep) {
            const int ia = p % a.np, jb = p / a.np;
            coef.push_back(a.c[ia + a.np * ka] * b.c[jb + b.np * kb]);
          }
      int ne, emin;
      std::vector<double> H = hrr_matrix(h, a.l, b.l, a.A, b.A, ne, emin);
      d.ne = ne; d.emin = emin;
      d.hrr_off = hrr.size();
      hrr.insert(hrr.end(), H.begin(), H.end());
      h->pairs.push_back(d);
    }
  h->prim_kept = kept;
  h->prim_total = total;
  h->tot_np = zeta.size();
  std::vector<double> izeta(zeta.size());
  for (size_t i = 0; i < zeta.size(); ++i) izeta[i] = 1.0 / zeta[i];
  std::vector<double> prim;
  for (auto* v : {&zeta, &kappa, &px, &py, &pz, &al, &be, &izeta}) prim.insert(prim.end(), v->begin(), v->end());
  if (dev_malloc(&h->d_prim, sizeof(double) * prim.size()) != cudaSuccess ||
      dev_malloc(&h->d_coef, sizeof(double) * std::max<size_t>(coef.size(), 1)) != cudaSuccess ||
      dev_malloc(&h->d_hrr, sizeof(double) * std::max<size_t>(hrr.size(), 1)) != cudaSuccess ||
      dev_malloc(&h->d_pairs, sizeof(DPair) * h->pairs.size()) != cudaSuccess) {
    h->err = "cudaMalloc pair data";
    return 1;
  }
  cudaMemcpy(h->d_prim, prim.data(), sizeof(double) * prim.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_coef, coef.data(), sizeof(double) * coef.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_hrr, hrr.data(), sizeof(double) * hrr.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(h->d_pairs, h->pairs.data(), sizeof(DPair) * h->pairs.size(), cudaMemcpyHostToDevice);
  return 0;
}

void* ws_get(Handle* h, size_t bytes, cudaStream_t st) {
  if (bytes <= h->ws.size) return h->ws.ptr;
  if (h->ws.ptr) {
    cudaStreamSynchronize(st);
    cudaFree(h->ws.ptr);
  }
  h->ws.ptr = nullptr;
  h->ws.size = 0;
  size_t sz = std::max(bytes, (size_t)1 << 20);
  if (dev_malloc(&h->ws.ptr, sz) != cudaSuccess) return nullptr;
  h->ws.size = sz;
  return h->ws.ptr;
}

}  // namespace mg
