// Pivoted Cholesky decomposition of the ERI matrix on the GPU with the
// semantics of OpenMolcas's default algorithm 4 (cholesky_util):
//
//   pass loop  CHO_DECDRV          cho_decdrv.F90:98-260
//   SetPass    max diag, DiaMin    cho_setpass.F90:29-47
//   GetMaxShl  one shell pair      cho_getmaxshl.F90, MXSHPR=1 (cho_inp.F90:709-715)
//   Qualify_2  diag >= DiaMin      cho_qualify_2.F90 (IALQUA = 2, cho_inp.F90:156), MaxQual = 100
//   columns    (CD|AB) all CD      cho_mca_calcint_1.F90 + PLF_Cho
//   Dec_Qual   Q = MQ - LQ LQ^T    cho_dec_qual.F90:57-83 (Thr = max(ThrCom, Dmax Span))
//   CD_InCore_1p pivot rule        cd_incore_1p.F90:33-85 (Acc tie rule, host FP64)
//   Subtr      X -= L LQ^T         cho_vecbuf_subtr.F90:188-215 (DGEMM)
//   CompVec    scale/diag update   cho_compvec.F90:40-120 + Cho_ChkDia_A4
//   SetRed     damped screening    cho_setred.F90:72-100 (MODE_SCREEN 1)
//
// Device work: ERI diagonal and columns (eri.cu kernels), column gather,
// DGEMM, row-parallel CompVec, reductions.  Host work per pass: the choice
// of shell pair, the qualification list and the in-core CD of the <=100 x 100
// qualified block (sequential, exact reference semantics).  Vectors are FP64
// in reduced-set ("rs") layout, blocks of kVecBlock columns.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "cho_qualify.h"
#include "kern_common.cuh"
#include "mg_internal.h"

namespace mg {

// from capi.cu

// ------------------------------------------------------------------ kernels
// rs descriptor: AO pair (a,b) with its shell pair and local indices
struct RsDev {
  int sp;          // shell pair id
  short ma, ka;    // component and contracted index of a in its shell
  short mb, kb;    // same for b
};

// diag[t] = (ab|ab) from the diagonal quartet blocks
__global__ void k_extract_diag(const RsDev* __restrict__ rs, int64_t nrs, const DPair* __restrict__ pairs,
                               const int64_t* __restrict__ blk_off, const double* __restrict__ blk,
                               double* __restrict__ diag) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  const RsDev r = rs[t];
  const DPair& P = pairs[r.sp];
  const int nij = P.nci * P.ncj;
  const int ij = r.ka + P.nci * r.kb;
  const int64_t ijkl = ij + (int64_t)nij * ij;
  const int64_t nijkl = (int64_t)nij * nij;
  const int sab = r.ma + P.nsa * r.mb;
  const int nsab = P.nsa * P.nsb;
  diag[t] = blk[blk_off[r.sp] + ijkl + nijkl * (sab + (int64_t)nsab * sab)];
}

// xint[t + nrs*q] = (row_t | col_q) from the (CD|AB) blocks; 0 outside the
// reduced set.  col: the rs index of each qualified column (all in pair AB).
__global__ void k_gather_columns(const RsDev* __restrict__ rs, int64_t nrs, const unsigned char* __restrict__ inred,
                                 const DPair* __restrict__ pairs, const int64_t* __restrict__ blk_off,
                                 const double* __restrict__ blk, const int* __restrict__ cols, int ncol, int spab,
                                 double* __restrict__ xint) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  if (!inred[t]) {
    for (int q = 0; q < ncol; ++q) xint[t + nrs * q] = 0.0;
    return;
  }
  const RsDev r = rs[t];
  const DPair& C = pairs[r.sp];
  const DPair& A = pairs[spab];
  const int64_t base = blk_off[r.sp];
  const int nij = C.nci * C.ncj, nkl = A.nci * A.ncj;
  const int64_t nijkl = (int64_t)nij * nkl;
  const int ij = r.ka + C.nci * r.kb;
  const int sab = r.ma + C.nsa * r.mb, nsab = C.nsa * C.nsb;
  for (int q = 0; q < ncol; ++q) {
    const RsDev c = rs[cols[q]];
    const int kl = c.ka + A.nci * c.kb;
    const int scd = c.ma + A.nsa * c.mb;
    xint[t + nrs * q] = blk[base + ij + (int64_t)nij * kl + nijkl * (sab + (int64_t)nsab * scd)];
  }
}

// block max over the reduced set: out[0] = max |diag|, out[1] = max diag
__global__ void k_red_max(const double* __restrict__ diag, const unsigned char* __restrict__ inred, int64_t n,
                          double* __restrict__ out) {
  __shared__ double s0[256], s1[256];
  double m0 = 0.0, m1 = -1e300;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    if (inred[t]) {
      m0 = fmax(m0, fabs(diag[t]));
      m1 = fmax(m1, diag[t]);
    }
  s0[threadIdx.x] = m0;
  s1[threadIdx.x] = m1;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s0[threadIdx.x] = fmax(s0[threadIdx.x], s0[threadIdx.x + w]);
      s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = s0[0];
    out[2 * blockIdx.x + 1] = s1[0];
  }
}

// per shell pair max diag over the reduced set (CHO_SETMAXSHL)
__global__ void k_sp_max(const double* __restrict__ diag, const unsigned char* __restrict__ inred,
                         const int64_t* __restrict__ sp_first, const int* __restrict__ sp_count, int nsp,
                         double* __restrict__ diash) {
  int sp = blockIdx.x * blockDim.x + threadIdx.x;
  if (sp >= nsp) return;
  // diash[sp]: max(0, largest diagonal) over the pair's members in the
  // reduced set, -1 when none is in it; diash[nsp + sp]: their largest |diagonal|
  double m = -1.0, ma = 0.0;
  const int64_t f = sp_first[sp];
  for (int i = 0; i < sp_count[sp]; ++i)
    if (inred[f + i]) {
      m = fmax(m, fmax(diag[f + i], 0.0));
      ma = fmax(ma, fabs(diag[f + i]));
    }
  diash[sp] = m;
  diash[nsp + sp] = ma;
}

// Cho_CompVec for one pass, one thread per rs row (rows are independent:
// the reference's per-vector steps touch each row only through its own
// diagonal).  X: nrs x nk (column-major, this pass's columns after Subtr).
// K: nk x nk lower triangular in-block vectors; fac[i] = 1/sqrt(|QDiag_i|);
// qrs[i]: parent rs of vector i.  flags[0] set if a diagonal < TooNeg.
__global__ void k_compvec(double* __restrict__ X, int64_t nrs, int nk, const double* __restrict__ K,
                          const double* __restrict__ fac, const int* __restrict__ qrs, double* __restrict__ diag,
                          const unsigned char* __restrict__ inred, double qdmax, double damp, double thrcom,
                          double thrneg, double tooneg, int* __restrict__ flags) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nrs) return;
  if (!inred[t]) {  // vectors are zero outside the reduced set of their pass
    for (int i = 0; i < nk; ++i) X[t + nrs * i] = 0.0;
    return;
  }
  double d = diag[t];
  for (int i = 0; i < nk; ++i) {
    double x = X[t + nrs * i] * fac[i];
    if (d == 0.0) x = 0.0;
    d -= x * x;
    if (t == qrs[i]) d = 0.0;  // Cho_P_ZeroDiag
    if (d < 0.0 && d < thrneg) {  // Cho_ChkDia_A4
      if (d < tooneg) atomicOr(flags, 1);
      d = 0.0;
    }
    if (sqrt(fabs(d) * qdmax) * damp <= thrcom) d = 0.0;
    X[t + nrs * i] = x;
    for (int j = i + 1; j < nk; ++j) X[t + nrs * j] -= K[j + nk * i] * x;
  }
  diag[t] = d;
}

// Cho_SetRed mode 1 (no abs): keep diag > 0 with sqrt(diag*xm)*damp > thrcom
__global__ void k_setred(const double* __restrict__ diag, unsigned char* __restrict__ inred, int64_t n, double xm,
                         double damp, double thrcom, int conv) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (!inred[t]) return;
  const double d = diag[t];
  inred[t] = (!conv && d > 0.0 && sqrt(d * xm) * damp > thrcom) ? 1 : 0;
}

__global__ void k_init_red(double* __restrict__ diag, unsigned char* __restrict__ inred, int64_t n, double scrmax) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (diag[t] < scrmax) {
    diag[t] = 0.0;
    inred[t] = 0;
  } else {
    inred[t] = 1;
  }
}

// gather LQ rows: lq[i + nq*J] = L[qrow[i] + nrs*J]
__global__ void k_gather_rows(const double* __restrict__ L, int64_t nrs, int ncol, const int* __restrict__ rows, int nq,
                              double* __restrict__ lq) {
  int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (o >= (int64_t)nq * ncol) return;
  const int i = (int)(o % nq);
  const int64_t J = o / nq;
  lq[o] = L[rows[i] + nrs * J];
}

static inline unsigned nblk(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// --------------------------------------------------------------- host side
struct ChoState {
  int64_t nrs = 0;
  std::vector<int> rs_a, rs_b, rs_sp;
  std::vector<int64_t> sp_first;
  std::vector<int> sp_count;
  RsDev* d_rs = nullptr;
  int* d_rs_a = nullptr;        // AO indices of each rs entry (device)
  int* d_rs_b = nullptr;
  int64_t* d_sp_first = nullptr;
  int* d_sp_count = nullptr;
  double* d_diag = nullptr;     // working diagonal
  double* d_diag0 = nullptr;    // exact (ab|ab)
  unsigned char* d_inred = nullptr;
  std::vector<double*> Lblk;    // FP64 vector blocks, nrs x kVecBlock each
  int M = 0;
  std::vector<int> piv, pass_of;
  int npass = 0;
  cublasHandle_t cublas = nullptr;
  short* d_lexp = nullptr;      // row exponents of the square L_J (mixed J/K), M x lexp_ld
  int lexp_ld = 0;
};

static const int kVecBlock = 1024;

void cho_free(ChoState* c) {
  if (!c) return;
  cudaFree(c->d_rs); cudaFree(c->d_sp_first); cudaFree(c->d_sp_count); cudaFree(c->d_rs_a); cudaFree(c->d_rs_b);
  cudaFree(c->d_diag); cudaFree(c->d_diag0); cudaFree(c->d_inred); cudaFree(c->d_lexp);
  for (auto p : c->Lblk) cudaFree(p);
  if (c->cublas) cublasDestroy(c->cublas);
  delete c;
}

// AO-pair list in reduced-set order (plf_cho_diag.F90:60-72 conventions):
// every shell pair (keep == nullptr) or the shell pairs with keep[sp] set
// (the others get sp_first = -1 and no rows).  Replaces a previous list.
static void make_rs(Handle* h, ChoState* c, const std::vector<char>* keep = nullptr) {
  cudaFree(c->d_rs_a); cudaFree(c->d_rs_b); cudaFree(c->d_rs); cudaFree(c->d_sp_first); cudaFree(c->d_sp_count);
  c->rs_a.clear(); c->rs_b.clear(); c->rs_sp.clear(); c->sp_first.clear(); c->sp_count.clear();
  const int ns = h->sh.size();
  std::vector<RsDev> rsd;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j <= i; ++j) {
      const int sp = pair_id(i, j);
      if (keep && !(*keep)[sp]) {
        c->sp_first.push_back(-1);
        c->sp_count.push_back(0);
        continue;
      }
      const ShellH &A = h->sh[i], &B = h->sh[j];
      const int nA = A.nc * A.ncomp, nB = B.nc * B.ncomp;
      c->sp_first.push_back(c->rs_a.size());
      auto push = [&](int la, int lb) {
        c->rs_a.push_back(A.off + la);
        c->rs_b.push_back(B.off + lb);
        c->rs_sp.push_back(sp);
        RsDev r;
        r.sp = sp;
        r.ma = la / A.nc; r.ka = la % A.nc;
        r.mb = lb / B.nc; r.kb = lb % B.nc;
        rsd.push_back(r);
      };
      if (i != j) {
        for (int lb = 0; lb < nB; ++lb)
          for (int la = 0; la < nA; ++la) push(la, lb);
      } else {
        for (int la = 0; la < nA; ++la)
          for (int lb = 0; lb <= la; ++lb) push(la, lb);
      }
      c->sp_count.push_back((int)(c->rs_a.size() - c->sp_first.back()));
    }
  c->nrs = c->rs_a.size();
  dev_malloc(&c->d_rs_a, sizeof(int) * c->nrs);
  dev_malloc(&c->d_rs_b, sizeof(int) * c->nrs);
  cudaMemcpy(c->d_rs_a, c->rs_a.data(), sizeof(int) * c->nrs, cudaMemcpyHostToDevice);
  cudaMemcpy(c->d_rs_b, c->rs_b.data(), sizeof(int) * c->nrs, cudaMemcpyHostToDevice);
  dev_malloc(&c->d_rs, sizeof(RsDev) * c->nrs);
  cudaMemcpy(c->d_rs, rsd.data(), sizeof(RsDev) * c->nrs, cudaMemcpyHostToDevice);
  dev_malloc(&c->d_sp_first, sizeof(int64_t) * c->sp_first.size());
  cudaMemcpy(c->d_sp_first, c->sp_first.data(), sizeof(int64_t) * c->sp_first.size(), cudaMemcpyHostToDevice);
  dev_malloc(&c->d_sp_count, sizeof(int) * c->sp_count.size());
  cudaMemcpy(c->d_sp_count, c->sp_count.data(), sizeof(int) * c->sp_count.size(), cudaMemcpyHostToDevice);
}

// ERI blocks (q4 quartets) into a scratch buffer; offsets per quartet
static double* eri_blocks(Handle* h, const std::vector<int32_t>& q4, std::vector<int64_t>& off, double*& buf,
                          size_t& bufsz, cudaStream_t st, int& rc) {
  const int64_t nq = q4.size() / 4;
  off.assign(nq + 1, 0);
  for (int64_t t = 0; t < nq; ++t) {
    int64_t n = 1;
    for (int x = 0; x < 4; ++x) n *= (int64_t)h->sh[q4[4 * t + x]].nc * h->sh[q4[4 * t + x]].ncomp;
    off[t + 1] = off[t] + n;
  }
  const size_t need = sizeof(double) * std::max<int64_t>(off[nq], 1);
  if (need > bufsz) {
    cudaStreamSynchronize(st);
    cudaFree(buf);
    buf = nullptr;
    if (dev_malloc(&buf, need) != cudaSuccess) { rc = MG_ERR_MEMORY; bufsz = 0; return nullptr; }
    bufsz = need;
  }
  std::vector<EriItem> items;
  std::vector<EriClass> classes;
  rc = build_eri_items(h, q4.data(), nq, off.data(), items, classes);
  if (rc) return nullptr;
  rc = run_eri_items(h, items, classes, buf, st);
  return buf;
}

static double cho_default_damp(double thrcom) {  // cho_setdamp.F90
  if (thrcom > 9.99e-3) return 1e7;
  if (thrcom > 9.99e-4) return 1e6;
  if (thrcom > 9.99e-5) return 1e5;
  if (thrcom > 9.99e-6) return 1e4;
  if (thrcom > 9.99e-7) return 1e3;
  if (thrcom > 9.99e-8) return 1e2;
  if (thrcom > 9.99e-9) return 1e1;
  return 1.0;
}

// CD_InCore_1p on the host (identical arithmetic to the reference)
static int cd_incore_1p(std::vector<double>& X, int n, std::vector<double>& Vec, int& numcho, double thr,
                        std::vector<int>& iD) {
  const double thrneg = -1e-13, thrfail = -1e-8;
  numcho = 0;
  const double acc = std::min(1e-12, thr * 1e-2);
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
    const double xfac = 1.0 / std::sqrt(std::fabs(xmax));
    for (int j = 0; j < numcho; ++j) {
      const double v = Vec[imax + (size_t)n * j];
      for (int t = 0; t < n; ++t) x(t, imax) -= v * Vec[t + (size_t)n * j];
    }
    x(imax, imax) = xmax;
    const int k = numcho++;
    for (int i = 0; i < n; ++i) Vec[i + (size_t)n * k] = (x(i, i) == 0.0) ? 0.0 : xfac * x(i, imax);
    for (int i = 0; i < n; ++i) x(i, i) -= Vec[i + (size_t)n * k] * Vec[i + (size_t)n * k];
    x(imax, imax) = 0.0;
    iD.push_back(imax);
  }
  return 0;
}

static double red_max(const double* d_diag, const unsigned char* d_inred, int64_t n, double* d_tmp, int which,
                      cudaStream_t st) {
  const int nb = 296;
  k_red_max<<<nb, 256, 0, st>>>(d_diag, d_inred, n, d_tmp);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  std::vector<double> h(2 * nb);
  cudaMemcpyAsync(h.data(), d_tmp, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  double m = which == 0 ? 0.0 : -1e300;
  for (int b = 0; b < nb; ++b) m = std::max(m, h[2 * b + which]);
  return m;
}

int cho_decompose(Handle* h, const ChoCfgH& cfg, ChoState*& out, cudaStream_t st, std::string& err) {
  ChoState* c = new ChoState;
  out = c;
  make_rs(h, c);
  const int nsp = c->sp_count.size();
  const double damp = cho_default_damp(cfg.thrcom);
  if (cublasCreate(&c->cublas) != CUBLAS_STATUS_SUCCESS) { err = "cublasCreate failed"; return MG_ERR_CUDA; }
  cublasSetStream(c->cublas, st);
  double* d_tmp = nullptr;
  dev_malloc(&d_tmp, sizeof(double) * std::max<int64_t>(2 * 296, 2 * (int64_t)nsp));
  double* buf = nullptr;
  size_t bufsz = 0;
  int rc = 0;
  // ---- diagonal (CHO_GETDIAG): (AB|AB) for every shell pair, then the initial
  // screening (cho_calcdiag.F90:255-300): elements below
  // ScrMax = ThrCom^2 / (Damp DiaMax) leave the reduced set.  The vectors are
  // stored over the shell pairs that keep at least one element (their rows
  // outside a pass's reduced set are zero), so the rs list is rebuilt over them.
  double scrmax = 1e15;
  {
    std::vector<int32_t> q4;
    for (int sp = 0; sp < nsp; ++sp) {
      const int i = h->pairs[sp].i, j = h->pairs[sp].j;
      q4.insert(q4.end(), {i, j, i, j});
    }
    std::vector<int64_t> off;
    eri_blocks(h, q4, off, buf, bufsz, st, rc);
    if (rc) { err = "diagonal integrals failed: " + err; cudaFree(buf); cudaFree(d_tmp); return rc; }
    int64_t* d_off = nullptr;
    dev_malloc(&d_off, sizeof(int64_t) * nsp);
    cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * nsp, cudaMemcpyHostToDevice, st);
    // full diagonal, every shell pair
    double* d_full = nullptr;
    dev_malloc(&d_full, sizeof(double) * c->nrs);
    k_extract_diag<<<nblk(c->nrs), 256, 0, st>>>(c->d_rs, c->nrs, h->d_pairs, d_off, buf, d_full);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    std::vector<double> hd(c->nrs);
    cudaMemcpyAsync(hd.data(), d_full, sizeof(double) * c->nrs, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    cudaFree(d_full);
    double dm = 0;
    for (double v : hd) dm = std::max(dm, std::fabs(v));
    if (dm > 0) scrmax = cfg.thrcom * cfg.thrcom / damp / dm;
    std::vector<char> keep(nsp, 0);
    for (int64_t t = 0; t < c->nrs; ++t)
      if (!(hd[t] < scrmax)) keep[c->rs_sp[t]] = 1;
    make_rs(h, c, &keep);
    // the diagonal over the kept shell pairs, from the same integral blocks
    dev_malloc(&c->d_diag, sizeof(double) * std::max<int64_t>(c->nrs, 1));
    dev_malloc(&c->d_diag0, sizeof(double) * std::max<int64_t>(c->nrs, 1));
    dev_malloc(&c->d_inred, std::max<int64_t>(c->nrs, 1));
    k_extract_diag<<<nblk(std::max<int64_t>(c->nrs, 1)), 256, 0, st>>>(c->d_rs, c->nrs, h->d_pairs, d_off, buf,
                                                                        c->d_diag0);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaMemcpyAsync(c->d_diag, c->d_diag0, sizeof(double) * c->nrs, cudaMemcpyDeviceToDevice, st);
    cudaStreamSynchronize(st);
    cudaFree(d_off);
  }
  const int64_t nrs = c->nrs;
  k_init_red<<<nblk(std::max<int64_t>(nrs, 1)), 256, 0, st>>>(c->d_diag, c->d_inred, nrs, scrmax);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  int* d_flags = nullptr;
  dev_malloc(&d_flags, sizeof(int));
  cudaMemsetAsync(d_flags, 0, sizeof(int), st);
  double *d_xint = nullptr, *d_X = nullptr, *d_K = nullptr, *d_fac = nullptr, *d_lq = nullptr, *d_Q = nullptr;
  int *d_cols = nullptr, *d_qrs = nullptr;
  int64_t* d_off = nullptr;
  dev_malloc(&d_off, sizeof(int64_t) * nsp);
  const int MQ = cfg.maxqual;
  dev_malloc(&d_xint, sizeof(double) * nrs * MQ);
  dev_malloc(&d_X, sizeof(double) * nrs * MQ);
  dev_malloc(&d_K, sizeof(double) * MQ * MQ);
  dev_malloc(&d_fac, sizeof(double) * MQ);
  dev_malloc(&d_cols, sizeof(int) * MQ);
  dev_malloc(&d_qrs, sizeof(int) * MQ);
  dev_malloc(&d_Q, sizeof(double) * MQ * MQ);
  dev_malloc(&d_lq, sizeof(double) * (size_t)MQ * kVecBlock);
  std::vector<double> hdiash(2 * (size_t)nsp), hq;
  std::vector<int64_t> off_sp(nsp);
  auto Lcol = [&](int J) -> double* { return c->Lblk[J / kVecBlock] + (size_t)nrs * (J % kVecBlock); };
  for (int pass = 0; pass <= nrs; ++pass) {
    // ---- Cho_SetPass: the largest reduced-set diagonal of every shell pair
    // (-1: no member in the reduced set); their maximum is the pass's DGMax
    k_sp_max<<<nblk(nsp), 256, 0, st>>>(c->d_diag, c->d_inred, c->d_sp_first, c->d_sp_count, nsp, d_tmp);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaMemcpyAsync(hdiash.data(), d_tmp, sizeof(double) * 2 * nsp, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    double dgmax = 0.0;  // max |diagonal| over the reduced set
    for (int sp = 0; sp < nsp; ++sp) dgmax = std::max(dgmax, hdiash[nsp + sp]);
    if (dgmax < cfg.thrcom) break;
    const double diamin = std::max(dgmax * cfg.span, cfg.thrcom);
    double smax = -1e9;
    int spab = -1;
    for (int sp = 0; sp < nsp; ++sp) {
      const double v = hdiash[sp] > cfg.thrcom ? hdiash[sp] : 0.0;
      if (v > smax) { smax = v; spab = sp; }
    }
    if (smax == 0.0 || std::fabs(smax) < diamin) { rc = MG_ERR_DECOMP; err = "no qualifying diagonal (Cho_GetInt 104)"; break; }
    // ---- Cho_Qualify_2 within shell pair spab (cho_qualify.h)
    const int64_t f = c->sp_first[spab];
    const int cnt = c->sp_count[spab];
    std::vector<double> dpair(cnt);
    std::vector<unsigned char> rpair(cnt);
    cudaMemcpyAsync(dpair.data(), c->d_diag + f, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(rpair.data(), c->d_inred + f, cnt, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    // positions t inside the pair, then rs indices
    std::vector<int> qual = cho_qualify_2(dpair.data(), rpair.data(), cnt, diamin, cfg.maxqual);
    for (int& t : qual) t = (int)(f + t);
    const int nq = qual.size();
    if (nq == 0) { rc = MG_ERR_DECOMP; err = "empty qualification (Cho_GetInt 104)"; break; }
    // ---- integral columns (CD|AB) for every CD pair touching the reduced set
    // (the reduced set has not changed since the shell-pair maxima above)
    std::vector<int32_t> q4;
    std::vector<int> qsp;
    for (int sp = 0; sp < nsp; ++sp) {
      if (hdiash[sp] < 0.0) continue;
      q4.insert(q4.end(), {h->pairs[sp].i, h->pairs[sp].j, h->pairs[spab].i, h->pairs[spab].j});
      qsp.push_back(sp);
    }
    std::vector<int64_t> off;
    eri_blocks(h, q4, off, buf, bufsz, st, rc);
    if (rc) { err = "column integrals failed: " + err; break; }
    std::fill(off_sp.begin(), off_sp.end(), -1);
    for (size_t t = 0; t < qsp.size(); ++t) off_sp[qsp[t]] = off[t];
    cudaMemcpyAsync(d_off, off_sp.data(), sizeof(int64_t) * nsp, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_cols, qual.data(), sizeof(int) * nq, cudaMemcpyHostToDevice, st);
    k_gather_columns<<<nblk(nrs), 256, 0, st>>>(c->d_rs, nrs, c->d_inred, h->d_pairs, d_off, buf, d_cols, nq, spab,
                                                d_xint);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    // ---- Cho_Dec_Qual: Q = MQ - LQ LQ^T  (MQ = xint rows at the qualified positions)
    const int M = c->M;
    // MQ (rows of the qualified columns) then Q -= LQ LQ^T on the device
    std::vector<double> Q((size_t)nq * nq);
    k_gather_rows<<<nblk((int64_t)nq * nq), 256, 0, st>>>(d_xint, nrs, nq, d_cols, nq, d_Q);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    for (int b = 0; b * kVecBlock < M; ++b) {
      const int nc = std::min(kVecBlock, M - b * kVecBlock);
      k_gather_rows<<<nblk((int64_t)nq * nc), 256, 0, st>>>(c->Lblk[b], nrs, nc, d_cols, nq, d_lq);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      const double one = 1.0, mone = -1.0;
      cublasDgemm(c->cublas, CUBLAS_OP_N, CUBLAS_OP_T, nq, nq, nc, &mone, d_lq, nq, d_lq, nq, &one, d_Q, nq);
    }
    cudaMemcpyAsync(Q.data(), d_Q, sizeof(double) * nq * nq, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    std::vector<double> qdiag(nq);
    for (int q = 0; q < nq; ++q) qdiag[q] = Q[q + (size_t)nq * q];
    const double dmax = red_max(c->d_diag, c->d_inred, nrs, d_tmp, 1, st);  // Cho_P_MaxDX
    const double thr = std::max(cfg.thrcom, dmax * cfg.span);
    std::vector<double> Vec((size_t)nq * nq, 0.0);
    std::vector<int> iD;
    int nk = 0;
    if (cd_incore_1p(Q, nq, Vec, nk, thr, iD)) { rc = MG_ERR_DECOMP; err = "CD_InCore_1p failed (negative diagonal)"; break; }
    if (nk == 0) { rc = MG_ERR_DECOMP; err = "no vector from qualified block"; break; }
    if (M + nk > cfg.maxvec) { rc = MG_ERR_MEMORY; err = "too many Cholesky vectors (MaxVec)"; break; }
    // pivot order (cho_decom_a4.F90:120-170)
    std::vector<double> K((size_t)nk * nk), fac(nk), qd(nk);
    std::vector<int> qrs(nk), colsel(nk);
    for (int i = 0; i < nk; ++i)
      for (int j = 0; j < nk; ++j) K[j + (size_t)nk * i] = Vec[iD[j] + (size_t)nq * i];
    for (int i = 0; i < nk; ++i) { qd[i] = qdiag[iD[i]]; qrs[i] = qual[iD[i]]; colsel[i] = iD[i]; }
    const double qdmax = qd[0];
    for (int i = 0; i < nk; ++i) {
      fac[i] = 1.0 / std::sqrt(std::fabs(qd[i]));
      for (int j = i; j < nk; ++j) qd[j] -= K[j + (size_t)nk * i] * K[j + (size_t)nk * i];
      qd[i] = 0.0;
    }
    // destination columns of this pass
    while ((int)c->Lblk.size() * kVecBlock < M + nk) {
      double* p = nullptr;
      if (dev_malloc(&p, sizeof(double) * nrs * kVecBlock) != cudaSuccess) { rc = MG_ERR_MEMORY; break; }
      cudaMemsetAsync(p, 0, sizeof(double) * nrs * kVecBlock, st);
      c->Lblk.push_back(p);
    }
    if (rc) { err = "out of device memory for Cholesky vectors"; break; }
    // X[:, i] = xint[:, iD[i]] (pivot order, Cho_RdQCol_Indx) in a contiguous scratch
    for (int i = 0; i < nk; ++i)
      cudaMemcpyAsync(d_X + nrs * i, d_xint + nrs * colsel[i], sizeof(double) * nrs, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(d_qrs, qrs.data(), sizeof(int) * nk, cudaMemcpyHostToDevice, st);
    // ---- Cho_Subtr: X -= L_prev LQ^T  (DGEMM per vector block)
    for (int b = 0; b * kVecBlock < M; ++b) {
      const int ncb = std::min(kVecBlock, M - b * kVecBlock);
      k_gather_rows<<<nblk((int64_t)nk * ncb), 256, 0, st>>>(c->Lblk[b], nrs, ncb, d_qrs, nk, d_lq);
      g_launches.fetch_add(1, std::memory_order_relaxed);
      const double mone = -1.0, one = 1.0;
      cublasDgemm(c->cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)nrs, nk, ncb, &mone, c->Lblk[b], (int)nrs, d_lq, nk, &one,
                  d_X, (int)nrs);
    }
    // ---- Cho_CompVec (row-parallel)
    cudaMemcpyAsync(d_K, K.data(), sizeof(double) * nk * nk, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_fac, fac.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st);
    k_compvec<<<nblk(nrs), 256, 0, st>>>(d_X, nrs, nk, d_K, d_fac, d_qrs, c->d_diag, c->d_inred, qdmax, damp,
                                        cfg.thrcom, -1e-40, -1e-8, d_flags);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    for (int i = 0; i < nk; ++i)
      cudaMemcpyAsync(Lcol(M + i), d_X + nrs * i, sizeof(double) * nrs, cudaMemcpyDeviceToDevice, st);
    for (int i = 0; i < nk; ++i) { c->piv.push_back(qrs[i]); c->pass_of.push_back(pass); }
    c->M = M + nk;
    c->npass = pass + 1;
    // ---- Cho_SetRed (damped screening)
    const double xm = red_max(c->d_diag, c->d_inred, nrs, d_tmp, 0, st);
    k_setred<<<nblk(nrs), 256, 0, st>>>(c->d_diag, c->d_inred, nrs, xm, damp, cfg.thrcom, xm > cfg.thrcom ? 0 : 1);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    int hflag = 0;
    cudaMemcpyAsync(&hflag, d_flags, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if (hflag) { rc = MG_ERR_DECOMP; err = "diagonal too negative (Cho_ChkDia_A4 TooNeg)"; break; }
    if (cudaGetLastError() != cudaSuccess) { rc = MG_ERR_CUDA; err = "CUDA error in Cholesky pass"; break; }
  }
  cudaStreamSynchronize(st);
  cudaFree(buf); cudaFree(d_tmp); cudaFree(d_flags); cudaFree(d_xint); cudaFree(d_X); cudaFree(d_K); cudaFree(d_fac);
  cudaFree(d_lq); cudaFree(d_Q); cudaFree(d_cols); cudaFree(d_qrs); cudaFree(d_off);
  return rc;
}

int64_t cho_nrs(const ChoState* c) { return c->nrs; }
int cho_nvec(const ChoState* c) { return c->M; }
int cho_npass(const ChoState* c) { return c->npass; }
void cho_pivots(const ChoState* c, int32_t* piv, int32_t* pass_of) {
  for (int k = 0; k < c->M; ++k) {
    if (piv) piv[k] = c->piv[k];
    if (pass_of) pass_of[k] = c->pass_of[k];
  }
}
void cho_rs_list(const ChoState* c, int32_t* a, int32_t* b, int32_t* sp) {
  for (int64_t t = 0; t < c->nrs; ++t) {
    if (a) a[t] = c->rs_a[t];
    if (b) b[t] = c->rs_b[t];
    if (sp) sp[t] = c->rs_sp[t];
  }
}
int cho_copy_vectors(const ChoState* c, int first, int count, double* d_out, cudaStream_t st) {
  if (first < 0 || count < 0 || first + count > c->M) return MG_ERR_ARG;
  for (int k = 0; k < count; ++k) {
    const int J = first + k;
    cudaMemcpyAsync(d_out + c->nrs * k, c->Lblk[J / kVecBlock] + (size_t)c->nrs * (J % kVecBlock),
                    sizeof(double) * c->nrs, cudaMemcpyDeviceToDevice, st);
  }
  return 0;
}
const double* cho_diag0(const ChoState* c) { return c->d_diag0; }
cublasHandle_t cho_cublas(ChoState* c) { return c->cublas; }
const int* cho_rs_a_dev(const ChoState* c) { return c->d_rs_a; }
const int* cho_rs_b_dev(const ChoState* c) { return c->d_rs_b; }
// contiguous FP64 vectors [J0, J0+nb) (the range must not cross a storage block)
const double* cho_vec_ptr(const ChoState* c, int J0, int nb, cudaStream_t, Handle*) {
  if (J0 / kVecBlock != (J0 + nb - 1) / kVecBlock) return nullptr;
  return c->Lblk[J0 / kVecBlock] + (size_t)c->nrs * (J0 % kVecBlock);
}
int cho_vec_block() { return kVecBlock; }
const int64_t* cho_sp_first_dev(const ChoState* c) { return c->d_sp_first; }
short* cho_lexp(const ChoState* c, int ld) { return c->lexp_ld == ld ? c->d_lexp : nullptr; }
void cho_set_lexp(ChoState* c, short* p, int ld) {
  cudaFree(c->d_lexp);
  c->d_lexp = p;
  c->lexp_ld = ld;
}

// ------------------------------------------------- in-core decomposition
// CD_InCore (cholesky_util/cd_incore.F90:14 -> cd_incore_1.F90): pivoted
// Cholesky factor of a symmetric positive semidefinite n x n matrix X, left
// looking: each step takes the largest remaining diagonal (the first one,
// in index order, that exceeds the running maximum by more than
// Acc = min(1e-12, Thr/100)), updates only the pivot column against the
// previous vectors, scales it into the new vector and subtracts its square
// from the diagonal; diagonals below ThrNeg = -1e-13 are zeroed with their
// row and column, below ThrFail = -1e-8 the decomposition fails (irc 101);
// it stops when the largest diagonal is <= Thr.  One CTA: thread 0 scans the
// diagonal (shared memory) in index order, as the tie rule needs; the column
// update, the new vector and the diagonal update are row-parallel.
// out[0] = NumCho, out[1] = irc (0, 101, 102).
constexpr int kCdThreads = 1024;

__global__ void __launch_bounds__(kCdThreads) k_cd_incore(double* __restrict__ X, int n, double* __restrict__ Vec,
                                                          int maxvec, double thr, int* __restrict__ out) {
  extern __shared__ double cd_dg[];  // the diagonal of X, then n ints of zeroed indices
  int* zl = reinterpret_cast<int*>(cd_dg + n);
  __shared__ int s_imax, s_stop, s_nz;
  __shared__ double s_xmax;
  const double thrneg = -1.0e-13, thrfail = -1.0e-8;
  const double acc = fmin(1.0e-12, thr * 1.0e-2);
  for (int i = threadIdx.x; i < n; i += blockDim.x) cd_dg[i] = X[i + (size_t)n * i];
  __syncthreads();
  int numcho = 0, irc = 0;
  for (int pass = 0; pass < n; ++pass) {
    if (threadIdx.x == 0) {
      int nz = 0, imax = -1, stop = 0;
      double xmax = 0.0;
      for (int i = 0; i < n; ++i) {
        double d = cd_dg[i];
        if (d < thrneg) {
          if (d < thrfail) {
            stop = 101;
            break;
          }
          d = 0.0;
          cd_dg[i] = 0.0;
          zl[nz++] = i;
        }
        if (d > xmax + acc) {
          xmax = d;
          imax = i;
        }
      }
      if (!stop && xmax <= thr) stop = 1;  // converged
      if (!stop && numcho == maxvec) stop = 102;
      s_imax = imax;
      s_xmax = xmax;
      s_stop = stop;
      s_nz = nz;
    }
    __syncthreads();
    if (s_stop) {
      irc = s_stop == 1 ? 0 : s_stop;
      break;
    }
    for (int z = 0; z < s_nz; ++z) {  // rows and columns of the zeroed diagonals
      const int iz = zl[z];
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        X[k + (size_t)n * iz] = 0.0;
        X[iz + (size_t)n * k] = 0.0;
      }
    }
    __syncthreads();
    const int imax = s_imax;
    const double xmax = s_xmax, xfac = 1.0 / sqrt(fabs(xmax));
    double* vnew = Vec + (size_t)n * numcho;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double x = X[i + (size_t)n * imax];
      for (int j = 0; j < numcho; ++j) x -= Vec[imax + (size_t)n * j] * Vec[i + (size_t)n * j];
      if (i == imax) x = xmax;
      X[i + (size_t)n * imax] = x;
      const double v = cd_dg[i] == 0.0 ? 0.0 : xfac * x;
      vnew[i] = v;
      cd_dg[i] -= v * v;
    }
    __syncthreads();
    if (threadIdx.x == 0) cd_dg[imax] = 0.0;
    ++numcho;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = numcho;
    out[1] = irc;
  }
}

int cd_incore(Handle* h, double* d_X, int n, double thr, double* d_vec, int maxvec, int* numcho, cudaStream_t st) {
  *numcho = 0;
  if (n < 1) return 0;
  if (maxvec < 1) return -1;
  if (thr < 0.0) thr = 1.0e-6;  // CD_InCore's DefThr
  const size_t smem = (size_t)n * (sizeof(double) + sizeof(int));
  if (smem > 200 * 1024) {
    h->err = "in-core decomposition: n above 17066";
    return MG_ERR_ARG;
  }
  if (!smem_attr_once((const void*)k_cd_incore, 200 * 1024)) {
    h->err = "in-core decomposition: shared-memory limit could not be raised";
    return MG_ERR_CUDA;
  }
  int* d_out = (int*)ws_get(h, 2 * sizeof(int), st);
  if (!d_out) { h->err = "workspace allocation failed"; return MG_ERR_MEMORY; }
  k_cd_incore<<<1, kCdThreads, smem, st>>>(d_X, n, d_vec, maxvec, thr, d_out);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  int hout[2] = {0, 0};
  cudaMemcpyAsync(hout, d_out, sizeof(hout), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
    h->err = "in-core decomposition: CUDA error";
    return MG_ERR_CUDA;
  }
  *numcho = hout[0];
  return hout[1];
}

}  // namespace mg
