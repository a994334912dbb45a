// C ABI of libmolgpu: handle, basis, Schwarz bounds, batched ERIs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/molgpu.h"
#include "mg_internal.h"

struct mg_handle {
  mg::Handle h;
};

namespace mg {
std::atomic<long long> g_launches{0};
std::atomic<long long> g_allocs{0};

// Accumulator budget (doubles) of one work item: nc * nef <= this.
static const int kAccBudget = 12288;


// Split quartets into work items grouped by (la+lb, lc+ld) class; a work
// item covers a range of the ket contracted-pair index kl.
int build_eri_items(Handle* h, const int32_t* q4, int64_t nq, const int64_t* offsets, std::vector<EriItem>& items,
                    std::vector<EriClass>& classes) {
  std::vector<std::vector<EriItem>> byc(64);
  std::vector<ClassStats> st(64);
  const int ns = h->sh.size();
  for (int64_t t = 0; t < nq; ++t) {
    const int i = q4[4 * t], j = q4[4 * t + 1], k = q4[4 * t + 2], l = q4[4 * t + 3];
    if (i < 0 || j < 0 || k < 0 || l < 0 || i >= ns || j >= ns || k >= ns || l >= ns || i < j || k < l) {
      h->err = "mg_eri_quartets: shell indices out of range or non-canonical pair (need i>=j, k>=l)";
      return MG_ERR_ARG;
    }
    const int p = pair_id(i, j), q = pair_id(k, l);
    const DPair& P = h->pairs[p];
    const DPair& Q = h->pairs[q];
    const int nab = P.la + P.lb, ncd = Q.la + Q.lb;
    const int nef = P.ne * Q.ne;
    const int nij = P.nci * P.ncj, nkl = Q.nci * Q.ncj;
    if (nij * nef > kAccBudget) {
      h->err = "mg_eri_quartets: bra contraction block too large";
      return MG_ERR_ARG;
    }
    const int chunk = std::max(1, kAccBudget / (nij * nef));
    const int key = nab * 8 + ncd;
    ClassStats& cs = st[key];
    for (int c0 = 0; c0 < nkl; c0 += chunk) {
      EriItem it;
      it.p = p;
      it.q = q;
      it.c0 = c0;
      it.c1 = std::min(nkl, c0 + chunk);
      it.out_off = offsets[t];
      byc[key].push_back(it);
      const int nklc = it.c1 - it.c0;
      cs.max_acc = std::max(cs.max_acc, nij * nklc * nef);
      cs.max_nef = std::max(cs.max_nef, nef);
      cs.max_tmp = std::max(cs.max_tmp, nij * nklc * P.nsa * P.nsb * Q.ne);
      cs.max_nij = std::max(cs.max_nij, nij);
      cs.max_npab = std::max(cs.max_npab, P.np);
      cs.max_npcd = std::max(cs.max_npcd, Q.np);
      cs.max_cab = std::max(cs.max_cab, nij * P.np);
      cs.max_ccd = std::max(cs.max_ccd, nklc * Q.np);
      cs.max_ne = std::max(cs.max_ne, P.ne);
      cs.max_nf = std::max(cs.max_nf, Q.ne);
      cs.max_nc = std::max(cs.max_nc, nij * nklc);
      // primitive quartets x roots x (e0|f0) components, plus the contraction
      cs.work += (double)P.np * Q.np * (nab + ncd + 2) / 2 * nef + (double)nij * nklc * nef;
    }
  }
  items.clear();
  classes.clear();
  for (int key = 0; key < 64; ++key) {
    auto& v = byc[key];
    if (v.empty()) continue;
    EriClass c;
    c.nab = key / 8;
    c.ncd = key % 8;
    c.begin = items.size();
    c.count = v.size();
    c.plan = eri_plan(c.nab, c.ncd, st[key], h->eri_tpq[key], h->eri_order[key]);
    c.work = st[key].work;
    if (c.plan.PAB < 1) {
      h->err = "mg_eri_quartets: class does not fit in shared memory";
      return MG_ERR_ARG;
    }
    // heaviest quartets first so the groups of one CTA carry similar work
    std::stable_sort(v.begin(), v.end(), [&](const EriItem& a, const EriItem& b) {
      const long long wa = (long long)h->pairs[a.p].np * h->pairs[a.q].np * (a.c1 - a.c0);
      const long long wb = (long long)h->pairs[b.p].np * h->pairs[b.q].np * (b.c1 - b.c0);
      return wa > wb;
    });
    items.insert(items.end(), v.begin(), v.end());
    classes.push_back(c);
  }
  return 0;
}

int run_eri_items(Handle* h, const std::vector<EriItem>& items, const std::vector<EriClass>& classes, double* d_out,
                  cudaStream_t st) {
  if (items.empty()) return 0;
  if (!h->d_eri_counters && dev_malloc(&h->d_eri_counters, sizeof(int) * 64) != cudaSuccess) {
    h->err = "ERI work counters: allocation failed";
    return MG_ERR_MEMORY;
  }
  EriItem* d_items = (EriItem*)ws_get(h, sizeof(EriItem) * items.size(), st);
  if (!d_items) { h->err = "workspace allocation failed"; return MG_ERR_MEMORY; }
  cudaMemcpyAsync(d_items, items.data(), sizeof(EriItem) * items.size(), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(h->d_eri_counters, 0, sizeof(int) * 64, st);
  // The class kernels are independent (own counter, own output blocks): spread them over
  // the handle's side streams so that the tail of one class overlaps the next class,
  // the largest classes first (the small ones fill in behind them).
  int rc = side_streams_fork(h, st);
  if (rc) return rc;
  std::vector<int> order(classes.size());
  for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return classes[a].work > classes[b].work; });
  // profiled (mg_eri_profile): every class on the caller's stream between its own events
  if (h->eri_profile) {
    while (h->eri_ev.size() < 2 * classes.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) { h->err = "ERI profiling events"; return MG_ERR_CUDA; }
      h->eri_ev.push_back(e);
    }
    h->eri_ev_key.assign(classes.size(), 0);
    h->eri_ev_plan.assign(classes.size(), ClassPlan{});
    h->eri_ev_used = (int)classes.size();
  }
  for (size_t k = 0; k < order.size(); ++k) {
    const int ci = order[k];
    const EriClass& c = classes[ci];
    const cudaStream_t ks = h->eri_profile ? st : h->eri_streams[k % MG_ERI_STREAMS];
    if (h->eri_profile) {
      h->eri_ev_key[k] = c.nab * 8 + c.ncd;
      h->eri_ev_plan[k] = c.plan;
      cudaEventRecord(h->eri_ev[2 * k], ks);
    }
    if (eri_launch_class(h, d_items + c.begin, c.count, c.nab, c.ncd, c.plan, d_out, h->d_eri_counters + ci, ks)) {
      h->err = std::string("ERI kernel launch failed: ") + cudaGetErrorString(cudaGetLastError());
      return MG_ERR_CUDA;
    }
    if (h->eri_profile) cudaEventRecord(h->eri_ev[2 * k + 1], ks);
  }
  side_streams_join(h, st);
  return 0;
}

int side_streams_fork(Handle* h, cudaStream_t st) {
  if (!h->eri_streams[0]) {
    for (int k = 0; k < MG_ERI_STREAMS; ++k) {
      if (cudaStreamCreateWithFlags(&h->eri_streams[k], cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&h->eri_events[k], cudaEventDisableTiming) != cudaSuccess) {
        h->err = "side streams could not be created";
        return MG_ERR_CUDA;
      }
    }
    if (cudaEventCreateWithFlags(&h->eri_fork, cudaEventDisableTiming) != cudaSuccess) {
      h->err = "side streams could not be created";
      return MG_ERR_CUDA;
    }
  }
  cudaEventRecord(h->eri_fork, st);
  for (int k = 0; k < MG_ERI_STREAMS; ++k) cudaStreamWaitEvent(h->eri_streams[k], h->eri_fork, 0);
  return 0;
}

void side_streams_join(Handle* h, cudaStream_t st) {
  for (int k = 0; k < MG_ERI_STREAMS; ++k) {
    cudaEventRecord(h->eri_events[k], h->eri_streams[k]);
    cudaStreamWaitEvent(st, h->eri_events[k], 0);
  }
}

}  // namespace mg

using namespace mg;

extern "C" {

int mg_create(const char* rys_table_path, int device, mg_handle** out) {
  if (!out || !rys_table_path) return MG_ERR_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return MG_ERR_CUDA;
  mg_handle* H = new mg_handle;
  H->h.device = device;
  int rc = load_rys_table(&H->h, rys_table_path);
  if (rc) {
    delete H;
    return MG_ERR_ARG;
  }
  *out = H;
  return 0;
}

static void free_basis(Handle* h) {
  cho_free(h->cho);
  h->cho = nullptr;
  grad_free(h->grad);
  h->grad = nullptr;
  cudaFree(h->d_pairs); cudaFree(h->d_prim); cudaFree(h->d_coef); cudaFree(h->d_hrr); cudaFree(h->d_tmax);
  h->d_pairs = nullptr; h->d_prim = nullptr; h->d_coef = nullptr; h->d_hrr = nullptr; h->d_tmax = nullptr;
  h->tmax.clear();
}

int mg_destroy(mg_handle* H) {
  if (!H) return 0;
  Handle* h = &H->h;
  cudaSetDevice(h->device);
  free_basis(h);
  cudaFree(h->d_rys);
  cudaFree(h->d_eri_counters);
  cudaFree(h->d_lk);
  cudaFree(h->d_dcd);
  for (int k = 0; k < MG_ERI_STREAMS; ++k) {
    if (h->eri_streams[k]) cudaStreamDestroy(h->eri_streams[k]);
    if (h->eri_events[k]) cudaEventDestroy(h->eri_events[k]);
  }
  if (h->eri_fork) cudaEventDestroy(h->eri_fork);
  for (cudaEvent_t e : h->grad_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : h->eri_ev) cudaEventDestroy(e);
  if (h->ws.ptr) cudaFree(h->ws.ptr);
  delete H;
  return 0;
}

const char* mg_last_error(mg_handle* H) { return H ? H->h.err.c_str() : "null handle"; }

int mg_set_basis(mg_handle* H, int nshell, const double* xyz, const int* l, const int* nprim, const int* ncontr,
                 const int* atom, const double* exps, const double* coefs) {
  if (!H || nshell < 1) return MG_ERR_ARG;
  Handle* h = &H->h;
  cudaSetDevice(h->device);
  free_basis(h);
  h->sh.clear();
  size_t pe = 0, pc = 0;
  int off = 0, natom = 0, lmax = 0;
  for (int s = 0; s < nshell; ++s) {
    if (l[s] < 0 || l[s] > MG_MAX_L || nprim[s] < 1 || ncontr[s] < 1 || atom[s] < 0) {
      h->err = "mg_set_basis: unsupported shell (need 0<=l<=3, nprim>=1, ncontr>=1)";
      return MG_ERR_ARG;
    }
    ShellH sh;
    for (int x = 0; x < 3; ++x) sh.A[x] = xyz[3 * s + x];
    sh.l = l[s]; sh.np = nprim[s]; sh.nc = ncontr[s]; sh.atom = atom[s];
    sh.ncomp = ncomp(sh.l);
    sh.e.assign(exps + pe, exps + pe + sh.np);
    sh.c.assign(coefs + pc, coefs + pc + (size_t)sh.np * sh.nc);
    pe += sh.np;
    pc += (size_t)sh.np * sh.nc;
    sh.off = off;
    off += sh.nc * sh.ncomp;
    natom = std::max(natom, sh.atom + 1);
    lmax = std::max(lmax, sh.l);
    h->sh.push_back(sh);
  }
  h->nbf = off;
  h->natom = natom;
  h->lmax = lmax;
  build_sph(h, MG_MAX_L + 1);
  if (setup_pairs(h)) return MG_ERR_MEMORY;
  return 0;
}

int mg_nbf(mg_handle* H) { return H ? H->h.nbf : -1; }
int mg_natom(mg_handle* H) { return H ? H->h.natom : -1; }

int mg_eri_quartets_size(mg_handle* H, const int32_t* q4, int64_t nq, int64_t* offsets) {
  if (!H || (!q4 && nq) || !offsets) return MG_ERR_ARG;
  Handle* h = &H->h;
  const int ns = h->sh.size();
  int64_t o = 0;
  for (int64_t t = 0; t < nq; ++t) {
    offsets[t] = o;
    const int s[4] = {q4[4 * t], q4[4 * t + 1], q4[4 * t + 2], q4[4 * t + 3]};
    int64_t n = 1;
    for (int x = 0; x < 4; ++x) {
      if (s[x] < 0 || s[x] >= ns) { h->err = "shell index out of range"; return MG_ERR_ARG; }
      n *= (int64_t)h->sh[s[x]].nc * h->sh[s[x]].ncomp;
    }
    o += n;
  }
  offsets[nq] = o;
  return 0;
}

// Algorithmic work of mg_eri_quartets over a quartet list (FMA = 2 flops), the
// kernel's own stages: per primitive quartet the roots (2 x 7 FMA per root and
// weight + 30), the 2D recursion (3 directions x 4 NI NJ per root), [e0|f0]
// (3 flops per root per (e, f)) and the bra half-transform (2 nij nef); per
// bra-contracted block the ket half-transform (2 nij nkl nef per ket
// primitive pair); per contracted quartet the HRR + spherical transforms.
int mg_eri_work(mg_handle* H, const int32_t* q4, int64_t nq, double* prim_quartets, double* flops) {
  if (!H || (!q4 && nq) || !prim_quartets || !flops) return MG_ERR_ARG;
  Handle* h = &H->h;
  const int ns = h->sh.size();
  double pq = 0.0, f = 0.0;
  for (int64_t t = 0; t < nq; ++t) {
    const int i = q4[4 * t], j = q4[4 * t + 1], k = q4[4 * t + 2], l = q4[4 * t + 3];
    if (i < 0 || j < 0 || k < 0 || l < 0 || i >= ns || j >= ns || k >= ns || l >= ns || i < j || k < l) {
      h->err = "mg_eri_work: shell indices out of range or non-canonical pair";
      return MG_ERR_ARG;
    }
    const DPair& P = h->pairs[pair_id(i, j)];
    const DPair& Q = h->pairs[pair_id(k, l)];
    const int nab = P.la + P.lb, ncd = Q.la + Q.lb;
    const int NR = (nab + ncd) / 2 + 1, NI = nab + 1, NJ = ncd + 1;
    const double nef = (double)P.ne * Q.ne, nij = (double)P.nci * P.ncj, nkl = (double)Q.nci * Q.ncj;
    const double npq = (double)P.np * Q.np;
    const double per_prim = NR * 28.0 + 30.0 + 3.0 * NR * 4.0 * NI * NJ + 3.0 * NR * nef + 2.0 * nij * nef;
    const double ket = 2.0 * nij * nkl * nef * Q.np;
    const double hrr = 2.0 * nij * nkl * ((double)P.nsa * P.nsb * P.ne * Q.ne + (double)P.nsa * P.nsb * Q.nsa * Q.nsb * Q.ne);
    pq += npq;
    f += per_prim * npq + ket + hrr;
  }
  *prim_quartets = pq;
  *flops = f;
  return 0;
}

int mg_eri_quartets(mg_handle* H, const int32_t* q4, int64_t nq, const int64_t* offsets, double* d_out, void* stream) {
  if (!H || (!q4 && nq) || !offsets || (!d_out && nq)) return MG_ERR_ARG;
  Handle* h = &H->h;
  cudaSetDevice(h->device);
  std::vector<EriItem> items;
  std::vector<EriClass> classes;
  int rc = build_eri_items(h, q4, nq, offsets, items, classes);
  if (rc) return rc;
  return run_eri_items(h, items, classes, d_out, (cudaStream_t)stream);
}

int mg_twoel_nosym(mg_handle* H, const double* coor, int* noints, double* wrk, int64_t nwork, const int64_t* isd4,
                   int64_t nsd) {
  if (!H || !coor || !noints || !wrk || !isd4 || nsd < 20) return MG_ERR_ARG;
  Handle* h = &H->h;
  const int ns = h->sh.size();
  int sh[4];
  int64_t nijkl = 1, nabcd = 1;
  for (int x = 0; x < 4; ++x) {
    const int64_t* d = isd4 + (nsd + 1) * x;
    sh[x] = (int)d[20] - 1;
    if (sh[x] < 0 || sh[x] >= ns) { h->err = "mg_twoel_nosym: iSD4(20,*) is not a shell of the handle"; return MG_ERR_ARG; }
    const ShellH& S = h->sh[sh[x]];
    if (d[1] != S.l || d[3] != S.nc) {
      h->err = "mg_twoel_nosym: iSD4 angular momentum or contraction count differs from the handle's shell";
      return MG_ERR_ARG;
    }
    for (int c = 0; c < 3; ++c)
      if (std::fabs(coor[3 * x + c] - S.A[c]) > 1e-10 * std::max(1.0, std::fabs(S.A[c]))) {
        h->err = "mg_twoel_nosym: Coor differs from the handle's shell centre";
        return MG_ERR_ARG;
      }
    nijkl *= S.nc;
    nabcd *= S.ncomp;
  }
  if (nwork < nijkl * nabcd) { h->err = "mg_twoel_nosym: Wrk too small"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  // canonical quartet (i >= j, k >= l) for the batched kernel, then the block
  // is transposed back to the caller's shell order
  const bool sab = sh[0] < sh[1], scd = sh[2] < sh[3];
  const int32_t q[4] = {sab ? sh[1] : sh[0], sab ? sh[0] : sh[1], scd ? sh[3] : sh[2], scd ? sh[2] : sh[3]};
  int64_t off[2];
  int rc = mg_eri_quartets_size(H, q, 1, off);
  if (rc) return rc;
  const int64_t nout = off[1];
  std::vector<EriItem> items;
  std::vector<EriClass> classes;
  rc = build_eri_items(h, q, 1, off, items, classes);
  if (rc) return rc;
  double* blk = nullptr;
  if (dev_malloc(&blk, sizeof(double) * nout) != cudaSuccess) { h->err = "mg_twoel_nosym: allocation failed"; return MG_ERR_MEMORY; }
  rc = run_eri_items(h, items, classes, blk, nullptr);
  std::vector<double> hb(nout);
  if (!rc && cudaMemcpy(hb.data(), blk, sizeof(double) * nout, cudaMemcpyDeviceToHost) != cudaSuccess) rc = MG_ERR_CUDA;
  cudaFree(blk);
  if (rc) return rc;
  // canonical layout: [i'][j'][k'][l'] contracted (i' fastest) x [ci'][cj'][ck'][cl'] components
  const ShellH *A = &h->sh[sh[0]], *B = &h->sh[sh[1]], *Cs = &h->sh[sh[2]], *Ds = &h->sh[sh[3]];
  const int n0 = A->nc, n1 = B->nc, n2 = Cs->nc, n3 = Ds->nc;
  const int m0 = A->ncomp, m1 = B->ncomp, m2 = Cs->ncomp, m3 = Ds->ncomp;
  const int cn0 = sab ? n1 : n0, cn1 = sab ? n0 : n1, cn2 = scd ? n3 : n2;
  const int cm0 = sab ? m1 : m0, cm1 = sab ? m0 : m1, cm2 = scd ? m3 : m2;
  const int64_t cnijkl = nijkl;
  for (int d3 = 0; d3 < m3; ++d3)
    for (int d2 = 0; d2 < m2; ++d2)
      for (int d1 = 0; d1 < m1; ++d1)
        for (int d0 = 0; d0 < m0; ++d0) {
          const int e0 = sab ? d1 : d0, e1 = sab ? d0 : d1, e2 = scd ? d3 : d2, e3 = scd ? d2 : d3;
          const int64_t csrc = e0 + (int64_t)cm0 * (e1 + (int64_t)cm1 * (e2 + (int64_t)cm2 * e3));
          const int64_t cdst = d0 + (int64_t)m0 * (d1 + (int64_t)m1 * (d2 + (int64_t)m2 * d3));
          for (int i3 = 0; i3 < n3; ++i3)
            for (int i2 = 0; i2 < n2; ++i2)
              for (int i1 = 0; i1 < n1; ++i1)
                for (int i0 = 0; i0 < n0; ++i0) {
                  const int j0 = sab ? i1 : i0, j1 = sab ? i0 : i1, j2 = scd ? i3 : i2, j3 = scd ? i2 : i3;
                  const int64_t src = j0 + (int64_t)cn0 * (j1 + (int64_t)cn1 * (j2 + (int64_t)cn2 * j3));
                  const int64_t dst = i0 + (int64_t)n0 * (i1 + (int64_t)n1 * (i2 + (int64_t)n2 * i3));
                  wrk[dst + nijkl * cdst] = hb[src + cnijkl * csrc];
                }
        }
  *noints = 0;
  return 0;
}

int mg_schwarz(mg_handle* H, double* tmax) {
  if (!H || !tmax) return MG_ERR_ARG;
  Handle* h = &H->h;
  cudaSetDevice(h->device);
  const int ns = h->sh.size();
  if (h->tmax.empty()) {
    std::vector<int32_t> q;
    for (int i = 0; i < ns; ++i)
      for (int j = 0; j <= i; ++j) { q.push_back(i); q.push_back(j); q.push_back(i); q.push_back(j); }
    const int64_t nq = q.size() / 4;
    std::vector<int64_t> off(nq + 1);
    mg_eri_quartets_size(H, q.data(), nq, off.data());
    double* d_out = nullptr;
    if (dev_malloc(&d_out, sizeof(double) * std::max<int64_t>(off[nq], 1)) != cudaSuccess) {
      h->err = "cudaMalloc Schwarz";
      return MG_ERR_MEMORY;
    }
    int rc = mg_eri_quartets(H, q.data(), nq, off.data(), d_out, nullptr);
    std::vector<double> blk(off[nq]);
    if (!rc) rc = cudaMemcpy(blk.data(), d_out, sizeof(double) * off[nq], cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : MG_ERR_CUDA;
    cudaFree(d_out);
    if (rc) return rc;
    h->tmax.assign((size_t)ns * ns, 0.0);
    for (int64_t t = 0; t < nq; ++t) {
      const int i = q[4 * t], j = q[4 * t + 1];
      const ShellH &A = h->sh[i], &B = h->sh[j];
      const int nij = A.nc * B.nc, nijkl = nij * nij, nsa = A.ncomp, nsb = B.ncomp;
      double mx = 0;
      for (int sb = 0; sb < nsb; ++sb)
        for (int sa = 0; sa < nsa; ++sa)
          for (int kb = 0; kb < B.nc; ++kb)
            for (int ka = 0; ka < A.nc; ++ka) {
              const int ij = ka + A.nc * kb;
              const int64_t ijkl = ij + (int64_t)nij * ij;
              const int64_t sab = sa + nsa * sb;
              const double v = blk[off[t] + ijkl + nijkl * (sab + (int64_t)nsa * nsb * sab)];
              mx = std::max(mx, std::fabs(v));
            }
      h->tmax[(size_t)i * ns + j] = h->tmax[(size_t)j * ns + i] = std::sqrt(mx);
    }
  }
  std::copy(h->tmax.begin(), h->tmax.end(), tmax);
  return 0;
}

int mg_cho_default(mg_cho_cfg* cfg) {
  if (!cfg) return MG_ERR_ARG;
  cfg->thrcom = 1e-4;
  cfg->span = 1e-2;
  cfg->minqual = 50;
  cfg->maxqual = 100;
  cfg->maxvec = 0;
  return 0;
}

int mg_cho_drv(mg_handle* H, const mg_cho_cfg* cfg, void* stream) {
  if (!H || !cfg || cfg->thrcom <= 0 || cfg->maxqual < 1) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (h->pairs.empty()) { h->err = "mg_cho_drv: no basis"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  cho_free(h->cho);
  h->cho = nullptr;
  ChoCfgH c;
  c.thrcom = cfg->thrcom;
  c.span = cfg->span;
  c.minqual = cfg->minqual;
  c.maxqual = std::min(cfg->maxqual, 100000);
  c.maxvec = cfg->maxvec > 0 ? cfg->maxvec : h->nbf * (h->nbf + 1) / 2;
  ChoState* st = nullptr;
  int rc = cho_decompose(h, c, st, (cudaStream_t)stream, h->err);
  h->cho = st;
  return rc;
}

int mg_cho_info(mg_handle* H, int64_t* nrs, int* nvec, int* npass) {
  if (!H || !H->h.cho) return MG_ERR_ARG;
  if (nrs) *nrs = cho_nrs(H->h.cho);
  if (nvec) *nvec = cho_nvec(H->h.cho);
  if (npass) *npass = cho_npass(H->h.cho);
  return 0;
}

int mg_cho_pivots(mg_handle* H, int32_t* piv, int32_t* pass_of) {
  if (!H || !H->h.cho) return MG_ERR_ARG;
  cho_pivots(H->h.cho, piv, pass_of);
  return 0;
}

int mg_cho_rs_list(mg_handle* H, int32_t* a, int32_t* b, int32_t* sp) {
  if (!H || !H->h.cho) return MG_ERR_ARG;
  cho_rs_list(H->h.cho, a, b, sp);
  return 0;
}

int mg_cho_copy_vectors(mg_handle* H, int first, int count, double* d_out, void* stream) {
  if (!H || !H->h.cho || (!d_out && count)) return MG_ERR_ARG;
  cudaSetDevice(H->h.device);
  return cho_copy_vectors(H->h.cho, first, count, d_out, (cudaStream_t)stream);
}

int mg_cho_diag(mg_handle* H, double* d_diag, void* stream) {
  if (!H || !H->h.cho || !d_diag) return MG_ERR_ARG;
  cudaSetDevice(H->h.device);
  cudaMemcpyAsync(d_diag, cho_diag0(H->h.cho), sizeof(double) * cho_nrs(H->h.cho), cudaMemcpyDeviceToDevice,
                  (cudaStream_t)stream);
  return 0;
}

int mg_drvg1(mg_handle* H, const double* d_D, double cutint, double* d_grad, void* stream) {
  return mg_drvg1_x(H, d_D, nullptr, 1.0, 1.0, cutint, d_grad, stream);
}

int mg_drvg1_x(mg_handle* H, const double* d_D, const double* d_DS, double coulfac, double exfac, double cutint,
               double* d_grad, void* stream) {
  if (!H || !d_D || !d_grad) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (h->pairs.empty()) { h->err = "mg_drvg1: no basis"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  if (h->tmax.empty()) {
    std::vector<double> t((size_t)h->sh.size() * h->sh.size());
    int rc = mg_schwarz(H, t.data());
    if (rc) return rc;
  }
  if (!h->grad) h->grad = new GradPlan;
  if (h->grad->cutint != cutint) {
    int rc = grad_build(h, cutint, *h->grad);
    if (rc) return rc;
  }
  return grad_run(h, *h->grad, d_D, d_DS, coulfac, exfac, d_grad, (cudaStream_t)stream);
}

int mg_cho_jk(mg_handle* H, const double* d_C, int r, double* d_J, double* d_K, int precision, void* stream) {
  if (!H || !d_C || !d_J || !d_K || r < 1) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (!h->cho) { h->err = "mg_cho_jk: no Cholesky vectors (call mg_cho_drv)"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  if (precision == MG_PREC_FP64) return jk_fp64(h, d_C, r, d_J, d_K, (cudaStream_t)stream, 32);
  if (precision == MG_PREC_MIXED)
    return jk_mixed(h, d_C, r, d_J, d_K, (cudaStream_t)stream, 64, MG_JK_SLICES, MG_JK_SLICES_K);
  if (precision > 100 && precision <= 108)
    return jk_mixed(h, d_C, r, d_J, d_K, (cudaStream_t)stream, 64, precision - 100, precision - 100);
  h->err = "mg_cho_jk: unsupported precision";
  return MG_ERR_ARG;
}

int mg_cho_jk_batch(mg_handle* H, int ndens, const double* const* d_C, const int* r, double* const* d_J,
                    double* const* d_K, int precision, void* stream) {
  if (!H || ndens < 1 || ndens > 8 || !d_C || !r || !d_J || !d_K) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (!h->cho) { h->err = "mg_cho_jk_batch: no Cholesky vectors (call mg_cho_drv)"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == MG_PREC_FP64) return jk_fp64_batch(h, ndens, d_C, r, d_J, d_K, st, 32);
  if (precision == MG_PREC_MIXED) return jk_mixed_batch(h, ndens, d_C, r, d_J, d_K, st, 64, MG_JK_SLICES, MG_JK_SLICES_K);
  if (precision > 100 && precision <= 108)
    return jk_mixed_batch(h, ndens, d_C, r, d_J, d_K, st, 64, precision - 100, precision - 100);
  h->err = "mg_cho_jk_batch: unsupported precision";
  return MG_ERR_ARG;
}

int mg_cho_lk_scf(mg_handle* H, const double* d_C, int r, double factxi, double* d_FLT, int precision,
                  void* stream) {
  if (!H || !d_C || !d_FLT || r < 1) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (!h->cho) { h->err = "mg_cho_lk_scf: no Cholesky vectors (call mg_cho_drv)"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  const size_t nn = (size_t)h->nbf * h->nbf;
  if (h->lk_cap < nn) {
    cudaFree(h->d_lk);
    h->d_lk = nullptr;
    h->lk_cap = 0;
    if (dev_malloc(&h->d_lk, 2 * nn * sizeof(double)) != cudaSuccess) {
      h->err = "mg_cho_lk_scf: allocation failed";
      return MG_ERR_MEMORY;
    }
    h->lk_cap = nn;
  }
  int rc = mg_cho_jk(H, d_C, r, h->d_lk, h->d_lk + nn, precision, stream);
  if (rc) return rc;
  return fock_accumulate(d_FLT, h->d_lk, h->d_lk + nn, factxi, (int64_t)nn, (cudaStream_t)stream);
}

int mg_cd_incore(mg_handle* H, double* d_X, int n, double thr, double* d_vec, int maxvec, int* numcho,
                 void* stream) {
  if (!H || !numcho || (n > 0 && (!d_X || !d_vec))) return MG_ERR_ARG;
  cudaSetDevice(H->h.device);
  return cd_incore(&H->h, d_X, n, thr, d_vec, maxvec, numcho, (cudaStream_t)stream);
}

int mg_choscf_lk(mg_handle* H, const double* d_D, double factxi, double* d_FLT, int precision, int* nvec,
                 void* stream) {
  if (!H || !d_D || !d_FLT) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (!h->cho) { h->err = "mg_choscf_lk: no Cholesky vectors (call mg_cho_drv)"; return MG_ERR_ARG; }
  cudaSetDevice(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int n = h->nbf;
  const size_t nn = (size_t)n * n;
  if (h->dcd_cap < nn) {
    cudaFree(h->d_dcd);
    h->d_dcd = nullptr;
    h->dcd_cap = 0;
    if (dev_malloc(&h->d_dcd, 2 * nn * sizeof(double)) != cudaSuccess) {
      h->err = "mg_choscf_lk: allocation failed";
      return MG_ERR_MEMORY;
    }
    h->dcd_cap = nn;
  }
  double* X = h->d_dcd;
  double* Vec = h->d_dcd + nn;
  // Thr = 1e-8 of the largest diagonal of D (choscf_drv.F90:110-115)
  std::vector<double> dg(n);
  cudaMemcpy2DAsync(dg.data(), sizeof(double), d_D, sizeof(double) * (n + 1), sizeof(double), n,
                    cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(X, d_D, nn * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { h->err = "mg_choscf_lk: copy failed"; return MG_ERR_CUDA; }
  double ymax = 0.0;
  for (double v : dg) ymax = std::max(ymax, v);
  int numv = 0;
  const int rc = cd_incore(h, X, n, 1.0e-8 * ymax, Vec, n, &numv, st);
  if (nvec) *nvec = numv;
  if (rc) {
    if (rc > 100) h->err = "mg_choscf_lk: the density is not positive semidefinite (CD_InCore irc " + std::to_string(rc) + ")";
    return rc;
  }
  if (numv == 0) return 0;  // D = 0: nothing to add
  return mg_cho_lk_scf(H, Vec, numv, factxi, d_FLT, precision, stream);
}

int mg_sliced_selftest(mg_handle* H, int ld, int r, int slices, const double* d_A, const double* d_B, double* d_X,
                       double* d_K, void* d_slices, int* d_exps, void* stream) {
  if (!H || !d_A || !d_B || !d_X || !d_K) return MG_ERR_ARG;
  cudaSetDevice(H->h.device);
  return oz_selftest(&H->h, ld, r, slices, d_A, d_B, d_X, d_K, (uint8_t*)d_slices, d_exps, (cudaStream_t)stream);
}

long long mg_kernel_launches(void) { return g_launches.load(); }
long long mg_device_allocations(void) { return g_allocs.load(); }

int mg_rys_roots(mg_handle* H, int nrys, int64_t n, const double* T, double* x, double* w) {
  if (!H || nrys < 1 || nrys > MG_MAX_RYS || n < 0 || (n && (!T || !x || !w))) return MG_ERR_ARG;
  Handle* h = &H->h;
  for (int64_t i = 0; i < n; ++i)
    if (!(T[i] >= 0.0)) {
      h->err = "mg_rys_roots: negative or NaN argument";
      return MG_ERR_ARG;
    }
  if (n == 0) return 0;
  if (cudaSetDevice(h->device) != cudaSuccess) return MG_ERR_CUDA;
  double* d = nullptr;
  const size_t bytes = sizeof(double) * (size_t)n * (1 + 2 * nrys);
  if (dev_malloc(&d, bytes) != cudaSuccess) {
    h->err = "mg_rys_roots: device allocation failed";
    return MG_ERR_MEMORY;
  }
  double* dT = d;
  double* dx = d + n;
  double* dw = dx + n * nrys;
  cudaMemcpy(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice);
  int rc = rys_eval(h, nrys, n, dT, dx, dw);
  if (!rc && (cudaMemcpy(x, dx, sizeof(double) * n * nrys, cudaMemcpyDeviceToHost) != cudaSuccess ||
              cudaMemcpy(w, dw, sizeof(double) * n * nrys, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = MG_ERR_CUDA;
  cudaFree(d);
  if (rc) h->err = "mg_rys_roots: evaluation failed";
  return rc;
}

int mg_grad_set_tile(mg_handle* H, int nab1, int ncd1, int tpq, int order) {
  if (!H) return MG_ERR_ARG;
  Handle* h = &H->h;
  // order + 3: the same shrink order with the larger tile caps (32 x 16)
  if (nab1 < 1 || nab1 > 7 || ncd1 < 1 || ncd1 > 7 || (tpq != 0 && tpq != 128 && tpq != 256 && tpq != 512) ||
      order < 0 || order > 5) {
    h->err = "mg_grad_set_tile: class 1..7 x 1..7, tpq 0/128/256/512, order 0..5";
    return MG_ERR_ARG;
  }
  h->grad_tpq[nab1 * 8 + ncd1] = tpq;
  h->grad_order[nab1 * 8 + ncd1] = order % 3;
  h->grad_cap[nab1 * 8 + ncd1] = order / 3;
  if (h->grad) h->grad->cutint = -1;  // re-plan at the next gradient
  return 0;
}

int mg_grad_profile(mg_handle* H, int enable) {
  if (!H) return MG_ERR_ARG;
  H->h.grad_profile = enable != 0;
  H->h.grad_ev_used = 0;
  return 0;
}

int mg_grad_class_times(mg_handle* H, int* keys, double* ms, int maxn) {
  if (!H || (maxn > 0 && (!keys || !ms))) return MG_ERR_ARG;
  Handle* h = &H->h;
  const int n = std::min(maxn, h->grad_ev_used);
  for (int k = 0; k < n; ++k) {
    float t = 0.f;
    if (cudaEventSynchronize(h->grad_ev[2 * k + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&t, h->grad_ev[2 * k], h->grad_ev[2 * k + 1]) != cudaSuccess) {
      h->err = "mg_grad_class_times: no profiled gradient to read";
      return MG_ERR_CUDA;
    }
    keys[k] = h->grad_ev_key[k];
    ms[k] = t;
  }
  return h->grad_ev_used;
}

int mg_eri_set_tile(mg_handle* H, int nab, int ncd, int tpq, int order) {
  if (!H) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (nab < 0 || nab > 7 || ncd < 0 || ncd > 7 || (tpq != 0 && tpq != 64 && tpq != 128 && tpq != 256 && tpq != 512) ||
      order < 0 || order > 3) {
    h->err = "mg_eri_set_tile: class 0..7 x 0..7, tpq 0/64/128/256/512, order 0..3";
    return MG_ERR_ARG;
  }
  h->eri_tpq[nab * 8 + ncd] = tpq;
  h->eri_order[nab * 8 + ncd] = order;
  return 0;
}

int mg_eri_profile(mg_handle* H, int enable) {
  if (!H) return MG_ERR_ARG;
  H->h.eri_profile = enable != 0;
  H->h.eri_ev_used = 0;
  return 0;
}

int mg_eri_class_times(mg_handle* H, int* keys, double* ms, int* tpq, int* pab, int* pcd, int maxn) {
  if (!H || (maxn > 0 && (!keys || !ms || !tpq || !pab || !pcd))) return MG_ERR_ARG;
  Handle* h = &H->h;
  const int n = std::min(maxn, h->eri_ev_used);
  for (int k = 0; k < n; ++k) {
    float t = 0.f;
    if (cudaEventSynchronize(h->eri_ev[2 * k + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&t, h->eri_ev[2 * k], h->eri_ev[2 * k + 1]) != cudaSuccess) {
      h->err = "mg_eri_class_times: no profiled ERI batch to read";
      return MG_ERR_CUDA;
    }
    keys[k] = h->eri_ev_key[k];
    ms[k] = t;
    tpq[k] = h->eri_ev_plan[k].tpq;
    pab[k] = h->eri_ev_plan[k].PAB;
    pcd[k] = h->eri_ev_plan[k].PCD;
  }
  return h->eri_ev_used;
}

int mg_grad_plan_info(mg_handle* H, int* keys, int* tpq, int* pab, int* pcd, int* rw, int maxn) {
  if (!H || (maxn > 0 && (!keys || !tpq || !pab || !pcd || !rw))) return MG_ERR_ARG;
  Handle* h = &H->h;
  if (!h->grad || h->grad->cutint < 0) return 0;
  const std::vector<GradClass>& cl = h->grad->classes;
  for (int k = 0; k < std::min<int>(maxn, (int)cl.size()); ++k) {
    keys[k] = cl[k].nab1 * 8 + cl[k].ncd1;
    tpq[k] = cl[k].tpq;
    pab[k] = cl[k].pab;
    pcd[k] = cl[k].pcd;
    rw[k] = cl[k].rw;
  }
  return (int)cl.size();
}

double mg_drvg1_flops(mg_handle* H, double cutint) {
  if (!H) return -1;
  Handle* h = &H->h;
  if (h->tmax.empty()) {
    std::vector<double> t((size_t)h->sh.size() * h->sh.size());
    if (mg_schwarz(H, t.data())) return -1;
  }
  if (!h->grad) h->grad = new GradPlan;
  if (h->grad->cutint != cutint && grad_build(h, cutint, *h->grad)) return -1;
  return grad_plan_flops(h, *h->grad);
}

}  // extern "C"
