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

#include "grad_kernel.cuh"

namespace mg {

// Device copy of the per-CTA tables (layout in grad_kernel.cuh).
static int make_grad_tables(const Handle* h, double** d_tab) {
  std::vector<double> t(kGTabD, 0.0);
  int o = kGTabSph;
  for (int l = 0; l <= 3; ++l)
    for (double v : h->sph[l]) t[o++] = v;
  if (o != kGTabCart) return MG_ERR_ARG;
  int* cart = reinterpret_cast<int*>(t.data() + kGTabCart);
  int k = 0;
  for (int l = 0; l <= 7; ++l)
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) cart[k++] = lx | (ly << 8) | ((l - lx - ly) << 16);
  if (dev_malloc(d_tab, sizeof(double) * kGTabD) != cudaSuccess) return MG_ERR_MEMORY;
  cudaMemcpy(*d_tab, t.data(), sizeof(double) * kGTabD, cudaMemcpyHostToDevice);
  return 0;
}

static inline size_t ev2(size_t x) { return (x + 1) & ~(size_t)1; }

// Per-group shared memory (doubles) of one work item with PAB x PCD tiles:
//   hdr + Cab + Ccd + Y + IX + max(reduction, tile (cf + Gp + F + S))
// (the layout of grad_kernel, every region rounded to an even count)
static size_t grad_group_smem(const DPair& P, const DPair& Q, int nijc, int nklc, int pab, int pcd, int rw) {
  const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
  const int NR = (la + lb + lc + ld + 3) / 2;
  const size_t ncart4 = (size_t)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  const size_t n1d = (size_t)(la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
  const size_t nij = nijc, nc = nij * nklc;
  const bool multi = nc > 1;
  const size_t fixed = 8 + ev2(nij * P.np) + ev2((size_t)nklc * Q.np) + (multi ? ev2(nij * pcd * ncart4) : 0) +
                       ev2((ncart4 + 1) / 2);
  const size_t nt = (size_t)pab * pcd;
  const size_t w = std::min<size_t>(rw, NR);
  // padded strides of Gp and F (the kernel's Gs, J4 and St)
  const size_t gs = ncart4 | 1, j4 = 4 * n1d + 2, st = 3 * w * j4 + (w & 1 ? 0 : 2);
  const size_t tile = ev2(nt * ((size_t)NR * 10 + 5)) + ev2(nt * gs) + nt * st;
  return ev2(fixed + std::max(tile, (size_t)16 * 9));
}

// Global scratch (doubles) of one work item: contracted Cartesian 2-PDM and
// the stage-0 temporaries.
static size_t grad_item_scratch(const DPair& P, const DPair& Q, int nijc, int nklc) {
  const size_t ncart4 = (size_t)ncart(P.la) * ncart(P.lb) * ncart(Q.la) * ncart(Q.lb);
  const size_t nsp4 = (size_t)ncomp(P.la) * ncomp(P.lb) * ncomp(Q.la) * ncomp(Q.lb);
  const size_t nc = (size_t)nijc * nklc;
  return ev2(nc * ncart4) + nc * std::max(ncart4, nsp4);
}

// Largest run-time loop extent x divisor of one work item (the kernel's
// multiply-high division is exact below 2^32).
static double grad_div_bound(const DPair& P, const DPair& Q, int nij, int pab, int pcd, int rw) {
  const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
  const int NI = la + lb + 2, NR = (la + lb + lc + ld + 3) / 2;
  const double ncart4 = (double)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  const double n1d = (double)(la + 1) * (lb + 1) * (lc + 1) * (ld + 1);
  const double nV = (double)NI * (lc + 2) * (ld + 1);
  const double nt = (double)pab * pcd, w = std::min(rw, NR);
  return std::max({nt * ncart4 * ncart4, (double)nij * pcd * ncart4 * ncart4, nt * w * 3 * nV * nV,
                   nt * w * 3 * n1d * n1d, nt * NR * pab});
}

static inline int c_nab1(int key) { return key / 8; }
static inline int c_ncd1(int key) { return key % 8; }

// Shared memory of the one CTA per SM (bytes, tables included): 227 KB.
static const size_t kCtaLimit = 227 * 1024;
static const size_t kGradMaxBudget = kCtaLimit / 8 - kGTabD;  // one group, doubles

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
  size_t scratch_need = 0;
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
    // one 512-thread CTA per SM (128 registers per thread; measured faster than
    // 2 or 3 smaller CTAs whose register budgets spill); groups of tpq threads.
    // The class's tile choice (mg_grad_set_tile, written by the autotuner) may set
    // the first group size tried and the order in which the tile shrinks:
    // 0 ket primitives, bra primitives, roots per wave; 1 roots first; 2 bra first.
    {
      const size_t cta = kCtaLimit / 8 - kGTabD;
      const int nthr = GradThreads<1>::value;
      const int order = h->grad_order[key];
      const int cab = h->grad_cap[key] ? 32 : 16, ccd = h->grad_cap[key] ? 16 : 8;
      const int tpq0 = h->grad_tpq[key] ? h->grad_tpq[key] : (wmax <= 512 ? 128 : 256);
      // a tile fits when its shared memory is within the group's share and every
      // run-time loop extent x divisor of the kernel stays below 2^32
      auto div_ok = [&](int a, int c, int rw) {
        for (const GradItem& it : v)
          if (grad_div_bound(h->pairs[it.p], h->pairs[it.q], it.i1 - it.i0, a, c, rw) >= 4294967296.0) return false;
        return true;
      };
      for (int tpq = tpq0; tpq <= nthr && !c.tpq; tpq *= 2) {
        const int groups = nthr / tpq;
        const size_t gb = (cta / groups) & ~(size_t)1;
        int pab = std::max(1, std::min(m.npab, cab)), pcd = std::max(1, std::min(m.npcd, ccd)), rw = NRc;
        size_t need = worst(pab, pcd, rw);
        while ((need > gb || !div_ok(pab, pcd, rw)) && (pab > 1 || pcd > 1 || rw > 1)) {
          if (order == 1 && rw > 1) --rw;
          else if (order == 2 && pab > 1) pab = (pab + 1) / 2;
          else if (pcd > 1) pcd = (pcd + 1) / 2;
          else if (pab > 1) pab = (pab + 1) / 2;
          else --rw;
          need = worst(pab, pcd, rw);
        }
        if (need <= gb) {
          c.tpq = tpq;
          c.groups = groups;
          c.gsm = (int)need;
          c.rw = rw;
          c.pab = pab;
          c.pcd = pcd;
          c.minb = 1;
        }
      }
    }
    if (!c.tpq) { h->err = "gradient class does not fit in shared memory"; return MG_ERR_ARG; }
    for (const GradItem& it : v)
      if (grad_div_bound(h->pairs[it.p], h->pairs[it.q], it.i1 - it.i0, c.pab, c.pcd, c.rw) >= 4294967296.0) {
        h->err = "gradient work item exceeds the kernel's index range";
        return MG_ERR_ARG;
      }
    c.nab1 = key / 8;
    c.ncd1 = key % 8;
    c.begin = plan.items.size();
    c.count = v.size();
    c.work = 0;
    for (const GradItem& it : v) {  // primitive quartets x Cartesian components x roots
      const DPair &P = h->pairs[it.p], &Q = h->pairs[it.q];
      c.work += (double)P.np * Q.np * ncart(P.la) * ncart(P.lb) * ncart(Q.la) * ncart(Q.lb) * NRc;
    }
    c.scr = 0;
    for (const GradItem& it : v)
      c.scr = std::max<long long>(c.scr, grad_item_scratch(h->pairs[it.p], h->pairs[it.q], it.i1 - it.i0, it.c1 - it.c0));
    c.scr = (c.scr + 31) & ~31LL;  // 256-byte aligned slots
    {  // persistent grid: the CTAs that are resident at once
      GradFn k = grad_kernel_m1(c.nab1, c.ncd1);
      if (!k) { h->err = "gradient class out of range"; return MG_ERR_ARG; }
      int per_sm = 0, nsm = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, c.tpq * c.groups,
                                                    sizeof(double) * (kGTabD + (size_t)c.gsm * c.groups));
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
      if (per_sm < 1) { h->err = "gradient kernel cannot be resident"; return MG_ERR_CUDA; }
      c.grid = std::min<long long>((c.count + c.groups - 1) / c.groups, (long long)per_sm * nsm);
    }
    scratch_need = std::max<size_t>(scratch_need, (size_t)c.grid * c.groups * c.scr);
    plan.items.insert(plan.items.end(), v.begin(), v.end());
    plan.classes.push_back(c);
  }
  cudaFree(plan.d_items);
  plan.d_items = nullptr;
  if (!plan.items.empty()) {
    if (dev_malloc(&plan.d_items, sizeof(GradItem) * plan.items.size()) != cudaSuccess) return MG_ERR_MEMORY;
    cudaMemcpy(plan.d_items, plan.items.data(), sizeof(GradItem) * plan.items.size(), cudaMemcpyHostToDevice);
  }
  cudaFree(plan.d_scratch);
  cudaFree(plan.d_counters);
  plan.d_scratch = nullptr;
  plan.d_counters = nullptr;
  // one scratch region per side stream: class kernels on different streams run concurrently
  plan.scratch_stride = (std::max<size_t>(scratch_need, 32) + 31) & ~(size_t)31;
  if (dev_malloc(&plan.d_scratch, sizeof(double) * plan.scratch_stride * MG_ERI_STREAMS) != cudaSuccess ||
      dev_malloc(&plan.d_counters, sizeof(int) * std::max<size_t>(plan.classes.size(), 1)) != cudaSuccess) {
    h->err = "gradient scratch allocation failed";
    return MG_ERR_MEMORY;
  }
  if (!plan.d_tab) {
    const int rc = make_grad_tables(h, &plan.d_tab);
    if (rc) { h->err = "gradient tables"; return rc; }
  }
  plan.cutint = cutint;
  return 0;
}

int grad_run(Handle* h, const GradPlan& plan, const double* d_D, const double* d_DS, double coulfac, double exfac,
             double* d_grad, cudaStream_t st) {
  RysArgs ra;
  for (int i = 0; i < MG_MAX_RYS; ++i) ra.m[i] = h->rys_meta[i];
  ra.tab = h->d_rys;
  cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * h->natom, st);
  cudaMemsetAsync(plan.d_counters, 0, sizeof(int) * plan.classes.size(), st);
  // The class kernels are independent (own counter, own scratch region per stream, atomic
  // accumulation into the gradient): spread them over the handle's side streams so that the
  // tail of one class overlaps the next.
  int rc = side_streams_fork(h, st);
  if (rc) return rc;
  // largest classes first; the scratch region follows the stream (classes on one
  // stream run one after another).  Profiled: every class on the caller's stream,
  // between its own pair of events.
  if (h->grad_profile) {
    const size_t need = 2 * plan.classes.size();
    while (h->grad_ev.size() < need) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) { h->err = "gradient profiling events"; return MG_ERR_CUDA; }
      h->grad_ev.push_back(e);
    }
    h->grad_ev_key.assign(plan.classes.size(), 0);
    h->grad_ev_used = (int)plan.classes.size();
  }
  std::vector<int> order(plan.classes.size());
  for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return plan.classes[a].work > plan.classes[b].work; });
  for (size_t pos = 0; pos < order.size(); ++pos) {
    const size_t ci = order[pos];
    const GradClass& c = plan.classes[ci];
    GradFn k = grad_kernel_m1(c.nab1, c.ncd1);
    if (!k) { h->err = "gradient class out of range"; return MG_ERR_ARG; }
    const int sk = h->grad_profile ? 0 : (int)(pos % MG_ERI_STREAMS);
    const cudaStream_t ks = h->grad_profile ? st : h->eri_streams[sk];
    GradArgs a{plan.d_items + c.begin, c.count, h->d_pairs, h->d_prim, h->tot_np, h->d_coef, d_D, h->nbf,
               plan.d_tab, d_grad, plan.d_scratch + plan.scratch_stride * sk, c.scr, plan.d_counters + ci, c.tpq,
               c.gsm, c.pab, c.pcd, c.rw, d_DS, coulfac, 0.25 * exfac};
    if (h->grad_profile) {
      h->grad_ev_key[pos] = c.nab1 * 8 + c.ncd1;
      cudaEventRecord(h->grad_ev[2 * pos], ks);
    }
    k<<<(unsigned)c.grid, c.tpq * c.groups, sizeof(double) * (kGTabD + (size_t)c.gsm * c.groups), ks>>>(a, ra);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) { h->err = "gradient kernel launch failed"; return MG_ERR_CUDA; }
    if (h->grad_profile) cudaEventRecord(h->grad_ev[2 * pos + 1], ks);
  }
  side_streams_join(h, st);
  return 0;
}

void grad_free(GradPlan* p) {
  if (!p) return;
  cudaFree(p->d_items);
  cudaFree(p->d_tab);
  cudaFree(p->d_scratch);
  cudaFree(p->d_counters);
  delete p;
}

// Algorithmic FP64 flop count of a gradient plan (FMA = 2): per primitive
// quartet the Rys roots (2 x 7 FMA per root and weight + 30); per root and
// direction the 2D recursion (4 NI NJ), the ket transfer (2 NI NJ ld) and, per
// (c, d) column, the bra transfer with the derivative factors
// (3 NI + (lb+1)(8 (la+1) + 4 NI)); the bra half of the primitive 2-PDM
// (2 nij ncart4 when nc > 1) and Assg1 (24 flops per Cartesian quartet and
// root); per work item the 2-PDM, its spherical -> Cartesian transform and
// the ket half of the de-contraction.
double grad_plan_flops(const Handle* h, const GradPlan& plan) {
  double f = 0;
  for (const GradItem& it : plan.items) {
    const DPair &P = h->pairs[it.p], &Q = h->pairs[it.q];
    const int la = P.la, lb = P.lb, lc = Q.la, ld = Q.lb;
    const int NI = la + lb + 2, NJ = lc + ld + 2, NR = (la + lb + lc + ld + 3) / 2;
    const double ncart4 = (double)ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
    const double nsp4 = (double)ncomp(la) * ncomp(lb) * ncomp(lc) * ncomp(ld);
    const int nij = it.i1 - it.i0, nklc = it.c1 - it.c0, nc = nij * nklc;
    const double per_prim = NR * 28.0 + 30.0 +
                            3.0 * NR * (4.0 * NI * NJ + 2.0 * NI * NJ * ld +
                                        (lc + 1.0) * (ld + 1.0) * (3.0 * NI + (lb + 1.0) * (8.0 * (la + 1) + 4.0 * NI))) +
                            (nc > 1 ? 2.0 * nij * ncart4 : 0.0) + 24.0 * ncart4 * NR;
    const double per_item = nc * nsp4 * 8.0 + 2.0 * nc * ncart4 * 4.0 * std::max(ncomp(la), ncomp(ld)) +
                            (nc > 1 ? 2.0 * nc * ncart4 * Q.np : 0.0);
    f += per_prim * (double)P.np * Q.np + per_item;
  }
  return f;
}

}  // namespace mg
