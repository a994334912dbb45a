// Internal data structures of libmolgpu (host + device).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/molgpu.h"

#define MG_MAX_RYS 9
#define MG_ERI_STREAMS 4
#define MG_MAX_L 3

namespace mg {

// number of kernels of this library launched so far (all handles)
extern std::atomic<long long> g_launches;
// number of device allocations this library has requested so far (all handles)
extern std::atomic<long long> g_allocs;

// Every device allocation of the library goes through here (counted).
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  g_allocs.fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc((void**)p, bytes);
}

// Per-order metadata of the Rys root/weight table (constant memory).
struct RysMeta {
  double h, invh, tmax;
  int K;
  int off;  // offset (doubles) of this order's coefficients in the table
  double hx[MG_MAX_RYS], hw[MG_MAX_RYS];
};

// Canonical shell pair (i >= j) as the kernels see it.
struct DPair {
  int i, j;           // shells
  int la, lb;
  int na, nb;         // primitives
  int nci, ncj;       // contracted functions
  int np;             // na*nb primitive pairs, alpha fastest
  int prim_off;       // into pair-primitive pool (SoA, stride = total)
  int coef_off;       // into coefficient pool: Cab[ij][p], ij = i + nci*j
  int hrr_off;        // into HRR pool: H[e][sa][sb] (ne x nsa*nsb)
  int ne, emin;       // Cartesian (e0| block: e in [emin, la+lb]
  int nsa, nsb;       // spherical/Cartesian component counts
  int aeqb;
  double Ap[3];       // centre the (e0| lives on (A if la>=lb else B)
  double A[3], B[3];
  int atom_a, atom_b;
  int ao_a, ao_b;     // first AO of each shell
};

// One unit of ERI work: bra pair p, ket pair q, contracted range [c0, c1)
// of the combined index ijkl, output block offset.
struct EriItem {
  int p, q;
  int c0, c1;
  long long out_off;
};

// Launch plan of one ERI class (eri.cu) and per-class statistics.
struct ClassPlan {
  int tpq, PAB, PCD, gsm;
  size_t smem;
};
struct ClassStats {
  int max_acc = 0, max_nef = 0, max_tmp = 0, max_nij = 0, max_npab = 0, max_npcd = 0, max_cab = 0, max_ccd = 0;
  int max_ne = 0, max_nf = 0, max_nc = 0;
  double work = 0;  // estimated cost of the class's items (launch order only)
};
struct EriClass {
  int nab, ncd, begin, count;
  ClassPlan plan;
  double work;  // estimated cost: classes launch largest first
};

struct ShellH {
  double A[3];
  int l, np, nc, atom, off, ncomp;
  std::vector<double> e, c;  // c[p + np*k]
};

struct Workspace {
  void* ptr = nullptr;
  size_t size = 0;
};

struct Handle {
  int device = 0;
  std::vector<ShellH> sh;
  int nbf = 0, natom = 0, lmax = 0;
  // pairs (canonical, iTri order: pair id of (i,j), i>=j, is i*(i+1)/2+j)
  std::vector<DPair> pairs;
  std::vector<double> sph[MG_MAX_L + 3];  // Cartesian->spherical per l (ncart x ncomp, col-major)
  // device memory
  DPair* d_pairs = nullptr;
  double* d_prim = nullptr;   // SoA: [8][tot_np]: zeta, kappa, Px, Py, Pz, alpha, beta, 1/zeta
  int tot_np = 0;
  long long prim_kept = 0, prim_total = 0;  // primitive pairs after prescreening
  double* d_coef = nullptr;
  double* d_hrr = nullptr;
  double* d_rys = nullptr;
  RysMeta rys_meta[MG_MAX_RYS];
  int rys_nmax = 0, rys_degree = 0;
  std::vector<double> tmax;   // Schwarz bound per pair (sqrt max |(ab|ab)|)
  double* d_tmax = nullptr;
  Workspace ws;
  std::string err;
  struct ChoState* cho = nullptr;  // Cholesky vectors of the current basis
  struct GradPlan* grad = nullptr; // gradient work list (per Schwarz threshold)
  int* d_eri_counters = nullptr;   // one work counter per ERI class launch (64)
  cudaStream_t eri_streams[MG_ERI_STREAMS] = {};  // side streams of the ERI and gradient class launches
  cudaEvent_t eri_events[MG_ERI_STREAMS] = {};
  cudaEvent_t eri_fork = nullptr;
  double* d_lk = nullptr;          // J and K of mg_cho_lk_scf (2 nbf^2)
  size_t lk_cap = 0;
  double* d_dcd = nullptr;         // density copy and its Cholesky vectors of mg_choscf_lk (2 nbf^2)
  size_t dcd_cap = 0;
  // gradient tile choices per class key (nab1 * 8 + ncd1): threads per group
  // (0 = the planner's) and the order in which the tile shrinks to fit
  int grad_tpq[64] = {};
  int grad_order[64] = {};
  int grad_cap[64] = {};  // tile caps: 0 = 16 bra x 8 ket primitive pairs, 1 = 32 x 16
  // profiled gradients: classes one after another on the caller's stream, an
  // event pair around each (grad_ev[2k], grad_ev[2k + 1] for class key grad_ev_key[k])
  bool grad_profile = false;
  std::vector<cudaEvent_t> grad_ev;
  std::vector<int> grad_ev_key;
  int grad_ev_used = 0;
  // the same for the ERI classes (key nab * 8 + ncd; order 0 ket primitives
  // shrink first, 1 bra primitives), with each profiled class's plan
  int eri_tpq[64] = {};
  int eri_order[64] = {};
  bool eri_profile = false;
  std::vector<cudaEvent_t> eri_ev;
  std::vector<int> eri_ev_key;
  std::vector<ClassPlan> eri_ev_plan;
  int eri_ev_used = 0;
};

struct GradItem {
  int p, q;      // bra / ket canonical pairs
  int c0, c1;    // ket contracted-pair (kl) range
  int i0, i1;    // bra contracted-pair (ij) range
  double scale;  // 1/2 * degeneracy
};
struct GradClass {
  int nab1, ncd1, begin, count, tpq, gsm, groups, rw, pab, pcd;
  int minb;       // resident CTAs per SM the kernel variant is compiled for (1..3)
  long long scr;  // global scratch per group (doubles)
  long long grid; // persistent CTAs
  double work;    // estimated cost: classes launch largest first
};
struct GradPlan {
  std::vector<GradItem> items;
  std::vector<GradClass> classes;
  GradItem* d_items = nullptr;
  size_t scratch_stride = 0;     // doubles of scratch per side stream
  double* d_tab = nullptr;       // per-CTA tables of the gradient kernel
  double* d_scratch = nullptr;   // per-group 2-PDM slots
  int* d_counters = nullptr;     // one work counter per class
  double cutint = -1;
};
int grad_build(Handle* h, double cutint, GradPlan& plan);
// fork the handle's side streams from `st` (created on first use) / join them back into `st`
int side_streams_fork(Handle* h, cudaStream_t st);
void side_streams_join(Handle* h, cudaStream_t st);
int rys_eval(Handle* h, int nrys, int64_t n, const double* d_T, double* d_x, double* d_w);
int grad_run(Handle* h, const GradPlan& plan, const double* d_D, const double* d_DS, double coulfac, double exfac,
             double* d_grad, cudaStream_t st);
void grad_free(GradPlan* p);
double grad_plan_flops(const Handle* h, const GradPlan& plan);

struct ChoState;
struct ChoCfgH {
  double thrcom, span;
  int minqual, maxqual, maxvec;
};
int cho_decompose(Handle* h, const ChoCfgH& cfg, ChoState*& out, cudaStream_t st, std::string& err);
void cho_free(ChoState* c);
int64_t cho_nrs(const ChoState* c);
int cho_nvec(const ChoState* c);
int cho_npass(const ChoState* c);
void cho_pivots(const ChoState* c, int32_t* piv, int32_t* pass_of);
void cho_rs_list(const ChoState* c, int32_t* a, int32_t* b, int32_t* sp);
int cho_copy_vectors(const ChoState* c, int first, int count, double* d_out, cudaStream_t st);
const double* cho_diag0(const ChoState* c);
typedef struct cublasContext* cublasHandle_t;
cublasHandle_t cho_cublas(ChoState* c);
const int* cho_rs_a_dev(const ChoState* c);
const int* cho_rs_b_dev(const ChoState* c);
const double* cho_vec_ptr(const ChoState* c, int J0, int nb, cudaStream_t st, Handle* h);
int cho_vec_block();
// first rs index of every shell pair (pair_id order), device
const int64_t* cho_sp_first_dev(const ChoState* c);
// cached row exponents of the square Cholesky vectors (M x ld), owned by the state
short* cho_lexp(const ChoState* c, int ld);
void cho_set_lexp(ChoState* c, short* p, int ld);
int oz_selftest(Handle* h, int ld, int r, int s, const double* d_A, const double* d_B, double* d_X, double* d_K,
                uint8_t* d_slices, int* d_exps, cudaStream_t st);
// CD_InCore (cholesky_util/cd_incore.F90:14) on the device: returns irc
// (0, 101, 102, -1) or MG_ERR_*; X (n x n, column-major) is overwritten.
int cd_incore(Handle* h, double* d_X, int n, double thr, double* d_vec, int maxvec, int* numcho, cudaStream_t st);
int fock_accumulate(double* F, const double* J, const double* K, double factxi, int64_t n, cudaStream_t st);
int jk_fp64(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block);
int jk_mixed(Handle* h, const double* d_C, int r, double* d_J, double* d_K, cudaStream_t st, int block, int s, int sk);
// J/K of k (1..8) densities over one pass of the vectors (jk.cu)
int jk_mixed_batch(Handle* h, int k, const double* const* Cs, const int* rs, double* const* Js, double* const* Ks,
                   cudaStream_t st, int block, int s, int sk);
int jk_fp64_batch(Handle* h, int k, const double* const* Cs, const int* rs, double* const* Js, double* const* Ks,
                  cudaStream_t st, int block);

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
inline int ncart_cum(int l) { return l <= 0 ? 0 : l * (l + 1) * (l + 2) / 6; }
inline int ncomp(int l) { return l >= 2 ? 2 * l + 1 : ncart(l); }
inline int pair_id(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// host helpers (basis_host.cu)
int load_rys_table(Handle* h, const char* path);
void build_sph(Handle* h, int lmax);
std::vector<double> hrr_matrix(const Handle* h, int la, int lb, const double* A, const double* B, int& ne, int& emin);
int setup_pairs(Handle* h);
void* ws_get(Handle* h, size_t bytes, cudaStream_t st);

// ERI work lists (capi.cu) and launchers (eri.cu)
ClassPlan eri_plan(int nab, int ncd, const ClassStats& cs, int tpq0 = 0, int order = 0);
int eri_launch_class(Handle* h, const EriItem* d_items, int nitems, int nab, int ncd, const ClassPlan& pl, double* out,
                     int* d_counter, cudaStream_t st);
int build_eri_items(Handle* h, const int32_t* q4, int64_t nq, const int64_t* offsets, std::vector<EriItem>& items,
                    std::vector<EriClass>& classes);
int run_eri_items(Handle* h, const std::vector<EriItem>& items, const std::vector<EriClass>& classes, double* d_out,
                  cudaStream_t st);
int eri_run(Handle* h, const EriItem* d_items, const std::vector<int>& class_begin, const std::vector<int>& class_nab,
            const std::vector<int>& class_ncd, const std::vector<int>& class_np, const std::vector<size_t>& class_smem,
            double* out, cudaStream_t st);
void rys_upload_meta(Handle* h);

}  // namespace mg
