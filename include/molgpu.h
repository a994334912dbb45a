/* molgpu -- B200 (sm_100a) two-electron engine with a plain C ABI.
 *
 * Drop-in boundary for OpenMolcas's two-electron hot path.  Every entry
 * point names the reference routine it replaces (paths relative to the
 * OpenMolcas source tree).  All arrays are plain pointers; "d_" pointers are
 * CUDA device memory owned by the caller, everything else is host memory.
 * Every call returns 0 on success or a positive error code; the message is
 * available from mg_last_error().  Calls never block on device work except
 * where stated; `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Basis conventions (identical to the reference):
 *   - shells with general contraction, coefficient matrix nprim x ncontr
 *     (column-major), normalised as gateway_util/nrmlz.F90 does;
 *   - s and p shells Cartesian (p = x,y,z), d and f real spherical m=-l..l
 *     (integral_util/real_spherical.F90, rdctl_seward.F90:3863-3865);
 *   - AO order: shells in input order, inside a shell component-major with
 *     the contracted index fastest;
 *   - no point-group symmetry (TwoEl_NoSym path), l <= 3.
 */
#ifndef MOLGPU_H
#define MOLGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mg_handle mg_handle;

/* Error codes (mirroring Cho_Drv's iReturn 0/1/2, cholesky_util/
 * cho_drv_inner.F90:14-19, where they apply). */
#define MG_OK 0
#define MG_ERR_ARG 1       /* bad argument / unsupported input          */
#define MG_ERR_DECOMP 1    /* Cholesky decomposition failed (iReturn 1) */
#define MG_ERR_MEMORY 2    /* device allocation failed (iReturn 2)      */
#define MG_ERR_CUDA 3      /* CUDA launch or runtime error              */

/* Create a handle on `device`, loading the Rys root/weight table
 * (replaces SetUpR/Read_RysRW, rys_util/setupr.F90:15, read_rysrw.F90:14). */
int mg_create(const char* rys_table_path, int device, mg_handle** out);
int mg_destroy(mg_handle* h);
const char* mg_last_error(mg_handle* h);

/* Basis set (replaces the Basis_Info/Shells set-up consumed by Setup_Ints,
 * integral_util/setup_ints.F90:14, and the shell-pair precompute of
 * Drvk2/k2Loop, drvk2.F90:16, k2loop.F90:16).
 * xyz[3*nshell]; l, nprim, ncontr, atom [nshell]; exps concatenated;
 * coefs concatenated nprim x ncontr column-major per shell (normalised). */
int mg_set_basis(mg_handle* h, int nshell, const double* xyz, const int* l, const int* nprim, const int* ncontr,
                 const int* atom, const double* exps, const double* coefs);
int mg_nbf(mg_handle* h);
int mg_natom(mg_handle* h);

/* Shell-pair Schwarz bounds TMax(i,j) = sqrt(max |(ab|ab)|) for all shell
 * pairs (replaces Shell_MxSchwz, integral_util/shell_mxschwz.F90:12).
 * Synchronous; tmax is host nshell x nshell. */
int mg_schwarz(mg_handle* h, double* tmax);

/* Batched shell-quartet ERIs (replaces Drv2El -> Eval_IJKL -> TwoEl_NoSym,
 * integral_util/drv2el.F90:15, eval_ijkl.F90:16, twoel_nosym.F90:15).
 * quartets: host int32[4*nq] of shell indices (i>=j, k>=l).  Each quartet's
 * block is written to d_out at offsets[q] in the layout of Eval_IJKL's
 * AOInt(nijkl, iCmp1, iCmp2, iCmp3, iCmp4) (contracted index fastest,
 * i fastest inside ijkl).  offsets (host int64[nq+1]) is filled by
 * mg_eri_quartets_size. */
int mg_eri_quartets_size(mg_handle* h, const int32_t* quartets, int64_t nq, int64_t* offsets);

/* Algorithmic work of mg_eri_quartets on the same quartet list: the number of
 * primitive quartets after primitive-pair prescreening and the FP64 flop
 * count of the kernel's stages (roofline accounting; no reference
 * counterpart).  Host only. */
int mg_eri_work(mg_handle* h, const int32_t* quartets, int64_t nq, double* prim_quartets, double* flops);
int mg_eri_quartets(mg_handle* h, const int32_t* quartets, int64_t nq, const int64_t* offsets, double* d_out,
                    void* stream);

/* One shell quartet in the calling convention of the per-quartet kernel
 * Do_TwoEl (procedure(twoel_kernel), selected at integral_util/
 * eval_ijkl.F90:93-95; arguments in integral_util/twoel_interface.fh):
 * coor[12] = Coor(3,4) (checked against the handle's shell centres),
 * isd4 = iSD4(0:nsd, 4) (column-major, nsd+1 entries per shell; entry 20 is
 * the 1-based shell index nSkal of Def_Shells, integral_util/
 * def_shells.F90:148, entries 1 and 3 (l, nBasis) are checked), wrk[nwork]
 * (host) receives the AO integrals Wrk(1:nijkl*nabcd) in the layout of
 * Eval_IJKL (contracted index fastest, then iCmp1..iCmp4), any shell order.
 * *noints is set to 0 (integrals were computed).  Synchronous, one quartet:
 * a compatibility path, the batched entry point is the fast one. */
int mg_twoel_nosym(mg_handle* h, const double* coor, int* noints, double* wrk, int64_t nwork, const int64_t* isd4,
                   int64_t nsd);

/* Allocation-free variant of mg_eri_quartets.  No counterpart in the
 * reference.  For callers that cannot let the library allocate device memory
 * during a call: programs that reserve all device memory in their own pool
 * up front, frameworks whose caching allocator already holds it, or code that
 * must not get the device-wide synchronisation of cudaFree between its
 * stream-ordered work.  Same arguments and output as mg_eri_quartets; the
 * work list is staged in a fixed 1.5 MiB device array inside the library
 * (held by every GPU that loads the library until exit), so no cudaMalloc or
 * cudaFree is called.  At most 65536 work items per call (one per quartet,
 * more for quartets with large contracted blocks); larger lists are rejected
 * with MG_ERR_ARG.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and should come before any stream capture.
 * All calls share the array: calls that overlap on the GPU (different
 * streams, or different threads) race on it; calls on one stream are
 * ordered.  Nothing in the array needs to start at zero: each call overwrites
 * the entries it uses and every output element is written. */
int mg_eri_quartets_noalloc(mg_handle* h, const int32_t* quartets, int64_t nq, const int64_t* offsets,
                            double* d_out, void* stream);

/* ---------------------------------------------------------------------
 * Cholesky decomposition of the ERI matrix (replaces Cho_Drv / Cho_Drv_Inner
 * with the default algorithm 4, cholesky_util/cho_drv.F90:14,
 * cho_drv_inner.F90:14, cho_decom_a4.F90:12).  Vectors stay on the device
 * inside the handle, FP64, in reduced-set layout: AO pairs a>=b grouped by
 * shell pair (i>=j in iTri order); inside a pair a fastest (i>j) or iTri
 * (i==j) (cholesky_util/plf_cho_diag.F90:60-72).  Only the shell pairs with
 * at least one element that survives the initial screening of the diagonal
 * (diag >= ThrCom^2 / (Damp DiaMax), cho_calcdiag.F90:255-300) have rows
 * (their count is nrs of mg_cho_info; mg_cho_rs_list lists them); the
 * vectors are zero on the other AO pairs.
 */
typedef struct mg_cho_cfg {
  double thrcom; /* decomposition threshold ThrCom (cholesky.F90:128, 1e-4) */
  double span;   /* Span (cho_inp.F90:151, 1e-2)                            */
  int minqual;   /* MinQual (50)                                             */
  int maxqual;   /* MaxQual (100)                                            */
  int maxvec;    /* max. vectors (0 = nbf(nbf+1)/2, the most there can be)  */
} mg_cho_cfg;

int mg_cho_default(mg_cho_cfg* cfg);
/* Returns Cho_Drv's iReturn: 0 ok, 1 (MG_ERR_DECOMP) when the decomposition
 * failed (cho_drv_inner.F90:155,192: no qualifying diagonal, a negative
 * diagonal below TooNeg, CD_InCore failure; also an invalid argument), 2
 * (MG_ERR_MEMORY) when the vectors do not fit in device memory
 * (cho_drv_inner.F90:338); 3 on a CUDA error.  mg_last_error() names the
 * cause.  Synchronous. */
int mg_cho_drv(mg_handle* h, const mg_cho_cfg* cfg, void* stream);
int mg_cho_info(mg_handle* h, int64_t* nrs, int* nvec, int* npass);
/* pivot (rs index) and pass of every vector, in vector order */
int mg_cho_pivots(mg_handle* h, int32_t* piv, int32_t* pass_of);
/* AO indices and shell pair of every rs entry (host arrays of length nrs) */
int mg_cho_rs_list(mg_handle* h, int32_t* a, int32_t* b, int32_t* sp);
/* copy vectors [first, first+count) to d_out (nrs x count, column-major) */
int mg_cho_copy_vectors(mg_handle* h, int first, int count, double* d_out, void* stream);
/* exact diagonal (ab|ab) over the rs list (CHO_GETDIAG, cho_getdiag.F90:12) */
int mg_cho_diag(mg_handle* h, double* d_diag, void* stream);

/* ---------------------------------------------------------------------
 * Coulomb and exchange matrices from the Cholesky vectors of the handle
 * (replaces CHO_LK_SCF, fock_util/cho_lk_scf.F90:14, for one density):
 *   D = C C^T, C (nbf x r, column-major, device);
 *   J_ab = sum_cd (ab|cd) D_cd,  K_ab = sum_cd (ac|bd) D_cd
 * with (ab|cd) ~ sum_J L_ab,J L_cd,J.  J, K: nbf x nbf device, overwritten
 * (the reference accumulates into FLT/KLT; mg_cho_lk_scf below does).
 * precision:
 *   MG_PREC_FP64     FP64 vectors, FP64 products (DGEMM/DSYRK);
 *   MG_PREC_MIXED    FP64 vectors cut into 8-bit slices per row (power-of-two
 *                    row scaling): MG_JK_SLICES for the half-transform
 *                    X_J = L_J C, MG_JK_SLICES_K for the exchange product
 *                    K = sum X X^T; both GEMMs on the tensor cores in 8-bit
 *                    integers with exact INT32 accumulation and FP64
 *                    recombination; Coulomb part FP64.  Energy within 1e-8 Eh
 *                    of MG_PREC_FP64 at 1500 functions / 12865 vectors;
 *   MG_PREC_SLICED(s) the same with s slices for both GEMMs (2..8).
 */
#define MG_PREC_FP64 0
#define MG_PREC_MIXED 1
#define MG_PREC_SLICED(s) (100 + (s))
#define MG_JK_SLICES 6
#define MG_JK_SLICES_K 7
int mg_cho_jk(mg_handle* h, const double* d_C, int r, double* d_J, double* d_K, int precision, void* stream);
/* The accumulating form of CHO_LK_SCF (fock_util/cho_lk_scf.F90:14, one
 * density): d_FLT += J[D] - factxi * K[D] (FLT nbf x nbf, device), the sum the
 * reference builds into FLT (Coulomb, cho_lk_scf.F90:919) and KLT (exchange
 * with -FactXI, :785-831, added into FLT at :993-1018).  Synchronous. */
int mg_cho_lk_scf(mg_handle* h, const double* d_C, int r, double factxi, double* d_FLT, int precision,
                  void* stream);

/* ---------------------------------------------------------------------
 * Two-electron nuclear gradient (replaces Drvg1, alaska/drvg1.F90:15, with
 * the 1/2 of alaska.F90:236 applied): d_grad[3*natom] = dE/dR of
 * E = 1/2 tr(DJ) - 1/4 tr(DK) at fixed density, D the full nbf x nbf
 * symmetric density on the device (row-major = column-major).  Unique shell
 * quartets with TMax(ij) TMax(kl) < cutint are skipped (Shell_MxSchwz
 * screening).  Asynchronous on `stream`.
 */
int mg_drvg1(mg_handle* h, const double* d_D, double cutint, double* d_grad, void* stream);
/* The same with the full 2-PDM of PGet1 (integral_util/pget1.F90:15-110, as
 * PGet0 calls it at integral_util/pget0.F90:189 with D0, DS and the module
 * EtWas factors):
 *   E = coulfac/2 tr(D J[D]) - exfac/4 (tr(D K[D]) + tr(DS K[DS]))
 * DS the spin density (DSSO: D_alpha - D_beta for an open shell, D the total
 * density D_alpha + D_beta) or NULL for a closed shell; coulfac = CoulFac and
 * exfac = ExFac (the exact-exchange fraction of a hybrid functional, 0 for a
 * pure one).  mg_drvg1 is (DS = NULL, coulfac = 1, exfac = 1). */
int mg_drvg1_x(mg_handle* h, const double* d_D, const double* d_DS, double coulfac, double exfac, double cutint,
               double* d_grad, void* stream);
/* Algorithmic FP64 flop count of one mg_drvg1 call (roofline accounting;
 * no reference counterpart).  Negative on error. */
double mg_drvg1_flops(mg_handle* h, double cutint);

/* Gradient tile tuning (no reference counterpart; the knobs of the
 * project's autotuner, openmolcas_b200/autotune.py, whose table
 * grad_tiles.json the Python layer applies at handle creation).  The
 * gradient runs one persistent kernel per class (nab1, ncd1) = (la+lb+1,
 * lc+ld+1); each CTA is split into groups of tpq threads that take work
 * items, and each group's shared memory holds a tile of primitive quartets
 * (bra x ket) and the 2D records of some roots at a time.
 * mg_grad_set_tile: tpq = the first group size tried (128, 256, 512; 0 =
 * the planner's choice), order = the dimension the planner shrinks first
 * when the tile does not fit (0 ket primitives, 1 roots per wave, 2 bra
 * primitives; 3..5 the same with the tile starting from 32 x 16 primitive
 * pairs instead of 16 x 8).  Takes effect at the next gradient (re-plan).
 * mg_grad_profile(h, 1): later gradients launch their classes one after
 * another on the caller's stream with an event pair around each;
 * mg_grad_class_times then returns the classes of the last one (key =
 * nab1 * 8 + ncd1, kernel milliseconds; waits for them) and their count.
 * mg_grad_plan_info: the current plan's tile per class (group size,
 * primitive-quartet tile pab x pcd, roots per wave); returns the count. */
int mg_grad_set_tile(mg_handle* h, int nab1, int ncd1, int tpq, int order);
int mg_grad_profile(mg_handle* h, int enable);
int mg_grad_class_times(mg_handle* h, int* keys, double* ms, int maxn);
int mg_grad_plan_info(mg_handle* h, int* keys, int* tpq, int* pab, int* pcd, int* rw, int maxn);
/* The same for the ERI classes (nab, ncd) = (la+lb, lc+ld) of mg_eri_quartets
 * (and the Cholesky columns): tpq 0, 64, 128, 256 or 512; order 0 shrinks the
 * ket primitives of the tile first, 1 the bra primitives (+ 2: the tile starts
 * from 64 x 16 primitive pairs instead of 32 x 8).  Effective from the
 * next batch.  mg_eri_class_times reports the last profiled batch's classes
 * with their plan (group size, pab x pcd tile). */
int mg_eri_set_tile(mg_handle* h, int nab, int ncd, int tpq, int order);
int mg_eri_profile(mg_handle* h, int enable);
int mg_eri_class_times(mg_handle* h, int* keys, double* ms, int* tpq, int* pab, int* pcd, int maxn);

/* ---------------------------------------------------------------------
 * Rys roots and weights (replaces vRysRW, rys_util/vrysrw.F90:15, and the
 * RysNN table evaluation, rys22.F90:36-47, at the unit-test level): for the n
 * arguments T[] (host), x[i*nrys + k] = u^2 (the squared root, as vRysRW
 * returns it) and w[i*nrys + k] the weight of root k of order nrys (1..9),
 * evaluated on the device from the handle's table (asymptotic Hermite form
 * above the table's TMax).  Synchronous.  Returns MG_ERR_ARG for nrys outside
 * 1..9 or a negative T.
 */
int mg_rys_roots(mg_handle* h, int nrys, int64_t n, const double* T, double* x, double* w);

/* CHO_LK_SCF for ndens (1..8) densities at once (the several densities of
 * choscf_drv.F90's calls, e.g. alpha and beta, or a batch of states): the
 * same as ndens calls of mg_cho_jk, but every block of vectors is unpacked
 * once for all of them.  d_C[i] (nbf x r[i]), d_J[i], d_K[i]: device
 * pointers, in host arrays of length ndens.  Synchronous (mixed) or queued
 * on the stream (FP64), as mg_cho_jk. */
int mg_cho_jk_batch(mg_handle* h, int ndens, const double* const* d_C, const int* r, double* const* d_J,
                    double* const* d_K, int precision, void* stream);

/* CD_InCore (cholesky_util/cd_incore.F90:14, cd_incore_1.F90): pivoted
 * Cholesky vectors of a symmetric positive semidefinite n x n matrix X
 * (column-major, device memory, overwritten): d_vec (n x maxvec,
 * column-major) receives *numcho vectors with X ~ vec vec^T, stopping when
 * the largest remaining diagonal is <= thr (thr < 0: 1e-6).  Returns
 * CD_InCore's irc: 0; 101 a diagonal below -1e-8; 102 more than maxvec
 * vectors needed; -1 maxvec < 1; or MG_ERR_ARG / MG_ERR_CUDA.  Synchronous. */
int mg_cd_incore(mg_handle* h, double* d_X, int n, double thr, double* d_vec, int maxvec, int* numcho,
                 void* stream);

/* ChoSCF_Drv with a decomposed density (scf/choscf_drv.F90:99-135): the
 * density D (nbf x nbf, device, symmetric PSD; not modified) is cut into its
 * Cholesky vectors by CD_InCore at 1e-8 of its largest diagonal (held by the
 * handle), which then drive CHO_LK_SCF: FLT += J[D] - FactXI K[D] as
 * mg_cho_lk_scf.  *nvec (may be NULL) receives the number of vectors (the
 * occupied count for an idempotent closed-shell density).  Returns 0,
 * CD_InCore's irc 101/102, or MG_ERR_*.  Synchronous. */
int mg_choscf_lk(mg_handle* h, const double* d_D, double factxi, double* d_FLT, int precision, int* nvec,
                 void* stream);

/* The 8-bit sliced tensor-core engine of MG_PREC_MIXED on given dense FP64
 * matrices (verification; no reference counterpart): X = A B with A
 * (ld x ld), B (ld x r) and X (ld x r) column-major, then K = X X^T into
 * the lower triangle of K (column-major ld x ld; the upper part of the
 * diagonal 128 x 128 tiles is also written).  ld a multiple of
 * 128, slices 2..8.  d_slices (slices x ld x ld bytes) and d_exps (ld ints),
 * when not NULL, receive the 8-bit slices and row exponents of A; slice p
 * holds A's element (i, k) at byte ((i / 128) (ld / 32) + k / 32) 4096 +
 * (i % 128) 32 + k % 32 (tiles of 128 rows x 32 columns, each contiguous).
 * Synchronous. */
int mg_sliced_selftest(mg_handle* h, int ld, int r, int slices, const double* d_A, const double* d_B, double* d_X,
                       double* d_K, void* d_slices, int* d_exps, void* stream);

/* Number of kernels of this library launched so far in this process (library
 * calls such as cuBLAS are not counted).  No reference counterpart. */
long long mg_kernel_launches(void);
/* Number of device allocations (cudaMalloc) this library has made so far in
 * this process, all handles together (allocations inside cuBLAS are not
 * counted).  No reference counterpart. */
long long mg_device_allocations(void);

#ifdef __cplusplus
}
#endif
#endif
