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

/* Error codes (mirroring Cho_Drv's 0/1/2 where they apply). */
#define MG_OK 0
#define MG_ERR_ARG 1       /* bad argument / unsupported input          */
#define MG_ERR_MEMORY 2    /* device allocation failed                  */
#define MG_ERR_CUDA 3      /* CUDA launch or runtime error              */
#define MG_ERR_DECOMP 104  /* Cholesky decomposition error (Cho_Quit 104) */

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
int mg_eri_quartets(mg_handle* h, const int32_t* quartets, int64_t nq, const int64_t* offsets, double* d_out,
                    void* stream);

#ifdef __cplusplus
}
#endif
#endif
