// Internal data structures of libmolgpu (host + device).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#define MG_MAX_RYS 9
#define MG_MAX_L 3

namespace mg {

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
  double* d_prim = nullptr;   // SoA: [7][tot_np]: zeta, kappa, Px, Py, Pz, alpha, beta
  int tot_np = 0;
  double* d_coef = nullptr;
  double* d_hrr = nullptr;
  double* d_rys = nullptr;
  RysMeta rys_meta[MG_MAX_RYS];
  int rys_nmax = 0, rys_degree = 0;
  std::vector<double> tmax;   // Schwarz bound per pair (sqrt max |(ab|ab)|)
  double* d_tmax = nullptr;
  Workspace ws;
  std::string err;
};

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

// device launchers (eri.cu)
int eri_run(Handle* h, const EriItem* d_items, const std::vector<int>& class_begin, const std::vector<int>& class_nab,
            const std::vector<int>& class_ncd, const std::vector<int>& class_np, const std::vector<size_t>& class_smem,
            double* out, cudaStream_t st);
void rys_upload_meta(Handle* h);

}  // namespace mg
