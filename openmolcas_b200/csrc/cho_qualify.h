// Cho_Qualify_2 (cholesky_util/cho_qualify_2.F90; IALQUA = 2, the default of
// cho_inp.F90:156) for one shell pair: which of its reduced-set diagonals
// become columns of the next pass.  Host code, no CUDA: the device
// decomposition calls it between passes and a CPU test compiles it alone.
//
// diag[t], inred[t] for the cnt AO pairs t of the shell pair (in rs order);
// returns the chosen positions t.  With maxqual > 1 the diagonals >= diamin
// are taken in order; once maxqual are taken, a larger one replaces the
// smallest taken (the first of equal smallest).  With maxqual == 1 the
// largest >= diamin is taken (the last of equal largest).
#pragma once
#include <vector>

namespace mg {

inline std::vector<int> cho_qualify_2(const double* diag, const unsigned char* inred, int cnt, double diamin,
                                      int maxqual) {
  std::vector<int> qual;
  if (maxqual == 1) {
    double xmax = diamin;
    int imax = -1;
    for (int t = 0; t < cnt; ++t)
      if (inred[t] && diag[t] >= xmax) { xmax = diag[t]; imax = t; }
    if (imax >= 0) qual.push_back(imax);
    return qual;
  }
  for (int t = 0; t < cnt; ++t) {
    if (!inred[t] || !(diag[t] >= diamin)) continue;
    if ((int)qual.size() < maxqual) {
      qual.push_back(t);
    } else {
      size_t kmin = 0;
      for (size_t k = 1; k < qual.size(); ++k)
        if (diag[qual[k]] < diag[qual[kmin]]) kmin = k;
      if (diag[t] > diag[qual[kmin]]) qual[kmin] = t;
    }
  }
  return qual;
}

}  // namespace mg
