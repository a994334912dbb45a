// ERI kernel instantiations for la+lb = 0..3 (see eri_kernel.cuh).
#include "eri_kernel.cuh"

namespace mg {
EriFn eri_kernel_pick_lo(int nab, int ncd) {
  switch (nab) {
    case 0: return eri_fn_b<0>(ncd);
    case 1: return eri_fn_b<1>(ncd);
    case 2: return eri_fn_b<2>(ncd);
    case 3: return eri_fn_b<3>(ncd);
  }
  return nullptr;
}
}  // namespace mg
