// ERI kernel instantiations for la+lb = 4..6 (see eri_kernel.cuh).
#include "eri_kernel.cuh"

namespace mg {
EriFn eri_kernel_pick_hi(int nab, int ncd) {
  switch (nab) {
    case 4: return eri_fn_b<4>(ncd);
    case 5: return eri_fn_b<5>(ncd);
    case 6: return eri_fn_b<6>(ncd);
  }
  return nullptr;
}
}  // namespace mg
