// Gradient kernel instantiations for 3 resident CTA(s) per SM (register
// budget of __launch_bounds__(256, 3)); see grad_kernel.cuh.
#include "grad_kernel.cuh"

namespace mg {
GradFn grad_kernel_m3(int nab1, int ncd1) { return grad_pick<3>(nab1, ncd1); }
}  // namespace mg
