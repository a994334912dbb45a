// Gradient kernel instantiations: one 512-thread CTA per SM (register
// budget of the __launch_bounds__ of grad_kernel); see grad_kernel.cuh.
#include "grad_kernel.cuh"

namespace mg {
GradFn grad_kernel_m1(int nab1, int ncd1) { return grad_pick<1>(nab1, ncd1); }
}  // namespace mg
