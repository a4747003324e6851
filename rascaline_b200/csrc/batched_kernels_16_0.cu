// Instantiations of the batched kernel with CHUNK = 16, LAYOUT = 0
// (both NCAP variants), in a translation unit of their own so that the
// variants compile in parallel.
#include "batched_kernel.cuh"

namespace fb200 {
namespace batched_detail {

KernelFn kernel_16_0(bool small) {
    return small ? (KernelFn)batched_kernel<16, 0, 8> : (KernelFn)batched_kernel<16, 0, 16>;
}

}  // namespace batched_detail
}  // namespace fb200
