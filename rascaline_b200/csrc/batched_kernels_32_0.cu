// Instantiations of the batched kernel with CHUNK = 32, LAYOUT = 0
// (both NCAP variants), in a translation unit of their own so that the
// variants compile in parallel.
#include "batched_kernel.cuh"

namespace fb200 {
namespace batched_detail {

KernelFn kernel_32_0(bool small) {
    return small ? (KernelFn)batched_kernel<32, 0, 8> : (KernelFn)batched_kernel<32, 0, 16>;
}

}  // namespace batched_detail
}  // namespace fb200
