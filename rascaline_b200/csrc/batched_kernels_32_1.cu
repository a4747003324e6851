// Instantiations of the batched kernel with CHUNK = 32, LAYOUT = 1
// (both NCAP variants), in a translation unit of their own so that the
// variants compile in parallel.
#include "batched_kernel.cuh"

namespace fb200 {
namespace batched_detail {

KernelFn kernel_32_1(bool small) {
    return small ? (KernelFn)batched_kernel<32, 1, 8> : (KernelFn)batched_kernel<32, 1, 16>;
}

}  // namespace batched_detail
}  // namespace fb200
