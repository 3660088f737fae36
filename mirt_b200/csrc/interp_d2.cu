// interp_d2.cu -- instantiates the 2D gather / spread kernels (interp_impl.cuh).
#include "interp_impl.cuh"

namespace mirt {
namespace detail {
cudaError_t dispatch_d2(Req &r) { return by_cw<2>(r); }
}  // namespace detail
}  // namespace mirt
