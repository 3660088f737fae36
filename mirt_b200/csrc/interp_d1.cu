// interp_d1.cu -- instantiates the 1D gather / spread kernels (interp_impl.cuh).
#include "interp_impl.cuh"

namespace mirt {
namespace detail {
cudaError_t dispatch_d1(Req &r) { return by_cw<1>(r); }
}  // namespace detail
}  // namespace mirt
