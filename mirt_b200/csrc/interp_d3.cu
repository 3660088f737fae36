// interp_d3.cu -- instantiates the 3D gather / spread kernels (interp_impl.cuh).
#include "interp_impl.cuh"

namespace mirt {
namespace detail {
cudaError_t dispatch_d3(Req &r) { return by_cw<3>(r); }
}  // namespace detail
}  // namespace mirt
