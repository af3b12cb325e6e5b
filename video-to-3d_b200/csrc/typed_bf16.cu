// Kernels of the dense pass for __nv_bfloat16 pixel storage.
#include "typed_impl.cuh"

namespace v3d {
template struct Typed<__nv_bfloat16>;
}  // namespace v3d
