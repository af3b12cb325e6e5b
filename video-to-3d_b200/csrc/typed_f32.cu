// Kernels of the dense pass for float pixel storage.
#include "typed_impl.cuh"

namespace v3d {
template struct Typed<float>;
}  // namespace v3d
