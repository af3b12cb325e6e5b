// Kernels of the dense pass for __half pixel storage.
#include "typed_impl.cuh"

namespace v3d {
template struct Typed<__half>;
}  // namespace v3d
