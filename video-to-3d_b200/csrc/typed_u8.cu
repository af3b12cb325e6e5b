// Kernels of the dense pass for uint8_t pixel storage.
#include "typed_impl.cuh"

namespace v3d {
template struct Typed<uint8_t>;
}  // namespace v3d
