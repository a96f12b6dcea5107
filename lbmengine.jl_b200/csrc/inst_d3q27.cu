// Kernel instantiations for the D3Q27 velocity set.
#include "ops.cuh"
namespace lbm {
bool ops_d3q27(int storage, int trt, Ops* out) { return ops_for<D3Q27>(storage, trt, out); }
}  // namespace lbm
