// Kernel instantiations for the D3Q19 velocity set.
#include "ops.cuh"
namespace lbm {
bool ops_d3q19(int storage, int trt, Ops* out) { return ops_for<D3Q19>(storage, trt, out); }
}  // namespace lbm
