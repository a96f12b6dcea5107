// Kernel instantiations for the D3Q15 velocity set.
#include "ops.cuh"
namespace lbm {
bool ops_d3q15(int storage, int trt, Ops* out) { return ops_for<D3Q15>(storage, trt, out); }
}  // namespace lbm
