// Kernel instantiations for the D2Q9 velocity set.
#include "ops.cuh"
namespace lbm {
bool ops_d2q9(int storage, int trt, Ops* out) { return ops_for<D2Q9>(storage, trt, out); }
}  // namespace lbm
