// FP32 engines: plain FP32 PCG (FP64 reductions only), and the mixed form with
// FP64 residual replacement into an FP64 solution.
#include "engine.cuh"

namespace uaamg {
Engine* create_engine_f32(int mixed) { return new EngineT<float>(mixed != 0); }
}  // namespace uaamg
