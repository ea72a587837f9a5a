// FP32 engines: plain FP32 PCG (FP64 reductions only, FP32 couplings), and the
// mixed form: FP16-stored coarse couplings, FP32 V-cycle and CG, FP64 residual
// replacement into an FP64 solution.
#include "engine.cuh"

namespace uaamg {
Engine* create_engine_f32(int mixed) {
    if (mixed) return new EngineT<float, __half>(true);
    return new EngineT<float, float>(false);
}
}  // namespace uaamg
