// FP64 (reference-exact) engine.  Built with -fmad=false: every product and sum
// rounds separately, in the reference's order, so per-cell results (V-cycle,
// matvec) match its x86-64 build bit for bit.
#include "engine.cuh"

namespace uaamg {
Engine* create_engine_f64() { return new EngineT<double>(false); }
}  // namespace uaamg
