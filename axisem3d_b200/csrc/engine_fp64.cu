// FP64 engine: the reference built with -Ddouble=true.
#include "engine_impl.cuh"
namespace axg {
std::unique_ptr<EngineBase> make_engine_fp64(const axg_config &cfg) {
    return std::make_unique<Engine<double, double, double, false>>(cfg);
}
}  // namespace axg
