// Mixed engine: float stiffness, double attenuation memory variables, double
// Newmark displacement/velocity (optionally with compensated summation).
#include "engine_impl.cuh"
namespace axg {
std::unique_ptr<EngineBase> make_engine_mixed(const axg_config &cfg) {
    if (cfg.compensated) return std::make_unique<Engine<float, double, double, true>>(cfg);
    return std::make_unique<Engine<float, double, double, false>>(cfg);
}
}  // namespace axg
