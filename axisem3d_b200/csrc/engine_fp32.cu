// FP32 engine: the reference's default single-precision build.
#include "engine_impl.cuh"
namespace axg {
std::unique_ptr<EngineBase> make_engine_fp32(const axg_config &cfg) {
    return std::make_unique<Engine<float, float, float, false>>(cfg);
}
}  // namespace axg
