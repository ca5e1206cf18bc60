// amr_engine_f32.cu -- FP32 instantiation of the engine (the batched form): FP32 state,
// fluxes and accumulation; FP64 time, dt reduction, SRD weights, norms and loads.
#include "amr_engine_inst.cuh"

namespace amrb {
template struct EngineOps<float>;

std::unique_ptr<BatchBase> make_batch_f32(const amr_batch_config_t& config, std::string* error) {
  auto b = std::make_unique<Batch<float>>();
  if (!b->init(config, error)) return nullptr;
  return b;
}
}  // namespace amrb
