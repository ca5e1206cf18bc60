// amr_engine_f64.cu -- FP64 instantiation of the engine (the plain drop-in path).
// Built with -fmad=false: no contraction, so each expression rounds exactly as the
// reference CPU code it restates.
#include "amr_engine_inst.cuh"

namespace amrb {
template struct EngineOps<double>;

std::unique_ptr<BatchBase> make_batch_f64(const amr_batch_config_t& config, std::string* error) {
  auto b = std::make_unique<Batch<double>>();
  if (!b->init(config, error)) return nullptr;
  return b;
}
}  // namespace amrb
