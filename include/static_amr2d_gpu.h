// static_amr2d_gpu.h -- the reference's C++ session API, served by the B200 engine.
//
// Declares the same five entry points, option and statistics records as the reference header
// (src/static_amr2d_gpu.h:8-24 in the reference), so code written against that header links
// unchanged against libamr_b200.so plus csrc/static_amr2d_gpu_b200.cpp in place of the
// reference's src/static_amr2d_cuda.cu.  The mesh, parameter and state types come from the
// reference's own src/static_amr2d.h, which must be on the include path.  The include guard is
// the reference's, so a translation unit sees exactly one declaration of this API.
#ifndef CFD_STATIC_AMR2D_GPU_H
#define CFD_STATIC_AMR2D_GPU_H
#include <cstdint>
#include <string>

#include "static_amr2d.h"

namespace cfd {
struct StaticAmrGpu;

// batch_trials: trials per status poll (1..1024); graph: replay each poll from a CUDA graph;
// fused, sa_fused: accepted, the engine always runs its fused kernel; event_timing: CUDA-event
// time per poll in AmrGpuStats::advance_event_seconds.
struct AmrGpuOptions {
  int batch_trials = 32;
  bool graph = true;
  bool fused = false;
  bool event_timing = false;
  bool sa_fused = false;
};

struct AmrGpuStats {
  uint64_t allocated_bytes = 0, pinned_bytes = 0, geometry_h2d_bytes = 0, state_h2d_bytes = 0;
  uint64_t control_h2d_bytes = 0;
  uint64_t control_d2h_bytes = 0, state_d2h_bytes = 0, status_polls = 0, full_downloads = 0;
  double setup_seconds = 0, advance_seconds = 0, download_seconds = 0;
  double advance_event_seconds = 0;
  uint64_t event_batches = 0, graph_nodes_per_trial = 0;
};

// 0 on success; 1 with a message on invalid input or a CUDA failure (*out = nullptr).
int static_amr_gpu_create(const StaticAmrMesh2D&, const Params2D&, const StaticAmrState2D&, const AmrGpuOptions&,
                          StaticAmrGpu**, std::string*);
// Advances to tend (exactly, by clipping the last dt) or a fatal status; updates only the
// state's time/steps/rejected.  0 done, 1 fatal (status text; last accepted state kept), 2
// wall budget expired (resumable).
int static_amr_gpu_advance(StaticAmrGpu*, double tend, long maxsteps, StaticAmrState2D*, std::string*,
                           double wall_budget_seconds = 0);
// Copies the accepted state into state->u.
int static_amr_gpu_download(StaticAmrGpu*, StaticAmrState2D*, std::string*);
AmrGpuStats static_amr_gpu_stats(const StaticAmrGpu*);
void static_amr_gpu_destroy(StaticAmrGpu*);
}  // namespace cfd
#endif
