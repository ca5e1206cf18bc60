// amr_host.h -- host-side engine interface shared by the C ABI (amr_capi.cu) and the two
// precision instantiations (amr_engine_f64.cu, amr_engine_f32.cu).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/amr_b200.h"

namespace amrb {

// Host view of one case's device control record (mirrors CaseCtl).
struct CaseMeta {
  double time, target, dt, dt_trial;
  long long steps, rejected, maxsteps;
  int fatal, finished, active, live, cur;
};

// One admission request: mesh, parameters, initial state u0[u0_count] and the case's start
// (time, accepted and rejected steps) and first advance target.
struct AdmitSpec {
  const amr_mesh_view_t* mesh;
  const amr_params_t* params;
  const double* u0;
  uint64_t u0_count;
  double time0, target;
  long long steps0, rejected0, maxsteps;
};

class BatchBase {
 public:
  virtual ~BatchBase() = default;
  // Admits a case; returns 0, 1 (invalid input, message in *error) or 3 (no room).
  virtual int admit(const amr_mesh_view_t* mesh, const amr_params_t* params, const double* u0, uint64_t u0_count,
                    double time0, long long steps0, long long rejected0, double target, long long maxsteps,
                    int* slot, std::string* error) = 0;
  // Admits several cases, preparing them on `threads` host threads (0: up to 8); per case the
  // slot (-1 unless admitted), the status (0, 1 or 3 as admit) and the message of a status 1.
  // Slots and arena ranges go in request order whatever the thread count.  Returns 1 if any
  // case was invalid, else 3 if any found no room, else 0.
  virtual int admit_many(const std::vector<AdmitSpec>& specs, int threads, std::vector<int>* slots,
                         std::vector<int>* status, std::vector<std::string>* errors) = 0;
  virtual int release(int slot) = 0;
  // Runs `trials` trials of every live case and refreshes the host copies of the controls.
  virtual int advance(int trials, std::string* error) = 0;
  // advance in two halves: enqueue the trials (no wait), then wait and refresh the statuses.
  virtual int prepare_advance(int trials, std::string* error) = 0;
  virtual int advance_begin(int trials, std::string* error) = 0;
  virtual int advance_end(std::string* error) = 0;
  // The stream all of the batch's device work runs on (a group advance orders several batches'
  // streams against one start event).
  virtual cudaStream_t stream() const = 0;
  virtual int device() const = 0;
  // Sets a case's target time and step cap (the session's advance arguments).
  virtual int set_target(int slot, double target, long long maxsteps, std::string* error) = 0;
  // Residual of every live case's accepted state into the engine's residual buffer.
  virtual int residual(std::string* error) = 0;
  virtual int download_residual(int slot, double* out, uint64_t count, std::string* error) = 0;
  virtual int download(int slot, double* u, uint64_t count, std::string* error) = 0;
  virtual int download_many(const std::vector<int>& slots, double* const* outs, const uint64_t* counts,
                            std::string* error) = 0;
  // Compact results of one case from its accepted state, computed on the device: wall-stress
  // rows (14 per wall, viscous models), SA cell rows (3 per cell) and the convective and viscous
  // dt limits.  Runs one residual pass of the live cases first.
  virtual int export_case(int slot, double* wall_rows, uint64_t wall_count, double* sa_rows, uint64_t sa_count,
                          double* limits, std::string* error) = 0;
  virtual int n_walls(int slot) const = 0;
  // Region residual norms (5), region volume, Fx, Fy, Mz per requested case (9 doubles each).
  virtual int diagnostics(const std::vector<int>& slots, const std::vector<double>& region_moment,
                          std::vector<double>* out, std::string* error) = 0;
  virtual const CaseMeta& meta(int slot) const = 0;
  virtual int live_cases() const = 0;
  virtual int max_cases() const = 0;
  virtual uint64_t free_cells() const = 0;
  virtual int nv() const = 0;
  virtual int n_cells(int slot) const = 0;
  virtual double last_advance_seconds() const = 0;
  virtual uint64_t kernel_launches() const = 0;
  virtual amr_gpu_stats_t stats() const = 0;
  virtual int autotune(int trials, std::string* error) = 0;
  virtual void set_event_timing(bool on) = 0;
  virtual void set_graph(bool on) = 0;
  virtual int set_lanes(int lanes) = 0;  // 1 if lanes is not 1..4
  virtual std::string launch_config() const = 0;
};

std::unique_ptr<BatchBase> make_batch_f64(const amr_batch_config_t& config, std::string* error);
std::unique_ptr<BatchBase> make_batch_f32(const amr_batch_config_t& config, std::string* error);

}  // namespace amrb
