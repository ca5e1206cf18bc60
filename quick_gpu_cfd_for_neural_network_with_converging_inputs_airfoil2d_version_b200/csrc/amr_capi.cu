// amr_capi.cu -- the C ABI of include/amr_b200.h over the batch engine.
//
// The single-case session is a batch of one FP64 case; its five entry points keep the
// argument meaning, return codes and error texts of the reference session
// (src/static_amr2d_cuda.cu:274-366).  The batched API adds per-case steady retirement,
// evaluated on the device in FP64 with the reference driver's rule (src/quick_airfoil.cpp:180-208).
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "amr_host.h"

using amrb::BatchBase;
using amrb::AdmitSpec;

namespace {
void put(char* buf, uint64_t size, const std::string& text) {
  if (!buf || size == 0) return;
  const size_t n = std::min<size_t>(text.size(), size - 1);
  std::memcpy(buf, text.data(), n);
  buf[n] = 0;
}

int fail(char* buf, uint64_t size, const std::string& text) {
  put(buf, size, text);
  return 1;
}

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

std::unique_ptr<BatchBase> make_batch(const amr_batch_config_t& c, std::string* error) {
  if (c.precision == AMR_B200_PRECISION_FP64) return amrb::make_batch_f64(c, error);
  if (c.precision == AMR_B200_PRECISION_FP32) return amrb::make_batch_f32(c, error);
  if (error) *error = "precision must be 32 or 64";
  return nullptr;
}

// Exact table sizes of one mesh, for a batch that holds only it.
void size_for(const amr_mesh_view_t& m, amr_batch_config_t* c) {
  const uint64_t n = m.n_cells;
  c->max_cells = n;
  c->max_faces = (m.face_offsets ? m.face_offsets[n] : 0) + m.n_walls;  // face and wall slots
  c->max_walls = m.n_walls ? m.n_walls : 1;
  c->max_terms = (m.transport.model == AMR_B200_MODEL_LAMINAR && m.visc_offsets) ? m.visc_offsets[n] + 1 : 1;
  uint64_t nontrivial = 1;
  if (m.small_cells && m.member_offsets && m.group_offsets)
    for (uint64_t k = 0; k < n; ++k)
      if (m.member_offsets[k + 1] - m.member_offsets[k] != 1 || m.group_offsets[k + 1] - m.group_offsets[k] != 1) ++nontrivial;
  c->max_srd = nontrivial;
}
}  // namespace

struct amr_gpu_session {
  std::unique_ptr<BatchBase> batch;
  amr_gpu_options_t options;
  uint64_t n = 0;
  int nv = 4;
  double sa_nu_inf = 0;
  double setup_seconds = 0, advance_seconds = 0, download_seconds = 0;
};

extern "C" {

void amr_gpu_default_options(amr_gpu_options_t* o) {
  std::memset(o, 0, sizeof(*o));
  o->batch_trials = 32;
  o->graph = 1;
  o->fused = 1;
  o->sa_fused = 1;
  o->event_timing = 1;
}

int amr_gpu_create(const amr_mesh_view_t* mesh, const amr_params_t* params, const double* u0, uint64_t u0_count,
                   double time0, int64_t steps0, int64_t rejected0, const amr_gpu_options_t* options,
                   amr_gpu_session** out, char* error, uint64_t error_size) {
  if (!out) return 1;
  *out = nullptr;
  if (!mesh || !params || !u0 || !options) {
    put(error, error_size, "invalid AMR GPU configuration");
    return 1;
  }
  if (options->batch_trials < 1 || options->batch_trials > 1024) {
    put(error, error_size, "invalid AMR GPU configuration");
    return 1;
  }
  const double start = now();
  auto s = std::make_unique<amr_gpu_session>();
  s->options = *options;
  s->n = mesh->n_cells;
  s->nv = mesh->transport.sa_model ? 5 : 4;
  s->sa_nu_inf = mesh->transport.sa_nu_inf;
  amr_batch_config_t c;
  std::memset(&c, 0, sizeof(c));
  c.precision = AMR_B200_PRECISION_FP64;
  c.device = options->device;
  c.model = mesh->transport.model;
  c.sa_model = mesh->transport.sa_model;
  c.flux = params->flux;
  c.max_cases = 1;
  c.block_threads = options->block_threads;
  c.grid_blocks = options->grid_blocks;
  c.launch_mode = options->launch_mode;
  if (mesh->n_cells && mesh->face_offsets) size_for(*mesh, &c);
  std::string err;
  s->batch = make_batch(c, &err);
  if (!s->batch) {
    put(error, error_size, err);
    return 1;
  }
  int slot = -1;
  const int st = s->batch->admit(mesh, params, u0, u0_count, time0, steps0, rejected0, time0, 0, &slot, &err);
  if (st) {
    put(error, error_size, st == 3 ? std::string("AMR GPU arena too small") : err);
    return 1;
  }
  s->batch->set_graph(options->graph != 0);
  s->batch->set_event_timing(options->event_timing != 0);
  if (options->block_threads == 0 && options->grid_blocks == 0 && options->launch_mode == AMR_B200_LAUNCH_AUTO) {
    if (s->batch->set_target(0, 1e300, LLONG_MAX, &err) || s->batch->autotune(4, &err) ||
        s->batch->set_target(0, time0, 0, &err)) {
      put(error, error_size, "autotune: " + err);
      return 1;
    }
  }
  s->setup_seconds = now() - start;
  *out = s.release();
  return 0;
}

int amr_gpu_advance(amr_gpu_session* s, double tend, int64_t maxsteps, double wall_budget_seconds, amr_state_meta_t* meta,
                    char* error, uint64_t error_size) {
  if (!s || !meta || !std::isfinite(tend) || tend < s->batch->meta(0).time || maxsteps < 1 ||
      !std::isfinite(wall_budget_seconds) || wall_budget_seconds < 0) {
    put(error, error_size, "invalid AMR GPU advance");
    return 1;
  }
  const double start = now();
  std::string err;
  if (s->batch->set_target(0, tend, maxsteps, &err)) {
    put(error, error_size, err);
    return 1;
  }
  bool expired = false;
  for (;;) {
    if (s->batch->advance(s->options.batch_trials, &err)) {
      put(error, error_size, err);
      s->advance_seconds += now() - start;
      return 1;
    }
    const amrb::CaseMeta& m = s->batch->meta(0);
    if (m.fatal || m.finished) break;
    if (wall_budget_seconds > 0 && now() - start >= wall_budget_seconds) {
      expired = true;
      break;
    }
  }
  s->advance_seconds += now() - start;
  const amrb::CaseMeta& m = s->batch->meta(0);
  meta->time = m.time;
  meta->steps = m.steps;
  meta->rejected = m.rejected;
  meta->status = m.fatal;
  meta->finished = m.finished;
  if (m.fatal) {
    put(error, error_size, "AMR GPU stopped with status " + std::to_string(m.fatal) + "; last accepted state retained");
    return 1;
  }
  return expired ? 2 : 0;
}

int amr_gpu_download(amr_gpu_session* s, double* u, uint64_t count, amr_state_meta_t* meta, char* error,
                     uint64_t error_size) {
  if (!s || !u) {
    put(error, error_size, "invalid AMR GPU download");
    return 1;
  }
  const double start = now();
  std::string err;
  if (s->batch->download(0, u, count, &err)) {
    put(error, error_size, err);
    return 1;
  }
  if (meta) {
    const amrb::CaseMeta& m = s->batch->meta(0);
    meta->time = m.time;
    meta->steps = m.steps;
    meta->rejected = m.rejected;
    meta->status = m.fatal;
    meta->finished = m.finished;
  }
  s->download_seconds += now() - start;
  return 0;
}

int amr_gpu_stats(const amr_gpu_session* s, amr_gpu_stats_t* out) {
  if (!out) return 1;
  std::memset(out, 0, sizeof(*out));
  if (!s) return 0;
  *out = s->batch->stats();
  out->setup_seconds = s->setup_seconds;
  out->advance_seconds = s->advance_seconds;
  out->download_seconds = s->download_seconds;
  return 0;
}

void amr_gpu_destroy(amr_gpu_session* s) { delete s; }

int amr_gpu_residual(amr_gpu_session* s, double* r, uint64_t count, char* error, uint64_t error_size) {
  if (!s || !r) {
    put(error, error_size, "invalid AMR GPU residual");
    return 1;
  }
  std::string err;
  if (s->batch->residual(&err) || s->batch->download_residual(0, r, count, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_gpu_export(amr_gpu_session* s, double* wall_rows, uint64_t wall_count, double* sa_rows, uint64_t sa_count,
                   double limits[2], char* error, uint64_t error_size) {
  if (!s) {
    put(error, error_size, "invalid AMR GPU export");
    return 1;
  }
  std::string err;
  if (s->batch->export_case(0, wall_rows, wall_count, sa_rows, sa_count, limits, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_gpu_diagnostics(amr_gpu_session* s, const double region[4], double mx, double my, double out[8], char* error,
                        uint64_t error_size) {
  if (!s || !region || !out) {
    put(error, error_size, "invalid AMR GPU diagnostics");
    return 1;
  }
  std::vector<double> rm = {region[0], region[1], region[2], region[3], mx, my}, res;
  std::string err;
  if (s->batch->diagnostics({0}, rm, &res, &err)) {
    put(error, error_size, err);
    return 1;
  }
  const double volume = res[5];
  for (int v = 0; v < 5; ++v) out[v] = v < s->nv && volume > 0 ? res[v] / volume : 0.0;
  if (s->nv == 5) out[4] /= s->sa_nu_inf;
  out[5] = res[6];
  out[6] = res[7];
  out[7] = res[8];
  return 0;
}

}  // extern "C"

// ----------------------------------------------------------------------------------------
// Batched form.
// ----------------------------------------------------------------------------------------
struct CaseSteady {
  amr_case_control_t ctl;
  bool previous = false, converged = false, retired = false;
  double prevcl = 0, prevcd = 0, prevcm = 0, cl = 0, cd = 0, cm = 0;
  double res[5] = {0, 0, 0, 0, 0};
  int hold = 0, checks = 0;
  double sa_nu_inf = 0;
  int nv = 4;
};

struct amr_batch {
  std::unique_ptr<BatchBase> batch;
  std::vector<CaseSteady> steady;
};

extern "C" {

int amr_batch_create(const amr_batch_config_t* config, amr_batch** out, char* error, uint64_t error_size) {
  if (!out || !config) return 1;
  *out = nullptr;
  std::string err;
  auto b = std::make_unique<amr_batch>();
  b->batch = make_batch(*config, &err);
  if (!b->batch) {
    put(error, error_size, err);
    return 1;
  }
  b->steady.assign(config->max_cases, CaseSteady());
  *out = b.release();
  return 0;
}

int amr_batch_admit(amr_batch* b, const amr_mesh_view_t* mesh, const amr_params_t* params, const double* u0,
                    uint64_t u0_count, const amr_case_control_t* control, int32_t* slot, char* error,
                    uint64_t error_size) {
  if (!b || !mesh || !control || !slot) return 1;
  const amr_case_control_t& c = *control;
  const bool steady = c.check_period > 0;
  const double first = steady ? std::min(c.first_check, c.tend) : c.tend;
  std::string err;
  int s = -1;
  const int st = b->batch->admit(mesh, params, u0, u0_count, 0.0, 0, 0, first, c.maxsteps, &s, &err);
  if (st) {
    if (st != 3) put(error, error_size, err);
    return st;
  }
  CaseSteady cs;
  cs.ctl = c;
  cs.sa_nu_inf = mesh->transport.sa_nu_inf;
  cs.nv = mesh->transport.sa_model ? 5 : 4;
  b->steady[s] = cs;
  *slot = s;
  return 0;
}

int amr_batch_admit_many(amr_batch* b, uint64_t count, const amr_mesh_view_t* const* meshes,
                         const amr_params_t* const* params, const double* const* u0, const uint64_t* u0_counts,
                         const amr_case_control_t* const* controls, int32_t threads, int32_t* slots,
                         int32_t* status, char* error, uint64_t error_size) {
  if (!b || (count && (!meshes || !params || !u0 || !u0_counts || !controls || !slots || !status))) return 1;
  std::vector<AdmitSpec> specs(count);
  for (uint64_t i = 0; i < count; ++i) {
    if (!meshes[i] || !controls[i]) {
      put(error, error_size, "null mesh or control");
      return 1;
    }
    const amr_case_control_t& c = *controls[i];
    const double first = c.check_period > 0 ? std::min(c.first_check, c.tend) : c.tend;
    specs[i] = AdmitSpec{meshes[i], params[i], u0[i], u0_counts[i], 0.0, first, 0, 0, c.maxsteps};
  }
  std::vector<int> s, st;
  std::vector<std::string> errs;
  const int rc = b->batch->admit_many(specs, threads, &s, &st, &errs);
  bool reported = false;
  for (uint64_t i = 0; i < count; ++i) {
    slots[i] = s[i];
    status[i] = st[i];
    if (st[i] == 1 && !reported) {
      put(error, error_size, "case " + std::to_string(i) + ": " + errs[i]);
      reported = true;
    }
    if (st[i] != 0) continue;
    CaseSteady cs;
    cs.ctl = *controls[i];
    cs.sa_nu_inf = meshes[i]->transport.sa_nu_inf;
    cs.nv = meshes[i]->transport.sa_model ? 5 : 4;
    b->steady[s[i]] = cs;
  }
  return rc;
}

int amr_batch_advance(amr_batch* b, int32_t trials, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->advance(trials, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_advance_async(amr_batch* b, int32_t trials, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->advance_begin(trials, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_wait(amr_batch* b, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->advance_end(&err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_group_advance(amr_batch* const* batches, int32_t count, int32_t trials, double* device_seconds,
                            char* error, uint64_t error_size) {
  if (!batches || count < 1) return fail(error, error_size, "no batches");
  for (int i = 0; i < count; ++i) {
    if (!batches[i]) return fail(error, error_size, "null batch");
    for (int j = 0; j < i; ++j)
      if (batches[j] == batches[i]) return fail(error, error_size, "a batch appears twice");
    if (batches[i]->batch->device() != batches[0]->batch->device())
      return fail(error, error_size, "the batches are on different devices");
  }
  int previous = 0;
  if (cudaGetDevice(&previous) != cudaSuccess || cudaSetDevice(batches[0]->batch->device()) != cudaSuccess)
    return fail(error, error_size, "cannot select the batches' device");
  std::string err;
  std::vector<cudaEvent_t> ev(count + 1, nullptr);
  bool ok = true;
  // host-side preparation (uploads, graph captures) of every batch before the start event, so
  // that the device time covers the trials alone
  for (int i = 0; ok && i < count; ++i)
    if (batches[i]->batch->prepare_advance(trials, &err)) ok = false;
  for (int i = 0; ok && i <= count; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) {
      ok = false;
      err = "event creation";
    }
  // every batch's work starts after one start event; each batch's end is recorded on its stream
  if (ok && cudaEventRecord(ev[0], batches[0]->batch->stream()) != cudaSuccess) {
    ok = false;
    err = "start event";
  }
  for (int i = 1; ok && i < count; ++i)
    if (cudaStreamWaitEvent(batches[i]->batch->stream(), ev[0], 0) != cudaSuccess) {
      ok = false;
      err = "stream ordering";
    }
  int begun = 0;
  for (; ok && begun < count; ++begun)
    if (batches[begun]->batch->advance_begin(trials, &err)) ok = false;
  for (int i = 0; ok && i < count; ++i)
    if (cudaEventRecord(ev[i + 1], batches[i]->batch->stream()) != cudaSuccess) {
      ok = false;
      err = "end event";
    }
  // complete every advance that began, also on an error path
  for (int i = 0; i < begun; ++i) {
    std::string e;
    if (batches[i]->batch->advance_end(&e) && ok) {
      ok = false;
      err = e;
    }
  }
  double seconds = 0.0;
  for (int i = 0; ok && i < count; ++i) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ev[0], ev[i + 1]) != cudaSuccess) {
      ok = false;
      err = "event timing";
    }
    seconds = std::max(seconds, 1e-3 * (double)ms);
  }
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  cudaSetDevice(previous);
  if (!ok) return fail(error, error_size, err);
  if (device_seconds) *device_seconds = seconds;
  return 0;
}

uint64_t amr_batch_device_bytes(const amr_batch* b) { return b ? b->batch->stats().allocated_bytes : 0; }

int amr_device_memory(int32_t device, uint64_t* free_bytes, uint64_t* total_bytes) {
  if (!free_bytes || !total_bytes) return 1;
  int previous = 0;
  if (cudaGetDevice(&previous) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return 1;
  size_t f = 0, t = 0;
  const cudaError_t st = cudaMemGetInfo(&f, &t);
  cudaSetDevice(previous);
  if (st != cudaSuccess) return 1;
  *free_bytes = f;
  *total_bytes = t;
  return 0;
}

// Steady rule of the reference driver: residual norms over the region and the load changes
// must stay within tolerance for `hold` consecutive checks once time >= min_time.
int amr_batch_check(amr_batch* b, char* error, uint64_t error_size) {
  if (!b) return 1;
  BatchBase& B = *b->batch;
  std::vector<int> due;
  std::vector<double> rm;
  for (int s = 0; s < B.max_cases(); ++s) {
    CaseSteady& cs = b->steady[s];
    const amrb::CaseMeta& m = B.meta(s);
    if (!m.live || cs.retired) continue;
    if (m.fatal) {
      cs.retired = true;
      continue;
    }
    if (!m.finished) continue;
    if (cs.ctl.check_period <= 0 || m.time >= cs.ctl.tend) {
      if (cs.ctl.check_period <= 0) {
        cs.retired = true;
        continue;
      }
    }
    due.push_back(s);
    for (int v = 0; v < 4; ++v) rm.push_back(cs.ctl.region[v]);
    rm.push_back(cs.ctl.moment_x);
    rm.push_back(cs.ctl.moment_y);
  }
  if (due.empty()) return 0;
  std::vector<double> out;
  std::string err;
  if (B.diagnostics(due, rm, &out, &err)) {
    put(error, error_size, err);
    return 1;
  }
  for (size_t i = 0; i < due.size(); ++i) {
    const int s = due[i];
    CaseSteady& cs = b->steady[s];
    const amrb::CaseMeta& m = B.meta(s);
    const double* r = &out[9 * i];
    const double volume = r[5];
    for (int v = 0; v < 5; ++v) cs.res[v] = v < cs.nv && volume > 0 ? r[v] / volume : 0.0;
    if (cs.nv == 5) cs.res[4] /= cs.sa_nu_inf;
    const double a = cs.ctl.aoa_degrees * std::acos(-1.0) / 180, cosa = std::cos(a), sina = std::sin(a);
    const double q = .5 * cs.ctl.mach * cs.ctl.mach;
    const double fx = r[6], fy = r[7], mz = r[8];
    cs.cl = (-fx * sina + fy * cosa) / q;
    cs.cd = (fx * cosa + fy * sina) / q;
    cs.cm = mz / q;
    const double inf = INFINITY;
    const double dcl = cs.previous ? std::fabs(cs.cl - cs.prevcl) / std::max(.1, std::fabs(cs.cl)) : inf;
    const double dcd = cs.previous ? std::fabs(cs.cd - cs.prevcd) / std::max(.01, std::fabs(cs.cd)) : inf;
    const double dcm = cs.previous ? std::fabs(cs.cm - cs.prevcm) / std::max(.01, std::fabs(cs.cm)) : inf;
    const double rmax = *std::max_element(cs.res, cs.res + 5);
    if (m.time >= cs.ctl.min_time && rmax <= cs.ctl.raw_tol && dcl <= cs.ctl.load_tol && dcd <= cs.ctl.load_tol &&
        dcm <= cs.ctl.load_tol)
      ++cs.hold;
    else
      cs.hold = 0;
    cs.prevcl = cs.cl;
    cs.prevcd = cs.cd;
    cs.prevcm = cs.cm;
    cs.previous = true;
    ++cs.checks;
    if (cs.hold >= cs.ctl.hold) {
      cs.converged = true;
      cs.retired = true;
      continue;
    }
    if (m.time >= cs.ctl.tend) {
      cs.retired = true;
      continue;
    }
    const double next = cs.checks == 1 ? std::min(cs.ctl.tend, cs.ctl.check_period) : std::min(cs.ctl.tend, m.target + cs.ctl.check_period);
    if (B.set_target(s, next, cs.ctl.maxsteps, &err)) {
      put(error, error_size, err);
      return 1;
    }
  }
  return 0;
}

int amr_batch_status(const amr_batch* b, int32_t slot, amr_case_status_t* out) {
  if (!b || !out || slot < 0 || slot >= b->batch->max_cases()) return 1;
  const amrb::CaseMeta& m = b->batch->meta(slot);
  const CaseSteady& cs = b->steady[slot];
  std::memset(out, 0, sizeof(*out));
  out->time = m.time;
  out->steps = m.steps;
  out->rejected = m.rejected;
  out->status = m.fatal;
  out->finished = cs.retired ? 1 : 0;
  out->converged = cs.converged ? 1 : 0;
  out->checks = cs.checks;
  out->hold = cs.hold;
  for (int v = 0; v < 5; ++v) out->residual[v] = cs.res[v];
  out->cl = cs.cl;
  out->cd = cs.cd;
  out->cm = cs.cm;
  return 0;
}

int amr_batch_export(amr_batch* b, int32_t slot, double* wall_rows, uint64_t wall_count, double* sa_rows, uint64_t sa_count,
                     double limits[2], char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->export_case(slot, wall_rows, wall_count, sa_rows, sa_count, limits, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_download(amr_batch* b, int32_t slot, double* u, uint64_t count, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->download(slot, u, count, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_download_many(amr_batch* b, uint64_t count, const int32_t* slots, double* const* u_out,
                            const uint64_t* u_counts, char* error, uint64_t error_size) {
  if (!b || (count && (!slots || !u_out || !u_counts))) return 1;
  std::string err;
  if (b->batch->download_many(std::vector<int>(slots, slots + count), u_out, u_counts, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_release(amr_batch* b, int32_t slot) {
  if (!b) return 1;
  if (b->batch->release(slot)) return 1;
  b->steady[slot] = CaseSteady();
  return 0;
}

int amr_batch_live_cases(const amr_batch* b) { return b ? b->batch->live_cases() : 0; }
uint64_t amr_batch_free_cells(const amr_batch* b) { return b ? b->batch->free_cells() : 0; }
double amr_batch_last_advance_seconds(const amr_batch* b) { return b ? b->batch->last_advance_seconds() : 0.0; }
uint64_t amr_batch_kernel_launches(const amr_batch* b) { return b ? b->batch->kernel_launches() : 0; }
void amr_batch_destroy(amr_batch* b) { delete b; }

// Extra entry points used by the Python host mirror (not part of the reference surface).
int amr_batch_autotune(amr_batch* b, int32_t trials, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->autotune(trials, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_batch_launch_config(const amr_batch* b, char* out, uint64_t size) {
  if (!b) return 1;
  put(out, size, b->batch->launch_config());
  return 0;
}

int amr_batch_set_graph(amr_batch* b, int32_t on) {
  if (!b) return 1;
  b->batch->set_graph(on != 0);
  return 0;
}

int amr_batch_set_lanes(amr_batch* b, int32_t lanes) {
  if (!b) return 1;
  return b->batch->set_lanes(lanes);
}

int amr_batch_set_target(amr_batch* b, int32_t slot, double target, int64_t maxsteps, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->set_target(slot, target, maxsteps, &err)) {
    put(error, error_size, err);
    return 1;
  }
  b->steady[slot].ctl.tend = std::max(b->steady[slot].ctl.tend, target);
  return 0;
}

int amr_batch_residual(amr_batch* b, int32_t slot, double* r, uint64_t count, char* error, uint64_t error_size) {
  if (!b) return 1;
  std::string err;
  if (b->batch->residual(&err) || b->batch->download_residual(slot, r, count, &err)) {
    put(error, error_size, err);
    return 1;
  }
  return 0;
}

int amr_gpu_launch_config(const amr_gpu_session* s, char* out, uint64_t size) {
  if (!s) return 1;
  put(out, size, s->batch->launch_config());
  return 0;
}

uint64_t amr_gpu_kernel_launches(const amr_gpu_session* s) { return s ? s->batch->kernel_launches() : 0; }

}  // extern "C"
