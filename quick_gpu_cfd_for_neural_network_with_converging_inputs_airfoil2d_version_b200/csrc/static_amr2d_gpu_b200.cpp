// static_amr2d_gpu_b200.cpp -- the reference's C++ session API over the C ABI of amr_b200.h.
//
// Link-time replacement for the reference's src/static_amr2d_cuda.cu: compile this file against
// the reference's headers (src/ on the include path, ahead of nothing else that defines
// CFD_STATIC_AMR2D_GPU_H) and link libamr_b200.so.  The reference's mesh records are passed by
// pointer: their layouts equal the C ABI records, which the static_asserts below verify.
#include <cstddef>
#include <cstring>

#include "amr_b200.h"
#include "static_amr2d_gpu.h"

namespace cfd {

static_assert(sizeof(amr_cell_t) == sizeof(AmrCell2D) && offsetof(amr_cell_t, volume) == offsetof(AmrCell2D, volume) &&
                  offsetof(amr_cell_t, wall_begin) == offsetof(AmrCell2D, wall_begin),
              "AmrCell2D layout");
static_assert(sizeof(amr_face_t) == sizeof(AmrFace2D) && offsetof(amr_face_t, length) == offsetof(AmrFace2D, length),
              "AmrFace2D layout");
static_assert(sizeof(amr_wall_t) == sizeof(WallFragment2D) && offsetof(amr_wall_t, nx) == offsetof(WallFragment2D, nx) &&
                  offsetof(amr_wall_t, length) == offsetof(WallFragment2D, length),
              "WallFragment2D layout");
static_assert(sizeof(amr_gradient_term_t) == sizeof(AmrGradientTerm2D), "AmrGradientTerm2D layout");
static_assert(sizeof(amr_wall_sample_t) == sizeof(AmrWallSample2D), "AmrWallSample2D layout");
static_assert(sizeof(amr_face_geometry_t) == sizeof(AmrViscousFaceGeometry2D), "AmrViscousFaceGeometry2D layout");
static_assert(sizeof(amr_boundary_t) == sizeof(AmrBoundary2D) &&
                  offsetof(amr_boundary_t, wall_velocity) == offsetof(AmrBoundary2D, wall_velocity),
              "AmrBoundary2D layout");
static_assert(sizeof(amr_transport_t) == sizeof(AmrTransport2D) &&
                  offsetof(amr_transport_t, wall_probe_min_h) == offsetof(AmrTransport2D, wall_probe_min_h),
              "AmrTransport2D layout");
static_assert(sizeof(size_t) == sizeof(uint64_t), "LP64 target");
static_assert(sizeof(amr_gpu_stats_t) == sizeof(AmrGpuStats), "AmrGpuStats layout");

struct StaticAmrGpu {
  amr_gpu_session* session = nullptr;
  size_t values = 0;
};

namespace {
const uint64_t* u64(const std::vector<size_t>& v) { return reinterpret_cast<const uint64_t*>(v.data()); }

amr_mesh_view_t view_of(const StaticAmrMesh2D& m) {
  amr_mesh_view_t v;
  std::memset(&v, 0, sizeof(v));
  v.n_cells = m.cells.size();
  v.n_faces = m.faces.size();
  v.n_walls = m.walls.size();
  v.cells = reinterpret_cast<const amr_cell_t*>(m.cells.data());
  v.faces = reinterpret_cast<const amr_face_t*>(m.faces.data());
  v.walls = reinterpret_cast<const amr_wall_t*>(m.walls.data());
  v.face_offsets = u64(m.face_offsets);
  v.cell_faces = u64(m.cell_faces);
  v.group_offsets = u64(m.group_offsets);
  v.group_members = u64(m.group_members);
  v.member_offsets = u64(m.member_offsets);
  v.member_groups = u64(m.member_groups);
  v.group_volume = m.group_volume.data();
  v.small_cells = m.small_cells;
  v.agglomerate_small = m.options.agglomerate_small ? 1 : 0;
  for (int side = 0; side < 4; ++side) std::memcpy(&v.boundaries[side], &m.boundaries[side], sizeof(amr_boundary_t));
  std::memcpy(&v.transport, &m.transport, sizeof(amr_transport_t));
  if (m.transport.model == AMR_MODEL_LAMINAR) {
    v.visc_offsets = u64(m.viscous.offsets);
    v.visc_terms = reinterpret_cast<const amr_gradient_term_t*>(m.viscous.terms.data());
    v.wall_samples = reinterpret_cast<const amr_wall_sample_t*>(m.viscous.wall_samples.data());
    v.face_samples = reinterpret_cast<const amr_wall_sample_t*>(m.viscous.face_samples.data());
    v.face_geometry = reinterpret_cast<const amr_face_geometry_t*>(m.viscous.face_geometry.data());
    v.wall_distance = m.viscous.wall_distance.empty() ? nullptr : m.viscous.wall_distance.data();
  }
  return v;
}

amr_params_t params_of(const Params2D& p) {
  amr_params_t q;
  std::memset(&q, 0, sizeof(q));
  q.gamma = p.gamma;
  q.cfl = p.cfl;
  q.dt_fixed = p.dt_fixed;
  q.ausm_mco = p.ausm_mco;
  q.flux = p.flux;
  q.limiter = p.limiter;
  q.time_integrator = p.time_integrator;
  for (int i = 0; i < 4; ++i) q.bc[i] = p.bc[i];
  return q;
}

void set_error(std::string* error, const char* text) {
  if (error) *error = text;
}
}  // namespace

int static_amr_gpu_create(const StaticAmrMesh2D& m, const Params2D& p, const StaticAmrState2D& initial,
                          const AmrGpuOptions& options, StaticAmrGpu** result, std::string* error) {
  if (!result) return 1;
  *result = nullptr;
  if (!static_amr2d_viscous_ready(m) || m.cells.empty() || m.faces.empty() || m.face_offsets.size() != m.cells.size() + 1) {
    set_error(error, "invalid AMR GPU configuration");
    return 1;
  }
  const amr_mesh_view_t view = view_of(m);
  const amr_params_t params = params_of(p);
  amr_gpu_options_t o;
  amr_gpu_default_options(&o);
  o.batch_trials = options.batch_trials;
  o.graph = options.graph ? 1 : 0;
  o.fused = options.fused ? 1 : 0;
  o.event_timing = options.event_timing ? 1 : 0;
  o.sa_fused = options.sa_fused ? 1 : 0;
  char message[512] = {0};
  amr_gpu_session* session = nullptr;
  if (amr_gpu_create(&view, &params, initial.u.data(), initial.u.size(), initial.time, initial.steps, initial.rejected, &o,
                     &session, message, sizeof(message))) {
    set_error(error, message);
    return 1;
  }
  auto* g = new StaticAmrGpu;
  g->session = session;
  g->values = initial.u.size();
  *result = g;
  return 0;
}

int static_amr_gpu_advance(StaticAmrGpu* g, double tend, long maxsteps, StaticAmrState2D* state, std::string* error,
                           double wall_budget_seconds) {
  if (!g || !state) {
    set_error(error, "invalid AMR GPU advance");
    return 1;
  }
  amr_state_meta_t meta;
  std::memset(&meta, 0, sizeof(meta));
  char message[512] = {0};
  const int status = amr_gpu_advance(g->session, tend, maxsteps, wall_budget_seconds, &meta, message, sizeof(message));
  if (status == 1 && meta.steps == 0 && meta.time == 0 && std::strstr(message, "invalid")) {
    set_error(error, message);
    return 1;
  }
  state->time = meta.time;
  state->steps = meta.steps;
  state->rejected = meta.rejected;
  if (status == 1) set_error(error, message);
  return status;
}

int static_amr_gpu_download(StaticAmrGpu* g, StaticAmrState2D* state, std::string* error) {
  if (!g || !state) {
    set_error(error, "invalid AMR GPU download");
    return 1;
  }
  state->u.resize(g->values);
  amr_state_meta_t meta;
  char message[512] = {0};
  if (amr_gpu_download(g->session, state->u.data(), state->u.size(), &meta, message, sizeof(message))) {
    set_error(error, message);
    return 1;
  }
  state->time = meta.time;
  state->steps = meta.steps;
  state->rejected = meta.rejected;
  return 0;
}

AmrGpuStats static_amr_gpu_stats(const StaticAmrGpu* g) {
  AmrGpuStats out;
  if (!g) return out;
  amr_gpu_stats_t s;
  amr_gpu_stats(g->session, &s);
  std::memcpy(&out, &s, sizeof(out));
  return out;
}

void static_amr_gpu_destroy(StaticAmrGpu* g) {
  if (!g) return;
  amr_gpu_destroy(g->session);
  delete g;
}

}  // namespace cfd
