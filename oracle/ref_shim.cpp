// ref_shim.cpp -- TEST INFRASTRUCTURE, not product code.
//
// extern "C" wrapper around the reference's own CPU static-AMR core, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/.  Only tests/, the smoke check and
// the CPU-baseline leg of bench.py load it, as the checker and as the timed CPU baseline.
//
// It exposes: the reference mesh builder (static_amr2d_build, src/static_amr2d.cpp:229) with
// the viscous/SA table preparation (src/static_amr2d_viscous.cpp:123, src/static_amr2d_sa.cpp:5);
// the CPU integrator (static_amr2d_run, src/static_amr2d.cpp:384); the residual
// (static_amr2d_rhs, src/static_amr2d.cpp:369); and the driver's steady diagnostics
// (src/quick_airfoil.cpp:189-199).  With REF_WITH_CUDA it also wraps the reference CUDA
// session (src/static_amr2d_cuda.cu:274-366) so its kernels can be timed on the same GPU.
#include "static_amr2d.h"
#include "static_amr2d_binary.h"
#include "static_amr2d_gpu.h"
#include "amr_b200.h"

#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

using namespace cfd;

// The C ABI's record types must be layout-identical to the reference's records.
static_assert(sizeof(amr_cell_t) == sizeof(AmrCell2D), "cell layout");
static_assert(offsetof(amr_cell_t, volume) == offsetof(AmrCell2D, volume), "cell layout");
static_assert(offsetof(amr_cell_t, wall_count) == offsetof(AmrCell2D, wall_count), "cell layout");
static_assert(sizeof(amr_face_t) == sizeof(AmrFace2D), "face layout");
static_assert(offsetof(amr_face_t, length) == offsetof(AmrFace2D, length), "face layout");
static_assert(sizeof(amr_wall_t) == sizeof(WallFragment2D), "wall layout");
static_assert(offsetof(amr_wall_t, nx) == offsetof(WallFragment2D, nx), "wall layout");
static_assert(sizeof(amr_gradient_term_t) == sizeof(AmrGradientTerm2D), "term layout");
static_assert(sizeof(amr_wall_sample_t) == sizeof(AmrWallSample2D), "sample layout");
static_assert(sizeof(amr_face_geometry_t) == sizeof(AmrViscousFaceGeometry2D), "geometry layout");
static_assert(sizeof(amr_boundary_t) == sizeof(AmrBoundary2D), "boundary layout");
static_assert(offsetof(amr_boundary_t, wall_velocity) == offsetof(AmrBoundary2D, wall_velocity), "boundary layout");
static_assert(sizeof(amr_transport_t) == sizeof(AmrTransport2D), "transport layout");
static_assert(offsetof(amr_transport_t, wall_probe_min_h) == offsetof(AmrTransport2D, wall_probe_min_h), "transport layout");

struct ref_case {
  StaticAmrMesh2D mesh;
  Params2D params;
};

extern "C" {

typedef struct ref_mesh_options_t {
  int32_t nx, ny, levels, buffer;
  double xmin, xmax, ymin, ymax;
  uint64_t max_cells;
  int32_t agglomerate_small;
  int32_t n_boxes;
  const double* boxes; /* n_boxes x {x0, x1, y0, y1, level} */
} ref_mesh_options_t;

static void put_error(char* error, uint64_t size, const std::string& text) {
  if (!error || size == 0) return;
  std::strncpy(error, text.c_str(), size - 1);
  error[size - 1] = 0;
}

static Params2D to_params(const amr_params_t* p) {
  Params2D q = params2d_default();
  q.gamma = p->gamma;
  q.cfl = p->cfl;
  q.dt_fixed = p->dt_fixed;
  q.ausm_mco = p->ausm_mco;
  q.flux = p->flux;
  q.limiter = p->limiter;
  q.time_integrator = p->time_integrator;
  for (int i = 0; i < 4; ++i) q.bc[i] = p->bc[i];
  return q;
}

int ref_abi_version(void) { return AMR_B200_ABI_VERSION; }

ref_case* ref_case_build(const ref_mesh_options_t* o, const double* px, const double* py,
                         const int32_t* patches, int32_t npts, const amr_boundary_t* boundaries,
                         const amr_transport_t* transport, const amr_params_t* params,
                         char* error, uint64_t error_size) {
  auto* c = new ref_case;
  StaticAmrOptions2D options;
  options.nx = o->nx; options.ny = o->ny; options.levels = o->levels; options.buffer = o->buffer;
  options.xmin = o->xmin; options.xmax = o->xmax; options.ymin = o->ymin; options.ymax = o->ymax;
  options.max_cells = static_cast<size_t>(o->max_cells);
  options.agglomerate_small = o->agglomerate_small != 0;
  for (int b = 0; b < o->n_boxes; ++b) {
    const double* r = o->boxes + 5 * b;
    options.boxes.push_back({r[0], r[1], r[2], r[3], static_cast<int>(r[4])});
  }
  std::vector<double> x(px, px + npts), y(py, py + npts);
  std::vector<int> pt;
  if (patches) pt.assign(patches, patches + npts);
  std::string message;
  if (static_amr2d_build(options, x, y, pt, &c->mesh, &message)) {
    put_error(error, error_size, "build: " + message);
    delete c;
    return nullptr;
  }
  for (int side = 0; side < 4; ++side)
    std::memcpy(&c->mesh.boundaries[side], &boundaries[side], sizeof(AmrBoundary2D));
  std::memcpy(&c->mesh.transport, transport, sizeof(AmrTransport2D));
  c->params = to_params(params);
  if (static_amr2d_prepare_viscous(&c->mesh, c->params, &message)) {
    put_error(error, error_size, "viscous: " + message);
    delete c;
    return nullptr;
  }
  return c;
}

// Rebuilds a reference mesh object from a flat view (e.g. a mesh stored as a fixture).
ref_case* ref_case_from_view(const amr_mesh_view_t* v, const amr_params_t* params,
                             const ref_mesh_options_t* o) {
  auto* c = new ref_case;
  auto& m = c->mesh;
  m.options.nx = o->nx; m.options.ny = o->ny; m.options.levels = o->levels; m.options.buffer = o->buffer;
  m.options.xmin = o->xmin; m.options.xmax = o->xmax; m.options.ymin = o->ymin; m.options.ymax = o->ymax;
  m.options.max_cells = static_cast<size_t>(o->max_cells);
  m.options.agglomerate_small = v->agglomerate_small != 0;
  const size_t n = v->n_cells, nf = v->n_faces, nw = v->n_walls;
  m.cells.resize(n); std::memcpy(m.cells.data(), v->cells, n * sizeof(AmrCell2D));
  m.faces.resize(nf); std::memcpy(m.faces.data(), v->faces, nf * sizeof(AmrFace2D));
  m.walls.resize(nw); if (nw) std::memcpy(m.walls.data(), v->walls, nw * sizeof(WallFragment2D));
  m.face_offsets.assign(v->face_offsets, v->face_offsets + n + 1);
  m.cell_faces.assign(v->cell_faces, v->cell_faces + v->face_offsets[n]);
  m.group_offsets.assign(v->group_offsets, v->group_offsets + n + 1);
  m.group_members.assign(v->group_members, v->group_members + v->group_offsets[n]);
  m.member_offsets.assign(v->member_offsets, v->member_offsets + n + 1);
  m.member_groups.assign(v->member_groups, v->member_groups + v->member_offsets[n]);
  m.group_volume.assign(v->group_volume, v->group_volume + n);
  m.small_cells = v->small_cells;
  for (int side = 0; side < 4; ++side) std::memcpy(&m.boundaries[side], &v->boundaries[side], sizeof(AmrBoundary2D));
  std::memcpy(&m.transport, &v->transport, sizeof(AmrTransport2D));
  if (v->transport.model == AMR_B200_MODEL_LAMINAR) {
    auto& t = m.viscous;
    t.offsets.assign(v->visc_offsets, v->visc_offsets + n + 1);
    t.terms.resize(v->visc_offsets[n]);
    std::memcpy(t.terms.data(), v->visc_terms, t.terms.size() * sizeof(AmrGradientTerm2D));
    t.wall_samples.resize(nw); if (nw) std::memcpy(t.wall_samples.data(), v->wall_samples, nw * sizeof(AmrWallSample2D));
    t.face_samples.resize(nf); std::memcpy(t.face_samples.data(), v->face_samples, nf * sizeof(AmrWallSample2D));
    t.face_geometry.resize(nf); std::memcpy(t.face_geometry.data(), v->face_geometry, nf * sizeof(AmrViscousFaceGeometry2D));
    if (v->transport.sa_model) t.wall_distance.assign(v->wall_distance, v->wall_distance + n);
  }
  c->params = to_params(params);
  return c;
}

int ref_case_view(const ref_case* c, amr_mesh_view_t* v) {
  const auto& m = c->mesh;
  std::memset(v, 0, sizeof(*v));
  v->n_cells = m.cells.size(); v->n_faces = m.faces.size(); v->n_walls = m.walls.size();
  v->cells = reinterpret_cast<const amr_cell_t*>(m.cells.data());
  v->faces = reinterpret_cast<const amr_face_t*>(m.faces.data());
  v->walls = reinterpret_cast<const amr_wall_t*>(m.walls.data());
  static_assert(sizeof(size_t) == sizeof(uint64_t), "LP64");
  v->face_offsets = reinterpret_cast<const uint64_t*>(m.face_offsets.data());
  v->cell_faces = reinterpret_cast<const uint64_t*>(m.cell_faces.data());
  v->group_offsets = reinterpret_cast<const uint64_t*>(m.group_offsets.data());
  v->group_members = reinterpret_cast<const uint64_t*>(m.group_members.data());
  v->member_offsets = reinterpret_cast<const uint64_t*>(m.member_offsets.data());
  v->member_groups = reinterpret_cast<const uint64_t*>(m.member_groups.data());
  v->group_volume = m.group_volume.data();
  v->small_cells = m.small_cells;
  v->agglomerate_small = m.options.agglomerate_small ? 1 : 0;
  for (int side = 0; side < 4; ++side) std::memcpy(&v->boundaries[side], &m.boundaries[side], sizeof(AmrBoundary2D));
  std::memcpy(&v->transport, &m.transport, sizeof(AmrTransport2D));
  if (m.transport.model == AMR_MODEL_LAMINAR) {
    v->visc_offsets = reinterpret_cast<const uint64_t*>(m.viscous.offsets.data());
    v->visc_terms = reinterpret_cast<const amr_gradient_term_t*>(m.viscous.terms.data());
    v->wall_samples = reinterpret_cast<const amr_wall_sample_t*>(m.viscous.wall_samples.data());
    v->face_samples = reinterpret_cast<const amr_wall_sample_t*>(m.viscous.face_samples.data());
    v->face_geometry = reinterpret_cast<const amr_face_geometry_t*>(m.viscous.face_geometry.data());
    v->wall_distance = m.viscous.wall_distance.empty() ? nullptr : m.viscous.wall_distance.data();
  }
  return 0;
}

// counts: n, nf, nw, cell_faces, group_members, member_groups, terms, small_cells,
// coarse_fine_faces, background_leaves, split_leaves
int ref_case_counts(const ref_case* c, uint64_t* out) {
  const auto& m = c->mesh;
  out[0] = m.cells.size(); out[1] = m.faces.size(); out[2] = m.walls.size();
  out[3] = m.cell_faces.size(); out[4] = m.group_members.size(); out[5] = m.member_groups.size();
  out[6] = m.viscous.terms.size(); out[7] = m.small_cells; out[8] = m.coarse_fine_faces;
  out[9] = m.background_leaves; out[10] = m.split_leaves;
  return 0;
}

int ref_case_initialize(const ref_case* c, const double* w, double* u_out) {
  StaticAmrState2D s;
  if (static_amr2d_initialize(c->mesh, c->params, {w[0], w[1], w[2], w[3]}, &s)) return 1;
  std::memcpy(u_out, s.u.data(), s.u.size() * sizeof(double));
  return 0;
}

int ref_case_run(const ref_case* c, double* u, uint64_t count, double* time, int64_t* steps,
                 int64_t* rejected, double tend, int64_t maxsteps, char* error, uint64_t error_size) {
  StaticAmrState2D s;
  s.u.assign(u, u + count);
  s.time = *time; s.steps = *steps; s.rejected = *rejected;
  std::string message;
  const int status = static_amr2d_run(c->mesh, c->params, tend, maxsteps, &s, &message);
  std::memcpy(u, s.u.data(), count * sizeof(double));
  *time = s.time; *steps = s.steps; *rejected = s.rejected;
  if (status) put_error(error, error_size, message);
  return status;
}

// The reference's own result writers, for byte-for-byte comparison of the files.
int ref_case_write_mesh(const ref_case* c, const char* prefix, char* error, uint64_t error_size) {
  std::string message;
  const int st = static_amr_binary_mesh(c->mesh, c->params, prefix, &message);
  if (st) put_error(error, error_size, message);
  return st;
}

int ref_case_write_snapshot(const ref_case* c, const double* u, uint64_t count, double time, int64_t steps,
                            int64_t rejected, const char* prefix, const char* backend, char* error,
                            uint64_t error_size) {
  StaticAmrState2D s;
  s.u.assign(u, u + count);
  s.time = time; s.steps = steps; s.rejected = rejected;
  std::string message;
  const int st = static_amr_binary_snapshot(c->mesh, c->params, s, prefix, backend, &message);
  if (st) put_error(error, error_size, message);
  return st;
}

int ref_write_npy(const char* path, const double* values, uint64_t rows, uint64_t cols) {
  std::string message;
  return static_amr_write_npy(path, values, rows, cols, &message);
}

// Wall-clock seconds of ref_case_run, measured around the reference call alone.
double ref_case_run_timed(const ref_case* c, double* u, uint64_t count, double* time, int64_t* steps,
                          int64_t* rejected, double tend, int64_t maxsteps, int* status) {
  StaticAmrState2D s;
  s.u.assign(u, u + count);
  s.time = *time; s.steps = *steps; s.rejected = *rejected;
  std::string message;
  const auto t0 = std::chrono::steady_clock::now();
  *status = static_amr2d_run(c->mesh, c->params, tend, maxsteps, &s, &message);
  const auto t1 = std::chrono::steady_clock::now();
  std::memcpy(u, s.u.data(), count * sizeof(double));
  *time = s.time; *steps = s.steps; *rejected = s.rejected;
  return std::chrono::duration<double>(t1 - t0).count();
}

int ref_case_rhs(const ref_case* c, const double* u, double* r_out) {
  const size_t nv = c->mesh.transport.sa_model ? 5 : 4;
  std::vector<double> state(u, u + nv * c->mesh.cells.size()), r;
  if (static_amr2d_rhs(c->mesh, c->params, state, &r)) return 1;
  std::memcpy(r_out, r.data(), r.size() * sizeof(double));
  return 0;
}

int ref_case_redistribute(const ref_case* c, double* u) {
  const size_t nv = c->mesh.transport.sa_model ? 5 : 4;
  std::vector<double> state(u, u + nv * c->mesh.cells.size());
  if (static_amr2d_redistribute(c->mesh, &state)) return 1;
  std::memcpy(u, state.data(), state.size() * sizeof(double));
  return 0;
}

// Residual norms and loads exactly as the reference driver computes them
// (src/quick_airfoil.cpp:189-199): out[0..4] res, out[5..7] fx, fy, mz.
int ref_case_diagnostics(const ref_case* c, const double* u, const double* region, double mx,
                         double my, double* out) {
  const auto& mesh = c->mesh;
  const auto& p = c->params;
  const size_t n = mesh.cells.size();
  const int nv = mesh.transport.sa_model ? 5 : 4;
  std::vector<double> state(u, u + nv * n), rhs;
  if (static_amr2d_rhs(mesh, p, state, &rhs)) return 1;
  long double sum[5] = {}, volume = 0;
  for (size_t k = 0; k < n; ++k) {
    const auto& cell = mesh.cells[k];
    if (cell.cx < region[0] || cell.cx > region[1] || cell.cy < region[2] || cell.cy > region[3]) continue;
    volume += cell.volume;
    for (int v = 0; v < nv; ++v) sum[v] += cell.volume * std::fabs(rhs[v * n + k]);
  }
  for (int v = 0; v < 5; ++v) out[v] = v < nv && volume > 0 ? static_cast<double>(sum[v] / volume) : 0.0;
  if (mesh.transport.sa_model) out[4] /= mesh.transport.sa_nu_inf;
  AmrViscousFields2D visc;
  const bool viscous = mesh.transport.model == AMR_MODEL_LAMINAR;
  if (viscous && static_amr2d_viscous_diagnostics(mesh, p, state, &visc)) return 1;
  const size_t nw = mesh.walls.size();
  double fx = 0, fy = 0, mz = 0;
  for (size_t i = 0; i < nw; ++i) {
    const auto& w = mesh.walls[i];
    const size_t k = w.owner_cell;
    const double pressure = (p.gamma - 1) * (state[3 * n + k] - .5 * (state[n + k] * state[n + k] + state[2 * n + k] * state[2 * n + k]) / state[k]);
    const double a = pressure * w.nx * w.length - (viscous ? visc.wall_flux[nw + i] : 0.0);
    const double b = pressure * w.ny * w.length - (viscous ? visc.wall_flux[2 * nw + i] : 0.0);
    fx += a; fy += b;
    mz += ((w.x0 + w.x1) * .5 - mx) * b - ((w.y0 + w.y1) * .5 - my) * a;
  }
  out[5] = fx; out[6] = fy; out[7] = mz;
  return 0;
}

void ref_case_destroy(ref_case* c) { delete c; }

#ifdef REF_WITH_CUDA
struct ref_gpu {
  StaticAmrGpu* session = nullptr;
  StaticAmrState2D state;
};

void* ref_gpu_create(const ref_case* c, const double* u, int batch_trials, int graph, int fused,
                     int sa_fused, int event_timing, char* error, uint64_t error_size) {
  auto* g = new ref_gpu;
  const size_t nv = c->mesh.transport.sa_model ? 5 : 4;
  g->state.u.assign(u, u + nv * c->mesh.cells.size());
  AmrGpuOptions o;
  o.batch_trials = batch_trials; o.graph = graph != 0; o.fused = fused != 0;
  o.sa_fused = sa_fused != 0; o.event_timing = event_timing != 0;
  std::string message;
  if (static_amr_gpu_create(c->mesh, c->params, g->state, o, &g->session, &message)) {
    put_error(error, error_size, message);
    delete g;
    return nullptr;
  }
  return g;
}

int ref_gpu_advance(void* handle, double tend, int64_t maxsteps, double* time, int64_t* steps,
                    int64_t* rejected, char* error, uint64_t error_size) {
  auto* g = static_cast<ref_gpu*>(handle);
  std::string message;
  const int status = static_amr_gpu_advance(g->session, tend, maxsteps, &g->state, &message);
  *time = g->state.time; *steps = g->state.steps; *rejected = g->state.rejected;
  if (status) put_error(error, error_size, message);
  return status;
}

int ref_gpu_download(void* handle, double* u) {
  auto* g = static_cast<ref_gpu*>(handle);
  std::string message;
  if (static_amr_gpu_download(g->session, &g->state, &message)) return 1;
  std::memcpy(u, g->state.u.data(), g->state.u.size() * sizeof(double));
  return 0;
}

double ref_gpu_event_seconds(void* handle) {
  return static_amr_gpu_stats(static_cast<ref_gpu*>(handle)->session).advance_event_seconds;
}

uint64_t ref_gpu_graph_nodes(void* handle) {
  return static_amr_gpu_stats(static_cast<ref_gpu*>(handle)->session).graph_nodes_per_trial;
}

void ref_gpu_destroy(void* handle) {
  auto* g = static_cast<ref_gpu*>(handle);
  if (!g) return;
  static_amr_gpu_destroy(g->session);
  delete g;
}
#endif
}
