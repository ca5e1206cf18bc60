// amr_static.cu -- amr_euler_residual_static: the inviscid residual dU/dt without any device
// allocation.
//
// Who needs it: code that may not call cudaMalloc or cudaFree at the point where it wants a
// residual -- for example a host loop that runs inside another framework's memory pool or
// allocator (where a raw cudaMalloc would bypass the pool's accounting or be forbidden), a
// real-time or latency-critical path where an allocation would synchronise the device, or a
// plug-in that is handed device buffers but not allowed to own memory.  Such a caller passes
// its own device copies of the mesh records and the state; the scratch this computation needs
// (primitive variables and face fluxes) lives in one file-scope device array below.
//
// The arithmetic is the reference CPU residual for the inviscid model (src/static_amr2d.cpp:143-197
// in the reference): primitives, one flux per face (boundary ghost state, HLLC or AUSM+-up,
// times the open length), then the in-order signed gather of each cell's faces plus its wall
// pressure, R = -sum / V.  This unit is compiled like the FP64 engine (no contraction), so the
// result equals amr_gpu_residual's for the same state.
#include <cmath>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "../../include/amr_b200.h"
#include "amr_physics.cuh"

namespace {

using namespace amrb;

// Capacity of the static scratch: primitives of up to kMaxCells cells and fluxes of up to
// kMaxFaces faces, plus a status word.  4 * (16384 + 40960) doubles = 1.8 MB per device.
constexpr uint64_t kMaxCells = 16384;
constexpr uint64_t kMaxFaces = 40960;
constexpr uint64_t kScratchDoubles = 4 * (kMaxCells + kMaxFaces) + 2;

// Every GPU that loads this library holds this array until the process exits.  All calls on a
// device share it and it keeps the previous call's contents; calls whose kernels overlap on the
// GPU (different streams, or different host threads on one device) race on it.
static __device__ __align__(256) double g_residual_scratch[kScratchDoubles];

// Status bits the kernels raise: a nonphysical state or flux, and a mesh record whose indices
// point outside the arrays the caller passed (the access is skipped, nothing is read there).
constexpr int kBadState = 1;
constexpr int kBadMesh = 2;

struct StaticParams {
  double gamma, mco;
  int flux;
  int kind[4];
  Bnd<double> bnd[4];
};

__device__ __forceinline__ void flag_bad(int* status) { atomicOr(status, kBadState); }
__device__ __forceinline__ void flag_mesh(int* status) { atomicOr(status, kBadMesh); }

__global__ void static_primitive_kernel(const double* __restrict__ u, uint64_t n, double gamma, double* __restrict__ w,
                                        int* status) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double rho = u[k], mx = u[n + k], my = u[2 * n + k], energy = u[3 * n + k];
  const double vx = mx / rho, vy = my / rho, p = (gamma - 1) * (energy - 0.5 * (mx * vx + my * vy));
  if (!isfinite(rho) || !(rho > 0) || !isfinite(mx) || !isfinite(my) || !isfinite(energy) || !isfinite(p) || !(p > 0))
    flag_bad(status);
  w[k] = rho;
  w[n + k] = vx;
  w[2 * n + k] = vy;
  w[3 * n + k] = p;
}

__global__ void static_face_kernel(const amr_face_t* __restrict__ faces, uint64_t nf, uint64_t n, const double* __restrict__ w,
                                   StaticParams sp, double* __restrict__ flux, int* status) {
  const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (q >= nf) return;
  const amr_face_t f = faces[q];
  if (f.left >= (int64_t)n || f.right >= (int64_t)n || (f.left < 0 && f.right < 0) || f.boundary < -1 || f.boundary > 3 ||
      (f.boundary < 0 && (f.left < 0 || f.right < 0)) || (f.axis != 0 && f.axis != 1)) {
    flag_mesh(status);
    return;
  }
  const int inside = f.left >= 0 ? f.left : f.right;
  const int la = f.left >= 0 ? f.left : inside, rb = f.right >= 0 ? f.right : inside;
  double a[4], b[4];
  for (int v = 0; v < 4; ++v) {
    a[v] = w[v * n + la];
    b[v] = w[v * n + rb];
  }
  const int axis = f.axis;
  if (f.boundary >= 0) {
    const double wi[4] = {f.left < 0 ? b[0] : a[0], f.left < 0 ? b[1] : a[1], f.left < 0 ? b[2] : a[2], f.left < 0 ? b[3] : a[3]};
    double wo[4];
    if (!bc_state(sp.bnd[f.boundary], sp.kind[f.boundary], sp.gamma, f.boundary, wi, wo)) flag_bad(status);
    if (f.left < 0) { a[0] = wo[0]; a[1] = wo[1]; a[2] = wo[2]; a[3] = wo[3]; }
    else { b[0] = wo[0]; b[1] = wo[1]; b[2] = wo[2]; b[3] = wo[3]; }
  }
  const double an = axis ? a[2] : a[1], at = axis ? a[1] : a[2];
  const double bn = axis ? b[2] : b[1], bt = axis ? b[1] : b[2];
  double F[4];
  if (f.boundary >= 0 && sp.kind[f.boundary] == BC_NOSLIP) {
    F[0] = 0; F[1] = w[3 * n + inside]; F[2] = 0; F[3] = 0;
  } else if (sp.flux == AMR_B200_FLUX_HLLC) {
    flux_hllc(a[0], an, at, a[3], b[0], bn, bt, b[3], sp.gamma, F);
  } else {
    flux_ausmpup(a[0], an, at, a[3], b[0], bn, bt, b[3], sp.gamma, sp.mco, F);
  }
  for (int v = 0; v < 4; ++v)
    if (!isfinite(F[v])) flag_bad(status);
  flux[q] = F[0] * f.length;
  flux[(axis ? 2 : 1) * nf + q] = F[1] * f.length;
  flux[(axis ? 1 : 2) * nf + q] = F[2] * f.length;
  flux[3 * nf + q] = F[3] * f.length;
}

__global__ void static_gather_kernel(const amr_cell_t* __restrict__ cells, uint64_t n, const amr_face_t* __restrict__ faces,
                                     uint64_t nf, const amr_wall_t* __restrict__ walls, uint64_t nw,
                                     const uint64_t* __restrict__ offsets, const uint64_t* __restrict__ cell_faces,
                                     const double* __restrict__ w, const double* __restrict__ flux, double* __restrict__ r,
                                     int* status) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const amr_cell_t c = cells[k];
  // cell_faces holds offsets[n] entries, so every position below offsets[n] may be read
  const uint64_t begin = offsets[k], end = offsets[k + 1], total = offsets[n];
  if (begin > end || end > total || c.wall_begin > nw || c.wall_count > nw - c.wall_begin) {
    flag_mesh(status);
    return;
  }
  for (uint64_t pos = begin; pos < end; ++pos)
    if (cell_faces[pos] >= nf) {
      flag_mesh(status);
      return;
    }
  double sum[4] = {0, 0, 0, 0};
  for (uint64_t pos = begin; pos < end; ++pos) {
    const uint64_t face = cell_faces[pos];
    const double sign = faces[face].left == (int)k ? 1.0 : -1.0;
    for (int v = 0; v < 4; ++v) sum[v] += sign * flux[v * nf + face];
  }
  const double p = w[3 * n + k];
  for (uint64_t q = c.wall_begin; q < c.wall_begin + c.wall_count; ++q) {
    sum[1] += p * walls[q].nx * walls[q].length;
    sum[2] += p * walls[q].ny * walls[q].length;
  }
  for (int v = 0; v < 4; ++v) r[v * n + k] = -sum[v] / c.volume;
}

void put(char* buf, uint64_t size, const std::string& text) {
  if (!buf || size == 0) return;
  const size_t len = text.size() < size - 1 ? text.size() : size - 1;
  std::memcpy(buf, text.data(), len);
  buf[len] = 0;
}

bool check(cudaError_t st, char* error, uint64_t size, const char* what) {
  if (st == cudaSuccess) return true;
  put(error, size, std::string(what) + ": " + cudaGetErrorString(st));
  return false;
}

}  // namespace

extern "C" int amr_euler_residual_static(const amr_cell_t* cells, uint64_t n_cells, const amr_face_t* faces,
                                         uint64_t n_faces, const amr_wall_t* walls, uint64_t n_walls,
                                         const uint64_t* face_offsets, const uint64_t* cell_faces,
                                         const amr_boundary_t* boundaries, const amr_params_t* params, const double* u,
                                         double* r, void* stream, char* error, uint64_t error_size) {
  if (!cells || !faces || !face_offsets || !cell_faces || !boundaries || !params || !u || !r || (n_walls && !walls) ||
      n_cells == 0 || n_faces == 0) {
    put(error, error_size, "invalid static residual arguments");
    return 1;
  }
  if (n_cells > kMaxCells || n_faces > kMaxFaces) {
    put(error, error_size, "mesh exceeds the static scratch capacity (16384 cells, 40960 faces)");
    return 1;
  }
  const amr_params_t& p = *params;
  if (!std::isfinite(p.gamma) || !(p.gamma > 1) || !std::isfinite(p.ausm_mco) || p.ausm_mco <= 0 ||
      (p.flux != AMR_B200_FLUX_HLLC && p.flux != AMR_B200_FLUX_AUSMPUP)) {
    put(error, error_size, "invalid static residual parameters");
    return 1;
  }
  // The device address of the scratch array on the current device (the array's name in host code
  // is only a host-side handle).  It is looked up on every call rather than cached: the lookup is
  // cheap once the module is loaded, two host threads cannot race on a cache, and a device reset
  // (which reloads the module, possibly elsewhere) cannot leave a stale address behind.
  void* address = nullptr;
  if (!check(cudaGetSymbolAddress(&address, g_residual_scratch), error, error_size, "cudaGetSymbolAddress")) return 1;
  double* scratch = static_cast<double*>(address);
  double* w = scratch;                        // 4 * n_cells
  double* flux = scratch + 4 * kMaxCells;     // 4 * n_faces
  int* status = reinterpret_cast<int*>(scratch + 4 * (kMaxCells + kMaxFaces));
  StaticParams sp;
  std::memset(&sp, 0, sizeof(sp));
  sp.gamma = p.gamma;
  sp.mco = p.ausm_mco;
  sp.flux = p.flux;
  for (int side = 0; side < 4; ++side) {
    const amr_boundary_t& b = boundaries[side];
    sp.kind[side] = b.kind < 0 ? p.bc[side] : b.kind;
    Bnd<double>& d = sp.bnd[side];
    d.kind = sp.kind[side];
    for (int v = 0; v < 4; ++v) d.ref[v] = b.reference[v];
    d.total_pressure = b.total_pressure;
    d.total_temperature = b.total_temperature;
    d.gas_constant = b.gas_constant;
    d.dir[0] = b.direction[0];
    d.dir[1] = b.direction[1];
    d.outlet_pressure = b.outlet_pressure;
    d.wall_velocity[0] = b.wall_velocity[0];
    d.wall_velocity[1] = b.wall_velocity[1];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the status word must start at zero; primitives and fluxes are overwritten in full
  if (!check(cudaMemsetAsync(status, 0, sizeof(int), st), error, error_size, "status reset")) return 1;
  const int T = 128;
  static_primitive_kernel<<<(unsigned)((n_cells + T - 1) / T), T, 0, st>>>(u, n_cells, p.gamma, w, status);
  static_face_kernel<<<(unsigned)((n_faces + T - 1) / T), T, 0, st>>>(faces, n_faces, n_cells, w, sp, flux, status);
  static_gather_kernel<<<(unsigned)((n_cells + T - 1) / T), T, 0, st>>>(cells, n_cells, faces, n_faces, walls, n_walls,
                                                                        face_offsets, cell_faces, w, flux, r, status);
  if (!check(cudaGetLastError(), error, error_size, "static residual launch")) return 1;
  int host_status = 0;
  if (!check(cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, st), error, error_size,
             "status read-back") ||
      !check(cudaStreamSynchronize(st), error, error_size, "static residual sync"))
    return 1;
  if (host_status & kBadMesh) {
    put(error, error_size, "mesh record index out of range (face cell/boundary/axis, cell face range, face id or wall range)");
    return 1;
  }
  if (host_status) {
    put(error, error_size, "nonphysical state or nonfinite face flux");
    return 1;
  }
  return 0;
}
