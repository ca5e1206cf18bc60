// amr_engine.cuh -- the persistent trial kernel of the static-AMR explicit time step.
//
// Layout (device, one arena per batch; every index is int32 and global across cases):
//   cells   c_case, c_vol, c_area (CFL area), c_gvol (SRD group volume), c_flags (SRD-simple),
//           CSR offsets c_slot / c_wall / c_term (each case owns n+1 entries, so offset[k+1]
//           always closes cell k), c_wd (SA wall distance), state U[2][nv][ncap] (double
//           buffered: ctl.cur selects the accepted state), U2, R0, R.
//   slots   one per (cell, face) pair in the order of the reference's cell_faces CSR:
//           s_own, s_nb (-1 outside), s_meta (own-is-left | axis | boundary side | bc kind),
//           s_len, s_geo[6] (viscous face geometry dx,dy,ex,ey,distance + exterior sample
//           distance).  A face is evaluated once per side, so a cell's whole face sum lives in
//           one thread block and is formed in CSR order.
//   walls   per owner cell, CSR c_wall: normal, length, donor, donor distance, midpoint.
//   terms   per owner cell, CSR c_term: LSQ gradient weights (t_own, t_src, t_x, t_y).
//   SRD     only the non-trivial neighbourhoods: group members with their overlap counts and
//           group volumes, and the cells they touch with their group lists.
//   tiles   runs of whole cells of one case whose slots and terms fit one thread block.
//
// One trial (one attempt of one SSP-RK3 step of every live case) is the phase sequence
//   [G0] F0 DT+U1 [SRD] [G1] F1+U2 [SRD] [G2] F2+U3 [SRD] COMMIT
// separated by grid barriers: G = cell gradients/viscosity/SA source (laminar), F = face
// fluxes and in-order cell sums (residual, cell dt, stage update), SRD = state
// redistribution of the non-trivial neighbourhoods (one block per case), COMMIT = per-case
// accept/reject and the next trial's begin.  Per-case control (time, dt, retries, status)
// never leaves the device.
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "amr_physics.cuh"

namespace amrb {

enum { MODEL_EULER = 0, MODEL_LAMINAR = 1, MODEL_SA = 2 };
enum { FLUX_HLLC = 0, FLUX_AUSM = 1 };
enum { STAGE_BASE = 0, STAGE_1 = 1, STAGE_2 = 2, STAGE_DIAG = 3 };
enum { MODE_TRIALS = 0, MODE_RESIDUAL = 1 };
enum { STATUS_NONPHYSICAL_BASE = 2, STATUS_MAXSTEPS = 3, STATUS_DT_UNDERFLOW = 4, STATUS_REJECTIONS = 5,
       STATUS_BARRIER_TIMEOUT = 9 };
constexpr int MAX_BLOCK = 256;
constexpr unsigned long long DT_INF_BITS = 0x7FF0000000000000ull;

struct alignas(16) CaseCtl {
  double time, target, dt, dt_trial;
  long long steps, rejected, maxsteps;
  unsigned long long dtmin;  // bit pattern of the smallest cell dt of this trial (dt > 0)
  int bad, fatal, retrying, attempt, finished, active, cur, live;
};

template <class R> struct CaseCfg {
  double cfl, dt_fixed, viscous_cfl, sa_cfl;
  R gamma, mco;
  int kind[4];
  Bnd<R> bnd[4];
  Trn<R> trn;
  int agglomerated, has_srd;
  int srd_g0, srd_g1, srd_q0, srd_q1;  // SRD group / cell list ranges
  int srd_rate;                        // viscous dt limited through the SRD map of the rates
  int cell0, cell1;                    // the case's cell range
};

// A run of whole cells of one case: cells [c0, c1), their slots [s0, s1) and gradient terms [t0, t1).
struct Tile {
  int cs, c0, c1, leader, s0, s1, t0, t1;
};

// A block tile (tiled mode): cells [c0, c1) of case cs, their halo cells bt_halo[h0, h1) (face
// neighbours and wall donors outside the range), the face records bt_face[f0, f1) touching the
// cells, and the cells' wall fragments [w0, w1).
struct BTile {
  int cs, c0, c1, h0, h1, f0, f1, w0, w1;
};
#ifndef AMRB_BT_CELLS
#define AMRB_BT_CELLS 128
#endif
constexpr int BT_CELLS = AMRB_BT_CELLS;  // cells per block tile
constexpr int BT_DATA = 2 * BT_CELLS;    // tile + halo cells (packed records in shared memory)
constexpr int BT_FACES = 3 * BT_CELLS;   // face records per tile
constexpr int BT_WALLS = BT_CELLS;       // wall fragments per tile
constexpr int BT_THREADS = 2 * BT_CELLS;
constexpr int SLOT_WALL = 1 << 9;  // s_meta flag: the slot is a wall fragment of its owner cell
// A tile is processed by one warp: at most TILE_W slots and TILE_W gradient terms of whole cells,
// synchronised by __syncwarp only, so the warps of a block never wait for one another.
constexpr int TILE_W = 32;
constexpr int SM_COLS = 12;  // values per slot (shared-memory columns, face and wall records)
constexpr int CREC = 16;     // values in a packed cell record
// The split mode's global cell records.  FP32 viscous models store 12 values (48 bytes): state 0-4,
// gradient 5-8, SA phi gradient 9-10; the face kernel recomputes viscosity, eddy viscosity and the
// SA diffusion coefficient from the state (cell_transport), with the gradient kernel's expressions.
// FP64 keeps the full CREC layout (and the tiled mode's shared-memory records always do).
template <class R, int MODEL> struct CellRec {
  static constexpr bool compact = sizeof(R) == 4 && MODEL >= 1;
  static constexpr int stride = compact ? 12 : CREC;
};
constexpr unsigned FULL_MASK = 0xffffffffu;

struct GridBarrier {
  unsigned int count, gen;
  int timeout, pad;
  int live[4];
};

template <class R> struct Dev {
  CaseCtl* ctl;
  const CaseCfg<R>* cfg;
  const Tile* tiles;
  int n_tiles, n_cases;
  // cells
  const int* c_case;
  const double* c_vol;
  const double* c_area;
  const double* c_gvol;
  const unsigned char* c_flags;
  const int* c_slot;
  const int* c_wall;
  const int* c_term;
  const R* c_wd;
  // slots
  const int* s_own;
  const int* s_nb;
  const int* s_meta;
  const R* s_len;
  const R* s_geo;  // 6 per slot
  // walls
  const R* w_nx;
  const R* w_ny;
  const R* w_len;
  const R* w_dist;
  const int* w_donor;
  // terms
  const int* t_own;
  const int* t_src;
  const R* t_x;
  const R* t_y;
  // SRD
  const int* g_mem;     // group -> member offsets (global, n_groups+1 per case run closed)
  const int* g_cell;    // members (global cell)
  const double* g_cnt;  // overlap count of each member
  const double* g_vol;  // group volume
  const int* q_cell;    // non-trivial cells
  const int* q_grp;     // cell -> group-list offsets
  const int* q_list;    // group indices
  const double* q_cnt;  // overlap count of the cell
  double* qhat;         // 4 per group
  // state and scratch (stride ncap)
  R* U0;
  R* U1;
  R* U2;
  R* R0;
  R* Rr;
  // FP32 form: trailing words of the accepted state buffers U0 / U1 (null in FP64).  The value
  // of a variable is U + L; fluxes read U alone, the final stage of a step updates both.
  R* L0;
  R* L1;
  R* grad;
  R* mu;
  R* eddy;
  R* sgrad;
  R* sdiff;
  R* ssrc;
  R* srate;
  long long ncap;
  long long gcap;
  // split mode: one record per face and per wall, and the slot -> record map
  const int* f_case;
  const int* f_own;
  const int* f_nb;
  const int* f_meta;
  const R* f_len;
  const R* f_geo;   // 6 per face
  const int* w_owner;
  const int* s_item;
  R* fval;          // per face: 12 values, 8 in the compact FP32 viscous format (RecFormat)
  R* wval;          // per wall: the same
  R* fsa;           // compact FP32 SA format: the SA flux per face record (column 10)
  R* wsa;           // and per wall record
  R* crec;          // CREC per cell: packed state and gradient-phase fields (viscous models)
  // tiled mode
  const BTile* btiles;
  const int* bt_halo;   // global cell index per halo entry
  const int* bt_face;   // global face record index per tile face entry
  const int2* bt_floc;  // local (tile data) index of the face's own and other cell (-1 outside)
  const int* s_loc;     // per slot: 2 * tile face + (cell is the face's left), or the tile wall index
  const int* w_ldon;    // per wall: local data index of the donor cell
  double* ddt;      // 2 per cell: convective and viscous dt limits of the last residual pass
  int any_srd_rate; // some live case limits its viscous dt through the SRD map
  const double* w_xm;  // wall midpoints
  const double* w_ym;
  int n_faces, n_walls, n_cells;  // ends of the live face, wall and cell ranges (host copy)
  int cap_faces, cap_walls;       // record capacities
  const int* live_end;            // the same on the device: cells, faces, walls (read by the
                                  // graph-replayed kernels, so a graph outlives case changes)
  // Split mode in lanes: the split kernels of lane `lane` cover cells, faces and walls from
  // live_begin[0..2] to live_end[0..2] (null live_begin: from 0), and its per-case kernels only
  // the cases whose case_lane entry is `lane` (null case_lane: every case).
  const int* live_begin;
  const int* case_lane;
  int lane;
  GridBarrier* bar;
  unsigned long long barrier_cycles;
};

// ---- memory helpers -------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int* p) { return *(volatile const int*)p; }

// Start of every kernel of a launch chain (phase, split and tiled modes).  The chain is launched
// with programmatic stream serialization, so a kernel may be scheduled while its predecessor is
// still finishing: griddepcontrol.wait blocks until the predecessor has completed and its writes
// are visible, and no kernel touches memory before it.  launch_dependents then lets the next
// kernel be scheduled once every block of this one has started, so its blocks take SM slots
// during this kernel's tail instead of after it.  Launched without the attribute, both are no-ops.
__device__ __forceinline__ void chain_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Grid-wide barrier for a cooperative launch.  The wait is bounded: after
// barrier_cycles SM clocks the block records a timeout, every later barrier returns false at
// once, and the kernel unwinds.  Returns true when all blocks arrived.
__device__ __forceinline__ bool grid_barrier(GridBarrier* b, unsigned long long limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = !ld_volatile(&b->timeout);
    if (ok) {
      const unsigned int g = ld_acquire(&b->gen);
      __threadfence();
      const unsigned int arrived = atomicAdd(&b->count, 1u);
      if (arrived == gridDim.x - 1) {
        atomicExch(&b->count, 0u);
        __threadfence();
        st_release(&b->gen, g + 1);
      } else {
        const long long t0 = clock64();
        unsigned int spins = 0;
        while (ld_acquire(&b->gen) == g) {
          if (++spins > 32) __nanosleep(64);
          if ((spins & 255) == 0) {
            if (ld_volatile(&b->timeout)) { ok = 0; break; }
            if ((unsigned long long)(clock64() - t0) > limit) {
              atomicExch(&b->timeout, 1);
              ok = 0;
              break;
            }
          }
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <class R> struct Prim { R rho, u, v, p; };

// U: the state's SoA array, or any object whose [i] yields entry i of such an array (FusedIn).
template <class R, class In> __device__ __forceinline__ Prim<R> prim(const In& U, long long n, int k, R g) {
  Prim<R> w;
  const R rho = U[k], mx = U[n + k], my = U[2 * n + k], e = U[3 * n + k];
  w.rho = rho;
  w.u = mx / rho;
  w.v = my / rho;
  w.p = (g - R(1)) * (e - R(0.5) * (mx * w.u + my * w.v));
  return w;
}

template <class R, class In> __device__ __forceinline__ bool prim_ok(const In& U, long long n, int k, const Prim<R>& w) {
  const R mx = U[n + k], my = U[2 * n + k], e = U[3 * n + k];
  return isfinite(w.rho) && w.rho > R(0) && isfinite(mx) && isfinite(my) && isfinite(e) && isfinite(w.p) && w.p > R(0);
}

// The first stage's input U1 = U + dt R0, formed where it is read (split mode, viscous models
// without SRD, whose first update has no other effect), with the expression the first-update
// kernel stores.
template <class R> struct FusedIn {
  const R* U;
  const R* R0;
  R dt;
  __device__ __forceinline__ R operator[](long long i) const { return U[i] + dt * R0[i]; }
};

__device__ __forceinline__ void atomic_min_dt(unsigned long long* slot, double v) {
  atomicMin(slot, (unsigned long long)__double_as_longlong(v));
}

// Zero-degree SRD of a cell whose only neighbourhood is itself: Q = (V u / 1) / Vhat, u = Q / 1,
// evaluated exactly as the full redistribution does for such a cell.
template <class R> __device__ __forceinline__ R srd_self(R u, double vol, double gvol) {
  double s = 0.0;
  s += vol * (double)u / 1.0;
  const double q = s / gvol;
  double t = 0.0;
  t += q;
  return (R)(t / 1.0);
}

template <class R> struct Smem {
  R* a;  // [12][blockDim]
};

// A face or wall record is 12 values: flux 0-3, viscous flux 4-7, convective and viscous
// spectral radius 8-9, SA flux 10 and SA spectral term 11.  Records are 16-byte aligned and
// moved as 16-byte vectors; a model moves only the groups it uses (columns 8-11 ride with
// the spectral radius, which only the base stage needs beyond column 10).
template <class R> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int n = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int n = 2; };

template <class R> __device__ __forceinline__ void store_group(R* dst, const R* src) {
  using V = typename Vec16<R>::T;
  constexpr int m = Vec16<R>::n;
#pragma unroll
  for (int j = 0; j < 4 / m; ++j) {
    V v;
    R* e = reinterpret_cast<R*>(&v);
#pragma unroll
    for (int i = 0; i < m; ++i) e[i] = src[j * m + i];
    reinterpret_cast<V*>(dst)[j] = v;
  }
}

template <class R> __device__ __forceinline__ void load_group(const R* src, R* dst) {
  using V = typename Vec16<R>::T;
  constexpr int m = Vec16<R>::n;
#pragma unroll
  for (int j = 0; j < 4 / m; ++j) {
    const V v = __ldg(reinterpret_cast<const V*>(src) + j);
    const R* e = reinterpret_cast<const R*>(&v);
#pragma unroll
    for (int i = 0; i < m; ++i) dst[j * m + i] = e[i];
  }
}


// A packed cell record (split mode, viscous models) is CREC values, 16-byte aligned, moved as
// 16-byte vectors: state 0-4, gradient 5-8, mu 9, eddy 10, SA phi gradient 11-12, SA diffusion
// 13.  A laminar model uses the first twelve only.
template <class R, int MODEL> __device__ __forceinline__ void store_cell_record(R* dst, const R* c) {
  store_group(dst, c);
  store_group(dst + 4, c + 4);
  store_group(dst + 8, c + 8);
  if (MODEL == MODEL_SA) store_group(dst + 12, c + 12);
}

template <class R, int MODEL> __device__ __forceinline__ void load_cell_record(const R* src, R* c) {
  load_group(src, c);
  load_group(src + 4, c + 4);
  load_group(src + 8, c + 8);
  if (MODEL == MODEL_SA) {
    load_group(src + 12, c + 12);
  } else {
    c[4] = c[11] = c[12] = c[13] = R(0);
  }
}


// ------------------------------------------------------------------------------------------
// G phase: velocity gradients, viscosity, eddy viscosity, SA gradients and point model of
// every cell of a tile (reference src/static_amr2d_viscous.cpp:166-174, src/static_amr2d_sa.cpp:74-80).
// ------------------------------------------------------------------------------------------
// Cell part of the G phase from the summed LSQ contributions gr (velocity) and sg (SA phi and
// density): viscosity, eddy viscosity, SA point model and source.  Returns false on failure.
// With soa the per-cell fields go to the SoA scratch arrays; with rec (split mode) they also go
// to the cell's packed record: state 0-4, gradient 5-8, mu 9, eddy 10, SA phi gradient 11-12,
// SA diffusion 13.
template <class R, int MODEL, class In>
__device__ __forceinline__ bool grad_finish(const Dev<R>& d, const CaseCfg<R>& cf, int k, const In& Uin, const R* gr,
                                            const R* sg, bool soa = true, R* rec = nullptr, bool src_out = true,
                                            bool compact_rec = false) {
  const long long n = d.ncap;
  const Prim<R> w = prim(Uin, n, k, cf.gamma);
  const R mu = dyn_visc(cf.trn, w.p / (w.rho * cf.trn.gas_constant));
  bool bad = !(mu > R(0)) || !isfinite(mu);
  if (soa) {
    for (int v = 0; v < 4; ++v) d.grad[v * n + k] = gr[v];
    d.mu[k] = mu;
  }
  R eddy = 0, sdiff = 0;
  if (MODEL == MODEL_SA) {
    const R ph = Uin[4 * n + k] / w.rho;
    if (!isfinite(ph)) bad = true;
    eddy = w.rho * sa_eddy(ph, mu / w.rho);
    const SaPoint<R> pt = sa_neg(ph, mu / w.rho, d.c_wd[k], R(fabs(gr[2] - gr[1])));
    const R src = sa_corrected_source(pt, w.rho, sg[0], sg[1], sg[2], sg[3]);
    if (soa) {
      d.sgrad[k] = sg[0];
      d.sgrad[n + k] = sg[1];
      d.sdiff[k] = pt.diffusion;
    }
    sdiff = pt.diffusion;
    if (src_out) {
      d.ssrc[k] = src;
      d.srate[k] = pt.source_rate;
    }
    if (!(pt.diffusion > R(0)) || !isfinite(src) || !isfinite(pt.source_rate)) bad = true;
  }
  if (soa) d.eddy[k] = eddy;
  if (rec) {
    R c[CREC];
    for (int v = 0; v < 4; ++v) c[v] = Uin[v * n + k];
    c[4] = MODEL == MODEL_SA ? Uin[4 * n + k] : R(0);
    for (int v = 0; v < 4; ++v) c[5 + v] = gr[v];
    c[9] = mu;
    c[10] = eddy;
    c[11] = MODEL == MODEL_SA ? sg[0] : R(0);
    c[12] = MODEL == MODEL_SA ? sg[1] : R(0);
    c[13] = sdiff;
    c[14] = c[15] = R(0);
    if (compact_rec) {  // CellRec compact layout: the SA phi gradient follows the gradient
      c[9] = c[11];
      c[10] = c[12];
      c[11] = R(0);
      store_group(rec, c);
      store_group(rec + 4, c + 4);
      store_group(rec + 8, c + 8);
    } else {
      store_cell_record<R, MODEL>(rec, c);
    }
  }
  return !bad;
}

// LSQ contribution of one gradient term of cell k (reference src/static_amr2d_viscous.cpp:170-173,
// src/static_amr2d_sa.cpp:75-76): c[0..3] velocity, c[4..7] SA phi and density.
template <class R, int MODEL, class In>
__device__ __forceinline__ void term_values(const Dev<R>& d, const CaseCfg<R>& cf, int q, int k, const In& Uin, R* c) {
  const long long n = d.ncap;
  const int src = __ldg(d.t_src + q);
  const R x = __ldg(d.t_x + q), y = __ldg(d.t_y + q);
  const R rk = Uin[k], uk = Uin[n + k] / rk, vk = Uin[2 * n + k] / rk;
  R uu = 0, vv = 0;
  if (src >= 0) {
    const R rs = Uin[src];
    uu = Uin[n + src] / rs;
    vv = Uin[2 * n + src] / rs;
  } else if (src <= -2) {
    uu = cf.bnd[-2 - src].wall_velocity[0];
    vv = cf.bnd[-2 - src].wall_velocity[1];
  }
  const R du = uu - uk, dv = vv - vk;
  c[0] = x * du;
  c[1] = y * du;
  c[2] = x * dv;
  c[3] = y * dv;
  if (MODEL == MODEL_SA) {
    const R phk = Uin[4 * n + k] / rk;
    const R ph = src >= 0 ? Uin[4 * n + src] / Uin[src] : R(0);
    const R rho = src >= 0 ? Uin[src] : rk;
    c[4] = x * (ph - phk);
    c[5] = y * (ph - phk);
    c[6] = x * (rho - rk);
    c[7] = y * (rho - rk);
  }
}

template <class R, int MODEL>
__device__ void phase_gradients(const Dev<R>& d, const Tile& t, const R* Uin, R* sm) {
  const int B = TILE_W, i = threadIdx.x & 31;
  const CaseCfg<R>& cf = d.cfg[t.cs];
  const int t0 = t.t0, t1 = t.t1;
  if (i < t1 - t0) {
    const int q = t0 + i;
    R c[8];
    term_values<R, MODEL>(d, cf, q, __ldg(d.t_own + q), Uin, c);
    for (int v = 0; v < (MODEL == MODEL_SA ? 8 : 4); ++v) sm[v * B + i] = c[v];
  }
  __syncwarp();
  if (i < t.c1 - t.c0) {
    const int k = t.c0 + i;
    R gr[4] = {0, 0, 0, 0}, sg[4] = {0, 0, 0, 0};
    const int a = d.c_term[k] - t0, b = d.c_term[k + 1] - t0;
    for (int q = a; q < b; ++q)
      for (int v = 0; v < 4; ++v) gr[v] += sm[v * B + q];
    if (MODEL == MODEL_SA)
      for (int q = a; q < b; ++q)
        for (int v = 0; v < 4; ++v) sg[v] += sm[(4 + v) * B + q];
    if (!grad_finish<R, MODEL>(d, cf, k, Uin, gr, sg)) atomicOr(&d.ctl[t.cs].bad, 1);
  }
  __syncwarp();
}

// ------------------------------------------------------------------------------------------
// F phase: per-slot face fluxes (convective + viscous + SA), then per-cell in-order sums,
// residual, cell dt and the stage update (reference src/static_amr2d.cpp:163-204,
// src/static_amr2d_viscous.cpp:177-206, src/static_amr2d_sa.cpp:81-96, 395-426).
// ------------------------------------------------------------------------------------------
// Fluxes of one face seen from cell k (nb: the other cell, -1 outside).  Writes the 12 values
// dst[c*stride]: conserved flux (4), viscous flux (4), speed*length, viscous spectral coefficient,
// SA flux, SA spectral coefficient.  With signed = true the flux columns carry the orientation
// sign of cell k (slot form); otherwise they are in face orientation (item form).
// Everything one face's fluxes read: both cells' states and (viscous) gradients, viscosities,
// SA fields and the fixed face geometry.  k is the slot's cell, m the other cell (k itself
// outside the domain).
template <class R> struct FaceIn {
  R uk[5], um[5], gk[4], gm[4], geo[6];
  R mk, mm, ek, em, sgk[2], sgm[2], sdk, sdm;
};

// Loads a FaceIn from the SoA state and scratch arrays.  Every load is issued up front and
// unconditionally (an exterior face reads its own cell twice), so the whole neighbourhood
// arrives in one memory round trip.
template <class R, int MODEL>
__device__ __forceinline__ void face_in_soa(const Dev<R>& d, const R* gp, int k, int m, const R* Uin, FaceIn<R>& f) {
  const long long n = d.ncap;
  for (int v = 0; v < 4; ++v) { f.uk[v] = Uin[v * n + k]; f.um[v] = Uin[v * n + m]; }
  if (MODEL == MODEL_SA) { f.uk[4] = Uin[4 * n + k]; f.um[4] = Uin[4 * n + m]; }
  f.mk = f.mm = f.ek = f.em = f.sdk = f.sdm = 0;
  f.sgk[0] = f.sgk[1] = f.sgm[0] = f.sgm[1] = 0;
  if (MODEL >= MODEL_LAMINAR) {
    for (int v = 0; v < 4; ++v) { f.gk[v] = d.grad[v * n + k]; f.gm[v] = d.grad[v * n + m]; }
    f.mk = d.mu[k]; f.mm = d.mu[m]; f.ek = d.eddy[k]; f.em = d.eddy[m];
    for (int v = 0; v < 6; ++v) f.geo[v] = __ldg(gp + v);
    if (MODEL == MODEL_SA) {
      f.sgk[0] = d.sgrad[k]; f.sgk[1] = d.sgrad[n + k]; f.sgm[0] = d.sgrad[m]; f.sgm[1] = d.sgrad[n + m];
      f.sdk = d.sdiff[k]; f.sdm = d.sdiff[m];
    }
  }
}

// Loads a FaceIn from the two cells' packed records (split mode, viscous models).
// Viscosity, eddy viscosity and SA diffusion coefficient of a cell from its conserved state c[0..4],
// by grad_finish's expressions (prim, dyn_visc, sa_eddy and sa_neg's diffusion), for the compact
// records that do not store them.
template <class R, int MODEL>
__device__ __forceinline__ void cell_transport(const CaseCfg<R>& cf, const R* c, R& mu, R& eddy, R& sdiff) {
  const R rho = c[0], u = c[1] / rho, v = c[2] / rho;
  const R p = (cf.gamma - R(1)) * (c[3] - R(0.5) * (c[1] * u + c[2] * v));
  mu = dyn_visc(cf.trn, p / (rho * cf.trn.gas_constant));
  eddy = R(0);
  sdiff = R(0);
  if (MODEL == MODEL_SA) {
    const R ph = c[4] / rho, nu = mu / rho;
    eddy = rho * sa_eddy(ph, nu);
    if (ph < R(0)) {
      const R chi = ph / nu, cube = chi * chi * chi;
      const R fn = (R(16) + cube) / (R(16) - cube);
      sdiff = (nu + ph * fn) / R(AMRB_SIG);
    } else {
      sdiff = (nu + ph) / R(AMRB_SIG);
    }
  }
}

template <class R, int MODEL>
__device__ __forceinline__ void load_cell_rec(const Dev<R>& d, const CaseCfg<R>& cf, int k, R* a) {
  constexpr int S = CellRec<R, MODEL>::stride;
  if (CellRec<R, MODEL>::compact) {
    const R* src = d.crec + S * (long long)k;
    R c[12];
    load_group(src, c);
    load_group(src + 4, c + 4);
    load_group(src + 8, c + 8);
    for (int v = 0; v < 9; ++v) a[v] = c[v];
    a[11] = c[9];
    a[12] = c[10];
    if (MODEL != MODEL_SA) a[4] = a[11] = a[12] = R(0);
    cell_transport<R, MODEL>(cf, a, a[9], a[10], a[13]);
  } else {
    load_cell_record<R, MODEL>(d.crec + S * (long long)k, a);
  }
}

template <class R, int MODEL>
__device__ __forceinline__ void face_in_records(const Dev<R>& d, const CaseCfg<R>& cf, const R* gp, int k, int m,
                                                FaceIn<R>& f) {
  R a[CREC], b[CREC];
  load_cell_rec<R, MODEL>(d, cf, k, a);
  load_cell_rec<R, MODEL>(d, cf, m, b);
  for (int v = 0; v < 5; ++v) { f.uk[v] = a[v]; f.um[v] = b[v]; }
  for (int v = 0; v < 4; ++v) { f.gk[v] = a[5 + v]; f.gm[v] = b[5 + v]; }
  f.mk = a[9]; f.mm = b[9]; f.ek = a[10]; f.em = b[10];
  f.sgk[0] = a[11]; f.sgk[1] = a[12]; f.sgm[0] = b[11]; f.sgm[1] = b[12];
  f.sdk = a[13]; f.sdm = b[13];
  for (int v = 0; v < 6; ++v) f.geo[v] = __ldg(gp + v);
}

template <class R, int MODEL, int FLUX>
__device__ __forceinline__ void face_fluxes(const CaseCfg<R>& cf, const FaceIn<R>& f, R len, int nb, int meta, bool base,
                                            R* dst, int stride, bool signed_out, bool& bad);

template <class R, int MODEL, int FLUX>
__device__ __forceinline__ void slot_face(const Dev<R>& d, const CaseCfg<R>& cf, const R* gp, R len, int k, int nb,
                                          int meta, const R* Uin, bool base, R* dst, int stride, bool signed_out,
                                          bool& bad) {
  FaceIn<R> f;
  face_in_soa<R, MODEL>(d, gp, k, nb >= 0 ? nb : k, Uin, f);
  face_fluxes<R, MODEL, FLUX>(cf, f, len, nb, meta, base, dst, stride, signed_out, bad);
}

template <class R, int MODEL, int FLUX>
__device__ __forceinline__ void face_fluxes(const CaseCfg<R>& cf, const FaceIn<R>& f, R len, int nb, int meta, bool base,
                                            R* dst, int stride, bool signed_out, bool& bad) {
  const R g = cf.gamma;
  const bool own_left = meta & 1;
  const int axis = (meta >> 1) & 1, side = ((meta >> 2) & 7) - 1, kind = (meta >> 5) & 15;
  const R* uk = f.uk;
  const R* um = f.um;
  const R* gk = f.gk;
  const R* gm = f.gm;
  const R* geo = f.geo;
  const R mk = f.mk, mm = f.mm, ek = f.ek, em = f.em, sdk = f.sdk, sdm = f.sdm;
  const R* sgk = f.sgk;
  const R* sgm = f.sgm;
  Prim<R> wk, wn;
  wk.rho = uk[0]; wk.u = uk[1] / uk[0]; wk.v = uk[2] / uk[0]; wk.p = (g - R(1)) * (uk[3] - R(0.5) * (uk[1] * wk.u + uk[2] * wk.v));
  wn.rho = um[0]; wn.u = um[1] / um[0]; wn.v = um[2] / um[0]; wn.p = (g - R(1)) * (um[3] - R(0.5) * (um[1] * wn.u + um[2] * wn.v));
  // face-oriented states: a = left, b = right
  R a[4], b[4];
  a[0] = own_left ? wk.rho : wn.rho; a[1] = own_left ? wk.u : wn.u; a[2] = own_left ? wk.v : wn.v; a[3] = own_left ? wk.p : wn.p;
  b[0] = own_left ? wn.rho : wk.rho; b[1] = own_left ? wn.u : wk.u; b[2] = own_left ? wn.v : wk.v; b[3] = own_left ? wn.p : wk.p;
  if (side >= 0) {
    const R wi[4] = {wk.rho, wk.u, wk.v, wk.p};
    R wo[4];
    if (!bc_state(cf.bnd[side], kind, g, side, wi, wo)) bad = true;
    if (own_left) { b[0] = wo[0]; b[1] = wo[1]; b[2] = wo[2]; b[3] = wo[3]; }
    else { a[0] = wo[0]; a[1] = wo[1]; a[2] = wo[2]; a[3] = wo[3]; }
  }
  const R an = axis ? a[2] : a[1], at = axis ? a[1] : a[2];
  const R bn = axis ? b[2] : b[1], bt = axis ? b[1] : b[2];
  R F[4];
  if (side >= 0 && kind == BC_NOSLIP) {
    F[0] = 0; F[1] = wk.p; F[2] = 0; F[3] = 0;
  } else if (FLUX == FLUX_HLLC) {
    flux_hllc(a[0], an, at, a[3], b[0], bn, bt, b[3], g, F);
  } else {
    flux_ausmpup(a[0], an, at, a[3], b[0], bn, bt, b[3], g, cf.mco, F);
  }
  // conserved components: normal momentum goes to 1+axis, tangential to 2-axis
  const R f0 = F[0] * len, fn = F[1] * len, ft = F[2] * len, f3 = F[3] * len;
  for (int v = 0; v < 4; ++v) if (!isfinite(F[v])) bad = true;
  const R sg = signed_out ? (own_left ? R(1) : R(-1)) : R(1);
  dst[0 * stride] = sg * f0;
  dst[1 * stride] = sg * (axis ? ft : fn);
  dst[2 * stride] = sg * (axis ? fn : ft);
  dst[3 * stride] = sg * f3;
  if (base) {
    const R speed = rmax(R(fabs(an)) + sqrt(g * a[3] / a[0]), R(fabs(bn)) + sqrt(g * b[3] / b[0]));
    dst[8 * stride] = speed * len;
  }
  if (MODEL >= MODEL_LAMINAR) {
    R gv[4], mu, uf, vf, nu, distance;
    if (side < 0) {
      Prim<R> wl, wr;
      wl.rho = own_left ? wk.rho : wn.rho; wl.u = own_left ? wk.u : wn.u; wl.v = own_left ? wk.v : wn.v; wl.p = own_left ? wk.p : wn.p;
      wr.rho = own_left ? wn.rho : wk.rho; wr.u = own_left ? wn.u : wk.u; wr.v = own_left ? wn.v : wk.v; wr.p = own_left ? wn.p : wk.p;
      R gl[4], grr[4];
      for (int v = 0; v < 4; ++v) { gl[v] = own_left ? gk[v] : gm[v]; grr[v] = own_left ? gm[v] : gk[v]; }
      correct_gradient(gl, grr, geo[0], geo[1], wr.u - wl.u, wr.v - wl.v, gv);
      uf = R(.5) * (wl.u + wr.u) + gv[0] * geo[2] + gv[1] * geo[3];
      vf = R(.5) * (wl.v + wr.v) + gv[2] * geo[2] + gv[3] * geo[3];
      const R el = own_left ? ek : em, er = own_left ? em : ek, ml = own_left ? mk : mm, mr = own_left ? mm : mk;
      const R temp = R(.5) * (wl.p / wl.rho + wr.p / wr.rho) / cf.trn.gas_constant;
      mu = dyn_visc(cf.trn, temp) + R(.5) * (el + er);
      nu = rmax((ml + el) / wl.rho, (mr + er) / wr.rho);
      distance = geo[4];
    } else {
      for (int v = 0; v < 4; ++v) gv[v] = gk[v];
      mu = mk + ek;
      uf = wk.u;
      vf = wk.v;
      nu = mu / wk.rho;
      distance = geo[5];
      const R sside = side % 2 ? R(1) : R(-1);
      if (kind == BC_NOSLIP) {
        mu = mk;
        uf = cf.bnd[side].wall_velocity[0];
        vf = cf.bnd[side].wall_velocity[1];
        wall_gradient(axis == 0 ? sside : R(0), axis == 1 ? sside : R(0), distance, uf - wk.u, vf - wk.v, gv);
      } else if (kind == BC_REFLECT) {
        gv[1] = 0; gv[2] = 0;
        if (axis == 0) uf = 0; else vf = 0;
      } else {
        if (axis) { gv[1] = 0; gv[3] = 0; } else { gv[0] = 0; gv[2] = 0; }
        uf += gv[0] * geo[2] + gv[1] * geo[3];
        vf += gv[2] * geo[2] + gv[3] * geo[3];
      }
    }
    R fv[4];
    visc_flux(mu, gv, axis == 0 ? R(1) : R(0), axis == 1 ? R(1) : R(0), uf, vf, fv);
    for (int v = 0; v < 4; ++v) {
      if (!isfinite(fv[v])) bad = true;
      dst[(4 + v) * stride] = sg * (fv[v] * len);
    }
    if (base) dst[9 * stride] = R(4.0 / 3) * nu / distance * len;
    if (MODEL == MODEL_SA) {
      const R mass = f0 - fv[0] * len;
      const R phk = uk[4] / wk.rho;
      const R phn = nb >= 0 ? um[4] / wn.rho : cf.trn.sa_nu_inf;
      const R left = own_left ? phk : phn, right = own_left ? phn : phk;
      R diff = 0, fc = 0;
      if (side < 0) {
        const R gl[4] = {own_left ? sgk[0] : sgm[0], own_left ? sgk[1] : sgm[1], 0, 0};
        const R grr[4] = {own_left ? sgm[0] : sgk[0], own_left ? sgm[1] : sgk[1], 0, 0};
        R gs[4];
        correct_gradient(gl, grr, geo[0], geo[1], right - left, R(0), gs);
        const R rl = own_left ? wk.rho : wn.rho, rr = own_left ? wn.rho : wk.rho;
        const R dl = own_left ? sdk : sdm, dr = own_left ? sdm : sdk;
        const R coefficient = R(.5) * (rl * dl + rr * dr);
        diff = coefficient * (axis ? gs[1] : gs[0]) * len;
        fc = coefficient / geo[4] * len;
      } else {
        const bool inflow = own_left ? mass < R(0) : mass > R(0);
        const R sside = side % 2 ? R(1) : R(-1);
        if (kind == BC_NOSLIP || inflow) {
          const R wall = kind == BC_NOSLIP ? R(0) : cf.trn.sa_nu_inf;
          const R coefficient = kind == BC_NOSLIP ? mk / R(AMRB_SIG) : wk.rho * sdk;
          diff = sside * coefficient * (wall - phk) / distance * len;
          fc = coefficient / distance * len;
        }
      }
      dst[10 * stride] = sg * (mass * (mass >= R(0) ? left : right) - diff);
      if (base) dst[11 * stride] = fc;
    }
  }
}

// A wall fragment of cell k: pressure force (reference src/static_amr2d.cpp:193-195), viscous wall
// flux from the visible donor (src/static_amr2d_viscous.cpp:192-196) and the SA wall flux
// (src/static_amr2d_sa.cpp:91), with their spectral-radius contributions.
// The owner's conserved state and viscosity, the donor's state and viscosity.
template <class R> struct WallIn {
  R uk[4], ud[5], mk, md;
};

template <class R, int MODEL>
__device__ __forceinline__ void wall_fluxes(const CaseCfg<R>& cf, const WallIn<R>& w, R nx, R ny, R wdist, R wl, bool base,
                                            R* dst, int stride, bool& bad);

template <class R, int MODEL>
__device__ __forceinline__ void slot_wall(const Dev<R>& d, const CaseCfg<R>& cf, R nx, R ny, R wdist, R wl, int k, int dn,
                                          const R* Uin, bool base, R* dst, int stride, bool& bad) {
  const long long n = d.ncap;
  WallIn<R> w;
  for (int v = 0; v < 4; ++v) w.uk[v] = Uin[v * n + k];
  w.mk = w.md = 0;
  w.ud[0] = w.ud[1] = w.ud[2] = w.ud[3] = w.ud[4] = 0;
  if (MODEL >= MODEL_LAMINAR) {
    for (int v = 0; v < 3; ++v) w.ud[v] = Uin[v * n + dn];
    if (MODEL == MODEL_SA) w.ud[4] = Uin[4 * n + dn];
    w.md = d.mu[dn];
    w.mk = d.mu[k];
  }
  wall_fluxes<R, MODEL>(cf, w, nx, ny, wdist, wl, base, dst, stride, bad);
}

// The same from the packed cell records of the owner and the donor (split mode, viscous models).
template <class R, int MODEL>
__device__ __forceinline__ void slot_wall_records(const Dev<R>& d, const CaseCfg<R>& cf, R nx, R ny, R wdist, R wl, int k,
                                                  int dn, bool base, R* dst, int stride, bool& bad) {
  R a[CREC], b[CREC];
  load_cell_rec<R, MODEL>(d, cf, k, a);
  load_cell_rec<R, MODEL>(d, cf, dn, b);
  WallIn<R> w;
  for (int v = 0; v < 4; ++v) w.uk[v] = a[v];
  for (int v = 0; v < 5; ++v) w.ud[v] = b[v];
  w.mk = a[9];
  w.md = b[9];
  wall_fluxes<R, MODEL>(cf, w, nx, ny, wdist, wl, base, dst, stride, bad);
}

template <class R, int MODEL>
__device__ __forceinline__ void wall_fluxes(const CaseCfg<R>& cf, const WallIn<R>& w, R nx, R ny, R wdist, R wl, bool base,
                                            R* dst, int stride, bool& bad) {
  const R g = cf.gamma;
  Prim<R> wk;
  wk.rho = w.uk[0];
  wk.u = w.uk[1] / w.uk[0];
  wk.v = w.uk[2] / w.uk[0];
  wk.p = (g - R(1)) * (w.uk[3] - R(0.5) * (w.uk[1] * wk.u + w.uk[2] * wk.v));
  dst[0 * stride] = 0;
  dst[1 * stride] = wk.p * nx * wl;
  dst[2 * stride] = wk.p * ny * wl;
  dst[3 * stride] = 0;
  if (base) dst[8 * stride] = sqrt(g * wk.p / wk.rho) * wl;
  if (MODEL >= MODEL_LAMINAR) {
    const R rd = w.ud[0], ud = w.ud[1] / rd, vd = w.ud[2] / rd;
    const R md = w.md;
    R gw[4], fw[4];
    wall_gradient(nx, ny, wdist, -ud, -vd, gw);
    visc_flux(md, gw, nx, ny, R(0), R(0), fw);
    for (int v = 0; v < 4; ++v) {
      if (!isfinite(fw[v])) bad = true;
      dst[(4 + v) * stride] = fw[v] * wl;
    }
    if (base) dst[9 * stride] = R(4.0 / 3) * rmax(md / rd, w.mk / wk.rho) / wdist * wl;
    if (MODEL == MODEL_SA) {
      const R swc = md / R(AMRB_SIG) / wdist * wl;
      dst[10 * stride] = -swc * (w.ud[4] / rd);
      if (base) dst[11 * stride] = swc;
    }
  }
}

// Correctly rounded sums that the compiler neither contracts nor reorders, and Knuth's TwoSum:
// s + e == a + b exactly, s the rounded sum.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
template <class R> __device__ __forceinline__ void two_sum(R a, R b, R& s, R& e) {
  s = add_rn(a, b);
  const R bv = sub_rn(s, a);
  e = add_rn(sub_rn(a, sub_rn(s, bv)), sub_rn(b, bv));
}

// The 12 values of one slot, returned by value so that they stay in registers.
template <class R> struct Cols {
  R v[SM_COLS];
};

// A slot getter whose face columns 0-3 are already net fluxes (convective minus viscous) and whose
// walls yield only viscous columns 0 and 3 beside momentum columns 1-2 declares net_cols = true;
// the cell then keeps one running sum per variable instead of separate viscous sums.
template <class G, class = void> struct NetCols : std::false_type {};
#ifndef AMRB_GATHER_UNROLL
#define AMRB_GATHER_UNROLL 2
#endif
template <class G> struct NetCols<G, std::void_t<decltype(G::net_cols)>> : std::bool_constant<G::net_cols> {};

// Per-cell end of the F phase: in-order sums of the cell's slot values (faces [a, e) in CSR order,
// then walls [e, b)), residual, cell dt (base stage) and the stage update.  get(q, col) yields
// the 12 values of slot q with the flux columns signed for cell k.  Returns the cell dt.
template <class R, int MODEL, class In, bool NET = false>
__device__ __forceinline__ double finish_tail(const Dev<R>& d, const CaseCfg<R>& cf, int cs, int k, int stage,
                                              const In& Uin, R* Ub, R* Un, const R* sum, const R* vs, R spectral, R vspec,
                                              R snet, R sspec, bool& bad);

template <class R, int MODEL, class Get, class In>
__device__ __forceinline__ double finish_cell(const Dev<R>& d, const CaseCfg<R>& cf, int cs, int k, int stage, int a,
                                              int e, int b, const Get& get, const In& Uin, R* Ub, R* Un, bool& bad) {
  const bool base = stage == STAGE_BASE;
  const bool spec = base || stage == STAGE_DIAG;  // spectral sums wanted (dt, or the export's dt limits)
  R sum[4] = {0, 0, 0, 0}, vs[4] = {0, 0, 0, 0}, spectral = 0, vspec = 0, snet = 0, sspec = 0;
  const auto slot = [&](int q) {
    const bool wall = q >= e;
    const Cols<R> cc = get(q, wall);
    const R* col = cc.v;
    if (NetCols<Get>::value) {
      if (!wall) {
        for (int v = 0; v < 4; ++v) sum[v] += col[v];
      } else {
        sum[0] -= col[4];
        sum[1] += col[1];
        sum[2] += col[2];
        sum[3] -= col[7];
      }
    } else if (!wall) {
      for (int v = 0; v < 4; ++v) sum[v] += col[v];
    } else {
      sum[1] += col[1];
      sum[2] += col[2];
    }
    if (spec) spectral += col[8];
    if (MODEL >= MODEL_LAMINAR) {
      if (!NetCols<Get>::value)
        for (int v = 0; v < 4; ++v) vs[v] += col[4 + v];
      if (spec) vspec += col[9];
    }
    if (MODEL == MODEL_SA) {
      if (!wall) snet += col[10]; else snet -= col[10];
      if (spec) sspec += col[11];
    }
  };
  if constexpr (NetCols<Get>::value) {
    // stored records: two slots' id and record loads in flight together
    constexpr int kUnroll = AMRB_GATHER_UNROLL;
#pragma unroll kUnroll
    for (int q = a; q < b; ++q) slot(q);
  } else {
    for (int q = a; q < b; ++q) slot(q);
  }
  return finish_tail<R, MODEL, In, NetCols<Get>::value>(d, cf, cs, k, stage, Uin, Ub, Un, sum, vs, spectral, vspec, snet,
                                                        sspec, bad);
}

// The end of a cell's F phase after its in-order slot sums: residual, cell dt (base stage) and
// the stage update, or the residual and dt limits of the diagnostics pass.  Returns the cell dt.
template <class R, int MODEL, class In, bool NET>
__device__ __forceinline__ double finish_tail(const Dev<R>& d, const CaseCfg<R>& cf, int cs, int k, int stage,
                                              const In& Uin, R* Ub, R* Un, const R* sum, const R* vs, R spectral, R vspec,
                                              R snet, R sspec, bool& bad) {
  const long long n = d.ncap;
  const R g = cf.gamma;
  const bool base = stage == STAGE_BASE;
  double cell_dt = __longlong_as_double(0x7FF0000000000000ll);
  const double V = d.c_vol[k];
  const Prim<R> wk = prim(Uin, n, k, g);
  if (!prim_ok(Uin, n, k, wk)) bad = true;
  R res[5];
  if constexpr (sizeof(R) == 4) {
    // FP32 form: the residual in FP32 arithmetic, one reciprocal of the volume per cell (the FP64
    // divisions by V cost more than the rest of the cell's sums); dt stays FP64 below
    const R inv = R(1) / (R)V;
    for (int v = 0; v < 4; ++v) res[v] = -sum[v] * inv;
    if (MODEL >= MODEL_LAMINAR) {
      if (!NET)
        for (int v = 0; v < 4; ++v) res[v] += vs[v] * inv;
      if (MODEL == MODEL_SA) {
        res[4] = -snet * inv + d.ssrc[k];
        if (!isfinite(res[4])) bad = true;
      }
    }
  } else {
    for (int v = 0; v < 4; ++v) res[v] = (R)(-sum[v] / V);
    if (MODEL >= MODEL_LAMINAR) {
      for (int v = 0; v < 4; ++v) res[v] += (R)(vs[v] / V);
      if (MODEL == MODEL_SA) {
        res[4] = (R)(-snet / V) + d.ssrc[k];
        if (!isfinite(res[4])) bad = true;
      }
    }
  }
  const int nv = MODEL == MODEL_SA ? 5 : 4;
  if (base) {
    double vdt = __longlong_as_double(0x7FF0000000000000ll), sdt = vdt;
    if constexpr (sizeof(R) == 4) {
      // FP32 form: the cell's limits are quotients of FP32 sums, formed in FP32 and widened; the
      // per-case minimum, dt and time stay FP64
      if (spectral > R(0)) cell_dt = (double)((R)(cf.cfl * d.c_area[k]) / spectral);
      if (MODEL >= MODEL_LAMINAR && vspec > R(0)) vdt = (double)((R)(cf.viscous_cfl * V) / vspec);
      if (MODEL == MODEL_SA) {
        const R rate = R(2) * sspec / (wk.rho * (R)V) + d.srate[k];
        if (rate > R(0)) sdt = (double)((R)cf.sa_cfl / rate);
      }
    } else {
      if (spectral > R(0)) cell_dt = cf.cfl * d.c_area[k] / (double)spectral;
      if (MODEL >= MODEL_LAMINAR && vspec > R(0)) vdt = cf.viscous_cfl * V / (double)vspec;
      if (MODEL == MODEL_SA) {
        const double rate = 2 * (double)sspec / ((double)wk.rho * V) + (double)d.srate[k];
        if (rate > 0) sdt = cf.sa_cfl / rate;
      }
    }
    if (MODEL >= MODEL_LAMINAR) {
      if (cf.srd_rate) {
        d.ddt[n + k] = vdt;  // mapped through the SRD neighbourhoods before it joins the minimum
        cell_dt = rmin(cell_dt, sdt);
      } else {
        cell_dt = rmin(cell_dt, rmin(vdt, sdt));
      }
    }
    for (int v = 0; v < nv; ++v) d.R0[v * n + k] = res[v];
  } else if (stage == STAGE_DIAG) {
    for (int v = 0; v < nv; ++v) d.R0[v * n + k] = res[v];
    // convective and viscous dt limits of the cell, for the export (reference
    // src/static_amr2d_viscous.cpp:151-153 and :131)
    const double inf = __longlong_as_double(0x7FF0000000000000ll);
    d.ddt[k] = spectral > R(0) ? cf.cfl * d.c_area[k] / (double)spectral : inf;
    d.ddt[n + k] = MODEL >= MODEL_LAMINAR && vspec > R(0) ? cf.viscous_cfl * V / (double)vspec : inf;
  } else {
    const R dt = (R)d.ctl[cs].dt_trial;
    const bool simple = cf.has_srd && (d.c_flags[k] & 1);
    const bool check = stage == STAGE_2 && (!cf.has_srd || simple);
    R out[5];
    bool two_word = false;
    if constexpr (sizeof(R) == 4) {
      two_word = d.L0 != nullptr;
    }
    if (two_word) {
      // FP32 form: the accepted state is a two-word FP32 value (U leading, L trailing).  The
      // final stage U+ = U/3 + 2/3 (U2 + dt R2) is formed as U + 2/3 (D2 + dt R2), with
      // D2 = U2 - U = (dt R0 + dt R1) / 4, and added to U + L with an error-free FP32 sum
      // (Knuth's TwoSum), so increments below half an ulp of U accumulate in L instead of being
      // rounded away; with only a leading word a case stalls short of its steady state once dt R
      // falls below that size.  Stage 1 stores U2 for the fluxes and, in the trailing words of the
      // next state buffer (which the final stage rewrites), the unrounded increment D2.  Cases with
      // SRD redistribute the stage states afterwards and keep L = 0.
      const R* Lb = Ub == d.U0 ? d.L0 : d.L1;
      R* Ln = Un == d.U0 ? d.L0 : d.L1;
      for (int v = 0; v < nv; ++v) {
        const R ub = Ub[v * n + k];
        if (stage == STAGE_1) {
          out[v] = R(0.75) * ub + R(0.25) * (Uin[v * n + k] + dt * res[v]);
          if (!cf.has_srd) Ln[v * n + k] = R(0.25) * (dt * d.R0[v * n + k] + dt * res[v]);
        } else if (cf.has_srd) {
          out[v] = ub / R(3) + R(2.0 / 3) * (Uin[v * n + k] + dt * res[v]);
          Ln[v * n + k] = R(0);
        } else {
          const R inc = R(2.0 / 3) * (Ln[v * n + k] + dt * res[v]);
          two_sum(ub, add_rn(inc, Lb[v * n + k]), out[v], Ln[v * n + k]);
        }
      }
    }
    if (!two_word) {
      for (int v = 0; v < nv; ++v) {
        if (stage == STAGE_1)
          out[v] = R(0.75) * Ub[v * n + k] + R(0.25) * (Uin[v * n + k] + dt * res[v]);
        else
          out[v] = Ub[v * n + k] / R(3) + R(2.0 / 3) * (Uin[v * n + k] + dt * res[v]);
      }
    }
    if (simple)
      for (int v = 0; v < 4; ++v) out[v] = srd_self(out[v], V, d.c_gvol[k]);
    R* dst = stage == STAGE_1 ? d.U2 : Un;
    for (int v = 0; v < nv; ++v) dst[v * n + k] = out[v];
    if (check) {
      const R rho = out[0], mx = out[1], my = out[2], e = out[3];
      const R vx = mx / rho, vy = my / rho, p = (g - R(1)) * (e - R(0.5) * (mx * vx + my * vy));
      if (!isfinite(rho) || !(rho > R(0)) || !isfinite(mx) || !isfinite(my) || !isfinite(e) || !isfinite(p) || !(p > R(0)))
        bad = true;
      if (MODEL == MODEL_SA && !isfinite(out[4])) bad = true;
    }
  }
  return cell_dt;
}

template <class R> struct SmemSlots {
  const R* sm;
  __device__ __forceinline__ Cols<R> operator()(int q, bool) const {
    Cols<R> o;
    for (int c = 0; c < SM_COLS; ++c) o.v[c] = sm[c * TILE_W + q];
    return o;
  }
};

template <class R, int MODEL, int FLUX>
__device__ void phase_flux(const Dev<R>& d, const Tile& t, int stage, const R* Uin, R* Ub, R* Un, R* sm,
                           bool* warp_bad, double* warp_dt) {
  const int B = TILE_W, i = threadIdx.x & 31;
  const CaseCfg<R>& cf = d.cfg[t.cs];
  const int s0 = t.s0, s1 = t.s1;
  const bool base = stage == STAGE_BASE;
  const bool spec = base || stage == STAGE_DIAG;
  bool bad = false;
  if (i < s1 - s0) {
    const int s = s0 + i;
    const int k = __ldg(d.s_own + s), nb = __ldg(d.s_nb + s), meta = __ldg(d.s_meta + s);
    const R* gp = d.s_geo + 6 * (long long)s;
    const R len = __ldg(d.s_len + s);
    if (meta & SLOT_WALL)
      slot_wall<R, MODEL>(d, cf, __ldg(gp + 0), __ldg(gp + 1), __ldg(gp + 2), len, k, nb, Uin, spec, sm + i, B, bad);
    else
      slot_face<R, MODEL, FLUX>(d, cf, gp, len, k, nb, meta, Uin, spec, sm + i, B, true, bad);
  }
  __syncwarp();
  double cell_dt = __longlong_as_double(0x7FF0000000000000ll);
  if (i < t.c1 - t.c0) {
    const int k = t.c0 + i;
    const int a = d.c_slot[k] - s0, b = d.c_slot[k + 1] - s0;
    const int e = b - (d.c_wall[k + 1] - d.c_wall[k]);
    cell_dt = finish_cell<R, MODEL>(d, cf, t.cs, k, stage, a, e, b, SmemSlots<R>{sm}, Uin, Ub, Un, bad);
  }
  *warp_bad = __any_sync(FULL_MASK, bad);
  if (base)  // warp minimum of the cell dt (exact; order-free)
    for (int o = 16; o > 0; o >>= 1) cell_dt = rmin(cell_dt, __shfl_xor_sync(FULL_MASK, cell_dt, o));
  *warp_dt = cell_dt;
  __syncwarp();  // the warp's shared memory is reused by its next tile
}

// Per-case step size of the current trial (reference src/static_amr2d.cpp:395-411 and the
// device control of src/static_amr2d_cuda.cu:170-187).  Returns false when the case cannot
// proceed; *fatal receives the status to record.
__device__ __forceinline__ bool choose_dt(const CaseCtl& c, double dt_fixed, double* dt_out, int* fatal) {
  *fatal = 0;
  if (c.bad) { *fatal = STATUS_NONPHYSICAL_BASE; return false; }
  double dt;
  if (c.retrying) {
    dt = c.dt;
  } else {
    dt = dt_fixed > 0 ? dt_fixed : __longlong_as_double((long long)c.dtmin);
    const double remaining = c.target - c.time;
    dt = rmin(dt, remaining);
    const double tol = 32 * DBL_EPSILON * rmax(rmax(fabs(c.target), fabs(c.time)), dt);
    if (remaining - dt <= tol) dt = remaining;
  }
  if (!isfinite(dt) || !(dt > 0) || c.time + dt == c.time) { *fatal = STATUS_DT_UNDERFLOW; return false; }
  *dt_out = dt;
  return true;
}

// DT+U1 phase: U1 = U + dt R0 for the cells of a tile.
template <class R, int MODEL>
__device__ void phase_first_update(const Dev<R>& d, const Tile& t, const R* Ub, R* Un) {
  const long long n = d.ncap;
  const CaseCfg<R>& cf = d.cfg[t.cs];
  const CaseCtl& c = d.ctl[t.cs];
  double dt;
  int fatal;
  const bool ok = choose_dt(c, cf.dt_fixed, &dt, &fatal);
  const int lane = threadIdx.x & 31;
  if (lane == 0 && t.leader) {
    if (ok) {
      d.ctl[t.cs].dt_trial = dt;
      if (!c.retrying) d.ctl[t.cs].attempt = 0;
    } else {
      d.ctl[t.cs].fatal = fatal;
    }
  }
  if (!ok) return;
  const int nv = MODEL == MODEL_SA ? 5 : 4;
  const R dtr = (R)dt;
  for (int j = lane; j < t.c1 - t.c0; j += 32) {
    const int k = t.c0 + j;
    const bool simple = cf.has_srd && (d.c_flags[k] & 1);
    for (int v = 0; v < nv; ++v) {
      R u = Ub[v * n + k] + dtr * d.R0[v * n + k];
      if (simple && v < 4) u = srd_self(u, d.c_vol[k], d.c_gvol[k]);
      Un[v * n + k] = u;
    }
  }
}

// SRD of the non-trivial neighbourhoods of one case (reference src/static_amr2d.cpp:208-226):
// Qhat_g = sum_k V_k u_k / N_k / Vhat_g, then u_k = sum_g Qhat_g / N_k.
template <class R, int MODEL>
__device__ void phase_srd(const Dev<R>& d, int cs, R* u, bool check) {
  const long long n = d.ncap, gc = d.gcap;
  const CaseCfg<R>& cf = d.cfg[cs];
  // one pass over the members with the four sums side by side: each member's loads are issued
  // together, and each sum still adds its terms in member order
  for (int gi = cf.srd_g0 + threadIdx.x; gi < cf.srd_g1; gi += blockDim.x) {
    const int m0 = d.g_mem[gi], m1 = d.g_mem[gi + 1];
    double sum[4] = {0, 0, 0, 0};
    for (int q = m0; q < m1; ++q) {
      const int k = d.g_cell[q];
      const double vol = d.c_vol[k], cnt = d.g_cnt[q];
      const double uk[4] = {(double)u[k], (double)u[n + k], (double)u[2 * n + k], (double)u[3 * n + k]};
      for (int v = 0; v < 4; ++v) sum[v] += vol * uk[v] / cnt;
    }
    const double gv = d.g_vol[gi];
    for (int v = 0; v < 4; ++v) d.qhat[v * gc + gi] = sum[v] / gv;
  }
  __syncthreads();
  bool bad = false;
  const R g = cf.gamma;
  for (int qi = cf.srd_q0 + threadIdx.x; qi < cf.srd_q1; qi += blockDim.x) {
    const int k = d.q_cell[qi], a = d.q_grp[qi], b = d.q_grp[qi + 1];
    double sum[4] = {0, 0, 0, 0};
    for (int q = a; q < b; ++q) {
      const int gq = d.q_list[q];
      for (int v = 0; v < 4; ++v) sum[v] += d.qhat[v * gc + gq];
    }
    const double cnt = d.q_cnt[qi];
    R out[4];
    for (int v = 0; v < 4; ++v) {
      out[v] = (R)(sum[v] / cnt);
      u[v * n + k] = out[v];
    }
    if (check) {
      const R rho = out[0], mx = out[1], my = out[2], e = out[3];
      const R vx = mx / rho, vy = my / rho, p = (g - R(1)) * (e - R(0.5) * (mx * vx + my * vy));
      if (!isfinite(rho) || !(rho > R(0)) || !isfinite(mx) || !isfinite(my) || !isfinite(e) || !isfinite(p) || !(p > R(0)))
        bad = true;
      if (MODEL == MODEL_SA && !isfinite(u[4 * n + k])) bad = true;
    }
  }
  if (bad) atomicOr(&d.ctl[cs].bad, 1);
  __syncthreads();
}

// SRD-rate viscous stabilization of one case (reference src/static_amr2d_viscous.cpp:123-134):
// the viscous rates r_k = viscous_cfl / dt_k go through the same redistribution map as the state,
// R_g = sum_k V_k r_k / N_k / Vhat_g, then r'_k = sum_g R_g / N_k, and dt'_k = viscous_cfl / r'_k.
// With store the mapped dt'_k replace dt_k in ddt (export); otherwise they join the case's dt
// minimum.  One block per case; the non-trivial groups use the SRD lists, every other cell the
// exact one-member form of the same sums.
template <class R, int MODEL>
__device__ void srd_rate_case(const Dev<R>& d, int cs, bool store) {
  const long long n = d.ncap;
  const CaseCfg<R>& cf = d.cfg[cs];
  const double vcfl = cf.viscous_cfl, inf = __longlong_as_double(0x7FF0000000000000ll);
  for (int gi = cf.srd_g0 + threadIdx.x; gi < cf.srd_g1; gi += blockDim.x) {
    double sum = 0;
    for (int q = d.g_mem[gi]; q < d.g_mem[gi + 1]; ++q) {
      const int k = d.g_cell[q];
      sum += d.c_vol[k] * (vcfl / d.ddt[n + k]) / d.g_cnt[q];
    }
    d.qhat[gi] = sum / d.g_vol[gi];
  }
  __syncthreads();
  double best = inf;
  for (int qi = cf.srd_q0 + threadIdx.x; qi < cf.srd_q1; qi += blockDim.x) {
    double sum = 0;
    for (int q = d.q_grp[qi]; q < d.q_grp[qi + 1]; ++q) sum += d.qhat[d.q_list[q]];
    const double rate = sum / d.q_cnt[qi];
    const double dt = rate > 0 ? vcfl / rate : inf;
    if (store) d.ddt[n + d.q_cell[qi]] = dt;
    best = rmin(best, dt);
  }
  for (int k = cf.cell0 + threadIdx.x; k < cf.cell1; k += blockDim.x) {
    if (!(d.c_flags[k] & 1)) continue;  // non-trivial: done above
    double s = 0.0;
    s += d.c_vol[k] * (vcfl / d.ddt[n + k]) / 1.0;
    double t = 0.0;
    t += s / d.c_gvol[k];
    const double rate = t / 1.0;
    const double dt = rate > 0 ? vcfl / rate : inf;
    if (store) d.ddt[n + k] = dt;
    best = rmin(best, dt);
  }
  if (!store && best < inf) atomic_min_dt(&d.ctl[cs].dtmin, best);
  __syncthreads();
}

// Case begin logic (reference src/static_amr2d_cuda.cu:54-59).
__device__ __forceinline__ void case_begin(CaseCtl& c) {
  c.active = 0;
  if (!c.live || c.fatal || c.finished) return;
  if (c.time >= c.target) { c.finished = 1; return; }
  if (c.steps >= c.maxsteps) { c.fatal = STATUS_MAXSTEPS; return; }
  c.bad = 0;
  c.active = 1;
  c.dtmin = DT_INF_BITS;
}

// Accept or reject the trial (reference src/static_amr2d.cpp:426-427, src/static_amr2d_cuda.cu:212-216).
__device__ __forceinline__ void case_commit(CaseCtl& c) {
  if (!c.active || c.fatal) return;
  if (c.bad) {
    ++c.rejected;
    ++c.attempt;
    c.retrying = 1;
    c.dt = c.dt_trial * 0.5;
    if (c.attempt >= 21) c.fatal = STATUS_REJECTIONS;
  } else {
    const double remaining = c.target - c.time;
    c.time = c.dt_trial == remaining ? c.target : c.time + c.dt_trial;
    ++c.steps;
    c.retrying = 0;
    c.attempt = 0;
    c.finished = c.time >= c.target;
    c.cur ^= 1;
  }
}

template <class R> __device__ __forceinline__ R* state_buf(const Dev<R>& d, int which) { return which ? d.U1 : d.U0; }

// ------------------------------------------------------------------------------------------
// The persistent kernel.  MODE_TRIALS runs up to `trials` trials; MODE_RESIDUAL evaluates
// the residual of every live case's accepted state into R0 (no update).  Tiles are processed
// one per warp; a warp's skip decision is taken by lane 0 from the control word and broadcast,
// so every lane of a warp follows the same path through __syncwarp().
// ------------------------------------------------------------------------------------------
enum { SKIP_LIVE = 0, SKIP_ACTIVE = 1, SKIP_STAGE = 2 };

__device__ __forceinline__ bool skip_case(const CaseCtl& c, int rule) {
  if (rule == SKIP_LIVE) return !c.live;
  if (rule == SKIP_ACTIVE) return !c.active;
  return !c.active || c.fatal || c.bad;
}

struct TileView {
  Tile t;
  int cur;
  bool skip;
};

__device__ __forceinline__ TileView read_tile(const Tile* tiles, const CaseCtl* ctl, int ti, int rule) {
  TileView v;
  v.t = tiles[ti];
  int skip = 0, cur = 0;
  if ((threadIdx.x & 31) == 0) {
    const CaseCtl& c = ctl[v.t.cs];
    skip = skip_case(c, rule);
    cur = c.cur;
  }
  v.skip = __shfl_sync(FULL_MASK, skip, 0) != 0;
  v.cur = __shfl_sync(FULL_MASK, cur, 0);
  return v;
}

// Block-level variant for the per-case SRD phase.
__device__ __forceinline__ bool read_case_skip(const CaseCtl* ctl, int cs, int rule, bool extra, int* cur) {
  __shared__ int s[2];
  if (threadIdx.x == 0) {
    s[0] = skip_case(ctl[cs], rule) || extra;
    s[1] = ctl[cs].cur;
  }
  __syncthreads();
  const bool skip = s[0];
  *cur = s[1];
  __syncthreads();
  return skip;
}

template <class R> __device__ __forceinline__ const R* stage_input(const Dev<R>& d, int stage, int cur) {
  if (stage == STAGE_BASE || stage == STAGE_DIAG) return state_buf(d, cur);
  return stage == STAGE_1 ? state_buf(d, cur ^ 1) : d.U2;
}

// One phase over all tiles, one tile per warp.
template <class R, int MODEL, int FLUX, bool GRAD>
__device__ __forceinline__ void tile_sweep(const Dev<R>& d, int stage, R* sm_block) {
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  R* sm = sm_block + warp * (SM_COLS * TILE_W);
  const int rule = stage == STAGE_DIAG ? SKIP_LIVE : (stage == STAGE_BASE ? SKIP_ACTIVE : SKIP_STAGE);
  for (int ti = blockIdx.x * wpb + warp; ti < d.n_tiles; ti += gridDim.x * wpb) {
    const TileView v = read_tile(d.tiles, d.ctl, ti, rule);
    if (v.skip) continue;
    if (GRAD) {
      phase_gradients<R, MODEL>(d, v.t, stage_input(d, stage, v.cur), sm);
    } else {
      bool wbad;
      double wdt;
      phase_flux<R, MODEL, FLUX>(d, v.t, stage, stage_input(d, stage, v.cur), state_buf(d, v.cur),
                                 state_buf(d, v.cur ^ 1), sm, &wbad, &wdt);
      if (lane == 0 && stage != STAGE_DIAG) {
        if (wbad) atomicOr(&d.ctl[v.t.cs].bad, 1);
        if (stage == STAGE_BASE) atomic_min_dt(&d.ctl[v.t.cs].dtmin, wdt);
      }
    }
  }
}

template <class R, int MODEL, int FLUX, bool SRD>
__global__ void __launch_bounds__(MAX_BLOCK) trials_kernel(Dev<R> d, int trials, int mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  GridBarrier* bar = d.bar;
  const unsigned long long lim = d.barrier_cycles;
  const int gsz = gridDim.x * blockDim.x, gid = blockIdx.x * blockDim.x + threadIdx.x;

  if (mode == MODE_RESIDUAL) {
    if (MODEL >= MODEL_LAMINAR) {
      tile_sweep<R, MODEL, FLUX, true>(d, STAGE_DIAG, sm);
      if (!grid_barrier(bar, lim)) return;
    }
    tile_sweep<R, MODEL, FLUX, false>(d, STAGE_DIAG, sm);
    return;
  }

  // begin (first trial of this launch)
  for (int cs = gid; cs < d.n_cases; cs += gsz) {
    CaseCtl& c = d.ctl[cs];
    case_begin(c);
    if (c.active) atomicAdd(&bar->live[0], 1);
  }
  if (!grid_barrier(bar, lim)) return;
  if (ld_volatile(&bar->live[0]) == 0) return;

  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5;
  for (int trial = 0; trial < trials; ++trial) {
    // ---- stage 0: base residual and cell dt
    if (MODEL >= MODEL_LAMINAR) {
      tile_sweep<R, MODEL, FLUX, true>(d, STAGE_BASE, sm);
      if (!grid_barrier(bar, lim)) return;
    }
    tile_sweep<R, MODEL, FLUX, false>(d, STAGE_BASE, sm);
    if (!grid_barrier(bar, lim)) return;
    if (SRD && MODEL >= MODEL_LAMINAR && d.any_srd_rate) {
      for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
        int cur;
        if (read_case_skip(d.ctl, cs, SKIP_ACTIVE, !d.cfg[cs].srd_rate, &cur)) continue;
        srd_rate_case<R, MODEL>(d, cs, false);
      }
      if (!grid_barrier(bar, lim)) return;
    }
    // ---- dt and U1
    for (int ti = blockIdx.x * wpb + warp; ti < d.n_tiles; ti += gridDim.x * wpb) {
      const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_ACTIVE);
      if (v.skip) continue;
      phase_first_update<R, MODEL>(d, v.t, state_buf(d, v.cur), state_buf(d, v.cur ^ 1));
    }
    if (!grid_barrier(bar, lim)) return;
    for (int stage = 1; stage <= 2; ++stage) {
      if (SRD) {
        for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
          int cur;
          if (read_case_skip(d.ctl, cs, SKIP_STAGE, !d.cfg[cs].has_srd, &cur)) continue;
          phase_srd<R, MODEL>(d, cs, stage == 1 ? state_buf(d, cur ^ 1) : d.U2, false);
        }
        if (!grid_barrier(bar, lim)) return;
      }
      if (MODEL >= MODEL_LAMINAR) {
        tile_sweep<R, MODEL, FLUX, true>(d, stage, sm);
        if (!grid_barrier(bar, lim)) return;
      }
      tile_sweep<R, MODEL, FLUX, false>(d, stage, sm);
      if (!grid_barrier(bar, lim)) return;
    }
    if (SRD) {
      for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
        int cur;
        if (read_case_skip(d.ctl, cs, SKIP_STAGE, !d.cfg[cs].has_srd, &cur)) continue;
        phase_srd<R, MODEL>(d, cs, state_buf(d, cur ^ 1), true);
      }
      if (!grid_barrier(bar, lim)) return;
    }
    // ---- commit and begin the next trial
    const int next = (trial + 1) % 3;
    if (gid == 0) bar->live[(trial + 2) % 3] = 0;
    for (int cs = gid; cs < d.n_cases; cs += gsz) {
      CaseCtl& c = d.ctl[cs];
      case_commit(c);
      case_begin(c);
      if (c.active) atomicAdd(&bar->live[next], 1);
    }
    if (!grid_barrier(bar, lim)) return;
    if (ld_volatile(&bar->live[next]) == 0) return;
  }
}

// ------------------------------------------------------------------------------------------
// Phase kernels: the same phases as trials_kernel, one kernel per phase, for batches large
// enough to fill the GPU many times over.  A trial is the launch sequence
//   [grad 0] flux 0, first, [srd 1], [grad 1], flux 1, [srd 2], [grad 2], flux 2, [srd 3], commit
// and a CUDA graph replays `trials` such sequences.
// ------------------------------------------------------------------------------------------
// Phase kernels run 128-thread blocks; the occupancy target sets the register budget
// (FP32: 8 blocks -> 64 registers, FP64: 3 blocks -> 168 registers).
constexpr int PHASE_BLOCK = 128;
#ifndef AMRB_FLUX_MINB_F32
#define AMRB_FLUX_MINB_F32 8
#endif
template <class R> struct PhaseOcc;
template <> struct PhaseOcc<float> { static constexpr int flux = AMRB_FLUX_MINB_F32, grad = 8; };
template <> struct PhaseOcc<double> { static constexpr int flux = 3, grad = 4; };

// Compiled once per stage, like the split kernels, so that each instance carries its own path only.
template <class R, int MODEL, int STAGE>
__global__ void __launch_bounds__(PHASE_BLOCK, PhaseOcc<R>::grad) phase_grad_kernel(Dev<R> d) {
  chain_begin();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile_sweep<R, MODEL, 0, true>(d, STAGE, reinterpret_cast<R*>(smem_raw));
}

template <class R, int MODEL, int FLUX, int STAGE>
__global__ void __launch_bounds__(PHASE_BLOCK, PhaseOcc<R>::flux) phase_flux_kernel(Dev<R> d) {
  chain_begin();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  tile_sweep<R, MODEL, FLUX, false>(d, STAGE, reinterpret_cast<R*>(smem_raw));
}

// U1 = U + dt R0, one thread per cell (phase mode).  Every thread derives its case's step size
// from the control record; the first cell of each case records it.
template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK) phase_first_cells_kernel(Dev<R> d) {
  chain_begin();
  const long long n = d.ncap;
  const int ncells = d.live_end[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ncells; k += gridDim.x * blockDim.x) {
    const int cs = d.c_case[k];
    if (cs < 0) continue;
    const CaseCtl& c = d.ctl[cs];
    if (!c.active) continue;
    const CaseCfg<R>& cf = d.cfg[cs];
    double dt;
    int fatal;
    const bool ok = choose_dt(c, cf.dt_fixed, &dt, &fatal);
    if (k == 0 || d.c_case[k - 1] != cs) {
      if (ok) {
        d.ctl[cs].dt_trial = dt;
        if (!c.retrying) d.ctl[cs].attempt = 0;
      } else {
        d.ctl[cs].fatal = fatal;
      }
    }
    if (!ok) continue;
    const R dtr = (R)dt;
    R* Ub = state_buf(d, c.cur);
    R* Un = state_buf(d, c.cur ^ 1);
    const bool simple = cf.has_srd && (d.c_flags[k] & 1);
    const int nv = MODEL == MODEL_SA ? 5 : 4;
    for (int v = 0; v < nv; ++v) {
      R u = Ub[v * n + k] + dtr * d.R0[v * n + k];
      if (simple && v < 4) u = srd_self(u, d.c_vol[k], d.c_gvol[k]);
      Un[v * n + k] = u;
    }
  }
}

// The first update's control part alone, one thread per case (split mode with the fused first update: the
// state part, U1 = U + dt R0, is formed where the stage-1 kernels read it).  Same decisions as
// phase_first_cells_kernel makes at a case's first cell.
template <class R>
__global__ void __launch_bounds__(128) dt_cases_kernel(Dev<R> d) {
  chain_begin();
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= d.n_cases) return;
  if (d.case_lane && d.case_lane[cs] != d.lane) return;
  const CaseCtl& c = d.ctl[cs];
  if (!c.live || !c.active) return;
  double dt;
  int fatal;
  if (choose_dt(c, d.cfg[cs].dt_fixed, &dt, &fatal)) {
    d.ctl[cs].dt_trial = dt;
    if (!c.retrying) d.ctl[cs].attempt = 0;
  } else {
    d.ctl[cs].fatal = fatal;
  }
}

// stage 1: SRD of U1, stage 2: of U2, stage 3: of the final candidate with the admissibility check.
template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK) phase_srd_kernel(Dev<R> d, int stage) {
  chain_begin();
  for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
    int cur;
    if (read_case_skip(d.ctl, cs, SKIP_STAGE, !d.cfg[cs].has_srd, &cur)) continue;
    R* u = stage == 2 ? d.U2 : state_buf(d, cur ^ 1);
    phase_srd<R, MODEL>(d, cs, u, stage == 3);
  }
}

// Accept/reject the trial (unless begin_only) and begin the next one, one thread per case.
static __global__ void phase_commit_kernel(CaseCtl* ctl, int n_cases, int begin_only, const int* case_lane,
                                           int lane) {
  chain_begin();
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= n_cases) return;
  if (case_lane && case_lane[cs] != lane) return;
  CaseCtl& c = ctl[cs];
  if (!begin_only) case_commit(c);
  case_begin(c);
}

// ------------------------------------------------------------------------------------------
// Split mode: gradients one thread per cell, fluxes one thread per face or wall record (each face
// evaluated once, in face orientation), then one thread per cell gathering its records in the
// reference's order with the stage update.  Same arithmetic as the other modes.
// ------------------------------------------------------------------------------------------
#ifndef AMRB_SPLIT_MINB_F32
#define AMRB_SPLIT_MINB_F32 8
#endif
#ifndef AMRB_SPLIT_CELL_MINB_F32
#define AMRB_SPLIT_CELL_MINB_F32 12
#endif
template <class R> struct SplitOcc;
#ifndef AMRB_SPLIT_GATHER_MINB_F32
#define AMRB_SPLIT_GATHER_MINB_F32 AMRB_SPLIT_CELL_MINB_F32
#endif
template <> struct SplitOcc<float> {
  static constexpr int item = AMRB_SPLIT_MINB_F32, cell = AMRB_SPLIT_CELL_MINB_F32, gather = AMRB_SPLIT_GATHER_MINB_F32;
};
template <> struct SplitOcc<double> { static constexpr int item = 3, cell = 4, gather = 4; };
// Blocks per SM per stage and kernel (FP32), each defaulting to its kernel's SplitOcc value; FP32
// stage 1 forms U1 = U + dt R0 in place in its gradient and gather kernels (and its gather also keeps
// the stage increment), so those are the instances that need the most registers.
#ifndef AMRB_S0_CELL_F32
#define AMRB_S0_CELL_F32 AMRB_SPLIT_CELL_MINB_F32
#endif
#ifndef AMRB_S1_CELL_F32
#define AMRB_S1_CELL_F32 AMRB_SPLIT_CELL_MINB_F32
#endif
#ifndef AMRB_S2_CELL_F32
#define AMRB_S2_CELL_F32 AMRB_SPLIT_CELL_MINB_F32
#endif
#ifndef AMRB_S0_GATHER_F32
#define AMRB_S0_GATHER_F32 AMRB_SPLIT_GATHER_MINB_F32
#endif
#ifndef AMRB_S1_GATHER_F32
#define AMRB_S1_GATHER_F32 AMRB_SPLIT_GATHER_MINB_F32
#endif
#ifndef AMRB_S2_GATHER_F32
#define AMRB_S2_GATHER_F32 AMRB_SPLIT_GATHER_MINB_F32
#endif
#ifndef AMRB_S0_ITEM_F32
#define AMRB_S0_ITEM_F32 AMRB_SPLIT_MINB_F32
#endif
#ifndef AMRB_S12_ITEM_F32
#define AMRB_S12_ITEM_F32 AMRB_SPLIT_MINB_F32
#endif
template <class R, int STAGE> struct SplitStageOcc : SplitOcc<R> {};
template <> struct SplitStageOcc<float, 0> {
  static constexpr int item = AMRB_S0_ITEM_F32, cell = AMRB_S0_CELL_F32, gather = AMRB_S0_GATHER_F32;
};
template <> struct SplitStageOcc<float, 1> {
  static constexpr int item = AMRB_S12_ITEM_F32, cell = AMRB_S1_CELL_F32, gather = AMRB_S1_GATHER_F32;
};
template <> struct SplitStageOcc<float, 2> {
  static constexpr int item = AMRB_S12_ITEM_F32, cell = AMRB_S2_CELL_F32, gather = AMRB_S2_GATHER_F32;
};

__device__ __forceinline__ int stage_rule(int stage) {
  return stage == STAGE_DIAG ? SKIP_LIVE : (stage == STAGE_BASE ? SKIP_ACTIVE : SKIP_STAGE);
}

template <class R, int MODEL> __device__ __forceinline__ void store_record(R* dst, R* rec, bool base) {
  if (!base) rec[8] = rec[9] = rec[11] = R(0);
  if (MODEL < MODEL_SA) rec[10] = rec[11] = R(0);
  if (MODEL < MODEL_LAMINAR) rec[9] = R(0);
  store_group(dst, rec);
  if (MODEL >= MODEL_LAMINAR) store_group(dst + 4, rec + 4);
  if (base || MODEL == MODEL_SA) store_group(dst + 8, rec + 8);
}

template <class R, int MODEL> __device__ __forceinline__ void load_record(const R* src, R* col, bool base) {
  load_group(src, col);
  if (MODEL >= MODEL_LAMINAR) load_group(src + 4, col + 4);
  if (base || MODEL == MODEL_SA) load_group(src + 8, col + 8);
}

// FP32 viscous records in split mode are compact: 8 values, the net flux (convective minus
// viscous, which the cell sums only ever use as that difference) and the four spectral / SA
// columns, 32 bytes instead of 48.  A wall contributes only momentum columns 1-2 of its
// convective part, so its columns 0 and 3 carry the viscous values alone.  FP64 keeps all 12
// columns so that its sums are formed exactly as the reference forms them.
template <class R, int MODEL> struct RecFormat {
  static constexpr bool compact = sizeof(R) == 4 && MODEL >= MODEL_LAMINAR;
  static constexpr int stride = compact ? 8 : SM_COLS;
};

// The compact record's SA flux (column 10) lives in a per-record array of its own (sa_dst /
// sa_src), so that the stages after the first, which need no spectral columns, move 20 bytes per
// record instead of 32.
template <class R, int MODEL>
__device__ __forceinline__ void store_item(R* dst, R* rec, bool base, bool wall, R* sa_dst = nullptr) {
  if (!RecFormat<R, MODEL>::compact) {
    store_record<R, MODEL>(dst, rec, base);
    return;
  }
  if (!base) rec[8] = rec[9] = rec[11] = R(0);
  if (MODEL < MODEL_SA) rec[10] = rec[11] = R(0);
  R net[4];
  for (int v = 0; v < 4; ++v) net[v] = rec[v] - rec[4 + v];
  if (wall) {
    net[0] = rec[4];
    net[3] = rec[7];
  }
  store_group(dst, net);
  if (MODEL == MODEL_SA) *sa_dst = rec[10];
  if (base) store_group(dst + 4, rec + 8);
}

// The 12 columns of a stored item, flux columns multiplied by sg (the slot's orientation).
template <class R, int MODEL>
__device__ __forceinline__ void load_item(const R* src, R* col, bool base, bool wall, R sg, const R* sa_src = nullptr) {
  for (int c = 0; c < SM_COLS; ++c) col[c] = R(0);
  if (!RecFormat<R, MODEL>::compact) {
    load_record<R, MODEL>(src, col, base);
    for (int v = 0; v < 4; ++v) col[v] = sg * col[v];
    if (MODEL >= MODEL_LAMINAR)
      for (int v = 4; v < 8; ++v) col[v] = sg * col[v];
  } else {
    load_group(src, col);
    for (int v = 0; v < 4; ++v) col[v] = sg * col[v];
    if (wall) {  // the viscous columns the cell sums take from a wall
      col[4] = col[0];
      col[7] = col[3];
      col[0] = col[3] = R(0);
    }
    if (base) load_group(src + 4, col + 8);
    if (MODEL == MODEL_SA) col[10] = __ldg(sa_src);
  }
  if (MODEL == MODEL_SA) col[10] = sg * col[10];
}

// The split kernels are compiled once per stage (STAGE_BASE, STAGE_1, STAGE_2, STAGE_DIAG), and the
// stage-1 cell kernels once more for the in-place first update (FUSED: U1 = U + dt R0 formed where
// it is read): each instance carries only its own path, so its registers go to that path alone
// (the base stage's FP64 dt sums, the first stage's update and the final stage's two-word update
// are never live in one kernel).
template <class R, int MODEL, int STAGE, bool FUSED = false>
__global__ void __launch_bounds__(PHASE_BLOCK, SplitStageOcc<R, STAGE>::cell) grad_cells_kernel(Dev<R> d) {
  constexpr int stage = STAGE;
  chain_begin();
  const int rule = stage_rule(stage);
  const int ncells = d.live_end[0], c0 = d.live_begin ? d.live_begin[0] : 0;
  for (int k = c0 + blockIdx.x * blockDim.x + threadIdx.x; k < ncells; k += gridDim.x * blockDim.x) {
    const int cs = d.c_case[k];
    if (cs < 0) continue;
    const CaseCtl& c = d.ctl[cs];
    if (skip_case(c, rule)) continue;
    const CaseCfg<R>& cf = d.cfg[cs];
    const auto cell = [&](const auto& Uin) {
      R gr[4] = {0, 0, 0, 0}, sg[4] = {0, 0, 0, 0};
      for (int q = d.c_term[k]; q < d.c_term[k + 1]; ++q) {
        R t[8];
        term_values<R, MODEL>(d, cf, q, k, Uin, t);
        for (int v = 0; v < 4; ++v) gr[v] += t[v];
        if (MODEL == MODEL_SA)
          for (int v = 0; v < 4; ++v) sg[v] += t[4 + v];
      }
      // the packed record feeds the item kernel; the SoA copies only the residual-mode loads
      return grad_finish<R, MODEL>(d, cf, k, Uin, gr, sg, stage == STAGE_DIAG,
                                   d.crec + CellRec<R, MODEL>::stride * (long long)k, true, CellRec<R, MODEL>::compact);
    };
    const bool ok = FUSED && stage == STAGE_1
                        ? cell(FusedIn<R>{state_buf(d, c.cur), d.R0, (R)c.dt_trial})
                        : cell(stage_input(d, stage, c.cur));
    if (!ok) atomicOr(&d.ctl[cs].bad, 1);
  }
}

template <class R, int MODEL, int FLUX, int STAGE>
__global__ void __launch_bounds__(PHASE_BLOCK, SplitStageOcc<R, STAGE>::item) item_kernel(Dev<R> d) {
  constexpr int stage = STAGE;
  chain_begin();
  const int rule = stage_rule(stage);
  const bool base = stage == STAGE_BASE || stage == STAGE_DIAG;  // spectral columns wanted
  // this lane's faces [f0, nf), then its walls [w0, nw) at item indices nf - f0 on
  const int f0 = d.live_begin ? d.live_begin[1] : 0, w0 = d.live_begin ? d.live_begin[2] : 0;
  const int nf = d.live_end[1] - f0, total = nf + d.live_end[2] - w0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    bool bad = false;
    int cs;
    if (idx < nf) {
      const int f = f0 + idx;
      cs = d.f_case[f];
      if (cs < 0) continue;
      const CaseCtl& c = d.ctl[cs];
      if (skip_case(c, rule)) continue;
      R rec[SM_COLS];
      const int own = __ldg(d.f_own + f), nb = __ldg(d.f_nb + f);
      if (MODEL >= MODEL_LAMINAR) {
        FaceIn<R> in;
        face_in_records<R, MODEL>(d, d.cfg[cs], d.f_geo + 6 * (long long)f, own, nb >= 0 ? nb : own, in);
        face_fluxes<R, MODEL, FLUX>(d.cfg[cs], in, __ldg(d.f_len + f), nb, __ldg(d.f_meta + f), base, rec, 1, false, bad);
      } else {
        slot_face<R, MODEL, FLUX>(d, d.cfg[cs], d.f_geo + 6 * (long long)f, __ldg(d.f_len + f), own, nb,
                                  __ldg(d.f_meta + f), stage_input(d, stage, c.cur), base, rec, 1, false, bad);
      }
      store_item<R, MODEL>(d.fval + RecFormat<R, MODEL>::stride * (long long)f, rec, base, false, d.fsa + f);
    } else {
      const int w = w0 + idx - nf;
      const int owner = d.w_owner[w];
      if (owner < 0) continue;
      cs = d.c_case[owner];
      const CaseCtl& c = d.ctl[cs];
      if (skip_case(c, rule)) continue;
      R rec[SM_COLS];
      if (MODEL >= MODEL_LAMINAR)
        slot_wall_records<R, MODEL>(d, d.cfg[cs], __ldg(d.w_nx + w), __ldg(d.w_ny + w), __ldg(d.w_dist + w),
                                    __ldg(d.w_len + w), owner, __ldg(d.w_donor + w), base, rec, 1, bad);
      else
        slot_wall<R, MODEL>(d, d.cfg[cs], __ldg(d.w_nx + w), __ldg(d.w_ny + w), __ldg(d.w_dist + w), __ldg(d.w_len + w),
                            owner, __ldg(d.w_donor + w), stage_input(d, stage, c.cur), base, rec, 1, bad);
      store_item<R, MODEL>(d.wval + RecFormat<R, MODEL>::stride * (long long)w, rec, base, true, d.wsa + w);
    }
    if (bad && stage != STAGE_DIAG) atomicOr(&d.ctl[cs].bad, 1);
  }
}

// The 12 values of a slot's face or wall record, flux columns signed for the slot's cell.
template <class R, int MODEL> struct ItemSlots {
  static constexpr bool net_cols = RecFormat<R, MODEL>::compact;
  const Dev<R>* d;
  bool base;
  __device__ __forceinline__ Cols<R> operator()(int q, bool wall) const {
    const int id = __ldg(d->s_item + q);  // wall index, or 2 * face record + (cell is the face's left)
    constexpr int S = RecFormat<R, MODEL>::stride;
    const R* src = wall ? d->wval + S * (long long)id : d->fval + S * (long long)(id >> 1);
    const R* sa = wall ? d->wsa + id : d->fsa + (id >> 1);
    Cols<R> o;
    load_item<R, MODEL>(src, o.v, base, wall, (wall || (id & 1)) ? R(1) : R(-1), sa);
    return o;
  }
};

template <class R, int MODEL, int STAGE, bool FUSED = false>
__global__ void __launch_bounds__(PHASE_BLOCK, SplitStageOcc<R, STAGE>::gather) gather_kernel(Dev<R> d) {
  constexpr int stage = STAGE;
  chain_begin();
  const int rule = stage_rule(stage);
  const int ncells = d.live_end[0], c0 = d.live_begin ? d.live_begin[0] : 0;
  const bool base = stage == STAGE_BASE;
  const int lane = threadIdx.x & 31;
  // the loop bound is warp-uniform so the segmented shuffles below see full warps
  for (int k0 = c0 + blockIdx.x * blockDim.x; k0 < ncells; k0 += gridDim.x * blockDim.x) {
    const int k = k0 + threadIdx.x;
    int cs = -1, a = 0, b = 0, nw = 0;
    if (k < ncells) {
      // the cell's own table loads go out together, ahead of its case's skip test
      cs = d.c_case[k];
      a = d.c_slot[k];
      b = d.c_slot[k + 1];
      nw = d.c_wall[k + 1] - d.c_wall[k];
    }
    bool bad = false;
    double cell_dt = __longlong_as_double(0x7FF0000000000000ll);
    if (cs >= 0 && skip_case(d.ctl[cs], rule)) cs = -1;
    if (cs >= 0) {
      const CaseCtl& c = d.ctl[cs];
      const int e = b - nw;
      const ItemSlots<R, MODEL> get{&d, base || stage == STAGE_DIAG};
      if (FUSED && stage == STAGE_1)
        cell_dt = finish_cell<R, MODEL>(d, d.cfg[cs], cs, k, stage, a, e, b, get,
                                        FusedIn<R>{state_buf(d, c.cur), d.R0, (R)c.dt_trial}, state_buf(d, c.cur),
                                        state_buf(d, c.cur ^ 1), bad);
      else
        cell_dt = finish_cell<R, MODEL>(d, d.cfg[cs], cs, k, stage, a, e, b, get, stage_input(d, stage, c.cur),
                                        state_buf(d, c.cur), state_buf(d, c.cur ^ 1), bad);
      if (bad && stage != STAGE_DIAG) atomicOr(&d.ctl[cs].bad, 1);
    }
    if (base) {
      // per-case minimum over the warp: cells of a case are contiguous, so a segmented suffix
      // minimum leaves each segment's first lane with its segment's minimum
      unsigned long long bits = (unsigned long long)__double_as_longlong(cell_dt);
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long ob = __shfl_down_sync(FULL_MASK, bits, o);
        const int oc = __shfl_down_sync(FULL_MASK, cs, o);
        if (lane + o < 32 && oc == cs && ob < bits) bits = ob;
      }
      const int prev = __shfl_up_sync(FULL_MASK, cs, 1);
      if (cs >= 0 && (lane == 0 || prev != cs)) atomicMin(&d.ctl[cs].dtmin, bits);
    }
  }
}

template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK) srd_rate_kernel(Dev<R> d, int store_only_case) {
  chain_begin();
  for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
    int cur;
    if (store_only_case >= 0) {
      if (cs != store_only_case) continue;
      srd_rate_case<R, MODEL>(d, cs, true);
      continue;
    }
    if (read_case_skip(d.ctl, cs, SKIP_ACTIVE, !d.cfg[cs].srd_rate, &cur)) continue;
    srd_rate_case<R, MODEL>(d, cs, false);
  }
}

// ------------------------------------------------------------------------------------------
// Tiled mode: one kernel per stage.  Each block takes one block tile at a time and keeps every
// intermediate in shared memory: (A) the packed records of the tile's cells and halo cells
// (state, gradients, viscosity, SA fields; each cell's LSQ sums in term order), (B) the fluxes of
// every face record and wall fragment touching the tile's cells (a face on the tile's border is
// evaluated by both tiles, each time identically), (C) per cell, the in-order sums over its
// slots, the residual, dt and the stage update.  Same arithmetic as the other modes.
// ------------------------------------------------------------------------------------------
template <class R> struct TiledOcc;
template <> struct TiledOcc<float> { static constexpr int blocks = 512 / BT_CELLS; };
template <> struct TiledOcc<double> { static constexpr int blocks = 1; };

template <class R> __host__ __device__ constexpr size_t tiled_smem_bytes() {
  return sizeof(R) * ((size_t)BT_DATA * CREC + (size_t)(BT_FACES + BT_WALLS) * SM_COLS);
}

// A slot's record from the tile's shared-memory records, flux columns signed for the slot's cell.
template <class R, int MODEL> struct TileSlots {
  const R* fr;  // face records then wall records, SM_COLS each
  const int* s_loc;
  int nf;
  __device__ __forceinline__ Cols<R> operator()(int q, bool wall) const {
    const int loc = __ldg(s_loc + q);
    const R* src = fr + SM_COLS * (wall ? nf + loc : loc >> 1);
    const R sg = (wall || (loc & 1)) ? R(1) : R(-1);
    Cols<R> o;
    R* col = o.v;
    for (int c = 0; c < SM_COLS; ++c) col[c] = src[c];
    for (int v = 0; v < 4; ++v) col[v] = sg * col[v];
    if (MODEL >= MODEL_LAMINAR)
      for (int v = 4; v < 8; ++v) col[v] = sg * col[v];
    if (MODEL == MODEL_SA) col[10] = sg * col[10];
    return o;
  }
};

template <class R, int MODEL, int FLUX>
__global__ void __launch_bounds__(BT_THREADS, TiledOcc<R>::blocks) tiled_stage_kernel(Dev<R> d, int stage) {
  chain_begin();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* cr = reinterpret_cast<R*>(smem_raw);  // BT_DATA x CREC
  R* fr = cr + BT_DATA * CREC;             // (BT_FACES + BT_WALLS) x SM_COLS
  __shared__ unsigned long long block_dt;
  const int rule = stage_rule(stage);
  const bool base = stage == STAGE_BASE;
  const bool spec = base || stage == STAGE_DIAG;
  const long long n = d.ncap;
  const int ntiles = d.live_end[3];
  for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
    const BTile t = d.btiles[ti];
    int cur;
    // one thread reads the control word for the block (other tiles may flag the case meanwhile)
    if (read_case_skip(d.ctl, t.cs, rule, false, &cur)) continue;
    const CaseCfg<R>& cf = d.cfg[t.cs];
    const R* Uin = stage_input(d, stage, cur);
    const int nt = t.c1 - t.c0, nd = nt + (t.h1 - t.h0), nf = t.f1 - t.f0, nw = t.w1 - t.w0;
    if (threadIdx.x == 0) block_dt = DT_INF_BITS;
    bool bad = false;
    // (A) packed records of the tile and halo cells
    for (int i = threadIdx.x; i < nd; i += blockDim.x) {
      const bool own = i < nt;
      const int k = own ? t.c0 + i : __ldg(d.bt_halo + t.h0 + i - nt);
      R* rec = cr + CREC * i;
      if (MODEL >= MODEL_LAMINAR) {
        R gr[4] = {0, 0, 0, 0}, sg[4] = {0, 0, 0, 0};
        for (int q = d.c_term[k]; q < d.c_term[k + 1]; ++q) {
          R tv[8];
          term_values<R, MODEL>(d, cf, q, k, Uin, tv);
          for (int v = 0; v < 4; ++v) gr[v] += tv[v];
          if (MODEL == MODEL_SA)
            for (int v = 0; v < 4; ++v) sg[v] += tv[4 + v];
        }
        if (!grad_finish<R, MODEL>(d, cf, k, Uin, gr, sg, own && stage == STAGE_DIAG, rec, own) && own) bad = true;
      } else {
        for (int v = 0; v < 4; ++v) rec[v] = Uin[v * n + k];
        rec[4] = R(0);
      }
    }
    __syncthreads();
    // (B) face and wall fluxes into shared records
    for (int j = threadIdx.x; j < nf + nw; j += blockDim.x) {
      R* out = fr + SM_COLS * j;
      if (j < nf) {
        const int f = __ldg(d.bt_face + t.f0 + j);
        const int2 loc = d.bt_floc[t.f0 + j];
        const R* a = cr + CREC * loc.x;
        const R* b = cr + CREC * (loc.y >= 0 ? loc.y : loc.x);
        FaceIn<R> in;
        for (int v = 0; v < 5; ++v) { in.uk[v] = a[v]; in.um[v] = b[v]; }
        in.mk = in.mm = in.ek = in.em = in.sdk = in.sdm = 0;
        in.sgk[0] = in.sgk[1] = in.sgm[0] = in.sgm[1] = 0;
        if (MODEL >= MODEL_LAMINAR) {
          for (int v = 0; v < 4; ++v) { in.gk[v] = a[5 + v]; in.gm[v] = b[5 + v]; }
          in.mk = a[9]; in.mm = b[9]; in.ek = a[10]; in.em = b[10];
          if (MODEL == MODEL_SA) {
            in.sgk[0] = a[11]; in.sgk[1] = a[12]; in.sgm[0] = b[11]; in.sgm[1] = b[12];
            in.sdk = a[13]; in.sdm = b[13];
          }
          for (int v = 0; v < 6; ++v) in.geo[v] = __ldg(d.f_geo + 6 * (long long)f + v);
        }
        face_fluxes<R, MODEL, FLUX>(cf, in, __ldg(d.f_len + f), loc.y, __ldg(d.f_meta + f), spec, out, 1, false, bad);
      } else {
        const int w = t.w0 + j - nf;
        const R* a = cr + CREC * (d.w_owner[w] - t.c0);
        WallIn<R> in;
        for (int v = 0; v < 4; ++v) in.uk[v] = a[v];
        in.mk = in.md = 0;
        in.ud[0] = in.ud[1] = in.ud[2] = in.ud[3] = in.ud[4] = 0;
        if (MODEL >= MODEL_LAMINAR) {
          const R* b = cr + CREC * __ldg(d.w_ldon + w);
          for (int v = 0; v < 5; ++v) in.ud[v] = b[v];
          in.mk = a[9];
          in.md = b[9];
        }
        wall_fluxes<R, MODEL>(cf, in, __ldg(d.w_nx + w), __ldg(d.w_ny + w), __ldg(d.w_dist + w), __ldg(d.w_len + w),
                              spec, out, 1, bad);
      }
    }
    __syncthreads();
    // (C) per-cell sums, residual, dt and the stage update
    double cell_dt = __longlong_as_double(0x7FF0000000000000ll);
    for (int i = threadIdx.x; i < nt; i += blockDim.x) {
      const int k = t.c0 + i;
      const int a = d.c_slot[k], b = d.c_slot[k + 1];
      const int e = b - (d.c_wall[k + 1] - d.c_wall[k]);
      cell_dt = rmin(cell_dt, finish_cell<R, MODEL>(d, cf, t.cs, k, stage, a, e, b, TileSlots<R, MODEL>{fr, d.s_loc, nf},
                                                    Uin, state_buf(d, cur), state_buf(d, cur ^ 1), bad));
    }
    if (bad && stage != STAGE_DIAG) atomicOr(&d.ctl[t.cs].bad, 1);
    if (base) {
      for (int o = 16; o > 0; o >>= 1) cell_dt = rmin(cell_dt, __shfl_xor_sync(FULL_MASK, cell_dt, o));
      if ((threadIdx.x & 31) == 0 && cell_dt < __longlong_as_double(0x7FF0000000000000ll))
        atomicMin(&block_dt, (unsigned long long)__double_as_longlong(cell_dt));
    }
    __syncthreads();
    if (base && threadIdx.x == 0 && block_dt != DT_INF_BITS) atomicMin(&d.ctl[t.cs].dtmin, block_dt);
    __syncthreads();  // the shared records are reused by the next tile
  }
}

// The split mode in lanes: each lane's Dev (its ranges and case filter), and the auxiliary
// streams and fork/join events that run lanes 1.. beside lane 0.
constexpr int MAX_LANES = 4;
template <class R> struct SplitLanes {
  int n = 1;
  Dev<R> dev[MAX_LANES];
  cudaStream_t aux[MAX_LANES - 1] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[MAX_LANES - 1] = {};
};

// Host-visible launch helpers (defined in amr_engine_f64.cu / amr_engine_f32.cu).
template <class R> struct EngineOps {
  static cudaError_t launch(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int grid, int block,
                            cudaStream_t stream, bool cooperative);
  // One trial (or, with mode MODE_RESIDUAL, one residual evaluation) as a sequence of phase kernels.
  static cudaError_t launch_phases(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int block,
                                   cudaStream_t stream);
  // The same with the split kernels (gradients per cell, fluxes per face record, gather per cell).
  // With lanes, their trials run as independent chains (lanes->dev[0] on stream, dev[i] on
  // lanes->aux[i - 1]), so that one lane's kernels fill the tails of the others'.
  static cudaError_t launch_split(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode,
                                  cudaStream_t stream, int sms, const SplitLanes<R>* lanes = nullptr);
  // The same with one shared-memory tiled kernel per stage.
  static cudaError_t launch_tiled(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode,
                                  cudaStream_t stream, int sms);
  // Lets the tiled kernel of a model and flux use its shared-memory tile (above the 48 KB default).
  static cudaError_t tiled_setup(int model, int flux);
  static cudaError_t occupancy(int model, int flux, bool srd, int block, int* blocks_per_sm);
  static size_t smem_bytes(int block) { return size_t(12) * block * sizeof(R); }
};

}  // namespace amrb
