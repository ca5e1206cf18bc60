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
};

// A run of whole cells of one case: cells [c0, c1), their slots [s0, s1) and gradient terms [t0, t1).
struct Tile {
  int cs, c0, c1, leader, s0, s1, t0, t1;
};
constexpr int SLOT_WALL = 1 << 9;  // s_meta flag: the slot is a wall fragment of its owner cell

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
  R* grad;
  R* mu;
  R* eddy;
  R* sgrad;
  R* sdiff;
  R* ssrc;
  R* srate;
  long long ncap;
  long long gcap;
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

template <class R> __device__ __forceinline__ Prim<R> prim(const R* U, long long n, int k, R g) {
  Prim<R> w;
  const R rho = U[k], mx = U[n + k], my = U[2 * n + k], e = U[3 * n + k];
  w.rho = rho;
  w.u = mx / rho;
  w.v = my / rho;
  w.p = (g - R(1)) * (e - R(0.5) * (mx * w.u + my * w.v));
  return w;
}

template <class R> __device__ __forceinline__ bool prim_ok(const R* U, long long n, int k, const Prim<R>& w) {
  const R mx = U[n + k], my = U[2 * n + k], e = U[3 * n + k];
  return isfinite(w.rho) && w.rho > R(0) && isfinite(mx) && isfinite(my) && isfinite(e) && isfinite(w.p) && w.p > R(0);
}

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

// ------------------------------------------------------------------------------------------
// G phase: velocity gradients, viscosity, eddy viscosity, SA gradients and point model of
// every cell of a tile (reference src/static_amr2d_viscous.cpp:166-174, src/static_amr2d_sa.cpp:74-80).
// ------------------------------------------------------------------------------------------
template <class R, int MODEL>
__device__ void phase_gradients(const Dev<R>& d, const Tile& t, const R* Uin, R* sm) {
  const int B = blockDim.x, i = threadIdx.x;
  const long long n = d.ncap;
  const CaseCfg<R>& cf = d.cfg[t.cs];
  const R g = cf.gamma;
  const int t0 = t.t0, t1 = t.t1;
  if (i < t1 - t0) {
    const int q = t0 + i, k = __ldg(d.t_own + q), src = __ldg(d.t_src + q);
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
    sm[0 * B + i] = x * du;
    sm[1 * B + i] = y * du;
    sm[2 * B + i] = x * dv;
    sm[3 * B + i] = y * dv;
    if (MODEL == MODEL_SA) {
      const R phk = Uin[4 * n + k] / rk;
      const R ph = src >= 0 ? Uin[4 * n + src] / Uin[src] : R(0);
      const R rho = src >= 0 ? Uin[src] : rk;
      sm[4 * B + i] = x * (ph - phk);
      sm[5 * B + i] = y * (ph - phk);
      sm[6 * B + i] = x * (rho - rk);
      sm[7 * B + i] = y * (rho - rk);
    }
  }
  __syncthreads();
  if (i < t.c1 - t.c0) {
    const int k = t.c0 + i;
    const Prim<R> w = prim(Uin, n, k, g);
    const R mu = dyn_visc(cf.trn, w.p / (w.rho * cf.trn.gas_constant));
    bool bad = !(mu > R(0)) || !isfinite(mu);
    R gr[4] = {0, 0, 0, 0}, sg[4] = {0, 0, 0, 0};
    const int a = d.c_term[k] - t0, b = d.c_term[k + 1] - t0;
    for (int q = a; q < b; ++q) {
      gr[0] += sm[0 * B + q];
      gr[1] += sm[1 * B + q];
      gr[2] += sm[2 * B + q];
      gr[3] += sm[3 * B + q];
    }
    for (int v = 0; v < 4; ++v) d.grad[v * n + k] = gr[v];
    d.mu[k] = mu;
    R eddy = 0;
    if (MODEL == MODEL_SA) {
      const R ph = Uin[4 * n + k] / w.rho;
      if (!isfinite(ph)) bad = true;
      eddy = w.rho * sa_eddy(ph, mu / w.rho);
      for (int q = a; q < b; ++q) {
        sg[0] += sm[4 * B + q];
        sg[1] += sm[5 * B + q];
        sg[2] += sm[6 * B + q];
        sg[3] += sm[7 * B + q];
      }
      const SaPoint<R> pt = sa_neg(ph, mu / w.rho, d.c_wd[k], R(fabs(gr[2] - gr[1])));
      const R src = sa_corrected_source(pt, w.rho, sg[0], sg[1], sg[2], sg[3]);
      d.sgrad[k] = sg[0];
      d.sgrad[n + k] = sg[1];
      d.sdiff[k] = pt.diffusion;
      d.ssrc[k] = src;
      d.srate[k] = pt.source_rate;
      if (!(pt.diffusion > R(0)) || !isfinite(src) || !isfinite(pt.source_rate)) bad = true;
    }
    d.eddy[k] = eddy;
    if (bad) atomicOr(&d.ctl[t.cs].bad, 1);
  }
  __syncthreads();
}

// ------------------------------------------------------------------------------------------
// F phase: per-slot face fluxes (convective + viscous + SA), then per-cell in-order sums,
// residual, cell dt and the stage update (reference src/static_amr2d.cpp:163-204,
// src/static_amr2d_viscous.cpp:177-206, src/static_amr2d_sa.cpp:81-96, 395-426).
// ------------------------------------------------------------------------------------------
template <class R, int MODEL, int FLUX>
__device__ __forceinline__ void slot_face(const Dev<R>& d, const CaseCfg<R>& cf, int s, int k, int nb, int meta,
                                          const R* Uin, bool base, R* sm, int B, int i, bool& bad) {
  const long long n = d.ncap;
  const R g = cf.gamma;
  const bool own_left = meta & 1;
  const int axis = (meta >> 1) & 1, side = ((meta >> 2) & 7) - 1, kind = (meta >> 5) & 15;
  // Every load of this slot is issued up front and unconditionally (an exterior face reads its
  // own cell twice), so the whole neighbourhood arrives in one memory round trip.
  const int m = nb >= 0 ? nb : k;
  const R len = __ldg(d.s_len + s);
  R uk[5], um[5];
  for (int v = 0; v < 4; ++v) { uk[v] = Uin[v * n + k]; um[v] = Uin[v * n + m]; }
  if (MODEL == MODEL_SA) { uk[4] = Uin[4 * n + k]; um[4] = Uin[4 * n + m]; }
  R gk[4], gm[4], geo[6], mk = 0, mm = 0, ek = 0, em = 0, sgk[2] = {0, 0}, sgm[2] = {0, 0}, sdk = 0, sdm = 0;
  if (MODEL >= MODEL_LAMINAR) {
    for (int v = 0; v < 4; ++v) { gk[v] = d.grad[v * n + k]; gm[v] = d.grad[v * n + m]; }
    mk = d.mu[k]; mm = d.mu[m]; ek = d.eddy[k]; em = d.eddy[m];
    const R* gp = d.s_geo + 6 * (long long)s;
    for (int v = 0; v < 6; ++v) geo[v] = __ldg(gp + v);
    if (MODEL == MODEL_SA) {
      sgk[0] = d.sgrad[k]; sgk[1] = d.sgrad[n + k]; sgm[0] = d.sgrad[m]; sgm[1] = d.sgrad[n + m];
      sdk = d.sdiff[k]; sdm = d.sdiff[m];
    }
  }
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
  const R sg = own_left ? R(1) : R(-1);
  sm[0 * B + i] = sg * f0;
  sm[1 * B + i] = sg * (axis ? ft : fn);
  sm[2 * B + i] = sg * (axis ? fn : ft);
  sm[3 * B + i] = sg * f3;
  if (base) {
    const R speed = rmax(R(fabs(an)) + sqrt(g * a[3] / a[0]), R(fabs(bn)) + sqrt(g * b[3] / b[0]));
    sm[8 * B + i] = speed * len;
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
      sm[(4 + v) * B + i] = sg * (fv[v] * len);
    }
    if (base) sm[9 * B + i] = R(4.0 / 3) * nu / distance * len;
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
      sm[10 * B + i] = sg * (mass * (mass >= R(0) ? left : right) - diff);
      if (base) sm[11 * B + i] = fc;
    }
  }
}

// A wall fragment of cell k: pressure force (reference src/static_amr2d.cpp:193-195), viscous wall
// flux from the visible donor (src/static_amr2d_viscous.cpp:192-196) and the SA wall flux
// (src/static_amr2d_sa.cpp:91), with their spectral-radius contributions.
template <class R, int MODEL>
__device__ __forceinline__ void slot_wall(const Dev<R>& d, const CaseCfg<R>& cf, int s, int k, int dn,
                                          const R* Uin, bool base, R* sm, int B, int i, bool& bad) {
  const long long n = d.ncap;
  const R g = cf.gamma;
  const R wl = __ldg(d.s_len + s);
  const R* geo = d.s_geo + 6 * (long long)s;
  const R nx = __ldg(geo + 0), ny = __ldg(geo + 1);
  const Prim<R> wk = prim(Uin, n, k, g);
  sm[0 * B + i] = 0;
  sm[1 * B + i] = wk.p * nx * wl;
  sm[2 * B + i] = wk.p * ny * wl;
  sm[3 * B + i] = 0;
  if (base) sm[8 * B + i] = sqrt(g * wk.p / wk.rho) * wl;
  if (MODEL >= MODEL_LAMINAR) {
    const R wdist = __ldg(geo + 2);
    const R rd = Uin[dn], ud = Uin[n + dn] / rd, vd = Uin[2 * n + dn] / rd;
    const R md = d.mu[dn];
    R gw[4], fw[4];
    wall_gradient(nx, ny, wdist, -ud, -vd, gw);
    visc_flux(md, gw, nx, ny, R(0), R(0), fw);
    for (int v = 0; v < 4; ++v) {
      if (!isfinite(fw[v])) bad = true;
      sm[(4 + v) * B + i] = fw[v] * wl;
    }
    if (base) sm[9 * B + i] = R(4.0 / 3) * rmax(md / rd, d.mu[k] / wk.rho) / wdist * wl;
    if (MODEL == MODEL_SA) {
      const R swc = md / R(AMRB_SIG) / wdist * wl;
      sm[10 * B + i] = -swc * (Uin[4 * n + dn] / rd);
      if (base) sm[11 * B + i] = swc;
    }
  }
}

template <class R, int MODEL, int FLUX>
__device__ void phase_flux(const Dev<R>& d, const Tile& t, int stage, const R* Uin, R* Ub, R* Un, R* sm,
                           bool* tile_bad, double* tile_dt) {
  const int B = blockDim.x, i = threadIdx.x;
  const long long n = d.ncap;
  const CaseCfg<R>& cf = d.cfg[t.cs];
  const R g = cf.gamma;
  const int s0 = t.s0, s1 = t.s1;
  const bool base = stage == STAGE_BASE;
  bool bad = false;
  if (i < s1 - s0) {
    const int s = s0 + i;
    const int k = __ldg(d.s_own + s), nb = __ldg(d.s_nb + s), meta = __ldg(d.s_meta + s);
    if (meta & SLOT_WALL)
      slot_wall<R, MODEL>(d, cf, s, k, nb, Uin, base, sm, B, i, bad);
    else
      slot_face<R, MODEL, FLUX>(d, cf, s, k, nb, meta, Uin, base, sm, B, i, bad);
  }
  __syncthreads();
  double cell_dt = __longlong_as_double(0x7FF0000000000000ll);
  if (i < t.c1 - t.c0) {
    const int k = t.c0 + i;
    const double V = d.c_vol[k];
    const Prim<R> wk = prim(Uin, n, k, g);
    if (!prim_ok(Uin, n, k, wk)) bad = true;
    // slots of cell k: faces [a, e) in CSR order, then walls [e, b)
    const int a = d.c_slot[k] - s0, b = d.c_slot[k + 1] - s0;
    const int e = b - (d.c_wall[k + 1] - d.c_wall[k]);
    R sum[4] = {0, 0, 0, 0};
    for (int q = a; q < e; ++q)
      for (int v = 0; v < 4; ++v) sum[v] += sm[v * B + q];
    for (int q = e; q < b; ++q) {
      sum[1] += sm[1 * B + q];
      sum[2] += sm[2 * B + q];
    }
    R res[5];
    for (int v = 0; v < 4; ++v) res[v] = (R)(-sum[v] / V);
    R vspec = 0, sspec = 0;
    if (MODEL >= MODEL_LAMINAR) {
      R vs[4] = {0, 0, 0, 0};
      for (int q = a; q < b; ++q) {
        for (int v = 0; v < 4; ++v) vs[v] += sm[(4 + v) * B + q];
        if (base) vspec += sm[9 * B + q];
      }
      for (int v = 0; v < 4; ++v) res[v] += (R)(vs[v] / V);
      if (MODEL == MODEL_SA) {
        R snet = 0;
        for (int q = a; q < e; ++q) {
          snet += sm[10 * B + q];
          if (base) sspec += sm[11 * B + q];
        }
        for (int q = e; q < b; ++q) {
          snet -= sm[10 * B + q];
          if (base) sspec += sm[11 * B + q];
        }
        res[4] = (R)(-snet / V) + d.ssrc[k];
        if (!isfinite(res[4])) bad = true;
      }
    }
    const int nv = MODEL == MODEL_SA ? 5 : 4;
    if (base) {
      R spectral = 0;
      for (int q = a; q < b; ++q) spectral += sm[8 * B + q];
      if (spectral > R(0)) cell_dt = cf.cfl * d.c_area[k] / (double)spectral;
      if (MODEL >= MODEL_LAMINAR) {
        const double vdt = vspec > R(0) ? cf.viscous_cfl * V / (double)vspec : __longlong_as_double(0x7FF0000000000000ll);
        double sdt = __longlong_as_double(0x7FF0000000000000ll);
        if (MODEL == MODEL_SA) {
          const double rate = 2 * (double)sspec / ((double)wk.rho * V) + (double)d.srate[k];
          sdt = rate > 0 ? cf.sa_cfl / rate : sdt;
        }
        cell_dt = rmin(cell_dt, rmin(vdt, sdt));
      }
      for (int v = 0; v < nv; ++v) d.R0[v * n + k] = res[v];
    } else if (stage == STAGE_DIAG) {
      for (int v = 0; v < nv; ++v) d.R0[v * n + k] = res[v];
    } else {
      const R dt = (R)d.ctl[t.cs].dt_trial;
      const bool simple = cf.has_srd && (d.c_flags[k] & 1);
      const bool check = stage == STAGE_2 && (!cf.has_srd || simple);
      R out[5];
      for (int v = 0; v < nv; ++v) {
        if (stage == STAGE_1)
          out[v] = R(0.75) * Ub[v * n + k] + R(0.25) * (Uin[v * n + k] + dt * res[v]);
        else
          out[v] = Ub[v * n + k] / R(3) + R(2.0 / 3) * (Uin[v * n + k] + dt * res[v]);
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
  }
  if (bad) *tile_bad = true;
  if (base) {
    // block minimum of the cell dt (exact; order-free)
    for (int o = 16; o > 0; o >>= 1) cell_dt = rmin(cell_dt, __shfl_xor_sync(0xffffffffu, cell_dt, o));
    if ((i & 31) == 0 && cell_dt < *tile_dt) {
      atomicMin((unsigned long long*)tile_dt, (unsigned long long)__double_as_longlong(cell_dt));
    }
  }
  __syncthreads();
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
  if (threadIdx.x == 0 && t.leader) {
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
  for (int j = threadIdx.x; j < t.c1 - t.c0; j += blockDim.x) {
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
  for (int gi = cf.srd_g0 + threadIdx.x; gi < cf.srd_g1; gi += blockDim.x) {
    const int m0 = d.g_mem[gi], m1 = d.g_mem[gi + 1];
    for (int v = 0; v < 4; ++v) {
      double sum = 0;
      for (int q = m0; q < m1; ++q) {
        const int k = d.g_cell[q];
        sum += d.c_vol[k] * (double)u[v * n + k] / d.g_cnt[q];
      }
      d.qhat[v * gc + gi] = sum / d.g_vol[gi];
    }
  }
  __syncthreads();
  bool bad = false;
  const R g = cf.gamma;
  for (int qi = cf.srd_q0 + threadIdx.x; qi < cf.srd_q1; qi += blockDim.x) {
    const int k = d.q_cell[qi], a = d.q_grp[qi], b = d.q_grp[qi + 1];
    R out[4];
    for (int v = 0; v < 4; ++v) {
      double sum = 0;
      for (int q = a; q < b; ++q) sum += d.qhat[v * gc + d.q_list[q]];
      out[v] = (R)(sum / d.q_cnt[qi]);
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
// the residual of every live case's accepted state into R0 (no update).
// Every skip decision is taken by thread 0 from the control word and broadcast through
// shared memory, so all threads of a block pass the same __syncthreads().
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
  __shared__ TileView s;
  if (threadIdx.x == 0) {
    s.t = tiles[ti];
    const CaseCtl& c = ctl[s.t.cs];
    s.skip = skip_case(c, rule);
    s.cur = c.cur;
  }
  __syncthreads();
  const TileView v = s;
  __syncthreads();
  return v;
}

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

template <class R, int MODEL, int FLUX, bool SRD>
__global__ void __launch_bounds__(MAX_BLOCK) trials_kernel(Dev<R> d, int trials, int mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  __shared__ bool s_bad;
  __shared__ double s_dt;
  GridBarrier* bar = d.bar;
  const unsigned long long lim = d.barrier_cycles;
  const int gsz = gridDim.x * blockDim.x, gid = blockIdx.x * blockDim.x + threadIdx.x;
  const double inf = __longlong_as_double(0x7FF0000000000000ll);

  if (mode == MODE_RESIDUAL) {
    if (MODEL >= MODEL_LAMINAR) {
      for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
        const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_LIVE);
        if (v.skip) continue;
        phase_gradients<R, MODEL>(d, v.t, state_buf(d, v.cur), sm);
      }
      if (!grid_barrier(bar, lim)) return;
    }
    for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
      const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_LIVE);
      if (v.skip) continue;
      if (threadIdx.x == 0) { s_bad = false; s_dt = 0; }
      __syncthreads();
      R* ub = state_buf(d, v.cur);
      phase_flux<R, MODEL, FLUX>(d, v.t, STAGE_DIAG, ub, ub, ub, sm, &s_bad, &s_dt);
    }
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

  for (int trial = 0; trial < trials; ++trial) {
    // ---- stage 0: base residual and cell dt
    if (MODEL >= MODEL_LAMINAR) {
      for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
        const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_ACTIVE);
        if (v.skip) continue;
        phase_gradients<R, MODEL>(d, v.t, state_buf(d, v.cur), sm);
      }
      if (!grid_barrier(bar, lim)) return;
    }
    for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
      const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_ACTIVE);
      if (v.skip) continue;
      if (threadIdx.x == 0) { s_bad = false; s_dt = inf; }
      __syncthreads();
      R* ub = state_buf(d, v.cur);
      phase_flux<R, MODEL, FLUX>(d, v.t, STAGE_BASE, ub, ub, ub, sm, &s_bad, &s_dt);
      if (threadIdx.x == 0) {
        if (s_bad) atomicOr(&d.ctl[v.t.cs].bad, 1);
        atomic_min_dt(&d.ctl[v.t.cs].dtmin, s_dt);
      }
    }
    if (!grid_barrier(bar, lim)) return;
    // ---- dt and U1
    for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
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
        for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
          const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_STAGE);
          if (v.skip) continue;
          phase_gradients<R, MODEL>(d, v.t, stage == 1 ? state_buf(d, v.cur ^ 1) : d.U2, sm);
        }
        if (!grid_barrier(bar, lim)) return;
      }
      for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
        const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_STAGE);
        if (v.skip) continue;
        if (threadIdx.x == 0) { s_bad = false; s_dt = 0; }
        __syncthreads();
        R* ub = state_buf(d, v.cur);
        R* un = state_buf(d, v.cur ^ 1);
        phase_flux<R, MODEL, FLUX>(d, v.t, stage, stage == 1 ? un : d.U2, ub, un, sm, &s_bad, &s_dt);
        if (threadIdx.x == 0 && s_bad) atomicOr(&d.ctl[v.t.cs].bad, 1);
      }
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
// Phase kernels: the same phases as trials_kernel, one kernel per phase and one block per tile,
// for batches large enough to fill the GPU many times over.  A trial is the launch sequence
//   [grad 0] flux 0, first_update, [srd 1], [grad 1], flux 1, [srd 2], [grad 2], flux 2,
//   [srd 3], commit
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

template <class R> __device__ __forceinline__ const R* stage_input(const Dev<R>& d, int stage, int cur) {
  if (stage == STAGE_BASE || stage == STAGE_DIAG) return state_buf(d, cur);
  return stage == STAGE_1 ? state_buf(d, cur ^ 1) : d.U2;
}

template <class R, int MODEL>
__global__ void __launch_bounds__(PHASE_BLOCK, PhaseOcc<R>::grad) phase_grad_kernel(Dev<R> d, int stage) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  const int rule = stage == STAGE_DIAG ? SKIP_LIVE : (stage == STAGE_BASE ? SKIP_ACTIVE : SKIP_STAGE);
  for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
    const TileView v = read_tile(d.tiles, d.ctl, ti, rule);
    if (v.skip) continue;
    phase_gradients<R, MODEL>(d, v.t, stage_input(d, stage, v.cur), sm);
  }
}

template <class R, int MODEL, int FLUX>
__global__ void __launch_bounds__(PHASE_BLOCK, PhaseOcc<R>::flux) phase_flux_kernel(Dev<R> d, int stage) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sm = reinterpret_cast<R*>(smem_raw);
  __shared__ bool s_bad;
  __shared__ double s_dt;
  const int rule = stage == STAGE_DIAG ? SKIP_LIVE : (stage == STAGE_BASE ? SKIP_ACTIVE : SKIP_STAGE);
  for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
    const TileView v = read_tile(d.tiles, d.ctl, ti, rule);
    if (v.skip) continue;
    if (threadIdx.x == 0) { s_bad = false; s_dt = __longlong_as_double(0x7FF0000000000000ll); }
    __syncthreads();
    R* ub = state_buf(d, v.cur);
    R* un = state_buf(d, v.cur ^ 1);
    phase_flux<R, MODEL, FLUX>(d, v.t, stage, stage_input(d, stage, v.cur), ub, un, sm, &s_bad, &s_dt);
    if (threadIdx.x == 0 && stage != STAGE_DIAG) {
      if (s_bad) atomicOr(&d.ctl[v.t.cs].bad, 1);
      if (stage == STAGE_BASE) atomic_min_dt(&d.ctl[v.t.cs].dtmin, s_dt);
    }
  }
}

template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK, 4) phase_first_kernel(Dev<R> d) {
  for (int ti = blockIdx.x; ti < d.n_tiles; ti += gridDim.x) {
    const TileView v = read_tile(d.tiles, d.ctl, ti, SKIP_ACTIVE);
    if (v.skip) continue;
    phase_first_update<R, MODEL>(d, v.t, state_buf(d, v.cur), state_buf(d, v.cur ^ 1));
  }
}

// U1 = U + dt R0, one thread per cell (phase mode).  Every thread derives its case's step size
// from the control record; the first cell of each case records it.
template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK) phase_first_cells_kernel(Dev<R> d, int ncells) {
  const long long n = d.ncap;
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

// stage 1: SRD of U1, stage 2: of U2, stage 3: of the final candidate with the admissibility check.
template <class R, int MODEL>
__global__ void __launch_bounds__(MAX_BLOCK) phase_srd_kernel(Dev<R> d, int stage) {
  for (int cs = blockIdx.x; cs < d.n_cases; cs += gridDim.x) {
    int cur;
    if (read_case_skip(d.ctl, cs, SKIP_STAGE, !d.cfg[cs].has_srd, &cur)) continue;
    R* u = stage == 2 ? d.U2 : state_buf(d, cur ^ 1);
    phase_srd<R, MODEL>(d, cs, u, stage == 3);
  }
}

// Accept/reject the trial (unless begin_only) and begin the next one, one thread per case.
static __global__ void phase_commit_kernel(CaseCtl* ctl, int n_cases, int begin_only) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= n_cases) return;
  CaseCtl& c = ctl[cs];
  if (!begin_only) case_commit(c);
  case_begin(c);
}

// Host-visible launch helpers (defined in amr_engine_f64.cu / amr_engine_f32.cu).
template <class R> struct EngineOps {
  static cudaError_t launch(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int grid, int block,
                            cudaStream_t stream, bool cooperative);
  // One trial (or, with mode MODE_RESIDUAL, one residual evaluation) as a sequence of phase kernels.
  static cudaError_t launch_phases(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int block,
                                   cudaStream_t stream);
  static cudaError_t occupancy(int model, int flux, bool srd, int block, int* blocks_per_sm);
  static size_t smem_bytes(int block) { return size_t(12) * block * sizeof(R); }
};

}  // namespace amrb
