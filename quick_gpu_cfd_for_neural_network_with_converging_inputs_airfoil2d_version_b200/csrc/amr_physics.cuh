// amr_physics.cuh -- point-wise physics of the static-AMR time step, device side.
//
// Templated on the arithmetic type R (double for the plain path, float for the batched
// form).  Every expression keeps the operand order of the reference CPU code it restates,
// so that with R=double and contraction disabled (-fmad=false) each function returns the
// same IEEE double as the reference:
//   numerical fluxes        reference src/flux.h:19-26 (exact), 42-103 (HLLC), 121-176 (AUSM+-up)
//   boundary ghost states   reference src/static_amr2d_boundary.h:50-102
//   viscous pieces          reference src/static_amr2d_viscous.h:52-74
//   SA-neg point model      reference src/sa_model.h:12-39
#pragma once
#include <cfloat>
#include <cmath>
#include <cuda_runtime.h>

namespace amrb {

enum { BC_TRANSMISSIVE = 1, BC_REFLECT = 2, BC_FARFIELD = 3, BC_TOTAL_INLET = 4, BC_PRESSURE_OUTLET = 5, BC_NOSLIP = 6 };
enum { MU_CONSTANT = 0, MU_SUTHERLAND = 1 };

template <class R> __host__ __device__ __forceinline__ R rmin(R a, R b) { return b < a ? b : a; }
template <class R> __host__ __device__ __forceinline__ R rmax(R a, R b) { return a < b ? b : a; }
template <class R> __device__ __forceinline__ R tiny();
template <> __device__ __forceinline__ double tiny<double>() { return 1e-300; }
template <> __device__ __forceinline__ float tiny<float>() { return FLT_MIN; }

// Boundary record in the working precision (copied from the double host record).
template <class R> struct Bnd {
  int kind;
  R ref[4];
  R total_pressure, total_temperature, gas_constant;
  R dir[2];
  R outlet_pressure;
  R wall_velocity[2];
};

template <class R> struct Trn {
  int law;
  R mu_ref, gas_constant, temperature_ref, sutherland, viscous_cfl;
  R sa_nu_inf, sa_cfl;
};

// ---- fluxes -------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void flux_exact(R rho, R un, R ut, R p, R g, R* F) {
  const R E = p / (g - R(1)) + R(0.5) * rho * un * un + R(0.5) * rho * ut * ut;
  F[0] = rho * un;
  F[1] = rho * un * un + p;
  F[2] = rho * un * ut;
  F[3] = un * (E + p);
}

template <class R>
__device__ __forceinline__ void flux_hllc(R rl, R ul, R vl, R pl, R rr, R ur, R vr, R pr, R g, R* F) {
  const R al = sqrt(g * pl / rl), ar = sqrt(g * pr / rr);
  const R el = pl / (g - R(1)) + R(0.5) * rl * ul * ul + R(0.5) * rl * vl * vl;
  const R er = pr / (g - R(1)) + R(0.5) * rr * ur * ur + R(0.5) * rr * vr * vr;
  const R sl = sqrt(rl), sr = sqrt(rr);
  const R hl = (el + pl) / rl, hr = (er + pr) / rr;
  const R ut = (sl * ul + sr * ur) / (sl + sr);
  const R vt = (sl * vl + sr * vr) / (sl + sr);
  const R ht = (sl * hl + sr * hr) / (sl + sr);
  const R at = sqrt(rmax((g - R(1)) * (ht - R(0.5) * ut * ut - R(0.5) * vt * vt), tiny<R>()));
  const R SL = rmin(ul - al, ut - at), SR = rmax(ur + ar, ut + at);
  if (SL >= R(0)) { flux_exact(rl, ul, vl, pl, g, F); return; }
  if (SR <= R(0)) { flux_exact(rr, ur, vr, pr, g, F); return; }
  const R ss = (pr - pl + rl * ul * (SL - ul) - rr * ur * (SR - ur)) / (rl * (SL - ul) - rr * (SR - ur));
  R FS[4];
  if (ss >= R(0)) {
    flux_exact(rl, ul, vl, pl, g, FS);
    const R c = rl * (SL - ul) / (SL - ss);
    const R q3 = c * (el / rl + (ss - ul) * (ss + pl / (rl * (SL - ul))));
    F[0] = FS[0] + SL * (c - rl);
    F[1] = FS[1] + SL * (c * ss - rl * ul);
    F[2] = FS[2] + SL * (c * vl - rl * vl);
    F[3] = FS[3] + SL * (q3 - el);
  } else {
    flux_exact(rr, ur, vr, pr, g, FS);
    const R c = rr * (SR - ur) / (SR - ss);
    const R q3 = c * (er / rr + (ss - ur) * (ss + pr / (rr * (SR - ur))));
    F[0] = FS[0] + SR * (c - rr);
    F[1] = FS[1] + SR * (c * ss - rr * ur);
    F[2] = FS[2] + SR * (c * vr - rr * vr);
    F[3] = FS[3] + SR * (q3 - er);
  }
}

template <class R> __device__ __forceinline__ R ausm_m1(R m, int s) { return R(0.5) * (m + R(s) * fabs(m)); }
template <class R> __device__ __forceinline__ R ausm_m2(R m, int s) { return R(s) * R(0.25) * (m + R(s)) * (m + R(s)); }
template <class R> __device__ __forceinline__ R ausm_m4(R m, int s, R beta) {
  if (fabs(m) >= R(1)) return ausm_m1(m, s);
  return ausm_m2(m, s) * (R(1) - R(s) * R(16) * beta * ausm_m2(m, -s));
}
template <class R> __device__ __forceinline__ R ausm_p5(R m, int s, R alpha) {
  if (fabs(m) >= R(1)) return R(0.5) * (R(1) + R(s) * (m > R(0) ? R(1) : (m < R(0) ? R(-1) : R(0))));
  return ausm_m2(m, s) * ((R(s) * R(2) - m) - R(s) * R(16) * alpha * m * ausm_m2(m, -s));
}

template <class R>
__device__ __forceinline__ void flux_ausmpup(R rl, R ul, R vl, R pl, R rr, R ur, R vr, R pr, R g, R mco, R* F) {
  const R Kp = R(0.25), Ku = R(0.75), sigma = R(1), beta = R(0.125);
  const R al = sqrt(g * pl / rl), ar = sqrt(g * pr / rr);
  const R a12 = R(0.5) * (al + ar), r12 = R(0.5) * (rl + rr);
  const R ml = ul / a12, mr = ur / a12;
  const R mbar2 = R(0.5) * (ul * ul + ur * ur) / (a12 * a12);
  const R m02 = rmin(R(1), rmax(mbar2, mco * mco));
  const R m0 = sqrt(m02);
  const R fa = m0 * (R(2) - m0);
  const R alpha = R(3.0 / 16.0) * (R(-4) + R(5) * fa * fa);
  const R m12 = ausm_m4(ml, +1, beta) + ausm_m4(mr, -1, beta) -
                (Kp / fa) * rmax(R(1) - sigma * mbar2, R(0)) * (pr - pl) / (r12 * a12 * a12);
  const R pp = ausm_p5(ml, +1, alpha), pm = ausm_p5(mr, -1, alpha);
  const R p12 = pp * pl + pm * pr - Ku * pp * pm * (rl + rr) * (fa * a12) * (ur - ul);
  const bool left = m12 > R(0);
  const R rho = left ? rl : rr, u = left ? ul : ur, v = left ? vl : vr, p = left ? pl : pr;
  const R mdot = a12 * m12 * rho;
  const R E = p / (g - R(1)) + R(0.5) * rho * u * u + R(0.5) * rho * v * v;
  const R H = (E + p) / rho;
  F[0] = mdot;
  F[1] = mdot * u + p12;
  F[2] = mdot * v;
  F[3] = mdot * H;
}

// ---- boundary ghost state -----------------------------------------------------------
template <class R> __device__ __forceinline__ bool prim_valid(const R* w) {
  return isfinite(w[0]) && w[0] > R(0) && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]) && w[3] > R(0);
}

// kind is the resolved kind (record kind, or the legacy Params2D kind when the record inherits).
// wi = interior primitive state (rho,u,v,p), wb = exterior state.  Components are addressed by
// explicit selects on the axis so the states stay in registers.
template <class R>
__device__ __forceinline__ bool bc_state(const Bnd<R>& b, int kind, R g, int side, const R wi[4], R wb[4]) {
  const int axis = side / 2;
  const R sign = side % 2 ? R(1) : R(-1), gm = g - R(1);
  const R win = axis ? wi[2] : wi[1];   // normal velocity component
  const R wit = axis ? wi[1] : wi[2];   // tangential velocity component
  wb[0] = wi[0]; wb[1] = wi[1]; wb[2] = wi[2]; wb[3] = wi[3];
  if (kind == BC_TRANSMISSIVE) return true;
  if (kind == BC_NOSLIP) {
    wb[1] = R(2) * b.wall_velocity[0] - wi[1];
    wb[2] = R(2) * b.wall_velocity[1] - wi[2];
    return true;
  }
  if (kind == BC_REFLECT) {
    if (axis) wb[2] = -wi[2]; else wb[1] = -wi[1];
    return true;
  }
  if (!prim_valid(wi) || !(g > R(1))) return false;
  const R ai = sqrt(g * wi[3] / wi[0]), un = sign * win;
  if (kind == BC_TOTAL_INLET) {
    if (!(un < R(0) && un > -ai)) return false;
    const R dn = sign * (axis ? b.dir[1] : b.dir[0]), A = g * b.gas_constant * b.total_temperature;
    if (!(dn < R(0)) || !isfinite(A)) return false;
    const R rp = un + R(2) * ai / gm, upper = sqrt(R(2) * A / (gm + R(2) * dn * dn));
    const R f0 = R(2) * sqrt(A) / gm - rp;
    const R f1 = dn * upper + R(2) * sqrt(A - R(0.5) * gm * upper * upper) / gm - rp;
    if (!(f0 >= R(0) && f1 <= R(0))) return false;
    R lo = 0, hi = upper;
    for (int it = 0; it < 64; ++it) {  // fixed-count bisection (64 halvings)
      const R v = R(0.5) * (lo + hi), a = sqrt(A - R(0.5) * gm * v * v);
      if (dn * v + R(2) * a / gm > rp) lo = v; else hi = v;
    }
    const R v = R(0.5) * (lo + hi), temp = (A - R(0.5) * gm * v * v) / (g * b.gas_constant);
    const R pressure = b.total_pressure * pow(temp / b.total_temperature, g / gm);
    wb[0] = pressure / (b.gas_constant * temp);
    wb[1] = v * b.dir[0];
    wb[2] = v * b.dir[1];
    wb[3] = pressure;
    return prim_valid(wb);
  }
  if (kind == BC_PRESSURE_OUTLET && un >= R(0)) {
    if (un >= ai) return true;
    const R density = wi[0] * pow(b.outlet_pressure / wi[3], R(1) / g);
    const R ab = sqrt(g * b.outlet_pressure / density), ub = un + R(2) * (ai - ab) / gm;
    if (ub >= R(0)) {
      wb[0] = density;
      if (axis) wb[2] = sign * ub; else wb[1] = sign * ub;
      wb[3] = b.outlet_pressure;
      return prim_valid(wb);
    }
  }
  if (kind != BC_FARFIELD && kind != BC_PRESSURE_OUTLET) return false;
  if (un >= ai) return true;
  if (un <= -ai) {
    wb[0] = b.ref[0]; wb[1] = b.ref[1]; wb[2] = b.ref[2]; wb[3] = b.ref[3];
    return prim_valid(wb);
  }
  const R refn = axis ? b.ref[2] : b.ref[1], reft = axis ? b.ref[1] : b.ref[2];
  const R ar = sqrt(g * b.ref[3] / b.ref[0]);
  const R rp = un + R(2) * ai / gm, rm = sign * refn - R(2) * ar / gm;
  const R ab = R(0.25) * gm * (rp - rm), ub = R(0.5) * (rp + rm);
  if (!(ab > R(0)) || !isfinite(ab)) return false;
  const R advrho = un >= R(0) ? wi[0] : b.ref[0], advp = un >= R(0) ? wi[3] : b.ref[3];
  const R advt = un >= R(0) ? wit : reft;
  const R entropy = advp / pow(advrho, g);
  wb[0] = pow(ab * ab / (g * entropy), R(1) / gm);
  wb[3] = entropy * pow(wb[0], g);
  if (axis) { wb[2] = sign * ub; wb[1] = advt; } else { wb[1] = sign * ub; wb[2] = advt; }
  return prim_valid(wb);
}

// ---- viscous pieces -------------------------------------------------------------------
template <class R> __device__ __forceinline__ R dyn_visc(const Trn<R>& t, R temperature) {
  if (!(temperature > R(0)) || !isfinite(temperature)) return R(-1);
  if (t.law == MU_CONSTANT) return t.mu_ref;
  const R ratio = temperature / t.temperature_ref;
  return t.mu_ref * ratio * sqrt(ratio) * (t.temperature_ref + t.sutherland) / (temperature + t.sutherland);
}

template <class R>
__device__ __forceinline__ void visc_flux(R mu, const R* g, R nx, R ny, R u, R v, R* f) {
  const R dil = R(2.0 / 3) * (g[0] + g[3]);
  const R s0 = mu * (R(2) * g[0] - dil), s1 = mu * (g[1] + g[2]), s2 = mu * (R(2) * g[3] - dil);
  f[0] = 0;
  f[1] = s0 * nx + s1 * ny;
  f[2] = s1 * nx + s2 * ny;
  f[3] = u * f[1] + v * f[2];
}

template <class R>
__device__ __forceinline__ void correct_gradient(const R* l, const R* r, R dx, R dy, R du, R dv, R* g) {
  const R d2 = dx * dx + dy * dy;
  for (int q = 0; q < 4; ++q) g[q] = R(0.5) * (l[q] + r[q]);
  const R cu = (du - g[0] * dx - g[1] * dy) / d2, cv = (dv - g[2] * dx - g[3] * dy) / d2;
  g[0] += cu * dx; g[1] += cu * dy; g[2] += cv * dx; g[3] += cv * dy;
}

template <class R>
__device__ __forceinline__ void wall_gradient(R nx, R ny, R d, R du, R dv, R* g) {
  g[0] = nx * du / d; g[1] = ny * du / d; g[2] = nx * dv / d; g[3] = ny * dv / d;
}

// ---- SA-neg ------------------------------------------------------------------------------
// Model constants (NASA TMR SA-neg with ft2 and the Note 1c modified vorticity).
#define AMRB_CB1 0.1355
#define AMRB_CB2 0.622
#define AMRB_SIG (2.0 / 3)
#define AMRB_KAP 0.41
#define AMRB_CW1 (AMRB_CB1 / (AMRB_KAP * AMRB_KAP) + (1 + AMRB_CB2) / AMRB_SIG)

template <class R> struct SaPoint { R source, source_rate, diffusion; };

template <class R> __device__ __forceinline__ R sa_eddy(R working, R molecular) {
  if (working <= R(0)) return R(0);
  const R chi = working / molecular, cube = chi * chi * chi;
  return working * cube / (cube + R(7.1 * 7.1 * 7.1));
}

template <class R> __device__ __forceinline__ SaPoint<R> sa_neg(R working, R molecular, R distance, R omega) {
  const R cb1 = R(AMRB_CB1), sig = R(AMRB_SIG), kap = R(AMRB_KAP), cw1 = R(AMRB_CW1);
  SaPoint<R> a;
  const R chi = working / molecular, cube = chi * chi * chi, d2 = distance * distance;
  if (working < R(0)) {
    const R fn = (R(16) + cube) / (R(16) - cube);
    a.diffusion = (molecular + working * fn) / sig;
    a.source = cb1 * (R(1) - R(1.2)) * omega * working + cw1 * working * working / d2;
    a.source_rate = cb1 * R(.2) * omega + R(2) * cw1 * fabs(working) / d2;
    return a;
  }
  const R fv1 = cube / (cube + R(7.1 * 7.1 * 7.1));
  const R fv2 = R(1) - chi / (R(1) + chi * fv1);
  const R sbar = working * fv2 / (kap * kap * d2);
  const R mod = sbar >= R(-.7) * omega ? omega + sbar : omega * ((R(-.01) * omega - R(.1) * sbar) / (R(-.5) * omega - sbar));
  const R r = mod == R(0) ? R(10) : fmin(working / (mod * kap * kap * d2), R(10));
  const R r6 = r * r * r * r * r * r, gg = r + R(.3) * (r6 - r), g6 = gg * gg * gg * gg * gg * gg;
  const R fw = gg * pow(R(65) / (g6 + R(64)), R(1.0 / 6));
  const R ft2 = R(1.2) * exp(R(-.5) * chi * chi);
  const R production = cb1 * (R(1) - ft2) * mod, destruction = cw1 * fw - cb1 * ft2 / (kap * kap);
  a.source = production * working - destruction * working * working / d2;
  a.source_rate = fabs(production) + R(2) * fabs(destruction) * working / d2;
  a.diffusion = (molecular + working) / sig;
  return a;
}

template <class R>
__device__ __forceinline__ R sa_corrected_source(const SaPoint<R>& a, R rho, R gx, R gy, R rx, R ry) {
  return rho * (a.source + R(AMRB_CB2 / AMRB_SIG) * (gx * gx + gy * gy)) - a.diffusion * (rx * gx + ry * gy);
}

}  // namespace amrb
