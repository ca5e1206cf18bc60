/* amr_oracle.c -- TEST INFRASTRUCTURE: the CPU oracle of the static-AMR explicit time step.
 *
 * A restatement in plain C of the reference CPU integrator, written against the flat mesh
 * view of include/amr_b200.h.  It is the checker for the CUDA engine: only tests/, the smoke
 * check and the CPU-baseline leg of bench.py call it.  Every floating-point expression keeps
 * the reference's evaluation order (left-to-right, no contraction: built with
 * -ffp-contract=off), so on the same mesh it reproduces the reference CPU state bit for bit
 * (pinned by tests/test_oracle.py against oracle/_ref/libamr_ref.so).
 *
 * Reference map (paths inside the reference project):
 *   flux_euler_exact / flux_hllc / flux_ausmpup   src/flux.h:19-26, 42-103, 121-176
 *   bc_valid / bc_state                           src/static_amr2d_boundary.h:32-102
 *   dynamic_viscosity, stress, viscous_flux,
 *   correct_gradient, wall_gradient               src/static_amr2d_viscous.h:52-74
 *   sa_eddy / sa_neg_point / sa_corrected_source  src/sa_model.h:15-39
 *   primitive                                     src/static_amr2d.cpp:143-154
 *   residual (face sweep, gather, coupling)       src/static_amr2d.cpp:156-206
 *   viscous_evaluate                              src/static_amr2d_viscous.cpp:161-220
 *   sa_evaluate                                   src/static_amr2d_sa.cpp:70-98
 *   redistribute (SRD)                            src/static_amr2d.cpp:208-226
 *   run (dt, SSP-RK3, retries)                    src/static_amr2d.cpp:384-432
 *   diagnostics (norms, loads)                    src/quick_airfoil.cpp:189-199
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "amr_b200.h"

/* std::min / std::max semantics (return the first argument on ties and NaN-free inputs). */
static double mn(double a, double b) { return b < a ? b : a; }
static double mx(double a, double b) { return a < b ? b : a; }

/* ---- fluxes (src/flux.h) ------------------------------------------------------------ */
static void flux_exact(double rho, double un, double ut, double p, double g, double* F) {
  const double E = p / (g - 1.0) + 0.5 * rho * un * un + 0.5 * rho * ut * ut;
  F[0] = rho * un;
  F[1] = rho * un * un + p;
  F[2] = rho * un * ut;
  F[3] = un * (E + p);
}

static void flux_hllc(double rl, double ul, double vl, double pl, double rr, double ur, double vr,
                      double pr, double g, double* F) {
  const double al = sqrt(g * pl / rl), ar = sqrt(g * pr / rr);
  const double el = pl / (g - 1.0) + 0.5 * rl * ul * ul + 0.5 * rl * vl * vl;
  const double er = pr / (g - 1.0) + 0.5 * rr * ur * ur + 0.5 * rr * vr * vr;
  const double sl = sqrt(rl), sr = sqrt(rr);
  const double hl = (el + pl) / rl, hr = (er + pr) / rr;
  const double ut = (sl * ul + sr * ur) / (sl + sr);
  const double vt = (sl * vl + sr * vr) / (sl + sr);
  const double ht = (sl * hl + sr * hr) / (sl + sr);
  const double at = sqrt(mx((g - 1.0) * (ht - 0.5 * ut * ut - 0.5 * vt * vt), 1e-300));
  const double SL = mn(ul - al, ut - at), SR = mx(ur + ar, ut + at);
  double FL[4], FR[4];
  flux_exact(rl, ul, vl, pl, g, FL);
  flux_exact(rr, ur, vr, pr, g, FR);
  if (SL >= 0.0) { memcpy(F, FL, sizeof FL); return; }
  if (SR <= 0.0) { memcpy(F, FR, sizeof FR); return; }
  const double ss = (pr - pl + rl * ul * (SL - ul) - rr * ur * (SR - ur)) / (rl * (SL - ul) - rr * (SR - ur));
  if (ss >= 0.0) {
    const double c = rl * (SL - ul) / (SL - ss);
    const double q3 = c * (el / rl + (ss - ul) * (ss + pl / (rl * (SL - ul))));
    F[0] = FL[0] + SL * (c - rl);
    F[1] = FL[1] + SL * (c * ss - rl * ul);
    F[2] = FL[2] + SL * (c * vl - rl * vl);
    F[3] = FL[3] + SL * (q3 - el);
  } else {
    const double c = rr * (SR - ur) / (SR - ss);
    const double q3 = c * (er / rr + (ss - ur) * (ss + pr / (rr * (SR - ur))));
    F[0] = FR[0] + SR * (c - rr);
    F[1] = FR[1] + SR * (c * ss - rr * ur);
    F[2] = FR[2] + SR * (c * vr - rr * vr);
    F[3] = FR[3] + SR * (q3 - er);
  }
}

static double ausm_m1(double m, int s) { return 0.5 * (m + s * fabs(m)); }
static double ausm_m2(double m, int s) { return s * 0.25 * (m + s) * (m + s); }
static double ausm_m4(double m, int s, double beta) {
  if (fabs(m) >= 1.0) return ausm_m1(m, s);
  return ausm_m2(m, s) * (1.0 - s * 16.0 * beta * ausm_m2(m, -s));
}
static double ausm_p5(double m, int s, double alpha) {
  if (fabs(m) >= 1.0) return 0.5 * (1.0 + s * (m > 0.0 ? 1.0 : (m < 0.0 ? -1.0 : 0.0)));
  return ausm_m2(m, s) * ((s * 2.0 - m) - s * 16.0 * alpha * m * ausm_m2(m, -s));
}

static void flux_ausmpup(double rl, double ul, double vl, double pl, double rr, double ur, double vr,
                         double pr, double g, double mco, double* F) {
  const double Kp = 0.25, Ku = 0.75, sigma = 1.0, beta = 0.125;
  const double al = sqrt(g * pl / rl), ar = sqrt(g * pr / rr);
  const double a12 = 0.5 * (al + ar), r12 = 0.5 * (rl + rr);
  const double ml = ul / a12, mr = ur / a12;
  const double mbar2 = 0.5 * (ul * ul + ur * ur) / (a12 * a12);
  const double m02 = mn(1.0, mx(mbar2, mco * mco));
  const double m0 = sqrt(m02);
  const double fa = m0 * (2.0 - m0);
  const double alpha = 3.0 / 16.0 * (-4.0 + 5.0 * fa * fa);
  const double m12 = ausm_m4(ml, +1, beta) + ausm_m4(mr, -1, beta) -
                     (Kp / fa) * mx(1.0 - sigma * mbar2, 0.0) * (pr - pl) / (r12 * a12 * a12);
  const double pp = ausm_p5(ml, +1, alpha), pm = ausm_p5(mr, -1, alpha);
  const double p12 = pp * pl + pm * pr - Ku * pp * pm * (rl + rr) * (fa * a12) * (ur - ul);
  const int left = m12 > 0.0;
  const double mdot = a12 * m12 * (left ? rl : rr);
  const double rho = left ? rl : rr, u = left ? ul : ur, v = left ? vl : vr, p = left ? pl : pr;
  const double E = p / (g - 1.0) + 0.5 * rho * u * u + 0.5 * rho * v * v;
  const double H = (E + p) / rho;
  F[0] = mdot;
  F[1] = mdot * u + p12;
  F[2] = mdot * v;
  F[3] = mdot * H;
}

/* ---- boundary ghost states (src/static_amr2d_boundary.h) ----------------------------- */
static int prim_valid(const double* w) {
  return isfinite(w[0]) && w[0] > 0 && isfinite(w[1]) && isfinite(w[2]) && isfinite(w[3]) && w[3] > 0;
}
static int bc_kind(const amr_boundary_t* b, int legacy) { return b->kind < 0 ? legacy : b->kind; }

static int bc_valid(const amr_boundary_t* b, int legacy, int side) {
  if (b->kind < AMR_B200_BC_INHERIT) return 0;
  const int kind = bc_kind(b, legacy);
  if (kind == AMR_B200_BC_TRANSMISSIVE || kind == AMR_B200_BC_REFLECT) return 1;
  if (kind == AMR_B200_BC_NOSLIP)
    return isfinite(b->wall_velocity[0]) && isfinite(b->wall_velocity[1]) && b->wall_velocity[side / 2] == 0;
  if (kind < AMR_B200_BC_FARFIELD || kind > AMR_B200_BC_PRESSURE_OUTLET || !prim_valid(b->reference)) return 0;
  if (kind == AMR_B200_BC_PRESSURE_OUTLET) return isfinite(b->outlet_pressure) && b->outlet_pressure > 0;
  if (kind == AMR_B200_BC_TOTAL_INLET) {
    const double d2 = b->direction[0] * b->direction[0] + b->direction[1] * b->direction[1];
    const double dn = (side % 2 ? 1.0 : -1.0) * b->direction[side / 2];
    return isfinite(d2) && fabs(d2 - 1) < 1e-12 && dn < 0 && isfinite(b->total_pressure) && b->total_pressure > 0 &&
           isfinite(b->total_temperature) && b->total_temperature > 0 && isfinite(b->gas_constant) && b->gas_constant > 0;
  }
  return 1;
}

static int bc_state(const amr_boundary_t* b, int legacy, double g, int side, const double* wi, double* wb) {
  const int axis = side / 2, normal = axis + 1, tangent = 2 - axis;
  const double sign = side % 2 ? 1.0 : -1.0, gm = g - 1;
  const int kind = bc_kind(b, legacy);
  for (int v = 0; v < 4; ++v) wb[v] = wi[v];
  if (kind == AMR_B200_BC_TRANSMISSIVE) return 1;
  if (kind == AMR_B200_BC_NOSLIP) {
    wb[1] = 2 * b->wall_velocity[0] - wi[1];
    wb[2] = 2 * b->wall_velocity[1] - wi[2];
    return 1;
  }
  if (kind == AMR_B200_BC_REFLECT) { wb[normal] = -wi[normal]; return 1; }
  if (!prim_valid(wi) || !(g > 1)) return 0;
  const double ai = sqrt(g * wi[3] / wi[0]), un = sign * wi[normal];
  if (kind == AMR_B200_BC_TOTAL_INLET) {
    if (!(un < 0 && un > -ai)) return 0;
    const double dn = sign * b->direction[axis], A = g * b->gas_constant * b->total_temperature;
    if (!(dn < 0) || !isfinite(A)) return 0;
    const double rp = un + 2 * ai / gm, upper = sqrt(2 * A / (gm + 2 * dn * dn));
    const double f0 = 2 * sqrt(A) / gm - rp;
    const double f1 = dn * upper + 2 * sqrt(A - .5 * gm * upper * upper) / gm - rp;
    if (!(f0 >= 0 && f1 <= 0)) return 0;
    double lo = 0, hi = upper;
    for (int it = 0; it < 64; ++it) {
      const double v = .5 * (lo + hi), a = sqrt(A - .5 * gm * v * v);
      if (dn * v + 2 * a / gm > rp) lo = v; else hi = v;
    }
    const double v = .5 * (lo + hi), temp = (A - .5 * gm * v * v) / (g * b->gas_constant);
    const double pressure = b->total_pressure * pow(temp / b->total_temperature, g / gm);
    wb[0] = pressure / (b->gas_constant * temp);
    wb[1] = v * b->direction[0];
    wb[2] = v * b->direction[1];
    wb[3] = pressure;
    return prim_valid(wb);
  }
  if (kind == AMR_B200_BC_PRESSURE_OUTLET && un >= 0) {
    if (un >= ai) return 1;
    const double density = wi[0] * pow(b->outlet_pressure / wi[3], 1 / g);
    const double ab = sqrt(g * b->outlet_pressure / density), ub = un + 2 * (ai - ab) / gm;
    if (ub >= 0) {
      wb[0] = density;
      wb[normal] = sign * ub;
      wb[3] = b->outlet_pressure;
      return prim_valid(wb);
    }
  }
  if (kind != AMR_B200_BC_FARFIELD && kind != AMR_B200_BC_PRESSURE_OUTLET) return 0;
  if (un >= ai) return 1;
  if (un <= -ai) { for (int v = 0; v < 4; ++v) wb[v] = b->reference[v]; return prim_valid(wb); }
  const double* wr = b->reference;
  const double ar = sqrt(g * wr[3] / wr[0]);
  const double rp = un + 2 * ai / gm, rm = sign * wr[normal] - 2 * ar / gm;
  const double ab = .25 * gm * (rp - rm), ub = .5 * (rp + rm);
  if (!(ab > 0) || !isfinite(ab)) return 0;
  const double advrho = un >= 0 ? wi[0] : wr[0], advp = un >= 0 ? wi[3] : wr[3];
  const double advt = un >= 0 ? wi[tangent] : wr[tangent];
  const double entropy = advp / pow(advrho, g);
  wb[0] = pow(ab * ab / (g * entropy), 1 / gm);
  wb[3] = entropy * pow(wb[0], g);
  wb[normal] = sign * ub;
  wb[tangent] = advt;
  return prim_valid(wb);
}

/* ---- viscous pieces (src/static_amr2d_viscous.h) -------------------------------------- */
static double dyn_visc(const amr_transport_t* t, double temperature) {
  if (!(temperature > 0) || !isfinite(temperature)) return -1;
  if (t->law == AMR_B200_MU_CONSTANT) return t->mu_ref;
  const double ratio = temperature / t->temperature_ref;
  return t->mu_ref * ratio * sqrt(ratio) * (t->temperature_ref + t->sutherland) / (temperature + t->sutherland);
}
static void visc_flux(double mu, const double* g, double nx, double ny, double u, double v, double* f) {
  const double dil = (2.0 / 3) * (g[0] + g[3]);
  const double s0 = mu * (2 * g[0] - dil), s1 = mu * (g[1] + g[2]), s2 = mu * (2 * g[3] - dil);
  f[0] = 0;
  f[1] = s0 * nx + s1 * ny;
  f[2] = s1 * nx + s2 * ny;
  f[3] = u * f[1] + v * f[2];
}
static void correct_gradient(const double* l, const double* r, double dx, double dy, double du, double dv, double* g) {
  const double d2 = dx * dx + dy * dy;
  for (int q = 0; q < 4; ++q) g[q] = .5 * (l[q] + r[q]);
  const double cu = (du - g[0] * dx - g[1] * dy) / d2, cv = (dv - g[2] * dx - g[3] * dy) / d2;
  g[0] += cu * dx; g[1] += cu * dy; g[2] += cv * dx; g[3] += cv * dy;
}
static void wall_gradient(double nx, double ny, double d, double du, double dv, double* g) {
  g[0] = nx * du / d; g[1] = ny * du / d; g[2] = nx * dv / d; g[3] = ny * dv / d;
}

/* ---- SA-neg (src/sa_model.h) ---------------------------------------------------------- */
static const double cb1 = .1355, cb2 = .622, sig = 2.0 / 3, kap = .41;
#define CW1 (cb1 / (kap * kap) + (1 + cb2) / sig)
typedef struct { double fv1, modified_vorticity, fw, source, source_rate, diffusion; } sa_point_t;

static double sa_eddy(double working, double molecular) {
  if (working <= 0) return 0;
  const double chi = working / molecular, cube = chi * chi * chi;
  return working * cube / (cube + 7.1 * 7.1 * 7.1);
}
static sa_point_t sa_neg(double working, double molecular, double distance, double omega) {
  sa_point_t a;
  memset(&a, 0, sizeof a);
  const double cw1 = CW1;
  const double chi = working / molecular, cube = chi * chi * chi, d2 = distance * distance;
  if (working < 0) {
    const double fn = (16 + cube) / (16 - cube);
    a.diffusion = (molecular + working * fn) / sig;
    a.source = cb1 * (1 - 1.2) * omega * working + cw1 * working * working / d2;
    a.source_rate = cb1 * .2 * omega + 2 * cw1 * fabs(working) / d2;
    return a;
  }
  a.fv1 = cube / (cube + 7.1 * 7.1 * 7.1);
  const double fv2 = 1 - chi / (1 + chi * a.fv1);
  const double sbar = working * fv2 / (kap * kap * d2);
  a.modified_vorticity = sbar >= -.7 * omega ? omega + sbar : omega * ((-.01 * omega - .1 * sbar) / (-.5 * omega - sbar));
  const double r = a.modified_vorticity == 0 ? 10 : fmin(working / (a.modified_vorticity * kap * kap * d2), 10.);
  const double r6 = r * r * r * r * r * r, gg = r + .3 * (r6 - r), g6 = gg * gg * gg * gg * gg * gg;
  a.fw = gg * pow(65 / (g6 + 64), 1.0 / 6);
  const double ft2 = 1.2 * exp(-.5 * chi * chi);
  const double production = cb1 * (1 - ft2) * a.modified_vorticity, destruction = cw1 * a.fw - cb1 * ft2 / (kap * kap);
  a.source = production * working - destruction * working * working / d2;
  a.source_rate = fabs(production) + 2 * fabs(destruction) * working / d2;
  a.diffusion = (molecular + working) / sig;
  return a;
}
static double sa_corrected_source(const sa_point_t* a, double rho, double gx, double gy, double rx, double ry) {
  return rho * (a->source + cb2 / sig * (gx * gx + gy * gy)) - a->diffusion * (rx * gx + ry * gy);
}

/* ---- workspace --------------------------------------------------------------------- */
typedef struct {
  const amr_mesh_view_t* m;
  const amr_params_t* p;
  size_t n, nf, nw, nv;
  double *w, *flux, *speed, *r;
  /* viscous */
  double *grad, *mu, *vface, *vwall, *vres, *vdt, *fc, *wc, *eddy;
  /* SA */
  double *phi, *sgrad, *dgrad, *sdiff, *ssrc, *srate, *sface, *swall, *sres, *sdt, *sfc, *swc;
  /* SRD */
  double *qhat, *tmp;
} ws_t;

static int face_kind(const ws_t* s, int side) { return bc_kind(&s->m->boundaries[side], s->p->bc[side]); }

static int primitive(const ws_t* s, const double* u) {
  const size_t n = s->n;
  int bad = 0;
  for (size_t k = 0; k < n; ++k) {
    const double rho = u[k], mxv = u[n + k], myv = u[2 * n + k], energy = u[3 * n + k];
    if (!isfinite(rho) || !(rho > 0) || !isfinite(mxv) || !isfinite(myv) || !isfinite(energy)) { bad = 1; continue; }
    const double vx = mxv / rho, vy = myv / rho, p = (s->p->gamma - 1) * (energy - 0.5 * (mxv * vx + myv * vy));
    if (!isfinite(p) || !(p > 0)) { bad = 1; continue; }
    s->w[k] = rho; s->w[n + k] = vx; s->w[2 * n + k] = vy; s->w[3 * n + k] = p;
  }
  return !bad;
}

/* src/static_amr2d_viscous.cpp:161-220; needs s->w (and u for SA). Returns 0 on success. */
static int viscous_evaluate(ws_t* s, const double* u) {
  const amr_mesh_view_t* m = s->m;
  const amr_transport_t* t = &m->transport;
  const size_t n = s->n, nf = s->nf, nw = s->nw;
  const double* w = s->w;
  int bad = 0;
  memset(s->grad, 0, 4 * n * sizeof(double));
  memset(s->eddy, 0, n * sizeof(double));
  for (size_t k = 0; k < n; ++k) {
    s->mu[k] = dyn_visc(t, w[3 * n + k] / (w[k] * t->gas_constant));
    if (!(s->mu[k] > 0) || !isfinite(s->mu[k])) bad = 1;
    if (t->sa_model) {
      const double ph = u[4 * n + k] / w[k];
      if (!isfinite(ph)) { bad = 1; continue; }
      s->eddy[k] = w[k] * sa_eddy(ph, s->mu[k] / w[k]);
    }
    for (uint64_t q = m->visc_offsets[k]; q < m->visc_offsets[k + 1]; ++q) {
      const amr_gradient_term_t* term = &m->visc_terms[q];
      double uu = 0, vv = 0;
      if (term->source >= 0) { uu = w[n + term->source]; vv = w[2 * n + term->source]; }
      else if (term->source == -2) { uu = m->boundaries[term->side].wall_velocity[0]; vv = m->boundaries[term->side].wall_velocity[1]; }
      const double du = uu - w[n + k], dv = vv - w[2 * n + k];
      s->grad[k] += term->x * du; s->grad[n + k] += term->y * du;
      s->grad[2 * n + k] += term->x * dv; s->grad[3 * n + k] += term->y * dv;
    }
  }
  if (bad) return 1;
  for (size_t q = 0; q < nf; ++q) {
    const amr_face_t* f = &m->faces[q];
    const amr_face_geometry_t* geo = &m->face_geometry[q];
    const int k = f->left >= 0 ? f->left : f->right;
    double g[4], mu = s->mu[k] + s->eddy[k], uf = w[n + k], vf = w[2 * n + k], nu = mu / w[k], distance = geo->distance;
    for (int v = 0; v < 4; ++v) g[v] = s->grad[v * n + k];
    if (f->boundary < 0) {
      const int l = f->left, r = f->right;
      double gl[4], gr[4];
      for (int v = 0; v < 4; ++v) { gl[v] = s->grad[v * n + l]; gr[v] = s->grad[v * n + r]; }
      correct_gradient(gl, gr, geo->dx, geo->dy, w[n + r] - w[n + l], w[2 * n + r] - w[2 * n + l], g);
      uf = .5 * (w[n + l] + w[n + r]) + g[0] * geo->ex + g[1] * geo->ey;
      vf = .5 * (w[2 * n + l] + w[2 * n + r]) + g[2] * geo->ex + g[3] * geo->ey;
      const double temp = .5 * (w[3 * n + l] / w[l] + w[3 * n + r] / w[r]) / t->gas_constant;
      mu = dyn_visc(t, temp) + .5 * (s->eddy[l] + s->eddy[r]);
      nu = mx((s->mu[l] + s->eddy[l]) / w[l], (s->mu[r] + s->eddy[r]) / w[r]);
    } else {
      distance = m->face_samples[q].distance;
      const int bc = face_kind(s, f->boundary);
      const double sign = f->boundary % 2 ? 1 : -1;
      if (bc == AMR_B200_BC_NOSLIP) {
        mu = s->mu[k];
        uf = m->boundaries[f->boundary].wall_velocity[0];
        vf = m->boundaries[f->boundary].wall_velocity[1];
        wall_gradient(f->axis == 0 ? sign : 0, f->axis == 1 ? sign : 0, distance, uf - w[n + k], vf - w[2 * n + k], g);
      } else if (bc == AMR_B200_BC_REFLECT) {
        g[1] = 0; g[2] = 0;
        if (f->axis == 0) uf = 0; else vf = 0;
      } else {
        g[f->axis] = 0; g[2 + f->axis] = 0;
        uf += g[0] * geo->ex + g[1] * geo->ey;
        vf += g[2] * geo->ex + g[3] * geo->ey;
      }
    }
    double fl[4];
    visc_flux(mu, g, f->axis == 0 ? 1 : 0, f->axis == 1 ? 1 : 0, uf, vf, fl);
    for (int v = 0; v < 4; ++v) { s->vface[v * nf + q] = fl[v] * f->length; if (!isfinite(fl[v])) bad = 1; }
    s->fc[q] = (4.0 / 3) * nu / distance;
  }
  for (size_t q = 0; q < nw; ++q) {
    const amr_wall_t* wall = &m->walls[q];
    const amr_wall_sample_t* sm = &m->wall_samples[q];
    const int k = sm->donor, owner = (int)wall->owner_cell;
    double g[4], fl[4];
    wall_gradient(wall->nx, wall->ny, sm->distance, -w[n + k], -w[2 * n + k], g);
    visc_flux(s->mu[k], g, wall->nx, wall->ny, 0, 0, fl);
    for (int v = 0; v < 4; ++v) { s->vwall[v * nw + q] = fl[v] * wall->length; if (!isfinite(fl[v])) bad = 1; }
    s->wc[q] = (4.0 / 3) * mx(s->mu[k] / w[k], s->mu[owner] / w[owner]) / sm->distance;
  }
  if (bad) return 1;
  for (size_t k = 0; k < n; ++k) {
    const amr_cell_t* c = &m->cells[k];
    double sum[4] = {0, 0, 0, 0}, spectral = 0;
    for (uint64_t pos = m->face_offsets[k]; pos < m->face_offsets[k + 1]; ++pos) {
      const uint64_t q = m->cell_faces[pos];
      const double sign = m->faces[q].left == (int)k ? 1 : -1;
      for (int v = 0; v < 4; ++v) sum[v] += sign * s->vface[v * nf + q];
      spectral += s->fc[q] * m->faces[q].length;
    }
    for (uint64_t q = c->wall_begin; q < c->wall_begin + c->wall_count; ++q) {
      for (int v = 0; v < 4; ++v) sum[v] += s->vwall[v * nw + q];
      spectral += s->wc[q] * m->walls[q].length;
    }
    for (int v = 0; v < 4; ++v) s->vres[v * n + k] = sum[v] / c->volume;
    s->vdt[k] = spectral > 0 ? t->viscous_cfl * c->volume / spectral : INFINITY;
  }
  if (t->stabilization == AMR_B200_VISCOUS_SRD && m->small_cells) {
    double* rates = s->tmp;
    double* groups = s->qhat;
    for (size_t k = 0; k < n; ++k) rates[k] = t->viscous_cfl / s->vdt[k];
    for (size_t gi = 0; gi < n; ++gi) {
      double sum = 0;
      for (uint64_t pos = m->group_offsets[gi]; pos < m->group_offsets[gi + 1]; ++pos) {
        const uint64_t k = m->group_members[pos];
        sum += m->cells[k].volume * rates[k] / (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
      }
      groups[gi] = sum / m->group_volume[gi];
    }
    for (size_t k = 0; k < n; ++k) {
      double sum = 0;
      for (uint64_t pos = m->member_offsets[k]; pos < m->member_offsets[k + 1]; ++pos) sum += groups[m->member_groups[pos]];
      const double rate = sum / (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
      s->vdt[k] = rate > 0 ? t->viscous_cfl / rate : INFINITY;
    }
  }
  return 0;
}

/* src/static_amr2d_sa.cpp:70-98; meanflux = convective minus viscous face flux. */
static int sa_evaluate(ws_t* s, const double* u, const double* meanflux) {
  const amr_mesh_view_t* m = s->m;
  const amr_transport_t* t = &m->transport;
  const size_t n = s->n, nf = s->nf, nw = s->nw;
  const double* w = s->w;
  memset(s->sgrad, 0, 2 * n * sizeof(double));
  memset(s->dgrad, 0, 2 * n * sizeof(double));
  for (size_t k = 0; k < n; ++k) { s->phi[k] = u[4 * n + k] / w[k]; if (!isfinite(s->phi[k])) return 1; }
  for (size_t k = 0; k < n; ++k) {
    for (uint64_t q = m->visc_offsets[k]; q < m->visc_offsets[k + 1]; ++q) {
      const amr_gradient_term_t* tm = &m->visc_terms[q];
      const double ph = tm->source >= 0 ? s->phi[tm->source] : 0, rho = tm->source >= 0 ? w[tm->source] : w[k];
      s->sgrad[k] += tm->x * (ph - s->phi[k]); s->sgrad[n + k] += tm->y * (ph - s->phi[k]);
      s->dgrad[k] += tm->x * (rho - w[k]); s->dgrad[n + k] += tm->y * (rho - w[k]);
    }
    const sa_point_t a = sa_neg(s->phi[k], s->mu[k] / w[k], m->wall_distance[k], fabs(s->grad[2 * n + k] - s->grad[n + k]));
    s->sdiff[k] = a.diffusion;
    s->srate[k] = a.source_rate;
    s->ssrc[k] = sa_corrected_source(&a, w[k], s->sgrad[k], s->sgrad[n + k], s->dgrad[k], s->dgrad[n + k]);
    if (!(s->sdiff[k] > 0) || !isfinite(s->ssrc[k]) || !isfinite(s->srate[k])) return 1;
  }
  for (size_t q = 0; q < nf; ++q) {
    const amr_face_t* f = &m->faces[q];
    const amr_face_geometry_t* geo = &m->face_geometry[q];
    const int inside = f->left >= 0 ? f->left : f->right;
    const double mass = meanflux[q];
    const double left = f->left >= 0 ? s->phi[f->left] : t->sa_nu_inf, right = f->right >= 0 ? s->phi[f->right] : t->sa_nu_inf;
    double diff = 0, coefficient = 0;
    if (f->boundary < 0) {
      const int l = f->left, r = f->right;
      const double gl[4] = {s->sgrad[l], s->sgrad[n + l], 0, 0}, gr[4] = {s->sgrad[r], s->sgrad[n + r], 0, 0};
      double g[4];
      correct_gradient(gl, gr, geo->dx, geo->dy, s->phi[r] - s->phi[l], 0, g);
      coefficient = .5 * (w[l] * s->sdiff[l] + w[r] * s->sdiff[r]);
      diff = coefficient * g[f->axis] * f->length;
      s->sfc[q] = coefficient / geo->distance * f->length;
    } else {
      const int bc = face_kind(s, f->boundary);
      const int inflow = f->left < 0 ? mass > 0 : mass < 0;
      const double sign = f->boundary % 2 ? 1 : -1;
      if (bc == AMR_B200_BC_NOSLIP || inflow) {
        const double wall = bc == AMR_B200_BC_NOSLIP ? 0 : t->sa_nu_inf;
        coefficient = bc == AMR_B200_BC_NOSLIP ? s->mu[inside] / sig : w[inside] * s->sdiff[inside];
        diff = sign * coefficient * (wall - s->phi[inside]) / m->face_samples[q].distance * f->length;
        s->sfc[q] = coefficient / m->face_samples[q].distance * f->length;
      } else {
        s->sfc[q] = 0;
      }
    }
    s->sface[q] = mass * (mass >= 0 ? left : right) - diff;
  }
  for (size_t q = 0; q < nw; ++q) {
    const amr_wall_sample_t* sm = &m->wall_samples[q];
    const int k = sm->donor;
    s->swc[q] = s->mu[k] / sig / sm->distance * m->walls[q].length;
    s->swall[q] = -s->swc[q] * s->phi[k];
  }
  for (size_t k = 0; k < n; ++k) {
    const amr_cell_t* c = &m->cells[k];
    double net = 0, spectral = 0;
    for (uint64_t pos = m->face_offsets[k]; pos < m->face_offsets[k + 1]; ++pos) {
      const uint64_t q = m->cell_faces[pos];
      net += (m->faces[q].left == (int)k ? 1 : -1) * s->sface[q];
      spectral += s->sfc[q];
    }
    for (uint64_t q = c->wall_begin; q < c->wall_begin + c->wall_count; ++q) { net -= s->swall[q]; spectral += s->swc[q]; }
    s->sres[k] = -net / c->volume + s->ssrc[k];
    const double rate = 2 * spectral / (w[k] * c->volume) + s->srate[k];
    s->sdt[k] = rate > 0 ? t->sa_cfl / rate : INFINITY;
    if (!isfinite(s->sres[k])) return 1;
  }
  return 0;
}

/* src/static_amr2d.cpp:156-206.  Fills s->r (nv*n), s->w, s->flux, s->speed; with_dt also
 * fills s->vdt with min(viscous dt, SA dt).  Returns 1 on success. */
static int residual(ws_t* s, const double* u) {
  const amr_mesh_view_t* m = s->m;
  const amr_params_t* p = s->p;
  const size_t n = s->n, nf = s->nf;
  if (!primitive(s, u)) return 0;
  int bad = 0;
  for (size_t q = 0; q < nf; ++q) {
    const amr_face_t* f = &m->faces[q];
    const int inside = f->left >= 0 ? f->left : f->right;
    double a[4], b[4];
    for (int v = 0; v < 4; ++v) {
      a[v] = s->w[v * n + (f->left >= 0 ? f->left : inside)];
      b[v] = s->w[v * n + (f->right >= 0 ? f->right : inside)];
    }
    if (f->boundary >= 0) {
      double* outside = f->left < 0 ? a : b;
      const double* interior = f->left < 0 ? b : a;
      if (!bc_state(&m->boundaries[f->boundary], p->bc[f->boundary], p->gamma, f->boundary, interior, outside)) { bad = 1; continue; }
    }
    const int normal = 1 + f->axis, tangent = 2 - f->axis;
    double local[4];
    const int bc = f->boundary < 0 ? -1 : face_kind(s, f->boundary);
    if (bc == AMR_B200_BC_NOSLIP) { local[0] = 0; local[1] = s->w[3 * n + inside]; local[2] = 0; local[3] = 0; }
    else if (p->flux == AMR_B200_FLUX_HLLC) flux_hllc(a[0], a[normal], a[tangent], a[3], b[0], b[normal], b[tangent], b[3], p->gamma, local);
    else flux_ausmpup(a[0], a[normal], a[tangent], a[3], b[0], b[normal], b[tangent], b[3], p->gamma, p->ausm_mco, local);
    s->flux[q] = local[0] * f->length;
    s->flux[normal * nf + q] = local[1] * f->length;
    s->flux[tangent * nf + q] = local[2] * f->length;
    s->flux[3 * nf + q] = local[3] * f->length;
    s->speed[q] = mx(fabs(a[normal]) + sqrt(p->gamma * a[3] / a[0]), fabs(b[normal]) + sqrt(p->gamma * b[3] / b[0]));
    for (int v = 0; v < 4; ++v) if (!isfinite(local[v])) bad = 1;
  }
  if (bad) return 0;
  for (size_t k = 0; k < n; ++k) {
    const amr_cell_t* c = &m->cells[k];
    double sum[4] = {0, 0, 0, 0};
    for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q) {
      const uint64_t face = m->cell_faces[q];
      const double sign = m->faces[face].left == (int)k ? 1.0 : -1.0;
      for (int v = 0; v < 4; ++v) sum[v] += sign * s->flux[v * nf + face];
    }
    for (uint64_t q = c->wall_begin; q < c->wall_begin + c->wall_count; ++q) {
      const amr_wall_t* wall = &m->walls[q];
      sum[1] += s->w[3 * n + k] * wall->nx * wall->length;
      sum[2] += s->w[3 * n + k] * wall->ny * wall->length;
    }
    for (int v = 0; v < 4; ++v) s->r[v * n + k] = -sum[v] / c->volume;
  }
  if (m->transport.model == AMR_B200_MODEL_LAMINAR) {
    if (viscous_evaluate(s, u)) return 0;
    for (size_t q = 0; q < 4 * n; ++q) s->r[q] += s->vres[q];
    for (size_t q = 0; q < 4 * nf; ++q) s->flux[q] -= s->vface[q];
    if (m->transport.sa_model) {
      if (sa_evaluate(s, u, s->flux)) return 0;
      for (size_t k = 0; k < n; ++k) { s->r[4 * n + k] = s->sres[k]; s->vdt[k] = mn(s->vdt[k], s->sdt[k]); }
    }
  }
  return 1;
}

/* src/static_amr2d.cpp:208-226, first four variables, in place. */
static void redistribute(ws_t* s, double* u) {
  const amr_mesh_view_t* m = s->m;
  if (m->small_cells == 0) return;
  const size_t n = s->n;
  for (size_t g = 0; g < n; ++g)
    for (int v = 0; v < 4; ++v) {
      double sum = 0;
      for (uint64_t q = m->group_offsets[g]; q < m->group_offsets[g + 1]; ++q) {
        const uint64_t k = m->group_members[q];
        sum += m->cells[k].volume * u[v * n + k] / (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
      }
      s->qhat[v * n + g] = sum / m->group_volume[g];
    }
  for (size_t k = 0; k < n; ++k)
    for (int v = 0; v < 4; ++v) {
      double sum = 0;
      for (uint64_t q = m->member_offsets[k]; q < m->member_offsets[k + 1]; ++q) sum += s->qhat[v * n + m->member_groups[q]];
      s->tmp[v * n + k] = sum / (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
    }
  memcpy(u, s->tmp, 4 * n * sizeof(double));
}

static int ws_init(ws_t* s, const amr_mesh_view_t* m, const amr_params_t* p) {
  memset(s, 0, sizeof *s);
  s->m = m; s->p = p;
  s->n = m->n_cells; s->nf = m->n_faces; s->nw = m->n_walls;
  s->nv = m->transport.sa_model ? 5 : 4;
  const size_t n = s->n, nf = s->nf, nw = s->nw ? s->nw : 1;
  double** bufs[] = {&s->w, &s->flux, &s->speed, &s->r, &s->grad, &s->mu, &s->vface, &s->vwall, &s->vres, &s->vdt,
                     &s->fc, &s->wc, &s->eddy, &s->phi, &s->sgrad, &s->dgrad, &s->sdiff, &s->ssrc, &s->srate,
                     &s->sface, &s->swall, &s->sres, &s->sdt, &s->sfc, &s->swc, &s->qhat, &s->tmp};
  const size_t sizes[] = {4 * n, 4 * nf, nf, 5 * n, 4 * n, n, 4 * nf, 4 * nw, 4 * n, n,
                          nf, nw, n, n, 2 * n, 2 * n, n, n, n,
                          nf, nw, n, n, nf, nw, 4 * n, 5 * n};
  for (size_t i = 0; i < sizeof sizes / sizeof sizes[0]; ++i) {
    *bufs[i] = (double*)calloc(sizes[i] ? sizes[i] : 1, sizeof(double));
    if (!*bufs[i]) return 1;
  }
  return 0;
}

static void ws_free(ws_t* s) {
  double* bufs[] = {s->w, s->flux, s->speed, s->r, s->grad, s->mu, s->vface, s->vwall, s->vres, s->vdt, s->fc, s->wc,
                    s->eddy, s->phi, s->sgrad, s->dgrad, s->sdiff, s->ssrc, s->srate, s->sface, s->swall, s->sres,
                    s->sdt, s->sfc, s->swc, s->qhat, s->tmp};
  for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; ++i) free(bufs[i]);
}

static void message(char* buf, size_t size, const char* text) {
  if (buf && size) { strncpy(buf, text, size - 1); buf[size - 1] = 0; }
}

static int options_valid(const amr_mesh_view_t* m, const amr_params_t* p) {
  if (!m || !p || m->n_cells == 0 || !(p->gamma > 1) || !isfinite(p->gamma) || !(p->cfl > 0) || p->cfl > 0.5 ||
      !isfinite(p->dt_fixed) || p->dt_fixed < 0 || !isfinite(p->ausm_mco) || p->ausm_mco <= 0 ||
      p->time_integrator != AMR_B200_TIME_SSP_RK3 || p->limiter != AMR_B200_LIMITER_FIRST_ORDER ||
      (p->flux != AMR_B200_FLUX_HLLC && p->flux != AMR_B200_FLUX_AUSMPUP))
    return 0;
  for (int side = 0; side < 4; ++side) if (!bc_valid(&m->boundaries[side], p->bc[side], side)) return 0;
  return 1;
}

/* ---- public oracle API ----------------------------------------------------------------- */

/* Residual dU/dt of u (static_amr2d_rhs). Returns 0 on success. */
int oracle_rhs(const amr_mesh_view_t* m, const amr_params_t* p, const double* u, double* r_out) {
  if (!options_valid(m, p)) return 1;
  ws_t s;
  if (ws_init(&s, m, p)) { ws_free(&s); return 1; }
  const int ok = residual(&s, u);
  if (ok) memcpy(r_out, s.r, s.nv * s.n * sizeof(double));
  ws_free(&s);
  return ok ? 0 : 1;
}

/* In-place SRD of the first four variables (static_amr2d_redistribute). */
int oracle_redistribute(const amr_mesh_view_t* m, double* u) {
  ws_t s;
  if (ws_init(&s, m, NULL)) { ws_free(&s); return 1; }
  redistribute(&s, u);
  ws_free(&s);
  return 0;
}

/* static_amr2d_run: advances u until *time == tend; maxsteps bounds the cumulative step
 * count.  Returns 0, or 1 with a message (including "maxsteps reached before tend"). */
int oracle_run(const amr_mesh_view_t* m, const amr_params_t* p, double tend, int64_t maxsteps, double* u,
               double* time, int64_t* steps, int64_t* rejected, char* msg, size_t msg_size) {
  if (!options_valid(m, p) || !isfinite(*time) || *time < 0 || !isfinite(tend) || tend < *time || maxsteps < 1) {
    message(msg, msg_size, "static AMR requires first-order RK3, valid state/options and CFL <= 0.5");
    return 1;
  }
  ws_t s;
  if (ws_init(&s, m, p)) { ws_free(&s); message(msg, msg_size, "allocation"); return 1; }
  const size_t n = s.n, nv = s.nv, count = nv * n;
  double* base_r = (double*)malloc(count * sizeof(double));
  double* u1 = (double*)malloc(count * sizeof(double));
  double* u2 = (double*)malloc(count * sizeof(double));
  const int laminar = m->transport.model == AMR_B200_MODEL_LAMINAR;
  int status = 0;
  while (*time < tend) {
    if (*steps >= maxsteps) { message(msg, msg_size, "maxsteps reached before tend"); status = 1; break; }
    if (!residual(&s, u)) { message(msg, msg_size, "nonphysical base state or nonfinite face flux"); status = 1; break; }
    double dt = p->dt_fixed > 0 ? p->dt_fixed : INFINITY;
    if (p->dt_fixed == 0)
      for (size_t k = 0; k < n; ++k) {
        const amr_cell_t* c = &m->cells[k];
        double spectral = 0;
        for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q) {
          const uint64_t f = m->cell_faces[q];
          spectral += s.speed[f] * m->faces[f].length;
        }
        const double a = sqrt(p->gamma * s.w[3 * n + k] / s.w[k]);
        for (uint64_t q = c->wall_begin; q < c->wall_begin + c->wall_count; ++q) spectral += a * m->walls[q].length;
        if (spectral > 0) dt = mn(dt, p->cfl * (m->agglomerate_small ? c->volume : (c->x1 - c->x0) * (c->y1 - c->y0)) / spectral);
      }
    if (p->dt_fixed == 0 && laminar) for (size_t k = 0; k < n; ++k) dt = mn(dt, s.vdt[k]);
    const double remaining = tend - *time;
    dt = mn(dt, remaining);
    const double time_tol = 32 * DBL_EPSILON * mx(mx(fabs(tend), fabs(*time)), dt);
    if (remaining - dt <= time_tol) dt = remaining;
    memcpy(base_r, s.r, count * sizeof(double));
    int accepted = 0;
    for (int attempt = 0; attempt < 21; ++attempt) {
      if (!isfinite(dt) || !(dt > 0) || *time + dt == *time) { message(msg, msg_size, "physical time step underflow"); status = 1; break; }
      for (size_t q = 0; q < count; ++q) u1[q] = u[q] + dt * base_r[q];
      redistribute(&s, u1);
      int ok = residual(&s, u1);
      if (ok) {
        for (size_t q = 0; q < count; ++q) u2[q] = 0.75 * u[q] + 0.25 * (u1[q] + dt * s.r[q]);
        redistribute(&s, u2);
        ok = residual(&s, u2);
      }
      if (ok) {
        for (size_t q = 0; q < count; ++q) u1[q] = u[q] / 3 + (2.0 / 3) * (u2[q] + dt * s.r[q]);
        redistribute(&s, u1);
        ok = primitive(&s, u1);
        if (m->transport.sa_model) for (size_t k = 0; k < n; ++k) ok = ok && isfinite(u1[4 * n + k]);
      }
      if (ok) {
        memcpy(u, u1, count * sizeof(double));
        *time = dt == remaining ? tend : *time + dt;
        ++*steps;
        accepted = 1;
        break;
      }
      ++*rejected;
      dt *= 0.5;
    }
    if (status) break;
    if (!accepted) { message(msg, msg_size, "RK candidates failed admissibility after 21 trials; physical step not committed"); status = 1; break; }
  }
  free(base_r); free(u1); free(u2);
  ws_free(&s);
  return status;
}

/* Steady diagnostics of the reference driver (src/quick_airfoil.cpp:189-199):
 * out[0..4] region residual norms, out[5..7] fx, fy, mz. */
int oracle_diagnostics(const amr_mesh_view_t* m, const amr_params_t* p, const double* u, const double* region,
                       double mxr, double myr, double* out) {
  if (!options_valid(m, p)) return 1;
  ws_t s;
  if (ws_init(&s, m, p)) { ws_free(&s); return 1; }
  const size_t n = s.n, nw = s.nw;
  const int nv = (int)s.nv;
  int ok = residual(&s, u);
  if (ok) {
    long double sum[5] = {0, 0, 0, 0, 0}, volume = 0;
    for (size_t k = 0; k < n; ++k) {
      const amr_cell_t* c = &m->cells[k];
      if (c->cx < region[0] || c->cx > region[1] || c->cy < region[2] || c->cy > region[3]) continue;
      volume += c->volume;
      for (int v = 0; v < nv; ++v) sum[v] += c->volume * fabs(s.r[v * n + k]);
    }
    for (int v = 0; v < 5; ++v) out[v] = v < nv && volume > 0 ? (double)(sum[v] / volume) : 0.0;
    if (m->transport.sa_model) out[4] /= m->transport.sa_nu_inf;
  }
  /* viscous wall flux of the state itself (static_amr2d_viscous_diagnostics recomputes the
   * primitives and viscous operator; the residual above already did the same on u) */
  const int laminar = m->transport.model == AMR_B200_MODEL_LAMINAR;
  double fx = 0, fy = 0, mz = 0;
  if (ok) {
    for (size_t i = 0; i < nw; ++i) {
      const amr_wall_t* wl = &m->walls[i];
      const size_t k = wl->owner_cell;
      const double pressure = (p->gamma - 1) * (u[3 * n + k] - .5 * (u[n + k] * u[n + k] + u[2 * n + k] * u[2 * n + k]) / u[k]);
      const double a = pressure * wl->nx * wl->length - (laminar ? s.vwall[nw + i] : 0.0);
      const double b = pressure * wl->ny * wl->length - (laminar ? s.vwall[2 * nw + i] : 0.0);
      fx += a; fy += b;
      mz += ((wl->x0 + wl->x1) * .5 - mxr) * b - ((wl->y0 + wl->y1) * .5 - myr) * a;
    }
  }
  out[5] = fx; out[6] = fy; out[7] = mz;
  ws_free(&s);
  return ok ? 0 : 1;
}
