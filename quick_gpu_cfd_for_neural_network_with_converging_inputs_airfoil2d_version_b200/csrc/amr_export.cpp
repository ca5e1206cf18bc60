// amr_export.cpp -- the reference's mesh and snapshot files, written from this engine's results.
//
// The reference pipeline (pipeline/export.py) reads a mesh prefix (<raw>.cells.npy,
// <raw>.walls.npy, ...) and a snapshot prefix (<raw>.final.state.npy,
// <raw>.final.wall_stress.npy, <raw>.final.viscous_loads.json, ...).  These writers produce the
// same files, byte for byte, as the reference's static_amr_binary_mesh and
// static_amr_binary_snapshot (src/static_amr2d_binary.cpp:14-78, with
// static_amr2d_write_boundaries src/static_amr2d_boundary.cpp:6-26, static_amr2d_write_viscous
// and static_amr2d_write_viscous_snapshot src/static_amr2d_viscous.cpp:143-187): NPY v1 '<f8'
// C-order arrays, and JSON/CSV text formatted by the same iostream settings (17 significant
// digits).  The per-wall stress rows, the SA cell rows and the dt limits come from the device
// (amr_gpu_export / amr_batch_export); the state-wide scalars (extrema, pressure forces,
// integrated conserved quantities) are summed here in the reference's order and precision.
//
// Compiled with the system g++ without contraction, like the reference CPU core.
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/amr_b200.h"

namespace {

void put(char* buf, uint64_t size, const std::string& text) {
  if (!buf || size == 0) return;
  const size_t len = text.size() < size - 1 ? text.size() : size - 1;
  std::memcpy(buf, text.data(), len);
  buf[len] = 0;
}

bool npy(const std::string& path, const double* values, uint64_t rows, uint64_t cols, std::string* why) {
  const uint16_t probe = 1;
  if (*reinterpret_cast<const unsigned char*>(&probe) != 1) {
    *why = "NPY writer requires little-endian host";
    return false;
  }
  std::ostringstream h;
  h << "{'descr': '<f8', 'fortran_order': False, 'shape': (" << rows << ", " << cols << "), }";
  std::string header = h.str();
  // magic (6) + version (2) + length (2) + header + newline: a multiple of 64 bytes
  while ((10 + header.size() + 1) % 64) header += ' ';
  header += '\n';
  if (header.size() > 65535) {
    *why = "NPY v1 header too large";
    return false;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    *why = "cannot open " + path;
    return false;
  }
  const unsigned char lead[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, (unsigned char)(header.size() & 255),
                                  (unsigned char)(header.size() >> 8)};
  bool ok = std::fwrite(lead, 1, sizeof(lead), f) == sizeof(lead) &&
            std::fwrite(header.data(), 1, header.size(), f) == header.size();
  if (rows && cols) ok = ok && std::fwrite(values, sizeof(double), rows * cols, f) == rows * cols;
  const bool closed = std::fclose(f) == 0;
  if (!(ok && closed)) *why = "NPY write failed: " + path;
  return ok && closed;
}

int kind_of(const amr_mesh_view_t& m, const amr_params_t& p, int side) {
  return m.boundaries[side].kind < 0 ? p.bc[side] : m.boundaries[side].kind;
}

bool finite(double x) { return std::isfinite(x); }

// Boundary metadata check (reference src/static_amr2d_boundary.h:32-47).
bool boundary_valid(const amr_boundary_t& b, int legacy, int side) {
  if (b.kind < AMR_B200_BC_INHERIT) return false;
  const int kind = b.kind < 0 ? legacy : b.kind;
  if (kind == AMR_B200_BC_TRANSMISSIVE || kind == AMR_B200_BC_REFLECT) return true;
  if (kind == AMR_B200_BC_NOSLIP)
    return finite(b.wall_velocity[0]) && finite(b.wall_velocity[1]) && b.wall_velocity[side / 2] == 0;
  const double* w = b.reference;
  const bool prim = finite(w[0]) && w[0] > 0 && finite(w[1]) && finite(w[2]) && finite(w[3]) && w[3] > 0;
  if (kind < AMR_B200_BC_FARFIELD || kind > AMR_B200_BC_PRESSURE_OUTLET || !prim) return false;
  if (kind == AMR_B200_BC_PRESSURE_OUTLET) return finite(b.outlet_pressure) && b.outlet_pressure > 0;
  if (kind == AMR_B200_BC_TOTAL_INLET) {
    const double d2 = b.direction[0] * b.direction[0] + b.direction[1] * b.direction[1];
    const double dn = (side % 2 ? 1.0 : -1.0) * b.direction[side / 2];
    return finite(d2) && std::fabs(d2 - 1) < 1e-12 && dn < 0 && finite(b.total_pressure) && b.total_pressure > 0 &&
           finite(b.total_temperature) && b.total_temperature > 0 && finite(b.gas_constant) && b.gas_constant > 0;
  }
  return true;
}

// <prefix>.bc.json, then the transport/stabilization metadata and, for viscous models, the
// gradient table and wall samples (src/static_amr2d_boundary.cpp:6-26, src/static_amr2d_viscous.cpp:171-186).
bool boundary_files(const std::string& prefix, const amr_mesh_view_t& m, const amr_params_t& p, std::string* why) {
  const amr_transport_t& t = m.transport;
  const bool euler = t.model == AMR_B200_MODEL_EULER;
  {
    std::ofstream out(prefix + ".bc.json");
    out << std::setprecision(17);
    static const char* names[] = {"xmin", "xmax", "ymin", "ymax"};
    static const char* kinds[] = {"unsupported", "transmissive", "reflect", "farfield", "total-inlet", "pressure-outlet", "no-slip"};
    out << "{\"model\":\"" << (euler ? "perfect-gas Euler; slip" : "laminar mechanical viscous; kappa=0; no-slip")
        << "\",\"characteristic_classification\":\"interior outward normal velocity and sound speed\",\"boundaries\":[";
    for (int side = 0; side < 4; ++side) {
      const amr_boundary_t& b = m.boundaries[side];
      const int kind = kind_of(m, p, side);
      if (!boundary_valid(b, p.bc[side], side)) {
        *why = "invalid boundary metadata";
        return false;
      }
      if (side) out << ',';
      out << "{\"id\":" << side << ",\"marker\":\"" << names[side] << "\",\"kind\":\"" << kinds[kind] << "\",\"normal\":["
          << (side < 2 ? (side % 2 ? 1 : -1) : 0) << ',' << (side >= 2 ? (side % 2 ? 1 : -1) : 0)
          << "],\"reference_rho_u_v_p\":[" << b.reference[0] << ',' << b.reference[1] << ',' << b.reference[2] << ','
          << b.reference[3] << ']';
      if (kind == AMR_B200_BC_TOTAL_INLET)
        out << ",\"total_pressure\":" << b.total_pressure << ",\"total_temperature\":" << b.total_temperature
            << ",\"gas_constant\":" << b.gas_constant << ",\"direction\":[" << b.direction[0] << ',' << b.direction[1] << ']';
      if (kind == AMR_B200_BC_PRESSURE_OUTLET)
        out << ",\"static_pressure\":" << b.outlet_pressure
            << ",\"backflow\":\"characteristic reference; fixed pressure not enforced during reversal\"";
      if (kind == AMR_B200_BC_NOSLIP) out << ",\"wall_velocity\":[" << b.wall_velocity[0] << ',' << b.wall_velocity[1] << ']';
      out << '}';
    }
    out << "],\"units\":\"consistent solver units; T and R must match p/rho=RT\"}\n";
    out.close();
    if (!out) {
      *why = "cannot write boundary metadata";
      return false;
    }
  }
  const uint64_t n_terms = euler || !m.visc_offsets ? 0 : m.visc_offsets[m.n_cells];
  {
    std::ofstream f(prefix + ".transport.json");
    f << std::setprecision(17);
    f << "{\"model\":\"" << (euler ? "euler" : t.sa_model ? "sa-neg-mechanical" : "laminar") << "\",\"viscosity_law\":\""
      << (t.law == AMR_B200_MU_CONSTANT ? "constant" : "sutherland") << "\",\"mu_ref\":" << t.mu_ref
      << ",\"sa_model\":" << t.sa_model << ",\"sa_nu_inf\":" << t.sa_nu_inf << ",\"Rgas\":" << t.gas_constant
      << ",\"T_ref\":" << t.temperature_ref << ",\"S\":" << t.sutherland << ",\"viscous_cfl\":" << t.viscous_cfl
      << ",\"conductivity\":0,\"viscous_work\":true,\"body_wall\":\"" << (euler ? "slip" : "stationary no-slip")
      << "\",\"open_viscous_bc\":\"zero normal velocity derivative, tangential derivative retained\",\"gradient_terms\":"
      << n_terms << ",\"wall_samples\":" << (euler ? 0 : m.n_walls) << "}\n";
    f.close();
    if (!f) {
      *why = "cannot write transport metadata";
      return false;
    }
  }
  {
    std::ofstream mode(prefix + ".viscous_stabilization.json");
    mode << "{\"mode\":\"" << (t.stabilization == AMR_B200_VISCOUS_SRD ? "srd-rate" : "true-volume")
         << "\",\"redistribution\":\"original zero-degree SRD\",\"wall_probe_min_h\":" << t.wall_probe_min_h
         << ",\"general_stability_proof\":false}\n";
    mode.close();
    if (!mode) {
      *why = "cannot write viscous stabilization metadata";
      return false;
    }
  }
  if (euler) return true;
  std::ofstream g(prefix + ".gradient_table.csv");
  g << std::setprecision(17) << "owner,source,side,cx,cy\n";
  for (uint64_t k = 0; k < m.n_cells; ++k)
    for (uint64_t q = m.visc_offsets[k]; q < m.visc_offsets[k + 1]; ++q) {
      const amr_gradient_term_t& s = m.visc_terms[q];
      g << k << ',' << s.source << ',' << s.side << ',' << s.x << ',' << s.y << '\n';
    }
  g.close();
  std::ofstream w(prefix + ".wall_samples.csv");
  w << std::setprecision(17) << "wall_id,owner,donor,normal_distance\n";
  for (uint64_t q = 0; q < m.n_walls; ++q)
    w << q << ',' << m.walls[q].owner_cell << ',' << m.wall_samples[q].donor << ',' << m.wall_samples[q].distance << '\n';
  w.close();
  if (!(g && w)) {
    *why = "viscous table output failed";
    return false;
  }
  return true;
}

}  // namespace

extern "C" int amr_write_npy(const char* path, const double* values, uint64_t rows, uint64_t cols, char* error,
                             uint64_t error_size) {
  std::string why;
  if (!path || (rows && cols && !values)) {
    put(error, error_size, "invalid NPY arguments");
    return 1;
  }
  if (!npy(path, values, rows, cols, &why)) {
    put(error, error_size, why);
    return 1;
  }
  return 0;
}

extern "C" int amr_write_mesh_files(const char* prefix_c, const amr_mesh_view_t* mv, const amr_mesh_options_t* op,
                                    const amr_params_t* pp, const amr_mesh_extras_t* ex, char* error,
                                    uint64_t error_size) {
  if (!prefix_c || !mv || !op || !pp) {
    put(error, error_size, "invalid mesh export arguments");
    return 1;
  }
  const std::string prefix(prefix_c);
  const amr_mesh_view_t& m = *mv;
  const amr_mesh_options_t& o = *op;
  const amr_params_t& p = *pp;
  std::string why;
  std::error_code ec;
  const auto parent = std::filesystem::path(prefix).parent_path();
  if (!parent.empty()) std::filesystem::create_directories(parent, ec);
  if (ec) {
    put(error, error_size, "cannot create output folder: " + ec.message());
    return 1;
  }
  if (!boundary_files(prefix, m, p, &why)) {
    put(error, error_size, why);
    return 1;
  }
  std::vector<double> cells, faces, walls;
  cells.reserve(13 * m.n_cells);
  faces.reserve(9 * m.n_faces);
  walls.reserve(11 * m.n_walls);
  for (uint64_t k = 0; k < m.n_cells; ++k) {
    const amr_cell_t& c = m.cells[k];
    for (double v : {(double)c.ix, (double)c.iy, (double)c.span, (double)c.level, c.x0, c.x1, c.y0, c.y1, c.volume, c.cx, c.cy,
                     (double)c.wall_begin, (double)c.wall_count})
      cells.push_back(v);
  }
  for (uint64_t q = 0; q < m.n_faces; ++q) {
    const amr_face_t& f = m.faces[q];
    for (double v : {(double)f.left, (double)f.right, (double)f.axis, (double)f.boundary, f.coordinate, f.lo, f.hi, f.length,
                     f.centroid})
      faces.push_back(v);
  }
  for (uint64_t q = 0; q < m.n_walls; ++q) {
    const amr_wall_t& w = m.walls[q];
    for (double v : {(double)w.owner_cell, (double)w.source_edge_id, (double)w.body_id, (double)w.patch_id, w.x0, w.y0, w.x1,
                     w.y1, w.nx, w.ny, w.length})
      walls.push_back(v);
  }
  if (!npy(prefix + ".cells.npy", cells.data(), m.n_cells, 13, &why) ||
      !npy(prefix + ".faces.npy", faces.data(), m.n_faces, 9, &why) ||
      !npy(prefix + ".walls.npy", walls.data(), m.n_walls, 11, &why)) {
    put(error, error_size, why);
    return 1;
  }
  const uint64_t split_leaves = ex ? ex->split_leaves : 0, coarse_fine = ex ? ex->coarse_fine_faces : 0;
  if (split_leaves && ex && ex->leaf_components) {
    std::vector<double> mapping;
    for (uint64_t i = 0; i < ex->n_leaf_components; ++i) {
      mapping.push_back((double)ex->leaf_components[2 * i]);
      mapping.push_back((double)ex->leaf_components[2 * i + 1]);
    }
    if (!npy(prefix + ".leaf_components.npy", mapping.data(), ex->n_leaf_components, 2, &why)) {
      put(error, error_size, why);
      return 1;
    }
  }
  if (ex && ex->n_agglomeration && ex->agglomeration &&
      !npy(prefix + ".agglomeration.npy", ex->agglomeration, ex->n_agglomeration, 9, &why)) {
    put(error, error_size, why);
    return 1;
  }
  const amr_transport_t& t = m.transport;
  std::ofstream out(prefix + ".mesh.json");
  out << std::setprecision(17) << "{\n\"format\":\"NPY v1 <f8, C-order\",\n\"model\":\""
      << (t.model == AMR_B200_MODEL_EULER
              ? "2D Euler, static slip wall"
              : (t.sa_model ? "2D SA-neg mechanical viscous, kappa=0, stationary no-slip wall"
                            : "2D laminar mechanical viscous, kappa=0, stationary no-slip wall"))
      << (o.agglomerate_small ? ", agglomerated FV, no SRD, SSP-RK3\",\n" : ", zero-degree SRD, SSP-RK3\",\n")
      << "\"cells_columns\":[\"ix\",\"iy\",\"span\",\"level\",\"x0\",\"x1\",\"y0\",\"y1\",\"fluid_area\",\"cx\",\"cy\",\"wall_begin\",\"wall_count\"],\n"
      << "\"faces_columns\":[\"left\",\"right\",\"axis\",\"boundary\",\"coordinate\",\"lo\",\"hi\",\"open_length\",\"open_centroid\"],\n"
      << "\"walls_columns\":[\"owner\",\"source_edge\",\"body\",\"patch\",\"x0\",\"y0\",\"x1\",\"y1\",\"nx\",\"ny\",\"length\"],\n"
      << "\"state_shape\":[" << (t.sa_model ? 5 : 4) << "," << m.n_cells << "],\n\"state_rows\":[\"rho\",\"rho_u\",\"rho_v\",\"rho_E\""
      << (t.sa_model ? ",\"rho_nutilde\"" : "") << "],\n"
      << "\"bounds\":[" << o.xmin << ',' << o.xmax << ',' << o.ymin << ',' << o.ymax << "],\n\"base_shape\":[" << o.nx << ','
      << o.ny << "],\n\"levels\":" << o.levels << ",\n\"buffer\":" << o.buffer << ",\n\"gamma\":" << p.gamma
      << ",\n\"cfl\":" << p.cfl << ",\n\"fixed_dt\":" << p.dt_fixed << ",\n\"flux\":\""
      << (p.flux == AMR_B200_FLUX_HLLC ? "hllc" : "ausm") << "\",\n\"bc\":[" << kind_of(m, p, 0) << ',' << kind_of(m, p, 1)
      << ',' << kind_of(m, p, 2) << ',' << kind_of(m, p, 3) << "],\n\"coarse_fine_subfaces\":" << coarse_fine
      << ",\n\"small_cells\":" << m.small_cells << ",\n\"split_background_leaves\":" << split_leaves
      << ",\n\"redistribution_mode\":\"" << (o.agglomerate_small ? "agglomerated-no-SRD" : "state-SRD") << "\"\n}\n";
  out.close();
  if (!out) {
    put(error, error_size, "mesh JSON write failed");
    return 1;
  }
  return 0;
}

extern "C" int amr_write_snapshot_files(const char* prefix_c, const amr_mesh_view_t* mv, const amr_mesh_options_t* op,
                                        const amr_params_t* pp, const double* u, double time, int64_t steps,
                                        int64_t rejected, const char* backend, const amr_export_rows_t* rows,
                                        char* error, uint64_t error_size) {
  if (!prefix_c || !mv || !op || !pp || !u || !backend) {
    put(error, error_size, "invalid snapshot arguments");
    return 1;
  }
  const std::string prefix(prefix_c);
  const amr_mesh_view_t& m = *mv;
  const amr_params_t& p = *pp;
  const amr_transport_t& t = m.transport;
  const uint64_t n = m.n_cells, nw = m.n_walls, nv = t.sa_model ? 5 : 4;
  std::string why;
  // state-wide scalars (src/static_amr2d_binary.cpp:54-60)
  double rhomin = INFINITY, rhomax = 0, pmin = INFINITY, pmax = 0, fx = 0, fy = 0, mz = 0;
  long double totals[4] = {0, 0, 0, 0};
  for (uint64_t k = 0; k < n; ++k) {
    const double rho = u[k], vx = u[n + k] / rho, vy = u[2 * n + k] / rho;
    const double pressure = (p.gamma - 1) * (u[3 * n + k] - .5 * rho * (vx * vx + vy * vy));
    if (!std::isfinite(rho) || !(rho > 0) || !std::isfinite(pressure) || !(pressure > 0)) {
      put(error, error_size, "nonphysical snapshot; no file certified");
      return 1;
    }
    rhomin = std::min(rhomin, rho);
    rhomax = std::max(rhomax, rho);
    pmin = std::min(pmin, pressure);
    pmax = std::max(pmax, pressure);
    for (int v = 0; v < 4; ++v) totals[v] += static_cast<long double>(m.cells[k].volume) * u[v * n + k];
    const amr_cell_t& c = m.cells[k];
    for (uint64_t q = c.wall_begin; q < c.wall_begin + c.wall_count; ++q) {
      const amr_wall_t& w = m.walls[q];
      const double x = pressure * w.nx * w.length, y = pressure * w.ny * w.length;
      fx += x;
      fy += y;
      mz += .5 * (w.x0 + w.x1) * y - .5 * (w.y0 + w.y1) * x;
    }
  }
  if (!npy(prefix + ".state.npy", u, nv, n, &why)) {
    put(error, error_size, why);
    return 1;
  }
  {
    std::ofstream out(prefix + ".json");
    out << std::setprecision(17) << "{\"backend\":\"" << backend << "\",\"time\":" << time << ",\"steps\":" << steps
        << ",\"rejected\":" << rejected << ",\"rho_min\":" << rhomin << ",\"rho_max\":" << rhomax << ",\"p_min\":" << pmin
        << ",\"p_max\":" << pmax << ",\"fx_pressure\":" << fx << ",\"fy_pressure\":" << fy
        << ",\"mz_pressure_about_origin\":" << mz << ",\"integrated_conserved\":[" << totals[0] << ',' << totals[1] << ','
        << totals[2] << ',' << totals[3] << "],\"state_bytes\":" << nv * n * sizeof(double)
        << ",\"dimensional_units\":false}\n";
    out.close();
    if (!out) {
      put(error, error_size, "snapshot JSON write failed");
      return 1;
    }
  }
  if (t.model == AMR_B200_MODEL_EULER) return 0;
  // viscous snapshot (src/static_amr2d_viscous.cpp:143-170) from the device-computed rows
  if (!rows || (nw && !rows->wall_rows) || (t.sa_model && !rows->sa_rows)) {
    put(error, error_size, "viscous snapshot needs the exported wall (and SA) rows");
    return 1;
  }
  {
    std::ofstream limits(prefix + ".timestep_limits.json");
    limits << std::setprecision(17) << "{\"convective_dt\":" << rows->convective_dt << ",\"viscous_dt\":" << rows->viscous_dt
           << ",\"mode\":\"" << (t.stabilization == AMR_B200_VISCOUS_SRD ? "srd-rate" : "true-volume")
           << "\",\"fixed_dt\":" << p.dt_fixed << "}\n";
    limits.close();
    if (!limits) {
      put(error, error_size, "timestep limit output failed");
      return 1;
    }
  }
  std::map<int, std::array<double, 6>> loads;
  std::array<double, 6> total = {0, 0, 0, 0, 0, 0};
  for (uint64_t q = 0; q < nw; ++q) {
    const amr_wall_t& w = m.walls[q];
    const double* r = rows->wall_rows + 14 * q;
    const double x = .5 * (w.x0 + w.x1), y = .5 * (w.y0 + w.y1);
    const double px = r[9], py = r[10], vx = r[11], vy = r[12];
    const std::array<double, 6> values = {px, py, x * py - y * px, vx, vy, r[13]};
    auto& patch = loads[w.patch_id];
    for (int v = 0; v < 6; ++v) {
      patch[v] += values[v];
      total[v] += values[v];
    }
  }
  if (!npy(prefix + ".wall_stress.npy", rows->wall_rows, nw, 14, &why)) {
    put(error, error_size, why);
    return 1;
  }
  {
    std::ofstream f(prefix + ".viscous_loads.json");
    f << std::setprecision(17) << "{\"time\":" << time << ",\"model\":\"" << (t.sa_model ? "sa-neg-mechanical" : "laminar")
      << "\",\"conductivity\":0,\"load_columns\":[\"fx_pressure\",\"fy_pressure\",\"mz_pressure\",\"fx_viscous\",\"fy_viscous\",\"mz_viscous\"],\"total\":[";
    for (int v = 0; v < 6; ++v) {
      if (v) f << ',';
      f << total[v];
    }
    f << "],\"patches\":[";
    bool first = true;
    for (const auto& [id, value] : loads) {
      if (!first) f << ',';
      first = false;
      f << "{\"patch\":" << id << ",\"loads\":[";
      for (int v = 0; v < 6; ++v) {
        if (v) f << ',';
        f << value[v];
      }
      f << "]}";
    }
    f << "],\"viscous_dt_min\":" << rows->viscous_dt
      << ",\"wall_stress_columns\":[\"wall_id\",\"owner\",\"donor\",\"normal_distance\",\"mu\",\"tau_n_x\",\"tau_n_y\",\"tau_t_signed\",\"p\",\"fx_pressure\",\"fy_pressure\",\"fx_viscous\",\"fy_viscous\",\"mz_viscous\"],\"moment_reference\":[0,0],\"wall_normal\":\"fluid to solid\",\"wall_energy_flux\":0}\n";
    f.close();
    if (!f) {
      put(error, error_size, "viscous load output failed");
      return 1;
    }
  }
  if (t.sa_model) {
    if (!npy(prefix + ".sa.npy", rows->sa_rows, n, 3, &why)) {
      put(error, error_size, why);
      return 1;
    }
    std::ofstream desc(prefix + ".sa.json");
    desc << "{\"model\":\"SA-neg-ft2-Note1c-mechanical\",\"columns\":[\"nutilde\",\"mu_t\",\"wall_distance\"],\"nu_inf\":"
         << t.sa_nu_inf << ",\"wall_nutilde\":0,\"thermal_conductivity\":0}\n";
    desc.close();
    if (!desc) {
      put(error, error_size, "SA metadata failed");
      return 1;
    }
  }
  return 0;
}
