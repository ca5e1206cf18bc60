// amr_engine_inst.cuh -- kernel dispatch, diagnostics reductions and the launch autotuner.
// Included once per precision by amr_engine_f64.cu and amr_engine_f32.cu.
#pragma once
#include "amr_batch_impl.cuh"

namespace amrb {

template <class R> static const void* kernel_for(int model, int flux, bool srd) {
#define AMRB_K(M, F, S) reinterpret_cast<const void*>(&trials_kernel<R, M, F, S>)
  static const void* table[3][2][2] = {
      {{AMRB_K(0, 0, false), AMRB_K(0, 0, true)}, {AMRB_K(0, 1, false), AMRB_K(0, 1, true)}},
      {{AMRB_K(1, 0, false), AMRB_K(1, 0, true)}, {AMRB_K(1, 1, false), AMRB_K(1, 1, true)}},
      {{AMRB_K(2, 0, false), AMRB_K(2, 0, true)}, {AMRB_K(2, 1, false), AMRB_K(2, 1, true)}}};
#undef AMRB_K
  return table[model][flux][srd ? 1 : 0];
}

template <class R>
cudaError_t EngineOps<R>::launch(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int grid, int block,
                                 cudaStream_t stream, bool cooperative) {
  Dev<R> dd = d;
  int t = trials, m = mode;
  void* args[] = {&dd, &t, &m};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem_bytes(block);
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = cooperative ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, kernel_for<R>(model, flux, srd), args);
}

template <class R, int MODEL, int FLUX>
static cudaError_t launch_phases_t(const Dev<R>& d, bool srd, int trials, int mode, int block, cudaStream_t st) {
  const int tiles = d.n_tiles > 0 ? (d.n_tiles + block / 32 - 1) / (block / 32) : 1;  // blocks of block/32 tile-warps
  const size_t sm = EngineOps<R>::smem_bytes(block);
  const int cases = d.n_cases;
  const int cblocks = (cases + 127) / 128;
  if (mode == MODE_RESIDUAL) {
    if (MODEL >= MODEL_LAMINAR) phase_grad_kernel<R, MODEL><<<tiles, block, sm, st>>>(d, STAGE_DIAG);
    phase_flux_kernel<R, MODEL, FLUX><<<tiles, block, sm, st>>>(d, STAGE_DIAG);
    return cudaGetLastError();
  }
  phase_commit_kernel<<<cblocks, 128, 0, st>>>(d.ctl, cases, 1);
  for (int t = 0; t < trials; ++t) {
    if (MODEL >= MODEL_LAMINAR) phase_grad_kernel<R, MODEL><<<tiles, block, sm, st>>>(d, STAGE_BASE);
    phase_flux_kernel<R, MODEL, FLUX><<<tiles, block, sm, st>>>(d, STAGE_BASE);
    phase_first_cells_kernel<R, MODEL><<<(d.n_cells + 255) / 256 + 1, 256, 0, st>>>(d);
    for (int stage = 1; stage <= 2; ++stage) {
      if (srd) phase_srd_kernel<R, MODEL><<<cases, block, 0, st>>>(d, stage);
      if (MODEL >= MODEL_LAMINAR) phase_grad_kernel<R, MODEL><<<tiles, block, sm, st>>>(d, stage);
      phase_flux_kernel<R, MODEL, FLUX><<<tiles, block, sm, st>>>(d, stage);
    }
    if (srd) phase_srd_kernel<R, MODEL><<<cases, block, 0, st>>>(d, 3);
    phase_commit_kernel<<<cblocks, 128, 0, st>>>(d.ctl, cases, 0);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t EngineOps<R>::launch_phases(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode, int block,
                                        cudaStream_t stream) {
  if (model == MODEL_EULER)
    return flux == FLUX_HLLC ? launch_phases_t<R, MODEL_EULER, FLUX_HLLC>(d, srd, trials, mode, block, stream)
                             : launch_phases_t<R, MODEL_EULER, FLUX_AUSM>(d, srd, trials, mode, block, stream);
  if (model == MODEL_LAMINAR)
    return flux == FLUX_HLLC ? launch_phases_t<R, MODEL_LAMINAR, FLUX_HLLC>(d, srd, trials, mode, block, stream)
                             : launch_phases_t<R, MODEL_LAMINAR, FLUX_AUSM>(d, srd, trials, mode, block, stream);
  return flux == FLUX_HLLC ? launch_phases_t<R, MODEL_SA, FLUX_HLLC>(d, srd, trials, mode, block, stream)
                           : launch_phases_t<R, MODEL_SA, FLUX_AUSM>(d, srd, trials, mode, block, stream);
}

// Grids are fixed by the arena's capacity (grid-stride loops over the live ranges, which the
// kernels read from the device), so a captured graph stays valid when cases come and go.
template <class R, int MODEL, int FLUX>
static cudaError_t launch_split_t(const Dev<R>& d, bool srd, int trials, int mode, cudaStream_t st, int sms) {
  const int B = PHASE_BLOCK;
  const long long ncap = d.ncap, icap = (long long)d.cap_faces + d.cap_walls;
  const int cblocks = (int)std::min<long long>((ncap + B - 1) / B, (long long)sms * SplitOcc<R>::cell);
  const int iblocks = (int)std::min<long long>((icap + B - 1) / B, (long long)sms * SplitOcc<R>::item);
  const int fblocks = (int)std::min<long long>((ncap + 255) / 256, (long long)sms * 8);
  const int cases = d.n_cases;
  const int kblocks = (cases + 127) / 128;
  auto stage_seq = [&](int stage) {
    if (MODEL >= MODEL_LAMINAR) grad_cells_kernel<R, MODEL><<<cblocks, B, 0, st>>>(d, stage);
    item_kernel<R, MODEL, FLUX><<<iblocks, B, 0, st>>>(d, stage);
    gather_kernel<R, MODEL><<<cblocks, B, 0, st>>>(d, stage);
  };
  if (mode == MODE_RESIDUAL) {
    stage_seq(STAGE_DIAG);
    return cudaGetLastError();
  }
  phase_commit_kernel<<<kblocks, 128, 0, st>>>(d.ctl, cases, 1);
  for (int t = 0; t < trials; ++t) {
    stage_seq(STAGE_BASE);
    phase_first_cells_kernel<R, MODEL><<<fblocks, 256, 0, st>>>(d);
    for (int stage = 1; stage <= 2; ++stage) {
      if (srd) phase_srd_kernel<R, MODEL><<<cases, MAX_BLOCK, 0, st>>>(d, stage);
      stage_seq(stage);
    }
    if (srd) phase_srd_kernel<R, MODEL><<<cases, MAX_BLOCK, 0, st>>>(d, 3);
    phase_commit_kernel<<<kblocks, 128, 0, st>>>(d.ctl, cases, 0);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t EngineOps<R>::launch_split(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode,
                                       cudaStream_t stream, int sms) {
  if (model == MODEL_EULER)
    return flux == FLUX_HLLC ? launch_split_t<R, MODEL_EULER, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                             : launch_split_t<R, MODEL_EULER, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
  if (model == MODEL_LAMINAR)
    return flux == FLUX_HLLC ? launch_split_t<R, MODEL_LAMINAR, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                             : launch_split_t<R, MODEL_LAMINAR, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
  return flux == FLUX_HLLC ? launch_split_t<R, MODEL_SA, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                           : launch_split_t<R, MODEL_SA, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
}

template <class R> cudaError_t EngineOps<R>::occupancy(int model, int flux, bool srd, int block, int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel_for<R>(model, flux, srd), block,
                                                       smem_bytes(block));
}

// Per-tile partial sums of the steady diagnostics (reference driver src/quick_airfoil.cpp:189-199):
// [0..4] sum V|R_v| over cells with centroid inside the region, [5] region volume,
// [6..8] Fx, Fy, Mz from wall pressure minus viscous wall flux.  FP64 throughout; the
// reduction order inside a tile is a fixed tree, so the result does not depend on which
// other cases share the batch.
template <class R, int MODEL>
__global__ void diag_tile_kernel(Dev<R> d, const double* __restrict__ dcfg, double* __restrict__ part,
                                 const double* __restrict__ cx, const double* __restrict__ cy,
                                 const double* __restrict__ wxm, const double* __restrict__ wym) {
  extern __shared__ double red[];  // [9][blockDim]
  const int B = blockDim.x, i = threadIdx.x;
  const Tile t = d.tiles[blockIdx.x];
  const long long n = d.ncap;
  const int nv = MODEL == MODEL_SA ? 5 : 4;
  const double* c = dcfg + 7 * t.cs;
  const CaseCtl& ctl = d.ctl[t.cs];
  const R* U = ctl.cur ? d.U1 : d.U0;
  const double g = (double)d.cfg[t.cs].gamma;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = t.c0 + i; k < t.c1; k += B) {
    const double V = d.c_vol[k];
    if (!(cx[k] < c[0] || cx[k] > c[1] || cy[k] < c[2] || cy[k] > c[3])) {
      acc[5] += V;
      for (int v = 0; v < nv; ++v) acc[v] += V * fabs((double)d.R0[v * n + k]);
    }
    const double rho = U[k], mx = U[n + k], my = U[2 * n + k], e = U[3 * n + k];
    const double p = (g - 1) * (e - .5 * (mx * mx + my * my) / rho);
    for (int q = d.c_wall[k]; q < d.c_wall[k + 1]; ++q) {
      const double nx = d.w_nx[q], ny = d.w_ny[q], len = d.w_len[q];
      double vx = 0, vy = 0;
      if (MODEL >= MODEL_LAMINAR) {
        const int dn = d.w_donor[q];
        const R rd = U[dn], ud = U[n + dn] / rd, vd = U[2 * n + dn] / rd;
        R gw[4], fw[4];
        wall_gradient(d.w_nx[q], d.w_ny[q], d.w_dist[q], -ud, -vd, gw);
        visc_flux(d.mu[dn], gw, d.w_nx[q], d.w_ny[q], R(0), R(0), fw);
        vx = (double)(fw[1] * d.w_len[q]);
        vy = (double)(fw[2] * d.w_len[q]);
      }
      const double a = p * nx * len - vx, b = p * ny * len - vy;
      acc[6] += a;
      acc[7] += b;
      acc[8] += (wxm[q] - c[4]) * b - (wym[q] - c[5]) * a;
    }
  }
  for (int v = 0; v < 9; ++v) red[v * B + i] = acc[v];
  __syncthreads();
  for (int s = B / 2; s > 0; s >>= 1) {
    if (i < s)
      for (int v = 0; v < 9; ++v) red[v * B + i] += red[v * B + i + s];
    __syncthreads();
  }
  if (i < 9) part[9 * blockIdx.x + i] = red[i * B];
}

static __global__ void diag_case_kernel(const int* __restrict__ ranges, const double* __restrict__ part, double* __restrict__ out,
                                 int ncases) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= ncases) return;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int t = ranges[2 * cs]; t < ranges[2 * cs + 1]; ++t)
    for (int v = 0; v < 9; ++v) acc[v] += part[9 * t + v];
  for (int v = 0; v < 9; ++v) out[9 * cs + v] = acc[v];
}

template <class R>
int Batch<R>::diagnostics(const std::vector<int>& slots, const std::vector<double>& rm, std::vector<double>* out,
                          std::string* error) {
  if (live_ == 0) return fail1(error, "no live cases");
  std::vector<double> dcfg(7 * config_.max_cases, 0.0);
  for (size_t i = 0; i < slots.size(); ++i)
    for (int v = 0; v < 6; ++v) dcfg[7 * slots[i] + v] = rm[6 * i + v];
  if (residual(error)) return 1;
  bool ok = cuda_ok(cudaMemcpyAsync(diag_cfg_.p, dcfg.data(), sizeof(double) * dcfg.size(), cudaMemcpyHostToDevice, stream_),
                    error, "diag cfg");
  const int B = 256;
  if (ok && n_tiles_ > 0) {
    cudaGetLastError();
    const Dev<R> d = dev();
    const size_t sm = sizeof(double) * 9 * B;
    if (model_ == MODEL_EULER)
      diag_tile_kernel<R, MODEL_EULER><<<n_tiles_, B, sm, stream_>>>(d, diag_cfg_.p, diag_part_.p, c_cx_.p, c_cy_.p, w_xm_.p, w_ym_.p);
    else if (model_ == MODEL_LAMINAR)
      diag_tile_kernel<R, MODEL_LAMINAR><<<n_tiles_, B, sm, stream_>>>(d, diag_cfg_.p, diag_part_.p, c_cx_.p, c_cy_.p, w_xm_.p, w_ym_.p);
    else
      diag_tile_kernel<R, MODEL_SA><<<n_tiles_, B, sm, stream_>>>(d, diag_cfg_.p, diag_part_.p, c_cx_.p, c_cy_.p, w_xm_.p, w_ym_.p);
    diag_case_kernel<<<(config_.max_cases + 127) / 128, 128, 0, stream_>>>(case_tiles_.p, diag_part_.p, diag_out_.p,
                                                                           config_.max_cases);
    launches_ += 2;
    ok = cuda_ok(cudaGetLastError(), error, "diagnostics launch");
  }
  std::vector<double> all(9 * config_.max_cases);
  ok = ok && cuda_ok(cudaMemcpyAsync(all.data(), diag_out_.p, sizeof(double) * all.size(), cudaMemcpyDeviceToHost, stream_),
                     error, "diag read-back") &&
       cuda_ok(cudaStreamSynchronize(stream_), error, "diag sync");
  if (!ok) return 1;
  out->assign(9 * slots.size(), 0.0);
  for (size_t i = 0; i < slots.size(); ++i)
    for (int v = 0; v < 9; ++v) (*out)[9 * i + v] = all[9 * slots[i] + v];
  return 0;
}

// Picks the block size and grid size with the shortest trial time on the live cases, by
// running `trials` trials per candidate and restoring the state and controls after each.
template <class R> int Batch<R>::autotune(int trials, std::string* error) {
  if (live_ == 0) return 0;
  const long long nbytes = (long long)sizeof(R) * nv_ * cap_cells_;
  DevBuf<R> s0, s1;
  uint64_t dummy = 0;
  if (!s0.alloc(nv_ * cap_cells_, &dummy, error, "autotune") || !s1.alloc(nv_ * cap_cells_, &dummy, error, "autotune"))
    return 1;
  std::vector<CaseCtl> ctl_save(h_ctl_, h_ctl_ + config_.max_cases);
  cudaMemcpyAsync(s0.p, U0_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  cudaMemcpyAsync(s1.p, U1_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  double best = 1e30;
  int best_block = block_, best_grid = grid_request_;
  int best_mode = mode_;
  const bool graph_save = use_graph_;
  use_graph_ = false;
  for (int mode : {AMR_B200_LAUNCH_PERSISTENT, AMR_B200_LAUNCH_PHASES, AMR_B200_LAUNCH_SPLIT}) {
    for (int block : {128, 256}) {
      if (mode != AMR_B200_LAUNCH_PERSISTENT && block != PHASE_BLOCK) continue;
      mode_ = mode;
      block_ = block;
      grid_request_ = 0;
      if (!configure_grid(error)) continue;
      bool tiled = true;
      for (auto& c : cases_)
        if (c.live && !retile(c)) tiled = false;
      if (!tiled) continue;
      tiles_dirty_ = true;
      if (!sync_tiles(error)) return 1;
      std::vector<int> grids = {max_grid_};
      if (mode_ == AMR_B200_LAUNCH_PERSISTENT) {
        const int need = (n_tiles_ + block / 32 - 1) / (block / 32);  // one tile per warp
        if (need < max_grid_) grids.push_back(std::max(1, need));
        if (need / 2 < max_grid_ && need / 2 >= 8) grids.push_back(need / 2);
      }
      for (int grid : grids) {
        grid_request_ = grid;
        configure_grid(error);
        std::string e;
        // one untimed pass, then the timed one
        bool ok = advance(trials, &e) == 0;
        restore(ctl_save, s0, s1, nbytes);
        ok = ok && advance(trials, &e) == 0;
        const double t = last_seconds_;
        restore(ctl_save, s0, s1, nbytes);
        if (ok && t > 0 && t < best) {
          best = t;
          best_block = block;
          best_grid = grid;
          best_mode = mode_;
        }
      }
    }
  }
  mode_ = best_mode;
  block_ = best_block;
  grid_request_ = best_grid;
  configure_grid(error);
  for (auto& c : cases_)
    if (c.live) retile(c);
  tiles_dirty_ = true;
  use_graph_ = graph_save;
  graph_dirty_ = true;
  for (int i = 0; i < config_.max_cases; ++i) refresh_meta(i);
  s0.free();
  s1.free();
  return sync_tiles(error) ? 0 : 1;
}

template <class R>
void Batch<R>::restore(const std::vector<CaseCtl>& ctl_save, const DevBuf<R>& s0, const DevBuf<R>& s1, long long nbytes) {
  std::copy(ctl_save.begin(), ctl_save.end(), h_ctl_);
  cudaMemcpyAsync(ctl_.p, h_ctl_, sizeof(CaseCtl) * config_.max_cases, cudaMemcpyHostToDevice, stream_);
  cudaMemcpyAsync(U0_.p, s0.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  cudaMemcpyAsync(U1_.p, s1.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  cudaStreamSynchronize(stream_);
}

}  // namespace amrb
