// amr_engine_inst.cuh -- kernel dispatch, diagnostics reductions and the launch autotuner.
// Included once per precision by amr_engine_f64.cu and amr_engine_f32.cu.
#pragma once
#include <type_traits>

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

// One kernel launch of a chain (see chain_begin): programmatic stream serialization lets the
// kernel be scheduled during its predecessor's tail.  Errors surface through cudaGetLastError.
template <class... P, class... A>
static void chain(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <class R, int MODEL, int FLUX>
static cudaError_t launch_phases_t(const Dev<R>& d, bool srd, int trials, int mode, int block, cudaStream_t st) {
  const int tiles = d.n_tiles > 0 ? (d.n_tiles + block / 32 - 1) / (block / 32) : 1;  // blocks of block/32 tile-warps
  const size_t sm = EngineOps<R>::smem_bytes(block);
  const int cases = d.n_cases;
  const int cblocks = (cases + 127) / 128;
  auto phase_pair = [&](auto stage_tag) {
    constexpr int S = decltype(stage_tag)::value;
    if (MODEL >= MODEL_LAMINAR) chain(phase_grad_kernel<R, MODEL, S>, dim3(tiles), dim3(block), sm, st, d);
    chain(phase_flux_kernel<R, MODEL, FLUX, S>, dim3(tiles), dim3(block), sm, st, d);
  };
  if (mode == MODE_RESIDUAL) {
    phase_pair(std::integral_constant<int, STAGE_DIAG>{});
    return cudaGetLastError();
  }
  chain(phase_commit_kernel, dim3(cblocks), dim3(128), 0, st, d.ctl, cases, 1, (const int*)nullptr, 0);
  for (int t = 0; t < trials; ++t) {
    phase_pair(std::integral_constant<int, STAGE_BASE>{});
    if (srd && MODEL >= MODEL_LAMINAR && d.any_srd_rate) chain(srd_rate_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, st, d, -1);
    chain(phase_first_cells_kernel<R, MODEL>, dim3((d.n_cells + 255) / 256 + 1), dim3(256), 0, st, d);
    for (int stage = 1; stage <= 2; ++stage) {
      if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(block), 0, st, d, stage);
      if (stage == 1)
        phase_pair(std::integral_constant<int, STAGE_1>{});
      else
        phase_pair(std::integral_constant<int, STAGE_2>{});
    }
    if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(block), 0, st, d, 3);
    chain(phase_commit_kernel, dim3(cblocks), dim3(128), 0, st, d.ctl, cases, 0, (const int*)nullptr, 0);
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
static cudaError_t launch_split_t(const Dev<R>& d, bool srd, int trials, int mode, cudaStream_t st, int sms,
                                  const SplitLanes<R>* lanes) {
  const int B = PHASE_BLOCK;
  const long long ncap = d.ncap, icap = (long long)d.cap_faces + d.cap_walls;
  // grids of one wave of co-resident blocks at each kernel's register budget
  const auto cells_grid = [&](int per_sm) { return (int)std::min<long long>((ncap + B - 1) / B, (long long)sms * per_sm); };
  const auto items_grid = [&](int per_sm) { return (int)std::min<long long>((icap + B - 1) / B, (long long)sms * per_sm); };
  const int fblocks = (int)std::min<long long>((ncap + 255) / 256, (long long)sms * 8);
  const int cases = d.n_cases;
  const int kblocks = (cases + 127) / 128;
  // Viscous models without SRD: the first update only adds dt R0, so the stage-1 kernels form
  // U1 where they read it and one thread per case makes the update's control decisions.
  // (Euler reads U1 in the face kernel; SRD changes U1 between the update and stage 1.)
  const bool fused = MODEL >= MODEL_LAMINAR && !srd;
  // one lane's kernels on stream s
  const auto run = [&](const Dev<R>& dd, cudaStream_t s) {
    auto stage_kernels = [&](auto stage_tag) {
      constexpr int S = decltype(stage_tag)::value;
      using O = SplitStageOcc<R, S>;
      if constexpr (S == STAGE_1) {
        if (fused) {
          chain(grad_cells_kernel<R, MODEL, S, true>, dim3(cells_grid(O::cell)), dim3(B), 0, s, dd);
          chain(item_kernel<R, MODEL, FLUX, S>, dim3(items_grid(O::item)), dim3(B), 0, s, dd);
          chain(gather_kernel<R, MODEL, S, true>, dim3(cells_grid(O::gather)), dim3(B), 0, s, dd);
          return;
        }
      }
      if (MODEL >= MODEL_LAMINAR)
        chain(grad_cells_kernel<R, MODEL, S>, dim3(cells_grid(O::cell)), dim3(B), 0, s, dd);
      chain(item_kernel<R, MODEL, FLUX, S>, dim3(items_grid(O::item)), dim3(B), 0, s, dd);
      chain(gather_kernel<R, MODEL, S>, dim3(cells_grid(O::gather)), dim3(B), 0, s, dd);
    };
    auto stage_seq = [&](int stage) {
      switch (stage) {
        case STAGE_BASE: stage_kernels(std::integral_constant<int, STAGE_BASE>{}); break;
        case STAGE_1: stage_kernels(std::integral_constant<int, STAGE_1>{}); break;
        case STAGE_2: stage_kernels(std::integral_constant<int, STAGE_2>{}); break;
        default: stage_kernels(std::integral_constant<int, STAGE_DIAG>{}); break;
      }
    };
    if (mode == MODE_RESIDUAL) {
      stage_seq(STAGE_DIAG);
      return;
    }
    chain(phase_commit_kernel, dim3(kblocks), dim3(128), 0, s, dd.ctl, cases, 1, dd.case_lane, dd.lane);
    for (int t = 0; t < trials; ++t) {
      stage_seq(STAGE_BASE);
      if (srd && MODEL >= MODEL_LAMINAR && dd.any_srd_rate)
        chain(srd_rate_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, s, dd, -1);
      if (fused)
        chain(dt_cases_kernel<R>, dim3(kblocks), dim3(128), 0, s, dd);
      else
        chain(phase_first_cells_kernel<R, MODEL>, dim3(fblocks), dim3(256), 0, s, dd);
      for (int stage = 1; stage <= 2; ++stage) {
        if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, s, dd, stage);
        stage_seq(stage);
      }
      if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, s, dd, 3);
      chain(phase_commit_kernel, dim3(kblocks), dim3(128), 0, s, dd.ctl, cases, 0, dd.case_lane, dd.lane);
    }
  };
  if (mode == MODE_TRIALS && lanes && lanes->n >= 2) {
    // the other lanes' chains fork off the launch stream and join it at the end
    cudaEventRecord(lanes->fork, st);
    for (int l = 1; l < lanes->n; ++l) cudaStreamWaitEvent(lanes->aux[l - 1], lanes->fork, 0);
    run(lanes->dev[0], st);
    for (int l = 1; l < lanes->n; ++l) run(lanes->dev[l], lanes->aux[l - 1]);
    for (int l = 1; l < lanes->n; ++l) {
      cudaEventRecord(lanes->join[l - 1], lanes->aux[l - 1]);
      cudaStreamWaitEvent(st, lanes->join[l - 1], 0);
    }
  } else {
    run(d, st);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t EngineOps<R>::launch_split(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode,
                                       cudaStream_t stream, int sms, const SplitLanes<R>* lanes) {
  if (model == MODEL_EULER)
    return flux == FLUX_HLLC ? launch_split_t<R, MODEL_EULER, FLUX_HLLC>(d, srd, trials, mode, stream, sms, lanes)
                             : launch_split_t<R, MODEL_EULER, FLUX_AUSM>(d, srd, trials, mode, stream, sms, lanes);
  if (model == MODEL_LAMINAR)
    return flux == FLUX_HLLC ? launch_split_t<R, MODEL_LAMINAR, FLUX_HLLC>(d, srd, trials, mode, stream, sms, lanes)
                             : launch_split_t<R, MODEL_LAMINAR, FLUX_AUSM>(d, srd, trials, mode, stream, sms, lanes);
  return flux == FLUX_HLLC ? launch_split_t<R, MODEL_SA, FLUX_HLLC>(d, srd, trials, mode, stream, sms, lanes)
                           : launch_split_t<R, MODEL_SA, FLUX_AUSM>(d, srd, trials, mode, stream, sms, lanes);
}

template <class R, int MODEL, int FLUX>
static cudaError_t launch_tiled_t(const Dev<R>& d, bool srd, int trials, int mode, cudaStream_t st, int sms) {
  const size_t sm = tiled_smem_bytes<R>();
  const int grid = sms * TiledOcc<R>::blocks;
  const int cases = d.n_cases;
  const int kblocks = (cases + 127) / 128;
  const int fblocks = (int)std::min<long long>((d.ncap + 255) / 256, (long long)sms * 8);
  if (mode == MODE_RESIDUAL) {
    chain(tiled_stage_kernel<R, MODEL, FLUX>, dim3(grid), dim3(BT_THREADS), sm, st, d, STAGE_DIAG);
    return cudaGetLastError();
  }
  chain(phase_commit_kernel, dim3(kblocks), dim3(128), 0, st, d.ctl, cases, 1, (const int*)nullptr, 0);
  for (int t = 0; t < trials; ++t) {
    chain(tiled_stage_kernel<R, MODEL, FLUX>, dim3(grid), dim3(BT_THREADS), sm, st, d, STAGE_BASE);
    if (srd && MODEL >= MODEL_LAMINAR && d.any_srd_rate) chain(srd_rate_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, st, d, -1);
    chain(phase_first_cells_kernel<R, MODEL>, dim3(fblocks), dim3(256), 0, st, d);
    for (int stage = 1; stage <= 2; ++stage) {
      if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, st, d, stage);
      chain(tiled_stage_kernel<R, MODEL, FLUX>, dim3(grid), dim3(BT_THREADS), sm, st, d, stage);
    }
    if (srd) chain(phase_srd_kernel<R, MODEL>, dim3(cases), dim3(MAX_BLOCK), 0, st, d, 3);
    chain(phase_commit_kernel, dim3(kblocks), dim3(128), 0, st, d.ctl, cases, 0, (const int*)nullptr, 0);
  }
  return cudaGetLastError();
}

template <class R>
cudaError_t EngineOps<R>::launch_tiled(const Dev<R>& d, int model, int flux, bool srd, int trials, int mode,
                                       cudaStream_t stream, int sms) {
  if (model == MODEL_EULER)
    return flux == FLUX_HLLC ? launch_tiled_t<R, MODEL_EULER, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                             : launch_tiled_t<R, MODEL_EULER, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
  if (model == MODEL_LAMINAR)
    return flux == FLUX_HLLC ? launch_tiled_t<R, MODEL_LAMINAR, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                             : launch_tiled_t<R, MODEL_LAMINAR, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
  return flux == FLUX_HLLC ? launch_tiled_t<R, MODEL_SA, FLUX_HLLC>(d, srd, trials, mode, stream, sms)
                           : launch_tiled_t<R, MODEL_SA, FLUX_AUSM>(d, srd, trials, mode, stream, sms);
}

template <class R> cudaError_t EngineOps<R>::tiled_setup(int model, int flux) {
  const int bytes = (int)tiled_smem_bytes<R>();
  const void* k;
  if (model == MODEL_EULER)
    k = flux == FLUX_HLLC ? (const void*)tiled_stage_kernel<R, MODEL_EULER, FLUX_HLLC>
                          : (const void*)tiled_stage_kernel<R, MODEL_EULER, FLUX_AUSM>;
  else if (model == MODEL_LAMINAR)
    k = flux == FLUX_HLLC ? (const void*)tiled_stage_kernel<R, MODEL_LAMINAR, FLUX_HLLC>
                          : (const void*)tiled_stage_kernel<R, MODEL_LAMINAR, FLUX_AUSM>;
  else
    k = flux == FLUX_HLLC ? (const void*)tiled_stage_kernel<R, MODEL_SA, FLUX_HLLC>
                          : (const void*)tiled_stage_kernel<R, MODEL_SA, FLUX_AUSM>;
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
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
  // saved state buffers: leading words, then (FP32 form) the trailing words
  const int words = L0_.p ? 2 : 1;
  DevBuf<R> s0, s1;
  uint64_t dummy = 0;
  if (!s0.alloc(words * nv_ * cap_cells_, &dummy, error, "autotune") ||
      !s1.alloc(words * nv_ * cap_cells_, &dummy, error, "autotune"))
    return 1;
  std::vector<CaseCtl> ctl_save(h_ctl_, h_ctl_ + config_.max_cases);
  cudaMemcpyAsync(s0.p, U0_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  cudaMemcpyAsync(s1.p, U1_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  if (L0_.p) {
    cudaMemcpyAsync(s0.p + nv_ * cap_cells_, L0_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
    cudaMemcpyAsync(s1.p + nv_ * cap_cells_, L1_.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  }
  // the tuning runs are not the caller's work: the advance statistics are restored afterwards
  const amr_gpu_stats_t stats_save = stats_;
  double best = 1e30;
  int best_block = block_, best_grid = grid_request_;
  int best_mode = mode_;
  // candidates run the way they run in production: replayed from a CUDA graph when graphs are on
  // (direct launches would penalise the multi-kernel modes by their host launch cost)
  for (int mode : {AMR_B200_LAUNCH_PERSISTENT, AMR_B200_LAUNCH_PHASES, AMR_B200_LAUNCH_SPLIT, AMR_B200_LAUNCH_TILED}) {
    if (mode == AMR_B200_LAUNCH_TILED && !block_tiles_) continue;  // the cases carry no block tiles
    if ((mode == AMR_B200_LAUNCH_PERSISTENT || mode == AMR_B200_LAUNCH_PHASES) && !slot_fluxes_)
      continue;  // the slots carry no owner or geometry
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
        graph_dirty_ = true;  // a new launch configuration needs its own graph
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
  graph_dirty_ = true;
  for (int i = 0; i < config_.max_cases; ++i) refresh_meta(i);
  s0.free();
  s1.free();
  stats_ = stats_save;
  return sync_tiles(error) ? 0 : 1;
}

// Wall-stress rows of one case (reference src/static_amr2d_viscous.cpp:155-160): wall index,
// owner, donor, donor distance, donor viscosity, wall flux x and y per length, signed tangential
// stress, owner pressure, pressure force x/y, viscous force x/y and its moment about the origin.
// Evaluated in double from the accepted state and the viscosity of the last residual pass.
template <class R>
__global__ void export_walls_kernel(Dev<R> d, int cs, int w0, int nw, int cell0, double gamma, double* rows) {
  const long long n = d.ncap;
  const R* U = state_buf(d, d.ctl[cs].cur);
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nw; q += gridDim.x * blockDim.x) {
    const int w = w0 + q;
    const int k = d.w_owner[w], dn = d.w_donor[w];
    const double u0 = U[k], u1 = U[n + k], u2 = U[2 * n + k], u3 = U[3 * n + k];
    const double pressure = (gamma - 1) * (u3 - .5 * (u1 * u1 + u2 * u2) / u0);
    const double nx = d.w_nx[w], ny = d.w_ny[w], len = d.w_len[w], dist = d.w_dist[w];
    const double x = d.w_xm[w], y = d.w_ym[w];
    const double mu = d.mu[dn];
    const double rd = U[dn], ud = U[n + dn] / rd, vd = U[2 * n + dn] / rd;
    double gw[4], fw[4];
    wall_gradient(nx, ny, dist, -ud, -vd, gw);
    visc_flux(mu, gw, nx, ny, 0.0, 0.0, fw);
    const double fx = fw[1] * len, fy = fw[2] * len;
    const double px = pressure * nx * len, py = pressure * ny * len, vx = -fx, vy = -fy;
    double* r = rows + 14 * (long long)q;
    r[0] = q;
    r[1] = k - cell0;
    r[2] = dn - cell0;
    r[3] = dist;
    r[4] = mu;
    r[5] = fx / len;
    r[6] = fy / len;
    r[7] = (-ny * fx + nx * fy) / len;
    r[8] = pressure;
    r[9] = px;
    r[10] = py;
    r[11] = vx;
    r[12] = vy;
    r[13] = x * vy - y * vx;
  }
}

// SA cell rows (reference src/static_amr2d_viscous.cpp:164): nutilde, eddy viscosity, wall distance.
template <class R> __global__ void export_sa_kernel(Dev<R> d, int cs, int c0, int n_cells, double* rows) {
  const long long n = d.ncap;
  const R* U = state_buf(d, d.ctl[cs].cur);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cells; i += gridDim.x * blockDim.x) {
    const int k = c0 + i;
    rows[3 * (long long)i + 0] = (double)U[4 * n + k] / (double)U[k];
    rows[3 * (long long)i + 1] = d.eddy[k];
    rows[3 * (long long)i + 2] = d.c_wd[k];
  }
}

// Convective dt limit of each cell of a case as the reference's snapshot evaluates it
// (src/static_amr2d_viscous.cpp:146-153): primitives p = (gamma-1)(E - rho|v|^2/2), boundary ghost
// states, face rate max(|u_n| + c) * length summed in face order then walls, cfl * A / speed.
// Overwrites the case's convective entries of the last residual pass.
template <class R> __global__ void export_convective_kernel(Dev<R> d, int cs, int c0, int n_cells) {
  const long long n = d.ncap;
  const CaseCfg<R>& cf = d.cfg[cs];
  const R* U = state_buf(d, d.ctl[cs].cur);
  const double g = cf.gamma;
  const auto prim_of = [&](int k, double* w) {
    w[0] = U[k];
    w[1] = (double)U[n + k] / w[0];
    w[2] = (double)U[2 * n + k] / w[0];
    w[3] = (g - 1) * ((double)U[3 * n + k] - .5 * w[0] * (w[1] * w[1] + w[2] * w[2]));
  };
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cells; i += gridDim.x * blockDim.x) {
    const int k = c0 + i;
    double speed = 0;
    const int a = d.c_slot[k], b = d.c_slot[k + 1];
    const int e = b - (d.c_wall[k + 1] - d.c_wall[k]);
    double wk[4];
    prim_of(k, wk);
    for (int q = a; q < e; ++q) {
      const int meta = d.s_meta[q], nb = d.s_nb[q];
      const bool own_left = meta & 1;
      const int axis = (meta >> 1) & 1, side = ((meta >> 2) & 7) - 1, kind = (meta >> 5) & 15;
      double wn[4];
      if (nb >= 0) {
        prim_of(nb, wn);
      } else {
        Bnd<double> bd;
        const Bnd<R>& br = cf.bnd[side];
        bd.kind = br.kind;
        for (int v = 0; v < 4; ++v) bd.ref[v] = br.ref[v];
        bd.total_pressure = br.total_pressure;
        bd.total_temperature = br.total_temperature;
        bd.gas_constant = br.gas_constant;
        bd.dir[0] = br.dir[0];
        bd.dir[1] = br.dir[1];
        bd.outlet_pressure = br.outlet_pressure;
        bd.wall_velocity[0] = br.wall_velocity[0];
        bd.wall_velocity[1] = br.wall_velocity[1];
        bc_state(bd, kind, g, side, wk, wn);
      }
      const double* l = own_left ? wk : wn;
      const double* r = own_left ? wn : wk;
      const double ra = fabs(l[1 + axis]) + sqrt(g * l[3] / l[0]), rb = fabs(r[1 + axis]) + sqrt(g * r[3] / r[0]);
      speed += (ra < rb ? rb : ra) * (double)d.s_len[q];
    }
    for (int q = e; q < b; ++q) speed += sqrt(g * wk[3] / wk[0]) * (double)d.s_len[q];
    d.ddt[k] = speed > 0 ? cf.cfl * d.c_area[k] / speed : __longlong_as_double(0x7FF0000000000000ll);
  }
}

// Smallest convective and viscous dt limit over a case's cells (min is order-free).
template <class R> __global__ void export_limits_kernel(Dev<R> d, int c0, int n_cells, double* out) {
  __shared__ double sc[256], sv[256];
  const double inf = __longlong_as_double(0x7FF0000000000000ll);
  double c = inf, v = inf;
  for (int i = threadIdx.x; i < n_cells; i += blockDim.x) {
    c = fmin(c, d.ddt[c0 + i]);
    v = fmin(v, d.ddt[d.ncap + c0 + i]);
  }
  sc[threadIdx.x] = c;
  sv[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      sc[threadIdx.x] = fmin(sc[threadIdx.x], sc[threadIdx.x + s]);
      sv[threadIdx.x] = fmin(sv[threadIdx.x], sv[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sc[0];
    out[1] = sv[0];
  }
}

template <class R>
int Batch<R>::export_case(int slot, double* wall_rows, uint64_t wall_count, double* sa_rows, uint64_t sa_count,
                          double* limits, std::string* error) {
  if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return fail1(error, "no such case");
  const HostCase<R>& hc = cases_[slot];
  const long long n = hc.n, nw = hc.walls.n;
  const uint64_t want_walls = model_ >= MODEL_LAMINAR ? 14 * (uint64_t)nw : 0;
  const uint64_t want_sa = model_ == MODEL_SA ? 3 * (uint64_t)n : 0;
  if ((want_walls && !wall_rows) || wall_count != want_walls || (want_sa && !sa_rows) || sa_count != want_sa || !limits)
    return fail1(error, "export buffer sizes do not match the case (14 per wall for viscous models, 3 per cell for SA)");
  if (residual(error)) return 1;
  const uint64_t need = want_walls + want_sa + 2;
  if (ex_buf_.n < need) {
    ex_buf_.free();
    uint64_t dummy = 0;
    if (!ex_buf_.alloc(need, &dummy, error, "export")) return 1;
  }
  const Dev<R> d = dev();
  const int c0 = (int)hc.cells.b;
  double* dev_walls = ex_buf_.p;
  double* dev_sa = ex_buf_.p + want_walls;
  double* dev_lim = ex_buf_.p + want_walls + want_sa;
  if (want_walls && nw > 0)
    export_walls_kernel<R><<<(int)((nw + 127) / 128), 128, 0, stream_>>>(d, slot, (int)hc.walls.b, (int)nw, c0,
                                                                        (double)hc.cfg.gamma, dev_walls);
  if (want_sa) export_sa_kernel<R><<<(int)((n + 255) / 256), 256, 0, stream_>>>(d, slot, c0, (int)n, dev_sa);
  export_convective_kernel<R><<<(int)((n + 127) / 128), 128, 0, stream_>>>(d, slot, c0, (int)n);
  if (hc.cfg.srd_rate) {  // the snapshot's viscous dt is the SRD-mapped one
    if (model_ == MODEL_LAMINAR) srd_rate_kernel<R, MODEL_LAMINAR><<<config_.max_cases, MAX_BLOCK, 0, stream_>>>(d, slot);
    if (model_ == MODEL_SA) srd_rate_kernel<R, MODEL_SA><<<config_.max_cases, MAX_BLOCK, 0, stream_>>>(d, slot);
  }
  export_limits_kernel<R><<<1, 256, 0, stream_>>>(d, c0, (int)n, dev_lim);
  bool ok = cuda_ok(cudaGetLastError(), error, "export launch");
  launches_ += (want_walls && nw > 0) + (want_sa ? 1 : 0) + 2;
  if (ok && want_walls)
    ok = cuda_ok(cudaMemcpyAsync(wall_rows, dev_walls, sizeof(double) * want_walls, cudaMemcpyDeviceToHost, stream_),
                 error, "export copy");
  if (ok && want_sa)
    ok = cuda_ok(cudaMemcpyAsync(sa_rows, dev_sa, sizeof(double) * want_sa, cudaMemcpyDeviceToHost, stream_), error,
                 "export copy");
  ok = ok && cuda_ok(cudaMemcpyAsync(limits, dev_lim, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream_), error,
                     "export copy") &&
       cuda_ok(cudaStreamSynchronize(stream_), error, "export sync");
  if (ok) stats_.state_d2h_bytes += sizeof(double) * need;
  return ok ? 0 : 1;
}

template <class R>
void Batch<R>::restore(const std::vector<CaseCtl>& ctl_save, const DevBuf<R>& s0, const DevBuf<R>& s1, long long nbytes) {
  std::copy(ctl_save.begin(), ctl_save.end(), h_ctl_);
  cudaMemcpyAsync(ctl_.p, h_ctl_, sizeof(CaseCtl) * config_.max_cases, cudaMemcpyHostToDevice, stream_);
  cudaMemcpyAsync(U0_.p, s0.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  cudaMemcpyAsync(U1_.p, s1.p, nbytes, cudaMemcpyDeviceToDevice, stream_);
  if (L0_.p) {
    cudaMemcpyAsync(L0_.p, s0.p + nv_ * cap_cells_, nbytes, cudaMemcpyDeviceToDevice, stream_);
    cudaMemcpyAsync(L1_.p, s1.p + nv_ * cap_cells_, nbytes, cudaMemcpyDeviceToDevice, stream_);
  }
  cudaStreamSynchronize(stream_);
}

}  // namespace amrb
