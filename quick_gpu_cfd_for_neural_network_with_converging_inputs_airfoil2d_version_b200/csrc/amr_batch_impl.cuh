// amr_batch_impl.cuh -- the batch arena and its launches, templated on the state precision.
//
// A Batch owns device tables sized at creation (cells, slots, walls, gradient terms, SRD
// lists, cases, tiles).  Admission converts one reference-layout mesh into the engine layout
// (amr_engine.cuh) inside free ranges of those tables; release returns the ranges.  Advance
// replays one cooperative launch of the persistent trial kernel plus the control read-back,
// captured in a CUDA graph that is recaptured whenever the case set changes.
#pragma once
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "amr_engine.cuh"
#include "amr_host.h"

namespace amrb {

inline bool cuda_ok(cudaError_t st, std::string* error, const char* what) {
  if (st == cudaSuccess) return true;
  if (error) *error = std::string(what) + ": " + cudaGetErrorString(st);
  return false;
}

// First-fit allocator of index ranges.
class RangeAlloc {
 public:
  explicit RangeAlloc(long long capacity = 0) : capacity_(capacity) {
    if (capacity > 0) free_[0] = capacity;
  }
  long long alloc(long long n) {
    if (n <= 0) return 0;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const long long b = it->first, size = it->second;
        free_.erase(it);
        if (size > n) free_[b + n] = size - n;
        return b;
      }
    }
    return -1;
  }
  void release(long long b, long long n) {
    if (n <= 0) return;
    auto it = free_.emplace(b, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  long long free_total() const {
    long long s = 0;
    for (auto& kv : free_) s += kv.second;
    return s;
  }
  long long capacity() const { return capacity_; }

 private:
  long long capacity_;
  std::map<long long, long long> free_;
};

// One device allocation carved into a batch's tables.  Each cudaMalloc of a few MB or more costs
// about 0.3 ms whatever its size, and a batch has some 80 tables, so a batch's creation sizes them
// all in a planning pass, makes one allocation and carves it in a second pass (256-byte aligned).
struct Slab {
  char* base = nullptr;
  size_t used = 0;
  bool planning = true;
  void* take(size_t bytes) {
    const size_t off = used;
    used += (bytes + 255) & ~size_t(255);
    return planning ? nullptr : base + off;
  }
};
// The slab that DevBuf::alloc carves from on this host thread (none outside a batch's creation).
inline thread_local Slab* g_slab = nullptr;
struct SlabScope {
  explicit SlabScope(Slab* s) { g_slab = s; }
  ~SlabScope() { g_slab = nullptr; }
};

template <class T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  bool owned = false;  // allocated by itself (else carved from a slab)
  bool alloc(size_t count, uint64_t* counter, std::string* error, const char* what) {
    n = count ? count : 1;
    if (g_slab) {
      p = static_cast<T*>(g_slab->take(n * sizeof(T)));
      owned = false;
      if (!g_slab->planning && counter) *counter += n * sizeof(T);
      return true;
    }
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)), error, what)) return false;
    owned = true;
    if (counter) *counter += n * sizeof(T);
    return true;
  }
  void free() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    owned = false;
  }
};

// Page-locked host memory shared by every batch of the process and lent for the length of one
// call: admissions stage their tables in it and downloads land in it.  Page-locking runs at about
// 1 GB/s, longer than preparing and filling a bulk admission of a few hundred cases takes, so a
// block once locked is kept when given back (idle blocks up to 1 GB) and lent again.  Lending
// and giving back are thread-safe.  The pool is never destroyed: the runtime may be gone at exit.
class PinnedPool {
 public:
  struct Lease {
    char* p = nullptr;
    size_t size = 0;
    bool fresh = false;  // page-locked for this lease
  };
  static PinnedPool& get() {
    static PinnedPool* pool = new PinnedPool();
    return *pool;
  }
  // The idle block that fits `want` most tightly, else the largest idle one of at least
  // `least`, else a newly page-locked block of `want` bytes; an empty lease if that fails.
  Lease lend(size_t least, size_t want) {
    {
      std::lock_guard<std::mutex> hold(m_);
      int best = -1;
      for (int i = 0; i < (int)idle_.size(); ++i)
        if (idle_[i].size >= want && (best < 0 || idle_[i].size < idle_[best].size)) best = i;
      if (best < 0)
        for (int i = 0; i < (int)idle_.size(); ++i)
          if (idle_[i].size >= least && (best < 0 || idle_[i].size > idle_[best].size)) best = i;
      if (best >= 0) {
        Lease l = idle_[best];
        l.fresh = false;
        idle_.erase(idle_.begin() + best);
        idle_bytes_ -= l.size;
        return l;
      }
    }
    Lease l;
    if (cudaHostAlloc(reinterpret_cast<void**>(&l.p), want, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return Lease();
    }
    l.size = want;
    l.fresh = true;
    return l;
  }
  // Takes a lease back (no copy from or to it may be in flight); frees the oldest idle blocks
  // beyond the cap.
  void give_back(const Lease& l) {
    if (!l.p) return;
    std::vector<Lease> drop;
    {
      std::lock_guard<std::mutex> hold(m_);
      idle_.push_back(l);
      idle_bytes_ += l.size;
      while (idle_bytes_ > kKeep && !idle_.empty()) {
        drop.push_back(idle_.front());
        idle_bytes_ -= idle_.front().size;
        idle_.erase(idle_.begin());
      }
    }
    for (const Lease& d : drop) cudaFreeHost(d.p);
  }

 private:
  static constexpr size_t kKeep = size_t(1) << 30;
  std::mutex m_;
  std::vector<Lease> idle_;
  size_t idle_bytes_ = 0;
};

// A lease given back when the holder's scope ends, after the holder's stream has drained (so no
// copy into it is still in flight on an error path).
struct LeaseGuard {
  cudaStream_t stream;
  PinnedPool::Lease lease;
  LeaseGuard(cudaStream_t s, const PinnedPool::Lease& l) : stream(s), lease(l) {}
  LeaseGuard(const LeaseGuard&) = delete;
  LeaseGuard& operator=(const LeaseGuard&) = delete;
  ~LeaseGuard() {
    if (!lease.p) return;
    cudaStreamSynchronize(stream);
    PinnedPool::get().give_back(lease);
  }
};

// Host staging of one admission (or one download).  Tables are built straight into
// page-locked blocks by a bump allocator that is reset per call, so an upload needs no
// host-side copy: one DMA per used block into a device staging buffer laid out like the
// blocks, then one kernel scatters each table to its range.  The first block is normally a
// slice of the batch's staging arena (adopt); further blocks are allocated on demand and stay
// for the batch's lifetime; a block whose page-locked allocation fails is plain heap memory
// (correct, only a slower copy).
class PinnedStage {
 public:
  struct Block {
    char* p;
    size_t size, used, dev;  // dev: offset of the block in the device staging buffer
    bool pinned, owned;
  };
  ~PinnedStage() { release(); }
  // Replaces every block by caller-owned page-locked memory [p, p + size) (none if size is 0).
  void adopt(char* p, size_t size) {
    release();
    if (!p || !size) return;
    blocks_.push_back({p, size, 0, 0, true, false});
    total_ = size;
  }
  void reset() {
    for (Block& b : blocks_) b.used = 0;
    cur_ = 0;
  }
  void* take(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    while (cur_ < blocks_.size() && blocks_[cur_].used + bytes > blocks_[cur_].size) ++cur_;
    if (cur_ == blocks_.size()) {
      const size_t size = std::max(bytes, blocks_.empty() ? size_t(8) << 20 : 2 * blocks_.back().size);
      void* p = nullptr;
      bool pinned = cudaHostAlloc(&p, size, cudaHostAllocDefault) == cudaSuccess;
      if (!pinned) {
        cudaGetLastError();
        p = std::malloc(size);
        if (!p) throw std::bad_alloc();
      }
      blocks_.push_back({static_cast<char*>(p), size, 0, total_, pinned, true});
      total_ += size;
      if (pinned) pinned_ += size;
    }
    Block& b = blocks_[cur_];
    void* p = b.p + b.used;
    b.used += bytes;
    return p;
  }
  // offset in the device staging buffer of a host address inside a block, or -1
  long long dev_offset(const void* host) const {
    const char* h = static_cast<const char*>(host);
    for (const Block& b : blocks_)
      if (h >= b.p && h < b.p + b.size) return (long long)(b.dev + (size_t)(h - b.p));
    return -1;
  }
  const std::vector<Block>& blocks() const { return blocks_; }
  size_t total() const { return total_; }
  size_t pinned_bytes() const { return pinned_; }

 private:
  void release() {
    for (Block& b : blocks_)
      if (b.owned) b.pinned ? (void)cudaFreeHost(b.p) : std::free(b.p);
    blocks_.clear();
    cur_ = 0;
    total_ = 0;
  }
  std::vector<Block> blocks_;
  size_t cur_ = 0, total_ = 0, pinned_ = 0;
};

template <class T> struct PinAlloc {
  using value_type = T;
  PinnedStage* stage;
  explicit PinAlloc(PinnedStage* s) : stage(s) {}
  template <class U> PinAlloc(const PinAlloc<U>& o) : stage(o.stage) {}
  T* allocate(size_t n) { return static_cast<T*>(stage->take(n * sizeof(T))); }
  void deallocate(T*, size_t) {}  // released all at once by PinnedStage::reset
  template <class U> void construct(U* p) { ::new (static_cast<void*>(p)) U; }  // default-initialised
  template <class U, class A0, class... A> void construct(U* p, A0&& a0, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A0>(a0), std::forward<A>(a)...);
  }
  template <class U> bool operator==(const PinAlloc<U>& o) const { return stage == o.stage; }
  template <class U> bool operator!=(const PinAlloc<U>& o) const { return stage != o.stage; }
};
template <class T> using PVec = std::vector<T, PinAlloc<T>>;

// One scatter launch moves up to UPLOAD_TABLES tables from the device staging buffer.
constexpr int UPLOAD_TABLES = 64;
struct UploadTable {
  unsigned long long dst[UPLOAD_TABLES], src[UPLOAD_TABLES], bytes[UPLOAD_TABLES];
  int n;
};

// A uniform start state on the device: every cell of a case's range [c0, c0 + n) gets the
// conserved values hi[v] (and, in the FP32 form, the trailing words lo[v]); the case's padding
// cell c0 + n gets 1 and 0, as a staged state does.
template <class R> struct UniformState {
  R hi[5], lo[5];
};
template <class R>
static __global__ void fill_uniform_kernel(R* U, R* L, long long cap, int c0, int n, int nv, UniformState<R> w) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x)
    for (int v = 0; v < nv; ++v) {
      U[v * cap + c0 + k] = k < n ? w.hi[v] : R(1);
      if (L) L[v * cap + c0 + k] = k < n ? w.lo[v] : R(0);
    }
}

// blockIdx.y picks the table; the copy width is the widest of 8, 4 or 1 bytes that divides
// both addresses and the size.
static __global__ void scatter_uploads_kernel(const unsigned char* __restrict__ stage, UploadTable t) {
  const int i = blockIdx.y;
  if (i >= t.n) return;
  unsigned char* dst = reinterpret_cast<unsigned char*>(t.dst[i]);
  const unsigned char* src = stage + t.src[i];
  const unsigned long long nb = t.bytes[i];
  const unsigned long long a = t.dst[i] | reinterpret_cast<unsigned long long>(src) | nb;
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  if ((a & 7) == 0) {
    for (unsigned long long w = tid; w < nb / 8; w += stride)
      reinterpret_cast<unsigned long long*>(dst)[w] = reinterpret_cast<const unsigned long long*>(src)[w];
  } else if ((a & 3) == 0) {
    for (unsigned long long w = tid; w < nb / 4; w += stride)
      reinterpret_cast<unsigned int*>(dst)[w] = reinterpret_cast<const unsigned int*>(src)[w];
  } else {
    for (unsigned long long w = tid; w < nb; w += stride) dst[w] = src[w];
  }
}

struct Range {
  long long b = 0, n = 0;
};

template <class R> struct HostCase {
  bool live = false;
  int n = 0;
  Range cells, slots, walls, terms, groups, gmembers, qcells, qlist, faces, halo, tfaces;
  int slot = -1;
  std::vector<int> nslot, nterm;  // per-cell slot and gradient-term counts (for tiling)
  std::vector<int> slot_prefix, term_prefix;  // n+1 running sums of nslot / nterm
  std::vector<Tile> tiles;
  std::vector<BTile> btiles;  // block tiles (tiled mode), global indices
  CaseCfg<R> cfg;
};

template <class R> class Batch final : public BatchBase {
 public:
  Batch() = default;
  ~Batch() override { destroy(); }

  // The batch's device tables (DevBuf::alloc carves them from the slab in scope).
  bool alloc_tables(const amr_batch_config_t& c, std::string* error) {
    uint64_t* A = &stats_.allocated_bytes;
    const long long nc = cap_cells_;
    bool ok = lane_ranges_.alloc(8 * MAX_LANES, A, error, "lanes") && case_lane_.alloc(c.max_cases, A, error, "lanes") &&
              ctl_.alloc(c.max_cases, A, error, "ctl") && cfg_.alloc(c.max_cases, A, error, "cfg") &&
              tiles_.alloc(cap_tiles_, A, error, "tiles") && bar_.alloc(1, A, error, "barrier") &&
              c_case_.alloc(nc, A, error, "cells") && c_vol_.alloc(nc, A, error, "cells") &&
              c_area_.alloc(nc, A, error, "cells") && c_gvol_.alloc(nc, A, error, "cells") &&
              c_flags_.alloc(nc, A, error, "cells") && c_slot_.alloc(nc, A, error, "cells") &&
              c_wall_.alloc(nc, A, error, "cells") && c_term_.alloc(nc, A, error, "cells") &&
              c_cx_.alloc(nc, A, error, "cells") && c_cy_.alloc(nc, A, error, "cells") &&
              s_own_.alloc(slot_fluxes_ ? cap_slots_ : 0, A, error, "slots") && s_nb_.alloc(cap_slots_, A, error, "slots") &&
              s_meta_.alloc(cap_slots_, A, error, "slots") && s_len_.alloc(cap_slots_, A, error, "slots") &&
              w_nx_.alloc(cap_walls_, A, error, "walls") && w_ny_.alloc(cap_walls_, A, error, "walls") &&
              w_len_.alloc(cap_walls_, A, error, "walls") && w_dist_.alloc(cap_walls_, A, error, "walls") &&
              w_donor_.alloc(cap_walls_, A, error, "walls") && w_xm_.alloc(cap_walls_, A, error, "walls") &&
              w_ym_.alloc(cap_walls_, A, error, "walls") &&
              g_mem_.alloc(cap_groups_ + c.max_cases, A, error, "srd") && g_cell_.alloc(cap_gmem_, A, error, "srd") &&
              g_cnt_.alloc(cap_gmem_, A, error, "srd") && g_vol_.alloc(cap_groups_ + c.max_cases, A, error, "srd") &&
              q_cell_.alloc(cap_q_ + c.max_cases, A, error, "srd") && q_grp_.alloc(cap_q_ + c.max_cases, A, error, "srd") &&
              q_list_.alloc(cap_qlist_, A, error, "srd") && q_cnt_.alloc(cap_q_ + c.max_cases, A, error, "srd") &&
              qhat_.alloc(4 * (cap_groups_ + c.max_cases), A, error, "srd") &&
              U0_.alloc(nv_ * nc, A, error, "state") && U1_.alloc(nv_ * nc, A, error, "state") &&
              U2_.alloc(nv_ * nc, A, error, "state") && R0_.alloc(nv_ * nc, A, error, "state") &&
              diag_part_.alloc(9 * cap_tiles_, A, error, "diag") && diag_out_.alloc(9 * c.max_cases, A, error, "diag") &&
              diag_cfg_.alloc(7 * c.max_cases, A, error, "diag") && case_tiles_.alloc(2 * c.max_cases, A, error, "diag") &&
              ddt_.alloc(2 * nc, A, error, "diag");
    if (!ok) return false;
    if (sizeof(R) == 4 && !(L0_.alloc(nv_ * nc, A, error, "state") && L1_.alloc(nv_ * nc, A, error, "state")))
      return false;
    if (sizeof(R) == 4 && model_ == MODEL_SA &&
        !(fsa_.alloc(cap_faces_, A, error, "faces") && wsa_.alloc(cap_walls_, A, error, "walls")))
      return false;
    if (!s_geo_.alloc(slot_fluxes_ ? 6 * cap_slots_ : 0, A, error, "slots")) return false;
    // face and wall records of the split launch mode
    ok = s_item_.alloc(cap_slots_, A, error, "slots") && f_case_.alloc(cap_faces_, A, error, "faces") &&
         f_own_.alloc(cap_faces_, A, error, "faces") && f_nb_.alloc(cap_faces_, A, error, "faces") &&
         f_meta_.alloc(cap_faces_, A, error, "faces") && f_len_.alloc(cap_faces_, A, error, "faces") &&
         f_geo_.alloc(6 * cap_faces_, A, error, "faces") && fval_.alloc(rec_stride() * cap_faces_, A, error, "faces") &&
         w_owner_.alloc(cap_walls_, A, error, "walls") && wval_.alloc(rec_stride() * cap_walls_, A, error, "walls") &&
         live_end_.alloc(4, A, error, "ranges") && btiles_.alloc(cap_btiles_, A, error, "block tiles") &&
         bt_halo_.alloc(cap_halo_, A, error, "block tiles") && bt_face_.alloc(cap_tface_, A, error, "block tiles") &&
         bt_floc_.alloc(cap_tface_, A, error, "block tiles") &&
         s_loc_.alloc(block_tiles_ ? cap_slots_ : 0, A, error, "slots") &&
         w_ldon_.alloc(block_tiles_ ? cap_walls_ : 0, A, error, "walls");
    if (!ok) return false;
    if (model_ >= MODEL_LAMINAR) {
      ok = crec_.alloc(CREC * nc, A, error, "scratch") && t_own_.alloc(slot_fluxes_ ? cap_terms_ : 0, A, error, "terms") &&
           t_src_.alloc(cap_terms_, A, error, "terms") && t_x_.alloc(cap_terms_, A, error, "terms") &&
           t_y_.alloc(cap_terms_, A, error, "terms") && grad_.alloc(4 * nc, A, error, "scratch") &&
           mu_.alloc(nc, A, error, "scratch") && eddy_.alloc(nc, A, error, "scratch");
      if (!ok) return false;
    }
    if (model_ == MODEL_SA) {
      ok = c_wd_.alloc(nc, A, error, "cells") && sgrad_.alloc(2 * nc, A, error, "scratch") &&
           sdiff_.alloc(nc, A, error, "scratch") && ssrc_.alloc(nc, A, error, "scratch") &&
           srate_.alloc(nc, A, error, "scratch");
      if (!ok) return false;
    }
    return true;
  }

  bool init(const amr_batch_config_t& c, std::string* error) {
    config_ = c;
    model_ = c.model == AMR_B200_MODEL_EULER ? MODEL_EULER : (c.sa_model ? MODEL_SA : MODEL_LAMINAR);
    flux_ = c.flux == AMR_B200_FLUX_AUSMPUP ? FLUX_AUSM : FLUX_HLLC;
    nv_ = model_ == MODEL_SA ? 5 : 4;
    if (c.max_cases < 1) return fail(error, "max_cases must be positive");
    if (!cuda_ok(cudaSetDevice(c.device), error, "cudaSetDevice")) return false;
    int coop = 0;  // single attribute queries (a full property query costs milliseconds)
    if (!cuda_ok(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, c.device), error, "device attributes") ||
        !cuda_ok(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c.device), error, "device attributes"))
      return false;
    clock_khz_ = 1965000;
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrClockRate, c.device) == cudaSuccess && v > 0) clock_khz_ = v;
    if (!coop) return fail(error, "device lacks cooperative launch");
    long long cells = c.max_cells, slots = c.max_faces, walls = c.max_walls, terms = c.max_terms, srd = c.max_srd;
    if (cells == 0) {
      // size from the HBM budget: ~bytes per cell of tables and state for this model
      const double per_cell = (model_ == MODEL_EULER ? 260.0 : 520.0) * sizeof(R) / 4.0 + 120.0;
      const uint64_t budget = c.hbm_bytes ? c.hbm_bytes : (uint64_t)4 << 30;
      cells = (long long)(budget / per_cell);
    }
    const bool auto_faces = slots == 0;
    if (slots == 0) slots = 5 * cells;
    if (walls == 0) walls = cells / 8 + 64 * c.max_cases;
    if (terms == 0) terms = model_ == MODEL_EULER ? 1 : 6 * cells;
    if (srd == 0) srd = cells / 8 + 64 * c.max_cases;
    cap_cells_ = cells + c.max_cases;  // one closing entry per case
    cap_slots_ = slots;
    // every face is listed by at least one cell, so the slot count bounds the faces; a sized-from-
    // cells arena assumes instead the ~2 faces per cell of 2-D quadtree meshes (2.5 with margin)
    cap_faces_ = auto_faces ? std::min<long long>(slots, 5 * cells / 2 + 64ll * c.max_cases) : slots;
    cap_walls_ = walls;
    if (cap_faces_ >= (1ll << 30) || cap_walls_ >= (1ll << 30)) return fail(error, "arena too large for 32-bit record indices");
    cap_terms_ = std::max<long long>(terms, 1);
    cap_groups_ = srd;
    cap_gmem_ = 8 * srd;
    cap_q_ = 2 * srd;
    cap_qlist_ = 8 * srd;
    cap_tiles_ = cap_cells_ / 2 + 4 * c.max_cases;  // a tile holds at least one cell, normally 5-10
    a_cells_ = RangeAlloc(cap_cells_);
    a_slots_ = RangeAlloc(cap_slots_);
    a_faces_ = RangeAlloc(cap_faces_);
    // block tiles serve only the tiled mode, which a batch reaches by asking for it or by autotuning
    block_tiles_ = c.launch_mode == AMR_B200_LAUNCH_AUTO || c.launch_mode == AMR_B200_LAUNCH_TILED;
    // per-slot owner and geometry serve only the persistent and phase modes
    slot_fluxes_ = c.launch_mode == AMR_B200_LAUNCH_AUTO || c.launch_mode == AMR_B200_LAUNCH_PERSISTENT ||
                   c.launch_mode == AMR_B200_LAUNCH_PHASES;
    cap_halo_ = block_tiles_ ? 2 * cap_cells_ : 0;
    cap_tface_ = block_tiles_ ? 2 * cap_faces_ + 64 : 0;
    cap_btiles_ = block_tiles_ ? cap_cells_ / 16 + 4 * (long long)c.max_cases : 0;
    a_halo_ = RangeAlloc(cap_halo_);
    a_tface_ = RangeAlloc(cap_tface_);
    a_walls_ = RangeAlloc(cap_walls_);
    a_terms_ = RangeAlloc(cap_terms_);
    a_groups_ = RangeAlloc(cap_groups_ + c.max_cases);
    a_gmem_ = RangeAlloc(cap_gmem_);
    a_q_ = RangeAlloc(cap_q_ + c.max_cases);
    a_qlist_ = RangeAlloc(cap_qlist_);
    cases_.assign(c.max_cases, HostCase<R>());
    meta_.assign(c.max_cases, CaseMeta{});
    reserved_.assign(c.max_cases, 0);
    stagers_.clear();
    stagers_.emplace_back(new Stager());
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), error, "stream")) return false;
    // the split mode's other lanes: their streams and the events that fork them off and join them
    if (!cuda_ok(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), error, "event")) return false;
    for (int l = 0; l < MAX_LANES - 1; ++l)
      if (!cuda_ok(cudaStreamCreateWithFlags(&aux_[l], cudaStreamNonBlocking), error, "stream") ||
          !cuda_ok(cudaEventCreateWithFlags(&join_[l], cudaEventDisableTiming), error, "event"))
        return false;
    if (!cuda_ok(cudaEventCreate(&ev0_), error, "event") || !cuda_ok(cudaEventCreate(&ev1_), error, "event")) return false;
    // every table in one slab: a planning pass sizes them, one allocation, a carving pass
    Slab slab;
    {
      const SlabScope scope(&slab);
      if (!alloc_tables(c, error)) return false;
    }
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&slab_), slab.used), error, "tables")) return false;
    slab.base = slab_;
    slab.used = 0;
    slab.planning = false;
    {
      const SlabScope scope(&slab);
      if (!alloc_tables(c, error)) return false;
    }
    const long long nc = cap_cells_;
    cudaMemsetAsync(ctl_.p, 0, sizeof(CaseCtl) * c.max_cases, stream_);
    cudaMemsetAsync(c_case_.p, 0xff, sizeof(int) * nc, stream_);
    cudaMemsetAsync(f_case_.p, 0xff, sizeof(int) * cap_faces_, stream_);
    cudaMemsetAsync(w_owner_.p, 0xff, sizeof(int) * cap_walls_, stream_);
    cudaMemsetAsync(live_end_.p, 0, sizeof(int) * 4, stream_);
    if (!cuda_ok(cudaHostAlloc(reinterpret_cast<void**>(&h_ctl_), sizeof(CaseCtl) * c.max_cases, cudaHostAllocDefault), error,
                 "pinned control") ||
        !cuda_ok(cudaHostAlloc(reinterpret_cast<void**>(&h_bar_), sizeof(GridBarrier), cudaHostAllocDefault), error,
                 "pinned barrier"))
      return false;
    std::memset(h_ctl_, 0, sizeof(CaseCtl) * c.max_cases);
    std::memset(h_bar_, 0, sizeof(GridBarrier));
    cudaMemsetAsync(bar_.p, 0, sizeof(GridBarrier), stream_);
    stats_.pinned_bytes += sizeof(CaseCtl) * c.max_cases + sizeof(GridBarrier);
    block_ = c.block_threads > 0 ? c.block_threads : 256;
    if (block_ % 32 || block_ < 64 || block_ > MAX_BLOCK) return fail(error, "block_threads must be 64..256, a multiple of 32");
    grid_request_ = c.grid_blocks;
    if (c.launch_mode < AMR_B200_LAUNCH_AUTO || c.launch_mode > AMR_B200_LAUNCH_TILED)
      return fail(error, "unknown launch mode");
    if (!cuda_ok(EngineOps<R>::tiled_setup(model_, flux_), error, "tiled kernel shared memory")) return false;
    mode_ = c.launch_mode == AMR_B200_LAUNCH_AUTO ? AMR_B200_LAUNCH_PERSISTENT : c.launch_mode;
    if (mode_ != AMR_B200_LAUNCH_PERSISTENT && block_ != PHASE_BLOCK)
      return fail(error, "the phase, split and tiled launch modes take block_threads 128");
    if (!configure_grid(error)) return false;
    return cuda_ok(cudaStreamSynchronize(stream_), error, "batch init");
  }

  int admit(const amr_mesh_view_t* m, const amr_params_t* p, const double* u0, uint64_t u0_count, double time0,
            long long steps0, long long rejected0, double target, long long maxsteps, int* slot_out,
            std::string* error) override {
    AdmitSpec s{m, p, u0, u0_count, time0, target, steps0, rejected0, maxsteps};
    std::vector<int> slots, status;
    std::vector<std::string> errors;
    admit_many(std::vector<AdmitSpec>{s}, 1, &slots, &status, &errors);
    if (status[0] == 1 && error) *error = errors[0];
    if (status[0] == 0) *slot_out = slots[0];
    return status[0];
  }

  // Admission in four stages: prepare (case-local tables and checks; parallel), reserve (slot
  // and arena ranges; serial, in request order, so placement does not depend on the thread
  // count), fill (engine tables in page-locked staging and their upload; parallel, one staging
  // area per worker) and commit (controls, one stream synchronisation, host bookkeeping).
  int admit_many(const std::vector<AdmitSpec>& specs, int threads, std::vector<int>* slots, std::vector<int>* status,
                 std::vector<std::string>* errors) override {
    const size_t count = specs.size();
    slots->assign(count, -1);
    status->assign(count, 0);
    errors->assign(count, std::string());
    // preparing and filling 256 cases: 30 + 41 ms on 8 threads, 19 + 30 ms on 16, no gain beyond
    if (threads <= 0) threads = (int)std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
    threads = (int)std::max<size_t>(1, std::min<size_t>((size_t)threads, count));
    while ((int)stagers_.size() < threads) stagers_.emplace_back(new Stager());
    // The staging arena, sized by a bound over every request, is allocated on a helper thread
    // while the first cases are prepared (page-locking runs at about a GB/s).
    size_t bound = 0;
    for (const AdmitSpec& sp : specs) bound = std::max(bound, staged_bound(sp));
    // If it fails, the stages allocate their own blocks, as for a case above the bound.
    std::thread arena_thread;
    if (bound) {
      try {
        arena_thread = std::thread([&] {
          cudaSetDevice(config_.device);
          std::string ignored;
          if (!ensure_arena(threads, bound, &ignored)) cudaGetLastError();
        });
      } catch (const std::system_error&) {
        std::string ignored;
        if (!ensure_arena(threads, bound, &ignored)) cudaGetLastError();
      }
    }
    // chunks bound the host memory of prepared cases
    const size_t chunk = std::max<size_t>(32, 4 * (size_t)threads);
    bool invalid = false, full = false;
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
      const size_t c1 = std::min(count, c0 + chunk);
      std::vector<AdmitJob> jobs(c1 - c0);
      for (size_t i = c0; i < c1; ++i) jobs[i - c0].spec = specs[i];
      parallel_for(jobs.size(), threads, [&](size_t i, int) { guarded(jobs[i], [&] { prepare(jobs[i]); }); });
      for (AdmitJob& j : jobs)
        if (j.status == 0) guarded(j, [&] { reserve(j); });
      if (arena_thread.joinable()) arena_thread.join();
      parallel_for(jobs.size(), threads, [&](size_t i, int w) {
        if (jobs[i].status == 0) guarded(jobs[i], [&] { fill(jobs[i], *stagers_[w]); });
      });
      commit(jobs);
      for (size_t i = c0; i < c1; ++i) {
        AdmitJob& j = jobs[i - c0];
        (*status)[i] = j.status;
        (*slots)[i] = j.status == 0 ? j.slot : -1;
        (*errors)[i] = j.error;
        invalid = invalid || j.status == 1;
        full = full || j.status == 3;
      }
    }
    if (arena_thread.joinable()) arena_thread.join();
    return_arena_host();  // every admission above ended synchronised
    return invalid ? 1 : (full ? 3 : 0);
  }

  // One admission in flight: its request, the case-local tables prepare() builds, the slot and
  // ranges reserve() gives it, and its outcome (0 admitted, 1 invalid input, 3 no room).
  struct AdmitJob {
    AdmitSpec spec{};
    long long n = 0, nw = 0, ns = 0, nt = 0, nf = 0, ng = 0, gmem = 0, qlist = 0;
    bool has_srd = false;
    int kinds[4] = {0, 0, 0, 0};
    std::vector<unsigned char> simple;
    std::vector<int> group_index, rec, bt_halo, bt_face, s_loc, w_ldon;
    std::vector<long long> nontrivial;  // cells (and groups) with a non-trivial SRD neighbourhood
    std::vector<int2> bt_floc;
    HostCase<R> hc;
    int slot = -1;
    bool reserved = false;
    CaseCtl ctl{};
    uint64_t geometry_bytes = 0, state_bytes = 0;
    int status = 0;
    std::string error;
  };

  struct Upload {
    unsigned long long dst, src, bytes;
  };

  // A worker's staging: page-locked host blocks, their device copy and the pending uploads.
  struct Stager {
    PinnedStage stage;
    std::vector<Upload> uploads;
    DevBuf<unsigned char> dev;      // own device staging, used when the stage outgrows dev_ext
    unsigned char* dev_ext = nullptr;  // the device slice of the batch's staging arena
    size_t dev_ext_n = 0;
    cudaEvent_t done = nullptr;  // recorded after the stage's last flush
    bool pending = false;
    uint64_t allocated = 0;
    size_t pinned_seen = 0;
    ~Stager() {
      if (done) cudaEventDestroy(done);
      dev.free();
    }
  };

  template <class F> static void guarded(AdmitJob& j, F&& f) {
    try {
      f();
    } catch (const std::bad_alloc&) {
      j.status = 1;
      j.error = "host memory exhausted during admission";
    }
  }

  // Runs f(i, worker) for i in [0, n) on `threads` host threads (worker-indexed resources).
  template <class F> void parallel_for(size_t n, int threads, F&& f) {
    if (threads <= 1 || n <= 1) {
      for (size_t i = 0; i < n; ++i) f(i, 0);
      return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    const int t = (int)std::min<size_t>((size_t)threads, n);
    for (int w = 0; w < t; ++w) {
      try {
        pool.emplace_back([&, w] {
          cudaSetDevice(config_.device);  // the current device is per host thread
          for (size_t i = next++; i < n; i = next++) f(i, w);
        });
      } catch (const std::system_error&) {
        break;  // the threads that started take all the work
      }
    }
    if (pool.empty())
      for (size_t i = 0; i < n; ++i) f(i, 0);
    for (std::thread& th : pool) th.join();
  }

  static void job_fail(AdmitJob& j, int status, const std::string& text) {
    j.status = status;
    j.error = text;
  }

  // Bytes fill() stages for a prepared case (each table rounded to the 256-byte allocation
  // grain), which sizes the staging arena; a larger case only takes a slower overflow path.
  size_t staged_bytes(size_t n, size_t nw, size_t ns, size_t nt, size_t nf, size_t ng, size_t gm, size_t ql,
                      size_t halo, size_t tface, bool tiles) const {
    const size_t r = sizeof(R), n1 = n + 1, g1 = ng + 1, tl = tiles ? 1 : 0, sl = slot_fluxes_ ? 1 : 0;
    const size_t tables[] = {4 * n1, 4 * n1, 4 * n1, 4 * n1, 8 * n1, 8 * n1, 8 * n1, 8 * n1, 8 * n1, n1,
                             model_ == MODEL_SA ? r * n1 : 0, 4 * ns * sl, 4 * ns, 4 * ns, 4 * ns, r * ns, 6 * r * ns * sl,
                             r * nw, r * nw, r * nw, r * nw, 8 * nw, 8 * nw, 4 * nw, 4 * nw, 4 * nt, 4 * nt, r * nt,
                             r * nt, 4 * nf, 4 * nf, 4 * nf, 4 * nf, r * nf, 6 * r * nf, 4 * halo, 4 * tface,
                             8 * tface, 4 * ns * tl, 4 * nw * tl, 4 * g1, 4 * gm, 4 * g1, 4 * g1, 4 * ql, 8 * gm, 8 * g1, 8 * g1,
                             r * nv_ * n1, sizeof(CaseCfg<R>)};
    size_t total = 0;
    for (size_t b : tables) total += (b + 255) & ~size_t(255);
    return total;
  }

  // The same from a request's counts alone, with the block-tile tables at their arena bounds
  // (halo <= 2 cells, face records <= 2 faces + 64 per case); 0 for a request that does not
  // name its tables (it fails validation later).
  size_t staged_bound(const AdmitSpec& sp) const {
    const amr_mesh_view_t* m = sp.mesh;
    if (!m || !m->face_offsets || !m->n_cells) return 0;
    const size_t n = m->n_cells, nw = m->n_walls, nf = m->n_faces, ns = m->face_offsets[n] + nw;
    const size_t nt = model_ >= MODEL_LAMINAR && m->visc_offsets ? m->visc_offsets[n] : 0;
    const bool srd = m->small_cells && m->group_offsets && m->member_offsets;
    return staged_bytes(n, nw, ns, nt, nf, srd ? n : 0, srd ? m->group_offsets[n] : 0, srd ? m->member_offsets[n] : 0,
                        block_tiles_ ? 2 * n : 0, block_tiles_ ? 2 * nf + 64 : 0, block_tiles_);
  }

  // The staging arena: one device allocation cut into `stages` equal slices that the first
  // `stages` stagers use (grows only), and for the length of one call a page-locked host block of
  // the same layout lent by the PinnedPool (allocation calls contend in the driver, so one large
  // block replaces one per stage).  Every earlier upload has completed when called.
  bool ensure_arena(int stages, size_t slice, std::string* error) {
    slice = (slice + 4095) & ~size_t(4095);
    if (stages > arena_stages_ || slice > arena_slice_) {
      stages = std::max(stages, arena_stages_);
      slice = std::max(slice, arena_slice_);
      free_arena();
      const size_t bytes = (size_t)stages * slice;
      if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&arena_d_), bytes), error, "staging arena")) {
        free_arena();
        return false;
      }
      stats_.allocated_bytes += bytes;
      arena_stages_ = stages;
      arena_slice_ = slice;
      for (int i = 0; i < stages; ++i) {
        stagers_[i]->dev_ext = arena_d_ + (size_t)i * slice;
        stagers_[i]->dev_ext_n = slice;
      }
    }
    if (arena_lease_.p) return true;
    const size_t bytes = (size_t)arena_stages_ * arena_slice_;
    arena_lease_ = PinnedPool::get().lend(bytes, bytes);
    if (!arena_lease_.p) return fail(error, "staging arena: page-locked allocation failed");
    if (arena_lease_.fresh) stats_.pinned_bytes += arena_lease_.size;
    arena_h_ = arena_lease_.p;
    for (int i = 0; i < arena_stages_; ++i) {
      stagers_[i]->stage.adopt(arena_h_ + (size_t)i * arena_slice_, arena_slice_);
      stagers_[i]->pinned_seen = stagers_[i]->stage.pinned_bytes();
    }
    return true;
  }

  // Gives the arena's host block back to the pool at the end of a call, when every copy from it
  // has completed.
  void return_arena_host() {
    if (!arena_lease_.p) return;
    for (int i = 0; i < arena_stages_ && i < (int)stagers_.size(); ++i) {
      stagers_[i]->stage.adopt(nullptr, 0);
      stagers_[i]->pinned_seen = stagers_[i]->stage.pinned_bytes();
    }
    PinnedPool::get().give_back(arena_lease_);
    arena_lease_ = PinnedPool::Lease();
    arena_h_ = nullptr;
  }

  void free_arena() {
    return_arena_host();
    for (int i = 0; i < arena_stages_ && i < (int)stagers_.size(); ++i) {
      stagers_[i]->dev_ext = nullptr;
      stagers_[i]->dev_ext_n = 0;
    }
    if (arena_d_) cudaFree(arena_d_);
    arena_d_ = nullptr;
    arena_stages_ = 0;
    arena_slice_ = 0;
  }

  // Index checks the tables built before reservation rely on: offsets non-decreasing from zero,
  // every listed face index, wall, donor and gradient source in range, walls grouped by owner
  // cell, every face's cells and boundary marker consistent.  That each listed face names its
  // cell fill() checks where it reads the face anyway (here too when block tiles are built).
  bool check_topology(const AdmitJob& j, std::string* why) const {
    const amr_mesh_view_t* m = j.spec.mesh;
    const long long n = j.n, nf = j.nf, nw = j.nw;
    const bool viscous = model_ >= MODEL_LAMINAR;
    if (m->face_offsets[0] != 0 || (viscous && m->visc_offsets[0] != 0)) return fail(why, "offsets do not start at zero");
    if (nw && !m->walls) return fail(why, "wall table missing");
    long long wpos = 0;
    for (long long k = 0; k < n; ++k) {
      if (m->face_offsets[k + 1] < m->face_offsets[k] || (viscous && m->visc_offsets[k + 1] < m->visc_offsets[k]))
        return fail(why, "offsets decrease");
      for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q) {
        const uint64_t fi = m->cell_faces[q];
        if (fi >= (uint64_t)nf) return fail(why, "cell_faces index out of range");
        if (block_tiles_) {  // the block tiles, built before fill(), follow the faces' cells
          const amr_face_t& f = m->faces[fi];
          if (f.left != (int)k && f.right != (int)k) return fail(why, "cell_faces lists a face of another cell");
        }
      }
      const amr_cell_t& c = m->cells[k];
      if (c.wall_begin != (uint64_t)wpos) return fail(why, "walls are not grouped by owner cell");
      if (c.wall_begin + c.wall_count > (uint64_t)nw) return fail(why, "wall count mismatch");
      for (uint64_t q = c.wall_begin; q < c.wall_begin + c.wall_count; ++q) {
        if (m->walls[q].owner_cell != (uint64_t)k) return fail(why, "wall owner mismatch");
        if (viscous && (m->wall_samples[q].donor < 0 || m->wall_samples[q].donor >= n))
          return fail(why, "wall donor out of range");
      }
      wpos += (long long)c.wall_count;
      if (viscous)
        for (uint64_t q = m->visc_offsets[k]; q < m->visc_offsets[k + 1]; ++q) {
          const amr_gradient_term_t& t = m->visc_terms[q];
          if (t.source >= n) return fail(why, "gradient source out of range");
          if (t.source == -2 && (t.side < 0 || t.side > 3)) return fail(why, "gradient wall side out of range");
        }
    }
    if (wpos != nw) return fail(why, "wall count mismatch");
    for (long long fi = 0; fi < nf; ++fi) {
      const amr_face_t& f = m->faces[fi];
      const int own = f.left >= 0 ? f.left : f.right;
      const int other = f.left >= 0 ? f.right : -1;
      if (own < 0 || own >= (int)n || other >= (int)n || (other < 0) != (f.boundary >= 0) || f.boundary > 3)
        return fail(why, "face cells or boundary marker inconsistent");
    }
    return true;
  }

  // Stage 1 (any thread): validation and the case-local tables; touches no batch state.
  void prepare(AdmitJob& j) const {
    const AdmitSpec& s = j.spec;
    const amr_mesh_view_t* m = s.mesh;
    if (!m || !s.params || !s.u0) return job_fail(j, 1, "null mesh, parameters or state");
    std::string why;
    if (!validate(*m, *s.params, s.u0_count, &why)) return job_fail(j, 1, why);
    if (!std::isfinite(s.time0) || s.time0 < 0) return job_fail(j, 1, "invalid initial time");
    const long long n = j.n = (long long)m->n_cells;
    j.nw = (long long)m->n_walls;
    j.ns = (long long)m->face_offsets[n] + j.nw;  // face slots then wall slots, per cell
    j.nt = model_ >= MODEL_LAMINAR ? (long long)m->visc_offsets[n] : 0;
    j.nf = (long long)m->n_faces;
    if (!check_topology(j, &why)) return job_fail(j, 1, why);
    // SRD lists (only non-trivial neighbourhoods)
    j.has_srd = m->small_cells > 0;
    j.simple.assign(n, 1);
    j.group_index.assign(n, -1);
    if (j.has_srd) {
      for (long long k = 0; k < n; ++k) {
        if (m->member_offsets[k + 1] < m->member_offsets[k] || m->group_offsets[k + 1] < m->group_offsets[k])
          return job_fail(j, 1, "SRD offsets decrease");
        const uint64_t cnt = m->member_offsets[k + 1] - m->member_offsets[k];
        const uint64_t size = m->group_offsets[k + 1] - m->group_offsets[k];
        if (cnt == 0 || size == 0) return job_fail(j, 1, "empty SRD neighbourhood");
        for (uint64_t q = m->group_offsets[k]; q < m->group_offsets[k + 1]; ++q)
          if (m->group_members[q] >= (uint64_t)n) return job_fail(j, 1, "SRD group member out of range");
        for (uint64_t q = m->member_offsets[k]; q < m->member_offsets[k + 1]; ++q)
          if (m->member_groups[q] >= (uint64_t)n) return job_fail(j, 1, "SRD member group out of range");
        j.simple[k] = cnt == 1 && size == 1 && m->group_members[m->group_offsets[k]] == (uint64_t)k;
      }
      for (long long k = 0; k < n; ++k)
        if (!j.simple[k]) {
          j.group_index[k] = (int)j.nontrivial.size();
          j.nontrivial.push_back(k);
          j.gmem += (long long)(m->group_offsets[k + 1] - m->group_offsets[k]);
          j.qlist += (long long)(m->member_offsets[k + 1] - m->member_offsets[k]);
        }
      for (long long k : j.nontrivial)
        for (uint64_t q = m->member_offsets[k]; q < m->member_offsets[k + 1]; ++q)
          if (j.group_index[m->member_groups[q]] < 0) return job_fail(j, 1, "SRD neighbourhood references a trivial group");
    }
    j.ng = (long long)j.nontrivial.size();
    for (int side = 0; side < 4; ++side)
      j.kinds[side] = m->boundaries[side].kind < 0 ? s.params->bc[side] : m->boundaries[side].kind;
    // warp tiles (case-local; reserve() moves them to the case's ranges)
    HostCase<R>& hc = j.hc;
    hc.n = (int)n;
    hc.nslot.resize(n);
    hc.nterm.assign(n, 0);
    for (long long k = 0; k < n; ++k) {
      hc.nslot[k] = (int)(m->face_offsets[k + 1] - m->face_offsets[k] + m->cells[k].wall_count);
      if (model_ >= MODEL_LAMINAR) hc.nterm[k] = (int)(m->visc_offsets[k + 1] - m->visc_offsets[k]);
    }
    hc.slot_prefix.assign(n + 1, 0);
    hc.term_prefix.assign(n + 1, 0);
    for (long long k = 0; k < n; ++k) {
      hc.slot_prefix[k + 1] = hc.slot_prefix[k] + hc.nslot[k];
      hc.term_prefix[k + 1] = hc.term_prefix[k] + hc.nterm[k];
    }
    if (!make_tiles(hc, &why)) return job_fail(j, 1, why);
    // face records go in order of first reference by a cell, in slot order, so that the
    // records of neighbouring cells are neighbours in memory (the reference's face order runs
    // along grid lines)
    j.rec.assign(j.nf, -1);
    int next = 0;
    for (long long k = 0; k < n; ++k)
      for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q) {
        const uint64_t fi = m->cell_faces[q];
        if (j.rec[fi] < 0) j.rec[fi] = next++;
      }
    for (long long fi = 0; fi < j.nf; ++fi)
      if (j.rec[fi] < 0) j.rec[fi] = next++;  // a face no cell lists (still evaluated, never gathered)
    // block tiles (tiled mode), case-local
    if (block_tiles_) {
      j.s_loc.assign(j.ns, 0);
      j.w_ldon.assign(j.nw, 0);
      if (!make_block_tiles(m, n, j.rec, -1, &hc.btiles, &j.bt_halo, &j.bt_face, &j.bt_floc, &j.s_loc, &j.w_ldon, &why))
        return job_fail(j, 1, why);
    }
  }

  // Stage 2 (serial, request order): a free slot and the case's ranges of every arena table.
  void reserve(AdmitJob& j) {
    int slot = -1;
    for (int i = 0; i < config_.max_cases; ++i)
      if (!cases_[i].live && !reserved_[i]) {
        slot = i;
        break;
      }
    if (slot < 0) return job_fail(j, 3, "");
    HostCase<R>& hc = j.hc;
    const long long n = j.n;
    hc.cells = {a_cells_.alloc(n + 1), n + 1};
    hc.slots = {a_slots_.alloc(j.ns), j.ns};
    hc.walls = {a_walls_.alloc(j.nw), j.nw};
    hc.terms = {a_terms_.alloc(j.nt), j.nt};
    hc.groups = {a_groups_.alloc(j.ng + 1), j.ng + 1};
    hc.gmembers = {a_gmem_.alloc(j.gmem), j.gmem};
    hc.qcells = {a_q_.alloc(j.ng + 1), j.ng + 1};
    hc.qlist = {a_qlist_.alloc(j.qlist), j.qlist};
    hc.faces = {a_faces_.alloc(j.nf), j.nf};
    hc.halo = {a_halo_.alloc((long long)j.bt_halo.size()), (long long)j.bt_halo.size()};
    hc.tfaces = {a_tface_.alloc((long long)j.bt_face.size()), (long long)j.bt_face.size()};
    if (hc.cells.b < 0 || hc.slots.b < 0 || hc.walls.b < 0 || hc.terms.b < 0 || hc.groups.b < 0 || hc.gmembers.b < 0 ||
        hc.qcells.b < 0 || hc.qlist.b < 0 || hc.faces.b < 0 || hc.halo.b < 0 || hc.tfaces.b < 0 ||
        n_tiles_total() + pending_tiles_ + (long long)hc.tiles.size() > cap_tiles_ ||
        n_btiles_total() + pending_btiles_ + (long long)hc.btiles.size() > cap_btiles_) {
      release_ranges(hc);
      return job_fail(j, 3, "");
    }
    j.slot = hc.slot = slot;
    j.reserved = reserved_[slot] = 1;
    pending_tiles_ += (long long)hc.tiles.size();
    pending_btiles_ += (long long)hc.btiles.size();
    const int cb = (int)hc.cells.b;
    for (Tile& t : hc.tiles) {
      t.cs = slot;
      t.c0 += cb;
      t.c1 += cb;
      t.s0 += (int)hc.slots.b;
      t.s1 += (int)hc.slots.b;
      t.t0 += (int)hc.terms.b;
      t.t1 += (int)hc.terms.b;
    }
    for (BTile& t : hc.btiles) {
      t.cs = slot;
      t.c0 += cb;
      t.c1 += cb;
      t.h0 += (int)hc.halo.b;
      t.h1 += (int)hc.halo.b;
      t.f0 += (int)hc.tfaces.b;
      t.f1 += (int)hc.tfaces.b;
      t.w0 += (int)hc.walls.b;
      t.w1 += (int)hc.walls.b;
    }
  }

  // Stage 3 (any thread): the engine tables of one reserved case, written straight into the
  // worker's page-locked staging, and their upload (asynchronous on stream_).
  void fill(AdmitJob& j, Stager& st) {
    if (st.pending && !cuda_ok(cudaEventSynchronize(st.done), &j.error, "staging reuse")) return (void)(j.status = 1);
    st.pending = false;
    st.stage.reset();
    st.uploads.clear();
    PinnedStage& S = st.stage;
    const AdmitSpec& sp = j.spec;
    const amr_mesh_view_t* m = sp.mesh;
    const amr_params_t* p = sp.params;
    HostCase<R>& hc = j.hc;
    const long long n = j.n, nw = j.nw, ns = j.ns, nt = j.nt, nf = j.nf, ng = j.ng;
    const int slot = j.slot;
    const bool has_srd = j.has_srd, viscous = model_ >= MODEL_LAMINAR;
    const int* kinds = j.kinds;
    const std::vector<int>& rec = j.rec;
    const int cb = (int)hc.cells.b, sb = (int)hc.slots.b, wb = (int)hc.walls.b, tb = (int)hc.terms.b, fb = (int)hc.faces.b;
    // tables every entry of which the loops below write are left uninitialised (pvu)
    PVec<int> c_case = pv<int>(S, n + 1, slot), c_slot = pvu<int>(S, n + 1), c_wall = pvu<int>(S, n + 1),
              c_term = pvu<int>(S, n + 1);
    c_case[n] = -1;
    PVec<double> c_vol = pvu<double>(S, n + 1), c_area = pvu<double>(S, n + 1), c_gvol = pvu<double>(S, n + 1),
                 c_cx = pvu<double>(S, n + 1), c_cy = pvu<double>(S, n + 1);
    c_vol[n] = c_area[n] = c_gvol[n] = 1.0;
    c_cx[n] = c_cy[n] = 0.0;
    PVec<unsigned char> c_flags = pvu<unsigned char>(S, n + 1);
    c_flags[n] = 0;
    PVec<R> c_wd = pvu<R>(S, model_ == MODEL_SA ? n + 1 : 0);
    if (model_ == MODEL_SA) c_wd[n] = R(1);
    // owner and geometry per slot serve only the per-slot flux modes (persistent, phases)
    const bool sf = slot_fluxes_;
    PVec<int> s_own = pvu<int>(S, sf ? ns : 0), s_nb = pvu<int>(S, ns), s_meta = pvu<int>(S, ns),
              s_item = pvu<int>(S, ns);
    PVec<R> s_len = pvu<R>(S, ns), s_geo = pv<R>(S, sf ? 6 * ns : 0, R(0));
    PVec<R> w_nx = pvu<R>(S, nw), w_ny = pvu<R>(S, nw), w_len = pvu<R>(S, nw), w_dist = pv<R>(S, nw, R(1));
    PVec<double> w_xm = pvu<double>(S, nw), w_ym = pvu<double>(S, nw);
    PVec<int> w_donor = pv<int>(S, nw, cb), w_owner = pvu<int>(S, nw);
    PVec<int> t_own = pvu<int>(S, sf ? nt : 0), t_src = pvu<int>(S, nt);  // t_own: slot-tile modes only
    PVec<R> t_x = pvu<R>(S, nt), t_y = pvu<R>(S, nt);
    PVec<int> f_case = pv<int>(S, nf, slot), f_own = pvu<int>(S, nf), f_nb = pvu<int>(S, nf), f_meta = pvu<int>(S, nf);
    PVec<R> f_len = pvu<R>(S, nf), f_geo = viscous ? pvu<R>(S, 6 * nf) : pv<R>(S, 6 * nf, R(0));
    long long wpos = 0, spos = 0;
    for (long long k = 0; k < n; ++k) {
      const amr_cell_t& c = m->cells[k];
      c_vol[k] = c.volume;
      c_area[k] = m->agglomerate_small ? c.volume : (c.x1 - c.x0) * (c.y1 - c.y0);
      c_gvol[k] = has_srd ? m->group_volume[k] : 1.0;
      c_flags[k] = has_srd && j.simple[k] ? 1 : 0;
      c_cx[k] = c.cx;
      c_cy[k] = c.cy;
      c_slot[k] = sb + (int)spos;
      c_term[k] = tb + (viscous ? (int)m->visc_offsets[k] : 0);
      if (model_ == MODEL_SA) c_wd[k] = (R)m->wall_distance[k];
      for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q, ++spos) {
        const uint64_t fi = m->cell_faces[q];
        const amr_face_t& f = m->faces[fi];
        const bool own_left = f.left == (int)k;
        if (!own_left && f.right != (int)k) return job_fail(j, 1, "cell_faces lists a face of another cell");
        const int other = own_left ? f.right : f.left;
        const int side = f.boundary;
        if (other >= (int)n) return job_fail(j, 1, "face neighbour out of range");
        if ((other < 0) != (side >= 0) || side > 3) return job_fail(j, 1, "face boundary marker inconsistent");
        const int kind = side >= 0 ? kinds[side] : 0;
        if (sf) s_own[spos] = cb + (int)k;
        s_nb[spos] = other >= 0 ? cb + other : -1;
        s_meta[spos] = (own_left ? 1 : 0) | ((f.axis & 1) << 1) | ((side + 1) << 2) | ((kind & 15) << 5);
        s_len[spos] = (R)f.length;
        s_item[spos] = 2 * (fb + rec[fi]) + (own_left ? 1 : 0);  // record index and orientation
        if (viscous && sf) {
          const amr_face_geometry_t& g = m->face_geometry[fi];
          R* geo = &s_geo[6 * spos];
          geo[0] = (R)g.dx;
          geo[1] = (R)g.dy;
          geo[2] = (R)g.ex;
          geo[3] = (R)g.ey;
          geo[4] = (R)g.distance;
          geo[5] = (R)m->face_samples[fi].distance;
        }
      }
      c_wall[k] = wb + (int)wpos;
      for (uint64_t q = c.wall_begin; q < c.wall_begin + c.wall_count; ++q, ++wpos, ++spos) {
        const amr_wall_t& w = m->walls[q];
        w_nx[wpos] = (R)w.nx;
        w_ny[wpos] = (R)w.ny;
        w_len[wpos] = (R)w.length;
        w_xm[wpos] = (w.x0 + w.x1) * .5;
        w_ym[wpos] = (w.y0 + w.y1) * .5;
        if (sf) s_own[spos] = cb + (int)k;
        s_nb[spos] = -1;
        s_meta[spos] = SLOT_WALL;
        s_len[spos] = (R)w.length;
        s_item[spos] = wb + (int)wpos;
        w_owner[wpos] = cb + (int)k;
        if (sf) {
          s_geo[6 * spos + 0] = (R)w.nx;
          s_geo[6 * spos + 1] = (R)w.ny;
          s_geo[6 * spos + 2] = R(1);
        }
        if (viscous) {
          const amr_wall_sample_t& smp = m->wall_samples[q];
          w_donor[wpos] = cb + smp.donor;
          w_dist[wpos] = (R)smp.distance;
          s_nb[spos] = cb + smp.donor;
          if (sf) s_geo[6 * spos + 2] = (R)smp.distance;
        }
      }
      if (viscous)
        for (uint64_t q = m->visc_offsets[k]; q < m->visc_offsets[k + 1]; ++q) {
          const amr_gradient_term_t& t = m->visc_terms[q];
          if (sf) t_own[q] = cb + (int)k;
          t_src[q] = t.source >= 0 ? cb + t.source : (t.source == -1 ? -1 : -2 - t.side);
          t_x[q] = (R)t.x;
          t_y[q] = (R)t.y;
        }
    }
    // face records in face orientation (left to right; a boundary face's inside cell is its owner)
    for (long long fi = 0; fi < nf; ++fi) {
      const amr_face_t& f = m->faces[fi];
      const bool own_left = f.left >= 0;
      const int own = own_left ? f.left : f.right;
      const int other = own_left ? f.right : -1;
      const int side = f.boundary;
      const int kind = side >= 0 ? kinds[side] : 0;
      const long long r = rec[fi];
      f_own[r] = cb + own;
      f_nb[r] = other >= 0 ? cb + other : -1;
      f_meta[r] = (own_left ? 1 : 0) | ((f.axis & 1) << 1) | ((side + 1) << 2) | ((kind & 15) << 5);
      f_len[r] = (R)f.length;
      if (viscous) {
        const amr_face_geometry_t& g = m->face_geometry[fi];
        R* geo = &f_geo[6 * r];
        geo[0] = (R)g.dx;
        geo[1] = (R)g.dy;
        geo[2] = (R)g.ex;
        geo[3] = (R)g.ey;
        geo[4] = (R)g.distance;
        geo[5] = (R)m->face_samples[fi].distance;
      }
    }
    c_slot[n] = sb + (int)ns;
    c_wall[n] = wb + (int)nw;
    c_term[n] = tb + (int)nt;
    // block-tile tables in the case's ranges
    PVec<int> bt_halo = pvu<int>(S, j.bt_halo.size()), bt_face = pvu<int>(S, j.bt_face.size());
    for (size_t i = 0; i < j.bt_halo.size(); ++i) bt_halo[i] = j.bt_halo[i] + cb;
    for (size_t i = 0; i < j.bt_face.size(); ++i) bt_face[i] = j.bt_face[i] + fb;
    PVec<int2> bt_floc(j.bt_floc.begin(), j.bt_floc.end(), PinAlloc<int2>(&S));
    PVec<int> s_loc(j.s_loc.begin(), j.s_loc.end(), PinAlloc<int>(&S));
    PVec<int> w_ldon(j.w_ldon.begin(), j.w_ldon.end(), PinAlloc<int>(&S));
    // SRD arrays
    const int gb = (int)hc.groups.b, gmb = (int)hc.gmembers.b, qb = (int)hc.qcells.b, qlb = (int)hc.qlist.b;
    PVec<int> g_mem = pv<int>(S, ng + 1, 0), g_cell = pv<int>(S, j.gmem, 0), q_cell = pv<int>(S, ng + 1, cb + (int)n),
              q_grp = pv<int>(S, ng + 1, 0), q_list = pv<int>(S, j.qlist, 0);
    PVec<double> g_cnt = pv<double>(S, j.gmem, 0.0), g_vol = pv<double>(S, ng + 1, 1.0), q_cnt = pv<double>(S, ng + 1, 1.0);
    {
      long long pos = 0, lpos = 0;
      for (long long gi = 0; gi < ng; ++gi) {
        const long long g = j.nontrivial[gi];
        g_mem[gi] = gmb + (int)pos;
        g_vol[gi] = m->group_volume[g];
        for (uint64_t q = m->group_offsets[g]; q < m->group_offsets[g + 1]; ++q, ++pos) {
          const uint64_t k = m->group_members[q];
          g_cell[pos] = cb + (int)k;
          g_cnt[pos] = (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
        }
      }
      g_mem[ng] = gmb + (int)pos;
      for (long long qi = 0; qi < ng; ++qi) {
        const long long k = j.nontrivial[qi];
        q_cell[qi] = cb + (int)k;
        q_grp[qi] = qlb + (int)lpos;
        q_cnt[qi] = (double)(m->member_offsets[k + 1] - m->member_offsets[k]);
        for (uint64_t q = m->member_offsets[k]; q < m->member_offsets[k + 1]; ++q, ++lpos)
          q_list[lpos] = gb + j.group_index[m->member_groups[q]];
      }
      q_grp[ng] = qlb + (int)lpos;
    }
    // per-case constants
    CaseCfg<R>& cf = hc.cfg;
    std::memset(&cf, 0, sizeof(cf));
    cf.cfl = p->cfl;
    cf.dt_fixed = p->dt_fixed;
    cf.viscous_cfl = m->transport.viscous_cfl;
    cf.sa_cfl = m->transport.sa_cfl;
    cf.gamma = (R)p->gamma;
    cf.mco = (R)p->ausm_mco;
    for (int side = 0; side < 4; ++side) {
      const amr_boundary_t& b = m->boundaries[side];
      cf.kind[side] = kinds[side];
      Bnd<R>& d = cf.bnd[side];
      d.kind = kinds[side];
      for (int v = 0; v < 4; ++v) d.ref[v] = (R)b.reference[v];
      d.total_pressure = (R)b.total_pressure;
      d.total_temperature = (R)b.total_temperature;
      d.gas_constant = (R)b.gas_constant;
      d.dir[0] = (R)b.direction[0];
      d.dir[1] = (R)b.direction[1];
      d.outlet_pressure = (R)b.outlet_pressure;
      d.wall_velocity[0] = (R)b.wall_velocity[0];
      d.wall_velocity[1] = (R)b.wall_velocity[1];
    }
    cf.trn.law = m->transport.law;
    cf.trn.mu_ref = (R)m->transport.mu_ref;
    cf.trn.gas_constant = (R)m->transport.gas_constant;
    cf.trn.temperature_ref = (R)m->transport.temperature_ref;
    cf.trn.sutherland = (R)m->transport.sutherland;
    cf.trn.viscous_cfl = (R)m->transport.viscous_cfl;
    cf.trn.sa_nu_inf = (R)m->transport.sa_nu_inf;
    cf.trn.sa_cfl = (R)m->transport.sa_cfl;
    cf.agglomerated = m->agglomerate_small ? 1 : 0;
    cf.has_srd = has_srd && ng > 0 ? 1 : 0;
    cf.srd_g0 = gb;
    cf.srd_g1 = gb + (int)ng;
    cf.srd_q0 = qb;
    cf.srd_q1 = qb + (int)ng;
    cf.srd_rate = viscous && m->transport.stabilization == AMR_B200_VISCOUS_SRD && m->small_cells > 0 && cf.has_srd;
    cf.cell0 = cb;
    cf.cell1 = cb + (int)n;
    // state (variable-major, each variable's n cells then the padding cell).  A uniform start
    // (u0 holds nv values) is not staged: a kernel fills it on the device after the uploads.
    const bool uniform = uniform_start(sp.u0_count, n);
    const long long sn = uniform ? 0 : n + 1;
    PVec<R> u = pvu<R>(S, nv_ * sn);
    // FP32 form: the trailing word holds what the leading word rounds off the FP64 start state
    PVec<R> ulo = pvu<R>(S, sizeof(R) == 4 ? nv_ * sn : 0);
    if (!uniform) {
      for (int v = 0; v < nv_; ++v) {
        for (long long k = 0; k < n; ++k) u[v * (n + 1) + k] = (R)sp.u0[v * n + k];
        u[v * (n + 1) + n] = R(1);
      }
      if (sizeof(R) == 4)
        for (int v = 0; v < nv_; ++v) {
          for (long long k = 0; k < n; ++k)
            ulo[v * (n + 1) + k] = (R)(sp.u0[v * n + k] - (double)u[v * (n + 1) + k]);
          ulo[v * (n + 1) + n] = R(0);
        }
    }
    // control
    CaseCtl& ctl = j.ctl;
    std::memset(&ctl, 0, sizeof(ctl));
    ctl.time = sp.time0;
    ctl.target = sp.target;
    ctl.steps = sp.steps0;
    ctl.rejected = sp.rejected0;
    ctl.maxsteps = sp.maxsteps;
    ctl.finished = sp.time0 >= sp.target;
    ctl.live = 1;
    ctl.cur = 0;
    ctl.dtmin = DT_INF_BITS;
    // uploads
    uint64_t* G = &j.geometry_bytes;
    bool ok = up(st, c_case_.p + cb, c_case, G) && up(st, c_vol_.p + cb, c_vol, G) && up(st, c_area_.p + cb, c_area, G) &&
              up(st, c_gvol_.p + cb, c_gvol, G) && up(st, c_flags_.p + cb, c_flags, G) &&
              up(st, c_slot_.p + cb, c_slot, G) && up(st, c_wall_.p + cb, c_wall, G) && up(st, c_term_.p + cb, c_term, G) &&
              up(st, c_cx_.p + cb, c_cx, G) && up(st, c_cy_.p + cb, c_cy, G) && up(st, s_own_.p + sb, s_own, G) &&
              up(st, s_nb_.p + sb, s_nb, G) && up(st, s_meta_.p + sb, s_meta, G) && up(st, s_len_.p + sb, s_len, G) &&
              up(st, w_nx_.p + wb, w_nx, G) && up(st, w_ny_.p + wb, w_ny, G) && up(st, w_len_.p + wb, w_len, G) &&
              up(st, w_dist_.p + wb, w_dist, G) && up(st, w_donor_.p + wb, w_donor, G) && up(st, w_xm_.p + wb, w_xm, G) &&
              up(st, w_ym_.p + wb, w_ym, G) && up(st, g_mem_.p + gb, g_mem, G) && up(st, g_cell_.p + gmb, g_cell, G) &&
              up(st, g_cnt_.p + gmb, g_cnt, G) && up(st, g_vol_.p + gb, g_vol, G) && up(st, q_cell_.p + qb, q_cell, G) &&
              up(st, q_grp_.p + qb, q_grp, G) && up(st, q_list_.p + qlb, q_list, G) && up(st, q_cnt_.p + qb, q_cnt, G);
    ok = ok && up(st, s_geo_.p + 6 * (long long)sb, s_geo, G) && up(st, s_item_.p + sb, s_item, G) &&
         up(st, f_case_.p + fb, f_case, G) && up(st, f_own_.p + fb, f_own, G) && up(st, f_nb_.p + fb, f_nb, G) &&
         up(st, f_meta_.p + fb, f_meta, G) && up(st, f_len_.p + fb, f_len, G) &&
         up(st, f_geo_.p + 6 * (long long)fb, f_geo, G) && up(st, w_owner_.p + wb, w_owner, G) &&
         up(st, bt_halo_.p + hc.halo.b, bt_halo, G) && up(st, bt_face_.p + hc.tfaces.b, bt_face, G) &&
         up(st, bt_floc_.p + hc.tfaces.b, bt_floc, G) && up(st, s_loc_.p + sb, s_loc, G) &&
         up(st, w_ldon_.p + wb, w_ldon, G);  // the last five are empty without block tiles
    if (ok && viscous)
      ok = (!sf || up(st, t_own_.p + tb, t_own, G)) && up(st, t_src_.p + tb, t_src, G) && up(st, t_x_.p + tb, t_x, G) &&
           up(st, t_y_.p + tb, t_y, G);
    if (ok && model_ == MODEL_SA) ok = up(st, c_wd_.p + cb, c_wd, G);
    for (int v = 0; ok && !uniform && v < nv_; ++v) {
      ok = stage_up(st, U0_.p + v * cap_cells_ + cb, u.data() + v * (n + 1), sizeof(R) * (n + 1));
      j.state_bytes += sizeof(R) * (n + 1);
      if (ok && L0_.p) {
        ok = stage_up(st, L0_.p + v * cap_cells_ + cb, ulo.data() + v * (n + 1), sizeof(R) * (n + 1));
        j.state_bytes += sizeof(R) * (n + 1);
      }
    }
    CaseCfg<R>* cf_staged = static_cast<CaseCfg<R>*>(S.take(sizeof(cf)));
    *cf_staged = cf;
    ok = ok && stage_up(st, cfg_.p + slot, cf_staged, sizeof(cf));
    if (!ok) return job_fail(j, 1, "upload staging");
    if (!flush_uploads(st, &j.error)) return (void)(j.status = 1);
    if (uniform) {
      UniformState<R> w{};
      for (int v = 0; v < nv_; ++v) {
        w.hi[v] = (R)sp.u0[v];
        w.lo[v] = (R)(sp.u0[v] - (double)w.hi[v]);
      }
      const int blocks = (int)std::min<long long>((n + 256) / 256, 1024);
      fill_uniform_kernel<R><<<blocks, 256, 0, stream_>>>(U0_.p, L0_.p, cap_cells_, cb, (int)n, nv_, w);
      if (!cuda_ok(cudaGetLastError(), &j.error, "uniform start")) return (void)(j.status = 1);
      j.state_bytes += sizeof(w);
    }
    if (!st.done && !cuda_ok(cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming), &j.error, "staging event"))
      return (void)(j.status = 1);
    if (!cuda_ok(cudaEventRecord(st.done, stream_), &j.error, "staging event")) return (void)(j.status = 1);
    st.pending = true;
  }

  // Stage 4 (serial): control records of the filled cases, one synchronisation, then the
  // host bookkeeping in request order; failed cases give their slot and ranges back.
  void commit(std::vector<AdmitJob>& jobs) {
    for (AdmitJob& j : jobs)
      if (j.status == 0) {
        h_ctl_[j.slot] = j.ctl;
        if (!cuda_ok(cudaMemcpyAsync(ctl_.p + j.slot, &h_ctl_[j.slot], sizeof(CaseCtl), cudaMemcpyHostToDevice, stream_),
                     &j.error, "control upload"))
          j.status = 1;
      }
    // a case that failed after its fill began may have written its ranges' owner markers: mark
    // them free again (as release does), so no later case inherits those cells, faces or walls
    for (AdmitJob& j : jobs)
      if (j.status != 0 && j.reserved) unmark_ranges(j.hc);
    std::string err;
    const bool synced = cuda_ok(cudaStreamSynchronize(stream_), &err, "admit sync");
    for (std::unique_ptr<Stager>& s : stagers_) {
      s->pending = false;
      stats_.allocated_bytes += s->allocated;
      s->allocated = 0;
      stats_.pinned_bytes += s->stage.pinned_bytes() - s->pinned_seen;
      s->pinned_seen = s->stage.pinned_bytes();
    }
    for (AdmitJob& j : jobs) {
      if (j.status == 0 && !synced) job_fail(j, 1, err);
      if (j.reserved) {
        reserved_[j.slot] = 0;
        pending_tiles_ -= (long long)j.hc.tiles.size();
        pending_btiles_ -= (long long)j.hc.btiles.size();
      }
      if (j.status != 0) {
        if (j.reserved) release_ranges(j.hc);
        continue;
      }
      stats_.geometry_h2d_bytes += j.geometry_bytes;
      stats_.state_h2d_bytes += j.state_bytes;
      stats_.control_h2d_bytes += sizeof(CaseCtl);
      j.hc.live = true;
      cases_[j.slot] = std::move(j.hc);
      live_++;
      refresh_meta(j.slot);
      tiles_dirty_ = true;
    }
  }

  int release(int slot) override {
    if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return 1;
    // mark the control record dead on the device and in the mirror
    h_ctl_[slot].live = 0;
    h_ctl_[slot].active = 0;
    cudaMemcpyAsync(ctl_.p + slot, &h_ctl_[slot], sizeof(CaseCtl), cudaMemcpyHostToDevice, stream_);
    // the freed cell range no longer belongs to any case
    HostCase<R>& hc = cases_[slot];
    unmark_ranges(hc);
    cudaStreamSynchronize(stream_);
    release_ranges(hc);
    hc = HostCase<R>();
    live_--;
    refresh_meta(slot);
    tiles_dirty_ = true;
    return 0;
  }

  int set_target(int slot, double target, long long maxsteps, std::string* error) override {
    if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return fail1(error, "no such case");
    CaseCtl& c = h_ctl_[slot];
    c.target = target;
    c.maxsteps = maxsteps;
    c.finished = c.time >= target;
    stats_.control_h2d_bytes += sizeof(CaseCtl);
    if (!cuda_ok(cudaMemcpyAsync(ctl_.p + slot, &c, sizeof(CaseCtl), cudaMemcpyHostToDevice, stream_), error, "target"))
      return 1;
    refresh_meta(slot);
    return cuda_ok(cudaStreamSynchronize(stream_), error, "target sync") ? 0 : 1;
  }

  int advance(int trials, std::string* error) override {
    const int rc = advance_begin(trials, error);
    return rc ? rc : advance_end(error);
  }

  // First half of advance: everything up to the stream synchronisation (capture or replay of the
  // trials' graph, with the control read-back at its end), so that several batches can have
  // their trials in flight at once.  advance_end waits and refreshes the host-side statuses.
  // The host-side preparation of an advance of `trials` trials: tile and range uploads and, when
  // the case set or the trial count changed, the capture of the trials' graph.  advance_begin does
  // it itself; a group advance does it for every batch before its start event.
  int prepare_advance(int trials, std::string* error) override {
    if (in_flight_) return fail1(error, "an advance is already in flight");
    if (trials < 1 || trials > 1024) return fail1(error, "trials must be 1..1024");
    if (live_ == 0) return 0;
    if (!sync_tiles(error)) return 1;
    if (use_graph_ && (graph_dirty_ || graph_trials_ != trials)) {
      if (!capture(trials, error)) {
        use_graph_ = false;  // capture not available: launch directly
        cudaGetLastError();
      }
    }
    return 0;
  }

  int advance_begin(int trials, std::string* error) override {
    if (prepare_advance(trials, error)) return 1;
    if (live_ == 0) return 0;
    bool ok;
    cudaGetLastError();  // clear any stale error of an earlier runtime call
    if (use_graph_ && graph_exec_) {
      ok = cuda_ok(cudaEventRecord(ev0_, stream_), error, "event") &&
           cuda_ok(cudaGraphLaunch(graph_exec_, stream_), error, "graph launch") &&
           cuda_ok(cudaEventRecord(ev1_, stream_), error, "event");
    } else {
      ok = enqueue(trials, MODE_TRIALS, error);
    }
    if (!ok) {
      cudaStreamSynchronize(stream_);
      return 1;
    }
    in_flight_ = true;
    in_flight_trials_ = trials;
    return 0;
  }

  cudaStream_t stream() const override { return stream_; }
  int device() const override { return config_.device; }

  int advance_end(std::string* error) override {
    if (!in_flight_) return 0;
    in_flight_ = false;
    const int trials = in_flight_trials_;
    const bool ok = cuda_ok(cudaStreamSynchronize(stream_), error, "advance");
    launches_ += kernels_per_advance(trials);
    stats_.status_polls += 1;
    stats_.control_d2h_bytes += sizeof(CaseCtl) * config_.max_cases;
    float ms = 0;
    if (ok && cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) {
      last_seconds_ = ms * 1e-3;
      if (event_timing_) {
        stats_.advance_event_seconds += last_seconds_;
        stats_.event_batches += 1;
      }
    } else {
      cudaGetLastError();
    }
    if (!ok) return 1;
    if (mode_ == AMR_B200_LAUNCH_PERSISTENT && h_bar_->timeout) {
      // a grid barrier gave up: mark every live case and report
      for (int i = 0; i < config_.max_cases; ++i)
        if (cases_[i].live && !h_ctl_[i].fatal) h_ctl_[i].fatal = STATUS_BARRIER_TIMEOUT;
      cudaMemcpyAsync(ctl_.p, h_ctl_, sizeof(CaseCtl) * config_.max_cases, cudaMemcpyHostToDevice, stream_);
      cudaStreamSynchronize(stream_);
      for (int i = 0; i < config_.max_cases; ++i) refresh_meta(i);
      return fail1(error, "grid barrier timed out; cases marked with status 9");
    }
    for (int i = 0; i < config_.max_cases; ++i) refresh_meta(i);
    return 0;
  }

  int residual(std::string* error) override {
    if (live_ == 0) return 0;
    if (!sync_tiles(error)) return 1;
    cudaGetLastError();
    if (!enqueue(1, MODE_RESIDUAL, error)) return 1;
    launches_ += mode_ == AMR_B200_LAUNCH_PERSISTENT || mode_ == AMR_B200_LAUNCH_TILED
                     ? 1
                     : (model_ >= MODEL_LAMINAR ? 3 : 2) - (mode_ == AMR_B200_LAUNCH_PHASES);
    return cuda_ok(cudaStreamSynchronize(stream_), error, "residual") ? 0 : 1;
  }

  int download_residual(int slot, double* out, uint64_t count, std::string* error) override {
    return copy_out(R0_.p, slot, out, count, error);
  }

  int export_case(int slot, double* wall_rows, uint64_t wall_count, double* sa_rows, uint64_t sa_count, double* limits,
                  std::string* error) override;
  int n_walls(int slot) const override { return (int)cases_[slot].walls.n; }

  int download(int slot, double* u, uint64_t count, std::string* error) override {
    if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return fail1(error, "no such case");
    const int cur = h_ctl_[slot].cur;
    int ok = copy_out(cur ? U1_.p : U0_.p, slot, u, count, error);
    if (ok == 0 && L0_.p) {  // FP32 form: the value is the leading plus the trailing word
      std::vector<double> lo(count);
      ok = copy_out(cur ? L1_.p : L0_.p, slot, lo.data(), count, error);
      for (uint64_t i = 0; ok == 0 && i < count; ++i) u[i] += lo[i];
    }
    if (ok == 0) {
      stats_.state_d2h_bytes += sizeof(R) * count;
      stats_.full_downloads += 1;
    }
    return ok;
  }

  // Several cases' accepted states in one go: every case's rows (and, in FP32, its trailing words)
  // are queued into page-locked staging, then one synchronisation, then the conversion to FP64.
  int download_many(const std::vector<int>& slots, double* const* outs, const uint64_t* counts,
                    std::string* error) override {
    const size_t m = slots.size();
    for (size_t i = 0; i < m; ++i) {
      const int slot = slots[i];
      if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return fail1(error, "no such case");
      if (!outs[i] || counts[i] != (uint64_t)(nv_ * cases_[slot].n)) return fail1(error, "state size mismatch");
    }
    const int words = L0_.p ? 2 : 1;
    const auto grain = [](size_t b) { return (b + 255) & ~size_t(255); };
    // The cases go through page-locked memory lent by the pool, as many per round as fit; after
    // an admission the pool holds that admission's staging block, so nothing new is locked.
    size_t least = 0, want = 0;
    for (size_t i = 0; i < m; ++i) {
      const size_t b = words * grain(sizeof(R) * nv_ * cases_[slots[i]].n);
      least = std::max(least, b);
      want += b;
    }
    want = std::max(least, std::min(want, size_t(64) << 20));
    const LeaseGuard held(stream_, PinnedPool::get().lend(least, want));
    if (!held.lease.p) return fail1(error, "download staging: page-locked allocation failed");
    if (held.lease.fresh) stats_.pinned_bytes += held.lease.size;
    const size_t arena_bytes = held.lease.size;
    size_t arena_used = 0;
    const auto fits = [&](size_t b) { return arena_used + grain(b) <= arena_bytes; };
    const auto take = [&](size_t b) -> void* {
      void* p = held.lease.p + arena_used;
      arena_used += grain(b);
      return p;
    };
    std::vector<R*> tmp(m * words);
    for (size_t i0 = 0; i0 < m;) {
      arena_used = 0;
      size_t i1 = i0;
      for (; i1 < m; ++i1) {
        const HostCase<R>& hc = cases_[slots[i1]];
        const size_t bytes = sizeof(R) * nv_ * hc.n;
        if (i1 > i0 && !fits(words * grain(bytes))) break;
        const int cur = h_ctl_[slots[i1]].cur;
        for (int w = 0; w < words; ++w) {
          const R* buf = w == 0 ? (cur ? U1_.p : U0_.p) : (cur ? L1_.p : L0_.p);
          R* dst = static_cast<R*>(take(bytes));
          tmp[i1 * words + w] = dst;
          if (!cuda_ok(cudaMemcpy2DAsync(dst, sizeof(R) * hc.n, buf + hc.cells.b, sizeof(R) * cap_cells_,
                                         sizeof(R) * hc.n, nv_, cudaMemcpyDeviceToHost, stream_),
                       error, "download"))
            return 1;
        }
      }
      if (!cuda_ok(cudaStreamSynchronize(stream_), error, "download sync")) return 1;
      // the conversion to FP64 (leading plus trailing word) on up to 8 host threads, case by case
      const int threads = (int)std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()));
      parallel_for(i1 - i0, threads, [&](size_t j, int) {
        const size_t i = i0 + j;
        const R* hi = tmp[i * words];
        const R* lo = words == 2 ? tmp[i * words + 1] : nullptr;
        for (uint64_t q = 0; q < counts[i]; ++q) outs[i][q] = lo ? (double)hi[q] + (double)lo[q] : (double)hi[q];
      });
      for (size_t i = i0; i < i1; ++i) {
        stats_.state_d2h_bytes += sizeof(R) * words * counts[i];
        stats_.full_downloads += 1;
      }
      i0 = i1;
    }
    return 0;
  }

  int diagnostics(const std::vector<int>& slots, const std::vector<double>& rm, std::vector<double>* out,
                  std::string* error) override;

  const CaseMeta& meta(int slot) const override { return meta_[slot]; }
  int live_cases() const override { return live_; }
  int max_cases() const override { return config_.max_cases; }
  uint64_t free_cells() const override { return (uint64_t)a_cells_.free_total(); }
  int nv() const override { return nv_; }
  int n_cells(int slot) const override { return cases_[slot].n; }
  double last_advance_seconds() const override { return last_seconds_; }
  uint64_t kernel_launches() const override { return launches_; }
  amr_gpu_stats_t stats() const override {
    amr_gpu_stats_t s = stats_;
    s.graph_nodes_per_trial = graph_nodes_;
    return s;
  }
  void set_event_timing(bool on) override { event_timing_ = on; }
  void set_graph(bool on) override {
    use_graph_ = on;
    graph_dirty_ = true;
  }

  int set_lanes(int lanes) override {
    if (lanes < 1 || lanes > MAX_LANES) return 1;
    lanes_wanted_ = lanes;
    tiles_dirty_ = true;  // the next advance plans the lanes again
    return 0;
  }

  std::string launch_config() const override {
    const char* name = mode_ == AMR_B200_LAUNCH_PHASES  ? "mode=phases"
                       : mode_ == AMR_B200_LAUNCH_SPLIT ? "mode=split"
                       : mode_ == AMR_B200_LAUNCH_TILED ? "mode=tiled"
                                                        : "mode=persistent";
    const int grid = mode_ == AMR_B200_LAUNCH_PHASES  ? (n_tiles_ + block_ / 32 - 1) / (block_ / 32)
                     : mode_ == AMR_B200_LAUNCH_SPLIT ? (int)((hw_cells_ + PHASE_BLOCK - 1) / PHASE_BLOCK)
                     : mode_ == AMR_B200_LAUNCH_TILED ? sms_ * TiledOcc<R>::blocks
                                                      : grid_;
    return std::string(name) + " block=" + std::to_string(block_) + " grid=" + std::to_string(grid) +
           (use_graph_ ? " graph" : " direct") +
           (mode_ == AMR_B200_LAUNCH_SPLIT && lanes_ > 1 ? " lanes=" + std::to_string(lanes_) : "");
  }
  int autotune(int trials, std::string* error) override;
  void restore(const std::vector<CaseCtl>& ctl_save, const DevBuf<R>& s0, const DevBuf<R>& s1, long long nbytes);

 private:
  static bool fail(std::string* error, const std::string& text) {
    if (error) *error = text;
    return false;
  }
  static int fail1(std::string* error, const std::string& text) {
    if (error) *error = text;
    return 1;
  }
  int fail_release(HostCase<R>& hc, std::string* error, const std::string& text) {
    release_ranges(hc);
    return fail1(error, text);
  }

  template <class T> static PVec<T> pv(PinnedStage& S, size_t count, const T& value) {
    return PVec<T>(count, value, PinAlloc<T>(&S));
  }
  template <class T> static PVec<T> pvu(PinnedStage& S, size_t count) {  // contents left uninitialised
    return PVec<T>(count, PinAlloc<T>(&S));
  }

  // Records the upload of a staged table; flush_uploads moves them all.
  static bool stage_up(Stager& st, void* dst, const void* host, size_t bytes) {
    if (bytes == 0) return true;
    const long long off = st.stage.dev_offset(host);
    if (off < 0) return false;
    st.uploads.push_back({reinterpret_cast<unsigned long long>(dst), (unsigned long long)off, (unsigned long long)bytes});
    return true;
  }
  template <class T> static bool up(Stager& st, T* dst, const PVec<T>& src, uint64_t* counter) {
    *counter += sizeof(T) * src.size();
    return stage_up(st, dst, src.data(), sizeof(T) * src.size());
  }

  // One DMA per used staging block into the worker's device staging buffer, then the scatter
  // kernel; asynchronous on stream_ (the staging memory is reused only after the worker's event).
  bool flush_uploads(Stager& st, std::string* error) {
    unsigned char* base = st.dev_ext;
    if (!base || st.stage.total() > st.dev_ext_n) {
      if (st.dev.n < st.stage.total()) {
        st.allocated -= st.dev.p ? st.dev.n : 0;
        st.dev.free();
        if (!st.dev.alloc(st.stage.total(), &st.allocated, error, "upload staging")) return false;
      }
      base = st.dev.p;
    }
    for (const PinnedStage::Block& b : st.stage.blocks())
      if (b.used && !cuda_ok(cudaMemcpyAsync(base + b.dev, b.p, b.used, cudaMemcpyHostToDevice, stream_), error,
                             "staging upload"))
        return false;
    for (size_t i0 = 0; i0 < st.uploads.size(); i0 += UPLOAD_TABLES) {
      UploadTable t;
      t.n = (int)std::min<size_t>(UPLOAD_TABLES, st.uploads.size() - i0);
      unsigned long long most = 0;
      for (int i = 0; i < t.n; ++i) {
        t.dst[i] = st.uploads[i0 + i].dst;
        t.src[i] = st.uploads[i0 + i].src;
        t.bytes[i] = st.uploads[i0 + i].bytes;
        most = std::max(most, t.bytes[i]);
      }
      const unsigned gx = (unsigned)std::min<unsigned long long>(64, (most + 8191) / 8192);
      scatter_uploads_kernel<<<dim3(gx, (unsigned)t.n), 256, 0, stream_>>>(base, t);
      if (!cuda_ok(cudaGetLastError(), error, "upload scatter")) return false;
    }
    return true;
  }

  int copy_out(const R* buf, int slot, double* out, uint64_t count, std::string* error) {
    if (slot < 0 || slot >= config_.max_cases || !cases_[slot].live) return fail1(error, "no such case");
    const HostCase<R>& hc = cases_[slot];
    const long long n = hc.n;
    if (count != (uint64_t)(nv_ * n)) return fail1(error, "state size mismatch");
    // one strided copy of the nv variable rows into page-locked staging lent by the pool
    const size_t bytes = sizeof(R) * nv_ * n;
    const LeaseGuard held(stream_, PinnedPool::get().lend(bytes, bytes));
    if (!held.lease.p) return fail1(error, "download staging: page-locked allocation failed");
    if (held.lease.fresh) stats_.pinned_bytes += held.lease.size;
    R* tmp = reinterpret_cast<R*>(held.lease.p);
    if (!cuda_ok(cudaMemcpy2DAsync(tmp, sizeof(R) * n, buf + hc.cells.b, sizeof(R) * cap_cells_, sizeof(R) * n, nv_,
                                   cudaMemcpyDeviceToHost, stream_), error, "download"))
      return 1;
    if (!cuda_ok(cudaStreamSynchronize(stream_), error, "download sync")) return 1;
    for (long long i = 0; i < nv_ * n; ++i) out[i] = (double)tmp[i];
    return 0;
  }

  // A start state of nv values (rather than nv per cell) is the same state in every cell.
  bool uniform_start(uint64_t u0_count, long long n) const { return n > 1 && u0_count == (uint64_t)nv_; }

  bool validate(const amr_mesh_view_t& m, const amr_params_t& p, uint64_t u0_count, std::string* why) const {
    const auto finite = [](double x) { return std::isfinite(x); };
    if (m.n_cells == 0 || m.n_faces == 0 || !m.cells || !m.faces || !m.face_offsets || !m.cell_faces)
      return fail(why, "empty mesh");
    if (m.n_cells + 1 > (uint64_t)0x3fffffff || m.face_offsets[m.n_cells] > (uint64_t)0x3fffffff)
      return fail(why, "mesh too large for 32-bit indices");
    const int sa = m.transport.sa_model ? 1 : 0;
    const int model = m.transport.model == AMR_B200_MODEL_EULER ? MODEL_EULER : (sa ? MODEL_SA : MODEL_LAMINAR);
    if (model != model_) return fail(why, "flow model differs from the batch's");
    const int flux = p.flux == AMR_B200_FLUX_AUSMPUP ? FLUX_AUSM : FLUX_HLLC;
    if (flux != flux_ && model_ >= 0) return fail(why, "numerical flux differs from the batch's");
    if (u0_count != (uint64_t)(nv_ * m.n_cells) && !uniform_start(u0_count, (long long)m.n_cells))
      return fail(why, "initial state size mismatch");
    if (p.limiter != AMR_B200_LIMITER_FIRST_ORDER || p.time_integrator != AMR_B200_TIME_SSP_RK3 || !finite(p.gamma) ||
        !(p.gamma > 1) || !(p.cfl > 0) || p.cfl > .5 || !finite(p.dt_fixed) || p.dt_fixed < 0 || !finite(p.ausm_mco) ||
        p.ausm_mco <= 0 || (p.flux != AMR_B200_FLUX_HLLC && p.flux != AMR_B200_FLUX_AUSMPUP))
      return fail(why, "invalid AMR GPU configuration");
    // transport (reference src/static_amr2d_viscous.h:43-51)
    const amr_transport_t& t = m.transport;
    if (t.model == AMR_B200_MODEL_EULER) {
      if (t.sa_model) return fail(why, "invalid transport");
      for (int side = 0; side < 4; ++side)
        if (m.boundaries[side].kind == AMR_B200_BC_NOSLIP) return fail(why, "no-slip wall requires laminar model");
    } else {
      const bool sa_ok = !t.sa_model || (t.sa_model == 1 && finite(t.sa_nu_inf) && t.sa_nu_inf >= 0 && finite(t.sa_cfl) &&
                                         t.sa_cfl > 0 && t.sa_cfl <= .1);
      if (!sa_ok || t.model != AMR_B200_MODEL_LAMINAR || (t.law != AMR_B200_MU_CONSTANT && t.law != AMR_B200_MU_SUTHERLAND) ||
          !finite(t.mu_ref) || !(t.mu_ref > 0) || !finite(t.gas_constant) || !(t.gas_constant > 0) ||
          !finite(t.temperature_ref) || !(t.temperature_ref > 0) || !finite(t.sutherland) || t.sutherland < 0 ||
          !finite(t.viscous_cfl) || !(t.viscous_cfl > 0) || t.viscous_cfl > .2 ||
          (t.stabilization != AMR_B200_VISCOUS_VOLUME && t.stabilization != AMR_B200_VISCOUS_SRD) ||
          !finite(t.wall_probe_min_h) || t.wall_probe_min_h < 0 || t.wall_probe_min_h > 2)
        return fail(why, "invalid laminar transport parameters");
      if (!m.visc_offsets || !m.visc_terms || (m.n_walls && !m.wall_samples) || !m.face_samples || !m.face_geometry)
        return fail(why, "viscous tables missing");
      if (t.sa_model && !m.wall_distance) return fail(why, "SA wall distance missing");
    }
    if (m.small_cells && (!m.group_offsets || !m.group_members || !m.member_offsets || !m.member_groups || !m.group_volume))
      return fail(why, "SRD tables missing");
    // boundaries (reference src/static_amr2d_boundary.h:32-47)
    for (int side = 0; side < 4; ++side) {
      const amr_boundary_t& b = m.boundaries[side];
      if (b.kind < AMR_B200_BC_INHERIT) return fail(why, "invalid AMR GPU boundary configuration");
      const int kind = b.kind < 0 ? p.bc[side] : b.kind;
      if (kind == AMR_B200_BC_TRANSMISSIVE || kind == AMR_B200_BC_REFLECT) continue;
      if (kind == AMR_B200_BC_NOSLIP) {
        if (!finite(b.wall_velocity[0]) || !finite(b.wall_velocity[1]) || b.wall_velocity[side / 2] != 0)
          return fail(why, "invalid AMR GPU boundary configuration");
        continue;
      }
      const double* w = b.reference;
      const bool prim = finite(w[0]) && w[0] > 0 && finite(w[1]) && finite(w[2]) && finite(w[3]) && w[3] > 0;
      if (kind < AMR_B200_BC_FARFIELD || kind > AMR_B200_BC_PRESSURE_OUTLET || !prim)
        return fail(why, "invalid AMR GPU boundary configuration");
      if (kind == AMR_B200_BC_PRESSURE_OUTLET && !(finite(b.outlet_pressure) && b.outlet_pressure > 0))
        return fail(why, "invalid AMR GPU boundary configuration");
      if (kind == AMR_B200_BC_TOTAL_INLET) {
        const double d2 = b.direction[0] * b.direction[0] + b.direction[1] * b.direction[1];
        const double dn = (side % 2 ? 1.0 : -1.0) * b.direction[side / 2];
        if (!(finite(d2) && std::fabs(d2 - 1) < 1e-12 && dn < 0 && finite(b.total_pressure) && b.total_pressure > 0 &&
              finite(b.total_temperature) && b.total_temperature > 0 && finite(b.gas_constant) && b.gas_constant > 0))
          return fail(why, "invalid AMR GPU boundary configuration");
      }
    }
    return true;
  }

  bool make_tiles(HostCase<R>& hc, std::string* why) const {
    const long long n = hc.n;
    const int cb = (int)hc.cells.b;
    const int B = TILE_W;
    hc.tiles.clear();
    long long k = 0;
    bool first = true;
    while (k < n) {
      const long long start = k;
      long long slots = 0, terms = 0;
      while (k < n && k - start < B) {
        const long long ds = hc.nslot[k], dt = hc.nterm[k];
        if (slots + ds > B || terms + dt > B) break;
        slots += ds;
        terms += dt;
        ++k;
      }
      if (k == start) return fail(why, "a cell has more faces or gradient terms than a tile (32)");
      Tile t;
      t.cs = hc.slot;
      t.c0 = cb + (int)start;
      t.c1 = cb + (int)k;
      t.leader = first ? 1 : 0;
      t.s0 = (int)hc.slots.b + hc.slot_prefix[start];
      t.s1 = (int)hc.slots.b + hc.slot_prefix[k];
      t.t0 = (int)hc.terms.b + hc.term_prefix[start];
      t.t1 = (int)hc.terms.b + hc.term_prefix[k];
      hc.tiles.push_back(t);
      first = false;
    }
    return true;
  }

  bool retile(HostCase<R>& hc) {
    std::string why;
    return make_tiles(hc, &why);
  }

  long long n_btiles_total() const {
    long long s = 0;
    for (auto& c : cases_)
      if (c.live) s += (long long)c.btiles.size();
    return s;
  }

  // Block tiles of one case (case-local indices): runs of up to BT_CELLS consecutive cells whose
  // halo (face neighbours and wall donors outside the run), face records and wall fragments fit
  // the tiled kernel's shared memory.  Fills per slot its local record (2 * tile face + the cell
  // is the face's left, or the tile wall index) and per wall the donor's local index.
  bool make_block_tiles(const amr_mesh_view_t* m, long long n, const std::vector<int>& rec, int slot,
                        std::vector<BTile>* tiles, std::vector<int>* halo_out, std::vector<int>* face_out,
                        std::vector<int2>* floc_out, std::vector<int>* s_loc, std::vector<int>* w_ldon,
                        std::string* why) const {
    const long long nf = (long long)m->n_faces;
    const bool viscous = model_ >= MODEL_LAMINAR;
    std::vector<int> dstamp(n, -1), dloc(n, 0), fstamp(nf, -1), floc(nf, 0);
    std::vector<int> halo, faces;
    std::vector<long long> slot_base(n + 1, 0);  // case-local slot index of each cell's first slot
    for (long long k = 0; k < n; ++k)
      slot_base[k + 1] = slot_base[k] + (long long)(m->face_offsets[k + 1] - m->face_offsets[k] + m->cells[k].wall_count);
    int stamp = 0;
    long long start = 0;
    while (start < n) {
      long long end = std::min<long long>(n, start + BT_CELLS);
      for (;;) {
        ++stamp;
        halo.clear();
        faces.clear();
        const int nt = (int)(end - start);
        for (long long k = start; k < end; ++k) {
          dstamp[k] = stamp;
          dloc[k] = (int)(k - start);
        }
        auto add_cell = [&](long long c) {
          if (dstamp[c] == stamp) return;
          dstamp[c] = stamp;
          dloc[c] = nt + (int)halo.size();
          halo.push_back((int)c);
        };
        for (long long k = start; k < end; ++k) {
          for (uint64_t q = m->face_offsets[k]; q < m->face_offsets[k + 1]; ++q) {
            const uint64_t fi = m->cell_faces[q];
            const amr_face_t& f = m->faces[fi];
            if (fstamp[fi] != stamp) {
              fstamp[fi] = stamp;
              floc[fi] = (int)faces.size();
              faces.push_back((int)fi);
            }
            const int other = f.left == (int)k ? f.right : f.left;
            if (other >= 0) add_cell(other);
          }
          if (viscous)
            for (uint64_t q = m->cells[k].wall_begin; q < m->cells[k].wall_begin + m->cells[k].wall_count; ++q)
              add_cell(m->wall_samples[q].donor);
        }
        const long long nw = (long long)(m->cells[end - 1].wall_begin + m->cells[end - 1].wall_count) -
                             (long long)m->cells[start].wall_begin;
        if (nt + (long long)halo.size() <= BT_DATA && (long long)faces.size() <= BT_FACES && nw <= BT_WALLS) break;
        if (end - start == 1) return fail(why, "a cell's neighbourhood exceeds the block tile");
        end = start + std::max<long long>(1, (end - start) * 3 / 4);
      }
      BTile t;
      t.cs = slot;
      t.c0 = (int)start;
      t.c1 = (int)end;
      t.h0 = (int)halo_out->size();
      t.h1 = t.h0 + (int)halo.size();
      t.f0 = (int)face_out->size();
      t.f1 = t.f0 + (int)faces.size();
      t.w0 = (int)m->cells[start].wall_begin;
      t.w1 = (int)(m->cells[end - 1].wall_begin + m->cells[end - 1].wall_count);
      halo_out->insert(halo_out->end(), halo.begin(), halo.end());
      for (int fi : faces) {
        const amr_face_t& f = m->faces[fi];
        const int own = f.left >= 0 ? f.left : f.right, other = f.left >= 0 ? f.right : -1;
        face_out->push_back(rec[fi]);
        floc_out->push_back(make_int2(dloc[own], other >= 0 ? dloc[other] : -1));
      }
      for (long long k = start; k < end; ++k) {
        long long q = slot_base[k];
        for (uint64_t p = m->face_offsets[k]; p < m->face_offsets[k + 1]; ++p, ++q) {
          const uint64_t fi = m->cell_faces[p];
          (*s_loc)[q] = 2 * floc[fi] + (m->faces[fi].left == (int)k ? 1 : 0);
        }
        for (uint64_t w = m->cells[k].wall_begin; w < m->cells[k].wall_begin + m->cells[k].wall_count; ++w, ++q) {
          (*s_loc)[q] = (int)(w - (uint64_t)t.w0);
          if (viscous) (*w_ldon)[w] = dloc[m->wall_samples[w].donor];
        }
      }
      tiles->push_back(t);
      start = end;
    }
    return true;
  }

  long long n_tiles_total() const {
    long long s = 0;
    for (auto& c : cases_)
      if (c.live) s += (long long)c.tiles.size();
    return s;
  }

  // Marks a case's cells, faces and walls as belonging to no case (asynchronous on stream_).
  void unmark_ranges(const HostCase<R>& hc) {
    if (hc.cells.n) cudaMemsetAsync(c_case_.p + hc.cells.b, 0xff, sizeof(int) * hc.cells.n, stream_);
    if (hc.faces.n) cudaMemsetAsync(f_case_.p + hc.faces.b, 0xff, sizeof(int) * hc.faces.n, stream_);
    if (hc.walls.n) cudaMemsetAsync(w_owner_.p + hc.walls.b, 0xff, sizeof(int) * hc.walls.n, stream_);
  }

  void release_ranges(HostCase<R>& hc) {
    a_cells_.release(hc.cells.b, hc.cells.b >= 0 ? hc.cells.n : 0);
    a_slots_.release(hc.slots.b, hc.slots.b >= 0 ? hc.slots.n : 0);
    a_walls_.release(hc.walls.b, hc.walls.b >= 0 ? hc.walls.n : 0);
    a_terms_.release(hc.terms.b, hc.terms.b >= 0 ? hc.terms.n : 0);
    a_groups_.release(hc.groups.b, hc.groups.b >= 0 ? hc.groups.n : 0);
    a_gmem_.release(hc.gmembers.b, hc.gmembers.b >= 0 ? hc.gmembers.n : 0);
    a_q_.release(hc.qcells.b, hc.qcells.b >= 0 ? hc.qcells.n : 0);
    a_qlist_.release(hc.qlist.b, hc.qlist.b >= 0 ? hc.qlist.n : 0);
    a_faces_.release(hc.faces.b, hc.faces.b >= 0 ? hc.faces.n : 0);
    a_halo_.release(hc.halo.b, hc.halo.b >= 0 ? hc.halo.n : 0);
    a_tface_.release(hc.tfaces.b, hc.tfaces.b >= 0 ? hc.tfaces.n : 0);
    hc.cells = hc.slots = hc.walls = hc.terms = hc.groups = hc.gmembers = hc.qcells = hc.qlist = hc.faces = hc.halo =
        hc.tfaces = Range{0, 0};
  }

  void refresh_meta(int slot) {
    const CaseCtl& c = h_ctl_[slot];
    CaseMeta& m = meta_[slot];
    m.time = c.time;
    m.target = c.target;
    m.dt = c.dt;
    m.dt_trial = c.dt_trial;
    m.steps = c.steps;
    m.rejected = c.rejected;
    m.maxsteps = c.maxsteps;
    m.fatal = c.fatal;
    m.finished = c.finished;
    m.active = c.active;
    m.live = c.live;
    m.cur = c.cur;
  }

  // Split mode, viscous models without SRD: the live cases in up to lanes_wanted_ lanes of about
  // equal cells, each advanced by its own chain of kernels (so that one lane's kernels fill the
  // tails of the others').  A lane must own whole ranges: every case of a lane has its cells, faces
  // and walls below every case of the next lane, as after admissions in one order; otherwise (or
  // with fewer than two cases) one lane.
  bool plan_lanes(std::string* error) {
    lanes_ = 1;
    if (lanes_wanted_ < 2 || mode_ != AMR_B200_LAUNCH_SPLIT || model_ < MODEL_LAMINAR || any_srd()) return true;
    std::vector<int> live;
    for (int i = 0; i < config_.max_cases; ++i)
      if (cases_[i].live) live.push_back(i);
    const int want = std::min<int>(lanes_wanted_, (int)live.size());
    if (want < 2) return true;
    std::sort(live.begin(), live.end(), [&](int a, int b) { return cases_[a].cells.b < cases_[b].cells.b; });
    // cut[l]: the first case of lane l, where the cells before it first reach l / want of the
    // total, with at least one case in every lane
    const size_t m = live.size();
    std::vector<long long> before(m + 1, 0);
    for (size_t q = 0; q < m; ++q) before[q + 1] = before[q] + cases_[live[q]].cells.n;
    std::vector<size_t> cut(want + 1, 0);
    cut[want] = m;
    for (int l = 1; l < want; ++l) {
      size_t q = cut[l - 1] + 1;
      const size_t last = m - (size_t)(want - l);
      while (q < last && before[q] * want < (long long)l * before[m]) ++q;
      cut[l] = q;
    }
    std::vector<int> lane_of(m, 0);
    for (int l = 0; l < want; ++l)
      for (size_t q = cut[l]; q < cut[l + 1]; ++q) lane_of[q] = l;
    // per lane and table (cells, faces, walls): the lowest begin and the highest end of its ranges
    const long long hw[3] = {hw_cells_, hw_faces_, hw_walls_};
    long long lo[MAX_LANES][3], hi[MAX_LANES][3];
    for (int l = 0; l < want; ++l)
      for (int t = 0; t < 3; ++t) {
        lo[l][t] = hw[t];
        hi[l][t] = 0;
      }
    for (size_t q = 0; q < live.size(); ++q) {
      const HostCase<R>& hc = cases_[live[q]];
      const Range r[3] = {hc.cells, hc.faces, hc.walls};
      for (int t = 0; t < 3; ++t)
        if (r[t].n) {
          lo[lane_of[q]][t] = std::min(lo[lane_of[q]][t], r[t].b);
          hi[lane_of[q]][t] = std::max(hi[lane_of[q]][t], r[t].b + r[t].n);
        }
    }
    // lane boundaries from the top: lane l covers [bound[l], bound[l + 1])
    long long bound[MAX_LANES + 1][3];
    for (int t = 0; t < 3; ++t) {
      bound[want][t] = hw[t];
      for (int l = want - 1; l >= 1; --l) bound[l][t] = std::min(bound[l + 1][t], lo[l][t]);
      bound[0][t] = 0;
      for (int l = 0; l < want; ++l)
        if (hi[l][t] > bound[l + 1][t]) return true;  // interleaved ranges: one lane
    }
    for (int l = 0; l < want; ++l) {
      int* h = h_lane_ranges_ + 8 * l;
      for (int t = 0; t < 3; ++t) {
        h[t] = (int)bound[l + 1][t];
        h[4 + t] = (int)bound[l][t];
      }
      h[3] = h_live_end_[3];
      h[7] = 0;
    }
    h_case_lane_.assign(config_.max_cases, -1);
    for (size_t q = 0; q < live.size(); ++q) h_case_lane_[live[q]] = lane_of[q];
    if (!cuda_ok(cudaMemcpyAsync(lane_ranges_.p, h_lane_ranges_, sizeof(int) * 8 * want, cudaMemcpyHostToDevice, stream_),
                 error, "lanes") ||
        !cuda_ok(cudaMemcpyAsync(case_lane_.p, h_case_lane_.data(), sizeof(int) * h_case_lane_.size(),
                                 cudaMemcpyHostToDevice, stream_), error, "lanes"))
      return false;
    lanes_ = want;
    return true;
  }

  bool sync_tiles(std::string* error) {
    if (!tiles_dirty_) return true;
    std::vector<Tile> all;
    std::vector<int> ranges(2 * config_.max_cases, 0);
    for (int i = 0; i < config_.max_cases; ++i) {
      ranges[2 * i] = (int)all.size();
      if (cases_[i].live) all.insert(all.end(), cases_[i].tiles.begin(), cases_[i].tiles.end());
      ranges[2 * i + 1] = (int)all.size();
    }
    n_tiles_ = (int)all.size();
    hw_cells_ = hw_faces_ = hw_walls_ = 0;  // ends of the highest live ranges (split-mode grids)
    for (auto& c : cases_)
      if (c.live) {
        hw_cells_ = std::max(hw_cells_, c.cells.b + c.cells.n);
        hw_faces_ = std::max(hw_faces_, c.faces.b + c.faces.n);
        hw_walls_ = std::max(hw_walls_, c.walls.b + c.walls.n);
      }
    h_live_end_[0] = (int)hw_cells_;
    h_live_end_[1] = (int)hw_faces_;
    h_live_end_[2] = (int)hw_walls_;
    if (!plan_lanes(error)) return false;
    std::vector<BTile> all_bt;
    for (auto& c : cases_)
      if (c.live) all_bt.insert(all_bt.end(), c.btiles.begin(), c.btiles.end());
    h_live_end_[3] = (int)all_bt.size();
    if (!all_bt.empty() && !cuda_ok(cudaMemcpyAsync(btiles_.p, all_bt.data(), sizeof(BTile) * all_bt.size(),
                                                    cudaMemcpyHostToDevice, stream_), error, "block tiles"))
      return false;
    if (!cuda_ok(cudaMemcpyAsync(live_end_.p, h_live_end_, sizeof(h_live_end_), cudaMemcpyHostToDevice, stream_), error,
                 "live ranges"))
      return false;
    if (!all.empty() && !cuda_ok(cudaMemcpyAsync(tiles_.p, all.data(), sizeof(Tile) * all.size(), cudaMemcpyHostToDevice,
                                                 stream_), error, "tiles"))
      return false;
    if (!cuda_ok(cudaMemcpyAsync(case_tiles_.p, ranges.data(), sizeof(int) * ranges.size(), cudaMemcpyHostToDevice, stream_),
                 error, "tile ranges"))
      return false;
    case_tile_ranges_ = ranges;
    tiles_dirty_ = false;
    // a split-mode graph reads the live ranges from the device and keeps its grids; it is
    // recaptured only when the set of kernels changes (SRD launches appear or vanish)
    if ((mode_ != AMR_B200_LAUNCH_SPLIT && mode_ != AMR_B200_LAUNCH_TILED) || any_srd() != graph_srd_ ||
        any_srd_rate() != graph_srd_rate_ || lanes_ != graph_lanes_)
      graph_dirty_ = true;
    return cuda_ok(cudaStreamSynchronize(stream_), error, "tiles sync");
  }

  Dev<R> dev() const {
    Dev<R> d;
    std::memset(&d, 0, sizeof(d));
    d.ctl = ctl_.p;
    d.cfg = cfg_.p;
    d.tiles = tiles_.p;
    d.n_tiles = n_tiles_;
    d.n_cases = config_.max_cases;
    d.c_case = c_case_.p;
    d.c_vol = c_vol_.p;
    d.c_area = c_area_.p;
    d.c_gvol = c_gvol_.p;
    d.c_flags = c_flags_.p;
    d.c_slot = c_slot_.p;
    d.c_wall = c_wall_.p;
    d.c_term = c_term_.p;
    d.c_wd = c_wd_.p;
    d.s_own = s_own_.p;
    d.s_nb = s_nb_.p;
    d.s_meta = s_meta_.p;
    d.s_len = s_len_.p;
    d.s_geo = s_geo_.p;
    d.w_nx = w_nx_.p;
    d.w_ny = w_ny_.p;
    d.w_len = w_len_.p;
    d.w_dist = w_dist_.p;
    d.w_donor = w_donor_.p;
    d.t_own = t_own_.p;
    d.t_src = t_src_.p;
    d.t_x = t_x_.p;
    d.t_y = t_y_.p;
    d.g_mem = g_mem_.p;
    d.g_cell = g_cell_.p;
    d.g_cnt = g_cnt_.p;
    d.g_vol = g_vol_.p;
    d.q_cell = q_cell_.p;
    d.q_grp = q_grp_.p;
    d.q_list = q_list_.p;
    d.q_cnt = q_cnt_.p;
    d.qhat = qhat_.p;
    d.U0 = U0_.p;
    d.U1 = U1_.p;
    d.U2 = U2_.p;
    d.L0 = L0_.p;
    d.L1 = L1_.p;
    d.R0 = R0_.p;
    d.grad = grad_.p;
    d.mu = mu_.p;
    d.eddy = eddy_.p;
    d.sgrad = sgrad_.p;
    d.sdiff = sdiff_.p;
    d.ssrc = ssrc_.p;
    d.srate = srate_.p;
    d.f_case = f_case_.p;
    d.f_own = f_own_.p;
    d.f_nb = f_nb_.p;
    d.f_meta = f_meta_.p;
    d.f_len = f_len_.p;
    d.f_geo = f_geo_.p;
    d.w_owner = w_owner_.p;
    d.s_item = s_item_.p;
    d.fval = fval_.p;
    d.fsa = fsa_.p;
    d.wsa = wsa_.p;
    d.wval = wval_.p;
    d.crec = crec_.p;
    d.ddt = ddt_.p;
    d.any_srd_rate = any_srd_rate() ? 1 : 0;
    d.w_xm = w_xm_.p;
    d.w_ym = w_ym_.p;
    d.live_end = live_end_.p;
    d.btiles = btiles_.p;
    d.bt_halo = bt_halo_.p;
    d.bt_face = bt_face_.p;
    d.bt_floc = bt_floc_.p;
    d.s_loc = s_loc_.p;
    d.w_ldon = w_ldon_.p;
    d.cap_faces = (int)cap_faces_;
    d.cap_walls = (int)cap_walls_;
    d.n_faces = (int)hw_faces_;
    d.n_walls = (int)hw_walls_;
    d.n_cells = (int)hw_cells_;
    d.ncap = cap_cells_;
    d.gcap = cap_groups_ + config_.max_cases;
    d.bar = bar_.p;
    d.barrier_cycles = (unsigned long long)clock_khz_ * 1000ull * 2ull;  // about two seconds
    return d;
  }

  uint64_t kernels_per_advance(int trials) const {
    if (mode_ == AMR_B200_LAUNCH_PERSISTENT) return 1;
    // per trial: three flux stages (one kernel, or item + gather), gradients per stage, the
    // first update, SRD after each stage and the commit; plus the opening commit
    const uint64_t flux = mode_ == AMR_B200_LAUNCH_SPLIT ? 2 : 1;
    const uint64_t grad = model_ >= MODEL_LAMINAR && mode_ != AMR_B200_LAUNCH_TILED ? 3 : 0;
    const uint64_t per_trial = 3 * flux + grad + 1 + (any_srd() ? 3 : 0) + 1 + (any_srd_rate() ? 1 : 0);
    const uint64_t lanes = mode_ == AMR_B200_LAUNCH_SPLIT ? (uint64_t)lanes_ : 1;
    return lanes * (1 + per_trial * trials);
  }

  bool any_srd() const {
    for (auto& c : cases_)
      if (c.live && c.cfg.has_srd) return true;
    return false;
  }

  bool any_srd_rate() const {
    for (auto& c : cases_)
      if (c.live && c.cfg.srd_rate) return true;
    return false;
  }

  // values per stored face or wall record (the compact FP32 viscous format stores 8)
  long long rec_stride() const {
    return sizeof(R) == 4 && model_ >= MODEL_LAMINAR ? 8 : SM_COLS;
  }

  bool configure_grid(std::string* error) {
    int per_sm = 0;
    if (!cuda_ok(EngineOps<R>::occupancy(model_, flux_, true, block_, &per_sm), error, "occupancy")) return false;
    int per_sm2 = 0;
    if (!cuda_ok(EngineOps<R>::occupancy(model_, flux_, false, block_, &per_sm2), error, "occupancy")) return false;
    per_sm = std::min(per_sm, per_sm2);
    if (per_sm < 1) return fail(error, "kernel does not fit on an SM");
    max_grid_ = per_sm * sms_;
    grid_ = grid_request_ > 0 ? std::min(grid_request_, max_grid_) : max_grid_;
    return true;
  }

  // Launch sequence of one advance: barrier reset, the persistent kernel, and (trial mode)
  // the control and barrier read-back.  Timing events are recorded around it only when the
  // sequence is issued directly; a graph launch is timed by events outside the graph.
  bool enqueue(int trials, int mode, std::string* error, bool events = true) {
    bool ok = true;
    if (events) ok = cuda_ok(cudaEventRecord(ev0_, stream_), error, "event");
    if (mode_ == AMR_B200_LAUNCH_PHASES) {
      ok = ok && cuda_ok(EngineOps<R>::launch_phases(dev(), model_, flux_, any_srd(), trials, mode, block_, stream_), error,
                         "phase kernel launch");
    } else if (mode_ == AMR_B200_LAUNCH_SPLIT) {
      SplitLanes<R> lanes;
      if (lanes_ >= 2) {
        lanes.n = lanes_;
        for (int l = 0; l < lanes_; ++l) {
          lanes.dev[l] = dev();
          lanes.dev[l].live_end = lane_ranges_.p + 8 * l;
          lanes.dev[l].live_begin = lane_ranges_.p + 8 * l + 4;
          lanes.dev[l].case_lane = case_lane_.p;
          lanes.dev[l].lane = l;
        }
        for (int l = 0; l < MAX_LANES - 1; ++l) {
          lanes.aux[l] = aux_[l];
          lanes.join[l] = join_[l];
        }
        lanes.fork = fork_;
      }
      ok = ok && cuda_ok(EngineOps<R>::launch_split(dev(), model_, flux_, any_srd(), trials, mode, stream_, sms_, &lanes),
                         error, "split kernel launch");
    } else if (mode_ == AMR_B200_LAUNCH_TILED) {
      ok = ok && cuda_ok(EngineOps<R>::launch_tiled(dev(), model_, flux_, any_srd(), trials, mode, stream_, sms_), error,
                         "tiled kernel launch");
    } else {
      const int grid = mode == MODE_RESIDUAL ? std::min(grid_, std::max(1, (n_tiles_ + block_ / 32 - 1) / (block_ / 32))) : grid_;
      ok = ok && cuda_ok(cudaMemsetAsync(bar_.p, 0, sizeof(GridBarrier), stream_), error, "barrier reset") &&
           cuda_ok(EngineOps<R>::launch(dev(), model_, flux_, any_srd(), trials, mode, grid, block_, stream_, true), error,
                   "trial kernel launch");
    }
    if (events) ok = ok && cuda_ok(cudaEventRecord(ev1_, stream_), error, "event");
    if (ok && mode == MODE_TRIALS)
      ok = cuda_ok(cudaMemcpyAsync(h_ctl_, ctl_.p, sizeof(CaseCtl) * config_.max_cases, cudaMemcpyDeviceToHost, stream_),
                   error, "control read-back");
    if (ok && mode == MODE_TRIALS && mode_ == AMR_B200_LAUNCH_PERSISTENT)
      ok = cuda_ok(cudaMemcpyAsync(h_bar_, bar_.p, sizeof(GridBarrier), cudaMemcpyDeviceToHost, stream_), error,
                   "barrier read-back");
    return ok;
  }

  bool capture(int trials, std::string* error) {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
    if (!cuda_ok(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), error, "capture begin")) return false;
    std::string err;
    const bool ok = enqueue(trials, MODE_TRIALS, &err, false);
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(stream_, &g);
    if (!ok || end != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      if (error) *error = "graph capture failed: " + err;
      return false;
    }
    graph_ = g;
    if (cudaGraphInstantiate(&graph_exec_, graph_, nullptr, nullptr, 0) != cudaSuccess) {
      cudaGraphDestroy(graph_);
      graph_ = nullptr;
      graph_exec_ = nullptr;
      return false;
    }
    size_t nodes = 0;
    cudaGraphGetNodes(graph_, nullptr, &nodes);
    graph_nodes_ = nodes;
    graph_trials_ = trials;
    graph_srd_ = any_srd();
    graph_srd_rate_ = any_srd_rate();
    graph_lanes_ = lanes_;
    graph_dirty_ = false;
    return true;
  }

  void destroy() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
    DevBufFreeAll();
    if (h_ctl_) cudaFreeHost(h_ctl_);
    if (h_bar_) cudaFreeHost(h_bar_);
    h_ctl_ = nullptr;
    h_bar_ = nullptr;
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    ev0_ = ev1_ = nullptr;
    if (stream_) cudaStreamDestroy(stream_);
    for (int l = 0; l < MAX_LANES - 1; ++l) {
      if (aux_[l]) cudaStreamDestroy(aux_[l]);
      if (join_[l]) cudaEventDestroy(join_[l]);
      aux_[l] = nullptr;
      join_[l] = nullptr;
    }
    if (fork_) cudaEventDestroy(fork_);
    fork_ = nullptr;
    stream_ = nullptr;
  }

  void DevBufFreeAll() {
    free_arena();
    if (slab_) cudaFree(slab_);  // the carved tables below only forget their pointers
    slab_ = nullptr;
    stagers_.clear();
    ctl_.free(); cfg_.free(); tiles_.free(); bar_.free();
    c_case_.free(); c_vol_.free(); c_area_.free(); c_gvol_.free(); c_flags_.free(); c_slot_.free(); c_wall_.free();
    c_term_.free(); c_cx_.free(); c_cy_.free(); c_wd_.free();
    s_own_.free(); s_nb_.free(); s_meta_.free(); s_len_.free(); s_geo_.free(); s_item_.free();
    f_case_.free(); f_own_.free(); f_nb_.free(); f_meta_.free(); f_len_.free(); f_geo_.free(); fval_.free();
    w_owner_.free(); wval_.free(); crec_.free(); live_end_.free(); ddt_.free(); ex_buf_.free();
    btiles_.free(); bt_halo_.free(); bt_face_.free(); bt_floc_.free(); s_loc_.free(); w_ldon_.free();
    w_nx_.free(); w_ny_.free(); w_len_.free(); w_dist_.free(); w_donor_.free(); w_xm_.free(); w_ym_.free();
    t_own_.free(); t_src_.free(); t_x_.free(); t_y_.free();
    g_mem_.free(); g_cell_.free(); g_cnt_.free(); g_vol_.free(); q_cell_.free(); q_grp_.free(); q_list_.free(); q_cnt_.free();
    qhat_.free();
    U0_.free(); U1_.free(); U2_.free(); R0_.free(); L0_.free(); L1_.free(); fsa_.free(); wsa_.free(); grad_.free(); mu_.free(); eddy_.free(); sgrad_.free(); sdiff_.free();
    ssrc_.free(); srate_.free(); diag_part_.free(); diag_out_.free(); diag_cfg_.free(); case_tiles_.free();
  }

  amr_batch_config_t config_{};
  int model_ = 0, flux_ = 0, nv_ = 4, sms_ = 148, clock_khz_ = 1965000;
  int block_ = 256, grid_ = 0, max_grid_ = 0, grid_request_ = 0;
  bool in_flight_ = false;  // an advance_begin awaits its advance_end
  int in_flight_trials_ = 0;
  int mode_ = AMR_B200_LAUNCH_PERSISTENT;  // persistent cooperative kernel, one kernel per phase, or split
  long long hw_cells_ = 0, hw_faces_ = 0, hw_walls_ = 0;
  int h_live_end_[4] = {0, 0, 0, 0};
  bool graph_srd_ = false, graph_srd_rate_ = false;
  // split mode in lanes (plan_lanes): count, wanted count, the count the graph was captured with
  // (three lanes measured fastest on 256 cases: 0.72-0.73 ms/step, two 0.75, four 0.73-0.74, one 0.78)
  int lanes_ = 1, lanes_wanted_ = 3, graph_lanes_ = 1;
  int h_lane_ranges_[8 * MAX_LANES] = {};
  std::vector<int> h_case_lane_;
  cudaStream_t aux_[MAX_LANES - 1] = {};
  cudaEvent_t fork_ = nullptr, join_[MAX_LANES - 1] = {};
  DevBuf<int> lane_ranges_;  // per lane: ends of cells, faces, walls, block tiles; begins of cells, faces, walls
  DevBuf<int> case_lane_;    // per case slot: its lane (-1 not live)

  DevBuf<int> live_end_;
  long long cap_faces_ = 0;
  RangeAlloc a_faces_;
  long long cap_halo_ = 0, cap_tface_ = 0, cap_btiles_ = 0;
  RangeAlloc a_halo_, a_tface_;
  DevBuf<BTile> btiles_;
  DevBuf<int> bt_halo_, bt_face_, s_loc_, w_ldon_;
  DevBuf<int2> bt_floc_;
  long long cap_cells_ = 0, cap_slots_ = 0, cap_walls_ = 0, cap_terms_ = 0, cap_groups_ = 0, cap_gmem_ = 0, cap_q_ = 0,
            cap_qlist_ = 0, cap_tiles_ = 0;
  RangeAlloc a_cells_, a_slots_, a_walls_, a_terms_, a_groups_, a_gmem_, a_q_, a_qlist_;
  std::vector<HostCase<R>> cases_;
  std::vector<CaseMeta> meta_;
  int live_ = 0, n_tiles_ = 0;
  bool tiles_dirty_ = true, graph_dirty_ = true, use_graph_ = true, event_timing_ = true;
  int graph_trials_ = 0;
  uint64_t graph_nodes_ = 0, launches_ = 0;
  double last_seconds_ = 0;
  std::vector<int> case_tile_ranges_;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  CaseCtl* h_ctl_ = nullptr;
  GridBarrier* h_bar_ = nullptr;
  amr_gpu_stats_t stats_{};
  DevBuf<CaseCtl> ctl_;
  DevBuf<CaseCfg<R>> cfg_;
  DevBuf<Tile> tiles_;
  DevBuf<GridBarrier> bar_;
  DevBuf<int> c_case_, c_slot_, c_wall_, c_term_;
  DevBuf<double> c_vol_, c_area_, c_gvol_, c_cx_, c_cy_;
  DevBuf<unsigned char> c_flags_;
  DevBuf<R> c_wd_;
  DevBuf<int> s_own_, s_nb_, s_meta_, s_item_;
  DevBuf<R> s_len_, s_geo_;
  DevBuf<int> f_case_, f_own_, f_nb_, f_meta_, w_owner_;
  DevBuf<R> f_len_, f_geo_, fval_, wval_, crec_;
  DevBuf<R> w_nx_, w_ny_, w_len_, w_dist_;
  DevBuf<double> w_xm_, w_ym_;
  DevBuf<int> w_donor_;
  DevBuf<int> t_own_, t_src_;
  DevBuf<R> t_x_, t_y_;
  DevBuf<int> g_mem_, g_cell_, q_cell_, q_grp_, q_list_;
  DevBuf<double> g_cnt_, g_vol_, q_cnt_, qhat_;
  DevBuf<R> U0_, U1_, U2_, R0_, grad_, mu_, eddy_, sgrad_, sdiff_, ssrc_, srate_;
  DevBuf<R> L0_, L1_;  // FP32 form: trailing words of U0_ / U1_ (not allocated in FP64)
  DevBuf<R> fsa_, wsa_;  // compact FP32 SA records: the SA flux column per face and wall record
  DevBuf<double> diag_part_, diag_out_, diag_cfg_, ddt_, ex_buf_;
  DevBuf<int> case_tiles_;
  std::vector<std::unique_ptr<Stager>> stagers_;  // two per admission worker; the first also serves downloads
  char* slab_ = nullptr;                           // one allocation holding every table (alloc_tables)
  char* arena_h_ = nullptr;                        // staging arena's host block, during a call
  PinnedPool::Lease arena_lease_;                  // (ensure_arena, return_arena_host)
  unsigned char* arena_d_ = nullptr;
  size_t arena_slice_ = 0;
  int arena_stages_ = 0;
  std::vector<char> reserved_;                     // slots reserved by an admission in progress
  long long pending_tiles_ = 0, pending_btiles_ = 0;
  bool block_tiles_ = true;  // cases carry block tiles (the batch may run the tiled mode)
  bool slot_fluxes_ = true;  // slots carry owner and geometry (the batch may run a per-slot mode)
};

}  // namespace amrb
