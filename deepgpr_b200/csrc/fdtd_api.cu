// fdtd_api.cu -- C-ABI entry points of libdeepgpr_b200.so.
//
// ABI 6 of the reference (src/DeepGPR/lib/deepgpr.h:41-152) is exported
// unchanged, so the reference's own ctypes bridge can load this library in
// place of deepgpr.so.  The extensions (dgb_*) add an explicit CUDA stream,
// FP64 instantiations, FP8 histories and launch options; see
// include/deepgpr_b200.h for the full list.
//
// Execution model: one call = one time loop.  All work of a call runs on a
// private stream of the calling thread that is ordered after (and before)
// the caller's stream with events.  The time loop is issued in chunks of
// `chunk` steps; a chunk is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "fdtd_3d.cuh"
#include "fdtd_3d_adj.cuh"
#include "fdtd_3d_fast.cuh"
#include "fdtd_3d_wide.cuh"
#include "fdtd_3d_wide_adj.cuh"

#define DGB_API extern "C" __attribute__((visibility("default")))

namespace {

using namespace dg;

// storage_type bits (src/DeepGPR/config/constants.py:128-187)
constexpr int ST_KIND_MASK = 0x0f;
constexpr int ST_RHS_FROM_E = 1 << 4;
constexpr int ST_PHYSICAL = 1 << 5;
constexpr int ST_TM2D = 1 << 6;
constexpr int ST_DISABLED = 1 << 26;

thread_local char g_error[512];
int g_order = 2;  // process-global like the reference (set_fdtd_order)

struct ThreadOptions {
  cudaStream_t user_stream = nullptr;  // nullptr: legacy default stream
  bool user_stream_set = false;
  int acc64 = 1;          // FP64 accumulation of the material gradient
  int chunk = 32;         // time steps per launch chunk
  int use_graph = 1;      // capture a chunk into a CUDA graph and replay it
  int order_override = 0; // per-thread FDTD order (0: use the global)
  // launch-shape choices of the autotuner (0 / -1: the built-in heuristics)
  int tm_chunks = 0;       // 2D: row chunks of the interior rectangles
  int tm_frame_rows = 0;   // 2D: rows per frame warp chunk
  int k3_xchunks = 0;      // 3D: x chunks of the z-streamed and staged kernels
  int tma = -1;            // 3D FP32 forward family: 0 z-streamed, 1 staged (TMA), 2 wide, -1 automatic
};
thread_local ThreadOptions g_opt;

// Kernel timing (dgb_profile): when enabled, time steps are launched without
// graph capture and every grid kernel is bracketed by CUDA events on the
// library stream; durations are summed per kernel kind.
enum KernelKind { KK_FWD_H = 0, KK_FWD_E, KK_ADJ_E, KK_ADJ_H, KK_IMAGE, KK_COUNT };
// Process-wide (the autograd engine runs backward on its own thread).
struct ProfileState {
  std::atomic<bool> on{false};
  std::mutex mu;
  double ms[KK_COUNT] = {0};
  long long launches[KK_COUNT] = {0};
};
ProfileState g_prof;
thread_local std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> g_pending;
std::atomic<long long> g_launch_count{0};   // time-step kernels launched by the library

// Launch `fn` (which enqueues one kernel on st, or returns how many kernels
// it enqueued, all joined back to st), timing it when profiling.
template <typename F>
void timed(int kind, cudaStream_t st, F fn) {
  auto run = [&] {
    if constexpr (std::is_void_v<decltype(fn())>) {
      fn();
      ++g_launch_count;
    } else {
      g_launch_count += fn();
    }
  };
  if (!g_prof.on) {
    run();
    return;
  }
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, st);
  run();
  cudaEventRecord(b, st);
  g_pending.push_back({kind, {a, b}});
}

void harvest_profile() {
  for (auto& p : g_pending) {
    cudaEventSynchronize(p.second.second);
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
      std::lock_guard<std::mutex> lock(g_prof.mu);
      g_prof.ms[p.first] += ms;
      g_prof.launches[p.first] += 1;
    }
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  g_pending.clear();
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
}

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return false;
}

int radius_of(int order) { return order >= 8 ? 4 : (order >= 4 ? 2 : 1); }

// Per-thread, per-device private stream and events.
struct StreamSet {
  int device = -1;
  cudaStream_t work = nullptr;
  cudaEvent_t in = nullptr, out = nullptr;
  // side stream: 2D TM frame kernels run on it beside the interior kernels
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // second side stream: the imaging kernel beside the adjoint E step
  cudaStream_t side2 = nullptr;
  cudaEvent_t fork2 = nullptr, join2 = nullptr;
};
thread_local std::vector<StreamSet> g_streams;

// Scratch retention of the default memory pool.  With the CUDA default (a
// release threshold of 0) the pool unmaps a call's freed scratch at the next
// synchronisation and the next call maps it again; on virtualised hosts those
// mappings took 90-630 ms at random points of back-to-back solves (the GPU
// idle meanwhile).  So on first use of a device the library keeps up to
// min(4 GiB, 1/32 of the device memory) cached, unless the caller has set
// the retention (dgb_set_scratch_retention).
constexpr int kMaxDevices = 64;
std::atomic<bool> g_retention_set[kMaxDevices];

void default_retention(int dev) {
  if (dev < 0 || dev >= kMaxDevices || g_retention_set[dev].exchange(true)) return;
  size_t free_b = 0, total_b = 0;
  cudaMemPool_t pool;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  unsigned long long keep = std::min<unsigned long long>(4ULL << 30, total_b / 32);
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  cudaGetLastError();
}

StreamSet* stream_set() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  for (auto& s : g_streams)
    if (s.device == dev) return &s;
  default_retention(dev);
  StreamSet s;
  s.device = dev;
  if (cudaStreamCreateWithFlags(&s.work, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.in, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.out, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  if (cudaStreamCreateWithFlags(&s.side, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.fork, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  if (cudaStreamCreateWithFlags(&s.side2, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.fork2, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  if (cudaEventCreateWithFlags(&s.join2, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  g_streams.push_back(s);
  return &g_streams.back();
}

cudaStream_t caller_stream() { return g_opt.user_stream_set ? g_opt.user_stream : cudaStreamLegacy; }

// Scratch owned by one call; released (stream-ordered) on destruction.
struct Scratch {
  cudaStream_t st;
  std::vector<void*> blocks;
  bool failed = false;
  explicit Scratch(cudaStream_t s) : st(s) {}
  template <typename P>
  P* get(size_t bytes) {
    if (bytes == 0) bytes = 16;
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess) {
      set_error("cudaMallocAsync(%zu bytes): %s", bytes, cudaGetErrorString(e));
      failed = true;
      return nullptr;
    }
    blocks.push_back(p);
    return static_cast<P*>(p);
  }
  ~Scratch() {
    for (void* p : blocks) cudaFreeAsync(p, st);
  }
};

// ---------------------------------------------------------------------------
// Static device scratch of dgb_forward_noalloc.  Some callers cannot let a
// solve allocate device memory: a serving process that has handed the free
// memory of the GPU to its own pool (an allocation would fail or force the
// pool to trim), or code that owns a fixed per-request memory budget.  For
// them the forward solve takes its scratch (control block, source / receiver
// tables and bitmaps, the pitched 2D working copy) from this file-scope array
// instead of cudaMallocAsync.  A call whose scratch does not fit is rejected
// with an error before any time step runs.  Every byte a call uses is written
// by that call before it is read (tables and bitmaps are uploaded whole, the
// control block is set by k_set, the pitched copy is written by the pack
// kernels including its zero padding), so nothing needs clearing between
// calls.  All calls on a device share the array: overlapping calls (from two
// threads, or on two streams) race.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;   // 8 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Address of the static scratch on the current device.  It is looked up on
// every call (the lookup is cheap): an address cached across calls would go
// stale if the caller reset the device or its primary context was recreated,
// and the module holding the array was loaded again elsewhere.
char* noalloc_scratch_base() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_error("dgb_forward_noalloc: cudaGetSymbolAddress of the static scratch failed: %s", cudaGetErrorString(e));
    return nullptr;
  }
  return static_cast<char*>(p);
}

// Bump allocator over the static scratch, with the interface of Scratch.
struct StaticScratch {
  cudaStream_t st;
  char* base;
  size_t used = 0;
  bool failed = false;
  explicit StaticScratch(cudaStream_t s) : st(s), base(noalloc_scratch_base()) { failed = base == nullptr; }
  template <typename P>
  P* get(size_t bytes) {
    if (failed) return nullptr;
    if (bytes == 0) bytes = 16;
    const size_t off = (used + 255) & ~size_t(255);
    if (off + bytes > kNoAllocScratchBytes) {
      set_error("dgb_forward_noalloc: this solve needs more than the %zu bytes of static device scratch "
                "(%zu requested at offset %zu); use forward for it",
                kNoAllocScratchBytes, bytes, off);
      failed = true;
      return nullptr;
    }
    used = off + bytes;
    return reinterpret_cast<P*>(base + off);
  }
};

// ---------------------------------------------------------------------------
// Source and receiver point sets of one call, built together: one
// device->host read of both location arrays and one synchronisation, the
// tables, per-shot bitmaps and per-(shot, x) row flags built on the host, and
// one host->device copy of everything.  The copy leaves from a per-thread
// pinned staging buffer (its previous upload is awaited before the buffer is
// rewritten), so no further synchronisation is needed; the no-allocation
// entry point copies from pageable memory and synchronises instead.
// ---------------------------------------------------------------------------
struct PinnedStage {
  int device = -1;
  unsigned char* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
};
thread_local std::vector<PinnedStage> g_stages;

PinnedStage* pinned_stage(size_t bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  PinnedStage* ps = nullptr;
  for (auto& x : g_stages)
    if (x.device == dev) ps = &x;
  if (!ps) {
    g_stages.push_back(PinnedStage());
    ps = &g_stages.back();
    ps->device = dev;
    if (cudaEventCreateWithFlags(&ps->done, cudaEventDisableTiming) != cudaSuccess) return nullptr;
  }
  if (ps->pending) {
    cudaEventSynchronize(ps->done);
    ps->pending = false;
  }
  if (ps->cap < bytes) {
    // grown to the next power of two (at least 1 MiB); an outgrown buffer is
    // kept, not freed: freeing pinned memory synchronises the whole device,
    // which would stall every other solve in flight
    size_t want = size_t(1) << 20;
    while (want < bytes) want <<= 1;
    unsigned char* buf = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&buf), want, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    ps->buf = buf;
    ps->cap = want;
  }
  return ps;
}

template <typename Alloc>
struct UploadsPageable : std::false_type {};
template <>
struct UploadsPageable<StaticScratch> : std::true_type {};

// One point set's host-side image: the sorted table, bitmaps and row flags
// (see PointTable / PointSet).
struct HostPointSet {
  std::vector<int> table;          // cells | off | shot | idx
  int unique = 0, n = 0;
  std::vector<unsigned> bits;      // nshot * words_per_shot
  std::vector<unsigned char> rows; // nshot * NX
  std::vector<char> any;           // NX: some shot has a point there
};

bool host_pointset(const int* h, int nshot, int npts, const Grid& g, const char* what, bool want_rows,
                   HostPointSet& out) {
  const size_t n = (size_t)nshot * npts;
  struct E {
    int cell, shot, idx;
  };
  std::vector<E> ent(n);
  for (int s = 0; s < nshot; ++s)
    for (int m = 0; m < npts; ++m) {
      const int* p = &h[((size_t)s * npts + m) * 3];
      if (p[0] < 0 || p[0] >= g.NX || p[1] < 0 || p[1] >= g.NY || p[2] < 0 || p[2] >= g.NZ) {
        set_error("%s location (%d, %d, %d) of shot %d, index %d is outside the field grid (%d, %d, %d)", what, p[0],
                  p[1], p[2], s, m, g.NX, g.NY, g.NZ);
        return false;
      }
      ent[(size_t)s * npts + m] = E{p[0] * g.sx + p[1] * g.NZ + p[2], s, m};
    }
  std::sort(ent.begin(), ent.end(), [](const E& a, const E& b) {
    if (a.cell != b.cell) return a.cell < b.cell;
    if (a.shot != b.shot) return a.shot < b.shot;
    return a.idx < b.idx;
  });
  std::vector<int> cells, off, shot(n), idx(n);
  for (size_t e = 0; e < n; ++e) {
    if (e == 0 || ent[e].cell != ent[e - 1].cell) {
      cells.push_back(ent[e].cell);
      off.push_back((int)e);
    }
    shot[e] = ent[e].shot;
    idx[e] = ent[e].idx;
  }
  off.push_back((int)n);
  out.unique = (int)cells.size();
  out.n = (int)n;
  out.table.clear();
  out.table.reserve(cells.size() + off.size() + 2 * n);
  out.table.insert(out.table.end(), cells.begin(), cells.end());
  out.table.insert(out.table.end(), off.begin(), off.end());
  out.table.insert(out.table.end(), shot.begin(), shot.end());
  out.table.insert(out.table.end(), idx.begin(), idx.end());
  const int words = (g.cells + 31) / 32;
  out.bits.assign((size_t)nshot * words, 0u);
  out.any.assign(g.NX, 0);
  if (want_rows) out.rows.assign((size_t)nshot * g.NX, 0);
  for (int s = 0; s < nshot; ++s)
    for (int m = 0; m < npts; ++m) {
      const int* p = &h[((size_t)s * npts + m) * 3];
      const int c = p[0] * g.sx + p[1] * g.NZ + p[2];
      out.bits[(size_t)s * words + (c >> 5)] |= 1u << (c & 31);
      out.any[p[0]] = 1;
      if (want_rows) out.rows[(size_t)s * g.NX + p[0]] = 1;
    }
  return true;
}

// Builds the source set (when src_loc is given) and the receiver set (when
// rcv_loc is given) of a call.  rows_*: per (shot, x index) flags on the
// device, the plane holds a point of the shot; any_*: host mask over x
// indices, some shot has a point there.
template <typename Alloc>
bool build_points(const int* src_loc, int nsrc, const int* rcv_loc, int nrcv, const Grid& g, cudaStream_t st,
                  Alloc& scratch, PointSet* sps, PointTable* stb, PointSet* rps, PointTable* rtb,
                  const unsigned char** src_rows, const unsigned char** rcv_rows, std::vector<char>* src_any,
                  std::vector<char>* rcv_any) {
  PointSet* ps[2] = {sps, rps};
  PointTable* tbo[2] = {stb, rtb};
  const int* loc[2] = {src_loc, rcv_loc};
  const int np[2] = {nsrc, nrcv};
  const unsigned char** rows_out[2] = {src_rows, rcv_rows};
  std::vector<char>* any_out[2] = {src_any, rcv_any};
  const char* what[2] = {"source", "receiver"};
  bool use[2];
  std::vector<int> h[2];
  for (int q = 0; q < 2; ++q) {
    if (rows_out[q]) *rows_out[q] = nullptr;
    if (ps[q]) {
      ps[q]->tb.n = 0;
      ps[q]->tb.cells = ps[q]->tb.off = ps[q]->tb.shot = ps[q]->tb.idx = nullptr;
      ps[q]->bits = nullptr;
      ps[q]->words_per_shot = (g.cells + 31) / 32;
    }
    if (tbo[q]) *tbo[q] = PointTable{nullptr, nullptr, nullptr, nullptr, 0};
    use[q] = ps[q] != nullptr && loc[q] != nullptr && np[q] > 0 && g.nshot > 0;
    if (use[q]) {
      h[q].resize((size_t)g.nshot * np[q] * 3);
      if (!cuda_ok(cudaMemcpyAsync(h[q].data(), loc[q], h[q].size() * sizeof(int), cudaMemcpyDefault, st), what[q]))
        return false;
    }
  }
  if (!use[0] && !use[1]) return true;
  if (!cuda_ok(cudaStreamSynchronize(st), "point locations")) return false;
  HostPointSet hs[2];
  size_t off[2][3], total = 0;
  auto reserve = [&](size_t bytes) {
    const size_t o = (total + 255) & ~size_t(255);
    total = o + bytes;
    return o;
  };
  for (int q = 0; q < 2; ++q) {
    if (!use[q]) continue;
    if (!host_pointset(h[q].data(), g.nshot, np[q], g, what[q], rows_out[q] != nullptr, hs[q])) return false;
    off[q][0] = reserve(hs[q].table.size() * sizeof(int));
    off[q][1] = reserve(hs[q].bits.size() * sizeof(unsigned));
    off[q][2] = reserve(hs[q].rows.size());
  }
  unsigned char* dev = scratch.template get<unsigned char>(total);
  if (!dev) return false;
  std::vector<unsigned char> pageable;
  PinnedStage* stage = nullptr;
  unsigned char* host = nullptr;
  if (UploadsPageable<Alloc>::value) {
    pageable.resize(total);
    host = pageable.data();
  } else {
    stage = pinned_stage(total);
    if (!stage) {
      set_error("point tables: pinned staging buffer of %zu bytes could not be allocated", total);
      return false;
    }
    host = stage->buf;
  }
  for (int q = 0; q < 2; ++q) {
    if (!use[q]) continue;
    memcpy(host + off[q][0], hs[q].table.data(), hs[q].table.size() * sizeof(int));
    memcpy(host + off[q][1], hs[q].bits.data(), hs[q].bits.size() * sizeof(unsigned));
    if (!hs[q].rows.empty()) memcpy(host + off[q][2], hs[q].rows.data(), hs[q].rows.size());
  }
  if (!cuda_ok(cudaMemcpyAsync(dev, host, total, cudaMemcpyHostToDevice, st), "point tables upload")) return false;
  if (stage) {
    cudaEventRecord(stage->done, st);
    stage->pending = true;
  } else if (!cuda_ok(cudaStreamSynchronize(st), "point tables upload")) {
    return false;
  }
  for (int q = 0; q < 2; ++q) {
    if (!use[q]) continue;
    const int U = hs[q].unique, n = hs[q].n;
    int* t = reinterpret_cast<int*>(dev + off[q][0]);
    PointTable tb{t, t + U, t + U + (U + 1), t + U + (U + 1) + n, U};
    ps[q]->tb = tb;
    ps[q]->bits = reinterpret_cast<const unsigned*>(dev + off[q][1]);
    if (tbo[q]) *tbo[q] = tb;
    if (rows_out[q]) *rows_out[q] = dev + off[q][2];
    if (any_out[q]) *any_out[q] = hs[q].any;
  }
  return true;
}

// Elements past the last plane of the 2D TM working copy (see tm_plan).
constexpr size_t kTmTailPad = 4 * TMW + 64;

// Strip layout of the 2D TM path: padded pitch and 32-column strips; the
// rectangles and row chunking of each launch are set by tm_plan.
TmGeom tm_layout(const Grid& g) {
  TmGeom tg;
  memset(&tg, 0, sizeof(tg));
  tg.NYP = (g.NY + TMW - 1) / TMW * TMW;
  tg.nseg = tg.NYP / TMW;
  return tg;
}

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

template <typename K>
int blocks_per_sm(K kernel) {
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, 32 * TM_WARPS, 0) != cudaSuccess || blocks < 1) {
    cudaGetLastError();
    blocks = 4;
  }
  return blocks;
}

// Appends rectangle (warp strips of `width` columns starting at column
// 32 * seg0, nseg of them; rows [row0, row1)) with chunks of xc rows.
void tm_add_rect(TmGeom& tg, int nshot, int seg0, int nseg, int width, int row0, int row1, int xc,
                 int kind = kFrameGeneral) {
  if (nseg <= 0 || row1 <= row0 || tg.nrect >= kTmMaxRects) return;
  TmRect& r = tg.rect[tg.nrect++];
  r.kind = kind;
  r.seg0 = seg0;
  r.nseg = nseg;
  r.width = width;
  r.row0 = row0;
  r.row1 = row1;
  r.xc = std::max(1, std::min(xc, row1 - row0));
  r.nchunk = (row1 - row0 + r.xc - 1) / r.xc;
  r.warp0 = tg.nwarps;
  tg.nwarps += (long long)nseg * r.nchunk * nshot;
}

// Interior rectangle of one 2D TM half step and the frame of general work
// around it.  Interior rows: runs where tm_lean_ok holds along x and no shot
// has a source or receiver (at most 4, the longest); interior columns: the
// longest run of whole 32-column tiles where tm_lean_ok holds along y (so each
// FP8 scale tile is written by one kernel).  The interior kernels use
// 128-column strips from the first interior column (tiles past the interior
// are masked), chunked so a launch is about one wave of resident warps
// (occupancy `iblocks` CTAs per SM, chunks of at least 16 rows).  The frame
// is split by kind (see kFrameGeneral): edge tiles on x-lean rows, edge tiles
// elsewhere (corners, chunks of 2 rows), and interior tiles on the remaining
// rows (chunks of 16 rows), all in one launch.
struct TmPlan {
  TmGeom interior, frame;
};

TmPlan tm_plan(const TmGeom& base, const Grid& g, int kind, int R, const TmFaces& f, bool lean, int iblocks,
               const std::vector<char>* avoid = nullptr) {
  TmPlan pl;
  pl.interior = base;
  pl.frame = base;
  // the interior kernels index a shot plane with 32-bit offsets
  if ((long long)g.NX * base.NYP + (long long)kTmTailPad >= (1LL << 31)) lean = false;
  auto runs_of = [](int n, auto ok) {
    std::vector<std::pair<int, int>> r;
    int cur = -1;
    for (int c = 0; c <= n; ++c) {
      const bool y = c < n && ok(c);
      if (y && cur < 0) cur = c;
      if (!y && cur >= 0) {
        r.push_back({cur, c});
        cur = -1;
      }
    }
    return r;
  };
  auto complement = [](int n, const std::vector<std::pair<int, int>>& in) {
    std::vector<std::pair<int, int>> r;
    int prev = 0;
    for (auto& q : in) {
      if (q.first > prev) r.push_back({prev, q.first});
      prev = q.second;
    }
    if (n > prev) r.push_back({prev, n});
    return r;
  };
  std::vector<std::pair<int, int>> xl, rows;
  int tlo = 0, thi = 0;
  if (lean) {
    xl = runs_of(g.NX, [&](int i) { return tm_lean_ok(kind, 0, i, g.NX, R, f); });
    rows = runs_of(g.NX, [&](int i) {
      return tm_lean_ok(kind, 0, i, g.NX, R, f) && !(avoid && !avoid->empty() && (*avoid)[i]);
    });
    if (rows.size() > 4) {
      std::sort(rows.begin(), rows.end(), [](const std::pair<int, int>& x, const std::pair<int, int>& y) {
        return x.second - x.first > y.second - y.first;
      });
      rows.resize(4);
      std::sort(rows.begin(), rows.end());
    }
    const auto tiles = runs_of(base.nseg, [&](int q) {
      for (int j = q * TMW; j < (q + 1) * TMW; ++j)
        if (!tm_lean_ok(kind, 1, j, g.NY, R, f)) return false;
      return true;
    });
    for (auto& t : tiles)
      if (t.second - t.first > thi - tlo) {
        tlo = t.first;
        thi = t.second;
      }
  }
  const auto xg = complement(g.NX, xl);
  const auto mid = complement(g.NX, rows);
  const bool fits = 2 * xl.size() + 2 * xg.size() + mid.size() <= (size_t)kTmMaxRects;
  const int frame_xc = g_opt.tm_frame_rows > 0 ? g_opt.tm_frame_rows : 16, corner_xc = 2;
  if (!rows.empty() && thi > tlo && fits) {
    const int n128 = (thi - tlo + 3) / 4;
    int nrows = 0;
    for (auto& r : rows) nrows += r.second - r.first;
    const long long per = (long long)n128 * g.nshot;
    const long long resident = (long long)sm_count() * iblocks * TM_WARPS;
    long long chunks = std::max<long long>(1, resident / per);
    chunks = std::min<long long>(chunks, std::max(1, nrows / 16));
    if (g_opt.tm_chunks > 0) chunks = std::min(g_opt.tm_chunks, std::max(1, nrows));
    const int xc = (int)((nrows + chunks - 1) / chunks);
    for (auto& r : rows) tm_add_rect(pl.interior, g.nshot, tlo, n128, 4 * TMW, r.first, r.second, xc);
    pl.interior.col1 = thi * TMW;
    for (auto& r : xl) {
      tm_add_rect(pl.frame, g.nshot, 0, tlo, TMW, r.first, r.second, frame_xc, kFrameXLean);
      tm_add_rect(pl.frame, g.nshot, thi, base.nseg - thi, TMW, r.first, r.second, frame_xc, kFrameXLean);
    }
    for (auto& r : xg) {
      tm_add_rect(pl.frame, g.nshot, 0, tlo, TMW, r.first, r.second, corner_xc, kFrameGeneral);
      tm_add_rect(pl.frame, g.nshot, thi, base.nseg - thi, TMW, r.first, r.second, corner_xc, kFrameGeneral);
    }
    for (auto& r : mid) tm_add_rect(pl.frame, g.nshot, tlo, thi - tlo, TMW, r.first, r.second, frame_xc, kFrameYLean);
  } else {
    tm_add_rect(pl.frame, g.nshot, 0, base.nseg, TMW, 0, g.NX, frame_xc, kFrameGeneral);
  }
  return pl;
}

// 2D imaging kernel for the call's history format.
template <typename T, int KIND>
void launch_tm_image_k(bool e_only, bool acc64, cudaStream_t st, const AdjArgs<T>& a, const T* lam, const TmGeom& tg) {
  const unsigned blocks = (unsigned)((a.box.cells() + kImageThreads - 1) / kImageThreads);
  constexpr int B = kImageThreads;
  if (e_only) {
    if (acc64) tm_image<T, KIND, true, true><<<blocks, B, 0, st>>>(a, lam, tg.NYP, tg.nseg);
    else tm_image<T, KIND, true, false><<<blocks, B, 0, st>>>(a, lam, tg.NYP, tg.nseg);
  } else {
    if (acc64) tm_image<T, KIND, false, true><<<blocks, B, 0, st>>>(a, lam, tg.NYP, tg.nseg);
    else tm_image<T, KIND, false, false><<<blocks, B, 0, st>>>(a, lam, tg.NYP, tg.nseg);
  }
}

template <typename T>
void launch_tm_image(int kind, bool e_only, bool acc64, cudaStream_t st, const AdjArgs<T>& a, const T* lam,
                     const TmGeom& tg) {
  if constexpr (sizeof(T) == 8) {
    launch_tm_image_k<T, kF64>(e_only, acc64, st, a, lam, tg);
  } else {
    if (kind == kF16) launch_tm_image_k<T, kF16>(e_only, acc64, st, a, lam, tg);
    else if (kind == kBF16) launch_tm_image_k<T, kBF16>(e_only, acc64, st, a, lam, tg);
    else if (kind == kFP8) launch_tm_image_k<T, kFP8>(e_only, acc64, st, a, lam, tg);
    else if (kind == kI8) launch_tm_image_k<T, kI8>(e_only, acc64, st, a, lam, tg);
    else launch_tm_image_k<T, kF32>(e_only, acc64, st, a, lam, tg);
  }
}

template <typename T, int KIND, int NC>
void launch_k3_image_k(bool e_only, bool acc64, cudaStream_t st, const AdjArgs<T>& a, const K3Buf<T>& kb,
                       long long ls, int lp, int lr) {
  const unsigned blocks = (unsigned)((a.box.cells() + kImage3Threads - 1) / kImage3Threads);
  constexpr int B = kImage3Threads;
  if (e_only) {
    if (acc64) k3_image<T, KIND, true, true, NC><<<blocks, B, 0, st>>>(a, kb.Ex, kb.Ey, kb.Ez, ls, lp, lr);
    else k3_image<T, KIND, true, false, NC><<<blocks, B, 0, st>>>(a, kb.Ex, kb.Ey, kb.Ez, ls, lp, lr);
  } else {
    if (acc64) k3_image<T, KIND, false, true, NC><<<blocks, B, 0, st>>>(a, kb.Ex, kb.Ey, kb.Ez, ls, lp, lr);
    else k3_image<T, KIND, false, false, NC><<<blocks, B, 0, st>>>(a, kb.Ex, kb.Ey, kb.Ez, ls, lp, lr);
  }
}

// Imaging condition of a 3D solve on the pitched lambda_E of kb.
template <typename T>
void launch_k3_image(int kind, bool e_only, bool acc64, int mode, cudaStream_t st, const AdjArgs<T>& a,
                     const K3Buf<T>& kb, long long ls, int lp, int lr) {
  auto by_nc = [&](auto K) {
    constexpr int KD = decltype(K)::value;
    if (mode == 3) launch_k3_image_k<T, KD, 3>(e_only, acc64, st, a, kb, ls, lp, lr);
    else launch_k3_image_k<T, KD, 1>(e_only, acc64, st, a, kb, ls, lp, lr);
  };
  if constexpr (sizeof(T) == 8) {
    by_nc(std::integral_constant<int, kF64>());
  } else {
    if (kind == kF16) by_nc(std::integral_constant<int, kF16>());
    else if (kind == kBF16) by_nc(std::integral_constant<int, kBF16>());
    else if (kind == kFP8) by_nc(std::integral_constant<int, kFP8>());
    else if (kind == kI8) by_nc(std::integral_constant<int, kI8>());
    else by_nc(std::integral_constant<int, kF32>());
  }
}

// One 2D TM half step: the frame kernel on the side stream, forked from and
// joined back to st, beside the interior kernel on st.  Returns the number
// of kernels launched.
template <typename FrameFn, typename InteriorFn>
int split_launch(cudaStream_t st, const StreamSet* ss, const TmPlan& pl, FrameFn frame, InteriorFn interior) {
  const bool has_interior = pl.interior.nwarps > 0;
  if (!has_interior || ss == nullptr || ss->side == nullptr) {
    frame(st, pl.frame);
    if (has_interior) interior(st);
    return has_interior ? 2 : 1;
  }
  cudaEventRecord(ss->fork, st);
  cudaStreamWaitEvent(ss->side, ss->fork, 0);
  frame(ss->side, pl.frame);
  cudaEventRecord(ss->join, ss->side);
  interior(st);
  cudaStreamWaitEvent(st, ss->join, 0);
  return 2;
}

dim3 tm_grid(const TmGeom& tg) { return dim3((unsigned)std::max<long long>(1, (tg.nwarps + TM_WARPS - 1) / TM_WARPS)); }

bool env_flag(const char* name);

// A 2D half step: the frame and interior kernels as two launches on two
// streams, or fused into one launch (fused(grid, frame CTAs)) when
// DEEPGPR_B200_TM_FUSED=1 (measured 0-10 % slower per half step on the
// 400 x 800 x 32-shot grid).  Returns the number of kernels launched.
template <typename FusedFn, typename FrameFn, typename InteriorFn>
int tm_launch(cudaStream_t st, const StreamSet* ss, const TmPlan& pl, FusedFn fused, FrameFn frame,
              InteriorFn interior) {
  static const bool fuse = env_flag("DEEPGPR_B200_TM_FUSED");
  if (pl.interior.nwarps > 0 && fuse) {
    const unsigned nfb = (unsigned)((pl.frame.nwarps + TM_WARPS - 1) / TM_WARPS);
    const unsigned nib = (unsigned)((pl.interior.nwarps + TM_WARPS - 1) / TM_WARPS);
    fused(dim3(nfb + nib), nfb);
    return 1;
  }
  return split_launch(st, ss, pl, frame, interior);
}

// 3D working copy: z pitch, strips, y tiles and x chunks.  The chunking keeps
// the last wave of CTAs nearly full (occupancy of the forward H kernel).
// Calls f(R, EQ, GEN) with compile-time constants (std::integral_constant)
// for the runtime stencil radius, "dy == dz == dx" and "CPML faces of an axis
// may meet".  Double precision (the FP64 runs) is built for the general form
// only: per-axis curl scales and per-face CPML.
template <typename T, typename F>
void k3_variant(int R, bool eq, bool gen, F&& f) {
  auto by_r = [&](auto E, auto G) {
    if (R == 1) f(std::integral_constant<int, 1>(), E, G);
    else if (R == 2) f(std::integral_constant<int, 2>(), E, G);
    else f(std::integral_constant<int, 4>(), E, G);
  };
  if constexpr (sizeof(T) == 8) {
    by_r(std::false_type(), std::true_type());
  } else {
    if (gen) {
      if (eq) by_r(std::true_type(), std::true_type());
      else by_r(std::false_type(), std::true_type());
    } else {
      if (eq) by_r(std::true_type(), std::false_type());
      else by_r(std::false_type(), std::false_type());
    }
  }
}

// Calls f(R, EQ, CPM) for the forward kernels (CPM: kCpmSingle, kCpmGeneral
// or kCpmPass).  Double precision: per-axis curl scales, general CPML form.
template <typename T, typename F>
void k3_fwd_variant(int R, bool eq, int cpm, F&& f) {
  auto by_r = [&](auto E, auto C) {
    if (R == 1) f(std::integral_constant<int, 1>(), E, C);
    else if (R == 2) f(std::integral_constant<int, 2>(), E, C);
    else f(std::integral_constant<int, 4>(), E, C);
  };
  auto by_cpm = [&](auto E) {
    if (cpm == kCpmPass) by_r(E, std::integral_constant<int, kCpmPass>());
    else if (cpm == kCpmGeneral) by_r(E, std::integral_constant<int, kCpmGeneral>());
    else by_r(E, std::integral_constant<int, kCpmSingle>());
  };
  if constexpr (sizeof(T) == 8) {
    by_r(std::false_type(), std::integral_constant<int, kCpmGeneral>());
  } else {
    if (eq) by_cpm(std::true_type());
    else by_cpm(std::false_type());
  }
}

// CPML frame of the forward pass form: along each axis the cells 0 .. p_lo
// (the low face's CPML cells of E and H) and n-1-p_hi .. n-1, as six disjoint
// boxes (x slabs whole, y slabs within x's interior, z slabs within both).
K3Frame k3_frame(const Grid& g, const int* p) {
  K3Frame fr;
  memset(&fr, 0, sizeof(fr));
  const int n[3] = {g.NX, g.NY, g.NZ};
  for (int ax = 0; ax < 3; ++ax) {
    fr.lo[ax] = std::min(n[ax], p[2 * ax] + 1);
    fr.hi[ax] = std::max(fr.lo[ax], n[ax] - 1 - p[2 * ax + 1]);
  }
  const int x0 = fr.lo[0], x1 = fr.hi[0], y0 = fr.lo[1], y1 = fr.hi[1], z0 = fr.lo[2], z1 = fr.hi[2];
  const int box[6][6] = {
      {0, x0, 0, g.NY, 0, g.NZ},         {x1, g.NX - x1, 0, g.NY, 0, g.NZ},          // x low, x high
      {x0, x1 - x0, 0, y0, 0, g.NZ},     {x0, x1 - x0, y1, g.NY - y1, 0, g.NZ},      // y low, y high
      {x0, x1 - x0, y0, y1 - y0, 0, z0}, {x0, x1 - x0, y0, y1 - y0, z1, g.NZ - z1}};  // z low, z high
  unsigned cum = 0;
  for (int b = 0; b < 6; ++b) {
    for (int ax = 0; ax < 3; ++ax) {
      fr.o[b][ax] = box[b][2 * ax];
      fr.n[b][ax] = std::max(1, box[b][2 * ax + 1]);   // extents of empty boxes stay divisors
    }
    cum += (unsigned)((long long)std::max(0, box[b][1]) * std::max(0, box[b][3]) * std::max(0, box[b][5]));
    fr.cum[b] = cum;
  }
  return fr;
}

template <bool EFIELD>
void psi_counts(const Grid& g, const int* p, long long* out);

// Face slabs of k3p_adj_w for E (efield) or H: along the face axis the CPML
// cells of the face (H: 0 .. p-1 and n-1-p .. n-2; E: 1 .. p and
// n-1-p .. n-2), the other two axes whole.
K3Faces k3_faces(const Grid& g, const int* p, bool efield) {
  K3Faces fs;
  memset(&fs, 0, sizeof(fs));
  const int n[3] = {g.NX, g.NY, g.NZ};
  unsigned cum = 0;
  for (int b = 0; b < 6; ++b) {
    const int ax = b >> 1, pf = p[b];
    const int lo = (b & 1) ? n[ax] - 1 - pf : (efield ? 1 : 0);
    const int cnt = pf > 0 ? pf : 0;
    for (int d = 0; d < 3; ++d) {
      fs.o[b][d] = d == ax ? lo : 0;
      fs.n[b][d] = d == ax ? std::max(1, cnt) : n[d];
    }
    cum += (unsigned)((long long)cnt * n[(ax + 1) % 3] * n[(ax + 2) % 3]);
    fs.cum[b] = cum;
  }
  return fs;
}

// The 3D kernels' single-face CPML form: along every axis the two faces are
// at least 4 cells apart (a lane's two cells, a row and a plane lie in one
// face at most) and every CPML array is indexed in 32 bits.
bool k3_cpml_single(const Grid& g, const int* p) {
  if (g.NX < p[0] + p[1] + 4 || g.NY < p[2] + p[3] + 4 || g.NZ < p[4] + p[5] + 4) return false;
  long long ce[12], ch[12];
  psi_counts<true>(g, p, ce);
  psi_counts<false>(g, p, ch);
  for (int q = 0; q < 12; ++q)
    if (ce[q] >= (1LL << 31) || ch[q] >= (1LL << 31)) return false;
  return true;
}

// min_chunks: the fewest x chunks to use (capped at chunks of 16 planes).
// Measured on 320 x 320 x 160, 200^3 and 160^3 + CPML 10 (4 shots): the
// z-streamed adjoint steps are fastest at about 8 chunks (4-6 % faster than
// the wave-fill choice below, which assumes the forward kernels' residency),
// the z-streamed H step at about 12 (5-8 % faster).
K3Geom k3_layout(const Grid& g, int min_chunks) {
  K3Geom kg;
  memset(&kg, 0, sizeof(kg));
  kg.zp = (g.NZ + 31) / 32 * 32;
  kg.nzs = (g.NZ + K3W - 1) / K3W;
  kg.nyt = (g.NY + K3_WARPS - 1) / K3_WARPS;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k3v_fwd_h<float, 2, true, kCpmSingle>, 32 * K3_WARPS, 0) !=
          cudaSuccess ||
      blocks < 1) {
    cudaGetLastError();
    blocks = 4;
  }
  const double resident = (double)sm_count() * blocks;
  const long long per = (long long)g.nshot * kg.nzs * kg.nyt;
  int best = 1;
  double best_eff = -1.0;
  for (int n = 1; n <= std::max(1, std::min(64, g.NX / 16)); ++n) {
    const int xc = (g.NX + n - 1) / n;
    const int nch = (g.NX + xc - 1) / xc;
    const double nb = (double)per * nch;
    const double waves = std::ceil(nb / resident);
    const double eff = nb / (waves * resident) * (double)xc / (xc + 3.0);
    if (eff > best_eff + 1e-3) {
      best_eff = eff;
      best = n;
    }
  }
  best = std::max(best, std::min(min_chunks, std::max(1, g.NX / 16)));
  if (g_opt.k3_xchunks > 0) best = std::min(g_opt.k3_xchunks, g.NX);
  kg.xc = (g.NX + best - 1) / best;
  kg.nchunk = (g.NX + kg.xc - 1) / kg.xc;
  kg.nblocks = per * kg.nchunk;
  return kg;
}

// Allocates the 3D working copy and packs the fields and coefficients into it.
template <typename T, typename Alloc, typename CM>
bool k3_alloc_pack(Alloc& scratch, const Grid& g, const K3Geom& kg, const CM& cm, cudaStream_t st, K3Buf<T>& kf,
                   const T* Ex, const T* Ey, const T* Ez, const T* Hx, const T* Hy, const T* Hz) {
  const long long rows = (long long)g.NX * g.NY;
  const long long plane = rows * kg.zp;
  T* buf = scratch.template get<T>(((size_t)(6 * g.nshot + 5) * plane + 64) * sizeof(T));
  if (!buf) return false;
  T* fields[6];
  const T* srcs[6] = {Ex, Ey, Ez, Hx, Hy, Hz};
  for (int q = 0; q < 6; ++q) {
    fields[q] = buf + (long long)q * g.nshot * plane;
    k_pack_rows<T><<<2048, 256, 0, st>>>(srcs[q], fields[q], rows * g.nshot, g.NZ, kg.zp);
  }
  kf.Ex = fields[0]; kf.Ey = fields[1]; kf.Ez = fields[2];
  kf.Hx = fields[3]; kf.Hy = fields[4]; kf.Hz = fields[5];
  T* cf = buf + 6LL * g.nshot * plane;
  const T* coef[5] = {cm.ce_hist, cm.ce_curl, cm.ce_rhs, cm.ch_curl, cm.ch_rhs};
  for (int q = 0; q < 5; ++q) k_pack_rows<T><<<1024, 256, 0, st>>>(coef[q], cf + q * plane, rows, g.NZ, kg.zp);
  kf.ce_hist = cf;
  kf.ce_curl = cf + plane;
  kf.ce_rhs = cf + 2 * plane;
  kf.ch_curl = cf + 3 * plane;
  kf.ch_rhs = cf + 4 * plane;
  cudaMemsetAsync(cf + 5 * plane, 0, 64 * sizeof(T), st);
  return cuda_ok(cudaGetLastError(), "3D pack");
}

template <typename T>
bool k3_unpack(const Grid& g, const K3Geom& kg, cudaStream_t st, const K3Buf<T>& kf, T* Ex, T* Ey, T* Ez, T* Hx,
               T* Hy, T* Hz) {
  const long long rows = (long long)g.NX * g.NY * g.nshot;
  const T* srcs[6] = {kf.Ex, kf.Ey, kf.Ez, kf.Hx, kf.Hy, kf.Hz};
  T* dsts[6] = {Ex, Ey, Ez, Hx, Hy, Hz};
  for (int q = 0; q < 6; ++q) k_unpack_rows<T><<<2048, 256, 0, st>>>(srcs[q], dsts[q], rows, g.NZ, kg.zp);
  return cuda_ok(cudaGetLastError(), "3D unpack");
}

template <typename T>
TmFaces tm_faces(const Face<T>* eF, const Face<T>* hF, bool cpml) {
  TmFaces f;
  memset(&f, 0, sizeof(f));
  if (cpml) {
    f.hx0 = hF[0].p; f.hx1 = hF[1].p; f.hy0 = hF[2].p; f.hy1 = hF[3].p;
    f.ex0 = eF[0].p; f.ex1 = eF[1].p; f.ey0 = eF[2].p; f.ey1 = eF[3].p;
  }
  return f;
}


// x-chunk length that gives about 8 resident CTAs per SM.
int pick_xchunk(int NX, long long tiles_per_plane, int nshot, int min_chunk) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long target = (long long)sms * 8;
  const long long per = std::max<long long>(1, tiles_per_plane * nshot);
  long long chunks = (target + per - 1) / per;
  chunks = std::max<long long>(1, std::min<long long>(chunks, 65535));
  int xc = (int)((NX + chunks - 1) / chunks);
  xc = std::max(xc, std::min(min_chunk, NX));
  return xc;
}

long long tiles3(const Grid& g) { return (long long)((g.NY + TY - 1) / TY) * ((g.NZ + TZ - 1) / TZ); }

template <typename T>
__global__ void k_coeffs(const T* __restrict__ eps, const T* __restrict__ sig, const T* __restrict__ mu,
                         T* ce_hist, T* ce_curl, T* ce_rhs, T* ch_hist, T* ch_curl, T* ch_rhs, Grid g, T dt,
                         T dx) {
  // src/DeepGPR/lib/deepgpr_cpu.c:547-584; halo cells are set to zero.
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.cells) return;
  int i, j, k;
  cell_ijk(g, c, i, j, k);
  if (i >= g.NX - 1 || j >= g.NY - 1 || k >= g.NZ - 1) {
    ce_hist[c] = ce_curl[c] = ce_rhs[c] = ch_hist[c] = ch_curl[c] = ch_rhs[c] = T(0);
    return;
  }
  const T m0 = sizeof(T) == 4 ? T(1.25663706212e-06f) : T(1.25663706212e-06);
  const T e0 = Phys<T>::eps0();
  const T ha = m0 * mu[c] / dt;
  ch_hist[c] = T(1);
  ch_curl[c] = (T(1) / dx) / ha;
  ch_rhs[c] = T(1) / ha;
  if (sig[c] > Phys<T>::pec()) {
    ce_hist[c] = ce_curl[c] = ce_rhs[c] = T(0);
  } else {
    const T e = e0 * eps[c] / dt;
    const T s = T(0.5) * sig[c];
    const T a = e + s, b = e - s;
    ce_hist[c] = b / a;
    ce_curl[c] = (T(1) / dx) / a;
    ce_rhs[c] = T(1) / a;
  }
}

__global__ void k_advance(Control* ctrl, int delta) { ctrl->cur += delta; }

__global__ void k_set(Control* ctrl, int cur) {
  ctrl->cur = cur;
  ctrl->error = 0;
}

HBox make_box(const Grid& g, bool physical, const int* p) {
  HBox b;
  if (physical) {
    b.x0 = p[0];
    b.y0 = p[2];
    b.z0 = p[4];
    b.nx = g.NX - 1 - p[0] - p[1];
    b.ny = g.NY - 1 - p[2] - p[3];
    b.nz = g.NZ - 1 - p[4] - p[5];
  } else {
    b.x0 = b.y0 = b.z0 = 0;
    b.nx = g.NX - 1;
    b.ny = g.NY - 1;
    b.nz = g.NZ - 1;
  }
  return b;
}

// FP8 scale tiles: one per (x plane, y row, 32 z columns) in 3D, one per
// (row, 32-column strip) in 2D TM.
long long fp8_tiles(const Grid& g, bool tm2d) {
  return (long long)g.NX * (tm2d ? (long long)(g.NY + TMW - 1) / TMW : (long long)g.NY * ((g.NZ + 31) / 32));
}

// FP8 history buffer: payload (1 byte per value) padded to 256 bytes, then
// one float scale per (comp, slot, shot, tile).
long long fp8_payload_bytes(long long values) { return (values + 255) / 256 * 256; }

template <typename T>
struct Common {
  Grid g;
  T dx, dy, dz, dt;
  int nt, p[6];
  const T *eps, *sig, *mu;
  T *ce_hist, *ce_curl, *ce_rhs, *ch_hist, *ch_curl, *ch_rhs;
  const T* eR[6];
  const T* hR[6];
  T* ePsi[12];
  T* hPsi[12];
  int S, mode, storage_type;
};

template <typename T>
void fill_faces(Face<T>* F, const int* p, const T* const* R, T* const* psi) {
  for (int f = 0; f < 6; ++f) {
    F[f].R = R[f];
    F[f].psi1 = psi[2 * f];
    F[f].psi2 = psi[2 * f + 1];
    F[f].w1 = F[f].w2 = nullptr;
    F[f].p = p[f];
  }
}

template <typename T>
bool launch_coeffs(const Common<T>& cm, cudaStream_t st) {
  const int blocks = (cm.g.cells + 255) / 256;
  k_coeffs<T><<<blocks, 256, 0, st>>>(cm.eps, cm.sig, cm.mu, cm.ce_hist, cm.ce_curl, cm.ce_rhs, cm.ch_hist,
                                      cm.ch_curl, cm.ch_rhs, cm.g, cm.dt, cm.dx);
  return cuda_ok(cudaGetLastError(), "coefficient kernel");
}

// Instantiated time-loop graphs kept across calls, per thread, device and
// direction: a call captures its chunk and updates the kept executable in
// place (cudaGraphExecUpdate) when the captured topology is the same, which
// spares the instantiation; otherwise it instantiates anew.
struct GraphCache {
  int device, dir;
  cudaGraphExec_t exec;
};
thread_local std::vector<GraphCache> g_graphs;

cudaGraphExec_t* cached_exec(int dir) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  for (auto& c : g_graphs)
    if (c.device == dev && c.dir == dir) return &c.exec;
  g_graphs.push_back(GraphCache{dev, dir, nullptr});
  return &g_graphs.back().exec;
}

struct NoHook {
  bool operator()(int, int, int) const { return true; }
};

// Issue `steps` time steps through `issue(k)` in chunks, with graph replay.
// hook(t, K, phase) runs before (phase 0) and after (phase 1) the chunk of
// steps t .. t+K-1 is issued (host-side staging around chunks).
template <typename Issue, typename Hook = NoHook>
bool run_loop(int steps, int dir, Control* ctrl, cudaStream_t st, Issue issue, Hook hook = Hook()) {
  const int chunk = std::max(1, g_opt.chunk);
  cudaGraphExec_t exec = nullptr;
  bool owned = false;   // exec is not the kept one: destroy it at the end
  long long per_replay = 0;
  bool ok = true;
  int t = 0;
  while (ok && t < steps) {
    const int K = std::min(chunk, steps - t);
    if (!hook(t, K, 0)) return false;
    if (g_opt.use_graph && !g_prof.on && K == chunk && steps >= 2 * chunk) {
      if (!exec) {
        cudaGraph_t graph = nullptr;
        ok = cuda_ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (!ok) break;
        const long long before = g_launch_count.load();
        for (int k = 0; k < K; ++k) issue(k);
        k_advance<<<1, 1, 0, st>>>(ctrl, dir * K);
        per_replay = g_launch_count.load() - before + 1;
        g_launch_count -= per_replay - 1;   // captured, not yet launched
        cudaError_t e1 = cudaGetLastError();
        cudaError_t e2 = cudaStreamEndCapture(st, &graph);
        ok = cuda_ok(e1, "capture launch") && cuda_ok(e2, "end capture");
        if (!ok) break;
        cudaGraphExec_t* kept = cached_exec(dir);
        if (kept && *kept) {
          cudaGraphExecUpdateResultInfo info;
          if (cudaGraphExecUpdate(*kept, graph, &info) == cudaSuccess) {
            exec = *kept;
          } else {
            cudaGetLastError();
            cudaGraphExecDestroy(*kept);
            *kept = nullptr;
          }
        }
        if (!exec) {
          ok = cuda_ok(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
          if (ok && kept) *kept = exec;
          else owned = ok;
        }
        cudaGraphDestroy(graph);
        if (!ok) break;
      }
      ok = cuda_ok(cudaGraphLaunch(exec, st), "graph launch");
      g_launch_count += per_replay;
    } else {
      for (int k = 0; k < K; ++k) issue(k);
      k_advance<<<1, 1, 0, st>>>(ctrl, dir * K);
      ++g_launch_count;
      ok = cuda_ok(cudaGetLastError(), "time-step launch");
      if (g_prof.on) harvest_profile();
    }
    if (ok && !hook(t, K, 1)) ok = false;
    t += K;
  }
  if (exec && owned) cudaGraphExecDestroy(exec);
  return ok;
}

// ---------------------------------------------------------------------------
// Asynchronous history offload (use_async_offload): a history that lives in
// pinned host memory is written and read by the kernels through a pair of
// device ring buffers.  Every kernel indexes a history as
//   base + q * comp_stride + slot * frame + (cell offset),
// so a chunk of time steps touching the saved slots s0 .. s1-1 is pointed at
// ring buffer b with base = ring[b] - s0 * frame and comp_stride =
// ring_slots * frame; no kernel knows about the ring.  A copy stream moves
// each chunk's slots between the ring and the host while the next chunk
// computes: forward, the copy of chunk c runs beside chunk c+1 and buffer b
// is rewritten by chunk c+2 only after its copy ended; backward, the slots of
// chunk c+1 (and c+2) are staged ahead of their use.
// ---------------------------------------------------------------------------
bool is_host_memory(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

struct HistRing {
  bool on = false;
  int S = 1, nt = 0, nt_saved = 0, ncomp = 1, slots = 0, extra = 0;
  size_t frame_bytes = 0;       // one saved step of one component, all shots
  long long frame_elems = 0;
  char* host[2] = {nullptr, nullptr};   // E, R host histories (R: nullptr when not offloaded)
  char* ring[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [history][buffer]
  cudaStream_t copy = nullptr;
  cudaEvent_t done[2] = {nullptr, nullptr}, work[2] = {nullptr, nullptr};
  bool pending[2] = {false, false};

  // slots of forward chunk [t, t+K) and of reverse chunk (steps nt-1-t down to nt-t-K)
  void fwd_slots(int t, int K, int& s0, int& s1) const {
    s0 = (t + S - 1) / S;
    s1 = (t + K + S - 1) / S;
  }
  void bwd_slots(int t, int K, int& s0, int& s1) const {
    const int lo = std::max(0, nt - t - K), hi = nt - 1 - t;
    s0 = (lo + S - 1) / S;
    s1 = std::min(nt_saved, hi / S + 1 + extra);
  }
  template <typename Alloc>
  bool setup(Alloc& scratch, cudaStream_t st, void* e_host, void* r_host, int S_, int nt_, int nt_saved_, int ncomp_,
             long long frame, int elem, int chunk, int extra_) {
    S = S_;
    nt = nt_;
    nt_saved = nt_saved_;
    ncomp = ncomp_;
    extra = extra_;
    frame_elems = frame;
    frame_bytes = (size_t)frame * elem;
    slots = (chunk + S - 1) / S + 1 + extra;
    host[0] = static_cast<char*>(e_host);
    host[1] = static_cast<char*>(r_host);
    for (int h = 0; h < 2; ++h) {
      if (!host[h]) continue;
      for (int b = 0; b < 2; ++b) {
        ring[h][b] = scratch.template get<char>((size_t)ncomp * slots * frame_bytes);
        if (!ring[h][b]) return false;
      }
    }
    if (!cuda_ok(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking), "offload copy stream")) return false;
    for (int b = 0; b < 2; ++b)
      if (!cuda_ok(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "offload event") ||
          !cuda_ok(cudaEventCreateWithFlags(&work[b], cudaEventDisableTiming), "offload event"))
        return false;
    on = true;
    (void)st;
    return true;
  }
  // device base of history h for a chunk whose first slot is s0 in buffer b
  void* base(int h, int b, int s0) const { return ring[h][b] - (long long)s0 * (long long)frame_bytes; }
  long long comp_stride() const { return (long long)slots * frame_elems; }
  // copies slots s0 .. s1-1 of buffer b to (dir > 0) or from (dir < 0) the host, on the copy stream
  bool move(int b, int s0, int s1, bool to_host) {
    if (s1 <= s0) return true;
    for (int h = 0; h < 2; ++h) {
      if (!host[h]) continue;
      for (int q = 0; q < ncomp; ++q) {
        char* hp = host[h] + ((long long)q * nt_saved + s0) * (long long)frame_bytes;
        char* dp = ring[h][b] + (long long)q * slots * (long long)frame_bytes;
        const size_t n = (size_t)(s1 - s0) * frame_bytes;
        const cudaError_t e = to_host ? cudaMemcpyAsync(hp, dp, n, cudaMemcpyDeviceToHost, copy)
                                      : cudaMemcpyAsync(dp, hp, n, cudaMemcpyHostToDevice, copy);
        if (!cuda_ok(e, "history offload copy")) return false;
      }
    }
    return true;
  }
  void release() {
    if (copy) cudaStreamSynchronize(copy);
    for (int b = 0; b < 2; ++b) {
      if (done[b]) cudaEventDestroy(done[b]);
      if (work[b]) cudaEventDestroy(work[b]);
    }
    if (copy) cudaStreamDestroy(copy);
    copy = nullptr;
  }
  ~HistRing() { release(); }
};

// ---------------------------------------------------------------------------
// TMA-staged 3D forward kernels (fdtd_3d_fast.cuh): launch geometry, tensor
// maps and launches.
// ---------------------------------------------------------------------------
bool env_flag(const char* name) {
  const char* v = getenv(name);
  return v && v[0] && v[0] != '0';
}

// 3D FP32 kernel family: the tuning knob when set (0 z-streamed, 1 staged
// forward, 2 wide), else DEEPGPR_B200_TMA=1 (staged forward) or
// DEEPGPR_B200_NARROW=1 (z-streamed), else -1: the automatic choice of
// k3w_auto.  A family that does not take the solve falls back to the
// z-streamed kernels.
int k3_family() {
  if (g_opt.tma >= 0) return g_opt.tma;
  if (env_flag("DEEPGPR_B200_TMA")) return 1;
  return env_flag("DEEPGPR_B200_NARROW") ? 0 : -1;
}

// Fraction of the grid's cells outside every CPML slab and the grid ends.
double k3_interior_fraction(const Grid& g, const int* p) {
  auto f = [](int n, int lo, int hi) { return std::max(0.0, (double)(n - lo - hi - 2) / n); };
  return f(g.NX, p[0], p[1]) * f(g.NY, p[2], p[3]) * f(g.NZ, p[4], p[5]);
}

// Automatic family of a half step (FP32, wide kernels usable).  The wide
// kernels need busy lanes: the share of their 128-column strips' lanes that
// hold grid columns (the z-streamed kernels use 64-column strips).  The wide
// E forward step of the pass form is taken at 70 % busy lanes; the wide H
// forward step, E forward step with its CPML in the kernel and adjoint steps
// at 80 % busy lanes with at least 70 % of the cells outside the CPML frame.
// Measured against the z-streamed kernels, both at their best x chunks
// (k3_layout, k3w_layout): on 320 x 320 x 160 + CPML 10 (77 % outside, 71 %
// busy lanes) the wide E pass-form step is 11 % faster, the z-streamed H
// step 2 % and the z-streamed adjoint steps 10-11 % faster; on 200^3 + CPML
// 10 (74 %, 86 %) the wide H and adjoint steps are 10 % and 6-8 % faster; on
// 160^3 + CPML 10 (69 %, 71 %) the wide E pass-form step is 10 % faster and
// the wide adjoint steps 15 % slower; on 160 x 160 x 96 + CPML 10 (65 %,
// 91 %) the wide E pass-form step is 17 % faster and the others 8-34 %
// slower (they read the x- and y-face CPML operands where they are used);
// on 140^3 + CPML 10 (64 %, 63 %) the wide E pass-form step is 6 % slower.
double k3w_lane_use(const Grid& g) { return (double)g.NZ / (double)(((g.NZ + 31) / 32 * 32 + KWW - 1) / KWW * KWW); }
bool k3w_auto(bool e_pass, double interior, double lanes) {
  return e_pass ? lanes >= 0.7 : (lanes >= 0.8 && interior >= 0.7);
}

// Whether the wide kernels take a 3D FP32 forward solve: radius <= 2, the
// single-face CPML form (or none) and at most 64 z-face cells of E and of H
// in every 128-column strip.
bool k3w_usable(const Grid& g, const int* p, bool has_cpml, int R) {
  if (R > 2) return false;
  if (!has_cpml) return true;
  if (!k3_cpml_single(g, p)) return false;
  const int zp = (g.NZ + 31) / 32 * 32;
  for (int k0 = 0; k0 < zp; k0 += KWW)
    if (zslots<false>(p[4], p[5], g.NZ, k0).n() > 64 || zslots<true>(p[4], p[5], g.NZ, k0).n() > 64) return false;
  return true;
}

// x chunks of a streamed 3D launch of `per` CTAs per chunk: the count keeps
// the last wave nearly full and each chunk long against its halo planes.
int k3_pick_xchunks(int NX, long long per, double resident, double halo) {
  int best = 1;
  double best_eff = -1.0;
  for (int n = 1; n <= std::max(1, std::min(64, NX / 16)); ++n) {
    const int xc = (NX + n - 1) / n;
    const int nch = (NX + xc - 1) / xc;
    const double nb = (double)per * nch;
    const double waves = std::ceil(nb / resident);
    const double eff = nb / (waves * resident) * (double)xc / (xc + halo);
    if (eff > best_eff + 1e-3) {
      best_eff = eff;
      best = n;
    }
  }
  if (g_opt.k3_xchunks > 0) best = std::min(g_opt.k3_xchunks, NX);
  return best;
}

// Dynamic shared memory of a wide kernel (its staging ring), granted once.
// KIND: 0 H half step, 1 E half step, 2 E half step of the pass form.
template <int R, bool EQ, int KIND>
bool k3w_prepare() {
  static const bool ok = [] {
    auto kernel = KIND == 0 ? (void (*)(TiledFwd<float>, K3Buf<float>, K3WGeom))k3w_fwd_h<R, EQ>
                            : (KIND == 1 ? k3w_fwd_e<R, EQ, false> : k3w_fwd_e<R, EQ, true>);
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kw_smem_bytes<R, KIND != 0>()) == cudaSuccess;
  }();
  return ok;
}

template <int R>
bool k3w_ready_r() {
  return k3w_prepare<R, true, 0>() && k3w_prepare<R, true, 1>() && k3w_prepare<R, true, 2>() &&
         k3w_prepare<R, false, 0>() && k3w_prepare<R, false, 1>() && k3w_prepare<R, false, 2>();
}

// Every instantiation is granted its shared memory before any launch (the
// launches may be captured into graphs).
bool k3w_ready() { return k3w_ready_r<1>() && k3w_ready_r<2>(); }

template <int R, bool EQ>
bool k3w_adj_prepare() {
  static const bool ok =
      cudaFuncSetAttribute(k3w_adj_e<R, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, kw_adj_smem_bytes()) ==
          cudaSuccess &&
      cudaFuncSetAttribute(k3w_adj_h<R, EQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, kw_adj_smem_bytes()) ==
          cudaSuccess;
  return ok;
}
bool k3w_adj_ready() {
  return k3w_adj_prepare<1, true>() && k3w_adj_prepare<1, false>() && k3w_adj_prepare<2, true>() &&
         k3w_adj_prepare<2, false>();
}

// The wide adjoint kernels: KIND 0 the adjoint E step, 1 the adjoint H step.
template <int KIND>
void k3w_adj_launch(int R, bool eq, cudaStream_t st, const TiledAdj<float>& P, const K3Buf<float>& kf,
                    const K3WGeom& kg) {
  const dim3 grid((unsigned)kg.nblocks), block(32, KW_WARPS);
  const int bytes = kw_adj_smem_bytes();
  auto go = [&](auto RR, auto E) {
    constexpr int RV = decltype(RR)::value;
    constexpr bool EV = decltype(E)::value;
    if constexpr (KIND == 0) k3w_adj_e<RV, EV><<<grid, block, bytes, st>>>(P, kf, kg);
    else k3w_adj_h<RV, EV><<<grid, block, bytes, st>>>(P, kf, kg);
  };
  if (R == 1) {
    if (eq) go(std::integral_constant<int, 1>(), std::true_type());
    else go(std::integral_constant<int, 1>(), std::false_type());
  } else {
    if (eq) go(std::integral_constant<int, 2>(), std::true_type());
    else go(std::integral_constant<int, 2>(), std::false_type());
  }
}

// min_chunks as in k3_layout (the wide adjoint steps: 12 measured 2-3 %
// faster than the wave-fill choice on 320 x 320 x 160 + CPML 10).
K3WGeom k3w_layout(const Grid& g, int zp, int min_chunks) {
  K3WGeom kg;
  memset(&kg, 0, sizeof(kg));
  kg.zp = zp;
  kg.nzs = (zp + KWW - 1) / KWW;
  kg.nyt = (g.NY + KW_WARPS - 1) / KW_WARPS;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k3w_fwd_e<2, true, false>, 32 * KW_WARPS,
                                                    kw_smem_bytes<2, true>()) != cudaSuccess ||
      blocks < 1) {
    cudaGetLastError();
    blocks = KW_MIN_BLOCKS;
  }
  const long long per = (long long)g.nshot * kg.nzs * kg.nyt;
  int n = k3_pick_xchunks(g.NX, per, (double)sm_count() * blocks, 3.0);
  if (g_opt.k3_xchunks <= 0) n = std::max(n, std::min(min_chunks, std::max(1, g.NX / 16)));
  kg.xc = (g.NX + n - 1) / n;
  kg.nchunk = (g.NX + kg.xc - 1) / kg.xc;
  kg.nblocks = per * kg.nchunk;
  return kg;
}

// KIND: 0 H half step, 1 E half step, 2 E half step of the pass form
template <int KIND>
void k3w_launch(int R, bool eq, cudaStream_t st, const TiledFwd<float>& P, const K3Buf<float>& kf,
                const K3WGeom& kg) {
  const dim3 grid((unsigned)kg.nblocks), block(32, KW_WARPS);
  auto go = [&](auto RR, auto E) {
    constexpr int RV = decltype(RR)::value;
    constexpr bool EV = decltype(E)::value;
    constexpr int bytes = kw_smem_bytes<RV, KIND != 0>();
    if constexpr (KIND == 0) k3w_fwd_h<RV, EV><<<grid, block, bytes, st>>>(P, kf, kg);
    else k3w_fwd_e<RV, EV, KIND == 2><<<grid, block, bytes, st>>>(P, kf, kg);
  };
  if (R == 1) {
    if (eq) go(std::integral_constant<int, 1>(), std::true_type());
    else go(std::integral_constant<int, 1>(), std::false_type());
  } else {
    if (eq) go(std::integral_constant<int, 2>(), std::true_type());
    else go(std::integral_constant<int, 2>(), std::false_type());
  }
}

// Whether the staged kernels take a 3D FP32 forward solve: the single-face
// CPML form (or none), TMA plane coordinates inside int32, and the driver's
// tensor-map encoder available.
bool k3t_usable(const Grid& g, const int* p, bool has_cpml) {
  if (has_cpml && !k3_cpml_single(g, p)) return false;
  if ((long long)g.nshot * g.NX >= (1LL << 31)) return false;
  return encode_tiled_fn() != nullptr;
}

template <int R>
int k3t_resident_per_sm() {
  return kt_min_blocks<R>();
}

// Tiles, z strips and x chunks: the chunk count keeps the last wave of CTAs
// nearly full and each chunk long against its 2R - 1 halo planes.
K3TGeom k3t_layout(const Grid& g, int zp, int R) {
  K3TGeom tg;
  memset(&tg, 0, sizeof(tg));
  tg.zp = zp;
  tg.nyt = (g.NY + KT_TY - 1) / KT_TY;
  tg.nzs = (g.NZ + KT_TZ - 1) / KT_TZ;
  const int per_sm = R >= 4 ? 1 : (R >= 2 ? 2 : 3);
  const double resident = (double)sm_count() * per_sm;
  const long long per = (long long)g.nshot * tg.nzs * tg.nyt;
  int best = 1;
  double best_eff = -1.0;
  for (int n = 1; n <= std::max(1, std::min(64, g.NX / 8)); ++n) {
    const int xc = (g.NX + n - 1) / n;
    const int nch = (g.NX + xc - 1) / xc;
    const double nb = (double)per * nch;
    const double waves = std::ceil(nb / resident);
    const double eff = nb / (waves * resident) * (double)xc / (xc + 2.0 * R + 2.0);
    if (eff > best_eff + 1e-3) {
      best_eff = eff;
      best = n;
    }
  }
  if (g_opt.k3_xchunks > 0) best = std::min(g_opt.k3_xchunks, g.NX);
  tg.xc = (g.NX + best - 1) / best;
  tg.nchunk = (g.NX + tg.xc - 1) / tg.xc;
  tg.nblocks = per * tg.nchunk;
  return tg;
}

// Tensor maps of one half step (H when efield is false, E otherwise).
template <typename T>
bool k3t_maps(K3TMaps& m, const Grid& g, int zp, int R, const K3Buf<T>& kf, bool efield) {
  if constexpr (sizeof(T) != 4) {
    return false;
  } else {
    const long long planes = (long long)g.nshot * g.NX;
    const T* halo[3] = {efield ? kf.Hx : kf.Ex, efield ? kf.Hy : kf.Ey, efield ? kf.Hz : kf.Ez};
    const T* own[3] = {efield ? kf.Ex : kf.Hx, efield ? kf.Ey : kf.Hy, efield ? kf.Ez : kf.Hz};
    const T* coef[2] = {efield ? kf.ce_hist : kf.ch_curl, efield ? kf.ce_curl : kf.ch_curl};
    bool ok = true;
    for (int c = 0; c < 3; ++c) {
      ok = ok && make_map_f32(&m.halo[c], halo[c], g.NZ, zp, g.NY, planes, KT_BZ, KT_TY + 2 * R);
      ok = ok && make_map_f32(&m.own[c], own[c], g.NZ, zp, g.NY, planes, KT_TZ, KT_TY);
    }
    for (int c = 0; c < 2; ++c) ok = ok && make_map_f32(&m.coef[c], coef[c], g.NZ, zp, g.NY, g.NX, KT_TZ, KT_TY);
    if (!ok) set_error("forward: tensor map encoding failed");
    return ok;
  }
}

template <int R, bool EQ, bool EFIELD>
void k3t_launch_one(unsigned nblocks, cudaStream_t st, const K3TMaps& m, const TiledFwd<float>& P,
                    const K3Buf<float>& kf, const K3TGeom& tg) {
  constexpr int NOWN = EFIELD ? 5 : 4;
  constexpr size_t bytes = KtShape<R, NOWN>::BYTES;
  auto kernel = EFIELD ? k3t_fwd_e<R, EQ> : k3t_fwd_h<R, EQ>;
  static bool attr = [&] {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return true;
  }();
  (void)attr;
  kernel<<<nblocks, KT_THREADS, bytes, st>>>(m, P, kf, tg);
}

template <bool EFIELD>
void k3t_launch(int R, bool eq, cudaStream_t st, const K3TMaps& m, const TiledFwd<float>& P, const K3Buf<float>& kf,
                const K3TGeom& tg) {
  const unsigned nb = (unsigned)tg.nblocks;
  if (R == 1) {
    if (eq) k3t_launch_one<1, true, EFIELD>(nb, st, m, P, kf, tg);
    else k3t_launch_one<1, false, EFIELD>(nb, st, m, P, kf, tg);
  } else if (R == 2) {
    if (eq) k3t_launch_one<2, true, EFIELD>(nb, st, m, P, kf, tg);
    else k3t_launch_one<2, false, EFIELD>(nb, st, m, P, kf, tg);
  } else {
    if (eq) k3t_launch_one<4, true, EFIELD>(nb, st, m, P, kf, tg);
    else k3t_launch_one<4, false, EFIELD>(nb, st, m, P, kf, tg);
  }
}

template <typename T>
struct ForwardCall {
  Common<T> cm;
  void *E_saved, *R_saved;
  T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
  int nrx;
  const int* rx_loc;
  T* rx;
  int rx_comp;
  int nsrc;
  const int* src_loc;
  const T* wave;
  int src_comp;
  int save_model_history;
};

template <typename T, typename Alloc = Scratch>
void forward_impl(const ForwardCall<T>& fc) {
  g_error[0] = '\0';
  const Common<T>& cm = fc.cm;
  const Grid& g = cm.g;
  if (g.NX < 2 || g.NY < 2 || g.NZ < 2 || g.nshot < 1 || cm.nt < 0) {
    set_error("forward: invalid grid (%d, %d, %d), nshot %d, nt %d", g.NX, g.NY, g.NZ, g.nshot, cm.nt);
    return;
  }
  if ((long long)g.NX * g.NY * g.NZ > 0x7fffffffLL) {
    set_error("forward: %d x %d x %d field cells per shot exceed the 2^31 limit", g.NX, g.NY, g.NZ);
    return;
  }
  if (cm.S < 1) {
    set_error("forward: sampling interval must be positive");
    return;
  }
  const int kind = cm.storage_type & ST_KIND_MASK;
  const bool history = (cm.storage_type & ST_DISABLED) == 0;
  const bool e_only = history && fc.save_model_history && (cm.storage_type & ST_RHS_FROM_E);
  const bool keep_r = history && fc.save_model_history && !e_only;
  const bool physical = (cm.storage_type & ST_PHYSICAL) != 0;
  const bool tm2d = (cm.storage_type & ST_TM2D) != 0;
  const bool has_cpml = cm.p[0] || cm.p[1] || cm.p[2] || cm.p[3] || cm.p[4] || cm.p[5];
  if (history && fc.save_model_history && has_cpml && physical) {
    set_error("forward: material gradients with PML require extended wavefield history; "
              "physical history omits PML material sensitivities");
    return;
  }
  if (e_only && cm.S != 1) {
    set_error("forward: E-only wavefield history requires sampling interval 1");
    return;
  }
  if (history && kind != kF32 && kind != kF16 && kind != kBF16 && !is_tiled(kind) && kind != kF64) {
    set_error("forward: unsupported history storage kind %d", kind);
    return;
  }
  if (history && is_tiled(kind) && e_only) {
    set_error("forward: one-byte (FP8 / INT8) histories keep E and R (no E-only reconstruction)");
    return;
  }
  if (history && (kind == kF64) != (sizeof(T) == 8)) {
    set_error("forward: FP64 histories are used exactly by the FP64 entry points");
    return;
  }
  if (tm2d && (g.NZ != 2 || fc.src_comp != 2 || (history && cm.mode != 2))) {
    set_error("forward: the 2D TM path needs nz = 1, an Ez source and gradient mode 2");
    return;
  }
  StreamSet* ss = stream_set();
  if (!ss) {
    set_error("forward: cannot create the CUDA stream");
    return;
  }
  const cudaStream_t user = caller_stream();
  const cudaStream_t st = ss->work;
  if (!cuda_ok(cudaEventRecord(ss->in, user), "event record") || !cuda_ok(cudaStreamWaitEvent(st, ss->in, 0), "wait"))
    return;
  bool ok = true;
  {
    Alloc scratch(st);
    TiledFwd<T> P;
    memset(&P, 0, sizeof(P));
    FwdArgs<T>& a = P.a;
    a.g = g;
    a.dx = cm.dx;
    a.dy = cm.dy;
    a.dz = cm.dz;
    a.ddx = fixed_div(cm.dx);
    a.ddy = fixed_div(cm.dy);
    a.ddz = fixed_div(cm.dz);
    a.dy_eq = cm.dy == cm.dx;
    a.dz_eq = cm.dz == cm.dx;
    a.Ex = fc.Ex; a.Ey = fc.Ey; a.Ez = fc.Ez;
    a.Hx = fc.Hx; a.Hy = fc.Hy; a.Hz = fc.Hz;
    a.ce_hist = cm.ce_hist;
    a.ce_curl = cm.ce_curl;
    a.ce_rhs = cm.ce_rhs;
    a.ch_curl = cm.ch_curl;
    a.ch_rhs = cm.ch_rhs;
    fill_faces(a.eF, cm.p, cm.eR, cm.ePsi);
    fill_faces(a.hF, cm.p, cm.hR, cm.hPsi);
    a.has_cpml = has_cpml;
    a.nt = cm.nt;
    a.wave = fc.wave;
    a.src_comp = fc.src_comp;
    a.src_dl = fc.src_comp == 0 ? cm.dx : (fc.src_comp == 1 ? cm.dy : cm.dz);
    a.src_vol = cm.dx * cm.dy * cm.dz;
    a.rx = fc.rx;
    a.rx_comp = (fc.rx_comp < 0 || fc.rx_comp > 2) ? 2 : fc.rx_comp;  // deepgpr_cpu.c:620
    a.nrx = fc.nrx;
    a.save_e = history;
    a.keep_r = keep_r;
    a.S = cm.S;
    a.mode = cm.mode;
    a.kind = kind;
    a.nt_saved = (cm.nt + cm.S - 1) / cm.S;
    a.box = make_box(g, physical, cm.p);
    a.frame = (long long)g.nshot * a.box.cells();
    a.comp_stride = (long long)a.nt_saved * a.frame;
    a.E_saved = fc.E_saved;
    a.R_saved = fc.R_saved;
    a.ntiles = (int)fp8_tiles(g, tm2d);
    const int ncomp = cm.mode == 3 ? 3 : 1;
    if (history && is_tiled(kind)) {
      const long long vals = (long long)ncomp * a.comp_stride;
      a.e_scales = reinterpret_cast<float*>(static_cast<char*>(fc.E_saved) + fp8_payload_bytes(vals));
      if (keep_r) a.r_scales = reinterpret_cast<float*>(static_cast<char*>(fc.R_saved) + fp8_payload_bytes(vals));
    }
    Control* ctrl = scratch.template get<Control>(sizeof(Control));
    ok = !scratch.failed;
    const int R = radius_of(g_opt.order_override ? g_opt.order_override : g_order);
    TmGeom tg;
    memset(&tg, 0, sizeof(tg));
    if (tm2d) tg = tm_layout(g);
    // sources of an invalid component inject nothing (deepgpr_cpu.c:650)
    std::vector<char> src_any, rcv_any;
    const unsigned char *src_rows = nullptr, *rcv_rows = nullptr;
    if (ok) {
      const bool src_on = fc.src_comp >= 0 && fc.src_comp <= 2;
      ok = build_points(src_on ? fc.src_loc : nullptr, fc.nsrc, fc.rx_loc, fc.nrx, g, st, scratch, &P.src, &a.src,
                        &P.rcv, &a.rcv, &src_rows, &rcv_rows, tm2d ? &src_any : nullptr, tm2d ? &rcv_any : nullptr);
    }
    tg.src_rows = src_rows;
    tg.rcv_rows = rcv_rows;
    // rows with a source or receiver of any shot go to the general (frame) kernels
    std::vector<char> pt_rows(tm2d ? g.NX : 0, 0);
    for (int i = 0; i < (int)pt_rows.size(); ++i)
      pt_rows[i] = (i < (int)src_any.size() && src_any[i]) || (i < (int)rcv_any.size() && rcv_any[i]);
    if (ok) ok = launch_coeffs(cm, st);
    TmBuf<T> tf;
    memset(&tf, 0, sizeof(tf));
    const long long plane2 = (long long)g.NX * tg.NYP;
    if (ok && tm2d) {
      // + two y-scaled curl planes when dy != dx, + a tail pad: masked lanes of the
      // last interior strip may read up to 4 * 32 columns past a row end
      const int ncoef = cm.dy == cm.dx ? 5 : 7;
      T* buf = scratch.template get<T>(((size_t)(3 * g.nshot + ncoef) * plane2 + kTmTailPad) * sizeof(T));
      ok = buf != nullptr;
      if (ok) {
        tf.Ez = buf;
        tf.Hx = buf + g.nshot * plane2;
        tf.Hy = buf + 2 * g.nshot * plane2;
        T* cf = buf + 3 * g.nshot * plane2;
        const T* srcs[5] = {cm.ce_hist, cm.ce_curl, cm.ce_rhs, cm.ch_curl, cm.ch_rhs};
        for (int q = 0; q < 5; ++q) k_pack2d_pitch<T><<<1024, 256, 0, st>>>(srcs[q], cf + q * plane2, g.NX, g.NY, tg.NYP);
        tf.ce_hist = cf;
        tf.ce_curl = cf + plane2;
        tf.ce_rhs = cf + 2 * plane2;
        tf.ch_curl = cf + 3 * plane2;
        tf.ch_rhs = cf + 4 * plane2;
        tf.ce_curl_y = tf.ce_curl;
        tf.ch_curl_y = tf.ch_curl;
        if (ncoef == 7) {
          k_pack2d_pitch_ys<T><<<1024, 256, 0, st>>>(cm.ce_curl, cf + 5 * plane2, g.NX, g.NY, tg.NYP, cm.dx, cm.dy);
          k_pack2d_pitch_ys<T><<<1024, 256, 0, st>>>(cm.ch_curl, cf + 6 * plane2, g.NX, g.NY, tg.NYP, cm.dx, cm.dy);
          tf.ce_curl_y = cf + 5 * plane2;
          tf.ch_curl_y = cf + 6 * plane2;
        }
        cudaMemsetAsync(cf + ncoef * plane2, 0, kTmTailPad * sizeof(T), st);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(fc.Ez, tf.Ez, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(fc.Hx, tf.Hx, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(fc.Hy, tf.Hy, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        ok = cuda_ok(cudaGetLastError(), "pack");
      }
    }
    // 3D: z-pitched working copy of the fields and coefficients
    K3Buf<T> kf;
    memset(&kf, 0, sizeof(kf));
    K3Geom kg;
    memset(&kg, 0, sizeof(kg));
    const bool eq3 = cm.dy == cm.dx && cm.dz == cm.dx;
    // CPML form of the 3D forward kernels: in FP32 the E CPML frame is finished
    // by the per-cell pass when no R^n history is kept (R^n needs E^n, which the
    // streamed kernel overwrites); the H z faces by their own pass
    const int cpm_base = (a.has_cpml && !k3_cpml_single(g, cm.p)) ? kCpmGeneral : kCpmSingle;
    const bool pass3 = sizeof(T) == 4 && a.has_cpml && g.nshot <= 65535;
    const int cpm_h = cpm_base;
    const int cpm_e = (pass3 && !keep_r) ? kCpmPass : cpm_base;
    if (ok && !tm2d) {
      kg = k3_layout(g, 12);
      kg.src_rows = src_rows;
      kg.rcv_rows = rcv_rows;
      kg.cpml_single = k3_cpml_single(g, cm.p);
      kg.fr = k3_frame(g, cm.p);
      kg.zpost_h = sizeof(T) == 4 && a.has_cpml && kg.cpml_single && g.nshot <= 65535;
      ok = k3_alloc_pack(scratch, g, kg, cm, st, kf, fc.Ex, fc.Ey, fc.Ez, fc.Hx, fc.Hy, fc.Hz);
    }
    // TMA-staged kernels for the FP32 3D forward (the z-streamed kernels otherwise)
    const int fam3 = k3_family();
    const bool fast3 = sizeof(T) == 4 && ok && !tm2d && fam3 == 1 && k3t_usable(g, cm.p, a.has_cpml != 0);
    // wide kernels (fdtd_3d_wide.cuh) for the FP32 3D forward half steps
    const bool wide_ok = sizeof(T) == 4 && ok && !tm2d && !fast3 && (fam3 == 2 || fam3 < 0) &&
                         k3w_usable(g, cm.p, a.has_cpml != 0, R) && k3w_ready();
    const double inner3 = k3_interior_fraction(g, cm.p);
    const double lanes3 = k3w_lane_use(g);
    const bool wideH = wide_ok && (fam3 == 2 || k3w_auto(false, inner3, lanes3));
    const bool wideE = wide_ok && (fam3 == 2 || k3w_auto(cpm_e == kCpmPass, inner3, lanes3));
    K3WGeom kwg;
    memset(&kwg, 0, sizeof(kwg));
    if (wideH || wideE) {
      kwg = k3w_layout(g, kg.zp, 0);
      kwg.src_rows = src_rows;
      kwg.rcv_rows = rcv_rows;
      for (int ax = 0; ax < 3; ++ax) {
        kwg.lo[ax] = kg.fr.lo[ax];
        kwg.hi[ax] = kg.fr.hi[ax];
      }
    }
    K3TGeom ktg;
    memset(&ktg, 0, sizeof(ktg));
    K3TMaps kmH, kmE;
    if (fast3) {
      ktg = k3t_layout(g, kg.zp, R);
      ktg.src_rows = src_rows;
      ktg.rcv_rows = rcv_rows;
      ktg.ctrl = ctrl;
      ok = k3t_maps(kmH, g, kg.zp, R, kf, false) && k3t_maps(kmE, g, kg.zp, R, kf, true);
    }
    if (ok) {
      a.ctrl = ctrl;
      k_set<<<1, 1, 0, st>>>(ctrl, 0);
      const long long tiles = tm2d ? 1 : tiles3(g);
      P.xchunk = pick_xchunk(g.NX, tiles, g.nshot, 4 * R);
      P.tm2d = tm2d;
      dim3 grid((unsigned)tiles, (unsigned)((g.NX + P.xchunk - 1) / P.xchunk), (unsigned)g.nshot);
      const dim3 wblock(32, TM_WARPS);
      // 2D TM: general kernels on the CPML / boundary frame, interior kernels inside
      const bool lean2d = tm2d && a.box.z0 == 0 && a.box.nz == 1;
      const TmFaces tfc = tm_faces(a.eF, a.hF, a.has_cpml != 0);
      TmPlan pH, pE;
      if (tm2d) {
        const int bH = R == 1 ? blocks_per_sm(tmi_fwd_h<T, 1>) : R == 2 ? blocks_per_sm(tmi_fwd_h<T, 2>)
                                                                        : blocks_per_sm(tmi_fwd_h<T, 4>);
        const int bE = R == 1 ? blocks_per_sm(tmi_fwd_e<T, 1>) : R == 2 ? blocks_per_sm(tmi_fwd_e<T, 2>)
                                                                        : blocks_per_sm(tmi_fwd_e<T, 4>);
        pH = tm_plan(tg, g, 0, R, tfc, lean2d, bH);
        pE = tm_plan(tg, g, 1, R, tfc, lean2d, bE, &pt_rows);
      }
      auto issue = [&](int k) {
        TiledFwd<T> b = P;
        b.a.k_in_chunk = k;
        if (tm2d) {
          timed(KK_FWD_H, st, [&] {
            return tm_launch(
                st, ss, pH,
                [&](dim3 gfu, unsigned nfb) {
                  if (R == 1) tmf_fwd_h<T, 1><<<gfu, wblock, 0, st>>>(b, tf, pH.frame, pH.interior, nfb);
                  else if (R == 2) tmf_fwd_h<T, 2><<<gfu, wblock, 0, st>>>(b, tf, pH.frame, pH.interior, nfb);
                  else tmf_fwd_h<T, 4><<<gfu, wblock, 0, st>>>(b, tf, pH.frame, pH.interior, nfb);
                },
                [&](cudaStream_t q, const TmGeom& fg) {
                  const dim3 gf = tm_grid(fg);
                  if (R == 1) tm_fwd_h<T, 1><<<gf, wblock, 0, q>>>(b, tf, fg);
                  else if (R == 2) tm_fwd_h<T, 2><<<gf, wblock, 0, q>>>(b, tf, fg);
                  else tm_fwd_h<T, 4><<<gf, wblock, 0, q>>>(b, tf, fg);
                },
                [&](cudaStream_t q) {
                  const dim3 gi = tm_grid(pH.interior);
                  if (R == 1) tmi_fwd_h<T, 1><<<gi, wblock, 0, q>>>(b, tf, pH.interior);
                  else if (R == 2) tmi_fwd_h<T, 2><<<gi, wblock, 0, q>>>(b, tf, pH.interior);
                  else tmi_fwd_h<T, 4><<<gi, wblock, 0, q>>>(b, tf, pH.interior);
                });
          });
          timed(KK_FWD_E, st, [&] {
            return tm_launch(
                st, ss, pE,
                [&](dim3 gfu, unsigned nfb) {
                  if (R == 1) tmf_fwd_e<T, 1><<<gfu, wblock, 0, st>>>(b, tf, pE.frame, pE.interior, nfb);
                  else if (R == 2) tmf_fwd_e<T, 2><<<gfu, wblock, 0, st>>>(b, tf, pE.frame, pE.interior, nfb);
                  else tmf_fwd_e<T, 4><<<gfu, wblock, 0, st>>>(b, tf, pE.frame, pE.interior, nfb);
                },
                [&](cudaStream_t q, const TmGeom& fg) {
                  const dim3 gf = tm_grid(fg);
                  if (R == 1) tm_fwd_e<T, 1><<<gf, wblock, 0, q>>>(b, tf, fg);
                  else if (R == 2) tm_fwd_e<T, 2><<<gf, wblock, 0, q>>>(b, tf, fg);
                  else tm_fwd_e<T, 4><<<gf, wblock, 0, q>>>(b, tf, fg);
                },
                [&](cudaStream_t q) {
                  const dim3 gi = tm_grid(pE.interior);
                  if (R == 1) tmi_fwd_e<T, 1><<<gi, wblock, 0, q>>>(b, tf, pE.interior);
                  else if (R == 2) tmi_fwd_e<T, 2><<<gi, wblock, 0, q>>>(b, tf, pE.interior);
                  else tmi_fwd_e<T, 4><<<gi, wblock, 0, q>>>(b, tf, pE.interior);
                });
          });
        } else if (fast3) {
          if constexpr (sizeof(T) == 4) {
            timed(KK_FWD_H, st, [&] { k3t_launch<false>(R, eq3, st, kmH, b, kf, ktg); });
            timed(KK_FWD_E, st, [&] { k3t_launch<true>(R, eq3, st, kmE, b, kf, ktg); });
          }
        } else {
          const dim3 g3((unsigned)kg.nblocks), b3(32, K3_WARPS);
          const dim3 gfr((kg.fr.cum[5] + kBlock - 1) / kBlock, (unsigned)g.nshot);
          const int nyb = (g.NY + kZfRowsF - 1) / kZfRowsF;
          const dim3 gz((unsigned)(g.NX * nyb), (unsigned)g.nshot), bz(32, kZfRowsF);
          timed(KK_FWD_H, st, [&] {
            if constexpr (sizeof(T) == 4) {
              if (wideH) {
                k3w_launch<0>(R, eq3, st, b, kf, kwg);
                return 1;
              }
            }
            k3_fwd_variant<T>(R, eq3, cpm_h, [&](auto RR, auto E, auto C) {
              k3v_fwd_h<T, decltype(RR)::value, decltype(E)::value, decltype(C)::value><<<g3, b3, 0, st>>>(b, kf, kg);
              if (kg.zpost_h) k3z_fwd_h<T, decltype(RR)::value><<<gz, bz, 0, st>>>(b, kf, kg, nyb);
            });
            return kg.zpost_h ? 2 : 1;
          });
          timed(KK_FWD_E, st, [&] {
            if constexpr (sizeof(T) == 4) {
              if (wideE) {
                if (cpm_e != kCpmPass) {
                  k3w_launch<1>(R, eq3, st, b, kf, kwg);
                  return 1;
                }
                k3w_launch<2>(R, eq3, st, b, kf, kwg);
                if (R == 1) k3p_fwd_e<T, 1><<<gfr, kBlock, 0, st>>>(b, kf, kg);
                else k3p_fwd_e<T, 2><<<gfr, kBlock, 0, st>>>(b, kf, kg);
                return 2;
              }
            }
            k3_fwd_variant<T>(R, eq3, cpm_e, [&](auto RR, auto E, auto C) {
              k3v_fwd_e<T, decltype(RR)::value, decltype(E)::value, decltype(C)::value><<<g3, b3, 0, st>>>(b, kf, kg);
              if (cpm_e == kCpmPass) k3p_fwd_e<T, decltype(RR)::value><<<gfr, kBlock, 0, st>>>(b, kf, kg);
            });
            return cpm_e == kCpmPass ? 2 : 1;
          });
        }
      };
      // host-resident histories (use_async_offload): device rings and a copy stream
      HistRing hr;
      const ThreadOptions saved_opt = g_opt;
      const bool off_e = history && is_host_memory(fc.E_saved);
      const bool off_r = keep_r && is_host_memory(fc.R_saved);
      if (ok && (off_e || off_r)) {
        if (is_tiled(kind)) {
          set_error("forward: one-byte (FP8 / INT8) histories stay on the device (no offload)");
          ok = false;
        } else {
          g_opt.use_graph = 0;   // the ring base changes from chunk to chunk
          g_opt.chunk = std::max(g_opt.chunk, 32);
          ok = hr.setup(scratch, st, off_e ? fc.E_saved : nullptr, off_r ? fc.R_saved : nullptr, cm.S, cm.nt,
                        a.nt_saved, ncomp, a.frame, hist_elem_bytes(kind), g_opt.chunk, 0);
        }
      }
      const int clen = std::max(1, g_opt.chunk);
      auto fhook = [&](int t, int K, int phase) -> bool {
        if (!hr.on) return true;
        int s0, s1;
        hr.fwd_slots(t, K, s0, s1);
        const int b = (t / clen) & 1;
        if (phase == 0) {
          if (hr.pending[b] && !cuda_ok(cudaStreamWaitEvent(st, hr.done[b], 0), "offload wait")) return false;
          if (hr.host[0]) a.E_saved = hr.base(0, b, s0);
          if (hr.host[1]) a.R_saved = hr.base(1, b, s0);
          a.comp_stride = hr.comp_stride();
          return true;
        }
        if (!cuda_ok(cudaEventRecord(hr.work[b], st), "offload event") ||
            !cuda_ok(cudaStreamWaitEvent(hr.copy, hr.work[b], 0), "offload wait") || !hr.move(b, s0, s1, true))
          return false;
        hr.pending[b] = true;
        return cuda_ok(cudaEventRecord(hr.done[b], hr.copy), "offload event");
      };
      if (ok) ok = run_loop(cm.nt, +1, ctrl, st, issue, fhook);
      if (hr.on) {
        for (int b = 0; b < 2; ++b)
          if (hr.pending[b]) cudaStreamWaitEvent(st, hr.done[b], 0);
        a.E_saved = fc.E_saved;
        a.R_saved = fc.R_saved;
        a.comp_stride = (long long)a.nt_saved * a.frame;
      }
      g_opt = saved_opt;
      if (ok && fast3) {
        // a staged-tile wait that ran out leaves its bit in the control block
        int herr = 0;
        ok = cuda_ok(cudaMemcpyAsync(&herr, &ctrl->error, sizeof(int), cudaMemcpyDeviceToHost, st), "error readback") &&
             cuda_ok(cudaStreamSynchronize(st), "error readback");
        if (ok && (herr & kErrWaitTimeout)) {
          set_error("forward: a staged-tile copy did not arrive in time (device error bits %d)", herr);
          ok = false;
        }
      }
      if (ok && tm2d) {
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tf.Ez, fc.Ez, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tf.Hx, fc.Hx, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tf.Hy, fc.Hy, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        ok = cuda_ok(cudaGetLastError(), "unpack");
      }
      if (ok && !tm2d) ok = k3_unpack(g, kg, st, kf, fc.Ex, fc.Ey, fc.Ez, fc.Hx, fc.Hy, fc.Hz);
      if (ok && e_only) {
        // closing E^nt frame into R_saved (deepgpr_cpu.c:1919-1930)
        const long long bc = a.box.cells();
        for (int q = 0; q < ncomp; ++q) {
          const int fcmp = cm.mode == 3 ? q : 2;
          const T* E = fcmp == 0 ? fc.Ex : (fcmp == 1 ? fc.Ey : fc.Ez);
          void* dst = static_cast<char*>(fc.R_saved) + (long long)q * g.nshot * bc * hist_elem_bytes(kind);
          k_final_frame<T><<<512, 256, 0, st>>>(E, dst, g, a.box, kind);
        }
        ok = cuda_ok(cudaGetLastError(), "final frame");
      }
    }
  }
  cudaEventRecord(ss->out, st);
  cudaStreamWaitEvent(user, ss->out, 0);
  if (ok) cuda_ok(cudaGetLastError(), "forward");
}


template <typename T>
struct BackwardCall {
  Common<T> cm;
  const void *E_saved, *R_saved;
  T *lEx, *lEy, *lEz, *lHx, *lHy, *lHz;
  int ndata;
  const int* rx_loc;
  const T* data_grad;
  int rx_comp;
  int nsrc;
  const int* src_loc;
  int src_comp;
  T* grad_source;
  int want_src;
  T *grad_eps, *grad_sig;
  int want_eps, want_sig;
};

// Element counts of the 12 psi arrays of one field (E or H), in the order
// x0 psi1, x0 psi2, xm psi1, ..., zm psi2.
template <bool EFIELD>
void psi_counts(const Grid& g, const int* p, long long* out) {
  for (int f = 0; f < 6; ++f) {
    const int axis = f / 2, q = p[f];
    for (int slot = 1; slot <= 2; ++slot) {
      long long a, b, c;
      const int pe = EFIELD ? q + 1 : q;
      if (axis == 0) {
        a = pe;
        b = slot == 1 ? (EFIELD ? g.NY - 1 : g.NY) : (EFIELD ? g.NY : g.NY - 1);
        c = slot == 1 ? (EFIELD ? g.NZ : g.NZ - 1) : (EFIELD ? g.NZ - 1 : g.NZ);
      } else if (axis == 1) {
        a = slot == 1 ? (EFIELD ? g.NX - 1 : g.NX) : (EFIELD ? g.NX : g.NX - 1);
        b = pe;
        c = slot == 1 ? (EFIELD ? g.NZ : g.NZ - 1) : (EFIELD ? g.NZ - 1 : g.NZ);
      } else {
        a = slot == 1 ? (EFIELD ? g.NX - 1 : g.NX) : (EFIELD ? g.NX : g.NX - 1);
        b = slot == 1 ? (EFIELD ? g.NY : g.NY - 1) : (EFIELD ? g.NY - 1 : g.NY);
        c = pe;
      }
      out[2 * f + slot - 1] = q > 0 ? (long long)g.nshot * a * b * c : 0;
    }
  }
}

template <typename T>
void backward_impl(const BackwardCall<T>& bc) {
  g_error[0] = '\0';
  const Common<T>& cm = bc.cm;
  const Grid& g = cm.g;
  if (g.NX < 2 || g.NY < 2 || g.NZ < 2 || g.nshot < 1 || cm.nt < 0 || cm.S < 1) {
    set_error("backward: invalid grid (%d, %d, %d), nshot %d, nt %d, interval %d", g.NX, g.NY, g.NZ, g.nshot,
              cm.nt, cm.S);
    return;
  }
  if ((long long)g.NX * g.NY * g.NZ > 0x7fffffffLL) {
    set_error("backward: %d x %d x %d field cells per shot exceed the 2^31 limit", g.NX, g.NY, g.NZ);
    return;
  }
  const int kind = cm.storage_type & ST_KIND_MASK;
  const bool want_model = bc.want_eps || bc.want_sig;
  const bool e_only = want_model && (cm.storage_type & ST_RHS_FROM_E);
  const bool physical = (cm.storage_type & ST_PHYSICAL) != 0;
  const bool tm2d = (cm.storage_type & ST_TM2D) != 0;
  const bool has_cpml = cm.p[0] || cm.p[1] || cm.p[2] || cm.p[3] || cm.p[4] || cm.p[5];
  if (want_model && has_cpml && physical) {
    set_error("backward: material gradients with PML require extended wavefield history; "
              "physical history omits PML material sensitivities");
    return;
  }
  if (e_only && cm.S != 1) {
    set_error("backward: E-only wavefield history requires sampling interval 1");
    return;
  }
  if (want_model && is_tiled(kind) && e_only) {
    set_error("backward: one-byte (FP8 / INT8) histories keep E and R (no E-only reconstruction)");
    return;
  }
  if (want_model && (kind == kF64) != (sizeof(T) == 8)) {
    set_error("backward: FP64 histories are used exactly by the FP64 entry points");
    return;
  }
  if (tm2d && (g.NZ != 2 || bc.src_comp != 2 || (want_model && cm.mode != 2))) {
    set_error("backward: the 2D TM path needs nz = 1, an Ez source and gradient mode 2");
    return;
  }
  StreamSet* ss = stream_set();
  if (!ss) {
    set_error("backward: cannot create the CUDA stream");
    return;
  }
  const cudaStream_t user = caller_stream();
  const cudaStream_t st = ss->work;
  if (!cuda_ok(cudaEventRecord(ss->in, user), "event record") || !cuda_ok(cudaStreamWaitEvent(st, ss->in, 0), "wait"))
    return;
  bool ok = true;
  {
    Scratch scratch(st);
    TiledAdj<T> P;
    memset(&P, 0, sizeof(P));
    AdjArgs<T>& a = P.a;
    a.g = g;
    a.dx = cm.dx;
    a.dy = cm.dy;
    a.dz = cm.dz;
    a.ddt = fixed_div(cm.dt);
    a.ddy = fixed_div(cm.dy);
    a.ddz = fixed_div(cm.dz);
    a.inv_dx = T(1) / cm.dx;
    a.inv_dy = T(1) / cm.dy;
    a.inv_dz = T(1) / cm.dz;
    a.dy_eq = cm.dy == cm.dx;
    a.dz_eq = cm.dz == cm.dx;
    a.lEx = bc.lEx; a.lEy = bc.lEy; a.lEz = bc.lEz;
    a.lHx = bc.lHx; a.lHy = bc.lHy; a.lHz = bc.lHz;
    a.ce_hist = cm.ce_hist;
    a.ce_curl = cm.ce_curl;
    a.ce_rhs = cm.ce_rhs;
    a.ch_curl = cm.ch_curl;
    a.ch_rhs = cm.ch_rhs;
    fill_faces(a.eF, cm.p, cm.eR, cm.ePsi);
    fill_faces(a.hF, cm.p, cm.hR, cm.hPsi);
    a.has_cpml = has_cpml;
    a.nt = cm.nt;
    a.data_grad = bc.data_grad;
    a.rx_comp = bc.rx_comp;
    a.nrx = bc.ndata;
    a.want_src = bc.want_src == 1 && bc.src_comp >= 0 && bc.src_comp <= 2 && bc.nsrc > 0;
    a.nsrc = bc.nsrc;
    a.src_comp = bc.src_comp;
    a.grad_source = bc.grad_source;
    {
      const T dl = bc.src_comp == 0 ? cm.dx : (bc.src_comp == 1 ? cm.dy : cm.dz);
      a.src_geo = dl / (cm.dx * cm.dy * cm.dz);
    }
    a.want_eps = bc.want_eps == 1;
    a.want_sig = bc.want_sig == 1;
    a.acc64 = (sizeof(T) == 8) ? 1 : g_opt.acc64;
    a.g_eps = bc.grad_eps;
    a.g_sig = bc.grad_sig;
    a.sigma = cm.sig;
    a.dt = cm.dt;
    a.S = cm.S;
    a.mode = cm.mode;
    a.kind = kind;
    a.e_only = e_only;
    a.nt_saved = (cm.nt + cm.S - 1) / cm.S;
    a.box = make_box(g, physical, cm.p);
    a.frame = (long long)g.nshot * a.box.cells();
    a.comp_stride = (long long)a.nt_saved * a.frame;
    a.E_saved = bc.E_saved;
    a.R_saved = bc.R_saved;
    a.ntiles = (int)fp8_tiles(g, tm2d);
    const int ncomp = cm.mode == 3 ? 3 : 1;
    if (want_model && is_tiled(kind)) {
      const long long vals = (long long)ncomp * a.comp_stride;
      a.e_scales = reinterpret_cast<const float*>(static_cast<const char*>(bc.E_saved) + fp8_payload_bytes(vals));
      a.r_scales = reinterpret_cast<const float*>(static_cast<const char*>(bc.R_saved) + fp8_payload_bytes(vals));
    }
    Control* ctrl = scratch.get<Control>(sizeof(Control));
    ok = !scratch.failed;
    // CPML weight scratch, shaped like the psi arrays
    if (ok && has_cpml) {
      long long ce[12], ch[12], tot = 0;
      psi_counts<true>(g, cm.p, ce);
      psi_counts<false>(g, cm.p, ch);
      for (int q = 0; q < 12; ++q) tot += ce[q] + ch[q];
      T* w = scratch.get<T>((size_t)tot * sizeof(T));
      ok = w != nullptr;
      if (ok) {
        cudaMemsetAsync(w, 0, (size_t)tot * sizeof(T), st);
        long long o = 0;
        for (int f = 0; f < 6; ++f) {
          a.eF[f].w1 = w + o; o += ce[2 * f];
          a.eF[f].w2 = w + o; o += ce[2 * f + 1];
        }
        for (int f = 0; f < 6; ++f) {
          a.hF[f].w1 = w + o; o += ch[2 * f];
          a.hF[f].w2 = w + o; o += ch[2 * f + 1];
        }
      }
    }
    const int R = radius_of(g_opt.order_override ? g_opt.order_override : g_order);
    TmGeom tg;
    memset(&tg, 0, sizeof(tg));
    if (tm2d) tg = tm_layout(g);
    K3Geom kg;
    memset(&kg, 0, sizeof(kg));
    std::vector<char> src_any, rcv_any;
    const unsigned char *src_rows = nullptr, *rcv_rows = nullptr;
    if (ok && a.want_src) {
      a.srcv = scratch.get<T>((size_t)g.nshot * bc.nsrc * sizeof(T));
      ok = a.srcv != nullptr;
      if (ok) cudaMemsetAsync(a.srcv, 0, (size_t)g.nshot * bc.nsrc * sizeof(T), st);
    }
    if (ok) {
      const bool rx_on = bc.rx_comp >= 0 && bc.rx_comp <= 2;
      ok = build_points(a.want_src ? bc.src_loc : nullptr, bc.nsrc, rx_on ? bc.rx_loc : nullptr, bc.ndata, g, st,
                        scratch, &P.src, &a.src, &P.rcv, &a.rcv, &src_rows, &rcv_rows, tm2d ? &src_any : nullptr,
                        tm2d ? &rcv_any : nullptr);
    }
    tg.src_rows = src_rows;
    tg.rcv_rows = rcv_rows;
    // rows with a receiver or source of any shot go to the general (frame) kernels
    std::vector<char> pt_rows(tm2d ? g.NX : 0, 0);
    for (int i = 0; i < (int)pt_rows.size(); ++i)
      pt_rows[i] = (i < (int)src_any.size() && src_any[i]) || (i < (int)rcv_any.size() && rcv_any[i]);
    const long long ncell_ext = (long long)(g.NX - 1) * (g.NY - 1) * (g.NZ - 1);
    if (ok && want_model && a.acc64) {
      a.g_eps64 = scratch.get<double>((size_t)ncell_ext * sizeof(double));
      a.g_sig64 = scratch.get<double>((size_t)ncell_ext * sizeof(double));
      ok = !scratch.failed;
      if (ok) {
        cudaMemsetAsync(a.g_eps64, 0, (size_t)ncell_ext * sizeof(double), st);
        cudaMemsetAsync(a.g_sig64, 0, (size_t)ncell_ext * sizeof(double), st);
      }
    }
    if (ok) ok = launch_coeffs(cm, st);
    TmBuf<T> tl;
    memset(&tl, 0, sizeof(tl));
    const long long plane2 = (long long)g.NX * tg.NYP;
    if (ok && tm2d) {
      const int ncoef = cm.dy == cm.dx ? 5 : 7;
      T* buf = scratch.get<T>(((size_t)(3 * g.nshot + ncoef) * plane2 + kTmTailPad) * sizeof(T));
      ok = buf != nullptr;
      if (ok) {
        tl.Ez = buf;
        tl.Hx = buf + g.nshot * plane2;
        tl.Hy = buf + 2 * g.nshot * plane2;
        T* cf = buf + 3 * g.nshot * plane2;
        const T* srcs[5] = {cm.ce_hist, cm.ce_curl, cm.ce_rhs, cm.ch_curl, cm.ch_rhs};
        for (int q = 0; q < 5; ++q) k_pack2d_pitch<T><<<1024, 256, 0, st>>>(srcs[q], cf + q * plane2, g.NX, g.NY, tg.NYP);
        tl.ce_hist = cf;
        tl.ce_curl = cf + plane2;
        tl.ce_rhs = cf + 2 * plane2;
        tl.ch_curl = cf + 3 * plane2;
        tl.ch_rhs = cf + 4 * plane2;
        tl.ce_curl_y = tl.ce_curl;
        tl.ch_curl_y = tl.ch_curl;
        if (ncoef == 7) {
          k_pack2d_pitch_ys<T><<<1024, 256, 0, st>>>(cm.ce_curl, cf + 5 * plane2, g.NX, g.NY, tg.NYP, cm.dx, cm.dy);
          k_pack2d_pitch_ys<T><<<1024, 256, 0, st>>>(cm.ch_curl, cf + 6 * plane2, g.NX, g.NY, tg.NYP, cm.dx, cm.dy);
          tl.ce_curl_y = cf + 5 * plane2;
          tl.ch_curl_y = cf + 6 * plane2;
        }
        cudaMemsetAsync(cf + ncoef * plane2, 0, kTmTailPad * sizeof(T), st);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(bc.lEz, tl.Ez, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(bc.lHx, tl.Hx, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_pack2d_pitch<T><<<2048, 256, 0, st>>>(bc.lHy, tl.Hy, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        ok = cuda_ok(cudaGetLastError(), "pack");
      }
    }
    // 3D: lambda and coefficients in the z-pitched working copy
    K3Buf<T> kb;
    memset(&kb, 0, sizeof(kb));
    if (ok && !tm2d) {
      kg = k3_layout(g, 8);
      kg.src_rows = src_rows;
      kg.rcv_rows = rcv_rows;
      kg.cpml_single = k3_cpml_single(g, cm.p);
      ok = k3_alloc_pack(scratch, g, kg, cm, st, kb, bc.lEx, bc.lEy, bc.lEz, bc.lHx, bc.lHy, bc.lHz);
    }
    const dim3 kblock(32, K3_WARPS);
    const bool eq3 = cm.dy == cm.dx && cm.dz == cm.dx;
    // general CPML form where faces of an axis may meet, or past the z-face pass's grid limit
    const bool gen3 = has_cpml && (!kg.cpml_single || g.nshot > 65535);
    // wide adjoint kernels (fdtd_3d_wide_adj.cuh) for FP32 with the single-face CPML form (or none)
    const int fam3 = k3_family();
    const bool wide3 = sizeof(T) == 4 && ok && !tm2d && !gen3 && (fam3 == 2 || fam3 < 0) &&
                       (fam3 == 2 || k3w_auto(false, k3_interior_fraction(g, cm.p), k3w_lane_use(g))) &&
                       k3w_usable(g, cm.p, has_cpml, R) && k3w_adj_ready();
    K3WGeom kwg;
    memset(&kwg, 0, sizeof(kwg));
    if (wide3) {
      kwg = k3w_layout(g, kg.zp, 12);
      kwg.src_rows = src_rows;
      kwg.rcv_rows = rcv_rows;
    }
    if (ok && !tm2d) {
      // the double-precision stages exceed the 48 KB default
      k3_variant<T>(R, eq3, gen3, [&](auto RR, auto E, auto G) {
        constexpr int r = decltype(RR)::value;
        constexpr bool e = decltype(E)::value, gn = decltype(G)::value;
        const void* fns[2] = {(const void*)k3v_adj_e<T, r, e, gn>, (const void*)k3v_adj_h<T, r, e, gn>};
        for (const void* fn : fns)
          if (ok)
            ok = cuda_ok(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k3_adj_smem_bytes<T, r>()),
                         "adjoint shared memory attribute");
      });
    }
    if (ok && cm.nt > 0) {
      a.ctrl = ctrl;
      k_set<<<1, 1, 0, st>>>(ctrl, cm.nt - 1);
      const long long tiles = tm2d ? 1 : tiles3(g);
      const dim3 wblock(32, TM_WARPS);
      const bool lean2d = tm2d && a.box.z0 == 0 && a.box.nz == 1;
      const TmFaces tfc = tm_faces(a.eF, a.hF, a.has_cpml != 0);
      TmPlan pE, pH, pP;
      if (tm2d) {
        const int bE = R == 1 ? blocks_per_sm(tmi_adj_e<T, 1>) : R == 2 ? blocks_per_sm(tmi_adj_e<T, 2>)
                                                                        : blocks_per_sm(tmi_adj_e<T, 4>);
        const int bH = R == 1 ? blocks_per_sm(tmi_adj_h<T, 1>) : R == 2 ? blocks_per_sm(tmi_adj_h<T, 2>)
                                                                        : blocks_per_sm(tmi_adj_h<T, 4>);
        pE = tm_plan(tg, g, 2, R, tfc, lean2d, bE);
        pE.frame.sum_source = 1;   // the adjoint-E frame launch sums the step's source gradient
        pH = tm_plan(tg, g, 3, R, tfc, lean2d, bH, &pt_rows);
        pP = tm_plan(tg, g, 3, R, tfc, false, bH);   // prologue: general kernel everywhere
      }
      P.xchunk = pick_xchunk(g.NX, tiles, g.nshot, 4 * R);
      dim3 grid((unsigned)tiles, (unsigned)((g.NX + P.xchunk - 1) / P.xchunk), (unsigned)g.nshot);
      const unsigned img_blocks = (unsigned)((a.box.cells() + 255) / 256);
      // head of step nt-1
      {
        TiledAdj<T> b = P;
        b.a.k_in_chunk = 0;
        if (tm2d) {
          const TmGeom& fP = pP.frame;
          const dim3 gP = tm_grid(fP);
          if (R == 1) tm_adj_h<T, 1, true><<<gP, wblock, 0, st>>>(b, tl, fP);
          else if (R == 2) tm_adj_h<T, 2, true><<<gP, wblock, 0, st>>>(b, tl, fP);
          else tm_adj_h<T, 4, true><<<gP, wblock, 0, st>>>(b, tl, fP);
        } else {
          k3v_adj_head<T><<<(unsigned)kg.nblocks, kblock, 0, st>>>(b, kb, kg);
        }
        ok = cuda_ok(cudaGetLastError(), "adjoint prologue");
      }
      auto issue = [&](int k) {
        TiledAdj<T> b = P;
        b.a.k_in_chunk = k;
        // The imaging of step it reads lambda_E (which the adjoint E step only
        // reads) and the history, and writes the gradient sums: outside kernel
        // timing it runs on the second side stream beside the adjoint E step,
        // and the adjoint H step (which writes lambda_E) waits for it.
        const bool img = want_model && img_blocks > 0;
        const bool img_side = img && !g_prof.on && ss != nullptr && ss->side2 != nullptr;
        cudaStream_t ist = st;
        if (img_side) {
          cudaEventRecord(ss->fork2, st);
          cudaStreamWaitEvent(ss->side2, ss->fork2, 0);
          ist = ss->side2;
        }
        if (img) {
          if (tm2d)
            timed(KK_IMAGE, st, [&] { launch_tm_image<T>(kind, a.e_only != 0, a.acc64 != 0, ist, b.a, tl.Ez, tg); });
          else
            timed(KK_IMAGE, st, [&] {
              const long long ls = (long long)g.NX * g.NY * kg.zp;
              if (a.box.cells() < (1LL << 31))
                launch_k3_image<T>(kind, a.e_only != 0, a.acc64 != 0, cm.mode, ist, b.a, kb, ls, g.NY * kg.zp, kg.zp);
              else
                k_image<T><<<img_blocks, 256, 0, ist>>>(b.a, kb.Ex, kb.Ey, kb.Ez, ls, g.NY * kg.zp, kg.zp);
            });
        }
        if (img_side) cudaEventRecord(ss->join2, ss->side2);
        if (tm2d) {
          timed(KK_ADJ_E, st, [&] {
            return tm_launch(
                st, ss, pE,
                [&](dim3 gfu, unsigned nfb) {
                  if (R == 1) tmf_adj_e<T, 1><<<gfu, wblock, 0, st>>>(b, tl, pE.frame, pE.interior, nfb);
                  else if (R == 2) tmf_adj_e<T, 2><<<gfu, wblock, 0, st>>>(b, tl, pE.frame, pE.interior, nfb);
                  else tmf_adj_e<T, 4><<<gfu, wblock, 0, st>>>(b, tl, pE.frame, pE.interior, nfb);
                },
                [&](cudaStream_t q, const TmGeom& fg) {
                  const dim3 gf = tm_grid(fg);
                  if (R == 1) tm_adj_e<T, 1><<<gf, wblock, 0, q>>>(b, tl, fg);
                  else if (R == 2) tm_adj_e<T, 2><<<gf, wblock, 0, q>>>(b, tl, fg);
                  else tm_adj_e<T, 4><<<gf, wblock, 0, q>>>(b, tl, fg);
                },
                [&](cudaStream_t q) {
                  const dim3 gi = tm_grid(pE.interior);
                  if (R == 1) tmi_adj_e<T, 1><<<gi, wblock, 0, q>>>(b, tl, pE.interior);
                  else if (R == 2) tmi_adj_e<T, 2><<<gi, wblock, 0, q>>>(b, tl, pE.interior);
                  else tmi_adj_e<T, 4><<<gi, wblock, 0, q>>>(b, tl, pE.interior);
                });
          });
          if (img_side) cudaStreamWaitEvent(st, ss->join2, 0);   // the imaging read lambda_E
          timed(KK_ADJ_H, st, [&] {
            return tm_launch(
                st, ss, pH,
                [&](dim3 gfu, unsigned nfb) {
                  if (R == 1) tmf_adj_h<T, 1><<<gfu, wblock, 0, st>>>(b, tl, pH.frame, pH.interior, nfb);
                  else if (R == 2) tmf_adj_h<T, 2><<<gfu, wblock, 0, st>>>(b, tl, pH.frame, pH.interior, nfb);
                  else tmf_adj_h<T, 4><<<gfu, wblock, 0, st>>>(b, tl, pH.frame, pH.interior, nfb);
                },
                [&](cudaStream_t q, const TmGeom& fg) {
                  const dim3 gf = tm_grid(fg);
                  if (R == 1) tm_adj_h<T, 1, false><<<gf, wblock, 0, q>>>(b, tl, fg);
                  else if (R == 2) tm_adj_h<T, 2, false><<<gf, wblock, 0, q>>>(b, tl, fg);
                  else tm_adj_h<T, 4, false><<<gf, wblock, 0, q>>>(b, tl, fg);
                },
                [&](cudaStream_t q) {
                  const dim3 gi = tm_grid(pH.interior);
                  if (R == 1) tmi_adj_h<T, 1><<<gi, wblock, 0, q>>>(b, tl, pH.interior);
                  else if (R == 2) tmi_adj_h<T, 2><<<gi, wblock, 0, q>>>(b, tl, pH.interior);
                  else tmi_adj_h<T, 4><<<gi, wblock, 0, q>>>(b, tl, pH.interior);
                });
          });
        } else {
          const unsigned nb = (unsigned)kg.nblocks;
          // single-face form: the CPML weights in their own pass after each kernel
          const bool zpass = sizeof(T) == 4 && has_cpml && !gen3;
          const K3Faces fh = k3_faces(g, cm.p, false), fe = k3_faces(g, cm.p, true);
          const dim3 gph((fh.cum[5] + kBlock - 1) / kBlock, (unsigned)g.nshot);
          const dim3 gpe((fe.cum[5] + kBlock - 1) / kBlock, (unsigned)g.nshot);
          timed(KK_ADJ_E, st, [&] {
            if constexpr (sizeof(T) == 4) {
              if (wide3) k3w_adj_launch<0>(R, eq3, st, b, kb, kwg);
            }
            if (!wide3) {
              k3_variant<T>(R, eq3, gen3, [&](auto RR, auto E, auto G) {
                constexpr int r = decltype(RR)::value;
                k3v_adj_e<T, r, decltype(E)::value, decltype(G)::value>
                    <<<nb, kblock, k3_adj_smem_bytes<T, r>(), st>>>(b, kb, kg);
              });
            }
            if (zpass) k3p_adj_w<T, false><<<gph, kBlock, 0, st>>>(b, kb, kg, fh);
            return zpass ? 2 : 1;
          });
          if (img_side) cudaStreamWaitEvent(st, ss->join2, 0);   // the imaging read lambda_E
          timed(KK_ADJ_H, st, [&] {
            if constexpr (sizeof(T) == 4) {
              if (wide3) k3w_adj_launch<1>(R, eq3, st, b, kb, kwg);
            }
            if (!wide3) {
              k3_variant<T>(R, eq3, gen3, [&](auto RR, auto E, auto G) {
                constexpr int r = decltype(RR)::value;
                k3v_adj_h<T, r, decltype(E)::value, decltype(G)::value>
                    <<<nb, kblock, k3_adj_smem_bytes<T, r>(), st>>>(b, kb, kg);
              });
            }
            if (zpass) k3p_adj_w<T, true><<<gpe, kBlock, 0, st>>>(b, kb, kg, fe);
            return zpass ? 2 : 1;
          });
        }
      };
      // host-resident histories (use_async_offload): staged into device rings ahead of use
      HistRing hr;
      const ThreadOptions saved_opt = g_opt;
      const bool off_e = want_model && is_host_memory(bc.E_saved);
      const bool off_r = want_model && !e_only && is_host_memory(bc.R_saved);
      if (ok && (off_e || off_r)) {
        if (is_tiled(kind)) {
          set_error("backward: one-byte (FP8 / INT8) histories stay on the device (no offload)");
          ok = false;
        } else {
          g_opt.use_graph = 0;
          g_opt.chunk = std::max(g_opt.chunk, 32);
          ok = hr.setup(scratch, st, off_e ? const_cast<void*>(bc.E_saved) : nullptr,
                        off_r ? const_cast<void*>(bc.R_saved) : nullptr, cm.S, cm.nt, a.nt_saved, ncomp, a.frame,
                        hist_elem_bytes(kind), g_opt.chunk, e_only ? 1 : 0);
        }
      }
      const int clen = std::max(1, g_opt.chunk);
      // stages reverse chunk c (steps from nt-1-c*clen downwards) into buffer c & 1
      auto stage_chunk = [&](int c) -> bool {
        const int t = c * clen;
        if (t >= cm.nt) return true;
        int s0, s1;
        hr.bwd_slots(t, std::min(clen, cm.nt - t), s0, s1);
        const int b = c & 1;
        if (!hr.move(b, s0, s1, false)) return false;
        hr.pending[b] = true;
        return cuda_ok(cudaEventRecord(hr.done[b], hr.copy), "offload event");
      };
      if (ok && hr.on) {
        // the copy stream starts after everything the call enqueued so far
        ok = cuda_ok(cudaEventRecord(hr.work[0], st), "offload event") &&
             cuda_ok(cudaStreamWaitEvent(hr.copy, hr.work[0], 0), "offload wait") && stage_chunk(0) && stage_chunk(1);
      }
      auto bhook = [&](int t, int K, int phase) -> bool {
        if (!hr.on) return true;
        const int c = t / clen, b = c & 1;
        if (phase == 0) {
          int s0, s1;
          hr.bwd_slots(t, K, s0, s1);
          if (!cuda_ok(cudaStreamWaitEvent(st, hr.done[b], 0), "offload wait")) return false;
          if (hr.host[0]) a.E_saved = hr.base(0, b, s0);
          if (hr.host[1]) a.R_saved = hr.base(1, b, s0);
          a.comp_stride = hr.comp_stride();
          return true;
        }
        // buffer b is free once the work stream passes this point: stage chunk c + 2 into it
        return cuda_ok(cudaEventRecord(hr.work[b], st), "offload event") &&
               cuda_ok(cudaStreamWaitEvent(hr.copy, hr.work[b], 0), "offload wait") && stage_chunk(c + 2);
      };
      if (ok) ok = run_loop(cm.nt, -1, ctrl, st, issue, bhook);
      if (hr.on) {
        for (int b = 0; b < 2; ++b)
          if (hr.pending[b]) cudaStreamWaitEvent(st, hr.done[b], 0);
        a.E_saved = bc.E_saved;
        a.R_saved = bc.R_saved;
        a.comp_stride = (long long)a.nt_saved * a.frame;
      }
      g_opt = saved_opt;
      if (ok && !tm2d) ok = k3_unpack(g, kg, st, kb, bc.lEx, bc.lEy, bc.lEz, bc.lHx, bc.lHy, bc.lHz);
      if (ok && tm2d) {
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tl.Ez, bc.lEz, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tl.Hx, bc.lHx, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        k_unpack2d_pitch<T><<<2048, 256, 0, st>>>(tl.Hy, bc.lHy, (long long)g.nshot * g.NX, g.NY, tg.NYP);
        ok = cuda_ok(cudaGetLastError(), "unpack");
      }
      if (ok && want_model && a.acc64) {
        if (a.want_eps) k_fold_acc64<T><<<1024, 256, 0, st>>>(bc.grad_eps, a.g_eps64, ncell_ext);
        if (a.want_sig) k_fold_acc64<T><<<1024, 256, 0, st>>>(bc.grad_sig, a.g_sig64, ncell_ext);
        ok = cuda_ok(cudaGetLastError(), "gradient fold");
      }
    }
  }
  cudaEventRecord(ss->out, st);
  cudaStreamWaitEvent(user, ss->out, 0);
  if (ok) cuda_ok(cudaGetLastError(), "backward");
}


Grid make_grid(int NX, int NY, int NZ, int nshot) {
  Grid g;
  g.NX = NX;
  g.NY = NY;
  g.NZ = NZ;
  g.sx = NY * NZ;
  g.cells = NX * NY * NZ;
  g.nshot = nshot;
  // Split shots over gridDim.y only when one shot does not fill the GPU.
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long target = (long long)sms * 8 * kBlock;  // threads for a full machine
  int groups = 1;
  if (g.cells > 0 && (long long)g.cells < target) groups = (int)std::min<long long>(nshot, target / g.cells + 1);
  groups = std::max(1, std::min(groups, kMaxShotGroups));
  g.shots_per_group = (nshot + groups - 1) / groups;
  return g;
}

}  // namespace

// ===========================================================================
// Exported symbols.
// ===========================================================================

// Parameter lists shared by the FP32 ABI-6 entry points and the FP64
// extensions (src/DeepGPR/lib/deepgpr.h:89-152, same order and meaning).
#define DGB_FWD_PARAMS(T)                                                                                       \
  const T *eps_r_pad, const T *sigma_pad, const T *mu_r_pad, void *E_saved, void *R_saved, T *Ex, T *Ey,       \
      T *Ez, T *Hx, T *Hy, T *Hz, T *ce_hist, T *ce_curl, T *ce_rhs, T *ch_hist, T *ch_curl, T *ch_rhs,        \
      T *x0e1, T *x0e2, T *x0h1, T *x0h2, T *xme1, T *xme2, T *xmh1, T *xmh2, T *y0e1, T *y0e2, T *y0h1,       \
      T *y0h2, T *yme1, T *yme2, T *ymh1, T *ymh2, T *z0e1, T *z0e2, T *z0h1, T *z0h2, T *zme1, T *zme2,       \
      T *zmh1, T *zmh2, int p0, int p1, int p2, int p3, int p4, int p5, const T *x0E, const T *xmE,           \
      const T *y0E, const T *ymE, const T *z0E, const T *zmE, const T *x0H, const T *xmH, const T *y0H,      \
      const T *ymH, const T *z0H, const T *zmH, T dt, int nt, int nshot, int nrx, T dx, T dy, T dz,           \
      const int *rx_loc, T *rx_out, int rx_comp, int NX, int NY, int NZ, int nsrc, const int *src_loc,        \
      const T *src_wave, int src_comp, int S, int mode, int storage_type, int save_model_history,             \
      int use_async_offload

#define DGB_BWD_PARAMS(T)                                                                                       \
  const T *eps_r_pad, const T *sigma_pad, const T *mu_r_pad, const void *E_saved, const void *R_saved,         \
      T *lex, T *ley, T *lez, T *lhx, T *lhy, T *lhz, T *ce_hist, T *ce_curl, T *ce_rhs, T *ch_hist,           \
      T *ch_curl, T *ch_rhs, T *x0e1, T *x0e2, T *x0h1, T *x0h2, T *xme1, T *xme2, T *xmh1, T *xmh2, T *y0e1,  \
      T *y0e2, T *y0h1, T *y0h2, T *yme1, T *yme2, T *ymh1, T *ymh2, T *z0e1, T *z0e2, T *z0h1, T *z0h2,       \
      T *zme1, T *zme2, T *zmh1, T *zmh2, int p0, int p1, int p2, int p3, int p4, int p5, const T *x0E,       \
      const T *xmE, const T *y0E, const T *ymE, const T *z0E, const T *zmE, const T *x0H, const T *xmH,      \
      const T *y0H, const T *ymH, const T *z0H, const T *zmH, T dt, int nt, int nshot, int nrx, T dx, T dy,   \
      T dz, int NX, int NY, int NZ, int ndata, const int *rx_loc, const T *data_grad, int rx_comp, int nsrc,  \
      const int *src_loc, int src_comp, T *grad_source, int want_src, T *grad_eps, T *grad_sig, int want_eps,  \
      int want_sig, int S, int mode, int storage_type, int use_async_offload

#define DGB_FILL_COMMON(cm)                                                                                     \
  do {                                                                                                          \
    (cm).g = make_grid(NX, NY, NZ, nshot);                                                                      \
    (cm).dx = dx; (cm).dy = dy; (cm).dz = dz; (cm).dt = dt; (cm).nt = nt;                                       \
    const int pp[6] = {p0, p1, p2, p3, p4, p5};                                                                 \
    for (int f_ = 0; f_ < 6; ++f_) (cm).p[f_] = pp[f_];                                                         \
    (cm).eps = eps_r_pad; (cm).sig = sigma_pad; (cm).mu = mu_r_pad;                                            \
    (cm).ce_hist = ce_hist; (cm).ce_curl = ce_curl; (cm).ce_rhs = ce_rhs;                                      \
    (cm).ch_hist = ch_hist; (cm).ch_curl = ch_curl; (cm).ch_rhs = ch_rhs;                                      \
    (cm).eR[0] = x0E; (cm).eR[1] = xmE; (cm).eR[2] = y0E; (cm).eR[3] = ymE; (cm).eR[4] = z0E; (cm).eR[5] = zmE; \
    (cm).hR[0] = x0H; (cm).hR[1] = xmH; (cm).hR[2] = y0H; (cm).hR[3] = ymH; (cm).hR[4] = z0H; (cm).hR[5] = zmH; \
    (cm).S = S; (cm).mode = mode; (cm).storage_type = storage_type;                                            \
  } while (0)

template <typename T>
static void forward_entry(ForwardCall<T>& fc) {
  forward_impl<T>(fc);
}

#define DGB_FORWARD_BODY(T)                                                                                     \
  ForwardCall<T> fc;                                                                                            \
  memset(&fc, 0, sizeof(fc));                                                                                   \
  DGB_FILL_COMMON(fc.cm);                                                                                       \
  T* ep[12] = {x0e1, x0e2, xme1, xme2, y0e1, y0e2, yme1, yme2, z0e1, z0e2, zme1, zme2};                         \
  T* hp[12] = {x0h1, x0h2, xmh1, xmh2, y0h1, y0h2, ymh1, ymh2, z0h1, z0h2, zmh1, zmh2};                         \
  for (int q_ = 0; q_ < 12; ++q_) { fc.cm.ePsi[q_] = ep[q_]; fc.cm.hPsi[q_] = hp[q_]; }                         \
  fc.E_saved = E_saved; fc.R_saved = R_saved;                                                                   \
  fc.Ex = Ex; fc.Ey = Ey; fc.Ez = Ez; fc.Hx = Hx; fc.Hy = Hy; fc.Hz = Hz;                                       \
  fc.nrx = nrx; fc.rx_loc = rx_loc; fc.rx = rx_out; fc.rx_comp = rx_comp;                                      \
  fc.nsrc = nsrc; fc.src_loc = src_loc; fc.wave = src_wave; fc.src_comp = src_comp;                            \
  fc.save_model_history = save_model_history;                                                                   \
  (void)use_async_offload;                                                                                      \
  forward_entry<T>(fc)

#define DGB_BACKWARD_BODY(T)                                                                                    \
  BackwardCall<T> bc;                                                                                           \
  memset(&bc, 0, sizeof(bc));                                                                                   \
  DGB_FILL_COMMON(bc.cm);                                                                                       \
  T* ep[12] = {x0e1, x0e2, xme1, xme2, y0e1, y0e2, yme1, yme2, z0e1, z0e2, zme1, zme2};                         \
  T* hp[12] = {x0h1, x0h2, xmh1, xmh2, y0h1, y0h2, ymh1, ymh2, z0h1, z0h2, zmh1, zmh2};                         \
  for (int q_ = 0; q_ < 12; ++q_) { bc.cm.ePsi[q_] = ep[q_]; bc.cm.hPsi[q_] = hp[q_]; }                         \
  bc.E_saved = E_saved; bc.R_saved = R_saved;                                                                   \
  bc.lEx = lex; bc.lEy = ley; bc.lEz = lez; bc.lHx = lhx; bc.lHy = lhy; bc.lHz = lhz;                           \
  bc.ndata = ndata; bc.rx_loc = rx_loc; bc.data_grad = data_grad; bc.rx_comp = rx_comp;                        \
  bc.nsrc = nsrc; bc.src_loc = src_loc; bc.src_comp = src_comp;                                                 \
  bc.grad_source = grad_source; bc.want_src = want_src;                                                         \
  bc.grad_eps = grad_eps; bc.grad_sig = grad_sig; bc.want_eps = want_eps; bc.want_sig = want_sig;              \
  (void)nrx; (void)use_async_offload;                                                                           \
  backward_impl<T>(bc)

DGB_API void forward(DGB_FWD_PARAMS(float)) { DGB_FORWARD_BODY(float); }

// forward() without device memory allocation: its scratch comes from the
// static array g_noalloc_scratch (8 MiB per device) and its time-step
// kernels are launched one by one.  See StaticScratch for the callers this
// serves, the size limit and why overlapping calls race.  Every call looks up
// the array's device address; the first call on a new thread also creates the
// library's stream and events for it: make that first call before any stream
// capture.
template <typename T>
static void forward_noalloc_entry(ForwardCall<T>& fc) {
  const int saved = g_opt.use_graph;
  g_opt.use_graph = 0;
  forward_impl<T, StaticScratch>(fc);
  g_opt.use_graph = saved;
}

DGB_API void dgb_forward_noalloc(DGB_FWD_PARAMS(float)) {
  ForwardCall<float> fc;
  memset(&fc, 0, sizeof(fc));
  DGB_FILL_COMMON(fc.cm);
  float* ep[12] = {x0e1, x0e2, xme1, xme2, y0e1, y0e2, yme1, yme2, z0e1, z0e2, zme1, zme2};
  float* hp[12] = {x0h1, x0h2, xmh1, xmh2, y0h1, y0h2, ymh1, ymh2, z0h1, z0h2, zmh1, zmh2};
  for (int q = 0; q < 12; ++q) {
    fc.cm.ePsi[q] = ep[q];
    fc.cm.hPsi[q] = hp[q];
  }
  fc.E_saved = E_saved;
  fc.R_saved = R_saved;
  fc.Ex = Ex; fc.Ey = Ey; fc.Ez = Ez; fc.Hx = Hx; fc.Hy = Hy; fc.Hz = Hz;
  fc.nrx = nrx; fc.rx_loc = rx_loc; fc.rx = rx_out; fc.rx_comp = rx_comp;
  fc.nsrc = nsrc; fc.src_loc = src_loc; fc.wave = src_wave; fc.src_comp = src_comp;
  fc.save_model_history = save_model_history;
  (void)use_async_offload;
  forward_noalloc_entry<float>(fc);
}
DGB_API void backward(DGB_BWD_PARAMS(float)) { DGB_BACKWARD_BODY(float); }
DGB_API void dgb_forward_f64(DGB_FWD_PARAMS(double)) { DGB_FORWARD_BODY(double); }
DGB_API void dgb_backward_f64(DGB_BWD_PARAMS(double)) { DGB_BACKWARD_BODY(double); }

// Exhaustive check of div_fixed against the division operator for one divisor.
__global__ void k_check_fixed_div(FixedDiv<float> d, unsigned long long* bad, unsigned* first) {
  const unsigned long long nth = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long cnt = 0;
  unsigned lowest = 0xffffffffu;
  for (unsigned long long u = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; u < (1ull << 32); u += nth) {
    const float a = __uint_as_float((unsigned)u);
    if (__float_as_uint(div_fixed(a, d)) != __float_as_uint(a / d.b)) {
      ++cnt;
      lowest = min(lowest, (unsigned)u);
    }
  }
  if (cnt) {
    atomicAdd(bad, cnt);
    atomicMin(first, lowest);
  }
}

// Diagnostic: the number of float dividends (all 2^32 bit patterns) whose
// correctly rounded division by `divisor` through the solver's fixed-divisor
// path differs from the division operator, and the lowest such bit pattern.
// Runs synchronously on the current device; returns 0, or -1 with the error.
DGB_API int dgb_check_fixed_division(float divisor, unsigned long long* mismatches, unsigned* first_bad) {
  void* buf = nullptr;
  if (!cuda_ok(cudaMalloc(&buf, 16), "dgb_check_fixed_division: cudaMalloc")) return -1;
  unsigned long long* bad = static_cast<unsigned long long*>(buf);
  unsigned* first = reinterpret_cast<unsigned*>(bad + 1);
  const unsigned init[4] = {0u, 0u, 0xffffffffu, 0u};
  bool ok = cuda_ok(cudaMemcpy(buf, init, 16, cudaMemcpyHostToDevice), "dgb_check_fixed_division: upload");
  if (ok) {
    k_check_fixed_div<<<sm_count() * 8, 256>>>(fixed_div(divisor), bad, first);
    ok = cuda_ok(cudaGetLastError(), "dgb_check_fixed_division: launch");
  }
  unsigned out[4] = {0u, 0u, 0u, 0u};
  if (ok) ok = cuda_ok(cudaMemcpy(out, buf, 16, cudaMemcpyDeviceToHost), "dgb_check_fixed_division: download");
  cudaFree(buf);
  if (!ok) return -1;
  unsigned long long n = 0;
  memcpy(&n, out, sizeof(n));
  if (mismatches) *mismatches = n;
  if (first_bad) *first_bad = out[2];
  return 0;
}

// Scratch retention: the solver's per-call scratch comes from the current
// device's default stream-ordered memory pool.  The library keeps up to
// min(4 GiB, 1/32 of the device memory) of freed scratch cached in it (see
// default_retention); a caller sets `bytes` instead (-1: no limit; 0: the
// CUDA default, every synchronisation returns freed memory to the system,
// and the pool is trimmed now).
DGB_API int dgb_set_scratch_retention(long long bytes) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "dgb_set_scratch_retention: device")) return -1;
  if (dev >= 0 && dev < kMaxDevices) g_retention_set[dev] = true;
  cudaMemPool_t pool;
  if (!cuda_ok(cudaDeviceGetDefaultMemPool(&pool, dev), "dgb_set_scratch_retention: pool")) return -1;
  unsigned long long v = bytes < 0 ? ~0ULL : (unsigned long long)bytes;   // the attribute is a 64-bit unsigned
  if (!cuda_ok(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &v),
               "dgb_set_scratch_retention: release threshold"))
    return -1;
  if (bytes == 0 && !cuda_ok(cudaMemPoolTrimTo(pool, 0), "dgb_set_scratch_retention: trim")) return -1;
  return 0;
}

// Diagnostic: bytes in use in the current device's default stream-ordered
// memory pool (the pool cudaMallocAsync draws on), and its high-water mark
// since the last reset; reset_high != 0 first resets the mark to the current
// use.  Returns 0, or -1 with the error.
DGB_API int dgb_default_pool_usage(long long* used, long long* high, int reset_high) {
  int dev = 0;
  if (!cuda_ok(cudaGetDevice(&dev), "dgb_default_pool_usage: device")) return -1;
  cudaMemPool_t pool;
  if (!cuda_ok(cudaDeviceGetDefaultMemPool(&pool, dev), "dgb_default_pool_usage: pool")) return -1;
  unsigned long long u = 0, h = 0;
  if (reset_high) {
    unsigned long long zero = 0;
    if (!cuda_ok(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero), "dgb_default_pool_usage: reset"))
      return -1;
  }
  if (!cuda_ok(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u), "dgb_default_pool_usage: used") ||
      !cuda_ok(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &h), "dgb_default_pool_usage: high"))
    return -1;
  if (used) *used = (long long)u;
  if (high) *high = (long long)h;
  return 0;
}

DGB_API int deepgpr_abi_version(void) { return 6; }
DGB_API int deepgpr_supports_error_reporting(void) { return 1; }
DGB_API const char* deepgpr_last_error(void) { return g_error; }
DGB_API void deepgpr_clear_last_error(void) { g_error[0] = '\0'; }
DGB_API void deepgpr_clear_cuda_resource_cache(void) { g_error[0] = '\0'; }
DGB_API int deepgpr_deterministic_adjoint(void) { return 1; }
DGB_API int deepgpr_supports_external_pml(void) { return 1; }
DGB_API int deepgpr_supports_pml_material_gradients(void) { return 1; }
DGB_API int deepgpr_supports_int8_wavefield(void) { return 0; }
DGB_API int deepgpr_supports_conversion_backends(void) { return 0; }
DGB_API int deepgpr_supports_int8_reduction_backends(void) { return 0; }
DGB_API int deepgpr_supports_rhs_reconstruction(void) { return 1; }
DGB_API int deepgpr_supports_physical_history(void) { return 1; }
DGB_API int deepgpr_supports_tm2d_fast_path(void) { return 1; }
DGB_API void set_fdtd_order(int order) { g_order = (order == 4 || order == 8) ? order : 2; }

DGB_API int dgb_version(void) { return 1; }

// Kernel timing of the calling thread: enable/disable (clears the totals on
// enable) and read the per-kind totals (fwd_h, fwd_e, adj_e, adj_h, image).
DGB_API void dgb_profile(int enable) {
  std::lock_guard<std::mutex> lock(g_prof.mu);
  if (enable)
    for (int k = 0; k < KK_COUNT; ++k) {
      g_prof.ms[k] = 0.0;
      g_prof.launches[k] = 0;
    }
  g_prof.on = enable != 0;
}

// Time-step kernels launched through the library so far, all threads
// (graph replays count every kernel node).
DGB_API long long dgb_launch_count(void) { return g_launch_count.load(); }

DGB_API int dgb_profile_read(double* ms, long long* launches, int n) {
  std::lock_guard<std::mutex> lock(g_prof.mu);
  const int m = n < KK_COUNT ? n : KK_COUNT;
  for (int k = 0; k < m; ++k) {
    ms[k] = g_prof.ms[k];
    launches[k] = g_prof.launches[k];
  }
  return KK_COUNT;
}
DGB_API int dgb_supports_fp8_history(void) { return 1; }

DGB_API int dgb_set_stream(void* stream) {
  g_opt.user_stream = static_cast<cudaStream_t>(stream);
  g_opt.user_stream_set = true;
  return 0;
}

DGB_API void dgb_clear_stream(void) {
  g_opt.user_stream = nullptr;
  g_opt.user_stream_set = false;
}

// Launch-shape choices for the calling thread's next solves (the autotuner's
// knobs): 2D interior row chunks and frame rows per warp chunk, 3D x chunks,
// 3D forward kernel family (1 staged, 0 z-streamed, -1 the environment's
// choice).  Zeros (and -1) restore the built-in heuristics.  Results do not
// depend on these choices.  Returns 0, or -1 for out-of-range values.
DGB_API int dgb_set_tuning(int tm_chunks, int tm_frame_rows, int k3_xchunks, int tma) {
  if (tm_chunks < 0 || tm_frame_rows < 0 || tm_frame_rows > 64 || k3_xchunks < 0 || tma < -1 || tma > 2) return -1;
  g_opt.tm_chunks = tm_chunks;
  g_opt.tm_frame_rows = tm_frame_rows;
  g_opt.k3_xchunks = k3_xchunks;
  g_opt.tma = tma;
  return 0;
}

DGB_API int dgb_set_options(int acc64, int chunk_steps, int use_graph, int fdtd_order) {
  if (chunk_steps < 1 || chunk_steps > 4096) return -1;
  g_opt.acc64 = acc64 ? 1 : 0;
  g_opt.chunk = chunk_steps;
  g_opt.use_graph = use_graph ? 1 : 0;
  g_opt.order_override = (fdtd_order == 2 || fdtd_order == 4 || fdtd_order == 8) ? fdtd_order : 0;
  return 0;
}

// Bytes of one history buffer (E_saved or R_saved) for a storage kind.
DGB_API long long dgb_history_bytes(int kind, int ncomp, int nt_saved, int nshot, long long box_cells,
                                    int NX, int NY, int NZ, int tm2d) {
  const long long vals = (long long)ncomp * nt_saved * nshot * box_cells;
  if (is_tiled(kind)) {
    Grid g;
    g.NX = NX; g.NY = NY; g.NZ = NZ;
    const long long tiles = fp8_tiles(g, tm2d != 0);
    return fp8_payload_bytes(vals) + (long long)ncomp * nt_saved * nshot * tiles * (long long)sizeof(float);
  }
  return vals * hist_elem_bytes(kind);
}
