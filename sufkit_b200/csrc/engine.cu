// sufgpu engine: context, device memory plan, build orchestration and the
// C ABI declared in include/sufgpu/sufgpu.h.
//
// Device layout for a build of n symbols (all coordinates 32-bit):
//   text  n+pad bytes      rank  4n (head row of each position's group; = ISA)
//   sa    4n               k0,k1 8n each (sort keys; later PHI/PLCP/LCP)
//   v0    4n               x,y   4n each (active lists, group tables, queues)
// plus look-back status words and radix histograms.  About 37n bytes in all.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cctype>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../../include/sufgpu/sufgpu.h"
#include "child.cuh"
#include "common.cuh"
#include "doubling.cuh"
#include "lcp.cuh"
#include "pack.cuh"
#include "prefixdir.cuh"
#include "crc32.cuh"
#include "fasta.cuh"
#include "radix.cuh"
#include "runs.cuh"
#include "seedsort.cuh"
#include "segsort.cuh"
#include "serve.cuh"

using namespace sufgpu;

namespace {

constexpr u64 kTextPad = 64;
constexpr u32 kMaxSegmentsPerLaunch = 8192;

struct CudaError {
  cudaError_t code;
  const char* what;
};

#define SG_CUDA(call)                                             \
  do {                                                            \
    cudaError_t sg_err_ = (call);                                 \
    if (sg_err_ != cudaSuccess) throw CudaError{sg_err_, #call};  \
  } while (0)

struct BuildError {
  sufgpu_status status;
  std::string message;
};

u64 round_up(u64 v, u64 a) { return (v + a - 1) / a * a; }

// One grown-on-demand device allocation carved into named regions.
struct Arena {
  void* base = nullptr;
  u64 bytes = 0;
  ~Arena() {
    if (base) cudaFree(base);
  }
  void reserve(u64 need) {
    if (need <= bytes) return;
    if (base) {
      cudaFree(base);
      base = nullptr;
      bytes = 0;
    }
    cudaError_t err = cudaMalloc(&base, need);
    if (err != cudaSuccess) {
      cudaGetLastError();
      base = nullptr;
      throw BuildError{SUFGPU_BUILD_FAILURE,
                       "cannot allocate " + std::to_string(need) +
                           " bytes of device memory: " + cudaGetErrorString(err)};
    }
    bytes = need;
  }
};

struct Layout {
  u8* text;
  u32* rank;
  u32* sa;
  u64* k0;
  u64* k1;
  u32* v0;
  u32* x;
  u32* y;
  u32* lcp;          // row-order LCP (seed-group heads from the seed keys)
  u64* status;       // look-back words: radix (tiles*256) or 2 scan arrays
  u64 status_words;
  u32* hist;         // radix histograms [seg][pass][256]
  u64* digit_start;  // [seg][pass][256]
  u64* seg_begin;    // count+1
  u32* seg_tiles;    // count+1
  u64* sort_begin;   // 2 entries: the active list as one sort segment
  u32* sort_tiles;   // 2 entries
  u32* counters;     // tile counters
  u64* scalars;      // device-written counts
  u32* alpha;        // 256 byte counts
  u16* code;         // 256 symbol codes (1..sigma)
  DeviceFlags* flags;
  // Long-run split (runs.cuh): boundary records, per-run and per-class
  // layout, the round lookup (sorted starts/ends) and its block bitmap.
  u64 run_cap;
  u64* run_starts;
  u64* run_ends;
  RunRecord* run_recs;
  RunClass* run_classes;
  u32* run_len;
  u64* run_prefix;
  u32* run_a;
  u32* run_e;
  u32* run_bitmap;
  u64 run_bitmap_words;
  u64 total;
};

// Most long runs one build splits directly (more are left to the rounds).
u64 run_capacity(u64 n) { return std::min<u64>(u64(1) << 17, n / 8 + 64); }

Layout plan_layout(u8* base, u64 n, u32 segments) {
  Layout l{};
  u64 off = 0;
  auto take = [&](u64 bytes) {
    u8* p = base + off;
    off += round_up(bytes, 256);
    return p;
  };
  const u64 n4 = std::max<u64>(n, 1) * 4;
  l.text = take(n + kTextPad);
  l.rank = reinterpret_cast<u32*>(take(n4));
  l.sa = reinterpret_cast<u32*>(take(n4));
  l.k0 = reinterpret_cast<u64*>(take(2 * n4));
  l.k1 = reinterpret_cast<u64*>(take(2 * n4));
  l.v0 = reinterpret_cast<u32*>(take(n4));
  l.x = reinterpret_cast<u32*>(take(n4));
  l.y = reinterpret_cast<u32*>(take(n4));
  l.lcp = reinterpret_cast<u32*>(take(n4));
  const u64 radix_tiles = (n + 2047) / 2048 + segments;  // smallest tile size
  const u64 scan_tiles = (n + kScanTile - 1) / kScanTile + 1;
  l.status_words = std::max<u64>(radix_tiles * kRadixDigits, 2 * scan_tiles);
  l.status = reinterpret_cast<u64*>(take(l.status_words * 8));
  l.hist = reinterpret_cast<u32*>(take(u64(segments) * kMaxPasses * kRadixDigits * 4));
  l.digit_start = reinterpret_cast<u64*>(take(u64(segments) * kMaxPasses * kRadixDigits * 8));
  l.seg_begin = reinterpret_cast<u64*>(take(u64(segments + 1) * 8));
  l.seg_tiles = reinterpret_cast<u32*>(take(u64(segments + 1) * 4));
  l.sort_begin = reinterpret_cast<u64*>(take(16));
  l.sort_tiles = reinterpret_cast<u32*>(take(8));
  l.counters = reinterpret_cast<u32*>(take(64 * 4));
  l.scalars = reinterpret_cast<u64*>(take(64 * 8));
  l.alpha = reinterpret_cast<u32*>(take(256 * 4));
  l.code = reinterpret_cast<u16*>(take(512));
  l.flags = reinterpret_cast<DeviceFlags*>(take(sizeof(DeviceFlags)));
  l.run_cap = run_capacity(n);
  l.run_starts = reinterpret_cast<u64*>(take(l.run_cap * 8));
  l.run_ends = reinterpret_cast<u64*>(take(l.run_cap * 8));
  l.run_recs = reinterpret_cast<RunRecord*>(take(l.run_cap * sizeof(RunRecord)));
  l.run_classes = reinterpret_cast<RunClass*>(take(2 * l.run_cap * sizeof(RunClass)));
  l.run_len = reinterpret_cast<u32*>(take(l.run_cap * 4));
  l.run_prefix = reinterpret_cast<u64*>(take(3 * l.run_cap * 8));
  l.run_a = reinterpret_cast<u32*>(take(l.run_cap * 4));
  l.run_e = reinterpret_cast<u32*>(take(l.run_cap * 4));
  l.run_bitmap_words = ((std::max<u64>(n, 1) - 1) >> kRunBlockBits) / 32 + 1;
  l.run_bitmap = reinterpret_cast<u32*>(take(l.run_bitmap_words * 4));
  l.total = off;
  return l;
}

using OnesweepFn = void (*)(const u64*, const u32*, u64*, u32*, SortSegments, u32, u32, u32,
                            const u64*, u64*, u32*, DeviceFlags*);

// Onesweep variants: ranking by ballots or match-any, 256x16 or 512x8 tiles,
// key-value pairs or keys only.
struct OnesweepVariant {
  OnesweepFn fn;
  u32 block;
  u64 smem;
};

template <bool kBallot, int kBlock, int kItems, bool kVals>
OnesweepVariant variant_of() {
  return {radix_onesweep_kernel<kBallot, kBlock, kItems, kVals>, kBlock,
          sizeof(OnesweepSmem<kBlock, kBlock * kItems, kVals>)};
}

template <bool kBallot, bool kVals>
OnesweepVariant variant_for(u32 block, u32 tile) {
  if (tile == 2048) return variant_of<kBallot, 256, 8, kVals>();
  return block == 512 ? variant_of<kBallot, 512, 8, kVals>() : variant_of<kBallot, 256, 16, kVals>();
}

// Onesweep variants: ranking by ballots or match-any; 4096-key tiles (256x16,
// 512x8) or 2048-key tiles (256x8); key-value pairs or keys only.  tma: the
// 256x16 tile's keys by one bulk copy (single-segment sorts only).
// Measured on B200 (one 8-bit pass over 10^9 random keys): pairs 8.7 ms as
// 256x16 (three blocks per SM) against 9.5 ms as 512x8; keys only 7.4 ms as
// 512x8 (three blocks) against 7.6 ms as 256x16 alone, but within 2% the
// other way round inside whole builds, where 256x16 stays the default.
OnesweepVariant onesweep_variant(bool ballot, u32 block, u32 tile, bool vals, bool tma = false) {
  if (tma && tile == 4096 && block == 256) {
    const u64 smem = vals ? sizeof(OnesweepSmem<256, 4096, true>) : sizeof(OnesweepSmem<256, 4096, false>);
    if (ballot) {
      return vals ? OnesweepVariant{radix_onesweep_kernel<true, 256, 16, true, true>, 256, smem}
                  : OnesweepVariant{radix_onesweep_kernel<true, 256, 16, false, true>, 256, smem};
    }
    return vals ? OnesweepVariant{radix_onesweep_kernel<false, 256, 16, true, true>, 256, smem}
                : OnesweepVariant{radix_onesweep_kernel<false, 256, 16, false, true>, 256, smem};
  }
  if (ballot) return vals ? variant_for<true, true>(block, tile) : variant_for<true, false>(block, tile);
  return vals ? variant_for<false, true>(block, tile) : variant_for<false, false>(block, tile);
}

// Build knobs.  Results are identical for every setting; only speed changes.
struct Tuning {
  // Symbols per seed key (0 = chosen from the instance size and entropy).
  u32 seed_symbols = 0;
  // Onesweep ranking: ballots over digit bits (true) or match-any (false).
  bool ballot_rank = true;
  // Ballot ranking only pays off on large sorts; smaller ones use match-any.
  u64 ballot_min_elems = u64(1) << 23;
  // Largest instance index width for the packed (keys-only) seed; 0 = never.
  u32 packed_max_bits = 24;
  // Split long single-symbol runs directly after the seed (runs.cuh).
  bool run_split = true;
  // Sort each round's groups in shared memory (segsort.cuh).
  bool seg_sort = true;
  // With seg_sort: the shared-memory sort also writes the round's SA rows,
  // ranks and next active list (seg_rank_kernel) instead of leaving sorted
  // keys to round_rank.
  bool seg_rank = false;
  // Rank write of one instance through 2^16-position windows held by a
  // cluster of 2 or 4 blocks (cluster_window_scatter_kernel,
  // cluster4_window_scatter_kernel) when that saves a grouping pass over
  // 2048-position windows; 0: never.
  u32 rank_cluster = 2;
  // Round sort blocks per SM the kernel's registers are capped for (2 or 3;
  // measured at 3.1 Gbp: 33.3 ms at three against 37.5 ms at two).
  u32 seg_blocks = 3;
  // Seed histograms with kSeedCountRun keys per thread when the fused first
  // pass writes the keys (instead of kSeedRun).
  bool seed_count_run = true;
  // Batches write ranks through 2^16-position windows per instance held by
  // clusters of two blocks (one grouping pass) instead of window slots.
  bool batch_cluster = true;
  // Run the rounds as captured CUDA graphs of two rounds (needs seg_sort;
  // builds with the per-kernel profile on are driven round by round).
  bool graph_rounds = true;
  // Onesweep block size (256 threads x 16 keys or 512 x 8) for key-value
  // sorts and for keys-only sorts (4096-key tiles).
  u32 sort_block = 256;
  u32 keys_sort_block = 256;
  // Keys per onesweep tile (2048 or 4096).
  u32 sort_tile = 4096;
  // Two-bit seed keys for single DNA-like texts of at least two_bit_min
  // symbols (rare symbols placed from a side list).
  bool two_bit_seed = true;
  u64 two_bit_min = u64(1) << 22;
  // Seed rank write by window slots (rank_slot kernels) instead of radix
  // passes grouping the pairs by window: 0 never, 1 batches only, 2 always.
  // Measured on B200: slots win for batches of bacterial references (the
  // grouping passes there run per instance) and lose for single texts of
  // 100 Mbp and more (atomic throughput).
  u32 rank_slots = 1;
  // Round sort tiles whose groups have at most this many rows rank by
  // counting inside each group (0: always the shared-memory radix passes).
  u32 seg_small_group = kSegSmallGroup;
  // Onesweep tiles of single-segment sorts loaded by one bulk (TMA) copy.
  bool tma_tile = false;
  // Two-bit seed keys for batches too (per-instance rare lists).
  bool two_bit_batch = true;
  // Seed keys of one instance generated by the kernel that also does the
  // first radix pass (seedsort.cuh) instead of written in position order.
  bool seed_fused = true;
  // Round compaction: the graph rounds switch to a graph captured for a
  // smaller power-of-two bound once the active count falls below
  // bound / graph_shrink (kernels are launched for the bound).
  u32 graph_shrink = 4;
};

// Overrides for builds whose longest instance has at most max_symbols symbols.
struct TuningClass {
  u64 max_symbols;
  std::vector<std::pair<std::string, int64_t>> settings;
};

// Applies one knob; returns an error message or an empty string.
std::string apply_tuning(Tuning& t, const std::string& k, int64_t value) {
  if (k == "seed_symbols") {
    if (value < 0 || value > 64) return "seed_symbols out of range";
    t.seed_symbols = static_cast<u32>(value);
  } else if (k == "ballot_rank") {
    t.ballot_rank = value != 0;
  } else if (k == "ballot_min_elems") {
    if (value < 0) return "ballot_min_elems must be >= 0";
    t.ballot_min_elems = static_cast<u64>(value);
  } else if (k == "packed_max_bits") {
    if (value < 0 || value > 32) return "packed_max_bits out of range";
    t.packed_max_bits = static_cast<u32>(value);
  } else if (k == "sort_tile") {
    if (value != 2048 && value != 4096) return "sort_tile must be 2048 or 4096";
    t.sort_tile = static_cast<u32>(value);
  } else if (k == "seg_sort") {
    t.seg_sort = value != 0;
  } else if (k == "seg_rank") {
    t.seg_rank = value != 0;
  } else if (k == "rank_cluster") {
    if (value != 0 && value != 2 && value != 4) return "rank_cluster must be 0, 2 or 4";
    t.rank_cluster = static_cast<u32>(value);
  } else if (k == "batch_cluster") {
    t.batch_cluster = value != 0;
  } else if (k == "seed_count_run") {
    t.seed_count_run = value != 0;
  } else if (k == "seg_blocks") {
    if (value != 2 && value != 3) return "seg_blocks must be 2 or 3";
    t.seg_blocks = static_cast<u32>(value);
  } else if (k == "graph_rounds") {
    t.graph_rounds = value != 0;
  } else if (k == "run_split") {
    t.run_split = value != 0;
  } else if (k == "two_bit_seed") {
    t.two_bit_seed = value != 0;
  } else if (k == "two_bit_min") {
    if (value < 0) return "two_bit_min must be >= 0";
    t.two_bit_min = static_cast<u64>(value);
  } else if (k == "seg_small_group") {
    if (value < 0 || value > 4096) return "seg_small_group must be in [0, 4096]";
    t.seg_small_group = static_cast<u32>(value);
  } else if (k == "tma_tile") {
    t.tma_tile = value != 0;
  } else if (k == "two_bit_batch") {
    t.two_bit_batch = value != 0;
  } else if (k == "seed_fused") {
    t.seed_fused = value != 0;
  } else if (k == "graph_shrink") {
    if (value < 2 || value > 1024) return "graph_shrink must be in [2, 1024]";
    t.graph_shrink = static_cast<u32>(value);
  } else if (k == "rank_slots") {
    if (value < 0 || value > 2) return "rank_slots must be 0, 1 or 2";
    t.rank_slots = static_cast<u32>(value);
  } else if (k == "sort_block") {
    if (value != 256 && value != 512) return "sort_block must be 256 or 512";
    t.sort_block = static_cast<u32>(value);
  } else if (k == "keys_sort_block") {
    if (value != 256 && value != 512) return "keys_sort_block must be 256 or 512";
    t.keys_sort_block = static_cast<u32>(value);
  } else {
    return "unknown tuning key " + k;
  }
  return {};
}

}  // namespace

struct PendingLaunch {
  const char* name;
  u64 bytes;
  cudaEvent_t before, after;
};

struct KernelTotals {
  std::string name;
  u64 launches = 0;
  double seconds = 0;
  u64 bytes = 0;
};

// Reusable CUDA events for the per-kernel profile.
struct EventPool {
  std::vector<cudaEvent_t> all;
  size_t next = 0;
  cudaEvent_t take() {
    if (next == all.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) throw CudaError{cudaErrorMemoryAllocation, "cudaEventCreate"};
      all.push_back(e);
    }
    return all[next++];
  }
  void reset() { next = 0; }
  ~EventPool() {
    for (auto e : all) cudaEventDestroy(e);
  }
};

struct sufgpu_ctx {
  int device = 0;
  bool profiling = false;
  EventPool event_pool;
  std::vector<PendingLaunch> pending;
  std::vector<KernelTotals> profile;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  // Output copies that overlap the LCP phase (single builds): a second
  // stream, ordered after the compute stream by copy_ready, joined back by
  // copy_done.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
  // Host threads zero-filling output planes that need no copy (the high
  // planes of split40/48 coordinates below 2^32); the build joins them
  // before it returns.
  std::vector<std::thread> fillers;
  Arena arena;
  std::string last_error;
  u64* host_scalars = nullptr;  // pinned readback slots
  u8* host_small = nullptr;     // pinned staging for small uploads (1 MiB)
  std::vector<u8> anchor_pos;
  std::vector<u8> anchor_val;
  cudaEvent_t ev[8] = {};
  u32 launches = 0;
  // Build knobs (sufgpu_set_tuning) and per-size overrides
  // (sufgpu_set_tuning_class, written by the autotuner).
  Tuning tune;
  std::vector<TuningClass> tuning_classes;
  // Instantiated round-pair graphs, reused by later builds with the same
  // layout (most recent last; the oldest is dropped beyond a few).
  struct CachedGraph {
    std::vector<u64> key;
    cudaGraphExec_t exec;
    u32 kernels;
  };
  std::vector<CachedGraph> round_graphs;
  // Fold buffers of sufgpu_crc32_device (grown on demand).
  u32* crc_scratch = nullptr;
  u64 crc_scratch_words = 0;
  // Layouts of recent builds: a layout's rounds are captured from its second
  // build on, so one-off builds never pay for a capture.
  std::vector<std::vector<u64>> seen_layouts;
  // sufgpu_build_collection: helper contexts on the same device (one host
  // thread each) and the anchors of its sub-batches (valid until the next
  // collection build on this context).
  std::vector<sufgpu_ctx*> helpers;
  std::vector<std::vector<u8>> collection_anchors;
  // Per sub-batch of the last collection build: worker, and seconds since
  // the call began at which it started, took the gate, left it and ended.
  struct PartTrace {
    u32 worker;
    double start, gate_in, gate_out, end;
  };
  std::vector<PartTrace> collection_trace;
  void drop_round_graphs() {
    for (auto& g : round_graphs) cudaGraphExecDestroy(g.exec);
    round_graphs.clear();
  }
};

namespace {

struct Engine {
  sufgpu_ctx& c;
  Layout L{};
  std::vector<u64> begin;  // host segment offsets (count+1)
  u32 segs = 1;
  u64 n = 0;
  sufgpu_build_stats st{};
  // After the doubling: where the sorted SA lives, and the other n-row u32
  // buffer (free for PHI flags and byte-coded primaries).
  u32* sa = nullptr;
  u32* spare = nullptr;
  u32 seed_length = 0;  // symbols every seed group shares
  u64 rank_rows = 0;    // rows a rank may name (n, or the arena capacity)
  // Long-run split (runs.cuh): allowed by suffix_sort, on once runs were
  // found and laid out.  The host vectors back the uploads until the build ends.
  // Plane checksums (SUFGPU_FLAG_PLANE_CRC, single builds): CRC-32 of each
  // plane's bytes as copied out, into st.plane_crc.
  bool want_crc = false;
  bool allow_runs = false;
  bool allow_two_bit = false;  // the served engine's shared arena keeps the code-table seed
  // Collection workers share one gate: a build holds it from its first kernel
  // to its last, so that one worker's output copies run while another
  // computes instead of all workers computing, then copying, in step.
  std::mutex* gate = nullptr;
  bool gate_held = false;
  // Host clock readings of the gate (steady_clock), for the collection trace.
  std::chrono::steady_clock::time_point gate_in{}, gate_out{};
  void gate_enter() {
    if (!gate) return;
    gate->lock();
    gate_held = true;
    gate_in = std::chrono::steady_clock::now();
  }
  void gate_leave() {  // after the build's last kernel is enqueued
    if (!gate_held) return;
    SG_CUDA(cudaEventRecord(c.ev[6], c.stream));
    SG_CUDA(cudaEventSynchronize(c.ev[6]));
    gate_held = false;
    gate_out = std::chrono::steady_clock::now();
    gate->unlock();
  }
  void join_fillers() {
    for (auto& t : c.fillers) {
      if (t.joinable()) t.join();
    }
    c.fillers.clear();
  }
  ~Engine() {
    join_fillers();
    if (gate_held) gate->unlock();
  }
  bool runs_on = false;
  u32 run_count = 0;
  u64 run_members = 0;
  u64 run_active = 0;
  RunIndex run_index{};
  std::vector<RunRecord> h_recs;
  std::vector<RunClass> h_classes;
  std::vector<u32> h_len, h_a, h_e, h_bitmap;
  std::vector<u64> h_prefix;

  explicit Engine(sufgpu_ctx& ctx) : c(ctx) {}

  Segments segments() const { return Segments{L.seg_begin, segs}; }

  void sync() { SG_CUDA(cudaStreamSynchronize(c.stream)); }

  u64 read_scalar(int slot) {
    SG_CUDA(cudaMemcpyAsync(c.host_scalars + slot, L.scalars + slot, 8,
                            cudaMemcpyDeviceToHost, c.stream));
    sync();
    return c.host_scalars[slot];
  }

  void upload(void* dst, const void* src, u64 bytes) {
    if (bytes <= (1u << 20)) {
      sync();  // the staging buffer may still feed an earlier copy
      std::memcpy(c.host_small, src, bytes);
      SG_CUDA(cudaMemcpyAsync(dst, c.host_small, bytes, cudaMemcpyHostToDevice, c.stream));
    } else {
      SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
    }
  }

  void zero(void* p, u64 bytes) { SG_CUDA(cudaMemsetAsync(p, 0, bytes, c.stream)); }

  // Launches one kernel on the context stream.  `name` and `bytes` (the
  // kernel's algorithmic bytes: what it must read and write at minimum) feed
  // the optional per-kernel profile.
  template <class K, class... Args>
  void launch(const char* name, u64 bytes, K kernel, u64 grid, u32 block, u64 smem,
              Args... args) {
    if (grid == 0) return;
    cudaEvent_t before = nullptr, after = nullptr;
    if (c.profiling) {
      before = c.event_pool.take();
      after = c.event_pool.take();
      SG_CUDA(cudaEventRecord(before, c.stream));
    }
    kernel<<<static_cast<unsigned>(grid), block, smem, c.stream>>>(args...);
    SG_CUDA(cudaGetLastError());
    ++c.launches;
    if (c.profiling) {
      SG_CUDA(cudaEventRecord(after, c.stream));
      c.pending.push_back(PendingLaunch{name, bytes, before, after});
    }
  }

  u64 grid_stride_blocks(u64 work, u32 block) {
    const u64 want = (work + block - 1) / block;
    return std::max<u64>(1, std::min<u64>(want, u64(c.sm_count) * 16));
  }

  // Radix sort (keys, vals) in place over [begin_bit, end_bit) using the
  // alternates as ping-pong buffers.  seg_begin/seg_tiles must be uploaded.
  // Returns true when the result ended in the alternate buffers.
  // With pass0 set, the first pass is done by that callback (after the digit
  // offsets are known) into keys/vals, and the launches start at pass 1.
  bool radix_sort(const char* name, u64* keys, u32* vals, u64* keys_alt, u32* vals_alt,
                  const u64* seg_begin, const u32* seg_tiles, u32 seg_count,
                  u32 total_tiles, u64 sort_elems, u32 begin_bit, u32 end_bit,
                  bool check_needed, bool hist_ready = false,
                  const std::function<void()>& pass0 = {}) {
    if (end_bit <= begin_bit || total_tiles == 0) return false;
    const u32 passes = (end_bit - begin_bit + kRadixBits - 1) / kRadixBits;
    SortSegments ss{seg_begin, seg_tiles, seg_count, total_tiles, c.tune.sort_tile};
    const u64 elems = sort_elems;
    u32 needed[kMaxPasses];
    for (u32 p = 0; p < passes; ++p) needed[p] = 1;
    if (check_needed) {
      zero(L.counters + 32, 4 * kMaxPasses);
      if (!hist_ready) {
        zero(L.hist, u64(seg_count) * passes * kRadixDigits * 4);
        launch("radix_histogram", elems * 8, radix_histogram_kernel, total_tiles, kSortBlock, 0,
               keys, ss, begin_bit, passes, L.hist);
      }
      launch("radix_offsets", u64(seg_count) * passes * kRadixDigits * 12, radix_offsets_kernel,
             seg_count, kRadixDigits, 0, L.hist, seg_begin, passes, L.digit_start,
             L.counters + 32);
      SG_CUDA(cudaMemcpyAsync(c.host_small, L.counters + 32, 4 * passes,
                              cudaMemcpyDeviceToHost, c.stream));
      sync();
      std::memcpy(needed, c.host_small, 4 * passes);
    } else {
      if (!hist_ready) {
        zero(L.hist, u64(seg_count) * passes * kRadixDigits * 4);
        launch("radix_histogram", elems * 8, radix_histogram_kernel, total_tiles, kSortBlock, 0,
               keys, ss, begin_bit, passes, L.hist);
      }
      launch("radix_offsets", u64(seg_count) * passes * kRadixDigits * 12, radix_offsets_kernel,
             seg_count, kRadixDigits, 0, L.hist, seg_begin, passes, L.digit_start,
             L.counters + 32);
    }
    bool swapped = false;
    u64* kin = keys;
    u32* vin = vals;
    u64* kout = keys_alt;
    u32* vout = vals_alt;
    if (pass0) pass0();
    for (u32 p = pass0 ? 1 : 0; p < passes; ++p) {
      if (!needed[p]) continue;
      zero(L.status, u64(total_tiles) * kRadixDigits * 8);
      zero(L.counters, 4);
      const OnesweepVariant v = onesweep_variant(c.tune.ballot_rank && elems >= c.tune.ballot_min_elems,
                                                 vals ? c.tune.sort_block : c.tune.keys_sort_block,
                                                 c.tune.sort_tile, vals != nullptr,
                                                 c.tune.tma_tile && seg_count == 1);
      launch(name, elems * (vals ? 24 : 16), v.fn, total_tiles, v.block, v.smem,
             kin, vin, kout, vout, ss, begin_bit + p * kRadixBits, p, passes,
             L.digit_start, L.status, L.counters, L.flags);
      std::swap(kin, kout);
      std::swap(vin, vout);
      swapped = !swapped;
    }
    return swapped;
  }

  // Digit counts of a radix sort whose keys hold a permutation of [0, n) at
  // key bit 32 (the rank write's (position << 32 | head) pairs): for the
  // digit of position bits [b, b + 8), each period of 2^(b+8) positions gives
  // every digit 2^b of them, and the remainder fills digits from 0 upwards.
  // Written to L.hist for one segment, so the sort needs no histogram pass.
  // counts: one entry per segment (a batch: each instance's local positions
  // are a permutation of [0, its length)); layout [segment][pass][digit].
  void upload_permutation_hist(const std::vector<u64>& counts, u32 begin_bit, u32 end_bit) {
    const u32 passes = (end_bit - begin_bit + kRadixBits - 1) / kRadixBits;
    std::vector<u32> h(counts.size() * passes * kRadixDigits);
    for (size_t j = 0; j < counts.size(); ++j) {
      const u64 count = counts[j];
      for (u32 p = 0; p < passes; ++p) {
        const u32 b = begin_bit + p * kRadixBits - 32;
        const u64 width = u64(1) << b;
        const u64 period = width << kRadixBits;
        const u64 full = count / period, rem = count % period;
        for (u32 d = 0; d < kRadixDigits; ++d) {
          const u64 lo = u64(d) * width;
          const u64 extra = rem > lo ? std::min<u64>(width, rem - lo) : 0;
          h[(j * passes + p) * kRadixDigits + d] = static_cast<u32>(full * width + extra);
        }
      }
    }
    upload(L.hist, h.data(), h.size() * 4);
  }

  void upload_segments(const std::vector<u64>& b) {
    std::vector<u32> tiles(b.size());
    tiles[0] = 0;
    for (size_t j = 0; j + 1 < b.size(); ++j) {
      tiles[j + 1] = tiles[j] + static_cast<u32>((b[j + 1] - b[j] + c.tune.sort_tile - 1) / c.tune.sort_tile);
    }
    std::vector<u8> blob(b.size() * 12);
    std::memcpy(blob.data(), b.data(), b.size() * 8);
    std::memcpy(blob.data() + b.size() * 8, tiles.data(), b.size() * 4);
    sync();
    std::memcpy(c.host_small, blob.data(), blob.size());
    SG_CUDA(cudaMemcpyAsync(L.seg_begin, c.host_small, b.size() * 8, cudaMemcpyHostToDevice, c.stream));
    SG_CUDA(cudaMemcpyAsync(L.seg_tiles, c.host_small + b.size() * 8, b.size() * 4,
                            cudaMemcpyHostToDevice, c.stream));
    last_tiles = tiles.back();
  }
  u32 last_tiles = 0;

  // ---- CRC-32 (zlib's crc32(crc_in, data, bytes)) of device memory: the
  // bytes before the first 16-byte boundary on the host (the chunk kernel
  // loads 16-byte vectors), full 16 KiB chunks on the device (crc32.cuh)
  // folded to one remainder, the tail on the host.  scratch holds
  // 2 * ceil(bytes / 16 KiB) words.
  u32 crc32_device(const void* data, u64 bytes, u32 crc_in, u32* scratch) {
    static const std::vector<u32> table = [] {
      std::vector<u32> t(256);
      for (u32 i = 0; i < 256; ++i) t[i] = crc_table_entry(i);
      return t;
    }();
    const u8* p = static_cast<const u8*>(data);
    u32 state = crc_in ^ 0xffffffffu;
    const u64 head = std::min<u64>(bytes, (16 - (reinterpret_cast<uintptr_t>(p) & 15)) & 15);
    if (head) {
      u8 host[16];
      SG_CUDA(cudaMemcpyAsync(host, p, head, cudaMemcpyDefault, c.stream));
      sync();
      for (u64 i = 0; i < head; ++i) state = table[(state ^ host[i]) & 0xffu] ^ (state >> 8);
      p += head;
      bytes -= head;
    }
    const u64 full = bytes / kCrcChunk;
    if (full) {
      launch("crc32", full * kCrcChunk, crc_chunks_kernel, std::min<u64>(full, u64(c.sm_count) * 8),
             kCrcBlock, 0, p, full, scratch);
      u32* in = scratch;
      u32* out = scratch + full;
      u64 count = full, width = kCrcChunk, last = kCrcChunk;
      while (count > 1) {
        launch("crc32_fold", count * 4, crc_fold_kernel, grid_stride_blocks((count + 1) / 2, 256),
               256, 0, static_cast<const u32*>(in), count, width, last,
               crc_shift_factor(width), out);
        last = (count & 1) ? last : width + last;
        width *= 2;
        count = (count + 1) / 2;
        std::swap(in, out);
      }
      SG_CUDA(cudaMemcpyAsync(c.host_scalars + 30, in, 4, cudaMemcpyDeviceToHost, c.stream));
      sync();
      u32 raw = 0;
      std::memcpy(&raw, c.host_scalars + 30, 4);
      state = crc_mulmod(state, crc_shift_factor(full * kCrcChunk)) ^ raw;
    }
    const u64 tail = bytes - full * kCrcChunk;
    if (tail) {
      std::vector<u8> host(tail);
      SG_CUDA(cudaMemcpyAsync(host.data(), p + full * kCrcChunk, tail, cudaMemcpyDefault, c.stream));
      sync();
      for (u8 b : host) state = table[(state ^ b) & 0xffu] ^ (state >> 8);
    }
    return state ^ 0xffffffffu;
  }

  // ---- Long runs of one symbol: find them, pair starts with ends and lay out
  // their sub-groups (runs.cuh).  Leaves runs_on false when there are none,
  // too many, or the seed is too short for the split to pay.  With `keep`,
  // runs of the other byte values are left to the rounds.
  void plan_runs(u32 s, const bool* keep = nullptr) {
    runs_on = false;
    run_index = RunIndex{};
    if (!allow_runs || !c.tune.run_split || s < 8 || n < 2 * u64(s)) return;
    zero(L.scalars + 8, 16);
    launch("long_runs", n, long_runs_kernel,
           grid_stride_blocks((n + kRunChunk - 1) / kRunChunk, 256), 256, 0, L.text, n,
           segments(), s, L.run_starts, L.run_ends, L.run_cap, L.scalars + 8);
    SG_CUDA(cudaMemcpyAsync(c.host_scalars + 8, L.scalars + 8, 16, cudaMemcpyDeviceToHost,
                            c.stream));
    sync();
    u64 count = c.host_scalars[8];
    if (count != c.host_scalars[9]) {
      throw BuildError{SUFGPU_BUILD_FAILURE, "long-run starts and ends do not pair"};
    }
    if (count == 0 || count > L.run_cap) return;
    std::vector<u64> starts(count), ends(count);
    SG_CUDA(cudaMemcpyAsync(starts.data(), L.run_starts, count * 8, cudaMemcpyDeviceToHost,
                            c.stream));
    SG_CUDA(cudaMemcpyAsync(ends.data(), L.run_ends, count * 8, cudaMemcpyDeviceToHost,
                            c.stream));
    sync();
    std::sort(starts.begin(), starts.end());
    std::sort(ends.begin(), ends.end());
    if (keep) {  // starts and ends pair by rank (runs do not overlap)
      u64 kept = 0;
      for (u64 i = 0; i < count; ++i) {
        if (!keep[starts[i] & 0xff]) continue;
        starts[kept] = starts[i];
        ends[kept] = ends[i];
        ++kept;
      }
      count = kept;
      starts.resize(count);
      ends.resize(count);
      if (count == 0) return;
    }
    // Runs in position order; key (instance, symbol, class) names the class.
    std::vector<u64> key(count);
    std::vector<u32> len(count);
    h_a.resize(count);
    h_e.resize(count);
    for (u64 i = 0; i < count; ++i) {
      const u64 a = starts[i] >> 8, e = ends[i] >> 1;
      const u64 sym = starts[i] & 0xff, cls = ends[i] & 1;
      if (e <= a || e - a < s || (i > 0 && a < h_e[i - 1])) {
        throw BuildError{SUFGPU_BUILD_FAILURE, "inconsistent long-run boundaries"};
      }
      const u64 seg = segs == 1 ? 0
          : static_cast<u64>(std::upper_bound(begin.begin(), begin.end(), a) - begin.begin()) - 1;
      if (e > begin[seg + 1]) throw BuildError{SUFGPU_BUILD_FAILURE, "long run crosses an instance"};
      h_a[i] = static_cast<u32>(a);
      h_e[i] = static_cast<u32>(e);
      len[i] = static_cast<u32>(e - a);
      key[i] = (seg << 9) | (sym << 1) | cls;
    }
    std::map<u64, std::vector<u32>> classes;
    for (u32 i = 0; i < count; ++i) classes[key[i]].push_back(i);
    std::map<u64, u64> class0_size;  // per (instance, symbol)
    for (const auto& kv : classes) {
      if (kv.first & 1) continue;
      u64 size = 0;
      for (u32 i : kv.second) size += len[i] - s + 1;
      class0_size[kv.first >> 1] = size;
    }
    h_recs.assign(count, RunRecord{});
    h_classes.clear();
    h_len.clear();
    h_prefix.clear();
    run_active = 0;
    for (auto& kv : classes) {
      std::vector<u32>& idx = kv.second;
      std::stable_sort(idx.begin(), idx.end(), [&](u32 x, u32 y) { return len[x] < len[y]; });
      RunClass k{};
      k.cls = static_cast<u32>(kv.first & 1);
      k.m = static_cast<u32>(idx.size());
      k.off = static_cast<u32>(h_len.size());
      k.poff = static_cast<u32>(h_prefix.size());
      u64 acc = 0, size = 0;
      h_prefix.push_back(0);
      for (u32 t = 0; t < k.m; ++t) {
        const u32 L_t = len[idx[t]];
        h_len.push_back(L_t);
        acc += k.cls == 0 ? L_t - s + 1 : L_t;
        h_prefix.push_back(acc);
        size += L_t - s + 1;
        h_recs[idx[t]].slot = k.m - 1 - t;
        h_recs[idx[t]].desc = static_cast<u32>(h_classes.size());
      }
      // Sub-groups of two or more rows: d <= the second-longest run.
      u64 act = 0;
      if (k.m >= 2) {
        const u64 second = h_len[k.off + k.m - 2];
        for (u32 t = 0; t < k.m; ++t) act += std::min<u64>(len[idx[t]], second) - s + 1;
      }
      k.size = size;
      k.act_count = act;
      k.base_rel = k.cls == 0 ? 0 : class0_size[kv.first >> 1];
      k.act_first_rel = k.cls == 0 ? 0 : size - act;
      k.act_off = run_active;
      run_active += act;
      h_classes.push_back(k);
    }
    run_members = 0;
    h_bitmap.assign(L.run_bitmap_words, 0);
    for (u64 i = 0; i < count; ++i) {
      h_recs[i].first_member = run_members;
      h_recs[i].a = h_a[i];
      h_recs[i].e = h_e[i];
      run_members += len[i] - s + 1;
      const u64 last_member = h_e[i] - s;
      for (u64 b = h_a[i] >> kRunBlockBits; b <= (last_member >> kRunBlockBits); ++b) {
        h_bitmap[b >> 5] |= 1u << (b & 31);
      }
    }
    auto put = [&](void* dst, const void* src, u64 bytes) {
      SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
    };
    put(L.run_recs, h_recs.data(), count * sizeof(RunRecord));
    put(L.run_classes, h_classes.data(), h_classes.size() * sizeof(RunClass));
    put(L.run_len, h_len.data(), h_len.size() * 4);
    put(L.run_prefix, h_prefix.data(), h_prefix.size() * 8);
    put(L.run_a, h_a.data(), count * 4);
    put(L.run_e, h_e.data(), count * 4);
    put(L.run_bitmap, h_bitmap.data(), h_bitmap.size() * 4);
    run_count = static_cast<u32>(count);
    run_index = RunIndex{L.run_a, L.run_e, L.run_bitmap, run_count};
    runs_on = true;
    st.long_runs = count;
  }

  // ---- Seed phase: alphabet remap, seed keys, the segmented seed sort and
  // seed ranks.  Leaves SA in `sa` (sa_out when given), head-row ranks in
  // L.rank, seed-boundary LCPs in L.lcp and the active list in L.x; returns
  // the active count.
  u64 seed_phase(u32* sa_out = nullptr) {
    // Alphabet remap.
    zero(L.alpha, 256 * 4);
    launch("alphabet_histogram", n, alphabet_histogram_kernel,
           grid_stride_blocks(n / 16 + 1, 256), 256, 0,
           L.text, n, L.alpha);
    u32 counts[256];
    SG_CUDA(cudaMemcpyAsync(c.host_small, L.alpha, sizeof(counts), cudaMemcpyDeviceToHost, c.stream));
    sync();
    std::memcpy(counts, c.host_small, sizeof(counts));
    u16 code[256];
    u32 sigma = 0;
    for (int b = 0; b < 256; ++b) code[b] = counts[b] ? static_cast<u16>(++sigma) : 0;
    const u32 bits = std::max<u32>(1, bits_for(sigma));
    u64 longest = 1;
    for (u32 j = 0; j < segs; ++j) longest = std::max<u64>(longest, begin[j + 1] - begin[j]);
    // Seed length: enough symbols that two seed keys of one instance rarely
    // collide by chance, log2(longest) / H + 2.5 with H the text's entropy in
    // bits per symbol, plus one per doubling beyond 2^27 symbols (larger
    // genomes hold more repeat copies), rounded up to whole 8-bit radix
    // passes of the sort key.  Longer seeds cost a pass per 8 bits; shorter
    // ones leave more rows to the rounds.  0 = no rule (near-constant text).
    u32 need = 0;
    {
      double entropy = 0;
      for (int b = 0; b < 256; ++b) {
        if (!counts[b]) continue;
        const double q = static_cast<double>(counts[b]) / static_cast<double>(n);
        entropy -= q * std::log2(q);
      }
      if (entropy > 0.5) {
        const double lg = std::log2(static_cast<double>(longest));
        need = static_cast<u32>(std::ceil(lg / entropy + 2.5 + std::max(0.0, lg - 27.0)));
      }
    }
    // Two-bit seed: one instance whose text is four consecutive byte values
    // (A, C, G, T) but for a few others (sentinel, separators, N), which the
    // rare list places exactly.  The exact keys of rare rows hold s symbols
    // of `bits`, so s <= 64 / bits.
    TwoBitSeed tb{};
    bool two_bit = false;
    bool keep_runs[256] = {};
    if (allow_two_bit && (segs == 1 || c.tune.two_bit_batch) && c.tune.two_bit_seed &&
        n >= c.tune.two_bit_min && sigma >= 4 && bits <= 4) {
      int lo_byte = -1;
      u64 best = 0;
      for (int b = 0; b + 3 < 256; ++b) {
        if (!counts[b] || !counts[b + 1] || !counts[b + 2] || !counts[b + 3]) continue;
        const u64 c4 = u64(counts[b]) + counts[b + 1] + counts[b + 2] + counts[b + 3];
        if (c4 > best) {
          best = c4;
          lo_byte = b;
        }
      }
      int top_byte = 255;
      while (top_byte > 0 && !counts[top_byte]) --top_byte;
      if (lo_byte >= 0) {
        const bool has_hi = top_byte > lo_byte + 3;
        const u64 other = n - best - (has_hi ? counts[top_byte] : 0);
        if (other * 64 <= n) {
          two_bit = true;
          tb.lo = code[lo_byte];
          tb.hi = has_hi ? code[top_byte] : 0;
          for (int b = lo_byte; b < lo_byte + 4; ++b) keep_runs[b] = true;
          if (has_hi) keep_runs[top_byte] = true;
        }
      }
    }
    const u32 index_bits = std::max<u32>(1, bits_for(longest - 1));
    upload(L.code, code, sizeof(code));
    upload_segments(begin);
    const u32 seed_tiles = last_tiles;
    u32 symbols = 0, packed_shift = 0, seed_bits = 0;
    u64* keys = nullptr;
    u64 rare_count = 0;
    // Rare list in rank (free until the window scatter): exact keys, their
    // sort's second buffer, two-bit keys, positions and their second buffer.
    const u64 rare_cap = n / 16;  // 32 bytes each: half of rank's 4n
    u64* rare_key = reinterpret_cast<u64*>(L.rank);
    u64* rare_key_alt = rare_key + rare_cap;
    u64* rare_k2 = rare_key_alt + rare_cap;
    u32* rare_pos = reinterpret_cast<u32*>(rare_k2 + rare_cap);
    u32* rare_pos_alt = rare_pos + rare_cap;
    for (int attempt = 0;; ++attempt) {
      if (attempt > 0) two_bit = false;  // too many rare rows: the code-table seed
      // Symbols per key: sym_bits each (+ 2 tag bits for the two-bit key).
      const u32 sym_bits = two_bit ? 2 : bits;
      const u32 tag = two_bit ? 2 : 0;
      // A batch's rare list keys carry the instance above the exact key.
      const u32 inst_bits = segs > 1 ? std::max<u32>(1, bits_for(segs - 1)) : 0;
      const u32 cap_symbols = two_bit ? std::min<u32>((64 - inst_bits) / bits, 31) : 64 / bits;
      symbols = (64 - tag) / sym_bits;
      if (c.tune.seed_symbols) {
        symbols = std::min(symbols, c.tune.seed_symbols);
      } else if (need) {
        const u32 passes = (need * sym_bits + tag + kRadixBits - 1) / kRadixBits;
        symbols = std::min(symbols, std::max<u32>(1, (passes * kRadixBits - tag) / sym_bits));
      }
      symbols = std::min(symbols, cap_symbols);
      // Packed seed: when every instance fits 2^packed_max_bits symbols, its
      // local index rides in the low key bits and the sort moves keys only.
      packed_shift = 0;
      if (c.tune.packed_max_bits && index_bits <= c.tune.packed_max_bits) {
        // No longer than the seed rule asks (fewer passes), no longer than
        // the bits beside the index allow.
        u32 packed_symbols = std::min({(64 - index_bits - tag) / sym_bits, cap_symbols, symbols});
        if (packed_symbols >= std::min<u32>(symbols, 12)) {
          packed_shift = index_bits;
          symbols = packed_symbols;
        }
      }
      st.seed_symbols = symbols;
      st.seed_code_bits = sym_bits;
      plan_runs(symbols, two_bit ? keep_runs : nullptr);

      // Seed keys and the segmented seed sort.
      seed_bits = sym_bits * symbols + tag;
      const bool fused = c.tune.seed_fused && c.tune.sort_tile == kSortTile;
      // With the fused first pass this kernel only counts: long runs per thread.
      const bool counts_only = fused && c.tune.seed_count_run;
      const u64 count_blocks = (n + u64(kSeedBlock) * kSeedCountRun - 1) / (u64(kSeedBlock) * kSeedCountRun);
      const u32 seed_passes = (seed_bits + kRadixBits - 1) / kRadixBits;
      zero(L.hist, u64(segs) * seed_passes * kRadixDigits * 4);
      if (two_bit) {
        tb.all_hi = 0;
        for (u32 k = 0; k < symbols; ++k) tb.all_hi = (tb.all_hi << bits) | tb.hi;
        tb.rare_key = rare_key;
        tb.rare_pos = rare_pos;
        tb.rare_cap = rare_cap;
        tb.rare_count = L.scalars + 44;
        tb.inst_shift = segs > 1 ? bits * symbols : 0;
        zero(L.scalars + 44, 8);
        if (counts_only) {
          launch("seed_keys", n, seed_keys_kernel<true, kSeedCountRun>, count_blocks, kSeedBlock,
                 sizeof(SeedSmemT<kSeedCountRun>), L.text, n, segments(),
                 static_cast<const u16*>(L.code), bits, symbols, seed_passes, L.hist, packed_shift,
                 nullptr, nullptr, tb);
        } else {
          launch("seed_keys", fused ? n : (packed_shift ? n * 9 : n * 13), seed_keys_kernel<true>,
                 (n + kSeedTile - 1) / kSeedTile, kSeedBlock, sizeof(SeedSmem), L.text, n,
                 segments(), static_cast<const u16*>(L.code), bits, symbols, seed_passes, L.hist,
                 packed_shift, fused ? nullptr : L.k0, fused ? nullptr : L.v0, tb);
        }
        // Read back with the sort's pass check below (one synchronisation).
        SG_CUDA(cudaMemcpyAsync(c.host_scalars + 44, L.scalars + 44, 8, cudaMemcpyDeviceToHost,
                                c.stream));
      } else if (counts_only) {
        launch("seed_keys", n, seed_keys_kernel<false, kSeedCountRun>, count_blocks, kSeedBlock,
               sizeof(SeedSmemT<kSeedCountRun>), L.text, n, segments(),
               static_cast<const u16*>(L.code), bits, symbols, seed_passes, L.hist, packed_shift,
               nullptr, nullptr, TwoBitSeed{});
      } else {
        launch("seed_keys", fused ? n : (packed_shift ? n * 9 : n * 13),
               seed_keys_kernel<false>, (n + kSeedTile - 1) / kSeedTile, kSeedBlock,
               sizeof(SeedSmem), L.text, n, segments(), static_cast<const u16*>(L.code), bits,
               symbols, seed_passes, L.hist, packed_shift, fused ? nullptr : L.k0,
               fused ? nullptr : L.v0, TwoBitSeed{});
      }
      // The fused first pass (seedsort.cuh): generates the keys again and
      // writes them into (k0, v0) partitioned by the lowest sorted digit.
      const std::function<void()> pass0 = [&, two_bit_now = two_bit] {
        zero(L.status, u64(seed_tiles) * kRadixDigits * 8);
        zero(L.counters, 4);
        const SortSegments ss{L.seg_begin, L.seg_tiles, segs, seed_tiles, kSortTile};
        if (two_bit_now) {
          launch("seed_sorted", n * (packed_shift ? 9 : 13), seed_sorted_kernel<true>, seed_tiles,
                 kSortBlock, sizeof(SeedSortSmem), L.text, ss, static_cast<const u16*>(L.code),
                 bits, symbols, packed_shift, seed_passes, static_cast<const u64*>(L.digit_start),
                 L.k0, L.v0, L.status, L.counters, L.flags, tb);
        } else {
          launch("seed_sorted", n * (packed_shift ? 9 : 13), seed_sorted_kernel<false>,
                 seed_tiles, kSortBlock, sizeof(SeedSortSmem), L.text, ss,
                 static_cast<const u16*>(L.code), bits, symbols, packed_shift, seed_passes,
                 static_cast<const u64*>(L.digit_start), L.k0, L.v0, L.status, L.counters,
                 L.flags, TwoBitSeed{});
        }
      };
      keys = L.k0;
      if (packed_shift) {
        const bool swapped = radix_sort("seed_onesweep", L.k0, nullptr, L.k1, nullptr, L.seg_begin,
                                        L.seg_tiles, segs, seed_tiles, n, packed_shift,
                                        packed_shift + seed_bits, true, true,
                                        fused ? pass0 : std::function<void()>());
        keys = swapped ? L.k1 : L.k0;
        sa = L.sa;
        spare = L.v0;
      } else {
        const bool swapped = radix_sort("seed_onesweep", L.k0, L.v0, L.k1, L.sa, L.seg_begin,
                                        L.seg_tiles, segs, seed_tiles, n, 0, seed_bits, true, true,
                                        fused ? pass0 : std::function<void()>());
        if (swapped) {
          keys = L.k1;
          sa = L.sa;
          spare = L.v0;
        } else {
          keys = L.k0;
          sa = L.v0;
          spare = L.sa;
        }
      }
      if (!two_bit) break;
      rare_count = c.host_scalars[44];
      if (rare_count <= rare_cap) break;
    }
    st.seed_rare_rows = two_bit ? static_cast<u32>(std::min<u64>(rare_count, 0xffffffffu)) : 0;
    RareRows rare{};
    if (two_bit && rare_count > 0) {
      // The rare rows in exact order, and their two-bit keys.
      const u32 t = static_cast<u32>((rare_count + c.tune.sort_tile - 1) / c.tune.sort_tile);
      const u64 b2[2] = {0, rare_count};
      const u32 t2[2] = {0, t};
      // A staging slot no other copy of this build uses: no synchronisation.
      std::memcpy(c.host_small + 16384, b2, 16);
      std::memcpy(c.host_small + 16384 + 16, t2, 8);
      SG_CUDA(cudaMemcpyAsync(L.sort_begin, c.host_small + 16384, 16, cudaMemcpyHostToDevice, c.stream));
      SG_CUDA(cudaMemcpyAsync(L.sort_tiles, c.host_small + 16384 + 16, 8, cudaMemcpyHostToDevice,
                              c.stream));
      const u32 rare_bits = bits * symbols + (segs > 1 ? std::max<u32>(1, bits_for(segs - 1)) : 0);
      const bool sw = radix_sort("rare_sort", rare_key, rare_pos, rare_key_alt, rare_pos_alt,
                                 L.sort_begin, L.sort_tiles, 1, t, rare_count, 0, rare_bits,
                                 false);
      rare.key = sw ? rare_key_alt : rare_key;
      rare.pos = sw ? rare_pos_alt : rare_pos;
      rare.k2 = rare_k2;
      rare.count = rare_count;
      rare.text = L.text;
      launch("rare_two_bit", rare_count * 16, rare_two_bit_kernel,
             grid_stride_blocks(rare_count, 256), 256, 0, rare.key, rare_count, symbols, bits, tb,
             rare_k2);
    }
    // Seed ranks and the initial active list (in x).
    const u64 scan_tiles = (n + kScanTile - 1) / kScanTile;
    zero(L.status, 2 * (scan_tiles + 1) * 8);
    zero(L.counters, 4);
    u64* status_max = L.status;
    u64* status_sum = L.status + scan_tiles + 1;
    u64* pairs = keys == L.k0 ? L.k1 : L.k0;
    launch("seed_rank", n * 24, two_bit ? seed_rank_kernel<true> : seed_rank_kernel<false>,
           scan_tiles, kScanBlock, 0, static_cast<const u64*>(keys), sa, n, segments(),
           packed_shift, bits, symbols, pairs, L.lcp, L.x, status_max, status_sum, L.counters,
           L.scalars + 0, L.flags, runs_on ? 1u : 0u, segs > 1 ? 1u : 0u);
    if (rare.count > 0) {
      launch("rare_place", rare.count * 32, rare_place_kernel, grid_stride_blocks(rare.count, 256),
             256, 0, static_cast<const u64*>(keys), n, packed_shift, rare, bits, symbols, segments(), sa,
             pairs, L.lcp, L.flags);
      // Rare rows in shared windows join the active list (count in [45]).
      const u64 rare_tiles = (rare.count + kScanTile - 1) / kScanTile;
      zero(L.status, (rare_tiles + 1) * 8);
      zero(L.counters + 2, 4);
      zero(L.scalars + 45, 8);
      launch("rare_active", rare.count * 16, rare_active_kernel, rare_tiles, kScanBlock, 0,
             rare.key, rare.pos, rare.count, L.x, static_cast<const u64*>(L.scalars + 0),
             L.scalars + 45, L.status, L.counters + 2, L.flags);
      SG_CUDA(cudaMemcpyAsync(c.host_scalars + 45, L.scalars + 45, 8, cudaMemcpyDeviceToHost,
                              c.stream));
    }
    // rank[SA[r]] = head: group the pairs by 2048-position window (keys-only
    // passes over the position's high bits), then one coalesced window write.
    // A batch groups instance-local positions inside each instance (a pass
    // per 8 bits of the longest instance above 11, not of the whole batch).
    const u32 pos_bits = std::max<u32>(1, bits_for(n - 1));
    u64* grouped = pairs;
    // Windows of 2^16 positions (a cluster of two blocks) when they take
    // fewer grouping passes than 2048-position windows.
    auto group_passes = [&](u32 w) { return pos_bits > w ? (pos_bits - w + 7) / 8 : 0u; };
    const bool cluster_window = segs == 1 && c.tune.rank_cluster && c.tune.rank_slots != 2 &&
                                group_passes(kClusterWindowBits) < group_passes(kWindowBits);
    const u32 window_bits = cluster_window ? kClusterWindowBits : kWindowBits;
    // A batch by 2^16-position windows per instance (clusters of two blocks)
    // when that saves a grouping pass over 2048-position windows.
    u64 batch_longest = 1;
    for (u32 j = 0; j < segs; ++j) batch_longest = std::max<u64>(batch_longest, begin[j + 1] - begin[j]);
    const u32 batch_bits = std::max<u32>(1, bits_for(batch_longest - 1));
    auto batch_passes = [&](u32 w) { return batch_bits > w ? (batch_bits - w + 7) / 8 : 0u; };
    const bool batch_cluster = segs > 1 && c.tune.batch_cluster && c.tune.rank_cluster &&
                               batch_passes(kClusterWindowBits) < batch_passes(kWindowBits);
    if (batch_cluster) {
      std::vector<u64> wbegin(segs + 1, 0);
      for (u32 j = 0; j < segs; ++j) {
        const u64 len = begin[j + 1] - begin[j];
        wbegin[j + 1] = wbegin[j] + ((len + (u64(1) << kClusterWindowBits) - 1) >> kClusterWindowBits);
      }
      if (batch_bits > kClusterWindowBits) {
        u64* other_keys = pairs == L.k0 ? L.k1 : L.k0;
        std::vector<u64> lens(segs);
        for (u32 j = 0; j < segs; ++j) lens[j] = begin[j + 1] - begin[j];
        upload_permutation_hist(lens, 32 + kClusterWindowBits, 32 + batch_bits);
        const bool sw = radix_sort("rank_group", pairs, nullptr, other_keys, nullptr, L.seg_begin,
                                   L.seg_tiles, segs, seed_tiles, n, 32 + kClusterWindowBits,
                                   32 + batch_bits, false, true);
        grouped = sw ? other_keys : pairs;
      }
      sync();
      std::memcpy(c.host_small, wbegin.data(), (segs + 1) * 8);
      SG_CUDA(cudaMemcpyAsync(L.digit_start, c.host_small, (segs + 1) * 8, cudaMemcpyHostToDevice,
                              c.stream));
      launch("window_scatter", n * 12, cluster_segment_window_scatter_kernel, wbegin[segs] * 2,
             ClusterWindow<2>::kBlock, ClusterWindow<2>::kSlice * 4,
             static_cast<const u64*>(grouped), segments(), static_cast<const u64*>(L.digit_start),
             L.rank, L.flags);
    } else if (segs > 1 && c.tune.rank_slots >= 1) {
      // Window slots per instance (rank_slot_segments_kernel): no grouping passes.
      std::vector<u64> wbegin(segs + 1, 0);
      for (u32 j = 0; j < segs; ++j) {
        wbegin[j + 1] = wbegin[j] + (begin[j + 1] - begin[j] + kSlotWindow - 1) / kSlotWindow;
      }
      const u64 windows = wbegin[segs];
      u32* fill = reinterpret_cast<u32*>(L.status);  // windows words: n/8192 + segs
      u64* slotted = pairs == L.k0 ? L.k1 : L.k0;
      sync();
      std::memcpy(c.host_small, wbegin.data(), (segs + 1) * 8);
      SG_CUDA(cudaMemcpyAsync(L.digit_start, c.host_small, (segs + 1) * 8, cudaMemcpyHostToDevice,
                              c.stream));
      zero(fill, windows * 4);
      launch("rank_slot", n * 16, rank_slot_segments_kernel, grid_stride_blocks(n, 256), 256, 0,
             static_cast<const u64*>(pairs), segments(), static_cast<const u64*>(L.digit_start),
             fill, slotted, L.flags);
      launch("window_scatter", n * 12, slot_segment_window_scatter_kernel, windows, 256,
             kSlotWindow * 4, static_cast<const u64*>(slotted), segments(),
             static_cast<const u64*>(L.digit_start), L.rank, L.flags);
    } else if (segs > 1) {
      u64 longest = 1;
      std::vector<u64> wbegin(segs + 1, 0);
      for (u32 j = 0; j < segs; ++j) {
        const u64 len = begin[j + 1] - begin[j];
        longest = std::max(longest, len);
        wbegin[j + 1] = wbegin[j] + (len + kWindow - 1) / kWindow;
      }
      const u32 local_bits = std::max<u32>(1, bits_for(longest - 1));
      if (local_bits > kWindowBits) {
        u64* other_keys = pairs == L.k0 ? L.k1 : L.k0;
        const bool sw = radix_sort("rank_group", pairs, nullptr, other_keys, nullptr, L.seg_begin,
                                   L.seg_tiles, segs, seed_tiles, n, 32 + kWindowBits,
                                   32 + local_bits, false);
        grouped = sw ? other_keys : pairs;
      }
      sync();
      std::memcpy(c.host_small, wbegin.data(), (segs + 1) * 8);
      SG_CUDA(cudaMemcpyAsync(L.digit_start, c.host_small, (segs + 1) * 8, cudaMemcpyHostToDevice,
                              c.stream));
      launch("window_scatter", n * 12, segment_window_scatter_kernel, wbegin[segs], 256, 0,
             static_cast<const u64*>(grouped), segments(), static_cast<const u64*>(L.digit_start),
             L.rank, L.flags);
    } else if (pos_bits > kWindowBits && c.tune.rank_slots == 2) {
      const u64 windows = (n + kSlotWindow - 1) >> kSlotBits;
      u32* fill = reinterpret_cast<u32*>(L.status);  // windows words: n/8192 << status size
      u64* slotted = pairs == L.k0 ? L.k1 : L.k0;
      zero(fill, windows * 4);
      launch("rank_slot", n * 16, rank_slot_kernel, grid_stride_blocks(n, 256), 256, 0,
             static_cast<const u64*>(pairs), n, fill, slotted, L.flags);
      launch("window_scatter", n * 12, slot_window_scatter_kernel, windows, 256,
             kSlotWindow * 4, static_cast<const u64*>(slotted), n, L.rank, L.flags);
    } else if (pos_bits > window_bits) {
      const u64 b2[2] = {0, n};
      const u32 t = static_cast<u32>((n + c.tune.sort_tile - 1) / c.tune.sort_tile);
      const u32 t2[2] = {0, t};
      sync();
      std::memcpy(c.host_small + 4096, b2, 16);
      std::memcpy(c.host_small + 4096 + 16, t2, 8);
      SG_CUDA(cudaMemcpyAsync(L.sort_begin, c.host_small + 4096, 16, cudaMemcpyHostToDevice, c.stream));
      SG_CUDA(cudaMemcpyAsync(L.sort_tiles, c.host_small + 4096 + 16, 8, cudaMemcpyHostToDevice, c.stream));
      u64* other_keys = pairs == L.k0 ? L.k1 : L.k0;
      upload_permutation_hist({n}, 32 + window_bits, 32 + pos_bits);
      const bool sw = radix_sort("rank_group", pairs, nullptr, other_keys, nullptr, L.sort_begin,
                                 L.sort_tiles, 1, t, n, 32 + window_bits, 32 + pos_bits, false,
                                 true);
      grouped = sw ? other_keys : pairs;
    }
    if (cluster_window) {
      const u64 windows = (n + (u64(1) << kClusterWindowBits) - 1) >> kClusterWindowBits;
      if (c.tune.rank_cluster == 4) {
        launch("window_scatter", n * 12, cluster4_window_scatter_kernel, windows * 4,
               ClusterWindow<4>::kBlock, ClusterWindow<4>::kSlice * 4,
               static_cast<const u64*>(grouped), n, L.rank, L.flags);
      } else {
        launch("window_scatter", n * 12, cluster_window_scatter_kernel, windows * 2,
               ClusterWindow<2>::kBlock, ClusterWindow<2>::kSlice * 4,
               static_cast<const u64*>(grouped), n, L.rank, L.flags);
      }
    } else if (segs == 1 && !(pos_bits > kWindowBits && c.tune.rank_slots == 2)) {
      launch("window_scatter", n * 12, window_scatter_kernel, (n + kWindow - 1) / kWindow, 256, 0,
             static_cast<const u64*>(grouped), n, L.rank, L.flags);
    }
    u64 active = read_scalar(0);
    if (rare.count > 0) active += c.host_scalars[45];
    if (runs_on) {
      // Members of long runs: sub-group rows and ranks, and the rows in
      // sub-groups of two or more appended to the active list.
      launch("run_heads", u64(run_count) * 8, run_heads_kernel, (run_count + 255) / 256, 256, 0,
             L.run_recs, run_count, static_cast<const u32*>(L.rank));
      launch("run_split", run_members * 12, run_split_kernel, grid_stride_blocks(run_members, 256),
             256, 0, static_cast<const RunRecord*>(L.run_recs), run_count,
             static_cast<const RunClass*>(L.run_classes), static_cast<const u32*>(L.run_len),
             static_cast<const u64*>(L.run_prefix), symbols, run_members, n, sa, L.rank, L.x,
             active, L.flags);
      active += run_active;
    }
    if (sa_out && sa_out != sa) {
      SG_CUDA(cudaMemcpyAsync(sa_out, sa, n * 4, cudaMemcpyDeviceToDevice, c.stream));
      spare = sa;  // the scratch buffer the sort ended in is free again
      sa = sa_out;
    }
    st.active_first = active;
    seed_length = symbols;
    return active;
  }


  // ---- Doubling rounds.  Device round state lives in L.scalars:
  // [16]/[17] the active count read / written by a round (they alternate),
  // [18] h, [19] abort (a round whose groups need the host), [20]/[21]
  // totals (active rows, rounds).  The kernels read the count there and are
  // launched for an upper bound, so rounds can run without the host.
  static constexpr int kCountA = 16, kCountB = 17, kH = 18, kAbort = 19, kTotals = 20;

  u32* ghead() const { return L.y; }
  u32* gstart() const { return L.y + (n - n / 2); }  // G <= active/2 <= n/2 each

  RoundState round_state(int in, bool graph) {
    return RoundState{L.scalars + in, L.scalars + (in == kCountA ? kCountB : kCountA),
                      L.scalars + kH, graph ? L.scalars + kAbort : nullptr,
                      L.scalars + kTotals, 1u};
  }

  // Round step 1 (composite keys) for up to `bound` active rows.
  void round_keys(const u32* act, u32* other, const RoundState& rs, u64 bound,
                  const u64* inst_h, Segments segs) {
    const u64 tiles = (bound + kScanTile - 1) / kScanTile;
    zero(L.status, (tiles + 1) * 8);
    zero(L.counters, 4);
    launch("round_keys", bound * 28, round_keys_kernel, tiles, kScanBlock, 0, act, rs,
           static_cast<const u32*>(L.rank), inst_h, segs, bits_for(n), L.k0, other, ghead(),
           gstart(), u64(n / 2), L.status, L.counters, L.scalars + 1, L.flags,
           inst_h ? RunIndex{} : run_index);
  }

  // Shared-memory group sort: (k0, other) -> (k1, act).  abort: the device
  // abort word (graph rounds) or null.
  void round_seg_sort(const u32* other, u32* act, const RoundState& rs, u64 bound, u64* abort,
                      u64 tag) {
    zero(L.counters + 48, 4);
    launch("seg_sort", bound * 24, c.tune.seg_blocks == 3 ? seg_sort_kernel<3> : seg_sort_kernel<2>,
           (bound + kSegWindow - 1) / kSegWindow,
           kSegBlock, sizeof(SegSortSmem), static_cast<const u64*>(L.k0), other, rs.count,
           static_cast<const u32*>(gstart()), static_cast<const u64*>(L.scalars + 1),
           bits_for(n), L.k1, act, L.counters + 48, abort, tag, L.flags, c.tune.seg_small_group);
  }

  // Fused group sort and round step 2: (k0, other) -> SA rows, ranks and the
  // next active list in act (*big > 0: a window did not fit; the host redoes
  // the round).  abort: the device abort word (graph rounds) or null.
  void round_seg_rank(const u32* other, u32* act, const RoundState& rs, u64 bound, u64* abort,
                      u64 tag) {
    const u64 windows = (bound + kSegWindow - 1) / kSegWindow;
    zero(L.status, (windows + 1) * 8);
    zero(L.counters, 4);
    zero(L.counters + 48, 4);
    launch("seg_rank", bound * 36, seg_rank_kernel, windows, kSegBlock, sizeof(SegRankSmem),
           static_cast<const u64*>(L.k0), static_cast<const u32*>(other), rs,
           static_cast<const u32*>(gstart()), static_cast<const u32*>(ghead()),
           static_cast<const u64*>(L.scalars + 1), u64(n / 2), bits_for(n), rank_rows, sa, L.rank,
           act, L.status, L.counters, L.counters + 48, abort, tag, L.flags, c.tune.seg_small_group);
  }

  // The round's h doubling and totals after seg_rank (graph rounds).
  void round_close(const RoundState& rs) {
    launch("round_close", 0, round_close_kernel, 1, 1, 0, rs);
  }

  bool fused_rounds() const { return c.tune.seg_sort && c.tune.seg_rank; }

  // Global passes over (id, second) bits for `active` rows: (k0, other) ->
  // (k1, act) or back in place; returns true when the result is in (k1, act).
  bool round_global_sort(u32* act, u32* other, u64 active) {
    const u32 id_bits = bits_for(active / 2 > 0 ? active / 2 - 1 : 0);
    const u32 t = static_cast<u32>((active + c.tune.sort_tile - 1) / c.tune.sort_tile);
    const u64 b2[2] = {0, active};
    const u32 t2[2] = {0, t};
    sync();
    std::memcpy(c.host_small + 4096, b2, 16);
    std::memcpy(c.host_small + 4096 + 16, t2, 8);
    SG_CUDA(cudaMemcpyAsync(L.sort_begin, c.host_small + 4096, 16, cudaMemcpyHostToDevice, c.stream));
    SG_CUDA(cudaMemcpyAsync(L.sort_tiles, c.host_small + 4096 + 16, 8, cudaMemcpyHostToDevice, c.stream));
    return radix_sort("round_onesweep", L.k0, other, L.k1, act, L.sort_begin, L.sort_tiles, 1, t,
                      active, 0, bits_for(n) + id_bits, false);
  }

  // Round step 2 (ranks, SA rows, next active list) from (ck, cv) into next.
  void round_rank(const u64* ck, const u32* cv, u32* next, const RoundState& rs, u64 bound) {
    const u64 tiles = (bound + kScanTile - 1) / kScanTile;
    zero(L.status, 2 * (tiles + 1) * 8);
    zero(L.counters, 4);
    launch("round_rank", bound * 32, round_rank_kernel, tiles, kScanBlock, 0, ck, cv, rs,
           bits_for(n), static_cast<const u32*>(ghead()), static_cast<const u32*>(gstart()),
           u64(n / 2), rank_rows, sa, L.rank, next, L.status, L.status + tiles + 1, L.counters,
           L.flags);
  }

  void put_scalar(int slot, u64 value) {
    c.host_scalars[40 + slot - kCountA] = value;
    SG_CUDA(cudaMemcpyAsync(L.scalars + slot, c.host_scalars + 40 + slot - kCountA, 8,
                            cudaMemcpyHostToDevice, c.stream));
  }

  // ---- One doubling round over the active list act[0, active), driven by
  // the host: prefix h (or per-segment lengths inst_h with the segment table
  // `segs`).  The next active list replaces act (act/other swap roles as
  // needed).  Returns the next active count.
  u64 round_step(u32*& act, u32*& other, u64 active, u64 h, const u64* inst_h,
                 Segments segs) {
    st.active_rows += active;
    put_scalar(kCountA, active);
    put_scalar(kH, h);
    RoundState rs = round_state(kCountA, false);
    rs.totals = nullptr;
    rs.double_h = 0;
    round_keys(act, other, rs, active, inst_h, segs);
    // Rows only move inside their groups: sort whole groups in shared memory
    // (segsort.cuh) unless some group is too large for a block, in which case
    // the round takes the global passes over (id, second) bits.
    if (fused_rounds()) {
      round_seg_rank(other, act, rs, active, nullptr, 0);
      SG_CUDA(cudaMemcpyAsync(c.host_small + 8192, L.counters + 48, 4, cudaMemcpyDeviceToHost,
                              c.stream));
      sync();
      u32 big = 0;
      std::memcpy(&big, c.host_small + 8192, 4);
      if (big == 0) return read_scalar(kCountB);  // next active list in act
      ++st.seg_sort_fallbacks;
      const bool sw = round_global_sort(act, other, active);
      u64* ck = sw ? L.k1 : L.k0;
      u32* cv = sw ? act : other;
      u32* next = sw ? other : act;
      round_rank(ck, cv, next, rs, active);
      const u64 next_count = read_scalar(kCountB);
      other = sw ? act : other;
      act = next;
      return next_count;
    }
    bool sw = false;
    bool sorted = false;
    if (c.tune.seg_sort) {
      round_seg_sort(other, act, rs, active, nullptr, 0);
      SG_CUDA(cudaMemcpyAsync(c.host_small + 8192, L.counters + 48, 4, cudaMemcpyDeviceToHost,
                              c.stream));
      sync();
      u32 big = 0;
      std::memcpy(&big, c.host_small + 8192, 4);
      if (big == 0) {
        sw = true;
        sorted = true;
      } else {
        ++st.seg_sort_fallbacks;
      }
    }
    if (!sorted) sw = round_global_sort(act, other, active);
    u64* ck = sw ? L.k1 : L.k0;
    u32* cv = sw ? act : other;
    u32* next = sw ? other : act;
    round_rank(ck, cv, next, rs, active);
    const u64 next_count = read_scalar(kCountB);  // synchronizes: host_small may be reused
    other = sw ? act : other;
    act = next;
    return next_count;
  }

  // ---- Host-free rounds: two rounds (their buffers swap roles twice, so the
  // pair returns to its starting roles) captured once as a CUDA graph for an
  // upper bound on the active count and launched until the count reaches
  // zero, one synchronization per pair.  A round whose groups do not fit the
  // shared-memory sort stops the pair (abort); the host finishes that round
  // with the global passes and the graph continues from there.
  // The graph of a round pair for `bound` active rows with these buffers:
  // from the context's cache when an earlier build had the same layout and
  // the same round knobs, else captured and cached.
  const sufgpu_ctx::CachedGraph& round_graph(u32* act, u32* other, u64 bound) {
    const std::vector<u64> key = {reinterpret_cast<u64>(c.arena.base), n, segs, bound,
                                  reinterpret_cast<u64>(act), reinterpret_cast<u64>(other),
                                  run_count, reinterpret_cast<u64>(L.seg_begin),
                                  u64(fused_rounds()), u64(c.tune.seg_small_group),
                                  u64(c.tune.seg_blocks)};
    auto& cache = c.round_graphs;
    for (size_t i = 0; i < cache.size(); ++i) {
      if (cache[i].key == key) {
        std::rotate(cache.begin() + i, cache.begin() + i + 1, cache.end());
        return cache.back();
      }
    }
    const u32 before = c.launches;
    SG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
      for (int r = 0; r < 2; ++r) {
        const RoundState rs = round_state(r == 0 ? kCountA : kCountB, true);
        round_keys(act, other, rs, bound, nullptr, segments());
        if (fused_rounds()) {
          // The next active list replaces act: no buffer swap.
          round_seg_rank(other, act, rs, bound, L.scalars + kAbort, r + 1);
          round_close(rs);
        } else {
          round_seg_sort(other, act, rs, bound, L.scalars + kAbort, r + 1);
          round_rank(L.k1, act, other, rs, bound);
          std::swap(act, other);
        }
      }
    } catch (...) {
      cudaStreamEndCapture(c.stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      c.launches = before;
      throw;
    }
    SG_CUDA(cudaStreamEndCapture(c.stream, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    SG_CUDA(err);
    const u32 kernels = c.launches - before;
    c.launches = before;
    if (cache.size() >= 8) {
      cudaGraphExecDestroy(cache.front().exec);
      cache.erase(cache.begin());
    }
    cache.push_back(sufgpu_ctx::CachedGraph{key, exec, kernels});
    return cache.back();
  }

  void graph_rounds(u32*& act, u32*& other, u64 active, u64 h) {
    put_scalar(kCountA, active);
    put_scalar(kH, h);
    zero(L.scalars + kAbort, 24);  // abort and the two totals
    // Bounds are powers of two, so builds of similar sizes share graphs.
    auto pow2 = [](u64 v) { return u64(1) << bits_for(v > 1 ? v - 1 : 1); };
    u64 bound = pow2(active);
    u64 fallback_rows = 0, fallback_rounds = 0;
    for (u32 pairs = 0;; ++pairs) {
      if (pairs > 64) throw BuildError{SUFGPU_BUILD_FAILURE, "prefix doubling did not converge"};
      const sufgpu_ctx::CachedGraph& g = round_graph(act, other, std::min<u64>(bound, n));
      SG_CUDA(cudaGraphLaunch(g.exec, c.stream));
      c.launches += g.kernels;
      SG_CUDA(cudaMemcpyAsync(c.host_scalars + kCountA, L.scalars + kCountA, 32,
                              cudaMemcpyDeviceToHost, c.stream));
      sync();
      const u64 abort = c.host_scalars[kAbort];
      if (abort) {
        // Round abort-1 of the pair stopped after its keys; rounds before it
        // are complete.  Its active count is in A (first round) or B.
        ++st.seg_sort_fallbacks;
        const int in = abort == 1 ? kCountA : kCountB;
        // Unfused pairs swap the buffers once per round; fused ones never.
        if (abort == 2 && !fused_rounds()) std::swap(act, other);
        const u64 count = c.host_scalars[in];
        fallback_rows += count;
        ++fallback_rounds;
        const bool sw = round_global_sort(act, other, count);
        RoundState rs = round_state(in, false);
        rs.totals = nullptr;
        u64* ck = sw ? L.k1 : L.k0;
        u32* cv = sw ? act : other;
        u32* next = sw ? other : act;
        round_rank(ck, cv, next, rs, count);
        other = sw ? act : other;
        act = next;
        // Continue from a clean state: the next count in A, abort cleared.
        const u64 next_count = read_scalar(in == kCountA ? kCountB : kCountA);
        put_scalar(kCountA, next_count);
        zero(L.scalars + kAbort, 8);
        if (next_count == 0) break;
        bound = std::min(bound, pow2(next_count));
        continue;
      }
      const u64 count = c.host_scalars[kCountA];
      if (count == 0) break;
      // A much smaller count than the graph's bound wastes empty blocks:
      // switch to the graph of a smaller bound.
      if (count < bound / c.tune.graph_shrink) bound = pow2(count);
    }
    SG_CUDA(cudaMemcpyAsync(c.host_scalars + kTotals, L.scalars + kTotals, 16,
                            cudaMemcpyDeviceToHost, c.stream));
    sync();
    st.active_rows += c.host_scalars[kTotals] + fallback_rows;
    st.rounds = static_cast<u32>(c.host_scalars[kTotals + 1] + fallback_rounds);
  }

  // True when a recent build had this build's layout (and remembers it).
  bool layout_seen() {
    const std::vector<u64> key = {reinterpret_cast<u64>(c.arena.base), n, segs, run_count,
                                  reinterpret_cast<u64>(spare)};
    auto& seen = c.seen_layouts;
    for (size_t i = 0; i < seen.size(); ++i) {
      if (seen[i] == key) return true;
    }
    if (seen.size() >= 16) seen.erase(seen.begin());
    seen.push_back(key);
    return false;
  }

  // ---- The doubling sort: leaves SA in `sa` and ISA (global rows) in rank.
  void suffix_sort() {
    allow_runs = true;
    allow_two_bit = true;
    u64 active = seed_phase();
    // Rounds.  act and other alternate between x and the spare SA-sized
    // buffer; y holds the per-group tables.
    u32* act = L.x;
    u32* other = spare;
    u64 h = seed_length;
    if (active > 0 && c.tune.graph_rounds && c.tune.seg_sort && !c.profiling && layout_seen()) {
      graph_rounds(act, other, active, h);
      return;
    }
    u32 rounds = 0;
    while (active > 0) {
      if (++rounds > 64) throw BuildError{SUFGPU_BUILD_FAILURE, "prefix doubling did not converge"};
      active = round_step(act, other, active, h, nullptr, segments());
      h *= 2;
    }
    st.rounds = rounds;
  }

  // ---- LCP phase: final row-order LCP (u32) in the first half of k1.  The
  // position-sorted long irreducible rows stay in k0 (positions) and the
  // second half of k1 (values) for the anchor pass; their count is returned.
  struct LcpPhase {
    u32* lcp;
    const u64* sorted_pos;
    const u32* sorted_val;
    u64 longs;
  };
  LcpPhase lcp_phase() {
    u32* lcp = L.lcp;
    LongRow* longs = reinterpret_cast<LongRow*>(L.x);  // x and y: 8n bytes
    const u64 long_cap = std::max<u64>(n, 1) * 8 / sizeof(LongRow);
    u32* pending = spare;
    const u64 pending_cap = n;
    zero(L.scalars + 5, 16);
    launch("lcp_rows", n * 4 + st.active_first * 9, lcp_rows_kernel,
           grid_stride_blocks((n + kLcpChunk / 32 - 1) / (kLcpChunk / 32), kLcpRowsBlock),
           kLcpRowsBlock, 0, L.text, static_cast<const u32*>(sa), n, segments(), seed_length, lcp, longs,
           long_cap, L.scalars + 5, pending, pending_cap, L.scalars + 6, L.flags);
    SG_CUDA(cudaMemcpyAsync(c.host_scalars + 5, L.scalars + 5, 16, cudaMemcpyDeviceToHost, c.stream));
    sync();
    const u64 q_all = c.host_scalars[5], pend_all = c.host_scalars[6];
    if (q_all > long_cap || pend_all > pending_cap) {
      throw BuildError{SUFGPU_BUILD_FAILURE, "long-LCP queue overflow"};
    }
    const u64 q = q_all;
    st.irreducible_long = q;
    u64* spos = L.k0;
    u64* spos_alt = L.k0 + n / 2 + 1;
    u32* sval = reinterpret_cast<u32*>(L.k1);
    u32* sval_alt = sval + n / 2 + 1;
    const u64* sorted_pos = spos;
    const u32* sorted_val = sval;
    if (q > 0) {
      launch("long_rows", 0, long_rows_kernel, u64(c.sm_count) * 8, 256, 0, L.text,
             static_cast<const LongRow*>(longs), static_cast<const u64*>(L.scalars + 5),
             long_cap, segments(), lcp, spos, sval);
      const u32 t = static_cast<u32>((q + c.tune.sort_tile - 1) / c.tune.sort_tile);
      const u64 b2[2] = {0, q};
      const u32 t2[2] = {0, t};
      std::memcpy(c.host_small + 4096, b2, 16);
      std::memcpy(c.host_small + 4096 + 16, t2, 8);
      SG_CUDA(cudaMemcpyAsync(L.sort_begin, c.host_small + 4096, 16, cudaMemcpyHostToDevice, c.stream));
      SG_CUDA(cudaMemcpyAsync(L.sort_tiles, c.host_small + 4096 + 16, 8, cudaMemcpyHostToDevice, c.stream));
      const bool sw = radix_sort("long_sort", spos, sval, spos_alt, sval_alt, L.sort_begin,
                                 L.sort_tiles, 1, t, q, 0, std::max<u32>(1, bits_for(n)), false);
      if (sw) {
        sorted_pos = spos_alt;
        sorted_val = sval_alt;
      }
    }
    if (pend_all > 0) {
      if (q == 0) throw BuildError{SUFGPU_BUILD_FAILURE, "reducible long row without an anchor row"};
      launch("pending_rows", pend_all * 16, pending_rows_kernel, grid_stride_blocks(pend_all, 256),
             256, 0, static_cast<const u32*>(sa), static_cast<const u32*>(pending),
             static_cast<const u64*>(L.scalars + 6), pending_cap, sorted_pos, sorted_val,
             static_cast<const u64*>(L.scalars + 5), long_cap, lcp, L.flags);
    }
    return LcpPhase{lcp, sorted_pos, sorted_val, q};
  }
};

sufgpu_status fail(sufgpu_ctx* ctx, sufgpu_status s, const std::string& m) {
  if (ctx) ctx->last_error = m;
  return s;
}

bool valid_width(u32 bits) { return bits == 32 || bits == 40 || bits == 48 || bits == 64; }

// Copies `bytes` from device src to dst (host or device) on the stream.
void copy_out(sufgpu_ctx& c, void* dst, const void* src, u64 bytes) {
  if (!dst || bytes == 0) return;
  SG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c.stream));
}

// Plane slots of Engine::plane_crc.
enum : int { kCrcSaLow = 0, kCrcSaHigh, kCrcIsaLow, kCrcIsaHigh, kCrcLcp };

// copy_out of a whole plane (device source), with its CRC-32 when asked.
void copy_plane(Engine& e, void* dst, const void* src, u64 bytes, int slot) {
  copy_out(e.c, dst, src, bytes);
  if (e.want_crc && dst) e.st.plane_crc[slot] = e.crc32_device(src, bytes, 0, reinterpret_cast<u32*>(e.L.status));
}

u64 high_bytes(u32 bits, u64 rows) { return bits == 40 ? rows : bits == 48 ? 2 * rows : 0; }

// Everything after the sort: ISA and SA packing, validation, LCP (raw or
// byte-coded with anchors) and the copies into each instance's planes.
// Sampled outputs (rate K > 1): complete SA, ISA and row LCP first, then the
// kept rows (sample_kernel) packed into each instance's planes of
// ceil(n_i / K) rows.
void emit_sampled(Engine& e, const sufgpu_build_desc& d, sufgpu_outputs* outs,
                  sufgpu_anchors* anchors, u32 count) {
  sufgpu_ctx& c = e.c;
  Layout& L = e.L;
  const u64 n = e.n;
  const u32 rate = d.sampling_rate;
  if (d.flags & SUFGPU_FLAG_VALIDATE) {
    e.launch("validate", n * 8, validate_kernel, e.grid_stride_blocks(n, 256), 256, 0, e.sa,
             L.rank, n, e.segments(), L.flags);
  }
  SG_CUDA(cudaEventRecord(c.ev[3], c.stream));
  const bool want_lcp = d.lcp_encoding != SUFGPU_LCP_NONE;
  const u32* lcp = want_lcp ? e.lcp_phase().lcp : nullptr;
  // Per-instance sampled offsets.
  std::vector<u64> off(count + 1, 0);
  for (u32 j = 0; j < count; ++j) {
    off[j + 1] = off[j] + (e.begin[j + 1] - e.begin[j] + rate - 1) / rate;
  }
  const u64 kept = off[count];
  e.sync();
  std::memcpy(c.host_small, off.data(), (count + 1) * 8);
  SG_CUDA(cudaMemcpyAsync(L.digit_start, c.host_small, (count + 1) * 8, cudaMemcpyHostToDevice,
                          c.stream));
  u32* sa_k = reinterpret_cast<u32*>(L.k0);
  u32* isa_k = sa_k + kept;
  u32* lcp_k = isa_k + kept;
  if (want_lcp) SG_CUDA(cudaMemsetAsync(lcp_k, 0xff, kept * 4, c.stream));
  const u64 tiles = (n + kScanTile - 1) / kScanTile;
  e.zero(L.status, (tiles + 1) * 8);
  e.zero(L.counters, 4);
  e.launch("sample", n * (want_lcp ? 12 : 8) + kept * 12, sample_kernel, tiles, kScanBlock, 0,
           static_cast<const u32*>(e.sa), lcp, n, e.segments(), rate,
           static_cast<const u64*>(L.digit_start), kept, sa_k, isa_k, lcp_k, L.status,
           L.counters, L.flags);
  // Pack and copy: sampled values are instance-local already (one segment).
  const u64 b2[2] = {0, kept};
  std::memcpy(c.host_small + 4096, b2, 16);
  SG_CUDA(cudaMemcpyAsync(L.sort_begin, c.host_small + 4096, 16, cudaMemcpyHostToDevice, c.stream));
  const Segments whole{L.sort_begin, 1};
  u8* low = reinterpret_cast<u8*>(L.k1);
  u8* high = low + kept * 8;
  auto emit = [&](const u32* values, u32 bits, bool isa) {
    const u64 w = bits == 64 ? 8 : 4;
    e.launch("pack", kept * (4 + w + high_bytes(bits, 1)), pack_kernel,
             e.grid_stride_blocks(kept, 256), 256, 0, values, kept, whole, bits,
             static_cast<void*>(low), static_cast<void*>(high));
    for (u32 j = 0; j < count; ++j) {
      const u64 rows = off[j + 1] - off[j];
      const int slot = isa ? kCrcIsaLow : kCrcSaLow;
      copy_plane(e, isa ? outs[j].isa_low : outs[j].sa_low, low + off[j] * w, rows * w, slot);
      if (high_bytes(bits, 1)) {
        copy_plane(e, isa ? outs[j].isa_high : outs[j].sa_high, high + high_bytes(bits, off[j]),
                   high_bytes(bits, rows), slot + 1);
      }
    }
  };
  if (d.isa_storage_bits) emit(isa_k, d.isa_storage_bits, true);
  emit(sa_k, d.sa_storage_bits, false);
  SG_CUDA(cudaEventRecord(c.ev[4], c.stream));
  const bool byte_coded =
      d.lcp_encoding == SUFGPU_LCP_BYTE32 || d.lcp_encoding == SUFGPU_LCP_BYTE64;
  if (want_lcp && !byte_coded) {
    const bool wide = d.lcp_encoding == SUFGPU_LCP_RAW64;
    const u8* src = reinterpret_cast<const u8*>(lcp_k);
    if (wide) {
      e.launch("lcp_widen", kept * 12, widen_kernel<u64>, e.grid_stride_blocks(kept, 256), 256, 0,
               static_cast<const u32*>(lcp_k), kept, reinterpret_cast<u64*>(low));
      src = low;
    }
    const u64 w = wide ? 8 : 4;
    for (u32 j = 0; j < count; ++j) {
      copy_plane(e, outs[j].lcp, src + off[j] * w, (off[j + 1] - off[j]) * w, kCrcLcp);
    }
  } else if (byte_coded) {
    // Primary bytes of the sampled rows, then the anchors in sample order
    // (sampled_anchor_kernel) with per-instance counts after the offsets.
    u8* primary = low;  // the packed SA planes above are copied by now (same stream)
    e.launch("lcp_primary", kept * 5, lcp_primary_kernel, e.grid_stride_blocks(kept, 256), 256,
             0, static_cast<const u32*>(lcp_k), kept, primary);
    for (u32 j = 0; j < count; ++j) {
      copy_plane(e, outs[j].lcp, primary + off[j], off[j + 1] - off[j], kCrcLcp);
    }
    const bool wide = d.lcp_encoding == SUFGPU_LCP_BYTE64;
    const u64 w = wide ? 8 : 4;
    const u64 cap = (std::max<u64>(n, 1) * 4) / w;  // each of x and y holds 4n bytes
    u8* pos = reinterpret_cast<u8*>(L.x);
    u8* val = reinterpret_cast<u8*>(L.y);
    u64* inst_count = L.digit_start + count + 1;
    e.zero(inst_count, u64(count) * 8);
    const u64 atiles = (kept + kScanTile - 1) / kScanTile;
    e.zero(L.scalars + 4, 8);
    e.zero(L.status, (atiles + 1) * 8);
    e.zero(L.counters, 4);
    if (wide) {
      e.launch("anchors", kept * 12, sampled_anchor_kernel<u64>, atiles, kScanBlock, 0,
               static_cast<const u32*>(isa_k), static_cast<const u32*>(lcp_k),
               static_cast<const u64*>(L.digit_start), count, kept, rate,
               reinterpret_cast<u64*>(pos), reinterpret_cast<u64*>(val), cap, inst_count,
               L.status, L.counters, L.scalars + 4, L.flags);
    } else {
      e.launch("anchors", kept * 12, sampled_anchor_kernel<u32>, atiles, kScanBlock, 0,
               static_cast<const u32*>(isa_k), static_cast<const u32*>(lcp_k),
               static_cast<const u64*>(L.digit_start), count, kept, rate,
               reinterpret_cast<u32*>(pos), reinterpret_cast<u32*>(val), cap, inst_count,
               L.status, L.counters, L.scalars + 4, L.flags);
    }
    const u64 total = atiles ? e.read_scalar(4) : 0;
    e.st.anchors = total;
    if (total > cap) throw BuildError{SUFGPU_BUILD_FAILURE, "anchor buffer overflow"};
    std::vector<u64> per(count, 0);
    SG_CUDA(cudaMemcpyAsync(per.data(), inst_count, u64(count) * 8, cudaMemcpyDeviceToHost,
                            c.stream));
    c.anchor_pos.resize(std::max<u64>(total * w, 8));
    c.anchor_val.resize(std::max<u64>(total * w, 8));
    SG_CUDA(cudaMemcpyAsync(c.anchor_pos.data(), pos, total * w, cudaMemcpyDeviceToHost, c.stream));
    SG_CUDA(cudaMemcpyAsync(c.anchor_val.data(), val, total * w, cudaMemcpyDeviceToHost, c.stream));
    e.sync();
    u64 at = 0;
    for (u32 j = 0; j < count; ++j) {
      if (anchors) {
        anchors[j] = sufgpu_anchors{c.anchor_pos.data() + at * w, c.anchor_val.data() + at * w,
                                    per[j], static_cast<u32>(w * 8)};
      }
      at += per[j];
    }
    if (at != total) throw BuildError{SUFGPU_BUILD_FAILURE, "sampled anchor counts disagree"};
  }
  SG_CUDA(cudaEventRecord(c.ev[5], c.stream));
  e.sync();
}

// Fills an output plane of `bytes` zero bytes: on the copy stream for device
// memory, else by host threads (started now, joined before the build ends).
void zero_plane(Engine& e, void* dst, u64 bytes) {
  if (!dst || bytes == 0) return;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, dst) != cudaSuccess) cudaGetLastError();
  if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) {
    SG_CUDA(cudaMemsetAsync(dst, 0, bytes, e.c.copy_stream));
    return;
  }
  const u64 parts = std::max<u64>(1, std::min<u64>(8, bytes >> 26));
  const u64 step = (bytes + parts - 1) / parts;
  for (u64 k = 0; k < parts; ++k) {
    u8* at = static_cast<u8*>(dst) + k * step;
    const u64 len = std::min(step, bytes - std::min(bytes, k * step));
    if (len) e.c.fillers.emplace_back([at, len] { std::memset(at, 0, len); });
  }
}

// CHILD table of the row LCP (child.cuh) into dst (host or device): the
// minima tree and the nse/up/down arrays in k0/k1 (free once the LCP planes
// are out), the table staged in x.
void emit_child(Engine& e, const u32* lcp, void* dst) {
  Layout& L = e.L;
  const u64 n = e.n;
  u32* nse = reinterpret_cast<u32*>(L.k0);
  u32* down = nse + n;
  u32* up = reinterpret_cast<u32*>(L.k1);
  u32* tree = up + n;
  MinTree t{};
  t.level[0] = lcp;
  t.size[0] = n;
  t.levels = 1;
  u32* at = tree;
  while (t.size[t.levels - 1] > kChildFan) {
    if (t.levels >= kChildMaxLevels) throw BuildError{SUFGPU_BUILD_FAILURE, "CHILD tree too deep"};
    const u64 below = t.size[t.levels - 1];
    const u64 size = (below + kChildFan - 1) / kChildFan;
    e.launch("child_tree", below * 4 + size * 4, child_min_level_kernel,
             e.grid_stride_blocks(size, 256), 256, 0, t.level[t.levels - 1], below, at, size);
    t.level[t.levels] = at;
    t.size[t.levels] = size;
    ++t.levels;
    at += size;
  }
  e.zero(down, n * 4);
  SG_CUDA(cudaMemsetAsync(up, 0xff, n * 4, e.c.stream));  // > every row: atomicMin start
  e.launch("child_links", n * 12, child_links_kernel, e.grid_stride_blocks(n, 256), 256, 0, t,
           nse, down, up);
  u32* child = L.x;
  e.launch("child_final", n * 20, child_final_kernel, e.grid_stride_blocks(n, 256), 256, 0, lcp,
           n, static_cast<const u32*>(nse), static_cast<const u32*>(down),
           static_cast<const u32*>(up), child);
  copy_out(e.c, dst, child, n * 4);
}

void emit_outputs(Engine& e, const sufgpu_build_desc& d, sufgpu_outputs* outs,
                  sufgpu_anchors* anchors, u32 count) {
  sufgpu_ctx& c = e.c;
  Layout& L = e.L;
  const u64 n = e.n;
  if (d.sampling_rate > 1) {
    emit_sampled(e, d, outs, anchors, count);
    return;
  }

  // ISA: rank holds global rows.  Stage packed planes in k0/k1 when the
  // layout differs from the device one, then copy each instance's rows.
  const bool want_isa = d.isa_storage_bits != 0;
  // A gated build (collection worker) without ISA, with a 32-bit SA and raw or
  // no LCP computes every plane first (the packed SA staged in rank, free
  // once validated) and leaves the gate before its copies.
  const bool raw_lcp = d.lcp_encoding == SUFGPU_LCP_RAW32 || d.lcp_encoding == SUFGPU_LCP_RAW64;
  if (e.gate && !want_isa && d.sa_storage_bits == 32 &&
      (raw_lcp || d.lcp_encoding == SUFGPU_LCP_NONE) && !e.want_crc) {
    SG_CUDA(cudaEventRecord(c.ev[3], c.stream));
    if (d.flags & SUFGPU_FLAG_VALIDATE) {
      e.launch("validate", n * 8, validate_kernel, e.grid_stride_blocks(n, 256), 256, 0, e.sa,
               L.rank, n, e.segments(), L.flags);
    }
    const bool direct = count == 1;
    const u32* sa_plane = e.sa;
    if (!direct) {
      e.launch("pack", n * 8, pack_kernel, e.grid_stride_blocks(n, 256), 256, 0, e.sa, n,
               e.segments(), 32u, static_cast<void*>(L.rank), static_cast<void*>(nullptr));
      sa_plane = L.rank;
    }
    SG_CUDA(cudaEventRecord(c.ev[4], c.stream));
    const u8* lcp_src = nullptr;
    const u64 lw = d.lcp_encoding == SUFGPU_LCP_RAW64 ? 8 : 4;
    if (raw_lcp) {
      const Engine::LcpPhase ph = e.lcp_phase();
      lcp_src = reinterpret_cast<const u8*>(ph.lcp);
      if (lw == 8) {
        e.launch("lcp_widen", n * 12, widen_kernel<u64>, e.grid_stride_blocks(n, 256), 256, 0,
                 static_cast<const u32*>(ph.lcp), n, L.k0);
        lcp_src = reinterpret_cast<const u8*>(L.k0);
      }
    }
    e.gate_leave();
    for (u32 j = 0; j < count; ++j) {
      const u64 b = e.begin[j], rows = e.begin[j + 1] - e.begin[j];
      copy_out(c, outs[j].sa_low, sa_plane + b, rows * 4);
      if (lcp_src) copy_out(c, outs[j].lcp, lcp_src + b * lw, rows * lw);
    }
    SG_CUDA(cudaEventRecord(c.ev[5], c.stream));
    return;
  }
  auto emit = [&](const u32* values, u32 bits, bool isa) {
    const bool direct = bits == 32 && count == 1;
    u8* low = reinterpret_cast<u8*>(L.k0);
    u8* high = reinterpret_cast<u8*>(L.k1);
    if (!direct) {
      e.launch("pack", n * (4 + (bits == 64 ? 8 : 4) + high_bytes(bits, 1)), pack_kernel,
               e.grid_stride_blocks(n, 256), 256, 0, values, n,
               e.segments(), bits, static_cast<void*>(low), static_cast<void*>(high));
    }
    for (u32 j = 0; j < count; ++j) {
      const u64 b = e.begin[j], rows = e.begin[j + 1] - e.begin[j];
      void* dst_low = isa ? outs[j].isa_low : outs[j].sa_low;
      void* dst_high = isa ? outs[j].isa_high : outs[j].sa_high;
      const u64 w = bits == 64 ? 8 : 4;
      const int slot = isa ? kCrcIsaLow : kCrcSaLow;
      if (direct) copy_plane(e, dst_low, values + b, rows * 4, slot);
      else copy_plane(e, dst_low, low + b * w, rows * w, slot);
      if (!direct && high_bytes(bits, 1)) {
        copy_plane(e, dst_high, high + b * high_bytes(bits, 1), high_bytes(bits, rows), slot + 1);
      }
    }
  };
  // A single build whose coordinates fit 32 bits copies its 32/40/48-bit SA
  // and ISA low planes straight from the device arrays on the copy stream,
  // so the copies run under the LCP phase; their high planes are all zero
  // and are filled without a copy.  64-bit planes are packed and copied on
  // the compute stream.
  const bool overlap = count == 1 && !e.want_crc && n <= 0xffffffffull;
  auto fits32 = [](u32 bits) { return bits == 32 || bits == 40 || bits == 48; };
  if (overlap) {
    if (want_isa && !fits32(d.isa_storage_bits)) emit(L.rank, d.isa_storage_bits, true);
    SG_CUDA(cudaEventRecord(c.ev[3], c.stream));
    if (d.flags & SUFGPU_FLAG_VALIDATE) {
      e.launch("validate", n * 8, validate_kernel, e.grid_stride_blocks(n, 256), 256, 0, e.sa,
               L.rank, n, e.segments(), L.flags);
    }
    if (!fits32(d.sa_storage_bits)) emit(e.sa, d.sa_storage_bits, false);
    SG_CUDA(cudaEventRecord(c.copy_ready, c.stream));
    SG_CUDA(cudaStreamWaitEvent(c.copy_stream, c.copy_ready, 0));
    if (want_isa && fits32(d.isa_storage_bits)) {
      SG_CUDA(cudaMemcpyAsync(outs[0].isa_low, L.rank, n * 4, cudaMemcpyDefault, c.copy_stream));
      zero_plane(e, outs[0].isa_high, high_bytes(d.isa_storage_bits, n));
    }
    if (fits32(d.sa_storage_bits)) {
      SG_CUDA(cudaMemcpyAsync(outs[0].sa_low, e.sa, n * 4, cudaMemcpyDefault, c.copy_stream));
      zero_plane(e, outs[0].sa_high, high_bytes(d.sa_storage_bits, n));
    }
    SG_CUDA(cudaEventRecord(c.ev[4], c.stream));
  } else {
    if (want_isa) emit(L.rank, d.isa_storage_bits, true);
    SG_CUDA(cudaEventRecord(c.ev[3], c.stream));
    if (d.flags & SUFGPU_FLAG_VALIDATE) {
      e.launch("validate", n * 8, validate_kernel, e.grid_stride_blocks(n, 256), 256, 0, e.sa,
               L.rank,
               n, e.segments(), L.flags);
    }
    emit(e.sa, d.sa_storage_bits, false);
    SG_CUDA(cudaEventRecord(c.ev[4], c.stream));
  }

  // LCP.
  if (d.lcp_encoding != SUFGPU_LCP_NONE) {
    const Engine::LcpPhase ph = e.lcp_phase();
    if (d.lcp_encoding == SUFGPU_LCP_RAW32 || d.lcp_encoding == SUFGPU_LCP_RAW64) {
      const bool wide = d.lcp_encoding == SUFGPU_LCP_RAW64;
      const u8* src = reinterpret_cast<const u8*>(ph.lcp);
      if (wide) {
        e.launch("lcp_widen", n * 12, widen_kernel<u64>, e.grid_stride_blocks(n, 256), 256, 0,
                 static_cast<const u32*>(ph.lcp), n, L.k0);
        src = reinterpret_cast<const u8*>(L.k0);
      }
      const u64 w = wide ? 8 : 4;
      for (u32 j = 0; j < count; ++j) {
        const u64 b = e.begin[j], rows = e.begin[j + 1] - e.begin[j];
        copy_plane(e, outs[j].lcp, src + b * w, rows * w, kCrcLcp);
      }
    } else {
      const bool wide = d.lcp_encoding == SUFGPU_LCP_BYTE64;
      u8* primary = reinterpret_cast<u8*>(e.spare);
      e.launch("lcp_primary", n * 5, lcp_primary_kernel, e.grid_stride_blocks(n, 256), 256, 0,
               static_cast<const u32*>(ph.lcp), n, primary);
      for (u32 j = 0; j < count; ++j) {
        const u64 b = e.begin[j], rows = e.begin[j + 1] - e.begin[j];
        copy_plane(e, outs[j].lcp, primary + b, rows, kCrcLcp);
      }
      // Anchors into x/y (8n bytes): a filter of the sorted long rows.
      const u64 w = wide ? 8 : 4;
      const u64 cap = (std::max<u64>(n, 1) * 8) / (2 * w);
      u8* pos = reinterpret_cast<u8*>(L.x);
      u8* val = pos + cap * w;
      const u64 tiles = (ph.longs + kScanTile - 1) / kScanTile;
      e.zero(L.scalars + 4, 8);
      e.zero(L.status, (tiles + 1) * 8);
      e.zero(L.counters, 4);
      if (wide) {
        e.launch("anchors", ph.longs * 24, anchor_kernel<u64>, tiles, kScanBlock, 0,
                 ph.sorted_pos, ph.sorted_val, static_cast<const u64*>(L.scalars + 5),
                 n, e.segments(), static_cast<const u32*>(L.rank),
                 static_cast<const u32*>(ph.lcp), reinterpret_cast<u64*>(pos),
                 reinterpret_cast<u64*>(val), cap, L.status, L.counters, L.scalars + 4, L.flags);
      } else {
        e.launch("anchors", ph.longs * 24, anchor_kernel<u32>, tiles, kScanBlock, 0,
                 ph.sorted_pos, ph.sorted_val, static_cast<const u64*>(L.scalars + 5),
                 n, e.segments(), static_cast<const u32*>(L.rank),
                 static_cast<const u32*>(ph.lcp), reinterpret_cast<u32*>(pos),
                 reinterpret_cast<u32*>(val), cap, L.status, L.counters, L.scalars + 4, L.flags);
      }
      const u64 total = e.read_scalar(4);
      e.st.anchors = total;
      if (total > cap) throw BuildError{SUFGPU_BUILD_FAILURE, "anchor buffer overflow"};
      c.anchor_pos.resize(std::max<u64>(total * w, 8));
      c.anchor_val.resize(std::max<u64>(total * w, 8));
      SG_CUDA(cudaMemcpyAsync(c.anchor_pos.data(), pos, total * w, cudaMemcpyDeviceToHost, c.stream));
      SG_CUDA(cudaMemcpyAsync(c.anchor_val.data(), val, total * w, cudaMemcpyDeviceToHost, c.stream));
      e.sync();
      // Anchors arrive in global text order, so each instance owns one
      // contiguous run; convert its positions to instance coordinates.
      if (anchors) {
        u64 at = 0;
        for (u32 j = 0; j < count; ++j) {
          const u64 first = at;
          while (at < total) {
            const u64 p = wide ? reinterpret_cast<u64*>(c.anchor_pos.data())[at]
                               : reinterpret_cast<u32*>(c.anchor_pos.data())[at];
            if (p >= e.begin[j + 1]) break;
            const u64 local = p - e.begin[j];
            if (wide) reinterpret_cast<u64*>(c.anchor_pos.data())[at] = local;
            else reinterpret_cast<u32*>(c.anchor_pos.data())[at] = static_cast<u32>(local);
            ++at;
          }
          anchors[j] = sufgpu_anchors{c.anchor_pos.data() + first * w,
                                      c.anchor_val.data() + first * w, at - first,
                                      static_cast<u32>(w * 8)};
        }
      }
    }
    if (d.flags & SUFGPU_FLAG_CHILD) emit_child(e, ph.lcp, outs[0].child);
  }
  if (overlap) {  // the compute stream ends after the overlapped copies
    SG_CUDA(cudaEventRecord(c.copy_done, c.copy_stream));
    SG_CUDA(cudaStreamWaitEvent(c.stream, c.copy_done, 0));
  }
  SG_CUDA(cudaEventRecord(c.ev[5], c.stream));
  e.sync();
  e.join_fillers();
}

// The knobs of one build: the context's, overridden by the first size class
// that holds the build's longest instance; restored when the build ends.
struct TuningScope {
  sufgpu_ctx& c;
  Tuning saved;
  TuningScope(sufgpu_ctx& ctx, u64 longest) : c(ctx), saved(ctx.tune) {
    for (const TuningClass& k : ctx.tuning_classes) {
      if (longest > k.max_symbols) continue;
      for (const auto& kv : k.settings) apply_tuning(ctx.tune, kv.first, kv.second);
      break;
    }
  }
  ~TuningScope() { c.tune = saved; }
};

// The Fast index's k-mer prefix directory from the final SA (prefixdir.cuh),
// staged in k1 (free until the outputs are packed) and copied out at once.
void emit_prefix_directory(Engine& e, const sufgpu_build_desc& d, const sufgpu_outputs& out) {
  sufgpu_ctx& c = e.c;
  Layout& L = e.L;
  const u64 entries = u64(1) << (2 * d.prefix_k);
  u64* table = L.k1;
  e.launch("prefix_fill", entries * 8, prefix_fill_kernel, e.grid_stride_blocks(entries, 256),
           256, 0, table, entries, e.n | (e.n << 32));
  e.zero(L.scalars + 24, 16);
  e.launch("prefix_directory", e.n * (4 + d.prefix_k) + entries * 8, prefix_directory_kernel,
           (e.n + kDirTile - 1) / kDirTile, kDirTile, 0, static_cast<const u8*>(L.text),
           static_cast<const u32*>(e.sa), e.n, d.prefix_k, table,
           reinterpret_cast<unsigned long long*>(L.scalars + 24), L.flags);
  copy_out(c, out.prefix_intervals, table, entries * 8);
  SG_CUDA(cudaMemcpyAsync(c.host_scalars + 24, L.scalars + 24, 16, cudaMemcpyDeviceToHost,
                          c.stream));
  e.sync();
  e.st.prefix_kmers = c.host_scalars[24];
  e.st.prefix_entries = c.host_scalars[25];
}

// Shared build body for one or many instances (already concatenated in
// L.text).  outs[j] receives instance j's planes.
void run_build(Engine& e, const sufgpu_build_desc& d, sufgpu_outputs* outs,
               sufgpu_anchors* anchors, u32 count) {
  SG_CUDA(cudaEventRecord(e.c.ev[1], e.c.stream));
  e.suffix_sort();
  SG_CUDA(cudaEventRecord(e.c.ev[2], e.c.stream));
  if (d.prefix_k) emit_prefix_directory(e, d, outs[0]);
  emit_outputs(e, d, outs, anchors, count);
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

static thread_local std::string g_create_error;

sufgpu_status sufgpu_create(sufgpu_ctx** out, int device) {
  if (!out) return SUFGPU_INVALID_INPUT;
  *out = nullptr;
  auto* ctx = new sufgpu_ctx();
  try {
    ctx->device = device;
    SG_CUDA(cudaSetDevice(device));
    int sms = 0;
    SG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    ctx->sm_count = sms;
    SG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    SG_CUDA(cudaEventCreateWithFlags(&ctx->copy_ready, cudaEventDisableTiming));
    SG_CUDA(cudaEventCreateWithFlags(&ctx->copy_done, cudaEventDisableTiming));
    SG_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ctx->host_scalars), 64 * 8));
    SG_CUDA(cudaMallocHost(reinterpret_cast<void**>(&ctx->host_small), 1u << 20));
    for (auto& ev : ctx->ev) SG_CUDA(cudaEventCreate(&ev));
    SG_CUDA(cudaFuncSetAttribute(seg_sort_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SegSortSmem))));
    SG_CUDA(cudaFuncSetAttribute(seg_sort_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SegSortSmem))));
    SG_CUDA(cudaFuncSetAttribute(seg_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SegRankSmem))));
    SG_CUDA(cudaFuncSetAttribute(cluster_window_scatter_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(ClusterWindow<2>::kSlice * 4)));
    SG_CUDA(cudaFuncSetAttribute(cluster_segment_window_scatter_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(ClusterWindow<2>::kSlice * 4)));
    SG_CUDA(cudaFuncSetAttribute(cluster4_window_scatter_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(ClusterWindow<4>::kSlice * 4)));
    SG_CUDA(cudaFuncSetAttribute(seed_sorted_kernel<true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SeedSortSmem))));
    SG_CUDA(cudaFuncSetAttribute(seed_sorted_kernel<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(SeedSortSmem))));
    SG_CUDA(cudaFuncSetAttribute(slot_segment_window_scatter_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kSlotWindow * 4)));
    SG_CUDA(cudaFuncSetAttribute(slot_window_scatter_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kSlotWindow * 4)));
    for (bool ballot : {true, false}) {
      for (u32 tile : {2048u, 4096u}) {
        for (u32 block : {256u, 512u}) {
          for (bool vals : {true, false}) {
            for (bool tma : {false, true}) {
              const OnesweepVariant v = onesweep_variant(ballot, block, tile, vals, tma);
              SG_CUDA(cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(v.smem)));
            }
          }
        }
      }
    }
  } catch (const CudaError& err) {
    g_create_error = std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code);
    sufgpu_destroy(ctx);
    return SUFGPU_BUILD_FAILURE;
  }
  *out = ctx;
  return SUFGPU_OK;
}

void sufgpu_destroy(sufgpu_ctx* ctx) {
  if (!ctx) return;
  for (sufgpu_ctx* h : ctx->helpers) sufgpu_destroy(h);
  ctx->helpers.clear();
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  for (auto& ev : ctx->ev) {
    if (ev) cudaEventDestroy(ev);
  }
  if (ctx->copy_ready) cudaEventDestroy(ctx->copy_ready);
  if (ctx->copy_done) cudaEventDestroy(ctx->copy_done);
  ctx->drop_round_graphs();
  if (ctx->crc_scratch) cudaFree(ctx->crc_scratch);
  if (ctx->host_scalars) cudaFreeHost(ctx->host_scalars);
  if (ctx->host_small) cudaFreeHost(ctx->host_small);
  if (ctx->arena.base) {
    cudaFree(ctx->arena.base);
    ctx->arena.base = nullptr;
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  delete ctx;
}

const char* sufgpu_last_error(const sufgpu_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

uint64_t sufgpu_max_symbols(void) { return 0xffffffffull; }

sufgpu_status sufgpu_crc32_device(sufgpu_ctx* ctx, const void* data, uint64_t bytes,
                                  uint32_t crc_in, uint32_t* crc_out) {
  if (!ctx || !crc_out || (bytes && !data)) return SUFGPU_INVALID_INPUT;
  try {
    SG_CUDA(cudaSetDevice(ctx->device));
    const u64 words = 2 * (bytes / kCrcChunk + 1);
    if (ctx->crc_scratch_words < words) {
      if (ctx->crc_scratch) cudaFree(ctx->crc_scratch);
      ctx->crc_scratch = nullptr;
      ctx->crc_scratch_words = 0;
      SG_CUDA(cudaMalloc(&ctx->crc_scratch, words * 4));
      ctx->crc_scratch_words = words;
    }
    Engine e(*ctx);
    *crc_out = e.crc32_device(data, bytes, crc_in, ctx->crc_scratch);
    return SUFGPU_OK;
  } catch (const CudaError& err) {
    cudaGetLastError();
    return fail(ctx, SUFGPU_BUILD_FAILURE,
                std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code));
  }
}

sufgpu_status sufgpu_encode_fasta_device(sufgpu_ctx* ctx, const uint8_t* raw, uint64_t bytes,
                                         uint8_t* out, uint64_t cap, uint64_t* size,
                                         uint64_t* fingerprint, uint64_t* records) {
  if (!ctx || !size || (bytes > 0 && !raw)) return SUFGPU_INVALID_INPUT;
  *size = 0;
  // The first record starts at the first '>' or '@' (kseq skips to it).
  u64 first = 0;
  while (first < bytes && raw[first] != '>' && raw[first] != '@') ++first;
  if (first == bytes) return fail(ctx, SUFGPU_INVALID_INPUT, "reference must contain at least one FASTA record");
  if (raw[first] == '@') return fail(ctx, SUFGPU_UNSUPPORTED, "FASTQ input: use sufgpu_encode_fasta");
  try {
    SG_CUDA(cudaSetDevice(ctx->device));
    sufgpu_ctx& c = *ctx;
    const u64 tiles = (bytes + kFastaTile - 1) / kFastaTile;
    const u64 header_cap = std::min<u64>(bytes / 2 + 2, u64(1) << 24);
    const u64 chunk = bytes > (u64(64) << 20) ? 16384 : 4096;  // FNV chunk (16-byte multiple)
    const u64 max_chunks = (bytes + 1 + chunk - 1) / chunk;
    const u64 raw_bytes = round_up(bytes + 64, 256);
    const u64 out_bytes = round_up(bytes + 64, 256);
    const u64 status_bytes = round_up(2 * (tiles + 1) * 8, 256);
    const u64 header_bytes = round_up(header_cap * sizeof(FastaHeader), 256);
    const u64 fnv_bytes = round_up(max_chunks * 18, 256);
    const u64 small_bytes = 256 + round_up(sizeof(DeviceFlags), 64);
    c.arena.reserve(raw_bytes + out_bytes + status_bytes + header_bytes + fnv_bytes + small_bytes);
    u8* at = static_cast<u8*>(c.arena.base);
    u8* d_raw = at; at += raw_bytes;
    u8* d_out = at; at += out_bytes;
    u64* status = reinterpret_cast<u64*>(at); at += status_bytes;
    FastaHeader* headers = reinterpret_cast<FastaHeader*>(at); at += header_bytes;
    u64* mult = reinterpret_cast<u64*>(at);
    u64* add = mult + max_chunks;
    u8* fnv_start = reinterpret_cast<u8*>(add + max_chunks);
    u8* fnv_end = fnv_start + max_chunks;
    at += fnv_bytes;
    u64* scalars = reinterpret_cast<u64*>(at);  // [0] header count, [1] out total, [2] counter|unsupported
    DeviceFlags* flags = reinterpret_cast<DeviceFlags*>(at + 256);
    cudaStream_t st = c.stream;
    SG_CUDA(cudaMemcpyAsync(d_raw, raw, bytes, cudaMemcpyDefault, st));
    SG_CUDA(cudaMemsetAsync(d_raw + bytes, 0, raw_bytes - bytes, st));
    SG_CUDA(cudaMemsetAsync(status, 0, status_bytes, st));
    SG_CUDA(cudaMemsetAsync(scalars, 0, small_bytes, st));
    u32* counters = reinterpret_cast<u32*>(scalars + 2);  // [0] tile counter, [1] unsupported
    fasta_normalize_kernel<<<static_cast<unsigned>(tiles), kFastaBlock, 0, st>>>(
        d_raw, bytes, first, d_out, out_bytes - 1, status, status + tiles + 1, counters,
        headers, header_cap, scalars + 0, counters + 1, scalars + 1, flags);
    SG_CUDA(cudaGetLastError());
    ++c.launches;
    u64 host_scalars[3] = {0, 0, 0};
    DeviceFlags host_flags{};
    SG_CUDA(cudaMemcpyAsync(host_scalars, scalars, sizeof(host_scalars), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaMemcpyAsync(&host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    if (host_flags.error) return fail(ctx, SUFGPU_BUILD_FAILURE, "device check failed in FASTA normalisation");
    u32 unsupported = 0;
    std::memcpy(&unsupported, reinterpret_cast<const u8*>(host_scalars + 2) + 4, 4);
    if (unsupported & kFastaFastq) return fail(ctx, SUFGPU_UNSUPPORTED, "FASTQ records: use sufgpu_encode_fasta");
    if (unsupported) {
      return fail(ctx, SUFGPU_UNSUPPORTED,
                  "a lone carriage-return line after a header: use sufgpu_encode_fasta");
    }
    const u64 heads = host_scalars[0];
    u64 total = host_scalars[1];
    if (heads > header_cap) return fail(ctx, SUFGPU_INVALID_INPUT, "too many FASTA records");
    std::vector<FastaHeader> h(heads);
    if (heads) {
      SG_CUDA(cudaMemcpyAsync(h.data(), headers, heads * sizeof(FastaHeader), cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
      std::sort(h.begin(), h.end(), [](const FastaHeader& a, const FastaHeader& b) { return a.raw < b.raw; });
    }
    // Records: the first at `first`, one more per later header.  A bare '>' at
    // the very end of the input opens no record (its 1 closes the previous one).
    bool trailing_bare = heads > 0 && h.back().raw + 1 == bytes;
    const u64 count = heads + (trailing_bare ? 0 : 1);
    auto name_of = [&](u64 pos) {
      u64 e = pos + 1;
      while (e < bytes && !std::isspace(static_cast<unsigned char>(raw[e]))) ++e;
      return std::string(reinterpret_cast<const char*>(raw + pos + 1), e - pos - 1);
    };
    std::unordered_set<std::string> names;
    u64 start_out = 0;
    for (u64 k = 0; k < count; ++k) {
      const u64 pos = k == 0 ? first : h[k - 1].raw;
      const u64 sep = k < heads ? h[k].out : total;  // where record k's 1 goes
      const std::string name = name_of(pos);
      if (name.empty()) return fail(ctx, SUFGPU_INVALID_INPUT, "FASTA record name must not be empty");
      if (!names.insert(name).second) return fail(ctx, SUFGPU_INVALID_INPUT, "duplicate FASTA record name: " + name);
      if (sep <= start_out) return fail(ctx, SUFGPU_INVALID_INPUT, "FASTA record must not be empty: " + name);
      start_out = sep + 1;
    }
    if (!trailing_bare) {
      SG_CUDA(cudaMemsetAsync(d_out + total, 1, 1, st));
      ++total;
    }
    *size = total;
    if (records) *records = count;
    if (total > cap) return fail(ctx, SUFGPU_INVALID_INPUT, "output buffer too small");
    if (out) SG_CUDA(cudaMemcpyAsync(out, d_out, total, cudaMemcpyDefault, st));
    if (fingerprint) {
      // FNV-1a 64 of the logical bytes (fasta.cuh): low byte at every chunk
      // start from eight XOR-scanned passes, then one affine map per chunk.
      constexpr u64 kBasis = 14695981039346656037ull;
      const u64 chunks = (total + chunk - 1) / chunk;
      std::vector<u8> start(chunks, 0), end_bit(chunks);
      start[0] = static_cast<u8>(kBasis & 0xff);
      const unsigned grid = static_cast<unsigned>(std::min<u64>((chunks + 255) / 256, u64(c.sm_count) * 16));
      for (u32 j = 0; j < 8; ++j) {
        SG_CUDA(cudaMemcpyAsync(fnv_start, start.data(), chunks, cudaMemcpyHostToDevice, st));
        fnv_level_kernel<<<grid, 256, 0, st>>>(d_out, total, chunk, chunks, fnv_start, j, fnv_end);
        SG_CUDA(cudaGetLastError());
        SG_CUDA(cudaMemcpyAsync(end_bit.data(), fnv_end, chunks, cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        u8 carry = 0;  // bit j at the start of chunk k: XOR of the end bits before it
        for (u64 k = 0; k + 1 < chunks; ++k) {
          carry ^= end_bit[k];
          start[k + 1] |= static_cast<u8>(carry << j);
        }
      }
      std::vector<u64> m(chunks), a(chunks);
      SG_CUDA(cudaMemcpyAsync(fnv_start, start.data(), chunks, cudaMemcpyHostToDevice, st));
      fnv_affine_kernel<<<grid, 256, 0, st>>>(d_out, total, chunk, chunks, fnv_start, mult, add);
      SG_CUDA(cudaGetLastError());
      SG_CUDA(cudaMemcpyAsync(m.data(), mult, chunks * 8, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaMemcpyAsync(a.data(), add, chunks * 8, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
      u64 hash = kBasis;
      for (u64 k = 0; k < chunks; ++k) hash = hash * m[k] + a[k];
      *fingerprint = hash;
      c.launches += 9;
    }
    SG_CUDA(cudaStreamSynchronize(st));
    return SUFGPU_OK;
  } catch (const CudaError& err) {
    cudaGetLastError();
    return fail(ctx, SUFGPU_BUILD_FAILURE,
                std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code));
  } catch (const BuildError& err) {
    return fail(ctx, err.status, err.message);
  } catch (const std::exception& err) {
    return fail(ctx, SUFGPU_BUILD_FAILURE, err.what());
  }
}

uint32_t sufgpu_prefix_select_k(uint64_t suffix_count, uint64_t resident_core_bytes) {
  // FastPrefixIndexOptions defaults: k in [8, 10], 2500 basis points of the
  // resident core arrays, at least 2^16 suffixes; 32-bit rows below 2^32.
  if (suffix_count < (u64(1) << 16)) return 0;
  const u64 budget = (resident_core_bytes / 10000) * 2500 + ((resident_core_bytes % 10000) * 2500) / 10000;
  const u64 row_bytes = suffix_count <= 0xffffffffull ? 4 : 8;
  for (u32 k = 10; k >= 8; --k) {
    if ((u64(1) << (2 * k)) * 2 * row_bytes <= budget) return k;
  }
  return 0;
}

uint64_t sufgpu_device_bytes(uint64_t n, const sufgpu_build_desc*) {
  return plan_layout(nullptr, n, 1).total;
}

void* sufgpu_host_alloc(uint64_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void sufgpu_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

static sufgpu_status check_desc(sufgpu_ctx* ctx, const sufgpu_build_desc* d) {
  if (!d) return fail(ctx, SUFGPU_INVALID_INPUT, "build descriptor is null");
  if (!valid_width(d->sa_storage_bits)) return fail(ctx, SUFGPU_INVALID_INPUT, "invalid SA storage width");
  if (d->isa_storage_bits && !valid_width(d->isa_storage_bits))
    return fail(ctx, SUFGPU_INVALID_INPUT, "invalid ISA storage width");
  if (d->lcp_encoding > SUFGPU_LCP_BYTE64) return fail(ctx, SUFGPU_INVALID_INPUT, "invalid LCP encoding");
  if (d->prefix_k > 10) return fail(ctx, SUFGPU_INVALID_INPUT, "prefix directory k must be at most 10");
  if (d->prefix_k && d->sampling_rate > 1) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "the prefix directory needs a complete suffix array");
  }
  if ((d->flags & SUFGPU_FLAG_CHILD) &&
      (d->sampling_rate > 1 || d->lcp_encoding == SUFGPU_LCP_NONE)) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "CHILD needs a complete build with LCP");
  }
  return SUFGPU_OK;
}

static sufgpu_status finish(sufgpu_ctx* ctx, Engine& e, sufgpu_build_stats* stats,
                            std::chrono::steady_clock::time_point t0) {
  // The build's stream is non-blocking: wait for it before reading its error
  // flags and events (a legacy-stream copy would not), and so that every
  // output copy has landed when the call returns.
  SG_CUDA(cudaStreamSynchronize(ctx->stream));
  DeviceFlags flags{};
  SG_CUDA(cudaMemcpyAsync(&flags, e.L.flags, sizeof(flags), cudaMemcpyDeviceToHost, ctx->stream));
  SG_CUDA(cudaStreamSynchronize(ctx->stream));
  if (flags.error) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "device check failed (flags 0x%x, site %u)", flags.error,
                  flags.timeout_site);
    return fail(ctx, SUFGPU_BUILD_FAILURE, buf);
  }
  if (ctx->profiling) {
    for (const auto& p : ctx->pending) {
      float kms = 0;
      SG_CUDA(cudaEventElapsedTime(&kms, p.before, p.after));
      auto it = std::find_if(ctx->profile.begin(), ctx->profile.end(),
                             [&](const KernelTotals& k) { return k.name == p.name; });
      if (it == ctx->profile.end()) {
        ctx->profile.push_back(KernelTotals{p.name});
        it = ctx->profile.end() - 1;
      }
      it->launches += 1;
      it->seconds += kms / 1e3;
      it->bytes += p.bytes;
    }
    ctx->pending.clear();
    ctx->event_pool.reset();
  }
  if (stats) {
    float ms = 0;
    auto span = [&](int a, int b) {
      cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]);
      return ms / 1e3;
    };
    e.st.h2d_seconds = span(0, 1);
    e.st.sa_seconds = span(1, 2);
    e.st.isa_seconds = span(2, 3);
    e.st.storage_seconds = span(3, 4);
    e.st.lcp_seconds = span(4, 5);
    e.st.device_seconds = span(0, 5);
    e.st.total_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    e.st.symbols = e.n;
    *stats = e.st;
  }
  return SUFGPU_OK;
}

sufgpu_status sufgpu_build(sufgpu_ctx* ctx, const uint8_t* text, uint64_t n,
                           const sufgpu_build_desc* desc, const sufgpu_outputs* out,
                           sufgpu_anchors* anchors, sufgpu_build_stats* stats) {
  if (!ctx) return SUFGPU_INVALID_INPUT;
  if (auto s = check_desc(ctx, desc)) return s;
  if (n > sufgpu_max_symbols()) return fail(ctx, SUFGPU_INVALID_INPUT, "text exceeds 2^32-1 symbols");
  if (n > 0 && !text) return fail(ctx, SUFGPU_INVALID_INPUT, "text is null");
  if (!out) return fail(ctx, SUFGPU_INVALID_INPUT, "outputs are null");
  if ((desc->flags & SUFGPU_FLAG_CHILD) && n > 0 && !out->child) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "child is null");
  }
  if (desc->prefix_k) {
    if (!out->prefix_intervals) return fail(ctx, SUFGPU_INVALID_INPUT, "prefix_intervals is null");
    // The directory is staged in the 8n-byte key buffer.
    if ((u64(8) << (2 * desc->prefix_k)) > 8 * std::max<u64>(n, 1) + 256) {
      return fail(ctx, SUFGPU_INVALID_INPUT, "prefix directory larger than the text allows");
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  ctx->launches = 0;
  ctx->pending.clear();
  ctx->event_pool.reset();
  if (anchors) *anchors = sufgpu_anchors{nullptr, nullptr, 0, 0};
  if (n == 0) {
    if (stats) *stats = sufgpu_build_stats{};
    return SUFGPU_OK;
  }
  try {
    SG_CUDA(cudaSetDevice(ctx->device));
    TuningScope scope(*ctx, n);
    Engine e(*ctx);
    e.n = n;
    e.rank_rows = n;
    e.segs = 1;
    e.begin = {0, n};
    const Layout probe = plan_layout(nullptr, n, 1);
    ctx->arena.reserve(probe.total);
    e.L = plan_layout(static_cast<u8*>(ctx->arena.base), n, 1);
    SG_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    e.zero(e.L.flags, sizeof(DeviceFlags));
    SG_CUDA(cudaMemcpyAsync(e.L.text, text, n, cudaMemcpyDefault, ctx->stream));
    e.zero(e.L.text + n, kTextPad);
    e.want_crc = (desc->flags & SUFGPU_FLAG_PLANE_CRC) != 0;
    sufgpu_outputs o = *out;
    run_build(e, *desc, &o, anchors, 1);
    e.st.kernel_launches = ctx->launches;
    return finish(ctx, e, stats, t0);
  } catch (const CudaError& err) {
    cudaGetLastError();
    return fail(ctx, SUFGPU_BUILD_FAILURE,
                std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code));
  } catch (const BuildError& err) {
    return fail(ctx, err.status, err.message);
  } catch (const std::exception& err) {
    return fail(ctx, SUFGPU_BUILD_FAILURE, err.what());
  }
}

int sufgpu_divsufsort64(sufgpu_ctx* ctx, const uint8_t* T, int64_t* SA, int64_t n) {
  if (!ctx || !T || !SA || n < 0) return -1;
  if (n <= 1) {
    if (n == 1) SA[0] = 0;
    return 0;
  }
  sufgpu_build_desc d{64, 0, SUFGPU_LCP_NONE, 0};
  sufgpu_outputs o{SA, nullptr, nullptr, nullptr, nullptr};
  return sufgpu_build(ctx, T, static_cast<u64>(n), &d, &o, nullptr, nullptr) == SUFGPU_OK ? 0 : -2;
}

int sufgpu_divsufsort(sufgpu_ctx* ctx, const uint8_t* T, int32_t* SA, int32_t n) {
  if (!ctx || !T || !SA || n < 0) return -1;
  if (n <= 1) {
    if (n == 1) SA[0] = 0;
    return 0;
  }
  sufgpu_build_desc d{32, 0, SUFGPU_LCP_NONE, 0};
  sufgpu_outputs o{SA, nullptr, nullptr, nullptr, nullptr};
  return sufgpu_build(ctx, T, static_cast<u64>(n), &d, &o, nullptr, nullptr) == SUFGPU_OK ? 0 : -2;
}

}  // extern "C"

// sufgpu_build_batch; a collection worker passes the workers' shared gate and
// receives the host clock readings of its gate (unchanged without one).
struct GateTimes {
  std::chrono::steady_clock::time_point in{}, out{};
};
static sufgpu_status build_batch(sufgpu_ctx* ctx, sufgpu_instance* instances, uint32_t count,
                                 const sufgpu_build_desc* desc, sufgpu_build_stats* stats,
                                 std::mutex* gate, GateTimes* times = nullptr);

extern "C" sufgpu_status sufgpu_build_batch(sufgpu_ctx* ctx, sufgpu_instance* instances,
                                            uint32_t count, const sufgpu_build_desc* desc,
                                            sufgpu_build_stats* stats) {
  return build_batch(ctx, instances, count, desc, stats, nullptr);
}

static sufgpu_status build_batch(sufgpu_ctx* ctx, sufgpu_instance* instances, uint32_t count,
                                 const sufgpu_build_desc* desc, sufgpu_build_stats* stats,
                                 std::mutex* gate, GateTimes* times) {
  if (!ctx) return SUFGPU_INVALID_INPUT;
  if (auto s = check_desc(ctx, desc)) return s;
  if (count == 0) {
    if (stats) *stats = sufgpu_build_stats{};
    return SUFGPU_OK;
  }
  if (!instances) return fail(ctx, SUFGPU_INVALID_INPUT, "instances are null");
  if (count > kMaxSegmentsPerLaunch) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "too many instances in one batch launch");
  }
  if (desc->prefix_k) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "the prefix directory is built for single references");
  }
  if (desc->flags & SUFGPU_FLAG_PLANE_CRC) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "plane checksums are kept for single builds");
  }
  if (desc->flags & SUFGPU_FLAG_CHILD) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "the CHILD table is built for single references");
  }
  std::vector<u64> begin(count + 1, 0);
  for (u32 j = 0; j < count; ++j) {
    if (instances[j].n == 0) return fail(ctx, SUFGPU_INVALID_INPUT, "batch instance is empty");
    if (!instances[j].text) return fail(ctx, SUFGPU_INVALID_INPUT, "batch instance text is null");
    begin[j + 1] = begin[j] + instances[j].n;
    if (begin[j + 1] > sufgpu_max_symbols()) {
      return fail(ctx, SUFGPU_INVALID_INPUT, "batch exceeds 2^32-1 symbols");
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  ctx->launches = 0;
  ctx->pending.clear();
  ctx->event_pool.reset();
  try {
    SG_CUDA(cudaSetDevice(ctx->device));
    u64 longest = 0;
    for (u32 j = 0; j < count; ++j) longest = std::max<u64>(longest, instances[j].n);
    TuningScope scope(*ctx, longest);
    Engine e(*ctx);
    e.n = begin[count];
    e.rank_rows = e.n;
    e.segs = count;
    e.begin = begin;
    const Layout probe = plan_layout(nullptr, e.n, count);
    ctx->arena.reserve(probe.total);
    e.L = plan_layout(static_cast<u8*>(ctx->arena.base), e.n, count);
    SG_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    e.zero(e.L.flags, sizeof(DeviceFlags));
    for (u32 j = 0; j < count; ++j) {
      SG_CUDA(cudaMemcpyAsync(e.L.text + begin[j], instances[j].text, instances[j].n,
                              cudaMemcpyDefault, ctx->stream));
    }
    e.zero(e.L.text + e.n, kTextPad);
    std::vector<sufgpu_outputs> outs(count);
    std::vector<sufgpu_anchors> anchors(count);
    for (u32 j = 0; j < count; ++j) outs[j] = instances[j].out;
    e.gate = gate;
    e.gate_enter();  // the text copies above run while another worker computes
    run_build(e, *desc, outs.data(), anchors.data(), count);
    for (u32 j = 0; j < count; ++j) instances[j].anchors = anchors[j];
    e.st.kernel_launches = ctx->launches;
    const sufgpu_status st = finish(ctx, e, stats, t0);
    if (e.gate_held) {  // a build without the compute-first path leaves here
      e.gate_held = false;
      e.gate_out = std::chrono::steady_clock::now();
      gate->unlock();
    }
    if (times && gate) *times = GateTimes{e.gate_in, e.gate_out};
    return st;
  } catch (const CudaError& err) {
    cudaGetLastError();
    return fail(ctx, SUFGPU_BUILD_FAILURE,
                std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code));
  } catch (const BuildError& err) {
    return fail(ctx, err.status, err.message);
  } catch (const std::exception& err) {
    return fail(ctx, SUFGPU_BUILD_FAILURE, err.what());
  }
}

extern "C" sufgpu_status sufgpu_build_collection(sufgpu_ctx* ctx, sufgpu_instance* instances,
                                                 uint64_t count, const sufgpu_build_desc* desc,
                                                 uint64_t batch_symbols, uint32_t workers,
                                                 sufgpu_build_stats* stats) {
  if (!ctx) return SUFGPU_INVALID_INPUT;
  if (auto s = check_desc(ctx, desc)) return s;
  if (count > 0 && !instances) return fail(ctx, SUFGPU_INVALID_INPUT, "instances are null");
  if (desc->prefix_k || (desc->flags & SUFGPU_FLAG_PLANE_CRC)) {
    return fail(ctx, SUFGPU_INVALID_INPUT, "prefix directories and plane checksums are kept for single builds");
  }
  if (workers == 0 || workers > 8) return fail(ctx, SUFGPU_INVALID_INPUT, "workers must be 1..8");
  if (batch_symbols == 0) batch_symbols = u64(1) << 30;
  // Sub-batches in order: at most batch_symbols symbols (a larger instance
  // alone) and kMaxSegmentsPerLaunch instances each.
  std::vector<std::pair<u64, u32>> parts;  // (first instance, count)
  for (u64 j = 0; j < count;) {
    u64 syms = 0;
    u32 m = 0;
    while (j + m < count && m < kMaxSegmentsPerLaunch &&
           (m == 0 || syms + instances[j + m].n <= batch_symbols)) {
      syms += instances[j + m].n;
      ++m;
    }
    parts.emplace_back(j, m);
    j += m;
  }
  if (ctx->profiling) workers = 1;  // the per-kernel profile is kept per context
  workers = static_cast<u32>(std::min<u64>(workers, std::max<size_t>(parts.size(), 1)));
  const auto t0 = std::chrono::steady_clock::now();
  while (ctx->helpers.size() + 1 < workers) {
    sufgpu_ctx* h = nullptr;
    if (sufgpu_status st = sufgpu_create(&h, ctx->device)) {
      return fail(ctx, st, "cannot create a helper context: " + g_create_error);
    }
    ctx->helpers.push_back(h);
  }
  std::vector<sufgpu_ctx*> pool{ctx};
  for (u32 w = 1; w < workers; ++w) {
    sufgpu_ctx* h = ctx->helpers[w - 1];
    h->tune = ctx->tune;
    h->tuning_classes = ctx->tuning_classes;
    pool.push_back(h);
  }
  const bool byte_coded =
      desc->lcp_encoding == SUFGPU_LCP_BYTE32 || desc->lcp_encoding == SUFGPU_LCP_BYTE64;
  ctx->collection_anchors.assign(byte_coded ? 2 * parts.size() : 0, {});
  std::vector<sufgpu_build_stats> part_stats(parts.size());
  std::atomic<size_t> next{0};
  std::atomic<bool> failed{false};
  std::mutex error_mu, gate;
  sufgpu_status first_status = SUFGPU_OK;
  std::string first_error;
  auto record_failure = [&](sufgpu_status st, const std::string& message) {
    std::lock_guard<std::mutex> lock(error_mu);
    if (first_status == SUFGPU_OK) {
      first_status = st;
      first_error = message;
    }
    failed = true;
  };
  ctx->collection_trace.assign(parts.size(), sufgpu_ctx::PartTrace{});
  auto since = [&](std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double>(t - t0).count();
  };
  auto build_parts = [&](sufgpu_ctx* w, u32 worker) {
    while (!failed.load()) {
      const size_t i = next.fetch_add(1);
      if (i >= parts.size()) return;
      sufgpu_instance* inst = instances + parts[i].first;
      const auto started = std::chrono::steady_clock::now();
      GateTimes gt{started, started};
      const sufgpu_status st = build_batch(w, inst, parts[i].second, desc, &part_stats[i],
                                           workers > 1 ? &gate : nullptr, &gt);
      const auto ended = std::chrono::steady_clock::now();
      if (workers == 1) gt.out = ended;
      ctx->collection_trace[i] =
          sufgpu_ctx::PartTrace{worker, since(started), since(gt.in), since(gt.out), since(ended)};
      if (st != SUFGPU_OK) {
        record_failure(st, w->last_error);
        return;
      }
      if (byte_coded) {  // keep this sub-batch's anchors past the worker's next build
        const u64 w_bytes = desc->lcp_encoding == SUFGPU_LCP_BYTE64 ? 8 : 4;
        u64 total = 0;
        for (u32 j = 0; j < parts[i].second; ++j) total += inst[j].anchors.count;
        std::vector<u8>& pos = ctx->collection_anchors[2 * i];
        std::vector<u8>& val = ctx->collection_anchors[2 * i + 1];
        pos.resize(std::max<u64>(total * w_bytes, 8));
        val.resize(std::max<u64>(total * w_bytes, 8));
        u64 at = 0;
        for (u32 j = 0; j < parts[i].second; ++j) {
          sufgpu_anchors& a = inst[j].anchors;
          const u64 bytes = a.count * w_bytes;
          if (bytes) {
            std::memcpy(pos.data() + at, a.positions, bytes);
            std::memcpy(val.data() + at, a.values, bytes);
          }
          a.positions = pos.data() + at;
          a.values = val.data() + at;
          at += bytes;
        }
      }
    }
  };
  auto work = [&](sufgpu_ctx* w, u32 worker) {
    try {
      build_parts(w, worker);
    } catch (const std::exception& err) {  // host allocation in the anchor copies
      record_failure(SUFGPU_BUILD_FAILURE, err.what());
    }
  };
  std::vector<std::thread> threads;
  try {
    for (u32 w = 1; w < workers; ++w) threads.emplace_back(work, pool[w], w);
  } catch (const std::system_error&) {
    // No more host threads: the workers started so far take every sub-batch.
  }
  work(pool[0], 0u);
  for (auto& t : threads) t.join();
  if (first_status != SUFGPU_OK) return fail(ctx, first_status, first_error);
  if (stats) {
    sufgpu_build_stats sum{};
    for (const auto& p : part_stats) {
      sum.h2d_seconds += p.h2d_seconds;
      sum.sa_seconds += p.sa_seconds;
      sum.isa_seconds += p.isa_seconds;
      sum.lcp_seconds += p.lcp_seconds;
      sum.storage_seconds += p.storage_seconds;
      sum.d2h_seconds += p.d2h_seconds;
      sum.device_seconds += p.device_seconds;
      sum.symbols += p.symbols;
      sum.rounds = std::max(sum.rounds, p.rounds);
      sum.seed_symbols = std::max(sum.seed_symbols, p.seed_symbols);
      sum.active_rows += p.active_rows;
      sum.active_first += p.active_first;
      sum.irreducible_long += p.irreducible_long;
      sum.anchors += p.anchors;
      sum.kernel_launches += p.kernel_launches;
      sum.long_runs += p.long_runs;
      sum.seg_sort_fallbacks += p.seg_sort_fallbacks;
      sum.seed_code_bits = std::max(sum.seed_code_bits, p.seed_code_bits);
    }
    sum.total_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *stats = sum;
  }
  return SUFGPU_OK;
}

extern "C" uint64_t sufgpu_collection_parts(const sufgpu_ctx* ctx) {
  return ctx ? ctx->collection_trace.size() : 0;
}

extern "C" sufgpu_status sufgpu_collection_trace(const sufgpu_ctx* ctx, uint64_t index,
                                                 uint32_t* worker, double* times) {
  if (!ctx || index >= ctx->collection_trace.size() || !times) return SUFGPU_INVALID_INPUT;
  const auto& t = ctx->collection_trace[index];
  if (worker) *worker = t.worker;
  times[0] = t.start;
  times[1] = t.gate_in;
  times[2] = t.gate_out;
  times[3] = t.end;
  return SUFGPU_OK;
}

extern "C" void sufgpu_set_profiling(sufgpu_ctx* ctx, int enable) {
  if (!ctx) return;
  ctx->profiling = enable != 0;
  ctx->profile.clear();
  ctx->pending.clear();
  ctx->event_pool.reset();
}

extern "C" uint32_t sufgpu_profile_count(const sufgpu_ctx* ctx) {
  return ctx ? static_cast<uint32_t>(ctx->profile.size()) : 0;
}

extern "C" sufgpu_status sufgpu_profile_entry(const sufgpu_ctx* ctx, uint32_t index,
                                              const char** name, uint64_t* launches,
                                              double* seconds, uint64_t* bytes) {
  if (!ctx || index >= ctx->profile.size()) return SUFGPU_INVALID_INPUT;
  const auto& k = ctx->profile[index];
  if (name) *name = k.name.c_str();
  if (launches) *launches = k.launches;
  if (seconds) *seconds = k.seconds;
  if (bytes) *bytes = k.bytes;
  return SUFGPU_OK;
}

extern "C" sufgpu_status sufgpu_set_tuning(sufgpu_ctx* ctx, const char* key, int64_t value) {
  if (!ctx || !key) return SUFGPU_INVALID_INPUT;
  const std::string err = apply_tuning(ctx->tune, key, value);
  if (!err.empty()) return fail(ctx, SUFGPU_INVALID_INPUT, err);
  return SUFGPU_OK;
}

extern "C" sufgpu_status sufgpu_set_tuning_class(sufgpu_ctx* ctx, uint64_t max_symbols,
                                                 const char* key, int64_t value) {
  if (!ctx || !key) return SUFGPU_INVALID_INPUT;
  Tuning probe = ctx->tune;
  const std::string err = apply_tuning(probe, key, value);
  if (!err.empty()) return fail(ctx, SUFGPU_INVALID_INPUT, err);
  auto& classes = ctx->tuning_classes;
  auto it = std::find_if(classes.begin(), classes.end(),
                         [&](const TuningClass& c) { return c.max_symbols == max_symbols; });
  if (it == classes.end()) {
    classes.push_back(TuningClass{max_symbols, {}});
    std::sort(classes.begin(), classes.end(),
              [](const TuningClass& a, const TuningClass& b) { return a.max_symbols < b.max_symbols; });
    it = std::find_if(classes.begin(), classes.end(),
                      [&](const TuningClass& c) { return c.max_symbols == max_symbols; });
  }
  it->settings.emplace_back(key, value);
  return SUFGPU_OK;
}

extern "C" void sufgpu_clear_tuning_classes(sufgpu_ctx* ctx) {
  if (ctx) ctx->tuning_classes.clear();
}

// ===========================================================================
// Served build engine: continuous batching at doubling-round granularity.
//
// One persistent arena (text, SA, ranks, LCP indexed by arena position) holds
// every in-flight reference.  Each iteration of the worker
//   1. admits queued requests into one free arena range (HBM admission: a
//      request waits while no range can hold it) and seeds them as a group;
//      their ranks are relocated to arena rows and their unsorted rows are
//      appended to the shared active list;
//   2. runs one doubling round over the shared active list, every reference
//      with its own prefix length h (references admitted at different times
//      advance side by side in the same launches);
//   3. finalizes references with no unsorted rows left (LCP, packing, copies
//      into the caller's planes) and frees their arena range.
// ===========================================================================
namespace {

struct ServedRequest {
  u64 ticket = 0;
  const u8* text = nullptr;
  u64 n = 0;
  sufgpu_build_desc desc{};
  sufgpu_outputs out{};
  u64 begin = 0;  // arena position while in flight
  u64 h = 0;
  u32 seed_length = 0;
  u32 rounds = 0;
  bool done = false;
  sufgpu_status status = SUFGPU_OK;
  std::string error;
  std::vector<u8> anchor_pos, anchor_val;
  u64 anchor_count = 0;
  u32 anchor_bits = 0;
  // Worker iterations (doubling rounds of the shared batch) completed when
  // the request was admitted and when it finished, and how many requests
  // were already in flight (mid-rounds) at its admission.
  u64 admit_iteration = 0, finish_iteration = 0;
  u32 inflight_at_admit = 0;
  std::chrono::steady_clock::time_point submitted, admitted, finished;
};

using ReqPtr = std::shared_ptr<ServedRequest>;

}  // namespace

struct sufgpu_server {
  sufgpu_ctx* ctx = nullptr;
  u64 capacity = 0;
  u32 max_instances = 0;
  Layout L{};
  u32* g0 = nullptr;  // shared active list (ping-pong pair)
  u32* g1 = nullptr;
  u32* w = nullptr;   // rebased ranks of a finishing reference
  u32* rebased_sa = nullptr;
  u8* text_copy = nullptr;  // compacted text of finishing references
  u32* lcp_copy = nullptr;  // their LCP rows
  u64* inst_begin = nullptr;
  u64* inst_end = nullptr;
  u64* inst_h = nullptr;
  u8* alive = nullptr;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  std::deque<ReqPtr> queue;
  std::unordered_map<u64, ReqPtr> requests;
  std::vector<ReqPtr> inflight;  // sorted by arena position
  std::map<u64, u64> free_ranges;  // begin -> length
  u64 next_ticket = 1;
  bool stopping = false;
  std::thread worker;
  std::vector<double> latencies;
  u64 completed = 0, symbols_done = 0, iterations = 0, max_inflight = 0;
  std::chrono::steady_clock::time_point first_submit, last_done;
  bool any_submitted = false;
  std::string fatal;
};

namespace {

constexpr u64 kArenaAlign = 64;

u64 align_up(u64 v, u64 a) { return (v + a - 1) / a * a; }

void release_range(sufgpu_server* S, u64 begin, u64 length) {
  auto it = S->free_ranges.emplace(begin, length).first;
  auto next = std::next(it);
  if (next != S->free_ranges.end() && it->first + it->second == next->first) {
    it->second += next->second;
    S->free_ranges.erase(next);
  }
  if (it != S->free_ranges.begin()) {
    auto prev = std::prev(it);
    if (prev->first + prev->second == it->first) {
      prev->second += it->second;
      S->free_ranges.erase(it);
    }
  }
}

// An Engine whose layout is the server arena, optionally viewed from an
// offset (text/rank/sa/lcp shifted; scratch shared).
Engine arena_engine(sufgpu_server* S, u64 offset, u64 n) {
  Engine e(*S->ctx);
  e.L = S->L;
  e.L.text += offset;
  e.L.rank += offset;
  e.L.sa += offset;
  e.L.lcp += offset;
  e.n = n;
  e.rank_rows = n;
  e.sa = e.L.sa;
  e.spare = e.L.v0;
  return e;
}

void seed_group(sufgpu_server* S, std::vector<ReqPtr>& group, u32*& act, u64& active) {
  sufgpu_ctx& c = *S->ctx;
  const u64 R = group.front()->begin;
  std::vector<u64> begin{0};
  for (auto& r : group) begin.push_back(begin.back() + r->n);
  const u64 m = begin.back();
  for (auto& r : group) {
    SG_CUDA(cudaMemcpyAsync(S->L.text + r->begin, r->text, r->n, cudaMemcpyDefault, c.stream));
  }
  Engine e = arena_engine(S, R, m);
  e.segs = static_cast<u32>(group.size());
  e.begin = begin;
  const u64 fresh = e.seed_phase(S->L.sa + R);
  // Arena coordinates: SA values and ranks shift by R; the group's active
  // rows (in L.x) join the shared list after the current ones.
  e.launch("serve_relocate", m * 16, relocate_kernel, e.grid_stride_blocks(m, 256), 256, 0,
           S->L.sa + R, S->L.rank + R, m, static_cast<u32>(R));
  if (fresh) {
    e.launch("serve_append", fresh * 8, shift_kernel, e.grid_stride_blocks(fresh, 256), 256, 0,
             static_cast<const u32*>(S->L.x), fresh, static_cast<long long>(R), act + active);
    active += fresh;
  }
  for (auto& r : group) {
    r->h = e.seed_length;
    r->seed_length = e.seed_length;
  }
}

// Output phase for every reference that finished in this iteration: those
// with the same descriptor are compacted into one contiguous batch and go
// through the batched output path together.
void finalize_batch(sufgpu_server* S, std::vector<ReqPtr>& done_now, u32* free_list) {
  sufgpu_ctx& c = *S->ctx;
  std::vector<bool> taken(done_now.size(), false);
  for (size_t i = 0; i < done_now.size(); ++i) {
    if (taken[i]) continue;
    const sufgpu_build_desc d = done_now[i]->desc;
    std::vector<ReqPtr> group;
    for (size_t k = i; k < done_now.size(); ++k) {
      const sufgpu_build_desc& o = done_now[k]->desc;
      if (!taken[k] && o.sa_storage_bits == d.sa_storage_bits &&
          o.isa_storage_bits == d.isa_storage_bits && o.lcp_encoding == d.lcp_encoding &&
          o.flags == d.flags) {
        taken[k] = true;
        group.push_back(done_now[k]);
      }
    }
    const u32 count = static_cast<u32>(group.size());
    std::vector<u64> dst{0}, src;
    u32 seed_min = ~0u;
    for (auto& r : group) {
      src.push_back(r->begin);
      dst.push_back(dst.back() + r->n);
      seed_min = std::min(seed_min, r->seed_length);
    }
    const u64 m = dst.back();
    Engine f(c);
    f.L = S->L;
    f.n = m;
    f.rank_rows = m;
    f.segs = count;
    f.begin = dst;
    f.seed_length = seed_min;  // every reference shares at least this prefix
    f.upload_segments(dst);    // batch offsets -> L.seg_begin
    SG_CUDA(cudaMemcpyAsync(S->inst_begin, src.data(), count * 8, cudaMemcpyHostToDevice, c.stream));
    f.launch("serve_gather", m * 29, gather_finished_kernel, f.grid_stride_blocks(m, 256), 256, 0,
             static_cast<const u8*>(S->L.text), static_cast<const u32*>(S->L.sa),
             static_cast<const u32*>(S->L.rank), static_cast<const u32*>(S->L.lcp),
             static_cast<const u64*>(S->L.seg_begin), static_cast<const u64*>(S->inst_begin),
             count, m, S->text_copy, S->rebased_sa, S->w, S->lcp_copy);
    f.zero(S->text_copy + m, kTextPad);
    f.L.text = S->text_copy;
    f.L.rank = S->w;
    f.L.lcp = S->lcp_copy;
    f.sa = S->rebased_sa;
    f.spare = free_list;
    std::vector<sufgpu_outputs> outs(count);
    std::vector<sufgpu_anchors> anchors(count);
    for (u32 j = 0; j < count; ++j) outs[j] = group[j]->out;
    emit_outputs(f, d, outs.data(), anchors.data(), count);
    for (u32 j = 0; j < count; ++j) {
      auto& r = group[j];
      const auto& a = anchors[j];
      const u64 w = a.coordinate_bits / 8;
      if (a.count) {
        r->anchor_pos.assign(static_cast<const u8*>(a.positions),
                             static_cast<const u8*>(a.positions) + a.count * w);
        r->anchor_val.assign(static_cast<const u8*>(a.values),
                             static_cast<const u8*>(a.values) + a.count * w);
      }
      r->anchor_count = a.count;
      r->anchor_bits = a.coordinate_bits ? a.coordinate_bits
                                         : (d.lcp_encoding == SUFGPU_LCP_BYTE64 ? 64 : 32);
    }
  }
}

void fail_request(sufgpu_server* S, const ReqPtr& r, sufgpu_status status, const std::string& why) {
  r->status = status;
  r->error = why;
  r->done = true;
  r->finished = std::chrono::steady_clock::now();
  S->cv_done.notify_all();
}

void server_loop(sufgpu_server* S) {
  cudaSetDevice(S->ctx->device);
  u32* act = S->g0;
  u32* other = S->g1;
  u64 active = 0;
  while (true) {
    std::vector<ReqPtr> group;
    {
      std::unique_lock<std::mutex> lock(S->m);
      S->cv_work.wait(lock, [&] {
        return S->stopping || !S->queue.empty() || !S->inflight.empty();
      });
      if (S->queue.empty() && S->inflight.empty()) {
        if (S->stopping) break;
        continue;
      }
      // Admission: as many queued requests (in order) as one free range and
      // the instance slots can hold.
      u64 best_begin = 0, best_len = 0;
      for (auto& fr : S->free_ranges) {
        const u64 start = align_up(fr.first, kArenaAlign);
        const u64 len = fr.first + fr.second > start ? fr.first + fr.second - start : 0;
        if (len > best_len) {
          best_len = len;
          best_begin = start;
        }
      }
      u64 total = 0;
      while (!S->queue.empty() && S->inflight.size() + group.size() < S->max_instances) {
        ReqPtr r = S->queue.front();
        if (r->n + kArenaAlign > S->capacity) {
          S->queue.pop_front();
          fail_request(S, r, SUFGPU_INVALID_INPUT, "reference exceeds the server arena");
          continue;
        }
        if (total + r->n > best_len) break;
        r->begin = best_begin + total;
        r->admitted = std::chrono::steady_clock::now();
        r->admit_iteration = S->iterations;
        r->inflight_at_admit = static_cast<u32>(S->inflight.size());
        total += r->n;
        group.push_back(r);
        S->queue.pop_front();
      }
      if (total) {
        // Carve [best_begin, best_begin + total) out of its free range.
        auto it = std::prev(S->free_ranges.upper_bound(best_begin));
        const u64 fb = it->first, fl = it->second;
        S->free_ranges.erase(it);
        if (best_begin > fb) S->free_ranges.emplace(fb, best_begin - fb);
        const u64 tail = best_begin + total;
        if (fb + fl > tail) S->free_ranges.emplace(tail, fb + fl - tail);
      }
    }
    std::vector<ReqPtr> finished;
    try {
      SG_CUDA(cudaMemsetAsync(S->L.flags, 0, sizeof(DeviceFlags), S->ctx->stream));
      if (!group.empty()) {
        seed_group(S, group, act, active);
        std::lock_guard<std::mutex> lock(S->m);
        for (auto& r : group) S->inflight.push_back(r);
        std::sort(S->inflight.begin(), S->inflight.end(),
                  [](const ReqPtr& a, const ReqPtr& b) { return a->begin < b->begin; });
        S->max_inflight = std::max<u64>(S->max_inflight, S->inflight.size());
      }
      std::vector<ReqPtr> live;
      {
        std::lock_guard<std::mutex> lock(S->m);
        live = S->inflight;
      }
      const u32 K = static_cast<u32>(live.size());
      Engine e = arena_engine(S, 0, S->capacity);
      std::vector<u64> hb(K), he(K), hh(K);
      for (u32 j = 0; j < K; ++j) {
        hb[j] = live[j]->begin;
        he[j] = live[j]->begin + live[j]->n;
        hh[j] = live[j]->h;
      }
      std::vector<u8> alive(K, 0);
      if (K > 0) {
        SG_CUDA(cudaMemcpyAsync(S->inst_begin, hb.data(), K * 8, cudaMemcpyHostToDevice, S->ctx->stream));
        SG_CUDA(cudaMemcpyAsync(S->inst_end, he.data(), K * 8, cudaMemcpyHostToDevice, S->ctx->stream));
        SG_CUDA(cudaMemcpyAsync(S->inst_h, hh.data(), K * 8, cudaMemcpyHostToDevice, S->ctx->stream));
        const Segments segs{S->inst_begin, K, S->inst_end};
        if (active > 0) {
          active = e.round_step(act, other, active, 0, S->inst_h, segs);
          ++S->iterations;
          for (auto& r : live) {
            r->h *= 2;
            ++r->rounds;
          }
        }
        e.zero(S->alive, K);
        if (active > 0) {
          e.launch("serve_alive", active * 4, alive_kernel, e.grid_stride_blocks(active, 256), 256, 0,
                   static_cast<const u32*>(act), active, segs, S->alive);
        }
        SG_CUDA(cudaMemcpyAsync(alive.data(), S->alive, K, cudaMemcpyDeviceToHost, S->ctx->stream));
        e.sync();
        for (u32 j = 0; j < K; ++j) {
          if (!alive[j]) finished.push_back(live[j]);
        }
      }
      if (!finished.empty()) finalize_batch(S, finished, other);
      DeviceFlags flags{};  // read on the engine's (non-blocking) stream
      SG_CUDA(cudaMemcpyAsync(&flags, S->L.flags, sizeof(flags), cudaMemcpyDeviceToHost,
                              S->ctx->stream));
      SG_CUDA(cudaStreamSynchronize(S->ctx->stream));
      if (flags.error) throw BuildError{SUFGPU_BUILD_FAILURE, "device check failed in the served engine"};
    } catch (const CudaError& err) {
      cudaGetLastError();
      S->fatal = std::string("CUDA error in ") + err.what + ": " + cudaGetErrorString(err.code);
    } catch (const BuildError& err) {
      S->fatal = err.message;
    } catch (const std::exception& err) {
      S->fatal = err.what();
    }
    std::lock_guard<std::mutex> lock(S->m);
    const auto now = std::chrono::steady_clock::now();
    if (!S->fatal.empty()) {
      // Every in-flight reference fails with the error; the arena resets.
      for (auto& r : S->inflight) fail_request(S, r, SUFGPU_BUILD_FAILURE, S->fatal);
      for (auto& r : group) {
        if (!r->done) fail_request(S, r, SUFGPU_BUILD_FAILURE, S->fatal);
      }
      S->inflight.clear();
      S->free_ranges.clear();
      S->free_ranges.emplace(0, S->capacity);
      active = 0;
      S->fatal.clear();
      continue;
    }
    for (auto& r : finished) {
      r->done = true;
      r->finished = now;
      r->finish_iteration = S->iterations;
      S->latencies.push_back(std::chrono::duration<double>(now - r->submitted).count());
      ++S->completed;
      S->symbols_done += r->n;
      S->last_done = now;
      release_range(S, r->begin, r->n);
      S->inflight.erase(std::find(S->inflight.begin(), S->inflight.end(), r));
    }
    if (!finished.empty()) S->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

sufgpu_status sufgpu_server_create(sufgpu_server** out, int device,
                                   const sufgpu_server_config* config) {
  if (!out) return SUFGPU_INVALID_INPUT;
  *out = nullptr;
  auto* S = new sufgpu_server();
  S->capacity = config && config->capacity_symbols ? config->capacity_symbols : (u64(1) << 29);
  S->max_instances = config && config->max_instances ? config->max_instances : 1024;
  if (S->capacity > sufgpu_max_symbols() || S->max_instances > kMaxSegmentsPerLaunch) {
    delete S;
    return SUFGPU_INVALID_INPUT;
  }
  sufgpu_status st = sufgpu_create(&S->ctx, device);
  if (st != SUFGPU_OK) {
    delete S;
    return st;
  }
  try {
    const u64 C = S->capacity;
    const Layout probe = plan_layout(nullptr, C, S->max_instances);
    const u64 extra = 5 * round_up(C * 4, 256) + round_up(C + kTextPad, 256) +
                      3 * round_up(u64(S->max_instances) * 8, 256) + round_up(S->max_instances, 256);
    S->ctx->arena.reserve(probe.total + extra);
    u8* base = static_cast<u8*>(S->ctx->arena.base);
    S->L = plan_layout(base, C, S->max_instances);
    u8* p = base + probe.total;
    auto take = [&](u64 bytes) {
      u8* q = p;
      p += round_up(bytes, 256);
      return q;
    };
    S->g0 = reinterpret_cast<u32*>(take(C * 4));
    S->g1 = reinterpret_cast<u32*>(take(C * 4));
    S->w = reinterpret_cast<u32*>(take(C * 4));
    S->rebased_sa = reinterpret_cast<u32*>(take(C * 4));
    S->lcp_copy = reinterpret_cast<u32*>(take(C * 4));
    S->text_copy = take(C + kTextPad);
    S->inst_begin = reinterpret_cast<u64*>(take(u64(S->max_instances) * 8));
    S->inst_end = reinterpret_cast<u64*>(take(u64(S->max_instances) * 8));
    S->inst_h = reinterpret_cast<u64*>(take(u64(S->max_instances) * 8));
    S->alive = take(S->max_instances);
    SG_CUDA(cudaMemsetAsync(S->L.text + C, 0, kTextPad, S->ctx->stream));
    SG_CUDA(cudaStreamSynchronize(S->ctx->stream));
  } catch (const BuildError& err) {
    S->ctx->last_error = err.message;
    sufgpu_destroy(S->ctx);
    delete S;
    return SUFGPU_BUILD_FAILURE;
  } catch (const CudaError&) {
    cudaGetLastError();
    sufgpu_destroy(S->ctx);
    delete S;
    return SUFGPU_BUILD_FAILURE;
  }
  S->free_ranges.emplace(0, S->capacity);
  S->worker = std::thread(server_loop, S);
  *out = S;
  return SUFGPU_OK;
}

void sufgpu_server_destroy(sufgpu_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lock(S->m);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  sufgpu_destroy(S->ctx);
  delete S;
}

sufgpu_status sufgpu_server_submit(sufgpu_server* S, const uint8_t* text, uint64_t n,
                                   const sufgpu_build_desc* desc, const sufgpu_outputs* out,
                                   uint64_t* ticket) {
  if (!S || !desc || !out || !ticket || (n && !text)) return SUFGPU_INVALID_INPUT;
  if (auto s = check_desc(S->ctx, desc)) return s;
  // Served builds return complete arrays without the prefix directory.
  if (desc->sampling_rate > 1 || desc->prefix_k || (desc->flags & SUFGPU_FLAG_CHILD)) {
    return SUFGPU_INVALID_INPUT;
  }
  if (n == 0 || n > sufgpu_max_symbols()) return SUFGPU_INVALID_INPUT;
  auto r = std::make_shared<ServedRequest>();
  r->text = text;
  r->n = n;
  r->desc = *desc;
  r->out = *out;
  r->submitted = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lock(S->m);
    r->ticket = S->next_ticket++;
    S->requests.emplace(r->ticket, r);
    S->queue.push_back(r);
    if (!S->any_submitted) {
      S->any_submitted = true;
      S->first_submit = r->submitted;
    }
  }
  S->cv_work.notify_all();
  *ticket = r->ticket;
  return SUFGPU_OK;
}

static sufgpu_status request_info(const ReqPtr& r, sufgpu_request_info* info) {
  if (info) {
    info->queue_seconds = std::chrono::duration<double>(r->admitted - r->submitted).count();
    info->latency_seconds = std::chrono::duration<double>(r->finished - r->submitted).count();
    info->rounds = r->rounds;
    info->seed_symbols = r->seed_length;
    info->anchors = sufgpu_anchors{r->anchor_pos.empty() ? nullptr : r->anchor_pos.data(),
                                   r->anchor_val.empty() ? nullptr : r->anchor_val.data(),
                                   r->anchor_count, r->anchor_bits};
    info->admit_iteration = r->admit_iteration;
    info->finish_iteration = r->finish_iteration;
    info->inflight_at_admit = r->inflight_at_admit;
    info->reserved = 0;
  }
  return r->status;
}

sufgpu_status sufgpu_server_wait(sufgpu_server* S, uint64_t ticket, sufgpu_request_info* info) {
  if (!S) return SUFGPU_INVALID_INPUT;
  std::unique_lock<std::mutex> lock(S->m);
  auto it = S->requests.find(ticket);
  if (it == S->requests.end()) return SUFGPU_INVALID_INPUT;
  ReqPtr r = it->second;
  S->cv_done.wait(lock, [&] { return r->done; });
  return request_info(r, info);
}

sufgpu_status sufgpu_server_poll(sufgpu_server* S, uint64_t ticket, int* done) {
  if (!S || !done) return SUFGPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(S->m);
  auto it = S->requests.find(ticket);
  if (it == S->requests.end()) return SUFGPU_INVALID_INPUT;
  *done = it->second->done ? 1 : 0;
  return SUFGPU_OK;
}

sufgpu_status sufgpu_server_release(sufgpu_server* S, uint64_t ticket) {
  if (!S) return SUFGPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(S->m);
  auto it = S->requests.find(ticket);
  if (it == S->requests.end() || !it->second->done) return SUFGPU_INVALID_INPUT;
  S->requests.erase(it);
  return SUFGPU_OK;
}

sufgpu_status sufgpu_server_get_stats(sufgpu_server* S, sufgpu_server_stats* out) {
  if (!S || !out) return SUFGPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lock(S->m);
  std::vector<double> lat = S->latencies;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double q) {
    if (lat.empty()) return 0.0;
    const size_t i = std::min(lat.size() - 1, static_cast<size_t>(q * (lat.size() - 1) + 0.5));
    return lat[i];
  };
  *out = sufgpu_server_stats{};
  out->completed = S->completed;
  out->symbols = S->symbols_done;
  out->iterations = S->iterations;
  out->max_inflight = S->max_inflight;
  out->p50_seconds = pct(0.50);
  out->p99_seconds = pct(0.99);
  const double span = S->completed
                          ? std::chrono::duration<double>(S->last_done - S->first_submit).count()
                          : 0.0;
  out->span_seconds = span;
  out->symbols_per_second = span > 0 ? S->symbols_done / span : 0.0;
  out->queued = S->queue.size();
  out->inflight = S->inflight.size();
  return SUFGPU_OK;
}

}  // extern "C"
