/* sufgpu: B200 construction engine for sufkit's SA + ISA + LCP build path.
 *
 * Plain C ABI: opaque context, plain pointers and sizes, status codes, no C++
 * exceptions and no torch types across the boundary.  A context owns one CUDA
 * device, one stream and the device buffers it grows as builds need them; it
 * is thread-compatible (one thread at a time per context).
 *
 * Every build sorts all suffixes of the given byte string exactly as
 * libdivsufsort does (unsigned byte order, a proper prefix first), so the SA,
 * ISA and LCP equal the reference's divsufsort64 build word for word.  Inside
 * the device all coordinates are 32-bit, which bounds one instance (and one
 * batch) to 2^32 - 1 symbols; outputs are written in any stored width.
 *
 * Citations name files of the sufkit project (malabz/sufkit).
 */
#ifndef SUFGPU_SUFGPU_H
#define SUFGPU_SUFGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SUFGPU_ABI_VERSION 1

#if defined(__GNUC__)
#define SUFGPU_API __attribute__((visibility("default")))
#else
#define SUFGPU_API
#endif

/* Status codes.  Non-zero values are sufkit::ErrorCode + 1
 * (include/sufkit/types.hpp:708-721), so an adapter maps them one to one. */
typedef enum sufgpu_status {
  SUFGPU_OK = 0,
  SUFGPU_INVALID_INPUT = 1,    /* ErrorCode::kInvalidInput */
  SUFGPU_IO_ERROR = 2,         /* ErrorCode::kIoError */
  SUFGPU_UNSUPPORTED = 3,      /* ErrorCode::kUnsupportedBackend */
  SUFGPU_CORRUPT_INDEX = 4,    /* ErrorCode::kCorruptIndex */
  SUFGPU_VERSION_MISMATCH = 5, /* ErrorCode::kVersionMismatch */
  SUFGPU_BUILD_FAILURE = 6     /* ErrorCode::kBuildFailure (CUDA errors, OOM) */
} sufgpu_status;

/* LCP layouts; values equal detail::LcpEncoding (src/lcp_storage.hpp:53-59). */
typedef enum sufgpu_lcp_encoding {
  SUFGPU_LCP_NONE = 0,
  SUFGPU_LCP_RAW32 = 1,   /* uint32 per row */
  SUFGPU_LCP_RAW64 = 2,   /* uint64 per row */
  SUFGPU_LCP_BYTE32 = 3,  /* uint8 primary + uint32 anchors */
  SUFGPU_LCP_BYTE64 = 4   /* uint8 primary + uint64 anchors */
} sufgpu_lcp_encoding;

/* Build flags. */
#define SUFGPU_FLAG_VALIDATE 1u /* check the SA is a permutation (device) */
/* CRC-32 (zlib's crc32, the checksum of a .sufidx section) of every output
 * plane, computed on the device before the plane is copied out, into
 * stats.plane_crc (single builds).  A section's CRC follows from its header
 * bytes and these with zlib's crc32_combine. */
#define SUFGPU_FLAG_PLANE_CRC 2u
/* Also build the compact CHILD table (up / down / next-L links, one row
 * index per row, n = no link) of the row LCP into outputs.child as uint32
 * rows; the table BuildChildFor (src/suffix_array.cpp:1438-1496) builds for
 * the kLcpChild and kFull accelerations.  Single complete builds with an LCP
 * encoding other than none. */
#define SUFGPU_FLAG_CHILD 4u

/* What to build.  Stored widths follow CoordinateStorageWidth
 * (include/sufkit/types.hpp:100-111): 32 native, 40 split low32+high8,
 * 48 split low32+high16, 64 native. */
typedef struct sufgpu_build_desc {
  uint32_t sa_storage_bits;  /* 32, 40, 48 or 64 */
  uint32_t isa_storage_bits; /* 0 = no ISA output, else 32, 40, 48 or 64 */
  uint32_t lcp_encoding;     /* sufgpu_lcp_encoding */
  uint32_t flags;            /* SUFGPU_FLAG_* */
  /* 0 or 1 = complete arrays.  K > 1 keeps the suffixes at positions that are
   * multiples of K, as BuildDivsufsort's sampling_rate does
   * (src/divsufsort_backend.cpp:62-150): every plane then has ceil(n / K)
   * rows per instance, ISA[p / K] = sampled row, LCP = lcp of consecutive
   * sampled rows; byte-coded LCP puts anchors at sampled text positions
   * (src/lcp_storage.cpp:304-420 with rate K). */
  uint32_t sampling_rate;
  /* 0 = none.  1..10 = also build the Fast index's exact k-mer prefix
   * directory for this k (FastPrefixIndex, src/fast_prefix_index.cpp) into
   * outputs.prefix_intervals: 4^k uint64 entries begin | end << 32, (n, n) for
   * k-mers that do not occur (single complete builds; pick k with
   * sufgpu_prefix_select_k). */
  uint32_t prefix_k;
} sufgpu_build_desc;

/* Caller-owned output planes of one instance (n rows each).  Each pointer may
 * be host memory (pageable or pinned) or device memory of the context's
 * device; NULL skips that plane.
 *   sa_low/isa_low: uint32 rows for 32/40/48-bit widths, uint64 for 64;
 *   sa_high/isa_high: uint8 (40) or uint16 (48) rows, unused otherwise;
 *   lcp: uint32 / uint64 rows (raw) or uint8 primary bytes (byte-coded). */
typedef struct sufgpu_outputs {
  void *sa_low;
  void *sa_high;
  void *isa_low;
  void *isa_high;
  void *lcp;
  void *prefix_intervals; /* 4^prefix_k uint64 entries (desc.prefix_k > 0) */
  void *child;            /* n uint32 rows (SUFGPU_FLAG_CHILD) */
} sufgpu_outputs;

/* Byte-coded overflow anchors (text-ordered positions with their LCP values,
 * coordinates of 32 or 64 bits per the encoding).  Library-owned host memory,
 * valid until the next build on the same context or sufgpu_destroy. */
typedef struct sufgpu_anchors {
  const void *positions;
  const void *values;
  uint64_t count;
  uint32_t coordinate_bits;
} sufgpu_anchors;

/* Phase timings (CUDA events, seconds) and work counters of one build. */
typedef struct sufgpu_build_stats {
  double h2d_seconds;    /* text upload */
  double sa_seconds;     /* seed sort + doubling rounds (SA and ISA final) */
  double isa_seconds;    /* ISA packing */
  double lcp_seconds;    /* PHI, PLCP, row gather / byte coding */
  double storage_seconds;/* SA packing + validation */
  double d2h_seconds;    /* output download (not overlapped part) */
  double total_seconds;  /* whole call, wall clock */
  double device_seconds; /* first to last device event of the call */
  uint64_t symbols;
  uint32_t rounds;            /* doubling rounds after the seed */
  uint32_t seed_symbols;      /* symbols packed per seed key */
  uint64_t active_rows;       /* sum over rounds of still-unsorted rows */
  uint64_t active_first;      /* rows still unsorted after the seed */
  uint64_t irreducible_long;  /* PLCP positions finished by a warp */
  uint64_t anchors;
  uint32_t kernel_launches;   /* kernels launched by this call */
  uint32_t long_runs;         /* single-symbol runs split directly after the seed */
  uint32_t seg_sort_fallbacks;/* rounds whose groups did not fit the shared-memory sort */
  uint32_t seed_rare_rows;    /* two-bit seed: rows placed from the rare list */
  uint64_t prefix_kmers;      /* rows with a canonical k-mer (FastPrefixIndex::IndexedKmers) */
  uint64_t prefix_entries;    /* k-mers present (FastPrefixIndex::NonemptyEntries) */
  /* SUFGPU_FLAG_PLANE_CRC: CRC-32 of sa_low, sa_high, isa_low, isa_high, lcp
   * as written (0 for planes not written). */
  uint32_t plane_crc[5];
  uint32_t seed_code_bits;    /* bits per symbol of the seed sort key (2: two-bit seed) */
} sufgpu_build_stats;

typedef struct sufgpu_ctx sufgpu_ctx;

/* Context lifetime.  device is a CUDA ordinal. */
SUFGPU_API sufgpu_status sufgpu_create(sufgpu_ctx **ctx, int device);
SUFGPU_API void sufgpu_destroy(sufgpu_ctx *ctx);

/* Last error message of the context (or of a failed sufgpu_create when ctx is
 * NULL). */
SUFGPU_API const char *sufgpu_last_error(const sufgpu_ctx *ctx);

/* Largest text (symbols, sentinel included) one build accepts. */
SUFGPU_API uint64_t sufgpu_max_symbols(void);

/* zlib's crc32(crc_in, data, bytes) of device memory of the context's device
 * (the .sufidx section checksum, src/serialization.cpp:47-56, without a trip
 * through the host): 16 KiB chunks in parallel, folded by polynomial
 * multiplication.  No counterpart in the reference. */
SUFGPU_API sufgpu_status sufgpu_crc32_device(sufgpu_ctx *ctx, const void *data, uint64_t bytes,
                                             uint32_t crc_in, uint32_t *crc_out);

/* k of the Fast index's prefix directory, as FastPrefixIndex::SelectK with
 * its default options (src/fast_prefix_index.cpp:280-301): the largest k in
 * 8..10 whose directory (4^k entries of two 32-bit rows) fits 25% of
 * resident_core_bytes; 0 (no directory) below 2^16 suffixes. */
SUFGPU_API uint32_t sufgpu_prefix_select_k(uint64_t suffix_count, uint64_t resident_core_bytes);

/* Device bytes one build of n symbols needs with this descriptor. */
SUFGPU_API uint64_t sufgpu_device_bytes(uint64_t n, const sufgpu_build_desc *desc);

/* One complete build of text[0..n) (the logical text with its sentinel, as
 * SuffixArray::Build hands it to the constructor, src/suffix_array.cpp:
 * 4113-4117).  Replaces detail::BuildDivsufsort32/64
 * (src/divsufsort_backend.hpp:27-33, src/divsufsort_backend.cpp:24-157)
 * followed by RepackSuffixArray (src/suffix_array.cpp:852-910), BuildIsa
 * (src/suffix_array.cpp:1025-1047) and BuildLcp / BuildByteCodedLcpDirect /
 * FinalizeLcpStorage (src/suffix_array.cpp:1073-1170).
 * text may be host or device memory.  anchors may be NULL unless the encoding
 * is byte-coded.  stats may be NULL. */
SUFGPU_API sufgpu_status sufgpu_build(sufgpu_ctx *ctx, const uint8_t *text, uint64_t n,
                           const sufgpu_build_desc *desc,
                           const sufgpu_outputs *out, sufgpu_anchors *anchors,
                           sufgpu_build_stats *stats);

/* Drop-in for the libdivsufsort C entry point
 * saint_t divsufsort64(const sauchar_t *T, saidx64_t *SA, saidx64_t n)
 * (third_party/libdivsufsort/include/divsufsort64.h; divsufsort.c:331-358):
 * same arguments, same return codes (0 ok, -1 bad arguments, -2 failure). */
SUFGPU_API int sufgpu_divsufsort64(sufgpu_ctx *ctx, const uint8_t *T, int64_t *SA,
                        int64_t n);

/* Same for the 32-bit entry point divsufsort (divsufsort.h). */
SUFGPU_API int sufgpu_divsufsort(sufgpu_ctx *ctx, const uint8_t *T, int32_t *SA,
                      int32_t n);

/* One independent reference of a batch. */
typedef struct sufgpu_instance {
  const uint8_t *text; /* host or device */
  uint64_t n;
  sufgpu_outputs out;
  sufgpu_anchors anchors; /* filled for byte-coded encodings */
} sufgpu_instance;

/* Batched build: many references of uneven size sorted by the same launches
 * (per-instance segment offsets; rounds continue only while some instance has
 * unsorted groups).  Each instance's outputs equal its own sufgpu_build.
 * The sum of the sizes must not exceed sufgpu_max_symbols().  The reference
 * has no counterpart; it builds one reference per SuffixArray::Build call. */
SUFGPU_API sufgpu_status sufgpu_build_batch(sufgpu_ctx *ctx, sufgpu_instance *instances,
                                 uint32_t count, const sufgpu_build_desc *desc,
                                 sufgpu_build_stats *stats);

/* A collection larger than one launch (no counterpart in the reference, which
 * builds one reference per call): the instances are split in order into
 * sub-batches of at most batch_symbols symbols (0 = 2^30; a larger instance
 * alone) and 8192 instances, and `workers` contexts on this context's device
 * (this one plus up to 7 helpers it creates and keeps) build them side by side
 * from host threads, so one sub-batch's host copies overlap another's kernels.
 * Each sub-batch is one sufgpu_build_batch; every instance's planes equal a
 * single build of it.  Byte-coded anchors stay valid until the next
 * collection build or sufgpu_destroy.  stats: phase seconds, device_seconds
 * and counters summed over the sub-batches, total_seconds the whole call. */
SUFGPU_API sufgpu_status sufgpu_build_collection(sufgpu_ctx *ctx, sufgpu_instance *instances,
                                                 uint64_t count, const sufgpu_build_desc *desc,
                                                 uint64_t batch_symbols, uint32_t workers,
                                                 sufgpu_build_stats *stats);

/* Trace of the last sufgpu_build_collection on this context, one entry per
 * sub-batch in order: the worker that built it and the host clock (seconds
 * since the call began) when it started, took the workers' compute gate, left
 * it, and finished (copies included).  With one worker the gate times are the
 * start and the end. */
SUFGPU_API uint64_t sufgpu_collection_parts(const sufgpu_ctx *ctx);
SUFGPU_API sufgpu_status sufgpu_collection_trace(const sufgpu_ctx *ctx, uint64_t index,
                                                 uint32_t *worker, double times[4]);

/* Per-kernel profile: when enabled, every launch is bracketed by CUDA events
 * on the context stream and accumulated per kernel name with its algorithmic
 * bytes (the minimum it must read and write).  Enabling resets the totals. */
SUFGPU_API void sufgpu_set_profiling(sufgpu_ctx *ctx, int enable);
SUFGPU_API uint32_t sufgpu_profile_count(const sufgpu_ctx *ctx);
SUFGPU_API sufgpu_status sufgpu_profile_entry(const sufgpu_ctx *ctx, uint32_t index,
                                              const char **name, uint64_t *launches,
                                              double *seconds, uint64_t *bytes);

/* Tuning knobs (the autotuner, python -m sufkit_b200.autotune, sweeps them
 * per size class and writes sufkit_b200/tuning.json, which the Python
 * Context loads into sufgpu_set_tuning_class):
 *   "seed_symbols"  symbols packed per seed key, 0 = as many as fit 64 bits;
 *   "ballot_rank"   1 = onesweep ranks digits with ballots, 0 = match-any;
 *   "ballot_min_elems" smallest sort that uses ballot ranking;
 *   "sort_tile"     keys per onesweep tile: 2048 or 4096;
 *   "sort_block"    onesweep threads per 4096-key tile: 256 or 512 (2048-key
 *                   tiles always use 256);
 *   "packed_max_bits" instances of at most 2^v symbols use the packed
 *                   keys-only seed (index in the low key bits); 0 = never;
 *   "run_split"     1 = suffixes inside long single-symbol runs (N gaps) are
 *                   ordered directly after the seed, 0 = by the rounds;
 *   "seg_sort"      1 = each round sorts its groups inside shared memory
 *                   (global passes only when a group exceeds a block), 0 =
 *                   every round takes the global passes;
 *   "graph_rounds"  1 = a layout built before runs its rounds as a cached
 *                   CUDA graph of two rounds (one host synchronization per
 *                   pair), 0 = the host drives every round.  Builds with the
 *                   per-kernel profile on are always host-driven;
 *   "two_bit_seed"  1 = a single text of four consecutive byte values (A, C,
 *                   G, T) and few others sorts 2-bit seed keys, the windows
 *                   that hold another symbol placed exactly from a side
 *                   list; 0 = keys of the text's own code width always;
 *   "two_bit_min"   smallest text (symbols) that uses the two-bit seed;
 *   "two_bit_batch" 1 = batches use two-bit seeds too (per-instance side
 *                   lists);
 *   "seed_fused"    1 = the first seed pass generates its keys from the text
 *                   (no key write in position order);
 *   "seed_count_run" 1 = the histogram pass before a fused first pass counts
 *                   64 keys per thread, 0 = 16;
 *   "keys_sort_block" onesweep threads per 4096-key tile of keys-only sorts:
 *                   256 or 512;
 *   "rank_slots"    seed rank write by window slots: 0 never, 1 batches
 *                   only, 2 always (else by grouping passes);
 *   "rank_cluster"  0, 2 or 4: blocks per cluster that hold a 65536-position
 *                   window of a single text's rank write (0 = 2048-position
 *                   windows in one block);
 *   "batch_cluster" 1 = batches write ranks through 65536-position windows
 *                   per instance held by two-block clusters, 0 = by window
 *                   slots or 2048-position windows;
 *   "seg_small_group" round tiles whose groups have at most this many rows
 *                   rank by counting (0 = always radix passes);
 *   "seg_blocks"    round sort compiled for 2 or 3 blocks per SM;
 *   "seg_rank"      1 = the round sort also writes SA rows, ranks and the
 *                   next active list (no round_rank pass);
 *   "graph_shrink"  the graph rounds switch to a smaller bound once the
 *                   active rows fall below bound / graph_shrink;
 *   "tma_tile"      1 = single-segment onesweep tiles arrive by one bulk copy.
 * Results are identical for every setting; only speed changes. */
SUFGPU_API sufgpu_status sufgpu_set_tuning(sufgpu_ctx *ctx, const char *key, int64_t value);

/* Per-size overrides (the autotuner's table): a build whose longest instance
 * has at most max_symbols symbols applies the settings of the smallest such
 * class on top of the context's knobs, for that build only.  Keys and values
 * as for sufgpu_set_tuning (checked here). */
SUFGPU_API sufgpu_status sufgpu_set_tuning_class(sufgpu_ctx *ctx, uint64_t max_symbols,
                                                 const char *key, int64_t value);
SUFGPU_API void sufgpu_clear_tuning_classes(sufgpu_ctx *ctx);

/* ------------------------------------------------------------------------
 * Served builds (continuous batching).  A server owns one device arena and a
 * worker thread.  Requests are admitted while a free arena range can hold
 * them (HBM footprint); admitted references are seeded as a group and then
 * advance one doubling round per engine iteration side by side with every
 * other in-flight reference (each with its own prefix length), so requests
 * that arrive while others are on the GPU join the running work at the next
 * round.  A reference leaves as soon as it has no unsorted rows: its LCP is
 * computed, its planes are copied into the caller's outputs and its arena
 * range is freed.  Each result equals sufgpu_build of the same text.
 * The reference (sufkit) has no counterpart; it builds one reference per
 * SuffixArray::Build call on the calling thread.
 * ---------------------------------------------------------------------- */
typedef struct sufgpu_server sufgpu_server;

typedef struct sufgpu_server_config {
  uint64_t capacity_symbols; /* arena size in symbols (0 = 2^29); ~53 B each */
  uint32_t max_instances;    /* in-flight references (0 = 1024) */
  uint32_t flags;
} sufgpu_server_config;

typedef struct sufgpu_request_info {
  double queue_seconds;   /* submit -> admitted */
  double latency_seconds; /* submit -> outputs complete */
  uint32_t rounds;        /* doubling rounds the reference took */
  uint32_t seed_symbols;
  sufgpu_anchors anchors; /* byte-coded encodings; valid until release */
  /* Continuous batching: the server's iteration count (shared doubling
   * rounds completed) when the request was admitted and when it finished,
   * and how many requests were already in flight, mid-rounds, when it was
   * merged into the running batch. */
  uint64_t admit_iteration;
  uint64_t finish_iteration;
  uint32_t inflight_at_admit;
  uint32_t reserved;
} sufgpu_request_info;

typedef struct sufgpu_server_stats {
  uint64_t completed;
  uint64_t symbols;
  uint64_t iterations;
  uint64_t max_inflight;
  uint64_t queued;
  uint64_t inflight;
  double p50_seconds;
  double p99_seconds;
  double span_seconds;      /* first submit -> last completion */
  double symbols_per_second;
} sufgpu_server_stats;

SUFGPU_API sufgpu_status sufgpu_server_create(sufgpu_server **server, int device,
                                              const sufgpu_server_config *config);
/* Finishes every queued and in-flight request, then frees the server. */
SUFGPU_API void sufgpu_server_destroy(sufgpu_server *server);
/* text and the output planes are caller memory (host or device) that must
 * stay valid until the request completes. */
SUFGPU_API sufgpu_status sufgpu_server_submit(sufgpu_server *server, const uint8_t *text,
                                              uint64_t n, const sufgpu_build_desc *desc,
                                              const sufgpu_outputs *out, uint64_t *ticket);
/* Blocks until the request completes; returns its status. */
SUFGPU_API sufgpu_status sufgpu_server_wait(sufgpu_server *server, uint64_t ticket,
                                            sufgpu_request_info *info);
SUFGPU_API sufgpu_status sufgpu_server_poll(sufgpu_server *server, uint64_t ticket, int *done);
/* Forgets a completed request (its anchors become invalid). */
SUFGPU_API sufgpu_status sufgpu_server_release(sufgpu_server *server, uint64_t ticket);
SUFGPU_API sufgpu_status sufgpu_server_get_stats(sufgpu_server *server,
                                                 sufgpu_server_stats *stats);

/* Pinned host memory helpers (fast transfers for callers that can use them). */
SUFGPU_API void *sufgpu_host_alloc(uint64_t bytes);
SUFGPU_API void sufgpu_host_free(void *ptr);

/* Largest n accepted by sufgpu_lcp_noalloc. */
#define SUFGPU_NOALLOC_MAX_SYMBOLS (1u << 18)

/* LCP[r] = lcp(SA[r-1], SA[r]) of a device-resident text and suffix array,
 * written to a device array, for callers that can't allocate device memory:
 * code running under another framework's allocator (its pool owns the
 * device, so a foreign cudaMalloc fails or fragments it), callbacks that run
 * while an allocation lock is held, and loops that cannot block on an
 * allocation.  Its scratch is one fixed array compiled into the library
 * (11.4 MiB, held on every GPU that loads the library until exit); it calls
 * no cudaMalloc, cudaFree or allocating library routine.  n above
 * SUFGPU_NOALLOC_MAX_SYMBOLS returns SUFGPU_INVALID_INPUT.  sa must be a
 * permutation of [0, n); an entry outside that range is detected on the
 * device and returns SUFGPU_BUILD_FAILURE.  All calls share the array (each
 * clears what must start at zero), so calls that overlap on the GPU race and
 * must be serialized by the caller.  The first call on a device does that
 * device's set-up (resolves the array's address and a kernel attribute with
 * the device current); make it before any stream capture begins.  stream is
 * a cudaStream_t (NULL = default stream); the call returns after the result
 * is complete.  This entry point has no counterpart in the reference. */
SUFGPU_API sufgpu_status sufgpu_lcp_noalloc(const uint8_t *text, const uint32_t *sa,
                                            uint64_t n, uint32_t *lcp, void *stream);

/* Normalizes FASTA (plain or gzip) exactly like GenomeReference::FromFasta
 * (src/genome_reference.cpp:30-57, 131-156, 222-268): A/C/G/T (any case) ->
 * 2..5, every other byte -> 6, a 1 after every record.  Writes at most cap
 * bytes to out (no sentinel) and stores the full size in *size; returns
 * SUFGPU_INVALID_INPUT for malformed input, SUFGPU_IO_ERROR if unreadable.
 * fingerprint (FNV-1a 64 of the bytes, src/genome_reference.cpp:125-129) and
 * records may be NULL. */
SUFGPU_API sufgpu_status sufgpu_encode_fasta(const char *path, uint8_t *out, uint64_t cap,
                                  uint64_t *size, uint64_t *fingerprint,
                                  uint64_t *records);

/* The same normalisation on the device, for FASTA already in memory: raw is
 * `bytes` bytes of plain (uncompressed) FASTA in host memory; out (host or
 * device, cap bytes) receives the logical bytes without the sentinel, *size
 * their count, *fingerprint their FNV-1a 64 (computed on the device; may be
 * NULL) and *records the record count (may be NULL).  Record names and
 * sequences are validated as GenomeReference::FromFasta does
 * (src/genome_reference.cpp:88-122, 222-268).  Returns SUFGPU_UNSUPPORTED for
 * input this path does not parse -- FASTQ records ('@' headers, '+' lines)
 * and a lone carriage-return line right after a header, which kseq keeps as
 * a base -- so the caller reads those with sufgpu_encode_fasta.  Replaces
 * the per-byte loop of ReferenceBuilder::AppendRecord / AppendByte
 * (src/genome_reference.cpp:125-156). */
SUFGPU_API sufgpu_status sufgpu_encode_fasta_device(sufgpu_ctx *ctx, const uint8_t *raw,
                                                    uint64_t bytes, uint8_t *out, uint64_t cap,
                                                    uint64_t *size, uint64_t *fingerprint,
                                                    uint64_t *records);

#ifdef __cplusplus
}
#endif

#endif /* SUFGPU_SUFGPU_H */
