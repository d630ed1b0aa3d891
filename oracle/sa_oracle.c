/* Test infrastructure only: CPU oracle for the SA + ISA + LCP build path.
 * See sa_oracle.h for the contract and how parity with the reference is
 * pinned.  Citations are paths inside the sufkit project. */
#include "sa_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * Suffix sort by prefix doubling with two stable counting-sort passes per
 * round (Manber-Myers).  rank 0 means "past the end of the text", so a proper
 * prefix sorts before any extension, which is the order libdivsufsort gives
 * for the sentinel-terminated text built at src/suffix_array.cpp:4113-4117.
 * ------------------------------------------------------------------------- */
static int counting_pass(const uint64_t *in, uint64_t *out, uint64_t n,
                         const uint64_t *key, uint64_t key_range,
                         uint64_t *count) {
  memset(count, 0, (size_t)(key_range + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n; ++i) count[key[in[i]] + 1]++;
  for (uint64_t k = 1; k <= key_range; ++k) count[k] += count[k - 1];
  for (uint64_t i = 0; i < n; ++i) out[count[key[in[i]]]++] = in[i];
  return 0;
}

int oracle_suffix_sort(const uint8_t *text, uint64_t n, uint64_t *sa) {
  if (n == 0) return 0;
  uint64_t *rank = malloc((size_t)n * sizeof(uint64_t));
  uint64_t *second = malloc((size_t)n * sizeof(uint64_t));
  uint64_t *tmp = malloc((size_t)n * sizeof(uint64_t));
  uint64_t range = n + 2 > 258 ? n + 2 : 258;
  uint64_t *count = malloc((size_t)(range + 1) * sizeof(uint64_t));
  if (!rank || !second || !tmp || !count) {
    free(rank); free(second); free(tmp); free(count);
    return -1;
  }
  for (uint64_t i = 0; i < n; ++i) {
    rank[i] = (uint64_t)text[i] + 1;
    sa[i] = i;
  }
  uint64_t key_range = 257;
  for (uint64_t h = 1;; h <<= 1) {
    for (uint64_t i = 0; i < n; ++i) second[i] = i + h < n ? rank[i + h] : 0;
    counting_pass(sa, tmp, n, second, key_range, count);
    counting_pass(tmp, sa, n, rank, key_range, count);
    /* New ranks: 1 + number of distinct (rank, second) pairs before. */
    tmp[sa[0]] = 1;
    uint64_t classes = 1;
    for (uint64_t r = 1; r < n; ++r) {
      const uint64_t a = sa[r - 1], b = sa[r];
      if (rank[a] != rank[b] || second[a] != second[b]) ++classes;
      tmp[b] = classes;
    }
    memcpy(rank, tmp, (size_t)n * sizeof(uint64_t));
    key_range = classes + 1;
    if (classes == n || h >= n) break;
  }
  free(rank); free(second); free(tmp); free(count);
  return 0;
}

/* ISA scatter: src/suffix_array.cpp:976-1047 (BuildIsaFor) with K = 1. */
int oracle_isa(const uint64_t *sa, uint64_t n, uint64_t *isa) {
  if (!oracle_is_permutation(sa, n)) return -1;
  for (uint64_t r = 0; r < n; ++r) isa[sa[r]] = r;
  return 0;
}

/* Permutation bitmap: src/suffix_array.cpp:852-910 (RepackSuffixArray). */
int oracle_is_permutation(const uint64_t *sa, uint64_t n) {
  uint8_t *seen = calloc((size_t)(n ? n : 1), 1);
  if (!seen) return 0;
  int ok = 1;
  for (uint64_t r = 0; r < n && ok; ++r) {
    if (sa[r] >= n || seen[sa[r]]) ok = 0;
    else seen[sa[r]] = 1;
  }
  free(seen);
  return ok;
}

static uint64_t common_prefix(const uint8_t *a, const uint8_t *b,
                              uint64_t limit) {
  uint64_t i = 0;
  while (i < limit && a[i] == b[i]) ++i;
  return i;
}

/* Generalized Kasai with K = 1: src/divsufsort_backend.cpp:121-150; the byte
 * scan is LongestCommonPrefixBytes, src/sequence_compare.hpp:153-157. */
void oracle_kasai_lcp(const uint8_t *text, uint64_t n, const uint64_t *sa,
                      const uint64_t *isa, uint64_t *lcp) {
  uint64_t common = 0;
  memset(lcp, 0, (size_t)n * sizeof(uint64_t));
  for (uint64_t p = 0; p < n; ++p) {
    const uint64_t row = isa[p];
    if (row != 0) {
      const uint64_t prev = sa[row - 1];
      if (p + common < n && prev + common < n) {
        const uint64_t a = n - (p + common), b = n - (prev + common);
        common += common_prefix(text + p + common, text + prev + common,
                                a < b ? a : b);
      }
      lcp[row] = common;
    }
    common = common > 1 ? common - 1 : 0;
  }
}

/* BuildByteDataDirect with K = 1: src/lcp_storage.cpp:304-420.  An anchor
 * opens at text position p when LCP >= 255 and p does not continue the run
 * of p-1 (previous overflow value minus one equals this value). */
int64_t oracle_bytecode_lcp(const uint8_t *text, uint64_t n,
                            const uint64_t *sa, const uint64_t *isa,
                            int coordinate_width, uint8_t *primary,
                            uint64_t *anchor_pos, uint64_t *anchor_val,
                            uint64_t anchor_cap) {
  const uint64_t limit = coordinate_width == 32 ? 0xffffffffull : ~0ull;
  uint64_t common = 0, anchors = 0, prev_value = 0;
  int prev_overflow = 0;
  for (uint64_t p = 0; p < n; ++p) {
    const uint64_t row = isa[p];
    uint64_t value = 0;
    if (row == 0) {
      common = 0;
    } else {
      const uint64_t prev = sa[row - 1];
      const uint64_t a = n - p - common, b = n - prev - common;
      common += common_prefix(text + p + common, text + prev + common,
                              a < b ? a : b);
      value = common;
    }
    if (value > limit) return -1;
    primary[row] = (uint8_t)(value < 255 ? value : 255);
    if (value < 255) {
      prev_overflow = 0;
    } else {
      const int continues =
          prev_overflow && prev_value >= 1 && prev_value - 1 == value;
      if (!continues) {
        if (anchors >= anchor_cap) return -1;
        anchor_pos[anchors] = p;
        anchor_val[anchors] = value;
        ++anchors;
      }
      prev_overflow = 1;
      prev_value = value;
    }
    common = common > 1 ? common - 1 : 0;
  }
  return (int64_t)anchors;
}

/* BuildGuide: src/lcp_storage.cpp:54-95. */
uint64_t oracle_bytecode_guide(const uint64_t *anchor_pos, uint64_t anchors,
                               uint64_t n, uint64_t *guide) {
  if (n == 0) return 0;
  const uint64_t blocks = 1 + (n - 1) / 4096;
  uint64_t a = 0;
  for (uint64_t b = 0; b <= blocks; ++b) {
    while (a < anchors && anchor_pos[a] < b * 4096) ++a;
    guide[b] = a;
  }
  return blocks + 1;
}

/* DecodeByte / FindAnchor: src/lcp_storage.cpp:165-215 (K = 1). */
uint64_t oracle_bytecode_exact(const uint8_t *primary,
                               const uint64_t *anchor_pos,
                               const uint64_t *anchor_val, uint64_t anchors,
                               uint64_t row, uint64_t suffix) {
  if (primary[row] < 255) return primary[row];
  uint64_t lo = 0, hi = anchors; /* last anchor with position <= suffix */
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (anchor_pos[mid] <= suffix) lo = mid + 1;
    else hi = mid;
  }
  if (lo == 0) return ~0ull;
  return anchor_val[lo - 1] - (suffix - anchor_pos[lo - 1]);
}

/* Width policy and packing: SelectCoordinateStorageWidth /
 * ResolveCoordinateStorageWidth (src/coordinate_storage.cpp:363-393),
 * ValidateValues (src/coordinate_storage.cpp:60-77) and Pack32/40/48/64
 * (src/coordinate_storage.cpp:131-173). */
int oracle_pack(const uint64_t *values, uint64_t count, uint64_t symbol_count,
                int storage_bits, uint32_t *low32, void *high,
                uint64_t *native64) {
  if (symbol_count == 0) return -1;
  const uint64_t top = symbol_count - 1;
  int width = storage_bits;
  if (width == 0) {
    width = top <= 0xffffffffull ? 32
            : top <= 0xffffffffffull ? 40
            : top <= 0xffffffffffffull ? 48 : 64;
  }
  const uint64_t maximum = width == 32 ? 0xffffffffull
                           : width == 40 ? 0xffffffffffull
                           : width == 48 ? 0xffffffffffffull : ~0ull;
  if (width != 32 && width != 40 && width != 48 && width != 64) return -1;
  if (top > maximum) return -1;
  for (uint64_t i = 0; i < count; ++i) {
    if (values[i] >= symbol_count || values[i] > maximum) return -1;
  }
  for (uint64_t i = 0; i < count; ++i) {
    const uint64_t v = values[i];
    if (width == 64) {
      native64[i] = v;
    } else {
      low32[i] = (uint32_t)v;
      if (width == 40) ((uint8_t *)high)[i] = (uint8_t)(v >> 32);
      if (width == 48) ((uint16_t *)high)[i] = (uint16_t)(v >> 32);
    }
  }
  return width;
}

/* Compact CHILD table (up / down / next-L links in one entry per row) of a
 * row-order LCP array: BuildChildFor, src/suffix_array.cpp:1438-1496.  The
 * first monotone-stack pass writes down links at the stack entry below each
 * popped interval and up links at index - 1; the second pass writes next-L
 * links between equal LCP values, overriding.  `none` (n) marks no link. */
void oracle_child(const uint64_t *lcp, uint64_t n, uint64_t *child) {
  if (n == 0) return;
  const uint64_t none = n;
  uint64_t *stack = (uint64_t *)malloc(n * sizeof(uint64_t));
  if (!stack) return;
  for (uint64_t i = 0; i < n; ++i) child[i] = none;
  uint64_t top = 0; /* number of entries */
  stack[top++] = 0;
  for (uint64_t i = 1; i < n; ++i) {
    const uint64_t cur = lcp[i];
    uint64_t last = none;
    while (top > 0 && cur < lcp[stack[top - 1]]) {
      last = stack[--top];
      if (top > 0 && cur <= lcp[stack[top - 1]] && lcp[stack[top - 1]] != lcp[last]) {
        child[stack[top - 1]] = last;
      }
    }
    if (last != none) child[i - 1] = last;
    stack[top++] = i;
  }
  while (top > 0 && lcp[stack[top - 1]] > 0) {
    const uint64_t last = stack[--top];
    if (top > 0 && lcp[stack[top - 1]] != lcp[last]) child[stack[top - 1]] = last;
  }
  top = 0;
  stack[top++] = 0;
  for (uint64_t i = 1; i < n; ++i) {
    while (top > 0 && lcp[i] < lcp[stack[top - 1]]) --top;
    if (top > 0 && lcp[i] == lcp[stack[top - 1]]) {
      const uint64_t last = stack[--top];
      child[last] = i;
    }
    stack[top++] = i;
  }
  free(stack);
}
