/* Test infrastructure only: the CPU oracle for the SA + ISA + LCP build path.
 *
 * A plain-C restatement of the reference's build path, used by tests/ (as the
 * checker), by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py.
 * The product library never links or loads it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own compiled code (oracle/_ref/libsufref.so, built from the
 * sufkit sources by oracle/Makefile) and against the golden vectors committed
 * under tests/golden/.
 *
 * The suffix order itself is unique once every suffix is distinct (the build
 * appends a unique 0 sentinel), so the sort below is a straightforward
 * prefix-doubling sort rather than a restatement of libdivsufsort's induced
 * sorting; its output is compared word for word with divsufsort64.
 */
#ifndef SUFGPU_ORACLE_H
#define SUFGPU_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Complete suffix array of text[0..n) in unsigned-byte order, a proper prefix
 * ordering first.  Returns 0, or -1 on allocation failure. */
int oracle_suffix_sort(const uint8_t *text, uint64_t n, uint64_t *sa);

/* isa[sa[r]] = r; returns -1 if sa is not a permutation of [0, n). */
int oracle_isa(const uint64_t *sa, uint64_t n, uint64_t *isa);

/* Kasai LCP in row order (LCP[0] = 0). */
void oracle_kasai_lcp(const uint8_t *text, uint64_t n, const uint64_t *sa,
                      const uint64_t *isa, uint64_t *lcp);

/* Byte-coded LCP: primary[row] = min(LCP, 255) plus text-ordered overflow
 * anchors.  Returns the anchor count, or -1 when anchor_cap is too small or
 * an LCP value exceeds the coordinate width (32 or 64). */
int64_t oracle_bytecode_lcp(const uint8_t *text, uint64_t n,
                            const uint64_t *sa, const uint64_t *isa,
                            int coordinate_width, uint8_t *primary,
                            uint64_t *anchor_pos, uint64_t *anchor_val,
                            uint64_t anchor_cap);

/* Derived 4096-symbol guide: guide[b] = first anchor at or after b*4096,
 * for b in [0, blocks]; blocks = 1 + (n-1)/4096.  Returns guide length. */
uint64_t oracle_bytecode_guide(const uint64_t *anchor_pos, uint64_t anchors,
                               uint64_t n, uint64_t *guide);

/* Decodes one byte-coded row (the value LcpStorage::Exact returns). */
uint64_t oracle_bytecode_exact(const uint8_t *primary,
                               const uint64_t *anchor_pos,
                               const uint64_t *anchor_val, uint64_t anchors,
                               uint64_t row, uint64_t suffix);

/* Coordinate packing with range validation.  storage_bits 32/40/48/64 (0 =
 * narrowest).  Writes low32 (+ high plane) or native64.  Returns the resolved
 * width, or -1 (a value >= symbol_count or above the width's maximum). */
int oracle_pack(const uint64_t *values, uint64_t count, uint64_t symbol_count,
                int storage_bits, uint32_t *low32, void *high,
                uint64_t *native64);

/* Permutation check used before packing: every value < n and seen once. */
int oracle_is_permutation(const uint64_t *sa, uint64_t n);

/* Compact CHILD table of a row-order LCP (src/suffix_array.cpp:1438-1496);
 * child[i] = n marks no link. */
void oracle_child(const uint64_t *lcp, uint64_t n, uint64_t *child);

#ifdef __cplusplus
}
#endif

#endif
