/*
 * oracle/pss_oracle.h -- TEST INFRASTRUCTURE, not part of the product.
 *
 * Plain-C restatement of the reference pS5 path, used only as a checker by
 * tests/, the smoke check and the CPU-baseline leg of bench.py. Parity of this
 * restatement is pinned against the reference pS5 itself (oracle/_ref,
 * compiled from the reference sources) by tests/test_oracle.py.
 *
 * String model (the reference's UCharStringSet, src/tools/stringset.hpp):
 * string i starts at chars + offs[i] and ends at its first NUL byte. String
 * ids are u32. Sorted outputs are permutations of ids; LCP arrays follow the
 * reference convention lcp[i] = LCP(str[i-1], str[i]) for i >= 1 and lcp[0]
 * is never written (src/parallel/bingmann-parallel_sample_sort.hpp:1759-1769).
 */
#ifndef PSS_ORACLE_H
#define PSS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 8 chars at s+depth, big-endian, bytes from the first NUL on are zero. */
uint64_t pso_get_uint64(const uint8_t* s, size_t depth);
/* chars shared by two keys (8 if equal). */
unsigned pso_lcp_key_type(uint64_t a, uint64_t b);
/* number of non-NUL chars held by a key. */
unsigned pso_lcp_key_depth(uint64_t a);

/* Sort ids (in place) by the strings they name; lcp may be NULL. */
void pso_sort_lcp(const uint8_t* chars, const uint64_t* offs, uint32_t* ids,
                  size_t n, uint64_t* lcp);

/* Bucket ids of keys under a sorted splitter array of length k: 2*r where
 * r = #splitters < key, plus 1 when key equals splitter r. */
void pso_classify(const uint64_t* splitters, size_t k, const uint64_t* keys,
                  size_t n, uint16_t* out);

/* -1 when ids are in non-decreasing string order, else the first index i
 * with str[i-1] > str[i]. */
int64_t pso_check_order(const uint8_t* chars, const uint64_t* offs,
                        const uint32_t* ids, size_t n);
/* 1 when ids is a permutation of 0..n-1. */
int pso_check_permutation(const uint32_t* ids, size_t n);
/* lcp[i] = LCP(str[ids[i-1]], str[ids[i]]) for i >= 1; lcp[0] untouched. */
void pso_lcp_array(const uint8_t* chars, const uint64_t* offs,
                   const uint32_t* ids, size_t n, uint64_t* lcp);
/* -1 when the u32 LCP array matches the strings, else the first bad index. */
int64_t pso_check_lcp32(const uint8_t* chars, const uint64_t* offs,
                        const uint32_t* ids, size_t n, const uint32_t* lcp);
/* Distinguishing prefix D and LCP sum of a sorted id list
 * (src/tools/checker.hpp:155-180). */
uint64_t pso_dprefix(const uint8_t* chars, const uint64_t* offs,
                     const uint32_t* ids, size_t n, uint64_t* lcpsum);

#ifdef __cplusplus
}
#endif

#endif
