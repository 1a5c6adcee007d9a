/* CPU oracle for maximal k-biplex enumeration -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the oracle the tests and bench.py's CPU leg compare the
 * CUDA enumerator against.  The product never links or calls it.
 *
 * Graph: CSR over global ids, U = [0, n_left), V = [n_left, n); rows sorted.
 * Result set: every maximal k-biplex (X, Y), X in U, Y in V, both non-empty.
 * A result's canonical hash is gmk_result_hash() over its member ids; a set of
 * results is summarised by (count, wrapping sum of h1, xor of h2).
 */
#ifndef GMK_KBIPLEX_ORACLE_H
#define GMK_KBIPLEX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t count;
    uint64_t hash_sum;   /* sum of h1 over results, mod 2^64 */
    uint64_t hash_xor;   /* xor of h2 over results */
    uint64_t nodes;      /* search-tree nodes visited */
    int      truncated;  /* 1 if result_limit stopped the run */
} oracle_stats;

/* Called once per result; X and Y hold global ids, sorted ascending.
 * Return non-zero to stop the enumeration. */
typedef int (*oracle_sink)(void* user, const uint32_t* x, uint32_t nx,
                           const uint32_t* y, uint32_t ny);

/* Enumerate all maximal k-biplexes (k >= 1).  n must be <= ORACLE_MAX_N.
 * result_limit 0 = unlimited.  Returns 0, or -1 on bad arguments. */
int oracle_enumerate(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                     uint32_t n_left, uint32_t k, uint64_t result_limit,
                     oracle_sink sink, void* user, oracle_stats* out);

/* Same, restricted to the roots x (smallest U vertex of a result) with
 * x % nshards == shard: the shards partition the result set. */
int oracle_enumerate_shard(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                           uint32_t n_left, uint32_t k, uint64_t result_limit,
                           uint32_t shard, uint32_t nshards,
                           oracle_sink sink, void* user, oracle_stats* out);

/* Canonical per-result hash pair of a vertex-id set (order-independent). */
void oracle_result_hash(const uint32_t* ids, uint32_t n_ids, uint32_t nx,
                        uint32_t ny, uint64_t* h1, uint64_t* h2);

/* Is (X, Y) a k-biplex, and is it maximal?  Returns 0 not a k-biplex,
 * 1 k-biplex but not maximal, 2 maximal. */
int oracle_classify(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                    uint32_t n_left, uint32_t k, const uint32_t* x, uint32_t nx,
                    const uint32_t* y, uint32_t ny);

#define ORACLE_MAX_N 16384u

#ifdef __cplusplus
}
#endif
#endif
