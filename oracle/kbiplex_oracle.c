/* CPU oracle for maximal k-biplex enumeration -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/ and by bench.py's CPU leg as the oracle; the product path
 * (gmkbe_b200's CUDA library) never links, loads or calls this file.
 *
 * It restates, on a dense adjacency matrix and with one plain recursion, the
 * semantics of the reference enumerator:
 *   - the top-level loop over U vertices in id order, earlier vertices forming
 *     the exclusion queue (reference src/main.cu:1078-1111 loop over Cand_exts,
 *     src/main.cu:1489 new_Cand_q->push);
 *   - the candidate filter "a V vertex stays while it misses at most k of X"
 *     (G_state[y] >= |X|-k, reference src/main.cu:504-523 and :1270-1278) and
 *     its mirror for U vertices against Y (ext_q / ext_p filters, reference
 *     include/for_generate.cuh:407-429);
 *   - the exclusion test "an excluded vertex that fits every extension kills
 *     the branch" (reference src/main.cu:1290-1304 any_satisfied over Cand_q);
 *   - the maximality test "no excluded vertex can be added: it misses more
 *     than k of the other side, or misses a vertex that already misses k"
 *     (reference include/for_checkmaximality.cuh:3109-3303, difference-set
 *     test at :70-175).
 * Unlike the reference GPU code (theta fixed to 1 at src/main.cu:1585, whose
 * recursive branch at :1120 is then unreachable), the recursion here explores
 * both sides fully, so the output is the complete set of maximal k-biplexes
 * with both sides non-empty -- the set the reference's BPPivot baseline
 * (baselines/MaximalBiPlex, src/biplex/biplex.cpp:781-1082) prints with -q 1.
 */
#include "kbiplex_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ hashing */

static uint64_t mix64(uint64_t z) {
    /* splitmix64 finaliser (Steele, Lea, Flood 2014) */
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void oracle_result_hash(const uint32_t* ids, uint32_t n_ids, uint32_t nx, uint32_t ny,
                        uint64_t* h1, uint64_t* h2) {
    uint64_t a = 0, b = 0;
    for (uint32_t i = 0; i < n_ids; ++i) {
        uint64_t e = mix64((uint64_t)ids[i] * 2u + 1u);
        a += e;
        b += mix64(e ^ 0x5851F42D4C957F2Dull);
    }
    *h1 = mix64(a + (uint64_t)nx * 0x100000001B3ull + (uint64_t)ny);
    *h2 = mix64(b ^ (((uint64_t)nx << 32) | (uint64_t)ny));
}

/* ------------------------------------------------------------------ context */

typedef struct {
    uint32_t n, nl, k, words;
    uint64_t* adjbits;          /* n rows of `words` u64 */
    uint64_t limit;
    oracle_sink sink;
    void* user;
    oracle_stats* st;
    int stop;
    uint32_t* S;                /* members of the current biplex */
    uint32_t* mc;               /* mc[v]: misses of member v inside S (indexed by id) */
    uint32_t ns, ns_side[2];
    uint32_t* scratch;          /* result emission buffer */
    uint64_t* sc_bits[2];       /* per-depth scratch: (S u C) per side, reused */
} ctx_t;

static inline int side_of(const ctx_t* c, uint32_t v) { return v >= c->nl; }

static inline int adjacent(const ctx_t* c, uint32_t a, uint32_t b) {
    return (int)((c->adjbits[(size_t)a * c->words + (b >> 6)] >> (b & 63)) & 1u);
}

/* Can w join S?  w misses at most k members of S on the other side, and every
 * member it misses still has room (misses < k). */
static int compatible(const ctx_t* c, uint32_t w) {
    int s = side_of(c, w);
    uint32_t miss = 0;
    if (c->ns_side[1 - s] == 0) return 1;
    for (uint32_t i = 0; i < c->ns; ++i) {
        uint32_t m = c->S[i];
        if (side_of(c, m) == s || adjacent(c, w, m)) continue;
        if (++miss > c->k || c->mc[m] >= c->k) return 0;
    }
    return 1;
}

static void push_member(ctx_t* c, uint32_t v) {
    int s = side_of(c, v);
    uint32_t miss = 0;
    for (uint32_t i = 0; i < c->ns; ++i) {
        uint32_t m = c->S[i];
        if (side_of(c, m) == s || adjacent(c, v, m)) continue;
        ++miss;
        ++c->mc[m];
    }
    c->mc[v] = miss;
    c->S[c->ns++] = v;
    c->ns_side[s]++;
}

static void pop_member(ctx_t* c) {
    uint32_t v = c->S[--c->ns];
    int s = side_of(c, v);
    c->ns_side[s]--;
    for (uint32_t i = 0; i < c->ns; ++i) {
        uint32_t m = c->S[i];
        if (side_of(c, m) == s || adjacent(c, v, m)) continue;
        --c->mc[m];
    }
    c->mc[v] = 0;
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return (x > y) - (x < y);
}

static void emit(ctx_t* c) {
    uint32_t* buf = c->scratch;
    memcpy(buf, c->S, c->ns * sizeof(uint32_t));
    qsort(buf, c->ns, sizeof(uint32_t), cmp_u32);
    uint32_t nx = c->ns_side[0], ny = c->ns_side[1];
    uint64_t h1, h2;
    oracle_result_hash(buf, c->ns, nx, ny, &h1, &h2);
    c->st->count++;
    c->st->hash_sum += h1;
    c->st->hash_xor ^= h2;
    if (c->sink && c->sink(c->user, buf, nx, buf + nx, ny)) c->stop = 1;
    if (c->limit && c->st->count >= c->limit) {
        c->stop = 1;
        c->st->truncated = 1;
    }
}

/* Exclusion prune: some excluded e would be addable to every leaf below,
 * i.e. to every S u T with T a subset of C.  Sufficient: e misses at most k
 * of (S u C) on the other side and each member w it misses has fewer than k
 * misses inside S u C. */
static int excluded_vertex_dominates(ctx_t* c, const uint32_t* C, uint32_t nc,
                                     const uint32_t* E, uint32_t ne) {
    if (ne == 0) return 0;
    uint32_t W = c->words;
    uint64_t* sc[2] = {c->sc_bits[0], c->sc_bits[1]};
    memset(sc[0], 0, W * sizeof(uint64_t));
    memset(sc[1], 0, W * sizeof(uint64_t));
    uint32_t cnt[2] = {0, 0};
    for (uint32_t i = 0; i < c->ns; ++i) {
        uint32_t v = c->S[i];
        sc[side_of(c, v)][v >> 6] |= 1ull << (v & 63);
        cnt[side_of(c, v)]++;
    }
    for (uint32_t i = 0; i < nc; ++i) {
        uint32_t v = C[i];
        sc[side_of(c, v)][v >> 6] |= 1ull << (v & 63);
        cnt[side_of(c, v)]++;
    }
    for (uint32_t i = 0; i < ne; ++i) {
        uint32_t e = E[i];
        int s = side_of(c, e), o = 1 - s;
        const uint64_t* row = c->adjbits + (size_t)e * W;
        uint32_t hit = 0;
        for (uint32_t w = 0; w < W; ++w) hit += (uint32_t)__builtin_popcountll(row[w] & sc[o][w]);
        if (cnt[o] - hit > c->k) continue;
        /* every member w of (S u C) on side o that e misses needs < k misses */
        int ok = 1;
        for (uint32_t w = 0; w < W && ok; ++w) {
            uint64_t missed = sc[o][w] & ~row[w];
            while (missed && ok) {
                uint32_t v = (w << 6) + (uint32_t)__builtin_ctzll(missed);
                missed &= missed - 1;
                const uint64_t* rv = c->adjbits + (size_t)v * W;
                uint32_t h = 0;
                for (uint32_t q = 0; q < W; ++q) h += (uint32_t)__builtin_popcountll(rv[q] & sc[s][q]);
                if (cnt[s] - h >= c->k) ok = 0;
            }
        }
        if (ok) return 1;
    }
    return 0;
}

/* C: compatible undecided vertices (V first, then U, each in id order).
 * E: compatible excluded vertices.  Both are owned by the caller. */
static void branch(ctx_t* c, const uint32_t* C, uint32_t nc, const uint32_t* E, uint32_t ne) {
    if (c->stop) return;
    c->st->nodes++;
    if (c->ns_side[1] == 0) {                 /* Y must end up non-empty */
        int anyV = 0;
        for (uint32_t i = 0; i < nc && !anyV; ++i) anyV = side_of(c, C[i]);
        if (!anyV) return;
    }
    if (nc == 0) {                            /* leaf: E holds exactly the addable outsiders */
        if (ne == 0 && c->ns_side[0] && c->ns_side[1]) emit(c);
        return;
    }
    if (excluded_vertex_dominates(c, C, nc, E, ne)) return;

    uint32_t* nC = (uint32_t*)malloc((size_t)(nc + 1) * sizeof(uint32_t));
    uint32_t* nE = (uint32_t*)malloc((size_t)(ne + nc + 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < nc && !c->stop; ++i) {
        uint32_t v = C[i];
        push_member(c, v);
        uint32_t a = 0, b = 0;
        for (uint32_t j = i + 1; j < nc; ++j)
            if (compatible(c, C[j])) nC[a++] = C[j];
        for (uint32_t j = 0; j < ne; ++j)
            if (compatible(c, E[j])) nE[b++] = E[j];
        for (uint32_t j = 0; j < i; ++j)      /* earlier siblings are excluded */
            if (compatible(c, C[j])) nE[b++] = C[j];
        branch(c, nC, a, nE, b);
        pop_member(c);
    }
    free(nC);
    free(nE);
}

int oracle_enumerate(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                     uint32_t n_left, uint32_t k, uint64_t result_limit,
                     oracle_sink sink, void* user, oracle_stats* out) {
    return oracle_enumerate_shard(offsets, adj, n, n_left, k, result_limit, 0, 1, sink, user, out);
}

int oracle_enumerate_shard(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                           uint32_t n_left, uint32_t k, uint64_t result_limit,
                           uint32_t shard, uint32_t nshards,
                           oracle_sink sink, void* user, oracle_stats* out) {
    if (!offsets || !out || n > ORACLE_MAX_N || n_left > n || k < 1) return -1;
    if (nshards == 0 || shard >= nshards) return -1;
    memset(out, 0, sizeof(*out));
    ctx_t c;
    memset(&c, 0, sizeof(c));
    c.n = n; c.nl = n_left; c.k = k;
    c.words = (n + 63) / 64;
    c.adjbits = (uint64_t*)calloc((size_t)n * c.words + 1, sizeof(uint64_t));
    for (uint32_t v = 0; v < n; ++v)
        for (uint32_t p = offsets[v]; p < offsets[v + 1]; ++p) {
            uint32_t w = adj[p];
            if (w >= n) { free(c.adjbits); return -1; }
            c.adjbits[(size_t)v * c.words + (w >> 6)] |= 1ull << (w & 63);
        }
    c.limit = result_limit; c.sink = sink; c.user = user; c.st = out;
    c.S = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    c.mc = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    c.scratch = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    c.sc_bits[0] = (uint64_t*)calloc(c.words + 1, sizeof(uint64_t));
    c.sc_bits[1] = (uint64_t*)calloc(c.words + 1, sizeof(uint64_t));
    uint32_t* C = (uint32_t*)malloc((size_t)(n + 1) * sizeof(uint32_t));
    uint32_t* E = (uint32_t*)malloc((size_t)(n + 1) * sizeof(uint32_t));
    for (uint32_t x = 0; x < n_left && !c.stop; ++x) {
        if (x % nshards != shard) continue;
        uint32_t nc = 0, ne = 0;
        for (uint32_t v = n_left; v < n; ++v) C[nc++] = v;        /* V first */
        for (uint32_t u = x + 1; u < n_left; ++u) C[nc++] = u;    /* later U */
        for (uint32_t u = 0; u < x; ++u) E[ne++] = u;             /* earlier U */
        push_member(&c, x);
        branch(&c, C, nc, E, ne);
        pop_member(&c);
    }
    free(C); free(E);
    free(c.sc_bits[0]); free(c.sc_bits[1]);
    free(c.scratch); free(c.mc); free(c.S); free(c.adjbits);
    return 0;
}

int oracle_classify(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                    uint32_t n_left, uint32_t k, const uint32_t* x, uint32_t nx,
                    const uint32_t* y, uint32_t ny) {
    /* direct definition, sparse: used to validate individual printed sets */
    uint32_t* mark = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    uint32_t* miss = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
    int result = 2;
    for (uint32_t i = 0; i < nx; ++i) mark[x[i]] = 1;
    for (uint32_t i = 0; i < ny; ++i) mark[y[i]] = 1;
    /* misses of members */
    for (int s = 0; s < 2; ++s) {
        const uint32_t* A = s ? y : x; uint32_t na = s ? ny : nx;
        uint32_t nopp = s ? nx : ny;
        for (uint32_t i = 0; i < na; ++i) {
            uint32_t v = A[i], hit = 0;
            for (uint32_t p = offsets[v]; p < offsets[v + 1]; ++p) hit += mark[adj[p]];
            miss[v] = nopp - hit;
            if (miss[v] > k) result = 0;
        }
    }
    if (result == 0) { free(mark); free(miss); return 0; }
    /* can any outside vertex be added? */
    for (uint32_t w = 0; w < n && result == 2; ++w) {
        if (mark[w]) continue;
        int s = w >= n_left;
        const uint32_t* O = s ? x : y; uint32_t no = s ? nx : ny;
        uint32_t hit = 0, bad = 0;
        for (uint32_t p = offsets[w]; p < offsets[w + 1]; ++p) hit += mark[adj[p]];
        if (no - hit > k) continue;
        /* members on the other side that w misses must have room */
        for (uint32_t i = 0; i < no && !bad; ++i) {
            uint32_t m = O[i];
            int adjw = 0;
            for (uint32_t p = offsets[w]; p < offsets[w + 1]; ++p) if (adj[p] == m) { adjw = 1; break; }
            if (!adjw && miss[m] >= k) bad = 1;
        }
        if (!bad) result = 1;
    }
    free(mark); free(miss);
    return result;
}
