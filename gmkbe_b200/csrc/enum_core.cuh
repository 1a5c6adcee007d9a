// Maximal k-biplex enumeration: the per-task depth-first search.
//
// One search task = all maximal k-biplexes (X, Y) whose smallest U vertex is
// the task's root x (the reference's top-level loop over Cand_exts with the
// earlier vertices moved to Cand_q, src/main.cu:1078-1111 and :1489).  A task
// is a branch-and-bound over
//   S        the current k-biplex (members with their miss counts, the
//            reference's G_state counters, src/main.cu:472-535);
//   C_U, C_V the undecided vertices compatible with S on each side.
// Vertices outside S u C are the exclusion set (the reference's Cand_q /
// ext_q); it is never stored: every test on it is answered from the CSR.
//
// A side's candidate set is either GLOBAL -- every vertex of that side with a
// larger id, which is exactly the compatible set while the other side of S
// has at most k members and none of them has used up its k misses -- or a
// LOCAL explicit list of (id, misses-in-S) pairs.  Global sets cost nothing
// to hold; they turn local as soon as a member saturates or the other side
// reaches k+1 members, at which point candidates must be adjacent to the
// saturated member (or to one of k+1 members), so the list is gathered from
// those neighbourhoods only.
//
// Rules at a node whose two candidate sides are local (all proven in the
// design notes):
//   * shortcut: if S u C is itself a k-biplex it is the only possible maximal
//     leaf below (the reference's CheckMaximality_for_Gnerate direct case,
//     include/for_generate.cuh:432-477);
//   * forcing: a candidate that misses <= k of (S u C) on the other side, and
//     only members that miss <= k inside S u C, belongs to every maximal leaf
//     below and is taken without branching (the reference's "Component",
//     src/main.cu:1305-1339);
//   * exclusion prune: an outside vertex addable to every leaf below ends the
//     branch (the Cand_q test of src/main.cu:1290-1304, generalised);
//   * leaf check: a leaf is emitted iff no outside vertex can be added
//     (CheckMaximality, include/for_checkmaximality.cuh:3109-3303).
// Each root-to-leaf path fixes include/exclude decisions, so leaves are
// distinct and every maximal k-biplex is emitted exactly once.
//
// The code is plain per-thread C++ so that the host can run the same search;
// the CUDA kernel (enum_kernel.cu) runs one task per thread.
#pragma once
#include <stdint.h>

#ifndef GMK_HD
#ifdef __CUDACC__
#define GMK_HD __host__ __device__ __forceinline__
#else
#define GMK_HD inline
#endif
#endif

// Hook for host-side measurement tools (the arena's high-water mark); empty in
// the library.
#ifndef GMK_TRACE_TOP
#define GMK_TRACE_TOP(task, top) ((void)0)
#endif

#ifndef GMK_LOCAL_ORDER
#define GMK_LOCAL_ORDER(n0, n1) ((n1) < (n0) ? 1u : 0u)
#endif

namespace gmk {

// ----------------------------------------------------------------- hashing

GMK_HD uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
GMK_HD uint64_t elem_a(uint32_t v) { return mix64((uint64_t)v * 2u + 1u); }
GMK_HD uint64_t elem_b(uint64_t a) { return mix64(a ^ 0x5851F42D4C957F2Dull); }
GMK_HD uint64_t final_h1(uint64_t a, uint32_t nx, uint32_t ny) {
    return mix64(a + (uint64_t)nx * 0x100000001B3ull + (uint64_t)ny);
}
GMK_HD uint64_t final_h2(uint64_t b, uint32_t nx, uint32_t ny) {
    return mix64(b ^ (((uint64_t)nx << 32) | (uint64_t)ny));
}

// ----------------------------------------------------------------- graph

struct GraphView {
    const uint32_t* off;   // N+1
    const uint32_t* adj;   // 2|E|, rows sorted ascending
    uint32_t n, nl;
};

GMK_HD uint32_t degree(const GraphView& g, uint32_t v) { return g.off[v + 1] - g.off[v]; }
GMK_HD int side_of(const GraphView& g, uint32_t v) { return v >= g.nl; }
GMK_HD uint32_t side_begin(const GraphView& g, int s) { return s ? g.nl : 0u; }
GMK_HD uint32_t side_end(const GraphView& g, int s) { return s ? g.n : g.nl; }

// Binary search of b in row a; adds the words read to *words (4 offset words
// for the degree comparison in adjacent(), then one per probe).
GMK_HD bool row_contains(const GraphView& g, uint32_t a, uint32_t b, unsigned long long* words) {
    uint32_t lo = g.off[a], hi = g.off[a + 1];
    const uint32_t end = hi;
    uint32_t probes = 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (g.adj[mid] < b) lo = mid + 1; else hi = mid;
        ++probes;
    }
    *words += 4 + probes;
    return lo < end && g.adj[lo] == b;
}
// Searches the shorter row.
GMK_HD bool adjacent(const GraphView& g, uint32_t a, uint32_t b, unsigned long long* words) {
    return degree(g, a) <= degree(g, b) ? row_contains(g, a, b, words)
                                        : row_contains(g, b, a, words);
}

// ----------------------------------------------------------------- task state

// Frame words (a frame lives in the task's arena, followed by its lists).
enum : uint32_t {
    F_NS = 0,        // |S| when the frame was created
    F_FLAGS,         // bit0/1: side 0/1 global; bit2: entry done; bit3: no more children
    F_LO0, F_LO1,    // global side: candidates are ids > lo
    F_CNT0, F_CNT1,  // local side: entries
    F_OFF0, F_OFF1,  // local side: arena word offset of (id, misses) pairs
    F_ORDER,         // side iterated first
    F_PHASE,         // 0,1 = iterating order side / other side; 2 = finished
    F_POS,           // next position (local) or next id (global)
    F_TOP,           // arena words used up to the end of this frame's lists
    F_PARENT_SLOT,   // parent frame offset (kNoPos for the root)
    F_END,           // global side iterated first: stop before this id
    F_WORDS
};
enum : uint32_t { FL_G0 = 1u, FL_G1 = 2u, FL_ENTERED = 4u };

enum : int {
    TASK_OK = 0,
    TASK_E_ARENA = 1,   // task arena too small
    TASK_E_SMAX = 2,    // |S| above the member capacity
    TASK_E_TIMEOUT = 3, // watchdog deadline passed
    TASK_E_OUTBUF = 4,  // a result record found no room and could not be deferred
    TASK_E_RECORD = 5,  // a split or donated task record failed its checks (internal error)
};

struct Outputs {
    unsigned long long* count;      // results emitted (may pass the limit by a batch)
    unsigned long long* hash_sum;
    unsigned long long* hash_xor;
    unsigned long long* nodes;
    unsigned long long* work;       // adjacency words touched (algorithmic traffic)
    int* stop;                      // set once the limit is reached or on error
    int* error;                     // first error code
    unsigned long long limit;       // 0 = unlimited
    uint32_t* out_buf;              // optional result records: nx, ny, X..., Y...
    unsigned long long* out_pos;
    unsigned long long out_cap;     // words
    unsigned long long deadline_ns; // 0 = none; compared with the device's global timer
    unsigned long long* out_fail;   // warp engine: lowest record position that found no room
    int* gstop;                     // warp engine, batches: this graph's limit was reached
                                    //   (null: the limit raises `stop`)
};

struct Task {
    GraphView g;
    uint32_t k;
    uint32_t* arena;      // frames + lists
    uint32_t cap;         // arena words
    uint32_t* sid;        // S members
    uint32_t* smc;        // misses of each member inside S
    uint32_t smax;
    uint32_t ns, nss[2];
    uint32_t scan_limit;  // skip the pairwise node rules above this many candidate pairs
    int err;
    // batched counters, flushed to Outputs
    unsigned long long cnt, hsum, hxor, nodes, work;
};

// ----------------------------------------------------------------- members

// Misses of w against S on the other side; also checks every missed member
// still has room.  Returns misses, or k+1 if w is not compatible.
GMK_HD uint32_t compat_misses(Task& t, uint32_t w) {
    const int s = side_of(t.g, w);
    uint32_t miss = 0;
    if (t.nss[1 - s] == 0) return 0;
    for (uint32_t i = 0; i < t.ns; ++i) {
        uint32_t m = t.sid[i];
        if (side_of(t.g, m) == s) continue;
        if (adjacent(t.g, w, m, &t.work)) continue;
        if (++miss > t.k || t.smc[i] >= t.k) return t.k + 1;
    }
    return miss;
}

// Add c to S; returns its misses.  `sat` receives the other-side members
// that reached k misses because of c (at most `satcap`), *nsat their count.
GMK_HD uint32_t push_member(Task& t, uint32_t c, uint32_t* sat, uint32_t satcap, uint32_t* nsat) {
    const int s = side_of(t.g, c);
    uint32_t miss = 0, ns_ = 0;
    for (uint32_t i = 0; i < t.ns; ++i) {
        uint32_t m = t.sid[i];
        if (side_of(t.g, m) == s) continue;
        if (adjacent(t.g, c, m, &t.work)) continue;
        ++miss;
        if (++t.smc[i] == t.k && ns_ < satcap) sat[ns_++] = m;
    }
    t.sid[t.ns] = c;
    t.smc[t.ns] = miss;
    t.ns++;
    t.nss[s]++;
    if (nsat) *nsat = ns_;
    return miss;
}

GMK_HD void pop_member(Task& t) {
    const uint32_t c = t.sid[--t.ns];
    const int s = side_of(t.g, c);
    t.nss[s]--;
    for (uint32_t i = 0; i < t.ns; ++i) {
        uint32_t m = t.sid[i];
        if (side_of(t.g, m) == s) continue;
        if (!adjacent(t.g, c, m, &t.work)) --t.smc[i];
    }
}

GMK_HD void pop_to(Task& t, uint32_t ns) {
    while (t.ns > ns) pop_member(t);
}

// ----------------------------------------------------------------- leaf / prune test

// Is some vertex outside L = S u C (C given by two local lists) addable to
// every leaf below?  tot[] holds, for S members then list-0 entries then
// list-1 entries, the misses inside L.  With `strict`, members with tot == k
// block (they would gain a miss); this is exactly addability to L when C is
// empty, and the exclusion prune otherwise.
GMK_HD bool outsider_addable(Task& t, const uint32_t* l0, uint32_t n0, const uint32_t* l1,
                             uint32_t n1, const uint32_t* tot) {
    const GraphView& g = t.g;
    const uint32_t* lst[2] = {l0, l1};
    const uint32_t cnt[2] = {n0, n1};
    const uint32_t* tots[2] = {tot + t.ns, tot + t.ns + n0};
    for (int s = 0; s < 2; ++s) {
        const int o = 1 - s;
        const uint32_t nopp = t.nss[o] + cnt[o];
        const uint32_t nown = t.nss[s] + cnt[s];
        // pick where candidate outsiders can come from
        uint32_t hard = 0xFFFFFFFFu, hard_deg = 0xFFFFFFFFu;
        for (uint32_t i = 0; i < t.ns; ++i)
            if (side_of(g, t.sid[i]) == o && tot[i] >= t.k && degree(g, t.sid[i]) < hard_deg) {
                hard = t.sid[i]; hard_deg = degree(g, hard);
            }
        for (uint32_t i = 0; i < cnt[o]; ++i)
            if (tots[o][i] >= t.k && degree(g, lst[o][2 * i]) < hard_deg) {
                hard = lst[o][2 * i]; hard_deg = degree(g, hard);
            }
        uint32_t src[4];
        uint32_t nsrc = 0;
        if (hard != 0xFFFFFFFFu) {
            src[nsrc++] = hard;
        } else if (nopp >= t.k + 1) {
            // any k+1 members: an addable outsider misses at most k of them
            for (uint32_t i = 0; i < t.ns && nsrc < t.k + 1; ++i)
                if (side_of(g, t.sid[i]) == o) src[nsrc++] = t.sid[i];
            for (uint32_t i = 0; i < cnt[o] && nsrc < t.k + 1; ++i) src[nsrc++] = lst[o][2 * i];
        } else {
            // at most k members on the other side, none blocking: every
            // outsider of side s fits
            if (side_end(g, s) - side_begin(g, s) > nown) return true;
            continue;
        }
        for (uint32_t q = 0; q < nsrc; ++q) {
            const uint32_t m = src[q];
            t.work += degree(g, m);
            for (uint32_t p = g.off[m]; p < g.off[m + 1]; ++p) {
                const uint32_t e = g.adj[p];
                // visit e once: at the first source it is adjacent to
                bool seen = false;
                for (uint32_t r = 0; r < q && !seen; ++r) seen = adjacent(g, e, src[r], &t.work);
                if (seen) continue;
                bool inside = false;
                for (uint32_t i = 0; i < t.ns && !inside; ++i) inside = t.sid[i] == e;
                for (uint32_t i = 0; i < cnt[s] && !inside; ++i) inside = lst[s][2 * i] == e;
                if (inside) continue;
                uint32_t miss = 0;
                bool ok = true;
                for (uint32_t i = 0; i < t.ns && ok; ++i) {
                    const uint32_t w = t.sid[i];
                    if (side_of(g, w) != o || adjacent(g, e, w, &t.work)) continue;
                    if (++miss > t.k || tot[i] >= t.k) ok = false;
                }
                for (uint32_t i = 0; i < cnt[o] && ok; ++i) {
                    const uint32_t w = lst[o][2 * i];
                    if (adjacent(g, e, w, &t.work)) continue;
                    if (++miss > t.k || tots[o][i] >= t.k) ok = false;
                }
                if (ok) return true;
            }
        }
    }
    return false;
}

// Neighbours of w with id > lo.
GMK_HD uint32_t count_above(const GraphView& g, uint32_t w, uint32_t lo,
                            unsigned long long* words) {
    uint32_t a = g.off[w], b = g.off[w + 1];
    const uint32_t end = b;
    uint32_t probes = 2;
    while (a < b) {
        uint32_t mid = (a + b) >> 1;
        if (g.adj[mid] <= lo) a = mid + 1; else b = mid;
        ++probes;
    }
    *words += probes;
    return end - a;
}

// Exclusion prune at a node whose side s is global (candidates: ids > lo)
// and side o = 1-s local (list l, n entries): is some outsider of side s
// (id <= lo, not in S) addable to every leaf below?  Members w of (S u C)_o
// block when their misses inside S_s u C_s reach k; those misses count the
// whole global range above lo.  `tot` is scratch for nss[o] + n words.
GMK_HD bool outsider_addable_mixed(Task& t, int s, uint32_t lo, const uint32_t* l, uint32_t n,
                                   uint32_t* tot) {
    const GraphView& g = t.g;
    const int o = 1 - s;
    const uint32_t G = side_end(g, s) - lo - 1;
    uint32_t* mem = tot + n;          // S_o member ids after the list totals
    uint32_t nm = 0;
    uint32_t hard = 0xFFFFFFFFu, hard_deg = 0xFFFFFFFFu;
    for (uint32_t i = 0; i < t.ns; ++i) {
        const uint32_t w = t.sid[i];
        if (side_of(g, w) != o) continue;
        const uint32_t tw = t.smc[i] + G - count_above(g, w, lo, &t.work);
        mem[nm++] = w;
        if (tw >= t.k && degree(g, w) < hard_deg) { hard = w; hard_deg = degree(g, w); }
    }
    for (uint32_t q = 0; q < n; ++q) {
        const uint32_t w = l[2 * q];
        tot[q] = l[2 * q + 1] + G - count_above(g, w, lo, &t.work);
        if (tot[q] >= t.k && degree(g, w) < hard_deg) { hard = w; hard_deg = degree(g, w); }
    }
    const uint32_t nopp = nm + n;
    uint32_t src[17];
    uint32_t nsrc = 0;
    if (hard != 0xFFFFFFFFu) {
        src[nsrc++] = hard;
    } else if (nopp >= t.k + 1) {
        for (uint32_t i = 0; i < nm && nsrc < t.k + 1; ++i) src[nsrc++] = mem[i];
        for (uint32_t q = 0; q < n && nsrc < t.k + 1; ++q) src[nsrc++] = l[2 * q];
    } else {
        return (lo + 1 - side_begin(g, s)) > t.nss[s];
    }
    for (uint32_t q = 0; q < nsrc; ++q) {
        const uint32_t m = src[q];
        t.work += degree(g, m);
        for (uint32_t p = g.off[m]; p < g.off[m + 1]; ++p) {
            const uint32_t e = g.adj[p];
            if (e > lo) break;                       // rows are sorted: the rest is in C
            bool seen = false;
            for (uint32_t r = 0; r < q && !seen; ++r) seen = adjacent(g, e, src[r], &t.work);
            if (seen) continue;
            bool inside = false;
            for (uint32_t i = 0; i < t.ns && !inside; ++i) inside = t.sid[i] == e;
            if (inside) continue;
            uint32_t miss = 0;
            bool ok = true;
            for (uint32_t i = 0; i < t.ns && ok; ++i) {
                const uint32_t w = t.sid[i];
                if (side_of(g, w) != o || adjacent(g, e, w, &t.work)) continue;
                if (++miss > t.k || t.smc[i] + G - count_above(g, w, lo, &t.work) >= t.k) ok = false;
            }
            for (uint32_t r = 0; r < n && ok; ++r) {
                if (adjacent(g, e, l[2 * r], &t.work)) continue;
                if (++miss > t.k || tot[r] >= t.k) ok = false;
            }
            if (ok) return true;
        }
    }
    return false;
}

// ----------------------------------------------------------------- counters

#if defined(__CUDA_ARCH__)
GMK_HD unsigned long long atomic_add_u64(unsigned long long* p, unsigned long long v) {
    return atomicAdd(p, v);
}
GMK_HD void atomic_xor_u64(unsigned long long* p, unsigned long long v) { atomicXor(p, v); }
GMK_HD int load_flag(const int* p) { return *(volatile const int*)p; }
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
GMK_HD void store_flag(int* p, int v) { atomicExch(p, v); }
GMK_HD void first_error(int* p, int v) { atomicCAS(p, 0, v); }
#else
GMK_HD unsigned long long atomic_add_u64(unsigned long long* p, unsigned long long v) {
    return __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
GMK_HD void atomic_xor_u64(unsigned long long* p, unsigned long long v) {
    __atomic_fetch_xor(p, v, __ATOMIC_RELAXED);
}
GMK_HD int load_flag(const int* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
GMK_HD unsigned long long now_ns() { return 0; }
GMK_HD void store_flag(int* p, int v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
GMK_HD void first_error(int* p, int v) {
    int z = 0;
    __atomic_compare_exchange_n(p, &z, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
}
#endif

// Results are counted per task in batches; the global count may pass the
// limit by less than one batch per running task, and readers clamp it.
static constexpr unsigned long long kFlushBatch = 64;

GMK_HD void flush(Task& t, const Outputs& o) {
    if (t.cnt) {
        unsigned long long before = atomic_add_u64(o.count, t.cnt);
        atomic_add_u64(o.hash_sum, t.hsum);
        atomic_xor_u64(o.hash_xor, t.hxor);
        if (o.limit && before + t.cnt >= o.limit) store_flag(o.stop, 1);
    }
    if (t.nodes) atomic_add_u64(o.nodes, t.nodes);
    if (t.work) atomic_add_u64(o.work, t.work);
    t.cnt = t.hsum = t.hxor = t.nodes = t.work = 0;
}

GMK_HD void fail(Task& t, const Outputs& o, int code) {
    if (!t.err) t.err = code;
    first_error(o.error, code);
    store_flag(o.stop, 1);
}

// Emit L = S u list0 u list1 (lists hold (id, misses) pairs).
GMK_HD void emit(Task& t, const Outputs& o, const uint32_t* l0, uint32_t n0, const uint32_t* l1,
                 uint32_t n1) {
    uint64_t a = 0, b = 0;
    for (uint32_t i = 0; i < t.ns; ++i) {
        uint64_t e = elem_a(t.sid[i]);
        a += e; b += elem_b(e);
    }
    for (uint32_t i = 0; i < n0; ++i) { uint64_t e = elem_a(l0[2 * i]); a += e; b += elem_b(e); }
    for (uint32_t i = 0; i < n1; ++i) { uint64_t e = elem_a(l1[2 * i]); a += e; b += elem_b(e); }
    const uint32_t nx = t.nss[0] + n0, ny = t.nss[1] + n1;
    if (o.out_buf) {
        // record mode: one reservation per result, exact limit
        const unsigned long long words = 2ull + nx + ny;
        unsigned long long c = atomic_add_u64(o.count, 1ull);
        if (o.limit && c >= o.limit) { store_flag(o.stop, 1); return; }
        if (o.limit && c + 1 >= o.limit) store_flag(o.stop, 1);
        atomic_add_u64(o.hash_sum, final_h1(a, nx, ny));
        atomic_xor_u64(o.hash_xor, final_h2(b, nx, ny));
        unsigned long long at = atomic_add_u64(o.out_pos, words);
        if (at + words > o.out_cap) return;   // host sees out_pos > cap and reports overflow
        uint32_t* r = o.out_buf + at;
        r[0] = nx; r[1] = ny;
        uint32_t px = 2, py = 2 + nx;
        for (uint32_t i = 0; i < t.ns; ++i) {
            uint32_t v = t.sid[i];
            if (side_of(t.g, v)) r[py++] = v; else r[px++] = v;
        }
        for (uint32_t i = 0; i < n0; ++i) r[px++] = l0[2 * i];
        for (uint32_t i = 0; i < n1; ++i) r[py++] = l1[2 * i];
        return;
    }
    t.cnt++;
    t.hsum += final_h1(a, nx, ny);
    t.hxor ^= final_h2(b, nx, ny);
    if (t.cnt >= kFlushBatch) flush(t, o);
}

// ----------------------------------------------------------------- frames

GMK_HD bool is_global(const uint32_t* f, int s) { return f[F_FLAGS] & (s ? FL_G1 : FL_G0); }

// A global side whose id range is used up becomes an empty local side.
GMK_HD void normalise(const GraphView& g, uint32_t* f) {
    for (int s = 0; s < 2; ++s)
        if (is_global(f, s) && f[F_LO0 + s] + 1 >= side_end(g, s)) {
            f[F_FLAGS] &= ~(s ? FL_G1 : FL_G0);
            f[F_CNT0 + s] = 0;
        }
}

enum : int { ENTER_ITERATE = 0, ENTER_DONE = 1, ENTER_PUSHED = 2 };
static constexpr uint32_t kNoPos = 0xFFFFFFFFu;
static constexpr uint32_t kSatCap = 16;   // k <= 16

// Build the child "S + c" of frame `cur` at the arena top.  c is on side s,
// at local position p (kNoPos for a global side).  `forced`: every other
// candidate stays (no sibling exclusion).  `opp_done`: the other side was
// iterated before this one, so it has no candidates left.
// Returns the child's frame offset or kNoPos on arena overflow (task failed).
GMK_HD uint32_t build_child(Task& t, const Outputs& o, uint32_t cur, uint32_t c, int s, uint32_t p,
                            bool forced, bool opp_done) {
    const GraphView& g = t.g;
    uint32_t* f = t.arena + cur;
    pop_to(t, f[F_NS]);
    if (t.ns + 1 > t.smax) { fail(t, o, TASK_E_SMAX); return kNoPos; }
    uint32_t sat[kSatCap];
    uint32_t nsat = 0;
    const uint32_t mcc = push_member(t, c, sat, kSatCap, &nsat);
    const int os = 1 - s;

    const uint32_t nc = f[F_TOP];
    uint32_t* ch = t.arena + nc;
    uint32_t w = nc + F_WORDS;
    if (w > t.cap) { fail(t, o, TASK_E_ARENA); return kNoPos; }
    ch[F_NS] = t.ns;
    ch[F_FLAGS] = 0;
    ch[F_ORDER] = 0; ch[F_PHASE] = 0; ch[F_POS] = 0;
    ch[F_PARENT_SLOT] = cur;
    ch[F_END] = 0xFFFFFFFFu;

    // ---- same side as c
    ch[F_OFF0 + s] = w;
    uint32_t cnt = 0;
    bool shared = false;
    if (is_global(f, s)) {
        if (nsat == 0) {
            ch[F_FLAGS] |= s ? FL_G1 : FL_G0;
            ch[F_LO0 + s] = c;
        } else {
            uint32_t z = sat[0];
            for (uint32_t i = 1; i < nsat; ++i) if (degree(g, sat[i]) < degree(g, z)) z = sat[i];
            if (w + 2 * degree(g, z) > t.cap) { fail(t, o, TASK_E_ARENA); return kNoPos; }
            t.work += degree(g, z);
            for (uint32_t q = g.off[z]; q < g.off[z + 1]; ++q) {
                const uint32_t v = g.adj[q];
                if (v <= c) continue;
                const uint32_t m = compat_misses(t, v);
                if (m > t.k) continue;
                t.arena[w + 2 * cnt] = v; t.arena[w + 2 * cnt + 1] = m; ++cnt;
            }
        }
    } else if (!forced && nsat == 0) {
        // nothing to filter: the rest of the parent's list, read in place
        // (nothing is stored after the frame for this side)
        const uint32_t n = f[F_CNT0 + s];
        ch[F_OFF0 + s] = f[F_OFF0 + s] + 2 * (p + 1);
        shared = true;
        cnt = n > p + 1 ? n - p - 1 : 0u;
    } else {
        const uint32_t* lst = t.arena + f[F_OFF0 + s];
        const uint32_t n = f[F_CNT0 + s];
        if (w + 2 * n > t.cap) { fail(t, o, TASK_E_ARENA); return kNoPos; }
        for (uint32_t q = forced ? 0 : p + 1; q < n; ++q) {
            if (q == p) continue;
            const uint32_t v = lst[2 * q];
            bool ok = true;
            for (uint32_t i = 0; i < nsat && ok; ++i) ok = adjacent(g, v, sat[i], &t.work);
            if (!ok) continue;
            t.arena[w + 2 * cnt] = v; t.arena[w + 2 * cnt + 1] = lst[2 * q + 1]; ++cnt;
        }
    }
    ch[F_CNT0 + s] = cnt;
    if (!shared) w += 2 * cnt;

    // ---- other side
    ch[F_OFF0 + os] = w;
    cnt = 0;
    if (opp_done) {
        // nothing left on that side
    } else if (is_global(f, os)) {
        const uint32_t lo = f[F_LO0 + os];
        if (t.nss[s] <= t.k && mcc < t.k) {
            ch[F_FLAGS] |= os ? FL_G1 : FL_G0;
            ch[F_LO0 + os] = lo;
        } else {
            // candidates must touch c (saturated) or one of the k+1 members of side s
            uint32_t src[kSatCap + 1];
            uint32_t nsrc = 0;
            if (mcc >= t.k) {
                src[nsrc++] = c;
            } else {
                for (uint32_t i = 0; i < t.ns && nsrc < t.k + 1; ++i)
                    if (side_of(g, t.sid[i]) == s) src[nsrc++] = t.sid[i];
            }
            uint64_t bound = 0;
            for (uint32_t q = 0; q < nsrc; ++q) bound += degree(g, src[q]);
            if (w + 2 * bound > t.cap) { fail(t, o, TASK_E_ARENA); return kNoPos; }
            for (uint32_t q = 0; q < nsrc; ++q) {
                const uint32_t m = src[q];
                t.work += degree(g, m);
                for (uint32_t e = g.off[m]; e < g.off[m + 1]; ++e) {
                    const uint32_t v = g.adj[e];
                    if (v <= lo) continue;
                    bool seen = false;
                    for (uint32_t r = 0; r < q && !seen; ++r) seen = adjacent(g, v, src[r], &t.work);
                    if (seen) continue;
                    const uint32_t mm = compat_misses(t, v);
                    if (mm > t.k) continue;
                    t.arena[w + 2 * cnt] = v; t.arena[w + 2 * cnt + 1] = mm; ++cnt;
                }
            }
        }
    } else {
        const uint32_t* lst = t.arena + f[F_OFF0 + os];
        const uint32_t n = f[F_CNT0 + os];
        if (w + 2 * n > t.cap) { fail(t, o, TASK_E_ARENA); return kNoPos; }
        for (uint32_t q = 0; q < n; ++q) {
            const uint32_t v = lst[2 * q];
            const uint32_t cm = lst[2 * q + 1];
                const bool a = adjacent(g, v, c, &t.work);
            if (!a && (cm + 1 > t.k || mcc >= t.k)) continue;
            t.arena[w + 2 * cnt] = v; t.arena[w + 2 * cnt + 1] = cm + (a ? 0u : 1u); ++cnt;
        }
    }
    ch[F_CNT0 + os] = cnt;
    w += 2 * cnt;
    ch[F_TOP] = w;
    GMK_TRACE_TOP(t, w);
    normalise(g, ch);
    return nc;
}

// Node rules; see the file comment.  May push a forced child (then *next
// is its offset).
GMK_HD int enter_node(Task& t, const Outputs& o, uint32_t cur, uint32_t* next) {
    const GraphView& g = t.g;
    uint32_t* f = t.arena + cur;
    pop_to(t, f[F_NS]);
    const bool g0 = is_global(f, 0), g1 = is_global(f, 1);
    // Y must end up non-empty
    if (t.nss[1] == 0 && !g1 && f[F_CNT1] == 0) return ENTER_DONE;
    // X is never empty (the root is in S)
    if (g0 != g1) {
        const int s = g0 ? 0 : 1, os = 1 - s;
        const uint32_t n = f[F_CNT0 + os];
        const uint32_t base = f[F_TOP];
        if (base + n + t.ns > t.cap) { fail(t, o, TASK_E_ARENA); return ENTER_DONE; }
        if (outsider_addable_mixed(t, s, f[F_LO0 + s], t.arena + f[F_OFF0 + os], n,
                                   t.arena + base))
            return ENTER_DONE;
    }
    if (!g0 && !g1) {
        const uint32_t n0 = f[F_CNT0], n1 = f[F_CNT1];
        const uint32_t* l0 = t.arena + f[F_OFF0];
        const uint32_t* l1 = t.arena + f[F_OFF1];
        const uint64_t pairs = (uint64_t)(t.ns + n0) * (uint64_t)(t.ns + n1);
        if (n0 + n1 == 0 || pairs <= t.scan_limit) {
            const uint32_t base = f[F_TOP];
            if (base + t.ns + n0 + n1 > t.cap) { fail(t, o, TASK_E_ARENA); return ENTER_DONE; }
            uint32_t* tot = t.arena + base;
            uint32_t* tot0 = tot + t.ns;
            uint32_t* tot1 = tot0 + n0;
            // misses inside S u C
            for (uint32_t i = 0; i < t.ns; ++i) {
                const uint32_t v = t.sid[i];
                const int sv = side_of(g, v);
                const uint32_t* lo = sv ? l0 : l1;
                const uint32_t no = sv ? n0 : n1;
                uint32_t m = t.smc[i];
                for (uint32_t q = 0; q < no; ++q) m += adjacent(g, v, lo[2 * q], &t.work) ? 0u : 1u;
                tot[i] = m;
            }
            for (uint32_t q = 0; q < n0; ++q) tot0[q] = l0[2 * q + 1];
            for (uint32_t q = 0; q < n1; ++q) tot1[q] = l1[2 * q + 1];
            for (uint32_t a = 0; a < n0; ++a)
                for (uint32_t b = 0; b < n1; ++b)
                    if (!adjacent(g, l0[2 * a], l1[2 * b], &t.work)) { ++tot0[a]; ++tot1[b]; }
            bool biplex = true;
            for (uint32_t i = 0; i < t.ns + n0 + n1 && biplex; ++i) biplex = tot[i] <= t.k;
            if (biplex) {
                // S u C is a k-biplex: the only leaf that can be maximal
                if (!outsider_addable(t, l0, n0, l1, n1, tot)) emit(t, o, l0, n0, l1, n1);
                return ENTER_DONE;
            }
            if (outsider_addable(t, l0, n0, l1, n1, tot)) return ENTER_DONE;
            // forced candidate: fits every leaf that lacks it
            for (int s = 0; s < 2; ++s) {
                const uint32_t* ls = s ? l1 : l0;
                const uint32_t* ts = s ? tot1 : tot0;
                const uint32_t ns_ = s ? n1 : n0;
                const uint32_t* lo = s ? l0 : l1;
                const uint32_t* to = s ? tot0 : tot1;
                const uint32_t no = s ? n0 : n1;
                for (uint32_t q = 0; q < ns_; ++q) {
                    if (ts[q] > t.k) continue;
                    const uint32_t c = ls[2 * q];
                    bool ok = true;
                    for (uint32_t i = 0; i < t.ns && ok; ++i) {
                        const uint32_t v = t.sid[i];
                        if (side_of(g, v) == s || adjacent(g, c, v, &t.work)) continue;
                        ok = tot[i] <= t.k;
                    }
                    for (uint32_t r = 0; r < no && ok; ++r)
                        if (!adjacent(g, c, lo[2 * r], &t.work)) ok = to[r] <= t.k;
                    if (!ok) continue;
                    const uint32_t ch = build_child(t, o, cur, c, s, q, true, false);
                    if (ch == kNoPos) return ENTER_DONE;
                    *next = ch;
                    return ENTER_PUSHED;
                }
            }
        }
    }
    // iterate: local sides before global ones; between two local sides the shorter first
    uint32_t order;
    if (cur == 0) order = 1u;   // the root branches on V first; root chunks rely on it
    else if (g0 != g1) order = g0 ? 1u : 0u;
    else if (!g0) order = GMK_LOCAL_ORDER(f[F_CNT0], f[F_CNT1]);
    else order = 1u;
    f[F_ORDER] = order;
    f[F_PHASE] = 0;
    f[F_POS] = is_global(f, (int)order) ? f[F_LO0 + order] + 1 : 0;
    return ENTER_ITERATE;
}

// Next child of frame `cur`; kNoPos when the frame is finished.
GMK_HD uint32_t next_child(Task& t, const Outputs& o, uint32_t cur) {
    const GraphView& g = t.g;
    uint32_t* f = t.arena + cur;
    while (f[F_PHASE] < 2) {
        const int s = f[F_PHASE] == 0 ? (int)f[F_ORDER] : 1 - (int)f[F_ORDER];
        const bool opp_done = f[F_PHASE] == 1;
        uint32_t c, p;
        bool have = false;
        if (is_global(f, s)) {
            const uint32_t end = f[F_PHASE] == 0 && f[F_END] < side_end(g, s) ? f[F_END]
                                                                             : side_end(g, s);
            if (f[F_POS] < end) { c = f[F_POS]; p = kNoPos; f[F_POS]++; have = true; }
        } else if (f[F_POS] < f[F_CNT0 + s]) {
            p = f[F_POS]; c = t.arena[f[F_OFF0 + s] + 2 * p]; f[F_POS]++; have = true;
        }
        // U children after the V side is exhausted need a V member in S
        if (have && opp_done && s == 0) {
            uint32_t nv = 0;
            for (uint32_t i = 0; i < f[F_NS]; ++i) nv += side_of(g, t.sid[i]);
            if (nv == 0) have = false, f[F_PHASE] = 2;
        }
        if (!have) {
            if (f[F_PHASE] == 2) break;
            f[F_PHASE]++;
            if (f[F_PHASE] == 1) {
                const int s2 = 1 - (int)f[F_ORDER];
                f[F_POS] = is_global(f, s2) ? f[F_LO0 + s2] + 1 : 0;
            }
            continue;
        }
        return build_child(t, o, cur, c, s, p, false, opp_done);
    }
    return kNoPos;
}

// Run one task to completion, or until stop is raised: root x in U, and of
// its children (S = {x, y}, the V side is branched first) those with
// y in [first, last).  Together the chunks of a root cover its search tree.
GMK_HD void run_task(Task& t, const Outputs& o, uint32_t root, uint32_t first, uint32_t last) {
    const GraphView& g = t.g;
    t.ns = 0; t.nss[0] = t.nss[1] = 0;
    push_member(t, root, nullptr, 0, nullptr);
    uint32_t* f = t.arena;
    f[F_NS] = 1;
    f[F_FLAGS] = FL_G0 | FL_G1;
    f[F_LO0] = root;
    f[F_LO1] = g.nl - 1;
    f[F_CNT0] = f[F_CNT1] = 0;
    f[F_OFF0] = f[F_OFF1] = F_WORDS;
    f[F_TOP] = F_WORDS;
    f[F_PARENT_SLOT] = kNoPos;
    f[F_END] = last;
    normalise(g, f);
    uint32_t cur = 0;
    uint32_t polls = 0;
    while (cur != kNoPos) {
        if (t.err) break;
        if ((++polls & 255u) == 0) {
            if (load_flag(o.stop)) break;
            if (o.deadline_ns && now_ns() > o.deadline_ns) { fail(t, o, TASK_E_TIMEOUT); break; }
        }
        f = t.arena + cur;
        if (!(f[F_FLAGS] & FL_ENTERED)) {
            f[F_FLAGS] |= FL_ENTERED;
            t.nodes++;
            uint32_t nxt = kNoPos;
            const int r = enter_node(t, o, cur, &nxt);
            if (r == ENTER_PUSHED) { f[F_PHASE] = 2; cur = nxt; continue; }
            if (r == ENTER_DONE) { f[F_PHASE] = 2; cur = f[F_PARENT_SLOT]; continue; }
            if (cur == 0 && f[F_ORDER] == 1u && is_global(f, 1))
                f[F_POS] = first > f[F_POS] ? first : f[F_POS];
        }
        const uint32_t ch = next_child(t, o, cur);
        if (ch == kNoPos) { cur = f[F_PARENT_SLOT]; continue; }
        cur = ch;
    }
    pop_to(t, 0);
}

}  // namespace gmk
