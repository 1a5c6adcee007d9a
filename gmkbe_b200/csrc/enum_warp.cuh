// Warp-cooperative maximal k-biplex search (sm_100a device code).
//
// One warp runs one search task at a time.  The search is the one in
// enum_core.cuh -- same frames, same node rules (shortcut, forcing, exclusion
// prune, leaf test), same child order -- so the emitted set is identical; what
// changes is how a node's work is spread over the 32 lanes:
//   * every loop over a long dimension (a candidate list, a CSR row, the
//     members of S) runs one element per lane, with ballot-based compaction
//     so that child lists keep the parent's order and are written coalesced;
//   * the short dimension (the members an element is tested against) runs
//     sequentially per lane, all lanes in lockstep, so those reads broadcast;
//     where there are only a few rows (the usual node: a handful of members
//     and candidates), each row is spread over a group of lanes instead
//     (make_groups), so the idle lanes share its probes;
//   * adjacency is one probe of a device edge hash table (one 32-byte bucket
//     almost always) instead of a binary search over a CSR row -- the
//     reference's membership test is binarySearch over sorted rows,
//     include/gpu_utils.cuh:258-282;
//   * the search state (frames, lists, S) lives in a per-warp arena, so the
//     hot part of 4-10k warps' state stays in L2 instead of 150k threads'.
// Work that outgrows its warp is split: when the task queue of a round is
// empty, a busy warp writes every frame that still has unexplored children
// (plus its current node) as separate tasks for the next round.  Together
// they cover exactly the unexplored part of its search tree.
//
// Every search loop carries `#pragma unroll 1`.  The kernel is bound by
// instruction fetch (the whole search is one kernel, and each warp is at its
// own point of it): unrolled, the loops and the hash probes inlined into each
// copy made the count-only kernel 271 KB of machine code; rolled it is 176 KB
// and 1.07-1.31x faster, the shorter trip counts notwithstanding.  Code size
// is not the whole story, though: one run_dfs call site for root tasks and
// records is 1.1-1.5x faster than two inlined copies in the k = 1 kernels,
// and 1.1x slower in the k >= 2 ones, which keep two.
#pragma once
#include "enum_core.cuh"

namespace gmk {
namespace warp {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kSrcCap = 17;          // k + 1 sources, k <= 16
constexpr uint32_t FL_ROOT = 16u;         // frame flag: the task's root frame
constexpr uint32_t FL_BITS0 = 32u;        // frame flags: filter bitmaps of list 0 / list 1
constexpr uint32_t FL_BITS1 = 64u;        //   follow the frame's lists (add_filter_bits)
constexpr uint32_t FL_ONE_PHASE = 128u;   // frame flag: iterate the current phase only (a
                                          //   donated range of its first side's children)
constexpr uint32_t FL_SHARED0 = 256u;     // frame flags: list 0 / list 1 is a suffix of the
constexpr uint32_t FL_SHARED1 = 512u;     //   parent's list, read in place (not stored after
                                          //   the frame)
constexpr uint32_t kBitsMinList = 64;     // default: shorter lists filter their children by
                                          //   probing (gmk_opts.bits_min_list)
constexpr uint32_t kBitsMaxZ = 8;         // bitmaps for at most this many members
constexpr unsigned long long kEmptyKey = ~0ull;

// Open-addressing set of edges, keys (u << 32 | v) with u in U, v in V, in
// buckets of four 8-byte keys (one 32-byte sector).  Keys fill a bucket left
// to right and spill to the next bucket, so an empty slot ends a search.
struct EdgeHash {
    const unsigned long long* slots;
    unsigned long long bmask;   // buckets - 1 (a power of two)
};

__device__ __forceinline__ unsigned long long edge_key(uint32_t a, uint32_t b) {
    return a < b ? ((unsigned long long)a << 32) | b : ((unsigned long long)b << 32) | a;
}

// Bucket of a key: a 32-bit multiply-xorshift mix of its two ids (the
// multiplicative constants of the 32-bit golden-ratio / murmur3 finaliser
// family), cheaper on the GPU than a 64-bit mix; buckets <= 2^32.
__device__ __forceinline__ unsigned long long bucket_of(unsigned long long key,
                                                        unsigned long long bmask) {
    uint32_t h = (uint32_t)(key >> 32) * 0x9E3779B1u ^ (uint32_t)key * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 13;
    return (unsigned long long)h & bmask;
}

__device__ __noinline__ bool has_edge_tail(const EdgeHash& h, unsigned long long key,
                                           unsigned long long bk) {
    #pragma unroll 1
    for (unsigned long long it = 0; it < h.bmask; ++it) {
        bk = (bk + 1) & h.bmask;
        const ulonglong2* p = reinterpret_cast<const ulonglong2*>(h.slots + bk * 4);
        const ulonglong2 x = __ldg(p), y = __ldg(p + 1);
        if (x.x == key || x.y == key || y.x == key || y.y == key) return true;
        if (x.x == kEmptyKey || x.y == kEmptyKey || y.x == kEmptyKey || y.y == kEmptyKey)
            return false;
    }
    return false;
}

__device__ __forceinline__ bool has_edge(const EdgeHash& h, uint32_t a, uint32_t b) {
    const unsigned long long key = edge_key(a, b);
    const unsigned long long bk = bucket_of(key, h.bmask);
    const ulonglong2* p = reinterpret_cast<const ulonglong2*>(h.slots + bk * 4);
    const ulonglong2 x = __ldg(p), y = __ldg(p + 1);
    if (x.x == key || x.y == key || y.x == key || y.y == key) return true;
    if (x.x == kEmptyKey || x.y == kEmptyKey || y.x == kEmptyKey || y.y == kEmptyKey) return false;
    return has_edge_tail(h, key, bk);
}

// Inserts every edge of the CSR (one thread per U-row entry).
__global__ void build_edge_hash(const uint32_t* off, const uint32_t* adj, uint32_t nl,
                                unsigned long long* slots, unsigned long long bmask) {
    const unsigned long long e = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t m = off[nl];
    if (e >= m) return;
    // row u holding entry e: the last u with off[u] <= e
    uint32_t lo = 0, hi = nl;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= e) lo = mid; else hi = mid;
    }
    const unsigned long long key = edge_key(lo, adj[e]);
    unsigned long long bk = bucket_of(key, bmask);
    #pragma unroll 1
    for (unsigned long long it = 0; it <= bmask; ++it) {
        for (int j = 0; j < 4; ++j) {
            const unsigned long long prev = atomicCAS(slots + bk * 4 + j, kEmptyKey, key);
            if (prev == kEmptyKey || prev == key) return;
        }
        bk = (bk + 1) & bmask;
    }
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
// Warp reductions of 64-bit values with the 32-bit redux unit (one
// instruction per 32-bit reduction instead of five shuffle rounds).
// Minimum: the high words first, then the low words of the lanes holding the
// minimal high word -- the lexicographic, i.e. numeric, minimum.
__device__ __forceinline__ unsigned long long warp_min64(unsigned long long v) {
    const uint32_t hi = __reduce_min_sync(kFull, (uint32_t)(v >> 32));
    const uint32_t lo = __reduce_min_sync(kFull, (uint32_t)(v >> 32) == hi ? (uint32_t)v : ~0u);
    return ((unsigned long long)hi << 32) | lo;
}
// Sum modulo 2^64: three limbs of 22, 22 and 20 bits; 32 lanes' limbs sum to
// under 2^27, so each 32-bit reduction is exact.
__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
    const uint32_t l0 = __reduce_add_sync(kFull, (uint32_t)(v & 0x3FFFFFu));
    const uint32_t l1 = __reduce_add_sync(kFull, (uint32_t)((v >> 22) & 0x3FFFFFu));
    const uint32_t l2 = __reduce_add_sync(kFull, (uint32_t)(v >> 44));
    return (unsigned long long)l0 + ((unsigned long long)l1 << 22) + ((unsigned long long)l2 << 44);
}
template <class T>
__device__ __forceinline__ T bcast(T v) { return __shfl_sync(kFull, v, 0); }

// Lane groups for loops over a few short rows (the usual search node: a
// handful of members and candidates).  Each row gets G = 2^lg lanes, G the
// largest power of two with rows * G <= 32 and no larger than the row length
// rounded up to a power of two; lane = row slot * G + column slot, and a lane
// walks columns slot, slot + G, ...  So a pass covers 32 / G rows, and a row
// of c columns takes ceil(c / G) steps instead of c.  Group results are
// combined with a ballot (flags) or xor shuffles inside the aligned group
// (counts).
struct Groups {
    uint32_t lg, G, rows;    // G = 1 << lg lanes per row; rows per pass = 32 >> lg
    uint32_t row, slot;      // this lane's row within a pass, its column slot
    uint32_t mask;           // the lanes of this lane's group
    uint32_t lead;           // one bit per group: its column-slot-0 lane
};

__device__ __forceinline__ Groups make_groups(uint32_t rows, uint32_t cols, uint32_t lane) {
    const int lr = rows <= 1 ? 0 : 32 - __clz(rows - 1);   // log2 of rows rounded up
    const int lc = cols <= 1 ? 0 : 32 - __clz(cols - 1);   // log2 of cols rounded up
    int lg = 5 - lr;
    lg = lg < 0 ? 0 : lg;
    lg = lg < lc ? lg : lc;
    Groups gr;
    gr.lg = (uint32_t)lg;
    gr.G = 1u << lg;
    gr.rows = 32u >> lg;
    gr.row = lane >> lg;
    gr.slot = lane & (gr.G - 1u);
    gr.mask = (lg == 5 ? kFull : (1u << gr.G) - 1u) << (lane & ~(gr.G - 1u));
    uint32_t lead = 1u;
    #pragma unroll 1
    for (uint32_t s = gr.G; s < 32; s <<= 1) lead |= lead << s;
    gr.lead = lead;
    return gr;
}

// Sum of v over this lane's group (every lane gets it; all 32 lanes call).
__device__ __forceinline__ uint32_t group_sum(uint32_t v, const Groups& gr) {
    #pragma unroll 1
    for (uint32_t o = gr.G >> 1; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Does any lane of this lane's group hold `f`?  (All 32 lanes call.)
__device__ __forceinline__ bool group_any(bool f, const Groups& gr) {
    return (__ballot_sync(kFull, f) & gr.mask) != 0;
}

// Next-round task list: records [ns, cnt0, cnt1, graph, sid[ns], smc[ns],
// frame[F_WORDS], list0[2 cnt0], list1[2 cnt1]] addressed by an index array.
constexpr uint32_t kRecHeader = 4;
struct SplitBuf {
    uint32_t* words;
    unsigned long long* idx;
    int* refused;                 // first reason a split was refused (diagnostics; 0 = none)
    unsigned long long* used;     // words reserved (may pass word_cap: those failed)
    unsigned long long* count;    // records reserved (may pass idx_cap)
    unsigned long long* count_fail;   // lowest record index whose reservation failed (~0: none)
    unsigned long long word_cap;
    unsigned long long idx_cap;
};

// Two per-side values.  Selected with a conditional, never indexed, so that
// they stay in registers (an indexed 2-array would live in local memory).
struct U2 {
    uint32_t a, b;
    __device__ __forceinline__ uint32_t get(int s) const { return s ? b : a; }
    __device__ __forceinline__ void set(int s, uint32_t v) {
        a = s ? a : v;
        b = s ? v : b;
    }
};

struct Ctx {
    GraphView g;
    EdgeHash eh;
    uint32_t k;
    uint32_t gid;                                // graph of the current task (batched launches)
    uint32_t* arena;
    uint32_t cap;
    uint32_t* sid;
    uint32_t* smc;
    uint32_t* smask;       // smask[i]: members below i that member i missed, bit j = member j
                           // (valid for mask_base <= i <= 32)
    uint32_t mask_base;    // members restored from a split record carry no mask
    uint32_t smax;
    uint32_t ns;
    U2 nss;                                      // |S| per side
    uint32_t scan_limit;
    uint32_t bits_min;     // k >= 2: lists of at least this many entries get filter bitmaps
    int err;
    unsigned long long cnt, hsum, hxor, nodes;   // warp-uniform
    unsigned long long work;                     // per-lane share
    uint32_t* sat;                               // shared: kSatCap per warp
    uint32_t* src;                               // shared: kSrcCap per warp
    uint32_t lane;
};

__device__ __forceinline__ bool adj_test(Ctx& t, uint32_t a, uint32_t b) {
    t.work += 2;   // one 8-byte key
    return has_edge(t.eh, a, b);
}
__device__ __forceinline__ uint32_t gbit(int s) { return s ? FL_G1 : FL_G0; }

// ----------------------------------------------------------------- counters

__device__ void flush(Ctx& t, const Outputs& o) {
    const unsigned long long work = warp_sum64(t.work);
    if (t.lane == 0) {
        if (t.cnt) {
            const unsigned long long before = atomicAdd(o.count, t.cnt);
            atomicAdd(o.hash_sum, t.hsum);
            atomicXor(o.hash_xor, t.hxor);
            if (o.limit && before + t.cnt >= o.limit) atomicExch(o.gstop ? o.gstop : o.stop, 1);
        }
        if (t.nodes) atomicAdd(o.nodes, t.nodes);
        if (work) atomicAdd(o.work, work);
    }
    t.cnt = t.hsum = t.hxor = t.nodes = 0;
    t.work = 0;
    __syncwarp();
}

// A child or a node's scratch did not fit the arena.  Not an error yet: the
// search loop moves the path into the next round's task list, where each
// frame restarts at the bottom of an empty arena (run_dfs).
// The failing frame and the site (1: a node's scratch, 2: a child) go to two
// spare words after the warp's source list in shared memory, not to registers:
// the search loop carries no extra state for this rare case.
constexpr int TASK_ARENA_FULL = 99;
constexpr uint32_t kSiteNode = 1, kSiteChild = 2;
__device__ __forceinline__ void arena_full(Ctx& t, uint32_t cur, uint32_t site) {
    if (t.lane == 0) { t.src[kSrcCap] = cur; t.src[kSrcCap + 1] = site; }
    __syncwarp();
    t.err = TASK_ARENA_FULL;
}

__device__ void fail(Ctx& t, const Outputs& o, int code) {
    if (!t.err) t.err = code;
    if (t.lane == 0) {
        atomicCAS(o.error, 0, code);
        atomicExch(o.stop, 1);
    }
}

// ----------------------------------------------------------------- members

// Misses of w against the other side of S, or k+1 if w cannot join S
// (per lane; the same test as compat_misses in enum_core.cuh).
__device__ uint32_t compat_lane(Ctx& t, uint32_t w) {
    const int s = side_of(t.g, w);
    if (t.nss.get(1 - s) == 0) return 0;
    uint32_t miss = 0;
    #pragma unroll 1
    for (uint32_t i = 0; i < t.ns; ++i) {
        const uint32_t m = t.sid[i];
        if (side_of(t.g, m) == s) continue;
        if (adj_test(t, w, m)) continue;
        if (++miss > t.k || t.smc[i] >= t.k) return t.k + 1;
    }
    return miss;
}

// Adds c to S (warp); returns its misses.  The members that reach k misses
// because of c go to t.sat (first kSatCap, in S order), their count to *nsat.
__device__ uint32_t push_member(Ctx& t, uint32_t c, uint32_t* nsat_out) {
    const int s = side_of(t.g, c);
    uint32_t miss = 0, nsat = 0, mask0 = 0;
    #pragma unroll 1
    for (uint32_t base = 0; base < t.ns; base += 32) {
        const uint32_t i = base + t.lane;
        bool nm = false, sat = false;
        uint32_t m = 0;
        if (i < t.ns) {
            m = t.sid[i];
            if (side_of(t.g, m) != s && !adj_test(t, c, m)) {
                nm = true;
                const uint32_t v = t.smc[i] + 1;
                t.smc[i] = v;
                sat = v == t.k;
            }
        }
        const uint32_t nmask = __ballot_sync(kFull, nm);
        if (base == 0) mask0 = nmask;
        miss += __popc(nmask);
        const uint32_t sm = __ballot_sync(kFull, sat);
        if (sat) {
            const uint32_t r = nsat + __popc(sm & lanemask_lt());
            if (r < kSatCap) t.sat[r] = m;
        }
        nsat += __popc(sm);
    }
    if (t.lane == 0) {
        t.sid[t.ns] = c;
        t.smc[t.ns] = miss;
        t.smask[t.ns] = mask0;
    }
    __syncwarp();
    t.ns++;
    t.nss.set(s, t.nss.get(s) + 1);
    if (nsat_out) *nsat_out = nsat < kSatCap ? nsat : kSatCap;
    return miss;
}

__device__ void pop_member(Ctx& t) {
    const uint32_t c = t.sid[t.ns - 1];
    t.ns--;
    const int s = side_of(t.g, c);
    t.nss.set(s, t.nss.get(s) - 1);
    if (t.ns <= 32 && t.ns >= t.mask_base) {
        // the members c missed, as recorded when c was pushed
        const uint32_t mask = t.smask[t.ns];
        if (t.lane < t.ns && ((mask >> t.lane) & 1u)) t.smc[t.lane]--;
    } else {
        #pragma unroll 1
        for (uint32_t base = 0; base < t.ns; base += 32) {
            const uint32_t i = base + t.lane;
            if (i < t.ns) {
                const uint32_t m = t.sid[i];
                if (side_of(t.g, m) != s && !adj_test(t, c, m)) t.smc[i]--;
            }
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void pop_to(Ctx& t, uint32_t ns) {
    while (t.ns > ns) pop_member(t);
}

// The first `want` members of side `s` in S order into dst (warp); returns
// how many were found.
__device__ uint32_t first_members(Ctx& t, int s, uint32_t want, uint32_t* dst) {
    uint32_t got = 0;
    #pragma unroll 1
    for (uint32_t base = 0; base < t.ns && got < want; base += 32) {
        const uint32_t i = base + t.lane;
        const bool on = i < t.ns && side_of(t.g, t.sid[i]) == s;
        const uint32_t mask = __ballot_sync(kFull, on);
        if (on) {
            const uint32_t r = got + __popc(mask & lanemask_lt());
            if (r < want) dst[r] = t.sid[i];
        }
        got += __popc(mask);
    }
    __syncwarp();
    return got < want ? got : want;
}

// ----------------------------------------------------------------- leaf / prune tests

// Warp form of outsider_addable (enum_core.cuh): both candidate sides local.
__device__ bool outsider_addable(Ctx& t, const uint32_t* l0, uint32_t n0, const uint32_t* l1,
                                 uint32_t n1, const uint32_t* tot) {
    const GraphView& g = t.g;
    // blockers (tot >= k) of both sides in one pass: key (degree, position),
    // S members at positions 0..ns-1, list entries after them
    unsigned long long bk0 = ~0ull, bk1 = ~0ull;
    #pragma unroll 1
    for (uint32_t i = t.lane; i < t.ns; i += 32) {
        if (tot[i] >= t.k) {
            const uint32_t m = t.sid[i];
            const unsigned long long key = ((unsigned long long)degree(g, m) << 32) | i;
            if (side_of(g, m)) bk1 = key < bk1 ? key : bk1;
            else bk0 = key < bk0 ? key : bk0;
        }
    }
    #pragma unroll 1
    for (uint32_t q = t.lane; q < n0 + n1; q += 32) {
        const bool one = q >= n0;
        const uint32_t qq = one ? q - n0 : q;
        if (tot[t.ns + q] >= t.k) {
            const unsigned long long key =
                ((unsigned long long)degree(g, (one ? l1 : l0)[2 * qq]) << 32) | (t.ns + qq);
            if (one) bk1 = key < bk1 ? key : bk1;
            else bk0 = key < bk0 ? key : bk0;
        }
    }
    bk0 = warp_min64(bk0);
    bk1 = warp_min64(bk1);
    if (bk0 != ~0ull && bk1 != ~0ull) {
        // Both sides have a blocker (the usual case): an outsider of side s
        // must be adjacent to side o's blocker, so each side scans one row.
        // Both rows go through one pass of lane groups (side-0 entries first),
        // so that their dependent loads overlap; the answer is the same "or".
        const uint32_t b1 = (uint32_t)bk1, b0 = (uint32_t)bk0;
        const uint32_t m0 = b1 < t.ns ? t.sid[b1] : l1[2 * (b1 - t.ns)];   // rows of side-0 outsiders
        const uint32_t m1 = b0 < t.ns ? t.sid[b0] : l0[2 * (b0 - t.ns)];   // rows of side-1 outsiders
        const uint32_t d0 = degree(g, m0), d = d0 + degree(g, m1);
        const uint32_t* r0 = g.adj + g.off[m0];
        const uint32_t* r1 = g.adj + g.off[m1];
        if (t.lane == 0) t.work += d;
        const Groups gr = make_groups(d, t.ns + (n0 > n1 ? n0 : n1), t.lane);
        #pragma unroll 1
        for (uint32_t base = 0; base < d; base += gr.rows) {
            const uint32_t p = base + gr.row;
            const bool live = p < d;
            const int s = p >= d0;                     // the outsider's side
            const uint32_t e = live ? (s ? r1[p - d0] : r0[p]) : 0u;
            const uint32_t* ls = s ? l1 : l0;
            const uint32_t* lo = s ? l0 : l1;
            const uint32_t cs = s ? n1 : n0, co = s ? n0 : n1;
            const uint32_t* tots_o = tot + t.ns + (s ? 0u : n0);
            // skipped: in S or in C_s
            bool skip = false;
            if (live) {
                #pragma unroll 1
                for (uint32_t j = gr.slot; j < t.ns + cs && !skip; j += gr.G)
                    skip = j < t.ns ? t.sid[j] == e : ls[2 * (j - t.ns)] == e;
            }
            skip = group_any(skip, gr);
            // misses against S_o u C_o: at most k, none on a member already at k
            bool bad = !live || skip;
            uint32_t miss = 0;
            if (!bad) {
                #pragma unroll 1
                for (uint32_t j = gr.slot; j < t.ns + co && !bad; j += gr.G) {
                    if (j < t.ns) {
                        const uint32_t w = t.sid[j];
                        if (side_of(g, w) == s || adj_test(t, e, w)) continue;
                        bad = ++miss > t.k || tot[j] >= t.k;
                    } else {
                        if (adj_test(t, e, lo[2 * (j - t.ns)])) continue;
                        bad = ++miss > t.k || tots_o[j - t.ns] >= t.k;
                    }
                }
            }
            bad = group_any(bad, gr);
            miss = group_sum(miss, gr);
            if (__any_sync(kFull, !bad && miss <= t.k)) return true;
        }
        return false;
    }
    #pragma unroll 1
    for (int s = 0; s < 2; ++s) {
        const int o = 1 - s;
        const uint32_t* ls = s ? l1 : l0;
        const uint32_t* lo = s ? l0 : l1;
        const uint32_t cs = s ? n1 : n0, co = s ? n0 : n1;
        const uint32_t* tots_o = tot + t.ns + (o ? n0 : 0);
        const uint32_t nopp = t.nss.get(o) + co, nown = t.nss.get(s) + cs;
        // the lowest-degree blocking member of side o, S members first
        const unsigned long long best = o ? bk1 : bk0;
        uint32_t nsrc = 0;
        if (best != ~0ull) {
            const uint32_t pos = (uint32_t)best;
            if (t.lane == 0) t.src[0] = pos < t.ns ? t.sid[pos] : lo[2 * (pos - t.ns)];
            __syncwarp();
            nsrc = 1;
        } else if (nopp >= t.k + 1) {
            nsrc = first_members(t, o, t.k + 1, t.src);
            if (nsrc < t.k + 1) {
                #pragma unroll 1
                for (uint32_t q = t.lane; q + nsrc < t.k + 1 && q < co; q += 32)
                    t.src[nsrc + q] = lo[2 * q];
                __syncwarp();
                const uint32_t more = t.k + 1 - nsrc;
                nsrc += more < co ? more : co;
            }
        } else {
            if (side_end(g, s) - side_begin(g, s) > nown) return true;
            continue;
        }
        // outsiders of side s adjacent to a source, one lane group per row entry
        #pragma unroll 1
        for (uint32_t q = 0; q < nsrc; ++q) {
            const uint32_t m = t.src[q];
            const uint32_t d = degree(g, m);
            const uint32_t* row = g.adj + g.off[m];
            if (t.lane == 0) t.work += d;
            const uint32_t nskip = q + t.ns + cs, nmiss = t.ns + co;
            const Groups gr = make_groups(d, nskip > nmiss ? nskip : nmiss, t.lane);
            #pragma unroll 1
            for (uint32_t base = 0; base < d; base += gr.rows) {
                const uint32_t p = base + gr.row;
                const bool live = p < d;
                const uint32_t e = live ? row[p] : 0u;
                // skipped: adjacent to an earlier source (seen there), in S or in C_s
                bool skip = false;
                if (live) {
                    #pragma unroll 1
                    for (uint32_t j = gr.slot; j < nskip && !skip; j += gr.G) {
                        if (j < q) skip = adj_test(t, e, t.src[j]);
                        else if (j < q + t.ns) skip = t.sid[j - q] == e;
                        else skip = ls[2 * (j - q - t.ns)] == e;
                    }
                }
                skip = group_any(skip, gr);
                // misses against S_o u C_o: at most k, none on a member already at k
                bool bad = !live || skip;
                uint32_t miss = 0;
                if (!bad) {
                    #pragma unroll 1
                    for (uint32_t j = gr.slot; j < nmiss && !bad; j += gr.G) {
                        if (j < t.ns) {
                            const uint32_t w = t.sid[j];
                            if (side_of(g, w) != o || adj_test(t, e, w)) continue;
                            bad = ++miss > t.k || tot[j] >= t.k;
                        } else {
                            if (adj_test(t, e, lo[2 * (j - t.ns)])) continue;
                            bad = ++miss > t.k || tots_o[j - t.ns] >= t.k;
                        }
                    }
                }
                bad = group_any(bad, gr);
                miss = group_sum(miss, gr);
                if (__any_sync(kFull, !bad && miss <= t.k)) return true;
            }
        }
    }
    return false;
}

// Warp form of outsider_addable_mixed (enum_core.cuh): side s global (ids >
// lo), side o local (list l, n entries).  Scratch at `tot`: n list totals,
// then the S_o member ids and their totals (2 ns words).
__device__ bool outsider_addable_mixed(Ctx& t, int s, uint32_t lo, const uint32_t* l, uint32_t n,
                                       uint32_t* tot) {
    const GraphView& g = t.g;
    const int o = 1 - s;
    const uint32_t G = side_end(g, s) - lo - 1;
    uint32_t* mem = tot + n;
    uint32_t* memtot = mem + t.ns;
    uint32_t nm = 0;
    unsigned long long best = ~0ull;
    #pragma unroll 1
    for (uint32_t base = 0; base < t.ns; base += 32) {
        const uint32_t i = base + t.lane;
        const bool on = i < t.ns && side_of(g, t.sid[i]) == o;
        const uint32_t mask = __ballot_sync(kFull, on);
        if (on) {
            const uint32_t w = t.sid[i];
            const uint32_t r = nm + __popc(mask & lanemask_lt());
            const uint32_t tw = t.smc[i] + G - count_above(g, w, lo, &t.work);
            mem[r] = w;
            memtot[r] = tw;
            if (tw >= t.k) {
                const unsigned long long key = ((unsigned long long)degree(g, w) << 32) | i;
                best = key < best ? key : best;
            }
        }
        nm += __popc(mask);
    }
    #pragma unroll 1
    for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t q = base + t.lane;
        if (q < n) {
            const uint32_t w = l[2 * q];
            const uint32_t tq = l[2 * q + 1] + G - count_above(g, w, lo, &t.work);
            tot[q] = tq;
            if (tq >= t.k) {
                const unsigned long long key = ((unsigned long long)degree(g, w) << 32) | (t.ns + q);
                best = key < best ? key : best;
            }
        }
    }
    best = warp_min64(best);
    __syncwarp();
    const uint32_t nopp = nm + n;
    uint32_t nsrc = 0;
    if (best != ~0ull) {
        const uint32_t pos = (uint32_t)best;
        if (t.lane == 0) t.src[0] = pos < t.ns ? t.sid[pos] : l[2 * (pos - t.ns)];
        nsrc = 1;
    } else if (nopp >= t.k + 1) {
        #pragma unroll 1
        for (uint32_t j = t.lane; j < t.k + 1; j += 32) t.src[j] = j < nm ? mem[j] : l[2 * (j - nm)];
        nsrc = t.k + 1;
    } else {
        return (lo + 1 - side_begin(g, s)) > t.nss.get(s);
    }
    __syncwarp();
    #pragma unroll 1
    for (uint32_t q = 0; q < nsrc; ++q) {
        const uint32_t m = t.src[q];
        const uint32_t d = degree(g, m);
        const uint32_t* row = g.adj + g.off[m];
        if (t.lane == 0) t.work += d;
        #pragma unroll 1
        for (uint32_t base = 0; base < d; base += 32) {
            const uint32_t p = base + t.lane;
            bool ok = false, past = false;
            if (p < d) {
                const uint32_t e = row[p];
                past = e > lo;                  // rows are sorted: the rest is in C
                if (!past) {
                    bool skip = false;
                    #pragma unroll 1
                    for (uint32_t r = 0; r < q && !skip; ++r) skip = adj_test(t, e, t.src[r]);
                    #pragma unroll 1
                    for (uint32_t i = 0; i < t.ns && !skip; ++i) skip = t.sid[i] == e;
                    if (!skip) {
                        uint32_t miss = 0;
                        ok = true;
                        #pragma unroll 1
                        for (uint32_t i = 0; i < nm && ok; ++i) {
                            if (adj_test(t, e, mem[i])) continue;
                            if (++miss > t.k || memtot[i] >= t.k) ok = false;
                        }
                        #pragma unroll 1
                        for (uint32_t r = 0; r < n && ok; ++r) {
                            if (adj_test(t, e, l[2 * r])) continue;
                            if (++miss > t.k || tot[r] >= t.k) ok = false;
                        }
                    }
                }
            }
            if (__any_sync(kFull, ok)) return true;
            if (__any_sync(kFull, past)) break;
        }
    }
    return false;
}

// ----------------------------------------------------------------- emission

// Counts (and in record mode writes) the result S u list0 u list1.  Returns
// false only in record mode when the record found no room.
template <bool kRec>
__device__ bool emit(Ctx& t, const Outputs& o, const uint32_t* l0, uint32_t n0, const uint32_t* l1,
                     uint32_t n1) {
    unsigned long long a = 0, b = 0;
    #pragma unroll 1
    for (uint32_t i = t.lane; i < t.ns; i += 32) {
        const unsigned long long e = elem_a(t.sid[i]);
        a += e; b += elem_b(e);
    }
    #pragma unroll 1
    for (uint32_t i = t.lane; i < n0; i += 32) {
        const unsigned long long e = elem_a(l0[2 * i]);
        a += e; b += elem_b(e);
    }
    #pragma unroll 1
    for (uint32_t i = t.lane; i < n1; i += 32) {
        const unsigned long long e = elem_a(l1[2 * i]);
        a += e; b += elem_b(e);
    }
    a = warp_sum64(a);
    b = warp_sum64(b);
    const uint32_t nx = t.nss.a + n0, ny = t.nss.b + n1;
    if (kRec) {
        // record mode: room first, then the count (exact limit).  A record
        // that finds no room is not counted: the caller defers the node to
        // the next round, after the host has drained the buffer.
        const unsigned long long words = 2ull + nx + ny;
        unsigned long long at = 0;
        int room = 0, keep = 0;
        if (t.lane == 0) {
            at = atomicAdd(o.out_pos, words);
            room = at + words <= o.out_cap;
            if (!room) {
                atomicMin(o.out_fail, at);
            } else {
                const unsigned long long c = atomicAdd(o.count, 1ull);
                keep = !(o.limit && c >= o.limit);
                if (o.limit && c + 1 >= o.limit) atomicExch(o.stop, 1);
                if (keep) {
                    atomicAdd(o.hash_sum, final_h1(a, nx, ny));
                    atomicXor(o.hash_xor, final_h2(b, nx, ny));
                }
            }
        }
        room = bcast(room);
        keep = bcast(keep);
        at = bcast(at);
        if (!room) return false;
        uint32_t* r = o.out_buf + at;
        if (!keep) {
            // past the limit: a skip record of the same length
            if (t.lane == 0) { r[0] = 0xFFFFFFFFu; r[1] = (uint32_t)(words - 2); }
            __syncwarp();
            return true;
        }
        if (t.lane == 0) { r[0] = nx; r[1] = ny; }
        uint32_t px = 2, py = 2 + nx;
        #pragma unroll 1
        for (uint32_t base = 0; base < t.ns; base += 32) {
            const uint32_t i = base + t.lane;
            const bool in = i < t.ns;
            const uint32_t v = in ? t.sid[i] : 0;
            const bool isy = in && side_of(t.g, v);
            const uint32_t my = __ballot_sync(kFull, isy);
            const uint32_t mx = __ballot_sync(kFull, in && !isy);
            if (isy) r[py + __popc(my & lanemask_lt())] = v;
            else if (in) r[px + __popc(mx & lanemask_lt())] = v;
            px += __popc(mx);
            py += __popc(my);
        }
        #pragma unroll 1
        for (uint32_t i = t.lane; i < n0; i += 32) r[px + i] = l0[2 * i];
        #pragma unroll 1
        for (uint32_t i = t.lane; i < n1; i += 32) r[py + i] = l1[2 * i];
        __syncwarp();
        return true;
    }
    t.cnt++;
    t.hsum += final_h1(a, nx, ny);
    t.hxor ^= final_h2(b, nx, ny);
    if (t.cnt >= kFlushBatch) flush(t, o);
    return true;
}

// ----------------------------------------------------------------- frames

struct Hdr {
    uint32_t ns, flags;
    U2 lo, cnt, off;
    uint32_t order, phase, pos, top, parent, end;
};

__device__ __forceinline__ Hdr read_hdr(const uint32_t* f) {
    Hdr h;
    h.ns = f[F_NS]; h.flags = f[F_FLAGS];
    h.lo.a = f[F_LO0]; h.lo.b = f[F_LO1];
    h.cnt.a = f[F_CNT0]; h.cnt.b = f[F_CNT1];
    h.off.a = f[F_OFF0]; h.off.b = f[F_OFF1];
    h.order = f[F_ORDER]; h.phase = f[F_PHASE]; h.pos = f[F_POS];
    h.top = f[F_TOP]; h.parent = f[F_PARENT_SLOT]; h.end = f[F_END];
    return h;
}

__device__ __forceinline__ void write_hdr(uint32_t* f, const Hdr& h) {
    f[F_NS] = h.ns; f[F_FLAGS] = h.flags;
    f[F_LO0] = h.lo.a; f[F_LO1] = h.lo.b;
    f[F_CNT0] = h.cnt.a; f[F_CNT1] = h.cnt.b;
    f[F_OFF0] = h.off.a; f[F_OFF1] = h.off.b;
    f[F_ORDER] = h.order; f[F_PHASE] = h.phase; f[F_POS] = h.pos;
    f[F_TOP] = h.top; f[F_PARENT_SLOT] = h.parent; f[F_END] = h.end;
}

__device__ __forceinline__ void set_word(Ctx& t, uint32_t at, uint32_t v) {
    if (t.lane == 0) t.arena[at] = v;
    __syncwarp();
}

// Appends the lanes' kept (v, m) pairs at arena[w + 2 cnt], in lane order.
__device__ __forceinline__ void append_pair(Ctx& t, uint32_t w, uint32_t& cnt, bool keep,
                                            uint32_t v, uint32_t m) {
    const uint32_t mask = __ballot_sync(kFull, keep);
    if (keep) {
        const uint32_t r = cnt + __popc(mask & lanemask_lt());
        t.arena[w + 2 * r] = v;
        t.arena[w + 2 * r + 1] = m;
    }
    cnt += __popc(mask);
}

// Filter bitmaps.  When a child S + c of a frame is built, the members of the
// other side that c brings to k misses (sat(c)) must be adjacent to every
// candidate kept on c's side.  sat(c) lies in Z, the other side's members at
// k - 1 misses in the frame.  For a long list that adjacency test repeats for
// every child (O(n^2) probes per frame), so a frame that branches on a list
// of bits_min (kBitsMinList by default) or more entries gets one bitmap per member of Z (up to
// kBitsMaxZ): bit q = list entry q is adjacent to z.  Layout, right after the
// frame's lists (list 0's region first when both exist):
//   [nz, z_0 .. z_nz-1, end_0 .. end_nz-1,
//    bitmap of z_0 (ceil(n / 32) words), ..., bitmap of z_nz-1]
// end_j = 1 + the last list position adjacent to z_j (0: none), so a child
// whose candidates start past it keeps nothing without reading the bitmap.
// Split records do not carry them; a restored frame filters by probing.
__device__ __forceinline__ uint32_t bits_region(const Ctx& t, uint32_t cur, const Hdr& f, int s) {
    // after the lists the frame stores itself (global and shared sides store none)
    uint32_t at = cur + F_WORDS + 2 * (((f.flags & (FL_G0 | FL_SHARED0)) ? 0u : f.cnt.a) +
                                       ((f.flags & (FL_G1 | FL_SHARED1)) ? 0u : f.cnt.b));
    if (s == 1 && (f.flags & FL_BITS0)) {
        const uint32_t nz0 = t.arena[at];
        at += 1 + 2 * nz0 + nz0 * ((f.cnt.a + 31) >> 5);
    }
    return at;
}

// Builds the bitmaps of frame cur (called when it starts branching).
__device__ __forceinline__ void add_filter_bits(Ctx& t, uint32_t cur, const Hdr& f) {
    uint32_t top = f.top, flags = 0;
    #pragma unroll 1
    for (int s = 0; s < 2; ++s) {
        const uint32_t n = f.cnt.get(s);
        if ((f.flags & gbit(s)) || n < t.bits_min) continue;
        const int o = 1 - s;
        // Z: members of side o at k - 1 misses, in S order
        uint32_t nz = 0;
        #pragma unroll 1
        for (uint32_t base = 0; base < t.ns; base += 32) {
            const uint32_t i = base + t.lane;
            const bool on = i < t.ns && side_of(t.g, t.sid[i]) == o && t.smc[i] + 1 == t.k;
            const uint32_t mask = __ballot_sync(kFull, on);
            if (on) {
                const uint32_t r = nz + __popc(mask & lanemask_lt());
                if (r < kBitsMaxZ && top + 1 + r < t.cap) t.arena[top + 1 + r] = t.sid[i];
            }
            nz += __popc(mask);
        }
        const uint32_t nw = (n + 31) >> 5;
        if (nz == 0 || nz > kBitsMaxZ) continue;
        if (top + 1ull + 2 * nz + (unsigned long long)nz * nw > t.cap) break;   // no room: children probe
        if (t.lane == 0) t.arena[top] = nz;
        __syncwarp();
        const uint32_t* lst = t.arena + f.off.get(s);
        uint32_t* bm = t.arena + top + 1 + 2 * nz;
        #pragma unroll 1
        for (uint32_t j = 0; j < nz; ++j) {
            const uint32_t z = t.arena[top + 1 + j];
            uint32_t end = 0;
            #pragma unroll 1
            for (uint32_t base = 0; base < n; base += 32) {
                const uint32_t q = base + t.lane;
                const bool a = q < n && adj_test(t, lst[2 * q], z);
                const uint32_t word = __ballot_sync(kFull, a);
                if (word) end = base + 32 - __clz(word);
                if (t.lane == 0) bm[j * nw + (base >> 5)] = word;
            }
            if (t.lane == 0) t.arena[top + 1 + nz + j] = end;
        }
        flags |= s ? FL_BITS1 : FL_BITS0;
        top += 1 + 2 * nz + nz * nw;
    }
    if (flags) {
        if (t.lane == 0) {
            t.arena[cur + F_FLAGS] |= flags;
            t.arena[cur + F_TOP] = top;
        }
        __syncwarp();
    }
}

// Warp form of build_child (enum_core.cuh): the child "S + c" of frame cur.
template <bool kBits>
__device__ uint32_t build_child(Ctx& t, const Outputs& o, uint32_t cur, uint32_t c, int s,
                                uint32_t p, bool forced, bool opp_done) {
    const GraphView& g = t.g;
    const Hdr f = read_hdr(t.arena + cur);
    pop_to(t, f.ns);
    if (t.ns + 1 > t.smax) { fail(t, o, TASK_E_SMAX); return kNoPos; }
    uint32_t nsat = 0;
    const uint32_t mcc = push_member(t, c, &nsat);
    const int os = 1 - s;
    const uint32_t nc = f.top;
    uint32_t w = nc + F_WORDS;
    if (w > t.cap) { arena_full(t, cur, kSiteChild); return kNoPos; }
    Hdr ch;
    ch.ns = t.ns; ch.flags = 0; ch.lo.a = ch.lo.b = 0; ch.cnt.a = ch.cnt.b = 0; ch.off.a = ch.off.b = 0;
    ch.order = 0; ch.phase = 0; ch.pos = 0; ch.parent = cur; ch.end = 0xFFFFFFFFu;

    // ---- same side as c
    ch.off.set(s, w);
    uint32_t cnt = 0;
    if (f.flags & gbit(s)) {
        if (nsat == 0) {
            ch.flags |= gbit(s);
            ch.lo.set(s, c);
        } else {
            uint32_t z = t.sat[0];
            #pragma unroll 1
            for (uint32_t i = 1; i < nsat; ++i)
                if (degree(g, t.sat[i]) < degree(g, z)) z = t.sat[i];
            const uint32_t dz = degree(g, z);
            if (w + 2ull * dz > t.cap) { arena_full(t, cur, kSiteChild); return kNoPos; }
            if (t.lane == 0) t.work += dz;
            const uint32_t* row = g.adj + g.off[z];
            #pragma unroll 1
            for (uint32_t base = 0; base < dz; base += 32) {
                const uint32_t q = base + t.lane;
                bool keep = false;
                uint32_t v = 0, m = 0;
                if (q < dz) {
                    v = row[q];
                    if (v > c) {
                        m = compat_lane(t, v);
                        keep = m <= t.k;
                    }
                }
                append_pair(t, w, cnt, keep, v, m);
            }
        }
    } else if (!forced && nsat == 0) {
        // nothing to filter: the child's list is the rest of the parent's,
        // read in place (a chain of such children -- a hub's neighbours taken
        // one by one -- then costs a frame per level, not a list per level)
        const uint32_t n = f.cnt.get(s);
        ch.off.set(s, f.off.get(s) + 2 * (p + 1));
        cnt = n > p + 1 ? n - p - 1 : 0u;
        ch.flags |= s ? FL_SHARED1 : FL_SHARED0;
    } else {
        const uint32_t* lst = t.arena + f.off.get(s);
        const uint32_t n = f.cnt.get(s);
        if (w + 2ull * n > t.cap) { arena_full(t, cur, kSiteChild); return kNoPos; }
        const uint32_t start = forced ? 0u : p + 1;
        // the frame's filter bitmaps, when it has them: sel = the rows of sat(c)
        const uint32_t* bm = nullptr;
        uint32_t sel = 0, nw = 0, end = n;
        if (kBits && nsat && (f.flags & (s ? FL_BITS1 : FL_BITS0))) {
            const uint32_t* reg = t.arena + bits_region(t, cur, f, s);
            const uint32_t nz = reg[0];
            bool all = true;
            #pragma unroll 1
            for (uint32_t i = 0; i < nsat && all; ++i) {
                uint32_t j = 0;
                #pragma unroll 1
                while (j < nz && reg[1 + j] != t.sat[i]) ++j;
                all = j < nz;
                if (all) {
                    sel |= 1u << j;
                    end = reg[1 + nz + j] < end ? reg[1 + nz + j] : end;
                }
            }
            if (all) { bm = reg + 1 + 2 * nz; nw = (n + 31) >> 5; }
        }
        if (kBits && bm) {
            // The keep mask of list entries 32 wi .. 32 wi + 31 is the AND of
            // sat(c)'s bitmap words wi.  Lane i computes word wbase + i; the
            // warp then copies only the kept entries of the non-empty words.
            const uint32_t nwe = (end + 31) >> 5;   // words up to the last kept candidate
            #pragma unroll 1
            for (uint32_t wbase = start >> 5; wbase < nwe; wbase += 32) {
                const uint32_t wi = wbase + t.lane;
                uint32_t mask = 0;
                if (wi < nwe) {
                    mask = ~0u;
                    #pragma unroll 1
                    for (uint32_t r = sel; r; r &= r - 1) mask &= bm[(__ffs(r) - 1) * nw + wi];
                    const uint32_t q0 = wi << 5;
                    if (q0 < start) mask &= start - q0 < 32 ? ~0u << (start - q0) : 0u;
                    if (n - q0 < 32) mask &= (1u << (n - q0)) - 1u;
                    if (p >= q0 && p - q0 < 32) mask &= ~(1u << (p - q0));
                }
                uint32_t live = __ballot_sync(kFull, mask != 0);
                #pragma unroll 1
                while (live) {
                    const uint32_t j = __ffs(live) - 1;
                    live &= live - 1;
                    const uint32_t mj = __shfl_sync(kFull, mask, j);
                    const uint32_t q = ((wbase + j) << 5) + t.lane;
                    if ((mj >> t.lane) & 1u) {
                        const uint32_t r = cnt + __popc(mj & lanemask_lt());
                        t.arena[w + 2 * r] = lst[2 * q];
                        t.arena[w + 2 * r + 1] = lst[2 * q + 1];
                    }
                    cnt += __popc(mj);
                }
            }
            __syncwarp();
        } else {
            #pragma unroll 1
            for (uint32_t base = start; base < n; base += 32) {
                const uint32_t q = base + t.lane;
                bool keep = false;
                uint32_t v = 0, m = 0;
                if (q < n && q != p) {
                    v = lst[2 * q];
                    m = lst[2 * q + 1];
                    keep = true;
                    #pragma unroll 1
                    for (uint32_t i = 0; i < nsat && keep; ++i) keep = adj_test(t, v, t.sat[i]);
                }
                append_pair(t, w, cnt, keep, v, m);
            }
        }
    }
    ch.cnt.set(s, cnt);
    if (!(ch.flags & (FL_SHARED0 | FL_SHARED1))) w += 2 * cnt;

    // ---- other side
    ch.off.set(os, w);
    cnt = 0;
    if (opp_done) {
        // that side was iterated first: nothing left on it
    } else if (f.flags & gbit(os)) {
        const uint32_t lo = f.lo.get(os);
        if (t.nss.get(s) <= t.k && mcc < t.k) {
            ch.flags |= gbit(os);
            ch.lo.set(os, lo);
        } else {
            // candidates touch c (saturated) or one of k+1 members of side s
            uint32_t nsrc;
            if (mcc >= t.k) {
                if (t.lane == 0) t.src[0] = c;
                __syncwarp();
                nsrc = 1;
            } else {
                nsrc = first_members(t, s, t.k + 1, t.src);
            }
            unsigned long long bound = 0;
            #pragma unroll 1
            for (uint32_t q = 0; q < nsrc; ++q) bound += degree(g, t.src[q]);
            if (w + 2 * bound > t.cap) { arena_full(t, cur, kSiteChild); return kNoPos; }
            #pragma unroll 1
            for (uint32_t q = 0; q < nsrc; ++q) {
                const uint32_t m = t.src[q];
                const uint32_t d = degree(g, m);
                const uint32_t* row = g.adj + g.off[m];
                if (t.lane == 0) t.work += d;
                #pragma unroll 1
                for (uint32_t base = 0; base < d; base += 32) {
                    const uint32_t e = base + t.lane;
                    bool keep = false;
                    uint32_t v = 0, mm = 0;
                    if (e < d) {
                        v = row[e];
                        if (v > lo) {
                            bool seen = false;
                            #pragma unroll 1
                            for (uint32_t r = 0; r < q && !seen; ++r) seen = adj_test(t, v, t.src[r]);
                            if (!seen) {
                                mm = compat_lane(t, v);
                                keep = mm <= t.k;
                            }
                        }
                    }
                    append_pair(t, w, cnt, keep, v, mm);
                }
            }
        }
    } else {
        const uint32_t* lst = t.arena + f.off.get(os);
        const uint32_t n = f.cnt.get(os);
        if (w + 2ull * n > t.cap) { arena_full(t, cur, kSiteChild); return kNoPos; }
        #pragma unroll 1
        for (uint32_t base = 0; base < n; base += 32) {
            const uint32_t q = base + t.lane;
            bool keep = false;
            uint32_t v = 0, m = 0;
            if (q < n) {
                v = lst[2 * q];
                const uint32_t cm = lst[2 * q + 1];
                const bool a = adj_test(t, v, c);
                keep = a || (cm + 1 <= t.k && mcc < t.k);
                m = cm + (a ? 0u : 1u);
            }
            append_pair(t, w, cnt, keep, v, m);
        }
    }
    ch.cnt.set(os, cnt);
    w += 2 * cnt;
    ch.top = w;
    #pragma unroll 1
    for (int s2 = 0; s2 < 2; ++s2)
        if ((ch.flags & gbit(s2)) && ch.lo.get(s2) + 1 >= side_end(g, s2)) {
            ch.flags &= ~gbit(s2);
            ch.cnt.set(s2, 0);
        }
    if (t.lane == 0) write_hdr(t.arena + nc, ch);
    __syncwarp();
    return nc;
}

// ----------------------------------------------------------------- small subtrees

// The subtree of a node whose sides are both local yields exactly the maximal
// k-biplexes L with S ⊆ L ⊆ S ∪ C that have a V member: the node rules and
// the branching only drop subsets of C that are no such L.  When C has at most
// kSmallMax entries and S at most 32 members, solve_small tests every subset T
// of C at once, one subset per lane, on bit masks, instead of walking the
// subtree node by node:
//  * S ∪ T is a k-biplex when every member misses at most k of the other side
//    of S ∪ T: its misses inside S (smc, or the list's miss count for a
//    candidate) plus popc(T & its candidate-miss mask);
//  * it is maximal when no vertex outside it can join.  A vertex joins when it
//    misses at most k of L's other side and none of those has k misses in L
//    already (a blocker).  Left-out candidates are tested on their masks.  An
//    outsider of side s that joins some L misses at most k members of S_o and
//    no member with k misses inside S, so it lies in the row of such a
//    saturated member (the lowest-degree one), or in one of the rows of any
//    k + 1 members of S_o.  Those rows are scanned once; each outsider found
//    is kept as two masks: the members of S_o and the candidates of C_o it
//    misses.
// Count mode hashes the results into the warp's counters.  Record mode
// reserves room for all of the node's records at once (as emit does for one):
// no room leaves everything untouched and the node is deferred to the next
// round; then the results are counted (exact limit: past it, skip records)
// and written.  Returns kSmallNo, having changed nothing, when the node does
// not qualify: a side whose outsiders are not bounded that way (S_o has at
// most k members, none saturated), source rows longer than kSmallScanMax in
// total, too little arena room at `scratch` for the outsiders' masks, or (in
// record mode) records that would fill more than half the record buffer.
#ifndef GMK_SMALL_MAX
#define GMK_SMALL_MAX 6
#endif
constexpr uint32_t kSmallMax = GMK_SMALL_MAX;   // 2^6 = 64 subsets: two per lane
#ifndef GMK_SMALL_SCAN_MAX
#define GMK_SMALL_SCAN_MAX 1024
#endif
constexpr uint32_t kSmallScanMax = GMK_SMALL_SCAN_MAX;   // outsider source-row entries
constexpr int kSmallNo = 0, kSmallDone = 1, kSmallDefer = 2;

__device__ __forceinline__ unsigned long long warp_xor64(unsigned long long v) {
    #pragma unroll
    for (int d = 16; d; d >>= 1) v ^= __shfl_xor_sync(kFull, v, d);
    return v;
}

// Inclusive warp prefix sum.
__device__ __forceinline__ uint32_t warp_scan(uint32_t v, uint32_t lane) {
    #pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t x = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v += x;
    }
    return v;
}

template <bool kRec>
__device__ __forceinline__ int solve_small(Ctx& t, const Outputs& o, const uint32_t* l0, uint32_t n0,
                                           const uint32_t* l1, uint32_t n1, uint32_t scratch) {
    const GraphView& g = t.g;
    const uint32_t ns = t.ns, m = n0 + n1, k = t.k, lane = t.lane;
    // lane i < ns holds member i, lane j < m candidate j (list 0, then list 1)
    const bool is_mem = lane < ns;
    const uint32_t my_v = is_mem ? t.sid[lane] : 0u;
    const uint32_t my_smc = is_mem ? t.smc[lane] : 0u;
    const uint32_t mem1 = __ballot_sync(kFull, is_mem && side_of(g, my_v));
    const uint32_t mem0 = __ballot_sync(kFull, is_mem) & ~mem1;
    const bool is_cand = lane < m;
    const bool c_one = lane >= n0;
    const uint32_t* lc = c_one ? l1 + 2 * (lane - n0) : l0 + 2 * lane;
    const uint32_t my_c = is_cand ? lc[0] : 0u;
    const uint32_t my_cm = is_cand ? lc[1] : 0u;
    const uint32_t cand0 = (1u << n0) - 1u;
    const uint32_t cand1 = ((1u << m) - 1u) & ~cand0;

    // outsider sources per outsider side s, as member masks of S_o
    unsigned long long key0 = ~0ull, key1 = ~0ull;
    if (is_mem && my_smc >= k) {
        const unsigned long long key = ((unsigned long long)degree(g, my_v) << 32) | lane;
        if (side_of(g, my_v)) key1 = key; else key0 = key;
    }
    key0 = warp_min64(key0);
    key1 = warp_min64(key1);
    uint32_t srcm[2];
    uint32_t total = 0;
    #pragma unroll 1
    for (int s = 0; s < 2; ++s) {
        const unsigned long long key = s ? key0 : key1;   // side o = 1 - s
        uint32_t memo = s ? mem0 : mem1;
        uint32_t sm = 0;
        if (key != ~0ull) {
            sm = 1u << (uint32_t)key;
        } else {
            if ((uint32_t)__popc(memo) < k + 1) return kSmallNo;
            #pragma unroll 1
            for (uint32_t c = 0; c <= k; ++c) { sm |= memo & (0u - memo); memo &= memo - 1; }
        }
        srcm[s] = sm;
        #pragma unroll 1
        for (uint32_t x = sm; x; x &= x - 1) total += degree(g, __shfl_sync(kFull, my_v, __ffs(x) - 1));
    }
    if (total > kSmallScanMax || scratch + 2ull * total > t.cap) return kSmallNo;

    // candidate j: the other side's candidates and members it misses
    uint32_t my_mcc = 0, my_mcs = 0;
    #pragma unroll 1
    for (uint32_t j = 0; j < m; ++j) {
        const uint32_t cj = __shfl_sync(kFull, my_c, j);
        if (is_cand && c_one != (j >= n0) && !has_edge(t.eh, my_c, cj)) my_mcc |= 1u << j;
    }
    #pragma unroll 1
    for (uint32_t x = c_one ? mem0 : mem1, y = mem0 | mem1; y; y &= y - 1) {
        const uint32_t i = __ffs(y) - 1;
        const uint32_t vi = __shfl_sync(kFull, my_v, i);
        if (is_cand && ((x >> i) & 1u) && !has_edge(t.eh, my_c, vi)) my_mcs |= 1u << i;
    }
    // member i: the candidates it misses (the transpose of the above)
    uint32_t my_msc = 0;
    #pragma unroll 1
    for (uint32_t j = 0; j < m; ++j)
        if ((__shfl_sync(kFull, my_mcs, j) >> lane) & 1u) my_msc |= 1u << j;

    // outsiders: masks (members of S_o missed, candidates of C_o missed)
    uint32_t* ob = t.arena + scratch;
    uint32_t n_out = 0;
    #pragma unroll 1
    for (int s = 0; s < 2; ++s) {
        const uint32_t mems = s ? mem1 : mem0, memo = s ? mem0 : mem1;
        const uint32_t cands = s ? cand1 : cand0, cando = s ? cand0 : cand1;
        uint32_t seen_src = 0;
        #pragma unroll 1
        for (uint32_t sm = srcm[s]; sm; sm &= sm - 1) {
            const uint32_t qi = __ffs(sm) - 1;
            const uint32_t src = __shfl_sync(kFull, my_v, qi);
            const uint32_t d = degree(g, src);
            const uint32_t* row = g.adj + g.off[src];
            #pragma unroll 1
            for (uint32_t base = 0; base < d; base += 32) {
                const uint32_t p = base + lane;
                bool keep = p < d;
                const uint32_t e = keep ? row[p] : 0u;
                // in S_s or C_s: not an outsider (every shuffle is taken by
                // all lanes: none sits behind a short-circuit)
                #pragma unroll 1
                for (uint32_t y = mems; y; y &= y - 1) {
                    const uint32_t vi = __shfl_sync(kFull, my_v, __ffs(y) - 1);
                    keep = keep && vi != e;
                }
                #pragma unroll 1
                for (uint32_t y = cands; y; y &= y - 1) {
                    const uint32_t cj = __shfl_sync(kFull, my_c, __ffs(y) - 1);
                    keep = keep && cj != e;
                }
                // found at an earlier source already
                #pragma unroll 1
                for (uint32_t y = seen_src; y; y &= y - 1) {
                    const uint32_t vr = __shfl_sync(kFull, my_v, __ffs(y) - 1);
                    keep = keep && !has_edge(t.eh, e, vr);
                }
                // misses against S_o: at most k, none on a member with k misses
                uint32_t mos = 0;
                #pragma unroll 1
                for (uint32_t y = memo; y; y &= y - 1) {
                    const uint32_t i = __ffs(y) - 1;
                    const uint32_t vi = __shfl_sync(kFull, my_v, i);
                    const uint32_t si = __shfl_sync(kFull, my_smc, i);
                    if (keep && !has_edge(t.eh, e, vi)) {
                        mos |= 1u << i;
                        keep = si < k && (uint32_t)__popc(mos) <= k;
                    }
                }
                uint32_t moc = 0;
                #pragma unroll 1
                for (uint32_t y = cando; y; y &= y - 1) {
                    const uint32_t j = __ffs(y) - 1;
                    const uint32_t cj = __shfl_sync(kFull, my_c, j);
                    if (keep && !has_edge(t.eh, e, cj)) moc |= 1u << j;
                }
                const uint32_t km = __ballot_sync(kFull, keep);
                if (keep) {
                    const uint32_t r = n_out + __popc(km & lanemask_lt());
                    ob[2 * r] = mos;
                    ob[2 * r + 1] = moc;
                }
                n_out += __popc(km);
            }
            seen_src |= 1u << qi;
        }
    }
    __syncwarp();

    // hash elements: S's sums, and each candidate's
    unsigned long long ea = is_mem ? elem_a(my_v) : 0ull;
    const unsigned long long a_s = warp_sum64(ea);
    const unsigned long long b_s = warp_sum64(is_mem ? elem_b(ea) : 0ull);
    const unsigned long long my_ea = is_cand ? elem_a(my_c) : 0ull;
    const unsigned long long my_eb = is_cand ? elem_b(my_ea) : 0ull;

    // every subset T of C, one per lane; found bit r: subset 32 r + lane is a result
    unsigned long long cnt = 0, h1 = 0, h2 = 0;
    uint32_t found = 0;
    const uint32_t nsub = 1u << m;
    #pragma unroll 1
    for (uint32_t base = 0; base < nsub; base += 32) {
        const uint32_t T = base + lane;
        bool alive = T < nsub && t.nss.b + __popc(T & cand1) > 0;   // a V member
        uint32_t bs = 0, bt = 0;
        #pragma unroll 1
        for (uint32_t y = mem0 | mem1; y; y &= y - 1) {
            const uint32_t i = __ffs(y) - 1;
            const uint32_t tt = __shfl_sync(kFull, my_smc, i) + __popc(T & __shfl_sync(kFull, my_msc, i));
            alive = alive && tt <= k;
            bs |= tt >= k ? 1u << i : 0u;
        }
        #pragma unroll 1
        for (uint32_t j = 0; j < m; ++j) {
            const uint32_t tt = __shfl_sync(kFull, my_cm, j) + __popc(T & __shfl_sync(kFull, my_mcc, j));
            if ((T >> j) & 1u) {
                alive = alive && tt <= k;
                bt |= tt >= k ? 1u << j : 0u;
            }
        }
        // left-out candidates, then outsiders: none may join
        #pragma unroll 1
        for (uint32_t j = 0; j < m; ++j) {
            const uint32_t mcc = __shfl_sync(kFull, my_mcc, j);
            const uint32_t mcs = __shfl_sync(kFull, my_mcs, j);
            const uint32_t cm = __shfl_sync(kFull, my_cm, j);
            if (!((T >> j) & 1u) && cm + __popc(T & mcc) <= k && !(mcs & bs) && !(mcc & bt))
                alive = false;
        }
        #pragma unroll 1
        for (uint32_t x = 0; x < n_out; ++x) {
            if ((x & 15u) == 0 && !__any_sync(kFull, alive)) break;
            const uint32_t mos = ob[2 * x], moc = ob[2 * x + 1];
            if (__popc(mos) + __popc(T & moc) <= k && !(mos & bs) && !(moc & bt)) alive = false;
        }
        if (alive) found |= 1u << (base >> 5);
        if (kRec || !__any_sync(kFull, alive)) continue;
        unsigned long long a = a_s, b = b_s;
        #pragma unroll 1
        for (uint32_t j = 0; j < m; ++j) {
            const unsigned long long aj = __shfl_sync(kFull, my_ea, j);
            const unsigned long long bj = __shfl_sync(kFull, my_eb, j);
            if ((T >> j) & 1u) { a += aj; b += bj; }
        }
        if (alive) {
            const uint32_t nx = t.nss.a + __popc(T & cand0), ny = t.nss.b + __popc(T & cand1);
            cnt += 1;
            h1 += final_h1(a, nx, ny);
            h2 ^= final_h2(b, nx, ny);
        }
    }
    if (!kRec) {
        t.cnt += warp_sum64(cnt);
        t.hsum += warp_sum64(h1);
        t.hxor ^= warp_xor64(h2);
        return kSmallDone;
    }
    // record mode: room for every record of the node first, then the count
    uint32_t nres = __popc(found), words = 0;
    #pragma unroll 1
    for (uint32_t x = found; x; x &= x - 1) {
        const uint32_t T = ((__ffs(x) - 1) << 5) + lane;
        words += 2 + ns + __popc(T);
    }
    uint32_t rank = warp_scan(nres, lane), off = warp_scan(words, lane);
    const uint32_t n_res = __shfl_sync(kFull, rank, 31), n_words = __shfl_sync(kFull, off, 31);
    rank -= nres;
    off -= words;
    if (n_res == 0) return kSmallDone;
    // records that would fill more than half the buffer go one by one (emit)
    // down the usual path: a node must never need more room than a drained
    // buffer has
    if (2ull * n_words > o.out_cap) return kSmallNo;
    unsigned long long at = 0, c0 = 0;
    int room = 0;
    if (lane == 0) {
        at = atomicAdd(o.out_pos, (unsigned long long)n_words);
        room = at + n_words <= o.out_cap;
        if (!room) {
            atomicMin(o.out_fail, at);
        } else {
            c0 = atomicAdd(o.count, (unsigned long long)n_res);
            if (o.limit && c0 + n_res >= o.limit) atomicExch(o.stop, 1);
        }
    }
    if (!bcast(room)) return kSmallDefer;
    at = bcast(at);
    c0 = bcast(c0);
    #pragma unroll 1
    for (uint32_t base = 0; base < nsub; base += 32) {
        const uint32_t T = base + lane;
        unsigned long long a = a_s, b = b_s;
        #pragma unroll 1
        for (uint32_t j = 0; j < m; ++j) {
            const unsigned long long aj = __shfl_sync(kFull, my_ea, j);
            const unsigned long long bj = __shfl_sync(kFull, my_eb, j);
            if ((T >> j) & 1u) { a += aj; b += bj; }
        }
        if (!((found >> (base >> 5)) & 1u)) continue;
        const uint32_t nx = t.nss.a + __popc(T & cand0), ny = t.nss.b + __popc(T & cand1);
        uint32_t* r = o.out_buf + at + off;
        off += 2 + nx + ny;
        if (o.limit && c0 + rank++ >= o.limit) {
            // past the limit: a skip record of the same length
            r[0] = 0xFFFFFFFFu;
            r[1] = nx + ny;
            continue;
        }
        h1 += final_h1(a, nx, ny);
        h2 ^= final_h2(b, nx, ny);
        r[0] = nx;
        r[1] = ny;
        uint32_t px = 2, py = 2 + nx;
        #pragma unroll 1
        for (uint32_t i = 0; i < ns; ++i) {
            const uint32_t v = t.sid[i];
            if (side_of(g, v)) r[py++] = v; else r[px++] = v;
        }
        #pragma unroll 1
        for (uint32_t j = 0; j < m; ++j)
            if ((T >> j) & 1u) {
                if (j < n0) r[px++] = l0[2 * j];
                else r[py++] = l1[2 * (j - n0)];
            }
    }
    h1 = warp_sum64(h1);
    h2 = warp_xor64(h2);
    if (lane == 0) {
        atomicAdd(o.hash_sum, h1);
        atomicXor(o.hash_xor, h2);
    }
    __syncwarp();
    return kSmallDone;
}

// enter_node: the node's result record found no room in the record buffer.
constexpr int ENTER_DEFER = 3;

// The child a node asks for: "S + c", c on side s at list position p.
struct ChildReq {
    uint32_t c, p;
    int s;
    bool forced, opp_done;
};

// Warp form of enter_node (enum_core.cuh).  ENTER_PUSHED: a forced candidate
// was found; *req describes the child to build.
template <bool kRec, bool kBits>
__device__ int enter_node(Ctx& t, const Outputs& o, uint32_t cur, ChildReq* req) {
    const GraphView& g = t.g;
    const Hdr f = read_hdr(t.arena + cur);
    pop_to(t, f.ns);
    const bool g0 = f.flags & FL_G0, g1 = f.flags & FL_G1;
    if (t.nss.b == 0 && !g1 && f.cnt.b == 0) return ENTER_DONE;   // Y must end up non-empty
    if (g0 != g1) {
        const int s = g0 ? 0 : 1, os = 1 - s;
        const uint32_t n = f.cnt.get(os);
        const uint32_t base = f.top;
        if (base + n + 2ull * t.ns > t.cap) { arena_full(t, cur, kSiteNode); return ENTER_DONE; }
        if (outsider_addable_mixed(t, s, f.lo.get(s), t.arena + f.off.get(os), n, t.arena + base))
            return ENTER_DONE;
    }
    if (!g0 && !g1) {
        const uint32_t n0 = f.cnt.a, n1 = f.cnt.b;
        const uint32_t* l0 = t.arena + f.off.a;
        const uint32_t* l1 = t.arena + f.off.b;
        const unsigned long long pairs = (unsigned long long)(t.ns + n0) * (t.ns + n1);
        if (n0 + n1 == 0 || pairs <= t.scan_limit) {
            const uint32_t base = f.top;
            if (base + (unsigned long long)t.ns + n0 + n1 > t.cap) {
                arena_full(t, cur, kSiteNode);
                return ENTER_DONE;
            }
            uint32_t* tot = t.arena + base;
            uint32_t* tot0 = tot + t.ns;
            uint32_t* tot1 = tot0 + n0;
            // misses inside S u C.  S members: one lane group per member,
            // over the other side's candidates
            {
                const Groups gr = make_groups(t.ns, n0 > n1 ? n0 : n1, t.lane);
                #pragma unroll 1
                for (uint32_t base = 0; base < t.ns; base += gr.rows) {
                    const uint32_t i = base + gr.row;
                    uint32_t m = 0;
                    if (i < t.ns) {
                        const uint32_t v = t.sid[i];
                        const int sv = side_of(g, v);
                        const uint32_t* lo = sv ? l0 : l1;
                        const uint32_t no = sv ? n0 : n1;
                        #pragma unroll 1
                        for (uint32_t q = gr.slot; q < no; q += gr.G)
                            m += adj_test(t, v, lo[2 * q]) ? 0u : 1u;
                    }
                    m = group_sum(m, gr);
                    if (i < t.ns && gr.slot == 0) tot[i] = t.smc[i] + m;
                }
            }
            #pragma unroll 1
            for (uint32_t q = t.lane; q < n1; q += 32) tot1[q] = l1[2 * q + 1];
            __syncwarp();
            // candidate pairs: one lane group per list-0 entry, over list 1;
            // lane j < G adds column (b + j)'s misses of the pass to tot1
            {
                const Groups gr = make_groups(n0, n1, t.lane);
                #pragma unroll 1
                for (uint32_t abase = 0; abase < n0; abase += gr.rows) {
                    const uint32_t a = abase + gr.row;
                    const bool live = a < n0;
                    const uint32_t va = live ? l0[2 * a] : 0u;
                    uint32_t ta = 0;
                    #pragma unroll 1
                    for (uint32_t bbase = 0; bbase < n1; bbase += gr.G) {
                        const uint32_t b = bbase + gr.slot;
                        const bool miss = live && b < n1 && !adj_test(t, va, l1[2 * b]);
                        ta += miss ? 1u : 0u;
                        const uint32_t mm = __ballot_sync(kFull, miss);
                        if (t.lane < gr.G && bbase + t.lane < n1) {
                            const uint32_t mb = __popc(mm & (gr.lead << t.lane));
                            if (mb) tot1[bbase + t.lane] += mb;
                        }
                    }
                    ta = group_sum(ta, gr);
                    if (live && gr.slot == 0) tot0[a] = l0[2 * a + 1] + ta;
                }
            }
            __syncwarp();
            bool bad = false;
            #pragma unroll 1
            for (uint32_t i = t.lane; i < t.ns + n0 + n1; i += 32) bad |= tot[i] > t.k;
            const bool biplex = !__any_sync(kFull, bad);
            const bool addable = outsider_addable(t, l0, n0, l1, n1, tot);
            if (biplex) {
                // S u C is a k-biplex: the only leaf that can be maximal
                if (!addable && !emit<kRec>(t, o, l0, n0, l1, n1)) return ENTER_DEFER;
                return ENTER_DONE;
            }
            if (addable) return ENTER_DONE;
            // a small candidate set: every subset at once (solve_small; in the
            // k = 1 kernels only -- the k >= 2 ones ran 5-25 % slower with it)
            if (!kBits && n0 + n1 <= kSmallMax && t.ns <= 32) {
                const int r = solve_small<kRec>(t, o, l0, n0, l1, n1, base + t.ns + n0 + n1);
                if (r == kSmallDefer) return ENTER_DEFER;
                if (r == kSmallDone) {
                    if (!kRec && t.cnt >= kFlushBatch) flush(t, o);
                    return ENTER_DONE;
                }
            }
            // forced candidate: fits every leaf that lacks it (first in list order)
            #pragma unroll 1
            for (int s = 0; s < 2; ++s) {
                const uint32_t* ls = s ? l1 : l0;
                const uint32_t* ts = s ? tot1 : tot0;
                const uint32_t cs = s ? n1 : n0;
                const uint32_t* lo = s ? l0 : l1;
                const uint32_t* to = s ? tot0 : tot1;
                const uint32_t co = s ? n0 : n1;
                // one lane group per candidate, over S_o then C_o
                const Groups gr = make_groups(cs, t.ns + co, t.lane);
                #pragma unroll 1
                for (uint32_t qbase = 0; qbase < cs; qbase += gr.rows) {
                    const uint32_t q = qbase + gr.row;
                    bool bad = !(q < cs && ts[q] <= t.k);
                    if (!bad) {
                        const uint32_t c = ls[2 * q];
                        #pragma unroll 1
                        for (uint32_t j = gr.slot; j < t.ns + co && !bad; j += gr.G) {
                            if (j < t.ns) {
                                const uint32_t v = t.sid[j];
                                if (side_of(g, v) == s || adj_test(t, c, v)) continue;
                                bad = tot[j] > t.k;
                            } else if (!adj_test(t, c, lo[2 * (j - t.ns)])) {
                                bad = to[j - t.ns] > t.k;
                            }
                        }
                    }
                    const bool gbad = group_any(bad, gr);   // every lane takes the ballot
                    const bool ok = gr.slot == 0 && !gbad;
                    const uint32_t mask = __ballot_sync(kFull, ok);
                    if (mask) {
                        const uint32_t qq = qbase + ((uint32_t)(__ffs(mask) - 1) >> gr.lg);
                        req->c = ls[2 * qq];
                        req->s = s;
                        req->p = qq;
                        req->forced = true;
                        req->opp_done = false;
                        return ENTER_PUSHED;
                    }
                }
            }
        }
    }
    // iterate: local sides before global ones; between two local sides the shorter first
    uint32_t order;
    if (f.flags & FL_ROOT) order = 1u;   // the root branches on V first; root chunks rely on it
    else if (g0 != g1) order = g0 ? 1u : 0u;
    else if (!g0) order = GMK_LOCAL_ORDER(f.cnt.a, f.cnt.b);
    else order = 1u;
    if (t.lane == 0) {
        uint32_t* fw = t.arena + cur;
        fw[F_ORDER] = order;
        fw[F_PHASE] = 0;
        fw[F_POS] = (f.flags & gbit((int)order)) ? f.lo.get(order) + 1 : 0;
    }
    __syncwarp();
    if (kBits && ((!g0 && f.cnt.a >= t.bits_min) || (!g1 && f.cnt.b >= t.bits_min)))
        add_filter_bits(t, cur, f);
    return ENTER_ITERATE;
}

// Warp form of next_child (enum_core.cuh): advances frame cur to its next
// child and describes it in *req; false when the frame is finished.
__device__ bool next_child(Ctx& t, uint32_t cur, ChildReq* req) {
    const GraphView& g = t.g;
    uint32_t* f = t.arena + cur;
    const Hdr h = read_hdr(f);
    uint32_t phase = h.phase, pos = h.pos;
    while (phase < 2) {
        const int s = phase == 0 ? (int)h.order : 1 - (int)h.order;
        const bool opp_done = phase == 1;
        uint32_t c = 0, p = kNoPos;
        bool have = false;
        // F_END bounds the current phase's positions: a root chunk's last
        // V child, or the end of a donated range of children
        if (h.flags & gbit(s)) {
            const uint32_t end = h.end < side_end(g, s) ? h.end : side_end(g, s);
            if (pos < end) { c = pos; p = kNoPos; ++pos; have = true; }
        } else if (pos < (h.end < h.cnt.get(s) ? h.end : h.cnt.get(s))) {
            p = pos;
            c = t.arena[h.off.get(s) + 2 * p];
            ++pos;
            have = true;
        }
        // U children after the V side is exhausted need a V member in S
        if (have && opp_done && s == 0) {
            bool anyv = false;
            #pragma unroll 1
            for (uint32_t i = t.lane; i < h.ns; i += 32) anyv |= side_of(g, t.sid[i]) != 0;
            if (!__any_sync(kFull, anyv)) { have = false; phase = 2; }
        }
        if (!have) {
            if (phase == 2) break;
            ++phase;
            if (phase == 1 && (h.flags & FL_ONE_PHASE)) phase = 2;
            if (phase == 1) {
                const int s2 = 1 - (int)h.order;
                pos = (h.flags & gbit(s2)) ? h.lo.get(s2) + 1 : 0;
            }
            continue;
        }
        if (t.lane == 0) { f[F_PHASE] = phase; f[F_POS] = pos; }
        __syncwarp();
        req->c = c;
        req->s = s;
        req->p = p;
        req->forced = false;
        req->opp_done = opp_done;
        return true;
    }
    if (t.lane == 0) { f[F_PHASE] = phase; f[F_POS] = pos; }
    __syncwarp();
    return false;
}

// ----------------------------------------------------------------- splitting

// Does frame x still have children to explore (or, for the current frame,
// anything to do)?
__device__ __forceinline__ bool frame_pending(const uint32_t* f, bool is_cur) {
    if (!(f[F_FLAGS] & FL_ENTERED)) return is_cur;
    return f[F_PHASE] < 2;
}

__device__ __forceinline__ uint32_t frame_list_words(const uint32_t* f) {
    const uint32_t c0 = (f[F_FLAGS] & FL_G0) ? 0u : f[F_CNT0];
    const uint32_t c1 = (f[F_FLAGS] & FL_G1) ? 0u : f[F_CNT1];
    return 2 * (c0 + c1);
}

// Reserves `words` words and `recs` index slots of the next round's task list
// (warp-uniform result).  Reservations are plain atomic adds: thousands of
// warps split at once when a round winds down.  Positions only grow, so once
// one reservation fails every later one fails too: the records below
// count_fail are the complete, written ones.  A failed word reservation is
// simply left unused.
__device__ bool reserve_records(Ctx& t, const SplitBuf& sb, unsigned long long words,
                                unsigned long long recs, unsigned long long* w0_out,
                                unsigned long long* r0_out) {
    unsigned long long w0 = 0, r0 = 0;
    int ok = 0;
    if (t.lane == 0) {
        w0 = atomicAdd(sb.used, words);
        if (w0 + words <= sb.word_cap) {
            r0 = atomicAdd(sb.count, recs);
            if (r0 + recs <= sb.idx_cap) ok = 1;
            else { atomicMin(sb.count_fail, r0); atomicCAS(sb.refused, 0, 4); }
        } else {
            atomicCAS(sb.refused, 0, 3);
        }
    }
    if (!bcast(ok)) return false;
    *w0_out = bcast(w0);
    *r0_out = bcast(r0);
    return true;
}

// Copies a record of this round unchanged into the next round's task list
// (a round that winds down hands its queued records on instead of starting
// them).  False when the list has no room.
__device__ bool forward_record(Ctx& t, const SplitBuf& sb, const uint32_t* r) {
    const uint32_t ns = r[0], c0 = r[1], c1 = r[2];
    const unsigned long long words = kRecHeader + 2ull * ns + F_WORDS + 2ull * (c0 + c1);
    unsigned long long w0 = 0, r0 = 0;
    if (!reserve_records(t, sb, words, 1, &w0, &r0)) return false;
    uint32_t* dst = sb.words + w0;
    #pragma unroll 1
    for (unsigned long long i = t.lane; i < words; i += 32) dst[i] = r[i];
    if (t.lane == 0) sb.idx[r0] = w0;
    __syncwarp();
    return true;
}

// Writes every pending frame on the path from `cur` to the root as a task of
// the next round.  All-or-nothing: returns false (and writes nothing) when
// the buffer cannot take them all.
__device__ bool split_path(Ctx& t, const SplitBuf& sb, uint32_t cur) {
    // sizes first
    unsigned long long words = 0, recs = 0;
    #pragma unroll 1
    for (uint32_t x = cur; x != kNoPos; x = t.arena[x + F_PARENT_SLOT]) {
        const uint32_t* f = t.arena + x;
        if (!frame_pending(f, x == cur)) continue;
        if ((f[F_FLAGS] & FL_ROOT) && !(f[F_FLAGS] & FL_ENTERED)) {
            if (t.lane == 0) atomicCAS(sb.refused, 0, 1);
            return false;
        }
        words += kRecHeader + 2ull * f[F_NS] + F_WORDS + frame_list_words(f);
        ++recs;
    }
    if (recs == 0) {
        if (t.lane == 0) atomicCAS(sb.refused, 0, 2);
        return false;
    }
    unsigned long long w0 = 0, r0 = 0;
    if (!reserve_records(t, sb, words, recs, &w0, &r0)) return false;
    unsigned long long wp = w0, rp = r0;
    #pragma unroll 1
    for (uint32_t x = cur; x != kNoPos; x = t.arena[x + F_PARENT_SLOT]) {
        const uint32_t* f = t.arena + x;
        if (!frame_pending(f, x == cur)) continue;
        pop_to(t, f[F_NS]);
        const uint32_t ns = f[F_NS];
        const uint32_t c0 = (f[F_FLAGS] & FL_G0) ? 0u : f[F_CNT0];
        const uint32_t c1 = (f[F_FLAGS] & FL_G1) ? 0u : f[F_CNT1];
        uint32_t* r = sb.words + wp;
        if (t.lane == 0) { r[0] = ns; r[1] = c0; r[2] = c1; r[3] = t.gid; sb.idx[rp] = wp; }
        uint32_t* rs = r + kRecHeader;
        #pragma unroll 1
        for (uint32_t i = t.lane; i < ns; i += 32) { rs[i] = t.sid[i]; rs[ns + i] = t.smc[i]; }
        uint32_t* fr = rs + 2 * ns;
        if (t.lane < F_WORDS) fr[t.lane] = f[t.lane];
        uint32_t* lr = fr + F_WORDS;
        const uint32_t* a0 = t.arena + f[F_OFF0];
        const uint32_t* a1 = t.arena + f[F_OFF1];
        #pragma unroll 1
        for (uint32_t i = t.lane; i < 2 * c0; i += 32) lr[i] = a0[i];
        #pragma unroll 1
        for (uint32_t i = t.lane; i < 2 * c1; i += 32) lr[2 * c0 + i] = a1[i];
        wp += kRecHeader + 2ull * ns + F_WORDS + 2ull * (c0 + c1);
        ++rp;
    }
    __syncwarp();
    return true;
}

// ----------------------------------------------------------------- work sharing

// In-launch work sharing.  A warp that runs out of tasks takes a ticket t (a
// counter) and waits on slot t of the record index.  A busy warp that sees
// more tickets than reserved slots (at its poll points) splits the shallowest
// frame of its path that still has unexplored children: the first half of
// that frame's remaining children in the current phase goes into a record
// (F_POS .. F_END, one phase only), the warp keeps the rest.  So the work
// spreads by halving, and each waiting warp watches its own slot -- no retry
// loops on shared counters.  `outstanding` counts the launch's unfinished
// tasks (the queue's entries plus the donations, minus the finished), offset
// by the queue length: the launch's work is done when it is -queue_len.
// Records live in a bump-allocated buffer for the launch; once it is full,
// donation stops and busy warps split into the next round as before.
struct Donation {
    uint32_t* words;
    unsigned long long word_cap;
    unsigned long long* idx;          // slot -> record offset + 1 (0: not yet written)
    unsigned long long idx_cap;
    unsigned long long* used;         // words reserved
    unsigned long long* tail;         // slots reserved
    unsigned long long* claim;        // tickets taken by waiting warps
    unsigned long long* outstanding;  // unfinished tasks - queue_len (mod 2^64)
    unsigned long long* donated;      // records published (statistics)
    int* full;                        // a reservation failed: no more donations
    uint32_t min_nodes;               // a task donates only after this many nodes
};

// Positions left in the current phase of entered frame f ([pos, lim)), and
// whether a second phase follows.
struct Rest {
    uint32_t pos, lim;
    bool next_phase;
};

__device__ __forceinline__ Rest frame_rest(const GraphView& g, const uint32_t* f) {
    Rest r{0, 0, false};
    const uint32_t phase = f[F_PHASE];
    if (phase >= 2) return r;
    const uint32_t order = f[F_ORDER];
    const int s = phase == 0 ? (int)order : 1 - (int)order;
    const uint32_t flags = f[F_FLAGS];
    const uint32_t side = (flags & (s ? FL_G1 : FL_G0)) ? side_end(g, s) : f[F_CNT0 + s];
    r.pos = f[F_POS];
    r.lim = f[F_END] < side ? f[F_END] : side;
    if (r.pos > r.lim) r.pos = r.lim;
    if (phase == 0 && !(flags & FL_ONE_PHASE)) {
        const int s2 = 1 - s;
        r.next_phase = (flags & (s2 ? FL_G1 : FL_G0)) ? f[F_LO0 + s2] + 1 < side_end(g, s2)
                                                      : f[F_CNT0 + s2] > 0;
    }
    return r;
}

// Donates part of the shallowest entered frame above or at `cur` that has
// work left: half of its current phase's remaining children (the first
// half), or the one child left, or -- when the current phase is used up --
// the whole second phase.  Returns true when a record was published.
// Inlined: an out-of-line call makes the search loop save its live
// registers around the call site (ptxas: 48 -> 270 bytes of stack and 5x
// the spill loads).
#ifndef GMK_DONATE_PARTS
#define GMK_DONATE_PARTS 4   // records handed out per poll, at most (1-4: 1.2x on short complete runs)
#endif
constexpr uint32_t kMaxDonateParts = GMK_DONATE_PARTS;

__device__ __forceinline__ bool donate_top(Ctx& t, const Donation& db, uint32_t cur,
                                           unsigned long long want) {
    uint32_t best = kNoPos;
    Rest rb{0, 0, false};
    #pragma unroll 1
    for (uint32_t x = cur; x != kNoPos; x = t.arena[x + F_PARENT_SLOT]) {
        const uint32_t* f = t.arena + x;
        if (!(f[F_FLAGS] & FL_ENTERED)) continue;
        const Rest r = frame_rest(t.g, f);
        if (r.lim > r.pos || r.next_phase) { best = x; rb = r; }
    }
    if (best == kNoPos) return false;
    const uint32_t* f = t.arena + best;
    const uint32_t ns = f[F_NS];
    const uint32_t c0 = (f[F_FLAGS] & FL_G0) ? 0u : f[F_CNT0];
    const uint32_t c1 = (f[F_FLAGS] & FL_G1) ? 0u : f[F_CNT1];
    const unsigned long long words = kRecHeader + 2ull * ns + F_WORDS + 2ull * (c0 + c1);
    // the split: `parts` records of q children each from the front of the
    // current phase's remaining children (one record takes half; with many
    // warps waiting, up to kMaxDonateParts records of equal shares), the
    // donor keeps the rest
    const uint32_t rem = rb.lim - rb.pos;
    uint32_t parts = 1;
    if (rem >= 3 && want > 1) {
        const unsigned long long cap = want < kMaxDonateParts ? want : kMaxDonateParts;
        parts = (uint32_t)(cap < rem - 1 ? cap : rem - 1);
    }
    unsigned long long w0 = 0, slot = 0;
    int ok = 0;
    if (t.lane == 0) {
        w0 = atomicAdd(db.used, words * parts);
        if (w0 + words * parts <= db.word_cap) {
            slot = atomicAdd(db.tail, (unsigned long long)parts);
            ok = slot + parts <= db.idx_cap;
        }
        if (!ok) atomicExch(db.full, 1);
    }
    if (!bcast(ok)) return false;
    w0 = bcast(w0);
    slot = bcast(slot);
    uint32_t r_phase = f[F_PHASE], r_pos = rb.pos, q = 1, r_flags = f[F_FLAGS], r_end = 0;
    uint32_t keep_phase = f[F_PHASE], keep_pos;
    if (rem >= 1) {
        q = rem >= 2 ? rem / (parts + 1) : 1u;
        r_flags |= FL_ONE_PHASE;
        keep_pos = rb.pos + parts * q;
    } else {
        // the current phase is used up: the record takes the second phase
        const int s2 = f[F_ORDER] ? 0 : 1;
        r_phase = 1;
        r_pos = (f[F_FLAGS] & (s2 ? FL_G1 : FL_G0)) ? f[F_LO0 + s2] + 1 : 0u;
        r_end = 0xFFFFFFFFu;
        keep_phase = 2;
        keep_pos = f[F_POS];
    }
    uint32_t* r = db.words + w0;
    if (t.lane < parts) {
        uint32_t* rp = r + t.lane * words;
        rp[0] = ns; rp[1] = c0; rp[2] = c1; rp[3] = t.gid;
    }
    // members as of the frame, with their misses at that depth: the deeper
    // members' misses are taken off (recorded masks where they exist, else
    // adjacency tests), so the warp's own S stays as it is
    #pragma unroll 1
    for (uint32_t i = t.lane; i < ns; i += 32) {
        const uint32_t m = t.sid[i];
        const int sm = side_of(t.g, m);
        uint32_t miss = t.smc[i];
        #pragma unroll 1
        for (uint32_t j = ns; j < t.ns; ++j) {
            if (j <= 32 && j >= t.mask_base) {
                miss -= (i < 32 && ((t.smask[j] >> i) & 1u)) ? 1u : 0u;
            } else {
                const uint32_t c = t.sid[j];
                if (side_of(t.g, c) != sm && !adj_test(t, c, m)) --miss;
            }
        }
        #pragma unroll 1
        for (uint32_t pp = 0; pp < parts; ++pp) {
            uint32_t* rs = r + pp * words + kRecHeader;
            rs[i] = m;
            rs[ns + i] = miss;
        }
    }
    const uint32_t* a0 = t.arena + f[F_OFF0];
    const uint32_t* a1 = t.arena + f[F_OFF1];
    #pragma unroll 1
    for (uint32_t pp = 0; pp < parts; ++pp) {
        uint32_t* fr = r + pp * words + kRecHeader + 2 * ns;
        if (t.lane < F_WORDS) {
            uint32_t v = f[t.lane];
            v = t.lane == F_PHASE ? r_phase : v;
            v = t.lane == F_POS ? (rem >= 1 ? r_pos + pp * q : r_pos) : v;
            v = t.lane == F_END ? (rem >= 1 ? r_pos + (pp + 1) * q : r_end) : v;
            v = t.lane == F_FLAGS ? r_flags : v;
            fr[t.lane] = v;
        }
        uint32_t* lr = fr + F_WORDS;
        #pragma unroll 1
        for (uint32_t i = t.lane; i < 2 * c0; i += 32) lr[i] = a0[i];
        #pragma unroll 1
        for (uint32_t i = t.lane; i < 2 * c1; i += 32) lr[2 * c0 + i] = a1[i];
    }
    __threadfence();                       // every lane's record words before the slots
    __syncwarp();
    if (t.lane == 0) {
        atomicAdd(db.outstanding, (unsigned long long)parts);   // before they can finish
        atomicAdd(db.donated, (unsigned long long)parts);
        __threadfence();
        #pragma unroll 1
        for (uint32_t pp = 0; pp < parts; ++pp) atomicExch(db.idx + slot + pp, w0 + pp * words + 1);
        t.arena[best + F_PHASE] = keep_phase;   // the donor keeps the rest
        t.arena[best + F_POS] = keep_pos;
    }
    __syncwarp();
    return true;
}

// ----------------------------------------------------------------- tasks

struct RunLimits {
    uint32_t split_min_nodes;           // 0: never split for load balance
    const unsigned long long* queue;    // the round's queue head
    unsigned long long queue_len;       // entries this warp's round hands out
    // record mode: once *out_pos passes drain_at the round winds down -- every
    // task is split into the next round after one node, so the host can drain
    // the record buffer (0 = no draining)
    const unsigned long long* out_pos;
    unsigned long long drain_at;
};

__device__ __forceinline__ bool draining(const RunLimits& lim) {
    return lim.drain_at && *(volatile const unsigned long long*)lim.out_pos >= lim.drain_at;
}

// Depth-first search from the frame at arena offset 0; returns the nodes it
// entered.
template <bool kRec, bool kBits>
__device__ __forceinline__ unsigned long long run_dfs(Ctx& t, const Outputs& o, uint32_t first,
                                                     const SplitBuf* sb, const RunLimits& lim,
                                                     const Donation* db) {
    uint32_t cur = 0;
    uint32_t polls = 0;
    unsigned long long task_nodes = 0;
    bool may_split = sb != nullptr && (lim.split_min_nodes != 0 || lim.drain_at != 0);
    while (cur != kNoPos) {
        if (t.err) break;
#ifndef GMK_POLL_MASK
#define GMK_POLL_MASK 7u    // stop / watchdog / split / donation checks every 8 loop steps
#endif
        if ((++polls & GMK_POLL_MASK) == 0) {
            int stop = 0, late = 0, hungry = 0, give = 0;
            if (t.lane == 0) {
                stop = load_flag(o.stop) || (o.gstop && load_flag(o.gstop));
                late = o.deadline_ns && now_ns() > o.deadline_ns;
                // in-launch sharing while its buffer has room; splitting into
                // the next round otherwise
                const bool share = !kRec && db && !load_flag(db->full);
                if (share && task_nodes >= db->min_nodes) {
                    // waiting warps without a record: tickets beyond the reserved slots
                    const long long want = (long long)(*(volatile const unsigned long long*)db->claim -
                                                       *(volatile const unsigned long long*)db->tail);
                    give = want > 0 ? (int)(want < 32 ? want : 32) : 0;
                }
                hungry = may_split && task_nodes >= 1 &&
                         ((!share && lim.split_min_nodes && task_nodes >= lim.split_min_nodes &&
                           *(volatile const unsigned long long*)lim.queue >= lim.queue_len) ||
                          (kRec && draining(lim)));
            }
            stop = bcast(stop); late = bcast(late); hungry = bcast(hungry); give = bcast(give);
            if (stop) break;
            if (late) { fail(t, o, TASK_E_TIMEOUT); break; }
            if (!kRec && give) donate_top(t, *db, cur, (unsigned long long)give);
            if (hungry) {
                if (split_path(t, *sb, cur)) break;
                may_split = false;   // buffer full: finish this task here
            }
        }
        uint32_t* f = t.arena + cur;
        const uint32_t flags = f[F_FLAGS];
        ChildReq req;
        bool want = false;
        if (!(flags & FL_ENTERED)) {
            if (t.lane == 0) f[F_FLAGS] = flags | FL_ENTERED;
            __syncwarp();
            t.nodes++;
            task_nodes++;
            const int r = enter_node<kRec, kBits>(t, o, cur, &req);
            if (kRec && r == ENTER_DEFER) {
                // re-enter this node next round, after the host drained the buffer
                set_word(t, cur + F_FLAGS, flags);
                t.nodes--;
                task_nodes--;
                if (sb && split_path(t, *sb, cur)) break;
                fail(t, o, TASK_E_OUTBUF);
                break;
            }
            if (r == ENTER_DONE) { set_word(t, cur + F_PHASE, 2); cur = f[F_PARENT_SLOT]; continue; }
            if (r == ENTER_PUSHED) {
                set_word(t, cur + F_PHASE, 2);   // the forced child is its only child
                want = true;
            } else if ((flags & FL_ROOT) && f[F_ORDER] == 1u && (f[F_FLAGS] & FL_G1)) {
                const uint32_t p = f[F_POS];
                set_word(t, cur + F_POS, first > p ? first : p);
            }
        }
        if (!want) want = next_child(t, cur, &req);
        if (!want) { cur = f[F_PARENT_SLOT]; continue; }
        const uint32_t ch = build_child<kBits>(t, o, cur, req.c, req.s, req.p, req.forced, req.opp_done);
        cur = ch == kNoPos ? f[F_PARENT_SLOT] : ch;   // kNoPos: t.err is set, the loop ends
    }
    if (t.err == TASK_ARENA_FULL) {
        // A node's scratch or a child did not fit.  Put the frame back as it
        // was -- the node is entered again (its scratch, or a forced child:
        // phase 2), or steps back one position in its phase -- and move the
        // path to the next round, where each frame starts an empty arena.
        // Only a task's base frame that cannot hold its node or one child is
        // an arena overflow (the split list's refusal reason 5 says so).
        const uint32_t at = t.src[kSrcCap], site = t.src[kSrcCap + 1];
        uint32_t* f = t.arena + at;
        const bool reenter = site == kSiteNode || f[F_PHASE] == 2;
        if (t.lane == 0) {
            if (reenter) f[F_FLAGS] &= ~FL_ENTERED;
            else f[F_POS] -= 1;
        }
        __syncwarp();
        if (reenter) t.nodes--;
        t.err = 0;
        if (at == 0 && sb && t.lane == 0) atomicCAS(sb->refused, 0, 5);
        if (!(at != 0 && sb && split_path(t, *sb, at))) fail(t, o, TASK_E_ARENA);
    }
    pop_to(t, 0);
    return task_nodes;
}

// Root task: x in U with its first-level children y in [first, last); the
// search starts at y = first (run_dfs's first).
__device__ __forceinline__ void prep_root(Ctx& t, uint32_t root, uint32_t last) {
    t.ns = 0; t.nss.a = t.nss.b = 0;
    t.mask_base = 0;
    push_member(t, root, nullptr);
    Hdr h;
    h.ns = 1; h.flags = FL_G0 | FL_G1 | FL_ROOT;
    h.lo.a = root; h.lo.b = t.g.nl - 1;
    h.cnt.a = h.cnt.b = 0;
    h.off.a = h.off.b = F_WORDS;
    h.order = 0; h.phase = 0; h.pos = 0;
    h.top = F_WORDS; h.parent = kNoPos; h.end = last;
    #pragma unroll 1
    for (int s = 0; s < 2; ++s)
        if ((h.flags & gbit(s)) && h.lo.get(s) + 1 >= side_end(t.g, s)) {
            h.flags &= ~gbit(s);
            h.cnt.set(s, 0);
        }
    if (t.lane == 0) write_hdr(t.arena, h);
    __syncwarp();
}

// Resumed task: a frame written by split_path or donate_top (its S starts
// with the root); false (and the task's error set) when it does not fit this
// warp's member arrays or arena.  Records are read with L2-coherent loads
// (__ldcg): a donated one was written moments ago by a warp on another SM.
__device__ __forceinline__ bool prep_record(Ctx& t, const Outputs& o, const uint32_t* r) {
    const uint32_t ns = __ldcg(r), c0 = __ldcg(r + 1), c1 = __ldcg(r + 2);
    if (ns > t.smax) { fail(t, o, TASK_E_SMAX); return false; }
    if (F_WORDS + 2ull * (c0 + c1) > t.cap) { fail(t, o, TASK_E_ARENA); return false; }
    // Every id and position of the record is checked before the search uses
    // it: a record that fails is reported (TASK_E_RECORD), never followed.
    bool bad = ns == 0;
    uint32_t nv = 0;
    const uint32_t* rs = r + kRecHeader;
    #pragma unroll 1
    for (uint32_t base = 0; base < ns; base += 32) {
        const uint32_t i = base + t.lane;
        bool isv = false;
        if (i < ns) {
            const uint32_t v = __ldcg(rs + i);
            bad |= v >= t.g.n;
            t.sid[i] = v < t.g.n ? v : 0u;
            t.smc[i] = __ldcg(rs + ns + i);
            isv = side_of(t.g, v) != 0;
        }
        nv += __popc(__ballot_sync(kFull, isv));
    }
    t.ns = ns; t.nss.b = nv; t.nss.a = ns - nv;
    t.mask_base = ns;
    const uint32_t* fr = rs + 2 * ns;
    Hdr h;
    h.ns = __ldcg(fr + F_NS); h.flags = __ldcg(fr + F_FLAGS);
    h.lo.a = __ldcg(fr + F_LO0); h.lo.b = __ldcg(fr + F_LO1);
    h.order = __ldcg(fr + F_ORDER); h.phase = __ldcg(fr + F_PHASE); h.pos = __ldcg(fr + F_POS);
    h.end = __ldcg(fr + F_END);
    h.cnt.a = c0; h.cnt.b = c1;
    bad |= h.ns != ns || h.order > 1 || h.phase > 2 ||
           ((h.flags & FL_G0) && h.lo.a >= t.g.nl) ||
           ((h.flags & FL_G1) && (h.lo.b + 1 < t.g.nl || h.lo.b >= t.g.n));
    // bitmaps are not part of a record, and its lists are stored after the frame
    h.flags &= ~(FL_BITS0 | FL_BITS1 | FL_SHARED0 | FL_SHARED1);
    h.off.a = F_WORDS;
    h.off.b = F_WORDS + 2 * c0;
    h.top = F_WORDS + 2 * (c0 + c1);
    h.parent = kNoPos;
    const uint32_t* lr = fr + F_WORDS;
    #pragma unroll 1
    for (uint32_t i = t.lane; i < 2 * (c0 + c1); i += 32) {
        uint32_t x = __ldcg(lr + i);
        if (!(i & 1u) && x >= t.g.n) { bad = true; x = 0; }   // list entries: (id, misses)
        t.arena[F_WORDS + i] = x;
    }
    if (__any_sync(kFull, bad)) { fail(t, o, TASK_E_RECORD); return false; }
    if (t.lane == 0) write_hdr(t.arena, h);
    __syncwarp();
    return true;
}

}  // namespace warp
}  // namespace gmk
