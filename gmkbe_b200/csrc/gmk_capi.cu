// libgmk.so: the C ABI of include/gmk.h over the sm_100a enumeration kernels.
//
// Host side: .graph.bin reading and CSR validation, device residency of the
// graph and of its edge hash table, a cached per-device workspace (search
// arenas, member buffers, split buffers, record buffer), the round loop of
// persistent-kernel launches, and delivery of result records to the caller's
// sink.  Device side: enumerate_warp_kernel (one search task per warp at a
// time, tasks from a device work queue, unfinished search trees split into
// the next round's tasks) and enumerate_kernel (one task per thread; kept as
// a second, independent implementation for differential tests).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/gmk.h"
#include "enum_core.cuh"
#include "enum_warp.cuh"
#include "mlp.cuh"

namespace {

thread_local std::string g_cuda_err;

int cuda_fail(cudaError_t e, const char* what) {
    g_cuda_err = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return GMK_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GMK_E_NODEV;
    return GMK_E_CUDA;
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

struct Counters {
    unsigned long long count, hash_sum, hash_xor, nodes, work, next_task, out_pos, tasks_done;
    int stop, error;
    unsigned long long t0_ns;   // device clock at the first task (watchdog origin)
};

// Per-round queue, split-buffer and record-buffer counters of the warp engine.
struct RoundCounters {
    unsigned long long next_task, tasks_done, next_used, next_count, out_pos;
    unsigned long long out_fail;    // lowest record position that found no room (~0: none)
    unsigned long long next_fail;   // lowest split-record index that found no room (~0: none)
    int split_refused;              // first reason a split was refused (0 = none)
    int pad;
    // in-launch work sharing (gmk::warp::Donation); the polled counters sit on
    // their own 128-byte lines
    unsigned long long dq_used, donated;
    int dq_full, pad2;
    alignas(128) unsigned long long dq_tail;
    alignas(128) unsigned long long dq_claim;
    alignas(128) unsigned long long outstanding;
};

constexpr int kBlock = 128;
// Edge hash: at most this percentage of its slots hold keys (one per bucket of
// four).  25 % rather than 50 %: a probe's chain is shorter, and each of six
// tuned workloads (complete and result-limited, k = 1 and 2) ran 3-6 % faster
// at 25 %, for twice the hash's memory (12.3 M edges: 537 MB).
constexpr uint32_t kDefaultHashLoad = 25;
constexpr uint32_t kDefaultArena = 1u << 16;
constexpr uint32_t kDefaultSmax = 2048;
// Node rules run while |S u C_U| x |S u C_V| is at most this (gmk_opts.pair_limit 0).
#ifndef GMK_PAIR_LIMIT
#define GMK_PAIR_LIMIT 4096
#endif
constexpr uint32_t kDefaultPairLimit = GMK_PAIR_LIMIT;

// A planned search task (gmk_plan_tasks): root x and the first-level V
// children [first, last) of its search.
struct TaskEntry {
    uint32_t root, first, last, pad;
};

__global__ void __launch_bounds__(kBlock)
enumerate_kernel(gmk::GraphView g, uint32_t k, Counters* ctr, uint32_t* arenas,
                 uint32_t arena_words, uint32_t* sbuf, uint32_t smax, uint32_t pair_limit,
                 unsigned long long n_tasks, uint32_t chunk, uint32_t chunks_per_root,
                 const TaskEntry* tasks, uint32_t root_base, unsigned long long limit,
                 uint32_t* out_buf, unsigned long long out_cap, unsigned long long watchdog_ns) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    gmk::Outputs o;
    o.count = &ctr->count; o.hash_sum = &ctr->hash_sum; o.hash_xor = &ctr->hash_xor;
    o.nodes = &ctr->nodes; o.work = &ctr->work; o.stop = &ctr->stop; o.error = &ctr->error;
    o.limit = limit; o.out_buf = out_buf; o.out_pos = &ctr->out_pos; o.out_cap = out_cap;
    o.out_fail = nullptr;
    o.gstop = nullptr;
    o.deadline_ns = watchdog_ns ? gmk::now_ns() + watchdog_ns : 0ull;
    gmk::Task t;
    t.g = g; t.k = k;
    t.arena = arenas + tid * arena_words; t.cap = arena_words;
    t.sid = sbuf + tid * 2ull * smax; t.smc = t.sid + smax; t.smax = smax;
    t.ns = 0; t.nss[0] = t.nss[1] = 0;
    t.scan_limit = pair_limit; t.err = 0;
    t.cnt = t.hsum = t.hxor = t.nodes = t.work = 0;
    while (!gmk::load_flag(o.stop)) {
        const unsigned long long id = atomicAdd(&ctr->next_task, 1ull);
        if (id >= n_tasks) break;
        atomicAdd(&ctr->tasks_done, 1ull);
        uint32_t root, first, last;
        if (tasks) {
            const TaskEntry e = tasks[id];
            root = e.root; first = e.first; last = e.last;
        } else {
            root = root_base + (uint32_t)(id / chunks_per_root);
            const uint32_t c = (uint32_t)(id % chunks_per_root);
            first = g.nl + c * chunk;
            const uint64_t end = (uint64_t)first + chunk;
            last = end < g.n ? (uint32_t)end : g.n;
        }
        gmk::run_task(t, o, root, first, last);
        gmk::flush(t, o);
        if (t.err) break;
    }
    gmk::flush(t, o);
}

// One warp per block: warps are independent (no block-level sharing), and
// single-warp blocks let the register file's last partial block count.  With
// 25 resident blocks as the target, ptxas allocates 72 registers a thread (a
// few spills) and 28 warps fit per SM; that measured 2-5 % faster on B200 than
// 4-warp blocks at 80 registers (24 warps).  Among 4-warp blocks, 6 per SM (80
// registers) was 6 % faster than 5 (96 registers, no spills) and 20 % faster
// than 4; 7 and 8 (72 / 64 registers) lost to spills.
#ifndef GMK_WARP_BLOCK
#define GMK_WARP_BLOCK 32                    // threads per block of the warp engine
#endif
constexpr int kWBlock = GMK_WARP_BLOCK;
constexpr int kWarpsPerBlock = kWBlock / 32;
// Resident blocks per SM the register allocation targets.
#ifndef GMK_IDLE_SLEEP_MAX
#define GMK_IDLE_SLEEP_MAX 1024u             // ns: longest back-off of a warp waiting for a record
#endif
#ifndef GMK_WARP_MIN_BLOCKS
#define GMK_WARP_MIN_BLOCKS 25
#endif
// The batch instantiation reads each task's graph from memory instead of the
// kernel parameters, so it holds more live registers: at 72 it spilled 0.9 KB a
// thread; 20 blocks (96 registers, 21 warps per SM) ran the mixed batch 7 %
// faster than 25.
constexpr int kBatchMinBlocks = 20;
constexpr uint32_t kDefaultWarpArena = 1u << 18;
// In-launch sharing: a task donates only after this many nodes of its own
// (gmk_opts.donate_min_nodes 0).
#ifndef GMK_DONATE_MIN
#define GMK_DONATE_MIN 16
#endif
constexpr uint32_t kDefaultDonateMin = GMK_DONATE_MIN;

// One graph of a launch.  A launch enumerates one graph (gmk_enumerate) or a
// batch of graphs (gmk_enumerate_batch); each has its own k, chunking, root
// order and counters, and its root tasks occupy [task_begin, task_begin +
// n_roots * chunks) of the launch's task numbering.
struct GraphTask {
    gmk::GraphView g;
    gmk::warp::EdgeHash eh;
    uint32_t k;
    uint32_t chunk, n_roots, root_base;
    unsigned long long limit;          // batches: this graph's result cap (0: none)
    Counters* ctr;                     // counts, hashes, nodes, work of this graph
    unsigned long long* root_nodes;    // optional per-root node log
    unsigned long long task_begin;
};

struct WarpArgs {
    GraphTask single;                  // the graph of a one-graph launch (kernel parameter)
    const GraphTask* graphs;           // the graphs of a batch launch
    uint32_t n_graphs;
    Counters* ctr;                     // stop / error / watchdog origin of the launch
    RoundCounters* rc;
    uint32_t* arenas;
    uint32_t arena_words;
    uint32_t* sbuf;
    uint32_t smax;
    uint32_t pair_limit;
    uint32_t bits_min_list;            // k >= 2: filter bitmaps for lists this long
    // the round's queue: entries [0, n_records) are split records, the rest
    // root tasks root_task_base, root_task_base + 1, ... (this shard's numbering)
    unsigned long long n_records;
    unsigned long long root_task_base;
    unsigned long long queue_len;
    unsigned long long drain_at;       // record mode: wind the round down past this out_pos
    const uint32_t* cur_words;         // split records of the previous round
    const unsigned long long* cur_idx;
    gmk::warp::SplitBuf next;
    uint32_t split_min_nodes;          // 0: never split
    unsigned long long limit;
    uint32_t* out_buf;
    unsigned long long out_cap;
    unsigned long long watchdog_ns;
    const TaskEntry* tasks;            // planned root tasks (pad = graph), or null: each
                                       // graph's roots chunk-major (GraphTask)
    gmk::warp::Donation share;         // in-launch work sharing (share.words null: off)
};

// A waiting warp gives up when the launch's remaining work shows no change
// (no task finished, no record reserved) for this long: a safety net that
// turns a lost task into an error instead of a kernel that never ends.
constexpr unsigned long long kIdleLimitNs = 10ull * 1000000000ull;

// Points the warp's context and counters at graph gid of the launch.  A
// one-graph launch reads its graph from the kernel parameters, so the values
// stay rematerialisable instead of occupying registers.
template <bool kBatch>
__device__ __forceinline__ const GraphTask& use_graph(const WarpArgs& a, uint32_t gid,
                                                     gmk::warp::Ctx& t, gmk::Outputs& o) {
    const GraphTask& G = kBatch ? a.graphs[gid] : a.single;
    t.g = G.g;
    t.eh = G.eh;
    t.k = G.k;
    t.gid = gid;
    o.count = &G.ctr->count; o.hash_sum = &G.ctr->hash_sum; o.hash_xor = &G.ctr->hash_xor;
    o.nodes = &G.ctr->nodes; o.work = &G.ctr->work;
    if (kBatch) {
        // each graph of a batch has its own cap; reaching it stops that graph only
        o.limit = G.limit;
        o.gstop = &G.ctr->stop;
    }
    return G;
}

// kBatch: several graphs per launch; kRec: results written as records (the
// count-only instantiation carries none of the record and drain code).
template <bool kBatch, bool kRec, bool kBits>
__global__ void __launch_bounds__(kWBlock, kBatch ? kBatchMinBlocks : GMK_WARP_MIN_BLOCKS)
enumerate_warp_kernel(const __grid_constant__ WarpArgs a) {
    __shared__ uint32_t s_sat[kWarpsPerBlock][gmk::kSatCap];
    __shared__ uint32_t s_src[kWarpsPerBlock][gmk::warp::kSrcCap + 2];   // + arena-overflow note
    using namespace gmk::warp;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t lane = lane_id();
    const unsigned long long wid = (unsigned long long)blockIdx.x * kWarpsPerBlock + wib;
    Counters* ctr = a.ctr;
    gmk::Outputs o;
    o.count = &ctr->count; o.hash_sum = &ctr->hash_sum; o.hash_xor = &ctr->hash_xor;
    o.nodes = &ctr->nodes; o.work = &ctr->work; o.stop = &ctr->stop; o.error = &ctr->error;
    o.limit = a.limit; o.out_buf = a.out_buf; o.out_pos = &a.rc->out_pos; o.out_cap = a.out_cap;
    o.out_fail = &a.rc->out_fail;
    o.gstop = nullptr;
    o.deadline_ns = 0;
    if (a.watchdog_ns) {
        // the first warp of the first round fixes the origin of the watchdog
        unsigned long long t0 = 0;
        if (lane == 0) {
            const unsigned long long now = gmk::now_ns();
            const unsigned long long old = atomicCAS(&ctr->t0_ns, 0ull, now);
            t0 = old ? old : now;
        }
        o.deadline_ns = bcast(t0) + a.watchdog_ns;
    }
    Ctx t;
    use_graph<kBatch>(a, 0, t, o);
    t.arena = a.arenas + wid * a.arena_words; t.cap = a.arena_words;
    t.sid = a.sbuf + wid * 3ull * a.smax; t.smc = t.sid + a.smax; t.smask = t.smc + a.smax;
    t.smax = a.smax; t.mask_base = 0;
    t.ns = 0; t.nss.a = t.nss.b = 0;
    t.scan_limit = a.pair_limit; t.err = 0;
    t.bits_min = a.bits_min_list;
    t.cnt = t.hsum = t.hxor = t.nodes = 0; t.work = 0;
    t.sat = s_sat[wib]; t.src = s_src[wib]; t.lane = lane;
    RunLimits lim;
    lim.split_min_nodes = a.split_min_nodes;
    lim.queue = &a.rc->next_task;
    lim.queue_len = a.queue_len;
    lim.out_pos = &a.rc->out_pos;
    lim.drain_at = a.drain_at;
    // the next round's task list: load balance and record draining split into
    // it, and so does any path that outgrows the arena (plain schedule too)
    const SplitBuf* sb = &a.next;
    const Donation* db = (!kRec && a.share.words) ? &a.share : nullptr;
    for (;;) {
        unsigned long long j = ~0ull;
        int stop = 0;
        if (lane == 0) {
            stop = gmk::load_flag(o.stop);
            if (!stop) {
                if (!(kRec && draining(lim))) {
                    j = atomicAdd(&a.rc->next_task, 1ull);
                } else {
                    // winding down: take only split records (they must all be
                    // taken, to be split again), leave the root tasks queued
                    unsigned long long h = *(volatile unsigned long long*)&a.rc->next_task;
                    for (int tries = 0; tries < (1 << 20) && h < a.n_records; ++tries) {
                        const unsigned long long prev = atomicCAS(&a.rc->next_task, h, h + 1);
                        if (prev == h) { j = h; break; }
                        h = prev;
                    }
                    if (j == ~0ull && h < a.n_records) {
                        atomicCAS(o.error, 0, gmk::TASK_E_TIMEOUT);
                        atomicExch(o.stop, 1);
                    }
                }
            }
        }
        stop = bcast(stop);
        j = bcast(j);
        if (stop) break;
        const uint32_t* rec = nullptr;
        if (j >= a.queue_len) {
            // the queue is empty: take a ticket and wait for its slot's
            // donated record, or for the end of the launch's work (no task
            // outstanding)
            if (!db) break;
            unsigned long long w = 0;
            int quit = 0;
            if (lane == 0) {
                const unsigned long long ticket = atomicAdd(db->claim, 1ull);
                unsigned long long seen = ~0ull, t_seen = gmk::now_ns();
                unsigned sleep_ns = 64;
                for (uint32_t spin = 0;; ++spin) {
                    if (ticket < db->idx_cap) {
                        w = *(volatile unsigned long long*)(db->idx + ticket);
                        if (w) break;
                    }
                    if ((spin & 7u) == 7u) {
                        if (gmk::load_flag(o.stop)) { quit = 1; break; }
                        const unsigned long long out = *(volatile unsigned long long*)db->outstanding;
                        if (out + a.queue_len == 0) { quit = 1; break; }
                        // safety net: the work left must change (a task ends or a
                        // record is reserved) within the limit, else give up
                        const unsigned long long sig = out + 0x9E3779B97F4A7C15ull *
                                                       *(volatile unsigned long long*)db->tail;
                        const unsigned long long now = gmk::now_ns();
                        if (sig != seen) {
                            seen = sig;
                            t_seen = now;
                        } else if (now - t_seen > kIdleLimitNs) {
                            atomicCAS(o.error, 0, gmk::TASK_E_TIMEOUT);
                            atomicExch(o.stop, 1);
                            quit = 1;
                            break;
                        }
                    }
                    __nanosleep(sleep_ns);
                    sleep_ns = sleep_ns < GMK_IDLE_SLEEP_MAX ? sleep_ns * 2 : sleep_ns;
                }
                __threadfence();
            }
            quit = bcast(quit);
            if (quit) break;
            w = bcast(w);
            rec = db->words + (w - 1);
        } else {
            if (lane == 0) atomicAdd(&a.rc->tasks_done, 1ull);
            if (j < a.n_records) rec = a.cur_words + a.cur_idx[j];
        }
        // Either kind of task writes its base frame, then enters the search.
        // k = 1 kernels: one run_dfs call site for both kinds (the search loop
        // is inlined once): 1.1-1.5x faster on complete runs than two inlined
        // copies.  k >= 2 kernels (filter bitmaps): one copy per kind, which
        // measured 1.1x faster there.
        uint32_t first = 0, attr = 0;
        bool go = false;
        unsigned long long* root_nodes = nullptr;
        if (rec) {
            // a record: of the previous round, or donated in this launch
            const GraphTask& G = use_graph<kBatch>(a, kBatch ? __ldcg(rec + 3) : 0u, t, o);
            root_nodes = G.root_nodes;
            attr = __ldcg(rec + gmk::warp::kRecHeader);
            // a round that winds down hands its queued records on unchanged
            if (!(kRec && sb && draining(lim) && forward_record(t, *sb, rec)))
                go = gmk::warp::prep_record(t, o, rec);
            if constexpr (kBits) {
                if (go) {
                    const unsigned long long nodes = gmk::warp::run_dfs<kRec, kBits>(t, o, 0, sb, lim, db);
                    if (root_nodes && lane == 0) atomicAdd(root_nodes + attr, nodes);
                    go = false;
                }
            }
        } else {
            const unsigned long long id = a.root_task_base + (j - a.n_records);
            uint32_t root, last, gi = 0;
            TaskEntry e{0, 0, 0, 0};
            if (a.tasks) {
                // planned: per-root chunks in proportion to the predicted
                // cost, largest first (plan_tasks)
                e = a.tasks[id];
                gi = e.pad;
            } else if (kBatch) {
                // the graph whose task range holds id (the last with task_begin <= id)
                uint32_t hi = a.n_graphs;
                while (hi - gi > 1) {
                    const uint32_t mid = (gi + hi) >> 1;
                    if (a.graphs[mid].task_begin <= id) gi = mid; else hi = mid;
                }
            }
            const GraphTask& G = use_graph<kBatch>(a, gi, t, o);
            root_nodes = G.root_nodes;
            if (a.tasks) {
                root = e.root; first = e.first; last = e.last;
            } else {
                // chunk-major: every root's first chunk of children, then
                // every root's second, ... (the low-degree V children first)
                const unsigned long long local = id - G.task_begin;
                root = G.root_base + (uint32_t)(local % G.n_roots);
                const uint32_t c = (uint32_t)(local / G.n_roots);
                first = t.g.nl + c * G.chunk;
                const unsigned long long end = (unsigned long long)first + G.chunk;
                last = end < t.g.n ? (uint32_t)end : t.g.n;
            }
            attr = root;
            if (!(kBatch && gmk::load_flag(o.gstop))) {   // a capped graph's tasks end at once
                gmk::warp::prep_root(t, root, last);
                if constexpr (kBits) {
                    const unsigned long long nodes = gmk::warp::run_dfs<kRec, kBits>(t, o, first, sb, lim, db);
                    if (root_nodes && lane == 0) atomicAdd(root_nodes + attr, nodes);
                } else {
                    go = true;
                }
            }
        }
        if (!kBits && go) {
            const unsigned long long nodes = gmk::warp::run_dfs<kRec, kBits>(t, o, first, sb, lim, db);
            if (root_nodes && lane == 0) atomicAdd(root_nodes + attr, nodes);
        }
        if (db && lane == 0) atomicAdd(db->outstanding, ~0ull);   // this task is finished
        flush(t, o);
        if (t.err) break;
    }
    flush(t, o);
}

// CSR check on the device: thread i checks vertex i (offsets non-decreasing
// and within adj) and adjacency entry i (inside its row, ascending, an id of
// the other side), so a hub's row is spread over many threads.  It also folds
// the CSR into an order-dependent 64-bit sum (the graph's fingerprint, used
// to match checkpoints to graphs).
__global__ void csr_check_kernel(const uint32_t* off, const uint32_t* adj, uint32_t n, uint32_t nl,
                                 unsigned long long adj_len, int* bad, unsigned long long* fp) {
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long h = 0;
    if (i < n) {
        const uint32_t a = off[i], b = off[i + 1];
        if (a > b || b > adj_len) atomicExch(bad, 1);
        h += gmk::mix64(((unsigned long long)i << 32 | a) ^ 0x6A09E667F3BCC909ull);
    }
    if (i < adj_len) {
        // the row holding entry i: the last v with off[v] <= i
        uint32_t lo = 0, hi = n;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (off[mid] <= i) lo = mid; else hi = mid;
        }
        const uint32_t w = adj[i];
        const uint32_t side_lo = lo < nl ? nl : 0u, side_hi = lo < nl ? n : nl;
        if (w < side_lo || w >= side_hi || (i > off[lo] && adj[i - 1] >= w)) atomicExch(bad, 1);
        h += gmk::mix64((i << 32 | w) ^ 0xBB67AE8584CAA73Bull);
    }
    // one atomic per warp: same-address atomics serialise in L2 (a million
    // of them took 0.6 ms); the sum is order-independent
    for (int o = 16; o; o >>= 1) h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
    if ((threadIdx.x & 31u) == 0 && h) atomicAdd(fp, h);
}

// Cost proxy of every root task x (one warp per root): 1 + the sum over its
// neighbours y of |N(y) above x| -- the U vertices that can join x through a
// common neighbour, i.e. the 2-hop candidates of the task.  The schedule's
// default when no learned cost is given.
__global__ void root_cost_kernel(gmk::GraphView g, float* out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t x = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (x >= g.nl) return;
    const uint32_t d = gmk::degree(g, (uint32_t)x);
    const uint32_t* row = g.adj + g.off[x];
    unsigned long long above = 0, words = 0;
    for (uint32_t i = lane; i < d; i += 32) above += gmk::count_above(g, row[i], (uint32_t)x, &words);
    for (int o = 16; o; o >>= 1) above += __shfl_xor_sync(0xFFFFFFFFu, above, o);
    if (lane == 0) out[x] = 1.f + (float)above;
}

bool read_file(const char* path, std::vector<uint32_t>& words) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (sz < 0 || sz % 4) { std::fclose(fp); return false; }
    words.resize((size_t)sz / 4);
    size_t got = std::fread(words.data(), 4, words.size(), fp);
    std::fclose(fp);
    return got == words.size();
}

}  // namespace

struct gmk_graph {
    int device = 0;
    uint32_t n = 0, nl = 0;
    uint64_t adj_len = 0;
    uint64_t fingerprint = 0;   // hash of the CSR (checkpoint identity)
    uint32_t max_degree = 0;
    uint32_t max_degree_side[2] = {0, 0};   // U side, V side
    uint32_t* d_off = nullptr;
    uint32_t* d_adj = nullptr;
    Counters* d_ctr = nullptr;
    unsigned long long* d_eh = nullptr;   // edge hash: buckets of 4 keys
    unsigned long long eh_bmask = 0;
    size_t eh_bytes = 0;
    unsigned long long u_edges = 0;       // |E| (entries of the U rows)
    uint32_t hash_load = 0;               // the edge hash's maximum load, percent
    unsigned long long* d_root_nodes = nullptr;   // per-root node log (on demand)
    __half* d_feat = nullptr;                     // root features (on demand)
    float* d_cost = nullptr;                      // root cost proxy (on demand)
    std::vector<float> cost;                      // its host copy, computed once
    TaskEntry* d_tasks = nullptr;                 // planned task table (grown on demand)
    size_t tasks_bytes = 0;
    RoundCounters* d_rc = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;   // record delivery, overlapping the next round
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

// Bytes of a graph's root-feature buffer: one FP16 row per U vertex.
size_t feat_bytes(const gmk_graph* g) {
    return (size_t)std::max<uint32_t>(g->nl, 1) * gmk::mlp::F * sizeof(__half);
}

// Search arenas, member buffers and the record buffer are large and outlive
// any one graph: one set per device, grown on demand, kept until exit.
// Calls on the same device are serialised by the mutex.
struct Workspace {
    std::mutex mu;
    uint32_t* d_arena = nullptr;
    size_t arena_bytes = 0;
    uint32_t* d_sbuf = nullptr;
    size_t sbuf_bytes = 0;
    uint32_t* d_out = nullptr;
    size_t out_bytes = 0;
    void* d_graphs = nullptr;     // the launch's GraphTask array
    Counters* d_launch = nullptr; // batches: the launch's own stop / error / watchdog words
    size_t launch_bytes = 0;
    size_t graphs_bytes = 0;
    // two split buffers (this round's records, the next round's)
    uint32_t* d_split_words[2] = {nullptr, nullptr};
    size_t split_words_bytes[2] = {0, 0};
    unsigned long long* d_split_idx[2] = {nullptr, nullptr};
    size_t split_idx_bytes[2] = {0, 0};
    // in-launch work sharing: donated records and their slot index (slots the
    // last launch may have written are cleared before the next one)
    uint32_t* d_dq_words = nullptr;
    size_t dq_words_bytes = 0;
    unsigned long long* d_dq_idx = nullptr;
    size_t dq_idx_bytes = 0;
    unsigned long long dq_dirty = 0;
    // pinned staging of the planned task table: the call does not wait for its
    // copy; the next call waits on tasks_ev before it refills the buffer
    void* h_tasks = nullptr;
    size_t h_tasks_bytes = 0;
    cudaEvent_t tasks_ev = nullptr;
};
constexpr int kMaxDevices = 64;
Workspace g_ws[kMaxDevices];

// Per-device launch facts, looked up once (under the workspace mutex).
struct DeviceInfo {
    bool ready = false;
    int sms = 0, per_sm_warp = 0, per_sm_batch = 0, per_sm_thread = 0;
};
DeviceInfo g_dev[kMaxDevices];

}  // namespace

namespace {

int grow(void** p, size_t* have, size_t need) {
    if (*have >= need && *p) return GMK_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMalloc(p, need);
    if (e != cudaSuccess) { *p = nullptr; return cuda_fail(e, "cudaMalloc(workspace)"); }
    *have = need;
    return GMK_OK;
}

// Per-device cache of graph buffers, streams and events.  Loading and freeing
// graphs one after another (a service handling many requests, the bench's
// end-to-end loop) then reuses device memory instead of paying cudaMalloc /
// cudaFree (which synchronises the device) and stream creation every time.
// At most kPoolCap bytes stay cached per device; the rest is freed.
constexpr size_t kPoolCap = 2ull << 30;
struct DevPool {
    std::mutex mu;
    std::multimap<size_t, void*> blocks;   // size -> block
    size_t cached = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
};
DevPool g_pool[64];

size_t pool_round(size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) / 256 * 256; }

cudaError_t pool_alloc(int dev, void** p, size_t bytes) {
    bytes = pool_round(bytes);
    {
        DevPool& pl = g_pool[dev];
        std::lock_guard<std::mutex> lock(pl.mu);
        auto it = pl.blocks.find(bytes);   // exact sizes only: graph buffers repeat exactly
        if (it != pl.blocks.end()) {
            *p = it->second;
            pl.cached -= it->first;
            pl.blocks.erase(it);
            return cudaSuccess;
        }
    }
    return cudaMalloc(p, bytes);
}

void pool_free(int dev, void* p, size_t bytes) {
    if (!p) return;
    bytes = pool_round(bytes);
    DevPool& pl = g_pool[dev];
    std::lock_guard<std::mutex> lock(pl.mu);
    if (pl.cached + bytes <= kPoolCap) {
        pl.blocks.emplace(bytes, p);
        pl.cached += bytes;
    } else {
        cudaFree(p);
    }
}

// grow() over the pool, for per-graph buffers that come and go with the graph.
int pool_grow(int dev, void** p, size_t* have, size_t need) {
    if (*have >= need && *p) return GMK_OK;
    pool_free(dev, *p, *have);
    *p = nullptr;
    *have = 0;
    const cudaError_t e = pool_alloc(dev, p, need);
    if (e != cudaSuccess) { *p = nullptr; return cuda_fail(e, "cudaMalloc(pool)"); }
    *have = need;
    return GMK_OK;
}

cudaError_t pool_stream(int dev, cudaStream_t* s) {
    {
        DevPool& pl = g_pool[dev];
        std::lock_guard<std::mutex> lock(pl.mu);
        if (!pl.streams.empty()) { *s = pl.streams.back(); pl.streams.pop_back(); return cudaSuccess; }
    }
    return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
}

cudaError_t pool_event(int dev, cudaEvent_t* ev) {
    {
        DevPool& pl = g_pool[dev];
        std::lock_guard<std::mutex> lock(pl.mu);
        if (!pl.events.empty()) { *ev = pl.events.back(); pl.events.pop_back(); return cudaSuccess; }
    }
    return cudaEventCreate(ev);
}

void pool_return(int dev, cudaStream_t s, cudaEvent_t ev) {
    DevPool& pl = g_pool[dev];
    std::lock_guard<std::mutex> lock(pl.mu);
    if (s) pl.streams.push_back(s);
    if (ev) pl.events.push_back(ev);
}

// Copies `words` record words from the device and hands every record to the
// sink (ids sorted per side).  Runs on the graph's copy stream, so it overlaps
// the round the enumeration stream is running.
int deliver_records(gmk_graph* g, const uint32_t* d_rec, unsigned long long words, gmk_sink sink,
                    void* user);

// Edge hash of g at a maximum load of load_pct percent of its slots (buckets
// of four 8-byte keys, a power of two of them); replaces any earlier one.
int build_hash(gmk_graph* g, uint32_t load_pct) {
    const unsigned long long edges = g->u_edges;
    unsigned long long buckets = 1;
    while (buckets * 4ull * load_pct < edges * 100ull) buckets <<= 1;
    if (g->d_eh) pool_free(g->device, g->d_eh, g->eh_bytes);
    g->d_eh = nullptr;
    g->eh_bmask = buckets - 1;
    g->eh_bytes = buckets * 4 * sizeof(unsigned long long);
    g->hash_load = load_pct;
    CK(pool_alloc(g->device, (void**)&g->d_eh, g->eh_bytes));
    CK(cudaMemsetAsync(g->d_eh, 0xFF, g->eh_bytes, g->stream));
    if (edges) {
        const unsigned grid = (unsigned)((edges + 255) / 256);
        gmk::warp::build_edge_hash<<<grid, 256, 0, g->stream>>>(g->d_off, g->d_adj, g->nl, g->d_eh,
                                                                 g->eh_bmask);
        CK(cudaGetLastError());
    }
    return GMK_OK;
}

int upload(const uint32_t* off, const uint32_t* adj, uint32_t n, uint32_t nl, int device,
           gmk_graph** out) {
    if (nl > n || off[0] != 0) return GMK_E_FORMAT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_cuda_err = "no CUDA device";
        return GMK_E_NODEV;
    }
    if (device < 0 || device >= ndev || device >= kMaxDevices) return GMK_E_INVAL;
    CK(cudaSetDevice(device));
    gmk_graph* g = new (std::nothrow) gmk_graph();
    if (!g) return GMK_E_NOMEM;
    g->device = device; g->n = n; g->nl = nl; g->adj_len = off[n];
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t d = off[v + 1] > off[v] ? off[v + 1] - off[v] : 0u;
        g->max_degree = std::max(g->max_degree, d);
        uint32_t& side_max = g->max_degree_side[v < nl ? 0 : 1];
        side_max = std::max(side_max, d);
    }
    auto bail = [&](int code) { gmk_graph_free(g); return code; };
    cudaError_t e;
    if ((e = pool_stream(device, &g->stream)) != cudaSuccess ||
        (e = pool_stream(device, &g->copy_stream)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaStreamCreate"));
    if ((e = pool_event(device, &g->ev0)) != cudaSuccess || (e = pool_event(device, &g->ev1)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaEventCreate"));
    if ((e = pool_alloc(device, (void**)&g->d_off, sizeof(uint32_t) * (n + 1ull))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(offsets)"));
    if ((e = pool_alloc(device, (void**)&g->d_adj, sizeof(uint32_t) * std::max<uint64_t>(1, g->adj_len))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(adj)"));
    if ((e = cudaMemcpyAsync(g->d_off, off, sizeof(uint32_t) * (n + 1ull), cudaMemcpyHostToDevice,
                             g->stream)) != cudaSuccess)
        return bail(cuda_fail(e, "H2D offsets"));
    if (g->adj_len && (e = cudaMemcpyAsync(g->d_adj, adj, sizeof(uint32_t) * g->adj_len,
                                           cudaMemcpyHostToDevice, g->stream)) != cudaSuccess)
        return bail(cuda_fail(e, "H2D adj"));
    if ((e = pool_alloc(device, (void**)&g->d_ctr, sizeof(Counters))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(counters)"));
    if ((e = pool_alloc(device, (void**)&g->d_rc, sizeof(RoundCounters))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(round counters)"));
    // check the CSR on the device before anything reads it as a graph
    {
        struct Check { int bad; int pad; unsigned long long fp; } hc;
        Check* dc = reinterpret_cast<Check*>(g->d_rc);   // scratch until the first enumeration
        if ((e = cudaMemsetAsync(dc, 0, sizeof(Check), g->stream)) != cudaSuccess)
            return bail(cuda_fail(e, "memset(check)"));
        const unsigned long long items = std::max<unsigned long long>(n, g->adj_len);
        if (items) {
            csr_check_kernel<<<(unsigned)((items + 255) / 256), 256, 0, g->stream>>>(
                g->d_off, g->d_adj, n, nl, g->adj_len, &dc->bad, &dc->fp);
            if ((e = cudaGetLastError()) != cudaSuccess) return bail(cuda_fail(e, "csr_check"));
        }
        if ((e = cudaMemcpyAsync(&hc, dc, sizeof(hc), cudaMemcpyDeviceToHost, g->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(g->stream)) != cudaSuccess)
            return bail(cuda_fail(e, "csr_check read-back"));
        if (hc.bad) return bail(GMK_E_FORMAT);
        g->fingerprint = gmk::mix64(hc.fp ^ (((uint64_t)n << 32) | nl));
    }
    g->u_edges = off[nl];
    if (int rc = build_hash(g, kDefaultHashLoad)) return bail(rc);
    if ((e = cudaStreamSynchronize(g->stream)) != cudaSuccess) return bail(cuda_fail(e, "upload"));
    *out = g;
    return GMK_OK;
}

}  // namespace

namespace {

int deliver_records(gmk_graph* g, const uint32_t* d_rec, unsigned long long words, gmk_sink sink,
                    void* user) {
    if (!words) return GMK_OK;
    std::vector<uint32_t> rec(words);
    CK(cudaMemcpyAsync(rec.data(), d_rec, 4ull * words, cudaMemcpyDeviceToHost, g->copy_stream));
    CK(cudaStreamSynchronize(g->copy_stream));
    size_t p = 0;
    while (p + 2 <= rec.size()) {
        const uint32_t nx = rec[p], ny = rec[p + 1];
        if (nx == 0xFFFFFFFFu) { p += 2ull + ny; continue; }   // past the result limit
        if (p + 2ull + nx + ny > rec.size()) break;
        uint32_t* x = rec.data() + p + 2;
        uint32_t* y = x + nx;
        std::sort(x, x + nx);
        std::sort(y, y + ny);
        if (sink(user, x, nx, y, ny)) return GMK_E_SINK;
        p += 2ull + nx + ny;
    }
    return GMK_OK;
}

}  // namespace

extern "C" {

int gmk_abi_version(void) { return GMK_ABI_VERSION; }

const char* gmk_last_cuda_error(void) { return g_cuda_err.c_str(); }

const char* gmk_strerror(int code) {
    switch (code) {
        case GMK_OK: return "ok";
        case GMK_E_INVAL: return "invalid argument";
        case GMK_E_IO: return "cannot read input file";
        case GMK_E_FORMAT: return "malformed graph (header, ids, sides or unsorted rows)";
        case GMK_E_CUDA: return "CUDA runtime error";
        case GMK_E_NOMEM: return "device out of memory";
        case GMK_E_ARENA: return "search task outgrew its arena (raise arena_words)";
        case GMK_E_SMAX: return "k-biplex larger than max_members";
        case GMK_E_TIMEOUT: return "watchdog expired";
        case GMK_E_OUTBUF: return "record buffer too small (raise out_words)";
        case GMK_E_SINK: return "stopped by the sink";
        case GMK_E_NODEV: return "no usable CUDA device";
        case GMK_E_CHECKPOINT: return "checkpoint unreadable or written for another graph / k";
        case GMK_E_SCRATCH: return "request does not fit the static scratch (GMK_STATIC_SCRATCH_BYTES)";
        case GMK_PAUSED: return "paused (checkpoint written, work remains)";
        default: return "unknown error";
    }
}

void gmk_result_hash(const uint32_t* ids, uint32_t n_ids, uint32_t nx, uint32_t ny, uint64_t* h1,
                     uint64_t* h2) {
    uint64_t a = 0, b = 0;
    for (uint32_t i = 0; i < n_ids; ++i) {
        uint64_t e = gmk::elem_a(ids[i]);
        a += e;
        b += gmk::elem_b(e);
    }
    if (h1) *h1 = gmk::final_h1(a, nx, ny);
    if (h2) *h2 = gmk::final_h2(b, nx, ny);
}

int gmk_graph_load(const char* path, int device, gmk_graph** out) {
    if (!path || !out) return GMK_E_INVAL;
    *out = nullptr;
    std::vector<uint32_t> w;
    if (!read_file(path, w)) return GMK_E_IO;
    if (w.size() < 3) return GMK_E_FORMAT;
    const uint32_t adj_len = w[0], n = w[1], nl = w[2];
    if (nl > n) return GMK_E_FORMAT;
    std::vector<uint32_t> off(n + 1ull, 0), adj;
    adj.reserve(adj_len);
    size_t pos = 3;
    for (uint32_t i = 0; i < n; ++i) {
        if (pos + 2 > w.size() || w[pos] != i) return GMK_E_FORMAT;
        const uint32_t d = w[pos + 1];
        pos += 2;
        if (pos + d > w.size()) return GMK_E_FORMAT;
        adj.insert(adj.end(), w.begin() + pos, w.begin() + pos + d);
        pos += d;
        if (adj.size() > 0xFFFFFFFFull) return GMK_E_FORMAT;
        off[i + 1] = (uint32_t)adj.size();
    }
    if (adj.size() != adj_len) return GMK_E_FORMAT;
    return upload(off.data(), adj.data(), n, nl, device, out);
}

int gmk_graph_from_csr(const uint32_t* offsets, const uint32_t* adj, uint32_t n, uint32_t n_left,
                       int device, gmk_graph** out) {
    if (!offsets || !out || (!adj && offsets[n] != 0)) return GMK_E_INVAL;
    *out = nullptr;
    static const uint32_t none = 0;
    return upload(offsets, adj ? adj : &none, n, n_left, device, out);
}

int gmk_graph_info(const gmk_graph* g, uint32_t* n, uint32_t* n_left, uint64_t* adj_len) {
    if (!g) return GMK_E_INVAL;
    if (n) *n = g->n;
    if (n_left) *n_left = g->nl;
    if (adj_len) *adj_len = g->adj_len;
    return GMK_OK;
}

int gmk_graph_set_hash_load(gmk_graph* g, uint32_t load_pct) {
    if (!g || load_pct < 10 || load_pct > 100) return GMK_E_INVAL;
    CK(cudaSetDevice(g->device));
    if (load_pct == g->hash_load) return GMK_OK;
    if (int rc = build_hash(g, load_pct)) return rc;
    CK(cudaStreamSynchronize(g->stream));
    return GMK_OK;
}

int gmk_graph_fingerprint(const gmk_graph* g, uint64_t* out) {
    if (!g || !out) return GMK_E_INVAL;
    *out = g->fingerprint;
    return GMK_OK;
}

void gmk_graph_free(gmk_graph* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    const int d = g->device;
    pool_free(d, g->d_off, sizeof(uint32_t) * (g->n + 1ull));
    pool_free(d, g->d_adj, sizeof(uint32_t) * std::max<uint64_t>(1, g->adj_len));
    pool_free(d, g->d_ctr, sizeof(Counters));
    pool_free(d, g->d_rc, sizeof(RoundCounters));
    pool_free(d, g->d_eh, g->eh_bytes);
    pool_free(d, g->d_root_nodes, 8ull * std::max<uint32_t>(g->nl, 1));
    pool_free(d, g->d_feat, feat_bytes(g));
    pool_free(d, g->d_cost, 4ull * std::max<uint32_t>(g->nl, 1));
    pool_free(d, g->d_tasks, g->tasks_bytes);
    pool_return(d, g->stream, g->ev0);
    pool_return(d, g->copy_stream, g->ev1);
    delete g;
}

void gmk_opts_default(gmk_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->k = 1;
    o->schedule = GMK_SCHEDULE_BATCHED;
}

}  // extern "C"

namespace {

// Root costs of the proxy (root_cost_kernel), computed once per graph.
int proxy_costs(gmk_graph* g, const float** out) {
    if (g->cost.size() != g->nl) {
        if (!g->d_cost) CK(pool_alloc(g->device, (void**)&g->d_cost, 4ull * std::max<uint32_t>(g->nl, 1)));
        gmk::GraphView gv{g->d_off, g->d_adj, g->n, g->nl};
        const uint64_t threads = (uint64_t)g->nl * 32;
        root_cost_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, g->stream>>>(gv, g->d_cost);
        CK(cudaGetLastError());
        std::vector<float> c(g->nl);
        CK(cudaMemcpyAsync(c.data(), g->d_cost, 4ull * g->nl, cudaMemcpyDeviceToHost, g->stream));
        CK(cudaStreamSynchronize(g->stream));
        g->cost.swap(c);
    }
    *out = g->cost.data();
    return GMK_OK;
}

// Roots at positions [rb, re) of the cost order of a graph's nl roots
// (largest cost first, ties by id).
std::vector<uint32_t> select_roots(uint32_t nl, const float* cost, uint32_t rb, uint32_t re) {
    std::vector<uint32_t> order(nl);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [cost](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
    return std::vector<uint32_t>(order.begin() + rb, order.begin() + re);
}

// Splits each root into m chunks of its first-level V children in proportion
// to its cost (m = ceil(cost / unit), at most max_chunks, chunks at least 16
// children wide) and appends them with per-task cost cost / m and graph
// index gi, largest per-task cost first, ties in `roots` order.  That is the
// order a stable sort of the tasks by cost gives (a root's chunks share one
// cost and stay together), at the price of sorting the roots only: for the
// headline graph 623 roots instead of 24 k tasks.
void chunk_roots(uint32_t nl, uint32_t n, const std::vector<uint32_t>& roots, const float* cost,
                 double unit, uint32_t max_chunks, uint32_t gi, std::vector<gmk_task>& out) {
    const uint32_t nv = n - nl;
    if (!nv) return;
    const uint32_t wide = std::max<uint32_t>(1, nv / 16);
    struct RootChunks { uint32_t r, m; float c; };
    std::vector<RootChunks> rc;
    rc.reserve(roots.size());
    uint64_t total = 0;
    for (const uint32_t r : roots) {
        const double c = std::max<double>(cost[r], 0.0);
        double want = unit > 0 ? std::ceil(c / unit) : 1.0;
        want = std::max(1.0, std::min(want, (double)std::min(max_chunks, wide)));
        const uint32_t m = (uint32_t)want;
        rc.push_back({r, m, (float)(c / m)});
        total += m;
    }
    std::stable_sort(rc.begin(), rc.end(),
                     [](const RootChunks& a, const RootChunks& b) { return a.c > b.c; });
    out.reserve(out.size() + total);
    for (const RootChunks& x : rc) {
        const uint32_t width = (nv + x.m - 1) / x.m;
        for (uint32_t i = 0; i < x.m; ++i) {
            const uint64_t first = (uint64_t)nl + (uint64_t)i * width;
            if (first >= n) break;
            const uint32_t last = (uint32_t)std::min<uint64_t>(n, first + width);
            out.push_back(gmk_task{x.r, (uint32_t)first, last, gi, x.c});
        }
    }
}

// Largest cost first (stable; `sorted`: the tasks already are, as chunk_roots
// leaves one graph's), then longest-processing-time assignment to nshards
// shards (each task to the least-loaded shard, lowest index on ties); keeps
// the tasks of `shard`.  Every rank computes the same partition from the same
// costs.
void order_and_shard(std::vector<gmk_task>& tasks, uint32_t nshards, uint32_t shard, bool sorted) {
    if (!sorted)
        std::stable_sort(tasks.begin(), tasks.end(),
                         [](const gmk_task& a, const gmk_task& b) { return a.cost > b.cost; });
    if (nshards <= 1) return;
    std::vector<double> load(nshards, 0.0);
    std::vector<gmk_task> mine;
    for (const gmk_task& t : tasks) {
        uint32_t best = 0;
        for (uint32_t s = 1; s < nshards; ++s)
            if (load[s] < load[best]) best = s;
        load[best] += std::max<double>(t.cost, 1e-9);
        if (best == shard) mine.push_back(t);
    }
    tasks.swap(mine);
}

// One graph of a launch, host side.
struct GraphJob {
    gmk_graph* g;
    uint32_t k;
    uint64_t limit;               // batches: the graph's result cap (0: none)
    uint32_t root_begin, root_end;
    const float* task_cost;       // ORDERED schedule: one cost per root
    uint64_t* root_nodes;         // optional host log
};

// Enumerates the jobs' graphs (all on one device) in one run of launches and
// fills outs[i] per graph.  The single-graph call and the batch call share it;
// a batch needs the warp engine, no records and no sharding (checked by the
// caller).
int run_jobs(std::vector<GraphJob>& jobs, const gmk_opts* opts, gmk_sink sink, void* user,
             gmk_stats* outs) {
    gmk_graph* g0 = jobs[0].g;
    const int device = g0->device;
    const bool warp = opts->engine == GMK_ENGINE_WARP;
    Workspace& ws = g_ws[device];
    std::lock_guard<std::mutex> lock(ws.mu);
    DeviceInfo& di = g_dev[device];
    if (!di.ready) {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &di.per_sm_warp, enumerate_warp_kernel<false, false, false>, kWBlock, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &di.per_sm_batch, enumerate_warp_kernel<true, false, false>, kWBlock, 0));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&di.per_sm_thread, enumerate_kernel,
                                                         kBlock, 0));
        di.sms = sms;
        di.ready = true;
    }
    // resident blocks per SM of the instantiation this run launches
    const int per_sm = std::max(!warp ? di.per_sm_thread : jobs.size() > 1 ? di.per_sm_batch : di.per_sm_warp, 1);
    const int block = warp ? kWBlock : kBlock;
    const uint32_t lanes_per_worker = warp ? 32u : 1u;
    uint32_t max_degree = 0, max_k = 1;
    for (const GraphJob& j : jobs) {
        max_degree = std::max(max_degree, j.g->max_degree);
        max_k = std::max(max_k, j.k);
    }
    // A warp's arena holds its stack of child lists: a list gathered from a hub's
    // row is up to 2 deg words, and nested lists shrink; (k + 2) such lists
    // per warp cover the depths seen on power-law graphs.
    uint32_t arena_words = opts->arena_words;
    if (!arena_words) {
        arena_words = warp ? kDefaultWarpArena : kDefaultArena;
        if (warp) {
            const uint64_t hub = 2ull * max_degree * (max_k + 2) + (1u << 16);
            arena_words = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(arena_words, hub),
                                                        1ull << 30);
        }
    }
    // Members of a k-biplex: every x misses at most k of Y, so |Y| <= (max U
    // degree) + k, and |X| <= (max V degree) + k.  The warp engine sizes its
    // member buffers to that bound (the thread engine keeps the default).
    uint32_t smax = opts->max_members ? opts->max_members : kDefaultSmax;
    if (warp && !opts->max_members) {
        uint64_t bound = 0;
        for (const GraphJob& j : jobs)
            bound = std::max<uint64_t>(bound, (uint64_t)j.g->max_degree_side[0] +
                                                  j.g->max_degree_side[1] + 2ull * j.k + 2);
        smax = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(smax, bound), 1ull << 24);
    }
    // workers: threads (thread engine) or warps (warp engine)
    uint64_t threads = opts->threads ? opts->threads : (uint64_t)di.sms * per_sm * block;
    threads = std::max<uint64_t>(threads, (uint64_t)block);
    // keep the search arenas within 40% of free device memory (asked only when
    // the cached workspace is too small)
    const uint64_t per_worker = 4ull * arena_words + 12ull * smax;
    uint64_t workers = threads / lanes_per_worker;
    if (workers * 4ull * arena_words > ws.arena_bytes || workers * 12ull * smax > ws.sbuf_bytes) {
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const uint64_t budget = (uint64_t)((double)(free_b + ws.arena_bytes + ws.sbuf_bytes) * 0.4);
        if (workers * per_worker > budget)
            workers = std::max<uint64_t>(block / lanes_per_worker, budget / per_worker);
    }
    threads = (workers * lanes_per_worker + block - 1) / block * block;
    workers = threads / lanes_per_worker;
    int rc;
    if ((rc = grow((void**)&ws.d_arena, &ws.arena_bytes, workers * 4ull * arena_words))) return rc;
    if ((rc = grow((void**)&ws.d_sbuf, &ws.sbuf_bytes, workers * 12ull * smax))) return rc;

    // Search tasks.  Planned (the ordered schedule, or a shard of several):
    // roots split by cost into chunks of their first-level children, largest
    // first, longest-processing-time partition over the shards.  Otherwise
    // each graph's roots in id order, every root cut into equal chunks,
    // chunk-major.
    const size_t ng = jobs.size();
    std::vector<GraphTask> gt(ng);
    std::vector<uint32_t> chunks(ng), cprs(ng);
    const uint32_t nsh = opts->nshards > 1 ? opts->nshards : 1u;
    const uint32_t sh = nsh > 1 ? opts->shard : 0u;
    const uint32_t tasks_per = opts->tasks_per_worker ? opts->tasks_per_worker : 8u;
    // (a plain run given costs keeps one task per root and no splitting, but
    // starts the largest predicted roots first: the static schedule with the
    // learned order)
    const bool planned = opts->schedule == GMK_SCHEDULE_ORDERED || nsh > 1 || opts->tasks ||
                         (opts->schedule == GMK_SCHEDULE_PLAIN && jobs[0].task_cost);
    std::vector<gmk_task> plan;
    if (opts->tasks) {
        // the caller's list, as given (checked by gmk_enumerate)
        plan.assign(opts->tasks, opts->tasks + opts->n_tasks);
        for (gmk_task& t : plan) t.graph = 0;
    } else if (planned) {
        std::vector<const float*> costs(ng);
        std::vector<std::vector<uint32_t>> roots(ng);
        double total = 0;
        for (size_t i = 0; i < ng; ++i) {
            const GraphJob& j = jobs[i];
            costs[i] = j.task_cost;
            if (!costs[i] && (rc = proxy_costs(j.g, &costs[i]))) return rc;
            roots[i] = select_roots(j.g->nl, costs[i], j.root_begin, j.root_end);
            for (const uint32_t r : roots[i]) total += std::max<double>(costs[i][r], 0.0);
        }
        const uint32_t max_chunks = opts->schedule == GMK_SCHEDULE_PLAIN ? 1u : 0xFFFFFFFFu;
        const double unit = total / (double)std::max<uint64_t>(1, (uint64_t)tasks_per * workers);
        for (size_t i = 0; i < ng; ++i)
            chunk_roots(jobs[i].g->nl, jobs[i].g->n, roots[i], costs[i], unit, max_chunks,
                        (uint32_t)i, plan);
        order_and_shard(plan, nsh, sh, ng == 1);
        // Under a result limit (the run's, or a batch graph's cap) balance does
        // not matter (every warp stays busy until the limit); how many search
        // nodes the first `limit` results cost does, and that depends on the
        // order.  The model predicts node counts, not result density: largest
        // first took 4-36x longer to the limit than id order, cheapest first
        // 1.1-1.25x less at k = 2 but 1.4-7x more at k = 1 (cl500k: 632 M
        // nodes for 10^8 results against 60 M).  So capped runs keep each
        // graph's roots in id order (the plain schedule's), chunks as planned.
        bool capped = opts->result_limit != 0;
        for (const GraphJob& j : jobs) capped |= j.limit != 0;
        if (capped) {
            std::sort(plan.begin(), plan.end(), [](const gmk_task& a, const gmk_task& b) {
                if (a.graph != b.graph) return a.graph < b.graph;
                return a.root != b.root ? a.root < b.root : a.first < b.first;
            });
        }
    }
    unsigned long long n_tasks = 0;
    for (size_t i = 0; i < ng; ++i) {
        const GraphJob& j = jobs[i];
        gmk_graph* g = j.g;
        const uint32_t nv = g->n - g->nl;
        const uint32_t nroots = j.root_end - j.root_begin;
        uint32_t chunk = std::max<uint32_t>(nv, 1);
        if (opts->schedule != GMK_SCHEDULE_PLAIN && nv) {
            if (opts->chunk) {
                chunk = std::min(opts->chunk, nv);
            } else {
                // about tasks_per (8) tasks per worker, but no chunk below 16 children
                const uint64_t want = (uint64_t)tasks_per * workers;
                const uint64_t per_root = (want + g->nl - 1) / std::max<uint32_t>(g->nl, 1);
                chunk = (uint32_t)std::max<uint64_t>(16, (nv + per_root - 1) / std::max<uint64_t>(1, per_root));
                chunk = std::min(chunk, nv);
            }
        }
        chunks[i] = chunk;
        cprs[i] = nv ? (nv + chunk - 1) / chunk : 0;
        GraphTask& t = gt[i];
        t.g = gmk::GraphView{g->d_off, g->d_adj, g->n, g->nl};
        t.eh.slots = g->d_eh;
        t.eh.bmask = g->eh_bmask;
        t.k = j.k;
        t.chunk = chunk;
        t.n_roots = nroots;
        t.root_base = j.root_begin;
        t.limit = j.limit;
        t.ctr = g->d_ctr;
        t.root_nodes = nullptr;
        if (j.root_nodes) {
            if (!g->d_root_nodes)
                CK(pool_alloc(g->device, (void**)&g->d_root_nodes, 8ull * std::max<uint32_t>(g->nl, 1)));
            CK(cudaMemsetAsync(g->d_root_nodes, 0, 8ull * g->nl, g0->stream));
            t.root_nodes = g->d_root_nodes;
        }
        t.task_begin = n_tasks;
        if (!planned) n_tasks += (unsigned long long)nroots * cprs[i];
        CK(cudaMemsetAsync(g->d_ctr, 0, sizeof(Counters), g0->stream));
    }
    const TaskEntry* d_tasks = nullptr;
    if (planned) {
        n_tasks = plan.size();
        if (!plan.empty()) {
            const size_t bytes = sizeof(TaskEntry) * plan.size();
            if (!ws.tasks_ev) CK(cudaEventCreateWithFlags(&ws.tasks_ev, cudaEventDisableTiming));
            CK(cudaEventSynchronize(ws.tasks_ev));   // the last call's copy has left the buffer
            if (ws.h_tasks_bytes < bytes) {
                if (ws.h_tasks) CK(cudaFreeHost(ws.h_tasks));
                ws.h_tasks = nullptr;
                ws.h_tasks_bytes = 0;
                CK(cudaHostAlloc(&ws.h_tasks, bytes, cudaHostAllocDefault));
                ws.h_tasks_bytes = bytes;
            }
            TaskEntry* tab = static_cast<TaskEntry*>(ws.h_tasks);
            for (size_t i = 0; i < plan.size(); ++i)
                tab[i] = TaskEntry{plan[i].root, plan[i].first, plan[i].last, plan[i].graph};
            if ((rc = pool_grow(g0->device, (void**)&g0->d_tasks, &g0->tasks_bytes, bytes))) return rc;
            CK(cudaMemcpyAsync(g0->d_tasks, tab, bytes, cudaMemcpyHostToDevice, g0->stream));
            CK(cudaEventRecord(ws.tasks_ev, g0->stream));
            d_tasks = g0->d_tasks;
        }
    }
    const unsigned long long my_tasks = n_tasks;
    if ((rc = grow((void**)&ws.d_graphs, &ws.graphs_bytes, sizeof(GraphTask) * ng))) return rc;
    CK(cudaMemcpyAsync(ws.d_graphs, gt.data(), sizeof(GraphTask) * ng, cudaMemcpyHostToDevice,
                       g0->stream));

    uint64_t out_words = 0;
    if (opts->emit) {
        // the warp engine streams through two buffers of out_words each, at
        // least 128 words a warp (a smaller buffer would wind every round down
        // after a few results and multiply the split tasks)
        out_words = opts->out_words ? opts->out_words : (warp ? (16ull << 20) : (64ull << 20));
        if (warp) out_words = std::max<uint64_t>(out_words, workers * 128ull);
        if ((rc = grow((void**)&ws.d_out, &ws.out_bytes, out_words * 4ull * (warp ? 2 : 1))))
            return rc;
    }
    // the warp engine splits unfinished trees (batched / ordered schedules)
    const uint32_t split_min = (!warp || opts->schedule == GMK_SCHEDULE_PLAIN)
                                   ? 0u
                                   : (opts->split_min_nodes ? opts->split_min_nodes : 64u);
    unsigned long long split_word_cap = 0, split_idx_cap = 0;
    if (warp) {   // split records: load balance, record-buffer draining, and round bookkeeping
        split_word_cap = std::max<unsigned long long>(1ull << 22, workers * 8192ull);
        split_idx_cap = std::max<unsigned long long>(1ull << 16, workers * 256ull);
        for (int b = 0; b < 2; ++b) {
            if ((rc = grow((void**)&ws.d_split_words[b], &ws.split_words_bytes[b], split_word_cap * 4)))
                return rc;
            if ((rc = grow((void**)&ws.d_split_idx[b], &ws.split_idx_bytes[b], split_idx_cap * 8)))
                return rc;
        }
    }
    // in-launch work sharing (count-only warp runs that split: batched / ordered)
    const bool share = warp && split_min && !opts->emit && !opts->no_sharing;
    unsigned long long dq_word_cap = 0, dq_idx_cap = 0;
    if (share) {
        dq_word_cap = std::max<unsigned long long>(1ull << 22, workers * 4096ull);
        dq_idx_cap = std::max<unsigned long long>(1ull << 16, workers * 64ull);
        const size_t had = ws.dq_idx_bytes;
        const void* had_p = ws.d_dq_idx;
        if ((rc = grow((void**)&ws.d_dq_words, &ws.dq_words_bytes, dq_word_cap * 4))) return rc;
        if ((rc = grow((void**)&ws.d_dq_idx, &ws.dq_idx_bytes, dq_idx_cap * 8))) return rc;
        if (ws.dq_idx_bytes != had || ws.d_dq_idx != had_p) ws.dq_dirty = ws.dq_idx_bytes / 8;
    }
    const unsigned grid = (unsigned)(threads / block);
    const unsigned long long watchdog_ns = (unsigned long long)opts->watchdog_ms * 1000000ull;
    const uint32_t pair_limit = opts->pair_limit ? opts->pair_limit : kDefaultPairLimit;
    // launch-wide flags: graph 0's counters for one graph; a batch has its own
    // block, since each graph's `stop` there means "this graph reached its cap"
    Counters* launch_ctr = g0->d_ctr;
    if (ng > 1) {
        if ((rc = grow((void**)&ws.d_launch, &ws.launch_bytes, sizeof(Counters)))) return rc;
        CK(cudaMemsetAsync(ws.d_launch, 0, sizeof(Counters), g0->stream));
        launch_ctr = ws.d_launch;
    }
    const unsigned long long single_limit = opts->result_limit ? opts->result_limit : jobs[0].limit;
    Counters h;          // launch-wide flags
    unsigned long long tasks_total = 0, tasks_done = 0, donations = 0;
    uint32_t rounds = 0;
    int warp_emit_rc = GMK_OK;
    CK(cudaEventRecord(g0->ev0, g0->stream));
    if (!warp) {
        const GraphJob& j = jobs[0];
        enumerate_kernel<<<grid, kBlock, 0, g0->stream>>>(
            gt[0].g, j.k, g0->d_ctr, ws.d_arena, arena_words, ws.d_sbuf, smax, pair_limit, n_tasks,
            chunks[0], cprs[0], d_tasks, j.root_begin, opts->result_limit,
            opts->emit ? ws.d_out : nullptr, out_words, watchdog_ns);
        CK(cudaGetLastError());
        CK(cudaEventRecord(g0->ev1, g0->stream));
        CK(cudaMemcpyAsync(&h, g0->d_ctr, sizeof(h), cudaMemcpyDeviceToHost, g0->stream));
        CK(cudaStreamSynchronize(g0->stream));
        tasks_total = my_tasks;
        tasks_done = std::min<unsigned long long>(h.tasks_done, my_tasks);
        rounds = 1;
    } else {
        WarpArgs a;
        a.single = gt[0];
        a.graphs = static_cast<const GraphTask*>(ws.d_graphs);
        a.n_graphs = (uint32_t)ng;
        a.ctr = launch_ctr;
        a.rc = g0->d_rc;
        a.arenas = ws.d_arena;
        a.arena_words = arena_words;
        a.sbuf = ws.d_sbuf;
        a.smax = smax;
        a.pair_limit = pair_limit;
        a.bits_min_list = opts->bits_min_list ? opts->bits_min_list : gmk::warp::kBitsMinList;
        a.split_min_nodes = split_min;
        a.limit = single_limit;
        a.out_buf = opts->emit ? ws.d_out : nullptr;
        a.out_cap = out_words;
        a.watchdog_ns = watchdog_ns;
        a.tasks = d_tasks;
        std::memset(&a.share, 0, sizeof(a.share));
        if (share) {
            RoundCounters* rcd = g0->d_rc;
            a.share.words = ws.d_dq_words;
            a.share.word_cap = dq_word_cap;
            a.share.idx = ws.d_dq_idx;
            a.share.idx_cap = dq_idx_cap;
            a.share.used = &rcd->dq_used;
            a.share.tail = &rcd->dq_tail;
            a.share.claim = &rcd->dq_claim;
            a.share.outstanding = &rcd->outstanding;
            a.share.donated = &rcd->donated;
            a.share.full = &rcd->dq_full;
            a.share.min_nodes = opts->donate_min_nodes ? opts->donate_min_nodes : kDefaultDonateMin;
        }
        // Record mode streams: each round writes one of two record buffers,
        // and while the next round runs the host hands the previous round's
        // records to the sink.  A round winds down (splits its tasks into the
        // next round) once its buffer is half full.
        uint32_t* outb[2] = {ws.d_out, opts->emit ? ws.d_out + out_words : nullptr};
        a.drain_at = opts->emit ? std::max<uint64_t>(1, out_words / 2) : 0;
        unsigned long long root_next = 0, n_records = 0;
        int cur = 0, pending = -1;
        unsigned long long pending_words = 0;
        int sink_rc = GMK_OK;
        const auto host_t0 = std::chrono::steady_clock::now();
        for (int round = 0;; ++round) {
            a.n_records = n_records;
            a.root_task_base = root_next;
            a.queue_len = n_records + (my_tasks - root_next);
            a.cur_words = ws.d_split_words[cur];
            a.cur_idx = ws.d_split_idx[cur];
            a.next.words = ws.d_split_words[cur ^ 1];
            a.next.idx = ws.d_split_idx[cur ^ 1];
            a.next.used = &g0->d_rc->next_used;
            a.next.count = &g0->d_rc->next_count;
            a.next.count_fail = &g0->d_rc->next_fail;
            a.next.refused = &g0->d_rc->split_refused;
            a.next.word_cap = split_word_cap;
            a.next.idx_cap = split_idx_cap;
            a.out_buf = opts->emit ? outb[round & 1] : nullptr;
            CK(cudaMemsetAsync(g0->d_rc, 0, sizeof(RoundCounters), g0->stream));
            CK(cudaMemsetAsync(&g0->d_rc->out_fail, 0xFF, 2 * sizeof(unsigned long long), g0->stream));
            if (share && ws.dq_dirty) {
                // every slot an earlier launch may have written, not only this one's
                CK(cudaMemsetAsync(ws.d_dq_idx, 0,
                                   8ull * std::min<unsigned long long>(ws.dq_dirty, ws.dq_idx_bytes / 8),
                                   g0->stream));
                ws.dq_dirty = 0;
            }
            // k >= 2: the instantiation with filter bitmaps for long lists
            // (at k = 1 their code alone cost 15 %, so it is a separate kernel)
            const bool bits = a.single.k >= 2;
            if (ng == 1 && !opts->emit && !bits)
                enumerate_warp_kernel<false, false, false><<<grid, kWBlock, 0, g0->stream>>>(a);
            else if (ng == 1 && !opts->emit)
                enumerate_warp_kernel<false, false, true><<<grid, kWBlock, 0, g0->stream>>>(a);
            else if (ng == 1 && !bits)
                enumerate_warp_kernel<false, true, false><<<grid, kWBlock, 0, g0->stream>>>(a);
            else if (ng == 1)
                enumerate_warp_kernel<false, true, true><<<grid, kWBlock, 0, g0->stream>>>(a);
            else   // a batch has no records
                enumerate_warp_kernel<true, false, false><<<grid, kWBlock, 0, g0->stream>>>(a);
            CK(cudaGetLastError());
            if (pending >= 0 && sink_rc == GMK_OK) {
                sink_rc = deliver_records(g0, outb[pending], pending_words, sink, user);
                pending = -1;
            }
            RoundCounters r;
            CK(cudaMemcpyAsync(&r, g0->d_rc, sizeof(r), cudaMemcpyDeviceToHost, g0->stream));
            CK(cudaMemcpyAsync(&h, launch_ctr, sizeof(h), cudaMemcpyDeviceToHost, g0->stream));
            CK(cudaStreamSynchronize(g0->stream));
            ++rounds;
            tasks_total += a.queue_len;
            tasks_done += std::min<unsigned long long>(r.tasks_done, a.queue_len);
            if (share) {
                ws.dq_dirty = std::max<unsigned long long>(ws.dq_dirty, std::min(r.dq_tail, dq_idx_cap));
                donations += r.donated;
            }
            if (opts->emit) {
                // records end where the first one found no room
                pending = round & 1;
                pending_words = std::min({r.out_pos, (unsigned long long)out_words, r.out_fail});
            }
            const unsigned long long consumed = std::min(r.next_task, a.queue_len);
            if (consumed > n_records) root_next += consumed - n_records;
            if (h.error == gmk::TASK_E_OUTBUF || h.error == gmk::TASK_E_ARENA) {
                static const char* why[] = {"", "unentered root frame", "nothing pending",
                                            "split words full", "split index full",
                                            "a task's base frame cannot hold one child"};
                g_cuda_err = std::string(h.error == gmk::TASK_E_ARENA ? "arena overflow: "
                                                                       : "record deferral failed: ") +
                             why[r.split_refused >= 0 && r.split_refused <= 5 ? r.split_refused : 0];
            }
            if (h.error || h.stop || sink_rc != GMK_OK) break;
            const unsigned long long next = std::min({r.next_count, split_idx_cap, r.next_fail});
            if (next == 0 && root_next >= my_tasks) break;
            if (watchdog_ns) {
                const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                                                host_t0).count();
                if (el * 1e9 > (double)watchdog_ns) { h.error = gmk::TASK_E_TIMEOUT; break; }
            }
            n_records = next;
            cur ^= 1;
        }
        CK(cudaEventRecord(g0->ev1, g0->stream));
        CK(cudaStreamSynchronize(g0->stream));
        if (pending >= 0 && sink_rc == GMK_OK && !h.error)
            sink_rc = deliver_records(g0, outb[pending], pending_words, sink, user);
        if (sink_rc < 0 && sink_rc != GMK_E_SINK) return sink_rc;
        if (sink_rc == GMK_E_SINK) warp_emit_rc = GMK_E_SINK;
        for (size_t i = 0; i < ng; ++i) {
            if (!jobs[i].root_nodes) continue;
            gmk_graph* g = jobs[i].g;
            std::vector<unsigned long long> rn(g->nl);
            CK(cudaMemcpy(rn.data(), g->d_root_nodes, 8ull * g->nl, cudaMemcpyDeviceToHost));
            for (uint32_t v = 0; v < g->nl; ++v) jobs[i].root_nodes[v] += rn[v];
        }
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, g0->ev0, g0->ev1));
    for (size_t i = 0; i < ng; ++i) {
        Counters hc = h;
        if (ng > 1) CK(cudaMemcpy(&hc, jobs[i].g->d_ctr, sizeof(hc), cudaMemcpyDeviceToHost));
        gmk_stats* out = outs + i;
        const unsigned long long cap = ng > 1 ? jobs[i].limit : single_limit;
        out->count = cap ? std::min<unsigned long long>(hc.count, cap) : hc.count;
        out->hash_sum = hc.hash_sum;
        out->hash_xor = hc.hash_xor;
        out->nodes = hc.nodes;
        out->algo_bytes = 4ull * hc.work;
        out->tasks = tasks_total;
        out->tasks_done = tasks_done;
        out->kernel_ms = ms;
        out->truncated = cap && hc.count >= cap;
        out->threads = (uint32_t)threads;
        out->rounds = rounds;
        out->donations = donations;
    }
    switch (h.error) {
        case gmk::TASK_OK: break;
        case gmk::TASK_E_ARENA: return GMK_E_ARENA;
        case gmk::TASK_E_SMAX: return GMK_E_SMAX;
        case gmk::TASK_E_TIMEOUT: return GMK_E_TIMEOUT;
        case gmk::TASK_E_OUTBUF: return GMK_E_OUTBUF;
        case gmk::TASK_E_RECORD:
            g_cuda_err = "a split or donated task record failed its checks (internal error)";
            return GMK_E_CUDA;
        default: return GMK_E_CUDA;
    }
    if (warp) return warp_emit_rc;
    if (opts->emit) {
        if (h.out_pos > out_words) return GMK_E_OUTBUF;
        std::vector<uint32_t> rec(h.out_pos);
        if (h.out_pos)
            CK(cudaMemcpy(rec.data(), ws.d_out, 4ull * h.out_pos, cudaMemcpyDeviceToHost));
        size_t p = 0;
        while (p + 2 <= rec.size()) {
            const uint32_t nx = rec[p], ny = rec[p + 1];
            uint32_t* x = rec.data() + p + 2;
            uint32_t* y = x + nx;
            std::sort(x, x + nx);
            std::sort(y, y + ny);
            if (sink(user, x, nx, y, ny)) return GMK_E_SINK;
            p += 2ull + nx + ny;
        }
    }
    return GMK_OK;
}

int check_opts(const gmk_opts* opts) {
    if (opts->k < 1 || opts->k > 15) return GMK_E_INVAL;
    if (opts->schedule < GMK_SCHEDULE_PLAIN || opts->schedule > GMK_SCHEDULE_ORDERED)
        return GMK_E_INVAL;
    if (opts->nshards && opts->shard >= opts->nshards) return GMK_E_INVAL;
    if (opts->engine != GMK_ENGINE_WARP && opts->engine != GMK_ENGINE_THREAD) return GMK_E_INVAL;
    return GMK_OK;
}

}  // namespace

extern "C" {

int gmk_plan_tasks(uint32_t n, uint32_t n_left, const float* root_cost, uint32_t root_begin,
                   uint32_t root_end, uint64_t target_tasks, uint32_t max_chunks,
                   uint32_t nshards, uint32_t shard, gmk_task* out, uint64_t* n_out) {
    if (!n_out || n_left > n || (!root_cost && n_left) || root_begin > root_end ||
        root_end > n_left || (nshards > 1 && shard >= nshards))
        return GMK_E_INVAL;
    std::vector<uint32_t> roots = select_roots(n_left, root_cost, root_begin, root_end);
    double total = 0;
    for (const uint32_t r : roots) total += std::max<double>(root_cost[r], 0.0);
    std::vector<gmk_task> plan;
    chunk_roots(n_left, n, roots, root_cost, total / (double)std::max<uint64_t>(1, target_tasks),
                max_chunks ? max_chunks : 0xFFFFFFFFu, 0, plan);
    order_and_shard(plan, nshards, shard, true);
    if (out) std::copy(plan.begin(), plan.end(), out);
    *n_out = plan.size();
    return GMK_OK;
}

int gmk_root_costs(gmk_graph* g, float* out) {
    if (!g || !out) return GMK_E_INVAL;
    CK(cudaSetDevice(g->device));
    if (g->nl == 0) return GMK_OK;
    const float* c = nullptr;
    if (int rc = proxy_costs(g, &c)) return rc;
    std::copy(c, c + g->nl, out);
    return GMK_OK;
}

int gmk_enumerate(gmk_graph* g, const gmk_opts* opts, gmk_sink sink, void* user, gmk_stats* out) {
    if (!g || !opts || !out) return GMK_E_INVAL;
    if (int rc = check_opts(opts)) return rc;
    if (opts->emit && !sink) return GMK_E_INVAL;
    if (opts->schedule == GMK_SCHEDULE_ORDERED && !opts->task_cost) return GMK_E_INVAL;
    if (opts->root_nodes && opts->engine != GMK_ENGINE_WARP) return GMK_E_INVAL;
    const uint32_t root_end = opts->root_end ? opts->root_end : g->nl;
    if (root_end > g->nl || opts->root_begin > root_end) return GMK_E_INVAL;
    if (opts->tasks) {
        if (opts->nshards > 1 || opts->root_begin || opts->root_end) return GMK_E_INVAL;
        for (uint64_t i = 0; i < opts->n_tasks; ++i) {
            const gmk_task& t = opts->tasks[i];
            if (t.root >= g->nl || t.first < g->nl || t.first >= t.last || t.last > g->n)
                return GMK_E_INVAL;
        }
    }
    std::memset(out, 0, sizeof(*out));
    CK(cudaSetDevice(g->device));
    if (g->nl == 0 || g->n == g->nl || opts->root_begin == root_end) return GMK_OK;   // nothing to do
    std::vector<GraphJob> jobs{{g, opts->k, 0, opts->root_begin, root_end, opts->task_cost,
                                opts->root_nodes}};
    return run_jobs(jobs, opts, sink, user, out);
}

int gmk_enumerate_batch(gmk_graph* const* graphs, uint32_t n_graphs, const uint32_t* ks,
                        const uint64_t* limits, const float* const* task_costs,
                        const gmk_opts* opts, gmk_stats* outs) {
    if (!graphs || !opts || !outs || n_graphs == 0) return GMK_E_INVAL;
    if (int rc = check_opts(opts)) return rc;
    if (opts->engine != GMK_ENGINE_WARP || opts->emit || opts->result_limit || opts->root_nodes ||
        opts->root_begin || opts->root_end || (opts->nshards > 1) || opts->tasks)
        return GMK_E_INVAL;
    std::memset(outs, 0, sizeof(gmk_stats) * n_graphs);
    std::vector<GraphJob> jobs;
    std::vector<uint32_t> slot;   // jobs[i] is graphs[slot[i]]
    for (uint32_t i = 0; i < n_graphs; ++i) {
        gmk_graph* g = graphs[i];
        if (!g || g->device != graphs[0]->device) return GMK_E_INVAL;
        const uint32_t k = ks ? ks[i] : opts->k;
        if (k < 1 || k > 15) return GMK_E_INVAL;
        if (opts->schedule == GMK_SCHEDULE_ORDERED && (!task_costs || !task_costs[i]))
            return GMK_E_INVAL;
        for (uint32_t j = 0; j < i; ++j)
            if (graphs[j] == g) return GMK_E_INVAL;   // each graph's counters are its own
        if (g->nl == 0 || g->n == g->nl) continue;    // a side is empty: no k-biplex
        jobs.push_back({g, k, limits ? limits[i] : 0ull, 0, g->nl,
                        task_costs ? task_costs[i] : nullptr, nullptr});
        slot.push_back(i);
    }
    if (jobs.empty()) return GMK_OK;
    CK(cudaSetDevice(graphs[0]->device));
    std::vector<gmk_stats> tmp(jobs.size());
    const int rc = run_jobs(jobs, opts, nullptr, nullptr, tmp.data());
    for (size_t i = 0; i < jobs.size(); ++i) outs[slot[i]] = tmp[i];
    return rc;
}

// ---------------------------------------------------------------- learned schedule

struct gmk_mlp {
    int device = 0;
    float* d_master = nullptr;   // FP32 master weights
    __half* d_w = nullptr;       // FP16 working copy
    float* d_m = nullptr;        // Adam moments
    float* d_v = nullptr;
    float* d_grad = nullptr;
    float* d_loss = nullptr;
    uint64_t steps = 0;
    // per-call sample buffers, grown on demand
    __half* d_x = nullptr;
    float* d_xf = nullptr;
    float* d_y = nullptr;
    float* d_act = nullptr;
    float* d_out = nullptr;
    uint32_t cap = 0;
};

namespace {

using gmk::mlp::NP;

int mlp_reserve(gmk_mlp* m, uint32_t n) {
    if (n <= m->cap) return GMK_OK;
    cudaFree(m->d_x); cudaFree(m->d_xf); cudaFree(m->d_y); cudaFree(m->d_act); cudaFree(m->d_out);
    m->d_x = nullptr; m->d_xf = nullptr; m->d_y = nullptr; m->d_act = nullptr; m->d_out = nullptr;
    m->cap = 0;
    const uint64_t nn = n;
    CK(cudaMalloc(&m->d_x, nn * gmk::mlp::F * sizeof(__half)));
    CK(cudaMalloc(&m->d_xf, nn * gmk::mlp::F * sizeof(float)));
    CK(cudaMalloc(&m->d_y, nn * sizeof(float)));
    CK(cudaMalloc(&m->d_act, nn * 2 * gmk::mlp::H * sizeof(float)));
    CK(cudaMalloc(&m->d_out, nn * sizeof(float)));
    m->cap = n;
    return GMK_OK;
}

// Uploads n samples (features rounded to FP16 on the device) and, if y, targets.
int mlp_upload(gmk_mlp* m, const float* x, const float* y, uint32_t n) {
    if (int rc = mlp_reserve(m, n)) return rc;
    const uint64_t nf = (uint64_t)n * gmk::mlp::F;
    CK(cudaMemcpy(m->d_xf, x, nf * sizeof(float), cudaMemcpyHostToDevice));
    gmk::mlp::float_to_half_kernel<<<(unsigned)((nf + 255) / 256), 256>>>(m->d_xf, m->d_x, nf);
    CK(cudaGetLastError());
    if (y) CK(cudaMemcpy(m->d_y, y, (uint64_t)n * sizeof(float), cudaMemcpyHostToDevice));
    return GMK_OK;
}

// Forward + backward of the MSE over n uploaded samples into d_grad / d_loss.
int mlp_grad(gmk_mlp* m, uint32_t n) {
    CK(cudaMemset(m->d_grad, 0, NP * sizeof(float)));
    CK(cudaMemset(m->d_loss, 0, sizeof(float)));
    const unsigned grid = (n + gmk::mlp::kBlock - 1) / gmk::mlp::kBlock;
    gmk::mlp::forward_kernel<<<grid, gmk::mlp::kBlock>>>(m->d_w, m->d_x, n, m->d_act, m->d_out);
    CK(cudaGetLastError());
    gmk::mlp::backward_kernel<<<grid, gmk::mlp::kBlock>>>(m->d_w, m->d_x, m->d_y, m->d_act,
                                                         m->d_out, n, m->d_grad, m->d_loss);
    CK(cudaGetLastError());
    return GMK_OK;
}

}  // namespace

int gmk_root_features(const gmk_graph* g, uint32_t k, float* out) {
    if (!g || !out || k < 1) return GMK_E_INVAL;
    CK(cudaSetDevice(g->device));
    if (g->nl == 0) return GMK_OK;
    gmk_graph* gm = const_cast<gmk_graph*>(g);
    if (!gm->d_feat) CK(pool_alloc(g->device, (void**)&gm->d_feat, feat_bytes(g)));
    gmk::GraphView gv{g->d_off, g->d_adj, g->n, g->nl};
    const uint64_t threads = (uint64_t)g->nl * 32;
    gmk::mlp::root_features_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, g->stream>>>(
        gv, k, gm->d_feat);
    CK(cudaGetLastError());
    std::vector<__half> h((uint64_t)g->nl * gmk::mlp::F);
    CK(cudaMemcpyAsync(h.data(), gm->d_feat, h.size() * sizeof(__half), cudaMemcpyDeviceToHost,
                       g->stream));
    CK(cudaStreamSynchronize(g->stream));
    for (size_t i = 0; i < h.size(); ++i) out[i] = __half2float(h[i]);
    return GMK_OK;
}

int gmk_mlp_create(int device, uint64_t seed, gmk_mlp** out) {
    if (!out) return GMK_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        g_cuda_err = "no CUDA device";
        return GMK_E_NODEV;
    }
    if (device < 0 || device >= ndev) return GMK_E_INVAL;
    CK(cudaSetDevice(device));
    gmk_mlp* m = new (std::nothrow) gmk_mlp();
    if (!m) return GMK_E_NOMEM;
    m->device = device;
    auto bail = [&](int code) { gmk_mlp_free(m); return code; };
    cudaError_t e;
    if ((e = cudaMalloc(&m->d_master, NP * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&m->d_w, NP * sizeof(__half))) != cudaSuccess ||
        (e = cudaMalloc(&m->d_m, NP * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&m->d_v, NP * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&m->d_grad, NP * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&m->d_loss, sizeof(float))) != cudaSuccess)
        return bail(cuda_fail(e, "cudaMalloc(mlp)"));
    // He-uniform initialisation from a splitmix64 stream; biases zero
    std::vector<float> w(NP, 0.f);
    uint64_t st = seed;
    auto uni = [&st]() {
        st += 0x9E3779B97F4A7C15ull;
        return (double)(gmk::mix64(st) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    const int H = gmk::mlp::H, F = gmk::mlp::F;
    for (int i = 0; i < H * F; ++i) w[gmk::mlp::OFF_W1 + i] = (float)(uni() * std::sqrt(6.0 / F));
    for (int i = 0; i < H * H; ++i) w[gmk::mlp::OFF_W2 + i] = (float)(uni() * std::sqrt(6.0 / H));
    for (int i = 0; i < H; ++i) w[gmk::mlp::OFF_W3 + i] = (float)(uni() * std::sqrt(6.0 / H));
    const int rc = gmk_mlp_params(m, nullptr, w.data());
    if (rc) return bail(rc);
    *out = m;
    return GMK_OK;
}

void gmk_mlp_free(gmk_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    cudaFree(m->d_master); cudaFree(m->d_w); cudaFree(m->d_m); cudaFree(m->d_v);
    cudaFree(m->d_grad); cudaFree(m->d_loss);
    cudaFree(m->d_x); cudaFree(m->d_xf); cudaFree(m->d_y); cudaFree(m->d_act); cudaFree(m->d_out);
    delete m;
}

int gmk_mlp_params(gmk_mlp* m, float* get, const float* set) {
    if (!m) return GMK_E_INVAL;
    CK(cudaSetDevice(m->device));
    if (set) {
        CK(cudaMemcpy(m->d_master, set, NP * sizeof(float), cudaMemcpyHostToDevice));
        gmk::mlp::to_half_kernel<<<(NP + 255) / 256, 256>>>(m->d_master, m->d_w);
        CK(cudaGetLastError());
        CK(cudaMemset(m->d_m, 0, NP * sizeof(float)));
        CK(cudaMemset(m->d_v, 0, NP * sizeof(float)));
        m->steps = 0;
    }
    if (get) CK(cudaMemcpy(get, m->d_master, NP * sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaDeviceSynchronize());
    return GMK_OK;
}

int gmk_mlp_gradient(gmk_mlp* m, const float* x, const float* y, uint32_t n, float* grad,
                     float* loss) {
    if (!m || !x || !y || n == 0) return GMK_E_INVAL;
    CK(cudaSetDevice(m->device));
    if (int rc = mlp_upload(m, x, y, n)) return rc;
    if (int rc = mlp_grad(m, n)) return rc;
    if (grad) CK(cudaMemcpy(grad, m->d_grad, NP * sizeof(float), cudaMemcpyDeviceToHost));
    float l = 0.f;
    CK(cudaMemcpy(&l, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return GMK_OK;
}

int gmk_mlp_train(gmk_mlp* m, const float* x, const float* y, uint32_t n, uint32_t epochs,
                  float lr, float* loss) {
    if (!m || !x || !y || n == 0) return GMK_E_INVAL;
    CK(cudaSetDevice(m->device));
    if (int rc = mlp_upload(m, x, y, n)) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        if (int rc = mlp_grad(m, n)) return rc;
        ++m->steps;
        const float c1 = 1.f - std::pow(b1, (float)m->steps);
        const float c2 = 1.f - std::pow(b2, (float)m->steps);
        gmk::mlp::adam_kernel<<<(NP + 255) / 256, 256>>>(m->d_master, m->d_w, m->d_grad, m->d_m,
                                                         m->d_v, lr, b1, b2, eps, c1, c2);
        CK(cudaGetLastError());
    }
    // loss of the final weights
    if (int rc = mlp_grad(m, n)) return rc;
    float l = 0.f;
    CK(cudaMemcpy(&l, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return GMK_OK;
}

int gmk_mlp_predict_roots(gmk_mlp* m, const gmk_graph* g, uint32_t k, float* out) {
    if (!m || !g || !out || k < 1 || m->device != g->device) return GMK_E_INVAL;
    CK(cudaSetDevice(g->device));
    if (g->nl == 0) return GMK_OK;
    gmk_graph* gm = const_cast<gmk_graph*>(g);
    if (!gm->d_feat) CK(pool_alloc(g->device, (void**)&gm->d_feat, feat_bytes(g)));
    if (int rc = mlp_reserve(m, g->nl)) return rc;
    gmk::GraphView gv{g->d_off, g->d_adj, g->n, g->nl};
    const uint64_t threads = (uint64_t)g->nl * 32;
    gmk::mlp::root_features_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, g->stream>>>(
        gv, k, gm->d_feat);
    CK(cudaGetLastError());
    const unsigned grid = (g->nl + gmk::mlp::kBlock - 1) / gmk::mlp::kBlock;
    gmk::mlp::forward_kernel<<<grid, gmk::mlp::kBlock, 0, g->stream>>>(m->d_w, gm->d_feat, g->nl,
                                                                      nullptr, m->d_out);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, m->d_out, 4ull * g->nl, cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return GMK_OK;
}

int gmk_mlp_predict(gmk_mlp* m, const float* x, uint32_t n, float* out) {
    if (!m || !x || !out) return GMK_E_INVAL;
    if (n == 0) return GMK_OK;
    CK(cudaSetDevice(m->device));
    if (int rc = mlp_upload(m, x, nullptr, n)) return rc;
    const unsigned grid = (n + gmk::mlp::kBlock - 1) / gmk::mlp::kBlock;
    gmk::mlp::forward_kernel<<<grid, gmk::mlp::kBlock>>>(m->d_w, m->d_x, n, nullptr, m->d_out);
    CK(cudaGetLastError());
    CK(cudaMemcpy(out, m->d_out, (uint64_t)n * sizeof(float), cudaMemcpyDeviceToHost));
    return GMK_OK;
}

namespace {

// Scratch of gmk_enumerate_noalloc: counters, then the search arenas, then the
// member buffers.  Host code must not use the symbol's host-side shadow as a
// device address; noalloc_scratch() returns the real address per device.
static __device__ __align__(256) unsigned char g_static_scratch[GMK_STATIC_SCRATCH_BYTES];
// Head of the scratch: the counters at 0, the CSR check's words at 128; the
// arenas start at 256.
constexpr uint64_t kNoallocHead = 256;
constexpr uint64_t kNoallocCheck = 128;
static_assert(sizeof(Counters) <= kNoallocCheck, "counters overlap the check words");

std::mutex g_static_mu;
void* g_static_addr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (looked up once).
int noalloc_scratch(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
        g_static_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_static_addr[device]);
    return GMK_OK;
}

}  // namespace

int gmk_enumerate_noalloc(const uint32_t* d_offsets, const uint32_t* d_adj, uint32_t n,
                          uint32_t n_left, uint32_t k, uint64_t result_limit, uint32_t threads,
                          uint32_t arena_words, uint32_t max_members, void* stream,
                          gmk_stats* out) {
    if (!d_offsets || !out || (!d_adj && n > 0) || n_left > n) return GMK_E_INVAL;
    if (k < 1 || k > 15) return GMK_E_INVAL;
    std::memset(out, 0, sizeof(*out));
    // sizes in 64 bits: a thread count near 2^32 must not wrap to a small one
    uint64_t nthreads = threads ? threads : 2048u;
    nthreads = (nthreads + kBlock - 1) / kBlock * kBlock;
    arena_words = arena_words ? arena_words : 4096u;
    max_members = max_members ? max_members : 512u;
    const uint64_t need = kNoallocHead + nthreads * (4ull * arena_words + 8ull * max_members);
    if (need > GMK_STATIC_SCRATCH_BYTES) return GMK_E_SCRATCH;
    threads = (uint32_t)nthreads;
    int device = 0;
    CK(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) return GMK_E_INVAL;
    if (n_left == 0 || n == n_left) return GMK_OK;   // a side is empty: no k-biplex
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(device, &base)) return rc;
    Counters* ctr = reinterpret_cast<Counters*>(base);
    uint32_t* arenas = reinterpret_cast<uint32_t*>(base + kNoallocHead);
    uint32_t* sbuf = arenas + (uint64_t)threads * arena_words;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const auto t0 = std::chrono::steady_clock::now();
    // The caller's CSR is checked on the device before the search reads it as
    // a graph (as gmk_graph_from_csr does): offsets non-decreasing from 0 and
    // within adj, rows ascending, every id on the other side.  The two ends of
    // the offsets come back through plain copies; the check's flag and
    // fingerprint words live in the scratch's head, after the counters.
    {
        uint32_t ends[2] = {1u, 0u};
        CK(cudaMemcpyAsync(&ends[0], d_offsets, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&ends[1], d_offsets + n, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (ends[0] != 0) return GMK_E_FORMAT;
        const unsigned long long adj_len = ends[1];
        if (adj_len && !d_adj) return GMK_E_INVAL;
        struct Check { int bad; int pad; unsigned long long fp; };
        Check* dc = reinterpret_cast<Check*>(base + kNoallocCheck);
        CK(cudaMemsetAsync(dc, 0, sizeof(Check), s));
        const unsigned long long items = std::max<unsigned long long>(n, adj_len);
        if (items) {
            csr_check_kernel<<<(unsigned)((items + 255) / 256), 256, 0, s>>>(
                d_offsets, d_adj, n, n_left, adj_len, &dc->bad, &dc->fp);
            CK(cudaGetLastError());
        }
        int bad = 0;
        CK(cudaMemcpyAsync(&bad, &dc->bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (bad) return GMK_E_FORMAT;
    }
    // tasks: root x with chunks of its first-level children, about 8 per thread
    const uint32_t nv = n - n_left;
    const uint64_t per_root = (8ull * threads + n_left - 1) / n_left;
    uint32_t chunk = (uint32_t)std::max<uint64_t>(16, (nv + per_root - 1) / per_root);
    chunk = std::min(chunk, nv);
    const uint32_t chunks_per_root = (nv + chunk - 1) / chunk;
    const unsigned long long n_tasks = (unsigned long long)n_left * chunks_per_root;
    CK(cudaMemsetAsync(ctr, 0, sizeof(Counters), s));
    gmk::GraphView gv{d_offsets, d_adj, n, n_left};
    enumerate_kernel<<<threads / kBlock, kBlock, 0, s>>>(
        gv, k, ctr, arenas, arena_words, sbuf, max_members, kDefaultPairLimit, n_tasks, chunk,
        chunks_per_root, nullptr, 0u, result_limit, nullptr, 0ull, 0ull);
    CK(cudaGetLastError());
    Counters h;
    CK(cudaMemcpyAsync(&h, ctr, sizeof(h), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out->kernel_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out->count = result_limit ? std::min<unsigned long long>(h.count, result_limit) : h.count;
    out->hash_sum = h.hash_sum;
    out->hash_xor = h.hash_xor;
    out->nodes = h.nodes;
    out->algo_bytes = 4ull * h.work;
    out->tasks = n_tasks;
    out->tasks_done = std::min<unsigned long long>(h.tasks_done, n_tasks);
    out->truncated = result_limit && h.count >= result_limit;
    out->threads = threads;
    out->rounds = 1;
    switch (h.error) {
        case gmk::TASK_OK: return GMK_OK;
        case gmk::TASK_E_ARENA: return GMK_E_ARENA;
        case gmk::TASK_E_SMAX: return GMK_E_SMAX;
        case gmk::TASK_E_TIMEOUT: return GMK_E_TIMEOUT;
        default: return GMK_E_CUDA;
    }
}

namespace {

// Text checkpoint, format 2: besides the graph, k, schedule and root order it
// records the shard and the result limit, so that a checkpoint is resumed only
// by a run over the same task set.
struct Checkpoint {
    uint64_t fingerprint = 0;
    uint32_t k = 0, schedule = 0, next_root = 0, done = 0;
    uint32_t shard = 0, nshards = 1;
    uint64_t limit = 0;
    uint64_t order_hash = 0, count = 0, hash_sum = 0, hash_xor = 0, nodes = 0;
};

bool read_checkpoint(const char* path, Checkpoint& c, bool& exists) {
    FILE* fp = std::fopen(path, "r");
    exists = fp != nullptr;
    if (!fp) return false;
    unsigned long long fpv = 0, oh = 0, cnt = 0, hs = 0, hx = 0, nd = 0, lim = 0;
    unsigned k = 0, sch = 0, nr = 0, dn = 0, sh = 0, nsh = 0;
    const int got = std::fscanf(fp,
                                "gmk-checkpoint 2\ngraph %llx\nk %u\nschedule %u\norder %llx\n"
                                "shard %u\nnshards %u\nresult_limit %llu\n"
                                "next_root %u\ncount %llu\nhash_sum %llx\nhash_xor %llx\n"
                                "nodes %llu\ndone %u\n",
                                &fpv, &k, &sch, &oh, &sh, &nsh, &lim, &nr, &cnt, &hs, &hx, &nd, &dn);
    std::fclose(fp);
    if (got != 13) return false;
    c.fingerprint = fpv; c.k = k; c.schedule = sch; c.order_hash = oh; c.next_root = nr;
    c.shard = sh; c.nshards = nsh; c.limit = lim;
    c.count = cnt; c.hash_sum = hs; c.hash_xor = hx; c.nodes = nd; c.done = dn;
    return true;
}

bool write_checkpoint(const char* path, const Checkpoint& c) {
    const std::string tmp = std::string(path) + ".tmp";
    FILE* fp = std::fopen(tmp.c_str(), "w");
    if (!fp) return false;
    std::fprintf(fp,
                 "gmk-checkpoint 2\ngraph %016llx\nk %u\nschedule %u\norder %016llx\n"
                 "shard %u\nnshards %u\nresult_limit %llu\n"
                 "next_root %u\ncount %llu\nhash_sum %016llx\nhash_xor %016llx\nnodes %llu\n"
                 "done %u\n",
                 (unsigned long long)c.fingerprint, c.k, c.schedule,
                 (unsigned long long)c.order_hash, c.shard, c.nshards,
                 (unsigned long long)c.limit, c.next_root, (unsigned long long)c.count,
                 (unsigned long long)c.hash_sum, (unsigned long long)c.hash_xor,
                 (unsigned long long)c.nodes, c.done);
    const bool ok = std::fflush(fp) == 0;
    std::fclose(fp);
    return ok && std::rename(tmp.c_str(), path) == 0;
}

uint64_t order_hash(const gmk_graph* g, const gmk_opts* o) {
    if ((o->schedule != GMK_SCHEDULE_ORDERED && o->schedule != GMK_SCHEDULE_PLAIN) || !o->task_cost)
        return 0;
    uint64_t h = 0x51ED270B7A3C2D1Full;
    for (uint32_t i = 0; i < g->nl; ++i) {
        uint32_t bits;
        std::memcpy(&bits, o->task_cost + i, 4);
        h = gmk::mix64(h ^ bits);
    }
    return h;
}

}  // namespace

int gmk_enumerate_resumable(gmk_graph* g, const gmk_opts* opts, const char* checkpoint_path,
                            uint32_t batch_roots, uint32_t max_batches, gmk_sink sink,
                            void* user, gmk_stats* out) {
    if (!g || !opts || !out || !checkpoint_path || opts->tasks) return GMK_E_INVAL;
    std::memset(out, 0, sizeof(*out));
    Checkpoint c;
    bool exists = false;
    const uint64_t oh = order_hash(g, opts);
    const uint32_t nsh = opts->nshards > 1 ? opts->nshards : 1u;
    const uint32_t sh = nsh > 1 ? opts->shard : 0u;
    if (read_checkpoint(checkpoint_path, c, exists)) {
        if (c.fingerprint != g->fingerprint || c.k != opts->k ||
            c.schedule != (uint32_t)opts->schedule || c.order_hash != oh || c.next_root > g->nl ||
            c.shard != sh || c.nshards != nsh || c.limit != opts->result_limit)
            return GMK_E_CHECKPOINT;
    } else if (exists) {
        return GMK_E_CHECKPOINT;
    } else {
        c.fingerprint = g->fingerprint;
        c.k = opts->k;
        c.schedule = (uint32_t)opts->schedule;
        c.order_hash = oh;
        c.shard = sh;
        c.nshards = nsh;
        c.limit = opts->result_limit;
    }
    const uint32_t batch = batch_roots ? batch_roots : std::max<uint32_t>(1, (g->nl + 63) / 64);
    uint32_t batches = 0;
    double ms = 0;
    int rc = GMK_OK;
    while (!c.done) {
        const bool limit_hit = opts->result_limit && c.count >= opts->result_limit;
        if (c.next_root >= g->nl || limit_hit) {
            c.done = 1;
            if (!write_checkpoint(checkpoint_path, c)) return GMK_E_IO;
            break;
        }
        if (max_batches && batches >= max_batches) { rc = GMK_PAUSED; break; }
        gmk_opts o = *opts;
        o.root_begin = c.next_root;
        o.root_end = (uint32_t)std::min<uint64_t>(g->nl, (uint64_t)c.next_root + batch);
        o.result_limit = opts->result_limit ? opts->result_limit - c.count : 0;
        gmk_stats st;
        const int r = gmk_enumerate(g, &o, sink, user, &st);
        if (r) return r;
        c.count += st.count;
        c.hash_sum += st.hash_sum;
        c.hash_xor ^= st.hash_xor;
        c.nodes += st.nodes;
        c.next_root = o.root_end;
        ms += st.kernel_ms;
        out->algo_bytes += st.algo_bytes;
        out->tasks += st.tasks;
        out->tasks_done += st.tasks_done;
        out->rounds += st.rounds;
        out->donations += st.donations;
        out->threads = st.threads;
        ++batches;
        if (!write_checkpoint(checkpoint_path, c)) return GMK_E_IO;
    }
    out->count = c.count;
    out->hash_sum = c.hash_sum;
    out->hash_xor = c.hash_xor;
    out->nodes = c.nodes;
    out->kernel_ms = ms;
    out->truncated = opts->result_limit && c.count >= opts->result_limit;
    return rc;
}

}  // extern "C"
