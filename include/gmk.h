/* gmk.h -- C ABI of the B200 maximal k-biplex enumerator (libgmk.so).
 *
 * The reference (GMkBPE) has no library API: its boundary is the `gmkbpe`
 * executable.  Each entry point below replaces one step of that executable so
 * that a host program (C, C++, Python ctypes, Go cgo, ...) can drive the same
 * path without a process boundary.  Plain pointers and sizes only.
 *
 * Graph ids follow the `.graph.bin` numbering: U = [0, n_left), V = [n_left, n).
 * Results are maximal k-biplexes (X in U, Y in V, both non-empty).
 * All functions return GMK_OK (0) or a negative GMK_E* code; gmk_strerror()
 * names it.  A gmk_graph may not be used by two gmk_enumerate calls at once.
 */
#ifndef GMK_H
#define GMK_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GMK_ABI_VERSION 3

enum {
    GMK_OK = 0,
    GMK_E_INVAL = -1,    /* bad argument */
    GMK_E_IO = -2,       /* cannot open / read the file */
    GMK_E_FORMAT = -3,   /* malformed .graph.bin or CSR (ids, sides, unsorted rows) */
    GMK_E_CUDA = -4,     /* CUDA runtime error (message via gmk_last_cuda_error) */
    GMK_E_NOMEM = -5,    /* device allocation failed */
    GMK_E_ARENA = -6,    /* a search task outgrew its arena; raise arena_words */
    GMK_E_SMAX = -7,     /* a k-biplex larger than max_members */
    GMK_E_TIMEOUT = -8,  /* watchdog_ms elapsed; counts cover the work done so far */
    GMK_E_OUTBUF = -9,   /* record buffer too small for emit mode; raise out_words */
    GMK_E_SINK = -10,    /* the sink asked to stop (not an error for the caller's data) */
    GMK_E_NODEV = -11,   /* no CUDA device / extension not usable */
    GMK_E_CHECKPOINT = -12, /* checkpoint file unreadable, or written for another run
                               (graph, k, schedule, order, shard or result limit) */
    GMK_E_SCRATCH = -13, /* gmk_enumerate_noalloc: the request does not fit the static scratch */
    GMK_PAUSED = 1       /* not an error: max_batches reached, the checkpoint holds the rest */
};

typedef struct gmk_graph gmk_graph;

/* Replaces: load_graph_from_bin (reference data/src/tmp_load.h:213-295) plus
 * the CSR upload of testEnumerate (reference src/main.cu:1680-1690).
 * Reads a .graph.bin file and makes the CSR resident on `device`. */
int gmk_graph_load(const char* path, int device, gmk_graph** out);

/* Same, from caller-owned host CSR arrays (copied; the caller keeps them).
 * offsets: n+1 entries; adj: offsets[n] global ids, each row sorted ascending,
 * U rows hold V ids and V rows hold U ids. */
int gmk_graph_from_csr(const uint32_t* offsets, const uint32_t* adj, uint32_t n,
                       uint32_t n_left, int device, gmk_graph** out);

/* Sizes of a loaded graph (any pointer may be NULL): the header fields the
 * reference reads in load_graph_from_bin (data/src/tmp_load.h:213-295). */
int gmk_graph_info(const gmk_graph* g, uint32_t* n, uint32_t* n_left, uint64_t* adj_len);

/* No counterpart in the reference.  64-bit order-dependent hash of the graph's
 * CSR, computed on the device at load; the identity that checkpoints and tuning
 * caches record. */
int gmk_graph_fingerprint(const gmk_graph* g, uint64_t* out);

/* No counterpart in the reference (its membership test is a binary search of
 * sorted rows, include/gpu_utils.cuh:258-282).  Rebuilds the graph's device
 * edge hash -- the membership structure of every adjacency test -- so that at
 * most load_pct percent of its slots hold keys (10..100; 50 at load).  A
 * lower load costs memory and keeps probes inside one 32-byte bucket; a
 * higher one shrinks the table (fewer L2 misses on large graphs).  The
 * autotuner picks it per graph. */
int gmk_graph_set_hash_load(gmk_graph* g, uint32_t load_pct);

/* Releases the graph's device memory (its buffers go to a per-device cache for
 * the next load).  The reference frees its device arrays when the process
 * exits; there is no separate call. */
void gmk_graph_free(gmk_graph* g);

/* Schedules of the search tasks (one task = a root U vertex and a chunk of its
 * first-level children). */
enum {
    GMK_SCHEDULE_PLAIN = 0,    /* one task per root, roots in id order (largest task_cost
                                  first when one is given), no splitting */
    GMK_SCHEDULE_BATCHED = 1,  /* roots split into chunks, persistent work queue; unfinished
                                  search trees are split into the next round's tasks */
    GMK_SCHEDULE_ORDERED = 2   /* batched over planned tasks: roots split into chunks in
                                  proportion to a caller-given cost (task_cost, e.g. the
                                  subtree-size model's prediction); largest first for a
                                  complete run (balance); under a result limit in root id
                                  order, as PLAIN (the cost predicts nodes, not how soon
                                  results come) */
};

/* Search engines (same rules, same result set). */
enum {
    GMK_ENGINE_WARP = 0,       /* one task per warp, lanes share each node's work (default) */
    GMK_ENGINE_THREAD = 1      /* one task per thread, no splitting */
};

typedef struct {
    uint32_t k;               /* -k: misses allowed per vertex (>= 1) */
    uint64_t result_limit;    /* -r: stop after this many results; 0 = enumerate all */
    int32_t schedule;         /* GMK_SCHEDULE_* */
    int32_t emit;             /* 0: count + set hash only; 1: also deliver every result to the sink */
    uint32_t chunk;           /* first-level children per task (batched); 0 = automatic */
    uint32_t threads;         /* resident search threads; 0 = automatic */
    uint32_t arena_words;     /* per-thread search arena (u32 words); 0 = automatic */
    uint32_t max_members;     /* largest |X|+|Y| a task may hold; 0 = the bound
                                 (max U degree + max V degree + 2k + 2, at least 2048)
                                 for the warp engine, 2048 for the thread engine */
    uint32_t watchdog_ms;     /* stop with GMK_E_TIMEOUT after this long; 0 = none */
    uint64_t out_words;       /* emit-mode record buffer (u32 words); 0 = automatic */
    const float* task_cost;   /* one cost per root U vertex (n_left): required by
                                 GMK_SCHEDULE_ORDERED; orders the roots of a PLAIN run */
    uint32_t pair_limit;      /* node rules (shortcut, forcing, exclusion prune) run while
                                 (|S|+|C_U|)*(|S|+|C_V|) <= pair_limit; 0 = 4096 */
    uint32_t shard, nshards;  /* one GPU of several: run only this shard's tasks of the
                                 longest-processing-time partition of gmk_plan_tasks (costs:
                                 task_cost, else gmk_root_costs); nshards 0 or 1 = all */
    int32_t engine;           /* GMK_ENGINE_* */
    uint32_t split_min_nodes; /* warp engine, batched/ordered: a task is split only after this
                                 many nodes; 0 = 64 */
    uint32_t root_begin;      /* only roots at positions [root_begin, root_end) of the root
                                 order (id order, or cost order for ORDERED); the ranges of */
    uint32_t root_end;        /* consecutive calls partition the result set; root_end 0 = all.
                                 Used for checkpoint / resume. */
    uint64_t* root_nodes;     /* optional, warp engine: host array of n_left counters; the
                                 search nodes of each root's tasks are added to its entry
                                 (the subtree sizes the learned schedule trains on) */
    uint32_t donate_min_nodes; /* warp engine, batched/ordered, emit = 0: in-launch work
                                 sharing -- a busy task that has run this many nodes gives the
                                 shallowest unexplored part of its tree to an idle warp;
                                 0 = 16 */
    int32_t no_sharing;       /* 1: no in-launch sharing (unfinished trees only split into the
                                 next launch, as emit = 1 runs do) */
    const struct gmk_task_* tasks; /* optional explicit task list (gmk_task, e.g. from
                                 gmk_plan_tasks): run exactly these tasks in this order,
                                 instead of planning; needs nshards <= 1, no root range,
                                 and one graph.  Used to re-run a failed rank's shard. */
    uint64_t n_tasks;         /* entries of tasks */
    uint32_t tasks_per_worker; /* batched / ordered: root tasks planned per warp; 0 = 8 */
    uint32_t bits_min_list;   /* warp engine, k >= 2: the intersection strategy by list length --
                                 a branching node's candidate lists of at least this many entries
                                 get filter bitmaps (bit tests), shorter ones are filtered by
                                 edge-hash probes; 0 = 64, 0xFFFFFFFF = probes only */
} gmk_opts;

typedef struct {
    uint64_t count;           /* results (clamped to result_limit) */
    uint64_t hash_sum;        /* wrapping sum of per-result h1 */
    uint64_t hash_xor;        /* xor of per-result h2.  Both hashes describe the result set
                                 only when truncated == 0.  A count-only run (emit = 0) that a
                                 result_limit stopped counts results in batches per worker, so
                                 its hashes may include results past the limit and are not a
                                 summary of any particular `count` results; emit = 1 runs hash
                                 exactly the delivered results. */
    uint64_t nodes;           /* search-tree nodes */
    uint64_t algo_bytes;      /* adjacency/counter bytes the search read (4 per word) */
    uint64_t tasks;           /* search tasks in the queue */
    uint64_t tasks_done;      /* tasks taken from the queue */
    double kernel_ms;         /* device time of the enumeration kernel (CUDA events) */
    int32_t truncated;        /* 1 if result_limit stopped the search */
    uint32_t threads;         /* search threads used */
    uint32_t rounds;          /* kernel launches (rounds of split tasks) */
    uint64_t donations;       /* search-tree pieces handed to idle warps inside launches */
} gmk_stats;

/* Called from the calling thread after the kernel finished, once per result;
 * x and y hold global ids sorted ascending.  Return non-zero to stop. */
typedef int (*gmk_sink)(void* user, const uint32_t* x, uint32_t nx, const uint32_t* y,
                        uint32_t ny);

/* Fills *o with the defaults: k = 1 as the reference's -k (src/main.cu:1722-1732),
 * no result limit (the gmk CLI applies the reference's -r default of 10^7), the
 * batched schedule and the warp engine. */
void gmk_opts_default(gmk_opts* o);

/* Replaces: enumerate_GPU (reference src/main.cu:999-1580) with everything it
 * calls -- Generate_GPU (include/for_generate.cuh:300-512), ListBFS2_GPU
 * (include/for_BFS.cuh:463-777), Special_GPU (include/for_special.cuh:274-683)
 * and the CheckMaximality family (include/for_checkmaximality.cuh) -- and the
 * result printer (include/output.cuh:93-150) when emit = 1.
 * Enumerates the maximal k-biplexes of g on its device. */
int gmk_enumerate(gmk_graph* g, const gmk_opts* opts, gmk_sink sink, void* user,
                  gmk_stats* out);

/* No counterpart in the reference (one graph per gmkbpe process).  Enumerates
 * n_graphs graphs, all loaded on the same device, in one run of persistent
 * launches: the root tasks of every graph share one device work queue, so
 * many small or uneven graphs keep the GPU busy together.  ks[i] is graph i's
 * k (NULL: opts->k for all); limits[i] is graph i's result cap (NULL or 0: all
 * of its results) -- a graph that reaches its cap stops alone, the others go
 * on; with GMK_SCHEDULE_ORDERED, task_costs[i] gives graph i's per-root costs.
 * opts must have emit = 0, result_limit = 0, no root range, no root_nodes, no
 * sharding, no task list, and the warp engine.  outs[i] receives graph i's
 * count (clamped to its cap, truncated set when reached) and set hash (a set
 * summary only when not truncated); kernel_ms, rounds and tasks are those of
 * the whole batch.  A graph may appear only once. */
int gmk_enumerate_batch(gmk_graph* const* graphs, uint32_t n_graphs, const uint32_t* ks,
                        const uint64_t* limits, const float* const* task_costs,
                        const gmk_opts* opts, gmk_stats* outs);

/* No counterpart in the reference, which has no resume (its "checkpoints" are
 * result-count milestones, src/main.cu:1753-1761).  Runs gmk_enumerate over
 * consecutive batches of `batch_roots` roots (0 = automatic) and, after each
 * batch, atomically rewrites `checkpoint_path` with the next root position
 * and the running count and set hash.  If the file exists when the call
 * starts, the run resumes from it (it must have been written for the same
 * graph, k, schedule, root order, shard and result limit; else
 * GMK_E_CHECKPOINT).  Results of finished batches
 * are not delivered again.  With max_batches > 0 the call returns GMK_PAUSED
 * after that many batches if work remains.  *out holds the totals of the
 * whole run, resumed part included; a finished run leaves the file marked
 * done. */
int gmk_enumerate_resumable(gmk_graph* g, const gmk_opts* opts, const char* checkpoint_path,
                            uint32_t batch_roots, uint32_t max_batches, gmk_sink sink,
                            void* user, gmk_stats* out);

/* No counterpart in the reference.  An entry point for callers that must not
 * allocate device memory: code running where cudaMalloc is unavailable or
 * forbidden (inside a host allocator's own callbacks, under an external memory
 * pool that owns all device memory, in a process that has pinned its device
 * footprint before the search starts).  The caller passes the graph as device
 * CSR arrays it owns (d_offsets: n+1 words, d_adj: d_offsets[n] words, rows
 * sorted, U rows hold V ids and vice versa) and receives the counts and set
 * hash in *out.  The CSR is checked on the device first (offsets from 0,
 * non-decreasing and within d_offsets[n]; rows ascending; ids on the other
 * side): a malformed one returns GMK_E_FORMAT before the search reads it.
 * d_adj must really hold d_offsets[n] words; that cannot be checked.
 * The search runs the one-task-per-thread engine with the batched schedule
 * (no tree splitting); its arenas, member buffers and counters live in one
 * static device array of GMK_STATIC_SCRATCH_BYTES that every GPU loading
 * libgmk.so holds until the process exits.  The call itself allocates
 * nothing: no cudaMalloc, no cudaFree, no events.
 *   threads:     search threads (0 = 2048), a multiple of 128 is used;
 *   arena_words: per-thread search arena in u32 words (0 = 4096);
 *   max_members: largest |X|+|Y| (0 = 512).
 * threads x (4 arena_words + 8 max_members) bytes plus 256 for the counters must
 * fit GMK_STATIC_SCRATCH_BYTES, else GMK_E_SCRATCH.  A search that outgrows its
 * arena returns GMK_E_ARENA (gmk_enumerate would split the task instead).
 * Set-up: the first call on a device looks up the array's device address
 * (once per device, with that device made current).  Under CUDA's lazy module
 * loading that first call may also be what loads libgmk's device code and so
 * creates the array: make one call at initialisation (a warm-up on a tiny
 * graph), before entering the code that must not allocate, and before any
 * stream capture begins.  The call runs on `stream` (a cudaStream_t, NULL =
 * the legacy default stream) and returns after the search finished.  All calls
 * on a device share the one array, which keeps the last call's contents; each
 * call clears the counters it needs.  Calls that overlap on the GPU (from
 * several host threads or streams) race on the array and must be serialised by
 * the caller.  out->kernel_ms is host wall time of the check, launch and wait. */
#define GMK_STATIC_SCRATCH_BYTES (64u << 20)
int gmk_enumerate_noalloc(const uint32_t* d_offsets, const uint32_t* d_adj, uint32_t n,
                          uint32_t n_left, uint32_t k, uint64_t result_limit, uint32_t threads,
                          uint32_t arena_words, uint32_t max_members, void* stream,
                          gmk_stats* out);

/* ---- learned schedule: subtree-size model (no counterpart in the reference)
 * A 16-64-64-1 ReLU perceptron with FP16 weights and inputs and FP32
 * accumulation, trained and run on the GPU by the library's own kernels.  It
 * predicts log1p(search nodes) of each root task from 16 integer-derived
 * features; GMK_SCHEDULE_ORDERED then starts the largest predicted roots
 * first.  It orders work only and never prunes. */
typedef struct gmk_mlp gmk_mlp;
#define GMK_MLP_FEATURES 16
#define GMK_MLP_PARAMS 5313   /* W1[64][16] b1[64] W2[64][64] b2[64] W3[64] b3 */

/* The 16 features of every root x in U (n_left x 16 floats, row-major), computed
 * on the graph's device and rounded to FP16 as the model reads them. */
int gmk_root_features(const gmk_graph* g, uint32_t k, float* out);

/* A model on `device` with He-uniform weights drawn from `seed`. */
int gmk_mlp_create(int device, uint64_t seed, gmk_mlp** out);
void gmk_mlp_free(gmk_mlp* m);
/* Copies the FP32 master weights out (get != NULL) and/or in (set != NULL). */
int gmk_mlp_params(gmk_mlp* m, float* get, const float* set);
/* Mean squared error of n samples and its gradient (GMK_MLP_PARAMS floats),
 * without updating the weights. */
int gmk_mlp_gradient(gmk_mlp* m, const float* x, const float* y, uint32_t n, float* grad,
                     float* loss);
/* `epochs` full-batch Adam steps on (x, y); *loss receives the last loss. */
int gmk_mlp_train(gmk_mlp* m, const float* x, const float* y, uint32_t n, uint32_t epochs,
                  float lr, float* loss);
int gmk_mlp_predict(gmk_mlp* m, const float* x, uint32_t n, float* out);
/* The model's prediction for every root x in U of g (n_left floats): the
 * features and the forward pass both run on the device, on the graph's stream,
 * with no host round trip in between; the same values as gmk_root_features
 * followed by gmk_mlp_predict.  m and g must be on the same device. */
int gmk_mlp_predict_roots(gmk_mlp* m, const gmk_graph* g, uint32_t k, float* out);

/* ---- task planning (no counterpart in the reference, whose host loop takes the
 * top-level vertices one at a time in id order, src/main.cu:1078-1111) */

/* One search task: root x (a U vertex) with the first-level V children
 * [first, last) of its search -- the maximal k-biplexes whose smallest U
 * vertex is x and whose smallest V vertex lies in [first, last). */
typedef struct gmk_task_ {
    uint32_t root, first, last;
    uint32_t graph;           /* index of the graph in a batch (0 for one graph) */
    float cost;               /* predicted cost of the task */
} gmk_task;

/* Cost proxy of every root task (n_left floats): 1 + sum over the root's
 * neighbours y of |N(y) above x| -- the U vertices that can join x through a
 * common neighbour.  Computed on the graph's device once and cached. */
int gmk_root_costs(gmk_graph* g, float* out);

/* Host-only planner, the one the ordered schedule and sharding use.  The roots
 * at positions [root_begin, root_end) of the cost order (largest first, ties
 * by id) are each split into ceil(cost / unit) chunks of their first-level V
 * children (unit = total cost / target_tasks; at most max_chunks per root,
 * chunks at least 16 children wide), ordered by per-task cost (largest first)
 * and, with nshards > 1, assigned to shards by longest processing time (each
 * task to the least-loaded shard, lowest index on ties).  Writes this shard's
 * tasks to out (NULL: count only) and their number to *n_out; out must hold
 * *n_out entries from a counting call with the same arguments. */
int gmk_plan_tasks(uint32_t n, uint32_t n_left, const float* root_cost, uint32_t root_begin,
                   uint32_t root_end, uint64_t target_tasks, uint32_t max_chunks,
                   uint32_t nshards, uint32_t shard, gmk_task* out, uint64_t* n_out);

/* No counterpart in the reference.  Canonical per-result hash pair (the set
 * summary's h1/h2): ids are the global ids of X u Y in any order, nx = |X|,
 * ny = |Y|.  Host-only. */
void gmk_result_hash(const uint32_t* ids, uint32_t n_ids, uint32_t nx, uint32_t ny,
                     uint64_t* h1, uint64_t* h2);

/* Replace CUDA_ERROR_CHECK's message-and-exit(1) (include/utils.h:42-49): the
 * name of a GMK_E* code, and the text of the last CUDA failure on this thread. */
const char* gmk_strerror(int code);
const char* gmk_last_cuda_error(void);
/* No counterpart in the reference: GMK_ABI_VERSION of the loaded library. */
int gmk_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GMK_H */
