// gmk: drop-in command line for the reference's `gmkbpe` executable.
//
// Same flags as reference src/main.cu:1719-1775:
//   -f <file.graph.bin>  -k <k> (default 1)  -r <result limit> (default 1e7)
//   -q <print results, 0/1> (default 0)  -d <device> (default 0)
//   -m / -g are accepted and ignored (verbose dump / unused group size).
// Output: "Using GPU: <name>, GPU id: <d>", the "Graph size: ..." header,
// "Result N: X: x1 x2 | Y: y1 y2 " lines when -q 1 (format of reference
// include/output.cuh:102-145), then "Running Time: <ms> ms".
// Progress as the reference reports it (src/main.cu:1752-1760,
// include/output.cuh:350-372): "Output <n>, cost Time: <ms> ms" on stderr when
// the result count reaches 10^i or the limit (every one with -q 1; the final
// one in count mode, which has no per-result host step), and the time to the
// limit kept in <dir>/<stem>.gpu<k>.json as {"<k>": {"<limit>": ms}}
// (include/timer.cuh:85-185: merged into an existing file, 5 h written until
// the limit is reached).  The file is named for the graph given with -f (the
// reference takes the first .bin of its directory).
// Extra: --all (no result limit), --schedule plain|batched, --stats,
// --threads N / --arena WORDS (resident search threads, per-worker arena),
// --engine warp|thread, --checkpoint FILE [--batch-roots N] (resumable run:
// the file is rewritten after every batch of roots and a restarted command
// continues from it), --no-time-file.
#include <cctype>
#include <charconv>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gmk.h"
#include "time_file.h"

using gmk_cli::TimeTable;
using gmk_cli::read_time_table;
using gmk_cli::time_file_path;
using gmk_cli::write_time_table;

namespace {

// Result lines in the reference's format (include/output.cuh:102-145):
// "Result <n>: X: x1 x2 | Y: y1 y2 \n" -- X ids joined by single spaces, each Y
// id followed by one.  Lines are formatted into a 4 MiB buffer and written
// with fwrite when it fills (one printf per id measured 4-5x slower).
struct Printer {
    unsigned long long n = 0;
    std::vector<char> buf = std::vector<char>(4u << 20);
    size_t len = 0;
    FILE* out = stdout;
    // progress: the next count to report (10^i, then the limit), the limit
    // (0: none), the run's start and the time at which the limit was reached
    unsigned long long next_mark = 1, limit = 0;
    std::chrono::steady_clock::time_point t0;
    double limit_ms = -1.0;

    void flush() {
        if (len) std::fwrite(buf.data(), 1, len, out);
        len = 0;
    }
    char* room(size_t need) {
        if (len + need > buf.size()) flush();
        if (need > buf.size()) buf.resize(need);
        return buf.data() + len;
    }
    static char* put_u64(char* p, unsigned long long v) {
        return std::to_chars(p, p + 24, v).ptr;
    }
};

int print_result(void* user, const uint32_t* x, uint32_t nx, const uint32_t* y, uint32_t ny) {
    Printer* pr = static_cast<Printer*>(user);
    // at most 11 bytes per id, 40 for the fixed text and the counter
    char* p = pr->room(64 + 11ull * (nx + ny));
    char* const start = p;
    std::memcpy(p, "Result ", 7);
    p = Printer::put_u64(p + 7, ++pr->n);
    std::memcpy(p, ": X:", 4);
    p += 4;
    for (uint32_t i = 0; i < nx; ++i) {
        *p++ = ' ';
        p = Printer::put_u64(p, x[i]);
    }
    std::memcpy(p, " | Y: ", 6);
    p += 6;
    for (uint32_t i = 0; i < ny; ++i) {
        p = Printer::put_u64(p, y[i]);
        *p++ = ' ';
    }
    *p++ = '\n';
    pr->len += (size_t)(p - start);
    if (pr->n == pr->next_mark) {
        // a progress mark: results so far go out first, as the reference's
        // writer flushes at each mark
        pr->flush();
        std::fflush(pr->out);
        const double ms = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - pr->t0).count();
        std::fprintf(stderr, "Output %llu, cost Time: %g ms\n", pr->n, ms);
        if (pr->n == pr->limit) pr->limit_ms = ms;
        const unsigned long long next = pr->next_mark * 10;
        pr->next_mark = pr->limit && next >= pr->limit ? pr->limit : next;
        if (pr->limit && pr->n >= pr->limit) pr->next_mark = 0;   // nothing after the limit
    }
    return 0;
}

void usage() {
    std::fprintf(stderr,
                 "usage: gmk -f <graph.bin> [-k K] [-r LIMIT] [-q 0|1] [-d DEV] [--all]\n"
                 "           [--schedule plain|batched] [--stats] [--threads N] [--arena WORDS]\n"
                 "           [--engine warp|thread] [--checkpoint FILE [--batch-roots N]]\n"
                 "           [--no-time-file]\n");
}

}  // namespace

int main(int argc, char** argv) {
    std::string file;
    gmk_opts o;
    gmk_opts_default(&o);
    o.result_limit = 10000000ull;
    int quiet = 0, dev = 0, stats = 0, time_file = 1;
    std::string checkpoint;
    uint32_t batch_roots = 0;
    for (int i = 1; i < argc; ++i) {
        auto val = [&](const char* name) -> const char* {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", name); std::exit(2); }
            return argv[++i];
        };
        if (!std::strcmp(argv[i], "-f")) file = val("-f");
        else if (!std::strcmp(argv[i], "-k")) o.k = (uint32_t)std::strtoul(val("-k"), nullptr, 10);
        else if (!std::strcmp(argv[i], "-r")) o.result_limit = std::strtoull(val("-r"), nullptr, 10);
        else if (!std::strcmp(argv[i], "-q")) quiet = std::atoi(val("-q"));
        else if (!std::strcmp(argv[i], "-d")) dev = std::atoi(val("-d"));
        else if (!std::strcmp(argv[i], "-m") || !std::strcmp(argv[i], "-g")) (void)val(argv[i]);
        else if (!std::strcmp(argv[i], "--all")) o.result_limit = 0;
        else if (!std::strcmp(argv[i], "--stats")) stats = 1;
        else if (!std::strcmp(argv[i], "--no-time-file")) time_file = 0;
        else if (!std::strcmp(argv[i], "--threads"))
            o.threads = (uint32_t)std::strtoul(val("--threads"), nullptr, 10);
        else if (!std::strcmp(argv[i], "--checkpoint")) checkpoint = val("--checkpoint");
        else if (!std::strcmp(argv[i], "--batch-roots"))
            batch_roots = (uint32_t)std::strtoul(val("--batch-roots"), nullptr, 10);
        else if (!std::strcmp(argv[i], "--engine"))
            o.engine = !std::strcmp(val("--engine"), "thread") ? GMK_ENGINE_THREAD : GMK_ENGINE_WARP;
        else if (!std::strcmp(argv[i], "--arena"))
            o.arena_words = (uint32_t)std::strtoul(val("--arena"), nullptr, 10);
        else if (!std::strcmp(argv[i], "--schedule")) {
            const char* s = val("--schedule");
            o.schedule = !std::strcmp(s, "plain") ? GMK_SCHEDULE_PLAIN : GMK_SCHEDULE_BATCHED;
            if (std::strcmp(s, "plain") && std::strcmp(s, "batched")) { usage(); return 2; }
        } else if (!std::strcmp(argv[i], "-h") || !std::strcmp(argv[i], "--help")) {
            usage();
            return 0;
        } else {
            usage();
            return 2;
        }
    }
    if (file.empty()) { usage(); return 2; }
    // the reference's first line (src/main.cu:1766-1770)
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
        std::printf("Using GPU: %s, GPU id: %d\n", prop.name, dev);
        std::fflush(stdout);
    }
    gmk_graph* g = nullptr;
    int rc = gmk_graph_load(file.c_str(), dev, &g);
    if (rc) {
        std::fprintf(stderr, "gmk: %s (%s)\n", gmk_strerror(rc), gmk_last_cuda_error());
        return 1;
    }
    uint32_t n = 0, nl = 0;
    uint64_t m = 0;
    gmk_graph_info(g, &n, &nl, &m);
    // the reference's header line (src/main.cu:1593-1595; its theta is fixed to 1)
    std::printf("Graph size: %u, edge num: %llu, bipartite index: %u, k = %u, theta = 1\n", n,
                (unsigned long long)m, nl, o.k);
    std::fflush(stdout);
    // the time file holds 5 h for this (k, limit) until the limit is reached
    const std::string limit_key = std::to_string(o.result_limit);
    const std::string tpath = time_file_path(file, o.k);
    TimeTable table;
    if (time_file && o.result_limit) {
        table = read_time_table(tpath);
        table[std::to_string(o.k)][limit_key] = "18000000";
        write_time_table(tpath, table);
    }
    Printer p;
    p.limit = o.result_limit;
    p.next_mark = o.result_limit && o.result_limit <= 1 ? o.result_limit : 1;
    o.emit = quiet ? 1 : 0;
    gmk_stats st;
    const auto t0 = std::chrono::steady_clock::now();
    p.t0 = t0;
    // results stream through the library's record buffers; no retry is needed
    rc = checkpoint.empty() ? gmk_enumerate(g, &o, quiet ? print_result : nullptr, &p, &st)
                            : gmk_enumerate_resumable(g, &o, checkpoint.c_str(), batch_roots, 0,
                                                      quiet ? print_result : nullptr, &p, &st);
    p.flush();
    std::fflush(stdout);
    const double wall_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (rc) {
        std::fprintf(stderr, "gmk: %s (%s)\n", gmk_strerror(rc), gmk_last_cuda_error());
        gmk_graph_free(g);
        return 1;
    }
    // the double in its shortest round-trip form, as the reference's fmt prints it
    // (src/main.cu:1709)
    if (!quiet && st.count) {
        // count mode: the final mark only (no host step per result)
        std::fprintf(stderr, "Output %llu, cost Time: %g ms\n", (unsigned long long)st.count, wall_ms);
        if (o.result_limit && st.count >= o.result_limit) p.limit_ms = wall_ms;
    }
    if (time_file && o.result_limit && p.limit_ms >= 0) {
        char v[64];
        *std::to_chars(v, v + sizeof(v) - 1, p.limit_ms).ptr = 0;
        table[std::to_string(o.k)][limit_key] = v;
        write_time_table(tpath, table);
    }
    char ms[64];
    *std::to_chars(ms, ms + sizeof(ms) - 1, st.kernel_ms).ptr = 0;
    std::printf("Running Time: %s ms\n", ms);
    if (stats)
        std::printf("results %llu hash_sum %016llx hash_xor %016llx nodes %llu tasks %llu threads %u "
                    "rounds %u lines %llu wall_ms %.3f lines_per_s %.0f\n",
                    (unsigned long long)st.count, (unsigned long long)st.hash_sum,
                    (unsigned long long)st.hash_xor, (unsigned long long)st.nodes,
                    (unsigned long long)st.tasks, st.threads, st.rounds, p.n, wall_ms,
                    wall_ms > 0 ? p.n / (wall_ms / 1e3) : 0.0);
    gmk_graph_free(g);
    return 0;
}
