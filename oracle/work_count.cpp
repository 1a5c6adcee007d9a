// Algorithmic bytes of an enumeration -- TEST / MEASUREMENT INFRASTRUCTURE.
//
// Runs the per-thread restatement of the search (gmkbe_b200/csrc/enum_core.cuh,
// compiled for the host) over every root task in id order, one task per root
// (the plain schedule), and counts the adjacency words it reads: every element
// of a CSR row it scans, and for every membership test by binary search the
// row's two offset words, the other row's two and one word per probe step
// (row_contains).  The count is fixed per (graph, k, result limit): it does not
// depend on the GPU's schedule, chunking or tree splitting, so bench.py can use
// 4 x words / results as the bytes one result costs (the roofline's
// algorithmic bytes).  The product never runs this file.
//
//   work_count <file.graph.bin> <k> [result_limit] [--per-root]
// prints one JSON line: results, nodes, adjacency_words, algo_bytes (and with
// --per-root the search nodes of every root task, "root_nodes").
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../gmkbe_b200/csrc/enum_core.cuh"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: work_count <file.graph.bin> <k> [result_limit]\n");
        return 2;
    }
    const unsigned k = (unsigned)std::strtoul(argv[2], nullptr, 10);
    const unsigned long long limit = argc > 3 ? std::strtoull(argv[3], nullptr, 10) : 0ull;
    const bool per_root = argc > 4 && std::string(argv[4]) == "--per-root";
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) { std::perror(argv[1]); return 1; }
    std::vector<uint32_t> w;
    uint32_t buf[1 << 14];
    size_t got;
    while ((got = std::fread(buf, 4, sizeof(buf) / 4, fp)) > 0) w.insert(w.end(), buf, buf + got);
    std::fclose(fp);
    if (w.size() < 3) return 1;
    const uint32_t n = w[1], nl = w[2];
    std::vector<uint32_t> off(n + 1ull, 0), adj;
    size_t pos = 3;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t d = w[pos + 1];
        pos += 2;
        adj.insert(adj.end(), w.begin() + pos, w.begin() + pos + d);
        pos += d;
        off[i + 1] = (uint32_t)adj.size();
    }
    if (adj.empty()) adj.push_back(0);

    unsigned long long count = 0, hsum = 0, hxor = 0, nodes = 0, work = 0;
    int stop = 0, error = 0;
    unsigned long long out_pos = 0;
    gmk::Outputs o{};
    o.count = &count; o.hash_sum = &hsum; o.hash_xor = &hxor; o.nodes = &nodes; o.work = &work;
    o.stop = &stop; o.error = &error; o.limit = limit; o.out_buf = nullptr; o.out_pos = &out_pos;
    o.out_cap = 0; o.deadline_ns = 0; o.out_fail = nullptr;

    // members are bounded by the degree bound of a k-biplex
    uint32_t maxd[2] = {0, 0};
    for (uint32_t v = 0; v < n; ++v) {
        const uint32_t d = off[v + 1] - off[v];
        uint32_t& m = maxd[v < nl ? 0 : 1];
        m = d > m ? d : m;
    }
    const uint32_t smax = maxd[0] + maxd[1] + 2 * k + 2;
    uint32_t cap = 1u << 22;
    std::vector<uint32_t> arena(cap), sid(smax), smc(smax);
    gmk::Task t{};
    t.g = gmk::GraphView{off.data(), adj.data(), n, nl};
    t.k = k;
    t.arena = arena.data(); t.cap = cap;
    t.sid = sid.data(); t.smc = smc.data(); t.smax = smax;
    t.scan_limit = 4096;
    std::vector<unsigned long long> root_nodes(nl, 0);
    for (uint32_t root = 0; root < nl && !stop; ++root) {
        const unsigned long long before = nodes + t.nodes;
        gmk::run_task(t, o, root, nl, n);
        root_nodes[root] = nodes + t.nodes - before;
        gmk::flush(t, o);
        if (t.err) { std::fprintf(stderr, "task error %d at root %u\n", t.err, root); return 1; }
    }
    gmk::flush(t, o);
    std::printf("{\"results\": %llu, \"nodes\": %llu, \"adjacency_words\": %llu, "
                "\"algo_bytes\": %llu, \"hash_sum\": \"%016llx\", \"hash_xor\": \"%016llx\", "
                "\"k\": %u, \"result_limit\": %llu",
                count, nodes, work, 4ull * work, hsum, hxor, k, limit);
    if (per_root) {
        std::printf(", \"root_nodes\": [");
        for (uint32_t r = 0; r < nl; ++r) std::printf(r ? ", %llu" : "%llu", root_nodes[r]);
        std::printf("]");
    }
    std::printf("}\n");
    return 0;
}
