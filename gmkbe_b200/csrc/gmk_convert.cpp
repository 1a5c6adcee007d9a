// gmk-convert: text edge list -> .graph.bin, multi-threaded, byte-identical to
// the reference's converter (preprocess/graph_conver.cpp, `graph_convert -i
// <edges> -o <prefix|file.graph.bin>`).
//
// Input rules (the reference scanner, graph_conver.cpp:433-441 and :529-549):
// blank characters (\n \r space \t) are skipped; a line whose first character
// is % or # is a comment; otherwise the next two runs of decimal digits are an
// edge (u, v), each taken modulo 2^32 -- the second run may lie on a later line
// when a line holds only one -- and the rest of the line holding the second
// run is ignored.  Output rules (graph_conver.cpp:566-810): ids are compacted
// per side in numeric order, parallel edges dropped, and each side ordered by
// (log32 bucket of d', d', compact id) with d' = deg - 2 on the left and
// deg - 1 on the right in wrapping 32-bit arithmetic.  The bucket is a
// non-decreasing function of d', so that order is simply (d', compact id).
//
// One input form is read differently by the reference depending on its thread
// count: a record whose second number sits on a later line is cut at the end
// of the reference's OpenMP chunk (its scanner stops at the chunk end and reads
// 0).  Here records are read whole at any thread count, which equals the
// reference run with one thread.
//
// Pipeline: parse chunks of the file in parallel (a record that crosses a
// chunk boundary is repaired by re-parsing the next chunk from the first
// record start the previous chunk reaches), compact the ids by a rank table
// (or a parallel sort for sparse id ranges), drop parallel edges with a
// parallel LSD radix sort of (u, v) keys, order each side with a second radix
// sort of (d', id) keys, scatter the CSR rows and write the file from a
// buffer filled in parallel.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

using u32 = uint32_t;
using u64 = uint64_t;

int g_threads = 1;
size_t g_min_chunk = 1 << 16;   // bytes of input per parsing thread, at least

template <class F>
void parallel_for(size_t n, F f) {
    // f(begin, end, thread)
    const int T = (int)std::min<size_t>(std::max(1, g_threads), std::max<size_t>(n, 1));
    if (T <= 1) { f((size_t)0, n, 0); return; }
    std::vector<std::thread> th;
    const size_t step = (n + T - 1) / T;
    for (int t = 0; t < T; ++t) {
        const size_t b = std::min(n, (size_t)t * step), e = std::min(n, b + step);
        th.emplace_back([=]() { f(b, e, t); });
    }
    for (auto& x : th) x.join();
}

inline bool is_blank(char c) { return c == '\n' || c == '\r' || c == ' ' || c == '\t'; }
inline bool is_digit(char c) { return c >= '0' && c <= '9'; }

struct Parsed {
    std::vector<u32> u, v;
    std::vector<size_t> start;   // byte offset where each record begins
    size_t stop = 0;             // first record start at or after the chunk end
};

// Parses records that start in [p, end) of data[0, n); a record that begins
// before `end` is read to completion even past it.
void parse_from(const char* data, size_t n, size_t p, size_t end, Parsed& out) {
    out.u.clear(); out.v.clear(); out.start.clear();
    while (p < n) {
        const char c = data[p];
        if (is_blank(c)) { ++p; continue; }
        if (p >= end) break;
        if (c == '%' || c == '#') {
            const void* nl = std::memchr(data + p, '\n', n - p);
            p = nl ? (size_t)((const char*)nl - data) : n;
            continue;
        }
        const size_t rec = p;
        u32 vals[2] = {0, 0};
        for (int i = 0; i < 2; ++i) {
            while (p < n && !is_digit(data[p])) ++p;
            u32 x = 0;
            while (p < n && is_digit(data[p])) { x = x * 10u + (u32)(data[p] - '0'); ++p; }
            vals[i] = x;
        }
        out.start.push_back(rec);
        out.u.push_back(vals[0]);
        out.v.push_back(vals[1]);
        const void* nl = p < n ? std::memchr(data + p, '\n', n - p) : nullptr;
        p = nl ? (size_t)((const char*)nl - data) : n;
    }
    out.stop = p < n ? p : n;
}

// Parallel parse with boundary repair; returns all records in file order.
void parse_all(const char* data, size_t n, std::vector<u32>& U, std::vector<u32>& V) {
    const int T = std::max(1, std::min<int>(g_threads, (int)(n / std::max<size_t>(1, g_min_chunk)) + 1));
    std::vector<size_t> cut(T + 1, n);
    cut[0] = 0;
    for (int t = 1; t < T; ++t) {
        // chunk starts just after a newline (a line start)
        size_t p = n * (size_t)t / T;
        const void* nl = std::memchr(data + p, '\n', n - p);
        cut[t] = nl ? (size_t)((const char*)nl - data) + 1 : n;
        if (cut[t] < cut[t - 1]) cut[t] = cut[t - 1];
    }
    std::vector<Parsed> part(T);
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t)
        th.emplace_back([&, t]() { parse_from(data, n, cut[t], cut[t + 1], part[t]); });
    for (auto& x : th) x.join();
    // repair: chunk t must continue exactly where chunk t-1 stopped
    for (int t = 1; t < T; ++t) {
        const size_t want = part[t - 1].stop;
        Parsed& q = part[t];
        if (want == cut[t]) continue;
        auto it = std::lower_bound(q.start.begin(), q.start.end(), want);
        if (it != q.start.end() && *it == want) {
            const size_t drop = (size_t)(it - q.start.begin());
            q.u.erase(q.u.begin(), q.u.begin() + drop);
            q.v.erase(q.v.begin(), q.v.begin() + drop);
            q.start.erase(q.start.begin(), q.start.begin() + drop);
        } else {
            // a record crossed the boundary in a way this chunk's guess missed
            parse_from(data, n, want, std::max(want, cut[t + 1]), q);
        }
    }
    size_t total = 0;
    for (auto& q : part) total += q.u.size();
    U.resize(total);
    V.resize(total);
    size_t at = 0;
    for (auto& q : part) {
        std::copy(q.u.begin(), q.u.end(), U.begin() + at);
        std::copy(q.v.begin(), q.v.end(), V.begin() + at);
        at += q.u.size();
    }
}

}  // namespace

namespace {

// Parallel LSD radix sort of 64-bit keys on their low `bits` bits (8 per pass).
void radix_sort(std::vector<u64>& a, int bits) {
    std::vector<u64> b(a.size());
    const size_t n = a.size();
    const int T = std::max(1, std::min<int>(g_threads, (int)(n / 4096) + 1));
    std::vector<size_t> hist((size_t)T * 256);
    for (int shift = 0; shift < bits; shift += 8) {
        std::fill(hist.begin(), hist.end(), 0);
        const size_t step = (n + T - 1) / T;
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t]() {
                const size_t lo = std::min(n, (size_t)t * step), hi = std::min(n, lo + step);
                size_t* h = hist.data() + (size_t)t * 256;
                for (size_t i = lo; i < hi; ++i) ++h[(a[i] >> shift) & 255u];
            });
        for (auto& x : th) x.join();
        th.clear();
        // bucket-major, thread-minor prefix: a stable scatter
        size_t sum = 0;
        for (int d = 0; d < 256; ++d)
            for (int t = 0; t < T; ++t) {
                const size_t c = hist[(size_t)t * 256 + d];
                hist[(size_t)t * 256 + d] = sum;
                sum += c;
            }
        for (int t = 0; t < T; ++t)
            th.emplace_back([&, t]() {
                const size_t lo = std::min(n, (size_t)t * step), hi = std::min(n, lo + step);
                size_t* h = hist.data() + (size_t)t * 256;
                for (size_t i = lo; i < hi; ++i) b[h[(a[i] >> shift) & 255u]++] = a[i];
            });
        for (auto& x : th) x.join();
        a.swap(b);
    }
}

int bits_for(u64 maxv) {
    int b = 0;
    while (b < 64 && (maxv >> b)) ++b;
    return (b + 7) / 8 * 8;
}

// Ranks of ids among the distinct values of x (x replaced by its rank);
// returns the number of distinct values.
u32 compact(std::vector<u32>& x) {
    u32 mx = 0;
    for (const u32 v : x) mx = v > mx ? v : mx;
    const size_t n = x.size();
    if ((u64)mx <= 4ull * n + (1ull << 20)) {
        // dense id range: presence table, prefix sum, lookup
        std::vector<u32> rank((size_t)mx + 2, 0);
        for (size_t i = 0; i < n; ++i) rank[x[i]] = 1;
        u32 r = 0;
        for (size_t i = 0; i <= mx; ++i) {
            const u32 here = rank[i];
            rank[i] = r;
            r += here;
        }
        parallel_for(n, [&](size_t b, size_t e, int) {
            for (size_t i = b; i < e; ++i) x[i] = rank[x[i]];
        });
        return r;
    }
    std::vector<u64> keys(n);
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t i = b; i < e; ++i) keys[i] = x[i];
    });
    radix_sort(keys, 32);
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t i = b; i < e; ++i)
            x[i] = (u32)(std::lower_bound(keys.begin(), keys.end(), (u64)x[i]) - keys.begin());
    });
    return (u32)keys.size();
}

// New ids of one side: positions in (d', compact id) order, d' = deg - sub
// in wrapping 32-bit arithmetic; `base` is added (0 for U, |U| for V).
std::vector<u32> side_order(const std::vector<u32>& deg, u32 sub, u32 base) {
    const size_t n = deg.size();
    std::vector<u64> keys(n);
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t i = b; i < e; ++i) keys[i] = ((u64)(u32)(deg[i] - sub) << 32) | (u64)i;
    });
    radix_sort(keys, 64);
    std::vector<u32> newid(n);
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t p = b; p < e; ++p) newid[(u32)keys[p]] = base + (u32)p;
    });
    return newid;
}

}  // namespace

namespace {

bool ends_with(const std::string& s, const char* suf) {
    const size_t n = std::strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

double secs_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int convert(const std::string& in, std::string out, bool timing) {
    const auto t0 = std::chrono::steady_clock::now();
    FILE* fp = std::fopen(in.c_str(), "rb");
    if (!fp) { std::perror(in.c_str()); return 1; }
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    std::vector<char> data(sz > 0 ? (size_t)sz : 1);
    if (sz > 0 && std::fread(data.data(), 1, (size_t)sz, fp) != (size_t)sz) {
        std::fclose(fp);
        std::fprintf(stderr, "%s: short read\n", in.c_str());
        return 1;
    }
    std::fclose(fp);
    const double t_read = secs_since(t0);
    std::vector<u32> U, V;
    parse_all(data.data(), sz > 0 ? (size_t)sz : 0, U, V);
    data.clear();
    data.shrink_to_fit();
    const double t_parse = secs_since(t0);
    const size_t m = U.size();
    const u32 nl = m ? compact(U) : 0, nr = m ? compact(V) : 0;
    // parallel edges: sort (u, v) keys and drop repeats
    std::vector<u64> key(m);
    parallel_for(m, [&](size_t b, size_t e, int) {
        for (size_t i = b; i < e; ++i) key[i] = ((u64)U[i] << 32) | V[i];
    });
    U.clear(); U.shrink_to_fit();
    V.clear(); V.shrink_to_fit();
    radix_sort(key, 32 + bits_for(nl ? nl - 1 : 0));
    key.erase(std::unique(key.begin(), key.end()), key.end());
    const size_t me = key.size();
    const double t_dedup = secs_since(t0);
    std::vector<u32> degl(nl, 0), degr(nr, 0);
    for (size_t i = 0; i < me; ++i) {
        ++degl[(u32)(key[i] >> 32)];
        ++degr[(u32)key[i]];
    }
    const std::vector<u32> newl = side_order(degl, 2u, 0u);
    const std::vector<u32> newr = side_order(degr, 1u, nl);
    const u32 n = nl + nr;
    // CSR in new ids: offsets from the degrees, rows filled then sorted
    std::vector<u64> off((size_t)n + 1, 0);
    for (u32 x = 0; x < nl; ++x) off[(size_t)newl[x] + 1] = degl[x];
    for (u32 y = 0; y < nr; ++y) off[(size_t)newr[y] + 1] = degr[y];
    for (size_t i = 0; i < n; ++i) off[i + 1] += off[i];
    std::vector<u32> adj(2 * me);
    {
        std::vector<u64> cur(off.begin(), off.end() - 1);
        for (size_t i = 0; i < me; ++i) {
            const u32 a = newl[(u32)(key[i] >> 32)], b = newr[(u32)key[i]];
            adj[cur[a]++] = b;
            adj[cur[b]++] = a;
        }
    }
    key.clear(); key.shrink_to_fit();
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t v = b; v < e; ++v) std::sort(adj.begin() + off[v], adj.begin() + off[v + 1]);
    });
    const double t_csr = secs_since(t0);
    // file: 2|E|, N, |U|, then per vertex: id, degree, neighbours
    const size_t words = 3 + 2 * (size_t)n + adj.size();
    std::vector<u32> buf(words);
    buf[0] = (u32)adj.size();
    buf[1] = n;
    buf[2] = nl;
    parallel_for(n, [&](size_t b, size_t e, int) {
        for (size_t v = b; v < e; ++v) {
            u32* w = buf.data() + 3 + 2 * v + off[v];
            w[0] = (u32)v;
            w[1] = (u32)(off[v + 1] - off[v]);
            std::memcpy(w + 2, adj.data() + off[v], 4 * (off[v + 1] - off[v]));
        }
    });
    if (!ends_with(out, ".graph.bin")) out += ".graph.bin";
    FILE* fo = std::fopen(out.c_str(), "wb");
    if (!fo) { std::perror(out.c_str()); return 1; }
    const bool ok = std::fwrite(buf.data(), 4, words, fo) == words;
    if (std::fclose(fo) != 0 || !ok) { std::fprintf(stderr, "%s: write failed\n", out.c_str()); return 1; }
    if (timing)
        std::fprintf(stderr,
                     "gmk-convert: %zu records, |U| %u |V| %u |E| %zu, %d threads; read %.3f s, "
                     "parse %.3f, compact+dedup %.3f, order+csr %.3f, total %.3f s\n",
                     m, nl, nr, me, g_threads, t_read, t_parse - t_read, t_dedup - t_parse,
                     t_csr - t_dedup, secs_since(t0));
    std::printf("%s\n", out.c_str());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    std::string in, out;
    bool timing = false;
    g_threads = (int)std::max(1u, std::thread::hardware_concurrency());
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "missing value for %s\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "-i") in = val();
        else if (a == "-o") out = val();
        else if (a == "-t" || a == "--threads") g_threads = std::max(1, std::atoi(val().c_str()));
        else if (a == "--timing") timing = true;
        else if (a == "--min-chunk") g_min_chunk = (size_t)std::strtoull(val().c_str(), nullptr, 10);
        else {
            std::fprintf(stderr, "usage: gmk-convert -i <edges> -o <prefix|file.graph.bin> "
                                 "[--threads N] [--timing]\n");
            return a == "-h" || a == "--help" ? 0 : 2;
        }
    }
    if (in.empty() || out.empty()) {
        std::fprintf(stderr, "usage: gmk-convert -i <edges> -o <prefix|file.graph.bin>\n");
        return 2;
    }
    return convert(in, out, timing);
}
