// The reference's time file, <dir>/<stem>.gpu<k>.json (include/timer.cuh:85-185):
// a JSON object of objects of numbers, {"<k>": {"<limit>": ms}}.  Read
// leniently (anything unreadable starts an empty object, as the reference
// does); written with four-space indents and keys in string order.  Host-only
// C++17, used by the gmk CLI (and compiled alone by its CPU test).
#pragma once
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

namespace gmk_cli {

using TimeTable = std::map<std::string, std::map<std::string, std::string>>;

inline bool parse_string(const std::string& s, size_t& i, std::string& out) {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    if (i >= s.size() || s[i] != '"') return false;
    const size_t j = s.find('"', i + 1);
    if (j == std::string::npos) return false;
    out = s.substr(i + 1, j - i - 1);
    i = j + 1;
    return true;
}

inline bool expect(const std::string& s, size_t& i, char c) {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    if (i >= s.size() || s[i] != c) return false;
    ++i;
    return true;
}

inline bool peek(const std::string& s, size_t& i, char c) {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    return i < s.size() && s[i] == c;
}

inline TimeTable read_time_table(const std::string& path) {
    TimeTable t;
    std::ifstream f(path);
    if (!f) return t;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string s = ss.str();
    size_t i = 0;
    TimeTable parsed;
    if (!expect(s, i, '{')) return t;
    while (!peek(s, i, '}')) {
        std::string k;
        if (!parse_string(s, i, k) || !expect(s, i, ':') || !expect(s, i, '{')) return t;
        auto& row = parsed[k];
        while (!peek(s, i, '}')) {
            std::string key;
            if (!parse_string(s, i, key) || !expect(s, i, ':')) return t;
            while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
            const size_t b = i;
            while (i < s.size() && (std::isdigit((unsigned char)s[i]) || std::strchr("+-.eE", s[i]))) ++i;
            if (i == b) return t;
            row[key] = s.substr(b, i - b);
            if (!peek(s, i, '}') && !expect(s, i, ',')) return t;
        }
        ++i;
        if (!peek(s, i, '}') && !expect(s, i, ',')) return t;
    }
    return parsed;
}

inline void write_time_table(const std::string& path, const TimeTable& t) {
    std::ofstream f(path);
    if (!f) {
        std::fprintf(stderr, "Error: Cannot write to file: %s\n", path.c_str());
        return;
    }
    f << "{";
    bool first = true;
    for (const auto& [k, row] : t) {
        f << (first ? "\n" : ",\n") << "    \"" << k << "\": {";
        bool first2 = true;
        for (const auto& [key, v] : row) {
            f << (first2 ? "\n" : ",\n") << "        \"" << key << "\": " << v;
            first2 = false;
        }
        f << (row.empty() ? "}" : "\n    }");
        first = false;
    }
    f << (t.empty() ? "}" : "\n}");
}

// <dir>/<stem>.gpu<k>.json for the graph file `graph`.
inline std::string time_file_path(const std::string& graph, uint32_t k) {
    const size_t slash = graph.find_last_of('/');
    const std::string dir = slash == std::string::npos ? "" : graph.substr(0, slash + 1);
    std::string stem = slash == std::string::npos ? graph : graph.substr(slash + 1);
    const size_t dot = stem.find_last_of('.');
    if (dot != std::string::npos && dot > 0) stem = stem.substr(0, dot);
    return dir + stem + ".gpu" + std::to_string(k) + ".json";
}

}  // namespace gmk_cli
