// Cache of autotuner results (pcx_plan_tune), keyed by GPU name, transform
// size, element type and batch (rows, bucketed by powers of two), stored as a
// small JSON file:
//
//   {"version": 1, "entries": [
//     {"gpu": "NVIDIA B200", "n": 1048576, "dtype": "f32", "batch_log2": 7,
//      "form": 2, "rounds": 3, "chunk_bytes": 0,
//      "split": [10, 10], "blocks_per_sm": 1, "stages": 2, "ms": 0.1234}, ...]}
//
// Host code only: loading, saving and lookups need no GPU.
#include "pcx_host.hpp"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct entry {
    std::string     gpu;
    size_t          n          = 0;
    int             dtype      = PCX_F32;
    int             batch_log2 = 0;
    pcx_tune_result r{};
};

std::mutex         g_mu;
std::vector<entry> g_entries;

int bucket(size_t batch) {
    int b = 0;
    while (batch > 1) {
        batch >>= 1;
        ++b;
    }
    return b;
}

// ---- a reader for the flat JSON this file writes ----------------------------
struct reader {
    const std::string& s;
    size_t             i = 0;
    bool               ok = true;

    void ws() {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
    }
    bool eat(char c) {
        ws();
        if (i < s.size() && s[i] == c) {
            ++i;
            return true;
        }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) ok = false;
    }
    std::string str() {
        ws();
        std::string out;
        if (!eat('"')) {
            ok = false;
            return out;
        }
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) ++i;
            out += s[i++];
        }
        if (i >= s.size()) ok = false;
        ++i;
        return out;
    }
    double num() {
        ws();
        const char* b = s.c_str() + i;
        char*       e = nullptr;
        const double v = std::strtod(b, &e);
        if (e == b) ok = false;
        i += (size_t)(e - b);
        return v;
    }
    // skips any value (used for unknown keys)
    void skip() {
        ws();
        if (i >= s.size()) {
            ok = false;
            return;
        }
        if (s[i] == '"') {
            str();
        } else if (s[i] == '[' || s[i] == '{') {
            const char open = s[i], close = open == '[' ? ']' : '}';
            int        depth = 0;
            do {
                if (s[i] == '"') {
                    str();
                    continue;
                }
                if (s[i] == open) ++depth;
                if (s[i] == close) --depth;
                ++i;
            } while (i < s.size() && depth > 0);
        } else {
            num();
        }
    }
};

bool parse_entry(reader& rd, entry& e) {
    rd.expect('{');
    bool first = true;
    while (rd.ok && !rd.eat('}')) {
        if (!first) rd.expect(',');
        first = false;
        const std::string k = rd.str();
        rd.expect(':');
        if (k == "gpu") {
            e.gpu = rd.str();
        } else if (k == "n") {
            e.n = (size_t)rd.num();
        } else if (k == "dtype") {
            e.dtype = rd.str() == "f64" ? PCX_F64 : PCX_F32;
        } else if (k == "batch_log2") {
            e.batch_log2 = (int)rd.num();
        } else if (k == "form") {
            e.r.form = (int)rd.num();
        } else if (k == "rounds") {
            e.r.rounds = (int)rd.num();
        } else if (k == "chunk_bytes") {
            e.r.chunk_bytes = (size_t)rd.num();
        } else if (k == "split") {
            rd.expect('[');
            e.r.log_n1 = (int)rd.num();
            rd.expect(',');
            e.r.log_n2 = (int)rd.num();
            rd.expect(']');
        } else if (k == "blocks_per_sm") {
            e.r.blocks_per_sm = (int)rd.num();
        } else if (k == "stages") {
            e.r.stages = (int)rd.num();
        } else if (k == "ms") {
            e.r.ms = rd.num();
        } else {
            rd.skip();
        }
    }
    return rd.ok;
}

std::string escape(const std::string& s) {
    std::string o;
    for (char c: s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

}    // namespace

extern "C" int pcx_tune_cache_clear(void) {
    std::lock_guard<std::mutex> g(g_mu);
    g_entries.clear();
    return PCX_OK;
}

extern "C" size_t pcx_tune_cache_size(void) {
    std::lock_guard<std::mutex> g(g_mu);
    return g_entries.size();
}

extern "C" int pcx_tune_cache_put(const char* gpu, size_t n, int dtype, size_t batch, const pcx_tune_result* r) {
    return pcx_guard([&]() -> int {
        if (!gpu || !r) return pcx_fail(PCX_ERR_INVALID, "null argument");
        std::lock_guard<std::mutex> g(g_mu);
        const int                   b = bucket(batch);
        for (auto& e: g_entries) {
            if (e.gpu == gpu && e.n == n && e.dtype == dtype && e.batch_log2 == b) {
                e.r = *r;
                return PCX_OK;
            }
        }
        g_entries.push_back({gpu, n, dtype, b, *r});
        return PCX_OK;
    });
}

extern "C" int pcx_tune_cache_get(const char* gpu, size_t n, int dtype, size_t batch, pcx_tune_result* r) {
    return pcx_guard([&]() -> int {
        if (!gpu || !r) return pcx_fail(PCX_ERR_INVALID, "null argument");
        std::lock_guard<std::mutex> g(g_mu);
        const int                   b = bucket(batch);
        for (const auto& e: g_entries) {
            if (e.gpu == gpu && e.n == n && e.dtype == dtype && e.batch_log2 == b) {
                *r = e.r;
                return PCX_OK;
            }
        }
        return pcx_fail(PCX_ERR_INVALID, "no cached tuning for this GPU, size, type and batch");
    });
}

extern "C" int pcx_tune_cache_save(const char* path) {
    return pcx_guard([&]() -> int {
        if (!path) return pcx_fail(PCX_ERR_INVALID, "null path");
        std::ostringstream o;
        {
            std::lock_guard<std::mutex> g(g_mu);
            o << "{\"version\": 1, \"entries\": [";
            for (size_t i = 0; i < g_entries.size(); ++i) {
                const entry& e = g_entries[i];
                char         ms[64];
                std::snprintf(ms, sizeof ms, "%.6g", e.r.ms);
                o << (i ? ",\n  " : "\n  ") << "{\"gpu\": \"" << escape(e.gpu) << "\", \"n\": " << e.n
                  << ", \"dtype\": \"" << (e.dtype == PCX_F64 ? "f64" : "f32") << "\", \"batch_log2\": " << e.batch_log2
                  << ", \"form\": " << e.r.form << ", \"rounds\": " << e.r.rounds
                  << ", \"chunk_bytes\": " << e.r.chunk_bytes << ", \"split\": [" << e.r.log_n1 << ", " << e.r.log_n2
                  << "], \"blocks_per_sm\": " << e.r.blocks_per_sm << ", \"stages\": " << e.r.stages
                  << ", \"ms\": " << ms << "}";
            }
            o << "\n]}\n";
        }
        const std::string tmp = std::string(path) + ".tmp";
        {
            std::ofstream f(tmp, std::ios::trunc);
            if (!f) return pcx_fail(PCX_ERR_INVALID, std::string("cannot write ") + tmp);
            f << o.str();
            if (!f) return pcx_fail(PCX_ERR_INVALID, std::string("cannot write ") + tmp);
        }
        if (std::rename(tmp.c_str(), path) != 0) return pcx_fail(PCX_ERR_INVALID, std::string("cannot replace ") + path);
        return PCX_OK;
    });
}

extern "C" int pcx_tune_cache_load(const char* path) {
    return pcx_guard([&]() -> int {
        if (!path) return pcx_fail(PCX_ERR_INVALID, "null path");
        std::ifstream f(path);
        if (!f) return pcx_fail(PCX_ERR_INVALID, std::string("cannot read ") + path);
        std::stringstream ss;
        ss << f.rdbuf();
        const std::string text = ss.str();
        reader            rd{text};
        std::vector<entry> got;
        rd.expect('{');
        bool first = true;
        while (rd.ok && !rd.eat('}')) {
            if (!first) rd.expect(',');
            first = false;
            const std::string k = rd.str();
            rd.expect(':');
            if (k == "entries") {
                rd.expect('[');
                bool f2 = true;
                while (rd.ok && !rd.eat(']')) {
                    if (!f2) rd.expect(',');
                    f2 = false;
                    entry e;
                    if (parse_entry(rd, e)) got.push_back(e);
                }
            } else {
                rd.skip();
            }
        }
        if (!rd.ok) return pcx_fail(PCX_ERR_INVALID, std::string("malformed tuning cache ") + path);
        for (const entry& e: got) {
            if (int rc = pcx_tune_cache_put(e.gpu.c_str(), e.n, e.dtype, (size_t)1 << e.batch_log2, &e.r)) return rc;
        }
        return PCX_OK;
    });
}
