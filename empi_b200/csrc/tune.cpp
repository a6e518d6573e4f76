// Tuned launch shapes: the cache file written by empi_b200/autotune.py and
// read by the engine (empi_engine_opts.tune_cache).
//
// The file is JSON: {"version": 1, "entries": [{...}, ...]} where each entry
// holds the key of a workload -- "mode" (0 single-channel loops: SMP and
// MMP2's channel sum, 1 MMP1, 3 MMP3), "channels" (per MP loop), "fs",
// "samples", "energy_error" -- and the tuned shape: "transform_cap" (largest
// shared-memory sub-FFT), "iterations_per_graph" and "wide_mask" (bit lg set:
// the refresh kernel of sub-FFT size 2^lg runs one 128-register CTA per SM
// instead of two 64-register ones), optionally "persistent" (1: the MP loop
// runs as one persistent kernel per chunk of iterations, 0: as the CUDA graph).  Other keys (timings, the GPU's name) are
// ignored.  The reader below accepts exactly this flat shape: objects of
// string keys and number or string values inside one array.
#include "tune.hpp"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

namespace empi {

namespace {

struct Cursor {
    const std::string& s;
    size_t i = 0;
    explicit Cursor(const std::string& str) : s(str) {}
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
    bool string(std::string& out) {
        ws();
        if (i >= s.size() || s[i] != '"') return false;
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            if (s[i] == '\\' && i + 1 < s.size()) ++i;
            out += s[i++];
        }
        if (i >= s.size()) return false;
        ++i;
        return true;
    }
    bool number(double& v) {
        ws();
        const char* b = s.c_str() + i;
        char* e = nullptr;
        v = std::strtod(b, &e);
        if (e == b) return false;
        i += (size_t)(e - b);
        return true;
    }
    // skips any value (used for keys this reader does not need)
    bool skip() {
        ws();
        if (i >= s.size()) return false;
        std::string tmp;
        double d;
        if (s[i] == '"') return string(tmp);
        if (s[i] == '{' || s[i] == '[') {
            const char open = s[i], close = open == '{' ? '}' : ']';
            int depth = 0;
            for (; i < s.size(); ++i) {
                if (s[i] == '"') {
                    if (!string(tmp)) return false;
                    --i;
                } else if (s[i] == open) {
                    ++depth;
                } else if (s[i] == close && --depth == 0) {
                    ++i;
                    return true;
                }
            }
            return false;
        }
        if (s.compare(i, 4, "true") == 0 || s.compare(i, 4, "null") == 0) {
            i += 4;
            return true;
        }
        if (s.compare(i, 5, "false") == 0) {
            i += 5;
            return true;
        }
        return number(d);
    }
};

// one {"key": number, ...} object; string values are skipped
bool read_object(Cursor& c, std::map<std::string, double>& kv) {
    if (!c.eat('{')) return false;
    if (c.eat('}')) return true;
    for (;;) {
        std::string k;
        if (!c.string(k) || !c.eat(':')) return false;
        c.ws();
        double v;
        if (c.i < c.s.size() && (c.s[c.i] == '-' || std::isdigit((unsigned char)c.s[c.i]))) {
            if (!c.number(v)) return false;
            kv[k] = v;
        } else if (!c.skip()) {
            return false;
        }
        if (c.eat('}')) return true;
        if (!c.eat(',')) return false;
    }
}

bool same(double a, double b) { return std::fabs(a - b) <= 1e-9 * std::max(1.0, std::fabs(b)); }

}  // namespace

bool tune_lookup(const char* path, const TuneKey& key, TuneParams& out, std::string& err) {
    std::ifstream f(path);
    if (!f) {
        err = "couldNotOpenTuneCache";
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    Cursor c(text);
    if (!c.eat('{')) {
        err = "invalidTuneCache";
        return false;
    }
    bool found = false;
    for (;;) {
        std::string k;
        if (!c.string(k) || !c.eat(':')) {
            err = "invalidTuneCache";
            return false;
        }
        if (k == "entries") {
            if (!c.eat('[')) {
                err = "invalidTuneCache";
                return false;
            }
            if (!c.eat(']')) {
                for (;;) {
                    std::map<std::string, double> kv;
                    if (!read_object(c, kv)) {
                        err = "invalidTuneCache";
                        return false;
                    }
                    if (!found && kv.count("mode") && kv.count("channels") && kv.count("fs") &&
                        kv.count("samples") && kv.count("energy_error") && (int)kv["mode"] == key.mode &&
                        (int)kv["channels"] == key.channels && same(kv["fs"], key.fs) &&
                        (int)kv["samples"] == key.samples && same(kv["energy_error"], key.energy_error)) {
                        out = TuneParams{};
                        if (kv.count("transform_cap")) out.transform_cap = (int)kv["transform_cap"];
                        if (kv.count("iterations_per_graph")) out.iterations_per_graph = (int)kv["iterations_per_graph"];
                        if (kv.count("wide_mask")) out.wide_mask = (int)kv["wide_mask"];
                        if (kv.count("persistent")) out.persistent = kv["persistent"] != 0.0 ? 1 : 0;
                        found = true;
                    }
                    if (c.eat(']')) break;
                    if (!c.eat(',')) {
                        err = "invalidTuneCache";
                        return false;
                    }
                }
            }
        } else if (!c.skip()) {
            err = "invalidTuneCache";
            return false;
        }
        if (c.eat('}')) break;
        if (!c.eat(',')) {
            err = "invalidTuneCache";
            return false;
        }
    }
    if (!found) err = "noTunedEntry";
    return found;
}

}  // namespace empi
