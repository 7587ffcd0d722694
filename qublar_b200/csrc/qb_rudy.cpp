// Reader of rudy / G-set graph text, the input format of the reference's
// integer engine (parse_rudy, src/ising_weighted.hpp:83-149): a header "n m",
// then m lines "u v [w]" with 1-based vertices and w = +1 when absent. The
// same inputs are refused for the same reasons: a bad header, a token that is
// not an integer (a real weight belongs to the float path), a weight outside
// int32, a trailing token on an edge line, a vertex out of range, a self-loop,
// an edge count that differs from the header, a duplicate edge in either
// orientation. Host code only.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "qb_internal.hpp"

struct qb_graph {
    int32_t n = 0;
    std::vector<int32_t> eu, ev, ew;
};

namespace {

// The text as lines of tokens separated by blanks (space, tab, CR).
struct Reader {
    const char* p;
    const char* end;
    static bool blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }
    void skip_blanks() {
        while (p < end && blank(*p)) ++p;
    }
    void skip_space() {
        while (p < end && (blank(*p) || *p == '\n')) ++p;
    }
    bool line_done() {
        skip_blanks();
        return p >= end || *p == '\n';
    }
    // Next token of the current line into [s, e); false at the end of the line.
    bool next(const char** s, const char** e) {
        skip_blanks();
        if (p >= end || *p == '\n') return false;
        *s = p;
        while (p < end && !blank(*p) && *p != '\n') ++p;
        *e = p;
        return true;
    }
};

// Optional sign, then decimal digits; magnitudes above 2^40 are refused.
bool to_int(const char* s, const char* e, int64_t* v) {
    if (s == e) return false;
    bool neg = false;
    if (*s == '-' || *s == '+') {
        neg = *s == '-';
        ++s;
    }
    if (s == e) return false;
    int64_t acc = 0;
    for (; s < e; ++s) {
        if (*s < '0' || *s > '9') return false;
        acc = acc * 10 + (*s - '0');
        if (acc > (int64_t(1) << 40)) return false;
    }
    *v = neg ? -acc : acc;
    return true;
}

}  // namespace

extern "C" qb_status qb_parse_rudy(const char* text, size_t size, qb_graph** out) {
    return qb::guarded("qb_parse_rudy", [&]() -> qb_status {
        using qb::fail;
        if (!out || (!text && size > 0)) return fail(QB_EINVAL, "qb_parse_rudy: null argument");
        *out = nullptr;
        Reader r{text, text + size};
        const char *s = nullptr, *e = nullptr;
        int64_t n = 0, m = 0;
        r.skip_space();
        if (!r.next(&s, &e) || !to_int(s, e, &n) || n <= 0 || n > (int64_t(1) << 30))
            return fail(QB_EINVAL, "bad header: n");
        if (!r.next(&s, &e) || !to_int(s, e, &m) || m < 0) return fail(QB_EINVAL, "bad header: m");
        qb_graph* g = new (std::nothrow) qb_graph();
        if (!g) return fail(QB_ENOMEM, "qb_parse_rudy: out of host memory");
        g->n = int32_t(n);
        auto refuse = [&](const std::string& why) {
            delete g;
            return fail(QB_EINVAL, why);
        };
        int64_t count = 0;
        for (;;) {
            r.skip_space();
            if (r.p >= r.end) break;
            int64_t u = 0, v = 0, w = 1;
            if (!r.next(&s, &e) || !to_int(s, e, &u)) return refuse("bad vertex token '" + std::string(s ? s : "", s ? size_t(e - s) : 0) + "'");
            const char *s2 = nullptr, *e2 = nullptr;
            if (!r.next(&s2, &e2) || !to_int(s2, e2, &v)) {
                const std::string t = s2 ? std::string(s2, size_t(e2 - s2)) : std::string(s, size_t(e - s));
                return refuse("bad vertex token '" + t + "'");
            }
            const char *s3 = nullptr, *e3 = nullptr;
            if (r.next(&s3, &e3)) {
                if (!to_int(s3, e3, &w))
                    return refuse("weight '" + std::string(s3, size_t(e3 - s3)) +
                                  "' is not an integer; the float path is BinaryProblem");
                if (w < INT32_MIN || w > INT32_MAX) return refuse("weight out of int32 range");
                if (!r.line_done()) return refuse("trailing token on an edge line");
            }
            if (u < 1 || u > n || v < 1 || v > n) return refuse("vertex index out of range");
            if (u == v) return refuse("self-loop");
            g->eu.push_back(int32_t(u - 1));
            g->ev.push_back(int32_t(v - 1));
            g->ew.push_back(int32_t(w));
            ++count;
        }
        if (count != m)
            return refuse("header says " + std::to_string(m) + " edges, file has " + std::to_string(count));
        std::vector<uint64_t> key(g->eu.size());
        for (size_t k = 0; k < key.size(); ++k)
            key[k] = (uint64_t(std::min(g->eu[k], g->ev[k])) << 32) | uint64_t(std::max(g->eu[k], g->ev[k]));
        std::sort(key.begin(), key.end());
        for (size_t k = 1; k < key.size(); ++k)
            if (key[k] == key[k - 1]) return refuse("duplicate edge");
        *out = g;
        return QB_OK;
    });
}

extern "C" qb_status qb_graph_desc(const qb_graph* g, qb_ising_desc* d) {
    if (!g || !d) return qb::fail(QB_EINVAL, "qb_graph_desc: null argument");
    d->n = g->n;
    d->m = int64_t(g->eu.size());
    d->eu = g->eu.data();
    d->ev = g->ev.data();
    d->ew = g->ew.data();
    return QB_OK;
}

extern "C" void qb_graph_destroy(qb_graph* g) { delete g; }
