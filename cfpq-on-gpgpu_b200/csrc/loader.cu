// Parallel loader of the reference's graph text format (host code).
//
// Format and semantics: cfpq-cpp/Graph.cpp:11-20 reads `from label to`
// triples with `while (in >> from >> label >> to)`: whitespace-separated
// tokens, vertex ids as unsigned int, the first triple that does not parse
// ends the edge list, vertices_count = max id + 1.  Here a vertex token must
// be a decimal number of at most 4294967295 (a token that is not ends the
// list, as the stream extraction fails there).
//
// The file is read once and cut into chunks at line starts; threads parse
// their chunks line by line (3 tokens per line), each interning labels in its
// own table, then the tables are merged in file order, so label ids are
// numbered by first appearance in the file, as a sequential reader would.
// A non-empty line that does not hold exactly 3 tokens breaks the line-chunk
// view of the token stream (a triple may span lines); the file is then parsed
// again by one sequential tokenizer with the same rules.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cfpq_b200.h"

int set_error(int code, const char *fmt, ...);

namespace {

struct ChunkOut {
    std::vector<uint32_t> from, to, lid;
    std::vector<std::string_view> labels;  // local first-seen order
    bool stopped = false;                  // a malformed triple ended the list in this chunk
    bool irregular = false;                // a line without exactly 3 tokens
    uint32_t max_id = 0;
};

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

inline bool parse_u32(std::string_view t, uint32_t *out) {
    if (t.empty() || t.size() > 10) return false;
    uint64_t v = 0;
    for (char c : t) {
        if (c < '0' || c > '9') return false;
        v = v * 10 + (uint64_t)(c - '0');
    }
    if (v > 0xFFFFFFFFull) return false;
    *out = (uint32_t)v;
    return true;
}

struct Interner {
    std::unordered_map<std::string_view, uint32_t> ids;
    std::vector<std::string_view> *names;
    uint32_t get(std::string_view s) {
        auto it = ids.find(s);
        if (it != ids.end()) return it->second;
        const uint32_t id = (uint32_t)names->size();
        ids.emplace(s, id);
        names->push_back(s);
        return id;
    }
};

// Lines of [b, e): "from label to" each.
void parse_lines(const char *b, const char *e, ChunkOut *o) {
    Interner in{{}, &o->labels};
    const char *p = b;
    while (p < e && !o->stopped && !o->irregular) {
        const char *eol = static_cast<const char *>(memchr(p, '\n', (size_t)(e - p)));
        if (!eol) eol = e;
        std::string_view tok[3];
        int nt = 0;
        const char *q = p;
        while (q < eol) {
            while (q < eol && is_ws(*q)) ++q;
            if (q >= eol) break;
            const char *s = q;
            while (q < eol && !is_ws(*q)) ++q;
            if (nt < 3) tok[nt] = std::string_view(s, (size_t)(q - s));
            ++nt;
        }
        if (nt != 0 && nt != 3) {
            o->irregular = true;
            break;
        }
        if (nt == 3) {
            uint32_t a, c;
            if (!parse_u32(tok[0], &a) || !parse_u32(tok[2], &c)) {
                o->stopped = true;
                break;
            }
            o->from.push_back(a);
            o->to.push_back(c);
            o->lid.push_back(in.get(tok[1]));
            o->max_id = std::max(o->max_id, std::max(a, c));
        }
        p = eol + 1;
    }
}

// The token stream of the whole file, one triple at a time (any layout).
void parse_tokens(const char *b, const char *e, ChunkOut *o) {
    Interner in{{}, &o->labels};
    const char *p = b;
    auto next = [&](std::string_view *t) {
        while (p < e && is_ws(*p)) ++p;
        if (p >= e) return false;
        const char *s = p;
        while (p < e && !is_ws(*p)) ++p;
        *t = std::string_view(s, (size_t)(p - s));
        return true;
    };
    std::string_view t0, t1, t2;
    while (next(&t0) && next(&t1) && next(&t2)) {
        uint32_t a, c;
        if (!parse_u32(t0, &a) || !parse_u32(t2, &c)) break;
        o->from.push_back(a);
        o->to.push_back(c);
        o->lid.push_back(in.get(t1));
        o->max_id = std::max(o->max_id, std::max(a, c));
    }
}

}  // namespace

extern "C" int cfpq_graph_load(const char *path, int threads, cfpq_edge_list **out) {
    if (!path || !out) return set_error(CFPQ_ERR_INVALID, "null argument");
    *out = nullptr;
    FILE *f = fopen(path, "rb");
    if (!f) return set_error(CFPQ_ERR_IO, "cannot open graph file %s", path);
    std::string text;
    if (fseek(f, 0, SEEK_END) == 0) {
        const long size = ftell(f);
        if (size > 0) {
            text.resize((size_t)size);
            fseek(f, 0, SEEK_SET);
            if (fread(&text[0], 1, (size_t)size, f) != (size_t)size) {
                fclose(f);
                return set_error(CFPQ_ERR_IO, "cannot read graph file %s", path);
            }
        }
    }
    fclose(f);
    const char *b = text.data(), *e = b + text.size();
    size_t nt = threads > 0 ? (size_t)threads : std::max(1u, std::thread::hardware_concurrency());
    nt = std::max<size_t>(1, std::min(nt, text.size() / (1 << 16) + 1));  // >= 64 KiB per thread
    std::vector<const char *> cut(nt + 1);
    cut[0] = b;
    cut[nt] = e;
    for (size_t k = 1; k < nt; ++k) {
        const char *c = b + text.size() * k / nt;
        c = std::max(c, cut[k - 1]);
        const char *nl = static_cast<const char *>(memchr(c, '\n', (size_t)(e - c)));
        cut[k] = nl ? nl + 1 : e;
    }
    std::vector<ChunkOut> parts(nt);
    {
        std::vector<std::thread> pool;
        for (size_t k = 1; k < nt; ++k) pool.emplace_back(parse_lines, cut[k], cut[k + 1], &parts[k]);
        parse_lines(cut[0], cut[1], &parts[0]);
        for (auto &t : pool) t.join();
    }
    // the list ends at the first malformed triple; a layout with triples
    // across lines is parsed again as one token stream
    size_t used = nt;
    bool irregular = false;
    for (size_t k = 0; k < nt; ++k) {
        if (parts[k].irregular) {
            irregular = true;
            break;
        }
        if (parts[k].stopped) {
            used = k + 1;
            break;
        }
    }
    if (irregular) {
        parts.assign(1, ChunkOut());
        parse_tokens(b, e, &parts[0]);
        used = 1;
    }
    // merge label tables in file order, remap, concatenate
    std::unordered_map<std::string_view, uint32_t> global;
    std::vector<std::string_view> names;
    std::vector<std::vector<uint32_t>> remap(used);
    size_t total = 0, label_bytes = 0;
    uint32_t max_id = 0;
    bool any = false;
    for (size_t k = 0; k < used; ++k) {
        for (std::string_view s : parts[k].labels) {
            auto it = global.find(s);
            if (it == global.end()) {
                it = global.emplace(s, (uint32_t)names.size()).first;
                names.push_back(s);
                label_bytes += s.size() + 1;
            }
            remap[k].push_back(it->second);
        }
        total += parts[k].from.size();
        if (!parts[k].from.empty()) {
            max_id = std::max(max_id, parts[k].max_id);
            any = true;
        }
    }
    // one allocation: the record, the three arrays, the label pointers and names
    const size_t arr = total ? total : 1;
    const size_t bytes = sizeof(cfpq_edge_list) + 3 * arr * sizeof(uint32_t) + (names.size() + 1) * sizeof(char *) +
                         label_bytes + 1;
    char *mem = static_cast<char *>(malloc(bytes));
    if (!mem) return set_error(CFPQ_ERR_OOM, "host allocation of %zu bytes failed", bytes);
    cfpq_edge_list *el = reinterpret_cast<cfpq_edge_list *>(mem);
    char *p = mem + sizeof(cfpq_edge_list);
    el->from = reinterpret_cast<uint32_t *>(p);
    el->label = el->from + arr;
    el->to = el->label + arr;
    p += 3 * arr * sizeof(uint32_t);
    el->labels = reinterpret_cast<const char **>(p);
    p += (names.size() + 1) * sizeof(char *);
    for (size_t i = 0; i < names.size(); ++i) {
        memcpy(p, names[i].data(), names[i].size());
        p[names[i].size()] = '\0';
        el->labels[i] = p;
        p += names[i].size() + 1;
    }
    el->labels[names.size()] = nullptr;
    el->nedges = total;
    el->nlabels = (uint32_t)names.size();
    el->nvertices = any ? max_id + 1 : 0;
    if (any && max_id == 0xFFFFFFFFu) {
        free(mem);
        return set_error(CFPQ_ERR_UNSUPPORTED, "vertex id 4294967295: the vertex count does not fit 32 bits");
    }
    size_t off = 0;
    std::vector<size_t> offs(used);
    for (size_t k = 0; k < used; ++k) {
        offs[k] = off;
        off += parts[k].from.size();
    }
    {
        auto fill = [&](size_t k) {
            const ChunkOut &c = parts[k];
            const size_t o = offs[k];
            memcpy(el->from + o, c.from.data(), c.from.size() * sizeof(uint32_t));
            memcpy(el->to + o, c.to.data(), c.to.size() * sizeof(uint32_t));
            for (size_t i = 0; i < c.lid.size(); ++i) el->label[o + i] = remap[k][c.lid[i]];
        };
        std::vector<std::thread> pool;
        for (size_t k = 1; k < used; ++k) pool.emplace_back(fill, k);
        if (used) fill(0);
        for (auto &t : pool) t.join();
    }
    *out = el;
    return CFPQ_OK;
}

extern "C" void cfpq_edge_list_free(cfpq_edge_list *e) { free(e); }
