/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the CFPQ closure path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg /
 * reference arm may load, link or execute this code, and only as the checker
 * or the timed CPU baseline.  The product path (the CUDA library) never calls
 * it.
 *
 * It restates, in plain C, the reference's CPU path:
 *   - grammar loader     cfpq-cpp/Grammar.cpp:17-51 (CNF text, first-seen
 *                        nonterminal indexing, arity 1 = epsilon rule,
 *                        arity 2 = terminal rule, arity 3 = binary rule)
 *   - graph loader       cfpq-cpp/Graph.cpp:11-20 ("from label to" triples,
 *                        vertices_count = max id + 1)
 *   - closure driver     cfpq-cpp/Grammar.h:23-81 (matrix init from edges and
 *                        epsilon diagonals, worklist of rules re-queued when
 *                        their head changes)
 *   - add_mul semantics  m4ri/m4ri_matrix.cpp:20-28 (C |= A*B over (OR, AND),
 *                        returns whether any bit of C changed; operands may
 *                        alias C, the product then uses the operands' values
 *                        from before the call, as the reference GPU backends
 *                        do with their temporary/extra matrix,
 *                        cuda/naive-gpu/Multiplication.cu:146-158 and
 *                        cuda/methodOf4RusBooleanSemiringGpu/
 *                        methodOf4RusBooleanSemiringMatrix.cu:62-67)
 *   - result printer     cfpq-cpp/Grammar.cpp:81-100 (per nonterminal in name
 *                        order: polynomial row hash with bases 11 / 13 modulo
 *                        1e9+7, and the number of set bits)
 *
 * Worklist order: the reference pops from an unordered_set (arbitrary order);
 * the oracle uses FIFO order.  The closure is the unique least fixpoint, so the
 * final matrices do not depend on the order; the number of products does.
 *
 * Deviation: an empty (whitespace-only) grammar line is undefined behaviour in
 * the reference (terms[0] of an empty vector, Grammar.cpp:29); the oracle skips
 * such lines.
 */
#define _GNU_SOURCE
#include "m4ri_restated.h"

#include <stdio.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>
#include <time.h>

#define ORC_HASH_BASE0 11ULL        /* Grammar.cpp:12 */
#define ORC_HASH_BASE1 13ULL        /* Grammar.cpp:13 */
#define ORC_HASH_MOD 1000000007ULL  /* Grammar.cpp:14 */

enum { ORC_METHOD_NAIVE = 0, ORC_METHOD_M4RM = 1 };

typedef struct {
    char **items;
    int count, cap;
} strlist;

static int strlist_find(const strlist *l, const char *s) {
    for (int i = 0; i < l->count; ++i)
        if (strcmp(l->items[i], s) == 0) return i;
    return -1;
}

static int strlist_add(strlist *l, const char *s) {
    if (l->count == l->cap) {
        l->cap = l->cap ? 2 * l->cap : 16;
        l->items = (char **)realloc(l->items, (size_t)l->cap * sizeof(char *));
    }
    l->items[l->count] = strdup(s);
    return l->count++;
}

static void strlist_free(strlist *l) {
    for (int i = 0; i < l->count; ++i) free(l->items[i]);
    free(l->items);
    l->items = NULL;
    l->count = l->cap = 0;
}

typedef struct {
    int *v;
    int n, cap;
} intvec;

static void intvec_push(intvec *a, int x) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 8;
        a->v = (int *)realloc(a->v, (size_t)a->cap * sizeof(int));
    }
    a->v[a->n++] = x;
}

typedef struct orc_problem {
    /* grammar */
    strlist nonterminals;   /* index -> name, first-seen order */
    int nrules;
    int *rules;             /* (head, body1, body2) triples, file order */
    intvec eps;             /* epsilon nonterminals */
    strlist terminals;      /* terminal names */
    intvec *term_nts;       /* per terminal: nonterminals deriving it */
    /* graph */
    unsigned vertices;
    size_t nedges;
    unsigned *edge_from, *edge_to;
    int *edge_term;         /* terminal index or -1 */
    strlist edge_labels_unknown;
    /* closure state */
    int wpr;
    uint64_t **mats;
    long long products;
} orc_problem;

static int grammar_nt_index(orc_problem *p, const char *name) {
    int i = strlist_find(&p->nonterminals, name);
    return i >= 0 ? i : strlist_add(&p->nonterminals, name);
}

static int parse_grammar(orc_problem *p, const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char *line = NULL;
    size_t cap = 0;
    ssize_t len;
    int rules_cap = 0;
    while ((len = getline(&line, &cap, f)) >= 0) {
        char *tok[4];
        int nt = 0;
        char *save = NULL;
        for (char *t = strtok_r(line, " \t\r\n\v\f", &save); t; t = strtok_r(NULL, " \t\r\n\v\f", &save)) {
            if (nt < 4) tok[nt] = t;
            ++nt;
        }
        if (nt == 0) continue; /* see header: deviation from UB */
        const int head = grammar_nt_index(p, tok[0]);
        if (nt == 1) {
            intvec_push(&p->eps, head);
        } else if (nt == 2) {
            int t = strlist_find(&p->terminals, tok[1]);
            if (t < 0) {
                t = strlist_add(&p->terminals, tok[1]);
                p->term_nts = (intvec *)realloc(p->term_nts, (size_t)p->terminals.cap * sizeof(intvec));
                memset(&p->term_nts[t], 0, sizeof(intvec));
            }
            intvec_push(&p->term_nts[t], head);
        } else if (nt == 3) {
            const int b1 = grammar_nt_index(p, tok[1]);
            const int b2 = grammar_nt_index(p, tok[2]);
            if (p->nrules == rules_cap) {
                rules_cap = rules_cap ? 2 * rules_cap : 16;
                p->rules = (int *)realloc(p->rules, (size_t)rules_cap * 3 * sizeof(int));
            }
            p->rules[3 * p->nrules + 0] = head;
            p->rules[3 * p->nrules + 1] = b1;
            p->rules[3 * p->nrules + 2] = b2;
            ++p->nrules;
        }
        /* arity > 3: the head is indexed, the line is otherwise ignored */
    }
    free(line);
    fclose(f);
    return 0;
}

static int parse_graph(orc_problem *p, const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    size_t cap = 0;
    unsigned from, to;
    char label[4096];
    int last_term = -1;
    char last_label[4096] = "";
    while (fscanf(f, "%u %4095s %u", &from, label, &to) == 3) {
        if (p->nedges == cap) {
            cap = cap ? 2 * cap : 1024;
            p->edge_from = (unsigned *)realloc(p->edge_from, cap * sizeof(unsigned));
            p->edge_to = (unsigned *)realloc(p->edge_to, cap * sizeof(unsigned));
            p->edge_term = (int *)realloc(p->edge_term, cap * sizeof(int));
        }
        int t;
        if (last_label[0] && strcmp(label, last_label) == 0) {
            t = last_term;
        } else {
            t = strlist_find(&p->terminals, label);
            strcpy(last_label, label);
            last_term = t;
        }
        p->edge_from[p->nedges] = from;
        p->edge_to[p->nedges] = to;
        p->edge_term[p->nedges] = t;
        ++p->nedges;
        const unsigned m = (from > to ? from : to) + 1;
        if (m > p->vertices) p->vertices = m;
    }
    fclose(f);
    return 0;
}

orc_problem *orc_load(const char *grammar_path, const char *graph_path) {
    orc_problem *p = (orc_problem *)calloc(1, sizeof(orc_problem));
    if (parse_grammar(p, grammar_path) != 0 || parse_graph(p, graph_path) != 0) {
        free(p);
        return NULL;
    }
    return p;
}

void orc_free(orc_problem *p) {
    if (!p) return;
    if (p->mats) {
        for (int i = 0; i < p->nonterminals.count; ++i) free(p->mats[i]);
        free(p->mats);
    }
    for (int t = 0; t < p->terminals.count; ++t) free(p->term_nts[t].v);
    free(p->term_nts);
    strlist_free(&p->nonterminals);
    strlist_free(&p->terminals);
    free(p->rules);
    free(p->eps.v);
    free(p->edge_from);
    free(p->edge_to);
    free(p->edge_term);
    free(p);
}

int orc_num_nonterminals(const orc_problem *p) { return p->nonterminals.count; }
unsigned orc_vertices(const orc_problem *p) { return p->vertices; }
int orc_num_rules(const orc_problem *p) { return p->nrules; }
const int *orc_rules(const orc_problem *p) { return p->rules; }
const char *orc_nonterminal_name(const orc_problem *p, int i) { return p->nonterminals.items[i]; }
int orc_words_per_row(const orc_problem *p) { return p->wpr; }
const uint64_t *orc_matrix(const orc_problem *p, int i) { return p->mats ? p->mats[i] : NULL; }
long long orc_products(const orc_problem *p) { return p->products; }

/* C |= A*B with the operands' values from before the call; returns 1 if C changed. */
int orc_add_mul(int n, uint64_t *c, const uint64_t *a, const uint64_t *b, int method, int threads) {
    const int wpr = (n + 63) / 64;
    const size_t words = (size_t)n * wpr;
    if (words == 0) return 0;
    uint64_t *t = (uint64_t *)calloc(words, sizeof(uint64_t));
    if (!t) abort();
    if (method == ORC_METHOD_M4RM)
        orc_m4rm_product_or(n, wpr, a, b, t, threads);
    else
        orc_naive_product_or(n, wpr, a, b, t, threads);
    int changed = 0;
    for (size_t i = 0; i < words; ++i) {
        const uint64_t nv = c[i] | t[i];
        if (nv != c[i]) {
            changed = 1;
            c[i] = nv;
        }
    }
    free(t);
    return changed;
}

/* Rows rows[0..nrows-1] of C | A*B (the same semantics as orc_add_mul,
 * restricted to a sample of rows): out receives nrows rows of wpr words, row
 * i = C[rows[i]] | OR of B[k] over the set bits k of A[rows[i]].  For checking
 * products whose full CPU evaluation would take hours (n = 65536); rows run
 * in parallel. */
void orc_add_mul_rows(int n, uint64_t *out, const uint64_t *c, const uint64_t *a, const uint64_t *b,
                      const uint32_t *rows, int nrows, int threads) {
    const int wpr = (n + 63) / 64;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < nrows; ++i) {
        const size_t r = rows[i];
        uint64_t *acc = out + (size_t)i * wpr;
        memcpy(acc, c + r * wpr, (size_t)wpr * sizeof(uint64_t));
        const uint64_t *ar = a + r * wpr;
        for (int w = 0; w < wpr; ++w) {
            uint64_t bits = ar[w];
            while (bits) {
                const int k = w * 64 + __builtin_ctzll(bits);
                bits &= bits - 1;
                if (k >= n) break;
                const uint64_t *br = b + (size_t)k * wpr;
                for (int j = 0; j < wpr; ++j) acc[j] |= br[j];
            }
        }
    }
}

/* The reference's per-bit loop (Grammar.cpp:84-97). */
void orc_hash_count(int n, const uint64_t *m, uint64_t *hash_out, uint64_t *count_out) {
    const int wpr = (n + 63) / 64;
    unsigned long long hash = 0, count = 0;
    for (int row = 0; row < n; ++row) {
        unsigned long long line_hash = 0;
        const uint64_t *r = m + (size_t)row * wpr;
        for (int col = 0; col < n; ++col) {
            line_hash *= ORC_HASH_BASE0;
            if ((r[col / 64] >> (col % 64)) & 1u) {
                ++count;
                ++line_hash;
            }
            line_hash %= ORC_HASH_MOD;
        }
        hash = (hash * ORC_HASH_BASE1 + line_hash) % ORC_HASH_MOD;
    }
    *hash_out = hash;
    *count_out = count;
}

static double now_ms(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec / 1e6;
}

/* Grammar.h:23-81 with a FIFO worklist.  Returns 0 on success. */
int orc_closure(orc_problem *p, int method, int threads, double *algo_ms) {
    const int nnt = p->nonterminals.count;
    const int n = (int)p->vertices;
    p->wpr = (n + 63) / 64;
    const size_t words = (size_t)n * p->wpr;
    if (p->mats) {
        for (int i = 0; i < nnt; ++i) free(p->mats[i]);
        free(p->mats);
    }
    p->mats = (uint64_t **)calloc(nnt ? nnt : 1, sizeof(uint64_t *));
    for (int i = 0; i < nnt; ++i) {
        p->mats[i] = (uint64_t *)calloc(words ? words : 1, sizeof(uint64_t));
        if (!p->mats[i]) return -1;
    }
    /* rules_with_nonterminal (Grammar.h:35-39) */
    intvec *users = (intvec *)calloc(nnt ? nnt : 1, sizeof(intvec));
    for (int r = 0; r < p->nrules; ++r) {
        intvec_push(&users[p->rules[3 * r + 1]], r);
        intvec_push(&users[p->rules[3 * r + 2]], r);
    }
    /* edges (Grammar.h:41-45) */
    for (size_t e = 0; e < p->nedges; ++e) {
        const int t = p->edge_term[e];
        if (t < 0) continue;
        for (int j = 0; j < p->term_nts[t].n; ++j) {
            uint64_t *m = p->mats[p->term_nts[t].v[j]];
            m[(size_t)p->edge_from[e] * p->wpr + p->edge_to[e] / 64] |= 1ULL << (p->edge_to[e] % 64);
        }
    }
    /* epsilon diagonals (Grammar.h:47-51) */
    for (int j = 0; j < p->eps.n; ++j) {
        uint64_t *m = p->mats[p->eps.v[j]];
        for (int i = 0; i < n; ++i) m[(size_t)i * p->wpr + i / 64] |= 1ULL << (i % 64);
    }
    /* worklist (Grammar.h:58-69) */
    const int qcap = p->nrules + 1;
    int *queue = (int *)malloc((size_t)qcap * sizeof(int));
    char *queued = (char *)calloc(qcap, 1);
    int qhead = 0, qsize = 0;
    for (int r = 0; r < p->nrules; ++r) {
        queue[(qhead + qsize++) % qcap] = r;
        queued[r] = 1;
    }
    p->products = 0;
    const double t0 = now_ms();
    while (qsize > 0) {
        const int r = queue[qhead];
        qhead = (qhead + 1) % qcap;
        --qsize;
        queued[r] = 0;
        const int C = p->rules[3 * r], A = p->rules[3 * r + 1], B = p->rules[3 * r + 2];
        ++p->products;
        if (orc_add_mul(n, p->mats[C], p->mats[A], p->mats[B], method, threads)) {
            for (int j = 0; j < users[C].n; ++j) {
                const int u = users[C].v[j];
                if (!queued[u]) {
                    queued[u] = 1;
                    queue[(qhead + qsize++) % qcap] = u;
                }
            }
        }
    }
    if (algo_ms) *algo_ms = now_ms() - t0;
    free(queue);
    free(queued);
    for (int i = 0; i < nnt; ++i) free(users[i].v);
    free(users);
    return 0;
}

static int cmp_name_idx(const void *a, const void *b, void *ctx) {
    const orc_problem *p = (const orc_problem *)ctx;
    return strcmp(p->nonterminals.items[*(const int *)a], p->nonterminals.items[*(const int *)b]);
}

/* Grammar.cpp:81-100: one "name hash count" line per nonterminal in name order. */
int orc_write_results(const orc_problem *p, const char *out_path) {
    FILE *f = fopen(out_path, "w");
    if (!f) return -1;
    const int nnt = p->nonterminals.count;
    int *order = (int *)malloc((size_t)(nnt ? nnt : 1) * sizeof(int));
    for (int i = 0; i < nnt; ++i) order[i] = i;
    qsort_r(order, nnt, sizeof(int), cmp_name_idx, (void *)p);
    for (int j = 0; j < nnt; ++j) {
        const int i = order[j];
        uint64_t h = 0, c = 0;
        if (p->mats) orc_hash_count((int)p->vertices, p->mats[i], &h, &c);
        fprintf(f, "%s %llu %llu\n", p->nonterminals.items[i], (unsigned long long)h, (unsigned long long)c);
    }
    free(order);
    fclose(f);
    return 0;
}

#ifdef ORACLE_MAIN
/* Same argv / stdout / answer-file contract as the reference mains
 * (m4ri/main.cpp:7-15): <grammar> <graph> <out>; prints "total_ms algo_ms". */
int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s <grammar> <graph> <out> [naive|m4rm] [threads]\n", argv[0]);
        return 2;
    }
    const int method = (argc > 4 && strcmp(argv[4], "naive") == 0) ? ORC_METHOD_NAIVE : ORC_METHOD_M4RM;
    const int threads = argc > 5 ? atoi(argv[5]) : 0;
    orc_problem *p = orc_load(argv[1], argv[2]);
    if (!p) {
        fprintf(stderr, "cannot read input files\n");
        return 1;
    }
    const double t0 = now_ms();
    double algo = 0;
    if (orc_closure(p, method, threads, &algo) != 0) return 1;
    const double total = now_ms() - t0;
    printf("%u %u\n", (unsigned)total, (unsigned)algo);
    orc_write_results(p, argv[3]);
    orc_free(p);
    return 0;
}
#endif
