// Test program for the C++ host API (cfpq-on-gpgpu_b200/cpp): a plain CPU
// bitset Matrix backend plugged into Grammar::intersection_with_graph, once
// through the driver's worklist and once through the environment_closure
// hook.  Same argv / stdout / answer-file contract as the reference mains:
//   cpu_backend_main <grammar> <graph> <answer> worklist|hook
#include <cstdint>
#include <cstring>
#include <iostream>
#include <vector>

#include "cfpq/Grammar.h"
#include "cfpq/Graph.h"

class BitsetMatrix : public Matrix {
public:
    explicit BitsetMatrix(unsigned n) : Matrix(n), n_(n), wpr_((n + 63) / 64), w_((size_t)n * wpr_, 0) {}

    void set_bit(unsigned r, unsigned c) override { w_[(size_t)r * wpr_ + c / 64] |= 1ULL << (c % 64); }

    unsigned get_bit(unsigned r, unsigned c) override { return (w_[(size_t)r * wpr_ + c / 64] >> (c % 64)) & 1u; }

    bool add_mul(Matrix *left, Matrix *right) override {
        auto *a = dynamic_cast<BitsetMatrix *>(left);
        auto *b = dynamic_cast<BitsetMatrix *>(right);
        const std::vector<uint64_t> A = a->w_, B = b->w_;  // snapshot (aliasing)
        bool changed = false;
        for (unsigned i = 0; i < n_; ++i)
            for (unsigned kw = 0; kw < wpr_; ++kw)
                for (uint64_t x = A[(size_t)i * wpr_ + kw]; x; x &= x - 1) {
                    const unsigned k = kw * 64 + __builtin_ctzll(x);
                    for (unsigned j = 0; j < wpr_; ++j) {
                        uint64_t &o = w_[(size_t)i * wpr_ + j];
                        const uint64_t nv = o | B[(size_t)k * wpr_ + j];
                        changed |= nv != o;
                        o = nv;
                    }
                }
        return changed;
    }

private:
    unsigned n_, wpr_;
    std::vector<uint64_t> w_;
};

// Runs the fixpoint itself (repeat all rules until no change) and tells the
// driver to skip its worklist.
class HookEnv : public MatricesEnv {
public:
    bool environment_closure(const std::vector<cfpq_rule_entry> &rules, const std::vector<Matrix *> &m) override {
        for (bool changed = true; changed;) {
            changed = false;
            for (const auto &r : rules) changed |= m[r.first]->add_mul(m[r.second.first], m[r.second.second]);
        }
        return true;
    }
};

int main(int argc, char **argv) {
    if (argc < 5) return 2;
    Grammar grammar = Grammar(argv[1]);
    Graph graph = Graph(argv[2]);
    std::pair<unsigned, unsigned> t;
    if (!std::strcmp(argv[4], "hook"))
        t = grammar.intersection_with_graph<BitsetMatrix, HookEnv>(graph);
    else
        t = grammar.intersection_with_graph<BitsetMatrix>(graph);
    std::cout << t.first << ' ' << t.second << std::endl;
    grammar.print_results(argv[3]);
    return 0;
}
