// Grammar loader and result printer (see cfpq/Grammar.h).
#include "cfpq/Grammar.h"

#include <fstream>
#include <sstream>
#include <stdexcept>

namespace {
constexpr unsigned long long kBase0 = 11;          // per-column base, cfpq-cpp/Grammar.cpp:12
constexpr unsigned long long kBase1 = 13;          // per-row base,    cfpq-cpp/Grammar.cpp:13
constexpr unsigned long long kMod = 1000000007ULL;  // modulus,        cfpq-cpp/Grammar.cpp:14
}  // namespace

unsigned int Grammar::index_of(const std::string &name) {
    auto it = nonterminal_to_index.find(name);
    if (it != nonterminal_to_index.end()) return it->second;
    nonterminal_to_index.emplace(name, nonterminals_count);
    return nonterminals_count++;
}

// One rule per line, whitespace separated (cfpq-cpp/Grammar.cpp:17-51):
//   "A"      epsilon rule,  "A x" terminal rule,  "A B C" binary rule A -> B C.
// Nonterminals are numbered in order of first appearance.  A line with more
// than three tokens only registers its head.  A line without tokens is
// skipped (the reference reads terms[0] of an empty vector there).
Grammar::Grammar(const std::string &grammar_filename) {
    std::ifstream in(grammar_filename);
    if (!in) throw std::runtime_error("cannot open grammar file " + grammar_filename);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::vector<std::string> tok;
        for (std::string t; ls >> t;) tok.push_back(t);
        if (tok.empty()) continue;
        const unsigned int head = index_of(tok[0]);
        switch (tok.size()) {
            case 1:
                epsilon_nonterminals.push_back(head);
                break;
            case 2:
                terminal_to_nonterminals[tok[1]].push_back((int)head);
                break;
            case 3: {
                const unsigned int b1 = index_of(tok[1]);
                const unsigned int b2 = index_of(tok[2]);
                rules.push_back({head, {b1, b2}});
                break;
            }
            default:
                break;
        }
    }
}

Grammar::Grammar(Grammar &&o) noexcept
    : nonterminals_count(o.nonterminals_count),
      vertices_count(o.vertices_count),
      nonterminal_to_index(std::move(o.nonterminal_to_index)),
      epsilon_nonterminals(std::move(o.epsilon_nonterminals)),
      terminal_to_nonterminals(std::move(o.terminal_to_nonterminals)),
      rules(std::move(o.rules)),
      matrices(std::move(o.matrices)) {
    o.matrices.clear();
}

Grammar::~Grammar() {
    for (Matrix *m : matrices) delete m;
}

unsigned int Grammar::get_rules_size() { return (unsigned int)rules.size(); }

const std::unordered_map<std::string, std::vector<int>> &Grammar::get_nonterminal_from_terminal() {
    return terminal_to_nonterminals;
}

// Rule arrays of the single-matrix nonterminal-set formulation
// (cfpq-cpp/Grammar.cpp:63-75): head as a one-hot word, bodies packed.
void Grammar::toArrays(unsigned int *grammar_body, unsigned long long *grammar_tail) {
    for (size_t i = 0; i < rules.size(); ++i) {
        grammar_body[i] = Matrix::toBoolVector(rules[i].first);
        grammar_tail[i] = ((unsigned long long)Matrix::toBoolVector(rules[i].second.first) << 32) |
                          (unsigned long long)Matrix::toBoolVector(rules[i].second.second);
    }
}

void Grammar::toArrays8(unsigned char *grammar_body, unsigned int *grammar_tail) {
    for (size_t i = 0; i < rules.size(); ++i) {
        grammar_body[i] = Matrix::toBoolVector8(rules[i].first);
        grammar_tail[i] = ((unsigned int)Matrix::toBoolVector8(rules[i].second.first) << 8) |
                          (unsigned int)Matrix::toBoolVector8(rules[i].second.second);
    }
}

// "name hash count" per nonterminal in name order (cfpq-cpp/Grammar.cpp:81-100).
// hash: per row, Horner over columns with base 11; over rows with base 13;
// modulo 1e9+7.  Backends that implement Matrix::hash_count supply the line
// without n^2 get_bit calls.
void Grammar::print_results(const std::string &output_filename) {
    std::ofstream out(output_filename);
    if (!out) throw std::runtime_error("cannot open output file " + output_filename);
    for (const auto &kv : nonterminal_to_index) {
        unsigned long long hash = 0;
        unsigned long count = 0;
        Matrix *m = kv.second < matrices.size() ? matrices[kv.second] : nullptr;
        if (m && !m->hash_count(&hash, &count)) {
            hash = 0;
            count = 0;
            for (unsigned int row = 0; row < vertices_count; ++row) {
                unsigned long long line = 0;
                for (unsigned int col = 0; col < vertices_count; ++col) {
                    line *= kBase0;
                    if (m->get_bit(row, col)) {
                        ++count;
                        ++line;
                    }
                    line %= kMod;
                }
                hash = (hash * kBase1 + line) % kMod;
            }
        }
        out << kv.first << ' ' << hash << ' ' << count << '\n';
    }
}
