// CNF grammar loader and the CFPQ closure driver, with the public API of the
// reference's cfpq-cpp/Grammar.h:16-100 (constructor from a file,
// intersection_with_graph<T1, T2>, print_results, get_rules_size,
// get_nonterminal_from_terminal, toArrays, toArrays8).
//
// Driver semantics (cfpq-cpp/Grammar.h:23-81): one T1 matrix per nonterminal;
// edge bits and epsilon diagonals set through Matrix::set_bit; then
// environment_preprocessing, the fixpoint, environment_postprocessing.  The
// fixpoint is delegated to MatricesEnv::environment_closure when the backend
// provides it; otherwise the worklist of rules is run with Matrix::add_mul,
// re-queueing every rule whose body contains a head that changed.  Returns
// (total ms, algorithm ms) measured like the reference.
#ifndef CFPQ_B200_GRAMMAR_H
#define CFPQ_B200_GRAMMAR_H

#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "Graph.h"
#include "Matrix.h"

using nonterminals_pair = std::pair<unsigned int, unsigned int>;

class Grammar {
public:
    explicit Grammar(const std::string &grammar_filename);

    virtual ~Grammar();

    Grammar(const Grammar &) = delete;
    Grammar &operator=(const Grammar &) = delete;
    Grammar(Grammar &&other) noexcept;

    template <class T1 = Matrix, class T2 = MatricesEnv>
    std::pair<unsigned int, unsigned int> intersection_with_graph(Graph &graph) {
        std::unique_ptr<T2> environment(new T2());
        vertices_count = graph.vertices_count;
        matrices.reserve(nonterminals_count);
        std::vector<std::vector<unsigned int>> users(nonterminals_count);
        for (unsigned int i = 0; i < nonterminals_count; ++i) matrices.push_back(new T1(vertices_count));

        std::deque<unsigned int> worklist;
        std::vector<char> queued(rules.size(), 1);
        for (unsigned int r = 0; r < rules.size(); ++r) {
            users[rules[r].second.first].push_back(r);
            users[rules[r].second.second].push_back(r);
            worklist.push_back(r);
        }

        for (const auto &e : graph.edges) {
            auto it = terminal_to_nonterminals.find(e.first);
            if (it == terminal_to_nonterminals.end()) continue;
            for (int nt : it->second) matrices[nt]->set_bit(e.second.first, e.second.second);
        }
        for (unsigned int nt : epsilon_nonterminals)
            for (unsigned int v = 0; v < vertices_count; ++v) matrices[nt]->set_bit(v, v);

        using clock = std::chrono::high_resolution_clock;
        const auto t_begin = clock::now();
        environment->environment_preprocessing(matrices);
        const auto t_algo_begin = clock::now();

        if (!environment->environment_closure(rules, matrices)) {
            while (!worklist.empty()) {
                const unsigned int r = worklist.front();
                worklist.pop_front();
                queued[r] = 0;
                const unsigned int head = rules[r].first;
                if (matrices[head]->add_mul(matrices[rules[r].second.first], matrices[rules[r].second.second])) {
                    for (unsigned int u : users[head]) {
                        if (!queued[u]) {
                            queued[u] = 1;
                            worklist.push_back(u);
                        }
                    }
                }
            }
        }

        const auto t_algo_end = clock::now();
        environment->environment_postprocessing(matrices);
        const auto t_end = clock::now();
        environment.reset();

        using std::chrono::duration_cast;
        using std::chrono::milliseconds;
        return std::make_pair(static_cast<unsigned int>(duration_cast<milliseconds>(t_end - t_begin).count()),
                              static_cast<unsigned int>(duration_cast<milliseconds>(t_algo_end - t_algo_begin).count()));
    }

    void print_results(const std::string &output_filename);

    unsigned int get_rules_size();

    const std::unordered_map<std::string, std::vector<int>> &get_nonterminal_from_terminal();

    void toArrays(unsigned int *grammar_body, unsigned long long *grammar_tail);

    void toArrays8(unsigned char *grammar_body, unsigned int *grammar_tail);

    // Accessors not in the reference API (read-only views for tools and tests).
    unsigned int get_nonterminals_count() const { return nonterminals_count; }
    const std::vector<cfpq_rule_entry> &get_rules() const { return rules; }
    const std::map<std::string, unsigned int> &get_nonterminal_index() const { return nonterminal_to_index; }
    const std::vector<unsigned int> &get_epsilon_nonterminals() const { return epsilon_nonterminals; }
    Matrix *get_matrix(unsigned int i) const { return i < matrices.size() ? matrices[i] : nullptr; }
    unsigned int get_vertices_count() const { return vertices_count; }

private:
    unsigned int nonterminals_count = 0;
    unsigned int vertices_count = 0;

    std::map<std::string, unsigned int> nonterminal_to_index;
    std::vector<unsigned int> epsilon_nonterminals;
    std::unordered_map<std::string, std::vector<int>> terminal_to_nonterminals;
    std::vector<cfpq_rule_entry> rules;
    std::vector<Matrix *> matrices;

    unsigned int index_of(const std::string &name);
};

#endif  // CFPQ_B200_GRAMMAR_H
