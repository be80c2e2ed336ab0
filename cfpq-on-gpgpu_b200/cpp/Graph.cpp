// Graph loader (see cfpq/Graph.h).
#include "cfpq/Graph.h"

#include <algorithm>
#include <fstream>
#include <stdexcept>

#include "cfpq/Matrix.h"

// Reads "from label to" triples until the first malformed one, like the
// reference's `while (in >> from >> label >> to)` loop (cfpq-cpp/Graph.cpp:15).
Graph::Graph(const std::string &graph_filename) {
    std::ifstream in(graph_filename);
    if (!in) throw std::runtime_error("cannot open graph file " + graph_filename);
    unsigned int from = 0, to = 0;
    std::string label;
    while (in >> from >> label >> to) {
        edges.push_back({label, {from, to}});
        vertices_count = std::max(vertices_count, std::max(from, to) + 1);
    }
}

template <class W, class F>
static void fill_sets(const std::vector<edge> &edges, W **matrix,
                      const std::unordered_map<std::string, std::vector<int>> &t2n, F one_hot) {
    for (const auto &e : edges) {
        auto it = t2n.find(e.first);
        if (it == t2n.end()) continue;
        W set = 0;
        for (int nt : it->second) set |= one_hot((unsigned)nt);
        matrix[e.second.first][e.second.second] = set;
    }
}

void Graph::fillMatrix(unsigned int **matrix,
                       const std::unordered_map<std::string, std::vector<int>> &terminal_to_nonterminals) {
    fill_sets(edges, matrix, terminal_to_nonterminals, [](unsigned nt) { return Matrix::toBoolVector(nt); });
}

void Graph::fillMatrix(unsigned char **matrix,
                       const std::unordered_map<std::string, std::vector<int>> &terminal_to_nonterminals) {
    fill_sets(edges, matrix, terminal_to_nonterminals, [](unsigned nt) { return Matrix::toBoolVector8(nt); });
}
