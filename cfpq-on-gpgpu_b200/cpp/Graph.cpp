// Graph loader (see cfpq/Graph.h).
#include "cfpq/Graph.h"

#include <algorithm>
#include <stdexcept>

#include "cfpq/Matrix.h"
#include "cfpq_b200.h"

// Reads "from label to" triples until the first malformed one, like the
// reference's `while (in >> from >> label >> to)` loop (cfpq-cpp/Graph.cpp:15),
// with the library's parallel loader (cfpq_graph_load).
Graph::Graph(const std::string &graph_filename) {
    cfpq_edge_list *el = nullptr;
    if (cfpq_graph_load(graph_filename.c_str(), 0, &el) != CFPQ_OK)
        throw std::runtime_error(std::string("cannot read graph file ") + graph_filename + ": " + cfpq_last_error());
    std::vector<std::string> names(el->labels, el->labels + el->nlabels);
    edges.reserve(el->nedges);
    for (size_t i = 0; i < el->nedges; ++i) edges.push_back({names[el->label[i]], {el->from[i], el->to[i]}});
    vertices_count = el->nvertices;
    cfpq_edge_list_free(el);
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
