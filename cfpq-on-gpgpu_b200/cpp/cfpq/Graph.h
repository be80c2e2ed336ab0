// Edge-labelled graph loader with the reference's file format and members
// (cfpq-cpp/Graph.h:9-26, Graph.cpp:11-20): one "from label to" triple per
// line; vertices_count = max vertex id + 1.
#ifndef CFPQ_B200_GRAPH_H
#define CFPQ_B200_GRAPH_H

#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

using edge = std::pair<std::string, std::pair<unsigned int, unsigned int>>;

class Graph {
public:
    explicit Graph(const std::string &graph_filename);

    virtual ~Graph() = default;

    std::vector<edge> edges;

    unsigned int vertices_count = 0;

    // Nonterminal-set matrices of the single-matrix formulation
    // (cfpq-cpp/Graph.cpp:22-48): matrix[from][to] = OR of the bits of the
    // nonterminals deriving the edge's label.
    void fillMatrix(unsigned int **matrix,
                    const std::unordered_map<std::string, std::vector<int>> &terminal_to_nonterminals);

    void fillMatrix(unsigned char **matrix,
                    const std::unordered_map<std::string, std::vector<int>> &terminal_to_nonterminals);
};

#endif  // CFPQ_B200_GRAPH_H
