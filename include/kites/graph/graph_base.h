// graph_base.h -- vertex and edge counts shared by the graph classes
// (farkhor/KiTES kites/graph/graph_base.h:9-38).
#ifndef KITES_B200_GRAPH_BASE_H_
#define KITES_B200_GRAPH_BASE_H_

#include <cstddef>

namespace kites {

class graph_base {
 protected:
  std::size_t numVertices;
  std::size_t numEdges;

 public:
  graph_base(std::size_t nV = 0, std::size_t nE = 0) : numVertices(nV), numEdges(nE) {}
  void set_num_vertices(std::size_t n) { numVertices = n; }
  void set_num_edges(std::size_t n) { numEdges = n; }
  std::size_t get_num_vertices() const { return numVertices; }
  std::size_t get_num_edges() const { return numEdges; }
};

}  // namespace kites

#endif
