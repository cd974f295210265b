// Drop-in GraphWalker API: top-N vertices of a vertex-value file
// (the reference's src/util/toplist.hpp:86-183, used by its stale apps).
#ifndef DEF_GRAPHCHI_TOPLIST
#define DEF_GRAPHCHI_TOPLIST

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "api/datatype.hpp"

template <typename VertexDataType>
struct vertex_value {
  vid_t vertex;
  VertexDataType value;
  vertex_value() {}
  vertex_value(vid_t v, VertexDataType x) : vertex(v), value(x) {}
};

// Reads `count` values of type T from `fname` (the vertex-value file an app
// wrote) and returns the ntop largest with their vertex ids, largest first.
template <typename VertexDataType>
std::vector<vertex_value<VertexDataType>> get_top_vertices(std::string fname, int ntop, vid_t from = 0,
                                                          vid_t to = 0) {
  std::vector<vertex_value<VertexDataType>> out;
  FILE* f = fopen(fname.c_str(), "rb");
  if (!f) return out;
  std::vector<VertexDataType> vals;
  VertexDataType x;
  while (fread(&x, sizeof x, 1, f) == 1) vals.push_back(x);
  fclose(f);
  if (to == 0 || to > vals.size()) to = (vid_t)vals.size();
  for (vid_t v = from; v < to; ++v) out.emplace_back(v, vals[v]);
  const size_t k = std::min<size_t>(ntop, out.size());
  std::partial_sort(out.begin(), out.begin() + k, out.end(),
                    [](const vertex_value<VertexDataType>& a, const vertex_value<VertexDataType>& b) {
                      return a.value != b.value ? a.value > b.value : a.vertex < b.vertex;
                    });
  out.resize(k);
  return out;
}

#endif
