// Drop-in GraphWalker API: relative error of top-N visit frequencies against
// an accurate list (the reference's src/util/comperror.hpp:8-97).
#ifndef DEF_GRAPHWALKER_COMPERROR
#define DEF_GRAPHWALKER_COMPERROR

#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "api/datatype.hpp"
#include "util/toplist.hpp"

// Writes `n` zero values of T to <base>_GraphWalker/<sizeof(T)>B.vvalue.
template <typename T>
void initialVertexValue(vid_t n, std::string base) {
  std::ofstream o((base + "_GraphWalker/" + std::to_string(sizeof(T)) + "B.vvalue").c_str(), std::ios::binary);
  const T zero = 0;
  for (vid_t i = 0; i < n; ++i) o.write((const char*)&zero, sizeof zero);
}

// Writes (vertex, value) pairs of a top list, one per line.
template <typename T>
void writeFile(std::string fname, const std::vector<vertex_value<T>>& top) {
  std::ofstream o(fname.c_str());
  for (auto& e : top) o << e.vertex << " " << e.value << "\n";
}

// Mean relative error of `approx` against the accurate list read from
// `accurate_file` ("vertex value" lines), over the vertices of the accurate list.
template <typename T>
double computeError(const std::vector<vertex_value<T>>& approx, std::string accurate_file) {
  std::ifstream in(accurate_file.c_str());
  vid_t v;
  double x;
  double err = 0;
  int n = 0;
  while (in >> v >> x) {
    double a = 0;
    for (auto& e : approx)
      if (e.vertex == v) a = (double)e.value;
    if (x != 0) err += std::fabs(a - x) / x;
    ++n;
  }
  return n ? err / n : 0.0;
}

#endif
