// Link-time fix-ups for building the reference's sources (TEST INFRASTRUCTURE
// ONLY; used by oracle/Makefile for oracle/_ref/).
#include <tuple>
#include <vector>

// Replacement for the reference's indices_to_delete (smearing.cpp:361-379),
// whose symbol oracle/Makefile makes weak. The reference function only ever
// returns an empty list (it never appends), but on the way it reads
// indices[3] of a 3-element vector, which crashes. Same result, no read.
std::vector<std::tuple<int, int, int>>
indices_to_delete(std::vector<std::vector<std::tuple<int, int, int>>> &,
                  std::vector<std::tuple<int, int, int>> &, int) {
  return {};
}
