// Command-line wrapper of the UNMODIFIED reference's text edge-list reader
// (src/io.cpp:23-53 over src/csr_graph.cpp), compiled by oracle/Makefile
// into oracle/_ref/ref_io_tool.  TEST INFRASTRUCTURE ONLY.
//
// The reader runs in a process of its own: called in-process from a Python
// interpreter that had imported numpy, the reference's std::istream parsing
// reported trailing data on well-formed lines, so the checker must not run
// inside the test process.
//
//   ref_io_tool <path> <directed 0|1>
// prints "ok <V> <arcs>" and one line per vertex with its ascending row, or
// "runtime_error <message>" / "overflow_error <message>"; exit code 0.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

#include "velographx/io.hpp"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  try {
    const auto g = velographx::load_edge_list(argv[1], std::atoi(argv[2]) != 0);
    std::printf("ok %zu %zu\n", g.vertex_count(), g.edge_entry_count());
    for (std::size_t u = 0; u < g.vertex_count(); ++u) {
      for (auto v : g.neighbors(static_cast<velographx::VertexId>(u))) std::printf("%u ", v);
      std::printf("\n");
    }
  } catch (const std::overflow_error& e) {
    std::printf("overflow_error %s\n", e.what());
  } catch (const std::runtime_error& e) {
    std::printf("runtime_error %s\n", e.what());
  }
  return 0;
}
