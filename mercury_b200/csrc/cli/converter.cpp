// converter <mtx|tsv|snap> <edge file> <output prefix> [...]
//
// Stands in for the reference's dataset converter, which ships only as a
// closed binary and is called as `converter mtx $DATA $OUTPUT_DIR/graph 1 0
// 0 0` (datasets/converter.sh:5). It writes <prefix>.meta.txt,
// <prefix>.vertex.bin and <prefix>.edge.bin, the triple that tc_challenge and
// sm read. The arguments after the prefix are accepted and ignored. The
// input ids are 1-based for mtx and tsv; the program built as
// converter_vidfrom0 (the reference's 0-based variant,
// datasets/converter.sh:6) reads them 0-based. The CSR (symmetric, no
// self-loops, no duplicates, rows sorted) is built on the GPU.
#include <cinttypes>
#include <cstdio>
#include <cstring>

#include "mercury.h"

#ifndef MC_VID_FROM0
#define MC_VID_FROM0 0
#endif

static int fail(const char *what, int rc) {
  std::fprintf(stderr, "error: %s: %s\n", what, mc_strerror(rc));
  return 1;
}

int main(int argc, char *argv[]) {
  if (argc < 4) {
    std::printf("Usage: %s <mtx|tsv|snap> <edge file> <output prefix>\n", argv[0]);
    std::printf("Example: %s mtx /data/amazon0302.mtx /graph_inputs/amazon0302/graph\n", argv[0]);
    return 1;
  }
  int format = 0;
  if (!std::strcmp(argv[1], "mtx")) format = MC_EDGES_MTX;
  else if (!std::strcmp(argv[1], "tsv")) format = MC_EDGES_TSV;
  else if (!std::strcmp(argv[1], "snap")) format = MC_EDGES_SNAP;
  else {
    std::fprintf(stderr, "error: unknown input format '%s' (mtx, tsv or snap)\n", argv[1]);
    return 1;
  }
  const int base = MC_VID_FROM0 ? 0 : -1;
  mc_edges_t *e = nullptr;
  int rc = mc_edges_load(argv[2], format, base, &e);
  if (rc != MC_OK) return fail("reading the edge list", rc);
  int64_t m = 0, n = 0;
  mc_edges_info(e, &m, &n);
  std::printf("input: %s, %" PRId64 " vertices, %" PRId64 " edge lines\n", argv[2], n, m);
  mc_graph_t *g = nullptr;
  mc_timing_t t{};
  rc = mc_csr_build(mc_edges_src(e), mc_edges_dst(e), m, n, 0, nullptr, &g, &t);
  mc_edges_free(e);
  if (rc != MC_OK) return fail("building the CSR", rc);
  int64_t nv = 0, nnz = 0, md = 0;
  mc_graph_info(g, &nv, &nnz, &md);
  rc = mc_graph_write(g, argv[3]);
  mc_graph_free(g);
  if (rc != MC_OK) return fail("writing the graph", rc);
  std::printf("|V|: %" PRId64 ", |E|: %" PRId64 " (undirected), Max Degree: %" PRId64 "\n", nv,
              nnz / 2, md);
  std::printf("CSR build on the device = %g sec\n", t.count_ms / 1e3);
  std::printf("output: %s.meta.txt %s.vertex.bin %s.edge.bin\n", argv[3], argv[3], argv[3]);
  return 0;
}
