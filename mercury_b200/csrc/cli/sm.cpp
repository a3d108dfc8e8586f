// sm <graph_prefix> <P1..P8> -- drop-in for the reference's pattern-count
// program sm_multigpu (subgraph_matching/main_mpi.cpp:7-36,
// subgraph_matching/sm_multigpu.cu:97-239) on one GPU without MPI.  Same
// output labels: "Subgraph matching", "Total runtime  = X sec" and
// "total_num_triangles = N" (the reference prints that label for every
// pattern).  A third argument (the reference's device count) is accepted and
// ignored: this program runs on the current device.
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>

#include "mercury.h"

static int fail(const char *what, int rc) {
  std::fprintf(stderr, "error: %s: %s\n", what, mc_strerror(rc));
  return 1;
}

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::printf("Usage: %s <graph> <pattern> [devices]\n", argv[0]);
    std::printf("Example: %s /graph_inputs/mico/graph P1\n", argv[0]);
    return 1;
  }
  const std::string pat(argv[2]);
  int k = 0;
  if (pat.size() == 2 && pat[0] == 'P' && pat[1] >= '1' && pat[1] <= '8') k = pat[1] - '0';
  std::printf("Subgraph matching \n");
  if (k == 0) {
    std::printf("Not support.\n");
    return 1;
  }
  mc_graph_t *hg = nullptr;
  int rc = mc_graph_load(argv[1], &hg);
  if (rc != MC_OK) return fail("loading the graph", rc);
  int64_t n = 0, nnz = 0, md = 0;
  mc_graph_info(hg, &n, &nnz, &md);
  std::printf("|V|: %" PRId64 ", |E|: %" PRId64 ", Max Degree: %" PRId64 "\n", n, nnz, md);
  mc_dgraph_t *dg = nullptr;
  rc = mc_dgraph_create(mc_graph_rowptr(hg), mc_graph_col(hg), n, nnz, nullptr, 0, &dg);
  if (rc != MC_OK) {
    mc_graph_free(hg);
    return fail("uploading the graph", rc);
  }
  uint64_t total = 0;
  mc_timing_t t{};
  rc = mc_pattern_count(dg, k, &total, &t);
  if (rc != MC_OK) {
    mc_dgraph_free(dg);
    mc_graph_free(hg);
    return fail("counting", rc);
  }
  std::printf("Rank:0 runtime  = %g sec\n", t.count_ms / 1e3);
  std::printf("Total runtime  = %g sec\n", t.count_ms / 1e3);
  std::printf("total_num_triangles = %" PRIu64 "\n", total);
  mc_dgraph_free(dg);
  mc_graph_free(hg);
  return 0;
}
