// ORACLE -- test infrastructure, not product code.
//
// One-rank host driver for the reference's own pattern kernels
// (subgraph_matching/pattern_kernels.cuh, included unmodified from the
// reference tree by oracle/ref.mk).  It follows the host flow of
// SMSolverMultiGPU (subgraph_matching/sm_multigpu.cu:97-221) with nranks = 1
// and without MPI: the whole COO edge list is the rank's task list, so the
// round-robin split (and its nnz > 8192 assert, :18) is not needed.
//   usage: sm_patterns <graph_prefix> <P1..P8>
// Prints "Total runtime  = X sec" and "total_num_triangles = N" like the
// reference program (subgraph_matching/main_mpi.cpp:35-36).
#include <cub/cub.cuh>

#include "timer.h"
#include "edgelist.h"
#include "graph_gpu.h"
#include "operations.cuh"
#include "cuda_launch_config.hpp"

typedef cub::BlockReduce<AccType, BLOCK_SIZE> BlockReduce;
#include "pattern_kernels.cuh"

int main(int argc, char *argv[]) {
  if (argc < 3) {
    std::cout << "usage: " << argv[0] << " <graph> <P1..P8>\n";
    return 1;
  }
  Graph g(argv[1]);
  const std::string pattern(argv[2]);
  const auto nv = g.num_vertices();
  const auto md = g.get_max_degree();
  const int nblocks = 1024, nthreads = 256, list_num = 8;

  size_t per_block = WARPS_PER_BLOCK * list_num * size_t(md) * sizeof(int);
  AccType first_task = nblocks * nthreads / WARP_SIZE;
  int *frontier = nullptr;
  CUDA_SAFE_CALL(cudaMalloc((void **)&frontier, nblocks * per_block));
  AccType *index0, *index1;
  CUDA_SAFE_CALL(cudaMalloc((void **)&index0, sizeof(AccType)));
  CUDA_SAFE_CALL(cudaMalloc((void **)&index1, sizeof(AccType)));
  CUDA_SAFE_CALL(cudaMemcpy(index0, &first_task, sizeof(AccType), cudaMemcpyHostToDevice));
  CUDA_SAFE_CALL(cudaMemcpy(index1, &first_task, sizeof(AccType), cudaMemcpyHostToDevice));
  std::vector<AccType> h_total(6, 0);
  AccType *d_total;
  CUDA_SAFE_CALL(cudaMalloc((void **)&d_total, sizeof(AccType) * 6));
  CUDA_SAFE_CALL(cudaMemcpy(d_total, h_total.data(), sizeof(AccType) * 6, cudaMemcpyHostToDevice));

  const eidType nnz = g.init_edgelist();
  std::vector<eidType> lens(1, nnz);
  std::vector<vidType *> srcs(1, g.get_src_ptr()), dsts(1, g.get_dst_ptr());
  GraphGPU gg(g);
  gg.copy_edgelist_to_device(lens, srcs, dsts, 0);
  const int ne = (int)nnz;

  Timer t;
  t.Start();
  if (pattern == "P1") {
    P1_frequency_count<<<nblocks, nthreads>>>(nv, gg, frontier, md, d_total, index0);
    P1_count_correction<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index1);
  } else if (pattern == "P2") {
    P2_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P3") {
    P3_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P4") {
    P4_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P5") {
    P5_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P6") {
    P6_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P7") {
    P7_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else if (pattern == "P8") {
    P8_subgraph_matching<<<nblocks, nthreads>>>(ne, gg, frontier, md, d_total, index0);
  } else {
    std::cout << "Not support." << std::endl;
    return 1;
  }
  CUDA_SAFE_CALL(cudaDeviceSynchronize());
  t.Stop();
  CUDA_SAFE_CALL(cudaMemcpy(h_total.data(), d_total, sizeof(AccType) * 6, cudaMemcpyDeviceToHost));
  AccType total = 0;
  if (pattern == "P4" || pattern == "P6") total = h_total[1];
  else total = h_total[1] - h_total[2];
  std::cout << "Total runtime  = " << t.Seconds() << " sec\n";
  std::cout << "total_num_triangles = " << total << "\n";
  return 0;
}
