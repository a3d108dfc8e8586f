# Compiles the reference's own triangle-count program from its sources where
# they lie (read-only) into oracle/_ref/, for sm_100a, without the reference's
# own build system.  Outputs only go to _ref/ (git-ignored; it travels to the
# GPU machine with the rest of the tree).  Used to pin parity against the
# reference itself and to time it on the same GPU.
# REF: the reference checkout (pass REF=...; default: "reference" beside the
# repository root).
REF ?= $(abspath ../../reference)
OUT := _ref
NVCC ?= nvcc
CXX := g++
ARCH := -gencode arch=compute_100a,code=sm_100a
INC := -I$(REF)/include -I$(REF)/gpu_kernels
CXXFLAGS := -O3 -std=c++14 -fopenmp -w $(INC)
NVFLAGS := -O3 -w $(ARCH) -DUSE_GPU $(INC)

all: $(OUT)/tc_challenge $(OUT)/sm_patterns

$(OUT):
	mkdir -p $(OUT)

$(OUT)/%.o: $(REF)/%.cc | $(OUT)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/tc_challenge.o: $(REF)/tc_challenge.cu | $(OUT)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/tc_challenge: $(OUT)/main.o $(OUT)/graph.o $(OUT)/VertexSet.o $(OUT)/tc_challenge.o
	$(NVCC) $(ARCH) $^ -o $@ -lgomp

# The pattern kernels run through a one-rank shim (no MPI) that follows the
# reference host driver; see ref_sm_shim.cu.
$(OUT)/ref_sm_shim.o: ref_sm_shim.cu | $(OUT)
	$(NVCC) $(NVFLAGS) -I$(REF)/subgraph_matching -c $< -o $@

$(OUT)/sm_patterns: $(OUT)/graph.o $(OUT)/VertexSet.o $(OUT)/ref_sm_shim.o
	$(NVCC) $(ARCH) $^ -o $@ -lgomp

.PHONY: all
