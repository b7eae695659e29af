# Builds the reference's out-of-core `GEM` binary from its own sources, where
# they lie, into oracle/_ref/GEM_ooc — test and measurement infrastructure:
# its stdout times the reference's own host-side (OpenMP) filter and
# edge-table build (`Filter time`, `construct time`) and its GPU join
# (`Join Time`), on a GPU machine.  A recipe of our own; the reference's CMake
# build is not run.  Its settings restated for this toolchain: CUDA 12.9 at
# /usr/local/cuda, sm_100a, separable compilation, -O3, OpenMP (-fopenmp,
# libgomp), --extended-lambda for the structure library; the dead
# lib/filter/src/filter_kernel.cu is left out (no symbol of it is used, and
# its kernels exceed the static shared-memory limit).
#   make -f oracle/ref/Makefile.ooc REF=/root/reference
REF    ?= /root/reference
OOC    := $(REF)/out-of-core
OUT    ?= $(dir $(lastword $(MAKEFILE_LIST)))../_ref
OBJ    := $(OUT)/obj_ooc
NVCC   ?= /usr/local/cuda/bin/nvcc
INC    := $(foreach d,utils graph io structure filter plan join,-I$(OOC)/lib/$(d)/include) -I$(OOC)/include
NVFLAGS := -O3 -std=c++17 -rdc=true -gencode arch=compute_100a,code=sm_100a -w --extended-lambda \
           -Xcompiler -fopenmp $(INC)
CXXFLAGS := -O3 -std=c++17 -w -fopenmp $(INC) -I/usr/local/cuda/include

CU_SRC  := lib/utils/src/cuda_helpers.cu lib/utils/src/globals.cu lib/io/src/io.cu \
           lib/structure/src/construct_kernel.cu lib/structure/src/cuckooHash.cu \
           lib/structure/src/memory_manager.cu lib/structure/src/host_memory_manager.cu \
           lib/structure/src/unifiedTrie.cu lib/filter/src/filter.cu \
           lib/join/src/join_trie.cu lib/join/src/join_trie_kernel.cu src/main.cu
CPP_SRC := lib/graph/src/cpuGraph.cpp lib/graph/src/gpuGraph.cpp lib/plan/src/relax.cpp \
           lib/structure/src/lattice.cpp lib/structure/src/policy.cpp

CU_OBJ  := $(addprefix $(OBJ)/,$(subst /,_,$(CU_SRC:.cu=.o)))
CPP_OBJ := $(addprefix $(OBJ)/,$(subst /,_,$(CPP_SRC:.cpp=.o)))

all: $(OUT)/GEM_ooc

$(OBJ):
	mkdir -p $(OBJ)

define cu_rule
$(OBJ)/$(subst /,_,$(1:.cu=.o)): $(OOC)/$(1) | $(OBJ)
	$(NVCC) $(NVFLAGS) -c $$< -o $$@
endef
define cpp_rule
$(OBJ)/$(subst /,_,$(1:.cpp=.o)): $(OOC)/$(1) | $(OBJ)
	g++ $(CXXFLAGS) -c $$< -o $$@
endef
$(foreach s,$(CU_SRC),$(eval $(call cu_rule,$(s))))
$(foreach s,$(CPP_SRC),$(eval $(call cpp_rule,$(s))))

$(OUT)/GEM_ooc: $(CU_OBJ) $(CPP_OBJ)
	$(NVCC) -rdc=true -gencode arch=compute_100a,code=sm_100a $^ -o $@ -Xcompiler -fopenmp -lgomp

clean:
	rm -rf $(OBJ) $(OUT)/GEM_ooc
.PHONY: all clean
