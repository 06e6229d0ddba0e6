# Builds the reference's own `codrel` tool (and its super-A fork and the
# ANcandidates pre-filter) from their unmodified sources, in place where they
# lie, into oracle/_ref/.  The reference's CMake files target sm_35/37,
# which CUDA 12.9 no longer accepts, so this recipe calls nvcc on the sources
# directly with sm_100a.  Only the CPU paths (-c, -e 1 -c, -e 2/3/4) are used as
# checker and CPU baseline; nothing here is linked into the product.
#
#   make -f oracle/ref.mk REF=/path/to/coding_reliability
#
# REF is required (oracle/build.py passes $CODREL_REFERENCE, or the checkout
# named `reference` beside this repository).
ifndef REF
$(error REF=<reference checkout> is required)
endif
OUT      ?= $(dir $(lastword $(MAKEFILE_LIST)))_ref
NVCC     ?= nvcc
DD       := $(REF)/distance_distribution
SRC      := $(DD)/src
HELPER   := $(DD)/lib/helper
SUPA     := $(REF)/distance_distribution_super_a

CODREL_SRCS := $(addprefix $(SRC)/,main.cpp globals.cpp hamming.cpp hamming_native.cpp \
    hamming_native_short.cpp hamming_native_short_ordering.cpp hamming_grid.cu hamming.cu \
    hamming_mc.cu an_coding.cu an_coding.cpp an_coding_mc.cu an_coding_grid.cu \
    test_curand.cu rand_gen.cu) \
    $(addprefix $(HELPER)/src/,statistics.cpp timestatistics.cpp timer.cpp)

SUPA_SRCS := $(addprefix $(SUPA)/src/,main.cpp globals.cpp an_coding.cu an_coding_grid.cu) \
    $(addprefix $(SUPA)/lib/helper/src/,statistics.cpp timestatistics.cpp timer.cpp)

FLAGS := -O3 -std=c++17 -w -gencode arch=compute_100a,code=sm_100a -Xcompiler -fopenmp

all: $(OUT)/ref_codrel $(OUT)/ref_codrel_supera $(OUT)/ref_ancandidates

$(OUT)/ref_codrel: $(CODREL_SRCS)
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -I$(HELPER) -I$(HELPER)/inc -o $@ $^ -lcurand -lgomp -lrt

$(OUT)/ref_codrel_supera: $(SUPA_SRCS)
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -I$(SUPA)/lib/helper -I$(SUPA)/lib/helper/inc -o $@ $^ -lgomp -lrt

.PHONY: all

$(OUT)/ref_ancandidates: $(REF)/ANcandidates/ANcandidates.cpp
	@mkdir -p $(OUT)
	g++ -std=c++17 -O3 -w -fopenmp -o $@ $^
