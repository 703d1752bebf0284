# The reference's evaluation harness (evaluation/universal_bench*.cu, unchanged),
# built against this library through include/universal_bench/gpu_masstree_adapter.hpp
# (found before the reference's own adapter on the include path).  Measurement
# infrastructure: it runs the reference's harness phases (lookup, scan, update,
# insert/delete, mixed, YCSB, space) on libmt_b200.so; the reference's own GPU
# index is not run.  Output only under oracle/_ref/.
#   make -f oracle/universal_bench.mk        -> oracle/_ref/universal_bench
REF ?= /root/reference
ROOT := $(abspath $(dir $(lastword $(MAKEFILE_LIST)))/..)
OUT := $(ROOT)/oracle/_ref
EVAL := $(REF)/evaluation
NVCC ?= nvcc
FLAGS := -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a -maxrregcount=64 \
         --expt-extended-lambda --expt-relaxed-constexpr \
         -I$(ROOT)/include/universal_bench -I$(EVAL) -I$(REF)/include
TUS := universal_bench universal_bench_gpu_masstree universal_bench_gpu_chainhashtable \
       universal_bench_gpu_cuckoohashtable universal_bench_gpu_extendhashtable
OBJS := $(addprefix $(OUT)/,$(addsuffix .o,$(TUS)))

all: $(OUT)/universal_bench

$(OUT)/%.o: $(EVAL)/%.cu $(ROOT)/include/universal_bench/gpu_masstree_adapter.hpp
	mkdir -p $(OUT)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/universal_bench: $(OBJS)
	$(NVCC) -gencode arch=compute_100a,code=sm_100a $(OBJS) -o $@ -L$(ROOT)/indexingpu_b200 -lmt_b200 \
	  -lstdc++fs -Xlinker -rpath -Xlinker $(ROOT)/indexingpu_b200

.PHONY: all
