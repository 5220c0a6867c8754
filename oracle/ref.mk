# Builds the reference's own code from its sources where they lie (REF, read-only) into oracle/_ref/.
# Test infrastructure only: the outputs pin the oracle and serve as the timed CPU reference arm.
# Flags follow the reference Makefile (-ffp-contract=off is what makes its sampler round like Java);
# -march=x86-64-v3 (its `bundle` target's host flags) instead of -march=native so the binaries run on
# any AVX2 host the build is copied to.  This recipe is the one place that knows where the reference checkout
# lies by default; `make ref REF=...` (or REF in the environment) points it elsewhere.  Without a checkout
# it builds nothing (the GPU machines use the binaries built here).
REF      ?= /root/reference
OUT      := oracle/_ref
CXXFLAGS := -O3 -march=x86-64-v3 -ffp-contract=off -std=c++20 -pthread -I$(REF)/src
NVCC     ?= nvcc
GPUARCH  := -gencode arch=compute_100a,code=sm_100a

REFHDR := $(wildcard $(REF)/src/*.hpp) $(REF)/src/dsearch_desert.cpp

ifeq ($(wildcard $(REF)/src/dsearch_desert.cpp),)
all:
	@echo "oracle/ref.mk: no reference checkout at REF=$(REF); oracle/_ref not rebuilt"
else
all: $(OUT)/dsearch_desert $(OUT)/dflood $(OUT)/libref_cpu.so $(OUT)/libref_gate.so $(OUT)/tgate $(OUT)/dsearch_desert_gpu $(OUT)/dsearch_desert_shim

$(OUT):
	mkdir -p $@
$(OUT)/dsearch_desert: $(REF)/src/dsearch_desert.cpp $(REFHDR) | $(OUT)
	g++ $(CXXFLAGS) $< -o $@
$(OUT)/dflood: $(REF)/tools/dflood.cpp $(REFHDR) | $(OUT)
	g++ $(CXXFLAGS) $< -o $@
$(OUT)/libref_cpu.so: oracle/ref/ref_cpu.cpp $(REFHDR) | $(OUT)
	g++ $(CXXFLAGS) -fPIC -shared $< -o $@
# The reference GPU gate for sm_100a (its Makefile uses -arch=native; the compute capability is the only change).
$(OUT)/libref_gate.so: oracle/ref/ref_gate.cu $(REF)/src/gpu/gate.cuh $(REF)/src/gpu/tgate.cu | $(OUT)
	$(NVCC) -O3 -std=c++20 $(GPUARCH) -I$(REF)/src -Xcompiler -fPIC -shared $< -o $@
$(OUT)/tgate: $(REF)/src/gpu/tgate.cu $(REF)/src/gpu/gate.cuh | $(OUT)
	$(NVCC) -O3 -std=c++20 $(GPUARCH) $< -o $@

.PHONY: all

# The reference's unmodified searcher with -DDRIP_GPU linked against this repository's engine instead of its own:
# the gproxy interface (its header) implemented over libdsgpu's C ABI (desert-search_b200/shim/gproxy_dsgpu.cpp).
SHIM := desert-search_b200/shim/gproxy_dsgpu.cpp
DSGLIB := desert-search_b200/lib/libdsgpu.so
$(OUT)/dsearch_desert_shim: $(REF)/src/dsearch_desert.cpp $(REFHDR) $(REF)/src/gpu/gproxy.h $(SHIM) include/dsgpu.h $(DSGLIB) | $(OUT)
	g++ $(CXXFLAGS) -DDRIP_GPU -I$(REF)/src/gpu -Iinclude $(REF)/src/dsearch_desert.cpp $(SHIM) -L$(dir $(DSGLIB)) -ldsgpu \
	    -Wl,-rpath,'$$ORIGIN/../../desert-search_b200/lib' -o $@

# The reference's GPU searcher (Makefile:43-46): its engine gproxy.cu for sm_100a, the searcher with -DDRIP_GPU.
$(OUT)/gproxy.o: $(REF)/src/gpu/gproxy.cu $(REF)/src/gpu/gate.cuh $(REF)/src/gpu/gproxy.h | $(OUT)
	$(NVCC) -O3 -std=c++20 $(GPUARCH) -c $< -o $@
$(OUT)/dsearch_desert_gpu: $(REF)/src/dsearch_desert.cpp $(REFHDR) $(OUT)/gproxy.o | $(OUT)
	g++ $(CXXFLAGS) -DDRIP_GPU -I/usr/local/cuda/include $< $(OUT)/gproxy.o -L/usr/local/cuda/lib64 -lcudart_static -ldl -lrt -o $@
endif
