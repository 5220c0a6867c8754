# desert-search-b200 build.  `make` builds the CUDA library (sm_100a), the host tools and the test
# oracle; `make ref` additionally compiles the reference's own sources in place into oracle/_ref
# (needs the reference checkout: oracle/ref.mk holds its default location, REF=... overrides it).
NVCC     ?= nvcc
CXX      ?= g++
PY       ?= python3
PKG      := desert-search_b200
B        := _build
GPUARCH  := -gencode arch=compute_100a,code=sm_100a
# -fmad=false: every product kernel states its fused multiply-adds explicitly (__fmaf_rn / __fma_rn),
# so results are fixed by the source, as the bit-exact contract with the CPU path requires.
NVFLAGS  := -O3 -std=c++20 $(GPUARCH) -lineinfo -fmad=false -Xptxas -v -Xcompiler -fPIC -I$(PKG)/csrc -Iinclude
HOSTFLAGS:= -I/usr/local/cuda/include -O3 -march=x86-64-v3 -ffp-contract=off -std=c++20 -pthread -Iinclude -I$(PKG)/csrc
ORCFLAGS := -O3 -march=x86-64-v3 -ffp-contract=off -std=c++20 -pthread -fPIC

CU_SRC   := $(wildcard $(PKG)/csrc/*.cu)
CU_HDR   := $(wildcard $(PKG)/csrc/*.cuh) $(wildcard $(PKG)/csrc/*.h) $(wildcard include/*.h)
CU_OBJ   := $(patsubst $(PKG)/csrc/%.cu,$(B)/%.o,$(CU_SRC))
LIB      := $(PKG)/lib/libdsgpu.so
HOST_BIN := $(patsubst $(PKG)/host/%.cpp,$(PKG)/bin/%,$(wildcard $(PKG)/host/*.cpp))
ORC_LIB  := oracle/liborc.so

all: $(LIB) $(HOST_BIN) $(ORC_LIB)
lib: $(LIB)
oracle: $(ORC_LIB)
ref:
	$(MAKE) -f oracle/ref.mk $(if $(REF),REF=$(REF))

$(B) $(PKG)/lib $(PKG)/bin:
	mkdir -p $@

$(B)/dsw_blob.c: $(PKG)/data/worldgen.bin $(PKG)/data/embed_blob.py | $(B)
	$(PY) $(PKG)/data/embed_blob.py $< $@ dsw_worldgen_blob
$(B)/orc_blob.c: $(PKG)/data/worldgen.bin $(PKG)/data/embed_blob.py | $(B)
	$(PY) $(PKG)/data/embed_blob.py $< $@ orc_worldgen_blob
$(B)/dsw_blob.o: $(B)/dsw_blob.c
	gcc -O1 -fPIC -c $< -o $@
$(B)/orc_blob.o: $(B)/orc_blob.c
	gcc -O1 -fPIC -c $< -o $@

# ---- CUDA library (C ABI in include/dsgpu.h)
# taps.cu keeps nvcc's default contraction: it evaluates expf exactly as the reference kernels do.
$(B)/taps.o: $(PKG)/csrc/taps.cu $(CU_HDR) | $(B)
	$(NVCC) $(filter-out -fmad=false,$(NVFLAGS)) -c $< -o $@ 2> $(B)/taps.ptxas.txt || (cat $(B)/taps.ptxas.txt; false)
# proxy_f32.cu likewise: the FP32 proxy of the reference's GPU engine, with the engine's contraction.
$(B)/proxy_f32.o: $(PKG)/csrc/proxy_f32.cu $(CU_HDR) | $(B)
	$(NVCC) $(filter-out -fmad=false,$(NVFLAGS)) -c $< -o $@ 2> $(B)/proxy_f32.ptxas.txt || (cat $(B)/proxy_f32.ptxas.txt; false)
$(B)/%.o: $(PKG)/csrc/%.cu $(CU_HDR) | $(B)
	$(NVCC) $(NVFLAGS) -c $< -o $@ 2> $(B)/$*.ptxas.txt || (cat $(B)/$*.ptxas.txt; false)
$(B)/host_%.o: $(PKG)/csrc/%.cpp $(CU_HDR) | $(B)
	$(CXX) $(HOSTFLAGS) -fPIC -c $< -o $@
$(LIB): $(CU_OBJ) $(patsubst $(PKG)/csrc/%.cpp,$(B)/host_%.o,$(wildcard $(PKG)/csrc/*.cpp)) $(B)/dsw_blob.o | $(PKG)/lib
	$(NVCC) $(GPUARCH) -shared -o $@ $^ -lcudart_static -lpthread -ldl -lrt

# ---- host tools (C++; reach the GPU only through the C ABI)
$(PKG)/bin/%: $(PKG)/host/%.cpp $(wildcard $(PKG)/host/*.hpp) include/dsgpu.h $(LIB) | $(PKG)/bin
	$(CXX) $(HOSTFLAGS) $< -o $@ -L$(PKG)/lib -ldsgpu -Wl,-rpath,'$$ORIGIN/../lib'

# ---- oracle (test infrastructure)
$(ORC_LIB): oracle/orc_capi.cpp oracle/orc_core.hpp oracle/orc_data.hpp $(B)/orc_blob.o
	$(CXX) $(ORCFLAGS) -shared oracle/orc_capi.cpp $(B)/orc_blob.o -o $@

clean:
	rm -rf $(B) $(PKG)/lib $(PKG)/bin $(ORC_LIB)

.PHONY: all lib oracle ref clean
