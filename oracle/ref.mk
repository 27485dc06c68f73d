# Builds oracle/_ref/libufo_ref.so: the reference's own filter/backproject task
# sources and OpenCL kernels (plus the flat-field and cone-beam weight kernels)
# compiled for the CPU from where they lie under the
# reference tree, against the shims in refshim/.  Kernel sources get one
# mechanical rewrite (OpenCL vector literals "(float2)(a, b)" -> make_float2(a, b))
# into _ref/gen/; nothing is copied into the repository.  Test infrastructure only.
REF ?= /root/reference
OUT := _ref
GEN := $(OUT)/gen
CC := gcc
CXX := g++
CFLAGS := -O2 -fopenmp -fPIC -w -Irefshim -I$(REF)/src -I$(REF)/src/common
CXXFLAGS := -O2 -fopenmp -fPIC -std=c++17 -w -mfma -ffp-contract=fast -Irefshim -I$(REF)/src -I$(GEN)
KERNELS := backproject filter fft forwardproject
KERNELS_PRE := ffc conebeam

all: $(OUT)/libufo_ref.so

$(GEN)/%.cl.cpp: $(REF)/src/kernels/%.cl
	@mkdir -p $(GEN)
	sed -E 's/\((float[24])\) *\(/make_\1(/g' $< > $@

$(OUT)/kernels.o: refshim/ref_kernels.cpp refshim/clc_shim.hpp refshim/clc_types.hpp $(KERNELS:%=$(GEN)/%.cl.cpp)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/kernels_pre.o: refshim/ref_kernels_pre.cpp refshim/clc_shim.hpp refshim/clc_types.hpp $(KERNELS_PRE:%=$(GEN)/%.cl.cpp)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/runtime.o: refshim/ref_runtime.cpp refshim/refshim_internal.h refshim/clc_types.hpp
	@mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/filter_task.o: refshim/ref_filter_task.c refshim/refshim_internal.h $(REF)/src/ufo-filter-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/backproject_task.o: refshim/ref_backproject_task.c refshim/refshim_internal.h $(REF)/src/ufo-backproject-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/libufo_ref.so: $(OUT)/kernels.o $(OUT)/kernels_pre.o $(OUT)/runtime.o $(OUT)/filter_task.o $(OUT)/backproject_task.o
	$(CXX) -shared -fopenmp -o $@ $^

clean:
	rm -rf $(OUT)

.PHONY: all clean
