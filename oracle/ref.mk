# Builds oracle/_ref/libufo_ref.so: the reference's own task sources (filter,
# backproject, general-backproject, lamino-backproject, stacked-backproject, with the common/
# helpers they use)
# and OpenCL kernels (plus the flat-field and cone-beam weight kernels) compiled
# for the CPU from where they lie under the reference tree, against the shims
# in refshim/.  Static kernel sources get one mechanical rewrite (OpenCL vector
# literals "(float2)(a, b)" -> make_float2(a, b)) into _ref/gen/; kernels the
# tasks generate at run time are compiled by refshim/ref_clc_jit.cpp into
# _ref/jit/.  Nothing is copied into the repository.  Test infrastructure only.
# The reference tree is taken from UFO_FILTERS_SOURCE when set.
REF ?= $(or $(UFO_FILTERS_SOURCE),/root/reference)
OUT := _ref
GEN := $(OUT)/gen
CC := gcc
CXX := g++
CFLAGS := -O2 -fopenmp -fPIC -w -Irefshim -I$(REF)/src -I$(REF)/src/common
CXXFLAGS := -O2 -fopenmp -fPIC -std=c++17 -w -mfma -ffp-contract=fast -Irefshim -I$(REF)/src -I$(GEN)
KERNELS := backproject filter fft forwardproject
KERNELS_PRE := ffc conebeam
COMMON := ufo-scarray ufo-ctgeometry ufo-conebeam

all: $(OUT)/libufo_ref.so

$(GEN)/%.cl.cpp: $(REF)/src/kernels/%.cl
	@mkdir -p $(GEN)
	sed -E 's/\((float[24])\) *\(/make_\1(/g' $< > $@

$(OUT)/kernels.o: refshim/ref_kernels.cpp refshim/clc_shim.hpp refshim/clc_types.hpp $(KERNELS:%=$(GEN)/%.cl.cpp)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/kernels_pre.o: refshim/ref_kernels_pre.cpp refshim/clc_shim.hpp refshim/clc_types.hpp $(KERNELS_PRE:%=$(GEN)/%.cl.cpp)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/%.o: refshim/%.cpp refshim/refshim_internal.h refshim/clc_types.hpp refshim/glib.h refshim/ufo/ufo.h refshim/CL/cl.h
	@mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/common_%.o: $(REF)/src/common/%.c refshim/glib.h refshim/ufo/ufo.h
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/filter_task.o: refshim/ref_filter_task.c refshim/refshim_internal.h $(REF)/src/ufo-filter-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/backproject_task.o: refshim/ref_backproject_task.c refshim/refshim_internal.h $(REF)/src/ufo-backproject-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/gbp_task.o: refshim/ref_gbp_task.c refshim/refshim_internal.h refshim/glib.h $(REF)/src/ufo-general-backproject-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/stacked_task.o: refshim/ref_stacked_task.c refshim/refshim_internal.h refshim/glib.h $(REF)/src/ufo-stacked-backproject-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/lamino_task.o: refshim/ref_lamino_task.c refshim/refshim_internal.h refshim/glib.h $(REF)/src/ufo-lamino-backproject-task.c
	@mkdir -p $(OUT)
	$(CC) $(CFLAGS) -c $< -o $@

OBJS := $(OUT)/kernels.o $(OUT)/kernels_pre.o $(OUT)/ref_runtime.o $(OUT)/ref_glib.o $(OUT)/ref_clc_jit.o \
	$(OUT)/filter_task.o $(OUT)/backproject_task.o $(OUT)/gbp_task.o $(OUT)/lamino_task.o $(OUT)/stacked_task.o \
	$(COMMON:%=$(OUT)/common_%.o)

$(OUT)/libufo_ref.so: $(OBJS)
	$(CXX) -shared -fopenmp -o $@ $^ -ldl

clean:
	rm -rf $(OUT)

.PHONY: all clean
