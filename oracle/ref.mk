# Builds the libWetCloth reference Core straight from its sources (read in
# place, never copied) plus the harness oracle/ref_harness.cpp into two shared
# libraries under oracle/_ref/:
#   libwcref.so      serial stand-in for TBB  -> bitwise reproducible (fixtures)
#   libwcref_omp.so  OpenMP stand-in for TBB  -> timed CPU baseline
# Test infrastructure only.  Usage:  make -f oracle/ref.mk -j8 [REF=/path/to/libwetcloth]
REF ?= /root/reference
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
OUT := $(HERE)_ref
CORE := $(REF)/libWetCloth/Core

SRCS := $(shell find $(CORE) -name '*.cpp' | sort)
OBJS_S := $(patsubst $(CORE)/%.cpp,$(OUT)/obj-serial/%.o,$(SRCS))
OBJS_P := $(patsubst $(CORE)/%.cpp,$(OUT)/obj-omp/%.o,$(SRCS))

CXX ?= g++
# Same definitions as the reference's Release build (CMakeLists.txt): -O3,
# NDEBUG, no Eigen alignment.  No -march flags, so no FMA contraction.
BASEFLAGS := -std=c++14 -O3 -fPIC -DNDEBUG -DEIGEN_DONT_ALIGN \
  -DEIGEN_DONT_ALIGN_STATICALLY -DLIBWETCLOTH_VERSION=\"2018\" \
  -include $(HERE)refshim/compat.h -I$(HERE)refshim -I$(REF)/include \
  -I$(REF)/include/eigen -I$(CORE) -w
SFLAGS := $(BASEFLAGS)
PFLAGS := $(BASEFLAGS) -fopenmp -DWCREF_OMP
# Link the process-wide shared libstdc++ (the one Python already has loaded)
# rather than a private static copy, so std::cout and locales are shared.
STDCXX := $(firstword $(wildcard /usr/lib/x86_64-linux-gnu/libstdc++.so.6 /usr/lib64/libstdc++.so.6))
# OpenMP runtime linked directly (the compiler driver's libgomp.spec may be absent)
GOMP := $(firstword $(wildcard /usr/lib/x86_64-linux-gnu/libgomp.so.1 /usr/lib64/libgomp.so.1))

# The compiled reference-side binding (binding/GpuWetClothCore.h) with its
# test harness, linked against the serial reference and libwcgpu.so.
WCGPU_DIR := $(abspath $(HERE)../libwetcloth_b200)
BFLAGS := $(SFLAGS) -I$(HERE)binding -I$(HERE)../include

all: $(OUT)/libwcref.so $(OUT)/libwcref_omp.so $(OUT)/libwcbinding.so

$(OUT)/obj-serial/%.o: $(CORE)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(SFLAGS) -c $< -o $@

$(OUT)/obj-omp/%.o: $(CORE)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(PFLAGS) -c $< -o $@

$(OUT)/harness-serial.o: $(HERE)ref_harness.cpp
	@mkdir -p $(OUT)
	$(CXX) $(SFLAGS) -c $< -o $@

$(OUT)/harness-omp.o: $(HERE)ref_harness.cpp
	@mkdir -p $(OUT)
	$(CXX) $(PFLAGS) -c $< -o $@

$(OUT)/libwcref.so: $(OBJS_S) $(OUT)/harness-serial.o
	$(CXX) -shared -o $@ $^ $(STDCXX) -lpthread

$(OUT)/libwcref_omp.so: $(OBJS_P) $(OUT)/harness-omp.o
	$(CXX) -shared -o $@ $^ $(STDCXX) $(GOMP) -lpthread

.PHONY: all

$(OUT)/binding-harness.o: $(HERE)binding/binding_harness.cpp $(HERE)binding/GpuWetClothCore.h $(HERE)../include/wetcloth_gpu.h
	@mkdir -p $(OUT)
	$(CXX) $(BFLAGS) -c $< -o $@

$(OUT)/libwcbinding.so: $(OUT)/binding-harness.o $(OUT)/libwcref.so $(WCGPU_DIR)/libwcgpu.so
	$(CXX) -shared -o $@ $(OUT)/binding-harness.o -L$(OUT) -lwcref -L$(WCGPU_DIR) -lwcgpu \
	  -Wl,-rpath,'$$ORIGIN' -Wl,-rpath,'$$ORIGIN/../../libwetcloth_b200' $(STDCXX) -lpthread
