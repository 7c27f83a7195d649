# Builds the libuw12 reference from its unmodified sources -- TEST
# INFRASTRUCTURE ONLY (the checker and the CPU baseline; never product code).
#
#   make -f oracle/ref.mk REF=<libuw12 source tree>
#
# Inputs: libuw12's src/**/*.cpp and libuw12.cpp where they lie under $(REF)
# (nothing is copied), the project's own Armadillo-subset header
# (oracle/refshim/armadillo) and the OpenBLAS that scipy ships (LP64,
# symbols prefixed "scipy_"). libuw12's CMake-generated config.hpp
# (src/config.hpp.in: LINALG_KEY, PARALLEL_KEY, source_dir) is written here
# with USE_ARMA and USE_OMP, the reference's OpenMP build.
# Outputs (git-ignored):
#   oracle/_ref/libuw12_ref.so         parity build, libuw12's own parallel.hpp
#   oracle/_ref/libuw12_ref_timing.so  timing build: the same sources with the
#       loop dispatcher oracle/refshim/timing/utils/parallel.hpp first on the
#       include path (full or sampled loops, for the CPU baseline)

REF ?= /root/reference
HERE := $(patsubst %/,%,$(dir $(abspath $(lastword $(MAKEFILE_LIST)))))
OUT := $(HERE)/_ref
PY ?= python3
REFCXX ?= /usr/bin/g++
BLAS_DIR := $(shell $(PY) -c "import os, scipy; print(os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), os.pardir, 'scipy.libs')))")
BLAS_LIB := $(firstword $(wildcard $(BLAS_DIR)/libscipy_openblas-*.so))

SRCS := $(REF)/src/integrals/base_integrals.cpp \
        $(REF)/src/integrals/integrals.cpp \
        $(REF)/src/two_electron/two_electron.cpp \
        $(REF)/src/three_electron/direct_utils.cpp \
        $(REF)/src/three_electron/indirect_utils.cpp \
        $(REF)/src/three_electron/three_electron.cpp \
        $(REF)/src/four_electron/four_electron_utils.cpp \
        $(REF)/src/four_electron/four_electron.cpp \
        $(REF)/src/uw12.cpp \
        $(REF)/libuw12.cpp
OBJS := $(patsubst $(REF)/%.cpp,$(OUT)/obj/%.o,$(SRCS)) $(OUT)/obj/ref_capi.o
TOBJS := $(patsubst $(REF)/%.cpp,$(OUT)/tobj/%.o,$(SRCS)) $(OUT)/tobj/ref_capi.o

CXXFLAGS := -std=c++17 -O3 -DNDEBUG -fPIC -fopenmp -w \
            -DUW12REF_BLAS_PREFIX=scipy_ \
            -I$(HERE)/refshim -I$(OUT)/gen -I$(REF)/src -I$(REF)

all: $(OUT)/libuw12_ref.so $(OUT)/libuw12_ref_timing.so

$(OUT)/libuw12_ref.so: $(OBJS)
	@test -n "$(BLAS_LIB)" || (echo "scipy's OpenBLAS not found under $(BLAS_DIR)" && false)
	$(REFCXX) -shared -fopenmp -o $@ $(OBJS) $(BLAS_LIB) -Wl,-rpath,$(BLAS_DIR)

$(OUT)/gen/config.hpp:
	@mkdir -p $(OUT)/gen
	printf '#ifndef CONFIG_HPP\n#define CONFIG_HPP\nconstexpr char source_dir[] = "$(REF)";\n#define USE_ARMA 1\n#define USE_OMP 1\n#endif\n' > $@

$(OUT)/obj/%.o: $(REF)/%.cpp $(OUT)/gen/config.hpp $(HERE)/refshim/armadillo
	@mkdir -p $(dir $@)
	$(REFCXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/ref_capi.o: $(HERE)/refshim/ref_capi.cpp $(OUT)/gen/config.hpp $(HERE)/refshim/armadillo
	@mkdir -p $(dir $@)
	$(REFCXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/libuw12_ref_timing.so: $(TOBJS)
	@test -n "$(BLAS_LIB)" || (echo "scipy's OpenBLAS not found under $(BLAS_DIR)" && false)
	$(REFCXX) -shared -fopenmp -o $@ $(TOBJS) $(BLAS_LIB) -Wl,-rpath,$(BLAS_DIR)

$(OUT)/tobj/%.o: $(REF)/%.cpp $(OUT)/gen/config.hpp $(HERE)/refshim/armadillo $(HERE)/refshim/timing/utils/parallel.hpp
	@mkdir -p $(dir $@)
	$(REFCXX) -I$(HERE)/refshim/timing -DUW12REF_TIMING_BUILD $(CXXFLAGS) -c $< -o $@

$(OUT)/tobj/ref_capi.o: $(HERE)/refshim/ref_capi.cpp $(OUT)/gen/config.hpp $(HERE)/refshim/armadillo $(HERE)/refshim/timing/utils/parallel.hpp
	@mkdir -p $(dir $@)
	$(REFCXX) -I$(HERE)/refshim/timing -DUW12REF_TIMING_BUILD $(CXXFLAGS) -c $< -o $@

.PHONY: all clean
clean:
	rm -rf $(OUT)
