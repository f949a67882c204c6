# Builds the reference's CUDA path (YRT-PET 2.0.7 with BUILD_CUDA) straight
# from its sources with nvcc and g++, without its CMake project, into
# oracle/_ref_cuda/.  Test infrastructure only: the reference's own GPU
# projectors and OSEM_GPU driver, run on the same inputs as the product
# library, check results (second oracle) and give the "plain single-frame GPU
# form" that the benchmark times beside the product.  Never linked into the
# product.
#
#   make -f oracle/ref_cuda.mk -j8 REF=<yrt-pet source tree> JSON_HPP=<nlohmann/json.hpp>
#
# The CUDA sources are compiled for sm_100a only (the reference's CMake takes
# the architecture from CMAKE_CUDA_ARCHITECTURES; its CUDA flags are otherwise
# empty, so nvcc's defaults apply).  Every C++ source is compiled with
# BUILD_CUDA defined, as the reference's CMake does when USE_CUDA=ON, so that
# createOSEM(scanner, true) and the util::forwProject/backProject GPU branch
# exist.  The CUDA headers go on the C++ include path because the reference's
# .cpp files include cuda_runtime.h through GPUUtils.cuh.
ifndef REF
$(error REF=<path of the yrt-pet source tree> is required)
endif
OUT      ?= oracle/_ref_cuda
NVCC     ?= nvcc
CXX      ?= g++
CUDA_DIR := $(patsubst %/bin/,%,$(dir $(shell command -v $(NVCC))))
ARCH     := -gencode arch=compute_100a,code=sm_100a
DEFS     := -DHAVE_ZLIB -DBUILD_CUDA
INCS     := -I$(REF)/include -I$(OUT)/include -I$(CUDA_DIR)/include
CXXFLAGS := -O3 -std=c++20 -fPIC -w $(DEFS) $(INCS)
NVFLAGS  := -O3 -std=c++20 $(ARCH) -Xcompiler -fPIC -w $(DEFS) $(INCS)

CPP_SRCS := $(shell find $(REF)/src -name '*.cpp' ! -name 'pybind11.cpp' | sort)
CU_SRCS  := $(shell find $(REF)/src -name '*.cu' | sort)
OBJS     := $(patsubst $(REF)/src/%.cpp,$(OUT)/obj/%.o,$(CPP_SRCS)) \
            $(patsubst $(REF)/src/%.cu,$(OUT)/obj/%.cu.o,$(CU_SRCS))

all: $(OUT)/libyrtref_cuda.a $(OUT)/libyrtref_gpu_harness.so $(OUT)/libyrtref_b200_harness.so

$(OUT)/include/nlohmann/json.hpp:
ifndef JSON_HPP
	$(error JSON_HPP=<path of nlohmann/json.hpp 3.11> is required)
endif
	@mkdir -p $(OUT)/include/nlohmann $(OUT)/include/yrt-pet
	cp $(JSON_HPP) $@
	printf '#pragma once\n#include "json.hpp"\n' > $(OUT)/include/nlohmann/json_fwd.hpp
	printf '#pragma once\n#define YRT_PET_VERSION_STRING "%s"\n' "$$(tr -d '[:space:]' < $(REF)/VERSION.txt)" > $(OUT)/include/yrt-pet/version.h

$(OUT)/obj/%.o: $(REF)/src/%.cpp $(OUT)/include/nlohmann/json.hpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/obj/%.cu.o: $(REF)/src/%.cu $(OUT)/include/nlohmann/json.hpp
	@mkdir -p $(dir $@)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(OUT)/libyrtref_cuda.a: $(OBJS)
	rm -f $@ && ar rcs $@ $^

# The harness (oracle/ref_harness.cpp with REF_HARNESS_GPU defined) is a
# shared library loaded through ctypes: the reference archive is linked whole,
# with symbols bound inside the library (-Bsymbolic, --exclude-libs) so that it
# cannot interpose on the Python process or on the CPU reference harness, and
# the CUDA runtime linked statically.
$(OUT)/libyrtref_gpu_harness.so: oracle/ref_harness.cpp $(OUT)/libyrtref_cuda.a
	$(CXX) $(CXXFLAGS) -DREF_HARNESS_GPU -shared $< -o $@ -Wl,--whole-archive $(OUT)/libyrtref_cuda.a -Wl,--no-whole-archive -L$(CUDA_DIR)/lib64 -lcudart_static -lz -lpthread -ldl -lrt -Wl,-Bsymbolic -Wl,--exclude-libs,ALL

# The reference's drivers on the product's binding (REF_HARNESS_B200):
# OSEM_GPU_B200 / OperatorProjectorB200 (yrt-pet_b200/binding, compiled by its
# own recipe) over libyrtb.so, found at run time next to this tree's copy.
B200_OBJ := yrt-pet_b200/lib/yrtb_yrtpet.o
LIBYRTB  := yrt-pet_b200/lib/libyrtb.so

$(B200_OBJ): yrt-pet_b200/binding/yrtb_yrtpet.cu yrt-pet_b200/binding/yrtb_yrtpet.cuh include/yrt_b200.h $(OUT)/include/nlohmann/json.hpp
	$(MAKE) -f yrt-pet_b200/binding/binding.mk REF=$(REF) INC="-I$(OUT)/include" NVCC=$(NVCC)

$(OUT)/obj/ref_harness_b200.o: oracle/ref_harness.cpp yrt-pet_b200/binding/yrtb_yrtpet.cuh include/yrt_b200.h $(OUT)/include/nlohmann/json.hpp
	@mkdir -p $(dir $@)
	$(NVCC) $(NVFLAGS) -Iinclude -Iyrt-pet_b200/binding -DREF_HARNESS_GPU -DREF_HARNESS_B200 -x cu -c $< -o $@

$(OUT)/libyrtref_b200_harness.so: $(OUT)/obj/ref_harness_b200.o $(OUT)/libyrtref_cuda.a $(B200_OBJ) $(LIBYRTB)
	$(CXX) -shared $(OUT)/obj/ref_harness_b200.o $(B200_OBJ) -o $@ \
	    -Wl,--whole-archive $(OUT)/libyrtref_cuda.a -Wl,--no-whole-archive \
	    -Lyrt-pet_b200/lib -lyrtb -L$(CUDA_DIR)/lib64 -lcudart_static -lz -lpthread -ldl -lrt \
	    -Wl,-rpath,'$$ORIGIN/../../yrt-pet_b200/lib' -Wl,-Bsymbolic -Wl,--exclude-libs,ALL

.PHONY: all
