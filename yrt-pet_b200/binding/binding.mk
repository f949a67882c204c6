# Compiles the libyrtb binding for YRT-PET's own C++ classes
# (OperatorProjectorB200, OSEM_GPU_B200: yrt-pet_b200/binding/yrtb_yrtpet.cu)
# against a YRT-PET source tree configured with CUDA, into one object that a
# YRT-PET build links beside libyrtb.so.  A maintainer adding the binding to
# YRT-PET's own CMake project lists yrtb_yrtpet.cu among its CUDA sources
# instead.
#
#   make -f yrt-pet_b200/binding/binding.mk REF=<yrt-pet source tree> INC="-I<dir with nlohmann/json.hpp and yrt-pet/version.h>"
ifndef REF
$(error REF=<path of the yrt-pet source tree> is required)
endif
NVCC ?= nvcc
INC  ?=
OUT  ?= yrt-pet_b200/lib/yrtb_yrtpet.o
SRC  := yrt-pet_b200/binding/yrtb_yrtpet.cu
DEPS := $(SRC) yrt-pet_b200/binding/yrtb_yrtpet.cuh include/yrt_b200.h

$(OUT): $(DEPS)
	@mkdir -p $(dir $@)
	$(NVCC) -O3 -std=c++20 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC \
	    -DBUILD_CUDA -DHAVE_ZLIB -w -Iinclude -I$(REF)/include $(INC) -c $(SRC) -o $@
