# Builds the reference's CPU path (YRT-PET 2.0.7) straight from its sources with
# g++, without its CMake project, into oracle/_ref/.  Test infrastructure only:
# the outputs check results and give the timed CPU baseline, never the product.
#
#   make -f oracle/ref.mk -j8 REF=<yrt-pet source tree> JSON_HPP=<nlohmann/json.hpp>
#
# Needs: g++ (C++20), zlib headers + libz, and the header-only nlohmann/json
# 3.11 (JSON_HPP; only read when oracle/_ref/include does not hold it yet).
ifndef REF
$(error REF=<path of the yrt-pet source tree> is required)
endif
OUT      ?= oracle/_ref
CXX      ?= g++
# Same flags as the reference's Release build (-O3, no -march, C++20, -fPIC).
CXXFLAGS := -O3 -std=c++20 -fPIC -DHAVE_ZLIB -w -I$(REF)/include -I$(OUT)/include

SRCS := $(shell find $(REF)/src -name '*.cpp' ! -name 'pybind11.cpp' | sort)
OBJS := $(patsubst $(REF)/src/%.cpp,$(OUT)/obj/%.o,$(SRCS))

all: $(OUT)/libyrtref.a $(OUT)/libyrtref_harness.so

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

$(OUT)/libyrtref.a: $(OBJS)
	rm -f $@ && ar rcs $@ $^

$(OUT)/libyrtref_harness.so: oracle/ref_harness.cpp $(OUT)/libyrtref.a
	$(CXX) $(CXXFLAGS) -shared $< -o $@ -Wl,--whole-archive $(OUT)/libyrtref.a -Wl,--no-whole-archive -lz -lpthread -Wl,-Bsymbolic -Wl,--exclude-libs,ALL

.PHONY: all
