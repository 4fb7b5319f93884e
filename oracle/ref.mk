# Recipe that builds the reference's own CPU code for the integrator path into oracle/_ref/.
#
# Test infrastructure only: nothing in the product links against these outputs.
#   oracle/_ref/libpythia8.a      Pythia 8.317 compiled file-by-file from its sources
#   oracle/_ref/pythia_ref        driver over the Pythia API (oracle/ref_pythia.cc)
#   oracle/_ref/libcupythia_ref.so cuPythia's host/device headers (common/rng.cuh,
#                                 pipeline/physics.cuh) compiled as plain C++ (oracle/ref_cupythia.cc)
#   oracle/_ref/xmldoc/, tunes/   copies of Pythia's settings database and tune files, read at init
#   oracle/_ref/pythia_plugin_check (target `plugin`, after the CUDA library is built) the test
#                                 program of the Pythia plug-in cupythia_b200/pythia/CpSigmaQCD.*,
#                                 linked against this Pythia and libcupythia_b200.so
#
# Usage: make -f oracle/ref.mk -j8 REF=<reference root>   (or CUPYTHIA_REFERENCE in the environment)
REF     ?= $(CUPYTHIA_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF=<reference root> or CUPYTHIA_REFERENCE)
endif
PY8     := $(REF)/pythia8317
OUT     := oracle/_ref
CXX     ?= g++
PYFLAGS := -O2 -std=c++11 -fPIC -w -I$(PY8)/include -DXMLDIR=\"xmldoc\"

PY8_SRC := $(wildcard $(PY8)/src/*.cc)
PY8_OBJ := $(patsubst $(PY8)/src/%.cc,$(OUT)/obj/%.o,$(PY8_SRC))

all: $(OUT)/libcupythia_ref.so $(OUT)/pythia_ref $(OUT)/xmldoc/.stamp $(OUT)/tunes/.stamp

$(OUT)/obj/%.o: $(PY8)/src/%.cc
	@mkdir -p $(OUT)/obj
	$(CXX) $(PYFLAGS) -c $< -o $@

$(OUT)/libpythia8.a: $(PY8_OBJ)
	ar rcs $@ $^

$(OUT)/pythia_ref: oracle/ref_pythia.cc $(OUT)/libpythia8.a
	$(CXX) -O2 -std=c++17 -I$(PY8)/include $< -o $@ $(OUT)/libpythia8.a -ldl -lpthread

$(OUT)/libcupythia_ref.so: oracle/ref_cupythia.cc
	@mkdir -p $(OUT)
	$(CXX) -O2 -std=c++17 -fPIC -shared -I$(REF)/cuPythia $< -o $@

$(OUT)/xmldoc/.stamp: $(wildcard $(PY8)/share/Pythia8/xmldoc/*)
	@mkdir -p $(OUT)/xmldoc
	cp -r $(PY8)/share/Pythia8/xmldoc/. $(OUT)/xmldoc/
	touch $@

$(OUT)/tunes/.stamp: $(wildcard $(PY8)/share/Pythia8/tunes/*)
	@mkdir -p $(OUT)/tunes
	cp -r $(PY8)/share/Pythia8/tunes/. $(OUT)/tunes/
	touch $@

CUDA_HOME ?= /usr/local/cuda
PLUGIN_SRC := tests/pythia_plugin_check.cc cupythia_b200/pythia/CpSigmaQCD.cc
plugin: $(OUT)/pythia_plugin_check

$(OUT)/pythia_plugin_check: $(PLUGIN_SRC) cupythia_b200/pythia/CpSigmaQCD.h include/cupythia_b200.h $(OUT)/libpythia8.a cupythia_b200/libcupythia_b200.so
	$(CXX) -O2 -std=c++17 -Wall -I$(PY8)/include -Iinclude -Icupythia_b200/pythia -I$(CUDA_HOME)/include $(PLUGIN_SRC) \
	  -o $@ $(OUT)/libpythia8.a -Lcupythia_b200 -lcupythia_b200 -L$(CUDA_HOME)/lib64 -lcudart \
	  -Wl,-rpath,'$$ORIGIN/../../cupythia_b200' -ldl -lpthread

.PHONY: all plugin
