# Recipe that compiles the reference's own GPU stage programs for sm_100a into oracle/_ref/gpu/,
# from their sources where they lie, so they can be run on a B200 beside this library's drivers
# (the "reference on the same box" measurement; oracle/ref_gpu_run.sh runs them).
#
# Test infrastructure only: nothing in the product links against or calls these programs.
#   fused_gg2gg     cuPythia/03_fused_resident_me/fused_gg2gg.cu
#   fp32_gg2gg      cuPythia/06_fp32_mixed/fp32_gg2gg.cu
#   vegas           cuPythia/11_vegas_importance/vegas.cu
#   cub_compaction  cuPythia/10_cub_compaction/cub_compaction.cu
#   unweight_lhe    cuPythia/07_unweighting_lhe/unweight_lhe.cu
#   pdf_xsec        cuPythia/pipeline/pdf_xsec.cu
#   generate        cuPythia/pipeline/generate.cu
# The reference builds them with `nvcc -O3 [-std=c++17] -arch=sm_120`; here the same flags with
# the B200's architecture.
#
# Usage: make -f oracle/ref_gpu.mk -j8 REF=<reference root>   (or CUPYTHIA_REFERENCE in the environment)
REF   ?= $(CUPYTHIA_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF=<reference root> or CUPYTHIA_REFERENCE)
endif
CUP   := $(REF)/cuPythia
OUT   := oracle/_ref/gpu
NVCC  ?= nvcc
FLAGS := -O3 -std=c++17 -gencode arch=compute_100a,code=sm_100a -w

PROGS := fused_gg2gg fp32_gg2gg vegas cub_compaction unweight_lhe pdf_xsec generate
all: $(addprefix $(OUT)/,$(PROGS))

$(OUT)/fused_gg2gg: $(CUP)/03_fused_resident_me/fused_gg2gg.cu $(CUP)/common/rng.cuh
$(OUT)/fp32_gg2gg: $(CUP)/06_fp32_mixed/fp32_gg2gg.cu $(CUP)/common/rng.cuh
$(OUT)/vegas: $(CUP)/11_vegas_importance/vegas.cu $(CUP)/common/rng.cuh
$(OUT)/cub_compaction: $(CUP)/10_cub_compaction/cub_compaction.cu $(CUP)/common/rng.cuh
$(OUT)/unweight_lhe: $(CUP)/07_unweighting_lhe/unweight_lhe.cu $(CUP)/common/rng.cuh
$(OUT)/pdf_xsec: $(CUP)/pipeline/pdf_xsec.cu $(wildcard $(CUP)/pipeline/*.cuh)
$(OUT)/generate: $(CUP)/pipeline/generate.cu $(wildcard $(CUP)/pipeline/*.cuh)

$(OUT)/%:
	@mkdir -p $(OUT)
	$(NVCC) $(FLAGS) $< -o $@

.PHONY: all
