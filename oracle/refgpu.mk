# Builds the reference's own GPU step (data/src/selm-main/src/cuda/
# SELM_Eulerian_Period.cu and SELM_Kernel.cu, compiled unchanged from where
# they lie) for sm_100a with the project's stub driver (oracle/refgpu_stub.cu)
# into oracle/_ref/libselm_refgpu.so.  TEST AND BENCH INFRASTRUCTURE ONLY:
# the reference-GPU bar and the cuFFT cross-check; never linked into the product.
# Usage: make -f oracle/refgpu.mk
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
SELM_REFERENCE_ROOT ?= /root/reference
REFCUDA ?= $(SELM_REFERENCE_ROOT)/data/src/selm-main/src/cuda
NVCC ?= /usr/local/cuda/bin/nvcc
OUT := $(HERE)_ref/libselm_refgpu.so
# -include cstdio: SELM_Kernel.cu calls printf without including its header
FLAGS := -std=c++17 -O3 -rdc=true -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -include cstdio -w
OBJ := $(HERE)_ref/refgpu_eul.o $(HERE)_ref/refgpu_kern.o $(HERE)_ref/refgpu_stub.o

all: $(OUT)

$(HERE)_ref/refgpu_eul.o: $(REFCUDA)/SELM_Eulerian_Period.cu
	@mkdir -p $(HERE)_ref
	$(NVCC) $(FLAGS) -I$(REFCUDA) -c $< -o $@
$(HERE)_ref/refgpu_kern.o: $(REFCUDA)/SELM_Kernel.cu
	@mkdir -p $(HERE)_ref
	$(NVCC) $(FLAGS) -I$(REFCUDA) -c $< -o $@
$(HERE)_ref/refgpu_stub.o: $(HERE)refgpu_stub.cu
	@mkdir -p $(HERE)_ref
	$(NVCC) $(FLAGS) -I$(REFCUDA) -c $< -o $@

$(OUT): $(OBJ)
	$(NVCC) -shared -rdc=true -gencode arch=compute_100a,code=sm_100a -o $@ $(OBJ) -lcufft -lcurand

clean:
	rm -f $(OUT) $(OBJ)

.PHONY: all clean
