# Compiles the reference's own CUDA library (NethermindEth/stwo-gpu, cuda/src) from its
# sources where they lie, unmodified, into oracle/_ref/libgpubackend_ref.so for sm_100a.
# Used only as a cross-check of our kernels and as the reference GPU timing; never on
# the product path. Run from the repository root:  make -f oracle/ref.mk
REF      ?= /root/reference/cuda
OUT      := oracle/_ref
NVCC     ?= /usr/local/cuda/bin/nvcc
SRCS     := batch_inverse.cu bit_reverse.cu poly/eval_at_point.cu poly/ifft.cu poly/rfft.cu \
            poly/twiddles.cu poly/utils.cu fri/fold_line.cu fri/fold_circle_into_line.cu fri/utils.cu \
            utils.cu accumulate.cu fields.cu blake2s.cu quotients.cu example.cu gkr.cu mle.cu \
            examples/wide_fibonacci.cu
OBJS     := $(patsubst %.cu,$(OUT)/obj/%.o,$(SRCS))
FLAGS    := -gencode arch=compute_100a,code=sm_100a -O3 -rdc=true -Xcompiler -fPIC -std=c++14 -w -I$(REF)/include

ifeq ($(wildcard $(REF)/src),)
all:
	@echo "oracle/ref.mk: no reference tree at $(REF); oracle/_ref left as it is"
else
all: $(OUT)/libgpubackend_ref.so
endif

$(OUT)/obj/%.o: $(REF)/src/%.cu
	@mkdir -p $(dir $@)
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libgpubackend_ref.so: $(OBJS)
	$(NVCC) -gencode arch=compute_100a,code=sm_100a -shared -o $@ $(OBJS) -lcudart

clean:
	rm -rf $(OUT)

.PHONY: all clean
