# oracle/refgpu.mk - builds the reference's own GPU search (maddog107/av1gpu: the encoder/src kernels and host
# orchestration, av1core's GPU back end and av1f, which pipeline.cpp links against) for sm_100 - the reference's own
# "100-real" target, CMakeLists.txt:85 - from its sources where they lie, plus oracle/ref_gpu.cpp, into
# oracle/_ref/libref_gpu.so.  Measurement infrastructure only (the speed bar and the reference's decisions for
# BD-rate comparisons); the reference's image readers (libpng / libjpeg / libwebp / nvJPEG) are not needed and not built.
#   make -C oracle -f refgpu.mk REF=<path of the reference checkout> -j8
ifeq ($(strip $(REF)),)
$(error REF is not set: pass REF=<path of the reference checkout>)
endif
NVCC ?= nvcc
ARCH := -gencode arch=compute_100,code=sm_100
INC := -I$(REF)/encoder/src -I$(REF)/av1core/include -I$(REF)/av1core/src -I$(REF)/av1f/include
CUFLAGS := -std=c++17 -O3 $(ARCH) --expt-relaxed-constexpr -Xcompiler -fPIC $(INC)
CXXFLAGS := -std=c++17 -O2 -fPIC -w $(INC) -I/usr/local/cuda/include
O := _ref/refgpu
ENC_CU := k_misc k_imageops k_an_a k_an_b k_an_c k_an_d k_an_x k_an_uv k_recon k_recon_444_8 k_recon_420_10 k_recon_444_10 \
          k_recon_order k_leafprep k_lossless k_pal entropy_dev
ENC_CPP := pipeline imageops entropy_gpu
OBJS := $(addprefix $(O)/enc_,$(addsuffix .o,$(ENC_CU) $(ENC_CPP))) $(O)/core_encoder.o $(O)/core_avif.o $(O)/core_gpu_entropy.o \
        $(O)/core_gpu_postfilter.o $(O)/f_varboost.o $(O)/f_lfsearch.o $(O)/ref_gpu.o

all: _ref/libref_gpu.so

$(O)/enc_%.o: $(REF)/encoder/src/%.cu
	@mkdir -p $(O)
	$(NVCC) $(CUFLAGS) -c $< -o $@
$(O)/enc_%.o: $(REF)/encoder/src/%.cpp
	@mkdir -p $(O)
	g++ $(CXXFLAGS) -c $< -o $@
$(O)/core_gpu_%.o: $(REF)/av1core/src/gpu_%.cu
	@mkdir -p $(O)
	$(NVCC) $(CUFLAGS) --default-stream per-thread -c $< -o $@
$(O)/core_%.o: $(REF)/av1core/src/%.cpp
	@mkdir -p $(O)
	g++ $(CXXFLAGS) -c $< -o $@
$(O)/f_%.o: $(REF)/av1f/src/%.cu
	@mkdir -p $(O)
	$(NVCC) $(CUFLAGS) -c $< -o $@
$(O)/ref_gpu.o: ref_gpu.cpp
	@mkdir -p $(O)
	g++ $(CXXFLAGS) -c $< -o $@

_ref/libref_gpu.so: $(OBJS)
	$(NVCC) -shared $(ARCH) -o $@ $(OBJS) -lpthread

clean:
	rm -rf $(O) _ref/libref_gpu.so
.PHONY: all clean
