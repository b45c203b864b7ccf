# Compiles the reference's own sources, unmodified and in place, plus the harness in this
# directory into _ref/libhvvr_ref.so. Test infrastructure only: run from oracle/ by the
# oracle Makefile when the reference tree is present (REF_ROOT: from the environment, else the
# reference checkout beside the repository). Output goes to _ref/ (git-ignored).
REF_ROOT ?= $(abspath $(CURDIR)/../../reference)
RC = $(REF_ROOT)/libraries/hvvr/raycaster
SH = $(REF_ROOT)/libraries/hvvr/shared
SS = $(REF_ROOT)/libraries/hvvr/samples_shared
CUDA_INC ?= /usr/local/cuda/include
CXX ?= g++
# -ffp-contract=off: the reference's host code is built without contraction (MSVC /fp:precise)
REF_FLAGS = -std=c++17 -O2 -fPIC -mavx2 -mfma -mf16c -mbmi -mbmi2 -ffp-contract=off -fpermissive -w -pthread \
            -include refshim/compat/hvvr_gcc_compat.h -Irefshim/compat -I$(SH) -I$(RC) -I$(SS) -I$(CUDA_INC)
REF_SRCS = $(RC)/traverse_avx.cpp $(RC)/sample_hierarchy.cpp $(RC)/samples.cpp $(RC)/camera.cpp \
           $(RC)/foveated.cpp $(SH)/bvh.cpp $(SH)/debug.cpp $(SS)/model_import_bin.cpp
OBJS = $(patsubst %.cpp,_ref/obj/%.o,$(notdir $(REF_SRCS))) _ref/obj/frusta.o _ref/obj/ref_harness.o _ref/obj/ref_stubs.o

NVCC ?= nvcc
# the reference's texture creation and sampling built for the GPU (its project compiles CUDA with
# fast math), with the harness in ref_gpu_harness.cu
REF_GPU_FLAGS = -gencode arch=compute_100a,code=sm_100a -use_fast_math -std=c++17 -Xcompiler -fPIC,-mf16c -w \
                -include refshim/compat/hvvr_nvcc_compat.h -I$(SH) -I$(RC)

all: _ref/libhvvr_ref.so _ref/libhvvr_ref_gpu.so

_ref/libhvvr_ref_gpu.so: _ref/obj/texture.cu.o _ref/obj/gpu_image.cu.o _ref/obj/ref_gpu_harness.cu.o \
                         _ref/obj/ref_gpu_foveated.cu.o _ref/obj/ref_gpu_intersect.cu.o \
                         _ref/obj/ref_gpu_scene.cu.o
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $^
_ref/obj/%.cu.o: $(RC)/%.cu refshim/compat/hvvr_nvcc_compat.h
	@mkdir -p _ref/obj
	$(NVCC) $(REF_GPU_FLAGS) -c $< -o $@
# includes the reference's intersect.cu and resolve.cu to launch their kernels at every MSAA rate
_ref/obj/ref_gpu_intersect.cu.o: refshim/ref_gpu_intersect.cu $(RC)/intersect.cu $(RC)/resolve.cu \
                                 refshim/compat/hvvr_nvcc_compat.h
	@mkdir -p _ref/obj
	$(NVCC) $(REF_GPU_FLAGS) -c $< -o $@
# includes the reference's gpu_foveated.cu to launch its resolve kernels
_ref/obj/ref_gpu_foveated.cu.o: refshim/ref_gpu_foveated.cu $(RC)/gpu_foveated.cu refshim/compat/hvvr_nvcc_compat.h
	@mkdir -p _ref/obj
	$(NVCC) $(REF_GPU_FLAGS) -c $< -o $@
# includes the reference's gpu_scene_state.cu to launch its scene update kernels
# (its bvh_node.h declares structs inside an anonymous union, which gcc takes with -fpermissive)
_ref/obj/ref_gpu_scene.cu.o: refshim/ref_gpu_scene.cu $(RC)/gpu_scene_state.cu refshim/compat/hvvr_nvcc_compat.h
	@mkdir -p _ref/obj
	$(NVCC) $(REF_GPU_FLAGS) -Xcompiler -fpermissive -c $< -o $@
_ref/obj/ref_gpu_harness.cu.o: refshim/ref_gpu_harness.cu refshim/compat/hvvr_nvcc_compat.h
	@mkdir -p _ref/obj
	$(NVCC) $(REF_GPU_FLAGS) -c $< -o $@

# -Bsymbolic: the host stand-ins for the CUDA runtime calls (ref_stubs.cpp) must bind inside this
# library even when a real libcudart is already loaded into the process
_ref/libhvvr_ref.so: $(OBJS)
	$(CXX) -shared -pthread -Wl,-Bsymbolic -o $@ $(OBJS)

_ref/obj/%.o: $(RC)/%.cpp refshim/compat/hvvr_gcc_compat.h refshim/compat/avx.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -c $< -o $@
_ref/obj/%.o: $(SH)/%.cpp refshim/compat/hvvr_gcc_compat.h refshim/compat/avx.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -c $< -o $@
_ref/obj/%.o: $(SS)/%.cpp refshim/compat/hvvr_gcc_compat.h refshim/compat/avx.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -c $< -o $@
# frusta.cu holds host code only on the path used (ComputeEyeSpaceFrusta); compiled as C++
_ref/obj/frusta.o: $(RC)/frusta.cu refshim/compat/hvvr_gcc_compat.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -x c++ -c $< -o $@
_ref/obj/ref_harness.o: refshim/ref_harness.cpp hvvr_oracle.h ../include/hvvr_c.h refshim/compat/hvvr_gcc_compat.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -c $< -o $@
_ref/obj/ref_stubs.o: refshim/ref_stubs.cpp refshim/compat/hvvr_gcc_compat.h
	@mkdir -p _ref/obj
	$(CXX) $(REF_FLAGS) -c $< -o $@
