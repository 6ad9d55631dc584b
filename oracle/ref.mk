# Build recipe for the reference checker: compiles Manta's ray-query hot path
# (DynBVH, WaldTriangle, KenslerShirleyTriangle, Mesh, RayPacket, HardShadows,
# Lambertian, PointLight, Raytracer and the Core/Interface code they need)
# straight from the reference sources, plus this project's harness
# (oracle/ref_harness.cc), into oracle/_ref/.
#
#   make -f oracle/ref.mk REF=/path/to/rfManta -j8
#
# Two variants are produced:
#   oracle/_ref/libmanta_ref.so      MANTA_SSE off (scalar IEEE float paths):
#                                    the parity checker.
#   oracle/_ref/libmanta_ref_sse.so  MANTA_SSE on (rcpps/rsqrtps fast paths):
#                                    the reference's fast default, used only as
#                                    the timed CPU baseline.
#
# The reference's own CMake build is not used: it needs X11/GL, Embree and
# Rayforce, none of which exist here.  The generated config headers are made
# from include/*.CMakeTemplate with the reference's default cache values
# (include/CMakeLists.txt): Real=float, T_EPSILON 1.e-4, MAXT 1.e19,
# RAYPACKET_MAXSIZE 64, SCRATCHPAD_MAXSIZE 128, MAXCACHELINESIZE 128,
# DynBVH ports/approximate/lazy all off.  Nothing is written outside _ref/.

# The reference checkout: REF=..., else $RFMANTA_REFERENCE, else a checkout
# named `reference` beside this repository.
HERE := $(dir $(lastword $(MAKEFILE_LIST)))
REF ?= $(if $(RFMANTA_REFERENCE),$(RFMANTA_REFERENCE),$(abspath $(HERE)../../reference))
OUT := $(HERE)_ref
# The system compiler driver links libstdc++ as a shared library, so the
# checker shares one C++ runtime with the Python process that loads it.
CXX := /usr/bin/g++

CORE_SRC := \
  Core/Containers/StringUtil.cc \
  Core/Color/ColorDB.cc Core/Color/RGBColor.cc Core/Color/RGBTraits.cc \
  Core/Color/GrayColor.cc Core/Color/Spectrum.cc Core/Color/RegularColorMap.cc \
  Core/Exceptions/BadPrimitive.cc Core/Exceptions/ErrnoException.cc \
  Core/Exceptions/Exception.cc Core/Exceptions/FileNotFound.cc \
  Core/Exceptions/IllegalArgument.cc Core/Exceptions/InputError.cc \
  Core/Exceptions/InternalError.cc Core/Exceptions/InvalidState.cc \
  Core/Exceptions/NullPointerException.cc Core/Exceptions/OutputError.cc \
  Core/Exceptions/SerializationError.cc Core/Exceptions/UnknownColor.cc \
  Core/Exceptions/UnknownComponent.cc Core/Exceptions/UnknownPixelFormat.cc \
  Core/Geometry/AffineTransform.cc Core/Geometry/AffineTransformT.cc \
  Core/Geometry/BBox.cc Core/Geometry/Vector.cc Core/Geometry/VectorT.cc \
  Core/Math/CheapRNG.cc Core/Math/ExponSSE.cc Core/Math/HaltonSequence.cc \
  Core/Math/KorobovRNG.cc Core/Math/MiscMath.cc Core/Math/MT_RNG.cc \
  Core/Math/Noise.cc Core/Math/SSEDefs.cc Core/Math/TrigSSE.cc \
  Core/Persistent/Archive.cc Core/Persistent/ArchiveElement.cc \
  Core/Persistent/MantaRTTI.cc \
  Core/Thread/CleanupManager.cc Core/Thread/Guard.cc Core/Thread/ParallelBase.cc \
  Core/Thread/Runnable.cc Core/Thread/Thread.cc Core/Thread/ThreadError.cc \
  Core/Thread/SimpleReducer.cc Core/Thread/ThreadLock.cc Core/Thread/ThreadGroup.cc \
  Core/Thread/Thread_unix.cc Core/Thread/ThreadPool.cc Core/Thread/WorkQueue.cc \
  Core/Thread/Thread_pthreads.cc Core/Thread/Time_unix.cc \
  Core/Util/AlignedAllocator.cc Core/Util/Args.cc Core/Util/CallbackHelpers.cc \
  Core/Util/CPUTime.cc Core/Util/LargeFile.cc Core/Util/rgbe.cc \
  Core/Util/ThreadStorage.cc Core/Util/Timer.cc Core/Util/Logger.cc

IFACE_SRC := $(patsubst $(REF)/%,%,$(wildcard $(REF)/Interface/*.cc))

MODEL_SRC := \
  Model/Groups/DynBVH.cc Model/Groups/Group.cc Model/Groups/Mesh.cc \
  Model/Groups/TreeTraversalProbability.cc \
  Model/Primitives/WaldTriangle.cc Model/Primitives/KenslerShirleyTriangle.cc \
  Model/Primitives/MeshTriangle.cc \
  Model/Materials/Lambertian.cc Model/Materials/LitMaterial.cc \
  Model/Materials/OpaqueShadower.cc Model/Materials/Phong.cc \
  Model/Textures/Constant.cc \
  Model/Lights/PointLight.cc \
  Model/AmbientLights/ConstantAmbient.cc \
  Model/AmbientLights/EyeAmbient.cc \
  Model/Backgrounds/ConstantBackground.cc \
  Model/Backgrounds/LinearBackground.cc \
  Model/Cameras/PinholeCamera.cc \
  Model/Lights/AreaLight.cc Model/Primitives/Parallelogram.cc \
  Model/Primitives/PrimitiveCommon.cc Model/TexCoordMappers/UniformMapper.cc \
  Model/Instances/InstanceT.cc Model/Instances/InstanceMaterial.cc \
  Model/Readers/PlyReader.cc \
  Model/Groups/ObjGroup.cc Model/Readers/glm/glm.cc \
  Model/Materials/Dielectric.cc Model/Materials/Transparent.cc Model/Materials/Flat.cc \
  Model/Textures/NormalTexture.cc Model/Primitives/MovingKSTriangle.cc

ENGINE_SRC := \
  Engine/Shadows/HardShadows.cc Engine/Renderers/Raytracer.cc \
  Engine/SampleGenerators/ConstantSampleGenerator.cc \
  Engine/SampleGenerators/UniformRandomGenerator.cc \
  Engine/Renderers/KajiyaPathtracer.cc Engine/Shadows/NoDirect.cc

SRC := $(CORE_SRC) $(IFACE_SRC) $(MODEL_SRC) $(ENGINE_SRC)

COMMON_FLAGS := -std=gnu++98 -O2 -fPIC -w -pthread -fno-strict-aliasing

# C sources (the PLY parser the reference vendors, Model/Readers/rply)
C_SRC := Model/Readers/rply/rply.c
CC := /usr/bin/gcc

OBJ_NOSSE := $(patsubst %.cc,$(OUT)/obj_nosse/%.o,$(SRC)) $(patsubst %.c,$(OUT)/obj_c/%.o,$(C_SRC))
OBJ_SSE   := $(patsubst %.cc,$(OUT)/obj_sse/%.o,$(SRC)) $(patsubst %.c,$(OUT)/obj_c/%.o,$(C_SRC))

all: $(OUT)/libmanta_ref.so $(OUT)/libmanta_ref_sse.so

# The same checker with this project's C++ drop-in (rfmanta_b200/manta/
# GpuDynBVH) compiled against the reference headers and linked to the CUDA
# library: the reference's renderers running on the device path.
dropin: $(OUT)/libmanta_dropin.so $(OUT)/libmanta_dropin_sse.so

# ---- generated config headers (one set per SSE variant) -------------------
define GEN_HEADERS
$(OUT)/gen_$(1)/include/.stamp: $(wildcard $(REF)/include/*Template)
	mkdir -p $(OUT)/gen_$(1)/include
	for t in $(REF)/include/*.CMakeTemplate $(REF)/include/*.CmakeTemplate; do \
	  b=$$$$(basename $$$$t); b=$$$${b%.CMakeTemplate}; b=$$$${b%.CmakeTemplate}; \
	  sed -e 's/$$$${MANTA_REAL}/float/g' \
	      -e 's/$$$${MANTA_COLOR_COMPONENT}/float/g' \
	      -e 's/$$$${MANTA_RAYPACKET_MAXSIZE}/64/g' \
	      -e 's/$$$${MANTA_SCRATCHPAD_MAXSIZE}/128/g' \
	      -e 's/$$$${MANTA_FRAGMENT_MAXSIZE}/64/g' \
	      -e 's/$$$${MANTA_SSE_DEF}/$(2)/g' \
	      -e 's/$$$${MANTA_SSE_GCC_DEF}/$(2)/g' \
	      -e 's/$$$${MANTA_SSE_CAST_DEF}/$(2)/g' \
	      -e 's/$$$${MANTA_USE_DYNBVH_PORTS_DEF}/0/g' \
	      -e 's/$$$${MANTA_USE_DYNBVH_APPROXIMATE_DEF}/0/g' \
	      -e 's/$$$${MANTA_USE_DYNBVH_LAZY_DEF}/0/g' \
	      -e 's/$$$${MANTA_MAXCACHELINESIZE}/128/g' \
	      -e 's/$$$${MANTA_T_EPSILON}/1.e-4/g' \
	      -e 's/$$$${MANTA_DENORM_EPSILON}/1.e-6/g' \
	      -e 's/$$$${MANTA_COLOR_EPSILON}/1.e-4/g' \
	      -e 's/$$$${MANTA_MAXT}/1.e19/g' \
	      -e 's/$$$${MANTA_IMAGE_ROW_BYTES}/32/g' \
	      -e 's/$$$${MANTA_X86_DEF}/1/g' \
	      -e 's/$$$${PABST_FOUND_DEF}/0/g' \
	      -e 's/$$$${USE_MPI_DEF}/0/g' \
	      -e 's/$$$${FOUND_TEEM_DEF}/0/g' \
	      -e 's/$$$${USE_PRIVATE_CODE_DEF}/0/g' \
	      -e 's/$$$${USE_STATS_COLLECTOR_DEF}/0/g' \
	      -e 's/$$$${ABOUT_STRING}/manta-ref-checker/g' \
	      $$$$t > $(OUT)/gen_$(1)/include/$$$$b; \
	done
	touch $$@
endef
$(eval $(call GEN_HEADERS,nosse,0))
$(eval $(call GEN_HEADERS,sse,1))

INC_NOSSE := -I$(REF) -I$(OUT)/gen_nosse/include
INC_SSE   := -I$(REF) -I$(OUT)/gen_sse/include

$(OUT)/obj_nosse/%.o: $(REF)/%.cc $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) $(INC_NOSSE) -c $< -o $@

$(OUT)/obj_sse/%.o: $(REF)/%.cc $(OUT)/gen_sse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) -msse4.1 $(INC_SSE) -c $< -o $@

$(OUT)/obj_c/%.o: $(REF)/%.c
	@mkdir -p $(dir $@)
	$(CC) -O2 -fPIC -w -c $< -o $@

# The harness is this project's code: it drives the reference classes above.
$(OUT)/obj_nosse/harness.o: $(HERE)ref_harness.cc $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) $(INC_NOSSE) -c $< -o $@

$(OUT)/obj_sse/harness.o: $(HERE)ref_harness.cc $(OUT)/gen_sse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) -msse4.1 $(INC_SSE) -c $< -o $@

REPO := $(abspath $(HERE)..)

$(OUT)/obj_nosse/harness_dropin.o: $(HERE)ref_harness.cc $(REPO)/rfmanta_b200/manta/GpuDynBVH.h $(REPO)/rfmanta_b200/manta/GpuHardShadows.h $(REPO)/rfmanta_b200/manta/GpuMeshPrimitive.h $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) -DMREF_DROPIN $(INC_NOSSE) -I$(REPO) -c $< -o $@

$(OUT)/obj_nosse/GpuDynBVH.o: $(REPO)/rfmanta_b200/manta/GpuDynBVH.cc $(REPO)/rfmanta_b200/manta/GpuDynBVH.h $(REPO)/include/rfmanta_b200.h $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) $(INC_NOSSE) -I$(REPO) -c $< -o $@

$(OUT)/obj_nosse/GpuHardShadows.o: $(REPO)/rfmanta_b200/manta/GpuHardShadows.cc $(REPO)/rfmanta_b200/manta/GpuHardShadows.h $(REPO)/rfmanta_b200/manta/GpuDynBVH.h $(REPO)/include/rfmanta_b200.h $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) $(INC_NOSSE) -I$(REPO) -c $< -o $@

$(OUT)/obj_nosse/GpuMeshPrimitive.o: $(REPO)/rfmanta_b200/manta/GpuMeshPrimitive.cc $(REPO)/rfmanta_b200/manta/GpuMeshPrimitive.h $(REPO)/rfmanta_b200/manta/GpuDynBVH.h $(REPO)/include/rfmanta_b200.h $(OUT)/gen_nosse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) $(INC_NOSSE) -I$(REPO) -c $< -o $@

DROPIN_OBJ := $(OUT)/obj_nosse/harness_dropin.o $(OUT)/obj_nosse/GpuDynBVH.o \
  $(OUT)/obj_nosse/GpuHardShadows.o $(OUT)/obj_nosse/GpuMeshPrimitive.o

$(OUT)/libmanta_dropin.so: $(OBJ_NOSSE) $(DROPIN_OBJ) $(REPO)/rfmanta_b200/librfmanta_b200.so
	$(CXX) -shared -pthread -o $@ $(OBJ_NOSSE) $(DROPIN_OBJ) -L$(REPO)/rfmanta_b200 -lrfmanta_b200 -Wl,-rpath,'$$ORIGIN/../../rfmanta_b200' -Wl,--no-as-needed -lstdc++ -lm

# The drop-in over the MANTA_SSE build of the reference classes (the build
# the CPU baseline is timed in), for timing the reference's renderer with
# GpuDynBVH swapped in.
DROPIN_HDRS := $(REPO)/rfmanta_b200/manta/GpuDynBVH.h $(REPO)/rfmanta_b200/manta/GpuHardShadows.h \
  $(REPO)/rfmanta_b200/manta/GpuMeshPrimitive.h $(REPO)/include/rfmanta_b200.h

$(OUT)/obj_sse/harness_dropin.o: $(HERE)ref_harness.cc $(DROPIN_HDRS) $(OUT)/gen_sse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) -msse4.1 -DMREF_DROPIN $(INC_SSE) -I$(REPO) -c $< -o $@

$(OUT)/obj_sse/Gpu%.o: $(REPO)/rfmanta_b200/manta/Gpu%.cc $(DROPIN_HDRS) $(OUT)/gen_sse/include/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(COMMON_FLAGS) -msse4.1 $(INC_SSE) -I$(REPO) -c $< -o $@

DROPIN_SSE_OBJ := $(OUT)/obj_sse/harness_dropin.o $(OUT)/obj_sse/GpuDynBVH.o \
  $(OUT)/obj_sse/GpuHardShadows.o $(OUT)/obj_sse/GpuMeshPrimitive.o

$(OUT)/libmanta_dropin_sse.so: $(OBJ_SSE) $(DROPIN_SSE_OBJ) $(REPO)/rfmanta_b200/librfmanta_b200.so
	$(CXX) -shared -pthread -o $@ $(OBJ_SSE) $(DROPIN_SSE_OBJ) -L$(REPO)/rfmanta_b200 -lrfmanta_b200 -Wl,-rpath,'$$ORIGIN/../../rfmanta_b200' -Wl,--no-as-needed -lstdc++ -lm

$(OUT)/libmanta_ref.so: $(OBJ_NOSSE) $(OUT)/obj_nosse/harness.o
	$(CXX) -shared -pthread -o $@ $^ -Wl,--no-as-needed -lstdc++ -lm

$(OUT)/libmanta_ref_sse.so: $(OBJ_SSE) $(OUT)/obj_sse/harness.o
	$(CXX) -shared -pthread -o $@ $^ -Wl,--no-as-needed -lstdc++ -lm

.PHONY: all dropin
