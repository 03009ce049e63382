# Builds the reference's vendored Embree 2.17.4 (src/External/Embree) from its sources where
# they lie, with plain g++ and this file: no CMake, no change to the reference tree.  The
# settings are the ones the reference's top-level CMakeLists.txt forces on Embree (static
# library, internal tasking, no ISPC, ray mask and intersection filter on, backface culling
# off) and Embree's own default ISA set for x86-64 (EMBREE_MAX_ISA = AVX2: SSE2 as the lowest
# ISA plus SSE4.2, AVX and AVX2 kernels selected at run time).  Its configure-time headers
# (kernels/config.h, kernels/hash.h, include/embree2/rtcore_version.h) ship pre-generated in the
# vendored tree, so nothing is generated here.
#
# TEST INFRASTRUCTURE ONLY: the library is linked into oracle/_ref/ programs (the reference's
# own renderer and its hit-record harness) and never into the product.
#
#   make -C oracle embree REF_SRC=<reference>/src   -> oracle/_ref/embree/libembree_ref.a

EMB      := $(REF_SRC)/External/Embree
EOBJ     := $(HERE)_ref/embree
# gcc.cmake: FLAGS_* and the common/release flags; -w silences 2018-era warnings under GCC 13
EFLAGS   := -O3 -DNDEBUG -fPIC -std=c++11 -fvisibility=hidden -fvisibility-inlines-hidden \
            -fno-strict-aliasing -fno-tree-vectorize -w \
            -DEMBREE_STATIC_LIB -DTASKING_INTERNAL \
            -DEMBREE_TARGET_SSE2 -DEMBREE_TARGET_SSE42 -DEMBREE_TARGET_AVX -DEMBREE_TARGET_AVX2
F_SSE2   := -msse2
F_SSE42  := -msse4.2
F_AVX    := -mavx
F_AVX2   := -mf16c -mavx2 -mfma -mlzcnt -mbmi -mbmi2

# common/{sys,math,simd,lexers,tasking,algorithms}/CMakeLists.txt
E_COMMON := common/sys/sysinfo.cpp common/sys/alloc.cpp common/sys/filename.cpp common/sys/library.cpp \
            common/sys/thread.cpp common/sys/string.cpp common/sys/regression.cpp common/sys/mutex.cpp \
            common/sys/condition.cpp common/sys/barrier.cpp common/math/constants.cpp common/simd/sse.cpp \
            common/lexers/stringstream.cpp common/lexers/tokenstream.cpp \
            common/tasking/taskschedulerinternal.cpp \
            common/algorithms/parallel_for.cpp common/algorithms/parallel_reduce.cpp \
            common/algorithms/parallel_prefix_sum.cpp common/algorithms/parallel_for_for.cpp \
            common/algorithms/parallel_for_for_prefix_sum.cpp common/algorithms/parallel_partition.cpp \
            common/algorithms/parallel_sort.cpp common/algorithms/parallel_set.cpp \
            common/algorithms/parallel_map.cpp common/algorithms/parallel_filter.cpp

# kernels/CMakeLists.txt EMBREE_LIBRARY_FILES (+ subdiv and ray-packet files, both on in
# kernels/config.h), compiled for the lowest ISA with EMBREE_LOWEST_ISA
E_BASE   := common/device.cpp common/stat.cpp common/acceln.cpp common/accelset.cpp common/state.cpp \
            common/rtcore.cpp common/rtcore_builder.cpp common/scene.cpp common/alloc.cpp common/geometry.cpp \
            common/tasksys.cpp common/scene_user_geometry.cpp common/scene_instance.cpp \
            common/scene_geometry_instance.cpp common/scene_triangle_mesh.cpp common/scene_quad_mesh.cpp \
            common/scene_bezier_curves.cpp common/scene_line_segments.cpp subdiv/bezier_curve.cpp \
            subdiv/bspline_curve.cpp geometry/primitive.cpp geometry/instance_intersector.cpp \
            builders/primrefgen.cpp bvh/bvh.cpp bvh/bvh_statistics.cpp bvh/bvh4_factory.cpp \
            bvh/bvh8_factory.cpp bvh/bvh_rotate.cpp bvh/bvh_refit.cpp bvh/bvh_builder.cpp \
            bvh/bvh_builder_hair.cpp bvh/bvh_builder_hair_mb.cpp bvh/bvh_builder_morton.cpp \
            bvh/bvh_builder_sah.cpp bvh/bvh_builder_twolevel.cpp bvh/bvh_builder_instancing.cpp \
            bvh/bvh_intersector1_bvh4.cpp \
            common/scene_subdiv_mesh.cpp subdiv/tessellation_cache.cpp subdiv/subdivpatch1base.cpp \
            subdiv/catmullclark_coefficients.cpp geometry/grid_soa.cpp subdiv/subdivpatch1base_eval.cpp \
            bvh/bvh_builder_subdiv.cpp \
            common/rtcore_ispc.cpp bvh/bvh_intersector_hybrid4_bvh4.cpp bvh/bvh_intersector_stream_bvh4.cpp \
            bvh/bvh_intersector_stream_filters.cpp

# kernels/CMakeLists.txt embree_files(<list> <ISA>) with ISA_LOWEST = SSE2
E_SUBDIV := common/scene_subdiv_mesh.cpp geometry/grid_soa.cpp subdiv/subdivpatch1base_eval.cpp
E_PKT4   := bvh/bvh_intersector_hybrid4_bvh4.cpp bvh/bvh_intersector_stream_bvh4.cpp \
            bvh/bvh_intersector_stream_filters.cpp
E_PKT8   := bvh/bvh_intersector_hybrid8_bvh4.cpp bvh/bvh_intersector_hybrid4_bvh8.cpp \
            bvh/bvh_intersector_hybrid8_bvh8.cpp bvh/bvh_intersector_stream_bvh8.cpp
E_BLD    := common/scene_triangle_mesh.cpp common/scene_quad_mesh.cpp common/scene_bezier_curves.cpp \
            common/scene_line_segments.cpp bvh/bvh_refit.cpp bvh/bvh_builder.cpp bvh/bvh_builder_hair.cpp \
            bvh/bvh_builder_hair_mb.cpp bvh/bvh_builder_sah.cpp bvh/bvh_builder_twolevel.cpp \
            bvh/bvh_builder_instancing.cpp bvh/bvh_builder_subdiv.cpp
E_MORTON := bvh/bvh_builder_morton.cpp bvh/bvh_rotate.cpp builders/primrefgen.cpp
E_SSE42  := geometry/instance_intersector.cpp bvh/bvh_intersector1_bvh4.cpp $(E_SUBDIV) $(E_PKT4)
E_AVX    := geometry/instance_intersector.cpp bvh/bvh_intersector1_bvh4.cpp $(E_BLD) $(E_MORTON) \
            bvh/bvh_intersector1_bvh8.cpp bvh/bvh.cpp bvh/bvh_statistics.cpp $(E_SUBDIV) $(E_PKT4) $(E_PKT8)
E_AVX2   := geometry/instance_intersector.cpp bvh/bvh_intersector1_bvh4.cpp $(E_MORTON) \
            bvh/bvh_intersector1_bvh8.cpp $(E_SUBDIV) $(E_PKT4) $(E_PKT8)

E_OBJS   := $(E_COMMON:%.cpp=$(EOBJ)/common_sse2/%.o) \
            $(E_BASE:%.cpp=$(EOBJ)/sse2/%.o) \
            $(E_SSE42:%.cpp=$(EOBJ)/sse42/%.o) \
            $(E_AVX:%.cpp=$(EOBJ)/avx/%.o) \
            $(E_AVX2:%.cpp=$(EOBJ)/avx2/%.o)

EMBREE_LIB := $(EOBJ)/libembree_ref.a

$(EOBJ)/common_sse2/%.o: $(EMB)/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(EFLAGS) $(F_SSE2) -c $< -o $@

$(EOBJ)/sse2/%.o: $(EMB)/kernels/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(EFLAGS) $(F_SSE2) -DEMBREE_LOWEST_ISA -c $< -o $@

$(EOBJ)/sse42/%.o: $(EMB)/kernels/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(EFLAGS) $(F_SSE42) -c $< -o $@

$(EOBJ)/avx/%.o: $(EMB)/kernels/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(EFLAGS) $(F_AVX) -c $< -o $@

$(EOBJ)/avx2/%.o: $(EMB)/kernels/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(EFLAGS) $(F_AVX2) -c $< -o $@

$(EMBREE_LIB): $(E_OBJS)
	rm -f $@
	ar rcs $@ $^

embree: $(EMBREE_LIB)

.PHONY: embree
