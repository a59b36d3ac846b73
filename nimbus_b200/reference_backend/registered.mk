# The reference's own program, nimbus_sim, with the CUDA backend registered as
# its `cuda` compute backend: what a maintainer gets after applying
# registration.patch (a Cuda backend kind, its name and parser entries, the
# factory case, the configuration enum and the CLI override) and linking the
# adapter (nimbus_compute_backend.cpp) and libnimbus_cuda.so into the program.
#
#   make -f nimbus_b200/reference_backend/registered.mk REF=/path/to/reference -j8
#
# The reference tree is copied (src/ and include/) into $(OUT)/tree and
# patched there; the source tree itself is never written.  Every translation
# unit of the copy is compiled flat, with the portable flags of a CPU-only
# build, and linked with the adapter into $(OUT)/nimbus_sim_cuda, which finds
# libnimbus_cuda.so in nimbus_b200/lib by its run path.  This is not the
# reference's build system.
REF      ?= $(NIMBUS_REFERENCE_DIR)
ifeq ($(strip $(REF)),)
$(error REF (or NIMBUS_REFERENCE_DIR) must name the reference solver's source tree)
endif
HERE     := nimbus_b200/reference_backend
OUT      ?= $(HERE)/_registered
TREE     := $(OUT)/tree
OBJDIR   := $(OUT)/obj
LIBDIR   := nimbus_b200/lib
CXX      ?= g++
CXXFLAGS := -std=c++17 -O2 -fPIC -fopenmp -ffp-contract=off -w \
            -DNIMBUS_CPU_ONLY -DNIMBUS_PORTABLE_BUILD -I $(TREE)/include -I $(TREE)/src
GOMP_LIBS ?= -L/usr/lib/gcc/x86_64-linux-gnu/13 -lgomp -lpthread

# Objects and link run in a second make, once the patched tree exists.
all: $(TREE)/.patched
	$(MAKE) -f $(HERE)/registered.mk REF=$(REF) OUT=$(OUT) program

$(TREE)/.patched: $(HERE)/registration.patch
	rm -rf $(TREE)
	mkdir -p $(TREE)
	cp -r $(REF)/src $(REF)/include $(TREE)/
	patch -s -p1 -d $(TREE) < $(HERE)/registration.patch
	touch $@

ifneq ($(wildcard $(TREE)/.patched),)
SRCS     := $(filter-out $(TREE)/src/tools/%,$(shell find $(TREE)/src -name '*.cpp' | sort))
OBJS     := $(patsubst $(TREE)/src/%.cpp,$(OBJDIR)/%.o,$(SRCS))
endif

$(OBJDIR)/%.o: $(TREE)/src/%.cpp $(TREE)/.patched
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/adapter.o: $(HERE)/nimbus_compute_backend.cpp $(TREE)/.patched
	$(CXX) $(CXXFLAGS) -c $< -o $@

program: $(OUT)/nimbus_sim_cuda

$(OUT)/nimbus_sim_cuda: $(OBJS) $(OUT)/adapter.o $(LIBDIR)/libnimbus_cuda.so
	$(CXX) $(OBJS) $(OUT)/adapter.o -o $@ -L $(LIBDIR) -lnimbus_cuda -Wl,-rpath,'$$ORIGIN/../../lib' $(GOMP_LIBS)

.PHONY: all program
