# Builds the reference Nimbus CPU solver's own sources, where they lie, into
# oracle/_ref/ (git-ignored). This is test infrastructure: the archive and the
# harness library built from it serve only as the checker for the CUDA path
# and as the timed CPU baseline. It is NOT the reference's build system; it is
# a flat compile of every solver translation unit with portable flags.
#
#   make -f oracle/ref.mk REF=/path/to/reference -j8
#
# REF is required (the build recipe passes NIMBUS_REFERENCE_DIR).
#
# Portability: no -march=native (the archive must run on any x86-64 host the
# library travels to) and -ffp-contract=off (no FMA contraction), so the
# reference's arithmetic is the plain IEEE sequence its sources spell out.
REF      ?= $(NIMBUS_REFERENCE_DIR)
ifeq ($(strip $(REF)),)
$(error REF (or NIMBUS_REFERENCE_DIR) must name the reference solver's source tree)
endif
OUT      ?= oracle/_ref
OBJDIR   := $(OUT)/obj
CXX      ?= g++
CXXFLAGS := -std=c++17 -O2 -fPIC -fopenmp -ffp-contract=off -w \
            -DNIMBUS_CPU_ONLY -DNIMBUS_PORTABLE_BUILD -I $(REF)/include -I $(REF)/src
SRCS     := $(filter-out $(REF)/src/tools/%,\
              $(shell find $(REF)/src -name '*.cpp' | sort))
OBJS     := $(patsubst $(REF)/src/%.cpp,$(OBJDIR)/%.o,$(SRCS))

all: $(OUT)/libnimbus_ref.a

# The CLI translation unit also defines helpers other units call; its main()
# is renamed so the archive can be linked into a shared library.
$(OBJDIR)/core/runtime/nimbus_sim.o: CXXFLAGS += -Dmain=nimbus_reference_cli_main

$(OBJDIR)/%.o: $(REF)/src/%.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -c $< -o $@ || (echo "SKIP $<" && rm -f $@ && touch $@.skip)

$(OUT)/libnimbus_ref.a: $(OBJS)
	rm -f $@
	ar rcs $@ $(filter-out %.skip,$(wildcard $(OBJS)))

.PHONY: all

# The harness library the tests and the CPU baseline load.  The archive is
# linked whole-program style: only objects the harness reaches are pulled in.
GOMP_LIBS ?= -L/usr/lib/gcc/x86_64-linux-gnu/13 -lgomp -lpthread
harness: $(OUT)/libnimbus_ref_harness.so

$(OUT)/libnimbus_ref_harness.so: oracle/ref_harness.cpp $(OUT)/libnimbus_ref.a
	$(CXX) $(CXXFLAGS) -c oracle/ref_harness.cpp -o $(OUT)/ref_harness.o
	$(CXX) -shared $(OUT)/ref_harness.o -o $@ $(OUT)/libnimbus_ref.a $(GOMP_LIBS) -Wl,--no-undefined

.PHONY: harness

# The reference's command-line program from the same objects (its main() is
# compiled as nimbus_reference_cli_main): the stock CPU path bench.py times.
cli: $(OUT)/nimbus_sim_ref

$(OUT)/nimbus_sim_ref: oracle/ref_cli.cpp $(OUT)/libnimbus_ref.a
	$(CXX) -std=c++17 -O2 -c oracle/ref_cli.cpp -o $(OUT)/ref_cli.o
	$(CXX) $(OUT)/ref_cli.o -o $@ -Wl,--whole-archive $(OUT)/libnimbus_ref.a -Wl,--no-whole-archive $(GOMP_LIBS)

.PHONY: cli
