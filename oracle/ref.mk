# Builds the reference itself (vaishna77/RCS) from its unmodified sources,
# where they lie, into oracle/_ref/aifmm_ref -- TEST INFRASTRUCTURE ONLY.
# Eigen 3, which the reference includes as <Eigen/Dense>, is not installed
# on this machine; the project-written subset in include/aifmm/Eigen stands in
# for it (the include directory below holds only that subset).  The compile
# definitions are the reference's CMake choices (CMakeLists.txt: DIM THREE,
# DTYPE complex64, C++17, OpenMP); -ffp-contract=off keeps a*b+c unfused as in
# its x86-64 build without -march flags.
#
#   make -f oracle/ref.mk REF=<path of the reference tree>
#
# The fixture scripts under tests/golden/ run the result; nothing in the
# product links or loads it.
REF      ?= $(AIFMM_REFERENCE_ROOT)
HERE     := $(dir $(lastword $(MAKEFILE_LIST)))
OUT      := $(HERE)_ref
CXX      := /usr/bin/g++
CXXFLAGS := -O2 -ffp-contract=off -fopenmp -std=c++17 -DUSE_THREE -DUSE_COMPLEX64 -w
SRCS     := includes.cpp kernel.cpp Patch.cpp EFIEMatrix.cpp AIFMMBox.cpp ACA.cpp AIFMM.cpp rrqr.cpp
OBJS     := $(addprefix $(OUT)/,$(SRCS:.cpp=.o))
EIGENDIR := $(OUT)/eigen_include

all: $(OUT)/aifmm_ref

$(EIGENDIR)/Eigen/Dense: $(HERE)../include/aifmm/Eigen/Dense $(HERE)../include/aifmm/Eigen/Core
	@test -n "$(REF)" || (echo "set REF or AIFMM_REFERENCE_ROOT to the reference tree" && false)
	@mkdir -p $(EIGENDIR)/Eigen
	cp $(HERE)../include/aifmm/Eigen/Dense $(HERE)../include/aifmm/Eigen/Core $(EIGENDIR)/Eigen/

$(OUT)/%.o: $(REF)/src/%.cpp $(EIGENDIR)/Eigen/Dense
	$(CXX) $(CXXFLAGS) -I$(EIGENDIR) -I$(REF)/include -c $< -o $@

$(OUT)/ref_driver.o: $(HERE)ref_driver.cpp $(EIGENDIR)/Eigen/Dense
	$(CXX) $(CXXFLAGS) -I$(EIGENDIR) -I$(REF)/include -c $< -o $@

$(OUT)/aifmm_ref: $(OBJS) $(OUT)/ref_driver.o
	$(CXX) -fopenmp -o $@ $^

clean:
	rm -rf $(OUT)

.PHONY: all clean
