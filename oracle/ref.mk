# Builds oracle/_ref/kat_runner: the reference's own unit-test sources for the
# hot path's integer/bit-level helpers, the BSDF lobes' sampling statistics
# and the gradient aggregation (hypothesis' chi^2 header from the reference's
# external/include), compiled from where they lie under the
# reference tree (read-only), with oracle/ref_shim standing in for Falcor's
# test framework and the oracle standing in for the Slang test programs; plus
# the reference's Utils/Math/Float16.cpp.  Test infrastructure only; the
# outputs go to oracle/_ref/ (git-ignored).  Run from oracle/:
#   make -f ref.mk            (FALCOR_REF names the reference checkout)
FALCOR_REF ?= /root/reference
REF ?= $(FALCOR_REF)/Source
TESTS := $(REF)/Tools/FalcorTest/Tests
CXX ?= g++
CXXFLAGS ?= -O2 -std=gnu++20 -ffp-contract=off -Wno-unused-function -Wno-unused-variable
OUT := _ref
SRCS := $(TESTS)/Sampling/PseudorandomTests.cpp $(TESTS)/Utils/HashUtilsTests.cpp $(TESTS)/Utils/BitTricksTests.cpp \
        $(TESTS)/Utils/GeometryHelpersTests.cpp $(TESTS)/Scene/Material/BSDFTests.cpp \
        $(TESTS)/DiffRendering/SceneGradientsTest.cpp $(REF)/Falcor/Utils/Math/Float16.cpp kat_main.cpp kat_bsdf.cpp

all: $(OUT)/kat_runner

$(OUT)/kat_runner: $(SRCS) ref_shim/Testing/UnitTest.h ref_shim/DiffRendering/SceneGradients.h oracle_math.h oracle_gradients.h \
                   ../falcor_b200/csrc/fmath.h
	@mkdir -p $(OUT)
	$(CXX) $(CXXFLAGS) -I ref_shim -I $(REF)/Falcor -I $(FALCOR_REF)/external/include -I . -o $@ $(SRCS) -lpthread

.PHONY: all
