# Builds fvhyper's example programs, unchanged, against the B200 fvhyper API
# (include/fvhyper/*.h + libfvhyper_gpu.a + libfvgpu.so).  The example sources
# are compiled where they lie in the reference checkout (REF); the programs go
# to shim/_examples/, which is not committed.
#   make -C finite-volume-2d-cpp_b200/shim -f examples.mk REF=<fvhyper checkout>
REF ?= $(FVHYPER_SRC)
CXX ?= g++
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
PKG := $(abspath $(HERE)..)
OUT := $(HERE)_examples
EXAMPLES := shockTube forwardStep naca burgers flatPlate heatTransfer nacaTransient

ifeq ($(strip $(REF)),)
all:
	@echo "examples: set FVHYPER_SRC (or REF=...) to the fvhyper source checkout" >&2; exit 1
else
all: $(EXAMPLES:%=$(OUT)/%) $(OUT)/naca0012_129.su2
endif

# the SU2 mesh fvhyper ships for its NACA example (read directly by the shim)
$(OUT)/naca0012_129.su2: $(REF)/examples/naca/naca0012_129.su2 | $(OUT)
	cp $< $@

$(OUT):
	mkdir -p $(OUT)

# the user physics callbacks keep the reference's FP semantics (no contraction)
$(OUT)/%: $(REF)/examples/%/main.cpp $(PKG)/libfvhyper_gpu.a $(PKG)/libfvgpu.so | $(OUT)
	$(CXX) -O2 -std=c++17 -ffp-contract=off -fno-fast-math -w -I$(PKG)/../include $< \
	    $(PKG)/libfvhyper_gpu.a -L$(PKG) -lfvgpu -Wl,-rpath,'$$ORIGIN/..:$$ORIGIN/../..' -o $@

.PHONY: all
