# Builds QPhiX's own code-generated Dslash kernels and drives them through the
# reference's own class templates -- TEST INFRASTRUCTURE AND CPU BASELINE ONLY.
#
#   make -f codegen.mk ISA=scalar    -> ../_ref/libqphix_ref_dslash_scalar.so
#   make -f codegen.mk ISA=avx512    -> ../_ref/libqphix_ref_dslash_avx512.so
#
# Steps (none of them runs the reference's CMake build):
#  1. the generator (codegen/codegen.cc, data_types.cc, dslash.cc,
#     dslash_common.cc, inst_*.cc) is compiled with g++ once per
#     (PRECISION, VECLEN, SOALEN), with the option macros that
#     codegen/CMakeLists.txt sets for the ISA, and run: it writes the kernel
#     bodies to $(BUILD)/generated/$(ISA)/generated/;
#  2. codegen/jinja/generate_files.py renders the specialisation sources
#     (one per kernel, FT, V, S, compress12 and twisted-boundary pattern);
#  3. the specialisations of the variants below are compiled with g++ and
#     linked with ref_dslash.cc and lib/print_utils.cc.
# Everything is written under oracle/_build/ (intermediates) and oracle/_ref/.
REF ?= /root/reference
ISA ?= scalar
PY ?= python3
CG := $(REF)/codegen
BUILD := $(abspath ../_build/codegen/$(ISA))
OUT := $(abspath ../_ref)
CXX := g++

GEN_SRC := $(CG)/codegen.cc $(CG)/data_types.cc $(CG)/dslash.cc $(CG)/dslash_common.cc \
           $(CG)/inst_dp_vec8.cc $(CG)/inst_sp_vec16.cc $(CG)/inst_dp_vec4.cc $(CG)/inst_sp_vec8.cc \
           $(CG)/inst_sp_vec4.cc $(CG)/inst_dp_vec2.cc $(CG)/inst_scalar.cc

# option macros of codegen/CMakeLists.txt for each ISA; variants are
# PRECISION_VECLEN_SOALEN (generator) and fptype_VECLEN_SOALEN (specialisations)
ifeq ($(ISA),scalar)
GEN_DEFS := -DSERIAL_SPIN -DUSE_LDUNPK -DUSE_PKST -DENABLE_STREAMING_STORES -DUSE_PACKED_GAUGES \
            -DUSE_PACKED_CLOVER -DNO_HW_MASKING -DNO_MASKS
GEN_VARIANTS := 2_1_1 1_1_1
SPEC_VARIANTS := double_1_1 float_1_1
ARCH_FLAGS :=
ISA_DEF := -DQPHIX_REF_ISA_SCALAR
else ifeq ($(ISA),avx512)
GEN_DEFS := -DSERIAL_SPIN -DUSE_LDUNPK -DUSE_PKST -DENABLE_STREAMING_STORES -DUSE_PACKED_GAUGES \
            -DUSE_PACKED_CLOVER -DAVX512
GEN_VARIANTS := 2_8_4 2_8_8 1_16_8
SPEC_VARIANTS := double_8_4 double_8_8 float_16_8
# AVX-512 F/CD/BW/DQ/VL only, so the library runs on any AVX-512 Xeon host
ARCH_FLAGS := -march=skylake-avx512 -mtune=skylake-avx512
ISA_DEF := -DQPHIX_REF_ISA_AVX512
else
$(error ISA must be scalar or avx512)
endif

KERNELS := dslash clov_dslash tm_clov_dslash tm_dslash
TBC := $(foreach a,s t,$(foreach b,s t,$(foreach c,s t,$(foreach d,s t,$(a)$(b)$(c)$(d)))))
SPEC_NAMES := $(foreach k,$(KERNELS),$(foreach v,$(SPEC_VARIANTS),$(foreach c,compress12 compress18,\
                $(k)_$(ISA)_spec_$(v)_$(c) $(foreach t,$(TBC),$(k)_$(ISA)_spec_$(v)_$(c)_$(t)))))
SPEC_OBJS := $(addprefix $(BUILD)/obj/,$(addsuffix .o,$(SPEC_NAMES)))

LIB_FLAGS := -std=c++14 -O2 -fPIC -fopenmp -w -Drestrict=__restrict__ -include cstdint -include cassert \
             $(ARCH_FLAGS) $(ISA_DEF)
LIB_INC := -I$(abspath shim) -I$(BUILD)/generated/$(ISA) -I$(BUILD)/inc -I$(REF)/include

LIBSO := $(OUT)/libqphix_ref_dslash_$(ISA).so

all: $(LIBSO)

# 1. generator binaries and their output
$(BUILD)/gen_%/output_dir.h:
	@mkdir -p $(dir $@)
	printf '#ifndef _OUTPUT_DIR_H\n#define _OUTPUT_DIR_H\n#include <string>\nstd::string output_dir = "%s";\n#endif\n' \
	  "$(BUILD)" > $@

$(BUILD)/gen_%/codegen: $(BUILD)/gen_%/output_dir.h
	$(CXX) -O1 -std=c++11 -w $(GEN_DEFS) \
	  -DPRECISION=$(word 1,$(subst _, ,$*)) -DVECLEN=$(word 2,$(subst _, ,$*)) -DSOALEN=$(word 3,$(subst _, ,$*)) \
	  -I$(dir $@) -I$(CG) $(GEN_SRC) -o $@

$(BUILD)/gen_%/generated.stamp: $(BUILD)/gen_%/codegen
	@mkdir -p $(BUILD)/generated/$(ISA)/generated
	$< > $(BUILD)/gen_$*/codegen.log
	touch $@

# 2. specialisation sources (run from a directory beside generated/, as the
#    script expects)
$(BUILD)/jinja.stamp: $(foreach v,$(GEN_VARIANTS),$(BUILD)/gen_$(v)/generated.stamp)
	@mkdir -p $(BUILD)/jinja
	cd $(BUILD)/jinja && $(PY) $(CG)/jinja/generate_files.py $(ISA) > generate_files.log
	@mkdir -p $(BUILD)/inc/qphix_codegen
	cp $(BUILD)/generated/*_generated.h $(BUILD)/generated/$(ISA)/include/*_decl.h $(BUILD)/inc/qphix_codegen/
	touch $@

# 3. compiled specialisations and the harness
$(BUILD)/obj/%.o: $(BUILD)/jinja.stamp
	@mkdir -p $(BUILD)/obj
	$(CXX) $(LIB_FLAGS) $(LIB_INC) -c $(BUILD)/generated/$(ISA)/src/$*.cpp -o $@

$(BUILD)/obj/ref_dslash.o: ref_dslash.cc $(BUILD)/jinja.stamp $(wildcard shim/qphix/*.h)
	@mkdir -p $(BUILD)/obj
	$(CXX) $(LIB_FLAGS) $(LIB_INC) -c ref_dslash.cc -o $@

$(LIBSO): $(BUILD)/obj/ref_dslash.o $(SPEC_OBJS)
	@mkdir -p $(OUT)
	$(CXX) -shared -fopenmp -o $@ $(BUILD)/obj/ref_dslash.o $(SPEC_OBJS) \
	  $(LIB_FLAGS) $(LIB_INC) $(REF)/lib/print_utils.cc

# generated intermediates are kept between runs
.SECONDARY:

clean:
	rm -rf $(BUILD) $(LIBSO)
.PHONY: all clean
