# Compiles the reference's own vanilla kernels (unchanged, from the reference checkout) into
# oracle/_ref/libedgeref_O<order>_R<runs>_M<mechanisms>.so, driven by ref_driver.cpp.
# TEST INFRASTRUCTURE ONLY; needs the reference sources: EDGE_REF (or the EDGE_REFERENCE
# environment variable), else a checkout named "reference" beside this repository.
#   make -f ref.mk            builds the default configurations
#   make -f ref.mk CFGS="4_1_0"
EDGE_REF ?= $(or $(EDGE_REFERENCE),$(abspath $(CURDIR)/../../reference))
# the image exports CXX without OpenMP runtime files; the system compiler has them
CXX := $(if $(wildcard /usr/bin/g++),/usr/bin/g++,g++)
OUT := _ref
CFGS ?= 3_1_0 4_1_0 5_1_0 6_1_0 4_1_3 4_8_3 5_16_0
CXXFLAGS ?= -O3 -march=native -fopenmp -fPIC -std=c++11 -w
INC := -I$(EDGE_REF)/src -I$(EDGE_REF) -Ishim -I..
# the reference build's defines for a tet4 seismic FP64 vanilla binary (SConstruct:435-525)
defs = -DPP_T_EQUATIONS_SEISMIC -DPP_T_ELEMENTS_TET4 -DPP_PRECISION=64 -DPP_T_KERNELS_VANILLA \
       -DPP_ORDER=$(word 1,$(subst _, ,$1)) -DPP_N_CRUNS=$(word 2,$(subst _, ,$1)) \
       -DPP_N_RELAXATION_MECHANISMS=$(word 3,$(subst _, ,$1))
SRCS := $(EDGE_REF)/src/dg/Basis.cpp $(EDGE_REF)/src/impl/seismic/setups/Elasticity.cpp \
        $(EDGE_REF)/src/data/Dynamic.cpp $(EDGE_REF)/submodules/FastGL/fastgl.cpp

LIBS := $(foreach c,$(CFGS),$(OUT)/libedgeref_O$(word 1,$(subst _, ,$c))_R$(word 2,$(subst _, ,$c))_M$(word 3,$(subst _, ,$c)).so)
# the reference's AderDg class itself (local / neigh with the LTS branches), elastic
LTS_CFGS ?= 3_1 4_1 4_4
LTS_LIBS := $(foreach c,$(LTS_CFGS),$(OUT)/libedgeref_lts_O$(word 1,$(subst _, ,$c))_R$(word 2,$(subst _, ,$c)).so)

all: $(LIBS) $(LTS_LIBS)

$(OUT)/libedgeref_lts_O%.so: ref_lts.cpp
	@mkdir -p $(OUT)
	$(eval C := $(subst _R,_,$*))
	$(CXX) $(CXXFLAGS) $(INC) $(call defs,$(C)_0) -shared -o $@ ref_lts.cpp $(SRCS) $(EDGE_REF)/src/parallel/global.cpp

$(OUT)/libedgeref_O%.so: ref_driver.cpp
	@mkdir -p $(OUT)
	$(eval C := $(subst _R,_,$(subst _M,_,$*)))
	$(CXX) $(CXXFLAGS) $(INC) $(call defs,$(C)) -shared -o $@ ref_driver.cpp $(SRCS)

clean:
	rm -rf $(OUT)

.PHONY: all clean
