# Builds the reference (pnnl/ripples) CPU path from its own sources, where they
# lie, into oracle/_ref/ (git-ignored; it still travels to the GPU box).
# Third-party pieces absent offline are replaced by the project's interface
# shims (oracle/shims: trng4 lcg64 + distributions, CLI11 App); spdlog (bundled
# fmt) and nlohmann_json come from header trees vendored in this image.
# Flags mirror the reference's default compile definitions (CMakeLists.txt:57-67).
#
#   make -f oracle/ref.mk            (from the repository root)
# The sources are found through REF, else RIPPLES_REFERENCE_DIR from the
# environment, else the recipe's default location.
REF      ?= $(or $(RIPPLES_REFERENCE_DIR),/root/reference)
SITE     ?= $(shell python -c "import site;print(site.getsitepackages()[0])")
SPDLOG   ?= $(SITE)/flashinfer/data/spdlog/include
NLOHMANN ?= $(SITE)/include/cudnn_frontend/thirdparty
OUT      ?= oracle/_ref
REFCXX   ?= g++
DEFS     := -DNDEBUG -DSORTING=1 -DREORDERING=1 -DRIPPLES_ENABLE_FLOAT_WEIGHTS=1
INC      := -I$(REF)/include -Ioracle/shims -I$(SPDLOG) -I$(NLOHMANN)
FLAGS    := -O3 -fopenmp -std=c++17 -w $(DEFS) $(INC)

all: $(OUT)/imm $(OUT)/opimc $(OUT)/simulator $(OUT)/libref_harness.so $(OUT)/adapter_imm

$(OUT):
	mkdir -p $(OUT)

$(OUT)/imm: $(REF)/tools/imm.cc | $(OUT)
	$(REFCXX) $(FLAGS) $< -o $@

$(OUT)/opimc: $(REF)/tools/opimc.cc | $(OUT)
	$(REFCXX) $(FLAGS) $< -o $@

$(OUT)/simulator: $(REF)/tools/simulator.cc | $(OUT)
	$(REFCXX) $(FLAGS) $< -o $@

# Integration check of the drop-in adapter (include/ripples_b200/imm_adapter.hpp)
# compiled against the reference headers and linked to the in-tree library.
LIBDIR   := $(abspath ripples_b200/_lib)
$(OUT)/adapter_imm: tests/integration/adapter_imm.cc include/ripples_b200/imm_adapter.hpp include/ripples_b200.h $(LIBDIR)/libripples_b200.so | $(OUT)
	$(REFCXX) $(FLAGS) -Iinclude $< -o $@ -L$(LIBDIR) -lripples_b200 -Wl,-rpath,'$$ORIGIN/../../ripples_b200/_lib'

$(OUT)/libref_harness.so: oracle/ref_harness.cpp | $(OUT)
	$(REFCXX) $(FLAGS) -fPIC -shared $< -o $@

.PHONY: all
