# Compiles the reference's own `cuttlefish build` path -- Application, dBG_Contractor,
# Graph_Partitioner (RabbitFX reader), Subgraphs_Manager, Subgraph, the atlases and
# buckets, and the discontinuity-graph phases -- from its sources where they lie, into
# oracle/_ref/cuttlefish_ref_<k> (git-ignored), one binary per k (the reference fixes k
# at build time the same way with FIXED_K).  oracle/ref_shim/ holds stand-ins for what
# the reference tree does not vendor: parlaylib (a thread pool), cereal (no-op
# archives), boost's preprocessor repeat (unused with FIXED_K) and concurrent_flat_map
# (colored runs only), rapidgzip, and lz4's header (the system library is linked);
# ref_rabbit_reader.cpp stands in for RabbitFX's FileReader.cpp, which needs ISA-L.
# jemalloc is left out.  Test and baseline infrastructure.
#   make -f ref_app.mk REF=<reference tree>
ifndef REF
$(error REF=<reference tree> is required)
endif
CXX      ?= g++
OUT      := _ref
KS       := 31 63 95 127
BASE     := -std=c++17 -O3 -w -DL1_CACHE_LINE_SIZE=64 -DFMT_HEADER_ONLY -pthread -include cstdint \
            -include ref_shim/flushing_ofstream.hpp
INC      := -Iref_shim_app -Iref_shim -I$(REF)/include -I$(REF)/include/RabbitFX -I$(REF)/src
SRC      := dBG_Contractor Graph_Partitioner Subgraphs_Manager Subgraph Atlas Super_Kmer_Bucket Super_Kmer_Chunk \
            HyperLogLog Color_Table Color_Repo State_Config Build_Params Seq_Input utility Data_Logistics \
            Discontinuity_Graph Discontinuity_Graph_Contractor Contracted_Graph_Expander Unitig_Collator Edge_Matrix \
            Unitig_File Maximal_Unitig_Scratch Character_Buffer_Flusher Async_Logger_Wrapper DNA_Utility Kmer_Utility \
            Unitig_Coord_Bucket Minimizer_Instance_Iterator Minimizer_Policy
RABBIT   := Formater FastxStream
LZ4      := /usr/lib/x86_64-linux-gnu/liblz4.so.1

all: $(foreach k,$(KS),$(OUT)/cuttlefish_ref_$(k))

define per_k
$(OUT)/app$(1)/%.o: $(REF)/src/%.cpp
	@mkdir -p $(OUT)/app$(1)
	$(CXX) $(BASE) -DFIXED_K=$(1) $(INC) -c -o $$@ $$<
$(OUT)/app$(1)/rabbit_%.o: $(REF)/include/RabbitFX/io/%.cpp
	@mkdir -p $(OUT)/app$(1)
	$(CXX) $(BASE) -DFIXED_K=$(1) $(INC) -c -o $$@ $$<
$(OUT)/app$(1)/ref_rabbit_reader.o: ref_rabbit_reader.cpp
	@mkdir -p $(OUT)/app$(1)
	$(CXX) $(BASE) -DFIXED_K=$(1) $(INC) -c -o $$@ $$<
$(OUT)/cuttlefish_ref_$(1): ref_app.cpp $(foreach s,$(SRC),$(OUT)/app$(1)/$(s).o) $(foreach s,$(RABBIT),$(OUT)/app$(1)/rabbit_$(s).o) $(OUT)/app$(1)/ref_rabbit_reader.o $(OUT)/xxhash.o
	$(CXX) $(BASE) -DFIXED_K=$(1) $(INC) -o $$@ $$^ $(LZ4) -lz
endef
$(foreach k,$(KS),$(eval $(call per_k,$(k))))

$(OUT)/xxhash.o: $(REF)/src/xxHash/xxhash.c
	@mkdir -p $(OUT)
	gcc -O2 -I$(REF)/include -c -o $@ $<

.PHONY: all
