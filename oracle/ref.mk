# Compiles oracle/ref_driver.cpp against the reference's own headers and the
# few source files that define what those headers declare, where they lie,
# into oracle/_ref/ref_driver (git-ignored).  Test infrastructure only.
# Needs nothing beyond the reference tree: FIXED_K turns off the one boost macro
# that include/globals.hpp would use (ref_shim/ holds an empty stand-in for that
# include), and the vendored fmt is used header-only.  The driver is built with
# FIXED_K=127 (INSTANCE_COUNT 64: Kmer<k> for every k <= 127).
# REF: the reference tree, given on the command line (make -f ref.mk REF=<dir>)
ifndef REF
$(error REF=<reference tree> is required)
endif
CXX      ?= g++
OUT      := _ref
KS       := 3 5 7 9 15 23 31 63 95 127
BASE     := -std=c++17 -O2 -w -DL1_CACHE_LINE_SIZE=64 -DFMT_HEADER_ONLY -Iref_shim -I$(REF)/include
MUS_OBJ  := $(foreach k,$(KS),$(OUT)/mus_$(k).o)

$(OUT)/ref_driver: ref_driver.cpp $(MUS_OBJ) ref_shim/boost/preprocessor/repetition/repeat.hpp
	@mkdir -p $(OUT)
	$(CXX) $(BASE) -DFIXED_K=127 -o $@ ref_driver.cpp $(REF)/src/State_Config.cpp \
	    $(REF)/src/Character_Buffer_Flusher.cpp $(MUS_OBJ)

# src/Maximal_Unitig_Scratch.cpp instantiates only FIXED_K; build it once per k.
$(OUT)/mus_%.o: $(REF)/src/Maximal_Unitig_Scratch.cpp
	@mkdir -p $(OUT)
	$(CXX) $(BASE) -DFIXED_K=$* -c -o $@ $<
