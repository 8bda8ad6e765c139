# Builds oracle/_ref/history_ref: the reference's header-only IntersectionHistory
# (src/CPU/IntersectionHistory.h) compiled where it lies, with the program
# history_ref_main.cpp.  Test infrastructure; needs the reference tree (REF) and
# CUDA's vector_types.h.  Usage: make -f history_ref.mk REF=<reference root>
ifndef REF
$(error REF must name the reference project's root directory)
endif
CUDA ?= /usr/local/cuda
CXX ?= g++
HERE := $(dir $(lastword $(MAKEFILE_LIST)))

$(HERE)_ref/history_ref: $(HERE)history_ref_main.cpp $(REF)/src/CPU/IntersectionHistory.h
	mkdir -p $(HERE)_ref
	$(CXX) -O2 -std=c++17 -I$(REF)/src -I$(CUDA)/include $(HERE)history_ref_main.cpp -o $@
