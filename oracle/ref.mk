# Builds the reference's own CPU path (data/src/selm-main/src/mpi/SELM.cpp,
# SELM_Eulerian_Period.cpp, SELM_Lagrangian_LAMMPS.cpp, compiled unchanged from
# where they lie) against the project's single-rank MPI / FFTW-MPI / LAMMPS
# shims, into oracle/_ref/libselm_ref.so.  TEST INFRASTRUCTURE ONLY.
# Usage: make -f oracle/ref.mk
HERE := $(dir $(abspath $(lastword $(MAKEFILE_LIST))))
# the reference project root comes from SELM_REFERENCE_ROOT (default /root/reference)
SELM_REFERENCE_ROOT ?= /root/reference
REF ?= $(SELM_REFERENCE_ROOT)/data/src/selm-main/src/mpi
OUT := $(HERE)_ref/libselm_ref.so
CXX := $(firstword $(wildcard /usr/bin/g++) g++)
CC := $(firstword $(wildcard /usr/bin/gcc) gcc)
FLAGS := -O2 -fPIC -ffp-contract=off -w
SRC := $(REF)/SELM.cpp $(REF)/SELM_Eulerian_Period.cpp $(REF)/SELM_Lagrangian_LAMMPS.cpp \
       $(HERE)shim/shim.cpp $(HERE)ref_driver.cpp

all: $(OUT)

$(HERE)_ref/selm_oracle.o: $(HERE)selm_oracle.c $(HERE)selm_oracle.h
	@mkdir -p $(HERE)_ref
	$(CC) $(FLAGS) -std=c11 -c -o $@ $<

$(OUT): $(SRC) $(HERE)_ref/selm_oracle.o $(wildcard $(HERE)shim/include/*.h)
	@mkdir -p $(HERE)_ref
	$(CXX) $(FLAGS) -std=c++17 -include typeinfo -I$(HERE)shim/include -I$(REF) -shared -o $@ $(SRC) \
	    $(HERE)_ref/selm_oracle.o -lm

clean:
	rm -rf $(HERE)_ref

.PHONY: all clean
