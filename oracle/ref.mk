# Builds the Jet reference's own CPU code into oracle/_ref/ -- TEST
# INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).
#
# The reference sources are compiled where they lie, unmodified, with g++
# against the Kokkos stand-in in kokkos_shim/ (the reference needs Kokkos and
# KokkosKernels, which are not installed) and CUDA's bundled static Metis.
# Outputs (all under _ref/, which is git-ignored):
#   jet_serial, jet_host, pstat      the reference's own apps (app/driver.cpp
#                                    with -DSERIAL / -DHOST, app/part_eval.cpp)
#   libjet_ref_serial.so             ref_harness.cpp over the reference, Serial
#   libjet_ref_host.so               the same over OpenMP (all host cores)
#
#   make -f ref.mk [REF=/path/to/reference]
REF ?= /root/reference
METIS_LIB ?= /usr/local/cuda/targets/x86_64-linux/lib/libmetis_static.a
# g++ from PATH (it has OpenMP); an inherited CXX may point at a compiler without libgomp.
REFCXX ?= g++
FLAGS = -O2 -std=c++17 -I kokkos_shim -I $(REF)/header -I $(REF)/src -I $(REF)/app
SHIM = $(wildcard kokkos_shim/*.h kokkos_shim/*.hpp)
REFSRC = $(wildcard $(REF)/src/*.hpp $(REF)/src/*.cpp $(REF)/header/*)
ENTRY = $(REF)/src/jet.cpp $(REF)/src/jet_big.cpp $(REF)/src/jet_biggest.cpp

all: _ref/libjet_ref_serial.so _ref/libjet_ref_host.so _ref/jet_serial _ref/jet_host _ref/pstat

_ref/libjet_ref_serial.so: ref_harness.cpp $(SHIM) $(REFSRC)
	mkdir -p _ref
	$(REFCXX) $(FLAGS) -fPIC -shared -DSERIAL -o $@ ref_harness.cpp $(ENTRY) $(METIS_LIB) -lm

_ref/libjet_ref_host.so: ref_harness.cpp $(SHIM) $(REFSRC)
	mkdir -p _ref
	$(REFCXX) $(FLAGS) -fPIC -shared -fopenmp -DHOST -o $@ ref_harness.cpp $(ENTRY) $(METIS_LIB) -lm

_ref/jet_serial: $(SHIM) $(REFSRC) $(REF)/app/driver.cpp $(REF)/app/io.hpp
	mkdir -p _ref
	$(REFCXX) $(FLAGS) -DSERIAL -o $@ $(REF)/app/driver.cpp $(REF)/src/jet.cpp $(METIS_LIB) -lm

_ref/jet_host: $(SHIM) $(REFSRC) $(REF)/app/driver.cpp $(REF)/app/io.hpp
	mkdir -p _ref
	$(REFCXX) $(FLAGS) -fopenmp -DHOST -o $@ $(REF)/app/driver.cpp $(REF)/src/jet.cpp $(METIS_LIB) -lm

_ref/pstat: $(SHIM) $(REFSRC) $(REF)/app/part_eval.cpp $(REF)/app/io.hpp
	mkdir -p _ref
	$(REFCXX) $(FLAGS) -fopenmp -DHOST -o $@ $(REF)/app/part_eval.cpp $(METIS_LIB) -lm

clean:
	rm -rf _ref

.PHONY: all clean
