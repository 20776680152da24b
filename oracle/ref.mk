# Compile the reference N-body client's CPU path straight from its sources.
#
# Test infrastructure only: the products land in oracle/_ref/ (git-ignored) and are
# used by the tests and by bench.py's CPU baseline as the checker, never by the
# product path.  No CMake is run: the few configuration headers the reference
# generates with CMake are instantiated from its own *.h.in templates by
# configure_ref.py, and the one source that is a missing blob in the reference
# tree (nbody/src/nbody_bessel.c, used only by the exponential disks) is replaced
# by bessel_placeholder.c, which fails loudly if it is ever called.
#
#   make -f oracle/ref.mk REF=/path/to/reference        (run from the repo root)
#
# Without REF, the reference checkout is looked for beside this repository (../reference
# relative to the repository root); a variable MILKYWAY_REFERENCE_SRC in the environment
# overrides that.
#
# Products:
#   oracle/_ref/milkyway_nbody   the reference executable (golden likelihood runs)
#   oracle/_ref/libnbref.so      the reference objects + ref_shim.c (ctypes entry points)
#   oracle/_ref/milkyway_nbody_cuda
#                                the reference executable with the B200 binding compiled in:
#                                milkywayathome_client_b200/reference_binding/nbody_cuda.c and
#                                the reference's nbody.c, nbody_plain.c and nbody_types.c with
#                                its dispatches added (oracle/apply_cuda_binding.py), linked
#                                against milkywayathome_client_b200/libnbody_b200.so; it steps
#                                on the GPU when NBODY_CUDA_DEVICE names one, else on the CPU

REPO    := $(abspath $(dir $(lastword $(MAKEFILE_LIST)))..)
REF     ?= $(or $(MILKYWAY_REFERENCE_SRC),$(abspath $(REPO)/../reference))
OUT     := oracle/_ref
OBJ     := $(OUT)/obj
GEN     := $(OUT)/include
CC      := /usr/bin/gcc
CXX     := /usr/bin/g++

# Flags the reference's CMake build uses on x86-64 (CMakeLists.txt: -std=gnu99,
# -fno-unsafe-math-optimizations; cmake_modules/CheckSSE2.cmake: -mfpmath=sse -msse2;
# Release -O3 -DNDEBUG; dSFMT -DDSFMT_MEXP=19937; OpenMP on).
DEFS    := -DDOUBLEPREC=1 -DDSFMT_MEXP=19937 -DNDEBUG -DHAVE_CONFIG_H \
           -DSCS_NB_WORDS=8 -DSCS_NB_BITS=30 -DCRLIBM_TYPECPU_AMD64 -DLUA_USE_APICHECK
INCS    := -I$(GEN) -I$(REF)/milkyway/include -I$(REF)/nbody/include -I$(REF)/lua/include \
           -I$(REF)/dSFMT -I$(REF)/crlibm -I$(REF)/popt/include -I$(REF)/openpa/include
CFLAGS  := -O3 -std=gnu99 -fPIC -fopenmp -fno-unsafe-math-optimizations -mfpmath=sse -msse2 \
           -w $(DEFS) $(INCS)
CXXFLAGS:= -O3 -fPIC -fopenmp -fno-unsafe-math-optimizations -mfpmath=sse -msse2 -w $(DEFS) $(INCS)

CRLIBM_SRC := crlibm_private.c triple-double.c exp-td.c exp-td-standalone.c expm1-standalone.c \
              expm1.c log.c log1p.c rem_pio2_accurate.c trigo_fast.c trigo_accurate.c trigpi.c \
              asincos.c pow.c atan_fast.c atan_accurate.c csh_fast.c \
              scs_lib/scs_private.c scs_lib/addition_scs.c scs_lib/division_scs.c \
              scs_lib/print_scs.c scs_lib/double2scs.c scs_lib/zero_scs.c \
              scs_lib/multiplication_scs.c scs_lib/scs2double.c
LUA_SRC    := lapi.c lcode.c ldebug.c ldo.c ldump.c lfunc.c lgc.c llex.c lmem.c lobject.c \
              lopcodes.c lparser.c lstate.c lstring.c ltable.c ltm.c lundump.c lvm.c lzio.c \
              lauxlib.c lbaselib.c ldblib.c liolib.c lmathlib.c loslib.c ltablib.c lstrlib.c \
              linit.c loadlib_rel.c
POPT_SRC   := popt.c poptparse.c poptconfig.c popthelp.c poptint.c
MW_SRC     := milkyway_util.c milkyway_alloc.c milkyway_rename.c milkyway_show.c \
              milkyway_cpuid.c milkyway_timing.c milkyway_lua_marshal.c milkyway_lua_util.c \
              milkyway_lua_math.c milkyway_lua_vector.c milkyway_lua_dsfmt.c milkyway_lua_types.c
MW_CXX     := milkyway_boinc_util.cc
NB_SRC     := nbody_chisq.c nbody_grav.c nbody_io.c nbody_curses.c nbody_types.c nbody_tree.c \
              nbody_orbit_integrator.c nbody_potential.c nbody_virial.c nbody_density.c \
              nbody_friction.c nbody.c nbody_plain.c nbody_check_params.c nbody_isotropic.c \
              nbody_mixeddwarf.c nbody_manual_bodies.c nbody_dwarf_potential.c nbody_plummer.c \
              nbody_nfw.c nbody_hernq.c nbody_show.c nbody_checkpoint.c nbody_defaults.c \
              nbody_coordinates.c nbody_shmem.c nbody_util.c nbody_emd.c nbody_mass.c \
              nbody_devoptions.c nbody_likelihood.c nbody_histogram.c nbody_caustic.c \
              nbody_particle_data.c blender_visualizer.c \
              nbody_lua.c nbody_lua_models.c nbody_lua_util.c nbody_lua_misc.c \
              nbody_lua_types/nbody_lua_types.c nbody_lua_types/nbody_lua_type_marshal.c \
              nbody_lua_types/nbody_lua_nbodystate.c nbody_lua_types/nbody_lua_nbodyctx.c \
              nbody_lua_types/nbody_lua_body.c nbody_lua_types/nbody_lua_halo.c \
              nbody_lua_types/nbody_lua_disk.c nbody_lua_types/nbody_lua_spherical.c \
              nbody_lua_types/nbody_lua_dwarf.c nbody_lua_types/nbody_lua_potential.c \
              nbody_lua_types/nbody_lua_histogram_params.c

OBJS := $(addprefix $(OBJ)/crlibm/,$(CRLIBM_SRC:.c=.o)) \
        $(OBJ)/dsfmt/dSFMT.o \
        $(addprefix $(OBJ)/lua/,$(LUA_SRC:.c=.o)) \
        $(addprefix $(OBJ)/popt/,$(POPT_SRC:.c=.o)) \
        $(addprefix $(OBJ)/milkyway/,$(MW_SRC:.c=.o)) \
        $(addprefix $(OBJ)/milkyway/,$(MW_CXX:.cc=.o)) \
        $(addprefix $(OBJ)/nbody/,$(NB_SRC:.c=.o)) \
        $(OBJ)/local/bessel_placeholder.o

all: $(OUT)/milkyway_nbody $(OUT)/libnbref.so

LIBDIR   := milkywayathome_client_b200
BIND     := $(LIBDIR)/reference_binding
CUDA_SRC := $(OUT)/cuda_src
PATCHED  := nbody.c nbody_plain.c nbody_types.c
CUDA_OBJS := $(addprefix $(OBJ)/cuda/,$(PATCHED:.c=.o)) $(OBJ)/cuda/nbody_cuda.o

$(GEN)/.stamp: oracle/configure_ref.py
	python3 oracle/configure_ref.py $(REF) $(GEN)
	touch $@

$(OBJ)/crlibm/%.o: $(REF)/crlibm/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -I$(REF)/crlibm/scs_lib -c $< -o $@

$(OBJ)/dsfmt/%.o: $(REF)/dSFMT/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -finline-functions -fno-strict-aliasing -c $< -o $@

$(OBJ)/lua/%.o: $(REF)/lua/src/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@

$(OBJ)/popt/%.o: $(REF)/popt/src/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@

# per-library compile definitions from milkyway/CMakeLists.txt:176-188 and
# nbody/CMakeLists.txt:250-252
$(OBJ)/milkyway/milkyway_lua_%.o: $(REF)/milkyway/src/milkyway_lua_%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -DMILKYWAY_LUA_COMPILATION -c $< -o $@

$(OBJ)/milkyway/%.o: $(REF)/milkyway/src/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -DMILKYWAY_MATH_COMPILATION -c $< -o $@

$(OBJ)/milkyway/%.o: $(REF)/milkyway/src/%.cc $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -DMILKYWAY_MATH_COMPILATION -c $< -o $@

$(OBJ)/nbody/nbody_lua%.o: $(REF)/nbody/src/nbody_lua%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -DNBODY_LUA_TYPES_COMPILATION -c $< -o $@

$(OBJ)/nbody/%.o: $(REF)/nbody/src/%.c $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@

$(OBJ)/local/%.o: oracle/%.c oracle/ref.mk $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -Iinclude -I$(REF)/nbody/src -c $< -o $@

$(OUT)/milkyway_nbody: $(OBJ)/nbody/main.o $(OBJS)
	$(CXX) -fopenmp -o $@ $^ -lm -lrt -lpthread -ldl

# ref_shim.c compiles nbody_grav.c itself (for its file-static walk), so the library takes
# every reference object except nbody_grav.o
$(OUT)/libnbref.so: $(OBJ)/local/ref_shim.o $(filter-out $(OBJ)/nbody/nbody_grav.o,$(OBJS))
	$(CXX) -shared -fopenmp -o $@ $^ -lm -lrt -lpthread -ldl

# the reference executable with the B200 binding (needs libnbody_b200.so built first)
cuda: $(OUT)/milkyway_nbody_cuda

$(CUDA_SRC)/.stamp: oracle/apply_cuda_binding.py $(addprefix $(REF)/nbody/src/,$(PATCHED))
	python3 oracle/apply_cuda_binding.py $(REF) $(CUDA_SRC)
	touch $@

$(CUDA_SRC)/%.c: $(CUDA_SRC)/.stamp ;

$(OBJ)/cuda/%.o: $(CUDA_SRC)/%.c $(BIND)/nbody_cuda.h $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -I$(BIND) -I$(REF)/nbody/src -c $< -o $@

$(OBJ)/cuda/nbody_cuda.o: $(BIND)/nbody_cuda.c $(BIND)/nbody_cuda.h $(BIND)/nbody_cuda_ctx.h \
                          include/nbody_b200.h $(GEN)/.stamp
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -Iinclude -I$(BIND) -c $< -o $@

$(OUT)/milkyway_nbody_cuda: $(OBJ)/nbody/main.o $(CUDA_OBJS) \
                            $(filter-out $(addprefix $(OBJ)/nbody/,$(PATCHED:.c=.o)),$(OBJS)) \
                            $(LIBDIR)/libnbody_b200.so
	$(CXX) -fopenmp -o $@ $(filter %.o,$^) -L$(LIBDIR) -lnbody_b200 \
	    -Wl,-rpath,'$$ORIGIN/../../$(LIBDIR)' -lm -lrt -lpthread -ldl

.PHONY: all cuda
