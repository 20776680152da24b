#!/usr/bin/env python3
"""Instantiate the reference's ``*.h.in`` configuration templates for the oracle build.

This is test infrastructure: it only serves ``oracle/ref.mk``, which compiles the
reference N-body client's CPU path straight from its sources (no CMake) into
``oracle/_ref/``.  The reference configures these headers with CMake's
``configure_file``; this script performs the same substitution for the fixed
configuration the oracle uses (Linux x86-64, double precision, crlibm on,
OpenCL/BOINC/GL/curses off).

Templates read (paths inside the reference tree):
  milkyway/include/milkyway_config.h.in, milkyway/include/milkyway_git_version.h.in,
  nbody/include/nbody_config.h.in, lua/include/luaconf.h.in,
  popt/include/popt_config.h.in, openpa/include/opa_config.h.in,
  crlibm/crlibm_config.h.in (written twice: into the output directory for
  ``#include "crlibm_config.h"`` and into its parent, where crlibm's
  ``scs_lib/scs.h`` finds ``#include "../crlibm_config.h"`` through ``-I<output>``)

Usage: configure_ref.py <reference-root> <output-include-dir>
"""
import os
import re
import sys

VALUES = {
    # milkyway_config.h.in
    "BOINC_APPLICATION": "0", "DOUBLEPREC": "1", "MW_ENABLE_DEBUG": "0",
    "HAVE_EXP10": "1", "HAVE_EXP2": "1", "HAVE_SINCOS": "1", "HAVE_FMAX": "1",
    "HAVE_FMIN": "1", "HAVE_UNISTD_H": "1", "HAVE_WINDOWS_H": "0", "HAVE_DIRECT_H": "0",
    "HAVE_FCNTL_H": "1", "HAVE_SIGNAL_H": "1", "HAVE_PROCESS_H": "0",
    "HAVE_INTTYPES_H": "1", "HAVE_STDINT_H": "1", "HAVE_MALLOC_H": "1",
    "HAVE_FLOAT_H": "1", "HAVE_FPU_CONTROL_H": "1", "HAVE_SYS_RESOURCE_H": "1",
    "HAVE_SYS_MMAN_H": "1", "HAVE_SYS_TYPES_H": "1", "HAVE_SYS_STAT_H": "1",
    "HAVE_SYS_WAIT_H": "1", "HAVE_SYS_TIME_H": "1", "HAVE_ASPRINTF": "1",
    "HAVE_POSIX_MEMALIGN": "1", "HAVE__ALIGNED_MALLOC": "0",
    "HAVE___MINGW_ALIGNED_MALLOC": "0", "HAVE_CLOCK_GETTIME": "1",
    "HAVE_MACH_ABSOLUTE_TIME": "0", "HAVE_GETTIMEOFDAY": "1", "HAVE_SIGACTION": "1",
    "CMAKE_SYSTEM_NAME": "Linux",
    "MILKYWAY_GIT_COMMIT_ID": "oracle", "MILKYWAY_GIT_DESCRIBE": "oracle",
    # nbody_config.h.in
    "nbody_VERSION_MAJOR": "1", "nbody_VERSION_MINOR": "93", "nbody_VERSION": "1.93",
    "NBODY_OPENCL": "0", "NBODY_CRLIBM": "1", "USE_GL3W": "0", "ENABLE_CURSES": "0",
    "PROJECT_NAME": "nbody", "NBODY_BIN_NAME": "milkyway_nbody",
    "NBODY_GRAPHICS_BIN_NAME": "milkyway_nbody_graphics",
    # luaconf.h.in
    "LUA_USE_POSIX": "1", "LUA_USE_MKSTEMP": "1", "LUA_USE_ISATTY": "1",
    "LUA_USE_POPEN": "1", "LUA_PATH": "LUA_PATH", "LUA_CPATH": "LUA_CPATH",
    "LUA_INIT": "LUA_INIT", "LUA_DIRSEP": "/", "LUA_IDSIZE": "60",
    "LUA_PROMPT": "> ", "LUA_PROMPT2": ">> ", "LUA_MAXINPUT": "512",
    "LUA_PATH_DEFAULT": "./?.lua", "LUA_CPATH_DEFAULT": "./?.so",
    # popt_config.h.in
    "HAVE_DLFCN_H": "1", "HAVE_FNMATCH_H": "1", "HAVE_GLOB_H": "1",
    "HAVE_LANGINFO_H": "1", "HAVE_MEMORY_H": "1", "HAVE_SRANDOM": "1",
    "HAVE_STDLIB_H": "1", "HAVE_STPCPY": "1", "HAVE_STRERROR": "1",
    "HAVE_VASPRINTF": "1", "STDC_HEADERS": "1", "PROTOTYPES": "1", "__PROTOTYPES": "1",
    "POPT_VERSION": "1.16", "CMAKE_INSTALL_PREFIX": "/usr/local",
    # opa_config.h.in
    "OPA_HAVE_GCC_ATTRIBUTE": "1", "OPA_HAVE_GCC_INTRINSIC_ATOMICS": "1",
    "OPA_HAVE_GCC_X86_32_64": "1", "OPA_HAVE_GCC_X86_32_64_P3": "1",
    "OPA_HAVE_LIBPTHREAD": "1", "OPA_HAVE_PTHREAD_H": "1", "OPA_HAVE_PTHREAD_YIELD": "1",
    "OPA_HAVE_SCHED_YIELD": "1", "OPA_HAVE_STDDEF_H": "1",
    "MAX_NTHREADS": "100", "SIZEOF_INT": "4", "SIZEOF_VOID_P": "8",
    # crlibm_config.h.in
    "HAVE_FENV_H": "1",
}

TEMPLATES = [
    ("milkyway/include/milkyway_config.h.in", "milkyway_config.h"),
    ("milkyway/include/milkyway_git_version.h.in", "milkyway_git_version.h"),
    ("nbody/include/nbody_config.h.in", "nbody_config.h"),
    ("lua/include/luaconf.h.in", "luaconf.h"),
    ("popt/include/popt_config.h.in", "popt_config.h"),
    ("openpa/include/opa_config.h.in", "opa_config.h"),
    ("crlibm/crlibm_config.h.in", "crlibm_config.h"),
    ("crlibm/crlibm_config.h.in", os.path.join(os.pardir, "crlibm_config.h")),
]


def subst(text):
    text = re.sub(r"\$\{(\w+)\}", lambda m: VALUES.get(m.group(1), ""), text)
    return re.sub(r"@(\w+)@", lambda m: VALUES.get(m.group(1), ""), text)


def configure(src):
    out = []
    for line in src.splitlines():
        m = re.match(r"\s*#cmakedefine01\s+(\w+)", line)
        if m:
            out.append("#define %s %s" % (m.group(1), VALUES.get(m.group(1), "0")))
            continue
        m = re.match(r"\s*#cmakedefine\s+(\w+)(.*)$", line)
        if m:
            name, rest = m.group(1), m.group(2)
            if VALUES.get(name, "0") not in ("0", ""):
                rest = subst(rest).strip()
                if not rest or rest.startswith("/*"):
                    rest = "1"
                out.append("#define %s %s" % (name, rest))
            else:
                out.append("/* #undef %s */" % name)
            continue
        out.append(subst(line))
    return "\n".join(out) + "\n"


def main():
    ref, dst = sys.argv[1], sys.argv[2]
    os.makedirs(dst, exist_ok=True)
    for rel, name in TEMPLATES:
        with open(os.path.join(ref, rel)) as f:
            text = configure(f.read())
        path = os.path.join(dst, name)
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)


if __name__ == "__main__":
    main()
