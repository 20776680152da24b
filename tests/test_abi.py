"""The C ABI: every entry point include/nbody_b200.h declares is exported by the built
library and bound by the Python mirror; the struct layouts agree.  No GPU calls."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nbody_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:NBodyCudaStatus|void|uint64_t|const char\*)\s+(nb\w+)\s*\(",
                       text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("nbInitCUDA", "nbDestroyCUDA", "nbMarshalBodiesCUDA", "nbGravMapCUDA",
                 "nbStepSystemCUDA", "nbRunStepsCUDA", "nbMakeTreeCUDA", "nbExtAccelerationCUDA"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from milkywayathome_client_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from milkywayathome_client_b200 import _lib
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_struct_layouts():
    from milkywayathome_client_b200 import _lib
    # NBodyCudaCtx: 4 doubles, 6 ints, then the potential (aligned to 8)
    assert _lib.Ctx.pot.offset == 56
    assert ctypes.sizeof(_lib.Spherical) == 24
    assert ctypes.sizeof(_lib.Disk) == 48
    assert ctypes.sizeof(_lib.Halo) == 112
    assert ctypes.sizeof(_lib.Potential) == 24 + 48 + 48 + 112
    assert ctypes.sizeof(_lib.TreeInfo) == 8 + 7 * 4 + 4


# every struct of the C ABI and its ctypes mirror (field names as in C, but for renames)
MIRRORS = [("NBodyCudaSpherical", "Spherical"), ("NBodyCudaDisk", "Disk"), ("NBodyCudaHalo", "Halo"),
           ("NBodyCudaPotential", "Potential"), ("NBodyCudaCtx", "Ctx"),
           ("NBodyCudaTreeInfo", "TreeInfo"), ("NBodyCudaHistogramParams", "HistParams"),
           ("NBodyCudaDataHistogram", "DataHist"), ("NBodyCudaRunParams", "RunParams"),
           ("NBodyCudaRunResult", "RunResult"), ("NBodyCudaPlummerDwarf", "PlummerDwarf"),
           ("NBodyCudaDwarfComponent", "DwarfComponent"), ("NBodyCudaMixedDwarf", "MixedDwarf"),
           ("NBodyCudaDwarf", "Dwarf")]
RENAMED = {"lambda_": "lambda"}


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and every field's offset of each C struct (compiled against the header by the C
    compiler) equal the ctypes mirror's: a field added on one side only fails here."""
    import subprocess
    from milkywayathome_client_b200 import _lib
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nbody_b200.h"', 'int main(void) {']
    want = []
    for cname, pyname in MIRRORS:
        cls = getattr(_lib, pyname)
        lines.append('printf("%%zu\\n", sizeof(%s));' % cname)
        want.append(ctypes.sizeof(cls))
        for f in cls._fields_:
            lines.append('printf("%%zu\\n", offsetof(%s, %s));' % (cname, RENAMED.get(f[0], f[0])))
            want.append(getattr(cls, f[0]).offset)
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == want


def test_library_built_for_sm100a_only():
    """The shared library carries sm_100a code (no other architecture, no PTX fallback)."""
    from milkywayathome_client_b200 import build
    flags = build.ARCH
    assert flags == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_missing_library_fails_loudly(tmp_path):
    from milkywayathome_client_b200 import _lib
    with pytest.raises(FileNotFoundError):
        _lib.load(str(tmp_path / "absent.so"))
