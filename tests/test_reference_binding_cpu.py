"""The reference executable with the B200 binding compiled in (oracle/_ref/milkyway_nbody_cuda,
oracle/ref.mk target `cuda`), no GPU: without NBODY_CUDA_DEVICE the dispatches leave the
reference's CPU step in charge and the executable prints the golden likelihood of the
unmodified reference; the patch applies to the reference's sources only at its anchors."""
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)


def test_binding_executable_keeps_the_cpu_step_without_a_device(tmp_path):
    from test_gpu_reference_binding import EXE, _golden, _run
    if not os.path.exists(EXE):
        pytest.skip("reference executable with the binding (oracle/ref.mk cuda) not built")
    got, text = _run(tmp_path, "100", "543966758", "5", None)
    assert "CUDA device" not in text
    assert abs(got - _golden()["models"]["5"]["100"]["543966758"]) < 1e-10


def test_patch_anchors_occur_once(tmp_path):
    """Every dispatch is inserted at text that occurs exactly once in the reference file."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import apply_cuda_binding as acb
    ref = os.environ.get("MILKYWAY_REFERENCE_SRC") or os.path.join(os.path.dirname(ROOT), "reference")
    if not os.path.isdir(os.path.join(ref, "nbody")):
        pytest.skip("reference sources not present")
    acb.main(ref, str(tmp_path))
    for name in acb.EDITS:
        text = open(tmp_path / name).read()
        assert '#include "nbody_cuda.h"' in text
        for _, new in acb.EDITS[name]:
            assert text.count(new) == 1
