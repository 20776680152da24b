"""The reference executable stepping on the GPU through the binding a maintainer adds.

oracle/_ref/milkyway_nbody_cuda (oracle/ref.mk target `cuda`) is the reference's own
executable with milkywayathome_client_b200/reference_binding/nbody_cuda.c compiled in and the
dispatches of nbody_cuda.h added to its nbody.c, nbody_plain.c and nbody_types.c
(oracle/apply_cuda_binding.py), linked against libnbody_b200.so.  With NBODY_CUDA_DEVICE=0 its
run loop (nbRunSystemPlain, nbody/src/nbody_plain.c:366-461) takes every force evaluation and
step on the GPU through the C ABI, marshalling the bodies out (nbMarshalBodiesCUDA) for the
best-likelihood histograms and at the end; the Lua set-up, the histogram, the likelihood and
the output are the reference's own host code.  Its <search_likelihood> must equal the golden
values of the reference's RunTestUnits.lua to 1e-10, as the unmodified executable's do --
including model_bar, whose best-likelihood window and two calibration runs restart the GPU
state from the initial bodies, and model_LMC, whose LMC moves on the GPU.
"""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "milkyway_nbody_cuda")

CASES = [("4", "100", "430281807"), ("5", "100", "543966758"), ("5", "1024", "430281807"),
         ("bar", "100", "430281807"), ("LMC", "100", "543966758")]


def _golden():
    with open(os.path.join(GOLDEN, "golden_likelihoods.json")) as f:
        return json.load(f)


def _run(tmp_path, nbody, seed, variant, device):
    env = dict(os.environ)
    env.pop("NBODY_CUDA_DEVICE", None)
    if device is not None:
        env["NBODY_CUDA_DEVICE"] = str(device)
    out = subprocess.run(
        [EXE, "--checkpoint-interval=-1", "-g", "-f", os.path.join(GOLDEN, "orphan_dwarf.lua"),
         "-h", os.path.join(GOLDEN, "orphan_model_histogram_3"), "--seed", seed,
         "--ignore-checkpoint", nbody, variant], capture_output=True, text=True, timeout=900,
        cwd=str(tmp_path), env=env)
    text = out.stderr + out.stdout
    lines = [l for l in text.splitlines() if l.startswith("<search_likelihood>")]
    assert lines, text[-2000:]
    return -float(lines[0].split(">")[1].split("<")[0]), text


@pytest.mark.parametrize("variant,nbody,seed", CASES)
def test_reference_executable_on_the_gpu_reproduces_the_golden(tmp_path, variant, nbody, seed):
    if not os.path.exists(EXE):
        pytest.skip("reference executable with the binding (oracle/ref.mk cuda) not built")
    got, text = _run(tmp_path, nbody, seed, variant, 0)
    assert "Stepping on CUDA device 0" in text              # the GPU path ran
    want = _golden()["models"][variant][nbody][seed]
    assert abs(got - want) < 1e-10, (got, want)
