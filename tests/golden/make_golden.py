#!/usr/bin/env python3
"""Generate the golden fixtures of tests/golden/ from the reference tree (run once, here).

  * golden_likelihoods.json -- the reference's own golden end-to-end likelihoods
    (nbody/tests/RunTestUnits.lua refResults) of the single-Plummer Orphan models that
    tests/golden/orphan_dwarf.lua restates (MODELS below: every model whose components this
    build and the reference build here both evaluate -- models 1, 2, 3 and 7 need the
    exponential disks' Bessel source, which the reference tree lacks);
  * orphan_model_histogram_3 -- the data histogram those tests match against
    (nbody/tests/orphan_models/orphan_model_histogram_3), copied verbatim (data).

Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


# variant of tests/golden/orphan_dwarf.lua -> the reference model it restates
MODELS = {"4": "model_4", "5": "model_5", "5b": "model_5_bounds_test", "6": "model_6",
          "8": "model_8", "9": "model_9", "ninkovic": "model_ninkovic",
          "triaxial": "model_triaxial", "newhist1": "model_newhist1",
          "newhist2": "model_newhist2", "newhist3": "model_newhist3", "bar": "model_bar",
          "LMC": "model_LMC", "LMC_bar": "model_LMC_bar"}


def parse_results(text, model):
    start = text.index('["%s"]' % model)
    nxt = text.find('\n   ["', start + 1)         # the next model's entry, or the table's end
    block = text[start:nxt if nxt >= 0 else len(text)]
    out = {}
    for nb, body in re.findall(r'\["(\d+)"\]\s*=\s*\{(.*?)\}', block, flags=re.S):
        out[nb] = {seed: float(v) for seed, v in re.findall(r'\["(\d+)"\]\s*=\s*([0-9.eE+-]+)', body)}
    return out


def main():
    # the reference checkout: the first argument, MILKYWAY_REFERENCE_SRC, or `reference` beside
    # this repository
    repo = os.path.dirname(os.path.dirname(HERE))
    ref = (sys.argv[1] if len(sys.argv) > 1 else
           os.environ.get("MILKYWAY_REFERENCE_SRC") or os.path.join(os.path.dirname(repo), "reference"))
    tests = os.path.join(ref, "nbody", "tests")
    text = open(os.path.join(tests, "RunTestUnits.lua")).read()
    golden = {
        "source": "nbody/tests/RunTestUnits.lua (refResults), tolerance 1e-10",
        "tolerance": 1e-10,
        "models": {variant: parse_results(text, model) for variant, model in MODELS.items()},
    }
    with open(os.path.join(HERE, "golden_likelihoods.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    shutil.copyfile(os.path.join(tests, "orphan_models", "orphan_model_histogram_3"),
                    os.path.join(HERE, "orphan_model_histogram_3"))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
