#!/usr/bin/env python3
"""Generate the golden fixtures of tests/golden/ from the reference tree (run once, here).

  * golden_likelihoods.json -- the reference's own golden end-to-end likelihoods for the
    single-Plummer Orphan models 4 and 5 (nbody/tests/RunTestUnits.lua:105-156) and the
    triaxial-halo (model_triaxial, :313-338) and orbiting-bar (model_bar, :443-468) models, which
    tests/golden/orphan_dwarf.lua restates;
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


def parse_results(text, model):
    start = text.index('["%s"]' % model)
    block = text[start:text.index("\n   },", start)]
    out = {}
    for nb, body in re.findall(r'\["(\d+)"\]\s*=\s*\{(.*?)\}', block, flags=re.S):
        out[nb] = {seed: float(v) for seed, v in re.findall(r'\["(\d+)"\]\s*=\s*([0-9.eE+-]+)', body)}
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    tests = os.path.join(ref, "nbody", "tests")
    text = open(os.path.join(tests, "RunTestUnits.lua")).read()
    golden = {
        "source": "nbody/tests/RunTestUnits.lua (refResults), tolerance 1e-10",
        "tolerance": 1e-10,
        "models": {"4": parse_results(text, "model_4"), "5": parse_results(text, "model_5"),
                   "triaxial": parse_results(text, "model_triaxial"),
                   "bar": parse_results(text, "model_bar")},
    }
    with open(os.path.join(HERE, "golden_likelihoods.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    shutil.copyfile(os.path.join(tests, "orphan_models", "orphan_model_histogram_3"),
                    os.path.join(HERE, "orphan_model_histogram_3"))
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
