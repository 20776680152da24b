"""Histogram files (no GPU): the reference's Orphan data file parses as nbReadHistogram reads
it (the extended 15-column format: counts plus histograms 1..5), a written histogram reads
back unchanged, and the parameter struct carries the reference's likelihood defaults."""
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_orphan_data_file_parses_like_the_reference():
    from milkywayathome_client_b200 import read_histogram
    d = read_histogram(os.path.join(GOLDEN, "orphan_model_histogram_3"))
    assert d.totalNum == 6047 and d.totalSimulated == 10000 and d.nbins == 34
    assert d.massPerParticle == 0.0012 and d.betaDispBins == 0
    assert [c is not None for c in d.components] == [True] * 5 + [False] * 2
    # first row: beta dispersion 0.977160295101465 +- 0.125080520413684, distance 60.5566...
    assert d.components[0][0][0] == 0.977160295101465
    assert d.components[0][1][0] == 0.125080520413684
    assert d.components[4][0][0] == 60.556607458973268
    assert np.all(d.useBin == 1)
    s = d.struct()
    assert s.nBins == 34 and s.compVariable[0][0] == 0.977160295101465
    assert not s.compVariable[5] and not s.compErr[6]


@pytest.mark.parametrize("full", [False, True])
def test_written_histogram_reads_back(tmp_path, full):
    from milkywayathome_client_b200 import (HistogramParams, data_from_counts, read_histogram,
                                            write_histogram)
    params = HistogramParams(lambdaBins=12, usePropMot=full)
    rng = np.random.default_rng(3)
    counts = rng.integers(0, 40, params.nbins)
    comps = rng.standard_normal((7, 2, params.nbins)).round(9)
    data = data_from_counts(params, counts, 1000, 0.5, comps)
    data.betaDispBins = 3
    path = str(tmp_path / "h")
    write_histogram(path, params, data)
    back = read_histogram(path)
    assert back.totalNum == counts.sum() and back.totalSimulated == 1000
    assert back.betaDispBins == 3
    built = 7 if full else 2
    assert [c is not None for c in back.components] == [True] * built + [False] * (7 - built)
    np.testing.assert_allclose(back.variable, data.variable, atol=1e-15)
    for k in range(built):
        np.testing.assert_allclose(back.components[k][0], comps[k, 0], atol=1e-15)
        np.testing.assert_allclose(back.components[k][1], comps[k, 1], atol=1e-15)


def test_parameter_struct_defaults():
    from milkywayathome_client_b200 import HistogramParams
    h = HistogramParams().struct()
    assert (h.useBetaDisp, h.useVelDisp, h.useBetaComp, h.useVlos, h.useDist, h.usePropMot) == \
        (1, 0, 0, 0, 0, 0)
    assert h.iterMax == 6 and h.betaSigma == 2.5 and h.betaCorrect == 1.111
    assert h.NGPdec == 27.4 * math.pi / 180.0 and h.lNCP == 123 * math.pi / 180.0
    assert (h.sunVelx, h.sunVely, h.sunVelz) == (10.3, 229.2, 6.9)


def test_emd_range_is_read_as_the_reference_reads_it(tmp_path):
    """EMDRange lines (nbReadHistogram: sscanf " EMDRange = {%s}", strtok, strtof): float
    values, the first white-space-free token only, and a write/read round trip."""
    import numpy as np
    from milkywayathome_client_b200 import HistogramParams, read_histogram, write_histogram
    src = open(os.path.join(GOLDEN, "orphan_model_histogram_3")).read()
    path = tmp_path / "h"
    path.write_text(src.replace("betaBins = 1\n", "betaBins = 1\nEMDRange = {-40,-10.3,10.3,40}\n"))
    h = read_histogram(str(path))
    assert list(h.emdRange) == [-40.0, float(np.float32(-10.3)), float(np.float32(10.3)), 40.0]
    d = h.struct()
    assert d.nRange == 4 and d.emdRange[1] == float(np.float32(-10.3))
    out = tmp_path / "h2"
    write_histogram(str(out), HistogramParams(lambdaBins=h.nbins), h)
    assert np.array_equal(read_histogram(str(out)).emdRange, h.emdRange)
    path.write_text(src.replace("betaBins = 1\n", "betaBins = 1\nEMDRange = { -40, -10 }\n"))
    assert list(read_histogram(str(path)).emdRange) == [-40.0]     # an odd count: NaN EMD
    assert read_histogram(os.path.join(GOLDEN, "orphan_model_histogram_3")).struct().nRange == 0
