"""CGFDM parity: the CUDA library against the reference's own CPU build.

Each case is written in the reference's input formats, run through the
reference binary built from its sources (oracle/_ref/cgfdm_ref) and through
the library's C ABI.  The "exact" library build rounds every float operation
as the reference's CPU path does, so its CJM, station traces and final
wavefield must be bit-identical; the "fast" build (FMA contraction) must
agree to the north-star tolerance, 1e-5 relative L2 on seismograms and on
the final wavefield.
"""

import os

import numpy as np
import pytest

import parity_util as pu
import refrun
from cgfdm import Session, cases

TOL_FAST = 1e-5

def _case(mk):
    return lambda d: cases.write_case(mk(), d)


def _terrain_fault(d):
    # the benchmark workload's generators at a small size: raw height map and
    # medium volume (routed into the reference through its oracle hooks),
    # 40x20 finite fault, 400 stations
    from cgfdm import configs

    configs.terrain_fault(d, steps=60, NX=64, NY=60, NZ=40, nPML=6)


CASES = {
    "halfspace": _case(lambda: pu.small_halfspace(steps=48)),
    "gauss_hill": _case(lambda: pu.small_hill(steps=48)),
    "multi_fault": _case(lambda: pu.multi_fault(steps=48)),
    "ricker_point": _case(lambda: pu.ricker_point(steps=48)),
    "double_couple": _case(lambda: pu.double_couple(steps=48)),
    "terrain_fault": _terrain_fault,
}


@pytest.fixture(scope="module")
def ref_runs(tmp_path_factory):
    if not refrun.available("CGFDM"):
        pytest.skip("reference CPU build oracle/_ref/cgfdm_ref not built")
    root = tmp_path_factory.mktemp("cg")
    dirs = {}
    for name, write in CASES.items():
        dirs[name] = str(root / name)
        write(dirs[name])
    refrun.run_many(list(dirs.values()), "CGFDM")
    return {name: (d, refrun.read_outputs(d)) for name, d in dirs.items()}


def _lib(d, flavor, options=None):
    s = Session(d, options=options, flavor=flavor)
    s.run(s.info.NT)
    res = {"stations": s.stations(), "W": s.wavefield(), "CJM": s.cjm(), "PGV": s.pgv(), "info": s.info}
    s.close()
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_exact_bitwise(ref_runs, name):
    d, ref = ref_runs[name]
    lib = _lib(d, "exact")
    assert lib["info"].NT == ref["stations"].shape[1]
    # metric + medium (setup kernels are exact in every build)
    np.testing.assert_array_equal(lib["CJM"], ref["CJM"])
    diff_st = np.abs(lib["stations"] - ref["stations"]).max()
    diff_w = np.abs(lib["W"] - ref["W"]).max()
    assert diff_st == 0.0 and diff_w == 0.0, (
        f"{name}: max |stations diff| {diff_st}, max |W diff| {diff_w}, "
        f"rel L2 stations {pu.rel_l2(lib['stations'], ref['stations']):.3e}, W {pu.rel_l2(lib['W'], ref['W']):.3e}")
    np.testing.assert_array_equal(lib["PGV"], ref["PGV"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_fast_tolerance(ref_runs, name):
    d, ref = ref_runs[name]
    lib = _lib(d, "fast")
    np.testing.assert_array_equal(lib["CJM"], ref["CJM"])
    e_st = pu.rel_l2(lib["stations"][:, :, :3], ref["stations"][:, :, :3])
    e_w = pu.rel_l2(lib["W"], ref["W"])
    assert e_st <= TOL_FAST, f"{name}: seismogram rel L2 {e_st:.3e}"
    assert e_w <= TOL_FAST, f"{name}: wavefield rel L2 {e_w:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_exact_bitwise_ring_pipeline(ref_runs, name):
    """The ring stage pipeline (six full halo planes; the one batches, linked
    parts and FP16 storage use) moves the data differently from the default
    split pipeline and does the same arithmetic: bit-identical too."""
    d, ref = ref_runs[name]
    lib = _lib(d, "exact", '{"stagePipeline": "ring"}')
    np.testing.assert_array_equal(lib["stations"], ref["stations"])
    np.testing.assert_array_equal(lib["W"], ref["W"])
    np.testing.assert_array_equal(lib["PGV"], ref["PGV"])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["terrain_fault", "multi_fault"])
def test_exact_bitwise_tile_heights(ref_runs, name):
    """The split pipeline runs 32 x 8 column tiles by default; 32 x 4 tiles
    (a second compilation of the same kernel) move the data in other boxes
    and do the same arithmetic: bit-identical to the reference as well."""
    d, ref = ref_runs[name]
    lib = _lib(d, "exact", '{"stageTile": 4}')
    np.testing.assert_array_equal(lib["stations"], ref["stations"])
    np.testing.assert_array_equal(lib["W"], ref["W"])
    np.testing.assert_array_equal(lib["PGV"], ref["PGV"])
