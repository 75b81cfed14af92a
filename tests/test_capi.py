"""C-ABI boundary on CPU: the library loads, exports every function that
include/yg.h declares, and the factory (VisGridderFactory::make) validates the
parset keys the way the reference does (no GPU needed for these paths)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "yg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(yg_[a-z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(ygmod):
    lib = ctypes.CDLL(ygmod.LIBPATH)
    names = _declared()
    assert len(names) > 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(ygmod):
    assert set(_declared()) <= set(ygmod.EXPORTS)


def test_unknown_gridder(ygmod):
    # TableVisGridderTest::testUnknownGridder
    with pytest.raises(ygmod.AskapError) as e:
        ygmod.VisGridderFactory.make({"gridder": "AGridderWithSuchNameShouldDefinitelyBeUnknownToTheSystsem"})
    assert "Unknown gridder" in str(e.value)


def test_missing_gridder_key(ygmod):
    # TableVisGridderTest::testCreateAbstract: no gridder named
    with pytest.raises(ygmod.AskapError):
        ygmod.VisGridderFactory.make({})


@pytest.mark.parametrize("bad,msg", [
    ({"gridder.WProject.nwplanes": 64}, "must be odd"),
    ({"gridder.WProject.cutoff": 1.5}, "less than 1.0"),
    ({"gridder.WProject.cutoff": -0.1}, "positive"),
    ({"gridder.WProject.offsetsupport": True}, "variablesupport"),
    ({"gridder.WProject.wsampling": "cubic"}, "not implemented"),
    ({"gridder.WProject.wsampling": "gaussian", "gridder.WProject.wsampling.nwplanes50": 60}, "nwplanes"),
    ({"gridder.WProject.oversample": 0}, "Oversampling"),
])
def test_wproject_parset_checks(ygmod, bad, msg):
    ps = {"gridder": "WProject"}
    ps.update(bad)
    with pytest.raises(ygmod.AskapError) as e:
        ygmod.VisGridderFactory.make(ps)
    assert msg in str(e.value)


def test_parsets_accepted(ygmod):
    for ps in [{"gridder": "SphFunc", "gridder.SphFunc.support": 3, "gridder.SphFunc.oversample": 128},
               {"gridder": "WStack", "gridder.WStack.wmax": 10000, "gridder.WStack.nwplanes": 9},
               {"gridder": "WProject", "gridder.WProject.wsampling": "powerlaw",
                "gridder.WProject.wsampling.exponent": 0.5},
               {"gridder": "AWProject", "gridder.AWProject.diameter": "12m", "gridder.AWProject.blockage": "1m",
                "gridder.AWProject.freqtolerance": "infinite"},
               {"Cimager.gridder": "WProject", "Cimager.gridder.WProject.wmax": 8000, "visweights": "MFS"}]:
        g = ygmod.VisGridderFactory.make(ps)
        g.clone()


def test_aw_needs_disk_keys(ygmod):
    with pytest.raises(ygmod.AskapError):
        ygmod.VisGridderFactory.make({"gridder": "AWProject"})


def test_unsupported_adapters_fail_loudly(ygmod):
    for k in ["gridder.snapshotimaging", "gridder.bwsmearing", "gridder.parotation"]:
        with pytest.raises(ygmod.AskapError):
            ygmod.VisGridderFactory.make({"gridder": "WProject", k: True})
