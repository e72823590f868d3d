"""The C ABI library: it loads, exports every symbol include/lsfdtd.h declares, and its host-side helpers
agree with the plan code (no GPU needed)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO


def _header_symbols():
    text = open(os.path.join(REPO, "include", "lsfdtd.h")).read()
    return sorted(set(re.findall(r"\b(lsfdtd_[a-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from lightsmith_b200 import _abi, build

    build.build()
    return _abi.lib()


def test_library_exports_every_declared_symbol(lib):
    from lightsmith_b200 import _abi

    declared = _header_symbols()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_abi.SIGNATURES), "ctypes signatures out of step with the header"
    assert lib.lsfdtd_abi_version() == _abi.ABI_VERSION


def test_cpml_slabs_match_plan_terms(lib):
    from lightsmith_b200.plan import PMLSpec, cpml_terms

    shape, per = (20, 17, 23), (False, True, False)
    spec = PMLSpec(cells=((4, 3), (0, 0), (5, 6)))
    want = {}
    for t in cpml_terms(spec, shape, per):
        side = 0 if t["region"][t["d"]][0] < shape[t["d"]] // 2 else 1
        want[(t["field"], t["c"], t["d"], side)] = t["region"][t["d"]]
    shp, pr = (C.c_int32 * 3)(*shape), (C.c_int32 * 3)(*per)
    got = {}
    for d in (0, 2):
        lo, hi = spec.cells[d]
        for f, fld in enumerate("EH"):
            for c in range(3):
                for side in range(2):
                    st, ln = C.c_int32(), C.c_int32()
                    assert lib.lsfdtd_cpml_slab(shp, pr, d, lo, hi, f, c, side, C.byref(st), C.byref(ln)) == 0
                    if ln.value:
                        got[(fld, c, d, side)] = (st.value, st.value + ln.value)
    assert got == want


def test_invalid_arguments_are_reported(lib):
    from lightsmith_b200 import _abi

    st, ln = C.c_int32(), C.c_int32()
    shp = (C.c_int32 * 3)(8, 8, 8)
    assert lib.lsfdtd_cpml_slab(shp, shp, 5, 1, 1, 0, 0, 0, C.byref(st), C.byref(ln)) == _abi.EINVAL
    assert b"out of range" in lib.lsfdtd_last_error()
    g = _abi.GridDesc()
    h = C.c_void_p()
    assert lib.lsfdtd_engine_create(C.byref(g), C.byref(h)) == _abi.EINVAL


def test_group_state_length(lib):
    poles = (C.c_int32 * 4)(3, 2, 0, 0)
    assert lib.lsfdtd_group_state_len(0, 1, poles) == 2 + 2 * 3
    assert lib.lsfdtd_group_state_len(1, 2, poles) == 3 + 2 + 4 * 5


def test_plan_roundtrip(golden):
    from lightsmith_b200 import plan as P

    d = golden("engine_tfsf_table")
    again = P.loads({k: v for k, v in np.load(__import__("io").BytesIO(P.to_bytes(d))).items()})
    assert np.array_equal(again["plan"]["inv_eps"], d["plan"]["inv_eps"])
    assert np.array_equal(again["plan"]["sources"][0].E.node, d["plan"]["sources"][0].E.node)
