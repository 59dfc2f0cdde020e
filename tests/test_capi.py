"""CPU tests of the C ABI: the library loads, exports everything the
headers declare, and the host-side logic (weights, validation, footprint)
works without a GPU.  No device computation runs here."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from quest_b200 import capi, inputs as I
from tests.conftest import ROOT


def declared_functions():
    names = set()
    for path in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(qg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_functions()
    assert "qg_create" in names and "qg_run" in names
    for name in names:
        assert hasattr(L, name), name
    assert set(names) <= set(capi.EXPORTS) | set(names)
    for name in capi.EXPORTS:
        assert name in names, f"{name} bound in capi.py but not declared in include/"


def test_pc_weights_match_golden(golden_weights):
    ps, cs, fc = capi.pc_weights(18, 22, 3.15)
    gps, gcs, gfc = golden_weights
    np.testing.assert_array_equal(ps, gps)
    np.testing.assert_array_equal(cs, gcs)
    assert fc == gfc


def test_pc_weights_rejects_bad_sizes():
    with pytest.raises(capi.QuestError) as e:
        capi.pc_weights(18, 40, 3.15)
    assert e.value.code == capi.QG_ERR_INVALID_ARG
    with pytest.raises(capi.QuestError):
        capi.pc_weights(50, 22, 3.15)


@pytest.mark.parametrize("field,value,code", [
    ("n", 0, capi.QG_ERR_INVALID_ARG),
    ("interpolation_order", 0, capi.QG_ERR_INVALID_ARG),
    ("interpolation_order", 9, capi.QG_ERR_INVALID_ARG),
    ("dt", -1.0, capi.QG_ERR_INVALID_ARG),
    ("frame", 7, capi.QG_ERR_INVALID_ARG),
])
def test_create_validates_before_touching_the_device(field, value, code):
    wl = I.plain_small(n=8, steps=10)
    c = wl.constants
    n = wl.n
    if field == "n":
        n = value
    elif hasattr(c, field):
        setattr(c, field, value)
    p = capi.make_params(c)
    h = ctypes.c_void_p()
    rc = capi.lib().qg_create(capi.dots_array(wl.dots), n, ctypes.byref(capi.pulse_struct(wl.pulse)),
                              ctypes.byref(p), None, ctypes.byref(h))
    assert rc == code
    assert capi.lib().qg_last_error().decode()
    assert not h.value


def test_footprint_grows_with_n():
    c = I.Constants()
    a = capi.footprint(1024, c, 0.2)
    b = capi.footprint(4096, c, 0.2)
    assert b > 8 * a
    # the FP64 table dominates: 100 bytes per unordered pair at q = 5
    assert b > 4096 * 4095 // 2 * 100
