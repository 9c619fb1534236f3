"""The physical constants every implementation here uses are the upstream's
rounded SI values, pinned as the upstream's own known-answer test pins them
(test/unit/constantTest.cpp:3-32): PI, EPSILON0, EL_MASS, EL_CHARGE,
LIGHT_SPEED, MAGN_CONST.  Checked in the CUDA sources, the oracle's C
restatement, the C++ class layer, and the Python workload and diagnostic
modules."""
import os
import re

from oracle import diagnostics
from pdp3_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
UPSTREAM = {"PI": 3.1415926535897932, "EPSILON0": 8.85e-12, "EL_MASS": 9.1e-31,
            "EL_CHARGE": 1.6e-19, "LIGHT_SPEED": 3.0e8, "MAGN_CONST": 1.26e-6}


def defined(path, pattern):
    text = open(os.path.join(ROOT, path)).read()
    return {m.group(1): float(m.group(2)) for m in re.finditer(pattern, text)}


def test_cuda_constants():
    got = defined("pdp3_b200/csrc/pdp3g_internal.cuh",
                  r"constexpr double (\w+) = ([-+0-9.eE]+);")
    for name, value in UPSTREAM.items():
        assert got[name] == value, name
    assert got["LIGHT_SPEED_POW_2"] == UPSTREAM["LIGHT_SPEED"] ** 2


def test_oracle_constants():
    got = defined("oracle/pic_oracle.c", r"#define (\w+) ([-+0-9.eE]+)\s")
    for name, value in UPSTREAM.items():
        assert got[name] == value, name


def test_host_layer_constants():
    got = defined("pdp3_b200/host/pdp3_classes.cpp", r"constexpr double (\w+) = ([-+0-9.eE]+);")
    for name in ("EL_CHARGE", "EL_MASS", "PI"):
        assert got[name] == UPSTREAM[name], name


def test_python_constants():
    assert W.EL_CHARGE == UPSTREAM["EL_CHARGE"]
    assert W.EL_MASS == UPSTREAM["EL_MASS"]
    assert W.LIGHT_SPEED == UPSTREAM["LIGHT_SPEED"]
    assert diagnostics.LIGHT_SPEED == UPSTREAM["LIGHT_SPEED"]
    assert diagnostics.PI == UPSTREAM["PI"]
    assert diagnostics.EL_MASS == UPSTREAM["EL_MASS"]
