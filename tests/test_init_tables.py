"""The velocity sampler's inverse-CDF tables (pdp3_b200/csrc/mj_tables.h) are
what gen_mj_tables.py derives from their definitions: spot entries recomputed
with mpmath equal the committed doubles, and both tables are monotone."""
import os
import re

import numpy as np

from pdp3_b200.csrc import gen_mj_tables as G

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "pdp3_b200", "csrc", "mj_tables.h")


def table(name):
    src = open(HEADER).read()
    i = src.index("{", src.index(name))
    j = src.index("}", i)
    return np.array([float(x) for x in re.findall(r"[-+]?[0-9.]+(?:e[-+]?[0-9]+)?",
                                                 src[i + 1:j])])


def test_tables_match_their_definition():
    f, h = table("LN_INV_F"), table("LN_INV_H")
    assert f.size == h.size == G.N
    mp = G.mp
    for j in (0, 1, 137, 500, 654, 700, 755, 799, 998, 999):
        assert float(G.inv_f(mp.mpf(-19) + j * mp.mpf(21) / 999)) == f[j], j
        y = mp.exp(mp.mpf(-30) + j * mp.mpf(42) / 999)
        assert float(mp.log(G.inv_h(y))) == h[j], j
    # P(3/2, x) falls as ln(-ln U) grows; H^-1 grows with its argument
    assert np.all(np.diff(f) < 0)
    assert np.all(np.diff(h) > 0)
