"""The arc cosine's polynomial (fn_detmath.h) is reproducible: the committed
fitting script regenerates every coefficient of the header bit for bit."""
import os
import re

import pytest

from conftest import ROOT


def header_coefficients():
    text = open(os.path.join(ROOT, "fibrenet_b200", "csrc", "fn_detmath.h")).read()
    body = re.search(r"const double c\[14\] = \{(.*?)\};", text, re.S).group(1)
    return [float(x) for x in body.replace("\n", " ").split(",")]


def test_fit_regenerates_header_coefficients():
    pytest.importorskip("mpmath")
    import detmath_fit
    got = detmath_fit.coefficients()
    want = header_coefficients()
    assert len(want) == 14
    assert got == want
