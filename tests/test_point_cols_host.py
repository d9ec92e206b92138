"""The host encoding of a mode's kernel for the point kernel (blml_b200.binned.point_cols, include/blml_b200.h
blml_point_col): one-column units, ball groups (the group's first column carries prod fc, D and the unit ball's
volume p(0), blml_trivial.py:135-143), and the kinds it does not take."""
import math

import numpy as np
import pytest


def _cols(modes, d):
    from blml_b200.spec import parse_modes
    from blml_b200.binned import point_cols
    specs, _ = parse_modes(modes, d)
    c = point_cols(specs[0], d)
    return [(x.kind, x.M, x.Mi, x.f, x.fi, x.P) for x in c]


def test_ball_group_and_sinc():
    from blml_b200 import _lib
    from blml_b200.spec import make_modes
    c = _cols(make_modes([0.4, 0.3, 0.4], ['ball', 'sinc', 'ball']), 3)
    assert c[0] == (_lib.PT_BALL, 0b101, 2, 0.4, pytest.approx(0.16), pytest.approx(math.pi / 4))
    assert c[2][:2] == (_lib.PT_BALL, 0b101) and c[2][4] == 0.0
    assert c[1][0] == _lib.PT_SINC and c[1][3] == 0.3


def test_ball_volume_in_three_dims():
    from blml_b200.spec import make_modes
    c = _cols(make_modes([0.45] * 3, ['ball'] * 3), 3)
    # p(0) = pi^(3/2) (1/2)^3 / Gamma(5/2): the volume of the ball of radius 1/2
    assert c[0][5] == pytest.approx(4.0 / 3.0 * math.pi * 0.125)
    assert c[0][4] == pytest.approx(0.45 ** 3) and c[0][2] == 3


def test_pball_is_not_a_point_column():
    from blml_b200.workloads import pball_modes
    with pytest.raises(NotImplementedError):
        _cols(pball_modes((16, 16), 0.3), 2)
