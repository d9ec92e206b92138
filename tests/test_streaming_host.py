"""Host logic of the streaming fits against the reference's own helpers (tests/golden/stream_helpers.json, made by
tests/golden/make_stream_helpers_golden.py): the Adam step on log fc and the batch order, bit for bit; the modes
helpers the burn-in selection uses (templates with missing fc, trainability, with_fc)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from blml_b200.streaming import adam_log_step, batch_order
from blml_b200.spec import parse_modes, modes_fc, modes_trainable, with_fc

with open(os.path.join(GOLDEN, 'stream_helpers.json')) as fh:
    GOLD = json.load(fh)


@pytest.mark.parametrize('i', range(6))
def test_adam_matches_reference(i):
    c = GOLD['adam'][i]
    st, v = [0.0, 0.0, 0], c['v0']
    for g, want in zip(c['grads'], c['traj']):
        v = float(adam_log_step(v, g, st, 0.1, (0.9, 0.999)))
        assert v == want


@pytest.mark.parametrize('i', range(3))
def test_batch_order_matches_reference(i):
    c = GOLD['order'][i]
    got = batch_order(c['nb'], c['groups'], np.random.default_rng(c['seed']))
    assert [int(x) for x in got] == c['order']


def test_mode_templates():
    m = [{0: dict(kind='sinc', fc=dict(value=0.3, trainable=False)), 1: dict(kind='sinc')},
         {(0, 1): dict(kind='ball', fc=0.2)}]
    sp = parse_modes(m, 2, need_fc=False)[0]
    assert np.isnan(sp[0]['fc'][1]) and list(sp[0]['fc_trainable']) == [False, True]
    assert list(sp[1]['fc_trainable']) == [True, True]
    F = modes_fc(m)
    assert F.shape == (2, 2) and np.isnan(F[0, 1]) and F[1, 0] == F[1, 1] == 0.2
    assert modes_trainable(m).tolist() == [[False, True], [True, True]]
    filled = with_fc(m, [[0.3, 0.15], [0.25, 0.25]])
    assert filled[0][0]['fc'] == dict(value=0.3, trainable=False) and filled[0][1]['fc'] == 0.15
    assert filled[1][(0, 1)]['fc'] == 0.25
    with pytest.raises(ValueError):
        parse_modes(m, 2)                                    # fc missing outside a template
    with pytest.raises(ValueError):
        parse_modes([{0: dict(kind='sinc', fc=dict(trainable=False))}], 1, need_fc=False)
