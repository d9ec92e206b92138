"""Host-side pieces of the warm start: the network's input features, the BF16 weight files (round to nearest even,
exact round trip of BF16 values), the training-set workload (deterministic per seed, counts finite for both pupil
kinds, the slit spectrum never empty on small lattices)."""
import numpy as np

from blml_b200 import workloads
from blml_b200.warmstart import features, KINDS, IN_CH
from blml_b200.warmstart_job import to_bf16_bits, from_bf16_bits


def test_features_layout():
    rng = np.random.default_rng(0)
    c = [rng.poisson(3.0, (16, 24)).astype(float) for _ in range(2)]
    x = features(c, [0.2, 0.3], ['pball', 'slits'])
    assert x.shape == (2, 16, 24, IN_CH) and x.dtype == np.float32
    assert np.allclose(x[0, ..., 0], np.log1p(c[0]) / 8.0) and np.allclose(x[1, ..., 1], 1.2)
    assert np.all(x[0, ..., 2 + KINDS.index('pball')] == 1) and np.all(x[0, ..., 2 + KINDS.index('slits')] == 0)
    assert np.allclose(x[1, ..., 4], np.log10(c[1].sum()) / 6.0) and np.all(x[..., 5:] == 0)


def test_bf16_bits_round_to_nearest_even():
    a = np.float32([1.0, -2.5, 3.14159e-3, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, 0.0, -0.0])
    back = from_bf16_bits(to_bf16_bits(a))
    assert back[0] == 1.0 and back[1] == -2.5
    assert back[3] == 1.0                       # halfway (1 + 2^-8): ties to the even mantissa
    assert back[4] == np.float32(1.0 + 2.0 ** -7)   # 1 + 3 2^-9 rounds up
    assert np.all(np.abs(back[:3] - a[:3]) <= np.abs(a[:3]) * 2.0 ** -8)
    assert np.array_equal(from_bf16_bits(to_bf16_bits(back)), back)


def test_warm_start_set_is_deterministic_and_finite():
    a = workloads.warm_start_set(6, seed=3, shape=(32, 32))
    b = workloads.warm_start_set(6, seed=3, shape=(32, 32))
    for fa, fb in zip(a, b):
        assert fa['kind'] == fb['kind'] and fa['fc'] == fb['fc'] and np.array_equal(fa['counts'], fb['counts'])
        assert np.all(np.isfinite(fa['counts'])) and fa['counts'].sum() > 0
    for shape in ((32, 32), (64, 384)):
        for fc in (0.1, 0.4):
            assert workloads.two_slit_field(shape, fc=fc, N=1e4, seed=0).sum() > 0
