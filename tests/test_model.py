"""Volume consumer (model.py:18-29, otsu_threshold): the oracle against the reference's
own output, and the host half of the device path (the percentile interpolation from
order statistics) against numpy.percentile; the device passes are in test_model_gpu.py."""
import numpy as np
import pytest

from conftest import golden
from oracle import model as om
from tomography_local_demo_b200 import model as M


def test_oracle_matches_reference_golden():
    d = golden("misc.npz")
    assert om.otsu_threshold(d["otsu_vol"]) == float(d["otsu"])


def _cases():
    rng = np.random.default_rng(0)
    yield rng.gamma(2.0, 0.1, 1000).astype(np.float32)
    yield rng.normal(0, 1, 12345).astype(np.float32)
    yield np.round(rng.normal(0, 3, 5000)).astype(np.float32)          # ties
    yield np.array([3.5], np.float32)
    yield np.array([-1.0, 2.0], np.float32)
    yield np.array([1.0, 1.0, 1.0], np.float32)
    yield (rng.uniform(-1, 1, 777) * 1e30).astype(np.float32)
    yield np.concatenate([np.full(10, 2.0), rng.uniform(0, 1, 3)]).astype(np.float32)
    for n in (2, 3, 4, 7, 1001, 2000, 2001, 10 ** 5 + 3):
        yield rng.lognormal(0, 2, n).astype(np.float32)


@pytest.mark.parametrize("q", [(0.1, 99.95), (0.0, 100.0), (50.0,), (12.5, 37.5, 99.0)])
def test_percentile_from_order_statistics_equals_numpy(q):
    for v in _cases():
        s = np.sort(v)
        got = M.percentile_linear(len(v), q, lambda r: s[np.asarray(r)])
        want = np.percentile(v, list(q))
        np.testing.assert_array_equal(got, want)
        assert got.dtype == want.dtype


def test_percentile_of_nothing_raises_like_numpy():
    with pytest.raises(IndexError):
        M.percentile_linear(0, (0.1, 99.95), lambda r: r)
    with pytest.raises(IndexError):
        np.percentile(np.zeros(0, np.float32), [0.1, 99.95])
