"""The oracle reproduces the committed golden vectors (tests/golden/golden.npz, written by
tests/golden/make_golden.py) exactly: a regression pin on the checker itself."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def test_golden_matches_oracle(golden, oracle_lib):
    from tests.golden.make_golden import make
    now = make()
    assert sorted(now) == sorted(golden)
    for k in golden:
        np.testing.assert_array_equal(now[k], golden[k], err_msg=k)


def test_golden_sanity(golden):
    assert golden["hit_prim"].shape == (4096,) and (golden["hit_prim"] >= 0).mean() > 0.2
    assert golden["hit_ties"].max() <= 1
    assert np.all((golden["rng_out"] >= 0) & (golden["rng_out"] < 1))
    assert np.all(golden["box_mean"][..., 3] == 1.0)        # the closed box covers every pixel
    assert np.any(golden["box_grad"][:3, :3] != 0)
    assert set(np.unique(golden["delta_sample_in"][:, 0])) == {2.0, 4.0}
    assert np.all(golden["env_sample_out"][:, 4] > 0)                  # env map pdfs
    assert np.all(golden["glass_mean"][..., 3] == 1.0)
