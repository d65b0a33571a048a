"""The seeded workload generator: deterministic, in range, right mix."""
import numpy as np

import msm_helpers as H
import synth


def test_uniform_below_r_and_deterministic():
    a = synth.uniform_scalars(1, 5000)
    b = synth.uniform_scalars(1, 5000)
    assert (a == b).all()
    assert all(H.to_int(a[i]) < H.R for i in range(0, 5000, 7))
    assert not (a == synth.uniform_scalars(2, 5000)).all()


def test_base_multipliers_nonzero():
    k = synth.base_multipliers(3, 4000)
    assert (k != 0).any(axis=1).all()


def test_skewed_mix():
    n = 10000
    s = synth.skewed_scalars(2, n)
    vals = [H.to_int(s[i]) * pow(2, -256, H.R) % H.R for i in range(n)]
    zero = sum(v == 0 for v in vals)
    one = sum(v == 1 for v in vals)
    small = sum(1 < v < (1 << 16) for v in vals)
    assert abs(zero - 0.4 * n) < 0.01 * n + 60  # the uniform-small class adds a few zeros/ones
    assert abs(one - 0.2 * n) < 0.01 * n + 10
    assert abs(small - 0.2 * n) < 0.01 * n + 10
    # shuffled: no long runs of one category at the start
    assert len(set(vals[:50])) > 10
