"""The NumPy twin of the model-error generator (oracle/model_error_oracle.py):
properties that pin it without a GPU."""

import numpy as np

from oracle import model_error_oracle as M


def test_philox_is_a_keyed_bijection_of_the_counter():
    g = np.arange(4096, dtype=np.uint64)
    a = M.philox4x32_10(g, 0, 0, 0, 1, 2)
    b = M.philox4x32_10(g, 0, 0, 0, 1, 3)
    words_a = np.stack(a, 1)
    assert len({tuple(r) for r in words_a.tolist()}) == 4096          # distinct outputs
    assert not np.array_equal(words_a, np.stack(b, 1))               # the key matters
    c = M.philox4x32_10(g, 1, 0, 0, 1, 2)
    assert not np.array_equal(words_a, np.stack(c, 1))               # the event word matters
    assert all(int(w.max()) <= 0xFFFFFFFF for w in a)


def test_uniforms_stay_inside_the_open_interval():
    x = np.array([0, 511, 512, 0xFFFFFFFF], dtype=np.uint64)
    u = M.unit_open(x)
    assert np.all(u > 0) and np.all(u < 1)
    assert u[0] == u[1] == 2.0 ** -24


def test_normals_have_unit_moments():
    z = M.normals(np.arange(1 << 18, dtype=np.uint64), 3, 20245, 7)
    assert abs(z.mean()) < 0.01
    assert abs(z.var() - 1.0) < 0.01
    assert abs(np.mean(z ** 4) / z.var() ** 2 - 3.0) < 0.05


def test_field_variance_and_gaussian_correlation():
    f = M.field(384, 320, 20245, 4, 2, 15.0)
    assert abs(f.mean()) < 0.1
    assert abs(f.std() - 1.0) < 0.08
    c = np.mean(f[:, :-15] * f[:, 15:]) / f.var()
    assert abs(c - np.exp(-0.5)) < 0.06
    w, R = M.filter_weights(15.0)
    assert R == 32 and abs(np.sum(w * w) - 1.0) < 1e-12


def test_periodic_rows_wrap():
    f = M.field(64, 48, 1, 2, 3, 6.0, periodic_y=True)
    # a periodic field in y: the gap across the wrap is like any other gap
    d_wrap = np.mean((f[0] - f[-1]) ** 2)
    d_in = np.mean((f[1:] - f[:-1]) ** 2)
    assert d_wrap < 3.0 * d_in
