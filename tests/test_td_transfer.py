"""The transfer-function post-processing of TdSession.transfer_function
(session.rs:1238-1261) on the host: the one-sided forward spectra of drive and
response, H = R / G inside the pulse band (|G| above 1e-2 of its peak) and
zero outside, frequencies k / (n dt); and the TdTransfer return type
(problem/td.py:140-167)."""
import numpy as np
import pytest

from rapidfem_b200 import td as T


def _dft(x):
    n = x.size
    k = np.arange(n // 2 + 1)[:, None]
    j = np.arange(n)[None, :]
    return (x[None, :] * np.exp(-2j * np.pi * k * j / n)).sum(axis=1)


def test_transfer_matches_a_direct_dft():
    rng = np.random.default_rng(3)
    for n in (1, 2, 7, 64, 201):
        g = rng.normal(size=n)
        r = rng.normal(size=n)
        f, h = T.transfer(g, r, 0.125)
        sg, sr = _dft(g), _dft(r)
        assert f.shape == h.shape == (n // 2 + 1,)
        assert np.allclose(f, np.arange(n // 2 + 1) / (n * 0.125))
        band = np.abs(sg) > 1e-2 * np.abs(sg).max()
        assert np.allclose(h[band], sr[band] / sg[band], rtol=1e-10, atol=0)
        assert np.all(h[~band] == 0)


def test_transfer_of_a_one_sample_delay():
    """A response that is the drive one sample later (the pulse ends near zero,
    so the circular shift is the delay): H = exp(-2 pi i f dt) in the band,
    zero outside it."""
    n, dt = 256, 0.05
    t = np.arange(n) * dt
    g = np.exp(-(((t - 3.0) / 0.4) ** 2)) * np.cos(2 * np.pi * 1.5 * (t - 3.0))
    r = np.roll(g, 1)
    f, h = T.transfer(g, r, dt)
    sg = np.abs(np.fft.rfft(g))
    band = sg > T.TRANSFER_BAND_FRACTION * sg.max()
    assert 5 < band.sum() < f.size
    assert np.allclose(h[band], np.exp(-2j * np.pi * f[band] * dt), rtol=0, atol=1e-12)
    assert np.all(h[~band] == 0)


def test_transfer_edge_cases():
    f, h = T.transfer([], [], 0.1)
    assert f.size == 0 and h.size == 0 and h.dtype == np.complex128
    with pytest.raises(ValueError, match="lengths differ"):
        T.transfer([1.0, 2.0], [1.0], 0.1)
    # an all-zero drive has no band: H is zero everywhere
    f, h = T.transfer(np.zeros(8), np.ones(8), 0.1)
    assert np.all(h == 0)


def test_tdtransfer_type():
    tf = T.TdTransfer([0.0, 1.0], [1 + 0j, 0j], source_label="E_z @ (0.3, 0.5, 0.5)", probe_label="p")
    f, h = tf
    assert np.array_equal(f, [0.0, 1.0]) and np.array_equal(h, [1 + 0j, 0j])
    assert repr(tf) == "TdTransfer(n_freq=2)"
    assert T._point_label(((0.3, 0.5, 0.5), "E", "z")) == "E_z @ (0.3, 0.5, 0.5)"
