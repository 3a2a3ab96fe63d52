"""The workload generator: the device synthesis of a self-affine gap equals
the host one (same phases, same spectrum) up to FFT rounding (CPU torch)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_device_synthesis_matches_host():
    from aspher_b200.surfaces import self_affine_gap, self_affine_gap_device
    for Ns, kw in ((64, {}), (128, dict(hurst=0.6, rms=0.02, k_lo=12.0, k_hi=0.33 * 128))):
        g = self_affine_gap(Ns, seed=7, **kw)
        gd = self_affine_gap_device(Ns, seed=7, device="cpu", **kw).numpy()
        assert np.max(np.abs(gd - g)) < 1e-12 * np.max(np.abs(g))
