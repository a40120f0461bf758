"""The HHG post-processing restated from the reference (CPU)."""
import numpy as np


def test_spectrum_peaks_at_the_carrier(pkg):
    hhg = pkg.hhg
    FS = 41.341373335182113
    t = np.arange(0, 4000) * 0.005 * FS  # 20 fs at 0.005 fs
    w0_eV = 3.0
    w0_au = w0_eV / 27.211386245988
    J = np.stack([np.cos(w0_au * t), 0.5 * np.sin(w0_au * t), np.zeros_like(t)])
    f, s = hhg.spectrum(t, J, smearing_eV=0.2)
    assert abs(f[1] - f[0] - 0.001) < 1e-5  # the 1 meV grid of fouriertransform.py
    pos = f > 0.5
    assert abs(f[pos][np.argmax(s[pos])] - w0_eV) < 0.01


def test_rel_err_scales_with_the_perturbation(pkg):
    hhg = pkg.hhg
    t = np.arange(0, 2000) * 0.2
    rng = np.random.default_rng(0)
    J = np.stack([np.cos(0.05 * t) + 0.1 * np.cos(0.15 * t), np.zeros_like(t), np.zeros_like(t)])
    assert hhg.rel_err(t, J, J, 1.5) == 0.0
    e1 = hhg.rel_err(t, J, J + 1e-6 * rng.normal(size=J.shape), 1.5)
    e2 = hhg.rel_err(t, J, J + 1e-4 * rng.normal(size=J.shape), 1.5)
    assert 0 < e1 < e2 and 30 < e2 / e1 < 300
