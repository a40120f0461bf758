"""High-harmonic (HHG) spectrum of the current, as the reference post-processes it.

The reference's Postproces/HHG.py reads the velocity trace (Velocity.txt: the
complex Tr(rho v) per axis, Postproces/custom_functions/read.py:17-20), Fourier
transforms it with custom_functions/fouriertransform.py:7-35 -- the trace times
the window exp(-t smearing), inverse FFT zero-padded to a 1 meV frequency
grid, sign flipped, fftshift-ed -- with a smearing of 1 eV, and plots the norm
over the three axes, |J(w)|.  `spectrum` restates those steps; `rel_err`
compares two spectra the way the precision forms are judged here: the relative
L2 difference of |J(w)| over 0 <= w <= `harmonics` times the photon energy.
"""
from __future__ import annotations

import numpy as np
from scipy import constants

_AU_TIME_S = constants.physical_constants["atomic unit of time"][0]
_EV_HZ = constants.physical_constants["electron volt-hertz relationship"][0]
_EV_HARTREE = constants.physical_constants["electron volt-hartree relationship"][0]


def fourier_transform(t_au: np.ndarray, J: np.ndarray, smearing_eV: float = 1.0):
    """fouriertransform.py:7-35: J has shape [3][T] (or [T]); returns
    (freq_eV, J(w) [3][n]) on the fftshift-ed grid of 1 meV resolution."""
    t_au = np.asarray(t_au, dtype=np.float64)
    J = np.atleast_2d(np.asarray(J))
    dt_s = (t_au[1] - t_au[0]) * _AU_TIME_S
    total_s_wanted = 1.0 / 0.001 / _EV_HZ
    n = int(total_s_wanted / dt_s)
    window = np.exp(-t_au * (smearing_eV * _EV_HARTREE))
    Jw = -np.array([np.fft.fftshift(np.fft.ifft(window * J[ix], n=n)) for ix in range(J.shape[0])])
    freq_eV = np.fft.fftshift(np.fft.fftfreq(n, d=dt_s)) / _EV_HZ
    return freq_eV, Jw


def spectrum(t_au: np.ndarray, J: np.ndarray, smearing_eV: float = 1.0):
    """HHG.py: |J(w)|, the norm over the axes of the transformed trace."""
    f, Jw = fourier_transform(t_au, J, smearing_eV)
    return f, np.linalg.norm(Jw, axis=0)


def rel_err(t_au: np.ndarray, J_ref: np.ndarray, J: np.ndarray, photon_eV: float, harmonics: float = 30.0,
            smearing_eV: float = 1.0) -> float:
    """Relative L2 difference of |J(w)| against the reference trace's over
    0 <= w <= harmonics * photon energy."""
    f, s_ref = spectrum(t_au, J_ref, smearing_eV)
    _, s = spectrum(t_au, J, smearing_eV)
    band = (f >= 0.0) & (f <= harmonics * photon_eV)
    den = float(np.linalg.norm(s_ref[band]))
    return float(np.linalg.norm(s[band] - s_ref[band]) / den) if den > 0 else float("nan")
