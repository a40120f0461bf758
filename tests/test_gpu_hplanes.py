"""GPU parity of the Hermitian-plane form (EDUS_PREC_HPLANES).

The form keeps the FP64 form's state, commutators and stage updates and
transforms only the band pairs n <= m; the gradient and Hamiltonian planes of
(m, n) are the conjugates of those of (n, m).  On an odd grid that is the
reference's generator, so the form must match the unmodified oracle at the
FP64 bar; on an even grid it is the generator's Hermitian part, which the
oracle's `hermitian_nyquist` switch computes (as for the packed forms).
"""
import numpy as np
import pytest

from test_gpu_packed import make_packed
from test_gpu_parity import lasers_of, model_input, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("coulomb", [False, True])
def test_hplanes_odd_grid_matches_reference_oracle(pkg, po, tmp_path, coulomb):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "hodd", (7, 9, 1), nb=4, coulomb=coulomb, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HPLANES, hermitian_nyquist=False)
    for chunk in (1, 9):
        s.step(chunk)
        o.step(chunk)
        assert rel(s.get_state(), o.get("rho")) < TOL, chunk


CASES = [
    # name, grid, nb, coulomb, solver, order
    ("h2d", (6, 10, 1), 3, False, "RK", 4),
    ("h2d_hsex", (8, 6, 1), 4, True, "RK", 4),
    ("h_ab4", (10, 9, 1), 4, True, "AB", 4),
    ("h13", (8, 9, 1), 13, True, "RK", 4),           # FP64 tensor-core commutator
    ("h13_odd", (9, 7, 1), 13, True, "RK", 4),
    ("h72", (72, 8, 1), 6, True, "RK", 4),           # radix 8 x 9 axis (specialised plane kernel)
    ("h_bulk_ipa", (72, 64, 1), 3, False, "RK", 4),  # 4608 points: bulk copies in and out
    ("h_bulk_hsex", (72, 64, 1), 3, True, "RK", 4),
]


@pytest.mark.parametrize("name,grid,nb,coulomb,solver,order", CASES)
def test_hplanes_matches_hermitian_oracle(pkg, po, tmp_path, name, grid, nb, coulomb, solver, order):
    E = pkg.edus
    inp = model_input(pkg, tmp_path, name, grid, nb=nb, coulomb=coulomb, solver=solver, order=order, dt=0.01,
                      envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HPLANES)
    for chunk in (1, 3, 8):
        s.step(chunk)
        o.step(chunk)
        assert rel(s.get_state(), o.get("rho")) < TOL, (name, chunk)
    assert abs(s.time - o.time) < 1e-12


def test_hplanes_batch(pkg, po, tmp_path):
    """Solves under different pulses in one launch each match their own run."""
    E = pkg.edus
    inp = model_input(pkg, tmp_path, "hb", (9, 7, 1), nb=4, coulomb=True, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HPLANES, batch=3, hermitian_nyquist=False)
    lasers = lasers_of(pkg, cfg)
    for b in range(3):
        L = lasers[0]
        s.set_lasers([pkg.Laser(L.intensity * (1 + 0.5 * b), L.omega, L.pol, L.cycles, L.t0, L.phase, L.fwhm,
                                L.envelope)] + lasers[1:], b)
    s.step(6)
    for b in range(3):
        cb = po.load_input(inp)
        cb.lasers[0].intensity *= 1 + 0.5 * b
        ob = po.Oracle(cb)
        ob.step(6)
        assert rel(s.get_state(b), ob.get("rho")) < TOL, b


def test_hplanes_refuses_what_it_does_not_cover(pkg, po, tmp_path):
    E = pkg.edus
    with pytest.raises(E.EdusError):
        E.Solver((4, 3, 5), 2, 0.01, precision=E.PREC_HPLANES)  # 3-D grid
    with pytest.raises(E.EdusError):
        E.Solver((120, 120, 1), 2, 0.01, precision=E.PREC_HPLANES)  # plane beyond the persistent kernel
    inp = model_input(pkg, tmp_path, "hr", (8, 6, 1), nb=2, dt=0.01, envelope="gauss")
    cfg, o, s = make_packed(pkg, po, inp, E.PREC_HPLANES)
    with pytest.raises(E.EdusError):
        s.set_peierls(True)
