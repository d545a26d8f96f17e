"""NSCF occupations (abacus-develop_b200/nscf.py) against the reference's own occupation code compiled from
module_elecstate/occupy.cpp (oracle/_ref; skipped where it was not built): smeared weights, Fermi energy and
band-energy correction for every smearing method the reference accepts, and the fixed-occupation rule."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import ref_david

need_ref = pytest.mark.skipif(not ref_david.available(), reason="oracle/_ref/libref_david.so not built")


def _bands(seed=4, nks=4, nband=10):
    rng = np.random.default_rng(seed)
    ekb = np.sort(rng.uniform(-0.6, 0.9, (nks, nband)), axis=1)
    wk = rng.uniform(0.2, 0.8, nks)
    return ekb, wk * (2.0 / wk.sum())  # weights sum to 2 (spin degeneracy), as K_Vectors' wk for nspin 1


@need_ref
@pytest.mark.parametrize("method,ngauss", [("gaussian", 0), ("mp", 1), ("mp2", 2), ("cold", -1), ("fd", -99)])
@pytest.mark.parametrize("sigma", [0.002, 0.02])
def test_smearing_weights_match_the_reference(pkg, method, ngauss, sigma):
    ekb, wk = _bands()
    nelec = 11.0  # partly filled bands: a metal
    wg, ef, demet = pkg.nscf.smearing_weights(ekb, wk, nelec, sigma, method)
    wg_r, ef_r, demet_r = ref_david.gweights(ekb, wk, nelec, sigma, ngauss)
    assert abs(ef - ef_r) <= 1e-14 and abs(demet - demet_r) <= 1e-14
    assert np.max(np.abs(wg - wg_r)) <= 1e-14
    assert abs(wg.sum() - nelec) < 1e-8 or ngauss > 0  # MP weights may leave [0, 1], the count still holds
    assert abs(pkg.nscf._sumkg(ekb, wk, sigma, ngauss, ef) - nelec) < 1e-9


def test_smearing_decision_and_fixed_rule(pkg):
    N = pkg.nscf
    assert [N.smearing_type(m) for m in ("gauss", "methfessel-paxton", "mp2", "marzari-vanderbilt", "fermi-dirac")] \
        == [0, 1, 2, -1, -99]
    with pytest.raises(ValueError):
        N.smearing_type("mp3")
    with pytest.raises(ValueError):
        N.smearing_weights(np.zeros((1, 2)), [2.0], 2.0, 0.0)
    ekb, wk = _bands()
    wg, ef = N.occupation_weights(ekb, wk, 8.0)
    assert np.all(wg[:, :4] == wk[:, None]) and np.all(wg[:, 4:] == 0.0) and ef == ekb[:, 3].max()
    with pytest.raises(ValueError, match="not a semiconductor"):
        N.occupation_weights(ekb, wk, 9.0)
