"""Device power spectrum against numpy (needs a B200).

P(k) of delta = |psi|^2/<|psi|^2> - 1 on the full FFT grid, binned by |kappa|
with the same edges, normalised by L^3/N^6; FP64 arithmetic on both sides,
so agreement to 1e-11 relative per bin.  Mode counts are integers and must
match exactly; repeated calls agree bit for bit.
"""

import numpy as np
import pytest

from ifdm_code_b200 import IfdmError, Simulation
from ifdm_code_b200.synthetic_ic import zeldovich_psi

pytestmark = pytest.mark.gpu

XMAX, MFDM, H = 5.0, 2.5e-24, 0.677


def numpy_pk(psi, edges, L):
    N = psi.shape[0]
    rho = np.abs(psi) ** 2
    mean = rho.mean()
    dk = np.fft.fftn(rho / mean - 1.0)
    p = np.abs(dk) ** 2
    kap = np.fft.fftfreq(N) * N
    kk = np.sqrt(kap[:, None, None] ** 2 + kap[None, :, None] ** 2 + kap[None, None, :] ** 2).ravel()
    nb = len(edges) - 1
    idx = np.digitize(kk, edges) - 1
    ok = (idx >= 0) & (idx < nb)
    cnt = np.bincount(idx[ok], minlength=nb)
    s = np.bincount(idx[ok], weights=p.ravel()[ok], minlength=nb)
    ks = np.bincount(idx[ok], weights=kk[ok], minlength=nb)
    with np.errstate(invalid="ignore", divide="ignore"):
        pk = np.where(cnt > 0, s / cnt * L ** 3 / N ** 6, 0.0)
        k = np.where(cnt > 0, ks / cnt * 2 * np.pi / L, 0.0)
    return k, pk, cnt, mean


@pytest.mark.parametrize("N,nbins,log", [(32, 12, True), (64, 24, True), (48, 10, False)])
def test_power_spectrum_matches_numpy(tmp_path, N, nbins, log):
    psi = zeldovich_psi(N, xmax=XMAX, seed=N, a=1 / 51, mfdm=MFDM)
    L = 2 * XMAX / H
    edges = np.logspace(0, np.log10(N / 2), nbins + 1) if log else np.linspace(0.5, N / 2 + 0.5, nbins + 1)
    with Simulation(MFDM, 0.0, XMAX, N, opath=str(tmp_path) + "/") as s:
        s.set_psi(psi, 1 / 51)
        got = s.power_spectrum(nbins, edges)
        again = s.power_spectrum(nbins, edges)
        dflt = s.power_spectrum(nbins)
    k, pk, cnt, mean = numpy_pk(psi, edges, L)
    np.testing.assert_array_equal(got["modes"], cnt)
    np.testing.assert_allclose(got["pk"], pk, rtol=1e-11, atol=0)
    np.testing.assert_allclose(got["k"], k, rtol=1e-13)
    assert got["mean_rho"] == pytest.approx(mean, rel=1e-13)
    for key in ("k", "pk", "modes"):
        assert np.array_equal(got[key], again[key])
    # default bins: log-spaced from exactly 1 to exactly N/2, so together
    # they hold every mode with 1 <= |kappa| < N/2
    kap = np.fft.fftfreq(N) * N
    kk = np.sqrt(kap[:, None, None] ** 2 + kap[None, :, None] ** 2 + kap[None, None, :] ** 2)
    assert int(dflt["modes"].sum()) == int(((kk >= 1) & (kk < N / 2)).sum())


def test_power_spectrum_after_steps_and_arguments(tmp_path):
    N = 32
    psi = zeldovich_psi(N, xmax=XMAX, seed=3, a=1 / 51, mfdm=MFDM)
    with Simulation(MFDM, 0.0, XMAX, N, opath=str(tmp_path) + "/", precision="fp32") as s:
        with pytest.raises(IfdmError):
            s.power_spectrum(8)  # no psi yet
        s.set_psi(psi, 1 / 51)
        s.step(5, 0.1)
        now = s.get_psi()
        edges = np.geomspace(1.0, N / 2, 9)
        got = s.power_spectrum(8, edges)
        with pytest.raises(IfdmError):
            s.power_spectrum(65)
        with pytest.raises(IfdmError):
            s.power_spectrum(3, np.array([1.0, 3.0, 2.0, 8.0]))
        assert np.array_equal(s.get_psi(), now)  # the state is untouched
    _, pk, cnt, _ = numpy_pk(now, edges, 2 * XMAX / H)
    np.testing.assert_array_equal(got["modes"], cnt)
    np.testing.assert_allclose(got["pk"], pk, rtol=1e-10)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_field_means_match_numpy(tmp_path, prec):
    # grid means for the energy terms against numpy on the state the library
    # reports (get_psi / get_phi): FP64 sums on both sides
    N = 32
    psi0 = zeldovich_psi(N, xmax=XMAX, seed=5, a=1 / 51, mfdm=MFDM)
    with Simulation(MFDM, 0.0, XMAX, N, opath=str(tmp_path) + "/", precision=prec) as s:
        s.set_psi(psi0, 1 / 51)
        s.step(4, 0.1)
        psi, phi = s.get_psi(), s.get_phi()
        got = s.energies()
        again = s.energies()
    rho = np.abs(psi) ** 2
    kap = np.fft.fftfreq(N) * N
    k2 = (kap[:, None, None] ** 2 + kap[None, :, None] ** 2 + kap[None, None, :] ** 2) * (np.pi / (XMAX / H)) ** 2
    want = {"mean_rho": rho.mean(), "mean_rho2": (rho ** 2).mean(), "mean_phi_rho": (phi * rho).mean(),
            "mean_grad2": float((k2 * np.abs(np.fft.fftn(psi)) ** 2).sum()) / N ** 6}
    for k, v in want.items():
        assert got[k] == pytest.approx(v, rel=1e-12), k
    assert got == again
