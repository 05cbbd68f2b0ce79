"""The CPU oracle, pinned against the reference's own code (CPU only).

The golden files were written by oracle/_ref/BECMPI_ref -- the reference's
unmodified sources compiled against single-rank MPI/FFTW/GSL shims -- from the
committed synthetic ICs (tests/golden/make_golden.py).  The restatement in
oracle/ifdm_oracle.c must reproduce them byte for byte.
"""

import os

import numpy as np
import pytest

from oracle import IC_EXACT, Oracle, OracleArgs
from tests.snapshot_util import read_snapshot


def _run_oracle(tmp_path, case, golden_dir, manifest, stan=0):
    m = manifest[case]
    a = m["args"]
    out = str(tmp_path) + "/"
    o = Oracle(OracleArgs(mfdm=float(a[0]), g=float(a[1]), xmax=float(a[2]), res=int(a[3]), t_write=int(a[4]),
                          t_stop=int(a[5]), ti=int(a[6]), opath=out,
                          icpath=os.path.join(golden_dir, m.get("ic", "")), stan=stan))
    o.load_ic()
    o.simulation()
    o.close()
    return out


@pytest.mark.parametrize("case,stan", [("ref16", 0), ("ref16_stan", 1), ("ref16_g", 0), ("ref32", 0)])
def test_oracle_matches_reference_bytes(tmp_path, golden_dir, manifest, case, stan):
    out = _run_oracle(tmp_path, case, golden_dir, manifest, stan)
    for f in manifest[case]["files"]:
        ref = open(os.path.join(golden_dir, case, f), "rb").read()
        got = open(os.path.join(out, f), "rb").read()
        assert got == ref, f"{case}/{f} differs"


def test_oracle_rerun_matches_reference(tmp_path, golden_dir, manifest):
    m = manifest["ref16_rerun"]
    a = m["args"]
    out = str(tmp_path) + "/"
    o = Oracle(OracleArgs(mfdm=float(a[0]), g=float(a[1]), xmax=float(a[2]), res=int(a[3]), t_write=int(a[4]),
                          t_stop=int(a[5]), ti=int(a[6]), opath=out,
                          icpath=os.path.join(golden_dir, "ref16") + "/", rerun=1))
    o.read_rerun(int(a[6]))
    o.simulation()
    for f in m["files"]:
        assert open(os.path.join(out, f), "rb").read() == open(os.path.join(golden_dir, "ref16_rerun", f),
                                                                 "rb").read(), f


def test_golden_snapshot_layout(golden_dir, manifest):
    """output<t>.dat = f64 mfdm, f64 g, f64 a, f64 x[N], c128 psi[N^3]."""
    hdr, x, psi = read_snapshot(os.path.join(golden_dir, "ref16", "output1.dat"), 16)
    assert hdr["mfdm"] == 2.5e-24 and hdr["g"] == 0.0
    xmax = 5.0 / 0.677
    assert np.allclose(x, xmax / 16 - xmax + np.arange(16) * (2 * xmax / 16), rtol=0, atol=1e-12)
    assert np.all(np.isfinite(psi)) and np.abs(psi).max() > 0


def test_exact_ic_mode_counts_each_particle_once(tmp_path, golden_dir):
    """IC_EXACT deposits the total particle mass once; REF1 adds the doubled
    last half cell and the zero particles at the origin."""
    ic = os.path.join(golden_dir, "ic16_s1")
    tot = {}
    for mode in (0, IC_EXACT):
        o = Oracle(OracleArgs(res=16, opath=str(tmp_path) + "/", icpath=ic, ic_mode=mode))
        o.load_ic()
        # psi = 1.225 sqrt(rho h^2 1e9 / m_solar) e^{i..}: recover the CIC mass
        ms = 2.5e-24 * 1.783e-36 / 1.989e30
        rho = np.abs(o.psi()) ** 2 / 1.225**2 * ms / (0.677**2 * 1e9)
        tot[mode] = rho.sum()
        o.close()
    box = 10000.0
    lg3 = (box / 16) ** 3
    from ifdm_code_b200.synthetic_ic import read_gadget_chunk

    hdr, _, _ = read_gadget_chunk(ic + ".0")
    mass = hdr["mass"][1] * 1e10
    assert tot[IC_EXACT] * lg3 == pytest.approx(16**3 * mass, rel=1e-10)
    assert tot[0] > tot[IC_EXACT]
