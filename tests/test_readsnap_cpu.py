"""The snapshot slice tool against the reference's src/readsnap.cpp (no GPU).

Golden slices in tests/golden/readsnap/ were made by the reference's own tool
(compiled unmodified as oracle/_ref/readsnap_ref) from snapshots the
reference wrote (tests/golden/ref16/); the comparison is byte for byte, file
and stdout.  When oracle/_ref/readsnap_ref is present the two tools are also
run side by side on a random snapshot.
"""

import json
import os
import subprocess

import numpy as np
import pytest

from ifdm_code_b200.build import build_readsnap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
REF_TOOL = os.path.join(ROOT, "oracle", "_ref", "readsnap_ref")
CASES = json.load(open(os.path.join(GOLD, "manifest.json")))["readsnap"]["cases"]


@pytest.fixture(scope="module")
def tool():
    return build_readsnap()


def _run(exe, N, z, t, src, out):
    return subprocess.run([exe, str(N), str(z), str(t), src, out], capture_output=True, text=True, check=True).stdout


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["file"])
def test_slice_matches_reference_golden(tool, tmp_path, case):
    stdout = _run(tool, case["N"], case["z"], case["t"], os.path.join(GOLD, case["src"]), str(tmp_path))
    got = (tmp_path / case["file"]).read_bytes()
    want = open(os.path.join(GOLD, "readsnap", case["file"]), "rb").read()
    assert got == want
    stdout = stdout.replace(os.path.join(GOLD, case["src"]) + "/", "<golden>/" + case["src"] + "/")
    stdout = stdout.replace(str(tmp_path) + "/", "<golden>/readsnap/")
    assert stdout == open(os.path.join(GOLD, "readsnap", case["file"] + ".stdout")).read()


def _write_snapshot(path, N, seed):
    rng = np.random.default_rng(seed)
    psi = (rng.standard_normal((N, N, N)) + 1j * rng.standard_normal((N, N, N))) * 1e45
    psi[0, 0, 0] = 0  # arg(0) and a zero density
    psi[1, 2, 3] = -1e44 + 0j  # arg = pi on the branch cut
    x = np.linspace(-4.9, 4.9, N)
    with open(path, "wb") as f:
        np.array([3.1e-24, 7.0e-60, 0.4321], dtype=np.float64).tofile(f)
        x.astype(np.float64).tofile(f)
        psi.astype(np.complex128).tofile(f)


@pytest.mark.skipif(not os.path.exists(REF_TOOL), reason="oracle/_ref/readsnap_ref not built")
@pytest.mark.parametrize("N,z", [(8, 0), (8, 3), (12, 11)])
def test_slice_matches_reference_tool(tool, tmp_path, N, z):
    src, a, b = tmp_path / "snap", tmp_path / "a", tmp_path / "b"
    for d in (src, a, b):
        d.mkdir()
    _write_snapshot(src / "output7.dat", N, seed=N + z)
    so_a = _run(tool, N, z, 7, str(src), str(a))
    so_b = _run(REF_TOOL, N, z, 7, str(src), str(b))
    name = f"output7.dat.z{z}"
    assert (a / name).read_bytes() == (b / name).read_bytes()
    assert so_a.replace(str(a), "") == so_b.replace(str(b), "")


def test_wrong_argument_count(tool):
    r = subprocess.run([tool, "16", "0"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout == "ERROR: Arguments 3!= 5 \n"


def test_missing_snapshot_reports_and_writes_zeros(tool, tmp_path):
    out = _run(tool, 4, 1, 3, str(tmp_path / "nowhere"), str(tmp_path))
    assert out.startswith("ERROR: cant read binary file !!\n")
    lines = (tmp_path / "output3.dat.z1").read_text().splitlines()
    assert len(lines) == 16 and all(l == "0 0 0 0" for l in lines)
