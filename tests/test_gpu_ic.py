"""Gadget IC loading at sizes where the chunk files stream in several pieces,
and the loader's file errors (needs a B200).

The loader reads the four chunk files side by side, each in 32 MiB pieces
through pinned buffers, and copies the pieces straight to their particle slots
on the device (ghost copies and the zero particle of one reference rank
included).  At 256^3 every position and velocity block is 50 MB, so each
block crosses piece boundaries; the result must equal the oracle's IC (the
reference's arithmetic): voutput.dat bit for bit, psi to the FP64 bar.
"""

import os

import numpy as np
import pytest

from ifdm_code_b200 import IfdmError, Simulation
from ifdm_code_b200.synthetic_ic import make_ic
from oracle import IC_EXACT, Oracle, OracleArgs
from tests.snapshot_util import rel_l2

pytestmark = pytest.mark.gpu

PSI_TOL = 1e-10


@pytest.fixture(scope="module")
def ic256(tmp_path_factory):
    d = tmp_path_factory.mktemp("ic256")
    make_ic(str(d / "ic"), 256, seed=9)
    return str(d / "ic")


@pytest.mark.parametrize("exact", [False, True])
def test_ic_256_streamed_in_pieces_matches_oracle(ic256, tmp_path, exact):
    od, gd = tmp_path / "oracle", tmp_path / "gpu"
    od.mkdir()
    gd.mkdir()
    o = Oracle(OracleArgs(res=256, opath=str(od) + "/", icpath=ic256, ic_mode=IC_EXACT if exact else 0))
    o.load_ic()
    want = o.psi()
    o.close()
    with Simulation(2.5e-24, 0.0, 5.0, 256, opath=str(gd) + "/", icpath=ic256,
                    ic_mode="exact" if exact else "ref1") as s:
        s.load_ic()
        got = s.get_psi()
    assert rel_l2(got, want) <= PSI_TOL
    assert (gd / "voutput.dat").read_bytes() == (od / "voutput.dat").read_bytes()


def test_ic_file_errors(tmp_path, golden_dir):
    src = os.path.join(golden_dir, "ic16_s1")
    # chunk 2 missing: the first three pass their checks, then the read fails
    d = tmp_path / "missing"
    d.mkdir()
    for c in (0, 1, 3):
        (d / f"ic.{c}").write_bytes(open(f"{src}.{c}", "rb").read())
    with Simulation(2.5e-24, 0.0, 5.0, 16, opath=str(tmp_path) + "/", icpath=str(d / "ic")) as s:
        with pytest.raises(IfdmError, match=r"IO.*ic\.2"):
            s.load_ic()
    # chunk 1 cut inside its velocity block
    d = tmp_path / "trunc"
    d.mkdir()
    for c in range(4):
        raw = open(f"{src}.{c}", "rb").read()
        if c == 1:
            n = int(np.frombuffer(raw[8:12], dtype="<i4")[0])  # npart[1] of the io_header
            raw = raw[:4 + 256 + 4 + 4 + 12 * n + 8 + 6 * n]
        (d / f"ic.{c}").write_bytes(raw)
    with Simulation(2.5e-24, 0.0, 5.0, 16, opath=str(tmp_path) + "/", icpath=str(d / "ic")) as s:
        with pytest.raises(IfdmError, match="truncated Gadget blocks"):
            s.load_ic()
