"""Snapshot streaming (needs a B200).

Snapshots are staged on the device, copied to pinned host memory on a copy
stream and written by a writer thread while the steps go on.  Checked here:
the files are the bytes the blocking path writes (whole reference runs), a
queued snapshot holds the state at the time it was queued even though later
steps and other outputs reuse the staging buffer, and write errors reach the
caller.
"""

import os

import numpy as np
import pytest

from ifdm_code_b200 import IfdmError, Simulation
from tests.snapshot_util import read_snapshot

pytestmark = pytest.mark.gpu


def _run_case(m, golden_dir, out, streaming):
    a = m["args"]
    with Simulation(mfdm=float(a[0]), g=float(a[1]), xmax=float(a[2]), res=int(a[3]), t_write=int(a[4]),
                    t_stop=int(a[5]), ti=int(a[6]), opath=out, icpath=os.path.join(golden_dir, m["ic"])) as s:
        s.set_snapshot_streaming(streaming)
        s.load_ic()
        s.run()
        return s.snapshots_written


@pytest.mark.parametrize("case", ["ref16", "ref32"])
def test_streamed_run_writes_the_blocking_runs_bytes(tmp_path, golden_dir, manifest, case):
    m = manifest[case]
    a_dir, b_dir = str(tmp_path / "stream") + "/", str(tmp_path / "block") + "/"
    os.makedirs(a_dir)
    os.makedirs(b_dir)
    n_streamed = _run_case(m, golden_dir, a_dir, True)
    n_blocking = _run_case(m, golden_dir, b_dir, False)
    files = sorted(os.listdir(a_dir))
    assert files == sorted(os.listdir(b_dir))
    snaps = [f for f in files if f.startswith("output")]
    assert n_streamed == len(snaps) and n_blocking == 0 and len(snaps) >= 3
    for f in files:
        assert open(a_dir + f, "rb").read() == open(b_dir + f, "rb").read(), f


def test_queued_snapshot_holds_the_state_at_queue_time(tmp_path, golden_dir, manifest):
    m = manifest["ref32"]
    out = str(tmp_path) + "/"
    with Simulation(2.5e-24, 0.0, 5.0, 32, opath=out, icpath=os.path.join(golden_dir, m["ic"])) as s:
        s.load_ic()
        s.step(3, 0.05)
        psi0, a0 = s.get_psi(), s.state()["a"]
        s.write_snapshot_async(7)
        s.step(20, 0.05)   # psi moves on while the file is copied and written
        s.get_phi()         # reuses the device staging buffer
        psi1 = s.get_psi()  # and again
        s.write_snapshot_async(8)
        s.flush_snapshots()
        assert s.snapshots_written == 2
    hdr, _, psi = read_snapshot(out + "output7.dat", 32)
    assert hdr["a"] == a0 and np.array_equal(psi, psi0)
    assert not np.array_equal(psi0, psi1)
    _, _, psi = read_snapshot(out + "output8.dat", 32)
    assert np.array_equal(psi, psi1)


def test_write_error_reaches_the_caller(tmp_path, golden_dir, manifest):
    # a directory where the file should go: fopen fails for every user
    m = manifest["ref16"]
    out = str(tmp_path) + "/"
    with Simulation(2.5e-24, 0.0, 5.0, 16, t_write=1, t_stop=3, opath=out,
                    icpath=os.path.join(golden_dir, m["ic"])) as s:
        s.load_ic()
        os.mkdir(out + "output5.dat")
        s.write_snapshot_async(5)  # queued: the error comes with the flush
        with pytest.raises(IfdmError, match="IFDM_ERR_IO"):
            s.flush_snapshots()
        s.write_snapshot(6)  # reported once; the context writes again
        assert os.path.getsize(out + "output6.dat") == (3 + 16 + 2 * 16**3) * 8
        os.mkdir(out + "output1.dat")  # the run's first snapshot
        with pytest.raises(IfdmError, match="IFDM_ERR_IO"):
            s.run()
