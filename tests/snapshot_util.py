"""Helpers to read and compare the reference's snapshot files (src/write3D.h:7-97)."""

from __future__ import annotations

import os

import numpy as np


def read_snapshot(path: str, N: int):
    raw = np.fromfile(path, dtype=np.float64)
    if raw.size != 3 + N + 2 * N**3:
        raise ValueError(f"{path}: {raw.size} doubles, expected {3 + N + 2 * N ** 3}")
    hdr = dict(mfdm=raw[0], g=raw[1], a=raw[2])
    x = raw[3:3 + N]
    psi = raw[3 + N:].view(np.complex128).reshape(N, N, N)
    return hdr, x, psi


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def compare_dirs(got_dir: str, ref_dir: str, files, N: int, psi_tol: float, a_tol: float = 1e-12):
    """Every reference snapshot must exist in got_dir with the same header and
    psi within psi_tol relative L2.  Returns the worst psi error."""
    worst = 0.0
    for f in files:
        if not f.startswith("output"):
            continue
        gp = os.path.join(got_dir, f)
        assert os.path.exists(gp), f"missing {f}"
        h1, x1, p1 = read_snapshot(gp, N)
        h0, x0, p0 = read_snapshot(os.path.join(ref_dir, f), N)
        assert h1["mfdm"] == h0["mfdm"] and h1["g"] == h0["g"], f
        assert abs(h1["a"] - h0["a"]) <= a_tol * abs(h0["a"]), (f, h1["a"], h0["a"])
        assert np.array_equal(x1, x0), f
        e = rel_l2(p1, p0)
        assert e <= psi_tol, (f, e)
        worst = max(worst, e)
    extra = sorted(set(f for f in os.listdir(got_dir) if f.endswith(".dat")) - set(files))
    assert not extra, f"unexpected files {extra}"
    return worst
