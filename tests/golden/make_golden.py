"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run in a container that has the reference tree (it builds oracle/_ref, the
reference sources compiled unmodified against single-rank MPI/FFTW/GSL shims):

    python tests/golden/make_golden.py

Each case runs ``oracle/_ref/BECMPI_ref`` (or ``BECMPI_ref_stan``) with the
reference's 10-argument command line on a seeded synthetic IC and keeps the
snapshot files it writes.  ``manifest.json`` records the command lines.
``readsnap/`` holds the text slices the reference's ``src/readsnap.cpp``
(``oracle/_ref/readsnap_ref``) makes of some of those snapshots;
``python tests/golden/make_golden.py readsnap`` regenerates only them.
"""

from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ifdm_code_b200.synthetic_ic import make_ic  # noqa: E402
from oracle import build, ref_binary  # noqa: E402

MFDM = "2.5e-24"
XMAX = "5"
# g chosen so the self-interaction criterion limits some steps (n = 4)
G_SELF = "1e-62"

CASES = [
    # name, binary (stan?), N, seed, g, t_write, t_stop, keep (None = all)
    ("ref16", False, 16, 1, "0", 5, 400, None),
    ("ref16_stan", True, 16, 1, "0", 5, 400, None),
    ("ref16_g", False, 16, 1, G_SELF, 5, 400, None),
    ("ref32", False, 32, 2, "0", 10, 400, ["output1.dat", "output999994.dat", "output999997.dat"]),
]


def run_case(name, stan, N, seed, g, t_write, t_stop, keep):
    out = os.path.join(HERE, name)
    if os.path.exists(out):
        shutil.rmtree(out)
    os.makedirs(out)
    icdir = os.path.join(HERE, f"ic{N}_s{seed}")
    if not os.path.exists(icdir + ".0"):
        make_ic(icdir, N, seed=seed)
    args = [MFDM, g, XMAX, str(N), str(t_write), str(t_stop), "0", out + "/", icdir, "0"]
    r = subprocess.run([ref_binary(stan)] + args, capture_output=True, text=True, check=True)
    with open(os.path.join(out, "stdout.txt"), "w") as f:
        f.write(r.stdout)
    files = sorted(f for f in os.listdir(out) if f.endswith(".dat"))
    if keep is not None:
        for f in files:
            if f not in keep and f != "voutput.dat":
                os.remove(os.path.join(out, f))
        files = sorted(f for f in os.listdir(out) if f.endswith(".dat"))
    # paths are recorded relative to this folder: the output prefix as <golden>/<case>/
    rec = ["<ic>" if a == icdir else a.replace(HERE + "/", "<golden>/") for a in args]
    return {"binary": os.path.basename(ref_binary(stan)), "args": rec,
            "ic": os.path.basename(icdir), "files": files}


def run_rerun():
    """rerun = 1 from a snapshot of ref16: exercises read_rerun."""
    src = os.path.join(HERE, "ref16")
    out = os.path.join(HERE, "ref16_rerun")
    if os.path.exists(out):
        shutil.rmtree(out)
    os.makedirs(out)
    snaps = sorted(int(f[6:-4]) for f in os.listdir(src) if f.startswith("output") and f[6:-4].isdigit())
    ti = [s for s in snaps if s < 999990][1]
    args = [MFDM, "0", XMAX, "16", "2", str(ti + 6), str(ti), out + "/", src + "/", "1"]
    r = subprocess.run([ref_binary(False)] + args, capture_output=True, text=True, check=True)
    with open(os.path.join(out, "stdout.txt"), "w") as f:
        f.write(r.stdout)
    return {"binary": "BECMPI_ref", "args": [a.replace(HERE + "/", "") for a in args], "ti": ti,
            "files": sorted(f for f in os.listdir(out) if f.endswith(".dat"))}


# readsnap cases: snapshot of ref16 (written by the reference), z slices
READSNAP_CASES = [("ref16", 16, 11, 0), ("ref16", 16, 11, 5), ("ref16", 16, 999997, 15)]


def run_readsnap():
    """The reference's slice tool (oracle/_ref/readsnap_ref) on reference snapshots."""
    tool = os.path.join(ROOT, "oracle", "_ref", "readsnap_ref")
    out = os.path.join(HERE, "readsnap")
    if os.path.exists(out):
        shutil.rmtree(out)
    os.makedirs(out)
    cases = []
    for src, N, t, z in READSNAP_CASES:
        r = subprocess.run([tool, str(N), str(z), str(t), os.path.join(HERE, src), out], capture_output=True,
                           text=True, check=True)
        name = f"output{t}.dat.z{z}"
        with open(os.path.join(out, name + ".stdout"), "w") as f:
            f.write(r.stdout.replace(HERE + "/", "<golden>/"))
        cases.append({"src": src, "N": N, "t": t, "z": z, "file": name})
    return {"binary": "readsnap_ref", "cases": cases}


def main():
    build()
    if ref_binary() is None:
        raise SystemExit("oracle/_ref/BECMPI_ref is not built (reference sources absent)")
    if sys.argv[1:] == ["readsnap"]:
        with open(os.path.join(HERE, "manifest.json")) as f:
            manifest = json.load(f)
        manifest["readsnap"] = run_readsnap()
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(manifest, f, indent=1)
        return
    manifest = {}
    for c in CASES:
        manifest[c[0]] = run_case(*c)
    manifest["ref16_rerun"] = run_rerun()
    manifest["readsnap"] = run_readsnap()
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(json.dumps({k: len(v["files"]) for k, v in manifest.items()}))


if __name__ == "__main__":
    main()
