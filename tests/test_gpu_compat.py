"""The reference-signature shim (hegjoin_b200/compat) driven by a caller that
only knows the reference's interface (tests/compat/compat_main.cpp)."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from hegjoin_b200 import workloads

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

BUILDS = {"d18": (18, 6, "float"), "d2": (2, 2, "double")}


def _exe(cfg):
    d, k, t = BUILDS[cfg]
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "compat"), f"CFG={cfg}", f"D={d}", f"K={k}",
                    f"T={t}"], check=True)
    return os.path.join(ROOT, "_build", "compat", cfg, "compat_main")


@pytest.mark.parametrize("text", [False, True])
@pytest.mark.parametrize("cfg,n,seed,eps", [("d18", 6000, 61, 0.07), ("d2", 8000, 62, 0.006)])
def test_reference_signatures_end_to_end(cuda, tmp_path, cfg, n, seed, eps, text):
    d, k, t = BUILDS[cfg]
    dt = np.float32 if t == "float" else np.float64
    db = workloads.exp40(seed, n, d, dt)
    if text:
        # the reference generator's text format, read back by the importer shim (importNDDataset)
        path = tmp_path / "db.txt"
        with open(path, "w") as f:
            for row in db:
                f.write(", ".join("%.17g" % float(v) for v in row) + "\n")
    else:
        path = tmp_path / "db.bin"
        with open(path, "wb") as f:
            np.array([n, d, db.dtype.itemsize], np.uint32).tofile(f)
            db.tofile(f)
    out = tmp_path / "out.bin"
    p = subprocess.run([_exe(cfg), str(path), repr(float(eps)), str(out)], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    assert "[RESULT] ~ Total result set size:" in p.stdout
    raw = out.read_bytes()
    tneigh, tcand = np.frombuffer(raw, np.uint64, 2)
    ncell = np.frombuffer(raw, np.uint32, 1, 16)[0]
    off = np.frombuffer(raw, np.uint64, n + 1, 20)
    vals = np.frombuffer(raw, np.uint32, int(off[-1]), 20 + 8 * (n + 1))
    mn, _, nc, _ = oracle.geometry(db, k, eps)
    ref_off, ref_vals = oracle.join(db, k, eps, mn, nc)
    nb, total_cand = oracle.cell_workload(db, k, eps, mn, nc)
    assert int(tneigh) == int(ref_off[-1]) == int(off[-1])
    assert int(tcand) == total_cand and int(ncell) == len(nb)
    assert np.array_equal(off, ref_off)
    assert np.array_equal(vals, ref_vals)
