"""The drop-in claim: the reference's own, unchanged NeighborList and md.nve (baseline/_ref)
run on this package's operator library exactly as on the reference's own CUDA operator.

Each arm runs in its own process (tests/reference_dropin.py), since both libraries register
the namespace nabladyn_neighbors. Pair sets, rebuild counts and capacities must be equal bit
for bit; after 20 float64 NVE steps the positions agree to 1e-9 nm and the velocities to 1e-8
nm/ps (only the order of the pairs differs, hence the summation order of the forces), with the
same images and rebuilds. Skipped when baseline/_ref holds no reference build.
"""

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
REFERENCE = ROOT / "baseline" / "_ref" / "nabladyn" / "neighbors"

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not any(REFERENCE.glob("_C*.so")), reason="no reference build"),
]


def run_arm(tmp_path, mode: str):
    outputs = tmp_path / f"{mode}.npz"
    subprocess.run([sys.executable, str(ROOT / "tests" / "reference_dropin.py"), mode,
                    str(outputs)], check=True, timeout=1200)
    return dict(np.load(outputs))


def test_reference_runs_unchanged_on_our_operator(tmp_path):
    own = run_arm(tmp_path, "own")
    ours = run_arm(tmp_path, "b200")
    for k in range(3):
        np.testing.assert_array_equal(ours[f"keys_{k}"], own[f"keys_{k}"])
        assert int(ours[f"rebuilds_{k}"]) == int(own[f"rebuilds_{k}"])
        assert int(ours[f"capacity_{k}"]) == int(own[f"capacity_{k}"])
    assert [int(own[f"rebuilds_{k}"]) for k in range(3)] == [1, 1, 2]
    assert int(ours["md_rebuilds"]) == int(own["md_rebuilds"])
    np.testing.assert_array_equal(ours["images"], own["images"])
    np.testing.assert_allclose(ours["positions"], own["positions"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(ours["velocities"], own["velocities"], rtol=0, atol=1e-8)
