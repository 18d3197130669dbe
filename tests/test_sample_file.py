"""Sample files (md/_output.py) against an in-memory h5py stand-in (tests/fake_h5py.py): the
datasets, shapes, dtypes, units and attributes of the reference's layout
(src/nabladyn/md/_output.py:44-133), samples read back as written, a file of another schema
rejected. A GPU test runs Simulation.run(..., sample_file=...) through the same stand-in."""

import sys

import numpy as np
import pytest

import fake_h5py
from nabladyn_b200.md import _output, read_sample_file


@pytest.fixture
def h5py(monkeypatch):
    monkeypatch.setitem(sys.modules, "h5py", fake_h5py)
    fake_h5py.FILES.clear()
    return fake_h5py


def frame(n, k, dtype):
    rng = np.random.default_rng(k)
    return {"positions": rng.uniform(0, 3, (n, 3)).astype(dtype),
            "velocities": rng.normal(size=(n, 3)).astype(dtype),
            "forces": rng.normal(size=(n, 3)).astype(dtype),
            "cell": np.full(3, 3.0, dtype=dtype),
            "images": rng.integers(-2, 3, (n, 3)).astype(np.int64)}


def test_samples_round_trip(h5py):
    n, dtype = 5, np.float32
    fields = ("potential_energy", "kinetic_energy", "total_energy", "temperature", "pressure")
    writer = _output.SampleWriter("run.h5", masses=np.full(n, 39.948, dtype=dtype),
                                  fields=fields, attributes={"ensemble": "NVE", "timestep": 0.004,
                                                             "cutoff": 1.0})
    frames = [frame(n, k, dtype) for k in range(3)]
    for k, f in enumerate(frames):
        writer.write(10 * (k + 1), 0.04 * (k + 1), f, [float(k + v) for v in range(5)])
    writer.close()
    assert h5py.FILES["run.h5"].closed
    samples, attributes = read_sample_file("run.h5")
    assert attributes == {"schema": "nabladyn.samples", "schema_version": 1, "ensemble": "NVE",
                          "timestep": 0.004, "cutoff": 1.0}
    np.testing.assert_array_equal(samples["step"], [10, 20, 30])
    np.testing.assert_allclose(samples["time"], [0.04, 0.08, 0.12])
    for name in _output.FRAME:
        np.testing.assert_array_equal(samples[name], np.stack([f[name] for f in frames]))
    assert samples["positions"].dtype == np.float32 and samples["images"].dtype == np.int64
    np.testing.assert_array_equal(samples["temperature"], [3.0, 4.0, 5.0])
    np.testing.assert_array_equal(samples["masses"], np.full(n, 39.948, dtype=np.float32))
    stored = h5py.FILES["run.h5"]
    assert stored["pressure"].attrs["unit"] == "kJ/mol/nm^3"
    assert stored["positions"].attrs["unit"] == "nm" and stored["masses"].attrs["unit"] == "Da"
    assert stored["positions"].maxshape == (None, n, 3)


def test_a_foreign_file_is_rejected(h5py):
    other = h5py.File("other.h5", "w")
    other.attrs["schema"] = "something.else"
    with pytest.raises(ValueError, match="not a NablaDyn sample file"):
        read_sample_file("other.h5")
