"""Sample files: each sample's frame and panel in an HDF5 file, readable back as arrays.

The file layout is the reference's (src/nabladyn/md/_output.py:44-133), so files from either
build read in the other: root attributes ``schema`` = "nabladyn.samples", ``schema_version`` = 1,
the ensemble's settings, ``timestep`` (ps) and ``cutoff`` (nm); a ``masses`` dataset; and one
growable dataset per sampled quantity (``step``, ``time``, the frame arrays ``positions``,
``velocities``, ``forces``, ``cell``, ``images``, then the panel fields), each with a ``unit``
attribute. h5py is imported only when a file is written or read, as there: a run without a
sample file needs nothing more.
"""

from __future__ import annotations

import os

import numpy as np

SCHEMA, SCHEMA_VERSION = "nabladyn.samples", 1

# The frame arrays of a sample, all in the run's dtype but images (int64).
FRAME = ("positions", "velocities", "forces", "cell", "images")

UNITS = {
    "step": "1", "time": "ps", "masses": "Da", "positions": "nm", "velocities": "nm/ps",
    "forces": "kJ/mol/nm", "cell": "nm", "images": "1", "potential_energy": "kJ/mol",
    "kinetic_energy": "kJ/mol", "total_energy": "kJ/mol", "temperature": "K",
    "pressure": "kJ/mol/nm^3", "volume": "nm^3", "conserved_energy": "kJ/mol",
}


class SampleWriter:
    """One sample file, created (or overwritten) at ``path``; ``write`` appends a sample."""

    def __init__(self, path, *, masses: np.ndarray, fields: tuple[str, ...], attributes: dict):
        import h5py  # only a run that writes a file needs it

        n, dtype = masses.shape[0], masses.dtype
        per_sample = {"step": ((), np.int64), "time": ((), np.float64)}
        per_sample.update({name: ((n, 3), dtype) for name in ("positions", "velocities", "forces")})
        per_sample["cell"] = ((3,), dtype)
        per_sample["images"] = ((n, 3), np.int64)
        per_sample.update({name: ((), dtype) for name in fields})
        self._file = h5py.File(os.fspath(path), "w")
        self._file.attrs.update({"schema": SCHEMA, "schema_version": SCHEMA_VERSION,
                                 **attributes})
        self._file.create_dataset("masses", data=masses).attrs["unit"] = UNITS["masses"]
        for name, (shape, kind) in per_sample.items():
            dataset = self._file.create_dataset(name, (0, *shape), maxshape=(None, *shape),
                                                dtype=kind, chunks=(64, *shape))
            dataset.attrs["unit"] = UNITS[name]
        self._fields = tuple(fields)
        self._rows = 0

    def write(self, step: int, time: float, frame: dict, values: list[float]) -> None:
        """Append one sample: its step, time (ps), frame arrays (FRAME) and panel values."""
        sample = {"step": step, "time": time, **{name: frame[name] for name in FRAME},
                  **dict(zip(self._fields, values))}
        for name, value in sample.items():
            dataset = self._file[name]
            dataset.resize(self._rows + 1, axis=0)
            dataset[self._rows] = value
        self._rows += 1

    def close(self) -> None:
        self._file.close()


def read_sample_file(path: str | os.PathLike) -> tuple[dict[str, np.ndarray], dict]:
    """The samples of a sample file as arrays by dataset name, and its attributes (ensemble
    settings, timestep in ps, cutoff in nm). Not a restart: it holds no chain or barostat
    state; continue a run from ``Simulation.state()``.

    Raises ``ValueError`` for a file that is not a sample file of this layout.
    """
    import h5py  # only reading a file needs it

    with h5py.File(os.fspath(path), "r") as file:
        if file.attrs.get("schema") != SCHEMA:
            raise ValueError(f"{path} is not a NablaDyn sample file")
        samples = {name: file[name][()] for name in file}
        attributes = {name: value.item() if isinstance(value, np.generic) else value
                      for name, value in file.attrs.items()}
    return samples, attributes


__all__ = ("FRAME", "SampleWriter", "read_sample_file")
