"""A stand-in for the part of h5py that sample files use, held in memory (h5py is not installed
in this image): File(path, mode) with attrs, create_dataset (data, or an empty growable shape
with maxshape, dtype and chunks), dataset resize along axis 0, item assignment and reads,
iteration over names and the context-manager protocol. Files live in ``FILES`` by path, so a
file written can be read back in the same process. Used by tests/test_sample_file*.py."""

from __future__ import annotations

import numpy as np

FILES: dict[str, "File"] = {}


class Dataset:
    def __init__(self, data: np.ndarray, maxshape=None):
        self.data = data
        self.maxshape = maxshape
        self.attrs: dict = {}

    def resize(self, size: int, axis: int = 0) -> None:
        assert axis == 0 and self.maxshape is not None and self.maxshape[0] is None
        grown = np.zeros((size, *self.data.shape[1:]), dtype=self.data.dtype)
        grown[: min(size, self.data.shape[0])] = self.data[:size]
        self.data = grown

    def __setitem__(self, index, value) -> None:
        self.data[index] = value

    def __getitem__(self, index):
        return self.data[index]


class File:
    def __init__(self, path: str, mode: str = "r"):
        if mode == "w":
            self.attrs: dict = {}
            self.datasets: dict[str, Dataset] = {}
            FILES[path] = self
        else:
            stored = FILES[path]
            self.attrs, self.datasets = stored.attrs, stored.datasets
        self.closed = False

    def create_dataset(self, name, shape=None, maxshape=None, dtype=None, chunks=None, data=None):
        array = np.array(data) if data is not None else np.zeros(shape, dtype=dtype)
        self.datasets[name] = Dataset(array, maxshape)
        return self.datasets[name]

    def __getitem__(self, name: str) -> Dataset:
        return self.datasets[name]

    def __iter__(self):
        return iter(self.datasets)

    def close(self) -> None:
        self.closed = True

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
