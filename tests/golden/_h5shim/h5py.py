"""Read-only stand-in for h5py, used ONLY by tests/golden/make_golden.py.

h5py is not installed in this image, and the reference imports it at module
load to read its shipped rate table (qed/rejection_sampling_tables.py:14-26).
That file stores two contiguous little-endian float64 datasets of 1024 values
at byte offsets 2048 ('int_Ai') and 10240 ('Aip'); their attributes are
z_N=1024, z_range=(0, 100), z_delta=(100-0)/(1024-1) (the generator's values,
qed/rejection_sampling_tables.py:91-112).  This shim serves exactly that and
refuses anything else.
"""
import numpy as np

_LAYOUT = {"int_Ai": 2048, "Aip": 10240}
_ATTRS = {"z_N": 1024, "z_range": np.array([0.0, 100.0]), "z_delta": (100.0 - 0.0) / (1024 - 1)}


class _Dataset:
    def __init__(self, arr):
        self._arr = arr
        self.attrs = dict(_ATTRS)

    def __getitem__(self, key):
        if key == ():
            return self._arr.copy()
        return self._arr[key]


class File:
    def __init__(self, path, mode="r"):
        if mode != "r":
            raise OSError("h5py shim is read-only")
        with open(path, "rb") as f:
            self._data = f.read()
        self.attrs = {}

    def __getitem__(self, name):
        off = _LAYOUT[name]
        return _Dataset(np.frombuffer(self._data[off:off + 8 * 1024], dtype="<f8").copy())

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
