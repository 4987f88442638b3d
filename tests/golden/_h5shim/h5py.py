"""Read-only stand-in for h5py, used ONLY by tests/golden/make_golden.py.

h5py is not installed in this image, and the reference imports it at module
load to read its shipped rate table (qed/rejection_sampling_tables.py:14-26).
That file stores two contiguous little-endian float64 datasets of 1024 values
at byte offsets 2048 ('int_Ai') and 10240 ('Aip'); their attributes are
z_N=1024, z_range=(0, 100), z_delta=(100-0)/(1024-1) (the generator's values,
qed/rejection_sampling_tables.py:91-112).  This shim serves exactly that.

The reference ships no optical-depth table (qed/optical_depth_tables.py:14-31
reads optical_depth_tables.h5 when present).  make_golden.py runs that mode
from a scratch copy of the reference package, where it writes an .npz archive
under that file name: datasets are its arrays, file attributes its 'attr_*'
entries.  Anything else is refused.
"""
import zipfile

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
        self._npz = None
        self.attrs = {}
        if zipfile.is_zipfile(path):
            with np.load(path) as z:
                self._npz = {k: z[k] for k in z.files}
            # scalar attributes as numpy scalars, as h5py returns them
            self.attrs = {k[5:]: (v[()] if v.ndim == 0 else v) for k, v in self._npz.items() if k.startswith("attr_")}
            return
        with open(path, "rb") as f:
            self._data = f.read()

    def __getitem__(self, name):
        if self._npz is not None:
            return _Dataset(np.array(self._npz[name]))
        off = _LAYOUT[name]
        return _Dataset(np.frombuffer(self._data[off:off + 8 * 1024], dtype="<f8").copy())

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
