"""WRF NetCDF files without xarray: the classic (NetCDF-3) format through scipy.

The reference opens its three input files with ``xarray.open_dataset``
(pywrf/solver.py:22-46) and reads every variable as ``ds[name][...].data``.
:func:`open_dataset` gives the same access (``ds[name]`` -> a numpy array
with the file's shape) for classic-format files when xarray is not
installed; :func:`write_dataset` writes such a file from WRF-named arrays (for
example a synthetic case from :mod:`pywrf_b200.synthetic`).  NetCDF-4 (HDF5)
files need xarray with a netCDF4 or h5netcdf backend: :func:`open_dataset`
refuses them with a message that says so.
"""
from __future__ import annotations

import os
from typing import Mapping

import numpy as np

_HDF5_MAGIC = b"\x89HDF\r\n\x1a\n"


class NetcdfDataset(dict):
    """Variables of one file by name, as numpy arrays (read into memory)."""

    def __init__(self, path: str, arrays: Mapping[str, np.ndarray]):
        super().__init__(arrays)
        self.path = path


def open_dataset(path: str) -> NetcdfDataset:
    """Read every variable of a classic-format NetCDF file."""
    from scipy.io import netcdf_file

    with open(path, "rb") as f:
        head = f.read(8)
    if head == _HDF5_MAGIC:
        raise ValueError(f"{path}: a NetCDF-4 (HDF5) file; reading it needs xarray with a netCDF4 backend")
    if head[:3] != b"CDF":
        raise ValueError(f"{path}: not a NetCDF file")
    out = {}
    with netcdf_file(path, "r", mmap=False) as nc:
        for name, var in nc.variables.items():
            a = np.array(var.data, copy=True)
            out[name] = a.astype(a.dtype.newbyteorder("="), copy=False)
    return NetcdfDataset(path, out)


def write_dataset(path: str, arrays: Mapping[str, np.ndarray]) -> None:
    """Write WRF-named arrays to a classic-format (64-bit offset) NetCDF file;
    each variable gets dimensions named after its extents."""
    from scipy.io import netcdf_file

    tmp = path + ".tmp"
    with netcdf_file(tmp, "w", version=2) as nc:
        made = set()
        for name, a in arrays.items():
            a = np.asarray(a)
            if a.dtype == np.float64:
                a = a.astype(np.float32)
            dims = []
            for n in a.shape:
                d = f"d{n}"
                if d not in made:
                    nc.createDimension(d, n)
                    made.add(d)
                dims.append(d)
            v = nc.createVariable(name, a.dtype, tuple(dims))
            v[...] = a
    os.replace(tmp, path)
