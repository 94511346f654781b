"""Duogrid geometry generation: the ``make field`` step of the barotropic path.

Python face of ``libduogrid.so`` (``csrc/duogrid_gen.cpp``), the C++ restatement
of the reference's Fortran generator.  It replaces the reference's
``DuogridFieldGenerator`` (src/initial_field/main.py:25-142) together with its
ctypes layer (src/initial_field/_c_duogrid_function.py): the NPZ written here
has the same file name (``duogrid_C{nx}.npz``), field names, dtypes and
(6, nx+6, nx+6[, 2[, 2]]) layouts, so the loader in :mod:`.duogrid` and the
reference's ``Dg.configure`` read the same file.
"""

from __future__ import annotations

import ctypes
import os
from typing import Dict, Iterable, Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libduogrid.so")

# src/initial_field/main.py:30-39
ESSENTIAL_FIELDS = frozenset({
    "a_sina", "a_f", "rdx", "rdy", "rda", "a_gct",
    "k2e_coef", "k2e_loc_i", "k2e_loc_j", "a_c2l", "a_l2c",
    "c_dy", "d_dx",
    "a_pt",
})

_lib = None


class DuogridError(RuntimeError):
    """Raised when the native generator reports an error."""


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise FileNotFoundError(
            f"{_LIB_PATH} is missing; build it with `python -m licom4py_gpu_b200.build`")
    lib = ctypes.CDLL(_LIB_PATH)
    lib.ldg_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.ldg_create.restype = ctypes.c_int
    lib.ldg_destroy.argtypes = [ctypes.c_void_p]
    lib.ldg_destroy.restype = None
    lib.ldg_field_shape.argtypes = [ctypes.c_void_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_long)]
    lib.ldg_field_shape.restype = ctypes.c_int
    lib.ldg_num_fields.argtypes = []
    lib.ldg_num_fields.restype = ctypes.c_int
    lib.ldg_field_name.argtypes = [ctypes.c_int]
    lib.ldg_field_name.restype = ctypes.c_char_p
    lib.ldg_field_is_int.argtypes = [ctypes.c_char_p]
    lib.ldg_field_is_int.restype = ctypes.c_int
    lib.ldg_get_f64.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    lib.ldg_get_f64.restype = ctypes.c_int
    lib.ldg_get_i32.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
    lib.ldg_get_i32.restype = ctypes.c_int
    lib.ldg_last_error.argtypes = []
    lib.ldg_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise DuogridError(_load().ldg_last_error().decode())


def all_field_names() -> list[str]:
    lib = _load()
    return [lib.ldg_field_name(i).decode() for i in range(lib.ldg_num_fields())]


def generate(nx: int, fields: Optional[Iterable[str]] = None,
             full_export: bool = False) -> Dict[str, np.ndarray]:
    """Generate the duogrid geometry at resolution ``nx`` (C{nx}).

    ``fields`` defaults to the reference's essential set, or every exported
    field when ``full_export`` is true (src/initial_field/main.py:81-90).
    Float fields are float64, the k2e location tables int32.
    """
    lib = _load()
    if fields is None:
        fields = all_field_names() if full_export else sorted(ESSENTIAL_FIELDS)
    handle = ctypes.c_void_p()
    _check(lib.ldg_create(int(nx), ctypes.byref(handle)))
    out: Dict[str, np.ndarray] = {}
    try:
        for name in fields:
            bname = name.encode()
            nd = ctypes.c_int()
            shape = (ctypes.c_long * 5)()
            _check(lib.ldg_field_shape(handle, bname, ctypes.byref(nd), shape))
            shp = tuple(shape[i] for i in range(nd.value))
            if lib.ldg_field_is_int(bname):
                arr = np.empty(shp, dtype=np.int32)
                _check(lib.ldg_get_i32(handle, bname, arr.ctypes.data))
            else:
                arr = np.empty(shp, dtype=np.float64)
                _check(lib.ldg_get_f64(handle, bname, arr.ctypes.data))
            out[name] = arr
    finally:
        lib.ldg_destroy(handle)
    return out


def npz_name(nx: int) -> str:
    """File name of the serialised grid (src/initial_field/main.py:96)."""
    return f"duogrid_C{nx}.npz"


def cache_dir() -> str:
    """Directory of the per-resolution NPZ cache: ``$LICOM_BT_FIELD_DIR``, else
    ``~/.cache/licom4py_gpu_b200/field`` (the reference keeps its files in ``field/``)."""
    return os.environ.get("LICOM_BT_FIELD_DIR",
                          os.path.join(os.path.expanduser("~"), ".cache", "licom4py_gpu_b200", "field"))


def load_or_generate(nx: int, directory: Optional[str] = None) -> Tuple[Dict[str, np.ndarray], bool]:
    """The C{nx} geometry from ``duogrid_C{nx}.npz`` in ``directory`` (default
    :func:`cache_dir`), generating and writing the file on the first request.

    The reference generates the file once (``make field``,
    src/initial_field/main.py:81-98) and every run loads it
    (src/licom/duogrid/duogrid.py:58-59); this does both, so repeated runs at
    one resolution skip the generator.  Returns (fields, cache_hit).  A file
    that lacks an essential field or has the wrong shape is regenerated.
    """
    d = directory if directory is not None else cache_dir()
    path = os.path.join(d, npz_name(nx))
    m = int(nx) + 6
    if os.path.exists(path):
        try:
            with np.load(path) as z:
                data = {k: z[k] for k in z.files}
            if ESSENTIAL_FIELDS <= set(data) and data["rdx"].shape == (6, m, m):
                return data, True
        except (OSError, ValueError, KeyError):
            pass
    data = generate(nx)
    try:
        os.makedirs(d, exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp.npz"
        np.savez(tmp, **data)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only cache directory only costs the regeneration next time
    return data, False


class DuogridFieldGenerator:
    """Writes ``duogrid_C{nx}.npz`` like the reference generator of the same name.

    Mirrors src/initial_field/main.py:25-142: ``run()`` serialises the
    essential fields (or every field with ``full_export``) to the current
    working directory, or to ``out_dir`` when given.
    """

    ESSENTIAL_FIELDS = ESSENTIAL_FIELDS

    def __init__(self, nx: int, full_export: bool = False, out_dir: Optional[str] = None):
        self.nx = int(nx)
        self.full_export = full_export
        self.out_dir = out_dir
        self.target_dim = self.nx + 6

    def run(self) -> str:
        data = generate(self.nx, full_export=self.full_export)
        out_dir = self.out_dir if self.out_dir is not None else os.getcwd()
        os.makedirs(out_dir, exist_ok=True)
        path = os.path.join(out_dir, npz_name(self.nx))
        np.savez(path, **data)
        return path


def main(argv=None) -> None:
    import argparse
    p = argparse.ArgumentParser(description="Generate the duogrid geometry NPZ")
    p.add_argument("--nx", type=int, default=int(os.environ.get("FIELD_NX", 96)))
    p.add_argument("--full", action="store_true", help="export every field")
    p.add_argument("--out-dir", default=None)
    a = p.parse_args(argv)
    print(DuogridFieldGenerator(a.nx, a.full, a.out_dir).run())


if __name__ == "__main__":
    main()
