"""Duogrid geometry container: the source of the barotropic path's 17 constants.

Mirrors the reference's ``Duogrid`` (``Dg``) singleton (src/licom/duogrid/duogrid.py):
``configure`` loads ``duogrid_C{nx}.npz`` (or generates it in-process with the
C++ generator), builds the ``inner``/``outer`` masks (duogrid.py:159-190), the
constant depth fields ``dzph``/``dzph_x``/``dzph_y`` (duogrid.py:192-229) and the
local k2e index tables ``loc_i_local``/``loc_j_local`` (duogrid.py:75-81,
src/licom/kernel/cube.py:166-207, which are the global tables when
px = py = 1).  Everything lives on the host as float64/int32 NumPy arrays; the
solver plan uploads what it needs once.

One GPU holds all six faces, so there is no sharding: ``pdev = px = py = 1``.
"""

from __future__ import annotations

import os
from typing import Dict, Optional

import numpy as np

from . import duogrid_gen

HALO = 3
NTILE = 6
DEFAULT_DEPTH = 5600.0   # src/licom/duogrid/duogrid.py:213


class Duogrid:
    """Class-level singleton like the reference's ``Dg``."""

    ntile: int = NTILE
    halo: int = HALO
    nx: int = 0
    nx_local: int = 0
    ny_local: int = 0
    px: int = 1
    py: int = 1
    depth: float = DEFAULT_DEPTH

    @classmethod
    def configure(cls, nx: int, npz_path: Optional[str] = None,
                  depth: float = DEFAULT_DEPTH, data: Optional[Dict[str, np.ndarray]] = None):
        """Load (or generate) the C{nx} geometry and derive the mask/depth/index fields.

        ``npz_path``: an existing ``duogrid_C{nx}.npz``; when omitted and
        ``data`` is None, the geometry is generated in-process.
        Raises ``FileNotFoundError`` like duogrid.py:58-59 when a given path is missing.
        """
        if data is None:
            if npz_path is not None:
                if not os.path.exists(npz_path):
                    raise FileNotFoundError(f"Duogrid NPZ file not found: {npz_path}")
                with np.load(npz_path) as z:
                    data = {k: z[k] for k in z.files}
            else:
                data = duogrid_gen.generate(nx)
        cls.nx = cls.nx_local = cls.ny_local = int(nx)
        cls.depth = float(depth)
        M = nx + 2 * HALO
        for name, arr in data.items():
            if name.startswith("k2e_loc"):
                setattr(cls, name, np.asarray(arr, dtype=np.int32))
            else:
                setattr(cls, name, np.asarray(arr, dtype=np.float64))
        inner = np.zeros((NTILE, M, M), dtype=np.float64)
        inner[:, HALO:-HALO, HALO:-HALO] = 1.0
        cls.inner = inner
        cls.outer = 1.0 - inner
        cls.dzph = np.full((NTILE, M, M), cls.depth, dtype=np.float64)
        cls.dzph_x = cls.dzph
        cls.dzph_y = cls.dzph
        cls.loc_i_local = np.asarray(data["k2e_loc_i"], dtype=np.int32)
        cls.loc_j_local = np.asarray(data["k2e_loc_j"], dtype=np.int32)
        return cls

    @classmethod
    def grid_dict(cls) -> Dict[str, np.ndarray]:
        names = ("a_pt", "a_l2c", "a_c2l", "rdx", "rdy", "rda", "a_f", "a_gct", "a_sina",
                 "c_dy", "d_dx", "k2e_coef", "k2e_loc_i", "k2e_loc_j")
        return {n: getattr(cls, n) for n in names if hasattr(cls, n)}


def make_consts(data: Dict[str, np.ndarray], depth: float = DEFAULT_DEPTH):
    """Build the 17-tuple in CONST_SOURCES order (src/licom/mymodule/schedule.py:95-116)
    from a generated grid dict, without touching the class-level singleton."""
    M = data["rdx"].shape[-1]
    inner = np.zeros((NTILE, M, M), dtype=np.float64)
    inner[:, HALO:-HALO, HALO:-HALO] = 1.0
    outer = 1.0 - inner
    dzph = np.full((NTILE, M, M), float(depth), dtype=np.float64)
    return (
        dzph, dzph, data["rdx"], data["rdy"], data["a_f"],
        data["k2e_coef"], data["k2e_loc_i"].astype(np.int32), data["k2e_loc_j"].astype(np.int32),
        data["a_c2l"], data["a_l2c"], inner, outer,
        data["a_gct"], data["a_sina"], data["rda"], data["c_dy"], data["d_dx"],
    )
