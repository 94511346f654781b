"""Per-resolution geometry cache: duogrid_C{N}.npz written once, loaded afterwards.

The reference writes the file once (src/initial_field/main.py:81-98) and the
solver loads it (src/licom/duogrid/duogrid.py:58-59).
"""
import os

import numpy as np

from licom4py_gpu_b200 import duogrid_gen


def test_first_request_generates_and_writes_second_loads(tmp_path):
    d = str(tmp_path)
    a, hit_a = duogrid_gen.load_or_generate(12, d)
    assert not hit_a
    assert os.path.exists(os.path.join(d, "duogrid_C12.npz"))
    b, hit_b = duogrid_gen.load_or_generate(12, d)
    assert hit_b
    assert set(a) == set(b) == set(duogrid_gen.ESSENTIAL_FIELDS)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
        assert a[k].dtype == b[k].dtype


def test_damaged_cache_file_is_regenerated(tmp_path):
    d = str(tmp_path)
    path = os.path.join(d, "duogrid_C8.npz")
    with open(path, "wb") as f:
        f.write(b"not an npz file")
    data, hit = duogrid_gen.load_or_generate(8, d)
    assert not hit and data["rdx"].shape == (6, 14, 14)
    assert duogrid_gen.load_or_generate(8, d)[1]


def test_wrong_resolution_in_file_is_regenerated(tmp_path):
    d = str(tmp_path)
    np.savez(os.path.join(d, "duogrid_C10.npz"), **duogrid_gen.generate(8))
    data, hit = duogrid_gen.load_or_generate(10, d)
    assert not hit and data["rdx"].shape == (6, 16, 16)
