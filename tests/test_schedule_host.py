"""Host-side scheduler logic: the reference's own Namelist object is accepted.

The reference's Namelist is a frozen dataclass whose derived values are the
private fields _start_datetime and _total_baroclinic_steps
(src/licom/readnamelist/time_data.py:61, namelist_data.py:56), which its
Schedule.configure reads (src/licom/mymodule/schedule.py:216-218).
"""
import datetime
from dataclasses import dataclass, field
from typing import Optional

import pytest

from licom4py_gpu_b200 import schedule
from licom4py_gpu_b200.momentum import Namelist


@dataclass(frozen=True)
class RefLikeNamelist:
    """Only the fields the reference's Schedule.configure reads, named as the reference names them."""
    baroclinic_dt: int = 3600
    diag_freq: Optional[int] = 6
    async_threads: int = 2
    _total_baroclinic_steps: int = field(default=48)
    _start_datetime: datetime.datetime = field(default=datetime.datetime(2001, 3, 4, 5))


def test_reference_namelist_private_fields_are_read():
    nl = RefLikeNamelist()
    assert not hasattr(nl, "total_baroclinic_steps") and not hasattr(nl, "start_datetime")
    assert schedule._namelist_value(nl, "total_baroclinic_steps") == 48
    assert schedule._namelist_value(nl, "start_datetime") == datetime.datetime(2001, 3, 4, 5)


def test_package_namelist_public_names_are_read():
    nl = Namelist(baroclinic_dt=3600.0, integration_days=2.0, start_year=1999, start_month=7, start_day=2)
    assert schedule._namelist_value(nl, "total_baroclinic_steps") == 48
    assert schedule._namelist_value(nl, "start_datetime") == datetime.datetime(1999, 7, 2)


def test_namelist_without_the_value_raises():
    @dataclass(frozen=True)
    class Bare:
        baroclinic_dt: int = 3600
    with pytest.raises(AttributeError):
        schedule._namelist_value(Bare(), "total_baroclinic_steps")
