"""Host logic of the serving loop (no GPU): admission by slots and HBM footprint, footprint model."""
import sys
import threading
import time
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "neural-galerkin_b200"))

from jspsr.serving import Admission, footprint_bytes   # noqa: E402


def test_admission_slots():
    adm = Admission(slots=2, budget_bytes=1 << 40)
    a = adm.acquire(10)
    b = adm.acquire(10)
    with pytest.raises(TimeoutError):
        adm.acquire(10, timeout=0.05)
    adm.release(a)
    c = adm.acquire(10, timeout=1.0)
    assert adm.busy == 2 and adm.in_use == 20
    adm.release(b)
    adm.release(c)
    assert adm.busy == 0 and adm.in_use == 0


def test_admission_waits_for_memory_then_admits():
    adm = Admission(slots=8, budget_bytes=100)
    big = adm.acquire(70)
    admitted = []

    def second():
        admitted.append(adm.acquire(50))
    t = threading.Thread(target=second)
    t.start()
    time.sleep(0.1)
    assert not admitted                       # 70 + 50 > 100: held back
    adm.release(big)
    t.join(timeout=2)
    assert admitted == [50] and adm.waits == 1 and adm.peak_in_use == 70


def test_request_larger_than_budget_runs_alone():
    adm = Admission(slots=4, budget_bytes=100)
    assert adm.acquire(1000) == 100
    with pytest.raises(TimeoutError):
        adm.acquire(1, timeout=0.05)


def test_footprint_grows_with_points_and_resolution():
    assert footprint_bytes(500_000, 1 / 512) > footprint_bytes(1000, 1 / 512)
    assert footprint_bytes(500_000, 1 / 512) > footprint_bytes(500_000, 1 / 64)
    assert footprint_bytes(1000, 1 / 64) >= 64 << 20
