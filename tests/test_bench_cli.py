"""bench.py's launch pinning (host logic, no GPU): --driver MODE,BLOCKS,THREADS[,LANES]
binds that launch instead of running the autotuner."""

import argparse
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


class _Recorder:
    def __init__(self):
        self.calls = []
        self.lanes = 8

    def set_driver(self, *a):
        self.calls.append(("set_driver", a))

    def _bind(self):
        self.calls.append(("bind",))

    def autotune(self, frames=3):
        self.calls.append(("autotune", frames))
        return {"ms_per_frame": {"x": 1.0}}


def test_driver_pins_the_launch():
    s = _Recorder()
    rep = bench.pin_or_tune(s, argparse.Namespace(driver="0,296,256,1"))
    assert s.calls == [("set_driver", (0, 296, 256)), ("bind",)]
    assert s.lanes == 1
    assert rep == {"ms_per_frame": {}, "pinned": "0,296,256,1"}


def test_driver_without_lanes_keeps_them():
    s = _Recorder()
    bench.pin_or_tune(s, argparse.Namespace(driver="2,16,512"))
    assert s.calls[0] == ("set_driver", (2, 16, 512)) and s.lanes == 8


def test_no_driver_runs_the_autotuner():
    s = _Recorder()
    rep = bench.pin_or_tune(s, argparse.Namespace(driver=""))
    assert s.calls == [("autotune", 3)]
    assert rep == {"ms_per_frame": {"x": 1.0}}


def test_batch_launch_claim_counts_the_sort_passes():
    """74,138 pile bodies in 128 scenes: 37-bit keys, five sort passes of five
    launches plus the copy back, beside the eleven other pile kernels and the
    cloths' frame kernel."""
    assert bench.lbvh_sort_launches(1440, 1) == 1
    assert bench.lbvh_sort_launches(74138, 128) == 26

    class _Piles:
        num_bodies = 74138
        n_scenes = 128

    class _Batch:
        piles = _Piles()

    assert bench.batch_launches_per_frame(_Batch()) == 38


def test_sort_launches_by_size_and_bits():
    assert bench.sort_launches(16384, 63) == 1
    assert bench.sort_launches(16385, 63) == 40  # eight passes, even: no copy back
    assert bench.sort_launches(100000, 40) == 26  # five passes and the copy back
