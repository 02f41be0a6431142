"""The autotuner's cache (mpcd_tune_key, mpcd_tune_cache_lookup/store): host
code of the library, checked without a GPU."""
import ctypes as C

import pytest

from mpcd_b200 import abi, gpu
from mpcd_b200 import workloads as W


def _choice(kernel, strategy=-1, tile=0, sort=30, us=12.5):
    c = abi.TuneChoice()
    c.kernel, c.strategy, c.tile_particles, c.sort_interval, c.us_per_step = \
        kernel, strategy, tile, sort, us
    return c


def test_key_names_the_workload_and_device():
    cfg = W.cfg_channel3d((16, 8, 8), g=1e-3, precision=abi.PREC_MIXED)
    k = gpu.tune_key(cfg, 20480, "NVIDIA B200")
    assert k.startswith("NVIDIA B200|dim=3|L=16x8x8|n=20480|op=3|lc=0|prec=1|")
    assert "solid=2|phantom=2|species=1|grav=1" in k
    assert gpu.tune_key(cfg, 20481, "NVIDIA B200") != k
    cfg2 = W.cfg_channel3d((16, 8, 8), g=1e-3, precision=abi.PREC_FP64)
    assert gpu.tune_key(cfg2, 20480, "NVIDIA B200") != k
    assert gpu.tune_key(cfg, 20480, "other|gpu\tname").startswith("other_gpu_name|")


def test_cache_round_trip_last_entry_wins(tmp_path):
    path = tmp_path / "tune.txt"
    key = gpu.tune_key(W.cfg_srd3d((8, 8, 8)), 5120, "dev")
    assert gpu.tune_cache_lookup(path, key) is None  # no file yet
    gpu.tune_cache_store(path, key, _choice(abi.KERNEL_TILE, abi.STRATEGY_SCATTER, 1024))
    gpu.tune_cache_store(path, "another|key", _choice(abi.KERNEL_SPLIT))
    gpu.tune_cache_store(path, key, _choice(abi.KERNEL_RESIDENT, sort=20, us=7.25))
    c = gpu.tune_cache_lookup(path, key)
    assert (c.kernel, c.sort_interval, c.us_per_step, c.from_cache) == \
        (abi.KERNEL_RESIDENT, 20, pytest.approx(7.25), 1)
    assert gpu.tune_cache_lookup(path, key + "x") is None
    assert gpu.tune_cache_lookup(path, "another|key").kernel == abi.KERNEL_SPLIT


def test_cache_skips_malformed_lines_and_rejects_bad_keys(tmp_path):
    path = tmp_path / "tune.txt"
    key = "k1"
    path.write_text("k1\tnot numbers\n" "k1\t99\t0\t0\t30\t1.0\n" "k1\t4\t-1\t0\t10\t3.5\n"
                    "k1\t1\t0\n")
    c = gpu.tune_cache_lookup(path, key)
    assert (c.kernel, c.sort_interval) == (abi.KERNEL_RESIDENT, 10)
    lib = gpu.load()
    assert lib.mpcd_tune_cache_store(str(path).encode(), b"a\tb", C.byref(_choice(1))) == \
        abi.ERR_ARG
