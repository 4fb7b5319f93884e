"""Stage drivers (C++ mains over the C ABI with the reference's argv, output and exit codes:
0 = VALIDATION: PASS, 2 = FAIL, 1 = CUDA / library error).  Without a GPU every driver must stop
with exit code 1 and the library's error message; on a GPU each must validate at small sizes."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(os.path.dirname(HERE), "cupythia_b200", "bin")
SMALL = {"fused_gg2gg": ["100"], "vegas": ["100"], "pdf_xsec": ["16"], "cub_compaction": ["4194304"],
         "unweight_lhe": ["256"], "generate": ["200000"]}


@pytest.fixture(scope="module")
def drivers():
    from cupythia_b200 import build
    return {os.path.basename(p): p for p in build.build_drivers()}


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_drivers_report_cuda_errors_with_exit_code_1(drivers, tmp_path):
    for name, exe in drivers.items():
        r = subprocess.run([exe] + SMALL[name], capture_output=True, text=True, cwd=tmp_path, timeout=120)
        assert r.returncode == 1, (name, r.returncode, r.stdout, r.stderr)
        assert "cupythia_b200 error" in r.stdout, (name, r.stdout)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SMALL))
def test_driver_validates_on_gpu(drivers, name, tmp_path):
    r = subprocess.run([drivers[name]] + SMALL[name], capture_output=True, text=True, cwd=tmp_path, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "VALIDATION: PASS" in r.stdout
    if name == "unweight_lhe":
        assert (tmp_path / "events.lhe").read_text().count("<event>") == 1000


@pytest.mark.gpu
def test_sharded_drivers_cover_disjoint_points(drivers, tmp_path):
    """CUPYTHIA_SHARD / CUPYTHIA_SHARD_N offset the point indices (cuPythia/common/rng.cuh:14-19):
    two shards of the compaction driver validate on their own ranges."""
    for shard in ("0", "1"):
        env = dict(os.environ, CUPYTHIA_SHARD=shard, CUPYTHIA_SHARD_N="4194304")
        r = subprocess.run([drivers["cub_compaction"], "4194304"], capture_output=True, text=True, cwd=tmp_path,
                           env=env, timeout=600)
        assert r.returncode == 0 and "VALIDATION: PASS" in r.stdout, r.stdout
