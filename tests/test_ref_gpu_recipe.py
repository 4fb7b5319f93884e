"""The recipe and runner of the reference's GPU stage programs (no GPU needed): the runner parses
as bash, the recipe names the seven programs, and this library has a stage driver for each one
of them except the reference's FP32-versus-FP64 demonstration."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_runner_parses():
    subprocess.run(["bash", "-n", os.path.join(ROOT, "oracle", "ref_gpu_run.sh")], check=True)


def test_recipe_names_the_seven_programs_and_their_drivers():
    with open(os.path.join(ROOT, "oracle", "ref_gpu.mk")) as f:
        mk = f.read()
    progs = re.search(r"^PROGS\s*:=\s*(.*)$", mk, re.M).group(1).split()
    assert progs == ["fused_gg2gg", "fp32_gg2gg", "vegas", "cub_compaction", "unweight_lhe", "pdf_xsec", "generate"]
    assert "arch=compute_100a,code=sm_100a" in mk
    from cupythia_b200 import build
    assert sorted(set(progs) - {"fp32_gg2gg"}) == sorted(build.DRIVERS)
    with open(os.path.join(ROOT, "oracle", "ref_gpu_run.sh")) as f:
        assert f.read().count(" ".join(progs)) == 1   # the runner runs the same programs
