"""CPU: the lucasntt program's options, result files and failure without a GPU.

The option resolution (LucasNTT.ini, argv, resume from the stats file) and
the .dat / .txt formats are checked by a native test linked with the
program's own sources; the program itself must refuse to run, with the
reference's message and exit status 1, when there is no CUDA device.
"""
import subprocess
from pathlib import Path

import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]
HOST = ROOT / "cuda_b200" / "host"


def test_options_and_files_native(tmp_path):
    exe = tmp_path / "cli_selftest"
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "cli_selftest.cpp"),
                    str(HOST / "ini_file.cpp"), str(HOST / "options.cpp"), str(HOST / "residue_files.cpp")],
                   check=True)
    work = tmp_path / "work"
    work.mkdir()
    r = subprocess.run([str(exe), str(work)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "cli selftest ok" in r.stdout


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_program_without_device_fails_loudly(tmp_path):
    exe = ROOT / "cuda_b200" / "lucasntt"
    if not exe.exists():
        subprocess.run(["make", "-C", str(ROOT / "cuda_b200"), "lucasntt"], check=True)
    r = subprocess.run([str(exe), "9689"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    assert "Exponent = 9689" in r.stdout and "CUDA" in r.stdout
    assert not (tmp_path / "LucasNTT_results.txt").exists()
