"""The finite-size-scaling driver bin/rlm_fss: several n_phi per run, one
energy_Chern_No_n<N>.txt per size in the reference's line format, resumable by sample."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_ROOT, golden

EXE = os.path.join(PKG_ROOT, "bin", "rlm_fss")


def _run(args, cwd):
    return subprocess.run([EXE] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


@pytest.mark.parametrize("args", [["-p", "bogus"], ["-n", ","], ["-b", "0"], ["-z"]])
def test_bad_options_print_usage(tmp_path, args):
    if not os.path.exists(EXE):
        pytest.skip("driver not built")
    r = _run(args, tmp_path)
    assert r.returncode == 2
    assert r.stdout.startswith("Usage: ")


def _parse(path):
    return np.array([[float(v) for v in ln.split()] for ln in open(path).read().splitlines()])


@pytest.mark.gpu
def test_fss_matches_reference_and_resumes(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(EXE):
        pytest.skip("driver not built")
    args = ["-n", "16,32", "-g", "4", "-c", "3", "-s", "7", "-b", "2"]
    r = _run(args, tmp_path)
    assert r.returncode == 0, r.stderr
    a32 = _parse(tmp_path / "energy_Chern_No_n32.txt")
    assert a32.shape == (3 * 32, 3)
    assert np.array_equal(a32[:, 0], np.repeat(np.arange(3), 32))
    # sample 0 of n_phi = 32, g = 4, seed 7 against the reference fixture
    d = golden("rlm_n32_g4_c1_s7.npz")
    assert np.abs(a32[:32, 1] - d["energies"][0]).max() <= 1e-7 * np.abs(d["energies"][0]).max()
    assert np.array_equal(np.rint(a32[:32, 2]), np.rint(d["chern"][0]))
    # interrupt: keep 1.5 samples of n_phi = 16, rerun, and get the same file back
    full16 = (tmp_path / "energy_Chern_No_n16.txt").read_text()
    lines = full16.splitlines(keepends=True)
    (tmp_path / "energy_Chern_No_n16.txt").write_text("".join(lines[:24]))
    r = _run(args, tmp_path)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "energy_Chern_No_n16.txt").read_text() == full16
    assert "samples 1..2" in r.stderr and "samples 3..2" in r.stderr
