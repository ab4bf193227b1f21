"""The rlm / hlm command-line drivers against the reference's own programs.

CPU: usage text, exit codes and log files are byte-identical to the reference's
(oracle/_ref/{rlm,hlm}_cpu_dp, built from the reference sources).
GPU: energy_Chern_No.txt has the reference's format and values."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_ROOT, REPO, golden

BIN = os.path.join(PKG_ROOT, "bin")
REF = os.path.join(REPO, "oracle", "_ref")


def _run(exe, args, cwd):
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    return subprocess.run([exe] + args, cwd=cwd, env=env, capture_output=True, text=True, timeout=600)


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{path} not built")


@pytest.mark.parametrize("prog,args", [("rlm", ["-h"]), ("rlm", ["-h", "1"]), ("rlm", ["-d", "5"]),
                                       ("hlm", ["-h", "x"]), ("hlm", ["-z"])])
def test_usage_and_exit_code_match_reference(tmp_path, prog, args):
    ours, ref = os.path.join(BIN, prog), os.path.join(REF, f"{prog}_cpu_dp")
    _need(ours)
    _need(ref)
    a = _run(ours, args, tmp_path)
    b = _run(ref, args, tmp_path)
    assert a.returncode == b.returncode == 2
    assert a.stdout.replace(ours, "PROG") == b.stdout.replace(ref, "PROG")


@pytest.mark.parametrize("prog,args,log", [
    ("rlm", ["-n", "16", "-i", "16", "-g", "2", "-c", "1", "-s", "7", "-q", "1"], "log_rlm.txt"),
    ("hlm", ["-x", "6", "-y", "6", "-q", "3", "-g", "2", "-b", "0", "-c", "1", "-s", "3", "-t", "2"], "log_hlm.txt")])
def test_log_file_matches_reference(tmp_path, prog, args, log):
    ours, ref = os.path.join(BIN, prog), os.path.join(REF, f"{prog}_cpu_dp")
    _need(ours)
    _need(ref)
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    _run(ours, args, tmp_path / "a")   # without a GPU it stops after writing the log
    _run(ref, args, tmp_path / "b")
    assert (tmp_path / "a" / log).read_bytes() == (tmp_path / "b" / log).read_bytes()


def _parse(txt):
    return np.array([[float(v) for v in ln.split()] for ln in txt.strip().splitlines()])


@pytest.mark.gpu
@pytest.mark.parametrize("prog,args,gold", [
    ("rlm", ["-n", "16", "-i", "16", "-g", "64", "-c", "2", "-s", "1", "-t", "4"], "rlm_n16_g64_c2_s1.npz"),
    ("hlm", ["-x", "3", "-y", "3", "-q", "3", "-g", "64", "-b", "0", "-c", "2", "-s", "1", "-t", "4"],
     "hlm_3x3_q3_g64_c2_s1.npz")])
def test_output_file_matches_reference(tmp_path, prog, args, gold):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ours = os.path.join(BIN, prog)
    _need(ours)
    r = _run(ours, args, tmp_path)
    assert r.returncode == 0, r.stderr
    for line in ("diagonalization time/k-point:", "Chern No. calculation time/k-point:",
                 "estimated total time:", "estimated # of samples/hour:", "# module"):
        assert line in r.stderr
    txt = (tmp_path / "energy_Chern_No.txt").read_text()
    ref_txt = str(golden(gold)["text"])
    a, b = _parse(txt), _parse(ref_txt)
    assert a.shape == b.shape
    assert np.array_equal(a[:, 0], b[:, 0])
    assert np.abs(a[:, 1] - b[:, 1]).max() <= 1e-7 * np.abs(b[:, 1]).max()
    assert np.array_equal(np.rint(a[:, 2]), np.rint(b[:, 2]))
    # same column layout: widths of the sample and energy fields
    la, lb = txt.splitlines(), ref_txt.rstrip("\n").splitlines()
    for x, y in zip(la, lb):
        assert x[:9] == y[:9]
        assert len(x.split(" ")[0]) == len(y.split(" ")[0])
