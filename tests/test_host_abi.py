"""CPU checks of the product library: it loads without a GPU, exports every entry point
include/rlm_b200.h declares, and its host-side stages are bit-exact with the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO, golden

import rlmb


def _declared_symbols():
    txt = open(os.path.join(REPO, "include", "rlm_b200.h")).read()
    return sorted(set(re.findall(r"\b(rlmb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = rlmb.lib()
    names = _declared_symbols()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name


def test_python_signatures_cover_the_header():
    assert set(_declared_symbols()) == set(rlmb._SIGNATURES)


def test_status_strings_and_no_device_error():
    lib = rlmb.lib()
    assert lib.rlmb_status_string(0) == b"ok"
    assert lib.rlmb_status_string(-1) == b"invalid argument"
    assert lib.rlmb_status_string(3).startswith(b"eigenvectors")
    h = ctypes.c_void_p()
    rc = lib.rlmb_create(ctypes.byref(h), 0)
    import torch
    if not torch.cuda.is_available():
        assert rc == -4 and not h.value
    else:
        assert rc == 0
        lib.rlmb_destroy(h)


def test_argument_errors_are_reported_not_crashing():
    lib = rlmb.lib()
    assert lib.rlmb_heevd_batched(None, None, None, 4, 1, None) == -1
    assert lib.rlmb_rlm_coeff_tables(16, 9, 18, 4, 4.0, 4.0, None, None, None) == -1
    assert lib.rlmb_rlm_disorder(0, 4.0, 4.0, 1, 0, None, None, None) == -1
    assert lib.rlmb_hlm_potentials(1, 0, 1, None) == -1
    assert lib.rlmb_rlm_mesh_solve(None, 16, 1.0, 16.0, 4, 1, 0, 1, None, None) == -1


def test_noalloc_order_limit_checked_on_the_host():
    """rlmb_heevd_batched_noalloc sizes its scratch on the host before any CUDA call: orders up
    to 927 fit its 32 MiB array (an empty batch returns at once), 928 does not.  The device
    pointers are placeholders that are never dereferenced."""
    lib = rlmb.lib()
    fake = ctypes.c_void_p(256)
    assert lib.rlmb_heevd_batched_noalloc(fake, fake, 927, 0, None, None) == 0
    rc = lib.rlmb_heevd_batched_noalloc(fake, fake, 928, 1, None, None)
    assert rc == -5
    assert b"scratch limit" in lib.rlmb_status_string(rc)
    assert lib.rlmb_heevd_batched_noalloc(None, fake, 16, 1, None, None) == -1


@pytest.mark.parametrize("name", ["rlm_n16_g64_c2_s1.npz", "rlm_n16_g8_c2_s1.npz",
                                  "rlm_n32_g4_c1_s7.npz", "rlm_n64_g4_c1_s3.npz",
                                  "rlm_n128_g2_c1_s5.npz"])
def test_rlm_host_tables_and_disorder_bit_exact(name):
    d = golden(name)
    n_phi, g = int(d["n_phi"]), int(d["n_mesh"])
    p = rlmb.rlm_params(n_phi, float(d["qc"]), float(d["ic"]))
    assert p["impurity_num"] == int(d["impurity_num"]) and p["off_head"] == int(d["off_head"])
    cmn, cmt, cjm = rlmb.rlm_coeff_tables(n_phi, p["off_head"], g, p["L1"], p["L2"])
    assert np.array_equal(cmn, d["coeff_mn"])
    assert np.array_equal(cmt, d["coeff_m_theta"])
    assert np.array_equal(cjm, d["coeff_jm"])
    for n in range(int(d["n_sample"])):
        x, y, s = rlmb.rlm_disorder(p["impurity_num"], p["L1"], p["L2"], int(d["seed"]), n)
        assert np.array_equal(x, d["x"][n]) and np.array_equal(y, d["y"][n])
        assert np.array_equal(s, d["s"][n])


@pytest.mark.parametrize("name", ["hlm_3x3_q3_g64_c2_s1.npz", "hlm_6x6_q3_b0_g8_c2_s1.npz",
                                  "hlm_48x16_q3_b0_g2_c1_s1.npz"])
def test_hlm_host_potentials_bit_exact(name):
    d = golden(name)
    pots = rlmb.hlm_potentials(int(d["seed"]), int(d["lx"]) * int(d["ly"]), int(d["n_sample"]))
    assert np.array_equal(pots, d["potentials"])
