"""Host side of the CUDA library, checked without a GPU: the shared library
loads and exports every entry point that include/qlat_b200.h declares, and
its host RngState (split / rand_gen / u_rand_gen / g_rand_gen) is bit-exact
with the oracle."""

import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    hdrs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    names = set()
    for h in hdrs:
        txt = open(h).read()
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(qgb_\w+)\s*\(", txt, re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from qlat_b200 import build as B
    path = B.build()
    return ctypes.CDLL(path)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 40
    assert "qgb_set_gm_force" in names and "qgb_run_hmc_evolve_mixed" in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    from qlat_b200 import _lib
    declared = set(declared_symbols()) - {"qgb_last_error"}
    assert declared == set(_lib.SIGNATURES), declared ^ set(_lib.SIGNATURES)


def test_host_rng_matches_oracle(oracle):
    import qlat_b200 as q
    for seed in ["seed", "run_hmc-test-4nt8", "x" * 130]:
        a, b = q.RngState(seed), oracle.RngState(seed)
        assert (a.export() == b.export()).all()
        for sidx in ["gf-init", 7, "set_rand_gauge_momentum", "y" * 100]:
            a2, b2 = a.split(sidx), b.split(sidx)
            assert (a2.export() == b2.export()).all()
            for _ in range(20):
                assert a2.rand_gen() == b2.rand_gen()
                assert a2.u_rand_gen(1.0, -1.0) == b2.u_rand_gen(1.0, -1.0)
                assert a2.g_rand_gen(0.3, 0.7) == b2.g_rand_gen(0.3, 0.7)
            assert (a2.export() == b2.export()).all()
    assert (q.RngState().export() == oracle.RngState().export()).all()


def test_metropolis_cpp_semantics(oracle):
    import qlat_b200 as q
    rs = q.RngState("metropolis")
    for dh in [-0.5, 0.0, 0.01, 0.3, 2.0]:
        flag, prob = q.metropolis_accept_cpp(dh, 1, rs)
        f2, p2 = oracle.metropolis_accept_cpp(dh, oracle.RngState("metropolis"))
        assert flag == f2 and prob == p2


def test_field_creation_fails_loudly_without_device():
    import qlat_b200 as q
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(q.QlatB200Error) as e:
        q.GaugeField(q.Geometry((4, 4, 4, 4)))
    assert e.value.code == 8


def test_missing_library_fails_loudly():
    """Without the CUDA library the package raises at its first call; nothing
    falls back to another implementation."""
    import subprocess
    import sys
    code = ("import qlat_b200._lib as L\n"
            "L.LIB_PATH = '/nonexistent/libqlat_b200.so'\n"
            "L._lib = None\n"
            "import qlat_b200 as q\n"
            "try:\n"
            "    q.GaugeField(q.Geometry((4, 4, 4, 4)))\n"
            "except RuntimeError as e:\n"
            "    print('raised:', e)\n")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                       cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "raised:" in r.stdout and "is missing" in r.stdout
