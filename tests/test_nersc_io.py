"""NERSC gauge files (save_gauge_field / load_gauge_field, qcd.h:66-250).

CPU: the library's host-side format code against files that the reference
library itself writes and reads (oracle/_ref/ref_nersc, built from the
reference's sources): byte-identical data, identical header, both checksums,
both directions.  GPU: GaugeField.save / GaugeField.load through the C ABI,
and a chain resumed from a checkpoint file.
"""

import ctypes
import json
import os
import subprocess
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_NERSC = os.path.join(ROOT, "oracle", "_ref", "ref_nersc")
TS = (4, 4, 4, 8)
DATE = b"Thu Jan  1 00:00:00 1970\n"


def _call(name, *args):
    from qlat_b200._lib import call
    return call(name, *args)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def write_host(path, links, ts, plaq=1.0, trace=0.0, date=DATE, **kw):
    from qlat_b200._lib import i32x4
    n = ctypes.c_int64()
    _call("qgb_nersc_write_host", str(path).encode(), _dp(links), i32x4(*ts), float(plaq), float(trace), None, None,
          None, date, float(kw.get("beta", 0.0)), int(kw.get("seq", 0)), ctypes.byref(n))
    return n.value


def read_host(path, ts):
    from qlat_b200._lib import i32x4
    out = np.zeros((int(np.prod(ts)), 4, 3, 3), dtype=np.complex128)
    c, n = ctypes.c_int32(), ctypes.c_int64()
    _call("qgb_nersc_read_host", str(path).encode(), _dp(out), i32x4(*ts), ctypes.byref(c), ctypes.byref(n))
    return out, c.value, n.value


def split(path):
    raw = open(path, "rb").read()
    k = raw.index(b"END_HEADER\n") + len(b"END_HEADER\n")
    return raw[:k], raw[k:]


def test_host_round_trip_and_checksums(tmp_path):
    ts = (2, 2, 2, 4)
    rng = np.random.default_rng(1)
    a = rng.standard_normal((32, 4, 3, 3)) + 1j * rng.standard_normal((32, 4, 3, 3))
    p = tmp_path / "a.lat"
    nbytes = write_host(p, a, ts, plaq=0.5, trace=0.25, beta=6.0, seq=7)
    assert nbytes == 32 * 4 * 12 * 8
    header, data = split(p)
    assert len(data) == nbytes
    # data: rows 0-1 of each link, IEEE64BIG
    two = a[:, :, :2, :].reshape(-1).view(np.float64)
    assert data == two.astype(">f8").tobytes()
    h = header.decode()
    assert f"CRC32HASH = {zlib.crc32(data):08x}\n" in h
    assert f"CHECKSUM = {int(two.view(np.uint32).sum(dtype=np.uint64)) & 0xffffffff:08x}\n" in h
    assert "BETA = 6.000000000000\nSEQUENCE_NUMBER = 7\nFLOATING_POINT = IEEE64BIG\nEND_HEADER\n" in h
    from qlat_b200 import read_gauge_field_header
    info = read_gauge_field_header(str(p))
    assert info["total_site"] == list(ts) and info["n_rows"] == 2 and info["big_endian"] == 1
    b, checks, n = read_host(p, ts)
    assert checks == 7 and n == nbytes  # CRC ok, simple checksum ok, two-row
    assert np.array_equal(b[:, :, :2, :], a[:, :, :2, :])
    assert not b[:, :, 2, :].any()
    # a damaged byte is reported through the check bits, not as an error
    raw = bytearray(open(p, "rb").read())
    raw[-3] ^= 0x10
    open(p, "wb").write(bytes(raw))
    _, checks, _ = read_host(p, ts)
    assert checks & 3 == 0


def test_host_rejects_other_lattice_and_non_nersc(tmp_path):
    from qlat_b200 import QlatB200Error
    a = np.zeros((16, 4, 3, 3), dtype=np.complex128)
    p = tmp_path / "a.lat"
    write_host(p, a, (2, 2, 2, 2))
    with pytest.raises(QlatB200Error):
        read_host(p, (2, 2, 2, 4))
    q = tmp_path / "b.lat"
    q.write_bytes(b"not a gauge file\n")
    with pytest.raises(QlatB200Error) as e:
        read_host(q, (2, 2, 2, 2))
    assert e.value.code == 9


def _ref(*args, cwd):
    env = dict(os.environ, q_verbose="-1", OMP_NUM_THREADS="2")
    r = subprocess.run([REF_NERSC, *map(str, args)], capture_output=True, text=True, env=env, cwd=cwd, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])


needs_ref = pytest.mark.skipif(not os.path.exists(REF_NERSC), reason="oracle/_ref/ref_nersc not built")


@needs_ref
def test_same_file_as_the_reference(tmp_path, oracle):
    """The reference saves a hot start; the library's writer, given the same links
    (the oracle's bit-identical hot start) and the reference file's date,
    writes the same bytes; and reads the reference's file back exactly."""
    ref_path = tmp_path / "ref.lat"
    r = _ref("save", ref_path, *TS, 0.5, 2, "nersc-test", cwd=tmp_path)
    links = oracle.new_field(TS)
    oracle.gf_set_rand(links, TS, oracle.RngState("nersc-test").split("gf-init"), 0.5, 2)
    assert abs(oracle.gf_avg_plaq(links, TS) - r["plaq"]) < 1e-14
    ref_header, ref_data = split(ref_path)
    date = [ln for ln in ref_header.decode().splitlines(True) if ln.startswith("ARCHIVE_DATE = ")][0]
    ours = tmp_path / "ours.lat"
    write_host(ours, links, TS, plaq=r["plaq"], trace=r["link_trace"], date=date[len("ARCHIVE_DATE = "):].encode())
    our_header, our_data = split(ours)
    assert our_data == ref_data
    assert our_header == ref_header
    got, checks, _ = read_host(ref_path, TS)
    assert checks == 7
    assert np.array_equal(got[:, :, :2, :], links[:, :, :2, :])


@needs_ref
def test_reference_reads_our_file(tmp_path, oracle):
    links = oracle.new_field(TS)
    oracle.gf_set_rand(links, TS, oracle.RngState("nersc-test-2").split("gf-init"), 0.3, 1)
    p = tmp_path / "ours.lat"
    write_host(p, links, TS, plaq=oracle.gf_avg_plaq(links, TS))
    r = _ref("load", p, tmp_path / "links.bin", cwd=tmp_path)
    got = np.fromfile(tmp_path / "links.bin", dtype=np.complex128).reshape(links.shape)
    # the reference re-unitarizes the two stored rows (qcd.h:244-246)
    assert np.abs(got - links).max() < 1e-14
    assert abs(r["plaq"] - oracle.gf_avg_plaq(links, TS)) < 1e-13


@pytest.mark.gpu
def test_gpu_save_load_round_trip(q, tmp_path):
    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(q.RngState("nersc-gpu").split("gf-init"), 0.5, 2)
    p = tmp_path / "gpu.lat"
    n = gf.save(str(p), beta=2.13, sequence_num=12)
    assert n == 4 * 4 * 4 * 8 * 4 * 12 * 8
    info = q.read_gauge_field_header(str(p))
    assert abs(info["plaq"] - gf.plaq()) < 1e-11
    g2 = q.GaugeField()
    assert g2.load(str(p)) == n
    assert tuple(g2.geo.total_site) == TS
    assert np.abs(np.asarray(g2) - np.asarray(gf)).max() < 1e-14
    assert abs(g2.plaq() - gf.plaq()) < 1e-14


@pytest.mark.gpu
@needs_ref
def test_gpu_loads_reference_file(q, oracle, tmp_path):
    ref_path = tmp_path / "ref.lat"
    _ref("save", ref_path, *TS, 0.5, 2, "nersc-test", cwd=tmp_path)
    links = oracle.new_field(TS)
    oracle.gf_set_rand(links, TS, oracle.RngState("nersc-test").split("gf-init"), 0.5, 2)
    gf = q.GaugeField()
    gf.load(str(ref_path))
    assert np.abs(np.asarray(gf) - links).max() < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_chain_resumes_from_checkpoint(q, tmp_path, precision):
    """The checkpoint / resume pattern of examples-py/hmc-pure-gauge.py:67-79:
    a chain saved after 3 of 6 trajectories, read back into a fresh field and
    continued with the same counter-based RNG splits, makes the same
    accept / reject decisions as the uninterrupted chain, with plaquettes
    within 1e-10 and delta_h within 1e-8 (the file keeps two rows of each
    link; the third is rebuilt on reading, as qcd.h:244-246 does)."""
    ga = q.GaugeAction(2.13, -0.331)
    rs = q.RngState("resume")

    def chain(gf, trajs):
        rows = []
        for t in trajs:
            flag, dh = q.run_hmc_pure_gauge(gf, ga, t, rs.split("hmc"), n_step=6, is_always_accept=t <= 2,
                                            precision=precision)
            rows.append((bool(flag), dh, gf.plaq()))
        return rows

    gf = q.GaugeField(q.Geometry(TS))
    gf.set_rand(rs.split("gf-init"), 0.1, 2)
    g_ref = gf.copy()
    full = chain(g_ref, range(1, 7))
    first = chain(gf, range(1, 4))
    p = tmp_path / f"ckpoint_lat.{precision}.3"
    gf.save(str(p), beta=2.13, sequence_num=3)
    g2 = q.GaugeField()
    g2.load(str(p))
    rest = chain(g2, range(4, 7))
    for (f, dh, pl), (rf, rdh, rpl) in zip(first + rest, full):
        assert f == rf
        assert abs(dh - rdh) < 1e-8
        assert abs(pl - rpl) < 1e-10
