"""The C++ drop-in layer (phobic-gpu_b200/cpp): its encoders against the
reference's, byte for byte, and a reference-style C++ program built against it.

The encoders are header-only host code; the harness tests/cpp/encode_check.cpp
exposes them behind the same arguments as the reference wrapper's ref_encode."""
import ctypes as C
import hashlib
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O

ROOT = Path(__file__).resolve().parents[1]
NAMES = {0: "interleaved_compact", 1: "interleaved_dictionary", 2: "interleaved_rice", 3: "mono_compact",
         4: "mono_dictionary", 5: "dual_rice_compact", 6: "interleaved_elias_fano", 7: "interleaved_sdc",
         8: "mono_rice"}


@pytest.fixture(scope="module")
def mine(tmp_path_factory):
    out = tmp_path_factory.mktemp("cpp") / "libencode_check.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'phobic-gpu_b200' / 'cpp'}", "-o", str(out), str(ROOT / "tests/cpp/encode_check.cpp")],
                   check=True)
    lib = C.CDLL(str(out))
    lib.mine_encode.restype = C.c_size_t
    lib.mine_encode.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_uint32,
                                C.c_float, C.c_void_p, C.c_size_t, C.POINTER(C.c_double)]
    lib.mine_query.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_uint32, C.c_void_p,
                               C.c_uint64, C.c_void_p]
    lib.mine_roundtrip.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_uint32,
                                   C.c_void_p, C.c_uint64]
    lib.mine_layout_and_save.argtypes = [C.c_char_p, C.c_double, C.c_void_p, C.c_uint64]
    return lib


def encode(lib, kind, off_kind, r, lam, P):
    bpk = C.c_double()
    size = lib.mine_encode(kind, off_kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data, r["partitions"], lam, P,
                           0.5, None, 0, C.byref(bpk))
    buf = np.zeros(size, np.uint8)
    lib.mine_encode(kind, off_kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data, r["partitions"], lam, P, 0.5,
                    buf.ctypes.data, size, C.byref(bpk))
    return buf, bpk.value


@pytest.mark.parametrize("case,seed,n,lam,P", [("C1_u64_seed1_n1e6_l5_P2048", 1, 1_000_000, 5.0, 2048),
                                               ("C2_sample_u64_seed2_n2e6_l7_P2500", 2, 2_000_000, 7.0, 2500)])
def test_encoded_bytes_match_reference_golden(mine, golden, case, seed, n, lam, P):
    B, f = O.config(lam, P)
    r = O.build(O.hash_keys(O.splitmix64(seed, n), "u64"), P, B, f)
    want = golden["builds"][case]["encoded"]
    for kind, name in NAMES.items():
        for off_kind, off_name in ((0, "diff"), (1, "direct")):
            buf, bpk = encode(mine, kind, off_kind, r, lam, P)
            w = want[f"{name}+{off_name}"]
            assert len(buf) == w["bytes"], name
            assert hashlib.sha256(buf.tobytes()).hexdigest() == w["sha256"], (name, off_name)
            assert abs(bpk - w["bits_per_key"]) < 1e-6


@pytest.mark.skipif(not O.ref_available(), reason="reference wrapper not built")
@pytest.mark.parametrize("n,lam,P,seed", [(50_000, 3.0, 1024, 3), (5, 5.0, 2048, 4), (30_000, 9.0, 4096, 5)])
def test_encoded_bytes_match_reference_encoders(mine, n, lam, P, seed):
    B, f = O.config(lam, P)
    r = O.build(O.hash_keys(O.splitmix64(seed, n), "u64"), P, B, f)
    for kind in NAMES:
        for off_kind in (0, 1):
            buf, _ = encode(mine, kind, off_kind, r, lam, P)
            bpk = C.c_double()
            size = O.ref().ref_encode(kind, off_kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data,
                                      r["partitions"], lam, P, 0.5, None, 0, C.byref(bpk))
            ref = np.zeros(size, np.uint8)
            O.ref().ref_encode(kind, off_kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data, r["partitions"], lam,
                               P, 0.5, ref.ctypes.data, size, C.byref(bpk))
            assert np.array_equal(buf, ref), (kind, off_kind)


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 5, 6, 7, 8])
def test_query_through_every_encoder_is_a_bijection(mine, kind):
    n, lam, P = 80_000, 6.0, 2048
    keys = O.splitmix64(12, n)
    B, f = O.config(lam, P)
    r = O.build(O.hash_keys(keys, "u64"), P, B, f)
    pos = np.zeros(n, np.uint32)
    assert mine.mine_query(kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data, r["partitions"], lam, P,
                           keys.ctypes.data, n, pos.ctypes.data) == 0
    assert O.is_bijection(pos)


@pytest.mark.gpu
def test_reference_style_program_on_the_gpu(phobic, golden, tmp_path):
    exe = tmp_path / "example_b200"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'phobic-gpu_b200' / 'cpp'}", "-o", str(exe), str(ROOT / "tests/cpp/example_b200.cpp"),
                    f"-L{phobic.LIB_PATH.parent}", "-lphobic_b200", f"-Wl,-rpath,{phobic.LIB_PATH.parent}"], check=True)
    dump = tmp_path / "c1.bin"
    out = subprocess.run([str(exe), str(dump)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "OK" in out.stdout
    want = golden["builds"]["C1_u64_seed1_n1e6_l5_P2048"]["encoded"]["interleaved_compact+diff"]
    assert hashlib.sha256(dump.read_bytes()).hexdigest() == want["sha256"]


def test_abi_encode_matches_reference_golden(phobic, golden):
    """phobic_encode (C ABI, host only) yields the reference encoders' bytes."""
    B, f = O.config(7.0, 2500)
    r = O.build(O.hash_keys(O.splitmix64(2, 2_000_000), "u64"), 2500, B, f)
    cfg = phobic.MPHFconfig(7.0, 2500)
    built = phobic.BuildResult(r["pilots"], r["offsets"], r["partitions"], B)
    want = golden["builds"]["C2_sample_u64_seed2_n2e6_l7_P2500"]["encoded"]
    for name in NAMES.values():
        for off_name in ("diff", "direct"):
            data, bpk = phobic.encode(built, cfg, name, off_name)
            assert hashlib.sha256(data).hexdigest() == want[f"{name}+{off_name}"]["sha256"], (name, off_name)


@pytest.mark.parametrize("kind", [0, 1, 3])
@pytest.mark.parametrize("off_kind", [0, 1])
@pytest.mark.parametrize("n", [1, 2049, 60_000])
def test_load_encoded_bytes_round_trip(mine, kind, off_kind, n):
    """MPHF::loadEncoded (the state setData leaves, read back from the encoders' bytes,
    as MPHFbuilder does with the bytes of phobic_encode_gpu) answers every key like
    the function it was saved from, re-serialises to the same bytes, and rejects a
    truncated byte string."""
    lam, P = 6.0, 2048
    keys = O.splitmix64(40 + n, n)
    B, f = O.config(lam, P)
    r = O.build(O.hash_keys(keys, "u64"), P, B, f)
    rc = mine.mine_roundtrip(kind, off_kind, r["pilots"].ctypes.data, r["offsets"].ctypes.data, r["partitions"],
                             lam, P, keys.ctypes.data, n)
    assert rc == 0, rc


@pytest.mark.parametrize("n,lam,P", [(1, 5.0, 2048), (70_000, 7.0, 2500)])
def test_pilot_layout_file_and_mphf_save_load(mine, phobic, tmp_path, n, lam, P):
    """A build's pilot layout written by the Python binding is read by the C++
    layer's loadPilotLayout, encoded, saved with MPHF::save and loaded with
    MPHF::load: every key maps to the same slot, the reloaded function saves the
    same bytes, truncated bytes are rejected; the Python reader returns the arrays."""
    keys = O.splitmix64(77 + n, n)
    B, f = O.config(lam, P)
    r = O.build(O.hash_keys(keys, "u64"), P, B, f)
    cfg = phobic.MPHFconfig(lam, P)
    built = phobic.BuildResult(r["pilots"], r["offsets"], r["partitions"], B)
    path = tmp_path / "layout.bin"
    phobic.save_layout(path, built, cfg)
    back, psize = phobic.load_layout(path)
    assert psize == P and back.partitions == r["partitions"] and back.buckets == B
    assert (back.pilots == r["pilots"]).all() and (back.partition_offsets == r["offsets"]).all()
    assert mine.mine_layout_and_save(str(path).encode(), lam, keys.ctypes.data, n) == 0
    data = path.read_bytes()
    path.write_bytes(data[:-4])
    with pytest.raises(ValueError):
        phobic.load_layout(path)
    assert mine.mine_layout_and_save(str(path).encode(), lam, keys.ctypes.data, n) == 2
