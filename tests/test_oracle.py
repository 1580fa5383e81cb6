"""The oracle against the golden fixtures (made from the reference's own host
code and the xxhash module), and its internal cross-checks.  CPU only."""
import hashlib
import json

import numpy as np
import pytest

import keygen
import oracle_lib as O

GOLDEN_DIR = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def det_bytes(seed, n):
    return O.splitmix64(seed, (n + 7) // 8 + 1).tobytes()[:n]


def test_xxh3_known_answers():
    vec = json.loads((GOLDEN_DIR / "xxh3_vectors.json").read_text())["vectors"]
    assert len(vec) > 260
    for v in vec:
        b = det_bytes(v["seed"], v["len"])
        assert f"{O.xxh3_128(b):032x}" == v["xxh3_128"], v["len"]


def test_xxh3_against_xxhash_module():
    xxhash = pytest.importorskip("xxhash")
    rng = np.random.default_rng(5)
    for L in list(range(0, 260)) + [777, 1024, 3000]:
        b = rng.integers(0, 256, L, dtype=np.uint8).tobytes()
        assert O.xxh3_128(b) == xxhash.xxh3_128_intdigest(b)


def test_fulcrums_match_reference_config(golden, golden_fulcrums):
    for name, meta in golden["fulcrums"].items():
        B, f = O.config(meta["lambda"], meta["P"], meta["bucketer"], bool(meta["bucketer_ctor"]))
        assert B == meta["buckets"], name
        assert (f == golden_fulcrums[name]).all(), name
        assert O.orc().orc_max_partition_size(meta["P"]) == 32 * (meta["partition_max_size"] // 32)


def test_known_answer_c2_config():
    B, f = O.config(7.0, 2500)
    assert (B, int(f[1]), int(f[2047])) == (358, 323, 23461888)


@pytest.mark.parametrize("name,kind", [("c1_u64_1e6", "u64"), ("pairs_4096", "pairs"), ("keys16_4096", "keys16")])
def test_hash_matches_reference_hasher(golden, name, kind):
    g = golden["hashes"][name]
    if kind == "u64":
        keys = O.splitmix64(g["seed"], g["n"])
    elif kind == "pairs":
        keys = O.splitmix64(g["seed"], 2 * g["n"]).reshape(g["n"], 2)
    else:
        keys = O.splitmix64(g["seed"], 2 * g["n"]).view(np.uint32).reshape(g["n"], 4)
    assert sha(O.hash_keys(keys, kind)) == g["keys4_sha256"]


def test_string_hash_matches_reference_hasher(golden):
    g = golden["hashes"]["strings_c3_2e4"]
    d, o = keygen.strings(g["seed"], g["n"])
    assert sha(d) == g["bytes_sha256"] and sha(o) == g["offsets_sha256"]
    assert sha(O.hash_keys((d, o), "strings")) == g["keys4_sha256"]
    g = golden["hashes"]["strings_len0_299"]
    dd = np.frombuffer(det_bytes(77, 300 * 301 // 2), np.uint8).copy()
    do = np.zeros(301, np.uint64)
    np.cumsum(np.arange(300, dtype=np.uint64), out=do[1:])
    assert sha(O.hash_keys((dd, do), "strings")) == g["keys4_sha256"]
    g = golden["hashes"]["example_strings_1e5"]
    ex = [str(i).encode() for i in range(100000)]
    eo = np.zeros(len(ex) + 1, np.uint64)
    np.cumsum([len(e) for e in ex], out=eo[1:])
    assert sha(O.hash_keys((np.frombuffer(b"".join(ex), np.uint8).copy(), eo), "strings")) == g["keys4_sha256"]


def _check_build(rec, keys4):
    B, f = O.config(rec["lambda"], rec["P"])
    assert B == rec["buckets"]
    r = O.build(keys4, rec["P"], B, f, intermediates=True)
    assert r["status"] == 0
    assert sha(keys4) == rec["keys_sha256"]
    for k in ("pilots", "offsets", "bucket_sizes", "histo", "perm", "sorted_lowers"):
        assert sha(r[k]) == rec[f"{k}_sha256"], k
    pos = O.query(keys4, r["partitions"], B, f, r["pilots"], r["offsets"])
    assert O.is_bijection(pos)
    return r


@pytest.mark.parametrize("n", [1, 2, 31, 2047, 2049, 10000])
def test_small_builds_match_golden(golden, small_builds, n):
    rec = golden["builds"][f"u64_seed1_n{n}_l5_P2048"]
    assert rec["reference_query_bijection"]
    r = _check_build(rec, O.hash_keys(O.splitmix64(1, n), "u64"))
    assert (r["pilots"] == small_builds[f"n{n}_pilots"]).all()
    assert (r["offsets"] == small_builds[f"n{n}_offsets"]).all()


def test_c1_build_matches_golden(golden):
    rec = golden["builds"]["C1_u64_seed1_n1e6_l5_P2048"]
    _check_build(rec, O.hash_keys(O.splitmix64(1, 1_000_000), "u64"))


def test_c2_sample_build_matches_golden(golden):
    rec = golden["builds"]["C2_sample_u64_seed2_n2e6_l7_P2500"]
    _check_build(rec, O.hash_keys(O.splitmix64(2, 2_000_000), "u64"))


def test_c3_sample_build_matches_golden(golden):
    rec = golden["builds"]["C3_sample_strings_seed3_n2e4_l6_P2048"]
    _check_build(rec, O.hash_keys(keygen.strings(3, 20000), "strings"))


@pytest.mark.parametrize("n,lam,P", [(5000, 5.0, 2048), (20000, 7.0, 2500), (3000, 2.0, 256), (1500, 3.0, 128)])
def test_naive_offset_scan_equals_windowed(n, lam, P):
    keys4 = O.hash_keys(O.splitmix64(9, n), "u64")
    B, f = O.config(lam, P)
    a = O.build(keys4, P, B, f, naive=False)
    b = O.build(keys4, P, B, f, naive=True)
    assert a["status"] == b["status"] == 0
    assert (a["pilots"] == b["pilots"]).all()


def test_sorted_order_is_stable_within_buckets():
    n = 5000
    keys4 = O.hash_keys(O.splitmix64(4, n), "u64")
    B, f = O.config(5.0, 2048)
    r = O.build(keys4, 2048, B, f, intermediates=True)
    # sorted lowers grouped by partition: each partition's multiset equals its keys' lowers
    parts = r["partitions"]
    pid = ((keys4[:, 0].astype(np.uint64) * parts) >> 32).astype(np.int64)
    for p in range(parts):
        a, b = r["offsets"][p], r["offsets"][p + 1]
        got = r["sorted_lowers"][a:b]
        want = keys4[pid == p][:, 2:4]
        assert sorted(map(tuple, got)) == sorted(map(tuple, want))


def test_error_partition_overflow():
    keys4 = O.hash_keys(O.splitmix64(1, 4000), "u64")
    keys4[:, 0] = 7  # every key in partition 0
    B, f = O.config(5.0, 2048)
    r = O.build(keys4, 2048, B, f)
    assert r["status"] == 4 and r["stats"].err_partition == 0


def test_error_bucket_overflow():
    keys4 = O.hash_keys(O.splitmix64(1, 3000), "u64")
    keys4[:300, 1] = 5  # 300 keys in one bucket of partition-of-their-own
    keys4[:300, 0] = keys4[0, 0]
    B, f = O.config(5.0, 2048)
    r = O.build(keys4, 2048, B, f)
    assert r["status"] == 3


def test_error_duplicate_keys():
    keys4 = O.hash_keys(O.splitmix64(1, 3000), "u64")
    keys4[1] = keys4[0]
    B, f = O.config(5.0, 2048)
    r = O.build(keys4, 2048, B, f)
    assert r["status"] == 8


def test_error_search_limit():
    keys4 = O.hash_keys(O.splitmix64(1, 4000), "u64")
    B, f = O.config(5.0, 2048)
    r = O.build(keys4, 2048, B, f, max_k=1)
    assert r["status"] == 5


def test_error_invalid_bucket_from_fulcrums():
    keys4 = O.hash_keys(O.splitmix64(1, 100), "u64")
    B, f = O.config(5.0, 2048)
    f = f.copy()
    f[1000:2047] = (B + 5) << 16
    r = O.build(keys4, 2048, B, f)
    assert r["status"] == 1


def test_empty_input():
    B, f = O.config(5.0, 2048)
    r = O.build(np.zeros((0, 4), np.uint32), 2048, B, f)
    assert r["status"] == 0 and r["partitions"] == 0 and list(r["offsets"]) == [0]
