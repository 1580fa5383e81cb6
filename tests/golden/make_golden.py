"""Generates the golden fixtures in tests/golden/ (run in a container that has
the reference checkout, so that oracle/_ref/libphobic_ref.so can be built).

Sources of truth, in order:
  * the `xxhash` Python module (libxxhash 0.8.2) for XXH3-128 known answers;
  * the reference's own host code compiled in place (oracle/_ref): xxhash::hash
    for u64 / pair / Key / std::string keys, MPHFconfig fulcrum tables, the
    encoders, and MPHF::operator() for the bijection check;
  * the oracle restatement of the shaders (oracle/build/liborc.so) for bucket
    sizes, histograms, permutations, sorted order, partition offsets and pilots.
    Its pilots are accepted only when the reference's own query maps every key
    to a distinct slot in [0, n).

    python tests/golden/make_golden.py              # everything
    python tests/golden/make_golden.py --full-only  # only the full-size builds (C2, C3, C4)

The full-size builds pin the workloads at the sizes they are quoted on: all 10^8 keys
of C2, all 5*10^7 strings of C3 and every set of one C4 batch (4096 sets).  Only
SHA-256 digests are stored; the GPU tests compare element by element with the
oracle and then with these digests.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
import oracle_lib as O  # noqa: E402

import ctypes as C  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def det_bytes(seed: int, n: int) -> bytes:
    """Deterministic test bytes from the splitmix64 stream."""
    w = O.splitmix64(seed, (n + 7) // 8 + 1)
    return w.tobytes()[:n]


def xxh3_vectors() -> dict:
    import xxhash

    lens = list(range(0, 257)) + [300, 511, 512, 513, 1023, 1024, 1025, 2048, 4095, 5000]
    out = []
    for L in lens:
        b = det_bytes(1000 + L, L)
        out.append({"len": L, "seed": 1000 + L, "xxh3_128": f"{xxhash.xxh3_128_intdigest(b):032x}"})
    return {"source": f"python xxhash {xxhash.VERSION} (libxxhash {xxhash.XXHASH_VERSION})", "vectors": out}


CONFIGS = [  # (name, lambda, P)
    ("C1", 5.0, 2048),
    ("C2", 7.0, 2500),
    ("C3", 6.0, 2048),
    ("C5", 7.0, 2048),
    ("example", 4.5, 2500),
    ("benchmark", 7.5, 2048),
]


def fulcrum_tables() -> dict:
    tables = {}
    for name, lam, P in CONFIGS:
        for bucketer in (0, 1, 2):
            for ctor in (0, 1):
                if ctor == 0 and bucketer != 0:
                    continue  # the default constructor always uses OptBucketer
                f = np.zeros(2048, np.uint32)
                mx = C.c_uint32()
                B = O.ref().ref_config(lam, P, bucketer, ctor, f.ctypes.data, C.byref(mx))
                tables[f"{name}_b{bucketer}_c{ctor}"] = {
                    "lambda": lam, "P": P, "bucketer": bucketer, "bucketer_ctor": ctor, "buckets": int(B),
                    "partition_max_size": int(mx.value), "fulcrums": f,
                }
    return tables


def ref_keys(kind: str, keys) -> np.ndarray:
    if kind == "u64":
        n = len(keys)
        out = np.zeros((n, 4), np.uint32)
        O.ref().ref_hash_u64(keys.ctypes.data, n, out.ctypes.data)
    elif kind == "pairs":
        n = keys.shape[0]
        out = np.zeros((n, 4), np.uint32)
        O.ref().ref_hash_pairs(keys.ctypes.data, n, out.ctypes.data)
    elif kind == "keys16":
        n = keys.shape[0]
        out = np.zeros((n, 4), np.uint32)
        O.ref().ref_hash_keys16(keys.ctypes.data, n, out.ctypes.data)
    else:
        data, offs = keys
        n = len(offs) - 1
        out = np.zeros((n, 4), np.uint32)
        O.ref().ref_hash_strings(data.ctypes.data if data.size else None, offs.ctypes.data, n, out.ctypes.data)
    return out


def ref_bijection(pilots, offsets, parts, lam, P, keys) -> bool:
    n = len(keys)
    pos = np.zeros(max(n, 1), np.uint32)
    O.ref().ref_query_u64(pilots.ctypes.data, offsets.ctypes.data, parts, lam, P, keys.ctypes.data, n,
                          pos.ctypes.data)
    return O.is_bijection(pos[:n])


def encoded(pilots, offsets, parts, lam, P) -> dict:
    out = {}
    names = {0: "interleaved_compact", 1: "interleaved_dictionary", 2: "interleaved_rice", 3: "mono_compact",
             4: "mono_dictionary", 5: "dual_rice_compact", 6: "interleaved_elias_fano", 7: "interleaved_sdc",
             8: "mono_rice"}
    for kind, name in names.items():
        for off_kind, off_name in ((0, "diff"), (1, "direct")):
            bpk = C.c_double()
            size = O.ref().ref_encode(kind, off_kind, pilots.ctypes.data, offsets.ctypes.data, parts, lam, P, 0.5,
                                      None, 0, C.byref(bpk))
            buf = np.zeros(size, np.uint8)
            O.ref().ref_encode(kind, off_kind, pilots.ctypes.data, offsets.ctypes.data, parts, lam, P, 0.5,
                               buf.ctypes.data, size, C.byref(bpk))
            out[f"{name}+{off_name}"] = {"bytes": int(size), "sha256": hashlib.sha256(buf.tobytes()).hexdigest(),
                                          "bits_per_key": float(bpk.value)}
    return out


def build_case(name, keys4, lam, P, keys_u64=None):
    B, f = O.config(lam, P)
    r = O.build(keys4, P, B, f, intermediates=True)
    assert r["status"] == 0, (name, r["status"])
    parts = r["partitions"]
    pos = O.query(keys4, parts, B, f, r["pilots"], r["offsets"])
    assert O.is_bijection(pos), name
    rec = {"lambda": lam, "P": P, "buckets": B, "partitions": parts, "n": int(keys4.shape[0]),
           "keys_sha256": sha(keys4), "pilots_sha256": sha(r["pilots"]), "offsets_sha256": sha(r["offsets"]),
           "bucket_sizes_sha256": sha(r["bucket_sizes"]), "histo_sha256": sha(r["histo"]),
           "perm_sha256": sha(r["perm"]), "sorted_lowers_sha256": sha(r["sorted_lowers"]),
           "max_bucket": int(r["stats"].max_bucket), "max_partition": int(r["stats"].max_partition),
           "max_k": int(r["stats"].max_k)}
    if keys_u64 is not None:
        rec["reference_query_bijection"] = ref_bijection(r["pilots"], r["offsets"], parts, lam, P, keys_u64)
        assert rec["reference_query_bijection"], name
    return rec, r


def full_size_builds() -> dict:
    """Oracle builds of the whole C2, C3 and C4 workloads (digests only)."""
    sys.path.insert(0, str(HERE.parents[1] / "phobic-gpu_b200"))
    import keygen

    out = {}
    c2 = O.splitmix64(2, 100_000_000)
    k4 = ref_keys("u64", c2)
    rec, r = build_case("C2", k4, 7.0, 2500, c2)
    out["C2_u64_seed2_n1e8_l7_P2500"] = {k: v for k, v in rec.items() if k not in (
        "bucket_sizes_sha256", "histo_sha256", "perm_sha256", "sorted_lowers_sha256")}
    del c2, k4, r
    sd, so = keygen.strings(3, 50_000_000)
    k4 = ref_keys("strings", (sd, so))
    rec, r = build_case("C3", k4, 6.0, 2048)
    rec.update({"bytes_sha256": sha(sd), "offsets_input_sha256": sha(so)})
    out["C3_strings_seed3_n5e7_l6_P2048"] = {k: v for k, v in rec.items() if k not in (
        "bucket_sizes_sha256", "histo_sha256", "perm_sha256", "sorted_lowers_sha256")}
    del sd, so, k4, r
    # C4: 4096 sets, one splitmix64(seed 4) stream split in order into sets of sizes
    # log-uniform in [1e3, 4*2^20]; digests over the sets' pilots (and offsets) in set order.
    sizes = keygen.set_sizes(4, 4096, 1000, 4 << 20)
    B, f = O.config(6.0, 2048)
    hp, ho = hashlib.sha256(), hashlib.sha256()
    start, max_k = 0, 0
    for n in sizes:
        keys = O.splitmix64(4, int(n), start=start)
        r = O.build(ref_keys("u64", keys), 2048, B, f)
        assert r["status"] == 0
        hp.update(np.ascontiguousarray(r["pilots"]).tobytes())
        ho.update(np.ascontiguousarray(r["offsets"]).tobytes())
        max_k = max(max_k, int(r["stats"].max_k))
        start += int(n)
    out["C4_batch_u64_seed4_4096sets_l6_P2048"] = {
        "lambda": 6.0, "P": 2048, "buckets": int(B), "sets": len(sizes), "total_keys": int(start),
        "pilots_concat_sha256": hp.hexdigest(), "offsets_concat_sha256": ho.hexdigest(), "max_k": max_k}
    return out


def main() -> None:
    if "--full-only" in sys.argv:
        g = json.loads((HERE / "golden.json").read_text())
        g["full_builds"] = full_size_builds()
        (HERE / "golden.json").write_text(json.dumps(g, indent=1))
        print("updated full_builds in golden.json")
        return
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libphobic_ref.so missing: make -C oracle (needs the reference checkout)")
    (HERE / "xxh3_vectors.json").write_text(json.dumps(xxh3_vectors(), indent=1))

    tables = fulcrum_tables()
    np.savez_compressed(HERE / "fulcrums.npz", **{k: v["fulcrums"] for k, v in tables.items()})
    meta = {k: {kk: vv for kk, vv in v.items() if kk != "fulcrums"} for k, v in tables.items()}

    # Keys through the reference's own hasher (hasher.hpp:30-67).
    hashes = {}
    u64 = O.splitmix64(1, 1_000_000)
    hashes["c1_u64_1e6"] = {"seed": 1, "n": 1_000_000, "keys4_sha256": sha(ref_keys("u64", u64))}
    pairs = O.splitmix64(11, 2 * 4096).reshape(4096, 2)
    hashes["pairs_4096"] = {"seed": 11, "n": 4096, "keys4_sha256": sha(ref_keys("pairs", pairs))}
    k16 = O.splitmix64(12, 2 * 4096).view(np.uint32).reshape(4096, 4)
    hashes["keys16_4096"] = {"seed": 12, "n": 4096, "keys4_sha256": sha(ref_keys("keys16", k16))}
    sys.path.insert(0, str(HERE.parents[1] / "phobic-gpu_b200"))
    import keygen

    sd, so = keygen.strings(3, 20000)
    hashes["strings_c3_2e4"] = {"seed": 3, "n": 20000, "bytes_sha256": sha(sd), "offsets_sha256": sha(so),
                                "keys4_sha256": sha(ref_keys("strings", (sd, so)))}
    dd = np.frombuffer(det_bytes(77, 300 * 301 // 2), np.uint8).copy()
    do = np.zeros(301, np.uint64)
    np.cumsum(np.arange(300, dtype=np.uint64), out=do[1:])
    hashes["strings_len0_299"] = {"seed": 77, "n": 300, "keys4_sha256": sha(ref_keys("strings", (dd, do)))}
    example = [str(i).encode() for i in range(100000)]  # example.cpp:23-28 keys
    eo = np.zeros(len(example) + 1, np.uint64)
    np.cumsum([len(e) for e in example], out=eo[1:])
    ed = np.frombuffer(b"".join(example), np.uint8).copy()
    hashes["example_strings_1e5"] = {"n": 100000, "keys4_sha256": sha(ref_keys("strings", (ed, eo)))}

    # Builds: oracle pipeline, accepted by the reference's query.
    builds = {}
    arrays = {}
    for n in (1, 2, 31, 2047, 2049, 10000):
        keys = O.splitmix64(1, n)
        k4 = ref_keys("u64", keys)
        rec, r = build_case(f"small_{n}", k4, 5.0, 2048, keys)
        builds[f"u64_seed1_n{n}_l5_P2048"] = rec
        arrays[f"n{n}_pilots"] = r["pilots"]
        arrays[f"n{n}_offsets"] = r["offsets"]
    k4 = ref_keys("u64", u64)
    rec, r = build_case("C1", k4, 5.0, 2048, u64)
    rec["encoded"] = encoded(r["pilots"], r["offsets"], r["partitions"], 5.0, 2048)
    builds["C1_u64_seed1_n1e6_l5_P2048"] = rec
    c2s = O.splitmix64(2, 2_000_000)
    rec, r = build_case("C2s", ref_keys("u64", c2s), 7.0, 2500, c2s)
    rec["encoded"] = encoded(r["pilots"], r["offsets"], r["partitions"], 7.0, 2500)
    builds["C2_sample_u64_seed2_n2e6_l7_P2500"] = rec
    rec, r = build_case("C3s", ref_keys("strings", (sd, so)), 6.0, 2048)
    builds["C3_sample_strings_seed3_n2e4_l6_P2048"] = rec

    np.savez_compressed(HERE / "small_builds.npz", **arrays)
    full = full_size_builds()
    (HERE / "golden.json").write_text(json.dumps({"fulcrums": meta, "hashes": hashes, "builds": builds,
                                                  "full_builds": full}, indent=1))
    print("wrote", [p.name for p in HERE.iterdir()])


if __name__ == "__main__":
    main()
