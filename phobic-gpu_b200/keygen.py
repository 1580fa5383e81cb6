"""Seeded synthetic key sets for the build workloads.

No public dataset is involved: every workload is generated from a seed.
  * u64 keys: the splitmix64 stream (Vigna's public generator; state starts at the
    seed, output i is the finalizer of seed + (i+1) * 0x9E3779B97F4A7C15).  It is
    a bijection of the counter, so the keys are unique.
  * strings: lengths uniform in [8, 64], bytes uniform over printable ASCII
    (0x20..0x7E), duplicates replaced (only short strings can collide); a device
    generator (strings_cuda) of the same distribution serves the request stream.
  * batched sets: sizes log-uniform in [lo, hi].
  * served stream: Poisson arrivals, sizes log-uniform, a u64/string mix.
"""
from __future__ import annotations

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int, start: int = 0, chunk: int = 1 << 24) -> np.ndarray:
    out = np.empty(n, np.uint64)
    with np.errstate(over="ignore"):
        for lo in range(0, n, chunk):
            hi = min(n, lo + chunk)
            z = np.arange(start + lo + 1, start + hi + 1, dtype=np.uint64) * GAMMA + np.uint64(seed)
            z = (z ^ (z >> np.uint64(30))) * M1
            z = (z ^ (z >> np.uint64(27))) * M2
            out[lo:hi] = z ^ (z >> np.uint64(31))
    return out


def strings(seed: int, n: int, min_len: int = 8, max_len: int = 64) -> tuple[np.ndarray, np.ndarray]:
    """(bytes uint8[total], offsets uint64[n+1]) of n distinct printable strings."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(min_len, max_len + 1, n, dtype=np.int64)
    offs = np.zeros(n + 1, np.uint64)
    np.cumsum(lens, out=offs[1:])
    data = rng.integers(0x20, 0x7F, int(offs[-1]), dtype=np.uint8)
    # Strings of 8..10 bytes are the only ones with a non-negligible collision
    # chance at these sizes; replace any repeat among them.
    for L in range(min_len, min(max_len, 10) + 1):
        idx = np.nonzero(lens == L)[0]
        while idx.size:
            rows = data[offs[idx].astype(np.int64)[:, None] + np.arange(L)]
            _, first = np.unique(rows, axis=0, return_index=True)
            dup = np.setdiff1d(np.arange(idx.size), first)
            if not dup.size:
                break
            for d in idx[dup]:
                s = int(offs[d])
                data[s:s + L] = rng.integers(0x20, 0x7F, L, dtype=np.uint8)
    return data, offs


def set_sizes(seed: int, count: int, lo: int, hi: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)


def request_stream(seed: int, rate: float, seconds: float, lo: int, hi: int, string_frac: float):
    """Arrival times (s), sizes and kinds ('u64' / 'strings') of a Poisson request stream."""
    rng = np.random.default_rng(seed)
    t, times = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        times.append(t)
    k = len(times)
    sizes = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), k))).astype(np.int64)
    kinds = np.where(rng.uniform(size=k) < string_frac, "strings", "u64")
    return np.array(times), sizes, kinds


def splitmix64_cuda(seed: int, n: int, start: int = 0, device: str = "cuda"):
    """The splitmix64 stream generated on the device (torch int64 with wrapping
    arithmetic; logical shifts emulated by masking the arithmetic ones)."""
    import torch

    def s64(v: int) -> int:
        return v - (1 << 64) if v >= 1 << 63 else v

    def lsr(x, s: int):
        return (x >> s) & ((1 << (64 - s)) - 1)

    z = torch.arange(start + 1, start + n + 1, dtype=torch.int64, device=device)
    z.mul_(s64(int(GAMMA))).add_(s64(seed % (1 << 64)))
    z = (z ^ lsr(z, 30)).mul_(s64(int(M1)))
    z = (z ^ lsr(z, 27)).mul_(s64(int(M2)))
    return z ^ lsr(z, 31)


def strings_cuda(seed: int, n: int, min_len: int = 8, max_len: int = 64, device: str = "cuda"):
    """(bytes uint8[total], offsets int64[n+1]) of n strings generated on the device:
    lengths uniform in [min_len, max_len] and bytes uniform over printable ASCII, both
    from splitmix64 streams (lengths from seed, bytes from seed ^ 0x5bd1e995, four bytes
    per output word: 0x20 + (16-bit piece * 95 >> 16)).  Not deduplicated: two strings
    of 8 printable bytes or more coincide with probability below 1e-4 at 5e7 strings."""
    import torch

    span = max_len - min_len + 1
    lens = (splitmix64_cuda(seed, n, device=device) & 0x7FFFFFFF) % span + min_len
    offs = torch.zeros(n + 1, dtype=torch.int64, device=device)
    torch.cumsum(lens, 0, out=offs[1:])
    del lens
    total = int(offs[-1])
    data = torch.empty(total, dtype=torch.uint8, device=device)
    words = (total + 3) // 4
    chunk = 1 << 26
    for w0 in range(0, words, chunk):
        w1 = min(words, w0 + chunk)
        z = splitmix64_cuda(seed ^ 0x5BD1E995, w1 - w0, start=w0, device=device)
        pieces = z.view(torch.int16).to(torch.int32) & 0xFFFF  # four 16-bit pieces per word
        b = (0x20 + ((pieces * 95) >> 16)).to(torch.uint8)
        lo, hi = 4 * w0, min(total, 4 * w1)
        data[lo:hi] = b[: hi - lo]
    return data, offs
