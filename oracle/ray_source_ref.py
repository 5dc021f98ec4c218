"""Test infrastructure (the oracle of the ray source's shuffle): the keyed permutation of
cpx_ray_source in numpy -- SplitMix64 round keys from the seed, a 4-round Feistel network with
MurmurHash3's 32-bit finaliser as the round function on the next even power of two >= n, cycle
walking back below n.  No reference counterpart: the reference shuffles on the host with rand()
(ShuffleRank, SparseVolumeRadianceField/Utils.cu:488-506); only the rays of each sample are the
reference's, which the GPU tests check separately."""
import numpy as np

M32 = np.uint64(0xFFFFFFFF)


def splitmix64_keys(seed: int, count: int = 4):
    x = int(seed) & 0xFFFFFFFFFFFFFFFF
    out = []
    for _ in range(count):
        x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        out.append(z & 0xFFFFFFFF)
    return out


def fmix32(h):
    h = np.asarray(h, np.uint64) & M32
    h ^= h >> np.uint64(16)
    h = (h * np.uint64(0x85EBCA6B)) & M32
    h ^= h >> np.uint64(13)
    h = (h * np.uint64(0xC2B2AE35)) & M32
    h ^= h >> np.uint64(16)
    return h


def half_bits(n: int) -> int:
    bits = 2
    while bits < 64 and (1 << bits) < n:
        bits += 2
    return bits // 2


def feistel4(x, hb: int, keys):
    x = np.asarray(x, np.uint64)
    mask = np.uint64((1 << hb) - 1)
    L = x >> np.uint64(hb)
    R = x & mask
    for r in range(4):
        f = fmix32((R & M32) ^ np.uint64(keys[r])) & mask
        L, R = R, L ^ f
    return (L << np.uint64(hb)) | R


def permute(i, n: int, keys, hb: int | None = None):
    """permute(i) for an array of sample numbers i < n."""
    hb = half_bits(n) if hb is None else hb
    j = feistel4(np.asarray(i, np.uint64), hb, keys)
    for _ in range(4096):
        bad = j >= np.uint64(n)
        if not bad.any():
            return j.astype(np.int64)
        j[bad] = feistel4(j[bad], hb, keys)
    raise RuntimeError("cycle walk did not end")
