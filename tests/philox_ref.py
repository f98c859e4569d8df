"""Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
easy as 1, 2, 3", SC'11) restated in numpy for the tests: 10 rounds of the
4x32 bijection (multipliers 0xD2511F53, 0xCD9E8D57; Weyl key increments
0x9E3779B9, 0xBB67AE85), and the published known-answer vectors of the
Random123 distribution for philox4x32 with 10 rounds.

Test infrastructure only: it checks the device generator behind
DVM_RNG_PHILOX, which has no counterpart in the reference (whose walk draws
from std::mt19937).
"""
import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
MASK = np.uint64(0xFFFFFFFF)

# (counter[4], key[2]) -> output[4]
KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox4x32_10(ctr, key):
    """ctr (n, 4), key (n, 2) integer arrays -> (n, 4) uint32."""
    c = np.asarray(ctr, dtype=np.uint64).reshape(-1, 4).copy()
    k = np.asarray(key, dtype=np.uint64).reshape(-1, 2).copy()
    for _ in range(10):
        p0 = M0 * c[:, 0]  # exact: 32 x 32 bits fit in 64
        p1 = M1 * c[:, 2]
        c = np.stack([((p1 >> np.uint64(32)) ^ c[:, 1] ^ k[:, 0]) & MASK, p1 & MASK,
                      ((p0 >> np.uint64(32)) ^ c[:, 3] ^ k[:, 1]) & MASK, p0 & MASK], axis=1)
        k = np.stack([(k[:, 0] + W0) & MASK, (k[:, 1] + W1) & MASK], axis=1)
    return c.astype(np.uint32)


def uniforms2(out):
    """The walk's two 53-bit uniforms in (0, 1] from each output block."""
    o = out.astype(np.uint64)
    s = 1.0 / 9007199254740992.0
    r1 = (((o[:, 0] >> np.uint64(5)) << np.uint64(26)) | (o[:, 1] >> np.uint64(6))).astype(np.float64)
    r2 = (((o[:, 2] >> np.uint64(5)) << np.uint64(26)) | (o[:, 3] >> np.uint64(6))).astype(np.float64)
    return (r1 + 1.0) * s, (r2 + 1.0) * s
