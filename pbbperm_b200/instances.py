"""Flow-shop instances: the project's seeded generator and the VRF file format.

The generator is splitmix64 with rejection sampling: p = lo + (u mod span),
drawing again while u falls in the last, incomplete block of 2^64 values, row-major
machine-major (m x n), the order of the reference's instance stream
(bounds/src/instance_flowshop.cpp:91-101).  It is identical bit for bit in
oracle/pbb_oracle.c (orc_synthetic_instance) and pbbperm_b200/csrc/ini.h.
"""
import os

import numpy as np

_M64 = (1 << 64) - 1


def _splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & _M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return state, z ^ (z >> 31)


def synthetic_instance(seed, n, m, lo=1, hi=99):
    """U[lo,hi] int32 processing times, shape (m, n)."""
    span = hi - lo + 1
    limit = _M64 - (_M64 % span)
    s = seed & _M64
    out = np.empty(n * m, dtype=np.int32)
    for i in range(n * m):
        while True:
            s, u = _splitmix64(s)
            if u < limit:
                break
        out[i] = lo + (u % span)
    return out.reshape(m, n)


def read_vrf(path):
    """Read a VRF `<name>_Gap.txt` file (bounds/src/instance_vrf.cpp:32-69):
    `n m` then n lines of (machine, time) pairs; returns p of shape (m, n)."""
    with open(path) as f:
        tok = f.read().split()
    n, m = int(tok[0]), int(tok[1])
    vals = [int(x) for x in tok[2:]]
    times = vals[1::2]
    if len(times) < n * m:
        raise ValueError("truncated VRF file %s" % path)
    p = np.array(times[: n * m], dtype=np.int32).reshape(n, m).T.copy()
    return p


def write_vrf(path, p):
    """Write p (m x n) in the VRF format read by read_vrf and by the reference."""
    m, n = p.shape
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("%d %d\n" % (n, m))
        for j in range(n):
            f.write(" ".join("%d %d" % (k, p[k, j]) for k in range(m)) + "\n")
