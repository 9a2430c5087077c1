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


def _draw(state, lo, hi):
    span = hi - lo + 1
    limit = _M64 - (_M64 % span)
    while True:
        state, u = _splitmix64(state)
        if u < limit:
            return state, lo + (u % span)


def batch_instance(seed):
    """Instance of the batched workload: n uniform in {12..20} jobs and m in
    {5, 10, 20} machines drawn first from the seed's splitmix64 stream, then
    U[1,99] processing times from the same stream (row-major m x n)."""
    s = seed & _M64
    s, n = _draw(s, 12, 20)
    s, k = _draw(s, 0, 2)
    m = (5, 10, 20)[k]
    p = np.empty(n * m, dtype=np.int32)
    for i in range(n * m):
        s, p[i] = _draw(s, 1, 99)
    return p.reshape(m, n)


def serving_instance(seed):
    """Instance of the serving workload: n uniform in {10..22}, m uniform in
    {5..20}, then U[1,99] times, all from the seed's splitmix64 stream."""
    s = seed & _M64
    s, n = _draw(s, 10, 22)
    s, m = _draw(s, 5, 20)
    p = np.empty(n * m, dtype=np.int32)
    for i in range(n * m):
        s, p[i] = _draw(s, 1, 99)
    return p.reshape(m, n)


def poisson_arrivals(seed, rate, count):
    """Arrival times (s) of a Poisson stream: exponential gaps of mean 1/rate
    from the seed's splitmix64 stream (53-bit uniforms)."""
    s = seed & _M64
    t = 0.0
    out = np.empty(count)
    for i in range(count):
        s, u = _splitmix64(s)
        x = ((u >> 11) + 1) / float(1 << 53)   # (0, 1]
        t += -np.log(x) / rate
        out[i] = t
    return out
