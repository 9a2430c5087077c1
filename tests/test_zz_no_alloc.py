"""pbb_bound_children_noalloc: the bound entry point for callers that cannot
allocate GPU memory (they hand over device buffers they already own; the
function keeps its tables in a static device array instead of calling
cudaMalloc).  Checked through the C ABI against pbb_bound_children, on two
calls in a row with different instances, so that tables left in the shared
array by the first call cannot leak into the second.  Collected last on
purpose: a failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

_i32p = ctypes.POINTER(ctypes.c_int32)


def _fn():
    L = pb.lib()
    f = L.pbb_bound_children_noalloc
    f.argtypes = [ctypes.POINTER(pb._Instance), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_rejects_instances_beyond_the_scratch():
    p = synthetic_instance(3, 30, 21)            # 21 machines > 20
    inst = pb._Instance(30, 21, p.ctypes.data_as(_i32p))
    rc = _fn()(ctypes.byref(inst), 0, 0, None, 0, None, None, None, None, None, None, None, None, None)
    assert rc == pb.PBB_E_INVAL
    assert b"64 jobs and 20 machines" in pb.lib().pbb_last_error()


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    f = _fn()
    rng = np.random.default_rng(77)
    cases = [(50, 20, 2, 700), (20, 5, 0, 300)]   # second call: other instance, one-word rows
    for n, m, seed, count in cases:
        p = synthetic_instance(seed, n, m)
        sched = np.stack([rng.permutation(n) for _ in range(count)]).astype(np.int32)
        nf = rng.integers(0, n, size=count)
        nb = np.array([rng.integers(0, n - x + 1) for x in nf])
        l1 = (nf - 1).astype(np.int32)
        l2 = (n - nb).astype(np.int32)
        keep = l1 < l2
        sched, l1, l2 = sched[keep], l1[keep], l2[keep]
        cnt = len(sched)
        want = pb.bound_children(p, sched, l1, l2)

        dev = torch.device("cuda:0")
        d_s = torch.from_numpy(sched).to(dev)
        d_l1 = torch.from_numpy(l1).to(dev)
        d_l2 = torch.from_numpy(l2).to(dev)
        outs = [torch.full((cnt, n), -7, dtype=torch.int32, device=dev) for _ in range(4)]
        nodes = [torch.full((cnt,), -7, dtype=torch.int32, device=dev) for _ in range(2)]
        torch.cuda.synchronize()
        inst = pb._Instance(n, m, p.ctypes.data_as(_i32p))
        rc = f(ctypes.byref(inst), 0, 0, None, cnt, d_s.data_ptr(), d_l1.data_ptr(), d_l2.data_ptr(),
               outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), outs[3].data_ptr(),
               nodes[0].data_ptr(), nodes[1].data_ptr())
        assert rc == pb.PBB_OK, pb.lib().pbb_last_error()
        got = dict(weak_begin=outs[0], weak_end=outs[1], strong_begin=outs[2], strong_end=outs[3],
                   node_weak=nodes[0], node_strong=nodes[1])
        for k, v in got.items():
            assert np.array_equal(v.cpu().numpy(), want[k]), (n, m, k)   # integer bounds: exact


@pytest.mark.gpu
def test_noalloc_rejects_a_bad_node_on_device():
    import torch

    f = _fn()
    n, m = 12, 6
    p = synthetic_instance(5, n, m)
    sched = np.tile(np.arange(n, dtype=np.int32), (4, 1))
    sched[2, 3] = sched[2, 4]                     # not a permutation
    l1 = np.full(4, -1, np.int32)
    l2 = np.full(4, n, np.int32)
    dev = torch.device("cuda:0")
    bufs = [torch.from_numpy(a).to(dev) for a in (sched, l1, l2)]
    outs = [torch.zeros((4, n), dtype=torch.int32, device=dev) for _ in range(4)]
    nodes = [torch.zeros(4, dtype=torch.int32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    inst = pb._Instance(n, m, p.ctypes.data_as(_i32p))
    rc = f(ctypes.byref(inst), 0, 0, None, 4, *[b.data_ptr() for b in bufs], *[o.data_ptr() for o in outs],
           *[x.data_ptr() for x in nodes])
    assert rc == pb.PBB_E_INVAL
