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


def _random_nodes(rng, n, count):
    sched = np.stack([rng.permutation(n) for _ in range(count)]).astype(np.int32)
    nf = rng.integers(0, n, size=count)
    nb = np.array([rng.integers(0, n - x + 1) for x in nf])
    l1 = (nf - 1).astype(np.int32)
    l2 = (n - nb).astype(np.int32)
    keep = l1 < l2
    return sched[keep], l1[keep], l2[keep]


def _call_noalloc(f, p, johnson_mode, sched, l1, l2):
    """One call through the C ABI with device buffers; returns the outputs as
    numpy arrays (the buffers start at -7 so that unwritten cells show)."""
    import torch

    m, n = p.shape
    cnt = len(sched)
    dev = torch.device("cuda:0")
    d_s = torch.from_numpy(sched).to(dev)
    d_l1 = torch.from_numpy(l1).to(dev)
    d_l2 = torch.from_numpy(l2).to(dev)
    outs = [torch.full((cnt, n), -7, dtype=torch.int32, device=dev) for _ in range(4)]
    nodes = [torch.full((cnt,), -7, dtype=torch.int32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    inst = pb._Instance(n, m, p.ctypes.data_as(_i32p))
    rc = f(ctypes.byref(inst), johnson_mode, 0, None, cnt, d_s.data_ptr(), d_l1.data_ptr(), d_l2.data_ptr(),
           outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), outs[3].data_ptr(),
           nodes[0].data_ptr(), nodes[1].data_ptr())
    assert rc == pb.PBB_OK, pb.lib().pbb_last_error()
    return dict(weak_begin=outs[0].cpu().numpy(), weak_end=outs[1].cpu().numpy(),
                strong_begin=outs[2].cpu().numpy(), strong_end=outs[3].cpu().numpy(),
                node_weak=nodes[0].cpu().numpy(), node_strong=nodes[1].cpu().numpy())


@pytest.mark.gpu
@pytest.mark.parametrize("johnson_mode", [0, 1, 2])
def test_noalloc_matches_allocating_entry_point_twice(johnson_mode):
    """Two calls in a row with different instances (the second one leaves
    tables of another size and row width in the shared array), each equal to
    pbb_bound_children with the same machine-pair mode."""
    f = _fn()
    rng = np.random.default_rng(77 + johnson_mode)
    cases = [(50, 20, 2, 700), (20, 5, 0, 300)]   # second call: other instance, one-word rows
    for n, m, seed, count in cases:
        p = synthetic_instance(seed, n, m)
        sched, l1, l2 = _random_nodes(rng, n, count)
        want = pb.bound_children(p, sched, l1, l2, johnson_mode=johnson_mode)
        got = _call_noalloc(f, p, johnson_mode, sched, l1, l2)
        for k, v in got.items():
            assert np.array_equal(v, want[k]), (n, m, johnson_mode, k)   # integer bounds: exact


@pytest.mark.gpu
def test_noalloc_allocates_no_device_memory():
    """After a warm-up call (which loads the kernels and looks the scratch
    array up), further calls leave the device's free memory and torch's
    allocator untouched."""
    import torch

    f = _fn()
    rng = np.random.default_rng(9)
    work = []
    for n, m, seed in [(40, 12, 31), (24, 20, 32), (40, 12, 33), (24, 20, 34)]:
        p = synthetic_instance(seed, n, m)
        work.append((p,) + _random_nodes(rng, n, 256))
    # warm-up: both row widths (one- and two-word rows use different kernels)
    _call_noalloc(f, *work[0][:1], 0, *work[0][1:])
    _call_noalloc(f, *work[1][:1], 0, *work[1][1:])
    torch.cuda.synchronize()
    # the call's own device buffers are made before measuring
    dev = torch.device("cuda:0")
    bufs = []
    for p, sched, l1, l2 in work[2:]:
        m, n = p.shape
        cnt = len(sched)
        bufs.append((p, [torch.from_numpy(a).to(dev) for a in (sched, l1, l2)],
                     [torch.zeros((cnt, n), dtype=torch.int32, device=dev) for _ in range(4)],
                     [torch.zeros(cnt, dtype=torch.int32, device=dev) for _ in range(2)]))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for p, ins, outs, nodes in bufs:
        m, n = p.shape
        inst = pb._Instance(n, m, p.ctypes.data_as(_i32p))
        rc = f(ctypes.byref(inst), 0, 0, None, len(ins[0]), *[b.data_ptr() for b in ins],
               *[o.data_ptr() for o in outs], *[x.data_ptr() for x in nodes])
        assert rc == pb.PBB_OK, pb.lib().pbb_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_allocated() == alloc0


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
