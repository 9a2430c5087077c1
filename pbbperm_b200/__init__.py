"""B200 IVM branch-and-bound for the permutation flow-shop (makespan).

Host-side mirror of the reference's engine and bounds interfaces over the C
ABI of libpbbperm.so (include/pbbperm.h):

  Engine         gpubb (gpu/include/gpubb.h): create / solve / start / explore
  bound_children bound_abstract::boundChildren + bornes_calculer
                 (bounds/include/bound_abstract.h) for a batch of nodes
  neh            fastNEH::runNEH initial upper bound
  Config         the reference's ini keys (common/src/arguments.cpp:80-132)

All compute runs in CUDA kernels; there is no CPU fallback.  Loading fails
loudly when the native library is missing.
"""
import ctypes
import os

import numpy as np

from .instances import synthetic_instance, read_vrf, write_vrf  # noqa: F401

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libpbbperm.so")

PBB_OK = 0
PBB_E_INVAL = -1
PBB_E_NOMEM = -2
PBB_E_CUDA = -3
PBB_E_TIMEOUT = -4
PBB_E_UNSUPPORTED = -5
MAX_JOBS = 64
INF = 2**31 - 1
UB_NEH = -1          # initial bound: NEH computed on the device

_i32p = ctypes.POINTER(ctypes.c_int32)


class PbbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("pbbperm error %d: %s" % (code, msg))
        self.code = code


class _Instance(ctypes.Structure):
    _fields_ = [("n_jobs", ctypes.c_int32), ("n_machines", ctypes.c_int32), ("p", _i32p)]


class _Config(ctypes.Structure):
    _fields_ = [("bounding_mode", ctypes.c_int32), ("branching_mode", ctypes.c_int32),
                ("find_all", ctypes.c_int32), ("johnson_mode", ctypes.c_int32),
                ("early_stop_johnson", ctypes.c_int32), ("sorted_dfs", ctypes.c_int32),
                ("nb_ivms", ctypes.c_int32), ("device", ctypes.c_int32),
                ("warps_per_cta", ctypes.c_int32), ("ctas", ctypes.c_int32),
                ("sorting_criterion", ctypes.c_int32), ("core_warps", ctypes.c_int32),
                ("split_depth", ctypes.c_int32), ("share_after", ctypes.c_int32)]


class _Stats(ctypes.Structure):
    _fields_ = [("decomposed", ctypes.c_uint64), ("johnson_bounds", ctypes.c_uint64),
                ("simple_bounds", ctypes.c_uint64), ("leaves", ctypes.c_uint64),
                ("steals", ctypes.c_uint64)]


class _Result(ctypes.Structure):
    _fields_ = [("complete", ctypes.c_int32), ("found", ctypes.c_int32), ("cost", ctypes.c_int32),
                ("n_jobs", ctypes.c_int32), ("perm", ctypes.c_int32 * MAX_JOBS), ("stats", _Stats),
                ("device_seconds", ctypes.c_double), ("has_perm", ctypes.c_int32), ("pad", ctypes.c_int32)]


class _Work(ctypes.Structure):
    _fields_ = [("device_seconds", ctypes.c_double), ("n_jobs", ctypes.c_int32), ("n_machines", ctypes.c_int32),
                ("machine_pairs", ctypes.c_int32), ("explorers", ctypes.c_int32), ("warps", ctypes.c_int32),
                ("status", ctypes.c_int32), ("decomposed", ctypes.c_uint64), ("simple_bounds", ctypes.c_uint64),
                ("johnson_bounds", ctypes.c_uint64), ("johnson_sweeps", ctypes.c_uint64),
                ("sweep_free_jobs", ctypes.c_uint64), ("sweep_children", ctypes.c_uint64),
                ("direct_children", ctypes.c_uint64), ("direct_free_jobs", ctypes.c_uint64)]


class _PoolConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("max_jobs", ctypes.c_int32), ("max_machines", ctypes.c_int32),
                ("max_resident", ctypes.c_int32), ("warps_per_cta", ctypes.c_int32),
                ("ctas_per_instance", ctypes.c_int32), ("explorers_per_instance", ctypes.c_int32),
                ("tail_warps", ctypes.c_int32), ("window_s", ctypes.c_double), ("explorer_bytes", ctypes.c_int64),
                ("core_warps", ctypes.c_int32), ("split_depth", ctypes.c_int32),
                ("share_after", ctypes.c_int32), ("pad", ctypes.c_int32)]


class _PoolResult(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_int64), ("windows", ctypes.c_int32), ("status", ctypes.c_int32),
                ("result", _Result)]


class _BoundOut(ctypes.Structure):
    _fields_ = [(k, _i32p) for k in ("weak_begin", "weak_end", "strong_begin", "strong_end", "node_weak",
                                     "node_strong", "prio_begin", "prio_end", "strong_idle")]


_lib = None


def lib():
    """Load libpbbperm.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpbbperm.so not built: run `python -m pbbperm_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.pbb_last_error.restype = ctypes.c_char_p
        L.pbb_config_default.argtypes = [ctypes.POINTER(_Config)]
        L.pbb_engine_create.argtypes = [ctypes.POINTER(_Instance), ctypes.POINTER(_Config),
                                        ctypes.POINTER(ctypes.c_void_p)]
        L.pbb_engine_destroy.argtypes = [ctypes.c_void_p]
        L.pbb_solve.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p, ctypes.c_double, ctypes.POINTER(_Result)]
        L.pbb_start.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p]
        L.pbb_explore.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_int32)]
        L.pbb_get_result.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Result)]
        L.pbb_bound_children.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]
        L.pbb_neh.argtypes = [ctypes.POINTER(_Instance), _i32p, _i32p]
        L.pbb_bound_children_ex.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.POINTER(_BoundOut)]
        L.pbb_neh_batch.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.c_int32, _i32p, _i32p]
        L.pbb_ig_batch.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_uint64, _i32p, _i32p]
        L.pbb_start_interval.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p, _i32p, _i32p]
        L.pbb_init_from_fac.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p, _i32p, _i32p]
        L.pbb_get_intervals.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p, _i32p, _i32p,
                                        ctypes.POINTER(ctypes.c_int32)]
        L.pbb_set_ub.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        L.pbb_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.pbb_save_checkpoint.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.pbb_load_checkpoint.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]
        L.pbb_fact_to_decimal.argtypes = [ctypes.c_int32, _i32p, ctypes.c_char_p, ctypes.c_int32]
        L.pbb_decimal_to_fact.argtypes = [ctypes.c_int32, ctypes.c_char_p, _i32p]
        L.pbb_diag_set_step_limits.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
        L.pbb_diag_sample_nodes.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
        L.pbb_diag_get_samples.argtypes = [ctypes.c_void_p, ctypes.c_int32, _i32p, ctypes.POINTER(ctypes.c_int32)]
        L.pbb_work_counters.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Work)]
        L.pbb_diag_bound_children.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.c_int32,
                                               ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p,
                                               _i32p, _i32p, _i32p, _i32p]
        L.pbb_pool_config_default.argtypes = [ctypes.POINTER(_PoolConfig)]
        L.pbb_pool_create.argtypes = [ctypes.POINTER(_PoolConfig), ctypes.POINTER(ctypes.c_void_p)]
        L.pbb_pool_destroy.argtypes = [ctypes.c_void_p]
        L.pbb_pool_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Instance), ctypes.POINTER(_Config),
                                      ctypes.c_int32, _i32p, ctypes.c_int64]
        L.pbb_pool_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.pbb_pool_poll.argtypes = [ctypes.c_void_p, ctypes.POINTER(_PoolResult), ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_int32)]
        L.pbb_batch_solve.argtypes = [ctypes.POINTER(_Instance), ctypes.c_int32, ctypes.POINTER(_Config), _i32p,
                                      ctypes.POINTER(_PoolConfig), ctypes.POINTER(_Result)]
        L.pbb_diag_int32_peak.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]
        _lib = L
    return _lib


def _check(rc):
    if rc != PBB_OK:
        raise PbbError(rc, lib().pbb_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(_i32p) if a is not None else None


def _instance(p):
    p = np.ascontiguousarray(p, dtype=np.int32)
    if p.ndim != 2:
        raise ValueError("p must be a (machines x jobs) matrix")
    inst = _Instance(p.shape[1], p.shape[0], _ptr(p))
    return inst, p


class Config:
    """Search settings, named after the reference ini keys."""

    def __init__(self, boundingMode=2, adaptiveBranchingMode=3, findAll=False, JohnsonMode=0,
                 earlyStopJohnson=False, sortedDFS=0, nbIVMs=16384, device=0, warps_per_cta=0, ctas=0,
                 sortingCriterion=1, core_warps=0, split_depth=0, share_after=0):
        self.boundingMode = boundingMode
        self.adaptiveBranchingMode = adaptiveBranchingMode
        self.findAll = findAll
        self.JohnsonMode = JohnsonMode
        self.earlyStopJohnson = earlyStopJohnson
        self.sortedDFS = sortedDFS
        self.nbIVMs = nbIVMs
        self.device = device
        self.warps_per_cta = warps_per_cta
        self.ctas = ctas
        self.sortingCriterion = sortingCriterion
        self.core_warps = core_warps
        self.split_depth = split_depth
        self.share_after = share_after

    def _c(self):
        return _Config(self.boundingMode, self.adaptiveBranchingMode, 1 if self.findAll else 0, self.JohnsonMode,
                       1 if self.earlyStopJohnson else 0, self.sortedDFS, self.nbIVMs, self.device,
                       self.warps_per_cta, self.ctas, self.sortingCriterion, self.core_warps, self.split_depth,
                       self.share_after)


def _result(r):
    n = r.n_jobs
    return dict(complete=bool(r.complete), found=bool(r.found), cost=r.cost, has_perm=bool(r.has_perm),
                perm=np.array(r.perm[:n], dtype=np.int32),
                decomposed=r.stats.decomposed, johnson_bounds=r.stats.johnson_bounds,
                simple_bounds=r.stats.simple_bounds, leaves=r.stats.leaves, steals=r.stats.steals,
                device_seconds=r.device_seconds)


class Engine:
    """One instance resident on one GPU (class gpubb, gpu/include/gpubb.h:24-173)."""

    def __init__(self, p, config=None):
        self.config = config or Config()
        inst, self._p = _instance(p)
        self.m, self.n = self._p.shape
        h = ctypes.c_void_p()
        cfg = self.config._c()
        _check(lib().pbb_engine_create(ctypes.byref(inst), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().pbb_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def solve(self, ub=INF, root=None, time_limit=0.0):
        r = _Result()
        root = None if root is None else np.ascontiguousarray(root, dtype=np.int32)
        _check(lib().pbb_solve(self._h, int(ub), _ptr(root), float(time_limit), ctypes.byref(r)))
        return _result(r)

    def start(self, ub=INF, root=None):
        root = None if root is None else np.ascontiguousarray(root, dtype=np.int32)
        _check(lib().pbb_start(self._h, int(ub), _ptr(root)))

    def start_interval(self, ub, pos, end, root=None):
        """Start on the factoradic interval [pos, end] (gpubb::initAtInterval)."""
        root = None if root is None else np.ascontiguousarray(root, dtype=np.int32)
        pos = np.ascontiguousarray(pos, dtype=np.int32)
        end = np.ascontiguousarray(end, dtype=np.int32)
        _check(lib().pbb_start_interval(self._h, int(ub), _ptr(root), _ptr(pos), _ptr(end)))

    def init_from_fac(self, ub, pos, end, ids=None, root=None):
        """Start explorer ids[k] (k by default) on interval k: pos and end are
        (count, n) factoradic digit arrays (gpubb::initFromFac)."""
        root = None if root is None else np.ascontiguousarray(root, dtype=np.int32)
        pos = np.ascontiguousarray(pos, dtype=np.int32)
        end = np.ascontiguousarray(end, dtype=np.int32)
        count = pos.shape[0]
        if pos.ndim != 2 or end.shape != pos.shape:
            raise ValueError("pos and end must be (count, n) arrays of the same shape")
        ids = None if ids is None else np.ascontiguousarray(ids, dtype=np.int32)
        _check(lib().pbb_init_from_fac(self._h, int(ub), _ptr(root), int(count), _ptr(ids), _ptr(pos), _ptr(end)))

    def get_intervals(self):
        """(pos, end, ids) of the explorers still holding work, between windows
        (gpubb::getIntervals); pos and end are (count, n) arrays."""
        n = self.n
        cnt = ctypes.c_int32(0)
        rc = lib().pbb_get_intervals(self._h, 0, None, None, None, ctypes.byref(cnt))
        if rc != 0 and cnt.value == 0:
            _check(rc)
        k = max(1, cnt.value)
        pos = np.zeros((k, n), np.int32)
        end = np.zeros((k, n), np.int32)
        ids = np.zeros(k, np.int32)
        _check(lib().pbb_get_intervals(self._h, k, _ptr(pos), _ptr(end), _ptr(ids), ctypes.byref(cnt)))
        c = cnt.value
        return pos[:c], end[:c], ids[:c]

    def set_ub(self, ub):
        """Lower the incumbent to a bound found elsewhere (no permutation)."""
        _check(lib().pbb_set_ub(self._h, int(ub)))

    def save_checkpoint(self, path):
        """Write the search's state between windows in the reference's
        works::save form (root, bound count, incumbent, intervals)."""
        _check(lib().pbb_save_checkpoint(self._h, os.fsencode(path)))

    def load_checkpoint(self, path):
        """Resume a checkpoint file; returns the bound count it stored."""
        v = ctypes.c_uint64(0)
        _check(lib().pbb_load_checkpoint(self._h, os.fsencode(path), ctypes.byref(v)))
        return v.value

    def set_wait_limit(self, seconds):
        """Longest host wait for one window (< 0: window + 60 s, 0: none);
        explore() raises PbbError(PBB_E_TIMEOUT) when it runs out, and the
        next call accounts for the window."""
        _check(lib().pbb_set_wait_limit(self._h, float(seconds)))

    def sample_nodes(self, capacity, rate_log2):
        """Diagnostic: from the next window on, record nodes the explorer
        bounds (hash-sampled at 2^-rate_log2, at most `capacity`; 0 = off)."""
        _check(lib().pbb_diag_sample_nodes(self._h, int(capacity), int(rate_log2)))

    def sample_count(self):
        """Nodes recorded so far (at most the capacity)."""
        cnt = ctypes.c_int32(0)
        _check(lib().pbb_diag_get_samples(self._h, 0, None, ctypes.byref(cnt)))
        return cnt.value

    def samples(self):
        """Recorded nodes as a dict of arrays: explorer, line, limit1, limit2,
        side, best, k (count,) and sched, weak_begin, weak_end, strong_begin,
        strong_end (count, n) -- include/pbbperm_diag.h's record layout."""
        n = self.n
        cnt = ctypes.c_int32(0)
        _check(lib().pbb_diag_get_samples(self._h, 0, None, ctypes.byref(cnt)))
        stride = 8 + 5 * n
        buf = np.zeros((max(1, cnt.value), stride), np.int32)
        _check(lib().pbb_diag_get_samples(self._h, cnt.value, _ptr(buf), ctypes.byref(cnt)))
        buf = buf[:cnt.value]
        out = {k: buf[:, i].copy() for i, k in enumerate(("explorer", "line", "limit1", "limit2", "side", "best", "k"))}
        for i, k in enumerate(("sched", "weak_begin", "weak_end", "strong_begin", "strong_end")):
            out[k] = buf[:, 8 + i * n: 8 + (i + 1) * n].copy()
        return out

    def set_step_limits(self, select_budget=4096, max_rounds=2**31 - 1):
        """Diagnostic: selection steps per explorer step and loop rounds per
        window launch (tests of the bounded loops)."""
        _check(lib().pbb_diag_set_step_limits(self._h, int(select_budget), int(max_rounds)))

    def kernel_stats(self):
        """Work of the explorer kernels since start, with the INT32 op model
        of the bounds: weak child 5m ops (add/max chain per machine); per
        Johnson sweep and machine pair, 5 ops per free job and pass (forward,
        backward), 9 ops per evaluated child; per directly scanned child and
        pair, 4 ops per free job (add, add, max, add)."""
        w = _Work()
        _check(lib().pbb_work_counters(self._h, ctypes.byref(w)))
        m, n, P = w.n_machines, w.n_jobs, w.machine_pairs
        ops = (5 * m * w.simple_bounds +
               P * (10 * w.sweep_free_jobs + 9 * w.sweep_children) +
               P * 4 * w.direct_free_jobs)
        return dict(device_seconds=w.device_seconds, int32_ops=float(ops), decomposed=w.decomposed,
                    simple_bounds=w.simple_bounds, johnson_bounds=w.johnson_bounds,
                    johnson_sweeps=w.johnson_sweeps, sweep_free_jobs=w.sweep_free_jobs,
                    sweep_children=w.sweep_children, direct_children=w.direct_children,
                    direct_free_jobs=w.direct_free_jobs,
                    explorers=w.explorers, warps=w.warps, status=w.status,
                    work_model="5m per weak child + P*(10 per swept free job + 9 per swept child)"
                               " + P*4 per free job of a directly scanned child")

    def explore(self, seconds):
        done = ctypes.c_int32(0)
        _check(lib().pbb_explore(self._h, float(seconds), ctypes.byref(done)))
        return bool(done.value)

    def result(self):
        r = _Result()
        _check(lib().pbb_get_result(self._h, ctypes.byref(r)))
        return _result(r)


def bound_children(p, sched, limit1, limit2, johnson_mode=0, device=0, method=None):
    """Children LBs of a batch of nodes on the GPU.

    Returns dict of (count x n) arrays weak_begin, weak_end, strong_begin,
    strong_end (by job id, 0 for fixed jobs) and (count,) node_weak,
    node_strong.  method (diagnostic): 0 = sweeps, 1 = direct per-child
    scans; None = the default entry point."""
    inst, p = _instance(p)
    n = p.shape[1]
    sched = np.ascontiguousarray(sched, dtype=np.int32).reshape(-1, n)
    cnt = sched.shape[0]
    l1 = np.ascontiguousarray(limit1, dtype=np.int32).reshape(cnt)
    l2 = np.ascontiguousarray(limit2, dtype=np.int32).reshape(cnt)
    out = {k: np.zeros((cnt, n), np.int32) for k in ("weak_begin", "weak_end", "strong_begin", "strong_end")}
    out["node_weak"] = np.zeros(cnt, np.int32)
    out["node_strong"] = np.zeros(cnt, np.int32)
    outs = (_ptr(out["weak_begin"]), _ptr(out["weak_end"]), _ptr(out["strong_begin"]), _ptr(out["strong_end"]),
            _ptr(out["node_weak"]), _ptr(out["node_strong"]))
    if method is None:
        _check(lib().pbb_bound_children(ctypes.byref(inst), johnson_mode, device, cnt, _ptr(sched), _ptr(l1), _ptr(l2),
                                        *outs))
    else:
        _check(lib().pbb_diag_bound_children(ctypes.byref(inst), johnson_mode, device, method, cnt, _ptr(sched),
                                             _ptr(l1), _ptr(l2), *outs))
    return out


def fact_to_decimal(digits):
    """Factoradic vector (digit i in [0, n-i)) -> decimal index string."""
    d = np.ascontiguousarray(digits, dtype=np.int32)
    buf = ctypes.create_string_buffer(128)
    _check(lib().pbb_fact_to_decimal(len(d), _ptr(d), buf, 128))
    return buf.value.decode()


def decimal_to_fact(n, decimal):
    """Decimal index (below n!) -> factoradic vector of n digits."""
    d = np.zeros(n, np.int32)
    _check(lib().pbb_decimal_to_fact(int(n), str(decimal).encode(), _ptr(d)))
    return d


def bound_children_ex(p, sched, limit1, limit2, johnson_mode=0, device=0):
    """bound_children plus the weak bound's idle-time priorities of every
    child (prio_begin / prio_end, (count, n) by job id) and the Johnson
    bound's couts[1] per node (strong_idle)."""
    inst, p = _instance(p)
    n = p.shape[1]
    sched = np.ascontiguousarray(sched, dtype=np.int32).reshape(-1, n)
    cnt = sched.shape[0]
    l1 = np.ascontiguousarray(limit1, dtype=np.int32).reshape(cnt)
    l2 = np.ascontiguousarray(limit2, dtype=np.int32).reshape(cnt)
    out = {k: np.zeros((cnt, n), np.int32) for k in ("weak_begin", "weak_end", "strong_begin", "strong_end",
                                                      "prio_begin", "prio_end")}
    for k in ("node_weak", "node_strong", "strong_idle"):
        out[k] = np.zeros(cnt, np.int32)
    o = _BoundOut(**{k: _ptr(v) for k, v in out.items()})
    _check(lib().pbb_bound_children_ex(ctypes.byref(inst), johnson_mode, device, cnt, _ptr(sched), _ptr(l1),
                                       _ptr(l2), ctypes.byref(o)))
    return out


def int32_peak(device=0):
    """Measured INT32 add+max throughput of the GPU in Gop/s."""
    g = ctypes.c_double(0.0)
    t = ctypes.c_double(0.0)
    _check(lib().pbb_diag_int32_peak(device, ctypes.byref(g), ctypes.byref(t)))
    return g.value


def neh(p):
    """NEH upper bound (host code): (cost, permutation)."""
    inst, p = _instance(p)
    perm = np.zeros(p.shape[1], np.int32)
    cost = np.zeros(1, np.int32)
    _check(lib().pbb_neh(ctypes.byref(inst), _ptr(perm), _ptr(cost)))
    return int(cost[0]), perm


def neh_batch(instances, device=0):
    """NEH of many instances on the device (one warp each): list of
    (cost, permutation), equal to neh() for each."""
    cnt = len(instances)
    keep = [np.ascontiguousarray(p, dtype=np.int32) for p in instances]
    arr = (_Instance * cnt)(*[_Instance(p.shape[1], p.shape[0], _ptr(p)) for p in keep])
    perms = np.zeros((cnt, MAX_JOBS), np.int32)
    costs = np.zeros(cnt, np.int32)
    _check(lib().pbb_neh_batch(arr, cnt, int(device), _ptr(perms), _ptr(costs)))
    return [(int(costs[i]), perms[i, :keep[i].shape[1]].copy()) for i in range(cnt)]


def ig_batch(instances, iterations=100, seed=0, device=0):
    """Seeded iterated greedy from NEH on the device (one warp per instance):
    list of (cost, permutation); instance i draws from seed + i."""
    cnt = len(instances)
    keep = [np.ascontiguousarray(p, dtype=np.int32) for p in instances]
    arr = (_Instance * cnt)(*[_Instance(p.shape[1], p.shape[0], _ptr(p)) for p in keep])
    perms = np.zeros((cnt, MAX_JOBS), np.int32)
    costs = np.zeros(cnt, np.int32)
    _check(lib().pbb_ig_batch(arr, cnt, int(device), int(iterations), int(seed), _ptr(perms), _ptr(costs)))
    return [(int(costs[i]), perms[i, :keep[i].shape[1]].copy()) for i in range(cnt)]


class PoolConfig:
    """Resident pool shape (include/pbbperm.h pbb_pool_config)."""

    def __init__(self, max_jobs=32, max_machines=20, max_resident=0, warps_per_cta=8, ctas_per_instance=0,
                 explorers_per_instance=0, window_s=0.005, explorer_bytes=8 << 30, device=0, tail_warps=0,
                 core_warps=0, split_depth=0, share_after=0):
        self.max_jobs = max_jobs
        self.max_machines = max_machines
        self.max_resident = max_resident
        self.warps_per_cta = warps_per_cta
        self.ctas_per_instance = ctas_per_instance
        self.explorers_per_instance = explorers_per_instance
        self.window_s = window_s
        self.explorer_bytes = explorer_bytes
        self.device = device
        self.tail_warps = tail_warps
        self.core_warps = core_warps
        self.split_depth = split_depth
        self.share_after = share_after

    def _c(self):
        return _PoolConfig(self.device, self.max_jobs, self.max_machines, self.max_resident, self.warps_per_cta,
                           self.ctas_per_instance, self.explorers_per_instance, self.tail_warps, self.window_s,
                           self.explorer_bytes, self.core_warps, self.split_depth, self.share_after)


class Pool:
    """Many instances resident on one GPU; continuous batching by windows."""

    def __init__(self, config=None):
        self.config = config or PoolConfig()
        h = ctypes.c_void_p()
        c = self.config._c()
        _check(lib().pbb_pool_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h
        self._inst = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().pbb_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, p, tag, ub=INF, config=None, root=None):
        inst, pp = _instance(p)
        cfg = (config or Config())._c()
        root = None if root is None else np.ascontiguousarray(root, dtype=np.int32)
        _check(lib().pbb_pool_submit(self._h, ctypes.byref(inst), ctypes.byref(cfg), int(ub), _ptr(root), int(tag)))

    def step(self):
        """One window; returns (resident, queued)."""
        r = ctypes.c_int32(0)
        q = ctypes.c_int32(0)
        _check(lib().pbb_pool_step(self._h, ctypes.byref(r), ctypes.byref(q)))
        return r.value, q.value

    def poll(self, max_results=4096):
        buf = (_PoolResult * max_results)()
        got = ctypes.c_int32(0)
        _check(lib().pbb_pool_poll(self._h, buf, max_results, ctypes.byref(got)))
        out = []
        for i in range(got.value):
            d = _result(buf[i].result)
            d["tag"] = buf[i].tag
            d["windows"] = buf[i].windows
            d["status"] = buf[i].status
            out.append(d)
        return out


def batch_solve(instances, ubs=None, config=None, pool_config=None):
    """Solve many instances through one resident pool (pbb_batch_solve)."""
    cnt = len(instances)
    keep = [np.ascontiguousarray(p, dtype=np.int32) for p in instances]
    arr = (_Instance * cnt)(*[_Instance(p.shape[1], p.shape[0], _ptr(p)) for p in keep])
    cfg = (config or Config())._c()
    u = None if ubs is None else np.ascontiguousarray(ubs, dtype=np.int32)
    res = (_Result * cnt)()
    pc = None if pool_config is None else ctypes.byref(pool_config._c())
    _check(lib().pbb_batch_solve(arr, cnt, ctypes.byref(cfg), _ptr(u), pc, res))
    return [_result(r) for r in res]
