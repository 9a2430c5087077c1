"""Test oracle for the PBBPerm flow-shop hot path (TEST INFRASTRUCTURE ONLY).

`liboracle.so` is a plain-C restatement (oracle/pbb_oracle.c) of the
reference's bounds (bounds/src/bound_fsp_weak.cpp, bound_fsp_strong.cpp) and
of its sequential IVM branch-and-bound (multicore/src/sequentialbb.cpp,
ivm.cpp, ivm_bound.cpp).  `Reference` wraps the reference's own bounds library
and multicore binaries compiled by oracle/build_ref.py into oracle/_ref/.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package; the product (pbbperm_b200) never imports it.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_i32p = ctypes.POINTER(ctypes.c_int32)


def build_oracle(force=False):
    """Compile oracle/pbb_oracle.c into oracle/liboracle.so."""
    src = os.path.join(HERE, "pbb_oracle.c")
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", LIB_PATH, src])
    return LIB_PATH


class _OrcCfg(ctypes.Structure):
    _fields_ = [("bound_mode", ctypes.c_int), ("branch_mode", ctypes.c_int),
                ("find_all", ctypes.c_int), ("sort_nodes", ctypes.c_int), ("node_limit", ctypes.c_int64),
                ("sort_crit", ctypes.c_int)]


class _OrcResult(ctypes.Structure):
    _fields_ = [("decomposed", ctypes.c_int64), ("johnson_bounds", ctypes.c_int64),
                ("simple_bounds", ctypes.c_int64), ("leaves", ctypes.c_int64),
                ("best", ctypes.c_int), ("found", ctypes.c_int), ("complete", ctypes.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_eval.argtypes = [ctypes.c_void_p, _i32p]
        L.orc_weak_node.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int, ctypes.c_int]
        L.orc_weak_children.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _i32p, _i32p, _i32p, _i32p]
        L.orc_strong_node.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int, ctypes.c_int]
        L.orc_strong_idle.argtypes = [ctypes.c_void_p, _i32p, ctypes.c_int, ctypes.c_int]
        L.orc_johnson_row.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p]
        L.orc_lag_row.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p]
        L.orc_min_times.argtypes = [ctypes.c_void_p, _i32p, _i32p]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(_OrcCfg), ctypes.c_int, _i32p,
                                ctypes.POINTER(_OrcResult), _i32p]
        L.orc_solve_interval.argtypes = [ctypes.c_void_p, ctypes.POINTER(_OrcCfg), ctypes.c_int, _i32p, _i32p,
                                         _i32p, ctypes.POINTER(_OrcResult), _i32p]
        L.orc_neh.argtypes = [ctypes.c_void_p, _i32p]
        L.orc_ig.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_uint64, _i32p]
        L.orc_synthetic_instance.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _i32p]
        L.orc_taillard_instance.argtypes = [ctypes.c_long, ctypes.c_int, ctypes.c_int, _i32p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_i32p)


def synthetic_instance(seed, n, m, lo=1, hi=99):
    """U[lo,hi] int32 instance, row-major m x n, from the project splitmix64 stream."""
    p = np.zeros(n * m, dtype=np.int32)
    lib().orc_synthetic_instance(seed, n, m, lo, hi, _ptr(p))
    return p.reshape(m, n)


def taillard_instance(time_seed, n, m):
    p = np.zeros(n * m, dtype=np.int32)
    lib().orc_taillard_instance(time_seed, n, m, _ptr(p))
    return p.reshape(m, n)


class Oracle:
    """Bounds and sequential B&B of one instance (p: m x n int32)."""

    def __init__(self, p, pair_mode=0):
        p = np.ascontiguousarray(p, dtype=np.int32)
        self.m, self.n = p.shape
        self.p = p
        self._h = lib().orc_create(self.n, self.m, _ptr(p.ravel()), pair_mode)
        if not self._h:
            raise ValueError("oracle: unsupported instance size")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def eval(self, perm):
        return lib().orc_eval(self._h, _ptr(np.ascontiguousarray(perm, dtype=np.int32)))

    def weak_node(self, sched, l1, l2):
        return lib().orc_weak_node(self._h, _ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2)

    def weak_children(self, sched, l1, l2, both=True):
        cb = np.zeros(self.n, np.int32); ce = np.zeros(self.n, np.int32)
        pb = np.zeros(self.n, np.int32); pe = np.zeros(self.n, np.int32)
        lib().orc_weak_children(self._h, _ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2,
                                1 if both else 0, _ptr(cb), _ptr(ce), _ptr(pb), _ptr(pe))
        return cb, ce, pb, pe

    def strong_node(self, sched, l1, l2):
        return lib().orc_strong_node(self._h, _ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2)

    def strong_node_idle(self, sched, l1, l2):
        """couts[1] of the Johnson bound: idle time of the fixed jobs' schedules
        (0 when nothing is fixed at the back or at most one job is free)."""
        return lib().orc_strong_idle(self._h, _ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2)

    def strong_children(self, sched, l1, l2, front):
        """Johnson LB of every free job appended at the front (or back), by job id."""
        sched = np.array(sched, dtype=np.int32)
        out = np.zeros(self.n, np.int32)
        L1 = l1 + (1 if front else 0)
        L2 = l2 - (0 if front else 1)
        fill = L1 if front else L2
        for i in range(l1 + 1, l2):
            j = sched[i]
            s = sched.copy()
            s[fill], s[i] = s[i], s[fill]
            out[j] = self.strong_node(s, L1, L2)
        return out

    def johnson_row(self, s):
        out = np.zeros(self.n, np.int32)
        lib().orc_johnson_row(self._h, s, _ptr(out))
        return out

    def lag_row(self, s):
        out = np.zeros(self.n, np.int32)
        lib().orc_lag_row(self._h, s, _ptr(out))
        return out

    def min_times(self):
        a = np.zeros(self.m, np.int32); d = np.zeros(self.m, np.int32)
        lib().orc_min_times(self._h, _ptr(a), _ptr(d))
        return a, d

    def neh(self):
        perm = np.zeros(self.n, np.int32)
        c = lib().orc_neh(self._h, _ptr(perm))
        return c, perm

    def ig(self, iterations, seed, destruct=2, destruct_max=5, ls_passes=64):
        """The engine's seeded iterated greedy, restated (see orc_ig)."""
        perm = np.zeros(self.n, np.int32)
        c = lib().orc_ig(self._h, iterations, destruct, destruct_max, ls_passes, seed, _ptr(perm))
        return c, perm

    def solve(self, ub, bound_mode=2, branch_mode=3, find_all=False, root=None, node_limit=0, pos=None, end=None,
              sorted_dfs=0, sorting_criterion=1):
        cfg = _OrcCfg(bound_mode, branch_mode, 1 if find_all else 0, int(sorted_dfs), node_limit,
                      int(sorting_criterion))
        res = _OrcResult()
        root = np.arange(self.n, dtype=np.int32) if root is None else np.ascontiguousarray(root, dtype=np.int32)
        perm = np.zeros(self.n, np.int32)
        pos = None if pos is None else np.ascontiguousarray(pos, dtype=np.int32)
        end = None if end is None else np.ascontiguousarray(end, dtype=np.int32)
        rc = lib().orc_solve_interval(self._h, ctypes.byref(cfg), int(ub), _ptr(root), _ptr(pos) if pos is not None
                                      else None, _ptr(end) if end is not None else None, ctypes.byref(res),
                                      _ptr(perm))
        if rc != 0:
            raise RuntimeError("oracle solve failed")
        return dict(decomposed=res.decomposed, johnson_bounds=res.johnson_bounds,
                    simple_bounds=res.simple_bounds, leaves=res.leaves, best=res.best,
                    found=bool(res.found), complete=bool(res.complete), perm=perm)


# --------------------------------------------------------------------------
# the reference's own code (oracle/_ref, built by oracle/build_ref.py)
# --------------------------------------------------------------------------

def reference_available():
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in ("libref_bounds.so", "bb", "bbJ"))


class Reference:
    """The reference's bounds library through oracle/ref_shim.cpp (one instance at a time)."""

    _L = None

    def __init__(self, p):
        if Reference._L is None:
            L = ctypes.CDLL(os.path.join(REF_DIR, "libref_bounds.so"))
            L.ref_taillard.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, ctypes.c_int]
            L.ref_set_instance.argtypes = [ctypes.c_int, ctypes.c_int, _i32p]
            L.ref_eval.argtypes = [_i32p]
            L.ref_weak_node.argtypes = [_i32p, ctypes.c_int, ctypes.c_int]
            L.ref_weak_children.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _i32p]
            L.ref_strong_node.argtypes = [_i32p, ctypes.c_int, ctypes.c_int]
            L.ref_strong_node_idle.argtypes = [_i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.ref_johnson_row.argtypes = [ctypes.c_int, _i32p]
            L.ref_children_batch.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, _i32p, _i32p, _i32p, _i32p,
                                             _i32p, _i32p, _i32p, _i32p]
            Reference._L = L
        p = np.ascontiguousarray(p, dtype=np.int32)
        self.m, self.n = p.shape
        self.p = p
        Reference._L.ref_set_instance(self.n, self.m, _ptr(p.ravel()))

    @staticmethod
    def taillard(idx):
        Reference(np.ones((2, 2), np.int32))  # load the library
        n = np.zeros(1, np.int32); m = np.zeros(1, np.int32)
        buf = np.zeros(500 * 20, np.int32)
        if Reference._L.ref_taillard(idx, _ptr(n), _ptr(m), _ptr(buf), buf.size) != 0:
            raise ValueError("taillard instance too large")
        return buf[: n[0] * m[0]].reshape(m[0], n[0]).copy()

    def eval(self, perm):
        return Reference._L.ref_eval(_ptr(np.ascontiguousarray(perm, dtype=np.int32)))

    def weak_node(self, sched, l1, l2):
        return Reference._L.ref_weak_node(_ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2)

    def weak_children(self, sched, l1, l2):
        cb = np.zeros(self.n, np.int32); ce = np.zeros(self.n, np.int32)
        pb = np.zeros(self.n, np.int32); pe = np.zeros(self.n, np.int32)
        Reference._L.ref_weak_children(_ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2,
                                       _ptr(cb), _ptr(ce), _ptr(pb), _ptr(pe))
        return cb, ce, pb, pe

    def strong_node(self, sched, l1, l2):
        return Reference._L.ref_strong_node(_ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2)

    def strong_node_idle(self, sched, l1, l2, unset=-1):
        """couts[1] of the reference's Johnson bornes_calculer (`unset` where it
        leaves the value untouched: at most one free job)."""
        return Reference._L.ref_strong_node_idle(_ptr(np.ascontiguousarray(sched, dtype=np.int32)), l1, l2, unset)

    def johnson_row(self, s):
        out = np.zeros(self.n, np.int32)
        Reference._L.ref_johnson_row(s, _ptr(out))
        return out

    def children_batch(self, sched, l1, l2, want_front, want_back):
        """Reference children LBs of many nodes: weak front/back of every free
        job, Johnson of the children flagged in want_front / want_back (all
        (count, n) arrays by job id; 0 where not computed)."""
        sched = np.ascontiguousarray(sched, dtype=np.int32)
        cnt, n = sched.shape
        l1 = np.ascontiguousarray(l1, dtype=np.int32)
        l2 = np.ascontiguousarray(l2, dtype=np.int32)
        wf = np.ascontiguousarray(want_front, dtype=np.int32)
        wk = np.ascontiguousarray(want_back, dtype=np.int32)
        out = [np.zeros((cnt, n), np.int32) for _ in range(4)]
        Reference._L.ref_children_batch(cnt, n, _ptr(sched), _ptr(l1), _ptr(l2), _ptr(wf), _ptr(wk),
                                        *[_ptr(o) for o in out])
        return out


def write_vrf(dirpath, name, p, ub=None):
    """Write `p` (m x n) as a VRF instance the reference can read
    (bounds/src/instance_vrf.cpp:32-69) plus its instancesVRF.data line
    (common/src/arguments.cpp:182-212)."""
    m, n = p.shape
    vdir = os.path.join(dirpath, "parameters", "vrf_parameters")
    os.makedirs(vdir, exist_ok=True)
    with open(os.path.join(vdir, name + "_Gap.txt"), "w") as f:
        f.write("%d %d\n" % (n, m))
        for j in range(n):
            f.write(" ".join("%d %d" % (k, p[k, j]) for k in range(m)) + "\n")
    with open(os.path.join(dirpath, "parameters", "instancesVRF.data"), "w") as f:
        f.write("header\n%s %d %d 1 %d 0\n" % (name, n, m, ub if ub is not None else 2147483647))


def run_reference_bb(p, ub=None, bound_mode=2, branch_mode=3, threads=0, johnson=True,
                     time_limit=None, find_all=False, timeout=3600, sorted_dfs=0, early_stop=False,
                     johnson_mode=0, sorting_criterion=-1):
    """Run the reference multicore B&B (oracle/_ref/bb or bbJ) on instance p.

    ub=None means UB=+inf.  The ini keys follow common/src/arguments.cpp:80-132
    (earlyStopJohnson, JohnsonMode, sortedDFS, sortingCriterion).  Returns the
    parsed stats dict."""
    exe = os.path.join(REF_DIR, "bbJ" if johnson else "bb")
    with tempfile.TemporaryDirectory(prefix="pbbrun_") as d:
        name = "VPBB%dx%d" % (p.shape[1], p.shape[0])
        write_vrf(d, name, np.asarray(p), ub)
        with open(os.path.join(d, "mcconfig.ini"), "w") as f:
            f.write("[problem]\nproblem = flowshop\ninstance = %s\n" % name)
            f.write("[initial]\nub = %d\n" % (0 if ub is not None else 3))
            f.write("[bb]\nsingleNode = true\nsortedDFS = %d\nsortingCriterion = %d\n"
                    % (sorted_dfs, sorting_criterion))
            f.write("boundingMode = %d\nadaptiveBranchingMode = %d\nJohnsonMode = %d\n"
                    % (bound_mode, branch_mode, johnson_mode))
            f.write("earlyStopJohnson = %s\nfindAll = %s\n" % ("true" if early_stop else "false",
                                                              "true" if find_all else "false"))
            f.write("[verbose]\nprintSolutions = false\n")
            f.write("[multicore]\nthreads = %d\nworksteal = o\n" % threads)
        env = dict(os.environ)
        if time_limit:
            env["BB_TIME_LIMIT"] = str(time_limit)
        args = [exe, "-z", "p=fsp,i=%s%s" % (name, ",o" if ub is not None else "")]
        r = subprocess.run(args, cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                           timeout=timeout, env=env)
        return parse_bb_output(r.stdout)


def parse_bb_output(text):
    out = {"raw": text}
    lines = text.splitlines()
    for i, line in enumerate(lines):
        key, _, val = line.partition(":")
        val = val.strip()
        if key == "TOTdecomposed":
            out["decomposed"] = int(val)
        elif key == "TOTjohnson LBs":
            out["johnson_bounds"] = int(val)
        elif key == "TOTsimple LBs":
            out["simple_bounds"] = int(val)
        elif key == "TOTleaves":
            out["leaves"] = int(val)
        elif key.startswith("Walltime"):
            out["walltime"] = float(val)
        elif line.startswith("Found optimal solution"):
            out["found"] = True
            out["best"] = int(lines[i + 2])
            out["perm"] = [int(x) for x in lines[i + 3].split()]
        elif line.startswith("Optimal makespan is >="):
            out["found"] = False
            out["best"] = int(line.split(">=")[1].split()[0])
    return out
