"""include/pbbperm_bounds.hpp: the reference's bound_abstract member functions
(set_instance from an instance_abstract-like stream, bornes_calculer,
boundChildren, evalSolution) over the C ABI.  A small C++ program written the
way the reference's engines call their bounds is compiled against the header
and checked against the oracle (bit-exact integers)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import Oracle
from pbbperm_b200.instances import synthetic_instance

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "pbbperm_b200")

DRIVER = r"""
#include <cstdio>
#include <sstream>
#include <vector>
#include "pbbperm_bounds.hpp"

struct instance_abstract { int size; std::stringstream* data; };   // as bounds/include/instance_abstract.h

int main()
{
    int n, m, count;
    if (scanf("%d %d", &n, &m) != 2) return 2;
    std::stringstream data;
    data << n << " " << m << " ";
    for (int i = 0; i < n * m; i++) { int v; if (scanf("%d", &v) != 1) return 2; data << v << " "; }
    instance_abstract inst{n, &data};
    pbbperm::bound_fsp_gpu weak(pbbperm::bound_fsp_gpu::WEAK), strong(pbbperm::bound_fsp_gpu::STRONG);
    weak.set_instance(&inst);
    strong.set_instance(&inst);
    weak.init();
    strong.init();
    if (scanf("%d", &count) != 1) return 2;
    std::vector<int> perm(n), cb(n), ce(n), pb(n), pe(n);
    for (int c = 0; c < count; c++) {
        int l1, l2;
        if (scanf("%d %d", &l1, &l2) != 2) return 2;
        for (int i = 0; i < n; i++) if (scanf("%d", &perm[i]) != 1) return 2;
        int cw[2] = {0, 0}, cs[2] = {0, 0};
        weak.bornes_calculer(perm.data(), l1, l2, cw, 1 << 30);
        strong.bornes_calculer(perm.data(), l1, l2, cs, 1 << 30);
        printf("%d %d %d\n", cw[0], cs[0], strong.evalSolution(perm.data()));
        weak.boundChildren(perm.data(), l1, l2, cb.data(), ce.data(), pb.data(), pe.data());
        for (int j = 0; j < n; j++) printf("%d ", cb[j]);
        printf("\n");
        for (int j = 0; j < n; j++) printf("%d ", ce[j]);
        printf("\n");
        strong.boundChildren(perm.data(), l1, l2, cb.data(), ce.data(), nullptr, nullptr);
        for (int j = 0; j < n; j++) printf("%d ", cb[j]);
        printf("\n");
        for (int j = 0; j < n; j++) printf("%d ", ce[j]);
        printf("\n");
    }
    weak.freeMem();
    strong.freeMem();
    return 0;
}
"""


def compile_driver(tmp_path, syntax_only=False):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    cmd = ["g++", "-std=c++17", "-O1", "-I", INC, str(src)]
    cmd += ["-fsyntax-only"] if syntax_only else ["-o", str(exe), "-L", LIBDIR, "-lpbbperm",
                                                  "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    return exe


def test_header_compiles_against_the_bound_abstract_calls(tmp_path):
    compile_driver(tmp_path, syntax_only=True)


@pytest.mark.gpu
def test_shim_matches_the_oracle(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libpbbperm.so")):
        pytest.skip("library not built")
    exe = compile_driver(tmp_path)
    n, m = 20, 10
    p = synthetic_instance(61, n, m)
    O = Oracle(p)
    rng = np.random.default_rng(61)
    nodes = []
    for _ in range(25):
        perm = rng.permutation(n).astype(np.int32)
        nf = int(rng.integers(0, n))
        nb = int(rng.integers(0, n - nf + 1))
        l1, l2 = nf - 1, n - nb
        if l1 < l2:
            nodes.append((l1, l2, perm))
    text = "%d %d\n%s\n%d\n" % (n, m, " ".join(str(v) for v in p.reshape(-1)), len(nodes))
    text += "".join("%d %d %s\n" % (l1, l2, " ".join(map(str, perm))) for l1, l2, perm in nodes)
    r = subprocess.run([str(exe)], input=text, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 5 * len(nodes)
    for i, (l1, l2, perm) in enumerate(nodes):
        w, s, mk = map(int, lines[5 * i].split())
        assert w == O.weak_node(perm, l1, l2)
        assert s == O.strong_node(perm, l1, l2)
        assert mk == O.eval(perm)
        cb, ce, _, _ = O.weak_children(perm, l1, l2)
        assert [int(x) for x in lines[5 * i + 1].split()] == list(cb)
        assert [int(x) for x in lines[5 * i + 2].split()] == list(ce)
        assert [int(x) for x in lines[5 * i + 3].split()] == list(O.strong_children(perm, l1, l2, True))
        assert [int(x) for x in lines[5 * i + 4].split()] == list(O.strong_children(perm, l1, l2, False))


def _reference_tree():
    ref = os.environ.get("PBB_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    return ref if os.path.isdir(os.path.join(ref, "bounds", "include")) else None


def test_adapter_derives_from_the_reference_bound_abstract():
    """With the reference's bound_abstract.h included first, the header's
    bound_fsp_gpu_abstract derives from it (compile check)."""
    ref = _reference_tree()
    if ref is None or not shutil.which("g++"):
        pytest.skip("reference tree or g++ not available")
    src = os.path.join(ROOT, "oracle", "abstract_driver.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ref, "bounds", "include"),
                        "-I", INC, src], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout


@pytest.mark.gpu
def test_adapter_through_the_reference_base_class():
    """oracle/_ref/abstract_driver (built with the reference's bound_abstract)
    calls the GPU bounds through bound_abstract pointers: node LBs, couts[1],
    weak children with their priorities, Johnson children -- all equal to the
    oracle's."""
    exe = os.path.join(ROOT, "oracle", "_ref", "abstract_driver")
    if not os.path.exists(exe):
        pytest.skip("abstract driver not built (oracle/build_ref.py)")
    n, m = 18, 9
    p = synthetic_instance(62, n, m)
    O = Oracle(p)
    rng = np.random.default_rng(62)
    nodes = []
    for _ in range(30):
        perm = rng.permutation(n).astype(np.int32)
        nf = int(rng.integers(0, n))
        nb = int(rng.integers(0, n - nf + 1))
        l1, l2 = nf - 1, n - nb
        if l1 < l2:
            nodes.append((l1, l2, perm))
    text = "%d %d\n%s\n%d\n" % (n, m, " ".join(str(v) for v in p.reshape(-1)), len(nodes))
    text += "".join("%d %d %s\n" % (l1, l2, " ".join(map(str, perm))) for l1, l2, perm in nodes)
    r = subprocess.run([exe], input=text, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 7 * len(nodes)
    for i, (l1, l2, perm) in enumerate(nodes):
        w, s, idle, mk = map(int, lines[7 * i].split())
        assert w == O.weak_node(perm, l1, l2) and s == O.strong_node(perm, l1, l2) and mk == O.eval(perm)
        assert idle == (O.strong_node_idle(perm, l1, l2) if l2 - l1 > 2 else -1)
        cb, ce, pb_, pe_ = O.weak_children(perm, l1, l2)
        got = [[int(x) for x in lines[7 * i + r].split()] for r in range(1, 7)]
        free = perm[l1 + 1:l2]
        assert got[0] == list(cb) and got[1] == list(ce)
        assert [got[2][j] for j in free] == list(pb_[free]) and [got[3][j] for j in free] == list(pe_[free])
        assert got[4] == list(O.strong_children(perm, l1, l2, True))
        assert got[5] == list(O.strong_children(perm, l1, l2, False))
