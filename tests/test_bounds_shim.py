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
