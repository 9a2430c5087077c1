#!/usr/bin/env python3
"""Build the reference's own CPU code into oracle/_ref/ (test infrastructure).

This recipe compiles jangmys/PBBPerm sources where they lie (read-only tree:
PBB_REFERENCE, else a `reference` directory beside the repository) from a scratch copy
under /tmp, with g++ invoked directly on the source files (the reference's own
makefiles are not used).  Outputs, all git-ignored:

  oracle/_ref/libref_bounds.so   bounds/src (weak + strong FSP bounds, Taillard
                                 and VRF instance readers) + oracle/ref_shim.cpp
  oracle/_ref/testBounds         bounds/test/testBounds.cpp (known-answer tool)
  oracle/_ref/bb                 multicore/ B&B, weak re-evaluation as shipped
  oracle/_ref/bbJ                multicore/ B&B with the Johnson call restored
  oracle/_ref/abstract_driver    oracle/abstract_driver.cpp: the engine's bounds adapter
                                 derived from the reference's bound_abstract (its header and
                                 bounds/src/bound_abstract.cpp), linked with libpbbperm.so

Patches applied to the scratch copy (the shipped tree does not compile):
  P1 common/include/arguments.h + common/src/arguments.cpp: declare/define
     `arguments::init_solution` (used at common/src/pbab.cpp:165); value 0 =
     identity root permutation, no random IG start.
  P2 multicore/include/sequentialbb.h:25: declare `bool next();` (the
     definition at multicore/src/sequentialbb.cpp:110 takes no argument).
  P3 common/include/solution.h:24: restore `volatile bool newBest` (read at
     multicore/src/matrix_controller.cpp:515).
  P4 (bbJ only) multicore/src/ivm_bound.cpp:170: call bound[STRONG] instead of
     bound[WEAK] in computeStrongBounds (the Johnson call is commented out at
     :171).
  P5 multicore/src/main.cpp: when BB_TIME_LIMIT (seconds) is set, a detached
     thread calls matrix_controller::interruptExploration() after that time so
     that a fixed-window nodes/s figure is printed.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference tree: PBB_REFERENCE, else a `reference` directory beside the repository
REF = os.environ.get("PBB_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def _patch(path, old, new, count=1):
    with open(path) as f:
        s = f.read()
    if s.count(old) < 1:
        raise RuntimeError("patch anchor not found in %s: %r" % (path, old))
    s = s.replace(old, new, count)
    with open(path, "w") as f:
        f.write(s)


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-4000:])
        raise RuntimeError("command failed: %s" % " ".join(cmd))


def build(verbose=False):
    if not os.path.isdir(os.path.join(REF, "bounds")):
        raise FileNotFoundError("reference tree not found at %s" % REF)
    os.makedirs(OUT, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="pbbref_")
    try:
        for d in ("bounds", "common", "multicore", "heuristic"):
            shutil.copytree(os.path.join(REF, d), os.path.join(tmp, d))
        # P1
        _patch(os.path.join(tmp, "common/include/arguments.h"),
               "static int initial_ub;", "static int initial_ub;\n    static int init_solution;")
        _patch(os.path.join(tmp, "common/src/arguments.cpp"),
               "int arguments::init_mode = 1;", "int arguments::init_mode = 1;\nint arguments::init_solution = 0;")
        # P2
        _patch(os.path.join(tmp, "multicore/include/sequentialbb.h"),
               "bool next(bool &foundNew);", "bool next();")
        # P3
        _patch(os.path.join(tmp, "common/include/solution.h"),
               "// volatile bool newBest;", "volatile bool newBest = false;")
        # P5
        mainf = os.path.join(tmp, "multicore/src/main.cpp")
        _patch(mainf, '#include "../include/sequentialbb.h"',
               '#include "../include/sequentialbb.h"\n#include <thread>\n#include <chrono>\n#include <cstdlib>')
        _patch(mainf, "matrix_controller *mc = new matrix_controller(pbb);\n\t\t\tmc->initFullInterval();",
               "matrix_controller *mc = new matrix_controller(pbb);\n"
               "\t\t\tif (getenv(\"BB_TIME_LIMIT\")) {\n"
               "\t\t\t\tdouble lim = atof(getenv(\"BB_TIME_LIMIT\"));\n"
               "\t\t\t\tstd::thread([mc, lim]() { std::this_thread::sleep_for(std::chrono::duration<double>(lim));"
               " mc->interruptExploration(); }).detach();\n"
               "\t\t\t}\n"
               "\t\t\tmc->initFullInterval();")

        inc = ["-I", os.path.join(tmp, "bounds/include"), "-I", os.path.join(tmp, "common/include"),
               "-I", os.path.join(tmp, "multicore/include"), "-I", os.path.join(tmp, "heuristic/include")]
        flags = ["-O3", "-std=c++14", "-w", "-fPIC"]
        bsrc = [os.path.join(tmp, "bounds/src", f) for f in sorted(os.listdir(os.path.join(tmp, "bounds/src")))]

        # libbounds + our C shim
        _run(["g++"] + flags + ["-shared", "-o", os.path.join(OUT, "libref_bounds.so"),
                                os.path.join(HERE, "ref_shim.cpp")] + bsrc + inc + ["-lm"], tmp)
        # testBounds
        _run(["g++"] + flags + ["-o", os.path.join(OUT, "testBounds"),
                                os.path.join(tmp, "bounds/test/testBounds.cpp")] + bsrc + inc + ["-lm"], tmp)
        # multicore bb (as shipped) and bbJ (P4)
        common = [os.path.join(tmp, "common/src", f) for f in
                  ("arguments.cpp", "pbab.cpp", "solution.cpp", "subproblem.cpp", "ttime.cpp")]
        heur = [os.path.join(tmp, "heuristic/src", f) for f in sorted(os.listdir(os.path.join(tmp, "heuristic/src")))]
        mc = [os.path.join(tmp, "multicore/src", f) for f in
              ("main.cpp", "sequentialbb.cpp", "bbthread.cpp", "matrix_controller.cpp", "ivm.cpp", "ivm_bound.cpp")]
        srcs = bsrc + common + heur + mc
        _run(["g++"] + flags + ["-o", os.path.join(OUT, "bb")] + srcs + inc + ["-lpthread", "-lm", "-ldl"], tmp)
        _patch(os.path.join(tmp, "multicore/src/ivm_bound.cpp"),
               "bound[WEAK]->bornes_calculer(node->schedule, _limit1, _limit2, costs, arguments::earlyStopJohnson?local_best:-1);",
               "bound[STRONG]->bornes_calculer(node->schedule, _limit1, _limit2, costs, arguments::earlyStopJohnson?local_best:-1);")
        _run(["g++"] + flags + ["-o", os.path.join(OUT, "bbJ")] + srcs + inc + ["-lpthread", "-lm", "-ldl"], tmp)
        # the bounds adapter as a bound_abstract (needs the engine library built)
        pkg = os.path.join(os.path.dirname(HERE), "pbbperm_b200")
        if os.path.exists(os.path.join(pkg, "libpbbperm.so")):
            _run(["g++", "-O1", "-std=c++17", "-o", os.path.join(OUT, "abstract_driver"),
                  os.path.join(HERE, "abstract_driver.cpp"), os.path.join(tmp, "bounds/src/bound_abstract.cpp"),
                  "-I", os.path.join(tmp, "bounds/include"), "-I", os.path.join(os.path.dirname(HERE), "include"),
                  "-L", pkg, "-lpbbperm", "-Wl,-rpath,$ORIGIN/../../pbbperm_b200"], tmp)
        if verbose:
            print("reference checker built into", OUT)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    build(verbose=True)
