// C entry points over the reference's own bounds library (bounds/src), so the
// Python test-suite can call it through ctypes.  Test infrastructure only:
// compiled into oracle/_ref/libref_bounds.so by oracle/build_ref.py.
//
// The reference keeps the strong bound's tables in static pointers that are
// allocated once for the first instance (bounds/src/bound_fsp_strong.cpp:249-262),
// so ref_set_instance() clears those pointers before building a new instance.
#include <sstream>
#include <string>
#include <cstring>
#include <cstdio>

#include "libbounds.h"

static instance_abstract* g_inst = nullptr;
static bound_fsp_weak* g_weak = nullptr;
static bound_fsp_strong* g_strong = nullptr;
static int g_n = 0, g_m = 0;

struct shim_instance : public instance_abstract {
    shim_instance(int n, int m, const int* p) {
        std::ostringstream os;
        os << n << " " << m << " ";
        for (int i = 0; i < n * m; i++) os << p[i] << " ";
        data = new std::stringstream(os.str());
        size = n;
    }
};

extern "C" {

// Processing times of Taillard instance `taN` as produced by the reference's
// generator (bounds/src/instance_flowshop.cpp:91-101); row-major m x n.
int ref_taillard(int id, int* n, int* m, int* p, int cap) {
    char name[32];
    snprintf(name, sizeof(name), "ta%d", id);
    instance_flowshop inst(name);
    inst.data->seekg(0);
    *inst.data >> *n >> *m;
    if ((*n) * (*m) > cap) return -1;
    for (int i = 0; i < (*n) * (*m); i++) *inst.data >> p[i];
    return 0;
}

int ref_set_instance(int n, int m, const int* p) {
    g_n = n; g_m = m;
    g_inst = new shim_instance(n, m, p);   // leaked on purpose: the bounds keep a pointer
    bound_fsp_strong::tempsJob = NULL;
    bound_fsp_strong::tabJohnson = NULL;
    bound_fsp_strong::tempsLag = NULL;
    bound_fsp_strong::minTempsDep = NULL;
    bound_fsp_strong::minTempsArr = NULL;
    bound_fsp_strong::machine = NULL;
    g_weak = new bound_fsp_weak();
    g_weak->set_instance(g_inst);
    g_weak->init();
    g_weak->branchingMode = 1;
    g_strong = new bound_fsp_strong();
    g_strong->set_instance(g_inst);
    g_strong->init();
    g_strong->branchingMode = 1;
    g_strong->earlyExit = 0;
    g_strong->machinePairs = 0;
    return 0;
}

int ref_eval(const int* perm) {
    return g_weak->evalSolution(const_cast<int*>(perm));
}

int ref_weak_node(const int* sched, int l1, int l2) {
    int c[2] = {0, 0};
    g_weak->bornes_calculer(const_cast<int*>(sched), l1, l2, c, -1);
    return c[0];
}

void ref_weak_children(const int* sched, int l1, int l2, int* cb, int* ce, int* pb, int* pe) {
    g_weak->boundChildren(const_cast<int*>(sched), l1, l2, cb, ce, pb, pe);
}

int ref_strong_node(const int* sched, int l1, int l2) {
    int c[2] = {0, 0};
    int tmp[1024];
    memcpy(tmp, sched, g_n * sizeof(int));
    g_strong->bornes_calculer(tmp, l1, l2, c, -1);
    return c[0];
}

// couts[1] of bound_fsp_strong::bornes_calculer (idle time of the fixed
// jobs' schedules); `unset` is returned where the reference leaves it as it was.
int ref_strong_node_idle(const int* sched, int l1, int l2, int unset) {
    int c[2] = {0, unset};
    int tmp[1024];
    memcpy(tmp, sched, g_n * sizeof(int));
    g_strong->bornes_calculer(tmp, l1, l2, c, -1);
    return c[1];
}

// Johnson order of machine pair s (bounds/src/bound_fsp_strong.cpp:343-354).
void ref_johnson_row(int s, int* out) {
    memcpy(out, bound_fsp_strong::tabJohnson + s * g_n, g_n * sizeof(int));
}

// Reference children bounds of `count` nodes (schedule row-major count x n,
// node i fixes sched[0..l1[i]] in front and sched[l2[i]..n) at the back):
// weak front / back LBs of every free job (boundChildren), and the Johnson LB
// of each child whose entry in want_front / want_back is nonzero, computed as
// ivm_bound::computeStrongBounds does (multicore/src/ivm_bound.cpp:141-195):
// the child's job swapped into the fill slot, bornes_calculer with no early
// exit.  All outputs by job id, 0 where not computed.
void ref_children_batch(int count, int n, const int* sched, const int* l1, const int* l2, const int* want_front,
                        const int* want_back, int* wb, int* we, int* sb, int* se) {
    int s[1024], pb[1024], pe[1024];
    for (int i = 0; i < count; i++) {
        const int* sc = sched + (size_t)i * n;
        const int a = l1[i], b = l2[i];
        memcpy(s, sc, n * sizeof(int));
        g_weak->boundChildren(s, a, b, wb + (size_t)i * n, we + (size_t)i * n, pb, pe);
        for (int j = 0; j < n; j++) { sb[(size_t)i * n + j] = 0; se[(size_t)i * n + j] = 0; }
        for (int side = 0; side < 2; side++) {
            const int* want = (side == 0 ? want_front : want_back) + (size_t)i * n;
            int* out = (side == 0 ? sb : se) + (size_t)i * n;
            const int L1 = a + (side == 0 ? 1 : 0), L2 = b - (side == 0 ? 0 : 1);
            const int fill = side == 0 ? L1 : L2;
            for (int q = a + 1; q < b; q++) {
                const int job = sc[q];
                if (!want[job]) continue;
                memcpy(s, sc, n * sizeof(int));
                const int t = s[fill]; s[fill] = s[q]; s[q] = t;
                int c[2] = {0, 0};
                g_strong->bornes_calculer(s, L1, L2, c, -1);
                out[job] = c[0];
            }
        }
    }
}

}
