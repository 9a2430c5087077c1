// Test driver (built by oracle/build_ref.py into oracle/_ref/abstract_driver):
// pbbperm::bound_fsp_gpu_abstract compiled against the reference's own
// bound_abstract (bounds/include/bound_abstract.h) and linked with its
// bound_abstract.cpp, used the way multicore/src/ivm_bound.cpp uses its
// bounds: through `bound_abstract* bound[2]`, set_instance then init.
// Reads "n m p..." then count and nodes "l1 l2 perm..." on stdin; prints per
// node the weak and Johnson node LBs with couts[1], then the weak children
// (costs and priorities, both sides) and the Johnson children.
#include <cstdio>
#include <sstream>
#include <vector>

#include "bound_abstract.h"
#include "pbbperm_bounds.hpp"

int main()
{
    int n, m, count;
    if (scanf("%d %d", &n, &m) != 2) return 2;
    std::stringstream data;
    data << n << " " << m << " ";
    for (int i = 0; i < n * m; i++) {
        int v;
        if (scanf("%d", &v) != 1) return 2;
        data << v << " ";
    }
    instance_abstract inst;
    inst.size = n;
    inst.data = &data;
    bound_abstract* bound[2];
    bound[0] = new pbbperm::bound_fsp_gpu_abstract(pbbperm::bound_fsp_gpu::WEAK);
    bound[1] = new pbbperm::bound_fsp_gpu_abstract(pbbperm::bound_fsp_gpu::STRONG);
    for (int k = 0; k < 2; k++) {
        bound[k]->set_instance(&inst);
        bound[k]->init();
    }
    if (scanf("%d", &count) != 1) return 2;
    std::vector<int> perm(n), cb(n), ce(n), pb(n), pe(n);
    for (int c = 0; c < count; c++) {
        int l1, l2;
        if (scanf("%d %d", &l1, &l2) != 2) return 2;
        for (int i = 0; i < n; i++)
            if (scanf("%d", &perm[i]) != 1) return 2;
        int cw[2] = {0, 0}, cs[2] = {0, -1};
        bound[0]->bornes_calculer(perm.data(), l1, l2, cw, -1);
        bound[1]->bornes_calculer(perm.data(), l1, l2, cs, -1);
        printf("%d %d %d %d\n", cw[0], cs[0], cs[1], bound[1]->evalSolution(perm.data()));
        std::fill(pb.begin(), pb.end(), 0);
        std::fill(pe.begin(), pe.end(), 0);
        bound[0]->boundChildren(perm.data(), l1, l2, cb.data(), ce.data(), pb.data(), pe.data());
        for (int* v : {cb.data(), ce.data(), pb.data(), pe.data()}) {
            for (int j = 0; j < n; j++) printf("%d ", v[j]);
            printf("\n");
        }
        bound[1]->boundChildren(perm.data(), l1, l2, cb.data(), ce.data(), nullptr, nullptr);
        for (int* v : {cb.data(), ce.data()}) {
            for (int j = 0; j < n; j++) printf("%d ", v[j]);
            printf("\n");
        }
    }
    for (int k = 0; k < 2; k++) {
        bound[k]->freeMem();
        delete bound[k];
    }
    return 0;
}
