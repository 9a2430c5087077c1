/*
 * pbbperm_bounds.hpp -- the reference's bounds-library interface over the C ABI.
 *
 * The reference's branch-and-bound engines call their bounds through
 * `struct bound_abstract` (bounds/include/bound_abstract.h:6-34), implemented by
 * bound_fsp_weak (bounds/src/bound_fsp_weak.cpp) and bound_fsp_strong
 * (bounds/src/bound_fsp_strong.cpp), with the instance handed over as
 * `instance_abstract {int size; std::stringstream* data}` holding
 * "n m p[0][0..n) ... p[m-1][0..n)" (bounds/src/instance_flowshop.cpp:91-101).
 *
 * pbbperm::bound_fsp_gpu offers the same member functions, computed by
 * pbb_bound_children_ex on the GPU.  When the reference's bound_abstract.h is
 * included before this header, pbbperm::bound_fsp_gpu_abstract also derives
 * from the reference's bound_abstract, so it drops into the arrays the
 * engines hold (`bound_abstract* bound[2]`, multicore/include/ivm_bound.h);
 * the program then links the reference's bound_abstract.cpp (set_instance and
 * the destructor are defined there).
 *
 * Behaviour, member by member:
 *   - bornes_calculer(perm, l1, l2, couts, best): couts[0] = the node's LB;
 *     the strong flavour also sets couts[1] = the idle time of the fixed jobs'
 *     schedules (as the reference, 0 when nothing is fixed at the back) and,
 *     with at most one free job, returns the schedule's makespan leaving
 *     couts[1] as it was.  `best` is accepted: the early Johnson exit only
 *     changes the value of a child that is pruned anyway, so it is not taken;
 *   - bornes_calculer(perm, l1, l2): empty, as in both reference bounds;
 *   - boundChildren (weak): costs and idle-time priorities of every free job
 *     at the front and at the back, by job id, 0 for fixed jobs; with
 *     branchingMode <= 0 only the front side is written, as the reference
 *     (bound_fsp_weak.cpp:209-216);
 *   - boundChildren (strong): the Johnson LBs of the same children (the
 *     reference declares this member for the strong bound but gathers those
 *     values one child at a time); priorities are the children's weak ones;
 *   - evalSolution: makespan of a complete permutation.
 * One GPU call per member call: this adapter is for drop-in use and parity
 * checks; batched work should call pbb_bound_children(_ex) directly.
 */
#ifndef PBBPERM_BOUNDS_HPP
#define PBBPERM_BOUNDS_HPP

#include <algorithm>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "pbbperm.h"

namespace pbbperm {

class bound_fsp_gpu {
public:
    enum Kind { WEAK = 0, STRONG = 1 };

    int branchingMode = 1;   // as bound_fsp_weak::branchingMode (bounds/include/bound_fsp_weak.h:13)

    explicit bound_fsp_gpu(Kind kind, int device = 0, int johnson_mode = 0)
        : kind_(kind), device_(device), johnson_mode_(johnson_mode) {}

    /* bound_abstract::set_instance: any type with a std::stringstream* `data`
     * holding "n m p..." (machine-major). */
    template <class Instance>
    void set_instance(Instance* in)
    {
        std::stringstream s(in->data->str());
        int n = 0, m = 0;
        if (!(s >> n >> m) || n < 1 || m < 1) throw std::runtime_error("bound_fsp_gpu: bad instance data");
        p_.assign((size_t)n * m, 0);
        for (auto& v : p_)
            if (!(s >> v)) throw std::runtime_error("bound_fsp_gpu: truncated instance data");
        n_ = n;
        m_ = m;
    }

    void init() {}
    void freeMem() {}

    void bornes_calculer(int permutation[], int limite1, int limite2, int* couts, int /*best*/)
    {
        int32_t nw = 0, ns = 0, idle = 0;
        pbb_bound_out o;
        std::memset(&o, 0, sizeof(o));
        o.node_weak = &nw;
        o.node_strong = &ns;
        if (kind_ == STRONG) o.strong_idle = &idle;
        call(permutation, limite1, limite2, o);
        couts[0] = kind_ == WEAK ? nw : ns;
        if (kind_ == STRONG && limite2 - limite1 > 2) couts[1] = idle;
    }
    void bornes_calculer(int*, int, int) {}

    void boundChildren(int* schedule, int limit1, int limit2, int* costsBegin, int* costsEnd, int* prioBegin,
                       int* prioEnd)
    {
        std::vector<int32_t> b((size_t)n_), e((size_t)n_), pb((size_t)n_), pe((size_t)n_);
        pbb_bound_out o;
        std::memset(&o, 0, sizeof(o));
        if (kind_ == WEAK) {
            o.weak_begin = b.data();
            o.weak_end = e.data();
        } else {
            o.strong_begin = b.data();
            o.strong_end = e.data();
        }
        o.prio_begin = pb.data();
        o.prio_end = pe.data();
        call(schedule, limit1, limit2, o);
        const bool both = kind_ == STRONG || branchingMode > 0;
        for (int j = 0; j < n_; j++) {
            if (costsBegin) costsBegin[j] = b[j];
            if (both && costsEnd) costsEnd[j] = e[j];
        }
        // priorities of the free jobs only (the reference writes no others)
        for (int i = limit1 + 1; i < limit2; i++) {
            const int j = schedule[i];
            if (prioBegin) prioBegin[j] = pb[j];
            if (both && prioEnd) prioEnd[j] = pe[j];
        }
    }

    /* makespan of a complete permutation (bound_fsp_strong.cpp:563-580) */
    int evalSolution(int* permut) const
    {
        std::vector<int> t((size_t)m_, 0);
        for (int i = 0; i < n_; i++) {
            const int j = permut[i];
            t[0] += p_[(size_t)j];
            for (int k = 1; k < m_; k++) t[k] = std::max(t[k], t[k - 1]) + p_[(size_t)k * n_ + j];
        }
        return t[m_ - 1];
    }

    int jobs() const { return n_; }
    int machines() const { return m_; }

private:
    void call(const int* sched, int l1, int l2, const pbb_bound_out& o)
    {
        if (n_ < 1) throw std::runtime_error("bound_fsp_gpu: set_instance first");
        pbb_instance inst{n_, m_, p_.data()};
        std::vector<int32_t> s(sched, sched + n_);
        const int32_t a = l1, b = l2;
        const int rc = pbb_bound_children_ex(&inst, johnson_mode_, device_, 1, s.data(), &a, &b, &o);
        if (rc != PBB_OK) throw std::runtime_error(std::string("pbb_bound_children_ex: ") + pbb_last_error());
    }

    Kind kind_;
    int device_, johnson_mode_;
    int n_ = 0, m_ = 0;
    std::vector<int32_t> p_;
};

}  // namespace pbbperm

#endif /* PBBPERM_BOUNDS_HPP */

/* The reference's own base class is visible (its header guard): the drop-in
 * bound_abstract implementation. */
#if defined(BOUND_ABSTRACT_H) && !defined(PBBPERM_BOUNDS_ABSTRACT_HPP)
#define PBBPERM_BOUNDS_ABSTRACT_HPP
namespace pbbperm {

struct bound_fsp_gpu_abstract : public bound_abstract {
    explicit bound_fsp_gpu_abstract(bound_fsp_gpu::Kind kind, int device = 0, int johnson_mode = 0)
        : impl(kind, device, johnson_mode) {}
    /* set_instance (the reference's, non-virtual) stores the instance; init
     * reads it, as the reference's bounds do */
    void init() override { impl.set_instance(instance); }
    void bornes_calculer(int permutation[], int limite1, int limite2, int* couts, int best) override
    {
        impl.bornes_calculer(permutation, limite1, limite2, couts, best);
    }
    void bornes_calculer(int permutation[], int limite1, int limite2) override
    {
        impl.bornes_calculer(permutation, limite1, limite2);
    }
    void boundChildren(int* schedule, int limit1, int limit2, int* costsBegin, int* costsEnd, int* prioBegin,
                       int* prioEnd) override
    {
        impl.boundChildren(schedule, limit1, limit2, costsBegin, costsEnd, prioBegin, prioEnd);
    }
    void freeMem() override {}
    int evalSolution(int* permut) override { return impl.evalSolution(permut); }
    ~bound_fsp_gpu_abstract() override {}

    bound_fsp_gpu impl;
};

}  // namespace pbbperm
#endif
