/*
 * pbbperm_bounds.hpp -- the reference's bounds-library interface over the C ABI.
 *
 * The reference's branch-and-bound engines call their bounds through
 * `struct bound_abstract` (bounds/include/bound_abstract.h:6-34), implemented by
 * bound_fsp_weak (bounds/src/bound_fsp_weak.cpp) and bound_fsp_strong
 * (bounds/src/bound_fsp_strong.cpp), with the instance handed over as
 * `instance_abstract {int size; std::stringstream* data}` holding
 * "n m p[0][0..n) ... p[m-1][0..n)" (bounds/src/instance_flowshop.cpp:91-101).
 * pbbperm::bound_fsp_gpu offers the same member functions, computed by
 * pbb_bound_children on the GPU, so code written against bound_abstract can
 * switch by deriving a thin wrapper (or by templating on the bound type).
 *
 * Differences, all documented by the C ABI:
 *   - bornes_calculer never exits early (the reference's earlyStopJohnson =
 *     false; `best` is accepted and ignored);
 *   - the idle-time priorities (prioBegin / prioEnd, and couts[1] of the strong
 *     bound) are not computed and are set to 0;
 *   - boundChildren always fills both sides (the reference's weak bound skips
 *     the END side when its branching rule is fixed).
 * One GPU call per member call: this adapter is for drop-in use and parity
 * checks; batched work should call pbb_bound_children directly.
 */
#ifndef PBBPERM_BOUNDS_HPP
#define PBBPERM_BOUNDS_HPP

#include <algorithm>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "pbbperm.h"

namespace pbbperm {

class bound_fsp_gpu {
public:
    enum Kind { WEAK = 0, STRONG = 1 };

    explicit bound_fsp_gpu(Kind kind, int device = 0, int johnson_mode = 0)
        : kind_(kind), device_(device), johnson_mode_(johnson_mode) {}

    /* bound_abstract::set_instance: any type with `size` and a
     * std::stringstream* `data` holding "n m p..." (machine-major). */
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

    /* bound_fsp_weak / bound_fsp_strong ::bornes_calculer(perm, l1, l2, couts, best):
     * couts[0] = the node's LB (for the strong bound with at most one free job,
     * the makespan of the schedule as given). */
    void bornes_calculer(int permutation[], int limite1, int limite2, int* couts, int /*best*/)
    {
        std::vector<int32_t> nw(1), ns(1);
        call(permutation, limite1, limite2, nullptr, nullptr, nullptr, nullptr, nw.data(), ns.data());
        couts[0] = kind_ == WEAK ? nw[0] : ns[0];
        if (kind_ == STRONG && limite2 - limite1 > 2) couts[1] = 0;
    }
    void bornes_calculer(int*, int, int) {}

    /* bound_fsp_weak::boundChildren: LBs of every free job appended at the
     * front (costsBegin) and at the back (costsEnd), indexed by job id, 0 for
     * fixed jobs.  The strong flavour returns the Johnson LBs of the same
     * children (what ivm_bound::computeStrongBounds gathers one by one). */
    void boundChildren(int* schedule, int limit1, int limit2, int* costsBegin, int* costsEnd, int* prioBegin,
                       int* prioEnd)
    {
        std::vector<int32_t> b((size_t)n_), e((size_t)n_);
        if (kind_ == WEAK)
            call(schedule, limit1, limit2, b.data(), e.data(), nullptr, nullptr, nullptr, nullptr);
        else
            call(schedule, limit1, limit2, nullptr, nullptr, b.data(), e.data(), nullptr, nullptr);
        for (int j = 0; j < n_; j++) {
            if (costsBegin) costsBegin[j] = b[j];
            if (costsEnd) costsEnd[j] = e[j];
            if (prioBegin) prioBegin[j] = 0;
            if (prioEnd) prioEnd[j] = 0;
        }
    }

    /* evalSolution: makespan of a complete permutation (host recurrence, as
     * bound_fsp_strong::evalSolution bounds/src/bound_fsp_strong.cpp:563-580). */
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
    void call(const int* sched, int l1, int l2, int32_t* wb, int32_t* we, int32_t* sb, int32_t* se, int32_t* nw,
              int32_t* ns)
    {
        if (n_ < 1) throw std::runtime_error("bound_fsp_gpu: set_instance first");
        pbb_instance inst{n_, m_, p_.data()};
        std::vector<int32_t> s(sched, sched + n_);
        const int32_t a = l1, b = l2;
        const int rc = pbb_bound_children(&inst, johnson_mode_, device_, 1, s.data(), &a, &b, wb, we, sb, se, nw, ns);
        if (rc != PBB_OK) throw std::runtime_error(std::string("pbb_bound_children: ") + pbb_last_error());
    }

    Kind kind_;
    int device_, johnson_mode_;
    int n_ = 0, m_ = 0;
    std::vector<int32_t> p_;
};

}  // namespace pbbperm

#endif /* PBBPERM_BOUNDS_HPP */
