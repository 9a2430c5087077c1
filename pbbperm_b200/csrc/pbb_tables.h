// Instance tables built on the host (shared by the engine and the pool).
#pragma once
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "pbb_types.h"
#include "../../include/pbbperm.h"

namespace pbbh {
void set_error(const char* msg);
}

namespace pbbt {

inline int fail(int code, const char* msg)
{
    pbbh::set_error(msg);
    return code;
}

// ---------------------------------------------------------------------------
// instance tables
// ---------------------------------------------------------------------------
struct HostTables {
    int n = 0, m = 0, P = 0, Ppad = 0;
    std::vector<int> p, min_arr, min_dep;
    std::vector<unsigned long long> je;
    std::vector<unsigned char> pm0, pm1, posj;
};

// Johnson's rule with the reference's tie order: keys (group, value); group 1
// (first machine strictly shorter) ascending by p_a + lag, then group 2
// descending by p_b + lag; equal keys stay in the order left by a Hoare
// partition quicksort that pivots on the first element
// (bounds/src/bound_fsp_strong.cpp:359-436).  The order among ties changes
// the bound's value, so the partition scheme is part of the contract.
struct JohnsonKeys {
    std::vector<int> grp, val;
    bool before(int x, int y) const
    {
        if (grp[x] != grp[y]) return grp[x] < grp[y];
        return grp[x] == 1 ? val[x] < val[y] : val[x] > val[y];
    }
    bool after(int x, int y) const
    {
        if (grp[x] != grp[y]) return grp[x] > grp[y];
        return grp[x] == 1 ? val[x] > val[y] : val[x] < val[y];
    }
};

inline void hoare_sort(const JohnsonKeys& K, std::vector<int>& v, int lo, int hi)
{
    while (lo < hi) {
        const int pivot = v[lo];
        int i = lo - 1, j = hi + 1;
        while (true) {
            do { --j; } while (K.after(v[j], pivot));
            do { ++i; } while (K.before(v[i], pivot));
            if (i >= j) break;
            std::swap(v[i], v[j]);
        }
        hoare_sort(K, v, lo, j);
        lo = j + 1;
    }
}

inline int build_tables(const pbb_instance* inst, int johnson_mode, HostTables& H)
{
    if (!inst || !inst->p) return fail(PBB_E_INVAL, "instance is NULL");
    const int n = inst->n_jobs, m = inst->n_machines;
    if (n < 2 || n > PBB_MAX_JOBS) return fail(PBB_E_INVAL, "n_jobs must be in [2, 64]");
    if (m < 2 || m > PBB_MAX_MACHINES) return fail(PBB_E_INVAL, "n_machines must be in [2, 32]");
    if (johnson_mode < 0 || johnson_mode > 2) return fail(PBB_E_UNSUPPORTED, "JohnsonMode must be 0, 1 or 2");
    H.n = n; H.m = m;
    H.p.assign(inst->p, inst->p + n * m);
    long long total = 0;
    for (int j = 0; j < n; j++) {
        long long s = 0;
        for (int k = 0; k < m; k++) {
            const int v = H.p[k * n + j];
            if (v < 0 || v > 65535) return fail(PBB_E_INVAL, "processing times must be in [0, 65535]");
            s += v;
        }
        if (s > 32767) return fail(PBB_E_INVAL, "a job's total processing time must be <= 32767");
        total += s;
    }
    if (total > (1 << 26)) return fail(PBB_E_INVAL, "instance total processing time too large");
    // earliest start / minimum run-out per machine (bound_fsp_weak.cpp:249-286)
    H.min_arr.assign(m, INT_MAX);
    H.min_dep.assign(m, INT_MAX);
    H.min_arr[0] = 0;
    H.min_dep[m - 1] = 0;
    for (int j = 0; j < n; j++) {
        int head = 0;
        for (int k = 1; k < m; k++) {
            head += H.p[(k - 1) * n + j];
            H.min_arr[k] = std::min(H.min_arr[k], head);
        }
        int tail = 0;
        for (int k = m - 2; k >= 0; k--) {
            tail += H.p[(k + 1) * n + j];
            H.min_dep[k] = std::min(H.min_dep[k], tail);
        }
    }
    // machine pairs in the reference's order (bound_fsp_strong.cpp:283-297),
    // filtered by JohnsonMode (:133-135)
    std::vector<std::pair<int, int>> pairs;
    for (int a = 0; a < m - 1; a++)
        for (int b = a + 1; b < m; b++) {
            if (johnson_mode == 1 && b < m - 1) continue;
            if (johnson_mode == 2 && b != a + 1) continue;
            pairs.push_back({a, b});
        }
    H.P = (int)pairs.size();
    H.Ppad = (H.P + 31) / 32 * 32;
    H.je.assign((size_t)n * H.Ppad, 0ull);
    H.posj.assign((size_t)n * H.Ppad, 0);
    H.pm0.assign(H.Ppad, 0);
    H.pm1.assign(H.Ppad, 0);
    JohnsonKeys K;
    K.grp.resize(n);
    K.val.resize(n);
    std::vector<int> lag(n), order(n);
    for (int i = 0; i < H.P; i++) {
        const int a = pairs[i].first, b = pairs[i].second;
        H.pm0[i] = (unsigned char)a;
        H.pm1[i] = (unsigned char)b;
        for (int j = 0; j < n; j++) {
            int l = 0;
            for (int k = a + 1; k < b; k++) l += H.p[k * n + j];
            lag[j] = l;
            const int pa = H.p[a * n + j], pb = H.p[b * n + j];
            K.grp[j] = pa < pb ? 1 : 2;
            K.val[j] = (pa < pb ? pa : pb) + l;
            order[j] = j;
        }
        hoare_sort(K, order, 0, n - 1);
        for (int t = 0; t < n; t++) {
            const int j = order[t];
            const unsigned long long e = JE_PACK(j, H.p[a * n + j], H.p[b * n + j], lag[j]);
            H.je[(size_t)t * H.Ppad + i] = e;
            H.posj[(size_t)j * H.Ppad + i] = (unsigned char)t;
        }
    }
    return PBB_OK;
}

}  // namespace pbbt
