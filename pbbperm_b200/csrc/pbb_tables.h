// Instance tables built on the host (shared by the engine, the pool and the
// no-alloc bound entry point).  The core builder works on caller-provided
// arrays and fixed-size stack scratch only, so the entry point that must not
// allocate uses exactly the same code, tie order included.
#pragma once
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <vector>

#include "pbb_types.h"
#include "../../include/pbbperm.h"

namespace pbbh {
void set_error(const char* msg);
int check_search(const pbb_config* c);   // pbb_host.cu: settings every entry point accepts
}

namespace pbbt {

inline int fail(int code, const char* msg)
{
    pbbh::set_error(msg);
    return code;
}

// Johnson's rule with the reference's tie order: keys (group, value); group 1
// (first machine strictly shorter) ascending by p_a + lag, then group 2
// descending by p_b + lag; equal keys stay in the order left by a Hoare
// partition quicksort that pivots on the first element
// (bounds/src/bound_fsp_strong.cpp:359-436).  The order among ties changes
// the bound's value, so the partition scheme is part of the contract.
struct JohnsonKeys {
    int grp[PBB_MAX_N];
    int val[PBB_MAX_N];
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

inline void hoare_sort(const JohnsonKeys& K, int* v, int lo, int hi)
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

// machine pairs (a < b) in the reference's order (bound_fsp_strong.cpp:283-297),
// filtered by JohnsonMode (:133-135): 0 all, 1 (k, m-1), 2 (k, k+1)
inline bool pair_used(int a, int b, int m, int johnson_mode)
{
    if (johnson_mode == 1 && b < m - 1) return false;
    if (johnson_mode == 2 && b != a + 1) return false;
    return true;
}

inline int count_pairs(int m, int johnson_mode)
{
    int P = 0;
    for (int a = 0; a < m - 1; a++)
        for (int b = a + 1; b < m; b++) P += pair_used(a, b, m, johnson_mode) ? 1 : 0;
    return P;
}

// Checks shared by every entry point: processing times in [0, 65535] (two
// times share a 32-bit word of a Johnson entry) and a job's total at most
// 32767 (per-child head/tail deltas are int16).
inline int check_times(const int32_t* p, int n, int m)
{
    long long total = 0;
    for (int j = 0; j < n; j++) {
        long long s = 0;
        for (int k = 0; k < m; k++) {
            const int v = p[k * n + j];
            if (v < 0 || v > 65535) return fail(PBB_E_INVAL, "processing times must be in [0, 65535]");
            s += v;
        }
        if (s > 32767) return fail(PBB_E_INVAL, "a job's total processing time must be <= 32767");
        total += s;
    }
    if (total > (1 << 26)) return fail(PBB_E_INVAL, "instance total processing time too large");
    return PBB_OK;
}

// Destination arrays of one instance's tables (any may be NULL except je,
// pm0, pm1, min_arr, min_dep).
struct TableSpans {
    unsigned long long* je;   // [n][Ppad] packed Johnson entries, pair-minor
    unsigned char* posj;      // [n][Ppad] Johnson position of each job per pair
    unsigned char* pm0;       // [Ppad] first machine of each pair
    unsigned char* pm1;       // [Ppad] second machine
    int* min_arr;             // [m] earliest start per machine
    int* min_dep;             // [m] minimum run-out per machine
};

// Fill the tables of a checked instance (n <= 64).  Uses no heap memory.
inline void fill_tables(const int32_t* p, int n, int m, int johnson_mode, int Ppad, const TableSpans& T)
{
    // earliest start / minimum run-out per machine (bound_fsp_weak.cpp:249-286)
    for (int k = 0; k < m; k++) { T.min_arr[k] = INT_MAX; T.min_dep[k] = INT_MAX; }
    T.min_arr[0] = 0;
    T.min_dep[m - 1] = 0;
    for (int j = 0; j < n; j++) {
        int head = 0;
        for (int k = 1; k < m; k++) {
            head += p[(k - 1) * n + j];
            T.min_arr[k] = std::min(T.min_arr[k], head);
        }
        int tail = 0;
        for (int k = m - 2; k >= 0; k--) {
            tail += p[(k + 1) * n + j];
            T.min_dep[k] = std::min(T.min_dep[k], tail);
        }
    }
    memset(T.je, 0, sizeof(unsigned long long) * n * Ppad);
    if (T.posj) memset(T.posj, 0, (size_t)n * Ppad);
    memset(T.pm0, 0, Ppad);
    memset(T.pm1, 0, Ppad);
    JohnsonKeys K;
    int lag[PBB_MAX_N], order[PBB_MAX_N];
    int i = 0;
    for (int a = 0; a < m - 1; a++)
        for (int b = a + 1; b < m; b++) {
            if (!pair_used(a, b, m, johnson_mode)) continue;
            T.pm0[i] = (unsigned char)a;
            T.pm1[i] = (unsigned char)b;
            for (int j = 0; j < n; j++) {
                int l = 0;
                for (int k = a + 1; k < b; k++) l += p[k * n + j];
                lag[j] = l;
                const int pa = p[a * n + j], pb = p[b * n + j];
                K.grp[j] = pa < pb ? 1 : 2;
                K.val[j] = (pa < pb ? pa : pb) + l;
                order[j] = j;
            }
            hoare_sort(K, order, 0, n - 1);
            for (int t = 0; t < n; t++) {
                const int j = order[t];
                T.je[(size_t)t * Ppad + i] = JE_PACK(j, p[a * n + j], p[b * n + j], lag[j]);
                if (T.posj) T.posj[(size_t)j * Ppad + i] = (unsigned char)t;
            }
            i++;
        }
}

// ---------------------------------------------------------------------------
// instance tables in host vectors (engine and pool)
// ---------------------------------------------------------------------------
struct HostTables {
    int n = 0, m = 0, P = 0, Ppad = 0;
    std::vector<int> p, min_arr, min_dep;
    std::vector<unsigned long long> je;
    std::vector<unsigned char> pm0, pm1, posj;
};

inline int build_tables(const pbb_instance* inst, int johnson_mode, HostTables& H)
{
    if (!inst || !inst->p) return fail(PBB_E_INVAL, "instance is NULL");
    const int n = inst->n_jobs, m = inst->n_machines;
    if (n < 2 || n > PBB_MAX_JOBS) return fail(PBB_E_INVAL, "n_jobs must be in [2, 64]");
    if (m < 2 || m > PBB_MAX_MACHINES) return fail(PBB_E_INVAL, "n_machines must be in [2, 32]");
    if (johnson_mode < 0 || johnson_mode > 2) return fail(PBB_E_UNSUPPORTED, "JohnsonMode must be 0, 1 or 2");
    const int rc = check_times(inst->p, n, m);
    if (rc) return rc;
    H.n = n; H.m = m;
    H.p.assign(inst->p, inst->p + n * m);
    H.P = count_pairs(m, johnson_mode);
    H.Ppad = (H.P + 31) / 32 * 32;
    H.min_arr.assign(m, 0);
    H.min_dep.assign(m, 0);
    H.je.assign((size_t)n * H.Ppad, 0ull);
    H.posj.assign((size_t)n * H.Ppad, 0);
    H.pm0.assign(H.Ppad, 0);
    H.pm1.assign(H.Ppad, 0);
    TableSpans T{H.je.data(), H.posj.data(), H.pm0.data(), H.pm1.data(), H.min_arr.data(), H.min_dep.data()};
    fill_tables(H.p.data(), n, m, johnson_mode, H.Ppad, T);
    return PBB_OK;
}

}  // namespace pbbt
