// Checkpoint files of a search, in the form the reference's distributed
// master writes (works::save, distributed/src/works.cpp:172-190, read back by
// works::init_infile :61-90):
//
//   root solution       n \n cost \n perm[0] ... perm[n-1] \n   (solution::operator<<,
//                                                              common/src/solution.cpp:118-130)
//   simple bounds       count followed by a space
//   best solution       n \n cost \n perm ... \n
//   works               number of works \n, then per work
//                       "id end_updated max_intervals explored nb_intervals" \n
//                       (work::writeHeader, distributed/src/work.cpp:535-550)
//                       one line "id begin end" per interval, then the work's
//                       size (work::writeIntervals :553-575)
//
// An interval's ends are permutation indices in decimal: the factoradic
// vector (digit i in [0, n-i)) read as the number sum_i d_i (n-1-i)!
// (fact_work::VectToBigint, distributed/src/fact_work.cpp:74-87).  The engine
// writes one work holding the intervals of its explorers between windows
// (pbb_get_intervals), and resumes a file with pbb_init_from_fac.  Host code
// only; the decimal arithmetic is a small base-10^9 integer of its own.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "pbb_types.h"
#include "pbb_tables.h"
#include "../../include/pbbperm.h"

struct pbb_engine;
namespace pbbh {
int engine_jobs(const pbb_engine* e);
int engine_explorers(const pbb_engine* e);
const std::vector<int32_t>& engine_root(const pbb_engine* e);
void engine_set_start_perm(pbb_engine* e, const int32_t* perm);
}  // namespace pbbh

namespace {

// non-negative integer, base 10^9 limbs, least significant first
struct Big {
    std::vector<uint32_t> l;
    static const uint32_t B = 1000000000u;
    void mul_add(uint32_t mul, uint32_t add)
    {
        uint64_t carry = add;
        for (auto& x : l) {
            const uint64_t v = (uint64_t)x * mul + carry;
            x = (uint32_t)(v % B);
            carry = v / B;
        }
        while (carry) {
            l.push_back((uint32_t)(carry % B));
            carry /= B;
        }
    }
    uint32_t divmod(uint32_t d)   // *this /= d, returns the remainder
    {
        uint64_t r = 0;
        for (size_t i = l.size(); i-- > 0;) {
            const uint64_t v = r * B + l[i];
            l[i] = (uint32_t)(v / d);
            r = v % d;
        }
        while (!l.empty() && l.back() == 0) l.pop_back();
        return (uint32_t)r;
    }
    std::string str() const
    {
        if (l.empty()) return "0";
        std::string s = std::to_string(l.back());
        char buf[16];
        for (size_t i = l.size() - 1; i-- > 0;) {
            snprintf(buf, sizeof(buf), "%09u", l[i]);
            s += buf;
        }
        return s;
    }
    static bool parse(const std::string& s, Big& out)
    {
        out.l.clear();
        if (s.empty()) return false;
        for (char c : s) {
            if (c < '0' || c > '9') return false;
            out.mul_add(10, (uint32_t)(c - '0'));
        }
        return true;
    }
    bool less(const Big& o) const
    {
        if (l.size() != o.l.size()) return l.size() < o.l.size();
        for (size_t i = l.size(); i-- > 0;)
            if (l[i] != o.l[i]) return l[i] < o.l[i];
        return false;
    }
    void add(const Big& o)
    {
        uint64_t carry = 0;
        for (size_t i = 0; i < o.l.size() || carry; i++) {
            if (i == l.size()) l.push_back(0);
            const uint64_t v = (uint64_t)l[i] + (i < o.l.size() ? o.l[i] : 0) + carry;
            l[i] = (uint32_t)(v % B);
            carry = v / B;
        }
    }
    void sub(const Big& o)   // requires *this >= o
    {
        int64_t borrow = 0;
        for (size_t i = 0; i < l.size(); i++) {
            int64_t v = (int64_t)l[i] - (i < o.l.size() ? o.l[i] : 0) - borrow;
            borrow = v < 0;
            if (v < 0) v += B;
            l[i] = (uint32_t)v;
        }
        while (!l.empty() && l.back() == 0) l.pop_back();
    }
};

// factoradic digits -> index (Horner in the mixed radix n, n-1, ..., 1)
bool fact_to_big(int n, const int32_t* d, Big& v)
{
    v.l.clear();
    for (int i = 0; i < n; i++) {
        if (d[i] < 0 || d[i] >= n - i) return false;
        v.mul_add((uint32_t)(n - i), (uint32_t)d[i]);
    }
    return true;
}

// index -> factoradic digits; false when the index is n! or more
bool big_to_fact(int n, Big v, int32_t* d)
{
    for (int i = n - 1; i >= 0; i--) d[i] = (int32_t)v.divmod((uint32_t)(n - i));
    return v.l.empty();
}

int cfail(int code, const std::string& msg) { return pbbt::fail(code, msg.c_str()); }

}  // namespace

extern "C" int pbb_fact_to_decimal(int32_t n, const int32_t* digits, char* out, int32_t out_len)
{
    if (n < 1 || n > PBB_MAX_JOBS || !digits || !out || out_len < 2) return cfail(PBB_E_INVAL, "bad arguments");
    Big v;
    if (!fact_to_big(n, digits, v)) return cfail(PBB_E_INVAL, "digit i must be in [0, n-i)");
    const std::string s = v.str();
    if ((int)s.size() + 1 > out_len) return cfail(PBB_E_INVAL, "output buffer too small");
    memcpy(out, s.c_str(), s.size() + 1);
    return PBB_OK;
}

extern "C" int pbb_decimal_to_fact(int32_t n, const char* decimal, int32_t* digits)
{
    if (n < 1 || n > PBB_MAX_JOBS || !decimal || !digits) return cfail(PBB_E_INVAL, "bad arguments");
    Big v;
    if (!Big::parse(decimal, v)) return cfail(PBB_E_INVAL, "not a decimal integer");
    if (!big_to_fact(n, v, digits)) return cfail(PBB_E_INVAL, "index is not below n!");
    return PBB_OK;
}

extern "C" int pbb_save_checkpoint(pbb_engine* e, const char* path)
{
    if (!e || !path) return cfail(PBB_E_INVAL, "NULL argument");
    const int n = pbbh::engine_jobs(e);
    const int B = pbbh::engine_explorers(e);
    pbb_result r;
    int rc = pbb_get_result(e, &r);
    if (rc) return rc;
    std::vector<int32_t> pos((size_t)B * n), end((size_t)B * n), ids(B);
    int32_t cnt = 0;
    rc = pbb_get_intervals(e, B, pos.data(), end.data(), ids.data(), &cnt);
    if (rc) return rc;
    const std::vector<int32_t>& root = pbbh::engine_root(e);
    std::ostringstream os;
    // root solution: the root permutation with the bound the search started from
    os << n << "\n" << r.cost << "\n";
    for (int i = 0; i < n; i++) os << root[i] << " ";
    os << "\n";
    os << r.stats.simple_bounds << " ";
    // best solution: the incumbent (the root permutation when no schedule is known)
    os << n << "\n" << r.cost << "\n";
    for (int i = 0; i < n; i++) os << (r.has_perm ? r.perm[i] : root[i]) << " ";
    os << "\n";
    os << 1 << "\n";
    os << 0 << " " << 0 << " " << cnt << " " << r.stats.decomposed << " " << cnt << "\n";
    Big size;
    for (int k = 0; k < cnt; k++) {
        Big a, b;
        if (!fact_to_big(n, &pos[(size_t)k * n], a) || !fact_to_big(n, &end[(size_t)k * n], b))
            return cfail(PBB_E_CUDA, "corrupt interval");
        os << ids[k] << " " << a.str() << " " << b.str() << "\n";
        if (a.less(b)) {
            b.sub(a);
            size.add(b);
        }
    }
    os << size.str() << "\n";
    std::ofstream f(path, std::ios::out | std::ios::trunc);
    if (!f) return cfail(PBB_E_INVAL, std::string("cannot write ") + path);
    f << os.str();
    f.close();
    if (!f) return cfail(PBB_E_INVAL, std::string("write failed: ") + path);
    return PBB_OK;
}

extern "C" int pbb_load_checkpoint(pbb_engine* e, const char* path, uint64_t* saved_simple_bounds)
{
    if (!e || !path) return cfail(PBB_E_INVAL, "NULL argument");
    const int n = pbbh::engine_jobs(e);
    const int B = pbbh::engine_explorers(e);
    std::ifstream f(path);
    if (!f) return cfail(PBB_E_INVAL, std::string("cannot read ") + path);
    auto bad = [&](const char* what) { return cfail(PBB_E_INVAL, std::string("checkpoint ") + path + ": " + what); };
    int rn = 0, root_cost = 0, bn = 0, best_cost = 0;
    std::vector<int32_t> root(n), best(n);
    if (!(f >> rn >> root_cost) || rn != n) return bad("root solution of another size");
    for (int i = 0; i < n; i++)
        if (!(f >> root[i])) return bad("truncated root solution");
    unsigned long long simple = 0;
    if (!(f >> simple)) return bad("missing bound count");
    if (!(f >> bn >> best_cost) || bn != n) return bad("best solution of another size");
    for (int i = 0; i < n; i++)
        if (!(f >> best[i])) return bad("truncated best solution");
    std::vector<int> seen(n, 0);
    for (int i = 0; i < n; i++) {
        if (root[i] < 0 || root[i] >= n || seen[root[i]]) return bad("root is not a permutation");
        seen[root[i]] = 1;
    }
    bool best_ok = true;
    std::fill(seen.begin(), seen.end(), 0);
    for (int i = 0; i < n; i++) {
        if (best[i] < 0 || best[i] >= n || seen[best[i]]) best_ok = false;
        else seen[best[i]] = 1;
    }
    int works = 0;
    if (!(f >> works) || works < 0) return bad("missing work count");
    std::vector<int32_t> pos, end;
    for (int w = 0; w < works; w++) {
        long long id = 0, updated = 0, maxi = 0;
        std::string explored;
        long long nb = 0;
        if (!(f >> id >> updated >> maxi >> explored >> nb) || nb < 0) return bad("bad work header");
        for (long long k = 0; k < nb; k++) {
            std::string iid, sb, se;
            if (!(f >> iid >> sb >> se)) return bad("truncated interval");
            Big a, b;
            std::vector<int32_t> da(n), db(n);
            if (!Big::parse(sb, a) || !Big::parse(se, b) || !big_to_fact(n, a, da.data()) ||
                !big_to_fact(n, b, db.data()))
                return bad("interval end is not an index below n!");
            if (b.less(a)) continue;   // empty interval
            pos.insert(pos.end(), da.begin(), da.end());
            end.insert(end.end(), db.begin(), db.end());
        }
        std::string size;
        if (!(f >> size)) return bad("missing work size");
    }
    const int cnt = (int)(pos.size() / n);
    if (cnt > B) return bad("more intervals than the engine has explorers");
    if (saved_simple_bounds) *saved_simple_bounds = simple;
    if (cnt == 0) {
        // nothing left to explore: an empty search that reports the incumbent
        std::vector<int32_t> p0(n, 0), e0(n, 0);
        p0[0] = n - 1;
        int rc = pbb_start_interval(e, best_cost, root.data(), p0.data(), e0.data());
        if (rc) return rc;
    } else {
        int rc = pbb_init_from_fac(e, best_cost, root.data(), cnt, nullptr, pos.data(), end.data());
        if (rc) return rc;
    }
    if (best_ok) pbbh::engine_set_start_perm(e, best.data());
    return PBB_OK;
}
