// `bb` -- drop-in command line of the GPU branch-and-bound
// (gpu/src/main.cpp:12-77 of the reference): reads ./gpuconfig.ini, takes
// `-z p=fsp,i=<instance>[,o]` (common/src/arguments.cpp:215-271), solves on
// GPU 0 through the C ABI, and prints the reference's statistics block
// (common/src/pbab.cpp:40-74) and `Walltime :` line.
//
// Instances (pbab::set_instance, common/src/pbab.cpp:92-122):
//   taN        Taillard instance N: the generator is Taillard's (1993) LCG; the
//              time seeds are read from ./parameters/taillard_seeds.txt (one
//              per line, ta1 first), which this project does not ship
//   V<name>    ./parameters/vrf_parameters/<name>_Gap.txt (VRF format)
//   s<seed>_<n>x<m>  the project's seeded U[1,99] generator
// Upper bound ([initial] ub, common/src/arguments.cpp:93, :144-213): 0 or `,o`
// = best known value from ./parameters/instances.data (ta) or
// ./parameters/instancesVRF.data (V); 1 = NEH; otherwise +inf.  [initial]
// sol = 1 starts from the NEH permutation as root row, 0 from the identity.
#include <getopt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <climits>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "pbbperm.h"
#include "ini.h"

namespace {

struct Args {
    std::string problem = "flowshop", inst = "UNKNOWN", inifile = "./gpuconfig.ini";
    int init_mode = -1, init_sol = 0;
    int bound_mode = 2, branch_mode = 3, johnson_mode = 1, sorted = 1, sort_crit = 1, nb_ivms = 4096;
    bool early_stop = true, find_all = false, print_solutions = false;
    double time_limit = 0;
};

// Taillard's generator: Park-Miller minimal standard LCG (Schrage's
// decomposition), value in [low, high] through a single-precision ratio.
long taillard_unif(long* seed, long low, long high)
{
    const long M = 2147483647, A = 16807, Q = 127773, R = 2836;
    long k = *seed / Q;
    *seed = A * (*seed % Q) - k * R;
    if (*seed < 0) *seed += M;
    double u = (float)*seed / (float)M;
    return low + (long)(u * (high - low + 1));
}

int taillard_jobs(int id) { return id > 110 ? 500 : id > 90 ? 200 : id > 60 ? 100 : id > 30 ? 50 : 20; }
int taillard_machines(int id)
{
    if (id > 100) return 20;
    if (id > 90) return 10;
    if (id > 80) return 20;
    if (id > 70) return 10;
    if (id > 60) return 5;
    if (id > 50) return 20;
    if (id > 40) return 10;
    if (id > 30) return 5;
    if (id > 20) return 20;
    if (id > 10) return 10;
    return 5;
}

uint64_t splitmix(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

bool load_instance(const std::string& name, int& n, int& m, std::vector<int32_t>& p, std::string& err)
{
    if (name.size() > 2 && name[0] == 't' && name[1] == 'a') {
        int id = atoi(name.c_str() + 2);
        std::ifstream f("./parameters/taillard_seeds.txt");
        if (!f) {
            err = "taN instances need ./parameters/taillard_seeds.txt (Taillard's time seeds, one per line)";
            return false;
        }
        std::vector<long> seeds;
        long v;
        while (f >> v) seeds.push_back(v);
        if (id < 1 || id > (int)seeds.size()) { err = "no seed for " + name; return false; }
        n = taillard_jobs(id);
        m = taillard_machines(id);
        long s = seeds[id - 1];
        p.resize((size_t)n * m);
        for (int k = 0; k < m; k++)
            for (int j = 0; j < n; j++) p[(size_t)k * n + j] = (int32_t)taillard_unif(&s, 1, 99);
        return true;
    }
    if (!name.empty() && name[0] == 'V') {
        std::string path = "./parameters/vrf_parameters/" + name + "_Gap.txt";
        std::ifstream f(path);
        if (!f) { err = "Error opening file: " + path; return false; }
        if (!(f >> n >> m) || n < 1 || m < 1) { err = "infile read error"; return false; }
        std::vector<int> t((size_t)n * m);
        for (int j = 0; j < n; j++)
            for (int k = 0; k < m; k++) {
                int mach;
                if (!(f >> mach >> t[(size_t)j * m + k])) { err = "truncated " + path; return false; }
            }
        p.resize((size_t)n * m);
        for (int k = 0; k < m; k++)
            for (int j = 0; j < n; j++) p[(size_t)k * n + j] = t[(size_t)j * m + k];
        return true;
    }
    if (!name.empty() && name[0] == 's') {
        unsigned long long seed = 0;
        if (sscanf(name.c_str() + 1, "%llu_%dx%d", &seed, &n, &m) != 3) { err = "use s<seed>_<n>x<m>"; return false; }
        p.resize((size_t)n * m);
        uint64_t st = seed;
        const uint64_t span = 99, limit = UINT64_MAX - (UINT64_MAX % span);
        for (size_t i = 0; i < p.size(); i++) {
            uint64_t u;
            do { u = splitmix(&st); } while (u >= limit);
            p[i] = (int32_t)(1 + u % span);
        }
        return true;
    }
    err = "unknown instance name " + name;
    return false;
}

// best-known upper bound (common/src/arguments.cpp:154-212)
int best_known(const std::string& name)
{
    if (name[0] == 't') {
        std::ifstream f("./parameters/instances.data");
        std::string key = "instance" + std::to_string(atoi(name.c_str() + 2)) + "i", line;
        while (std::getline(f, line)) {
            if (line.compare(0, key.size(), key) == 0) {
                std::istringstream s(line);
                std::string t;
                int j, mm, v;
                if (s >> t >> j >> mm >> v) return v;
            }
        }
        return INT_MAX;
    }
    std::ifstream f("./parameters/instancesVRF.data");
    std::string line;
    while (std::getline(f, line)) {
        if (line.compare(0, name.size(), name) == 0) {
            std::istringstream s(line);
            std::string t;
            int j, mm, no, v;
            if (s >> t >> j >> mm >> no >> v) return v;
        }
    }
    return INT_MAX;
}

}  // namespace

int main(int argc, char** argv)
{
    Args a;
    IniFile ini;
    printf("reading config from:\t%s\n", a.inifile.c_str());
    if (ini.load(a.inifile)) {
        a.problem = ini.get("problem", "problem", "UNKNOWN");
        a.inst = ini.get("problem", "instance", "UNKNOWN");
        a.init_mode = (int)ini.get_int("initial", "ub", -1);
        a.init_sol = (int)ini.get_int("initial", "sol", 0);
        a.nb_ivms = (int)ini.get_int("gpu", "nbIVMs", 4096);
        a.sorted = (int)ini.get_int("bb", "sortedDFS", 1);
        a.sort_crit = (int)ini.get_int("bb", "sortingCriterion", 1);
        a.early_stop = ini.get_bool("bb", "earlyStopJohnson", true);
        a.bound_mode = (int)ini.get_int("bb", "boundingMode", 2);
        a.johnson_mode = (int)ini.get_int("bb", "JohnsonMode", 1);
        a.find_all = ini.get_bool("bb", "findAll", false);
        a.branch_mode = (int)ini.get_int("bb", "adaptiveBranchingMode", 3);
        a.print_solutions = ini.get_bool("verbose", "printSolutions", false);
        a.time_limit = (double)ini.get_int("time", "limit", 0);
    } else {
        printf("Can't load %s\n", a.inifile.c_str());
    }
    // -z p=<problem>,i=<instance>[,o]   -m (single node: always the case here)
    int c;
    while ((c = getopt(argc, argv, "z:ftm")) != -1) {
        if (c != 'z') continue;
        std::string opts = optarg;
        std::stringstream ss(opts);
        std::string item;
        while (std::getline(ss, item, ',')) {
            if (item.rfind("p=", 0) == 0) a.problem = item.substr(2);
            else if (item.rfind("i=", 0) == 0) a.inst = item.substr(2);
            else if (item == "o") a.init_mode = 0;
        }
    }
    printf("=== solving %s / instance %s\n", a.problem.c_str(), a.inst.c_str());
    if (a.problem.empty() || a.problem[0] != 'f') {
        fprintf(stderr, "only the flow-shop problem (p=fsp) is supported\n");
        return 2;
    }
    int n = 0, m = 0;
    std::vector<int32_t> p;
    std::string err;
    if (!load_instance(a.inst, n, m, p, err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    pbb_instance inst{n, m, p.data()};

    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int32_t ub = INT32_MAX;
    std::vector<int32_t> root(n), neh(n);
    for (int i = 0; i < n; i++) root[i] = i;
    int32_t neh_cost = INT32_MAX;
    if (a.init_mode == 1 || a.init_sol == 1) pbb_neh(&inst, neh.data(), &neh_cost);
    if (a.init_mode == 0) ub = best_known(a.inst);
    else if (a.init_mode == 1) ub = neh_cost;
    if (a.init_sol == 1) root = neh;
    clock_gettime(CLOCK_MONOTONIC, &t1);
    printf("T(InitialSolution):\t%f\t%d\n", (t1.tv_sec - t0.tv_sec) + (t1.tv_nsec - t0.tv_nsec) / 1e9, ub);

    pbb_config cfg;
    pbb_config_default(&cfg);
    cfg.bounding_mode = a.bound_mode;
    cfg.branching_mode = a.branch_mode;
    cfg.find_all = a.find_all;
    cfg.johnson_mode = a.johnson_mode;
    cfg.early_stop_johnson = a.early_stop;
    cfg.sorted_dfs = a.sorted;
    cfg.sorting_criterion = a.sort_crit;
    cfg.nb_ivms = a.nb_ivms;
    pbb_engine* e = nullptr;
    struct timespec ts, te;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    int rc = pbb_engine_create(&inst, &cfg, &e);
    if (rc != PBB_OK) {
        fprintf(stderr, "engine: %s\n", pbb_last_error());
        return 1;
    }
    printf("=== Device 0 ==\n=== FSP\n");
    pbb_result r;
    rc = pbb_solve(e, ub, root.data(), a.time_limit, &r);
    if (rc != PBB_OK) {
        fprintf(stderr, "solve: %s\n", pbb_last_error());
        pbb_engine_destroy(e);
        return 1;
    }
    pbb_engine_destroy(e);
    clock_gettime(CLOCK_MONOTONIC, &te);

    printf("=================\nExploration stats\n=================\n");
    printf("TOTdecomposed:\t %llu\n", (unsigned long long)r.stats.decomposed);
    printf("TOTjohnson LBs:\t %llu\n", (unsigned long long)r.stats.johnson_bounds);
    printf("TOTsimple LBs:\t %llu\n", (unsigned long long)r.stats.simple_bounds);
    printf("TOTleaves:\t %llu\n", (unsigned long long)r.stats.leaves);
    if (a.branch_mode > 0 && r.stats.decomposed > 0) {
        printf("AvgBranchingFactor:\t %f\n", (double)(r.stats.simple_bounds / 2) / r.stats.decomposed);
        printf("LB1-PruningRate:\t %f\n", 1.0 - (double)r.stats.decomposed / (r.stats.simple_bounds / 2));
        if (a.bound_mode == 2)
            printf("LB2-SuccessRate:\t %f\n",
                   ((double)r.stats.johnson_bounds - (double)r.stats.decomposed) / r.stats.decomposed);
    }
    printf("\n");
    if (!r.complete) printf("Time limit reached: exploration incomplete.\n");
    if (r.found) {
        printf("Found optimal solution.\n%d\n%d\n", n, r.cost);
        for (int i = 0; i < n; i++) printf("%d ", r.perm[i]);
        printf("\n");
    } else {
        printf("Not improved...\nOptimal makespan is >= %d (initial solution) \n", r.cost);
    }
    printf("\nWalltime :\t %2.8f\n", (te.tv_sec - ts.tv_sec) + (te.tv_nsec - ts.tv_nsec) / 1e9);
    return 0;
}
