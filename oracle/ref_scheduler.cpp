// Reference harness, scheduler part -- TEST INFRASTRUCTURE (linked into
// oracle/_ref/libmarqov_ref.so beside ref_harness.cpp; used by tests/ only).
//
// Compiles the reference's CXX11Scheduler (src/libmarqov/marqovscheduler.h)
// without its Core: core.h needs HDF5, so its include guard is predefined and
// makeCore only declared (the scheduler's templates name it; nothing here
// instantiates them).  The exported functions run the reference's own
//   calcMHratio            marqovscheduler.h:44-57
//   CXX11Scheduler::calcprob  marqovscheduler.h:445-465
// on stand-in simulations whose action of a state is beta times the state's
// total energy (what Core::calcAction computes, core.h:1145-1151).
#include <dirent.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#define CORE_H 1
#define MLOG_EXTLEVEL 0
#include "libmarqov/mlog.h"
#include "libmarqov/rngcache.h"
namespace MARQOV {
template <class... Ts, class... Args>
int makeCore(Args&&...);
}
// calcprob is private; the harness calls it directly
#define private public
#include "libmarqov/marqovscheduler.h"
#undef private

namespace {
struct Space {
    double energy;
};
struct StandIn {
    double beta;
    Space statespace;
    double calcAction(Space& s) const { return beta * s.energy; }
};
}  // namespace

extern "C" double ref_calc_mh_ratio(double en) { return MARQOV::calcMHratio(en); }

// mhratio[i] = calcprob(sim a_i, sim b_i) for the given (beta, total energy)
// pairs.  The scheduler writes its log file into a scratch directory.
extern "C" int ref_pt_calcprob(int n, const double* beta_a, const double* e_a, const double* beta_b,
                               const double* e_b, double* mhratio)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return 1;
    char dir[] = "/tmp/marqov_ref_schedXXXXXX";
    if (!mkdtemp(dir) || chdir(dir) != 0) return 2;
    {
        MARQOV::CXX11Scheduler<StandIn> sched(1, 1, 0);
        for (int i = 0; i < n; ++i) {
            StandIn a{beta_a[i], Space{e_a[i]}}, b{beta_b[i], Space{e_b[i]}};
            mhratio[i] = sched.calcprob(a, b);
        }
    }
    // the log files the scheduler and its logger opened there
    if (DIR* d = opendir(dir)) {
        while (const dirent* f = readdir(d))
            if (std::strcmp(f->d_name, ".") && std::strcmp(f->d_name, ".."))
                unlink((std::string(dir) + "/" + f->d_name).c_str());
        closedir(d);
    }
    rmdir(dir);
    return chdir(cwd) == 0 ? 0 : 3;
}
