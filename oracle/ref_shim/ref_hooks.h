/* Test infrastructure: force-included (g++ -include) ahead of every CETASim
 * source compiled into the oracle harness under oracle/_ref.  The sources
 * stay unmodified; three of their library calls are redirected so that the
 * harness can run them reproducibly and inside a test process:
 *
 *  - std::random_device (MPBunch.cpp:104, Bunch.cpp:989,
 *    LatticeInterActionPoint.cpp:990, ...) draws from a seeded sequence
 *    (splitmix64 of a base seed and a call counter) that cg_ref_seed() sets,
 *    so mt19937 streams seeded from it repeat run to run;
 *  - time(0) in the srand() seeds of the initial distribution
 *    (MPBunch.cpp:118, Global.cpp:77) returns a value cg_ref_seed() sets;
 *  - exit(code) (transmission < 0.5 at Bunch.cpp:194-197, ion overflow at
 *    LatticeInterActionPoint.cpp:1043-1048, bad input) throws
 *    cg_ref_exit_signal, which the harness turns into an error status
 *    instead of ending the test process.
 */
#ifndef CG_REF_HOOKS_H
#define CG_REF_HOOKS_H

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <stdlib.h>
#include <time.h>
#include <sys/time.h>

struct cg_ref_exit_signal {
    int code;
};

extern "C" void cg_ref_seed(unsigned long long seed, long long fixed_time);
unsigned int cg_ref_next_device_value();
time_t cg_ref_time(time_t *t);
[[noreturn]] void cg_ref_exit(int code);

namespace std {
class cg_ref_random_device {
public:
    typedef unsigned int result_type;
    cg_ref_random_device() {}
    explicit cg_ref_random_device(const std::string &) {}
    result_type operator()() { return cg_ref_next_device_value(); }
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return 0xFFFFFFFFu; }
    double entropy() const noexcept { return 32.0; }
};
}  // namespace std

#define random_device cg_ref_random_device
#define time(t) cg_ref_time(t)
#define exit(c) cg_ref_exit(c)

#endif
