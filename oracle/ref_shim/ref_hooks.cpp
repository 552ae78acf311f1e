// Test infrastructure: bodies of the hooks ref_hooks.h redirects the
// reference's std::random_device, time(0) and exit() to (see that header).
// Linked into every build of the reference's sources under oracle/_ref.
#include "ref_hooks.h"

namespace {
unsigned long long g_seed = 0x5eedULL;
unsigned long long g_device_calls = 0;
long long g_fixed_time = 0;

unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
}  // namespace

extern "C" void cg_ref_seed(unsigned long long seed, long long fixed_time) {
    g_seed = seed;
    g_device_calls = 0;
    g_fixed_time = fixed_time;
}

unsigned int cg_ref_next_device_value() {
    return static_cast<unsigned int>(splitmix64(g_seed * 0x100000001B3ULL + g_device_calls++) >> 32);
}

#undef time
time_t cg_ref_time(time_t *t) {
    if (t) *t = static_cast<time_t>(g_fixed_time);
    return static_cast<time_t>(g_fixed_time);
}

#undef exit
[[noreturn]] void cg_ref_exit(int code) { throw cg_ref_exit_signal{code}; }
