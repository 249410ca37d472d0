// Test infrastructure only (never part of the product path).
//
// The reference's own askja program (sun.cpp, #included through -I at build
// time, never copied into this repository) with time() replaced by a clock
// that advances by one on every call.  The reference seeds its generator from
// time(NULL) before every momentum refresh and every Metropolis uniform
// (sun.cpp:1268-1311); a run faster than one trajectory per second would
// reuse seeds, i.e. repeat the same momenta and uniforms over consecutive
// trajectories, and sample a biased ensemble.  With this clock every seed is
// new and the run is reproducible.  Everything else is the reference's code.
#include <time.h>

static unsigned long askja_ref_clock = 1000;
static time_t askja_ref_fake_time(time_t*) { return (time_t)(askja_ref_clock++); }

#define time(x) askja_ref_fake_time(x)
#include <sun.cpp>
#undef time
