// A process-wide pool of host worker threads for the per-context set-up
// (the stars of every mesh point, the tetrahedron table).  Creating and
// joining a thread costs tens of microseconds, and a context's set-up ran two
// pools of up to 32 threads each; the workers here are created once, on the
// first use, and wait on a condition variable between jobs.
//
// run_parallel(n, f) calls f(0) .. f(n-1), each exactly once, on the pool's
// workers and on the calling thread, and returns when all have returned.
// Calls from several host threads at once are served in turn: each caller
// also works on its own job, so a job always finishes.
#pragma once

#include <functional>

namespace ald {

void run_parallel(int ntask, const std::function<void(int)>& f);

// workers plus the calling thread: the natural number of stripes for a job
int pool_width();

}  // namespace ald
