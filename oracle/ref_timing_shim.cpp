// Wall-clock timers around the reference's two sweep entry points.
//
// The reference's Sweep.cpp is compiled with InfectSweep/IncubRecoverySweep renamed
// to ref_InfectSweep/ref_IncubRecoverySweep (see the Makefile); this file then owns
// the original symbols declared at src/Sweep.h:7-8 and called from RunModel
// (src/CovidSim.cpp:1488,1490).  The reference's printed "Model ran in" figure is
// clock() CPU time summed over threads (src/CovidSim.cpp:418), not wall time, so the
// baseline is taken from omp_get_wtime() here.  At exit one line per realisation
// is written to stderr:
//   REFTIMING run=<r> pop=<N> threads=<T> steps=<k> infect_s=<s> incub_s=<s> first_t=<d> last_t=<d> loop_s=<s>
// loop_s is the wall clock from the run's first InfectSweep call to the end of its
// last IncubRecoverySweep: RunModel's time stepping with the host code between sweeps.
#include <cstdio>
#include <cstdlib>
#include <omp.h>
#include <vector>

#include "Param.h"
#include "Sweep.h"

void ref_InfectSweep(double t, int run);
void ref_IncubRecoverySweep(double t);

namespace {
struct RunTiming {
    int run;
    double infect = 0.0, incub = 0.0, first = -1.0, last = -1.0, loop_start = -1.0, loop_end = -1.0;
    long steps = 0;
};
std::vector<RunTiming> g_runs;
bool g_registered = false;

void report()
{
    for (const RunTiming& r : g_runs)
        std::fprintf(stderr, "\nREFTIMING run=%d pop=%d threads=%d steps=%ld infect_s=%.6f incub_s=%.6f first_t=%.4f last_t=%.4f"
                             " loop_s=%.6f\n",
                     r.run, P.PopSize, P.NumThreads, r.steps, r.infect, r.incub, r.first, r.last, r.loop_end - r.loop_start);
}
}

void InfectSweep(double t, int run)
{
    if (!g_registered) { std::atexit(report); g_registered = true; }
    if (g_runs.empty() || g_runs.back().run != run) { g_runs.push_back(RunTiming()); g_runs.back().run = run; }
    RunTiming& r = g_runs.back();
    if (r.first < 0) r.first = t;
    r.last = t;
    double t0 = omp_get_wtime();
    if (r.loop_start < 0) r.loop_start = t0;
    ref_InfectSweep(t, run);
    r.infect += omp_get_wtime() - t0;
    r.steps++;
}

void IncubRecoverySweep(double t)
{
    double t0 = omp_get_wtime();
    ref_IncubRecoverySweep(t);
    if (!g_runs.empty()) {
        const double t1 = omp_get_wtime();
        g_runs.back().incub += t1 - t0;
        g_runs.back().loop_end = t1;
    }
}
