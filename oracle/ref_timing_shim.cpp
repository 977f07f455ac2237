// Wall-clock timers around the reference's two sweep entry points.
//
// The reference's Sweep.cpp is compiled with InfectSweep/IncubRecoverySweep renamed
// to ref_InfectSweep/ref_IncubRecoverySweep (see the Makefile); this file then owns
// the original symbols declared at src/Sweep.h:7-8 and called from RunModel
// (src/CovidSim.cpp:1488,1490).  The reference's printed "Model ran in" figure is
// clock() CPU time summed over threads (src/CovidSim.cpp:418), not wall time, so the
// baseline is taken from omp_get_wtime() here.  At exit one line is written to
// stderr:
//   REFTIMING pop=<N> threads=<T> steps=<k> infect_s=<s> incub_s=<s> first_t=<d> last_t=<d>
#include <cstdio>
#include <cstdlib>
#include <omp.h>

#include "Param.h"
#include "Sweep.h"

void ref_InfectSweep(double t, int run);
void ref_IncubRecoverySweep(double t);

namespace {
double g_infect = 0.0, g_incub = 0.0, g_first = -1.0, g_last = -1.0;
long g_steps = 0;
bool g_registered = false;

void report()
{
	std::fprintf(stderr, "\nREFTIMING pop=%d threads=%d steps=%ld infect_s=%.6f incub_s=%.6f first_t=%.4f last_t=%.4f\n",
		P.PopSize, P.NumThreads, g_steps, g_infect, g_incub, g_first, g_last);
}
}

void InfectSweep(double t, int run)
{
	if (!g_registered) { std::atexit(report); g_registered = true; }
	if (g_first < 0) g_first = t;
	g_last = t;
	double t0 = omp_get_wtime();
	ref_InfectSweep(t, run);
	g_infect += omp_get_wtime() - t0;
	g_steps++;
}

void IncubRecoverySweep(double t)
{
	double t0 = omp_get_wtime();
	ref_IncubRecoverySweep(t);
	g_incub += omp_get_wtime() - t0;
}
