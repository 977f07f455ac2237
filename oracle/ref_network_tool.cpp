// TEST AND CPU-BASELINE INFRASTRUCTURE: the reference's own set-up with a fast place
// assignment, used once per population to write a network file (/S) that the
// reference executable and the drop-in then load with /L.
//
// The reference assigns people to places one person at a time on one thread, each
// search spiralling over microcells (src/SetupModel.cpp:1989-2466); at 10M people
// on 240 x 240 cells that step alone runs for hours, far longer than any timed
// run.  oracle/Makefile links the reference's SetupModel object with its
// AssignPeopleToPlaces made a weak symbol, so the set-up calls the definition in
// this file instead.  It fills
// Hosts[].PlaceLinks exactly where LoadPeopleToPlaces would (src/SetupModel.cpp:
// 2603-2659): the set-up reseeds its random numbers right after either call
// (src/SetupModel.cpp:294-296), so what follows -- groups, kernels, InitModel --
// is the reference's own code on the same footing as a /L run.
//
// The replacement keeps the reference's rules where they shape the network and
// simplifies the search:
//   * who attends a place type: the age table PropPlaces and one place per person
//     (src/SetupModel.cpp:2022-2040);
//   * place capacities: the type's size distribution, the 43/40 Poisson
//     adjustment and the total of 1.075 / 1.125 x demand (src/SetupModel.cpp:
//     2062-2210, P.nsp = 0);
//   * the choice: among the nearest places with room (the type's
//     "closest places" count, 24 where the reference samples all places), with
//     probability proportional to the type's kernel K(d) x remaining capacity, the
//     weight the reference's searches use (src/SetupModel.cpp:2265-2290, 2404-2415).
// Age-restricted availability (AvailByAge) is not modelled.
//
// With CS_NETGEN_LOAD=<file> in the environment the replacement assigns nothing
// itself: it calls the reference's own LoadPeopleToPlaces on that file, so that a
// /S run writes back, through the reference's SavePeopleToPlaces, exactly the links
// the reference's loader read (the reference's command line refuses /L and /S
// together).  Tests use it to show that a network file written elsewhere is read
// link for link.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <string>
#include <vector>

#include "Constants.h"
#include "Dist.h"
#include "Error.h"
#include "Kernels.h"
#include "Model.h"
#include "Param.h"
#include "SetupModel.h"

extern double PropPlaces[NUM_AGE_GROUPS * AGE_GROUP_WIDTH][MAX_NUM_PLACE_TYPES];

namespace {

struct Grid {
    int nx, ny;
    std::vector<int> start, items;   // places bucketed by cell
};

Grid bucket_places(int tp)
{
    Grid g{P.ncw, P.nch, std::vector<int>((size_t)P.ncw * P.nch + 1, 0), std::vector<int>(P.Nplace[tp])};
    auto cell_of = [](const Place& pl) {
        int x = std::min(std::max((int)(pl.loc.x / P.in_cells_.width), 0), P.ncw - 1);
        int y = std::min(std::max((int)(pl.loc.y / P.in_cells_.height), 0), P.nch - 1);
        return x * P.nch + y;
    };
    for (int i = 0; i < P.Nplace[tp]; i++) g.start[cell_of(Places[tp][i]) + 1]++;
    for (size_t c = 0; c + 1 < g.start.size(); c++) g.start[c + 1] += g.start[c];
    std::vector<int> fill(g.start.begin(), g.start.end() - 1);
    for (int i = 0; i < P.Nplace[tp]; i++) g.items[fill[cell_of(Places[tp][i])]++] = i;
    return g;
}

int capacity_draw(int tp, std::mt19937_64& rng)
{
    std::uniform_real_distribution<double> U(0.0, 1.0);
    int j;
    if (P.PlaceTypeSizePower[tp] == 0 && P.PlaceTypeSizeSD[tp] == 0) {
        std::poisson_distribution<int> pois(std::max(P.PlaceTypeMeanSize[tp] - 1, 1e-9));
        j = 1 + pois(rng);
    } else if (P.PlaceTypeSizePower[tp] == 0) {
        std::lognormal_distribution<double> ln(std::log(P.PlaceTypeMeanSize[tp]), P.PlaceTypeSizeSD[tp] / P.PlaceTypeMeanSize[tp]);
        do j = (int)ln(rng); while (j < P.PlaceTypeSizeMin[tp] || j > P.PlaceTypeSizeMax[tp]);
    } else {
        const double s = std::pow(P.PlaceTypeSizeOffset[tp] / (P.PlaceTypeSizeOffset[tp] + P.PlaceTypeSizeMax[tp] - P.PlaceTypeSizeMin[tp]),
                                  P.PlaceTypeSizePower[tp]);
        j = (int)std::floor(P.PlaceTypeSizeOffset[tp] * std::pow((1 - s) * U(rng) + s, -1 / P.PlaceTypeSizePower[tp]) +
                            P.PlaceTypeSizeMin[tp] - P.PlaceTypeSizeOffset[tp]);
    }
    return std::min(std::max(j, 1), (int)USHRT_MAX - 1);
}

}  // namespace

void AssignPeopleToPlaces()
{
    if (const char* load = std::getenv("CS_NETGEN_LOAD")) {
        LoadPeopleToPlaces(std::string(load));
        return;
    }
    std::mt19937_64 rng(((uint64_t)(uint32_t)P.setupSeed1 << 32) ^ (uint32_t)P.setupSeed2 ^ 0x6E657467656E2121ull);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    for (int i = 0; i < P.PopSize; i++)
        for (int tp = 0; tp < MAX_NUM_PLACE_TYPES; tp++) Hosts[i].PlaceLinks[tp] = -1;
    for (int tp = 0; tp < P.NumPlaceTypes; tp++) {
        if (tp == P.HotelPlaceType || P.Nplace[tp] == 0) continue;
        // who attends: age table, one place per person, in cell order
        std::vector<int> people;
        for (int a = 0; a < P.NumPopulatedCells; a++) {
            Cell* c = CellLookup[a];
            for (int j = 0; j < c->n; j++) {
                const int i = c->members[j], k = Hosts[i].age;
                bool f = PropPlaces[k][tp] > 0 && U(rng) < PropPlaces[k][tp];
                for (int t2 = 0; t2 < tp && f; t2++) if (Hosts[i].PlaceLinks[t2] >= 0) f = false;
                if (f) people.push_back(i);
            }
        }
        std::shuffle(people.begin(), people.end(), rng);
        // capacities
        std::vector<int> cap(P.Nplace[tp]);
        long long total = 0;
        for (int i = 0; i < P.Nplace[tp]; i++) {
            int c0 = capacity_draw(tp, rng);
            std::poisson_distribution<int> pois(std::max((double)c0 * 43 / 40 - 1, 1e-9));
            total += cap[i] = 1 + pois(rng);
        }
        long long want = (long long)((double)people.size() * 1.125);
        std::uniform_int_distribution<int> pick(0, P.Nplace[tp] - 1);
        for (long long d = want - total; d > 0; d--) cap[pick(rng)]++;
        for (long long d = total - want; d > 0; d--) {
            int j;
            do j = pick(rng); while (cap[j] < 2);
            cap[j]--;
        }
        // the type's own kernel, as the reference's search evaluates it
        P.Kernel.type_ = P.PlaceTypeKernelType[tp];
        P.Kernel.scale_ = P.PlaceTypeKernelScale[tp];
        P.Kernel.shape_ = P.PlaceTypeKernelShape[tp];
        P.Kernel.p3_ = P.PlaceTypeKernelP3[tp];
        P.Kernel.p4_ = P.PlaceTypeKernelP4[tp];
        P.KernelLookup.init(1.0, P.Kernel);
        const Grid g = bucket_places(tp);
        const int nn = P.PlaceTypeNearestNeighb[tp] > 0 ? P.PlaceTypeNearestNeighb[tp] : 24;
        std::vector<std::pair<double, int>> cand;
        long long assigned = 0;
        for (size_t q = 0; q < people.size(); q++) {
            const int i = people[q];
            const Household& h = Households[Hosts[i].hh];
            const int cx = std::min(std::max((int)(h.loc.x / P.in_cells_.width), 0), P.ncw - 1);
            const int cy = std::min(std::max((int)(h.loc.y / P.in_cells_.height), 0), P.nch - 1);
            cand.clear();
            // rings of cells until nn places with room are in hand, then one ring more
            int extra = -1;
            auto visit = [&](int x, int y) {
                if (x < 0 || y < 0 || x >= P.ncw || y >= P.nch) return;
                const int c = x * P.nch + y;
                for (int k = g.start[c]; k < g.start[c + 1]; k++) {
                    const int pl = g.items[k];
                    if (cap[pl] <= 0) continue;
                    const double d2 = dist2_raw(h.loc.x, h.loc.y, Places[tp][pl].loc.x, Places[tp][pl].loc.y);
                    cand.emplace_back(d2, pl);
                }
            };
            for (int r = 0; r < std::max(P.ncw, P.nch) && extra != 0; r++) {
                if (r == 0) visit(cx, cy);
                for (int k = -r; k <= r && r > 0; k++) {     // the ring's perimeter
                    visit(cx + k, cy - r);
                    visit(cx + k, cy + r);
                    if (k > -r && k < r) { visit(cx - r, cy + k); visit(cx + r, cy + k); }
                }
                if (extra > 0) extra--;
                else if (extra < 0 && (int)cand.size() >= nn) extra = 1;
            }
            if (cand.empty()) continue;
            const size_t m = std::min(cand.size(), (size_t)nn);
            std::partial_sort(cand.begin(), cand.begin() + m, cand.end());
            double tot = 0;
            std::vector<double> w(m);
            for (size_t k = 0; k < m; k++) tot += w[k] = P.KernelLookup.num(cand[k].first) * (double)cap[cand[k].second];
            if (!(tot > 0)) continue;
            double u = U(rng) * tot;
            size_t k = 0;
            while (k + 1 < m && u >= w[k]) { u -= w[k]; k++; }
            const int pl = cand[k].second;
            Hosts[i].PlaceLinks[tp] = pl;
            cap[pl]--;
            assigned++;
        }
        std::fprintf(stderr, "netgen: %lld of %zu people assigned to place type %d (%d places)\n", assigned, people.size(),
                     tp, P.Nplace[tp]);
    }
}
