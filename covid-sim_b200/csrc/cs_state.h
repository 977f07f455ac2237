// Device-resident layout of one population and its dynamic state.
//
// People: one 32-byte record per person (PersonHot) holding every field a gather
// of "another person" reads in the sweeps (infection state, household, microcell,
// susceptibility, absence/isolation/quarantine times, age, flags), so that a
// random person costs one 32-byte DRAM sector; fields only the person's own
// transitions touch live in separate arrays (structure of arrays).
// Cells: Cell::susceptible lists (src/Models/Cell.h:11-20) concatenated cell by
// cell in `slots`, each partitioned [S | L | I | R and D] exactly as the
// reference maintains them.
#pragma once

#include <cstdint>

#include "covidsim_b200.h"

namespace csb {

struct __align__(16) PersonHot {
    int32_t hh;                // Person::hh
    int32_t mcell;             // microcell index
    float susc;                // Person::susc
    float infness;             // Person::infectiousness (negative when symptomatic)
    uint16_t latent_time;      // Person::latent_time
    uint16_t absent_start;     // Person::absent_start_time
    uint16_t absent_stop;      // Person::absent_stop_time
    uint16_t isolation_start;  // Person::isolation_start_time
    uint16_t quar_start;       // HostsQuarantine[].start_time
    int8_t inf;                // InfStat
    uint8_t age;               // Person::age
    uint8_t pflags;            // CS_PF_* (static)
    uint8_t dflags;            // CS_DF_* (to_die, detected, quarantine compliance)
    uint8_t sev;               // Severity_Current | Severity_Final << 4
    uint8_t pad;
};
static_assert(sizeof(PersonHot) == 32, "PersonHot must fill one 32-byte sector");

// Place memberships of one person, in one 32-byte sector: the place of each type
// (-1 for none) and the group within it.
struct __align__(16) PersonLinks {
    int32_t link[CS_MAX_PLACE_TYPES];
    uint16_t group[CS_MAX_PLACE_TYPES];
    uint16_t pad;
};
static_assert(sizeof(PersonLinks) == 32, "PersonLinks must fill one 32-byte sector");

// One household: location, first member (members are contiguous), size, and the
// size the household kernel is normalised by (Household::nhr).
struct __align__(16) HouseholdRec {
    float x, y;
    int32_t first;
    uint16_t nh, nhr;
};
static_assert(sizeof(HouseholdRec) == 16, "HouseholdRec is one 16-byte load");

// One cell of a proposal block's cell list: running S0 of the block up to and
// including this cell, the cell, its first slot and its S0 (one 16-byte load).
struct __align__(16) BlockCell {
    int32_t cum, m, start, s0;
};
// A proposal block: its S0 and its range [kb, ke) of the block cell list.
struct __align__(16) BlockInfo {
    long long S0;
    int32_t kb, ke;
};

struct DevPlaces {
    int32_t n;
    const int32_t* mcell;
    const int32_t* member_ofs;
    const int32_t* members;
    const int32_t* group_ofs;
    const int32_t* group_start;
    const int32_t* group_size;
    const float* x;            // location (blanket movement restrictions measure to it)
    const float* y;
    uint16_t* close_start;
    uint16_t* close_end;
    float* prob_close;
};

// Intervention windows: the policy durations, and each admin unit's start times
// (AdUnits[a].CaseIsolationTimeStart and .HQuarantineTimeStart), NA entries each.
struct DevIv {
    double ci_dur, hq_dur;
    double* ci_start;
    double* hq_start;
};

// Scalars of the current timestep, written on the device by k_set_step so that a
// captured step graph needs only that one kernel's arguments changed per replay.
struct DevStep {
    double t, fp, seas, sp_beta, hh_beta;
    int32_t ts;
    int32_t blanket;           // blanket movement restrictions in place (src/Sweep.cpp:301)
    unsigned long long seed;
};

// Transition flags per person for one IncubRecoverySweep.
enum : uint8_t { kStepLtoI = 1, kStepItoRD = 2 };

// Everything the kernels need, passed by value.
struct DevPop {
    int32_t N, NH, NC, NM, NPT, NB, nbx, nby, bs;
    int32_t NA;                // admin units with intervention windows (at least 1)
    const cs_params* P;
    PersonHot* hot;
    const PersonLinks* links;  // [N]
    const HouseholdRec* hhr;   // [NH]
    const int32_t* mcell_cell;
    const int32_t* mcell_adunit;
    const int32_t* cell_grid;
    const int32_t* cell_start;
    const int32_t* cell_members;
    const double* klookup;
    const double* khires;
    const float* klookup_f;    // the same tables in FP32, for the spatial pass's acceptance test
    const float* khires_f;
    DevPlaces pl[CS_MAX_PLACE_TYPES];
    // cold per-person state
    uint16_t* infection_time;
    uint16_t* recovery_time;
    uint16_t* sari_time;
    uint16_t* critical_time;
    uint16_t* stepdown_time;
    uint16_t* detected_time;
    // Each latent or infectious person's next transition time: the least of the
    // times IncubRecoverySweep tests (latent_time; case onset, recovery and the
    // severity times) that is not yet past, 0xFFFF when none is.  The transition
    // gather reads it alone; k_incub_events re-tests the person's own times.
    // ev_init, when nonzero, has the next gather form it from those times (set by
    // a state upload or run reset).
    uint16_t* next_ev;
    int32_t* ev_init;
    float* prob_absent;
    float* prob_care;
    int32_t* infector;
    int32_t* listpos;
    int16_t* infect_type;
    uint8_t* pstep;
    // cells
    int32_t* S;
    int32_t* L;
    int32_t* I;
    int32_t* R;
    int32_t* D;
    int32_t* S0;
    double* tot_prob;
    int32_t* slots;
    uint8_t* mark;
    // microcells
    uint8_t* socdist;
    uint8_t* moverest;
    DevIv* iv;
    DevStep* step;
    const unsigned long long* seed_src;  // the run's seed, written by begin_run / upload_state
    const double* t_src;                 // when set (batched graphs), k_set_step takes t from here
    int32_t* step_clock;                 // when set (day graphs), k_set_step takes t = clock * dt and advances it
    const int32_t* gate;                 // when set (day graphs), UpdateProbs kernels run only if *gate
    int32_t* close_window;     // [2] every place closed at ts has [0] <= ts < [1]
    // spatial proposal blocks
    const int32_t* cell_block;
    const int32_t* block_cell_ofs;
    const int32_t* block_cells;
    BlockCell* block_cell_info;  // [NC], rebuilt with S0
    BlockInfo* block_info;       // [NB], S0 rebuilt with S0
    double* block_row_cum;     // [NB][NB]
    // bound(b, B), which depends on the row of b, the row of B and the distance of
    // their columns only: [nby][nby][nbx], FP32 rounded up, filled once per geometry
    const float* bound_c;
    double* block_bound_tab;   // [NB][NB] bound(b, B) evaluated per UpdateProbs call, when bound_c
                               // could not be filled (a distance beyond the kernel table)
    int32_t bounds_static;     // 1: bound_c holds every bound; 0: k_block_rows fills block_bound_tab
                               // for the blocks with people
    int16_t* block_guide;      // [NB][NB] cut points of each row (Chen & Asau guide table)
    int16_t* cell_guide;       // [NC] cut points of each block's cell list
    // per-step scratch
    unsigned long long* claim; // [N], UINT64_MAX when unclaimed
    int32_t* queue;            // [N] newly infected people
    int32_t* counts;           // [kCntN] device-side sizes (see kCnt*)
    int32_t* touched;          // [NC] cells whose lists change this phase
    uint8_t* cell_flag;        // [NC]
    int32_t* act;              // [N] active people (infectors / latent+infectious)
    int32_t* act_cell;         // [N]
    int32_t* cnt;              // [NC] per-cell moves of the current phase (zero between phases)
    int32_t* cnt_ofs;          // [N] first contact-map entry of each active infector
    int32_t* cmap;             // [2N] active-list index of the infector owning each spatial contact
    int32_t cmap_cap;
    uint8_t* act_closed;       // [N] infector's place-closed-and-absent flag
    int2* place_work;          // [N * NPT] (active index << 3 | place type, place) of each place pass
    uint8_t* hh_flag;          // [NH] deferred household actions
    int32_t* hh_list;          // [NH]
    // households a place closure sends an adult home to (the host closure queue of
    // DoPlaceClose, src/Update.cpp:1220-1231): window packed as
    // (0xFFFF - start) << 16 | stop, 0 when none; listed once in carer_list
    uint32_t* carer_win;       // [NH]
    int32_t* carer_list;       // [NH]
    double* rad_origin;        // [2] where infection radii are measured from
    uint32_t* fc_flag;         // [N/32 + 1] people with a false-positive entry this step
    int32_t* fc_queue;         // [N] those people, once each
    cs_counters* C;
};

// kCntHH is last: the infect sweep zeroes the counters before it (kCntN - 1 of
// them) and leaves the household list, which its false cases may have filled, to
// the incub sweep's household pass.  The step's transition events are two lists in
// act / act_cell: latent people from the front (kCntEvents), infectious people
// from the back (kCntEventsInf), so that a warp of the transition kernel mostly
// takes one branch.
enum { kCntQueue = 0, kCntTouched = 1, kCntAct = 2, kCntContacts = 3, kCntPlaceWork = 4, kCntEvents = 5,
       kCntCarer = 6, kCntFalse = 7, kCntEventsInf = 8, kCntHH = 9, kCntN = 10 };

}  // namespace csb
