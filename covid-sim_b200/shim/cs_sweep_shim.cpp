// Drop-in replacement of the reference's two sweep entry points by the sm_100a
// library, for linking into the reference executable.
//
// The reference's Sweep.cpp is compiled with InfectSweep/IncubRecoverySweep renamed
// (-DInfectSweep=ref_InfectSweep -DIncubRecoverySweep=ref_IncubRecoverySweep) and
// this file provides the original symbols (src/Sweep.h:7-8), called by RunModel at
// src/CovidSim.cpp:1488 and 1490.  Everything else -- parameter files, population
// set-up, InitModel/SeedInfection, RecordSample and the output files -- stays the
// reference's own code.
//
//   first call           build cs_population / cs_params from the reference's
//                        globals (Hosts, Households, Mcells, CellLookup, Places, P)
//                        and create the device context;
//   first call of a run  copy the host state InitModel + SeedInfection left behind
//                        (people, cell lists, S0, tot_prob) to the device;
//   every step           run the device sweeps (one replay of the captured timestep
//                        graph: RunModel calls IncubRecoverySweep right after
//                        InfectSweep) and wait for them;
//   every output step    copy back what RecordSample reads on its next call:
//                        per-cell S/L/I/R/D and the StateT counters;
//   UpdateProbs          RunModel's own test (src/CovidSim.cpp:1515-1521: the
//                        susceptible fraction of State.S fell by more than 0.2 since
//                        the last call), evaluated at the same point of the step, then
//                        UpdateProbs recomputed on the device from its own counts;
//   interventions        the host's own trigger logic (RecordSample's start times,
//                        src/CovidSim.cpp:3598-3649) and TreatSweep
//                        (src/Sweep.cpp:1324-2004) keep running on the host; before
//                        each step what they changed is handed to the device: the
//                        parameter block (ControlPropCasesId, efficacies, CFR
//                        scales), each admin unit's case-isolation and household-
//                        quarantine start times, the microcells' social-distancing
//                        and movement-restriction status, and the outcome of every
//                        DoPlaceClose / DoPlaceOpen call TreatSweep made.  Those two
//                        calls and TreatSweep itself reach this file because the
//                        drop-in compiles Sweep.cpp with them renamed (oracle/Makefile),
//                        as it does the sweeps;
//   CS_DUMP_BLOCKS=<p>   (optional) each realisation's counter blocks -- t = 0 and
//                        every output step, what RecordSample reads, in the layout
//                        cs_gpu_run returns -- appended to <p>.<run>.blocks;
//   timing               the wall time of each realisation's sweep calls (from its
//                        first call on, the device context's creation excluded)
//                        and of the hand-over after TreatSweep,
//                        written to stderr at exit as oracle/ref_timing_shim.cpp
//                        writes the reference's:  SWEEPTIMING run=.. pop=.. threads=..
//                        steps=.. infect_s=.. incub_s=..
//
// Features outside the device sweep (digital contact tracing, airports, blanket
// movement restrictions, treatment/vaccination/key-worker prophylaxis, false
// positives, holidays, intervention delays by admin unit, and triggers counted per
// microcell or place rather than globally or per admin unit) stop the run with
// ERR_CRITICAL, the reference's own failure convention, rather than silently
// computing something else -- at set-up when the parameters rule them in, else at
// the first step at which they could act.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include <vector>

#include "Constants.h"
#include "Dist.h"
#include "Error.h"
#include "InfStat.h"
#include "Model.h"
#include "Param.h"
#include "Rand.h"
#include "Sweep.h"
#include "Update.h"

#include "covidsim_b200.h"

namespace {

cs_gpu_ctx* g_ctx = nullptr;
int g_run = -1;
PopVar g_base;  // StateT[0] as InitModel + SeedInfection left it; device counters add to it
double g_prev_prop = 1.0;      // RunModel's PreviousProportionSusceptible (src/CovidSim.cpp:1395)
bool g_update_probs = false;   // RunModel called UpdateProbs(0) after the last step
long g_step_in_run = 0;        // timesteps of the current realisation so far
int64_t g_tg_base = 0, g_si_base = 0, g_ntg_base = 0, g_tg_set = 0, g_si_set = 0, g_ntg_set = 0;
// A page-locked host array (cs_host_alloc): the state upload at a realisation's
// start and the copies back at output steps run at the link's rate from it.
template <typename T>
struct Pinned {
    T* p = nullptr;
    size_t n = 0;
    Pinned() = default;
    Pinned(const Pinned&) = delete;
    Pinned& operator=(const Pinned&) = delete;
    ~Pinned() { cs_host_free(p); }
    void resize(size_t m)
    {
        if (m == n) return;
        cs_host_free(p);
        p = (T*)cs_host_alloc(sizeof(T) * (m ? m : 1));
        if (!p) ERR_CRITICAL("GPU sweep: page-locked host allocation failed\n");
        n = m;
    }
    void assign(size_t m, T v)
    {
        resize(m);
        for (size_t i = 0; i < m; i++) p[i] = v;
    }
    size_t size() const { return n; }
    T* data() { return p; }
    T& operator[](size_t i) { return p[i]; }
    const T& operator[](size_t i) const { return p[i]; }
};

Pinned<int32_t> g_cells5;                     // S, L, I, R, D of every cell, side by side
int32_t *g_S = nullptr, *g_L = nullptr, *g_I = nullptr, *g_R = nullptr, *g_D = nullptr;
// When every cell fits 16 bits: the counter block and S, L, I, R, D of every cell as
// 16-bit values in one page-locked buffer (one copy per sample), and what the host's
// cells hold, so that a sample writes only the cells whose counts changed
Pinned<unsigned char> g_packed;
std::vector<uint16_t> g_host16;
bool g_use16 = false;
bool g_sample_queued = false;   // the packed copy back of the timestep in flight is queued
cs_params g_params;
// what the device holds of the host's intervention state
std::vector<uint8_t> g_sd, g_mr;              // per microcell: socdist, moverest (TreatStat)
std::vector<double> g_ci_start, g_hq_start;   // per admin unit start times
double g_ci_dur = -1, g_hq_dur = -1;
bool g_iv_sent = false;
std::vector<cs_place_event> g_events;         // TreatSweep's closures since the last step
// what the last microcell scan found: populated microcells untreated / treated for
// social distancing, and the earliest end of a treated one (TimeStepNow units)
long long g_sd_untreated = 0, g_sd_treated = 0;
unsigned int g_sd_min_end = 0xFFFFFFFFu;
struct RunTiming {
    int run;
    long steps = 0;
    double infect = 0.0, incub = 0.0;
    double upload = 0.0, copyback = 0.0;   // parts of the two above
    double wait = 0.0, scatter = 0.0, handover = 0.0;   // finer parts: the wait for the device's
                                                        // timestep, the copy into the host's cells,
                                                        // the hand-over after TreatSweep
    long scans = 0;                                     // microcell scans of the hand-over
    double upload_device = 0.0;                         // the upload's part in cs_gpu_upload_state
    double loop_start = -1.0, loop_end = -1.0;          // wall clock at the run's first sweep call and
                                                        // at the end of its last: RunModel's time
                                                        // stepping with the host code between sweeps
};
double g_upload_device = 0.0;   // the last upload's time in cs_gpu_upload_state
std::vector<RunTiming> g_timing;
FILE* g_dump = nullptr;

void check(int rc, const char* what)
{
    if (rc != CS_OK) ERR_CRITICAL_FMT("%s failed (%d): %s\n", what, rc, cs_gpu_last_error(g_ctx));
}

int8_t inf_of(const Person& a)
{
    if (a.is_susceptible()) return CS_INF_SUSCEPTIBLE;
    if (a.is_latent()) return CS_INF_LATENT;
    if (a.is_infectious_almost_symptomatic()) return CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC;
    if (a.is_infectious_asymptomatic_not_case()) return CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE;
    if (a.is_case()) return CS_INF_CASE;
    if (a.is_recovered_symp()) return CS_INF_RECOVERED_FROM_SYMP;
    if (a.is_recovered()) return CS_INF_RECOVERED_FROM_ASYMP;
    if (a.is_immune_at_start()) return CS_INF_IMMUNE_AT_START;
    if (a.is_dead_was_symp()) return CS_INF_DEAD_WAS_SYMP;
    return CS_INF_DEAD_WAS_ASYMP;
}

void copy_icdf(cs_icdf& dst, InverseCdf& src)
{
    for (int i = 0; i <= CDF_RES; i++) dst.v[i] = src[i];
}

cs_params params_from_reference()
{
    cs_params p;
    std::memset(&p, 0, sizeof(p));
    p.TimeStepsPerDay = P.TimeStepsPerDay;
    p.ModelTimeStep = P.ModelTimeStep;
    p.DoHouseholds = P.DoHouseholds; p.DoPlaces = P.DoPlaces; p.DoSpatial = 1; p.DoSymptoms = P.DoSymptoms;
    p.DoSeverity = P.DoSeverity; p.DoLatent = P.DoLatent; p.DoInfectiousnessProfile = P.DoInfectiousnessProfile;
    p.NoInfectiousnessSDinHH = P.NoInfectiousnessSDinHH; p.DoUTM_coords = P.DoUTM_coords;
    p.DoPeriodicBoundaries = P.DoPeriodicBoundaries; p.DoRealSymptWithdrawal = P.DoRealSymptWithdrawal;
    p.DoDeathCountsInS0 = P.DoDeath;
    p.NumPlaceTypes = P.NumPlaceTypes; p.HotelPlaceType = P.HotelPlaceType; p.CareHomePlaceType = P.CareHomePlaceType;
    p.PlaceTypeNoAirNum = P.PlaceTypeNoAirNum; p.IncludeStepDownToDeath = P.IncludeStepDownToDeath;
    p.CaseAbsentChildAgeCutoff = P.CaseAbsentChildAgeCutoff; p.DoHQretrigger = P.DoHQretrigger;
    p.LocalBeta = P.LocalBeta; p.HouseholdTrans = P.HouseholdTrans; p.FalsePositiveRate = P.FalsePositiveRate;
    p.CaseOrDeathThresholdBeforeAlert = P.CaseOrDeathThresholdBeforeAlert;
    p.cumDC_at_sample = P.FalsePositiveRate > 0 ? State.cumDC : 0;   // RecordSample's, read by DoFalseCase
    p.Seasonality = 1.0;
    for (int i = 0; i < MAX_HOUSEHOLD_SIZE; i++) p.HouseholdDenomLookup[i] = P.HouseholdDenomLookup[i];
    for (int i = 0; i < MAX_INFECTIOUS_STEPS; i++) p.infectiousness[i] = P.infectiousness[i];
    for (int t = 0; t < MAX_NUM_PLACE_TYPES; t++) {
        p.PlaceTypeTrans[t] = P.PlaceTypeTrans[t];
        p.PlaceTypeGroupSizeParam1[t] = (t < P.NumPlaceTypes) ? P.PlaceTypeGroupSizeParam1[t] : 1.0;
        p.PlaceTypePropBetweenGroupLinks[t] = P.PlaceTypePropBetweenGroupLinks[t];
        p.SymptPlaceTypeContactRate[t] = P.SymptPlaceTypeContactRate[t];
        p.SymptPlaceTypeWithdrawalProp[t] = P.SymptPlaceTypeWithdrawalProp[t];
    }
    p.SymptSpatialContactRate = P.SymptSpatialContactRate;
    for (int a = 0; a < NUM_AGE_GROUPS; a++) {
        p.RelativeSpatialContact[a] = P.RelativeSpatialContact[a];
        p.RelativeSpatialContactSusc[a] = P.RelativeSpatialContactSusc[a];
        p.AgeSusceptibility[a] = P.AgeSusceptibility[a];
        p.AgeInfectiousness[a] = P.AgeInfectiousness[a];
        p.ProportionSymptomatic[a] = P.ProportionSymptomatic[a];
        for (int b = 0; b < NUM_AGE_GROUPS; b++) {
            p.WAIFW_Matrix[a][b] = P.WAIFW_Matrix[a][b];
            p.WAIFW_Matrix_SpatialOnly[a][b] = P.WAIFW_Matrix_SpatialOnly[a][b];
        }
        p.Mean_MildToRecovery[a] = P.Mean_MildToRecovery[a]; p.Mean_ILIToRecovery[a] = P.Mean_ILIToRecovery[a];
        p.Mean_SARIToRecovery[a] = P.Mean_SARIToRecovery[a]; p.Mean_CriticalToCritRecov[a] = P.Mean_CriticalToCritRecov[a];
        p.Mean_CritRecovToRecov[a] = P.Mean_CritRecovToRecov[a]; p.Mean_StepdownToDeath[a] = P.Mean_StepdownToDeath[a];
        p.Mean_ILIToSARI[a] = P.Mean_ILIToSARI[a]; p.Mean_SARIToCritical[a] = P.Mean_SARIToCritical[a];
        p.Mean_CriticalToDeath[a] = P.Mean_CriticalToDeath[a]; p.Mean_SARIToDeath[a] = P.Mean_SARIToDeath[a];
        p.Mean_ILIToDeath[a] = P.Mean_ILIToDeath[a];
        p.Prop_ILI_ByAge[a] = P.Prop_ILI_ByAge[a]; p.Prop_SARI_ByAge[a] = P.Prop_SARI_ByAge[a];
        p.Prop_Critical_ByAge[a] = P.Prop_Critical_ByAge[a];
        p.CFR_SARI_ByAge[a] = P.CFR_SARI_ByAge[a]; p.CFR_Critical_ByAge[a] = P.CFR_Critical_ByAge[a];
        p.CFR_ILI_ByAge[a] = P.CFR_ILI_ByAge[a];
    }
    p.CareHomeResidentHouseholdScaling = P.CareHomeResidentHouseholdScaling;
    p.CareHomeResidentSpatialScaling = P.CareHomeResidentSpatialScaling;
    p.CareHomeWorkerGroupScaling = P.CareHomeWorkerGroupScaling;
    p.CareHomeResidentPlaceScaling = P.CareHomeResidentPlaceScaling;
    p.CareHomeRelProbHosp = P.CareHomeRelProbHosp;
    for (int i = 0; i < CS_NUM_NPI; i++)
        for (int j = 0; j < CS_NUM_SETTINGS; j++) p.Efficacies[i][j] = P.Efficacies[i][j];
    p.MoveRestrEffect = P.MoveRestrEffect;
    p.DoBlanketMoveRestr = P.DoBlanketMoveRestr;
    p.MoveRestrTimeStart = P.MoveRestrTimeStart; p.MoveRestrDuration = P.MoveRestrDuration;
    p.MoveRestrRadius2 = P.MoveRestrRadius2;
    p.LocationInitialInfection[0] = P.LocationInitialInfection[0][0];
    p.LocationInitialInfection[1] = P.LocationInitialInfection[0][1];
    p.LatentPeriod = P.LatentPeriod; p.InfectiousPeriod = P.InfectiousPeriod; p.LatentToSymptDelay = P.LatentToSymptDelay;
    p.SymptInfectiousness = P.SymptInfectiousness; p.AsymptInfectiousness = P.AsymptInfectiousness;
    p.InfectiousnessSD = P.InfectiousnessSD;
    copy_icdf(p.latent_icdf, P.latent_icdf); copy_icdf(p.infectious_icdf, P.infectious_icdf);
    copy_icdf(p.MildToRecovery_icdf, P.MildToRecovery_icdf); copy_icdf(p.ILIToRecovery_icdf, P.ILIToRecovery_icdf);
    copy_icdf(p.SARIToRecovery_icdf, P.SARIToRecovery_icdf); copy_icdf(p.CriticalToCritRecov_icdf, P.CriticalToCritRecov_icdf);
    copy_icdf(p.CritRecovToRecov_icdf, P.CritRecovToRecov_icdf); copy_icdf(p.ILIToSARI_icdf, P.ILIToSARI_icdf);
    copy_icdf(p.SARIToCritical_icdf, P.SARIToCritical_icdf); copy_icdf(p.ILIToDeath_icdf, P.ILIToDeath_icdf);
    copy_icdf(p.SARIToDeath_icdf, P.SARIToDeath_icdf); copy_icdf(p.StepdownToDeath_icdf, P.StepdownToDeath_icdf);
    copy_icdf(p.CriticalToDeath_icdf, P.CriticalToDeath_icdf);
    p.CFR_Critical_Scale_Current = P.CFR_Critical_Scale_Current; p.CFR_SARI_Scale_Current = P.CFR_SARI_Scale_Current;
    p.CFR_ILI_Scale_Current = P.CFR_ILI_Scale_Current;
    p.ControlPropCasesId = P.ControlPropCasesId;
    p.CaseIsolationProp = P.CaseIsolationProp; p.HQuarantinePropHouseCompliant = P.HQuarantinePropHouseCompliant;
    p.HQuarantinePropIndivCompliant = P.HQuarantinePropIndivCompliant; p.HQuarantineDelay = P.HQuarantineDelay;
    p.CaseAbsentChildPropAdultCarers = P.CaseAbsentChildPropAdultCarers;
    for (int t = 0; t < MAX_NUM_PLACE_TYPES; t++)
        p.PlaceClosePropAttending[t] = (t < P.NumPlaceTypes) ? P.PlaceClosePropAttending[t] : 0.0;
    p.usCaseIsolationDelay = P.usCaseIsolationDelay; p.usCaseIsolationDuration = P.usCaseIsolationDuration;
    p.usCaseAbsenteeismDelay = P.usCaseAbsenteeismDelay; p.usCaseAbsenteeismDuration = P.usCaseAbsenteeismDuration;
    p.usHQuarantineHouseDuration = P.usHQuarantineHouseDuration;
    p.ncw = P.ncw; p.nch = P.nch;
    p.cell_width = P.in_cells_.width; p.cell_height = P.in_cells_.height;
    p.width_deg = P.in_degrees_.width; p.height_deg = P.in_degrees_.height;
    p.bbox_bottom_left_y = P.SpatialBoundingBox.bottom_left().y;
    for (int i = 0; i <= DEGREES_PER_TURN; i++) { p.sinx[i] = P.sinx[i]; p.cosx[i] = P.cosx[i]; }
    for (int i = 0; i <= 1000; i++) p.asin2sqx[i] = P.asin2sqx[i];
    p.kernel_size = P.KernelLookup.size_;
    p.kernel_expansion = P.KernelLookup.expansion_factor_;
    p.block_cells = 0;
    return p;
}

void unsupported_features()
{
    if (P.DoDigitalContactTracing) ERR_CRITICAL("GPU sweep: digital contact tracing is not supported\n");
    if (P.DoAirports) ERR_CRITICAL("GPU sweep: airports / travel are not supported\n");
    if (P.DoInterventionDelaysByAdUnit) ERR_CRITICAL("GPU sweep: intervention delays by admin unit are not supported\n");
    if (P.InfectionImportRate1 > 0 || P.InfectionImportRate2 > 0 || P.DurImportTimeProfile > 0)
        ERR_CRITICAL("GPU sweep: importation of infections during a run is not supported\n");
    if (P.FalsePositivePerCapitaIncidence > 0)
        ERR_CRITICAL("GPU sweep: false-positive cases drawn at a per-capita incidence are not supported\n");
    if (P.DoSI) ERR_CRITICAL("GPU sweep: the SI model (no IncubRecoverySweep) is not supported\n");
    if (P.DoAdUnits && P.DoAdminTriggers && P.NumAdunits > CS_MAX_ADUNITS)
        ERR_CRITICAL_FMT("GPU sweep: admin-unit triggers over more than %d admin units are not supported\n", CS_MAX_ADUNITS);
}

// Host interventions the device does not model, checked at each step against the
// host's current start times (t is the time of the TreatSweep that just ran).
void unsupported_at(double t)
{
    if (t >= P.TreatTimeStart) ERR_CRITICAL("GPU sweep: treatment is not supported\n");
    if (t >= P.VaccTimeStart || t >= P.VaccTimeStartGeo) ERR_CRITICAL("GPU sweep: vaccination is not supported\n");
    if (t >= P.KeyWorkerProphTimeStart) ERR_CRITICAL("GPU sweep: key-worker prophylaxis is not supported\n");
    const bool any = t >= P.PlaceCloseTimeStart || t >= P.SocDistTimeStart || t >= P.MoveRestrTimeStart;
    if (any && !P.DoGlobalTriggers && !P.DoAdminTriggers)
        ERR_CRITICAL("GPU sweep: triggers counted per microcell are not supported (use global or admin-unit triggers)\n");
    // DoDetectedCase's and DoCase's own place closures (src/Update.cpp:544-560, 821-830)
    if (t >= P.PlaceCloseTimeStart && P.DoPlaces) {
        if (!P.AbsenteeismPlaceClosure && !P.DoAdminTriggers && !(P.DoGlobalTriggers && P.PlaceCloseCellIncThresh < 1000000000))
            ERR_CRITICAL("GPU sweep: place closure by detected cases is not supported\n");
        if (P.AbsenteeismPlaceClosure && !P.DoAdminTriggers && !P.DoGlobalTriggers)
            ERR_CRITICAL("GPU sweep: place closure by absenteeism is not supported\n");
        if (P.PlaceCloseByAdminUnit) ERR_CRITICAL("GPU sweep: place closure by admin-unit case proportions is not supported\n");
    }
}

void create_context()
{
    unsupported_features();
    const int N = P.PopSize, NH = P.NumHouseholds, NC = P.NumPopulatedCells, NM = P.NumMicrocells, NPT = P.NumPlaceTypes;
    static std::vector<int32_t> hh(N), mc(N), place((size_t)NPT * N), hh_first(NH), mcell_cell(NM, 0), mcell_ad(NM),
        cell_grid(NC), cell_start(NC + 1), cell_members(N);
    static std::vector<uint8_t> age(N), flags(N);
    static std::vector<uint16_t> group((size_t)NPT * N), hh_nh(NH), hh_nhr(NH);
    static std::vector<float> hx(NH), hy(NH);
    for (int i = 0; i < N; i++) {
        hh[i] = Hosts[i].hh;
        mc[i] = Hosts[i].mcell;
        age[i] = Hosts[i].age;
        flags[i] = (Hosts[i].care_home_resident ? CS_PF_CARE_HOME_RESIDENT : 0) |
                   (Hosts[i].esocdist_comply ? CS_PF_ESOCDIST_COMPLY : 0) | (Hosts[i].keyworker ? CS_PF_KEYWORKER : 0);
        for (int t = 0; t < NPT; t++) {
            place[(size_t)t * N + i] = Hosts[i].PlaceLinks[t];
            group[(size_t)t * N + i] = Hosts[i].PlaceGroupLinks[t];
        }
    }
    for (int h = 0; h < NH; h++) {
        hh_first[h] = Households[h].FirstPerson;
        hh_nh[h] = Households[h].nh;
        hh_nhr[h] = Households[h].nhr;
        hx[h] = Households[h].loc.x;
        hy[h] = Households[h].loc.y;
    }
    cell_start[0] = 0;
    for (int c = 0; c < NC; c++) {
        Cell* ct = CellLookup[c];
        cell_grid[c] = (int32_t)(ct - Cells);
        for (int k = 0; k < ct->n; k++) cell_members[cell_start[c] + k] = ct->members[k];
        cell_start[c + 1] = cell_start[c] + ct->n;
    }
    std::vector<int32_t> cell_index_of_grid(P.NumCells, -1);
    for (int c = 0; c < NC; c++) cell_index_of_grid[cell_grid[c]] = c;
    for (int m = 0; m < NM; m++) {
        int x = m / P.total_microcells_high_, y = m % P.total_microcells_high_;
        int grid = (x / P.NMCL) * P.nch + (y / P.NMCL);
        mcell_cell[m] = cell_index_of_grid[grid] >= 0 ? cell_index_of_grid[grid] : 0;
        mcell_ad[m] = Mcells[m].adunit;
    }
    static std::vector<int32_t> pl_mcell[MAX_NUM_PLACE_TYPES], pl_mofs[MAX_NUM_PLACE_TYPES], pl_members[MAX_NUM_PLACE_TYPES],
        pl_gofs[MAX_NUM_PLACE_TYPES], pl_gstart[MAX_NUM_PLACE_TYPES], pl_gsize[MAX_NUM_PLACE_TYPES];
    static std::vector<float> pl_x[MAX_NUM_PLACE_TYPES], pl_y[MAX_NUM_PLACE_TYPES];
    cs_population pop;
    std::memset(&pop, 0, sizeof(pop));
    for (int t = 0; t < NPT; t++) {
        int np = P.Nplace[t];
        pl_mcell[t].resize(np); pl_x[t].resize(np); pl_y[t].resize(np);
        pl_mofs[t].assign(np + 1, 0); pl_gofs[t].assign(np + 1, 0);
        for (int l = 0; l < np; l++) {
            Place& pp = Places[t][l];
            pl_mcell[t][l] = pp.mcell;
            pl_x[t][l] = pp.loc.x;
            pl_y[t][l] = pp.loc.y;
            pl_mofs[t][l + 1] = pl_mofs[t][l] + pp.n;
            pl_gofs[t][l + 1] = pl_gofs[t][l] + pp.ng;
        }
        pl_members[t].resize(pl_mofs[t][np]);
        pl_gstart[t].resize(pl_gofs[t][np]);
        pl_gsize[t].resize(pl_gofs[t][np]);
        for (int l = 0; l < np; l++) {
            Place& pp = Places[t][l];
            for (int k = 0; k < pp.n; k++) pl_members[t][pl_mofs[t][l] + k] = pp.members[k];
            for (int g = 0; g < pp.ng; g++) {
                pl_gstart[t][pl_gofs[t][l] + g] = pp.group_start[g];
                pl_gsize[t][pl_gofs[t][l] + g] = pp.group_size[g];
            }
        }
        pop.n_places[t] = np;
        pop.place_mcell[t] = pl_mcell[t].data(); pop.place_x[t] = pl_x[t].data(); pop.place_y[t] = pl_y[t].data();
        pop.place_member_ofs[t] = pl_mofs[t].data(); pop.place_members[t] = pl_members[t].data();
        pop.place_group_ofs[t] = pl_gofs[t].data(); pop.group_start[t] = pl_gstart[t].data();
        pop.group_size[t] = pl_gsize[t].data();
    }
    // the spatial kernel table exactly as KernelLookup::setup/init built it at the end
    // of set-up (src/SetupModel.cpp:196-209, 308-309)
    double longest = dist2_raw(0, 0, P.in_degrees_.width, P.in_degrees_.height);
    double tw = dist2_raw(0, 0, P.in_degrees_.width, 0), th = dist2_raw(0, 0, 0, P.in_degrees_.height);
    if (tw > longest) longest = tw;
    if (th > longest) longest = th;
    if (P.DoPeriodicBoundaries) longest *= 0.25;
    static std::vector<double> klook(P.KernelLookup.size_ + 1), khi(P.KernelLookup.size_ + 1);
    g_params = params_from_reference();
    if (cs_build_kernel_table(P.Kernel.type_, P.Kernel.scale_, P.Kernel.shape_, P.Kernel.p3_, P.Kernel.p4_, longest,
                              P.KernelLookup.size_, P.KernelLookup.expansion_factor_, klook.data(), khi.data(),
                              &g_params.kernel_delta) != CS_OK)
        ERR_CRITICAL("GPU sweep: kernel table\n");
    pop.n_people = N; pop.n_households = NH; pop.n_cells = NC; pop.n_mcells = NM; pop.num_place_types = NPT;
    pop.n_adunits = P.NumAdunits;
    pop.person_hh = hh.data(); pop.person_mcell = mc.data(); pop.person_age = age.data(); pop.person_flags = flags.data();
    pop.person_place = place.data(); pop.person_group = group.data();
    pop.hh_first = hh_first.data(); pop.hh_nh = hh_nh.data(); pop.hh_nhr = hh_nhr.data(); pop.hh_x = hx.data(); pop.hh_y = hy.data();
    pop.mcell_cell = mcell_cell.data(); pop.mcell_adunit = mcell_ad.data();
    pop.cell_grid = cell_grid.data(); pop.cell_start = cell_start.data(); pop.cell_members = cell_members.data();
    pop.kernel_lookup = klook.data(); pop.kernel_hi_res = khi.data();
    int rc = cs_gpu_create(&pop, &g_params, 0, &g_ctx);
    check(rc, "cs_gpu_create");
    g_cells5.resize(5 * (size_t)NC);
    g_S = g_cells5.data(); g_L = g_S + NC; g_I = g_L + NC; g_R = g_I + NC; g_D = g_R + NC;
    {   // the copies back travel as 16-bit counts when no cell holds more than 65,535 people
        int most = 0;
        for (int c = 0; c < NC; c++) most = CellLookup[c]->n > most ? CellLookup[c]->n : most;
        g_use16 = most <= 65535;
        if (g_use16) {
            g_packed.resize(cs_gpu_sample_packed_bytes(g_ctx));
            g_host16.assign(5 * (size_t)NC, 0);
        }
    }
    std::fprintf(stderr, "GPU sweep: %d people, %d populated cells on device\n", N, NC);
}

void dump_block();

// Host staging of the start state, kept from run to run so that later runs write
// into memory that is already mapped.
struct Staging {
    Pinned<int8_t> inf;
    Pinned<uint8_t> sev, fl;
    Pinned<uint16_t> it, lt, rt, st, ct, sd, as, ae, iso, qs, dt;
    Pinned<float> infn, susc, pa, pc;
    Pinned<int32_t> infector, listpos, slots, S0, cS, cL, cI, cR, cD;
    std::vector<int32_t> cell_ofs;
    Pinned<int16_t> itype;
    Pinned<double> tp;
};
Staging g_stage;

void upload_run_state(int run)
{
    const int N = P.PopSize, NC = P.NumPopulatedCells;
    Staging& g = g_stage;
    if ((int)g.inf.size() != N || (int)g.tp.size() != NC) {
        for (auto* v : {&g.sev, &g.fl}) v->resize(N);
        for (auto* v : {&g.it, &g.lt, &g.rt, &g.st, &g.ct, &g.sd, &g.as, &g.ae, &g.iso, &g.qs, &g.dt}) v->resize(N);
        for (auto* v : {&g.infn, &g.susc, &g.pa, &g.pc}) v->resize(N);
        for (auto* v : {&g.infector, &g.listpos, &g.slots}) v->resize(N);
        for (auto* v : {&g.S0, &g.cS, &g.cL, &g.cI, &g.cR, &g.cD}) v->resize(NC);
        g.inf.resize(N); g.itype.resize(N); g.tp.resize(NC);
        g.cell_ofs.assign(NC + 1, 0);
        for (int c = 0; c < NC; c++) g.cell_ofs[c + 1] = g.cell_ofs[c] + CellLookup[c]->n;
    }
    cs_state_view v;
    std::memset(&v, 0, sizeof(v));
    v.inf = g.inf.data(); v.severity = g.sev.data(); v.flags = g.fl.data(); v.infection_time = g.it.data();
    v.latent_time = g.lt.data(); v.recovery_or_death_time = g.rt.data(); v.SARI_time = g.st.data();
    v.Critical_time = g.ct.data(); v.Stepdown_time = g.sd.data(); v.absent_start_time = g.as.data();
    v.absent_stop_time = g.ae.data(); v.isolation_start_time = g.iso.data(); v.quar_start_time = g.qs.data();
    v.detected_time = g.dt.data(); v.infectiousness = g.infn.data(); v.susc = g.susc.data(); v.ProbAbsent = g.pa.data();
    v.ProbCare = g.pc.data(); v.infector = g.infector.data(); v.infect_type = g.itype.data(); v.listpos = g.listpos.data();
    v.cell_S = g.cS.data(); v.cell_L = g.cL.data(); v.cell_I = g.cI.data(); v.cell_R = g.cR.data(); v.cell_D = g.cD.data();
    v.cell_S0 = g.S0.data(); v.cell_tot_prob = g.tp.data(); v.cell_slots = g.slots.data();
    // the people in slices: each is sent (cs_gpu_upload_people) as soon as it is
    // filled, so its copy to the device runs while the next slice is filled
    double t_sent = 0.0;
    const int kSlices = 8;
    for (int q = 0; q < kSlices; q++) {
        const int lo = (int)((long long)N * q / kSlices), hi = (int)((long long)N * (q + 1) / kSlices);
#pragma omp parallel for schedule(static)
        for (int i = lo; i < hi; i++) {
            const Person& a = Hosts[i];
            g.inf[i] = inf_of(a);
            g.sev[i] = (uint8_t)((int)a.Severity_Current | ((int)a.Severity_Final << 4));
            g.fl[i] = (uint8_t)((a.to_die ? CS_DF_TO_DIE : 0) | (a.detected ? CS_DF_DETECTED : 0) |
                                ((HostsQuarantine[i].comply & 3) << CS_DF_QUAR_COMPLY_SHIFT));
            g.it[i] = a.infection_time; g.lt[i] = a.latent_time; g.rt[i] = a.recovery_or_death_time;
            g.st[i] = a.SARI_time; g.ct[i] = a.Critical_time; g.sd[i] = a.Stepdown_time;
            g.as[i] = a.absent_start_time; g.ae[i] = a.absent_stop_time; g.iso[i] = a.isolation_start_time;
            g.qs[i] = HostsQuarantine[i].start_time; g.dt[i] = a.detected_time;
            g.infn[i] = a.infectiousness; g.susc[i] = a.susc; g.pa[i] = a.ProbAbsent; g.pc[i] = a.ProbCare;
            g.infector[i] = a.infector; g.itype[i] = a.infect_type; g.listpos[i] = a.listpos;
        }
        const double t0 = omp_get_wtime();
        check(cs_gpu_upload_people(g_ctx, &v, lo, hi - lo), "cs_gpu_upload_people");
        t_sent += omp_get_wtime() - t0;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int c = 0; c < NC; c++) {
        const Cell* x = CellLookup[c];
        std::memcpy(g.slots.data() + g.cell_ofs[c], x->susceptible, sizeof(int32_t) * (size_t)x->n);
        g.cS[c] = x->S; g.cL[c] = x->L; g.cI[c] = x->I; g.cR[c] = x->R; g.cD[c] = x->D; g.S0[c] = x->S0;
        g.tp[c] = x->tot_prob;
        if (g_use16) {   // what the host's cells hold: the copies back compare against it
            uint16_t* h = g_host16.data();
            h[c] = (uint16_t)x->S; h[NC + c] = (uint16_t)x->L; h[2 * NC + c] = (uint16_t)x->I;
            h[3 * NC + c] = (uint16_t)x->R; h[4 * NC + c] = (uint16_t)x->D;
        }
    }
    uint64_t seed = ((uint64_t)(uint32_t)P.runSeed1 << 32) ^ (uint32_t)P.runSeed2 ^ (0x9E3779B97F4A7C15ull * (uint64_t)(run + 1));
    const double t_up = omp_get_wtime();
    check(cs_gpu_upload_state(g_ctx, seed, &v), "cs_gpu_upload_state");
    g_upload_device = omp_get_wtime() - t_up + t_sent;
    // seeding ran DoInfect on the host (thread 0's counters); the device counts from zero
    for (int j = 1; j < P.NumThreads; j++)
        if (StateT[j].cumI || StateT[j].cumC) ERR_CRITICAL("GPU sweep: host counters outside thread 0 at run start\n");
    std::memcpy(&g_base, &StateT[0], sizeof(PopVar));
    // the upload reset the device's closures, microcell status and windows, as
    // InitModel reset the host's
    g_sd.assign(P.NumMicrocells, (uint8_t)CS_TREAT_UNTREATED);
    g_mr.assign(P.NumMicrocells, (uint8_t)CS_TREAT_UNTREATED);
    g_sd_untreated = P.NumPopulatedMicrocells;
    g_sd_treated = 0;
    g_sd_min_end = 0xFFFFFFFFu;
    g_iv_sent = false;
    g_events.clear();
    g_prev_prop = 1.0;
    g_update_probs = false;
    g_step_in_run = 0;
    g_tg_base = g_si_base = g_ntg_base = 0;
    g_tg_set = g_si_set = g_ntg_set = 0;
    if (const char* dump = std::getenv("CS_DUMP_BLOCKS")) {
        if (g_dump) std::fclose(g_dump);
        char path[4096];
        std::snprintf(path, sizeof(path), "%s.%d.blocks", dump, run);
        g_dump = std::fopen(path, "wb");
        if (!g_dump) ERR_CRITICAL_FMT("GPU sweep: cannot write %s\n", path);
        dump_block();
    }
}

// Below this many cells the copy into the host's cells runs on one thread: waking
// the team costs more than the loop.
constexpr int kParallelCells = 16384;

// RecordSample (src/CovidSim.cpp:3024-3120) reads per-cell counts and StateT[].
void sync_back()
{
    cs_counters k;
    const int NC = P.NumPopulatedCells;
    if (g_use16) {
        if (g_sample_queued) check(cs_gpu_sample_packed_end(g_ctx, g_packed.data()), "cs_gpu_sample_packed_end");
        else check(cs_gpu_get_sample_packed(g_ctx, g_packed.data(), g_packed.size()), "cs_gpu_get_sample_packed");
        g_sample_queued = false;
        std::memcpy(&k, g_packed.data(), sizeof k);
    } else {
        check(cs_gpu_get_sample(g_ctx, g_S, g_L, g_I, g_R, g_D, &k), "cs_gpu_get_sample");
    }
    const double t_sc = omp_get_wtime();
    if (g_use16) {
        // only the cells whose counts changed since the last sample are written: the
        // host's cells change through these writes alone between uploads
        const uint16_t* v = reinterpret_cast<const uint16_t*>(g_packed.data() + sizeof(cs_counters));
        uint16_t* h = g_host16.data();
#pragma omp parallel for schedule(static) if (NC >= kParallelCells)
        for (int c = 0; c < NC; c++) {
            if (v[c] == h[c] && v[NC + c] == h[NC + c] && v[2 * NC + c] == h[2 * NC + c] &&
                v[3 * NC + c] == h[3 * NC + c] && v[4 * NC + c] == h[4 * NC + c])
                continue;
            Cell* x = CellLookup[c];
            x->S = h[c] = v[c]; x->L = h[NC + c] = v[NC + c]; x->I = h[2 * NC + c] = v[2 * NC + c];
            x->R = h[3 * NC + c] = v[3 * NC + c]; x->D = h[4 * NC + c] = v[4 * NC + c];
        }
    } else {
#pragma omp parallel for schedule(static) if (NC >= kParallelCells)
        for (int c = 0; c < NC; c++) {
            Cell* x = CellLookup[c];
            x->S = g_S[c]; x->L = g_L[c]; x->I = g_I[c]; x->R = g_R[c]; x->D = g_D[c];
        }
    }
    if (!g_timing.empty()) g_timing.back().scatter += omp_get_wtime() - t_sc;
    PopVar& s = StateT[0];
    const PopVar& b = g_base;
    s.cumI = b.cumI + (int)k.cumI; s.cumC = b.cumC + (int)k.cumC; s.cumDC = b.cumDC + (int)k.cumDC;
    s.cumFC = b.cumFC + (int)k.cumFC; s.cumHQ = b.cumHQ + (int)k.cumHQ; s.cumAC = b.cumAC + (int)k.cumAC;
    s.cumAA = b.cumAA + (int)k.cumAA; s.cumACS = b.cumACS + (int)k.cumACS;
    for (int i = 0; i < INFECT_TYPE_MASK; i++) s.cumItype[i] = b.cumItype[i] + (int)k.cumItype[i];
    for (int a = 0; a < NUM_AGE_GROUPS; a++) {
        s.cumIa[a] = b.cumIa[a] + (int)k.cumIa[a];
        s.cumCa[a] = b.cumCa[a] + (int)k.cumCa[a];
        s.cumDa[a] = b.cumDa[a] + (int)k.cumDa[a];
    }
    s.Mild = b.Mild + (int)k.Mild; s.ILI = b.ILI + (int)k.ILI; s.SARI = b.SARI + (int)k.SARI;
    s.Critical = b.Critical + (int)k.Critical; s.CritRecov = b.CritRecov + (int)k.CritRecov;
    s.cumMild = b.cumMild + (int)k.cumMild; s.cumILI = b.cumILI + (int)k.cumILI; s.cumSARI = b.cumSARI + (int)k.cumSARI;
    s.cumCritical = b.cumCritical + (int)k.cumCritical; s.cumCritRecov = b.cumCritRecov + (int)k.cumCritRecov;
    s.cumDeath_ILI = b.cumDeath_ILI + (int)k.cumDeath_ILI; s.cumDeath_SARI = b.cumDeath_SARI + (int)k.cumDeath_SARI;
    s.cumDeath_Critical = b.cumDeath_Critical + (int)k.cumDeath_Critical;
    for (int i = 0; i < 2; i++) {
        s.cumI_keyworker[i] = b.cumI_keyworker[i] + (int)k.cumI_keyworker[i];
        s.cumC_keyworker[i] = b.cumC_keyworker[i] + (int)k.cumC_keyworker[i];
    }
    // per admin unit: what RecordSample's admin-unit triggers and tables read
    // (src/CovidSim.cpp:3433-3450)
    if (P.DoAdUnits)
        for (int a = 0; a < P.NumAdunits && a < CS_MAX_ADUNITS; a++) {
            s.cumI_adunit[a] = b.cumI_adunit[a] + (int)k.cumI_adunit[a];
            s.cumC_adunit[a] = b.cumC_adunit[a] + (int)k.cumC_adunit[a];
            s.cumD_adunit[a] = b.cumD_adunit[a] + (int)k.cumD_adunit[a];
            s.cumDC_adunit[a] = b.cumDC_adunit[a] + (int)k.cumDC_adunit[a];
            s.cumCritical_adunit[a] = b.cumCritical_adunit[a] + (int)k.cumCritical_adunit[a];
            s.Critical_adunit[a] = b.Critical_adunit[a] + (int)k.Critical_adunit[a];
        }
    // infection radii (DoInfect, src/Update.cpp:116-127): the device's since the upload
    s.sumRad2 = b.sumRad2 + (double)k.sumRad2_q / 4294967296.0;
    {
        double m;
        std::memcpy(&m, &k.maxRad2_bits, sizeof m);
        s.maxRad2 = m > b.maxRad2 ? m : b.maxRad2;
    }
    // generation-time sums are read and zeroed by each RecordSample: hand over increments
    if (s.cumTG != g_tg_set || s.nTG != g_ntg_set) { g_tg_base += g_tg_set; g_si_base += g_si_set; g_ntg_base += g_ntg_set; }
    g_tg_set = k.cumTG - g_tg_base; g_si_set = k.cumSI - g_si_base; g_ntg_set = k.nTG - g_ntg_base;
    s.cumTG = (int)g_tg_set; s.cumSI = (int)g_si_set; s.nTG = (int)g_ntg_set;
}

// One counter block of the realisation, as RecordSample would sum it now: the
// cells' S/L/I/R/D, thread 0's counters (the only ones the drop-in writes) and the
// device's cumulative generation-time sums.
void dump_block()
{
    if (!g_dump) return;
    cs_counters b;
    std::memset(&b, 0, sizeof(b));
    for (int c = 0; c < P.NumPopulatedCells; c++) {
        const Cell* x = CellLookup[c];
        b.S += x->S; b.L += x->L; b.I += x->I; b.R += x->R; b.D += x->D;
    }
    b.cumR = b.R; b.cumD = b.D;   // as RecordSample sets them (src/CovidSim.cpp:3055-3056)
    const PopVar& s = StateT[0];
    b.cumI = s.cumI; b.cumC = s.cumC; b.cumDC = s.cumDC; b.cumFC = s.cumFC; b.cumHQ = s.cumHQ;
    b.cumAC = s.cumAC; b.cumAA = s.cumAA; b.cumACS = s.cumACS;
    for (int i = 0; i < INFECT_TYPE_MASK; i++) b.cumItype[i] = s.cumItype[i];
    for (int a = 0; a < NUM_AGE_GROUPS; a++) { b.cumIa[a] = s.cumIa[a]; b.cumCa[a] = s.cumCa[a]; b.cumDa[a] = s.cumDa[a]; }
    b.Mild = s.Mild; b.ILI = s.ILI; b.SARI = s.SARI; b.Critical = s.Critical; b.CritRecov = s.CritRecov;
    b.cumMild = s.cumMild; b.cumILI = s.cumILI; b.cumSARI = s.cumSARI; b.cumCritical = s.cumCritical;
    b.cumCritRecov = s.cumCritRecov; b.cumDeath_ILI = s.cumDeath_ILI; b.cumDeath_SARI = s.cumDeath_SARI;
    b.cumDeath_Critical = s.cumDeath_Critical;
    if (P.DoAdUnits)
        for (int a = 0; a < P.NumAdunits && a < CS_MAX_ADUNITS; a++) {
            b.cumI_adunit[a] = s.cumI_adunit[a]; b.cumC_adunit[a] = s.cumC_adunit[a];
            b.cumD_adunit[a] = s.cumD_adunit[a]; b.cumDC_adunit[a] = s.cumDC_adunit[a];
            b.cumCritical_adunit[a] = s.cumCritical_adunit[a]; b.Critical_adunit[a] = s.Critical_adunit[a];
        }
    cs_counters k;
    check(cs_gpu_get_counters(g_ctx, &k), "cs_gpu_get_counters");
    b.cumTG = g_base.cumTG + k.cumTG; b.cumSI = g_base.cumSI + k.cumSI; b.nTG = g_base.nTG + k.nTG;
    b.sumRad2_q = (int64_t)(s.sumRad2 * 4294967296.0);
    std::memcpy(&b.maxRad2_bits, &s.maxRad2, sizeof(double));
    if (std::fwrite(&b, sizeof(b), 1, g_dump) != 1) ERR_CRITICAL("GPU sweep: writing the counter blocks failed\n");
}

// Everything the host's run loop changed between two sweeps that the device sweep
// reads, handed over before the next sweep (t is the coming step's time).
void mirror_host_interventions(double t)
{
    const double t_prev = t - P.ModelTimeStep;   // the time TreatSweep last ran at
    if (t_prev >= 0) unsupported_at(t_prev);
    // the parameter block.  During a run the reference changes parameters only in
    // RecordSample (ControlPropCasesId after the alert, src/CovidSim.cpp:3592) and
    // UpdateCFRs (the CFR scales, :2840-2867), and seasonality is read per day
    // (src/Sweep.cpp:296); the efficacies are fixed after reading.  The whole block
    // is built at a realisation's first timestep; every timestep compares the
    // fields that can move and hands over a change.
    const double seas = P.DoSeasonality ? P.Seasonality[((int)t) % DAYS_PER_YEAR] : 1.0;
    const int dc_gate = P.FalsePositiveRate > 0 ? State.cumDC : 0;   // RecordSample's, read by DoFalseCase
    if (g_step_in_run == 0) {   // a realisation's first timestep: the whole block
        cs_params cur = params_from_reference();
        cur.kernel_delta = g_params.kernel_delta;
        cur.Seasonality = seas;
        if (std::memcmp(&cur, &g_params, sizeof(cs_params)) != 0) {
            g_params = cur;
            check(cs_gpu_set_params(g_ctx, &g_params), "cs_gpu_set_params");
        }
    } else if (seas != g_params.Seasonality || P.ControlPropCasesId != g_params.ControlPropCasesId ||
               P.CFR_Critical_Scale_Current != g_params.CFR_Critical_Scale_Current ||
               P.CFR_SARI_Scale_Current != g_params.CFR_SARI_Scale_Current ||
               P.CFR_ILI_Scale_Current != g_params.CFR_ILI_Scale_Current || dc_gate != g_params.cumDC_at_sample) {
        // the fields the run loop moves; nothing else in the block changes during a run
        g_params.Seasonality = seas;
        g_params.ControlPropCasesId = P.ControlPropCasesId;
        g_params.CFR_Critical_Scale_Current = P.CFR_Critical_Scale_Current;
        g_params.CFR_SARI_Scale_Current = P.CFR_SARI_Scale_Current;
        g_params.CFR_ILI_Scale_Current = P.CFR_ILI_Scale_Current;
        g_params.cumDC_at_sample = dc_gate;
        check(cs_gpu_set_params(g_ctx, &g_params), "cs_gpu_set_params");
    }
    // case isolation and household quarantine windows of each admin unit
    // (RecordSample, src/CovidSim.cpp:3598-3609; read by DoDetectedCase)
    const int na = P.NumAdunits > 0 ? P.NumAdunits : 1;
    bool iv = !g_iv_sent || g_ci_dur != P.CaseIsolationPolicyDuration || g_hq_dur != P.HQuarantinePolicyDuration;
    g_ci_start.resize(na);
    g_hq_start.resize(na);
    for (int a = 0; a < na; a++) {
        const double ci = P.NumAdunits > 0 ? AdUnits[a].CaseIsolationTimeStart : 1e10;
        const double hq = P.NumAdunits > 0 ? AdUnits[a].HQuarantineTimeStart : 1e10;
        iv |= ci != g_ci_start[a] || hq != g_hq_start[a];
        g_ci_start[a] = ci;
        g_hq_start[a] = hq;
    }
    if (iv) {
        cs_interventions w;
        std::memset(&w, 0, sizeof(w));
        w.CaseIsolationPolicyDuration = g_ci_dur = P.CaseIsolationPolicyDuration;
        w.HQuarantinePolicyDuration = g_hq_dur = P.HQuarantinePolicyDuration;
        w.CaseIsolationTimeStart = g_ci_start[0];
        w.HQuarantineTimeStart = g_hq_start[0];
        w.adunit_CaseIsolationTimeStart = g_ci_start.data();
        w.adunit_HQuarantineTimeStart = g_hq_start.data();
        check(cs_gpu_set_interventions(g_ctx, &w), "cs_gpu_set_interventions");
        g_iv_sent = true;
    }
}

// The global trigger value as TreatSweep forms it (src/Sweep.cpp:1342-1347).
int global_trig_value()
{
    if (!P.DoGlobalTriggers) return 0;
    if (P.DoPerCapitaTriggers) return (int)floor(((double)State.trigDetectedCases) * P.GlobalIncThreshPop / ((double)P.PopSize));
    return State.trigDetectedCases;
}

// What TreatSweep(t) changed, handed to the device right after it ran.  Microcell
// status changes only where TreatSweep's own conditions allow (src/Sweep.cpp:
// 1839-1912): social distancing switches on when the trigger reached its threshold
// and untreated microcells remain, and off when a treated microcell's end time has
// come or the trigger fell below the stop threshold; movement restrictions only
// from their start time on.  The microcells are scanned only then: a scan touches
// every populated microcell's record (2.7 M of them at 10 M people on 240 x 240
// cells).  Admin-unit triggers are compared per unit, so with them every step from
// the start time on is scanned.
void mirror_treat_sweep(double t, int gt)
{
    const unsigned int ts = (unsigned short int)(P.TimeStepsPerDay * t);
    bool sd = false;
    if (t >= P.SocDistTimeStart) {
        if (!P.DoGlobalTriggers) sd = true;
        else sd = (g_sd_untreated > 0 && gt >= P.SocDistCellIncThresh) ||
                  (g_sd_treated > 0 && (gt < P.SocDistCellIncStopThresh || ts >= g_sd_min_end));
    }
    const bool mr = t >= P.MoveRestrTimeStart;
    if (sd || mr) {
        // the scan over every populated microcell runs on the host's OpenMP threads;
        // the changed ones are then listed in microcell order.  Each thread scans one
        // contiguous share of the populated microcells and keeps its changes in its
        // own list; after a prefix over the threads the lists are copied into the
        // change list, so it stays in microcell order and each microcell is read once.
        const int npm = P.NumPopulatedMicrocells;
        static std::vector<int32_t> ms;
        static std::vector<uint8_t> vs, vm;
        static std::vector<long long> thread_n;
        static std::vector<std::vector<int32_t>> local;
        ms.resize(npm); vs.resize(npm); vm.resize(npm);
        long long untreated = 0, treated = 0, nchg = 0;
        unsigned int min_end = 0xFFFFFFFFu;
#pragma omp parallel reduction(+ : untreated, treated) reduction(min : min_end)
        {
            const int T = omp_get_num_threads(), k = omp_get_thread_num();
#pragma omp single
            {
                thread_n.assign((size_t)T + 1, 0);
                local.resize((size_t)T);
            }
            std::vector<int32_t>& mine = local[k];
            mine.clear();
            const int i0 = (int)((long long)npm * k / T), i1 = (int)((long long)npm * (k + 1) / T);
            for (int i = i0; i < i1; i++) {
                const int m = (int)(McellLookup[i] - Mcells);
                const uint8_t a = (uint8_t)Mcells[m].socdist, b = (uint8_t)Mcells[m].moverest;
                if (Mcells[m].socdist == TreatStat::Untreated) untreated++;
                else if (Mcells[m].socdist == TreatStat::Treated) {
                    treated++;
                    if (Mcells[m].socdist_end_time < min_end) min_end = Mcells[m].socdist_end_time;
                }
                if (a != g_sd[m] || b != g_mr[m]) {
                    g_sd[m] = a;
                    g_mr[m] = b;
                    mine.push_back(m);
                }
            }
            thread_n[k + 1] = (long long)mine.size();
#pragma omp barrier
#pragma omp single
            for (int j = 0; j < T; j++) thread_n[j + 1] += thread_n[j];
            long long o = thread_n[k];
            for (const int32_t m : mine) {
                ms[o] = m;
                vs[o] = g_sd[m];
                vm[o] = g_mr[m];
                o++;
            }
#pragma omp single
            nchg = thread_n[T];
        }
        ms.resize(nchg); vs.resize(nchg); vm.resize(nchg);
        if (!g_timing.empty()) g_timing.back().scans++;
        g_sd_untreated = untreated;
        g_sd_treated = treated;
        g_sd_min_end = min_end;
        if (!ms.empty())
            check(cs_gpu_set_mcell_status(g_ctx, ms.data(), vs.data(), vm.data(), (int)ms.size()), "cs_gpu_set_mcell_status");
    }
    // the closures and openings TreatSweep made
    if (!g_events.empty()) {
        check(cs_gpu_place_events(g_ctx, g_events.data(), (int)g_events.size()), "cs_gpu_place_events");
        g_events.clear();
    }
}

// Holidays (the start of IncubRecoverySweep, src/Sweep.cpp:889-918): at the timestep
// a holiday starts in, each place of a type the holiday affects is chosen (all of
// them when HolidayEffect is 0, else with probability 1 - HolidayEffect), its window
// on the host widens as the reference's loop widens it, and the device receives the
// same choice as CS_PLACE_EV_HOLIDAY events, which widen the members' absences.  The
// events go to the device before the timestep's sweeps: the holiday starts at
// HolidayStart = (int)(ht * TimeStepsPerDay), which is past the timestep when the
// holiday begins on a timestep boundary (ht in (t, t + dt]), so the timestep's
// InfectSweep sees no difference.
std::vector<cs_place_event> g_holiday;

void holidays(double t)
{
    if (!P.DoPlaces || P.NumHolidays <= 0) return;
    g_holiday.clear();
    const unsigned short int ts = (unsigned short int)(P.TimeStepsPerDay * t);
    for (int h = 0; h < P.NumHolidays; h++) {
        const double ht = P.HolidayStartTime[h] + P.HolidaysStartDay_SimTime;
        if (!((t + P.ModelTimeStep >= ht) && (t < ht))) continue;
        const int hs = (int)(ht * P.TimeStepsPerDay), he = (int)((ht + P.HolidayDuration[h]) * P.TimeStepsPerDay);
        for (int pt = 0; pt < P.NumPlaceTypes; pt++) {
            if (!(P.HolidayEffect[pt] < 1)) continue;
            for (int i = 0; i < P.Nplace[pt]; i++) {
                if (!((P.HolidayEffect[pt] == 0) || (ranf_mt(0) >= P.HolidayEffect[pt]))) continue;
                Place& pl = Places[pt][i];
                if (pl.close_start_time > hs) pl.close_start_time = (unsigned short)hs;
                if (pl.close_end_time < he) pl.close_end_time = (unsigned short)he;
                cs_place_event e;
                std::memset(&e, 0, sizeof(e));
                e.place = i;
                e.place_type = (uint8_t)pt;
                e.kind = CS_PLACE_EV_HOLIDAY;
                e.ts = ts;
                e.win_start = (uint16_t)hs;
                e.win_stop = (uint16_t)he;
                g_holiday.push_back(e);
            }
        }
    }
    if (!g_holiday.empty())
        check(cs_gpu_place_events(g_ctx, g_holiday.data(), (int)g_holiday.size()), "cs_gpu_place_events (holidays)");
}

void report_timing()
{
    for (const RunTiming& r : g_timing)
        std::fprintf(stderr, "\nSWEEPTIMING run=%d pop=%d threads=%d steps=%ld infect_s=%.6f incub_s=%.6f upload_s=%.6f copyback_s=%.6f"
                             " wait_s=%.6f scatter_s=%.6f handover_s=%.6f mcell_scans=%ld upload_device_s=%.6f cell_bytes=%d loop_s=%.6f\n",
                     r.run, P.PopSize, P.NumThreads, r.steps, r.infect, r.incub, r.upload, r.copyback, r.wait, r.scatter,
                     r.handover, r.scans, r.upload_device, g_use16 ? 2 : 4, r.loop_end - r.loop_start);
}

}  // namespace

void InfectSweep(double t, int run)
{
    if (!g_ctx) {
        create_context();
        std::atexit(report_timing);
    }
    const double t0 = omp_get_wtime();
    double upload = 0.0;
    if (run != g_run) {
        upload_run_state(run);
        g_run = run;
        upload = omp_get_wtime() - t0;
    } else if (g_update_probs) {
        check(cs_gpu_update_probs(g_ctx, 0), "cs_gpu_update_probs");  // the host ran UpdateProbs(0)
        g_update_probs = false;
    }
    mirror_host_interventions(t);
    holidays(t);
    // RunModel calls IncubRecoverySweep(t) right after this call (src/CovidSim.cpp:
    // 1488-1490), so the whole timestep runs here as one replay of its graph
    check(cs_gpu_step(g_ctx, t, run), "cs_gpu_step");
    // a timestep whose results RecordSample reads: the packed copy back is queued
    // behind it now, so it follows the timestep on the device without a round trip
    g_sample_queued = false;
    if (g_use16 && (P.LimitNumInfections || (g_step_in_run + 1) % P.NumModelTimeStepsPerOutputTimeStep == 0)) {
        check(cs_gpu_sample_packed_begin(g_ctx, g_packed.data(), g_packed.size()), "cs_gpu_sample_packed_begin");
        g_sample_queued = true;
    }
    if (g_timing.empty() || g_timing.back().run != run) {
        g_timing.push_back(RunTiming());
        g_timing.back().run = run;
        g_timing.back().loop_start = t0;
    }
    g_timing.back().infect += omp_get_wtime() - t0;
    g_timing.back().upload += upload;
    if (upload > 0.0) g_timing.back().upload_device += g_upload_device;
    g_timing.back().steps++;
}

// TreatSweep (src/Sweep.cpp:1324-2004) runs on the host as the reference's own
// function; the drop-in's Sweep.cpp has it renamed to ref_TreatSweep.
int ref_TreatSweep(double t);
int TreatSweep(double t)
{
    double t0 = omp_get_wtime();
    const int gt = global_trig_value();   // the value the reference's TreatSweep will use
    double spent = omp_get_wtime() - t0;
    const int r = ref_TreatSweep(t);
    if (g_ctx && g_run >= 0) {
        t0 = omp_get_wtime();
        mirror_treat_sweep(t, gt);
        // the hand-over is the drop-in's own work: timed with its sweeps
        spent += omp_get_wtime() - t0;
        if (!g_timing.empty()) { g_timing.back().infect += spent; g_timing.back().handover += spent; }
        // RunModel's UpdateProbs test runs next in this timestep on the State.S the
        // last RecordSample set, which no call in between changes
        const double prop = ((double)(State.S)) / ((double)P.PopSize);
        if ((g_prev_prop - prop) > 0.2) {
            g_prev_prop = prop;
            g_update_probs = true;
        }
    }
    return r;
}
// TreatSweep's place closures (src/Sweep.cpp:1686, 1733): the drop-in's Sweep.cpp
// calls these in place of DoPlaceClose / DoPlaceOpen.  Each runs the reference's own
// function on the host's Places, so the host's place state and its outputs stay the
// reference's, and records the outcome for the device.  Members' absences are the
// device's to apply (the host's person records are not current between steps).
// Called from TreatSweep's OpenMP threads, one microcell's places per thread.
void cs_shim_DoPlaceClose(int i, int j, unsigned short int TimeStepNow, int tn, int DoAnyway)
{
    if (!DoAnyway) ERR_CRITICAL("GPU sweep: place closure by case counts is not supported\n");
    Place& pl = Places[i][j];
    const unsigned short int ce0 = pl.close_end_time;
    DoPlaceClose(i, j, TimeStepNow, tn, DoAnyway);
    if (pl.close_end_time == ce0) return;   // DoPlaceClose changes close_end_time whenever it acts
    cs_place_event e;
    std::memset(&e, 0, sizeof(e));
    e.place = j;
    e.place_type = (uint8_t)i;
    e.kind = CS_PLACE_EV_CLOSE;
    e.members = pl.ProbClose >= P.Efficacies[PlaceClosure][i];   // HasPlaceClosed (src/Update.cpp:1178)
    e.ts = TimeStepNow;
    e.close_start = pl.close_start_time;
    e.close_end = pl.close_end_time;
    e.win_start = (uint16_t)(TimeStepNow + ((unsigned short int)(P.TimeStepsPerDay * P.PlaceCloseDelayMean)));
    e.win_stop = (uint16_t)(TimeStepNow + ((unsigned short int)(P.TimeStepsPerDay * (P.PlaceCloseDelayMean + P.PlaceCloseDuration))));
#pragma omp critical(cs_shim_place_events)
    g_events.push_back(e);
}

void cs_shim_DoPlaceOpen(int i, int j, unsigned short int TimeStepNow)
{
    const unsigned short int ce0 = Places[i][j].close_end_time;
    DoPlaceOpen(i, j, TimeStepNow);
    if (!(TimeStepNow < ce0)) return;
    cs_place_event e;
    std::memset(&e, 0, sizeof(e));
    e.place = j;
    e.place_type = (uint8_t)i;
    e.kind = CS_PLACE_EV_OPEN;
    e.ts = TimeStepNow;
#pragma omp critical(cs_shim_place_events)
    g_events.push_back(e);
}


// The timestep's device work runs on while the host goes on to TreatSweep: the host
// reads nothing the sweeps change until RecordSample, at the start of the next
// output step, so the wait for the device comes at the last timestep of each output
// step (and at every step of a run with a limit on infections, whose test reads
// State.cumI each step).  What the host hands the device in between (parameters,
// place events, microcell status) is copied from pageable memory in stream order,
// behind the work in flight.  RunModel stops calling the sweeps mid-output-step only
// once State.L + State.I was 0 at the last RecordSample, after which no sweep changes
// anything.
void IncubRecoverySweep(double t)
{
    const double t0 = omp_get_wtime();
    (void)t;
    g_step_in_run++;
    const bool output_step = g_step_in_run % P.NumModelTimeStepsPerOutputTimeStep == 0;
    const bool read_back = P.LimitNumInfections || output_step;
    if (read_back) {
        check(cs_gpu_sync(g_ctx), "cs_gpu_sync");   // the output step's device work, all of it timed
        if (!g_timing.empty()) g_timing.back().wait += omp_get_wtime() - t0;
        const double t1 = omp_get_wtime();
        sync_back();
        if (output_step) dump_block();
        if (!g_timing.empty()) g_timing.back().copyback += omp_get_wtime() - t1;
    }
    if (!g_timing.empty()) {
        g_timing.back().incub += omp_get_wtime() - t0;
        g_timing.back().loop_end = omp_get_wtime();
    }
}
