/*
 * covidsim_b200.h -- C ABI of the B200 (sm_100a) per-timestep sweep of CovidSim.
 *
 * The reference model runs one timestep as (src/CovidSim.cpp:1488-1490):
 *     InfectSweep(t, run);            // src/Sweep.cpp:283-881
 *     IncubRecoverySweep(t);          // src/Sweep.cpp:883-979
 * with UpdateProbs(0) (src/CovidSim.cpp:2752-2802) re-normalising the spatial
 * sampler whenever the susceptible fraction has fallen by 0.2 (:1515-1521).
 * This header declares drop-in replacements for those three calls that run on one
 * GPU, plus the set-up, state transfer and counter entry points a host needs around
 * them.  Everything here is plain C: pointers, sizes and fixed-width integers.
 *
 * Ownership: the host owns every array passed in; the context copies what it needs
 * to device memory during the call and keeps no host pointer afterwards.  The
 * context owns the device copies and is authoritative for dynamic per-person state
 * between cs_gpu_begin_run / cs_gpu_upload_state and cs_gpu_download_state.
 *
 * Errors: every function returning int returns CS_OK (0) or a negative CS_E* code;
 * cs_gpu_last_error() then holds a one-line message.  The reference aborts through
 * ERR_CRITICAL (src/Error.cpp:13); a host that wants that behaviour maps a non-zero
 * status to its own fatal error.  No device code traps: bounded loops count their
 * give-ups in cs_counters.err_* and the next call reports them.
 *
 * Threading: one host thread per context; calls on a context are serialised on
 * the context's own CUDA stream and are not re-entrant.
 */
#ifndef COVIDSIM_B200_H
#define COVIDSIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_ABI_VERSION 4            /* 2: per admin unit windows in cs_interventions, cs_run_policy;
                                       3: PlaceClosePropAttending, cs_gpu_place_events,
                                          cs_gpu_set_mcell_status;
                                       4: population set-up (cs_gpu_setup_*) */

/* Sizes fixed by the reference (src/Constants.h, src/Country.h). */
#define CS_MAX_PLACE_TYPES 5        /* MAX_NUM_PLACE_TYPES   (Country.h:15)   */
#define CS_NUM_AGE_GROUPS 17        /* NUM_AGE_GROUPS        (Constants.h:77) */
#define CS_AGE_GROUP_WIDTH 5        /* AGE_GROUP_WIDTH       (Constants.h:78) */
#define CS_CDF_RES 20               /* CDF_RES               (Constants.h:75) */
#define CS_MAX_INFECTIOUS_STEPS 2550 /* MAX_INFECTIOUS_STEPS (Constants.h:86) */
#define CS_INFECT_TYPE_MASK 16      /* INFECT_TYPE_MASK      (Constants.h:80) */
#define CS_MAX_HOUSEHOLD_SIZE 10    /* MAX_HOUSEHOLD_SIZE    (Country.h:5)    */
#define CS_NUM_SETTINGS (CS_MAX_PLACE_TYPES + 2) /* place types, House, Spatial (Constants.h:117-118) */
#define CS_NUM_NPI 6                /* CaseIsolation..DigContactTracing (Constants.h:121-126) */
#define CS_SETTING_HOUSE CS_MAX_PLACE_TYPES
#define CS_SETTING_SPATIAL (CS_MAX_PLACE_TYPES + 1)
#define CS_NPI_CASE_ISOLATION 0
#define CS_NPI_HOME_QUARANTINE 1
#define CS_NPI_PLACE_CLOSURE 2
#define CS_NPI_SOCIAL_DISTANCING 3
#define CS_NPI_ENHANCED_SOCIAL_DISTANCING 4
#define CS_NPI_DIG_CONTACT_TRACING 5
#define CS_MAX_ADUNITS 128          /* counters kept per admin unit on the device */
#define CS_USHRT_MAX_M1 65534u      /* USHRT_MAX - 1: the reference's "never" time */

/* Status codes. */
#define CS_OK 0
#define CS_E_ARG (-1)          /* bad argument or inconsistent sizes            */
#define CS_E_CUDA (-2)         /* a CUDA runtime call failed                     */
#define CS_E_UNSUPPORTED (-3)  /* parameter combination outside this sweep       */
#define CS_E_OVERFLOW (-4)     /* a device queue or bounded loop gave up         */
#define CS_E_STATE (-5)        /* call order violated (e.g. sweep before run)    */
#define CS_E_RANGE (-6)        /* kernel distance beyond the lookup table        */

/* Infection states: numeric values of InfStat (src/InfStat.h:12-44). */
#define CS_INF_SUSCEPTIBLE 0
#define CS_INF_LATENT 1
#define CS_INF_INFECTIOUS_ALMOST_SYMPTOMATIC (-1)
#define CS_INF_INFECTIOUS_ASYMPTOMATIC_NOT_CASE 2
#define CS_INF_CASE (-2)
#define CS_INF_RECOVERED_FROM_ASYMP 3
#define CS_INF_RECOVERED_FROM_SYMP (-3)
#define CS_INF_IMMUNE_AT_START 4
#define CS_INF_DEAD_WAS_ASYMP 5
#define CS_INF_DEAD_WAS_SYMP (-5)

/* Severity classes: order of Severity (src/InfStat.h:47-58). */
#define CS_SEV_ASYMPTOMATIC 0
#define CS_SEV_MILD 1
#define CS_SEV_ILI 2
#define CS_SEV_SARI 3
#define CS_SEV_CRITICAL 4
#define CS_SEV_STEPDOWN 5
#define CS_SEV_DEAD 6
#define CS_SEV_RECOVERED 7

/*
 * Random streams.  Every draw comes from Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11) keyed by the run seed
 * (key = {seed & 0xffffffff, seed >> 32}) with counter
 *     {block, entity, timestep | purpose << 16, sub}
 * where entity is a person, place or cell index and sub separates several streams of
 * one entity in one step (contact number, place type).  Each block yields two
 * doubles in [0,1) from the 53 high bits of (x1:x0) and (x3:x2).  Results therefore
 * depend on (seed, step, entity, purpose) only, never on launch geometry or thread
 * count -- unlike the reference's per-thread streams (src/Rand.cpp:28-46).
 */
#define CS_RNG_HOUSEHOLD 1        /* entity infector                      */
#define CS_RNG_PLACE_GROUP 2      /* entity infector, sub place type      */
#define CS_RNG_PLACE_BETWEEN 3    /* entity infector, sub place type      */
#define CS_RNG_SPATIAL_COUNT 4    /* entity infector                      */
#define CS_RNG_SPATIAL_CONTACT 5  /* entity infector, sub contact number  */
#define CS_RNG_LATENT 6           /* entity infectee                      */
#define CS_RNG_INCUB 7            /* entity person                        */
#define CS_RNG_CASE 8             /* entity person                        */
#define CS_RNG_DETECTED 9         /* entity person                        */
#define CS_RNG_HQ 10              /* entity household                     */
#define CS_RNG_RUN_INIT 11        /* entity person, timestep 0            */
#define CS_RNG_PLACE_INIT 12      /* entity place, sub place type         */
#define CS_RNG_FALSE_POSITIVE 13  /* entity infector, sub infectee, block infection type */
#define CS_RNG_FALSE_CASE 14      /* entity person                        */
/* Population set-up (cs_gpu_setup_run); timestep field = round where noted. */
#define CS_RNG_SETUP_DENSITY 20   /* entity microcell grid index          */
#define CS_RNG_SETUP_BLOB 21      /* entity blob                          */
#define CS_RNG_SETUP_PERSON 22    /* entity draw k (64-bit integer)       */
#define CS_RNG_SETUP_HH 23        /* entity microcell grid index          */
#define CS_RNG_SETUP_HH_LOC 24    /* entity microcell grid index, sub household ordinal */
#define CS_RNG_SETUP_AGE 25       /* entity person                        */
#define CS_RNG_SETUP_ATTEND 26    /* entity person, sub 4 * place type + band */
#define CS_RNG_SETUP_PLACE_SIZE 27 /* entity place draw, sub place type   */
#define CS_RNG_SETUP_PLACE_LOC 28 /* entity place, sub place type (block 0: 64-bit person draw) */
#define CS_RNG_SETUP_CHOOSE 29    /* entity person, sub place type, timestep round */
#define CS_RNG_SETUP_ACCEPT 30    /* entity person, sub place type, timestep round */
#define CS_RNG_SETUP_SHUFFLE 31   /* entity person, sub place type (32-bit key) */

/* Static per-person flag bits (cs_population.person_flags). */
#define CS_PF_CARE_HOME_RESIDENT 0x01u
#define CS_PF_ESOCDIST_COMPLY 0x02u
#define CS_PF_KEYWORKER 0x04u

/* Dynamic per-person flag bits (cs_person_state.flags). */
#define CS_DF_TO_DIE 0x01u
#define CS_DF_DETECTED 0x02u
#define CS_DF_QUAR_COMPLY_SHIFT 2   /* 2 bits: HostsQuarantine[].comply 0/1/2 */
#define CS_DF_QUAR_COMPLY_MASK 0x0Cu

/* Microcell intervention status: TreatStat (src/Models/Microcell.h:6-17). */
#define CS_TREAT_UNTREATED 0
#define CS_TREAT_TO_BE_TREATED 1
#define CS_TREAT_TREATED 2
#define CS_TREAT_DONT_TREAT_AGAIN 3

/*
 * Inverse CDF table: the reference's InverseCdf after assign_exponent(), i.e. the
 * values exp(-x_i) that InverseCdf::choose (src/InverseCdf.cpp:60-74) interpolates.
 */
typedef struct cs_icdf {
    double v[CS_CDF_RES + 1];
} cs_icdf;

/*
 * Every scalar and table the two sweeps read from the reference's global Param P
 * (src/Param.h).  Field names follow the reference's.  Only the intervention
 * settings the sweep itself consumes are here; trigger logic stays on the host and
 * reaches the device through cs_gpu_set_interventions / cs_gpu_close_places.
 */
typedef struct cs_params {
    /* time */
    double TimeStepsPerDay;            /* P.TimeStepsPerDay                     */
    double ModelTimeStep;              /* P.ModelTimeStep                       */
    /* switches */
    int32_t DoHouseholds, DoPlaces, DoSpatial, DoSymptoms, DoSeverity, DoLatent;
    int32_t DoInfectiousnessProfile, NoInfectiousnessSDinHH, DoUTM_coords, DoPeriodicBoundaries;
    int32_t DoRealSymptWithdrawal, DoDeathCountsInS0;  /* the latter is P.DoDeath (UpdateProbs) */
    int32_t NumPlaceTypes, HotelPlaceType, CareHomePlaceType, PlaceTypeNoAirNum;
    int32_t IncludeStepDownToDeath, CaseAbsentChildAgeCutoff, DoHQretrigger, _pad0;
    /* transmission */
    double LocalBeta, HouseholdTrans, FalsePositiveRate, Seasonality;
    /* DoFalseCase counts a false case as detected only once the detected cases at the
     * last sample (State.cumDC) reached P.CaseOrDeathThresholdBeforeAlert
     * (src/Update.cpp:901); the host refreshes cumDC_at_sample at each sample */
    int32_t CaseOrDeathThresholdBeforeAlert, cumDC_at_sample;
    double HouseholdDenomLookup[CS_MAX_HOUSEHOLD_SIZE];
    double infectiousness[CS_MAX_INFECTIOUS_STEPS];     /* P.infectiousness[] */
    double PlaceTypeTrans[CS_MAX_PLACE_TYPES];
    double PlaceTypeGroupSizeParam1[CS_MAX_PLACE_TYPES];
    double PlaceTypePropBetweenGroupLinks[CS_MAX_PLACE_TYPES];
    double SymptPlaceTypeContactRate[CS_MAX_PLACE_TYPES];
    double SymptPlaceTypeWithdrawalProp[CS_MAX_PLACE_TYPES];
    double SymptSpatialContactRate;
    double RelativeSpatialContact[CS_NUM_AGE_GROUPS];
    double RelativeSpatialContactSusc[CS_NUM_AGE_GROUPS];
    double AgeSusceptibility[CS_NUM_AGE_GROUPS];
    double AgeInfectiousness[CS_NUM_AGE_GROUPS];
    double WAIFW_Matrix[CS_NUM_AGE_GROUPS][CS_NUM_AGE_GROUPS];
    double WAIFW_Matrix_SpatialOnly[CS_NUM_AGE_GROUPS][CS_NUM_AGE_GROUPS];
    double CareHomeResidentHouseholdScaling, CareHomeResidentSpatialScaling;
    double CareHomeWorkerGroupScaling, CareHomeResidentPlaceScaling, CareHomeRelProbHosp;
    double Efficacies[CS_NUM_NPI][CS_NUM_SETTINGS];    /* P.Efficacies[npi][setting] */
    double MoveRestrEffect;
    /* blanket movement restrictions (P.DoBlanketMoveRestr, src/Sweep.cpp:300-301):
     * from MoveRestrTimeStart for MoveRestrDuration days, a contact whose two ends
     * lie more than sqrt(MoveRestrRadius2) apart (dist2_raw) is scaled by
     * MoveRestrEffect, in place of the microcells' movement-restriction test */
    int32_t DoBlanketMoveRestr, _pad3;
    double MoveRestrTimeStart, MoveRestrDuration, MoveRestrRadius2;
    /* the point infection radii are measured from (P.LocationInitialInfection[0];
     * seeding moves it to the last seed's household, src/CovidSim.cpp:1358-1359) */
    double LocationInitialInfection[2];
    /* natural history */
    double LatentPeriod, InfectiousPeriod, LatentToSymptDelay;
    double SymptInfectiousness, AsymptInfectiousness, InfectiousnessSD;
    double ProportionSymptomatic[CS_NUM_AGE_GROUPS];
    cs_icdf latent_icdf, infectious_icdf;
    cs_icdf MildToRecovery_icdf, ILIToRecovery_icdf, SARIToRecovery_icdf;
    cs_icdf CriticalToCritRecov_icdf, CritRecovToRecov_icdf, ILIToSARI_icdf;
    cs_icdf SARIToCritical_icdf, ILIToDeath_icdf, SARIToDeath_icdf;
    cs_icdf StepdownToDeath_icdf, CriticalToDeath_icdf;
    double Mean_MildToRecovery[CS_NUM_AGE_GROUPS], Mean_ILIToRecovery[CS_NUM_AGE_GROUPS];
    double Mean_SARIToRecovery[CS_NUM_AGE_GROUPS], Mean_CriticalToCritRecov[CS_NUM_AGE_GROUPS];
    double Mean_CritRecovToRecov[CS_NUM_AGE_GROUPS], Mean_StepdownToDeath[CS_NUM_AGE_GROUPS];
    double Mean_ILIToSARI[CS_NUM_AGE_GROUPS], Mean_SARIToCritical[CS_NUM_AGE_GROUPS];
    double Mean_CriticalToDeath[CS_NUM_AGE_GROUPS], Mean_SARIToDeath[CS_NUM_AGE_GROUPS];
    double Mean_ILIToDeath[CS_NUM_AGE_GROUPS];
    double Prop_ILI_ByAge[CS_NUM_AGE_GROUPS], Prop_SARI_ByAge[CS_NUM_AGE_GROUPS];
    double Prop_Critical_ByAge[CS_NUM_AGE_GROUPS];
    double CFR_SARI_ByAge[CS_NUM_AGE_GROUPS], CFR_Critical_ByAge[CS_NUM_AGE_GROUPS];
    double CFR_ILI_ByAge[CS_NUM_AGE_GROUPS];
    double CFR_Critical_Scale_Current, CFR_SARI_Scale_Current, CFR_ILI_Scale_Current;
    double ControlPropCasesId;
    /* interventions consumed inside the sweep (DoCase/DoDetectedCase) */
    double CaseIsolationProp, HQuarantinePropHouseCompliant, HQuarantinePropIndivCompliant;
    double HQuarantineDelay, CaseAbsentChildPropAdultCarers;
    double PlaceClosePropAttending[CS_MAX_PLACE_TYPES]; /* DoPlaceClose's attendance filter */
    uint16_t usCaseIsolationDelay, usCaseIsolationDuration, usCaseAbsenteeismDelay;
    uint16_t usCaseAbsenteeismDuration, usHQuarantineHouseDuration, _pad1[3];
    /* geometry: degrees relative to the bounding box's bottom-left corner */
    int32_t ncw, nch;                  /* cells wide / high                    */
    double cell_width, cell_height;    /* P.in_cells_ (degrees)                */
    double width_deg, height_deg;      /* P.in_degrees_                         */
    double bbox_bottom_left_y;         /* P.SpatialBoundingBox.bottom_left().y */
    double sinx[361], cosx[361], asin2sqx[1001];  /* P.sinx/cosx/asin2sqx    */
    /* spatial kernel lookup (KernelLookup, src/Kernels.h:66-119) */
    int32_t kernel_size, kernel_expansion; /* size_, expansion_factor_          */
    double kernel_delta;               /* delta_                                */
    /* sampler blocking: cells per side of a proposal block (0 = choose) */
    int32_t block_cells, _pad2;
} cs_params;

/*
 * Static population structure.  Arrays are host pointers read during
 * cs_gpu_create only.  Index spaces follow the reference: people are numbered as
 * Hosts[] (contiguous by household, src/SetupModel.cpp:1224-1253); cells are the
 * populated cells in CellLookup order; microcells are the populated microcells.
 */
typedef struct cs_population {
    int32_t n_people, n_households, n_cells, n_mcells;
    int32_t num_place_types, n_adunits;
    int32_t n_places[CS_MAX_PLACE_TYPES];
    /* people */
    const int32_t* person_hh;          /* Person::hh                            */
    const int32_t* person_mcell;       /* index into the mcell_* arrays         */
    const uint8_t* person_age;         /* Person::age (years)                   */
    const uint8_t* person_flags;       /* CS_PF_* bits                          */
    const int32_t* person_place;       /* [num_place_types][n_people] PlaceLinks */
    const uint16_t* person_group;      /* [num_place_types][n_people] PlaceGroupLinks */
    /* households */
    const int32_t* hh_first;           /* Household::FirstPerson                */
    const uint16_t* hh_nh;             /* Household::nh                         */
    const uint16_t* hh_nhr;            /* Household::nhr                        */
    const float* hh_x;                 /* Household::loc.x                      */
    const float* hh_y;                 /* Household::loc.y                      */
    /* microcells */
    const int32_t* mcell_cell;         /* populated-cell index of the microcell */
    const int32_t* mcell_adunit;       /* Microcell::adunit                     */
    /* populated cells */
    const int32_t* cell_grid;          /* grid index x*nch+y (Cells - CellLookup[i]) */
    const int32_t* cell_start;         /* [n_cells+1] offsets into cell_members */
    const int32_t* cell_members;       /* [n_people] Cell::members, cell by cell */
    /* places of type t: CSR member lists and groups */
    const int32_t* place_mcell[CS_MAX_PLACE_TYPES];
    const float* place_x[CS_MAX_PLACE_TYPES];
    const float* place_y[CS_MAX_PLACE_TYPES];
    const int32_t* place_member_ofs[CS_MAX_PLACE_TYPES]; /* [n_places+1]             */
    const int32_t* place_members[CS_MAX_PLACE_TYPES];    /* Place::members            */
    const int32_t* place_group_ofs[CS_MAX_PLACE_TYPES];  /* [n_places+1] into groups  */
    const int32_t* group_start[CS_MAX_PLACE_TYPES];      /* Place::group_start        */
    const int32_t* group_size[CS_MAX_PLACE_TYPES];       /* Place::group_size         */
    /* spatial kernel table (double[kernel_size+1] each) */
    const double* kernel_lookup;
    const double* kernel_hi_res;
} cs_population;

/*
 * Dynamic per-person and per-cell state, for cs_gpu_upload_state /
 * cs_gpu_download_state.  All arrays have n_people (or n_cells) elements; any
 * pointer may be NULL on download to skip that field.
 */
typedef struct cs_state_view {
    int8_t* inf;                       /* InfStat value                         */
    uint8_t* severity;                 /* Severity_Current | Severity_Final<<4  */
    uint8_t* flags;                    /* CS_DF_* bits                          */
    uint16_t* infection_time;
    uint16_t* latent_time;
    uint16_t* recovery_or_death_time;
    uint16_t* SARI_time;
    uint16_t* Critical_time;
    uint16_t* Stepdown_time;
    uint16_t* absent_start_time;
    uint16_t* absent_stop_time;
    uint16_t* isolation_start_time;
    uint16_t* quar_start_time;         /* HostsQuarantine[].start_time          */
    uint16_t* detected_time;
    float* infectiousness;
    float* susc;
    float* ProbAbsent;
    float* ProbCare;
    int32_t* infector;
    int16_t* infect_type;
    int32_t* listpos;
    /* cells */
    int32_t* cell_S;
    int32_t* cell_L;
    int32_t* cell_I;
    int32_t* cell_R;
    int32_t* cell_D;
    int32_t* cell_S0;
    double* cell_tot_prob;
    int32_t* cell_slots;               /* [n_people] Cell::susceptible lists     */
} cs_state_view;

/* Intervention state the host's trigger logic hands to the sweep. */
typedef struct cs_interventions {
    /* windows in days, as AdUnits[].X TimeStart and P.X PolicyDuration */
    double CaseIsolationTimeStart, CaseIsolationPolicyDuration;
    double HQuarantineTimeStart, HQuarantinePolicyDuration;
    /* microcell status arrays (n_mcells) or NULL to leave unchanged */
    const uint8_t* mcell_socdist;      /* Microcell::socdist (TreatStat)        */
    const uint8_t* mcell_moverest;     /* Microcell::moverest (TreatStat)       */
    /* per admin unit start times (n_adunits entries, AdUnits[a].CaseIsolationTimeStart
       and .HQuarantineTimeStart), or NULL for the scalar start in every admin unit */
    const double* adunit_CaseIsolationTimeStart;
    const double* adunit_HQuarantineTimeStart;
} cs_interventions;

/* Counters: the StateT[] fields RecordSample reduces (src/Model.h:68-122). */
typedef struct cs_counters {
    int64_t S, L, I, R, D;
    int64_t cumI, cumC, cumDC, cumFC, cumR, cumD;
    int64_t cumTG, cumSI, nTG, cumHQ, cumAC, cumAA, cumACS;
    int64_t cumItype[CS_INFECT_TYPE_MASK];
    int64_t cumIa[CS_NUM_AGE_GROUPS], cumCa[CS_NUM_AGE_GROUPS], cumDa[CS_NUM_AGE_GROUPS];
    int64_t Mild, ILI, SARI, Critical, CritRecov;
    int64_t cumMild, cumILI, cumSARI, cumCritical, cumCritRecov;
    int64_t cumDeath_ILI, cumDeath_SARI, cumDeath_Critical;
    int64_t cumI_keyworker[2], cumC_keyworker[2];
    int64_t cumI_adunit[CS_MAX_ADUNITS], cumC_adunit[CS_MAX_ADUNITS], cumD_adunit[CS_MAX_ADUNITS];
    int64_t cumDC_adunit[CS_MAX_ADUNITS], cumCritical_adunit[CS_MAX_ADUNITS];
    int64_t Critical_adunit[CS_MAX_ADUNITS];
    /* infection radii from LocationInitialInfection (DoInfect, src/Update.cpp:116-127,
     * 1477): the sum of squared radii in units of 2^-32 square degrees (an integer, so
     * the sum does not depend on order) and the largest squared radius as the bits of
     * a non-negative double; a seed's own radius is 0, as the reference measures it */
    int64_t sumRad2_q, maxRad2_bits;
    /* work done by the sweeps (for the HBM roofline) */
    int64_t work_infectors, work_hh_members, work_place_candidates;
    int64_t work_spatial_contacts, work_spatial_draws, work_new_infections;
    int64_t work_transitions, work_cells_touched, work_incub_people;
    /* give-ups of bounded device loops; non-zero means the results are suspect */
    int64_t err_spatial_tries, err_queue_overflow, err_kernel_range;
} cs_counters;

typedef struct cs_gpu_ctx cs_gpu_ctx;

/* Library identification; lets a binding check it loaded the header it expects. */
int cs_abi_version(void);
size_t cs_sizeof_params(void);
size_t cs_sizeof_population(void);
size_t cs_sizeof_counters(void);
size_t cs_sizeof_interventions(void);
size_t cs_sizeof_run_policy(void);

/*
 * The architecture the library's sweep kernels were compiled for, as the CUDA
 * runtime reports it for the current device (cudaFuncAttributes.binaryVersion and
 * ptxVersion, major*10 + minor: 100 for sm_100a machine code).  Needs a device;
 * returns CS_E_CUDA without one.
 */
int cs_kernel_arch(int* binary_version, int* ptx_version);

/*
 * Build the spatial kernel lookup tables exactly as KernelLookup::setup/init
 * (src/Kernels.cpp:8-46) with norm 1: lookup[i] = K(i*delta), hi_res[i] =
 * K(i*delta/expansion), delta = longest_d2/size.  kernel_type follows
 * src/Kernels.cpp:25-40 (1 exponential ... 7 power_exp).  Host-only, no GPU.
 */
int cs_build_kernel_table(int kernel_type, double scale, double shape, double p3, double p4,
                          double longest_d2, int size, int expansion,
                          double* lookup_out, double* hi_res_out, double* delta_out);

/* Host-side evaluation of KernelLookup::num (src/Kernels.cpp:108-129). */
double cs_kernel_num(const double* lookup, const double* hi_res, int size, int expansion,
                     double delta, double r2);

/* Create a context on CUDA device `device`: uploads population and parameters. */
int cs_gpu_create(const cs_population* pop, const cs_params* params, int device, cs_gpu_ctx** out);
void cs_gpu_destroy(cs_gpu_ctx* ctx);
const char* cs_gpu_last_error(const cs_gpu_ctx* ctx);

/* Replace the parameter block (e.g. a new R0 or CFR scale) between steps. */
int cs_gpu_set_params(cs_gpu_ctx* ctx, const cs_params* params);

/*
 * Start a realisation: the per-person and per-cell resets of InitModel
 * (src/CovidSim.cpp:1006-1127, no initial immunity), UpdateProbs(0) when
 * `update_probs` is set, then DoInfect (src/Update.cpp:100-195) at t = 0 on the
 * n_seed people in `seed_people` (the host's SeedInfection choices,
 * src/CovidSim.cpp:1244-1374).  `seed` keys every random stream of the run.
 */
int cs_gpu_begin_run(cs_gpu_ctx* ctx, uint64_t seed, const int32_t* seed_people, int n_seed,
                     int update_probs);

/* Load dynamic state prepared by a host (the reference's own InitModel).  State
 * outside the view (place closures and closure thresholds, social-distancing and
 * movement flags, intervention windows) is reset as cs_gpu_begin_run resets it. */
int cs_gpu_upload_state(cs_gpu_ctx* ctx, uint64_t seed, const cs_state_view* state);
/* The per-person arrays of the next cs_gpu_upload_state, sent ahead in slices that
 * follow one another from person 0: people [first, first + n) of every per-person
 * array of `state` are queued for copying and the call returns at once, so a host
 * can fill the next slice while this one crosses (page-locked arrays, from
 * cs_host_alloc, copy without a staging pass).  The slices' memory must stay as it
 * is until that cs_gpu_upload_state returns; it sends the people not sent yet.
 * A slice out of order is CS_E_ARG. */
int cs_gpu_upload_people(cs_gpu_ctx* ctx, const cs_state_view* state, int64_t first, int64_t n);
int cs_gpu_download_state(cs_gpu_ctx* ctx, const cs_state_view* state);

/* Infect people chosen by the host at time t (importation, SeedInfection). */
int cs_gpu_seed_infections(cs_gpu_ctx* ctx, double t, const int32_t* people, int n);

/* Drop-in for InfectSweep(t, run)       (src/Sweep.cpp:283-881).  */
int cs_gpu_infect_sweep(cs_gpu_ctx* ctx, double t, int run);
/* Drop-in for IncubRecoverySweep(t)     (src/Sweep.cpp:883-979), holidays excluded. */
int cs_gpu_incub_recovery_sweep(cs_gpu_ctx* ctx, double t);
/* Drop-in for UpdateProbs(do_place)     (src/CovidSim.cpp:2752-2802). */
int cs_gpu_update_probs(cs_gpu_ctx* ctx, int do_place);
/* No counterpart in the reference.  The same computation as cs_gpu_update_probs,
 * bit for bit, for callers that must not allocate device memory at that point (a
 * process whose device memory is reserved by another allocator's pool; a caller
 * that must not let a free synchronise the device under other streams).  Its
 * scratch is one fixed array inside the library, 2 x 4 B x CS_STATIC_MAX_GRID_CELLS
 * + CS_STATIC_MAX_GRID_ROWS bytes (4.0 MiB), per device; grids with more cells or
 * rows are rejected with CS_E_RANGE.  The context's device must be current
 * (CS_E_STATE otherwise).  Each call looks up the array's device address in the
 * current CUDA context (a lookup, no allocation); the first call in a context also
 * loads the library's device code there, so make it before any stream capture.  All calls
 * on one device share that array: calls that overlap in time, from two contexts
 * or two streams, race on it and must be serialised by the caller. */
#define CS_STATIC_MAX_GRID_CELLS 524288
#define CS_STATIC_MAX_GRID_ROWS 4096
int cs_gpu_update_probs_static(cs_gpu_ctx* ctx, int do_place);
/* One full model timestep: the two sweeps back to back.  The first call captures
 * the timestep's kernels as a CUDA graph and later calls replay it (unless
 * cs_gpu_use_graphs(ctx, 0) or per-kernel profiling is on); results are the same
 * either way. */
int cs_gpu_step(cs_gpu_ctx* ctx, double t, int run);
int cs_gpu_use_graphs(cs_gpu_ctx* ctx, int enable);

/* Blocks of the grid-stride kernels (default 8 per SM).  Results do not depend
 * on it: every list the kernels fill is read order-independently.  A captured
 * step graph is dropped and captured again. */
int cs_gpu_set_grid(cs_gpu_ctx* ctx, int blocks);
int cs_gpu_grid(const cs_gpu_ctx* ctx);
/* Lanes that test one spatial contact's candidate draws together: 2, 4, 8
 * (default) or 16.  Also a launch-shape choice: results do not depend on it. */
int cs_gpu_set_spatial_lanes(cs_gpu_ctx* ctx, int lanes);

/* ---- Realisations stepped together.  No counterpart in the reference, which
 * runs realisations one after another (src/CovidSim.cpp:371-399).
 *
 * cs_gpu_create_replica: a context for another realisation of `base`'s population.
 * It shares base's static device arrays (households, place memberships, cell
 * lists, kernel tables, proposal-block layout, UpdateProbs rows) and allocates
 * only dynamic state; the shared arrays live until the last sharing context is
 * destroyed.  Its parameters start as base's; cs_gpu_set_params may change them
 * except the geometry.
 *
 * cs_gpu_batch: n member contexts (replicas, or contexts of other populations,
 * on one device) advanced by one CUDA graph per timestep in which each of the
 * step's kernels is launched once for all members (one grid row per member).
 * While the batch exists, members' own calls run on the batch's stream, ordered
 * with the batched steps.  Destroy the batch before its members. */
int cs_gpu_create_replica(const cs_gpu_ctx* base, cs_gpu_ctx** out);

typedef struct cs_gpu_batch cs_gpu_batch;
int cs_gpu_batch_create(cs_gpu_ctx* const* members, int n, cs_gpu_batch** out);
/* One timestep (InfectSweep + IncubRecoverySweep) of every member at time t. */
int cs_gpu_batch_step(cs_gpu_batch* batch, double t, int run);
/* cs_gpu_set_grid for every member (members must share one launch shape). */
int cs_gpu_batch_set_grid(cs_gpu_batch* batch, int blocks);
/* Spatial lanes of the batched launches (2, 4, 8 or 16). */
int cs_gpu_batch_set_spatial_lanes(cs_gpu_batch* batch, int lanes);
int cs_gpu_batch_sync(cs_gpu_batch* batch);
void* cs_gpu_batch_stream(cs_gpu_batch* batch);
const char* cs_gpu_batch_last_error(const cs_gpu_batch* batch);
void cs_gpu_batch_destroy(cs_gpu_batch* batch);

/* ---- Scenario surrogate.  No counterpart in the reference, which has no learned
 * model.  A network mapping 8 scenario parameters (scaled to [0, 1]) to 365
 * days x 4 daily outputs, trained on the simulator's own trajectories and used
 * to screen scenario sweeps; the simulator re-runs what it ranks highly.
 *   x [n, 8] -> 4 x (Linear 512 + ReLU) -> Linear 256 + ReLU -> Linear 2944 + ReLU
 *   -> [n, 46, 64] -> 3 x (nearest upsample x2, Conv1d k=5 pad 2): 64 -> 64 -> 32 -> 4,
 *      ReLU after the first two -> first 365 time points -> y [n, 365, 4]
 * Matrix products run on the tensor cores in BF16 with FP32 accumulation; master
 * weights, gradients and Adam moments are FP32.  Parameters travel as one flat
 * FP32 array: per layer its weight [out, in] (a convolution's [out, tap * in + c])
 * then its bias [out], layers in the order above. */
typedef struct cs_sur cs_sur;
size_t cs_sur_num_params(void);
int cs_sur_create(int max_batch, int device, cs_sur** out);
void cs_sur_destroy(cs_sur* sur);
const char* cs_sur_last_error(const cs_sur* sur);
/* Set the FP32 weights (and reset the Adam moments); read them back. */
int cs_sur_set_params(cs_sur* sur, const float* flat);
int cs_sur_get_params(cs_sur* sur, float* flat);
/* y [n, 365, 4] for x [n, 8]; any n (processed in batches of max_batch). */
int cs_sur_forward(cs_sur* sur, const float* x, int n, float* y);
/* Mean squared error against target [n, 365, 4] and, when grad is not NULL, its
 * gradient in the flat layout; n <= max_batch. */
int cs_sur_loss_grad(cs_sur* sur, const float* x, const float* target, int n, float* loss, float* grad);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8; weight_decay applied to the
 * weights directly, as AdamW) on a batch; loss may be NULL. */
int cs_sur_train_step(cs_sur* sur, const float* x, const float* target, int n, float lr, float weight_decay,
                      float* loss);
/* Matrix products on tcgen05 (0, the default: tensor memory accumulators, one
 * thread issuing the MMAs) or on mma.sync.m16n8k16 (1).  Both accumulate in FP32
 * from the same BF16 operands; only the summation order differs. */
int cs_sur_set_gemm(cs_sur* sur, int impl);

int cs_gpu_set_interventions(cs_gpu_ctx* ctx, const cs_interventions* iv);
/* DoPlaceClose with DoAnyway = 1 (src/Update.cpp:1095-1240, as TreatSweep calls it
 * at src/Sweep.cpp:1730-1733) for every place of type t in the listed microcells
 * (all when mcells == NULL), closing [start, stop) in timesteps: a place closes if
 * its ProbClose passes Efficacies[PlaceClosure][t]; then each member attending
 * (PlaceClosePropAttending) is made absent over [start, stop) and, for a child at
 * home with no adult there, the household's first living adult too (the host
 * closure queue, applied as UpdateHostClosure does, src/Update.cpp:1243-1258).
 * Members' states are evaluated at timestep `start`. */
int cs_gpu_close_places(cs_gpu_ctx* ctx, int place_type, const int32_t* mcells, int n_mcells,
                        uint16_t start, uint16_t stop);

/*
 * Place closures decided by a host's own TreatSweep.  A host that keeps the
 * reference's TreatSweep (src/Sweep.cpp:1324-2004) records each call it makes of
 * DoPlaceClose (DoAnyway = 1) and DoPlaceOpen (src/Update.cpp:1095-1240, 1260-1294)
 * and hands the outcomes over before the next sweep.  For a close the context sets
 * the place's window to the host's result (close_start, close_end) and, when the
 * place closed (HasPlaceClosed), runs DoPlaceClose's member loop over [win_start,
 * win_stop) at timestep ts, as cs_gpu_close_places does.  For an open it runs
 * DoPlaceOpen at ts on its own copy of the place (which equals the host's when
 * every close was handed over).  Opens are applied before closes, and each kind
 * place type by place type; the carers' absences follow the last close.  Hand
 * over the events of one host timestep per call.
 */
#define CS_PLACE_EV_CLOSE 1
#define CS_PLACE_EV_OPEN 2
/* A holiday closure (IncubRecoverySweep, src/Sweep.cpp:889-918): the place's window
 * widens to include [win_start, win_stop) and so does every member's absence,
 * whatever their state.  Applied after the call's opens and closes. */
#define CS_PLACE_EV_HOLIDAY 3
typedef struct cs_place_event {
    int32_t place;                     /* index within its type (Places[place_type][place]) */
    uint8_t place_type;
    uint8_t kind;                      /* CS_PLACE_EV_CLOSE, _OPEN or _HOLIDAY */
    uint8_t members;                   /* close: 1 when the place closed (its members' loop runs) */
    uint8_t _pad0;
    uint16_t ts;                       /* TimeStepNow of the host's call */
    uint16_t close_start, close_end;   /* close: the place's window after the host's call */
    uint16_t win_start, win_stop;      /* close: t_start_place_close, t_stop_place_close */
    uint16_t _pad1;
} cs_place_event;
int cs_gpu_place_events(cs_gpu_ctx* ctx, const cs_place_event* events, int n);

/* Microcell status a host's TreatSweep set (Microcell::socdist and ::moverest,
 * TreatStat values) for the n listed microcells; either array may be NULL to leave
 * that status unchanged.  The sparse form of cs_interventions' full arrays. */
int cs_gpu_set_mcell_status(cs_gpu_ctx* ctx, const int32_t* mcells, const uint8_t* socdist,
                            const uint8_t* moverest, int n);

/* Copy the device counter block (cumulative since the run began). */
int cs_gpu_get_counters(cs_gpu_ctx* ctx, cs_counters* out);

/* What the run loop between timesteps does (the host side of RunModel,
 * src/CovidSim.cpp:1420-1527): the UpdateProbs test on the susceptible fraction,
 * and a global critical-care trigger (src/CovidSim.cpp:3150-3159, global
 * thresholds) that switches interventions on for `duration` days. */
typedef struct cs_run_policy {
    int32_t icu_trigger;            /* 1: the trigger below is active */
    int32_t icu_threshold;          /* critical-care admissions over icu_window days that fire it */
    int32_t icu_window;             /* days */
    int32_t case_isolation;         /* 1: case isolation switches with the trigger */
    int32_t household_quarantine;   /* 1: household quarantine switches with the trigger */
    int32_t social_distancing;      /* 1: every microcell's social distancing switches with it */
    uint32_t close_place_types;     /* bit t set: places of type t close when it fires */
    int32_t probs_every_step;       /* 1: test the susceptible fraction after every timestep,
                                       as the reference does; 0: at the end of each day */
    int32_t per_adunit;             /* 1: one trigger per admin unit (the first CS_MAX_ADUNITS;
                                       DoAdminTriggers, src/Sweep.cpp:1478-1482) on its own
                                       admissions, firing when they exceed icu_threshold and
                                       switching its case isolation, household quarantine,
                                       microcells and places only */
    double duration;                /* days the interventions stay on */
} cs_run_policy;

/* A whole realisation on the device: `days` days of timesteps from t = 0 (after
 * cs_gpu_begin_run or cs_gpu_upload_state), with the run loop's logic between
 * timesteps evaluated by kernels rather than the host, so no host round trip
 * happens until the run ends.  daily[d] (days entries, may be NULL) receives the
 * counters at the end of day d, as cs_gpu_get_counters would return them there.
 * policy NULL: no trigger, UpdateProbs tested at day ends.  Gives the same state
 * and counters as stepping with cs_gpu_step and applying the same logic on the
 * host (cs_gpu_get_counters, cs_gpu_update_probs(ctx, 0), cs_gpu_set_interventions,
 * cs_gpu_close_places). */
int cs_gpu_run(cs_gpu_ctx* ctx, int days, const cs_run_policy* policy, cs_counters* daily);
/* cs_gpu_run for every member of a batch at once, one graph per day: policies[k]
 * (n entries, or NULL for none) is member k's; daily (n * days entries, may be
 * NULL) receives member k's day d at daily[k * days + d].  Members need the same
 * whole number of timesteps per day. */
int cs_gpu_batch_run(cs_gpu_batch* batch, int days, const cs_run_policy* policies, cs_counters* daily);
/* Per-cell S, L, I, R, D (each n_cells) for RecordSample (src/CovidSim.cpp:3044-3056). */
int cs_gpu_get_cell_counts(cs_gpu_ctx* ctx, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D);
/* cs_gpu_get_cell_counts and cs_gpu_get_counters in one call, with one wait: what
 * RecordSample (src/CovidSim.cpp:3024-3120) reads at each output step.  Any of the
 * five cell arrays may be NULL; when they lie side by side in one buffer (L = S +
 * n_cells, ..., D = R + n_cells) they arrive in a single copy. */
int cs_gpu_get_sample(cs_gpu_ctx* ctx, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D,
                      cs_counters* out);
/* cs_gpu_get_sample with the five cell arrays as 16-bit values side by side in
 * cells[5 * n_cells] (S, L, I, R, D): half the bytes to copy.  CS_E_RANGE when a cell
 * holds more than 65,535 people. */
int cs_gpu_get_sample16(cs_gpu_ctx* ctx, uint16_t* cells, cs_counters* out);
/* What RecordSample reads, in one copy into one buffer of
 * cs_gpu_sample_packed_bytes(ctx) bytes (page-locked, from cs_host_alloc, for the
 * link's rate): the counter block with S..D left 0, then S, L, I, R, D of every cell
 * as 16-bit values side by side.  CS_E_RANGE when a cell holds more than 65,535
 * people. */
size_t cs_gpu_sample_packed_bytes(const cs_gpu_ctx* ctx);
int cs_gpu_get_sample_packed(cs_gpu_ctx* ctx, void* buf, size_t bytes);
/* The same in two halves: _begin queues the packing and the copy behind the work
 * already on the context's stream (a timestep just launched) and returns at once;
 * _end waits for the stream and checks the counter block's error fields.  buf is
 * not to be read or reused between the two. */
int cs_gpu_sample_packed_begin(cs_gpu_ctx* ctx, void* buf, size_t bytes);
int cs_gpu_sample_packed_end(cs_gpu_ctx* ctx, const void* buf);
/* Page-locked host memory (NULL on failure) for a host's staging buffers: copies
 * between it and the device run at the link's full rate and never through an
 * intermediate buffer.  Free with cs_host_free. */
void* cs_host_alloc(size_t bytes);
void cs_host_free(void* p);
/* Wait for the context's stream; returns a deferred device error if any. */
int cs_gpu_sync(cs_gpu_ctx* ctx);
/* The CUDA stream the context launches on (a cudaStream_t), for host-side timing. */
void* cs_gpu_stream(cs_gpu_ctx* ctx);
/* Number of kernels launched on the context since creation. */
int64_t cs_gpu_launch_count(const cs_gpu_ctx* ctx);
/*
 * Per-kernel device time: with enable = 1 every launch is bracketed by CUDA events
 * on the context's stream; 2 also clears the totals; 0 stops recording.  Inside
 * cs_gpu_run the day graph is captured with event-record nodes around each kernel
 * and replayed as usual, so those times are kernel times between back-to-back
 * launches; elsewhere launches are eager while profiling.
 * cs_gpu_profile_entry reads entry i (name, summed milliseconds, launches) and
 * returns CS_E_RANGE past the last entry.
 */
int cs_gpu_profile(cs_gpu_ctx* ctx, int enable);
int cs_gpu_profile_entry(cs_gpu_ctx* ctx, int i, char* name, int cap, double* total_ms, int64_t* launches);

/*
 * Population set-up on the GPU: the steps of the reference's SetupModel that build
 * the hot path's inputs (src/SetupModel.cpp:1137-1290 microcell populations,
 * households and their locations; :1989-2466 AssignPeopleToPlaces), restated as
 * parallel kernels on the counter-based streams (CS_RNG_SETUP_*), so the result
 * depends on the spec and its seed only.
 *
 *  - microcell weights lognormal(0, sigma) per microcell (optionally blended with
 *    Gaussian urban blobs holding blob_share of the weight), quantised to integers;
 *    every person then draws its microcell by inverse CDF over the integer prefix
 *    sums: the counts are multinomial, the law of the reference's sequential
 *    binomial allocation (:1137-1156);
 *  - people numbered as the reference numbers Hosts[]: populated cells in grid
 *    order, within a cell its microcells x-major (:1163-1185), within a microcell
 *    household by household;
 *  - households per microcell with the reference's rule (:1224-1253): a size drawn
 *    from the cumulative distribution hh_cdf, cut at the microcell's remaining
 *    people and at CS_MAX_HOUSEHOLD_SIZE; located uniformly in the microcell
 *    (:1272-1290);
 *  - ages: a 5-year band from age_cdf, a year uniform in it, at most 84;
 *  - per place type: attendance by age band (at most one place per person, types
 *    in order), place sizes drawn until they cover the attendees (gamma(4) about
 *    mean_size, or the offset power law of :2100-2108), places located in
 *    microcells drawn in proportion to their people, capacity = ceil(size *
 *    capacity_slack);
 *  - assignment: in each of `rounds` rounds every attendee without a place looks at
 *    the `nearest` nearest places with room (rings of buckets until that many are
 *    in hand, then one ring more, as the reference's microcell spiral gathers them)
 *    and proposes to one with probability proportional to K(d) * room, the weight of
 *    the reference's searches (:2265-2290); a place with more proposals than room
 *    accepts each with probability room / proposals.  A last round ignores
 *    capacity.  K is the type's kernel table (cs_build_kernel_table layout, with
 *    the size, expansion and delta of the cs_params passed in);
 *  - member lists in a random order, groups of about group_size members.
 */
#define CS_SETUP_SIZE_GAMMA 0
#define CS_SETUP_SIZE_POWER 1
#define CS_SETUP_MAX_BLOBS 64
#define CS_SETUP_MAX_NEAREST 32
typedef struct cs_setup_place_type {
    double band_lo[3], band_hi[3], band_prop[3];   /* attendance: age in [lo, hi) years, probability */
    double mean_size;                  /* PlaceTypeMeanSize                   */
    double size_offset, size_power, size_max;      /* CS_SETUP_SIZE_POWER: P(S > s) = ((off+1)/(off+s))^power */
    double capacity_slack;             /* capacity = ceil(size * slack)       */
    int32_t size_kind;                 /* CS_SETUP_SIZE_GAMMA or CS_SETUP_SIZE_POWER */
    int32_t nearest;                   /* places the choice is among (1..CS_SETUP_MAX_NEAREST) */
    int32_t group_size;                /* PlaceTypeGroupSizeParam1            */
    int32_t _pad;
    const double* kernel_lookup;       /* K over distance^2 (cs_build_kernel_table)  */
    const double* kernel_hi_res;
} cs_setup_place_type;

typedef struct cs_setup_spec {
    int32_t n_people;
    int32_t ncw, nch, nmcl;            /* grid cells, microcells per cell side   */
    double cell_width, cell_height;    /* degrees                                */
    double sigma;                      /* lognormal sigma of microcell weights   */
    double blob_share;                 /* weight share of the blobs (0: none)    */
    int32_t n_blobs;                   /* <= CS_SETUP_MAX_BLOBS                  */
    int32_t adunit_grid;               /* admin units on an a x a grid (0: one)  */
    uint64_t seed;
    double hh_cdf[CS_MAX_HOUSEHOLD_SIZE];   /* cumulative household size distribution */
    double age_cdf[CS_NUM_AGE_GROUPS];      /* cumulative age band distribution       */
    int32_t num_place_types;
    int32_t rounds;                    /* capacity-respecting assignment rounds  */
    cs_setup_place_type pt[CS_MAX_PLACE_TYPES];
} cs_setup_spec;

/* What a set-up produced.  cs_gpu_setup_sizes fills the counts; for
 * cs_gpu_setup_download the caller points the arrays at buffers of those sizes
 * (any may be NULL to skip it).  person_place and person_group are
 * [num_place_types][n_people].  People are numbered cell by cell, so a cell's
 * members are [cell_start[c], cell_start[c+1]) in order. */
typedef struct cs_setup_out {
    int32_t n_people, n_households, n_cells, n_mcells, n_adunits, num_place_types;
    int32_t n_places[CS_MAX_PLACE_TYPES];
    int32_t n_groups[CS_MAX_PLACE_TYPES];
    int32_t n_attendees[CS_MAX_PLACE_TYPES];
    int32_t forced[CS_MAX_PLACE_TYPES];   /* attendees placed by the capacity-free last round */
    double device_ms;                  /* device time of the set-up's kernels    */
    int32_t* person_hh;
    int32_t* person_mcell;
    uint8_t* person_age;
    int32_t* person_place;
    uint16_t* person_group;
    int32_t* hh_first;
    uint16_t* hh_nh;
    float* hh_x;
    float* hh_y;
    int32_t* mcell_cell;
    int32_t* mcell_adunit;
    int64_t* mcell_grid;               /* microcell grid index mx * nch * nmcl + my */
    int32_t* cell_grid;
    int32_t* cell_start;               /* n_cells + 1 */
    int32_t* place_mcell[CS_MAX_PLACE_TYPES];
    float* place_x[CS_MAX_PLACE_TYPES];
    float* place_y[CS_MAX_PLACE_TYPES];
    int32_t* place_member_ofs[CS_MAX_PLACE_TYPES];   /* n_places + 1 */
    int32_t* place_members[CS_MAX_PLACE_TYPES];
    int32_t* place_group_ofs[CS_MAX_PLACE_TYPES];    /* n_places + 1 */
    int32_t* group_start[CS_MAX_PLACE_TYPES];
    int32_t* group_size[CS_MAX_PLACE_TYPES];
} cs_setup_out;

typedef struct cs_setup cs_setup;
/* Run the set-up on CUDA device `device`; the result stays in device memory until
 * cs_gpu_setup_destroy.  `params` supplies the geometry (DoUTM_coords, the distance
 * tables, bbox) and the kernel table's size, expansion and delta.  On failure *out
 * may still hold a handle whose last error says why (destroy it). */
size_t cs_sizeof_setup_spec(void);
size_t cs_sizeof_setup_out(void);
int cs_gpu_setup_run(const cs_setup_spec* spec, const cs_params* params, int device, cs_setup** out);
int cs_gpu_setup_sizes(cs_setup* setup, cs_setup_out* sizes);
int cs_gpu_setup_download(cs_setup* setup, const cs_setup_out* dst);
const char* cs_gpu_setup_last_error(const cs_setup* setup);
void cs_gpu_setup_destroy(cs_setup* setup);

#ifdef __cplusplus
}
#endif
#endif /* COVIDSIM_B200_H */
