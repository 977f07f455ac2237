"""Parameter blocks for the sweep (cs_params), built the way the reference derives
them from its parameter files (src/ReadParams.cpp).

`natural_history()` holds the disease-progression values of the reference's
published UK parameter set (data/param_files/preUK_R0=2.0.txt: latent period,
infectiousness profile, severity proportions, case fatality and the inverse CDFs of
every transition delay) -- configuration data, restated so that a run does not need
the reference checkout.  `build_params()` turns a configuration into the C struct:
the infectiousness profile interpolation (ReadParams.cpp:1996-2016), inverse-CDF
exponentiation (InverseCdf.cpp:15-45), household denominators
(ReadParams.cpp:574-577), efficacy table (CovidSim.cpp:825-866), the haversine
tables (ReadParams.cpp:2333-2346) and the spatial kernel lookup
(Kernels.cpp:8-46, through the library's cs_build_kernel_table).
"""
import ctypes as C
import math

import numpy as np

from . import abi

NAG = abi.CS_NUM_AGE_GROUPS
NPT_MAX = abi.CS_MAX_PLACE_TYPES
REF_PI = 3.1415926535  # src/Constants.h:27


def natural_history():
    """Disease natural history of the UK parameter set (values as published)."""
    icdf_mild = [0, 0.341579599, 0.436192391, 0.509774887, 0.574196702, 0.633830053, 0.690927761, 0.74691114,
                 0.802830695, 0.859578883, 0.918015187, 0.97906363, 1.043815683, 1.113669859, 1.190557274,
                 1.277356871, 1.378761429, 1.50338422, 1.670195767, 1.938414132, 2.511279379]
    return dict(
        LatentPeriod=4.59,
        latent_icdf=[0, 0.098616903, 0.171170649, 0.239705594, 0.307516598, 0.376194441, 0.446827262, 0.520343677,
                     0.597665592, 0.679808341, 0.767974922, 0.863671993, 0.968878064, 1.086313899, 1.219915022,
                     1.37573215, 1.563841395, 1.803041398, 2.135346254, 2.694118208, 3.964172493],
        InfectiousPeriod=14.0,
        infectious_prof=[0.487464241, 1, 1.229764827, 1.312453175, 1.307955665, 1.251658756, 1.166040358, 1.065716869,
                         0.960199498, 0.855580145, 0.755628835, 0.662534099, 0.577412896, 0.500665739, 0.432225141,
                         0.371729322, 0.318643018, 0.272340645, 0.232162632, 0.19745264, 0.167581252, 0.141960133,
                         0.120049578, 0.101361532, 0.085459603, 0.071957123, 0.060514046, 0.050833195, 0.04265624,
                         0.035759641, 0.029950735, 0.025064045, 0.02095788, 0.017511251, 0.014621091, 0.012199802,
                         0.010173075, 0.008477992, 0.007061366, 0.005878301, 0.00489096, 0.004067488, 0.003381102,
                         0.00280931, 0.002333237, 0.001937064, 0.001607543, 0.001333589, 0.001105933, 0.00091683,
                         0.000759816, 0.000629496, 0.000521372, 0.000431695, 0.000357344, 0.000295719],
        k_infectiousness=1.0,  # [k of individual variation in infectiousness]: InfectiousnessSD = 1/sqrt(k)
        LatentToSymptDelay=0.5,
        ProportionSymptomatic=[0.66] * NAG,
        SymptInfectiousness=1.5,
        AsymptInfectiousness=1.0,
        SymptSpatialContactRate=0.5,
        SymptPlaceAttendance=[0.25, 0.25, 0.5, 0.5],
        RelativeSpatialContact=[0.6, 0.7, 0.75, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0.75, 0.5],
        HouseholdAttackRate=0.1,
        HouseholdTransPow=0.8,
        PlaceTypeTrans=[0.14, 0.14, 0.1, 0.07],
        PlaceTypePropBetweenGroupLinks=[0.25, 0.25, 0.25, 0.25],
        PlaceTypeGroupSizeParam1=[25, 25, 100, 10],
        CaseAbsentChildAgeCutoff=16,
        CaseAbsentChildPropAdultCarers=1.0,
        CaseAbsenteeismDuration=7.0,
        Mean_MildToRecovery=7, Mean_ILIToRecovery=7, Mean_ILIToSARI=5, Mean_SARIToRecovery=1, Mean_SARIToDeath=1,
        Mean_SARIToCritical=1, Mean_CriticalToCritRecov=1, Mean_CriticalToDeath=1, Mean_CritRecovToRecov=1,
        Mean_ILIToDeath=7,
        MildToRecovery_icdf=icdf_mild, ILIToRecovery_icdf=icdf_mild, ILIToSARI_icdf=icdf_mild,
        SARIToRecovery_icdf=[0, 0.634736097, 1.217461548, 1.805695261, 2.41206761, 3.044551205, 3.71010552, 4.415905623,
                             5.170067405, 5.982314035, 6.864787504, 7.833196704, 8.908589322, 10.12027655, 11.51100029,
                             13.14682956, 15.13821107, 17.69183155, 21.27093904, 27.35083955, 41.35442157],
        SARIToDeath_icdf=[0, 1.703470233, 2.39742257, 2.970367222, 3.491567676, 3.988046604, 4.474541783, 4.960985883,
                          5.455292802, 5.964726999, 6.496796075, 7.06004732, 7.665014091, 8.325595834, 9.061367792,
                          9.901900127, 10.8958347, 12.133068, 13.81280888, 16.56124574, 22.5803431],
        SARIToCritical_icdf=[0, 0.108407687, 0.220267228, 0.337653773, 0.46159365, 0.593106462, 0.733343356, 0.88367093,
                             1.045760001, 1.221701998, 1.414175806, 1.62669998, 1.864032461, 2.132837436, 2.442868902,
                             2.809242289, 3.257272257, 3.834402667, 4.647120033, 6.035113821, 9.253953212],
        CriticalToCritRecov_icdf=[0, 1.308310071, 1.87022015, 2.338694632, 2.76749788, 3.177830401, 3.581381361,
                                  3.986127838, 4.398512135, 4.824525291, 5.270427517, 5.743406075, 6.252370864,
                                  6.809125902, 7.430338867, 8.141231404, 8.983341913, 10.03350866, 11.46214198,
                                  13.80540164, 18.95469153],
        CriticalToDeath_icdf=[0, 1.60649128, 2.291051747, 2.860938008, 3.382077741, 3.880425012, 4.37026577,
                              4.861330415, 5.361460943, 5.877935626, 6.4183471, 6.991401405, 7.607881726, 8.282065409,
                              9.034104744, 9.894486491, 10.91341144, 12.18372915, 13.9113346, 16.74394356, 22.96541429],
        CritRecovToRecov_icdf=[0, 0.133993315, 0.265922775, 0.402188416, 0.544657341, 0.694774487, 0.853984373,
                               1.023901078, 1.206436504, 1.403942719, 1.619402771, 1.856711876, 2.121118605, 2.419957988,
                               2.763950408, 3.169692564, 3.664959893, 4.301777536, 5.196849239, 6.7222126, 10.24997697],
        ILIToDeath_icdf=[0, 2.257735908, 3.171065856, 3.924183798, 4.608738224, 5.260437017, 5.898728066, 6.53669783,
                         7.184755068, 7.852438367, 8.549591424, 9.287408763, 10.07967529, 10.94457146, 11.90769274,
                         13.00769447, 14.3081531, 15.92655201, 18.12320384, 21.71626849, 29.58154704],
        Prop_ILI_ByAge=[0.333122437, 0.333153617, 0.333001453, 0.332654731, 0.33181821, 0.330417289, 0.328732618,
                        0.326716425, 0.325130732, 0.322392505, 0.316971878, 0.312809664, 0.304540269, 0.300182488,
                        0.2919304, 0.283276936, 0.282323232],
        Prop_SARI_ByAge=[0.000557744, 0.000475283, 0.000877703, 0.001794658, 0.004006955, 0.007711884, 0.012167229,
                         0.017359248, 0.021140307, 0.027047193, 0.03708932, 0.039871236, 0.040788928, 0.027444452,
                         0.101605674, 0.142001415, 0.150469697],
        Prop_Critical_ByAge=[7.49444E-05, 6.38641E-05, 0.000117937, 0.000241149, 0.000538417, 0.00103625, 0.001634918,
                             0.002491477, 0.003467496, 0.005775292, 0.011995047, 0.021699771, 0.045590266,
                             0.072008084, 0.022603126, 0.008167778, 0.002560606],
        CFR_Critical_ByAge=[0.5234896] * NAG,
        CFR_SARI_ByAge=[0.125893251, 0.12261338, 0.135672867, 0.152667869, 0.174303077, 0.194187895, 0.209361731,
                        0.224432564, 0.237013516, 0.257828065, 0.290874602, 0.320763971, 0.362563751, 0.390965457,
                        0.421151485, 0.447545892, 0.482],
        CFR_ILI_ByAge=[0.0] * NAG,
    )


def interventions_c1():
    """Intervention efficacies of the 10 M configuration (case isolation 0.7,
    household quarantine 0.5, school/university closure, 75% social distancing),
    with the residual-contact values of the reference's p_PC7_CI_HQ_SD set."""
    return dict(
        CaseIsolationProp=0.7, CaseIsolationEffectiveness=0.25, CaseIsolationHouseEffectiveness=0.5,
        CaseIsolationDelay=1.0, CaseIsolationDuration=7.0,
        HQuarantinePropHouseCompliant=0.5, HQuarantinePropIndivCompliant=1.0, HQuarantineDelay=1.0,
        HQuarantineHouseDuration=14.0, HQuarantineHouseEffect=1.5, HQuarantinePlaceEffect=[0.25] * 4,
        HQuarantineSpatialEffect=0.25,
        PlaceCloseEffect=[0.0, 0.0, 0.0, 1.0], PlaceCloseHouseholdRelContact=1.5, PlaceCloseSpatialRelContact=1.25,
        SocDistPlaceEffect=[1.0, 1.0, 0.25, 0.25], SocDistHouseholdEffect=1.25, SocDistSpatialEffect=0.25,
        EnhancedSocDistPlaceEffect=[0.25] * 4, EnhancedSocDistHouseholdEffect=1.0, EnhancedSocDistSpatialEffect=0.25,
    )


def haversine_tables():
    """P.sinx/cosx/asin2sqx (src/ReadParams.cpp:2333-2346)."""
    asin2 = np.empty(1001)
    for i in range(1001):
        a = math.asin(math.sqrt(i / 1000.0))
        asin2[i] = a * a
    sinx = np.empty(361)
    cosx = np.empty(361)
    for i in range(361):
        t = REF_PI * i / 180
        sinx[i] = math.sin(t)
        cosx[i] = math.cos(t)
    return sinx, cosx, asin2


def infectiousness_profile(prof, infectious_period, dt):
    """P.infectiousness[] from the profile (src/ReadParams.cpp:1996-2016)."""
    res = len(prof)
    prof = list(prof) + [0.0]
    k = int(math.ceil(infectious_period / dt))
    out = np.zeros(abi.CS_MAX_INFECTIOUS_STEPS)
    s = 0.0
    for i in range(k):
        t = i * dt / infectious_period * res
        j = int(t)
        t -= j
        out[i] = prof[j] * (1 - t) + prof[j + 1] * t if j < res else prof[res]
        s += out[i]
    s /= k
    out[:k + 1] /= s
    return out


def _set_icdf(icdf, values):
    for i, v in enumerate(values):
        icdf.v[i] = math.exp(-v)


def longest_distance2(p):
    """Square of the longest distance across the domain (src/SetupModel.cpp:196-208)."""
    from .geometry import dist2_raw
    t = dist2_raw(p, 0, 0, p.width_deg, p.height_deg)
    tw = dist2_raw(p, 0, 0, p.width_deg, 0)
    th = dist2_raw(p, 0, 0, 0, p.height_deg)
    t = max(t, tw, th)
    if p.DoPeriodicBoundaries:
        t *= 0.25
    return t


def build_params(grid, nh=None, iv=None, r0_local_beta=None, kernel=(5, 4000.0, 3.0, 0.0, 0.0),
                 kernel_size=4000000, kernel_expansion=None, num_place_types=4, severity=True, seasonality=1.0):
    """Return (cs_params, kernel_lookup, kernel_hi_res) for a grid description.

    grid: dict with ncw, nch, cell_width, cell_height (degrees), bbox_bottom_left_y.
    """
    nh = dict(natural_history(), **(nh or {}))
    p = abi.cs_params()
    p.TimeStepsPerDay = 4.0
    p.ModelTimeStep = 0.25
    p.DoHouseholds = 1
    p.DoPlaces = 1 if num_place_types > 0 else 0
    p.DoSpatial = 1
    p.DoSymptoms = 1
    p.DoSeverity = 1 if severity else 0
    p.DoLatent = 1
    p.DoInfectiousnessProfile = 1
    p.NoInfectiousnessSDinHH = 0
    p.DoUTM_coords = 1
    p.DoPeriodicBoundaries = 0
    p.DoRealSymptWithdrawal = 1
    p.DoDeathCountsInS0 = 0
    p.NumPlaceTypes = num_place_types
    p.HotelPlaceType = num_place_types      # no airports: hotel type == NumPlaceTypes
    p.CareHomePlaceType = -1
    p.PlaceTypeNoAirNum = num_place_types
    p.IncludeStepDownToDeath = 0
    p.CaseAbsentChildAgeCutoff = nh["CaseAbsentChildAgeCutoff"]
    p.DoHQretrigger = 0
    p.LocalBeta = 0.0 if r0_local_beta is None else r0_local_beta
    p.HouseholdTrans = nh["HouseholdAttackRate"]
    p.FalsePositiveRate = 0.0
    p.Seasonality = seasonality
    p.HouseholdDenomLookup[0] = 1.0
    for i in range(1, abi.CS_MAX_HOUSEHOLD_SIZE):
        p.HouseholdDenomLookup[i] = 1 / ((1.0 + i) ** nh["HouseholdTransPow"])
    prof = infectiousness_profile(nh["infectious_prof"], nh["InfectiousPeriod"], p.ModelTimeStep)
    for i in range(abi.CS_MAX_INFECTIOUS_STEPS):
        p.infectiousness[i] = prof[i]
    for t in range(NPT_MAX):
        if t < num_place_types:
            p.PlaceTypeTrans[t] = nh["PlaceTypeTrans"][t]
            p.PlaceTypeGroupSizeParam1[t] = nh["PlaceTypeGroupSizeParam1"][t]
            p.PlaceTypePropBetweenGroupLinks[t] = nh["PlaceTypePropBetweenGroupLinks"][t]
            att = nh["SymptPlaceAttendance"][t]
        else:
            p.PlaceTypeGroupSizeParam1[t] = 1.0
            att = 0.0
        # DoRealSymptWithdrawal: attendance becomes a withdrawal probability (ReadParams.cpp:2065-2071)
        p.SymptPlaceTypeWithdrawalProp[t] = 1.0 - att
        p.SymptPlaceTypeContactRate[t] = 1.0
    p.SymptSpatialContactRate = nh["SymptSpatialContactRate"]
    for a in range(NAG):
        p.RelativeSpatialContact[a] = nh["RelativeSpatialContact"][a]
        p.RelativeSpatialContactSusc[a] = 1.0
        p.AgeSusceptibility[a] = 1.0
        p.AgeInfectiousness[a] = 1.0
        p.ProportionSymptomatic[a] = nh["ProportionSymptomatic"][a]
        for b in range(NAG):
            p.WAIFW_Matrix[a][b] = 1.0
            p.WAIFW_Matrix_SpatialOnly[a][b] = 1.0
    p.CareHomeResidentHouseholdScaling = p.CareHomeResidentSpatialScaling = 1.0
    p.CareHomeWorkerGroupScaling = p.CareHomeResidentPlaceScaling = p.CareHomeRelProbHosp = 1.0
    ivp = dict(interventions_c1(), **(iv or {}))
    E = p.Efficacies
    S_HOUSE, S_SP = abi.CS_SETTING_HOUSE, abi.CS_SETTING_SPATIAL
    for t in range(NPT_MAX):
        tt = min(t, 3)
        E[0][t] = ivp["CaseIsolationEffectiveness"]
        E[1][t] = ivp["HQuarantinePlaceEffect"][tt]
        E[2][t] = ivp["PlaceCloseEffect"][tt]
        E[3][t] = ivp["SocDistPlaceEffect"][tt]
        E[4][t] = ivp["EnhancedSocDistPlaceEffect"][tt]
        E[5][t] = 1.0
    E[0][S_HOUSE], E[0][S_SP] = ivp["CaseIsolationHouseEffectiveness"], ivp["CaseIsolationEffectiveness"]
    E[1][S_HOUSE], E[1][S_SP] = ivp["HQuarantineHouseEffect"], ivp["HQuarantineSpatialEffect"]
    E[2][S_HOUSE], E[2][S_SP] = ivp["PlaceCloseHouseholdRelContact"], ivp["PlaceCloseSpatialRelContact"]
    E[3][S_HOUSE], E[3][S_SP] = ivp["SocDistHouseholdEffect"], ivp["SocDistSpatialEffect"]
    E[4][S_HOUSE], E[4][S_SP] = ivp["EnhancedSocDistHouseholdEffect"], ivp["EnhancedSocDistSpatialEffect"]
    E[5][S_HOUSE] = E[5][S_SP] = 1.0
    p.MoveRestrEffect = 0.0
    p.LatentPeriod = nh["LatentPeriod"]
    p.InfectiousPeriod = nh["InfectiousPeriod"]
    p.LatentToSymptDelay = nh["LatentToSymptDelay"]
    p.SymptInfectiousness = nh["SymptInfectiousness"]
    p.AsymptInfectiousness = nh["AsymptInfectiousness"]
    p.InfectiousnessSD = 1.0 / math.sqrt(nh["k_infectiousness"])
    _set_icdf(p.latent_icdf, nh["latent_icdf"])
    # with an infectiousness profile the infectious ICDF is a constant exp(-1) (ReadParams.cpp:2016)
    for i in range(abi.CS_CDF_RES + 1):
        p.infectious_icdf.v[i] = math.exp(-1.0)
    for name in ("MildToRecovery", "ILIToRecovery", "SARIToRecovery", "CriticalToCritRecov", "CritRecovToRecov",
                 "ILIToSARI", "SARIToCritical", "ILIToDeath", "SARIToDeath", "CriticalToDeath"):
        _set_icdf(getattr(p, name + "_icdf"), nh[name + "_icdf"])
        arr = getattr(p, "Mean_" + name)
        for a in range(NAG):
            arr[a] = nh["Mean_" + name]
    # IncludeStepDownToDeath == 0: stepdown->death copies critrecov->recovery (ReadParams.cpp:797-803)
    for i in range(abi.CS_CDF_RES + 1):
        p.StepdownToDeath_icdf.v[i] = p.CritRecovToRecov_icdf.v[i]
    for a in range(NAG):
        p.Mean_StepdownToDeath[a] = p.Mean_CritRecovToRecov[a]
        p.Prop_ILI_ByAge[a] = nh["Prop_ILI_ByAge"][a]
        p.Prop_SARI_ByAge[a] = nh["Prop_SARI_ByAge"][a]
        p.Prop_Critical_ByAge[a] = nh["Prop_Critical_ByAge"][a]
        p.CFR_Critical_ByAge[a] = nh["CFR_Critical_ByAge"][a]
        p.CFR_SARI_ByAge[a] = nh["CFR_SARI_ByAge"][a]
        p.CFR_ILI_ByAge[a] = nh["CFR_ILI_ByAge"][a]
    p.CFR_Critical_Scale_Current = p.CFR_SARI_Scale_Current = p.CFR_ILI_Scale_Current = 1.0
    p.ControlPropCasesId = 1.0
    p.CaseIsolationProp = ivp["CaseIsolationProp"]
    p.HQuarantinePropHouseCompliant = ivp["HQuarantinePropHouseCompliant"]
    p.HQuarantinePropIndivCompliant = ivp["HQuarantinePropIndivCompliant"]
    p.HQuarantineDelay = ivp["HQuarantineDelay"]
    p.CaseAbsentChildPropAdultCarers = nh["CaseAbsentChildPropAdultCarers"]
    spd = p.TimeStepsPerDay
    p.usCaseIsolationDelay = int(ivp["CaseIsolationDelay"] * spd)
    p.usCaseIsolationDuration = int(ivp["CaseIsolationDuration"] * spd)
    p.usCaseAbsenteeismDelay = 0
    p.usCaseAbsenteeismDuration = int(nh["CaseAbsenteeismDuration"] * spd)
    p.usHQuarantineHouseDuration = int(ivp["HQuarantineHouseDuration"] * spd)
    p.ncw, p.nch = grid["ncw"], grid["nch"]
    p.cell_width, p.cell_height = grid["cell_width"], grid["cell_height"]
    p.width_deg, p.height_deg = p.ncw * p.cell_width, p.nch * p.cell_height
    p.bbox_bottom_left_y = grid["bbox_bottom_left_y"]
    sinx, cosx, asin2 = haversine_tables()
    for i in range(361):
        p.sinx[i], p.cosx[i] = sinx[i], cosx[i]
    for i in range(1001):
        p.asin2sqx[i] = asin2[i]
    p.block_cells = 0
    # spatial kernel table
    lib = abi.load_library()
    ktype, kscale, kshape, kp3, kp4 = kernel
    p.kernel_size = kernel_size
    p.kernel_expansion = kernel_expansion or kernel_size // 1600
    lookup = np.empty(kernel_size + 1)
    hires = np.empty(kernel_size + 1)
    delta = C.c_double()
    rc = lib.cs_build_kernel_table(ktype, kscale, kshape, kp3, kp4, longest_distance2(p), kernel_size,
                                   p.kernel_expansion, lookup.ctypes.data, hires.ctypes.data, C.byref(delta))
    if rc != 0:
        raise abi.CovidSimError("cs_build_kernel_table failed (%d)" % rc)
    p.kernel_delta = delta.value
    return p, lookup, hires
