"""Write a synthetic workload in the reference's own input formats.

The reference executable reads three `[Key]` parameter files (pre-parameters /PP,
administrative-unit parameters /A, parameters /P; src/ReadParams.cpp) and a
population density file /D with one line "x y population country admin-unit" per
microcell (src/SetupModel.cpp:73-104).  This module emits those files for a
population from covidsim_b200.population, so the reference builds its own
households, ages and places from the same microcell populations and runs the same
disease model and interventions.  Values are the published UK parameter set
(covidsim_b200.params.natural_history) and the workload's intervention settings.
"""
import os

import numpy as np

from . import params as prm
from .population import AGE_DIST, GROUP_SIZE_PARAM1, HH_SIZE_DIST, PLACE_AGE_BANDS, PLACE_MEAN_SIZE

ADMIN_CODE = 560300        # one level-1 admin unit: (code % 100000) / 100 = 603
COUNTRY_CODE = 5


def _fmt(v):
    if isinstance(v, (list, tuple, np.ndarray)):
        if len(v) and isinstance(v[0], (list, tuple, np.ndarray)):
            return "\n".join(_fmt(r) for r in v)
        return "\t".join(_fmt(x) for x in v)
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    if isinstance(v, np.integer):
        return str(int(v))
    return str(v)


def write_params(path, d):
    with open(path, "w") as f:
        for k, v in d.items():
            f.write("[%s]\n%s\n\n" % (k, _fmt(v)))


def pre_params(days, grid, r0, n_seed, nh=None):
    nh = dict(prm.natural_history(), **(nh or {}))
    nag = 17
    return {
        "Output every realisation": 1, "Output bitmap": 0, "OutputAge": 0, "OutputSeverityAdminUnit": 0,
        "OutputR0": 0, "OutputControls": 0, "OutputCountry": 0, "OutputAdUnitVar": 0, "OutputHousehold": 0,
        "OutputInfType": 0, "OutputNonSeverity": 0, "OutputNonSummaryResults": 0,
        "Output incidence by administrative unit": 0, "Output infection tree": 0,
        "Only output non-extinct realisations": 0,
        "Include administrative units within countries": 1,
        "Update timestep": 0.25, "Equilibriation time": 0, "Sampling timestep": 1, "Sampling time": days,
        "Grid size": grid["cell_width"],
        "Spatial domain for simulation": [[grid["bbox_bottom_left_x"], grid["bbox_bottom_left_y"]],
                                          [grid["bbox_bottom_left_x"] + grid["ncw"] * grid["cell_width"],
                                           grid["bbox_bottom_left_y"] + grid["nch"] * grid["cell_height"]]],
        "Number of micro-cells per spatial cell width": grid["nmcl"],
        "Initial immunity profile by age": [0] * nag, "Initial immunity applied to all household members": 1,
        "Relative spatial contact rates by age": nh["RelativeSpatialContact"],
        "Household attack rate": nh["HouseholdAttackRate"],
        "Household transmission denominator power": nh["HouseholdTransPow"],
        "Relative transmission rates for place types": nh["PlaceTypeTrans"],
        "Proportion of between group place links": nh["PlaceTypePropBetweenGroupLinks"],
        "Include symptoms": 1, "Delay from end of latent period to start of symptoms": nh["LatentToSymptDelay"],
        "Proportion symptomatic by age group": nh["ProportionSymptomatic"],
        "Symptomatic infectiousness relative to asymptomatic": nh["SymptInfectiousness"],
        "Relative rate of random contacts if symptomatic": nh["SymptSpatialContactRate"],
        "Relative level of place attendance if symptomatic": nh["SymptPlaceAttendance"],
        "Model symptomatic withdrawal to home as true absenteeism": 1,
        "Maximum age of child at home for whom one adult also stays at home": nh["CaseAbsentChildAgeCutoff"],
        "Proportion of children at home for whom one adult also stays at home": nh["CaseAbsentChildPropAdultCarers"],
        "Duration of place absenteeism for cases who withdraw": nh["CaseAbsenteeismDuration"],
        "Place close round household": 1, "Absenteeism place closure": 0,
        "Initial number of infecteds": n_seed, "Time when infection rate changes": 30,
        "Initial rate of importation of infections": 0, "Changed rate of importation of infections": 0,
        "Length of importation time profile provided": 0, "Daily importation time profile": [0.0],
        "Reproduction number": r0, "Power of scaling of spatial R0 with density": 0,
        "Include latent period": 1, "Latent period": nh["LatentPeriod"],
        "Latent period inverse CDF": nh["latent_icdf"], "Model time varying infectiousness": 1,
        "Infectiousness profile": nh["infectious_prof"], "Infectious period": nh["InfectiousPeriod"],
        "Infectious period inverse CDF": [0, 0.171566836, 0.424943468, 0.464725594, 0.50866631, 0.55773764,
                                          0.613298069, 0.67732916, 0.752886568, 0.843151261, 0.895791527,
                                          0.955973422, 1.026225109, 1.110607115, 1.216272375, 1.336349102,
                                          1.487791911, 1.701882384, 1.865779085, 2.126940581, 2.524164972],
        "k of individual variation in infectiousness": nh["k_infectiousness"],
        "Use global triggers for interventions": 1, "Use admin unit triggers for interventions": 0,
        "Number of sampling intervals over which cumulative incidence measured for global trigger": 7,
        "Use cases per thousand threshold for area controls": 0,
        "Divisor for per-capita global threshold (default 1000)": 1000,
        "Divisor for per-capita area threshold (default 1000)": 1000,
        "Trigger alert on deaths": 0, "Number of deaths accummulated before alert": 0,
        "Number of days to accummulate cases/deaths before alert": 100, "Day of year trigger is reached": 0,
        "Alert trigger starts after interventions": 0, "Day of year interventions start": 0,
        "Proportion of cases detected for treatment": 1, "Treatment trigger incidence per cell": 100000,
        "Places close only once": 1, "Social distancing only once": 1, "Use ICU case triggers for interventions": 1,
        "Proportion of cases detected before outbreak alert": 1,
        "Number of detected cases needed before outbreak alert triggered": 0,
        "Number of realisations": 1, "Number of non-extinct realisations": 1,
        "Maximum number of cases defining small outbreak": 100, "Do one generation": 0, "Bitmap scale": 60,
        "Bitmap y:x aspect scaling": 1.5, "Calculate spatial correlations": 0, "Bitmap movie frame interval": 300,
        "Record infection events": 0, "Record infection events per run": 0,
        "Max number of infection events to record": 1000, "Limit number of infections": 0,
        "Max number of infections": 1000000000, "Do Severity Analysis": 1,
        "Mean_MildToRecovery": nh["Mean_MildToRecovery"], "Mean_ILIToRecovery": nh["Mean_ILIToRecovery"],
        "Mean_ILIToSARI": nh["Mean_ILIToSARI"], "Mean_SARIToRecovery": nh["Mean_SARIToRecovery"],
        "Mean_SARIToDeath": nh["Mean_SARIToDeath"], "Mean_SARIToCritical": nh["Mean_SARIToCritical"],
        "Mean_CriticalToCritRecov": nh["Mean_CriticalToCritRecov"], "Mean_CriticalToDeath": nh["Mean_CriticalToDeath"],
        "Mean_CritRecovToRecov": nh["Mean_CritRecovToRecov"], "MeanTimeToTest": 4, "MeanTimeToTestOffset": 1,
        "MeanTimeToTestCriticalOffset": 3.3, "MeanTimeToTestCritRecovOffset": 9.32,
        "MildToRecovery_icdf": nh["MildToRecovery_icdf"], "ILIToRecovery_icdf": nh["ILIToRecovery_icdf"],
        "ILIToSARI_icdf": nh["ILIToSARI_icdf"], "SARIToRecovery_icdf": nh["SARIToRecovery_icdf"],
        "SARIToDeath_icdf": nh["SARIToDeath_icdf"], "SARIToCritical_icdf": nh["SARIToCritical_icdf"],
        "CriticalToCritRecov_icdf": nh["CriticalToCritRecov_icdf"], "CriticalToDeath_icdf": nh["CriticalToDeath_icdf"],
        "CritRecovToRecov_icdf": nh["CritRecovToRecov_icdf"],
        "Prop_Mild_ByAge": list(1 - np.asarray(nh["Prop_ILI_ByAge"]) - np.asarray(nh["Prop_SARI_ByAge"])
                                - np.asarray(nh["Prop_Critical_ByAge"])),
        "Prop_ILI_ByAge": nh["Prop_ILI_ByAge"], "Prop_SARI_ByAge": nh["Prop_SARI_ByAge"],
        "Prop_Critical_ByAge": nh["Prop_Critical_ByAge"], "CFR_Critical_ByAge": nh["CFR_Critical_ByAge"],
        "CFR_SARI_ByAge": nh["CFR_SARI_ByAge"], "CFR_ILI_ByAge": nh["CFR_ILI_ByAge"],
        "Mean_ILIToDeath": nh["Mean_ILIToDeath"], "ILIToDeath_icdf": nh["ILIToDeath_icdf"],
        "Mean child age gap": 2, "Min adult age": 19, "Max MF partner age gap": 5, "Max FM partner age gap": 5,
        "Min parent age gap": 19, "Max parent age gap": 44, "Max child age": 20, "One Child Two Pers Prob": 0.08,
        "Two Child Three Pers Prob": 0.11, "One Pers House Prob Old": 0.5, "Two Pers House Prob Old": 0.5,
        "One Pers House Prob Young": 0.23, "Two Pers House Prob Young": 0.23,
        "One Child Prob Youngest Child Under Five": 0.5, "Two Children Prob Youngest Under Five": 0.0,
        "Prob Youngest Child Under Five": 0, "Zero Child Three Pers Prob": 0.25, "One Child Four Pers Prob": 0.2,
        "Young And Single Slope": 0.7, "Young And Single": 36, "No Child Pers Age": 44, "Old Pers Age": 60,
        "Three Child Five Pers Prob": 0.5, "Older Gen Gap": 19,
    }


def admin_params(n_people, n_seed, kernel=(5, 4000.0, 3.0)):
    ad = np.asarray(AGE_DIST, dtype=float)
    ad /= ad.sum()
    hh = list(HH_SIZE_DIST) + [0.0] * (10 - len(HH_SIZE_DIST))
    return {
        "Number of seed locations": 1, "Initial number of infecteds": n_seed,
        "Administrative unit to seed initial infection into": 0, "Population size": n_people,
        "Fix population size at specified value": 1, "Number of countries to include": 0,
        "List of names of countries to include": "Synthetica",
        "Number of level 1 administrative units to include": 1, "List of level 1 administrative units to include": "Region",
        "Codes and country/province names for admin units": "%d\tSynthetica\tRegion" % ADMIN_CODE,
        "Mask for level 1 administrative units": 100000, "Divisor for level 1 administrative units": 100,
        "Divisor for countries": 100000, "Correct administrative unit populations": 0,
        "Age distribution of population": list(ad), "Household size distribution": hh,
        "Correct age distribution after household allocation to exactly match specified demography": 1,
        "Include places": 1, "Place overlap matrix": [[1 if i == j else 0 for j in range(4)] for i in range(4)],
        "Number of types of places": 4,
        "Proportion of age group 1 in place types": [b[0][2] for b in PLACE_AGE_BANDS],
        "Minimum age for age group 1 in place types": [b[0][0] for b in PLACE_AGE_BANDS],
        "Maximum age for age group 1 in place types": [b[0][1] for b in PLACE_AGE_BANDS],
        "Proportion of age group 2 in place types": [b[1][2] for b in PLACE_AGE_BANDS],
        "Minimum age for age group 2 in place types": [b[1][0] for b in PLACE_AGE_BANDS],
        "Maximum age for age group 2 in place types": [b[1][1] for b in PLACE_AGE_BANDS],
        "Proportion of age group 3 in place types": [b[2][2] for b in PLACE_AGE_BANDS],
        "Minimum age for age group 3 in place types": [b[2][0] for b in PLACE_AGE_BANDS],
        "Maximum age for age group 3 in place types": [b[2][1] for b in PLACE_AGE_BANDS],
        "Kernel shape params for place types": [kernel[2]] * 4, "Kernel scale params for place types": [kernel[1]] * 4,
        "Mean size of place types": PLACE_MEAN_SIZE, "Number of closest places people pick from (0=all) for place types": [3, 3, 6, 0],
        "Param 1 of place group size distribution": GROUP_SIZE_PARAM1, "Power of place size distribution": [0, 0, 0, 1.34],
        "Offset of place size distribution": [0, 0, 0, 5.35], "Maximum of place size distribution": [0, 0, 0, 5000],
        "Kernel type": kernel[0], "Kernel scale": kernel[1], "Kernel Shape": kernel[2],
        "Include holidays": 0, "Number of holidays": 0,
    }


def intervention_params(interventions, duration=90.0, threshold=100):
    """p_NoInt-style file; with interventions, the global ICU trigger of the 10 M
    workload switches CI, HQ, school/university closure and SD on for `duration`."""
    iv = prm.interventions_c1()
    never = 100000
    on = interventions
    st = 0 if on else never
    return {
        "Include intervention delays by admin unit": 0, "Vary efficacies over time": 0,
        "Place closure start time": st, "Place closure second start time": never,
        "Delay to place closure by admin unit": [0], "Duration of place closure by admin unit": [0],
        "Place closure in administrative units rather than rings": 0, "Administrative unit divisor for place closure": 1,
        "Place types to close for admin unit closure (0/1 array)": [1, 1, 1, 0],
        "Cumulative proportion of place members needing to become sick for admin unit closure": 1,
        "Proportion of places in admin unit needing to pass threshold for place closure": 1,
        "Delay to start place closure": 0, "Duration of place closure": duration if on else 0,
        "Proportion of places remaining open after closure by place type": iv["PlaceCloseEffect"],
        "Relative household contact rate after closure": iv["PlaceCloseHouseholdRelContact"],
        "Relative spatial contact rate after closure": iv["PlaceCloseSpatialRelContact"],
        "Minimum radius for place closure": 1,
        "Place closure incidence threshold": threshold if on else 1000000000,
        "Place closure fractional incidence threshold": 0, "Trigger incidence per cell for place closure": 1000000000,
        "Household quarantine start time": st, "Delay to start household quarantine": iv["HQuarantineDelay"],
        "Delay to household quarantine by admin unit": [0], "Duration of household quarantine by admin unit": [0],
        "Household quarantine trigger incidence per cell": threshold if on else 1000000000,
        "Length of time households are quarantined": iv["HQuarantineHouseDuration"],
        "Duration of household quarantine policy": duration if on else 0,
        "Relative household contact rate after quarantine": iv["HQuarantineHouseEffect"],
        "Residual place contacts after household quarantine by place type": iv["HQuarantinePlaceEffect"],
        "Residual spatial contacts after household quarantine": iv["HQuarantineSpatialEffect"],
        "Household level compliance with quarantine": iv["HQuarantinePropHouseCompliant"],
        "Individual level compliance with quarantine": iv["HQuarantinePropIndivCompliant"],
        "Case isolation start time": st, "Delay to case isolation by admin unit": [0],
        "Duration of case isolation by admin unit": [0],
        "Case isolation trigger incidence per cell": threshold if on else 1000000000,
        "Proportion of detected cases isolated": iv["CaseIsolationProp"],
        "Delay to start case isolation": iv["CaseIsolationDelay"], "Duration of case isolation": iv["CaseIsolationDuration"],
        "Duration of case isolation policy": duration if on else 0,
        "Residual contacts after case isolation": iv["CaseIsolationEffectiveness"],
        "Residual household contacts after case isolation": iv["CaseIsolationHouseEffectiveness"],
        "Social distancing start time": st, "Delay to social distancing by admin unit": [0],
        "Duration of social distancing": duration if on else 0, "Duration of social distancing by admin unit": [0],
        "Trigger incidence per cell for social distancing": threshold if on else 1000000000,
        "Relative place contact rate given social distancing by place type": iv["SocDistPlaceEffect"],
        "Relative household contact rate given social distancing": iv["SocDistHouseholdEffect"],
        "Relative spatial contact rate given social distancing": iv["SocDistSpatialEffect"],
        "Minimum radius for social distancing": 1, "Proportion compliant with enhanced social distancing": 0.0,
        "Proportion compliant with enhanced social distancing by age group": [0] * 17,
        "Relative place contact rate given enhanced social distancing by place type": iv["EnhancedSocDistPlaceEffect"],
        "Relative household contact rate given enhanced social distancing": iv["EnhancedSocDistHouseholdEffect"],
        "Relative spatial contact rate given enhanced social distancing": iv["EnhancedSocDistSpatialEffect"],
        "Delay for change in effectiveness of social distancing": 1000,
        "Relative place contact rate given social distancing by place type after change": iv["SocDistPlaceEffect"],
        "Relative household contact rate given social distancing after change": iv["SocDistHouseholdEffect"],
        "Relative spatial contact rate given social distancing after change": iv["SocDistSpatialEffect"],
    }


def write_density(path, pop):
    """One line per populated microcell: centre x, y (degrees), people, country,
    admin unit; plus the two far corners with no people so the reference's bounding
    box covers the whole grid."""
    g = pop.grid
    th = g["nch"] * g["nmcl"]
    mcw, mch = g["cell_width"] / g["nmcl"], g["cell_height"] / g["nmcl"]
    mc = pop.mcell_grid
    counts = np.bincount(pop.person_mcell, minlength=pop.n_mcells)
    x = g["bbox_bottom_left_x"] + (mc // th + 0.5) * mcw
    y = g["bbox_bottom_left_y"] + (mc % th + 0.5) * mch
    x0, y0 = g["bbox_bottom_left_x"] + 0.5 * mcw, g["bbox_bottom_left_y"] + 0.5 * mch
    x1 = g["bbox_bottom_left_x"] + (g["ncw"] * g["nmcl"] - 0.5) * mcw
    y1 = g["bbox_bottom_left_y"] + (g["nch"] * g["nmcl"] - 0.5) * mch
    with open(path, "w") as f:
        f.write("%.9f %.9f 0 %d %d\n" % (x0, y0, COUNTRY_CODE, ADMIN_CODE))
        f.write("%.9f %.9f 0 %d %d\n" % (x1, y1, COUNTRY_CODE, ADMIN_CODE))
        for a, b, c in zip(x, y, counts):
            f.write("%.9f %.9f %d %d %d\n" % (a, b, c, COUNTRY_CODE, ADMIN_CODE))


def write_workload(outdir, pop, days, r0=2.4, n_seed=100, interventions=False):
    os.makedirs(outdir, exist_ok=True)
    files = dict(pre=os.path.join(outdir, "pre-params.txt"), admin=os.path.join(outdir, "admin-params.txt"),
                 params=os.path.join(outdir, "params.txt"), density=os.path.join(outdir, "density.txt"))
    write_params(files["pre"], pre_params(days, pop.grid, r0, n_seed))
    write_params(files["admin"], admin_params(pop.n_people, n_seed))
    write_params(files["params"], intervention_params(interventions))
    write_density(files["density"], pop)
    return files
