// Golden vectors from the reference's own leaf functions, for pinning the oracle.
//
// Links the reference's Kernels.cpp, Dist.cpp, InverseCdf.cpp, CalcInfSusc.cpp,
// Person.cpp and Rand.cpp (built from their sources by oracle/Makefile) and defines
// the few globals those files read, so no set-up code runs.  Prints one JSON
// document on stdout; tests/golden/make_ref_pins.py stores it as
// tests/golden/ref_pins.json.  Every value is printed with 17 significant digits,
// enough to round-trip a double.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "CalcInfSusc.h"
#include "Constants.h"
#include "Dist.h"
#include "InverseCdf.h"
#include "Kernels.h"
#include "Model.h"
#include "ModelMacros.h"
#include "Param.h"
#include "Rand.h"

// ---- globals the linked reference files expect (defined by CovidSim.cpp there)
Param P;
Person* Hosts;
std::vector<PersonQuarantine> HostsQuarantine;
Household* Households;
PopVar State, StateT[MAX_NUM_THREADS];
Cell* Cells;
Cell** CellLookup;
Microcell* Mcells;
Microcell** McellLookup;
Place** Places;
AdminUnit AdUnits[MAX_ADUNITS];

static void arr(const char* name, const double* v, int n, bool last = false)
{
    printf("\"%s\": [", name);
    for (int i = 0; i < n; i++) printf("%s%.17g", i ? ", " : "", v[i]);
    printf("]%s\n", last ? "" : ",");
}

static void setup_utm_tables()
{
    // the same tables src/ReadParams.cpp:2333-2346 builds
    for (int i = 0; i <= 1000; i++) {
        P.asin2sqx[i] = asin(sqrt(i / 1000.0));
        P.asin2sqx[i] = P.asin2sqx[i] * P.asin2sqx[i];
    }
    for (int i = 0; i <= DEGREES_PER_TURN; i++) {
        double t = PI * i / 180;
        P.sinx[i] = sin(t);
        P.cosx[i] = cos(t);
    }
}

static double lcg_u(unsigned long long& s)
{
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

int main()
{
    unsigned long long rs = 12345;
    printf("{\n");
    // ------------------------------------------------------------ geometry
    P.DoUTM_coords = 1;
    P.DoPeriodicBoundaries = 0;
    P.SpatialBoundingBox.bottom_left() = CovidSim::Geometry::Vector2d(0.0, 50.0);
    P.in_cells_.width = P.in_cells_.height = 1.0 / 120;
    P.nch = P.ncw = 240;
    P.in_degrees_.width = P.in_degrees_.height = 2.0;
    setup_utm_tables();
    {
        const int n = 400;
        std::vector<double> x1(n), y1(n), x2(n), y2(n), d(n);
        for (int i = 0; i < n; i++) {
            x1[i] = 2.0 * lcg_u(rs); y1[i] = 2.0 * lcg_u(rs);
            x2[i] = (i % 4 == 0) ? x1[i] + 0.01 * lcg_u(rs) : 2.0 * lcg_u(rs);
            y2[i] = 2.0 * lcg_u(rs);
            d[i] = dist2_raw(x1[i], y1[i], x2[i], y2[i]);
        }
        printf("\"utm\": {\"bbox_y\": 50.0, \"width\": 2.0,\n");
        arr("x1", x1.data(), n); arr("y1", y1.data(), n); arr("x2", x2.data(), n); arr("y2", y2.data(), n);
        arr("d2", d.data(), n, true);
        printf("},\n");
        // dist2_cc_min on grid cells (cell index = x * nch + y)
        Cells = new Cell[P.ncw * P.nch];
        std::vector<double> l(n), m(n), dc(n);
        for (int i = 0; i < n; i++) {
            int a = (int)(lcg_u(rs) * P.ncw * P.nch), b = (i % 3 == 0) ? a + 1 : (int)(lcg_u(rs) * P.ncw * P.nch);
            if (b >= P.ncw * P.nch) b = a;
            l[i] = a; m[i] = b;
            dc[i] = dist2_cc_min(Cells + a, Cells + b);
        }
        printf("\"cc_min\": {\"nch\": %d, \"cell\": %.17g,\n", P.nch, P.in_cells_.width);
        arr("l", l.data(), n); arr("m", m.data(), n); arr("d2", dc.data(), n, true);
        printf("},\n");
    }
    // -------------------------------------------------------- kernel lookup
    {
        double longest = dist2_raw(0, 0, P.in_degrees_.width, P.in_degrees_.height);
        double tw = dist2_raw(0, 0, P.in_degrees_.width, 0), th = dist2_raw(0, 0, 0, P.in_degrees_.height);
        if (tw > longest) longest = tw;
        if (th > longest) longest = th;
        P.KernelLookup.size_ = 4000000;
        P.KernelLookup.expansion_factor_ = P.KernelLookup.size_ / 1600;
        P.KernelLookup.setup(longest);
        P.Kernel.type_ = 5; P.Kernel.scale_ = 4000; P.Kernel.shape_ = 3; P.Kernel.p3_ = 0; P.Kernel.p4_ = 0;
        P.KernelLookup.init(1.0, P.Kernel);
        const int n = 500;
        std::vector<double> r2(n), v(n);
        for (int i = 0; i < n; i++) {
            double u = lcg_u(rs);
            r2[i] = (i % 2) ? u * longest : u * u * u * longest * 1e-3;
            v[i] = P.KernelLookup.num(r2[i]);
        }
        printf("\"kernel\": {\"type\": 5, \"scale\": 4000.0, \"shape\": 3.0, \"longest_d2\": %.17g, \"size\": %d, \"expansion\": %d,\n",
               longest, P.KernelLookup.size_, P.KernelLookup.expansion_factor_);
        arr("r2", r2.data(), n); arr("num", v.data(), n, true);
        printf("},\n");
        // type 2 (the shipped country files) too
        P.Kernel.type_ = 2;
        P.KernelLookup.init(1.0, P.Kernel);
        for (int i = 0; i < n; i++) v[i] = P.KernelLookup.num(r2[i]);
        printf("\"kernel2\": {\"type\": 2, \"scale\": 4000.0, \"shape\": 3.0, \"longest_d2\": %.17g, \"size\": %d, \"expansion\": %d,\n",
               longest, P.KernelLookup.size_, P.KernelLookup.expansion_factor_);
        arr("r2", r2.data(), n); arr("num", v.data(), n, true);
        printf("},\n");
    }
    // -------------------------------------------------- random generator state
    Xcg1 = (int32_t*)calloc(MAX_NUM_THREADS * CACHE_LINE_SIZE, sizeof(int32_t));
    Xcg2 = (int32_t*)calloc(MAX_NUM_THREADS * CACHE_LINE_SIZE, sizeof(int32_t));
    P.NumThreads = 1;
    int32_t s1 = 98798150, s2 = 729101;
    setall(&s1, &s2);
    // ---------------------------------------------------------- inverse CDF
    {
        static const double raw[CDF_RES + 1] = {0, 0.098616903, 0.171170649, 0.239705594, 0.307516598, 0.376194441,
                                                0.446827262, 0.520343677, 0.597665592, 0.679808341, 0.767974922,
                                                0.863671993, 0.968878064, 1.086313899, 1.219915022, 1.37573215,
                                                1.563841395, 1.803041398, 2.135346254, 2.694118208, 3.964172493};
        InverseCdf icdf;
        for (int i = 0; i <= CDF_RES; i++) icdf[i] = raw[i];
        icdf.assign_exponent();
        const int n = 300;
        std::vector<double> u(n), mean(n), out(n);
        for (int i = 0; i < n; i++) {
            // choose() draws ranf_mt(0): read the value it will draw, then rewind
            int32_t a = Xcg1[0], b = Xcg2[0];
            u[i] = ranf_mt(0);
            Xcg1[0] = a; Xcg2[0] = b;
            mean[i] = 0.5 + 20.0 * lcg_u(rs);
            out[i] = icdf.choose(mean[i], 0, 4.0);
        }
        printf("\"icdf\": {\"steps_per_day\": 4.0,\n");
        arr("raw", raw, CDF_RES + 1); arr("u", u.data(), n); arr("mean", mean.data(), n); arr("value", out.data(), n, true);
        printf("},\n");
    }
    // ------------------------------------------- samplers (distribution pins)
    {
        printf("\"samplers\": {\n");
        const double lams[] = {0.05, 0.7, 3.0, 9.5, 25.0, 140.0};
        printf("\"poisson\": [");
        for (int k = 0; k < 6; k++) {
            const int n = 100000;
            double s = 0, ss = 0;
            std::vector<int> hist(64, 0);
            for (int i = 0; i < n; i++) {
                int x = ignpoi_mt(lams[k], 0);
                s += x; ss += (double)x * x;
                int b = x - (int)lams[k] + 32;
                if (b >= 0 && b < 64) hist[b]++;
            }
            printf("%s{\"lambda\": %.17g, \"n\": %d, \"mean\": %.17g, \"var\": %.17g, \"offset\": %d, \"hist\": [", k ? ", " : "",
                   lams[k], n, s / n, ss / n - (s / n) * (s / n), (int)lams[k] - 32);
            for (int b = 0; b < 64; b++) printf("%s%d", b ? ", " : "", hist[b]);
            printf("]}");
        }
        printf("],\n");
        struct { int n; double p; } bins[] = {{25, 0.004}, {25, 0.3}, {230, 0.02}, {1000, 0.4}, {3300, 0.01}};
        printf("\"binomial\": [");
        for (int k = 0; k < 5; k++) {
            const int n = 100000;
            double s = 0, ss = 0;
            for (int i = 0; i < n; i++) {
                int x = ignbin_mt(bins[k].n, bins[k].p, 0);
                s += x; ss += (double)x * x;
            }
            printf("%s{\"trials\": %d, \"p\": %.17g, \"n\": %d, \"mean\": %.17g, \"var\": %.17g}", k ? ", " : "",
                   bins[k].n, bins[k].p, n, s / n, ss / n - (s / n) * (s / n));
        }
        printf("],\n");
        const double shapes[] = {0.5, 1.0, 4.0};
        printf("\"gamma\": [");
        for (int k = 0; k < 3; k++) {
            const int n = 100000;
            double s = 0, ss = 0;
            std::vector<int> hist(40, 0);
            for (int i = 0; i < n; i++) {
                double x = gen_gamma_mt(shapes[k], shapes[k], 0);
                s += x; ss += x * x;
                int b = (int)(x * 8);
                if (b < 40) hist[b]++;
            }
            printf("%s{\"shape\": %.17g, \"n\": %d, \"mean\": %.17g, \"var\": %.17g, \"hist\": [", k ? ", " : "", shapes[k], n,
                   s / n, ss / n - (s / n) * (s / n));
            for (int b = 0; b < 40; b++) printf("%s%d", b ? ", " : "", hist[b]);
            printf("]}");
        }
        printf("]\n},\n");
    }
    // ------------------------------- infectiousness / susceptibility products
    {
        const int N = 48, NH = 12, NM = 4;
        P.NumPlaceTypes = 4;
        P.TimeStepsPerDay = 4;
        P.Efficacies = new double*[6];
        for (int i = 0; i < 6; i++) {
            P.Efficacies[i] = new double[MAX_NUM_PLACE_TYPES + 2];
            for (int j = 0; j < MAX_NUM_PLACE_TYPES + 2; j++) P.Efficacies[i][j] = 0.1 + 0.13 * i + 0.07 * j;
        }
        P.WAIFW_Matrix = new double*[NUM_AGE_GROUPS];
        for (int i = 0; i < NUM_AGE_GROUPS; i++) {
            P.WAIFW_Matrix[i] = new double[NUM_AGE_GROUPS];
            for (int j = 0; j < NUM_AGE_GROUPS; j++) P.WAIFW_Matrix[i][j] = 0.5 + 0.5 * lcg_u(rs);
            P.AgeSusceptibility[i] = 0.6 + 0.4 * lcg_u(rs);
            P.RelativeSpatialContact[i] = 0.5 + 0.5 * lcg_u(rs);
            P.RelativeSpatialContactSusc[i] = 0.7 + 0.3 * lcg_u(rs);
        }
        for (int i = 0; i < MAX_HOUSEHOLD_SIZE; i++) P.HouseholdDenomLookup[i] = 1.0 / pow(1.0 + i, 0.8);
        for (int i = 0; i < 200; i++) P.infectiousness[i] = 0.2 + lcg_u(rs);
        for (int pt = 0; pt < MAX_NUM_PLACE_TYPES; pt++) {
            P.PlaceTypeTrans[pt] = 0.05 + 0.1 * lcg_u(rs);
            P.PlaceTypeGroupSizeParam1[pt] = 10 + pt * 15;
            P.SymptPlaceTypeContactRate[pt] = 0.25 + 0.5 * lcg_u(rs);
        }
        P.SymptSpatialContactRate = 0.5;
        P.SymptInfectiousness = 1.5;
        P.AsymptInfectiousness = 1.0;
        P.NoInfectiousnessSDinHH = 0;
        P.CareHomeResidentHouseholdScaling = 0.6;
        P.TreatInfDrop = P.VaccInfDrop = P.TreatSuscDrop = P.VaccSuscDrop = P.VaccSuscDrop2 = 1.0;
        P.usVaccTimeToEfficacy = 0;
        P.usCaseIsolationDelay = 4;
        P.usCaseIsolationDuration = 28;
        P.usHQuarantineHouseDuration = 56;
        Hosts = new Person[N]();
        Households = new Household[NH]();
        Mcells = new Microcell[NM]();
        HostsQuarantine.assign(N, PersonQuarantine());
        for (int h = 0; h < NH; h++) { Households[h].FirstPerson = 4 * h; Households[h].nh = 4; Households[h].nhr = 1 + h % 4; }
        for (int m = 0; m < NM; m++) Mcells[m].socdist = (m % 2) ? TreatStat::Treated : TreatStat::Untreated;
        const unsigned short ts = 100;
        std::vector<double> rows;
        for (int p = 0; p < N; p++) {
            Person& a = Hosts[p];
            a.hh = p / 4;
            a.mcell = (p / 3) % NM;
            a.age = (unsigned char)((p * 7) % 85);
            a.susc = (float)(0.3 + 0.7 * lcg_u(rs));
            a.infectiousness = (float)((p % 3 == 0 ? -1.0 : 1.0) * (0.2 + 2.0 * lcg_u(rs)));
            a.latent_time = (unsigned short)(ts - 1 - (p % 40));
            a.isolation_start_time = (p % 5 == 0) ? (unsigned short)(ts - 2 - (p % 7)) : (unsigned short)(USHRT_MAX - 1);
            a.treat_start_time = a.vacc_start_time = USHRT_MAX - 1;
            a.treat_stop_time = 0;
            a.care_home_resident = (p % 11 == 0);
            a.esocdist_comply = (p % 4 == 1);
            a.digitalContactTraced = 0;
            if (p % 6 == 0) a.set_case(); else if (p % 6 == 1) a.set_infectious_almost_symptomatic(); else a.set_susceptible();
            HostsQuarantine[p].comply = (uint8_t)(p % 3);
            HostsQuarantine[p].start_time = (p % 2) ? (unsigned short)(ts - 10) : (unsigned short)(USHRT_MAX - 1);
        }
        printf("\"calc\": {\"ts\": %d, \"n\": %d,\n", ts, N);
        std::vector<double> col(N);
        auto dump_people = [&]() {
            for (int p = 0; p < N; p++) col[p] = Hosts[p].hh; arr("hh", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].mcell; arr("mcell", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].age; arr("age", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].susc; arr("susc", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].infectiousness; arr("infectiousness", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].latent_time; arr("latent_time", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].isolation_start_time; arr("isolation_start_time", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].care_home_resident; arr("care_home", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].esocdist_comply; arr("esocdist", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = Hosts[p].is_case() ? -2 : (Hosts[p].is_infectious_almost_symptomatic() ? -1 : 0); arr("inf", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = HostsQuarantine[p].comply; arr("quar_comply", col.data(), N);
            for (int p = 0; p < N; p++) col[p] = HostsQuarantine[p].start_time; arr("quar_start", col.data(), N);
            for (int h = 0; h < NH; h++) col[h] = Households[h].nhr; arr("hh_nhr", col.data(), NH);
            for (int m = 0; m < NM; m++) col[m] = (Mcells[m].socdist == TreatStat::Treated) ? 2 : 0; arr("mcell_socdist", col.data(), NM);
        };
        dump_people();
        std::vector<double> e; for (int i = 0; i < 6; i++) for (int j = 0; j < MAX_NUM_PLACE_TYPES + 2; j++) e.push_back(P.Efficacies[i][j]);
        arr("efficacies", e.data(), (int)e.size());
        std::vector<double> w; for (int i = 0; i < NUM_AGE_GROUPS; i++) for (int j = 0; j < NUM_AGE_GROUPS; j++) w.push_back(P.WAIFW_Matrix[i][j]);
        arr("waifw", w.data(), (int)w.size());
        arr("age_susc", P.AgeSusceptibility, NUM_AGE_GROUPS);
        arr("rel_spatial", P.RelativeSpatialContact, NUM_AGE_GROUPS);
        arr("rel_spatial_susc", P.RelativeSpatialContactSusc, NUM_AGE_GROUPS);
        arr("hh_denom", P.HouseholdDenomLookup, MAX_HOUSEHOLD_SIZE);
        arr("infectiousness_profile", P.infectiousness, 200);
        arr("place_trans", P.PlaceTypeTrans, MAX_NUM_PLACE_TYPES);
        arr("group_size_param1", P.PlaceTypeGroupSizeParam1, MAX_NUM_PLACE_TYPES);
        arr("sympt_place_contact", P.SymptPlaceTypeContactRate, MAX_NUM_PLACE_TYPES);
        printf("\"care_home_hh_scaling\": %.17g, \"sympt_spatial\": %.17g, \"sympt_inf\": %.17g, \"asympt_inf\": %.17g,\n",
               P.CareHomeResidentHouseholdScaling, P.SymptSpatialContactRate, P.SymptInfectiousness, P.AsymptInfectiousness);
        printf("\"us_iso_delay\": %d, \"us_iso_dur\": %d, \"us_hq_dur\": %d,\n", P.usCaseIsolationDelay, P.usCaseIsolationDuration,
               P.usHQuarantineHouseDuration);
        std::vector<double> hi(N), si(N), pi(N * 4), hs(N), ss(N), ps(N * 4), pss(N);
        for (int p = 0; p < N; p++) {
            int q = (p * 5 + 3) % N;  // an infector for the two-person products
            hi[p] = CalcHouseInf(p, ts);
            si[p] = CalcSpatialInf(p, ts);
            for (int pt = 0; pt < 4; pt++) pi[p * 4 + pt] = CalcPlaceInf(p, pt, ts);
            hs[p] = CalcHouseSusc(p, ts, q);
            ss[p] = CalcSpatialSusc(p, ts);
            for (int pt = 0; pt < 4; pt++) ps[p * 4 + pt] = CalcPlaceSusc(p, pt, ts);
            pss[p] = CalcPersonSusc(p, ts, q);
        }
        arr("house_inf", hi.data(), N); arr("spatial_inf", si.data(), N); arr("place_inf", pi.data(), N * 4);
        arr("house_susc", hs.data(), N); arr("spatial_susc", ss.data(), N); arr("place_susc", ps.data(), N * 4);
        arr("person_susc", pss.data(), N, true);
        printf("}\n");
    }
    printf("}\n");
    return 0;
}
