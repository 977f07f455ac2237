/*
 * cs_oracle.h -- CPU oracle for the B200 sweep.  TEST INFRASTRUCTURE ONLY.
 *
 * A sequential C restatement of CovidSim's per-timestep sweep (src/Sweep.cpp:283-979,
 * src/Update.cpp:100-998, src/CalcInfSusc.cpp, src/Kernels.cpp, src/Dist.cpp,
 * src/InverseCdf.cpp, src/CovidSim.cpp:2752-2802) over the population layout of
 * include/covidsim_b200.h, drawing its random numbers from the same counter-based
 * streams as the GPU library so the two can be compared state for state.  Only the
 * tests, the smoke check and the CPU-baseline leg of bench.py call it; the product
 * never links it.
 *
 * Parity pins: the leaf arithmetic (kernel lookup, distances, inverse CDF, the
 * infectiousness/susceptibility products) is checked against values produced by the
 * reference's own functions (oracle/ref_pins.cpp -> tests/golden/ref_pins.json); the
 * whole-epidemic behaviour is checked statistically against runs of the reference
 * executable built by oracle/Makefile.
 */
#ifndef CS_ORACLE_H
#define CS_ORACLE_H

#include "covidsim_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cs_cpu_ctx cs_cpu_ctx;

int cs_cpu_create(const cs_population* pop, const cs_params* params, cs_cpu_ctx** out);
void cs_cpu_destroy(cs_cpu_ctx* ctx);
const char* cs_cpu_last_error(const cs_cpu_ctx* ctx);
int cs_cpu_set_params(cs_cpu_ctx* ctx, const cs_params* params);
int cs_cpu_begin_run(cs_cpu_ctx* ctx, uint64_t seed, const int32_t* seed_people, int n_seed,
                     int update_probs);
int cs_cpu_seed_infections(cs_cpu_ctx* ctx, double t, const int32_t* people, int n);
int cs_cpu_infect_sweep(cs_cpu_ctx* ctx, double t, int run);
int cs_cpu_incub_recovery_sweep(cs_cpu_ctx* ctx, double t);
int cs_cpu_update_probs(cs_cpu_ctx* ctx, int do_place);
int cs_cpu_step(cs_cpu_ctx* ctx, double t, int run);
int cs_cpu_set_interventions(cs_cpu_ctx* ctx, const cs_interventions* iv);
int cs_cpu_close_places(cs_cpu_ctx* ctx, int place_type, const int32_t* mcells, int n_mcells,
                        uint16_t start, uint16_t stop);
int cs_cpu_place_events(cs_cpu_ctx* ctx, const cs_place_event* events, int n);
int cs_cpu_set_mcell_status(cs_cpu_ctx* ctx, const int32_t* mcells, const uint8_t* socdist,
                            const uint8_t* moverest, int n);
int cs_cpu_download_state(cs_cpu_ctx* ctx, const cs_state_view* state);
int cs_cpu_get_counters(cs_cpu_ctx* ctx, cs_counters* out);

/* Leaf functions exposed for the pin tests. */
int cs_cpu_upload_state(cs_cpu_ctx* ctx, uint64_t seed, const cs_state_view* state);
double cs_cpu_calc(const cs_cpu_ctx* ctx, int kind, int p, int q, int pt, int ts);
int cs_cpu_sample_many(int kind, uint64_t seed, double a, double b, int n, double* out);
double cs_cpu_kernel_num(const cs_cpu_ctx* ctx, double r2);
/* The spatial proposal's bound(b, B) and its block geometry {bs, nbx, nby, tabulated}. */
double cs_cpu_block_bound(const cs_cpu_ctx* ctx, int b, int B);
void cs_cpu_block_geometry(const cs_cpu_ctx* ctx, int32_t* out);
/* KernelLookup::num over FP32 copies of the tables (the spatial acceptance test). */
double cs_cpu_kernel_num_f32(const float* lookup, const float* hi_res, int size, int expansion, double delta, double r2);
double cs_cpu_dist2_raw(const cs_params* p, double ax, double ay, double bx, double by);
double cs_cpu_dist2_cc_min(const cs_params* p, int grid_l, int grid_m);
uint16_t cs_cpu_icdf_choose(const cs_icdf* icdf, double mean, double u, double steps_per_day);
void cs_cpu_philox(uint32_t key0, uint32_t key1, const uint32_t ctr[4], uint32_t out[4]);
int cs_cpu_build_kernel_table(int kernel_type, double scale, double shape, double p3, double p4,
                              double longest_d2, int size, int expansion, double* lookup_out,
                              double* hi_res_out, double* delta_out);

int cs_cpu_get_cells16(cs_cpu_ctx* ctx, uint16_t* out);
size_t cs_cpu_sample_packed_bytes(const cs_cpu_ctx* ctx);

/* Population set-up, restated: the same results as cs_gpu_setup_run on the same
 * spec, array for array. */
typedef struct cs_cpu_setup cs_cpu_setup;
int cs_cpu_setup_run(const cs_setup_spec* spec, const cs_params* params, cs_cpu_setup** out);
int cs_cpu_setup_sizes(cs_cpu_setup* setup, cs_setup_out* sizes);
int cs_cpu_setup_download(cs_cpu_setup* setup, const cs_setup_out* dst);
const char* cs_cpu_setup_last_error(const cs_cpu_setup* setup);
void cs_cpu_setup_destroy(cs_cpu_setup* setup);

#ifdef __cplusplus
}
#endif
#endif
