/*
 * cs_oracle_as_gpu_abi.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The subset of the cs_gpu_* entry points that the drop-in shim
 * (covid-sim_b200/shim/cs_sweep_shim.cpp) calls, implemented by the CPU oracle.
 * Linking the shim against this file instead of the GPU library gives a reference
 * executable whose sweeps are the oracle's (oracle/_ref/CovidSim_oracle), so the
 * oracle's whole-epidemic behaviour can be compared with the reference's own on
 * the CPU.
 */
#include <stdlib.h>
#include <string.h>

#include "cs_oracle.h"

struct cs_gpu_ctx;

int cs_build_kernel_table(int kernel_type, double scale, double shape, double p3, double p4, double longest_d2, int size,
                          int expansion, double* lookup_out, double* hi_res_out, double* delta_out)
{
    return cs_cpu_build_kernel_table(kernel_type, scale, shape, p3, p4, longest_d2, size, expansion, lookup_out,
                                     hi_res_out, delta_out);
}

int cs_gpu_create(const cs_population* pop, const cs_params* params, int device, cs_gpu_ctx** out)
{
    (void)device;
    return cs_cpu_create(pop, params, (cs_cpu_ctx**)out);
}

const char* cs_gpu_last_error(const cs_gpu_ctx* c) { return cs_cpu_last_error((const cs_cpu_ctx*)c); }
int cs_gpu_set_params(cs_gpu_ctx* c, const cs_params* p) { return cs_cpu_set_params((cs_cpu_ctx*)c, p); }
int cs_gpu_upload_state(cs_gpu_ctx* c, uint64_t seed, const cs_state_view* v) { return cs_cpu_upload_state((cs_cpu_ctx*)c, seed, v); }
int cs_gpu_update_probs(cs_gpu_ctx* c, int do_place) { return cs_cpu_update_probs((cs_cpu_ctx*)c, do_place); }
int cs_gpu_infect_sweep(cs_gpu_ctx* c, double t, int run) { return cs_cpu_infect_sweep((cs_cpu_ctx*)c, t, run); }
int cs_gpu_incub_recovery_sweep(cs_gpu_ctx* c, double t) { return cs_cpu_incub_recovery_sweep((cs_cpu_ctx*)c, t); }
int cs_gpu_step(cs_gpu_ctx* c, double t, int run)
{
    int r = cs_cpu_infect_sweep((cs_cpu_ctx*)c, t, run);
    return r ? r : cs_cpu_incub_recovery_sweep((cs_cpu_ctx*)c, t);
}
int cs_gpu_sync(cs_gpu_ctx* c) { (void)c; return 0; }
int cs_gpu_get_counters(cs_gpu_ctx* c, cs_counters* out) { return cs_cpu_get_counters((cs_cpu_ctx*)c, out); }
int cs_gpu_set_interventions(cs_gpu_ctx* c, const cs_interventions* iv) { return cs_cpu_set_interventions((cs_cpu_ctx*)c, iv); }
int cs_gpu_place_events(cs_gpu_ctx* c, const cs_place_event* ev, int n) { return cs_cpu_place_events((cs_cpu_ctx*)c, ev, n); }
int cs_gpu_set_mcell_status(cs_gpu_ctx* c, const int32_t* m, const uint8_t* sd, const uint8_t* mr, int n)
{
    return cs_cpu_set_mcell_status((cs_cpu_ctx*)c, m, sd, mr, n);
}

int cs_gpu_get_cell_counts(cs_gpu_ctx* c, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D)
{
    cs_state_view v;
    memset(&v, 0, sizeof(v));
    v.cell_S = S; v.cell_L = L; v.cell_I = I; v.cell_R = R; v.cell_D = D;
    return cs_cpu_download_state((cs_cpu_ctx*)c, &v);
}

int cs_gpu_get_sample(cs_gpu_ctx* c, int32_t* S, int32_t* L, int32_t* I, int32_t* R, int32_t* D, cs_counters* out)
{
    int r = cs_gpu_get_cell_counts(c, S, L, I, R, D);
    return r ? r : cs_cpu_get_counters((cs_cpu_ctx*)c, out);
}

void* cs_host_alloc(size_t bytes) { return malloc(bytes ? bytes : 1); }
void cs_host_free(void* p) { free(p); }

int cs_gpu_get_sample16(cs_gpu_ctx* c, uint16_t* cells, cs_counters* out)
{
    int r = cs_cpu_get_cells16((cs_cpu_ctx*)c, cells);
    return r ? r : cs_cpu_get_counters((cs_cpu_ctx*)c, out);
}

size_t cs_gpu_sample_packed_bytes(const cs_gpu_ctx* c) { return cs_cpu_sample_packed_bytes((const cs_cpu_ctx*)c); }
int cs_gpu_get_sample_packed(cs_gpu_ctx* c, void* buf, size_t bytes)
{
    if (bytes < cs_cpu_sample_packed_bytes((const cs_cpu_ctx*)c)) return CS_E_ARG;
    cs_counters* k = (cs_counters*)buf;
    int r = cs_cpu_get_counters((cs_cpu_ctx*)c, k);
    if (r) return r;
    k->S = k->L = k->I = k->R = k->D = 0;
    return cs_cpu_get_cells16((cs_cpu_ctx*)c, (uint16_t*)((char*)buf + sizeof(cs_counters)));
}
int cs_gpu_sample_packed_begin(cs_gpu_ctx* c, void* buf, size_t bytes) { return cs_gpu_get_sample_packed(c, buf, bytes); }
int cs_gpu_sample_packed_end(cs_gpu_ctx* c, const void* buf) { (void)c; (void)buf; return CS_OK; }
/* The oracle reads the whole view in cs_gpu_upload_state: slices sent ahead need no work. */
int cs_gpu_upload_people(cs_gpu_ctx* c, const cs_state_view* v, int64_t first, int64_t n)
{
    (void)c; (void)v; (void)first; (void)n;
    return CS_OK;
}
