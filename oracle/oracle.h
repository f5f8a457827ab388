/*
 * oracle.h — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * C interface of the CPU oracle: a restatement of the reference's CPU engine
 * (js/fisica-cpu.js, js/pressao-cpu.js, js/ar.js, js/cena.js, js/constantes.js) used only by
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as the checker.
 *
 * The simulation entry points mirror include/tanque.h one to one with a `tqo_` prefix, so a
 * test drives the oracle and the CUDA library through the same calls.  The oracle takes two
 * extra options through tq_options: p2g_mode (TQ_P2G_FLOAT = the reference CPU's float sums,
 * TQ_P2G_FIXED = the integer sums the CUDA library uses) and, through tqo_create_fp64, an
 * all-double storage variant (the FP64 oracle).
 */
#ifndef TANQUE_ORACLE_H
#define TANQUE_ORACLE_H

#include "../include/tanque.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- scene (js/cena.js) */
typedef struct tqo_scene tqo_scene;
tqo_scene* tqo_scene_new(int32_t nx, int32_t ny, double h);
void tqo_scene_free(tqo_scene* c);
void tqo_scene_trace(tqo_scene* c, double x0, double y0, double x1, double y1, double radius,
                     int32_t erase);
void tqo_scene_clear(tqo_scene* c);
const float* tqo_scene_sdf(tqo_scene* c);
double tqo_scene_distance(tqo_scene* c, double x, double y);
void tqo_scene_normal(tqo_scene* c, double x, double y, double* nx, double* ny);
int32_t tqo_scene_solid_cell(tqo_scene* c, int32_t i, int32_t j);

/* ---- constants and helpers (js/constantes.js, testes/apoio.js, js/fisica-cpu.js:705-727) */
double tqo_passo_maximo(double h, double altura, double vmax, int32_t has_vmax, double dt_frame);
void tqo_dimensoes(double largura, double altura, int32_t celulas, double h_min, int32_t* nx,
                   int32_t* ny, double* h);
/* semearRetangulo with the seeded LCG of testes/apoio.js:4-9; *seed is advanced.  Returns
 * the particle count; `out` (may be null to query) receives 12 floats per particle. */
int32_t tqo_semear_retangulo(double x0, double y0, double x1, double y1, double h,
                             const double* absorb, uint32_t* seed, float* out, int32_t cap);

/* ---- simulation (SimulacaoCPU), same semantics as include/tanque.h */
typedef struct tqo_sim tqo_sim;
int tqo_create(const tq_options* o, tqo_sim** out);
int tqo_create_fp64(const tq_options* o, tqo_sim** out);
int tqo_destroy(tqo_sim* s);
int tqo_set_walls(tqo_sim* s, const float* sdf, int32_t mw, int32_t mh);
int tqo_add_particles(tqo_sim* s, const float* list, int32_t n, int32_t check_full,
                      int32_t* accepted);
int tqo_clear_particles(tqo_sim* s);
int tqo_apply_tool(tqo_sim* s, const tq_tool* tool);
int tqo_advance(tqo_sim* s, double dt, int32_t substeps);
int tqo_substep(tqo_sim* s, double dt);
int tqo_update_air(tqo_sim* s);
int tqo_reset_air(tqo_sim* s);
int tqo_count(tqo_sim* s, int32_t* n);
int tqo_get_particles(tqo_sim* s, float* out, int32_t cap, int32_t* n);
int tqo_set_particles(tqo_sim* s, const float* list, int32_t n);
int tqo_get_field(tqo_sim* s, int32_t field, void* out, int64_t bytes);
int tqo_set_field(tqo_sim* s, int32_t field, const void* in, int64_t bytes);
int tqo_get_scalar(tqo_sim* s, int32_t which, double* out);
int tqo_set_scalar(tqo_sim* s, int32_t which, double value);
int tqo_last_norms(tqo_sim* s, double* out, int32_t cap, int32_t* n);

/* ---- standalone solver (js/pressao-cpu.js exports) */
int tqo_solve_pressure(int32_t nx, int32_t ny, const uint8_t* tipo, const float* div, float* q,
                       int32_t iterations, double tolerance, const tq_bubbles* bubbles,
                       int32_t preconditioner, double* norms, int32_t norms_cap, int32_t* n_norms,
                       tq_solve_info* info);
int tqo_vcycle(int32_t nx, int32_t ny, const uint8_t* tipo, const float* b, float* x);

/* ---- the FP64 CPU adjoint (adjunto_oracle.cpp), the checker of tq_adj_*.  record = 1 records
 * the discrete structure of the run; record = 0 reuses the last recorded one (frozen), so central
 * finite differences see the same smooth map as the adjoint.  Velocities in double. */
typedef struct tqo_adj tqo_adj;
int tqo_adj_create(const tq_adj_scene* scene, tqo_adj** out);
int tqo_adj_destroy(tqo_adj* a);
int tqo_adj_forward(tqo_adj* a, const double* v0, const double* theta, int32_t record, double* loss);
int tqo_adj_backward(tqo_adj* a, double* dv0, double* dtheta);
int tqo_adj_count(tqo_adj* a, int32_t* n);

const char* tqo_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
