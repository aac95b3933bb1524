/*
 * lbm_oracle.h — CPU oracle for the double-distribution (DDF) lattice Boltzmann
 * Rayleigh–Bénard time step of Summer536/LBM_DDF (single-GPU src/ path).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load
 * it.  The product path (lbm_ddf_b200, liblbm_ddf.so) never calls it and has no
 * CPU fallback.
 *
 * It restates, in plain C, FP64, the reference's per-step algorithm in the
 * reference's own operation order and storage layout:
 *   idx = (iz*LY + iy)*LX + ix, population ip stored at ip*N + idx   (src/rb3d.h, src/streaming.cu:9)
 *   vertical axis y: hot plate at iy = 0, cold plate at iy = LY-1       (src/streaming.cu:205,217)
 * and adds one mode the reference cannot run: periodic x and z sides.
 *
 * Parity pin: outputs of the reference binary itself (src/ rebuilt for sm_100a
 * by oracle/Makefile into oracle/_ref/, run through its restart path on seeded
 * states) are stored as fixtures under tests/golden/ and checked by
 * tests/test_oracle_golden.py.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_Q 27

/* Type of the populations, macroscopic fields and step arithmetic: double
 * (the reference's FP64; this build is pinned bitwise to its outputs), or
 * float when built with -DORC_REAL=float (liblbm_oracle_f32.so: the same
 * transcription in FP32, a CPU baseline only). */
#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL orc_real;

typedef struct orc_params {
    int32_t lx, ly, lz;          /* LX, LY, LZ of src/parameters.h:8-10 */
    int32_t periodic_sides;      /* 0 = closed box (reference), 1 = x and z periodic */
    double rayleigh, prandtl;    /* RAYLEIGH, PRANDTL        src/parameters.h:21-22 */
    double t_hot, t_cold;        /* T_HOT, T_COLD            src/parameters.h:23-24 */
    double gravity, beta;        /* GRAVITY, BETA            src/parameters.h:25-26 */
    /* derived by orc_derive (src/globals.cu:13-23) */
    double visc, tau, u0, diff, tauc, t0;
} orc_params;

typedef struct orc_state orc_state;

/* Derived parameters, src/globals.cu:13-23. Returns 0, or -1 on a bad grid. */
int orc_derive(orc_params *p);

/* Allocates the reference's 4x27 + 8 fields (src/initial.cu:5-18). */
orc_state *orc_create(const orc_params *p);
void orc_destroy(orc_state *s);
const orc_params *orc_get_params(const orc_state *s);
int64_t orc_nodes(const orc_state *s);

/* Field pointers (reference layout, length N or 27*N). which: 0 f, 1 g,
 * 2 rho, 3 ux, 4 uy, 5 uz, 6 phi, 7 force_x, 8 force_y, 9 force_z. */
orc_real *orc_field(orc_state *s, int which);

/* Rest state of init_arrays, src/initial.cu:208-241. */
void orc_init_rest(orc_state *s);

/* Seeded conduction state.  phi(node) = T_hot - (T_hot-T_cold)*iy/(LY-1.0)
 * (Parallel/initial.cu:89) + amplitude*(2u-1), u from orc_noise_uniform;
 * f = 0 (equilibrium of rho=0, u=0), g_i = w_i*phi, and the carried previous
 * temperature phi_prev = phi.  Stores rho, u, phi as macrovar would have them
 * (see orc_set_populations). */
void orc_init_conduction(orc_state *s, uint64_t seed, double amplitude);

/* Counter-based uniform draw in [0,1) for node `node` of a case seeded `seed`:
 * splitmix64(splitmix64(seed) + node) >> 11, times 2^-53. */
double orc_noise_uniform(uint64_t seed, uint64_t node);

/* Sets f and g (27*N each, reference layout) and derives the macroscopic
 * fields exactly as src/macrovar.cu:3-34 and the force as src/macrovar.cu:36-47
 * would leave them after a step whose force was built from phi_prev:
 *   F_y = g*beta*(phi_prev - t0), rho = sum f, u = sum c f + F/2, phi = sum g.
 * phi_prev == NULL means phi_prev = t0 (zero force). */
void orc_set_populations(orc_state *s, const orc_real *f, const orc_real *g,
                         const orc_real *phi_prev);

/* Restart path (src/initial.cu:110-205): copies rho, ux, uy, uz, phi, f, g
 * verbatim and then runs `forcing` (src/initial.cu:202). */
void orc_load_restart(orc_state *s, const orc_real *rho, const orc_real *ux,
                      const orc_real *uy, const orc_real *uz, const orc_real *phi,
                      const orc_real *f, const orc_real *g);

/* nsteps time steps of src/main.cu:27-46:
 * forcing -> collision_BGK -> collision_BGK_scalar -> streaming (+copy)
 * -> streaming_scalar (+copy) -> macrovar.  OpenMP over z-planes. */
void orc_step(orc_state *s, int nsteps);

/* Observables of the stored macroscopic fields.
 * out[0] Nu_bulk, out[1] Nu_top, out[2] Nu_bottom   (src/output.cu:199-256)
 * out[3] KE = 0.5*<ux^2+uy^2+uz^2>, out[4] Re = sqrt(<|u|^2>)*LY/visc
 * out[5..8] means of ux, uy, uz, phi                 (src/output.cu:24-34)
 * out[9] 1.0 if any stored field is NaN/Inf else 0.0 */
void orc_observables(const orc_state *s, double out[10]);

/* Vertical profile, src/output.cu:336-368: for each iy, 5 values
 * <ux>, <uy>, <uz>, <phi>, phi_rms, written to out[5*iy + k]. */
void orc_profile(const orc_state *s, double *out);

/* Collision model: ORC_COLLISION_BGK (default) is the reference's; the
 * regularised BGK of Latt and Chopard (2006) is an engine option the
 * reference does not have (see lbm_oracle.c k_collide_f_reg). */
#define ORC_COLLISION_BGK 0
#define ORC_COLLISION_REGULARIZED 1
void orc_set_collision(orc_state *s, int model);
int orc_get_collision(const orc_state *s);

/* Contraction model (see lbm_oracle.c): 1 = round as the nvcc-built
 * reference does (default), 0 = every operation rounded separately. */
void orc_set_contract(int on);
int orc_get_contract(void);

/* Number of OpenMP threads the step uses (1 when built without OpenMP). */
int orc_threads(void);

#ifdef __cplusplus
}
#endif

#endif
