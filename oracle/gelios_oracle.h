/* Test infrastructure only: the CPU restatement of the Gelios_2D plasma time
 * step used as the checker for the CUDA path.  Never linked by the product.
 *
 * Parity of this restatement is pinned against the reference itself
 * (oracle/_ref/libgelios_ref.so, compiled from the unmodified reference
 * sources): with the reference's compile-time constants as parameters it
 * reproduces Go_stationary, Go_5_komponent__MK2 and
 * Go_stationary_5_komponent_inner_MK2 bit for bit (tests/test_oracle_pin.py).
 */
#ifndef GELIOS_ORACLE_H
#define GELIOS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same field order as gelios_params in include/gelios_b200.h. */
typedef struct go_params {
    double gamma;          /* ga / ggg, Help.h:39-40 */
    double kurant;         /* Help.h:57 */
    double chi;            /* chi_real, Help.h:56: inner-sphere wind speed */
    double inner_mach;     /* 10.0 in Gran.cpp:241 */
    double in_ro, in_p, in_u, in_v, in_Q; /* Input BC, Gran.cpp:279-281 */
    double extern_u_par;   /* -0.1, Gran.cpp:216-219 */
    double extern_u_tvd;   /* -0.01, Gran.cpp:477-480 */
    double R11;            /* MK2 skip radius, Setka.cpp:10169 */
    double rad_stat;       /* 95, Setka.cpp:5256 */
    double R1, R111, R5, Left; /* rail geometry, Help.h:79-89 */
    double koef;           /* Move_surface damping, Setka.cpp:3380 */
    double src_rmin, src_rmax; /* Cell.cpp:528 */
    double src_coef;       /* n_p_LISM_/Kn_, Cell.cpp:648 */
    double a_2;            /* sigma(U) coefficient, Help.h:64 */
    double ro_floor, p_floor; /* Setka.cpp:10435, 10452 */
    double dt0;            /* 1e-8, Setka.cpp:10129 */
    int32_t n_inner;       /* Help.h:71 */
    int32_t n_outer_shock; /* Help.h:72 */
    int32_t godunov_max_iter; /* 1100, Solvers.cpp:1206 */
    int32_t pad_;
} go_params;

typedef struct go_mesh {
    int32_t dims[8]; /* N1..M4 of Setka(N1..M4) (zeros without rails) */
    int32_t n_points;
    const double *x, *y;
    const int32_t *point_type;
    int32_t n_cells;
    const int32_t *cell_type, *contour_start, *contour, *gran_start, *gran;
    const int32_t *cell_back, *cell_next;
    const double *r_istoch;
    int32_t n_faces, n_main;
    const int32_t *face_A, *face_B, *face_type, *face_master, *face_sosed, *face_copy;
    const int32_t *face_sosed_up, *face_sosed_down;
    int32_t n_rails;
    const int32_t *rail_type;
    const double *rail_s;
    const int32_t *rail_M, *rail_pstart, *rail_points, *rail_kstart, *rail_keys;
    int32_t n_contact, n_inner_line, n_outer_line;
    const int32_t *line_contact, *line_inner, *line_outer;
} go_mesh;

void *go_create(const go_params *prm, const go_mesh *mesh);
void go_destroy(void *h);
/* hydrogen fluids of par[buf] (Go_5_komponent): rows16 = ro, p, u, v of H1..H4 */
void go_set_hydrogen(void *h, int buf, const double *rows16);
void go_get_hydrogen(void *h, int buf, double *rows16);
void go_5_komponent(void *h, int step);
void go_move_setka1(void *h, double dt);
void go_set_state(void *h, int buf, const double *ro, const double *p, const double *u, const double *v,
                  const double *Q);
void go_get_state(void *h, int buf, double *ro, double *p, double *u, double *v, double *Q);
/* Monte-Carlo moments: Hn/Hu/Hv/HT [cell*4 + k], ku/kv/kT [cell] */
void go_set_mc(void *h, const double *Hn, const double *Hu, const double *Hv, const double *HT,
               const double *ku, const double *kv, const double *kT);
void go_set_inner_list(void *h, const int32_t *cells, int32_t n);
void go_get_points(void *h, double *x, double *y, double *x2, double *y2, double *Vx, double *Vy,
                   int32_t *count);
/* status: bit0 Newton/bisection cap hit, bit1 non-positive TVD state, bit2
 * negative Newton pressure; counters of clamps */
void go_status(void *h, int64_t *out4);
/* Time loops; each call restarts dt at dt0 like the reference. */
void go_stationary(void *h, int steps);
void go_mk2(void *h, int steps);
void go_inner_mk2(void *h, int steps);
/* phases (for phase-level parity) */
void go_move_surface(void *h, int ii, double dt);
void go_move_setka2(void *h, double dt);
void go_commit_points(void *h);
double go_last_dt(void *h);

/* MHD + pickup-proton moving-grid step (no reference step exists; this is
 * the project's own restatement, written per cell and per face from each
 * side like the reference's loops, as the checker of the device's
 * once-per-face units).  Same field order as gelios_mhd_params. */
typedef struct go_mhd_params {
    double lism_bx, lism_by, lism_bz, inner_bphi, pui_in_ro, pui_in_p, pui_inner_ro, pui_inner_p;
} go_mhd_params;
/* extra rows of par[buf]: w, Bx, By, Bz, ro_pui, p_pui, u_pui, v_pui */
void go_set_mhd(void *h, int buf, const double *rows8);
void go_get_mhd(void *h, int buf, double *rows8);
void go_set_sources(void *h, const double *q1, const double *q2, const double *q3);
void go_mhd(void *h, const go_mhd_params *mp, int steps);

/* per-face kernels */
double go_hllc(const go_params *prm, const double *L5, const double *R5, double W, double *P4, double *PQ,
               double n1, double n2, double rad, int metod, double *VlVcVp, int nul_potok);
double go_godunov(const go_params *prm, const double *q1, const double *q2, const double *n3, double *q5,
                  double *dsl_dsp_dsc, double w, double dist, int *status);
double go_hlldq(const go_params *prm, const double *L9, const double *R9, double *P8, double *PQ, const double *n3,
                double rad, int metod);
double go_hlld(const go_params *prm, const double *q1, const double *q2, const double *n3, double *q8,
               double *dsl_dsp_dsc, double w, double dist, int *status);
void go_face_par(void *h, int f, int which, int buf, double *out5);
void go_cell_geom(void *h, int c, double *out8);
void go_source_mk1(void *h, int c, double u, double v, double ro, double p, double *q3);

#ifdef __cplusplus
}
#endif
#endif
