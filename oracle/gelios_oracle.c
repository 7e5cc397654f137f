/* Test infrastructure only (never linked by the product): CPU restatement of
 * the Gelios_2D plasma time step, used as the checker of the CUDA path.
 *
 * Every function states the reference lines it follows (paths within the
 * SergeyMSU/Gelios_2D tree).  Operation order follows the reference so that,
 * built without FMA contraction and given the reference's compile-time
 * constants as parameters, results agree with the compiled reference bit for
 * bit.  Data are structure-of-arrays indexed by the unified numbering of the
 * mesh (cells in All_Cells order, faces = All_Gran then All_Gran_copy).
 *
 * Where the reference calls exit(-1) (Newton/bisection caps, non-positive
 * TVD states) this restatement raises a status bit and carries on.
 */
#include "gelios_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_ 3.14159265358979323846
#define kv(x) ((x) * (x))

enum { T_USUALY = 0, T_INNER_SPHERE, T_EXTERN, T_INPUT, T_AXIS, T_UPPER_WALL };
enum { C_1 = 0, C_2, C_3, C_4, C_5, C_CENTR };
enum { P_CONTACT = 6, P_INNER_SHOCK = 7, P_OUTER_SHOCK = 8 };
enum { R_A = 0, R_B, R_C, R_D };

typedef struct {
    double ro, p, u, v, Q;
} st5;

typedef struct ctx {
    go_params prm;
    go_mesh m;
    /* owned copies of mutable geometry */
    double *x, *y, *x2, *y2, *Vx, *Vy;
    int32_t *count;
    /* state par[2], 5 fields each */
    double *par[2][5];
    /* hydrogen fluids of par[2]: ro, p, u, v of H1..H4 (Go_5_komponent) */
    double *hpar[2][16];
    /* MC moments */
    double *Hn, *Hu, *Hv, *HT, *ku, *kv_, *kT;
    /* fixed charge-exchange sources of the MHD form (ion momentum x, y, energy) */
    double *qfix[3];
    int32_t *inner;
    int32_t n_inner_cells;
    int64_t status, n_ro_clamp, n_p_clamp, n_tvd_bad;
    double last_dt;
} ctx;

/* ------------------------------------------------------------------ helpers */
static double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */

/* sign, minmod: Help.cpp:67-94 */
static double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
static double minmod(double x, double y) {
    if (sgn(x) + sgn(y) == 0) return 0.0;
    return ((sgn(x) + sgn(y)) / 2.0) * dmin(fabs(x), fabs(y));
}
/* linear, 3-point minmod: Help.cpp:96-113 */
static double linear3(double x1, double t1, double x2, double t2, double x3, double t3, double y) {
    double d = minmod((t1 - t2) / (x1 - x2), (t2 - t3) / (x2 - x3));
    return (d * (y - x2) + t2);
}
/* linear, 2-point: Help.cpp:115-120 */
static double linear2(double x1, double t1, double x2, double t2, double y) {
    double d = (t1 - t2) / (x1 - x2);
    return (d * (y - x2) + t2);
}
/* polar_angle: Help.cpp:37-65 (RR_ in the threshold is the geometry scale) */
static double polar_angle(double x, double y, double tiny) {
    if (fabs(x) + fabs(y) < tiny) return 0.0;
    if (x < 0) return atan(y / x) + 1.0 * PI_;
    else if (x > 0 && y >= 0) return atan(y / x);
    else if (x > 0 && y < 0) return atan(y / x) + 2.0 * PI_;
    else if (y > 0 && x >= 0 && x <= 0) return PI_ / 2.0;
    else if (y < 0 && x >= 0 && x <= 0) return 3.0 * PI_ / 2.0;
    return 0.0;
}
/* polar_perenos: Help.cpp:3-14 */
static void polar_perenos(double x1, double y1, double x2, double y2, double *u, double *v, double tiny) {
    double phi1 = polar_angle(x1, y1, tiny);
    double phi2 = polar_angle(x2, y2, tiny);
    double fr = *u * cos(phi1) + *v * sin(phi1);
    double ff = -*u * sin(phi1) + *v * cos(phi1);
    *u = fr * cos(phi2) - ff * sin(phi2);
    *v = fr * sin(phi2) + ff * cos(phi2);
}
/* the polar_angle threshold is 0.000001/RR_ (Help.cpp:39); RR_ = 390.222 */
#define TINY_ANGLE (0.000001 / 390.222)

/* ------------------------------------------------------------------ geometry */
/* Cell::Get_Center / Get_Center_posle: Cell.cpp:66-111 */
static void cell_center(const ctx *c, int k, int posle, double *ox, double *oy) {
    const double *X = posle ? c->x2 : c->x, *Y = posle ? c->y2 : c->y;
    int s = c->m.contour_start[k], e = c->m.contour_start[k + 1], n = e - s;
    double A = 0.0, Gx = 0.0, Gy = 0.0;
    for (int i = 0; i < n; i++) {
        int a = c->m.contour[s + i];
        int j = i + 1;
        if (j == n) j = 0;
        int b = c->m.contour[s + j];
        A = A + (X[a] * Y[b] - Y[a] * X[b]);
        Gx = Gx + (X[a] + X[b]) * (X[a] * Y[b] - Y[a] * X[b]);
        Gy = Gy + (Y[a] + Y[b]) * (X[a] * Y[b] - Y[a] * X[b]);
    }
    A = A * 0.5;
    Gx = Gx / (6.0 * A);
    Gy = Gy / (6.0 * A);
    *ox = Gx;
    *oy = Gy;
}
/* Cell::Get_Volume / Get_Volume_posle: Cell.cpp:146-254 */
static double cell_volume(const ctx *c, int k, int posle) {
    const double *X = posle ? c->x2 : c->x, *Y = posle ? c->y2 : c->y;
    int s = c->m.contour_start[k], n = c->m.contour_start[k + 1] - s;
    const int32_t *ct = c->m.contour + s;
    if (n == 4) {
        double a1 = X[ct[0]] - X[ct[2]];
        double a2 = Y[ct[0]] - Y[ct[2]];
        double a = sqrt(kv(a1) + kv(a2));
        double b1 = X[ct[1]] - X[ct[3]];
        double b2 = Y[ct[1]] - Y[ct[3]];
        double b = sqrt(kv(b1) + kv(b2));
        a1 = a1 / a;
        a2 = a2 / a;
        b1 = b1 / b;
        b2 = b2 / b;
        double cc = a1 * b1 + a2 * b2;
        double sn = sqrt(1 - kv(cc));
        return 0.5 * a * b * sn;
    }
    double x = 0.0, y = 0.0;
    if (!posle) {
        cell_center(c, k, 0, &x, &y);
    } else {
        for (int i = 0; i < n; i++) {
            x += X[ct[i]];
            y += Y[ct[i]];
        }
        x = x / (1.0 * n);
        y = y / (1.0 * n);
    }
    double S = 0.0;
    for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
        int f = c->m.gran[g];
        int pa = c->m.face_A[f], pb = c->m.face_B[f];
        double a1 = sqrt(kv(X[pa] - x) + kv(Y[pa] - y));
        double a2 = sqrt(kv(X[pb] - x) + kv(Y[pb] - y));
        double a3 = sqrt(kv(X[pa] - X[pb]) + kv(Y[pa] - Y[pb]));
        double p = (a1 + a2 + a3) / 2.0;
        S = S + sqrt(p * (p - a1) * (p - a2) * (p - a3));
    }
    return S;
}
/* Cell::Get_Volume_rotate / Get_Volume_posle_rotate: Cell.cpp:188-206, 256-275 */
static double cell_volume_rotate(const ctx *c, int k, int posle, double angle) {
    const double *X = posle ? c->x2 : c->x, *Y = posle ? c->y2 : c->y;
    int s = c->m.contour_start[k], n = c->m.contour_start[k + 1] - s;
    double A = 0.0, G = 0.0;
    for (int i = 0; i < n; i++) {
        int a = c->m.contour[s + i];
        int j = i + 1;
        if (j == n) j = 0;
        int b = c->m.contour[s + j];
        A = A + (X[a] * Y[b] - Y[a] * X[b]);
        G = G + (Y[a] + Y[b]) * (X[a] * Y[b] - Y[a] * X[b]);
    }
    A = A * 0.5;
    return fabs(A) * (1.0 / (6.0 * A)) * G * PI_ * angle / 180.0;
}
/* Gran::Get_Center(_posle), Get_normal, Get_square: Gran.cpp:159-198 */
static void face_center(const ctx *c, int f, int posle, double *ox, double *oy) {
    const double *X = posle ? c->x2 : c->x, *Y = posle ? c->y2 : c->y;
    int a = c->m.face_A[f], b = c->m.face_B[f];
    *ox = (X[a] + X[b]) / 2.0;
    *oy = (Y[a] + Y[b]) / 2.0;
}
static void face_normal(const ctx *c, int f, double *n1, double *n2) {
    int a = c->m.face_A[f], b = c->m.face_B[f];
    double t1 = c->x[b] - c->x[a];
    double t2 = c->y[b] - c->y[a];
    double n = sqrt(kv(t1) + kv(t2));
    t1 = t1 / n;
    t2 = t2 / n;
    *n1 = t2;
    *n2 = -t1;
}
static double face_square(const ctx *c, int f) {
    int a = c->m.face_A[f], b = c->m.face_B[f];
    return sqrt(kv(c->x[b] - c->x[a]) + kv(c->y[b] - c->y[a]));
}

static st5 cell_state(const ctx *c, int k, int buf) {
    st5 s;
    s.ro = c->par[buf][0][k];
    s.p = c->par[buf][1][k];
    s.u = c->par[buf][2][k];
    s.v = c->par[buf][3][k];
    s.Q = c->par[buf][4][k];
    return s;
}

static int cell_has_axis(const ctx *c, int k) {
    for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++)
        if (c->m.face_type[c->m.gran[g]] == T_AXIS) return 1;
    return 0;
}

/* ------------------------------------------------------------------ boundary / reconstruction */
/* Inner_sphere BC state: Gran.cpp:234-265 (Get_par) and 520-534 (Get_par_TVD) */
static st5 inner_sphere_state(const ctx *c, int f) {
    const go_params *P = &c->prm;
    double x, y;
    face_center(c, f, 0, &x, &y);
    double dist = sqrt(x * x + y * y);
    double ro = 1.0 / (kv(P->chi) * dist * dist);
    double P_E = ro * P->chi * P->chi / (P->gamma * P->inner_mach * P->inner_mach);
    st5 s = {ro, P_E, P->chi * x / dist, P->chi * y / dist, ro};
    return s;
}
static st5 input_state(const ctx *c) {
    st5 s = {c->prm.in_ro, c->prm.in_p, c->prm.in_u, c->prm.in_v, c->prm.in_Q};
    return s;
}

/* Gran::Get_par: Gran.cpp:205-289 */
static st5 get_par(const ctx *c, int f, int buf) {
    int t = c->m.face_type[f];
    st5 s = {0, 0, 0, 0, 0};
    if (t == T_USUALY) {
        s = cell_state(c, c->m.face_sosed[f], buf);
    } else if (t == T_EXTERN) {
        s = cell_state(c, c->m.face_master[f], buf);
        if (s.u >= 0.0) s.u = c->prm.extern_u_par;
    } else if (t == T_UPPER_WALL) {
        s = cell_state(c, c->m.face_master[f], buf);
    } else if (t == T_AXIS) {
        s = cell_state(c, c->m.face_master[f], buf);
        s.v = -s.v;
    } else if (t == T_INNER_SPHERE) {
        s = inner_sphere_state(c, f);
    } else if (t == T_INPUT) {
        s = input_state(c);
    }
    return s;
}

static int is_tracked_face(const ctx *c, int f) {
    int ta = c->m.point_type[c->m.face_A[f]], tb = c->m.point_type[c->m.face_B[f]];
    return (ta == P_CONTACT && tb == P_CONTACT) || (ta == P_INNER_SHOCK && tb == P_INNER_SHOCK) ||
           (ta == P_OUTER_SHOCK && tb == P_OUTER_SHOCK);
}

/* Gran::Get_par_TVD: Gran.cpp:292-559.  `io` holds the caller's incoming
 * values (the reference writes into the caller's Parametr in place). */
static void get_par_tvd(ctx *c, int f, int buf, st5 *io) {
    int t = c->m.face_type[f];
    int M = c->m.face_master[f];
    if (t == T_USUALY) {
        int Sd = c->m.face_sosed_down[f];
        int So = c->m.face_sosed[f];
        if (Sd < 0) {
            if (cell_has_axis(c, M)) { /* Gran.cpp:308-338 */
                double x, y, x2, y2, dist1, dist2, dist3;
                st5 par = cell_state(c, M, buf);
                face_center(c, f, 0, &x, &y);
                st5 par2 = cell_state(c, M, buf);
                st5 par1 = cell_state(c, M, buf);
                par1.v = -par1.v;
                st5 par3 = cell_state(c, So, buf);
                cell_center(c, M, 0, &x2, &y2);
                dist2 = sqrt(kv(x - x2) + kv(y - y2));
                cell_center(c, So, 0, &x2, &y2);
                dist3 = sqrt(kv(x - x2) + kv(y - y2));
                cell_center(c, M, 0, &x2, &y2);
                y2 = -y2;
                dist1 = sqrt(kv(x - x2) + kv(y - y2));
                par.v = linear3(-dist1, par1.v, -dist2, par2.v, dist3, par3.v, 0.0);
                *io = par;
            } else {
                *io = cell_state(c, M, buf);
            }
            return;
        }
        if (is_tracked_face(c, f)) { /* Gran.cpp:345-426 */
            double x, y, x2, y2, dist1, dist2;
            face_center(c, f, 0, &x, &y);
            st5 par2 = cell_state(c, M, buf);
            st5 par1 = cell_state(c, Sd, buf);
            cell_center(c, M, 0, &x2, &y2);
            dist2 = sqrt(kv(x - x2) + kv(y - y2));
            cell_center(c, Sd, 0, &x2, &y2);
            dist1 = sqrt(kv(x - x2) + kv(y - y2));
            io->ro = linear2(-dist1, par1.ro, -dist2, par2.ro, 0.0);
            io->p = linear2(-dist1, par1.p, -dist2, par2.p, 0.0);
            io->u = linear2(-dist1, par1.u, -dist2, par2.u, 0.0);
            io->v = linear2(-dist1, par1.v, -dist2, par2.v, 0.0);
            io->Q = linear2(-dist1, par1.Q, -dist2, par2.Q, 0.0);
            if (io->ro <= 0.0) io->ro = par2.ro;
            if (io->p <= 0.0) io->p = par2.p;
            return;
        }
        /* Gran.cpp:427-472 */
        double x, y, x2, y2, dist1, dist2, dist3;
        face_center(c, f, 0, &x, &y);
        st5 par2 = cell_state(c, M, buf);
        st5 par1 = cell_state(c, Sd, buf);
        st5 par3 = cell_state(c, So, buf);
        cell_center(c, M, 0, &x2, &y2);
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, So, 0, &x2, &y2);
        dist3 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, Sd, 0, &x2, &y2);
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
        io->ro = linear3(-dist1, par1.ro, -dist2, par2.ro, dist3, par3.ro, 0.0);
        io->p = linear3(-dist1, par1.p, -dist2, par2.p, dist3, par3.p, 0.0);
        io->u = linear3(-dist1, par1.u, -dist2, par2.u, dist3, par3.u, 0.0);
        io->v = linear3(-dist1, par1.v, -dist2, par2.v, dist3, par3.v, 0.0);
        io->Q = linear3(-dist1, par1.Q, -dist2, par2.Q, dist3, par3.Q, 0.0);
        if (io->ro <= 0.0 || io->p <= 0.0) { /* reference: exit(-1), Gran.cpp:444-455 */
            c->status |= 2;
            c->n_tvd_bad++;
        }
    } else if (t == T_EXTERN) {
        *io = cell_state(c, M, buf);
        if (io->u >= 0.0) io->u = c->prm.extern_u_tvd;
    } else if (t == T_UPPER_WALL) {
        *io = cell_state(c, M, buf);
    } else if (t == T_AXIS) { /* Gran.cpp:486-519 */
        double x, y, x2, y2, dist1, dist2;
        int Sd = c->m.face_sosed_down[f];
        face_center(c, f, 0, &x, &y);
        st5 par2 = cell_state(c, M, buf);
        st5 par1 = cell_state(c, Sd, buf);
        cell_center(c, M, 0, &x2, &y2);
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, Sd, 0, &x2, &y2);
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
        *io = par2;
        io->v = linear3(-dist1, par1.v, -dist2, par2.v, dist2, -par2.v, 0.0);
    } else if (t == T_INNER_SPHERE) {
        *io = inner_sphere_state(c, f);
    } else if (t == T_INPUT) {
        *io = input_state(c);
    }
}

/* Gran::Get_par_TVD_radial: Gran.cpp:562-675; only ro and p are consumed by
 * the callers (Setka.cpp:10228-10230, 10246-10248, 7083-7089).  Non-Usualy
 * faces leave the caller's fresh Parametr untouched (zeros). */
static void get_par_tvd_radial(const ctx *c, int f, int buf, double *oro, double *op) {
    const double g2 = 2.0 * c->prm.gamma;
    *oro = 0.0;
    *op = 0.0;
    if (c->m.face_type[f] != T_USUALY) return;
    int M = c->m.face_master[f], So = c->m.face_sosed[f], Sd = c->m.face_sosed_down[f];
    if (Sd < 0) {
        if (cell_has_axis(c, M)) { /* Gran.cpp:580-626 */
            double x, y, x2, y2, dist1, dist2, dist3;
            face_center(c, f, 0, &x, &y);
            double r = sqrt(kv(x) + kv(y));
            st5 par2 = cell_state(c, M, buf);
            st5 par1 = par2;
            par1.v = -par1.v;
            st5 par3 = cell_state(c, So, buf);
            cell_center(c, M, 0, &x2, &y2);
            double r2 = sqrt(kv(x2) + kv(y2));
            dist2 = sqrt(kv(x - x2) + kv(y - y2));
            cell_center(c, So, 0, &x2, &y2);
            double r3 = sqrt(kv(x2) + kv(y2));
            dist3 = sqrt(kv(x - x2) + kv(y - y2));
            cell_center(c, M, 0, &x2, &y2);
            y2 = -y2;
            double r1 = sqrt(kv(x2) + kv(y2));
            dist1 = sqrt(kv(x - x2) + kv(y - y2));
            *oro = linear3(-dist1, par1.ro * kv(r1), -dist2, par2.ro * kv(r2), dist3, par3.ro * kv(r3), 0.0) / kv(r);
            *op = linear3(-dist1, par1.p * pow(r1, g2), -dist2, par2.p * pow(r2, g2), dist3, par3.p * pow(r3, g2),
                          0.0) /
                  pow(r, g2);
        } else {
            st5 s = cell_state(c, M, buf);
            *oro = s.ro;
            *op = s.p;
        }
        return;
    }
    double x, y, x2, y2, dist1, dist2, dist3;
    face_center(c, f, 0, &x, &y);
    double r = sqrt(kv(x) + kv(y));
    st5 par2 = cell_state(c, M, buf);
    st5 par1 = cell_state(c, Sd, buf);
    st5 par3 = cell_state(c, So, buf);
    cell_center(c, M, 0, &x2, &y2);
    double r2 = sqrt(kv(x2) + kv(y2));
    dist2 = sqrt(kv(x - x2) + kv(y - y2));
    cell_center(c, So, 0, &x2, &y2);
    double r3 = sqrt(kv(x2) + kv(y2));
    dist3 = sqrt(kv(x - x2) + kv(y - y2));
    cell_center(c, Sd, 0, &x2, &y2);
    double r1 = sqrt(kv(x2) + kv(y2));
    dist1 = sqrt(kv(x - x2) + kv(y - y2));
    *oro = linear3(-dist1, par1.ro * kv(r1), -dist2, par2.ro * kv(r2), dist3, par3.ro * kv(r3), 0.0) / kv(r);
    *op = linear3(-dist1, par1.p * pow(r1, g2), -dist2, par2.p * pow(r2, g2), dist3, par3.p * pow(r3, g2), 0.0) /
          pow(r, g2);
}

/* ------------------------------------------------------------------ Riemann solvers */
/* Setka::HLLC_2d_Korolkov_b_s: Setka.cpp:10484-10700 */
static double hllc(const go_params *prm, double ro_L, double Q_L, double p_L, double v1_L, double v2_L, double ro_R,
                   double Q_R, double p_R, double v1_R, double v2_R, double W, double *P, double *PQ, double n1,
                   double n2, double rad, int metod, double *Vl, double *Vc, double *Vp, int nul_potok) {
    const double ggg = prm->gamma, g1 = prm->gamma - 1.0;
    double t1 = n2;
    double t2 = -n1;
    double u1 = v1_L * n1 + v2_L * n2;
    double v1 = v1_L * t1 + v2_L * t2;
    double u2 = v1_R * n1 + v2_R * n2;
    double v2 = v1_R * t1 + v2_R * t2;
    double cL = sqrt(ggg * p_L / ro_L);
    double cR = sqrt(ggg * p_R / ro_R);
    double uu_L = (kv(v1_L) + kv(v2_L)) / 2.0;
    double uu_R = (kv(v1_R) + kv(v2_R)) / 2.0;
    double SL = dmin(u1, u2) - dmax(cL, cR);
    double SR = dmax(u1, u2) + dmax(cL, cR);
    *Vl = SL;
    *Vp = SR;
    double suR = (SR - u2);
    double suL = (SL - u1);
    double SM = (suR * ro_R * u2 - suL * ro_L * u1 - p_R + p_L) / (suR * ro_R - suL * ro_L);
    *Vc = SM;
    double UU = dmax(fabs(SL), fabs(SR));
    double time = prm->kurant * rad / UU;
    double FL[5], FR[5], UL[5], UR[5];
    double e1 = p_L / g1 + ro_L * uu_L;
    double e2 = p_R / g1 + ro_R * uu_R;
    FL[0] = ro_L * u1;
    FL[1] = ro_L * u1 * u1 + p_L;
    FL[2] = ro_L * u1 * v1;
    FL[3] = (e1 + p_L) * u1;
    FL[4] = Q_L * u1;
    FR[0] = ro_R * u2;
    FR[1] = ro_R * u2 * u2 + p_R;
    FR[2] = ro_R * u2 * v2;
    FR[3] = (e2 + p_R) * u2;
    FR[4] = Q_R * u2;
    UL[0] = ro_L;
    UL[1] = ro_L * u1;
    UL[2] = ro_L * v1;
    UL[3] = e1;
    UL[4] = Q_L;
    UR[0] = ro_R;
    UR[1] = ro_R * u2;
    UR[2] = ro_R * v2;
    UR[3] = e2;
    UR[4] = Q_R;
    if (SL >= W) {
        P[1] = n1 * (FL[1] - W * UL[1]) + t1 * (FL[2] - W * UL[2]);
        P[2] = n2 * (FL[1] - W * UL[1]) + t2 * (FL[2] - W * UL[2]);
        P[0] = FL[0] - W * UL[0];
        P[3] = FL[3] - W * UL[3];
        *PQ = FL[4] - W * UL[4];
        return time;
    }
    if (SR <= W) {
        P[1] = n1 * (FR[1] - W * UR[1]) + t1 * (FR[2] - W * UR[2]);
        P[2] = n2 * (FR[1] - W * UR[1]) + t2 * (FR[2] - W * UR[2]);
        P[0] = FR[0] - W * UR[0];
        P[3] = FR[3] - W * UR[3];
        *PQ = FR[4] - W * UR[4];
        return time;
    }
    double ro_LL = ro_L * (SL - u1) / (SL - SM);
    double ro_RR = ro_R * (SR - u2) / (SR - SM);
    double Q_LL = Q_L * (SL - u1) / (SL - SM);
    double Q_RR = Q_R * (SR - u2) / (SR - SM);
    double UZ0 = (SR * UR[0] - SL * UL[0] + FL[0] - FR[0]) / (SR - SL);
    double UZ1 = (SR * UR[1] - SL * UL[1] + FL[1] - FR[1]) / (SR - SL);
    double UZ2 = (SR * UR[2] - SL * UL[2] + FL[2] - FR[2]) / (SR - SL);
    double UZ3 = (SR * UR[3] - SL * UL[3] + FL[3] - FR[3]) / (SR - SL);
    double UZ4 = (SR * UR[4] - SL * UL[4] + FL[4] - FR[4]) / (SR - SL);
    if (metod == 0) {
        double PO[5];
        for (int i = 0; i < 5; i++) PO[i] = (SR * FL[i] - SL * FR[i] + SR * SL * (UR[i] - UL[i])) / (SR - SL);
        P[1] = n1 * (PO[1] - W * UZ1) + t1 * (PO[2] - W * UZ2);
        P[2] = n2 * (PO[1] - W * UZ1) + t2 * (PO[2] - W * UZ2);
        P[0] = PO[0] - W * UZ0;
        P[3] = PO[3] - W * UZ3;
        *PQ = PO[4] - W * UZ4;
        return time;
    }
    double suRm = suR / (SR - SM);
    double suLm = suL / (SL - SM);
    double ptzR = p_R + ro_R * suR * (SM - u2);
    double ptzL = p_L + ro_L * suL * (SM - u1);
    double ptz = (ptzR + ptzL) / 2.0;
    double vLL, vRR;
    if (nul_potok) {
        vRR = UZ2 / UZ0;
        vLL = vRR;
    } else {
        vLL = v1;
        vRR = v2;
    }
    double ee2 = e2 * suRm + (ptz * SM - p_R * u2) / (SR - SM);
    double ee1 = e1 * suLm + (ptz * SM - p_L * u1) / (SL - SM);
    double ULL[5], URR[5], PO[5] = {0, 0, 0, 0, 0};
    ULL[0] = ro_LL;
    ULL[1] = ro_LL * SM;
    ULL[2] = ro_LL * vLL;
    ULL[3] = ee1;
    ULL[4] = Q_LL;
    URR[0] = ro_RR;
    URR[1] = ro_RR * SM;
    URR[2] = ro_RR * vRR;
    URR[3] = ee2;
    URR[4] = Q_RR;
    if (SL < W && SM >= W) {
        for (int i = 0; i < 5; i++) PO[i] = FL[i] + SL * ULL[i] - SL * UL[i] - W * ULL[i];
    } else if (SR > W && SM < W) {
        for (int i = 0; i < 5; i++) PO[i] = FR[i] + SR * URR[i] - SR * UR[i] - W * URR[i];
    }
    P[1] = n1 * PO[1] + t1 * PO[2];
    P[2] = n2 * PO[1] + t2 * PO[2];
    P[0] = PO[0];
    P[3] = PO[3];
    *PQ = PO[4];
    return time;
}

/* Solvers::lev: Solvers.cpp:1307-1321 */
static double lev(double ga, double enI, double pI, double rI, double enII, double pII, double rII, double uuu) {
    const double g1 = ga - 1.0, g2 = ga + 1.0, gp = (g2 / ga) / 2.0, gm = (g1 / ga) / 2.0;
    double cI = sqrt(ga * pI / rI);
    double cII = sqrt(ga * pII / rII);
    double fI = (uuu - pI) / (rI * cI * sqrt(gp * uuu / pI + gm));
    double fII = 2.0 / g1 * cII * (pow((uuu / pII), gm) - 1.0);
    double f1 = fI + fII;
    double f2 = enI - enII;
    (void)cI;
    return f1 - f2;
}
/* Solvers::devtwo: Solvers.cpp:1231-1305 (bisection) */
static double devtwo(double ga, double enI, double pI, double rI, double enII, double pII, double rII, int cap,
                     int *status) {
    const double epsil = 10e-10;
    double kl = pI, kp = pII, kc, ksi, ksir, ksit;
    ksi = lev(ga, enI, pI, rI, enII, pII, rII, kl);
    ksir = lev(ga, enI, pI, rI, enII, pII, rII, kp);
    if (fabs(ksi) <= epsil) return kl;
    if (fabs(ksir) <= epsil) return kp;
    int k = 0;
    for (;;) {
        k = k + 1;
        if (k == cap) {
            *status |= 1;
            return (kl + kp) / 2.0;
        }
        kc = (kl + kp) / 2.0;
        ksit = lev(ga, enI, pI, rI, enII, pII, rII, kc);
        if (fabs(ksit) <= epsil) return kc;
        if ((ksi * ksit) <= 0.0) {
            kp = kc;
            ksir = ksit;
        } else {
            kl = kc;
            ksi = ksit;
        }
    }
}
/* Solvers::newton: Solvers.cpp:1174-1229 */
static double newton(double ga, double enI, double pI, double rI, double enII, double pII, double rII, int cap,
                     int *status) {
    const double eps = 10e-10;
    const double g1 = ga - 1.0, g2 = ga + 1.0, gp = (g2 / ga) / 2.0, gm = (g1 / ga) / 2.0;
    (void)g1;
    double fI, fIs, fII, fIIs, p;
    double cI = sqrt(ga * pI / rI);
    double cII = sqrt(ga * pII / rII);
    double pn = pI * rII * cII + pII * rI * cI + (enI - enII) * rI * cI * rII * cII;
    pn = pn / (rI * cI + rII * cII);
    double pee = pn;
    int kiter = 0;
    for (;;) {
        p = pn;
        if (p <= 0.0) {
            *status |= 4;
            return p;
        }
        kiter = kiter + 1;
        fI = (p - pI) / (rI * cI * sqrt(gp * p / pI + gm));
        fIs = (ga + 1.0) * p / pI + (3.0 * ga - 1.0);
        fIs = fIs / (4.0 * ga * rI * cI * pow((gp * p / pI + gm), (3.0 / 2.0)));
        fII = (p - pII) / (rII * cII * sqrt(gp * p / pII + gm));
        fIIs = (ga + 1.0) * p / pII + (3.0 * ga - 1.0);
        fIIs = fIIs / (4.0 * ga * rII * cII * pow((gp * p / pII + gm), (3.0 / 2.0)));
        if (kiter == cap) {
            *status |= 1;
            return p;
        }
        pn = p - (fI + fII - (enI - enII)) / (fIs + fIIs);
        if (!(fabs(pn / pee - p / pee) >= eps)) break;
    }
    return pn;
}

/* Solvers::Godunov_Solver_Alexashov: Solvers.cpp:693-1172.  q1, q2 = (ro, p,
 * u, v, w); n[3] unit normal; output qqq[5] = mass, 3 momentum, energy flux
 * in the moving frame w. */
static double godunov(const go_params *prm, const double *qqq1, const double *qqq2, const double *n, double *qqq,
                      double *dsl, double *dsp, double *dsc, double w, double DIST, int *status) {
    const double ga = prm->gamma, g1 = ga - 1.0, g2 = ga + 1.0, gm = (g1 / ga) / 2.0;
    const double gg1 = g1, gg2 = g2, gga = ga;
    const double eps = 10e-10, eps8 = 10e-8;
    const int cap = prm->godunov_max_iter;
    double al = n[0], be = n[1], ge = n[2];
    double time = 0.0;
    double al2 = be, be2 = -al, ge2 = 0.0;
    double al3 = 0.0, be3 = 0.0, ge3 = 1.0;
    double enI = al * qqq1[2] + be * qqq1[3] + ge * qqq1[4];
    double teI2 = al2 * qqq1[2] + be2 * qqq1[3] + ge2 * qqq1[4];
    double teI3 = al3 * qqq1[2] + be3 * qqq1[3] + ge3 * qqq1[4];
    double enII = al * qqq2[2] + be * qqq2[3] + ge * qqq2[4];
    double teII2 = al2 * qqq2[2] + be2 * qqq2[3] + ge2 * qqq2[4];
    double teII3 = al3 * qqq2[2] + be3 * qqq2[3] + ge3 * qqq2[4];
    double pI = qqq1[1], pII = qqq2[1], rI = qqq1[0], rII = qqq2[0];
    int ipiz = 0;
    if (pI > pII) {
        double eno2 = enII, teo22 = teII2, teo23 = teII3, p2 = pII, r2 = rII;
        double eno1 = enI, teo12 = teI2, teo13 = teI3, p1 = pI, r1 = rI;
        enI = -eno2; teI2 = teo22; teI3 = teo23; pI = p2; rI = r2;
        enII = -eno1; teII2 = teo12; teII3 = teo13; pII = p1; rII = r1;
        w = -w;
        ipiz = 1;
    }
    double cI = 0.0, cII = 0.0;
    if (pI != 0.0) cI = sqrt(ga * pI / rI);
    if (pII != 0.0) cII = sqrt(ga * pII / rII);
    double a = sqrt(rI * (g2 * pII + g1 * pI) / 2.0);
    double Uud = (pII - pI) / a;
    double Urz = -2.0 * cII / g1 * (1.0 - pow((pI / pII), gm));
    double Uvk = -2.0 * (cII + cI) / g1;
    double Udf = enI - enII;
    int il = -2, ip = -2;
    double p = 0.0, r = 0.0, te2 = 0.0, te3 = 0.0, en = 0.0;
    if (Udf < Uvk) {
        il = -1; ip = -1;
    } else if ((Udf >= Uvk) && (Udf <= Urz)) {
        p = pI * pow(((Udf - Uvk) / (Urz - Uvk)), (1.0 / gm));
        il = 0; ip = 0;
    } else if ((Udf > Urz) && (Udf <= Uud)) {
        p = devtwo(ga, enI, pI, rI, enII, pII, rII, cap, status);
        il = 1; ip = 0;
    } else if (Udf > Uud) {
        p = newton(ga, enI, pI, rI, enII, pII, rII, cap, status);
        il = 1; ip = 1;
    }
    if ((il == 1) && (ip == 1)) { /* TWO SHOCKS */
        double aI = sqrt(rI * (g2 / 2.0 * p + g1 / 2.0 * pI));
        double aII = sqrt(rII * (g2 / 2.0 * p + g1 / 2.0 * pII));
        double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        double dI = enI - aI / rI;
        double dII = enII + aII / rII;
        *dsl = dI; *dsp = dII; *dsc = u;
        double UU = dmax(fabs(*dsl), fabs(*dsp));
        time = (UU > eps8) ? prm->kurant * DIST / UU : prm->kurant * DIST / eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        } else if ((w > dI) && (w <= u)) {
            en = u; r = rI * aI / (aI - rI * (enI - u)); te2 = teI2; te3 = teI3;
        } else if ((w > u) && (w < dII)) {
            en = u; r = rII * aII / (aII + rII * (enII - u)); te2 = teII2; te3 = teII3;
        } else if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 1) && (ip == 0)) { /* LEFT SHOCK, RIGHT EXPANSION */
        double aI = sqrt(rI * (g2 / 2.0 * p + g1 / 2.0 * pI));
        double aII;
        if (fabs(p - pII) < eps) aII = rII * cII;
        else aII = gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), gm));
        double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        double dI = enI - aI / rI;
        double dII = enII + cII;
        double ddII = u + cII - g1 * (enII - u) / 2.0;
        *dsl = dI; *dsp = dII; *dsc = u;
        double UU = dmax(fabs(*dsl), fabs(*dsp));
        UU = dmax(UU, fabs(ddII));
        time = (UU > eps8) ? prm->kurant * DIST / UU : prm->kurant * DIST / eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w <= u)) {
            en = u; r = rI * aI / (aI - rI * (enI - u)); te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            double ce = cII - g1 / 2.0 * (enII - u);
            en = u; r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            double ce = -g1 / g2 * (enII - w) + 2.0 / g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 0) && (ip == 0)) { /* TWO EXPANSION FANS */
        double aI, aII;
        if (fabs(p - pI) < eps) aI = rI * cI;
        else aI = gm * rI * cI * (1.0 - p / pI) / (1.0 - pow((p / pI), gm));
        if (fabs(p - pII) < eps) aII = rII * cII;
        else aII = gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), gm));
        double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        double dI = enI - cI;
        double ddI = u - cI - g1 * (enI - u) / 2.0;
        double dII = enII + cII;
        double ddII = u + cII - g1 * (enII - u) / 2.0;
        *dsl = dI; *dsp = dII; *dsc = u;
        double UU = dmax(fabs(*dsl), fabs(*dsp));
        UU = dmax(UU, fabs(ddII));
        UU = dmax(UU, fabs(ddI));
        time = (UU > eps8) ? prm->kurant * DIST / UU : prm->kurant * DIST / eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            double ce = g1 / g2 * (enI - w) + 2.0 / g2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / gm)); r = ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= u)) {
            double ce = cI + g1 / 2.0 * (enI - u);
            en = u; r = ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            double ce = cII - g1 / 2.0 * (enII - u);
            en = u; r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            double ce = -g1 / g2 * (enII - w) + 2.0 / g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == -1) && (ip == -1)) { /* VACUUM */
        double dI = enI - cI;
        double ddI = enI + 2.0 / gg1 * cI;
        double dII = enII + cII;
        double ddII = enII - 2.0 / gg1 * cII;
        *dsl = dI; *dsp = dII; *dsc = (dI + dII) / 2.0;
        double UU = dmax(fabs(*dsl), fabs(*dsp));
        UU = dmax(UU, fabs(ddII));
        UU = dmax(UU, fabs(ddI));
        time = (UU > eps8) ? prm->kurant * DIST / UU : prm->kurant * DIST / eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            double ce = gg1 / gg2 * (enI - w) + 2.0 / gg2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / gm)); r = gga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= ddII)) {
            en = w; p = 0.0; r = 0.0; te2 = 0.0; te3 = 0.0;
        }
        if ((w > ddII) && (w < dII)) {
            double ce = -gg1 / gg2 * (enII - w) + 2.0 / gg2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = gga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if (ipiz == 1) {
        en = -en;
        double dsl1 = *dsl, dsp1 = *dsp;
        *dsl = -dsp1;
        *dsp = -dsl1;
        *dsc = -*dsc;
        w = -w;
    }
    double uo = al * en + al2 * te2 + al3 * te3;
    double vo = be * en + be2 * te2 + be3 * te3;
    double wo = ge * en + ge2 * te2 + ge3 * te3;
    double eo = p / g1 + 0.5 * r * (uo * uo + vo * vo + wo * wo);
    en = al * uo + be * vo + ge * wo;
    qqq[0] = (r * (en - w));
    qqq[1] = (r * (en - w) * uo + al * p);
    qqq[2] = (r * (en - w) * vo + be * p);
    qqq[3] = (r * (en - w) * wo + ge * p);
    qqq[4] = ((en - w) * eo + en * p);
    return time;
}

/* ------------------------------------------------------------------ charge-exchange source */
/* Cell::Get_Sourse_MK1: Cell.cpp:498-665 */
static void source_mk1(ctx *c, int k, double u, double v, double ro, double p, double *q1, double *q2, double *q3) {
    const go_params *P = &c->prm;
    double xx, yy;
    cell_center(c, k, 0, &xx, &yy);
    double rr = sqrt(kv(xx) + kv(yy));
    double uH[4], vH[4], roH[4], pH[4];
    double ku = c->ku[k], kvv = c->kv_[k], kT = c->kT[k];
    if (rr > P->src_rmin && rr < P->src_rmax && xx >= 0.0) {
        int K_do = c->m.cell_back[k], K_posle = c->m.cell_next[k];
        double r1, r2;
        if (rr < c->m.r_istoch[k]) {
            r1 = c->m.r_istoch[k];
            while (r1 > rr) {
                if (K_do < 0) { c->status |= 8; *q1 = *q2 = *q3 = 0.0; return; }
                r1 = c->m.r_istoch[K_do];
                K_do = c->m.cell_back[K_do];
            }
            if (K_do < 0) { c->status |= 8; *q1 = *q2 = *q3 = 0.0; return; }
            K_do = c->m.cell_next[K_do];
            K_posle = c->m.cell_next[K_do];
        } else {
            r2 = c->m.r_istoch[k];
            while (r2 < rr) {
                if (K_posle < 0) { c->status |= 8; *q1 = *q2 = *q3 = 0.0; return; }
                r2 = c->m.r_istoch[K_posle];
                K_posle = c->m.cell_next[K_posle];
            }
            if (K_posle < 0) { c->status |= 8; *q1 = *q2 = *q3 = 0.0; return; }
            K_posle = c->m.cell_back[K_posle];
            K_do = c->m.cell_back[K_posle];
        }
        r1 = c->m.r_istoch[K_do];
        r2 = c->m.r_istoch[K_posle];
        double TH[4];
        for (int s = 0; s < 4; s++) uH[s] = linear2(r1, c->Hu[4 * K_do + s], r2, c->Hu[4 * K_posle + s], rr);
        for (int s = 0; s < 4; s++) vH[s] = linear2(r1, c->Hv[4 * K_do + s], r2, c->Hv[4 * K_posle + s], rr);
        for (int s = 0; s < 4; s++) roH[s] = linear2(r1, c->Hn[4 * K_do + s], r2, c->Hn[4 * K_posle + s], rr);
        for (int s = 0; s < 4; s++) TH[s] = linear2(r1, c->HT[4 * K_do + s], r2, c->HT[4 * K_posle + s], rr);
        ku = linear2(r1, c->ku[K_do], r2, c->ku[K_posle], rr);
        kvv = linear2(r1, c->kv_[K_do], r2, c->kv_[K_posle], rr);
        kT = linear2(r1, c->kT[K_do], r2, c->kT[K_posle], rr);
        for (int s = 0; s < 4; s++) pH[s] = 0.5 * TH[s] * roH[s];
    } else {
        for (int s = 0; s < 4; s++) {
            uH[s] = c->Hu[4 * k + s];
            vH[s] = c->Hv[4 * k + s];
            roH[s] = c->Hn[4 * k + s];
            pH[s] = 0.5 * c->HT[4 * k + s] * c->Hn[4 * k + s];
        }
    }
    for (int s = 0; s < 4; s++)
        if (roH[s] <= 0.0) {
            roH[s] = 0.0000001;
            pH[s] = 0.0;
        }
    double UM[4], UH[4], sig[4], nu[4];
    for (int s = 0; s < 4; s++)
        UM[s] = sqrt(kv(u - uH[s]) + kv(v - vH[s]) + (64.0 / (9.0 * PI_)) * (p / ro + 2.0 * pH[s] / roH[s]));
    for (int s = 0; s < 4; s++)
        UH[s] = sqrt(kv(u - uH[s]) + kv(v - vH[s]) + (4.0 / PI_) * (p / ro + 2.0 * pH[s] / roH[s]));
    for (int s = 0; s < 4; s++) sig[s] = kv(1.0 - P->a_2 * log(UM[s]));
    for (int s = 0; s < 4; s++) nu[s] = ro * roH[s] * UM[s] * sig[s];
    double Mu = P->src_coef * (nu[0] * (uH[0] - u) + nu[1] * (uH[1] - u) + nu[2] * (uH[2] - u) + nu[3] * (uH[3] - u));
    double Mv = P->src_coef * (nu[0] * (vH[0] - v) + nu[1] * (vH[1] - v) + nu[2] * (vH[2] - v) + nu[3] * (vH[3] - v));
    double e[4];
    for (int s = 0; s < 4; s++)
        e[s] = nu[s] * ((kv(uH[s]) + kv(vH[s]) - kv(u) - kv(v)) / 2.0 + (UH[s] / UM[s]) * (2.0 * pH[s] / roH[s] - p / ro));
    double MT = P->src_coef * (e[0] + e[1] + e[2] + e[3]);
    *q1 = Mu * ku;
    *q2 = Mv * kvv;
    *q3 = MT * kT;
}

/* ------------------------------------------------------------------ step forms */
static void write_state(ctx *c, int k, int buf, double ro, double Q, double p, double u, double v) {
    c->par[buf][0][k] = ro;
    c->par[buf][1][k] = p;
    c->par[buf][2][k] = u;
    c->par[buf][3][k] = v;
    c->par[buf][4][k] = Q;
}

/* Setka::Go_stationary: Setka.cpp:5205-5343 */
void go_stationary(void *h, int step) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double ggg = P->gamma, g2 = 2 * P->gamma;
    int now1 = 1, now2 = 0;
    double T[2];
    T[0] = T[1] = P->dt0;
    for (int st = 0; st < step; st++) {
        now1 = (now1 + 1) % 2;
        now2 = (now2 + 1) % 2;
        double time = 10000000;
        T[now2] = 100000000;
        for (int k = 0; k < c->m.n_cells; k++) {
            double Potok[5] = {0, 0, 0, 0, 0};
            double Pf[4], PQ = 0.0;
            st5 par1 = cell_state(c, k, now1);
            double n1, n2, dist, x, y;
            cell_center(c, k, 0, &x, &y);
            double rad = sqrt(kv(x) + kv(y));
            if (c->m.cell_type[k] == C_CENTR) continue;
            for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
                int f = c->m.gran[g];
                double x2, y2;
                double S = face_square(c, f);
                face_center(c, f, 0, &x2, &y2);
                dist = sqrt(kv(x - x2) + kv(y - y2));
                st5 par11 = par1;
                st5 par2 = get_par(c, f, now1);
                face_normal(c, f, &n1, &n2);
                double Vc, Vl, Vp;
                int met = 1;
                int ft = c->m.face_type[f];
                if (rad < P->rad_stat && ft == T_USUALY) {
                    double x3, y3;
                    cell_center(c, c->m.face_sosed[f], 0, &x3, &y3);
                    double dd = sqrt(kv(x3) + kv(y3));
                    par11.ro = par11.ro * kv(rad) / (kv(x2) + kv(y2));
                    par2.ro = par2.ro * kv(dd) / (kv(x2) + kv(y2));
                    par11.p = par11.p * pow(rad / sqrt(kv(x2) + kv(y2)), g2);
                    par2.p = par2.p * pow(dd / sqrt(kv(x2) + kv(y2)), g2);
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    polar_perenos(x3, y3, x2, y2, &par2.u, &par2.v, TINY_ANGLE);
                } else if (ft == T_INNER_SPHERE) {
                    par11.ro = par11.ro * kv(rad) / (kv(x2) + kv(y2));
                    par11.p = par11.p * pow(rad / sqrt(kv(x2) + kv(y2)), g2);
                } else if (rad < P->rad_stat && ft == T_AXIS) {
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    par11.v = 0.0;
                    par2 = par11;
                } else if (ft == T_AXIS) {
                    par11.v = 0.0;
                    par2 = par11;
                }
                time = dmin(time, hllc(P, par11.ro, par11.Q, par11.p, par11.u, par11.v, par2.ro, par2.Q, par2.p,
                                       par2.u, par2.v, 0.0, Pf, &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, 0));
                for (int q = 0; q < 4; q++) Potok[q] = Potok[q] + Pf[q] * S;
                Potok[4] = Potok[4] + PQ * S;
            }
            if (time < T[now2]) T[now2] = time;
            double ro3, p3, u3, v3, Q33;
            double Volume = cell_volume(c, k, 0);
            ro3 = par1.ro - T[now1] * (Potok[0] / Volume + par1.ro * par1.v / y);
            Q33 = par1.Q - (T[now1] / Volume) * Potok[4] - T[now1] * par1.Q * par1.v / y;
            if (ro3 <= 0) {
                ro3 = P->ro_floor;
                c->n_ro_clamp++;
            }
            u3 = (par1.ro * par1.u - T[now1] * (Potok[1] / Volume + par1.ro * par1.v * par1.u / y)) / ro3;
            v3 = (par1.ro * par1.v - T[now1] * (Potok[2] / Volume + par1.ro * par1.v * par1.v / y)) / ro3;
            p3 = (((par1.p / (ggg - 1) + par1.ro * (par1.u * par1.u + par1.v * par1.v) * 0.5) -
                   T[now1] * (Potok[3] / Volume +
                              +par1.v * (ggg * par1.p / (ggg - 1) + par1.ro * (par1.u * par1.u + par1.v * par1.v) * 0.5) / y)) -
                  0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                 (ggg - 1);
            if (p3 <= 0) {
                p3 = P->p_floor;
                c->n_p_clamp++;
            }
            write_state(c, k, now2, ro3, Q33, p3, u3, v3);
        }
    }
    c->last_dt = T[now2];
}

/* Setka::Move_surface: Setka.cpp:3378-3844 (including its index quirks:
 * the averaging loops of the inner and outer shocks walk Line_Contact). */
void go_move_surface(void *h, int ii, double dt) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double koef = P->koef, ggg = P->gamma, g2 = 2.0 * P->gamma;
    const int nC = c->m.n_contact, nI = c->m.n_inner_line, nO = c->m.n_outer_line;
    const int32_t *LC = c->m.line_contact, *LI = c->m.line_inner, *LO = c->m.line_outer;
    const int32_t *fA = c->m.face_A, *fB = c->m.face_B;
    int stt = 0;
    if (nC > 0) { /* contact, Setka.cpp:3394-3542 */
        for (int j = 0; j < nC; j++) {
            int f = LC[j];
            st5 par1 = {0, 0, 0, 0, 0}, par2 = {0, 0, 0, 0, 0};
            get_par_tvd(c, f, ii, &par1);
            int fc = c->m.face_copy[f];
            get_par_tvd(c, fc, ii, &par2);
            double n1, n2, nn[3], q1[5], q2[5], qq[5], VV, Vl, Vp;
            face_normal(c, f, &n1, &n2);
            nn[0] = n1; nn[1] = n2; nn[2] = 0.0;
            q1[0] = par1.ro; q1[1] = par1.p; q1[2] = par1.u; q1[3] = par1.v; q1[4] = 0.0;
            q2[0] = par2.ro; q2[1] = par2.p; q2[2] = par2.u; q2[3] = par2.v; q2[4] = 0.0;
            godunov(P, q1, q2, nn, qq, &Vl, &Vp, &VV, 0.0, 0.0, &stt);
            VV = VV * koef * 0.3;
            int b = fB[f];
            c->Vx[b] += VV * n1;
            c->Vy[b] += VV * n2;
            c->count[b]++;
        }
        for (int j = 0; j < nC; j++) {
            int a = fA[LC[j]];
            if (c->count[a] > 0) {
                c->Vx[a] /= (1.0 * c->count[a]);
                c->Vy[a] /= (1.0 * c->count[a]);
            }
        }
        {
            int a0 = fA[LC[0]], b0 = fB[LC[0]];
            c->Vx[a0] = c->Vx[b0] + (c->x[b0] - c->x[a0]) / dt;
            int a1 = fA[LC[nC - 1]], b1 = fB[LC[nC - 1]];
            c->Vy[b1] = c->Vy[a1] + (c->y[a1] - c->y[b1]) / dt;
        }
    }
    if (nI > 0) { /* inner shock, Setka.cpp:3545-3738 */
        for (int j = 0; j < nI; j++) {
            int f = LI[j];
            int M = c->m.face_master[f];
            st5 par1 = cell_state(c, M, ii);
            double x, y, x2, y2;
            cell_center(c, M, 0, &x, &y);
            double radius = sqrt(kv(x) + kv(y));
            face_center(c, f, 0, &x2, &y2);
            double dis = sqrt(kv(x2) + kv(y2));
            int fc = c->m.face_copy[f];
            st5 par2 = {0, 0, 0, 0, 0};
            get_par_tvd(c, fc, ii, &par2);
            double n1, n2, nn[3], q1[5], q2[5], qq[5], VV, Vl, Vp;
            face_normal(c, f, &n1, &n2);
            par1.ro = par1.ro * kv(radius) / kv(dis);
            par1.p = par1.p * pow(radius / dis, g2);
            polar_perenos(x, y, x2, y2, &par1.u, &par1.v, TINY_ANGLE);
            nn[0] = n1; nn[1] = n2; nn[2] = 0.0;
            q1[0] = par1.ro; q1[1] = par1.p; q1[2] = par1.u; q1[3] = par1.v; q1[4] = 0.0;
            q2[0] = par2.ro; q2[1] = par2.p; q2[2] = par2.u; q2[3] = par2.v; q2[4] = 0.0;
            godunov(P, q1, q2, nn, qq, &Vl, &Vp, &VV, 0.0, 0.0, &stt);
            Vl = Vl * koef * 0.1;
            double t1 = -n2, t2 = n1;
            int a = fA[f], b = fB[f];
            if (fabs(par2.u * t1 + par2.v * t2) < 0.1) {
                c->Vx[a] += Vl * n1;
                c->Vy[a] += Vl * n2;
                c->count[a]++;
                c->Vx[b] += Vl * n1;
                c->Vy[b] += Vl * n2;
                c->count[b]++;
            } else {
                c->Vx[b] += Vl * n1;
                c->Vy[b] += Vl * n2;
                c->count[b]++;
            }
        }
        /* walks Line_Contact (Setka.cpp:3718-3731); the reference reads past
         * its end when Line_Inner is longer, here the walk stops there */
        for (int j = 0; j < nI && j < nC; j++) {
            int a = fA[LC[j]];
            if (c->count[a] > 0) {
                c->Vx[a] /= (1.0 * c->count[a]);
                c->Vy[a] /= (1.0 * c->count[a]);
            }
        }
        {
            int a0 = fA[LI[0]], b0 = fB[LI[0]];
            c->Vx[a0] = c->Vx[b0] + (c->x[b0] - c->x[a0]) / dt;
            int a1 = fA[LI[nI - 1]], b1 = fB[LI[nI - 1]];
            c->Vx[b1] = c->Vx[a1] + (c->x[a1] - c->x[b1]) / dt;
        }
    }
    if (nO > 0) { /* outer shock, Setka.cpp:3741-3843 */
        const int lim = P->n_outer_shock + c->m.dims[0] + c->m.dims[1] + 1;
        for (int j = 0; j < nO; j++) {
            if (j >= lim) continue;
            int f = LO[j];
            st5 par1 = {0, 0, 0, 0, 0}, par2 = {0, 0, 0, 0, 0};
            get_par_tvd(c, f, ii, &par1);
            int fc = c->m.face_copy[f];
            get_par_tvd(c, fc, ii, &par2);
            double n1, n2, nn[3], q1[5], q2[5], qq[5], VV, Vl, Vp;
            face_normal(c, f, &n1, &n2);
            nn[0] = n1; nn[1] = n2; nn[2] = 0.0;
            q1[0] = par1.ro; q1[1] = par1.p; q1[2] = par1.u; q1[3] = par1.v; q1[4] = 0.0;
            q2[0] = par2.ro; q2[1] = par2.p; q2[2] = par2.u; q2[3] = par2.v; q2[4] = 0.0;
            godunov(P, q1, q2, nn, qq, &Vl, &Vp, &VV, 0.0, 0.0, &stt);
            Vp = Vp * koef;
            double t1 = -n2, t2 = n1;
            int a = fA[f], b = fB[f];
            if ((kv(par1.u) + kv(par1.v) + kv(0.0)) / (ggg * par1.p / par1.ro) > 1.0) {
                c->Vx[b] += Vp * n1;
                c->Vy[b] += Vp * n2;
                c->count[b]++;
            } else {
                if (fabs(par1.u * t1 + par1.v * t2) < 0.01) {
                    c->Vx[a] += Vp * n1;
                    c->Vy[a] += Vp * n2;
                    c->count[a]++;
                    c->Vx[b] += Vp * n1;
                    c->Vy[b] += Vp * n2;
                    c->count[b]++;
                } else if (par1.u * t1 + par1.v * t2 > 0) {
                    c->Vx[b] += Vp * n1;
                    c->Vy[b] += Vp * n2;
                    c->count[b]++;
                } else {
                    c->Vx[a] += Vp * n1;
                    c->Vy[a] += Vp * n2;
                    c->count[a]++;
                }
            }
        }
        for (int j = 0; j < nO && j < nC; j++) { /* walks Line_Contact (Setka.cpp:3829-3837) */
            int a = fA[LC[j]];
            if (c->count[a] > 0) {
                c->Vx[a] /= (1.0 * c->count[a]);
                c->Vy[a] /= (1.0 * c->count[a]);
            }
        }
        {
            int a0 = fA[LO[0]], b0 = fB[LO[0]];
            c->Vx[a0] = c->Vx[b0] + (c->x[b0] - c->x[a0]) / dt;
            int a1 = fA[LO[nO - 1]], b1 = fB[LO[nO - 1]];
            c->Vy[b1] = c->Vy[a1] + (c->y[a1] - c->y[b1]) / dt;
        }
    }
    if (stt) c->status |= stt;
}

/* Setka::Move_Setka_Calculate_2: Setka.cpp:4324-4759 */
/* Setka::Move_Setka_Calculate (Setka.cpp:4761-5147) equals
 * Move_Setka_Calculate_2 except that it does not copy the outer-shock key
 * height along the D rails beyond n_outer_shock (Setka.cpp:4725-4728). */
static void move_setka(ctx *c, double dt, int copy_outer_shock);
void go_move_setka2(void *h, double dt) { move_setka((ctx *)h, dt, 1); }
void go_move_setka1(void *h, double dt) { move_setka((ctx *)h, dt, 0); }

static void move_setka(ctx *c, double dt, int copy_outer_shock) {
    const go_params *P = &c->prm;
    const int ni = P->n_inner;
    const double R1 = P->R1, R111 = P->R111, R5 = P->R5;
    double *X = c->x, *Y = c->y, *X2 = c->x2, *Y2 = c->y2;
    double V, R2, R3, R4, r, x;
    for (int q = 0; q < c->m.n_rails; q++) {
        const int32_t *ap = c->m.rail_points + c->m.rail_pstart[q];
        const int32_t *kp = c->m.rail_keys + c->m.rail_kstart[q];
        const int np = c->m.rail_pstart[q + 1] - c->m.rail_pstart[q];
        const int M1 = c->m.rail_M[4 * q], M2 = c->m.rail_M[4 * q + 1], M3 = c->m.rail_M[4 * q + 2],
                  M4 = c->m.rail_M[4 * q + 3];
        const double s = c->m.rail_s[q];
        const int t = c->m.rail_type[q];
        if (t == R_A) { /* Setka.cpp:4331-4457 */
            for (int kk = 0; kk < 3; kk++) {
                int K = kp[kk];
                V = c->Vx[K] * cos(s) + c->Vy[K] * sin(s);
                X2[K] = X[K] + dt * V * cos(s);
                Y2[K] = Y[K] + dt * V * sin(s);
            }
            X2[kp[3]] = X[kp[3]];
            Y2[kp[3]] = Y[kp[3]];
            R2 = sqrt(kv(X2[kp[0]]) + kv(Y2[kp[0]]));
            for (int j = 0; j < ni; j++) {
                x = j * 1.0 / (ni);
                r = R1 + pow(x, 1.3) * (R111 - R1);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            for (int j = ni; j < M1 - 1; j++) {
                x = (j - ni) * 1.0 / (M1 - 1 - ni);
                r = R111 + pow(x, 1.05) * (R2 - R111);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            R3 = sqrt(kv(X2[kp[1]]) + kv(Y2[kp[1]]));
            for (int j = 0; j < M2 - 1; j++) {
                r = R2 + (R3 - R2) * (j + 1) / (M2);
                X2[ap[M1 + j]] = r * cos(s);
                Y2[ap[M1 + j]] = r * sin(s);
            }
            R3 = sqrt(kv(X2[kp[1]]) + kv(Y2[kp[1]]));
            R4 = sqrt(kv(X2[kp[2]]) + kv(Y2[kp[2]]));
            for (int j = 0; j < M3 - 1; j++) {
                r = R3 + (R4 - R3) * (j + 1) / (M3);
                X2[ap[M1 + M2 + j]] = r * cos(s);
                Y2[ap[M1 + M2 + j]] = r * sin(s);
            }
            R4 = sqrt(kv(X2[kp[2]]) + kv(Y2[kp[2]]));
            for (int j = 0; j < M4; j++) {
                x = (j + 1) * 1.0 / (M4);
                double dd = 1.5708 / sqrt(1.0 - 1.0 / 1.76);
                r = R4 + pow(x, 1.76 * (1.0 - kv(s / dd))) * (R5 - R4);
                X2[ap[M1 + M2 + M3 + j]] = r * cos(s);
                Y2[ap[M1 + M2 + M3 + j]] = r * sin(s);
            }
        } else if (t == R_B) { /* Setka.cpp:4467-4595 */
            int K0 = kp[0], K1 = kp[1], K2 = kp[2], K3 = kp[3];
            V = c->Vx[K0] * cos(s) + c->Vy[K0] * sin(s);
            X2[K0] = X[K0] + dt * V * cos(s);
            Y2[K0] = Y[K0] + dt * V * sin(s);
            V = c->Vx[K1] * 0.0 + c->Vy[K1] * 1.0;
            X2[K1] = X2[K0];
            Y2[K1] = Y[K1] + dt * V;
            V = c->Vx[K2] * 0.0 + c->Vy[K2] * 1.0;
            X2[K2] = X2[K0];
            Y2[K2] = Y[K2] + dt * V;
            X2[K3] = X2[K0];
            Y2[K3] = Y[K3];
            R2 = sqrt(kv(X2[K0]) + kv(Y2[K0]));
            for (int j = 0; j < ni; j++) {
                x = j * 1.0 / (ni);
                r = R1 + pow(x, 1.3) * (R111 - R1);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            for (int j = ni; j < M1 - 1; j++) {
                x = (j - ni) * 1.0 / (M1 - 1 - ni);
                r = R111 + pow(x, 1.05) * (R2 - R111);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            R2 = Y2[K0];
            R3 = Y2[K1];
            for (int j = 0; j < M2 - 1; j++) {
                r = R2 + (R3 - R2) * (j + 1) / (M2);
                X2[ap[M1 + j]] = X2[K0];
                Y2[ap[M1 + j]] = r;
            }
            R3 = Y2[K1];
            R4 = Y2[K2];
            for (int j = 0; j < M3 - 1; j++) {
                r = R3 + (R4 - R3) * (j + 1) / (M3);
                X2[ap[M1 + M2 + j]] = X2[K0];
                Y2[ap[M1 + M2 + j]] = r;
            }
            for (int j = 0; j < M4; j++) {
                r = R4 + (R5 - R4) * (j + 1) / (M4);
                X2[ap[M1 + M2 + M3 + j]] = X2[K0];
                Y2[ap[M1 + M2 + M3 + j]] = r;
            }
        } else if (t == R_C) { /* Setka.cpp:4597-4674 */
            int K0 = kp[0], K1 = kp[1];
            V = c->Vx[K0] * cos(s) + c->Vy[K0] * sin(s);
            X2[K0] = X[K0] + dt * V * cos(s);
            Y2[K0] = Y[K0] + dt * V * sin(s);
            X2[K1] = P->Left;
            Y2[K1] = Y[K1];
            R2 = sqrt(kv(X2[K0]) + kv(Y2[K0]));
            for (int j = 0; j < ni; j++) {
                x = j * 1.0 / (ni);
                r = R1 + pow(x, 1.3) * (R111 - R1);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            for (int j = ni; j < M1 - 1; j++) {
                x = (j - ni) * 1.0 / (M1 - 1 - ni);
                r = R111 + pow(x, 1.05) * (R2 - R111);
                X2[ap[j]] = r * cos(s);
                Y2[ap[j]] = r * sin(s);
            }
            R2 = X2[K0];
            R3 = X2[K1];
            x = pow(R3 / (R2), 1.0 / (M2));
            for (int j = M1; j < np; j++) {
                r = R2 * pow(x, j + 1 - M1);
                X2[ap[j]] = r;
                Y2[ap[j]] = Y2[K0];
            }
        }
    }
    /* D rails after all C rails: Setka.cpp:4676-4758 */
    const int sM2 = c->m.dims[5], sM3 = c->m.dims[6], sM4 = c->m.dims[7];
    int jj = 0;
    int prev_k2 = -1;
    for (int q = 0; q < c->m.n_rails; q++) {
        if (c->m.rail_type[q] != R_D) continue;
        const int32_t *ap = c->m.rail_points + c->m.rail_pstart[q];
        const int32_t *kp = c->m.rail_keys + c->m.rail_kstart[q];
        const int M2 = c->m.rail_M[4 * q + 1], M3 = c->m.rail_M[4 * q + 2], M4 = c->m.rail_M[4 * q + 3];
        int K0 = kp[0], K1 = kp[1], K2 = kp[2], K3 = kp[3];
        V = c->Vy[K1];
        X2[K1] = X2[K0];
        Y2[K1] = Y[K1] + dt * V;
        V = c->Vy[K2];
        X2[K2] = X2[K0];
        Y2[K2] = Y[K2] + dt * V;
        if (copy_outer_shock && jj >= P->n_outer_shock) Y2[K2] = Y2[prev_k2];
        X2[K3] = X2[K0];
        Y2[K3] = Y[K3];
        R2 = Y2[K0];
        R3 = Y2[K1];
        for (int j = 0; j < sM2 - 1; j++) {
            r = R2 + (R3 - R2) * (j + 1) / (M2);
            X2[ap[j + 1]] = X2[K0];
            Y2[ap[j + 1]] = r;
        }
        R3 = Y2[K1];
        R4 = Y2[K2];
        for (int j = 0; j < sM3 - 1; j++) {
            r = R3 + (R4 - R3) * (j + 1) / (M3);
            X2[ap[sM2 + j + 1]] = X2[K0];
            Y2[ap[sM2 + j + 1]] = r;
        }
        for (int j = 0; j < sM4; j++) {
            r = R4 + (R5 - R4) * (j + 1) / (M4);
            X2[ap[sM2 + sM3 + j + 1]] = X2[K0];
            Y2[ap[sM2 + sM3 + j + 1]] = r;
        }
        prev_k2 = K2;
        jj++;
    }
}

void go_commit_points(void *h) {
    ctx *c = (ctx *)h;
    for (int i = 0; i < c->m.n_points; i++) {
        c->x[i] = c->x2[i];
        c->y[i] = c->y2[i];
        c->Vx[i] = 0.0;
        c->Vy[i] = 0.0;
        c->count[i] = 0;
    }
}

static int face_np_flag(const ctx *c, int f) { /* Setka.cpp:10301-10324 */
    int ta = c->m.point_type[c->m.face_A[f]], tb = c->m.point_type[c->m.face_B[f]];
    if (ta == P_CONTACT && tb != P_CONTACT) return 1;
    if (ta != P_CONTACT && tb == P_CONTACT) return 1;
    if (ta == P_INNER_SHOCK && tb != P_INNER_SHOCK) return 1;
    if (ta != P_INNER_SHOCK && tb == P_INNER_SHOCK) return 1;
    if (ta == P_OUTER_SHOCK && tb != P_OUTER_SHOCK) return 1;
    if (ta != P_OUTER_SHOCK && tb == P_OUTER_SHOCK) return 1;
    return 0;
}

/* Setka::Go_5_komponent__MK2: Setka.cpp:10121-10482 */
void go_mk2(void *h, int step) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double ggg = P->gamma, g2 = 2 * P->gamma;
    int now1 = 1, now2 = 0;
    double T[2];
    T[0] = T[1] = P->dt0;
    for (int st = 0; st < step; st++) {
        now1 = (now1 + 1) % 2;
        now2 = (now2 + 1) % 2;
        double time = 10000000;
        T[now2] = 100000000;
        go_move_surface(c, now1, T[now1]);
        go_move_setka2(c, T[now1]);
        for (int k = 0; k < c->m.n_cells; k++) {
            double Potok[5] = {0, 0, 0, 0, 0};
            double Pf[4], PQ = 0.0;
            st5 par1 = cell_state(c, k, now1);
            double n1, n2, dist, x, y;
            cell_center(c, k, 0, &x, &y);
            double vs1 = cell_volume(c, k, 0);
            double vs2 = cell_volume(c, k, 1);
            double radius = sqrt(kv(x) + kv(y));
            if (radius < P->R11) continue;
            double Volume = cell_volume_rotate(c, k, 0, 360.0) / (2.0 * PI_);
            double Volume2 = cell_volume_rotate(c, k, 1, 360.0) / (2.0 * PI_);
            double W = 0.0;
            int np = 1;
            const int kt = c->m.cell_type[k];
            for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
                int f = c->m.gran[g];
                double x2, y2, x4, y4;
                double S = face_square(c, f) * (c->y[c->m.face_A[f]] + c->y[c->m.face_B[f]]) * 0.5;
                face_center(c, f, 0, &x2, &y2);
                face_center(c, f, 1, &x4, &y4);
                dist = sqrt(kv(x - x2) + kv(y - y2));
                st5 par11 = par1;
                st5 par2 = get_par(c, f, now1);
                face_normal(c, f, &n1, &n2);
                double Vc, Vl, Vp;
                W = ((x4 - x2) * n1 + (y4 - y2) * n2) / T[now1];
                int met = 0;
                double dis = sqrt(kv(x2) + kv(y2));
                int ft = c->m.face_type[f];
                if (ft == T_USUALY) {
                    int So = c->m.face_sosed[f];
                    double x3, y3;
                    cell_center(c, So, 0, &x3, &y3);
                    double dd = sqrt(kv(x3) + kv(y3));
                    if (kt == C_1) {
                        par11.ro = par11.ro * kv(radius) / kv(dis);
                        par11.Q = par11.Q * kv(radius) / kv(dis);
                        par11.p = par11.p * pow(radius / dis, g2);
                        polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                        double pro, pp;
                        get_par_tvd_radial(c, f, now1, &pro, &pp);
                        par11.ro = pro;
                        par11.p = pp;
                    } else {
                        get_par_tvd(c, f, now1, &par11);
                    }
                    int fc = c->m.face_copy[f];
                    if (c->m.cell_type[So] == C_1) {
                        par2.ro = par2.ro * kv(dd) / kv(dis);
                        par2.Q = par2.Q * kv(dd) / kv(dis);
                        par2.p = par2.p * pow(dd / dis, g2);
                        polar_perenos(x3, y3, x2, y2, &par2.u, &par2.v, TINY_ANGLE);
                        double pro, pp;
                        get_par_tvd_radial(c, fc, now1, &pro, &pp);
                        par2.ro = pro;
                        par2.p = pp;
                    } else {
                        get_par_tvd(c, fc, now1, &par2);
                    }
                } else if (ft == T_INNER_SPHERE) {
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                } else if (kt == C_1 && ft == T_AXIS) {
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    par2 = par11;
                    par2.v = -par2.v;
                } else if (kt != C_1 && ft == T_AXIS) {
                    get_par_tvd(c, f, now1, &par11);
                    par2 = par11;
                    par2.v = -par2.v;
                }
                np = face_np_flag(c, f);
                int god = is_tracked_face(c, f);
                if (god) {
                    double Vl2, Vp2, VV, nn[3], q1[5], q2[5], qq[5];
                    nn[0] = n1; nn[1] = n2; nn[2] = 0.0;
                    q1[0] = par11.ro; q1[1] = par11.p; q1[2] = par11.u; q1[3] = par11.v; q1[4] = 0.0;
                    q2[0] = par2.ro; q2[1] = par2.p; q2[2] = par2.u; q2[3] = par2.v; q2[4] = 0.0;
                    int stt = 0;
                    time = dmin(time, godunov(P, q1, q2, nn, qq, &Vl2, &Vp2, &VV, W, dist, &stt));
                    c->status |= stt;
                    Potok[0] = Potok[0] + qq[0] * S;
                    Potok[1] = Potok[1] + qq[1] * S;
                    Potok[2] = Potok[2] + qq[2] * S;
                    Potok[3] = Potok[3] + qq[4] * S;
                    time = dmin(time, hllc(P, par11.ro, par11.Q, par11.p, par11.u, par11.v, par2.ro, par2.Q, par2.p,
                                           par2.u, par2.v, W, Pf, &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, np));
                    Potok[4] = Potok[4] + PQ * S;
                } else {
                    time = dmin(time, hllc(P, par11.ro, par11.Q, par11.p, par11.u, par11.v, par2.ro, par2.Q, par2.p,
                                           par2.u, par2.v, W, Pf, &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, np));
                    for (int q = 0; q < 4; q++) Potok[q] = Potok[q] + Pf[q] * S;
                    Potok[4] = Potok[4] + PQ * S;
                }
            }
            if (time < T[now2]) T[now2] = time;
            double u = par1.u, v = par1.v, ro = par1.ro, p = par1.p, Q = par1.Q;
            double q2_1, q2_2, q3;
            source_mk1(c, k, u, v, ro, p, &q2_1, &q2_2, &q3);
            double ro3, Q33, u3, v3, p3;
            if (kt != C_CENTR) {
                ro3 = ro * Volume / Volume2 - T[now1] * (Potok[0] / Volume2);
                Q33 = Q * Volume / Volume2 - (T[now1] / Volume2) * Potok[4];
                if (ro3 <= 0.0) {
                    ro3 = P->ro_floor;
                    c->n_ro_clamp++;
                }
                u3 = (ro * u * Volume / Volume2 - T[now1] * (Potok[1] / Volume2 - q2_1)) / ro3;
                v3 = (ro * v * Volume / Volume2 - T[now1] * ((Potok[2] - p * 0.5 * (vs1 + vs2)) / Volume2 - q2_2)) / ro3;
                p3 = (((p / (ggg - 1) + ro * (u * u + v * v) * 0.5) * Volume / Volume2 -
                       T[now1] * (Potok[3] / Volume2 - q3)) -
                      0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                     (ggg - 1);
                if (p3 <= 0) {
                    p3 = P->p_floor;
                    c->n_p_clamp++;
                }
                write_state(c, k, now2, ro3, Q33, p3, u3, v3);
            } else {
                st5 s = cell_state(c, k, now1);
                write_state(c, k, now2, s.ro, s.Q, s.p, s.u, s.v);
            }
        }
        go_commit_points(c);
    }
    c->last_dt = T[now2];
}

/* Setka::Go_stationary_5_komponent_inner_MK2: Setka.cpp:6999-7212 */
void go_inner_mk2(void *h, int step) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double ggg = P->gamma, g2 = 2.0 * P->gamma;
    int now1 = 1, now2 = 0;
    double T[2];
    T[0] = T[1] = P->dt0;
    for (int st = 0; st < step; st++) {
        now1 = (now1 + 1) % 2;
        now2 = (now2 + 1) % 2;
        double time = 10000000;
        T[now2] = 100000000;
        for (int ic = 0; ic < c->n_inner_cells; ic++) {
            int k = c->inner[ic];
            const int kt = c->m.cell_type[k];
            if (kt == C_CENTR) continue;
            double Potok[5] = {0, 0, 0, 0, 0};
            double Pf[4], PQ = 0.0;
            st5 par1 = cell_state(c, k, now1);
            double n1, n2, dist, x, y;
            cell_center(c, k, 0, &x, &y);
            double vs1 = cell_volume(c, k, 0);
            double vs2 = cell_volume(c, k, 1);
            double radius = sqrt(kv(x) + kv(y));
            double Volume = cell_volume_rotate(c, k, 0, 360.0) / (2.0 * PI_);
            for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
                int f = c->m.gran[g];
                double x2, y2;
                double S = face_square(c, f) * (c->y[c->m.face_A[f]] + c->y[c->m.face_B[f]]) * 0.5;
                face_center(c, f, 0, &x2, &y2);
                dist = sqrt(kv(x - x2) + kv(y - y2));
                st5 par11 = par1;
                st5 par2 = get_par(c, f, now1);
                face_normal(c, f, &n1, &n2);
                double Vc, Vl, Vp;
                int met = 1;
                double dis = sqrt(kv(x2) + kv(y2));
                int ft = c->m.face_type[f];
                if (ft == T_USUALY) {
                    int So = c->m.face_sosed[f];
                    double x3, y3;
                    cell_center(c, So, 0, &x3, &y3);
                    double dd = sqrt(kv(x3) + kv(y3));
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par2.ro = par2.ro * kv(dd) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par2.Q = par2.Q * kv(dd) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                    par2.p = par2.p * pow(dd / dis, g2);
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    polar_perenos(x3, y3, x2, y2, &par2.u, &par2.v, TINY_ANGLE);
                    if (kt == C_1 && c->m.cell_type[So] == C_1) {
                        double r1, p1, r2, p2;
                        get_par_tvd_radial(c, f, now1, &r1, &p1);
                        get_par_tvd_radial(c, c->m.face_copy[f], now1, &r2, &p2);
                        par11.ro = r1;
                        par2.ro = r2;
                        par11.p = p1;
                        par2.p = p2;
                    }
                } else if (ft == T_INNER_SPHERE) {
                    par11 = par2;
                } else if (ft == T_AXIS) {
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    par2 = par11;
                    par2.v = -par2.v;
                    met = 0;
                }
                time = dmin(time, hllc(P, par11.ro, par11.Q, par11.p, par11.u, par11.v, par2.ro, par2.Q, par2.p,
                                       par2.u, par2.v, 0.0, Pf, &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, 0));
                for (int q = 0; q < 4; q++) Potok[q] = Potok[q] + Pf[q] * S;
                Potok[4] = Potok[4] + PQ * S;
            }
            if (time < T[now2]) T[now2] = time;
            double u = par1.u, v = par1.v, ro = par1.ro, p = par1.p, Q = par1.Q;
            double q2_1, q2_2, q3;
            source_mk1(c, k, u, v, ro, p, &q2_1, &q2_2, &q3);
            double ro3, Q33, u3, v3, p3;
            ro3 = ro - T[now1] * (Potok[0] / Volume);
            Q33 = Q - (T[now1] / Volume) * Potok[4] - T[now1];
            if (ro3 <= 0) {
                ro3 = P->ro_floor;
                c->n_ro_clamp++;
            }
            u3 = (ro * u - T[now1] * (Potok[1] / Volume - q2_1)) / ro3;
            v3 = (ro * v - T[now1] * ((Potok[2] - p * 0.5 * (vs1 + vs2)) / Volume - q2_2)) / ro3;
            p3 = (((p / (ggg - 1) + ro * (u * u + v * v) * 0.5) - T[now1] * (Potok[3] / Volume - q3)) -
                  0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                 (ggg - 1);
            if (p3 <= 0) {
                p3 = P->p_floor;
                c->n_p_clamp++;
            }
            write_state(c, k, now2, ro3, Q33, p3, u3, v3);
        }
    }
    c->last_dt = T[now2];
}

/* ------------------------------------------------------------------ lifecycle */
static void *dup(const void *src, size_t bytes) {
    void *p = malloc(bytes ? bytes : 1);
    if (src && bytes) memcpy(p, src, bytes);
    else memset(p, 0, bytes ? bytes : 1);
    return p;
}

void *go_create(const go_params *prm, const go_mesh *m) {
    ctx *c = (ctx *)calloc(1, sizeof(ctx));
    c->prm = *prm;
    c->m = *m;
    const int np = m->n_points, nc = m->n_cells, nf = m->n_faces;
    const int nct = m->contour_start[nc], ngt = m->gran_start[nc];
    c->m.point_type = (const int32_t *)dup(m->point_type, sizeof(int32_t) * np);
    c->m.cell_type = (const int32_t *)dup(m->cell_type, sizeof(int32_t) * nc);
    c->m.contour_start = (const int32_t *)dup(m->contour_start, sizeof(int32_t) * (nc + 1));
    c->m.contour = (const int32_t *)dup(m->contour, sizeof(int32_t) * nct);
    c->m.gran_start = (const int32_t *)dup(m->gran_start, sizeof(int32_t) * (nc + 1));
    c->m.gran = (const int32_t *)dup(m->gran, sizeof(int32_t) * ngt);
    c->m.cell_back = (const int32_t *)dup(m->cell_back, sizeof(int32_t) * nc);
    c->m.cell_next = (const int32_t *)dup(m->cell_next, sizeof(int32_t) * nc);
    c->m.r_istoch = (const double *)dup(m->r_istoch, sizeof(double) * nc);
    c->m.face_A = (const int32_t *)dup(m->face_A, sizeof(int32_t) * nf);
    c->m.face_B = (const int32_t *)dup(m->face_B, sizeof(int32_t) * nf);
    c->m.face_type = (const int32_t *)dup(m->face_type, sizeof(int32_t) * nf);
    c->m.face_master = (const int32_t *)dup(m->face_master, sizeof(int32_t) * nf);
    c->m.face_sosed = (const int32_t *)dup(m->face_sosed, sizeof(int32_t) * nf);
    c->m.face_copy = (const int32_t *)dup(m->face_copy, sizeof(int32_t) * nf);
    c->m.face_sosed_up = (const int32_t *)dup(m->face_sosed_up, sizeof(int32_t) * nf);
    c->m.face_sosed_down = (const int32_t *)dup(m->face_sosed_down, sizeof(int32_t) * nf);
    const int nr = m->n_rails;
    c->m.rail_type = (const int32_t *)dup(m->rail_type, sizeof(int32_t) * nr);
    c->m.rail_s = (const double *)dup(m->rail_s, sizeof(double) * nr);
    c->m.rail_M = (const int32_t *)dup(m->rail_M, sizeof(int32_t) * 4 * nr);
    c->m.rail_pstart = (const int32_t *)dup(m->rail_pstart, sizeof(int32_t) * (nr + 1));
    c->m.rail_kstart = (const int32_t *)dup(m->rail_kstart, sizeof(int32_t) * (nr + 1));
    c->m.rail_points = (const int32_t *)dup(m->rail_points, sizeof(int32_t) * (nr ? m->rail_pstart[nr] : 0));
    c->m.rail_keys = (const int32_t *)dup(m->rail_keys, sizeof(int32_t) * (nr ? m->rail_kstart[nr] : 0));
    c->m.line_contact = (const int32_t *)dup(m->line_contact, sizeof(int32_t) * m->n_contact);
    c->m.line_inner = (const int32_t *)dup(m->line_inner, sizeof(int32_t) * m->n_inner_line);
    c->m.line_outer = (const int32_t *)dup(m->line_outer, sizeof(int32_t) * m->n_outer_line);
    c->x = (double *)dup(m->x, sizeof(double) * np);
    c->y = (double *)dup(m->y, sizeof(double) * np);
    c->x2 = (double *)dup(m->x, sizeof(double) * np);
    c->y2 = (double *)dup(m->y, sizeof(double) * np);
    c->Vx = (double *)dup(NULL, sizeof(double) * np);
    c->Vy = (double *)dup(NULL, sizeof(double) * np);
    c->count = (int32_t *)dup(NULL, sizeof(int32_t) * np);
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 5; q++) c->par[b][q] = (double *)dup(NULL, sizeof(double) * nc);
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 16; q++) c->hpar[b][q] = (double *)dup(NULL, sizeof(double) * nc);
    c->Hn = (double *)dup(NULL, sizeof(double) * 4 * nc);
    c->Hu = (double *)dup(NULL, sizeof(double) * 4 * nc);
    c->Hv = (double *)dup(NULL, sizeof(double) * 4 * nc);
    c->HT = (double *)dup(NULL, sizeof(double) * 4 * nc);
    c->ku = (double *)dup(NULL, sizeof(double) * nc);
    c->kv_ = (double *)dup(NULL, sizeof(double) * nc);
    c->kT = (double *)dup(NULL, sizeof(double) * nc);
    c->inner = (int32_t *)dup(NULL, sizeof(int32_t));
    for (int q = 0; q < 3; q++) c->qfix[q] = (double *)dup(NULL, sizeof(double) * nc);
    return c;
}

void go_destroy(void *h) {
    ctx *c = (ctx *)h;
    if (!c) return;
    free((void *)c->m.point_type); free((void *)c->m.cell_type); free((void *)c->m.contour_start);
    free((void *)c->m.contour); free((void *)c->m.gran_start); free((void *)c->m.gran);
    free((void *)c->m.cell_back); free((void *)c->m.cell_next); free((void *)c->m.r_istoch);
    free((void *)c->m.face_A); free((void *)c->m.face_B); free((void *)c->m.face_type);
    free((void *)c->m.face_master); free((void *)c->m.face_sosed); free((void *)c->m.face_copy);
    free((void *)c->m.face_sosed_up); free((void *)c->m.face_sosed_down);
    free((void *)c->m.rail_type); free((void *)c->m.rail_s); free((void *)c->m.rail_M);
    free((void *)c->m.rail_pstart); free((void *)c->m.rail_kstart); free((void *)c->m.rail_points);
    free((void *)c->m.rail_keys); free((void *)c->m.line_contact); free((void *)c->m.line_inner);
    free((void *)c->m.line_outer);
    free(c->x); free(c->y); free(c->x2); free(c->y2); free(c->Vx); free(c->Vy); free(c->count);
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 5; q++) free(c->par[b][q]);
    for (int b = 0; b < 2; b++)
        for (int q = 0; q < 16; q++) free(c->hpar[b][q]);
    free(c->Hn); free(c->Hu); free(c->Hv); free(c->HT); free(c->ku); free(c->kv_); free(c->kT);
    for (int q = 0; q < 3; q++) free(c->qfix[q]);
    free(c->inner);
    free(c);
}

void go_set_state(void *h, int buf, const double *ro, const double *p, const double *u, const double *v,
                  const double *Q) {
    ctx *c = (ctx *)h;
    size_t n = sizeof(double) * c->m.n_cells;
    memcpy(c->par[buf][0], ro, n);
    memcpy(c->par[buf][1], p, n);
    memcpy(c->par[buf][2], u, n);
    memcpy(c->par[buf][3], v, n);
    memcpy(c->par[buf][4], Q, n);
}

void go_get_state(void *h, int buf, double *ro, double *p, double *u, double *v, double *Q) {
    ctx *c = (ctx *)h;
    size_t n = sizeof(double) * c->m.n_cells;
    memcpy(ro, c->par[buf][0], n);
    memcpy(p, c->par[buf][1], n);
    memcpy(u, c->par[buf][2], n);
    memcpy(v, c->par[buf][3], n);
    memcpy(Q, c->par[buf][4], n);
}

void go_set_mc(void *h, const double *Hn, const double *Hu, const double *Hv, const double *HT, const double *ku,
               const double *kv, const double *kT) {
    ctx *c = (ctx *)h;
    size_t n = sizeof(double) * c->m.n_cells;
    memcpy(c->Hn, Hn, 4 * n);
    memcpy(c->Hu, Hu, 4 * n);
    memcpy(c->Hv, Hv, 4 * n);
    memcpy(c->HT, HT, 4 * n);
    memcpy(c->ku, ku, n);
    memcpy(c->kv_, kv, n);
    memcpy(c->kT, kT, n);
}

void go_set_inner_list(void *h, const int32_t *cells, int32_t n) {
    ctx *c = (ctx *)h;
    free(c->inner);
    c->inner = (int32_t *)dup(cells, sizeof(int32_t) * (n > 0 ? n : 1));
    c->n_inner_cells = n;
}

void go_get_points(void *h, double *x, double *y, double *x2, double *y2, double *Vx, double *Vy, int32_t *count) {
    ctx *c = (ctx *)h;
    size_t n = sizeof(double) * c->m.n_points;
    memcpy(x, c->x, n);
    memcpy(y, c->y, n);
    memcpy(x2, c->x2, n);
    memcpy(y2, c->y2, n);
    memcpy(Vx, c->Vx, n);
    memcpy(Vy, c->Vy, n);
    memcpy(count, c->count, sizeof(int32_t) * c->m.n_points);
}

void go_status(void *h, int64_t *out4) {
    ctx *c = (ctx *)h;
    out4[0] = c->status;
    out4[1] = c->n_ro_clamp;
    out4[2] = c->n_p_clamp;
    out4[3] = c->n_tvd_bad;
}

double go_last_dt(void *h) { return ((ctx *)h)->last_dt; }

double go_hllc(const go_params *prm, const double *L5, const double *R5, double W, double *P4, double *PQ, double n1,
               double n2, double rad, int metod, double *VlVcVp, int nul_potok) {
    return hllc(prm, L5[0], L5[1], L5[2], L5[3], L5[4], R5[0], R5[1], R5[2], R5[3], R5[4], W, P4, PQ, n1, n2, rad,
                metod, &VlVcVp[0], &VlVcVp[1], &VlVcVp[2], nul_potok);
}

double go_godunov(const go_params *prm, const double *q1, const double *q2, const double *n3, double *q5,
                  double *dsl_dsp_dsc, double w, double dist, int *status) {
    return godunov(prm, q1, q2, n3, q5, &dsl_dsp_dsc[0], &dsl_dsp_dsc[1], &dsl_dsp_dsc[2], w, dist, status);
}

/* ---------------------------------------------------------------- MHD fluxes
 * (the same two solvers as the device code; magnetic fields in Gaussian
 * units, scaled by 1/sqrt(4 pi) inside, Solvers.h:12) */
// Solvers::HLLDQ_Korolkov (Solvers.cpp:1642-2185).  L, R = (ro, Q, p, v1,
// v2, v3, Bx, By, Bz); the normal must be a coordinate axis (the tangent
// pair is picked from its sign and direction).  metod 2: HLLC-type MHD
// flux, metod 3: HLLD.  Pout[8] = mass, momentum x3, B flux x3, energy (the
// reference's final reordering), *PQ = flux of Q.  Returns kurant*rad/max|S|.
// Other metods leave Pout and *PQ untouched, as the reference does.
/* W: face speed at which the HLLD fan (metod 3) is sampled; the flux is then
 * F - W U of the region containing W (the moving-face treatment of
 * HLLC_2d_Korolkov_b_s, Setka.cpp:10604-10699).  W = 0 is the reference's
 * HLLDQ_Korolkov exactly (pinned by the golden vectors). */
static double hlldq(double ga, double kurant, const double* L, const double* R, double n1,
                    double n2, double n3, double rad, int metod, double* Pout, double* PQ, double W) {
    const double spi4 = sqrt(4.0 * PI_);
    const double g1 = ga - 1.0;
    const double ro_L = L[0], Q_L = L[1], p_L = L[2], v1_L = L[3], v2_L = L[4], v3_L = L[5];
    const double ro_R = R[0], Q_R = R[1], p_R = R[2], v1_R = R[3], v2_R = R[4], v3_R = R[5];
    const double bx_L = L[6] / spi4, by_L = L[7] / spi4, bz_L = L[8] / spi4;
    const double bx_R = R[6] / spi4, by_R = R[7] / spi4, bz_R = R[8] / spi4;
    double t1 = 0.0, t2 = 0.0, t3 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
    if (n1 > 0.1) {
        t2 = 1.0; m3 = 1.0;
    } else if (n2 > 0.1) {
        t3 = 1.0; m1 = 1.0;
    } else if (n3 > 0.1) {
        t1 = 1.0; m2 = 1.0;
    } else if (n1 < -0.1) {
        t3 = -1.0; m2 = -1.0;
    } else if (n2 < -0.1) {
        t1 = -1.0; m3 = -1.0;
    } else if (n3 < -0.1) {
        t1 = -1.0; m2 = -1.0;
    }
    const double u1 = v1_L * n1 + v2_L * n2 + v3_L * n3;
    const double v1 = v1_L * t1 + v2_L * t2 + v3_L * t3;
    const double w1 = v1_L * m1 + v2_L * m2 + v3_L * m3;
    const double u2 = v1_R * n1 + v2_R * n2 + v3_R * n3;
    const double v2 = v1_R * t1 + v2_R * t2 + v3_R * t3;
    const double w2 = v1_R * m1 + v2_R * m2 + v3_R * m3;
    const double bn1 = bx_L * n1 + by_L * n2 + bz_L * n3;
    const double bt1 = bx_L * t1 + by_L * t2 + bz_L * t3;
    const double bm1 = bx_L * m1 + by_L * m2 + bz_L * m3;
    const double bn2 = bx_R * n1 + by_R * n2 + bz_R * n3;
    const double bt2 = bx_R * t1 + by_R * t2 + bz_R * t3;
    const double bm2 = bx_R * m1 + by_R * m2 + bz_R * m3;
    const double bb_L = kv(bx_L) + kv(by_L) + kv(bz_L);
    const double bb_R = kv(bx_R) + kv(by_R) + kv(bz_R);
    const double uu_L = (kv(v1_L) + kv(v2_L) + kv(v3_L)) / 2.0;
    const double uu_R = (kv(v1_R) + kv(v2_R) + kv(v3_R)) / 2.0;
    const double cfL = sqrt((ga * p_L + bb_L + sqrt(kv(ga * p_L + bb_L) - 4.0 * ga * p_L * kv(bn1))) / (2.0 * ro_L));
    const double cfR = sqrt((ga * p_R + bb_R + sqrt(kv(ga * p_R + bb_R) - 4.0 * ga * p_R * kv(bn2))) / (2.0 * ro_R));
    const double SL = dmin(u1, u2) - dmax(cfL, cfR);
    const double SR = dmax(u1, u2) + dmax(cfL, cfR);
    const double pTL = p_L + bb_L / 2.0;
    const double pTR = p_R + bb_R / 2.0;
    const double suR = SR - u2, suL = SL - u1;
    const double SM = (suR * ro_R * u2 - suL * ro_L * u1 - pTR + pTL) / (suR * ro_R - suL * ro_L);
    const double PTT = (suR * ro_R * pTL - suL * ro_L * pTR + ro_L * ro_R * suR * suL * (u2 - u1)) /
                       (suR * ro_R - suL * ro_L);
    const double UU = dmax(fabs(SL), fabs(SR));
    const double time = kurant * rad / UU;
    if (metod != 2 && metod != 3) return time;
    const double e1 = p_L / g1 + ro_L * uu_L + bb_L / 2.0;
    const double e2 = p_R / g1 + ro_R * uu_R + bb_R / 2.0;
    const double FL[9] = {ro_L * u1,
                          ro_L * u1 * u1 + pTL - kv(bn1),
                          ro_L * u1 * v1 - bn1 * bt1,
                          ro_L * u1 * w1 - bn1 * bm1,
                          (e1 + pTL) * u1 - bn1 * (u1 * bn1 + v1 * bt1 + w1 * bm1),
                          0.0,
                          u1 * bt1 - v1 * bn1,
                          u1 * bm1 - w1 * bn1,
                          Q_L * u1};
    const double FR[9] = {ro_R * u2,
                          ro_R * u2 * u2 + pTR - kv(bn2),
                          ro_R * u2 * v2 - bn2 * bt2,
                          ro_R * u2 * w2 - bn2 * bm2,
                          (e2 + pTR) * u2 - bn2 * (u2 * bn2 + v2 * bt2 + w2 * bm2),
                          0.0,
                          u2 * bt2 - v2 * bn2,
                          u2 * bm2 - w2 * bn2,
                          Q_R * u2};
    const double UL[9] = {ro_L, ro_L * u1, ro_L * v1, ro_L * w1, e1, bn1, bt1, bm1, Q_L};
    const double UR[9] = {ro_R, ro_R * u2, ro_R * v2, ro_R * w2, e2, bn2, bt2, bm2, Q_R};
    const double bn = (SR * UR[5] - SL * UL[5] + FL[5] - FR[5]) / (SR - SL);
    const double bt = (SR * UR[6] - SL * UL[6] + FL[6] - FR[6]) / (SR - SL);
    const double bm = (SR * UR[7] - SL * UL[7] + FL[7] - FR[7]) / (SR - SL);
    const double bbn = bn * bn;
    const double ro_LL = ro_L * (SL - u1) / (SL - SM);
    const double ro_RR = ro_R * (SR - u2) / (SR - SM);
    const double Q_LL = Q_L * (SL - u1) / (SL - SM);
    const double Q_RR = Q_R * (SR - u2) / (SR - SM);
    double PO[9];
    if (metod == 2) {  // HLLC + MHD (Solvers.cpp:1817-1973)
        const double sbv1 = u1 * bn1 + v1 * bt1 + w1 * bm1;
        const double sbv2 = u2 * bn2 + v2 * bt2 + w2 * bm2;
        const double UZ0 = (SR * UR[0] - SL * UL[0] + FL[0] - FR[0]) / (SR - SL);
        const double UZ1 = (SR * UR[1] - SL * UL[1] + FL[1] - FR[1]) / (SR - SL);
        const double UZ2 = (SR * UR[2] - SL * UL[2] + FL[2] - FR[2]) / (SR - SL);
        const double UZ3 = (SR * UR[3] - SL * UL[3] + FL[3] - FR[3]) / (SR - SL);
        const double suRm = suR / (SR - SM);
        const double suLm = suL / (SL - SM);
        const double ptzR = pTR + ro_R * suR * (SM - u2);
        const double ptzL = pTL + ro_L * suL * (SM - u1);
        const double ptz = (ptzR + ptzL) / 2.0;
        const double vRR = UZ2 / UZ0, wRR = UZ3 / UZ0;
        const double vLL = vRR, wLL = wRR;
        const double btt2 = bt, bmm2 = bm, btt1 = btt2, bmm1 = bmm2;
        const double sbvz = (bn * UZ1 + bt * UZ2 + bm * UZ3) / UZ0;
        const double ee2 = e2 * suRm + (ptz * SM - pTR * u2 + bn * (sbv2 - sbvz)) / (SR - SM);
        const double ee1 = e1 * suLm + (ptz * SM - pTL * u1 + bn * (sbv1 - sbvz)) / (SL - SM);
        const double ULL[9] = {ro_LL, ro_LL * SM, ro_LL * vLL, ro_LL * wLL, ee1, bn, btt1, bmm1, Q_LL};
        const double URR[9] = {ro_RR, ro_RR * SM, ro_RR * vRR, ro_RR * wRR, ee2, bn, btt2, bmm2, Q_RR};
        for (int i = 0; i < 9; i++) PO[i] = 0.0;
        if (SL >= 0.0) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i];
        } else if (SL < 0.0 && SM >= 0.0) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] + SL * ULL[i] - SL * UL[i];
        } else if (SR > 0.0 && SM < 0.0) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] + SR * URR[i] - SR * UR[i];
        } else if (SR <= 0.0) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i];
        }
    } else {  // HLLD (Solvers.cpp:1975-2180)
        const double ttL = ro_L * suL * (SL - SM) - bbn;
        const double ttR = ro_R * suR * (SR - SM) - bbn;
        double vLL, wLL, vRR, wRR, btt1, bmm1, btt2, bmm2;
        if (fabs(ttL) >= 0.000001) {
            vLL = v1 - bn * bt1 * (SM - u1) / ttL;
            wLL = w1 - bn * bm1 * (SM - u1) / ttL;
            btt1 = bt1 * (ro_L * suL * suL - bbn) / ttL;
            bmm1 = bm1 * (ro_L * suL * suL - bbn) / ttL;
        } else {
            vLL = v1; wLL = w1; btt1 = 0.0; bmm1 = 0.0;
        }
        if (fabs(ttR) >= 0.000001) {
            vRR = v2 - bn * bt2 * (SM - u2) / ttR;
            wRR = w2 - bn * bm2 * (SM - u2) / ttR;
            btt2 = bt2 * (ro_R * suR * suR - bbn) / ttR;
            bmm2 = bm2 * (ro_R * suR * suR - bbn) / ttR;
        } else {
            vRR = v2; wRR = w2; btt2 = 0.0; bmm2 = 0.0;
        }
        const double eLL = (e1 * suL + PTT * SM - pTL * u1 +
                            bn * ((u1 * bn1 + v1 * bt1 + w1 * bm1) - (SM * bn + vLL * btt1 + wLL * bmm1))) /
                           (SL - SM);
        const double eRR = (e2 * suR + PTT * SM - pTR * u2 +
                            bn * ((u2 * bn2 + v2 * bt2 + w2 * bm2) - (SM * bn + vRR * btt2 + wRR * bmm2))) /
                           (SR - SM);
        const double sqrtroLL = sqrt(ro_LL), sqrtroRR = sqrt(ro_RR);
        double SLL = SM - fabs(bn) / sqrtroLL;
        double SRR = SM + fabs(bn) / sqrtroRR;
        double idbn;
        if (fabs(bn) > 0.001) {
            idbn = 1.0 * sgn(bn);
        } else {
            idbn = 0.0;
            SLL = SM;
            SRR = SM;
        }
        const double vLLL = (sqrtroLL * vLL + sqrtroRR * vRR + idbn * (btt2 - btt1)) / (sqrtroLL + sqrtroRR);
        const double wLLL = (sqrtroLL * wLL + sqrtroRR * wRR + idbn * (bmm2 - bmm1)) / (sqrtroLL + sqrtroRR);
        const double bttt = (sqrtroLL * btt2 + sqrtroRR * btt1 + idbn * sqrtroLL * sqrtroRR * (vRR - vLL)) /
                            (sqrtroLL + sqrtroRR);
        const double bmmm = (sqrtroLL * bmm2 + sqrtroRR * bmm1 + idbn * sqrtroLL * sqrtroRR * (wRR - wLL)) /
                            (sqrtroLL + sqrtroRR);
        const double eLLL = eLL - idbn * sqrtroLL * ((SM * bn + vLL * btt1 + wLL * bmm1) -
                                                     (SM * bn + vLLL * bttt + wLLL * bmmm));
        const double eRRR = eRR + idbn * sqrtroRR * ((SM * bn + vRR * btt2 + wRR * bmm2) -
                                                     (SM * bn + vLLL * bttt + wLLL * bmmm));
        const double ULL[9] = {ro_LL, ro_LL * SM, ro_LL * vLL, ro_LL * wLL, eLL, bn, btt1, bmm1, Q_LL};
        const double URR[9] = {ro_RR, ro_RR * SM, ro_RR * vRR, ro_RR * wRR, eRR, bn, btt2, bmm2, Q_RR};
        const double ULLL[9] = {ro_LL, ro_LL * SM, ro_LL * vLLL, ro_LL * wLLL, eLLL, bn, bttt, bmmm, Q_LL};
        const double URRR[9] = {ro_RR, ro_RR * SM, ro_RR * vLLL, ro_RR * wLLL, eRRR, bn, bttt, bmmm, Q_RR};
        for (int i = 0; i < 9; i++) PO[i] = 0.0;
        if (SL >= W) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] - W * UL[i];
        } else if (SL < W && SLL >= W) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] + SL * ULL[i] - SL * UL[i] - W * ULL[i];
        } else if (SLL <= W && SM >= W) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] + SLL * ULLL[i] - (SLL - SL) * ULL[i] - SL * UL[i] - W * ULLL[i];
        } else if (SM < W && SRR > W) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] + SRR * URRR[i] - (SRR - SR) * URR[i] - SR * UR[i] - W * URRR[i];
        } else if (SR > W && SRR <= W) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] + SR * URR[i] - SR * UR[i] - W * URR[i];
        } else if (SR <= W) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] - W * UR[i];
        }
    }
    const double SN = dmax(fabs(SL), fabs(SR));
    PO[5] = -SN * (bn2 - bn1) - W * bn;
    // back to (x, y, z), then the reference's reordering: B fluxes before energy
    Pout[0] = PO[0];
    Pout[1] = n1 * PO[1] + t1 * PO[2] + m1 * PO[3];
    Pout[2] = n2 * PO[1] + t2 * PO[2] + m2 * PO[3];
    Pout[3] = n3 * PO[1] + t3 * PO[2] + m3 * PO[3];
    Pout[4] = spi4 * (n1 * PO[5] + t1 * PO[6] + m1 * PO[7]);
    Pout[5] = spi4 * (n2 * PO[5] + t2 * PO[6] + m2 * PO[7]);
    Pout[6] = spi4 * (n3 * PO[5] + t3 * PO[6] + m3 * PO[7]);
    Pout[7] = PO[4];
    *PQ = PO[8];
    return time;
}

// Solvers::HLLD_Solver_Alexashov (Solvers.cpp:92-691).  q = (ro, p, u, v, w,
// bx, by, bz) in the (x, y, z) frame, n a unit normal (any direction: the
// frame is built from the mean field), face speed w.  The reference fixes
// n_state = 1 (Solvers.cpp:95), so the flux it returns is the HLL flux of
// the MHD system in the moving frame (Solvers.cpp:313-374); its n_state = 3
// branch is unreachable and is not restated.  q_out[8] = mass, momentum x3,
// B flux x3, energy; ds = dsl, dsp, dsc.  Where the reference exits
// (SR <= SL, or SM outside (SL, SR): Solvers.cpp:244-271) ST_WAVE_ORDER is
// raised instead.  Returns kurant*DIST/max(|dsl|, |dsp|).
static double hlld(double ga, double kurant, const double* qqq1, const double* qqq2,
                                        const double* n, double* qqq, double* ds, double wv, double DIST,
                                        int* status) {
    const double spi4 = sqrt(4.0 * PI_);
    const double eps = 10e-10;
    const double g1 = ga - 1.0;
    const double r1 = qqq1[0], u1 = qqq1[2], v1 = qqq1[3], w1 = qqq1[4], p1 = qqq1[1];
    const double bx1 = qqq1[5] / spi4, by1 = qqq1[6] / spi4, bz1 = qqq1[7] / spi4;
    const double r2 = qqq2[0], u2 = qqq2[2], v2 = qqq2[3], w2 = qqq2[4], p2 = qqq2[1];
    const double bx2 = qqq2[5] / spi4, by2 = qqq2[6] / spi4, bz2 = qqq2[7] / spi4;
    const double abx = (bx2 + bx1) / 2.0, aby = (by2 + by1) / 2.0, abz = (bz2 + bz1) / 2.0;
    const double bk = abx * n[0] + aby * n[1] + abz * n[2];
    const double b2 = kv(abx) + kv(aby) + kv(abz);
    double d = b2 - kv(bk);
    double aco[3][3];
    aco[0][0] = n[0];
    aco[1][0] = n[1];
    aco[2][0] = n[2];
    if (d > eps) {
        d = sqrt(d);
        aco[0][1] = (abx - bk * n[0]) / d;
        aco[1][1] = (aby - bk * n[1]) / d;
        aco[2][1] = (abz - bk * n[2]) / d;
        aco[0][2] = (aby * n[2] - abz * n[1]) / d;
        aco[1][2] = (abz * n[0] - abx * n[2]) / d;
        aco[2][2] = (abx * n[1] - aby * n[0]) / d;
    } else {
        double aix, aiy, aiz;
        if ((fabs(n[0]) < fabs(n[1])) && (fabs(n[0]) < fabs(n[2]))) {
            aix = 1.0; aiy = 0.0; aiz = 0.0;
        } else if (fabs(n[1]) < fabs(n[2])) {
            aix = 0.0; aiy = 1.0; aiz = 0.0;
        } else {
            aix = 0.0; aiy = 0.0; aiz = 1.0;
        }
        const double aik = aix * n[0] + aiy * n[1] + aiz * n[2];
        d = sqrt(1.0 - kv(aik));
        aco[0][1] = (aix - aik * n[0]) / d;
        aco[1][1] = (aiy - aik * n[1]) / d;
        aco[2][1] = (aiz - aik * n[2]) / d;
        aco[0][2] = (aiy * n[2] - aiz * n[1]) / d;
        aco[1][2] = (aiz * n[0] - aix * n[2]) / d;
        aco[2][2] = (aix * n[1] - aiy * n[0]) / d;
    }
    double vL[3], vR[3], bL[3], bR[3];
    for (int i = 0; i < 3; i++) {
        vL[i] = aco[0][i] * u1 + aco[1][i] * v1 + aco[2][i] * w1;
        vR[i] = aco[0][i] * u2 + aco[1][i] * v2 + aco[2][i] * w2;
        bL[i] = aco[0][i] * bx1 + aco[1][i] * by1 + aco[2][i] * bz1;
        bR[i] = aco[0][i] * bx2 + aco[1][i] * by2 + aco[2][i] * bz2;
    }
    const double aaL = bL[0] / sqrt(r1);
    const double b2L = kv(bL[0]) + kv(bL[1]) + kv(bL[2]);
    const double b21 = b2L / r1;
    const double cL = sqrt(ga * p1 / r1);
    double qp = sqrt(b21 + cL * (cL + 2.0 * aaL));
    double qm = sqrt(b21 + cL * (cL - 2.0 * aaL));
    const double cfL = (qp + qm) / 2.0;
    const double ptL = p1 + b2L / 2.0;
    const double aaR = bR[0] / sqrt(r2);
    const double b2R = kv(bR[0]) + kv(bR[1]) + kv(bR[2]);
    const double b22 = b2R / r2;
    const double cR = sqrt(ga * p2 / r2);
    qp = sqrt(b22 + cR * (cR + 2.0 * aaR));
    qm = sqrt(b22 + cR * (cR - 2.0 * aaR));
    const double cfR = (qp + qm) / 2.0;
    const double ptR = p2 + b2R / 2.0;
    const double SL = dmin((vL[0] - cfL), (vR[0] - cfR));
    const double SR = dmax((vL[0] + cfL), (vR[0] + cfR));
    const double suR = SR - vR[0], suL = SL - vL[0];
    const double SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    if (SR <= SL || SM >= SR || SM <= SL) *status |= 32; /* ST_WAVE_ORDER */
    ds[0] = SL;
    ds[1] = SR;
    ds[2] = SM;
    const double UU = dmax(fabs(SL), fabs(SR));
    const double time = kurant * DIST / UU;
    const double upt1 = (kv(u1) + kv(v1) + kv(w1)) / 2.0;
    const double sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const double upt2 = (kv(u2) + kv(v2) + kv(w2)) / 2.0;
    const double sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    const double e1 = p1 / g1 + r1 * upt1 + b2L / 2.0;
    const double e2 = p2 / g1 + r2 * upt2 + b2R / 2.0;
    const double FL[8] = {r1 * vL[0],
                          r1 * vL[0] * vL[0] + ptL - kv(bL[0]),
                          r1 * vL[0] * vL[1] - bL[0] * bL[1],
                          r1 * vL[0] * vL[2] - bL[0] * bL[2],
                          (e1 + ptL) * vL[0] - bL[0] * sbv1,
                          0.0,
                          vL[0] * bL[1] - vL[1] * bL[0],
                          vL[0] * bL[2] - vL[2] * bL[0]};
    const double FR[8] = {r2 * vR[0],
                          r2 * vR[0] * vR[0] + ptR - kv(bR[0]),
                          r2 * vR[0] * vR[1] - bR[0] * bR[1],
                          r2 * vR[0] * vR[2] - bR[0] * bR[2],
                          (e2 + ptR) * vR[0] - bR[0] * sbv2,
                          0.0,
                          vR[0] * bR[1] - vR[1] * bR[0],
                          vR[0] * bR[2] - vR[2] * bR[0]};
    const double UL[8] = {r1, r1 * vL[0], r1 * vL[1], r1 * vL[2], e1, bL[0], bL[1], bL[2]};
    const double UR[8] = {r2, r2 * vR[0], r2 * vR[1], r2 * vR[2], e2, bR[0], bR[1], bR[2]};
    double UZ[8], dq[8], FW[8];
    for (int ik = 0; ik < 8; ik++) {
        UZ[ik] = (SR * UR[ik] - SL * UL[ik] + FL[ik] - FR[ik]) / (SR - SL);
        dq[ik] = UR[ik] - UL[ik];
        FW[ik] = 0.0;
    }
    double TL = SL, TR = SR;
    if (SL > wv) {
        TL = 0.0;
        for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UL[ik];
    }
    if ((SL <= wv) && (wv <= SR))
        for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UZ[ik];
    if (SR < wv) {
        TR = 0.0;
        for (int ik = 0; ik < 8; ik++) FW[ik] = wv * UR[ik];
    }
    const double a = TR * TL, b = TR - TL;
    double qv[3], qb[3];
    const double q0 = (TR * FL[0] - TL * FR[0] + a * dq[0]) / b - FW[0];
    const double q4 = (TR * FL[4] - TL * FR[4] + a * dq[4]) / b - FW[4];
    for (int ik = 1; ik < 4; ik++) qv[ik - 1] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
    for (int ik = 5; ik < 8; ik++) qb[ik - 5] = (TR * FL[ik] - TL * FR[ik] + a * dq[ik]) / b - FW[ik];
    qqq[0] = q0;
    for (int i = 0; i < 3; i++) {
        qqq[i + 1] = aco[i][0] * qv[0] + aco[i][1] * qv[1] + aco[i][2] * qv[2];
        qqq[i + 4] = spi4 * (aco[i][0] * qb[0] + aco[i][1] * qb[1] + aco[i][2] * qb[2]);
    }
    qqq[7] = q4;
    return time;
}

double go_hlldq(const go_params *prm, const double *L9, const double *R9, double *P8, double *PQ, const double *n3,
                double rad, int metod) {
    return hlldq(prm->gamma, prm->kurant, L9, R9, n3[0], n3[1], n3[2], rad, metod, P8, PQ, 0.0);
}

double go_hlld(const go_params *prm, const double *q1, const double *q2, const double *n3, double *q8,
               double *dsl_dsp_dsc, double w, double dist, int *status) {
    return hlld(prm->gamma, prm->kurant, q1, q2, n3, q8, dsl_dsp_dsc, w, dist, status);
}

void go_face_par(void *h, int f, int which, int buf, double *out5) {
    ctx *c = (ctx *)h;
    st5 s = {0, 0, 0, 0, 0};
    if (which == 0) {
        s = get_par(c, f, buf);
    } else if (which == 1) {
        int M = c->m.face_master[f];
        if (M >= 0) s = cell_state(c, M, buf);
        get_par_tvd(c, f, buf, &s);
    } else {
        get_par_tvd_radial(c, f, buf, &s.ro, &s.p);
    }
    out5[0] = s.ro; out5[1] = s.p; out5[2] = s.u; out5[3] = s.v; out5[4] = s.Q;
}

void go_cell_geom(void *h, int k, double *out) {
    ctx *c = (ctx *)h;
    cell_center(c, k, 0, &out[0], &out[1]);
    cell_center(c, k, 1, &out[2], &out[3]);
    out[4] = cell_volume(c, k, 0);
    out[5] = cell_volume(c, k, 1);
    out[6] = cell_volume_rotate(c, k, 0, 360.0) / (2.0 * PI_);
    out[7] = cell_volume_rotate(c, k, 1, 360.0) / (2.0 * PI_);
}

void go_source_mk1(void *h, int k, double u, double v, double ro, double p, double *q3) {
    source_mk1((ctx *)h, k, u, v, ro, p, &q3[0], &q3[1], &q3[2]);
}

/* ================================================================== four hydrogen fluids
 * Setka::Go_5_komponent (Setka.cpp:8269-8950): the plasma and the four
 * hydrogen fluids H1..H4 of Parametr, each with its own HLLC flux per face
 * side, on the grid moved by Move_surface + Move_Setka_Calculate.  The
 * 21-field state is (ro, p, u, v, Q, ro_H1, p_H1, u_H1, v_H1, ..., v_H4),
 * the member order of Parametr's aggregate initialisers (Gran.cpp:262-265). */
enum { F_RO = 0, F_P, F_U, F_V, F_Q };
#define FH(k, j) (5 + 4 * (k) + (j)) /* hydrogen fluid k (0..3): j = 0 ro, 1 p, 2 u, 3 v */
#define H_POW 0.5                     /* Help.h:90 */
#define N_H_OVER_KN (1.0 / 6.0)       /* n_H_LISM_ / Kn_, Help.h:60, 65 */

typedef struct {
    double f[21];
} st21;

static st21 cell_state21(const ctx *c, int k, int buf) {
    st21 s;
    for (int q = 0; q < 5; q++) s.f[q] = c->par[buf][q][k];
    /* par rows are (ro, p, u, v, Q) */
    for (int q = 0; q < 16; q++) s.f[5 + q] = c->hpar[buf][q][k];
    return s;
}

static void mirror_v21(st21 *s) {
    s->f[F_V] = -s->f[F_V];
    for (int k = 0; k < 4; k++) s->f[FH(k, 3)] = -s->f[FH(k, 3)];
}

/* Inner_sphere state with the hydrogen fluids (Gran.cpp:236-265, 520-534):
 * plasma and H1 from the solar wind, H2..H4 from the master cell. */
static st21 inner_sphere21(const ctx *c, int f, int buf) {
    const go_params *P = &c->prm;
    st21 s = cell_state21(c, c->m.face_master[f], buf);
    double x, y;
    face_center(c, f, 0, &x, &y);
    double dist = sqrt(x * x + y * y);
    double ro = 1.0 / (kv(P->chi) * dist * dist);
    double P_E = ro * P->chi * P->chi / (P->gamma * P->inner_mach * P->inner_mach);
    s.f[F_RO] = ro;
    s.f[F_P] = P_E;
    s.f[F_U] = P->chi * x / dist;
    s.f[F_V] = P->chi * y / dist;
    s.f[F_Q] = ro;
    s.f[FH(0, 0)] = 0.0000001;
    s.f[FH(0, 1)] = (0.0000001 * P->chi * P->chi / (P->gamma * 14.1344 * 14.1344));
    s.f[FH(0, 2)] = P->chi * x / dist;
    s.f[FH(0, 3)] = P->chi * y / dist;
    return s;
}

/* Input state (Gran.cpp:267-276, 536-545): plasma and H4 from the LISM,
 * H1..H3 from the master cell. */
static st21 input21(const ctx *c, int f, int buf) {
    st21 s = cell_state21(c, c->m.face_master[f], buf);
    s.f[F_RO] = c->prm.in_ro;
    s.f[F_P] = c->prm.in_p;
    s.f[F_U] = c->prm.in_u;
    s.f[F_V] = c->prm.in_v;
    s.f[F_Q] = c->prm.in_Q;
    s.f[FH(3, 0)] = 1.0;
    s.f[FH(3, 1)] = 0.5;
    s.f[FH(3, 2)] = c->prm.in_u; /* Velosity_inf */
    s.f[FH(3, 3)] = 0.0;
    return s;
}

/* Gran::Get_par with the hydrogen fluids (Gran.cpp:205-289) */
static st21 get_par21(const ctx *c, int f, int buf) {
    int t = c->m.face_type[f];
    st21 s;
    memset(&s, 0, sizeof(s));
    if (t == T_USUALY) {
        s = cell_state21(c, c->m.face_sosed[f], buf);
    } else if (t == T_EXTERN) {
        s = cell_state21(c, c->m.face_master[f], buf);
        if (s.f[F_U] >= 0.0) s.f[F_U] = c->prm.extern_u_par;
    } else if (t == T_UPPER_WALL) {
        s = cell_state21(c, c->m.face_master[f], buf);
    } else if (t == T_AXIS) {
        s = cell_state21(c, c->m.face_master[f], buf);
        mirror_v21(&s);
    } else if (t == T_INNER_SPHERE) {
        s = inner_sphere21(c, f, buf);
    } else if (t == T_INPUT) {
        s = input21(c, f, buf);
    }
    return s;
}

/* Gran::Get_par_TVD with the hydrogen fluids (Gran.cpp:292-559) */
static void get_par_tvd21(ctx *c, int f, int buf, st21 *io) {
    int t = c->m.face_type[f];
    int M = c->m.face_master[f];
    if (t == T_USUALY) {
        int Sd = c->m.face_sosed_down[f];
        int So = c->m.face_sosed[f];
        if (Sd < 0) {
            if (cell_has_axis(c, M)) { /* Gran.cpp:308-338 */
                double x, y, x2, y2, dist1, dist2, dist3;
                st21 par = cell_state21(c, M, buf);
                face_center(c, f, 0, &x, &y);
                st21 par2 = cell_state21(c, M, buf);
                st21 par1 = par2;
                mirror_v21(&par1);
                st21 par3 = cell_state21(c, So, buf);
                cell_center(c, M, 0, &x2, &y2);
                dist2 = sqrt(kv(x - x2) + kv(y - y2));
                cell_center(c, So, 0, &x2, &y2);
                dist3 = sqrt(kv(x - x2) + kv(y - y2));
                cell_center(c, M, 0, &x2, &y2);
                y2 = -y2;
                dist1 = sqrt(kv(x - x2) + kv(y - y2));
                const int vi[5] = {F_V, FH(0, 3), FH(1, 3), FH(2, 3), FH(3, 3)};
                for (int q = 0; q < 5; q++)
                    par.f[vi[q]] = linear3(-dist1, par1.f[vi[q]], -dist2, par2.f[vi[q]], dist3, par3.f[vi[q]], 0.0);
                *io = par;
            } else {
                *io = cell_state21(c, M, buf);
            }
            return;
        }
        if (is_tracked_face(c, f)) { /* Gran.cpp:345-426 */
            double x, y, x2, y2, dist1, dist2;
            face_center(c, f, 0, &x, &y);
            st21 par2 = cell_state21(c, M, buf);
            st21 par1 = cell_state21(c, Sd, buf);
            cell_center(c, M, 0, &x2, &y2);
            dist2 = sqrt(kv(x - x2) + kv(y - y2));
            cell_center(c, Sd, 0, &x2, &y2);
            dist1 = sqrt(kv(x - x2) + kv(y - y2));
            for (int q = 0; q < 21; q++) io->f[q] = linear2(-dist1, par1.f[q], -dist2, par2.f[q], 0.0);
            if (io->f[F_RO] <= 0.0) io->f[F_RO] = par2.f[F_RO];
            if (io->f[F_P] <= 0.0) io->f[F_P] = par2.f[F_P];
            for (int k = 0; k < 4; k++) {
                if (io->f[FH(k, 0)] <= 0.0) io->f[FH(k, 0)] = par2.f[FH(k, 0)];
                if (io->f[FH(k, 1)] <= 0.0) io->f[FH(k, 1)] = par2.f[FH(k, 1)];
            }
            return;
        }
        /* Gran.cpp:427-472 */
        double x, y, x2, y2, dist1, dist2, dist3;
        face_center(c, f, 0, &x, &y);
        st21 par2 = cell_state21(c, M, buf);
        st21 par1 = cell_state21(c, Sd, buf);
        st21 par3 = cell_state21(c, So, buf);
        cell_center(c, M, 0, &x2, &y2);
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, So, 0, &x2, &y2);
        dist3 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, Sd, 0, &x2, &y2);
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
        for (int q = 0; q < 21; q++) io->f[q] = linear3(-dist1, par1.f[q], -dist2, par2.f[q], dist3, par3.f[q], 0.0);
        if (io->f[F_RO] <= 0.0 || io->f[F_P] <= 0.0) { /* reference: exit(-1), Gran.cpp:444-455 */
            c->status |= 2;
            c->n_tvd_bad++;
        }
    } else if (t == T_EXTERN) {
        *io = cell_state21(c, M, buf);
        if (io->f[F_U] >= 0.0) io->f[F_U] = c->prm.extern_u_tvd;
    } else if (t == T_UPPER_WALL) {
        *io = cell_state21(c, M, buf);
    } else if (t == T_AXIS) { /* Gran.cpp:486-519 */
        double x, y, x2, y2, dist1, dist2;
        int Sd = c->m.face_sosed_down[f];
        face_center(c, f, 0, &x, &y);
        st21 par2 = cell_state21(c, M, buf);
        st21 par1 = cell_state21(c, Sd, buf);
        cell_center(c, M, 0, &x2, &y2);
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, Sd, 0, &x2, &y2);
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
        *io = par2;
        const int vi[5] = {F_V, FH(0, 3), FH(1, 3), FH(2, 3), FH(3, 3)};
        for (int q = 0; q < 5; q++)
            io->f[vi[q]] = linear3(-dist1, par1.f[vi[q]], -dist2, par2.f[vi[q]], dist2, -par2.f[vi[q]], 0.0);
    } else if (t == T_INNER_SPHERE) {
        *io = inner_sphere21(c, f, buf);
    } else if (t == T_INPUT) {
        *io = input21(c, f, buf);
    }
}

/* Gran::Get_par_TVD_radial (Gran.cpp:562-675) with the H1 fields; the step
 * consumes ro, p, p_H1 and ro_H1 of it (Setka.cpp:8342-8349, 8368-8375). */
static void get_par_tvd_radial21(const ctx *c, int f, int buf, double *o) {
    const double g2 = 2.0 * c->prm.gamma;
    o[0] = o[1] = o[2] = o[3] = 0.0;
    if (c->m.face_type[f] != T_USUALY) return;
    int M = c->m.face_master[f], So = c->m.face_sosed[f], Sd = c->m.face_sosed_down[f];
    st21 par1, par2, par3;
    double x, y, x2, y2, dist1, dist2, dist3, r1, r2, r3;
    face_center(c, f, 0, &x, &y);
    double r = sqrt(kv(x) + kv(y));
    if (Sd < 0) {
        if (!cell_has_axis(c, M)) {
            st21 s = cell_state21(c, M, buf);
            o[0] = s.f[F_RO];
            o[1] = s.f[F_P];
            o[2] = s.f[FH(0, 1)];
            o[3] = s.f[FH(0, 0)];
            return;
        }
        /* Gran.cpp:580-626 */
        par2 = cell_state21(c, M, buf);
        par1 = par2;
        mirror_v21(&par1);
        par3 = cell_state21(c, So, buf);
        cell_center(c, M, 0, &x2, &y2);
        r2 = sqrt(kv(x2) + kv(y2));
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, So, 0, &x2, &y2);
        r3 = sqrt(kv(x2) + kv(y2));
        dist3 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, M, 0, &x2, &y2);
        y2 = -y2;
        r1 = sqrt(kv(x2) + kv(y2));
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
    } else {
        par2 = cell_state21(c, M, buf);
        par1 = cell_state21(c, Sd, buf);
        par3 = cell_state21(c, So, buf);
        cell_center(c, M, 0, &x2, &y2);
        r2 = sqrt(kv(x2) + kv(y2));
        dist2 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, So, 0, &x2, &y2);
        r3 = sqrt(kv(x2) + kv(y2));
        dist3 = sqrt(kv(x - x2) + kv(y - y2));
        cell_center(c, Sd, 0, &x2, &y2);
        r1 = sqrt(kv(x2) + kv(y2));
        dist1 = sqrt(kv(x - x2) + kv(y - y2));
    }
    o[0] = linear3(-dist1, par1.f[F_RO] * kv(r1), -dist2, par2.f[F_RO] * kv(r2), dist3, par3.f[F_RO] * kv(r3), 0.0) /
           kv(r);
    o[1] = linear3(-dist1, par1.f[F_P] * pow(r1, g2), -dist2, par2.f[F_P] * pow(r2, g2), dist3,
                   par3.f[F_P] * pow(r3, g2), 0.0) /
           pow(r, g2);
    o[2] = linear3(-dist1, par1.f[FH(0, 1)], -dist2, par2.f[FH(0, 1)], dist3, par3.f[FH(0, 1)], 0.0);
    o[3] = linear3(-dist1, par1.f[FH(0, 0)] * pow(r1, H_POW), -dist2, par2.f[FH(0, 0)] * pow(r2, H_POW), dist3,
                   par3.f[FH(0, 0)] * pow(r3, H_POW), 0.0) /
           pow(r, H_POW);
}

/* radial scaling of a side's state to the face centre (Setka.cpp:8337-8341) */
static void radial_scale21(st21 *s, double rc, double dis, double g2) {
    s->f[F_RO] = s->f[F_RO] * kv(rc) / kv(dis);
    s->f[FH(0, 0)] = s->f[FH(0, 0)] * pow(rc / dis, H_POW);
    s->f[F_Q] = s->f[F_Q] * kv(rc) / kv(dis);
    s->f[F_P] = s->f[F_P] * pow(rc / dis, g2);
}

/* conservative update of one hydrogen fluid (Setka.cpp:8808-8940) */
static void update_h(ctx *c, int k, int buf_out, int hk, const double *pot, double ro_H, double p_H, double u_H,
                     double v_H, double q1, double q21, double q22, double q3, double Volume, double Volume2, double y,
                     double dt, double ro_floor, double p_floor) {
    const double ggg = c->prm.gamma;
    double ro3 = ro_H * Volume / Volume2 - dt * (pot[0] / Volume2 + ro_H * v_H / y - q1);
    if (ro3 <= 0) {
        ro3 = ro_floor;
        c->n_ro_clamp++;
    }
    double u3 = (ro_H * u_H * Volume / Volume2 - dt * (pot[1] / Volume2 + ro_H * v_H * u_H / y - q21)) / ro3;
    double v3 = (ro_H * v_H * Volume / Volume2 - dt * (pot[2] / Volume2 + ro_H * v_H * v_H / y - q22)) / ro3;
    double p3 = (((p_H / (ggg - 1) + ro_H * (u_H * u_H + v_H * v_H) * 0.5) * Volume / Volume2 -
                  dt * (pot[3] / Volume2 + +v_H * (ggg * p_H / (ggg - 1) + ro_H * (u_H * u_H + v_H * v_H) * 0.5) / y -
                        q3)) -
                 0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                (ggg - 1);
    if (p3 <= 0) {
        p3 = p_floor;
        c->n_p_clamp++;
    }
    c->hpar[buf_out][4 * hk + 0][k] = ro3;
    c->hpar[buf_out][4 * hk + 1][k] = p3;
    c->hpar[buf_out][4 * hk + 2][k] = u3;
    c->hpar[buf_out][4 * hk + 3][k] = v3;
}

void go_set_hydrogen(void *h, int buf, const double *rows16) {
    ctx *c = (ctx *)h;
    const int nc = c->m.n_cells;
    for (int q = 0; q < 16; q++) memcpy(c->hpar[buf][q], rows16 + (size_t)q * nc, sizeof(double) * nc);
}

void go_get_hydrogen(void *h, int buf, double *rows16) {
    ctx *c = (ctx *)h;
    const int nc = c->m.n_cells;
    for (int q = 0; q < 16; q++) memcpy(rows16 + (size_t)q * nc, c->hpar[buf][q], sizeof(double) * nc);
}

/* Setka::Go_5_komponent: Setka.cpp:8269-8950 */
void go_5_komponent(void *h, int step) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double ggg = P->gamma, g2 = 2 * P->gamma;
    int now1 = 1, now2 = 0;
    double T[2];
    T[0] = T[1] = P->dt0;
    for (int st = 0; st < step; st++) {
        now1 = (now1 + 1) % 2;
        now2 = (now2 + 1) % 2;
        double time = 10000000;
        T[now2] = 100000000;
        go_move_surface(c, now1, T[now1]);
        go_move_setka1(c, T[now1]);
        for (int k = 0; k < c->m.n_cells; k++) {
            double Potok[5] = {0, 0, 0, 0, 0};
            double PH[4][4] = {{0}};
            double Pf[4], PQ = 0.0;
            st21 par1 = cell_state21(c, k, now1);
            double n1, n2, dist, x, y;
            cell_center(c, k, 0, &x, &y);
            double radius = sqrt(kv(x) + kv(y));
            if (radius < P->R11) continue;
            double Volume = cell_volume(c, k, 0);
            double Volume2 = cell_volume(c, k, 1);
            double W = 0.0;
            const int kt = c->m.cell_type[k];
            for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
                int f = c->m.gran[g];
                double x2, y2, x4, y4;
                double S = face_square(c, f);
                face_center(c, f, 0, &x2, &y2);
                face_center(c, f, 1, &x4, &y4);
                dist = sqrt(kv(x - x2) + kv(y - y2));
                st21 par11 = par1;
                st21 par2 = get_par21(c, f, now1);
                face_normal(c, f, &n1, &n2);
                double Vc, Vl, Vp;
                W = ((x4 - x2) * n1 + (y4 - y2) * n2) / T[now1];
                int met = 1;
                double dis = sqrt(kv(x2) + kv(y2));
                int ft = c->m.face_type[f];
                if (ft == T_USUALY) {
                    int So = c->m.face_sosed[f];
                    double x3, y3;
                    cell_center(c, So, 0, &x3, &y3);
                    double dd = sqrt(kv(x3) + kv(y3));
                    if (kt == C_1) {
                        radial_scale21(&par11, radius, dis, g2);
                        polar_perenos(x, y, x2, y2, &par11.f[F_U], &par11.f[F_V], TINY_ANGLE);
                        polar_perenos(x, y, x2, y2, &par11.f[FH(0, 2)], &par11.f[FH(0, 3)], TINY_ANGLE);
                        double o[4];
                        get_par_tvd_radial21(c, f, now1, o);
                        par11.f[F_RO] = o[0];
                        par11.f[F_P] = o[1];
                        par11.f[FH(0, 1)] = o[2];
                        par11.f[FH(0, 0)] = o[3];
                    } else {
                        get_par_tvd21(c, f, now1, &par11);
                    }
                    int fc = c->m.face_copy[f];
                    if (c->m.cell_type[So] == C_1) {
                        radial_scale21(&par2, dd, dis, g2);
                        polar_perenos(x3, y3, x2, y2, &par2.f[F_U], &par2.f[F_V], TINY_ANGLE);
                        polar_perenos(x3, y3, x2, y2, &par2.f[FH(0, 2)], &par2.f[FH(0, 3)], TINY_ANGLE);
                        double o[4];
                        get_par_tvd_radial21(c, fc, now1, o);
                        par2.f[F_RO] = o[0];
                        par2.f[F_P] = o[1];
                        par2.f[FH(0, 1)] = o[2];
                        par2.f[FH(0, 0)] = o[3];
                    } else {
                        get_par_tvd21(c, fc, now1, &par2);
                    }
                } else if (ft == T_INNER_SPHERE) {
                    radial_scale21(&par11, radius, dis, g2);
                } else if (kt == C_1 && ft == T_AXIS) {
                    radial_scale21(&par11, radius, dis, g2);
                    polar_perenos(x, y, x2, y2, &par11.f[F_U], &par11.f[F_V], TINY_ANGLE);
                    polar_perenos(x, y, x2, y2, &par11.f[FH(0, 2)], &par11.f[FH(0, 3)], TINY_ANGLE);
                    par2 = par11;
                    mirror_v21(&par2);
                } else if (kt != C_1 && ft == T_AXIS) {
                    get_par_tvd21(c, f, now1, &par11);
                    par2 = par11;
                    mirror_v21(&par2);
                }
                int np = face_np_flag(c, f);
                int god = is_tracked_face(c, f);
                for (int hk = 0; hk < 4; hk++) {
                    if (hk == 0 && kt == C_CENTR) continue;
                    time = dmin(time, hllc(P, par11.f[FH(hk, 0)], par11.f[F_Q], par11.f[FH(hk, 1)], par11.f[FH(hk, 2)],
                                           par11.f[FH(hk, 3)], par2.f[FH(hk, 0)], par2.f[F_Q], par2.f[FH(hk, 1)],
                                           par2.f[FH(hk, 2)], par2.f[FH(hk, 3)], W, Pf, &PQ, n1, n2, dist, met, &Vl,
                                           &Vc, &Vp, 0));
                    for (int q = 0; q < 4; q++) PH[hk][q] = PH[hk][q] + Pf[q] * S;
                }
                if (god) {
                    double Vl2, Vp2, VV, nn[3], q1[5], q2[5], qq[5];
                    nn[0] = n1; nn[1] = n2; nn[2] = 0.0;
                    q1[0] = par11.f[F_RO]; q1[1] = par11.f[F_P]; q1[2] = par11.f[F_U]; q1[3] = par11.f[F_V]; q1[4] = 0.0;
                    q2[0] = par2.f[F_RO]; q2[1] = par2.f[F_P]; q2[2] = par2.f[F_U]; q2[3] = par2.f[F_V]; q2[4] = 0.0;
                    int stt = 0;
                    time = dmin(time, godunov(P, q1, q2, nn, qq, &Vl2, &Vp2, &VV, W, dist, &stt));
                    c->status |= stt;
                    Potok[0] = Potok[0] + qq[0] * S;
                    Potok[1] = Potok[1] + qq[1] * S;
                    Potok[2] = Potok[2] + qq[2] * S;
                    Potok[3] = Potok[3] + qq[4] * S;
                    time = dmin(time, hllc(P, par11.f[F_RO], par11.f[F_Q], par11.f[F_P], par11.f[F_U], par11.f[F_V],
                                           par2.f[F_RO], par2.f[F_Q], par2.f[F_P], par2.f[F_U], par2.f[F_V], W, Pf,
                                           &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, np));
                    Potok[4] = Potok[4] + PQ * S;
                } else {
                    time = dmin(time, hllc(P, par11.f[F_RO], par11.f[F_Q], par11.f[F_P], par11.f[F_U], par11.f[F_V],
                                           par2.f[F_RO], par2.f[F_Q], par2.f[F_P], par2.f[F_U], par2.f[F_V], W, Pf,
                                           &PQ, n1, n2, dist, met, &Vl, &Vc, &Vp, np));
                    for (int q = 0; q < 4; q++) Potok[q] = Potok[q] + Pf[q] * S;
                    Potok[4] = Potok[4] + PQ * S;
                }
            }
            if (time < T[now2]) T[now2] = time;
            /* multi-fluid charge exchange (Setka.cpp:8575-8660) */
            const double u = par1.f[F_U], v = par1.f[F_V], ro = par1.f[F_RO], p = par1.f[F_P], Q = par1.f[F_Q];
            double UM[4], UH[4], nu[4], uH[4], vH[4], roH[4], pH[4];
            for (int hk = 0; hk < 4; hk++) {
                roH[hk] = par1.f[FH(hk, 0)];
                pH[hk] = par1.f[FH(hk, 1)];
                uH[hk] = par1.f[FH(hk, 2)];
                vH[hk] = par1.f[FH(hk, 3)];
            }
            for (int hk = 0; hk < 4; hk++)
                UM[hk] = sqrt(kv(u - uH[hk]) + kv(v - vH[hk]) + (64.0 / (9.0 * PI_)) * (p / ro + 2.0 * pH[hk] / roH[hk]));
            for (int hk = 0; hk < 4; hk++)
                UH[hk] = sqrt(kv(u - uH[hk]) + kv(v - vH[hk]) + (4.0 / PI_) * (p / ro + 2.0 * pH[hk] / roH[hk]));
            for (int hk = 0; hk < 4; hk++) {
                const double sigma = kv(1.0 - P->a_2 * log(UM[hk]));
                nu[hk] = ro * roH[hk] * UM[hk] * sigma;
            }
            const double cp = P->src_coef; /* n_p_LISM_ / Kn_ */
            const double q2_1 = cp * (nu[0] * (uH[0] - u) + nu[1] * (uH[1] - u) + nu[2] * (uH[2] - u) +
                                      nu[3] * (uH[3] - u));
            const double q2_2 = cp * (nu[0] * (vH[0] - v) + nu[1] * (vH[1] - v) + nu[2] * (vH[2] - v) +
                                      nu[3] * (vH[3] - v));
            double e[4];
            for (int hk = 0; hk < 4; hk++)
                e[hk] = nu[hk] * ((kv(uH[hk]) + kv(vH[hk]) - kv(u) - kv(v)) / 2.0 +
                                  (UH[hk] / UM[hk]) * (2.0 * pH[hk] / roH[hk] - p / ro));
            const double q3 = cp * (e[0] + e[1] + e[2] + e[3]);
            const double dt = T[now1];
            if (kt != C_CENTR) {
                double ro3 = ro * Volume / Volume2 - dt * (Potok[0] / Volume2 + ro * v / y);
                double Q33 = Q * Volume / Volume2 - (dt / Volume2) * Potok[4] - dt * Q * v / y;
                if (ro3 <= 0.0) {
                    ro3 = P->ro_floor;
                    c->n_ro_clamp++;
                }
                double u3 = (ro * u * Volume / Volume2 - dt * (Potok[1] / Volume2 + ro * v * u / y - q2_1)) / ro3;
                double v3 = (ro * v * Volume / Volume2 - dt * (Potok[2] / Volume2 + ro * v * v / y - q2_2)) / ro3;
                double p3 = (((p / (ggg - 1) + ro * (u * u + v * v) * 0.5) * Volume / Volume2 -
                              dt * (Potok[3] / Volume2 + +v * (ggg * p / (ggg - 1) + ro * (u * u + v * v) * 0.5) / y -
                                    q3)) -
                             0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                            (ggg - 1);
                if (p3 <= 0) {
                    p3 = P->p_floor;
                    c->n_p_clamp++;
                }
                write_state(c, k, now2, ro3, Q33, p3, u3, v3);
            } else {
                st5 s = cell_state(c, k, now1);
                write_state(c, k, now2, s.ro, s.Q, s.p, s.u, s.v);
            }
            /* sources of the hydrogen fluids (Setka.cpp:8734-8806) */
            int kk[4] = {0, 0, 0, 0};
            if (kt == C_CENTR || kt == C_1 || kt == C_2 || kt == C_3) {
                if (kt == C_1 || kt == C_CENTR) kk[0] = 1;
                else kk[1] = 1;
            } else {
                if (kt == C_4) kk[2] = 1;
                else kk[3] = 1;
            }
            const double S1 = nu[0] + nu[1] + nu[2] + nu[3];
            double s2[4];
            for (int hk = 0; hk < 4; hk++) s2[hk] = nu[hk] * ((kv(u) + kv(v)) / 2.0 + (UH[hk] / UM[hk]) * (p / ro));
            const double S2 = s2[0] + s2[1] + s2[2] + s2[3];
            for (int hk = 0; hk < 4; hk++) {
                const double q1h = N_H_OVER_KN * (kk[hk] * S1 - nu[hk]);
                const double q21h = N_H_OVER_KN * (kk[hk] * S1 * u - nu[hk] * uH[hk]);
                const double q22h = N_H_OVER_KN * (kk[hk] * S1 * v - nu[hk] * vH[hk]);
                const double q3h = N_H_OVER_KN * (kk[hk] * S2 - nu[hk] * ((kv(uH[hk]) + kv(vH[hk])) / 2.0 +
                                                                        (UH[hk] / UM[hk]) * 2.0 * (pH[hk] / roH[hk])));
                if (hk == 0 && kt == C_CENTR) {
                    for (int j = 0; j < 4; j++) c->hpar[now2][j][k] = c->hpar[now1][j][k];
                    continue;
                }
                /* floors: Setka.cpp:8817, 8829, 8859, 8871, 8893, 8905, 8927, 8939 */
                const double rf = hk == 0 ? 0.0000001 : 0.000001;
                const double pf = hk == 3 ? 0.0000001 : 0.000001;
                update_h(c, k, now2, hk, PH[hk], roH[hk], pH[hk], uH[hk], vH[hk], q1h, q21h, q22h, q3h, Volume,
                         Volume2, y, dt, rf, pf);
            }
        }
        go_commit_points(c);
    }
    c->last_dt = T[now2];
}

/* ------------------------------------------------------------------ MHD + pickup protons
 * The MHD form of the moving-grid step (GELIOS_FORM_MHD_PUI of the device
 * library).  No reference step exists: this is the project's definition,
 * assembled from the reference's parts:
 *   - grid motion, ion reconstruction and boundary states: go_mk2 above
 *     (Setka.cpp:10121-10482), run on the ion fluid's gas-dynamic rows;
 *   - extra rows (w, B, pickup protons): Get_par's boundary rules and
 *     Get_par_TVD's minmod stencil (Gran.cpp:205-473), first order in C_1
 *     cells and without a Sosed_down;
 *   - ion flux: hlldq (Solvers::HLLDQ_Korolkov, metod 3) in the face frame
 *     with its fan sampled at the face speed W (F - W U of the region that
 *     contains W, like HLLC_2d_Korolkov_b_s on moving faces);
 *   - pickup flux: hllc (HLLC_2d_Korolkov_b_s, metod 1);
 *   - update: the MK2 update with the axisymmetric terms of both fluids and
 *     the fixed charge-exchange sources.
 * Every face is evaluated from each side, as the reference's cell loops do. */
void go_set_mhd(void *h, int buf, const double *rows8) {
    ctx *c = (ctx *)h;
    const int nc = c->m.n_cells;
    for (int q = 0; q < 8; q++) memcpy(c->hpar[buf][q], rows8 + (size_t)q * nc, sizeof(double) * nc);
}
void go_get_mhd(void *h, int buf, double *rows8) {
    ctx *c = (ctx *)h;
    const int nc = c->m.n_cells;
    for (int q = 0; q < 8; q++) memcpy(rows8 + (size_t)q * nc, c->hpar[buf][q], sizeof(double) * nc);
}
void go_set_sources(void *h, const double *q1, const double *q2, const double *q3) {
    ctx *c = (ctx *)h;
    const int nc = c->m.n_cells;
    memcpy(c->qfix[0], q1, sizeof(double) * nc);
    memcpy(c->qfix[1], q2, sizeof(double) * nc);
    memcpy(c->qfix[2], q3, sizeof(double) * nc);
}

enum { X_W = 0, X_BX, X_BY, X_BZ, X_RO, X_P, X_U, X_V };
typedef struct {
    double f[8];
} ext8;

static ext8 cell_ext(const ctx *c, int k, int buf) {
    ext8 e;
    for (int q = 0; q < 8; q++) e.f[q] = c->hpar[buf][q][k];
    return e;
}

/* boundary rule of the extra rows across face f of its master cell */
static ext8 get_par_ext(const ctx *c, const go_mhd_params *mp, int f, int buf) {
    const go_params *P = &c->prm;
    const int t = c->m.face_type[f];
    ext8 e = cell_ext(c, c->m.face_master[f], buf);
    if (t == T_USUALY) {
        e = cell_ext(c, c->m.face_sosed[f], buf);
    } else if (t == T_EXTERN) {
        if (e.f[X_U] >= 0.0) e.f[X_U] = P->extern_u_par;
    } else if (t == T_AXIS) {
        e.f[X_W] = -e.f[X_W];
        e.f[X_BY] = -e.f[X_BY];
        e.f[X_BZ] = -e.f[X_BZ];
        e.f[X_V] = -e.f[X_V];
    } else if (t == T_INNER_SPHERE) {
        double x, y;
        face_center(c, f, 0, &x, &y);
        const double dist = sqrt(x * x + y * y);
        const st5 wind = inner_sphere_state(c, f);
        e.f[X_W] = 0.0;
        e.f[X_BX] = 0.0;
        e.f[X_BY] = 0.0;
        e.f[X_BZ] = mp->inner_bphi * (P->R1 / dist) * (y / dist);
        e.f[X_RO] = mp->pui_inner_ro * wind.ro;
        e.f[X_P] = mp->pui_inner_p * wind.p;
        e.f[X_U] = wind.u;
        e.f[X_V] = wind.v;
    } else if (t == T_INPUT) {
        e.f[X_W] = 0.0;
        e.f[X_BX] = mp->lism_bx;
        e.f[X_BY] = mp->lism_by;
        e.f[X_BZ] = mp->lism_bz;
        e.f[X_RO] = mp->pui_in_ro;
        e.f[X_P] = mp->pui_in_p;
        e.f[X_U] = P->in_u;
        e.f[X_V] = P->in_v;
    }
    return e;
}

/* Get_par_TVD's stencil (Gran.cpp:340-472) for the extra rows of a Usualy
 * face f seen from its master */
static ext8 get_par_tvd_ext(const ctx *c, int f, int buf) {
    const int M = c->m.face_master[f], So = c->m.face_sosed[f], Sd = c->m.face_sosed_down[f];
    ext8 own = cell_ext(c, M, buf);
    if (Sd < 0) return own;
    double x, y, x2, y2;
    face_center(c, f, 0, &x, &y);
    ext8 e1 = cell_ext(c, Sd, buf), o;
    cell_center(c, M, 0, &x2, &y2);
    const double dist2 = sqrt(kv(x - x2) + kv(y - y2));
    cell_center(c, Sd, 0, &x2, &y2);
    const double dist1 = sqrt(kv(x - x2) + kv(y - y2));
    if (is_tracked_face(c, f)) {
        for (int q = 0; q < 8; q++) o.f[q] = linear2(-dist1, e1.f[q], -dist2, own.f[q], 0.0);
    } else {
        ext8 e3 = cell_ext(c, So, buf);
        cell_center(c, So, 0, &x2, &y2);
        const double dist3 = sqrt(kv(x - x2) + kv(y - y2));
        for (int q = 0; q < 8; q++) o.f[q] = linear3(-dist1, e1.f[q], -dist2, own.f[q], dist3, e3.f[q], 0.0);
    }
    if (!(o.f[X_RO] > 0.0)) o.f[X_RO] = own.f[X_RO];
    if (!(o.f[X_P] > 0.0)) o.f[X_P] = own.f[X_P];
    return o;
}

/* ion flux through a face (n1, n2) moving with normal speed W: hlldq in the
 * face frame with its fan sampled at W (F - W U).  out: mass, mom x, mom y,
 * mom phi, energy, Bx, By, Bphi, Q; returns 1/max(|SL|,|SR|) */
static double mhd_flux(double ga, st5 iL, ext8 eL, st5 iR, ext8 eR, double n1, double n2, double W, double *out) {
    const double t1 = -n2, t2 = n1;
    double L[9] = {iL.ro, iL.Q, iL.p, iL.u * n1 + iL.v * n2, iL.u * t1 + iL.v * t2, eL.f[X_W],
                   eL.f[X_BX] * n1 + eL.f[X_BY] * n2, eL.f[X_BX] * t1 + eL.f[X_BY] * t2, eL.f[X_BZ]};
    double R[9] = {iR.ro, iR.Q, iR.p, iR.u * n1 + iR.v * n2, iR.u * t1 + iR.v * t2, eR.f[X_W],
                   eR.f[X_BX] * n1 + eR.f[X_BY] * n2, eR.f[X_BX] * t1 + eR.f[X_BY] * t2, eR.f[X_BZ]};
    double F[8], FQ;
    const double tinv = hlldq(ga, 1.0, L, R, 1.0, 0.0, 0.0, 1.0, 3, F, &FQ, W);
    out[0] = F[0];
    out[1] = n1 * F[1] + t1 * F[2];
    out[2] = n2 * F[1] + t2 * F[2];
    out[3] = F[3];
    out[4] = F[7];
    out[5] = n1 * F[4] + t1 * F[5];
    out[6] = n2 * F[4] + t2 * F[5];
    out[7] = F[6];
    out[8] = FQ;
    return tinv;
}

void go_mhd(void *h, const go_mhd_params *mp, int step) {
    ctx *c = (ctx *)h;
    const go_params *P = &c->prm;
    const double ggg = P->gamma, g2 = 2 * P->gamma;
    const double i4p = 1.0 / (4.0 * PI_), i8p = 1.0 / (8.0 * PI_);
    int now1 = 1, now2 = 0;
    double T[2];
    T[0] = T[1] = P->dt0;
    for (int st = 0; st < step; st++) {
        now1 = (now1 + 1) % 2;
        now2 = (now2 + 1) % 2;
        T[now2] = 100000000;
        go_move_surface(c, now1, T[now1]);
        go_move_setka2(c, T[now1]);
        for (int k = 0; k < c->m.n_cells; k++) {
            double time = 10000000;
            double Pt[13];
            for (int q = 0; q < 13; q++) Pt[q] = 0.0;
            st5 par1 = cell_state(c, k, now1);
            ext8 ex1 = cell_ext(c, k, now1);
            double x, y;
            cell_center(c, k, 0, &x, &y);
            double vs1 = cell_volume(c, k, 0);
            double vs2 = cell_volume(c, k, 1);
            double radius = sqrt(kv(x) + kv(y));
            if (radius < P->R11) continue;
            double Volume = cell_volume_rotate(c, k, 0, 360.0) / (2.0 * PI_);
            double Volume2 = cell_volume_rotate(c, k, 1, 360.0) / (2.0 * PI_);
            const int kt = c->m.cell_type[k];
            for (int g = c->m.gran_start[k]; g < c->m.gran_start[k + 1]; g++) {
                int f = c->m.gran[g];
                double x2, y2, x4, y4, n1, n2;
                double S = face_square(c, f) * (c->y[c->m.face_A[f]] + c->y[c->m.face_B[f]]) * 0.5;
                face_center(c, f, 0, &x2, &y2);
                face_center(c, f, 1, &x4, &y4);
                double dist = sqrt(kv(x - x2) + kv(y - y2));
                st5 par11 = par1;
                st5 par2 = get_par(c, f, now1);
                ext8 e11 = ex1;
                ext8 e2 = get_par_ext(c, mp, f, now1);
                face_normal(c, f, &n1, &n2);
                double W = ((x4 - x2) * n1 + (y4 - y2) * n2) / T[now1];
                double dis = sqrt(kv(x2) + kv(y2));
                int ft = c->m.face_type[f];
                if (ft == T_USUALY) {
                    int So = c->m.face_sosed[f];
                    double x3, y3;
                    cell_center(c, So, 0, &x3, &y3);
                    double dd = sqrt(kv(x3) + kv(y3));
                    if (kt == C_1) {
                        par11.ro = par11.ro * kv(radius) / kv(dis);
                        par11.Q = par11.Q * kv(radius) / kv(dis);
                        par11.p = par11.p * pow(radius / dis, g2);
                        polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                        double pro, pp;
                        get_par_tvd_radial(c, f, now1, &pro, &pp);
                        par11.ro = pro;
                        par11.p = pp;
                    } else {
                        get_par_tvd(c, f, now1, &par11);
                        e11 = get_par_tvd_ext(c, f, now1);
                    }
                    int fc = c->m.face_copy[f];
                    if (c->m.cell_type[So] == C_1) {
                        par2.ro = par2.ro * kv(dd) / kv(dis);
                        par2.Q = par2.Q * kv(dd) / kv(dis);
                        par2.p = par2.p * pow(dd / dis, g2);
                        polar_perenos(x3, y3, x2, y2, &par2.u, &par2.v, TINY_ANGLE);
                        double pro, pp;
                        get_par_tvd_radial(c, fc, now1, &pro, &pp);
                        par2.ro = pro;
                        par2.p = pp;
                    } else {
                        get_par_tvd(c, fc, now1, &par2);
                        e2 = get_par_tvd_ext(c, fc, now1);
                    }
                } else if (ft == T_INNER_SPHERE) {
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                } else if (kt == C_1 && ft == T_AXIS) {
                    par11.ro = par11.ro * kv(radius) / kv(dis);
                    par11.Q = par11.Q * kv(radius) / kv(dis);
                    par11.p = par11.p * pow(radius / dis, g2);
                    polar_perenos(x, y, x2, y2, &par11.u, &par11.v, TINY_ANGLE);
                    par2 = par11;
                    par2.v = -par2.v;
                } else if (kt != C_1 && ft == T_AXIS) {
                    get_par_tvd(c, f, now1, &par11);
                    par2 = par11;
                    par2.v = -par2.v;
                }
                double F[9];
                const double tI = mhd_flux(ggg, par11, e11, par2, e2, n1, n2, W, F);
                double Gp[4], GQ, Vl, Vc, Vp;
                const double tP = hllc(P, e11.f[X_RO], 0.0, e11.f[X_P], e11.f[X_U], e11.f[X_V], e2.f[X_RO], 0.0,
                                       e2.f[X_P], e2.f[X_U], e2.f[X_V], W, Gp, &GQ, n1, n2, dist, 1, &Vl, &Vc, &Vp, 0);
                time = dmin(time, P->kurant * dist * tI);
                time = dmin(time, tP);
                for (int q = 0; q < 9; q++) Pt[q] = Pt[q] + F[q] * S;
                for (int q = 0; q < 4; q++) Pt[9 + q] = Pt[9 + q] + Gp[q] * S;
            }
            if (time < T[now2]) T[now2] = time;
            if (kt == C_CENTR) {
                st5 s0 = cell_state(c, k, now1);
                write_state(c, k, now2, s0.ro, s0.Q, s0.p, s0.u, s0.v);
                for (int q = 0; q < 8; q++) c->hpar[now2][q][k] = ex1.f[q];
                continue;
            }
            const double dt = T[now1];
            const double Am = 0.5 * (vs1 + vs2);
            const double q1 = c->qfix[0][k], q2 = c->qfix[1][k], q3 = c->qfix[2][k];
            const double ro = par1.ro, p = par1.p, u = par1.u, v = par1.v, Q = par1.Q;
            const double w = ex1.f[X_W], bx = ex1.f[X_BX], by = ex1.f[X_BY], bz = ex1.f[X_BZ];
            const double bb = bx * bx + by * by + bz * bz;
            const double Sy = p + bb * i8p + ro * w * w - bz * bz * i4p;
            const double Sphi = -(ro * v * w - by * bz * i4p);
            const double Sbz = v * bz - w * by;
            double ro3 = ro * Volume / Volume2 - dt * (Pt[0] / Volume2);
            const double Q3 = Q * Volume / Volume2 - (dt / Volume2) * Pt[8];
            if (ro3 <= 0.0) {
                ro3 = P->ro_floor;
                c->n_ro_clamp++;
            }
            const double u3 = (ro * u * Volume / Volume2 - dt * (Pt[1] / Volume2 - q1)) / ro3;
            const double v3 = (ro * v * Volume / Volume2 - dt * ((Pt[2] - Sy * Am) / Volume2 - q2)) / ro3;
            const double w3 = (ro * w * Volume / Volume2 - dt * ((Pt[3] - Sphi * Am) / Volume2)) / ro3;
            const double E = p / (ggg - 1) + ro * (u * u + v * v + w * w) * 0.5 + bb * i8p;
            const double E3 = E * Volume / Volume2 - dt * (Pt[4] / Volume2 - q3);
            const double bx3 = bx * Volume / Volume2 - dt * (Pt[5] / Volume2);
            const double by3 = by * Volume / Volume2 - dt * (Pt[6] / Volume2);
            const double bz3 = bz * Volume / Volume2 - dt * ((Pt[7] - Sbz * Am) / Volume2);
            double p3 = (E3 - 0.5 * ro3 * (u3 * u3 + v3 * v3 + w3 * w3) - (bx3 * bx3 + by3 * by3 + bz3 * bz3) * i8p) *
                        (ggg - 1);
            if (p3 <= 0) {
                p3 = P->p_floor;
                c->n_p_clamp++;
            }
            const double rp = ex1.f[X_RO], pp = ex1.f[X_P], up = ex1.f[X_U], vp = ex1.f[X_V];
            double rp3 = rp * Volume / Volume2 - dt * (Pt[9] / Volume2);
            if (rp3 <= 0.0) {
                rp3 = P->ro_floor;
                c->n_ro_clamp++;
            }
            const double up3 = (rp * up * Volume / Volume2 - dt * (Pt[10] / Volume2)) / rp3;
            const double vp3 = (rp * vp * Volume / Volume2 - dt * ((Pt[11] - pp * Am) / Volume2)) / rp3;
            const double Ep = pp / (ggg - 1) + rp * (up * up + vp * vp) * 0.5;
            double pp3 = ((Ep * Volume / Volume2 - dt * (Pt[12] / Volume2)) - 0.5 * rp3 * (up3 * up3 + vp3 * vp3)) *
                         (ggg - 1);
            if (pp3 <= 0) {
                pp3 = P->p_floor;
                c->n_p_clamp++;
            }
            write_state(c, k, now2, ro3, Q3, p3, u3, v3);
            const double outx[8] = {w3, bx3, by3, bz3, rp3, pp3, up3, vp3};
            for (int q = 0; q < 8; q++) c->hpar[now2][q][k] = outx[q];
        }
        go_commit_points(c);
    }
    c->last_dt = T[now2];
}
