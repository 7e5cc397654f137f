// sm_100a kernels of the Gelios_2D plasma time step.
//
// One time step of Setka::Go_5_komponent__MK2 (Setka.cpp:10121-10482) is,
// on two streams:
//   mk2_recon_tracked_kernel  TVD states of the tracked face units (pre-motion)
//   mk2_tracked_solve_kernel  star pressures of the tracked faces' exact
//                             Riemann problems (warp per face)
//   mk2_source_kernel         charge-exchange source (Get_Sourse_MK1), 32
//                             cells per warp: a cell phase (one lane per
//                             cell), then a species phase (one lane per cell
//                             and hydrogen species)
//   surface_faces_kernel      Move_surface (Setka.cpp:3378-3844): exact
//                             Godunov speeds of the tracked faces (warp per
//                             face)
//   rails_kernel              node velocities of the key points, then
//                             Move_Setka_Calculate_2 (Setka.cpp:4324-4759):
//                             one CTA per rail
//   mk2_flux_tracked_kernel   tracked faces: HLL + the Riemann solution
//                             sampled at the moved face speed
//   mk2_tile_kernel           one tile of cells per block: reconstruction and
//                             HLL flux of every other face unit touching the
//                             tile (face speed from the moved points), slot
//                             fluxes in shared memory, then the per-cell sums
//                             in Grans order, the conservative ALE update,
//                             the next step's geometry cache, CFL block-min
//   commit_kernel             x = x2; dt of the next step
// Go_stationary (Setka.cpp:5205-5343) and
// Go_stationary_5_komponent_inner_MK2 (Setka.cpp:6999-7212) are
// stationary_cell_kernel / inner_cell_kernel + dt_finalize_kernel.
//
// Owner-computes: a thread owns a cell and sums its faces in the reference's
// Grans order, so no floating-point atomics are needed and results are
// deterministic run to run.  The CFL minimum is exact under any order
// (atomicMin on the bit pattern of non-negative doubles).
#include <cuda_runtime.h>

#include <cstdint>

#include <cooperative_groups.h>

#include "physics.cuh"
#include "step_kernels.cuh"

namespace cg = cooperative_groups;

// Minimum resident blocks per SM of the grid-wide moving-grid kernels
// (register caps: 128 threads x 65536/(128 x minBlocks) registers).
#ifndef GELIOS_SOURCE_MINB
#define GELIOS_SOURCE_MINB 10
#endif
// Source kernel arrangement: 32 cells per warp in a cell phase and a
// species phase (1), or four lanes per cell throughout (0).
#ifndef GELIOS_SOURCE_WARP
#define GELIOS_SOURCE_WARP 1
#endif

namespace gelios {

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ St5 load_state(const double* const* st, int c) {
    St5 s;
    s.ro = st[0][c];
    s.p = st[1][c];
    s.u = st[2][c];
    s.v = st[3][c];
    s.Q = st[4][c];
    return s;
}

// Cell::Get_Center (Cell.cpp:66-88) on coordinates X, Y.
__device__ __forceinline__ void centroid(const int32_t* contour, int n, const double* X, const double* Y, double& ox,
                                         double& oy) {
    double A = 0.0, Gx = 0.0, Gy = 0.0;
    int a = contour[0];
    double xa = X[a], ya = Y[a];
    const double x0 = xa, y0 = ya;
    for (int i = 0; i < n; i++) {
        double xb, yb;
        if (i + 1 == n) {
            xb = x0;
            yb = y0;
        } else {
            const int b = contour[i + 1];
            xb = X[b];
            yb = Y[b];
        }
        const double cr = xa * yb - ya * xb;
        A = A + cr;
        Gx = Gx + (xa + xb) * cr;
        Gy = Gy + (ya + yb) * cr;
        xa = xb;
        ya = yb;
    }
    A = A * 0.5;
    ox = Gx / (6.0 * A);
    oy = Gy / (6.0 * A);
}

// Cell::Get_Volume_rotate(360)/(2 pi) (Cell.cpp:188-206) on X, Y.
__device__ __forceinline__ double volume_rotate(const int32_t* contour, int n, const double* X, const double* Y) {
    double A = 0.0, G = 0.0;
    int a = contour[0];
    double xa = X[a], ya = Y[a];
    const double x0 = xa, y0 = ya;
    for (int i = 0; i < n; i++) {
        double xb, yb;
        if (i + 1 == n) {
            xb = x0;
            yb = y0;
        } else {
            const int b = contour[i + 1];
            xb = X[b];
            yb = Y[b];
        }
        const double cr = xa * yb - ya * xb;
        A = A + cr;
        G = G + (ya + yb) * cr;
        xa = xb;
        ya = yb;
    }
    A = A * 0.5;
    return fabs(A) * (1.0 / (6.0 * A)) * G * kPi * 360.0 / 180.0 / (2.0 * kPi);
}

// Cell::Get_Volume / Get_Volume_posle (Cell.cpp:146-186, 208-254).
// posle selects the arithmetic-mean centre of the non-quad branch.
__device__ double area(const int32_t* contour, int n, const int32_t* sA, const int32_t* sB, int g0, int g1,
                       const double* X, const double* Y, bool posle) {
    if (n == 4) {
        const int p0 = contour[0], p1 = contour[1], p2 = contour[2], p3 = contour[3];
        double a1 = X[p0] - X[p2];
        double a2 = Y[p0] - Y[p2];
        const double a = sqrt(sq(a1) + sq(a2));
        double b1 = X[p1] - X[p3];
        double b2 = Y[p1] - Y[p3];
        const double b = sqrt(sq(b1) + sq(b2));
        a1 = a1 / a;
        a2 = a2 / a;
        b1 = b1 / b;
        b2 = b2 / b;
        const double c = a1 * b1 + a2 * b2;
        const double s = sqrt(1 - sq(c));
        return 0.5 * a * b * s;
    }
    double x = 0.0, y = 0.0;
    if (!posle) {
        centroid(contour, n, X, Y, x, y);
    } else {
        for (int i = 0; i < n; i++) {
            x += X[contour[i]];
            y += Y[contour[i]];
        }
        x = x / (1.0 * n);
        y = y / (1.0 * n);
    }
    double S = 0.0;
    for (int g = g0; g < g1; g++) {
        const int pa = sA[g], pb = sB[g];
        const double a1 = sqrt(sq(X[pa] - x) + sq(Y[pa] - y));
        const double a2 = sqrt(sq(X[pb] - x) + sq(Y[pb] - y));
        const double a3 = sqrt(sq(X[pa] - X[pb]) + sq(Y[pa] - Y[pb]));
        const double p = (a1 + a2 + a3) / 2.0;
        S = S + sqrt(p * (p - a1) * (p - a2) * (p - a3));
    }
    return S;
}

// centroid, area (Get_Volume) and rotated volume of a quadrilateral whose
// corners (contour order) are in registers: the operations of centroid(),
// area() (n == 4) and volume_rotate() in the same order.
__device__ __forceinline__ void quad_geometry(const double (&X)[4], const double (&Y)[4], double& ox, double& oy,
                                              double& vs, double& vol) {
    double A = 0.0, Gx = 0.0, Gy = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const double xa = X[i], ya = Y[i], xb = X[(i + 1) & 3], yb = Y[(i + 1) & 3];
        const double cr = xa * yb - ya * xb;
        A = A + cr;
        Gx = Gx + (xa + xb) * cr;
        Gy = Gy + (ya + yb) * cr;
    }
    A = A * 0.5;
    ox = Gx / (6.0 * A);
    oy = Gy / (6.0 * A);
    vol = fabs(A) * (1.0 / (6.0 * A)) * Gy * kPi * 360.0 / 180.0 / (2.0 * kPi);
    double a1 = X[0] - X[2];
    double a2 = Y[0] - Y[2];
    const double a = sqrt(sq(a1) + sq(a2));
    double b1 = X[1] - X[3];
    double b2 = Y[1] - Y[3];
    const double bb = sqrt(sq(b1) + sq(b2));
    a1 = a1 / a;
    a2 = a2 / a;
    b1 = b1 / bb;
    b2 = b2 / bb;
    const double cc = a1 * b1 + a2 * b2;
    const double sn = sqrt(1 - sq(cc));
    vs = 0.5 * a * bb * sn;
}

// Inner_sphere BC state (Gran.cpp:234-265, 520-534) at face centre (x, y).
__device__ __forceinline__ St5 inner_sphere_state(const gelios_params& P, double x, double y) {
    const double dist = sqrt(x * x + y * y);
    const double ro = 1.0 / (sq(P.chi) * dist * dist);
    const double P_E = ro * P.chi * P.chi / (P.gamma * P.inner_mach * P.inner_mach);
    St5 s;
    s.ro = ro;
    s.p = P_E;
    s.u = P.chi * x / dist;
    s.v = P.chi * y / dist;
    s.Q = ro;
    return s;
}
__device__ __forceinline__ St5 input_state(const gelios_params& P) {
    St5 s;
    s.ro = P.in_ro;
    s.p = P.in_p;
    s.u = P.in_u;
    s.v = P.in_v;
    s.Q = P.in_Q;
    return s;
}

// Gran::Get_par (Gran.cpp:205-289) for a face of the owning cell `own`.
__device__ __forceinline__ St5 get_par(const gelios_params& P, int ft, const St5& own, const double* const* st,
                                       int nb, double fx, double fy) {
    St5 s = own;
    if (ft == G_USUALY) {
        s = load_state(st, nb);
    } else if (ft == G_EXTERN) {
        if (s.u >= 0.0) s.u = P.extern_u_par;
    } else if (ft == G_AXIS) {
        s.v = -s.v;
    } else if (ft == G_INNER_SPHERE) {
        s = inner_sphere_state(P, fx, fy);
    } else if (ft == G_INPUT) {
        s = input_state(P);
    }
    return s;
}

// dM, dS: distances from the face centre to the centroids of M and So (the
// face unit computes them for its CFL candidates; passed in, not recomputed).
__device__ St5 tvd_usualy_d(const double* const* st, const double* cx, const double* cy, double fx, double fy,
                            const St5& Ms, double Mx, double My, int So, int Sd, bool m_has_axis, bool tracked,
                            double dM, double dS, int* status) {
    if (Sd < 0) {
        St5 par = Ms;
        if (m_has_axis) {  // Gran.cpp:308-338
            const St5 par3 = load_state(st, So);
            const double dist2 = dM;
            const double dist3 = dS;
            const double dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
            par.v = linear3(-dist1, -Ms.v, -dist2, Ms.v, dist3, par3.v, 0.0);
        }
        return par;
    }
    const St5 par1 = load_state(st, Sd);
    const double dist2 = dM;
    if (tracked) {  // Gran.cpp:345-426
        const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
        // linear(-dist1, t1, -dist2, t2, 0) with one reciprocal
        const double r = 1.0 / (-dist1 - (-dist2)), x2 = -dist2;
        St5 o;
        o.ro = (par1.ro - Ms.ro) * r * (0.0 - x2) + Ms.ro;
        o.p = (par1.p - Ms.p) * r * (0.0 - x2) + Ms.p;
        o.u = (par1.u - Ms.u) * r * (0.0 - x2) + Ms.u;
        o.v = (par1.v - Ms.v) * r * (0.0 - x2) + Ms.v;
        o.Q = (par1.Q - Ms.Q) * r * (0.0 - x2) + Ms.Q;
        if (o.ro <= 0.0) o.ro = Ms.ro;
        if (o.p <= 0.0) o.p = Ms.p;
        return o;
    }
    const St5 par3 = load_state(st, So);
    const double dist3 = dS;
    const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    // linear(-dist1, t1, -dist2, t2, dist3, t3, 0) for the five fields
    const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3), x2 = -dist2;
    St5 o;
    o.ro = linear3r(par1.ro, Ms.ro, par3.ro, r12, r23, x2);
    o.p = linear3r(par1.p, Ms.p, par3.p, r12, r23, x2);
    o.u = linear3r(par1.u, Ms.u, par3.u, r12, r23, x2);
    o.v = linear3r(par1.v, Ms.v, par3.v, r12, r23, x2);
    o.Q = linear3r(par1.Q, Ms.Q, par3.Q, r12, r23, x2);
    if (o.ro <= 0.0 || o.p <= 0.0) *status |= ST_TVD_BAD;  // the reference exits (Gran.cpp:444-455)
    return o;
}

// Gran::Get_par_TVD (Gran.cpp:292-473) of a Usualy face seen from Master M
// (state Ms, centre Mx,My) with Sosed So and Sosed_down Sd.
__device__ St5 tvd_usualy(const double* const* st, const double* cx, const double* cy, double fx, double fy,
                          const St5& Ms, double Mx, double My, int So, int Sd, bool m_has_axis, bool tracked,
                          int* status) {
    const double dM = sqrt(sq(fx - Mx) + sq(fy - My));
    const double dS = (Sd < 0 && !m_has_axis) || (Sd >= 0 && tracked) ? 0.0 : sqrt(sq(fx - cx[So]) + sq(fy - cy[So]));
    return tvd_usualy_d(st, cx, cy, fx, fy, Ms, Mx, My, So, Sd, m_has_axis, tracked, dM, dS, status);
}

// Gran::Get_par_TVD of an Axis face (Gran.cpp:486-519).
__device__ __forceinline__ St5 tvd_axis(const double* const* st, const double* cx, const double* cy, double fx,
                                        double fy, const St5& Ms, double Mx, double My, int Sd) {
    St5 o = Ms;
    if (Sd < 0) return o;  // no TVD partner: the upload rejects such a grid for the MK2 form
    const St5 par1 = load_state(st, Sd);
    const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
    const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    o.v = linear3(-dist1, par1.v, -dist2, Ms.v, dist2, -Ms.v, 0.0);
    return o;
}

// Gran::Get_par_TVD_radial (Gran.cpp:562-675), ro and p only (the callers
// use no other field).  rp[c] = |centroid of c|^(2 gamma) is computed once
// per cell and step; pdis = |face centre|^(2 gamma) once per face (the
// reference evaluates pow at every use).
// r: |face centre|, r2 / r3: |centroid| of M / So, dM / dS: distances from
// the face centre to those centroids (computed by the face unit, passed in).
__device__ void tvd_radial_d(const double* const* st, const double* cx, const double* cy, const double* rp,
                             double fx, double fy, const St5& Ms, double Mx, double My, double rpM, int So, int Sd,
                             bool m_has_axis, double pdis, double r, double r2, double r3, double dM, double dS,
                             double& oro, double& op) {
    if (Sd < 0) {
        if (!m_has_axis) {
            oro = Ms.ro;
            op = Ms.p;
            return;
        }
        const St5 par3 = load_state(st, So);
        const double dist2 = dM;
        const double dist3 = dS;
        const double dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
        const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3);
        // the mirrored centre has the radius of M itself
        oro = linear3r(Ms.ro * sq(r2), Ms.ro * sq(r2), par3.ro * sq(r3), r12, r23, -dist2) / sq(r);
        op = linear3r(Ms.p * rpM, Ms.p * rpM, par3.p * rp[So], r12, r23, -dist2) / pdis;
        return;
    }
    const St5 par1 = load_state(st, Sd);
    const St5 par3 = load_state(st, So);
    const double dist2 = dM;
    const double dist3 = dS;
    const double dx = cx[Sd], dy = cy[Sd];
    const double r1 = sqrt(sq(dx) + sq(dy));
    const double dist1 = sqrt(sq(fx - dx) + sq(fy - dy));
    const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3);
    oro = linear3r(par1.ro * sq(r1), Ms.ro * sq(r2), par3.ro * sq(r3), r12, r23, -dist2) / sq(r);
    op = linear3r(par1.p * rp[Sd], Ms.p * rpM, par3.p * rp[So], r12, r23, -dist2) / pdis;
}
__device__ void tvd_radial(const double* const* st, const double* cx, const double* cy, const double* rp, double fx,
                           double fy, const St5& Ms, double Mx, double My, double rpM, int So, int Sd,
                           bool m_has_axis, double pdis, double& oro, double& op) {
    const double r = sqrt(sq(fx) + sq(fy));
    if (Sd < 0) {
        if (!m_has_axis) {
            oro = Ms.ro;
            op = Ms.p;
            return;
        }
        const St5 par3 = load_state(st, So);
        const double r2 = sqrt(sq(Mx) + sq(My));
        const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
        const double sx = cx[So], sy = cy[So];
        const double r3 = sqrt(sq(sx) + sq(sy));
        const double dist3 = sqrt(sq(fx - sx) + sq(fy - sy));
        const double dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
        const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3);
        // the mirrored centre has the radius of M itself
        oro = linear3r(Ms.ro * sq(r2), Ms.ro * sq(r2), par3.ro * sq(r3), r12, r23, -dist2) / sq(r);
        op = linear3r(Ms.p * rpM, Ms.p * rpM, par3.p * rp[So], r12, r23, -dist2) / pdis;
        return;
    }
    const St5 par1 = load_state(st, Sd);
    const St5 par3 = load_state(st, So);
    const double r2 = sqrt(sq(Mx) + sq(My));
    const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
    const double sx = cx[So], sy = cy[So];
    const double r3 = sqrt(sq(sx) + sq(sy));
    const double dist3 = sqrt(sq(fx - sx) + sq(fy - sy));
    const double dx = cx[Sd], dy = cy[Sd];
    const double r1 = sqrt(sq(dx) + sq(dy));
    const double dist1 = sqrt(sq(fx - dx) + sq(fy - dy));
    const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3);
    oro = linear3r(par1.ro * sq(r1), Ms.ro * sq(r2), par3.ro * sq(r3), r12, r23, -dist2) / sq(r);
    op = linear3r(par1.p * rp[Sd], Ms.p * rpM, par3.p * rp[So], r12, r23, -dist2) / pdis;
}

// Get_Sourse_MK1 (Cell.cpp:528-555): the pair of cells of k's radial chain
// whose r_istoch bracket the centroid radius rr (K_posle = Next(K_do)).
// Returns false (and raises ST_CHAIN) where the reference would follow a
// missing Back/Next link.
// `cached` (out): the cache entry read, so that the caller rewrites it only
// where the bracket changed.
__device__ bool source_bracket(const DevMesh& d, int k, double rr, int& K_do, int& K_posle, int* status,
                               int2* cached_out = nullptr) {
    K_do = d.cback[k];
    K_posle = d.cnext[k];
    const double ri = d.r_istoch[k];
    const int2 cpair = d.src_lo ? d.src_lo[k] : make_int2(-1, -1);
    if (cached_out) *cached_out = cpair;
    const int cached = cpair.x;
    if (cached >= 0) {
        // The reference walks the radial chain from the cell itself.  Along
        // a chain r_istoch increases strictly (checked at upload), so the
        // bracket it finds is unique: r[lo] <= rr < r[hi] when rr <
        // r_istoch, r[lo] < rr <= r[hi] otherwise, with hi = Next(lo).
        // Searching from last step's bracket finds the same pair in a step
        // or two.
        const bool caseA = rr < ri;
        {
            // the walk's first step, from the cached pair (hi = Next(lo)
            // cached too): both radii and the link the reference
            // dereferences are loaded together, one level of loads
            const int hi = cpair.y;
            const double rlo = d.r_istoch[cached], rhi = d.r_istoch[hi];
            const int link = caseA ? d.cback[cached] : d.cnext[hi];
            const bool below = caseA ? (rr < rlo) : !(rr > rlo);
            const bool above = caseA ? !(rr < rhi) : (rr > rhi);
            if (!below && !above) {
                if (link < 0) {
                    *status |= ST_CHAIN;
                    return false;
                }
                K_do = cached;
                K_posle = hi;
                return true;
            }
        }
        int lo = cached;
        int guard = 0;
        for (;;) {
            const int hi = d.cnext[lo];
            if (hi < 0 || ++guard > d.n_cells) {
                lo = -1;
                break;
            }
            const double rlo = d.r_istoch[lo], rhi = d.r_istoch[hi];
            const bool below = caseA ? (rr < rlo) : !(rr > rlo);
            const bool above = caseA ? !(rr < rhi) : (rr > rhi);
            if (below) {
                lo = d.cback[lo];
                if (lo < 0) break;
            } else if (above) {
                lo = hi;
            } else {
                break;
            }
        }
        // the reference dereferences Back of the lower cell (rr < r_istoch)
        // or Next of the upper cell (otherwise); a missing link is its crash
        if (lo < 0 || (caseA ? d.cback[lo] < 0 : d.cnext[d.cnext[lo]] < 0)) {
            *status |= ST_CHAIN;
            return false;
        }
        K_do = lo;
        K_posle = d.cnext[lo];
    } else if (rr < ri) {
        double r1 = ri;
        int guard = 0;
        while (r1 > rr) {
            if (K_do < 0 || ++guard > d.n_cells) {
                *status |= ST_CHAIN;
                return false;
            }
            r1 = d.r_istoch[K_do];
            K_do = d.cback[K_do];
        }
        if (K_do < 0) {
            *status |= ST_CHAIN;
            return false;
        }
        K_do = d.cnext[K_do];
        K_posle = K_do >= 0 ? d.cnext[K_do] : -1;
    } else {
        double r2 = ri;
        int guard = 0;
        while (r2 < rr) {
            if (K_posle < 0 || ++guard > d.n_cells) {
                *status |= ST_CHAIN;
                return false;
            }
            r2 = d.r_istoch[K_posle];
            K_posle = d.cnext[K_posle];
        }
        if (K_posle < 0) {
            *status |= ST_CHAIN;
            return false;
        }
        K_posle = d.cback[K_posle];
        K_do = K_posle >= 0 ? d.cback[K_posle] : -1;
    }
    if (K_do < 0 || K_posle < 0) {
        *status |= ST_CHAIN;
        return false;
    }
    return true;
}

// Monte-Carlo moments of species s seen by cell k (Cell.cpp:528-589): radial
// interpolation between the chain cells K_do and K_posle inside the source
// region, the cell's own moments outside it.  Also the k_u, k_v, k_T factors.
struct SrcMoments {
    double uH, vH, roH, pH, ku, kv, kT;
};
__device__ __forceinline__ SrcMoments source_moments(const DevMesh& d, int k, int s, bool interp, int K_do, int K_posle,
                                                     double rr, bool with_k = true) {
    SrcMoments m;
    if (interp) {
        const double r1 = d.r_istoch[K_do];
        const double r2 = d.r_istoch[K_posle];
        // linear(r1, t1, r2, t2, rr) with one reciprocal for all fields
        const double ir = 1.0 / (r1 - r2), dr = rr - r2;
        auto lin = [&](double t1, double t2) { return (t1 - t2) * ir * dr + t2; };
        m.uH = lin(d.Hu[4 * K_do + s], d.Hu[4 * K_posle + s]);
        m.vH = lin(d.Hv[4 * K_do + s], d.Hv[4 * K_posle + s]);
        m.roH = lin(d.Hn[4 * K_do + s], d.Hn[4 * K_posle + s]);
        const double TH = lin(d.HT[4 * K_do + s], d.HT[4 * K_posle + s]);
        m.ku = m.kv = m.kT = 0.0;
        if (with_k) {
            m.ku = lin(d.ku[K_do], d.ku[K_posle]);
            m.kv = lin(d.kv[K_do], d.kv[K_posle]);
            m.kT = lin(d.kT[K_do], d.kT[K_posle]);
        }
        m.pH = 0.5 * TH * m.roH;
    } else {
        m.uH = d.Hu[4 * k + s];
        m.vH = d.Hv[4 * k + s];
        m.roH = d.Hn[4 * k + s];
        m.pH = 0.5 * d.HT[4 * k + s] * d.Hn[4 * k + s];
        m.ku = with_k ? d.ku[k] : 0.0;
        m.kv = with_k ? d.kv[k] : 0.0;
        m.kT = with_k ? d.kT[k] : 0.0;
    }
    return m;
}

// Charge-exchange momentum / energy exchange rates of one species
// (Cell.cpp:590-660): nu_u, nu_v, nu_e before the sum over species.
__device__ __forceinline__ void source_rates(const gelios_params& P, SrcMoments m, double u, double v, double ro,
                                             double pro, double kin, double& nuu, double& nuv, double& nue) {
    if (m.roH <= 0.0) {
        m.roH = 0.0000001;
        m.pH = 0.0;
    }
    const double th = 2.0 * m.pH / m.roH;
    const double du2 = sq(u - m.uH) + sq(v - m.vH);
    const double UM = sqrt(du2 + (64.0 / (9.0 * kPi)) * (pro + th));
    const double UH = sqrt(du2 + (4.0 / kPi) * (pro + th));
    const double sig = sq(1.0 - P.a_2 * log(UM));
    const double nu = ro * m.roH * UM * sig;
    nuu = nu * (m.uH - u);
    nuv = nu * (m.vH - v);
    nue = nu * ((sq(m.uH) + sq(m.vH) - kin) / 2.0 + (UH / UM) * (th - pro));
}

// Cell::Get_Sourse_MK1 (Cell.cpp:498-665), one thread per cell.
__device__ void source_mk1(const DevMesh& d, const gelios_params& P, int k, double xx, double yy, double u, double v,
                           double ro, double p, double& q1, double& q2, double& q3, int* status) {
    const double rr = sqrt(sq(xx) + sq(yy));
    const bool interp = rr > P.src_rmin && rr < P.src_rmax && xx >= 0.0;
    int K_do = -1, K_posle = -1;
    if (interp) {
        if (!source_bracket(d, k, rr, K_do, K_posle, status)) {
            q1 = q2 = q3 = 0.0;
            return;
        }
        if (d.src_lo_out) d.src_lo_out[k] = make_int2(K_do, K_posle);
    }
    const double pro = p / ro;
    const double kin = sq(u) + sq(v);
    double nuu[4], nuv[4], nue[4];
    SrcMoments m;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        m = source_moments(d, k, s, interp, K_do, K_posle, rr);
        source_rates(P, m, u, v, ro, pro, kin, nuu[s], nuv[s], nue[s]);
    }
    const double Mu = P.src_coef * (nuu[0] + nuu[1] + nuu[2] + nuu[3]);
    const double Mv = P.src_coef * (nuv[0] + nuv[1] + nuv[2] + nuv[3]);
    const double MT = P.src_coef * (nue[0] + nue[1] + nue[2] + nue[3]);
    q1 = Mu * m.ku;
    q2 = Mv * m.kv;
    q3 = MT * m.kT;
}

// Block-level minimum of `t` (non-negative doubles; NaN ignored) folded into
// the device word acc with one atomicMin per block; clamp counters likewise.
__device__ __forceinline__ void block_reduce_commit(double t, int nro, int np_, int status, unsigned long long* acc,
                                                    unsigned long long* counters, int* status_word) {
    __shared__ double smin[32];
    __shared__ int sro[32], sp[32], sst[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ot = __shfl_down_sync(0xffffffffu, t, o);
        t = (ot < t) ? ot : t;
        nro += __shfl_down_sync(0xffffffffu, nro, o);
        np_ += __shfl_down_sync(0xffffffffu, np_, o);
        status |= __shfl_down_sync(0xffffffffu, status, o);
    }
    if (lane == 0) {
        smin[wid] = t;
        sro[wid] = nro;
        sp[wid] = np_;
        sst[wid] = status;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        t = lane < nw ? smin[lane] : __longlong_as_double(0x7ff0000000000000LL);
        nro = lane < nw ? sro[lane] : 0;
        np_ = lane < nw ? sp[lane] : 0;
        status = lane < nw ? sst[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ot = __shfl_down_sync(0xffffffffu, t, o);
            t = (ot < t) ? ot : t;
            nro += __shfl_down_sync(0xffffffffu, nro, o);
            np_ += __shfl_down_sync(0xffffffffu, np_, o);
            status |= __shfl_down_sync(0xffffffffu, status, o);
        }
        if (lane == 0) {
            if (t >= 0.0 && t < __longlong_as_double(0x7ff0000000000000LL))
                atomicMin(acc, static_cast<unsigned long long>(__double_as_longlong(t)));
            if (nro) atomicAdd(&counters[0], static_cast<unsigned long long>(nro));
            if (np_) atomicAdd(&counters[1], static_cast<unsigned long long>(np_));
            if (status) atomicOr(status_word, status);
        }
    }
}

// ------------------------------------------------------------------ kernels
__global__ void centroid_kernel(DevMesh d, const double* __restrict__ X, const double* __restrict__ Y, double* cx,
                                double* cy, double* rp, double g2, double* vs, double* vol) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.n_cells) return;
    const int s = d.cstart[c], n = d.cstart[c + 1] - s;
    double x, y;
    centroid(d.contour + s, n, X, Y, x, y);
    cx[c] = x;
    cy[c] = y;
    rp[c] = pow2g(sqrt(sq(x) + sq(y)), g2);
    if (vs) {
        vs[c] = area(d.contour + s, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], X, Y, false);
        vol[c] = volume_rotate(d.contour + s, n, X, Y);
    }
}

// ------------------------------------------------------------------ face units
// A face unit is one flux evaluation: an interior face (Usualy main face,
// evaluated once for both sides: the reference evaluates it from each side
// and the two results are the negatives of each other up to rounding,
// Setka.cpp:10195-10380) or a one-sided face (boundary types, evaluated for
// its owner only).  Each unit writes F*S into the per-slot flux buffer of the
// owner slot (and -F*S into the twin's slot of the neighbour), and folds the
// CFL candidates of the sides whose cell is updated this step into the dt
// word.  The cell kernels then sum their slots in Grans order.

// Geometry of a face unit as its owner sees it: face centre (x2, y2), unit
// normal (n1, n2) for the end points in the owner's order, |centre|^2, the
// face length S, and the distances owner centroid - face centre and
// neighbour centroid - face centre (0 without a neighbour).  The same
// expressions as Setka.cpp:5244-5306 (t = B - A normalised, n = (t2, -t1));
// the twin's view has the normal negated and the two distances swapped.
struct FaceGeo {
    double x2, y2, n1, n2, f2, S, dist, distn;
};
constexpr int kFaceGeoRows = 8;
__device__ __forceinline__ FaceGeo face_geo(double xa, double ya, double xb, double yb, double x, double y,
                                            bool has_nb, double x3, double y3) {
    FaceGeo f;
    f.x2 = (xa + xb) / 2.0;
    f.y2 = (ya + yb) / 2.0;
    double t1 = xb - xa, t2 = yb - ya;
    const double nn = sqrt(sq(t1) + sq(t2));
    f.S = nn;
    t1 = t1 / nn;
    t2 = t2 / nn;
    f.n1 = t2;
    f.n2 = -t1;
    f.f2 = sq(f.x2) + sq(f.y2);
    f.dist = sqrt(sq(x - f.x2) + sq(y - f.y2));
    f.distn = has_nb ? sqrt(sq(x3 - f.x2) + sq(y3 - f.y2)) : 0.0;
    return f;
}

// Go_stationary flux of one side (Setka.cpp:5244-5306): owner state `own`
// at centre (x, y), radius rad; face centre (x2, y2), normal (n1, n2) and
// |centre|^2 f2 as seen from the owner; neighbour (for Usualy faces)
// state, centre and radius rad_nb.  pfc: |face centre|^(2 gamma) if cached,
// else negative.
template <typename TF>
__device__ __forceinline__ double stationary_side(const gelios_params& P, int ft, const St5& own, double x, double y,
                                                  double rad, double rpo, double x2, double y2, double n1, double n2,
                                                  double f2, const St5& nbs, double x3, double y3, double rad_nb,
                                                  double rpn, double pfc, FluxOut<double>& F) {
    const double g2 = 2 * P.gamma;
    St5 par11 = own;
    St5 par2 = own;
    if (ft == G_USUALY) par2 = nbs;
    else if (ft == G_EXTERN) {
        if (par2.u >= 0.0) par2.u = P.extern_u_par;
    } else if (ft == G_AXIS) par2.v = -par2.v;
    else if (ft == G_INNER_SPHERE) par2 = inner_sphere_state(P, x2, y2);
    else if (ft == G_INPUT) par2 = input_state(P);
    if (rad < P.rad_stat && ft == G_USUALY) {
        const double pf = pfc >= 0.0 ? pfc : pow2g(sqrt(f2), g2);  // (rad/fr)^(2g) = rad^(2g) / fr^(2g)
        par11.ro = par11.ro * sq(rad) / f2;
        par2.ro = par2.ro * sq(rad_nb) / f2;
        par11.p = par11.p * (rpo / pf);
        par2.p = par2.p * (rpn / pf);
        polar_perenos(x, y, x2, y2, par11.u, par11.v);
        polar_perenos(x3, y3, x2, y2, par2.u, par2.v);
    } else if (ft == G_INNER_SPHERE) {
        par11.ro = par11.ro * sq(rad) / f2;
        par11.p = par11.p * (rpo / (pfc >= 0.0 ? pfc : pow2g(sqrt(f2), g2)));
    } else if (rad < P.rad_stat && ft == G_AXIS) {
        polar_perenos(x, y, x2, y2, par11.u, par11.v);
        par11.v = 0.0;
        par2 = par11;
    } else if (ft == G_AXIS) {
        par11.v = 0.0;
        par2 = par11;
    }
    return hllc_flux<TF>(P.gamma, P.kurant, par11, par2, 0.0, n1, n2, 1.0, 1, false, F);  // UU
}

// One Go_stationary face unit: slot fluxes of the owner (and of the twin)
// and the minimum of its CFL candidates (+inf if none).  Inlined into the
// per-step kernel and into the cooperative multi-step kernel; the two
// compilations may contract multiply-adds differently (last-bit
// differences, a non-inlined body costs 12% per step).
template <typename TF>
__device__ __forceinline__ double stationary_unit_body(const DevMesh& d, const gelios_params& P, const StepBuffers& b,
                                                       double* __restrict__ fl, int u) {
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    const size_t ng = d.n_slots;
    {
        const int g = d.u_slot[u], K = d.u_cell[u], gt = d.u_twin[u];
        const bool procK = !(d.cflags[K] & CF_CENTR);
        const int nb = gt >= 0 ? d.snb[g] : -1;
        const bool procN = nb >= 0 && !(d.cflags[nb] & CF_CENTR);
        if (procK || procN) {
            const int ft = d.sinfo[g] & SI_TYPE_MASK;
            const double x = b.cx[K], y = b.cy[K];
            const double rad = sqrt(sq(x) + sq(y));
            const St5 own = load_state(b.cur, K);
            St5 nbs = own;
            double x3 = 0.0, y3 = 0.0, radn = 0.0;
            if (nb >= 0) {
                nbs = load_state(b.cur, nb);
                x3 = b.cx[nb];
                y3 = b.cy[nb];
                radn = sqrt(sq(x3) + sq(y3));
            }
            FaceGeo f;
            if (b.ugeo) {
                const size_t nu = d.n_units;
                f.x2 = b.ugeo[u];
                f.y2 = b.ugeo[nu + u];
                f.n1 = b.ugeo[2 * nu + u];
                f.n2 = b.ugeo[3 * nu + u];
                f.f2 = b.ugeo[4 * nu + u];
                f.S = b.ugeo[5 * nu + u];
                f.dist = b.ugeo[6 * nu + u];
                f.distn = b.ugeo[7 * nu + u];
            } else {
                const int A = d.sA[g], B = d.sB[g];
                f = face_geo(d.X[A], d.Y[A], d.X[B], d.Y[B], x, y, nb >= 0, x3, y3);
            }
            const double S = f.S;
            FluxOut<double> F;
            const double rpK = b.rp[K], rpN = nb >= 0 ? b.rp[nb] : 0.0;
            const double pfc = b.upf ? b.upf[u] : -1.0;
            const double UU = stationary_side<TF>(P, ft, own, x, y, rad, rpK, f.x2, f.y2, f.n1, f.n2, f.f2, nbs, x3,
                                                  y3, radn, rpN, pfc, F);
            fl[0 * ng + g] = F.P0 * S;
            fl[1 * ng + g] = F.P1 * S;
            fl[2 * ng + g] = F.P2 * S;
            fl[3 * ng + g] = F.P3 * S;
            fl[4 * ng + g] = F.PQ * S;
            if (procK) tmin_u = dmin_ref(tmin_u, P.kurant * f.dist / UU);
            if (gt >= 0) {
                // the twin's evaluation mirrors this one unless the radial
                // scaling switches at rad_stat between the two cells
                const bool same = (rad < P.rad_stat) == (radn < P.rad_stat);
                if (same) {
                    fl[0 * ng + gt] = -(F.P0 * S);
                    fl[1 * ng + gt] = -(F.P1 * S);
                    fl[2 * ng + gt] = -(F.P2 * S);
                    fl[3 * ng + gt] = -(F.P3 * S);
                    fl[4 * ng + gt] = -(F.PQ * S);
                    if (procN) tmin_u = dmin_ref(tmin_u, P.kurant * f.distn / UU);
                } else {
                    FluxOut<double> G;
                    const double Un = stationary_side<TF>(P, ft, nbs, x3, y3, radn, rpN, f.x2, f.y2, -f.n1, -f.n2,
                                                          f.f2, own, x, y, rad, rpK, pfc, G);
                    fl[0 * ng + gt] = G.P0 * S;
                    fl[1 * ng + gt] = G.P1 * S;
                    fl[2 * ng + gt] = G.P2 * S;
                    fl[3 * ng + gt] = G.P3 * S;
                    fl[4 * ng + gt] = G.PQ * S;
                    if (procN) tmin_u = dmin_ref(tmin_u, P.kurant * f.distn / Un);
                }
            }
        }
    }
    return tmin_u;
}

template <typename TF>
__global__ void __launch_bounds__(128) stationary_unit_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                              double* __restrict__ fl) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    if (u < d.n_units) tmin_u = stationary_unit_body<TF>(d, P, b, fl, u);
    block_reduce_commit(tmin_u, 0, 0, 0, b.dt_acc, b.counters, b.status);
}

// Go_stationary cell update (Setka.cpp:5309-5341) of cell c from the summed
// slots; folds its `time` mark and clamps into tmark, nro, npc.
__device__ __forceinline__ void stationary_update_body(const DevMesh& d, const gelios_params& P, const StepBuffers& b,
                                                       const double* __restrict__ fl, int c, double& tmark, int& nro,
                                                       int& npc) {
    const size_t ng = d.n_slots;
    if (!(d.cflags[c] & CF_CENTR)) {
        tmark = dmin_ref(tmark, 10000000.0);  // `time` starts at 1e7 in every step (Setka.cpp:5222)
        const double dt = *b.dt_cur;
        const St5 par1 = load_state(b.cur, c);
        const double y = b.cy[c];
        const int g0 = d.gstart[c], g1 = d.gstart[c + 1];
        double Pt0 = 0.0, Pt1 = 0.0, Pt2 = 0.0, Pt3 = 0.0, Pt4 = 0.0;
        for (int g = g0; g < g1; g++) {
            Pt0 = Pt0 + fl[0 * ng + g];
            Pt1 = Pt1 + fl[1 * ng + g];
            Pt2 = Pt2 + fl[2 * ng + g];
            Pt3 = Pt3 + fl[3 * ng + g];
            Pt4 = Pt4 + fl[4 * ng + g];
        }
        // the cell's area: cached with the centroids (the plain grid does not
        // move), or computed here when no cache is given
        double Volume;
        if (b.vs) {
            Volume = b.vs[c];
        } else {
            const int s0 = d.cstart[c], n = d.cstart[c + 1] - s0;
            Volume = area(d.contour + s0, n, d.sA, d.sB, g0, g1, d.X, d.Y, false);
        }
        const double gm1 = P.gamma - 1;
        double ro3 = par1.ro - dt * (Pt0 / Volume + par1.ro * par1.v / y);
        const double Q33 = par1.Q - (dt / Volume) * Pt4 - dt * par1.Q * par1.v / y;
        if (ro3 <= 0) {
            ro3 = P.ro_floor;
            nro++;
        }
        const double uu = par1.u * par1.u + par1.v * par1.v;
        const double u3 = (par1.ro * par1.u - dt * (Pt1 / Volume + par1.ro * par1.v * par1.u / y)) / ro3;
        const double v3 = (par1.ro * par1.v - dt * (Pt2 / Volume + par1.ro * par1.v * par1.v / y)) / ro3;
        double p3 = (((par1.p / gm1 + par1.ro * uu * 0.5) -
                      dt * (Pt3 / Volume + par1.v * (P.gamma * par1.p / gm1 + par1.ro * uu * 0.5) / y)) -
                     0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                    gm1;
        if (p3 <= 0) {
            p3 = P.p_floor;
            npc++;
        }
        b.nxt[0][c] = ro3;
        b.nxt[1][c] = p3;
        b.nxt[2][c] = u3;
        b.nxt[3][c] = v3;
        b.nxt[4][c] = Q33;
    }
}

__global__ void __launch_bounds__(128) stationary_update_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                                const double* __restrict__ fl) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double tmark = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0;
    if (c < d.n_cells) stationary_update_body(d, P, b, fl, c, tmark, nro, npc);
    block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
}

// `nsteps` Go_stationary steps in one cooperative launch: every block
// strides over the face units, then (grid barrier) over the cells, then
// (barrier) one thread turns the CFL minimum into the next step's dt
// (barrier).  The same unit and cell bodies as the three-kernel path; the
// grid is sized to be fully resident (cooperative launch).  21 us per step
// against 29 us for three launches per step on the 180 x 120 grid.
// bs[0] / bs[1]: the buffers of even / odd steps.
template <typename TF>
__global__ void __launch_bounds__(128) stationary_persistent_kernel(DevMesh d, gelios_params P, StepBuffers b0,
                                                                    StepBuffers b1, double* __restrict__ fl,
                                                                    int nsteps) {
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    for (int st = 0; st < nsteps; st++) {
        const StepBuffers& b = (st & 1) ? b1 : b0;
        double tmin = __longlong_as_double(0x7ff0000000000000LL);
        for (int u = tid; u < d.n_units; u += nth) tmin = dmin_ref(tmin, stationary_unit_body<TF>(d, P, b, fl, u));
        block_reduce_commit(tmin, 0, 0, 0, b.dt_acc, b.counters, b.status);
        grid.sync();
        double tmark = __longlong_as_double(0x7ff0000000000000LL);
        int nro = 0, npc = 0;
        for (int c = tid; c < d.n_cells; c += nth) stationary_update_body(d, P, b, fl, c, tmark, nro, npc);
        block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
        grid.sync();
        if (tid == 0) {
            const unsigned long long a = *b.dt_acc;
            *b.dt_next = (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
            *b.dt_acc = 0x7ff0000000000000ULL;
        }
        grid.sync();
    }
}

// `nsteps` Go_stationary steps of many instances in one cooperative launch.
// The instances share the mesh (topology and geometry) and have their own
// parameters (inflow and inner-wind states), state buffers, flux slots and
// dt words.  Work is dealt in 128-wide tiles of one instance each, so every
// block folds its CFL minimum into one instance's dt word; after the cell
// phase one thread per instance turns its minimum into the next dt.  The
// unit and cell bodies are the one-instance kernels'.  `active` lists the
// instances advanced by this launch (the others keep their state).
template <typename TF>
__global__ void __launch_bounds__(128) stationary_batch_kernel(DevMesh d, const PlainInstance* __restrict__ inst,
                                                               const int* __restrict__ active, int n_active,
                                                               int nsteps) {
    cg::grid_group grid = cg::this_grid();
    const int ut = (d.n_units + 127) / 128, ct = (d.n_cells + 127) / 128;
    for (int st = 0; st < nsteps; st++) {
        const int par = st & 1;
        for (int t = blockIdx.x; t < n_active * ut; t += gridDim.x) {
            const PlainInstance& I = inst[active[t / ut]];
            const int u = (t % ut) * 128 + threadIdx.x;
            double tmin = __longlong_as_double(0x7ff0000000000000LL);
            if (u < d.n_units) tmin = stationary_unit_body<TF>(d, I.P, I.b[par], I.fl, u);
            __syncthreads();  // the previous tile's reduction has read its shared words
            block_reduce_commit(tmin, 0, 0, 0, I.b[par].dt_acc, I.b[par].counters, I.b[par].status);
        }
        grid.sync();
        for (int t = blockIdx.x; t < n_active * ct; t += gridDim.x) {
            const PlainInstance& I = inst[active[t / ct]];
            const int c = (t % ct) * 128 + threadIdx.x;
            double tmark = __longlong_as_double(0x7ff0000000000000LL);
            int nro = 0, npc = 0;
            if (c < d.n_cells) stationary_update_body(d, I.P, I.b[par], I.fl, c, tmark, nro, npc);
            __syncthreads();
            block_reduce_commit(tmark, nro, npc, 0, I.b[par].dt_acc, I.b[par].counters, I.b[par].status);
        }
        grid.sync();
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_active; k += gridDim.x * blockDim.x) {
            const StepBuffers& b = inst[active[k]].b[par];
            const unsigned long long a = *b.dt_acc;
            *b.dt_next = (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
            *b.dt_acc = 0x7ff0000000000000ULL;
        }
        grid.sync();
    }
}

// Go_5_komponent__MK2 face reconstruction of one side (Setka.cpp:10213-10276)
// for a Usualy face: owner M (state Ms, centre Mx,My, flags mf), across the
// face the cell So; Sd = Sosed_down of the face as seen from M.
__device__ __forceinline__ St5 mk2_usualy_side(const double* const* st, const double* cx, const double* cy,
                                               const double* rp, double fx, double fy, double dis, double pdis,
                                               const St5& Ms, double Mx, double My, double rpM, uint32_t mf, int So,
                                               int Sd, bool tracked, int* status) {
    if (mf & CF_C1) {
        const double radius = sqrt(sq(Mx) + sq(My));
        St5 o = Ms;
        o.ro = o.ro * sq(radius) / sq(dis);
        o.Q = o.Q * sq(radius) / sq(dis);
        o.p = o.p * (rpM / pdis);
        polar_perenos(Mx, My, fx, fy, o.u, o.v);
        tvd_radial(st, cx, cy, rp, fx, fy, Ms, Mx, My, rpM, So, Sd, (mf & CF_AXIS) != 0, pdis, o.ro, o.p);
        return o;
    }
    return tvd_usualy(st, cx, cy, fx, fy, Ms, Mx, My, So, Sd, (mf & CF_AXIS) != 0, tracked, status);
}
// The same for a face unit that has computed the distances already: rM, rS
// = |centroid| of M and So, dM, dS = face centre to those centroids.
__device__ __forceinline__ St5 mk2_usualy_side_d(const double* const* st, const double* cx, const double* cy,
                                                 const double* rp, double fx, double fy, double dis, double pdis,
                                                 const St5& Ms, double Mx, double My, double rpM, uint32_t mf, int So,
                                                 int Sd, bool tracked, double rM, double rS, double dM, double dS,
                                                 int* status) {
    if (mf & CF_C1) {
        const double radius = rM;
        St5 o = Ms;
        o.ro = o.ro * sq(radius) / sq(dis);
        o.Q = o.Q * sq(radius) / sq(dis);
        o.p = o.p * (rpM / pdis);
        polar_perenos(Mx, My, fx, fy, o.u, o.v);
        tvd_radial_d(st, cx, cy, rp, fx, fy, Ms, Mx, My, rpM, So, Sd, (mf & CF_AXIS) != 0, pdis, dis, rM, rS, dM, dS,
                     o.ro, o.p);
        return o;
    }
    return tvd_usualy_d(st, cx, cy, fx, fy, Ms, Mx, My, So, Sd, (mf & CF_AXIS) != 0, tracked, dM, dS, status);
}

// One MK2 face unit before the grid moves (Setka.cpp:10204-10276): the two
// reconstructed face states (TVD / radial TVD / boundary states), the face
// normal, S = |AB| (yA + yB) / 2, the face centre and the two CFL distances
// (negative: that side is not updated this step).  Everything here reads the
// points before the motion (X, Y) and the cached centroids, never the moved
// points, so it may run before or after the rails.
struct RecUnit {
    St5 a, o;                  // owner side, other side
    double n1, n2, S, x2, y2;  // face normal, S, face centre
    double dist, distn;        // owner / other centroid to the face centre, -1 if not updated
};

// L1 prefetch of one global address (no register, no wait).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// Prefetch into L1 of everything mk2_recon_unit / mk2_flux_unit gather for
// face unit u: state rows and centroids of the owner, the neighbour and both
// Sosed_down cells (and |c|^(2 gamma) where RP: the radial reconstruction),
// the end points before and after the motion.
template <bool RP>
__device__ __forceinline__ void mk2_prefetch_unit(const DevMesh& d, const StepBuffers& b, int u) {
    const int K = d.u_cell[u], nb = d.u_nb[u], A = d.u_A[u], B = d.u_B[u];
    const int sd = d.u_sd[u], sd2 = d.u_sd2[u];
    auto cell = [&](int c) {
#pragma unroll
        for (int k = 0; k < 5; k++) prefetch_l1(b.cur[k] + c);
        prefetch_l1(b.cx + c);
        prefetch_l1(b.cy + c);
        if (RP) prefetch_l1(b.rp + c);
    };
    cell(K);
    if (nb >= 0) cell(nb);
    if (sd >= 0) cell(sd);
    if (sd2 >= 0) cell(sd2);
    prefetch_l1(d.X + A);
    prefetch_l1(d.Y + A);
    prefetch_l1(d.X + B);
    prefetch_l1(d.Y + B);
    prefetch_l1(d.X2 + A);
    prefetch_l1(d.Y2 + A);
    prefetch_l1(d.X2 + B);
    prefetch_l1(d.Y2 + B);
}

// GROUP: the unit group the caller knows the unit to be in, so that branches
// drop out at compile time: kPlainGroup [0, u_c1) (a Usualy face, neither
// cell C_1, not tracked), kC1Group [u_c1, u_tr0) (a Usualy face with a C_1
// side, not tracked), kAnyGroup (no assumption).
constexpr int kPlainGroup = 0, kC1Group = 1, kAnyGroup = 2;
template <int GROUP = kAnyGroup>
__device__ __forceinline__ void mk2_recon_unit(const DevMesh& d, const gelios_params& P, const StepBuffers& b, int u,
                                               RecUnit& r, int* status) {
    constexpr bool PLAIN = GROUP == kPlainGroup, USUALY = GROUP != kAnyGroup;
    const int K = d.u_cell[u], nb = d.u_nb[u];
    const uint32_t info = d.u_info[u];
    const double x = b.cx[K], y = b.cy[K];
    // centroid radii (where a radial reconstruction needs them) and
    // face-centre-to-centroid distances, computed once for the R11 test, the
    // CFL candidates and both reconstructions
    const double aK = sq(x) + sq(y);
    const bool procK = !(aK < d.r11_sq);
    const double rK = PLAIN ? 0.0 : sqrt(aK);
    double x3 = 0.0, y3 = 0.0, rN = 0.0;
    bool procN = false;
    if (nb >= 0) {
        x3 = b.cx[nb];
        y3 = b.cy[nb];
        const double aN = sq(x3) + sq(y3);
        procN = !(aN < d.r11_sq);
        rN = PLAIN ? 0.0 : sqrt(aN);
    }
    const int A = d.u_A[u], B = d.u_B[u];
    const double xa = d.X[A], ya = d.Y[A], xb = d.X[B], yb = d.Y[B];
    const double x2 = (xa + xb) / 2.0, y2 = (ya + yb) / 2.0;
    const double dK = sqrt(sq(x - x2) + sq(y - y2));
    const double dN = sqrt(sq(x3 - x2) + sq(y3 - y2));
    {
        double t1 = xb - xa, t2 = yb - ya;
        const double nn = sqrt(sq(t1) + sq(t2));
        t1 = t1 / nn;
        t2 = t2 / nn;
        r.n1 = t2;
        r.n2 = -t1;
        r.S = sqrt(sq(xb - xa) + sq(yb - ya)) * (ya + yb) * 0.5;
        r.x2 = x2;
        r.y2 = y2;
        r.dist = procK ? dK : -1.0;
        r.distn = procN ? dN : -1.0;
    }
    if (!(procK || procN)) return;
    const int ft = USUALY ? static_cast<int>(G_USUALY) : static_cast<int>(info & SI_TYPE_MASK);
    const uint32_t cf = (info >> UI_CF_OWN) & (PLAIN ? (15u & ~CF_C1) : 15u);
    const double g2 = 2 * P.gamma;
    const St5 par1 = load_state(b.cur, K);
    St5 par11 = par1;
    St5 par2 = get_par(P, ft, par1, b.cur, nb, x2, y2);
    const double dis = sqrt(sq(x2) + sq(y2));
    const bool tracked = !USUALY && (info & SI_GOD) != 0;
    const uint32_t nbf = (info >> UI_CF_NB) & (PLAIN ? (15u & ~CF_C1) : 15u);
    const bool radial = ((cf & CF_C1) && (ft == G_USUALY || ft == G_AXIS)) || ft == G_INNER_SPHERE ||
                        (ft == G_USUALY && (nbf & CF_C1));
    const double pdis = radial ? pow2g(dis, g2) : 1.0;
    if (ft == G_USUALY) {
        r.a = mk2_usualy_side_d(b.cur, b.cx, b.cy, b.rp, x2, y2, dis, pdis, par1, x, y, b.rp[K], cf, nb, d.u_sd[u],
                                tracked, rK, rN, dK, dN, status);
        r.o = mk2_usualy_side_d(b.cur, b.cx, b.cy, b.rp, x2, y2, dis, pdis, par2, x3, y3, b.rp[nb], nbf, K,
                                d.u_sd2[u], tracked, rN, rK, dN, dK, status);
        return;
    }
    if (ft == G_INNER_SPHERE) {
        const double radius = rK;
        par11.ro = par11.ro * sq(radius) / sq(dis);
        par11.Q = par11.Q * sq(radius) / sq(dis);
        par11.p = par11.p * (b.rp[K] / pdis);
    } else if (ft == G_AXIS) {
        if (cf & CF_C1) {
            const double radius = rK;
            par11.ro = par11.ro * sq(radius) / sq(dis);
            par11.Q = par11.Q * sq(radius) / sq(dis);
            par11.p = par11.p * (b.rp[K] / pdis);
            polar_perenos(x, y, x2, y2, par11.u, par11.v);
        } else {
            par11 = tvd_axis(b.cur, b.cx, b.cy, x2, y2, par1, x, y, d.u_sd[u]);
        }
        par2 = par11;
        par2.v = -par2.v;
    }
    r.a = par11;
    r.o = par2;
}

// The flux of one MK2 face unit once the grid has moved (Setka.cpp:10198-10209,
// 10335-10393): face speed W from the moved points, HLL (`metod 0`), exact
// Godunov sampled at W on tracked faces (star pressure pstar solved before the
// motion), F.S to the owner slot and -F.S to the twin slot, CFL candidates.
template <typename TF, bool TRACKED>
__device__ __forceinline__ void mk2_flux_unit(const DevMesh& d, const gelios_params& P, const StepBuffers& b, int u,
                                              const RecUnit& r, double* __restrict__ fl, const double* pstar,
                                              double& tmin_u, int* status) {
    const bool procK = !(r.dist < 0.0), procN = !(r.distn < 0.0);
    if (!(procK || procN)) return;
    const size_t ng = d.n_slots;
    const double dt = *b.dt_cur;
    const int A = d.u_A[u], B = d.u_B[u];
    const double x4 = (d.X2[A] + d.X2[B]) / 2.0, y4 = (d.Y2[A] + d.Y2[B]) / 2.0;
    const double W = ((x4 - r.x2) * r.n1 + (y4 - r.y2) * r.n2) / dt;
    const int g = d.u_slot[u], gt = d.u_twin[u];
    const bool np = (d.u_info[u] & SI_NP) != 0;
    FluxOut<double> F;
    const double UU = hllc_flux<TF>(P.gamma, P.kurant, r.a, r.o, W, r.n1, r.n2, 1.0, 0, np, F);
    const double S = r.S;
    double fm0 = F.P0 * S, fm1 = F.P1 * S, fm2 = F.P2 * S, fm3 = F.P3 * S;
    double UG = 1.0;
    if (TRACKED) {
        double q1[5] = {r.a.ro, r.a.p, r.a.u, r.a.v, 0.0};
        double q2[5] = {r.o.ro, r.o.p, r.o.u, r.o.v, 0.0};
        double nv[3] = {r.n1, r.n2, 0.0};
        double qq[5], ds[3];
        UG = godunov_dev<false>(P.gamma, P.kurant, q1, q2, nv, qq, ds, W, 1.0, P.godunov_max_iter, status, pstar);
        fm0 = qq[0] * S;
        fm1 = qq[1] * S;
        fm2 = qq[2] * S;
        fm3 = qq[4] * S;
    }
    const double fq = F.PQ * S;
    // the slots are read once, by the update: streaming stores keep the
    // gathered cell data in L2
    __stcs(fl + 0 * ng + g, fm0);
    __stcs(fl + 1 * ng + g, fm1);
    __stcs(fl + 2 * ng + g, fm2);
    __stcs(fl + 3 * ng + g, fm3);
    __stcs(fl + 4 * ng + g, fq);
    if (procK) {
        // reference order: Godunov candidate first, then HLL (Setka.cpp:10359, 10366)
        if (TRACKED) tmin_u = dmin_ref(tmin_u, P.kurant * r.dist / UG);
        tmin_u = dmin_ref(tmin_u, P.kurant * r.dist / UU);
    }
    if (gt >= 0) {
        __stcs(fl + 0 * ng + gt, -fm0);
        __stcs(fl + 1 * ng + gt, -fm1);
        __stcs(fl + 2 * ng + gt, -fm2);
        __stcs(fl + 3 * ng + gt, -fm3);
        __stcs(fl + 4 * ng + gt, -fq);
        if (procN) {
            if (TRACKED) tmin_u = dmin_ref(tmin_u, P.kurant * r.distn / UG);
            tmin_u = dmin_ref(tmin_u, P.kurant * r.distn / UU);
        }
    }
}

// Rows of the tracked units' reconstruction (kRecRows rows of n_tracked
// doubles; row r of tracked unit i at rec[r * n_tracked + i]).
__device__ __forceinline__ void rec_store(double* __restrict__ rec, size_t n, int i, const RecUnit& r) {
    const double v[kRecRows] = {r.a.ro, r.a.p, r.a.u, r.a.v, r.a.Q, r.o.ro, r.o.p, r.o.u, r.o.v,
                                r.o.Q, r.n1,  r.n2,  r.S,   r.x2,  r.y2,  r.dist, r.distn};
#pragma unroll
    for (int k = 0; k < kRecRows; k++) rec[k * n + i] = v[k];
}
__device__ __forceinline__ RecUnit rec_load(const double* __restrict__ rec, size_t n, int i) {
    RecUnit r;
    r.a.ro = rec[0 * n + i];
    r.a.p = rec[1 * n + i];
    r.a.u = rec[2 * n + i];
    r.a.v = rec[3 * n + i];
    r.a.Q = rec[4 * n + i];
    r.o.ro = rec[5 * n + i];
    r.o.p = rec[6 * n + i];
    r.o.u = rec[7 * n + i];
    r.o.v = rec[8 * n + i];
    r.o.Q = rec[9 * n + i];
    r.n1 = rec[10 * n + i];
    r.n2 = rec[11 * n + i];
    r.S = rec[12 * n + i];
    r.x2 = rec[13 * n + i];
    r.y2 = rec[14 * n + i];
    r.dist = rec[15 * n + i];
    r.distn = rec[16 * n + i];
    return r;
}

// The tracked face units (grouped in [u_tr0, u_tr1)) are reconstructed before
// the motion: their exact Riemann problems are solved while the grid moves.
__global__ void __launch_bounds__(128) mk2_recon_tracked_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                                double* __restrict__ rec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = d.u_tr1 - d.u_tr0;
    int status = 0;
    if (i < nt) {
        RecUnit r;
        r.a = St5{};
        r.o = St5{};
        mk2_recon_unit(d, P, b, d.u_tr0 + i, r, &status);
        rec_store(rec, nt, i, r);
    }
    if (status) atomicOr(b.status, status);
}

// Tracked units after the motion: sampling of the solved Riemann problems
// at the face speed (one thread per unit).
template <typename TF>
__global__ void __launch_bounds__(32) mk2_flux_tracked_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                              const double* __restrict__ rec, double* __restrict__ fl,
                                                              const double* __restrict__ pstar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = d.u_tr1 - d.u_tr0;
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    int status = 0;
    if (i < nt) {
        const RecUnit r = rec_load(rec, nt, i);
        mk2_flux_unit<TF, true>(d, P, b, d.u_tr0 + i, r, fl, pstar + i, tmin_u, &status);
    }
    block_reduce_commit(tmin_u, 0, 0, status, b.dt_acc, b.counters, b.status);
}

// Every other face unit after the motion, reconstruction and flux in one
// pass: the reconstructed states stay in registers (no per-unit scratch);
// F.S to the owner's flux slot and -F.S to the twin's.  Index i is remapped
// around the tracked range [u_tr0, u_tr1).
// One launch per unit group (compiled without the branches the group cannot
// take): kPlainGroup [0, u_c1), kC1Group [u_c1, u_tr0), kAnyGroup the
// one-sided units [u_tr1, n_units).
// PF: every gathered address of the unit is prefetched into L1 as soon as
// the unit's indices are in (mk2_prefetch_unit), so that the loads of the
// reconstruction's later levels hit L1 instead of waiting for L2 / DRAM one
// level at a time; the arithmetic is the same code.
template <typename TF, int MINB, int GROUP, bool PF = false>
__global__ void __launch_bounds__(128, MINB) mk2_face_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                           double* __restrict__ fl, int n_launch) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    int status = 0;
    if (i < n_launch) {
        const int u = GROUP == kPlainGroup ? i : GROUP == kC1Group ? d.u_c1 + i : d.u_tr1 + i;
        if (PF) mk2_prefetch_unit<GROUP != kPlainGroup>(d, b, u);
        RecUnit r;
        r.a = St5{};
        r.o = St5{};
        mk2_recon_unit<GROUP>(d, P, b, u, r, &status);
        mk2_flux_unit<TF, false>(d, P, b, u, r, fl, nullptr, tmin_u, &status);
    }
    block_reduce_commit(tmin_u, 0, 0, status, b.dt_acc, b.counters, b.status);
}

// Star pressure of the exact Godunov problem of every tracked-face unit
// (Solvers.cpp:1174-1305).  It depends on the reconstructed states and on
// the face normal before the motion, not on the face speed, so it runs on a
// side stream while the grid moves; mk2_flux_tracked_kernel samples the
// solution at the face speed afterwards.  One warp per unit (warp-cooperative
// bisection); pstar[i] belongs to unit u_tr0 + i.
__global__ void __launch_bounds__(64) mk2_tracked_solve_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                               const double* __restrict__ rec,
                                                               double* __restrict__ pstar) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nt = d.u_tr1 - d.u_tr0;
    if (i >= nt) return;
    int status = 0;
    const size_t n = nt;
    // a unit with neither side updated has no flux (rows 15 and 16)
    if (rec[15 * n + i] < 0.0 && rec[16 * n + i] < 0.0) return;
    double q1[5] = {rec[0 * n + i], rec[1 * n + i], rec[2 * n + i], rec[3 * n + i], 0.0};
    double q2[5] = {rec[5 * n + i], rec[6 * n + i], rec[7 * n + i], rec[8 * n + i], 0.0};
    double nv[3] = {rec[10 * n + i], rec[11 * n + i], 0.0};
    double qq[5], ds[3], p = 0.0;
    godunov_dev<true>(P.gamma, P.kurant, q1, q2, nv, qq, ds, 0.0, 1.0, P.godunov_max_iter, &status, nullptr, &p);
    if ((threadIdx.x & 31) == 0) {
        pstar[i] = p;
        if (status) atomicOr(b.status, status);
    }
}

// The term of the MK2 cell update that depends neither on the fluxes nor on
// the motion: the charge-exchange source Get_Sourse_MK1 (Cell.cpp:498-665).
// Runs on a side stream while surface tracking and the rails move the grid.
// aux rows: q1, q2, q3
#if GELIOS_SOURCE_WARP
// 32 cells per warp in two phases, every lane busy in both.  Cell phase: one
// lane per cell decides whether the cell takes part, finds the bracket of
// the radial interpolation, loads the cell's state and interpolates the
// k_u, k_v, k_T factors; the per-cell values go to shared memory.  Species
// phase: four rounds of eight cells x four hydrogen species, one (cell,
// species) pair per lane: the species' moments at the cell and its exchange
// rates; the four rates are summed on the cell's first species lane in the
// reference's order (H1 + H2 + H3 + H4), which writes the cell's q1..q3.
__global__ void __launch_bounds__(128, GELIOS_SOURCE_MINB) mk2_source_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                                             double* __restrict__ aux) {
    // per-cell values of the block's 128 cells, one row per quantity
    __shared__ double sd[10][128];  // u, v, ro, p/ro, u^2+v^2, 1/(r1-r2), rr-r2, k_u, k_v, k_T
    __shared__ int si[3][128];      // K_do, K_posle, flags (1 takes part, 2 bracket found, 4 interpolated)
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
    const int c0 = blockIdx.x * blockDim.x + wbase;  // the warp's first cell
    int status = 0;
    {
        const int c = c0 + lane, t = threadIdx.x;
        int flags = 0, K_do = -1, K_posle = -1;
        double e[10] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (c < d.n_cells) {
            const double x = b.cx[c], y = b.cy[c];
            const double rr = sqrt(sq(x) + sq(y));
            const bool proc = !(rr < P.R11);
            const bool interp = proc && rr > P.src_rmin && rr < P.src_rmax && x >= 0.0;
            bool ok = true;
            if (interp) {
                int2 cached;
                ok = source_bracket(d, c, rr, K_do, K_posle, &status, &cached);
                if (ok && d.src_lo_out && cached.x != K_do) d.src_lo_out[c] = make_int2(K_do, K_posle);
            }
            if (proc && ok) {
                const St5 par1 = load_state(b.cur, c);
                e[0] = par1.u;
                e[1] = par1.v;
                e[2] = par1.ro;
                e[3] = par1.p / par1.ro;
                e[4] = sq(par1.u) + sq(par1.v);
                if (interp) {
                    const double r1 = d.r_istoch[K_do], r2 = d.r_istoch[K_posle];
                    const double ir = 1.0 / (r1 - r2), dr = rr - r2;
                    auto lin = [&](double t1, double t2) { return (t1 - t2) * ir * dr + t2; };
                    e[5] = ir;
                    e[6] = dr;
                    e[7] = lin(d.ku[K_do], d.ku[K_posle]);
                    e[8] = lin(d.kv[K_do], d.kv[K_posle]);
                    e[9] = lin(d.kT[K_do], d.kT[K_posle]);
                } else {
                    e[7] = d.ku[c];
                    e[8] = d.kv[c];
                    e[9] = d.kT[c];
                }
            }
            flags = (proc ? 1 : 0) | (ok ? 2 : 0) | (interp ? 4 : 0);
        }
#pragma unroll
        for (int k = 0; k < 10; k++) sd[k][t] = e[k];
        si[0][t] = K_do;
        si[1][t] = K_posle;
        si[2][t] = flags;
    }
    __syncwarp();
    const int sp = lane & 3, q0 = lane & ~3;
#pragma unroll 1
    for (int r = 0; r < 4; r++) {
        const int t = wbase + 8 * r + (lane >> 2);  // the lane's cell, as a block slot
        const int c = c0 + 8 * r + (lane >> 2);
        const int flags = c < d.n_cells ? si[2][t] : 0;
        double nuu = 0.0, nuv = 0.0, nue = 0.0;
        if ((flags & 3) == 3) {
            SrcMoments m;
            if (flags & 4) {
                const int K_do = si[0][t], K_posle = si[1][t];
                const double ir = sd[5][t], dr = sd[6][t];
                auto lin = [&](double t1, double t2) { return (t1 - t2) * ir * dr + t2; };
                m.uH = lin(d.Hu[4 * K_do + sp], d.Hu[4 * K_posle + sp]);
                m.vH = lin(d.Hv[4 * K_do + sp], d.Hv[4 * K_posle + sp]);
                m.roH = lin(d.Hn[4 * K_do + sp], d.Hn[4 * K_posle + sp]);
                const double TH = lin(d.HT[4 * K_do + sp], d.HT[4 * K_posle + sp]);
                m.pH = 0.5 * TH * m.roH;
            } else {
                m.uH = d.Hu[4 * c + sp];
                m.vH = d.Hv[4 * c + sp];
                m.roH = d.Hn[4 * c + sp];
                m.pH = 0.5 * d.HT[4 * c + sp] * d.Hn[4 * c + sp];
            }
            m.ku = m.kv = m.kT = 0.0;
            source_rates(P, m, sd[0][t], sd[1][t], sd[2][t], sd[3][t], sd[4][t], nuu, nuv, nue);
        }
        double su[3], sv[3], se[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            su[j] = __shfl_sync(full, nuu, q0 + 1 + j);
            sv[j] = __shfl_sync(full, nuv, q0 + 1 + j);
            se[j] = __shfl_sync(full, nue, q0 + 1 + j);
        }
        if (sp == 0 && (flags & 1)) {
            const size_t n = d.n_cells;
            double q1 = 0.0, q2 = 0.0, q3 = 0.0;
            if (flags & 2) {
                const double Mu = P.src_coef * (nuu + su[0] + su[1] + su[2]);
                const double Mv = P.src_coef * (nuv + sv[0] + sv[1] + sv[2]);
                const double MT = P.src_coef * (nue + se[0] + se[1] + se[2]);
                q1 = Mu * sd[7][t];
                q2 = Mv * sd[8][t];
                q3 = MT * sd[9][t];
            }
            aux[0 * n + c] = q1;
            aux[1 * n + c] = q2;
            aux[2 * n + c] = q3;
        }
    }
    if (status) atomicOr(b.status, status);
}
#else
__global__ void __launch_bounds__(128, GELIOS_SOURCE_MINB) mk2_source_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                         double* __restrict__ aux) {
    // four lanes per cell, one hydrogen species per lane; the cell's first
    // lane finds the bracket of the radial interpolation and hands it to the
    // others; the four rates are summed on it in the reference's order
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t >> 2, sp = t & 3;
    const unsigned full = 0xffffffffu;
    const int q0 = (threadIdx.x & 31) & ~3;
    int status = 0;
    bool proc = false, interp = false;
    double x = 0.0, y = 0.0, rr = 0.0;
    if (c < d.n_cells) {
        x = b.cx[c];
        y = b.cy[c];
        rr = sqrt(sq(x) + sq(y));
        proc = !(rr < P.R11);
        interp = proc && rr > P.src_rmin && rr < P.src_rmax && x >= 0.0;
    }
    int K_do = -1, K_posle = -1, ok = 1;
    if (interp && sp == 0) {
        int2 cached;
        ok = source_bracket(d, c, rr, K_do, K_posle, &status, &cached) ? 1 : 0;
        if (ok && d.src_lo_out && cached.x != K_do) d.src_lo_out[c] = make_int2(K_do, K_posle);
    }
    K_do = __shfl_sync(full, K_do, q0);
    K_posle = __shfl_sync(full, K_posle, q0);
    ok = __shfl_sync(full, ok, q0);
    double nuu = 0.0, nuv = 0.0, nue = 0.0;
    SrcMoments m{};
    if (proc && ok) {
        const St5 par1 = load_state(b.cur, c);
        m = source_moments(d, c, sp, interp, K_do, K_posle, rr, sp == 0);
        source_rates(P, m, par1.u, par1.v, par1.ro, par1.p / par1.ro, sq(par1.u) + sq(par1.v), nuu, nuv, nue);
    }
    double su[3], sv[3], se[3];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        su[j] = __shfl_sync(full, nuu, q0 + 1 + j);
        sv[j] = __shfl_sync(full, nuv, q0 + 1 + j);
        se[j] = __shfl_sync(full, nue, q0 + 1 + j);
    }
    if (proc && sp == 0) {
        const size_t n = d.n_cells;
        double q1 = 0.0, q2 = 0.0, q3 = 0.0;
        if (ok) {
            const double Mu = P.src_coef * (nuu + su[0] + su[1] + su[2]);
            const double Mv = P.src_coef * (nuv + sv[0] + sv[1] + sv[2]);
            const double MT = P.src_coef * (nue + se[0] + se[1] + se[2]);
            q1 = Mu * m.ku;
            q2 = Mv * m.kv;
            q3 = MT * m.kT;
        }
        aux[0 * n + c] = q1;
        aux[1 * n + c] = q2;
        aux[2 * n + c] = q3;
    }
    if (status) atomicOr(b.status, status);
}
#endif

// Go_5_komponent__MK2 cell update (Setka.cpp:10386-10468) of cell c from its
// face slots' fluxes (fetch(k, j): row k of the cell's j-th slot, Grans
// order).  The area and rotated volume before the motion come from the cache
// (b.vs, b.vol); the cache is refilled for the next step from the moved
// points: centroid, and area and rotated volume of every cell but the C_centr
// ones (the points after the commit are these moved points, bit for bit),
// |centroid|^(2 gamma) of the cells flagged CF_RP.  For a quadrilateral
// Get_Volume and Get_Volume_posle are the same formula; other cells get the
// Get_Volume form for the cache.
template <typename Fetch>
__device__ __forceinline__ void mk2_update_cell(const DevMesh& d, const gelios_params& P, const StepBuffers& b, int c,
                                                Fetch fetch, const double* __restrict__ aux, double& tmark, int& nro,
                                                int& npc) {
    const uint32_t cfl = d.cflags[c];
    const double x = b.cx[c], y = b.cy[c];
    double xn, yn, vs2 = 0.0, Volume2 = 0.0;
    // quadrilaterals: the corner indices in one 16-byte load (qcorner), so
    // the moved points are the second level of dependent loads, not the third
    const int4 qc = d.qcorner ? d.qcorner[c] : make_int4(-1, -1, -1, -1);
    if (qc.x >= 0) {
        // the four moved points once, in registers (the same operations as
        // centroid / area / volume_rotate)
        const double qx[4] = {d.X2[qc.x], d.X2[qc.y], d.X2[qc.z], d.X2[qc.w]};
        const double qy[4] = {d.Y2[qc.x], d.Y2[qc.y], d.Y2[qc.z], d.Y2[qc.w]};
        quad_geometry(qx, qy, xn, yn, vs2, Volume2);
        if (!(cfl & CF_CENTR)) {
            b.vs_next[c] = vs2;
            b.vol_next[c] = Volume2;
        }
    } else if (const int n4 = d.cstart[c + 1] - d.cstart[c]; n4 == 4) {
        const int32_t* con = d.contour + d.cstart[c];
        const int p0 = con[0], p1 = con[1], p2 = con[2], p3 = con[3];
        const double qx[4] = {d.X2[p0], d.X2[p1], d.X2[p2], d.X2[p3]};
        const double qy[4] = {d.Y2[p0], d.Y2[p1], d.Y2[p2], d.Y2[p3]};
        quad_geometry(qx, qy, xn, yn, vs2, Volume2);
        if (!(cfl & CF_CENTR)) {
            b.vs_next[c] = vs2;
            b.vol_next[c] = Volume2;
        }
    } else {
        const int s0 = d.cstart[c], n = d.cstart[c + 1] - s0;
        const int32_t* con = d.contour + s0;
        centroid(con, n, d.X2, d.Y2, xn, yn);
        if (!(cfl & CF_CENTR)) {
            vs2 = area(con, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], d.X2, d.Y2, true);
            Volume2 = volume_rotate(con, n, d.X2, d.Y2);
            b.vs_next[c] = area(con, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], d.X2, d.Y2, false);
            b.vol_next[c] = Volume2;
        }
    }
    b.cx_next[c] = xn;
    b.cy_next[c] = yn;
    if (cfl & CF_RP) b.rp_next[c] = pow2g(sqrt(sq(xn) + sq(yn)), 2 * P.gamma);
    if (sqrt(sq(x) + sq(y)) < P.R11) return;
    tmark = dmin_ref(tmark, 10000000.0);  // `time` starts at 1e7 in every step (Setka.cpp:10141)
    const double dt = *b.dt_cur;
    const int nf = d.gstart[c + 1] - d.gstart[c];
    double Pt0 = 0.0, Pt1 = 0.0, Pt2 = 0.0, Pt3 = 0.0, Pt4 = 0.0;
    if (nf == 4) {  // quadrilaterals: all slot loads in flight together
        double a[5][4];
#pragma unroll
        for (int k = 0; k < 5; k++)
#pragma unroll
            for (int j = 0; j < 4; j++) a[k][j] = fetch(k, j);
        Pt0 = (((Pt0 + a[0][0]) + a[0][1]) + a[0][2]) + a[0][3];
        Pt1 = (((Pt1 + a[1][0]) + a[1][1]) + a[1][2]) + a[1][3];
        Pt2 = (((Pt2 + a[2][0]) + a[2][1]) + a[2][2]) + a[2][3];
        Pt3 = (((Pt3 + a[3][0]) + a[3][1]) + a[3][2]) + a[3][3];
        Pt4 = (((Pt4 + a[4][0]) + a[4][1]) + a[4][2]) + a[4][3];
    } else {
        for (int j = 0; j < nf; j++) {
            Pt0 = Pt0 + fetch(0, j);
            Pt1 = Pt1 + fetch(1, j);
            Pt2 = Pt2 + fetch(2, j);
            Pt3 = Pt3 + fetch(3, j);
            Pt4 = Pt4 + fetch(4, j);
        }
    }
    const St5 par1 = load_state(b.cur, c);
    const size_t nc = d.n_cells;
    const double q2_1 = aux[0 * nc + c], q2_2 = aux[1 * nc + c], q3 = aux[2 * nc + c];
    if (!(cfl & CF_CENTR)) {
        const double vs1 = b.vs[c];
        const double Volume = b.vol[c];
        const double ro = par1.ro, u = par1.u, v = par1.v, p = par1.p, Q = par1.Q;
        const double gm1 = P.gamma - 1;
        const double rV2 = 1.0 / Volume2, VV = Volume * rV2;
        double ro3 = ro * VV - dt * (Pt0 * rV2);
        const double Q33 = Q * VV - (dt * rV2) * Pt4;
        if (ro3 <= 0.0) {
            ro3 = P.ro_floor;
            nro++;
        }
        const double rro3 = 1.0 / ro3;
        const double u3 = (ro * u * VV - dt * (Pt1 * rV2 - q2_1)) * rro3;
        const double v3 = (ro * v * VV - dt * ((Pt2 - p * 0.5 * (vs1 + vs2)) * rV2 - q2_2)) * rro3;
        double p3 =
            (((p / gm1 + ro * (u * u + v * v) * 0.5) * VV - dt * (Pt3 * rV2 - q3)) - 0.5 * ro3 * (u3 * u3 + v3 * v3)) *
            gm1;
        if (p3 <= 0) {
            p3 = P.p_floor;
            npc++;
        }
        b.nxt[0][c] = ro3;
        b.nxt[1][c] = p3;
        b.nxt[2][c] = u3;
        b.nxt[3][c] = v3;
        b.nxt[4][c] = Q33;
    } else {
        b.nxt[0][c] = par1.ro;
        b.nxt[1][c] = par1.p;
        b.nxt[2][c] = par1.u;
        b.nxt[3][c] = par1.v;
        b.nxt[4][c] = par1.Q;
    }
}

// The face units and the cell update of the moving-grid step, one tile of
// cells per block (tiles: spatially compact groups built at upload).  Phase
// 1: every face unit that touches the tile's cells, reconstruction and flux
// in registers, F.S (owner side) / -F.S (other side) into the tile-local
// slots in shared memory; a unit whose two cells lie in different tiles is
// evaluated by both (same inputs, same code: the same bits on both sides).
// Tracked units take the fluxes the tracked-face kernel left in `fl`.
// Phase 2: the update of every cell of the tile from its slots.  No flux
// leaves the SM.  The CFL candidate of a side is taken by the tile that holds
// that side's cell, so each is taken once.
template <typename TF, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) mk2_tile_kernel(DevMesh d, gelios_params P, StepBuffers b, TileView t,
                                                           const double* __restrict__ fl,
                                                           const double* __restrict__ aux) {
    extern __shared__ double sfl[];  // 5 rows of t.max_slots
    const int tile = blockIdx.x;
    const int ms = t.max_slots;
    const size_t ng = d.n_slots;
    double tmin = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0, status = 0;
    const int f0 = t.fstart[tile], f1 = t.fstart[tile + 1];
    for (int j = f0 + threadIdx.x; j < f1; j += NT) {
        const int2 rec = t.faces[j];
        const int u = rec.x;
        const int own = rec.y & 0xffff, tw = (rec.y >> 16) & 0xffff;
        if (u >= d.u_tr0 && u < d.u_tr1) {
            const int g = d.u_slot[u], gt = d.u_twin[u];
#pragma unroll
            for (int k = 0; k < 5; k++) {
                if (own != kTileNone) sfl[k * ms + own] = fl[k * ng + g];
                if (tw != kTileNone) sfl[k * ms + tw] = fl[k * ng + gt];
            }
            continue;
        }
        RecUnit r;
        r.a = St5{};
        r.o = St5{};
        mk2_recon_unit(d, P, b, u, r, &status);
        const bool procK = !(r.dist < 0.0), procN = !(r.distn < 0.0);
        if (!(procK || procN)) continue;
        const double dt = *b.dt_cur;
        const int A = d.u_A[u], B = d.u_B[u];
        const double x4 = (d.X2[A] + d.X2[B]) / 2.0, y4 = (d.Y2[A] + d.Y2[B]) / 2.0;
        const double W = ((x4 - r.x2) * r.n1 + (y4 - r.y2) * r.n2) / dt;
        const bool np = (d.u_info[u] & SI_NP) != 0;
        FluxOut<double> F;
        const double UU = hllc_flux<TF>(P.gamma, P.kurant, r.a, r.o, W, r.n1, r.n2, 1.0, 0, np, F);
        const double S = r.S;
        const double fm[5] = {F.P0 * S, F.P1 * S, F.P2 * S, F.P3 * S, F.PQ * S};
        if (own != kTileNone) {
#pragma unroll
            for (int k = 0; k < 5; k++) sfl[k * ms + own] = fm[k];
            if (procK) tmin = dmin_ref(tmin, P.kurant * r.dist / UU);
        }
        if (tw != kTileNone) {
#pragma unroll
            for (int k = 0; k < 5; k++) sfl[k * ms + tw] = -fm[k];
            if (procN) tmin = dmin_ref(tmin, P.kurant * r.distn / UU);
        }
    }
    __syncthreads();
    const int c0 = t.cstart[tile], c1 = t.cstart[tile + 1];
    for (int i = c0 + threadIdx.x; i < c1; i += NT) {
        const int c = t.cells[i];
        const int base = t.lbase[i];
        mk2_update_cell(d, P, b, c, [&](int k, int jj) { return sfl[k * ms + base + jj]; }, aux, tmin, nro, npc);
    }
    block_reduce_commit(tmin, nro, npc, status, b.dt_acc, b.counters, b.status);
}

// The cell update alone, from the flux slots in global memory (the update
// phase of the tile kernel for the face-kernel arrangement).
// MODE kUpdAll: every cell, the 1e7 start of the CFL minimum folded into the
// accumulator (the reference's `time`, Setka.cpp:10141) when a cell takes
// part.  The pipelined step leaves that to its dt finalisation
// (dt_finalize_cap_kernel, commit with cap) and updates in two parts:
// kUpdEarly the listed cells (CF_EARLY), kUpdRest every other cell;
// kUpdAllNoMark every cell (its last step).
enum : int { kUpdAll = 0, kUpdEarly = 1, kUpdRest = 2, kUpdAllNoMark = 3 };
template <int MODE>
__global__ void __launch_bounds__(128, 8) mk2_update_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                          const double* __restrict__ fl,
                                                          const double* __restrict__ aux,
                                                          const int32_t* __restrict__ list, int n_list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double tmark = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0;
    const size_t ng = d.n_slots;
    int c = -1;
    if (MODE == kUpdEarly) {
        if (i < n_list) c = list[i];
    } else if (i < d.n_cells) {
        c = i;
        if (MODE == kUpdRest && (d.cflags[c] & CF_EARLY)) c = -1;
    }
    if (c >= 0) {
        const int g0 = d.gstart[c];
        mk2_update_cell(d, P, b, c, [&](int k, int j) { return __ldcs(fl + k * ng + g0 + j); }, aux, tmark, nro, npc);
    }
    if (MODE != kUpdAll) tmark = __longlong_as_double(0x7ff0000000000000LL);
    block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
}

// Go_stationary_5_komponent_inner_MK2 cell update (Setka.cpp:7021-7210).
template <typename TF>
__global__ void __launch_bounds__(128) inner_cell_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                         const int32_t* __restrict__ list, int n_list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double tmin_c = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0, status = 0;
    const double* const* st = b.cur;
    const int c = i < n_list ? list[i] : -1;
    if (c >= 0 && !(d.cflags[c] & CF_CENTR)) {
        const double dt = *b.dt_cur;
        const uint32_t cf = d.cflags[c];
        const int s0 = d.cstart[c], n = d.cstart[c + 1] - s0;
        const int32_t* con = d.contour + s0;
        const int g0 = d.gstart[c], g1 = d.gstart[c + 1];
        const St5 par1 = load_state(st, c);
        const double x = b.cx[c], y = b.cy[c];
        const double vs1 = area(con, n, d.sA, d.sB, g0, g1, d.X, d.Y, false);
        const double vs2 = area(con, n, d.sA, d.sB, g0, g1, d.X2, d.Y2, true);
        const double radius = sqrt(sq(x) + sq(y));
        const double Volume = volume_rotate(con, n, d.X, d.Y);
        const double g2 = 2.0 * P.gamma;
        double Pt0 = 0.0, Pt1 = 0.0, Pt2 = 0.0, Pt3 = 0.0, Pt4 = 0.0;
        double time = 10000000.0;
        for (int g = g0; g < g1; g++) {
            const int A = d.sA[g], B = d.sB[g];
            const uint32_t info = d.sinfo[g];
            const int ft = info & SI_TYPE_MASK;
            const double xa = d.X[A], ya = d.Y[A], xb = d.X[B], yb = d.Y[B];
            const double S = sqrt(sq(xb - xa) + sq(yb - ya)) * (ya + yb) * 0.5;
            const double x2 = (xa + xb) / 2.0, y2 = (ya + yb) / 2.0;
            const double dist = sqrt(sq(x - x2) + sq(y - y2));
            const int nb = d.snb[g];
            St5 par11 = par1;
            St5 par2 = get_par(P, ft, par1, st, nb, x2, y2);
            double t1 = xb - xa, t2 = yb - ya;
            const double nn = sqrt(sq(t1) + sq(t2));
            t1 = t1 / nn;
            t2 = t2 / nn;
            const double n1 = t2, n2 = -t1;
            int met = 1;
            const double dis = sqrt(sq(x2) + sq(y2));
            if (ft == G_USUALY) {
                const double x3 = b.cx[nb], y3 = b.cy[nb];
                const double dd = sqrt(sq(x3) + sq(y3));
                par11.ro = par11.ro * sq(radius) / sq(dis);
                par2.ro = par2.ro * sq(dd) / sq(dis);
                par11.Q = par11.Q * sq(radius) / sq(dis);
                par2.Q = par2.Q * sq(dd) / sq(dis);
                const double pdis = pow2g(dis, g2);
                par11.p = par11.p * (b.rp[c] / pdis);
                par2.p = par2.p * (b.rp[nb] / pdis);
                polar_perenos(x, y, x2, y2, par11.u, par11.v);
                polar_perenos(x3, y3, x2, y2, par2.u, par2.v);
                const uint32_t nbf = d.cflags[nb];
                if ((cf & CF_C1) && (nbf & CF_C1)) {
                    const St5 nbs = load_state(st, nb);
                    tvd_radial(st, b.cx, b.cy, b.rp, x2, y2, par1, x, y, b.rp[c], nb, d.ssd[g], (cf & CF_AXIS) != 0,
                               pdis, par11.ro, par11.p);
                    tvd_radial(st, b.cx, b.cy, b.rp, x2, y2, nbs, x3, y3, b.rp[nb], c, d.ssd2[g],
                               (nbf & CF_AXIS) != 0, pdis, par2.ro, par2.p);
                }
            } else if (ft == G_INNER_SPHERE) {
                par11 = par2;
            } else if (ft == G_AXIS) {
                par11.ro = par11.ro * sq(radius) / sq(dis);
                par11.Q = par11.Q * sq(radius) / sq(dis);
                par11.p = par11.p * (b.rp[c] / pow2g(dis, g2));
                polar_perenos(x, y, x2, y2, par11.u, par11.v);
                par2 = par11;
                par2.v = -par2.v;
                met = 0;
            }
            FluxOut<double> F;
            time = dmin_ref(time, P.kurant * dist / hllc_flux<TF>(P.gamma, P.kurant, par11, par2, 0.0, n1, n2, dist,
                                                                  met, false, F));
            Pt0 = Pt0 + F.P0 * S;
            Pt1 = Pt1 + F.P1 * S;
            Pt2 = Pt2 + F.P2 * S;
            Pt3 = Pt3 + F.P3 * S;
            Pt4 = Pt4 + F.PQ * S;
        }
        tmin_c = time;
        double q2_1, q2_2, q3;
        source_mk1(d, P, c, x, y, par1.u, par1.v, par1.ro, par1.p, q2_1, q2_2, q3, &status);
        const double ro = par1.ro, u = par1.u, v = par1.v, p = par1.p, Q = par1.Q;
        const double gm1 = P.gamma - 1;
        double ro3 = ro - dt * (Pt0 / Volume);
        const double Q33 = Q - (dt / Volume) * Pt4 - dt;
        if (ro3 <= 0) {
            ro3 = P.ro_floor;
            nro = 1;
        }
        const double u3 = (ro * u - dt * (Pt1 / Volume - q2_1)) / ro3;
        const double v3 = (ro * v - dt * ((Pt2 - p * 0.5 * (vs1 + vs2)) / Volume - q2_2)) / ro3;
        double p3 = (((p / gm1 + ro * (u * u + v * v) * 0.5) - dt * (Pt3 / Volume - q3)) - 0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                    gm1;
        if (p3 <= 0) {
            p3 = P.p_floor;
            npc = 1;
        }
        b.nxt[0][c] = ro3;
        b.nxt[1][c] = p3;
        b.nxt[2][c] = u3;
        b.nxt[3][c] = v3;
        b.nxt[4][c] = Q33;
    }
    block_reduce_commit(tmin_c, nro, npc, status, b.dt_acc, b.counters, b.status);
}

// T[now2] of the reference: min(1e7, all face candidates) if any cell took
// part, 1e8 otherwise; re-arm the accumulator.
__global__ void dt_finalize_kernel(StepBuffers b) {
    const unsigned long long a = *b.dt_acc;
    double t = (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
    *b.dt_next = t;
    *b.dt_acc = 0x7ff0000000000000ULL;
}

// T[now2] when the update did not fold the 1e7 start of the CFL minimum in
// (the pipelined moving-grid step): a face candidate exists exactly when a
// cell takes part (a cell that takes part gives its faces a candidate), so
// min(1e7, candidates) if there is one, 1e8 otherwise; re-arm the
// accumulator.
__device__ __forceinline__ void dt_finalize_cap(const StepBuffers& b) {
    const unsigned long long a = *b.dt_acc;
    const double t = (a == 0x7ff0000000000000ULL)
                         ? 100000000.0
                         : dmin_ref(10000000.0, __longlong_as_double(static_cast<long long>(a)));
    *b.dt_next = t;
    *b.dt_acc = 0x7ff0000000000000ULL;
}
__global__ void dt_finalize_cap_kernel(StepBuffers b) { dt_finalize_cap(b); }

// x = x2, y = y2 (Setka.cpp:10473-10480; the zeroed V and count are never
// stored, see point_velocity) + dt finalisation (CAP: dt_finalize_cap).
template <bool CAP>
__global__ void commit_kernel(DevMesh d, StepBuffers b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        if (CAP) {
            dt_finalize_cap(b);
        } else {
            const unsigned long long a = *b.dt_acc;
            double t = (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
            *b.dt_next = t;
            *b.dt_acc = 0x7ff0000000000000ULL;
        }
    }
    if (i < d.n_points) {
        d.X[i] = d.X2[i];
        d.Y[i] = d.Y2[i];
    }
}

// ------------------------------------------------------------------ node velocities
// Move_surface, part 2 (Setka.cpp:3522-3535, 3718-3736, 3829-3842): the
// velocity of a tracked-surface node.  The reference accumulates the face
// speeds into Point::Vx/Vy/count in one serial pass per line, runs three
// averaging loops that all walk Line_Contact, and fixes up the end nodes of
// each line in between.  The three lines touch disjoint point sets, so the
// value of one node depends only on its own face incidences (sp_inc, in line
// order), on the averaging passes in which it is the A end of a contact face
// (sp_ainc), and, for the end nodes, on the first-pass values of the other
// end nodes of its line.  point_velocity replays exactly those operations for
// one point, so the rails can evaluate their key points directly from the
// per-face speeds (bit-identical to the serial passes).
__device__ __forceinline__ void node_pass1(const DevMesh& d, const double* __restrict__ scratch, int i, double& v,
                                           double& w, int& c) {
    const int line = d.sp_line[i];
    v = 0.0;
    w = 0.0;
    c = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int e = d.sp_inc[4 * i + k];
        if (e < 0) break;
        const int j = e >> 1, role = e & 1;  // role 0: A end, 1: B end
        const double* f = scratch + 4 * j;
        const double br = f[3];
        bool add;
        if (line == 0) add = role == 1;
        else if (line == 1) add = role == 1 || br != 0.0;
        else add = (br == 1.0) || (role == 1 && (br == 0.0 || br == 2.0)) || (role == 0 && br == 3.0);
        if (add) {
            v += f[0] * f[1];
            w += f[0] * f[2];
            c++;
        }
    }
    if (line == 0) {  // first averaging pass: every contact face (Setka.cpp:3522-3530)
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int j = d.sp_ainc[4 * i + k];
            if (j < 0) break;
            if (c > 0) {
                v /= (1.0 * c);
                w /= (1.0 * c);
            }
        }
    }
}

// Vx, Vy of point p after Move_surface (0 for points off the tracked lines:
// every step starts from zero velocities, Setka.cpp:10473-10480).
__device__ void point_velocity(const DevMesh& d, const double* __restrict__ scratch, double dt, int p, double& vx,
                               double& vy) {
    const int i = d.sp_of_point[p];
    vx = 0.0;
    vy = 0.0;
    if (i < 0) return;
    int c;
    node_pass1(d, scratch, i, vx, vy, c);
    const int line = d.sp_line[i];
    const int32_t* fx = d.sp_fix + 4 * line;  // a0, b0 (first face), a_last, b_last
    if (i == fx[0] || i == fx[3]) {
        // replay the end-node fix-ups of this line in the reference's order
        // on local copies of the four end nodes (aliases kept in sync)
        int id[4];
        double lx[4], ly[4];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            id[m] = fx[m];
            int cm;
            node_pass1(d, scratch, id[m], lx[m], ly[m], cm);
        }
        auto setx = [&](int node, double val) {
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (id[m] == node) lx[m] = val;
        };
        auto sety = [&](int node, double val) {
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (id[m] == node) ly[m] = val;
        };
        const double* X = d.X;
        const double* Y = d.Y;
        const int pa0 = d.sp_point[id[0]], pb0 = d.sp_point[id[1]], pa1 = d.sp_point[id[2]], pb1 = d.sp_point[id[3]];
        // fx[0]: vx[a0] = vx[b0] + (X[b0] - X[a0]) / dt on every line
        setx(id[0], lx[1] + (X[pb0] - X[pa0]) / dt);
        if (line == 1) {
            // inner shock: vx[b1] = vx[a1] + (X[a1] - X[b1]) / dt (Setka.cpp:3733-3736)
            double a1x = lx[2];
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (id[m] == id[2]) a1x = lx[m];
            setx(id[3], a1x + (X[pa1] - X[pb1]) / dt);
        } else {
            // contact / outer shock: vy[b1] = vy[a1] + (Y[a1] - Y[b1]) / dt
            sety(id[3], ly[2] + (Y[pa1] - Y[pb1]) / dt);
        }
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (id[m] == i) {
                vx = lx[m];
                vy = ly[m];
            }
    }
    if (line == 0) {
        // second and third passes walk Line_Contact up to the inner/outer
        // line lengths (Setka.cpp:3718-3731, 3829-3837)
        const int nC = d.n_lc, nI = d.n_li, nO = d.n_lo;
        const int lim2 = nI > 0 ? (nI < nC ? nI : nC) : 0;
        const int lim3 = nO > 0 ? (nO < nC ? nO : nC) : 0;
        for (int pass = 0; pass < 2; pass++) {
            const int lim = pass == 0 ? lim2 : lim3;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int j = d.sp_ainc[4 * i + k];
                if (j < 0) break;
                if (j < lim && c > 0) {
                    vx /= (1.0 * c);
                    vy /= (1.0 * c);
                }
            }
        }
    }
}

// ------------------------------------------------------------------ grid motion
// Move_Setka_Calculate_2 (Setka.cpp:4324-4759) in one launch, one CTA per
// rail.  The reference moves the A rails, then the B rails, then the C rails,
// then the D rails, and two of them share points:
//  * C_Rails[0] starts with the first M1 points of the last B rail and
//    overwrites them (with its own angle), so the last B rail leaves those
//    points to C_Rails[0] and uses its own value of its key point 0 for the
//    points above it, as the reference's B pass does;
//  * the first point of every D rail is a point of C_Rails[0]; the D block
//    recomputes that point's new position from C_Rails[0]'s key point with
//    the same operations (bit-identical to reading it back).
__device__ __forceinline__ void c0_key(const DevMesh& d, int q, double dt, double vx, double vy, double& x2,
                                       double& y2) {
    const int K0 = d.rkeys[d.rkstart[q]];
    const double s = d.rs[q], cs = cos(s), sn = sin(s);
    const double V = vx * cs + vy * sn;
    x2 = d.X[K0] + dt * V * cs;
    y2 = d.Y[K0] + dt * V * sn;
}

// copy_outer_shock: Move_Setka_Calculate_2 gives the D rails beyond
// n_outer_shock the outer-shock key height of the last D rail before them
// (Setka.cpp:4725-4728); Move_Setka_Calculate (Setka.cpp:4761-5147, used by
// Go_5_komponent) is otherwise the same and moves them on their own.
// One rail q (the body of rails_kernel; every thread of the block calls it).
__device__ __forceinline__ void rails_body(const DevMesh& d, const gelios_params& P, const double* __restrict__ dtp,
                                           const double* __restrict__ scratch, bool copy_outer_shock, int q) {
    const double dt = *dtp;
    const int32_t* ap = d.rpts + d.rpstart[q];
    const int np = d.rpstart[q + 1] - d.rpstart[q];
    const int32_t* kp = d.rkeys + d.rkstart[q];
    const int M1 = d.rM[4 * q], M2 = d.rM[4 * q + 1], M3 = d.rM[4 * q + 2], M4 = d.rM[4 * q + 3];
    const int t = d.rtype[q];
    const int first_c = d.n_rail_a + d.n_rail_b, first_d = first_c + d.n_rail_c;
    // the last B rail hands its first M1 points to C_Rails[0]
    const bool handoff = (t == 1) && (q == first_c - 1) && d.n_rail_c > 0;
    double* X2 = d.X2;
    double* Y2 = d.Y2;
    const double* X = d.X;
    const double* Y = d.Y;
    __shared__ double sh[6];
    const int ni = P.n_inner;
    // velocities of the key points this rail reads, one thread each
    __shared__ double kvx[4], kvy[4];
    if (threadIdx.x < 4) {
        int pt = -1;
        const int k = threadIdx.x;
        if (t == 0 || t == 1) {
            if (k < 3) pt = kp[k];
        } else if (t == 2) {
            if (k == 0) pt = kp[0];
        } else {
            if (k == 0) pt = d.rkeys[d.rkstart[first_c]];  // key point 0 of C_Rails[0]
            else if (k < 3) pt = kp[k];
            else if (copy_outer_shock && q - first_d >= P.n_outer_shock && P.n_outer_shock >= 1)
                pt = d.rkeys[d.rkstart[first_d + P.n_outer_shock - 1] + 2];
        }
        double vx = 0.0, vy = 0.0;
        if (pt >= 0) point_velocity(d, scratch, dt, pt, vx, vy);
        kvx[k] = vx;
        kvy[k] = vy;
    }
    __syncthreads();
    if (t == 0 || t == 1 || t == 2) {
        const double s = d.rs[q];
        const double cs = cos(s), sn = sin(s);
        if (threadIdx.x == 0) {
            if (t == 0) {  // A rail, Setka.cpp:4331-4356
                for (int kk = 0; kk < 3; kk++) {
                    const int K = kp[kk];
                    const double V = kvx[kk] * cs + kvy[kk] * sn;
                    X2[K] = X[K] + dt * V * cs;
                    Y2[K] = Y[K] + dt * V * sn;
                }
                X2[kp[3]] = X[kp[3]];
                Y2[kp[3]] = Y[kp[3]];
                sh[0] = sqrt(sq(X2[kp[0]]) + sq(Y2[kp[0]]));
                sh[1] = sqrt(sq(X2[kp[1]]) + sq(Y2[kp[1]]));
                sh[2] = sqrt(sq(X2[kp[2]]) + sq(Y2[kp[2]]));
            } else if (t == 1) {  // B rail, Setka.cpp:4469-4502
                const int K0 = kp[0], K1 = kp[1], K2 = kp[2], K3 = kp[3];
                double V = kvx[0] * cs + kvy[0] * sn;
                const double x0 = X[K0] + dt * V * cs, y0 = Y[K0] + dt * V * sn;
                if (!handoff) {
                    X2[K0] = x0;
                    Y2[K0] = y0;
                }
                V = kvx[1] * 0.0 + kvy[1] * 1.0;
                X2[K1] = x0;
                Y2[K1] = Y[K1] + dt * V;
                V = kvx[2] * 0.0 + kvy[2] * 1.0;
                X2[K2] = x0;
                Y2[K2] = Y[K2] + dt * V;
                X2[K3] = x0;
                Y2[K3] = Y[K3];
                sh[0] = sqrt(sq(x0) + sq(y0));
                sh[1] = Y2[K1];
                sh[2] = Y2[K2];
                sh[3] = x0;
                sh[4] = y0;
            } else {  // C rail, Setka.cpp:4603-4614
                const int K0 = kp[0], K1 = kp[1];
                const double V = kvx[0] * cs + kvy[0] * sn;
                X2[K0] = X[K0] + dt * V * cs;
                Y2[K0] = Y[K0] + dt * V * sn;
                X2[K1] = P.Left;
                Y2[K1] = Y[K1];
                sh[0] = sqrt(sq(X2[K0]) + sq(Y2[K0]));
                sh[3] = X2[K0];
                sh[4] = Y2[K0];
            }
        }
        __syncthreads();
        const double R2 = sh[0];
        if (!handoff) {  // inner layer, Setka.cpp:4390-4406 (and 4532-4548, 4644-4660)
            for (int j = threadIdx.x; j < M1 - 1; j += blockDim.x) {
                double r;
                if (j < ni) {
                    const double x = j * 1.0 / (ni);
                    r = P.R1 + pow(x, 1.3) * (P.R111 - P.R1);
                } else {
                    const double x = (j - ni) * 1.0 / (M1 - 1 - ni);
                    r = P.R111 + pow(x, 1.05) * (R2 - P.R111);
                }
                X2[ap[j]] = r * cs;
                Y2[ap[j]] = r * sn;
            }
        }
        if (t == 0) {  // Setka.cpp:4411-4456
            const double R3 = sh[1], R4 = sh[2];
            for (int j = threadIdx.x; j < M2 - 1; j += blockDim.x) {
                const double r = R2 + (R3 - R2) * (j + 1) / (M2);
                X2[ap[M1 + j]] = r * cs;
                Y2[ap[M1 + j]] = r * sn;
            }
            for (int j = threadIdx.x; j < M3 - 1; j += blockDim.x) {
                const double r = R3 + (R4 - R3) * (j + 1) / (M3);
                X2[ap[M1 + M2 + j]] = r * cs;
                Y2[ap[M1 + M2 + j]] = r * sn;
            }
            const double dd = 1.5708 / sqrt(1.0 - 1.0 / 1.76);
            const double e = 1.76 * (1.0 - sq(s / dd));
            for (int j = threadIdx.x; j < M4; j += blockDim.x) {
                const double x = (j + 1) * 1.0 / (M4);
                const double r = R4 + pow(x, e) * (P.R5 - R4);
                X2[ap[M1 + M2 + M3 + j]] = r * cs;
                Y2[ap[M1 + M2 + M3 + j]] = r * sn;
            }
        } else if (t == 1) {  // Setka.cpp:4552-4593
            const double R2y = sh[4], R3 = sh[1], R4 = sh[2], xk = sh[3];
            for (int j = threadIdx.x; j < M2 - 1; j += blockDim.x) {
                X2[ap[M1 + j]] = xk;
                Y2[ap[M1 + j]] = R2y + (R3 - R2y) * (j + 1) / (M2);
            }
            for (int j = threadIdx.x; j < M3 - 1; j += blockDim.x) {
                X2[ap[M1 + M2 + j]] = xk;
                Y2[ap[M1 + M2 + j]] = R3 + (R4 - R3) * (j + 1) / (M3);
            }
            for (int j = threadIdx.x; j < M4; j += blockDim.x) {
                X2[ap[M1 + M2 + M3 + j]] = xk;
                Y2[ap[M1 + M2 + M3 + j]] = R4 + (P.R5 - R4) * (j + 1) / (M4);
            }
        } else {  // Setka.cpp:4662-4673
            const double R2x = sh[3], yk = sh[4];
            const double x = pow(P.Left / (R2x), 1.0 / (M2));
            for (int j = M1 + threadIdx.x; j < np; j += blockDim.x) {
                X2[ap[j]] = R2x * pow(x, static_cast<double>(j + 1 - M1));
                Y2[ap[j]] = yk;
            }
        }
        return;
    }
    // D rail, Setka.cpp:4676-4758
    const int jj = q - first_d;
    const int sM2 = d.dims[5], sM3 = d.dims[6], sM4 = d.dims[7];
    if (threadIdx.x == 0) {
        const int K1 = kp[1], K2 = kp[2], K3 = kp[3];
        // key point 0 = point M1 + jj of C_Rails[0], as the C pass moves it
        double c0x, c0y;
        c0_key(d, first_c, dt, kvx[0], kvy[0], c0x, c0y);
        const int Mc1 = d.rM[4 * first_c], Mc2 = d.rM[4 * first_c + 1];
        const int j = Mc1 + jj;
        const double xr = pow(P.Left / (c0x), 1.0 / (Mc2));
        const double x0 = c0x * pow(xr, static_cast<double>(j + 1 - Mc1));
        const double y0 = c0y;
        double V = kvy[1];
        X2[K1] = x0;
        Y2[K1] = Y[K1] + dt * V;
        V = kvy[2];
        X2[K2] = x0;
        if (copy_outer_shock && jj >= P.n_outer_shock && P.n_outer_shock >= 1) {
            const int qs = first_d + P.n_outer_shock - 1;
            const int Ks = d.rkeys[d.rkstart[qs] + 2];
            Y2[K2] = Y[Ks] + dt * kvy[3];
        } else {
            Y2[K2] = Y[K2] + dt * V;
        }
        X2[K3] = x0;
        Y2[K3] = Y[K3];
        sh[0] = y0;
        sh[1] = Y2[K1];
        sh[2] = Y2[K2];
        sh[3] = x0;
    }
    __syncthreads();
    const double R2 = sh[0], R3 = sh[1], R4 = sh[2], xk = sh[3];
    for (int j = threadIdx.x; j < sM2 - 1; j += blockDim.x) {
        X2[ap[j + 1]] = xk;
        Y2[ap[j + 1]] = R2 + (R3 - R2) * (j + 1) / (M2);
    }
    for (int j = threadIdx.x; j < sM3 - 1; j += blockDim.x) {
        X2[ap[sM2 + j + 1]] = xk;
        Y2[ap[sM2 + j + 1]] = R3 + (R4 - R3) * (j + 1) / (M3);
    }
    for (int j = threadIdx.x; j < sM4; j += blockDim.x) {
        X2[ap[sM2 + sM3 + j + 1]] = xk;
        Y2[ap[sM2 + sM3 + j + 1]] = R4 + (P.R5 - R4) * (j + 1) / (M4);
    }
}

__global__ void __launch_bounds__(128) rails_kernel(DevMesh d, gelios_params P, const double* __restrict__ dtp,
                                                    const double* __restrict__ scratch, bool copy_outer_shock) {
    rails_body(d, P, dtp, scratch, copy_outer_shock, blockIdx.x);
}

// ------------------------------------------------------------------ surface tracking
// Get_par_TVD of a main/copy face f read through the face table.
__device__ St5 face_tvd(const DevMesh& d, const double* const* st, const double* cx, const double* cy, int f,
                        int* status) {
    const int ft = d.ftype[f];
    const int M = d.fmaster[f];
    const int a = d.fA[f], bb = d.fB[f];
    const double fx = (d.X[a] + d.X[bb]) / 2.0, fy = (d.Y[a] + d.Y[bb]) / 2.0;
    const St5 Ms = load_state(st, M);
    if (ft == G_USUALY) {
        const int ta = d.ptype[a], tb = d.ptype[bb];
        const bool tracked = (ta == P_CONTACT && tb == P_CONTACT) || (ta == P_INNER_SHOCK && tb == P_INNER_SHOCK) ||
                             (ta == P_OUTER_SHOCK && tb == P_OUTER_SHOCK);
        return tvd_usualy(st, cx, cy, fx, fy, Ms, cx[M], cy[M], d.fsosed[f], d.fsdown[f],
                          (d.cflags[M] & CF_AXIS) != 0, tracked, status);
    }
    if (ft == G_AXIS) return tvd_axis(st, cx, cy, fx, fy, Ms, cx[M], cy[M], d.fsdown[f]);
    St5 o = Ms;
    return o;  // Extern/Upper_wall/Input/Inner faces do not occur on tracked lines
}

// Move_surface (Setka.cpp:3378-3844), part 1: one thread per tracked face
// (contact, inner shock, outer shock) computes its exact-Godunov wave speed,
// the face normal and the branch the reference takes.
// scratch layout per face j of the concatenated lines (contact, inner, outer):
//   [0] speed  [1] n1  [2] n2  [3] branch
//   branch: contact 0 (B only); inner 0 (B only) / 1 (A and B);
//           outer -1 (skipped) / 0 B / 1 A and B / 2 B / 3 A
// One warp per face: the lanes hold identical copies of the face's data, the
// exact solver runs warp-cooperatively, lane 0 writes.
// Tracked face j of the concatenated lines, all 32 lanes of a warp (the
// body of surface_faces_kernel).
__device__ __forceinline__ void surface_face_body(const DevMesh& d, const gelios_params& P, const StepBuffers& b,
                                                  double* __restrict__ scratch, int j, int lane) {
    const int nC = d.n_lc, nI = d.n_li;
    const double* const* st = b.cur;
    int status = 0;
    const double ga = P.gamma, g2 = 2.0 * P.gamma;
    double nv[3], q1[5], q2[5], qq[5], ds[3];
    int f;
    if (j < nC) f = d.lc[j];
    else if (j < nC + nI) f = d.li[j - nC];
    else f = d.lo[j - nC - nI];
    const int a = d.fA[f], bb = d.fB[f];
    double t1 = d.X[bb] - d.X[a], t2 = d.Y[bb] - d.Y[a];
    const double nn = sqrt(sq(t1) + sq(t2));
    t1 /= nn;
    t2 /= nn;
    const double n1 = t2, n2 = -t1;
    nv[0] = n1; nv[1] = n2; nv[2] = 0.0;
    double o0 = 0.0, o3 = 0.0;
    // TVD states of the face (even lanes) and of its twin (odd lanes),
    // exchanged between lane pairs
    auto tvd_pair = [&](St5& pf, St5& pc) {
        const St5 mine = face_tvd(d, st, b.cx, b.cy, (lane & 1) ? d.fcopy[f] : f, &status);
        St5 other;
        other.ro = __shfl_xor_sync(0xffffffffu, mine.ro, 1);
        other.p = __shfl_xor_sync(0xffffffffu, mine.p, 1);
        other.u = __shfl_xor_sync(0xffffffffu, mine.u, 1);
        other.v = __shfl_xor_sync(0xffffffffu, mine.v, 1);
        other.Q = __shfl_xor_sync(0xffffffffu, mine.Q, 1);
        pf = (lane & 1) ? other : mine;
        pc = (lane & 1) ? mine : other;
    };
    if (j < nC) {
        St5 p1, p2;
        tvd_pair(p1, p2);
        q1[0] = p1.ro; q1[1] = p1.p; q1[2] = p1.u; q1[3] = p1.v; q1[4] = 0.0;
        q2[0] = p2.ro; q2[1] = p2.p; q2[2] = p2.u; q2[3] = p2.v; q2[4] = 0.0;
        godunov_dev<true>(ga, P.kurant, q1, q2, nv, qq, ds, 0.0, 0.0, P.godunov_max_iter, &status);
        o0 = ds[2] * P.koef * 0.3;
        o3 = 0.0;
    } else if (j < nC + nI) {
        const int M = d.fmaster[f];
        St5 p1 = load_state(st, M);
        const double x = b.cx[M], y = b.cy[M];
        const double radius = sqrt(sq(x) + sq(y));
        const double x2 = (d.X[a] + d.X[bb]) / 2.0, y2 = (d.Y[a] + d.Y[bb]) / 2.0;
        const double dis = sqrt(sq(x2) + sq(y2));
        const St5 p2 = face_tvd(d, st, b.cx, b.cy, d.fcopy[f], &status);
        p1.ro = p1.ro * sq(radius) / sq(dis);
        p1.p = p1.p * (b.rp[M] / pow2g(dis, g2));
        polar_perenos(x, y, x2, y2, p1.u, p1.v);
        q1[0] = p1.ro; q1[1] = p1.p; q1[2] = p1.u; q1[3] = p1.v; q1[4] = 0.0;
        q2[0] = p2.ro; q2[1] = p2.p; q2[2] = p2.u; q2[3] = p2.v; q2[4] = 0.0;
        godunov_dev<true>(ga, P.kurant, q1, q2, nv, qq, ds, 0.0, 0.0, P.godunov_max_iter, &status);
        o0 = ds[0] * P.koef * 0.1;
        const double tt1 = -n2, tt2 = n1;
        o3 = (fabs(p2.u * tt1 + p2.v * tt2) < 0.1) ? 1.0 : 0.0;
    } else {
        const int jj = j - nC - nI;
        const int lim = P.n_outer_shock + d.dims[0] + d.dims[1] + 1;
        if (jj >= lim) {
            o0 = 0.0;
            o3 = -1.0;
        } else {
            St5 p1, p2;
            tvd_pair(p1, p2);
            q1[0] = p1.ro; q1[1] = p1.p; q1[2] = p1.u; q1[3] = p1.v; q1[4] = 0.0;
            q2[0] = p2.ro; q2[1] = p2.p; q2[2] = p2.u; q2[3] = p2.v; q2[4] = 0.0;
            godunov_dev<true>(ga, P.kurant, q1, q2, nv, qq, ds, 0.0, 0.0, P.godunov_max_iter, &status);
            o0 = ds[1] * P.koef;
            const double tt1 = -n2, tt2 = n1;
            double br;
            if ((sq(p1.u) + sq(p1.v) + sq(0.0)) / (ga * p1.p / p1.ro) > 1.0) br = 0.0;
            else if (fabs(p1.u * tt1 + p1.v * tt2) < 0.01) br = 1.0;
            else if (p1.u * tt1 + p1.v * tt2 > 0) br = 2.0;
            else br = 3.0;
            o3 = br;
        }
    }
    status = static_cast<int>(__reduce_or_sync(0xffffffffu, static_cast<unsigned>(status)));
    if (lane == 0) {
        double* out = scratch + 4 * j;
        out[0] = o0;
        out[1] = n1;
        out[2] = n2;
        out[3] = o3;
        if (status) atomicOr(b.status, status);
    }
}

__global__ void __launch_bounds__(64) surface_faces_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                           double* __restrict__ scratch) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (j >= d.n_lc + d.n_li + d.n_lo) return;
    surface_face_body(d, P, b, scratch, j, threadIdx.x & 31);
}

// ------------------------------------------------------------------ per-face batches (known-answer checks)
__global__ void hllc_batch_kernel(gelios_params P, int n, const double* __restrict__ in, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + 16 * i;
    St5 L, R;
    L.ro = a[0]; L.Q = a[1]; L.p = a[2]; L.u = a[3]; L.v = a[4];
    R.ro = a[5]; R.Q = a[6]; R.p = a[7]; R.u = a[8]; R.v = a[9];
    FluxOut<double> F;
    double t;
    if (P.precision == GELIOS_PREC_FP32_FLUX)
        t = hllc_flux<float>(P.gamma, P.kurant, L, R, a[10], a[11], a[12], a[13], (int)a[14], a[15] != 0.0, F);
    else if (P.precision == GELIOS_PREC_FP32_WAVES)
        t = hllc_flux<WaveF32>(P.gamma, P.kurant, L, R, a[10], a[11], a[12], a[13], (int)a[14], a[15] != 0.0, F);
    else
        t = hllc_flux<double>(P.gamma, P.kurant, L, R, a[10], a[11], a[12], a[13], (int)a[14], a[15] != 0.0, F);
    t = P.kurant * a[13] / t;
    double* o = out + 9 * i;
    o[0] = t;
    o[1] = F.P0;
    o[2] = F.P1;
    o[3] = F.P2;
    o[4] = F.P3;
    o[5] = F.PQ;
    // wave speeds (Vl, Vc, Vp) recomputed in FP64 for the check
    const double n1 = a[11], n2 = a[12];
    const double u1 = L.u * n1 + L.v * n2, u2 = R.u * n1 + R.v * n2;
    const double cL = sqrt(P.gamma * L.p / L.ro), cR = sqrt(P.gamma * R.p / R.ro);
    const double SL = dmin_ref(u1, u2) - dmax_ref(cL, cR);
    const double SR = dmax_ref(u1, u2) + dmax_ref(cL, cR);
    const double suR = SR - u2, suL = SL - u1;
    o[6] = SL;
    o[7] = (suR * R.ro * u2 - suL * L.ro * u1 - R.p + L.p) / (suR * R.ro - suL * L.ro);
    o[8] = SR;
}

// One warp per problem (the warp-cooperative solver of the step kernels).
__global__ void godunov_batch_kernel(gelios_params P, int n, const double* __restrict__ in, double* __restrict__ out) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;
    const double* a = in + 15 * i;
    double q1[5], q2[5], nv[3], qq[5], ds[3];
    for (int k = 0; k < 5; k++) {
        q1[k] = a[k];
        q2[k] = a[5 + k];
    }
    nv[0] = a[10]; nv[1] = a[11]; nv[2] = a[12];
    int status = 0;
    const double t = P.kurant * a[14] / godunov_dev<true>(P.gamma, P.kurant, q1, q2, nv, qq, ds, a[13], a[14],
                                                          P.godunov_max_iter, &status);
    if ((threadIdx.x & 31) != 0) return;
    double* o = out + 10 * i;
    o[0] = t;
    for (int k = 0; k < 5; k++) o[1 + k] = qq[k];
    o[6] = ds[0];
    o[7] = ds[1];
    o[8] = ds[2];
    o[9] = status;
}

// HLLDQ_Korolkov batch: in[23] = L[9], R[9], n[3], rad, metod; out[10] =
// time, P[8], PQ.
__global__ void hlldq_batch_kernel(gelios_params P, int n, const double* __restrict__ in, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + 23 * i;
    double L[9], R[9], Po[8], PQ = 0.0;
    for (int k = 0; k < 9; k++) {
        L[k] = a[k];
        R[k] = a[9 + k];
    }
    for (int k = 0; k < 8; k++) Po[k] = 0.0;
    const double t = hlldq_korolkov(P.gamma, P.kurant, L, R, a[18], a[19], a[20], a[21], static_cast<int>(a[22]),
                                    Po, &PQ);
    double* o = out + 10 * i;
    o[0] = t;
    for (int k = 0; k < 8; k++) o[1 + k] = Po[k];
    o[9] = PQ;
}

// HLLD_Solver_Alexashov batch: in[21] = q1[8], q2[8], n[3], w, dist; out[13]
// = time, q[8], dsl, dsp, dsc, status.
__global__ void hlld_batch_kernel(gelios_params P, int n, const double* __restrict__ in, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* a = in + 21 * i;
    double q1[8], q2[8], nv[3], q[8], ds[3];
    for (int k = 0; k < 8; k++) {
        q1[k] = a[k];
        q2[k] = a[8 + k];
    }
    nv[0] = a[16];
    nv[1] = a[17];
    nv[2] = a[18];
    int status = 0;
    const double t = hlld_alexashov(P.gamma, P.kurant, q1, q2, nv, q, ds, a[19], a[20], &status);
    double* o = out + 13 * i;
    o[0] = t;
    for (int k = 0; k < 8; k++) o[1 + k] = q[k];
    o[9] = ds[0];
    o[10] = ds[1];
    o[11] = ds[2];
    o[12] = status;
}

// ------------------------------------------------------------------ four hydrogen fluids
// Setka::Go_5_komponent (Setka.cpp:8269-8950): the plasma and four hydrogen
// fluids H1..H4, each with its own HLLC flux, on the grid moved by
// Move_surface + Move_Setka_Calculate.  The 21-field state follows the
// member order of Parametr's aggregate initialisers (Gran.cpp:262-265):
// ro, p, u, v, Q, then ro, p, u, v of H1..H4.  One thread per cell, faces in
// Grans order, every face evaluated from each side as the reference does.
struct St21 {
    double f[21];
};
constexpr int kRo = 0, kP = 1, kU = 2, kV = 3, kQ = 4;
__device__ __forceinline__ int fh(int k, int j) { return 5 + 4 * k + j; }  // hydrogen fluid k: ro, p, u, v
constexpr double kHPow = 0.5;              // H_pow, Help.h:90
constexpr double kNHOverKn = 1.0 / 6.0;   // n_H_LISM_ / Kn_, Help.h:60, 65

__device__ __forceinline__ St21 load21(const double* const* st, const double* __restrict__ hs, size_t nc, int c) {
    St21 s;
#pragma unroll
    for (int q = 0; q < 5; q++) s.f[q] = st[q][c];
#pragma unroll
    for (int q = 0; q < 16; q++) s.f[5 + q] = hs[q * nc + c];
    return s;
}
__device__ __forceinline__ void mirror21(St21& s) {
    s.f[kV] = -s.f[kV];
#pragma unroll
    for (int k = 0; k < 4; k++) s.f[fh(k, 3)] = -s.f[fh(k, 3)];
}

// Inner_sphere with the hydrogen fluids (Gran.cpp:236-265, 520-534): plasma
// and H1 of the solar wind, H2..H4 of the master cell.
__device__ __forceinline__ St21 inner_sphere21(const gelios_params& P, double x, double y, const St21& master) {
    St21 s = master;
    const St5 w = inner_sphere_state(P, x, y);
    s.f[kRo] = w.ro;
    s.f[kP] = w.p;
    s.f[kU] = w.u;
    s.f[kV] = w.v;
    s.f[kQ] = w.Q;
    const double dist = sqrt(x * x + y * y);
    s.f[fh(0, 0)] = 0.0000001;
    s.f[fh(0, 1)] = (0.0000001 * P.chi * P.chi / (P.gamma * 14.1344 * 14.1344));
    s.f[fh(0, 2)] = P.chi * x / dist;
    s.f[fh(0, 3)] = P.chi * y / dist;
    return s;
}
// Input (Gran.cpp:267-276, 536-545): plasma and H4 of the LISM, H1..H3 of the master cell.
__device__ __forceinline__ St21 input21(const gelios_params& P, const St21& master) {
    St21 s = master;
    s.f[kRo] = P.in_ro;
    s.f[kP] = P.in_p;
    s.f[kU] = P.in_u;
    s.f[kV] = P.in_v;
    s.f[kQ] = P.in_Q;
    s.f[fh(3, 0)] = 1.0;
    s.f[fh(3, 1)] = 0.5;
    s.f[fh(3, 2)] = P.in_u;  // Velosity_inf
    s.f[fh(3, 3)] = 0.0;
    return s;
}

// Gran::Get_par with the hydrogen fluids (Gran.cpp:205-289); own = the face
// master's state.
__device__ St21 get_par21(const gelios_params& P, int ft, const St21& own, const double* const* st,
                          const double* __restrict__ hs, size_t nc, int nb, double fx, double fy) {
    switch (ft) {
        case G_USUALY: return load21(st, hs, nc, nb);
        case G_EXTERN: {
            St21 s = own;
            if (s.f[kU] >= 0.0) s.f[kU] = P.extern_u_par;
            return s;
        }
        case G_AXIS: {
            St21 s = own;
            mirror21(s);
            return s;
        }
        case G_INNER_SPHERE: return inner_sphere21(P, fx, fy, own);
        case G_INPUT: return input21(P, own);
        default: return own;  // Upper_wall
    }
}

// Gran::Get_par_TVD of an Usualy face with the hydrogen fluids
// (Gran.cpp:296-472): master M (state Ms, centroid Mx, My), Sosed So,
// Sosed_down Sd, face centre (fx, fy).
__device__ St21 tvd21_usualy(const double* const* st, const double* __restrict__ hs, size_t nc, const double* cx,
                             const double* cy, double fx, double fy, const St21& Ms, double Mx, double My, int So,
                             int Sd, bool m_has_axis, bool tracked, int* status) {
    if (Sd < 0) {
        St21 par = Ms;
        if (m_has_axis) {  // Gran.cpp:308-338: mirrored master below the axis
            const St21 par3 = load21(st, hs, nc, So);
            const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
            const double dist3 = sqrt(sq(fx - cx[So]) + sq(fy - cy[So]));
            const double dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
            const int vi[5] = {kV, fh(0, 3), fh(1, 3), fh(2, 3), fh(3, 3)};
#pragma unroll
            for (int q = 0; q < 5; q++)
                par.f[vi[q]] = linear3(-dist1, -Ms.f[vi[q]], -dist2, Ms.f[vi[q]], dist3, par3.f[vi[q]], 0.0);
        }
        return par;
    }
    const St21 par1 = load21(st, hs, nc, Sd);
    const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
    St21 o;
    if (tracked) {  // Gran.cpp:345-426
        const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
        const double r = 1.0 / (-dist1 - (-dist2)), x2 = -dist2;
#pragma unroll
        for (int q = 0; q < 21; q++) o.f[q] = (par1.f[q] - Ms.f[q]) * r * (0.0 - x2) + Ms.f[q];
        if (o.f[kRo] <= 0.0) o.f[kRo] = Ms.f[kRo];
        if (o.f[kP] <= 0.0) o.f[kP] = Ms.f[kP];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (o.f[fh(k, 0)] <= 0.0) o.f[fh(k, 0)] = Ms.f[fh(k, 0)];
            if (o.f[fh(k, 1)] <= 0.0) o.f[fh(k, 1)] = Ms.f[fh(k, 1)];
        }
        return o;
    }
    const St21 par3 = load21(st, hs, nc, So);
    const double dist3 = sqrt(sq(fx - cx[So]) + sq(fy - cy[So]));
    const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3), x2 = -dist2;
#pragma unroll
    for (int q = 0; q < 21; q++) o.f[q] = linear3r(par1.f[q], Ms.f[q], par3.f[q], r12, r23, x2);
    if (o.f[kRo] <= 0.0 || o.f[kP] <= 0.0) *status |= ST_TVD_BAD;  // the reference exits (Gran.cpp:444-455)
    return o;
}

// Gran::Get_par_TVD of an Axis face with the hydrogen fluids (Gran.cpp:486-519).
__device__ St21 tvd21_axis(const double* const* st, const double* __restrict__ hs, size_t nc, const double* cx,
                           const double* cy, double fx, double fy, const St21& Ms, double Mx, double My, int Sd) {
    St21 o = Ms;
    if (Sd < 0) return o;
    const St21 par1 = load21(st, hs, nc, Sd);
    const double dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
    const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    const int vi[5] = {kV, fh(0, 3), fh(1, 3), fh(2, 3), fh(3, 3)};
#pragma unroll
    for (int q = 0; q < 5; q++)
        o.f[vi[q]] = linear3(-dist1, par1.f[vi[q]], -dist2, Ms.f[vi[q]], dist2, -Ms.f[vi[q]], 0.0);
    return o;
}

// Gran::Get_par_TVD_radial with the H1 fields (Gran.cpp:562-675): o = ro,
// p, p_H1, ro_H1 (the fields Go_5_komponent takes from it,
// Setka.cpp:8342-8349).
__device__ void tvd21_radial(const double* const* st, const double* __restrict__ hs, size_t nc, const double* cx,
                             const double* cy, double fx, double fy, const St21& Ms, double Mx, double My, int So,
                             int Sd, bool m_has_axis, double g2, double* o) {
    const double r = sqrt(sq(fx) + sq(fy));
    St21 par1, par3;
    double r1, r2, r3, dist1, dist2, dist3;
    if (Sd < 0) {
        if (!m_has_axis) {
            o[0] = Ms.f[kRo];
            o[1] = Ms.f[kP];
            o[2] = Ms.f[fh(0, 1)];
            o[3] = Ms.f[fh(0, 0)];
            return;
        }
        par1 = Ms;
        mirror21(par1);
        par3 = load21(st, hs, nc, So);
        r2 = sqrt(sq(Mx) + sq(My));
        dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
        r3 = sqrt(sq(cx[So]) + sq(cy[So]));
        dist3 = sqrt(sq(fx - cx[So]) + sq(fy - cy[So]));
        r1 = sqrt(sq(Mx) + sq(-My));
        dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
    } else {
        par1 = load21(st, hs, nc, Sd);
        par3 = load21(st, hs, nc, So);
        r2 = sqrt(sq(Mx) + sq(My));
        dist2 = sqrt(sq(fx - Mx) + sq(fy - My));
        r3 = sqrt(sq(cx[So]) + sq(cy[So]));
        dist3 = sqrt(sq(fx - cx[So]) + sq(fy - cy[So]));
        r1 = sqrt(sq(cx[Sd]) + sq(cy[Sd]));
        dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    }
    const double r12 = 1.0 / (-dist1 - (-dist2)), r23 = 1.0 / (-dist2 - dist3), x2 = -dist2;
    o[0] = linear3r(par1.f[kRo] * sq(r1), Ms.f[kRo] * sq(r2), par3.f[kRo] * sq(r3), r12, r23, x2) / sq(r);
    o[1] = linear3r(par1.f[kP] * pow(r1, g2), Ms.f[kP] * pow(r2, g2), par3.f[kP] * pow(r3, g2), r12, r23, x2) /
           pow(r, g2);
    o[2] = linear3r(par1.f[fh(0, 1)], Ms.f[fh(0, 1)], par3.f[fh(0, 1)], r12, r23, x2);
    o[3] = linear3r(par1.f[fh(0, 0)] * pow(r1, kHPow), Ms.f[fh(0, 0)] * pow(r2, kHPow),
                    par3.f[fh(0, 0)] * pow(r3, kHPow), r12, r23, x2) /
           pow(r, kHPow);
}

// radial scaling of a side's state to the face centre (Setka.cpp:8337-8341)
__device__ __forceinline__ void radial_scale21(St21& s, double rc, double dis, double g2) {
    s.f[kRo] = s.f[kRo] * sq(rc) / sq(dis);
    s.f[fh(0, 0)] = s.f[fh(0, 0)] * pow(rc / dis, kHPow);
    s.f[kQ] = s.f[kQ] * sq(rc) / sq(dis);
    s.f[kP] = s.f[kP] * pow(rc / dis, g2);
}

// conservative update of one hydrogen fluid with its sources and the
// cylindrical terms (Setka.cpp:8808-8940)
__device__ __forceinline__ void k5_update_h(double ga, const double* pot, double ro_H, double p_H, double u_H,
                                            double v_H, double q1, double q21, double q22, double q3, double VV,
                                            double rV2, double y, double dt, double ro_floor, double p_floor,
                                            double* out, int& nro, int& npc) {
    double ro3 = ro_H * VV - dt * (pot[0] * rV2 + ro_H * v_H / y - q1);
    if (ro3 <= 0) {
        ro3 = ro_floor;
        nro++;
    }
    const double rro3 = 1.0 / ro3;
    const double u3 = (ro_H * u_H * VV - dt * (pot[1] * rV2 + ro_H * v_H * u_H / y - q21)) * rro3;
    const double v3 = (ro_H * v_H * VV - dt * (pot[2] * rV2 + ro_H * v_H * v_H / y - q22)) * rro3;
    double p3 = (((p_H / (ga - 1) + ro_H * (u_H * u_H + v_H * v_H) * 0.5) * VV -
                  dt * (pot[3] * rV2 + v_H * (ga * p_H / (ga - 1) + ro_H * (u_H * u_H + v_H * v_H) * 0.5) / y - q3)) -
                 0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                (ga - 1);
    if (p3 <= 0) {
        p3 = p_floor;
        npc++;
    }
    out[0] = ro3;
    out[1] = p3;
    out[2] = u3;
    out[3] = v3;
}

// Go_5_komponent face units (the face loop of Setka.cpp:8300-8570): each
// face once, after the motion.  Both sides' 21-field reconstructions (the
// plasma and H1..H4; radial in C_1 cells), four hydrogen HLLC problems and
// the plasma's HLLC (exact Godunov plus HLLC's tracer flux on tracked
// faces); F*S to the owner slot, -F*S to the twin (the reference evaluates
// the face from each side; the two results are negatives of each other up to
// rounding).  Flux rows: plasma mass, mom x, mom y, energy, Q (0-4), then
// mass, mom x, mom y, energy of H1..H4 (5-20).  CFL candidates of each
// updated side, H1's only where that side is not C_centr (Setka.cpp:8500).
__global__ void __launch_bounds__(128) k5_face_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                      const double* __restrict__ hcur, double* __restrict__ fl) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    double tmin = __longlong_as_double(0x7ff0000000000000LL);
    int status = 0;
    if (u < d.n_units) {
        const size_t nc = d.n_cells, ng = d.n_slots;
        const int c = d.u_cell[u], nb = d.u_nb[u];
        const uint32_t info = d.u_info[u];
        const uint32_t cf = (info >> UI_CF_OWN) & 15u, nbf = (info >> UI_CF_NB) & 15u;
        const double x = b.cx[c], y = b.cy[c];
        const double radius = sqrt(sq(x) + sq(y));
        const bool procK = !(radius < P.R11);
        double x3 = 0.0, y3 = 0.0;
        bool procN = false;
        if (nb >= 0) {
            x3 = b.cx[nb];
            y3 = b.cy[nb];
            procN = !(sqrt(sq(x3) + sq(y3)) < P.R11);
        }
        if (procK || procN) {
            const double ga = P.gamma, g2 = 2.0 * P.gamma;
            const double dt = *b.dt_cur;
            const bool kC1 = (cf & CF_C1) != 0;
            const St21 par1 = load21(b.cur, hcur, nc, c);
            const int ft = info & SI_TYPE_MASK;
            const int A = d.u_A[u], B = d.u_B[u];
            const double xa = d.X[A], ya = d.Y[A], xb = d.X[B], yb = d.Y[B];
            const double S = sqrt(sq(xb - xa) + sq(yb - ya));
            const double x2 = (xa + xb) / 2.0, y2 = (ya + yb) / 2.0;
            const double x4 = (d.X2[A] + d.X2[B]) / 2.0, y4 = (d.Y2[A] + d.Y2[B]) / 2.0;
            const double dist = sqrt(sq(x - x2) + sq(y - y2));
            St21 par11 = par1;
            St21 par2 = get_par21(P, ft, par1, b.cur, hcur, nc, nb, x2, y2);
            double t1 = xb - xa, t2 = yb - ya;
            const double nn = sqrt(sq(t1) + sq(t2));
            t1 = t1 / nn;
            t2 = t2 / nn;
            const double n1 = t2, n2 = -t1;
            const double W = ((x4 - x2) * n1 + (y4 - y2) * n2) / dt;
            const double dis = sqrt(sq(x2) + sq(y2));
            const bool tracked = (info & SI_GOD) != 0;
            if (ft == G_USUALY) {
                const double dd = sqrt(sq(x3) + sq(y3));
                if (kC1) {
                    radial_scale21(par11, radius, dis, g2);
                    polar_perenos(x, y, x2, y2, par11.f[kU], par11.f[kV]);
                    polar_perenos(x, y, x2, y2, par11.f[fh(0, 2)], par11.f[fh(0, 3)]);
                    double o[4];
                    tvd21_radial(b.cur, hcur, nc, b.cx, b.cy, x2, y2, par1, x, y, nb, d.u_sd[u], (cf & CF_AXIS) != 0,
                                 g2, o);
                    par11.f[kRo] = o[0];
                    par11.f[kP] = o[1];
                    par11.f[fh(0, 1)] = o[2];
                    par11.f[fh(0, 0)] = o[3];
                } else {
                    par11 = tvd21_usualy(b.cur, hcur, nc, b.cx, b.cy, x2, y2, par1, x, y, nb, d.u_sd[u],
                                         (cf & CF_AXIS) != 0, tracked, &status);
                }
                if (nbf & CF_C1) {
                    const St21 parN = par2;  // the neighbour's stored state
                    radial_scale21(par2, dd, dis, g2);
                    polar_perenos(x3, y3, x2, y2, par2.f[kU], par2.f[kV]);
                    polar_perenos(x3, y3, x2, y2, par2.f[fh(0, 2)], par2.f[fh(0, 3)]);
                    double o[4];
                    tvd21_radial(b.cur, hcur, nc, b.cx, b.cy, x2, y2, parN, x3, y3, c, d.u_sd2[u],
                                 (nbf & CF_AXIS) != 0, g2, o);
                    par2.f[kRo] = o[0];
                    par2.f[kP] = o[1];
                    par2.f[fh(0, 1)] = o[2];
                    par2.f[fh(0, 0)] = o[3];
                } else {
                    par2 = tvd21_usualy(b.cur, hcur, nc, b.cx, b.cy, x2, y2, par2, x3, y3, c, d.u_sd2[u],
                                        (nbf & CF_AXIS) != 0, tracked, &status);
                }
            } else if (ft == G_INNER_SPHERE) {
                radial_scale21(par11, radius, dis, g2);
            } else if (kC1 && ft == G_AXIS) {
                radial_scale21(par11, radius, dis, g2);
                polar_perenos(x, y, x2, y2, par11.f[kU], par11.f[kV]);
                polar_perenos(x, y, x2, y2, par11.f[fh(0, 2)], par11.f[fh(0, 3)]);
                par2 = par11;
                mirror21(par2);
            } else if (!kC1 && ft == G_AXIS) {
                par11 = tvd21_axis(b.cur, hcur, nc, b.cx, b.cy, x2, y2, par1, x, y, d.u_sd[u]);
                par2 = par11;
                mirror21(par2);
            }
            const bool np = (info & SI_NP) != 0;
            const int g = d.u_slot[u], gt = d.u_twin[u];
            FluxOut<double> F;
            double UUh[4];
            for (int hk = 0; hk < 4; hk++) {
                St5 L, R;
                L.ro = par11.f[fh(hk, 0)];
                L.p = par11.f[fh(hk, 1)];
                L.u = par11.f[fh(hk, 2)];
                L.v = par11.f[fh(hk, 3)];
                L.Q = par11.f[kQ];
                R.ro = par2.f[fh(hk, 0)];
                R.p = par2.f[fh(hk, 1)];
                R.u = par2.f[fh(hk, 2)];
                R.v = par2.f[fh(hk, 3)];
                R.Q = par2.f[kQ];
                UUh[hk] = hllc_flux<double>(ga, P.kurant, L, R, W, n1, n2, 1.0, 1, false, F);
                const double h[4] = {F.P0 * S, F.P1 * S, F.P2 * S, F.P3 * S};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    fl[(5 + 4 * hk + j) * ng + g] = h[j];
                    if (gt >= 0) fl[(5 + 4 * hk + j) * ng + gt] = -h[j];
                }
            }
            St5 L, R;
            L.ro = par11.f[kRo];
            L.p = par11.f[kP];
            L.u = par11.f[kU];
            L.v = par11.f[kV];
            L.Q = par11.f[kQ];
            R.ro = par2.f[kRo];
            R.p = par2.f[kP];
            R.u = par2.f[kU];
            R.v = par2.f[kV];
            R.Q = par2.f[kQ];
            double pl[5];
            double UG = 0.0;
            if (tracked) {
                double q1[5] = {L.ro, L.p, L.u, L.v, 0.0};
                double q2[5] = {R.ro, R.p, R.u, R.v, 0.0};
                double nvv[3] = {n1, n2, 0.0};
                double qq[5], ds[3];
                UG = godunov_dev<false>(ga, P.kurant, q1, q2, nvv, qq, ds, W, dist, P.godunov_max_iter, &status);
                pl[0] = qq[0] * S;
                pl[1] = qq[1] * S;
                pl[2] = qq[2] * S;
                pl[3] = qq[4] * S;
            }
            const double UU = hllc_flux<double>(ga, P.kurant, L, R, W, n1, n2, 1.0, 1, np, F);
            if (!tracked) {
                pl[0] = F.P0 * S;
                pl[1] = F.P1 * S;
                pl[2] = F.P2 * S;
                pl[3] = F.P3 * S;
            }
            pl[4] = F.PQ * S;
#pragma unroll
            for (int j = 0; j < 5; j++) {
                fl[j * ng + g] = pl[j];
                if (gt >= 0) fl[j * ng + gt] = -pl[j];
            }
            // CFL candidates in the reference's order per side (Setka.cpp:8500-8560)
            auto side = [&](double dd, bool centr) {
                for (int hk = 0; hk < 4; hk++)
                    if (!(hk == 0 && centr)) tmin = dmin_ref(tmin, P.kurant * dd / UUh[hk]);
                if (tracked) tmin = dmin_ref(tmin, P.kurant * dd / UG);
                tmin = dmin_ref(tmin, P.kurant * dd / UU);
            };
            if (procK) side(dist, (cf & CF_CENTR) != 0);
            if (gt >= 0 && procN) side(sqrt(sq(x3 - x2) + sq(y3 - y2)), (nbf & CF_CENTR) != 0);
        }
    }
    block_reduce_commit(tmin, 0, 0, status, b.dt_acc, b.counters, b.status);
}

// Go_5_komponent cell update (Setka.cpp:8570-8950) from the summed face
// slots: multi-fluid charge exchange, cylindrical 1/y terms, clamps; it also
// refills the geometry cache for the next step.
__global__ void __launch_bounds__(128) k5_update_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                        const double* __restrict__ fl,
                                                        const double* __restrict__ hcur, double* __restrict__ hnxt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double tmin = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0, status = 0;
    const size_t nc = d.n_cells;
    if (c < d.n_cells) {
        {  // the next step's geometry cache from the moved points (see mk2_update_cell)
            const int s0 = d.cstart[c], n = d.cstart[c + 1] - s0;
            const int32_t* con = d.contour + s0;
            double xn, yn;
            centroid(con, n, d.X2, d.Y2, xn, yn);
            b.cx_next[c] = xn;
            b.cy_next[c] = yn;
            const uint32_t cfl = d.cflags[c];
            if (cfl & CF_RP) b.rp_next[c] = pow2g(sqrt(sq(xn) + sq(yn)), 2 * P.gamma);
            if (!(cfl & CF_CENTR)) {
                b.vs_next[c] = area(con, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], d.X2, d.Y2, false);
                b.vol_next[c] = volume_rotate(con, n, d.X2, d.Y2);
            }
        }
        const double x = b.cx[c], y = b.cy[c];
        const double radius = sqrt(sq(x) + sq(y));
        if (!(radius < P.R11)) {
            tmin = 10000000.0;  // `time` starts at 1e7 in every step (Setka.cpp:8286)
            const double ga = P.gamma;
            const double dt = *b.dt_cur;
            const int kt = d.ctype[c];
            const St21 par1 = load21(b.cur, hcur, nc, c);
            const int s0 = d.cstart[c], nv = d.cstart[c + 1] - s0;
            const int32_t* con = d.contour + s0;
            const int g0 = d.gstart[c], g1 = d.gstart[c + 1];
            const double Volume = area(con, nv, d.sA, d.sB, g0, g1, d.X, d.Y, false);
            const double Volume2 = area(con, nv, d.sA, d.sB, g0, g1, d.X2, d.Y2, true);
            // face fluxes summed in Grans order: plasma rows 0-4, hydrogen
            // fluid k rows 5 + 4k .. 8 + 4k
            const size_t ng = d.n_slots;
            double Potok[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            double PH[4][4];
#pragma unroll
            for (int k = 0; k < 4; k++)
#pragma unroll
                for (int j = 0; j < 4; j++) PH[k][j] = 0.0;
            for (int g = g0; g < g1; g++) {
#pragma unroll
                for (int j = 0; j < 5; j++) Potok[j] = Potok[j] + fl[j * ng + g];
#pragma unroll
                for (int k = 0; k < 4; k++)
#pragma unroll
                    for (int j = 0; j < 4; j++) PH[k][j] = PH[k][j] + fl[(5 + 4 * k + j) * ng + g];
            }
            // multi-fluid charge exchange (Setka.cpp:8575-8660)
            const double u = par1.f[kU], v = par1.f[kV], ro = par1.f[kRo], p = par1.f[kP], Q = par1.f[kQ];
            double UM[4], UH[4], nu[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double roH = par1.f[fh(k, 0)], pH = par1.f[fh(k, 1)];
                const double uH = par1.f[fh(k, 2)], vH = par1.f[fh(k, 3)];
                UM[k] = sqrt(sq(u - uH) + sq(v - vH) + (64.0 / (9.0 * kPi)) * (p / ro + 2.0 * pH / roH));
                UH[k] = sqrt(sq(u - uH) + sq(v - vH) + (4.0 / kPi) * (p / ro + 2.0 * pH / roH));
                nu[k] = ro * roH * UM[k] * sq(1.0 - P.a_2 * log(UM[k]));
            }
            const double cp = P.src_coef;  // n_p_LISM_ / Kn_
            const double q2_1 = cp * (nu[0] * (par1.f[fh(0, 2)] - u) + nu[1] * (par1.f[fh(1, 2)] - u) +
                                      nu[2] * (par1.f[fh(2, 2)] - u) + nu[3] * (par1.f[fh(3, 2)] - u));
            const double q2_2 = cp * (nu[0] * (par1.f[fh(0, 3)] - v) + nu[1] * (par1.f[fh(1, 3)] - v) +
                                      nu[2] * (par1.f[fh(2, 3)] - v) + nu[3] * (par1.f[fh(3, 3)] - v));
            double e[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double roH = par1.f[fh(k, 0)], pH = par1.f[fh(k, 1)];
                const double uH = par1.f[fh(k, 2)], vH = par1.f[fh(k, 3)];
                e[k] = nu[k] * ((sq(uH) + sq(vH) - sq(u) - sq(v)) / 2.0 + (UH[k] / UM[k]) * (2.0 * pH / roH - p / ro));
            }
            const double q3 = cp * (e[0] + e[1] + e[2] + e[3]);
            const double rV2 = 1.0 / Volume2, VV = Volume * rV2;
            if (kt != C_CENTR) {
                double ro3 = ro * VV - dt * (Potok[0] * rV2 + ro * v / y);
                const double Q33 = Q * VV - (dt * rV2) * Potok[4] - dt * Q * v / y;
                if (ro3 <= 0.0) {
                    ro3 = P.ro_floor;
                    nro++;
                }
                const double rro3 = 1.0 / ro3;
                const double u3 = (ro * u * VV - dt * (Potok[1] * rV2 + ro * v * u / y - q2_1)) * rro3;
                const double v3 = (ro * v * VV - dt * (Potok[2] * rV2 + ro * v * v / y - q2_2)) * rro3;
                double p3 = (((p / (ga - 1) + ro * (u * u + v * v) * 0.5) * VV -
                              dt * (Potok[3] * rV2 + v * (ga * p / (ga - 1) + ro * (u * u + v * v) * 0.5) / y - q3)) -
                             0.5 * ro3 * (u3 * u3 + v3 * v3)) *
                            (ga - 1);
                if (p3 <= 0) {
                    p3 = P.p_floor;
                    npc++;
                }
                b.nxt[0][c] = ro3;
                b.nxt[1][c] = p3;
                b.nxt[2][c] = u3;
                b.nxt[3][c] = v3;
                b.nxt[4][c] = Q33;
            } else {
#pragma unroll
                for (int q = 0; q < 5; q++) b.nxt[q][c] = par1.f[q];
            }
            // hydrogen sources by cell kind (Setka.cpp:8734-8806)
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
#pragma unroll
            for (int k = 0; k < 4; k++) s2[k] = nu[k] * ((sq(u) + sq(v)) / 2.0 + (UH[k] / UM[k]) * (p / ro));
            const double S2 = s2[0] + s2[1] + s2[2] + s2[3];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const double roH = par1.f[fh(k, 0)], pH = par1.f[fh(k, 1)];
                const double uH = par1.f[fh(k, 2)], vH = par1.f[fh(k, 3)];
                double out[4];
                if (k == 0 && kt == C_CENTR) {
                    out[0] = roH;
                    out[1] = pH;
                    out[2] = uH;
                    out[3] = vH;
                } else {
                    const double q1h = kNHOverKn * (kk[k] * S1 - nu[k]);
                    const double q21h = kNHOverKn * (kk[k] * S1 * u - nu[k] * uH);
                    const double q22h = kNHOverKn * (kk[k] * S1 * v - nu[k] * vH);
                    const double q3h = kNHOverKn * (kk[k] * S2 - nu[k] * ((sq(uH) + sq(vH)) / 2.0 +
                                                                         (UH[k] / UM[k]) * 2.0 * (pH / roH)));
                    // floors: Setka.cpp:8817, 8829, 8859, 8871, 8893, 8905, 8927, 8939
                    const double rf = k == 0 ? 0.0000001 : 0.000001;
                    const double pf = k == 3 ? 0.0000001 : 0.000001;
                    k5_update_h(ga, PH[k], roH, pH, uH, vH, q1h, q21h, q22h, q3h, VV, rV2, y, dt, rf, pf, out, nro,
                                npc);
                }
#pragma unroll
                for (int j = 0; j < 4; j++) hnxt[(4 * k + j) * nc + c] = out[j];
            }
        }
    }
    block_reduce_commit(tmin, nro, npc, status, b.dt_acc, b.counters, b.status);
}

// ------------------------------------------------------------------ MHD + pickup protons
// GELIOS_FORM_MHD_PUI (no reference step).  The ion fluid's gas-dynamic
// rows (ro, p, u, v, Q) are the state rows of the moving-grid step, so
// surface tracking and the rails run on them unchanged; the extra rows hold
// the ion's w (u_phi) and B (x, y, phi) and the pickup protons' ro, p, u, v.
enum : int { kXw = 0, kXbx, kXby, kXbz, kXro, kXp, kXu, kXv, kMhdExtra };
constexpr int kMhdFlux = 13;  // per slot: ion mass, mom x, y, phi, energy, Bx, By, Bphi, Q; pickup mass, mom x, y, energy

struct Ext8 {
    double f[kMhdExtra];
};

__device__ __forceinline__ Ext8 load_ext(const double* __restrict__ hs, size_t nc, int c) {
    Ext8 e;
#pragma unroll
    for (int k = 0; k < kMhdExtra; k++) e.f[k] = hs[k * nc + c];
    return e;
}
// mirror image across the axis: radial and azimuthal components change sign
__device__ __forceinline__ void mirror_ext(Ext8& e) {
    e.f[kXw] = -e.f[kXw];
    e.f[kXby] = -e.f[kXby];
    e.f[kXbz] = -e.f[kXbz];
    e.f[kXv] = -e.f[kXv];
}

// Gran::Get_par's boundary rules (Gran.cpp:205-289) applied to the extra
// rows; `ion` is the ion state the same rule gave (inner sphere: the wind).
__device__ __forceinline__ Ext8 get_par_ext(const gelios_params& P, const gelios_mhd_params& M, int ft,
                                            const Ext8& own, const double* __restrict__ hs, size_t nc, int nb,
                                            double fx, double fy, const St5& ion) {
    Ext8 e = own;
    if (ft == G_USUALY) {
        e = load_ext(hs, nc, nb);
    } else if (ft == G_EXTERN) {
        if (e.f[kXu] >= 0.0) e.f[kXu] = P.extern_u_par;
    } else if (ft == G_AXIS) {
        mirror_ext(e);
    } else if (ft == G_INNER_SPHERE) {
        const double dist = sqrt(fx * fx + fy * fy);
        e.f[kXw] = 0.0;
        e.f[kXbx] = 0.0;
        e.f[kXby] = 0.0;
        e.f[kXbz] = M.inner_bphi * (P.R1 / dist) * (fy / dist);
        e.f[kXro] = M.pui_inner_ro * ion.ro;
        e.f[kXp] = M.pui_inner_p * ion.p;
        e.f[kXu] = ion.u;
        e.f[kXv] = ion.v;
    } else if (ft == G_INPUT) {
        e.f[kXw] = 0.0;
        e.f[kXbx] = M.lism_bx;
        e.f[kXby] = M.lism_by;
        e.f[kXbz] = M.lism_bz;
        e.f[kXro] = M.pui_in_ro;
        e.f[kXp] = M.pui_in_p;
        e.f[kXu] = P.in_u;
        e.f[kXv] = P.in_v;
    }
    return e;
}

// All 13 rows at a Usualy face seen from M (ion Ms, extra Me, centre Mx,My,
// flags mf), with the cell So across the face already loaded (Ss, Se,
// centre Sx,Sy) and Sosed_down Sd: the ion rows follow mk2_usualy_side
// (Get_par_TVD / Get_par_TVD_radial in C_1 cells), the extra rows tvd_ext's
// rule, with the stencil distances computed once for both.
__device__ __forceinline__ void mhd_usualy_side(const double* const* st, const double* __restrict__ hs, size_t nc,
                                                const double* cx, const double* cy, const double* rp, double fx,
                                                double fy, double dis, double pdis, const St5& Ms, const Ext8& Me,
                                                double Mx, double My, double rpM, uint32_t mf, int So, const St5& Ss,
                                                const Ext8& Se, double Sx, double Sy, int Sd, bool tracked,
                                                double rM, double rS, double dM, double dS, St5& oi, Ext8& oe,
                                                int* status) {
    // rM, rS: |centroid| of M and So; dM, dS: face centre to those centroids
    if (mf & CF_C1) {
        oi = mk2_usualy_side_d(st, cx, cy, rp, fx, fy, dis, pdis, Ms, Mx, My, rpM, mf, So, Sd, tracked, rM, rS, dM,
                               dS, status);
        oe = Me;
        return;
    }
    oi = Ms;
    oe = Me;
    if (Sd < 0) {
        if (mf & CF_AXIS) {  // Gran.cpp:308-338
            const double dist2 = dM;
            const double dist3 = dS;
            const double dist1 = sqrt(sq(fx - Mx) + sq(fy - (-My)));
            oi.v = linear3(-dist1, -Ms.v, -dist2, Ms.v, dist3, Ss.v, 0.0);
        }
        return;
    }
    const St5 s1 = load_state(st, Sd);
    const Ext8 e1 = load_ext(hs, nc, Sd);
    const double dist2 = dM;
    const double dist1 = sqrt(sq(fx - cx[Sd]) + sq(fy - cy[Sd]));
    const double r12 = 1.0 / (-dist1 - (-dist2)), x2 = -dist2;
    if (tracked) {  // Gran.cpp:345-426
        oi.ro = (s1.ro - Ms.ro) * r12 * (0.0 - x2) + Ms.ro;
        oi.p = (s1.p - Ms.p) * r12 * (0.0 - x2) + Ms.p;
        oi.u = (s1.u - Ms.u) * r12 * (0.0 - x2) + Ms.u;
        oi.v = (s1.v - Ms.v) * r12 * (0.0 - x2) + Ms.v;
        oi.Q = (s1.Q - Ms.Q) * r12 * (0.0 - x2) + Ms.Q;
        if (oi.ro <= 0.0) oi.ro = Ms.ro;
        if (oi.p <= 0.0) oi.p = Ms.p;
#pragma unroll
        for (int k = 0; k < kMhdExtra; k++) oe.f[k] = (e1.f[k] - Me.f[k]) * r12 * (0.0 - x2) + Me.f[k];
    } else {
        const double dist3 = dS;
        const double r23 = 1.0 / (-dist2 - dist3);
        oi.ro = linear3r(s1.ro, Ms.ro, Ss.ro, r12, r23, x2);
        oi.p = linear3r(s1.p, Ms.p, Ss.p, r12, r23, x2);
        oi.u = linear3r(s1.u, Ms.u, Ss.u, r12, r23, x2);
        oi.v = linear3r(s1.v, Ms.v, Ss.v, r12, r23, x2);
        oi.Q = linear3r(s1.Q, Ms.Q, Ss.Q, r12, r23, x2);
        if (oi.ro <= 0.0 || oi.p <= 0.0) *status |= ST_TVD_BAD;  // the reference exits (Gran.cpp:444-455)
#pragma unroll
        for (int k = 0; k < kMhdExtra; k++) oe.f[k] = linear3r(e1.f[k], Me.f[k], Se.f[k], r12, r23, x2);
    }
    if (!(oe.f[kXro] > 0.0)) oe.f[kXro] = Me.f[kXro];
    if (!(oe.f[kXp] > 0.0)) oe.f[kXp] = Me.f[kXp];
}

// Ion MHD flux through a face with unit normal (n1, n2) moving with normal
// speed W: both states go to the face frame (normal n, tangent t = (-n2,
// n1), phi), Solvers::HLLDQ_Korolkov's HLLD (metod 3) solves along the
// frame's x axis with its fan sampled at W (hlldq_impl<true>: F - W U of
// the region containing W, as HLLC_2d_Korolkov_b_s does for moving faces),
// and the momentum and field fluxes go back to (x, y).  out: mass, mom x,
// mom y, mom phi, energy, Bx, By, Bphi, Q.  Returns 1 / max(|SL|, |SR|).
template <typename TF>
__device__ __forceinline__ double mhd_face_flux(double ga, const St5& iL, const Ext8& eL, const St5& iR,
                                                const Ext8& eR, double n1, double n2, double W, double* out) {
    const double t1 = -n2, t2 = n1;
    double L[9], R[9];
    L[0] = iL.ro;
    L[1] = iL.Q;
    L[2] = iL.p;
    L[3] = iL.u * n1 + iL.v * n2;
    L[4] = iL.u * t1 + iL.v * t2;
    L[5] = eL.f[kXw];
    L[6] = eL.f[kXbx] * n1 + eL.f[kXby] * n2;
    L[7] = eL.f[kXbx] * t1 + eL.f[kXby] * t2;
    L[8] = eL.f[kXbz];
    R[0] = iR.ro;
    R[1] = iR.Q;
    R[2] = iR.p;
    R[3] = iR.u * n1 + iR.v * n2;
    R[4] = iR.u * t1 + iR.v * t2;
    R[5] = eR.f[kXw];
    R[6] = eR.f[kXbx] * n1 + eR.f[kXby] * n2;
    R[7] = eR.f[kXbx] * t1 + eR.f[kXby] * t2;
    R[8] = eR.f[kXbz];
    double F[8], FQ;
    const double tinv = hlld_face_moving<TF>(ga, L, R, W, F, &FQ);
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

// One face unit of the MHD form, after the motion: reconstructions of both
// sides (ion rows: the moving-grid rules of Setka.cpp:10204-10276, extra
// rows: mhd_usualy_side / get_par_ext) on the pre-motion points, face speed
// from the moved points, HLLD for the ions and HLLC for the pickup protons,
// 13 flux rows times S to the owner slot and their negatives to the twin,
// CFL candidates of both fluids.  BLOCK x MINB: the launch shape (threads
// per block, minimum resident blocks per SM, which caps the registers).
// PLAIN: a unit of the plain interior group [0, u_c1) (see mk2_recon_unit).
template <typename TF, bool PLAIN = false>
__device__ __forceinline__ double mhd_face_body(const DevMesh& d, const gelios_params& P, const gelios_mhd_params& M,
                                                const StepBuffers& b, const double* __restrict__ hs,
                                                double* __restrict__ fl, int u, int& status) {
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    {
        const size_t nc = d.n_cells, ng = d.n_slots;
        const int K = d.u_cell[u], nb = d.u_nb[u];
        const uint32_t info = d.u_info[u];
        const double x = b.cx[K], y = b.cy[K];
        // as mk2_recon_unit: the R11 test without a square root, the radii
        // only where a radial reconstruction reads them, the distances once
        const double aK = sq(x) + sq(y);
        const bool procK = !(aK < d.r11_sq);
        double x3 = 0.0, y3 = 0.0, aN = 0.0;
        bool procN = false;
        if (nb >= 0) {
            x3 = b.cx[nb];
            y3 = b.cy[nb];
            aN = sq(x3) + sq(y3);
            procN = !(aN < d.r11_sq);
        }
        if (procK || procN) {
            const double rK = PLAIN ? 0.0 : sqrt(aK), rN = PLAIN ? 0.0 : sqrt(aN);
            const int A = d.u_A[u], B = d.u_B[u];
            const double xa = d.X[A], ya = d.Y[A], xb = d.X[B], yb = d.Y[B];
            const double x2 = (xa + xb) / 2.0, y2 = (ya + yb) / 2.0;
            const double dK = sqrt(sq(x - x2) + sq(y - y2));
            const double dN = sqrt(sq(x3 - x2) + sq(y3 - y2));
            double t1 = xb - xa, t2 = yb - ya;
            const double nn = sqrt(sq(t1) + sq(t2));
            t1 = t1 / nn;
            t2 = t2 / nn;
            const double n1 = t2, n2 = -t1;
            const double S = nn * (ya + yb) * 0.5;
            const double x4 = (d.X2[A] + d.X2[B]) / 2.0, y4 = (d.Y2[A] + d.Y2[B]) / 2.0;
            const double dt = *b.dt_cur;
            const double W = ((x4 - x2) * n1 + (y4 - y2) * n2) / dt;
            const int ft = PLAIN ? static_cast<int>(G_USUALY) : static_cast<int>(info & SI_TYPE_MASK);
            const uint32_t cmask = PLAIN ? (15u & ~CF_C1) : 15u;
            const uint32_t cf = (info >> UI_CF_OWN) & cmask, nbf = (info >> UI_CF_NB) & cmask;
            const double g2 = 2 * P.gamma;
            const St5 par1 = load_state(b.cur, K);
            const Ext8 ex1 = load_ext(hs, nc, K);
            St5 par11 = par1, par2 = get_par(P, ft, par1, b.cur, nb, x2, y2);
            Ext8 e11 = ex1, e2 = get_par_ext(P, M, ft, ex1, hs, nc, nb, x2, y2, par2);
            const double dis = sqrt(sq(x2) + sq(y2));
            const bool tracked = !PLAIN && (info & SI_GOD) != 0;
            const bool radial = ((cf & CF_C1) && (ft == G_USUALY || ft == G_AXIS)) || ft == G_INNER_SPHERE ||
                                (ft == G_USUALY && (nbf & CF_C1));
            const double pdis = radial ? pow2g(dis, g2) : 1.0;
            if (ft == G_USUALY) {
                const St5 sN = par2;
                const Ext8 eN = e2;
                mhd_usualy_side(b.cur, hs, nc, b.cx, b.cy, b.rp, x2, y2, dis, pdis, par1, ex1, x, y, b.rp[K], cf, nb,
                                sN, eN, x3, y3, d.u_sd[u], tracked, rK, rN, dK, dN, par11, e11, &status);
                mhd_usualy_side(b.cur, hs, nc, b.cx, b.cy, b.rp, x2, y2, dis, pdis, sN, eN, x3, y3, b.rp[nb], nbf, K,
                                par1, ex1, x, y, d.u_sd2[u], tracked, rN, rK, dN, dK, par2, e2, &status);
            } else if (ft == G_INNER_SPHERE) {
                const double radius = rK;
                par11.ro = par11.ro * sq(radius) / sq(dis);
                par11.Q = par11.Q * sq(radius) / sq(dis);
                par11.p = par11.p * (b.rp[K] / pdis);
            } else if (ft == G_AXIS) {
                if (cf & CF_C1) {
                    const double radius = sqrt(sq(x) + sq(y));
                    par11.ro = par11.ro * sq(radius) / sq(dis);
                    par11.Q = par11.Q * sq(radius) / sq(dis);
                    par11.p = par11.p * (b.rp[K] / pdis);
                    polar_perenos(x, y, x2, y2, par11.u, par11.v);
                } else {
                    par11 = tvd_axis(b.cur, b.cx, b.cy, x2, y2, par1, x, y, d.u_sd[u]);
                }
                par2 = par11;
                par2.v = -par2.v;
            }
            double F[kMhdFlux];
            const double tI = mhd_face_flux<TF>(P.gamma, par11, e11, par2, e2, n1, n2, W, F);
            St5 pL, pR;
            pL.ro = e11.f[kXro];
            pL.p = e11.f[kXp];
            pL.u = e11.f[kXu];
            pL.v = e11.f[kXv];
            pL.Q = 0.0;
            pR.ro = e2.f[kXro];
            pR.p = e2.f[kXp];
            pR.u = e2.f[kXu];
            pR.v = e2.f[kXv];
            pR.Q = 0.0;
            FluxOut<double> G;
            const double UUp = hllc_flux<TF>(P.gamma, P.kurant, pL, pR, W, n1, n2, 1.0, 1, false, G);
            F[9] = G.P0;
            F[10] = G.P1;
            F[11] = G.P2;
            F[12] = G.P3;
            const int g = d.u_slot[u], gt = d.u_twin[u];
            // slots are read once, by the update: streaming stores
#pragma unroll
            for (int k = 0; k < kMhdFlux; k++) __stcs(fl + k * ng + g, F[k] * S);
            if (gt >= 0) {
#pragma unroll
                for (int k = 0; k < kMhdFlux; k++) __stcs(fl + k * ng + gt, -(F[k] * S));
            }
            if (procK) {
                const double dist = dK;
                tmin_u = dmin_ref(tmin_u, P.kurant * dist * tI);
                tmin_u = dmin_ref(tmin_u, P.kurant * dist / UUp);
            }
            if (gt >= 0 && procN) {
                const double distn = dN;
                tmin_u = dmin_ref(tmin_u, P.kurant * distn * tI);
                tmin_u = dmin_ref(tmin_u, P.kurant * distn / UUp);
            }
        }
    }
    return tmin_u;
}

// PLAIN: the plain interior group [0, u_c1) (lean instance); otherwise the
// units [u_c1, n_units).
template <typename TF, int BLOCK, int MINB, bool PLAIN>
__global__ void __launch_bounds__(BLOCK, MINB) mhd_face_kernel(DevMesh d, gelios_params P, gelios_mhd_params M,
                                                               StepBuffers b, const double* __restrict__ hs,
                                                               double* __restrict__ fl) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int u = PLAIN ? i : d.u_c1 + i;
    double tmin_u = __longlong_as_double(0x7ff0000000000000LL);
    int status = 0;
    if (PLAIN ? u < d.u_c1 : u < d.n_units) tmin_u = mhd_face_body<TF, PLAIN>(d, P, M, b, hs, fl, u, status);
    block_reduce_commit(tmin_u, 0, 0, status, b.dt_acc, b.counters, b.status);
}

// Cell update of the MHD form: the MK2 update (Setka.cpp:10386-10468) for
// both fluids with their axisymmetric terms (area-weighted like the
// reference's p (vs1 + vs2)/2) and the fixed charge-exchange sources of the
// ion momentum and energy; refills the geometry cache like mk2_update_cell.
__device__ __forceinline__ void mhd_update_body(const DevMesh& d, const gelios_params& P, const StepBuffers& b,
                                                const double* __restrict__ fl, const double* __restrict__ src,
                                                const double* __restrict__ hcur, double* __restrict__ hnxt, int c,
                                                double& tmark, int& nro, int& npc) {
    const size_t ng = d.n_slots, nc = d.n_cells;
    {
        const uint32_t cfl = d.cflags[c];
        double xn, yn;
        double vs2 = 0.0, Volume2 = 0.0;
        // quadrilaterals: the four moved corners from one int4 load, the
        // operations of centroid / area / volume_rotate in registers
        const int4 qc = d.qcorner ? d.qcorner[c] : make_int4(-1, -1, -1, -1);
        if (qc.x >= 0) {
            const double qx[4] = {d.X2[qc.x], d.X2[qc.y], d.X2[qc.z], d.X2[qc.w]};
            const double qy[4] = {d.Y2[qc.x], d.Y2[qc.y], d.Y2[qc.z], d.Y2[qc.w]};
            double vq, volq;
            quad_geometry(qx, qy, xn, yn, vq, volq);
            if (!(cfl & CF_CENTR)) {
                vs2 = vq;
                Volume2 = volq;
                b.vs_next[c] = vq;
                b.vol_next[c] = volq;
            }
        } else {
            const int s0 = d.cstart[c], n = d.cstart[c + 1] - s0;
            const int32_t* con = d.contour + s0;
            centroid(con, n, d.X2, d.Y2, xn, yn);
            if (!(cfl & CF_CENTR)) {
                vs2 = area(con, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], d.X2, d.Y2, true);
                Volume2 = volume_rotate(con, n, d.X2, d.Y2);
                b.vs_next[c] =
                    n == 4 ? vs2 : area(con, n, d.sA, d.sB, d.gstart[c], d.gstart[c + 1], d.X2, d.Y2, false);
                b.vol_next[c] = Volume2;
            }
        }
        b.cx_next[c] = xn;
        b.cy_next[c] = yn;
        if (cfl & CF_RP) b.rp_next[c] = pow2g(sqrt(sq(xn) + sq(yn)), 2 * P.gamma);
        const double x = b.cx[c], y = b.cy[c];
        if (!(sqrt(sq(x) + sq(y)) < P.R11)) {
            tmark = 10000000.0;
            const St5 par1 = load_state(b.cur, c);
            const Ext8 e = load_ext(hcur, nc, c);
            if (!(cfl & CF_CENTR)) {
                const double dt = *b.dt_cur;
                const int g0 = d.gstart[c], g1 = d.gstart[c + 1];
                double Pt[kMhdFlux];
#pragma unroll
                for (int k = 0; k < kMhdFlux; k++) Pt[k] = 0.0;
                if (g1 - g0 == 4) {  // quadrilaterals: all slot loads in flight together
#pragma unroll
                    for (int k = 0; k < kMhdFlux; k++) {
                        const double* f = fl + k * ng + g0;
                        const double a0 = __ldcs(f), a1 = __ldcs(f + 1), a2 = __ldcs(f + 2), a3 = __ldcs(f + 3);
                        Pt[k] = (((Pt[k] + a0) + a1) + a2) + a3;
                    }
                } else {
                    for (int g = g0; g < g1; g++) {
#pragma unroll
                        for (int k = 0; k < kMhdFlux; k++) Pt[k] = Pt[k] + fl[k * ng + g];
                    }
                }
                const double q1 = src[c], q2 = src[nc + c], q3 = src[2 * nc + c];
                const double vs1 = b.vs[c], Volume = b.vol[c];
                const double gm1 = P.gamma - 1;
                const double rV2 = 1.0 / Volume2, VV = Volume * rV2;
                const double Am = 0.5 * (vs1 + vs2);
                const double i4p = 1.0 / (4.0 * kPi), i8p = 1.0 / (8.0 * kPi);
                // ions
                const double ro = par1.ro, p = par1.p, u = par1.u, v = par1.v, Q = par1.Q;
                const double w = e.f[kXw], bx = e.f[kXbx], by = e.f[kXby], bz = e.f[kXbz];
                const double bb = bx * bx + by * by + bz * bz;
                const double Sy = p + bb * i8p + ro * w * w - bz * bz * i4p;
                const double Sphi = -(ro * v * w - by * bz * i4p);
                const double Sbz = v * bz - w * by;
                double ro3 = ro * VV - dt * (Pt[0] * rV2);
                const double Q3 = Q * VV - (dt * rV2) * Pt[8];
                if (ro3 <= 0.0) {
                    ro3 = P.ro_floor;
                    nro++;
                }
                const double rro3 = 1.0 / ro3;
                const double u3 = (ro * u * VV - dt * (Pt[1] * rV2 - q1)) * rro3;
                const double v3 = (ro * v * VV - dt * ((Pt[2] - Sy * Am) * rV2 - q2)) * rro3;
                const double w3 = (ro * w * VV - dt * ((Pt[3] - Sphi * Am) * rV2)) * rro3;
                const double E = p / gm1 + ro * (u * u + v * v + w * w) * 0.5 + bb * i8p;
                const double E3 = E * VV - dt * (Pt[4] * rV2 - q3);
                const double bx3 = bx * VV - dt * (Pt[5] * rV2);
                const double by3 = by * VV - dt * (Pt[6] * rV2);
                const double bz3 = bz * VV - dt * ((Pt[7] - Sbz * Am) * rV2);
                double p3 = (E3 - 0.5 * ro3 * (u3 * u3 + v3 * v3 + w3 * w3) -
                             (bx3 * bx3 + by3 * by3 + bz3 * bz3) * i8p) *
                            gm1;
                if (p3 <= 0) {
                    p3 = P.p_floor;
                    npc++;
                }
                // pickup protons
                const double rp = e.f[kXro], pp = e.f[kXp], up = e.f[kXu], vp = e.f[kXv];
                double rp3 = rp * VV - dt * (Pt[9] * rV2);
                if (rp3 <= 0.0) {
                    rp3 = P.ro_floor;
                    nro++;
                }
                const double rrp3 = 1.0 / rp3;
                const double up3 = (rp * up * VV - dt * (Pt[10] * rV2)) * rrp3;
                const double vp3 = (rp * vp * VV - dt * ((Pt[11] - pp * Am) * rV2)) * rrp3;
                const double Ep = pp / gm1 + rp * (up * up + vp * vp) * 0.5;
                double pp3 = ((Ep * VV - dt * (Pt[12] * rV2)) - 0.5 * rp3 * (up3 * up3 + vp3 * vp3)) * gm1;
                if (pp3 <= 0) {
                    pp3 = P.p_floor;
                    npc++;
                }
                b.nxt[0][c] = ro3;
                b.nxt[1][c] = p3;
                b.nxt[2][c] = u3;
                b.nxt[3][c] = v3;
                b.nxt[4][c] = Q3;
                hnxt[kXw * nc + c] = w3;
                hnxt[kXbx * nc + c] = bx3;
                hnxt[kXby * nc + c] = by3;
                hnxt[kXbz * nc + c] = bz3;
                hnxt[kXro * nc + c] = rp3;
                hnxt[kXp * nc + c] = pp3;
                hnxt[kXu * nc + c] = up3;
                hnxt[kXv * nc + c] = vp3;
            } else {
                b.nxt[0][c] = par1.ro;
                b.nxt[1][c] = par1.p;
                b.nxt[2][c] = par1.u;
                b.nxt[3][c] = par1.v;
                b.nxt[4][c] = par1.Q;
#pragma unroll
                for (int k = 0; k < kMhdExtra; k++) hnxt[k * nc + c] = e.f[k];
            }
        }
    }
}

__global__ void __launch_bounds__(128) mhd_update_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                         const double* __restrict__ fl,
                                                         const double* __restrict__ src,
                                                         const double* __restrict__ hcur, double* __restrict__ hnxt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double tmark = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0;
    if (c < d.n_cells) mhd_update_body(d, P, b, fl, src, hcur, hnxt, c, tmark, nro, npc);
    block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
}

// ------------------------------------------------------------------ batched MHD step
// Many independent instances of the MHD + pickup step advance together: one
// launch per phase (surface tracking, rails, face units, cell update,
// commit) covers every instance.  A block finds its instance and first item
// in a static table (a block never straddles two instances, so the CFL
// block minimum goes to one instance's dt word) and copies the instance's
// descriptor into shared memory; the per-item work is the bodies of the
// one-instance kernels.
#ifndef GELIOS_BATCH_SMEM_DESC
#define GELIOS_BATCH_SMEM_DESC 0
#endif
#ifndef GELIOS_BATCH_FACE_MINB
#define GELIOS_BATCH_FACE_MINB 4
#endif
#if GELIOS_BATCH_SMEM_DESC
#define BATCH_INSTANCE(I, e)          \
    __shared__ BatchInstance I;       \
    load_instance(I, t.inst + (e).x);
#else
#define BATCH_INSTANCE(I, e) const BatchInstance& I = t.inst[(e).x];
#endif
__device__ __forceinline__ void load_instance(BatchInstance& dst, const BatchInstance* __restrict__ src) {
    static_assert(sizeof(BatchInstance) % 16 == 0, "instance descriptor is copied as int4");
    const int4* s4 = reinterpret_cast<const int4*>(src);
    int4* d4 = reinterpret_cast<int4*>(&dst);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(BatchInstance) / 16); i += blockDim.x) d4[i] = s4[i];
    __syncthreads();
}

__global__ void __launch_bounds__(64) batch_surface_kernel(BatchTables t, int parity) {
    const int2 e = t.surf[blockIdx.x];
    BATCH_INSTANCE(I, e)
    const int j = e.y + (threadIdx.x >> 5);
    if (j >= I.d.n_lc + I.d.n_li + I.d.n_lo) return;
    surface_face_body(I.d, I.P, I.b[parity], I.surface, j, threadIdx.x & 31);
}

__global__ void __launch_bounds__(128) batch_rails_kernel(BatchTables t, int parity) {
    const int2 e = t.rails[blockIdx.x];
    BATCH_INSTANCE(I, e)
    rails_body(I.d, I.P, I.b[parity].dt_cur, I.surface, true, e.y);
}

template <typename TF>
__global__ void __launch_bounds__(128, GELIOS_BATCH_FACE_MINB) batch_mhd_face_kernel(BatchTables t, int parity) {
    const int2 e = t.units[blockIdx.x];
    BATCH_INSTANCE(I, e)
    const int u = e.y + threadIdx.x;
    const StepBuffers& b = I.b[parity];
    double tmin = __longlong_as_double(0x7ff0000000000000LL);
    int status = 0;
    if (u < I.d.n_units) tmin = mhd_face_body<TF>(I.d, I.P, I.M, b, I.hs[parity], I.fl, u, status);
    block_reduce_commit(tmin, 0, 0, status, b.dt_acc, b.counters, b.status);
}

__global__ void __launch_bounds__(128) batch_mhd_update_kernel(BatchTables t, int parity) {
    const int2 e = t.cells[blockIdx.x];
    BATCH_INSTANCE(I, e)
    const int c = e.y + threadIdx.x;
    const StepBuffers& b = I.b[parity];
    double tmark = __longlong_as_double(0x7ff0000000000000LL);
    int nro = 0, npc = 0;
    if (c < I.d.n_cells) mhd_update_body(I.d, I.P, b, I.fl, I.src, I.hs[parity], I.hn[parity], c, tmark, nro, npc);
    block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
}

__global__ void __launch_bounds__(256) batch_commit_kernel(BatchTables t, int parity) {
    const int2 e = t.points[blockIdx.x];
    BATCH_INSTANCE(I, e)
    const StepBuffers& b = I.b[parity];
    if (e.y == 0 && threadIdx.x == 0) {
        const unsigned long long a = *b.dt_acc;
        *b.dt_next = (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
        *b.dt_acc = 0x7ff0000000000000ULL;
    }
    const int i = e.y + threadIdx.x;
    if (i < I.d.n_points) {
        I.d.X[i] = I.d.X2[i];
        I.d.Y[i] = I.d.Y2[i];
    }
}

// `nsteps` batched MHD + pickup steps of every instance in ONE cooperative
// launch: the five phases of launch_batch_mhd_step (tracked-face speeds,
// rails, face units, cell update, commit) with a grid barrier where a kernel
// boundary was.  The blocks deal each phase's table by grid stride (table
// entries are equal-sized tiles of one instance each, so every CFL block
// minimum still goes to one instance's dt word); the per-item work is the
// bodies of the per-phase kernels, so a call leaves the same state as the
// same number of per-phase steps.  The grid must be co-resident (launched
// by cudaLaunchCooperativeKernel, which refuses a grid that is not).
template <typename TF>
__global__ void __launch_bounds__(128, GELIOS_BATCH_FACE_MINB) batch_mhd_persistent_kernel(BatchTables t, int nsteps) {
    cg::grid_group grid = cg::this_grid();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int st = 0; st < nsteps; st++) {
        const int parity = st & 1;
        // tracked faces: a surf entry holds two faces (one warp each), so a
        // 128-thread block takes two entries per round
        for (int i = 2 * blockIdx.x + (warp >> 1); i < t.n_surf; i += 2 * gridDim.x) {
            const int2 e = t.surf[i];
            const BatchInstance& I = t.inst[e.x];
            const int j = e.y + (warp & 1);
            if (j < I.d.n_lc + I.d.n_li + I.d.n_lo) surface_face_body(I.d, I.P, I.b[parity], I.surface, j, lane);
        }
        grid.sync();
        for (int i = blockIdx.x; i < t.n_rails; i += gridDim.x) {
            const int2 e = t.rails[i];
            const BatchInstance& I = t.inst[e.x];
            rails_body(I.d, I.P, I.b[parity].dt_cur, I.surface, true, e.y);
            __syncthreads();  // the next rail reuses the block's shared words
        }
        grid.sync();
        for (int i = blockIdx.x; i < t.n_units; i += gridDim.x) {
            const int2 e = t.units[i];
            const BatchInstance& I = t.inst[e.x];
            const int u = e.y + threadIdx.x;
            const StepBuffers& b = I.b[parity];
            double tmin = __longlong_as_double(0x7ff0000000000000LL);
            int status = 0;
            if (u < I.d.n_units) tmin = mhd_face_body<TF>(I.d, I.P, I.M, b, I.hs[parity], I.fl, u, status);
            block_reduce_commit(tmin, 0, 0, status, b.dt_acc, b.counters, b.status);
            __syncthreads();  // the next tile reuses the reduction's shared words
        }
        grid.sync();
        for (int i = blockIdx.x; i < t.n_cells; i += gridDim.x) {
            const int2 e = t.cells[i];
            const BatchInstance& I = t.inst[e.x];
            const int c = e.y + threadIdx.x;
            const StepBuffers& b = I.b[parity];
            double tmark = __longlong_as_double(0x7ff0000000000000LL);
            int nro = 0, npc = 0;
            if (c < I.d.n_cells)
                mhd_update_body(I.d, I.P, b, I.fl, I.src, I.hs[parity], I.hn[parity], c, tmark, nro, npc);
            block_reduce_commit(tmark, nro, npc, 0, b.dt_acc, b.counters, b.status);
            __syncthreads();
        }
        grid.sync();
        // commit: a points entry covers 256 points (two per thread here)
        for (int i = blockIdx.x; i < t.n_points; i += gridDim.x) {
            const int2 e = t.points[i];
            const BatchInstance& I = t.inst[e.x];
            const StepBuffers& b = I.b[parity];
            if (e.y == 0 && threadIdx.x == 0) {
                const unsigned long long a = *b.dt_acc;
                *b.dt_next =
                    (a == 0x7ff0000000000000ULL) ? 100000000.0 : __longlong_as_double(static_cast<long long>(a));
                *b.dt_acc = 0x7ff0000000000000ULL;
            }
            for (int k = threadIdx.x; k < 256; k += blockDim.x) {
                const int p = e.y + k;
                if (p < I.d.n_points) {
                    I.d.X[p] = I.d.X2[p];
                    I.d.Y[p] = I.d.Y2[p];
                }
            }
        }
        grid.sync();
    }
}

// The dt / status words a call starts from: T[0] = T[1] = dt0, an empty CFL
// accumulator, zero clamp counters and status (layout: T[2], acc,
// counters[2], status).  A kernel rather than a copy from host memory: a
// copy from pageable memory would wait for the stream to drain.
__global__ void words_init_kernel(unsigned char* w, double dt0) {
    double* T = reinterpret_cast<double*>(w);
    unsigned long long* u = reinterpret_cast<unsigned long long*>(w + 16);
    T[0] = dt0;
    T[1] = dt0;
    u[0] = 0x7ff0000000000000ULL;
    u[1] = 0;
    u[2] = 0;
    *reinterpret_cast<int*>(w + 40) = 0;
}
__global__ void batch_words_init_kernel(BatchTables t, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BatchInstance& I = t.inst[i];
    double* T = const_cast<double*>(I.b[0].dt_cur);  // T[0]; b[1].dt_cur is T[1]
    T[0] = I.P.dt0;
    T[1] = I.P.dt0;
    *I.b[0].dt_acc = 0x7ff0000000000000ULL;
    I.b[0].counters[0] = 0;
    I.b[0].counters[1] = 0;
    *I.b[0].status = 0;
}

// ------------------------------------------------------------------ residual
// L1 change of one state row between the two buffers: per block the sums
// of |a - b| and |a| in a fixed order, then one block adds the partials in
// block order (deterministic, no atomics).
__global__ void __launch_bounds__(256) residual_partial_kernel(const double* __restrict__ a,
                                                               const double* __restrict__ b, int n,
                                                               double* __restrict__ part) {
    __shared__ double sd[256], sa[256];
    double dsum = 0.0, asum = 0.0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        dsum += fabs(a[i] - b[i]);
        asum += fabs(a[i]);
    }
    sd[threadIdx.x] = dsum;
    sa[threadIdx.x] = asum;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sd[threadIdx.x] += sd[threadIdx.x + o];
            sa[threadIdx.x] += sa[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sd[0];
        part[2 * blockIdx.x + 1] = sa[0];
    }
}
__global__ void residual_final_kernel(const double* __restrict__ part, int nb, double* __restrict__ out) {
    double d = 0.0, s = 0.0;
    for (int k = 0; k < nb; k++) {
        d += part[2 * k];
        s += part[2 * k + 1];
    }
    out[0] = d;
    out[1] = s;
}

// ------------------------------------------------------------------ launchers
namespace {
inline int blocks_for(int n, int t) { return (n + t - 1) / t; }
}

void launch_centroid(const DevMesh& d, const double* X, const double* Y, double* cx, double* cy, double* rp,
                     double gamma, cudaStream_t s, double* vs, double* vol) {
    if (d.n_cells > 0)
        centroid_kernel<<<blocks_for(d.n_cells, 256), 256, 0, s>>>(d, X, Y, cx, cy, rp, 2 * gamma, vs, vol);
}
void launch_stationary_units(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* fl,
                             cudaStream_t s) {
    if (P.precision == GELIOS_PREC_FP32_FLUX)
        stationary_unit_kernel<float><<<blocks_for(d.n_units, 128), 128, 0, s>>>(d, P, b, fl);
    else if (P.precision == GELIOS_PREC_FP32_WAVES)
        stationary_unit_kernel<WaveF32><<<blocks_for(d.n_units, 128), 128, 0, s>>>(d, P, b, fl);
    else
        stationary_unit_kernel<double><<<blocks_for(d.n_units, 128), 128, 0, s>>>(d, P, b, fl);
}
void launch_stationary_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                              cudaStream_t s) {
    stationary_update_kernel<<<blocks_for(d.n_cells, 128), 128, 0, s>>>(d, P, b, fl);
}
cudaError_t launch_stationary_persistent(const DevMesh& d, const gelios_params& P, const StepBuffers& b0,
                                         const StepBuffers& b1, double* fl, int nsteps, cudaStream_t s) {
    const void* fn = P.precision == GELIOS_PREC_FP32_FLUX
                         ? reinterpret_cast<const void*>(&stationary_persistent_kernel<float>)
                     : P.precision == GELIOS_PREC_FP32_WAVES
                         ? reinterpret_cast<const void*>(&stationary_persistent_kernel<WaveF32>)
                         : reinterpret_cast<const void*>(&stationary_persistent_kernel<double>);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int want = blocks_for(d.n_units > d.n_cells ? d.n_units : d.n_cells, 128);
    const int grid = want < per_sm * sms ? want : per_sm * sms;
    DevMesh dd = d;
    gelios_params pp = P;
    StepBuffers c0 = b0, c1 = b1;
    double* flp = fl;
    int n = nsteps;
    void* args[] = {&dd, &pp, &c0, &c1, &flp, &n};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(128), args, 0, s);
}
__global__ void unit_geometry_kernel(DevMesh d, double g2, const double* __restrict__ cx,
                                     const double* __restrict__ cy, double* __restrict__ upf) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= d.n_units) return;
    const int g = d.u_slot[u], K = d.u_cell[u];
    const int nb = d.u_twin[u] >= 0 ? d.snb[g] : -1;
    const int A = d.sA[g], B = d.sB[g];
    const FaceGeo f = face_geo(d.X[A], d.Y[A], d.X[B], d.Y[B], cx[K], cy[K], nb >= 0, nb >= 0 ? cx[nb] : 0.0,
                               nb >= 0 ? cy[nb] : 0.0);
    const size_t nu = d.n_units;
    upf[u] = pow2g(sqrt(f.f2), g2);
    double* geo = upf + nu;
    geo[u] = f.x2;
    geo[nu + u] = f.y2;
    geo[2 * nu + u] = f.n1;
    geo[3 * nu + u] = f.n2;
    geo[4 * nu + u] = f.f2;
    geo[5 * nu + u] = f.S;
    geo[6 * nu + u] = f.dist;
    geo[7 * nu + u] = f.distn;
}
void launch_unit_geometry(const DevMesh& d, double gamma, const double* cx, const double* cy, double* upf,
                          cudaStream_t s) {
    if (d.n_units > 0) unit_geometry_kernel<<<blocks_for(d.n_units, 128), 128, 0, s>>>(d, 2 * gamma, cx, cy, upf);
}
cudaError_t launch_stationary_batch(const DevMesh& d, const PlainInstance* inst, const int* active, int n_active,
                                    int nsteps, int prec, cudaStream_t s) {
    if (n_active <= 0 || nsteps <= 0) return cudaSuccess;
    const void* fn = prec == GELIOS_PREC_FP32_FLUX ? reinterpret_cast<const void*>(&stationary_batch_kernel<float>)
                     : prec == GELIOS_PREC_FP32_WAVES
                         ? reinterpret_cast<const void*>(&stationary_batch_kernel<WaveF32>)
                         : reinterpret_cast<const void*>(&stationary_batch_kernel<double>);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    const int64_t tiles = static_cast<int64_t>(n_active) * blocks_for(d.n_units > d.n_cells ? d.n_units : d.n_cells, 128);
    const int grid = tiles < static_cast<int64_t>(per_sm) * sms ? static_cast<int>(tiles) : per_sm * sms;
    DevMesh dd = d;
    const PlainInstance* ip = inst;
    const int* ap = active;
    int na = n_active, n = nsteps;
    void* args[] = {&dd, &ip, &ap, &na, &n};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(128), args, 0, s);
}
__global__ void plain_batch_words_init_kernel(const PlainInstance* inst, const int* active, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const PlainInstance& I = inst[active[k]];
    double* T = const_cast<double*>(I.b[0].dt_cur);  // T[0]; b[1].dt_cur is T[1]
    T[0] = I.P.dt0;
    T[1] = I.P.dt0;
    *I.b[0].dt_acc = 0x7ff0000000000000ULL;
    I.b[0].counters[0] = 0;
    I.b[0].counters[1] = 0;
    *I.b[0].status = 0;
}
void launch_plain_batch_words_init(const PlainInstance* inst, const int* active, int n, cudaStream_t s) {
    if (n > 0) plain_batch_words_init_kernel<<<blocks_for(n, 128), 128, 0, s>>>(inst, active, n);
}
void launch_mk2_recon(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* rec, cudaStream_t s) {
    const int nt = d.u_tr1 - d.u_tr0;
    if (nt > 0) mk2_recon_tracked_kernel<<<blocks_for(nt, 128), 128, 0, s>>>(d, P, b, rec);
}
// variant v of the tile kernel: threads per block x minimum resident blocks
// per SM (a register cap)
template <typename TF, int NT, int MINB>
static cudaError_t launch_tiles_v(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const TileView& t,
                                  const double* fl, const double* aux, cudaStream_t s) {
    const size_t smem = 5ull * static_cast<size_t>(t.max_slots) * sizeof(double);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(mk2_tile_kernel<TF, NT, MINB>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    mk2_tile_kernel<TF, NT, MINB><<<t.n_tiles, NT, smem, s>>>(d, P, b, t, fl, aux);
    return cudaGetLastError();
}
// Part 1 of a variant: the face units (none for the tile variants); part 2:
// the cell update (the whole tile kernel for the tile variants).  Part 1
// needs only the moved points; part 2 also the tracked-face fluxes and the
// source terms of the side stream.
template <typename TF, int MINB>
static void launch_faces_v(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* fl,
                           cudaStream_t s) {
    // the plain interior group in the variant's shape
    const int n0 = d.u_c1;
    if (n0 > 0) mk2_face_kernel<TF, MINB, kPlainGroup><<<blocks_for(n0, 128), 128, 0, s>>>(d, P, b, fl, n0);
}
// the plain interior group with the unit's gathers prefetched into L1
template <typename TF, int MINB>
static void launch_faces_pf(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* fl,
                            cudaStream_t s) {
    const int n0 = d.u_c1;
    if (n0 > 0) mk2_face_kernel<TF, MINB, kPlainGroup, true><<<blocks_for(n0, 128), 128, 0, s>>>(d, P, b, fl, n0);
}
// the C_1 interior and one-sided groups, each in an instance compiled for it
template <typename TF, bool PF>
static void launch_faces_rest(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* fl,
                              cudaStream_t s) {
    const int n1 = d.u_tr0 - d.u_c1, n3 = d.n_units - d.u_tr1;
    if (n1 > 0) mk2_face_kernel<TF, 6, kC1Group, PF><<<blocks_for(n1, 128), 128, 0, s>>>(d, P, b, fl, n1);
    if (n3 > 0) mk2_face_kernel<TF, 4, kAnyGroup, PF><<<blocks_for(n3, 128), 128, 0, s>>>(d, P, b, fl, n3);
}
template <typename TF>
static cudaError_t launch_cells_p(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const TileView& t,
                                  double* fl, const double* aux, cudaStream_t s, int variant, int part) {
    if (variant >= 4 && variant < 8) {
        if (part != 2) return cudaSuccess;
        switch (variant) {
            case 4: return launch_tiles_v<TF, 256, 3>(d, P, b, t, fl, aux, s);
            case 5: return launch_tiles_v<TF, 256, 2>(d, P, b, t, fl, aux, s);
            case 6: return launch_tiles_v<TF, 128, 5>(d, P, b, t, fl, aux, s);
            default: return launch_tiles_v<TF, 128, 4>(d, P, b, t, fl, aux, s);
        }
    }
    if (part == 2) {
        mk2_update_kernel<kUpdAll><<<blocks_for(d.n_cells, 128), 128, 0, s>>>(d, P, b, fl, aux, nullptr, 0);
        return cudaGetLastError();
    }
    if (part == 3) {
        if (variant >= 8)
            launch_faces_rest<TF, true>(d, P, b, fl, s);
        else
            launch_faces_rest<TF, false>(d, P, b, fl, s);
        return cudaGetLastError();
    }
    switch (variant) {
        case 1: launch_faces_v<TF, 5>(d, P, b, fl, s); break;
        case 2: launch_faces_v<TF, 6>(d, P, b, fl, s); break;
        case 3: launch_faces_v<TF, 4>(d, P, b, fl, s); break;
        case 8: launch_faces_pf<TF, 8>(d, P, b, fl, s); break;
        case 9: launch_faces_pf<TF, 6>(d, P, b, fl, s); break;
        case 10: launch_faces_pf<TF, 4>(d, P, b, fl, s); break;
        default: launch_faces_v<TF, 8>(d, P, b, fl, s); break;
    }
    return cudaGetLastError();
}
const char* mk2_variant_name(int v) {
    static const char* names[kMk2Variants] = {"faces 128x8 + update",         "faces 128x5 + update",
                                              "faces 128x6 + update",         "faces 128x4 + update",
                                              "tiles 256x3",                  "tiles 256x2",
                                              "tiles 128x5",                  "tiles 128x4",
                                              "faces prefetched 128x8 + update", "faces prefetched 128x6 + update",
                                              "faces prefetched 128x4 + update"};
    return (v >= 0 && v < kMk2Variants) ? names[v] : "?";
}
int mk2_variant_launches(const DevMesh& d, int v, int part) {
    const bool tiles = v >= 4 && v < 8;
    if (part == 2) return 1;
    if (tiles) return 0;
    if (part == 1) return d.u_c1 > 0 ? 1 : 0;
    return (d.u_tr0 > d.u_c1 ? 1 : 0) + (d.n_units > d.u_tr1 ? 1 : 0);
}
cudaError_t launch_mk2_cells(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const TileView& t,
                             double* fl, const double* aux, cudaStream_t s, int variant, int part) {
    if (P.precision == GELIOS_PREC_FP32_FLUX) return launch_cells_p<float>(d, P, b, t, fl, aux, s, variant, part);
    return launch_cells_p<double>(d, P, b, t, fl, aux, s, variant, part);
}
int launch_mk2_tracked_solve(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* rec,
                             double* pstar, cudaStream_t s) {
    const int nt = d.u_tr1 - d.u_tr0;
    if (nt <= 0) return 0;
    mk2_tracked_solve_kernel<<<blocks_for(nt, 2), 64, 0, s>>>(d, P, b, rec, pstar);
    return 1;
}
int launch_mk2_flux_tracked(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* rec,
                            const double* pstar, double* fl, cudaStream_t s) {
    const int nt = d.u_tr1 - d.u_tr0;
    if (nt <= 0) return 0;
    if (P.precision == GELIOS_PREC_FP32_FLUX)
        mk2_flux_tracked_kernel<float><<<blocks_for(nt, 32), 32, 0, s>>>(d, P, b, rec, fl, pstar);
    else
        mk2_flux_tracked_kernel<double><<<blocks_for(nt, 32), 32, 0, s>>>(d, P, b, rec, fl, pstar);
    return 1;
}
void launch_mk2_source(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* aux, cudaStream_t s) {
#if GELIOS_SOURCE_WARP
    mk2_source_kernel<<<blocks_for(d.n_cells, 128), 128, 0, s>>>(d, P, b, aux);
#else
    mk2_source_kernel<<<blocks_for(4 * d.n_cells, 128), 128, 0, s>>>(d, P, b, aux);
#endif
}
void launch_inner(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const int32_t* list, int n,
                  cudaStream_t s) {
    const int nb = blocks_for(n > 0 ? n : 1, 128);
    if (P.precision == GELIOS_PREC_FP32_FLUX)
        inner_cell_kernel<float><<<nb, 128, 0, s>>>(d, P, b, list, n);
    else
        inner_cell_kernel<double><<<nb, 128, 0, s>>>(d, P, b, list, n);
}
void launch_dt_finalize(const StepBuffers& b, cudaStream_t s) { dt_finalize_kernel<<<1, 1, 0, s>>>(b); }
void launch_commit(const DevMesh& d, const StepBuffers& b, cudaStream_t s, bool cap) {
    if (cap)
        commit_kernel<true><<<blocks_for(d.n_points > 0 ? d.n_points : 1, 256), 256, 0, s>>>(d, b);
    else
        commit_kernel<false><<<blocks_for(d.n_points > 0 ? d.n_points : 1, 256), 256, 0, s>>>(d, b);
}
void launch_dt_finalize_cap(const StepBuffers& b, cudaStream_t s) { dt_finalize_cap_kernel<<<1, 1, 0, s>>>(b); }
void launch_mk2_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       const double* aux, cudaStream_t s, int mode, const int32_t* list, int n_list) {
    if (mode == kUpdEarly) {
        if (n_list > 0)
            mk2_update_kernel<kUpdEarly><<<blocks_for(n_list, 128), 128, 0, s>>>(d, P, b, fl, aux, list, n_list);
        return;
    }
    const int nb = blocks_for(d.n_cells, 128);
    if (mode == kUpdRest)
        mk2_update_kernel<kUpdRest><<<nb, 128, 0, s>>>(d, P, b, fl, aux, list, n_list);
    else if (mode == kUpdAllNoMark)
        mk2_update_kernel<kUpdAllNoMark><<<nb, 128, 0, s>>>(d, P, b, fl, aux, list, n_list);
    else
        mk2_update_kernel<kUpdAll><<<nb, 128, 0, s>>>(d, P, b, fl, aux, list, n_list);
}
int launch_motion(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* scratch, cudaStream_t s,
                  bool copy_outer_shock) {
    int launches = 0;
    const int nf = d.n_lc + d.n_li + d.n_lo;
    if (nf > 0) {
        surface_faces_kernel<<<blocks_for(nf, 2), 64, 0, s>>>(d, P, b, scratch);
        launches += 1;
    }
    const int nr = d.n_rail_a + d.n_rail_b + d.n_rail_c + d.n_rail_d;
    if (nr > 0) {
        rails_kernel<<<nr, 128, 0, s>>>(d, P, b.dt_cur, scratch, copy_outer_shock);
        launches++;
    }
    return launches;
}
void launch_hllc_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s) {
    hllc_batch_kernel<<<blocks_for(n, 128), 128, 0, s>>>(P, n, in, out);
}
void launch_k5(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* hcur, double* hnxt,
               double* fl, cudaStream_t s) {
    if (d.n_units > 0) k5_face_kernel<<<blocks_for(d.n_units, 128), 128, 0, s>>>(d, P, b, hcur, fl);
    k5_update_kernel<<<blocks_for(d.n_cells, 128), 128, 0, s>>>(d, P, b, fl, hcur, hnxt);
}
void launch_hlldq_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s) {
    hlldq_batch_kernel<<<blocks_for(n, 128), 128, 0, s>>>(P, n, in, out);
}
void launch_hlld_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s) {
    hlld_batch_kernel<<<blocks_for(n, 128), 128, 0, s>>>(P, n, in, out);
}
void launch_godunov_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s) {
    godunov_batch_kernel<<<blocks_for(n, 2), 64, 0, s>>>(P, n, in, out);
}
namespace {
// The plain interior group in the variant's shape on stream s, the other
// groups (a few percent of the units, every branch) in one fixed shape on
// stream sr (s itself, or a stream the caller forks and joins).
template <int BLOCK, int MINB>
void mhd_faces_shape(const DevMesh& d, const gelios_params& P, const gelios_mhd_params& M, const StepBuffers& b,
                     const double* hcur, double* fl, cudaStream_t s, cudaStream_t sr) {
    const int n0 = d.u_c1, nr = d.n_units - d.u_c1;
    const bool f32 = P.precision == GELIOS_PREC_FP32_FLUX;
    if (n0 > 0) {
        if (f32)
            mhd_face_kernel<float, BLOCK, MINB, true><<<blocks_for(n0, BLOCK), BLOCK, 0, s>>>(d, P, M, b, hcur, fl);
        else
            mhd_face_kernel<double, BLOCK, MINB, true><<<blocks_for(n0, BLOCK), BLOCK, 0, s>>>(d, P, M, b, hcur, fl);
    }
    if (nr > 0) {
        if (f32)
            mhd_face_kernel<float, 128, 3, false><<<blocks_for(nr, 128), 128, 0, sr>>>(d, P, M, b, hcur, fl);
        else
            mhd_face_kernel<double, 128, 3, false><<<blocks_for(nr, 128), 128, 0, sr>>>(d, P, M, b, hcur, fl);
    }
}
}  // namespace

const char* mhd_face_variant_name(int v) {
    static const char* names[kMhdFaceVariants] = {"128x3", "128x1", "128x4", "64x6", "64x3", "256x1"};
    return (v >= 0 && v < kMhdFaceVariants) ? names[v] : "?";
}
int launch_mhd_faces(const DevMesh& d, const gelios_params& P, const gelios_mhd_params& M, const StepBuffers& b,
                     const double* hcur, double* fl, cudaStream_t s, int variant, cudaStream_t s_rest) {
    if (d.n_units <= 0) return 0;
    cudaStream_t sr = s_rest ? s_rest : s;
    switch (variant) {
        case 1: mhd_faces_shape<128, 1>(d, P, M, b, hcur, fl, s, sr); break;
        case 2: mhd_faces_shape<128, 4>(d, P, M, b, hcur, fl, s, sr); break;
        case 3: mhd_faces_shape<64, 6>(d, P, M, b, hcur, fl, s, sr); break;
        case 4: mhd_faces_shape<64, 3>(d, P, M, b, hcur, fl, s, sr); break;
        case 5: mhd_faces_shape<256, 1>(d, P, M, b, hcur, fl, s, sr); break;
        default: mhd_faces_shape<128, 3>(d, P, M, b, hcur, fl, s, sr); break;
    }
    return (d.u_c1 > 0 ? 1 : 0) + (d.n_units > d.u_c1 ? 1 : 0);
}
// Frozen-grid residual of the moving-grid operator, per block: over the
// cells that take part in a step (centroid radius >= R11, not C_centr) the
// sum of |sum of the mass fluxes F.S of the cell's face slots| / rotated
// volume (the density change per unit time the step's flux balance gives
// with the grid held still: d(rho V)/dt = -sum F.S, Setka.cpp:10425-10431),
// and the sum of |rho| over every cell.  Fixed-order tree sums.
__global__ void __launch_bounds__(256) op_residual_partial_kernel(DevMesh d, gelios_params P, StepBuffers b,
                                                                  const double* __restrict__ fl,
                                                                  double* __restrict__ part) {
    __shared__ double sd[256], sa[256];
    double dsum = 0.0, asum = 0.0;
    for (int c = blockIdx.x * 256 + threadIdx.x; c < d.n_cells; c += gridDim.x * 256) {
        asum += fabs(b.cur[0][c]);
        const double x = b.cx[c], y = b.cy[c];
        if (sqrt(sq(x) + sq(y)) < P.R11 || (d.cflags[c] & CF_CENTR)) continue;
        double pt = 0.0;
        for (int g = d.gstart[c]; g < d.gstart[c + 1]; g++) pt = pt + fl[g];
        dsum += fabs(pt) / b.vol[c];
    }
    sd[threadIdx.x] = dsum;
    sa[threadIdx.x] = asum;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sd[threadIdx.x] += sd[threadIdx.x + o];
            sa[threadIdx.x] += sa[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sd[0];
        part[2 * blockIdx.x + 1] = sa[0];
    }
}
int launch_op_residual(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       double* scratch, cudaStream_t s) {
    const int n = d.n_cells;
    const int nb = n > 0 ? (blocks_for(n, 256) < 296 ? blocks_for(n, 256) : 296) : 1;
    op_residual_partial_kernel<<<nb, 256, 0, s>>>(d, P, b, fl, scratch + 2);
    residual_final_kernel<<<1, 1, 0, s>>>(scratch + 2, nb, scratch);
    return 2;
}
int launch_residual(const double* a, const double* b, int n, double* scratch, cudaStream_t s) {
    const int nb = n > 0 ? (blocks_for(n, 256) < 296 ? blocks_for(n, 256) : 296) : 1;
    residual_partial_kernel<<<nb, 256, 0, s>>>(a, b, n, scratch + 2);
    residual_final_kernel<<<1, 1, 0, s>>>(scratch + 2, nb, scratch);
    return 2;
}
void launch_words_init(void* words, double dt0, cudaStream_t s) {
    words_init_kernel<<<1, 1, 0, s>>>(static_cast<unsigned char*>(words), dt0);
}
void launch_batch_words_init(const BatchTables& t, int n, cudaStream_t s) {
    if (n > 0) batch_words_init_kernel<<<blocks_for(n, 128), 128, 0, s>>>(t, n);
}
void launch_batch_mhd_step(const BatchTables& t, int parity, cudaStream_t s) {
    if (t.n_surf > 0) batch_surface_kernel<<<t.n_surf, 64, 0, s>>>(t, parity);
    if (t.n_rails > 0) batch_rails_kernel<<<t.n_rails, 128, 0, s>>>(t, parity);
    if (t.n_units > 0) {
        if (t.fp32)
            batch_mhd_face_kernel<float><<<t.n_units, 128, 0, s>>>(t, parity);
        else
            batch_mhd_face_kernel<double><<<t.n_units, 128, 0, s>>>(t, parity);
    }
    if (t.n_cells > 0) batch_mhd_update_kernel<<<t.n_cells, 128, 0, s>>>(t, parity);
    if (t.n_points > 0) batch_commit_kernel<<<t.n_points, 256, 0, s>>>(t, parity);
}
cudaError_t launch_batch_mhd_persistent(const BatchTables& t, int nsteps, int blocks_per_sm, cudaStream_t s,
                                        int* max_per_sm) {
    const void* fn = t.fp32 ? reinterpret_cast<const void*>(&batch_mhd_persistent_kernel<float>)
                            : reinterpret_cast<const void*>(&batch_mhd_persistent_kernel<double>);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
    if (e != cudaSuccess) return e;
    if (max_per_sm) *max_per_sm = per_sm;
    if (per_sm < 1 || blocks_per_sm > per_sm) return cudaErrorCooperativeLaunchTooLarge;
    if (nsteps <= 0) return cudaSuccess;
    const int k = blocks_per_sm > 0 ? blocks_per_sm : per_sm;
    BatchTables tt = t;
    int n = nsteps;
    void* args[] = {&tt, &n};
    return cudaLaunchCooperativeKernel(fn, dim3(k * sms), dim3(128), args, 0, s);
}
void launch_mhd_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       const double* src, const double* hcur, double* hnxt, cudaStream_t s) {
    mhd_update_kernel<<<blocks_for(d.n_cells, 128), 128, 0, s>>>(d, P, b, fl, src, hcur, hnxt);
}

}  // namespace gelios
