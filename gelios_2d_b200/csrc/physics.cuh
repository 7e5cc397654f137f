// Device physics of the Gelios_2D plasma step (sm_100a).
//
// Each function names the reference code it computes.  Formulas keep the
// reference's operation order where that costs nothing; where a cheaper
// equivalent exists it is used and its deviation is stated (all deviations
// are at the level of a few ulp of FP64 and are covered by the parity
// tolerance of the tests: 1e-12 relative per step).
#pragma once

#include <cstdint>

#include "../../include/gelios_b200.h"

namespace gelios {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTinyAngle = 0.000001 / 390.222;  // polar_angle threshold, Help.cpp:39

// Gran_type / Cell_type / Point_type values of the reference.
enum : int { G_USUALY = 0, G_INNER_SPHERE = 1, G_EXTERN = 2, G_INPUT = 3, G_AXIS = 4, G_UPPER_WALL = 5 };
enum : int { C_1 = 0, C_CENTR = 5 };
enum : int { P_CONTACT = 6, P_INNER_SHOCK = 7, P_OUTER_SHOCK = 8 };

// Slot (cell face) info bits.
enum : uint32_t {
    SI_TYPE_MASK = 7u,
    SI_GOD = 1u << 3,     // both end points on the same tracked surface (Setka.cpp:10287-10298)
    SI_NP = 1u << 4,      // exactly one end point on a tracked surface (Setka.cpp:10301-10324)
};
// Cell flag bits.
enum : uint32_t { CF_AXIS = 1u, CF_C1 = 2u, CF_CENTR = 4u };
// Status flag bits (gelios_status::flags).
enum : int { ST_ITER_CAP = 1, ST_TVD_BAD = 2, ST_NEWTON_NEG = 4, ST_CHAIN = 8, ST_DT_BAD = 16 };

struct St5 {
    double ro, p, u, v, Q;
};

__device__ __forceinline__ double dmin_ref(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax_ref(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ float fmin_ref(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fmax_ref(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ double sq(double x) { return x * x; }

// sign / minmod / linear: Help.cpp:67-120
__device__ __forceinline__ double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }
__device__ __forceinline__ double minmod(double x, double y) {
    const double s = sgn(x) + sgn(y);
    if (s == 0) return 0.0;
    return (s / 2.0) * dmin_ref(fabs(x), fabs(y));
}
__device__ __forceinline__ double linear3(double x1, double t1, double x2, double t2, double x3, double t3, double y) {
    const double d = minmod((t1 - t2) / (x1 - x2), (t2 - t3) / (x2 - x3));
    return (d * (y - x2) + t2);
}
// linear(x1,t1,x2,t2,x3,t3,0) with the reciprocals r12 = 1/(x1-x2) and
// r23 = 1/(x2-x3) computed once for all fields reconstructed at a face
// (products by a reciprocal instead of quotients: <= 1 ulp per slope).
__device__ __forceinline__ double linear3r(double t1, double t2, double t3, double r12, double r23, double x2) {
    const double d = minmod((t1 - t2) * r12, (t2 - t3) * r23);
    return d * (0.0 - x2) + t2;
}
__device__ __forceinline__ double linear2(double x1, double t1, double x2, double t2, double y) {
    const double d = (t1 - t2) / (x1 - x2);
    return (d * (y - x2) + t2);
}

// cos/sin of polar_angle(x, y) (Help.cpp:37-65).  The reference takes atan of
// y/x and then cos/sin of the angle; the unit vector (x, y)/r is the same
// quantity without the three transcendental calls (differences ~1 ulp).
__device__ __forceinline__ void polar_cs(double x, double y, double& c, double& s) {
    if (fabs(x) + fabs(y) < kTinyAngle) {
        c = 1.0;
        s = 0.0;
        return;
    }
    const double rinv = rsqrt(x * x + y * y);
    c = x * rinv;
    s = y * rinv;
}
// polar_perenos, Help.cpp:3-14: re-express a velocity given in the polar
// frame of point 1 in the polar frame of point 2.
__device__ __forceinline__ void polar_perenos(double x1, double y1, double x2, double y2, double& u, double& v) {
    double c1, s1, c2, s2;
    polar_cs(x1, y1, c1, s1);
    polar_cs(x2, y2, c2, s2);
    const double fr = u * c1 + v * s1;
    const double ff = -u * s1 + v * c1;
    u = fr * c2 - ff * s2;
    v = fr * s2 + ff * c2;
}

// a^(2*gamma): pow(a, 2*ggg) in the reference.
__device__ __forceinline__ double pow2g(double a, double g2) { return pow(a, g2); }

// ---------------------------------------------------------------- HLLC / HLL
// Setka::HLLC_2d_Korolkov_b_s, Setka.cpp:10484-10700.  metod == 0 -> HLL
// (10604-10618); otherwise HLLC with the optional tangential smoothing
// `nul_potok` (10644-10653).  Returns UU = max(|SL|,|SR|); the reference's
// CFL candidate is kurant*rad/UU (computed by the caller for each side).
// T is the arithmetic type of the solver (double: drop-in; float: the
// FP32-flux form, whose inputs/outputs stay double).
template <typename T>
struct FluxOut {
    T P0, P1, P2, P3, PQ;
};

template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T tsqrt(T a);
template <>
__device__ __forceinline__ double tsqrt<double>(double a) { return sqrt(a); }
template <>
__device__ __forceinline__ float tsqrt<float>(float a) { return sqrtf(a); }

template <typename T>
__device__ __forceinline__ double hllc_flux(double gamma, double kurant, const St5& L, const St5& R, double Wd,
                                            double n1d, double n2d, double rad, int metod, bool nul_potok,
                                            FluxOut<double>& out) {
    const T ggg = (T)gamma, g1 = (T)(gamma - 1.0);
    const T n1 = (T)n1d, n2 = (T)n2d, W = (T)Wd;
    const T ro_L = (T)L.ro, Q_L = (T)L.Q, p_L = (T)L.p, v1_L = (T)L.u, v2_L = (T)L.v;
    const T ro_R = (T)R.ro, Q_R = (T)R.Q, p_R = (T)R.p, v1_R = (T)R.u, v2_R = (T)R.v;
    const T t1 = n2, t2 = -n1;
    const T u1 = v1_L * n1 + v2_L * n2;
    const T v1 = v1_L * t1 + v2_L * t2;
    const T u2 = v1_R * n1 + v2_R * n2;
    const T v2 = v1_R * t1 + v2_R * t2;
    const T cL = tsqrt<T>(ggg * p_L / ro_L);
    const T cR = tsqrt<T>(ggg * p_R / ro_R);
    const T uu_L = (v1_L * v1_L + v2_L * v2_L) / (T)2;
    const T uu_R = (v1_R * v1_R + v2_R * v2_R) / (T)2;
    const T SL = tmin<T>(u1, u2) - tmax<T>(cL, cR);
    const T SR = tmax<T>(u1, u2) + tmax<T>(cL, cR);
    const T suR = (SR - u2);
    const T suL = (SL - u1);
    const T SM = (suR * ro_R * u2 - suL * ro_L * u1 - p_R + p_L) / (suR * ro_R - suL * ro_L);
    // wave-speed bound of the CFL candidate, FP64 (the reduction stays FP64)
    const double time = dmax_ref(fabs((double)SL), fabs((double)SR));
    (void)kurant;
    (void)rad;
    const T rg1 = (T)1 / g1;
    const T e1 = p_L * rg1 + ro_L * uu_L;
    const T e2 = p_R * rg1 + ro_R * uu_R;
    const T FL0 = ro_L * u1, FL1 = ro_L * u1 * u1 + p_L, FL2 = ro_L * u1 * v1, FL3 = (e1 + p_L) * u1, FL4 = Q_L * u1;
    const T FR0 = ro_R * u2, FR1 = ro_R * u2 * u2 + p_R, FR2 = ro_R * u2 * v2, FR3 = (e2 + p_R) * u2, FR4 = Q_R * u2;
    const T UL0 = ro_L, UL1 = ro_L * u1, UL2 = ro_L * v1, UL3 = e1, UL4 = Q_L;
    const T UR0 = ro_R, UR1 = ro_R * u2, UR2 = ro_R * v2, UR3 = e2, UR4 = Q_R;
    if (SL >= W) {
        out.P1 = n1 * (FL1 - W * UL1) + t1 * (FL2 - W * UL2);
        out.P2 = n2 * (FL1 - W * UL1) + t2 * (FL2 - W * UL2);
        out.P0 = FL0 - W * UL0;
        out.P3 = FL3 - W * UL3;
        out.PQ = FL4 - W * UL4;
        return time;
    }
    if (SR <= W) {
        out.P1 = n1 * (FR1 - W * UR1) + t1 * (FR2 - W * UR2);
        out.P2 = n2 * (FR1 - W * UR1) + t2 * (FR2 - W * UR2);
        out.P0 = FR0 - W * UR0;
        out.P3 = FR3 - W * UR3;
        out.PQ = FR4 - W * UR4;
        return time;
    }
    const T rRL = (T)1 / (SR - SL);
    const T UZ0 = (SR * UR0 - SL * UL0 + FL0 - FR0) * rRL;
    const T UZ1 = (SR * UR1 - SL * UL1 + FL1 - FR1) * rRL;
    const T UZ2 = (SR * UR2 - SL * UL2 + FL2 - FR2) * rRL;
    const T UZ3 = (SR * UR3 - SL * UL3 + FL3 - FR3) * rRL;
    const T UZ4 = (SR * UR4 - SL * UL4 + FL4 - FR4) * rRL;
    if (metod == 0) {
        const T SRSL = SR * SL;
        const T PO0 = (SR * FL0 - SL * FR0 + SRSL * (UR0 - UL0)) * rRL;
        const T PO1 = (SR * FL1 - SL * FR1 + SRSL * (UR1 - UL1)) * rRL;
        const T PO2 = (SR * FL2 - SL * FR2 + SRSL * (UR2 - UL2)) * rRL;
        const T PO3 = (SR * FL3 - SL * FR3 + SRSL * (UR3 - UL3)) * rRL;
        const T PO4 = (SR * FL4 - SL * FR4 + SRSL * (UR4 - UL4)) * rRL;
        out.P1 = n1 * (PO1 - W * UZ1) + t1 * (PO2 - W * UZ2);
        out.P2 = n2 * (PO1 - W * UZ1) + t2 * (PO2 - W * UZ2);
        out.P0 = PO0 - W * UZ0;
        out.P3 = PO3 - W * UZ3;
        out.PQ = PO4 - W * UZ4;
        return time;
    }
    const T rLM = (T)1 / (SL - SM), rRM = (T)1 / (SR - SM);
    const T suRm = suR * rRM;
    const T suLm = suL * rLM;
    const T ro_LL = ro_L * suLm;
    const T ro_RR = ro_R * suRm;
    const T Q_LL = Q_L * suLm;
    const T Q_RR = Q_R * suRm;
    const T ptzR = p_R + ro_R * suR * (SM - u2);
    const T ptzL = p_L + ro_L * suL * (SM - u1);
    const T ptz = (ptzR + ptzL) / (T)2;
    T vLL, vRR;
    if (nul_potok) {
        vRR = UZ2 / UZ0;
        vLL = vRR;
    } else {
        vLL = v1;
        vRR = v2;
    }
    const T ee2 = e2 * suRm + (ptz * SM - p_R * u2) * rRM;
    const T ee1 = e1 * suLm + (ptz * SM - p_L * u1) * rLM;
    T PO0 = 0, PO1 = 0, PO2 = 0, PO3 = 0, PO4 = 0;
    if (SL < W && SM >= W) {
        PO0 = FL0 + SL * ro_LL - SL * UL0 - W * ro_LL;
        PO1 = FL1 + SL * (ro_LL * SM) - SL * UL1 - W * (ro_LL * SM);
        PO2 = FL2 + SL * (ro_LL * vLL) - SL * UL2 - W * (ro_LL * vLL);
        PO3 = FL3 + SL * ee1 - SL * UL3 - W * ee1;
        PO4 = FL4 + SL * Q_LL - SL * UL4 - W * Q_LL;
    } else if (SR > W && SM < W) {
        PO0 = FR0 + SR * ro_RR - SR * UR0 - W * ro_RR;
        PO1 = FR1 + SR * (ro_RR * SM) - SR * UR1 - W * (ro_RR * SM);
        PO2 = FR2 + SR * (ro_RR * vRR) - SR * UR2 - W * (ro_RR * vRR);
        PO3 = FR3 + SR * ee2 - SR * UR3 - W * ee2;
        PO4 = FR4 + SR * Q_RR - SR * UR4 - W * Q_RR;
    }
    out.P1 = n1 * PO1 + t1 * PO2;
    out.P2 = n2 * PO1 + t2 * PO2;
    out.P0 = PO0;
    out.P3 = PO3;
    out.PQ = PO4;
    return time;
}

// ---------------------------------------------------------------- exact Godunov
// Solvers::lev, Solvers.cpp:1307-1321
__device__ __forceinline__ double lev_dev(double ga, double enI, double pI, double rI, double enII, double pII,
                                          double rII, double uuu) {
    const double g1 = ga - 1.0, g2 = ga + 1.0, gp = (g2 / ga) / 2.0, gm = (g1 / ga) / 2.0;
    const double cI = sqrt(ga * pI / rI);
    const double cII = sqrt(ga * pII / rII);
    const double fI = (uuu - pI) / (rI * cI * sqrt(gp * uuu / pI + gm));
    const double fII = 2.0 / g1 * cII * (pow((uuu / pII), gm) - 1.0);
    return (fI + fII) - (enI - enII);
}

// Solvers::devtwo (Solvers.cpp:1231-1305): bisection for the star pressure
// between pI and pII, stopping where |lev| <= 1e-9 (cap max_iter).
//
// COOP = true: the 32 lanes of a warp call it with identical arguments and
// walk the same bisection together.  Each round, lanes 0..30 evaluate lev at
// the 31 midpoints of the next five bisection levels (lane j = node j+1 of a
// heap-ordered binary tree, its interval derived from the round's interval by
// the same halvings the sequential loop performs), then every lane replays
// the five sequential decisions on the broadcast values.  The midpoints, the
// function values and the decisions are the ones of the sequential loop, so
// the result and the iteration count are the same; the latency is one lev
// evaluation per five iterations instead of five.
template <bool COOP>
__device__ __forceinline__ double godunov_devtwo(double ga, double enI, double pI, double rI, double enII, double pII,
                                                 double rII, int max_iter, int* status) {
    const double epsil = 10e-10;
    double kl = pI, kp = pII;
    double ksi = lev_dev(ga, enI, pI, rI, enII, pII, rII, kl);
    const double ksir0 = lev_dev(ga, enI, pI, rI, enII, pII, rII, kp);
    if (fabs(ksi) <= epsil) return kl;
    if (fabs(ksir0) <= epsil) return kp;
    int k = 0;
    if (!COOP) {
        for (;;) {
            k = k + 1;
            if (k >= max_iter) {
                *status |= ST_ITER_CAP;
                return (kl + kp) / 2.0;
            }
            const double kc = (kl + kp) / 2.0;
            const double ksit = lev_dev(ga, enI, pI, rI, enII, pII, rII, kc);
            if (fabs(ksit) <= epsil) return kc;
            if ((ksi * ksit) <= 0.0) {
                kp = kc;
            } else {
                kl = kc;
                ksi = ksit;
            }
        }
    }
    const int node = (threadIdx.x & 31) + 1;  // 1..32; node 32 (level 5) evaluates nothing
    const int L = 31 - __clz(node);
    const int idx = node - (1 << L);
    for (;;) {
        double a = kl, b = kp;
        for (int l = 0; l < L; l++) {
            const double c = (a + b) / 2.0;
            if ((idx >> (L - 1 - l)) & 1) a = c;
            else b = c;
        }
        double f = 0.0;
        if (L < 5) f = lev_dev(ga, enI, pI, rI, enII, pII, rII, (a + b) / 2.0);
        int nd = 1;
        for (int l = 0; l < 5; l++) {
            k = k + 1;
            if (k >= max_iter) {
                *status |= ST_ITER_CAP;
                return (kl + kp) / 2.0;
            }
            const double kc = (kl + kp) / 2.0;
            const double ksit = __shfl_sync(0xffffffffu, f, nd - 1);
            if (fabs(ksit) <= epsil) return kc;
            if ((ksi * ksit) <= 0.0) {
                kp = kc;
                nd = 2 * nd;
            } else {
                kl = kc;
                ksi = ksit;
                nd = 2 * nd + 1;
            }
        }
    }
}

// Solvers::newton (Solvers.cpp:1174-1229): Newton iteration for the star
// pressure of two shocks (cap max_iter; a non-positive iterate is returned
// as is, like the reference, and raises ST_NEWTON_NEG).
__device__ __forceinline__ double godunov_newton(double ga, double enI, double pI, double rI, double enII,
                                                 double pII, double rII, int max_iter, int* status) {
    const double gm = ((ga - 1.0) / ga) / 2.0, gp = ((ga + 1.0) / ga) / 2.0;
    const double eps = 10e-10;
    const double cIn = sqrt(ga * pI / rI);
    const double cIIn = sqrt(ga * pII / rII);
    double pn = pI * rII * cIIn + pII * rI * cIn + (enI - enII) * rI * cIn * rII * cIIn;
    pn = pn / (rI * cIn + rII * cIIn);
    const double pee = pn;
    int kiter = 0;
    for (;;) {
        const double pp = pn;
        if (pp <= 0.0) {
            *status |= ST_NEWTON_NEG;
            return pp;
        }
        kiter = kiter + 1;
        // pow(z, 3/2) of the reference as z*sqrt(z)
        const double zI = gp * pp / pI + gm, zII = gp * pp / pII + gm;
        const double sI = sqrt(zI), sII = sqrt(zII);
        const double fI = (pp - pI) / (rI * cIn * sI);
        double fIs = (ga + 1.0) * pp / pI + (3.0 * ga - 1.0);
        fIs = fIs / (4.0 * ga * rI * cIn * (zI * sI));
        const double fII = (pp - pII) / (rII * cIIn * sII);
        double fIIs = (ga + 1.0) * pp / pII + (3.0 * ga - 1.0);
        fIIs = fIIs / (4.0 * ga * rII * cIIn * (zII * sII));
        if (kiter >= max_iter) {
            *status |= ST_ITER_CAP;
            return pp;
        }
        pn = pp - (fI + fII - (enI - enII)) / (fIs + fIIs);
        if (!(fabs(pn / pee - pp / pee) >= eps)) return pn;
    }
}

// Solvers::Godunov_Solver_Alexashov with newton/devtwo, Solvers.cpp:693-1305.
// q = (ro, p, u, v, w); qqq[5] flux; ds[3] = dsl, dsp, dsc.  Returns the
// wave-speed bound UU of the reference's CFL candidate kurant*DIST/UU (UU is
// replaced by eps8 when it is not above it, Solvers.cpp:841-848).
// The Newton and bisection loops are capped at max_iter (the reference
// exits the program at 1100); hitting the cap raises ST_ITER_CAP.
//
// The star pressure of the two iterative branches does not depend on the
// face speed w: p_out (if given) receives the pressure after the branch
// selection, and p_in (if given) replaces the iteration by that value, so a
// caller can solve before the grid moves and sample after it.  COOP selects
// the warp-cooperative bisection (all 32 lanes, identical arguments).
template <bool COOP>
static __device__ __noinline__ double godunov_dev(double ga, double kurant, const double* qqq1, const double* qqq2,
                                           const double* n, double* qqq, double* ds, double w, double DIST,
                                           int max_iter, int* status, const double* p_in = nullptr,
                                           double* p_out = nullptr) {
    const double g1 = ga - 1.0, g2 = ga + 1.0, gm = (g1 / ga) / 2.0, gp = (g2 / ga) / 2.0;
    const double eps = 10e-10, eps8 = 10e-8;
    const double al = n[0], be = n[1], ge = n[2];
    double time = 0.0;
    const double al2 = be, be2 = -al, ge2 = 0.0;
    const double al3 = 0.0, be3 = 0.0, ge3 = 1.0;
    double enI = al * qqq1[2] + be * qqq1[3] + ge * qqq1[4];
    double teI2 = al2 * qqq1[2] + be2 * qqq1[3] + ge2 * qqq1[4];
    double teI3 = al3 * qqq1[2] + be3 * qqq1[3] + ge3 * qqq1[4];
    double enII = al * qqq2[2] + be * qqq2[3] + ge * qqq2[4];
    double teII2 = al2 * qqq2[2] + be2 * qqq2[3] + ge2 * qqq2[4];
    double teII3 = al3 * qqq2[2] + be3 * qqq2[3] + ge3 * qqq2[4];
    double pI = qqq1[1], pII = qqq2[1], rI = qqq1[0], rII = qqq2[0];
    int ipiz = 0;
    if (pI > pII) {
        const double eno2 = enII, teo22 = teII2, teo23 = teII3, p2 = pII, r2 = rII;
        const double eno1 = enI, teo12 = teI2, teo13 = teI3, p1 = pI, r1 = rI;
        enI = -eno2; teI2 = teo22; teI3 = teo23; pI = p2; rI = r2;
        enII = -eno1; teII2 = teo12; teII3 = teo13; pII = p1; rII = r1;
        w = -w;
        ipiz = 1;
    }
    double cI = 0.0, cII = 0.0;
    if (pI != 0.0) cI = sqrt(ga * pI / rI);
    if (pII != 0.0) cII = sqrt(ga * pII / rII);
    const double a = sqrt(rI * (g2 * pII + g1 * pI) / 2.0);
    const double Uud = (pII - pI) / a;
    const double Urz = -2.0 * cII / g1 * (1.0 - pow((pI / pII), gm));
    const double Uvk = -2.0 * (cII + cI) / g1;
    const double Udf = enI - enII;
    int il = -2, ip = -2;
    double p = 0.0, r = 0.0, te2 = 0.0, te3 = 0.0, en = 0.0;
    double dsl = 0.0, dsp = 0.0, dsc = 0.0;
    if (Udf < Uvk) {
        il = -1; ip = -1;
    } else if ((Udf >= Uvk) && (Udf <= Urz)) {
        p = pI * pow(((Udf - Uvk) / (Urz - Uvk)), (1.0 / gm));
        il = 0; ip = 0;
    } else if ((Udf > Urz) && (Udf <= Uud)) {  // devtwo
        p = p_in ? *p_in : godunov_devtwo<COOP>(ga, enI, pI, rI, enII, pII, rII, max_iter, status);
        il = 1; ip = 0;
    } else if (Udf > Uud) {  // newton
        p = p_in ? *p_in : godunov_newton(ga, enI, pI, rI, enII, pII, rII, max_iter, status);
        il = 1; ip = 1;
    }
    if (p_out) *p_out = p;
    if ((il == 1) && (ip == 1)) {  // two shocks
        const double aI = sqrt(rI * (g2 / 2.0 * p + g1 / 2.0 * pI));
        const double aII = sqrt(rII * (g2 / 2.0 * p + g1 / 2.0 * pII));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - aI / rI;
        const double dII = enII + aII / rII;
        dsl = dI; dsp = dII; dsc = u;
        const double UU = dmax_ref(fabs(dsl), fabs(dsp));
        time = (UU > eps8) ? UU : eps8;
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
    if ((il == 1) && (ip == 0)) {  // left shock, right expansion
        const double aI = sqrt(rI * (g2 / 2.0 * p + g1 / 2.0 * pI));
        double aII;
        if (fabs(p - pII) < eps) aII = rII * cII;
        else aII = gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), gm));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - aI / rI;
        const double dII = enII + cII;
        const double ddII = u + cII - g1 * (enII - u) / 2.0;
        dsl = dI; dsp = dII; dsc = u;
        double UU = dmax_ref(fabs(dsl), fabs(dsp));
        UU = dmax_ref(UU, fabs(ddII));
        time = (UU > eps8) ? UU : eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w <= u)) {
            en = u; r = rI * aI / (aI - rI * (enI - u)); te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            const double ce = cII - g1 / 2.0 * (enII - u);
            en = u; r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -g1 / g2 * (enII - w) + 2.0 / g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == 0) && (ip == 0)) {  // two expansion fans
        double aI, aII;
        if (fabs(p - pI) < eps) aI = rI * cI;
        else aI = gm * rI * cI * (1.0 - p / pI) / (1.0 - pow((p / pI), gm));
        if (fabs(p - pII) < eps) aII = rII * cII;
        else aII = gm * rII * cII * (1.0 - p / pII) / (1.0 - pow((p / pII), gm));
        const double u = (aI * enI + aII * enII + pI - pII) / (aI + aII);
        const double dI = enI - cI;
        const double ddI = u - cI - g1 * (enI - u) / 2.0;
        const double dII = enII + cII;
        const double ddII = u + cII - g1 * (enII - u) / 2.0;
        dsl = dI; dsp = dII; dsc = u;
        double UU = dmax_ref(fabs(dsl), fabs(dsp));
        UU = dmax_ref(UU, fabs(ddII));
        UU = dmax_ref(UU, fabs(ddI));
        time = (UU > eps8) ? UU : eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            const double ce = g1 / g2 * (enI - w) + 2.0 / g2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / gm)); r = ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= u)) {
            const double ce = cI + g1 / 2.0 * (enI - u);
            en = u; r = ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w > u) && (w <= ddII)) {
            const double ce = cII - g1 / 2.0 * (enII - u);
            en = u; r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -g1 / g2 * (enII - w) + 2.0 / g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if ((il == -1) && (ip == -1)) {  // vacuum
        const double dI = enI - cI;
        const double ddI = enI + 2.0 / g1 * cI;
        const double dII = enII + cII;
        const double ddII = enII - 2.0 / g1 * cII;
        dsl = dI; dsp = dII; dsc = (dI + dII) / 2.0;
        double UU = dmax_ref(fabs(dsl), fabs(dsp));
        UU = dmax_ref(UU, fabs(ddII));
        UU = dmax_ref(UU, fabs(ddI));
        time = (UU > eps8) ? UU : eps8;
        if (w <= dI) {
            en = enI; p = pI; r = rI; te2 = teI2; te3 = teI3;
        }
        if ((w > dI) && (w < ddI)) {
            const double ce = g1 / g2 * (enI - w) + 2.0 / g2 * cI;
            en = w + ce; p = pI * pow((ce / cI), (1.0 / gm)); r = ga * p / ce / ce; te2 = teI2; te3 = teI3;
        }
        if ((w >= ddI) && (w <= ddII)) {
            en = w; p = 0.0; r = 0.0; te2 = 0.0; te3 = 0.0;
        }
        if ((w > ddII) && (w < dII)) {
            const double ce = -g1 / g2 * (enII - w) + 2.0 / g2 * cII;
            en = w - ce; p = pII * pow((ce / cII), (1.0 / gm)); r = ga * p / ce / ce; te2 = teII2; te3 = teII3;
        }
        if (w >= dII) {
            en = enII; p = pII; r = rII; te2 = teII2; te3 = teII3;
        }
    }
    if (ipiz == 1) {
        en = -en;
        const double dsl1 = dsl, dsp1 = dsp;
        dsl = -dsp1;
        dsp = -dsl1;
        dsc = -dsc;
        w = -w;
    }
    const double uo = al * en + al2 * te2 + al3 * te3;
    const double vo = be * en + be2 * te2 + be3 * te3;
    const double wo = ge * en + ge2 * te2 + ge3 * te3;
    const double eo = p / g1 + 0.5 * r * (uo * uo + vo * vo + wo * wo);
    en = al * uo + be * vo + ge * wo;
    qqq[0] = (r * (en - w));
    qqq[1] = (r * (en - w) * uo + al * p);
    qqq[2] = (r * (en - w) * vo + be * p);
    qqq[3] = (r * (en - w) * wo + ge * p);
    qqq[4] = ((en - w) * eo + en * p);
    ds[0] = dsl;
    ds[1] = dsp;
    ds[2] = dsc;
    return time;
}

}  // namespace gelios
