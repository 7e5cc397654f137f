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
enum : int { C_1 = 0, C_2 = 1, C_3 = 2, C_4 = 3, C_5 = 4, C_CENTR = 5 };
enum : int { P_CONTACT = 6, P_INNER_SHOCK = 7, P_OUTER_SHOCK = 8 };

// Slot (cell face) info bits.
enum : uint32_t {
    SI_TYPE_MASK = 7u,
    SI_GOD = 1u << 3,     // both end points on the same tracked surface (Setka.cpp:10287-10298)
    SI_NP = 1u << 4,      // exactly one end point on a tracked surface (Setka.cpp:10301-10324)
};
// Cell flag bits.
// cell flags; CF_RP marks the cells whose |centroid|^(2 gamma) a moving-grid
// step reads (radial reconstructions, inner-shock masters)
// CF_EARLY: updated first by the pipelined moving-grid step (the next step's
// surface tracking and tracked-face reconstructions read the cell)
enum : uint32_t { CF_AXIS = 1u, CF_C1 = 2u, CF_CENTR = 4u, CF_RP = 8u, CF_EARLY = 16u };
// unit info: slot info (SI_*) in bits 0-7, the owner's cell flags from bit
// 8, the neighbour's from bit 12
enum : uint32_t { UI_CF_OWN = 8u, UI_CF_NB = 12u };
// Status flag bits (gelios_status::flags).
enum : int { ST_ITER_CAP = 1, ST_TVD_BAD = 2, ST_NEWTON_NEG = 4, ST_CHAIN = 8, ST_DT_BAD = 16, ST_WAVE_ORDER = 32 };

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

// Flux arithmetic tags: double (the drop-in), float (the FP32-flux form),
// WaveF32 (the wave-speed estimates SL, SR and the sound speeds behind them
// in FP32, every flux and star state in FP64).
struct WaveF32 {};
template <typename TF>
struct FluxArith {
    using type = TF;
};
template <>
struct FluxArith<WaveF32> {
    using type = double;
};
template <typename TF>
struct WaveArith {
    using type = TF;
};
template <>
struct WaveArith<WaveF32> {
    using type = float;
};

template <typename TF>
__device__ __forceinline__ double hllc_flux(double gamma, double kurant, const St5& L, const St5& R, double Wd,
                                            double n1d, double n2d, double rad, int metod, bool nul_potok,
                                            FluxOut<double>& out) {
    using T = typename FluxArith<TF>::type;
    using TW = typename WaveArith<TF>::type;
    const T ggg = (T)gamma, g1 = (T)(gamma - 1.0);
    const T n1 = (T)n1d, n2 = (T)n2d, W = (T)Wd;
    const T ro_L = (T)L.ro, Q_L = (T)L.Q, p_L = (T)L.p, v1_L = (T)L.u, v2_L = (T)L.v;
    const T ro_R = (T)R.ro, Q_R = (T)R.Q, p_R = (T)R.p, v1_R = (T)R.u, v2_R = (T)R.v;
    const T t1 = n2, t2 = -n1;
    const T u1 = v1_L * n1 + v2_L * n2;
    const T v1 = v1_L * t1 + v2_L * t2;
    const T u2 = v1_R * n1 + v2_R * n2;
    const T v2 = v1_R * t1 + v2_R * t2;
    // sound speeds and the HLL wave-speed estimates in the wave arithmetic
    // (the flux arithmetic except for WaveF32)
    const TW cL = tsqrt<TW>((TW)gamma * (TW)L.p / (TW)L.ro);
    const TW cR = tsqrt<TW>((TW)gamma * (TW)R.p / (TW)R.ro);
    const T uu_L = (v1_L * v1_L + v2_L * v2_L) / (T)2;
    const T uu_R = (v1_R * v1_R + v2_R * v2_R) / (T)2;
    const T SL = (T)((TW)tmin<T>(u1, u2) - tmax<TW>(cL, cR));
    const T SR = (T)((TW)tmax<T>(u1, u2) + tmax<TW>(cL, cR));
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
    const double g1 = ga - 1.0, g2 = ga + 1.0, gm = (g1 / ga) / 2.0;
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

// ---------------------------------------------------------------- MHD fluxes
// Magnetic fields enter these solvers in Gaussian units and are scaled by
// 1/sqrt(4 pi) inside (Solvers.h:12, Solvers.cpp:115-127, 1648-1654).
__device__ __forceinline__ double spi4_dev() { return sqrt(4.0 * kPi); }

// Solvers::HLLDQ_Korolkov (Solvers.cpp:1642-2185).  L, R = (ro, Q, p, v1,
// v2, v3, Bx, By, Bz); the normal must be a coordinate axis (the tangent
// pair is picked from its sign and direction).  metod 2: HLLC-type MHD
// flux, metod 3: HLLD.  Pout[8] = mass, momentum x3, B flux x3, energy (the
// reference's final reordering), *PQ = flux of Q.  Returns kurant*rad/max|S|.
// Other metods leave Pout and *PQ untouched, as the reference does.
//
// MOVING = true (metod 3 only) samples the HLLD fan at the face speed W
// instead of at 0 and returns the flux through the moving face, F - W U of
// the region that contains W, the way HLLC_2d_Korolkov_b_s treats moving
// faces (Setka.cpp:10604-10699); the normal-field term becomes
// -SN (bn2 - bn1) - W bn.  With MOVING = false the code is the reference's.
template <bool MOVING>
__device__ inline double hlldq_impl(double ga, double kurant, const double* L, const double* R, double n1, double n2,
                                    double n3, double rad, int metod, double* Pout, double* PQ, double W) {
    const double spi4 = spi4_dev();
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
    const double bb_L = sq(bx_L) + sq(by_L) + sq(bz_L);
    const double bb_R = sq(bx_R) + sq(by_R) + sq(bz_R);
    const double uu_L = (sq(v1_L) + sq(v2_L) + sq(v3_L)) / 2.0;
    const double uu_R = (sq(v1_R) + sq(v2_R) + sq(v3_R)) / 2.0;
    const double cfL = sqrt((ga * p_L + bb_L + sqrt(sq(ga * p_L + bb_L) - 4.0 * ga * p_L * sq(bn1))) / (2.0 * ro_L));
    const double cfR = sqrt((ga * p_R + bb_R + sqrt(sq(ga * p_R + bb_R) - 4.0 * ga * p_R * sq(bn2))) / (2.0 * ro_R));
    const double SL = dmin_ref(u1, u2) - dmax_ref(cfL, cfR);
    const double SR = dmax_ref(u1, u2) + dmax_ref(cfL, cfR);
    const double pTL = p_L + bb_L / 2.0;
    const double pTR = p_R + bb_R / 2.0;
    const double suR = SR - u2, suL = SL - u1;
    const double SM = (suR * ro_R * u2 - suL * ro_L * u1 - pTR + pTL) / (suR * ro_R - suL * ro_L);
    const double PTT = (suR * ro_R * pTL - suL * ro_L * pTR + ro_L * ro_R * suR * suL * (u2 - u1)) /
                       (suR * ro_R - suL * ro_L);
    const double UU = dmax_ref(fabs(SL), fabs(SR));
    const double time = kurant * rad / UU;
    if (metod != 2 && metod != 3) return time;
    const double e1 = p_L / g1 + ro_L * uu_L + bb_L / 2.0;
    const double e2 = p_R / g1 + ro_R * uu_R + bb_R / 2.0;
    const double FL[9] = {ro_L * u1,
                          ro_L * u1 * u1 + pTL - sq(bn1),
                          ro_L * u1 * v1 - bn1 * bt1,
                          ro_L * u1 * w1 - bn1 * bm1,
                          (e1 + pTL) * u1 - bn1 * (u1 * bn1 + v1 * bt1 + w1 * bm1),
                          0.0,
                          u1 * bt1 - v1 * bn1,
                          u1 * bm1 - w1 * bn1,
                          Q_L * u1};
    const double FR[9] = {ro_R * u2,
                          ro_R * u2 * u2 + pTR - sq(bn2),
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
        const double Ws = MOVING ? W : 0.0;
        if (SL >= Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * UL[i];
        } else if (SL < Ws && SLL >= Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] + SL * ULL[i] - SL * UL[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * ULL[i];
        } else if (SLL <= Ws && SM >= Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FL[i] + SLL * ULLL[i] - (SLL - SL) * ULL[i] - SL * UL[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * ULLL[i];
        } else if (SM < Ws && SRR > Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] + SRR * URRR[i] - (SRR - SR) * URR[i] - SR * UR[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * URRR[i];
        } else if (SR > Ws && SRR <= Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i] + SR * URR[i] - SR * UR[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * URR[i];
        } else if (SR <= Ws) {
            for (int i = 0; i < 9; i++) PO[i] = FR[i];
            if (MOVING)
                for (int i = 0; i < 9; i++) PO[i] -= W * UR[i];
        }
    }
    const double SN = dmax_ref(fabs(SL), fabs(SR));
    PO[5] = -SN * (bn2 - bn1);
    if (MOVING) PO[5] -= W * bn;
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
__device__ inline double hlldq_korolkov(double ga, double kurant, const double* L, const double* R, double n1,
                                        double n2, double n3, double rad, int metod, double* Pout, double* PQ) {
    return hlldq_impl<false>(ga, kurant, L, R, n1, n2, n3, rad, metod, Pout, PQ, 0.0);
}

// hlldq_impl<true>(ga, 1, L, R, 1, 0, 0, 1, 3, Pout, PQ, W) with the normal
// fixed to the x axis of the face frame, written for few registers: the
// wave speeds and star quantities first, then only the fan region that
// contains W, one component at a time.  The arithmetic of hlldq_impl, with
// shared reciprocals in place of repeated quotients.
// L, R = (ro, Q, p, u_n, u_t, u_phi, B_n, B_t, B_phi); Pout[8] = mass,
// momentum n, t, phi, B n, t, phi, energy; *PQ = Q flux.  Returns 1/max|S|.
template <typename T>
__device__ inline double hlld_face_moving(double gad, const double* L, const double* R, double Wd, double* Pout,
                                          double* PQ) {
    const T spi4 = (T)spi4_dev();
    const T ga = (T)gad, W = (T)Wd;
    const T g1 = ga - (T)1;
    auto sq = [](T x) { return x * x; };
    auto sqrt = [](T x) { return tsqrt<T>(x); };
    auto fabs = [](T x) -> T {
        if constexpr (sizeof(T) == 8) return ::fabs(x);
        else return fabsf(x);
    };
    auto dmin_ref = [](T a, T b) { return tmin<T>(a, b); };
    auto dmax_ref = [](T a, T b) { return tmax<T>(a, b); };
    auto sgn = [](T x) { return x > (T)0 ? (T)1 : (x < (T)0 ? (T)-1 : (T)0); };
    const T ro_L = (T)L[0], Q_L = (T)L[1], p_L = (T)L[2], u1 = (T)L[3], v1 = (T)L[4], w1 = (T)L[5];
    const T ro_R = (T)R[0], Q_R = (T)R[1], p_R = (T)R[2], u2 = (T)R[3], v2 = (T)R[4], w2 = (T)R[5];
    const T ispi4 = (T)1 / spi4;
    const T bn1 = (T)L[6] * ispi4, bt1 = (T)L[7] * ispi4, bm1 = (T)L[8] * ispi4;
    const T bn2 = (T)R[6] * ispi4, bt2 = (T)R[7] * ispi4, bm2 = (T)R[8] * ispi4;
    const T bb_L = sq(bn1) + sq(bt1) + sq(bm1);
    const T bb_R = sq(bn2) + sq(bt2) + sq(bm2);
    const T uu_L = (sq(u1) + sq(v1) + sq(w1)) * (T)0.5;
    const T uu_R = (sq(u2) + sq(v2) + sq(w2)) * (T)0.5;
    const T cfL = sqrt((ga * p_L + bb_L + sqrt(sq(ga * p_L + bb_L) - (T)4.0 * ga * p_L * sq(bn1))) / ((T)2.0 * ro_L));
    const T cfR = sqrt((ga * p_R + bb_R + sqrt(sq(ga * p_R + bb_R) - (T)4.0 * ga * p_R * sq(bn2))) / ((T)2.0 * ro_R));
    const T SL = dmin_ref(u1, u2) - dmax_ref(cfL, cfR);
    const T SR = dmax_ref(u1, u2) + dmax_ref(cfL, cfR);
    const T pTL = p_L + bb_L * (T)0.5;
    const T pTR = p_R + bb_R * (T)0.5;
    const T suR = SR - u2, suL = SL - u1;
    const T rden = (T)1 / (suR * ro_R - suL * ro_L);
    const T SM = (suR * ro_R * u2 - suL * ro_L * u1 - pTR + pTL) * rden;
    const T PTT = (suR * ro_R * pTL - suL * ro_L * pTR + ro_L * ro_R * suR * suL * (u2 - u1)) * rden;
    const T UU = dmax_ref(fabs(SL), fabs(SR));
    const double time = 1.0 * 1.0 / (double)UU;
    const T rg1 = (T)1 / g1;
    const T e1 = p_L * rg1 + ro_L * uu_L + bb_L * (T)0.5;
    const T e2 = p_R * rg1 + ro_R * uu_R + bb_R * (T)0.5;
    const T sbv1 = u1 * bn1 + v1 * bt1 + w1 * bm1, sbv2 = u2 * bn2 + v2 * bt2 + w2 * bm2;
    // fluxes of the two sides (the normal-field flux is 0)
    const T FLt = u1 * bt1 - v1 * bn1, FLm = u1 * bm1 - w1 * bn1;
    const T FRt = u2 * bt2 - v2 * bn2, FRm = u2 * bm2 - w2 * bn2;
    const T bn = (SR * bn2 - SL * bn1 + (T)0.0 - (T)0.0) / (SR - SL);
    const T bbn = bn * bn;
    const T rLM = (T)1 / (SL - SM), rRM = (T)1 / (SR - SM);
    const T ro_LL = ro_L * (SL - u1) * rLM;
    const T ro_RR = ro_R * (SR - u2) * rRM;
    const T Q_LL = Q_L * (SL - u1) * rLM;
    const T Q_RR = Q_R * (SR - u2) * rRM;
    const T ttL = ro_L * suL * (SL - SM) - bbn;
    const T ttR = ro_R * suR * (SR - SM) - bbn;
    T vLL, wLL, vRR, wRR, btt1, bmm1, btt2, bmm2;
    if (fabs(ttL) >= (T)0.000001) {
        const T r = (T)1 / ttL;
        vLL = v1 - bn * bt1 * (SM - u1) * r;
        wLL = w1 - bn * bm1 * (SM - u1) * r;
        btt1 = bt1 * (ro_L * suL * suL - bbn) * r;
        bmm1 = bm1 * (ro_L * suL * suL - bbn) * r;
    } else {
        vLL = v1; wLL = w1; btt1 = (T)0.0; bmm1 = (T)0.0;
    }
    if (fabs(ttR) >= (T)0.000001) {
        const T r = (T)1 / ttR;
        vRR = v2 - bn * bt2 * (SM - u2) * r;
        wRR = w2 - bn * bm2 * (SM - u2) * r;
        btt2 = bt2 * (ro_R * suR * suR - bbn) * r;
        bmm2 = bm2 * (ro_R * suR * suR - bbn) * r;
    } else {
        vRR = v2; wRR = w2; btt2 = (T)0.0; bmm2 = (T)0.0;
    }
    const T eLL = (e1 * suL + PTT * SM - pTL * u1 + bn * (sbv1 - (SM * bn + vLL * btt1 + wLL * bmm1))) * rLM;
    const T eRR = (e2 * suR + PTT * SM - pTR * u2 + bn * (sbv2 - (SM * bn + vRR * btt2 + wRR * bmm2))) * rRM;
    const T sqrtroLL = sqrt(ro_LL), sqrtroRR = sqrt(ro_RR);
    T SLL = SM - fabs(bn) / sqrtroLL;
    T SRR = SM + fabs(bn) / sqrtroRR;
    T idbn;
    if (fabs(bn) > (T)0.001) {
        idbn = (T)1.0 * sgn(bn);
    } else {
        idbn = (T)0.0;
        SLL = SM;
        SRR = SM;
    }
    // fan region containing W: 0 L, 1 L*, 2 L**, 3 R**, 4 R*, 5 R
    int reg = -1;
    if (SL >= W) reg = 0;
    else if (SL < W && SLL >= W) reg = 1;
    else if (SLL <= W && SM >= W) reg = 2;
    else if (SM < W && SRR > W) reg = 3;
    else if (SR > W && SRR <= W) reg = 4;
    else if (SR <= W) reg = 5;
    T PO[9];
    for (int i = 0; i < 9; i++) PO[i] = (T)0;
    const bool left = reg <= 2;
    // one side's state U, flux F, single-star state U* and the double-star
    // state U** (reg 2/3 only)
    const T ro = left ? ro_L : ro_R, uu = left ? u1 : u2, vv = left ? v1 : v2, ww = left ? w1 : w2;
    const T bnk = left ? bn1 : bn2, btk = left ? bt1 : bt2, bmk = left ? bm1 : bm2;
    const T ek = left ? e1 : e2, pTk = left ? pTL : pTR, Qk = left ? Q_L : Q_R;
    const T Sk = left ? SL : SR;
    const T U[9] = {ro, ro * uu, ro * vv, ro * ww, ek, bnk, btk, bmk, Qk};
    const T F[9] = {ro * uu,
                         ro * uu * uu + pTk - sq(bnk),
                         ro * uu * vv - bnk * btk,
                         ro * uu * ww - bnk * bmk,
                         (ek + pTk) * uu - bnk * (uu * bnk + vv * btk + ww * bmk),
                         (T)0.0,
                         left ? FLt : FRt,
                         left ? FLm : FRm,
                         Qk * uu};
    if (reg < 0) {
        // no region (non-finite speeds): zero flux, as the reference's chain of tests leaves it
    } else if (reg == 0 || reg == 5) {
        for (int i = 0; i < 9; i++) PO[i] = F[i] - W * U[i];
    } else {
        const T roS = left ? ro_LL : ro_RR, vS = left ? vLL : vRR, wS = left ? wLL : wRR;
        const T btS = left ? btt1 : btt2, bmS = left ? bmm1 : bmm2, eS = left ? eLL : eRR;
        const T QS = left ? Q_LL : Q_RR;
        const T US[9] = {roS, roS * SM, roS * vS, roS * wS, eS, bn, btS, bmS, QS};
        if (reg == 1 || reg == 4) {
            for (int i = 0; i < 9; i++) PO[i] = F[i] + Sk * US[i] - Sk * U[i] - W * US[i];
        } else {
            const T rs = (T)1 / (sqrtroLL + sqrtroRR);
            const T vLLL = (sqrtroLL * vLL + sqrtroRR * vRR + idbn * (btt2 - btt1)) * rs;
            const T wLLL = (sqrtroLL * wLL + sqrtroRR * wRR + idbn * (bmm2 - bmm1)) * rs;
            const T bttt = (sqrtroLL * btt2 + sqrtroRR * btt1 + idbn * sqrtroLL * sqrtroRR * (vRR - vLL)) * rs;
            const T bmmm = (sqrtroLL * bmm2 + sqrtroRR * bmm1 + idbn * sqrtroLL * sqrtroRR * (wRR - wLL)) * rs;
            T eSS;
            if (left)
                eSS = eLL - idbn * sqrtroLL * ((SM * bn + vLL * btt1 + wLL * bmm1) - (SM * bn + vLLL * bttt + wLLL * bmmm));
            else
                eSS = eRR + idbn * sqrtroRR * ((SM * bn + vRR * btt2 + wRR * bmm2) - (SM * bn + vLLL * bttt + wLLL * bmmm));
            const T USS[9] = {roS, roS * SM, roS * vLLL, roS * wLLL, eSS, bn, bttt, bmmm, QS};
            const T SS = left ? SLL : SRR;
            for (int i = 0; i < 9; i++) PO[i] = F[i] + SS * USS[i] - (SS - Sk) * US[i] - Sk * U[i] - W * USS[i];
        }
    }
    const T SN = dmax_ref(fabs(SL), fabs(SR));
    PO[5] = -SN * (bn2 - bn1);
    PO[5] -= W * bn;
    Pout[0] = (double)PO[0];
    Pout[1] = (double)PO[1];
    Pout[2] = (double)PO[2];
    Pout[3] = (double)PO[3];
    Pout[4] = (double)(spi4 * PO[5]);
    Pout[5] = (double)(spi4 * PO[6]);
    Pout[6] = (double)(spi4 * PO[7]);
    Pout[7] = (double)PO[4];
    *PQ = (double)PO[8];
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
__device__ inline double hlld_alexashov(double ga, double kurant, const double* qqq1, const double* qqq2,
                                        const double* n, double* qqq, double* ds, double wv, double DIST,
                                        int* status) {
    const double spi4 = spi4_dev();
    const double eps = 10e-10;
    const double g1 = ga - 1.0;
    const double r1 = qqq1[0], u1 = qqq1[2], v1 = qqq1[3], w1 = qqq1[4], p1 = qqq1[1];
    const double bx1 = qqq1[5] / spi4, by1 = qqq1[6] / spi4, bz1 = qqq1[7] / spi4;
    const double r2 = qqq2[0], u2 = qqq2[2], v2 = qqq2[3], w2 = qqq2[4], p2 = qqq2[1];
    const double bx2 = qqq2[5] / spi4, by2 = qqq2[6] / spi4, bz2 = qqq2[7] / spi4;
    const double abx = (bx2 + bx1) / 2.0, aby = (by2 + by1) / 2.0, abz = (bz2 + bz1) / 2.0;
    const double bk = abx * n[0] + aby * n[1] + abz * n[2];
    const double b2 = sq(abx) + sq(aby) + sq(abz);
    double d = b2 - sq(bk);
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
        d = sqrt(1.0 - sq(aik));
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
    const double b2L = sq(bL[0]) + sq(bL[1]) + sq(bL[2]);
    const double b21 = b2L / r1;
    const double cL = sqrt(ga * p1 / r1);
    double qp = sqrt(b21 + cL * (cL + 2.0 * aaL));
    double qm = sqrt(b21 + cL * (cL - 2.0 * aaL));
    const double cfL = (qp + qm) / 2.0;
    const double ptL = p1 + b2L / 2.0;
    const double aaR = bR[0] / sqrt(r2);
    const double b2R = sq(bR[0]) + sq(bR[1]) + sq(bR[2]);
    const double b22 = b2R / r2;
    const double cR = sqrt(ga * p2 / r2);
    qp = sqrt(b22 + cR * (cR + 2.0 * aaR));
    qm = sqrt(b22 + cR * (cR - 2.0 * aaR));
    const double cfR = (qp + qm) / 2.0;
    const double ptR = p2 + b2R / 2.0;
    const double SL = dmin_ref((vL[0] - cfL), (vR[0] - cfR));
    const double SR = dmax_ref((vL[0] + cfL), (vR[0] + cfR));
    const double suR = SR - vR[0], suL = SL - vL[0];
    const double SM = (suR * r2 * vR[0] - ptR + ptL - suL * r1 * vL[0]) / (suR * r2 - suL * r1);
    if (SR <= SL || SM >= SR || SM <= SL) *status |= ST_WAVE_ORDER;
    ds[0] = SL;
    ds[1] = SR;
    ds[2] = SM;
    const double UU = dmax_ref(fabs(SL), fabs(SR));
    const double time = kurant * DIST / UU;
    const double upt1 = (sq(u1) + sq(v1) + sq(w1)) / 2.0;
    const double sbv1 = u1 * bx1 + v1 * by1 + w1 * bz1;
    const double upt2 = (sq(u2) + sq(v2) + sq(w2)) / 2.0;
    const double sbv2 = u2 * bx2 + v2 * by2 + w2 * bz2;
    const double e1 = p1 / g1 + r1 * upt1 + b2L / 2.0;
    const double e2 = p2 / g1 + r2 * upt2 + b2R / 2.0;
    const double FL[8] = {r1 * vL[0],
                          r1 * vL[0] * vL[0] + ptL - sq(bL[0]),
                          r1 * vL[0] * vL[1] - bL[0] * bL[1],
                          r1 * vL[0] * vL[2] - bL[0] * bL[2],
                          (e1 + ptL) * vL[0] - bL[0] * sbv1,
                          0.0,
                          vL[0] * bL[1] - vL[1] * bL[0],
                          vL[0] * bL[2] - vL[2] * bL[0]};
    const double FR[8] = {r2 * vR[0],
                          r2 * vR[0] * vR[0] + ptR - sq(bR[0]),
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

}  // namespace gelios
