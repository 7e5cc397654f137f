// Native host-side grid builders of gelios_b200.
//
//  * gelios_mesh_build_setka: the rail grid of Setka::Setka(N1..M4)
//    (Setka.cpp:19-1076) with Rail::Init_start (Rail.cpp:15-182).  The
//    numbering of points, cells and faces and the order of every list are
//    part of the drop-in contract (the cell face order is the flux
//    summation order, the face numbers drive TVD_prepare), so the
//    construction steps below follow the reference's sequence one for one;
//    the data structures are flat index arrays instead of heap objects.
//  * gelios_mesh_build_polar: the axisymmetric polar half-plane grid of the
//    plain single-fluid workload (180 x 120 log-radial quads).
//  * gelios_mesh_tvd_prepare: Setka::TVD_prepare (Setka.cpp:1294-1492).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gelios_b200.h"

namespace gelios {
void set_error(const std::string& msg);
}

namespace {

constexpr double kPi = 3.14159265358979323846;
// Geometry scale and radii of the reference grid (Help.h:78-89).
constexpr double kRR = 390.222;
constexpr double kR1 = 1.0 / kRR;
constexpr double kR2 = 100.0 / kRR;
constexpr double kR3 = 150.0 / kRR;
constexpr double kR4 = 600.0 / kRR;
constexpr double kR5 = 2200.0 / kRR;
constexpr double kLeft = -1500.0 / kRR;

// Gran_type, Cell_type, Point_type, Rail_type values of the reference.
enum { G_USUALY = 0, G_INNER_SPHERE, G_EXTERN, G_INPUT, G_AXIS, G_UPPER_WALL, G_NO };
enum { C_1 = 0, C_2, C_3, C_4, C_5, C_CENTR, C_NO };
enum {
    P_USUALY = 0, P_U_1, P_U_2, P_U_3, P_U_4, P_U_5, P_CONTACT, P_INNER_SHOCK, P_OUTER_SHOCK,
    P_INNER_BOUNDARY, P_OUTER_BOUNDARY, P_NO, P_NULL
};
enum { R_A = 0, R_B, R_C, R_D };

inline double sq(double x) { return x * x; }

// polar_angle, Help.cpp:37-65
double polar_angle(double x, double y) {
    if (std::fabs(x) + std::fabs(y) < 0.000001 / kRR) return 0.0;
    if (x < 0) return std::atan(y / x) + 1.0 * kPi;
    if (x > 0 && y >= 0) return std::atan(y / x);
    if (x > 0 && y < 0) return std::atan(y / x) + 2.0 * kPi;
    if (y > 0 && x >= 0 && x <= 0) return kPi / 2.0;
    if (y < 0 && x >= 0 && x <= 0) return 3.0 * kPi / 2.0;
    return 0.0;
}

}  // namespace

struct gelios_mesh {
    int32_t dims[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::vector<double> x, y;
    std::vector<int32_t> ptype;
    std::vector<int32_t> ctype, cstart, contour, gstart, gran, cback, cnext;
    std::vector<double> r_istoch;
    int32_t n_main = 0;
    std::vector<int32_t> fA, fB, ftype, fmaster, fsosed, fcopy, fsup, fsdown;
    std::vector<int32_t> rtype, rM, rpstart, rpts, rkstart, rkeys;
    std::vector<double> rs;
    std::vector<int32_t> lcontact, linner, louter;
    // Gran::number as TVD_prepare sees it: 0 = the constructor's numbering
    // (All_Gran and All_Gran_copy each from 0, so numbers collide), 1 = the
    // unique numbering Download_Setka_ALL_ALPHA_2_0 gives (Setka.cpp:3213-3224)
    int32_t unique_face_numbers = 0;
};

namespace {

// Builder state mirroring the object graph the reference constructor creates.
struct Rail {
    int type;
    double s;
    int M1 = 0, M2 = 0, M3 = 0, M4 = 0;
    std::vector<int> pts, keys;
};
struct Face {  // a Gran object
    int A, B, type;
    int master = -1, sosed = -1;
    int copy = -1;  // tagged reference (see Builder::tag_*), -1 = none
    bool main_gran = true;
    bool is_copy = false;
};
struct CellB {
    int type = C_NO;
    std::vector<int> contour;
    std::vector<int> grans;  // tagged face references
};

struct Builder {
    std::vector<double> px, py;
    std::vector<int> pt;
    std::vector<CellB> cells;
    std::vector<Face> mainF, copyF;

    int point(double x, double y) {
        px.push_back(x);
        py.push_back(y);
        pt.push_back(P_NO);
        return static_cast<int>(px.size()) - 1;
    }
    int cell(int a, int b, int c, int d) {
        CellB k;
        k.contour = {a, b, c, d};
        cells.push_back(k);
        return static_cast<int>(cells.size()) - 1;
    }
    // tagged face references: main face i -> i, copy i -> -(i + 2), none -> -1
    static int tag_main(int i) { return i; }
    static int tag_copy(int i) { return -(i + 2); }
    Face& ref(int t) { return t >= 0 ? mainF[t] : copyF[-t - 2]; }

    int add_main(int A, int B, int type) {
        Face f{A, B, type};
        f.main_gran = true;
        mainF.push_back(f);
        return tag_main(static_cast<int>(mainF.size()) - 1);
    }
    int add_copy(int A, int B, int type) {
        Face f{A, B, type};
        f.main_gran = false;
        f.is_copy = true;
        copyF.push_back(f);
        return tag_copy(static_cast<int>(copyF.size()) - 1);
    }
    // An interior face G(K.a, K.b) with its reversed twin, Master K, Sosed F
    // (the repeated pattern of Setka.cpp:318-331 and siblings).
    void pair(int K, int F, int a, int b) {
        int G = add_main(a, b, G_USUALY);
        int G2 = add_copy(b, a, G_USUALY);
        ref(G).copy = G2;
        ref(G2).copy = G;
        ref(G).master = K;
        ref(G).sosed = F;
        ref(G2).master = F;
        ref(G2).sosed = K;
        cells[K].grans.push_back(G);
        cells[F].grans.push_back(G2);
    }
    // A boundary face without twin (Input/Upper_wall/Extern ends of the rays).
    void single(int K, int a, int b, int type) {
        int G = add_main(a, b, type);
        ref(G).master = K;
        cells[K].grans.push_back(G);
    }
};

void rail_init_start(Builder& B, Rail& R) {  // Rail::Init_start, Rail.cpp:15-182
    double r, l;
    if (R.type == R_A) {
        double x = std::pow(kR2 / kR1, 1.0 / (R.M1 - 1));
        for (int i = 0; i < R.M1; i++) {
            r = kR1 * std::pow(x, static_cast<double>(i));
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_1;
            if (i == R.M1 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_INNER_SHOCK;
            }
            if (i == 0) B.pt[K] = P_INNER_BOUNDARY;
        }
        for (int i = 0; i < R.M2; i++) {
            r = kR2 + (kR3 - kR2) * (i + 1) / (R.M2);
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_3;
            if (i == R.M2 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_CONTACT;
            }
        }
        for (int i = 0; i < R.M3; i++) {
            r = kR3 + (kR4 - kR3) * (i + 1) / (R.M3);
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_4;
            if (i == R.M3 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_SHOCK;
            }
        }
        x = std::pow(kR5 / kR4, 1.0 / (R.M4));
        for (int i = 0; i < R.M4; i++) {
            r = kR4 * std::pow(x, static_cast<double>(i + 1));
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_5;
            if (i == R.M4 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_BOUNDARY;
            }
        }
    } else if (R.type == R_B) {
        double x = std::pow(kR2 / kR1, 1.0 / (R.M1 - 1));
        for (int i = 0; i < R.M1; i++) {
            r = kR1 * std::pow(x, static_cast<double>(i));
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_1;
            if (i == R.M1 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_INNER_SHOCK;
            }
            if (i == 0) B.pt[K] = P_INNER_BOUNDARY;
        }
        for (int i = 0; i < R.M2; i++) {
            l = kR2 * std::sin(R.s) + (i + 1) * (kR3 - kR2 * std::sin(R.s)) / (R.M2);
            int K = B.point(kR2 * std::cos(R.s), l);
            R.pts.push_back(K);
            B.pt[K] = P_U_3;
            if (i == R.M2 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_CONTACT;
            }
        }
        for (int i = 0; i < R.M3; i++) {
            l = kR3 + (i + 1) * (kR4 - kR3) / R.M3;
            int K = B.point(kR2 * std::cos(R.s), l);
            R.pts.push_back(K);
            B.pt[K] = P_U_4;
            if (i == R.M3 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_SHOCK;
            }
        }
        double x4 = std::pow(kR5 / kR4, 1.0 / (R.M4));
        for (int i = 0; i < R.M4; i++) {
            l = kR4 * std::pow(x4, static_cast<double>(i + 1));
            int K = B.point(kR2 * std::cos(R.s), l);
            R.pts.push_back(K);
            B.pt[K] = P_U_5;
            if (i == R.M4 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_BOUNDARY;
            }
        }
    } else if (R.type == R_C) {
        double x = std::pow(kR2 / kR1, 1.0 / (R.M1 - 1));
        for (int i = 0; i < R.M1; i++) {
            r = kR1 * std::pow(x, static_cast<double>(i));
            int K = B.point(r * std::cos(R.s), r * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_1;
            if (i == R.M1 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_INNER_SHOCK;
            }
            if (i == 0) B.pt[K] = P_INNER_BOUNDARY;
        }
        x = std::pow(kLeft / (kR2 * std::cos(R.s)), 1.0 / (R.M2));
        for (int i = 0; i < R.M2; i++) {
            l = kR2 * std::cos(R.s) * std::pow(x, static_cast<double>(i + 1));
            int K = B.point(l, kR2 * std::sin(R.s));
            R.pts.push_back(K);
            B.pt[K] = P_U_2;
            if (i == R.M2 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_BOUNDARY;
            }
        }
    }
}

void finalize(Builder& B, gelios_mesh& m, const std::vector<Rail*>& rails) {
    const int nm = static_cast<int>(B.mainF.size());
    const int nc = static_cast<int>(B.copyF.size());
    auto uid = [&](int t) { return t >= 0 ? t : (t == -1 ? -1 : nm + (-t - 2)); };
    m.x = B.px;
    m.y = B.py;
    m.ptype.assign(B.pt.begin(), B.pt.end());
    const int ncell = static_cast<int>(B.cells.size());
    m.ctype.resize(ncell);
    m.cstart.assign(1, 0);
    m.gstart.assign(1, 0);
    m.contour.clear();
    m.gran.clear();
    for (int c = 0; c < ncell; c++) {
        m.ctype[c] = B.cells[c].type;
        for (int p : B.cells[c].contour) m.contour.push_back(p);
        for (int g : B.cells[c].grans) m.gran.push_back(uid(g));
        m.cstart.push_back(static_cast<int32_t>(m.contour.size()));
        m.gstart.push_back(static_cast<int32_t>(m.gran.size()));
    }
    m.cback.assign(ncell, -1);
    m.cnext.assign(ncell, -1);
    m.r_istoch.assign(ncell, 0.0);
    m.n_main = nm;
    const int nf = nm + nc;
    m.fA.resize(nf); m.fB.resize(nf); m.ftype.resize(nf); m.fmaster.resize(nf);
    m.fsosed.resize(nf); m.fcopy.resize(nf);
    m.fsup.assign(nf, -1);
    m.fsdown.assign(nf, -1);
    for (int f = 0; f < nf; f++) {
        const Face& F = f < nm ? B.mainF[f] : B.copyF[f - nm];
        m.fA[f] = F.A; m.fB[f] = F.B; m.ftype[f] = F.type;
        m.fmaster[f] = F.master; m.fsosed[f] = F.sosed;
        m.fcopy[f] = uid(F.copy);
    }
    m.rtype.clear(); m.rs.clear(); m.rM.clear();
    m.rpstart.assign(1, 0);
    m.rkstart.assign(1, 0);
    m.rpts.clear(); m.rkeys.clear();
    for (const Rail* R : rails) {
        m.rtype.push_back(R->type);
        m.rs.push_back(R->s);
        m.rM.push_back(R->M1); m.rM.push_back(R->M2); m.rM.push_back(R->M3); m.rM.push_back(R->M4);
        for (int p : R->pts) m.rpts.push_back(p);
        for (int p : R->keys) m.rkeys.push_back(p);
        m.rpstart.push_back(static_cast<int32_t>(m.rpts.size()));
        m.rkstart.push_back(static_cast<int32_t>(m.rkeys.size()));
    }
}

}  // namespace

namespace gelios {
// Owned copy of a caller's mesh view (used when the caller leaves the
// TVD_prepare outputs empty).
gelios_mesh* mesh_from_view(const gelios_mesh_view* v) {
    auto* m = new gelios_mesh();
    std::memcpy(m->dims, v->dims, sizeof(m->dims));
    const int np = v->n_points, nc = v->n_cells, nf = v->n_faces, nr = v->n_rails;
    m->x.assign(v->x, v->x + np);
    m->y.assign(v->y, v->y + np);
    m->ptype.assign(v->point_type, v->point_type + np);
    m->ctype.assign(v->cell_type, v->cell_type + nc);
    m->cstart.assign(v->contour_start, v->contour_start + nc + 1);
    m->contour.assign(v->contour, v->contour + m->cstart[nc]);
    m->gstart.assign(v->gran_start, v->gran_start + nc + 1);
    m->gran.assign(v->gran, v->gran + m->gstart[nc]);
    m->cback.assign(nc, -1);
    m->cnext.assign(nc, -1);
    m->r_istoch.assign(nc, 0.0);
    m->n_main = v->n_main;
    m->fA.assign(v->face_A, v->face_A + nf);
    m->fB.assign(v->face_B, v->face_B + nf);
    m->ftype.assign(v->face_type, v->face_type + nf);
    m->fmaster.assign(v->face_master, v->face_master + nf);
    m->fsosed.assign(v->face_sosed, v->face_sosed + nf);
    m->fcopy.assign(v->face_copy, v->face_copy + nf);
    m->fsup.assign(nf, -1);
    m->fsdown.assign(nf, -1);
    if (nr > 0) {
        m->rtype.assign(v->rail_type, v->rail_type + nr);
        m->rs.assign(v->rail_s, v->rail_s + nr);
        m->rM.assign(v->rail_M, v->rail_M + 4 * nr);
        m->rpstart.assign(v->rail_pstart, v->rail_pstart + nr + 1);
        m->rpts.assign(v->rail_points, v->rail_points + m->rpstart[nr]);
        m->rkstart.assign(v->rail_kstart, v->rail_kstart + nr + 1);
        m->rkeys.assign(v->rail_keys, v->rail_keys + m->rkstart[nr]);
    } else {
        m->rpstart.assign(1, 0);
        m->rkstart.assign(1, 0);
    }
    if (v->n_contact) m->lcontact.assign(v->line_contact, v->line_contact + v->n_contact);
    if (v->n_inner_line) m->linner.assign(v->line_inner, v->line_inner + v->n_inner_line);
    if (v->n_outer_line) m->louter.assign(v->line_outer, v->line_outer + v->n_outer_line);
    return m;
}
}  // namespace gelios

extern "C" gelios_mesh* gelios_mesh_build_setka(int N1, int N2, int N3, int N4, int M1, int M2, int M3, int M4) {
    if (N1 < 1 || N2 < 1 || N3 < 1 || N4 < 2 || M1 < 1 || M2 < 1 || M3 < 1 || M4 < 1) {
        gelios::set_error("gelios_mesh_build_setka: dimensions out of range");
        return nullptr;
    }
    auto* m = new gelios_mesh();
    const int d[8] = {N1, N2, N3, N4, M1, M2, M3, M4};
    std::memcpy(m->dims, d, sizeof(d));
    Builder B;
    N1++;
    N3++;
    M1++;
    double s = 0.0;
    int kk, kkk, kkkk;
    int n = M1 + M2 + M3 + M4 - 1;  // faces along a ray
    std::vector<Rail> Ar(N1), Br(N2), Cr(N3), Dr(N4);
    std::vector<int> centr_grans;  // Grans of the temporary central cell (tagged)

    for (int i = 0; i < N1; i++) {  // Setka.cpp:43-61
        s = i * (kPi / 2.0) / (N1 - 1.0);
        Rail& R = Ar[i];
        R.type = R_A; R.s = s;
        R.M1 = M1; R.M2 = M2; R.M3 = M3; R.M4 = M4;
        rail_init_start(B, R);
    }
    for (int i = 0; i < N2; i++) {  // Setka.cpp:63-79
        s = (kPi / 2.0) + (i + 1) * (kPi / 3.0) / (N2);
        Rail& R = Br[i];
        R.type = R_B; R.s = s;
        R.M1 = M1; R.M2 = M2; R.M3 = M3; R.M4 = M4;
        rail_init_start(B, R);
    }
    // C rails (Setka.cpp:81-96): rails 1.. create their points now but those
    // points join All_Points only after C_Rails[0] is completed.
    const size_t c_points_begin = B.px.size();
    for (int i = 0; i < N3; i++) {
        s = (5.0 * kPi / 6.0) + (i) * (kPi / 6.0) / (N3 - 1);
        Rail& R = Cr[i];
        R.type = R_C; R.s = s;
        R.M1 = M1; R.M2 = N4; R.M3 = 0; R.M4 = 0;
        if (i > 0) rail_init_start(B, R);
    }
    const size_t c_points_end = B.px.size();
    for (int i = 0; i < N4; i++) {  // Setka.cpp:98-108
        s = -kR1 - (i + 1) * (-kR1 - kLeft) / (N4);
        Rail& R = Dr[i];
        R.type = R_D; R.s = s;
        R.M1 = N3; R.M2 = M2; R.M3 = M3; R.M4 = M4;
    }
    // The points of C rails 1.. were appended to the coordinate arrays in
    // creation order; the reference appends them to All_Points later.  Keep
    // creation separate from numbering: collect their coordinates and
    // renumber below.
    std::vector<double> cx(B.px.begin() + c_points_begin, B.px.begin() + c_points_end);
    std::vector<double> cy(B.py.begin() + c_points_begin, B.py.begin() + c_points_end);
    std::vector<int> ct(B.pt.begin() + c_points_begin, B.pt.begin() + c_points_end);
    B.px.resize(c_points_begin);
    B.py.resize(c_points_begin);
    B.pt.resize(c_points_begin);

    Rail& C0 = Cr[0];  // Setka.cpp:110-138
    for (int i = 0; i < M1; i++) {
        C0.pts.push_back(Br[N2 - 1].pts[i]);
        if (i == M1 - 1) C0.keys.push_back(Br[N2 - 1].pts[i]);
    }
    double l;
    double pr = (5.0 * kPi / 6.0);
    for (int i = 0; i < N4; i++) {
        double x = std::pow(kLeft / (kR2 * std::cos(pr)), 1.0 / (N4));
        l = kR2 * std::cos(pr) * std::pow(x, static_cast<double>(i + 1));
        int K = B.point(l, kR2 * std::sin(pr));
        C0.pts.push_back(K);
        B.pt[K] = P_U_2;
        if (i == N4 - 1) {
            C0.keys.push_back(K);
            B.pt[K] = P_OUTER_BOUNDARY;
        }
    }
    // Setka.cpp:141-147: C rails 1.. join All_Points now.
    {
        const int base = static_cast<int>(B.px.size());
        const int delta = base - static_cast<int>(c_points_begin);
        for (size_t k = 0; k < cx.size(); k++) {
            B.px.push_back(cx[k]);
            B.py.push_back(cy[k]);
            B.pt.push_back(ct[k]);
        }
        for (int i = 1; i < N3; i++) {
            for (int& p : Cr[i].pts) p += delta;
            for (int& p : Cr[i].keys) p += delta;
        }
    }
    for (int i = 0; i < N4; i++) {  // Setka.cpp:150-195
        int P = C0.pts[M1 + i];
        Rail& R = Dr[i];
        R.pts.push_back(P);
        R.keys.push_back(P);
        for (int j = 0; j < M2; j++) {
            l = B.py[P] + (j + 1) * (kR3 - B.py[P]) / (M2);
            int K = B.point(B.px[P], l);
            R.pts.push_back(K);
            B.pt[K] = P_U_3;
            if (j == M2 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_CONTACT;
            }
        }
        for (int j = 0; j < M3; j++) {
            l = kR3 + (j + 1) * (kR4 - kR3) / M3;
            int K = B.point(B.px[P], l);
            R.pts.push_back(K);
            B.pt[K] = P_U_4;
            if (j == M3 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_SHOCK;
            }
        }
        double x = std::pow(kR5 / kR4, 1.0 / (M4));
        for (int j = 0; j < M4; j++) {
            l = kR4 * std::pow(x, static_cast<double>(j + 1));
            int K = B.point(B.px[P], l);
            R.pts.push_back(K);
            B.pt[K] = P_U_5;
            if (j == M4 - 1) {
                R.keys.push_back(K);
                B.pt[K] = P_OUTER_BOUNDARY;
            }
        }
    }

    // Cells, Setka.cpp:198-281
    auto strip = [&](std::vector<Rail>& rs) {
        for (size_t i = 0; i + 1 < rs.size(); i++)
            for (size_t j = 0; j + 1 < rs[0].pts.size(); j++)
                B.cell(rs[i].pts[j], rs[i].pts[j + 1], rs[i + 1].pts[j + 1], rs[i + 1].pts[j]);
    };
    strip(Ar);
    strip(Br);
    strip(Cr);
    strip(Dr);
    {
        Rail& P1 = Ar[Ar.size() - 1];
        Rail& P2 = Br[0];
        for (size_t j = 0; j + 1 < P1.pts.size(); j++) B.cell(P1.pts[j], P1.pts[j + 1], P2.pts[j + 1], P2.pts[j]);
    }
    {
        Rail& P1 = Br[Br.size() - 1];
        Rail& P2 = Dr[0];
        for (size_t j = 0; j + 1 < P2.pts.size(); j++)
            B.cell(P1.pts[j + M1 - 1], P1.pts[j + M1], P2.pts[j + 1], P2.pts[j]);
    }

    // Faces, Setka.cpp:303-851.  K->contour[k] is B.cells[K].contour[k].
    auto cc = [&](int K, int k) { return B.cells[K].contour[k]; };
    const int ncells0 = static_cast<int>(B.cells.size());
    for (int i = 0; i < n * (N1 - 1); i++) {
        if ((i + 1) % (n) == 0) {
            B.single(i, cc(i, 1), cc(i, 2), G_INPUT);
            continue;
        }
        B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    }
    for (int i = 0; i < n * (N1 - 2); i++) B.pair(i, i + n, cc(i, 2), cc(i, 3));
    for (int i = n * (N1 - 1); i < n * (N2 + N1 - 2); i++) {
        if ((i + 1) % (n) == 0) {
            B.single(i, cc(i, 1), cc(i, 2), G_UPPER_WALL);
            continue;
        }
        B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    }
    for (int i = n * (N1 - 1); i < n * (N2 + N1 - 3); i++) B.pair(i, i + n, cc(i, 2), cc(i, 3));
    for (int i = n * (N2 + N1 - 2); i < n * (N2 + N1 - 2) + (N3 - 1) * (N4 + M1 - 1); i++) {
        if ((i + 1 - n * (N2 + N1 - 2)) % (N4 + M1 - 1) == 0) {
            B.single(i, cc(i, 1), cc(i, 2), G_EXTERN);
            continue;
        }
        B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    }
    for (int i = n * (N2 + N1 - 2); i < n * (N2 + N1 - 2) + (N3 - 2) * (N4 + M1 - 1); i++)
        B.pair(i, i + (N4 + M1 - 1), cc(i, 2), cc(i, 3));
    kk = n * (N2 + N1 - 2) + (N3 - 1) * (N4 + M1 - 1);
    for (int i = kk; i < kk + (N4 - 1) * (M2 + M3 + M4); i++) {
        if ((i + 1 - kk) % (M2 + M3 + M4) == 0) {
            B.single(i, cc(i, 1), cc(i, 2), G_UPPER_WALL);
            continue;
        }
        B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    }
    for (int i = kk; i < kk + (N4 - 2) * (M2 + M3 + M4); i++) B.pair(i, i + (M2 + M3 + M4), cc(i, 2), cc(i, 3));
    kkk = kk + (N4 - 1) * (M2 + M3 + M4);
    for (int i = kkk; i < kkk + M1 + M2 + M3 + M4 - 2; i++) B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    for (int i = kkk; i < kkk + M1 + M2 + M3 + M4 - 1; i++) B.pair(i, n * (N1 - 2) + i - kkk, cc(i, 0), cc(i, 1));
    for (int i = kkk; i < kkk + M1 + M2 + M3 + M4 - 1; i++) B.pair(i, n * (N1 - 1) + i - kkk, cc(i, 2), cc(i, 3));
    kkkk = n * (N2 + N1 - 2);
    for (int i = kkkk; i < kkkk + M1 - 1; i++) B.pair(i, i - n, cc(i, 0), cc(i, 1));
    for (int i = ncells0 - M2 - M3 - M4; i < ncells0 - 1; i++) B.pair(i, i + 1, cc(i, 1), cc(i, 2));
    for (int i = ncells0 - M2 - M3 - M4; i < ncells0; i++)
        B.pair(i, kk + i - ncells0 + M2 + M3 + M4, cc(i, 2), cc(i, 3));
    for (int i = ncells0 - M2 - M3 - M4; i < ncells0; i++)
        B.pair(i, kkkk + M1 - n + i - (ncells0 - M2 - M3 - M4) - 1, cc(i, 0), cc(i, 1));
    {
        int K = ncells0 - M2 - M3 - M4;
        B.pair(K, kkkk + M1 - 1, cc(K, 3), cc(K, 0));
    }
    for (int i = kkkk + M1; i < kkkk + M1 + N4 - 1; i++)
        B.pair(i, kk + (i - kkkk - M1) * (M2 + M3 + M4), cc(i, 0), cc(i, 1));

    // Axis faces, Setka.cpp:710-742: twin has no Master and Sosed = K.
    auto axis = [&](int K, int a, int b) {
        int G = B.add_main(a, b, G_AXIS);
        int G2 = B.add_copy(b, a, G_AXIS);
        B.cells[K].grans.push_back(G);
        B.ref(G).master = K;
        B.ref(G2).master = -1;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
        B.ref(G2).sosed = K;
    };
    for (int i = 0; i < M1 + M2 + M3 + M4 - 1; i++) axis(i, cc(i, 0), cc(i, 1));
    for (int i = n * (N2 + N1 - 2) + (N3 - 2) * (N4 + M1 - 1); i < n * (N2 + N1 - 2) + (N3 - 1) * (N4 + M1 - 1); i++)
        axis(i, cc(i, 2), cc(i, 3));

    // Inner sphere faces, Setka.cpp:745-762: twin belongs to the central cell.
    auto inner = [&](int K) {
        int G = B.add_main(cc(K, 3), cc(K, 0), G_INNER_SPHERE);
        int G2 = B.add_copy(cc(K, 0), cc(K, 3), G_INNER_SPHERE);
        B.cells[K].grans.push_back(G);
        centr_grans.push_back(G2);
        B.ref(G).master = K;
        B.ref(G2).master = -1;  // the central fan cell, assigned below
        B.ref(G).sosed = -1;
        B.ref(G2).sosed = K;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
    };
    for (int i = 0; i < N1 + N2 - 2; i++) inner(i * (M1 + M2 + M3 + M4 - 1));
    // Upper-wall seam faces with twins, Setka.cpp:765-796
    auto upper = [&](int K) {
        int G = B.add_main(cc(K, 1), cc(K, 2), G_UPPER_WALL);
        int G2 = B.add_copy(cc(K, 2), cc(K, 1), G_UPPER_WALL);
        B.cells[K].grans.push_back(G);
        B.ref(G).master = K;
        B.ref(G2).sosed = K;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
    };
    upper(kkk + M1 + M2 + M3 + M4 - 2);
    upper(ncells0 - 1);
    {
        int h = (N1 + N2 - 2) * (M1 + M2 + M3 + M4 - 1);  // Setka.cpp:800-818
        for (int i = 0; i < N3 - 1; i++) inner(i * (M1 + N4 - 1) + h);
    }
    inner(kkk);  // Setka.cpp:820-835
    for (int i = kk + (N4 - 2) * (M2 + M3 + M4); i < kk + (N4 - 1) * (M2 + M3 + M4); i++) {  // 837-851
        int G = B.add_main(cc(i, 2), cc(i, 3), G_EXTERN);
        int G2 = B.add_copy(cc(i, 3), cc(i, 2), G_EXTERN);
        B.ref(G2).main_gran = true;
        B.cells[i].grans.push_back(G);
        B.ref(G).master = i;
        B.ref(G2).sosed = i;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
    }

    // Cell types, Setka.cpp:853-876
    for (auto& K : B.cells) {
        const int t0 = B.pt[K.contour[0]], t1 = B.pt[K.contour[1]], t2 = B.pt[K.contour[2]],
                  t3 = B.pt[K.contour[3]];
        if (t0 == P_INNER_BOUNDARY || t0 == P_U_1) K.type = C_1;
        else if (t3 == P_U_2 || t2 == P_U_2) K.type = C_2;
        if (t0 == P_U_3 || t1 == P_U_3 || t2 == P_U_3) K.type = C_3;
        else if (t0 == P_U_4 || t1 == P_U_4 || t2 == P_U_4) K.type = C_4;
        else if (t0 == P_U_5 || t1 == P_U_5 || t2 == P_U_5) K.type = C_5;
    }

    // Central fan cells, Setka.cpp:879-995
    {
        auto fc_angle = [&](int t) {
            const Face& F = B.ref(t);
            return polar_angle((B.px[F.A] + B.px[F.B]) / 2.0, (B.py[F.A] + B.py[F.B]) / 2.0);
        };
        std::sort(centr_grans.begin(), centr_grans.end(), [&](int a, int b) { return fc_angle(a) < fc_angle(b); });
        int kl = 8;
        while (centr_grans.size() % kl != 0) kl++;
        const int how = static_cast<int>(centr_grans.size()) / kl;
        std::vector<int> centr;
        for (int i = 0; i < kl; i++) {
            CellB A;
            A.type = C_CENTR;
            B.cells.push_back(A);
            int id = static_cast<int>(B.cells.size()) - 1;
            for (int j = i * how; j < (i + 1) * how; j++) {
                int g = centr_grans[j];
                B.cells[id].grans.push_back(g);
                B.ref(g).master = id;
                B.ref(B.ref(g).copy).sosed = id;
            }
            centr.push_back(id);
        }
        const int O = B.point(0.0, 0.0);
        B.pt[O] = P_NULL;
        for (int id : centr) {
            CellB& K = B.cells[id];
            K.contour.push_back(O);
            for (int g : K.grans) K.contour.push_back(B.ref(g).A);
            K.contour.push_back(B.ref(K.grans[K.grans.size() - 1]).B);
        }
        for (size_t i = 0; i + 1 < centr.size(); i++) {
            int K = centr[i];
            int vm = static_cast<int>(B.cells[K].contour.size());
            B.pair(K, centr[i + 1], B.cells[K].contour[vm - 1], B.cells[K].contour[0]);
        }
        {
            int PO = centr[0];
            int G2 = B.add_main(B.cells[PO].contour[0], B.cells[PO].contour[1], G_AXIS);
            int G3 = B.add_copy(B.cells[PO].contour[1], B.cells[PO].contour[0], G_AXIS);
            B.cells[PO].grans.push_back(G2);
            B.ref(G2).master = PO;
            B.ref(G3).sosed = PO;
            B.ref(G3).copy = G2;
            B.ref(G2).copy = G3;
        }
        {
            int PO = centr[centr.size() - 1];
            const int last = static_cast<int>(B.cells[PO].contour.size()) - 1;
            int G2 = B.add_main(B.cells[PO].contour[last], B.cells[PO].contour[0], G_AXIS);
            int G3 = B.add_copy(B.cells[PO].contour[0], B.cells[PO].contour[last], G_AXIS);
            B.cells[PO].grans.push_back(G2);
            B.ref(G2).master = PO;
            B.ref(G3).sosed = PO;
            B.ref(G3).copy = G2;
            B.ref(G2).copy = G3;
        }
    }

    // Rails in the order A, B, C, D
    std::vector<Rail*> rails;
    for (auto& R : Ar) rails.push_back(&R);
    for (auto& R : Br) rails.push_back(&R);
    for (auto& R : Cr) rails.push_back(&R);
    for (auto& R : Dr) rails.push_back(&R);
    finalize(B, *m, rails);

    // Tracked lines, Setka.cpp:1006-1049 (sorted by the polar angle of the face centre)
    auto face_angle = [&](int f) {
        return polar_angle((m->x[m->fA[f]] + m->x[m->fB[f]]) / 2.0, (m->y[m->fA[f]] + m->y[m->fB[f]]) / 2.0);
    };
    for (int f = 0; f < m->n_main; f++) {
        const int ta = m->ptype[m->fA[f]], tb = m->ptype[m->fB[f]];
        if (ta == P_CONTACT && tb == P_CONTACT) m->lcontact.push_back(f);
        if (ta == P_INNER_SHOCK && tb == P_INNER_SHOCK) m->linner.push_back(f);
        if (ta == P_OUTER_SHOCK && tb == P_OUTER_SHOCK) m->louter.push_back(f);
    }
    auto by_angle = [&](int a, int b) { return face_angle(a) < face_angle(b); };
    std::sort(m->lcontact.begin(), m->lcontact.end(), by_angle);
    std::sort(m->linner.begin(), m->linner.end(), by_angle);
    std::sort(m->louter.begin(), m->louter.end(), by_angle);
    return m;
}

extern "C" gelios_mesh* gelios_mesh_build_polar(int n_theta, int n_r, double r_in, double r_out) {
    if (n_theta < 2 || n_r < 2 || !(r_in > 0.0) || !(r_out > r_in)) {
        gelios::set_error("gelios_mesh_build_polar: bad arguments");
        return nullptr;
    }
    auto* m = new gelios_mesh();
    Builder B;
    // points: ray-major, ray i at theta_i = i*pi/n_theta, radius r_j log-spaced
    std::vector<std::vector<int>> P(n_theta + 1, std::vector<int>(n_r + 1));
    const double q = std::log(r_out / r_in);
    for (int i = 0; i <= n_theta; i++) {
        const double th = i * kPi / n_theta;
        for (int j = 0; j <= n_r; j++) {
            const double r = (j == n_r) ? r_out : r_in * std::exp(q * j / n_r);
            const int k = B.point(r * std::cos(th), r * std::sin(th));
            B.pt[k] = (j == 0) ? P_INNER_BOUNDARY : (j == n_r ? P_OUTER_BOUNDARY : P_USUALY);
        }
        for (int j = 0; j <= n_r; j++) P[i][j] = i * (n_r + 1) + j;
    }
    // cells: strip-major, same contour convention as Setka.cpp:202-203
    for (int i = 0; i < n_theta; i++)
        for (int j = 0; j < n_r; j++) {
            int c = B.cell(P[i][j], P[i][j + 1], P[i + 1][j + 1], P[i + 1][j]);
            B.cells[c].type = C_2;
        }
    auto cc = [&](int K, int k) { return B.cells[K].contour[k]; };
    // radial links + outer boundary (Input upstream, Extern downstream)
    for (int i = 0; i < n_theta; i++)
        for (int j = 0; j < n_r; j++) {
            const int c = i * n_r + j;
            if (j == n_r - 1) {
                B.single(c, cc(c, 1), cc(c, 2), (2 * i + 1 < n_theta) ? G_INPUT : G_EXTERN);
                continue;
            }
            B.pair(c, c + 1, cc(c, 1), cc(c, 2));
        }
    // angular links
    for (int i = 0; i + 1 < n_theta; i++)
        for (int j = 0; j < n_r; j++) {
            const int c = i * n_r + j;
            B.pair(c, c + n_r, cc(c, 2), cc(c, 3));
        }
    // symmetry axis on both rays (twins without Master, like Setka.cpp:710-742)
    auto axis = [&](int K, int a, int b) {
        int G = B.add_main(a, b, G_AXIS);
        int G2 = B.add_copy(b, a, G_AXIS);
        B.cells[K].grans.push_back(G);
        B.ref(G).master = K;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
        B.ref(G2).sosed = K;
    };
    for (int j = 0; j < n_r; j++) axis(j, cc(j, 0), cc(j, 1));
    for (int j = 0; j < n_r; j++) {
        const int c = (n_theta - 1) * n_r + j;
        axis(c, cc(c, 2), cc(c, 3));
    }
    // inner sphere (no central cell: the twin has neither Master nor Sosed cell)
    for (int i = 0; i < n_theta; i++) {
        const int c = i * n_r;
        int G = B.add_main(cc(c, 3), cc(c, 0), G_INNER_SPHERE);
        int G2 = B.add_copy(cc(c, 0), cc(c, 3), G_INNER_SPHERE);
        B.cells[c].grans.push_back(G);
        B.ref(G).master = c;
        B.ref(G).copy = G2;
        B.ref(G2).copy = G;
        B.ref(G2).sosed = c;
    }
    finalize(B, *m, {});
    return m;
}

extern "C" int gelios_mesh_tvd_prepare(gelios_mesh* m) {
    if (!m) {
        gelios::set_error("gelios_mesh_tvd_prepare: null mesh");
        return GELIOS_E_ARG;
    }
    const int nf = static_cast<int>(m->fA.size());
    const int nm = m->n_main;
    const int ncell = static_cast<int>(m->ctype.size());
    const bool uniq = m->unique_face_numbers != 0;
    auto number = [&](int f) { return (uniq || f < nm) ? f : f - nm; };  // Gran::number
    auto cell_center = [&](int k, double& ox, double& oy) {  // Cell::Get_Center, Cell.cpp:66-88
        const int s = m->cstart[k], e = m->cstart[k + 1], n = e - s;
        double A = 0.0, Gx = 0.0, Gy = 0.0;
        for (int i = 0; i < n; i++) {
            const int a = m->contour[s + i];
            int j = i + 1;
            if (j == n) j = 0;
            const int b = m->contour[s + j];
            A = A + (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
            Gx = Gx + (m->x[a] + m->x[b]) * (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
            Gy = Gy + (m->y[a] + m->y[b]) * (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
        }
        A = A * 0.5;
        Gx = Gx / (6.0 * A);
        Gy = Gy / (6.0 * A);
        ox = Gx;
        oy = Gy;
    };
    auto face_center = [&](int f, double& ox, double& oy) {
        ox = (m->x[m->fA[f]] + m->x[m->fB[f]]) / 2.0;
        oy = (m->y[m->fA[f]] + m->y[m->fB[f]]) / 2.0;
    };
    m->fsup.assign(nf, -1);
    m->fsdown.assign(nf, -1);
    // Sosed_up of every face (main list then copies, Setka.cpp:1306-1410)
    for (int i = 0; i < nf; i++) {
        const int So = m->fsosed[i];
        if (So < 0) {
            m->fsup[i] = -1;
            continue;
        }
        double x3, y3, x, y, x1, y1;
        cell_center(So, x3, y3);
        face_center(i, x, y);
        double n1 = x3 - x, n2 = y3 - y;
        double n = std::sqrt(sq(n1) + sq(n2));
        n1 = n1 / n;
        n2 = n2 / n;
        double N = -1.0;
        int Bf = -1;
        for (int g = m->gstart[So]; g < m->gstart[So + 1]; g++) {
            const int j = m->gran[g];
            if (m->ftype[j] == G_USUALY) {
                if (number(m->fcopy[j]) == number(i)) continue;
            }
            face_center(j, x1, y1);
            double a = x1 - x3, b = y1 - y3;
            n = std::sqrt(sq(a) + sq(b));
            a = a / n;
            b = b / n;
            if (a * n1 + b * n2 > N) {
                N = a * n1 + b * n2;
                Bf = j;
            }
        }
        if (Bf < 0) {
            gelios::set_error("gelios_mesh_tvd_prepare: no candidate face");
            return GELIOS_E_MESH;
        }
        m->fsup[i] = m->fsosed[Bf] >= 0 ? m->fsosed[Bf] : -1;
    }
    for (int i = 0; i < nf; i++) m->fsdown[i] = m->fcopy[i] >= 0 ? m->fsup[m->fcopy[i]] : -1;
    // radial source chains, Setka.cpp:1438-1489
    for (int k = 0; k < ncell; k++) {
        double xx, yy;
        cell_center(k, xx, yy);
        m->r_istoch[k] = std::sqrt(sq(xx) + sq(yy));
        if (xx >= 0.0) {
            const double a1 = xx / m->r_istoch[k];
            const double a2 = yy / m->r_istoch[k];
            for (int g = m->gstart[k]; g < m->gstart[k + 1]; g++) {
                const int j = m->gran[g];
                const int So = m->fsosed[j];
                if (So < 0) continue;
                double xx2, yy2;
                cell_center(So, xx2, yy2);
                double n1 = (xx2 - xx), n2 = (yy2 - yy);
                const double nn = std::sqrt(sq(n1) + sq(n2));
                n1 = n1 / nn;
                n2 = n2 / nn;
                const double sk = a1 * n1 + a2 * n2;
                if (std::fabs(1.0 - sk) < 0.001) {
                    m->cnext[k] = So;
                    if (std::sqrt(sq(xx2) + sq(yy2)) < m->r_istoch[k]) {
                        gelios::set_error("gelios_mesh_tvd_prepare: outward chain link points inward");
                        return GELIOS_E_MESH;
                    }
                } else if (std::fabs(-1.0 - sk) < 0.001) {
                    m->cback[k] = So;
                    if (std::sqrt(sq(xx2) + sq(yy2)) > m->r_istoch[k]) {
                        gelios::set_error("gelios_mesh_tvd_prepare: inward chain link points outward");
                        return GELIOS_E_MESH;
                    }
                }
            }
        }
    }
    return GELIOS_OK;
}

extern "C" int gelios_mesh_inner_cells(const gelios_mesh* m, double r_max, int32_t* out, int32_t cap) {
    if (!m) return GELIOS_E_ARG;
    int cnt = 0;
    const int ncell = static_cast<int>(m->ctype.size());
    for (int k = 0; k < ncell; k++) {
        const int s = m->cstart[k], e = m->cstart[k + 1], n = e - s;
        double A = 0.0, Gx = 0.0, Gy = 0.0;
        for (int i = 0; i < n; i++) {
            const int a = m->contour[s + i];
            int j = i + 1;
            if (j == n) j = 0;
            const int b = m->contour[s + j];
            A = A + (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
            Gx = Gx + (m->x[a] + m->x[b]) * (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
            Gy = Gy + (m->y[a] + m->y[b]) * (m->x[a] * m->y[b] - m->y[a] * m->x[b]);
        }
        A = A * 0.5;
        const double x = Gx / (6.0 * A), y = Gy / (6.0 * A);
        if (std::sqrt(x * x + y * y) <= r_max) {
            if (out && cnt < cap) out[cnt] = k;
            cnt++;
        }
    }
    return cnt;
}

extern "C" int gelios_mesh_get_view(const gelios_mesh* m, gelios_mesh_view* v) {
    if (!m || !v) return GELIOS_E_ARG;
    std::memset(v, 0, sizeof(*v));
    std::memcpy(v->dims, m->dims, sizeof(v->dims));
    v->n_points = static_cast<int32_t>(m->x.size());
    v->x = m->x.data();
    v->y = m->y.data();
    v->point_type = m->ptype.data();
    v->n_cells = static_cast<int32_t>(m->ctype.size());
    v->cell_type = m->ctype.data();
    v->contour_start = m->cstart.data();
    v->contour = m->contour.data();
    v->gran_start = m->gstart.data();
    v->gran = m->gran.data();
    v->cell_back = m->cback.data();
    v->cell_next = m->cnext.data();
    v->r_istoch = m->r_istoch.data();
    v->n_faces = static_cast<int32_t>(m->fA.size());
    v->n_main = m->n_main;
    v->face_A = m->fA.data();
    v->face_B = m->fB.data();
    v->face_type = m->ftype.data();
    v->face_master = m->fmaster.data();
    v->face_sosed = m->fsosed.data();
    v->face_copy = m->fcopy.data();
    v->face_sosed_up = m->fsup.data();
    v->face_sosed_down = m->fsdown.data();
    v->n_rails = static_cast<int32_t>(m->rtype.size());
    v->rail_type = m->rtype.data();
    v->rail_s = m->rs.data();
    v->rail_M = m->rM.data();
    v->rail_pstart = m->rpstart.data();
    v->rail_points = m->rpts.data();
    v->rail_kstart = m->rkstart.data();
    v->rail_keys = m->rkeys.data();
    v->n_contact = static_cast<int32_t>(m->lcontact.size());
    v->n_inner_line = static_cast<int32_t>(m->linner.size());
    v->n_outer_line = static_cast<int32_t>(m->louter.size());
    v->line_contact = m->lcontact.data();
    v->line_inner = m->linner.data();
    v->line_outer = m->louter.data();
    return GELIOS_OK;
}

extern "C" void gelios_mesh_free(gelios_mesh* m) { delete m; }

extern "C" int gelios_tvd_prepare_view_numbered(const gelios_mesh_view* v, int unique_face_numbers,
                                                int32_t* sosed_up, int32_t* sosed_down, int32_t* back,
                                                int32_t* next, double* r_istoch) {
    if (!v || v->n_cells <= 0 || v->n_faces <= 0) {
        gelios::set_error("gelios_tvd_prepare_view: empty view");
        return GELIOS_E_ARG;
    }
    gelios_mesh* m = gelios::mesh_from_view(v);
    m->unique_face_numbers = unique_face_numbers ? 1 : 0;
    const int rc = gelios_mesh_tvd_prepare(m);
    if (rc == GELIOS_OK) {
        if (sosed_up) std::copy(m->fsup.begin(), m->fsup.end(), sosed_up);
        if (sosed_down) std::copy(m->fsdown.begin(), m->fsdown.end(), sosed_down);
        if (back) std::copy(m->cback.begin(), m->cback.end(), back);
        if (next) std::copy(m->cnext.begin(), m->cnext.end(), next);
        if (r_istoch) std::copy(m->r_istoch.begin(), m->r_istoch.end(), r_istoch);
    }
    delete m;
    return rc;
}

extern "C" int gelios_tvd_prepare_view(const gelios_mesh_view* v, int32_t* sosed_up, int32_t* sosed_down,
                                       int32_t* back, int32_t* next, double* r_istoch) {
    return gelios_tvd_prepare_view_numbered(v, 0, sosed_up, sosed_down, back, next, r_istoch);
}
