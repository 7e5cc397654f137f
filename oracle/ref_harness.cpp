// Test infrastructure only: a thin extern "C" harness around the UNMODIFIED
// reference sources of SergeyMSU/Gelios_2D (compiled by oracle/Makefile from
// the reference tree, never copied into this repository).  It lets the tests
// and the CPU-baseline leg of bench.py
//   * build grids with the reference's own Setka constructor
//     (Setka.cpp:19-1076) or instantiate reference Point/Cell/Gran/Rail
//     objects from flat arrays,
//   * run the reference steps Go_stationary (Setka.cpp:5205-5343),
//     Go_5_komponent__MK2 (Setka.cpp:10121-10482) and
//     Go_stationary_5_komponent_inner_MK2 (Setka.cpp:6999-7212),
//   * run the per-face solvers HLLC_2d_Korolkov_b_s (Setka.cpp:10484-10700),
//     Godunov_Solver_Alexashov (Solvers.cpp:693-1172), HLLDQ_Korolkov
//     (Solvers.cpp:1642-2185), HLLD_Solver_Alexashov (Solvers.cpp:92-691),
//   * export topology/state as flat arrays.
// Nothing in the product links or loads this file.
#include "Help.h"

#include <omp.h>
#include <unistd.h>
#include <cstdint>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <unordered_map>

namespace {

// The reference prints progress to std::cout and opens "file_work.txt" in the
// working directory from its constructor; keep both away from the caller.
struct Quiet {
    std::streambuf* old;
    std::ostringstream sink;
    Quiet() { old = std::cout.rdbuf(sink.rdbuf()); }
    ~Quiet() { std::cout.rdbuf(old); }
};

struct InTmpDir {
    char prev[4096];
    bool ok;
    InTmpDir() {
        ok = getcwd(prev, sizeof(prev)) != nullptr;
        const char* t = getenv("TMPDIR");
        if (chdir(t ? t : "/tmp") != 0) ok = false;
    }
    ~InTmpDir() {
        if (ok) { int rc = chdir(prev); (void)rc; }
    }
};

struct Handle {
    Setka* S = nullptr;
    // unified face numbering: main faces [0, n_main) in All_Gran order,
    // copies [n_main, n_main + n_copy) in All_Gran_copy order
    std::unordered_map<const Gran*, int> face_id;
    std::unordered_map<const Cell*, int> cell_id;
    std::unordered_map<const Point*, int> point_id;
    std::vector<Rail*> rails;  // A, B, C, D in order
    void index() {
        face_id.clear(); cell_id.clear(); point_id.clear(); rails.clear();
        int k = 0;
        for (auto g : S->All_Gran) face_id[g] = k++;
        for (auto g : S->All_Gran_copy) face_id[g] = k++;
        k = 0;
        for (auto c : S->All_Cells) cell_id[c] = k++;
        k = 0;
        for (auto p : S->All_Points) point_id[p] = k++;
        for (auto r : S->A_Rails) rails.push_back(r);
        for (auto r : S->B_Rails) rails.push_back(r);
        for (auto r : S->C_Rails) rails.push_back(r);
        for (auto r : S->D_Rails) rails.push_back(r);
    }
    int fid(const Gran* g) const {
        if (!g) return -1;
        auto it = face_id.find(g);
        return it == face_id.end() ? -2 : it->second;
    }
    int cid(const Cell* c) const {
        if (!c) return -1;
        auto it = cell_id.find(c);
        return it == cell_id.end() ? -2 : it->second;
    }
    int pid(const Point* p) const {
        if (!p) return -1;
        auto it = point_id.find(p);
        return it == point_id.end() ? -2 : it->second;
    }
};

void zero_params(Setka* S) {
    for (auto c : S->All_Cells) {
        c->par[0] = Parametr{};
        c->par[1] = Parametr{};
        for (int k = 0; k < 4; ++k) {
            for (int b = 0; b < 2; ++b) {
                Parametr& p = c->par[b];
                p.H_n[k] = p.H_u[k] = p.H_v[k] = p.H_T[k] = 0.0;
                p.H_n2[k] = p.H_u2[k] = p.H_v2[k] = p.H_T2[k] = 0.0;
                p.H_n3[k] = p.H_u3[k] = p.H_v3[k] = p.H_T3[k] = 0.0;
                p.num_atoms[k] = 0;
                p.I1_mf[k] = p.I2_mf[k] = p.I3_mf[k] = 0.0;
                p.I1_mc[k] = p.I2_mc[k] = p.I3_mc[k] = 0.0;
            }
            for (int w = 0; w < 7; ++w) c->par[0].w_m[w] = c->par[1].w_m[w] = 0.0;
        }
        for (int k = 0; k < 5; ++k) c->Potok[k] = 0.0;
        c->Back = nullptr;
        c->Next = nullptr;
        c->r_istoch = 0.0;
    }
}

Setka* g_dummy = nullptr;
Setka* dummy() {
    if (!g_dummy) {
        Quiet q;
        InTmpDir t;
        g_dummy = new Setka();
    }
    return g_dummy;
}

}  // namespace

extern "C" {

// OpenMP threads of the reference loops (1 for parity runs: the reference's
// multithreaded dt reduction is racy, Setka.cpp:10141, 10359-10393).
void gref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int gref_max_threads(void) { return omp_get_num_procs(); }

// ---------------------------------------------------------------- lifecycle
void* gref_setka_new(int N1, int N2, int N3, int N4, int M1, int M2, int M3, int M4) {
    Quiet q;
    InTmpDir t;
    auto* h = new Handle();
    h->S = new Setka(N1, N2, N3, N4, M1, M2, M3, M4);
    zero_params(h->S);
    h->index();
    return h;
}

// Setka::Save_Setka_ALL_ALPHA (Setka.cpp:2355-2574) of a grid to a text file.
void gref_save_alpha(void* hv, const char* path) {
    Quiet q;
    auto* h = static_cast<Handle*>(hv);
    h->S->Save_Setka_ALL_ALPHA(std::string(path));
}

// A fresh Setka filled by Setka::Download_Setka_ALL_ALPHA_2_0
// (Setka.cpp:2899-3257).  The loader leaves the source chains unset; they
// start empty, as after the constructor.
void* gref_load_alpha(const char* path) {
    Quiet q;
    auto* h = new Handle();
    h->S = new Setka();
    h->S->Download_Setka_ALL_ALPHA_2_0(std::string(path));
    for (auto c : h->S->All_Cells) {
        c->Back = nullptr;
        c->Next = nullptr;
        c->r_istoch = 0.0;
        for (int k = 0; k < 5; ++k) c->Potok[k] = 0.0;
    }
    h->index();
    return h;
}

// Instantiates reference objects from flat arrays (same layout as the export).
// dims: N1..M4 of the Setka these arrays describe (used by Move_surface /
// Move_Setka_Calculate_2), or zeros for a grid without rails.
void* gref_setka_from_arrays(const int* dims8,
                             int n_points, const double* x, const double* y, const int* ptype,
                             int n_cells, const int* ctype, const int* contour_start, const int* contour,
                             const int* gran_start, const int* gran,
                             int n_main, int n_copy, const int* fA, const int* fB, const int* ftype,
                             const int* fmaster, const int* fsosed, const int* fcopy, const int* fmain,
                             int n_rails, const int* rtype, const double* rs, const int* rM,
                             const int* rp_start, const int* rpts, const int* rk_start, const int* rkeys,
                             int n_lc, const int* lcontact, int n_li, const int* linner,
                             int n_lo, const int* louter) {
    Quiet q;
    InTmpDir t;
    auto* h = new Handle();
    Setka* S = new Setka();
    h->S = S;
    S->N1 = dims8[0]; S->N2 = dims8[1]; S->N3 = dims8[2]; S->N4 = dims8[3];
    S->M1 = dims8[4]; S->M2 = dims8[5]; S->M3 = dims8[6]; S->M4 = dims8[7];
    std::vector<Point*> vp(n_points);
    for (int i = 0; i < n_points; ++i) {
        vp[i] = new Point(x[i], y[i]);
        vp[i]->type = static_cast<Point_type>(ptype[i]);
        vp[i]->number = i;
        S->All_Points.push_back(vp[i]);
    }
    std::vector<Cell*> vc(n_cells);
    for (int c = 0; c < n_cells; ++c) {
        vc[c] = new Cell();
        vc[c]->type = static_cast<Cell_type>(ctype[c]);
        vc[c]->number = c;
        for (int k = contour_start[c]; k < contour_start[c + 1]; ++k) {
            vc[c]->contour.push_back(vp[contour[k]]);
            vp[contour[k]]->my_cell.push_back(vc[c]);
        }
        S->All_Cells.push_back(vc[c]);
    }
    const int nf = n_main + n_copy;
    std::vector<Gran*> vg(nf);
    for (int f = 0; f < nf; ++f) {
        vg[f] = new Gran(vp[fA[f]], vp[fB[f]], static_cast<Gran_type>(ftype[f]));
        vg[f]->number = f < n_main ? f : f - n_main;
        vg[f]->main_gran = fmain[f] != 0;
    }
    for (int f = 0; f < nf; ++f) {
        vg[f]->Master = fmaster[f] >= 0 ? vc[fmaster[f]] : nullptr;
        vg[f]->Sosed = fsosed[f] >= 0 ? vc[fsosed[f]] : nullptr;
        vg[f]->Gran_copy = fcopy[f] >= 0 ? vg[fcopy[f]] : nullptr;
        if (f < n_main) S->All_Gran.push_back(vg[f]);
        else S->All_Gran_copy.push_back(vg[f]);
    }
    for (int c = 0; c < n_cells; ++c)
        for (int k = gran_start[c]; k < gran_start[c + 1]; ++k) vc[c]->Grans.push_back(vg[gran[k]]);
    for (int r = 0; r < n_rails; ++r) {
        auto* R = new Rail(rs[r]);
        R->type = static_cast<Rail_type>(rtype[r]);
        R->M1 = rM[4 * r + 0]; R->M2 = rM[4 * r + 1]; R->M3 = rM[4 * r + 2]; R->M4 = rM[4 * r + 3];
        for (int k = rp_start[r]; k < rp_start[r + 1]; ++k) R->All_point.push_back(vp[rpts[k]]);
        for (int k = rk_start[r]; k < rk_start[r + 1]; ++k) R->Key_point.push_back(vp[rkeys[k]]);
        switch (R->type) {
            case A: S->A_Rails.push_back(R); break;
            case B: S->B_Rails.push_back(R); break;
            case C: S->C_Rails.push_back(R); break;
            default: S->D_Rails.push_back(R); break;
        }
    }
    for (int i = 0; i < n_lc; ++i) S->Line_Contact.push_back(vg[lcontact[i]]);
    for (int i = 0; i < n_li; ++i) S->Line_Inner.push_back(vg[linner[i]]);
    for (int i = 0; i < n_lo; ++i) S->Line_Outer.push_back(vg[louter[i]]);
    zero_params(S);
    h->index();
    return h;
}

// ---------------------------------------------------------------- queries
// out[0..12] = n_points, n_cells, n_main, n_copy, contour_total, gran_total,
//              n_rails, rail_points_total, rail_keys_total, n_contact, n_inner,
//              n_outer, n_cells_inner
void gref_counts(void* hv, int64_t* out) {
    auto* h = static_cast<Handle*>(hv);
    Setka* S = h->S;
    int64_t ct = 0, gt = 0, rp = 0, rk = 0;
    for (auto c : S->All_Cells) { ct += c->contour.size(); gt += c->Grans.size(); }
    for (auto r : h->rails) { rp += r->All_point.size(); rk += r->Key_point.size(); }
    out[0] = S->All_Points.size();
    out[1] = S->All_Cells.size();
    out[2] = S->All_Gran.size();
    out[3] = S->All_Gran_copy.size();
    out[4] = ct;
    out[5] = gt;
    out[6] = h->rails.size();
    out[7] = rp;
    out[8] = rk;
    out[9] = S->Line_Contact.size();
    out[10] = S->Line_Inner.size();
    out[11] = S->Line_Outer.size();
    out[12] = S->All_Cells_Inner.size();
}

void gref_export_points(void* hv, double* x, double* y, double* x2, double* y2, int* type) {
    auto* h = static_cast<Handle*>(hv);
    int i = 0;
    for (auto p : h->S->All_Points) {
        x[i] = p->x; y[i] = p->y; x2[i] = p->x2; y2[i] = p->y2; type[i] = p->type;
        ++i;
    }
}

void gref_export_cells(void* hv, int* type, int* contour_start, int* contour, int* gran_start,
                       int* gran, int* back, int* next, double* r_istoch) {
    auto* h = static_cast<Handle*>(hv);
    int c = 0, kc = 0, kg = 0;
    contour_start[0] = 0;
    gran_start[0] = 0;
    for (auto K : h->S->All_Cells) {
        type[c] = K->type;
        for (auto p : K->contour) contour[kc++] = h->pid(p);
        for (auto g : K->Grans) gran[kg++] = h->fid(g);
        contour_start[c + 1] = kc;
        gran_start[c + 1] = kg;
        back[c] = h->cid(K->Back);
        next[c] = h->cid(K->Next);
        r_istoch[c] = K->r_istoch;
        ++c;
    }
}

void gref_export_faces(void* hv, int* A, int* B, int* type, int* master, int* sosed, int* copy,
                       int* sosed_up, int* sosed_down, int* main_flag) {
    auto* h = static_cast<Handle*>(hv);
    int f = 0;
    auto one = [&](Gran* g) {
        A[f] = h->pid(g->A); B[f] = h->pid(g->B); type[f] = g->type;
        master[f] = h->cid(g->Master); sosed[f] = h->cid(g->Sosed); copy[f] = h->fid(g->Gran_copy);
        sosed_up[f] = h->cid(g->Sosed_up); sosed_down[f] = h->cid(g->Sosed_down);
        main_flag[f] = g->main_gran ? 1 : 0;
        ++f;
    };
    for (auto g : h->S->All_Gran) one(g);
    for (auto g : h->S->All_Gran_copy) one(g);
}

void gref_export_rails(void* hv, int* type, double* s, int* M, int* p_start, int* pts, int* k_start, int* keys) {
    auto* h = static_cast<Handle*>(hv);
    int r = 0, kp = 0, kk = 0;
    p_start[0] = 0;
    k_start[0] = 0;
    for (auto R : h->rails) {
        type[r] = R->type; s[r] = R->s;
        M[4 * r + 0] = R->M1; M[4 * r + 1] = R->M2; M[4 * r + 2] = R->M3; M[4 * r + 3] = R->M4;
        for (auto p : R->All_point) pts[kp++] = h->pid(p);
        for (auto p : R->Key_point) keys[kk++] = h->pid(p);
        p_start[r + 1] = kp;
        k_start[r + 1] = kk;
        ++r;
    }
}

void gref_export_lines(void* hv, int* contact, int* inner, int* outer) {
    auto* h = static_cast<Handle*>(hv);
    int i = 0;
    for (auto g : h->S->Line_Contact) contact[i++] = h->fid(g);
    i = 0;
    for (auto g : h->S->Line_Inner) inner[i++] = h->fid(g);
    i = 0;
    for (auto g : h->S->Line_Outer) outer[i++] = h->fid(g);
}

void gref_export_inner_list(void* hv, int* cells) {
    auto* h = static_cast<Handle*>(hv);
    int i = 0;
    for (auto c : h->S->All_Cells_Inner) cells[i++] = h->cid(c);
}

// Sosed_up/Sosed_down/Back/Next/r_istoch: Setka::TVD_prepare (Setka.cpp:1294-1492)
void gref_tvd_prepare(void* hv) {
    Quiet q;
    static_cast<Handle*>(hv)->S->TVD_prepare();
}

// Setka::Init_conditions (Setka.cpp:5149-5203)
void gref_init_conditions(void* hv) {
    Quiet q;
    static_cast<Handle*>(hv)->S->Init_conditions();
}

// All_Cells_Inner as built by main (Gelios_2D.cpp:152-231): cells whose centroid
// radius is <= R111_, in All_Cells order; All_Cells_zero = the C_centr cells.
void gref_build_inner_list(void* hv) {
    Setka* S = static_cast<Handle*>(hv)->S;
    S->All_Cells_Inner.clear();
    S->All_Cells_zero.clear();
    for (auto i : S->All_Cells) {
        double x, y;
        i->Get_Center(x, y);
        if (sqrt(x * x + y * y) <= R111_) S->All_Cells_Inner.push_back(i);
        if (i->type == C_centr) S->All_Cells_zero.push_back(i);
    }
}

// ---------------------------------------------------------------- state
void gref_set_state(void* hv, int buf, const double* ro, const double* p, const double* u,
                    const double* v, const double* Q) {
    int c = 0;
    for (auto K : static_cast<Handle*>(hv)->S->All_Cells) {
        Parametr& P = K->par[buf];
        P.ro = ro[c]; P.p = p[c]; P.u = u[c]; P.v = v[c]; P.Q = Q[c];
        ++c;
    }
}

void gref_get_state(void* hv, int buf, double* ro, double* p, double* u, double* v, double* Q) {
    int c = 0;
    for (auto K : static_cast<Handle*>(hv)->S->All_Cells) {
        const Parametr& P = K->par[buf];
        ro[c] = P.ro; p[c] = P.p; u[c] = P.u; v[c] = P.v; Q[c] = P.Q;
        ++c;
    }
}

// Monte-Carlo moments left in par[0] by MK_start_new (Setka.cpp:12241-12449):
// H_n/H_u/H_v/H_T [cell][4] and k_u/k_v/k_T [cell].
void gref_set_mc(void* hv, const double* Hn, const double* Hu, const double* Hv, const double* HT,
                 const double* ku, const double* kv_, const double* kT) {
    int c = 0;
    for (auto K : static_cast<Handle*>(hv)->S->All_Cells) {
        Parametr& P = K->par[0];
        for (int k = 0; k < 4; ++k) {
            P.H_n[k] = Hn[4 * c + k]; P.H_u[k] = Hu[4 * c + k];
            P.H_v[k] = Hv[4 * c + k]; P.H_T[k] = HT[4 * c + k];
        }
        P.k_u = ku[c]; P.k_v = kv_[c]; P.k_T = kT[c];
        ++c;
    }
}

void gref_get_point_motion(void* hv, double* x, double* y, double* x2, double* y2, double* Vx,
                           double* Vy, int* count) {
    int i = 0;
    for (auto p : static_cast<Handle*>(hv)->S->All_Points) {
        x[i] = p->x; y[i] = p->y; x2[i] = p->x2; y2[i] = p->y2;
        Vx[i] = p->Vx; Vy[i] = p->Vy; count[i] = p->count;
        ++i;
    }
}

void gref_set_points(void* hv, const double* x, const double* y) {
    int i = 0;
    for (auto p : static_cast<Handle*>(hv)->S->All_Points) {
        p->x = p->x2 = x[i];
        p->y = p->y2 = y[i];
        p->Vx = p->Vy = 0.0;
        p->count = 0;
        ++i;
    }
}

// ---------------------------------------------------------------- steps
void gref_go_stationary(void* hv, int steps) {
    Quiet q;
    static_cast<Handle*>(hv)->S->Go_stationary(steps);
}

void gref_go_mk2(void* hv, int steps) {
    Quiet q;
    static_cast<Handle*>(hv)->S->Go_5_komponent__MK2(steps);
}

// Hydrogen fluids of par[buf]: rows16 = ro, p, u, v of H1..H4, each n_cells long.
void gref_set_hydrogen(void* hv, int buf, const double* rows16) {
    auto* h = static_cast<Handle*>(hv);
    const size_t n = h->S->All_Cells.size();
    for (size_t k = 0; k < n; ++k) {
        Parametr& p = h->S->All_Cells[k]->par[buf];
        double* f[16] = {&p.ro_H1, &p.p_H1, &p.u_H1, &p.v_H1, &p.ro_H2, &p.p_H2, &p.u_H2, &p.v_H2,
                         &p.ro_H3, &p.p_H3, &p.u_H3, &p.v_H3, &p.ro_H4, &p.p_H4, &p.u_H4, &p.v_H4};
        for (int q = 0; q < 16; ++q) *f[q] = rows16[q * n + k];
    }
}

void gref_get_hydrogen(void* hv, int buf, double* rows16) {
    auto* h = static_cast<Handle*>(hv);
    const size_t n = h->S->All_Cells.size();
    for (size_t k = 0; k < n; ++k) {
        const Parametr& p = h->S->All_Cells[k]->par[buf];
        const double f[16] = {p.ro_H1, p.p_H1, p.u_H1, p.v_H1, p.ro_H2, p.p_H2, p.u_H2, p.v_H2,
                              p.ro_H3, p.p_H3, p.u_H3, p.v_H3, p.ro_H4, p.p_H4, p.u_H4, p.v_H4};
        for (int q = 0; q < 16; ++q) rows16[q * n + k] = f[q];
    }
}

// Setka::Go_5_komponent (Setka.cpp:8269-8950)
void gref_go_5_komponent(void* hv, int steps) {
    Quiet q;
    static_cast<Handle*>(hv)->S->Go_5_komponent(steps);
}

void gref_go_inner_mk2(void* hv, int steps) {
    Quiet q;
    static_cast<Handle*>(hv)->S->Go_stationary_5_komponent_inner_MK2(steps);
}

void gref_move_surface(void* hv, int ii, double dt) {
    static_cast<Handle*>(hv)->S->Move_surface(ii, dt);
}

void gref_move_setka2(void* hv, double dt) {
    static_cast<Handle*>(hv)->S->Move_Setka_Calculate_2(dt);
}

// Get_par (which=0, Gran.cpp:205-289), Get_par_TVD (1, Gran.cpp:292-559),
// Get_par_TVD_radial (2, Gran.cpp:562-675) for unified face id f from par[ii].
// out = ro, p, u, v, Q
void gref_face_par(void* hv, int f, int which, int ii, double* out) {
    auto* h = static_cast<Handle*>(hv);
    Setka* S = h->S;
    const int nm = static_cast<int>(S->All_Gran.size());
    Gran* g = f < nm ? S->All_Gran[f] : S->All_Gran_copy[f - nm];
    Parametr par;
    if (which == 0) g->Get_par(par, ii);
    else if (which == 1) g->Get_par_TVD(par, ii);
    else g->Get_par_TVD_radial(par, ii);
    out[0] = par.ro; out[1] = par.p; out[2] = par.u; out[3] = par.v; out[4] = par.Q;
}

// Geometry of cell c: out = Get_Center x,y (Cell.cpp:66-88), Get_Center_posle
// x,y (90-111), Get_Volume (146-186), Get_Volume_posle (208-254),
// Get_Volume_rotate(360)/2pi (188-206), Get_Volume_posle_rotate(360)/2pi (256-275)
void gref_cell_geom(void* hv, int c, double* out) {
    Cell* K = static_cast<Handle*>(hv)->S->All_Cells[c];
    K->Get_Center(out[0], out[1]);
    K->Get_Center_posle(out[2], out[3]);
    out[4] = K->Get_Volume();
    out[5] = K->Get_Volume_posle();
    out[6] = K->Get_Volume_rotate(360.0) / (2.0 * pi_);
    out[7] = K->Get_Volume_posle_rotate(360.0) / (2.0 * pi_);
}

// Cell::Get_Sourse_MK1 (Cell.cpp:498-665) with the given plasma state.
void gref_source_mk1(void* hv, int c, double u, double v, double ro, double p, double* q3) {
    Cell* K = static_cast<Handle*>(hv)->S->All_Cells[c];
    K->Get_Sourse_MK1(q3[0], q3[1], q3[2], u, v, ro, p);
}

// ---------------------------------------------------------------- per-face KATs
double gref_hllc(double ro_L, double Q_L, double p_L, double v1_L, double v2_L, double ro_R, double Q_R,
                 double p_R, double v1_R, double v2_R, double W, double* P, double* PQ, double n1,
                 double n2, double rad, int metod, double* VlVcVp, int nul_potok) {
    double pq = 0.0, Vl = 0.0, Vc = 0.0, Vp = 0.0;
    double t = dummy()->HLLC_2d_Korolkov_b_s(ro_L, Q_L, p_L, v1_L, v2_L, ro_R, Q_R, p_R, v1_R, v2_R, W, P, pq,
                                              n1, n2, rad, metod, Vl, Vc, Vp, nul_potok != 0);
    *PQ = pq;
    VlVcVp[0] = Vl; VlVcVp[1] = Vc; VlVcVp[2] = Vp;
    return t;
}

// q1, q2 = (ro, p, u, v, w); n[3]; out q[5]; dsl_dsp_dsc[3]
double gref_godunov(const double* q1, const double* q2, const double* n, double* q, double* dsl_dsp_dsc,
                    double w, double dist) {
    Solvers S;
    std::vector<double> a(q1, q1 + 5), b(q2, q2 + 5), nn(n, n + 3), out(5);
    double dsl = 0, dsp = 0, dsc = 0;
    double t = S.Godunov_Solver_Alexashov(a, b, nn, out, dsl, dsp, dsc, w, dist);
    for (int k = 0; k < 5; ++k) q[k] = out[k];
    dsl_dsp_dsc[0] = dsl; dsl_dsp_dsc[1] = dsp; dsl_dsp_dsc[2] = dsc;
    return t;
}

// L[9], R[9] = (ro, Q, p, v1, v2, v3, Bx, By, Bz); P[8]; n[3]
double gref_hlldq(const double* L, const double* R, double* P, double* PQ, const double* n, double rad,
                  int metod) {
    Solvers S;
    double pq = 0.0;
    double t = S.HLLDQ_Korolkov(L[0], L[1], L[2], L[3], L[4], L[5], L[6], L[7], L[8], R[0], R[1], R[2], R[3],
                                R[4], R[5], R[6], R[7], R[8], P, pq, n[0], n[1], n[2], rad, metod);
    *PQ = pq;
    return t;
}

// q1, q2 = (ro, p, u, v, w, bx, by, bz); n[3]; out q[8]
double gref_hlld(const double* q1, const double* q2, const double* n, double* q, double* dsl_dsp_dsc,
                 double w, double dist) {
    Solvers S;
    std::vector<double> a(q1, q1 + 8), b(q2, q2 + 8), nn(n, n + 3), out(8);
    double dsl = 0, dsp = 0, dsc = 0;
    double t = S.HLLD_Solver_Alexashov(a, b, nn, out, dsl, dsp, dsc, w, dist);
    for (int k = 0; k < 8; ++k) q[k] = out[k];
    dsl_dsp_dsc[0] = dsl; dsl_dsp_dsc[1] = dsp; dsl_dsp_dsc[2] = dsc;
    return t;
}

// Reference constants the tests need to build a matching parameter set
// (Help.h:39-114): ga, kurant, Velosity_inf, chi_real, RR_, R1_, R11_, R111_,
// R2_, R3_, R4_, R5_, Left_, Kn_, a_2, n_p_LISM_, n_inner, n_outer_shock
void gref_constants(double* out) {
    out[0] = ga; out[1] = kurant; out[2] = Velosity_inf; out[3] = chi_real; out[4] = RR_;
    out[5] = R1_; out[6] = R11_; out[7] = R111_; out[8] = R2_; out[9] = R3_; out[10] = R4_;
    out[11] = R5_; out[12] = Left_; out[13] = Kn_; out[14] = a_2; out[15] = n_p_LISM_;
    out[16] = n_inner; out[17] = n_outer_shock;
}

}  // extern "C"

extern "C" {
// The reference Setka behind a handle (for the shim test harness).
Setka* gref_setka_ptr(void* hv) { return static_cast<Handle*>(hv)->S; }
}
