// gelios_setka_shim.hpp — the C++ shim that lets the reference's own driver
// (SergeyMSU/Gelios_2D) step its Setka on a B200 through include/gelios_b200.h.
//
// Header-only; compile it inside the reference's build, with the reference's
// headers on the include path.  It replaces the bodies of three member
// functions (Setka.h:176-186):
//
//   void Setka::Go_stationary(int step)
//       { gelios_shim::instance().step(this, GELIOS_FORM_STATIONARY, step); }
//   void Setka::Go_5_komponent__MK2(int step)
//       { gelios_shim::instance().step(this, GELIOS_FORM_MK2, step); }
//   void Setka::Go_stationary_5_komponent_inner_MK2(int step)
//       { gelios_shim::instance().step(this, GELIOS_FORM_INNER_MK2, step); }
//
// The reference's objects stay the source of truth.  The first call mirrors
// the topology (Point/Cell/Gran/Rail pointers become indices: Point::number,
// Cell::number, All_Gran then All_Gran_copy for faces) into a
// gelios_mesh_view and uploads it; every call copies par[0], par[1] and the
// Monte-Carlo moments of par[0] (H_n, H_u, H_v, H_T, k_u, k_v, k_T: what
// Cell::Get_Sourse_MK1 reads) to the device, steps, and writes par[0],
// par[1] and the moved points (x = x2, y = y2) back.  As in the reference,
// the buffer that holds the result after `step` steps is par[step % 2].
//
// Errors: the reference stops the process (exit(-1)) where a step cannot go
// on; step() returns the gelios error code or, for a step whose status
// flags are set, GELIOS_E_STATE, and the method bodies above may exit on a
// non-zero value like the reference does.
#pragma once

#include <cstdint>
#include <unordered_map>
#include <vector>

#include "Cell.h"
#include "Gran.h"
#include "Point.h"
#include "Rail.h"
#include "Setka.h"

// The reference's Help.h defines object-like macros that are also field
// names of gelios_params (kurant, a_2, n_inner, n_outer_shock): keep them out
// of the ABI header and restore them afterwards.
#pragma push_macro("kurant")
#pragma push_macro("a_2")
#pragma push_macro("n_inner")
#pragma push_macro("n_outer_shock")
#undef kurant
#undef a_2
#undef n_inner
#undef n_outer_shock
#include "gelios_b200.h"
#pragma pop_macro("n_outer_shock")
#pragma pop_macro("n_inner")
#pragma pop_macro("a_2")
#pragma pop_macro("kurant")

namespace gelios_shim {

struct Shim {
    gelios_ctx* ctx = nullptr;
    const Setka* mirrored = nullptr;  // the grid whose topology is on the device
    gelios_params prm{};
    bool have_prm = false;
    std::vector<double> x, y, rs, ri;
    std::vector<int32_t> pt, ct, cs, con, gs, gr, fa, fb, fty, fm, fso, fc, fsu, fsd, back, next;
    std::vector<int32_t> rty, rM, rps, rpts, rks, rkeys, lc, li, lo;
    gelios_mesh_view view{};
    gelios_status last{};

    ~Shim() {
        if (ctx) gelios_destroy(ctx);
    }

    // The run's constants (gelios_params); without a call the reference's
    // compile-time constants are used (gelios_params_reference).
    void set_params(const gelios_params& p) {
        prm = p;
        have_prm = true;
        if (ctx) gelios_set_params(ctx, &prm);
    }

    // Flat arrays of S's topology in the ABI's numbering (gelios_mesh_view).
    void mirror(const Setka* S) {
        for (auto* v : {&x, &y, &rs, &ri}) v->clear();
        for (auto* v : {&pt, &ct, &cs, &con, &gs, &gr, &fa, &fb, &fty, &fm, &fso, &fc, &fsu, &fsd, &back, &next, &rty,
                        &rM, &rps, &rpts, &rks, &rkeys, &lc, &li, &lo})
            v->clear();
        std::unordered_map<const Gran*, int32_t> fid;  // unified face numbering
        int32_t k = 0;
        for (auto g : S->All_Gran) fid[g] = k++;
        for (auto g : S->All_Gran_copy) fid[g] = k++;
        auto cid = [](const Cell* c) { return c ? static_cast<int32_t>(c->number) : -1; };
        auto face_id = [&](const Gran* g) { return g ? fid.at(g) : -1; };
        for (auto p : S->All_Points) {
            x.push_back(p->x);
            y.push_back(p->y);
            pt.push_back(static_cast<int32_t>(p->type));
        }
        cs.push_back(0);
        gs.push_back(0);
        for (auto c : S->All_Cells) {
            ct.push_back(static_cast<int32_t>(c->type));
            for (auto p : c->contour) con.push_back(p->number);
            for (auto g : c->Grans) gr.push_back(face_id(g));
            cs.push_back(static_cast<int32_t>(con.size()));
            gs.push_back(static_cast<int32_t>(gr.size()));
            back.push_back(cid(c->Back));
            next.push_back(cid(c->Next));
            ri.push_back(c->r_istoch);
        }
        auto face = [&](const Gran* g) {
            fa.push_back(g->A->number);
            fb.push_back(g->B->number);
            fty.push_back(static_cast<int32_t>(g->type));
            fm.push_back(cid(g->Master));
            fso.push_back(cid(g->Sosed));
            fc.push_back(face_id(g->Gran_copy));
            fsu.push_back(cid(g->Sosed_up));
            fsd.push_back(cid(g->Sosed_down));
        };
        for (auto g : S->All_Gran) face(g);
        for (auto g : S->All_Gran_copy) face(g);
        rps.push_back(0);
        rks.push_back(0);
        for (const auto* rails : {&S->A_Rails, &S->B_Rails, &S->C_Rails, &S->D_Rails})
            for (auto R : *rails) {
                rty.push_back(static_cast<int32_t>(R->type));
                rs.push_back(R->s);
                rM.insert(rM.end(), {R->M1, R->M2, R->M3, R->M4});
                for (auto p : R->All_point) rpts.push_back(p->number);
                for (auto p : R->Key_point) rkeys.push_back(p->number);
                rps.push_back(static_cast<int32_t>(rpts.size()));
                rks.push_back(static_cast<int32_t>(rkeys.size()));
            }
        for (auto g : S->Line_Contact) lc.push_back(face_id(g));
        for (auto g : S->Line_Inner) li.push_back(face_id(g));
        for (auto g : S->Line_Outer) lo.push_back(face_id(g));
        const int dims[8] = {S->N1, S->N2, S->N3, S->N4, S->M1, S->M2, S->M3, S->M4};
        view = gelios_mesh_view{};
        for (int i = 0; i < 8; i++) view.dims[i] = dims[i];
        view.n_points = static_cast<int32_t>(x.size());
        view.x = x.data();
        view.y = y.data();
        view.point_type = pt.data();
        view.n_cells = static_cast<int32_t>(ct.size());
        view.cell_type = ct.data();
        view.contour_start = cs.data();
        view.contour = con.data();
        view.gran_start = gs.data();
        view.gran = gr.data();
        view.cell_back = back.data();
        view.cell_next = next.data();
        view.r_istoch = ri.data();
        view.n_faces = static_cast<int32_t>(fa.size());
        view.n_main = static_cast<int32_t>(S->All_Gran.size());
        view.face_A = fa.data();
        view.face_B = fb.data();
        view.face_type = fty.data();
        view.face_master = fm.data();
        view.face_sosed = fso.data();
        view.face_copy = fc.data();
        view.face_sosed_up = fsu.data();
        view.face_sosed_down = fsd.data();
        view.n_rails = static_cast<int32_t>(rty.size());
        view.rail_type = rty.data();
        view.rail_s = rs.data();
        view.rail_M = rM.data();
        view.rail_pstart = rps.data();
        view.rail_points = rpts.data();
        view.rail_kstart = rks.data();
        view.rail_keys = rkeys.data();
        view.n_contact = static_cast<int32_t>(lc.size());
        view.n_inner_line = static_cast<int32_t>(li.size());
        view.n_outer_line = static_cast<int32_t>(lo.size());
        view.line_contact = lc.data();
        view.line_inner = li.data();
        view.line_outer = lo.data();
    }

    int state_to_device(const Setka* S) {
        const size_t n = S->All_Cells.size();
        std::vector<double> f[5];
        for (int b = 0; b < 2; b++) {
            for (auto& v : f) v.assign(n, 0.0);
            for (size_t c = 0; c < n; c++) {
                const Parametr& P = S->All_Cells[c]->par[b];
                f[0][c] = P.ro;
                f[1][c] = P.p;
                f[2][c] = P.u;
                f[3][c] = P.v;
                f[4][c] = P.Q;
            }
            const int rc = gelios_upload_state(ctx, b, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data());
            if (rc) return rc;
        }
        std::vector<double> Hn(4 * n), Hu(4 * n), Hv(4 * n), HT(4 * n), kU(n), kV(n), kT(n);
        for (size_t c = 0; c < n; c++) {
            const Parametr& P = S->All_Cells[c]->par[0];
            for (int s = 0; s < 4; s++) {
                Hn[4 * c + s] = P.H_n[s];
                Hu[4 * c + s] = P.H_u[s];
                Hv[4 * c + s] = P.H_v[s];
                HT[4 * c + s] = P.H_T[s];
            }
            kU[c] = P.k_u;
            kV[c] = P.k_v;
            kT[c] = P.k_T;
        }
        return gelios_upload_mc(ctx, Hn.data(), Hu.data(), Hv.data(), HT.data(), kU.data(), kV.data(), kT.data());
    }

    int state_from_device(Setka* S) {
        const size_t n = S->All_Cells.size();
        std::vector<double> f[5];
        for (int b = 0; b < 2; b++) {
            for (auto& v : f) v.assign(n, 0.0);
            const int rc =
                gelios_download_state(ctx, b, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data());
            if (rc) return rc;
            for (size_t c = 0; c < n; c++) {
                Parametr& P = S->All_Cells[c]->par[b];
                P.ro = f[0][c];
                P.p = f[1][c];
                P.u = f[2][c];
                P.v = f[3][c];
                P.Q = f[4][c];
            }
        }
        std::vector<double> px(S->All_Points.size()), py(S->All_Points.size());
        const int rc = gelios_download_points(ctx, px.data(), py.data());
        if (rc) return rc;
        for (size_t i = 0; i < px.size(); i++) {
            S->All_Points[i]->x = S->All_Points[i]->x2 = px[i];
            S->All_Points[i]->y = S->All_Points[i]->y2 = py[i];
        }
        return GELIOS_OK;
    }

    // `n` steps of `form` on S, in place of the reference's member function.
    int step(Setka* S, int form, int n, int device = 0) {
        int rc = GELIOS_OK;
        if (!ctx) {
            if (!have_prm) gelios_params_reference(&prm);
            rc = gelios_create(&ctx, &prm, device);
            if (rc) return rc;
        }
        if (mirrored != S) {
            mirror(S);
            rc = gelios_upload_topology(ctx, &view);
            if (rc) return rc;
            mirrored = S;
        }
        rc = state_to_device(S);
        if (rc) return rc;
        if (form == GELIOS_FORM_INNER_MK2) {
            std::vector<int32_t> inner;
            for (auto c : S->All_Cells_Inner) inner.push_back(c->number);
            rc = gelios_set_inner_cells(ctx, inner.data(), static_cast<int32_t>(inner.size()));
            if (rc) return rc;
        }
        rc = gelios_step(ctx, form, n, &last);
        if (rc) return rc;
        rc = state_from_device(S);
        if (rc) return rc;
        return last.flags ? GELIOS_E_STATE : GELIOS_OK;
    }
};

// One shim per process, as the reference keeps one Setka.
inline Shim& instance() {
    static Shim s;
    return s;
}

}  // namespace gelios_shim
