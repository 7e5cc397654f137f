// Test infrastructure: include/gelios_setka_shim.hpp driven on the reference's
// own Setka objects.  Built by oracle/Makefile into _ref/libgelios_shim.so
// together with the unmodified reference sources and ref_harness.cpp, and
// linked against the product library (gelios_2d_b200/_lib/libgelios_b200.so),
// the way a maintainer would build the shim into the reference's driver.
//
//   gshim_mirror_check  the shim's mirror() of a reference Setka against the
//                       product's native grid builder (Setka(N1..M4) +
//                       TVD_prepare): every array of the mesh view, exactly
//   gshim_new / gshim_step / gshim_free
//                       a shim that steps a reference Setka in place of
//                       Setka::Go_5_komponent__MK2 / Go_stationary /
//                       Go_stationary_5_komponent_inner_MK2
#include "Help.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../include/gelios_setka_shim.hpp"

extern "C" Setka* gref_setka_ptr(void* hv);

namespace {

template <typename T>
bool same(const char* name, const T* a, const T* b, int64_t n, std::string& first) {
    if (n == 0) return true;
    if ((a == nullptr) != (b == nullptr)) {
        if (first.empty()) first = name;
        return false;
    }
    if (std::memcmp(a, b, sizeof(T) * static_cast<size_t>(n)) != 0) {
        if (first.empty()) first = name;
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

// Number of view arrays (or counts) of the shim's mirror of the reference
// Setka behind `hv` that differ from gelios_mesh_build_setka(dims) +
// gelios_mesh_tvd_prepare; the first differing name goes to msg.
int gshim_mirror_check(void* hv, char* msg, int cap) {
    Setka* S = gref_setka_ptr(hv);
    gelios_shim::Shim sh;
    sh.mirror(S);
    const gelios_mesh_view& a = sh.view;
    gelios_mesh* m = gelios_mesh_build_setka(a.dims[0], a.dims[1], a.dims[2], a.dims[3], a.dims[4], a.dims[5],
                                             a.dims[6], a.dims[7]);
    if (!m) return -1;
    gelios_mesh_tvd_prepare(m);
    gelios_mesh_view b{};
    gelios_mesh_get_view(m, &b);
    std::string first;
    int bad = 0;
    auto cnt = [&](const char* name, int64_t x, int64_t y) {
        if (x != y) {
            bad++;
            if (first.empty()) first = name;
        }
    };
    cnt("n_points", a.n_points, b.n_points);
    cnt("n_cells", a.n_cells, b.n_cells);
    cnt("n_faces", a.n_faces, b.n_faces);
    cnt("n_main", a.n_main, b.n_main);
    cnt("n_rails", a.n_rails, b.n_rails);
    cnt("n_contact", a.n_contact, b.n_contact);
    cnt("n_inner_line", a.n_inner_line, b.n_inner_line);
    cnt("n_outer_line", a.n_outer_line, b.n_outer_line);
    if (bad == 0) {
        const int64_t np = a.n_points, nc = a.n_cells, nf = a.n_faces, nr = a.n_rails;
        bad += !same("x", a.x, b.x, np, first);
        bad += !same("y", a.y, b.y, np, first);
        bad += !same("point_type", a.point_type, b.point_type, np, first);
        bad += !same("cell_type", a.cell_type, b.cell_type, nc, first);
        bad += !same("contour_start", a.contour_start, b.contour_start, nc + 1, first);
        bad += !same("contour", a.contour, b.contour, a.contour_start[nc], first);
        bad += !same("gran_start", a.gran_start, b.gran_start, nc + 1, first);
        bad += !same("gran", a.gran, b.gran, a.gran_start[nc], first);
        bad += !same("cell_back", a.cell_back, b.cell_back, nc, first);
        bad += !same("cell_next", a.cell_next, b.cell_next, nc, first);
        bad += !same("r_istoch", a.r_istoch, b.r_istoch, nc, first);
        bad += !same("face_A", a.face_A, b.face_A, nf, first);
        bad += !same("face_B", a.face_B, b.face_B, nf, first);
        bad += !same("face_type", a.face_type, b.face_type, nf, first);
        bad += !same("face_master", a.face_master, b.face_master, nf, first);
        bad += !same("face_sosed", a.face_sosed, b.face_sosed, nf, first);
        bad += !same("face_copy", a.face_copy, b.face_copy, nf, first);
        bad += !same("face_sosed_up", a.face_sosed_up, b.face_sosed_up, nf, first);
        bad += !same("face_sosed_down", a.face_sosed_down, b.face_sosed_down, nf, first);
        bad += !same("rail_type", a.rail_type, b.rail_type, nr, first);
        bad += !same("rail_s", a.rail_s, b.rail_s, nr, first);
        bad += !same("rail_M", a.rail_M, b.rail_M, 4 * nr, first);
        bad += !same("rail_pstart", a.rail_pstart, b.rail_pstart, nr + 1, first);
        bad += !same("rail_points", a.rail_points, b.rail_points, a.rail_pstart[nr], first);
        bad += !same("rail_kstart", a.rail_kstart, b.rail_kstart, nr + 1, first);
        bad += !same("rail_keys", a.rail_keys, b.rail_keys, a.rail_kstart[nr], first);
        bad += !same("line_contact", a.line_contact, b.line_contact, a.n_contact, first);
        bad += !same("line_inner", a.line_inner, b.line_inner, a.n_inner_line, first);
        bad += !same("line_outer", a.line_outer, b.line_outer, a.n_outer_line, first);
        for (int i = 0; i < 8; i++) cnt("dims", a.dims[i], b.dims[i]);
    }
    gelios_mesh_free(m);
    if (msg && cap > 0) std::snprintf(msg, static_cast<size_t>(cap), "%s", first.c_str());
    return bad;
}

void* gshim_new() { return new gelios_shim::Shim(); }

void gshim_free(void* sh) { delete static_cast<gelios_shim::Shim*>(sh); }

// `n` steps of `form` (GELIOS_FORM_*) on the reference Setka behind hv,
// through the shim; returns the shim's code (0 = ok).
int gshim_step(void* sh, void* hv, int form, int n) {
    return static_cast<gelios_shim::Shim*>(sh)->step(gref_setka_ptr(hv), form, n);
}

}  // extern "C"
