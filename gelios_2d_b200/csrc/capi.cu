// C ABI of gelios_b200: the device context that stands in for a reference
// Setka during its time loops (Setka.h:176-186).  Host code only; kernels are
// in step_kernels.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gelios_b200.h"
#include "physics.cuh"
#include "step_kernels.cuh"

namespace gelios {
void set_error(const std::string& msg);
gelios_mesh* mesh_from_view(const gelios_mesh_view* v);
}  // namespace gelios

using namespace gelios;

namespace {

#define GELIOS_CUDA_TRY(expr)                                                              \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));                 \
            return GELIOS_E_CUDA;                                                          \
        }                                                                                  \
    } while (0)

// A device allocation owned by the context.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    int alloc(size_t n) {
        if (p) {
            cudaFree(p);
            p = nullptr;
        }
        bytes = n;
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
            p = nullptr;
            return GELIOS_E_CUDA;
        }
        return GELIOS_OK;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

template <typename T>
int upload(DBuf& b, const T* src, size_t n, cudaStream_t s) {
    int rc = b.alloc(n * sizeof(T));
    if (rc) return rc;
    if (n && src) {
        cudaError_t e = cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            set_error(std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
            return GELIOS_E_CUDA;
        }
    } else if (n) {
        cudaMemsetAsync(b.p, 0, n * sizeof(T), s);
    }
    return GELIOS_OK;
}

}  // namespace

struct gelios_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // side stream: the work of the moving-grid step that does not depend on
    // the motion runs there while the main stream moves the grid (one side
    // stream: a second one for the source terms made the main chain slower
    // through contention for the SMs)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_recon = nullptr, ev_rails = nullptr, ev_tracked = nullptr;
    // pipelined moving-grid step: the next step's surface tracking and rails
    // run on `motion` while the main stream updates the cells nobody of the
    // next step's motion reads (see mk2_pipelined)
    cudaStream_t motion = nullptr;
    cudaEvent_t ev_early = nullptr, ev_motion = nullptr, ev_side2 = nullptr;
    // the C_1 interior and one-sided face-unit groups beside the tracked-face
    // fluxes in a pipelined call
    cudaStream_t groups = nullptr;
    cudaEvent_t ev_groups = nullptr;
    DBuf early;       // cells flagged CF_EARLY, updated first
    int n_early = 0;
    bool pipelined = true;  // gelios_set_pipelined
    gelios_params prm{};
    bool have_mesh = false;
    DevMesh d;
    // topology / geometry
    DBuf X, Y, X2, Y2, ptype, cstart, contour, gstart, cflags, ctype, sA, sB, snb, ssd, ssd2, sinfo, qcorner;
    DBuf fA, fB, ftype, fmaster, fsosed, fcopy, fsdown;
    DBuf rtype, rM, rpstart, rpts, rkstart, rkeys, rs;
    DBuf lc, li, lo, sp_point, sp_line, sp_inc, sp_ainc, sp_fix, sp_of_point;
    DBuf u_slot, u_cell, u_twin, u_A, u_B, u_info, u_nb, u_sd, u_sd2, flux, aux, rec, pstar, src_lo;
    DBuf Hn, Hu, Hv, HT, ku, kv, kT, r_istoch, cback, cnext;
    // state par[2] x 5 fields, centroids [2], scratch
    DBuf state[2];
    // extra rows of par[0/1]: hydrogen fluids H1..H4 (16 rows, Go_5_komponent
    // form) or the MHD form's w, B and pickup protons (8 rows)
    DBuf hstate[2];
    gelios_mhd_params mprm{};
    DBuf src_fixed;  // MHD form: fixed charge-exchange sources (3 rows)
    DBuf flux_mhd;   // multi-fluid forms: 13 (MHD) or 21 (Go_5_komponent) flux rows per face slot, on first use
    int mhd_face_variant = 0;  // launch shape of the MHD face kernel (gelios_autotune)
    int mk2_variant = 0;  // arrangement / launch shape of the moving-grid face units + update (gelios_autotune)
    // tiles of the moving-grid step (see TileView)
    DBuf t_cstart, t_cells, t_lbase, t_fstart, t_faces;
    TileView tiles;
    DBuf resid;                // residual partial sums (gelios_residual)
    // streamed host I/O (gelios_run_streamed): copy streams, staging
    // buffers and their events, created on first use
    cudaStream_t io_h2d = nullptr, io_d2h = nullptr;
    DBuf io_in[2], io_out[2];
    cudaEvent_t ev_in_ready[2] = {nullptr, nullptr}, ev_in_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_out_ready[2] = {nullptr, nullptr}, ev_out_free[2] = {nullptr, nullptr};
    DBuf cen[2];
    DBuf words;    // T[2] (double), dt_acc (u64), counters[2] (u64), status (int)
    DBuf surface;  // Move_surface per-face speeds
    DBuf inner;
    int n_inner = 0;
    int n_sp = 0;
    // cen[0] holds the centroids of the current points (rows cx, cy,
    // |c|^(2 gamma), area, rotated volume); after a moving-grid call row 2
    // holds only the CF_RP cells, which the other forms do not accept
    bool cen_valid = false;
    bool cen_rp_partial = false;
    // |face centre|^(2 gamma) per face unit for the plain form; stale once
    // the points move, the topology or gamma changes
    DBuf upf;
    bool upf_valid = false;
    // Instantiated graphs of one moving-grid step, keyed by the buffers the
    // step reads (state parity and centroid buffer); dropped whenever the
    // topology or the parameters change.
    struct StepGraph {
        int form = -1;
        int kind = 0;   // 0: one whole step; 1-3: head / body / last part of a pipelined moving-grid call
        int first = 0;  // the first step of a call: the graph starts with the words' initialisation
        int parity = -1;
        const void* cen = nullptr;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
    };
    StepGraph graphs[16];
    bool graphs_off = false;  // capture failed once: launch directly
    bool coop_off = false;    // the cooperative plain step could not launch once: three kernels per step
    void drop_graphs() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g = StepGraph{};
        }
    }
    int64_t launches = 0;
    // phase timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    size_t ev_used = 0;
    double phase_ms[5] = {0, 0, 0, 0, 0};
    int64_t phase_launch[5] = {0, 0, 0, 0, 0};
    cudaEvent_t event() {
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }
    // records the start of a phase; returns the event (or nullptr if timing is off)
    cudaEvent_t phase_begin() {
        if (!timing) return nullptr;
        cudaEvent_t e = event();
        cudaEventRecord(e, stream);
        return e;
    }
    void phase_end(int phase, cudaEvent_t begin, int n_launch) {
        if (!timing || !begin) return;
        phase_launch[phase] += n_launch;
        cudaEvent_t e = event();
        cudaEventRecord(e, stream);
        pending.push_back({phase, {begin, e}});
    }
    void collect() {
        if (pending.empty()) return;
        cudaStreamSynchronize(stream);
        for (auto& p : pending) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.second.first, p.second.second);
            phase_ms[p.first] += ms;
        }
        pending.clear();
        ev_used = 0;
    }
    ~gelios_ctx() {
        drop_graphs();
        for (auto e : ev_pool) cudaEventDestroy(e);
    }

    double* T() const { return words.as<double>(); }
    unsigned long long* acc() const { return reinterpret_cast<unsigned long long*>(words.as<char>() + 16); }
    unsigned long long* counters() const { return reinterpret_cast<unsigned long long*>(words.as<char>() + 24); }
    int* status() const { return reinterpret_cast<int*>(words.as<char>() + 40); }
    double* field(int buf, int k) const { return state[buf].as<double>() + static_cast<size_t>(k) * d.n_cells; }
};

extern "C" void gelios_params_reference(gelios_params* o) {
    if (!o) return;
    const double RR = 390.222;
    std::memset(o, 0, sizeof(*o));
    o->gamma = 5.0 / 3.0;
    o->kurant = 0.1;
    o->chi = 36.1275;
    o->inner_mach = 10.0;
    o->in_ro = 1.0;
    o->in_p = 1.0;
    o->in_u = -2.54338;
    o->in_v = 0.0;
    o->in_Q = 100.0;
    o->extern_u_par = -0.1;
    o->extern_u_tvd = -0.01;
    o->R11 = 38.0 / RR;
    o->rad_stat = 95.0;
    o->R1 = 1.0 / RR;
    o->R111 = 50.0 / RR;
    o->R5 = 2200.0 / RR;
    o->Left = -1500.0 / RR;
    o->koef = 0.1;
    o->src_rmin = 10.0 / RR;
    o->src_rmax = 1500.0 / RR;
    o->src_coef = 3.0 / 6.0;
    o->a_2 = 0.1307345665;
    o->ro_floor = 0.00001;
    o->p_floor = 0.000001;
    o->dt0 = 0.00000001;
    o->n_inner = 20;
    o->n_outer_shock = 13;
    o->godunov_max_iter = 1100;
    o->precision = GELIOS_PREC_FP64;
}

extern "C" int gelios_create(gelios_ctx** out, const gelios_params* prm, int device) {
    if (!out || !prm) {
        set_error("gelios_create: null argument");
        return GELIOS_E_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("gelios_create: no CUDA device");
        return GELIOS_E_NODEVICE;
    }
    if (device < 0 || device >= ndev) {
        set_error("gelios_create: device index out of range");
        return GELIOS_E_ARG;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(device));
    auto ctx = std::make_unique<gelios_ctx>();
    ctx->device = device;
    ctx->prm = *prm;
    // The main stream carries the serial chain of the moving-grid step
    // (surface tracking -> rails -> fluxes -> update), whose kernels occupy
    // few SMs; it gets the highest priority so that its blocks are placed
    // first while the side streams' grid-wide kernels fill the rest.
    int prio_least = 0, prio_greatest = 0;
    GELIOS_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
    GELIOS_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_greatest));
    GELIOS_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, prio_least));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_recon, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_rails, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&ctx->ev_tracked, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->motion, cudaStreamNonBlocking, prio_greatest));
    GELIOS_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->groups, cudaStreamNonBlocking, prio_least));
    for (cudaEvent_t* e : {&ctx->ev_early, &ctx->ev_motion, &ctx->ev_side2, &ctx->ev_groups})
        GELIOS_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    if (ctx->words.alloc(64)) return GELIOS_E_CUDA;
    GELIOS_CUDA_TRY(cudaMemsetAsync(ctx->words.p, 0, 64, ctx->stream));
    *out = ctx.release();
    return GELIOS_OK;
}

namespace {
double sqrt_threshold(double R);
}

extern "C" int gelios_set_params(gelios_ctx* ctx, const gelios_params* prm) {
    if (!ctx || !prm) return GELIOS_E_ARG;
    ctx->prm = *prm;
    ctx->d.r11_sq = sqrt_threshold(prm->R11);
    ctx->cen_valid = false;  // the cached |centroid|^(2 gamma) depends on gamma
    ctx->upf_valid = false;
    ctx->drop_graphs();      // the parameters are kernel arguments
    return GELIOS_OK;
}

extern "C" void gelios_destroy(gelios_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    for (cudaStream_t* sp : {&ctx->side, &ctx->motion, &ctx->groups, &ctx->io_h2d, &ctx->io_d2h})
        if (*sp) {
            cudaStreamSynchronize(*sp);
            cudaStreamDestroy(*sp);
        }
    for (cudaEvent_t e : {ctx->ev_fork, ctx->ev_recon, ctx->ev_rails, ctx->ev_tracked, ctx->ev_early,
                          ctx->ev_motion, ctx->ev_side2, ctx->ev_groups})
        if (e) cudaEventDestroy(e);
    for (int j = 0; j < 2; j++)
        for (cudaEvent_t e : {ctx->ev_in_ready[j], ctx->ev_in_free[j], ctx->ev_out_ready[j], ctx->ev_out_free[j]})
            if (e) cudaEventDestroy(e);
    delete ctx;
}

namespace {

// Smallest a >= 0 with sqrt(a) >= R (sqrt correctly rounded, as on the
// device): !(sqrt(a) < R) holds exactly when !(a < threshold).
double sqrt_threshold(double R) {
    if (!(R > 0.0)) return 0.0;
    double t = R * R;
    while (t > 0.0 && std::sqrt(std::nextafter(t, 0.0)) >= R) t = std::nextafter(t, 0.0);
    while (std::sqrt(t) < R) t = std::nextafter(t, HUGE_VAL);
    return t;
}

// Tiles of the moving-grid step (TileView): recursive coordinate bisection of
// the cell centroids in (polar angle, log radius), each axis scaled by the
// median spacing of face neighbours along it so that a tile spans about as
// many cells in both directions; splits at multiples of kTileCells so that
// every tile but the last of a branch is full.  Then, per tile, its cells in
// index order with their local slot bases, and the face units that touch
// them (owner side, other side or both).
struct TileBuild {
    std::vector<int32_t> cstart, cells, lbase, fstart;
    std::vector<int2> faces;
    int max_slots = 0;
};

int build_tiles(const gelios_mesh_view* v, const std::vector<int32_t>& u_slot, const std::vector<int32_t>& u_cell,
                const std::vector<int32_t>& u_twin, const std::vector<int32_t>& snb, TileBuild& tb) {
    const int nc = v->n_cells;
    std::vector<double> kx(nc), ky(nc);
    for (int c = 0; c < nc; c++) {
        // polygon centroid (the tiling needs no exact geometry)
        double A = 0.0, gx = 0.0, gy = 0.0;
        const int s0 = v->contour_start[c], n = v->contour_start[c + 1] - s0;
        for (int i = 0; i < n; i++) {
            const int a = v->contour[s0 + i], b = v->contour[s0 + (i + 1) % n];
            const double cr = v->x[a] * v->y[b] - v->y[a] * v->x[b];
            A += cr;
            gx += (v->x[a] + v->x[b]) * cr;
            gy += (v->y[a] + v->y[b]) * cr;
        }
        double x = 0.0, y = 0.0;
        if (A != 0.0) {
            x = gx / (3.0 * A);
            y = gy / (3.0 * A);
        }
        const double r = std::sqrt(x * x + y * y);
        kx[c] = std::atan2(y, x);
        ky[c] = std::log(r > 1e-300 ? r : 1e-300);
    }
    // median neighbour spacing along each axis
    std::vector<double> dth, dlr;
    for (size_t u = 0; u < u_slot.size(); u++) {
        if (u_twin[u] < 0) continue;
        const int a = u_cell[u], b = snb[u_slot[u]];
        const double t = std::fabs(kx[a] - kx[b]), l = std::fabs(ky[a] - ky[b]);
        if (t > l)
            dth.push_back(t);
        else
            dlr.push_back(l);
    }
    auto median = [](std::vector<double>& w) {
        if (w.empty()) return 1.0;
        std::nth_element(w.begin(), w.begin() + w.size() / 2, w.end());
        const double m = w[w.size() / 2];
        return m > 0.0 ? m : 1.0;
    };
    const double sx = 1.0 / median(dth), sy = 1.0 / median(dlr);
    for (int c = 0; c < nc; c++) {
        kx[c] *= sx;
        ky[c] *= sy;
    }
    std::vector<int32_t> perm(nc);
    for (int c = 0; c < nc; c++) perm[c] = c;
    std::vector<std::pair<int, int>> stack{{0, nc}}, leaves;
    while (!stack.empty()) {
        const std::pair<int, int> range = stack.back();
        stack.pop_back();
        const int lo = range.first, hi = range.second, n = hi - lo;
        if (n <= kTileCells) {
            if (n > 0) leaves.push_back(range);
            continue;
        }
        double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
        for (int i = lo; i < hi; i++) {
            const int c = perm[i];
            x0 = std::min(x0, kx[c]);
            x1 = std::max(x1, kx[c]);
            y0 = std::min(y0, ky[c]);
            y1 = std::max(y1, ky[c]);
        }
        const std::vector<double>& key = (x1 - x0 >= y1 - y0) ? kx : ky;
        const int nt = (n + kTileCells - 1) / kTileCells;
        const int left = (nt / 2) * kTileCells;
        std::nth_element(perm.begin() + lo, perm.begin() + lo + left, perm.begin() + hi, [&](int a, int b) {
            return key[a] < key[b] || (key[a] == key[b] && a < b);
        });
        stack.push_back({lo + left, hi});
        stack.push_back({lo, lo + left});
    }
    std::sort(leaves.begin(), leaves.end());
    const int nt = static_cast<int>(leaves.size());
    std::vector<int32_t> tile_of(nc), local_of(nc);
    tb.cstart.assign(1, 0);
    tb.cells.clear();
    tb.lbase.clear();
    tb.max_slots = 0;
    for (int t = 0; t < nt; t++) {
        std::sort(perm.begin() + leaves[t].first, perm.begin() + leaves[t].second);
        int slots = 0;
        for (int i = leaves[t].first; i < leaves[t].second; i++) {
            const int c = perm[i];
            tile_of[c] = t;
            local_of[c] = slots;
            tb.cells.push_back(c);
            tb.lbase.push_back(slots);
            slots += v->gran_start[c + 1] - v->gran_start[c];
        }
        if (slots >= kTileNone) return GELIOS_E_LIMIT;
        tb.max_slots = std::max(tb.max_slots, slots);
        tb.cstart.push_back(static_cast<int32_t>(tb.cells.size()));
    }
    // face units per tile: by the owner cell's tile, and by the other side's
    // tile when that differs
    std::vector<std::vector<int2>> per(nt);
    for (size_t u = 0; u < u_slot.size(); u++) {
        const int K = u_cell[u], g = u_slot[u];
        const int tK = tile_of[K];
        const int own = local_of[K] + (g - v->gran_start[K]);
        int tw = kTileNone, tN = -1, other = kTileNone;
        if (u_twin[u] >= 0) {
            const int N = snb[g], gt = u_twin[u];
            tN = tile_of[N];
            other = local_of[N] + (gt - v->gran_start[N]);
            if (tN == tK) tw = other;
        }
        per[tK].push_back(make_int2(static_cast<int>(u), own | (tw << 16)));
        if (tN >= 0 && tN != tK) per[tN].push_back(make_int2(static_cast<int>(u), kTileNone | (other << 16)));
    }
    tb.fstart.assign(1, 0);
    tb.faces.clear();
    for (int t = 0; t < nt; t++) {
        std::sort(per[t].begin(), per[t].end(), [](const int2& a, const int2& b) { return a.x < b.x; });
        tb.faces.insert(tb.faces.end(), per[t].begin(), per[t].end());
        tb.fstart.push_back(static_cast<int32_t>(tb.faces.size()));
    }
    return GELIOS_OK;
}

}  // namespace

extern "C" int gelios_upload_topology(gelios_ctx* ctx, const gelios_mesh_view* v) {
    if (!ctx || !v) return GELIOS_E_ARG;
    ctx->drop_graphs();  // they hold the buffers about to be replaced
    if (v->n_points <= 0 || v->n_cells <= 0 || v->n_faces <= 0 || !v->x || !v->y || !v->point_type ||
        !v->cell_type || !v->contour_start || !v->contour || !v->gran_start || !v->gran || !v->face_A || !v->face_B ||
        !v->face_type || !v->face_master || !v->face_sosed || !v->face_copy) {
        set_error("gelios_upload_topology: incomplete mesh view");
        return GELIOS_E_ARG;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const int np = v->n_points, nc = v->n_cells, nf = v->n_faces;
    // TVD_prepare outputs: taken from the caller or computed here
    std::unique_ptr<gelios_mesh, void (*)(gelios_mesh*)> tmp(nullptr, gelios_mesh_free);
    const int32_t *fsdown = v->face_sosed_down, *cback = v->cell_back, *cnext = v->cell_next;
    const double* r_istoch = v->r_istoch;
    if (!fsdown || !cback || !cnext || !r_istoch) {
        tmp.reset(mesh_from_view(v));
        int rc = gelios_mesh_tvd_prepare(tmp.get());
        if (rc) return rc;
        gelios_mesh_view tv;
        gelios_mesh_get_view(tmp.get(), &tv);
        if (!fsdown) fsdown = tv.face_sosed_down;
        if (!cback) cback = tv.cell_back;
        if (!cnext) cnext = tv.cell_next;
        if (!r_istoch) r_istoch = tv.r_istoch;
    }
    const int ng = v->gran_start[nc];
    // per-slot arrays and per-cell flags
    std::vector<int32_t> sA(ng), sB(ng), snb(ng), ssd(ng), ssd2(ng);
    std::vector<uint32_t> sinfo(ng), cflags(nc, 0u);
    for (int c = 0; c < nc; c++) {
        if (v->cell_type[c] == C_1) cflags[c] |= CF_C1;
        if (v->cell_type[c] == C_CENTR) cflags[c] |= CF_CENTR;
        for (int g = v->gran_start[c]; g < v->gran_start[c + 1]; g++) {
            const int f = v->gran[g];
            if (f < 0 || f >= nf) {
                set_error("gelios_upload_topology: face index out of range");
                return GELIOS_E_MESH;
            }
            if (v->face_master[f] != c) {
                set_error("gelios_upload_topology: a face in Cell::Grans is not mastered by that cell");
                return GELIOS_E_MESH;
            }
            const int ft = v->face_type[f];
            if (ft == G_AXIS) cflags[c] |= CF_AXIS;
            sA[g] = v->face_A[f];
            sB[g] = v->face_B[f];
            snb[g] = v->face_sosed[f];
            ssd[g] = fsdown[f];
            const int fc = v->face_copy[f];
            ssd2[g] = fc >= 0 ? fsdown[fc] : -1;
            if (ft == G_USUALY && (snb[g] < 0 || fc < 0)) {
                set_error("gelios_upload_topology: interior face without neighbour or twin");
                return GELIOS_E_MESH;
            }
            const int ta = v->point_type[sA[g]], tb = v->point_type[sB[g]];
            uint32_t info = static_cast<uint32_t>(ft) & SI_TYPE_MASK;
            const bool god = (ta == P_CONTACT && tb == P_CONTACT) || (ta == P_INNER_SHOCK && tb == P_INNER_SHOCK) ||
                             (ta == P_OUTER_SHOCK && tb == P_OUTER_SHOCK);
            bool npf = false;
            if (ta == P_CONTACT && tb != P_CONTACT) npf = true;
            else if (ta != P_CONTACT && tb == P_CONTACT) npf = true;
            else if (ta == P_INNER_SHOCK && tb != P_INNER_SHOCK) npf = true;
            else if (ta != P_INNER_SHOCK && tb == P_INNER_SHOCK) npf = true;
            else if (ta == P_OUTER_SHOCK && tb != P_OUTER_SHOCK) npf = true;
            else if (ta != P_OUTER_SHOCK && tb == P_OUTER_SHOCK) npf = true;
            if (god) info |= SI_GOD;
            if (npf) info |= SI_NP;
            sinfo[g] = info;
        }
    }
    // rails must come grouped A, B, C, D (the export order of the reference lists)
    int na = 0, nb = 0, ncr = 0, nd = 0;
    for (int r = 0; r < v->n_rails; r++) {
        const int t = v->rail_type[r];
        const int expect_min = (nb + ncr + nd) ? ((ncr + nd) ? ((nd) ? 3 : 2) : 1) : 0;
        if (t < expect_min || t > 3) {
            set_error("gelios_upload_topology: rails must be ordered A, B, C, D");
            return GELIOS_E_MESH;
        }
        const int nk = v->rail_kstart[r + 1] - v->rail_kstart[r];
        if ((t != 2 && nk < 4) || (t == 2 && nk < 2)) {
            set_error("gelios_upload_topology: rail without its key points");
            return GELIOS_E_MESH;
        }
        (t == 0 ? na : t == 1 ? nb : t == 2 ? ncr : nd)++;
    }
    // face units: every slot of a cell except the twins of interior faces,
    // whose flux comes from the unit of the main face (see step_kernels.cu)
    std::vector<int32_t> u_slot, u_cell, u_twin;
    int u_c1 = 0, u_tr0 = 0, u_tr1 = 0;
    {
        std::vector<int32_t> slot_of_face(nf, -1);
        for (int c = 0; c < nc; c++)
            for (int g = v->gran_start[c]; g < v->gran_start[c + 1]; g++) slot_of_face[v->gran[g]] = g;
        for (int c = 0; c < nc; c++)
            for (int g = v->gran_start[c]; g < v->gran_start[c + 1]; g++) {
                const int f = v->gran[g];
                const bool interior = v->face_type[f] == G_USUALY;
                if (interior && f >= v->n_main) continue;  // twin of a main face
                int twin = -1;
                if (interior) {
                    twin = slot_of_face[v->face_copy[f]];
                    if (twin < 0) {
                        set_error("gelios_upload_topology: interior face whose twin is in no cell");
                        return GELIOS_E_MESH;
                    }
                }
                u_slot.push_back(g);
                u_cell.push_back(c);
                u_twin.push_back(twin);
            }
        // group units of the same kind (plain interior, interior with a C_1
        // side, tracked, one-sided) so that warps run one code path
        {
            const size_t nu = u_slot.size();
            std::vector<int> cls(nu);
            for (size_t u = 0; u < nu; u++) {
                const int g = u_slot[u];
                const int f = v->gran[g];
                const int ta = v->point_type[v->face_A[f]], tb = v->point_type[v->face_B[f]];
                const bool tracked = (ta == P_CONTACT && tb == P_CONTACT) || (ta == P_INNER_SHOCK && tb == P_INNER_SHOCK) ||
                                     (ta == P_OUTER_SHOCK && tb == P_OUTER_SHOCK);
                const bool c1 = v->cell_type[u_cell[u]] == C_1 ||
                                (u_twin[u] >= 0 && v->cell_type[v->face_sosed[f]] == C_1);
                cls[u] = tracked ? 2 : (u_twin[u] < 0 ? 3 : (c1 ? 1 : 0));
            }
            std::vector<size_t> order(nu);
            for (size_t u = 0; u < nu; u++) order[u] = u;
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return cls[a] < cls[b]; });
            std::vector<int32_t> s2(nu), c2(nu), t2(nu);
            for (size_t k = 0; k < nu; k++) {
                s2[k] = u_slot[order[k]];
                c2[k] = u_cell[order[k]];
                t2[k] = u_twin[order[k]];
            }
            u_slot.swap(s2);
            u_cell.swap(c2);
            u_twin.swap(t2);
            u_c1 = 0;
            while (u_c1 < static_cast<int>(nu) && cls[order[u_c1]] < 1) u_c1++;
            u_tr0 = 0;
            while (u_tr0 < static_cast<int>(nu) && cls[order[u_tr0]] < 2) u_tr0++;
            u_tr1 = u_tr0;
            while (u_tr1 < static_cast<int>(nu) && cls[order[u_tr1]] == 2) u_tr1++;
        }
        // every interior twin must be covered by its main face's unit
        std::vector<char> covered(ng, 0);
        for (size_t u = 0; u < u_slot.size(); u++) {
            covered[u_slot[u]] = 1;
            if (u_twin[u] >= 0) covered[u_twin[u]] = 1;
        }
        for (int g = 0; g < ng; g++)
            if (!covered[g]) {
                set_error("gelios_upload_topology: interior copy face without its main face in a cell");
                return GELIOS_E_MESH;
            }
    }
    // CF_RP: cells whose |centroid|^(2 gamma) a moving-grid step reads: the
    // cells of every radially reconstructed unit (its two cells and both
    // Sosed_down cells, see mk2_recon_unit) and the masters of the inner
    // shock's faces (surface_faces_kernel)
    for (size_t u = 0; u < u_slot.size(); u++) {
        const int g = u_slot[u], K = u_cell[u];
        const int nbu = u_twin[u] >= 0 ? snb[g] : -1;
        const int ft = static_cast<int>(sinfo[g] & SI_TYPE_MASK);
        const bool radial = ((cflags[K] & CF_C1) && (ft == G_USUALY || ft == G_AXIS)) || ft == G_INNER_SPHERE ||
                            (ft == G_USUALY && nbu >= 0 && (cflags[nbu] & CF_C1));
        if (!radial) continue;
        for (const int c : {K, nbu, ssd[g], ssd2[g]})
            if (c >= 0) cflags[c] |= CF_RP;
    }
    for (int j = 0; j < v->n_inner_line; j++) {
        const int f = v->line_inner[j];
        if (f >= 0 && f < nf && v->face_master[f] >= 0) cflags[v->face_master[f]] |= CF_RP;
    }
    // CF_EARLY: cells whose new state and geometry cache the next
    // moving-grid step reads before its face units: the four cells of every
    // tracked unit (both cells and both Sosed_down cells, mk2_recon_unit)
    // and, for every face of the three tracked lines and for its copy, the
    // master, the Sosed and the Sosed_down (face_tvd, surface_faces_kernel).
    // The pipelined step updates them first and moves the grid of the next
    // step while the other cells are updated.
    std::vector<int32_t> early;
    {
        auto mark = [&](int c) {
            if (c >= 0 && c < nc) cflags[c] |= CF_EARLY;
        };
        for (int u = u_tr0; u < u_tr1; u++) {
            const int g = u_slot[u];
            mark(u_cell[u]);
            mark(u_twin[u] >= 0 ? snb[g] : -1);
            mark(ssd[g]);
            mark(ssd2[g]);
        }
        const int32_t* lines[3] = {v->line_contact, v->line_inner, v->line_outer};
        const int nl[3] = {v->n_contact, v->n_inner_line, v->n_outer_line};
        for (int l = 0; l < 3; l++)
            for (int j = 0; j < nl[l]; j++) {
                const int f = lines[l][j];
                if (f < 0 || f >= nf) continue;
                for (const int ff : {f, v->face_copy[f]}) {
                    if (ff < 0 || ff >= nf) continue;
                    mark(v->face_master[ff]);
                    mark(v->face_sosed[ff]);
                    mark(fsdown[ff]);
                }
            }
        for (int c = 0; c < nc; c++)
            if (cflags[c] & CF_EARLY) early.push_back(c);
    }
    // surface-tracking nodes (see point_velocity)
    std::vector<int32_t> sp_point, sp_line, sp_inc, sp_ainc, sp_fix(12, 0);
    std::vector<int32_t> local(np, -1);
    {
        const int32_t* lines[3] = {v->line_contact, v->line_inner, v->line_outer};
        const int nl[3] = {v->n_contact, v->n_inner_line, v->n_outer_line};
        int base = 0;
        for (int L = 0; L < 3; L++) {
            for (int j = 0; j < nl[L]; j++) {
                const int f = lines[L][j];
                if (f < 0 || f >= nf) {
                    set_error("gelios_upload_topology: tracked-line face out of range");
                    return GELIOS_E_MESH;
                }
                const int ends[2] = {v->face_A[f], v->face_B[f]};
                for (int role = 0; role < 2; role++) {
                    const int p = ends[role];
                    int id = local[p];
                    if (id < 0) {
                        id = static_cast<int>(sp_point.size());
                        local[p] = id;
                        sp_point.push_back(p);
                        sp_line.push_back(L);
                        for (int k = 0; k < 4; k++) {
                            sp_inc.push_back(-1);
                            sp_ainc.push_back(-1);
                        }
                    } else if (sp_line[id] != L) {
                        set_error("gelios_upload_topology: a point lies on two tracked lines");
                        return GELIOS_E_MESH;
                    }
                    int k = 0;
                    while (k < 4 && sp_inc[4 * id + k] >= 0) k++;
                    if (k == 4) {
                        set_error("gelios_upload_topology: tracked-line point with more than 4 faces");
                        return GELIOS_E_MESH;
                    }
                    sp_inc[4 * id + k] = ((base + j) << 1) | role;
                    if (L == 0 && role == 0) {
                        int q = 0;
                        while (q < 4 && sp_ainc[4 * id + q] >= 0) q++;
                        if (q == 4) {
                            set_error("gelios_upload_topology: contact point is the A end of more than 4 faces");
                            return GELIOS_E_MESH;
                        }
                        sp_ainc[4 * id + q] = j;
                    }
                }
            }
            if (nl[L] > 0) {
                sp_fix[4 * L + 0] = local[v->face_A[lines[L][0]]];
                sp_fix[4 * L + 1] = local[v->face_B[lines[L][0]]];
                sp_fix[4 * L + 2] = local[v->face_A[lines[L][nl[L] - 1]]];
                sp_fix[4 * L + 3] = local[v->face_B[lines[L][nl[L] - 1]]];
            }
            base += nl[L];
        }
    }
    const int n_sp = static_cast<int>(sp_point.size());
    int rc = 0;
    rc |= upload(ctx->X, v->x, np, s);
    rc |= upload(ctx->Y, v->y, np, s);
    rc |= upload(ctx->X2, v->x, np, s);
    rc |= upload(ctx->Y2, v->y, np, s);
    rc |= upload(ctx->ptype, v->point_type, np, s);
    rc |= upload(ctx->cstart, v->contour_start, nc + 1, s);
    rc |= upload(ctx->contour, v->contour, v->contour_start[nc], s);
    {
        std::vector<int32_t> q(4 * static_cast<size_t>(nc), -1);
        for (int c = 0; c < nc; c++) {
            const int32_t s0 = v->contour_start[c];
            if (v->contour_start[c + 1] - s0 == 4)
                for (int k = 0; k < 4; k++) q[4 * static_cast<size_t>(c) + k] = v->contour[s0 + k];
        }
        rc |= upload(ctx->qcorner, q.data(), q.size(), s);
    }
    rc |= upload(ctx->gstart, v->gran_start, nc + 1, s);
    rc |= upload(ctx->cflags, cflags.data(), nc, s);
    rc |= upload(ctx->early, early.data(), early.size(), s);
    ctx->n_early = static_cast<int>(early.size());
    rc |= upload(ctx->ctype, v->cell_type, nc, s);
    rc |= upload<double>(ctx->hstate[0], nullptr, 16 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->hstate[1], nullptr, 16 * static_cast<size_t>(nc), s);
    rc |= upload(ctx->sA, sA.data(), ng, s);
    rc |= upload(ctx->sB, sB.data(), ng, s);
    rc |= upload(ctx->snb, snb.data(), ng, s);
    rc |= upload(ctx->ssd, ssd.data(), ng, s);
    rc |= upload(ctx->ssd2, ssd2.data(), ng, s);
    rc |= upload(ctx->sinfo, sinfo.data(), ng, s);
    rc |= upload(ctx->fA, v->face_A, nf, s);
    rc |= upload(ctx->fB, v->face_B, nf, s);
    rc |= upload(ctx->ftype, v->face_type, nf, s);
    rc |= upload(ctx->fmaster, v->face_master, nf, s);
    rc |= upload(ctx->fsosed, v->face_sosed, nf, s);
    rc |= upload(ctx->fcopy, v->face_copy, nf, s);
    rc |= upload(ctx->fsdown, fsdown, nf, s);
    const int nr = v->n_rails;
    if (nr > 0) {
        rc |= upload(ctx->rtype, v->rail_type, nr, s);
        rc |= upload(ctx->rM, v->rail_M, 4 * nr, s);
        rc |= upload(ctx->rpstart, v->rail_pstart, nr + 1, s);
        rc |= upload(ctx->rpts, v->rail_points, v->rail_pstart[nr], s);
        rc |= upload(ctx->rkstart, v->rail_kstart, nr + 1, s);
        rc |= upload(ctx->rkeys, v->rail_keys, v->rail_kstart[nr], s);
        rc |= upload(ctx->rs, v->rail_s, nr, s);
    }
    rc |= upload(ctx->lc, v->line_contact, v->n_contact, s);
    rc |= upload(ctx->li, v->line_inner, v->n_inner_line, s);
    rc |= upload(ctx->lo, v->line_outer, v->n_outer_line, s);
    rc |= upload(ctx->u_slot, u_slot.data(), u_slot.size(), s);
    {
        // unit-major copies of what a unit reads about its face and cells:
        // end points, slot info with both cells' flags, neighbour and the
        // two Sosed_down cells
        const size_t nu = u_slot.size();
        std::vector<int32_t> uA(nu), uB(nu), unb(nu), usd(nu), usd2(nu);
        std::vector<uint32_t> ui(nu);
        for (size_t u = 0; u < nu; u++) {
            const int g = u_slot[u];
            uA[u] = sA[g];
            uB[u] = sB[g];
            unb[u] = u_twin[u] >= 0 ? snb[g] : -1;
            usd[u] = ssd[g];
            usd2[u] = ssd2[g];
            const uint32_t nbf = unb[u] >= 0 ? cflags[unb[u]] : 0u;
            ui[u] = sinfo[g] | ((cflags[u_cell[u]] & 15u) << UI_CF_OWN) | ((nbf & 15u) << UI_CF_NB);
        }
        rc |= upload(ctx->u_A, uA.data(), nu, s);
        rc |= upload(ctx->u_B, uB.data(), nu, s);
        rc |= upload(ctx->u_info, ui.data(), nu, s);
        rc |= upload(ctx->u_nb, unb.data(), nu, s);
        rc |= upload(ctx->u_sd, usd.data(), nu, s);
        rc |= upload(ctx->u_sd2, usd2.data(), nu, s);
    }
    rc |= upload(ctx->u_cell, u_cell.data(), u_cell.size(), s);
    rc |= upload(ctx->u_twin, u_twin.data(), u_twin.size(), s);
    TileBuild tb;
    if (build_tiles(v, u_slot, u_cell, u_twin, snb, tb) != GELIOS_OK) {
        set_error("gelios_upload_topology: a tile of the moving-grid step has too many face slots");
        return GELIOS_E_LIMIT;
    }
    rc |= upload(ctx->t_cstart, tb.cstart.data(), tb.cstart.size(), s);
    rc |= upload(ctx->t_cells, tb.cells.data(), tb.cells.size(), s);
    rc |= upload(ctx->t_lbase, tb.lbase.data(), tb.lbase.size(), s);
    rc |= upload(ctx->t_fstart, tb.fstart.data(), tb.fstart.size(), s);
    rc |= upload(ctx->t_faces, tb.faces.data(), tb.faces.size(), s);
    rc |= upload<double>(ctx->flux, nullptr, 5 * static_cast<size_t>(ng), s);
    rc |= upload<double>(ctx->upf, nullptr, static_cast<size_t>(kUnitGeoRows) * u_slot.size(), s);
    rc |= upload<double>(ctx->aux, nullptr, 3 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->rec, nullptr, static_cast<size_t>(kRecRows) * (u_tr1 - u_tr0 + 1), s);
    rc |= upload<double>(ctx->pstar, nullptr, static_cast<size_t>(u_tr1 - u_tr0) + 1, s);
    rc |= upload(ctx->sp_point, sp_point.data(), sp_point.size(), s);
    rc |= upload(ctx->sp_line, sp_line.data(), sp_line.size(), s);
    rc |= upload(ctx->sp_inc, sp_inc.data(), sp_inc.size(), s);
    rc |= upload(ctx->sp_ainc, sp_ainc.data(), sp_ainc.size(), s);
    rc |= upload(ctx->sp_fix, sp_fix.data(), sp_fix.size(), s);
    rc |= upload(ctx->sp_of_point, local.data(), local.size(), s);
    rc |= upload<double>(ctx->Hn, nullptr, 4 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->Hu, nullptr, 4 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->Hv, nullptr, 4 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->HT, nullptr, 4 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->ku, nullptr, nc, s);
    rc |= upload<double>(ctx->kv, nullptr, nc, s);
    rc |= upload<double>(ctx->kT, nullptr, nc, s);
    rc |= upload(ctx->r_istoch, r_istoch, nc, s);
    rc |= upload(ctx->cback, cback, nc, s);
    rc |= upload(ctx->cnext, cnext, nc, s);
    // the bracket cache of the source interpolation needs doubly linked
    // chains with strictly increasing r_istoch along Next
    bool chains_ok = true;
    for (int c = 0; c < nc && chains_ok; c++) {
        const int nx = cnext[c], bk = cback[c];
        if (nx >= 0 && (cback[nx] != c || !(r_istoch[nx] > r_istoch[c]))) chains_ok = false;
        if (bk >= 0 && (cnext[bk] != c || !(r_istoch[bk] < r_istoch[c]))) chains_ok = false;
    }
    {
        std::vector<int32_t> minus1(nc, -1);
        std::vector<int32_t> minus1x2(2 * static_cast<size_t>(nc), -1);
        rc |= upload(ctx->src_lo, minus1x2.data(), minus1x2.size(), s);
    }
    rc |= upload<double>(ctx->state[0], nullptr, 5 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->state[1], nullptr, 5 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->cen[0], nullptr, 5 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->cen[1], nullptr, 5 * static_cast<size_t>(nc), s);
    rc |= upload<double>(ctx->surface, nullptr,
                         4 * (static_cast<size_t>(v->n_contact) + v->n_inner_line + v->n_outer_line) + 1, s);
    if (rc) return GELIOS_E_CUDA;
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    DevMesh& d = ctx->d;
    d = DevMesh();
    d.n_points = np;
    d.n_cells = nc;
    d.n_faces = nf;
    d.n_main = v->n_main;
    std::memcpy(d.dims, v->dims, sizeof(d.dims));
    d.X = ctx->X.as<double>();
    d.Y = ctx->Y.as<double>();
    d.X2 = ctx->X2.as<double>();
    d.Y2 = ctx->Y2.as<double>();
    d.ptype = ctx->ptype.as<int32_t>();
    d.r11_sq = sqrt_threshold(ctx->prm.R11);
    d.cstart = ctx->cstart.as<int32_t>();
    d.qcorner = reinterpret_cast<const int4*>(ctx->qcorner.as<int32_t>());
    d.contour = ctx->contour.as<int32_t>();
    d.gstart = ctx->gstart.as<int32_t>();
    d.cflags = ctx->cflags.as<uint32_t>();
    d.ctype = ctx->ctype.as<int32_t>();
    d.sA = ctx->sA.as<int32_t>();
    d.sB = ctx->sB.as<int32_t>();
    d.snb = ctx->snb.as<int32_t>();
    d.ssd = ctx->ssd.as<int32_t>();
    d.ssd2 = ctx->ssd2.as<int32_t>();
    d.sinfo = ctx->sinfo.as<uint32_t>();
    d.n_slots = ng;
    d.n_units = static_cast<int>(u_slot.size());
    d.u_slot = ctx->u_slot.as<int32_t>();
    d.u_A = ctx->u_A.as<int32_t>();
    d.u_B = ctx->u_B.as<int32_t>();
    d.u_info = ctx->u_info.as<uint32_t>();
    d.u_nb = ctx->u_nb.as<int32_t>();
    d.u_sd = ctx->u_sd.as<int32_t>();
    d.u_sd2 = ctx->u_sd2.as<int32_t>();
    d.u_cell = ctx->u_cell.as<int32_t>();
    d.u_twin = ctx->u_twin.as<int32_t>();
    d.u_c1 = u_c1;
    d.u_tr0 = u_tr0;
    d.u_tr1 = u_tr1;
    d.fA = ctx->fA.as<int32_t>();
    d.fB = ctx->fB.as<int32_t>();
    d.ftype = ctx->ftype.as<int32_t>();
    d.fmaster = ctx->fmaster.as<int32_t>();
    d.fsosed = ctx->fsosed.as<int32_t>();
    d.fcopy = ctx->fcopy.as<int32_t>();
    d.fsdown = ctx->fsdown.as<int32_t>();
    d.rtype = ctx->rtype.as<int32_t>();
    d.rM = ctx->rM.as<int32_t>();
    d.rpstart = ctx->rpstart.as<int32_t>();
    d.rpts = ctx->rpts.as<int32_t>();
    d.rkstart = ctx->rkstart.as<int32_t>();
    d.rkeys = ctx->rkeys.as<int32_t>();
    d.rs = ctx->rs.as<double>();
    d.n_rail_a = na;
    d.n_rail_b = nb;
    d.n_rail_c = ncr;
    d.n_rail_d = nd;
    d.lc = ctx->lc.as<int32_t>();
    d.li = ctx->li.as<int32_t>();
    d.lo = ctx->lo.as<int32_t>();
    d.n_lc = v->n_contact;
    d.n_li = v->n_inner_line;
    d.n_lo = v->n_outer_line;
    d.n_sp = n_sp;
    d.sp_point = ctx->sp_point.as<int32_t>();
    d.sp_line = ctx->sp_line.as<int32_t>();
    d.sp_inc = ctx->sp_inc.as<int32_t>();
    d.sp_ainc = ctx->sp_ainc.as<int32_t>();
    d.sp_fix = ctx->sp_fix.as<int32_t>();
    d.sp_of_point = ctx->sp_of_point.as<int32_t>();
    d.Hn = ctx->Hn.as<double>();
    d.Hu = ctx->Hu.as<double>();
    d.Hv = ctx->Hv.as<double>();
    d.HT = ctx->HT.as<double>();
    d.ku = ctx->ku.as<double>();
    d.kv = ctx->kv.as<double>();
    d.kT = ctx->kT.as<double>();
    d.r_istoch = ctx->r_istoch.as<double>();
    d.cback = ctx->cback.as<int32_t>();
    d.cnext = ctx->cnext.as<int32_t>();
    d.src_lo = chains_ok ? reinterpret_cast<const int2*>(ctx->src_lo.as<int32_t>()) : nullptr;
    d.src_lo_out = chains_ok ? reinterpret_cast<int2*>(ctx->src_lo.as<int32_t>()) : nullptr;
    ctx->tiles = TileView();
    ctx->tiles.n_tiles = static_cast<int>(tb.cstart.size()) - 1;
    ctx->tiles.max_slots = tb.max_slots;
    ctx->tiles.cstart = ctx->t_cstart.as<int32_t>();
    ctx->tiles.cells = ctx->t_cells.as<int32_t>();
    ctx->tiles.lbase = ctx->t_lbase.as<int32_t>();
    ctx->tiles.fstart = ctx->t_fstart.as<int32_t>();
    ctx->tiles.faces = ctx->t_faces.as<int2>();
    ctx->have_mesh = true;
    ctx->n_inner = 0;
    ctx->cen_valid = false;
    ctx->upf_valid = false;
    ctx->drop_graphs();
    return GELIOS_OK;
}

extern "C" int gelios_upload_state(gelios_ctx* ctx, int buf, const double* ro, const double* p, const double* u,
                                   const double* v, const double* Q) {
    if (!ctx || buf < 0 || buf > 1 || !ro || !p || !u || !v || !Q) return GELIOS_E_ARG;
    if (!ctx->have_mesh) {
        set_error("gelios_upload_state: no topology");
        return GELIOS_E_STATE;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * ctx->d.n_cells;
    const double* src[5] = {ro, p, u, v, Q};
    for (int k = 0; k < 5; k++)
        GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->field(buf, k), src[k], n, cudaMemcpyHostToDevice, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_download_state(gelios_ctx* ctx, int buf, double* ro, double* p, double* u, double* v,
                                     double* Q) {
    if (!ctx || buf < 0 || buf > 1 || !ro || !p || !u || !v || !Q) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * ctx->d.n_cells;
    double* dst[5] = {ro, p, u, v, Q};
    for (int k = 0; k < 5; k++)
        GELIOS_CUDA_TRY(cudaMemcpyAsync(dst[k], ctx->field(buf, k), n, cudaMemcpyDeviceToHost, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_set_mhd_params(gelios_ctx* ctx, const gelios_mhd_params* mp) {
    if (!ctx || !mp) return GELIOS_E_ARG;
    ctx->mprm = *mp;
    ctx->drop_graphs();  // the boundary data are kernel arguments
    return GELIOS_OK;
}

extern "C" int gelios_upload_mhd(gelios_ctx* ctx, int buf, const double* rows8) {
    if (!ctx || buf < 0 || buf > 1 || !rows8) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * 8 * ctx->d.n_cells;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->hstate[buf].p, rows8, n, cudaMemcpyHostToDevice, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_download_mhd(gelios_ctx* ctx, int buf, double* rows8) {
    if (!ctx || buf < 0 || buf > 1 || !rows8) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * 8 * ctx->d.n_cells;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(rows8, ctx->hstate[buf].p, n, cudaMemcpyDeviceToHost, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_upload_sources(gelios_ctx* ctx, const double* q1, const double* q2, const double* q3) {
    if (!ctx || !q1 || !q2 || !q3) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t nc = ctx->d.n_cells;
    if (ctx->src_fixed.bytes != 3 * nc * sizeof(double)) {
        ctx->drop_graphs();  // they hold the buffer about to be replaced
        if (ctx->src_fixed.alloc(3 * nc * sizeof(double))) return GELIOS_E_CUDA;
    }
    const double* q[3] = {q1, q2, q3};
    for (int k = 0; k < 3; k++)
        GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->src_fixed.as<double>() + k * nc, q[k], nc * sizeof(double),
                                        cudaMemcpyHostToDevice, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_upload_hydrogen(gelios_ctx* ctx, int buf, const double* rows16) {
    if (!ctx || buf < 0 || buf > 1 || !rows16) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * 16 * ctx->d.n_cells;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->hstate[buf].p, rows16, n, cudaMemcpyHostToDevice, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_download_hydrogen(gelios_ctx* ctx, int buf, double* rows16) {
    if (!ctx || buf < 0 || buf > 1 || !rows16) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * 16 * ctx->d.n_cells;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(rows16, ctx->hstate[buf].p, n, cudaMemcpyDeviceToHost, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_upload_mc(gelios_ctx* ctx, const double* Hn, const double* Hu, const double* Hv,
                                const double* HT, const double* ku, const double* kv, const double* kT) {
    if (!ctx || !Hn || !Hu || !Hv || !HT || !ku || !kv || !kT) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * ctx->d.n_cells;
    cudaStream_t s = ctx->stream;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->Hn.p, Hn, 4 * n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->Hu.p, Hu, 4 * n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->Hv.p, Hv, 4 * n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->HT.p, HT, 4 * n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->ku.p, ku, n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->kv.p, kv, n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->kT.p, kT, n, cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    return GELIOS_OK;
}

extern "C" int gelios_set_inner_cells(gelios_ctx* ctx, const int32_t* cells, int32_t n) {
    if (!ctx || n < 0 || (n > 0 && !cells)) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    for (int i = 0; i < n; i++)
        if (cells[i] < 0 || cells[i] >= ctx->d.n_cells) {
            set_error("gelios_set_inner_cells: cell index out of range");
            return GELIOS_E_ARG;
        }
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    if (upload(ctx->inner, cells, n, ctx->stream)) return GELIOS_E_CUDA;
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    ctx->n_inner = n;
    return GELIOS_OK;
}

namespace {

// Enqueues one moving-grid step on the context's streams; returns the
// number of kernels launched, or a negative error code.
int enqueue_mk2(gelios_ctx* ctx, const StepBuffers& b) {
    const DevMesh& d = ctx->d;
    const gelios_params& P = ctx->prm;
    cudaStream_t s = ctx->stream;
    // Two streams per step.
    //   side: the tracked face units' reconstructions and the star pressures
    //         of their exact Riemann problems, the charge-exchange source
    //         terms (none depends on the motion), then, once the rails have
    //         moved, the tracked-face fluxes (sampling of the solved Riemann
    //         problems at the face speed) and the C_1 interior and one-sided
    //         face units;
    //   main: surface tracking + rails, the plain interior face units, then
    //         (once the side stream is done) the cell update; the commit.
    //         The tile variants do the plain units' work inside the update.
    cudaStream_t sd = ctx->side;
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_fork, s));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sd, ctx->ev_fork, 0));
    launch_mk2_recon(d, P, b, ctx->rec.as<double>(), sd);
    const int nsv = launch_mk2_tracked_solve(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(), sd);
    launch_mk2_source(d, P, b, ctx->aux.as<double>(), sd);
    cudaEvent_t e1 = ctx->phase_begin();
    const int nm = launch_motion(d, P, b, ctx->surface.as<double>(), s);
    ctx->phase_end(2, e1, nm);  // Move_surface + rails
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_rails, s));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sd, ctx->ev_rails, 0));
    const int nft = launch_mk2_flux_tracked(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(),
                                            ctx->flux.as<double>(), sd);
    // the smaller unit groups (C_1 interior, one-sided) beside the plain group
    GELIOS_CUDA_TRY(
        launch_mk2_cells(d, P, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), sd, ctx->mk2_variant, 3));
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_tracked, sd));
    cudaEvent_t e3 = ctx->phase_begin();
    GELIOS_CUDA_TRY(
        launch_mk2_cells(d, P, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), s, ctx->mk2_variant, 1));
    // the cell update reads every face's flux and the source terms
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_tracked, 0));
    GELIOS_CUDA_TRY(
        launch_mk2_cells(d, P, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), s, ctx->mk2_variant, 2));
    const int ncl = mk2_variant_launches(d, ctx->mk2_variant, 1) + mk2_variant_launches(d, ctx->mk2_variant, 2) +
                    mk2_variant_launches(d, ctx->mk2_variant, 3);
    ctx->phase_end(1, e3, ncl + nft);  // face units + cell update
    cudaEvent_t e4 = ctx->phase_begin();
    launch_commit(d, b, s);
    ctx->phase_end(4, e4, 1);
    GELIOS_CUDA_TRY(cudaGetLastError());
    return (d.u_tr1 > d.u_tr0 ? 1 : 0) + nsv + 1 + nm + nft + ncl + 1;
}

// Enqueues one step of the MHD + pickup form on the main stream: Move_surface
// + rails, the face units, the cell update, the commit.
int enqueue_mhd(gelios_ctx* ctx, const StepBuffers& b) {
    const DevMesh& d = ctx->d;
    const gelios_params& P = ctx->prm;
    cudaStream_t s = ctx->stream;
    const int cur = b.cur[0] == ctx->field(0, 0) ? 0 : 1, nxt = cur ^ 1;
    cudaEvent_t e1 = ctx->phase_begin();
    const int nm = launch_motion(d, P, b, ctx->surface.as<double>(), s);
    ctx->phase_end(2, e1, nm);
    cudaEvent_t e3 = ctx->phase_begin();
    // the plain interior face units on the main stream, the other groups
    // (C_1, tracked, one-sided units) beside them on the side stream
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_fork, s));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
    const int nfc = launch_mhd_faces(d, P, ctx->mprm, b, ctx->hstate[cur].as<double>(), ctx->flux_mhd.as<double>(),
                                     s, ctx->mhd_face_variant, ctx->side);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_tracked, ctx->side));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_tracked, 0));
    ctx->phase_end(1, e3, nfc);
    cudaEvent_t e5 = ctx->phase_begin();
    launch_mhd_update(d, P, b, ctx->flux_mhd.as<double>(), ctx->src_fixed.as<double>(), ctx->hstate[cur].as<double>(),
                      ctx->hstate[nxt].as<double>(), s);
    ctx->phase_end(3, e5, 1);
    cudaEvent_t e4 = ctx->phase_begin();
    launch_commit(d, b, s);
    ctx->phase_end(4, e4, 1);
    GELIOS_CUDA_TRY(cudaGetLastError());
    return nm + nfc + 2;
}

int enqueue_form(gelios_ctx* ctx, const StepBuffers& b, int form) {
    return form == GELIOS_FORM_MHD_PUI ? enqueue_mhd(ctx, b) : enqueue_mk2(ctx, b);
}

// Replays the instantiated graph keyed by (form, kind, first, parity,
// centroid buffer), or captures `enqueue` (which enqueues on ctx->stream,
// may fork to the other streams and join them back, and returns its kernel
// count or a negative error code) into a new one and launches it.  Launches
// directly while phase timing is on or once a capture has failed.
template <class F>
int graph_or_direct(gelios_ctx* ctx, int form, int kind, bool first, int parity, const void* cen, F&& enqueue) {
    if (ctx->timing || ctx->graphs_off) return enqueue();
    for (auto& g : ctx->graphs)
        if (g.exec && g.form == form && g.kind == kind && g.first == static_cast<int>(first) && g.parity == parity &&
            g.cen == cen) {
            GELIOS_CUDA_TRY(cudaGraphLaunch(g.exec, ctx->stream));
            return g.launches;
        }
    cudaStream_t s = ctx->stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        ctx->graphs_off = true;
        return enqueue();
    }
    const int n = enqueue();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &graph);
    cudaGraphExec_t exec = nullptr;
    if (n < 0 || e != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        ctx->graphs_off = true;
        return enqueue();
    }
    cudaGraphDestroy(graph);
    gelios_ctx::StepGraph* slot = &ctx->graphs[0];
    for (auto& g : ctx->graphs)
        if (!g.exec) {
            slot = &g;
            break;
        }
    if (slot->exec) cudaGraphExecDestroy(slot->exec);
    slot->form = form;
    slot->kind = kind;
    slot->first = first;
    slot->parity = parity;
    slot->cen = cen;
    slot->exec = exec;
    slot->launches = n;
    GELIOS_CUDA_TRY(cudaGraphLaunch(exec, s));
    return n;
}

// One moving-grid step (MK2 or MHD form) as one graph: the instantiated graph
// of this form and these buffers (captured on first use), or direct launches
// while phase timing is on or if capture is unavailable.  Returns the kernel
// count or a negative error code.
// first: the first step of a call, whose graph begins with the initialisation
// of the dt / status words (one launch per step, not two).
int step_graph(gelios_ctx* ctx, const StepBuffers& b, int form, bool first) {
    const int parity = b.cur[0] == ctx->field(0, 0) ? 0 : 1;
    return graph_or_direct(ctx, form, 0, first, parity, b.cx, [&]() {
        if (first) launch_words_init(ctx->words.p, ctx->prm.dt0, ctx->stream);
        const int m = enqueue_form(ctx, b, form);
        return m < 0 ? m : m + (first ? 1 : 0);
    });
}

// ---- the pipelined moving-grid call
// A call of N steps runs as head(0), body(0), ..., body(N-2), last(N-1),
// each part one graph (or direct launches):
//   head(n): the tracked-face reconstructions and star pressures of step n
//            (side stream) and its motion: surface tracking + rails (motion
//            stream);
//   body(n): step n's source terms, tracked-face fluxes and C_1 / one-sided
//            face units (side) beside its plain face units (main); the
//            update of the CF_EARLY cells; then the dt of step n+1 and its
//            motion (motion stream) and its tracked-face reconstructions and
//            star pressures (side) while the main stream updates every other
//            cell of step n;
//   last(n): as body(n) without step n+1: one update of every cell, then the
//            commit (x = x2) and the dt that follows.
// The motion of a step is a chain of latency-bound kernels on few SMs; here
// it runs beside the memory-bound update of the step before instead of in
// front of the face units.  It reads only the CF_EARLY cells of that step
// (state, centroids, |c|^(2 gamma)), the points the step before moved and
// its dt.  The points are double-buffered: step n reads the points before
// its motion from X (n even) or X2 (n odd) and moves them into the other
// buffer, so step n+1's rails never overwrite points that step n's update
// still reads; the commit of the last step leaves the final points in X.
// The 1e7 start of the CFL minimum is folded in where dt is finalised
// (dt_finalize_cap) instead of by the update, so step n+1's dt is final once
// step n's face units are done.  The results are the bits of the
// one-graph-per-step arrangement (tested).
DevMesh pipe_mesh(const gelios_ctx* ctx, int st) {
    DevMesh d = ctx->d;
    if (st & 1) {
        std::swap(d.X, d.X2);
        std::swap(d.Y, d.Y2);
    }
    return d;
}

// Buffers of step st of a moving-grid call: state par[st & 1] -> par[st & 1
// ^ 1], the geometry cache of the current points in cen0 (st even) or cen1.
StepBuffers mk2_buffers(gelios_ctx* ctx, int st, double* cen0, double* cen1) {
    const size_t nc = ctx->d.n_cells;
    const int cur = st & 1, nxt = cur ^ 1;
    StepBuffers b;
    for (int k = 0; k < 5; k++) {
        b.cur[k] = ctx->field(cur, k);
        b.nxt[k] = ctx->field(nxt, k);
    }
    b.dt_cur = ctx->T() + cur;
    b.dt_next = ctx->T() + nxt;
    b.dt_acc = ctx->acc();
    b.counters = ctx->counters();
    b.status = ctx->status();
    double* cc = cur ? cen1 : cen0;
    double* cn = cur ? cen0 : cen1;
    b.cx = cc;
    b.cy = cc + nc;
    b.rp = cc + 2 * nc;
    b.vs = cc + 3 * nc;
    b.vol = cc + 4 * nc;
    b.cx_next = cn;
    b.cy_next = cn + nc;
    b.rp_next = cn + 2 * nc;
    b.vs_next = cn + 3 * nc;
    b.vol_next = cn + 4 * nc;
    return b;
}

int enqueue_pipe_head(gelios_ctx* ctx, int st, const StepBuffers& b, bool first) {
    const DevMesh d = pipe_mesh(ctx, st);
    const gelios_params& P = ctx->prm;
    cudaStream_t s = ctx->stream, sd = ctx->side, sm = ctx->motion;
    int n = 0;
    if (first) {
        launch_words_init(ctx->words.p, P.dt0, s);
        n++;
    }
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_fork, s));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sd, ctx->ev_fork, 0));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sm, ctx->ev_fork, 0));
    launch_mk2_recon(d, P, b, ctx->rec.as<double>(), sd);
    n += d.u_tr1 > d.u_tr0 ? 1 : 0;
    n += launch_mk2_tracked_solve(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(), sd);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_side2, sd));
    n += launch_motion(d, P, b, ctx->surface.as<double>(), sm);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_motion, sm));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_side2, 0));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_motion, 0));
    GELIOS_CUDA_TRY(cudaGetLastError());
    return n;
}

// body(st) when bn (the buffers of step st + 1) is given, last(st) otherwise
int enqueue_pipe_step(gelios_ctx* ctx, int st, const StepBuffers& b, const StepBuffers* bn) {
    const DevMesh d = pipe_mesh(ctx, st);
    const gelios_params& P = ctx->prm;
    const int v = ctx->mk2_variant;
    cudaStream_t s = ctx->stream, sd = ctx->side, sm = ctx->motion;
    double* fl = ctx->flux.as<double>();
    double* aux = ctx->aux.as<double>();
    int n = 0;
    // the tracked-face fluxes, then the source terms, on the (high-priority)
    // motion stream, idle until step st's early update; the C_1 interior
    // and one-sided face-unit groups on the groups stream, the plain face
    // units on the main stream.  The next step's tracked reconstructions
    // (side stream) overwrite the rows the tracked fluxes read: they wait
    // for the early update, which waits for the motion stream.
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_fork, s));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sm, ctx->ev_fork, 0));
    n += launch_mk2_flux_tracked(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(), fl, sm);
    launch_mk2_source(d, P, b, aux, sm);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_motion, sm));
    n++;
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(ctx->groups, ctx->ev_fork, 0));
    GELIOS_CUDA_TRY(launch_mk2_cells(d, P, b, ctx->tiles, fl, aux, ctx->groups, v, 3));
    n += mk2_variant_launches(d, v, 3);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_groups, ctx->groups));
    GELIOS_CUDA_TRY(launch_mk2_cells(d, P, b, ctx->tiles, fl, aux, s, v, 1));
    n += mk2_variant_launches(d, v, 1);
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_groups, 0));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_motion, 0));
    if (!bn) {
        launch_mk2_update(d, P, b, fl, aux, s, 3, nullptr, 0);
        launch_commit(d, b, s, true);
        GELIOS_CUDA_TRY(cudaGetLastError());
        return n + 2;
    }
    const DevMesh dn = pipe_mesh(ctx, st + 1);
    const int32_t* early = ctx->early.as<int32_t>();
    launch_mk2_update(d, P, b, fl, aux, s, 1, early, ctx->n_early);
    n += ctx->n_early > 0 ? 1 : 0;
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_early, s));
    // step st + 1: dt, then surface tracking + rails
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sm, ctx->ev_early, 0));
    launch_dt_finalize_cap(b, sm);
    n++;
    n += launch_motion(dn, P, *bn, ctx->surface.as<double>(), sm);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_motion, sm));
    // step st + 1: tracked-face reconstructions and star pressures
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(sd, ctx->ev_early, 0));
    launch_mk2_recon(dn, P, *bn, ctx->rec.as<double>(), sd);
    n += dn.u_tr1 > dn.u_tr0 ? 1 : 0;
    n += launch_mk2_tracked_solve(dn, P, *bn, ctx->rec.as<double>(), ctx->pstar.as<double>(), sd);
    GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_side2, sd));
    // step st: the other cells
    launch_mk2_update(d, P, b, fl, aux, s, 2, early, ctx->n_early);
    n++;
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_motion, 0));
    GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_side2, 0));
    GELIOS_CUDA_TRY(cudaGetLastError());
    return n;
}

bool pipe_ok(const gelios_ctx* ctx) {
    const int v = ctx->mk2_variant;
    return ctx->pipelined && !ctx->timing && !(v >= 4 && v < 8);
}

// nsteps (> 0) moving-grid steps as one pipelined call; returns the kernel
// count or a negative error code
int mk2_pipelined(gelios_ctx* ctx, int nsteps, double* cen0, double* cen1) {
    int launches = 0;
    StepBuffers b = mk2_buffers(ctx, 0, cen0, cen1);
    int n = graph_or_direct(ctx, GELIOS_FORM_MK2, 1, true, 0, b.cx,
                            [&]() { return enqueue_pipe_head(ctx, 0, b, true); });
    if (n < 0) return n;
    launches += n;
    for (int st = 0; st < nsteps; st++) {
        const bool last = st + 1 == nsteps;
        const StepBuffers bn = last ? b : mk2_buffers(ctx, st + 1, cen0, cen1);
        n = graph_or_direct(ctx, GELIOS_FORM_MK2, last ? 3 : 2, false, st & 1, b.cx,
                            [&]() { return enqueue_pipe_step(ctx, st, b, last ? nullptr : &bn); });
        if (n < 0) return n;
        launches += n;
        b = bn;
    }
    return launches;
}

}  // namespace

extern "C" int gelios_step(gelios_ctx* ctx, int form, int nsteps, gelios_status* status) {
    if (!ctx || nsteps < 0) return GELIOS_E_ARG;
    if (form != GELIOS_FORM_STATIONARY && form != GELIOS_FORM_MK2 && form != GELIOS_FORM_INNER_MK2 &&
        form != GELIOS_FORM_5_KOMPONENT && form != GELIOS_FORM_MHD_PUI) {
        set_error("gelios_step: unknown form");
        return GELIOS_E_ARG;
    }
    if (!ctx->have_mesh) {
        set_error("gelios_step: no topology uploaded");
        return GELIOS_E_STATE;
    }
    const DevMesh& d = ctx->d;
    const bool mhd = form == GELIOS_FORM_MHD_PUI;
    const bool moving = form == GELIOS_FORM_MK2 || form == GELIOS_FORM_5_KOMPONENT || mhd;
    if (moving && (d.n_rail_a + d.n_rail_b + d.n_rail_c + d.n_rail_d == 0 || d.n_lc == 0)) {
        set_error("gelios_step: the moving-grid form needs rails and tracked lines");
        return GELIOS_E_MESH;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const gelios_params& P = ctx->prm;
    // T[0] = T[1] = dt0, accumulator = +inf, counters = 0, status = 0
    struct Words {
        double T[2];
        unsigned long long acc;
        unsigned long long counters[2];
        int status;
        int pad[5];
    };
    static_assert(sizeof(Words) == 64, "device word layout");
    // the moving-grid and MHD forms initialise the words in their first
    // step (inside its graph); the others here
    const bool graph_form = form == GELIOS_FORM_MK2 || mhd;
    int64_t launches = 0;
    if (!graph_form || nsteps == 0) {
        launch_words_init(ctx->words.p, P.dt0, s);
        launches = 1;
    }
    double* cen0 = ctx->cen[0].as<double>();
    double* cen1 = ctx->cen[1].as<double>();
    if (ctx->ev_used > 4096) ctx->collect();
    const size_t ncz = d.n_cells;
    if (mhd && ctx->src_fixed.bytes != 3 * ncz * sizeof(double)) {
        set_error("gelios_step: the MHD form needs gelios_upload_sources");
        return GELIOS_E_STATE;
    }
    if (mhd || form == GELIOS_FORM_5_KOMPONENT) {
        // wide flux slots of the multi-fluid forms (13 or 21 rows)
        const int rows = mhd ? kMhdFluxRows : kK5FluxRows;
        const size_t fb = static_cast<size_t>(rows) * d.n_slots * sizeof(double);
        if (ctx->flux_mhd.bytes != fb) {
            ctx->drop_graphs();
            if (ctx->flux_mhd.alloc(fb)) return GELIOS_E_CUDA;
        }
    }
    // forms whose update refills the geometry cache (|c|^(2 gamma) only where read)
    const bool cached_form = form == GELIOS_FORM_MK2 || mhd || form == GELIOS_FORM_5_KOMPONENT;
    if (!ctx->cen_valid || (!cached_form && ctx->cen_rp_partial)) {
        cudaEvent_t e0 = ctx->phase_begin();
        launch_centroid(d, d.X, d.Y, cen0, cen0 + ncz, cen0 + 2 * ncz, P.gamma, s, cen0 + 3 * ncz, cen0 + 4 * ncz);
        ctx->phase_end(0, e0, 1);
        launches++;
        ctx->cen_rp_partial = false;
    }
    if (form == GELIOS_FORM_STATIONARY && !ctx->upf_valid && nsteps > 0) {
        launch_unit_geometry(d, P.gamma, cen0, cen0 + ncz, ctx->upf.as<double>(), s);
        launches++;
        ctx->upf_valid = true;
    }
    int first = 0;
    if (form == GELIOS_FORM_STATIONARY && nsteps > 0 && !ctx->timing && !ctx->coop_off) {
        // all steps of the plain form in one cooperative launch
        StepBuffers bb[2];
        for (int par = 0; par < 2; par++) {
            StepBuffers& b = bb[par];
            for (int k = 0; k < 5; k++) {
                b.cur[k] = ctx->field(par, k);
                b.nxt[k] = ctx->field(par ^ 1, k);
            }
            b.dt_cur = ctx->T() + par;
            b.dt_next = ctx->T() + (par ^ 1);
            b.dt_acc = ctx->acc();
            b.counters = ctx->counters();
            b.status = ctx->status();
            b.cx = cen0;
            b.cy = cen0 + ncz;
            b.rp = cen0 + 2 * ncz;
            b.vs = cen0 + 3 * ncz;
            b.upf = ctx->upf.as<double>();
            b.ugeo = b.upf + d.n_units;
        }
        if (launch_stationary_persistent(d, P, bb[0], bb[1], ctx->flux.as<double>(), nsteps, s) == cudaSuccess) {
            launches += 1;
            first = nsteps;
        } else {
            cudaGetLastError();
            ctx->coop_off = true;
        }
    }
    // a one-step call has no next step to overlap: one graph per step
    if (form == GELIOS_FORM_MK2 && nsteps > 1 && pipe_ok(ctx)) {
        const int n = mk2_pipelined(ctx, nsteps, cen0, cen1);
        if (n < 0) return n;
        launches += n;
        first = nsteps;
    }
    for (int st = first; st < nsteps; st++) {
        const int cur = st & 1, nxt = cur ^ 1;
        StepBuffers b;
        for (int k = 0; k < 5; k++) {
            b.cur[k] = ctx->field(cur, k);
            b.nxt[k] = ctx->field(nxt, k);
        }
        b.dt_cur = ctx->T() + cur;
        b.dt_next = ctx->T() + nxt;
        b.dt_acc = ctx->acc();
        b.counters = ctx->counters();
        b.status = ctx->status();
        if (mhd) {
            // moving-grid step of the MHD form on the main stream:
            // Move_surface + rails, face units, cell update, x = x2
            double* cc = (st & 1) ? cen1 : cen0;
            double* cn = (st & 1) ? cen0 : cen1;
            b.cx = cc;
            b.cy = cc + ncz;
            b.rp = cc + 2 * ncz;
            b.vs = cc + 3 * ncz;
            b.vol = cc + 4 * ncz;
            b.cx_next = cn;
            b.cy_next = cn + ncz;
            b.rp_next = cn + 2 * ncz;
            b.vs_next = cn + 3 * ncz;
            b.vol_next = cn + 4 * ncz;
            const int n = step_graph(ctx, b, GELIOS_FORM_MHD_PUI, st == 0);
            if (n < 0) return n;
            launches += n;
        } else if (form == GELIOS_FORM_MK2) {
            double* cc = (st & 1) ? cen1 : cen0;
            double* cn = (st & 1) ? cen0 : cen1;
            b.cx = cc;
            b.cy = cc + d.n_cells;
            b.rp = cc + 2 * static_cast<size_t>(d.n_cells);
            b.vs = cc + 3 * ncz;
            b.vol = cc + 4 * ncz;
            b.cx_next = cn;
            b.cy_next = cn + d.n_cells;
            b.rp_next = cn + 2 * static_cast<size_t>(d.n_cells);
            b.vs_next = cn + 3 * ncz;
            b.vol_next = cn + 4 * ncz;
            const int n = step_graph(ctx, b, GELIOS_FORM_MK2, st == 0);
            if (n < 0) return n;
            launches += n;
        } else if (form == GELIOS_FORM_5_KOMPONENT) {
            // Move_surface + Move_Setka_Calculate, the face units and the
            // five-fluid cell update (which refills the geometry cache for
            // the next step, like the moving-grid form), x = x2
            double* cc = (st & 1) ? cen1 : cen0;
            double* cn = (st & 1) ? cen0 : cen1;
            b.cx = cc;
            b.cy = cc + ncz;
            b.rp = cc + 2 * ncz;
            b.vs = cc + 3 * ncz;
            b.vol = cc + 4 * ncz;
            b.cx_next = cn;
            b.cy_next = cn + ncz;
            b.rp_next = cn + 2 * ncz;
            b.vs_next = cn + 3 * ncz;
            b.vol_next = cn + 4 * ncz;
            cudaEvent_t e1 = ctx->phase_begin();
            const int nm = launch_motion(d, P, b, ctx->surface.as<double>(), s, false);
            ctx->phase_end(2, e1, nm);
            cudaEvent_t e3 = ctx->phase_begin();
            launch_k5(d, P, b, ctx->hstate[cur].as<double>(), ctx->hstate[nxt].as<double>(), ctx->flux_mhd.as<double>(),
                      s);
            ctx->phase_end(3, e3, 2);
            cudaEvent_t e4 = ctx->phase_begin();
            launch_commit(d, b, s);
            ctx->phase_end(4, e4, 1);
            launches += nm + 3;
        } else {
            b.cx = cen0;
            b.cy = cen0 + d.n_cells;
            b.rp = cen0 + 2 * static_cast<size_t>(d.n_cells);
            if (form == GELIOS_FORM_STATIONARY) {
                b.vs = cen0 + 3 * static_cast<size_t>(d.n_cells);
                b.upf = ctx->upf.as<double>();
                b.ugeo = b.upf + d.n_units;
                cudaEvent_t e1 = ctx->phase_begin();
                launch_stationary_units(d, P, b, ctx->flux.as<double>(), s);
                ctx->phase_end(1, e1, 1);
                cudaEvent_t e3 = ctx->phase_begin();
                launch_stationary_update(d, P, b, ctx->flux.as<double>(), s);
                ctx->phase_end(3, e3, 1);
                launches += 2;
            } else {
                cudaEvent_t e3 = ctx->phase_begin();
                launch_inner(d, P, b, ctx->inner.as<int32_t>(), ctx->n_inner, s);
                ctx->phase_end(3, e3, 1);
                launches += 1;
            }
            cudaEvent_t e4 = ctx->phase_begin();
            launch_dt_finalize(b, s);
            ctx->phase_end(4, e4, 1);
            launches += 1;
        }
    }
    GELIOS_CUDA_TRY(cudaGetLastError());
    ctx->launches = launches;
    // centroids of the current points: after an odd number of moving-grid
    // steps they sit in the second buffer; swap so cen[0] holds them
    if (cached_form && (nsteps & 1)) std::swap(ctx->cen[0].p, ctx->cen[1].p);
    ctx->cen_valid = true;
    if (cached_form && nsteps > 0) {
        ctx->cen_rp_partial = true;
        ctx->upf_valid = false;
    }
    if (status) {
        Words r{};
        GELIOS_CUDA_TRY(cudaMemcpyAsync(&r, ctx->words.p, sizeof(r), cudaMemcpyDeviceToHost, s));
        GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
        std::memset(status, 0, sizeof(*status));
        status->flags = r.status;
        status->steps_done = nsteps;
        status->n_ro_clamp = static_cast<int64_t>(r.counters[0]);
        status->n_p_clamp = static_cast<int64_t>(r.counters[1]);
        status->result_buf = nsteps & 1;
        status->dt = r.T[nsteps & 1];
        if (!(status->dt == status->dt)) status->flags |= ST_DT_BAD;
    }
    return GELIOS_OK;
}

extern "C" int gelios_residual(gelios_ctx* ctx, int result_buf, double* residual) {
    if (!ctx || !residual || result_buf < 0 || result_buf > 1) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t need = kResidualScratch * sizeof(double);
    if (ctx->resid.bytes != need && ctx->resid.alloc(need)) return GELIOS_E_CUDA;
    cudaStream_t s = ctx->stream;
    launch_residual(ctx->field(result_buf, 0), ctx->field(result_buf ^ 1, 0), ctx->d.n_cells, ctx->resid.as<double>(),
                    s);
    double r[2] = {0.0, 0.0};
    GELIOS_CUDA_TRY(cudaMemcpyAsync(r, ctx->resid.p, sizeof(r), cudaMemcpyDeviceToHost, s));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    *residual = r[1] > 0.0 ? r[0] / r[1] : 0.0;
    return GELIOS_OK;
}

extern "C" int gelios_operator_residual(gelios_ctx* ctx, int form, int buf, double* residual) {
    if (!ctx || !residual || buf < 0 || buf > 1) return GELIOS_E_ARG;
    if (form != GELIOS_FORM_MK2 && form != GELIOS_FORM_MHD_PUI) {
        set_error("gelios_operator_residual: the moving-grid forms only (MK2, MHD + pickup)");
        return GELIOS_E_ARG;
    }
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    const bool mhd = form == GELIOS_FORM_MHD_PUI;
    const DevMesh& d = ctx->d;
    if (d.n_rail_a + d.n_rail_b + d.n_rail_c + d.n_rail_d == 0 || d.n_lc == 0) {
        set_error("gelios_operator_residual: the moving-grid form needs rails and tracked lines");
        return GELIOS_E_MESH;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const size_t need = (kResidualScratch + 8) * sizeof(double);
    if (ctx->resid.bytes < need && ctx->resid.alloc(need)) return GELIOS_E_CUDA;
    if (mhd) {
        const size_t fb = static_cast<size_t>(kMhdFluxRows) * d.n_slots * sizeof(double);
        if (ctx->flux_mhd.bytes != fb) {
            ctx->drop_graphs();  // they hold the buffer about to be replaced
            if (ctx->flux_mhd.alloc(fb)) return GELIOS_E_CUDA;
        }
    }
    const gelios_params& P = ctx->prm;
    const size_t nc = d.n_cells;
    double* cen0 = ctx->cen[0].as<double>();
    if (!ctx->cen_valid) {
        launch_centroid(d, d.X, d.Y, cen0, cen0 + nc, cen0 + 2 * nc, P.gamma, s, cen0 + 3 * nc, cen0 + 4 * nc);
        ctx->cen_valid = true;
        ctx->cen_rp_partial = false;
    }
    // the grid held still: moved points = current points, so every face
    // speed is 0; dt = 1 (it only divides the zero displacement) and CFL /
    // status words in scratch, so the context's own words stay untouched
    double* sc = ctx->resid.as<double>();
    double* words = sc + kResidualScratch;
    struct Words {
        double dt;
        unsigned long long acc;
        unsigned long long counters[2];
        int status;
        int pad[7];
    } w{};
    w.dt = 1.0;
    w.acc = 0x7ff0000000000000ULL;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(words, &w, sizeof(w), cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(d.X2, d.X, d.n_points * sizeof(double), cudaMemcpyDeviceToDevice, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(d.Y2, d.Y, d.n_points * sizeof(double), cudaMemcpyDeviceToDevice, s));
    StepBuffers b;
    for (int k = 0; k < 5; k++) {
        b.cur[k] = ctx->field(buf, k);
        b.nxt[k] = ctx->field(buf ^ 1, k);
    }
    b.dt_cur = words;
    b.dt_next = words;
    b.dt_acc = reinterpret_cast<unsigned long long*>(words + 1);
    b.counters = reinterpret_cast<unsigned long long*>(words + 2);
    b.status = reinterpret_cast<int*>(words + 4);
    b.cx = cen0;
    b.cy = cen0 + nc;
    b.rp = cen0 + 2 * nc;
    b.vs = cen0 + 3 * nc;
    b.vol = cen0 + 4 * nc;
    double* fl;
    if (mhd) {
        // the MHD form's face units (ion HLLD, pickup HLLC) into its 13 flux
        // rows; row 0 is the ion mass flux, state row 0 the ion density
        fl = ctx->flux_mhd.as<double>();
        launch_mhd_faces(d, P, ctx->mprm, b, ctx->hstate[buf].as<double>(), fl, s, ctx->mhd_face_variant);
    } else {
        const int v = (ctx->mk2_variant >= 4 && ctx->mk2_variant < 8) ? 0 : ctx->mk2_variant;
        fl = ctx->flux.as<double>();
        launch_mk2_recon(d, P, b, ctx->rec.as<double>(), s);
        launch_mk2_tracked_solve(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(), s);
        launch_mk2_flux_tracked(d, P, b, ctx->rec.as<double>(), ctx->pstar.as<double>(), fl, s);
        GELIOS_CUDA_TRY(launch_mk2_cells(d, P, b, ctx->tiles, fl, ctx->aux.as<double>(), s, v, 1));
        GELIOS_CUDA_TRY(launch_mk2_cells(d, P, b, ctx->tiles, fl, ctx->aux.as<double>(), s, v, 3));
    }
    launch_op_residual(d, P, b, fl, sc, s);
    GELIOS_CUDA_TRY(cudaGetLastError());
    double r[2] = {0.0, 0.0};
    GELIOS_CUDA_TRY(cudaMemcpyAsync(r, sc, sizeof(r), cudaMemcpyDeviceToHost, s));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    *residual = r[1] > 0.0 ? r[0] / r[1] : 0.0;
    return GELIOS_OK;
}

extern "C" int gelios_mk2_source_terms(gelios_ctx* ctx, int buf, double* q1, double* q2, double* q3) {
    if (!ctx || !q1 || !q2 || !q3 || buf < 0 || buf > 1) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const DevMesh& d = ctx->d;
    const gelios_params& P = ctx->prm;
    const size_t nc = d.n_cells;
    const size_t need = (kResidualScratch + 8) * sizeof(double);
    if (ctx->resid.bytes < need && ctx->resid.alloc(need)) return GELIOS_E_CUDA;
    double* cen0 = ctx->cen[0].as<double>();
    if (!ctx->cen_valid) {
        launch_centroid(d, d.X, d.Y, cen0, cen0 + nc, cen0 + 2 * nc, P.gamma, s, cen0 + 3 * nc, cen0 + 4 * nc);
        ctx->cen_valid = true;
        ctx->cen_rp_partial = false;
    }
    // the status word in scratch, so the context's own words stay untouched;
    // rows of cells the step does not update stay 0
    int* status = reinterpret_cast<int*>(ctx->resid.as<double>() + kResidualScratch);
    GELIOS_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), s));
    double* aux = ctx->aux.as<double>();
    GELIOS_CUDA_TRY(cudaMemsetAsync(aux, 0, 3 * nc * sizeof(double), s));
    StepBuffers b;
    for (int k = 0; k < 5; k++) {
        b.cur[k] = ctx->field(buf, k);
        b.nxt[k] = ctx->field(buf ^ 1, k);
    }
    b.cx = cen0;
    b.cy = cen0 + nc;
    b.status = status;
    launch_mk2_source(d, P, b, aux, s);
    GELIOS_CUDA_TRY(cudaGetLastError());
    GELIOS_CUDA_TRY(cudaMemcpyAsync(q1, aux, nc * sizeof(double), cudaMemcpyDeviceToHost, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(q2, aux + nc, nc * sizeof(double), cudaMemcpyDeviceToHost, s));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(q3, aux + 2 * nc, nc * sizeof(double), cudaMemcpyDeviceToHost, s));
    int st = 0;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    if (st) {
        set_error("gelios_mk2_source_terms: a source chain link the reference would follow is missing (status " +
                  std::to_string(st) + ")");
        return GELIOS_E_STATE;
    }
    return GELIOS_OK;
}

extern "C" int gelios_run_to_residual(gelios_ctx* ctx, int form, double tol, int64_t max_steps, int32_t check_every,
                                      int64_t* steps_done, double* residual_per_time, double* dt) {
    if (!ctx || check_every <= 0 || (check_every & 1) || max_steps < 0) return GELIOS_E_ARG;
    int64_t done = 0;
    double rpt = 0.0, last_dt = 0.0;
    while (done < max_steps) {
        const int n = static_cast<int>(std::min<int64_t>(check_every, max_steps - done) & ~1);
        if (n <= 0) break;
        gelios_status st{};
        int rc = gelios_step(ctx, form, n, &st);
        if (rc) return rc;
        done += n;
        double r = 0.0;
        rc = gelios_residual(ctx, st.result_buf, &r);
        if (rc) return rc;
        last_dt = st.dt;
        rpt = last_dt > 0.0 ? r / last_dt : 0.0;
        if (rpt <= tol) break;
    }
    if (steps_done) *steps_done = done;
    if (residual_per_time) *residual_per_time = rpt;
    if (dt) *dt = last_dt;
    return GELIOS_OK;
}

extern "C" int gelios_io_rows(int form) {
    return 5 + (form == GELIOS_FORM_5_KOMPONENT ? 16 : form == GELIOS_FORM_MHD_PUI ? 8 : 0);
}

extern "C" int gelios_run_streamed(gelios_ctx* ctx, int form, int nsteps, const double* const* host_in,
                                   double* const* host_out) {
    if (!ctx || nsteps < 0 || (nsteps > 0 && (!host_in || !host_out))) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    for (int k = 0; k < nsteps; k++)
        if (!host_in[k] || !host_out[k]) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t nc = ctx->d.n_cells;
    const int extra = gelios_io_rows(form) - 5;
    const size_t bytes = static_cast<size_t>(gelios_io_rows(form)) * nc * sizeof(double);
    if (!ctx->io_h2d) {
        GELIOS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->io_h2d, cudaStreamNonBlocking));
        GELIOS_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->io_d2h, cudaStreamNonBlocking));
        for (int j = 0; j < 2; j++)
            for (cudaEvent_t* e : {&ctx->ev_in_ready[j], &ctx->ev_in_free[j], &ctx->ev_out_ready[j], &ctx->ev_out_free[j]})
                GELIOS_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    for (int j = 0; j < 2; j++) {
        if (ctx->io_in[j].bytes != bytes && ctx->io_in[j].alloc(bytes)) return GELIOS_E_CUDA;
        if (ctx->io_out[j].bytes != bytes && ctx->io_out[j].alloc(bytes)) return GELIOS_E_CUDA;
    }
    cudaStream_t s = ctx->stream;
    // staging buffers are free at the start: the previous call ended with a synchronisation
    int64_t launches = 0;
    for (int k = 0; k < nsteps; k++) {
        const int j = k & 1;
        double* in = ctx->io_in[j].as<double>();
        double* out = ctx->io_out[j].as<double>();
        // input of call k: host -> staging (after call k-2 has read this staging buffer)
        if (k >= 2) GELIOS_CUDA_TRY(cudaStreamWaitEvent(ctx->io_h2d, ctx->ev_in_free[j], 0));
        GELIOS_CUDA_TRY(cudaMemcpyAsync(in, host_in[k], bytes, cudaMemcpyHostToDevice, ctx->io_h2d));
        GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_in_ready[j], ctx->io_h2d));
        // staging -> par[0] on the step's stream, then the step
        GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_in_ready[j], 0));
        GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->state[0].p, in, 5 * nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (extra)
            GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->hstate[0].p, in + 5 * nc, extra * nc * sizeof(double),
                                            cudaMemcpyDeviceToDevice, s));
        GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_in_free[j], s));
        const int rc = gelios_step(ctx, form, 1, nullptr);
        if (rc) {
            // no copy may touch the caller's blocks after we return
            cudaStreamSynchronize(ctx->io_h2d);
            cudaStreamSynchronize(ctx->io_d2h);
            cudaStreamSynchronize(s);
            return rc;
        }
        launches += ctx->launches;
        // par[1] -> staging (after call k-2's result has left it) -> host
        if (k >= 2) GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, ctx->ev_out_free[j], 0));
        GELIOS_CUDA_TRY(cudaMemcpyAsync(out, ctx->state[1].p, 5 * nc * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (extra)
            GELIOS_CUDA_TRY(cudaMemcpyAsync(out + 5 * nc, ctx->hstate[1].p, extra * nc * sizeof(double),
                                            cudaMemcpyDeviceToDevice, s));
        GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_out_ready[j], s));
        GELIOS_CUDA_TRY(cudaStreamWaitEvent(ctx->io_d2h, ctx->ev_out_ready[j], 0));
        GELIOS_CUDA_TRY(cudaMemcpyAsync(host_out[k], out, bytes, cudaMemcpyDeviceToHost, ctx->io_d2h));
        GELIOS_CUDA_TRY(cudaEventRecord(ctx->ev_out_free[j], ctx->io_d2h));
    }
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->io_d2h));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    ctx->launches = launches;
    return GELIOS_OK;
}

extern "C" int gelios_variant_count(int form) {
    return form == GELIOS_FORM_MHD_PUI ? kMhdFaceVariants : form == GELIOS_FORM_MK2 ? kMk2Variants : 1;
}

extern "C" int gelios_set_pipelined(gelios_ctx* ctx, int on) {
    if (!ctx) return GELIOS_E_ARG;
    ctx->pipelined = on != 0;
    return GELIOS_OK;
}

extern "C" int gelios_set_variant(gelios_ctx* ctx, int form, int32_t variant) {
    if (!ctx || variant < 0 || variant >= gelios_variant_count(form)) return GELIOS_E_ARG;
    if (form == GELIOS_FORM_MHD_PUI) {
        ctx->mhd_face_variant = variant;
        ctx->drop_graphs();  // the captured steps hold the old launch shape
    } else if (form == GELIOS_FORM_MK2) {
        ctx->mk2_variant = variant;
        ctx->drop_graphs();
    }
    return GELIOS_OK;
}

extern "C" int gelios_get_variant(gelios_ctx* ctx, int form, int32_t* variant) {
    if (!ctx || !variant) return GELIOS_E_ARG;
    *variant = form == GELIOS_FORM_MHD_PUI ? ctx->mhd_face_variant : form == GELIOS_FORM_MK2 ? ctx->mk2_variant : 0;
    return GELIOS_OK;
}

extern "C" int gelios_autotune(gelios_ctx* ctx, int form, int reps, int32_t* variant, double* ms) {
    if (!ctx || reps < 1) return GELIOS_E_ARG;
    const bool mhd = form == GELIOS_FORM_MHD_PUI;
    if (!mhd && form != GELIOS_FORM_MK2) {
        if (variant) *variant = 0;
        if (ms) *ms = 0.0;
        return GELIOS_OK;
    }
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    const DevMesh& d = ctx->d;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    if (mhd) {
        const size_t fb = static_cast<size_t>(kMhdFluxRows) * d.n_slots * sizeof(double);
        if (ctx->flux_mhd.bytes != fb) {
            ctx->drop_graphs();
            if (ctx->flux_mhd.alloc(fb)) return GELIOS_E_CUDA;
        }
    }
    // the words a step starts from (dt0, empty accumulator); reset again below
    struct Words {
        double T[2];
        unsigned long long acc;
        unsigned long long counters[2];
        int status;
        int pad[5];
    } w{};
    w.T[0] = w.T[1] = ctx->prm.dt0;
    w.acc = 0x7ff0000000000000ULL;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->words.p, &w, sizeof(w), cudaMemcpyHostToDevice, s));
    const size_t nc = d.n_cells;
    double* cen0 = ctx->cen[0].as<double>();
    if (!ctx->cen_valid || ctx->cen_rp_partial) {
        launch_centroid(d, d.X, d.Y, cen0, cen0 + nc, cen0 + 2 * nc, ctx->prm.gamma, s, cen0 + 3 * nc, cen0 + 4 * nc);
        ctx->cen_valid = true;
        ctx->cen_rp_partial = false;
    }
    StepBuffers b;
    for (int k = 0; k < 5; k++) {
        b.cur[k] = ctx->field(0, k);
        b.nxt[k] = ctx->field(1, k);
    }
    b.cx = cen0;
    b.cy = cen0 + nc;
    b.rp = cen0 + 2 * nc;
    b.vs = cen0 + 3 * nc;
    b.vol = cen0 + 4 * nc;
    b.dt_cur = ctx->T();
    b.dt_next = ctx->T() + 1;
    b.dt_acc = ctx->acc();
    b.counters = ctx->counters();
    b.status = ctx->status();
    cudaEvent_t e0, e1;
    GELIOS_CUDA_TRY(cudaEventCreate(&e0));
    GELIOS_CUDA_TRY(cudaEventCreate(&e1));
    int best = 0;
    double best_ms = 0.0;
    // the moving-grid update writes a next state and a next geometry cache:
    // give it scratch (the second cache buffer is free between calls)
    DBuf scratch;
    if (!mhd) {
        if (scratch.alloc(5 * nc * sizeof(double))) return GELIOS_E_CUDA;
        double* cen1 = ctx->cen[1].as<double>();
        for (int k = 0; k < 5; k++) b.nxt[k] = scratch.as<double>() + k * nc;
        b.cx_next = cen1;
        b.cy_next = cen1 + nc;
        b.rp_next = cen1 + 2 * nc;
        b.vs_next = cen1 + 3 * nc;
        b.vol_next = cen1 + 4 * nc;
    }
    // the dominant kernel of the form (only scratch and the dt / status
    // words, reset below, are written)
    auto faces = [&](int v) {
        if (mhd) {
            launch_mhd_faces(d, ctx->prm, ctx->mprm, b, ctx->hstate[0].as<double>(), ctx->flux_mhd.as<double>(), s,
                             v);
        } else {
            launch_mk2_cells(d, ctx->prm, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), s, v, 1);
            launch_mk2_cells(d, ctx->prm, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), s, v, 3);
            launch_mk2_cells(d, ctx->prm, b, ctx->tiles, ctx->flux.as<double>(), ctx->aux.as<double>(), s, v, 2);
        }
    };
    // mean ms of `reps` launches of fn(v) after one untimed launch
    auto time_ms = [&](auto fn, int v, double& out) -> cudaError_t {
        fn(v);
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; r++) fn(v);
        cudaEventRecord(e1, s);
        cudaError_t err = cudaEventSynchronize(e1);
        float t = 0.f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
        out = static_cast<double>(t) / reps;
        return err;
    };
    const int nv = mhd ? kMhdFaceVariants : kMk2TunedVariants;
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < nv && err == cudaSuccess; i++) {
        const int v = mhd ? i : kMk2Tuned[i];
        double m = 0.0;
        err = time_ms(faces, v, m);
        if (i == 0 || m < best_ms) {
            best = v;
            best_ms = m;
        }
    }
    if (err != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        set_error(std::string("gelios_autotune: ") + cudaGetErrorString(err));
        return GELIOS_E_CUDA;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GELIOS_CUDA_TRY(cudaMemcpyAsync(ctx->words.p, &w, sizeof(w), cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    int& current = mhd ? ctx->mhd_face_variant : ctx->mk2_variant;
    if (best != current) {
        current = best;
        ctx->drop_graphs();
    }
    if (variant) *variant = best;
    if (ms) *ms = best_ms;
    return GELIOS_OK;
}

// ---------------------------------------------------------------- batched instances
struct gelios_batch {
    int device = 0;
    std::vector<gelios_ctx*> ctxs;
    DBuf inst, surf, rails, units, cells, points;
    BatchTables tab;
    std::vector<BatchInstance> host_inst;  // one descriptor per instance, rebuilt per call
    BatchInstance* pinned = nullptr;       // staging of the descriptors' upload (pinned: the copy is asynchronous)
    cudaEvent_t ev = nullptr, ev_table = nullptr;
    bool table_pending = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graphs_off = false;
    // 0: one launch per phase, a captured graph per step; k > 0: all steps
    // of a call in one cooperative launch of k blocks per SM
    int schedule = 0;
    ~gelios_batch() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        if (ev) cudaEventDestroy(ev);
        if (ev_table) cudaEventDestroy(ev_table);
        if (pinned) cudaFreeHost(pinned);
    }
};

extern "C" int gelios_batch_create(gelios_batch** out, gelios_ctx* const* ctxs, int n) {
    if (!out || !ctxs || n < 1) return GELIOS_E_ARG;
    *out = nullptr;
    auto B = std::make_unique<gelios_batch>();
    B->device = ctxs[0] ? ctxs[0]->device : 0;
    std::vector<int2> surf, rails, units, cells, points;
    for (int i = 0; i < n; i++) {
        gelios_ctx* c = ctxs[i];
        if (!c || !c->have_mesh) {
            set_error("gelios_batch_create: a context without topology");
            return GELIOS_E_STATE;
        }
        if (c->device != B->device || c->prm.precision != ctxs[0]->prm.precision) {
            set_error("gelios_batch_create: contexts on different devices or with different flux precisions");
            return GELIOS_E_ARG;
        }
        const DevMesh& d = c->d;
        if (d.n_rail_a + d.n_rail_b + d.n_rail_c + d.n_rail_d == 0 || d.n_lc == 0) {
            set_error("gelios_batch_create: the moving-grid step needs rails and tracked lines");
            return GELIOS_E_MESH;
        }
        if (c->src_fixed.bytes != 3 * static_cast<size_t>(d.n_cells) * sizeof(double)) {
            set_error("gelios_batch_create: a context without gelios_upload_sources");
            return GELIOS_E_STATE;
        }
        GELIOS_CUDA_TRY(cudaSetDevice(c->device));
        const size_t fb = static_cast<size_t>(kMhdFluxRows) * d.n_slots * sizeof(double);
        if (c->flux_mhd.bytes != fb) {
            c->drop_graphs();
            if (c->flux_mhd.alloc(fb)) return GELIOS_E_CUDA;
        }
        const int nt = d.n_lc + d.n_li + d.n_lo;
        for (int j = 0; j < nt; j += 2) surf.push_back(make_int2(i, j));
        const int nr = d.n_rail_a + d.n_rail_b + d.n_rail_c + d.n_rail_d;
        for (int q = 0; q < nr; q++) rails.push_back(make_int2(i, q));
        for (int u = 0; u < d.n_units; u += 128) units.push_back(make_int2(i, u));
        for (int k = 0; k < d.n_cells; k += 128) cells.push_back(make_int2(i, k));
        for (int k = 0; k < d.n_points; k += 256) points.push_back(make_int2(i, k));
        B->ctxs.push_back(c);
    }
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    cudaStream_t s = ctxs[0]->stream;
    int rc = 0;
    rc |= upload(B->surf, surf.data(), surf.size(), s);
    rc |= upload(B->rails, rails.data(), rails.size(), s);
    rc |= upload(B->units, units.data(), units.size(), s);
    rc |= upload(B->cells, cells.data(), cells.size(), s);
    rc |= upload(B->points, points.data(), points.size(), s);
    if (B->inst.alloc(static_cast<size_t>(n) * sizeof(BatchInstance))) rc |= 1;
    if (rc) return GELIOS_E_CUDA;
    GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&B->ev, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaEventCreateWithFlags(&B->ev_table, cudaEventDisableTiming));
    GELIOS_CUDA_TRY(cudaMallocHost(&B->pinned, static_cast<size_t>(n) * sizeof(BatchInstance)));
    BatchTables& t = B->tab;
    t.surf = B->surf.as<int2>();
    t.rails = B->rails.as<int2>();
    t.units = B->units.as<int2>();
    t.cells = B->cells.as<int2>();
    t.points = B->points.as<int2>();
    t.n_surf = static_cast<int>(surf.size());
    t.n_rails = static_cast<int>(rails.size());
    t.n_units = static_cast<int>(units.size());
    t.n_cells = static_cast<int>(cells.size());
    t.n_points = static_cast<int>(points.size());
    t.fp32 = ctxs[0]->prm.precision == GELIOS_PREC_FP32_FLUX;
    B->host_inst.resize(static_cast<size_t>(n));
    *out = B.release();
    return GELIOS_OK;
}

extern "C" void gelios_batch_destroy(gelios_batch* batch) {
    if (!batch) return;
    cudaSetDevice(batch->device);
    if (!batch->ctxs.empty()) cudaStreamSynchronize(batch->ctxs[0]->stream);
    delete batch;
}

extern "C" int gelios_batch_step(gelios_batch* B, int form, int nsteps, gelios_status* statuses) {
    if (!B || nsteps < 0) return GELIOS_E_ARG;
    if (form != GELIOS_FORM_MHD_PUI) {
        set_error("gelios_batch_step: only the MHD form is batched");
        return GELIOS_E_ARG;
    }
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    const int n = static_cast<int>(B->ctxs.size());
    cudaStream_t s = B->ctxs[0]->stream;
    // order after each context's own pending work
    for (int i = 1; i < n; i++) {
        GELIOS_CUDA_TRY(cudaEventRecord(B->ev, B->ctxs[i]->stream));
        GELIOS_CUDA_TRY(cudaStreamWaitEvent(s, B->ev, 0));
    }
    struct Words {
        double T[2];
        unsigned long long acc;
        unsigned long long counters[2];
        int status;
        int pad[5];
    };
    static_assert(sizeof(Words) == 64, "device word layout");
    for (int i = 0; i < n; i++) {
        gelios_ctx* c = B->ctxs[i];
        const DevMesh& d = c->d;
        const size_t nc = d.n_cells;
        double* cen0 = c->cen[0].as<double>();
        double* cen1 = c->cen[1].as<double>();
        if (!c->cen_valid) {
            launch_centroid(d, d.X, d.Y, cen0, cen0 + nc, cen0 + 2 * nc, c->prm.gamma, s, cen0 + 3 * nc, cen0 + 4 * nc);
            c->cen_rp_partial = false;
        }
        {
            BatchInstance& I = B->host_inst[i];
            I.d = d;
            I.P = c->prm;
            I.M = c->mprm;
            for (int q = 0; q < 2; q++) {  // b[q]: the buffers of a step with parity q
                StepBuffers& b = I.b[q];
                b = StepBuffers();
                for (int k = 0; k < 5; k++) {
                    b.cur[k] = c->field(q, k);
                    b.nxt[k] = c->field(q ^ 1, k);
                }
                double* cc = q ? cen1 : cen0;
                double* cn = q ? cen0 : cen1;
                b.cx = cc;
                b.cy = cc + nc;
                b.rp = cc + 2 * nc;
                b.vs = cc + 3 * nc;
                b.vol = cc + 4 * nc;
                b.cx_next = cn;
                b.cy_next = cn + nc;
                b.rp_next = cn + 2 * nc;
                b.vs_next = cn + 3 * nc;
                b.vol_next = cn + 4 * nc;
                b.dt_cur = c->T() + q;
                b.dt_next = c->T() + (q ^ 1);
                b.dt_acc = c->acc();
                b.counters = c->counters();
                b.status = c->status();
                I.hs[q] = c->hstate[q].as<double>();
                I.hn[q] = c->hstate[q ^ 1].as<double>();
            }
            I.fl = c->flux_mhd.as<double>();
            I.src = c->src_fixed.as<double>();
            I.surface = c->surface.as<double>();
        }
    }
    // the kernels index b[parity], hs[parity], hn[parity]; the staging is
    // reused once the previous call's upload has been read
    if (B->table_pending) GELIOS_CUDA_TRY(cudaEventSynchronize(B->ev_table));
    std::memcpy(B->pinned, B->host_inst.data(), static_cast<size_t>(n) * sizeof(BatchInstance));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(B->inst.p, B->pinned, static_cast<size_t>(n) * sizeof(BatchInstance),
                                    cudaMemcpyHostToDevice, s));
    GELIOS_CUDA_TRY(cudaEventRecord(B->ev_table, s));
    B->table_pending = true;
    B->tab.inst = B->inst.as<BatchInstance>();
    launch_batch_words_init(B->tab, n, s);  // dt0, empty accumulators: every instance starts a call
    int64_t launches = 1;
    const int per_step = (B->tab.n_surf > 0) + (B->tab.n_rails > 0) + (B->tab.n_units > 0) + (B->tab.n_cells > 0) +
                         (B->tab.n_points > 0);
    if (B->schedule > 0 && nsteps > 0) {
        GELIOS_CUDA_TRY(launch_batch_mhd_persistent(B->tab, nsteps, B->schedule, s));
        launches += 1;
    }
    for (int st = 0; st < (B->schedule > 0 ? 0 : nsteps); st++) {
        const int par = st & 1;
        if (!B->graphs_off && !B->graph[par]) {
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                launch_batch_mhd_step(B->tab, par, s);
                if (cudaStreamEndCapture(s, &g) != cudaSuccess || !g ||
                    cudaGraphInstantiate(&B->graph[par], g, 0) != cudaSuccess) {
                    B->graph[par] = nullptr;
                    B->graphs_off = true;
                }
                if (g) cudaGraphDestroy(g);
            } else {
                B->graphs_off = true;
            }
            cudaGetLastError();
        }
        if (B->graph[par]) {
            GELIOS_CUDA_TRY(cudaGraphLaunch(B->graph[par], s));
        } else {
            launch_batch_mhd_step(B->tab, par, s);
        }
        launches += per_step;
    }
    GELIOS_CUDA_TRY(cudaGetLastError());
    // the contexts' own streams follow the batch
    GELIOS_CUDA_TRY(cudaEventRecord(B->ev, s));
    for (int i = 1; i < n; i++) GELIOS_CUDA_TRY(cudaStreamWaitEvent(B->ctxs[i]->stream, B->ev, 0));
    for (int i = 0; i < n; i++) {
        gelios_ctx* c = B->ctxs[i];
        if (nsteps & 1) std::swap(c->cen[0].p, c->cen[1].p);
        c->cen_valid = true;
        if (nsteps > 0) {
            c->cen_rp_partial = true;
            c->upf_valid = false;
        }
        c->launches = launches;
    }
    if (statuses) {
        std::vector<Words> r(n);
        for (int i = 0; i < n; i++)
            GELIOS_CUDA_TRY(cudaMemcpyAsync(&r[i], B->ctxs[i]->words.p, sizeof(Words), cudaMemcpyDeviceToHost, s));
        GELIOS_CUDA_TRY(cudaStreamSynchronize(s));
        for (int i = 0; i < n; i++) {
            gelios_status& o = statuses[i];
            std::memset(&o, 0, sizeof(o));
            o.flags = r[i].status;
            o.steps_done = nsteps;
            o.n_ro_clamp = static_cast<int64_t>(r[i].counters[0]);
            o.n_p_clamp = static_cast<int64_t>(r[i].counters[1]);
            o.result_buf = nsteps & 1;
            o.dt = r[i].T[nsteps & 1];
            if (!(o.dt == o.dt)) o.flags |= ST_DT_BAD;
        }
    }
    return GELIOS_OK;
}

extern "C" int gelios_batch_set_schedule(gelios_batch* B, int32_t schedule) {
    if (!B || schedule < 0) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    if (schedule > 0) {
        int max_per_sm = 0;
        const cudaError_t e = launch_batch_mhd_persistent(B->tab, 0, schedule, B->ctxs[0]->stream, &max_per_sm);
        if (e == cudaErrorCooperativeLaunchTooLarge) {
            set_error("gelios_batch_set_schedule: " + std::to_string(schedule) + " blocks per SM do not fit (at most " +
                      std::to_string(max_per_sm) + ")");
            return GELIOS_E_ARG;
        }
        GELIOS_CUDA_TRY(e);
    }
    B->schedule = schedule;
    return GELIOS_OK;
}

extern "C" int gelios_batch_get_schedule(gelios_batch* B, int32_t* schedule) {
    if (!B || !schedule) return GELIOS_E_ARG;
    *schedule = B->schedule;
    return GELIOS_OK;
}

extern "C" int gelios_batch_autotune(gelios_batch* B, int steps, int32_t* schedule, double* ms, double* each_ms,
                                     int n_each) {
    if (!B || steps < 1 || n_each < 0 || (n_each > 0 && !each_ms)) return GELIOS_E_ARG;
    for (int k = 0; k < n_each; k++) each_ms[k] = -1.0;
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    cudaStream_t s = B->ctxs[0]->stream;
    int max_per_sm = 0;
    GELIOS_CUDA_TRY(launch_batch_mhd_persistent(B->tab, 0, 0, s, &max_per_sm));
    cudaEvent_t e0, e1;
    GELIOS_CUDA_TRY(cudaEventCreate(&e0));
    GELIOS_CUDA_TRY(cudaEventCreate(&e1));
    int best = 0;
    double best_ms = -1.0;
    int rc = GELIOS_OK;
    // every candidate once untimed (graph capture, first touch), then timed
    for (int cand = 0; cand <= max_per_sm && rc == GELIOS_OK; cand++) {
        B->schedule = cand;
        for (int rep = 0; rep < 2 && rc == GELIOS_OK; rep++) {
            if (rep == 1 && cudaEventRecord(e0, s) != cudaSuccess) rc = GELIOS_E_CUDA;
            if (rc == GELIOS_OK) rc = gelios_batch_step(B, GELIOS_FORM_MHD_PUI, steps, nullptr);
            if (rc == GELIOS_OK && rep == 1) {
                float t = 0.f;
                if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                    cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) {
                    rc = GELIOS_E_CUDA;
                } else {
                    if (cand < n_each) each_ms[cand] = t / steps;
                    if (best_ms < 0.0 || t < best_ms) {
                        best_ms = t;
                        best = cand;
                    }
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B->schedule = best;
    if (rc != GELIOS_OK) return rc;
    if (schedule) *schedule = best;
    if (ms) *ms = best_ms / steps;
    return GELIOS_OK;
}

extern "C" int gelios_download_points(gelios_ctx* ctx, double* x, double* y) {
    if (!ctx || !x || !y) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t n = sizeof(double) * ctx->d.n_points;
    GELIOS_CUDA_TRY(cudaMemcpyAsync(x, ctx->X.p, n, cudaMemcpyDeviceToHost, ctx->stream));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(y, ctx->Y.p, n, cudaMemcpyDeviceToHost, ctx->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_synchronize(gelios_ctx* ctx) {
    if (!ctx) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GELIOS_OK;
}

extern "C" int gelios_state_device_ptr(gelios_ctx* ctx, int buf, double** dptr) {
    if (!ctx || buf < 0 || buf > 1 || !dptr) return GELIOS_E_ARG;
    if (!ctx->have_mesh) return GELIOS_E_STATE;
    *dptr = ctx->state[buf].as<double>();
    return GELIOS_OK;
}

extern "C" void* gelios_stream(gelios_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

extern "C" int64_t gelios_last_launch_count(gelios_ctx* ctx) { return ctx ? ctx->launches : 0; }

extern "C" int gelios_set_phase_timing(gelios_ctx* ctx, int enabled) {
    if (!ctx) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->collect();
    ctx->timing = enabled != 0;
    return GELIOS_OK;
}

extern "C" int gelios_phase_times(gelios_ctx* ctx, double* ms, int64_t* launches, int reset) {
    if (!ctx) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(ctx->device));
    ctx->collect();
    for (int k = 0; k < 5; k++) {
        if (ms) ms[k] = ctx->phase_ms[k];
        if (launches) launches[k] = ctx->phase_launch[k];
        if (reset) {
            ctx->phase_ms[k] = 0.0;
            ctx->phase_launch[k] = 0;
        }
    }
    return GELIOS_OK;
}

namespace {
enum BatchKind { B_HLLC, B_GODUNOV, B_HLLDQ, B_HLLD };
int run_batch(const gelios_params* prm, int n, const double* in, int in_w, double* out, int out_w, BatchKind kind) {
    if (!prm || n < 0 || (n > 0 && (!in || !out))) return GELIOS_E_ARG;
    if (n == 0) return GELIOS_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device");
        return GELIOS_E_NODEVICE;
    }
    DBuf din, dout;
    if (din.alloc(sizeof(double) * in_w * n) || dout.alloc(sizeof(double) * out_w * n)) return GELIOS_E_CUDA;
    GELIOS_CUDA_TRY(cudaMemcpy(din.p, in, sizeof(double) * in_w * n, cudaMemcpyHostToDevice));
    switch (kind) {
        case B_HLLC: launch_hllc_batch(*prm, n, din.as<double>(), dout.as<double>(), 0); break;
        case B_GODUNOV: launch_godunov_batch(*prm, n, din.as<double>(), dout.as<double>(), 0); break;
        case B_HLLDQ: launch_hlldq_batch(*prm, n, din.as<double>(), dout.as<double>(), 0); break;
        case B_HLLD: launch_hlld_batch(*prm, n, din.as<double>(), dout.as<double>(), 0); break;
    }
    GELIOS_CUDA_TRY(cudaGetLastError());
    GELIOS_CUDA_TRY(cudaMemcpy(out, dout.p, sizeof(double) * out_w * n, cudaMemcpyDeviceToHost));
    return GELIOS_OK;
}
}  // namespace

extern "C" int gelios_hllc_batch(const gelios_params* prm, int n, const double* in, double* out) {
    return run_batch(prm, n, in, 16, out, 9, B_HLLC);
}

extern "C" int gelios_godunov_batch(const gelios_params* prm, int n, const double* in, double* out) {
    return run_batch(prm, n, in, 15, out, 10, B_GODUNOV);
}

extern "C" int gelios_hlldq_batch(const gelios_params* prm, int n, const double* in, double* out) {
    return run_batch(prm, n, in, 23, out, 10, B_HLLDQ);
}

extern "C" int gelios_hlld_batch(const gelios_params* prm, int n, const double* in, double* out) {
    return run_batch(prm, n, in, 21, out, 13, B_HLLD);
}

// ------------------------------------------------------------------ plain-form batch
// Instances of the Go_stationary form that share one mesh, advanced together
// by one cooperative launch per chunk of steps (the converged states of an
// inflow-parameter sweep).  Each instance keeps its own context: state,
// parameters, flux slots and dt words.
struct gelios_plain_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<gelios_ctx*> ctxs;
    DBuf inst, active, resid;
    int prec = GELIOS_PREC_FP64;  // flux precision of every instance
    ~gelios_plain_batch() {
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" int gelios_plain_batch_create(gelios_plain_batch** out, gelios_ctx* const* ctxs, int n) {
    if (!out || !ctxs || n < 1) return GELIOS_E_ARG;
    *out = nullptr;
    auto B = std::make_unique<gelios_plain_batch>();
    const gelios_ctx* c0 = ctxs[0];
    if (!c0 || !c0->have_mesh) {
        set_error("gelios_plain_batch_create: a context without topology");
        return GELIOS_E_STATE;
    }
    B->device = c0->device;
    B->prec = c0->prm.precision;
    for (int i = 0; i < n; i++) {
        gelios_ctx* c = ctxs[i];
        if (!c || !c->have_mesh) {
            set_error("gelios_plain_batch_create: a context without topology");
            return GELIOS_E_STATE;
        }
        if (c->device != B->device || c->prm.precision != B->prec) {
            set_error("gelios_plain_batch_create: contexts on different devices or with different flux precisions");
            return GELIOS_E_ARG;
        }
        if (c->d.n_cells != c0->d.n_cells || c->d.n_units != c0->d.n_units || c->d.n_slots != c0->d.n_slots ||
            c->d.n_points != c0->d.n_points) {
            set_error("gelios_plain_batch_create: the instances must share one mesh");
            return GELIOS_E_MESH;
        }
        for (int j = 0; j < i; j++)
            if (ctxs[j] == c) {
                set_error("gelios_plain_batch_create: a context listed twice");
                return GELIOS_E_ARG;
            }
        B->ctxs.push_back(c);
    }
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    GELIOS_CUDA_TRY(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    if (B->inst.alloc(sizeof(PlainInstance) * n) || B->active.alloc(sizeof(int) * n) ||
        B->resid.alloc(sizeof(double) * kResidualScratch * n))
        return GELIOS_E_CUDA;
    *out = B.release();
    return GELIOS_OK;
}

extern "C" void gelios_plain_batch_destroy(gelios_plain_batch* B) {
    if (!B) return;
    cudaSetDevice(B->device);
    cudaStreamSynchronize(B->stream);
    delete B;
}

namespace {
// Centroid caches of every instance (the plain form reads cx, cy and
// |c|^(2 gamma) of all cells), the instance descriptors (rebuilt per call:
// parameters and buffers may have changed), then the dt words of the listed
// instances; the contexts' streams are drained first so their earlier work
// is ordered before the batch's.
int plain_batch_prepare(gelios_plain_batch* B, const std::vector<int>& list) {
    std::vector<PlainInstance> host(B->ctxs.size());
    for (size_t i = 0; i < B->ctxs.size(); i++) {
        gelios_ctx* c = B->ctxs[i];
        if (c->prm.precision != B->prec) {
            set_error("gelios_plain_batch: the instances' flux precisions differ");
            return GELIOS_E_ARG;
        }
        GELIOS_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (!c->cen_valid || c->cen_rp_partial) {
            const size_t ncz = c->d.n_cells;
            double* cen0 = c->cen[0].as<double>();
            launch_centroid(c->d, c->d.X, c->d.Y, cen0, cen0 + ncz, cen0 + 2 * ncz, c->prm.gamma, B->stream,
                            cen0 + 3 * ncz, cen0 + 4 * ncz);
            c->cen_valid = true;
            c->cen_rp_partial = false;
        }
        if (!c->upf_valid) {
            const double* cen = c->cen[0].as<double>();
            launch_unit_geometry(c->d, c->prm.gamma, cen, cen + c->d.n_cells, c->upf.as<double>(), B->stream);
            c->upf_valid = true;
        }
        PlainInstance& I = host[i];
        I.P = c->prm;
        const size_t ncz = c->d.n_cells;
        const double* cen0 = c->cen[0].as<double>();
        for (int par = 0; par < 2; par++) {
            StepBuffers& b = I.b[par];
            for (int k = 0; k < 5; k++) {
                b.cur[k] = c->field(par, k);
                b.nxt[k] = c->field(par ^ 1, k);
            }
            b.dt_cur = c->T() + par;
            b.dt_next = c->T() + (par ^ 1);
            b.dt_acc = c->acc();
            b.counters = c->counters();
            b.status = c->status();
            b.cx = cen0;
            b.cy = cen0 + ncz;
            b.rp = cen0 + 2 * ncz;
            b.vs = cen0 + 3 * ncz;
            b.upf = c->upf.as<double>();
            b.ugeo = b.upf + c->d.n_units;
        }
        I.fl = c->flux.as<double>();
    }
    GELIOS_CUDA_TRY(cudaMemcpyAsync(B->inst.p, host.data(), sizeof(PlainInstance) * host.size(), cudaMemcpyHostToDevice,
                                    B->stream));
    GELIOS_CUDA_TRY(cudaMemcpyAsync(B->active.p, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice,
                                    B->stream));
    launch_plain_batch_words_init(B->inst.as<PlainInstance>(), B->active.as<int>(), static_cast<int>(list.size()),
                                  B->stream);
    GELIOS_CUDA_TRY(cudaGetLastError());
    return GELIOS_OK;
}
}  // namespace

extern "C" int gelios_plain_batch_step(gelios_plain_batch* B, int nsteps, gelios_status* statuses) {
    if (!B || nsteps < 0) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    const int n = static_cast<int>(B->ctxs.size());
    std::vector<int> list(n);
    for (int i = 0; i < n; i++) list[i] = i;
    int rc = plain_batch_prepare(B, list);
    if (rc) return rc;
    GELIOS_CUDA_TRY(launch_stationary_batch(B->ctxs[0]->d, B->inst.as<PlainInstance>(), B->active.as<int>(), n, nsteps,
                                            B->prec, B->stream));
    GELIOS_CUDA_TRY(cudaStreamSynchronize(B->stream));
    for (int i = 0; i < n; i++) {
        gelios_ctx* c = B->ctxs[i];
        c->launches = 1;
        if (!statuses) continue;
        double T[2];
        unsigned long long cnt[2];
        int flags = 0;
        GELIOS_CUDA_TRY(cudaMemcpy(T, c->T(), sizeof(T), cudaMemcpyDeviceToHost));
        GELIOS_CUDA_TRY(cudaMemcpy(cnt, c->counters(), sizeof(cnt), cudaMemcpyDeviceToHost));
        GELIOS_CUDA_TRY(cudaMemcpy(&flags, c->status(), sizeof(int), cudaMemcpyDeviceToHost));
        gelios_status& o = statuses[i];
        std::memset(&o, 0, sizeof(o));
        o.flags = flags;
        o.steps_done = nsteps;
        o.n_ro_clamp = static_cast<int64_t>(cnt[0]);
        o.n_p_clamp = static_cast<int64_t>(cnt[1]);
        o.result_buf = nsteps & 1;
        o.dt = T[nsteps & 1];
        if (!(o.dt == o.dt)) o.flags |= ST_DT_BAD;
    }
    return GELIOS_OK;
}

extern "C" int gelios_plain_batch_run_to_residual(gelios_plain_batch* B, double tol, int64_t max_steps,
                                                  int32_t check_every, int64_t* steps_done,
                                                  double* residual_per_time, double* dt) {
    if (!B || check_every <= 0 || (check_every & 1) || max_steps < 0) return GELIOS_E_ARG;
    GELIOS_CUDA_TRY(cudaSetDevice(B->device));
    const int n = static_cast<int>(B->ctxs.size());
    std::vector<int64_t> done(n, 0);
    std::vector<double> rpt(n, 0.0), last_dt(n, 0.0);
    std::vector<int> list(n);
    for (int i = 0; i < n; i++) list[i] = i;
    std::vector<double> scratch(static_cast<size_t>(kResidualScratch) * n);
    int64_t total = 0;
    while (!list.empty() && total < max_steps) {
        const int chunk = static_cast<int>(std::min<int64_t>(check_every, max_steps - total) & ~1);
        if (chunk <= 0) break;
        int rc = plain_batch_prepare(B, list);
        if (rc) return rc;
        GELIOS_CUDA_TRY(launch_stationary_batch(B->ctxs[0]->d, B->inst.as<PlainInstance>(), B->active.as<int>(),
                                                static_cast<int>(list.size()), chunk, B->prec, B->stream));
        for (int i : list) {
            gelios_ctx* c = B->ctxs[i];
            double* sc = B->resid.as<double>() + static_cast<size_t>(kResidualScratch) * i;
            launch_residual(c->field(0, 0), c->field(1, 0), c->d.n_cells, sc, B->stream);
        }
        GELIOS_CUDA_TRY(cudaGetLastError());
        GELIOS_CUDA_TRY(cudaMemcpyAsync(scratch.data(), B->resid.p, sizeof(double) * scratch.size(),
                                        cudaMemcpyDeviceToHost, B->stream));
        GELIOS_CUDA_TRY(cudaStreamSynchronize(B->stream));
        total += chunk;
        std::vector<int> keep;
        for (int i : list) {
            gelios_ctx* c = B->ctxs[i];
            double T0 = 0.0;
            int flags = 0;
            GELIOS_CUDA_TRY(cudaMemcpy(&T0, c->T(), sizeof(double), cudaMemcpyDeviceToHost));
            GELIOS_CUDA_TRY(cudaMemcpy(&flags, c->status(), sizeof(int), cudaMemcpyDeviceToHost));
            const double* sc = scratch.data() + static_cast<size_t>(kResidualScratch) * i;
            const double r = sc[1] > 0.0 ? sc[0] / sc[1] : 0.0;
            done[i] += chunk;
            last_dt[i] = T0;
            rpt[i] = T0 > 0.0 ? r / T0 : 0.0;
            // an instance whose step reported a failure stops (its residual is kept)
            if (!(rpt[i] <= tol) && flags == 0 && rpt[i] == rpt[i]) keep.push_back(i);
        }
        list.swap(keep);
    }
    for (gelios_ctx* c : B->ctxs) c->launches = 1;
    for (int i = 0; i < n; i++) {
        if (steps_done) steps_done[i] = done[i];
        if (residual_per_time) residual_per_time[i] = rpt[i];
        if (dt) dt[i] = last_dt[i];
    }
    return GELIOS_OK;
}
