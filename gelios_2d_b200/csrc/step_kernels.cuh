// Device-side views shared by the step kernels and the context (capi.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gelios_b200.h"

namespace gelios {

// Read-mostly topology + mutable point geometry, SoA, all device pointers.
//
// Per-cell face slots ("s*" arrays) are laid out in the reference's Grans
// order: slot g of cell c is gstart[c] + k for its k-th face.  A slot holds
// what the owner cell needs about the face without chasing the face table:
//   sA/sB   end points            snb   Sosed (neighbour cell)
//   ssd     Sosed_down of the face (TVD on the owner side)
//   ssd2    Sosed_down of its twin (TVD on the neighbour side)
//   sinfo   face type | SI_GOD | SI_NP
struct DevMesh {
    int n_points = 0, n_cells = 0, n_faces = 0, n_main = 0;
    // smallest a with sqrt(a) >= R11 (IEEE sqrt, host-computed): a cell takes
    // part in a moving-grid step iff !(x^2 + y^2 < r11_sq), the same cells as
    // !(sqrt(x^2 + y^2) < R11) without the square root
    double r11_sq = 0.0;
    int dims[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double *X = nullptr, *Y = nullptr, *X2 = nullptr, *Y2 = nullptr;
    const int32_t* ptype = nullptr;
    const int32_t *cstart = nullptr, *contour = nullptr, *gstart = nullptr;
    // contour of every quadrilateral cell as one int4 ({-1, -1, -1, -1} for
    // other cells); may be null (the contour arrays are read instead)
    const int4* qcorner = nullptr;
    const uint32_t* cflags = nullptr;
    const int32_t* ctype = nullptr;  // Cell_type of every cell
    const int32_t *sA = nullptr, *sB = nullptr, *snb = nullptr, *ssd = nullptr, *ssd2 = nullptr;
    const uint32_t* sinfo = nullptr;
    // face units (one flux evaluation each, see step_kernels.cu): owner slot,
    // owner cell, slot of the twin face in the neighbour (-1: one-sided)
    int n_slots = 0, n_units = 0;
    // units are grouped: plain interior [0, u_c1), interior with a C_1 side
    // [u_c1, u_tr0), tracked [u_tr0, u_tr1), one-sided [u_tr1, n_units)
    int u_c1 = 0, u_tr0 = 0, u_tr1 = 0;
    const int32_t *u_slot = nullptr, *u_cell = nullptr, *u_twin = nullptr;
    const int32_t *u_A = nullptr, *u_B = nullptr;  // end points of the unit's face
    // slot info of the unit's face | owner flags << UI_CF_OWN | neighbour flags << UI_CF_NB
    const uint32_t* u_info = nullptr;
    // neighbour cell (-1: one-sided unit), Sosed_down of the face and of its twin
    const int32_t *u_nb = nullptr, *u_sd = nullptr, *u_sd2 = nullptr;
    const int32_t *fA = nullptr, *fB = nullptr, *ftype = nullptr, *fmaster = nullptr, *fsosed = nullptr,
                  *fcopy = nullptr, *fsdown = nullptr;
    const int32_t *rtype = nullptr, *rM = nullptr, *rpstart = nullptr, *rpts = nullptr, *rkstart = nullptr,
                  *rkeys = nullptr;
    const double* rs = nullptr;
    int n_rail_a = 0, n_rail_b = 0, n_rail_c = 0, n_rail_d = 0;
    const int32_t *lc = nullptr, *li = nullptr, *lo = nullptr;
    int n_lc = 0, n_li = 0, n_lo = 0;
    // surface-tracking nodes (points of the three tracked lines): point id,
    // line (0 contact, 1 inner, 2 outer), up to 4 face incidences (j << 1 |
    // end, j in the concatenated line order, end 0 = A, 1 = B; -1 = none),
    // up to 4 contact faces whose A end it is (-1 = none); fix-up node ids
    // (a0, b0, a_last, b_last) per line
    int n_sp = 0;
    const int32_t *sp_point = nullptr, *sp_line = nullptr, *sp_inc = nullptr, *sp_ainc = nullptr,
                  *sp_fix = nullptr;
    const int32_t* sp_of_point = nullptr;  // tracked-surface node of each point, -1 if none
    const double *Hn = nullptr, *Hu = nullptr, *Hv = nullptr, *HT = nullptr, *ku = nullptr, *kv = nullptr,
                 *kT = nullptr, *r_istoch = nullptr;
    const int32_t *cback = nullptr, *cnext = nullptr;
    // bracket of the source interpolation found in the previous step (lower
    // cell, -1 = none); used when the chains are consistent (see source_mk1)
    // (lower cell, Next of it) of the previous step's bracket, {-1, -1} = none
    const int2* src_lo = nullptr;
    int2* src_lo_out = nullptr;
};

// Buffers of one time step (double buffering of the state like par[now1] ->
// par[now2]; centroids of the current/next point positions; dt words).
// Rows of the tracked units' reconstruction array of the moving-grid step
// (unit-major, n_tracked = u_tr1 - u_tr0 doubles per row), written before the
// grid moves (the other units reconstruct in registers after the motion):
//   0-4   owner side TVD state ro, p, u, v, Q
//   5-9   other side TVD state
//   10,11 face normal n1, n2 (pre-motion points)
//   12    S = |AB| * (yA + yB) / 2
//   13,14 face centre x2, y2 (pre-motion)
//   15    distance owner centroid - face centre, -1 if the owner is skipped
//   16    distance other centroid - face centre, -1 if skipped or no twin
// A unit with rows 15 and 16 both negative has no flux this step.
constexpr int kRecRows = 17;

struct StepBuffers {
    const double* cur[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double* nxt[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    const double* cx = nullptr;
    const double* cy = nullptr;
    const double* rp = nullptr;  // |centroid|^(2 gamma) per cell
    // moving-grid step: area (Get_Volume) and rotated volume of every cell
    // before the motion, cached from the previous step's update
    const double* vs = nullptr;
    const double* vol = nullptr;
    double* cx_next = nullptr;
    double* cy_next = nullptr;
    double* rp_next = nullptr;
    double* vs_next = nullptr;
    double* vol_next = nullptr;
    // plain form (fixed grid): |face centre|^(2 gamma) of every face unit and
    // the units' face geometry (kUnitGeoRows - 1 unit-major rows, see
    // FaceGeo in step_kernels.cu), or nullptr (then computed per unit)
    const double* upf = nullptr;
    const double* ugeo = nullptr;
    const double* dt_cur = nullptr;
    double* dt_next = nullptr;
    unsigned long long* dt_acc = nullptr;
    unsigned long long* counters = nullptr;  // [0] ro clamps, [1] p clamps
    int* status = nullptr;
};

// Centroids and |centroid|^(2 gamma) of every cell; with vs/vol also the
// area (Get_Volume) and the rotated volume (rows of the moving-grid cache).
void launch_centroid(const DevMesh& d, const double* X, const double* Y, double* cx, double* cy, double* rp,
                     double gamma, cudaStream_t s, double* vs = nullptr, double* vol = nullptr);
// Per face unit of the plain form (its grid does not move): row 0
// |face centre|^(2 gamma), rows 1-8 the face geometry as the owner sees it
// (centre x, y, normal, |centre|^2, length, owner and neighbour centroid
// distances); needs the centroids cx, cy.
constexpr int kUnitGeoRows = 9;
void launch_unit_geometry(const DevMesh& d, double gamma, const double* cx, const double* cy, double* upf,
                          cudaStream_t s);
void launch_stationary_units(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* fl,
                             cudaStream_t s);
void launch_stationary_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                              cudaStream_t s);
// `nsteps` Go_stationary steps in one cooperative launch (b0: even steps,
// b1: odd steps); returns the launch's error code.
cudaError_t launch_stationary_persistent(const DevMesh& d, const gelios_params& P, const StepBuffers& b0,
                                         const StepBuffers& b1, double* fl, int nsteps, cudaStream_t s);
// Instances of the plain form that share one mesh: parameters, the buffers
// of even / odd steps (dt words included) and the flux slots of each.
struct PlainInstance {
    gelios_params P;
    StepBuffers b[2];
    double* fl;
};
// `nsteps` steps of the instances listed in `active` (device arrays) in one
// cooperative launch; returns the launch's error code.
cudaError_t launch_stationary_batch(const DevMesh& d, const PlainInstance* inst, const int* active, int n_active,
                                    int nsteps, int prec, cudaStream_t s);
void launch_plain_batch_words_init(const PlainInstance* inst, const int* active, int n, cudaStream_t s);
// Tiles of the moving-grid step, built at topology upload: spatially compact
// groups of at most kTileCells cells.  Cells of tile t are
// cells[cstart[t] .. cstart[t+1]); the j-th face slot (Grans order) of
// cells[i] is tile-local slot lbase[i] + j.  faces[fstart[t] .. fstart[t+1])
// are the face units that touch the tile's cells, in unit order: (unit,
// owner's local slot | other side's local slot << 16), kTileNone where that
// side's cell lies in another tile (or there is no other side).
constexpr int kTileCells = 256;
constexpr int kTileNone = 0xffff;
struct TileView {
    int n_tiles = 0, max_slots = 0;
    const int32_t* cstart = nullptr;
    const int32_t* cells = nullptr;
    const int32_t* lbase = nullptr;
    const int32_t* fstart = nullptr;
    const int2* faces = nullptr;
};
// Moving-grid step: reconstruction of the tracked units before the motion
// (rec: kRecRows x n_tracked); after it, every other face unit and the cell
// update in one of two arrangements, kMk2Variants launch shapes in all:
//   variants 0-3  mk2_face_kernel (reconstruction and flux in registers, F.S
//                 to the flux slots in global memory; 128 threads x 8, 5, 6,
//                 4 resident blocks; the plain interior group in its own
//                 launch of a lean instance) + mk2_update_kernel (slot sums,
//                 update);
//   variants 4-7  mk2_tile_kernel, one tile of cells per block, slot fluxes
//                 in shared memory (256 x 3, 256 x 2, 128 x 5, 128 x 4);
//   variants 8-10 as 0-3 with every gather of a face unit prefetched into
//                 L1 as soon as its indices are in (128 threads x 8, 6, 4
//                 resident blocks for the plain interior group).
// Variant 0 is the default; gelios_autotune picks the fastest of the face-
// kernel variants for a grid (kMk2Tuned; the tile kernel is slower in the
// whole step, where the face kernel overlaps the side stream and the tile
// kernel cannot, and is chosen only by hand).  All give the same bits.
void launch_mk2_recon(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* rec, cudaStream_t s);
constexpr int kMk2Variants = 11;
constexpr int kMk2TunedVariants = 7;
constexpr int kMk2Tuned[kMk2TunedVariants] = {0, 1, 2, 3, 8, 9, 10};
const char* mk2_variant_name(int v);
// part 1: the plain interior face units of the face-kernel variants (reads
// the moved points only); part 3: their other untracked units (C_1 interior,
// one-sided), launched on the side stream; part 2: the cell update, or the
// whole tile kernel (also reads the tracked-face fluxes and the source
// terms).  Returns the launch's error.
int mk2_variant_launches(const DevMesh& d, int v, int part);
cudaError_t launch_mk2_cells(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const TileView& t,
                             double* fl, const double* aux, cudaStream_t s, int variant, int part);
int launch_mk2_tracked_solve(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* rec,
                             double* pstar, cudaStream_t s);
int launch_mk2_flux_tracked(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* rec,
                            const double* pstar, double* fl, cudaStream_t s);
// Charge-exchange source terms of the moving-grid step (aux rows q1, q2, q3),
// 128 cells per block (a cell phase, then a species phase).
void launch_mk2_source(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* aux, cudaStream_t s);
void launch_inner(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const int32_t* list, int n,
                  cudaStream_t s);
void launch_dt_finalize(const StepBuffers& b, cudaStream_t s);
void launch_commit(const DevMesh& d, const StepBuffers& b, cudaStream_t s, bool cap = false);
// dt of the next step from the CFL accumulator when the update did not fold
// the 1e7 start in (the pipelined moving-grid step); re-arms the accumulator
void launch_dt_finalize_cap(const StepBuffers& b, cudaStream_t s);
// the moving-grid cell update: mode 0 every cell (1e7 start of the CFL
// minimum folded in), 1 the listed cells, 2 every cell not flagged CF_EARLY,
// 3 every cell (modes 1-3 fold nothing into the CFL accumulator)
void launch_mk2_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       const double* aux, cudaStream_t s, int mode, const int32_t* list, int n_list);
int launch_motion(const DevMesh& d, const gelios_params& P, const StepBuffers& b, double* scratch, cudaStream_t s,
                  bool copy_outer_shock = true);
// Go_5_komponent: face units then the cell update.  Hydrogen state rows
// (ro, p, u, v of H1..H4), 16 rows of n_cells each, of the current and the
// next buffer; fl: kK5FluxRows flux rows per face slot.
constexpr int kK5FluxRows = 21;
void launch_k5(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* hcur, double* hnxt,
               double* fl, cudaStream_t s);
// MHD + pickup-proton form: extra rows (8 x n_cells: w, Bx, By, Bz, pickup
// ro, p, u, v), 13 flux rows per slot, fixed sources (3 x n_cells).
constexpr int kMhdFluxRows = 13;
// The face kernel has kMhdFaceVariants launch shapes (threads per block x
// minimum blocks per SM); variant 0 is the default, gelios_autotune picks
// the fastest for a grid.  All shapes give the same bits.
constexpr int kMhdFaceVariants = 6;
const char* mhd_face_variant_name(int v);
// Returns the number of launches (the plain interior group, then the rest).
// s_rest: stream of the groups other than the plain interior one (null: s)
int launch_mhd_faces(const DevMesh& d, const gelios_params& P, const gelios_mhd_params& M, const StepBuffers& b,
                     const double* hcur, double* fl, cudaStream_t s, int variant = 0, cudaStream_t s_rest = nullptr);
void launch_mhd_update(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       const double* src, const double* hcur, double* hnxt, cudaStream_t s);
// ---- batched MHD step: many instances, one launch per phase
// One instance as the batched kernels read it (each block copies its
// instance into shared memory; the size is a multiple of 16 bytes).
struct alignas(16) BatchInstance {
    DevMesh d;
    gelios_params P;
    gelios_mhd_params M;
    StepBuffers b[2];          // buffers of the even / odd steps of a call
    const double* hs[2];       // extra rows read by the even / odd steps
    double* hn[2];             // extra rows written by them
    double* fl;                // 13 flux rows per face slot
    const double* src;         // fixed charge-exchange sources
    double* surface;           // Move_surface scratch
};
// Block -> (instance, first item) of every phase of a batched step.
struct BatchTables {
    const BatchInstance* inst = nullptr;
    const int2* surf = nullptr;    // 64-thread blocks, two tracked faces each
    const int2* rails = nullptr;   // one block per rail
    const int2* units = nullptr;   // 128 face units per block
    const int2* cells = nullptr;   // 128 cells per block
    const int2* points = nullptr;  // 256 points per block (y == 0: the block that also finalises the dt)
    int n_surf = 0, n_rails = 0, n_units = 0, n_cells = 0, n_points = 0;
    int fp32 = 0;                  // the instances' flux precision (all equal)
};
// sum |a - b| and sum |a| over n doubles into scratch[0], scratch[1]
// (scratch: 2 + 2 * 296 doubles); deterministic.  Returns the launch count.
constexpr int kResidualScratch = 2 + 2 * 296;
// frozen-grid operator residual of the moving-grid step from the mass-flux
// row of the face slots fl (see op_residual_partial_kernel): scratch[0] =
// sum over updated cells of |sum F.S| / volume, scratch[1] = sum |rho|
int launch_op_residual(const DevMesh& d, const gelios_params& P, const StepBuffers& b, const double* fl,
                       double* scratch, cudaStream_t s);
int launch_residual(const double* a, const double* b, int n, double* scratch, cudaStream_t s);
// Words a call starts from (dt0, empty accumulator, zero counters/status),
// on the stream: for one context / for every instance of a batch.
void launch_words_init(void* words, double dt0, cudaStream_t s);
void launch_batch_words_init(const BatchTables& t, int n, cudaStream_t s);
// The five launches of one batched MHD step (parity: even / odd step of the call).
void launch_batch_mhd_step(const BatchTables& t, int parity, cudaStream_t s);
// All phases of `nsteps` batched MHD steps in one cooperative launch of
// blocks_per_sm 128-thread blocks per SM (0: as many as fit); *max_per_sm
// (optional) receives how many fit.  Errors: cudaErrorCooperativeLaunchTooLarge
// when blocks_per_sm exceeds what fits.
cudaError_t launch_batch_mhd_persistent(const BatchTables& t, int nsteps, int blocks_per_sm, cudaStream_t s,
                                        int* max_per_sm = nullptr);

void launch_hllc_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s);
void launch_hlldq_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s);
void launch_hlld_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s);
void launch_godunov_batch(const gelios_params& P, int n, const double* in, double* out, cudaStream_t s);

}  // namespace gelios
