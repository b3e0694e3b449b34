// itlbm_internal.h -- definitions shared by the CUDA translation units of libitlbm.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/itlbm.h"

namespace itlbm {

constexpr int NV = 19;

// Tiles of the fused step: 256 threads, one node each (two in the fold, see rows_per_thread), in one
// of three shapes; the phase field is staged with a halo of up to HMAX nodes (1 for P1/P3/F3, 2 for
// F1/F2).  A case is tiled by 32 x 8 tiles (a warp per row of 32 nodes); the last tile column, when
// nx is not a multiple of 32,
// can instead be cut into 16 x 16 or 8 x 32 tiles (a warp covering 2 or 4 row pieces of 16 or 8
// nodes), which leaves fewer threads idle beyond the box's edge.  The shape changes no result: a
// node's update is the same whichever tile computes it.
constexpr int TX = 32;             // the base shape 32 x 8
constexpr int TY = 8;
constexpr int HMAX = 2;
constexpr int STEP_THREADS = 256;
enum { SHAPE_32x8 = 0, SHAPE_16x16 = 1, SHAPE_8x32 = 2, NSHAPE = 3 };
__host__ __device__ constexpr int shape_w(int s) { return s == SHAPE_32x8 ? 32 : (s == SHAPE_16x16 ? 16 : 8); }
__host__ __device__ constexpr int shape_h(int s) { return STEP_THREADS / shape_w(s); }
// Rows of a tile per thread: the fold's threads take two nodes each (rows ly and ly + 256 / W), so
// its tiles are 32 x 16 (or 16 x 32, 8 x 64 at a partial edge); the other storage forms take one.
// Measured on B200: two rows made the fold 13 % faster; for the D3Q19 FP32 form (38 values per node)
// they need 80-128 registers and were 7-12 % slower at 3 or 2 CTAs per SM.
#ifndef ITLBM_FOLD_ROWS
#define ITLBM_FOLD_ROWS 2
#endif
#ifndef ITLBM_F32_ROWS
#define ITLBM_F32_ROWS 1
#endif
__host__ __device__ constexpr int rows_per_thread(int prec) {
    return prec == ITLBM_PREC_F32_FOLD ? ITLBM_FOLD_ROWS : (prec == ITLBM_PREC_F32 ? ITLBM_F32_ROWS : 1);
}
// D3Q19 velocity set in the order of def_lattice_d3q19 (SimBoltz_Functions/LBM_functions.cpp:366-497)
__host__ __device__ constexpr int cx(int i) {
    constexpr int t[NV] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[i];
}
__host__ __device__ constexpr int cy(int i) {
    constexpr int t[NV] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, -1, 1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int cz(int i) {
    constexpr int t[NV] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, 1, -1};
    return t[i];
}
__host__ __device__ constexpr int cc(int i) { return cx(i) * cx(i) + cy(i) * cy(i) + cz(i) * cz(i); }
template <class T>
__host__ __device__ constexpr T wgt(int i) {
    return i == 0 ? T(1.) / T(3.) : (i < 7 ? T(1.) / T(18.) : T(1.) / T(36.));
}

// In-plane fold of D3Q19 for the one-node slab (FP32 fold storage, ITLBM_PREC_F32_FOLD).  With one
// node in z and periodic z, a direction with c_z = +-1 streams to the same (x, y) as its in-plane
// projection, and a z-symmetric state (every initial state here) stays z-symmetric, so the 19
// populations of a colour group into nine classes of equal in-plane velocity e_K whose sums evolve
// exactly as a D2Q9 lattice with weights W_K = sum of the members' w_i (4/9, 1/9, 1/36):
//   K0 {0, 5, 6}  K1 +x {1, 11, 13}  K2 -x {2, 12, 14}  K3 +y {3, 16, 18}  K4 -y {4, 15, 17}
//   K5 {7}  K6 {8}  K7 {9}  K8 {10}            (classes 2m - 1 and 2m are opposite, m = 1..4)
constexpr int NK = 9;
__host__ __device__ constexpr int fold_class(int i) {
    constexpr int t[NV] = {0, 1, 2, 3, 4, 0, 0, 5, 6, 7, 8, 1, 2, 1, 2, 4, 3, 4, 3};
    return t[i];
}
__host__ __device__ constexpr int kx(int K) {
    constexpr int t[NK] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
    return t[K];
}
__host__ __device__ constexpr int ky(int K) {
    constexpr int t[NK] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
    return t[K];
}
__host__ __device__ constexpr int kk(int K) { return kx(K) * kx(K) + ky(K) * ky(K); }
template <class T>
__host__ __device__ constexpr T wk(int K) {
    return K == 0 ? T(4.) / T(9.) : (K < 5 ? T(1.) / T(9.) : T(1.) / T(36.));
}

// storage planes per colour and bytes per element of a precision
__host__ __device__ constexpr int planes_of(int prec) { return prec == ITLBM_PREC_F32_FOLD ? NK : NV; }
__host__ __device__ constexpr int elem_of(int prec) { return prec == ITLBM_PREC_F64 ? 8 : 4; }
__host__ __device__ constexpr bool prec_valid(int prec) {
    return prec == ITLBM_PREC_F64 || prec == ITLBM_PREC_F32 || prec == ITLBM_PREC_F32_FOLD;
}

// Compile-time loop: f(std::integral_constant<int, i>) for i in [B, E).
template <int B, int E, class F>
__host__ __device__ __forceinline__ void sfor(F &&f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        sfor<B + 1, E>(f);
    }
}

// Per-case descriptor read by the step and diagnostic kernels (device memory).
//
// Layout of a state buffer: tile-major.  The box is cut into the 32 x 8 tiles of the step, stored
// in row-major order of tiles (tiles_x per tile row).  Each tile is one contiguous block of
// tile_elems = 2 colours x planes x 256 elements; plane q of the block (q = colour x planes + i)
// holds the tile's 256 nodes in row-major order.  Element (q, x, y) is node_off(x, y) + q * PLANE,
// so all planes of a node are at compile-time offsets from one address: the step forms one address
// per node it loads and one per neighbour it pushes to, instead of one per plane.  A tile reads each
// plane as one contiguous 1 KiB (FP32) block, and its halo and pushed values fall into at most eight
// neighbouring blocks.  On B200 the data movement of the step alone (76 planes read at the node and
// written at x + c_i) measured 5.9-6.1 TB/s with tile-blocked planes against 5.2-5.4 TB/s for planes
// of plain rows.  The auxiliary arrays keep plain rows (y * pitch + x): they are written at
// diagnostic steps only and copied to the host row by row.
struct CaseDev {
    void *buf[2];          // the two state buffers, buf_elems elements each (tile-major)
    double *aux;           // 4 arrays of aux_stride doubles in plain rows: Fx, Fy, Fz, |grad rho^N| (may be null)
    long long buf_elems;   // elements per state buffer: tiles * tile_elems
    long long aux_stride;  // elements per auxiliary array: pitch * ny
    int tile_elems;        // elements per tile block: 2 x planes x PLANE
    int nx, ny, pitch;     // box and row pitch of the auxiliary arrays (elements): pitch = 32 tiles_x
    int tiles_x, tiles;    // tiles of this case
    int tipo;              // ITLBM_OP_*
    int halo;              // phase-field halo: 1 (P1, P3, F3) or 2 (F1, F2)
    int prec;              // ITLBM_PREC_*
    int parity0;           // buffer index holding the state at sub-step k = 0
    int chunk_len;         // sub-steps to run in this launch sequence (INT_MAX for single cases)
    int aux_at_end;        // keep aux at sub-step chunk_len - 1
    double A;              // amplitude (class P)
    double sigma;          // tension (class F)
    double beta;           // recolouring factor
    double inv_tau;        // 1.0 / tau                       (Collision_operators.cpp:18)
    double src_factor;     // 1. - 1. / (2. * tau)             (LBM_functions.cpp:1648)
    double B0, B1, B2;     // coef_B of |c|^2 = 0, 1, 2        (Operadores_tensao.cpp:94-109)
    double kf, bf;         // F3: k = 3 sigma xi / 4, b = 3 sigma / (8 xi) (Operadores_tensao.cpp:240-241)
    double rho0;           // FP32 shifted storage: reference density of the shift below
    // FP32 shifted storage: e_i = f_i - s_i with s_i the equilibrium at density rho0 and velocity
    // U0 = (u0x, 0), the case's initial flow (a translating drop's v0 along x; zero otherwise):
    //   s_i = w_i rho0 (1 + 3 c_ix u0x + 4.5 (c_ix u0x)^2 - 1.5 u0x^2).
    // A uniform shift commutes with streaming, and with U0 the stored deviations stay small where the
    // fluid moves with the drop, so their rounding stays at the scale of the deviations.  The kernels
    // form s_i = w_i (c_ix == 0 ? s0 : sx +- j3) from three floats; sh and shk hold the same values,
    // formed by the host with the same float operations, for import, export and the diagnostics.
    double u0x;
    float sh[NV];          // s_i of each direction
    float shk[NK];         // fold: shift of each class, the sum of its members' s_i
    // The parameters of the FP32 kernels, rounded to float once by the host (the same roundings the
    // kernels made per thread before), in one 16-byte aligned block read with four vector loads.
    struct alignas(16) F32Par {
        float rho0, inv_tau, fac3, A;  // fac3 = 3 src_factor
        float B1, B2, Bax, beta;       // Bax = B1 + 2 B2 (the fold's axis classes)
        float sigma, kf, bf, j0x;      // j0x = rho0 u0x
        float u0b, s0, sx, j3;         // rho0 u0x^2; rho0 (1 - 1.5 u0x^2), the s_i / w_i of the
                                       // directions with c_ix = 0; s0 + 4.5 rho0 u0x^2; 3 rho0 u0x
    } pf;
};

// The FP32 parameter block of a case, four 16-byte loads.
__device__ __forceinline__ CaseDev::F32Par load_pf(const CaseDev &c) {
    const float4 *q = reinterpret_cast<const float4 *>(&c.pf);
    const float4 a = q[0], b = q[1], d = q[2], e = q[3];
    return CaseDev::F32Par{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, d.x, d.y, d.z, d.w, e.x, e.y, e.z, e.w};
}

// Offset of node (x, y) within a state buffer (tile-major, see CaseDev; plane q adds q * PLANE),
// and within an auxiliary array (plain rows).  Tile indices fit 32 bits (each side of a box is at
// most 8 x 65535 nodes); the offsets are 64-bit.
constexpr int PLANE = TX * TY;
__host__ __device__ __forceinline__ long long node_off(int tiles_x, int tile_elems, int x, int y) {
    return (long long)((y >> 3) * tiles_x + (x >> 5)) * tile_elems + (((y & 7) << 5) + (x & 31));
}
__host__ __device__ __forceinline__ long long node_off(const CaseDev &c, int x, int y) {
    return node_off(c.tiles_x, c.tile_elems, x, y);
}
__host__ __device__ __forceinline__ long long aux_off(const CaseDev &c, int x, int y) { return (long long)y * c.pitch + x; }
// Elements of one state buffer of an nx x ny box in storage form prec, and of one auxiliary array.
__host__ __device__ __forceinline__ long long buf_elems_of(int nx, int ny, int prec) {
    return (long long)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * (2 * planes_of(prec) * PLANE);
}
__host__ __device__ __forceinline__ long long aux_elems_of(int nx, int ny) {
    return (long long)((nx + TX - 1) / TX) * TX * ny;
}

// An entry of the work table: case index and work item within that case.  For the tile kernel the
// item is the tile's origin in units of 8 nodes, packed as ((y0 / 8) << 16) | (x0 / 8) (no division
// in the kernel).
struct TileRef {
    int case_id;
    int tile;
};
// Boxes whose sides do not fit 16 bits in units of 8 nodes are refused at creation.
constexpr int MAX_TILE_COORD = 65535;
inline bool box_tileable(int nx, int ny) {
    return (nx + 7) / 8 <= MAX_TILE_COORD && (ny + 7) / 8 <= MAX_TILE_COORD;
}
inline int tile_code(int x0, int y0) { return (int)(((unsigned)(y0 / 8) << 16) | (unsigned)(x0 / 8)); }

// The FP32 storage shift of a case: the equilibrium at density rho0 and velocity (u0x, 0).
void fill_shift(CaseDev &c, double rho0, double u0x);

// ---- kernel launchers (defined in the .cu files) -------------------------------------------
cudaError_t launch_step_f64(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                            const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s);
cudaError_t launch_step_f32(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                            const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s);
cudaError_t launch_step_fold(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                             const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s);
int step_occupancy_f64();
int step_occupancy_f32();
int step_occupancy(int prec);
void seam_perturb(int n, double A, double B0, double B1, double B2, const double *g, double *f);
void seam_source(int n, const double *F, const double *u, double factor, double *S);
void seam_colisao(int n, const CaseDev &c, bool force, double *fR, double *fB, const double *gm,
                  const double *F);
// Layout of a case's state and its tiles, and the binding of its state block.
void case_layout(CaseDev &h, int nx, int ny, int prec);
// The tiles of a case with index case_id, appended to out[shape] (NSHAPE vectors): 32 x 8, and with
// narrow_edges a last partial tile column of r = nx mod 32 columns cut into 8 x 32 tiles (r <= 8) or
// 16 x 16 tiles (8 < r <= 16).
void case_tiles(const CaseDev &h, bool narrow_edges, int case_id, std::vector<TileRef> *out);
cudaError_t case_bind(CaseDev &h, void *mem, size_t per_buf);
// Whether single cases cut a partial last tile column into narrow tiles (ITLBM_NARROW_EDGES=1): off
// by default, since each shape is a launch of its own and a single case's steps are launch-bound
// below about 10^6 nodes; the batch's autotuner chooses for itself.
bool narrow_edges_default();
// The step kernel of storage form `prec`; `shape` is the tile shape of every entry of `tiles`.
cudaError_t launch_step(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                        const int *ntiles_dev, int grid, int k, int aux_k, int prec, int shape,
                        cudaStream_t s);
cudaError_t launch_init(const CaseDev &c, const CaseDev *c_dev, const itlbm_case_desc &d,
                        cudaStream_t s);  // single cases: stages the profile, waits
size_t profile_len(const CaseDev &c, const itlbm_case_desc &d);
bool profile_on_device(const itlbm_case_desc &d);  // FP32 drops: the init kernel evaluates the profile
void init_profile(const CaseDev &c, const itlbm_case_desc &d, double *prof);  // host, profile_len values
void init_profile_rows(const CaseDev &c, const itlbm_case_desc &d, double *prof, int ya, int yb);
cudaError_t launch_init_from(const CaseDev &c, const CaseDev *c_dev, const itlbm_case_desc &d,
                             const double *prof, cudaStream_t s);  // prof readable by the device
// Export populations to FP64 AoS (reference layout).  which = 0: state of buffer `cur`;
// which = 1: post-collision of the last step (gathered from buffer `cur`).
cudaError_t launch_export(const CaseDev *c_dev, int nx, int ny, int cur, int which, double *fR,
                          double *fB, cudaStream_t s);
cudaError_t launch_import(const CaseDev *c_dev, int nx, int ny, int cur, const double *fR,
                          const double *fB, cudaStream_t s);

// One diagnostic of one case: where its case descriptor, its scratch and its result are, and what
// to measure.  The drop and strip diagnostics of any number of cases run as one sequence of launches
// over a table of these (itlbm_batch.cu), or of a single one passed by value (a single case).  Every
// case keeps the reduction order it has alone -- its own number of partial blocks, visited in the
// same order -- so a case gives the same bits alone and in a batch.
struct DiagJob {
    const CaseDev *c;             // the case descriptor (device memory)
    double *node;                 // drop: per node rho_R, rho_B, ux, uy, uz, phi (6 arrays of n)
    double *part;                 // per-block partials, nblocks rows
    unsigned long long *shell;    // drop: shell histogram (fixed point) and counts, 2 x nshell
    void *state;                  // running state of the diagnostic
    void *out;                    // itlbm_drop_diag or itlbm_strip_diag (device memory)
    double *rays;                 // drop: the harmonic products of the 256 rays, 7 x 256
    double v0, x_ini, y_ini;
    int cur, step, use_force;
    int n, nblocks, nshell;       // nodes, partial blocks and shells of the case
    int block0;                   // first block of this job in the grids of the full-field passes
    int p, q;                     // strip normal
};
// Layout of one job's scratch: bytes needed for an nx x ny case (a drop needs more than a strip), and
// the job's pointers laid out in a 256-byte aligned block of at least that many bytes.
size_t diag_job_bytes(int nx, int ny, int geometry);
void diag_job_layout(DiagJob &j, void *base, int nx, int ny, int geometry);
// Partial blocks of a full-field pass over n nodes (part of the reduction order of a case).
int diag_nblocks(long long n);
// A diagnostic of every job of a table on one stream: jobs_dev[njobs], all of one geometry, with the
// full-field passes over total_blocks blocks, blk_job[b] the job of block b.
cudaError_t launch_diag_jobs(const DiagJob *jobs_dev, int njobs, const int *blk_job, int total_blocks,
                             int geometry, cudaStream_t st);

// Diagnostic scratch of a single case, allocated on demand (or bound to a block the caller holds).
struct DiagScratch {
    void *base = nullptr;
    size_t bytes = 0;
    bool owned = false;
};
cudaError_t diag_alloc(DiagScratch &s, int nx, int ny);  // on failure s is left empty
void diag_free(DiagScratch &s);
// Bytes of one diagnostic scratch for an nx x ny case, and the same scratch laid out in a block the
// caller already holds (256-byte aligned, at least diag_bytes long); diag_bind allocates nothing and
// the block stays the caller's (diag_free leaves a bound block alone).
size_t diag_bytes(int nx, int ny);
cudaError_t diag_bind(DiagScratch &s, void *base, size_t bytes, int nx, int ny);
// Where a diagnostic on this scratch leaves its result when launched with out_dev == nullptr.
void *diag_scratch_out(const DiagScratch &s);
// The static scratch of itlbm_case_diag_drop_static on the current device: its address (looked up
// once per device) and its size in bytes.
cudaError_t static_diag_scratch(int device, void **base, size_t *bytes);
// One diagnostic of a single case on its scratch; out_dev receives the result (device memory).
cudaError_t launch_diag_drop(const CaseDev *c_dev, const CaseDev &c, DiagScratch &s, int cur,
                             int step, double v0, double x_ini, double y_ini, bool use_force,
                             itlbm_drop_diag *out_dev, cudaStream_t st);
cudaError_t launch_diag_strip(const CaseDev *c_dev, const CaseDev &c, DiagScratch &s, int cur,
                              int step, int p, int q, bool use_force, itlbm_strip_diag *out_dev,
                              cudaStream_t st);
cudaError_t launch_fields(const CaseDev *c_dev, const CaseDev &c, int cur, bool use_force, int form,
                          double *rho_R, double *rho_B, double *ux, double *uy, double *uz,
                          cudaStream_t st);

// ---- case snapshots (itlbm_snapshot.cu) ------------------------------------------------------
struct SnapHeader {
    char magic[8];            // "ITLBMST1"
    int version;              // 1
    itlbm_case_desc desc;
    long long steps;          // steps done: the state is the one at the top of step `steps`
};
// `state` is the device buffer holding the state at the top of the next step.
int snap_write(const char *path, const itlbm_case_desc &d, long long steps, const CaseDev &h, const void *state);
int snap_read_header(const char *path, SnapHeader &hd);
int snap_read_state(const char *path, const CaseDev &h, void *state);

// ---- error reporting -------------------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
// cudaSetDevice with its return checked: ITLBM_OK or the failure, with the message set.
int use_device(int device);

}  // namespace itlbm
