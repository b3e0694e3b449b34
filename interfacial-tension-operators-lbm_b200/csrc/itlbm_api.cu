// itlbm_api.cu -- the C ABI (include/itlbm.h): cases, stepping, diagnostics and the operator seam.
#include "itlbm_site.cuh"

#include <algorithm>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace itlbm {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    // consume the runtime's record of the failure, so that a later call's cudaGetLastError does not
    // report it again (a failed allocation leaves it set; a sticky error stays whatever is done)
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return ITLBM_E_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return ITLBM_E_NODEVICE;
    return ITLBM_E_CUDA;
}
int use_device(int device) {
    const cudaError_t e = cudaSetDevice(device);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "cudaSetDevice");
}

// Per-case parameters derived once on the host, with the reference's expressions so that the
// device sees the same doubles the reference computes inline.
void fill_params(CaseDev &c, const itlbm_operador &op, double tau, double A_fact, double beta,
                 double rho0) {
    c.tipo = op.tipo;
    c.halo = (op.tipo == ITLBM_OP_F1 || op.tipo == ITLBM_OP_F2) ? 2 : 1;
    c.A = A_fact;
    c.sigma = A_fact;
    c.beta = beta;
    c.inv_tau = 1.0 / tau;                // Collision_operators.cpp:18
    c.src_factor = (1. - 1. / (2. * tau));  // LBM_functions.cpp:1648
    if (op.tipo == ITLBM_OP_P1) {         // coef_B, Operadores_tensao.cpp:98
        c.B0 = (1. / 3.) / 3.0;
        c.B1 = (1. / 18.) / 3.0;
        c.B2 = (1. / 36.) / 3.0;
    } else {                              // Operadores_tensao.cpp:101-106
        const double chi = op.chi;
        const double den = 6.0 * chi + 24.0;
        c.B0 = -(2.0 + 2.0 * chi) / (3.0 * chi + 12.0);
        c.B1 = chi / den;
        c.B2 = 1.0 / den;
    }
    c.kf = 0.75 * A_fact * op.xi;           // Operadores_tensao.cpp:240
    c.bf = 3.0 * A_fact / (8.0 * op.xi);    // Operadores_tensao.cpp:241
    c.pf.inv_tau = (float)c.inv_tau;
    c.pf.fac3 = 3.0f * (float)c.src_factor;
    c.pf.A = (float)c.A;
    c.pf.B1 = (float)c.B1;
    c.pf.B2 = (float)c.B2;
    c.pf.Bax = (float)(c.B1 + 2.0 * c.B2);
    c.pf.beta = (float)c.beta;
    c.pf.sigma = (float)c.sigma;
    c.pf.kf = (float)c.kf;
    c.pf.bf = (float)c.bf;
    fill_shift(c, rho0, 0.0);
}

// The FP32 storage shift of a case (see CaseDev): the equilibrium at rho0 and U0 = (u0x, 0).
void fill_shift(CaseDev &c, double rho0, double u0x) {
    c.rho0 = rho0;
    c.u0x = u0x;
    const double u2 = u0x * u0x;
    CaseDev::F32Par &p = c.pf;
    p.rho0 = (float)rho0;
    p.j0x = (float)(rho0 * u0x);
    p.u0b = (float)(rho0 * u2);
    p.s0 = (float)(rho0 * (1.0 - 1.5 * u2));
    p.sx = (float)(rho0 * (1.0 + 3.0 * u2));  // s0 + 4.5 rho0 u0x^2
    p.j3 = (float)(3.0 * rho0 * u0x);
    // the float operations of shift_of (itlbm_site.cuh), so that host and device agree to the bit
    auto shift = [&](float w, int ex) { return w * (ex == 0 ? p.s0 : (ex > 0 ? p.sx + p.j3 : p.sx - p.j3)); };
    for (int i = 0; i < NV; i++) c.sh[i] = shift(wgt<float>(i), cx(i));
    for (int K = 0; K < NK; K++) c.shk[K] = shift(wk<float>(K), kx(K));
}

cudaError_t launch_step(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                        const int *ntiles_dev, int grid, int k, int aux_k, int prec,
                        int shape, cudaStream_t s) {
    if (prec == ITLBM_PREC_F64)
        return launch_step_f64(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
    if (prec == ITLBM_PREC_F32_FOLD)
        return launch_step_fold(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
    return launch_step_f32(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
}

bool narrow_edges_default() {
    const char *v = getenv("ITLBM_NARROW_EDGES");
    return v && std::strcmp(v, "1") == 0;
}

void case_layout(CaseDev &h, int nx, int ny, int prec) {
    h.nx = nx;
    h.ny = ny;
    h.tiles_x = (nx + TX - 1) / TX;
    h.pitch = h.tiles_x * TX;
    h.tiles = h.tiles_x * ((ny + TY - 1) / TY);
    h.tile_elems = 2 * planes_of(prec) * PLANE;
    h.buf_elems = buf_elems_of(nx, ny, prec);
    h.aux_stride = aux_elems_of(nx, ny);
    h.prec = prec;
}

void case_tiles(const CaseDev &h, bool narrow_edges, int case_id, std::vector<TileRef> *out) {
    const int r = h.nx % TX;                               // columns of a partial last tile column
    const int edge = !narrow_edges || r == 0 ? SHAPE_32x8 : (r <= 8 ? SHAPE_8x32 : (r <= 16 ? SHAPE_16x16 : SHAPE_32x8));
    const int full = edge == SHAPE_32x8 ? h.tiles_x : h.tiles_x - 1;  // columns of 32 x 8 tiles
    const int th = TY * rows_per_thread(h.prec);  // rows of a full-width tile
    for (int ty = 0; ty < (h.ny + th - 1) / th; ty++)
        for (int tx = 0; tx < full; tx++) out[SHAPE_32x8].push_back(TileRef{case_id, tile_code(tx * TX, ty * th)});
    if (edge != SHAPE_32x8) {
        const int eh = shape_h(edge) * rows_per_thread(h.prec);
        for (int y0 = 0; y0 < h.ny; y0 += eh) out[edge].push_back(TileRef{case_id, tile_code(full * TX, y0)});
    }
}

cudaError_t case_bind(CaseDev &h, void *mem, size_t per_buf) {
    h.buf[0] = mem;
    h.buf[1] = (char *)mem + per_buf;
    (void)per_buf;
    return cudaSuccess;
}

int step_occupancy(int prec) {
    return prec == ITLBM_PREC_F64 ? step_occupancy_f64() : step_occupancy_f32();
}

static bool op_valid(int t) {
    return t == ITLBM_OP_P1 || t == ITLBM_OP_P3 || t == ITLBM_OP_F1 || t == ITLBM_OP_F2 ||
           t == ITLBM_OP_F3;
}

}  // namespace itlbm

using namespace itlbm;

struct itlbm_case {
    itlbm_case_desc desc{};
    CaseDev host{};
    CaseDev *dev = nullptr;
    TileRef *tiles = nullptr;       // the case's tiles grouped by shape: [tile_off[s], tile_off[s + 1])
    int ntiles = 0;
    int tile_off[NSHAPE + 1] = {};
    void *mem = nullptr;
    double *aux = nullptr;
    double *tmp = nullptr;  // export / import staging (2 * 19 * n doubles)
    DiagScratch diag;
    long long steps = 0;
    int aux_valid = 0;
    int device = 0;
};

extern "C" {

const char *itlbm_version(void) { return "itlbm 0.1.0 (sm_100a)"; }

const char *itlbm_strerror(int code) {
    switch (code) {
        case ITLBM_OK: return "ok";
        case ITLBM_E_ARG: return "invalid argument";
        case ITLBM_E_OOM: return "out of memory";
        case ITLBM_E_CUDA: return "CUDA error";
        case ITLBM_E_NODEVICE: return "no CUDA device";
        case ITLBM_E_NONFINITE: return "non-finite state";
        case ITLBM_E_ADMISSION: return "admission refused";
        case ITLBM_E_TIMEOUT: return "wait timed out";
        case ITLBM_E_PARSE: return "parse error";
        case ITLBM_E_IO: return "I/O error";
        case ITLBM_E_STATE: return "invalid state";
        default: return "unknown error";
    }
}

const char *itlbm_last_error(void) { return g_err.c_str(); }

int itlbm_device_count(int *count) {
    if (!count) return fail(ITLBM_E_ARG, "count is NULL");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        return cuda_fail(e, "cudaGetDeviceCount");
    }
    *count = n;
    return ITLBM_OK;
}

// le_operador (Operadores_tensao.cpp:66-86) on a text: first word, then an optional number.
int itlbm_operador_parse(const char *text, itlbm_operador *op) {
    if (!text || !op) return fail(ITLBM_E_ARG, "NULL argument");
    std::istringstream in(text);
    std::string s;
    if (!(in >> s)) return fail(ITLBM_E_PARSE, "operador: empty");
    itlbm_operador o{};
    o.tipo = ITLBM_OP_P3;
    o.chi = 0.5;
    o.xi = 1.569988;
    std::snprintf(o.nome, sizeof(o.nome), "%s", s.c_str());
    double v;
    if (s == "P1") o.tipo = ITLBM_OP_P1;
    else if (s == "P3") {
        o.tipo = ITLBM_OP_P3;
        if (in >> v) o.chi = v;
    } else if (s == "F1") o.tipo = ITLBM_OP_F1;
    else if (s == "F2") o.tipo = ITLBM_OP_F2;
    else if (s == "F3") {
        o.tipo = ITLBM_OP_F3;
        if (in >> v) o.xi = v;
    } else
        return fail(ITLBM_E_PARSE, "operador: unknown operator '" + s + "'");
    *op = o;
    return ITLBM_OK;
}

int itlbm_operador_read(const char *path, itlbm_operador *op) {
    if (!path || !op) return fail(ITLBM_E_ARG, "NULL argument");
    std::ifstream f(path);
    if (!f) return fail(ITLBM_E_IO, std::string("cannot open ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    return itlbm_operador_parse(ss.str().c_str(), op);
}

void itlbm_case_destroy(itlbm_case *c) {
    if (!c) return;
    if (use_device(c->device) != ITLBM_OK) return;  // the device is gone: nothing left to free on it
    cudaDeviceSynchronize();
    if (c->dev) cudaFree(c->dev);
    if (c->tiles) cudaFree(c->tiles);
    if (c->mem) cudaFree(c->mem);
    if (c->aux) cudaFree(c->aux);
    if (c->tmp) cudaFree(c->tmp);
    diag_free(c->diag);
    delete c;
}

int itlbm_case_create(const itlbm_case_desc *d, itlbm_case **out) {
    if (!d || !out) return fail(ITLBM_E_ARG, "NULL argument");
    *out = nullptr;
    if (d->nx < 1 || d->ny < 1 || (long long)d->nx * d->ny > (1LL << 30) || !box_tileable(d->nx, d->ny))
        return fail(ITLBM_E_ARG, "box size out of range");
    if (!op_valid(d->op.tipo)) return fail(ITLBM_E_ARG, "unknown operator");
    if (!(d->tau > 0.0) || !std::isfinite(d->tau)) return fail(ITLBM_E_ARG, "tau must be > 0");
    if (!prec_valid(d->precision))
        return fail(ITLBM_E_ARG, "unknown precision");
    if (d->geometry == ITLBM_GEOM_STRIP) {
        if (d->nx != d->ny) return fail(ITLBM_E_ARG, "strip needs a square box (Imm_INCL.cpp:243)");
        if (d->p == 0 && d->q == 0) return fail(ITLBM_E_ARG, "strip normal (p, q) = (0, 0)");
    } else if (d->geometry != ITLBM_GEOM_DROP) {
        return fail(ITLBM_E_ARG, "unknown geometry");
    }
    if (d->op.tipo == ITLBM_OP_F3 && !(d->op.xi > 0.0)) return fail(ITLBM_E_ARG, "F3 needs xi > 0");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    itlbm_case *c = new itlbm_case();
    c->desc = *d;
    c->device = dev;
    CaseDev &h = c->host;
    case_layout(h, d->nx, d->ny, d->precision);
    h.parity0 = 0;
    h.chunk_len = INT_MAX;
    h.aux_at_end = 0;
    fill_params(h, d->op, d->tau, d->A_fact, d->beta, d->rho_B > 0 ? d->rho_B : 1.0);
    fill_shift(h, h.rho0, d->geometry == ITLBM_GEOM_DROP ? d->v0 : 0.0);
    const size_t elem = elem_of(d->precision);
    const size_t per_buf = (size_t)h.buf_elems * elem;
    if ((e = cudaMalloc(&c->mem, 2 * per_buf)) != cudaSuccess) {
        itlbm_case_destroy(c);
        return cuda_fail(e, "cudaMalloc(state)");
    }
    if ((e = case_bind(h, c->mem, per_buf)) != cudaSuccess) {
        itlbm_case_destroy(c);
        return cuda_fail(e, "state binding");
    }
    h.aux = nullptr;
    std::vector<TileRef> by_shape[NSHAPE], tl;
    case_tiles(h, narrow_edges_default(), 0, by_shape);
    for (int sh = 0; sh < NSHAPE; sh++) {
        c->tile_off[sh] = (int)tl.size();
        tl.insert(tl.end(), by_shape[sh].begin(), by_shape[sh].end());
    }
    c->tile_off[NSHAPE] = c->ntiles = (int)tl.size();
    if ((e = cudaMalloc(&c->tiles, sizeof(TileRef) * c->ntiles)) != cudaSuccess ||
        (e = cudaMalloc(&c->dev, sizeof(CaseDev))) != cudaSuccess) {
        itlbm_case_destroy(c);
        return cuda_fail(e, "cudaMalloc(tables)");
    }
    cudaMemcpy(c->tiles, tl.data(), sizeof(TileRef) * c->ntiles, cudaMemcpyHostToDevice);
    cudaMemcpy(c->dev, &h, sizeof(CaseDev), cudaMemcpyHostToDevice);
    cudaMemset(c->mem, 0, 2 * per_buf);
    if ((e = launch_init(h, c->dev, *d, 0)) != cudaSuccess ||
        (e = cudaDeviceSynchronize()) != cudaSuccess) {
        itlbm_case_destroy(c);
        return cuda_fail(e, "init");
    }
    *out = c;
    return ITLBM_OK;
}

static int ensure_aux(itlbm_case *c) {
    if (c->aux) return ITLBM_OK;
    cudaError_t e = cudaMalloc(&c->aux, sizeof(double) * 4 * (size_t)c->host.aux_stride);
    if (e != cudaSuccess) {
        c->aux = nullptr;
        return cuda_fail(e, "cudaMalloc(aux)");
    }
    cudaMemset(c->aux, 0, sizeof(double) * 4 * (size_t)c->host.aux_stride);
    c->host.aux = c->aux;
    e = cudaMemcpy(c->dev, &c->host, sizeof(CaseDev), cudaMemcpyHostToDevice);
    // a pageable copy may return before the data lands, and the steps may go to a non-blocking stream
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(case)");
    return ITLBM_OK;
}

int itlbm_case_step(itlbm_case *c, int nsteps, int flags, void *stream) {
    if (!c || nsteps < 0) return fail(ITLBM_E_ARG, "bad argument");
    if (nsteps == 0) return ITLBM_OK;
    if (int rd = use_device(c->device)) return rd;
    const bool keep = (flags & ITLBM_STEP_KEEP_AUX) != 0;
    if (keep) {
        int r = ensure_aux(c);
        if (r) return r;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (c->steps + nsteps > (long long)INT_MAX - 2) return fail(ITLBM_E_STATE, "step counter overflow");
    for (int i = 0; i < nsteps; i++) {
        const int k = (int)(c->steps + i);
        const int aux_k = (keep && i == nsteps - 1) ? k : -1;
        for (int sh = 0; sh < NSHAPE; sh++) {  // the tile shapes of one step touch disjoint nodes
            const int n = c->tile_off[sh + 1] - c->tile_off[sh];
            if (n == 0) continue;
            cudaError_t e = launch_step(c->dev, c->tiles + c->tile_off[sh], n, nullptr, n, k, aux_k,
                                        c->host.prec, sh, s);
            if (e != cudaSuccess) return cuda_fail(e, "step kernel");
        }
    }
    c->steps += nsteps;
    c->aux_valid = keep ? 1 : 0;
    return ITLBM_OK;
}

int itlbm_case_sync(itlbm_case *c) {
    if (!c) return fail(ITLBM_E_ARG, "NULL case");
    if (int rd = use_device(c->device)) return rd;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "synchronize");
    return ITLBM_OK;
}

long long itlbm_case_steps_done(const itlbm_case *c) { return c ? c->steps : -1; }

int itlbm_case_save(itlbm_case *c, const char *path) {
    if (!c || !path) return fail(ITLBM_E_ARG, "NULL argument");
    if (int rd = use_device(c->device)) return rd;
    cudaError_t e = cudaDeviceSynchronize();  // steps may have gone to another stream
    if (e != cudaSuccess) return cuda_fail(e, "synchronize");
    return snap_write(path, c->desc, c->steps, c->host, c->host.buf[c->steps & 1]);
}

int itlbm_snapshot_info(const char *path, itlbm_case_desc *desc, long long *steps) {
    if (!path || !desc || !steps) return fail(ITLBM_E_ARG, "NULL argument");
    SnapHeader hd;
    const int r = snap_read_header(path, hd);
    if (r) return r;
    *desc = hd.desc;
    *steps = hd.steps;
    return ITLBM_OK;
}

int itlbm_case_load(const char *path, itlbm_case **out) {
    if (!path || !out) return fail(ITLBM_E_ARG, "NULL argument");
    *out = nullptr;
    SnapHeader hd;
    int r = snap_read_header(path, hd);
    if (r) return r;
    itlbm_case *c = nullptr;
    if ((r = itlbm_case_create(&hd.desc, &c)) != ITLBM_OK) return r;
    c->steps = hd.steps;
    if ((r = snap_read_state(path, c->host, c->host.buf[c->steps & 1])) != ITLBM_OK) {
        itlbm_case_destroy(c);
        return r;
    }
    *out = c;
    return ITLBM_OK;
}

static int ensure_diag(itlbm_case *c) {
    const cudaError_t e = diag_alloc(c->diag, c->host.nx, c->host.ny);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "cudaMalloc(diagnostics)");
}

int itlbm_case_diag_drop(itlbm_case *c, int step, double x_ini, double y_ini, itlbm_drop_diag *out,
                         void *stream) {
    if (!c || !out) return fail(ITLBM_E_ARG, "NULL argument");
    if (c->steps < 1) return fail(ITLBM_E_STATE, "no step has run yet");
    const bool force = c->host.tipo >= ITLBM_OP_F1;
    if (force && !c->aux_valid)
        return fail(ITLBM_E_STATE, "class F: the last step must keep aux (ITLBM_STEP_KEEP_AUX)");
    if (int rd = use_device(c->device)) return rd;
    int r = ensure_diag(c);
    if (r) return r;
    cudaStream_t s = (cudaStream_t)stream;
    const int cur = (int)(c->steps & 1);
    itlbm_drop_diag *od = (itlbm_drop_diag *)diag_scratch_out(c->diag);
    cudaError_t e = launch_diag_drop(c->dev, c->host, c->diag, cur, step, c->desc.v0, x_ini, y_ini,
                                     force, od, s);
    if (e != cudaSuccess) return cuda_fail(e, "diagnostic kernels");
    if ((e = cudaMemcpyAsync(out, od, sizeof(itlbm_drop_diag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "diagnostic copy");
    out->step = step;
    return ITLBM_OK;
}

// The same kernels as itlbm_case_diag_drop on a fixed device scratch; no allocation of any kind.
int itlbm_case_diag_drop_static(itlbm_case *c, int step, double x_ini, double y_ini,
                                itlbm_drop_diag *out, void *stream) {
    if (!c || !out) return fail(ITLBM_E_ARG, "NULL argument");
    const int nx = c->host.nx, ny = c->host.ny;
    if (nx > ITLBM_STATIC_DIAG_MAX_SIDE || ny > ITLBM_STATIC_DIAG_MAX_SIDE ||
        (long long)nx * ny > ITLBM_STATIC_DIAG_MAX_NODES)
        return fail(ITLBM_E_ARG, "itlbm_case_diag_drop_static: case of " + std::to_string(nx) + " x " +
                                     std::to_string(ny) + " nodes is larger than the static scratch (at most " +
                                     std::to_string(ITLBM_STATIC_DIAG_MAX_NODES) + " nodes, sides up to " +
                                     std::to_string(ITLBM_STATIC_DIAG_MAX_SIDE) +
                                     "); use itlbm_case_diag_drop");
    if (c->steps < 1) return fail(ITLBM_E_STATE, "no step has run yet");
    const bool force = c->host.tipo >= ITLBM_OP_F1;
    if (force && !c->aux_valid)
        return fail(ITLBM_E_STATE, "class F: the last step must keep aux (ITLBM_STEP_KEEP_AUX)");
    if (int rd = use_device(c->device)) return rd;
    cudaError_t e;
    void *base = nullptr;
    size_t bytes = 0;
    if ((e = static_diag_scratch(c->device, &base, &bytes)) != cudaSuccess)
        return cuda_fail(e, "cudaGetSymbolAddress(static diagnostic scratch)");
    DiagScratch s;
    if ((e = diag_bind(s, base, bytes, nx, ny)) != cudaSuccess)
        return fail(ITLBM_E_ARG, "itlbm_case_diag_drop_static: case does not fit the static scratch");
    cudaStream_t st = (cudaStream_t)stream;
    itlbm_drop_diag *od = (itlbm_drop_diag *)diag_scratch_out(s);
    e = launch_diag_drop(c->dev, c->host, s, (int)(c->steps & 1), step, c->desc.v0, x_ini, y_ini, force,
                         od, st);
    if (e != cudaSuccess) return cuda_fail(e, "diagnostic kernels");
    if ((e = cudaMemcpyAsync(out, od, sizeof(itlbm_drop_diag), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "diagnostic copy");
    out->step = step;
    return ITLBM_OK;
}

int itlbm_case_diag_strip(itlbm_case *c, int step, itlbm_strip_diag *out, void *stream) {
    if (!c || !out) return fail(ITLBM_E_ARG, "NULL argument");
    if (c->desc.geometry != ITLBM_GEOM_STRIP) return fail(ITLBM_E_STATE, "not a strip case");
    if (c->steps < 1) return fail(ITLBM_E_STATE, "no step has run yet");
    if (!c->aux_valid) return fail(ITLBM_E_STATE, "the last step must keep aux (ITLBM_STEP_KEEP_AUX)");
    if (int rd = use_device(c->device)) return rd;
    int r = ensure_diag(c);
    if (r) return r;
    cudaStream_t s = (cudaStream_t)stream;
    const int cur = (int)(c->steps & 1);
    itlbm_strip_diag *od = (itlbm_strip_diag *)diag_scratch_out(c->diag);
    cudaError_t e = launch_diag_strip(c->dev, c->host, c->diag, cur, step, c->desc.p, c->desc.q,
                                      c->host.tipo >= ITLBM_OP_F1, od, s);
    if (e != cudaSuccess) return cuda_fail(e, "diagnostic kernels");
    if ((e = cudaMemcpyAsync(out, od, sizeof(itlbm_strip_diag), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return cuda_fail(e, "diagnostic copy");
    out->step = step;
    return ITLBM_OK;
}

static int ensure_tmp(itlbm_case *c) {
    if (c->tmp) return ITLBM_OK;
    const size_t n = (size_t)c->host.nx * c->host.ny;
    cudaError_t e = cudaMalloc(&c->tmp, sizeof(double) * 2 * NV * n);
    if (e != cudaSuccess) {
        c->tmp = nullptr;
        return cuda_fail(e, "cudaMalloc(staging)");
    }
    return ITLBM_OK;
}

int itlbm_case_read_pops(itlbm_case *c, int which, double *fR, double *fB) {
    if (!c || !fR || !fB || (which != 0 && which != 1)) return fail(ITLBM_E_ARG, "bad argument");
    if (which == 1 && c->steps < 1) return fail(ITLBM_E_STATE, "no step has run yet");
    if (int rd = use_device(c->device)) return rd;
    int r = ensure_tmp(c);
    if (r) return r;
    const size_t n = (size_t)c->host.nx * c->host.ny;
    const int cur = (int)(c->steps & 1);
    cudaError_t e = cudaDeviceSynchronize();  // steps may have gone to another stream
    if (e == cudaSuccess) e = launch_export(c->dev, c->host.nx, c->host.ny, cur, which, c->tmp, c->tmp + NV * n, 0);
    if (e == cudaSuccess) e = cudaMemcpy(fR, c->tmp, sizeof(double) * NV * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(fB, c->tmp + NV * n, sizeof(double) * NV * n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "read_pops");
}

int itlbm_case_write_pops(itlbm_case *c, const double *fR, const double *fB) {
    if (!c || !fR || !fB) return fail(ITLBM_E_ARG, "bad argument");
    if (int rd = use_device(c->device)) return rd;
    int r = ensure_tmp(c);
    if (r) return r;
    const size_t n = (size_t)c->host.nx * c->host.ny;
    const int cur = (int)(c->steps & 1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(c->tmp, fR, sizeof(double) * NV * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->tmp + NV * n, fB, sizeof(double) * NV * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_import(c->dev, c->host.nx, c->host.ny, cur, c->tmp, c->tmp + NV * n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    c->aux_valid = 0;
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "write_pops");
}

static int read_fields_as(itlbm_case *c, int form, double *rho_R, double *rho_B, double *ux, double *uy,
                          double *uz, double *force) {
    if (!c) return fail(ITLBM_E_ARG, "NULL case");
    if (c->steps < 1) return fail(ITLBM_E_STATE, "no step has run yet");
    const bool cls_f = c->host.tipo >= ITLBM_OP_F1;
    if ((cls_f || force) && !c->aux_valid)
        return fail(ITLBM_E_STATE, "the last step must keep aux (ITLBM_STEP_KEEP_AUX)");
    if (int rd = use_device(c->device)) return rd;
    int r = ensure_tmp(c);
    if (r) return r;
    const size_t n = (size_t)c->host.nx * c->host.ny;
    double *t = c->tmp;
    cudaError_t e = cudaDeviceSynchronize();  // steps may have gone to another stream
    if (e == cudaSuccess)
        e = launch_fields(c->dev, c->host, (int)(c->steps & 1), cls_f, form, t, t + n, t + 2 * n, t + 3 * n,
                          t + 4 * n, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    double *outs[5] = {rho_R, rho_B, ux, uy, uz};
    for (int k = 0; k < 5 && e == cudaSuccess; k++)
        if (outs[k]) e = cudaMemcpy(outs[k], t + k * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && force) {
        std::vector<double> a(3 * n);
        for (int k = 0; k < 3 && e == cudaSuccess; k++)
            e = cudaMemcpy2D(a.data() + k * n, sizeof(double) * c->host.nx,
                             c->aux + (size_t)k * c->host.aux_stride, sizeof(double) * c->host.pitch,
                             sizeof(double) * c->host.nx, c->host.ny, cudaMemcpyDeviceToHost);
        for (size_t p = 0; p < n; p++)
            for (int k = 0; k < 3; k++) force[3 * p + k] = a[k * n + p];
    }
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "read_fields");
}

int itlbm_case_read_fields(itlbm_case *c, double *rho_R, double *rho_B, double *ux, double *uy,
                           double *uz, double *force) {
    return read_fields_as(c, ITLBM_FIELDS_VTK, rho_R, rho_B, ux, uy, uz, force);
}

int itlbm_case_read_profile(itlbm_case *c, double *rho_R, double *rho_B, double *ux, double *uy) {
    return read_fields_as(c, ITLBM_FIELDS_PROFILE, rho_R, rho_B, ux, uy, nullptr, nullptr);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// operator seam on the device (kernels in itlbm_seam.cu)
// ---------------------------------------------------------------------------------------------
namespace itlbm {
namespace {
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};
}  // namespace
}  // namespace itlbm

extern "C" {

int itlbm_dev_perturbacao(const itlbm_operador *op, double A, int n, const double *g, double *f) {
    if (!op || n < 0 || (n > 0 && (!g || !f))) return fail(ITLBM_E_ARG, "bad argument");
    if (op->tipo != ITLBM_OP_P1 && op->tipo != ITLBM_OP_P3) return fail(ITLBM_E_ARG, "not a class-P operator");
    if (n == 0) return ITLBM_OK;
    CaseDev c{};
    fill_params(c, *op, 1.0, A, 0.0, 1.0);
    DevBuf dg, df;
    cudaError_t e = cudaMalloc(&dg.p, sizeof(double) * 3 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&df.p, sizeof(double) * NV * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(dg.p, g, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(df.p, f, sizeof(double) * NV * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        seam_perturb(n, A, c.B0, c.B1, c.B2, (const double *)dg.p, (double *)df.p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(f, df.p, sizeof(double) * NV * (size_t)n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "dev_perturbacao");
}

int itlbm_dev_source(int n, const double *F, const double *u, const double *rho, double tau, double *S) {
    (void)rho;  // source() receives rho but does not use it (LBM_functions.cpp:1603-1673)
    if (n < 0 || (n > 0 && (!F || !u || !S)) || !(tau > 0)) return fail(ITLBM_E_ARG, "bad argument");
    if (n == 0) return ITLBM_OK;
    DevBuf dF, du, dS;
    cudaError_t e = cudaMalloc(&dF.p, sizeof(double) * 3 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&du.p, sizeof(double) * 3 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dS.p, sizeof(double) * NV * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(dF.p, F, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(du.p, u, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        seam_source(n, (const double *)dF.p, (const double *)du.p, (1. - 1. / (2. * tau)),
                    (double *)dS.p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(S, dS.p, sizeof(double) * NV * (size_t)n, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "dev_source");
}

// Runs the fused step kernel itself on the given populations and returns the force it computed,
// so this check exercises exactly the device code of the hot path.
int itlbm_dev_calcula_forca(const itlbm_operador *op, double sigma, int nx, int ny,
                            const double *fR, const double *fB, double *F) {
    if (!op || !fR || !fB || !F) return fail(ITLBM_E_ARG, "NULL argument");
    if (op->tipo < ITLBM_OP_F1) return fail(ITLBM_E_ARG, "not a class-F operator");
    itlbm_case_desc d{};
    d.nx = nx;
    d.ny = ny;
    d.op = *op;
    d.tau = 1.0;
    d.beta = 0.8;
    d.A_fact = sigma;
    d.rho_R = 1.0;
    d.rho_B = 1.0;
    d.geometry = ITLBM_GEOM_DROP;
    d.precision = ITLBM_PREC_F64;
    itlbm_case *c = nullptr;
    int r = itlbm_case_create(&d, &c);
    if (r) return r;
    r = itlbm_case_write_pops(c, fR, fB);
    if (!r) r = itlbm_case_step(c, 1, ITLBM_STEP_KEEP_AUX, nullptr);
    if (!r) r = itlbm_case_sync(c);
    if (!r) {
        const size_t n = (size_t)nx * ny;
        std::vector<double> a(3 * n);
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < 3 && e == cudaSuccess; k++)
            e = cudaMemcpy2D(a.data() + k * n, sizeof(double) * nx, c->aux + (size_t)k * c->host.aux_stride,
                             sizeof(double) * c->host.pitch, sizeof(double) * nx, ny, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) r = cuda_fail(e, "dev_calcula_forca");
        else
            for (size_t p = 0; p < n; p++)
                for (int k = 0; k < 3; k++) F[3 * p + k] = a[k * n + p];
    }
    itlbm_case_destroy(c);
    return r;
}

int itlbm_dev_colisao_comum(const itlbm_operador *op, double tau, double A_fact, double beta, int n,
                            double *fR, double *fB, const double *gm, const double *F) {
    if (!op || n < 0 || (n > 0 && (!fR || !fB || !gm))) return fail(ITLBM_E_ARG, "bad argument");
    if (!op_valid(op->tipo) || !(tau > 0)) return fail(ITLBM_E_ARG, "bad operator or tau");
    const bool force = op->tipo >= ITLBM_OP_F1;
    if (force && !F) return fail(ITLBM_E_ARG, "class F needs F");
    if (n == 0) return ITLBM_OK;
    CaseDev c{};
    fill_params(c, *op, tau, A_fact, beta, 1.0);
    DevBuf dR, dB, dg, dF;
    const size_t m = sizeof(double) * NV * (size_t)n, v3 = sizeof(double) * 3 * (size_t)n;
    cudaError_t e = cudaMalloc(&dR.p, m);
    if (e == cudaSuccess) e = cudaMalloc(&dB.p, m);
    if (e == cudaSuccess) e = cudaMalloc(&dg.p, v3);
    if (e == cudaSuccess) e = cudaMalloc(&dF.p, v3);
    if (e == cudaSuccess) e = cudaMemcpy(dR.p, fR, m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB.p, fB, m, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dg.p, gm, v3, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && force) e = cudaMemcpy(dF.p, F, v3, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        seam_colisao(n, c, force, (double *)dR.p, (double *)dB.p, (const double *)dg.p,
                     (const double *)dF.p);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(fR, dR.p, m, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(fB, dB.p, m, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "dev_colisao_comum");
}

}  // extern "C"
