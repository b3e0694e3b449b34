// itlbm_diag.cu -- diagnostics of one case on the device (FP64 accumulation).
//
// The reference measures every PASSOS_DIAG steps on the host (Imm_OPS.cpp:293-342,
// Imm_INCL.cpp:400-434).  Here every full-field pass is a grid-stride kernel whose threads
// accumulate in FP64, reduce within the block by warp shuffles and write one partial per block; a
// one-block kernel then reduces the partials in block order.  The order depends only on the size of
// the case, so a case gives the same bits alone or in a batch.  The shell histogram of the logistic
// fit is accumulated in 64-bit fixed point (2^-40), which makes its atomics order-independent too.
// The scalar finalisation (centroid angle, fits, ratios) runs in single-thread kernels, so one
// diagnostic is a chain of launches on one stream with a single copy of the result at the end.
//
// Passes of a drop diagnostic (post-collision populations P(x)_i = dst(x + c_i, i)):
//   D1  calc_galilean's first loop (Galilean_diagnostics.cpp:31-60) and calc_drop_radius's first
//       loop (Other_functions.cpp:89-178); writes rho_R, rho_B, u, phi per node
//   F1  means, centroid, equimolar radius (Galilean_diagnostics.cpp:61-63, Other_functions.cpp:180-190)
//   D2  calc_drop_radius's second loop (:211-249), calc_laplace_tension's loop (:488-526),
//       calc_galilean's second loop (Galilean_diagnostics.cpp:68-87) and the shell histogram of
//       calc_perfil_logistico (Other_functions.cpp:341-377)
//   F2  pressures, sigma, axis ratio, line estimators (:530-553, Galilean_diagnostics.cpp:88-104)
//   FIT calc_perfil_logistico's fit (Other_functions.cpp:381-445)
//   MOD modos_interface (Operadores_tensao.cpp:382-449), one thread per ray
#include "itlbm_site.cuh"

#include <cfloat>
#include <math_constants.h>

namespace itlbm {

namespace {

constexpr int DT = 256;        // threads of the reduction kernels
constexpr int MAXB = 148 * 8;  // at most this many partials per pass
constexpr double FIX = 1099511627776.0;  // 2^40

// Post-collision populations of node (x, y) in FP64.
__device__ __forceinline__ void post_pops(const CaseDev &c, int cur, int x, int y, double *fR,
                                          double *fB) {
    const int xp = (x + 1 == c.nx) ? 0 : x + 1, xm = (x == 0) ? c.nx - 1 : x - 1;
    const int yp = (y + 1 == c.ny) ? 0 : y + 1, ym = (y == 0) ? c.ny - 1 : y - 1;
    if (c.prec == ITLBM_PREC_F64) {
        const double *d = (const double *)c.buf[cur];
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int xs = cx(i) == 0 ? x : (cx(i) > 0 ? xp : xm);
            const int ys = cy(i) == 0 ? y : (cy(i) > 0 ? yp : ym);
            const long long o = node_off(c, xs, ys);
            fR[i] = d[o + i * PLANE];
            fB[i] = d[o + (NV + i) * PLANE];
        });
    } else if (c.prec == ITLBM_PREC_F32) {
        const float *d = (const float *)c.buf[cur];
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const int xs = cx(i) == 0 ? x : (cx(i) > 0 ? xp : xm);
            const int ys = cy(i) == 0 ? y : (cy(i) > 0 ? yp : ym);
            const long long o = node_off(c, xs, ys);
            const double e = d[o + i * PLANE];
            const double dd = d[o + (NV + i) * PLANE];
            const double f = (double)c.sh[i] + e;
            fR[i] = 0.5 * (f + dd);
            fB[i] = 0.5 * (f - dd);
        });
    } else {  // fold: class K was pushed to x + e_K, the same in-plane shift as each of its members;
              // the class is split among its members by weight (exact for every moment)
        const float *d = (const float *)c.buf[cur];
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            constexpr int K = fold_class(i);
            const int xs = cx(i) == 0 ? x : (cx(i) > 0 ? xp : xm);
            const int ys = cy(i) == 0 ? y : (cy(i) > 0 ? yp : ym);
            const long long o = node_off(c, xs, ys);
            const double share = wgt<double>(i) / wk<double>(K);
            const double f = ((double)c.shk[K] + d[o + K * PLANE]) * share;
            const double dd = d[o + (NK + K) * PLANE] * share;
            fR[i] = 0.5 * (f + dd);
            fB[i] = 0.5 * (f - dd);
        });
    }
}

__device__ __forceinline__ bool finite_d(double v) { return isfinite(v); }

// Block reduction of Q quantities: [0, NS) sums, [NS, NS+NM) maxima, the rest minima.  Writes the
// block's result to out[0..Q).  Deterministic for a fixed block size.
template <int Q, int NS, int NM>
__device__ void block_reduce(double (&v)[Q], double *out) {
    __shared__ double sh[DT / 32][Q];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        double a = v[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double b = __shfl_down_sync(0xffffffffu, a, o);
            if (q < NS) a = a + b;
            else if (q < NS + NM) a = (a < b) ? b : a;
            else a = (b < a) ? b : a;
        }
        if (lane == 0) sh[warp][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        double a = sh[0][q];
        for (int w = 1; w < DT / 32; w++) {
            const double b = sh[w][q];
            if (q < NS) a = a + b;
            else if (q < NS + NM) a = (a < b) ? b : a;
            else a = (b < a) ? b : a;
        }
        out[q] = a;
    }
    __syncthreads();
}

template <int Q, int NS, int NM>
__device__ __forceinline__ void init_acc(double (&v)[Q]) {
#pragma unroll
    for (int q = 0; q < Q; q++) v[q] = (q < NS) ? 0.0 : (q < NS + NM ? -DBL_MAX : DBL_MAX);
}

// The job of this block of a full-field pass and the block's index within the job: a table of jobs
// with a block -> job map, or the single job passed by value (jobs == nullptr).
__device__ __forceinline__ const DiagJob &block_job(const DiagJob *jobs, const int *blk_job,
                                                    const DiagJob &one, int &lb) {
    if (!jobs) {
        lb = blockIdx.x;
        return one;
    }
    const DiagJob &J = jobs[blk_job[blockIdx.x]];
    lb = blockIdx.x - J.block0;
    return J;
}

// Reduce nb partials (rows of Q) in block order into res[0..Q) (one block).
template <int Q, int NS, int NM>
__device__ void reduce_rows(const double *__restrict__ part, int nb, double *__restrict__ res) {
    double v[Q];
    init_acc<Q, NS, NM>(v);
    for (int b = threadIdx.x; b < nb; b += DT) {
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const double x = part[(long long)b * Q + q];
            if (q < NS) v[q] = v[q] + x;
            else if (q < NS + NM) v[q] = (v[q] < x) ? x : v[q];
            else v[q] = (x < v[q]) ? x : v[q];
        }
    }
    block_reduce<Q, NS, NM>(v, res);
}

// ---------------------------------------------------------------------------------------------
// drop
// ---------------------------------------------------------------------------------------------
// D1 quantities
enum {
    A_MASS, A_MASSR, A_QXG, A_QYG, A_QZG, A_QRX, A_QRY, A_MASSA_R, A_MASSA_B, A_QXD, A_QYD, A_QZD,
    A_U2, A_AREA, A_CXC, A_CXS, A_CYC, A_CYS, A_BAD, A_NEGT, A_NEGC, A_RUIM,  // sums (22)
    A_UMAXD, A_MAXPHI,                                                        // maxima (2)
    A_MINF, A_MINRHO, A_MINPHI,                                               // minima (3)
    A_Q
};
constexpr int A_NS = 22, A_NM = 2;
// D2 quantities
enum {
    B_SOMW, B_SOMWR, B_SXE, B_SWE, B_SXD, B_SWD, B_PIN, B_PIN2, B_POUT, B_POUT2, B_PCTR, B_NIN,
    B_NOUT, B_NCTR, B_SREF, B_SMEAN, B_SLAB, B_WEIGHT, B_SX, B_SY, B_SXX, B_SYY, B_SXY, B_LW, B_LX,
    B_RW, B_RX,                       // sums (27)
    B_MAXREF, B_MAXMEAN, B_MAXLAB,    // maxima (3)
    B_Q
};
constexpr int B_NS = 27, B_NM = 3;

// device-side state of one drop diagnostic
struct DropState {
    double a[A_Q];
    double b[B_Q];
    int proceed;      // D1 passed (no bad node, positive masses)
    int y_lin, y_line;
    double r_in_max, r_out_min;
    double fit[6];
};

__global__ void __launch_bounds__(DT) k_drop_d1(const DiagJob *__restrict__ jobs,
                                                const int *__restrict__ blk_job,
                                                const __grid_constant__ DiagJob one) {
    int lb;
    const DiagJob &J = block_job(jobs, blk_job, one, lb);
    const CaseDev &c = *J.c;
    const int cur = J.cur, use_force = J.use_force, nb = J.nblocks;
    double *__restrict__ node = J.node;
    const int nx = c.nx, ny = c.ny;
    const long long n = (long long)nx * ny;
    const double pi = 3.14159265358979323846;
    const double tx = 2.0 * pi / (double)nx, ty = 2.0 * pi / (double)ny;
    double v[A_Q];
    init_acc<A_Q, A_NS, A_NM>(v);
    for (long long p = lb * (long long)DT + threadIdx.x; p < n; p += (long long)nb * DT) {
        const int x = (int)(p % nx), y = (int)(p / nx);
        double fR[NV], fB[NV];
        post_pops(c, cur, x, y, fR, fB);
        // calc_galilean, first loop
        double rr = 0, rb = 0, mx = 0, my = 0, mz = 0;
        int bad = 0;
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const double fr = fR[i], fb = fB[i];
            const double f = fr + fb;
            if (!finite_d(fr) || !finite_d(fb)) ++bad;
            v[A_MINF] = (f < v[A_MINF]) ? f : v[A_MINF];
            if (f < -1.e-12) v[A_NEGT] += 1.0;
            if (fr < -1.e-12) v[A_NEGC] += 1.0;
            if (fb < -1.e-12) v[A_NEGC] += 1.0;
            rr += fr;
            rb += fb;
            if constexpr (cx(i) == 1) mx += f;
            if constexpr (cx(i) == -1) mx -= f;
            if constexpr (cy(i) == 1) my += f;
            if constexpr (cy(i) == -1) my -= f;
            if constexpr (cz(i) == 1) mz += f;
            if constexpr (cz(i) == -1) mz -= f;
        });
        const double rho = rr + rb;
        double ux = 0, uy = 0, uz = 0, ph = 0;
        bool ok = true;
        if (!finite_d(rho) || rho <= 0 || !finite_d(mx) || !finite_d(my) || !finite_d(mz)) {
            ++bad;
            ok = false;
        }
        double F0 = 0, F1 = 0, F2 = 0;
        if (ok && use_force) {
            const long long o = aux_off(c, x, y);
            F0 = c.aux[o];
            F1 = c.aux[c.aux_stride + o];
            F2 = c.aux[2 * c.aux_stride + o];
            if (!finite_d(F0) || !finite_d(F1) || !finite_d(F2)) {
                ++bad;
                ok = false;
            } else {
                mx -= 0.5 * F0;
                my -= 0.5 * F1;
                mz -= 0.5 * F2;
            }
        }
        v[A_BAD] += bad;
        if (ok) {
            v[A_MINRHO] = (rho < v[A_MINRHO]) ? rho : v[A_MINRHO];
            ux = mx / rho;
            uy = my / rho;
            uz = mz / rho;
            ph = rr / rho;
            v[A_MINPHI] = (ph < v[A_MINPHI]) ? ph : v[A_MINPHI];
            v[A_MAXPHI] = (v[A_MAXPHI] < ph) ? ph : v[A_MAXPHI];
            v[A_MASS] += rho;
            v[A_MASSR] += rr;
            v[A_QXG] += mx;
            v[A_QYG] += my;
            v[A_QZG] += mz;
            v[A_QRX] += rr * ux;
            v[A_QRY] += rr * uy;
        }
        node[p] = rr;
        node[n + p] = rb;
        node[2 * n + p] = ux;
        node[3 * n + p] = uy;
        node[4 * n + p] = uz;
        node[5 * n + p] = ph;
        // calc_drop_radius, first loop (calcula per colour, LBM_functions.cpp:1100-1171)
        double mRx = 0, mRy = 0, mRz = 0, mBx = 0, mBy = 0, mBz = 0;
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            if constexpr (cx(i) == 1) { mRx += fR[i]; mBx += fB[i]; }
            if constexpr (cx(i) == -1) { mRx -= fR[i]; mBx -= fB[i]; }
            if constexpr (cy(i) == 1) { mRy += fR[i]; mBy += fB[i]; }
            if constexpr (cy(i) == -1) { mRy -= fR[i]; mBy -= fB[i]; }
            if constexpr (cz(i) == 1) { mRz += fR[i]; mBz += fB[i]; }
            if constexpr (cz(i) == -1) { mRz -= fR[i]; mBz -= fB[i]; }
        });
        const double rho_R = rr, rho_B = rb;
        double vxR = 0, vyR = 0, vzR = 0, vxB = 0, vyB = 0, vzB = 0;
        if (rho_R != 0.0) {
            const double inv = 1.0 / rho_R;
            vxR = mRx * inv; vyR = mRy * inv; vzR = mRz * inv;
        }
        if (rho_B != 0.0) {
            const double inv = 1.0 / rho_B;
            vxB = mBx * inv; vyB = mBy * inv; vzB = mBz * inv;
        }
        if (!(rho_R == rho_R) || !(rho_B == rho_B) || !(vxR == vxR) || !(vxB == vxB)) {
            v[A_RUIM] += 1.0;
            continue;
        }
        v[A_MASSA_R] += rho_R;
        v[A_MASSA_B] += rho_B;
        v[A_QXD] += rho_R * vxR + rho_B * vxB;
        v[A_QYD] += rho_R * vyR + rho_B * vyB;
        v[A_QZD] += rho_R * vzR + rho_B * vzB;
        const double rh = rho_R + rho_B;
        if (rh <= 0.0) continue;
        double uxd = (rho_R * vxR + rho_B * vxB) / rh;
        double uyd = (rho_R * vyR + rho_B * vyB) / rh;
        double uzd = (rho_R * vzR + rho_B * vzB) / rh;
        if (use_force) {
            const long long o = aux_off(c, x, y);
            const double G0 = c.aux[o], G1 = c.aux[c.aux_stride + o], G2 = c.aux[2 * c.aux_stride + o];
            uxd = uxd - 0.5 * G0 / rh;
            uyd = uyd - 0.5 * G1 / rh;
            uzd = uzd - 0.5 * G2 / rh;
            v[A_QXD] -= 0.5 * G0;
            v[A_QYD] -= 0.5 * G1;
            v[A_QZD] -= 0.5 * G2;
        }
        const double u2 = uxd * uxd + uyd * uyd + uzd * uzd;
        v[A_U2] += u2;
        const double u = sqrt(u2);
        if (u > v[A_UMAXD]) v[A_UMAXD] = u;
        const double phi = rho_R / rh;
        v[A_AREA] += phi;
        v[A_CXC] += phi * cos(tx * x);
        v[A_CXS] += phi * sin(tx * x);
        v[A_CYC] += phi * cos(ty * y);
        v[A_CYS] += phi * sin(ty * y);
    }
    block_reduce<A_Q, A_NS, A_NM>(v, J.part + (long long)lb * A_Q);
}

__global__ void k_drop_f1(const DiagJob *__restrict__ jobs, int njobs, const __grid_constant__ DiagJob one) {
    const int jid = blockIdx.x * blockDim.x + threadIdx.x;
    if (jid >= njobs) return;
    const DiagJob &J = jobs ? jobs[jid] : one;
    const CaseDev &c = *J.c;
    DropState *__restrict__ st = (DropState *)J.state;
    itlbm_drop_diag *__restrict__ d = (itlbm_drop_diag *)J.out;
    const double *a = st->a;
    const int nx = c.nx, ny = c.ny;
    const double pi = 3.14159265358979323846;
    d->bad = (int)a[A_BAD];
    d->min_f = a[A_MINF] == DBL_MAX ? INFINITY : a[A_MINF];
    d->min_rho = a[A_MINRHO] == DBL_MAX ? INFINITY : a[A_MINRHO];
    d->min_phi = a[A_MINPHI] > 1.0 ? 1.0 : a[A_MINPHI];
    d->max_phi = a[A_MAXPHI] < 0.0 ? 0.0 : a[A_MAXPHI];
    d->negative_total = (long long)a[A_NEGT];
    d->negative_color = (long long)a[A_NEGC];
    d->axis_ratio = 1.0;
    const double mass = a[A_MASS], mass_r = a[A_MASSR];
    st->proceed = !(d->bad || !(mass > 0) || !(mass_r > 0));
    d->ok = 0;
    if (!st->proceed) return;
    d->mean_x = a[A_QXG] / mass;
    d->mean_y = a[A_QYG] / mass;
    d->mean_z = a[A_QZG] / mass;
    d->drop_x = a[A_QRX] / mass_r;
    d->drop_y = a[A_QRY] / mass_r;
    // calc_drop_radius, Other_functions.cpp:180-190 (nz = 1, cilindro)
    const double tx = 2.0 * pi / (double)nx, ty = 2.0 * pi / (double)ny;
    double x0 = atan2(a[A_CXS], a[A_CXC]) / tx;
    if (x0 < 0.0) x0 += nx;
    double y0 = atan2(a[A_CYS], a[A_CYC]) / ty;
    if (y0 < 0.0) y0 += ny;
    const double area = a[A_AREA];
    const double raio = (area > 0.0) ? sqrt(area / (pi * 1.0)) : 0.0;
    d->x0 = x0;
    d->y0 = y0;
    d->area = area;
    d->raio = raio;
    d->massa_R = a[A_MASSA_R];
    d->massa_B = a[A_MASSA_B];
    d->qx = a[A_QXD];
    d->qy = a[A_QYD];
    d->qz = a[A_QZD];
    const int n_fluid = nx * ny;
    d->n_fluid = n_fluid;
    d->n_ruim = (int)a[A_RUIM];
    d->u_max = a[A_UMAXD] < 0 ? 0.0 : a[A_UMAXD];
    d->u_rms = (n_fluid > 0) ? sqrt(a[A_U2] / (double)n_fluid) : 0.0;
    int y_lin = (int)(y0 + 0.5);
    if (y_lin >= ny) y_lin -= ny;
    st->y_lin = y_lin;
    st->y_line = ((int)floor(y0 + 0.5)) % ny;
    // calc_laplace_tension region limits, Other_functions.cpp:471-479 (frac 0.5 / 2.0, 3.45)
    double r_in_max = 0.5 * raio, r_out_min = 2.0 * raio;
    if (r_out_min < raio + 4.0 * 3.45) r_out_min = raio + 4.0 * 3.45;
    const double r_caixa = 0.45 * (double)((nx < ny) ? nx : ny);
    if (r_out_min > r_caixa) r_out_min = r_caixa;
    st->r_in_max = r_in_max;
    st->r_out_min = r_out_min;
}

__device__ __forceinline__ double min_image(double dx, int L) {
    if (dx > 0.5 * L) dx -= L;
    if (dx < -0.5 * L) dx += L;
    return dx;
}
__device__ __forceinline__ double gi_image(double dx, double L) { return dx - L * floor(dx / L + 0.5); }

__global__ void __launch_bounds__(DT) k_drop_d2(const DiagJob *__restrict__ jobs,
                                                const int *__restrict__ blk_job,
                                                const __grid_constant__ DiagJob one) {
    int lb;
    const DiagJob &J = block_job(jobs, blk_job, one, lb);
    const DropState *__restrict__ st = (const DropState *)J.state;
    if (!st->proceed) return;
    const itlbm_drop_diag *__restrict__ d = (const itlbm_drop_diag *)J.out;
    const double v0 = J.v0;
    const double *__restrict__ node = J.node;
    unsigned long long *__restrict__ shell = J.shell;
    const int nshell = J.nshell, nb = J.nblocks;
    const CaseDev &c = *J.c;
    const int nx = c.nx, ny = c.ny;
    const long long n = (long long)nx * ny;
    const double x0 = d->x0, y0 = d->y0;
    const double mean_x = d->mean_x, mean_y = d->mean_y, mean_z = d->mean_z;
    const int y_lin = st->y_lin, y_line = st->y_line;
    const double r_in_max = st->r_in_max, r_out_min = st->r_out_min;
    double v[B_Q];
    init_acc<B_Q, B_NS, B_NM>(v);
    for (long long p = lb * (long long)DT + threadIdx.x; p < n; p += (long long)nb * DT) {
        const int x = (int)(p % nx), y = (int)(p / nx);
        const double rho_R = node[p], rho_B = node[n + p];
        const double ux = node[2 * n + p], uy = node[3 * n + p], uz = node[4 * n + p];
        const double phg = node[5 * n + p];
        // calc_drop_radius, second loop
        const double dx = min_image((double)x - x0, nx), dy = min_image((double)y - y0, ny);
        const double r = sqrt(dx * dx + dy * dy + 0.0 * 0.0);
        const double w = rho_R * rho_B;
        v[B_SOMW] += w;
        v[B_SOMWR] += w * r;
        if (y == y_lin) {
            if (dx < 0.0) { v[B_SXE] += w * (double)x; v[B_SWE] += w; }
            else { v[B_SXD] += w * (double)x; v[B_SWD] += w; }
        }
        // calc_laplace_tension
        const double pr = (1. / 3.) * (rho_R + rho_B);
        if (r < r_in_max) { v[B_PIN] += pr; v[B_PIN2] += pr * pr; v[B_NIN] += 1.0; }
        else if (r >= r_out_min) { v[B_POUT] += pr; v[B_POUT2] += pr * pr; v[B_NOUT] += 1.0; }
        if (r < 1.5) { v[B_PCTR] += pr; v[B_NCTR] += 1.0; }
        // calc_galilean, second loop
        const double a2 = (ux - v0) * (ux - v0) + uy * uy + uz * uz;
        const double b2 = (ux - mean_x) * (ux - mean_x) + (uy - mean_y) * (uy - mean_y) +
                          (uz - mean_z) * (uz - mean_z);
        const double c2 = ux * ux + uy * uy + uz * uz;
        v[B_SREF] += a2;
        v[B_SMEAN] += b2;
        v[B_SLAB] += c2;
        const double sa = sqrt(a2), sb = sqrt(b2), sc = sqrt(c2);
        v[B_MAXREF] = (v[B_MAXREF] < sa) ? sa : v[B_MAXREF];
        v[B_MAXMEAN] = (v[B_MAXMEAN] < sb) ? sb : v[B_MAXMEAN];
        v[B_MAXLAB] = (v[B_MAXLAB] < sc) ? sc : v[B_MAXLAB];
        const double gx = gi_image(x - x0, nx), gy = gi_image(y - y0, ny);
        v[B_WEIGHT] += phg;
        v[B_SX] += phg * gx;
        v[B_SY] += phg * gy;
        v[B_SXX] += phg * gx * gx;
        v[B_SYY] += phg * gy * gy;
        v[B_SXY] += phg * gx * gy;
        if (y == y_line) {
            const double wl = rho_R * rho_B;
            if (gx < 0) { v[B_LW] += wl; v[B_LX] += wl * gx; }
            else { v[B_RW] += wl; v[B_RX] += wl * gx; }
        }
        // calc_perfil_logistico shell histogram (half-node shells)
        const double rho = rho_R + rho_B;
        if (!(rho <= 1.0e-30)) {
            const int k = (int)(r / 0.5);
            if (k >= 0 && k < nshell) {
                const long long fx = __double2ll_rn((rho_R / rho) * FIX);
                atomicAdd(&shell[k], (unsigned long long)fx);
                atomicAdd(&shell[nshell + k], 1ULL);
            }
        }
    }
    block_reduce<B_Q, B_NS, B_NM>(v, J.part + (long long)lb * B_Q);
}

__global__ void k_drop_f2(const DiagJob *__restrict__ jobs, int njobs, const __grid_constant__ DiagJob one) {
    const int jid = blockIdx.x * blockDim.x + threadIdx.x;
    if (jid >= njobs) return;
    const DiagJob &J = jobs ? jobs[jid] : one;
    DropState *__restrict__ st = (DropState *)J.state;
    if (!st->proceed) return;
    itlbm_drop_diag *__restrict__ d = (itlbm_drop_diag *)J.out;
    const int step = J.step;
    const double v0 = J.v0, x_ini = J.x_ini, y_ini = J.y_ini;
    const double *__restrict__ node = J.node;
    const CaseDev &c = *J.c;
    const int nx = c.nx, ny = c.ny;
    const long long n = (long long)nx * ny;
    const double *b = st->b;
    d->raio_grad = (b[B_SOMW] > 0.0) ? b[B_SOMWR] / b[B_SOMW] : 0.0;
    const double raio_linha_d =
        (b[B_SWE] > 0.0 && b[B_SWD] > 0.0) ? 0.5 * (b[B_SXD] / b[B_SWD] - b[B_SXE] / b[B_SWE]) : 0.0;
    const int n_in = (int)b[B_NIN], n_out = (int)b[B_NOUT], n_ctr = (int)b[B_NCTR];
    const double p_in = (n_in > 0) ? b[B_PIN] / (double)n_in : 0.0;
    const double p_out = (n_out > 0) ? b[B_POUT] / (double)n_out : 0.0;
    const double var_in = (n_in > 0) ? b[B_PIN2] / (double)n_in - p_in * p_in : 0.0;
    const double var_out = (n_out > 0) ? b[B_POUT2] / (double)n_out - p_out * p_out : 0.0;
    d->p_in = p_in;
    d->sd_in = (var_in > 0.0) ? sqrt(var_in) : 0.0;
    d->p_out = p_out;
    d->sd_out = (var_out > 0.0) ? sqrt(var_out) : 0.0;
    d->n_in = n_in;
    d->n_out = n_out;
    d->delta_p = p_in - p_out;
    d->sigma = 1.0 * d->raio * d->delta_p;
    d->p_centro = (n_ctr > 0) ? b[B_PCTR] / (double)n_ctr : 0.0;
    d->p_canto = (1. / 3.) * (node[0] + node[n]);  // pos == 0
    d->sigma_linha = 1.0 * raio_linha_d * (d->p_centro - d->p_canto);
    d->raio_linha = raio_linha_d;
    // calc_galilean, Galilean_diagnostics.cpp:88-104
    const int nn = nx * ny;
    d->max_ref = b[B_MAXREF] < 0 ? 0.0 : b[B_MAXREF];
    d->max_mean = b[B_MAXMEAN] < 0 ? 0.0 : b[B_MAXMEAN];
    d->max_lab = b[B_MAXLAB] < 0 ? 0.0 : b[B_MAXLAB];
    d->rms_ref = sqrt(b[B_SREF] / nn);
    d->rms_mean = sqrt(b[B_SMEAN] / nn);
    d->rms_lab = sqrt(b[B_SLAB] / nn);
    const double weight = b[B_WEIGHT], sx = b[B_SX], sy = b[B_SY];
    const double xx = b[B_SXX] / weight - (sx / weight) * (sx / weight);
    const double yy = b[B_SYY] / weight - (sy / weight) * (sy / weight);
    const double xy = b[B_SXY] / weight - (sx / weight) * (sy / weight), trace = xx + yy;
    const double disc = sqrt((xx - yy) * (xx - yy) + 4 * xy * xy);
    d->axis_ratio = (trace > disc) ? sqrt((trace + disc) / (trace - disc)) : INFINITY;
    d->center_dx = gi_image(d->x0 - (x_ini + v0 * step), nx);
    d->center_dy = gi_image(d->y0 - y_ini, ny);
    d->x_unwrapped = x_ini + v0 * step + d->center_dx;
    d->raio_linha = (b[B_LW] > 0 && b[B_RW] > 0) ? 0.5 * (b[B_RX] / b[B_RW] - b[B_LX] / b[B_LW]) : 0;
    const int corner_x = ((int)floor(d->x0 + 0.5) + nx / 2) % nx;
    const int corner_y = ((int)floor(d->y0 + 0.5) + ny / 2) % ny;
    const long long pc = corner_x + (long long)nx * corner_y;
    d->p_canto = node[pc] * (1. / 3.) + node[n + pc] * (1. / 3.);
    d->sigma_linha = d->raio_linha * (d->p_centro - d->p_canto);
    d->u_max = d->max_ref;
    d->u_rms = d->rms_ref;
    d->ok = isfinite(d->sigma) && isfinite(d->max_ref) && isfinite(d->axis_ratio);
    st->proceed = d->ok;
}

// calc_perfil_logistico's fit over the shells (one block)
__global__ void __launch_bounds__(DT) k_drop_fit(const DiagJob *__restrict__ jobs,
                                                 const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x] : one;
    DropState *__restrict__ st = (DropState *)J.state;
    if (!st->proceed) return;
    itlbm_drop_diag *__restrict__ d = (itlbm_drop_diag *)J.out;
    const unsigned long long *__restrict__ shell = J.shell;
    const int nshell = J.nshell;
    const double eps = 1.0e-30, d_casca = 0.5;
    double v[6];
    init_acc<6, 6, 0>(v);
    for (int k = threadIdx.x; k < nshell; k += DT) {
        const double sn = (double)shell[nshell + k];
        if (sn < 1.0) continue;
        const double sphi = (double)(long long)shell[k] / FIX;
        const double phi = sphi / sn;
        if (phi <= 0.02 || phi >= 0.98) continue;
        const double r = ((double)k + 0.5) * d_casca;
        const double l = log(phi / (1.0 - phi));
        v[0] += 1.0;
        v[1] += r;
        v[2] += l;
        v[3] += r * r;
        v[4] += r * l;
        v[5] += 1.0;
    }
    __shared__ double res[6];
    block_reduce<6, 6, 0>(v, res);
    const double S = res[0], Sr = res[1], Sl = res[2], Srr = res[3], Srl = res[4];
    const int n_usadas = (int)res[5];
    double K = 0.0, r_meio = 0.0, a = 0.0, bb = 0.0;
    bool fit = false;
    if (n_usadas >= 3) {
        const double den = S * Srr - Sr * Sr;
        if (fabs(den) > eps) {
            a = (S * Srl - Sr * Sl) / den;
            bb = (Sl - a * Sr) / S;
            K = -a;
            if (fabs(a) > eps) r_meio = -bb / a;
            fit = true;
        }
    }
    double m[1] = {0.0};
    if (fit) {
        for (int k = threadIdx.x; k < nshell; k += DT) {
            const double sn = (double)shell[nshell + k];
            if (sn < 1.0) continue;
            const double phi = ((double)(long long)shell[k] / FIX) / sn;
            if (phi <= 0.02 || phi >= 0.98) continue;
            const double r = ((double)k + 0.5) * d_casca;
            const double dd = fabs(log(phi / (1.0 - phi)) - (a * r + bb));
            if (dd > m[0]) m[0] = dd;
        }
    }
    __shared__ double mres[1];
    block_reduce<1, 0, 1>(m, mres);
    if (threadIdx.x == 0) {
        d->K_perfil = K;
        d->r_perfil = r_meio;
        d->res_perfil = fit ? mres[0] : 0.0;
        d->esp_perfil = (K > eps) ? 2.0 * log(9.0) / K : 0.0;
        d->n_perfil = n_usadas;
    }
}

// modos_interface: one thread per ray, bisection on the bilinear rho^N field
__device__ double fase_em(const double *__restrict__ node, long long n, int nx, int ny, double x,
                          double y) {
    if (!isfinite(x) || !isfinite(y)) return 0.0;  // keeps every index below in range
    x = x - nx * floor(x / nx);
    y = y - ny * floor(y / ny);
    const int i0 = (int)floor(x), j0 = (int)floor(y);  // in [0, nx] x [0, ny]
    const double tx = x - i0, ty = y - j0;
    double v = 0.0;
    for (int dj = 0; dj < 2; dj++)
        for (int di = 0; di < 2; di++) {
            int ii = i0 + di, jj = j0 + dj;  // periodic image, without integer division
            if (ii >= nx) ii -= nx;
            if (ii >= nx) ii -= nx;
            if (jj >= ny) jj -= ny;
            if (jj >= ny) jj -= ny;
            const long long p = ii + (long long)jj * nx;
            const double rR = node[p], rB = node[n + p];
            const double wgt2 = (di ? tx : 1 - tx) * (dj ? ty : 1 - ty);
            v += wgt2 * (rR - rB) / (rR + rB);
        }
    return v;
}

// modos_interface: one warp per ray.  The reference bisects 60 times from [0.3 R, 1.7 R], keeping the
// sign of rho^N at the inner end; here each round evaluates, one point per lane, all 31 midpoints the
// next five bisections can visit (the 5-level tree under the current interval, each midpoint formed
// from its interval exactly as the serial bisection forms it), then walks the tree by the signs.  The
// 12 rounds take the same path and give the same interval, bit for bit, with 12 dependent
// evaluations instead of 60.
constexpr int RAYS_PER_BLOCK = DT / 32;
constexpr int MODE_BLOCKS = ITLBM_N_ANG / RAYS_PER_BLOCK;  // blocks per job
__global__ void __launch_bounds__(DT) k_drop_modes(const DiagJob *__restrict__ jobs,
                                                   const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x / MODE_BLOCKS] : one;
    const DropState *__restrict__ st = (const DropState *)J.state;
    if (!st->proceed) return;
    const itlbm_drop_diag *__restrict__ d = (const itlbm_drop_diag *)J.out;
    const CaseDev &c = *J.c;
    const int nx = c.nx, ny = c.ny;
    const long long n = (long long)nx * ny;
    const double *__restrict__ node = J.node;
    const int N_ANG = ITLBM_N_ANG;
    const int lane = threadIdx.x & 31;
    const int k = (blockIdx.x % MODE_BLOCKS) * RAYS_PER_BLOCK + (threadIdx.x >> 5);
    const double x0 = d->x0, y0 = d->y0, R_est = d->raio;
    const double th = 2.0 * 3.14159265358979323846 * k / N_ANG, ct = cos(th), st_ = sin(th);
    double a = 0.3 * R_est, b = 1.7 * R_est;
    const bool pos_a = fase_em(node, n, nx, ny, x0 + a * ct, y0 + a * st_) > 0;
    const int h = lane + 1;             // tree node of this lane (heap order; lane 31 idle)
    const int depth = 31 - __clz(h);
    for (int round = 0; round < 12; round++) {
        double lo = a, hi = b;
        for (int l = depth - 1; l >= 0; l--) {
            const double m = 0.5 * (lo + hi);
            if ((h >> l) & 1) lo = m;
            else hi = m;
        }
        const double mid = 0.5 * (lo + hi);
        bool right = false;
        if (lane < 31) right = (fase_em(node, n, nx, ny, x0 + mid * ct, y0 + mid * st_) > 0) == pos_a;
        const unsigned go_right = __ballot_sync(0xffffffffu, right);
        int v = 1;
        for (int l = 0; l < 5; l++) {
            const double m = __shfl_sync(0xffffffffu, mid, v - 1);
            const int r = (go_right >> (v - 1)) & 1;
            if (r) a = m;
            else b = m;
            v = 2 * v + r;
        }
    }
    if (lane == 0) {
        const double r = 0.5 * (a + b);
        double *__restrict__ rs = J.rays;
        rs[0 * N_ANG + k] = r;
        rs[1 * N_ANG + k] = r * cos(2 * th);
        rs[2 * N_ANG + k] = r * sin(2 * th);
        rs[3 * N_ANG + k] = r * cos(4 * th);
        rs[4 * N_ANG + k] = r * sin(4 * th);
        rs[5 * N_ANG + k] = r * cos(8 * th);
        rs[6 * N_ANG + k] = r * sin(8 * th);
    }
}

// The harmonic sums over the rays in ray order, as the reference loop accumulates them (one block
// per job).
__global__ void __launch_bounds__(ITLBM_N_ANG) k_drop_modes_sum(const DiagJob *__restrict__ jobs,
                                                                const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x] : one;
    if (!((const DropState *)J.state)->proceed) return;
    itlbm_drop_diag *__restrict__ d = (itlbm_drop_diag *)J.out;
    const int N_ANG = ITLBM_N_ANG;
    __shared__ double rs[7][ITLBM_N_ANG];
    const int k = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 7; q++) rs[q][k] = J.rays[q * N_ANG + k];
    __syncthreads();
    if (k == 0) {
        double c2 = 0, s2 = 0, c4 = 0, s4 = 0, c8 = 0, s8 = 0, soma = 0, rmin = 1e30, rmax = 0;
        for (int j = 0; j < N_ANG; j++) {
            const double rr = rs[0][j];
            soma += rr;
            c2 += rs[1][j];
            s2 += rs[2][j];
            c4 += rs[3][j];
            s4 += rs[4][j];
            c8 += rs[5][j];
            s8 += rs[6][j];
            rmin = fmin(rmin, rr);
            rmax = fmax(rmax, rr);
        }
        d->R0 = soma / N_ANG;
        d->a2 = 2.0 * sqrt(c2 * c2 + s2 * s2) / N_ANG / d->R0;
        d->a4 = 2.0 * sqrt(c4 * c4 + s4 * s4) / N_ANG / d->R0;
        d->a8 = 2.0 * sqrt(c8 * c8 + s8 * s8) / N_ANG / d->R0;
        d->rmin = rmin;
        d->rmax = rmax;
    }
}

// Clears what a drop diagnostic accumulates into: its output and its shell histogram (one block per
// job).
__global__ void __launch_bounds__(DT) k_drop_clear(const DiagJob *__restrict__ jobs,
                                                   const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x] : one;
    unsigned *o = (unsigned *)J.out;
    for (int w = threadIdx.x; w < (int)(sizeof(itlbm_drop_diag) / 4); w += DT) o[w] = 0u;
    for (int w = threadIdx.x; w < 2 * J.nshell; w += DT) J.shell[w] = 0ull;
}

// ---------------------------------------------------------------------------------------------
// inclined strip: mede_inclinada (Imm_INCL.cpp:85-189)
// ---------------------------------------------------------------------------------------------
enum {
    S_SIGPOP, S_INTGRAD, S_MASSR, S_MASSB, S_QX, S_QY, S_SFX, S_SFY, S_U2, S_SX, S_SY, S_SXX, S_SXY,
    S_NFIT, S_RUIM, S_NEGT, S_NEGC,  // sums (17)
    S_UMAX, S_UNMAX, S_UTMAX,        // maxima (3)
    S_MINF,                          // minimum (1)
    S_Q
};
constexpr int S_NS = 17, S_NM = 3;

struct StripState {
    double a[S_Q];
    double K, a0;
    int fit;
    double res[1];
};

__device__ __forceinline__ double dist_central(int x, int y, int p, int q, int N) {
    const double m = sqrt((double)(p * p + q * q));
    long long s = ((long long)p * x + (long long)q * y) % N;
    if (s < 0) s += N;
    double d = ((double)s - 0.5 * N);
    if (d >= 0.5 * N) d -= N;
    if (d < -0.5 * N) d += N;
    return -d / m;
}

__global__ void __launch_bounds__(DT) k_strip_s1(const DiagJob *__restrict__ jobs,
                                                 const int *__restrict__ blk_job,
                                                 const __grid_constant__ DiagJob one) {
    int lb;
    const DiagJob &J = block_job(jobs, blk_job, one, lb);
    const CaseDev &c = *J.c;
    const int cur = J.cur, p = J.p, q = J.q, use_force = J.use_force, nb = J.nblocks;
    const int N = c.nx;
    const long long n = (long long)N * N;
    const double m = sqrt((double)(p * p + q * q));
    const double nx_ = p / m, ny_ = q / m, tx_ = -ny_, ty_ = nx_;
    double v[S_Q];
    init_acc<S_Q, S_NS, S_NM>(v);
    for (long long t = lb * (long long)DT + threadIdx.x; t < n; t += (long long)nb * DT) {
        const int x = (int)(t % N), y = (int)(t / N);
        double fR[NV], fB[NV];
        post_pops(c, cur, x, y, fR, fB);
        double rR = 0, rB = 0, jx = 0, jy = 0, Pxx = 0, Pyy = 0, Pxy = 0, Pzz = 0;
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const double f = fR[i] + fB[i];
            if (!finite_d(fR[i]) || !finite_d(fB[i])) v[S_RUIM] += 1.0;
            if (f < -1e-12) v[S_NEGT] += 1.0;
            if (fR[i] < -1e-12) v[S_NEGC] += 1.0;
            if (fB[i] < -1e-12) v[S_NEGC] += 1.0;
            v[S_MINF] = (f < v[S_MINF]) ? f : v[S_MINF];
            rR += fR[i];
            rB += fB[i];
            if constexpr (cx(i) == 1) jx += f;
            if constexpr (cx(i) == -1) jx -= f;
            if constexpr (cy(i) == 1) jy += f;
            if constexpr (cy(i) == -1) jy -= f;
            if constexpr (cx(i) != 0) Pxx += f;
            if constexpr (cy(i) != 0) Pyy += f;
            if constexpr (cx(i) * cy(i) == 1) Pxy += f;
            if constexpr (cx(i) * cy(i) == -1) Pxy -= f;
            if constexpr (cz(i) != 0) Pzz += f;
        });
        const double rho = rR + rB;
        if (!(rho > 0)) {
            v[S_RUIM] += 1.0;
            continue;
        }
        const long long o = aux_off(c, x, y);
        if (use_force) {
            const double F0 = c.aux[o], F1 = c.aux[c.aux_stride + o];
            jx -= 0.5 * F0;
            jy -= 0.5 * F1;
            v[S_SFX] += F0;
            v[S_SFY] += F1;
        }
        const double ux = jx / rho, uy = jy / rho;
        v[S_MASSR] += rR;
        v[S_MASSB] += rB;
        v[S_QX] += jx;
        v[S_QY] += jy;
        const double u = hypot(ux, uy), un = fabs(ux * nx_ + uy * ny_), ut = fabs(ux * tx_ + uy * ty_);
        v[S_UMAX] = (v[S_UMAX] < u) ? u : v[S_UMAX];
        v[S_UNMAX] = (v[S_UNMAX] < un) ? un : v[S_UNMAX];
        v[S_UTMAX] = (v[S_UTMAX] < ut) ? ut : v[S_UTMAX];
        v[S_U2] += u * u;
        const double Pnn = nx_ * nx_ * Pxx + 2 * nx_ * ny_ * Pxy + ny_ * ny_ * Pyy;
        const double Ptt = tx_ * tx_ * Pxx + 2 * tx_ * ty_ * Pxy + ty_ * ty_ * Pyy;
        v[S_SIGPOP] += Pnn - 0.5 * (Ptt + Pzz);
        v[S_INTGRAD] += c.aux[3 * c.aux_stride + o];
        const double dd = dist_central(x, y, p, q, N);
        const double cR = rR / rho;
        if (cR > 0.02 && cR < 0.98 && fabs(dd) < 8.0) {
            const double l = log(cR / (1.0 - cR));
            v[S_SX] += dd;
            v[S_SY] += l;
            v[S_SXX] += dd * dd;
            v[S_SXY] += dd * l;
            v[S_NFIT] += 1.0;
        }
    }
    block_reduce<S_Q, S_NS, S_NM>(v, J.part + (long long)lb * S_Q);
}

__global__ void k_strip_f1(const DiagJob *__restrict__ jobs, int njobs, const __grid_constant__ DiagJob one) {
    const int jid = blockIdx.x * blockDim.x + threadIdx.x;
    if (jid >= njobs) return;
    const DiagJob &J = jobs ? jobs[jid] : one;
    StripState *__restrict__ st = (StripState *)J.state;
    itlbm_strip_diag *__restrict__ r = (itlbm_strip_diag *)J.out;
    const int p = J.p, q = J.q;
    const int N = J.c->nx;
    const double *a = st->a;
    const double m = sqrt((double)(p * p + q * q));
    const double comprimento = 2.0 * N * m;
    r->sigma_pop = a[S_SIGPOP] / comprimento;
    r->int_grad = a[S_INTGRAD] / comprimento;
    r->massa_R = a[S_MASSR];
    r->massa_B = a[S_MASSB];
    r->qx = a[S_QX];
    r->qy = a[S_QY];
    r->SFx = a[S_SFX];
    r->SFy = a[S_SFY];
    r->u_max = a[S_UMAX] < 0 ? 0.0 : a[S_UMAX];
    r->un_max = a[S_UNMAX] < 0 ? 0.0 : a[S_UNMAX];
    r->ut_max = a[S_UTMAX] < 0 ? 0.0 : a[S_UTMAX];
    r->min_f = a[S_MINF] == DBL_MAX ? 1e300 : a[S_MINF];
    r->neg_total = (long long)a[S_NEGT];
    r->neg_cor = (long long)a[S_NEGC];
    r->n_ruim = (int)a[S_RUIM];
    r->u_rms = sqrt(a[S_U2] / (N * N));
    const int nfit = (int)a[S_NFIT];
    r->n_ajuste = nfit;
    st->fit = 0;
    r->K = 0;
    r->d0 = 0;
    r->res = 0;
    if (nfit > 3) {
        const double Sx = a[S_SX], Sy = a[S_SY], Sxx = a[S_SXX], Sxy = a[S_SXY];
        const double K = (nfit * Sxy - Sx * Sy) / (nfit * Sxx - Sx * Sx);
        const double a0 = (Sy - K * Sx) / nfit;
        r->K = K;
        r->d0 = -a0 / K;
        st->K = K;
        st->a0 = a0;
        st->fit = 1;
    }
    r->ok = (r->n_ruim == 0 && isfinite(r->u_max));
}

__global__ void __launch_bounds__(DT) k_strip_s2(const DiagJob *__restrict__ jobs,
                                                 const int *__restrict__ blk_job,
                                                 const __grid_constant__ DiagJob one) {
    int lb;
    const DiagJob &J = block_job(jobs, blk_job, one, lb);
    const StripState *__restrict__ st = (const StripState *)J.state;
    const int cur = J.cur, p = J.p, q = J.q, nb = J.nblocks;
    double m[1] = {0.0};
    if (st->fit) {
        const CaseDev &c = *J.c;
        const int N = c.nx;
        const long long n = (long long)N * N;
        const double K = st->K, a0 = st->a0;
        for (long long t = lb * (long long)DT + threadIdx.x; t < n; t += (long long)nb * DT) {
            const int x = (int)(t % N), y = (int)(t / N);
            double fR[NV], fB[NV];
            post_pops(c, cur, x, y, fR, fB);
            double rR = 0, rB = 0;
            for (int i = 0; i < NV; i++) {
                rR += fR[i];
                rB += fB[i];
            }
            const double rho = rR + rB;
            if (!(rho > 0)) continue;
            const double dd = dist_central(x, y, p, q, N);
            const double cR = rR / rho;
            if (cR > 0.02 && cR < 0.98 && fabs(dd) < 8.0) {
                const double e = fabs(log(cR / (1.0 - cR)) - (a0 + K * dd));
                if (e > m[0]) m[0] = e;
            }
        }
    }
    block_reduce<1, 0, 1>(m, J.part + lb);
}

__global__ void k_strip_f2(const DiagJob *__restrict__ jobs, int njobs, const __grid_constant__ DiagJob one) {
    const int jid = blockIdx.x * blockDim.x + threadIdx.x;
    if (jid >= njobs) return;
    const DiagJob &J = jobs ? jobs[jid] : one;
    const StripState *__restrict__ st = (const StripState *)J.state;
    itlbm_strip_diag *__restrict__ r = (itlbm_strip_diag *)J.out;
    if (st->fit) r->res = st->res[0] < 0 ? 0.0 : st->res[0];
}

__global__ void __launch_bounds__(DT) k_strip_clear(const DiagJob *__restrict__ jobs,
                                                    const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x] : one;
    unsigned *o = (unsigned *)J.out;
    for (int w = threadIdx.x; w < (int)(sizeof(itlbm_strip_diag) / 4); w += DT) o[w] = 0u;
}

// The block reductions of the partials, one block per job, into the job's running state.
enum { R_DROP_A, R_DROP_B, R_STRIP_A, R_STRIP_RES };
template <int Q, int NS, int NM, int W>
__global__ void __launch_bounds__(DT) k_reduce_jobs(const DiagJob *__restrict__ jobs,
                                                    const __grid_constant__ DiagJob one) {
    const DiagJob &J = jobs ? jobs[blockIdx.x] : one;
    double *res;
    if constexpr (W == R_DROP_A) res = ((DropState *)J.state)->a;
    else if constexpr (W == R_DROP_B) res = ((DropState *)J.state)->b;
    else if constexpr (W == R_STRIP_A) res = ((StripState *)J.state)->a;
    else res = ((StripState *)J.state)->res;
    reduce_rows<Q, NS, NM>(J.part, J.nblocks, res);
}

// Per-node output fields of the post-collision state, each value formed with the reference's
// operations in its order and rounded as written (the __d*_rn intrinsics keep the compiler from
// contracting a product and a sum into one FMA, which would round differently):
//   rho_R, rho_B   density() of each colour, index order (LBM_functions.cpp:1582-1590);
//   FIELDS_VTK     rec_velocity's two-colour branch (LBM_functions.cpp:1349-1458): u_C = m_C * (1 / rho_C)
//                  by calcula (:1100-1171) for each colour, u = c_R u_R + c_B u_B with c_B = 1 - c_R,
//                  then u -= (0.5 F) / rho for a case with a force (rho > 0);
//   FIELDS_PROFILE perfil.dat of mede_inclinada (Imm_INCL.cpp:104-162): u = (sum_i f_i c_i - 0.5 F) / rho
//                  with f_i = f_R,i + f_B,i; a node with !(rho > 0) is skipped there and gets NaN here.
// Sums of +-f over the non-zero components of c_i equal the reference's sums of c_i * f (the zero
// terms add a signed zero, which changes no finite partial sum).
__global__ void k_fields(const CaseDev *__restrict__ cp, int cur, int use_force, int form,
                         double *rR_out, double *rB_out, double *ux_out, double *uy_out,
                         double *uz_out) {
    const CaseDev &c = *cp;
    const int nx = c.nx;
    const long long n = (long long)nx * c.ny;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
         p += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(p % nx), y = (int)(p / nx);
        double fR[NV], fB[NV];
        post_pops(c, cur, x, y, fR, fB);
        double rr = 0.0, rb = 0.0;
#pragma unroll
        for (int i = 0; i < NV; i++) rr = __dadd_rn(rr, fR[i]);
#pragma unroll
        for (int i = 0; i < NV; i++) rb = __dadd_rn(rb, fB[i]);
        const long long o = aux_off(c, x, y);
        double vx, vy, vz;
        if (form == ITLBM_FIELDS_VTK) {
            double m[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
            sfor<0, NV>([&](auto I) {
                constexpr int i = decltype(I)::value;
                if constexpr (cx(i) != 0) {
                    m[0][0] = __dadd_rn(m[0][0], cx(i) > 0 ? fR[i] : -fR[i]);
                    m[1][0] = __dadd_rn(m[1][0], cx(i) > 0 ? fB[i] : -fB[i]);
                }
                if constexpr (cy(i) != 0) {
                    m[0][1] = __dadd_rn(m[0][1], cy(i) > 0 ? fR[i] : -fR[i]);
                    m[1][1] = __dadd_rn(m[1][1], cy(i) > 0 ? fB[i] : -fB[i]);
                }
                if constexpr (cz(i) != 0) {
                    m[0][2] = __dadd_rn(m[0][2], cz(i) > 0 ? fR[i] : -fR[i]);
                    m[1][2] = __dadd_rn(m[1][2], cz(i) > 0 ? fB[i] : -fB[i]);
                }
            });
            double v[2][3];
            const double rc[2] = {rr, rb};
            for (int k = 0; k < 2; k++) {
                if (rc[k] != 0.0) {
                    const double inv = 1.0 / rc[k];
                    for (int a = 0; a < 3; a++) v[k][a] = __dmul_rn(m[k][a], inv);
                } else {
                    for (int a = 0; a < 3; a++) v[k][a] = 0.0;
                }
            }
            const double concR = rr / __dadd_rn(rr, rb);
            const double concB = __dsub_rn(1.0, concR);
            vx = __dadd_rn(__dmul_rn(concR, v[0][0]), __dmul_rn(concB, v[1][0]));
            vy = __dadd_rn(__dmul_rn(concR, v[0][1]), __dmul_rn(concB, v[1][1]));
            vz = __dadd_rn(__dmul_rn(concR, v[0][2]), __dmul_rn(concB, v[1][2]));
            const double rho = __dadd_rn(rr, rb);
            if (use_force && rho > 0.0) {
                vx = __dsub_rn(vx, __dmul_rn(0.5, c.aux[o]) / rho);
                vy = __dsub_rn(vy, __dmul_rn(0.5, c.aux[c.aux_stride + o]) / rho);
                vz = __dsub_rn(vz, __dmul_rn(0.5, c.aux[2 * c.aux_stride + o]) / rho);
            }
        } else {
            double jx = 0.0, jy = 0.0, jz = 0.0;
            sfor<0, NV>([&](auto I) {
                constexpr int i = decltype(I)::value;
                const double f = __dadd_rn(fR[i], fB[i]);
                if constexpr (cx(i) != 0) jx = __dadd_rn(jx, cx(i) > 0 ? f : -f);
                if constexpr (cy(i) != 0) jy = __dadd_rn(jy, cy(i) > 0 ? f : -f);
                if constexpr (cz(i) != 0) jz = __dadd_rn(jz, cz(i) > 0 ? f : -f);
            });
            const double rho = __dadd_rn(rr, rb);
            if (!(rho > 0)) {
                vx = vy = vz = CUDART_NAN;
            } else {
                if (use_force) {
                    jx = __dsub_rn(jx, __dmul_rn(0.5, c.aux[o]));
                    jy = __dsub_rn(jy, __dmul_rn(0.5, c.aux[c.aux_stride + o]));
                    jz = __dsub_rn(jz, __dmul_rn(0.5, c.aux[2 * c.aux_stride + o]));
                }
                vx = jx / rho;
                vy = jy / rho;
                vz = jz / rho;
            }
        }
        if (rR_out) rR_out[p] = rr;
        if (rB_out) rB_out[p] = rb;
        if (ux_out) ux_out[p] = vx;
        if (uy_out) uy_out[p] = vy;
        if (uz_out) uz_out[p] = vz;
    }
}

int nblocks_for(long long n) {
    long long b = (n + DT - 1) / DT;
    if (b > MAXB) b = MAXB;
    return (int)(b < 1 ? 1 : b);
}

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }
int nshell_for(int nx, int ny) { return (int)(sqrt((double)(nx * nx + ny * ny + 1)) / 0.5) + 2; }
constexpr size_t STATE_BYTES = sizeof(DropState) > sizeof(StripState) ? sizeof(DropState) : sizeof(StripState);
constexpr size_t OUT_BYTES =
    sizeof(itlbm_drop_diag) > sizeof(itlbm_strip_diag) ? sizeof(itlbm_drop_diag) : sizeof(itlbm_strip_diag);
constexpr int PART_COLS = 32;  // >= the quantities of any pass
static_assert(A_Q <= PART_COLS && B_Q <= PART_COLS && S_Q <= PART_COLS, "partial rows");

cudaError_t run_drop(const DiagJob *jobs, int njobs, const int *blk_job, int total_blocks, const DiagJob &one,
                     cudaStream_t st) {
    const int g32 = (njobs + 31) / 32;
    k_drop_clear<<<njobs, DT, 0, st>>>(jobs, one);
    k_drop_d1<<<total_blocks, DT, 0, st>>>(jobs, blk_job, one);
    k_reduce_jobs<A_Q, A_NS, A_NM, R_DROP_A><<<njobs, DT, 0, st>>>(jobs, one);
    k_drop_f1<<<g32, 32, 0, st>>>(jobs, njobs, one);
    k_drop_d2<<<total_blocks, DT, 0, st>>>(jobs, blk_job, one);
    k_reduce_jobs<B_Q, B_NS, B_NM, R_DROP_B><<<njobs, DT, 0, st>>>(jobs, one);
    k_drop_f2<<<g32, 32, 0, st>>>(jobs, njobs, one);
    k_drop_fit<<<njobs, DT, 0, st>>>(jobs, one);
    k_drop_modes<<<njobs * MODE_BLOCKS, DT, 0, st>>>(jobs, one);
    k_drop_modes_sum<<<njobs, ITLBM_N_ANG, 0, st>>>(jobs, one);
    return cudaGetLastError();
}

cudaError_t run_strip(const DiagJob *jobs, int njobs, const int *blk_job, int total_blocks, const DiagJob &one,
                      cudaStream_t st) {
    const int g32 = (njobs + 31) / 32;
    k_strip_clear<<<njobs, DT, 0, st>>>(jobs, one);
    k_strip_s1<<<total_blocks, DT, 0, st>>>(jobs, blk_job, one);
    k_reduce_jobs<S_Q, S_NS, S_NM, R_STRIP_A><<<njobs, DT, 0, st>>>(jobs, one);
    k_strip_f1<<<g32, 32, 0, st>>>(jobs, njobs, one);
    k_strip_s2<<<total_blocks, DT, 0, st>>>(jobs, blk_job, one);
    k_reduce_jobs<1, 0, 1, R_STRIP_RES><<<njobs, DT, 0, st>>>(jobs, one);
    k_strip_f2<<<g32, 32, 0, st>>>(jobs, njobs, one);
    return cudaGetLastError();
}

}  // namespace

int diag_nblocks(long long n) { return nblocks_for(n); }

size_t diag_job_bytes(int nx, int ny, int geometry) {
    const size_t n = (size_t)nx * ny;
    size_t b = up256(STATE_BYTES) + up256(OUT_BYTES) + up256(sizeof(double) * PART_COLS * nblocks_for((long long)n));
    if (geometry == ITLBM_GEOM_DROP)
        b += up256(sizeof(double) * 6 * n) + up256(sizeof(unsigned long long) * 2 * (size_t)nshell_for(nx, ny)) +
             up256(sizeof(double) * 7 * ITLBM_N_ANG);
    return b;
}

void diag_job_layout(DiagJob &j, void *base, int nx, int ny, int geometry) {
    const size_t n = (size_t)nx * ny;
    char *p = (char *)base;
    j.n = (int)n;
    j.nblocks = nblocks_for((long long)n);
    j.nshell = geometry == ITLBM_GEOM_DROP ? nshell_for(nx, ny) : 0;
    j.state = p;
    p += up256(STATE_BYTES);
    j.out = p;
    p += up256(OUT_BYTES);
    j.part = (double *)p;
    p += up256(sizeof(double) * PART_COLS * j.nblocks);
    j.node = nullptr;
    j.shell = nullptr;
    j.rays = nullptr;
    if (geometry == ITLBM_GEOM_DROP) {
        j.node = (double *)p;
        p += up256(sizeof(double) * 6 * n);
        j.shell = (unsigned long long *)p;
        p += up256(sizeof(unsigned long long) * 2 * (size_t)j.nshell);
        j.rays = (double *)p;
    }
    j.block0 = 0;
}

cudaError_t launch_diag_jobs(const DiagJob *jobs_dev, int njobs, const int *blk_job, int total_blocks,
                             int geometry, cudaStream_t st) {
    if (njobs <= 0) return cudaSuccess;
    const DiagJob none{};
    return geometry == ITLBM_GEOM_DROP ? run_drop(jobs_dev, njobs, blk_job, total_blocks, none, st)
                                       : run_strip(jobs_dev, njobs, blk_job, total_blocks, none, st);
}

size_t diag_bytes(int nx, int ny) { return diag_job_bytes(nx, ny, ITLBM_GEOM_DROP); }

void *diag_scratch_out(const DiagScratch &s) { return s.base ? (char *)s.base + up256(STATE_BYTES) : nullptr; }

cudaError_t diag_alloc(DiagScratch &s, int nx, int ny) {
    const size_t need = diag_bytes(nx, ny);
    if (s.base && s.bytes >= need) return cudaSuccess;
    diag_free(s);
    void *p = nullptr;
    const cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) return e;  // s stays empty: the next call tries again
    s.base = p;
    s.bytes = need;
    s.owned = true;
    return cudaSuccess;
}

cudaError_t diag_bind(DiagScratch &s, void *base, size_t bytes, int nx, int ny) {
    if (!base || ((uintptr_t)base & 255) || diag_bytes(nx, ny) > bytes) return cudaErrorInvalidValue;
    s.base = base;
    s.bytes = bytes;
    s.owned = false;
    return cudaSuccess;
}

void diag_free(DiagScratch &s) {
    if (s.owned && s.base) cudaFree(s.base);
    s = DiagScratch();
}

cudaError_t launch_diag_drop(const CaseDev *c_dev, const CaseDev &c, DiagScratch &s, int cur,
                             int step, double v0, double x_ini, double y_ini, bool use_force,
                             itlbm_drop_diag *out_dev, cudaStream_t st) {
    if (!s.base || s.bytes < diag_bytes(c.nx, c.ny)) return cudaErrorInvalidValue;
    DiagJob j{};
    diag_job_layout(j, s.base, c.nx, c.ny, ITLBM_GEOM_DROP);
    j.c = c_dev;
    if (out_dev) j.out = out_dev;
    j.cur = cur;
    j.step = step;
    j.v0 = v0;
    j.x_ini = x_ini;
    j.y_ini = y_ini;
    j.use_force = use_force ? 1 : 0;
    return run_drop(nullptr, 1, nullptr, j.nblocks, j, st);
}

cudaError_t launch_diag_strip(const CaseDev *c_dev, const CaseDev &c, DiagScratch &s, int cur,
                              int step, int p, int q, bool use_force, itlbm_strip_diag *out_dev,
                              cudaStream_t st) {
    if (!s.base || s.bytes < diag_job_bytes(c.nx, c.ny, ITLBM_GEOM_STRIP)) return cudaErrorInvalidValue;
    DiagJob j{};
    diag_job_layout(j, s.base, c.nx, c.ny, ITLBM_GEOM_STRIP);
    j.c = c_dev;
    if (out_dev) j.out = out_dev;
    j.cur = cur;
    j.step = step;
    j.p = p;
    j.q = q;
    j.use_force = use_force ? 1 : 0;
    return run_strip(nullptr, 1, nullptr, j.nblocks, j, st);
}

cudaError_t launch_fields(const CaseDev *c_dev, const CaseDev &c, int cur, bool use_force, int form,
                          double *rho_R, double *rho_B, double *ux, double *uy, double *uz,
                          cudaStream_t st) {
    const long long n = (long long)c.nx * c.ny;
    k_fields<<<nblocks_for(n), DT, 0, st>>>(c_dev, cur, use_force ? 1 : 0, form, rho_R, rho_B, ux, uy, uz);
    return cudaGetLastError();
}

}  // namespace itlbm
