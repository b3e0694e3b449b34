// itlbm_state.cu -- initial state and population export / import (compiled with --fmad=false).
//
// The initial profile rho^N(r) of a drop (or c_R(s) of a strip) contains exp(); it is evaluated on
// the host with the same expression as the reference and uploaded, and this kernel finishes the
// seeding with dist_eq in the reference's operation order, so the FP64 initial state is bit-identical
// to the reference's.
#include "itlbm_site.cuh"

#include <algorithm>
#include <cmath>
#include <functional>
#include <thread>
#include <vector>

namespace itlbm {

namespace {

__device__ __forceinline__ int wrapi(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

__device__ void store_state(const CaseDev &c, int buf, long long off, const double *fR,
                            const double *fB) {
    if (c.prec == ITLBM_PREC_F64) {
        double *d = (double *)c.buf[buf];
        for (int i = 0; i < NV; i++) {
            d[off + i * PLANE] = fR[i];
            d[off + (NV + i) * PLANE] = fB[i];
        }
    } else if (c.prec == ITLBM_PREC_F32) {
        float *d = (float *)c.buf[buf];
        for (int i = 0; i < NV; i++) {
            d[off + i * PLANE] = (float)((fR[i] + fB[i]) - (double)c.sh[i]);
            d[off + (NV + i) * PLANE] = (float)(fR[i] - fB[i]);
        }
    } else {  // fold: class sums of the members (FP64), then shifted and rounded
        float *d = (float *)c.buf[buf];
        double F[NK] = {}, Dk[NK] = {};
        for (int i = 0; i < NV; i++) {
            F[fold_class(i)] += fR[i] + fB[i];
            Dk[fold_class(i)] += fR[i] - fB[i];
        }
        for (int K = 0; K < NK; K++) {
            d[off + K * PLANE] = (float)(F[K] - (double)c.shk[K]);
            d[off + (NK + K) * PLANE] = (float)Dk[K];
        }
    }
}

// The 19 populations of a node of the fold: each class split among its members by weight (exact
// for the class sums and every moment; a member's own share is that of the split).
__device__ __forceinline__ void unfold_split(double E, double D, int K, int i, double sK, double &fR, double &fB) {
    const double share = wgt<double>(i) / wk<double>(K);
    const double f = (sK + E) * share, d = D * share;
    fR = 0.5 * (f + d);
    fB = 0.5 * (f - d);
}

// dist_eq (LBM_functions.cpp:890-945) of one colour
__device__ void dist_eq_dev(double *feq, double vx, double vy, double vz, double rho) {
    const double vquad = (vx * vx + vy * vy + vz * vz);
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const double cv = cdot<i>(vx, vy, vz);
        feq[i] = wgt<double>(i) * rho *
                 (1.0 + cv * 3.0 + 0.5 * cv * cv * 3.0 * 3.0 - 0.5 * vquad * 3.0);
    });
}

// initial_conditions_drop (Initial_conditions.cpp:37-169) as called at Imm_OPS.cpp:199-202, given
// phi(x) from the host: rho_tot = rho_B + phi (rho_R - rho_B) + phi * delta_rho (delta_rho = 0),
// f_R = dist_eq(v0, phi rho_tot), f_B = dist_eq(v0, (1 - phi) rho_tot).
// The logistic strip of Imm_INCL.cpp:309-334, given c_R(s) for s = (p x + q y) mod N:
// f_R = w_i c_R, f_B = w_i (1 - c_R).
// With prof == nullptr (FP32 storage forms only) the drop's profile is evaluated here with the
// device's sqrt and exp: within an ulp or two of the host's libm in FP64, and rounded to FP32 anyway.
__global__ void k_init(const CaseDev *__restrict__ cp, int geometry, const double *__restrict__ prof,
                       double v0, double rho_Ri, double rho_Bi, int p, int q, double radius, double k_perfil) {
    const CaseDev &c = *cp;
    const long long n = (long long)c.nx * c.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % c.nx), y = (int)(t / c.nx);
        double fR[NV], fB[NV];
        if (geometry == ITLBM_GEOM_DROP) {
            double phi;
            if (prof) {
                phi = prof[t];
            } else {  // the expressions of init_profile_rows
                const double dx = (double)(x - c.nx / 2), dy = (double)(y - c.ny / 2), dz = 0.0;
                const double r = sqrt(dx * dx + dy * dy + dz * dz);
                if (k_perfil > 0.0) {
                    double arg = k_perfil * (r - radius);
                    if (arg > 60.0) arg = 60.0;
                    if (arg < -60.0) arg = -60.0;
                    phi = 1.0 / (1.0 + exp(arg));
                } else {
                    phi = (r < radius) ? 1.0 : 0.0;
                }
            }
            const double rho_tot = rho_Bi + phi * (rho_Ri - rho_Bi) + phi * 0.0;
            dist_eq_dev(fR, v0, 0., 0., phi * rho_tot);
            dist_eq_dev(fB, v0, 0., 0., (1.0 - phi) * rho_tot);
        } else {
            const int N = c.nx;
            long long s = ((long long)p * x + (long long)q * y) % N;
            if (s < 0) s += N;
            const double cR = prof[s];
            for (int i = 0; i < NV; i++) {
                fR[i] = wgt<double>(i) * cR;
                fB[i] = wgt<double>(i) * (1.0 - cR);
            }
        }
        store_state(c, c.parity0, node_off(c, x, y), fR, fB);
    }
}

// FP64 AoS export (reference layout f[pto*19+i]); which = 1 gathers the post-collision values of
// the last step, dst(x + c_i, i).
__global__ void k_export(const CaseDev *__restrict__ cp, int cur, int which, double *__restrict__ oR,
                         double *__restrict__ oB) {
    const CaseDev &c = *cp;
    const long long n = (long long)c.nx * c.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % c.nx), y = (int)(t / c.nx);
        for (int i = 0; i < NV; i++) {
            int xs = x, ys = y;
            if (which) {
                xs = wrapi(x + cx(i), c.nx);
                ys = wrapi(y + cy(i), c.ny);
            }
            double r, b;
            if (c.prec == ITLBM_PREC_F32_FOLD) {
                const int K = fold_class(i);
                if (which) {  // the class was pushed to x + e_K
                    xs = wrapi(x + kx(K), c.nx);
                    ys = wrapi(y + ky(K), c.ny);
                }
                const long long off = node_off(c, xs, ys);
                const float *d = (const float *)c.buf[cur];
                unfold_split(d[off + K * PLANE], d[off + (NK + K) * PLANE], K, i,
                             (double)c.shk[K], r, b);
                oR[t * NV + i] = r;
                oB[t * NV + i] = b;
                continue;
            }
            const long long off = node_off(c, xs, ys);
            if (c.prec == ITLBM_PREC_F64) {
                const double *d = (const double *)c.buf[cur];
                r = d[off + i * PLANE];
                b = d[off + (NV + i) * PLANE];
            } else {
                const float *d = (const float *)c.buf[cur];
                const double e = d[off + i * PLANE];
                const double dd = d[off + (NV + i) * PLANE];
                const double f = (double)c.sh[i] + e;
                r = 0.5 * (f + dd);
                b = 0.5 * (f - dd);
            }
            oR[t * NV + i] = r;
            oB[t * NV + i] = b;
        }
    }
}

__global__ void k_import(const CaseDev *__restrict__ cp, int cur, const double *__restrict__ iR,
                         const double *__restrict__ iB) {
    const CaseDev &c = *cp;
    const long long n = (long long)c.nx * c.ny;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % c.nx), y = (int)(t / c.nx);
        store_state(c, cur, node_off(c, x, y), iR + t * NV, iB + t * NV);
    }
}

int grid_for(long long n, int threads) {
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 32) g = 148LL * 32;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

// Length of the initial profile of a case: one value per node for a drop, one per distance class
// for a strip.
size_t profile_len(const CaseDev &c, const itlbm_case_desc &d) {
    return d.geometry == ITLBM_GEOM_DROP ? (size_t)c.nx * c.ny : (size_t)c.nx;
}

// Host side of the initial profile: the expressions of Initial_conditions.cpp:66-86 (drop) and
// Imm_INCL.cpp:310-324 (strip), evaluated with the host's libm like the reference does.  A drop's
// profile is filled for rows [ya, yb); a strip's (one value per distance class) whole, for any range.
void init_profile_rows(const CaseDev &c, const itlbm_case_desc &d, double *prof, int ya, int yb) {
    if (d.geometry == ITLBM_GEOM_DROP) {
        const double radius = d.radius > 0.0 ? d.radius : 0.25 * (double)d.nx;
        const double k_perfil = d.k_profile;
        const int x0 = c.nx / 2, y0 = c.ny / 2;
        for (int y = ya; y < yb; y++)
            for (int x = 0; x < c.nx; x++) {
                const double dx = (double)(x - x0), dy = (double)(y - y0), dz = 0.0;
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                double phi;
                if (k_perfil > 0.0) {
                    double arg = k_perfil * (r - radius);
                    if (arg > 60.0) arg = 60.0;
                    if (arg < -60.0) arg = -60.0;
                    phi = 1.0 / (1.0 + std::exp(arg));
                } else {
                    phi = (r < radius) ? 1.0 : 0.0;
                }
                prof[(size_t)y * c.nx + x] = phi;
            }
    } else {
        const int N = c.nx, p = d.p, q = d.q;
        const double m = std::sqrt((double)(p * p + q * q));
        const double k = 2.0 * std::log(9.0) / 3.45;
        for (long long s2 = 0; s2 < N; s2++) {
            const double dred = (2 * s2 < N) ? std::min((double)s2, 0.5 * N - s2) / m
                                             : -std::min(s2 - 0.5 * N, (double)(N - s2)) / m;
            prof[s2] = 1.0 / (1.0 + std::exp(-k * dred));
        }
    }
}

// The whole profile; a large drop's rows are split over host threads (every node is independent).
void init_profile(const CaseDev &c, const itlbm_case_desc &d, double *prof) {
    const long long n = (long long)c.nx * c.ny;
    const int nthr = (d.geometry != ITLBM_GEOM_DROP || n < (1 << 16))
                         ? 1
                         : (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
    if (nthr == 1) {
        init_profile_rows(c, d, prof, 0, c.ny);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; t++)
        pool.emplace_back(init_profile_rows, std::cref(c), std::cref(d), prof, (int)((long long)c.ny * t / nthr),
                          (int)((long long)c.ny * (t + 1) / nthr));
    for (auto &th : pool) th.join();
}

// Whether a case's initial profile is evaluated on the device: drops in the FP32 storage forms (an FP64
// state must be the reference's to the bit, and takes its profile from the host's libm).
bool profile_on_device(const itlbm_case_desc &d) {
    return d.geometry == ITLBM_GEOM_DROP && d.precision != ITLBM_PREC_F64;
}

// The initial state from a profile already in memory the device can read (device memory, or
// mapped pinned host memory, which the kernel reads across the host link once per value), or, with
// prof == nullptr for a case with profile_on_device, from the profile evaluated by the kernel.
cudaError_t launch_init_from(const CaseDev &c, const CaseDev *c_dev, const itlbm_case_desc &d,
                             const double *prof, cudaStream_t s) {
    const long long n = (long long)c.nx * c.ny;
    const double radius = d.radius > 0.0 ? d.radius : 0.25 * (double)d.nx;
    k_init<<<grid_for(n, 256), 256, 0, s>>>(c_dev, d.geometry, prof, d.v0, d.rho_R, d.rho_B, d.p, d.q, radius,
                                            d.k_profile);
    return cudaGetLastError();
}

// Single cases: the profile is staged through device memory (or evaluated by the kernel) and the call
// waits for the state.
cudaError_t launch_init(const CaseDev &c, const CaseDev *c_dev, const itlbm_case_desc &d,
                        cudaStream_t s) {
    if (profile_on_device(d)) {
        const cudaError_t e = launch_init_from(c, c_dev, d, nullptr, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    }
    std::vector<double> prof(profile_len(c, d));
    init_profile(c, d, prof.data());
    double *dprof = nullptr;
    cudaError_t e = cudaMalloc(&dprof, sizeof(double) * prof.size());
    if (e != cudaSuccess) return e;
    // on the launch stream: a pageable copy may return before its data has reached the device, and
    // a non-blocking stream is not ordered after the legacy stream
    e = cudaMemcpyAsync(dprof, prof.data(), sizeof(double) * prof.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_init_from(c, c_dev, d, dprof, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(dprof);
    return e;
}

cudaError_t launch_export(const CaseDev *c_dev, int nx, int ny, int cur, int which, double *fR,
                          double *fB, cudaStream_t s) {
    k_export<<<grid_for((long long)nx * ny, 256), 256, 0, s>>>(c_dev, cur, which, fR, fB);
    return cudaGetLastError();
}

cudaError_t launch_import(const CaseDev *c_dev, int nx, int ny, int cur, const double *fR,
                          const double *fB, cudaStream_t s) {
    k_import<<<grid_for((long long)nx * ny, 256), 256, 0, s>>>(c_dev, cur, fR, fB);
    return cudaGetLastError();
}

}  // namespace itlbm
