// itlbm_seam.cu -- per-site kernels of the operator seam (compiled with --fmad=false): the reference's
// perturbacao, source and colisao_comum applied to independent sites, through the same device
// functions the fused step uses.
#include "itlbm_site.cuh"

namespace itlbm {

__global__ void k_perturb(int n, double A, double B0, double B1, double B2, const double *g, double *f) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double v[NV];
    for (int i = 0; i < NV; i++) v[i] = f[(size_t)k * NV + i];
    perturb_f64(v, g[3 * k], g[3 * k + 1], g[3 * k + 2], A, B0, B1, B2);
    for (int i = 0; i < NV; i++) f[(size_t)k * NV + i] = v[i];
}

__global__ void k_source(int n, const double *F, const double *u, double factor, double *S) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double Fx = F[3 * k], Fy = F[3 * k + 1], Fz = F[3 * k + 2];
    const double vx = u[3 * k], vy = u[3 * k + 1], vz = u[3 * k + 2];
    const double vF = Fx * vx + Fy * vy + Fz * vz;
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const double cv = cdot<i>(vx, vy, vz);
        S[(size_t)k * NV + i] = guo_source_f64<i>(factor, Fx, Fy, Fz, cv, vF);
    });
}

template <bool FORCE>
__global__ void k_colisao(int n, CaseDev c, double *fR, double *fB, const double *gm, const double *F) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double a[NV], b[NV];
    for (int i = 0; i < NV; i++) {
        a[i] = fR[(size_t)k * NV + i];
        b[i] = fB[(size_t)k * NV + i];
    }
    const double F0 = FORCE ? F[3 * k] : 0.0, F1 = FORCE ? F[3 * k + 1] : 0.0, F2 = FORCE ? F[3 * k + 2] : 0.0;
    colisao_site_f64<FORCE>(a, b, gm[3 * k], gm[3 * k + 1], gm[3 * k + 2], F0, F1, F2, c);
    for (int i = 0; i < NV; i++) {
        fR[(size_t)k * NV + i] = a[i];
        fB[(size_t)k * NV + i] = b[i];
    }
}


void seam_perturb(int n, double A, double B0, double B1, double B2, const double *g, double *f) {
    k_perturb<<<(n + 127) / 128, 128>>>(n, A, B0, B1, B2, g, f);
}
void seam_source(int n, const double *F, const double *u, double factor, double *S) {
    k_source<<<(n + 127) / 128, 128>>>(n, F, u, factor, S);
}
void seam_colisao(int n, const CaseDev &c, bool force, double *fR, double *fB, const double *gm,
                  const double *F) {
    if (force) k_colisao<true><<<(n + 127) / 128, 128>>>(n, c, fR, fB, gm, F);
    else k_colisao<false><<<(n + 127) / 128, 128>>>(n, c, fR, fB, gm, F);
}

}  // namespace itlbm

