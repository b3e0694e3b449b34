// itlbm_step.cu -- the fused time step, the initial state and population export/import.
//
// State layout in HBM (per case, per buffer): tile-major (CaseDev in itlbm_internal.h).  Each 32 x 8
// tile is one contiguous block of 2 colours x 19 directions planes of 256 nodes, so every plane of a
// node is at a compile-time offset (q x 256 elements) from the node's address.
//   FP64 plain:  plane (0, i) = f_R,i and (1, i) = f_B,i
//   FP32 shifted: plane (0, i) = e_i = f_i - w_i rho0 and (1, i) = d_i = f_R,i - f_B,i
// A buffer holds the populations at the top of a step -- the reference's inif_R / inif_B after the
// swap (Imm_OPS.cpp:368-371) -- so initial states need no shift.  The step reads buffer `src`,
// collides every node and pushes each post-collision population to its neighbour x + c_i in buffer
// `dst`, as propag_site does (SimBoltz_Functions/LBM_functions.cpp:1220-1247).  The post-collision
// values the diagnostics need are therefore dst(x + c_i, i).
//
// One CTA of 256 threads handles a tile of 256 nodes (512 in the fold, two rows per thread) of one
// case (the work table says which; its shape -- 32 x 8, or 16 x 16 / 8 x 32 at the edge of a box
// whose width is not a multiple of 32 -- is that of the kernel).  It stages rho^N for the tile plus a
// halo of 1 (P1, P3, F3) or 2 (F1, F2) nodes in shared memory -- the halo nodes are
// re-read from L2, where the neighbouring tiles keep them -- then evaluates the mediator gradient,
// the force of class F on a ring-1 region of auxiliary fields, and collides.  No mediator
// populations or force fields ever reach HBM.
#include "itlbm_site.cuh"

#include <climits>

namespace itlbm {

namespace {

// Global loads and stores of the step, with cache hints chosen by measurement (build-time switches;
// the differences measured on B200 were within 1 %: promotion on the own-node loads is kept, the
// streaming stores cost the FP64 step 3 %):
//   ITLBM_LD_HINT  0: plain read-only loads; 1: L2 256-byte sector promotion on the own-node loads;
//                  2: on the halo-ring loads too
//   ITLBM_ST_HINT  0: plain stores; 1: streaming (evict-first) stores
#ifndef ITLBM_LD_HINT
#define ITLBM_LD_HINT 1
#endif
#ifndef ITLBM_ST_HINT
#define ITLBM_ST_HINT 0
#endif
template <bool PROMOTE>
__device__ __forceinline__ float ldg(const float *p) {
    if constexpr (PROMOTE) {
        float v;
        asm("ld.global.nc.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
        return v;
    } else {
        return __ldg(p);
    }
}
template <bool PROMOTE>
__device__ __forceinline__ double ldg(const double *p) {
    if constexpr (PROMOTE) {
        double v;
        asm("ld.global.nc.L2::256B.f64 %0, [%1];" : "=d"(v) : "l"(p));
        return v;
    } else {
        return __ldg(p);
    }
}
constexpr bool LD_OWN = ITLBM_LD_HINT >= 1, LD_RING = ITLBM_LD_HINT >= 2;
__device__ __forceinline__ void stg(float *p, float v) {
#if ITLBM_ST_HINT == 1
    __stcs(p, v);
#else
    *p = v;
#endif
}
__device__ __forceinline__ void stg(double *p, double v) {
#if ITLBM_ST_HINT == 1
    __stcs(p, v);
#else
    *p = v;
#endif
}

__device__ __forceinline__ int wrapi(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}
// a in [-HMAX, n + HMAX) -> a mod n by compare and add; only boxes narrower than the halo take the
// division
__device__ __forceinline__ int wrap_near(int a, int n) {
    int r = a < 0 ? a + n : (a >= n ? a - n : a);
    if ((unsigned)r >= (unsigned)n) r = wrapi(r, n);
    return r;
}

// Stride of the per-node auxiliary values in shared memory: 7, odd, so that the 32 lanes reading one
// component of consecutive nodes hit distinct banks (a stride of 6 words, or 12 for doubles, puts two
// lanes on each bank).
constexpr int AUXS = 7;

// Shared memory of a W x Hh tile.
template <class S, int W, int Hh>
struct SmemT {
    static constexpr int PX = W + 2 * HMAX, PY = Hh + 2 * HMAX;  // staged phase tile
    static constexpr int QX = W + 2, QY = Hh + 2;                // ring-1 region of the F1/F2 auxiliaries
    S phi[PY][PX];        // rho^N of tile + halo (HMAX), position (px, py) = global (x0-2+px, y0-2+py)
    S g[QY][QX][3];       // ring-1 gradient (F1, F2)
    S aux[QY][QX][AUXS];  // ring-1 normal (F1) or stress (F2), 6 values at an odd stride
};

// rho^N from the two colour sums.  FP64: (rho_R - rho_B) / (rho_R + rho_B), Imm_OPS.cpp:255-258.
// FP32: the sums are sum e_i (rho - rho0) and sum d_i (rho_R - rho_B).
__device__ __forceinline__ double phase_of(double rR, double rB, float) {
    return (rR - rB) / (rR + rB);
}
__device__ __forceinline__ float phase_of(float drho, float D, float rho0) {
    return D / (rho0 + drho);
}

// ring position r -> staged-tile coordinates (px, py) for a halo of H (1 or 2) around the W x Hh
// interior; consecutive r run along x in the top and bottom bands, so loads of consecutive r
// coalesce.  The divisions by the band width B are a multiply by ceil(2^16 / B) and a shift, exact
// for r < 2^16 / B (r stays below the band length, at most 2 x 36, here).
template <int W, int Hh>
__device__ __forceinline__ void ring_pos(int r, int H, int &px, int &py) {
    constexpr int W1 = W + 2, W2 = W + 4;
    constexpr int M1 = (65536 + W1 - 1) / W1, M2 = (65536 + W2 - 1) / W2;
    static_assert(2 * W2 < 65536 / W2, "ring index range: the multiply-shift division is exact");
    const int B = W + 2 * H, M = H == 1 ? M1 : M2;
    const int nTop = H * B;
    if (r < 2 * nTop) {
        const int band = r < nTop ? 0 : 1;
        r -= band * nTop;
        const int q = (r * M) >> 16;
        py = band ? HMAX + Hh + q : HMAX - H + q;
        px = HMAX - H + (r - q * B);
    } else {
        r -= 2 * nTop;
        const int q = H == 1 ? (r >> 1) : (r >> 2);  // r / (2 H)
        const int k = r - q * 2 * H;
        py = HMAX + q;
        px = k < H ? HMAX - H + k : HMAX + W + (k - H);
    }
}

// One tile of one case.
//   phase A  each thread loads its node: FP64 keeps f_i = f_R,i + f_B,i and the colour sums (all
//            colisao_comum needs, Operadores_tensao.cpp:343-360), FP32 keeps e_i and the sums;
//            the halo ring is loaded as (ring node, colour) items spread over all threads, each an
//            ordered sum of 19 values, and the two colours' lanes form the ring node's rho^N;
//   phase B  F1 / F2: gradient and normal or stress on the ring-1 region;
//   phase C  mediator gradient, force, collision, recolouring, push to x + c_i.
// FOLD (FP32 only): the nine in-plane classes per colour instead of the 19 populations.
template <class S, bool FOLD, int W, int Hh, int R>
__device__ __forceinline__ void step_tile(const CaseDev &c, int tile, int k, int aux_k,
                                          SmemT<S, W, Hh> &sm) {
    constexpr int NP = FOLD ? NK : NV;  // storage planes per colour
    constexpr int QX = SmemT<S, W, Hh>::QX, QY = SmemT<S, W, Hh>::QY;
    constexpr int HT = Hh / R;          // rows of one pass of the CTA's threads
    static_assert(HT * W == STEP_THREADS, "a pass of the threads covers W x HT nodes");
    const int tid = threadIdx.x;
    const int lx = tid % W, ly = tid / W;  // the thread's nodes are rows ly + jr HT, jr < R
    const int nx = c.nx, ny = c.ny, tiles_x = c.tiles_x;
    constexpr int TE = 2 * NP * PLANE;  // elements per tile block
    // the address of node (x, y) in a buffer; plane q of the node is at [q * PLANE] from it
    auto node = [tiles_x](auto *buf, int x_, int y_) { return buf + node_off(tiles_x, TE, x_, y_); };
    const int x0 = (int)((unsigned)tile & 0xFFFFu) * 8, y0 = (int)((unsigned)tile >> 16) * 8;
    const int xe = min(x0 + W, nx), ye = min(y0 + Hh, ny);  // end of the valid interior
    const int H = c.halo;
    const int cur = (c.parity0 + k) & 1;
    const S *__restrict__ src = (const S *)c.buf[cur];
    S *__restrict__ dst = (S *)c.buf[cur ^ 1];
    const int tipo = c.tipo;
    const float rho0f = c.pf.rho0;  // FP32: the reference density in float (phase_of)

    // ---- phase A ----------------------------------------------------------------------------
    const int x = x0 + lx;
    S f[R][NP], sa[R], sb[R];
    double sbd[R];
#pragma unroll
    for (int jr = 0; jr < R; jr++) {
        const int lyj = ly + jr * HT, y = y0 + lyj;
        const bool valid = (x < xe) && (y < ye);
        sa[jr] = S(0);
        sb[jr] = S(0);
        sbd[jr] = 0.0;
        if (x < xe + H && y < ye + H) {
            const int xw = valid ? x : wrap_near(x, nx), yw = valid ? y : wrap_near(y, ny);
            const S *own = node(src, xw, yw);
            S a[NP], b[NP];
#pragma unroll
            for (int i = 0; i < NP; i++) a[i] = ldg<LD_OWN>(own + i * PLANE);
#pragma unroll
            for (int i = 0; i < NP; i++) b[i] = ldg<LD_OWN>(own + (NP + i) * PLANE);
#pragma unroll
            for (int i = 0; i < NP; i++) sa[jr] = sa[jr] + a[i];
#pragma unroll
            for (int i = 0; i < NP; i++) sb[jr] = sb[jr] + b[i];
            if constexpr (std::is_same<S, float>::value) {
                // FP32: rho^N from the FP32 sums (as for the halo nodes); the colour difference is
                // also summed in FP64 for the rest population's complement (see the split below)
#pragma unroll
                for (int i = 0; i < NP; i++) sbd[jr] += (double)b[i];
            }
            if constexpr (std::is_same<S, double>::value) {
#pragma unroll
                for (int i = 0; i < NP; i++) f[jr][i] = a[i] + b[i];
            } else {
#pragma unroll
                for (int i = 0; i < NP; i++) f[jr][i] = a[i];
            }
            sm.phi[lyj + HMAX][lx + HMAX] = phase_of(sa[jr], sb[jr], rho0f);
        }
    }
    // halo ring: item it = (ring node it / 2, colour it % 2), the two colours of a node on adjacent
    // lanes, which exchange their sums by a shuffle; the loop runs in whole warps (the bound is a
    // multiple of 32) so that every lane of a warp takes part in the shuffle
    const int nring = (W + 2 * H) * (Hh + 2 * H) - W * Hh;
    for (int it = tid; it < ((2 * nring + 31) & ~31); it += STEP_THREADS) {
        const int colour = it & 1, r = it >> 1;
        int px = 0, py = 0;
        if (r < nring) ring_pos<W, Hh>(r, H, px, py);
        const int gx = x0 - HMAX + px, gy = y0 - HMAX + py;
        const bool act = r < nring && gx < xe + H && gy < ye + H;
        S acc = S(0);
        if (act) {
            const S *rn = node(src, wrap_near(gx, nx), wrap_near(gy, ny)) + colour * NP * PLANE;
            S v[NP];
#pragma unroll
            for (int i = 0; i < NP; i++) v[i] = ldg<LD_RING>(rn + i * PLANE);
#pragma unroll
            for (int i = 0; i < NP; i++) acc = acc + v[i];
        }
        const S other = __shfl_xor_sync(0xffffffffu, acc, 1);
        if (act && colour == 0) sm.phi[py][px] = phase_of(acc, other, rho0f);
    }
    __syncthreads();

    // ---- phase B: ring-1 gradient and normal / stress (F1, F2) -------------------------------
    const bool ring_aux = (tipo == ITLBM_OP_F1 || tipo == ITLBM_OP_F2);
    if (ring_aux) {
        for (int q = tid; q < QX * QY; q += STEP_THREADS) {
            const int qx = q % QX, qy = q / QX;
            const int gx = x0 - 1 + qx, gy = y0 - 1 + qy;
            if (gx < xe + 1 && gy < ye + 1) {
                S g0, g1, g2;
                if constexpr (std::is_same<S, float>::value) {
                    // FP32 (both storage forms): the in-plane class forms, g_z = 0 on the slab
                    mediator_grad_fold([&](int dx, int dy) { return sm.phi[qy + 1 + dy][qx + 1 + dx]; }, g0, g1);
                    g0 = -g0;  // the isotropic gradient
                    g1 = -g1;
                    g2 = 0.f;
                    if (tipo == ITLBM_OP_F1) aux_normal_plane(g0, g1, sm.aux[qy][qx]);
                    else aux_stress_plane(g0, g1, c.pf.sigma, sm.aux[qy][qx]);
                } else {
                    iso_grad(sm.phi, qx + 1, qy + 1, g0, g1, g2);
                    if (tipo == ITLBM_OP_F1) aux_normal(g0, g1, g2, sm.aux[qy][qx]);
                    else aux_stress(g0, g1, g2, (S)c.sigma, sm.aux[qy][qx]);
                }
                sm.g[qy][qx][0] = g0;
                sm.g[qy][qx][1] = g1;
                sm.g[qy][qx][2] = g2;
            }
        }
        __syncthreads();
    }

    // ---- phase C: mediator gradient, force, collision, push ----------------------------------
#pragma unroll
    for (int jr = 0; jr < R; jr++) {
      const int lyj = ly + jr * HT, y = y0 + lyj;
      if ((x < xe) && (y < ye)) {
        CaseDev::F32Par pf{};  // FP32: the case's parameters in float
        if constexpr (std::is_same<S, float>::value) pf = load_pf(c);
        const int px = lx + HMAX, py = lyj + HMAX;
        S gmx, gmy, gmz;
        auto phi_at = [&](int dx, int dy) { return sm.phi[py + dy][px + dx]; };
        if constexpr (std::is_same<S, float>::value) {
            mediator_grad_fold(phi_at, gmx, gmy);  // FP32: class form, g_z = 0 on the slab
            gmz = S(0);
        } else mediator_grad(sm.phi, px, py, gmx, gmy, gmz);
        S Fx = S(0), Fy = S(0), Fz = S(0);
        const bool force = tipo >= ITLBM_OP_F1;
        if (tipo == ITLBM_OP_F1) {
            const int qx = lx + 1, qy = lyj + 1;
            S kappa;
            if constexpr (std::is_same<S, float>::value)
                kappa = curvature_plane([&](int dx, int dy) { return sm.aux[qy + dy][qx + dx]; });
            else
                kappa = curvature<S, AUXS>(sm.aux, qx, qy);
            S sig;
            if constexpr (std::is_same<S, float>::value) sig = pf.sigma;
            else sig = c.sigma;
            const S hs = (S(0.5) * sig) * kappa;
            Fx = hs * sm.g[qy][qx][0];
            Fy = hs * sm.g[qy][qx][1];
            Fz = hs * sm.g[qy][qx][2];
        } else if (tipo == ITLBM_OP_F2) {
            if constexpr (std::is_same<S, float>::value)
                stress_div_plane([&](int dx, int dy) { return sm.aux[lyj + 1 + dy][lx + 1 + dx]; }, Fx, Fy);
            else
                stress_div<S, AUXS>(sm.aux, lx + 1, lyj + 1, Fx, Fy, Fz);
        } else if (tipo == ITLBM_OP_F3) {
            S g0, g1, g2, mu;
            if constexpr (std::is_same<S, float>::value) {
                g0 = -gmx;  // the isotropic gradient is the exact negative of the mediator momentum
                g1 = -gmy;
                g2 = -gmz;
                mu = chem_pot_fold(phi_at, pf.kf, pf.bf);
            } else {
                iso_grad(sm.phi, px, py, g0, g1, g2);
                mu = chem_pot(sm.phi, px, py, (S)c.kf, (S)c.bf);
            }
            Fx = mu * g0;
            Fy = mu * g1;
            Fz = mu * g2;
        }
        // the destination node x + c_i (periodic) of D3Q19 direction i, or of class i of the fold
        const int xp = (x + 1 == nx) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
        const int yp = (y + 1 == ny) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
        auto dst_node = [&](int i) {
            const int ex = FOLD ? kx(i) : cx(i), ey = FOLD ? ky(i) : cy(i);
            return node(dst, ex == 0 ? x : (ex > 0 ? xp : xm), ey == 0 ? y : (ey > 0 ? yp : ym));
        };
        bool skip;
        if constexpr (FOLD) {
            RecolourFold rc;
            if (force) collide_fold<true>(f[jr], sa[jr], sb[jr], gmx, gmy, Fx, Fy, pf, rc);
            else collide_fold<false>(f[jr], sa[jr], sb[jr], gmx, gmy, Fx, Fy, pf, rc);
            skip = rc.skip;
            if (!skip) {
                double dsum = 0.0;
                sfor<0, 4>([&](auto M) {
                    constexpr int K = 2 * decltype(M)::value + 1;
                    float dK, dJ;
                    split_fold_pair<K>(rc, f[jr][K], f[jr][K + 1], shift_of<kx(K)>(pf, wk<float>(K)),
                                       shift_of<kx(K + 1)>(pf, wk<float>(K + 1)), dK, dJ);
                    dsum += (double)dK;
                    dsum += (double)dJ;
                    float *nK = dst_node(K), *nJ = dst_node(K + 1);
                    stg(nK + K * PLANE, f[jr][K]);
                    stg(nK + (NK + K) * PLANE, dK);
                    stg(nJ + (K + 1) * PLANE, f[jr][K + 1]);
                    stg(nJ + (NK + K + 1) * PLANE, dJ);
                });
                float *n0 = dst_node(0);
                stg(n0, f[jr][0]);
                stg(n0 + NK * PLANE, (float)(sbd[jr] - dsum));
            }
        } else if constexpr (std::is_same<S, double>::value) {
            Recolour64 rc;
            if (force) collide_f64<true>(f[jr], sa[jr], sb[jr], gmx, gmy, gmz, Fx, Fy, Fz, c, rc);
            else collide_f64<false>(f[jr], sa[jr], sb[jr], gmx, gmy, gmz, Fx, Fy, Fz, c, rc);
            skip = rc.skip;
            if (!skip) {
                sfor<0, NV>([&](auto I) {
                    constexpr int i = decltype(I)::value;
                    double r, b;
                    split64<i>(rc, f[jr][i], r, b);
                    double *n = dst_node(i);
                    stg(n + i * PLANE, r);
                    stg(n + (NV + i) * PLANE, b);
                });
            }
        } else {
            Recolour32 rc;
            if (force) collide_f32<true>(f[jr], sa[jr], sb[jr], gmx, gmy, gmz, Fx, Fy, Fz, pf, rc);
            else collide_f32<false>(f[jr], sa[jr], sb[jr], gmx, gmy, gmz, Fx, Fy, Fz, pf, rc);
            skip = rc.skip;
            if (!skip) {
                // d_0 is the complement of the moving d_i against the incoming D, both summed in
                // FP64: the d_i are O(w_i rho), so FP32 sums would round by ~1e-8 rho per node and
                // step, coherently over uniform regions, and drift the colour masses (1e-6 in 2000
                // steps); in FP64 the only rounding left is that of d_0 itself.
                double dsum = 0.0;
                sfor<0, 9>([&](auto M) {
                    constexpr int i = 2 * decltype(M)::value + 1;
                    float di, dj;
                    split32_pair<i>(rc, f[jr][i], f[jr][i + 1], shift_of<cx(i)>(pf, wgt<float>(i)),
                                    shift_of<cx(i + 1)>(pf, wgt<float>(i + 1)), di, dj);
                    dsum += (double)di;
                    dsum += (double)dj;
                    float *ni = dst_node(i), *nj = dst_node(i + 1);
                    stg(ni + i * PLANE, f[jr][i]);
                    stg(ni + (NV + i) * PLANE, di);
                    stg(nj + (i + 1) * PLANE, f[jr][i + 1]);
                    stg(nj + (NV + i + 1) * PLANE, dj);
                });
                float *n0 = dst_node(0);
                stg(n0, f[jr][0]);
                stg(n0 + NV * PLANE, (float)(sbd[jr] - dsum));
            }
        }
        if (skip) {  // rho <= 1e-30: the site is streamed unchanged (Operadores_tensao.cpp:347)
            const S *own = node(src, x, y);
            sfor<0, NP>([&](auto I) {
                constexpr int i = decltype(I)::value;
                S *n = dst_node(i);
                n[i * PLANE] = own[i * PLANE];
                n[(NP + i) * PLANE] = own[(NP + i) * PLANE];
            });
        }

        if (c.aux != nullptr && (k == aux_k || (c.aux_at_end && k == c.chunk_len - 1))) {
            const long long o = aux_off(c, x, y);
            const long long n = c.aux_stride;
            c.aux[o] = (double)Fx;
            c.aux[n + o] = (double)Fy;
            c.aux[2 * n + o] = (double)Fz;
            c.aux[3 * n + o] = sqrt((double)gmx * gmx + (double)gmy * gmy + (double)gmz * gmz);
        }
      }
    }
    __syncthreads();
}

// Resident CTAs per SM the register allocation is sized for: 2 x 256 threads for FP64, 4 x 256
// threads for FP32 (the kernel is latency-bound at lower occupancy; see the ncu summaries).
#ifndef ITLBM_F64_BLOCKS
#define ITLBM_F64_BLOCKS 2
#endif
#ifndef ITLBM_F32_BLOCKS
#define ITLBM_F32_BLOCKS 4
#endif
#ifndef ITLBM_FOLD_BLOCKS  // the fold at 5 or 6 CTAs per SM (48 or 40 registers, with spills) measured
#define ITLBM_FOLD_BLOCKS 4   // 17 % and 8 % slower on the 600-case batch
#endif
#ifdef ITLBM_STEP_F64
#define ITLBM_STEP_MIN_BLOCKS(fold) (ITLBM_F64_BLOCKS * 256 / STEP_THREADS)
#else
#define ITLBM_STEP_MIN_BLOCKS(fold) (((fold) ? ITLBM_FOLD_BLOCKS : ITLBM_F32_BLOCKS) * 256 / STEP_THREADS)
#endif

template <class S, bool FOLD, int W>
__global__ void __launch_bounds__(STEP_THREADS, ITLBM_STEP_MIN_BLOCKS(FOLD)) k_step(const CaseDev *__restrict__ cases,
                                                       const TileRef *__restrict__ tiles,
                                                       int ntiles, const int *__restrict__ ntiles_dev,
                                                       int k, int aux_k) {
    constexpr int R = FOLD ? ITLBM_FOLD_ROWS : (std::is_same<S, float>::value ? ITLBM_F32_ROWS : 1);  // rows per thread
    constexpr int Hh = R * STEP_THREADS / W;
    __shared__ SmemT<S, W, Hh> sm;
    const int nt = ntiles_dev ? *ntiles_dev : ntiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const TileRef tr = tiles[t];
        const CaseDev &c = cases[tr.case_id];
        if (k >= c.chunk_len) continue;
        step_tile<S, FOLD, W, Hh, R>(c, tr.tile, k, aux_k, sm);
    }
}

template <class S, bool FOLD>
cudaError_t launch_shape(const CaseDev *cases_dev, const TileRef *tiles, int ntiles, const int *ntiles_dev,
                         int grid, int k, int aux_k, int shape, cudaStream_t s) {
    if (grid <= 0) return cudaSuccess;
    switch (shape) {
        case SHAPE_32x8: k_step<S, FOLD, 32><<<grid, STEP_THREADS, 0, s>>>(cases_dev, tiles, ntiles, ntiles_dev, k, aux_k); break;
        case SHAPE_16x16: k_step<S, FOLD, 16><<<grid, STEP_THREADS, 0, s>>>(cases_dev, tiles, ntiles, ntiles_dev, k, aux_k); break;
        case SHAPE_8x32: k_step<S, FOLD, 8><<<grid, STEP_THREADS, 0, s>>>(cases_dev, tiles, ntiles, ntiles_dev, k, aux_k); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

// This file is compiled twice: with ITLBM_STEP_F64 (and --fmad=false, so that every FP64 operation
// rounds exactly as the reference's own code compiled with strict IEEE semantics) and without it.
#ifdef ITLBM_STEP_F64
cudaError_t launch_step_f64(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                            const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s) {
    return launch_shape<double, false>(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
}
// The occupancy queries also load every shape's kernel (with lazy module loading a kernel is loaded
// at its first launch, which would otherwise fall inside the batch's first timed tuning window).
int step_occupancy_f64() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<double, false, 32>, STEP_THREADS, 0);
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_step<double, false, 16>);
    cudaFuncGetAttributes(&a, k_step<double, false, 8>);
    return n;
}
#else
cudaError_t launch_step_f32(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                            const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s) {
    return launch_shape<float, false>(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
}
int step_occupancy_f32() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step<float, false, 32>, STEP_THREADS, 0);
    cudaFuncAttributes a;
    cudaFuncGetAttributes(&a, k_step<float, false, 16>);
    cudaFuncGetAttributes(&a, k_step<float, false, 8>);
    cudaFuncGetAttributes(&a, k_step<float, true, 32>);
    cudaFuncGetAttributes(&a, k_step<float, true, 16>);
    cudaFuncGetAttributes(&a, k_step<float, true, 8>);
    return n;
}
cudaError_t launch_step_fold(const CaseDev *cases_dev, const TileRef *tiles, int ntiles,
                             const int *ntiles_dev, int grid, int k, int aux_k, int shape, cudaStream_t s) {
    return launch_shape<float, true>(cases_dev, tiles, ntiles, ntiles_dev, grid, k, aux_k, shape, s);
}
#endif

}  // namespace itlbm
