// itlbm_march.cu -- the FP32 step as a march down column strips, fed by TMA.
//
// The tile kernel (itlbm_step.cu) reads every node of its tile once from HBM but re-reads a ring of
// halo nodes from L2, and a CTA's loads and its arithmetic alternate, so HBM idles while the CTA
// computes.  Here a CTA owns a strip of MW = 32 columns over a segment of up to SEG rows and walks
// it in slabs of MR = 4 rows:
//   * one thread issues, per row, two TMA copies (the 19 e-planes and the 19 d-planes of the columns
//     x0-4 .. x0+35) into shared memory, three slabs ahead of the slab being collided, so the copies
//     of the next slabs run while this one computes;
//   * rho^N of every staged row (interior and the 1- or 2-column halo) is formed once, into a ring of
//     rows; a row's halo above and below comes from the previous and next slab, so only the two halo
//     columns (and H rows per segment) are read twice;
//   * F1 / F2: the gradient and the normal (F1) or capillary stress (F2) of the ring-1 region go to a
//     ring of rows too;
//   * each warp collides one row of the slab with exactly the arithmetic of the tile kernel (the
//     site functions of itlbm_site.cuh, the same sums in the same order) and pushes to x + c_i.
// The result is bit-identical to the FP32 tile kernel.  Columns outside [0, nx) are wrapped with
// plain loads (the copies fill them with zeros), as are rows read from another segment's edge.
// Every wait on a copy is bounded (1 s); a CTA that gives up sets an error flag that the host reads
// (ITLBM_E_TIMEOUT) and returns once its other copies have landed or timed out as well.
#include "itlbm_site.cuh"
#include "itlbm_tma.cuh"

#include <cuda.h>

namespace itlbm {

namespace {

constexpr int MW = 32;                     // strip width (one warp)
constexpr int MR = 4;                      // rows per slab (one per warp)
constexpr int MT = MW * MR;                // threads per CTA
constexpr int BW = 40;                     // staged columns x0 - 4 .. x0 + 35
constexpr int ROWF = 768;                  // floats per staged row: 19 x 40 = 760, padded to 3072 B
constexpr unsigned ROW_TX = NV * BW * 4;   // bytes one row copy delivers (3040)
constexpr int PR = 16;                     // rows of the rho^N ring
constexpr int NR = 8;                      // rows of the D / drho / auxiliary rings
constexpr int AW = MW + 2;                 // auxiliary columns x0 - 1 .. x0 + 32

struct MarchSmem {
    alignas(128) float e[3][MR][ROWF];     // e-planes of three slabs
    alignas(128) float d[2][MR][ROWF];     // d-planes of two slabs
    float phi[PR][BW];                     // rho^N, column index x - x0 + 4
    double D[NR][MW];                      // sum d_i of the interior nodes (FP64)
    float Df[NR][MW];                      // the same in FP32, as rho^N uses it
    float drho[NR][MW];                    // sum e_i of the interior nodes
    float aux[NR][AW][6];                  // F1: normal 0..2, gradient 3..5; F2: stress 0..5
    alignas(8) unsigned long long bar[3];  // one per e-slot: both copies of a slab complete on it
    int fail;
};

__device__ int g_march_status = 0;

__device__ __forceinline__ int wrapm(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// One row: the 19 planes from `plane` of buffer `buf`, columns x .. x + 39 of row y.
__device__ __forceinline__ void tma_row(const CUtensorMap *map, float *dst, int x, int y, int plane, int buf,
                                        unsigned long long *bar) {
    tma_load_4d(map, dst, x, y, plane, buf, bar);
}

struct Item {
    int x0, y0, y1, H, cur, nslab;
};

// rows of slab s (s = -1 .. nslab) that are copied: the slab's rows within [y0 - H, y1 + H)
__device__ __forceinline__ void slab_rows(const Item &it, int s, int &r0, int &r1) {
    r0 = max(it.y0 + MR * s, it.y0 - it.H);
    r1 = min(it.y0 + MR * s + MR, it.y1 + it.H);
}
__device__ __forceinline__ int eslot(int s) { return (s % 3 + 3) % 3; }
__device__ __forceinline__ int dslot(int s) { return (s % 2 + 2) % 2; }

// Thread 0: issue the copies of slab s (nothing when it has no row to copy).
__device__ __forceinline__ void issue_slab(const CaseDev &c, const Item &it, int s, MarchSmem &sm) {
    int r0, r1;
    slab_rows(it, s, r0, r1);
    if (r1 <= r0) return;
    const int es = eslot(s), ds = dslot(s);
    unsigned long long *bar = &sm.bar[es];
    mbar_expect(bar, (unsigned)(r1 - r0) * 2u * ROW_TX);
    const int base = it.y0 + MR * s;
    for (int r = r0; r < r1; r++) {
        const int yw = wrapm(r, c.ny);
        tma_row(&c.tmap, sm.e[es][r - base], it.x0 - 4, yw, 0, it.cur, bar);
        tma_row(&c.tmap, sm.d[ds][r - base], it.x0 - 4, yw, NV, it.cur, bar);
    }
}

// All threads: wait (thread 0, bounded) for slab s; false if the copies did not land (the expected
// parity is then left as it was, for drain).
__device__ __forceinline__ bool wait_slab(const Item &it, int s, MarchSmem &sm, unsigned &phase) {
    int r0, r1;
    slab_rows(it, s, r0, r1);
    if (r1 <= r0) return true;
    const int es = eslot(s);
    if (threadIdx.x == 0) {
        if (!mbar_wait(&sm.bar[es], (phase >> es) & 1u)) sm.fail = 1;
    }
    __syncthreads();
    if (sm.fail) return false;
    phase ^= 1u << es;
    return true;
}

// rho^N of every staged node of slab s (interior and halo columns); the sums of the interior
// nodes are kept for the collision.
__device__ __forceinline__ void phi_pass(const CaseDev &c, const Item &it, int s, MarchSmem &sm) {
    int r0, r1;
    slab_rows(it, s, r0, r1);
    if (r1 <= r0) return;
    const int H = it.H, cols = MW + 2 * H;
    const int base = it.y0 + MR * s;
    const int es = eslot(s), ds = dslot(s);
    const float *__restrict__ src = (const float *)c.buf[it.cur];
    const float rho0 = (float)c.rho0;
    for (int q = threadIdx.x; q < (r1 - r0) * cols; q += MT) {
        const int r = r0 + q / cols;
        const int col = it.x0 - H + q % cols;
        const int bx = col - it.x0 + 4;  // staged column
        const int lx = col - it.x0;
        const bool own = (r >= it.y0 && r < it.y1 && lx >= 0 && lx < MW);
        float sa = 0.f, sb = 0.f;
        double sbd = 0.0;
        float d[NV];
        if (col >= 0 && col < c.nx) {
            const float *pe = &sm.e[es][r - base][bx];
            const float *pd = &sm.d[ds][r - base][bx];
#pragma unroll
            for (int i = 0; i < NV; i++) sa = sa + pe[i * BW];
#pragma unroll
            for (int i = 0; i < NV; i++) d[i] = pd[i * BW];
        } else {  // periodic wrap in x: not in the copy
            const long long off = (long long)wrapm(r, c.ny) * c.pitch + wrapm(col, c.nx);
#pragma unroll
            for (int i = 0; i < NV; i++) sa = sa + __ldg(src + (long long)i * c.stride + off);
#pragma unroll
            for (int i = 0; i < NV; i++) d[i] = __ldg(src + (long long)(NV + i) * c.stride + off);
        }
#pragma unroll
        for (int i = 0; i < NV; i++) sb = sb + d[i];
        sm.phi[(r - it.y0 + PR) & (PR - 1)][bx] = sb / (rho0 + sa);
        if (own) {
#pragma unroll
            for (int i = 0; i < NV; i++) sbd += (double)d[i];
            sm.D[(r - it.y0 + NR) & (NR - 1)][lx] = sbd;
            sm.Df[(r - it.y0 + NR) & (NR - 1)][lx] = sb;
            sm.drho[(r - it.y0 + NR) & (NR - 1)][lx] = sa;
        }
    }
}

// F1 / F2: gradient and normal or stress on rows [ra, rb), columns x0 - 1 .. x0 + 32.
__device__ __forceinline__ void aux_pass(const CaseDev &c, const Item &it, int ra, int rb, MarchSmem &sm) {
    for (int q = threadIdx.x; q < (rb - ra) * AW; q += MT) {
        const int r = ra + q / AW, ax = q % AW;
        const int pr = r - it.y0 + PR, bx = ax + 3;  // phi column of aux column ax
        auto phi = [&](int dx, int dy) { return sm.phi[(pr + dy) & (PR - 1)][bx + dx]; };
        float g0, g1;
        mediator_grad_fold(phi, g0, g1);  // the class form, as the tile kernel (g_z = 0 on the slab)
        g0 = -g0;
        g1 = -g1;
        float *a = sm.aux[(r - it.y0 + NR) & (NR - 1)][ax];
        if (c.tipo == ITLBM_OP_F1) {
            aux_normal_plane(g0, g1, a);
            a[3] = g0;
            a[4] = g1;
            a[5] = 0.f;
        } else {
            aux_stress_plane(g0, g1, (float)c.sigma, a);
        }
    }
}

// Collision and push of the node (x0 + lane, r), r a row of slab s.
__device__ __forceinline__ void collide_row(const CaseDev &c, const Item &it, int s, int r, int k, int aux_k,
                                            MarchSmem &sm) {
    const int lane = threadIdx.x % MW;
    const int x = it.x0 + lane, y = r;
    if (y >= it.y1 || x >= c.nx) return;
    const int nx = c.nx, ny = c.ny, pitch = c.pitch;
    const long long stride = c.stride;
    const int tipo = c.tipo;
    const float *src = (const float *)c.buf[it.cur];
    float *__restrict__ dst = (float *)c.buf[it.cur ^ 1];
    const float *pe = &sm.e[eslot(s)][r - (it.y0 + MR * s)][lane + 4];
    float f[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) f[i] = pe[i * BW];
    const int rr = (r - it.y0 + NR) & (NR - 1);
    const float sa = sm.drho[rr][lane];
    const double sbd = sm.D[rr][lane];
    const float sb = sm.Df[rr][lane];
    const int pr = r - it.y0 + PR, bx = lane + 4;
    auto phi = [&](int dx, int dy) { return sm.phi[(pr + dy) & (PR - 1)][bx + dx]; };
    float gmx, gmy;
    mediator_grad_fold(phi, gmx, gmy);
    const float gmz = 0.f;
    float Fx = 0.f, Fy = 0.f, Fz = 0.f;
    const bool force = tipo >= ITLBM_OP_F1;
    if (tipo == ITLBM_OP_F1 || tipo == ITLBM_OP_F2) {
        const int ar = r - it.y0 + NR, ax = lane + 1;
        auto aux = [&](int dx, int dy) -> const float * { return sm.aux[(ar + dy) & (NR - 1)][ax + dx]; };
        if (tipo == ITLBM_OP_F1) {
            const float kappa = curvature_plane(aux);
            const float hs = (0.5f * (float)c.sigma) * kappa;
            const float *g = aux(0, 0);
            Fx = hs * g[3];
            Fy = hs * g[4];
            Fz = hs * g[5];
        } else {
            stress_div_plane(aux, Fx, Fy);
        }
    } else if (tipo == ITLBM_OP_F3) {
        const float g0 = -gmx, g1 = -gmy, g2 = -gmz;  // the isotropic gradient, exactly
        const float mu = chem_pot_fold(phi, (float)c.kf, (float)c.bf);
        Fx = mu * g0;
        Fy = mu * g1;
        Fz = mu * g2;
    }
    const int xp = (x + 1 == nx) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
    const int yp = (y + 1 == ny) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
    auto dst_off = [&](int i) {
        const int xd = cx(i) == 0 ? x : (cx(i) > 0 ? xp : xm);
        const int yd = cy(i) == 0 ? y : (cy(i) > 0 ? yp : ym);
        return (long long)yd * pitch + xd;
    };
    Recolour32 rc;
    if (force) collide_f32<true>(f, sa, sb, gmx, gmy, gmz, Fx, Fy, Fz, c, rc);
    else collide_f32<false>(f, sa, sb, gmx, gmy, gmz, Fx, Fy, Fz, c, rc);
    if (!rc.skip) {
        // d_0 as the complement of the moving d_i against the incoming D, both in FP64
        const float rho0 = (float)c.rho0;
        double dsum = 0.0;
        sfor<0, 9>([&](auto M) {
            constexpr int i = 2 * decltype(M)::value + 1;
            float di, dj;
            split32_pair<i>(rc, f[i], f[i + 1], rho0, di, dj);
            dsum += (double)di;
            dsum += (double)dj;
            const long long oi = dst_off(i), oj = dst_off(i + 1);
            dst[(long long)i * stride + oi] = f[i];
            dst[(long long)(NV + i) * stride + oi] = di;
            dst[(long long)(i + 1) * stride + oj] = f[i + 1];
            dst[(long long)(NV + i + 1) * stride + oj] = dj;
        });
        const long long o0 = dst_off(0);
        dst[o0] = f[0];
        dst[(long long)NV * stride + o0] = (float)(sbd - dsum);
    } else {  // rho <= 1e-30: the site is streamed unchanged (Operadores_tensao.cpp:347)
        const long long off = (long long)y * pitch + x;
        sfor<0, NV>([&](auto I) {
            constexpr int i = decltype(I)::value;
            const long long o = dst_off(i);
            dst[(long long)i * stride + o] = src[(long long)i * stride + off];
            dst[(long long)(NV + i) * stride + o] = src[(long long)(NV + i) * stride + off];
        });
    }
    if (c.aux != nullptr && (k == aux_k || (c.aux_at_end && k == c.chunk_len - 1))) {
        const long long o = (long long)y * pitch + x;
        c.aux[o] = (double)Fx;
        c.aux[stride + o] = (double)Fy;
        c.aux[2 * stride + o] = (double)Fz;
        c.aux[3 * stride + o] = sqrt((double)gmx * gmx + (double)gmy * gmy + (double)gmz * gmz);
    }
}

// After a failed wait on slab s_first: wait again (bounded) for it and for every later slab in
// flight, up to s_last, then the CTA returns.
__device__ void drain(const Item &it, int s_first, int s_last, MarchSmem &sm, unsigned phase) {
    if (threadIdx.x == 0) {
        atomicExch(&g_march_status, 1);
        for (int s = s_first; s <= s_last; s++) {
            int r0, r1;
            slab_rows(it, s, r0, r1);
            if (r1 <= r0) continue;
            const int es = eslot(s);
            mbar_wait(&sm.bar[es], (phase >> es) & 1u);
            phase ^= 1u << es;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(MT, 3) k_march(const CaseDev *__restrict__ cases,
                                                 const TileRef *__restrict__ items, int nitems,
                                                 const int *__restrict__ nitems_dev, int k, int aux_k) {
    extern __shared__ __align__(128) unsigned char smraw[];
    // the row copies need 128-byte aligned destinations: align the block explicitly
    MarchSmem &sm = *reinterpret_cast<MarchSmem *>(((uintptr_t)smraw + 127) & ~(uintptr_t)127);
    const int nt = nitems_dev ? *nitems_dev : nitems;
    if (threadIdx.x == 0) {
        for (int b = 0; b < 3; b++) mbar_init(&sm.bar[b]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sm.fail = 0;
    }
    __syncthreads();
    unsigned phase = 0;  // expected parity of each e-slot barrier, uniform over the CTA
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const TileRef tr = items[t];
        const CaseDev &c = cases[tr.case_id];
        if (k >= c.chunk_len) continue;
        Item it;
        it.H = c.halo;
        it.cur = (c.parity0 + k) & 1;
        const int strip = tr.tile % c.m_strips, seg = tr.tile / c.m_strips;
        it.x0 = strip * MW;
        it.y0 = seg * MARCH_SEG;
        it.y1 = min(it.y0 + MARCH_SEG, c.ny);
        it.nslab = (it.y1 - it.y0 + MR - 1) / MR;
        const bool ring_aux = (c.tipo == ITLBM_OP_F1 || c.tipo == ITLBM_OP_F2);

        // prologue: the halo rows above, slab 0, then slabs 1 and 2 in flight
        if (threadIdx.x == 0) {
            // the map was written by the host before the launch; order this proxy's view after it
            tensormap_acquire(&c.tmap);
            issue_slab(c, it, -1, sm);
            issue_slab(c, it, 0, sm);
        }
        if (!wait_slab(it, -1, sm, phase)) {
            drain(it, -1, 0, sm, phase);
            return;
        }
        phi_pass(c, it, -1, sm);
        if (!wait_slab(it, 0, sm, phase)) {
            drain(it, 0, 0, sm, phase);
            return;
        }
        phi_pass(c, it, 0, sm);
        __syncthreads();  // slab -1 and the d-planes of slab 0 are consumed
        if (threadIdx.x == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_slab(c, it, 1, sm);
            issue_slab(c, it, 2, sm);
        }
        if (ring_aux) aux_pass(c, it, it.y0 - 1, min(it.y0 + 1, it.y1 + 1), sm);

        for (int j = 0; j < it.nslab; j++) {
            if (!wait_slab(it, j + 1, sm, phase)) {
                drain(it, j + 1, min(j + 2, it.nslab), sm, phase);
                return;
            }
            phi_pass(c, it, j + 1, sm);
            __syncthreads();
            if (ring_aux) {
                aux_pass(c, it, it.y0 + MR * j + 1, min(it.y0 + MR * j + MR + 1, it.y1 + 1), sm);
                __syncthreads();
            }
            collide_row(c, it, j, it.y0 + MR * j + threadIdx.x / MW, k, aux_k, sm);
            __syncthreads();  // slab j's e-planes and slab j + 1's d-planes are free
            if (threadIdx.x == 0 && j + 3 <= it.nslab) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue_slab(c, it, j + 3, sm);
            }
        }
    }
}

}  // namespace

size_t march_smem_bytes() { return sizeof(MarchSmem) + 128; }

// Opt the kernel in to its shared memory on the current device; call before any launch or stream
// capture on that device.
cudaError_t march_prepare() {
    return cudaFuncSetAttribute(k_march, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)march_smem_bytes());
}

cudaError_t launch_march_f32(const CaseDev *cases_dev, const TileRef *items, int nitems, const int *nitems_dev,
                             int grid, int k, int aux_k, cudaStream_t s) {
    if (grid <= 0) return cudaSuccess;
    k_march<<<grid, MT, march_smem_bytes(), s>>>(cases_dev, items, nitems, nitems_dev, k, aux_k);
    return cudaGetLastError();
}

int march_error_take() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_march_status, sizeof(int)) != cudaSuccess) return 0;
    if (v) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_march_status, &zero, sizeof(int));
    }
    return v;
}

// The 4-D view {nx, ny, 38 planes, 2 buffers} of an FP32 state for the row copies of k_march:
// boxes of 40 columns x 1 row x 19 planes; columns outside [0, nx) read as zeros.
namespace {
typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                             const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                             CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p) return nullptr;
        fn = (EncodeFn)p;
    }
    return fn;
}
}  // namespace

cudaError_t encode_state_map(CaseDev &h, void *mem, size_t per_buf) {
    const EncodeFn fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const cuuint64_t dims[4] = {(cuuint64_t)h.nx, (cuuint64_t)h.ny, (cuuint64_t)(2 * NV), 2};
    const cuuint64_t strides[3] = {(cuuint64_t)h.pitch * 4, (cuuint64_t)h.stride * 4, (cuuint64_t)per_buf};
    const cuuint32_t box[4] = {(cuuint32_t)BW, 1, (cuuint32_t)NV, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(&h.tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, mem, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace itlbm
