// itlbm_snapshot.cu -- saving and restoring the state of a case (host side).
//
// The reference restarts an interrupted batch from step 0 (rodar_lote.py:5-7).  A snapshot holds a
// case's description, its step count and its populations at the top of its next step, in its own
// precision and storage form (FP64 f_R, f_B or FP32 e, d), planes of nx * ny elements in plain rows
// (the device's tile-blocked planes are converted on the host).  Stepping a restored case gives the same bits the saved run would have given.
#include "itlbm_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace itlbm {

namespace {

constexpr char MAGIC[8] = {'I', 'T', 'L', 'B', 'M', 'S', 'T', '1'};

// Plane q of a state buffer (tile-major, node_off) to and from the file's plain nx * ny rows.
void unblock(const CaseDev &h, size_t elem, int q, const unsigned char *buf, unsigned char *rows) {
    for (int y = 0; y < h.ny; y++)
        for (int x0 = 0; x0 < h.nx; x0 += TX) {
            const size_t n = (size_t)std::min(TX, h.nx - x0) * elem;
            std::memcpy(rows + ((size_t)y * h.nx + x0) * elem, buf + (size_t)(node_off(h, x0, y) + q * PLANE) * elem, n);
        }
}
void reblock(const CaseDev &h, size_t elem, int q, const unsigned char *rows, unsigned char *buf) {
    for (int y = 0; y < h.ny; y++)
        for (int x0 = 0; x0 < h.nx; x0 += TX) {
            const size_t n = (size_t)std::min(TX, h.nx - x0) * elem;
            std::memcpy(buf + (size_t)(node_off(h, x0, y) + q * PLANE) * elem, rows + ((size_t)y * h.nx + x0) * elem, n);
        }
}

}  // namespace

int snap_write(const char *path, const itlbm_case_desc &d, long long steps, const CaseDev &h, const void *state) {
    SnapHeader hd{};
    std::memcpy(hd.magic, MAGIC, 8);
    hd.version = 2;  // 2: FP32 states are deviations from the equilibrium at the case's initial flow
    hd.desc = d;
    hd.steps = steps;
    const size_t elem = elem_of(h.prec);
    std::vector<unsigned char> whole(elem * (size_t)h.buf_elems), plane(elem * (size_t)h.nx * h.ny);
    const cudaError_t e = cudaMemcpy(whole.data(), state, whole.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "snapshot copy");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ITLBM_E_IO, std::string("cannot write ") + path);
    bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1;
    for (int q = 0; ok && q < 2 * planes_of(h.prec); q++) {
        unblock(h, elem, q, whole.data(), plane.data());
        ok = std::fwrite(plane.data(), 1, plane.size(), f) == plane.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? ITLBM_OK : fail(ITLBM_E_IO, std::string("short write to ") + path);
}

int snap_read_header(const char *path, SnapHeader &hd) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ITLBM_E_IO, std::string("cannot open ") + path);
    const bool ok = std::fread(&hd, sizeof hd, 1, f) == 1;
    std::fclose(f);
    if (!ok || std::memcmp(hd.magic, MAGIC, 8) != 0 || hd.version != 2)
        return fail(ITLBM_E_PARSE, std::string("not a case snapshot: ") + path);
    const itlbm_case_desc &d = hd.desc;
    if (d.nx < 1 || d.ny < 1 || (long long)d.nx * d.ny > (1LL << 30) || hd.steps < 0 ||
        !prec_valid(d.precision))
        return fail(ITLBM_E_PARSE, std::string("corrupt case snapshot: ") + path);
    return ITLBM_OK;
}

int snap_read_state(const char *path, const CaseDev &h, void *state) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ITLBM_E_IO, std::string("cannot open ") + path);
    const size_t elem = elem_of(h.prec);
    std::vector<unsigned char> whole(elem * (size_t)h.buf_elems, 0), plane(elem * (size_t)h.nx * h.ny);
    bool ok = std::fseek(f, (long)sizeof(SnapHeader), SEEK_SET) == 0;
    for (int q = 0; ok && q < 2 * planes_of(h.prec); q++) {
        ok = std::fread(plane.data(), 1, plane.size(), f) == plane.size();
        if (ok) reblock(h, elem, q, plane.data(), whole.data());
    }
    std::fclose(f);
    if (!ok) return fail(ITLBM_E_PARSE, std::string("truncated case snapshot: ") + path);
    cudaError_t e = cudaMemcpy(state, whole.data(), whole.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();  // the copy has landed before any stream uses it
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "snapshot copy");
}

}  // namespace itlbm
