// itlbm_snapshot.cu -- saving and restoring the state of a case (host side).
//
// The reference restarts an interrupted batch from step 0 (rodar_lote.py:5-7).  A snapshot holds a
// case's description, its step count and its populations at the top of its next step, in its own
// precision and storage form (FP64 f_R, f_B or FP32 e, d), planes of nx * ny elements in plain rows.
// The host converts them from and to the tile-major device buffer one tile row (8 box rows) at a time,
// so a snapshot needs host memory for one tile row, not for the state.  Stepping a restored case gives
// the same bits the saved run would have given.
#include "itlbm_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace itlbm {

namespace {

constexpr char MAGIC[8] = {'I', 'T', 'L', 'B', 'M', 'S', 'T', '1'};

// The state buffer is moved one tile row at a time: tile row ty (box rows 8 ty .. 8 ty + 7, every
// plane) is one contiguous range of tiles_x * tile_elems elements.  Plane q of its rows to and from
// the file's plain rows of nx elements.
void unblock_band(const CaseDev &h, size_t elem, int q, int nrows, const unsigned char *band, unsigned char *rows) {
    for (int r = 0; r < nrows; r++)
        for (int x0 = 0; x0 < h.nx; x0 += TX) {
            const size_t n = (size_t)std::min(TX, h.nx - x0) * elem;
            const size_t o = (size_t)(x0 / TX) * h.tile_elems + (size_t)q * PLANE + (size_t)r * TX;
            std::memcpy(rows + ((size_t)r * h.nx + x0) * elem, band + o * elem, n);
        }
}
void reblock_band(const CaseDev &h, size_t elem, int q, int nrows, const unsigned char *rows, unsigned char *band) {
    for (int r = 0; r < nrows; r++)
        for (int x0 = 0; x0 < h.nx; x0 += TX) {
            const size_t n = (size_t)std::min(TX, h.nx - x0) * elem;
            const size_t o = (size_t)(x0 / TX) * h.tile_elems + (size_t)q * PLANE + (size_t)r * TX;
            std::memcpy(band + o * elem, rows + ((size_t)r * h.nx + x0) * elem, n);
        }
}
// File offset of row y of plane q.
off_t row_at(const CaseDev &h, size_t elem, int q, int y) {
    return (off_t)sizeof(SnapHeader) + (off_t)(((long long)q * h.ny + y) * h.nx) * (off_t)elem;
}

}  // namespace

int snap_write(const char *path, const itlbm_case_desc &d, long long steps, const CaseDev &h, const void *state) {
    SnapHeader hd{};
    std::memcpy(hd.magic, MAGIC, 8);
    hd.version = 2;  // 2: FP32 states are deviations from the equilibrium at the case's initial flow
    hd.desc = d;
    hd.steps = steps;
    const size_t elem = elem_of(h.prec);
    const size_t band_elems = (size_t)h.tiles_x * h.tile_elems;
    std::vector<unsigned char> band(elem * band_elems), rows(elem * (size_t)h.nx * TY);
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ITLBM_E_IO, std::string("cannot write ") + path);
    bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1;
    for (int y0 = 0; ok && y0 < h.ny; y0 += TY) {
        const unsigned char *src = (const unsigned char *)state + (size_t)(y0 / TY) * band_elems * elem;
        const cudaError_t e = cudaMemcpy(band.data(), src, band.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            std::fclose(f);
            return cuda_fail(e, "snapshot copy");
        }
        const int nrows = std::min(TY, h.ny - y0);
        for (int q = 0; ok && q < 2 * planes_of(h.prec); q++) {
            unblock_band(h, elem, q, nrows, band.data(), rows.data());
            const size_t n = elem * (size_t)nrows * h.nx;
            ok = fseeko(f, row_at(h, elem, q, y0), SEEK_SET) == 0 && std::fwrite(rows.data(), 1, n, f) == n;
        }
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
    const size_t band_elems = (size_t)h.tiles_x * h.tile_elems;
    std::vector<unsigned char> band(elem * band_elems, 0), rows(elem * (size_t)h.nx * TY);
    bool ok = true;
    cudaError_t e = cudaSuccess;
    for (int y0 = 0; ok && e == cudaSuccess && y0 < h.ny; y0 += TY) {
        const int nrows = std::min(TY, h.ny - y0);
        for (int q = 0; ok && q < 2 * planes_of(h.prec); q++) {
            const size_t n = elem * (size_t)nrows * h.nx;
            ok = fseeko(f, row_at(h, elem, q, y0), SEEK_SET) == 0 && std::fread(rows.data(), 1, n, f) == n;
            if (ok) reblock_band(h, elem, q, nrows, rows.data(), band.data());
        }
        // synchronous: the band buffer is refilled for the next tile row
        if (ok) e = cudaMemcpy((unsigned char *)state + (size_t)(y0 / TY) * band_elems * elem, band.data(), band.size(),
                               cudaMemcpyHostToDevice);
    }
    std::fclose(f);
    if (!ok) return fail(ITLBM_E_PARSE, std::string("truncated case snapshot: ") + path);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();  // the copies have landed before any stream uses them
    return e == cudaSuccess ? ITLBM_OK : cuda_fail(e, "snapshot copy");
}

}  // namespace itlbm
