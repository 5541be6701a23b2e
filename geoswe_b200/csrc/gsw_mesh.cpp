// gsw_mesh.cpp -- compressed-mesh construction on the host (C++).
//
// Two layouts of the same stored cell set:
//
// 1. The reference's canonical tables (geoswe/compressed_mesh.py:112-187,
//    geoswe/compressed_rhs.py:194-349), bit for bit: stored = the inside mask dilated
//    `ring` times with the 4-neighbour cross (scipy.ndimage.binary_dilation's default
//    structure, out-of-grid = False); ids row-major with j fastest; neighbours in the
//    order E(+i), W(-i), N(+j), S(-j) as int16 deltas id = k + delta, -32768 = none;
//    is_active = inside at the stored cells; the coverage check of CompressedSWE._verify.
//
// 2. The execution layout of the flat kernels: the padded grid is cut into bricks of
//    GSW_BRICK_W (30) columns x brick_h rows, every brick holding a stored cell is kept,
//    bricks are ordered along a Hilbert curve of their (row, column) index, and each is
//    stored as brick_h rows of GSW_BRICK_PITCH (32) slots. A warp steps one brick down its
//    rows with the column march of the dense kernel: lanes 1..30 are the brick's columns,
//    lanes 0 and 31 read the neighbouring bricks' edge columns, and the rows above and
//    below come from the bricks above and below (brick index `n_bricks` is an all-zero
//    brick that stands for a missing neighbour). Neighbours inside a brick are plain
//    arithmetic; only the four brick links are tables.
#include <stdint.h>
#include <string.h>
#include <stdio.h>
#include <stdarg.h>
#include <vector>
#include <algorithm>
#include "../../include/gsw.h"

namespace gsw_rt { int set_error(int code, const char* fmt, ...); }
using gsw_rt::set_error;

namespace {

// stored = inside dilated `ring` times with the cross; border treated as False.
std::vector<uint8_t> dilate(const uint8_t* inside, int nx, int ny, int ring) {
    std::vector<uint8_t> a(inside, inside + (size_t)nx * ny), b((size_t)nx * ny);
    for (size_t k = 0; k < a.size(); ++k) a[k] = a[k] ? 1 : 0;
    for (int it = 0; it < ring; ++it) {
        for (int i = 0; i < nx; ++i) {
            const uint8_t* r = &a[(size_t)i * ny];
            uint8_t* o = &b[(size_t)i * ny];
            for (int j = 0; j < ny; ++j) {
                uint8_t v = r[j];
                if (!v && j > 0) v = r[j - 1];
                if (!v && j + 1 < ny) v = r[j + 1];
                if (!v && i > 0) v = a[(size_t)(i - 1) * ny + j];
                if (!v && i + 1 < nx) v = a[(size_t)(i + 1) * ny + j];
                o[j] = v;
            }
        }
        a.swap(b);
    }
    return a;
}

// Hilbert index of (x, y) on a 2^order square (the classic rotate-and-reflect walk).
uint64_t hilbert(uint32_t x, uint32_t y, int order) {
    uint64_t d = 0;
    for (uint32_t s = 1u << (order - 1); s > 0; s >>= 1) {
        const uint32_t rx = (x & s) ? 1u : 0u;
        const uint32_t ry = (y & s) ? 1u : 0u;
        d += (uint64_t)s * s * ((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) { x = s - 1 - x; y = s - 1 - y; }
            const uint32_t t = x; x = y; y = t;
        }
    }
    return d;
}

}  // namespace

extern "C" GSW_API int gsw_mesh_count(const uint8_t* inside, int nxp, int nyp, int ring,
                                      int64_t* n_stored, int64_t* n_active) {
    if (!inside || nxp <= 0 || nyp <= 0 || ring < 0 || !n_stored || !n_active)
        return set_error(GSW_ERR_INVALID, "mesh_count: bad arguments");
    std::vector<uint8_t> st = dilate(inside, nxp, nyp, ring);
    int64_t ns = 0, na = 0;
    for (size_t k = 0; k < st.size(); ++k) { ns += st[k]; na += inside[k] ? 1 : 0; }
    *n_stored = ns;
    *n_active = na;
    return GSW_OK;
}

// Canonical tables of geoswe's CompressedSWE. Any output pointer may be NULL.
//   ij         (N, 2) int32 padded (i, j) of each stored cell
//   nbr16      (N, 4) int16 deltas E, W, N, S
//   is_active  (N)    uint8
//   active_id  (nxp*nyp) int32, -1 where not stored
//   covered    1 when every active cell has its +-1 and +-2 neighbours stored
extern "C" GSW_API int gsw_mesh_build(const uint8_t* inside, int nxp, int nyp, int ring, int32_t* ij,
                                      int16_t* nbr16, uint8_t* is_active, int32_t* active_id,
                                      int32_t* covered) {
    if (!inside || nxp <= 0 || nyp <= 0 || ring < 0)
        return set_error(GSW_ERR_INVALID, "mesh_build: bad arguments");
    std::vector<uint8_t> st = dilate(inside, nxp, nyp, ring);
    const size_t P = (size_t)nxp * nyp;
    std::vector<int64_t> id(P, -1);
    int64_t N = 0;
    for (size_t k = 0; k < P; ++k)
        if (st[k]) id[k] = N++;
    if (N >= (int64_t)1 << 31) return set_error(GSW_ERR_RANGE, "mesh_build: %lld stored cells exceed int32", (long long)N);
    auto at = [&](int i, int j) -> int64_t {
        if (i < 0 || i >= nxp || j < 0 || j >= nyp) return -1;
        return id[(size_t)i * nyp + j];
    };
    // delta range first (the reference refuses before writing the table)
    int64_t worst = 0;
    static const int DI[4] = {1, -1, 0, 0}, DJ[4] = {0, 0, 1, -1};
    for (int i = 0; i < nxp; ++i)
        for (int j = 0; j < nyp; ++j) {
            const int64_t k = id[(size_t)i * nyp + j];
            if (k < 0) continue;
            for (int d = 0; d < 4; ++d) {
                const int64_t n = at(i + DI[d], j + DJ[d]);
                if (n >= 0) worst = std::max<int64_t>(worst, n > k ? n - k : k - n);
            }
        }
    if (worst >= 32768)
        return set_error(GSW_ERR_RANGE,
                         "neighbour delta %lld is outside int16: a stored row spans more than 32768 cells "
                         "(the flat table is int16, as in the reference); split the domain along y", (long long)worst);
    int ok1 = 1, ok2 = 1;
    for (int i = 0; i < nxp; ++i)
        for (int j = 0; j < nyp; ++j) {
            const int64_t k = id[(size_t)i * nyp + j];
            if (k < 0) continue;
            if (ij) { ij[2 * k] = i; ij[2 * k + 1] = j; }
            const bool act = inside[(size_t)i * nyp + j] != 0;
            if (is_active) is_active[k] = act ? 1 : 0;
            for (int d = 0; d < 4; ++d) {
                const int64_t n = at(i + DI[d], j + DJ[d]);
                if (nbr16) nbr16[4 * k + d] = (int16_t)(n >= 0 ? n - k : -32768);
                if (act) {
                    if (n < 0) ok1 = 0;
                    else if (at(i + 2 * DI[d], j + 2 * DJ[d]) < 0) ok2 = 0;
                }
            }
        }
    if (active_id)
        for (size_t k = 0; k < P; ++k) active_id[k] = (int32_t)id[k];
    if (covered) *covered = ok1 && ok2;
    return GSW_OK;
}

// Brick layout. Pass 1 (brick_ij == NULL) returns the brick count in *n_bricks; pass 2
// fills brick_ij (nb, 2) [brick row, brick column] in Hilbert order and brick_nbr (nb, 4)
// [up, down, left, right] (n_bricks for a missing neighbour).
extern "C" GSW_API int gsw_bricks_build(const uint8_t* stored, int nxp, int nyp, int brick_h,
                                        int64_t* n_bricks, int32_t* brick_ij, int32_t* brick_nbr) {
    if (!stored || nxp <= 0 || nyp <= 0 || brick_h < 2 || !n_bricks)
        return set_error(GSW_ERR_INVALID, "bricks_build: bad arguments (brick_h >= 2)");
    const int BI = (nxp + brick_h - 1) / brick_h, BJ = (nyp + GSW_BRICK_W - 1) / GSW_BRICK_W;
    std::vector<uint8_t> has((size_t)BI * BJ, 0);
    for (int i = 0; i < nxp; ++i)
        for (int j = 0; j < nyp; ++j)
            if (stored[(size_t)i * nyp + j]) has[(size_t)(i / brick_h) * BJ + j / GSW_BRICK_W] = 1;
    std::vector<std::pair<uint64_t, int64_t>> keys;
    int order = 1;
    while ((1 << order) < std::max(BI, BJ)) ++order;
    for (int a = 0; a < BI; ++a)
        for (int c = 0; c < BJ; ++c)
            if (has[(size_t)a * BJ + c]) keys.push_back({hilbert((uint32_t)a, (uint32_t)c, order), (int64_t)a * BJ + c});
    const int64_t nb = (int64_t)keys.size();
    if (!brick_ij) { *n_bricks = nb; return GSW_OK; }
    if (*n_bricks != nb) return set_error(GSW_ERR_INVALID, "bricks_build: n_bricks %lld != %lld",
                                          (long long)*n_bricks, (long long)nb);
    std::sort(keys.begin(), keys.end());
    std::vector<int64_t> bid((size_t)BI * BJ, nb);
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t lin = keys[b].second;
        bid[lin] = b;
        brick_ij[2 * b] = (int32_t)(lin / BJ);
        brick_ij[2 * b + 1] = (int32_t)(lin % BJ);
    }
    if (brick_nbr)
        for (int64_t b = 0; b < nb; ++b) {
            const int a = brick_ij[2 * b], c = brick_ij[2 * b + 1];
            brick_nbr[4 * b + 0] = (int32_t)(a > 0 ? bid[(size_t)(a - 1) * BJ + c] : nb);
            brick_nbr[4 * b + 1] = (int32_t)(a + 1 < BI ? bid[(size_t)(a + 1) * BJ + c] : nb);
            brick_nbr[4 * b + 2] = (int32_t)(c > 0 ? bid[(size_t)a * BJ + c - 1] : nb);
            brick_nbr[4 * b + 3] = (int32_t)(c + 1 < BJ ? bid[(size_t)a * BJ + c + 1] : nb);
        }
    return GSW_OK;
}

// The brick slot of every canonical cell: slot = brick * brick_h * GSW_BRICK_PITCH +
// (i mod brick_h) * GSW_BRICK_PITCH + (j mod GSW_BRICK_W) for the brick at
// (i / brick_h, j / GSW_BRICK_W). A host other than this package's Python side needs
// this map to place the reference's canonical flat arrays into brick storage and back.
extern "C" GSW_API int gsw_bricks_slot_of(const int32_t* ij, int64_t n_cells, const int32_t* brick_ij,
                                          int64_t n_bricks, int brick_h, int nxp, int nyp, int64_t* slot_of) {
    if (!ij || !brick_ij || !slot_of || n_cells < 0 || n_bricks < 0 || brick_h < 2 || nxp <= 0 || nyp <= 0)
        return set_error(GSW_ERR_INVALID, "bricks_slot_of: bad arguments");
    const int BI = (nxp + brick_h - 1) / brick_h, BJ = (nyp + GSW_BRICK_W - 1) / GSW_BRICK_W;
    std::vector<int64_t> bid((size_t)BI * BJ, -1);
    for (int64_t b = 0; b < n_bricks; ++b) {
        const int a = brick_ij[2 * b], c = brick_ij[2 * b + 1];
        if (a < 0 || a >= BI || c < 0 || c >= BJ) return set_error(GSW_ERR_INVALID, "bricks_slot_of: brick %lld "
                                                                     "outside the grid", (long long)b);
        bid[(size_t)a * BJ + c] = b;
    }
    const int64_t BS = (int64_t)brick_h * GSW_BRICK_PITCH;
    for (int64_t k = 0; k < n_cells; ++k) {
        const int i = ij[2 * k], j = ij[2 * k + 1];
        if (i < 0 || i >= nxp || j < 0 || j >= nyp) return set_error(GSW_ERR_INVALID, "bricks_slot_of: cell %lld "
                                                                     "outside the grid", (long long)k);
        const int64_t b = bid[(size_t)(i / brick_h) * BJ + j / GSW_BRICK_W];
        if (b < 0) return set_error(GSW_ERR_INVALID, "bricks_slot_of: cell %lld has no brick", (long long)k);
        slot_of[k] = b * BS + (int64_t)(i % brick_h) * GSW_BRICK_PITCH + (j % GSW_BRICK_W);
    }
    return GSW_OK;
}
