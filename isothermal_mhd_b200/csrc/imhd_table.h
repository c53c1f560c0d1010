// imhd_table.h -- host side of a box table: per-box block counts of every
// kernel decomposition, their prefixes, and the upload of the table.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "imhd_types.cuh"

namespace imhd {

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }
inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

inline bool row_capable(int nx, size_t esz) { return 13 * (size_t)nx * esz <= kRowSmemMax; }

inline int reduction_blocks(int n) {
    int b = ceil_div(n, kRedThreads);
    return b < kRedBlocksMax ? b : kRedBlocksMax;
}

// Blocks of box r for decomposition `kind`.
inline long blocks_of(const BoxRec& r, int kind, size_t esz) {
    const int tw = 1 << r.tws, th = kBX >> r.tws;
    long nbx = ceil_div(r.nx, tw), nby = ceil_div(r.ny, th), nbz = ceil_div(r.nz, th);
    if (kind == kKindCell) return nbx * nby * r.nz;
    if (kind == kKindCellZ) return nbx * nby * ceil_div(r.nz, 1 << r.segzs);
    if (kind == kKindRed) return r.nred;
    if (kind == kKindUpdTma) return r.nx % kTmaTile == 0 ? (long)(r.nx / kTmaTile) * r.ny * ceil_div(r.nz, kSegZ) : 0;
    if (kind == kKindUpdTma64)
        return (r.nx % kTmaTile != 0 && r.nx % (kTmaTile / 2) == 0 && r.ny % 2 == 0)
                   ? (long)(r.nx / (kTmaTile / 2)) * (r.ny / 2) * ceil_div(r.nz, kSegZ)
                   : 0;
    int scheme = 1 + (kind - kKindSolver0) / 5;
    int sub = (kind - kKindSolver0) % 5;
    if (scheme_of(box_solver(r), r.recon) != scheme) return 0;
    bool row = row_capable(r.nx, esz);
    switch (sub) {
        case kSubCell: return nbx * nby * ceil_div(r.nz, kSegZ);   // z columns of the predictor fluxes
        case kSubXRow: return row ? (long)r.ny * r.nz : 0;
        case kSubXTile: return row ? 0 : (long)ceil_div(r.nx, kTX) * r.ny * r.nz;
        case kSubMarchY: return nbx * nbz * ceil_div(r.ny, 1 << r.segs);   // (x, z) tiles marching along y
        default: return nbx * nby * ceil_div(r.nz, 1 << r.segs);           // (x, y) tiles marching along z
    }
}

// Prefix sums of every kind (kKinds rows of nbox+1 ints) and the launch
// parameters of the table.  Returns false when a launch would exceed the
// 2^31-1 block limit of a grid.
inline bool build_prefix(const std::vector<BoxRec>& recs, size_t esz, std::vector<int>& prefix, BatchDev& bd);

// Box of every block, per kind (for tables of more than one box).
inline void build_blk2box(const std::vector<int>& prefix, int nbox, const BatchDev& bd,
                          std::vector<std::vector<int>>& out) {
    out.assign(kKinds, std::vector<int>());
    for (int k = 0; k < kKinds; ++k) {
        out[k].resize((size_t)bd.totals[k]);
        for (int b = 0; b < nbox; ++b) {
            int lo = prefix[(size_t)k * (nbox + 1) + b], hi = prefix[(size_t)k * (nbox + 1) + b + 1];
            for (int i = lo; i < hi; ++i) out[k][(size_t)i] = b;
        }
    }
}

inline bool build_prefix(const std::vector<BoxRec>& recs, size_t esz, std::vector<int>& prefix, BatchDev& bd) {
    int nbox = (int)recs.size();
    prefix.assign((size_t)kKinds * (nbox + 1), 0);
    for (int k = 0; k < kKinds; ++k) {
        long acc = 0;
        for (int b = 0; b < nbox; ++b) {
            prefix[(size_t)k * (nbox + 1) + b] = (int)acc;
            acc += blocks_of(recs[b], k, esz);
            if (acc > 2147483647L) return false;
        }
        prefix[(size_t)k * (nbox + 1) + nbox] = (int)acc;
        bd.totals[k] = (int)acc;
    }
    bd.row_nx_max = 0;
    for (int s = 0; s <= kSchemes; ++s) bd.has_scheme[s] = false;
    bd.any_pass = false;
    bd.npass_max = 0;
    bd.any_zrange = false;
    bd.any_protect = false;
    for (const BoxRec& r : recs) {
        if (r.protect) bd.any_protect = true;
        if (r.riemann >= 1 && r.riemann <= 3 && r.recon >= 0 && r.recon < kRecons)
            bd.has_scheme[scheme_of(box_solver(r), r.recon)] = true;
        if (r.npass > 0) bd.any_pass = true;
        if (r.npass > bd.npass_max) bd.npass_max = r.npass;
        if (r.zlo != 0 || r.zhi != r.nz) bd.any_zrange = true;
        if (row_capable(r.nx, esz) && r.nx > bd.row_nx_max) bd.row_nx_max = r.nx;
    }
    bd.a.nbox = nbox;
    return true;
}

// Host side of a device table: block prefixes, block -> box lists and the
// device bytes of the whole table (records | prefix | one list per kind).
struct TablePlan {
    std::vector<int> prefix;
    std::vector<std::vector<int>> b2b;
    size_t bytes = 0;
};

inline bool plan_table(const std::vector<BoxRec>& recs, size_t esz, BatchDev& bd, TablePlan& tp) {
    if (!build_prefix(recs, esz, tp.prefix, bd)) return false;
    build_blk2box(tp.prefix, (int)recs.size(), bd, tp.b2b);
    tp.bytes = align256(sizeof(BoxRec) * recs.size()) + align256(tp.prefix.size() * sizeof(int));
    for (int k = 0; k < kKinds; ++k) tp.bytes += align256(tp.b2b[k].size() * sizeof(int) + 4);
    return true;
}

// Copy a planned table to `dev` (tp.bytes of device memory) and point the
// launch arguments at it.  The host vectors are pageable, so the copies are
// complete when this returns.
inline cudaError_t upload_table(void* dev, const std::vector<BoxRec>& recs, const TablePlan& tp, cudaStream_t st,
                                BatchArgs& a) {
    cudaError_t e = cudaMemcpyAsync(dev, recs.data(), sizeof(BoxRec) * recs.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    size_t off = align256(sizeof(BoxRec) * recs.size());
    e = cudaMemcpyAsync((char*)dev + off, tp.prefix.data(), tp.prefix.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    a.boxes = (BoxRec*)dev;
    a.prefix = (const int*)((char*)dev + off);
    off += align256(tp.prefix.size() * sizeof(int));
    for (int k = 0; k < kKinds; ++k) {
        if (!tp.b2b[k].empty()) {
            e = cudaMemcpyAsync((char*)dev + off, tp.b2b[k].data(), tp.b2b[k].size() * sizeof(int),
                                cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return e;
        }
        a.blk2box[k] = (const int*)((char*)dev + off);
        off += align256(tp.b2b[k].size() * sizeof(int) + 4);
    }
    a.nbox = (int)recs.size();
    a.use_one = 0;
    return cudaStreamSynchronize(st);
}

// Periodic ghost layers of a padded host field whose interior is filled
// (boundary_conditions_mod.f90:137-231 on the host side of the boundary).
inline void host_ghost_fill(int nx, int ny, int nz, double* h, int ng) {
    if (ng == 0) return;
    long Px = nx + 2 * ng, Py = ny + 2 * ng, Pz = nz + 2 * ng;
    auto wrap = [](long i, long n) { i %= n; return i < 0 ? i + n : i; };
    for (long k = 0; k < Pz; ++k)
        for (long j = 0; j < Py; ++j)
            for (long i = 0; i < Px; ++i) {
                bool in = i >= ng && i < ng + nx && j >= ng && j < ng + ny && k >= ng && k < ng + nz;
                if (in) continue;
                long ii = wrap(i - ng, nx) + ng, jj = wrap(j - ng, ny) + ng, kk = wrap(k - ng, nz) + ng;
                h[i + Px * (j + Py * k)] = h[ii + Px * (jj + Py * kk)];
            }
}

// Fill the geometry fields of a box record from its configuration.
inline void init_rec(BoxRec& r, int nx, int ny, int nz, int npass, int riemann, int recon, double cs, double cour,
                     double edot, double dt_turb, int protect = 0) {
    std::memset(&r, 0, sizeof(r));
    r.nx = nx; r.ny = ny; r.nz = nz; r.n = nx * ny * nz;
    r.npass = npass;
    r.riemann = riemann;
    r.recon = recon;
    r.protect = (riemann == 1 && protect) ? 1 : 0;   // protection fluxes exist for the Roe solver only
    r.zlo = 0;
    r.zhi = nz;
    // widest x tile that the row length divides (whole 128-byte segments per
    // warp, no idle threads), 32 when none does
    r.tws = (nx % 128 == 0) ? 7 : (nx % 64 == 0) ? 6 : 5;
    // y / z sweep segments: 32 faces per thread on long columns (measured at
    // 512^3: y 3.0 -> 2.9 ms, PPM 4.5 -> 4.3), 16 otherwise (more threads for
    // small boxes; batches tune this further)
    r.segs = (ny >= 256 && nz >= 256) ? kSegLog + 1 : kSegLog;
    r.segzs = kSegZLog;
    int pmax = ny * nz;
    if (nx * nz > pmax) pmax = nx * nz;
    if (nx * ny > pmax) pmax = nx * ny;
    r.plane_stride = pmax;
    r.nred = reduction_blocks(r.n);
    int nmax = nx > ny ? nx : ny;
    nmax = nmax > nz ? nmax : nz;
    r.dx = 1.0 / (double)nmax;                 // vanleer_mod.f90:177, driver.f90:254
    r.cs = cs;
    r.cour = cour;
    r.edot = edot;
    r.dt_turb = dt_turb;
    r.active = 1;
}

// Device bytes of one box's buffers (state x2, fluxes, EMFs, half-step
// scalars, boundary planes, partial sums, scalars), each 256-byte aligned.
// Capacity of a stage's bad-cell list under flux protection.
inline int prot_list_cap(int n) { return n < (1 << 20) ? n : (1 << 20); }
inline size_t box_bytes(const BoxRec& r, size_t esz, bool with_force) {
    size_t n = (size_t)r.n, nf = 10 + (size_t)r.npass;
    size_t b = 2 * align256(nf * n * esz) + align256(18 * n * esz) + align256(3 * n * esz);
    if (r.npass) b += align256((size_t)r.npass * n * esz) + align256(6 * (size_t)r.plane_stride * esz);
    if (with_force) b += align256(3 * n * esz);
    if (r.protect)
        b += align256(18 * n * esz) + align256(3 * n * esz) + align256(n) + align256(2 * (size_t)prot_list_cap(r.n) * 4);
    b += align256((size_t)r.nred * 6 * 8) + align256(sizeof(Scalars));
    return b;
}
// Carve the buffers of one box out of `base` (box_bytes of space).
inline void carve_box(BoxRec& r, unsigned char* base, size_t esz, bool with_force) {
    size_t n = (size_t)r.n, nf = 10 + (size_t)r.npass;
    unsigned char* p = base;
    r.S[0] = p; p += align256(nf * n * esz);
    r.S[1] = p; p += align256(nf * n * esz);
    r.F = p; p += align256(18 * n * esz);
    r.E = p; p += align256(3 * n * esz);
    if (r.npass) {
        r.SH = p; p += align256((size_t)r.npass * n * esz);
        r.mbnd = p; p += align256(6 * (size_t)r.plane_stride * esz);
    } else {
        r.SH = nullptr; r.mbnd = nullptr;
    }
    if (with_force) { r.delv = p; p += align256(3 * n * esz); } else r.delv = nullptr;
    if (r.protect) {   // the bad flags must start at zero: the whole pool is cleared after carving
        r.Fp = p; p += align256(18 * n * esz);
        r.Ep = p; p += align256(3 * n * esz);
        r.bad = p; p += align256(n);
        r.badcap = prot_list_cap(r.n);
        r.badlist = (int*)p; p += align256(2 * (size_t)r.badcap * 4);
    } else {
        r.Fp = r.Ep = nullptr; r.bad = nullptr; r.badlist = nullptr; r.badcap = 0;
    }
    r.partials = (double*)p; p += align256((size_t)r.nred * 6 * 8);
    r.sc = (Scalars*)p;
}

}  // namespace imhd
