// imhd_kernels.cuh -- CUDA kernels of one isothermal-MHD van Leer + CT step on
// a periodic box, templated on the arithmetic type (float / double).
//
// Data layout in HBM (one box): structure of arrays, x fastest, no ghost
// cells; the reference's nb-wide ghost zones (grid_data_mod.f90:38-43) become
// an index wrap.  A state buffer holds 10 + npass fields of N = nx*ny*nz:
//   0 rho, 1..3 momentum, 4..6 cell-centred B, 7..9 face B (x at i+1/2,
//   y at j+1/2, z at k+1/2, as bface_3d), 10.. passive scalars.
// Flux buffer: 18 fields, F[6*D + c] with c in the rotated order
// (rho, m_n, m_t1, m_t2, B_t1, B_t2) of sweep D, stored at the cell left of
// the face.  Corner EMF buffer: Ex(i,j+1/2,k+1/2), Ey(i+1/2,j,k+1/2),
// Ez(i+1/2,j+1/2,k), as emf_corner (vanleer_mod.f90:1868-1882).
//
// Because periodic ghost cells are exact images of interior cells, every
// flux, EMF and update the reference computes in its padded arrays is either
// computed here for the interior cell it images or is not needed by interior
// cells; interior results and the smax reduction are therefore identical.
// One exception is replicated explicitly: on drive steps the reference
// applies the forcing kick to interior cells only (turb_driver_mod.f90:437-453)
// and then builds the passive-scalar advection velocity from its ghost cells
// (passive_mod.f90:227-239), so the face velocity at the global boundary sees
// the unforced momentum of the ghost side (k_passive_corr below).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "imhd_physics_fast.cuh"
#include "imhd_types.cuh"

namespace imhd {

struct Dims {
    int nx, ny, nz;
    int n;        // nx*ny*nz (< 2^31)
};

// Box of the current block and the block's index within that box.  ONE: the
// launch covers a single box whose record is a kernel parameter (read from
// the constant bank, no dependent loads); otherwise the block looks its box up
// in the device table.
template <bool ONE>
__device__ __forceinline__ BoxRec resolve(const BatchArgs& ba, int kind, int& local) {
    if constexpr (ONE) {
        local = (int)blockIdx.x;
        return ba.one;
    } else {
        int b = __ldg(ba.blk2box[kind] + blockIdx.x);
        local = (int)blockIdx.x - __ldg(ba.prefix + kind * (ba.nbox + 1) + b);
        return ba.boxes[b];
    }
}
// Box b of the table (the kernels that run one thread or block per box).
__device__ __forceinline__ BoxRec box_at(const BatchArgs& ba, int b) { return ba.use_one ? ba.one : ba.boxes[b]; }
__device__ __forceinline__ Dims dims_of(const BoxRec& r) { return Dims{r.nx, r.ny, r.nz, r.n}; }
// kKindCell decomposition: (x, y) tiles of (1 << tws) x (kBX >> tws)
// threads per z plane (a single box launches the 3D grid (nbx, nby, nz) and
// needs no division).  j may exceed ny - 1 in the last tile row: callers test
// i < nx and j < ny.
template <bool ONE>
__device__ __forceinline__ void decode_cell(int local, const Dims& dm, int tws, int& i, int& j, int& k) {
    const int tw = 1 << tws, th = kBX >> tws;
    const int lx = (int)threadIdx.x & (tw - 1), ly = (int)threadIdx.x >> tws;
    if constexpr (ONE) {
        i = (int)blockIdx.x * tw + lx;
        j = (int)blockIdx.y * th + ly;
        k = (int)blockIdx.z;
    } else {
        int nbx = (dm.nx + tw - 1) >> tws, nby = (dm.ny + th - 1) / th;
        int bx = local % nbx, rest = local / nbx;
        i = bx * tw + lx;
        j = (rest % nby) * th + ly;
        k = rest / nby;
    }
}

// kKindCellZ decomposition: the same tiles per z segment of kSegZ planes
// (a compile-time length: the unrolled z loops are measurably faster with
// it); the thread's column is k0 <= k < k1 (a single box launches a 3D grid
// (nbx, nby, nseg)).
// Callers test i < nx and j < ny.
template <bool ONE>
__device__ __forceinline__ void decode_cellz(int local, const Dims& dm, int tws, int segzs, int& i, int& j, int& k0,
                                             int& k1) {
    const int tw = 1 << tws, th = kBX >> tws;
    const int lx = (int)threadIdx.x & (tw - 1), ly = (int)threadIdx.x >> tws;
    int seg;
    if constexpr (ONE) {
        i = (int)blockIdx.x * tw + lx;
        j = (int)blockIdx.y * th + ly;
        seg = (int)blockIdx.z;
    } else {
        int nbx = (dm.nx + tw - 1) >> tws, nby = (dm.ny + th - 1) / th;
        int bx = local % nbx, rest = local / nbx;
        i = bx * tw + lx;
        j = (rest % nby) * th + ly;
        seg = rest / nby;
    }
    (void)segzs;
    k0 = seg * kSegZ;
    k1 = min(k0 + kSegZ, dm.nz);
}

__device__ __forceinline__ int wrap_up(int i, int n) { return (i + 1 == n) ? 0 : i + 1; }
__device__ __forceinline__ int wrap_dn(int i, int n) { return (i == 0) ? n - 1 : i - 1; }
__device__ __forceinline__ int wrap_any(int i, int n) { i %= n; return i < 0 ? i + n : i; }

template <class T>
__device__ __forceinline__ const T* fld(const T* S, int f, int n) { return S + (size_t)f * (size_t)n; }
template <class T>
__device__ __forceinline__ T* fld(T* S, int f, int n) { return S + (size_t)f * (size_t)n; }

// max that keeps a NaN (speeds are otherwise >= 0, so the order of a max
// reduction does not change its value)
__device__ __forceinline__ double nmax(double a, double b) { return (a != a || a > b) ? a : b; }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Block-wide max folded into slots[block id mod kSlots] with one atomicMax on
// the bit pattern (NaN bits exceed every finite non-negative double).  Every
// thread of the block must call it (it synchronises the block).
template <int NT>
__device__ __forceinline__ void block_atomic_max(unsigned long long* slots, double v) {
    __shared__ double red[NT / 32];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) m = nmax(m, red[w]);
        unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        if (!(m <= 0.0)) atomicMax(&slots[bid % kSlots], (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

// Same as block_atomic_max for any blockDim.x that is a multiple of 32.
__device__ __forceinline__ void block_atomic_max_any(unsigned long long* slots, double v) {
    __shared__ double red[32];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        int nw = (int)(blockDim.x >> 5);
        for (int w = 1; w < nw; ++w) m = nmax(m, red[w]);
        unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        if (!(m <= 0.0)) atomicMax(&slots[bid % kSlots], (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
}

// rotated field indices of sweep D (vanleer_mod.f90:443-461, 605-630, 784-806)
template <int D> struct Rot {
    static constexpr int MN = 1 + D, MT1 = 1 + (D + 1) % 3, MT2 = 1 + (D + 2) % 3;
    static constexpr int BT1 = 4 + (D + 1) % 3, BT2 = 4 + (D + 2) % 3, BN = 7 + D;
};

// ============================================================ predictor flux
// First-order interface fluxes (compute_{x,y,z}fluxes_3d with
// corrector_stage = .FALSE., vanleer_mod.f90:441-478): left/right states are
// the cell values, the normal field the face value.  One kernel computes the
// three faces x+1/2, y+1/2, z+1/2 of every cell: a thread walks a column of
// kSegZ cells along z and carries the cell above (its z neighbour) into the
// next plane, so the cell state is read once for all three sweeps.
template <class T>
struct CellQ {
    T q[10];      // rho, mx, my, mz, Bx_cc, By_cc, Bz_cc, Bx_face, By_face, Bz_face
};
template <class T, int NF>
__device__ __forceinline__ void load_cell(const T* __restrict__ S, int n, int c, CellQ<T>& a) {
#pragma unroll
    for (int f = 0; f < NF; ++f) a.q[f] = fld(S, f, n)[c];
}
// rotated conserved state of sweep D (vanleer_mod.f90:443-461, 605-630,
// 784-806); the normal field is the face value of the left cell
template <class T, int D>
__device__ __forceinline__ void rotated(const CellQ<T>& a, T bn, T* u) {
    using R = Rot<D>;
    u[0] = a.q[0];
    u[1] = a.q[R::MN];
    u[2] = a.q[R::MT1];
    u[3] = a.q[R::MT2];
    u[4] = bn;
    u[5] = a.q[R::BT1];
    u[6] = a.q[R::BT2];
}

// Solver 4 (Roe with flux_protection, vanleer_mod.f90:81): the HLLE flux of
// the same interface states into the protection buffer Fp, and the HLLE
// wave speeds into smax, as the reference's extra compute_HLLE_fluxes_1d
// call does (:540, 703, 880, 2962).  Nothing for the other solvers.
template <class T, int SOLVER>
__device__ __forceinline__ void protection_flux(const T* uL, const T* uR, T cs, T asqr, T& smax, void* Fp, int D, int n,
                                                int c) {
    if constexpr (SOLVER == 4) {
        T Fh[7];
        riemann_flux<3>(uL, uR, cs, asqr, Fh, smax);
        T* Fd = (T*)Fp + (size_t)(6 * D) * n;
        Fd[c] = Fh[0];
        Fd[(size_t)n + c] = Fh[1];
        Fd[2 * (size_t)n + c] = Fh[2];
        Fd[3 * (size_t)n + c] = Fh[3];
        Fd[4 * (size_t)n + c] = Fh[5];
        Fd[5 * (size_t)n + c] = Fh[6];
    }
}

// FP32 occupancy, measured at 512^3: five blocks per SM for the Roe solver
// (96 registers; fewer registers spill more than the extra warps return), six
// for HLLD and HLLE (80 registers, 3.9 -> 3.7 ms).
template <class T, int SCHEME, bool ONE>
__global__ void __launch_bounds__(kBX, sizeof(T) == 4 ? (scheme_solver(SCHEME) % 3 == 1 ? 5 : 6) : 1)
k_pred_flux(BatchArgs ba) {
    constexpr int SOLVER = scheme_solver(SCHEME);
    int local;
    const BoxRec rp = resolve<ONE>(ba, scheme_kind(SCHEME, kSubCell), local);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[0];
    T* __restrict__ F = (T*)rp.F;
    const T cs = (T)rp.cs, asqr = (T)(rp.cs * rp.cs);
    unsigned long long* smax_slots = sc->smax_slots;
    int i, j, k0, k1;
    decode_cellz<ONE>(local, dm, rp.tws, rp.segzs, i, j, k0, k1);
    const bool valid = i < dm.nx && j < dm.ny;
    T smax = T(0);
    if (valid) {
        const int n = dm.n;
        const int plane = dm.nx * dm.ny;
        const int r0 = i + dm.nx * j;
        const int rx = wrap_up(i, dm.nx) + dm.nx * j, ry = i + dm.nx * wrap_up(j, dm.ny);
        CellQ<T> cur;
        load_cell<T, 10>(S, n, r0 + k0 * plane, cur);
        for (int k = k0; k < k1; ++k) {
            const int kp = k * plane;
            const int c = r0 + kp;
            CellQ<T> xn, yn, zn;
            load_cell<T, 7>(S, n, rx + kp, xn);
            load_cell<T, 7>(S, n, ry + kp, yn);
            load_cell<T, 10>(S, n, r0 + wrap_up(k, dm.nz) * plane, zn);
            T sdrop = T(0);     // faces outside zlo..zhi-1 do not enter smax
            T& sref = (k >= rp.zlo && k < rp.zhi) ? smax : sdrop;
            T uL[7], uR[7], Fo[7];
            // x face
            rotated<T, 0>(cur, cur.q[7], uL);
            rotated<T, 0>(xn, cur.q[7], uR);
            riemann_flux<SOLVER>(uL, uR, cs, asqr, Fo, sref);
            {
                T* Fd = F;
                Fd[c] = Fo[0]; Fd[(size_t)n + c] = Fo[1]; Fd[2 * (size_t)n + c] = Fo[2];
                Fd[3 * (size_t)n + c] = Fo[3]; Fd[4 * (size_t)n + c] = Fo[5]; Fd[5 * (size_t)n + c] = Fo[6];
            }
            protection_flux<T, SOLVER>(uL, uR, cs, asqr, sref, rp.Fp, 0, n, c);
            // y face
            rotated<T, 1>(cur, cur.q[8], uL);
            rotated<T, 1>(yn, cur.q[8], uR);
            riemann_flux<SOLVER>(uL, uR, cs, asqr, Fo, sref);
            {
                T* Fd = F + (size_t)6 * n;
                Fd[c] = Fo[0]; Fd[(size_t)n + c] = Fo[1]; Fd[2 * (size_t)n + c] = Fo[2];
                Fd[3 * (size_t)n + c] = Fo[3]; Fd[4 * (size_t)n + c] = Fo[5]; Fd[5 * (size_t)n + c] = Fo[6];
            }
            protection_flux<T, SOLVER>(uL, uR, cs, asqr, sref, rp.Fp, 1, n, c);
            // z face
            rotated<T, 2>(cur, cur.q[9], uL);
            rotated<T, 2>(zn, cur.q[9], uR);
            riemann_flux<SOLVER>(uL, uR, cs, asqr, Fo, sref);
            {
                T* Fd = F + (size_t)12 * n;
                Fd[c] = Fo[0]; Fd[(size_t)n + c] = Fo[1]; Fd[2 * (size_t)n + c] = Fo[2];
                Fd[3 * (size_t)n + c] = Fo[3]; Fd[4 * (size_t)n + c] = Fo[5]; Fd[5 * (size_t)n + c] = Fo[6];
            }
            protection_flux<T, SOLVER>(uL, uR, cs, asqr, sref, rp.Fp, 2, n, c);
            cur = zn;
        }
    }
    block_atomic_max<kBX>(smax_slots, (double)smax);
}

// ============================================================ corrector flux
// Primitive variables of a cell in the rotated frame of sweep D
// (vanleer_mod.f90:483-496): rho, v_n, v_t1, v_t2, B_t1, B_t2.
template <class T, int D>
__device__ __forceinline__ void load_prim(const T* __restrict__ S, int n, int c, T* w, T& bn) {
    using R = Rot<D>;
    T rho = fld(S, 0, n)[c];
    T irho = T(1) / rho;
    w[0] = rho;
    w[1] = fld(S, R::MN, n)[c] * irho;
    w[2] = fld(S, R::MT1, n)[c] * irho;
    w[3] = fld(S, R::MT2, n)[c] * irho;
    w[4] = fld(S, R::BT1, n)[c];
    w[5] = fld(S, R::BT2, n)[c];
    bn = fld(S, R::BN, n)[c];
}

template <class T>
__device__ __forceinline__ void store_flux(T* __restrict__ F, int D, int n, int c, const T* Fo) {
    T* Fd = F + (size_t)(6 * D) * n;
    Fd[c] = Fo[0];
    Fd[(size_t)n + c] = Fo[1];
    Fd[2 * (size_t)n + c] = Fo[2];
    Fd[3 * (size_t)n + c] = Fo[3];
    Fd[4 * (size_t)n + c] = Fo[5];
    Fd[5 * (size_t)n + c] = Fo[6];
}

// Sweeps along y (D=1) and z (D=2): one thread per (x, transverse) column
// marches along the sweep direction over a segment of faces.  PLM keeps the
// primitive window w(a-1..a+2) and the slopes delw(a), delw(a+1) in
// registers; PPM keeps w(a..a+3), the slopes delw(a), delw(a+1) and the right
// edge of cell a.  Loads stay coalesced along x.
// FP32: six blocks per SM (80 registers, a few spills): the z sweep had run
// four blocks at 104 registers; 3.4 -> 3.1 ms (Roe, PLM) at 512^3.
template <class T, int SCHEME, int D, bool ONE>
__global__ void __launch_bounds__(kBX, sizeof(T) == 4 ? 6 : 1) k_corr_flux_march(BatchArgs ba) {
    constexpr int SOLVER = scheme_solver(SCHEME);
    constexpr int RECON = scheme_recon(SCHEME);
    constexpr bool PPM = (RECON & 1) != 0, PRIM = (RECON & 2) != 0;
    int local;
    const BoxRec rp = resolve<ONE>(ba, scheme_kind(SCHEME, D == 1 ? kSubMarchY : kSubMarchZ), local);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[1];   // half-step state
    T* __restrict__ F = (T*)rp.F;
    const T cs = (T)rp.cs, asqr = (T)(rp.cs * rp.cs);
    unsigned long long* smax_slots = sc->smax_slots;
    const int seg = 1 << rp.segs;
    // (x, other) tiles of the box's shape, other = z for D=1 and y for D=2
    const int nother = (D == 1) ? dm.nz : dm.ny;
    const int tw = 1 << rp.tws, th = kBX >> rp.tws;
    int bx, bo, a0;
    if constexpr (ONE) {                        // grid (nbx, nbo, nseg)
        bx = (int)blockIdx.x; bo = (int)blockIdx.y; a0 = (int)blockIdx.z * seg;
    } else {
        int nbx = (dm.nx + tw - 1) >> rp.tws, nbo = (nother + th - 1) / th;
        int rest = local / nbx;
        bx = local % nbx;
        bo = rest % nbo;
        a0 = (rest / nbo) * seg;
    }
    const int i = bx * tw + ((int)threadIdx.x & (tw - 1));
    const int o = bo * th + ((int)threadIdx.x >> rp.tws);   // k for D=1, j for D=2
    int na = (D == 1) ? dm.ny : dm.nz;
    int a1 = min(a0 + seg, na);
    bool valid = i < dm.nx && o < nother;
    T smax = T(0);
    if (valid) {
        int stride = (D == 1) ? dm.nx : dm.nx * dm.ny;
        int base = (D == 1) ? i + dm.nx * dm.ny * o : i + dm.nx * o;
        if constexpr (!PPM) {
            T wa[6], wb_[6], wc[6], wd[6];   // w(a-1), w(a), w(a+1), w(a+2)
            T bnA, bnB, tmpbn;
            T dA[6], dB[6];                  // delw(a), delw(a+1)
            load_prim<T, D>(S, dm.n, base + wrap_any(a0 - 1, na) * stride, wa, tmpbn);
            load_prim<T, D>(S, dm.n, base + a0 * stride, wb_, bnA);
            load_prim<T, D>(S, dm.n, base + wrap_up(a0, na) * stride, wc, bnB);
            recon_slope<T, RECON>(wa, wb_, wc, wc, bnA, cs, asqr, dA);
            for (int a = a0; a < a1; ++a) {
                int ap1 = wrap_up(a, na);
                int ap2 = wrap_up(ap1, na);
                T bnC;
                load_prim<T, D>(S, dm.n, base + ap2 * stride, wd, bnC);
                recon_slope<T, RECON>(wb_, wc, wd, wd, bnB, cs, asqr, dB);
                T qL[7], qR[7], Fo[7];
                plm_left_state(wb_, dA, bnA, qL);
                plm_right_state(wc, dB, bnA, qR);
                const int kf = (D == 1) ? o : a;
                T sdrop = T(0);
                T& sref = (kf >= rp.zlo && kf < rp.zhi) ? smax : sdrop;
                riemann_flux<SOLVER>(qL, qR, cs, asqr, Fo, sref);
                store_flux(F, D, dm.n, base + a * stride, Fo);
                protection_flux<T, SOLVER>(qL, qR, cs, asqr, sref, rp.Fp, D, dm.n, base + a * stride);
#pragma unroll
                for (int m = 0; m < 6; ++m) { wb_[m] = wc[m]; wc[m] = wd[m]; dA[m] = dB[m]; }
                bnA = bnB; bnB = bnC;
            }
        } else {
            T w0[6], w1[6], w2[6], w3[6];    // w(a), w(a+1), w(a+2), w(a+3)
            T bn0, bn1, bn2, bn3;
            T d0[6], d1[6];                  // delw(a), delw(a+1)
            T r0[6];                         // right edge of cell a
            {
                T wm2[6], wm1[6], dm1[6], l0[6], bnm2, bnm1;
                load_prim<T, D>(S, dm.n, base + wrap_any(a0 - 2, na) * stride, wm2, bnm2);
                load_prim<T, D>(S, dm.n, base + wrap_any(a0 - 1, na) * stride, wm1, bnm1);
                load_prim<T, D>(S, dm.n, base + a0 * stride, w0, bn0);
                load_prim<T, D>(S, dm.n, base + wrap_any(a0 + 1, na) * stride, w1, bn1);
                load_prim<T, D>(S, dm.n, base + wrap_any(a0 + 2, na) * stride, w2, bn2);
                recon_slope<T, RECON>(wm2, wm1, w0, w1, bnm1, cs, asqr, dm1);
                recon_slope<T, RECON>(wm1, w0, w1, w2, bn0, cs, asqr, d0);
                ppm_edges<T, PRIM>(wm1, w0, w1, dm1, d0, l0, r0);
            }
            for (int a = a0; a < a1; ++a) {
                load_prim<T, D>(S, dm.n, base + wrap_any(a + 3, na) * stride, w3, bn3);
                recon_slope<T, RECON>(w0, w1, w2, w3, bn1, cs, asqr, d1);
                T l1[6], r1[6];
                ppm_edges<T, PRIM>(w0, w1, w2, d0, d1, l1, r1);
                T qL[7], qR[7], Fo[7];
                ppm_state(r0, bn0, qL);
                ppm_state(l1, bn0, qR);
                const int kf = (D == 1) ? o : a;
                T sdrop = T(0);
                T& sref = (kf >= rp.zlo && kf < rp.zhi) ? smax : sdrop;
                riemann_flux<SOLVER>(qL, qR, cs, asqr, Fo, sref);
                store_flux(F, D, dm.n, base + a * stride, Fo);
                protection_flux<T, SOLVER>(qL, qR, cs, asqr, sref, rp.Fp, D, dm.n, base + a * stride);
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    w0[m] = w1[m]; w1[m] = w2[m]; w2[m] = w3[m];
                    d0[m] = d1[m]; r0[m] = r1[m];
                }
                bn0 = bn1; bn1 = bn2; bn2 = bn3;
            }
        }
    }
    block_atomic_max<kBX>(smax_slots, (double)smax);
}

// Sweep along x: a block covers TX faces of one (j,k) row; primitives of the
// TX+3 cells (PLM; TX+5 for PPM) and the TX+1 slopes (TX+2) are staged in
// shared memory.
template <class T, int SCHEME, int TX, bool ONE>
__global__ void __launch_bounds__(TX) k_corr_flux_x(BatchArgs ba) {
    constexpr int SOLVER = scheme_solver(SCHEME);
    constexpr int RECON = scheme_recon(SCHEME);
    constexpr bool PPM = (RECON & 1) != 0, PRIM = (RECON & 2) != 0;
    constexpr int H = PPM ? 2 : 1;           // cells staged left of the tile
    constexpr int NW = TX + (PPM ? 5 : 3);   // staged cells
    constexpr int ND = TX + (PPM ? 2 : 1);   // staged slopes, cells i0-H+1 ...
    __shared__ T sw[6][NW];
    __shared__ T sbn[NW];
    __shared__ T sd[6][ND];
    int local;
    const BoxRec rp = resolve<ONE>(ba, scheme_kind(SCHEME, kSubXTile), local);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[1];   // half-step state
    T* __restrict__ F = (T*)rp.F;
    const T cs = (T)rp.cs, asqr = (T)(rp.cs * rp.cs);
    unsigned long long* smax_slots = sc->smax_slots;
    int i0, j, k;
    if constexpr (ONE) {                        // grid (nbt, ny, nz)
        i0 = (int)blockIdx.x * TX; j = (int)blockIdx.y; k = (int)blockIdx.z;
    } else {
        int nbt = (dm.nx + TX - 1) / TX;
        i0 = (local % nbt) * TX;
        j = (local / nbt) % dm.ny;
        k = (local / nbt) / dm.ny;
    }
    int row = dm.nx * (j + dm.ny * k);
    // staged cell t is i0 - H + t
    for (int t = threadIdx.x; t < NW; t += TX) {
        int ii = wrap_any(i0 - H + t, dm.nx);
        T w[6], bn;
        load_prim<T, 0>(S, dm.n, row + ii, w, bn);
#pragma unroll
        for (int m = 0; m < 6; ++m) sw[m][t] = w[m];
        sbn[t] = bn;
    }
    __syncthreads();
    // slope u is that of staged cell u + 1
    for (int u = threadIdx.x; u < ND; u += TX) {
        T wm[6], w0[6], wp[6], wp2[6], d[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            wm[m] = sw[m][u]; w0[m] = sw[m][u + 1]; wp[m] = sw[m][u + 2];
            wp2[m] = PPM ? sw[m][u + 3] : sw[m][u + 2];
        }
        recon_slope<T, RECON>(wm, w0, wp, wp2, sbn[u + 1], cs, asqr, d);
#pragma unroll
        for (int m = 0; m < 6; ++m) sd[m][u] = d[m];
    }
    __syncthreads();
    int t = threadIdx.x;
    int i = i0 + t;
    T smax = T(0);
    if (i < dm.nx) {
        // cell i is staged at t + H, its slope at t + H - 1
        T bn = sbn[t + H];
        T qL[7], qR[7], Fo[7];
        if constexpr (!PPM) {
            T wl[6], wr[6], dl[6], dr[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) { wl[m] = sw[m][t + 1]; wr[m] = sw[m][t + 2]; dl[m] = sd[m][t]; dr[m] = sd[m][t + 1]; }
            plm_left_state(wl, dl, bn, qL);
            plm_right_state(wr, dr, bn, qR);
        } else {
            T wm[6], w0[6], wp[6], wp2[6], dm1[6], d0[6], dp[6], l[6], r[6], l1[6], r1[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                wm[m] = sw[m][t + 1]; w0[m] = sw[m][t + 2]; wp[m] = sw[m][t + 3]; wp2[m] = sw[m][t + 4];
                dm1[m] = sd[m][t]; d0[m] = sd[m][t + 1]; dp[m] = sd[m][t + 2];
            }
            ppm_edges<T, PRIM>(wm, w0, wp, dm1, d0, l, r);      // cell i
            ppm_edges<T, PRIM>(w0, wp, wp2, d0, dp, l1, r1);    // cell i+1
            ppm_state(r, bn, qL);
            ppm_state(l1, bn, qR);
        }
        T sdrop = T(0);
        T& sref = (k >= rp.zlo && k < rp.zhi) ? smax : sdrop;
        riemann_flux<SOLVER>(qL, qR, cs, asqr, Fo, sref);
        store_flux(F, 0, dm.n, row + i, Fo);
        protection_flux<T, SOLVER>(qL, qR, cs, asqr, sref, rp.Fp, 0, dm.n, row + i);
    }
    block_atomic_max<TX>(smax_slots, (double)smax);
}

// Sweep along x over whole rows: one block per (j,k) row.  The primitives,
// face fields and slopes of the row live in shared memory and the periodic
// wrap is an index wrap inside the row, so every cell's slope is computed
// exactly once (the tiled kernel above recomputes slopes at tile edges and
// stages a halo).  PPM evaluates the edges of cells i and i+1 per face.
// Needs 13 * nx * sizeof(T) bytes of dynamic shared memory.
// FP32: 128-thread blocks (smaller barrier groups, 27 KB of shared memory
// each at nx = 512): 3.45 -> 3.22 ms (Roe, PLM) at 512^3 against four
// 256-thread blocks.  A single box runs six per SM at 80 registers without
// spills (3.22 -> 3.19 ms); a table keeps eight at 64 (six: batched workload
// 4.67 -> 4.58e9 cell-updates/s).
template <class T, int SCHEME, bool ONE>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? (ONE ? 6 : 8) : 1) k_corr_flux_xrow(BatchArgs ba) {
    constexpr int SOLVER = scheme_solver(SCHEME);
    constexpr int RECON = scheme_recon(SCHEME);
    constexpr bool PPM = (RECON & 1) != 0, PRIM = (RECON & 2) != 0;
    extern __shared__ __align__(16) unsigned char xrow_smem[];
    int local;
    const BoxRec rp = resolve<ONE>(ba, scheme_kind(SCHEME, kSubXRow), local);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[1];   // half-step state
    T* __restrict__ F = (T*)rp.F;
    const T cs = (T)rp.cs, asqr = (T)(rp.cs * rp.cs);
    unsigned long long* smax_slots = sc->smax_slots;
    const int nx = dm.nx;
    T* sw = (T*)xrow_smem;     // [6][nx] primitives
    T* sbn = sw + 6 * nx;      // [nx] face field at i+1/2
    T* sd = sbn + nx;          // [6][nx] slopes
    int j, k;
    if constexpr (ONE) {                        // grid (ny, nz)
        j = (int)blockIdx.x; k = (int)blockIdx.y;
    } else {
        j = local % dm.ny; k = local / dm.ny;
    }
    int row = nx * (j + dm.ny * k);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        T w[6], bn;
        load_prim<T, 0>(S, dm.n, row + i, w, bn);
#pragma unroll
        for (int m = 0; m < 6; ++m) sw[m * nx + i] = w[m];
        sbn[i] = bn;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        int im = wrap_dn(i, nx), ip = wrap_up(i, nx), ip2 = wrap_up(ip, nx);
        T wm[6], w0[6], wp[6], wp2[6], d[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            wm[m] = sw[m * nx + im]; w0[m] = sw[m * nx + i]; wp[m] = sw[m * nx + ip];
            wp2[m] = PPM ? sw[m * nx + ip2] : wp[m];
        }
        recon_slope<T, RECON>(wm, w0, wp, wp2, sbn[i], cs, asqr, d);
#pragma unroll
        for (int m = 0; m < 6; ++m) sd[m * nx + i] = d[m];
    }
    __syncthreads();
    T smax = T(0);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        int ip = wrap_up(i, nx);
        T bn = sbn[i];
        T qL[7], qR[7], Fo[7];
        if constexpr (!PPM) {
            T wl[6], wr[6], dl[6], dr[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                wl[m] = sw[m * nx + i]; wr[m] = sw[m * nx + ip];
                dl[m] = sd[m * nx + i]; dr[m] = sd[m * nx + ip];
            }
            plm_left_state(wl, dl, bn, qL);
            plm_right_state(wr, dr, bn, qR);
        } else {
            int im = wrap_dn(i, nx), ip2 = wrap_up(ip, nx);
            T wm[6], w0[6], wp[6], wp2[6], dm1[6], d0[6], dp[6], l[6], r[6], l1[6], r1[6];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                wm[m] = sw[m * nx + im]; w0[m] = sw[m * nx + i]; wp[m] = sw[m * nx + ip]; wp2[m] = sw[m * nx + ip2];
                dm1[m] = sd[m * nx + im]; d0[m] = sd[m * nx + i]; dp[m] = sd[m * nx + ip];
            }
            ppm_edges<T, PRIM>(wm, w0, wp, dm1, d0, l, r);      // cell i
            ppm_edges<T, PRIM>(w0, wp, wp2, d0, dp, l1, r1);    // cell i+1
            ppm_state(r, bn, qL);
            ppm_state(l1, bn, qR);
        }
        T sdrop = T(0);
        T& sref = (k >= rp.zlo && k < rp.zhi) ? smax : sdrop;
        riemann_flux<SOLVER>(qL, qR, cs, asqr, Fo, sref);
        store_flux(F, 0, dm.n, row + i, Fo);
        protection_flux<T, SOLVER>(qL, qR, cs, asqr, sref, rp.Fp, 0, dm.n, row + i);
    }
    block_atomic_max_any(smax_slots, (double)smax);
}

// ============================================================ corner EMF
// compute_cell_center_emf_3d (vanleer_mod.f90:1823-1862) evaluated on the fly
// and compute_cell_corner_emf_3d (:1884-2076).  Face EMFs come from the flux
// of the transverse field (:554-555, 726-727, 903-904).
template <class T>
__device__ __forceinline__ T ecc(const T* __restrict__ S, int n, int c, int comp) {
    T irho = T(1) / fld(S, 0, n)[c];
    T mx = fld(S, 1, n)[c], my = fld(S, 2, n)[c], mz = fld(S, 3, n)[c];
    T bx = fld(S, 4, n)[c], by = fld(S, 5, n)[c], bz = fld(S, 6, n)[c];
    if (comp == 0) return (by * mz - bz * my) * irho;
    if (comp == 1) return (bz * mx - bx * mz) * irho;
    return (bx * my - by * mx) * irho;
}
// all three components of the cell-centre EMF of one cell (one reciprocal)
template <class T>
__device__ __forceinline__ void ecc3(const T* __restrict__ S, int n, int c, T& ex, T& ey, T& ez) {
    T irho = T(1) / fld(S, 0, n)[c];
    T mx = fld(S, 1, n)[c], my = fld(S, 2, n)[c], mz = fld(S, 3, n)[c];
    T bx = fld(S, 4, n)[c], by = fld(S, 5, n)[c], bz = fld(S, 6, n)[c];
    ex = (by * mz - bz * my) * irho;
    ey = (bz * mx - bx * mz) * irho;
    ez = (bx * my - by * mx) * irho;
}
template <class T>
__device__ __forceinline__ T face_v(const T* __restrict__ S, int n, int c, int cn, int comp) {
    return T(0.5) * (fld(S, 1 + comp, n)[c] / fld(S, 0, n)[c] + fld(S, 1 + comp, n)[cn] / fld(S, 0, n)[cn]);
}
template <class T>
__device__ __forceinline__ void upwind_pair(T v, T L14, T R14, T L34, T R34, T& o14, T& o34) {
    if (v > T(kZERO)) { o14 = L14; o34 = L34; }
    else if (v < -T(kZERO)) { o14 = R14; o34 = R34; }
    else { o14 = T(0.5) * (L14 + R14); o34 = T(0.5) * (L34 + R34); }
}

// One cell's cell-centre EMF and velocity, from its 7 conserved fields.
template <class T>
struct CellEV {
    T ex, ey, ez;    // ecc3
    T ux, uy, uz;    // m / rho, as face_v divides
};
template <class T>
__device__ __forceinline__ CellEV<T> cell_ev(const T* __restrict__ S, int n, int c) {
    CellEV<T> o;
    ecc3(S, n, c, o.ex, o.ey, o.ez);
    const T r = fld(S, 0, n)[c];
    o.ux = fld(S, 1, n)[c] / r;
    o.uy = fld(S, 2, n)[c] / r;
    o.uz = fld(S, 3, n)[c] / r;
    return o;
}

// A thread walks a column of kSegZ cells along z.  The cell-centre EMFs and
// velocities of plane k+1 computed at one step are those of plane k at the
// next, and so are the z-face EMFs read at k+1, so each is loaded and
// computed once per column instead of once per neighbour.
// PROT: the corner EMFs of the protection fluxes (Fp -> Ep) of the boxes
// that compute them, the second compute_cell_corner_emf_3d call of
// vanleer_mod.f90:336, 396 (the cell-centre EMFs are the same).
// FP32 occupancy: six blocks per SM for a single box (eight spilled more than
// they gained, 2.2 -> 2.4 ms at 512^3); eight in a table, whose small boxes
// leave the loads less overlapped (the batched workload 4.48 -> 4.70e9
// cell-updates/s).
template <class T, bool ONE, bool PROT = false>
__global__ void __launch_bounds__(kBX, sizeof(T) == 4 ? (ONE ? 6 : 8) : 1) k_corner_emf(BatchArgs ba,
                                                                                       int half_step_state) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCellZ, local);
    if (!rp.active || (PROT && !rp.protect)) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)(half_step_state ? rp.S[1] : rp.S[0]);
    const T* __restrict__ F = (const T*)(PROT ? rp.Fp : rp.F);
    T* __restrict__ E = (T*)(PROT ? rp.Ep : rp.E);
    int i, j, k0, k1;
    decode_cellz<ONE>(local, dm, rp.tws, rp.segzs, i, j, k0, k1);
    if (i >= dm.nx || j >= dm.ny) return;
    const int n = dm.n;
    const int plane = dm.nx * dm.ny;
    const int ip = wrap_up(i, dm.nx), jp = wrap_up(j, dm.ny);
    const int r000 = i + dm.nx * j, r100 = ip + dm.nx * j, r010 = i + dm.nx * jp, r110 = ip + dm.nx * jp;
    // face EMFs: E_{t2} = -F_bt1, E_{t1} = F_bt2 of sweep D
    const T* Fx_bt1 = F + (size_t)4 * n;    // x sweep: -Ez at x-face
    const T* Fx_bt2 = F + (size_t)5 * n;    //           Ey at x-face
    const T* Fy_bt1 = F + (size_t)10 * n;   // y sweep: -Ex at y-face
    const T* Fy_bt2 = F + (size_t)11 * n;   //           Ez at y-face
    const T* Fz_bt1 = F + (size_t)16 * n;   // z sweep: -Ey at z-face
    const T* Fz_bt2 = F + (size_t)17 * n;   //           Ex at z-face
    CellEV<T> a000 = cell_ev(S, n, r000 + k0 * plane);
    CellEV<T> a100 = cell_ev(S, n, r100 + k0 * plane);
    CellEV<T> a010 = cell_ev(S, n, r010 + k0 * plane);
    T fx2_000 = Fx_bt2[r000 + k0 * plane], fy1_000 = Fy_bt1[r000 + k0 * plane];
#pragma unroll 2
    for (int k = k0; k < k1; ++k) {
        const int kp = wrap_up(k, dm.nz);
        const int c000 = r000 + k * plane, c100 = r100 + k * plane, c010 = r010 + k * plane;
        const int c110 = r110 + k * plane;
        const int c001 = r000 + kp * plane, c101 = r100 + kp * plane, c011 = r010 + kp * plane;
        const CellEV<T> a001 = cell_ev(S, n, c001);
        const CellEV<T> a101 = cell_ev(S, n, c101);
        const CellEV<T> a011 = cell_ev(S, n, c011);
        const T e110z = ecc(S, n, c110, 2);
        const T fx2_001 = Fx_bt2[c001], fy1_001 = Fy_bt1[c001];
        const T vx = T(0.5) * (a000.ux + a100.ux);
        const T vy = T(0.5) * (a000.uy + a010.uy);
        const T vz = T(0.5) * (a000.uz + a001.uz);
        // Ez at (i+1/2, j+1/2, k)
        {
            T E31_000 = -Fx_bt1[c000], E31_010 = -Fx_bt1[c010];
            T E32_000 = Fy_bt2[c000], E32_100 = Fy_bt2[c100];
            T E33_000 = a000.ez, E33_100 = a100.ez, E33_010 = a010.ez, E33_110 = e110z;
            T dyL14 = T(2) * (E32_000 - E33_000);
            T dyR14 = T(2) * (E32_100 - E33_100);
            T dyL34 = T(2) * (E33_010 - E32_000);
            T dyR34 = T(2) * (E33_110 - E32_100);
            T dy1214, dy1234;
            upwind_pair(vx, dyL14, dyR14, dyL34, dyR34, dy1214, dy1234);
            T dxL14 = T(2) * (E31_000 - E33_000);
            T dxR14 = T(2) * (E31_010 - E33_010);
            T dxL34 = T(2) * (E33_100 - E31_000);
            T dxR34 = T(2) * (E33_110 - E31_010);
            T dx1412, dx3412;
            upwind_pair(vy, dxL14, dxR14, dxL34, dxR34, dx1412, dx3412);
            E[(size_t)2 * n + c000] = T(0.25) * (E31_000 + E31_010 + E32_000 + E32_100) +
                                      T(0.125) * ((dy1214 - dy1234) + (dx1412 - dx3412));
        }
        // Ey at (i+1/2, j, k+1/2)
        {
            T E21_000 = fx2_000, E21_001 = fx2_001;
            T E22_000 = -Fz_bt1[c000], E22_100 = -Fz_bt1[c100];
            T E23_000 = a000.ey, E23_100 = a100.ey, E23_001 = a001.ey, E23_101 = a101.ey;
            T dzL14 = T(2) * (E22_000 - E23_000);
            T dzR14 = T(2) * (E22_100 - E23_100);
            T dzL34 = T(2) * (E23_001 - E22_000);
            T dzR34 = T(2) * (E23_101 - E22_100);
            T dz1214, dz1234;
            upwind_pair(vx, dzL14, dzR14, dzL34, dzR34, dz1214, dz1234);
            T dxL14 = T(2) * (E21_000 - E23_000);
            T dxR14 = T(2) * (E21_001 - E23_001);
            T dxL34 = T(2) * (E23_100 - E21_000);
            T dxR34 = T(2) * (E23_101 - E21_001);
            T dx1412, dx3412;
            upwind_pair(vz, dxL14, dxR14, dxL34, dxR34, dx1412, dx3412);
            E[(size_t)1 * n + c000] = T(0.25) * (E21_000 + E21_001 + E22_000 + E22_100) +
                                      T(0.125) * ((dz1214 - dz1234) + (dx1412 - dx3412));
        }
        // Ex at (i, j+1/2, k+1/2)
        {
            T E11_000 = -fy1_000, E11_001 = -fy1_001;
            T E12_000 = Fz_bt2[c000], E12_010 = Fz_bt2[c010];
            T E13_000 = a000.ex, E13_010 = a010.ex, E13_001 = a001.ex, E13_011 = a011.ex;
            T dzL14 = T(2) * (E12_000 - E13_000);
            T dzR14 = T(2) * (E12_010 - E13_010);
            T dzL34 = T(2) * (E13_001 - E12_000);
            T dzR34 = T(2) * (E13_011 - E12_010);
            T dz1214, dz1234;
            upwind_pair(vy, dzL14, dzR14, dzL34, dzR34, dz1214, dz1234);
            T dyL14 = T(2) * (E11_000 - E13_000);
            T dyR14 = T(2) * (E11_001 - E13_001);
            T dyL34 = T(2) * (E13_010 - E11_000);
            T dyR34 = T(2) * (E13_011 - E11_001);
            T dy1412, dy3412;
            upwind_pair(vz, dyL14, dyR14, dyL34, dyR34, dy1412, dy3412);
            E[c000] = T(0.25) * (E11_000 + E11_001 + E12_000 + E12_010) +
                      T(0.125) * ((dz1214 - dz1234) + (dy1412 - dy3412));
        }
        a000 = a001;
        a100 = a101;
        a010 = a011;
        fx2_000 = fx2_001;
        fy1_000 = fy1_001;
    }
}

// ============================================================ update
// update_hydro_state_3d + final_check_unphysical (vanleer_mod.f90:2080-2207,
// 3243-3262) and update_CT_3d with the cell-centre average (:2211-2259).
// Reads the step-start state S0 and writes Sout.  With do_cfl the fast-speed
// maximum of the new state (get_max_speed_vanleer :3281-3318) is folded in.
template <class T>
__device__ __forceinline__ T ct_bx(const T* __restrict__ S0, const T* __restrict__ E, int n, T dtdx, int c, int cym,
                                   int czm) {
    return fld(S0, 7, n)[c] - dtdx * ((E[2 * (size_t)n + c] - E[2 * (size_t)n + cym]) - (E[(size_t)n + c] - E[(size_t)n + czm]));
}
template <class T>
__device__ __forceinline__ T ct_by(const T* __restrict__ S0, const T* __restrict__ E, int n, T dtdx, int c, int czm,
                                   int cxm) {
    return fld(S0, 8, n)[c] - dtdx * ((E[c] - E[czm]) - (E[2 * (size_t)n + c] - E[2 * (size_t)n + cxm]));
}
template <class T>
__device__ __forceinline__ T ct_bz(const T* __restrict__ S0, const T* __restrict__ E, int n, T dtdx, int c, int cxm,
                                   int cym) {
    return fld(S0, 9, n)[c] - dtdx * ((E[(size_t)n + c] - E[(size_t)n + cxm]) - (E[c] - E[cym]));
}

// Time-averaged velocity of the passive corrector, vel_tavg = (v_old + v_new)/2
// (copy_velocity(.TRUE.), passive_mod.f90:227-239), written once per cell by
// the final update (and again by the forcing kick and the protected update,
// which change the new momentum) into three flux fields the update no longer
// reads (the face EMF components of the x and y sweeps), so that the passive
// corrector reads three values per cell instead of eight and divides nothing.
// The arithmetic is that of copy_velocity: m0 * (1/rho0) and m1 * (1/rho1).
template <class T>
__device__ __forceinline__ T vt_of(T rho0, T m0, T rho1, T m1) {
    const T vold = m0 * (T(1) / rho0);
    const T irho = T(1) / rho1;
    return T(0.5) * (vold + m1 * irho);
}
template <class T>
__device__ __forceinline__ T* vt_field(const BoxRec& r, int d) {
    return (T*)r.F + (size_t)(d == 2 ? 10 : 4 + d) * (size_t)r.n;
}

// Flux protection (flux_protection, vanleer_mod.f90:81, 2086-2202): a cell
// whose updated density fell below MIN_DENS is flagged and listed for the
// protection kernels of this update stage (0 predictor, 1 final).  A list
// that overflows sets IMHD_S_PROTECT.
constexpr unsigned kStatusProtect = 32u;   // IMHD_S_PROTECT
__device__ __forceinline__ void prot_mark_bad(const BoxRec& r, int stage, int c) {
    r.bad[c] = 1;
    const unsigned slot = atomicAdd(&r.sc->nbad[stage], 1u);
    if (slot < (unsigned)r.badcap) r.badlist[(size_t)stage * r.badcap + slot] = c;
    else atomicOr(&r.sc->status, kStatusProtect);
}

// A table's box goes to the bulk-copy fed update when its rows are whole
// 128-cell tiles (or 64-cell tiles with an even row count: a block then takes
// two rows) and the bases its copies read from are 16-byte aligned (both
// update kernels decide from the same record, so exactly one takes the box).
__host__ __device__ __forceinline__ int tma_row_tile(int nx, int ny) {
    return nx % kTmaTile == 0 ? kTmaTile : (nx % (kTmaTile / 2) == 0 && ny % 2 == 0) ? kTmaTile / 2 : 0;
}
__device__ __forceinline__ bool update_by_tma(const BoxRec& r) {
    return tma_row_tile(r.nx, r.ny) > 0 && (((uintptr_t)r.S[0] | (uintptr_t)r.F | (uintptr_t)r.E) & 15) == 0;
}

// A thread walks a column of kSegZ cells along z; the z-face fluxes, the
// corner EMFs at k and the new face field bz read or computed at plane k are
// the "k-1" values of plane k+1 and are carried instead of reloaded.
// ZR: some box of the table restricts its maxima to a z range (slabs); the
// other instantiation has no per-plane test on the hot path.
template <class T, bool ONE, bool ZR>
__global__ void __launch_bounds__(kBX, sizeof(T) == 4 ? 6 : 1) k_update(BatchArgs ba, double dt_scale, int final_stage) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCellZ, local);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    if (!ONE && update_by_tma(rp)) return;   // a table's 128k-cell rows go to k_update_tma
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ Sout = (T*)rp.S[1];
    const T* __restrict__ F = (const T*)rp.F;
    const T* __restrict__ E = (const T*)rp.E;
    const double dx = rp.dx;
    const T asqr = (T)(rp.cs * rp.cs);
    const int do_cfl = final_stage && !sc->drive;
    const bool write_vt = final_stage && rp.npass > 0;
    unsigned long long* cmax_slots = sc->cmax_slots;
    unsigned long long* floor_hits = &sc->floor_hits;
    unsigned int* status = &sc->status;
    int i, j, k0, k1;
    decode_cellz<ONE>(local, dm, rp.tws, rp.segzs, i, j, k0, k1);
    const bool valid = i < dm.nx && j < dm.ny;
    double cmax = 0.0;
    if (valid) {
        const int n = dm.n;
        const T dtdx = (T)(dt_scale * sc->dt / dx);
        const int plane = dm.nx * dm.ny;
        const int im = wrap_dn(i, dm.nx), jm = wrap_dn(j, dm.ny);
        const int r0 = i + dm.nx * j, rxm = im + dm.nx * j, rym = i + dm.nx * jm, rxmym = im + dm.nx * jm;
        const T* Ex = E;
        const T* Ey = E + (size_t)n;
        // values of plane k-1 (periodic image for the first cell of the column)
        T Fzm[4], Ex_zm, Ey_zm, Ex_ymzm, Ey_xmzm, bzm;
        {
            const int km = wrap_dn(k0, dm.nz);
            const int czm = r0 + km * plane, cxmzm = rxm + km * plane, cymzm = rym + km * plane;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                int fz = (v == 0) ? 0 : 1 + (v - 1 - 2 + 3) % 3;
                Fzm[v] = F[(size_t)(12 + fz) * n + czm];
            }
            Ex_zm = Ex[czm];
            Ey_zm = Ey[czm];
            Ex_ymzm = Ex[cymzm];
            Ey_xmzm = Ey[cxmzm];
            bzm = ct_bz(S0, E, n, dtdx, czm, cxmzm, cymzm);
        }
#pragma unroll 1
        for (int k = k0; k < k1; ++k) {
            const int c = r0 + k * plane, cxm = rxm + k * plane, cym = rym + k * plane, cxmym = rxmym + k * plane;
            T out[4], Fz0[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                // flux component of xyz variable v in sweep D: rho -> 0; momentum X -> 1 + (X - D) mod 3
                int fx = (v == 0) ? 0 : 1 + (v - 1 + 3) % 3;
                int fy = (v == 0) ? 0 : 1 + (v - 1 - 1 + 3) % 3;
                int fz = (v == 0) ? 0 : 1 + (v - 1 - 2 + 3) % 3;
                const T* Fx = F + (size_t)(0 + fx) * n;
                const T* Fy = F + (size_t)(6 + fy) * n;
                Fz0[v] = F[(size_t)(12 + fz) * n + c];
                out[v] = fld(S0, v, n)[c] - dtdx * ((Fx[c] - Fx[cxm]) + (Fy[c] - Fy[cym]) + (Fz0[v] - Fzm[v]));
            }
            const bool inz = !ZR || (k >= rp.zlo && k < rp.zhi);
            if (out[0] < T(kMIN_DENS)) {
                out[0] = T(kMIN_DENS);
                if (rp.protect) prot_mark_bad(rp, final_stage, c);   // updated again by k_prot_hydro
                else if (inz) atomicAdd(floor_hits, 1ull);
            }
            const T Ex0 = Ex[c], Ey0 = Ey[c], Ez0 = E[2 * (size_t)n + c];
            const T Ex_ym = Ex[cym], Ey_xm = Ey[cxm];
            const T Ez_ym = E[2 * (size_t)n + cym], Ez_xm = E[2 * (size_t)n + cxm], Ez_xmym = E[2 * (size_t)n + cxmym];
            // ct_bx / ct_by / ct_bz of the face fields at c and at the minus faces
            const T bx = fld(S0, 7, n)[c] - dtdx * ((Ez0 - Ez_ym) - (Ey0 - Ey_zm));
            const T by = fld(S0, 8, n)[c] - dtdx * ((Ex0 - Ex_zm) - (Ez0 - Ez_xm));
            const T bz = fld(S0, 9, n)[c] - dtdx * ((Ey0 - Ey_xm) - (Ex0 - Ex_ym));
            const T bxm = fld(S0, 7, n)[cxm] - dtdx * ((Ez_xm - Ez_xmym) - (Ey_xm - Ey_xmzm));
            const T bym = fld(S0, 8, n)[cym] - dtdx * ((Ex_ym - Ex_ymzm) - (Ez_ym - Ez_xmym));
            const T bxc = T(0.5) * (bx + bxm);
            const T byc = T(0.5) * (by + bym);
            const T bzc = T(0.5) * (bz + bzm);
#pragma unroll
            for (int v = 0; v < 4; ++v) fld(Sout, v, n)[c] = out[v];
            fld(Sout, 4, n)[c] = bxc;
            fld(Sout, 5, n)[c] = byc;
            fld(Sout, 6, n)[c] = bzc;
            fld(Sout, 7, n)[c] = bx;
            fld(Sout, 8, n)[c] = by;
            fld(Sout, 9, n)[c] = bz;
            if (write_vt) {
                const T r0 = fld(S0, 0, n)[c];
#pragma unroll
                for (int d = 0; d < 3; ++d) vt_field<T>(rp, d)[c] = vt_of(r0, fld(S0, 1 + d, n)[c], out[0], out[1 + d]);
            }
            if (do_cfl && inz)
                cmax = nmax(cmax, (double)cell_max_speed(out[0], out[1], out[2], out[3], bxc, byc, bzc, asqr));
            if (inz && !(isfinite(out[0]) && isfinite(out[1]) && isfinite(out[2]) && isfinite(out[3]) && isfinite(bx) &&
                         isfinite(by) && isfinite(bz)))
                atomicOr(status, 2u);
#pragma unroll
            for (int v = 0; v < 4; ++v) Fzm[v] = Fz0[v];
            Ex_zm = Ex0;
            Ey_zm = Ey0;
            Ex_ymzm = Ex_ym;
            Ey_xmzm = Ey_xm;
            bzm = bz;
        }
    }
    if (do_cfl) block_atomic_max<kBX>(cmax_slots, cmax);
}

// ------------------------------------------------------------ update, TMA-fed
// The same update for boxes whose rows are whole 128-cell tiles (TW = 128),
// or 64-cell tiles with an even row count (TW = 64, two rows per block): a
// block owns 128 cells of one or two rows and walks kSegZ planes; warp 0
// streams each plane's operands into shared memory with bulk asynchronous
// copies (cp.async.bulk, completion counted on an mbarrier), one plane ahead
// of the plane being computed, so that the loads' latency overlaps the
// arithmetic without registers held for them.  Per plane and row: 29 row
// segments (22 fields of row j, 7 of row j-1) and 8 16-byte segments that end
// at the cell left of the tile (the periodic image at i = nx-1 for the first
// tile), each stored just in front of its row so that the left neighbour of
// every cell is the element before it.  Lane R % 32 of warp 0 issues row R.
// Single boxes launch it alone; a table launches it beside k_update, which
// skips the boxes it takes (update_by_tma).
// Every wait is bounded: on time-out the kernel sets IMHD_S_WAIT in the
// status word, skips the arithmetic and drains its copies with a bounded
// wait before it exits.
constexpr int kTmaRows = 29;
constexpr int kTmaHalos = 8;
constexpr unsigned kStatusWait = 16u;        // IMHD_S_WAIT
constexpr long long kTmaSpin = 1ll << 24;   // try_wait polls before a wait gives up
template <class T>
constexpr int tma_row_stride() { return kTmaTile + 16 / (int)sizeof(T); }   // a 16-byte halo slot + the row
// a block stages kTmaTile / TW rows of TW-cell segments
template <class T, int TW>
constexpr int tma_copy_bytes() { return kTmaRows * kTmaTile * (int)sizeof(T) + (kTmaTile / TW) * kTmaHalos * 16; }
template <class T, int TW>
constexpr int tma_stage_bytes() {
    return ((kTmaTile / TW) * kTmaRows * (TW + 2 * (16 / (int)sizeof(T))) * (int)sizeof(T) + 127) / 128 * 128;
}
template <class T, int TW>
constexpr size_t update_tma_smem_bytes() { return 2 * (size_t)tma_stage_bytes<T, TW>(); }

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// true once the phase with the given parity has completed; false after kTmaSpin polls
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const unsigned a = smem_addr(bar);
    for (long long it = 0; it < kTmaSpin; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// global -> shared bulk copy of `bytes` (16-byte aligned ends), completion counted on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

template <class T, bool ZR, bool ONE, int TW>
__global__ void __launch_bounds__(kTmaTile, sizeof(T) == 4 ? 6 : 1)
    k_update_tma(BatchArgs ba, double dt_scale, int final_stage) {
    extern __shared__ __align__(128) unsigned char tma_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    constexpr int RB = kTmaTile / TW;    // rows per block
    int local;
    const BoxRec rp = resolve<ONE>(ba, TW == kTmaTile ? kKindUpdTma : kKindUpdTma64, local);
    Scalars* sc = rp.sc;
    if (!rp.active || (!ONE && !update_by_tma(rp))) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ Sout = (T*)rp.S[1];
    const T* __restrict__ F = (const T*)rp.F;
    const T* __restrict__ E = (const T*)rp.E;
    const T asqr = (T)(rp.cs * rp.cs);
    const int do_cfl = final_stage && !sc->drive;
    const bool write_vt = final_stage && rp.npass > 0;
    const int t = (int)threadIdx.x;
    const int lx = t % TW, ly = t / TW;
    int i0, j0, seg;
    if constexpr (ONE) {   // grid (nx / TW, ny / RB, z segments)
        i0 = (int)blockIdx.x * TW;
        j0 = (int)blockIdx.y * RB;
        seg = (int)blockIdx.z;
    } else {
        const int nbx = dm.nx / TW, nby = dm.ny / RB, rest = local / nbx;
        i0 = (local % nbx) * TW;
        j0 = (rest % nby) * RB;
        seg = rest / nby;
    }
    const int i = i0 + lx, j = j0 + ly;
    const int k0 = seg * kSegZ, k1 = min(k0 + kSegZ, dm.nz);
    const int n = dm.n, plane = dm.nx * dm.ny;
    const int jm = wrap_dn(j, dm.ny);
    const T dtdx = (T)(dt_scale * sc->dt / rp.dx);
    constexpr int HE = 16 / (int)sizeof(T);          // elements of a 16-byte segment
    const int ih = (i0 == 0 ? dm.nx : i0) - HE;       // segment ending at the cell left of the tile
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    // operand rows of plane k into stage g: row R = (block row) * 29 + r, and
    // its halo, by lane R % 32 of warp 0
    constexpr int RS = TW + 2 * HE;
    auto issue = [&](int g, int k) {
        T* rows = (T*)(tma_smem + (size_t)g * tma_stage_bytes<T, TW>());
        unsigned long long* bar = &bars[g];
        if (t == 0) mbar_expect_tx(bar, (unsigned)tma_copy_bytes<T, TW>());
        __syncwarp();
        for (int R = t; R < RB * kTmaRows; R += 32) {
            const int r = R % kTmaRows, jrow = j0 + R / kTmaRows, jm = wrap_dn(jrow, dm.ny);
            const T* base;
            int jr = jrow;
            if (r < 4) base = fld(S0, r, n);
            else if (r < 7) base = fld(S0, 3 + r, n);                                        // fields 7-9
            else if (r < 11) base = F + (size_t)(r - 7) * n;                                  // x fluxes
            else if (r < 15) base = F + (size_t)(6 + (r == 11 ? 0 : 1 + (r - 11 + 1) % 3)) * n;    // y, by variable
            else if (r < 19) base = F + (size_t)(12 + (r == 15 ? 0 : 1 + (r - 15) % 3)) * n;       // z, by variable
            else if (r < 22) base = E + (size_t)(r - 19) * n;
            else if (r < 26) { base = F + (size_t)(6 + (r == 22 ? 0 : 1 + (r - 22 + 1) % 3)) * n; jr = jm; }
            else if (r == 26) { base = fld(S0, 8, n); jr = jm; }
            else if (r == 27) { base = E; jr = jm; }
            else { base = E + 2 * (size_t)n; jr = jm; }
            const size_t ofs = (size_t)dm.nx * (jr + (size_t)dm.ny * k);
            bulk_g2s(rows + R * RS + HE, base + i0 + ofs, TW * (unsigned)sizeof(T), bar);
            // rows whose left neighbour is read: x fluxes, bx, Ey, Ez and Ez of row j-1
            if ((r >= 7 && r <= 10) || r == 4 || r == 20 || r == 21 || r == 28)
                bulk_g2s(rows + R * RS, base + ih + ofs, 16u, bar);
        }
    };
    if (t < 32) issue(0, k0);

    unsigned long long* cmax_slots = sc->cmax_slots;
    double cmax = 0.0;
    bool ok = true;
    // values of plane k-1 (periodic image for the first plane of the segment)
    const int im = wrap_dn(i, dm.nx);
    const int r0 = i + dm.nx * j, rxm = im + dm.nx * j, rym = i + dm.nx * jm;
    T Fzm[4], Ex_zm, Ey_zm, Ex_ymzm, Ey_xmzm, bzm;
    {
        const int km = wrap_dn(k0, dm.nz);
        const int czm = r0 + km * plane, cxmzm = rxm + km * plane, cymzm = rym + km * plane;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            int fz = (v == 0) ? 0 : 1 + (v - 1 - 2 + 3) % 3;
            Fzm[v] = F[(size_t)(12 + fz) * n + czm];
        }
        Ex_zm = E[czm];
        Ey_zm = E[(size_t)n + czm];
        Ex_ymzm = E[cymzm];
        Ey_xmzm = E[(size_t)n + cxmzm];
        bzm = ct_bz(S0, E, n, dtdx, czm, cxmzm, cymzm);
    }
    for (int k = k0; k < k1; ++k) {
        const int it = k - k0, g = it & 1;
        if (t < 32 && k + 1 < k1) issue(g ^ 1, k + 1);
        if (ok && !mbar_wait(&bars[g], (unsigned)((it >> 1) & 1))) {
            ok = false;
            atomicOr(&sc->status, kStatusWait);
        }
        if (ok) {
            const T* rows = (const T*)(tma_smem + (size_t)g * tma_stage_bytes<T, TW>()) + ly * kTmaRows * RS + HE + lx;
            auto at = [&](int r) { return rows[r * RS]; };
            auto xm = [&](int r, int) { return rows[r * RS - 1]; };
            const int c = r0 + k * plane;
            T out[4], Fz0[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Fz0[v] = at(15 + v);
                out[v] = at(v) - dtdx * ((at(7 + v) - xm(7 + v, v)) + (at(11 + v) - at(22 + v)) + (Fz0[v] - Fzm[v]));
            }
            const bool inz = !ZR || (k >= rp.zlo && k < rp.zhi);
            if (out[0] < T(kMIN_DENS)) {
                out[0] = T(kMIN_DENS);
                if (rp.protect) prot_mark_bad(rp, final_stage, c);   // updated again by k_prot_hydro
                else if (inz) atomicAdd(&sc->floor_hits, 1ull);
            }
            const T Ex0 = at(19), Ey0 = at(20), Ez0 = at(21);
            const T Ex_ym = at(27), Ey_xm = xm(20, 5);
            const T Ez_ym = at(28), Ez_xm = xm(21, 6), Ez_xmym = xm(28, 7);
            const T bx = at(4) - dtdx * ((Ez0 - Ez_ym) - (Ey0 - Ey_zm));
            const T by = at(5) - dtdx * ((Ex0 - Ex_zm) - (Ez0 - Ez_xm));
            const T bz = at(6) - dtdx * ((Ey0 - Ey_xm) - (Ex0 - Ex_ym));
            const T bxm = xm(4, 4) - dtdx * ((Ez_xm - Ez_xmym) - (Ey_xm - Ey_xmzm));
            const T bym = at(26) - dtdx * ((Ex_ym - Ex_ymzm) - (Ez_ym - Ez_xmym));
            const T bxc = T(0.5) * (bx + bxm);
            const T byc = T(0.5) * (by + bym);
            const T bzc = T(0.5) * (bz + bzm);
#pragma unroll
            for (int v = 0; v < 4; ++v) fld(Sout, v, n)[c] = out[v];
            fld(Sout, 4, n)[c] = bxc;
            fld(Sout, 5, n)[c] = byc;
            fld(Sout, 6, n)[c] = bzc;
            fld(Sout, 7, n)[c] = bx;
            fld(Sout, 8, n)[c] = by;
            fld(Sout, 9, n)[c] = bz;
            if (write_vt) {
#pragma unroll
                for (int d = 0; d < 3; ++d) vt_field<T>(rp, d)[c] = vt_of(at(0), at(1 + d), out[0], out[1 + d]);
            }
            if (do_cfl && inz)
                cmax = nmax(cmax, (double)cell_max_speed(out[0], out[1], out[2], out[3], bxc, byc, bzc, asqr));
            if (inz && !(isfinite(out[0]) && isfinite(out[1]) && isfinite(out[2]) && isfinite(out[3]) && isfinite(bx) &&
                         isfinite(by) && isfinite(bz)))
                atomicOr(&sc->status, 2u);
#pragma unroll
            for (int v = 0; v < 4; ++v) Fzm[v] = Fz0[v];
            Ex_zm = Ex0;
            Ey_zm = Ey0;
            Ex_ymzm = Ex_ym;
            Ey_xmzm = Ey_xm;
            bzm = bz;
        }
        __syncthreads();   // every thread is done with stage g before it is refilled
    }
    // a wait that gave up may leave copies in flight: let them land (bounded) before exit
    if (t == 0 && !ok) {
        const int last = k1 - 1 - k0;
        mbar_wait(&bars[last & 1], (unsigned)((last >> 1) & 1));
    }
    if (do_cfl) block_atomic_max<kTmaTile>(cmax_slots, cmax);
}

// ============================================================ flux protection
// The protected update of update_hydro_state_3d (vanleer_mod.f90:2086-2202)
// after an update stage that listed bad cells (prot_mark_bad).  The
// reference, for every bad cell, copies the protection (HLLE) fluxes of its
// six faces into the flux array and the protection corner EMFs of the four
// corners (i,j,k), (i-1,j,k), (i,j-1,k), (i,j,k-1) of each component into
// the corner array (:2147-2171), then updates the bad cells and their six
// neighbours again from the state before the update (:2179-2201); the CT
// update that follows uses the replaced corners.  So a face takes the
// protection flux when a cell on either side is bad, and corner (i,j,k) takes
// the protection EMF when one of the cells (i,j,k), (i+1,j,k), (i,j+1,k),
// (i,j,k+1) is bad.  kProtBlocks blocks per box walk the stage's list; a cell
// reached from several bad cells is written by the smallest of them (hydro)
// or rewritten with the same value (faces, cell centres).
constexpr int kProtBlocks = 32;

template <bool ONE>
__device__ __forceinline__ BoxRec prot_box(const BatchArgs& ba, int& local) {
    const int b = ONE ? 0 : (int)blockIdx.x / kProtBlocks;
    local = ONE ? (int)blockIdx.x : (int)blockIdx.x % kProtBlocks;
    return box_at(ba, b);
}
__device__ __forceinline__ int cell_at(const Dims& dm, int i, int j, int k) {
    return wrap_any(i, dm.nx) + dm.nx * (wrap_any(j, dm.ny) + dm.ny * wrap_any(k, dm.nz));
}
__device__ __forceinline__ void cell_ijk(const Dims& dm, int c, int& i, int& j, int& k) {
    const int plane = dm.nx * dm.ny;
    i = c % dm.nx;
    j = (c % plane) / dm.nx;
    k = c / plane;
}
// corner of component m (0 Ex, 1 Ey, 2 Ez) at cell (i,j,k) takes the protection EMF
__device__ __forceinline__ bool prot_corner(const unsigned char* __restrict__ bad, const Dims& dm, int i, int j, int k) {
    return bad[cell_at(dm, i, j, k)] | bad[cell_at(dm, i + 1, j, k)] | bad[cell_at(dm, i, j + 1, k)] |
           bad[cell_at(dm, i, j, k + 1)];
}

// Hydro variables of the bad cells and their neighbours, again from the
// state before the update with the protection fluxes on the faces of bad
// cells, then final_check_unphysical (:3243-3262) for them.
template <class T, bool ONE>
__global__ void __launch_bounds__(kBX) k_prot_hydro(BatchArgs ba, double dt_scale, int stage) {
    int local;
    const BoxRec rp = prot_box<ONE>(ba, local);
    if (!rp.active || !rp.protect) return;
    Scalars* sc = rp.sc;
    const unsigned nb = min(sc->nbad[stage], (unsigned)rp.badcap);
    if (nb == 0) return;
    const Dims dm = dims_of(rp);
    const int n = dm.n;
    const int* __restrict__ list = rp.badlist + (size_t)stage * rp.badcap;
    const unsigned char* __restrict__ bad = rp.bad;
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ Sout = (T*)rp.S[1];
    const T* __restrict__ F = (const T*)rp.F;
    const T* __restrict__ Fp = (const T*)rp.Fp;
    const T dtdx = (T)(dt_scale * sc->dt / rp.dx);
    for (long w = (long)local * blockDim.x + threadIdx.x; w < 7L * nb; w += (long)kProtBlocks * blockDim.x) {
        const int b = list[w / 7];
        const int slot = (int)(w % 7);
        int i, j, k;
        cell_ijk(dm, b, i, j, k);
        if (slot == 1) --i; else if (slot == 2) ++i;
        else if (slot == 3) --j; else if (slot == 4) ++j;
        else if (slot == 5) --k; else if (slot == 6) ++k;
        const int c = cell_at(dm, i, j, k);
        const int cxm = cell_at(dm, i - 1, j, k), cxp = cell_at(dm, i + 1, j, k);
        const int cym = cell_at(dm, i, j - 1, k), cyp = cell_at(dm, i, j + 1, k);
        const int czm = cell_at(dm, i, j, k - 1), czp = cell_at(dm, i, j, k + 1);
        const bool b0 = bad[c], bxm = bad[cxm], bxp = bad[cxp], bym = bad[cym], byp = bad[cyp];
        const bool bzm = bad[czm], bzp = bad[czp];
        // the smallest bad cell next to c (or c itself) writes it
        int owner = 0x7fffffff;
        if (b0) owner = c;
        if (bxm && cxm < owner) owner = cxm;
        if (bxp && cxp < owner) owner = cxp;
        if (bym && cym < owner) owner = cym;
        if (byp && cyp < owner) owner = cyp;
        if (bzm && czm < owner) owner = czm;
        if (bzp && czp < owner) owner = czp;
        if (owner != b) continue;
        const bool px = b0 || bxp, pxm = bxm || b0, py = b0 || byp, pym = bym || b0, pz = b0 || bzp, pzm = bzm || b0;
        T out[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int fx = (v == 0) ? 0 : 1 + (v - 1 + 3) % 3;
            const int fy = (v == 0) ? 0 : 1 + (v - 1 - 1 + 3) % 3;
            const int fz = (v == 0) ? 0 : 1 + (v - 1 - 2 + 3) % 3;
            const T Fxc = (px ? Fp : F)[(size_t)fx * n + c], Fxm = (pxm ? Fp : F)[(size_t)fx * n + cxm];
            const T Fyc = (py ? Fp : F)[(size_t)(6 + fy) * n + c], Fym = (pym ? Fp : F)[(size_t)(6 + fy) * n + cym];
            const T Fzc = (pz ? Fp : F)[(size_t)(12 + fz) * n + c], Fzm = (pzm ? Fp : F)[(size_t)(12 + fz) * n + czm];
            out[v] = fld(S0, v, n)[c] - dtdx * ((Fxc - Fxm) + (Fyc - Fym) + (Fzc - Fzm));
        }
        const bool inz = k >= rp.zlo && k < rp.zhi;
        if (out[0] < T(kMIN_DENS)) {
            out[0] = T(kMIN_DENS);
            if (inz) atomicAdd(&sc->floor_hits, 1ull);
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) fld(Sout, v, n)[c] = out[v];
        if (stage == 1 && rp.npass > 0) {
            const T r0 = fld(S0, 0, n)[c];
#pragma unroll
            for (int d = 0; d < 3; ++d) vt_field<T>(rp, d)[c] = vt_of(r0, fld(S0, 1 + d, n)[c], out[0], out[1 + d]);
        }
        if (inz && !(isfinite(out[0]) && isfinite(out[1]) && isfinite(out[2]) && isfinite(out[3])))
            atomicOr(&sc->status, 2u);
    }
}

// Face fields around the bad cells with the protection corner EMFs where
// they replace the corners (update_CT_3d, :2211-2245).
template <class T, bool ONE>
__global__ void __launch_bounds__(kBX) k_prot_faces(BatchArgs ba, double dt_scale, int stage) {
    int local;
    const BoxRec rp = prot_box<ONE>(ba, local);
    if (!rp.active || !rp.protect) return;
    Scalars* sc = rp.sc;
    const unsigned nb = min(sc->nbad[stage], (unsigned)rp.badcap);
    if (nb == 0) return;
    const Dims dm = dims_of(rp);
    const int n = dm.n;
    const int* __restrict__ list = rp.badlist + (size_t)stage * rp.badcap;
    const unsigned char* __restrict__ bad = rp.bad;
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ Sout = (T*)rp.S[1];
    const T* __restrict__ E = (const T*)rp.E;
    const T* __restrict__ Ep = (const T*)rp.Ep;
    const T dtdx = (T)(dt_scale * sc->dt / rp.dx);
    // corner EMF of component m at cell (i,j,k): the protection value where replaced
    auto corner = [&](int m, int i, int j, int k) -> T {
        const int q = cell_at(dm, i, j, k);
        return (prot_corner(bad, dm, i, j, k) ? Ep : E)[(size_t)m * n + q];
    };
    for (long w = (long)local * blockDim.x + threadIdx.x; w < 27L * nb; w += (long)kProtBlocks * blockDim.x) {
        int i, j, k;
        cell_ijk(dm, list[w / 27], i, j, k);
        const int o = (int)(w % 27);
        i += o % 3 - 1;
        j += (o / 3) % 3 - 1;
        k += o / 9 - 1;
        const int c = cell_at(dm, i, j, k);
        const T Ex0 = corner(0, i, j, k), Ey0 = corner(1, i, j, k), Ez0 = corner(2, i, j, k);
        const T bx = fld(S0, 7, n)[c] - dtdx * ((Ez0 - corner(2, i, j - 1, k)) - (Ey0 - corner(1, i, j, k - 1)));
        const T by = fld(S0, 8, n)[c] - dtdx * ((Ex0 - corner(0, i, j, k - 1)) - (Ez0 - corner(2, i - 1, j, k)));
        const T bz = fld(S0, 9, n)[c] - dtdx * ((Ey0 - corner(1, i - 1, j, k)) - (Ex0 - corner(0, i, j - 1, k)));
        fld(Sout, 7, n)[c] = bx;
        fld(Sout, 8, n)[c] = by;
        fld(Sout, 9, n)[c] = bz;
        const int kk = wrap_any(k, dm.nz);
        if (kk >= rp.zlo && kk < rp.zhi && !(isfinite(bx) && isfinite(by) && isfinite(bz))) atomicOr(&sc->status, 2u);
    }
}

// Cell-centred field of the cells next to those faces (update_CT_3d, :2248-2259).
template <class T, bool ONE>
__global__ void __launch_bounds__(kBX) k_prot_centres(BatchArgs ba, int stage) {
    int local;
    const BoxRec rp = prot_box<ONE>(ba, local);
    if (!rp.active || !rp.protect) return;
    Scalars* sc = rp.sc;
    const unsigned nb = min(sc->nbad[stage], (unsigned)rp.badcap);
    if (nb == 0) return;
    const Dims dm = dims_of(rp);
    const int n = dm.n;
    const int* __restrict__ list = rp.badlist + (size_t)stage * rp.badcap;
    T* __restrict__ Sout = (T*)rp.S[1];
    for (long w = (long)local * blockDim.x + threadIdx.x; w < 64L * nb; w += (long)kProtBlocks * blockDim.x) {
        int i, j, k;
        cell_ijk(dm, list[w / 64], i, j, k);
        const int o = (int)(w % 64);
        i += o % 4 - 1;
        j += (o / 4) % 4 - 1;
        k += o / 16 - 1;
        const int c = cell_at(dm, i, j, k);
        fld(Sout, 4, n)[c] = T(0.5) * (fld(Sout, 7, n)[c] + fld(Sout, 7, n)[cell_at(dm, i - 1, j, k)]);
        fld(Sout, 5, n)[c] = T(0.5) * (fld(Sout, 8, n)[c] + fld(Sout, 8, n)[cell_at(dm, i, j - 1, k)]);
        fld(Sout, 6, n)[c] = T(0.5) * (fld(Sout, 9, n)[c] + fld(Sout, 9, n)[cell_at(dm, i, j, k - 1)]);
    }
}

// The final stage's CFL maximum of the corrected state, into cfl_slots, when
// the stage had bad cells (k_finalize then takes it instead of the update's).
template <class T, bool ONE>
__global__ void __launch_bounds__(kRedThreads) k_prot_cfl(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindRed, local);
    if (!rp.active || !rp.protect) return;
    Scalars* sc = rp.sc;
    if (sc->nbad[1] == 0 || sc->drive) return;
    const T* __restrict__ S = (const T*)rp.S[1];
    const T asqr = (T)(rp.cs * rp.cs);
    const int n = rp.n, plane = rp.nx * rp.ny;
    double cm = 0.0;
    for (int c = local * blockDim.x + threadIdx.x; c < n; c += rp.nred * blockDim.x) {
        const int kc = c / plane;
        if (kc < rp.zlo || kc >= rp.zhi) continue;
        cm = nmax(cm, (double)cell_max_speed(fld(S, 0, n)[c], fld(S, 1, n)[c], fld(S, 2, n)[c], fld(S, 3, n)[c],
                                             fld(S, 4, n)[c], fld(S, 5, n)[c], fld(S, 6, n)[c], asqr));
    }
    block_atomic_max<kRedThreads>(sc->cfl_slots, cm);
}

// Clear the bad flags of a stage's list (the counts are reset by k_finalize).
template <bool ONE>
__global__ void __launch_bounds__(kBX) k_prot_clear(BatchArgs ba, int stage) {
    int local;
    const BoxRec rp = prot_box<ONE>(ba, local);
    if (!rp.active || !rp.protect) return;
    const unsigned nb = min(rp.sc->nbad[stage], (unsigned)rp.badcap);
    const int* __restrict__ list = rp.badlist + (size_t)stage * rp.badcap;
    for (long w = (long)local * blockDim.x + threadIdx.x; w < (long)nb; w += (long)kProtBlocks * blockDim.x)
        rp.bad[list[w]] = 0;
}

// ============================================================ passive scalars
// Upwind flux of compute_fluxes_1d (passive_mod.f90:594-627).  The
// reference's arithmetic form in FP32 too: a select of the upwind state
// (equal for finite operands) lets the compiler fold the two neighbour loads
// into one whose address waits on the velocity, and the z-marching passive
// predictor went from 1.35 to 1.61 ms at 512^3.
template <class T>
__device__ __forceinline__ T upwind_flux(T uL, T uR, T vavg) {
    T theta = (vavg >= T(0)) ? T(1) : T(-1);
    return T(0.5) * ((T(1) + theta) * uL + (T(1) - theta) * uR);
}
// The same flux where both states come from shared memory (the bulk-copy
// fed passive kernels): FP32 selects the upwind state, equal to the form
// above for finite operands, and there the select is cheaper (bulk-copy fed
// corrector 2.20 -> 2.05 ms at 512^3).
template <class T>
__device__ __forceinline__ T upwind_sel(T uL, T uR, T vavg) {
    if constexpr (sizeof(T) == 4) return (vavg >= T(0)) ? uL : uR;
    else return upwind_flux(uL, uR, vavg);
}
template <class T>
__device__ __forceinline__ T vel_of(const T* __restrict__ S, int n, int c, int comp) {
    T irho = T(1) / fld(S, 0, n)[c];
    return fld(S, 1 + comp, n)[c] * irho;
}

// Predictor: s_h = s - (dt/2dx) sum_d v_d (F_d(i+1/2) - F_d(i-1/2)) with
// first-order upwind fluxes and the step-start velocity (passive_mod.f90:
// 133-157, 204-224, 562-590).
// A thread walks a column of kSegZ cells along z, carrying the z velocity
// and the flux through the lower z face (the upper face's of the previous
// cell: the same operands).  The neighbour loads are
// latency-bound, so FP32 with up to four scalars runs eight blocks per SM
// (64 registers).
template <class T, bool ONE, int NP>
__global__ void __launch_bounds__(kBX, (sizeof(T) == 4 && NP <= 4) ? 8 : 1) k_passive_pred(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCellZ, local);
    const Scalars* sc = rp.sc;
    const int npass = rp.npass;
    if (!rp.active || npass == 0) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ SH = (T*)rp.SH;
    const double dx = rp.dx;
    int i, j, k0, k1;
    decode_cellz<ONE>(local, dm, rp.tws, rp.segzs, i, j, k0, k1);
    if (i >= dm.nx || j >= dm.ny) return;
    const int n = dm.n;
    const int plane = dm.nx * dm.ny;
    const T dtdx = (T)(0.5 * sc->dt / dx);
    const int r0 = i + dm.nx * j;
    const int rxm = wrap_dn(i, dm.nx) + dm.nx * j, rxp = wrap_up(i, dm.nx) + dm.nx * j;
    const int rym = i + dm.nx * wrap_dn(j, dm.ny), ryp = i + dm.nx * wrap_up(j, dm.ny);
    // z neighbours of the first cell
    const int ckm = r0 + wrap_dn(k0, dm.nz) * plane, ck0 = r0 + k0 * plane;
    T vz_0 = vel_of(S0, n, ck0, 2);
    T s_0[NP], fz_m[NP];
    {
        const T vz_m = vel_of(S0, n, ckm, 2);
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (p < npass) {
                s_0[p] = fld(S0, 10 + p, n)[ck0];
                fz_m[p] = upwind_flux(fld(S0, 10 + p, n)[ckm], s_0[p], T(0.5) * (vz_m + vz_0));
            }
    }
    for (int k = k0; k < k1; ++k) {
        const int c = r0 + k * plane, czp = r0 + wrap_up(k, dm.nz) * plane;
        const int cxm = rxm + k * plane, cxp = rxp + k * plane, cym = rym + k * plane, cyp = ryp + k * plane;
        const T vx0 = vel_of(S0, n, c, 0), vy0 = vel_of(S0, n, c, 1);
        const T vxm = vel_of(S0, n, cxm, 0), vxp = vel_of(S0, n, cxp, 0);
        const T vym = vel_of(S0, n, cym, 1), vyp = vel_of(S0, n, cyp, 1);
        const T vz_p = vel_of(S0, n, czp, 2);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (p >= npass) break;
            const T* s = fld(S0, 10 + p, n);
            const T s0 = s_0[p], s_zp = s[czp];
            T dF[3];
            dF[0] = upwind_flux(s0, s[cxp], T(0.5) * (vx0 + vxp)) - upwind_flux(s[cxm], s0, T(0.5) * (vxm + vx0));
            dF[1] = upwind_flux(s0, s[cyp], T(0.5) * (vy0 + vyp)) - upwind_flux(s[cym], s0, T(0.5) * (vym + vy0));
            const T fz_p = upwind_flux(s0, s_zp, T(0.5) * (vz_0 + vz_p));
            dF[2] = fz_p - fz_m[p];
            fld(SH, p, n)[c] = s0 - dtdx * (vx0 * dF[0] + vy0 * dF[1] + vz_0 * dF[2]);
            s_0[p] = s_zp;
            fz_m[p] = fz_p;
        }
        vz_0 = vz_p;
    }
}

// minmod slope (passive_mod.f90:517-532)
template <class T>
__device__ __forceinline__ T minmod(T wm, T w0, T wp) {
    T dL = w0 - wm;
    T dR = wp - w0;
    return T(0.5) * (sgn1(dL) + sgn1(dR)) * vmin(fabs(dL), fabs(dR));
}

// Corrector: MUSCL states from s_h, upwinded by the time-averaged velocity
// vel_tavg = (v_old + v_new)/2, applied to the step-start scalar
// (passive_mod.f90:159-201, 227-239).  mbnd holds, on drive steps, the
// unforced momentum of the boundary planes: [D][0] plane a = 0 and [D][1]
// plane a = n-1 of each axis (the ghost images the reference reads).
// The time-averaged velocity of cell c: the value the final update (or the
// kick) stored, or, across the global boundary on a drive step, that of the
// unforced momentum (unforced_m) computed here.
template <class T>
__device__ __forceinline__ T vtavg(const T* __restrict__ S0, const T* __restrict__ S1, const T* __restrict__ VT, int n,
                                   int c, int comp, const T* unforced_m) {
    if (!unforced_m) return VT[(size_t)(comp == 2 ? 6 : comp) * n + c];
    T vold = vel_of(S0, n, c, comp);
    T irho = T(1) / fld(S1, 0, n)[c];
    T m1 = *unforced_m;
    return T(0.5) * (vold + m1 * irho);
}

// A thread walks a column of kSegZ cells along z, carrying the z-neighbour
// time-averaged velocity, half-step scalars, their minmod slopes and the
// flux through the lower z face (the upper face's of the previous cell).
// Eight blocks per SM in FP32 with up to four scalars, as k_passive_pred
// (a few spilled values cost less than the lost occupancy).
template <class T, bool ONE, int NP>
__global__ void __launch_bounds__(kBX, (sizeof(T) == 4 && NP <= 4) ? 8 : 1) k_passive_corr(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCellZ, local);
    const Scalars* sc = rp.sc;
    const int npass = rp.npass;
    if (!rp.active || npass == 0) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ S1 = (T*)rp.S[1];
    const T* __restrict__ SH = (const T*)rp.SH;
    const T* __restrict__ VT = vt_field<T>(rp, 0);   // fields 0, 1 at +0, +n; field 2 at +6n (vt_field)
    const double dx = rp.dx;
    const int drive = sc->drive;
    const T* __restrict__ mbnd = (const T*)rp.mbnd;
    const int plane_stride = rp.plane_stride;
    int i, j, k0, k1;
    decode_cellz<ONE>(local, dm, rp.tws, rp.segzs, i, j, k0, k1);
    if (i >= dm.nx || j >= dm.ny) return;
    const int n = dm.n;
    const int plane = dm.nx * dm.ny;
    const T dtdx = (T)(sc->dt / dx);
    const int r0 = i + dm.nx * j;
    const int rxm = wrap_dn(i, dm.nx) + dm.nx * j, rxp = wrap_up(i, dm.nx) + dm.nx * j;
    const int rxm2 = wrap_any(i - 2, dm.nx) + dm.nx * j, rxp2 = wrap_any(i + 2, dm.nx) + dm.nx * j;
    const int rym = i + dm.nx * wrap_dn(j, dm.ny), ryp = i + dm.nx * wrap_up(j, dm.ny);
    const int rym2 = i + dm.nx * wrap_any(j - 2, dm.ny), ryp2 = i + dm.nx * wrap_any(j + 2, dm.ny);
    // on drive steps the velocity across the global boundary of axis d uses
    // the unforced momentum of the ghost image (mbnd planes, see k_force_kick)
    const T* um_x = (drive && i == 0) ? mbnd + (size_t)1 * plane_stride : nullptr;            // plane i = n-1
    const T* up_x = (drive && i == dm.nx - 1) ? mbnd + (size_t)0 * plane_stride : nullptr;    // plane i = 0
    const T* um_y = (drive && j == 0) ? mbnd + (size_t)3 * plane_stride : nullptr;
    const T* up_y = (drive && j == dm.ny - 1) ? mbnd + (size_t)2 * plane_stride : nullptr;
    const T* um_z = drive ? mbnd + (size_t)5 * plane_stride + (i + dm.nx * j) : nullptr;
    const T* up_z = drive ? mbnd + (size_t)4 * plane_stride + (i + dm.nx * j) : nullptr;
    // z neighbours of the first cell: velocity at k; scalars at k, k+1, the
    // minmod slope at k and the flux through the face k-1/2 (from the
    // velocities at k-1, k, the scalars at k-2..k+1 and the slopes at k-1, k)
    const int km = wrap_dn(k0, dm.nz);
    const int ckm = r0 + km * plane, ck0 = r0 + k0 * plane;
    T vz_0 = vtavg(S0, S1, VT, n, ck0, 2, (const T*)nullptr);
    T s_0[NP], s_p[NP], dl_0[NP], fz_m[NP];
    {
        const T vz_m = vtavg(S0, S1, VT, n, ckm, 2, (k0 == 0) ? um_z : (const T*)nullptr);
        const int ckm2 = r0 + wrap_any(k0 - 2, dm.nz) * plane, ckp = r0 + wrap_up(k0, dm.nz) * plane;
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (p < npass) {
                const T* s = fld(SH, p, n);
                const T sm2 = s[ckm2], sm = s[ckm];
                s_0[p] = s[ck0];
                s_p[p] = s[ckp];
                const T dlm = minmod(sm2, sm, s_0[p]);
                dl_0[p] = minmod(sm, s_0[p], s_p[p]);
                fz_m[p] = upwind_flux(sm + T(0.5) * dlm, s_0[p] - T(0.5) * dl_0[p], T(0.5) * (vz_m + vz_0));
            }
    }
    for (int k = k0; k < k1; ++k) {
        const int kp = wrap_up(k, dm.nz);
        const int c = r0 + k * plane, czp = r0 + kp * plane, czp2 = r0 + wrap_any(k + 2, dm.nz) * plane;
        const int cxm = rxm + k * plane, cxp = rxp + k * plane, cxm2 = rxm2 + k * plane, cxp2 = rxp2 + k * plane;
        const int cym = rym + k * plane, cyp = ryp + k * plane, cym2 = rym2 + k * plane, cyp2 = ryp2 + k * plane;
        const int pofs_x = j + dm.ny * k, pofs_y = i + dm.nx * k;
        const T vx0 = vtavg(S0, S1, VT, n, c, 0, (const T*)nullptr);
        const T vy0 = vtavg(S0, S1, VT, n, c, 1, (const T*)nullptr);
        const T vxm = vtavg(S0, S1, VT, n, cxm, 0, um_x ? um_x + pofs_x : (const T*)nullptr);
        const T vxp = vtavg(S0, S1, VT, n, cxp, 0, up_x ? up_x + pofs_x : (const T*)nullptr);
        const T vym = vtavg(S0, S1, VT, n, cym, 1, um_y ? um_y + pofs_y : (const T*)nullptr);
        const T vyp = vtavg(S0, S1, VT, n, cyp, 1, up_y ? up_y + pofs_y : (const T*)nullptr);
        const T vz_p = vtavg(S0, S1, VT, n, czp, 2, (k == dm.nz - 1) ? up_z : (const T*)nullptr);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (p >= npass) break;
            const T* s = fld(SH, p, n);
            const T s0 = s_0[p];
            T dF[3];
            {
                const T sm = s[cxm], sp = s[cxp], sm2 = s[cxm2], sp2 = s[cxp2];
                const T dlm = minmod(sm2, sm, s0), dl0 = minmod(sm, s0, sp), dlp = minmod(s0, sp, sp2);
                const T Fp = upwind_flux(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vx0 + vxp));
                const T Fm = upwind_flux(sm + T(0.5) * dlm, s0 - T(0.5) * dl0, T(0.5) * (vxm + vx0));
                dF[0] = Fp - Fm;
            }
            {
                const T sm = s[cym], sp = s[cyp], sm2 = s[cym2], sp2 = s[cyp2];
                const T dlm = minmod(sm2, sm, s0), dl0 = minmod(sm, s0, sp), dlp = minmod(s0, sp, sp2);
                const T Fp = upwind_flux(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vy0 + vyp));
                const T Fm = upwind_flux(sm + T(0.5) * dlm, s0 - T(0.5) * dl0, T(0.5) * (vym + vy0));
                dF[1] = Fp - Fm;
            }
            {
                const T sp = s_p[p], sp2 = s[czp2];
                const T dl0 = dl_0[p], dlp = minmod(s0, sp, sp2);
                const T Fp = upwind_flux(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vz_0 + vz_p));
                dF[2] = Fp - fz_m[p];
                fz_m[p] = Fp;
                s_0[p] = sp;
                s_p[p] = sp2;
                dl_0[p] = dlp;
            }
            fld(S1, 10 + p, n)[c] = fld(S0, 10 + p, n)[c] - dtdx * (vx0 * dF[0] + vy0 * dF[1] + vz_0 * dF[2]);
        }
        vz_0 = vz_p;
    }
}

// ------------------------------------------------------ passive corrector, bulk-copy fed
// The same corrector for single boxes whose rows are whole 128-cell tiles: a
// block owns a 128-cell segment of row j and walks kSegZ planes; lanes of
// warp 0 stream each plane's x/y stencil into shared memory with bulk
// asynchronous copies one plane ahead (two stages, mbarrier completion, as
// k_update_tma): per scalar the half-step rows j-2..j+2 (row j with 16-byte
// halo segments on both sides, for the x neighbours out to i +- 2) and the
// step-start row j; the time-averaged v_x of row j (halos on both sides) and
// v_y of rows j-1, j, j+1; and the new values of the z stencil, row j of each
// scalar at plane k+2 and of v_z at plane k+1 (the rest of the z stencil is
// carried).  On drive steps the neighbours
// across the global boundary take the unforced momentum (mbnd) as in
// k_passive_corr.  Waits are bounded (IMHD_S_WAIT on time-out).
template <class T, int NP>
constexpr int ptma_rows() { return 7 * NP + 5; }
template <class T>
constexpr int ptma_row_stride() { return kTmaTile + 2 * (16 / (int)sizeof(T)); }
template <class T, int NP>
constexpr size_t ptma_stage_bytes() {
    return ((size_t)ptma_rows<T, NP>() * ptma_row_stride<T>() * sizeof(T) + 127) / 128 * 128;
}
template <class T, int NP>
constexpr size_t passive_tma_smem_bytes() { return 2 * ptma_stage_bytes<T, NP>(); }

__host__ __device__ __forceinline__ bool passive_by_tma(int nx) { return nx % kTmaTile == 0; }

template <class T, int NP>
__global__ void __launch_bounds__(kTmaTile, 8) k_passive_corr_tma(BatchArgs ba) {
    extern __shared__ __align__(128) unsigned char ptma_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    const BoxRec rp = ba.one;
    Scalars* sc = rp.sc;
    const int npass = rp.npass;
    if (!rp.active || npass == 0) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ S1 = (T*)rp.S[1];
    const T* __restrict__ SH = (const T*)rp.SH;
    const T* __restrict__ VT = vt_field<T>(rp, 0);   // v_x, v_y at +0, +n; v_z at +6n
    const int drive = sc->drive;
    const T* __restrict__ mbnd = (const T*)rp.mbnd;
    const int plane_stride = rp.plane_stride;
    constexpr int HE = 16 / (int)sizeof(T);
    constexpr int RS = ptma_row_stride<T>();
    const int t = (int)threadIdx.x;
    const int i0 = (int)blockIdx.x * kTmaTile, j = (int)blockIdx.y, seg = (int)blockIdx.z;
    const int i = i0 + t;
    const int k0 = seg * kSegZ, k1 = min(k0 + kSegZ, dm.nz);
    const int n = dm.n, plane = dm.nx * dm.ny;
    const T dtdx = (T)(sc->dt / rp.dx);
    const int nrows = 7 * npass + 5;
    const int ih = (i0 == 0 ? dm.nx : i0) - HE;       // left halo: cells i0-HE .. i0-1
    const int ir = (i0 + kTmaTile) % dm.nx;            // right halo: cells i0+128 .. i0+128+HE-1
    // each staged row's source at plane 0 and plane offset (the z stencil's
    // rows lead by one or two planes), worked out once: scalar p: SH rows
    // j-2..j+2 at 6p..6p+4, step-start row j at 6p+5; then v_x row j, v_y
    // rows j-1, j, j+1; scalar p at k+2; v_z at k+1.  Rows 6p+2 and the v_x
    // row carry the 16-byte halo segments.
    __shared__ const T* row_src[ptma_rows<T, NP>()];
    __shared__ unsigned char row_dk[ptma_rows<T, NP>()];
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    for (int R = t; R < nrows; R += kTmaTile) {
        const T* base;
        int jr = j, dk = 0;
        if (R < 6 * npass) {
            const int p = R / 6, q = R % 6;
            if (q < 5) { base = fld(SH, p, n); jr = wrap_any(j + q - 2, dm.ny); }
            else base = fld(S0, 10 + p, n);
        } else if (R < 6 * npass + 4) {
            const int q = R - 6 * npass;
            if (q == 0) base = VT;
            else { base = VT + (size_t)n; jr = wrap_any(j + q - 2, dm.ny); }
        } else if (R < 7 * npass + 4) {
            base = fld(SH, R - 6 * npass - 4, n);
            dk = 2;
        } else {
            base = VT + (size_t)6 * n;
            dk = 1;
        }
        row_src[R] = base + i0 + (size_t)dm.nx * jr;
        row_dk[R] = (unsigned char)dk;
    }
    __syncthreads();
    const int hl = ih - i0, hr = ir - i0;       // halo segments relative to the row segment
    auto issue = [&](int g, int k) {
        T* rows = (T*)(ptma_smem + (size_t)g * ptma_stage_bytes<T, NP>());
        unsigned long long* bar = &bars[g];
        if (t == 0)
            mbar_expect_tx(bar, (unsigned)(nrows * kTmaTile * (int)sizeof(T) + (2 * npass + 2) * 16));
        __syncwarp();
        for (int R = t; R < nrows; R += 32) {
            int kr = k + row_dk[R];
            while (kr >= dm.nz) kr -= dm.nz;
            const T* src = row_src[R] + (size_t)plane * kr;
            bulk_g2s(rows + R * RS + HE, src, kTmaTile * (unsigned)sizeof(T), bar);
            if ((R < 6 * npass && R % 6 == 2) || R == 6 * npass) {
                bulk_g2s(rows + R * RS, src + hl, 16u, bar);
                bulk_g2s(rows + R * RS + HE + kTmaTile, src + hr, 16u, bar);
            }
        }
    };
    if (t < 32) issue(0, k0);

    const int r0 = i + dm.nx * j;
    // drive steps: the velocity across the global boundary of each axis uses
    // the unforced momentum of the ghost image (mbnd planes, see k_force_kick)
    const T* um_x = (drive && i == 0) ? mbnd + (size_t)1 * plane_stride : nullptr;
    const T* up_x = (drive && i == dm.nx - 1) ? mbnd + (size_t)0 * plane_stride : nullptr;
    const T* um_y = (drive && j == 0) ? mbnd + (size_t)3 * plane_stride : nullptr;
    const T* up_y = (drive && j == dm.ny - 1) ? mbnd + (size_t)2 * plane_stride : nullptr;
    const T* um_z = drive ? mbnd + (size_t)5 * plane_stride + r0 : nullptr;
    const T* up_z = drive ? mbnd + (size_t)4 * plane_stride + r0 : nullptr;
    const int rxm = wrap_dn(i, dm.nx) + dm.nx * j, rxp = wrap_up(i, dm.nx) + dm.nx * j;
    const int rym = i + dm.nx * wrap_dn(j, dm.ny), ryp = i + dm.nx * wrap_up(j, dm.ny);
    // z window of the column: v_z at k; scalars at k, k+1, the minmod slope
    // at k and the flux through the face k-1/2
    const int km = wrap_dn(k0, dm.nz);
    const int ckm = r0 + km * plane, ck0 = r0 + k0 * plane;
    T vz_0 = vtavg(S0, S1, VT, n, ck0, 2, (const T*)nullptr);
    T s_0[NP], s_p[NP], dl_0[NP], fz_m[NP];
    {
        const T vz_m = vtavg(S0, S1, VT, n, ckm, 2, (k0 == 0) ? um_z : (const T*)nullptr);
        const int ckm2 = r0 + wrap_any(k0 - 2, dm.nz) * plane, ckp = r0 + wrap_up(k0, dm.nz) * plane;
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (p < npass) {
                const T* s = fld(SH, p, n);
                const T sm2 = s[ckm2], sm = s[ckm];
                s_0[p] = s[ck0];
                s_p[p] = s[ckp];
                const T dlm = minmod(sm2, sm, s_0[p]);
                dl_0[p] = minmod(sm, s_0[p], s_p[p]);
                fz_m[p] = upwind_flux(sm + T(0.5) * dlm, s_0[p] - T(0.5) * dl_0[p], T(0.5) * (vz_m + vz_0));
            }
    }
    bool ok = true;
    for (int k = k0; k < k1; ++k) {
        const int it = k - k0, g = it & 1;
        if (t < 32 && k + 1 < k1) issue(g ^ 1, k + 1);
        if (ok && !mbar_wait(&bars[g], (unsigned)((it >> 1) & 1))) {
            ok = false;
            atomicOr(&sc->status, kStatusWait);
        }
        if (ok) {
            const T* rows = (const T*)(ptma_smem + (size_t)g * ptma_stage_bytes<T, NP>()) + HE + t;
            auto at = [&](int R, int dx) { return rows[R * RS + dx]; };
            const int c = r0 + k * plane;
            const int czp = r0 + wrap_up(k, dm.nz) * plane;
            const int vx_row = 6 * npass, vy_row = 6 * npass + 1;
            const T vx0 = at(vx_row, 0), vy0 = at(vy_row + 1, 0);
            const T vxm = um_x ? vtavg(S0, S1, VT, n, rxm + k * plane, 0, um_x + (j + dm.ny * k)) : at(vx_row, -1);
            const T vxp = up_x ? vtavg(S0, S1, VT, n, rxp + k * plane, 0, up_x + (j + dm.ny * k)) : at(vx_row, 1);
            const T vym = um_y ? vtavg(S0, S1, VT, n, rym + k * plane, 1, um_y + (i + dm.nx * k)) : at(vy_row, 0);
            const T vyp = up_y ? vtavg(S0, S1, VT, n, ryp + k * plane, 1, up_y + (i + dm.nx * k)) : at(vy_row + 2, 0);
            const T vz_p = (drive && k == dm.nz - 1) ? vtavg(S0, S1, VT, n, czp, 2, up_z) : at(7 * npass + 4, 0);
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                if (p >= npass) break;
                const int rj = 6 * p + 2;      // row j of scalar p
                const T s0 = s_0[p];
                T dF[3];
                {
                    const T sm = at(rj, -1), sp = at(rj, 1), sm2 = at(rj, -2), sp2 = at(rj, 2);
                    const T dlm = minmod(sm2, sm, s0), dl0 = minmod(sm, s0, sp), dlp = minmod(s0, sp, sp2);
                    const T Fp = upwind_sel(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vx0 + vxp));
                    const T Fm = upwind_sel(sm + T(0.5) * dlm, s0 - T(0.5) * dl0, T(0.5) * (vxm + vx0));
                    dF[0] = Fp - Fm;
                }
                {
                    const T sm = at(rj - 1, 0), sp = at(rj + 1, 0), sm2 = at(rj - 2, 0), sp2 = at(rj + 2, 0);
                    const T dlm = minmod(sm2, sm, s0), dl0 = minmod(sm, s0, sp), dlp = minmod(s0, sp, sp2);
                    const T Fp = upwind_sel(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vy0 + vyp));
                    const T Fm = upwind_sel(sm + T(0.5) * dlm, s0 - T(0.5) * dl0, T(0.5) * (vym + vy0));
                    dF[1] = Fp - Fm;
                }
                {
                    const T sp = s_p[p], sp2 = at(6 * npass + 4 + p, 0);
                    const T dl0 = dl_0[p], dlp = minmod(s0, sp, sp2);
                    const T Fp = upwind_sel(s0 + T(0.5) * dl0, sp - T(0.5) * dlp, T(0.5) * (vz_0 + vz_p));
                    dF[2] = Fp - fz_m[p];
                    fz_m[p] = Fp;
                    s_0[p] = sp;
                    s_p[p] = sp2;
                    dl_0[p] = dlp;
                }
                fld(S1, 10 + p, n)[c] = at(6 * p + 5, 0) - dtdx * (vx0 * dF[0] + vy0 * dF[1] + vz_0 * dF[2]);
            }
            vz_0 = vz_p;
        }
        __syncthreads();   // every thread is done with stage g before it is refilled
    }
    // a wait that gave up may leave copies in flight: let them land (bounded) before exit
    if (t == 0 && !ok) {
        const int last = k1 - 1 - k0;
        mbar_wait(&bars[last & 1], (unsigned)((last >> 1) & 1));
    }
}

// ------------------------------------------------------ passive predictor, bulk-copy fed
// k_passive_pred for single boxes whose rows are whole 128-cell tiles: a block
// owns a 128-cell segment of row j and walks kSegZ planes; lanes of warp 0
// stream each plane's rows into shared memory with bulk asynchronous copies
// one plane ahead (two stages, mbarrier completion, bounded waits as in
// k_update_tma): density and momenta of row j (density and x momentum with
// 16-byte halos on both sides), density and y momentum of rows j-1 and j+1,
// each scalar of row j (both halos), j-1 and j+1; the row sources are worked
// out once per block.  The z faces run one plane behind: at plane k the face
// k-1/2 completes cell k-1, and the last cell of the segment takes the plane
// above from global memory.  The same operations on the same operands: the
// results are those of k_passive_pred.
template <int NP>
constexpr int ppred_rows() { return 8 + 3 * NP; }
template <class T, int NP>
constexpr size_t ppred_stage_bytes() {
    return ((size_t)ppred_rows<NP>() * ptma_row_stride<T>() * sizeof(T) + 127) / 128 * 128;
}
template <class T, int NP>
constexpr size_t passive_pred_tma_smem_bytes() { return 2 * ppred_stage_bytes<T, NP>(); }

// FP32 occupancy: ten blocks per SM with up to two scalars (47 registers, no
// spills: 1.32 -> 1.21 ms at 512^3), eight with four (ten spill).
template <class T, int NP>
__global__ void __launch_bounds__(kTmaTile, sizeof(T) == 4 ? (NP <= 2 ? 10 : NP <= 4 ? 8 : 1) : 1)
    k_passive_pred_tma(BatchArgs ba) {
    extern __shared__ __align__(128) unsigned char pptma_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ const T* row_src[ppred_rows<NP>()];
    const BoxRec rp = ba.one;
    const Scalars* sc = rp.sc;
    const int npass = rp.npass;
    if (!rp.active || npass == 0) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ SH = (T*)rp.SH;
    constexpr int HE = 16 / (int)sizeof(T);
    constexpr int RS = ptma_row_stride<T>();
    const int t = (int)threadIdx.x;
    const int i0 = (int)blockIdx.x * kTmaTile, i = i0 + t, j = (int)blockIdx.y;
    const int k0 = (int)blockIdx.z * kSegZ, k1 = min(k0 + kSegZ, dm.nz);
    const int n = dm.n, plane = dm.nx * dm.ny;
    const int ih = (i0 == 0 ? dm.nx : i0) - HE;       // left halo: cells i0-HE .. i0-1
    const int ir = (i0 + kTmaTile) % dm.nx;            // right halo: cells i0+128 .. i0+128+HE-1
    const int hl = ih - i0, hr = ir - i0;
    const unsigned copy_bytes = (unsigned)((8 + 3 * npass) * kTmaTile * (int)sizeof(T) + 2 * (2 + npass) * 16);
    if (t == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    // rows 0-3: fields 0-3 of row j (0 and 1 with both halos); 4, 5: fields
    // 0 and 2 of row j-1; 6, 7: the same of row j+1; from 8: scalar p of row
    // j (both halos) at 8 + p, of row j-1 at 8 + NP + p, of row j+1 at
    // 8 + 2 NP + p (none for p >= npass)
    for (int R = t; R < ppred_rows<NP>(); R += kTmaTile) {
        const T* base = nullptr;
        int jr = j;
        if (R < 4) base = fld(S0, R, n);
        else if (R < 8) { base = fld(S0, (R & 1) ? 2 : 0, n); jr = R < 6 ? wrap_dn(j, dm.ny) : wrap_up(j, dm.ny); }
        else {
            const int q = R - 8, which = q / NP, p = q % NP;
            if (p < npass) {
                base = fld(S0, 10 + p, n);
                jr = which == 0 ? j : which == 1 ? wrap_dn(j, dm.ny) : wrap_up(j, dm.ny);
            }
        }
        row_src[R] = base ? base + i0 + (size_t)dm.nx * jr : nullptr;
    }
    __syncthreads();
    auto issue = [&](int g, int k) {
        T* rows = (T*)(pptma_smem + (size_t)g * ppred_stage_bytes<T, NP>());
        unsigned long long* bar = &bars[g];
        if (t == 0) mbar_expect_tx(bar, copy_bytes);
        __syncwarp();
        for (int R = t; R < ppred_rows<NP>(); R += 32) {
            const T* src0 = row_src[R];
            if (!src0) continue;
            const T* src = src0 + (size_t)plane * k;
            T* dst = rows + R * RS;
            bulk_g2s(dst + HE, src, kTmaTile * (unsigned)sizeof(T), bar);
            if (R < 2 || (R >= 8 && R < 8 + NP)) {
                bulk_g2s(dst, src + hl, 16u, bar);
                bulk_g2s(dst + HE + kTmaTile, src + hr, 16u, bar);
            }
        }
    };
    if (t < 32) issue(0, k0);
    const T dtdx = (T)(0.5 * sc->dt / rp.dx);
    const int r0 = i + dm.nx * j;
    // carried from plane k-1: scalar, velocities, x and y flux differences, z face below
    T ps[NP], pdx[NP], pdy[NP], pfz[NP];
    T pvx = T(0), pvy = T(0), pvz;
    {
        const int czm = r0 + wrap_dn(k0, dm.nz) * plane;
        pvz = vel_of(S0, n, czm, 2);
#pragma unroll
        for (int p = 0; p < NP; ++p)
            if (p < npass) ps[p] = fld(S0, 10 + p, n)[czm];
    }
    bool ok = true;
    for (int k = k0; k < k1; ++k) {
        const int it = k - k0, g = it & 1;
        if (t < 32 && k + 1 < k1) issue(g ^ 1, k + 1);
        if (ok && !mbar_wait(&bars[g], (unsigned)((it >> 1) & 1))) {
            ok = false;
            atomicOr(&rp.sc->status, kStatusWait);
        }
        if (ok) {
            const T* rows = (const T*)(pptma_smem + (size_t)g * ppred_stage_bytes<T, NP>()) + HE + t;
            auto at = [&](int R, int dx) { return rows[R * RS + dx]; };
            // velocities as vel_of: m * (1 / rho)
            const T vx0 = at(1, 0) * (T(1) / at(0, 0)), vy0 = at(2, 0) * (T(1) / at(0, 0));
            const T vz0 = at(3, 0) * (T(1) / at(0, 0));
            const T vxm = at(1, -1) * (T(1) / at(0, -1));
            const T vxp = at(1, 1) * (T(1) / at(0, 1));
            const T vym = at(5, 0) * (T(1) / at(4, 0));
            const T vyp = at(7, 0) * (T(1) / at(6, 0));
            const int c = r0 + k * plane;
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                if (p >= npass) break;
                const int rs = 8 + p;
                const T s0 = at(rs, 0), sxm = at(rs, -1), sxp = at(rs, 1);
                const T sym = at(rs + NP, 0), syp = at(rs + 2 * NP, 0);
                const T dfx = upwind_sel(s0, sxp, T(0.5) * (vx0 + vxp)) - upwind_sel(sxm, s0, T(0.5) * (vxm + vx0));
                const T dfy = upwind_sel(s0, syp, T(0.5) * (vy0 + vyp)) - upwind_sel(sym, s0, T(0.5) * (vym + vy0));
                const T fz = upwind_sel(ps[p], s0, T(0.5) * (pvz + vz0));   // face k-1/2
                if (k > k0) fld(SH, p, n)[c - plane] = ps[p] - dtdx * (pvx * pdx[p] + pvy * pdy[p] + pvz * (fz - pfz[p]));
                ps[p] = s0;
                pdx[p] = dfx;
                pdy[p] = dfy;
                pfz[p] = fz;
            }
            pvx = vx0;
            pvy = vy0;
            pvz = vz0;
        }
        __syncthreads();   // every thread is done with stage g before it is refilled
    }
    if (ok) {   // the last cell of the column: its face above takes plane k1 (periodic) from global memory
        const int cup = r0 + wrap_up(k1 - 1, dm.nz) * plane;
        const T vzu = vel_of(S0, n, cup, 2);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (p >= npass) break;
            const T fz = upwind_flux(ps[p], fld(S0, 10 + p, n)[cup], T(0.5) * (pvz + vzu));
            fld(SH, p, n)[r0 + (k1 - 1) * plane] = ps[p] - dtdx * (pvx * pdx[p] + pvy * pdy[p] + pvz * (fz - pfz[p]));
        }
    }
    if (t == 0 && !ok) {   // copies left in flight after a wait gave up: let them land (bounded)
        const int last = k1 - 1 - k0;
        mbar_wait(&bars[last & 1], (unsigned)((last >> 1) & 1));
    }
}

// ============================================================ forcing
// get_rho_turb sums (turb_driver_mod.f90:158-186) over the step-start state,
// per-block partial sums in FP64, reduced in a fixed order by k_force_reduce.
// sums_only: the sums of this box for the host (slab ranks add them up,
// turb_driver_mod.f90:184-189), whatever the drive flag; otherwise the sums
// of a drive step, unless the host has set all ranks' sums (ext_sums).
template <class T, bool ONE>
__global__ void __launch_bounds__(kRedThreads) k_force_sums(BatchArgs ba, int sums_only) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindRed, local);
    const Scalars* sc = rp.sc;
    if (!rp.active || (!sums_only && (!sc->drive || sc->ext_sums))) return;
    const T* __restrict__ S0 = (const T*)rp.S[0];
    const T* __restrict__ delv = (const T*)rp.delv;
    double* __restrict__ partials = rp.partials;
    const int n = rp.n;
    double s[5] = {0, 0, 0, 0, 0};
    const int plane = rp.nx * rp.ny;
    for (int c = local * blockDim.x + threadIdx.x; c < n; c += rp.nred * blockDim.x) {
        const int kc = c / plane;
        if (kc < rp.zlo || kc >= rp.zhi) continue;
        double rho = (double)fld(S0, 0, n)[c];
        double d1 = (double)delv[c], d2 = (double)delv[(size_t)n + c], d3 = (double)delv[2 * (size_t)n + c];
        s[0] += rho * (d1 * d1 + d2 * d2 + d3 * d3);
        s[1] += d1 * (double)fld(S0, 1, n)[c] + d2 * (double)fld(S0, 2, n)[c] + d3 * (double)fld(S0, 3, n)[c];
        s[2] += rho * d1;
        s[3] += rho * d2;
        s[4] += rho * d3;
    }
    __shared__ double red[5][8];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        double v = warp_sum(s[q]);
        if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        partials[(size_t)local * 5 + threadIdx.x] = v;
    }
}

// The constant-energy normalisation of add_random_force from the five sums
// (turb_driver_mod.f90:411-434): <rho delv> and constE, the larger root of
// the kinetic-energy quadratic.
__device__ __forceinline__ void force_normalise(Scalars* sc, const double* s, double dx, double edot, double dt_turb) {
    double dx3 = dx * dx * dx;
    if (s[0] <= 1.0e-20) {
        sc->status |= 8u;
        sc->constE = 0.0;
        sc->mavg[0] = sc->mavg[1] = sc->mavg[2] = 0.0;
        return;
    }
    sc->mavg[0] = s[2] * dx3;
    sc->mavg[1] = s[3] * dx3;
    sc->mavg[2] = s[4] * dx3;
    double tmp1 = edot * dt_turb / dx3;
    double tmp2 = sqrt(s[1] * s[1] + (4.0 * tmp1 * s[0]));
    sc->constE = 0.5 * (-s[1] + tmp2) / s[0];
}

// Sum the per-block partials in block order, then the normalisation of
// add_random_force (turb_driver_mod.f90:411-434).  The sums are this box's,
// or all ranks' when the host set them (ext_sums, consumed here);
// sums_only stops after storing this box's sums.
static __global__ void k_force_reduce(BatchArgs ba, int sums_only) {
    const BoxRec rp = box_at(ba, blockIdx.x);   // one block of 32 threads per box
    Scalars* sc = rp.sc;
    if (!rp.active || (!sums_only && !sc->drive)) return;
    if (!sums_only && sc->ext_sums) {
        if (threadIdx.x == 0) {
            sc->ext_sums = 0u;
            double s[5];
            for (int q = 0; q < 5; ++q) s[q] = sc->sums[q];
            force_normalise(sc, s, rp.dx, rp.edot, rp.dt_turb);
        }
        return;
    }
    const double* __restrict__ partials = rp.partials;
    const int nblocks = rp.nred;
    const double dx = rp.dx, edot = rp.edot, dt_turb = rp.dt_turb;
    __shared__ double acc[5][32];
    int t = threadIdx.x;
    for (int q = 0; q < 5; ++q) {
        double v = 0.0;
        for (int b = t; b < nblocks; b += 32) v += partials[(size_t)b * 5 + q];
        acc[q][t] = v;
    }
    __syncwarp();
    if (t == 0) {
        double s[5];
        for (int q = 0; q < 5; ++q) {
            double v = 0.0;
            for (int w = 0; w < 32; ++w) v += acc[q][w];
            s[q] = v;
        }
        s[0] = 0.5 * s[0];
        for (int q = 0; q < 5; ++q) sc->sums[q] = s[q];
        if (!sums_only) force_normalise(sc, s, dx, edot, dt_turb);
    }
}

// Kick m += constE (rho0 delv - <rho delv>) on the new state
// (turb_driver_mod.f90:437-453), delv_max, the CFL maximum of the kicked
// state, and the unforced boundary-plane momentum for k_passive_corr.
template <class T, bool ONE>
__global__ void __launch_bounds__(kBX) k_force_kick(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCell, local);
    Scalars* sc = rp.sc;
    if (!rp.active || !sc->drive) return;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S0 = (const T*)rp.S[0];
    T* __restrict__ S1 = (T*)rp.S[1];
    const T* __restrict__ delv = (const T*)rp.delv;
    T* __restrict__ mbnd = (T*)rp.mbnd;
    const int plane_stride = rp.plane_stride;
    const int save_bnd = rp.npass > 0;
    const T asqr = (T)(rp.cs * rp.cs);
    int i, j, k;
    decode_cell<ONE>(local, dm, rp.tws, i, j, k);
    bool valid = i < dm.nx && j < dm.ny;
    const bool inz = k >= rp.zlo && k < rp.zhi;
    double dvmax = 0.0, cmax = 0.0;
    if (valid) {
        const int n = dm.n;
        int c = i + dm.nx * (j + dm.ny * k);
        if (save_bnd) {
            int idx[3] = {i, j, k};
            int nn[3] = {dm.nx, dm.ny, dm.nz};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                int a = (d == 0) ? j : i;
                int b = (d == 2) ? j : k;
                int pn = (d == 0) ? dm.ny : dm.nx;
                int pofs = a + pn * b;
                if (idx[d] == 0) mbnd[(size_t)(2 * d + 0) * plane_stride + pofs] = fld(S1, 1 + d, n)[c];
                if (idx[d] == nn[d] - 1) mbnd[(size_t)(2 * d + 1) * plane_stride + pofs] = fld(S1, 1 + d, n)[c];
            }
        }
        double constE = sc->constE;
        double r0 = (double)fld(S0, 0, n)[c];
        double dmx = constE * (r0 * (double)delv[c] - sc->mavg[0]);
        double dmy = constE * (r0 * (double)delv[(size_t)n + c] - sc->mavg[1]);
        double dmz = constE * (r0 * (double)delv[2 * (size_t)n + c] - sc->mavg[2]);
        T mx = (T)((double)fld(S1, 1, n)[c] + dmx);
        T my = (T)((double)fld(S1, 2, n)[c] + dmy);
        T mz = (T)((double)fld(S1, 3, n)[c] + dmz);
        fld(S1, 1, n)[c] = mx;
        fld(S1, 2, n)[c] = my;
        fld(S1, 3, n)[c] = mz;
        if (save_bnd) {   // the time-averaged velocity of the kicked momentum
            const T rho0 = fld(S0, 0, n)[c], rho1 = fld(S1, 0, n)[c];
            vt_field<T>(rp, 0)[c] = vt_of(rho0, fld(S0, 1, n)[c], rho1, mx);
            vt_field<T>(rp, 1)[c] = vt_of(rho0, fld(S0, 2, n)[c], rho1, my);
            vt_field<T>(rp, 2)[c] = vt_of(rho0, fld(S0, 3, n)[c], rho1, mz);
        }
        if (inz) dvmax = vmax(vmax(vmax(dvmax, fabs(dmx) / r0), fabs(dmy) / r0), fabs(dmz) / r0);
        if (inz) cmax = (double)cell_max_speed(fld(S1, 0, n)[c], mx, my, mz, fld(S1, 4, n)[c], fld(S1, 5, n)[c],
                                      fld(S1, 6, n)[c], asqr);
    }
    block_atomic_max<kBX>(sc->dvmax_slots, dvmax);
    block_atomic_max<kBX>(sc->cmax_slots, cmax);
}

// ============================================================ dt and maxima
// compute_new_time_step (driver.f90:432-448) with the smax coupling of
// get_max_speed_vanleer (vanleer_mod.f90:3323); resets the step maxima.
static __global__ void k_finalize(BatchArgs ba, int device_driven) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ba.nbox) return;
    const BoxRec rp = box_at(ba, b);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    const double cour = rp.cour, dx = rp.dx;
    const int drive = sc->drive;
    double cell = 0.0, smax = 0.0, dvm = 0.0;
    // after a protected final update with bad cells the CFL maximum of the
    // corrected state is in cfl_slots (k_prot_cfl)
    const bool protected_cfl = rp.protect && sc->nbad[1] > 0 && !drive;
    for (int s = 0; s < kSlots; ++s) {
        cell = nmax(cell, __longlong_as_double((long long)(protected_cfl ? sc->cfl_slots[s] : sc->cmax_slots[s])));
        smax = nmax(smax, __longlong_as_double((long long)sc->smax_slots[s]));
        dvm = nmax(dvm, __longlong_as_double((long long)sc->dvmax_slots[s]));
        sc->cmax_slots[s] = 0ull;
        sc->smax_slots[s] = 0ull;
        sc->dvmax_slots[s] = 0ull;
        if (rp.protect) sc->cfl_slots[s] = 0ull;
    }
    sc->nbad[0] = sc->nbad[1] = 0u;
    double cmax = vmax(cell, smax + dvm);
    if (!(cmax == cmax) || cmax > 1.0e300) sc->status |= 2u;
    if (cmax < kZERO) sc->status |= 4u;
    double c = drive ? 0.5 * cour : cour;
    sc->cmax = cmax;
    sc->smax_last = smax;
    sc->dvmax_last = dvm;
    sc->dt_next = c * dx / cmax;
    sc->cur ^= 1;   // the new state is now current
    if (!ba.use_one) {
        BoxRec& tr = ba.boxes[b];
        void* s0 = tr.S[0];
        tr.S[0] = tr.S[1];
        tr.S[1] = s0;
    }
    if (device_driven) {
        // driver.f90:86-87 and :475 for this box
        sc->t = sc->t + sc->dt;
        sc->steps_done += 1;
        if (sc->steps_done >= sc->steps_target || !(sc->t < sc->t_end) || (sc->status & (6u | kStatusProtect))) {
            sc->active = 0;
            if (!ba.use_one) ba.boxes[b].active = 0;
        } else {
            sc->dt = vmin(sc->t_end - sc->t, sc->dt_next);
        }
        sc->drive = 0;
    }
}

// Drive decision of a device-driven step (driver.f90:57-70): a box drives
// when t_turb falls in (t, t + dt]; then t_turb advances and dt halves.
static __global__ void k_batch_begin(BatchArgs ba) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ba.nbox) return;
    const BoxRec rp = box_at(ba, b);
    Scalars* sc = rp.sc;
    if (!rp.active) return;
    int drive = 0;
    if (sc->forcing && (sc->t_turb > sc->t) && (sc->t_turb <= sc->t + sc->dt)) {
        drive = 1;
        sc->t_turb = vmax(sc->t_turb + sc->dt_turb_sched, sc->t + 1.0e-2 * sc->dt);
        sc->dt = 0.5 * sc->dt;
    }
    sc->drive = drive;
}

// Clocks of every box of a table, kClockWords doubles per box:
// t, steps made, running flag, current buffer, status bits, next dt.
constexpr int kClockWords = 6;
static __global__ void k_clocks(BatchArgs ba, double* __restrict__ out) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= ba.nbox) return;
    const Scalars* sc = box_at(ba, b).sc;
    double* o = out + (size_t)b * kClockWords;
    o[0] = sc->t;
    o[1] = (double)sc->steps_done;
    o[2] = (double)sc->active;
    o[3] = (double)sc->cur;
    o[4] = (double)sc->status;
    o[5] = sc->dt;
}

// cell fast-speed maximum of a state (imhd_max_speed)
template <class T, bool ONE>
__global__ void __launch_bounds__(kBX) k_cfl(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindCell, local);
    Scalars* sc = rp.sc;
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[0];
    const T asqr = (T)(rp.cs * rp.cs);
    unsigned long long* out_slots = sc->cfl_slots;
    int i, j, k;
    decode_cell<ONE>(local, dm, rp.tws, i, j, k);
    double cm = 0.0;
    if (i < dm.nx && j < dm.ny && k >= rp.zlo && k < rp.zhi) {
        const int n = dm.n;
        int c = i + dm.nx * (j + dm.ny * k);
        cm = (double)cell_max_speed(fld(S, 0, n)[c], fld(S, 1, n)[c], fld(S, 2, n)[c], fld(S, 3, n)[c],
                                    fld(S, 4, n)[c], fld(S, 5, n)[c], fld(S, 6, n)[c], asqr);
    }
    block_atomic_max<kBX>(out_slots, cm);
}

// ============================================================ diagnostics
// compute_KE (driver.f90:518-553) and compute_divB (:492-515) as FP64
// per-block partials; reduced by k_diag_reduce in block order.
template <class T, bool ONE>
__global__ void __launch_bounds__(kRedThreads) k_diag(BatchArgs ba) {
    int local;
    const BoxRec rp = resolve<ONE>(ba, kKindRed, local);
    const Dims dm = dims_of(rp);
    const T* __restrict__ S = (const T*)rp.S[0];
    double* __restrict__ partials = rp.partials;
    const int n = dm.n;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int c = local * blockDim.x + threadIdx.x; c < n; c += rp.nred * blockDim.x) {
        int i = c % dm.nx, j = (c / dm.nx) % dm.ny, k = c / (dm.nx * dm.ny);
        if (k < rp.zlo || k >= rp.zhi) continue;
        double rho = vmin(vmax((double)fld(S, 0, n)[c], 1.0e-15), 1.0e10);
        double mx = (double)fld(S, 1, n)[c], my = (double)fld(S, 2, n)[c], mz = (double)fld(S, 3, n)[c];
        double vsqr = vmin((mx * mx + my * my + mz * mz) / (rho * rho), 1.0e5);
        s[1] += vsqr;
        s[0] += rho * vsqr;
        s[2] += mx; s[3] += my; s[4] += mz;
        int cxm = wrap_dn(i, dm.nx) + dm.nx * (j + dm.ny * k);
        int cym = i + dm.nx * (wrap_dn(j, dm.ny) + dm.ny * k);
        int czm = i + dm.nx * (j + dm.ny * wrap_dn(k, dm.nz));
        s[5] += ((double)fld(S, 7, n)[c] - (double)fld(S, 7, n)[cxm]) + ((double)fld(S, 8, n)[c] - (double)fld(S, 8, n)[cym]) +
                ((double)fld(S, 9, n)[c] - (double)fld(S, 9, n)[czm]);
    }
    __shared__ double red[6][8];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double v = warp_sum(s[q]);
        if (lane == 0) red[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        partials[(size_t)local * 6 + threadIdx.x] = v;
    }
}

static __global__ void k_diag_reduce(BatchArgs ba) {
    if (threadIdx.x != 0) return;
    const BoxRec rp = box_at(ba, blockIdx.x);   // one block per box
    Scalars* sc = rp.sc;
    const double* __restrict__ partials = rp.partials;
    const int nblocks = rp.nred;
    const double dx = rp.dx;
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nblocks; ++b)
        for (int q = 0; q < 6; ++q) s[q] += partials[(size_t)b * 6 + q];
    double dx3 = dx * dx * dx;
    sc->diag[0] = 0.5 * s[0] * dx3;
    sc->diag[1] = s[1] * dx3;
    sc->diag[2] = s[2] * dx3;
    sc->diag[3] = s[3] * dx3;
    sc->diag[4] = s[4] * dx3;
    sc->diag[5] = s[5];
}

// ============================================================ Fourier fields
// v_d(x) = sum_m 2 Re(A_{m,d} exp(2 pi i k_m . x)) on the cell centres
// x = ((i+1/2)/nx, (j+1/2)/ny, (k+1/2)/nz): the solenoidal OU forcing and
// initial velocity fields (shells 1 <= |k| <= 2 carry ~16 modes).  target 0
// adds rho * scale * v to the momentum of state S[cur]; target 1 writes
// scale * v to the force field.  Phases are reduced in FP64.
template <class T>
__global__ void __launch_bounds__(kBX) k_fourier_field(BoxRec r, int cur, int target, const int* __restrict__ kv,
                                                       const double* __restrict__ amp, int nm, double scale) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= r.n) return;
    int i = c % r.nx, j = (c / r.nx) % r.ny, k = c / (r.nx * r.ny);
    double x = (i + 0.5) / r.nx, y = (j + 0.5) / r.ny, z = (k + 0.5) / r.nz;
    double v[3] = {0.0, 0.0, 0.0};
    for (int m = 0; m < nm; ++m) {
        double ph = kv[3 * m] * x + kv[3 * m + 1] * y + kv[3 * m + 2] * z;
        ph = 2.0 * (ph - floor(ph));
        double s, co;
        sincospi(ph, &s, &co);
#pragma unroll
        for (int d = 0; d < 3; ++d) v[d] += 2.0 * (amp[6 * m + 2 * d] * co - amp[6 * m + 2 * d + 1] * s);
    }
    if (target == 0) {
        T* S = (T*)(cur ? r.S[1] : r.S[0]);
        double rho = (double)S[c];
#pragma unroll
        for (int d = 0; d < 3; ++d) S[(size_t)(1 + d) * r.n + c] = (T)((double)S[(size_t)(1 + d) * r.n + c] + rho * scale * v[d]);
    } else {
        T* D = (T*)r.delv;
#pragma unroll
        for (int d = 0; d < 3; ++d) D[(size_t)d * r.n + c] = (T)(scale * v[d]);
    }
}

// Separable inverse DFT of the reference force generator
// (turb_driver_mod.f90:313-384, direct_idft_1d :461-486), one axis per pass,
// interior cells only.  A spectrum line of 2*km entries (k = -km..km-1) is
// summed over k = -(km-1)..km-1 in that order with the twiddles cos/sin of
// theta0 * i * k (i the 1-based cell index), tabulated on the host as
// tw[i0 * (2km-1) + (k + km-1)] (cos) and tw[ntw + ...] (sin).
__device__ __forceinline__ void idft_line(const double* __restrict__ re, const double* __restrict__ im, int stride,
                                          const double* __restrict__ cs, const double* __restrict__ sn, int km,
                                          double& ore, double& oim) {
    ore = 0.0;
    oim = 0.0;
    for (int jj = -(km - 1); jj <= km - 1; ++jj) {
        const double vr = re[(size_t)(jj + km) * stride], vi = im[(size_t)(jj + km) * stride];
        const double c = cs[jj + km - 1], s = sn[jj + km - 1];
        ore = ore + (vr * c + (-1.0) * vi * s);
        oim = oim + (vi * c - (-1.0) * vr * s);
    }
}

// pass 1: V[c][kz][ky][kx] (each of 2km) -> A1[c][kz][ky][x]
static __global__ void k_idft_x(const double* __restrict__ Vre, const double* __restrict__ Vim,
                                const double* __restrict__ tw, int ntw, int km, int nx, double* __restrict__ Are,
                                double* __restrict__ Aim) {
    const int nk = 2 * km;
    const long long total = 3LL * nk * nk * nx;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int x = (int)(t % nx);
        long long line = t / nx;               // (c, kz, ky)
        const double* cs = tw + (size_t)x * (nk - 1);
        double ore, oim;
        idft_line(Vre + line * nk, Vim + line * nk, 1, cs, cs + ntw, km, ore, oim);
        Are[t] = ore;
        Aim[t] = oim;
    }
}
// pass 2: A1[c][kz][ky][x] -> A2[c][kz][y][x]
static __global__ void k_idft_y(const double* __restrict__ Are, const double* __restrict__ Aim,
                                const double* __restrict__ tw, int ntw, int km, int nx, int ny,
                                double* __restrict__ Bre, double* __restrict__ Bim) {
    const int nk = 2 * km;
    const long long total = 3LL * nk * ny * nx;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int x = (int)(t % nx);
        int y = (int)((t / nx) % ny);
        long long ckz = t / ((long long)nx * ny);  // (c, kz)
        const double* cs = tw + (size_t)y * (nk - 1);
        const size_t base = (size_t)ckz * nk * nx + x;
        double ore, oim;
        idft_line(Are + base, Aim + base, nx, cs, cs + ntw, km, ore, oim);
        Bre[t] = ore;
        Bim[t] = oim;
    }
}
// pass 3: A2[c][kz][y][x] -> delv[c][z][y][x] = Re * idft_pre
template <class T>
__global__ void k_idft_z(const double* __restrict__ Bre, const double* __restrict__ Bim,
                         const double* __restrict__ tw, int ntw, int km, int nx, int ny, int nz, double idft_pre,
                         T* __restrict__ delv) {
    const int nk = 2 * km;
    const long long plane = (long long)nx * ny;
    const long long total = 3LL * nz * plane;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        long long xy = t % plane;
        int z = (int)((t / plane) % nz);
        int c = (int)(t / (plane * nz));
        const double* cs = tw + (size_t)z * (nk - 1);
        const size_t base = (size_t)c * nk * plane + xy;
        double ore, oim;
        idft_line(Bre + base, Bim + base, (int)plane, cs, cs + ntw, km, ore, oim);
        delv[t] = (T)(ore * idft_pre);
    }
}

// Uniform state of S[cur]: density rho, zero momentum, cell-centre and face
// field b0, passive scalars 0 (the homogenous_stationary set-up of
// init_domain_mod.f90:406-479 with a uniform field).
template <class T>
__global__ void __launch_bounds__(kBX) k_init_uniform(BoxRec r, int cur, double rho, double bx, double by, double bz) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= r.n) return;
    T* S = (T*)(cur ? r.S[1] : r.S[0]);
    const size_t n = (size_t)r.n;
    const T v[10] = {(T)rho, T(0), T(0), T(0), (T)bx, (T)by, (T)bz, (T)bx, (T)by, (T)bz};
#pragma unroll
    for (int f = 0; f < 10; ++f) S[f * n + c] = v[f];
    for (int p = 0; p < r.npass; ++p) S[(10 + p) * n + c] = T(0);
}

// ============================================================ host transfer
template <class T>
__global__ void k_from_f64(const double* __restrict__ src, T* __restrict__ dst, int n) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[c] = (T)src[c];
}
template <class T>
__global__ void k_to_f64(const T* __restrict__ src, double* __restrict__ dst, int n) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) dst[c] = (double)src[c];
}

}  // namespace imhd
