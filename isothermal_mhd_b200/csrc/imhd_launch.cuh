// imhd_launch.cuh -- host-side launch sequence of one step over a table of
// boxes (one box or a batch), templated on the arithmetic type.  Included by
// imhd_f64.cu (compiled with --fmad=false for bit parity with the FP64
// oracle) and imhd_f32.cu (FMA on), each of which instantiates one precision.
//
// Every launch covers all boxes of the table: the grid is the sum of the
// boxes' blocks for that kernel's decomposition (BatchDev::totals).  A single
// box travels in the kernel parameters (kernels instantiated with ONE); in a
// batch each block reads its box from the block -> box table.  A step never
// reads the host: dt, the drive flag and the current state buffer are device
// scalars of each box, so the sequence can be captured in a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

#include "imhd_kernels.cuh"

namespace imhd {

// Call f(std::integral_constant<int, s>) for every scheme s = 1..kSchemes.
template <class Fn, int... S>
inline void for_schemes_impl(Fn&& f, std::integer_sequence<int, S...>) {
    (f(std::integral_constant<int, S + 1>{}), ...);
}
template <class Fn>
inline void for_schemes(Fn&& f) {
    for_schemes_impl(f, std::make_integer_sequence<int, kSchemes>{});
}

inline void mark(BatchDev& b, int stage) {
    if (!b.prof) return;
    cudaEventRecord(b.ev[stage], b.st);
    b.prof_mask |= 1u << stage;
}

// Grid of a launch of decomposition `kind`: the table's total block count, or
// for a single box the 3D grid whose block indices the kernels read directly.
template <bool ONE>
static dim3 grid_of(const BatchDev& b, int kind) {
    if constexpr (!ONE) {
        return dim3((unsigned)b.totals[kind]);
    } else {
        const BoxRec& r = b.a.one;
        const int tw = 1 << r.tws, th = kBX >> r.tws;
        unsigned nbx = (unsigned)((r.nx + tw - 1) / tw), nby = (unsigned)((r.ny + th - 1) / th);
        unsigned nbz = (unsigned)((r.nz + th - 1) / th);
        if (kind == kKindCell) return dim3(nbx, nby, r.nz);
        const int sz = 1 << r.segzs, sg = 1 << r.segs;
        if (kind == kKindCellZ) return dim3(nbx, nby, (unsigned)((r.nz + sz - 1) / sz));
        if (kind == kKindRed) return dim3((unsigned)r.nred);
        switch ((kind - kKindSolver0) % 5) {
            case kSubCell: return dim3(nbx, nby, (unsigned)((r.nz + kSegZ - 1) / kSegZ));   // z columns
            case kSubXRow: return dim3(r.ny, r.nz);
            case kSubXTile: return dim3((unsigned)((r.nx + kTX - 1) / kTX), r.ny, r.nz);
            case kSubMarchY: return dim3(nbx, nbz, (unsigned)((r.ny + sg - 1) / sg));
            default: return dim3(nbx, nby, (unsigned)((r.nz + sg - 1) / sg));
        }
    }
}

// Corner EMFs of one stage (PROT: of the protection fluxes).
template <class T, bool ONE, bool PROT>
static void launch_emf(BatchDev& b, dim3 gz, int half_step_state) {
    k_corner_emf<T, ONE, PROT><<<gz, kBX, 0, b.st>>>(b.a, half_step_state);
    b.launches += 1;
}

template <class T, int SCHEME, bool ONE>
static void launch_fluxes_pred(BatchDev& b) {
    if (!b.has_scheme[SCHEME] || b.totals[scheme_kind(SCHEME, kSubCell)] == 0) return;
    dim3 g = grid_of<ONE>(b, scheme_kind(SCHEME, kSubCell));
    k_pred_flux<T, SCHEME, ONE><<<g, kBX, 0, b.st>>>(b.a);
    b.launches += 1;
}

// The x-row sweep needs more than 48 KiB of dynamic shared memory for long
// rows; the opt-in is per kernel and device and is done outside any capture.
template <class T, int SCHEME, bool ONE>
static void ensure_xrow_attr() {
    static bool attr_set[64] = {};   // per instantiation and device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaFuncSetAttribute(k_corr_flux_xrow<T, SCHEME, ONE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRowSmemMax);
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
}

// The TMA-fed update's two stages exceed 48 KiB of shared memory in FP64.
template <class T, int TW>
static void set_update_tma_attr() {
    const int bytes = (int)update_tma_smem_bytes<T, TW>();
    cudaFuncSetAttribute(k_update_tma<T, false, true, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_update_tma<T, true, true, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_update_tma<T, false, false, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_update_tma<T, true, false, TW>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <class T>
static void ensure_update_tma_attr() {
    static bool attr_set[64] = {};   // per precision and device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        set_update_tma_attr<T, kTmaTile>();
        set_update_tma_attr<T, kTmaTile / 2>();
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
}

template <class T, bool ONE, int TW>
static void launch_update_tma(BatchDev& b, dim3 g, double dt_scale, int final_stage) {
    const size_t smem = update_tma_smem_bytes<T, TW>();
    if (b.any_zrange) k_update_tma<T, true, ONE, TW><<<g, kTmaTile, smem, b.st>>>(b.a, dt_scale, final_stage);
    else k_update_tma<T, false, ONE, TW><<<g, kTmaTile, smem, b.st>>>(b.a, dt_scale, final_stage);
    b.launches += 1;
}

// Update of one stage: the TMA-fed kernel for a single box whose rows are
// whole 128-cell tiles, the z-column kernel otherwise.  A table launches both:
// the z-column kernel skips the boxes with such rows (every box of a table is
// carved on 256-byte boundaries), the TMA-fed kernel covers only those.
template <class T, bool ONE>
static void launch_update(BatchDev& b, double dt_scale, int final_stage) {
    const dim3 gz = grid_of<ONE>(b, kKindCellZ);
    // the bulk copies need 16-byte aligned sources: every row of a 128-cell
    // tile starts on one when the field bases do
    const bool aligned = ((uintptr_t)b.a.one.S[0] | (uintptr_t)b.a.one.F | (uintptr_t)b.a.one.E) % 16 == 0;
    const int tw = tma_row_tile(b.a.one.nx, b.a.one.ny);
    if (ONE && aligned && tw > 0) {
        ensure_update_tma_attr<T>();
        const dim3 g((unsigned)(b.a.one.nx / tw), (unsigned)(b.a.one.ny / (kTmaTile / tw)),
                     (unsigned)((b.a.one.nz + kSegZ - 1) / kSegZ));
        if (tw == kTmaTile) launch_update_tma<T, ONE, kTmaTile>(b, g, dt_scale, final_stage);
        else launch_update_tma<T, ONE, kTmaTile / 2>(b, g, dt_scale, final_stage);
        return;
    }
    if (b.any_zrange) k_update<T, ONE, true><<<gz, kBX, 0, b.st>>>(b.a, dt_scale, final_stage);
    else k_update<T, ONE, false><<<gz, kBX, 0, b.st>>>(b.a, dt_scale, final_stage);
    b.launches += 1;
    if (!ONE && (b.totals[kKindUpdTma] > 0 || b.totals[kKindUpdTma64] > 0)) {
        ensure_update_tma_attr<T>();
        if (b.totals[kKindUpdTma] > 0)
            launch_update_tma<T, ONE, kTmaTile>(b, dim3((unsigned)b.totals[kKindUpdTma]), dt_scale, final_stage);
        if (b.totals[kKindUpdTma64] > 0)
            launch_update_tma<T, ONE, kTmaTile / 2>(b, dim3((unsigned)b.totals[kKindUpdTma64]), dt_scale, final_stage);
    }
}

// The bulk-copy fed passive corrector's two stages exceed 48 KiB with many
// scalars (and in FP64).
template <class T>
static void ensure_passive_tma_attr() {
    static bool attr_set[64] = {};   // per precision and device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaFuncSetAttribute(k_passive_corr_tma<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_tma_smem_bytes<T, 2>());
        cudaFuncSetAttribute(k_passive_corr_tma<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_tma_smem_bytes<T, 4>());
        cudaFuncSetAttribute(k_passive_corr_tma<T, kMaxPass>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_tma_smem_bytes<T, kMaxPass>());
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
}

// Passive corrector: the bulk-copy fed kernel for a single box whose rows
// are whole 128-cell tiles (16-byte aligned rows of every field it streams),
// the z-column kernel otherwise; scalar arrays sized for the table's largest
// passive count.
template <class T>
static void ensure_passive_pred_tma_attr() {
    static bool attr_set[64] = {};   // per precision and device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaFuncSetAttribute(k_passive_pred_tma<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_pred_tma_smem_bytes<T, 2>());
        cudaFuncSetAttribute(k_passive_pred_tma<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_pred_tma_smem_bytes<T, 4>());
        cudaFuncSetAttribute(k_passive_pred_tma<T, kMaxPass>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)passive_pred_tma_smem_bytes<T, kMaxPass>());
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
}

// Passive predictor: the bulk-copy fed kernel for a single box whose rows are
// whole 128-cell tiles (16-byte aligned sources), the z-column kernel
// otherwise; scalar arrays sized for the table's largest passive count.
template <class T, bool ONE>
static void launch_passive_pred(BatchDev& b, dim3 gz) {
    const BoxRec& r = b.a.one;
    if (ONE && ((uintptr_t)r.S[0] | (uintptr_t)r.SH) % 16 == 0 && passive_by_tma(r.nx)) {
        ensure_passive_pred_tma_attr<T>();
        const dim3 g((unsigned)(r.nx / kTmaTile), (unsigned)r.ny, (unsigned)((r.nz + kSegZ - 1) / kSegZ));
        if (b.npass_max <= 2)
            k_passive_pred_tma<T, 2><<<g, kTmaTile, passive_pred_tma_smem_bytes<T, 2>(), b.st>>>(b.a);
        else if (b.npass_max <= 4)
            k_passive_pred_tma<T, 4><<<g, kTmaTile, passive_pred_tma_smem_bytes<T, 4>(), b.st>>>(b.a);
        else
            k_passive_pred_tma<T, kMaxPass><<<g, kTmaTile, passive_pred_tma_smem_bytes<T, kMaxPass>(), b.st>>>(b.a);
        b.launches += 1;
        return;
    }
    if (b.npass_max <= 2) k_passive_pred<T, ONE, 2><<<gz, kBX, 0, b.st>>>(b.a);
    else if (b.npass_max <= 4) k_passive_pred<T, ONE, 4><<<gz, kBX, 0, b.st>>>(b.a);
    else k_passive_pred<T, ONE, kMaxPass><<<gz, kBX, 0, b.st>>>(b.a);
    b.launches += 1;
}

template <class T, bool ONE>
static void launch_passive_corr(BatchDev& b, dim3 gz) {
    const BoxRec& r = b.a.one;
    if (ONE && ((uintptr_t)r.S[0] | (uintptr_t)r.SH | (uintptr_t)r.F) % 16 == 0 && passive_by_tma(r.nx)) {
        ensure_passive_tma_attr<T>();
        const dim3 g((unsigned)(r.nx / kTmaTile), (unsigned)r.ny, (unsigned)((r.nz + kSegZ - 1) / kSegZ));
        if (b.npass_max <= 2)
            k_passive_corr_tma<T, 2><<<g, kTmaTile, passive_tma_smem_bytes<T, 2>(), b.st>>>(b.a);
        else if (b.npass_max <= 4)
            k_passive_corr_tma<T, 4><<<g, kTmaTile, passive_tma_smem_bytes<T, 4>(), b.st>>>(b.a);
        else
            k_passive_corr_tma<T, kMaxPass><<<g, kTmaTile, passive_tma_smem_bytes<T, kMaxPass>(), b.st>>>(b.a);
        b.launches += 1;
        return;
    }
    if (b.npass_max <= 2) k_passive_corr<T, ONE, 2><<<gz, kBX, 0, b.st>>>(b.a);
    else if (b.npass_max <= 4) k_passive_corr<T, ONE, 4><<<gz, kBX, 0, b.st>>>(b.a);
    else k_passive_corr<T, ONE, kMaxPass><<<gz, kBX, 0, b.st>>>(b.a);
    b.launches += 1;
}

template <class T>
cudaError_t prepare_launch(BatchDev& b) {
    ensure_update_tma_attr<T>();
    ensure_passive_tma_attr<T>();
    ensure_passive_pred_tma_attr<T>();
    for_schemes([&](auto s) {
        if (b.has_scheme[s.value]) {
            ensure_xrow_attr<T, s.value, true>();
            ensure_xrow_attr<T, s.value, false>();
        }
    });
    return cudaGetLastError();
}

template <class T, int SCHEME, bool ONE>
static void launch_fluxes_corr_x(BatchDev& b) {
    if (!b.has_scheme[SCHEME]) return;
    if (b.totals[scheme_kind(SCHEME, kSubXRow)]) {
        dim3 gr = grid_of<ONE>(b, scheme_kind(SCHEME, kSubXRow));
        size_t smem = 13 * (size_t)b.row_nx_max * sizeof(T);
        ensure_xrow_attr<T, SCHEME, ONE>();
        int bd = b.row_nx_max >= 128 ? 128 : ((b.row_nx_max + 31) / 32) * 32;
        k_corr_flux_xrow<T, SCHEME, ONE><<<gr, bd, smem, b.st>>>(b.a);
        b.launches += 1;
    }
    if (b.totals[scheme_kind(SCHEME, kSubXTile)]) {
        dim3 gt = grid_of<ONE>(b, scheme_kind(SCHEME, kSubXTile));
        k_corr_flux_x<T, SCHEME, kTX, ONE><<<gt, kTX, 0, b.st>>>(b.a);
        b.launches += 1;
    }
}

template <class T, int SCHEME, int D, bool ONE>
static void launch_fluxes_corr_march(BatchDev& b) {
    const int kind = scheme_kind(SCHEME, D == 1 ? kSubMarchY : kSubMarchZ);
    if (!b.has_scheme[SCHEME] || b.totals[kind] == 0) return;
    dim3 g = grid_of<ONE>(b, kind);
    k_corr_flux_march<T, SCHEME, D, ONE><<<g, kBX, 0, b.st>>>(b.a);
    b.launches += 1;
}

// The protected update of flux_protection after update stage `stage`
// (vanleer_mod.f90:2086-2202): hydro variables of the bad cells and their
// neighbours, face fields, cell-centred field, the CFL maximum after the
// final stage, then the bad flags cleared.  Every kernel returns at once for
// a box whose stage listed no bad cell.
template <class T, bool ONE>
static void launch_protection(BatchDev& b, double dt_scale, int stage) {
    const unsigned g = ONE ? (unsigned)kProtBlocks : (unsigned)(kProtBlocks * b.a.nbox);
    k_prot_hydro<T, ONE><<<g, kBX, 0, b.st>>>(b.a, dt_scale, stage);
    k_prot_faces<T, ONE><<<g, kBX, 0, b.st>>>(b.a, dt_scale, stage);
    k_prot_centres<T, ONE><<<g, kBX, 0, b.st>>>(b.a, stage);
    b.launches += 3;
    if (stage == 1) {
        k_prot_cfl<T, ONE><<<b.totals[kKindRed], kRedThreads, 0, b.st>>>(b.a);
        b.launches += 1;
    }
    k_prot_clear<ONE><<<g, kBX, 0, b.st>>>(b.a, stage);
    b.launches += 1;
}

template <class T, bool ONE>
static cudaError_t run_step_t(BatchDev& b, int device_driven) {
    const dim3 gc = grid_of<ONE>(b, kKindCell);
    const dim3 gz = grid_of<ONE>(b, kKindCellZ);
    const int nfin = (b.a.nbox + 31) / 32;
    b.prof_mask = 0;
    if (device_driven) {
        k_batch_begin<<<nfin, 32, 0, b.st>>>(b.a);
        b.launches += 1;
    }
    if (b.drive_mode) {
        mark(b, kStForceSums);
        k_force_sums<T, ONE><<<b.totals[kKindRed], kRedThreads, 0, b.st>>>(b.a, 0);
        k_force_reduce<<<b.a.nbox, 32, 0, b.st>>>(b.a, 0);
        b.launches += 2;
    }
    // predictor: first-order fluxes, EMFs, half-dt update into the other buffer
    mark(b, kStPredFlux);
    for_schemes([&](auto s) { launch_fluxes_pred<T, s.value, ONE>(b); });
    mark(b, kStPredEmf);
    launch_emf<T, ONE, false>(b, gz, 0);
    if (b.any_protect) launch_emf<T, ONE, true>(b, gz, 0);
    mark(b, kStPredUpdate);
    launch_update<T, ONE>(b, 0.5, 0);   // counts its own launches
    if (b.any_protect) launch_protection<T, ONE>(b, 0.5, 0);
    // corrector: characteristic PLM fluxes of the half-step state, EMFs,
    // full-dt update of the step-start state
    mark(b, kStCorrFluxX);
    for_schemes([&](auto s) { launch_fluxes_corr_x<T, s.value, ONE>(b); });
    mark(b, kStCorrFluxY);
    for_schemes([&](auto s) { launch_fluxes_corr_march<T, s.value, 1, ONE>(b); });
    mark(b, kStCorrFluxZ);
    for_schemes([&](auto s) { launch_fluxes_corr_march<T, s.value, 2, ONE>(b); });
    mark(b, kStCorrEmf);
    launch_emf<T, ONE, false>(b, gz, 1);
    if (b.any_protect) launch_emf<T, ONE, true>(b, gz, 1);
    mark(b, kStFinalUpdate);
    launch_update<T, ONE>(b, 1.0, 1);
    if (b.any_protect) launch_protection<T, ONE>(b, 1.0, 1);
    if (b.drive_mode) {
        mark(b, kStForceKick);
        k_force_kick<T, ONE><<<gc, kBX, 0, b.st>>>(b.a);
        b.launches += 1;
    }
    if (b.any_pass) {
        mark(b, kStPassivePred);
        launch_passive_pred<T, ONE>(b, gz);
        mark(b, kStPassiveCorr);
        launch_passive_corr<T, ONE>(b, gz);
    }
    mark(b, kStFinalize);
    k_finalize<<<nfin, 32, 0, b.st>>>(b.a, device_driven);
    b.launches += 1;
    if (b.prof) cudaEventRecord(b.ev[kStages], b.st);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_step(BatchDev& b, int device_driven) {
    return b.a.use_one ? run_step_t<T, true>(b, device_driven) : run_step_t<T, false>(b, device_driven);
}

template <class T, bool ONE>
static cudaError_t run_max_speed_t(BatchDev& b) {
    k_cfl<T, ONE><<<grid_of<ONE>(b, kKindCell), kBX, 0, b.st>>>(b.a);
    b.launches += 1;
    return cudaGetLastError();
}

// This box's forcing sums of the current state (no normalisation, any step).
template <class T>
cudaError_t run_force_sums(BatchDev& b) {
    k_force_sums<T, true><<<b.totals[kKindRed], kRedThreads, 0, b.st>>>(b.a, 1);
    k_force_reduce<<<1, 32, 0, b.st>>>(b.a, 1);
    b.launches += 2;
    return cudaGetLastError();
}

template <class T>
cudaError_t run_max_speed(BatchDev& b) {
    return b.a.use_one ? run_max_speed_t<T, true>(b) : run_max_speed_t<T, false>(b);
}

template <class T, bool ONE>
static cudaError_t run_diag_t(BatchDev& b) {
    k_diag<T, ONE><<<b.totals[kKindRed], kRedThreads, 0, b.st>>>(b.a);
    k_diag_reduce<<<b.a.nbox, 32, 0, b.st>>>(b.a);
    b.launches += 2;
    return cudaGetLastError();
}

template <class T>
cudaError_t run_diag(BatchDev& b) {
    return b.a.use_one ? run_diag_t<T, true>(b) : run_diag_t<T, false>(b);
}

template <class T>
cudaError_t run_from_f64(cudaStream_t st, const double* src, void* dst, int n) {
    int blocks = (n + 255) / 256;
    if (blocks > 65535) blocks = 65535;
    k_from_f64<T><<<blocks, 256, 0, st>>>(src, (T*)dst, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_to_f64(cudaStream_t st, const void* src, double* dst, int n) {
    int blocks = (n + 255) / 256;
    if (blocks > 65535) blocks = 65535;
    k_to_f64<T><<<blocks, 256, 0, st>>>((const T*)src, dst, n);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_ou_field(cudaStream_t st, const BoxRec& r, int cur, int target, const int* kv, const double* amp,
                         int nm, double scale) {
    int blocks = (r.n + kBX - 1) / kBX;
    k_fourier_field<T><<<blocks, kBX, 0, st>>>(r, cur, target, kv, amp, nm, scale);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_clocks(BatchDev& b, double* out) {
    k_clocks<<<(b.a.nbox + 127) / 128, 128, 0, b.st>>>(b.a, out);
    b.launches += 1;
    return cudaGetLastError();
}

// The three inverse-DFT passes of the reference force field into r.delv.
// V: 3 x (2km)^3 spectrum (re, im); tw*: per-axis twiddle tables of
// n_axis x (2km-1) cos values followed by as many sin values; scratch: room
// for 2 x 3 x 2km x max(2km, ny) x nx doubles, twice.
template <class T>
cudaError_t run_ref_force(cudaStream_t st, const BoxRec& r, int km, const double* Vre, const double* Vim,
                          const double* twx, const double* twy, const double* twz, double* s1re, double* s1im,
                          double* s2re, double* s2im) {
    const int nk = 2 * km;
    auto blocks = [](long long n) { long long b = (n + 255) / 256; return (int)(b > 65535 * 8 ? 65535 * 8 : b); };
    k_idft_x<<<blocks(3LL * nk * nk * r.nx), 256, 0, st>>>(Vre, Vim, twx, r.nx * (nk - 1), km, r.nx, s1re, s1im);
    k_idft_y<<<blocks(3LL * nk * r.ny * r.nx), 256, 0, st>>>(s1re, s1im, twy, r.ny * (nk - 1), km, r.nx, r.ny, s2re,
                                                            s2im);
    const double idft_pre = 1.0 / (double)((long)r.nx * r.ny * r.nz);
    k_idft_z<T><<<blocks(3LL * r.nz * r.ny * r.nx), 256, 0, st>>>(s2re, s2im, twz, r.nz * (nk - 1), km, r.nx, r.ny,
                                                                  r.nz, idft_pre, (T*)r.delv);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_init_uniform(cudaStream_t st, const BoxRec& r, int cur, double rho, const double* b0) {
    int blocks = (r.n + kBX - 1) / kBX;
    k_init_uniform<T><<<blocks, kBX, 0, st>>>(r, cur, rho, b0[0], b0[1], b0[2]);
    return cudaGetLastError();
}

}  // namespace imhd

#define IMHD_INSTANTIATE(T)                                                        \
    namespace imhd {                                                               \
    template cudaError_t run_step<T>(BatchDev&, int);                              \
    template cudaError_t prepare_launch<T>(BatchDev&);                             \
    template cudaError_t run_max_speed<T>(BatchDev&);                              \
    template cudaError_t run_force_sums<T>(BatchDev&);                             \
    template cudaError_t run_diag<T>(BatchDev&);                                   \
    template cudaError_t run_from_f64<T>(cudaStream_t, const double*, void*, int); \
    template cudaError_t run_to_f64<T>(cudaStream_t, const void*, double*, int);   \
    template cudaError_t run_ou_field<T>(cudaStream_t, const BoxRec&, int, int, const int*, const double*, int, \
                                         double);                                  \
    template cudaError_t run_init_uniform<T>(cudaStream_t, const BoxRec&, int, double, const double*); \
    template cudaError_t run_clocks<T>(BatchDev&, double*);                       \
    template cudaError_t run_ref_force<T>(cudaStream_t, const BoxRec&, int, const double*, const double*, \
                                          const double*, const double*, const double*, double*, double*, \
                                          double*, double*);                       \
    }
