// imhd_launch.cuh -- host-side launch sequence of one step, templated on the
// arithmetic type.  Included by imhd_f64.cu (compiled with --fmad=false for
// bit parity with the FP64 oracle) and imhd_f32.cu (FMA on), each of which
// instantiates one precision.
#pragma once

#include <cuda_runtime.h>

#include "imhd_kernels.cuh"

namespace imhd {

inline void mark(BoxDev& b, int stage) {
    if (!b.prof) return;
    cudaEventRecord(b.ev[stage], b.st);
    b.prof_mask |= 1u << stage;
}

constexpr int kBX = 128;       // threads along x of the per-cell kernels
constexpr int kTX = 128;       // faces per block of the x sweep
constexpr int kSeg = 16;       // faces per thread of the y / z sweeps
constexpr size_t kRowSmemMax = 96 * 1024;   // dynamic shared memory of the x-row sweep

template <class T, int SOLVER>
static void launch_fluxes_pred(BoxDev& b) {
    const Dims& dm = b.dm;
    dim3 blk(kBX), grd((dm.nx + kBX - 1) / kBX, dm.ny, dm.nz);
    const T* S = (const T*)b.A;
    T* F = (T*)b.F;
    T cs = (T)b.cs, asqr = (T)(b.cs * b.cs);
    mark(b, kStPredFlux);
    k_pred_flux<T, SOLVER, 0><<<grd, blk, 0, b.st>>>(S, F, dm, cs, asqr, b.sc->smax_slots);
    k_pred_flux<T, SOLVER, 1><<<grd, blk, 0, b.st>>>(S, F, dm, cs, asqr, b.sc->smax_slots);
    k_pred_flux<T, SOLVER, 2><<<grd, blk, 0, b.st>>>(S, F, dm, cs, asqr, b.sc->smax_slots);
    b.launches += 3;
}

template <class T, int SOLVER>
static void launch_fluxes_corr(BoxDev& b) {
    const Dims& dm = b.dm;
    const T* S = (const T*)b.B;
    T* F = (T*)b.F;
    T cs = (T)b.cs, asqr = (T)(b.cs * b.cs);
    mark(b, kStCorrFluxX);
    size_t row_smem = 13 * (size_t)dm.nx * sizeof(T);
    if (row_smem <= kRowSmemMax) {
        static bool attr_set[64] = {};   // per instantiation and device
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !attr_set[dev]) {
            cudaFuncSetAttribute(k_corr_flux_xrow<T, SOLVER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kRowSmemMax);
            if (dev >= 0 && dev < 64) attr_set[dev] = true;
        }
        int bd = dm.nx >= 256 ? 256 : ((dm.nx + 31) / 32) * 32;
        k_corr_flux_xrow<T, SOLVER><<<dim3(dm.ny, dm.nz), bd, row_smem, b.st>>>(S, F, dm, cs, asqr, b.sc->smax_slots);
    } else {
        dim3 gx((dm.nx + kTX - 1) / kTX, dm.ny, dm.nz);
        k_corr_flux_x<T, SOLVER, kTX><<<gx, kTX, 0, b.st>>>(S, F, dm, cs, asqr, b.sc->smax_slots);
    }
    dim3 gy((dm.nx + kBX - 1) / kBX, dm.nz, (dm.ny + kSeg - 1) / kSeg);
    mark(b, kStCorrFluxY);
    k_corr_flux_march<T, SOLVER, 1><<<gy, kBX, 0, b.st>>>(S, F, dm, kSeg, cs, asqr, b.sc->smax_slots);
    dim3 gz((dm.nx + kBX - 1) / kBX, dm.ny, (dm.nz + kSeg - 1) / kSeg);
    mark(b, kStCorrFluxZ);
    k_corr_flux_march<T, SOLVER, 2><<<gz, kBX, 0, b.st>>>(S, F, dm, kSeg, cs, asqr, b.sc->smax_slots);
    b.launches += 3;
}

template <class T>
cudaError_t run_step(BoxDev& b, int drive) {
    const Dims& dm = b.dm;
    dim3 blk(kBX), grd((dm.nx + kBX - 1) / kBX, dm.ny, dm.nz);
    T asqr = (T)(b.cs * b.cs);
    const T* A = (const T*)b.A;
    T* Bs = (T*)b.B;
    b.prof_mask = 0;
    if (drive) {
        mark(b, kStForceSums);
        k_force_sums<T><<<b.nred, 256, 0, b.st>>>(A, (const T*)b.delv, dm, b.partials);
        k_force_reduce<<<1, 32, 0, b.st>>>(b.partials, b.nred, b.sc, b.dx, b.edot, b.dt_turb);
        b.launches += 2;
    }
    // predictor: first-order fluxes, EMFs, half-dt update into B
    switch (b.riemann) {
        case 1: launch_fluxes_pred<T, 1>(b); break;
        case 2: launch_fluxes_pred<T, 2>(b); break;
        default: launch_fluxes_pred<T, 3>(b); break;
    }
    mark(b, kStPredEmf);
    k_corner_emf<T><<<grd, blk, 0, b.st>>>(A, (const T*)b.F, (T*)b.E, dm);
    mark(b, kStPredUpdate);
    k_update<T><<<grd, blk, 0, b.st>>>(A, (const T*)b.F, (const T*)b.E, Bs, dm, b.sc, 0.5, b.dx, asqr, 0,
                                       b.sc->cmax_slots, &b.sc->floor_hits, &b.sc->status);
    b.launches += 2;
    // corrector: characteristic PLM fluxes of the half-step state, EMFs,
    // full-dt update of the step-start state into B
    switch (b.riemann) {
        case 1: launch_fluxes_corr<T, 1>(b); break;
        case 2: launch_fluxes_corr<T, 2>(b); break;
        default: launch_fluxes_corr<T, 3>(b); break;
    }
    mark(b, kStCorrEmf);
    k_corner_emf<T><<<grd, blk, 0, b.st>>>(Bs, (const T*)b.F, (T*)b.E, dm);
    mark(b, kStFinalUpdate);
    k_update<T><<<grd, blk, 0, b.st>>>(A, (const T*)b.F, (const T*)b.E, Bs, dm, b.sc, 1.0, b.dx, asqr, drive ? 0 : 1,
                                       b.sc->cmax_slots, &b.sc->floor_hits, &b.sc->status);
    b.launches += 2;
    if (drive) {
        mark(b, kStForceKick);
        k_force_kick<T><<<grd, blk, 0, b.st>>>(A, Bs, (const T*)b.delv, dm, b.sc, asqr, (T*)b.mbnd, b.plane_stride,
                                               b.npass > 0 ? 1 : 0);
        b.launches += 1;
    }
    if (b.npass > 0) {
        mark(b, kStPassivePred);
        k_passive_pred<T><<<grd, blk, 0, b.st>>>(A, (T*)b.SH, dm, b.npass, b.sc, b.dx);
        mark(b, kStPassiveCorr);
        k_passive_corr<T><<<grd, blk, 0, b.st>>>(A, (const T*)b.SH, Bs, dm, b.npass, b.sc, b.dx, drive,
                                                 (const T*)b.mbnd, b.plane_stride);
        b.launches += 2;
    }
    mark(b, kStFinalize);
    k_finalize<<<1, 1, 0, b.st>>>(b.sc, b.cour, b.dx, drive);
    b.launches += 1;
    if (b.prof) cudaEventRecord(b.ev[kStages], b.st);
    return cudaGetLastError();
}

template <class T>
cudaError_t run_max_speed(BoxDev& b) {
    const Dims& dm = b.dm;
    dim3 blk(kBX), grd((dm.nx + kBX - 1) / kBX, dm.ny, dm.nz);
    cudaMemsetAsync(b.sc->cfl_slots, 0, sizeof(b.sc->cfl_slots), b.st);
    k_cfl<T><<<grd, blk, 0, b.st>>>((const T*)b.A, dm, (T)(b.cs * b.cs), b.sc->cfl_slots);
    b.launches += 1;
    return cudaGetLastError();
}

template <class T>
cudaError_t run_diag(BoxDev& b) {
    k_diag<T><<<b.nred, 256, 0, b.st>>>((const T*)b.A, b.dm, b.partials);
    k_diag_reduce<<<1, 32, 0, b.st>>>(b.partials, b.nred, b.sc, b.dx);
    b.launches += 2;
    return cudaGetLastError();
}

template <class T>
cudaError_t run_from_f64(BoxDev& b, const double* src, void* dst) {
    int n = b.dm.n;
    int blocks = (n + 255) / 256;
    if (blocks > 65535) blocks = 65535;
    k_from_f64<T><<<blocks, 256, 0, b.st>>>(src, (T*)dst, n);
    b.launches += 1;
    return cudaGetLastError();
}

template <class T>
cudaError_t run_to_f64(BoxDev& b, const void* src, double* dst) {
    int n = b.dm.n;
    int blocks = (n + 255) / 256;
    if (blocks > 65535) blocks = 65535;
    k_to_f64<T><<<blocks, 256, 0, b.st>>>((const T*)src, dst, n);
    b.launches += 1;
    return cudaGetLastError();
}

}  // namespace imhd

#define IMHD_INSTANTIATE(T)                                                        \
    namespace imhd {                                                               \
    template cudaError_t run_step<T>(BoxDev&, int);                                \
    template cudaError_t run_max_speed<T>(BoxDev&);                                \
    template cudaError_t run_diag<T>(BoxDev&);                                     \
    template cudaError_t run_from_f64<T>(BoxDev&, const double*, void*);          \
    template cudaError_t run_to_f64<T>(BoxDev&, const void*, double*);            \
    }
