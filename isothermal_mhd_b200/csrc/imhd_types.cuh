// imhd_types.cuh -- plain data shared by the kernels, the launchers and the
// C ABI: box dimensions, the device scalar block and the device-side view of
// one box.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace imhd {

constexpr int kMaxPass = 8;

// stages of one step, in launch order (profiling slots)
enum Stage {
    kStForceSums = 0, kStPredFlux, kStPredEmf, kStPredUpdate, kStCorrFluxX, kStCorrFluxY, kStCorrFluxZ,
    kStCorrEmf, kStFinalUpdate, kStForceKick, kStPassivePred, kStPassiveCorr, kStFinalize, kStages
};

struct Dims {
    int nx, ny, nz;
    int n;        // nx*ny*nz (< 2^31)
};

// Device scalars of one box (FP64; maxima kept as the bit pattern of a
// non-negative double so that atomicMax on the integer is a max on the value).
constexpr int kSlots = 64;   // spread of the max reductions over addresses

struct Scalars {
    double dt;                       // current dt (input of every step kernel)
    double dt_next;                  // COUR*dx/cmax of the last step
    double sums[5];                  // quad_term1, quad_term2, momx/y/z_avg
    double constE;
    double mavg[3];
    double cmax;                     // combined max speed of the last step
    double smax_last, dvmax_last;
    double diag[6];
    unsigned int status;
    unsigned int pad;
    unsigned long long floor_hits;
    // per-block maxima land in slot (block id mod kSlots); k_finalize folds them
    unsigned long long smax_slots[kSlots];
    unsigned long long cmax_slots[kSlots];
    unsigned long long dvmax_slots[kSlots];
    unsigned long long cfl_slots[kSlots];
};

struct BoxDev {
    Dims dm;
    int riemann = 1, npass = 0;
    double cs = 1.0, dx = 1.0, cour = 0.35, edot = 1e-3, dt_turb = 0.05;
    void* A = nullptr;      // current state (10 + npass fields)
    void* B = nullptr;      // half-step, then new state
    void* F = nullptr;      // 18 flux fields
    void* E = nullptr;      // 3 corner EMF fields
    void* SH = nullptr;     // npass half-step scalars
    void* delv = nullptr;   // 3 forcing fields
    void* mbnd = nullptr;   // 6 boundary planes of unforced momentum
    int plane_stride = 0;
    double* partials = nullptr;
    int nred = 0;           // blocks of the reduction kernels
    Scalars* sc = nullptr;
    cudaStream_t st = nullptr;
    long long launches = 0;
    // optional per-stage timing: an event is recorded on `st` at the start of
    // every stage that runs (prof_mask bit set) and once at the end
    bool prof = false;
    cudaEvent_t ev[kStages + 1] = {};
    unsigned prof_mask = 0;
};

}  // namespace imhd
