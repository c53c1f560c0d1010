// imhd_types.cuh -- plain data shared by the kernels, the launchers and the
// C ABI: the device scalar block of a box, the device record of a box and the
// table that lets one launch cover many boxes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace imhd {

constexpr int kMaxPass = 8;
constexpr int kSlots = 64;     // spread of the max reductions over addresses
constexpr int kBX = 128;       // threads of the per-cell kernels, as a (1 << tws) x (kBX >> tws) tile
constexpr int kTX = 128;       // faces per block of the tiled x sweep
constexpr int kSegLog = 4;     // default faces per thread of the y / z sweeps: 1 << kSegLog
constexpr int kSegZLog = 4;    // cells per thread of the z-marching cell kernels: kSegZ = 1 << kSegZLog
constexpr int kSegZ = 1 << kSegZLog;
constexpr int kTmaTile = 128;   // row segment of a block of the bulk-copy fed kernels
constexpr int kRedThreads = 256;
constexpr int kRedBlocksMax = 1024;
constexpr size_t kRowSmemMax = 96 * 1024;   // dynamic shared memory of the x-row sweep

// stages of one step, in launch order (profiling slots)
enum Stage {
    kStForceSums = 0, kStPredFlux, kStPredEmf, kStPredUpdate, kStCorrFluxX, kStCorrFluxY, kStCorrFluxZ,
    kStCorrEmf, kStFinalUpdate, kStForceKick, kStPassivePred, kStPassiveCorr, kStFinalize, kStages
};

// Block-decomposition kinds: every launch covers the blocks of all boxes of a
// table, laid end to end; prefix[kind][b] is the first block of box b.
enum Kind {
    kKindCell = 0,     // (x, y) tiles of kBX threads per z plane, one cell per thread
    kKindRed = 1,      // min(kRedBlocksMax, ceil(n/kRedThreads)) blocks, grid-stride reductions
    kKindSolver0 = 2,  // + 5*(scheme-1) + {z column (predictor), x-row, x-tile, march-y, march-z}, 0 blocks if the box uses another scheme
    kKindCellZ = 82,   // (x, y) tiles per z segment, a z column of kSegZ cells per thread
    kKindUpdTma = 83,  // 128-cell row segments per z segment of the bulk-copy fed update (rows of 128k cells)
    kKindUpdTma64 = 84,// pairs of 64-cell row segments per z segment of it (rows of 64(2k+1) cells, even ny)
    kKinds = 85
};
// A scheme is a flux solver (1 Roe, 2 HLLD, 3 HLLE, 4 Roe with the HLLE
// protection fluxes beside it) with a reconstruction (0 PLM and 1 PPM of the
// characteristic variables, 2 PLM and 3 PPM of the primitive variables):
// scheme = solver + 4 * recon, 1..kSchemes.
constexpr int kSolvers = 4;
constexpr int kRecons = 4;
constexpr int kSchemes = kSolvers * kRecons;
static_assert(kKindSolver0 + 5 * kSchemes == kKindCellZ, "block-decomposition kinds overlap");
__host__ __device__ constexpr int scheme_of(int solver, int recon) { return solver + kSolvers * recon; }
__host__ __device__ constexpr int scheme_solver(int scheme) { return 1 + (scheme - 1) % kSolvers; }
__host__ __device__ constexpr int scheme_recon(int scheme) { return (scheme - 1) / kSolvers; }
__host__ __device__ constexpr int scheme_kind(int scheme, int sub) { return kKindSolver0 + 5 * (scheme - 1) + sub; }
enum SolverSub { kSubCell = 0, kSubXRow = 1, kSubXTile = 2, kSubMarchY = 3, kSubMarchZ = 4 };

// Device scalars of one box (FP64; maxima kept as the bit pattern of a
// non-negative double so that atomicMax on the integer is a max on the value).
struct Scalars {
    double dt;                       // current dt (input of every step kernel)
    int drive;                       // this step is a forcing step
    int cur;                         // which state buffer holds the current state
    double dt_next;                  // COUR*dx/cmax of the last step
    double sums[5];                  // quad_term1, quad_term2, momx/y/z_avg
    double constE;
    double mavg[3];
    double cmax;                     // combined max speed of the last step
    double smax_last, dvmax_last;
    double diag[6];
    unsigned int status;
    unsigned int ext_sums;           // sums[] hold all ranks' sums, set by the host for the next drive step
    unsigned long long floor_hits;
    // per-block maxima land in slot (block id mod kSlots); k_finalize folds them
    unsigned long long smax_slots[kSlots];
    unsigned long long cmax_slots[kSlots];
    unsigned long long dvmax_slots[kSlots];
    unsigned long long cfl_slots[kSlots];
    // flux protection: bad cells found by the predictor (0) and final (1) update
    unsigned int nbad[2];
    // batched driver state (driver.f90:35-186 per box)
    double t, t_end, t_turb, dt_turb_sched;
    long long steps_done, steps_target;
    int active, forcing;
};

// One box as the kernels see it.  S[0] is the current state (10 + npass
// fields of n elements), S[1] the half-step / new state; a step ends by
// swapping them (Scalars::cur counts the swaps for the host).
struct BoxRec {
    int nx, ny, nz, n;
    int npass, riemann, plane_stride, nred;
    int active, recon;      // running flag; 0 PLM, 1 PPM (characteristic), 2 PLM, 3 PPM (primitive)
    int zlo, zhi;           // z planes whose cells and faces enter the step's maxima and sums
    int tws, protect;       // x width of the cell tiles is 1 << tws (32, 64 or 128), height kBX >> tws;
                            // protect: HLLE protection fluxes of a Roe box (flux_protection)
    int segs, segzs;        // faces per thread of the y / z sweeps 1 << segs; segzs == kSegZLog (reserved)
    double dx, cs, cour, edot, dt_turb;
    void* S[2];
    void* F;        // 18 flux fields
    void* E;        // 3 corner EMF fields
    void* SH;       // npass half-step scalars
    void* delv;     // 3 forcing fields
    void* mbnd;     // 6 boundary planes of unforced momentum
    double* partials;   // nred * 6 FP64 partial sums
    Scalars* sc;
    // flux protection (protect != 0): HLLE fluxes and their corner EMFs, a
    // per-cell bad flag and per update stage a list of up to badcap bad cells
    void* Fp;
    void* Ep;
    unsigned char* bad;
    int* badlist;
    int badcap, pad3_;
};
// Flux solver of a box's scheme (4: Roe with protection fluxes).
__host__ __device__ inline int box_solver(const BoxRec& r) { return (r.riemann == 1 && r.protect) ? 4 : r.riemann; }

// A table of boxes for one set of launches.  A single box travels by value
// in the kernel parameters (use_one); a batch is a device table with, per
// decomposition kind, the box of every block (blk2box) and the first block of
// every box (prefix).
struct BatchArgs {
    BoxRec* boxes;
    const int* prefix;               // [kKinds][nbox + 1]
    const int* blk2box[kKinds];
    int nbox;
    int use_one;
    BoxRec one;
};

// Host-side view of a table, owned by a single box or by a batch.
struct BatchDev {
    BatchArgs a;               // device pointers
    int totals[kKinds];        // blocks per kind (grid sizes)
    int row_nx_max = 0;        // largest nx among boxes using the x-row sweep
    bool has_scheme[kSchemes + 1] = {};
    bool any_pass = false;
    int npass_max = 0;         // largest passive count of the table
    bool any_zrange = false;   // some box restricts its maxima to a z range
    bool any_protect = false;  // some box computes protection fluxes
    int drive_mode = 0;        // 0: no forcing, 1: every box drives (host decided), 2: per-box device flags
    int precision = 64;
    cudaStream_t st = nullptr;
    long long launches = 0;
    bool prof = false;
    cudaEvent_t ev[kStages + 1] = {};
    unsigned prof_mask = 0;
};

}  // namespace imhd
