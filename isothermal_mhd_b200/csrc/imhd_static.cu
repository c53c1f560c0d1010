// imhd_static.cu -- imhd_step_static: one time step that allocates nothing.
//
// Who needs it: hosts that own all device memory and may not call cudaMalloc
// themselves or let a library do it -- a Fortran or C driver whose arrays
// live in a pool or are managed by OpenACC / CUDA Fortran, whose runtime keeps
// the device heap to itself -- and real-time loops that forbid allocation
// after start-up.  They pass the state in and receive the state out; the
// step's work arrays (interface fluxes, corner EMFs, half-step passive
// scalars and the reduction scalars) live in one file-scope device array
// instead of in per-box allocations.  The step is undriven, with PLM
// reconstruction.
//
// Limits and sharing:
//  * the scratch array holds kStaticScratchBytes (48 MiB) on every GPU that
//    loads the library, until the process exits; a box needs
//    (21 + npass) * nx*ny*nz * (4 or 8) bytes plus 56 KiB, i.e. up to 64^3 in
//    FP64 with at most two passive scalars or about 80^3 in FP32 with two.
//    Larger boxes are rejected with IMHD_E_ARG; use imhd_create / imhd_step
//    for them;
//  * every call on a device uses the same array and leaves its contents
//    behind; the reduction scalars are cleared at the start of each call.
//    Calls that overlap on the GPU (two streams, two host threads) race on
//    the array and must be serialised by the caller;
//  * the first call on a device looks up the array's device address (with
//    that device current) and keeps it for the life of the process: a
//    cudaDeviceReset would leave it stale, so the library must not be used
//    across one.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/imhd.h"
#include "imhd_table.h"
#include "imhd_types.cuh"

namespace imhd {
template <class T> cudaError_t run_step(BatchDev&, int);
const char* set_last_error(int code, const char* msg);
}  // namespace imhd

namespace {

constexpr size_t kStaticScratchBytes = size_t(48) << 20;   // 48 MiB
constexpr size_t kScalarsBytes = 4096;                     // imhd::Scalars, rounded up
constexpr size_t kTableBytes = 4096;                       // box record + block prefixes
constexpr size_t kPartialBytes = 1024 * 6 * 8;             // reduction partials (unused: no forcing)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_step_scratch[kStaticScratchBytes];

// device address of g_step_scratch per device ordinal (the host-side name of
// the array is only a stand-in and must never be passed to a kernel)
unsigned char* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int scratch_address(int dev, unsigned char** out, std::string& err) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
        if (e != cudaSuccess) {
            err = std::string("cudaGetSymbolAddress(g_step_scratch): ") + cudaGetErrorString(e);
            return IMHD_E_CUDA;
        }
        g_scratch_ptr[dev] = (unsigned char*)p;
    }
    *out = g_scratch_ptr[dev];
    return IMHD_OK;
}

using imhd::align256;

}  // namespace

extern "C" int imhd_step_static(int precision, int nx, int ny, int nz, int riemann, int npass, double sound_speed,
                                double cour, const void* state_in, void* state_out, double dt, double* dt_next,
                                void* stream) {
    static_assert(sizeof(imhd::Scalars) <= kScalarsBytes, "scalar block outgrew its scratch slot");
    static_assert(256 + sizeof(int) * imhd::kKinds * 2 <= kTableBytes && sizeof(imhd::BoxRec) <= 256,
                  "box table outgrew its scratch slot");
    auto fail = [](int code, const std::string& m) { imhd::set_last_error(code, m.c_str()); return code; };
    if (precision != 32 && precision != 64) return fail(IMHD_E_ARG, "precision must be 32 or 64");
    if (nx < 4 || ny < 4 || nz < 4) return fail(IMHD_E_ARG, "every edge needs at least 4 cells");
    if (riemann < 1 || riemann > 3) return fail(IMHD_E_ARG, "riemann must be IMHD_ROE, IMHD_HLLD or IMHD_HLLE");
    if (npass < 0 || npass > imhd::kMaxPass) return fail(IMHD_E_ARG, "npass must be in 0..8");
    if (!(sound_speed > 0.0) || !(cour > 0.0) || !(dt > 0.0)) return fail(IMHD_E_ARG, "sound_speed, cour and dt must be positive");
    if (!state_in || !state_out || state_in == state_out) return fail(IMHD_E_ARG, "state_in and state_out must be distinct device buffers");
    size_t esz = precision == 64 ? 8 : 4;
    size_t n = (size_t)nx * ny * nz;
    size_t fields_bytes = align256(18 * n * esz) + align256(3 * n * esz) + align256((size_t)npass * n * esz);
    size_t need = kScalarsBytes + kTableBytes + kPartialBytes + fields_bytes;
    if (need > kStaticScratchBytes)
        return fail(IMHD_E_ARG, "box needs " + std::to_string(need) + " bytes of step scratch but imhd_step_static holds " +
                                    std::to_string(kStaticScratchBytes) +
                                    " (at most 64^3 in FP64 with two passive scalars, about 80^3 in FP32 with two); "
                                    "use imhd_create / imhd_step");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(IMHD_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(IMHD_E_ARG, "device ordinal out of range");
    unsigned char* base = nullptr;
    std::string err;
    int rc = scratch_address(dev, &base, err);
    if (rc) return fail(rc, err);

    imhd::BoxRec rec;
    imhd::init_rec(rec, nx, ny, nz, npass, riemann, IMHD_PLM, sound_speed, cour, 0.0, 0.0);
    rec.S[0] = const_cast<void*>(state_in);
    rec.S[1] = state_out;
    unsigned char* p = base;
    rec.sc = (imhd::Scalars*)p;  p += kScalarsBytes;
    unsigned char* table = p;    p += kTableBytes;
    rec.partials = (double*)p;   p += kPartialBytes;
    rec.F = p;  p += align256(18 * n * esz);
    rec.E = p;  p += align256(3 * n * esz);
    rec.SH = npass ? (void*)p : nullptr;
    rec.delv = nullptr;
    rec.mbnd = nullptr;
    imhd::BatchDev b;
    b.precision = precision;
    b.st = (cudaStream_t)stream;
    std::vector<imhd::BoxRec> recs(1, rec);
    std::vector<int> prefix;
    if (!imhd::build_prefix(recs, esz, prefix, b)) return fail(IMHD_E_ARG, "box too large for one launch");
    b.a.boxes = (imhd::BoxRec*)table;
    b.a.prefix = (const int*)(table + 256);
    b.a.use_one = 1;                                      // the box travels in the launch parameters
    b.a.one = rec;
    b.drive_mode = 0;
    imhd::Scalars init;
    std::memset(&init, 0, sizeof(init));
    init.active = 1;                                      // cur = 0: state_in is current
    init.dt = dt;

    double host_io[2] = {dt, 0.0};
    unsigned status = 0;
    // the scalars (maxima slots included) start from zero on every call
    e = cudaMemcpyAsync(rec.sc, &init, sizeof(init), cudaMemcpyHostToDevice, b.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(table, &rec, sizeof(rec), cudaMemcpyHostToDevice, b.st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(table + 256, prefix.data(), prefix.size() * sizeof(int), cudaMemcpyHostToDevice, b.st);
    if (e == cudaSuccess) e = precision == 64 ? imhd::run_step<double>(b, 0) : imhd::run_step<float>(b, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host_io[1], &rec.sc->dt_next, sizeof(double), cudaMemcpyDeviceToHost, b.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, &rec.sc->status, sizeof(unsigned), cudaMemcpyDeviceToHost, b.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b.st);
    if (e != cudaSuccess) return fail(IMHD_E_CUDA, std::string("imhd_step_static: ") + cudaGetErrorString(e));
    if (status & IMHD_S_WAIT) return fail(IMHD_E_CUDA, "a bounded wait for an asynchronous copy gave up");
    if (status & IMHD_S_NAN) return fail(IMHD_E_PHYSICS, "non-finite state or max speed: the step is not valid");
    if (status & IMHD_S_ZERO_SPEED) return fail(IMHD_E_PHYSICS, "zero max speed encountered");
    if (dt_next) *dt_next = host_io[1];
    return IMHD_OK;
}
