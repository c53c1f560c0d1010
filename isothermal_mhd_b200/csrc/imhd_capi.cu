// imhd_capi.cu -- the extern "C" boundary of libimhd.so (declared in
// include/imhd.h): box lifetime, host<->device transfer in the reference's
// array layout, and the per-step call sequence.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/imhd.h"
#include "imhd_table.h"
#include "imhd_types.cuh"

namespace imhd {
template <class T> cudaError_t run_step(BatchDev&, int);
template <class T> cudaError_t run_max_speed(BatchDev&);
template <class T> cudaError_t run_force_sums(BatchDev&);
template <class T> cudaError_t run_diag(BatchDev&);
template <class T> cudaError_t run_from_f64(cudaStream_t, const double*, void*, int);
template <class T> cudaError_t run_to_f64(cudaStream_t, const void*, double*, int);
template <class T> cudaError_t run_ou_field(cudaStream_t, const BoxRec&, int, int, const int*, const double*, int,
                                            double);
template <class T> cudaError_t run_init_uniform(cudaStream_t, const BoxRec&, int, double, const double*);
template <class T> cudaError_t run_ref_force(cudaStream_t, const BoxRec&, int, const double*, const double*,
                                             const double*, const double*, const double*, double*, double*, double*,
                                             double*);
}  // namespace imhd

struct imhd_box {
    imhd_config cfg;
    imhd::BoxRec rec;            // host copy of the device record
    imhd::BatchDev b;            // a table of one box
    size_t esz = 8;
    int cur = 0;                 // host mirror of Scalars::cur
    void* pool = nullptr;        // all buffers of the box
    void* table = nullptr;       // device BoxRec + prefix
    double* staging = nullptr;   // N doubles on the device
    double* hio = nullptr;       // pinned host scalars
    bool have_force = false;
    cudaStream_t own_stream = nullptr;
    double stage_ms[imhd::kStages] = {};
    long long stage_n[imhd::kStages] = {};
    // reference force generator: taus88 state, k_max and the unit wave
    // vectors khat(0:k_max, 0:k_max, 0:k_max, 3)
    uint32_t taus[3] = {0, 0, 0};
    int turb_km = 0;
    std::vector<double> khat;
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(IMHD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool is64(const imhd_box* x) { return x->cfg.precision == 64; }

// The box travels by value in the launch parameters, current state first.
void set_one(imhd_box* x) {
    x->b.a.use_one = 1;
    x->b.a.one = x->rec;
    x->b.a.one.S[0] = x->rec.S[x->cur];
    x->b.a.one.S[1] = x->rec.S[x->cur ^ 1];
    x->b.a.one.active = 1;
}

cudaError_t step_dispatch(imhd_box* x) {
    set_one(x);
    return is64(x) ? imhd::run_step<double>(x->b, 0) : imhd::run_step<float>(x->b, 0);
}

void* field_ptr(imhd_box* x, void* base, int f) { return (char*)base + (size_t)f * (size_t)x->rec.n * x->esz; }
void* cur_state(imhd_box* x) { return x->rec.S[x->cur]; }

// (Re)write the device table of the box: its record and block prefixes.
int upload_table(imhd_box* x) {
    std::vector<imhd::BoxRec> recs(1, x->rec);
    std::vector<int> prefix;
    if (!imhd::build_prefix(recs, x->esz, prefix, x->b)) return fail(IMHD_E_ARG, "box too large for one launch");
    CK(cudaMemcpyAsync(x->table, &x->rec, sizeof(imhd::BoxRec), cudaMemcpyHostToDevice, x->b.st));
    CK(cudaMemcpyAsync((char*)x->table + imhd::align256(sizeof(imhd::BoxRec)), prefix.data(), prefix.size() * sizeof(int),
                       cudaMemcpyHostToDevice, x->b.st));
    CK(cudaStreamSynchronize(x->b.st));
    x->b.a.boxes = (imhd::BoxRec*)x->table;
    x->b.a.prefix = (const int*)((char*)x->table + imhd::align256(sizeof(imhd::BoxRec)));
    set_one(x);
    return IMHD_OK;
}

// host field f of a Fortran array a(1-ng:n+ng, ..., nf)
const double* host_field(const imhd_box* x, const double* h, int f, int ng) {
    size_t P = (size_t)(x->cfg.nx + 2 * ng) * (x->cfg.ny + 2 * ng) * (x->cfg.nz + 2 * ng);
    return h + (size_t)f * P;
}

// Copy the interior of a padded host field into a dense device double array.
int copy_in_f64(imhd_box* x, const double* hfield, int ng, double* dst) {
    const imhd_config& c = x->cfg;
    if (ng == 0) {
        CK(cudaMemcpyAsync(dst, hfield, (size_t)x->rec.n * 8, cudaMemcpyHostToDevice, x->b.st));
        return IMHD_OK;
    }
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr((void*)hfield, (size_t)(c.nx + 2 * ng) * 8, (size_t)(c.nx + 2 * ng), (size_t)(c.ny + 2 * ng));
    p.srcPos = make_cudaPos((size_t)ng * 8, (size_t)ng, (size_t)ng);
    p.dstPtr = make_cudaPitchedPtr(dst, (size_t)c.nx * 8, (size_t)c.nx, (size_t)c.ny);
    p.dstPos = make_cudaPos(0, 0, 0);
    p.extent = make_cudaExtent((size_t)c.nx * 8, (size_t)c.ny, (size_t)c.nz);
    p.kind = cudaMemcpyHostToDevice;
    CK(cudaMemcpy3DAsync(&p, x->b.st));
    return IMHD_OK;
}

int copy_out_f64(imhd_box* x, const double* src, double* hfield, int ng) {
    const imhd_config& c = x->cfg;
    if (ng == 0) {
        CK(cudaMemcpyAsync(hfield, src, (size_t)x->rec.n * 8, cudaMemcpyDeviceToHost, x->b.st));
        return IMHD_OK;
    }
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr((void*)src, (size_t)c.nx * 8, (size_t)c.nx, (size_t)c.ny);
    p.srcPos = make_cudaPos(0, 0, 0);
    p.dstPtr = make_cudaPitchedPtr(hfield, (size_t)(c.nx + 2 * ng) * 8, (size_t)(c.nx + 2 * ng), (size_t)(c.ny + 2 * ng));
    p.dstPos = make_cudaPos((size_t)ng * 8, (size_t)ng, (size_t)ng);
    p.extent = make_cudaExtent((size_t)c.nx * 8, (size_t)c.ny, (size_t)c.nz);
    p.kind = cudaMemcpyDeviceToHost;
    CK(cudaMemcpy3DAsync(&p, x->b.st));
    return IMHD_OK;
}

// Upload one host field into device field slot `dst` of precision T.
int upload_field(imhd_box* x, const double* hfield, int ng, void* dst) {
    if (is64(x)) return copy_in_f64(x, hfield, ng, (double*)dst);
    int rc = copy_in_f64(x, hfield, ng, x->staging);
    if (rc) return rc;
    CK(imhd::run_from_f64<float>(x->b.st, x->staging, dst, x->rec.n));
    x->b.launches += 1;
    return IMHD_OK;
}

int download_field(imhd_box* x, const void* src, double* hfield, int ng) {
    if (is64(x)) return copy_out_f64(x, (const double*)src, hfield, ng);
    CK(imhd::run_to_f64<float>(x->b.st, src, x->staging, x->rec.n));
    x->b.launches += 1;
    return copy_out_f64(x, x->staging, hfield, ng);
}

// Periodic ghost fill of one padded host field (boundary_conditions_mod.f90:137-231).
void ghost_fill(const imhd_config& c, double* h, int ng) {
    if (ng == 0) return;
    long Px = c.nx + 2 * ng, Py = c.ny + 2 * ng, Pz = c.nz + 2 * ng;
    auto wrap = [](long i, long n) { i %= n; return i < 0 ? i + n : i; };
    for (long k = 0; k < Pz; ++k) {
        long kk = wrap(k - ng, c.nz) + ng;
        bool kin = (k >= ng && k < ng + c.nz);
        for (long j = 0; j < Py; ++j) {
            long jj = wrap(j - ng, c.ny) + ng;
            bool jin = (j >= ng && j < ng + c.ny);
            for (long i = 0; i < Px; ++i) {
                bool iin = (i >= ng && i < ng + c.nx);
                if (iin && jin && kin) continue;
                long ii = wrap(i - ng, c.nx) + ng;
                h[i + Px * (j + Py * k)] = h[ii + Px * (jj + Py * kk)];
            }
        }
    }
}

int sync_and_check(imhd_box* x) {
    CK(cudaStreamSynchronize(x->b.st));
    CK(cudaGetLastError());
    return IMHD_OK;
}

// Fold the events of the last step into the per-stage accumulators.
int accumulate_stage_times(imhd_box* x) {
    imhd::BatchDev& b = x->b;
    if (!b.prof) return IMHD_OK;
    for (int s = 0; s < imhd::kStages; ++s) {
        if (!(b.prof_mask & (1u << s))) continue;
        int nxt = s + 1;
        while (nxt < imhd::kStages && !(b.prof_mask & (1u << nxt))) ++nxt;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, b.ev[s], b.ev[nxt]));
        x->stage_ms[s] += ms;
        x->stage_n[s] += 1;
    }
    return IMHD_OK;
}

}  // namespace

namespace imhd {
// lets other translation units of the library report through imhd_last_error
const char* set_last_error(int code, const char* msg) {
    (void)code;
    g_err = msg;
    return g_err.c_str();
}

// Upload / download with explicit ghost widths (the C ABI uses the box's
// configured widths; restart files use the reference's nb and nb - 2).
int box_upload_padded(imhd_box* x, const double* q, const double* bface, const double* qpass, int ng, int ng_pass) {
    CK(cudaSetDevice(x->cfg.device));
    int rc;
    for (int f = 0; f < 7; ++f)
        if ((rc = upload_field(x, host_field(x, q, f, ng), ng, field_ptr(x, cur_state(x), f)))) return rc;
    for (int f = 0; f < 3; ++f)
        if ((rc = upload_field(x, host_field(x, bface, f, ng), ng, field_ptr(x, cur_state(x), 7 + f)))) return rc;
    for (int f = 0; f < x->cfg.npass; ++f)
        if ((rc = upload_field(x, host_field(x, qpass, f, ng_pass), ng_pass, field_ptr(x, cur_state(x), 10 + f))))
            return rc;
    return sync_and_check(x);
}

int box_download_padded(imhd_box* x, double* q, double* bface, double* qpass, int ng, int ng_pass) {
    CK(cudaSetDevice(x->cfg.device));
    int rc;
    const imhd_config& c = x->cfg;
    // the transfers of one field reuse the staging buffer, so each field is
    // completed (stream-ordered) before the next conversion overwrites it
    if (q)
        for (int f = 0; f < 7; ++f) {
            if ((rc = download_field(x, field_ptr(x, cur_state(x), f), (double*)host_field(x, q, f, ng), ng))) return rc;
            if ((rc = sync_and_check(x))) return rc;
        }
    if (bface)
        for (int f = 0; f < 3; ++f) {
            if ((rc = download_field(x, field_ptr(x, cur_state(x), 7 + f), (double*)host_field(x, bface, f, ng), ng)))
                return rc;
            if ((rc = sync_and_check(x))) return rc;
        }
    if (qpass && c.npass > 0)
        for (int f = 0; f < c.npass; ++f) {
            if ((rc = download_field(x, field_ptr(x, cur_state(x), 10 + f), (double*)host_field(x, qpass, f, ng_pass),
                                     ng_pass)))
                return rc;
            if ((rc = sync_and_check(x))) return rc;
        }
    if (q) for (int f = 0; f < 7; ++f) ghost_fill(c, (double*)host_field(x, q, f, ng), ng);
    if (bface) for (int f = 0; f < 3; ++f) ghost_fill(c, (double*)host_field(x, bface, f, ng), ng);
    if (qpass) for (int f = 0; f < c.npass; ++f) ghost_fill(c, (double*)host_field(x, qpass, f, ng_pass), ng_pass);
    return IMHD_OK;
}

// The current state buffer of a box and what is needed to read it on the
// box's stream (after the box's pending work).
int box_state_view(imhd_box* x, const void** state, int* nx, int* ny, int* nz, int* npass, int* precision,
                   cudaStream_t* st) {
    CK(cudaSetDevice(x->cfg.device));
    *state = cur_state(x);
    *nx = x->cfg.nx;
    *ny = x->cfg.ny;
    *nz = x->cfg.nz;
    *npass = x->cfg.npass;
    *precision = x->cfg.precision;
    *st = x->b.st;
    return IMHD_OK;
}
}  // namespace imhd

extern "C" {

void imhd_default_config(imhd_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->nx = c->ny = c->nz = 64;
    c->precision = 64;
    c->riemann = IMHD_HLLD;
    c->recon = IMHD_PLM;
    c->npass = 1;
    c->sound_speed = 1.0;
    c->cour = 0.35;
    c->edot = 1.0e-3;
    c->dt_turb = 0.05;
    c->ng = 6;
    c->ng_pass = 4;
    c->device = 0;
}

const char* imhd_last_error(void) { return g_err.c_str(); }

int imhd_create(const imhd_config* cfg, imhd_box** out) {
    if (!cfg || !out) return fail(IMHD_E_ARG, "null argument");
    *out = nullptr;
    const imhd_config& c = *cfg;
    if (c.nx < 4 || c.ny < 4 || c.nz < 4) return fail(IMHD_E_ARG, "every edge needs at least 4 cells");
    if ((double)c.nx * c.ny * c.nz >= 2147483647.0) return fail(IMHD_E_ARG, "box too large (nx*ny*nz must be < 2^31)");
    if (c.ny > 65535 || c.nz > 65535) return fail(IMHD_E_ARG, "ny and nz must be <= 65535");
    if (c.precision != 32 && c.precision != 64) return fail(IMHD_E_ARG, "precision must be 32 or 64");
    if (c.riemann < 1 || c.riemann > 3) return fail(IMHD_E_ARG, "riemann must be IMHD_ROE, IMHD_HLLD or IMHD_HLLE");
    if (c.recon < IMHD_PLM || c.recon > IMHD_PPM_PRIM) return fail(IMHD_E_ARG, "recon must be IMHD_PLM, IMHD_PPM, IMHD_PLM_PRIM or IMHD_PPM_PRIM");
    if (c.npass < 0 || c.npass > imhd::kMaxPass) return fail(IMHD_E_ARG, "npass must be in 0..8");
    if (!(c.sound_speed > 0.0) || !(c.cour > 0.0)) return fail(IMHD_E_ARG, "sound_speed and cour must be positive");
    if (c.ng < 0 || c.ng_pass < 0) return fail(IMHD_E_ARG, "ghost widths must be >= 0");
    if (c.protect != 0 && c.protect != 1) return fail(IMHD_E_ARG, "protect must be 0 or 1");
    if (c.protect && c.riemann != IMHD_ROE)
        return fail(IMHD_E_ARG, "protect needs IMHD_ROE (the reference computes protection fluxes for Roe only)");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (c.device < 0 || c.device >= ndev) return fail(IMHD_E_ARG, "no such CUDA device");
    CK(cudaSetDevice(c.device));

    imhd_box* x = new imhd_box();
    x->cfg = c;
    x->esz = c.precision == 64 ? 8 : 4;
    imhd::init_rec(x->rec, c.nx, c.ny, c.nz, c.npass, c.riemann, c.recon, c.sound_speed, c.cour, c.edot, c.dt_turb,
                   c.protect);
    imhd::BatchDev& b = x->b;
    b.precision = c.precision;
    size_t N = (size_t)x->rec.n;
    size_t table_bytes = imhd::align256(sizeof(imhd::BoxRec)) + (size_t)imhd::kKinds * 2 * sizeof(int);
    bool ok = cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking) == cudaSuccess;
    x->own_stream = b.st;
    ok = ok && cudaMalloc(&x->pool, imhd::box_bytes(x->rec, x->esz, false)) == cudaSuccess;
    ok = ok && cudaMalloc(&x->table, table_bytes) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&x->staging, N * 8) == cudaSuccess;
    ok = ok && cudaMallocHost((void**)&x->hio, 64 * sizeof(double)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        imhd_destroy(x);
        return fail(IMHD_E_NOMEM, "device allocation failed");
    }
    imhd::carve_box(x->rec, (unsigned char*)x->pool, x->esz, false);
    cudaMemsetAsync(x->pool, 0, imhd::box_bytes(x->rec, x->esz, false), b.st);
    imhd::Scalars init;
    std::memset(&init, 0, sizeof(init));
    init.active = 1;
    CK(cudaMemcpyAsync(x->rec.sc, &init, sizeof(init), cudaMemcpyHostToDevice, b.st));
    int rc = upload_table(x);
    if (!rc) rc = sync_and_check(x);
    if (rc) { imhd_destroy(x); return rc; }
    *out = x;
    return IMHD_OK;
}

void imhd_destroy(imhd_box* x) {
    if (!x) return;
    cudaSetDevice(x->cfg.device);
    if (x->b.st) cudaStreamSynchronize(x->b.st);
    if (x->own_stream) cudaStreamSynchronize(x->own_stream);
    void* ptrs[] = {x->pool, x->table, x->rec.delv, x->staging};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (x->hio) cudaFreeHost(x->hio);
    for (int s = 0; s <= imhd::kStages; ++s)
        if (x->b.ev[s]) cudaEventDestroy(x->b.ev[s]);
    if (x->own_stream) cudaStreamDestroy(x->own_stream);
    delete x;
}

int imhd_upload(imhd_box* x, const double* q, const double* bface, const double* qpass) {
    if (!x || !q || !bface) return fail(IMHD_E_ARG, "null argument");
    if (x->cfg.npass > 0 && !qpass) return fail(IMHD_E_ARG, "qpass is NULL but npass > 0");
    return imhd::box_upload_padded(x, q, bface, qpass, x->cfg.ng, x->cfg.ng_pass);
}

int imhd_download(imhd_box* x, double* q, double* bface, double* qpass) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    return imhd::box_download_padded(x, q, bface, qpass, x->cfg.ng, x->cfg.ng_pass);
}

int imhd_set_force(imhd_box* x, const double* delv) {
    if (!x || !delv) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    int rc;
    if (!x->rec.delv) {
        if (cudaMalloc(&x->rec.delv, 3 * (size_t)x->rec.n * x->esz) != cudaSuccess) {
            cudaGetLastError();
            return fail(IMHD_E_NOMEM, "device allocation of the force field failed");
        }
        if ((rc = upload_table(x))) return rc;
    }
    for (int f = 0; f < 3; ++f) {
        if ((rc = upload_field(x, host_field(x, delv, f, x->cfg.ng), x->cfg.ng, field_ptr(x, x->rec.delv, f)))) return rc;
        if ((rc = sync_and_check(x))) return rc;
    }
    x->have_force = true;
    return IMHD_OK;
}

int imhd_get_force(imhd_box* x, double* delv) {
    if (!x || !delv) return fail(IMHD_E_ARG, "null argument");
    if (!x->have_force || !x->rec.delv) return fail(IMHD_E_STATE, "the box has no force field");
    CK(cudaSetDevice(x->cfg.device));
    int rc;
    for (int f = 0; f < 3; ++f) {
        double* h = (double*)host_field(x, delv, f, x->cfg.ng);
        if ((rc = download_field(x, field_ptr(x, x->rec.delv, f), h, x->cfg.ng))) return rc;
        if ((rc = sync_and_check(x))) return rc;
        ghost_fill(x->cfg, h, x->cfg.ng);
    }
    return IMHD_OK;
}

int imhd_force_sums(imhd_box* x, double* sums) {
    if (!x || !sums) return fail(IMHD_E_ARG, "null argument");
    if (!x->have_force) return fail(IMHD_E_STATE, "imhd_force_sums before imhd_set_force");
    CK(cudaSetDevice(x->cfg.device));
    set_one(x);
    CK(is64(x) ? imhd::run_force_sums<double>(x->b) : imhd::run_force_sums<float>(x->b));
    CK(cudaMemcpyAsync(x->hio + 24, x->rec.sc->sums, 5 * sizeof(double), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    std::memcpy(sums, x->hio + 24, 5 * sizeof(double));
    return IMHD_OK;
}

int imhd_set_force_sums(imhd_box* x, const double* sums) {
    if (!x || !sums) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    std::memcpy(x->hio + 24, sums, 5 * sizeof(double));
    const unsigned one = 1u;
    std::memcpy(x->hio + 29, &one, sizeof(one));
    CK(cudaMemcpyAsync(x->rec.sc->sums, x->hio + 24, 5 * sizeof(double), cudaMemcpyHostToDevice, x->b.st));
    CK(cudaMemcpyAsync(&x->rec.sc->ext_sums, x->hio + 29, sizeof(unsigned), cudaMemcpyHostToDevice, x->b.st));
    return sync_and_check(x);
}

int imhd_step(imhd_box* x, double dt, int drive_next, double* dt_next) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    if (!(dt > 0.0)) return fail(IMHD_E_ARG, "dt must be positive");
    if (drive_next && !x->have_force) return fail(IMHD_E_STATE, "drive step requested before imhd_set_force");
    CK(cudaSetDevice(x->cfg.device));
    imhd::Scalars* sc = x->rec.sc;
    x->hio[0] = dt;
    int drive = drive_next ? 1 : 0;
    std::memcpy(x->hio + 4, &drive, sizeof(int));
    CK(cudaMemcpyAsync(&sc->dt, x->hio, sizeof(double), cudaMemcpyHostToDevice, x->b.st));
    CK(cudaMemcpyAsync(&sc->drive, x->hio + 4, sizeof(int), cudaMemcpyHostToDevice, x->b.st));
    x->b.drive_mode = drive;
    CK(step_dispatch(x));
    x->cur ^= 1;
    CK(cudaMemcpyAsync(x->hio + 1, &sc->dt_next, sizeof(double), cudaMemcpyDeviceToHost, x->b.st));
    CK(cudaMemcpyAsync((unsigned*)(x->hio + 2), &sc->status, sizeof(unsigned), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    if ((rc = accumulate_stage_times(x))) return rc;
    if (dt_next) *dt_next = x->hio[1];
    unsigned st = *(unsigned*)(x->hio + 2);
    if (st & IMHD_S_WAIT) return fail(IMHD_E_CUDA, "a bounded wait for an asynchronous copy gave up");
    if (st & IMHD_S_NAN) return fail(IMHD_E_PHYSICS, "non-finite state or max speed: the step is not valid");
    if (st & IMHD_S_ZERO_SPEED) return fail(IMHD_E_PHYSICS, "zero max speed encountered");
    if (st & IMHD_S_FORCE) return fail(IMHD_E_PHYSICS, "bad value in turbulence driver energy normalisation");
    if (st & IMHD_S_PROTECT) return fail(IMHD_E_PHYSICS, "more bad cells than the protection list holds");
    return IMHD_OK;
}

int imhd_max_speed(imhd_box* x, double* cmax) {
    if (!x || !cmax) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    CK(cudaMemsetAsync(x->rec.sc->cfl_slots, 0, sizeof(x->rec.sc->cfl_slots), x->b.st));
    set_one(x);
    CK(is64(x) ? imhd::run_max_speed<double>(x->b) : imhd::run_max_speed<float>(x->b));
    unsigned long long slots[imhd::kSlots];
    CK(cudaMemcpyAsync(slots, x->rec.sc->cfl_slots, sizeof(slots), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    double m = 0.0;
    for (int s = 0; s < imhd::kSlots; ++s) {
        double v;
        std::memcpy(&v, &slots[s], 8);
        if (v != v || v > m) m = v;
    }
    *cmax = m;
    return IMHD_OK;
}

int imhd_diagnostics(imhd_box* x, double out[6]) {
    if (!x || !out) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    set_one(x);
    CK(is64(x) ? imhd::run_diag<double>(x->b) : imhd::run_diag<float>(x->b));
    CK(cudaMemcpyAsync(x->hio + 8, &x->rec.sc->diag[0], 6 * sizeof(double), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    for (int q = 0; q < 6; ++q) out[q] = x->hio[8 + q];
    return IMHD_OK;
}

int imhd_status(imhd_box* x, unsigned* flags, long long* floor_hits, int reset) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    imhd::Scalars s;
    CK(cudaMemcpyAsync(&s, x->rec.sc, sizeof(s), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    unsigned f = s.status;
    if (s.floor_hits) f |= IMHD_S_FLOOR;
    if (flags) *flags = f;
    if (floor_hits) *floor_hits = (long long)s.floor_hits;
    if (reset) {
        CK(cudaMemsetAsync(&x->rec.sc->status, 0, sizeof(unsigned), x->b.st));
        CK(cudaMemsetAsync(&x->rec.sc->floor_hits, 0, sizeof(unsigned long long), x->b.st));
        return sync_and_check(x);
    }
    return IMHD_OK;
}

int imhd_wave_speeds(imhd_box* x, double* smax, double* delv_max) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    CK(cudaMemcpyAsync(x->hio + 16, &x->rec.sc->smax_last, 2 * sizeof(double), cudaMemcpyDeviceToHost, x->b.st));
    int rc = sync_and_check(x);
    if (rc) return rc;
    if (smax) *smax = x->hio[16];
    if (delv_max) *delv_max = x->hio[17];
    return IMHD_OK;
}

long long imhd_launch_count(imhd_box* x) { return x ? x->b.launches : 0; }

// ---- reference force generator (turb_driver_mod.f90) ---------------------
namespace {

// taus88 (turb_driver_mod.f90:104-126): three Tausworthe components with the
// 32-bit masks 0xFFFFFFFE, 0xFFFFFFF8, 0xFFFFFFF0 and logical shifts; the
// result is 0.5 + (signed 32-bit xor) * 2.3283064365e-10.
double taus88(uint32_t* s) {
    uint32_t b;
    b = ((s[0] << 13) ^ s[0]) >> 19;
    s[0] = ((s[0] & 0xFFFFFFFEu) << 12) ^ b;
    b = ((s[1] << 2) ^ s[1]) >> 25;
    s[1] = ((s[1] & 0xFFFFFFF8u) << 4) ^ b;
    b = ((s[2] << 3) ^ s[2]) >> 11;
    s[2] = ((s[2] & 0xFFFFFFF0u) << 17) ^ b;
    int32_t x = (int32_t)(s[0] ^ (s[1] ^ s[2]));
    return 0.5 + (double)x * 2.3283064365e-10;
}

double sqd(double v) { return v * v; }

}  // namespace

int imhd_init_turb(imhd_box* x, int s1, int s2, int s3, int k_max) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    const imhd_config& c = x->cfg;
    int nmin = c.nx < c.ny ? c.nx : c.ny;
    nmin = nmin < c.nz ? nmin : c.nz;
    // turb_driver_mod.f90:31-35
    if (k_max < 1 || k_max >= nmin / 2) return fail(IMHD_E_ARG, "k_max must be >= 1 and < min(nx, ny, nz) / 2");
    x->taus[0] = (uint32_t)s1;
    x->taus[1] = (uint32_t)s2;
    x->taus[2] = (uint32_t)s3;
    x->turb_km = k_max;
    // khat (turb_driver_mod.f90:46-66) for kx, ky, kz = 1..k_max; the entries
    // with a zero component are never assigned by the reference and are 0 here
    const int m = k_max + 1;
    x->khat.assign((size_t)m * m * m * 3, 0.0);
    const double TWOPI = 8.0 * std::atan(1.0);
    const double dx = x->rec.dx;
    const double kx0 = TWOPI / ((double)c.nx * dx), ky0 = TWOPI / ((double)c.ny * dx), kz0 = TWOPI / ((double)c.nz * dx);
    for (int kz = 1; kz <= k_max; ++kz)
        for (int ky = 1; ky <= k_max; ++ky)
            for (int kx = 1; kx <= k_max; ++kx) {
                double kk = std::sqrt(sqd(kx * kx0) + sqd(ky * ky0) + sqd(kz * kz0));
                double* h = &x->khat[(((size_t)kz * m + ky) * m + kx) * 3];
                h[0] = kx0 * kx / kk;
                h[1] = ky0 * ky / kk;
                h[2] = kz0 * kz / kk;
            }
    return IMHD_OK;
}

int imhd_turb_seeds(imhd_box* x, int* s1, int* s2, int* s3) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    if (s1) *s1 = (int)x->taus[0];
    if (s2) *s2 = (int)x->taus[1];
    if (s3) *s3 = (int)x->taus[2];
    return IMHD_OK;
}

// generate_rand_force (turb_driver_mod.f90:197-391) for one rank: the
// spectrum on the host (serial taus88 draws, k^6 exp(-8k/k_pk) power,
// solenoidal projection with khat, Hermitian mirror), the separable inverse
// DFT on the device; the field lands in the box's force buffer.
int imhd_generate_force(imhd_box* x) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    if (x->turb_km == 0) return fail(IMHD_E_STATE, "imhd_init_turb must come before imhd_generate_force");
    CK(cudaSetDevice(x->cfg.device));
    const imhd_config& c = x->cfg;
    const int km = x->turb_km, nk = 2 * km, m = km + 1;
    const double TWOPI = 8.0 * std::atan(1.0);
    const double dx = x->rec.dx;
    const double Lx = (double)c.nx * dx, Ly = (double)c.ny * dx, Lz = (double)c.nz * dx;
    const double kx0 = TWOPI / Lx, ky0 = TWOPI / Ly, kz0 = TWOPI / Lz;
    double Lmax = Lx > Ly ? Lx : Ly;
    Lmax = Lmax > Lz ? Lmax : Lz;
    const double k_pk = TWOPI / Lmax;
    const double sol_frac = 1.0;                         // turb_driver_mod.f90:214
    const double const_sol = std::sqrt(sol_frac);
    const double const_comp = std::sqrt(2.0 * (1.0 - sol_frac));
    // spectrum V[c][kz][ky][kx], k = -km..km-1 stored at k + km (the +km
    // entries of the reference's arrays are never read by the transform)
    std::vector<double> V((size_t)2 * 3 * nk * nk * nk, 0.0);
    double* Vre = V.data();
    double* Vim = V.data() + (size_t)3 * nk * nk * nk;
    auto K = [&](int kx, int ky, int kz, int cc) { return (((size_t)cc * nk + (kz + km)) * nk + (ky + km)) * nk + (kx + km); };
    for (int kz = 0; kz <= km - 1; ++kz)
        for (int ky = 0; ky <= km - 1; ++ky)
            for (int kx = 0; kx <= km - 1; ++kx) {
                double kk = std::sqrt(sqd(kx * kx0) + sqd(ky * ky0) + sqd(kz * kz0));
                double k3 = (kk * kk) * kk;                  // k**6 as (k*k*k)**2
                double Pk = (k3 * k3) * std::exp(-8.0 * kk / k_pk);
                double rn[6];
                for (int r = 0; r < 6; ++r) rn[r] = taus88(x->taus);
                double amp[3], ph[3], dre[3], dim[3];
                for (int q = 0; q < 3; ++q) amp[q] = std::sqrt(-2.0 * Pk * std::log(rn[q]));
                for (int q = 0; q < 3; ++q) ph[q] = TWOPI * rn[3 + q];
                for (int q = 0; q < 3; ++q) {
                    dre[q] = amp[q] * std::cos(ph[q]);
                    dim[q] = amp[q] * std::sin(ph[q]);
                }
                const double* kh = &x->khat[(((size_t)kz * m + ky) * m + kx) * 3];
                double dotre = kh[0] * dre[0] + kh[1] * dre[1] + kh[2] * dre[2];
                double dotim = kh[0] * dim[0] + kh[1] * dim[1] + kh[2] * dim[2];
                for (int q = 0; q < 3; ++q) {
                    double cre = kh[q] * dotre, cim = kh[q] * dotim;
                    double sre = dre[q] - cre, sim = dim[q] - cim;
                    Vre[K(kx, ky, kz, q)] = const_sol * sre + const_comp * cre;
                    Vim[K(kx, ky, kz, q)] = const_sol * sim + const_comp * cim;
                    Vre[K(-kx, -ky, -kz, q)] = Vre[K(kx, ky, kz, q)];
                    Vim[K(-kx, -ky, -kz, q)] = -Vim[K(kx, ky, kz, q)];
                }
            }
    // twiddles cos/sin(theta0 * i * k), i = 1..n the reference's cell index
    auto twiddles = [&](int n) {
        std::vector<double> tw((size_t)2 * n * (nk - 1));
        const double theta0 = TWOPI / (double)n;
        for (int i = 1; i <= n; ++i)
            for (int jj = -(km - 1); jj <= km - 1; ++jj) {
                double theta = theta0 * (double)i * (double)jj;
                tw[(size_t)(i - 1) * (nk - 1) + (jj + km - 1)] = std::cos(theta);
                tw[(size_t)n * (nk - 1) + (size_t)(i - 1) * (nk - 1) + (jj + km - 1)] = std::sin(theta);
            }
        return tw;
    };
    std::vector<double> twx = twiddles(c.nx), twy = twiddles(c.ny), twz = twiddles(c.nz);
    int rc;
    if (!x->rec.delv) {
        if (cudaMalloc(&x->rec.delv, 3 * (size_t)x->rec.n * x->esz) != cudaSuccess) {
            cudaGetLastError();
            return fail(IMHD_E_NOMEM, "device allocation of the force field failed");
        }
        if ((rc = upload_table(x))) return rc;
    }
    const size_t nV = V.size(), nX = twx.size(), nY = twy.size(), nZ = twz.size();
    const size_t n1 = (size_t)3 * nk * nk * c.nx, n2 = (size_t)3 * nk * c.ny * c.nx;
    double* d = nullptr;
    const size_t total = nV + nX + nY + nZ + 2 * n1 + 2 * n2;
    CK(cudaMallocAsync((void**)&d, total * sizeof(double), x->b.st));
    double* dV = d;
    double* dX = dV + nV;
    double* dY = dX + nX;
    double* dZ = dY + nY;
    double* s1 = dZ + nZ;
    double* s2 = s1 + 2 * n1;
    cudaError_t e = cudaMemcpyAsync(dV, V.data(), nV * 8, cudaMemcpyHostToDevice, x->b.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dX, twx.data(), nX * 8, cudaMemcpyHostToDevice, x->b.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dY, twy.data(), nY * 8, cudaMemcpyHostToDevice, x->b.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dZ, twz.data(), nZ * 8, cudaMemcpyHostToDevice, x->b.st);
    if (e == cudaSuccess)
        e = is64(x) ? imhd::run_ref_force<double>(x->b.st, x->rec, km, dV, dV + nV / 2, dX, dY, dZ, s1, s1 + n1, s2, s2 + n2)
                    : imhd::run_ref_force<float>(x->b.st, x->rec, km, dV, dV + nV / 2, dX, dY, dZ, s1, s1 + n1, s2, s2 + n2);
    x->b.launches += 3;
    if (e == cudaSuccess) e = cudaStreamSynchronize(x->b.st);   // host vectors stay alive until the copies end
    cudaFreeAsync(d, x->b.st);
    CK(e);
    x->have_force = true;
    return sync_and_check(x);
}

int imhd_set_geometry(imhd_box* x, double dx, int zlo, int zhi) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    if (!(dx > 0.0)) return fail(IMHD_E_ARG, "dx must be positive");
    if (zlo < 0 || zhi > x->cfg.nz || zlo >= zhi) return fail(IMHD_E_ARG, "need 0 <= zlo < zhi <= nz");
    CK(cudaSetDevice(x->cfg.device));
    x->rec.dx = dx;
    x->rec.zlo = zlo;
    x->rec.zhi = zhi;
    return upload_table(x);
}

int imhd_pack_planes(imhd_box* x, int z0, int nplanes, void* dst) {
    if (!x || !dst) return fail(IMHD_E_ARG, "null argument");
    if (z0 < 0 || nplanes < 0 || z0 + nplanes > x->cfg.nz) return fail(IMHD_E_ARG, "plane range outside the box");
    CK(cudaSetDevice(x->cfg.device));
    const size_t plane = (size_t)x->cfg.nx * x->cfg.ny * x->esz;
    const int nf = 10 + x->cfg.npass;
    for (int f = 0; f < nf; ++f)
        CK(cudaMemcpyAsync((char*)dst + (size_t)f * nplanes * plane,
                           (const char*)field_ptr(x, cur_state(x), f) + (size_t)z0 * plane, (size_t)nplanes * plane,
                           cudaMemcpyDeviceToDevice, x->b.st));
    return sync_and_check(x);
}

int imhd_unpack_planes(imhd_box* x, int z0, int nplanes, const void* src) {
    if (!x || !src) return fail(IMHD_E_ARG, "null argument");
    if (z0 < 0 || nplanes < 0 || z0 + nplanes > x->cfg.nz) return fail(IMHD_E_ARG, "plane range outside the box");
    CK(cudaSetDevice(x->cfg.device));
    const size_t plane = (size_t)x->cfg.nx * x->cfg.ny * x->esz;
    const int nf = 10 + x->cfg.npass;
    for (int f = 0; f < nf; ++f)
        CK(cudaMemcpyAsync((char*)field_ptr(x, cur_state(x), f) + (size_t)z0 * plane,
                           (const char*)src + (size_t)f * nplanes * plane, (size_t)nplanes * plane,
                           cudaMemcpyDeviceToDevice, x->b.st));
    return sync_and_check(x);
}

int imhd_init_uniform(imhd_box* x, double rho, const double* b0) {
    if (!x || !b0) return fail(IMHD_E_ARG, "null argument");
    if (!(rho > 0.0)) return fail(IMHD_E_ARG, "rho must be positive");
    CK(cudaSetDevice(x->cfg.device));
    CK(is64(x) ? imhd::run_init_uniform<double>(x->b.st, x->rec, x->cur, rho, b0)
               : imhd::run_init_uniform<float>(x->b.st, x->rec, x->cur, rho, b0));
    x->b.launches += 1;
    return sync_and_check(x);
}

int imhd_fourier_field(imhd_box* x, int target, const int* kvec, const double* amp, int nmodes, double scale) {
    if (!x || nmodes < 0 || (nmodes > 0 && (!kvec || !amp))) return fail(IMHD_E_ARG, "bad argument");
    if (target != 0 && target != 1) return fail(IMHD_E_ARG, "target must be 0 (velocity) or 1 (force)");
    CK(cudaSetDevice(x->cfg.device));
    int rc;
    if (target == 1 && !x->rec.delv) {
        if (cudaMalloc(&x->rec.delv, 3 * (size_t)x->rec.n * x->esz) != cudaSuccess) {
            cudaGetLastError();
            return fail(IMHD_E_NOMEM, "device allocation of the force field failed");
        }
        if ((rc = upload_table(x))) return rc;
    }
    int* kd = nullptr;
    double* ad = nullptr;
    if (nmodes) {
        CK(cudaMallocAsync((void**)&kd, (size_t)nmodes * 3 * sizeof(int), x->b.st));
        CK(cudaMallocAsync((void**)&ad, (size_t)nmodes * 6 * sizeof(double), x->b.st));
        CK(cudaMemcpyAsync(kd, kvec, (size_t)nmodes * 3 * sizeof(int), cudaMemcpyHostToDevice, x->b.st));
        CK(cudaMemcpyAsync(ad, amp, (size_t)nmodes * 6 * sizeof(double), cudaMemcpyHostToDevice, x->b.st));
    }
    cudaError_t e = is64(x) ? imhd::run_ou_field<double>(x->b.st, x->rec, x->cur, target, kd, ad, nmodes, scale)
                            : imhd::run_ou_field<float>(x->b.st, x->rec, x->cur, target, kd, ad, nmodes, scale);
    x->b.launches += 1;
    if (kd) cudaFreeAsync(kd, x->b.st);
    if (ad) cudaFreeAsync(ad, x->b.st);
    CK(e);
    if (target == 1) x->have_force = true;
    return sync_and_check(x);
}

int imhd_set_stream(imhd_box* x, void* stream) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    CK(cudaStreamSynchronize(x->b.st));
    x->b.st = stream ? (cudaStream_t)stream : x->own_stream;
    return IMHD_OK;
}

int imhd_profile(imhd_box* x, int enable) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    CK(cudaSetDevice(x->cfg.device));
    if (enable && !x->b.ev[0])
        for (int s = 0; s <= imhd::kStages; ++s) CK(cudaEventCreate(&x->b.ev[s]));
    x->b.prof = enable != 0;
    return IMHD_OK;
}

int imhd_stage_times(imhd_box* x, double* ms, long long* count, int n, int reset) {
    if (!x) return fail(IMHD_E_ARG, "null argument");
    if (n != imhd::kStages) return fail(IMHD_E_ARG, "n must be IMHD_NSTAGES");
    for (int s = 0; s < n; ++s) {
        if (ms) ms[s] = x->stage_ms[s];
        if (count) count[s] = x->stage_n[s];
        if (reset) { x->stage_ms[s] = 0.0; x->stage_n[s] = 0; }
    }
    return IMHD_OK;
}

}  // extern "C"
