// imhd_batch.cu -- many independent periodic boxes advanced together.
//
// All boxes of a batch share one table (imhd_table.h): every kernel launch of
// a step covers the blocks of all boxes, so small boxes no longer pay a full
// step's launch latency each and large and small boxes fill the GPU together.
// Each box keeps its own clock on the device (Scalars: t, dt, t_turb, steps),
// so a step reads nothing from the host: one step of the whole batch is
// captured once into a CUDA graph and replayed.  This is the reference's
// driver loop (driver.f90:35-186) run per box on the device.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/imhd.h"
#include "imhd_table.h"
#include "imhd_types.cuh"

namespace imhd {
template <class T> cudaError_t run_step(BatchDev&, int);
template <class T> cudaError_t prepare_launch(BatchDev&);
template <class T> cudaError_t run_max_speed(BatchDev&);
template <class T> cudaError_t run_diag(BatchDev&);
template <class T> cudaError_t run_from_f64(cudaStream_t, const double*, void*, int);
template <class T> cudaError_t run_to_f64(cudaStream_t, const void*, double*, int);
template <class T> cudaError_t run_ou_field(cudaStream_t, const BoxRec&, int, int, const int*, const double*, int,
                                            double);
template <class T> cudaError_t run_init_uniform(cudaStream_t, const BoxRec&, int, double, const double*);
const char* set_last_error(int code, const char* msg);
}  // namespace imhd

struct imhd_batch {
    std::vector<imhd_config> cfg;
    std::vector<imhd::BoxRec> rec;      // host copies of the device records
    imhd::BatchDev b;
    size_t esz = 8;
    int device = 0;
    void* pool = nullptr;
    void* table = nullptr;
    double* staging = nullptr;          // largest box, doubles
    int* modes_dev = nullptr;           // scratch of the field generator
    double* amps_dev = nullptr;
    int modes_cap = 0;
    cudaStream_t st = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_dirty = true;
    long long graph_kernels = 0;        // kernel launches of one replay
    size_t table_cap = 0;               // bytes of the device table
    // online tuning of the decomposition (x tile width policy, y/z sweep
    // segment, z column length): the first replays of a run time candidate
    // settings; they are real steps, and every setting computes the same bits
    bool tune = true;
    int tune_stage = 0;                 // 0: z column, 1: sweep segment, 2: tile policy, 3: done
    int tune_idx = 0;
    int cfg_tile = 0, cfg_segs = imhd::kSegLog, cfg_segzs = imhd::kSegZLog;   // current setting
    int best_tile = 0, best_segs = imhd::kSegLog, best_segzs = imhd::kSegZLog;
    float best_ms = 0.f;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

int bfail(int code, const std::string& m) {
    imhd::set_last_error(code, m.c_str());
    return code;
}

#define BCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return bfail(IMHD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

bool b64(const imhd_batch* x) { return x->b.precision == 64; }

const double* bhost_field(const imhd_config& c, const double* h, int f, int ng) {
    size_t P = (size_t)(c.nx + 2 * ng) * (c.ny + 2 * ng) * (c.nz + 2 * ng);
    return h + (size_t)f * P;
}

int bcopy(imhd_batch* x, const imhd_config& c, const void* src, void* dst, int ng, cudaMemcpyKind kind, bool padded_is_src) {
    if (ng == 0) {
        BCK(cudaMemcpyAsync(dst, src, (size_t)c.nx * c.ny * c.nz * 8, kind, x->st));
        return IMHD_OK;
    }
    cudaMemcpy3DParms p;
    std::memset(&p, 0, sizeof(p));
    cudaPitchedPtr padded = make_cudaPitchedPtr(const_cast<void*>(padded_is_src ? src : dst), (size_t)(c.nx + 2 * ng) * 8,
                                                (size_t)(c.nx + 2 * ng), (size_t)(c.ny + 2 * ng));
    cudaPitchedPtr dense = make_cudaPitchedPtr(const_cast<void*>(padded_is_src ? dst : src), (size_t)c.nx * 8,
                                               (size_t)c.nx, (size_t)c.ny);
    if (padded_is_src) {
        p.srcPtr = padded; p.srcPos = make_cudaPos((size_t)ng * 8, (size_t)ng, (size_t)ng);
        p.dstPtr = dense; p.dstPos = make_cudaPos(0, 0, 0);
    } else {
        p.srcPtr = dense; p.srcPos = make_cudaPos(0, 0, 0);
        p.dstPtr = padded; p.dstPos = make_cudaPos((size_t)ng * 8, (size_t)ng, (size_t)ng);
    }
    p.extent = make_cudaExtent((size_t)c.nx * 8, (size_t)c.ny, (size_t)c.nz);
    p.kind = kind;
    BCK(cudaMemcpy3DAsync(&p, x->st));
    return IMHD_OK;
}

int bupload_field(imhd_batch* x, int box, const double* h, int ng, void* dst) {
    const imhd_config& c = x->cfg[box];
    if (b64(x)) return bcopy(x, c, h, dst, ng, cudaMemcpyHostToDevice, true);
    int rc = bcopy(x, c, h, x->staging, ng, cudaMemcpyHostToDevice, true);
    if (rc) return rc;
    BCK(imhd::run_from_f64<float>(x->st, x->staging, dst, x->rec[box].n));
    x->b.launches += 1;
    return IMHD_OK;
}

int bdownload_field(imhd_batch* x, int box, const void* src, double* h, int ng) {
    const imhd_config& c = x->cfg[box];
    if (b64(x)) {
        int rc = bcopy(x, c, src, h, ng, cudaMemcpyDeviceToHost, false);
        if (rc) return rc;
    } else {
        BCK(imhd::run_to_f64<float>(x->st, src, x->staging, x->rec[box].n));
        x->b.launches += 1;
        int rc = bcopy(x, c, x->staging, h, ng, cudaMemcpyDeviceToHost, false);
        if (rc) return rc;
    }
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

void bghost_fill(const imhd_config& c, double* h, int ng) { imhd::host_ghost_fill(c.nx, c.ny, c.nz, h, ng); }

int read_scalars(imhd_batch* x, int box, imhd::Scalars& s) {
    BCK(cudaMemcpyAsync(&s, x->rec[box].sc, sizeof(s), cudaMemcpyDeviceToHost, x->st));
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}
int write_scalars(imhd_batch* x, int box, const imhd::Scalars& s) {
    BCK(cudaMemcpyAsync(x->rec[box].sc, &s, sizeof(s), cudaMemcpyHostToDevice, x->st));
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

bool check_box(imhd_batch* x, int box) { return x && box >= 0 && box < (int)x->rec.size(); }

// Box `box` of the batch alone, its record (current state first) in the
// kernel parameters: per-box operations launch over that box only.
imhd::BatchDev one_box(const imhd_batch* x, int box, int cur) {
    imhd::BatchDev d = x->b;
    const imhd::BoxRec& r = x->rec[box];
    d.a.use_one = 1;
    d.a.one = r;
    d.a.one.S[0] = r.S[cur];
    d.a.one.S[1] = r.S[cur ^ 1];
    d.a.one.active = 1;
    d.a.nbox = 1;
    for (int k = 0; k < imhd::kKinds; ++k) d.totals[k] = (int)imhd::blocks_of(r, k, x->esz);
    d.prof = false;
    d.launches = 0;
    return d;
}

}  // namespace

extern "C" {

int imhd_batch_create(const imhd_config* cfgs, int nbox, imhd_batch** out) {
    if (!cfgs || !out || nbox < 1) return bfail(IMHD_E_ARG, "need at least one box configuration");
    *out = nullptr;
    int prec = cfgs[0].precision, dev = cfgs[0].device;
    for (int i = 0; i < nbox; ++i) {
        const imhd_config& c = cfgs[i];
        if (c.precision != prec || c.device != dev) return bfail(IMHD_E_ARG, "all boxes of a batch share precision and device");
        if (c.nx < 4 || c.ny < 4 || c.nz < 4) return bfail(IMHD_E_ARG, "every edge needs at least 4 cells");
        if ((double)c.nx * c.ny * c.nz >= 2147483647.0) return bfail(IMHD_E_ARG, "box too large");
        if (c.precision != 32 && c.precision != 64) return bfail(IMHD_E_ARG, "precision must be 32 or 64");
        if (c.riemann < 1 || c.riemann > 3) return bfail(IMHD_E_ARG, "riemann must be IMHD_ROE, IMHD_HLLD or IMHD_HLLE");
        if (c.recon < IMHD_PLM || c.recon > IMHD_PPM_PRIM) return bfail(IMHD_E_ARG, "recon must be IMHD_PLM, IMHD_PPM, IMHD_PLM_PRIM or IMHD_PPM_PRIM");
        if (c.npass < 0 || c.npass > imhd::kMaxPass) return bfail(IMHD_E_ARG, "npass must be in 0..8");
        if (!(c.sound_speed > 0.0) || !(c.cour > 0.0)) return bfail(IMHD_E_ARG, "sound_speed and cour must be positive");
        if (c.protect != 0 && c.protect != 1) return bfail(IMHD_E_ARG, "protect must be 0 or 1");
        if (c.protect && c.riemann != IMHD_ROE) return bfail(IMHD_E_ARG, "protect needs IMHD_ROE");
    }
    int ndev = 0;
    BCK(cudaGetDeviceCount(&ndev));
    if (dev < 0 || dev >= ndev) return bfail(IMHD_E_ARG, "no such CUDA device");
    BCK(cudaSetDevice(dev));
    imhd_batch* x = new imhd_batch();
    x->cfg.assign(cfgs, cfgs + nbox);
    x->esz = prec == 64 ? 8 : 4;
    x->device = dev;
    x->b.precision = prec;
    x->rec.resize(nbox);
    size_t total = 0, maxn = 0;
    bool forcing = false;
    for (int i = 0; i < nbox; ++i) {
        const imhd_config& c = cfgs[i];
        imhd::init_rec(x->rec[i], c.nx, c.ny, c.nz, c.npass, c.riemann, c.recon, c.sound_speed, c.cour, c.edot, c.dt_turb,
                       c.protect);
        total += imhd::box_bytes(x->rec[i], x->esz, true);
        if ((size_t)x->rec[i].n > maxn) maxn = x->rec[i].n;
        forcing = forcing || c.edot > 0.0;
    }
    imhd::TablePlan plan;
    if (!imhd::plan_table(x->rec, x->esz, x->b, plan)) { delete x; return bfail(IMHD_E_ARG, "batch too large for one launch"); }
    size_t tab = plan.bytes;
    bool ok = cudaStreamCreateWithFlags(&x->st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&x->pool, total) == cudaSuccess;
    ok = ok && cudaMalloc(&x->table, tab) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&x->staging, maxn * 8) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        imhd_batch_destroy(x);
        return bfail(IMHD_E_NOMEM, "device allocation of the batch failed (" + std::to_string(total) + " bytes)");
    }
    x->b.st = x->st;
    unsigned char* p = (unsigned char*)x->pool;
    for (int i = 0; i < nbox; ++i) {
        imhd::carve_box(x->rec[i], p, x->esz, true);
        p += imhd::box_bytes(x->rec[i], x->esz, true);
        x->rec[i].active = 0;            // until scheduled
    }
    BCK(cudaMemsetAsync(x->pool, 0, total, x->st));
    for (int i = 0; i < nbox; ++i) {
        imhd::Scalars init;
        std::memset(&init, 0, sizeof(init));
        BCK(cudaMemcpyAsync(x->rec[i].sc, &init, sizeof(init), cudaMemcpyHostToDevice, x->st));
    }
    BCK(imhd::upload_table(x->table, x->rec, plan, x->st, x->b.a));
    x->table_cap = tab;
    x->b.a.use_one = 0;
    x->b.drive_mode = forcing ? 2 : 0;
    *out = x;
    return IMHD_OK;
}

void imhd_batch_destroy(imhd_batch* x) {
    if (!x) return;
    cudaSetDevice(x->device);
    if (x->st) cudaStreamSynchronize(x->st);
    if (x->exec) cudaGraphExecDestroy(x->exec);
    if (x->graph) cudaGraphDestroy(x->graph);
    if (x->ev0) cudaEventDestroy(x->ev0);
    if (x->ev1) cudaEventDestroy(x->ev1);
    void* ptrs[] = {x->pool, x->table, x->staging, x->modes_dev, x->amps_dev};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (x->st) cudaStreamDestroy(x->st);
    delete x;
}

int imhd_batch_upload(imhd_batch* x, int box, const double* q, const double* bface, const double* qpass) {
    if (!check_box(x, box) || !q || !bface) return bfail(IMHD_E_ARG, "bad box index or null array");
    const imhd_config& c = x->cfg[box];
    if (c.npass > 0 && !qpass) return bfail(IMHD_E_ARG, "qpass is NULL but npass > 0");
    BCK(cudaSetDevice(x->device));
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    imhd::BoxRec& r = x->rec[box];
    size_t fb = (size_t)r.n * x->esz;
    char* S = (char*)r.S[s.cur];
    for (int f = 0; f < 7; ++f)
        if ((rc = bupload_field(x, box, bhost_field(c, q, f, c.ng), c.ng, S + f * fb))) return rc;
    for (int f = 0; f < 3; ++f)
        if ((rc = bupload_field(x, box, bhost_field(c, bface, f, c.ng), c.ng, S + (7 + f) * fb))) return rc;
    for (int f = 0; f < c.npass; ++f)
        if ((rc = bupload_field(x, box, bhost_field(c, qpass, f, c.ng_pass), c.ng_pass, S + (10 + f) * fb))) return rc;
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

int imhd_batch_set_force(imhd_batch* x, int box, const double* delv) {
    if (!check_box(x, box) || !delv) return bfail(IMHD_E_ARG, "bad box index or null array");
    BCK(cudaSetDevice(x->device));
    const imhd_config& c = x->cfg[box];
    imhd::BoxRec& r = x->rec[box];
    size_t fb = (size_t)r.n * x->esz;
    int rc;
    for (int f = 0; f < 3; ++f)
        if ((rc = bupload_field(x, box, bhost_field(c, delv, f, c.ng), c.ng, (char*)r.delv + f * fb))) return rc;
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

int imhd_batch_download(imhd_batch* x, int box, double* q, double* bface, double* qpass) {
    if (!check_box(x, box)) return bfail(IMHD_E_ARG, "bad box index");
    BCK(cudaSetDevice(x->device));
    const imhd_config& c = x->cfg[box];
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    imhd::BoxRec& r = x->rec[box];
    size_t fb = (size_t)r.n * x->esz;
    const char* S = (const char*)r.S[s.cur];
    if (q)
        for (int f = 0; f < 7; ++f)
            if ((rc = bdownload_field(x, box, S + f * fb, (double*)bhost_field(c, q, f, c.ng), c.ng))) return rc;
    if (bface)
        for (int f = 0; f < 3; ++f)
            if ((rc = bdownload_field(x, box, S + (7 + f) * fb, (double*)bhost_field(c, bface, f, c.ng), c.ng))) return rc;
    if (qpass)
        for (int f = 0; f < c.npass; ++f)
            if ((rc = bdownload_field(x, box, S + (10 + f) * fb, (double*)bhost_field(c, qpass, f, c.ng_pass), c.ng_pass)))
                return rc;
    if (q) for (int f = 0; f < 7; ++f) bghost_fill(c, (double*)bhost_field(c, q, f, c.ng), c.ng);
    if (bface) for (int f = 0; f < 3; ++f) bghost_fill(c, (double*)bhost_field(c, bface, f, c.ng), c.ng);
    if (qpass) for (int f = 0; f < c.npass; ++f) bghost_fill(c, (double*)bhost_field(c, qpass, f, c.ng_pass), c.ng_pass);
    return IMHD_OK;
}

int imhd_batch_schedule(imhd_batch* x, int box, double t0, double t_end, long long steps, double dt0, int forcing) {
    if (!check_box(x, box)) return bfail(IMHD_E_ARG, "bad box index");
    if (steps < 0) return bfail(IMHD_E_ARG, "steps must be >= 0");
    if (forcing && x->b.drive_mode == 0) return bfail(IMHD_E_STATE, "forcing needs edot > 0 in the box configuration");
    BCK(cudaSetDevice(x->device));
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    const imhd::BoxRec& r = x->rec[box];
    if (!(dt0 > 0.0)) {
        // COUR*dx/cmax of the uploaded state (get_max_speed_vanleer without smax)
        for (int k = 0; k < imhd::kSlots; ++k) s.cfl_slots[k] = 0ull;
        if ((rc = write_scalars(x, box, s))) return rc;
        imhd::BatchDev d = one_box(x, box, s.cur);
        BCK(b64(x) ? imhd::run_max_speed<double>(d) : imhd::run_max_speed<float>(d));
        x->b.launches += d.launches;
        if ((rc = read_scalars(x, box, s))) return rc;
        double m = 0.0;
        for (int k = 0; k < imhd::kSlots; ++k) {
            double v;
            std::memcpy(&v, &s.cfl_slots[k], 8);
            if (v != v || v > m) m = v;
        }
        if (!(m > 0.0)) return bfail(IMHD_E_PHYSICS, "zero max speed encountered");
        dt0 = r.cour * r.dx / m;
    }
    s.t = t0;
    s.t_end = t_end;
    s.dt = (t_end - t0 < dt0) ? t_end - t0 : dt0;
    s.t_turb = t0 + r.dt_turb;          // driver.f90:342
    s.dt_turb_sched = r.dt_turb;
    s.steps_done = 0;
    s.steps_target = steps;
    s.forcing = forcing ? 1 : 0;
    s.active = (steps > 0 && t0 < t_end) ? 1 : 0;
    s.drive = 0;
    for (int k = 0; k < imhd::kSlots; ++k) s.smax_slots[k] = s.cmax_slots[k] = s.dvmax_slots[k] = 0ull;
    if ((rc = write_scalars(x, box, s))) return rc;
    // the device table holds the running flag the kernels read
    imhd::BoxRec* dev = (imhd::BoxRec*)x->table + box;
    BCK(cudaMemcpyAsync(&dev->active, &s.active, sizeof(int), cudaMemcpyHostToDevice, x->st));
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

namespace {

// x tile width of a box under a tile policy: 0 the widest that the row
// length divides, 1 always 32
int tile_of(int policy, int nx) {
    if (policy == 1) return 5;
    return (nx % 128 == 0) ? 7 : (nx % 64 == 0) ? 6 : 5;
}

// Re-key the table to a decomposition setting.  The device records carry the
// current state buffers and running flags, so they are read back, re-keyed
// and uploaded with new block lists.
int apply_setting(imhd_batch* x, int tile, int segs, int segzs) {
    const int nbox = (int)x->rec.size();
    std::vector<imhd::BoxRec> recs(nbox);
    BCK(cudaMemcpyAsync(recs.data(), x->table, sizeof(imhd::BoxRec) * nbox, cudaMemcpyDeviceToHost, x->st));
    BCK(cudaStreamSynchronize(x->st));
    for (imhd::BoxRec& r : recs) {
        r.tws = tile_of(tile, r.nx);
        r.segs = segs;
        r.segzs = segzs;
    }
    imhd::TablePlan plan;
    imhd::BatchDev nb = x->b;
    if (!imhd::plan_table(recs, x->esz, nb, plan)) return bfail(IMHD_E_ARG, "batch too large for one launch");
    if (plan.bytes > x->table_cap) {
        BCK(cudaStreamSynchronize(x->st));
        cudaFree(x->table);
        x->table = nullptr;
        BCK(cudaMalloc(&x->table, plan.bytes));
        x->table_cap = plan.bytes;
    }
    BCK(imhd::upload_table(x->table, recs, plan, x->st, nb.a));
    x->b = nb;
    x->cfg_tile = tile;
    x->cfg_segs = segs;
    x->cfg_segzs = segzs;
    x->graph_dirty = true;
    return IMHD_OK;
}

int capture(imhd_batch* x) {
    if (!x->graph_dirty) return IMHD_OK;
    BCK(b64(x) ? imhd::prepare_launch<double>(x->b) : imhd::prepare_launch<float>(x->b));
    if (x->exec) { cudaGraphExecDestroy(x->exec); x->exec = nullptr; }
    if (x->graph) { cudaGraphDestroy(x->graph); x->graph = nullptr; }
    BCK(cudaStreamBeginCapture(x->st, cudaStreamCaptureModeThreadLocal));
    const long long before = x->b.launches;
    cudaError_t e = b64(x) ? imhd::run_step<double>(x->b, 1) : imhd::run_step<float>(x->b, 1);
    x->graph_kernels = x->b.launches - before;    // kernels per replay
    x->b.launches = before;
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(x->st, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bfail(IMHD_E_CUDA, std::string("graph capture of the batch step failed: ") +
                                      cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    x->graph = g;
    BCK(cudaGraphInstantiate(&x->exec, x->graph, 0));
    x->graph_dirty = false;
    return IMHD_OK;
}

// Candidate settings by coordinate descent: sweep segment (16, 8, 32), then
// the tile policy at the best segment.
bool next_candidate(imhd_batch* x, int& tile, int& segs, int& segzs) {
    static const int kLogs[3] = {imhd::kSegLog, 3, 5};
    // In FP32 the first slope / edge / carried value of a column comes from a
    // separate copy of the code, whose FMA contraction may differ from the
    // loop's, so the segment lengths would move bits: FP32 tunes the tile
    // policy only (a pure thread-to-cell mapping).
    if (!b64(x) && x->tune_stage < 2) {
        x->tune_stage = 2;
        x->tune_idx = 0;
        if (x->best_ms == 0.f) {          // time the default setting first
            tile = 0; segs = x->best_segs; segzs = x->best_segzs;
            x->tune_idx = -1;
            return true;
        }
    }
    while (x->tune_stage < 3) {
        if (x->tune_stage == 0 && x->tune_idx < 3) {
            tile = x->best_tile; segzs = x->best_segzs; segs = kLogs[x->tune_idx];
            return true;
        }
        if (x->tune_stage == 1) {          // reserved (z column length: compile-time)
            x->tune_stage = 2;
            x->tune_idx = 0;
            continue;
        }
        if (x->tune_stage == 2 && x->tune_idx < 1) {
            tile = 1; segs = x->best_segs; segzs = x->best_segzs;
            return true;
        }
        x->tune_stage += 1;
        x->tune_idx = 0;
    }
    return false;
}

}  // namespace

int imhd_batch_run(imhd_batch* x, int replays) {
    if (!x || replays < 0) return bfail(IMHD_E_ARG, "bad argument");
    BCK(cudaSetDevice(x->device));
    int r = 0, rc;
    if (x->tune && x->tune_stage < 3 && replays > 0) {
        if (!x->ev0) {
            BCK(cudaEventCreate(&x->ev0));
            BCK(cudaEventCreate(&x->ev1));
        }
        int tile, segs, segzs;
        while (r < replays && next_candidate(x, tile, segs, segzs)) {
            if ((tile != x->cfg_tile || segs != x->cfg_segs || segzs != x->cfg_segzs) &&
                (rc = apply_setting(x, tile, segs, segzs)))
                return rc;
            if ((rc = capture(x))) return rc;
            BCK(cudaEventRecord(x->ev0, x->st));
            BCK(cudaGraphLaunch(x->exec, x->st));
            BCK(cudaEventRecord(x->ev1, x->st));
            BCK(cudaEventSynchronize(x->ev1));
            x->b.launches += x->graph_kernels;
            float ms = 0.f;
            BCK(cudaEventElapsedTime(&ms, x->ev0, x->ev1));
            if (x->best_ms == 0.f || ms < x->best_ms) {
                x->best_ms = ms;
                x->best_tile = tile;
                x->best_segs = segs;
                x->best_segzs = segzs;
            }
            x->tune_idx += 1;
            ++r;
        }
        if (x->tune_stage >= 3 &&
            (x->best_tile != x->cfg_tile || x->best_segs != x->cfg_segs || x->best_segzs != x->cfg_segzs) &&
            (rc = apply_setting(x, x->best_tile, x->best_segs, x->best_segzs)))
            return rc;
    }
    if ((rc = capture(x))) return rc;
    for (; r < replays; ++r) {
        BCK(cudaGraphLaunch(x->exec, x->st));
        x->b.launches += x->graph_kernels;
    }
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

int imhd_batch_tuning(imhd_batch* x, int enable, int* done, int* tile_policy, int* sweep_segment, int* z_column) {
    if (!x) return bfail(IMHD_E_ARG, "null argument");
    if (enable >= 0) x->tune = enable != 0;
    if (done) *done = x->tune_stage >= 3;
    if (tile_policy) *tile_policy = x->cfg_tile;
    if (sweep_segment) *sweep_segment = 1 << x->cfg_segs;
    if (z_column) *z_column = 1 << x->cfg_segzs;
    return IMHD_OK;
}

int imhd_batch_clock(imhd_batch* x, int box, double* t, long long* steps, double* dt, int* active) {
    if (!check_box(x, box)) return bfail(IMHD_E_ARG, "bad box index");
    BCK(cudaSetDevice(x->device));
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    if (t) *t = s.t;
    if (steps) *steps = s.steps_done;
    if (dt) *dt = s.dt;
    if (active) *active = s.active;
    if (s.status & (IMHD_S_NAN | IMHD_S_ZERO_SPEED | IMHD_S_FORCE | IMHD_S_PROTECT))
        return bfail(IMHD_E_PHYSICS, "box stopped on a physics error (non-finite state, zero max speed or forcing)");
    return IMHD_OK;
}

int imhd_batch_set_stream(imhd_batch* x, void* stream) {
    if (!x) return bfail(IMHD_E_ARG, "null argument");
    BCK(cudaSetDevice(x->device));
    BCK(cudaStreamSynchronize(x->st));
    x->b.st = stream ? (cudaStream_t)stream : x->st;
    x->st = x->b.st;
    return IMHD_OK;
}

long long imhd_batch_launch_count(imhd_batch* x) { return x ? x->b.launches : 0; }

// Fill one box from a sum of Fourier modes (see imhd_ou_field in imhd.h).
int imhd_batch_init_uniform(imhd_batch* x, int box, double rho, const double* b0) {
    if (!check_box(x, box) || !b0) return bfail(IMHD_E_ARG, "bad box index or null b0");
    if (!(rho > 0.0)) return bfail(IMHD_E_ARG, "rho must be positive");
    BCK(cudaSetDevice(x->device));
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    BCK(b64(x) ? imhd::run_init_uniform<double>(x->st, x->rec[box], s.cur, rho, b0)
               : imhd::run_init_uniform<float>(x->st, x->rec[box], s.cur, rho, b0));
    x->b.launches += 1;
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

int imhd_batch_fourier_field(imhd_batch* x, int box, int target, const int* kvec, const double* amp, int nmodes,
                             double scale) {
    if (!check_box(x, box) || nmodes < 0 || (nmodes > 0 && (!kvec || !amp))) return bfail(IMHD_E_ARG, "bad argument");
    if (target != 0 && target != 1) return bfail(IMHD_E_ARG, "target must be 0 (velocity) or 1 (force)");
    BCK(cudaSetDevice(x->device));
    if (nmodes > x->modes_cap) {
        if (x->modes_dev) cudaFree(x->modes_dev);
        if (x->amps_dev) cudaFree(x->amps_dev);
        x->modes_dev = nullptr; x->amps_dev = nullptr;
        BCK(cudaMalloc((void**)&x->modes_dev, (size_t)nmodes * 3 * sizeof(int)));
        BCK(cudaMalloc((void**)&x->amps_dev, (size_t)nmodes * 6 * sizeof(double)));
        x->modes_cap = nmodes;
    }
    imhd::Scalars s;
    int rc = read_scalars(x, box, s);
    if (rc) return rc;
    if (nmodes) {
        BCK(cudaMemcpyAsync(x->modes_dev, kvec, (size_t)nmodes * 3 * sizeof(int), cudaMemcpyHostToDevice, x->st));
        BCK(cudaMemcpyAsync(x->amps_dev, amp, (size_t)nmodes * 6 * sizeof(double), cudaMemcpyHostToDevice, x->st));
    }
    BCK(b64(x) ? imhd::run_ou_field<double>(x->st, x->rec[box], s.cur, target, x->modes_dev, x->amps_dev, nmodes, scale)
               : imhd::run_ou_field<float>(x->st, x->rec[box], s.cur, target, x->modes_dev, x->amps_dev, nmodes, scale));
    x->b.launches += 1;
    BCK(cudaStreamSynchronize(x->st));
    return IMHD_OK;
}

}  // extern "C"
