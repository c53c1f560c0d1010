// imhd_server.cu -- a request loop that serves box solves with continuous
// batching.
//
// Requests (a box configuration, a step count, an initial condition given as
// a uniform state plus Fourier velocity modes, and optional forcing modes)
// arrive through imhd_server_submit from any host thread.  One worker thread
// steps the resident boxes: all of them together with the batched step (one
// launch per stage over a table of every resident box, per-box device
// clocks, the step captured as a CUDA graph).  A builder thread admits queued
// requests in arrival order while their device bytes fit the HBM budget and
// builds each one (uniform state, Fourier velocity, force field, clock) on a
// stream of its own while the worker steps; built boxes join the resident
// set at the worker's next round.  Every few replays the worker reads all
// clocks in one copy and retires the boxes that finished to a harvester
// thread (download to host, free their memory), so requests that arrive
// while others run join the running batch.
//
// A box computes the same bits whatever else is resident: every launch runs
// the same kernels on each box's own data, and no box reads another's.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/imhd.h"
#include "imhd_table.h"
#include "imhd_types.cuh"

namespace imhd {
template <class T> cudaError_t run_step(BatchDev&, int);
template <class T> cudaError_t prepare_launch(BatchDev&);
template <class T> cudaError_t run_max_speed(BatchDev&);
template <class T> cudaError_t run_to_f64(cudaStream_t, const void*, double*, int);
template <class T> cudaError_t run_ou_field(cudaStream_t, const BoxRec&, int, int, const int*, const double*, int,
                                            double);
template <class T> cudaError_t run_init_uniform(cudaStream_t, const BoxRec&, int, double, const double*);
template <class T> cudaError_t run_clocks(BatchDev&, double*);
const char* set_last_error(int code, const char* msg);
}  // namespace imhd

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kClockWords = 6;   // t, steps, active, cur, status, dt (k_clocks)

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

struct Request {
    long long id = 0;
    imhd_config cfg{};
    long long steps = 0;
    double t_end = 0, dt0 = 0, rho = 1;
    double b0[3] = {0, 0, 0};
    std::vector<int> kvec;
    std::vector<double> amp_v, amp_f;
    double scale_v = 0, scale_f = 0;
    int forcing = 0;
    double t_submit = 0;
};

struct Resident {
    Request req;
    imhd::BoxRec rec{};        // carved buffers, S[0] / S[1] as carved
    void* mem = nullptr;
    size_t bytes = 0;
    int cur = 0;               // buffer holding the current state
    double t_admit = 0;
    cudaEvent_t ev = nullptr;  // end of the box's build on the builder's stream
};

struct Result {
    int state = IMHD_REQ_QUEUED;
    imhd_config cfg{};
    std::vector<unsigned char> raw;   // 10 + npass fields of nx*ny*nz in the device type
    int esz = 8;
    double t = 0, t_submit = 0, t_admit = 0, t_done = 0;
    long long steps = 0;
    unsigned status = 0;
    std::string error;
};

}  // namespace

struct imhd_server {
    imhd_server_config cfg{};
    size_t esz = 4;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request> queue;
    std::unordered_map<long long, Result> results;
    bool stopping = false, drain = true, stopped = false;
    long long next_id = 1;
    std::string fatal;                       // worker's CUDA error, if any
    // statistics (guarded by mu)
    long long admitted = 0, completed = 0, failed = 0, replays = 0, launches = 0, rebuilds = 0;
    size_t used_bytes = 0, peak_bytes = 0;
    long long resident = 0, peak_resident = 0;
    long long resident_cells_ = 0;
    double t_build = 0, t_rebuild = 0, t_step = 0, t_retire = 0, t_harvest = 0;   // seconds per phase
    // built boxes waiting to join the resident set (builder thread -> worker)
    std::deque<Resident> ready;
    int building = 0;                        // boxes the builder is building right now
    bool worker_exit = false;                // the worker left its loop (the builder stops too)
    // finished boxes waiting for their download (harvester thread)
    std::deque<Resident> harvest_q;
    std::condition_variable cv_h;
    bool harvest_stop = false;
};

namespace {

int sfail(int code, const std::string& m) {
    imhd::set_last_error(code, m.c_str());
    return code;
}

bool valid_box(const imhd_config& c, std::string& why) {
    if (c.nx < 4 || c.ny < 4 || c.nz < 4) { why = "every edge needs at least 4 cells"; return false; }
    if ((double)c.nx * c.ny * c.nz >= 2147483647.0) { why = "box too large"; return false; }
    if (c.riemann < 1 || c.riemann > 3) { why = "riemann must be IMHD_ROE, IMHD_HLLD or IMHD_HLLE"; return false; }
    if (c.recon < IMHD_PLM || c.recon > IMHD_PPM_PRIM) { why = "recon must be IMHD_PLM, IMHD_PPM, IMHD_PLM_PRIM or IMHD_PPM_PRIM"; return false; }
    if (c.protect != 0 && c.protect != 1) { why = "protect must be 0 or 1"; return false; }
    if (c.protect && c.riemann != IMHD_ROE) { why = "protect needs IMHD_ROE"; return false; }
    if (c.npass < 0 || c.npass > imhd::kMaxPass) { why = "npass must be in 0..8"; return false; }
    if (!(c.sound_speed > 0.0) || !(c.cour > 0.0)) { why = "sound_speed and cour must be positive"; return false; }
    if (c.ng < 0 || c.ng_pass < 0) { why = "ghost widths must be >= 0"; return false; }
    return true;
}

// Everything the worker thread owns.
struct Worker {
    imhd_server* s;
    bool f64;
    cudaStream_t st = nullptr;
    std::vector<Resident> live;
    imhd::BatchDev b;
    void* table = nullptr;
    size_t table_cap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long graph_kernels = 0;
    bool dirty = true;
    double* clocks_dev = nullptr;
    double* clocks_host = nullptr;   // pinned
    size_t clocks_cap = 0;
    // builder thread state (its stream, mode buffers and error)
    cudaStream_t bst = nullptr;
    int* modes_dev = nullptr;
    double* amps_dev = nullptr;
    size_t modes_cap = 0;
    std::string berr;
    std::string err;

    explicit Worker(imhd_server* srv) : s(srv), f64(srv->cfg.precision == 64) { b.precision = srv->cfg.precision; }

    bool ck(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        if (err.empty()) err = std::string(what) + ": " + cudaGetErrorString(e);
        return false;
    }

    void release_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }

    void teardown() {
        if (st) cudaStreamSynchronize(st);
        release_graph();
        for (Resident& r : live)
            if (r.mem) cudaFree(r.mem);
        live.clear();
        void* p[] = {table, clocks_dev, modes_dev, amps_dev};
        for (void* q : p)
            if (q) cudaFree(q);
        if (clocks_host) cudaFreeHost(clocks_host);
        if (st) cudaStreamDestroy(st);
        st = nullptr;
        if (bst) cudaStreamDestroy(bst);
        bst = nullptr;
    }

    // ---- builder thread: builds admitted boxes on a stream of its own
    bool bck(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        if (berr.empty()) berr = std::string(what) + ": " + cudaGetErrorString(e);
        return false;
    }

    bool ensure_modes(size_t m) {
        if (m <= modes_cap) return true;
        if (modes_dev) cudaFree(modes_dev);
        if (amps_dev) cudaFree(amps_dev);
        modes_dev = nullptr;
        amps_dev = nullptr;
        modes_cap = 0;
        if (!bck(cudaMalloc((void**)&modes_dev, m * 3 * sizeof(int)), "mode allocation")) return false;
        if (!bck(cudaMalloc((void**)&amps_dev, m * 6 * sizeof(double)), "mode allocation")) return false;
        modes_cap = m;
        return true;
    }

    // Build an admitted request on the device, on the builder's stream:
    // buffers, uniform state, Fourier velocity, force field, clock.  False:
    // out of device memory (nothing kept) or a CUDA error (berr set).
    bool build(Resident& r) {
        const Request& q = r.req;
        const imhd_config& c = q.cfg;
        imhd::init_rec(r.rec, c.nx, c.ny, c.nz, c.npass, c.riemann, c.recon, c.sound_speed, c.cour, c.edot, c.dt_turb,
                       c.protect);
        r.bytes = imhd::box_bytes(r.rec, s->esz, q.forcing != 0);
        cudaError_t e = cudaMallocAsync(&r.mem, r.bytes, bst);
        if (e != cudaSuccess) {
            cudaGetLastError();
            r.mem = nullptr;
            return false;
        }
        imhd::carve_box(r.rec, (unsigned char*)r.mem, s->esz, q.forcing != 0);
        r.cur = 0;
        if (!bck(cudaMemsetAsync(r.mem, 0, r.bytes, bst), "box clear")) return false;
        if (!bck(f64 ? imhd::run_init_uniform<double>(bst, r.rec, 0, q.rho, q.b0)
                    : imhd::run_init_uniform<float>(bst, r.rec, 0, q.rho, q.b0), "uniform state")) return false;
        size_t m = q.kvec.size() / 3;
        if (m) {
            if (!ensure_modes(m)) return false;
            if (!bck(cudaMemcpyAsync(modes_dev, q.kvec.data(), m * 3 * sizeof(int), cudaMemcpyHostToDevice, bst), "modes"))
                return false;
            if (!q.amp_v.empty()) {
                if (!bck(cudaMemcpyAsync(amps_dev, q.amp_v.data(), m * 6 * sizeof(double), cudaMemcpyHostToDevice, bst),
                        "velocity modes")) return false;
                if (!bck(f64 ? imhd::run_ou_field<double>(bst, r.rec, 0, 0, modes_dev, amps_dev, (int)m, q.scale_v)
                            : imhd::run_ou_field<float>(bst, r.rec, 0, 0, modes_dev, amps_dev, (int)m, q.scale_v),
                        "velocity field")) return false;
            }
            if (q.forcing) {
                // the velocity launch must finish reading amps_dev first
                if (!bck(cudaStreamSynchronize(bst), "velocity field")) return false;
                if (!bck(cudaMemcpyAsync(amps_dev, q.amp_f.data(), m * 6 * sizeof(double), cudaMemcpyHostToDevice, bst),
                        "force modes")) return false;
                if (!bck(f64 ? imhd::run_ou_field<double>(bst, r.rec, 0, 1, modes_dev, amps_dev, (int)m, q.scale_f)
                            : imhd::run_ou_field<float>(bst, r.rec, 0, 1, modes_dev, amps_dev, (int)m, q.scale_f),
                        "force field")) return false;
            }
        }
        imhd::Scalars sc;
        std::memset(&sc, 0, sizeof(sc));
        double dt0 = q.dt0;
        if (!(dt0 > 0.0)) {
            // COUR*dx/cmax of the initial state (get_max_speed_vanleer without smax)
            if (!bck(cudaMemcpyAsync(r.rec.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, bst), "clock")) return false;
            imhd::BatchDev d;
            d.precision = s->cfg.precision;
            d.a.use_one = 1;
            d.a.one = r.rec;
            d.a.one.active = 1;
            d.a.nbox = 1;
            for (int k = 0; k < imhd::kKinds; ++k) d.totals[k] = (int)imhd::blocks_of(r.rec, k, s->esz);
            d.st = bst;
            if (!bck(f64 ? imhd::run_max_speed<double>(d) : imhd::run_max_speed<float>(d), "initial CFL")) return false;
            imhd::Scalars back;
            if (!bck(cudaMemcpyAsync(&back, r.rec.sc, sizeof(back), cudaMemcpyDeviceToHost, bst), "initial CFL")) return false;
            if (!bck(cudaStreamSynchronize(bst), "initial CFL")) return false;
            double mx = 0.0;
            for (int k = 0; k < imhd::kSlots; ++k) {
                double v;
                std::memcpy(&v, &back.cfl_slots[k], 8);
                if (v != v || v > mx) mx = v;
            }
            dt0 = mx > 0.0 ? r.rec.cour * r.rec.dx / mx : 1.0e-15;
        }
        sc.t = 0.0;
        sc.t_end = q.t_end;
        sc.dt = q.t_end < dt0 ? q.t_end : dt0;
        sc.t_turb = r.rec.dt_turb;            // driver.f90:342
        sc.dt_turb_sched = r.rec.dt_turb;
        sc.steps_target = q.steps;
        sc.forcing = q.forcing;
        sc.active = (q.steps > 0 && 0.0 < q.t_end) ? 1 : 0;
        if (!bck(cudaMemcpyAsync(r.rec.sc, &sc, sizeof(sc), cudaMemcpyHostToDevice, bst), "clock")) return false;
        r.rec.active = sc.active;
        return bck(cudaStreamSynchronize(bst), "box build");
    }

    // Table of the resident boxes (current state first) and the step graph.
    bool rebuild() {
        release_graph();
        if (live.empty()) return true;
        std::vector<imhd::BoxRec> recs;
        recs.reserve(live.size());
        bool forcing = false;
        for (Resident& r : live) {
            imhd::BoxRec t = r.rec;
            t.S[0] = r.rec.S[r.cur];
            t.S[1] = r.rec.S[r.cur ^ 1];
            recs.push_back(t);
            forcing = forcing || r.req.forcing;
        }
        imhd::TablePlan plan;
        if (!imhd::plan_table(recs, s->esz, b, plan)) { err = "resident set too large for one launch"; return false; }
        if (plan.bytes > table_cap) {
            if (table) cudaFree(table);
            table = nullptr;
            table_cap = 0;
            if (!ck(cudaMalloc(&table, plan.bytes), "table allocation")) return false;
            table_cap = plan.bytes;
        }
        if (live.size() > clocks_cap) {
            if (clocks_dev) cudaFree(clocks_dev);
            if (clocks_host) cudaFreeHost(clocks_host);
            clocks_dev = nullptr;
            clocks_host = nullptr;
            size_t cap = live.size() * 2;
            if (!ck(cudaMalloc((void**)&clocks_dev, cap * kClockWords * 8), "clock allocation")) return false;
            if (!ck(cudaMallocHost((void**)&clocks_host, cap * kClockWords * 8), "clock allocation")) return false;
            clocks_cap = cap;
        }
        b.st = st;
        b.drive_mode = forcing ? 2 : 0;
        if (!ck(imhd::upload_table(table, recs, plan, st, b.a), "table upload")) return false;
        if (!ck(f64 ? imhd::prepare_launch<double>(b) : imhd::prepare_launch<float>(b), "launch set-up")) return false;
        if (!ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture")) return false;
        long long before = b.launches;
        cudaError_t e = f64 ? imhd::run_step<double>(b, 1) : imhd::run_step<float>(b, 1);
        graph_kernels = b.launches - before;
        b.launches = before;
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (!ck(e, "graph capture") || !ck(e2, "graph capture")) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        graph = g;
        if (!ck(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate")) return false;
        dirty = false;
        std::lock_guard<std::mutex> lk(s->mu);
        s->rebuilds += 1;
        return true;
    }

    // Builder thread: admit queued requests in arrival order while their
    // bytes fit the budget (and the resident cells the cell limit) and build
    // them on the builder's own stream, overlapping the worker's steps; a
    // built box waits in `ready` with an event the worker's stream waits on.
    void build_loop() {
        cudaSetDevice(s->cfg.device);
        const bool stream_ok = cudaStreamCreateWithFlags(&bst, cudaStreamNonBlocking) == cudaSuccess;
        // after an allocation failure: admit again only once the reserved
        // bytes fell below this mark (a retirement freed memory)
        size_t retry_below = 0;
        for (;;) {
            Request q;
            size_t need = 0;
            long long cells = 0;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                bool got = false;
                while (!got) {
                    if (s->worker_exit || (s->stopping && (!s->drain || s->queue.empty()))) {
                        if (bst) cudaStreamSynchronize(bst);
                        return;
                    }
                    if (!stream_ok) {
                        if (s->fatal.empty()) s->fatal = "builder stream creation failed";
                        s->cv.notify_all();
                        return;
                    }
                    if (retry_below && s->used_bytes < retry_below) retry_below = 0;
                    if (!s->queue.empty() && !retry_below) {
                        const Request& h = s->queue.front();
                        imhd::BoxRec probe;
                        imhd::init_rec(probe, h.cfg.nx, h.cfg.ny, h.cfg.nz, h.cfg.npass, h.cfg.riemann, h.cfg.recon,
                                       h.cfg.sound_speed, h.cfg.cour, h.cfg.edot, h.cfg.dt_turb, h.cfg.protect);
                        need = imhd::box_bytes(probe, s->esz, h.forcing != 0);
                        cells = (long long)h.cfg.nx * h.cfg.ny * h.cfg.nz;
                        // nothing resident, built or downloading: the request is alone
                        const bool alone = s->used_bytes == 0;
                        const bool over_budget = (double)(s->used_bytes + need) > s->cfg.hbm_budget_bytes;
                        const bool over_cells = s->cfg.max_resident_cells > 0 && !alone &&
                                                (s->resident_cells_ + cells) > s->cfg.max_resident_cells;
                        if (!(over_budget || over_cells)) {
                            q = std::move(s->queue.front());
                            s->queue.pop_front();
                            s->used_bytes += need;          // reserved until the harvester frees the box
                            s->resident_cells_ += cells;
                            s->building += 1;
                            got = true;
                            break;
                        }
                        if (alone && (double)need > s->cfg.hbm_budget_bytes) {
                            Result& res = s->results[h.id];
                            res.state = IMHD_REQ_FAILED;
                            res.error = "request needs more device memory than the whole budget";
                            res.t_done = now_s();
                            s->failed += 1;
                            s->queue.pop_front();
                            continue;
                        }
                    }
                    // wait for a request, or for a retirement to free memory
                    s->cv.wait_for(lk, std::chrono::milliseconds(20));
                }
            }
            Resident r;
            r.req = std::move(q);
            r.t_admit = now_s();
            const double t0 = now_s();
            bool ok = build(r);
            if (ok) ok = bck(cudaEventCreateWithFlags(&r.ev, cudaEventDisableTiming), "build event") &&
                         bck(cudaEventRecord(r.ev, bst), "build event");
            std::lock_guard<std::mutex> lk(s->mu);
            s->building -= 1;
            s->t_build += now_s() - t0;
            if (!ok) {
                s->used_bytes -= need;
                s->resident_cells_ -= cells;
                if (r.mem) cudaFreeAsync(r.mem, bst);
                if (r.ev) cudaEventDestroy(r.ev);
                if (!berr.empty()) {       // CUDA error: the server stops
                    if (s->fatal.empty()) s->fatal = berr;
                    Result& res = s->results[r.req.id];
                    res.state = IMHD_REQ_FAILED;
                    res.error = berr;
                    res.t_done = now_s();
                    s->failed += 1;
                    s->cv.notify_all();
                    return;
                }
                // device memory is short: back to the queue until a retirement,
                // or failed when nothing else holds memory
                if (s->used_bytes == 0) {
                    Result& res = s->results[r.req.id];
                    res.state = IMHD_REQ_FAILED;
                    res.error = "device allocation failed";
                    res.t_done = now_s();
                    s->failed += 1;
                } else {
                    s->queue.push_front(std::move(r.req));
                    retry_below = s->used_bytes;
                }
                continue;
            }
            Result& res = s->results[r.req.id];
            res.state = IMHD_REQ_RUNNING;
            res.t_admit = r.t_admit;
            s->admitted += 1;
            s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
            s->ready.push_back(std::move(r));
            s->cv.notify_all();
        }
    }

    // Worker: the built boxes join the resident set (the worker's stream
    // waits for their builds).  False on a CUDA error.
    bool take_ready() {
        std::deque<Resident> got;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            got.swap(s->ready);
        }
        if (got.empty()) return true;
        bool ok = true;
        for (Resident& r : got) {
            if (r.ev) {
                ok = ok && ck(cudaStreamWaitEvent(st, r.ev, 0), "build wait");
                cudaEventDestroy(r.ev);
                r.ev = nullptr;
            }
            live.push_back(std::move(r));
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident = (long long)live.size();
        s->peak_resident = std::max(s->peak_resident, s->resident);
        dirty = true;
        return ok;
    }

    // Read every clock; retire the boxes that stopped.
    bool retire() {
        const int nb = (int)live.size();
        if (!ck(f64 ? imhd::run_clocks<double>(b, clocks_dev) : imhd::run_clocks<float>(b, clocks_dev), "clocks"))
            return false;
        if (!ck(cudaMemcpyAsync(clocks_host, clocks_dev, (size_t)nb * kClockWords * 8, cudaMemcpyDeviceToHost, st),
                "clocks")) return false;
        if (!ck(cudaStreamSynchronize(st), "clocks")) return false;
        std::vector<Resident> keep;
        keep.reserve(live.size());
        for (int i = 0; i < nb; ++i) {
            Resident& r = live[i];
            const double* c = clocks_host + (size_t)i * kClockWords;
            r.cur = (int)c[3];
            const unsigned status = (unsigned)c[4];
            const bool bad = (status & (IMHD_S_NAN | IMHD_S_ZERO_SPEED | IMHD_S_FORCE | IMHD_S_PROTECT)) != 0;
            if (c[2] != 0.0 && !bad) {
                keep.push_back(std::move(r));
                continue;
            }
            std::lock_guard<std::mutex> lk(s->mu);
            s->resident_cells_ -= (long long)r.rec.n;
            Result& res = s->results[r.req.id];
            res.cfg = r.req.cfg;
            res.t = c[0];
            res.steps = (long long)c[1];
            res.status = status;
            res.t_submit = r.req.t_submit;
            res.t_admit = r.t_admit;
            if (bad) {
                res.state = IMHD_REQ_FAILED;
                res.error = "physics error (non-finite state, zero max speed or forcing normalisation)";
                res.t_done = now_s();
                s->failed += 1;
                r.req.steps = -1;          // nothing to download: the harvester only frees it
            }
            s->harvest_q.push_back(std::move(r));
            s->cv_h.notify_all();
            dirty = true;
        }
        live.swap(keep);
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident = (long long)live.size();
        return true;
    }

    void run() {
        if (!ck(cudaSetDevice(s->cfg.device), "cudaSetDevice") ||
            !ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream creation")) {
            finish();
            return;
        }
        // keep freed box memory in the stream-ordered pool for the next admissions
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, s->cfg.device) == cudaSuccess) {
            unsigned long long thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        const int per_round = s->cfg.steps_per_round > 0 ? s->cfg.steps_per_round : 4;
        std::thread harvester([this]() { harvest_loop(); });
        std::thread builder([this]() { build_loop(); });
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (!s->fatal.empty()) break;        // the builder stopped on a CUDA error
                const bool idle = live.empty() && s->ready.empty();
                if (s->stopping && (!s->drain || (s->queue.empty() && idle && s->building == 0))) break;
                if (idle) {
                    s->cv.wait_for(lk, std::chrono::milliseconds(5));
                    continue;
                }
            }
            double t1 = now_s();
            if (!take_ready()) break;
            if (live.empty()) continue;
            if (dirty && !rebuild()) break;
            double t2 = now_s();
            bool ok = true;
            for (int k = 0; k < per_round && ok; ++k) ok = ck(cudaGraphLaunch(exec, st), "graph launch");
            if (!ok) break;
            if (!ck(cudaStreamSynchronize(st), "step")) break;
            double t3 = now_s();
            if (!retire()) break;
            double t4 = now_s();
            std::lock_guard<std::mutex> lk(s->mu);
            s->replays += per_round;
            s->launches += per_round * graph_kernels;
            s->t_rebuild += t2 - t1;
            s->t_step += t3 - t2;
            s->t_retire += t4 - t3;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->worker_exit = true;
            s->cv.notify_all();
        }
        builder.join();
        // boxes built but never stepped (stop without drain, or an error)
        take_ready();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->harvest_stop = true;
            s->cv_h.notify_all();
        }
        harvester.join();
        finish();
    }

    // Download finished boxes on a stream of their own, so that the step
    // loop goes on while results travel to host memory; then free them.
    void harvest_loop() {
        cudaSetDevice(s->cfg.device);
        cudaStream_t hs = nullptr;
        if (cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->fatal.empty()) s->fatal = "harvester stream creation failed";
            hs = nullptr;
        }
        for (;;) {
            Resident r;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                s->cv_h.wait(lk, [this]() { return !s->harvest_q.empty() || s->harvest_stop; });
                if (s->harvest_q.empty()) break;
                r = std::move(s->harvest_q.front());
                s->harvest_q.pop_front();
            }
            double t0 = now_s();
            std::vector<unsigned char> raw;
            cudaError_t e = cudaSuccess;
            if (r.req.steps >= 0 && hs) {
                const size_t bytes = (size_t)(10 + r.rec.npass) * (size_t)r.rec.n * s->esz;
                raw.resize(bytes);
                e = cudaMemcpyAsync(raw.data(), r.rec.S[r.cur], bytes, cudaMemcpyDeviceToHost, hs);
                if (e == cudaSuccess) e = cudaStreamSynchronize(hs);
            }
            cudaFreeAsync(r.mem, hs ? hs : st);
            if (hs) cudaStreamSynchronize(hs);
            std::lock_guard<std::mutex> lk(s->mu);
            s->used_bytes -= r.bytes;
            s->t_harvest += now_s() - t0;
            s->cv.notify_all();           // the builder may admit now
            if (r.req.steps < 0) continue;               // failed: result already recorded
            Result& res = s->results[r.req.id];
            if (e != cudaSuccess || !hs) {
                res.state = IMHD_REQ_FAILED;
                res.error = std::string("result download failed: ") + cudaGetErrorString(e);
                s->failed += 1;
            } else {
                res.raw = std::move(raw);
                res.esz = (int)s->esz;
                res.state = IMHD_REQ_DONE;
                s->completed += 1;
            }
            res.t_done = now_s();
        }
        if (hs) cudaStreamDestroy(hs);
    }

    void finish() {
        teardown();
        std::lock_guard<std::mutex> lk(s->mu);
        if (!err.empty()) s->fatal = err;
        // whatever did not finish is cancelled (stop without drain) or failed (device error)
        for (Request& q : s->queue) {
            Result& res = s->results[q.id];
            res.state = err.empty() ? IMHD_REQ_CANCELLED : IMHD_REQ_FAILED;
            res.error = err.empty() ? "server stopped" : err;
            res.t_done = now_s();
        }
        s->queue.clear();
        for (auto& kv : s->results)
            if (kv.second.state == IMHD_REQ_RUNNING) {
                kv.second.state = err.empty() ? IMHD_REQ_CANCELLED : IMHD_REQ_FAILED;
                kv.second.error = err.empty() ? "server stopped" : err;
                kv.second.t_done = now_s();
            }
        s->used_bytes = 0;
        s->resident = 0;
        s->resident_cells_ = 0;
        s->stopped = true;
        s->cv.notify_all();
    }
};

}  // namespace

extern "C" {

void imhd_server_default_config(imhd_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->precision = 32;
    c->hbm_budget_bytes = 150.0e9;
    c->max_resident_cells = 0;
    c->steps_per_round = 4;
}

int imhd_server_start(const imhd_server_config* cfg, imhd_server** out) {
    if (!cfg || !out) return sfail(IMHD_E_ARG, "null argument");
    *out = nullptr;
    if (cfg->precision != 32 && cfg->precision != 64) return sfail(IMHD_E_ARG, "precision must be 32 or 64");
    if (!(cfg->hbm_budget_bytes > 0.0)) return sfail(IMHD_E_ARG, "hbm_budget_bytes must be positive");
    if (cfg->max_resident_cells < 0 || cfg->steps_per_round < 0) return sfail(IMHD_E_ARG, "negative limit");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess) return sfail(IMHD_E_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    if (cfg->device < 0 || cfg->device >= ndev) return sfail(IMHD_E_ARG, "no such CUDA device");
    imhd_server* s = new imhd_server();
    s->cfg = *cfg;
    s->esz = cfg->precision == 64 ? 8 : 4;
    s->worker = std::thread([s]() {
        Worker w(s);
        w.run();
    });
    *out = s;
    return IMHD_OK;
}

int imhd_server_submit(imhd_server* s, const imhd_request* r, long long* id) {
    if (!s || !r || !id) return sfail(IMHD_E_ARG, "null argument");
    std::string why;
    if (!valid_box(r->box, why)) return sfail(IMHD_E_ARG, why);
    if (r->steps < 0) return sfail(IMHD_E_ARG, "steps must be >= 0");
    if (!(r->rho > 0.0)) return sfail(IMHD_E_ARG, "rho must be positive");
    if (r->nmodes < 0 || (r->nmodes > 0 && (!r->kvec || (!r->amp_velocity && !r->amp_force))))
        return sfail(IMHD_E_ARG, "mode arrays missing");
    if (r->forcing && (!(r->box.edot > 0.0) || r->nmodes == 0 || !r->amp_force))
        return sfail(IMHD_E_ARG, "forcing needs edot > 0 and force modes");
    Request q;
    q.cfg = r->box;
    q.cfg.precision = s->cfg.precision;
    q.cfg.device = s->cfg.device;
    q.steps = r->steps;
    q.t_end = r->t_end > 0.0 ? r->t_end : 1.0e30;
    q.dt0 = r->dt0;
    q.rho = r->rho;
    for (int d = 0; d < 3; ++d) q.b0[d] = r->b0[d];
    if (r->nmodes > 0) {
        q.kvec.assign(r->kvec, r->kvec + 3 * (size_t)r->nmodes);
        if (r->amp_velocity) q.amp_v.assign(r->amp_velocity, r->amp_velocity + 6 * (size_t)r->nmodes);
        if (r->forcing) q.amp_f.assign(r->amp_force, r->amp_force + 6 * (size_t)r->nmodes);
    }
    q.scale_v = r->scale_velocity;
    q.scale_f = r->scale_force;
    q.forcing = r->forcing ? 1 : 0;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping || s->stopped) return sfail(IMHD_E_STATE, "server is stopping");
    q.id = s->next_id++;
    q.t_submit = now_s();
    Result& res = s->results[q.id];
    res.state = IMHD_REQ_QUEUED;
    res.cfg = q.cfg;
    res.t_submit = q.t_submit;
    *id = q.id;
    s->queue.push_back(std::move(q));
    s->cv.notify_all();
    return IMHD_OK;
}

int imhd_server_poll(imhd_server* s, long long id, int* state, double* q, double* bface, double* qpass, double* info) {
    if (!s || !state) return sfail(IMHD_E_ARG, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->results.find(id);
    if (it == s->results.end()) return sfail(IMHD_E_ARG, "unknown request id (or its result was already taken)");
    Result& res = it->second;
    *state = res.state;
    if (info) {
        info[0] = res.t;
        info[1] = (double)res.steps;
        info[2] = res.t_done > 0 ? res.t_done - res.t_submit : -1.0;     // latency: submit -> result on the host
        info[3] = res.t_admit > 0 ? res.t_admit - res.t_submit : -1.0;   // queue wait
        info[4] = (double)res.status;
    }
    if (res.state == IMHD_REQ_FAILED) {
        std::string e = res.error;
        return sfail(IMHD_E_PHYSICS, "request " + std::to_string(id) + " failed: " + e);
    }
    if (res.state != IMHD_REQ_DONE || (!q && !bface && !qpass)) return IMHD_OK;
    // copy out (padded with periodic ghosts as the host asked) and release
    Result done = std::move(res);
    s->results.erase(it);
    lk.unlock();
    const imhd_config& c = done.cfg;
    const size_t n = (size_t)c.nx * c.ny * c.nz;
    auto put = [&](double* dst, int f, int ng) {
        const size_t Px = c.nx + 2 * ng, Py = c.ny + 2 * ng;
        for (int k = 0; k < c.nz; ++k)
            for (int j = 0; j < c.ny; ++j) {
                double* row = dst + (ng + Px * ((j + ng) + Py * (size_t)(k + ng)));
                const size_t src = (size_t)f * n + (size_t)c.nx * (j + (size_t)c.ny * k);
                if (done.esz == 8) {
                    std::memcpy(row, done.raw.data() + src * 8, (size_t)c.nx * 8);
                } else {
                    const float* s32 = (const float*)done.raw.data() + src;
                    for (int i = 0; i < c.nx; ++i) row[i] = (double)s32[i];
                }
            }
        imhd::host_ghost_fill(c.nx, c.ny, c.nz, dst, ng);
    };
    auto P = [&](int ng) { return (size_t)(c.nx + 2 * ng) * (c.ny + 2 * ng) * (c.nz + 2 * ng); };
    if (q)
        for (int f = 0; f < 7; ++f) put(q + (size_t)f * P(c.ng), f, c.ng);
    if (bface)
        for (int f = 0; f < 3; ++f) put(bface + (size_t)f * P(c.ng), 7 + f, c.ng);
    if (qpass)
        for (int f = 0; f < c.npass; ++f) put(qpass + (size_t)f * P(c.ng_pass), 10 + f, c.ng_pass);
    return IMHD_OK;
}

int imhd_server_stats(imhd_server* s, double* out, int n) {
    if (!s || !out || n < IMHD_SERVER_NSTATS) return sfail(IMHD_E_ARG, "need IMHD_SERVER_NSTATS doubles");
    std::lock_guard<std::mutex> lk(s->mu);
    double v[IMHD_SERVER_NSTATS] = {(double)s->queue.size(), (double)s->resident, (double)s->admitted,
                                    (double)s->completed, (double)s->failed, (double)s->replays,
                                    (double)s->launches, (double)s->rebuilds, (double)s->used_bytes,
                                    (double)s->peak_bytes, (double)s->peak_resident, s->t_build,
                                    s->t_rebuild, s->t_step, s->t_retire, s->t_harvest};
    for (int i = 0; i < IMHD_SERVER_NSTATS; ++i) out[i] = v[i];
    return IMHD_OK;
}

int imhd_server_stop(imhd_server* s, int drain) {
    if (!s) return sfail(IMHD_E_ARG, "null argument");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->drain = drain != 0;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->fatal.empty()) return sfail(IMHD_E_CUDA, "server worker stopped on: " + s->fatal);
    return IMHD_OK;
}

void imhd_server_destroy(imhd_server* s) {
    if (!s) return;
    imhd_server_stop(s, 0);
    delete s;
}

}  // extern "C"
