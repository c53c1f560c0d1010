// imhd_io.cu -- the reference's output and restart files written from (and
// read into) a device-resident box.
//
// * xyzcube stream dump (io_mod.f90:249-277): for every interior cell, k
//   slowest and i fastest, q(1..7) and the first passive scalar, REAL*8 or
//   SNGL (REAL*4) with no record markers.
// * state dump of the parallel writer (io_mod.f90:378-432) for one rank:
//   the same per-cell records with every passive scalar.
// * cuts (io_mod.f90:62-240): lines through the box centre along x, y, z,
//   the xy and yz diagonals and the xy mid-plane, each cell as rho, v, B (the
//   diagonal cuts in rotated components), stream files named like the
//   reference's.
// * restart (io_mod.f90:440-517): Fortran sequential unformatted records
//   t_sim | q_3d | bface_3d | qpass_3d (npass > 0) | dump_count | s1 | s2 | s3
//   of the padded arrays (ghost width nb, nb-2 for the passive scalars), with
//   gfortran's 4-byte record markers and its sub-record split of records
//   longer than 2^31-9 bytes.
//
// The interleaved cell records are packed on the device (one pass over the
// field-major state), so a dump moves its bytes across PCIe once.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/imhd.h"
#include "imhd_types.cuh"

namespace imhd {
const char* set_last_error(int code, const char* msg);
int box_download_padded(imhd_box* x, double* q, double* bface, double* qpass, int ng, int ng_pass);
int box_upload_padded(imhd_box* x, const double* q, const double* bface, const double* qpass, int ng, int ng_pass);
int box_state_view(imhd_box* x, const void** state, int* nx, int* ny, int* nz, int* npass, int* precision,
                   cudaStream_t* st);
}  // namespace imhd

namespace {

int iofail(int code, const std::string& m) {
    imhd::set_last_error(code, m.c_str());
    return code;
}

#define ICK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return iofail(IMHD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Cell records: out[c * nout + f] = state field f of cell c (f < 7), then
// passive scalars 10.. for f >= 7, converted to O.
template <class T, class O>
__global__ void k_pack_cells(const T* __restrict__ S, int n, int npass_out, O* __restrict__ out) {
    const int nout = 7 + npass_out;
    const long long total = (long long)n * nout;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int c = (int)(t / nout), f = (int)(t % nout);
        int src = f < 7 ? f : 10 + (f - 7);
        out[t] = (O)S[(size_t)src * n + c];
    }
}

// Cut cells: rho, v (m / rho in FP64), B_cc; diag 1 rotates (x, y) and 2
// rotates (y, z) into (perp, par) as the reference's diagonal cuts do.
template <class T>
__global__ void k_pack_cut(const T* __restrict__ S, int n, const int* __restrict__ cells, int ncell, int diag,
                           double* __restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncell) return;
    int c = cells[t];
    double rho = (double)S[c];
    double vx = (double)S[(size_t)n + c] / rho, vy = (double)S[2 * (size_t)n + c] / rho,
           vz = (double)S[3 * (size_t)n + c] / rho;
    double bx = (double)S[4 * (size_t)n + c], by = (double)S[5 * (size_t)n + c], bz = (double)S[6 * (size_t)n + c];
    double* o = out + (size_t)t * 7;
    const double isqr2 = 1.0 / sqrt(2.0);
    o[0] = rho;
    if (diag == 0) {
        o[1] = vx; o[2] = vy; o[3] = vz; o[4] = bx; o[5] = by; o[6] = bz;
    } else if (diag == 1) {     // io_mod.f90:152-161
        o[1] = isqr2 * (vy + vx); o[2] = isqr2 * (vy - vx); o[3] = vz;
        o[4] = isqr2 * (by + bx); o[5] = isqr2 * (by - bx); o[6] = bz;
    } else {                    // io_mod.f90:180-189 (writes vz and B_z as the reference does)
        o[1] = isqr2 * (vz + vy); o[2] = isqr2 * (vz - vy); o[3] = vz;
        o[4] = isqr2 * (bz + by); o[5] = isqr2 * (bz - by); o[6] = bz;
    }
}

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) { f = std::fopen(path, mode); }
    ~File() {
        if (f) std::fclose(f);
    }
    bool ok() const { return f != nullptr; }
    bool put(const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f) == n; }
    bool get(void* p, size_t n) { return n == 0 || std::fread(p, 1, n, f) == n; }
};

// gfortran sequential unformatted records: 4-byte length markers around each
// record; a record longer than kMaxSub bytes is written as sub-records whose
// head marker is negative when another sub-record follows and whose tail
// marker is negative when one precedes.
constexpr int64_t kMaxSub = 2147483639;

struct RecordWriter {
    File& file;
    int64_t total = 0, done = 0, sub_left = 0, sub_len = 0;
    bool first = true, good = true;
    explicit RecordWriter(File& f) : file(f) {}
    void head() {
        int64_t rest = total - done;
        sub_len = rest > kMaxSub ? kMaxSub : rest;
        sub_left = sub_len;
        int32_t m = (int32_t)((rest > kMaxSub) ? -sub_len : sub_len);
        good = good && file.put(&m, 4);
    }
    void tail() {
        int32_t m = (int32_t)(first ? sub_len : -sub_len);
        good = good && file.put(&m, 4);
        first = false;
    }
    void begin(int64_t len) {
        total = len;
        done = 0;
        first = true;
        head();
        if (total == 0) tail();
    }
    void write(const void* p, int64_t n) {
        const char* c = (const char*)p;
        while (n > 0 && good) {
            int64_t k = n < sub_left ? n : sub_left;
            good = good && file.put(c, (size_t)k);
            c += k;
            n -= k;
            sub_left -= k;
            done += k;
            if (sub_left == 0) {
                tail();
                if (done < total) head();
            }
        }
    }
};

// Read one (possibly split) record of exactly `len` bytes into dst in pieces.
struct RecordReader {
    File& file;
    int64_t sub_left = 0, got = 0;
    bool more = false, first = true, good = true;
    explicit RecordReader(File& f) : file(f) {}
    bool head() {
        int32_t m;
        if (!file.get(&m, 4)) return false;
        more = m < 0;
        sub_left = m < 0 ? -(int64_t)m : m;
        return true;
    }
    bool tail() {
        int32_t m;
        return file.get(&m, 4);
    }
    bool begin() {
        got = 0;
        return head();
    }
    bool read(void* p, int64_t n) {
        char* c = (char*)p;
        while (n > 0) {
            if (sub_left == 0) {
                if (!more) return false;       // record shorter than expected
                if (!tail() || !head()) return false;
            }
            int64_t k = n < sub_left ? n : sub_left;
            if (!file.get(c, (size_t)k)) return false;
            c += k;
            n -= k;
            sub_left -= k;
            got += k;
        }
        return true;
    }
    bool end() { return sub_left == 0 && !more && tail(); }
};

// Pack the cell records of the current state on the device and write them.
int write_cells(imhd_box* box, const char* path, int double_prec, bool all_pass) {
    const void* S;
    int nx, ny, nz, npass, prec;
    cudaStream_t st;
    int rc = imhd::box_state_view(box, &S, &nx, &ny, &nz, &npass, &prec, &st);
    if (rc) return rc;
    const int npo = all_pass ? npass : (npass > 0 ? 1 : 0);
    const int n = nx * ny * nz;
    const size_t osz = double_prec ? 8 : 4;
    const size_t bytes = (size_t)n * (7 + npo) * osz;
    void* d = nullptr;
    void* h = nullptr;
    ICK(cudaMallocAsync(&d, bytes, st));
    int blocks = (int)(((long long)n * (7 + npo) + 255) / 256);
    if (blocks > 65535 * 4) blocks = 65535 * 4;
    if (prec == 64) {
        if (double_prec) k_pack_cells<double, double><<<blocks, 256, 0, st>>>((const double*)S, n, npo, (double*)d);
        else k_pack_cells<double, float><<<blocks, 256, 0, st>>>((const double*)S, n, npo, (float*)d);
    } else {
        if (double_prec) k_pack_cells<float, double><<<blocks, 256, 0, st>>>((const float*)S, n, npo, (double*)d);
        else k_pack_cells<float, float><<<blocks, 256, 0, st>>>((const float*)S, n, npo, (float*)d);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMallocHost(&h, bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(d, st);
    if (e != cudaSuccess) {
        if (h) cudaFreeHost(h);
        return iofail(IMHD_E_CUDA, std::string("cell record packing: ") + cudaGetErrorString(e));
    }
    File f(path, "wb");
    bool ok = f.ok() && f.put(h, bytes);
    cudaFreeHost(h);
    if (!ok) return iofail(IMHD_E_ARG, std::string("cannot write ") + path);
    return IMHD_OK;
}

}  // namespace

extern "C" {

int imhd_write_xyzcube(imhd_box* box, const char* path, int double_prec) {
    if (!box || !path) return iofail(IMHD_E_ARG, "null argument");
    return write_cells(box, path, double_prec, false);
}

int imhd_write_state_dump(imhd_box* box, const char* path, int double_prec) {
    if (!box || !path) return iofail(IMHD_E_ARG, "null argument");
    return write_cells(box, path, double_prec, true);
}

int imhd_write_cuts(imhd_box* box, const char* dir, int dump, int flags, int riemann_prefix, int double_prec) {
    if (!box || !dir) return iofail(IMHD_E_ARG, "null argument");
    const void* S;
    int nx, ny, nz, npass, prec;
    cudaStream_t st;
    int rc = imhd::box_state_view(box, &S, &nx, &ny, &nz, &npass, &prec, &st);
    if (rc) return rc;
    // Fortran mid indices nx/2 (1-based) -> 0-based nx/2 - 1
    const int im = nx / 2 - 1, jm = ny / 2 - 1, km = nz / 2 - 1;
    auto C = [&](int i, int j, int k) { return i + nx * (j + ny * k); };
    const char* solver = riemann_prefix == IMHD_HLLD ? "HLLD" : riemann_prefix == IMHD_HLLE ? "HLLE" : "ROE";
    struct Cut { int flag; std::string name; std::vector<int> cells; int diag; };
    std::vector<Cut> cuts;
    std::string dn = std::to_string(dump);
    if (flags & IMHD_CUT_X) {
        Cut c{IMHD_CUT_X, std::string("xcut_") + solver + "_rank=000_dump=" + dn + ".dat", {}, 0};
        for (int i = 0; i < nx; ++i) c.cells.push_back(C(i, jm, km));
        cuts.push_back(c);
    }
    if (flags & IMHD_CUT_Y) {
        Cut c{IMHD_CUT_Y, "ycut_rank=000_dump=" + dn + ".dat", {}, 0};
        for (int j = 0; j < ny; ++j) c.cells.push_back(C(im, j, km));
        cuts.push_back(c);
    }
    if (flags & IMHD_CUT_Z) {
        Cut c{IMHD_CUT_Z, "zcut_rank=000_dump=" + dn + ".dat", {}, 0};
        for (int k = 0; k < nz; ++k) c.cells.push_back(C(im, jm, k));
        cuts.push_back(c);
    }
    if (flags & IMHD_CUT_XYDIAG) {
        Cut c{IMHD_CUT_XYDIAG, "xydiagcut_rank=000_dump=" + dn + ".dat", {}, 1};
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                if (i == j) c.cells.push_back(C(i, j, km));
        cuts.push_back(c);
    }
    if (flags & IMHD_CUT_YZDIAG) {
        Cut c{IMHD_CUT_YZDIAG, "yzdiagcut_rank=000_dump=" + dn + ".dat", {}, 2};
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                if (j == k) c.cells.push_back(C(im, j, k));
        cuts.push_back(c);
    }
    if (flags & IMHD_CUT_XYPLANE) {
        Cut c{IMHD_CUT_XYPLANE, "xyplane_rank=000_dump=" + dn + ".dat", {}, 0};
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) c.cells.push_back(C(i, j, km));
        cuts.push_back(c);
    }
    for (const Cut& c : cuts) {
        const int m = (int)c.cells.size();
        if (m == 0) continue;
        int* dc = nullptr;
        double* dout = nullptr;
        ICK(cudaMallocAsync((void**)&dc, (size_t)m * sizeof(int), st));
        ICK(cudaMallocAsync((void**)&dout, (size_t)m * 7 * sizeof(double), st));
        ICK(cudaMemcpyAsync(dc, c.cells.data(), (size_t)m * sizeof(int), cudaMemcpyHostToDevice, st));
        if (prec == 64) k_pack_cut<double><<<(m + 127) / 128, 128, 0, st>>>((const double*)S, nx * ny * nz, dc, m, c.diag, dout);
        else k_pack_cut<float><<<(m + 127) / 128, 128, 0, st>>>((const float*)S, nx * ny * nz, dc, m, c.diag, dout);
        ICK(cudaGetLastError());
        std::vector<double> h((size_t)m * 7);
        ICK(cudaMemcpyAsync(h.data(), dout, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        ICK(cudaStreamSynchronize(st));
        cudaFreeAsync(dc, st);
        cudaFreeAsync(dout, st);
        std::string path = std::string(dir) + "/" + c.name;
        File f(path.c_str(), "wb");
        bool ok = f.ok();
        if (double_prec) {
            ok = ok && f.put(h.data(), h.size() * sizeof(double));
        } else {
            std::vector<float> s(h.size());
            for (size_t t = 0; t < h.size(); ++t) s[t] = (float)h[t];   // SNGL
            ok = ok && f.put(s.data(), s.size() * sizeof(float));
        }
        if (!ok) return iofail(IMHD_E_ARG, "cannot write " + path);
    }
    return IMHD_OK;
}

int imhd_write_restart(imhd_box* box, const char* path, double t_sim, int nb, int dump_count, int s1, int s2, int s3) {
    if (!box || !path) return iofail(IMHD_E_ARG, "null argument");
    if (nb < 2) return iofail(IMHD_E_ARG, "nb must be >= 2 (passive scalars use nb - 2)");
    const void* S;
    int nx, ny, nz, npass, prec;
    cudaStream_t st;
    int rc = imhd::box_state_view(box, &S, &nx, &ny, &nz, &npass, &prec, &st);
    if (rc) return rc;
    const int nbp = nb - 2;
    const size_t P = (size_t)(nx + 2 * nb) * (ny + 2 * nb) * (nz + 2 * nb);
    const size_t Pp = (size_t)(nx + 2 * nbp) * (ny + 2 * nbp) * (nz + 2 * nbp);
    std::vector<double> q(7 * P), b(3 * P), p(npass > 0 ? (size_t)npass * Pp : 0);
    if ((rc = imhd::box_download_padded(box, q.data(), b.data(), npass ? p.data() : nullptr, nb, nbp))) return rc;
    File f(path, "wb");
    if (!f.ok()) return iofail(IMHD_E_ARG, std::string("cannot open ") + path);
    RecordWriter w(f);
    w.begin(8); w.write(&t_sim, 8);
    w.begin((int64_t)(q.size() * 8)); w.write(q.data(), (int64_t)(q.size() * 8));
    w.begin((int64_t)(b.size() * 8)); w.write(b.data(), (int64_t)(b.size() * 8));
    if (npass > 0) { w.begin((int64_t)(p.size() * 8)); w.write(p.data(), (int64_t)(p.size() * 8)); }
    w.begin(4); w.write(&dump_count, 4);
    w.begin(4); w.write(&s1, 4);
    w.begin(4); w.write(&s2, 4);
    w.begin(4); w.write(&s3, 4);
    if (!w.good) return iofail(IMHD_E_ARG, std::string("cannot write ") + path);
    return IMHD_OK;
}

int imhd_read_restart(imhd_box* box, const char* path, int nb, double* t_sim, int* dump_count, int* s1, int* s2,
                      int* s3) {
    if (!box || !path) return iofail(IMHD_E_ARG, "null argument");
    if (nb < 2) return iofail(IMHD_E_ARG, "nb must be >= 2 (passive scalars use nb - 2)");
    const void* S;
    int nx, ny, nz, npass, prec;
    cudaStream_t st;
    int rc = imhd::box_state_view(box, &S, &nx, &ny, &nz, &npass, &prec, &st);
    if (rc) return rc;
    const int nbp = nb - 2;
    const size_t P = (size_t)(nx + 2 * nb) * (ny + 2 * nb) * (nz + 2 * nb);
    const size_t Pp = (size_t)(nx + 2 * nbp) * (ny + 2 * nbp) * (nz + 2 * nbp);
    std::vector<double> q(7 * P), b(3 * P), p(npass > 0 ? (size_t)npass * Pp : 0);
    File f(path, "rb");
    if (!f.ok()) return iofail(IMHD_E_ARG, std::string("cannot open ") + path);
    RecordReader r(f);
    double t = 0;
    int dc = 0, a1 = 0, a2 = 0, a3 = 0;
    bool ok = r.begin() && r.read(&t, 8) && r.end();
    ok = ok && r.begin() && r.read(q.data(), (int64_t)(q.size() * 8)) && r.end();
    ok = ok && r.begin() && r.read(b.data(), (int64_t)(b.size() * 8)) && r.end();
    if (npass > 0) ok = ok && r.begin() && r.read(p.data(), (int64_t)(p.size() * 8)) && r.end();
    ok = ok && r.begin() && r.read(&dc, 4) && r.end();
    ok = ok && r.begin() && r.read(&a1, 4) && r.end();
    ok = ok && r.begin() && r.read(&a2, 4) && r.end();
    ok = ok && r.begin() && r.read(&a3, 4) && r.end();
    if (!ok) return iofail(IMHD_E_ARG, std::string(path) + " is not a restart file of this box (record sizes differ)");
    if ((rc = imhd::box_upload_padded(box, q.data(), b.data(), npass ? p.data() : nullptr, nb, nbp))) return rc;
    if (t_sim) *t_sim = t;
    if (dump_count) *dump_count = dc;
    if (s1) *s1 = a1;
    if (s2) *s2 = a2;
    if (s3) *s3 = a3;
    return IMHD_OK;
}

}  // extern "C"
