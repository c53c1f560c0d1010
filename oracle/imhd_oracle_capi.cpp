// imhd_oracle_capi.cpp -- ctypes entry points of the FP64 oracle.
//
// TEST INFRASTRUCTURE ONLY (see imhd_oracle.hpp): loaded by tests/, by
// __graft_entry__.smoke() as the checker, and by bench.py's CPU baseline and
// reference legs.  The product library never links it.
//
// Host arrays exchanged here are unpadded, x fastest: field f of cell (i,j,k)
// (0-based) sits at f*nx*ny*nz + i + nx*(j + ny*k).  q has 7 fields
// (rho, mx, my, mz, Bx_cc, By_cc, Bz_cc), bface 3 (Bx at i+1/2, By at j+1/2,
// Bz at k+1/2), qpass npass.
#include "imhd_oracle.hpp"

using imhd_oracle::Config;
using imhd_oracle::Solver;

extern "C" {

// recon: bit 0 PPM (else PLM), bit 1 primitive-variable (else characteristic)
// reconstruction; bit 2 the HLLE protection fluxes of a Roe run.
void* oracle_create(int nx, int ny, int nz, int riemann, int recon, int npass, double sound_speed, int nthreads) {
    Config c;
    c.nx = nx; c.ny = ny; c.nz = nz;
    c.riemann = riemann; c.ppm = recon & 1; c.prim = (recon >> 1) & 1; c.protect = (recon >> 2) & 1;
    c.npass = npass;
    c.sound_speed = sound_speed; c.nthreads = nthreads;
    c.nb = 6;
    if (nx < 2 * c.nb || ny < 2 * c.nb || nz < 2 * c.nb) return nullptr;
    return new Solver(c);
}

void oracle_destroy(void* h) { delete static_cast<Solver*>(h); }

void oracle_set_threads(void* h, int n) { static_cast<Solver*>(h)->nthreads = n < 1 ? 1 : n; }

void oracle_set_force_params(void* h, double edot, double dt_turb) {
    auto* s = static_cast<Solver*>(h);
    s->cfg.edot = edot; s->cfg.dt_turb = dt_turb;
}

void oracle_set_state(void* h, const double* q, const double* bface, const double* qpass) {
    auto* s = static_cast<Solver*>(h);
    long n = (long)s->nx * s->ny * s->nz;
    for (long k = 0; k < s->nz; ++k)
        for (long j = 0; j < s->ny; ++j)
            for (long i = 0; i < s->nx; ++i) {
                long c = i + s->nx * (j + s->ny * k);
                for (int v = 1; v <= 7; ++v) s->q(i + 1, j + 1, k + 1, v) = q[(v - 1) * n + c];
                for (int v = 1; v <= 3; ++v) s->bface(i + 1, j + 1, k + 1, v) = bface[(v - 1) * n + c];
                for (int v = 1; v <= s->cfg.npass; ++v) s->qpass(i + 1, j + 1, k + 1, v) = qpass[(v - 1) * n + c];
            }
    s->boundary_conditions();
}

void oracle_get_state(void* h, double* q, double* bface, double* qpass) {
    auto* s = static_cast<Solver*>(h);
    long n = (long)s->nx * s->ny * s->nz;
    for (long k = 0; k < s->nz; ++k)
        for (long j = 0; j < s->ny; ++j)
            for (long i = 0; i < s->nx; ++i) {
                long c = i + s->nx * (j + s->ny * k);
                if (q) for (int v = 1; v <= 7; ++v) q[(v - 1) * n + c] = s->q(i + 1, j + 1, k + 1, v);
                if (bface) for (int v = 1; v <= 3; ++v) bface[(v - 1) * n + c] = s->bface(i + 1, j + 1, k + 1, v);
                if (qpass) for (int v = 1; v <= s->cfg.npass; ++v) qpass[(v - 1) * n + c] = s->qpass(i + 1, j + 1, k + 1, v);
            }
}

// Interior force field delv(i,j,k,1:3), same unpadded layout as q.
void oracle_set_force(void* h, const double* delv) {
    auto* s = static_cast<Solver*>(h);
    long n = (long)s->nx * s->ny * s->nz;
    for (long k = 0; k < s->nz; ++k)
        for (long j = 0; j < s->ny; ++j)
            for (long i = 0; i < s->nx; ++i) {
                long c = i + s->nx * (j + s->ny * k);
                for (int v = 1; v <= 3; ++v) s->delv(i + 1, j + 1, k + 1, v) = delv[(v - 1) * n + c];
            }
    s->have_force = true;
}

void oracle_get_force(void* h, double* delv) {
    auto* s = static_cast<Solver*>(h);
    long n = (long)s->nx * s->ny * s->nz;
    for (long k = 0; k < s->nz; ++k)
        for (long j = 0; j < s->ny; ++j)
            for (long i = 0; i < s->nx; ++i) {
                long c = i + s->nx * (j + s->ny * k);
                for (int v = 1; v <= 3; ++v) delv[(v - 1) * n + c] = s->delv(i + 1, j + 1, k + 1, v);
            }
}

void oracle_init_turb(void* h, int s1, int s2, int s3) { static_cast<Solver*>(h)->init_turb_driver(s1, s2, s3); }
void oracle_generate_force(void* h) { static_cast<Solver*>(h)->generate_rand_force(); }

// One step of the reference driver loop for one rank.  Returns cmax of
// get_max_speed_vanleer; the caller forms dt = COUR*dx/cmax.
double oracle_step(void* h, double dt, int drive) { return static_cast<Solver*>(h)->step(dt, drive != 0); }

double oracle_smax(void* h) { return static_cast<Solver*>(h)->smax; }
double oracle_delv_max(void* h) { return static_cast<Solver*>(h)->delv_max; }
double oracle_dx(void* h) { return static_cast<Solver*>(h)->dx; }
long oracle_floor_hits(void* h) { return static_cast<Solver*>(h)->floor_hits; }
long oracle_prot_cells(void* h) { return static_cast<Solver*>(h)->prot_cells; }
int oracle_force_error(void* h) { return static_cast<Solver*>(h)->force_error; }

// out = {KE, vrms, momx, momy, momz, divB} (driver.f90:492-553)
void oracle_diagnostics(void* h, double* out) {
    auto* s = static_cast<Solver*>(h);
    s->compute_KE(out);
    out[5] = s->compute_divB();
}

// Max speed of the current state alone (no smax), for dt of the initial state.
double oracle_max_speed(void* h) {
    auto* s = static_cast<Solver*>(h);
    double sm = s->smax, dm = s->delv_max;
    s->smax = 0.0; s->delv_max = 0.0;
    double r = s->get_max_speed_vanleer();
    s->smax = sm; s->delv_max = dm;
    return r;
}

}  // extern "C"
