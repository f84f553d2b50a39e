// swpc_pw.cu -- the side boundary of the plane-wave mode (pw_mode).
//
// In plane-wave mode the ADE-CFS PML keeps its vertical damping but the four
// side faces become zero-derivative boundaries: before the absorber updates
// the ghost plane next to each face is extrapolated linearly from the two
// cells inside, f(0) = 2 f(1) - f(2) and f(n+1) = 2 f(n) - f(n-1), for V
// before the stress update and for S before the velocity update
// (src/swpc_3d/m_absorb_p.f90:136-243, 324-431), over k = 1..nz and the other
// index 1..n.  On a single domain global__comm_vel / global__comm_stress then
// zero their ghost planes (m_global.f90:393-609): the library's kernels never
// write ghosts, so those planes only need clearing in this mode, whose
// initial condition (pw_setup) fills the whole memory box.
#include <cuda_runtime.h>

#include "swpc_ctx.h"

using namespace swpc;

namespace {

constexpr int kThreads = 256;

struct PwFields {
    float *f[6];
    int nf;
};

// one thread per (line, k) of the four ghost lines: t < ny: i = 0 face, then i = nx+1, then j = 0, then j = ny+1
__global__ void pw_fill_kernel(Geo g, PwFields a) {
    const long long nl = 2LL * g.ny + 2LL * g.nx;
    const long long n = nl * g.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(q % g.nz);
        long long t = q / g.nz;
        int gi, gj, i1, j1, i2, j2;   // ghost cell, first and second cell inside
        if (t < g.ny) {
            gj = j1 = j2 = 1 + (int)t; gi = 0; i1 = 1; i2 = 2;
        } else if ((t -= g.ny) < g.ny) {
            gj = j1 = j2 = 1 + (int)t; gi = g.nx + 1; i1 = g.nx; i2 = g.nx - 1;
        } else if ((t -= g.ny) < g.nx) {
            gi = i1 = i2 = 1 + (int)t; gj = 0; j1 = 1; j2 = 2;
        } else {
            t -= g.nx;
            gi = i1 = i2 = 1 + (int)t; gj = g.ny + 1; j1 = g.ny; j2 = g.ny - 1;
        }
        const long long eg = cell_index(g, k, gi, gj), e1 = cell_index(g, k, i1, j1), e2 = cell_index(g, k, i2, j2);
        for (int c = 0; c < a.nf; c++) a.f[c][eg] = 2 * a.f[c][e1] - a.f[c][e2];
    }
}

// the ghost planes one comm routine zeroes: field, plane index, axis (0: i plane over j = 1..ny, 1: j plane over
// i = 1..nx), k = 1..nz
struct Plane {
    int field, at, axis;
};
struct PwZero {
    float *f[6];
    Plane p[18];
    int np;
};

__global__ void pw_zero_kernel(Geo g, PwZero a) {
    const int span = g.nx > g.ny ? g.nx : g.ny;
    const long long n = (long long)a.np * span * g.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(q % g.nz);
        const int r = 1 + (int)((q / g.nz) % span);
        const Plane pl = a.p[q / ((long long)g.nz * span)];
        if (r > (pl.axis == 0 ? g.ny : g.nx)) continue;
        const long long e = pl.axis == 0 ? cell_index(g, k, pl.at, r) : cell_index(g, k, r, pl.at);
        a.f[pl.field][e] = 0.0f;
    }
}

int grid_for(long long n) {
    const long long b = (n + kThreads - 1) / kThreads;
    return (int)(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);
}

}  // namespace

namespace swpc {

int pw_fill(swpc_ctx *c, int which) {
    if (!c->pw_mode) return SWPC_OK;
    PwFields a;
    a.nf = which == 0 ? 3 : 6;
    for (int q = 0; q < a.nf; q++) a.f[q] = which == 0 ? c->V[q] : c->S[q];
    const long long n = (2LL * c->g.ny + 2LL * c->g.nx) * c->g.nz;
    pw_fill_kernel<<<grid_for(n), kThreads, 0, c->stream>>>(c->g, a);
    return cuda_check(c, cudaGetLastError(), "pw_fill_kernel");
}

int pw_comm_zero(swpc_ctx *c, int which) {
    if (!c->pw_mode) return SWPC_OK;
    const int nx = c->g.nx, ny = c->g.ny;
    PwZero a;
    if (which == 0) {
        // global__comm_vel's unpack (m_global.f90:462-492); fields 0 Vx 1 Vy 2 Vz
        for (int q = 0; q < 3; q++) a.f[q] = c->V[q];
        const Plane p[18] = {{0, -1, 0}, {0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {0, nx + 1, 0}, {1, nx + 1, 0},
                             {1, nx + 2, 0}, {2, nx + 1, 0}, {2, nx + 2, 0},
                             {0, 0, 1}, {1, -1, 1}, {1, 0, 1}, {2, 0, 1}, {0, ny + 1, 1}, {0, ny + 2, 1},
                             {1, ny + 1, 1}, {2, ny + 1, 1}, {2, ny + 2, 1}};
        for (int q = 0; q < 18; q++) a.p[q] = p[q];
    } else {
        // global__comm_stress's unpack (m_global.f90:574-604); fields 0 Sxx 1 Syy 2 Szz 3 Syz 4 Sxz 5 Sxy
        for (int q = 0; q < 6; q++) a.f[q] = c->S[q];
        const Plane p[18] = {{0, 0, 0}, {5, -1, 0}, {5, 0, 0}, {4, -1, 0}, {4, 0, 0}, {0, nx + 1, 0},
                             {0, nx + 2, 0}, {5, nx + 1, 0}, {4, nx + 1, 0},
                             {1, 0, 1}, {5, -1, 1}, {5, 0, 1}, {3, -1, 1}, {3, 0, 1}, {1, ny + 1, 1},
                             {1, ny + 2, 1}, {5, ny + 1, 1}, {3, ny + 1, 1}};
        for (int q = 0; q < 18; q++) a.p[q] = p[q];
    }
    a.np = 18;
    const long long n = 18LL * (nx > ny ? nx : ny) * c->g.nz;
    pw_zero_kernel<<<grid_for(n), kThreads, 0, c->stream>>>(c->g, a);
    return cuda_check(c, cudaGetLastError(), "pw_zero_kernel");
}

}  // namespace swpc

extern "C" int swpc_set_pw_mode(swpc_ctx *c, int on) {
    if (!c) return SWPC_ERR_ARG;
    if (on && c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "the plane-wave mode is a 3D mode");
    if (on && c->prec != SWPC_PREC_F32) return set_err(c, SWPC_ERR_ARG, "the plane-wave mode needs FP32 storage");
    if (on && c->abc != 0) return set_err(c, SWPC_ERR_ARG, "the plane-wave boundary belongs to the PML (abc_type 'pml')");
    if (on && (c->g.nx < 2 || c->g.ny < 2)) return set_err(c, SWPC_ERR_ARG, "the plane-wave mode needs nx, ny >= 2");
    if (on && c->sub) return set_err(c, SWPC_ERR_ARG, "the plane-wave mode runs on a single domain");
    c->pw_mode = on ? 1 : 0;
    c->desc_dirty = true;
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
    return SWPC_OK;
}
