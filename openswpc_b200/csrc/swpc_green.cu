// swpc_green.cu -- green__store (src/swpc_3d/m_green.f90:389-534): the
// reciprocity Green's functions at a list of grid points.
//
// In green mode the reference integrates, at every point of its green table,
// the nine velocity derivatives (4th-order differences, the off-diagonal
// ones averaged over the four staggered neighbours) into displacement
// derivatives, optionally the displacements themselves, and samples them
// every ntdec_w steps into gf(ntw, ncmp*ng).  The reference's main loop
// (main.f90:125-144) never calls it; here the per-step call sits beside
// wav__store at the start of the step (swpc_step and the captured graph
// include it once swpc_green_store_setup has run).  Every operation is
// rounded in the reference's order with explicit intrinsics (no
// contraction), in single precision as the MP = SP build.
#include <cuda_runtime.h>

#include <vector>

#include "swpc_ctx.h"

using namespace swpc;

#define CK(call)                                               \
    do {                                                       \
        int _rc = cuda_check(c, (call), #call);                \
        if (_rc) return _rc;                                   \
    } while (0)

namespace {

struct GreenArgs {
    Geo g;
    const float *Vx, *Vy, *Vz;
    const int *ijk;
    float *acc, *out;
    int ng, ncmp, ntw, ntdec, it;
    const int *d_it;
    float r40[3], r41[3], dt;
    long long vstride;   // field offset of member blockIdx.y (reciprocity batch; 0 for a context)
};

// (f(+0) - f(-1)) * r40 - (f(+1) - f(-2)) * r41 along stride P from e
__device__ __forceinline__ float dbwd(const float *f, long long e, long long P, float r40, float r41) {
    return __fsub_rn(__fmul_rn(__fsub_rn(f[e], f[e - P]), r40), __fmul_rn(__fsub_rn(f[e + P], f[e - 2 * P]), r41));
}
// (f(+1) - f(0)) * r40 - (f(+2) - f(-1)) * r41
__device__ __forceinline__ float dfwd(const float *f, long long e, long long P, float r40, float r41) {
    return __fsub_rn(__fmul_rn(__fsub_rn(f[e + P], f[e]), r40), __fmul_rn(__fsub_rn(f[e + 2 * P], f[e - P]), r41));
}
// (a + b + c + d) * 0.25
__device__ __forceinline__ float avg4(float a, float b, float c, float d) {
    return __fmul_rn(__fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d), 0.25f);
}

__global__ void green_store_kernel(const GreenArgs a) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.ng) return;
    const int it = a.d_it ? *a.d_it : a.it;
    const Geo &g = a.g;
    const long long PK = 1, PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    const long long e = cell_index(g, a.ijk[3 * n + 2], a.ijk[3 * n], a.ijk[3 * n + 1]);
    const long long mo = (long long)blockIdx.y * a.vstride;
    const float *Vx = a.Vx + mo, *Vy = a.Vy + mo, *Vz = a.Vz + mo;
    float *const acc = a.acc + (long long)blockIdx.y * 12 * a.ng;
    const float rx0 = a.r40[0], rx1 = a.r41[0], ry0 = a.r40[1], ry1 = a.r41[1], rz0 = a.r40[2], rz1 = a.r41[2];
    // m_green.f90:449-487
    const float dxVx = dbwd(Vx, e, PI, rx0, rx1);
    const float dyVy = dbwd(Vy, e, PJ, ry0, ry1);
    const float dzVz = dbwd(Vz, e, PK, rz0, rz1);
    const float dxVy = avg4(dfwd(Vy, e, PI, rx0, rx1), dfwd(Vy, e - PJ, PI, rx0, rx1), dbwd(Vy, e, PI, rx0, rx1),
                            dbwd(Vy, e - PJ, PI, rx0, rx1));
    const float dxVz = avg4(dfwd(Vz, e, PI, rx0, rx1), dfwd(Vz, e - PK, PI, rx0, rx1), dbwd(Vz, e, PI, rx0, rx1),
                            dbwd(Vz, e - PK, PI, rx0, rx1));
    const float dyVx = avg4(dfwd(Vx, e, PJ, ry0, ry1), dfwd(Vx, e - PI, PJ, ry0, ry1), dbwd(Vx, e, PJ, ry0, ry1),
                            dbwd(Vx, e - PI, PJ, ry0, ry1));
    const float dyVz = avg4(dfwd(Vz, e, PJ, ry0, ry1), dfwd(Vz, e - PK, PJ, ry0, ry1), dbwd(Vz, e, PJ, ry0, ry1),
                            dbwd(Vz, e - PK, PJ, ry0, ry1));
    const float dzVx = avg4(dfwd(Vx, e, PK, rz0, rz1), dfwd(Vx, e - PI, PK, rz0, rz1), dbwd(Vx, e, PK, rz0, rz1),
                            dbwd(Vx, e - PI, PK, rz0, rz1));
    const float dzVy = avg4(dfwd(Vy, e, PK, rz0, rz1), dfwd(Vy, e - PJ, PK, rz0, rz1), dbwd(Vy, e, PK, rz0, rz1),
                            dbwd(Vy, e - PJ, PK, rz0, rz1));
    const float d[9] = {dxVx, dxVy, dxVz, dyVx, dyVy, dyVz, dzVx, dzVy, dzVz};
    float u[12];
    const int ng = a.ng;
    // the totals start from zero at it == 1, where the reference allocates
    // them (m_green.f90:409-425): a rerun from step 1 of a context or a
    // batch does not carry the previous run's totals
    const bool first = it == 1;
#pragma unroll
    for (int q = 0; q < 9; q++) {
        u[q] = __fadd_rn(first ? 0.0f : acc[q * ng + n], __fmul_rn(d[q], a.dt));
        acc[q * ng + n] = u[q];
    }
    if (a.ncmp == 9) {
        // m_green.f90:499-503
        const float v3[3] = {__fadd_rn(Vx[e], Vx[e - PI]), __fadd_rn(Vy[e], Vy[e - PJ]), __fadd_rn(Vz[e], Vz[e - PK])};
#pragma unroll
        for (int q = 0; q < 3; q++) {
            u[9 + q] = __fadd_rn(first ? 0.0f : acc[(9 + q) * ng + n], __fmul_rn(__fmul_rn(0.5f, v3[q]), a.dt));
            acc[(9 + q) * ng + n] = u[9 + q];
        }
    }
    if ((it - 1) % a.ntdec != 0) return;
    const int itw = (it - 1) / a.ntdec + 1;
    if (itw < 1 || itw > a.ntw) return;
    // m_green.f90:506-526; column (n-1)*ncmp + j of gf(ntw, ncmp*ng)
    const float uc = 1e-15f, ub = 1e-12f;
    const float g6[6] = {u[0], u[4], u[8], __fadd_rn(u[5], u[7]), __fadd_rn(u[2], u[6]), __fadd_rn(u[1], u[3])};
    float *o = a.out + ((long long)blockIdx.y * a.ng + n) * a.ncmp * a.ntw + (itw - 1);
#pragma unroll
    for (int j = 0; j < 6; j++) o[(long long)j * a.ntw] = __fmul_rn(__fmul_rn(g6[j], uc), 1e9f);
    if (a.ncmp == 9)
        for (int j = 0; j < 3; j++) o[(long long)(6 + j) * a.ntw] = __fmul_rn(__fmul_rn(u[9 + j], ub), 1e9f);
}

}  // namespace

namespace swpc {

int green_store_members(swpc_ctx *c, float *const *V, long long vstride, int nmem, float *acc, float *out, int it,
                        const int *d_it) {
    if (c->ng <= 0) return SWPC_OK;
    GreenArgs a;
    a.g = c->g;
    a.Vx = V[0]; a.Vy = V[1]; a.Vz = V[2];
    a.ijk = c->g_ijk; a.acc = acc; a.out = out;
    a.ng = c->ng; a.ncmp = c->ng_cmp; a.ntw = c->ng_ntw; a.ntdec = c->ng_ntdec; a.it = it; a.d_it = d_it;
    for (int q = 0; q < 3; q++) { a.r40[q] = c->r40[q]; a.r41[q] = c->r41[q]; }
    a.dt = c->d.dt;
    a.vstride = vstride;
    green_store_kernel<<<dim3((c->ng + 127) / 128, nmem), 128, 0, c->stream>>>(a);
    return cuda_check(c, cudaGetLastError(), "green_store launch");
}

int green_store_launch(swpc_ctx *c, int it, const int *d_it) {
    return green_store_members(c, c->V, 0, 1, c->g_acc, c->g_out, it, d_it);
}

void green_free(swpc_ctx *c) {
    if (c->g_ijk) cudaFree(c->g_ijk);
    if (c->g_acc) cudaFree(c->g_acc);
    if (c->g_out) cudaFree(c->g_out);
    c->g_ijk = nullptr; c->g_acc = nullptr; c->g_out = nullptr;
    c->bytes -= c->g_bytes;
    c->g_bytes = 0;
    c->ng = 0;
}

}  // namespace swpc

extern "C" int swpc_green_store_setup(swpc_ctx *c, int ng, const int *ig, const int *jg, const int *kg, int bforce,
                                      int ntdec_w) {
    if (!c) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "green__store is a 3D routine");
    if (c->prec != SWPC_PREC_F32) return set_err(c, SWPC_ERR_ARG, "green__store reads FP32 velocities");
    if (ng < 0 || ntdec_w < 1 || (ng > 0 && (!ig || !jg || !kg))) return set_err(c, SWPC_ERR_ARG, "bad green table");
    const Geo &g = c->g;
    std::vector<int> ijk(3 * (size_t)std::max(ng, 1));
    for (int n = 0; n < ng; n++) {
        // the stencil reaches two cells below and above in every direction
        if (ig[n] < 1 || ig[n] > g.nx || jg[n] < 1 || jg[n] > g.ny || kg[n] < 1 || kg[n] > g.nz)
            return set_err(c, SWPC_ERR_ARG, "green point outside the grid");
        ijk[3 * n] = ig[n]; ijk[3 * n + 1] = jg[n]; ijk[3 * n + 2] = kg[n];
    }
    CK(cudaSetDevice(c->device));
    c->desc_dirty = true;
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
    green_free(c);
    if (ng == 0) return SWPC_OK;
    const int ncmp = bforce ? 9 : 6;
    const int ntw = (c->d.nt - 1) / ntdec_w + 1;   // m_green.f90 ntw as m_wav.f90
    const long long before = c->bytes;
    int rc = dalloc(c, &c->g_ijk, 3 * (size_t)ng);
    if (!rc) rc = dalloc(c, &c->g_acc, 12 * (size_t)ng);
    if (!rc) rc = dalloc(c, &c->g_out, (size_t)ntw * ncmp * ng);
    c->g_bytes = c->bytes - before;
    if (!rc) rc = cuda_check(c, cudaMemcpyAsync(c->g_ijk, ijk.data(), 3 * (size_t)ng * sizeof(int),
                                                cudaMemcpyHostToDevice, c->stream), "cudaMemcpyAsync");
    if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    if (rc) {
        green_free(c);
        return rc;
    }
    c->ng = ng; c->ng_cmp = ncmp; c->ng_ntw = ntw; c->ng_ntdec = ntdec_w;
    return SWPC_OK;
}

extern "C" int swpc_green_store(swpc_ctx *c, int it) {
    if (!c) return SWPC_ERR_ARG;
    CK(cudaSetDevice(c->device));
    return green_store_launch(c, it, nullptr);
}

extern "C" int swpc_green_fetch(swpc_ctx *c, float *out) {
    if (!c || !out) return SWPC_ERR_ARG;
    if (c->ng <= 0) return set_err(c, SWPC_ERR_STATE, "swpc_green_store_setup not called");
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)c->ng_ntw * c->ng_cmp * c->ng;
    CK(cudaMemcpyAsync(out, c->g_out, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}
