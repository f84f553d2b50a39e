// swpc_snap.cu -- snapshot planes of the 3D solver: snap__setup and
// snap__write (src/swpc_3d/m_snap.f90:95-322, 911-2185) for one domain.
//
// The reference computes each enabled plane into a buffer and writes it to a
// native or NetCDF file (after an MPI reduce).  Here every enabled plane
// keeps its frames in HBM for the whole run -- frame f is the plane at
// it = 1 + f*ntdec_s -- and the driver fetches them (swpc_snap_fetch) to
// write whatever format it wants.  One launch per step updates all planes:
// blockIdx.y picks the plane, one thread per decimated sample.  The
// displacement planes accumulate every step and the free-surface /
// ocean-bottom velocity and displacement planes update their running maxima
// every step, as wbuf_*_u and wbuf_fs_v / wbuf_ob_v do.
//
// Arithmetic keeps the reference's expression order (the file is compiled
// with -fmad=false), so the frames are bitwise those of the FP32 oracle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "swpc_ctx.h"

namespace swpc {
int graph_invalidate(swpc_ctx *c);
}

using namespace swpc;

namespace {

constexpr int kPlanes = 15;

struct SnapPlane {
    int plane;             // 3 * section + quantity
    int n1, n2, nv;        // buffer (n1, n2, nv) in Fortran order
    int a0, a1, b0, b1;    // sample ranges of the node (is0:is1 / js0:js1 / ks0:ks1)
    float *frames;         // (nframes, nv, n2, n1)
    float *ubuf;           // displacement accumulator (3, n2, n1), u planes only
    float *maxv;           // running maxima (3, n2, n1), fs/ob v and u planes only
};

struct SnapArgs {
    Geo g;
    const float *Vx, *Vy, *Vz, *lam, *muyz, *muxz, *muxy;
    const int *kfs, *kob;  // per column
    float r20x, r20y, r20z, UC, M0, dt;
    int idec, jdec, kdec, ntdec_s, nt, i0_yz, j0_xz, k0_xy;
    const int *d_it;
    int it;
    SnapPlane p[kPlanes];
};

__device__ __forceinline__ float fmax_ref(float a, float b) { return a > b ? a : b; }

__global__ void __launch_bounds__(256) snap3d_kernel(const SnapArgs a) {
    const int it = a.d_it ? *a.d_it : a.it;
    const SnapPlane &P = a.p[blockIdx.y];
    const int sec = P.plane / 3, q = P.plane % 3;
    const bool snap_step = ((it - 1) % a.ntdec_s == 0) || (it > a.nt);
    // ps planes and the cross-section v planes work only at snapshot steps;
    // u planes and the fs/ob v planes (running maxima) work every step
    if (q == 0 && !snap_step) return;
    if (q == 1 && !snap_step && sec < 3) return;
    const bool store = snap_step && it <= a.nt;
    const Geo g = a.g;
    const int na = P.a1 - P.a0 + 1, nb = P.b1 - P.b0 + 1;
    const long long npts = (long long)na * nb;
    const long long ns = (long long)P.n1 * P.n2;
    const long long PI = g.Kp, PJ = (long long)g.Kp * g.Ip;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < npts;
         t += (long long)gridDim.x * blockDim.x) {
        const int sa = P.a0 + (int)(t % na), sb = P.b0 + (int)(t / na);
        int i, j, k;
        if (sec == 0) {
            i = a.i0_yz; j = sa * a.jdec - a.jdec / 2; k = sb * a.kdec - a.kdec / 2;
        } else if (sec == 1) {
            i = sa * a.idec - a.idec / 2; j = a.j0_xz; k = sb * a.kdec - a.kdec / 2;
        } else {
            i = sa * a.idec - a.idec / 2; j = sb * a.jdec - a.jdec / 2;
            if (sec == 2) k = a.k0_xy;
            else k = (sec == 3 ? a.kfs : a.kob)[col_index(g, i, j)] + 1;
        }
        const long long e = cell_index(g, k, i, j);
        const long long o = (long long)(sb - 1) * P.n1 + (sa - 1);
        float v[4];
        if (q == 0) {
            // wbuf_*_ps (m_snap.f90:1004-1027)
            const float *Vx = a.Vx, *Vy = a.Vy, *Vz = a.Vz;
            float div = (Vx[e] - Vx[e - PI]) * a.r20x + (Vy[e] - Vy[e - PJ]) * a.r20y + (Vz[e] - Vz[e - 1]) * a.r20z;
            float rot_x = (Vz[e + PJ] - Vz[e]) * a.r20y - (Vy[e + 1] - Vy[e]) * a.r20z;
            float rot_y = (Vx[e + 1] - Vx[e]) * a.r20z - (Vz[e + PI] - Vz[e]) * a.r20x;
            float rot_z = (Vy[e + PI] - Vy[e]) * a.r20x - (Vx[e + PJ] - Vx[e]) * a.r20y;
            const float eps = 1.1920929e-07f;   // epsilon(1.0)
            const float lam = a.lam[e], muyz = a.muyz[e], muxz = a.muxz[e], muxy = a.muxy[e];
            div = div * lam / fabsf(lam + eps);
            rot_x = rot_x * muyz / fabsf(muyz + eps);
            rot_y = rot_y * muxz / fabsf(muxz + eps);
            rot_z = rot_z * muxy / fabsf(muxy + eps);
            v[0] = div * a.UC * a.M0 * 1e-3f;
            v[1] = rot_x * a.UC * a.M0 * 1e-3f;
            v[2] = rot_y * a.UC * a.M0 * 1e-3f;
            v[3] = rot_z * a.UC * a.M0 * 1e-3f;
        } else if (q == 1) {
            // wbuf_*_v (m_snap.f90:1466-1468)
            v[0] = a.Vx[e] * a.UC * a.M0;
            v[1] = a.Vy[e] * a.UC * a.M0;
            v[2] = a.Vz[e] * a.UC * a.M0;
        } else {
            // wbuf_*_u (m_snap.f90:1850-1852): time integration every step
            float *u = P.ubuf;
            v[0] = u[o] + a.Vx[e] * a.UC * a.M0 * a.dt;
            v[1] = u[ns + o] + a.Vy[e] * a.UC * a.M0 * a.dt;
            v[2] = u[2 * ns + o] + a.Vz[e] * a.UC * a.M0 * a.dt;
            u[o] = v[0];
            u[ns + o] = v[1];
            u[2 * ns + o] = v[2];
        }
        if (P.maxv) {
            // running maxima of the fs / ob planes (m_snap.f90:1691-1703)
            float *m = P.maxv;
            const float m1 = fmax_ref(m[o], fabsf(v[2]));
            const float m2 = fmax_ref(m[ns + o], sqrtf(v[0] * v[0] + v[1] * v[1]));
            m[o] = m1;
            m[ns + o] = m2;
            m[2 * ns + o] = sqrtf(m1 * m1 + m2 * m2);
        }
        if (store) {
            float *f = P.frames + (long long)((it - 1) / a.ntdec_s) * P.nv * ns;
            for (int c = 0; c < P.nv; c++) f[c * ns + o] = v[c];
        }
    }
}

}  // namespace

// snapshot state of a context
struct swpc_snap_state {
    swpc_snap_desc d;
    int nxs = 0, nys = 0, nzs = 0, nframes = 0;
    int is0 = 0, is1 = 0, js0 = 0, js1 = 0, ks0 = 0, ks1 = 0;
    std::vector<SnapPlane> planes;
    float *pool = nullptr;   // one allocation for frames, accumulators and maxima
    size_t pool_floats = 0;
    long long maxv_off[4] = {-1, -1, -1, -1};   // fs v, fs u, ob v, ob u
};

namespace swpc {

void snap_free(swpc_ctx *c) {
    if (!c->snp) return;
    if (c->snp->pool) cudaFree(c->snp->pool);
    delete c->snp;
    c->snp = nullptr;
}

int snap_clear(swpc_ctx *c) {
    if (!c->snp || !c->snp->pool) return SWPC_OK;
    return cuda_check(c, cudaMemsetAsync(c->snp->pool, 0, c->snp->pool_floats * sizeof(float), c->stream),
                      "cudaMemsetAsync");
}

int snap_launch(swpc_ctx *c, int it, const int *d_it) {
    swpc_snap_state *s = c->snp;
    if (!s || s->planes.empty()) return SWPC_OK;
    SnapArgs a;
    a.g = c->g;
    a.Vx = c->V[0]; a.Vy = c->V[1]; a.Vz = c->V[2];
    a.lam = c->med[1]; a.muyz = c->med[8]; a.muxz = c->med[9]; a.muxy = c->med[10];
    a.kfs = c->kfs; a.kob = c->kob;
    // r20 = 1 / d (m_snap.f90:311-313), real(MP) = single precision
    a.r20x = 1.0f / c->d.dx; a.r20y = 1.0f / c->d.dy; a.r20z = 1.0f / c->d.dz;
    a.UC = s->d.UC; a.M0 = s->d.M0; a.dt = c->d.dt;
    a.idec = s->d.idec; a.jdec = s->d.jdec; a.kdec = s->d.kdec; a.ntdec_s = s->d.ntdec_s; a.nt = c->d.nt;
    a.i0_yz = s->d.i0_yz; a.j0_xz = s->d.j0_xz; a.k0_xy = s->d.k0_xy;
    a.d_it = d_it; a.it = it;
    long long maxpts = 1;
    for (size_t n = 0; n < s->planes.size(); n++) {
        a.p[n] = s->planes[n];
        maxpts = std::max(maxpts, (long long)(a.p[n].a1 - a.p[n].a0 + 1) * (a.p[n].b1 - a.p[n].b0 + 1));
    }
    const int threads = 256;
    const long long bx = std::min<long long>((maxpts + threads - 1) / threads, 148LL * 8);
    snap3d_kernel<<<dim3((unsigned)bx, (unsigned)s->planes.size()), threads, 0, c->stream>>>(a);
    return cuda_check(c, cudaGetLastError(), "snap3d_kernel");
}

}  // namespace swpc

static void snap_shape(const swpc_snap_state *s, int plane, int *nv, int *n1, int *n2) {
    const int sec = plane / 3, q = plane % 3;
    *nv = q == 0 ? 4 : 3;
    if (sec == 0) { *n1 = s->nys; *n2 = s->nzs; }
    else if (sec == 1) { *n1 = s->nxs; *n2 = s->nzs; }
    else { *n1 = s->nxs; *n2 = s->nys; }
}

extern "C" int swpc_snap_setup(swpc_ctx *c, const swpc_snap_desc *d) {
    if (!c || !d) return SWPC_ERR_ARG;
    if (c->kind != SWPC_KIND_3D) return set_err(c, SWPC_ERR_ARG, "snapshots are implemented for the 3D solver");
    if (!c->medium_ready) return set_err(c, SWPC_ERR_STATE, "swpc_upload_medium must precede swpc_snap_setup");
    if (d->planes & ~0x7fff) return set_err(c, SWPC_ERR_ARG, "unknown snapshot plane bit");
    if (d->idec < 1 || d->jdec < 1 || d->kdec < 1 || d->ntdec_s < 1)
        return set_err(c, SWPC_ERR_ARG, "snapshot decimation factors must be >= 1");
    const int nx = c->d.nx, ny = c->d.ny, nz = c->d.nz;
    const bool yz = d->planes & 0x7, xz = d->planes & (0x7 << 3), xy = d->planes & (0x7 << 6);
    if ((yz && (d->i0_yz < 1 || d->i0_yz > nx)) || (xz && (d->j0_xz < 1 || d->j0_xz > ny)) ||
        (xy && (d->k0_xy < 1 || d->k0_xy > nz)))
        return set_err(c, SWPC_ERR_ARG, "snapshot section outside the domain");
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    graph_invalidate(c);
    snap_free(c);
    auto *s = new swpc_snap_state();
    c->snp = s;
    s->d = *d;
    // m_snap.f90:128-131 and 149-154 (single node: ibeg = 1, iend = nx, ...)
    s->nxs = (nx + d->idec / 2) / d->idec;
    s->nys = (ny + d->jdec / 2) / d->jdec;
    s->nzs = (nz + d->kdec / 2) / d->kdec;
    s->is0 = (int)std::ceil((float)(1 + d->idec / 2) / (float)d->idec);
    s->is1 = (int)std::floor((float)(nx + d->idec / 2) / (float)d->idec);
    s->js0 = (int)std::ceil((float)(1 + d->jdec / 2) / (float)d->jdec);
    s->js1 = (int)std::floor((float)(ny + d->jdec / 2) / (float)d->jdec);
    s->ks0 = (int)std::ceil((float)(1 + d->kdec / 2) / (float)d->kdec);
    s->ks1 = (int)std::floor((float)(nz + d->kdec / 2) / (float)d->kdec);
    s->nframes = (c->d.nt - 1) / d->ntdec_s + 1;
    // one pool: frames of every plane, u accumulators, fs/ob maxima
    size_t off = 0;
    struct Off { long long frames, ubuf, maxv; };
    std::vector<Off> offs;
    for (int p = 0; p < kPlanes; p++) {
        if (!(d->planes >> p & 1)) continue;
        int nv, n1, n2;
        snap_shape(s, p, &nv, &n1, &n2);
        const int sec = p / 3, q = p % 3;
        SnapPlane P{};
        P.plane = p; P.n1 = n1; P.n2 = n2; P.nv = nv;
        P.a0 = sec == 0 ? s->js0 : s->is0;
        P.a1 = sec == 0 ? s->js1 : s->is1;
        P.b0 = sec <= 1 ? s->ks0 : s->js0;
        P.b1 = sec <= 1 ? s->ks1 : s->js1;
        const size_t ns = (size_t)n1 * n2;
        Off o{(long long)off, -1, -1};
        off += (size_t)s->nframes * nv * ns;
        if (q == 2) { o.ubuf = (long long)off; off += 3 * ns; }
        if (sec >= 3 && q >= 1) {
            o.maxv = (long long)off;
            s->maxv_off[(sec - 3) * 2 + (q - 1)] = (long long)off;
            off += 3 * ns;
        }
        s->planes.push_back(P);
        offs.push_back(o);
    }
    s->pool_floats = off;
    if (off) {
        int rc = dalloc(c, &s->pool, off);
        if (rc) return rc;
        for (size_t n = 0; n < s->planes.size(); n++) {
            s->planes[n].frames = s->pool + offs[n].frames;
            s->planes[n].ubuf = offs[n].ubuf >= 0 ? s->pool + offs[n].ubuf : nullptr;
            s->planes[n].maxv = offs[n].maxv >= 0 ? s->pool + offs[n].maxv : nullptr;
        }
    }
    return SWPC_OK;
}

extern "C" int swpc_snap_write(swpc_ctx *c, int it) {
    if (!c) return SWPC_ERR_ARG;
    if (!c->snp) return set_err(c, SWPC_ERR_STATE, "swpc_snap_setup not called");
    if (it < 1 || it > c->d.nt + 1) return set_err(c, SWPC_ERR_ARG, "time step index outside 1..nt+1");
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    return snap_launch(c, it, nullptr);
}

extern "C" int swpc_snap_dims(const swpc_ctx *c, int plane, int *nvar, int *n1, int *n2, int *nframes) {
    if (!c || !c->snp || plane < 0 || plane >= kPlanes || !nvar || !n1 || !n2 || !nframes) return SWPC_ERR_ARG;
    snap_shape(c->snp, plane, nvar, n1, n2);
    *nframes = (c->snp->d.planes >> plane & 1) ? c->snp->nframes : 0;
    return SWPC_OK;
}

extern "C" int swpc_snap_fetch(swpc_ctx *c, int plane, float *out) {
    if (!c || !out) return SWPC_ERR_ARG;
    if (!c->snp) return set_err(c, SWPC_ERR_STATE, "swpc_snap_setup not called");
    for (const SnapPlane &P : c->snp->planes) {
        if (P.plane != plane) continue;
        if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
        const size_t bytes = sizeof(float) * (size_t)c->snp->nframes * P.nv * P.n1 * P.n2;
        int rc = cuda_check(c, cudaMemcpyAsync(out, P.frames, bytes, cudaMemcpyDeviceToHost, c->stream), "snap fetch");
        if (rc) return rc;
        return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    }
    return set_err(c, SWPC_ERR_ARG, "snapshot plane not enabled");
}

extern "C" int swpc_snap_fetch_max(swpc_ctx *c, int which, float *out) {
    if (!c || !out || which < 0 || which > 3) return SWPC_ERR_ARG;
    if (!c->snp) return set_err(c, SWPC_ERR_STATE, "swpc_snap_setup not called");
    const long long off = c->snp->maxv_off[which];
    if (off < 0) return set_err(c, SWPC_ERR_ARG, "maximum plane not enabled (needs the fs/ob v or u plane)");
    if (cudaSetDevice(c->device) != cudaSuccess) return set_err(c, SWPC_ERR_CUDA, "cudaSetDevice failed");
    const size_t bytes = sizeof(float) * 3 * (size_t)c->snp->nxs * c->snp->nys;
    int rc = cuda_check(c, cudaMemcpyAsync(out, c->snp->pool + off, bytes, cudaMemcpyDeviceToHost, c->stream),
                        "snap max fetch");
    if (rc) return rc;
    return cuda_check(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
}
