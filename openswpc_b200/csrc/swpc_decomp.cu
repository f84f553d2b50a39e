// swpc_decomp.cu -- one box of a decomposed grid and its halo exchange.
//
// The reference splits the horizontal plane over nproc_x x nproc_y ranks
// (3D; nproc_x for P-SV and SH), each holding its block ibeg:iend x
// jbeg:jend with a 3-cell sleeve (src/swpc_3d/m_global.f90:236-303), and
// after each half step trades the sleeve planes that the stencils of the
// next half step read (global__comm_stress / global__comm_vel,
// m_global.f90:393-609).  Here a context becomes such a block through
// swpc_set_subdomain: its grid is the block, the absorber and kernel region
// follow the global layout, and its halo planes are packed into / unpacked
// from flat buffers that the caller moves between neighbours (a device copy
// between contexts on one GPU, NCCL point-to-point or a peer-memory store
// between GPUs).  The pack kernel writes through any device pointer, a
// peer-mapped buffer included; nothing here waits on another GPU.
//
// Message layout: for each field of the half step's list, for each plane in
// ascending order, the plane's (perpendicular index, k) block with k fastest,
// k = 1..nz and the perpendicular index over the block's own extent (j = 1..ny
// for the x sides, i = 1..nx for the y sides: no corner cells, as the
// reference sends none).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "swpc_ctx.h"

using namespace swpc;

namespace swpc {
int build_tiles_2d(swpc_ctx *c);   // swpc2d_api.cu
}

#define CK(call)                                               \
    do {                                                       \
        int _rc = cuda_check(c, (call), #call);                \
        if (_rc) return _rc;                                   \
    } while (0)
#define RC(call)             \
    do {                     \
        int _rc = (call);    \
        if (_rc) return _rc; \
    } while (0)

namespace {

bool is3d(const swpc_ctx *c) { return c->kind == SWPC_KIND_3D; }

// The sleeve planes a field receives across one axis (the planes that
// global__comm_* overwrites): type A fields receive planes -1, 0 from the
// lower neighbour and n + 1 from the upper one, type B fields 0 from the
// lower and n + 1, n + 2 from the upper (m_global.f90:413-490, 521-603;
// src/swpc_psv/m_global.f90:356-414, src/swpc_sh/m_global.f90:340-388).
struct HaloField {
    int field;   // SWPC_F_*
    int type;    // 0: A (lower {-1, 0}, upper {1}), 1: B (lower {0}, upper {1, 2})
};

// fields of a half step (half 0: the stress exchange, half 1: the velocity
// exchange) across axis ax (0 x, 1 y)
std::vector<HaloField> halo_fields(int kind, int half, int ax) {
    if (kind == SWPC_KIND_PSV) {
        if (ax != 0) return {};
        return half == 0 ? std::vector<HaloField>{{SWPC_F_SXX, 1}, {SWPC_F_SXZ, 0}}
                         : std::vector<HaloField>{{SWPC_F_VX, 0}, {SWPC_F_VZ, 1}};
    }
    if (kind == SWPC_KIND_SH) {
        if (ax != 0) return {};
        return half == 0 ? std::vector<HaloField>{{SWPC_F_SXY, 0}} : std::vector<HaloField>{{SWPC_F_VY, 1}};
    }
    if (half == 0)
        return ax == 0 ? std::vector<HaloField>{{SWPC_F_SXX, 1}, {SWPC_F_SXY, 0}, {SWPC_F_SXZ, 0}}
                       : std::vector<HaloField>{{SWPC_F_SYY, 1}, {SWPC_F_SXY, 0}, {SWPC_F_SYZ, 0}};
    return ax == 0 ? std::vector<HaloField>{{SWPC_F_VX, 0}, {SWPC_F_VY, 1}, {SWPC_F_VZ, 1}}
                   : std::vector<HaloField>{{SWPC_F_VX, 1}, {SWPC_F_VY, 0}, {SWPC_F_VZ, 1}};
}

// offsets of the lower sleeve planes (relative to plane 0) and of the upper
// ones (relative to plane n) of a field type
const std::vector<int> &lower_planes(int type) {
    static const std::vector<int> a{-1, 0}, b{0};
    return type == 0 ? a : b;
}
const std::vector<int> &upper_planes(int type) {
    static const std::vector<int> a{1}, b{1, 2};
    return type == 0 ? a : b;
}

constexpr int kMaxPlanes = 12;

struct HaloPlan {
    int n;                       // planes of the message
    int ax;                      // 0: planes along i, 1: along j
    int np;                      // perpendicular extent (ny or nx; 1 in 2D)
    float *f[kMaxPlanes];
    int plane[kMaxPlanes];       // local plane index (i or j)
};

float *field_of(swpc_ctx *c, int field) {
    if (field >= SWPC_F_VX && field <= SWPC_F_VZ) return c->V[field - SWPC_F_VX];
    if (field >= SWPC_F_SXX && field <= SWPC_F_SXY) return c->S[field - SWPC_F_SXX];
    return nullptr;
}

// the planes this context sends to side `side` (pack) or receives from it
// (unpack): side 0 -x, 1 +x, 2 -y, 3 +y
int make_plan(swpc_ctx *c, int half, int side, bool pack, HaloPlan &p) {
    const int ax = side / 2;
    const bool upper = side % 2 == 1;
    const int n = ax == 0 ? c->g.nx : c->g.ny;
    p.n = 0;
    p.ax = ax;
    p.np = ax == 0 ? (is3d(c) ? c->g.ny : 1) : c->g.nx;
    for (const HaloField &h : halo_fields(c->kind, half, ax)) {
        float *f = field_of(c, h.field);
        if (!f) return set_err(c, SWPC_ERR_STATE, "halo field not allocated");
        // the upper neighbour receives into its lower planes, the lower one into its upper planes
        const std::vector<int> &offs = (upper == pack) ? lower_planes(h.type) : upper_planes(h.type);
        // packing, own planes n-1, n (to +) or 1, 2 (to -); unpacking, sleeve
        // planes n+1, n+2 (from +) or -1, 0 (from -)
        for (int o : offs) {
            if (p.n >= kMaxPlanes) return set_err(c, SWPC_ERR_STATE, "halo plan overflow");
            p.f[p.n] = f;
            p.plane[p.n] = upper ? n + o : o;
            p.n++;
        }
    }
    return SWPC_OK;
}

// one thread per (plane, perpendicular index, k) element of the message
__global__ void halo_kernel(const HaloPlan p, Geo g, bool threed, float *buf, int pack) {
    const long long per = (long long)p.np * g.nz;
    const long long total = per * p.n;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(q / per);
        const long long r = q - e * per;
        const int t = 1 + (int)(r / g.nz), k = 1 + (int)(r % g.nz);
        const int i = p.ax == 0 ? p.plane[e] : t;
        const int j = p.ax == 0 ? (threed ? t : -2) : p.plane[e];
        const long long cell = threed ? cell_index(g, k, i, j) : (long long)(i + 2) * g.Kp + (k - 1 + KH);
        if (pack) buf[q] = p.f[e][cell];
        else p.f[e][cell] = buf[q];
    }
}

int halo_run(swpc_ctx *c, int half, int side, float *buf, bool pack) {
    if (!c->sub) return set_err(c, SWPC_ERR_STATE, "swpc_set_subdomain was not called");
    if (half != 0 && half != 1) return set_err(c, SWPC_ERR_ARG, "half must be 0 (stress) or 1 (velocity)");
    if (side < 0 || side > 3 || (!is3d(c) && side > 1)) return set_err(c, SWPC_ERR_ARG, "side must be 0..3 (0..1 in 2D)");
    if (!buf) return set_err(c, SWPC_ERR_ARG, "halo buffer missing");
    HaloPlan p;
    RC(make_plan(c, half, side, pack, p));
    const long long total = (long long)p.n * p.np * c->g.nz;
    if (total == 0) return SWPC_OK;
    CK(cudaSetDevice(c->device));
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
    halo_kernel<<<blocks, 256, 0, c->stream>>>(p, c->g, is3d(c), buf, pack ? 1 : 0);
    return cuda_check(c, cudaGetLastError(), "halo_kernel");
}

// m_global.f90:236-303: the block of rank (px, py) has its first cell at
// global index ioff + 1; the kernel region of the block follows :349-378
void kernel_region(int beg, int end, int n, int na, int &bk, int &ek) {
    bk = beg;
    ek = end;
    if (end <= na) bk = end + 1;
    else if (beg <= na) bk = na + 1;
    if (beg >= n - na + 1) ek = beg - 1;
    else if (end >= n - na + 1) ek = n - na;
}

}  // namespace

extern "C" int swpc_set_subdomain(swpc_ctx *c, int nx_global, int ny_global, int ioff, int joff) {
    if (!c) return SWPC_ERR_ARG;
    if (c->medium_ready || c->absorb_ready || c->kernel_ready)
        return set_err(c, SWPC_ERR_STATE, "swpc_set_subdomain must precede the medium, kernel and absorber setup");
    const bool threed = is3d(c);
    if (!threed) { ny_global = 1; joff = 0; }
    const int na = c->d.na;
    if (ioff < 0 || joff < 0 || ioff + c->g.nx > nx_global || joff + c->g.ny > ny_global)
        return set_err(c, SWPC_ERR_ARG, "subdomain outside the global grid");
    if (2 * na >= nx_global || (threed && 2 * na >= ny_global))
        return set_err(c, SWPC_ERR_ARG, "absorber thickness na too large for the global grid");
    int ibk, iek, jbk = 1, jek = 1;
    kernel_region(ioff + 1, ioff + c->g.nx, nx_global, na, ibk, iek);
    if (threed) kernel_region(joff + 1, joff + c->g.ny, ny_global, na, jbk, jek);
    c->ibk = ibk - ioff;
    c->iek = iek - ioff;
    if (threed) { c->jbk = jbk - joff; c->jek = jek - joff; }
    c->nxg = nx_global;
    c->nyg = threed ? ny_global : 1;
    c->ioff = ioff;
    c->joff = joff;
    c->sub = true;
    c->na_wide = false;   // checked against the global grid above
    c->desc_dirty = true;
    // the 2D tile list flags interior and absorber tiles by the kernel region
    if (!threed) RC(build_tiles_2d(c));
    return SWPC_OK;
}

extern "C" int swpc_halo_count(swpc_ctx *c, int half, int side, long long *count) {
    if (!c || !count) return SWPC_ERR_ARG;
    if (side < 0 || side > 3 || (!is3d(c) && side > 1) || (half != 0 && half != 1))
        return set_err(c, SWPC_ERR_ARG, "half 0..1, side 0..3 (0..1 in 2D)");
    HaloPlan p;
    RC(make_plan(c, half, side, true, p));
    *count = (long long)p.n * p.np * c->g.nz;
    return SWPC_OK;
}

extern "C" int swpc_halo_pack(swpc_ctx *c, int half, int side, float *dst) {
    if (!c) return SWPC_ERR_ARG;
    return halo_run(c, half, side, dst, true);
}

extern "C" int swpc_halo_unpack(swpc_ctx *c, int half, int side, const float *src) {
    if (!c) return SWPC_ERR_ARG;
    return halo_run(c, half, side, const_cast<float *>(src), false);
}

// Lets kernels running on `device` store to (and load from) memory of `peer`,
// so that a block's pack kernel can write its message straight into a
// neighbour's receive buffer on another GPU (NVLink peer stores).  Returns
// SWPC_ERR_CUDA when the pair has no peer access; enabling it twice is fine.
extern "C" int swpc_enable_peer_access(int device, int peer) {
    if (device == peer) return SWPC_OK;
    int can = 0;
    if (cudaDeviceCanAccessPeer(&can, device, peer) != cudaSuccess || !can) return SWPC_ERR_CUDA;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaError_t e = cudaDeviceEnablePeerAccess(peer, 0);
    if (e == cudaErrorPeerAccessAlreadyEnabled) {
        cudaGetLastError();   // the call left this as the last error: clear it
        e = cudaSuccess;
    }
    cudaSetDevice(cur);
    return e == cudaSuccess ? SWPC_OK : SWPC_ERR_CUDA;
}
