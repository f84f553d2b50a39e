// swpc2d.cuh -- device descriptors of the 2D P-SV / SH solvers.
#pragma once

#include <cuda_runtime.h>

#include "swpc_ctx.h"

namespace swpc {

// One 2D model as the kernels see it (device-resident, one per ensemble
// member).  Cell (k, i) of a field is at (i + 2) * Kp + (k - 1 + KH).
//   P-SV: V0 = Vx, V1 = Vz; S0 = Sxx, S1 = Szz, S2 = Sxz; R[c*3+m], c = xx zz xz
//         aux = axVx azVx axVz azVz axSxx azSxz axSxz azSzz
//   SH:   V0 = Vy;          S0 = Syz, S1 = Sxy;          R[c*3+m], c = yz xy
//         aux = axVy azVy axSxy azSyz
struct Model2D {
    int nx, nz, Kp, nm;
    int ibk, iek, kek;
    float dt;
    float *V0, *V1;
    float *S0, *S1, *S2;
    float *R[9];
    const float *rho, *lam, *mu, *taup, *taus;
    const int4 *band;     // [i + 2]: kfs_top kfs_bot kob_top kob_bot
    const int2 *pmlcol;   // [i + 2]: kbeg_a, aux base
    float *aux[8];
    const float4 *gxc, *gxe, *gzc, *gze;
    float e40[2][2], e41[2][2];   // [axis x/z][0: 4th order, 1: 2nd-order band]
    float r20[2];
    float c1[NM_MAX], c2[NM_MAX], d1[NM_MAX], d2;
};

// A tile of 32 (k) x (tile step) (i) cells of one model; flags: the tile
// holds interior (kTileInterior) and absorber (kTileAbsorber) cells.
struct Tile2D {
    int model, k0, i0, flags;
};
constexpr int kTileInterior = 1, kTileAbsorber = 2;

struct Wav2Args {
    int Kp, nst, ntw, ntdec_w, what, psv;
    const int *st;            // (2, nst) i k
    const float *V0, *V1;
    float *uacc;              // (2, nst)
    float *wav_v, *wav_u;     // (ntw, ncmp, nst)
    float M0, UC, dt;
};

// Launch shape of the tile kernels: tiles of 32 (k) x (ti * ri) (i) cells,
// one block of 32 x ti threads per tile with ri rows per thread, and a
// persistent grid of 148 x blocks_per_sm blocks (0: one block per tile).
// The results do not depend on the shape.
struct TileShape {
    int ti, ri, blocks_per_sm;
};
constexpr TileShape kDefaultTiles{4, 4, 0};

// TMA-staged kernels (swpc2d_tma.cu): tiles of 32 (k) x kTileI2D (i), one
// CTA of 32 x ti threads per tile (ti = 4, 8 or 16), the operands of each
// model read through its tensor maps, which travel as a kernel parameter: a
// launch covers one model, or up to kGroup2D consecutive models of a batch
// (their sets fill the 32 KB parameter space).  Field indices of a model's
// slab: V at v, S at s (R follows S), lam taup taus mu rho from med.
constexpr int kTileI2D = 16;
constexpr int kGroup2D = 48;
struct Fields2D {
    int v, s, med;
};
// the tensor maps of one model for one phase (CUtensorMap: 128 bytes)
struct alignas(64) MapSet2D {
    unsigned char m[5][128];
};
struct Maps2D {
    MapSet2D str, vel;
};
Fields2D fields2d(int kind, int nm);
int slab_fields2d(int kind, int nm);
bool staged2d_ti_ok(int ti);
bool encode_maps2d(Maps2D &m, int kind, int nm, float *slab, const Geo &g);
// one launch over the ntiles tiles from `tiles`, all of models model0 ..
// model0 + nset - 1 (nset = 1 .. kGroup2D), whose map sets are sets[0 .. nset-1]
cudaError_t launch_stress2d_tma(int kind, int nm, int ti, const MapSet2D *sets, int nset, int model0,
                                const Model2D *models, const Tile2D *tiles, int ntiles, int mask, Fields2D f, int *err,
                                cudaStream_t st);
cudaError_t launch_vel2d_tma(int kind, int ti, const MapSet2D *sets, int nset, int model0, const Model2D *models,
                             const Tile2D *tiles, int ntiles, int mask, Fields2D f, int *err, cudaStream_t st);
// flags of the tile (k0, i0) of a model (tile extents 32 x ni)
int tile2d_flags(const swpc_ctx *c, int k0, int i0, int ni);

void launch_stress2d(int kind, int nm, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                     TileShape ts, cudaStream_t st);
void launch_vel2d(int kind, const Model2D *models, const Tile2D *tiles, int ntiles, int mask, TileShape ts,
                  cudaStream_t st);
void launch_wav2d(const Wav2Args *list, int nlist, int max_nst, int it, const int *d_it, cudaStream_t st);
void launch_vmax2d(const float *V0, const float *V1, const int *kob, int Kp, int i0, int i1, unsigned int *out,
                   cudaStream_t st);

}  // namespace swpc
