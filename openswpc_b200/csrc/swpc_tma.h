// swpc_tma.h -- launch interface of the TMA-staged 3D kernels (swpc3d_tma.cu).
#pragma once

#include <cuda_runtime.h>

#include "swpc_kernels.cuh"

namespace swpc {

// tile grid of a staged launch: tiles of kt (k) x bi (i) x bj (j) cells
struct TmaTiles {
    int nkt, nit, njt;
    int b_field;   // slab index of bx (velocity kernel)
    int *err;      // raised when a tile copy does not complete
};

// host copies of the tensor maps (CUtensorMap, 128 bytes, 64-byte aligned)
struct alignas(64) TmaMaps {
    unsigned char str[128];    // stress: S, medium, R of the tile
    unsigned char v3h[128];    // stress: V with halo
    unsigned char own3[128];   // velocity: V (and bx by bz) of the tile
    unsigned char va[128], vb[128], vc[128], vf[128], ve[128], vd[128];   // velocity: Sxx Syy Szz Syz Sxz Sxy
};

// tile shapes (kt = cells along k: 32 or 64; bi x bj columns) with compiled kernels
bool tma_shape_ok(int kt, int bi, int bj);       // stress tiles
bool tma_vel_shape_ok(int kt, int bi, int bj);   // velocity tiles
bool tma_encode_stress(TmaMaps &m, float *slab, const Geo &g, int nf, int nm, int kt, int bi, int bj);
bool tma_encode_vel(TmaMaps &m, float *slab, const Geo &g, int nf, int kt, int bi, int bj);
cudaError_t launch_stress3d_tma(const TmaMaps &m, const Str3Args &a, const TmaTiles &t, int nm, int kt, int bi, int bj,
                                cudaStream_t st);
cudaError_t launch_vel3d_tma(const TmaMaps &m, const Vel3Args &a, const TmaTiles &t, int kt, int bi, int bj,
                             cudaStream_t st);

}  // namespace swpc
