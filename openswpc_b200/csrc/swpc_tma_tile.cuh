// swpc_tma_tile.cuh -- tiles of the TMA-staged 3D kernels (swpc3d_tma.cu, and
// the staged adjoint kernels of swpc_adjoint.cu): which tile and member group
// a CTA owns, what the tile holds, and how many CTAs fit an SM.
#pragma once

#include "swpc_tma.h"

namespace swpc {
namespace tma {

constexpr int KT = 32;       // cells of a tile along k
constexpr int KB = KT + 8;   // k extent of a halo box: k0-4 .. k0+35 (16-byte aligned start)

struct Tile {
    int k0, i0, j0, m0, nmem;   // first cell, first member, members in the group
};

// Tile and member group of this CTA: member groups fastest, then the tiles
// (the medium of a tile is re-read from L2 by the groups that follow), or with
// t.tiles_first the tiles fastest and the groups one after another.  Within a
// group the tiles run k fastest, then over (i, j) in blocks of t.jblock
// consecutive j tiles: j fastest inside a block, then i, then the next block,
// so that the j halo of a tile comes from tiles launched a few CTAs earlier,
// still in L2, instead of a j plane of tiles earlier.
template <int M>
__device__ __forceinline__ Tile tile_of(const TmaTiles &t, int bi, int bj) {
    const int ntile = t.nkt * t.nit * t.njt;
    const int grp = t.tiles_first ? blockIdx.x / ntile : blockIdx.x % t.mgroups;
    const int b = t.tiles_first ? blockIdx.x % ntile : blockIdx.x / t.mgroups;
    const int kt = b % t.nkt, r = b / t.nkt;
    const int jb = t.jblock, blk = r / (t.nit * jb), rem = r - blk * t.nit * jb;
    const int nb = min(jb, t.njt - blk * jb);   // j tiles in this block (the last one may be short)
    const int it = rem / nb, jt = blk * jb + rem % nb;
    const int m0 = grp * M;
    return Tile{1 + KT * kt, 1 + bi * it, 1 + bj * jt, m0, min(M, t.nmem - m0)};
}

__device__ __forceinline__ bool tile_has_interior(const Tile &T, int bi, int bj, int ibk, int iek, int jbk, int jek,
                                                  int kek) {
    return T.k0 <= kek && T.i0 <= iek && T.i0 + bi - 1 >= ibk && T.j0 <= jek && T.j0 + bj - 1 >= jbk;
}
// does the tile hold absorber cells (cells of the grid outside the kernel region)?
__device__ __forceinline__ bool tile_has_absorber(const Tile &T, int bi, int bj, const Geo &g, int ibk, int iek,
                                                  int jbk, int jek, int kek) {
    const int i1 = min(T.i0 + bi - 1, g.nx), j1 = min(T.j0 + bj - 1, g.ny), k1 = min(T.k0 + KT - 1, g.nz);
    return T.i0 < ibk || i1 > iek || T.j0 < jbk || j1 > jek || k1 > kek;
}

template <int SMEM_FLOATS, int THREADS>
__host__ __device__ constexpr int blocks_per_sm() {
    constexpr int by_smem = (227 * 1024) / (SMEM_FLOATS * 4 + 128 + 1024);
    constexpr int by_threads = 1024 / THREADS;   // at least 64 registers a thread
    constexpr int n = by_smem < by_threads ? by_smem : by_threads;
    return n < 1 ? 1 : n;
}

}  // namespace tma
}  // namespace swpc
