// swpc2d_kernels.cu -- 2D P-SV and SH time-step kernels for sm_100a.
//
// Every launch works on a table of models and a list of 32 (k) x (TI*RI) (i)
// tiles covering all of them (a block of 32 x TI threads, RI rows per thread), walked by a persistent grid: one model is the
// single-run case, many models of uneven size are the batched ensemble, and
// both run the same code.  Per cell the kernels restate
//   P-SV: src/swpc_psv/m_kernel.f90:76-306 (interior) and
//         src/swpc_psv/m_absorb_p.f90:180-230, 337-385 (ADE-CFS PML),
//   SH:   src/swpc_sh/m_kernel.f90:77-221 and src/swpc_sh/m_absorb_p.f90,
// in the reference's expression order; the file is compiled with
// -fmad=false so the FP32 results are bitwise identical to the oracle.
#include <cuda_runtime.h>

#include "swpc_ctx.h"
#include "swpc2d.cuh"
#include "swpc2d_cell.cuh"

namespace swpc {

namespace {
// The block's copy of the model descriptor of the current tile.  Shared
// memory does not alias the fields the kernel stores to, so the descriptor
// is read once per tile instead of after every store, and consecutive tiles
// of the same model reuse it.  Uniform over the block.
__device__ __forceinline__ const Model2D &tile_model(const Model2D *__restrict__ models, int model, Model2D &sM,
                                                     int &cached) {
    if (model != cached) {
        __syncthreads();   // every thread is done with the previous copy
        const int nw = (int)(sizeof(Model2D) / sizeof(int));
        const int *src = reinterpret_cast<const int *>(models + model);
        int *dst = reinterpret_cast<int *>(&sM);
        for (int w = threadIdx.y * blockDim.x + threadIdx.x; w < nw; w += blockDim.x * blockDim.y) dst[w] = __ldg(src + w);
        __syncthreads();
        cached = model;
    }
    return sM;
}
}  // namespace

// ---------------------------------------------------------------------------
// stress and velocity: kernel__update_stress / kernel__update_vel with
// absorb_p__update_stress / absorb_p__update_vel, operands from global memory
// ---------------------------------------------------------------------------
// kind 0 P-SV, 1 SH; phase 0 stress, 1 velocity
template <int KIND, int PHASE, int NM>
__global__ void __launch_bounds__(256) tile2d_kernel(const Model2D *__restrict__ models,
                                                     const Tile2D *__restrict__ tiles, int ntiles, int mask, int ri) {
    __shared__ Model2D sM;
    int cached = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile2D tl = tiles[t];
        const Model2D &M = tile_model(models, tl.model, sM, cached);
        // ri rows of the tile per thread: the tile and model descriptors are
        // fetched once for ri cells
        for (int r = 0; r < ri; r++) {
            const int k = tl.k0 + threadIdx.x, i = tl.i0 + threadIdx.y + r * (int)blockDim.y;
            if (k > M.nz || i > M.nx) continue;
            const bool interior = i >= M.ibk && i <= M.iek && k <= M.kek;
            if (!(mask & (interior ? 1 : 2))) continue;
            const long long PI = M.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const G2Ops o{M, e, PI};
            const int s = interior ? band_sign2d(M, k, i) : -1;
            if (KIND == 0 && PHASE == 0) {
                if (interior) psv_stress_interior<NM>(M, o, s, e);
                else psv_stress_absorber(M, o, k, i, e);
            } else if (KIND == 0) {
                psv_vel_cell(M, o, k, i, e, s);
            } else if (PHASE == 0) {
                sh_stress_cell<NM>(M, o, k, i, e, s);
            } else {
                sh_vel_cell(M, o, k, i, e, s);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// recorder (src/swpc_psv/m_wav.f90:170-260, src/swpc_sh/m_wav.f90:170-250)
// and vmax (src/swpc_psv/m_kernel.f90:308-324)
// ---------------------------------------------------------------------------
__global__ void wav2d_kernel(const Wav2Args *__restrict__ list, int nlist, int it_arg, const int *d_it) {
    const int it = d_it ? *d_it : it_arg;
    for (int b = blockIdx.y; b < nlist; b += gridDim.y) {
        const Wav2Args &a = list[b];
        for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.nst; n += gridDim.x * blockDim.x) {
            const int i = a.st[2 * n], k = a.st[2 * n + 1];
            const long long PI = a.Kp;
            const long long e = (long long)(i + 2) * PI + (k - 1 + KH);
            const float dt = a.dt;
            if (a.what & SWPC_WAV_U) {
                if (a.psv) {
                    a.uacc[2 * n] = a.uacc[2 * n] + (a.V0[e] + a.V0[e - PI]) * 0.5f * dt;
                    a.uacc[2 * n + 1] = a.uacc[2 * n + 1] - (a.V1[e] + a.V1[e - 1]) * 0.5f * dt;
                } else {
                    a.uacc[2 * n] = a.uacc[2 * n] + a.V0[e] * dt;
                }
            }
            if (it < 1 || (it - 1) % a.ntdec_w != 0) continue;
            const int itw = (it - 1) / a.ntdec_w + 1;
            if (itw > a.ntw) continue;
            const long long ntw = a.ntw;
            const int nc = a.psv ? 2 : 1;
            const float M0 = a.M0, UC = a.UC;
            if (a.what & SWPC_WAV_V) {
                float *w = a.wav_v + (long long)n * nc * ntw + (itw - 1);
                if (a.psv) {
                    w[0] = (a.V0[e] + a.V0[e - PI]) / 2.0f * M0 * UC * 1e9f;
                    w[ntw] = -(a.V1[e] + a.V1[e - 1]) / 2.0f * M0 * UC * 1e9f;
                } else {
                    w[0] = a.V0[e] * M0 * UC * 1e9f;
                }
            }
            if (a.what & SWPC_WAV_U) {
                float *w = a.wav_u + (long long)n * nc * ntw + (itw - 1);
                w[0] = a.uacc[2 * n] * M0 * UC * 1e9f;
                if (a.psv) w[ntw] = a.uacc[2 * n + 1] * M0 * UC * 1e9f;
            }
        }
    }
}

__global__ void vmax2d_kernel(const float *V0, const float *V1, const int *kob, int Kp, int i0, int i1,
                              unsigned int *out) {
    unsigned int a = 0, b = 0;
    for (int i = i0 + blockIdx.x * blockDim.x + threadIdx.x; i <= i1; i += gridDim.x * blockDim.x) {
        const int k = kob[i + 2] + 1;
        const long long e = (long long)(i + 2) * Kp + (k - 1 + KH);
        a = max(a, __float_as_uint(fabsf(V0[e])));
        if (V1) b = max(b, __float_as_uint(fabsf(V1[e])));
    }
    for (int o = 16; o > 0; o >>= 1) {
        a = max(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], a);
        atomicMax(&out[1], b);
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int persistent_grid(int ntiles, int blocks_per_sm) {
    // 148 SMs x blocks_per_sm resident blocks, never more blocks than tiles;
    // blocks_per_sm = 0: one block per tile
    const int g = blocks_per_sm > 0 ? 148 * blocks_per_sm : ntiles;
    return ntiles < g ? (ntiles > 0 ? ntiles : 1) : g;
}

void launch_stress2d(int kind, int nm, const Model2D *models, const Tile2D *tiles, int ntiles, int mask,
                     TileShape ts, cudaStream_t st) {
    const dim3 block(32, ts.ti);
    const int grid = persistent_grid(ntiles, ts.blocks_per_sm);
    if (kind == SWPC_KIND_PSV) {
        switch (nm) {
        case 0: tile2d_kernel<0, 0, 0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 1: tile2d_kernel<0, 0, 1><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 2: tile2d_kernel<0, 0, 2><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        default: tile2d_kernel<0, 0, 3><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        }
    } else {
        switch (nm) {
        case 0: tile2d_kernel<1, 0, 0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 1: tile2d_kernel<1, 0, 1><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        case 2: tile2d_kernel<1, 0, 2><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        default: tile2d_kernel<1, 0, 3><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri); break;
        }
    }
}

void launch_vel2d(int kind, const Model2D *models, const Tile2D *tiles, int ntiles, int mask, TileShape ts,
                  cudaStream_t st) {
    const dim3 block(32, ts.ti);
    const int grid = persistent_grid(ntiles, ts.blocks_per_sm);
    if (kind == SWPC_KIND_PSV) tile2d_kernel<0, 1, 0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri);
    else tile2d_kernel<1, 1, 0><<<grid, block, 0, st>>>(models, tiles, ntiles, mask, ts.ri);
}

void launch_wav2d(const Wav2Args *list, int nlist, int max_nst, int it, const int *d_it, cudaStream_t st) {
    if (nlist <= 0 || max_nst <= 0) return;
    const int threads = 128;
    const dim3 grid((max_nst + threads - 1) / threads, nlist < 65535 ? nlist : 65535);
    wav2d_kernel<<<grid, threads, 0, st>>>(list, nlist, it, d_it);
}

void launch_vmax2d(const float *V0, const float *V1, const int *kob, int Kp, int i0, int i1, unsigned int *out,
                   cudaStream_t st) {
    vmax2d_kernel<<<8, 256, 0, st>>>(V0, V1, kob, Kp, i0, i1, out);
}

}  // namespace swpc
