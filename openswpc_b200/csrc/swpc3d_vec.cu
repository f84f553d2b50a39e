// swpc3d_vec.cu -- the fused 3D velocity update with four consecutive k per
// thread (kernel__update_vel, src/swpc_3d/m_kernel.f90:75-140, and
// absorb_p__update_vel, src/swpc_3d/m_absorb_p.f90:248-309).
//
// A warp covers 128 consecutive k of one (i, j) column.  Every operand of the
// four cells arrives as one 16-byte load (V, b and the i/j stencil planes),
// and the k stencil of Sxz, Syz and Szz comes from the neighbouring lanes by
// warp shuffles; only the two lanes at the ends of the run load their extra
// k neighbours directly.  That replaces the 36 scalar loads per cell of the
// one-cell-per-thread kernel by 7.5 vector loads, which takes the kernel
// from load-issue bound towards HBM bound.  Groups of four that are not
// entirely interior (absorber columns, the group holding the interior /
// absorber boundary, the end of a column) run the one-cell routine for each
// cell.  Per cell the arithmetic is that of vel_cell, in the same order, so
// the results are bitwise identical.
#include <cuda_runtime.h>

#include "swpc3d_cell.cuh"

namespace swpc {

__device__ __forceinline__ float4 ld4(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ float4 ld4s(const float *p) { return __ldcs(reinterpret_cast<const float4 *>(p)); }
__device__ __forceinline__ void st4s(float *p, const float4 v) { __stcs(reinterpret_cast<float4 *>(p), v); }
__device__ __forceinline__ float at(const float4 &v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) vel3d_vec_kernel(const Vel3Args a) {
    const Geo g = a.g;
    const int lane = threadIdx.x;
    const int k0 = 1 + 4 * (blockIdx.x * 32 + lane);
    const int i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    if (i > g.nx || j > g.ny) return;   // uniform over the warp, which spans k only
    const bool active = k0 <= g.nz;
    const bool interior_col = i >= a.ibk && i <= a.iek && j >= a.jbk && j <= a.jek;
    if (interior_col && (a.mask & 1)) {   // uniform over the warp
        const bool vec = active && k0 + 3 <= a.kek;
        const long long col = col_index(g, i, j);
        const long long e = col * g.Kp + (k0 - 1 + KH);   // 16-byte aligned: Kp % 8 == 0, KH % 4 == 0
        const long long PI = g.Kp;
        const long long PJ = (long long)g.Kp * g.Ip;
        // own k runs of the three k-stencil fields; every active lane loads
        // them so that its neighbours can take their halo by shuffle
        float4 xz = make_float4(0.f, 0.f, 0.f, 0.f), yz = xz, zz = xz;
        if (active) {
            xz = ld4(a.Sxz + e);
            yz = ld4(a.Syz + e);
            zz = ld4(a.Szz + e);
        }
        const unsigned full = 0xffffffffu;
        // windows k0-2 .. k0+4 (Sxz, Syz) and k0-1 .. k0+5 (Szz)
        float xzw[7], yzw[7], zzw[7];
        xzw[0] = __shfl_up_sync(full, xz.z, 1);
        xzw[1] = __shfl_up_sync(full, xz.w, 1);
        xzw[6] = __shfl_down_sync(full, xz.x, 1);
        yzw[0] = __shfl_up_sync(full, yz.z, 1);
        yzw[1] = __shfl_up_sync(full, yz.w, 1);
        yzw[6] = __shfl_down_sync(full, yz.x, 1);
        zzw[0] = __shfl_up_sync(full, zz.w, 1);
        zzw[5] = __shfl_down_sync(full, zz.x, 1);
        zzw[6] = __shfl_down_sync(full, zz.y, 1);
        if (vec) {
            if (lane == 0) {
                xzw[0] = __ldg(a.Sxz + e - 2);
                xzw[1] = __ldg(a.Sxz + e - 1);
                yzw[0] = __ldg(a.Syz + e - 2);
                yzw[1] = __ldg(a.Syz + e - 1);
                zzw[0] = __ldg(a.Szz + e - 1);
            }
            if (lane == 31 || k0 + 4 > g.nz) {   // k0 + 5 <= nz + 2 stays inside the memory box
                xzw[6] = __ldg(a.Sxz + e + 4);
                yzw[6] = __ldg(a.Syz + e + 4);
                zzw[5] = __ldg(a.Szz + e + 4);
                zzw[6] = __ldg(a.Szz + e + 5);
            }
            xzw[2] = xz.x; xzw[3] = xz.y; xzw[4] = xz.z; xzw[5] = xz.w;
            yzw[2] = yz.x; yzw[3] = yz.y; yzw[4] = yz.z; yzw[5] = yz.w;
            zzw[1] = zz.x; zzw[2] = zz.y; zzw[3] = zz.z; zzw[4] = zz.w;

            const float4 vx = ld4s(a.Vx + e), vy = ld4s(a.Vy + e), vz = ld4s(a.Vz + e);
            const float4 bx = ld4s(a.bx + e), by = ld4s(a.by + e), bz = ld4s(a.bz + e);
            const float4 xx0 = ld4(a.Sxx + e), xxp = ld4(a.Sxx + e + PI), xxp2 = ld4(a.Sxx + e + 2 * PI),
                         xxm = ld4(a.Sxx + e - PI);
            const float4 yy0 = ld4(a.Syy + e), yyp = ld4(a.Syy + e + PJ), yyp2 = ld4(a.Syy + e + 2 * PJ),
                         yym = ld4(a.Syy + e - PJ);
            const float4 xy0 = ld4(a.Sxy + e);
            const float4 xyjm = ld4(a.Sxy + e - PJ), xyjp = ld4(a.Sxy + e + PJ), xyjm2 = ld4(a.Sxy + e - 2 * PJ);
            const float4 xyim = ld4(a.Sxy + e - PI), xyip = ld4(a.Sxy + e + PI), xyim2 = ld4(a.Sxy + e - 2 * PI);
            const float4 xzim = ld4(a.Sxz + e - PI), xzip = ld4(a.Sxz + e + PI), xzim2 = ld4(a.Sxz + e - 2 * PI);
            const float4 yzjm = ld4(a.Syz + e - PJ), yzjp = ld4(a.Syz + e + PJ), yzjm2 = ld4(a.Syz + e - 2 * PJ);
            const int4 bd = __ldg(&a.band[col]);
            const float dt = a.dt;
            float ox[4], oy[4], oz[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int k = k0 + c;
                const int p1 = (k - bd.x) * (bd.y - k);
                const int p2 = (k - bd.z) * (bd.w - k);
                const int s = ((p1 > p2 ? p1 : p2) >= 0) ? 1 : 0;   // isign = +1 -> 2nd-order band
                const float re40x = a.e40[0][s], re41x = a.e41[0][s];
                const float re40y = a.e40[1][s], re41y = a.e41[1][s];
                const float re40z = a.e40[2][s], re41z = a.e41[2][s];
                const float d3Sx3 = (at(xxp, c) - at(xx0, c)) * re40x - (at(xxp2, c) - at(xxm, c)) * re41x
                                  + (at(xy0, c) - at(xyjm, c)) * re40y - (at(xyjp, c) - at(xyjm2, c)) * re41y
                                  + (xzw[c + 2] - xzw[c + 1]) * re40z - (xzw[c + 3] - xzw[c]) * re41z;
                const float d3Sy3 = (at(xy0, c) - at(xyim, c)) * re40x - (at(xyip, c) - at(xyim2, c)) * re41x
                                  + (at(yyp, c) - at(yy0, c)) * re40y - (at(yyp2, c) - at(yym, c)) * re41y
                                  + (yzw[c + 2] - yzw[c + 1]) * re40z - (yzw[c + 3] - yzw[c]) * re41z;
                const float d3Sz3 = (xzw[c + 2] - at(xzim, c)) * re40x - (at(xzip, c) - at(xzim2, c)) * re41x
                                  + (yzw[c + 2] - at(yzjm, c)) * re40y - (at(yzjp, c) - at(yzjm2, c)) * re41y
                                  + (zzw[c + 2] - zzw[c + 1]) * re40z - (zzw[c + 3] - zzw[c]) * re41z;
                ox[c] = at(vx, c) + at(bx, c) * d3Sx3 * dt;
                oy[c] = at(vy, c) + at(by, c) * d3Sy3 * dt;
                oz[c] = at(vz, c) + at(bz, c) * d3Sz3 * dt;
            }
            st4s(a.Vx + e, make_float4(ox[0], ox[1], ox[2], ox[3]));
            st4s(a.Vy + e, make_float4(oy[0], oy[1], oy[2], oy[3]));
            st4s(a.Vz + e, make_float4(oz[0], oz[1], oz[2], oz[3]));
            return;
        }
    }
    // groups that are not entirely interior: one cell at a time
    if (!active) return;
#pragma unroll 1
    for (int c = 0; c < 4; c++) {
        const int k = k0 + c;
        if (k <= g.nz) vel_cell<PREC_F32>(a, k, i, j);
    }
}

void launch_vel3d_vec(const Vel3Args &a, int minb, dim3 block, cudaStream_t st) {
    const Geo &g = a.g;
    const dim3 grid((g.nz + 127) / 128, (g.nx + block.y - 1) / block.y, (g.ny + block.z - 1) / block.z);
    switch (minb) {
    case 1: vel3d_vec_kernel<1><<<grid, block, 0, st>>>(a); break;
    case 2: vel3d_vec_kernel<2><<<grid, block, 0, st>>>(a); break;
    case 3: vel3d_vec_kernel<3><<<grid, block, 0, st>>>(a); break;
    default: vel3d_vec_kernel<4><<<grid, block, 0, st>>>(a); break;
    }
}

}  // namespace swpc
