// swpc3d_kernels.cu -- fused sm_100a kernels of the 3D viscoelastic step.
//
// One launch per half step covers the whole domain: cells of the interior
// kernel region (m_global.f90:349-378) run the 4th-order viscoelastic update
// of src/swpc_3d/m_kernel.f90, the remaining cells (k >= kbeg_a(i,j),
// m_global.f90:336-345) run the 2nd-order ADE-CFS PML update of
// src/swpc_3d/m_absorb_p.f90.  The two regions are disjoint and neither pass
// reads what the other writes within a half step, so the fused launch gives
// exactly the result of the two reference routines run one after the other.
//
// Arithmetic: every expression keeps the reference's left-to-right order and
// this file is compiled with -fmad=false, so each product and sum is rounded
// separately exactly as the single-precision (MP = SP) Fortran build spells
// it out; the results are bitwise identical to the CPU oracle.
//
// Thread mapping: a warp owns 32 consecutive k of one (i, j) column (one
// coalesced 128-byte row per field); block = 32 x BI x BJ columns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "swpc_ctx.h"
#include "swpc_kernels.cuh"
#include "swpc3d_cell.cuh"

namespace swpc {

// ---------------------------------------------------------------------------
// velocity: one thread per cell (vel_cell in swpc3d_cell.cuh)
// ---------------------------------------------------------------------------
template <int MINB, int PREC>
__global__ void __launch_bounds__(256, MINB) vel3d_kernel(const Vel3Args a) {
    const Geo g = a.g;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    vel_cell<PREC>(a, k, i, j);
}

// ---------------------------------------------------------------------------
// stress: kernel__update_stress (m_kernel.f90:142-326) +
//         absorb_p__update_stress (m_absorb_p.f90:424-503)
// ---------------------------------------------------------------------------
template <int NM, int MINB, int PREC>
__global__ void __launch_bounds__(256, MINB) stress3d_kernel(const Str3Args a) {
    const Geo g = a.g;
    const int k = 1 + blockIdx.x * 32 + threadIdx.x;
    const int i = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int j = 1 + blockIdx.z * blockDim.z + threadIdx.z;
    if (k > g.nz || i > g.nx || j > g.ny) return;
    stress_cell<NM, PREC>(a, k, i, j);
}

// MINB (minimum resident blocks per SM) trades registers for occupancy; the
// launch table picks it per kernel (swpc_set_launch)
template <int PREC>
static void vel_minb(const Vel3Args &a, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (minb) {
    case 1: vel3d_kernel<1, PREC><<<grid, block, 0, st>>>(a); break;
    case 2: vel3d_kernel<2, PREC><<<grid, block, 0, st>>>(a); break;
    case 3: vel3d_kernel<3, PREC><<<grid, block, 0, st>>>(a); break;
    default: vel3d_kernel<4, PREC><<<grid, block, 0, st>>>(a); break;
    }
}

void launch_vel3d(const Vel3Args &a, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st) {
    // S is read in FP16 only by the PREC_F16_SR form; the others share the FP32 kernel
    if (prec == PREC_F16_SR) vel_minb<PREC_F16_SR>(a, minb, grid, block, st);
    else vel_minb<PREC_F32>(a, minb, grid, block, st);
}

template <int NM, int PREC>
static void stress_minb(const Str3Args &a, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (minb) {
    case 1: stress3d_kernel<NM, 1, PREC><<<grid, block, 0, st>>>(a); break;
    case 2: stress3d_kernel<NM, 2, PREC><<<grid, block, 0, st>>>(a); break;
    case 3: stress3d_kernel<NM, 3, PREC><<<grid, block, 0, st>>>(a); break;
    default: stress3d_kernel<NM, 4, PREC><<<grid, block, 0, st>>>(a); break;
    }
}

template <int PREC>
static void stress_nm(const Str3Args &a, int nm, int minb, dim3 grid, dim3 block, cudaStream_t st) {
    switch (nm) {
    case 0: stress_minb<0, PREC>(a, minb, grid, block, st); break;
    case 1: stress_minb<1, PREC>(a, minb, grid, block, st); break;
    case 2: stress_minb<2, PREC>(a, minb, grid, block, st); break;
    default: stress_minb<3, PREC>(a, minb, grid, block, st); break;
    }
}

void launch_stress3d(const Str3Args &a, int nm, int minb, int prec, dim3 grid, dim3 block, cudaStream_t st) {
    switch (prec) {
    case PREC_BF16_R: stress_nm<PREC_BF16_R>(a, nm, minb, grid, block, st); break;
    case PREC_F16_SR: stress_nm<PREC_F16_SR>(a, nm, minb, grid, block, st); break;
    case PREC_F16_R: stress_nm<PREC_F16_R>(a, nm, minb, grid, block, st); break;
    default: stress_nm<PREC_F32>(a, nm, minb, grid, block, st); break;
    }
}

// ---------------------------------------------------------------------------
// point sources: source__stressglut (m_source.f90:798-826),
// source__bodyforce (:854-870), green__source (m_green.f90:615-627).
// Entries are applied in list order; when no two entries touch the same
// cell the host marks the list parallel and each entry gets a thread.
// ---------------------------------------------------------------------------
// S -= coef * sdrop / div on an FP16 stress array (SWPC_PREC_F16_SR)
__device__ __forceinline__ void glut_half(const InjArgs &a, const InjEntry &en, float sdrop, int div) {
    __half *h = reinterpret_cast<__half *>(a.fields[en.field]);
    const int c = en.field - SWPC_F_SXX;
    const float v = __half2float(h[en.cell]) * sc_sS(a.scale, c);
    const float w = div == 1 ? v - en.coef * sdrop : v - en.coef * sdrop / div;
    h[en.cell] = __float2half_rn(w * sc_iS(a.scale, c));
}

__device__ __forceinline__ void apply_entry(const InjArgs &a, const InjEntry &en, int it) {
    float *f = a.fields[en.field];
    const float st = a.stime[(long long)(it - 1) * a.nsrc + en.src];
    if (a.s_half && en.field >= SWPC_F_SXX && en.mode <= INJ_GLUT2) {
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        glut_half(a, en, sdrop, en.mode == INJ_GLUT ? 1 : (en.mode == INJ_GLUT4 ? 4 : 2));
        return;
    }
    switch (en.mode) {
    case INJ_GLUT: {        // S -= m * sdrop, sdrop = mo * stime * dt_dxyz
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop;
        break;
    }
    case INJ_GLUT4: {       // S -= m * sdrop / 4 (3D and P-SV shear cells)
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop / 4;
        break;
    }
    case INJ_GLUT2: {       // S -= m * sdrop / 2 (SH, src/swpc_sh/m_source.f90:583-587)
        const float sdrop = a.mo[en.src] * st * a.dt_dxyz;
        f[en.cell] = f[en.cell] - en.coef * sdrop / 2;
        break;
    }
    case INJ_BF3: {         // V += b * f * stime * dt_dxyz / 2 (m_source.f90:863-868)
        const float b = a.bfields[en.bfield][en.cell];
        f[en.cell] = f[en.cell] + b * en.coef * st * a.dt_dxyz / 2;
        break;
    }
    case INJ_GREEN: {       // fx = fx1 * dt_dxyz * stf ; V += b * fx / 2 (m_green.f90:617-627)
        const float fv = en.coef * a.dt_dxyz * st;
        const float b = a.bfields[en.bfield][en.cell];
        f[en.cell] = f[en.cell] + b * fv / 2;
        break;
    }
    case INJ_BFPSV: {       // V += f / rho(kk,ii) * stime * dt_dxz / 2 (src/swpc_psv/m_source.f90:640-645)
        const float rho = a.bfields[0][a.rho_cell[en.src]];
        f[en.cell] = f[en.cell] + en.coef / rho * st * a.dt_dxyz / 2;
        break;
    }
    case INJ_BFSH: {        // Vy += f / rho(kk,ii) * stime * dt_dxz (src/swpc_sh/m_source.f90:621)
        const float rho = a.bfields[0][a.rho_cell[en.src]];
        f[en.cell] = f[en.cell] + en.coef / rho * st * a.dt_dxyz;
        break;
    }
    default: break;
    }
}

__global__ void inject_kernel(const InjArgs a) {
    const int it = a.d_it ? *a.d_it : a.it;
    if (it < 1 || it > a.nt) return;
    if (a.serial) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (int n = 0; n < a.n; n++) apply_entry(a, a.list[n], it);
        return;
    }
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < a.n) apply_entry(a, a.list[n], it);
}

// many injection lists in one launch (batched ensembles): blockIdx.y picks
// the list; each list keeps its own serial / parallel mode
__global__ void inject_multi_kernel(const InjArgs *__restrict__ list, int nlist, const int *d_it, int it_arg) {
    const int it = d_it ? *d_it : it_arg;
    for (int b = blockIdx.y; b < nlist; b += gridDim.y) {
        const InjArgs &a = list[b];
        if (it < 1 || it > a.nt) continue;
        if (a.serial) {
            if (blockIdx.x == 0 && threadIdx.x == 0)
                for (int n = 0; n < a.n; n++) apply_entry(a, a.list[n], it);
            continue;
        }
        for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.n; n += gridDim.x * blockDim.x)
            apply_entry(a, a.list[n], it);
    }
}

void launch_inject_multi(const InjArgs *list, int nlist, int max_n, const int *d_it, int it, cudaStream_t st) {
    if (!list || nlist <= 0 || max_n <= 0) return;
    const int threads = 128;
    const dim3 grid((max_n + threads - 1) / threads, nlist < 65535 ? nlist : 65535);
    inject_multi_kernel<<<grid, threads, 0, st>>>(list, nlist, d_it, it);
}

void launch_inject(const InjArgs &a, cudaStream_t st) {
    if (a.n <= 0) return;
    const int threads = 128;
    const int blocks = a.serial ? 1 : (a.n + threads - 1) / threads;
    inject_kernel<<<blocks, threads, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// wav__store (m_wav.f90:433-620): one thread per station
// ---------------------------------------------------------------------------
__global__ void wav3d_kernel(const Wav3Args a) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.nst) return;
    wav_station(a, n);
}

void launch_wav3d(const Wav3Args &a, cudaStream_t st) {
    if (a.nst <= 0) return;
    const int threads = 128;
    wav3d_kernel<<<(a.nst + threads - 1) / threads, threads, 0, st>>>(a);
}

// ---------------------------------------------------------------------------
// kernel__vmax (m_kernel.f90:328-352): max |V(kob+1, i, j)|; |x| of a finite
// float orders like its bit pattern, so the max is an atomicMax on the bits.
// ---------------------------------------------------------------------------
__global__ void vmax3d_kernel(const VmaxArgs a) {
    const int ni = a.i1 - a.i0 + 1, nj = a.j1 - a.j0 + 1;
    const long long n = (long long)ni * nj;
    unsigned int mx = 0, my = 0, mz = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = a.i0 + (int)(t % ni), j = a.j0 + (int)(t / ni);
        const long long col = col_index(a.g, i, j);
        const int k = a.kob[col] + 1;
        const long long e = col * a.g.Kp + (k - 1 + KH);
        const unsigned int bx = __float_as_uint(fabsf(a.Vx[e]));
        const unsigned int by = __float_as_uint(fabsf(a.Vy[e]));
        const unsigned int bz = __float_as_uint(fabsf(a.Vz[e]));
        mx = max(mx, bx);
        my = max(my, by);
        mz = max(mz, bz);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        my = max(my, __shfl_xor_sync(0xffffffffu, my, o));
        mz = max(mz, __shfl_xor_sync(0xffffffffu, mz, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&a.out[0], mx);
        atomicMax(&a.out[1], my);
        atomicMax(&a.out[2], mz);
    }
}

void launch_vmax3d(const VmaxArgs &a, cudaStream_t st) {
    vmax3d_kernel<<<148, 256, 0, st>>>(a);
}

__global__ void advance_it_kernel(int *d_it) { *d_it = *d_it + 1; }
void launch_advance_it(int *d_it, cudaStream_t st) { advance_it_kernel<<<1, 1, 0, st>>>(d_it); }

}  // namespace swpc
