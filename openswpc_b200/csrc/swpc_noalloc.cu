// swpc_noalloc.cu -- the report maximum (kernel__vmax) for callers that own
// their wavefield and may not allocate device memory.
//
// Who calls this: a solver that keeps Vx, Vy, Vz and the ocean-bottom map in
// device arrays of its own -- an OpenACC build of the reference holds them
// resident through `!$acc enter data` for the whole run -- and that runs with
// its device memory claimed up front.  Such a caller has no swpc_ctx (whose
// creation allocates) and must not have a library allocate behind its back:
// cudaMalloc can fail once the memory is claimed, and cudaFree waits for the
// whole device, which would stall the time loop at every report.  This entry
// point therefore allocates nothing.  Its scratch is one fixed array in the
// library's own device data, which every GPU that loads the library holds
// until the process exits.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/swpc_gpu.h"

namespace {

constexpr int kMaxNy = SWPC_NOALLOC_MAX_NY;
constexpr int kResult = 3 * kMaxNy;   // first word of the 3-word result
constexpr int kWords = kResult + 64;  // row partials, result, padding to 256 B
constexpr int kThreads = 256;

// Scratch shared by every call on a device: 3 words (max |vx|, |vy|, |vz| as
// float bits) per row j of the reduced range, then the 3 result words.
// Neither part needs clearing between calls: pass 1 writes every row word
// that pass 2 reads, and pass 2 writes all three result words.  In host code
// `vmax_scratch` only names the symbol; its device address comes from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned int vmax_scratch[kWords];

// Device address of the scratch array on the current device.  It is looked
// up on every call rather than cached: after a cudaDeviceReset (or any new
// primary context) the array lives at a new address, and a cached one would
// send the kernels to memory that is no longer mapped.  The lookup allocates
// nothing and costs little once the module is loaded.
cudaError_t scratch_for(unsigned int **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, vmax_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<unsigned int *>(p);
    return cudaSuccess;
}

struct NoallocArgs {
    const float *vx, *vy, *vz;
    const int *kob;
    long long ld_k, ld_i;   // leading extents of the memory box (>= nz + 6, nx + 6)
    int nz, i0, i1, j0, nrows;
};

__device__ __forceinline__ unsigned int block_max(unsigned int v, unsigned int *sh) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    v = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0u;
    if (w == 0)
        for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    return v;
}

// Pass 1: one block per row j, max over i of |V| at k = kob(i,j) + 1.  The
// comparison is on the bit patterns of |V|, which order like the values (a
// NaN sorts above every number and so reaches the divergence check).
__global__ void __launch_bounds__(kThreads) vmax_rows_kernel(NoallocArgs a, unsigned int *scratch) {
    __shared__ unsigned int sh[kThreads / 32];
    for (int r = blockIdx.x; r < a.nrows; r += gridDim.x) {
        const int j = a.j0 + r;
        unsigned int mx = 0, my = 0, mz = 0;
        for (int i = a.i0 + threadIdx.x; i <= a.i1; i += blockDim.x) {
            const long long col = (long long)(j + 2) * a.ld_i + (i + 2);
            const int k = a.kob[col] + 1;
            if (k < -2 || k > a.nz + 3) continue;   // outside the memory box
            const long long e = col * a.ld_k + (k + 2);
            mx = max(mx, __float_as_uint(fabsf(a.vx[e])));
            my = max(my, __float_as_uint(fabsf(a.vy[e])));
            mz = max(mz, __float_as_uint(fabsf(a.vz[e])));
        }
        mx = block_max(mx, sh);
        my = block_max(my, sh);
        mz = block_max(mz, sh);
        if (threadIdx.x == 0) {
            scratch[3 * r + 0] = mx;
            scratch[3 * r + 1] = my;
            scratch[3 * r + 2] = mz;
        }
    }
}

// Pass 2: one block folds the row partials into the result words.
__global__ void __launch_bounds__(kThreads) vmax_fold_kernel(int nrows, unsigned int *scratch) {
    __shared__ unsigned int sh[kThreads / 32];
    unsigned int m[3] = {0u, 0u, 0u};
    for (int r = threadIdx.x; r < nrows; r += blockDim.x)
        for (int c = 0; c < 3; c++) m[c] = max(m[c], scratch[3 * r + c]);
    for (int c = 0; c < 3; c++) {
        const unsigned int v = block_max(m[c], sh);
        if (threadIdx.x == 0) scratch[kResult + c] = v;
    }
}

}  // namespace

extern "C" int swpc_vmax_noalloc(const float *vx, const float *vy, const float *vz, const int *kob, int nx, int ny,
                                 int nz, int na, int ld_k, int ld_i, float uc, void *stream, float out[3]) {
    if (!vx || !vy || !vz || !kob || !out) return SWPC_ERR_ARG;
    if (nx < 1 || ny < 1 || nz < 1 || na < 0 || ld_k < nz + 6 || ld_i < nx + 6) return SWPC_ERR_ARG;
    if (ny > kMaxNy) return SWPC_ERR_LIMIT;
    unsigned int *scratch = nullptr;
    if (scratch_for(&scratch) != cudaSuccess) return SWPC_ERR_CUDA;

    // range of kernel__vmax on a single node (m_kernel.f90:343-344)
    const int margin = 5;
    NoallocArgs a;
    a.vx = vx; a.vy = vy; a.vz = vz; a.kob = kob;
    a.ld_k = ld_k;
    a.ld_i = ld_i;
    a.nz = nz;
    a.i0 = na + margin + 1 > 1 ? na + margin + 1 : 1;
    a.i1 = nx - na - margin < nx ? nx - na - margin : nx;
    a.j0 = na + margin + 1 > 1 ? na + margin + 1 : 1;
    const int j1 = ny - na - margin < ny ? ny - na - margin : ny;
    a.nrows = (j1 >= a.j0 && a.i1 >= a.i0) ? j1 - a.j0 + 1 : 0;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (a.nrows > 0) {
        const int blocks = a.nrows < 148 * 8 ? a.nrows : 148 * 8;
        vmax_rows_kernel<<<blocks, kThreads, 0, st>>>(a, scratch);
    }
    vmax_fold_kernel<<<1, kThreads, 0, st>>>(a.nrows, scratch);
    if (cudaGetLastError() != cudaSuccess) return SWPC_ERR_CUDA;
    unsigned int bits[3];
    if (cudaMemcpyAsync(bits, scratch + kResult, sizeof(bits), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return SWPC_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SWPC_ERR_CUDA;
    std::memcpy(out, bits, sizeof(bits));
    float mx = out[0] > out[1] ? out[0] : out[1];
    mx = mx > out[2] ? mx : out[2];
    if (out[0] != out[0] || out[1] != out[1] || out[2] != out[2] || !(mx * uc <= 1e5f)) return SWPC_ERR_DIVERGED;
    return SWPC_OK;
}
