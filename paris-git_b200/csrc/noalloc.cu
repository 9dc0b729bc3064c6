// noalloc.cu -- calcResiduals (modules.f90:3313-3387) for callers that must
// not allocate device memory: a driver whose device memory is entirely owned
// by its own pool or by another runtime (for instance Fortran arrays placed on
// the device by a different toolchain), or one that runs under a fixed memory
// budget where a cudaMalloc in the time loop could fail, fragment the pool or
// synchronise the device.  The caller passes A and p already on the device;
// the only scratch is the per-block partial sums below, a file-scope device
// array that every GPU loading this library holds until the process exits.
//
// Limits and sharing:
//  - one block of kNaThreads threads per kNaThreads interior cells, so at most
//    kNaMaxCells = 16,777,216 interior cells (256^3); larger grids are rejected;
//  - every call on a device shares g_na_part / g_na_out and leaves its sums
//    there; each call overwrites every slot it reads, so nothing needs to be
//    cleared, but calls whose kernels overlap on the GPU race on the arrays;
//  - every call looks up the device addresses of the arrays for the current
//    device and context (cudaGetSymbolAddress, which allocates nothing), so a
//    device reset or another context is followed; with lazy module loading
//    (the CUDA default) the first call on a device may load this module and
//    place the arrays at that moment, so make a first call at set-up time;
//  - all cells count, as calcResiduals with ExcludeBoundCellCalcRes = F (the
//    reference's default); the variant that skips the cells next to walls
//    (modules.f90:3347-3359) is not provided.
#include "ctx.cuh"

static constexpr int kNaThreads = 256;
static constexpr long kNaMaxBlocks = 65536;
static constexpr long kNaMaxCells = kNaThreads * kNaMaxBlocks;

static __device__ __align__(256) double g_na_part[3 * kNaMaxBlocks];   // 1.5 MiB
static __device__ __align__(256) double g_na_out[3];

// |r| of every interior cell, one cell per thread; block sums of |r|, r^2, max|r|
__global__ void __launch_bounds__(kNaThreads) k_na_residuals(const double* __restrict__ A, const double* __restrict__ p,
                                                            int nx, int ny, int nz, int ng, double* __restrict__ part,
                                                            long nblocks) {
    __shared__ double sh[32];
    long N = (long)nx * ny * nz;
    long m = blockIdx.x * (long)kNaThreads + threadIdx.x;
    double s1 = 0.0, s2 = 0.0, smax = 0.0;
    if (m < N) {
        int i = (int)(m % nx), j = (int)((m / nx) % ny), k = (int)(m / ((long)nx * ny));
        long sy = nx + 2 * ng, sz = (long)sy * (ny + 2 * ng);
        long n = (i + ng) + sy * (j + ng) + sz * (k + ng);
        double r = fabs(-p[n] * A[6 * N + m] + A[0 * N + m] * p[n - 1] + A[1 * N + m] * p[n + 1] +
                        A[2 * N + m] * p[n - sy] + A[3 * N + m] * p[n + sy] + A[4 * N + m] * p[n - sz] +
                        A[5 * N + m] * p[n + sz] + A[7 * N + m]);
        s1 = r;
        s2 = r * r;
        smax = r;
    }
    s1 = block_sum<kNaThreads>(s1, sh);
    s2 = block_sum<kNaThreads>(s2, sh);
    smax = block_max<kNaThreads>(smax, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s1;
        part[nblocks + blockIdx.x] = s2;
        part[2 * nblocks + blockIdx.x] = smax;
    }
}

// slot s of the partials -> out[s] (sum for slots 0,1, max for slot 2)
__global__ void k_na_finish(const double* __restrict__ part, long nblocks, double* __restrict__ out) {
    __shared__ double sh[32];
    int slot = blockIdx.x;
    double v = 0.0;
    for (long b = threadIdx.x; b < nblocks; b += blockDim.x) {
        double x = part[slot * nblocks + b];
        v = slot == 2 ? fmax(v, x) : v + x;
    }
    v = slot == 2 ? block_max<256>(v, sh) : block_sum<256>(v, sh);
    if (threadIdx.x == 0) out[slot] = v;
}

// Device addresses of the scratch arrays in the current device's context.
static int na_scratch(double** part, double** out) {
    void* pp = nullptr;
    void* po = nullptr;
    if (cudaGetSymbolAddress(&pp, g_na_part) != cudaSuccess) return PARIS_CUDA_ERROR;
    if (cudaGetSymbolAddress(&po, g_na_out) != cudaSuccess) return PARIS_CUDA_ERROR;
    *part = (double*)pp;
    *out = (double*)po;
    return PARIS_OK;
}

extern "C" int paris_calc_residuals_noalloc(int32_t nx, int32_t ny, int32_t nz, int32_t ng, const double* A_dev,
                                            const double* p_dev, double* out3, void* stream) {
    if (!A_dev || !p_dev || !out3 || nx < 1 || ny < 1 || nz < 1 || ng < 1) return PARIS_BAD_ARGS;
    long N = (long)nx * ny * nz;
    if (N > kNaMaxCells) return PARIS_BAD_ARGS;   // scratch holds kNaMaxBlocks partial sums
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PARIS_NO_DEVICE;
    double* part = nullptr;
    double* dout = nullptr;
    int st = na_scratch(&part, &dout);
    if (st != PARIS_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    long nblocks = (N + kNaThreads - 1) / kNaThreads;
    k_na_residuals<<<(unsigned)nblocks, kNaThreads, 0, s>>>(A_dev, p_dev, nx, ny, nz, ng, part, nblocks);
    if (cudaGetLastError() != cudaSuccess) return PARIS_CUDA_ERROR;
    k_na_finish<<<3, 256, 0, s>>>(part, nblocks, dout);
    if (cudaGetLastError() != cudaSuccess) return PARIS_CUDA_ERROR;
    double sums[3];
    if (cudaMemcpyAsync(sums, dout, sizeof(sums), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PARIS_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PARIS_CUDA_ERROR;
    out3[0] = sums[0] / (double)nx / (double)ny / (double)nz;
    out3[1] = sqrt(sums[1] / (double)nx / (double)ny / (double)nz);
    out3[2] = sums[2];
    return PARIS_OK;
}
