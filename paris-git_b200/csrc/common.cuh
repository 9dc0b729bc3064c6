// common.cuh -- device layout, boundary rules and launch helpers shared by the
// kernels of the PARIS grid core on B200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include "../../include/paris_b200.h"

// ---------------------------------------------------------------------------
// Field layout in HBM: exactly the reference's array
// F(imin:imax,jmin:jmax,kmin:kmax) with Ng ghost layers, i fastest, so a
// Fortran array moves to and from the device as one contiguous copy.
//   elem(i,j,k) = base[off + i + pitch*j + plane*k], i,j,k interior-relative
//   (-Ng .. N+Ng-1).
// ---------------------------------------------------------------------------
struct Layout {
    int n[3];      // interior cells
    int ng;
    long pitch;    // elements per row (Nx + 2 Ng)
    long plane;    // elements per plane
    long off;      // offset of interior (0,0,0)
    long total;    // elements of the array
};

inline Layout make_layout(int nx, int ny, int nz, int ng) {
    Layout L;
    L.n[0] = nx; L.n[1] = ny; L.n[2] = nz; L.ng = ng;
    L.pitch = nx + 2 * ng;
    L.plane = L.pitch * (ny + 2 * ng);
    L.off = ng + L.pitch * ng + L.plane * ng;
    L.total = L.plane * (nz + 2 * ng);
    return L;
}

__host__ __device__ inline long lidx(const Layout& L, int i, int j, int k) {
    return L.off + i + L.pitch * (long)j + L.plane * (long)k;
}

// Boundary description handed to kernels by value.
struct Bnd {
    int per[3];       // 1: periodic in direction d
    int wall_lo[3];   // face mask 0 on the low wall face (bdry_cond 0 or 2)
    int wall_hi[3];
    int vofbc[6];     // vofbdry_cond
};

// ---- ghost cells ---------------------------------------------------------
// Enumerates the ghost cells of a ghosted field in three disjoint regions
// (x-slabs over all j,k; y-slabs over interior i, all k; z-slabs over interior
// i,j).  A ghost cell copies the cell obtained by wrapping its out-of-range
// periodic coordinates; walls are left untouched.  This equals ghost_x, then
// ghost_y, then ghost_z of modules.f90:1821-1970 on one rank.
__host__ __device__ inline bool ghost_cell(const Layout L, long t, int& i, int& j, int& k) {
    const int g = L.ng;
    const int tx = L.n[0] + 2 * g, ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
    long rx = 2L * g * ty * tz, ry = (long)L.n[0] * 2 * g * tz, rz = (long)L.n[0] * L.n[1] * 2 * g;
    if (t < rx) {
        int a = (int)(t % (2 * g)); long r = t / (2 * g);
        j = (int)(r % ty) - g; k = (int)(r / ty) - g;
        i = a < g ? a - g : L.n[0] + (a - g);
        return true;
    }
    t -= rx;
    if (t < ry) {
        i = (int)(t % L.n[0]); long r = t / L.n[0];
        int a = (int)(r % (2 * g)); k = (int)(r / (2 * g)) - g;
        j = a < g ? a - g : L.n[1] + (a - g);
        return true;
    }
    t -= ry;
    if (t < rz) {
        i = (int)(t % L.n[0]); long r = t / L.n[0];
        j = (int)(r % L.n[1]); int a = (int)(r / L.n[1]);
        k = a < g ? a - g : L.n[2] + (a - g);
        return true;
    }
    (void)tx;
    return false;
}

__host__ __device__ inline long ghost_count(const Layout& L) {
    const int g = L.ng;
    long ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
    return 2L * g * ty * tz + (long)L.n[0] * 2 * g * tz + (long)L.n[0] * L.n[1] * 2 * g;
}

// Compact interior-only index (MG levels, matrix A).
__host__ __device__ inline long cidx(int nx, int ny, int i, int j, int k) {
    return i + (long)nx * (j + (long)ny * k);
}

// Error reporting from the C++ side.
struct paris_ctx;
void ctx_set_error(paris_ctx* c, const char* fmt, ...);

#define PARIS_CUDA_TRY(ctx, expr)                                                   \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) {                                                    \
            ctx_set_error((ctx), "%s failed: %s (%s:%d)", #expr,                    \
                          cudaGetErrorString(_e), __FILE__, __LINE__);              \
            return PARIS_CUDA_ERROR;                                                \
        }                                                                           \
    } while (0)

// Optional per-kernel CUDA-event timing (paris_gpu_profile).
void prof_begin(paris_ctx* c, const char* name, long cells);
void prof_end(paris_ctx* c);
int prof_enabled(const paris_ctx* c);

// Launch with bookkeeping: counts every kernel the handle issues and checks
// the launch; `name` and `cells` label the launch in the profile.  Use inside
// functions returning int.
#define PARIS_LAUNCH_N(ctx, name, cells, kernel, grid, block, smem, ...)            \
    do {                                                                            \
        bool _prof = prof_enabled(ctx);                                             \
        if (_prof) prof_begin((ctx), (name), (cells));                              \
        kernel<<<(grid), (block), (smem), (ctx)->stream>>>(__VA_ARGS__);            \
        if (_prof) prof_end(ctx);                                                   \
        (ctx)->launches++;                                                          \
        cudaError_t _e = cudaGetLastError();                                        \
        if (_e != cudaSuccess) {                                                    \
            ctx_set_error((ctx), "launch of %s failed: %s", #kernel,                \
                          cudaGetErrorString(_e));                                  \
            return PARIS_CUDA_ERROR;                                                \
        }                                                                           \
    } while (0)

#define PARIS_LAUNCH(ctx, kernel, grid, block, smem, ...) \
    PARIS_LAUNCH_N(ctx, #kernel, 0L, kernel, grid, block, smem, __VA_ARGS__)

#define PARIS_CHECK(expr)                       \
    do {                                        \
        int _s = (expr);                        \
        if (_s != PARIS_OK) return _s;          \
    } while (0)

inline unsigned div_up(long a, long b) { return (unsigned)((a + b - 1) / b); }

// Deterministic block reduction of a double (fixed tree order).
__device__ inline int linear_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }

template <int BLOCK>
__device__ inline double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int tid = linear_tid();
    int lane = tid & 31, w = tid >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = lane < BLOCK / 32 ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;   // valid in the first thread
}

template <int BLOCK>
__device__ inline double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int tid = linear_tid();
    int lane = tid & 31, w = tid >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = lane < BLOCK / 32 ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

// Loops over the interior cells of an n0 x n1 x n2 box with blocks of
// (bx, by) threads: threadIdx.x runs along i, (blockIdx.x, threadIdx.y) over
// the rows (j,k) with a grid stride; no 64-bit divisions per cell.
#define ROWS_BEGIN(n0, n1, n2)                                                             \
    for (int _row = blockIdx.x * blockDim.y + threadIdx.y; _row < (n1) * (n2);             \
         _row += gridDim.x * blockDim.y) {                                                 \
        const int j = _row % (n1), k = _row / (n1);                                        \
        for (int i = threadIdx.x; i < (n0); i += blockDim.x) {
#define ROWS_END \
        }        \
    }
static const dim3 kRowBlock(128, 2, 1);
