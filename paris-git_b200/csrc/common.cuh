// common.cuh -- device layout, boundary rules and launch helpers shared by the
// kernels of the PARIS grid core on B200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include "../../include/paris_b200.h"

// ---------------------------------------------------------------------------
// Field layout in HBM.  A field with ghost layers keeps the reference's shape
// (Nx+2Ng)(Ny+2Ng)(Nz+2Ng), i fastest, but each x-row is padded so that the
// first interior cell of every row sits on a 128-byte boundary:
//   row  = [pad | Ng ghosts | Nx interior | Ng ghosts | pad]
//   elem(i,j,k) = base[off + i + pitch*j + plane*k], i,j,k interior-relative
//   (-Ng .. N+Ng-1).
// ---------------------------------------------------------------------------
struct Layout {
    int n[3];      // interior cells
    int ng;
    long pitch;    // elements per row
    long plane;    // elements per plane
    long off;      // offset of interior (0,0,0)
    long total;    // elements to allocate
};

static constexpr int kRowLead = 16;   // elements before interior i = 0

inline Layout make_layout(int nx, int ny, int nz, int ng) {
    Layout L;
    L.n[0] = nx; L.n[1] = ny; L.n[2] = nz; L.ng = ng;
    long need = kRowLead + nx + ng;
    L.pitch = (need + 15) / 16 * 16;
    L.plane = L.pitch * (ny + 2 * ng);
    L.off = kRowLead + L.pitch * ng + L.plane * ng;
    L.total = L.plane * (nz + 2 * ng) + 16;
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
template <int BLOCK>
__device__ inline double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = lane < BLOCK / 32 ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;   // valid in thread 0
}

template <int BLOCK>
__device__ inline double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
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
