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

// The inflow of a 'jet' VOF condition (x- face): inject(j,k) of SetVOFBC,
// vofmodules.f90:1797-1811, from the cell centres y(j), z(k).
struct VofJet {
    int type;                  // inject_type
    double yc, zc, rliq, rgas; // jetcenter_yc, jetcenter_zc, radius_liq_inject, radius_gas_inject
    const double* y;           // cell centres, ghosted index j + Ng
    const double* z;
};

__device__ inline int vof_inject(const VofJet& J, int ng, int j, int k) {
    const double yy = J.y[j + ng] - J.yc, zz = J.z[k + ng] - J.zc;
    if (J.type == 2 || J.type == 4) return yy * yy + zz * zz < J.rliq * J.rliq ? 1 : 0;
    if (J.type == 3) return yy <= J.rliq ? 1 : 0;
    if (J.type == 5) return (yy > J.rgas && yy < J.rliq) ? 1 : 0;
    return 0;
}

// SetVOFBC (vofmodules.f90:1694-1825) at ghost cell (i,j,k), together with the
// periodic wrap of do_all_ghost.  The orientations x- y- z- x+ y+ z+ write in
// that order, so the cell's value is found walking them backwards: the last
// one that writes the cell decides it.  'dry'/'wet' (both layers) and 'jet'
// (first layer at x-) fix the value; 'outflow' (both layers) and '90deg'
// (first layer) copy the adjacent cell as it stood after the orientations
// before them, so the walk continues from that cell.
//   SWEEP = true: swp's order, SetVOFBC then the wrap, which wins wherever the
//   velocity is periodic.  SWEEP = false: initconditions_VOF's order, the wrap
//   then SetVOFBC, which wins on every face whose VOF condition is not
//   periodic.
// Returns true with v set when a condition fixes the value.  Otherwise the
// ghost takes the value of cell s: an interior cell, or a ghost cell that no
// orientation writes (the second layer of a 'jet' or '90deg' face), which
// keeps the value it held.
template <bool SWEEP>
__device__ inline bool vof_ghost_rule(const Layout& L, const Bnd& B, const VofJet& J, int i, int j, int k, int s[3],
                                      double& v) {
    const int gc[3] = {i, j, k};
    s[0] = i; s[1] = j; s[2] = k;
    for (int d = 0; d < 3; d++)
        if (B.per[d]) {
            if (s[d] < 0) s[d] += L.n[d];
            else if (s[d] >= L.n[d]) s[d] -= L.n[d];
        }
    for (int o = 5; o >= 0; o--) {
        const int d = o % 3;
        const bool lo = o < 3;
        const int cond = B.vofbc[o];
        if (SWEEP ? B.per[d] != 0 : cond == PARIS_VOFBC_PERIODIC) continue;
        const int a = SWEEP ? s[d] : gc[d];
        const bool out = lo ? a < 0 : a >= L.n[d];
        if (!out) continue;
        const bool first = lo ? a == -1 : a == L.n[d];
        if (cond == PARIS_VOFBC_DRY || cond == PARIS_VOFBC_WET) {
            v = cond == PARIS_VOFBC_WET ? 1.0 : 0.0;
            return true;
        }
        if (cond == PARIS_VOFBC_JET) {
            if (!first) continue;
            v = (double)vof_inject(J, L.ng, s[1], s[2]);
            return true;
        }
        if (cond == PARIS_VOFBC_90DEG && !first) continue;
        s[d] = lo ? 0 : L.n[d] - 1;   // outflow, or the first layer of 90deg
    }
    return false;
}

__device__ inline bool vof_interior(const Layout& L, const int s[3]) {
    return s[0] >= 0 && s[0] < L.n[0] && s[1] >= 0 && s[1] < L.n[1] && s[2] >= 0 && s[2] < L.n[2];
}

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
