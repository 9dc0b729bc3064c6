// vof.cu -- split PLIC VOF advection on the B200: vofsweeps
// (vofmodules.f90:1340-1361) with swp (vofnonmodule.f90:27-48), the CIAM sweep
// swpz (:126-237) and the Weymouth-Yue sweep swpr (:664-754), the flags and
// clipping of get_flags_and_clip (vofmodules.f90:549-571), SetVOFBC
// (:1694-1825), linfunc (:171-218) and the sphere initialisation
// ls2vof_refined (:1195-1293).  Built with -fmad=false.
//
// Three kernels per split direction:
//  1. the mixed flux cells (0 < c < 1) as one dense list: each block of 1024
//     flux cells counts its mixed cells, takes room for them with a single
//     atomic add, and writes them there;
//  2. the PLIC fluxes of the listed cells, every lane a listed cell (so that
//     the geometry runs without divergence against the full and empty
//     cells), stored in sparse flux arrays;
//  3. the update: the new, clipped volume fraction and its flag from the
//     fluxes of each cell and its two neighbours along the sweep (closed form
//     for full cells, the stored fluxes for mixed ones), into the second
//     buffer, reading cvof and the face velocity once.
// A ghost kernel then applies SetVOFBC and the periodic wrap.  On a uniform
// grid whose spacing is a power of two, the divisions a = u dt / dxh are
// multiplications by the exact reciprocal, which round to the same double.
#include "ctx.cuh"
#include "plic.cuh"

struct SweepArgs {
    const double* c;     // old cvof (ghosted)
    double* cn;          // new cvof (ghosted)
    int8_t* flag;        // new flags
    const double* us;    // face velocity of the sweep direction
    const uint8_t* cg;   // c_mask (WY)
    double *v1, *v2, *v3;   // fluxes of the mixed cells (ghosted arrays, sparse)
    long* list;          // layout indices of the mixed flux cells
    int* count;          // their number
    long cap;            // room in the list
    Layout L;
    int d;               // 0,1,2
    int wy;              // 1: swpr
    double dt, dxyz;     // a = us*dt/dxyz with dxyz = dxh(is) (vofnonmodule.f90:140,682)
    double rdxyz;        // 1/dxyz when dxyz is a power of two (exact), else 0
    double epsc;
};

static constexpr int kVofListThreads = 256;
static constexpr int kVofPer = 4;                               // flux cells per thread of the list kernel
static constexpr int kVofSeg = kVofListThreads * kVofPer;       // flux cells per block of the list kernel

// a = u dt / dxyz, the Courant number of a face (vofnonmodule.f90:147-148,
// 686-687): the same double as the division when 1/dxyz is exact
__device__ inline double courant(const SweepArgs& a, double u) {
    return a.rdxyz != 0.0 ? u * a.dt * a.rdxyz : u * a.dt / a.dxyz;
}

// The flux cells of a sweep along d are the interior in the other two
// directions and -1..n along d (vofnonmodule.f90:143-145 loops over is-1..ie+1;
// only the d-neighbours of interior cells are used); flat index t over them,
// i fastest.
__device__ inline void flux_cell_of(const SweepArgs& a, unsigned t, int& i, int& j, int& k) {
    const unsigned e0 = a.L.n[0] + (a.d == 0 ? 2 : 0), e1 = a.L.n[1] + (a.d == 1 ? 2 : 0);
    const unsigned r = t / e0;
    i = (int)(t - r * e0);
    k = (int)(r / e1);
    j = (int)(r - (unsigned)k * e1);
    if (a.d == 0) i -= 1; else if (a.d == 1) j -= 1; else k -= 1;
}

// 1. the mixed flux cells, kVofSeg per block; each thread loads its kVofPer
// cells (strided by the block size, so the loads coalesce) before testing
// them, and the block appends its mixed cells with one atomic add.  A
// thread divides only for its first cell and steps the others on by the
// block size; the per-(cell slot, warp) counts are scanned by one warp.
static_assert(kVofPer * (kVofListThreads / 32) == 32, "one count per lane of the scanning warp");
__global__ void __launch_bounds__(kVofListThreads) k_vof_mixed_list(const SweepArgs a, unsigned F) {
    __shared__ int wcount[kVofPer * (kVofListThreads / 32)];
    __shared__ int wbase[kVofPer * (kVofListThreads / 32)];
    __shared__ int total, room;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int e0 = a.L.n[0] + (a.d == 0 ? 2 : 0), e1 = a.L.n[1] + (a.d == 1 ? 2 : 0);
    const unsigned t0 = blockIdx.x * (unsigned)kVofSeg + threadIdx.x;
    int i, j, k;
    flux_cell_of(a, t0 < F ? t0 : 0u, i, j, k);
    // flux_cell_of shifts the sweep direction's index by -1; step in the
    // unshifted (i, j, k) of the enumeration
    int ii = i + (a.d == 0), jj = j + (a.d == 1), kk = k + (a.d == 2);
    long n[kVofPer];
    double cc[kVofPer];
#pragma unroll
    for (int q = 0; q < kVofPer; q++) {
        const unsigned t = t0 + q * kVofListThreads;
        if (q > 0) {
            ii += kVofListThreads;
            while (ii >= e0) {
                ii -= e0;
                if (++jj >= e1) { jj = 0; kk++; }
            }
        }
        n[q] = t < F ? lidx(a.L, ii - (a.d == 0), jj - (a.d == 1), kk - (a.d == 2)) : -1;
    }
#pragma unroll
    for (int q = 0; q < kVofPer; q++) cc[q] = n[q] >= 0 ? a.c[n[q]] : 0.0;
    unsigned m[kVofPer];
#pragma unroll
    for (int q = 0; q < kVofPer; q++) {
        m[q] = __ballot_sync(0xffffffffu, cc[q] > 0.0 && cc[q] != 1.0);
        if (lane == 0) wcount[q * (kVofListThreads / 32) + w] = __popc(m[q]);
    }
    __syncthreads();
    // the block's mixed cells in the order (q, warp, lane): exclusive scan of
    // the 32 counts in that order
    if (w == 0) {
        const int c = wcount[lane];
        int s = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += v;
        }
        wbase[lane] = s - c;
        if (lane == 31) {
            total = s;
            if (s > 0) room = atomicAdd(a.count, s);
        }
    }
    __syncthreads();
    if (total == 0) return;
#pragma unroll
    for (int q = 0; q < kVofPer; q++)
        if ((m[q] >> lane) & 1u) {
            const long e = (long)room + wbase[q * (kVofListThreads / 32) + w] + __popc(m[q] & ((1u << lane) - 1u));
            if (e < a.cap) a.list[e] = n[q];
        }
}

// 2. PLIC fluxes of the listed cells: fit_plane_new + three FL3D for swpz
// (vofnonmodule.f90:166-186, 633-655), mycs + AL3D + two FL3D for swpr
// (:700-727)
__global__ void __launch_bounds__(128) k_vof_mixed_flux(const SweepArgs a) {
    const Layout& L = a.L;
    const long od = a.d == 0 ? 1 : (a.d == 1 ? L.pitch : L.plane);
    long cnt = *a.count;
    if (cnt > a.cap) cnt = a.cap;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < cnt; q += (long)gridDim.x * blockDim.x) {
        const long n = a.list[q];
        double cc = a.c[n];
        double a2 = courant(a, a.us[n]);
        double a1 = courant(a, a.us[n - od]);
        double st[27];
#pragma unroll
        for (int k1 = -1; k1 <= 1; k1++)
#pragma unroll
            for (int j1 = -1; j1 <= 1; j1++)
#pragma unroll
                for (int i1 = -1; i1 <= 1; i1++)
                    st[(i1 + 1) + 3 * (j1 + 1) + 9 * (k1 + 1)] = a.c[n + i1 + j1 * L.pitch + k1 * L.plane];
        double m[3], x0[3] = {0.0, 0.0, 0.0}, dx[3] = {1.0, 1.0, 1.0};
        plic::mycs(st, m);
        double f1 = 0.0, f2 = 0.0, f3 = 0.0;
        if (!a.wy) {
            if (!(m[0] == 0.0 && m[1] == 0.0 && m[2] == 0.0)) {
                double alpha = plic::al3d(m, cc);
                m[a.d] = m[a.d] / (1.0 - a1 + a2);
                alpha = alpha + m[a.d] * a1;
                double mm1 = plic::dmax1(a1, 0.0);
                double mm2 = 1.0 - mm1 + plic::dmin1(0.0, a2);
                if (a1 < 0.0) {
                    x0[a.d] = a1; dx[a.d] = -a1;
                    f1 = plic::fl3d(m, alpha, x0, dx);
                }
                if (a2 > 0.0) {
                    x0[a.d] = 1.0; dx[a.d] = a2;
                    f3 = plic::fl3d(m, alpha, x0, dx);
                }
                x0[a.d] = mm1; dx[a.d] = mm2;
                f2 = plic::fl3d(m, alpha, x0, dx);
            }
        } else {
            double alpha = plic::al3d(m, cc);
            if (a1 < 0.0) {
                dx[a.d] = -a1;
                f1 = plic::fl3d(m, alpha, x0, dx);
            }
            if (a2 > 0.0) {
                x0[a.d] = 1.0 - a2; dx[a.d] = a2;
                f3 = plic::fl3d(m, alpha, x0, dx);
            }
        }
        a.v1[n] = f1; a.v2[n] = f2; a.v3[n] = f3;
    }
}

// vof1/vof2/vof3 of one flux cell from its volume fraction cc and the
// Courant numbers of its low and high faces: closed form for cc == 1 (and 0
// for cc <= 0), the stored PLIC flux for a mixed cell (vofnonmodule.f90:155-186,
// :700-727)
__device__ inline double cell_flux(const SweepArgs& a, double cc, long n, double alo, double ahi, int which) {
    if (cc == 1.0) {
        if (which == 1) return plic::dmax1(-alo, 0.0);
        if (which == 3) return plic::dmax1(ahi, 0.0);
        return 1.0 - plic::dmax1(alo, 0.0) + plic::dmin1(ahi, 0.0);
    }
    if (cc > 0.0) return which == 1 ? a.v1[n] : (which == 2 ? a.v2[n] : a.v3[n]);
    return 0.0;
}

// 3. the update of the interior: new c, clipping (swpz :224-230 / swpr
// :731-745 and get_flags_and_clip) and the flag, into the second buffer.
// Each thread updates kVofUpd cells of a row, kVofUpdThreads apart; the
// volume fractions and face velocities of all of them are loaded before any
// test on them, so their loads are in flight together.
static constexpr int kVofUpdThreads = 128, kVofUpd = 2;
__global__ void __launch_bounds__(kVofUpdThreads) k_vof_update(const SweepArgs a) {
    const int j = blockIdx.y, k = blockIdx.z;
    const Layout& L = a.L;
    const long od = a.d == 0 ? 1 : (a.d == 1 ? L.pitch : L.plane);
    const int i0 = blockIdx.x * (kVofUpdThreads * kVofUpd) + threadIdx.x;
    double cm[kVofUpd], c0[kVofUpd], cp[kVofUpd], um[kVofUpd], u0[kVofUpd];
    long n[kVofUpd];
#pragma unroll
    for (int q = 0; q < kVofUpd; q++) {
        const int i = i0 + q * kVofUpdThreads;
        n[q] = lidx(L, i < L.n[0] ? i : L.n[0] - 1, j, k);
        cm[q] = a.c[n[q] - od]; c0[q] = a.c[n[q]]; cp[q] = a.c[n[q] + od];
        um[q] = a.us[n[q] - od]; u0[q] = a.us[n[q]];
    }
#pragma unroll
    for (int q = 0; q < kVofUpd; q++) {
        if (i0 + q * kVofUpdThreads >= L.n[0]) continue;
        const double a1 = courant(a, um[q]), a2 = courant(a, u0[q]);
        double cnew;
        if (!a.wy) {
            // vof3 of n-od needs only its high face (n-od), vof1 of n+od only its low face (n)
            cnew = cell_flux(a, cm[q], n[q] - od, 0.0, a1, 3) + cell_flux(a, c0[q], n[q], a1, a2, 2) +
                   cell_flux(a, cp[q], n[q] + od, a2, 0.0, 1);
            cnew = plic::dmax1(0.0, plic::dmin1(1.0, cnew));
        } else {
            cnew = c0[q] - (cell_flux(a, c0[q], n[q], a1, a2, 3) - cell_flux(a, cp[q], n[q] + od, a2, 0.0, 1)) +
                   (cell_flux(a, cm[q], n[q] - od, 0.0, a1, 3) - cell_flux(a, c0[q], n[q], a1, a2, 1)) +
                   (double)a.cg[n[q]] * (a2 - a1);
            if (cnew < a.epsc) cnew = 0.0;
            else if (cnew > 1.0 - a.epsc) cnew = 1.0;
        }
        int8_t fl;
        if (cnew <= a.epsc) { fl = 0; cnew = 0.0; }
        else if (cnew >= 1.0 - a.epsc) { fl = 1; cnew = 1.0; }
        else fl = 2;
        a.cn[n[q]] = cnew;
        a.flag[n[q]] = fl;
    }
}

// ghost cells of the new cvof and flags: SetVOFBC (x- y- z- x+ y+ z+ in that
// order), then the periodic wrap of do_all_ghost, then get_flags_and_clip.
// In swp the exchange of do_all_ghost comes after SetVOFBC, so where the
// velocity is periodic the wrap wins over the VOF condition.  A ghost that
// no condition writes (second layer of 'jet' or '90deg') keeps the value it
// held before the sweep, which is in the source buffer `old`.
__global__ void k_vof_ghosts(double* __restrict__ c, const double* __restrict__ old, int8_t* __restrict__ flag,
                             const Layout L, const Bnd B, const VofJet J, long G, double epsc) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= G) return;
    int i, j, k;
    if (!ghost_cell(L, t, i, j, k)) return;
    int s[3];
    double val;
    if (!vof_ghost_rule<true>(L, B, J, i, j, k, s, val)) {
        const long q = lidx(L, s[0], s[1], s[2]);
        val = vof_interior(L, s) ? c[q] : old[q];
    }
    int8_t fl;
    if (val <= epsc) { fl = 0; val = 0.0; }
    else if (val >= 1.0 - epsc) { fl = 1; val = 1.0; }
    else fl = 2;
    long n = lidx(L, i, j, k);
    c[n] = val;
    flag[n] = fl;
}

// c_mask(cvof, cbinary), vofmodules.f90:1295-1305 (whole ghosted array)
__global__ void k_c_mask(const double* __restrict__ c, uint8_t* __restrict__ cg, long total) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < total) cg[t] = c[t] > 0.5 ? 1 : 0;
}

// scratch of the sweeps, allocated with the handle (paris_gpu_init): the
// sparse flux arrays and the segmented list (sized for the largest flux
// domain of the three directions)
int vof_scratch(paris_ctx* c) {
    const Layout& L = c->L;
    if (c->vflux) return PARIS_OK;
    long F = 0;
    for (int d = 0; d < 3; d++) {
        long e = (long)(L.n[0] + (d == 0 ? 2 : 0)) * (L.n[1] + (d == 1 ? 2 : 0)) * (L.n[2] + (d == 2 ? 2 : 0));
        F = e > F ? e : F;
    }
    PARIS_CUDA_TRY(c, cudaMalloc(&c->vflux, 3 * L.total * sizeof(double)));
    PARIS_CUDA_TRY(c, cudaMalloc(&c->mixlist, F * sizeof(long)));
    PARIS_CUDA_TRY(c, cudaMalloc(&c->mixsegn, sizeof(int)));
    c->mixcap = F;
    return PARIS_OK;
}

int vof_sweep_dir(paris_ctx* c, int d, double dt, const double* src, double* dst, int8_t* flag, const double* us,
                  const uint8_t* cg) {
    const Layout& L = c->L;
    PARIS_CHECK(vof_scratch(c));
    SweepArgs a;
    a.c = src;
    a.cn = dst;
    a.flag = flag;
    a.us = us;
    a.cg = cg;
    a.v1 = c->vflux;
    a.v2 = c->vflux + L.total;
    a.v3 = c->vflux + 2 * L.total;
    a.list = c->mixlist;
    a.count = c->mixsegn;
    a.cap = c->mixcap;
    a.L = L;
    a.d = d;
    a.wy = c->d.vof_advect == PARIS_ADVECT_WY;
    a.dt = dt;
    a.dxyz = c->h_dxh[c->d.ng];
    int ex;
    a.rdxyz = frexp(a.dxyz, &ex) == 0.5 ? 1.0 / a.dxyz : 0.0;   // 1/2^k is exact
    a.epsc = c->d.epsc;
    const long F = (long)(L.n[0] + (d == 0 ? 2 : 0)) * (L.n[1] + (d == 1 ? 2 : 0)) * (L.n[2] + (d == 2 ? 2 : 0));
    // the four kernels of a direction share the profile label "vof_sweep",
    // with the direction's cells counted once (on the update)
    PARIS_CUDA_TRY(c, cudaMemsetAsync(c->mixsegn, 0, sizeof(int), c->stream));
    PARIS_LAUNCH_N(c, "vof_sweep", 0L, k_vof_mixed_list, div_up(F, kVofSeg), kVofListThreads, 0, a, (unsigned)F);
    PARIS_LAUNCH_N(c, "vof_sweep", 0L, k_vof_mixed_flux, c->nsm * 16, 128, 0, a);
    PARIS_LAUNCH_N(c, "vof_sweep", c->N, k_vof_update, dim3(div_up(L.n[0], kVofUpdThreads * kVofUpd), L.n[1], L.n[2]),
                   kVofUpdThreads, 0, a);
    long G = ghost_count(c->L);
    PARIS_LAUNCH_N(c, "vof_sweep", 0L, k_vof_ghosts, div_up(G, 256), 256, 0, dst, src, flag, c->L, c->bnd,
                   ctx_vof_jet(c), G, c->d.epsc);
    return PARIS_OK;
}

static int sweep(paris_ctx* c, int d, double dt) {
    PARIS_CHECK(vof_sweep_dir(c, d, dt, c->fld[PARIS_FIELD_CVOF], c->c2, c->flag, c->fld[PARIS_FIELD_U + d], c->cg));
    double* t = c->fld[PARIS_FIELD_CVOF];
    c->fld[PARIS_FIELD_CVOF] = c->c2;
    c->c2 = t;
    return PARIS_OK;
}

// test_cell_size (vofmodules.f90:1827-1834): VOF needs cubic cells
static bool cubic_cells(const paris_ctx* c) {
    int g = c->d.ng;
    double hx = c->h_dxh[g], hy = c->h_dyh[g], hz = c->h_dzh[g];
    return !(fabs(hy - hx) * 1e12 / hx > 1.0 || fabs(hz - hx) * 1e12 / hx > 1.0);
}

extern "C" int paris_vof_sweeps(paris_handle_t c, int32_t tswap, double dt) {
    if (!c) return PARIS_BAD_ARGS;
    if (!cubic_cells(c)) {
        ctx_set_error(c, "non-cubic cells");
        return PARIS_BAD_ARGS;
    }
    cudaSetDevice(c->dev);
    if (c->d.vof_advect == PARIS_ADVECT_WY) {
        if (!c->cg) PARIS_CUDA_TRY(c, cudaMalloc(&c->cg, c->L.total));
        PARIS_LAUNCH(c, k_c_mask, div_up(c->L.total, 256), 256, 0, c->fld[PARIS_FIELD_CVOF], c->cg, c->L.total);
    }
    int order[3];
    int m = ((tswap % 3) + 3) % 3;
    if (m == 0) { order[0] = 2; order[1] = 0; order[2] = 1; }        // z, x, y
    else if (m == 1) { order[0] = 1; order[1] = 2; order[2] = 0; }   // y, z, x
    else { order[0] = 0; order[1] = 1; order[2] = 2; }               // x, y, z
    for (int s = 0; s < 3; s++) PARIS_CHECK(sweep(c, order[s], dt));
    return PARIS_OK;
}

// linfunc(field,a1,a2,MeanFlag), vofmodules.f90:171-218, over every cell of
// the ghosted array (the 27-point filter where all neighbours exist), then
// do_all_ghost.  b1..b4 of initialize_linfunc (vofmodules.f90:133-147).
__global__ void k_linfunc(const double* __restrict__ c, double* __restrict__ f, const Layout L, double a1,
                          double a2, int harm, int filt) {
    // the whole ghosted array: the flat index is the cell's index itself; its
    // (ii, jj, kk) are needed only by the filter
    const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (n >= L.total) return;
    bool inner = false;
    if (filt) {
        const int g = L.ng, tx = L.n[0] + 2 * g, ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
        int ii, jj, kk;
        if (L.total <= 0xffffffffL) {
            const unsigned t = (unsigned)n, r = t / (unsigned)tx;
            ii = (int)(t - r * (unsigned)tx);
            kk = (int)(r / (unsigned)ty);
            jj = (int)(r - (unsigned)kk * (unsigned)ty);
        } else {
            ii = (int)(n % tx); jj = (int)((n / tx) % ty); kk = (int)(n / ((long)tx * ty));
        }
        inner = ii > 0 && ii < tx - 1 && jj > 0 && jj < ty - 1 && kk > 0 && kk < tz - 1;
    }
    double cf;
    if (inner) {
        const double b1 = 8.0 / 64, b2 = 4.0 / 64, b3 = 2.0 / 64, b4 = 1.0 / 64;
        long sy = L.pitch, sz = L.plane;
        cf = b1 * c[n] + b2 * (c[n - 1] + c[n - sy] + c[n - sz] + c[n + 1] + c[n + sy] + c[n + sz]) +
             b3 * (c[n + 1 + sy] + c[n + 1 - sy] + c[n - 1 + sy] + c[n - 1 - sy] + c[n + 1 + sz] + c[n + 1 - sz] +
                   c[n - 1 + sz] + c[n - 1 - sz] + c[n + sy + sz] + c[n + sy - sz] + c[n - sy + sz] + c[n - sy - sz]) +
             b4 * (c[n + 1 + sy + sz] + c[n + 1 + sy - sz] + c[n + 1 - sy + sz] + c[n + 1 - sy - sz] +
                   c[n - 1 + sy + sz] + c[n - 1 + sy - sz] + c[n - 1 - sy + sz] + c[n - 1 - sy - sz]);
    } else {
        cf = c[n];
    }
    if (!harm) {
        f[n] = cf * (a2 - a1) + a1;
    } else {
        double inva1 = 1.0 / (a1 + 1.e-50), inva2 = 1.0 / (a2 + 1.e-50);
        f[n] = 1.0 / (cf * (inva2 - inva1) + inva1);
    }
}

extern "C" int paris_linfunc(paris_handle_t c, int32_t which) {
    if (!c || (which != PARIS_FIELD_RHO && which != PARIS_FIELD_MU)) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, which));
    double a1 = which == PARIS_FIELD_RHO ? c->d.rho1 : c->d.mu1;
    double a2 = which == PARIS_FIELD_RHO ? c->d.rho2 : c->d.mu2;
    int mean = which == PARIS_FIELD_RHO ? c->d.dens_mean : c->d.visc_mean;
    int harm = mean == PARIS_MEAN_HARM;
    const long tot = c->L.total;
    PARIS_LAUNCH_N(c, "linfunc", tot, k_linfunc, div_up(tot, 256), 256, 0, c->fld[PARIS_FIELD_CVOF], c->fld[which], c->L, a1, a2,
                 harm, c->d.nfilter > 0 ? 1 : 0);
    PARIS_CHECK(ctx_ghost_fill(c, c->fld[which]));
    return PARIS_OK;
}

// ---- initial condition: spheres by ls2vof_refined -----------------------------
struct Spheres {
    const double *xc, *yc, *zc, *rad;
    int nb;
};

static constexpr int kMaxCand = 16;

// shapes2ls (vofmodules.f90:973-993) restricted to the bubbles that can be the
// max in the cell's stencil region (all bubbles when there are too many).
__device__ inline double shapes2ls(const Spheres& S, const int* cand, int nc, double xx, double yy, double zz) {
    double r = -2.0e6;
    for (int q = 0; q < nc; q++) {
        int ib = cand ? cand[q] : q;
        double dx = xx - S.xc[ib], dy = yy - S.yc[ib], dz = zz - S.zc[ib];
        double v = S.rad[ib] * S.rad[ib] - (1.0 * (dx * dx) + 1.0 * (dy * dy) + 1.0 * (dz * dz));
        r = r > v ? r : v;
    }
    return r;
}

// ls2vof_in_cell, vofnonmodule.f90:1142-1190
__device__ inline double ls2vof_in_cell(const double st[27], int& nflag) {
    double m[3], zero[3] = {0.0, 0.0, 0.0}, one[3] = {1.0, 1.0, 1.0};
    plic::fd32(st, m);
    m[0] = fabs(m[0]); m[1] = fabs(m[1]); m[2] = fabs(m[2]);
    double norml1 = m[0] + m[1] + m[2];
    m[0] = m[0] / norml1; m[1] = m[1] / norml1; m[2] = m[2] / norml1;
    double alpha = 32.0 * st[13] / norml1;
    alpha = alpha + 0.5;
    if (alpha >= 1.0) { nflag = 1; return 1.0; }
    if (alpha <= 0.0) { nflag = 0; return 0.0; }
    nflag = 2;
    return plic::fl3d(m, alpha, zero, one);
}

// One pass of ls2vof_refined over the interior.  pass 2 (n1 > 1) refines the
// cells whose 3x3x3 flag neighbourhood (flags of pass 1) is not isolated
// (notisolated, vofmodules.f90:1126-1150) and writes into cout/fout.
__global__ void k_ls2vof(const Spheres S, const Layout L, const double* __restrict__ xc, const double* __restrict__ yc,
                         const double* __restrict__ zc, const double* __restrict__ dxa, const double* __restrict__ dya,
                         const double* __restrict__ dza, int n1, const int8_t* __restrict__ fin,
                         const double* __restrict__ cin, double* __restrict__ cout, int8_t* __restrict__ fout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.n[0]) return;
    const int g = L.ng;
    long n = lidx(L, i, j, k);
    if (n1 > 1) {
        int nfrac = 0, nfull = 0, ncells = 0;
        for (int i0 = -1; i0 <= 1; i0++)
            for (int j0 = -1; j0 <= 1; j0++)
                for (int k0 = -1; k0 <= 1; k0++) {
                    int f = fin[n + i0 + j0 * L.pitch + k0 * L.plane];
                    nfrac += f / 2; nfull += f % 2; ncells++;
                }
        bool refine = !(nfrac == 0 && (nfull == 0 || nfull == ncells));
        if (!refine) {
            cout[n] = cin[n];
            fout[n] = fin[n];
            return;
        }
    }
    double x = xc[i + g], y = yc[j + g], z = zc[k + g];
    double dxc = dxa[i + g], dyc = dya[j + g], dzc = dza[k + g];
    double dx1 = dxc / n1, dy1 = dyc / n1, dz1 = dzc / n1;
    // candidate bubbles: upper bound of rad^2 - d^2 over the region reaches the
    // best lower bound (region radius generous; any superset gives the same max)
    int cand[kMaxCand];
    int nc = 0;
    bool all = false;
    {
        double hx = 0.5 * dxc + dx1, hy = 0.5 * dyc + dy1, hz = 0.5 * dzc + dz1;
        double R = 1.01 * sqrt(hx * hx + hy * hy + hz * hz);
        double lbmax = -1e300;
        for (int ib = 0; ib < S.nb; ib++) {
            double ddx = x - S.xc[ib], ddy = y - S.yc[ib], ddz = z - S.zc[ib];
            double D = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            double lb = S.rad[ib] * S.rad[ib] - (D + R) * (D + R);
            lbmax = lb > lbmax ? lb : lbmax;
        }
        for (int ib = 0; ib < S.nb; ib++) {
            double ddx = x - S.xc[ib], ddy = y - S.yc[ib], ddz = z - S.zc[ib];
            double D = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
            double dn = D - R > 0.0 ? D - R : 0.0;
            double ub = S.rad[ib] * S.rad[ib] - dn * dn;
            if (ub >= lbmax - 1e-9 * (fabs(lbmax) + 1.0)) {
                if (nc < kMaxCand) cand[nc++] = ib;
                else all = true;
            }
        }
    }
    const int* cp = all ? nullptr : cand;
    int ncu = all ? S.nb : nc;
    int nfrac = 0, nfull = 0;
    double b = 0.0;
    for (int l = 0; l < n1; l++)
        for (int m = 0; m < n1; m++)
            for (int q = 0; q < n1; q++) {
                double x0 = x - 0.5 * dxc + 0.5 * dx1 + dx1 * l;
                double y0 = y - 0.5 * dyc + 0.5 * dy1 + dy1 * m;
                double z0 = z - 0.5 * dzc + 0.5 * dz1 + dz1 * q;
                double st[27];
                for (int i0 = -1; i0 <= 1; i0++)
                    for (int j0 = -1; j0 <= 1; j0++)
                        for (int k0 = -1; k0 <= 1; k0++)
                            st[(i0 + 1) + 3 * (j0 + 1) + 9 * (k0 + 1)] =
                                shapes2ls(S, cp, ncu, x0 + i0 * dx1, y0 + j0 * dy1, z0 + k0 * dz1);
                int nflag;
                double a = ls2vof_in_cell(st, nflag);
                if (nflag == 2) nfrac++;
                else if (nflag == 1) nfull++;
                b = b + a;
            }
    double cv = b / (double)(n1 * n1 * n1);
    int8_t fl;
    if (nfrac > 0) fl = 2;
    else if (nfull == n1 * n1 * n1) { fl = 1; cv = 1.0; }
    else if (nfull == 0) { fl = 0; cv = 0.0; }
    else fl = 2;
    cout[n] = cv;
    fout[n] = fl;
}

// walls of the initial field, without the clipping of the sweeps: the
// ghosts of levelset2vof (vofmodules.f90:1098-1106), the periodic exchange
// where the velocity is periodic, then SetVOFBC on every face whose VOF
// condition is not periodic, over the exchanged value (a direction may be
// periodic for the velocity and dry/wet for the volume fraction).  Fixed
// values carry their flag, copies the flag of their source; a ghost that no
// condition writes keeps its value, with the flag of get_flags_and_clip.
__global__ void k_init_ghosts(double* __restrict__ c, int8_t* __restrict__ flag, const Layout L, const Bnd B,
                              const VofJet J, long G, double epsc) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= G) return;
    int i, j, k;
    if (!ghost_cell(L, t, i, j, k)) return;
    int s[3];
    double val;
    int8_t fl;
    if (vof_ghost_rule<false>(L, B, J, i, j, k, s, val)) {
        fl = (int8_t)val;
    } else {
        const long q = lidx(L, s[0], s[1], s[2]);
        val = c[q];
        if (vof_interior(L, s)) fl = flag[q];
        else fl = val <= epsc ? 0 : (val >= 1.0 - epsc ? 1 : 2);
    }
    long n = lidx(L, i, j, k);
    c[n] = val;
    flag[n] = fl;
}

extern "C" int paris_init_spheres(paris_handle_t c, int32_t nb, const double* xc, const double* yc, const double* zc,
                                  const double* rad, int32_t refinement) {
    if (!c || nb <= 0 || !xc || !yc || !zc || !rad || refinement < 1) return PARIS_BAD_ARGS;
    // ls2vof_refined stops with "bad flag" when a 'jet' or '90deg' face is
    // present: its second ghost layer still holds the vof_flag = 3 of the
    // allocation (vofmodules.f90:436-437,1222-1231).  Such runs start from an
    // uploaded field or a restart file.
    for (int o = 0; o < 6; o++)
        if (c->d.vofbdry_cond[o] == PARIS_VOFBC_JET || c->d.vofbdry_cond[o] == PARIS_VOFBC_90DEG) {
            ctx_set_error(c, "ls2vof_refined: bad flag (a 'jet' or '90deg' VOF face leaves vof_flag = 3 "
                             "in its second ghost layer)");
            return PARIS_BAD_ARGS;
        }
    cudaSetDevice(c->dev);
    double* dbuf = nullptr;
    PARIS_CUDA_TRY(c, cudaMalloc(&dbuf, 4L * nb * sizeof(double)));
    const double* src[4] = {xc, yc, zc, rad};
    for (int q = 0; q < 4; q++)
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(dbuf + q * nb, src[q], nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    Spheres S{dbuf, dbuf + nb, dbuf + 2 * nb, dbuf + 3 * nb, nb};
    int8_t* f2 = nullptr;
    PARIS_CUDA_TRY(c, cudaMalloc(&f2, c->L.total));
    PARIS_CUDA_TRY(c, cudaMemsetAsync(f2, 0, c->L.total, c->stream));
    dim3 grid(div_up(c->L.n[0], 64), c->L.n[1], c->L.n[2]);
    long G = ghost_count(c->L);
    double* cv = c->fld[PARIS_FIELD_CVOF];
    // pass 1 (n1 = 1) into c2/f2, ghosts, then pass 2 into cvof/flag
    PARIS_LAUNCH(c, k_ls2vof, grid, 64, 0, S, c->L, c->xc, c->yc, c->zc, c->dx, c->dy, c->dz, 1, (const int8_t*)nullptr,
                 (const double*)nullptr, c->c2, f2);
    PARIS_LAUNCH(c, k_init_ghosts, div_up(G, 256), 256, 0, c->c2, f2, c->L, c->bnd, ctx_vof_jet(c), G, c->d.epsc);
    PARIS_LAUNCH(c, k_ls2vof, grid, 64, 0, S, c->L, c->xc, c->yc, c->zc, c->dx, c->dy, c->dz, refinement, f2, c->c2,
                 cv, c->flag);
    PARIS_LAUNCH(c, k_init_ghosts, div_up(G, 256), 256, 0, cv, c->flag, c->L, c->bnd, ctx_vof_jet(c), G,
                 c->d.epsc);
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    cudaFree(dbuf);
    cudaFree(f2);
    return PARIS_OK;
}
