// ctx.cu -- life cycle of a handle, host<->device transfers in the
// reference's array layout, ghost-layer fills and deterministic reductions.
#include <stdarg.h>
#include <string.h>
#include <string>
#include "ctx.cuh"

void ctx_set_error(paris_ctx* c, const char* fmt, ...) {
    if (!c) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(c->err, sizeof(c->err), fmt, ap);
    va_end(ap);
}

// Coordinates of the reference's uniform grid, paris.f90:3057-3100 (xform=0).
static void make_axis(int n, int ng, double L, std::vector<double>& x, std::vector<double>& xh,
                      std::vector<double>& dx, std::vector<double>& dxh) {
    int nt = n + 2 * ng;
    xh.assign(nt, 0.0);
    x.assign(nt, 0.0); dx.assign(nt, 0.0); dxh.assign(nt, 0.0);
    const double form = 0.0;
    for (int f = 1; f <= nt; f++) {
        double s = (double)(f - ng) / (double)n;
        xh[f - 1] = L * (form * s * (0.5 - s) * (1.0 - s) + s);
    }
    for (int f = 2; f <= nt; f++) x[f - 1] = 0.5 * (xh[f - 1] + xh[f - 2]);
    x[0] = 2.0 * xh[0] - x[1];
    for (int f = 1; f <= nt - 1; f++) dxh[f - 1] = x[f] - x[f - 1];
    dxh[nt - 1] = dxh[nt - 2];
    for (int f = 2; f <= nt; f++) dx[f - 1] = xh[f - 1] - xh[f - 2];
    dx[0] = dx[1];
}

static int upload_vec(paris_ctx* c, double** d, const std::vector<double>& h) {
    PARIS_CUDA_TRY(c, cudaMalloc(d, h.size() * sizeof(double)));
    PARIS_CUDA_TRY(c, cudaMemcpy(*d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    return PARIS_OK;
}

int ctx_alloc_field(paris_ctx* c, int field) {
    if (field == PARIS_FIELD_VOF_FLAG) {
        if (!c->flag) {
            PARIS_CUDA_TRY(c, cudaMalloc(&c->flag, c->L.total));
            PARIS_CUDA_TRY(c, cudaMemsetAsync(c->flag, 0, c->L.total, c->stream));
        }
        return PARIS_OK;
    }
    if (field == PARIS_FIELD_HEIGHT) {
        if (!c->height) {
            PARIS_CUDA_TRY(c, cudaMalloc(&c->height, 6 * c->L.total * sizeof(double)));
            PARIS_CUDA_TRY(c, cudaMemsetAsync(c->height, 0, 6 * c->L.total * sizeof(double), c->stream));
        }
        return PARIS_OK;
    }
    if (field == PARIS_FIELD_A || field == PARIS_FIELD_VOF_PHASE) return PARIS_OK;
    if (field < 0 || field >= PARIS_NFIELDS) return PARIS_BAD_ARGS;
    if (!c->fld[field]) {
        PARIS_CUDA_TRY(c, cudaMalloc(&c->fld[field], c->L.total * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMemsetAsync(c->fld[field], 0, c->L.total * sizeof(double), c->stream));
    }
    return PARIS_OK;
}

// ---- ghost fills ----------------------------------------------------------
template <typename T>
__global__ void k_ghost_fill(T* __restrict__ f, const Layout L, const Bnd B) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int i, j, k;
    if (!ghost_cell(L, t, i, j, k)) return;
    int si = i, sj = j, sk = k;
    if (B.per[0]) { if (si < 0) si += L.n[0]; else if (si >= L.n[0]) si -= L.n[0]; }
    if (B.per[1]) { if (sj < 0) sj += L.n[1]; else if (sj >= L.n[1]) sj -= L.n[1]; }
    if (B.per[2]) { if (sk < 0) sk += L.n[2]; else if (sk >= L.n[2]) sk -= L.n[2]; }
    if (si == i && sj == j && sk == k) return;
    f[lidx(L, i, j, k)] = f[lidx(L, si, sj, sk)];
}

int ctx_ghost_fill(paris_ctx* c, double* f) {
    long G = ghost_count(c->L);
    PARIS_LAUNCH(c, k_ghost_fill<double>, div_up(G, 256), 256, 0, f, c->L, c->bnd);
    return PARIS_OK;
}

int ctx_ghost_fill_i8(paris_ctx* c, int8_t* f) {
    long G = ghost_count(c->L);
    PARIS_LAUNCH(c, k_ghost_fill<int8_t>, div_up(G, 256), 256, 0, f, c->L, c->bnd);
    return PARIS_OK;
}

// ---- reductions -----------------------------------------------------------
// Kernels write kRedBlocks partials per slot; this sums them in a fixed order.
__global__ void k_reduce_slots(const double* __restrict__ part, double* out, int op_max, int nb) {
    __shared__ double sh[32];
    int slot = blockIdx.x;
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        double x = part[(long)slot * kRedBlocks + b];
        v = op_max ? fmax(v, x) : v + x;
    }
    v = op_max ? block_max<256>(v, sh) : block_sum<256>(v, sh);
    if (threadIdx.x == 0) out[slot] = v;
}

// The reduced scalars are written by the kernel straight into mapped pinned
// host memory: a small device-to-host copy would queue on the copy engine
// behind any field download in flight on the transfer stream.
int ctx_reduce_finish(paris_ctx* c, int nslots, double* out_host, int op_max) {
    PARIS_LAUNCH(c, k_reduce_slots, nslots, 256, 0, c->red_part, c->red_host_dev, op_max, c->red_nb);
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int s = 0; s < nslots; s++) out_host[s] = c->red_host[s];
    return PARIS_OK;
}

// ---- int8 <-> int32 staging -----------------------------------------------
__global__ void k_i32_to_i8(const int32_t* __restrict__ src, int8_t* __restrict__ dst, const Layout L) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int g = L.ng, tx = L.n[0] + 2 * g, ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
    if (t >= (long)tx * ty * tz) return;
    int i = (int)(t % tx) - g, j = (int)((t / tx) % ty) - g, k = (int)(t / ((long)tx * ty)) - g;
    dst[lidx(L, i, j, k)] = (int8_t)src[t];
}
__global__ void k_i8_to_i32(const int8_t* __restrict__ src, int32_t* __restrict__ dst, const Layout L) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int g = L.ng, tx = L.n[0] + 2 * g, ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
    if (t >= (long)tx * ty * tz) return;
    int i = (int)(t % tx) - g, j = (int)((t / tx) % ty) - g, k = (int)(t / ((long)tx * ty)) - g;
    dst[t] = src[lidx(L, i, j, k)];
}
// vof_phase (get_vof_phase, vofmodules.f90:573-592), computed from cvof
__global__ void k_phase_i32(const double* __restrict__ c, int32_t* __restrict__ dst, const Layout L, double epsc) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    int g = L.ng, tx = L.n[0] + 2 * g, ty = L.n[1] + 2 * g, tz = L.n[2] + 2 * g;
    if (t >= (long)tx * ty * tz) return;
    int i = (int)(t % tx) - g, j = (int)((t / tx) % ty) - g, k = (int)(t / ((long)tx * ty)) - g;
    dst[t] = c[lidx(L, i, j, k)] < (0.5 - epsc) ? 0 : 1;
}

// ---- exported life cycle --------------------------------------------------
static int validate(const paris_grid_desc* d) {
    if (!d) return PARIS_BAD_ARGS;
    // at least four cells across, or Nz = 2: the reference's two-dimensional
    // runs (one cell of depth and its periodic image)
    if (d->nx < 4 || d->ny < 4 || (d->nz < 4 && d->nz != 2) || d->ng != 2) return PARIS_BAD_ARGS;
    if (d->nx > 32767 || d->ny > 32767 || d->nz > 32767) return PARIS_BAD_ARGS;
    for (int a = 0; a < 3; a++) {
        int lo = d->bdry_cond[a], hi = d->bdry_cond[a + 3];
        if (lo < 0 || lo > 2 || hi < 0 || hi > 2) return PARIS_BAD_ARGS;
        if ((lo == PARIS_BC_PERIODIC) != (hi == PARIS_BC_PERIODIC)) return PARIS_BAD_ARGS;
        // a periodic volume fraction needs a periodic velocity; a periodic
        // velocity may carry dry / wet / outflow VOF ghosts (SetVOFBC after the wrap)
        int vlo = d->vofbdry_cond[a], vhi = d->vofbdry_cond[a + 3];
        if (vlo == PARIS_VOFBC_PERIODIC && lo != PARIS_BC_PERIODIC) return PARIS_BAD_ARGS;
        if (vhi == PARIS_VOFBC_PERIODIC && hi != PARIS_BC_PERIODIC) return PARIS_BAD_ARGS;
        for (int v : {vlo, vhi})
            if (v < PARIS_VOFBC_DRY || v > PARIS_VOFBC_90DEG) return PARIS_BAD_ARGS;
        // SetVOFBC: "jet only at x-" (vofmodules.f90:1717)
        if (vhi == PARIS_VOFBC_JET || (a > 0 && vlo == PARIS_VOFBC_JET)) return PARIS_BAD_ARGS;
    }
    if (d->inject_type < 0 || d->inject_type > 5) return PARIS_BAD_ARGS;
    if (d->xlength <= 0 || d->ylength <= 0 || d->zlength <= 0) return PARIS_BAD_ARGS;
    return PARIS_OK;
}

extern "C" int paris_gpu_init(const paris_grid_desc* desc, paris_handle_t* out) {
    if (!out) return PARIS_BAD_ARGS;
    *out = nullptr;
    int st = validate(desc);
    if (st != PARIS_OK) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= desc->device || desc->device < 0) {
        cudaGetLastError();
        return PARIS_NO_DEVICE;
    }
    paris_ctx* c = new paris_ctx();
    c->d = *desc;
    if (c->d.epsc <= 0.0) c->d.epsc = 1e-12;
    if (c->d.nrelax <= 0) c->d.nrelax = 3;
    c->dev = desc->device;
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->dev);
    if (cudaSetDevice(c->dev) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return PARIS_CUDA_ERROR;
    }
    c->L = make_layout(desc->nx, desc->ny, desc->nz, desc->ng);
    c->N = (long)desc->nx * desc->ny * desc->nz;
    for (int a = 0; a < 3; a++) {
        c->bnd.per[a] = desc->bdry_cond[a] == PARIS_BC_PERIODIC;
        c->bnd.wall_lo[a] = desc->bdry_cond[a] == PARIS_BC_WALL || desc->bdry_cond[a] == PARIS_BC_SHEAR;
        c->bnd.wall_hi[a] = desc->bdry_cond[a + 3] == PARIS_BC_WALL || desc->bdry_cond[a + 3] == PARIS_BC_SHEAR;
    }
    for (int o = 0; o < 6; o++) c->bnd.vofbc[o] = desc->vofbdry_cond[o];
    make_axis(desc->nx, desc->ng, desc->xlength, c->h_x, c->h_xh, c->h_dx, c->h_dxh);
    make_axis(desc->ny, desc->ng, desc->ylength, c->h_y, c->h_yh, c->h_dy, c->h_dyh);
    make_axis(desc->nz, desc->ng, desc->zlength, c->h_z, c->h_zh, c->h_dz, c->h_dzh);
    int s = PARIS_OK;
    if (!s) s = upload_vec(c, &c->dx, c->h_dx);
    if (!s) s = upload_vec(c, &c->dxh, c->h_dxh);
    if (!s) s = upload_vec(c, &c->dy, c->h_dy);
    if (!s) s = upload_vec(c, &c->dyh, c->h_dyh);
    if (!s) s = upload_vec(c, &c->dz, c->h_dz);
    if (!s) s = upload_vec(c, &c->dzh, c->h_dzh);
    if (!s) s = upload_vec(c, &c->xc, c->h_x);
    if (!s) s = upload_vec(c, &c->yc, c->h_y);
    if (!s) s = upload_vec(c, &c->zc, c->h_z);
    if (!s) s = upload_vec(c, &c->xh, c->h_xh);
    if (!s) s = upload_vec(c, &c->yh, c->h_yh);
    if (!s) s = upload_vec(c, &c->zh, c->h_zh);
    if (!s && cudaMalloc(&c->red_part, 8L * kRedBlocks * sizeof(double)) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaMalloc(&c->debris_count, sizeof(int)) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaMalloc(&c->cg_scal, 8 * sizeof(double)) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaHostAlloc(&c->red_host, 8 * sizeof(double), cudaHostAllocMapped) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaHostAlloc(&c->err_host, sizeof(int), cudaHostAllocMapped) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaHostGetDevicePointer((void**)&c->err_dev, c->err_host, 0) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s) *c->err_host = 0;
    if (!s && cudaHostGetDevicePointer((void**)&c->red_host_dev, c->red_host, 0) != cudaSuccess) s = PARIS_CUDA_ERROR;
    for (int f : {PARIS_FIELD_CVOF, PARIS_FIELD_U, PARIS_FIELD_V, PARIS_FIELD_W, PARIS_FIELD_RHO, PARIS_FIELD_P})
        if (!s) s = ctx_alloc_field(c, f);
    if (!s) s = ctx_alloc_field(c, PARIS_FIELD_VOF_FLAG);
    if (!s && cudaMalloc(&c->c2, c->L.total * sizeof(double)) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s) s = vof_scratch(c);
    if (!s && cudaMemsetAsync(c->c2, 0, c->L.total * sizeof(double), c->stream) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (!s && cudaStreamSynchronize(c->stream) != cudaSuccess) s = PARIS_CUDA_ERROR;
    if (s) {
        paris_gpu_finalize(c);
        return s;
    }
    *out = c;
    return PARIS_OK;
}

static void free_ptr(void* p) {
    if (p) cudaFree(p);
}

extern "C" int paris_gpu_finalize(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int f = 0; f < PARIS_NFIELDS; f++) free_ptr(c->fld[f]);
    for (void* p : {(void*)c->dx, (void*)c->dxh, (void*)c->dy, (void*)c->dyh, (void*)c->dz, (void*)c->dzh,
                    (void*)c->xc, (void*)c->yc, (void*)c->zc, (void*)c->xh, (void*)c->yh, (void*)c->zh, (void*)c->c2, (void*)c->flag, (void*)c->cg,
                    (void*)c->height, (void*)c->i32stage, (void*)c->cx, (void*)c->cy, (void*)c->cz,
                    (void*)c->rhs, (void*)c->A, (void*)c->red_part, (void*)c->fast_r64,
                    (void*)c->fast_d64, (void*)c->fast_q64,
                    (void*)c->vflux, (void*)c->mixlist, (void*)c->mixsegn, (void*)c->kflag, (void*)c->st_list,
                    (void*)c->st_count, (void*)c->debris_count, (void*)c->cg_scal, (void*)c->adj, (void*)c->stats_part, (void*)c->stats_out, (void*)c->mom_tab,
                    (void*)c->mc_tmp, (void*)c->mc_tmp2, (void*)c->mc_work, (void*)c->mc_fv, (void*)c->mc_flag,
                    (void*)c->mc_cg})
        free_ptr(p);
    if (c->s_h2d) cudaStreamSynchronize(c->s_h2d);
    if (c->s_d2h) cudaStreamSynchronize(c->s_d2h);
    for (int f = 0; f < PARIS_NFIELDS; f++) {
        free_ptr(c->stage_in[f]);
        free_ptr(c->stage_out[f]);
        for (cudaEvent_t e : {c->ev_in_done[f], c->ev_in_free[f], c->ev_out_ready[f], c->ev_out_free[f]})
            if (e) cudaEventDestroy(e);
    }
    if (c->s_h2d) cudaStreamDestroy(c->s_h2d);
    if (c->s_d2h) cudaStreamDestroy(c->s_d2h);
    for (auto& l : c->ref) { free_ptr(l.K); free_ptr(l.p); free_ptr(l.e); }
    mg_fast_free_maps(c);
    for (auto& l : c->fl32) { free_ptr(l.cx); free_ptr(l.cy); free_ptr(l.cz); free_ptr(l.b); free_ptr(l.x); free_ptr(l.x2); }
    for (auto& l : c->fl64) { free_ptr(l.cx); free_ptr(l.cy); free_ptr(l.cz); free_ptr(l.b); free_ptr(l.x); free_ptr(l.x2); }
    if (c->red_host) cudaFreeHost(c->red_host);
    if (c->err_host) cudaFreeHost(c->err_host);
    for (auto e : c->evpool) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PARIS_OK;
}

static int ensure_stage(paris_ctx* c) {
    if (!c->i32stage) {
        long nt = (long)(c->d.nx + 4) * (c->d.ny + 4) * (c->d.nz + 4);
        PARIS_CUDA_TRY(c, cudaMalloc(&c->i32stage, nt * sizeof(int32_t)));
    }
    return PARIS_OK;
}

static long ghosted_cells(const paris_ctx* c) {
    return (long)(c->d.nx + 2 * c->d.ng) * (c->d.ny + 2 * c->d.ng) * (c->d.nz + 2 * c->d.ng);
}

// one contiguous copy: the device array has the Fortran layout
int copy_ghosted(paris_ctx* c, double* dev, const double* host, bool to_dev) {
    size_t bytes = (size_t)c->L.total * sizeof(double);
    if (to_dev)
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c->stream));
    else
        PARIS_CUDA_TRY(c, cudaMemcpyAsync((void*)host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    return PARIS_OK;
}

extern "C" int paris_gpu_upload(paris_handle_t c, int32_t field, const void* host) {
    if (!c || !host || field < 0 || field >= PARIS_NFIELDS) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, field));
    long nt = ghosted_cells(c);
    if (field == PARIS_FIELD_VOF_FLAG) {
        PARIS_CHECK(ensure_stage(c));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->i32stage, host, nt * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
        PARIS_LAUNCH(c, k_i32_to_i8, div_up(nt, 256), 256, 0, c->i32stage, c->flag, c->L);
    } else if (field == PARIS_FIELD_VOF_PHASE) {
        return PARIS_BAD_ARGS;   // derived from cvof
    } else if (field == PARIS_FIELD_A) {
        if (!c->A) PARIS_CUDA_TRY(c, cudaMalloc(&c->A, 8 * c->N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->A, host, 8 * c->N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        c->A_valid = 1;
        c->A_from_upload = 1;
        // the compact form used by the B200 solver: east/north/top faces + rhs
        PARIS_CHECK(ctx_ensure_matrix(c));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->cx, c->A + 1 * c->N, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->cy, c->A + 3 * c->N, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->cz, c->A + 5 * c->N, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->rhs, c->A + 7 * c->N, c->N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        c->have_matrix = 1;
    } else if (field == PARIS_FIELD_HEIGHT) {
        for (int q = 0; q < 6; q++)
            PARIS_CHECK(copy_ghosted(c, c->height + q * c->L.total, (const double*)host + q * nt, true));
    } else {
        PARIS_CHECK(copy_ghosted(c, c->fld[field], (const double*)host, true));
    }
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return PARIS_OK;
}

extern "C" int paris_gpu_download(paris_handle_t c, int32_t field, void* host) {
    if (!c || !host || field < 0 || field >= PARIS_NFIELDS) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    long nt = ghosted_cells(c);
    if (field == PARIS_FIELD_VOF_FLAG || field == PARIS_FIELD_VOF_PHASE) {
        PARIS_CHECK(ensure_stage(c));
        if (field == PARIS_FIELD_VOF_FLAG)
            PARIS_LAUNCH(c, k_i8_to_i32, div_up(nt, 256), 256, 0, c->flag, c->i32stage, c->L);
        else
            PARIS_LAUNCH(c, k_phase_i32, div_up(nt, 256), 256, 0, c->fld[PARIS_FIELD_CVOF], c->i32stage, c->L,
                         c->d.epsc);
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(host, c->i32stage, nt * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    } else if (field == PARIS_FIELD_A) {
        if (!c->have_matrix) return PARIS_BAD_ARGS;
        if (!c->A_valid) PARIS_CHECK(poisson_build_full_A(c));
        PARIS_CUDA_TRY(c, cudaMemcpyAsync(host, c->A, 8 * c->N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    } else if (field == PARIS_FIELD_HEIGHT) {
        if (!c->height) return PARIS_BAD_ARGS;
        for (int q = 0; q < 6; q++)
            PARIS_CHECK(copy_ghosted(c, c->height + q * c->L.total, (const double*)host + q * nt, false));
    } else {
        if (!c->fld[field]) return PARIS_BAD_ARGS;
        PARIS_CHECK(copy_ghosted(c, c->fld[field], (const double*)host, false));
    }
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return PARIS_OK;
}

static bool real_field(int f) {
    return f >= 0 && f < PARIS_NFIELDS && f != PARIS_FIELD_VOF_FLAG && f != PARIS_FIELD_A &&
           f != PARIS_FIELD_HEIGHT && f != PARIS_FIELD_VOF_PHASE;
}

// Device-to-device copy of n doubles on the handle's stream by the SMs, so
// that the copy engines stay free for the host transfers.
__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, long n) {
    const long n2 = n >> 1;
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n2; t += (long)gridDim.x * blockDim.x)
        d2[t] = s2[t];
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) dst[n - 1] = src[n - 1];
}

int ctx_copy(paris_ctx* c, double* dst, const double* src, long n) {
    PARIS_LAUNCH(c, k_copy, (unsigned)(c->nsm * 8), 256, 0, dst, src, n);
    return PARIS_OK;
}

// ---- asynchronous transfers --------------------------------------------------
// An upload fills a device staging copy of the field on the H2D stream; a
// commit makes the handle's stream wait for that copy at the point of the
// commit and move it into the field.  A download copies the field into its own
// staging buffer at the point of issue, and the D2H stream moves that to the
// host while the handle's stream runs on.  Each staging buffer is refilled
// only after the transfer before it has finished with it.
static int async_setup(paris_ctx* c, int f, bool in) {
    if (!c->s_h2d) {
        PARIS_CUDA_TRY(c, cudaStreamCreateWithFlags(&c->s_h2d, cudaStreamNonBlocking));
        PARIS_CUDA_TRY(c, cudaStreamCreateWithFlags(&c->s_d2h, cudaStreamNonBlocking));
    }
    double** buf = in ? &c->stage_in[f] : &c->stage_out[f];
    if (!*buf) {
        PARIS_CUDA_TRY(c, cudaMalloc(buf, c->L.total * sizeof(double)));
        cudaEvent_t* e0 = in ? &c->ev_in_done[f] : &c->ev_out_ready[f];
        cudaEvent_t* e1 = in ? &c->ev_in_free[f] : &c->ev_out_free[f];
        PARIS_CUDA_TRY(c, cudaEventCreateWithFlags(e0, cudaEventDisableTiming));
        PARIS_CUDA_TRY(c, cudaEventCreateWithFlags(e1, cudaEventDisableTiming));
    }
    return PARIS_OK;
}

extern "C" int paris_gpu_upload_async(paris_handle_t c, int32_t field, const void* host) {
    if (!c || !host || !real_field(field)) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, field));
    PARIS_CHECK(async_setup(c, field, true));
    const size_t bytes = (size_t)c->L.total * sizeof(double);
    PARIS_CUDA_TRY(c, cudaStreamWaitEvent(c->s_h2d, c->ev_in_free[field], 0));
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(c->stage_in[field], host, bytes, cudaMemcpyHostToDevice, c->s_h2d));
    PARIS_CUDA_TRY(c, cudaEventRecord(c->ev_in_done[field], c->s_h2d));
    return PARIS_OK;
}

extern "C" int paris_gpu_upload_commit(paris_handle_t c, int32_t field) {
    if (!c || !real_field(field) || !c->stage_in[field]) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_in_done[field], 0));
    PARIS_CHECK(ctx_copy(c, c->fld[field], c->stage_in[field], c->L.total));
    PARIS_CUDA_TRY(c, cudaEventRecord(c->ev_in_free[field], c->stream));
    return PARIS_OK;
}

extern "C" int paris_gpu_download_async(paris_handle_t c, int32_t field, void* host) {
    if (!c || !host || !real_field(field)) return PARIS_BAD_ARGS;
    if (!c->fld[field]) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(async_setup(c, field, false));
    const size_t bytes = (size_t)c->L.total * sizeof(double);
    PARIS_CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_out_free[field], 0));
    PARIS_CHECK(ctx_copy(c, c->stage_out[field], c->fld[field], c->L.total));
    PARIS_CUDA_TRY(c, cudaEventRecord(c->ev_out_ready[field], c->stream));
    PARIS_CUDA_TRY(c, cudaStreamWaitEvent(c->s_d2h, c->ev_out_ready[field], 0));
    PARIS_CUDA_TRY(c, cudaMemcpyAsync(host, c->stage_out[field], bytes, cudaMemcpyDeviceToHost, c->s_d2h));
    PARIS_CUDA_TRY(c, cudaEventRecord(c->ev_out_free[field], c->s_d2h));
    return PARIS_OK;
}

extern "C" int paris_gpu_sync_transfers(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    if (c->s_h2d) PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->s_h2d));
    if (c->s_d2h) PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->s_d2h));
    return PARIS_OK;
}

extern "C" int paris_gpu_copy_field(paris_handle_t c, int32_t dst, int32_t src) {
    if (!c || !real_field(dst) || !real_field(src) || !c->fld[src]) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, dst));
    return ctx_copy(c, c->fld[dst], c->fld[src], c->L.total);
}

__global__ void k_fill(double* __restrict__ f, double v, long n) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < n) f[t] = v;
}

extern "C" int paris_gpu_fill_field(paris_handle_t c, int32_t field, double value) {
    if (!c || !real_field(field)) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, field));
    PARIS_LAUNCH(c, k_fill, div_up(c->L.total, 256), 256, 0, c->fld[field], value, c->L.total);
    return PARIS_OK;
}

extern "C" int paris_gpu_sync(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    PARIS_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return PARIS_OK;
}

extern "C" void* paris_gpu_stream(paris_handle_t c) { return c ? (void*)c->stream : nullptr; }

extern "C" void* paris_gpu_field_ptr(paris_handle_t c, int32_t field) {
    if (!c || field < 0 || field >= PARIS_NFIELDS) return nullptr;
    if (field == PARIS_FIELD_VOF_FLAG) return c->flag;
    if (field == PARIS_FIELD_A) return c->A;
    if (field == PARIS_FIELD_HEIGHT) return c->height;
    if (field == PARIS_FIELD_VOF_PHASE) return nullptr;
    return c->fld[field];
}

extern "C" const char* paris_gpu_last_error(paris_handle_t c) { return c ? c->err : "null handle"; }

extern "C" int64_t paris_gpu_launch_count(paris_handle_t c) { return c ? c->launches : 0; }

// ---- per-kernel event timing --------------------------------------------------
int prof_enabled(const paris_ctx* c) { return c->prof_on; }

void prof_begin(paris_ctx* c, const char* name, long cells) {
    size_t need = 2 * (c->prof.size() + 1);
    while (c->evpool.size() < need) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) { c->prof_on = 0; return; }
        c->evpool.push_back(e);
    }
    int ev = (int)(2 * c->prof.size());
    c->prof.push_back(paris_ctx::ProfRec{name, cells, ev});
    cudaEventRecord(c->evpool[ev], c->stream);
}

void prof_end(paris_ctx* c) {
    if (c->prof.empty()) return;
    cudaEventRecord(c->evpool[c->prof.back().ev + 1], c->stream);
}

extern "C" int paris_gpu_profile(paris_handle_t c, int32_t enable) {
    if (!c) return PARIS_BAD_ARGS;
    if (enable) c->prof.clear();
    c->prof_on = enable ? 1 : 0;
    return PARIS_OK;
}

extern "C" int64_t paris_gpu_profile_report(paris_handle_t c, char* buf, int64_t len) {
    if (!c) return -1;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return -1;
    struct Acc { std::string name; long n; double ms; double cells; };
    std::vector<Acc> acc;
    for (const auto& r : c->prof) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->evpool[r.ev], c->evpool[r.ev + 1]);
        Acc* a = nullptr;
        for (auto& x : acc)
            if (x.name == r.name) { a = &x; break; }
        if (!a) { acc.push_back(Acc{r.name, 0, 0.0, 0.0}); a = &acc.back(); }
        a->n++;
        a->ms += ms;
        a->cells += (double)r.cells;
    }
    std::string out;
    char line[512];
    for (const auto& a : acc) {
        snprintf(line, sizeof(line), "%s\t%ld\t%.6f\t%.0f\n", a.name.c_str(), a.n, a.ms, a.cells);
        out += line;
    }
    int64_t need = (int64_t)out.size() + 1;
    if (buf && len > 0) {
        int64_t m = need < len ? need : len;
        memcpy(buf, out.c_str(), m - 1);
        buf[m - 1] = 0;
    }
    return need;
}

int ctx_ensure_matrix(paris_ctx* c) {
    if (!c->cx) {
        PARIS_CUDA_TRY(c, cudaMalloc(&c->cx, c->N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->cy, c->N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->cz, c->N * sizeof(double)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->rhs, c->N * sizeof(double)));
    }
    return PARIS_OK;
}
