// debris.cu -- clean_debris (vofmodules.f90:2087-2234) on the device.
//
// Methods 1 and 2 decide every interior cell from the volume fractions as
// they were before the call, so one pass computes the new fractions into the
// second cvof buffer and a copy puts them back.  Method 3 cleans the mixed
// cells in place in the reference's k, j, i order: a cell sees the cells
// cleaned before it in the same sweep.  The sweep runs exactly in parallel
// by wavefronts t = i + 2j + 4k: no neighbour of a cell (offsets of at most
// one in each index) lies on the cell's own wavefront, and a neighbour that
// comes earlier in the k, j, i order has a smaller t, a later one a larger t
// (|di + 2 dj| < 4, so the sign of the t difference is that of dk, then dj,
// then di).  Two neighbours of a cell may share a wavefront with each other,
// but never with the cell, so the cells of one wavefront are independent and
// the wavefronts in increasing t reproduce the sequential sweep.  One block
// walks them, with a barrier between wavefronts.  Ghost cells keep their
// values during a sweep (the reference refreshes them only between sweeps).
#include "ctx.cuh"

namespace {

// methods 1 and 2: the new volume fractions of the interior into out
__global__ void k_debris_filter(const double* __restrict__ c, double* __restrict__ out, const Layout L, int method,
                                int ni, int nj, int nk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.n[0]) return;
    const long n = lidx(L, i, j, k);
    const double cc = c[n];
    int cf = 0;
    if (method == 1) {
        const int ph = cc > 0.5 ? 1 : -1;
        cf = ph;
        for (int i0 = -ni; i0 <= ni && cf != 0; i0++)
            for (int j0 = -nj; j0 <= nj && cf != 0; j0++)
                for (int k0 = -nk; k0 <= nk && cf != 0; k0++)
                    if (ph * (c[lidx(L, i + i0, j + j0, k + k0)] > 0.5 ? 1 : -1) == -1) cf = 0;
    } else {
        const double cvof_min = 0.1, sum_cvof_min = 0.3;
        const double sum1 = (double)((1 + ni * 2) * (1 + nj * 2) * (1 + nk * 2));
        double sum_cvof = 0.0;
        for (int i0 = -ni; i0 <= ni; i0++)
            for (int j0 = -nj; j0 <= nj; j0++)
                for (int k0 = -nk; k0 <= nk; k0++) sum_cvof = sum_cvof + c[lidx(L, i + i0, j + j0, k + k0)];
        if (cc < cvof_min && sum_cvof < sum_cvof_min) cf = -1;
        if (cc > 1.0 - cvof_min && sum_cvof > sum1 - sum_cvof_min) cf = 1;
    }
    double v = cc;
    if (cf == -1 && cc > 0.0) v = 0.0;
    else if (cf == 1 && cc < 1.0) v = 1.0;
    out[n] = v;
}

__global__ void k_debris_copy_back(double* __restrict__ c, const double* __restrict__ src, const Layout L) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n[0]) return;
    const long n = lidx(L, i, blockIdx.y, blockIdx.z);
    c[n] = src[n];
}

constexpr int kDebrisThreads = 1024;

// method 3: one sweep over the wavefronts; *cleaned gets the number of cells
// cleaned
__global__ void __launch_bounds__(kDebrisThreads) k_debris_sweep(double* __restrict__ c, int8_t* __restrict__ flag,
                                                                 const Layout L, double epsc, int* cleaned) {
    __shared__ int s_count;
    if (threadIdx.x == 0) s_count = 0;
    const int n0 = L.n[0], n1 = L.n[1], n2 = L.n[2];
    const int tmax = (n0 - 1) + 2 * (n1 - 1) + 4 * (n2 - 1);
    const int jw = n0 / 2 + 1;   // j values per k on one wavefront, at most
    int mine = 0;
    __syncthreads();
    for (int t = 0; t <= tmax; t++) {
        // k with some j in [0, n1) and i = t - 2j - 4k in [0, n0)
        const int klo = max(0, (t - (n0 - 1) - 2 * (n1 - 1) + 3) / 4), khi = min(n2 - 1, t / 4);
        const int cells = (khi - klo + 1) * jw;
        for (int q = threadIdx.x; q < cells; q += blockDim.x) {
            const int k = klo + q / jw;
            const int r = t - 4 * k;   // i + 2j
            const int jlo = max(0, (r - (n0 - 1) + 1) / 2);
            const int j = jlo + q % jw;
            const int i = r - 2 * j;
            if (j >= n1 || i < 0 || i >= n0) continue;
            const long n = lidx(L, i, j, k);
            if (flag[n] != 2) continue;
            int nposit = 0;
            for (int m = -1; m <= 1; m++)
                for (int p = -1; p <= 1; p++)
                    for (int l = -1; l <= 1; l++)
                        if (flag[lidx(L, i + m, j + p, k + l)] == 2) nposit++;
            if (nposit < 6) {
                if (!(c[n] < 0.5 - epsc)) { c[n] = 1.0; flag[n] = 1; }
                else { c[n] = 0.0; flag[n] = 0; }
                mine++;
            }
        }
        __syncthreads();
    }
    if (mine) atomicAdd(&s_count, mine);
    __syncthreads();
    if (threadIdx.x == 0) *cleaned = s_count;
}

// get_flags_and_clip on the whole array, ghosts included
__global__ void k_flags_clip_all(double* __restrict__ c, int8_t* __restrict__ flag, long total, double epsc) {
    const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (n >= total) return;
    const double v = c[n];
    if (v <= epsc) { flag[n] = 0; c[n] = 0.0; }
    else if (v >= 1.0 - epsc) { flag[n] = 1; c[n] = 1.0; }
    else flag[n] = 2;
}

}  // namespace

extern "C" int paris_clean_debris(paris_handle_t c, int32_t method, int32_t neighbours, int32_t* sweeps) {
    if (!c || method < 1 || method > 3 || neighbours < 0 || neighbours > c->L.ng) {
        if (c) ctx_set_error(c, "clean_debris: method %d with %d neighbours (methods 1-3, at most Ng)", method,
                             neighbours);
        return PARIS_BAD_ARGS;
    }
    cudaSetDevice(c->dev);
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_CVOF));
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_VOF_FLAG));
    const Layout& L = c->L;
    double* cv = c->fld[PARIS_FIELD_CVOF];
    const dim3 g(div_up(L.n[0], 128), L.n[1], L.n[2]);
    int nsw = 0;
    if (method != 3) {
        const int ni = neighbours, nj = neighbours, nk = L.n[2] == 2 ? 0 : neighbours;
        PARIS_LAUNCH_N(c, "clean_debris", c->N, k_debris_filter, g, 128, 0, cv, c->c2, L, method, ni, nj, nk);
        PARIS_LAUNCH(c, k_debris_copy_back, g, 128, 0, cv, c->c2, L);
        nsw = 1;
    } else {
        int* d_cleaned = c->debris_count;   // written by every sweep
        int cleaned_mix = 0;
        bool all_clean = false;
        int st = PARIS_OK;
        for (int itr = 1; !all_clean && itr <= 11 && st == PARIS_OK; itr++) {
            nsw = itr;
            int cl = 0;
            PARIS_LAUNCH_N(c, "clean_debris", c->N, k_debris_sweep, 1, kDebrisThreads, 0, cv, c->flag, L, c->d.epsc,
                           d_cleaned);
            if (cudaMemcpyAsync(&cl, d_cleaned, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess) {
                st = PARIS_CUDA_ERROR;
                break;
            }
            cleaned_mix += cl;   // accumulates over the sweeps, as in the reference
            all_clean = cleaned_mix == 0;
            if (!all_clean) {
                // do_all_ghost(cvof), get_flags_and_clip(cvof, vof_flag)
                if (ctx_ghost_fill(c, cv) != PARIS_OK) { st = PARIS_CUDA_ERROR; break; }
                PARIS_LAUNCH(c, k_flags_clip_all, (unsigned)div_up(L.total, 256L), 256, 0, cv, c->flag, L.total,
                             c->d.epsc);
            }
        }
        if (st != PARIS_OK) {
            ctx_set_error(c, "clean_debris: a device transfer failed");
            return st;
        }
    }
    if (sweeps) *sweeps = nsw;
    return PARIS_OK;
}
