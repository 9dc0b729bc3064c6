// st.cu -- height functions, curvature and the CSF surface force on the B200:
// get_all_heights with get_heights_pass1/2 (surface_tension.f90:185-448),
// get_all_curvatures_pop with curvature_pop_pass1/2 and get_average
// (:620-1052) and surfaceForce (paris.f90:2862-2957).  Built with -fmad=false.
//
// Pass 1 of the heights runs one thread per pure cell.  In the reference's
// loop order the lower end of a stack (searching up) is visited before its
// upper end, and the upper end then finds the height already set.  So a
// downward search writes only what no lower start can write: a partial
// height at the domain edge, or a full height whose other end is a ghost
// cell.  Every other write comes from exactly one start, so no two threads
// write the same height.
#include "ctx.cuh"
#include "st_geom.cuh"

namespace {
constexpr int kNdepth = 3;
constexpr int kBigint = 100;
constexpr double kHalfBig = 50.0;
constexpr double kUncomputed = 2e6;
constexpr double kKappaMax = 4.0;
constexpr int kNfoundMin = 6;
constexpr double kTiny = 1e-50;
constexpr int kUndecided = 5;
constexpr int kUncomputable = 4;
}  // namespace

struct StArgs {
    const double* c;
    const int8_t* f;
    double* H;        // 6 ghosted arrays
    Layout L;
    long stride[3];   // 1, pitch, plane
};

__device__ inline double* Hidx(const StArgs& a, int index1) { return a.H + (long)(index1 - 1) * a.L.total; }

__device__ inline long at(const StArgs& a, const int c[3]) {
    return lidx(a.L, c[0], c[1], c[2]);
}

// Fortran index of interior-relative coordinate c: c + ng + 1
__device__ inline double fidx(const StArgs& a, int c) { return (double)(c + a.L.ng + 1); }

// get_heights_pass1 for one direction; grid = interior cells
__global__ void k_heights_pass1(const StArgs a, int d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= a.L.n[0]) return;
    long n = lidx(a.L, i, j, k);
    int f = a.f[n];
    if (f / 2 != 0) return;
    for (int sign = -1; sign <= 1; sign += 2) {
        int c[3] = {i, j, k};
        int normalsign = (2 * f - 1) * sign;
        int index = 2 * d + 1 + (-normalsign + 1) / 2;
        double* H = Hidx(a, index);
        int other = 1 - f;
        int climitp1 = (sign < 0 ? 0 : a.L.n[d] - 1) + sign;
        double hp = 0.0;
        int s = 0, c0 = c[d], c1 = c0 + sign * kNdepth;
        while (true) {
            long cc = at(a, c);
            int fc = a.f[cc];
            bool same = s > 0 && fc == f;
            hp = hp + (a.c[cc] - 0.5) * normalsign;
            bool abandon = same || fc == other || c[d] == climitp1 || s == 2 * kNdepth;
            if (!abandon) {
                s++;
                c[d] += sign;
                continue;
            }
            if (fc == other) {
                // full height; a downward search leaves interior stacks to their lower end
                if (sign < 0 && c[d] != climitp1) break;
                hp = hp + (2 * kNdepth - s) * (a.c[cc] - 0.5) * normalsign;
                while (c[d] != c0 - sign) {
                    H[at(a, c)] = hp + fidx(a, c1) - fidx(a, c[d]);
                    c[d] -= sign;
                }
            } else if (c[d] == climitp1) {
                hp = hp + (-a.c[cc] + 0.5) * normalsign;
                c[d] -= sign;
                H[at(a, c)] = hp + (double)(kBigint * s);
            }
            break;
        }
    }
}

// get_heights_pass2 for one direction; one thread per column (l, m)
__global__ void k_heights_pass2(const StArgs a, int d, int t2, int t3) {
    int l = blockIdx.x * blockDim.x + threadIdx.x, m = blockIdx.y;
    if (l >= a.L.n[t2] || m >= a.L.n[t3]) return;
    int c[3];
    c[t2] = l; c[t3] = m;
    for (int sign = -1; sign <= 1; sign += 2)
        for (int index = 2 * d + 1; index <= 2 * d + 2; index++) {
            double* H = Hidx(a, index);
            int cb = sign < 0 ? 0 : a.L.n[d] - 1;
            c[d] = cb;
            double hb = H[at(a, c)];
            if (!(hb > kHalfBig && hb < 1e6)) continue;
            c[d] = cb + sign;
            double ha = H[at(a, c)];
            c[d] = cb;
            if (ha < kHalfBig) {
                H[at(a, c)] = ha + sign;
            } else if (ha > kHalfBig && ha < 1e6) {
                int sbelow = (int)floorf(__fdiv_rn((float)(hb + kHalfBig), (float)kBigint));
                hb = hb - kBigint * sbelow;
                int sabove = (int)floorf(__fdiv_rn((float)(ha + kHalfBig), (float)kBigint));
                ha = ha - kBigint * sabove;
                if (sabove + sbelow - 1 <= 2 * kNdepth + 1) {
                    int c0 = cb - (sbelow - 1) * sign;
                    double cmiddle = fidx(a, c0) + sign * (sabove + sbelow - 1) * 0.5;
                    c[d] = cb + 2 * sign;
                    while (c[d] != c0 - sign) {
                        H[at(a, c)] = ha + hb + cmiddle - fidx(a, c[d]);
                        c[d] -= sign;
                    }
                }
            }
        }
}

__global__ void k_heights_reset(double* __restrict__ H, long total) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < total && H[t] > kHalfBig) H[t] = 2e6;
}

__global__ void k_fill_d(double* __restrict__ f, double v, long n) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < n) f[t] = v;
}

static StArgs st_args(paris_ctx* c) {
    StArgs a;
    a.c = c->fld[PARIS_FIELD_CVOF];
    a.f = c->flag;
    a.H = c->height;
    a.L = c->L;
    a.stride[0] = 1; a.stride[1] = c->L.pitch; a.stride[2] = c->L.plane;
    return a;
}

static int heights(paris_ctx* c) {
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_HEIGHT));
    const Layout& L = c->L;
    StArgs a = st_args(c);
    PARIS_LAUNCH(c, k_fill_d, div_up(6 * L.total, 256), 256, 0, c->height, 2e6, 6 * L.total);
    dim3 g(div_up(L.n[0], 128), L.n[1], L.n[2]);
    for (int d = 0; d < 3; d++) PARIS_LAUNCH_N(c, "heights_pass1", c->N, k_heights_pass1, g, 128, 0, a, d);
    for (int q = 0; q < 6; q++) PARIS_CHECK(ctx_ghost_fill(c, c->height + q * L.total));
    for (int d = 0; d < 3; d++) {
        int t2 = (d + 1) % 3, t3 = (d + 2) % 3;
        if (t2 > t3) { int t = t2; t2 = t3; t3 = t; }
        PARIS_LAUNCH_N(c, "heights_pass2", (long)L.n[t2] * L.n[t3], k_heights_pass2,
                       dim3(div_up(L.n[t2], 128), L.n[t3]), 128, 0, a, d, t2, t3);
        PARIS_LAUNCH(c, k_heights_reset, div_up(2 * L.total, 256), 256, 0, c->height + 2 * d * L.total,
                     2 * L.total);
    }
    for (int q = 0; q < 6; q++) PARIS_CHECK(ctx_ghost_fill(c, c->height + q * L.total));
    return PARIS_OK;
}

extern "C" int paris_get_all_heights(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    PARIS_CHECK(heights(c));
    return PARIS_OK;
}

// ---- curvature -----------------------------------------------------------
struct CurvArgs {
    StArgs s;
    double* kap;      // ghosted
    int8_t* kf;       // ghosted kappaflag
    const int* list;  // interior mixed cells (layout index, int32)
    const int* count;
    int do_rotation, use_full_heights;
    double epsc;
};

__device__ inline void block27(const StArgs& a, long n, double st[27]) {
    for (int e = -1; e <= 1; e++)
        for (int b = -1; b <= 1; b++)
            for (int q = -1; q <= 1; q++) st[(q + 1) + 3 * (b + 1) + 9 * (e + 1)] = a.c[n + q + b * a.L.pitch + e * a.L.plane];
}

__device__ inline void decode(const Layout& L, long n, int& i, int& j, int& k) {
    long r = n - L.off;   // interior-relative linear offset, may be negative in ghosts
    long kk = (r + L.plane * L.ng) / L.plane - L.ng;
    r -= kk * L.plane;
    long jj = (r + L.pitch * L.ng) / L.pitch - L.ng;
    r -= jj * L.pitch;
    i = (int)r; j = (int)jj; k = (int)kk;
}

// get_local_heights (surface_tension.f90:490-589); h[m+1][n+1]
__device__ int local_heights(const StArgs& a, int i, int j, int k, const double mxyz[3], int tr[3], double h[3][3],
                             double pts[stg::kNpos][3], int& nposit) {
    int nfound = 0;
    nposit = 0;
    for (int l = 0; l < 3; l++) {
        int d = tr[l];
        int si = d == 0, sj = d == 1, sk = d == 2;
        int index = mxyz[d] > 0 ? 2 * d + 1 : 2 * d + 2;
        const double* H = Hidx(a, index);
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) h[p][q] = 2e6;
        nfound = 0;
        for (int m = -1; m <= 1; m++)
            for (int nn = -1; nn <= 1; nn++) {
                int p[3];
                if (d == 0) { p[0] = i; p[1] = m + j; p[2] = nn + k; }
                else if (d == 1) { p[0] = m + i; p[1] = j; p[2] = nn + k; }
                else { p[0] = m + i; p[1] = nn + j; p[2] = k; }
                double hv = H[lidx(a.L, p[0], p[1], p[2])];
                bool got = false;
                if (hv < 1e6) {
                    h[m + 1][nn + 1] = hv;
                    got = true;
                } else {
                    for (int s = 1; s <= a.L.ng && !got; s++) {
                        double hu = H[lidx(a.L, p[0] + si * s, p[1] + sj * s, p[2] + sk * s)];
                        if (hu < 1e6) { h[m + 1][nn + 1] = hu + s; got = true; continue; }
                        double hd = H[lidx(a.L, p[0] - si * s, p[1] - sj * s, p[2] - sk * s)];
                        if (hd < 1e6) { h[m + 1][nn + 1] = hd - s; got = true; }
                    }
                }
                if (got) {
                    nfound++;
                    int q = nposit++;
                    double hl = h[m + 1][nn + 1];
                    pts[q][0] = hl * si + fidx(a, p[0]) - fidx(a, i);
                    pts[q][1] = hl * sj + fidx(a, p[1]) - fidx(a, j);
                    pts[q][2] = hl * sk + fidx(a, p[2]) - fidx(a, k);
                }
            }
        if (nfound == 9) {
            int t[3], nn = 1;
            for (int m = 0; m < 3; m++)
                if (m != d) t[nn++] = m;
            tr[0] = d; tr[1] = t[1]; tr[2] = t[2];
            return 9;
        }
    }
    return nfound;
}

// curvature_pop_pass1 (surface_tension.f90:827-932)
__device__ double curv_pass1(const CurvArgs& A, long n, int& nfound_out) {
    const StArgs& a = A.s;
    int i, j, k;
    decode(a.L, n, i, j, k);
    double st[27], mxyz[3], h[3][3], pts[stg::kNpos][3], bp[stg::kNpos][3], origin[3], mv[3], av[6], w[stg::kNpos];
    int tr[3], nposit;
    double kappa = kUncomputed;
    block27(a, n, st);
    plic::mycs(st, mxyz);
    stg::orientation(mxyz, tr);
    int nfound = local_heights(a, i, j, k, mxyz, tr, h, pts, nposit);
    if (fabs(mxyz[0]) < kTiny && fabs(mxyz[1]) < kTiny && fabs(mxyz[2]) < kTiny) {
        nfound_out = 21;
        return kappa;
    }
    if (nfound == 9 && A.use_full_heights) {
        double a1 = h[2][1] - 2.0 * h[1][1] + h[0][1];
        double a2 = h[1][2] - 2.0 * h[1][1] + h[1][0];
        double a3 = (h[2][2] - h[0][2] - h[2][0] + h[0][0]) / 4.0;
        double a4 = (h[2][1] - h[0][1]) / 2.0;
        double a5 = (h[1][2] - h[1][0]) / 2.0;
        kappa = (a1 * (1.0 + a5 * a5) + a2 * (1.0 + a4 * a4) - 2.0 * a3 * a4 * a5) / pow(1.0 + a4 * a4 + a5 * a5, 1.5);
        kappa = copysign(1.0, mxyz[tr[0]]) * kappa;
        nfound_out = 0;
        return kappa;
    }
    stg::find_cut_area_centroid(st, a.c[n], origin);
    nfound = stg::ind_pos_sorted_add(origin, pts, bp, nposit);
    mv[0] = mxyz[tr[1]]; mv[1] = mxyz[tr[2]]; mv[2] = mxyz[tr[0]];
    if (nfound > kNfoundMin + 1) {
        for (int q = 0; q < nfound; q++) {
            pts[q][0] = bp[q][tr[1]] - origin[tr[1]];
            pts[q][1] = bp[q][tr[2]] - origin[tr[2]];
            pts[q][2] = bp[q][tr[0]] - origin[tr[0]];
            w[q] = 1.0;
        }
        w[0] = 1e2 * plic::area3d(mxyz, a.c[n]);
        double ks;
        if (stg::parabola_fit_rot(pts, w, mv, nfound, av, ks, A.do_rotation, A.epsc)) {
            kappa = 2.0 * (av[0] * (1.0 + av[4] * av[4]) + av[1] * (1.0 + av[3] * av[3]) - av[2] * av[3] * av[4]) /
                    pow(1.0 + av[3] * av[3] + av[4] * av[4], 1.5);
            kappa = ks * kappa;
            nfound_out = -nfound;
            return kappa;
        }
        nfound_out = 16;
        return kappa;
    }
    nfound_out = nfound + 1;
    return kappa;
}

// curvature_pop_pass2 (surface_tension.f90:959-1052)
__device__ double curv_pass2(const CurvArgs& A, long n, int& nfound_out) {
    const StArgs& a = A.s;
    double st[27], mxyz[3], origin[3], mv[3], av[6], w[stg::kNpos], pts[stg::kNpos][3];
    int tr[3];
    double kappa = kUncomputed;
    block27(a, n, st);
    plic::fd32(st, mxyz);
    stg::orientation(mxyz, tr);
    if (fabs(mxyz[0]) < kTiny && fabs(mxyz[1]) < kTiny && fabs(mxyz[2]) < kTiny) {
        nfound_out = 21;
        return kappa;
    }
    stg::find_cut_area_centroid(st, a.c[n], origin);
    mv[0] = mxyz[tr[1]]; mv[1] = mxyz[tr[2]]; mv[2] = mxyz[tr[0]];
    int nposit = 0;
    for (int m = -1; m <= 1; m++)
        for (int nn = -1; nn <= 1; nn++)
            for (int l = -1; l <= 1; l++) {
                long q = n + m + nn * a.L.pitch + l * a.L.plane;
                double wg = a.c[q] * (1.0 - a.c[q]);
                if (a.f[q] == 2 && wg > 0.0) {
                    double sq[27], cen[3], off[3] = {(double)m, (double)nn, (double)l};
                    block27(a, q, sq);
                    stg::new_find_cut_area_centroid(sq, a.c[q], cen);
                    double fitq[3];
                    for (int s = 0; s < 3; s++) fitq[s] = cen[s] + off[s];
                    pts[nposit][0] = fitq[tr[1]] - origin[tr[1]];
                    pts[nposit][1] = fitq[tr[2]] - origin[tr[2]];
                    pts[nposit][2] = fitq[tr[0]] - origin[tr[0]];
                    w[nposit] = 1.0;
                    nposit++;
                }
            }
    if (nposit < 6) {
        nfound_out = nposit + 10;
        return kappa;
    }
    double ks;
    if (!stg::parabola_fit_rot(pts, w, mv, nposit, av, ks, A.do_rotation, A.epsc)) {
        nfound_out = 16;
        return kappa;
    }
    double sq = sqrt(1.0 + av[3] * av[3] + av[4] * av[4]);
    kappa = 2.0 * (av[0] * (1.0 + av[4] * av[4]) + av[1] * (1.0 + av[3] * av[3]) - av[2] * av[3] * av[4]) / (sq * sq * sq);
    kappa = ks * kappa;
    nfound_out = -nposit - 50;
    return kappa;
}

// interior mixed cells (flag 2), warp-aggregated append
__global__ void k_mixed_interior(const int8_t* __restrict__ f, const Layout L, int* list, int* count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    long n = i < L.n[0] ? lidx(L, i, j, k) : 0;
    bool mixed = i < L.n[0] && f[n] == 2;
    unsigned m = __ballot_sync(0xffffffffu, mixed);
    if (!m) return;
    int lane = threadIdx.x & 31, leader = __ffs(m) - 1, base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (mixed) list[base + __popc(m & ((1u << lane) - 1u))] = (int)n;
}

__global__ void k_curv_init(double* __restrict__ kap, int8_t* __restrict__ kf, const int8_t* __restrict__ f,
                            const Layout L, long total) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= total) return;
    kap[t] = kUncomputed;
    kf[t] = kUndecided;
}

__global__ void __launch_bounds__(128) k_curv_pass1(const CurvArgs A) {
    int cnt = *A.count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        long n = A.list[q];
        int nf;
        double kap = curv_pass1(A, n, nf);
        A.kap[n] = kap;
        if (nf == 0) A.kf[n] = 0;
        if (nf > -50 && nf < 0) A.kf[n] = 1;
    }
}

// get_average over the 3x3x3 cells with kappaflag 0 or 1
__global__ void k_curv_average(const CurvArgs A) {
    int cnt = *A.count;
    const Layout& L = A.s.L;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        long n = A.list[q];
        if (A.kf[n] <= 1) continue;
        int s = 0;
        double kappa = 0.0;
        for (int m = -1; m <= 1; m++)
            for (int nn = -1; nn <= 1; nn++)
                for (int l = -1; l <= 1; l++) {
                    long p = n + m + nn * L.pitch + l * L.plane;
                    if (A.kf[p] < 2) { s++; kappa = kappa + A.kap[p]; }
                }
        if (s > 0) {
            A.kap[n] = kappa / s;
            A.kf[n] = 2;
        }
    }
}

__global__ void __launch_bounds__(128) k_curv_pass2(const CurvArgs A) {
    int cnt = *A.count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        long n = A.list[q];
        if (A.kf[n] <= 2) continue;
        int nf;
        double kap = curv_pass2(A, n, nf);
        if (nf > 0) A.kf[n] = kUncomputable;
        else { A.kap[n] = kap; A.kf[n] = 3; }
    }
}

// pure interior cells are UNCOMPUTABLE
__global__ void k_curv_pure(const int8_t* __restrict__ f, int8_t* __restrict__ kf, const Layout L) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.n[0]) return;
    long n = lidx(L, i, j, k);
    if (f[n] != 2) kf[n] = kUncomputable;
}

__global__ void k_curv_clip(double* __restrict__ kap, const int8_t* __restrict__ kf, long total) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= total || kf[t] >= kUncomputable) return;
    double k = kap[t];
    if (fabs(k) > kKappaMax) k = copysign(1.0, k) * kKappaMax;
    kap[t] = k;
}

static int curvatures(paris_ctx* c) {
    const Layout& L = c->L;
    PARIS_CHECK(ctx_alloc_field(c, PARIS_FIELD_KAPPA));
    if (!c->kflag) PARIS_CUDA_TRY(c, cudaMalloc(&c->kflag, L.total));
    if (!c->st_list) {
        PARIS_CUDA_TRY(c, cudaMalloc(&c->st_list, c->N * sizeof(int)));
        PARIS_CUDA_TRY(c, cudaMalloc(&c->st_count, sizeof(int)));
    }
    CurvArgs A;
    A.s = st_args(c);
    A.kap = c->fld[PARIS_FIELD_KAPPA];
    A.kf = c->kflag;
    A.list = c->st_list;
    A.count = c->st_count;
    A.do_rotation = c->d.do_rotation;
    A.use_full_heights = c->d.use_full_heights;
    A.epsc = c->d.epsc;
    dim3 g(div_up(L.n[0], 128), L.n[1], L.n[2]);
    PARIS_CUDA_TRY(c, cudaMemsetAsync(c->st_count, 0, sizeof(int), c->stream));
    PARIS_LAUNCH(c, k_mixed_interior, g, 128, 0, c->flag, L, c->st_list, c->st_count);
    PARIS_LAUNCH(c, k_curv_init, div_up(L.total, 256), 256, 0, A.kap, A.kf, c->flag, L, L.total);
    unsigned gg = c->nsm * 8;
    PARIS_LAUNCH_N(c, "curvature_pass1", 0L, k_curv_pass1, gg, 128, 0, A);
    PARIS_CHECK(ctx_ghost_fill(c, A.kap));
    PARIS_CHECK(ctx_ghost_fill_i8(c, A.kf));
    PARIS_LAUNCH(c, k_curv_average, gg, 128, 0, A);
    PARIS_LAUNCH_N(c, "curvature_pass2", 0L, k_curv_pass2, gg, 128, 0, A);
    PARIS_LAUNCH(c, k_curv_pure, g, 128, 0, c->flag, A.kf, L);
    PARIS_CHECK(ctx_ghost_fill(c, A.kap));
    PARIS_CHECK(ctx_ghost_fill_i8(c, A.kf));
    PARIS_LAUNCH(c, k_curv_clip, div_up(L.total, 256), 256, 0, A.kap, A.kf, L.total);
    return PARIS_OK;
}

extern "C" int paris_get_all_curvatures(paris_handle_t c, double* kappa_host) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    if (!c->height) {
        ctx_set_error(c, "get_all_curvatures: call paris_get_all_heights first");
        return PARIS_BAD_ARGS;
    }
    PARIS_CHECK(curvatures(c));
    if (kappa_host) return paris_gpu_download(c, PARIS_FIELD_KAPPA, kappa_host);
    return PARIS_OK;
}

// surfaceForce (paris.f90:2862-2957): du,dv,dw += CSF force on faces with a
// jump of cvof, curvature = mean of the valid neighbour values / dx(nx)
__global__ void k_surface_force(const double* __restrict__ cv, const double* __restrict__ kap,
                                const double* __restrict__ rho, double* __restrict__ du, double* __restrict__ dv,
                                double* __restrict__ dw, const Layout L, const Bnd B, const double* __restrict__ dxh,
                                const double* __restrict__ dyh, const double* __restrict__ dzh, double deltax,
                                double sigma, double epsc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= L.n[0]) return;
    const int g = L.ng;
    long n = lidx(L, i, j, k);
    int c[3] = {i, j, k};
    double* out[3] = {du, dv, dw};
    const double* dh[3] = {dxh, dyh, dzh};
    long st[3] = {1, L.pitch, L.plane};
    for (int d = 0; d < 3; d++) {
        if (c[d] == L.n[d] - 1 && !B.per[d]) continue;   // is..ieu
        long o = st[d];
        if (fabs(cv[n + o] - cv[n]) > epsc / 1e1) {
            int cnt = 0;
            double kappa = 0.0;
            if (kap[n + o] < 1e6) { kappa = kappa + kap[n + o]; cnt++; }
            if (kap[n] < 1e6) { kappa = kappa + kap[n]; cnt++; }
            if (cnt > 0) {
                kappa = kappa / (deltax * cnt);
                out[d][n] = out[d][n] - kappa * sigma * (2.0 / dh[d][c[d] + g]) * (cv[n + o] - cv[n]) / (rho[n + o] + rho[n]);
            }
        }
    }
}

extern "C" int paris_surface_force(paris_handle_t c) {
    if (!c) return PARIS_BAD_ARGS;
    cudaSetDevice(c->dev);
    // surfaceForce calls get_all_curvatures itself (paris.f90:2874)
    if (!c->height) PARIS_CHECK(heights(c));
    PARIS_CHECK(curvatures(c));
    for (int f : {PARIS_FIELD_DU, PARIS_FIELD_DV, PARIS_FIELD_DW}) PARIS_CHECK(ctx_alloc_field(c, f));
    const Layout& L = c->L;
    double deltax = c->h_dx[c->d.nx - 1];   // dx(nx)
    PARIS_LAUNCH_N(c, "surface_force", c->N, k_surface_force, dim3(div_up(L.n[0], 128), L.n[1], L.n[2]), 128, 0,
                   c->fld[PARIS_FIELD_CVOF], c->fld[PARIS_FIELD_KAPPA], c->fld[PARIS_FIELD_RHO],
                   c->fld[PARIS_FIELD_DU], c->fld[PARIS_FIELD_DV], c->fld[PARIS_FIELD_DW], L, c->bnd, c->dxh, c->dyh,
                   c->dzh, deltax, c->d.sigma, c->d.epsc);
    return PARIS_OK;
}
