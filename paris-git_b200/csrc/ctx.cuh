// ctx.cuh -- the device-resident state behind a paris_handle_t and the
// internal entry points shared by the .cu files of the library.
#pragma once
#include <vector>
#include "common.cuh"

static constexpr int kRedBlocks = 1184;   // 148 SMs x 8: capacity of the partial-sum slots

// One level of the reference multigrid (DataMG/pMG/EMG of MGsolver.f90:26-30),
// interior-only arrays; the one-layer halo is resolved in the kernels
// (periodic wrap, zero at walls where ghost_MG_* never writes).
struct RefLevel {
    int n[3];
    long N;
    double* K;   // 8*N
    double* p;   // pMG
    double* e;   // EMG
};

// One level of the B200 multigrid: face coefficients (east/north/top of each
// cell) and work vectors, in T = float (inner cycle of the mixed solver) and
// double (the FP64 solver).
template <typename T>
struct FastLevel {
    int n[3];
    long N;
    T *cx, *cy, *cz;
    T *b, *x;
    T* x2;   // second iterate of the fused sweeps (they read one and write the other)
    void* tma = nullptr;   // FP32: tensor maps of the level for the TMA-staged sweep (mg_fast.cu)
    bool pairs = false;    // two consecutive sweeps run as one pass (k_rb_sweep4_cfg)
    bool rs = false;       // the last pre-smoothing sweep forms the coarse right-hand side (k_rb_sweep_rs)
    int merged = 0;        // FP32: the fused sweep with one barrier per step (1: 32x12 tiles, 2: 32x14)
    double omega = 1.0;    // relaxation factor of the red-black smoother, set by each solve
};

struct paris_ctx {
    paris_grid_desc d;
    int dev = 0;
    cudaStream_t stream = nullptr;
    Layout L;
    Bnd bnd;
    long N = 0;               // interior cells
    // metrics (index i+ng, i interior-relative), device copies
    double *dx = nullptr, *dxh = nullptr, *dy = nullptr, *dyh = nullptr, *dz = nullptr, *dzh = nullptr;
    double *xc = nullptr, *yc = nullptr, *zc = nullptr;   // cell centres x(i), y(j), z(k)
    double *xh = nullptr, *yh = nullptr, *zh = nullptr;   // face positions xh(i) (face i+1/2)
    std::vector<double> h_dx, h_dxh, h_dy, h_dyh, h_dz, h_dzh, h_x, h_y, h_z, h_xh, h_yh, h_zh;
    // ghosted fields (index PARIS_FIELD_*; VOF_FLAG/A/HEIGHT/PHASE kept apart)
    double* fld[PARIS_NFIELDS] = {};
    double* c2 = nullptr;          // second cvof buffer of the sweeps
    int8_t* flag = nullptr;        // vof_flag (ghosted)
    uint8_t* cg = nullptr;         // c_mask of the Weymouth-Yue sweeps
    double* height = nullptr;      // 6 ghosted fields
    int8_t* kflag = nullptr;       // kappaflag of the curvature passes
    double* vflux = nullptr;       // VOF sweeps: vof1/vof2/vof3 of the mixed cells (3 ghosted arrays, sparse)
    long* mixlist = nullptr;       // the mixed flux cells of the current sweep
    int* mixsegn = nullptr;        // their number
    long mixcap = 0;               // room in mixlist
    int* st_list = nullptr;        // interior mixed cells of the curvature passes
    int* st_count = nullptr;
    int* debris_count = nullptr;   // cells cleaned by a sweep of clean_debris method 3
    int32_t* i32stage = nullptr;   // staging for int32 host transfers
    // pressure equation, compact interior arrays (N each)
    double *cx = nullptr, *cy = nullptr, *cz = nullptr, *rhs = nullptr;
    double* A = nullptr;           // 8*N, reference layout, built on demand
    int have_matrix = 0;           // cx/cy/cz/rhs valid
    int A_valid = 0;               // A consistent with cx/cy/cz/rhs
    int A_from_upload = 0;         // A given by the caller (not rebuilt)
    double setup_dt = 0.0;
    // reductions
    double* red_part = nullptr;    // kRedBlocks partials * 4 slots
    int* err_host = nullptr;       // pinned and mapped: set by a kernel whose bounded wait ran out
    int* err_dev = nullptr;        // its device address
    double* red_host = nullptr;    // pinned and mapped
    double* red_host_dev = nullptr;   // its device address
    int red_nb = kRedBlocks;       // blocks of the last reduction launch
    int nsm = 148;
    std::vector<std::pair<const void*, int>> red_occ;   // kernel -> resident blocks per SM
    // multigrid hierarchies
    int ref_lmg = 0;
    std::vector<RefLevel> ref;     // index 1..LMG
    int fast_nl = 0;
    int fast_nuc = 0, fast_cf = 1, fast_ct = 0;   // sweeps on the levels fast_cf..fast_ct (0: nu1/nu2), set by each solve
    std::vector<FastLevel<float>> fl32;
    std::vector<FastLevel<double>> fl64;
    double* fast_r64 = nullptr;    // PCG vectors (N each)
    double* fast_d64 = nullptr;
    double* fast_q64 = nullptr;
    double* cg_scal = nullptr;     // device-side scalars of the CG loop (8 doubles, allocated at init)
    double* bx_part = nullptr;     // set around a preconditioning V-cycle: where its last finest-level
    int bx_blocks = 0;             // sweep writes the partials of r.z, and how many it wrote
    double* adj = nullptr;         // projection adjoint: 10 ghosted fields + N (allocated on first use)
    // asynchronous transfers: one stream per direction, a device staging copy
    // of each transferred field and the events that order them against `stream`
    cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
    double* stage_in[PARIS_NFIELDS] = {};
    double* stage_out[PARIS_NFIELDS] = {};
    cudaEvent_t ev_in_done[PARIS_NFIELDS] = {}, ev_in_free[PARIS_NFIELDS] = {};
    cudaEvent_t ev_out_ready[PARIS_NFIELDS] = {}, ev_out_free[PARIS_NFIELDS] = {};
    double* mom_tab = nullptr;     // momentum predictor: per-index QUICK coefficients and metric reciprocals
    int mom_tab_exact = 0;         // their reciprocals of k, 1-k, k-1, dx, dxh are exact (powers of two)
    double* mc_tmp = nullptr;      // momentum-conserving sweeps: advected fraction (two buffers),
    double* mc_tmp2 = nullptr;
    double* mc_work = nullptr;     // 3 ghosted work arrays (half fractions, momentum fluxes),
    double* mc_fv = nullptr;       // face velocity of a sweep, and flags / c_mask of the fraction
    int8_t* mc_flag = nullptr;
    uint8_t* mc_cg = nullptr;
    double* stats_part = nullptr;  // calcStats: PARIS_NSTATS slots of kRedBlocks partials (on first use)
    double* stats_out = nullptr;
    int64_t launches = 0;
    char err[512] = {0};
    // per-kernel event timing
    struct ProfRec {
        const char* name;
        long cells;
        int ev;   // index of the start event in evpool (stop = ev + 1)
    };
    int prof_on = 0;
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> evpool;
};


// Grid of a reduction kernel: one wave of resident blocks (at most
// kRedBlocks); records the block count for ctx_reduce_finish.
template <typename K>
unsigned red_grid(paris_ctx* c, K kernel, int threads) {
    const void* key = (const void*)kernel;
    int per = 0;
    for (auto& e : c->red_occ)
        if (e.first == key) per = e.second;
    if (!per) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess || per < 1) per = 1;
        c->red_occ.push_back({key, per});
    }
    int g = per * c->nsm;
    if (g > kRedBlocks) g = kRedBlocks;
    c->red_nb = g;
    return (unsigned)g;
}

// internal API (ctx.cu)
int ctx_alloc_field(paris_ctx* c, int field);
int ctx_ghost_fill(paris_ctx* c, double* f);         // do_all_ghost (periodic wrap)
int ctx_ghost_fill_i8(paris_ctx* c, int8_t* f);
int ctx_reduce_finish(paris_ctx* c, int nslots, double* out_host, int op_max = 0);
int ctx_ensure_matrix(paris_ctx* c);
int ctx_copy(paris_ctx* c, double* dst, const double* src, long n);   // device copy by a kernel

// vof.cu: the scratch of the VOF sweeps (flux arrays, mixed-cell list)
int vof_scratch(paris_ctx* c);
// mg_fast.cu: release the tensor maps of the FP32 levels
void mg_fast_free_maps(paris_ctx* c);
// vof.cu: SetVOFBC on the ghosts of a volume fraction and its flags (dry
// and wet walls fixed, periodic images, copies elsewhere), no clipping
__global__ void k_init_ghosts(double* __restrict__ c, int8_t* __restrict__ flag, const Layout L, const Bnd B,
                              const VofJet J, long G, double epsc);
// the 'jet' inflow parameters of the handle's descriptor
inline VofJet ctx_vof_jet(const paris_ctx* c) {
    VofJet J;
    J.type = c->d.inject_type;
    J.yc = c->d.jetcenter_yc;
    J.zc = c->d.jetcenter_zc;
    J.rliq = c->d.radius_liq_inject;
    J.rgas = c->d.radius_gas_inject;
    J.y = c->yc;
    J.z = c->zc;
    return J;
}
// vof.cu: one split sweep (swpz or swpr, then SetVOFBC, get_flags_and_clip
// and the ghosts) along d of the volume fraction src into dst with its flags;
// us: the face velocity of the sweep, cg: c_mask for the Weymouth-Yue sweep
int vof_sweep_dir(paris_ctx* c, int d, double dt, const double* src, double* dst, int8_t* flag, const double* us,
                  const uint8_t* cg);
// vof.cu: c_mask (vofmodules.f90:1295-1305) over total cells
__global__ void k_c_mask(const double* __restrict__ c, uint8_t* __restrict__ cg, long total);
// poisson.cu
int poisson_build_full_A(paris_ctx* c);
// mg_ref.cu
int mg_ref_solve(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* r);
// mg_fast.cu
int mg_fast_solve(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* r);
int mg_fast_solve_into(paris_ctx* c, const paris_solve_opts* o, paris_solve_result* r, const double* rhs, double* x);
