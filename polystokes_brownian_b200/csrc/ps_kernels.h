// ps_kernels.h -- host-side engine state shared by the .cu translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "ps_internal.h"

namespace ps {

// Per-replica MINRES scalars (device resident).  Paige & Saunders recurrences
// in the preconditioned form used by PETSc KSPMINRES.
struct MinresScal {
    double beta, oldb, dbar, epsln, phibar, cs, sn, np, ttol, alfa;
    double up_oldeps, up_delta, up_ginv, up_phi;   // pending w/x update
    double sinv;                                     // 1 / beta for the next matvec
    int it, done, reason, pending;
};

// Reduction block table entry: a contiguous range of one replica's segment.
struct RBlk { int rep; int start; int len; };

struct RedTable {
    int nblk = 0;
    RBlk *d_blk = nullptr;       // per block
    int *d_first = nullptr;      // per replica: first block
    int *d_count = nullptr;      // per replica: number of blocks
    int *d_counter = nullptr;    // per replica: arrival counter (reset by last block)
    double *d_part = nullptr;    // nblk x 4 partial sums
};

// Per-replica scalars of the lubricated resistance-form PCG.
struct PcgScal {
    double rz, alpha, beta, tol, err;
    int it, done, reason, pad;
};

struct Engine {
    int R = 0;
    int precision = PS_PREC_FP64;
    std::vector<ps_desc> desc;
    std::vector<Seg> segs;
    long ntot = 0, ncoll = 0, nvec = 0, ntop = 0, nvel = 0;
    int maxNp = 0;
    bool any_lub = false, any_shell_schur = false, any_kT = false, any_mmhi = false;
    bool any_aa_ref = false, any_aa_rpy = false;   // monomer HI replicas in the reference's / RPY pair scalars

    Seg *d_segs = nullptr;
    int *d_vec_offs = nullptr, *d_top_offs = nullptr, *d_vel_offs = nullptr, *d_bead_offs = nullptr;

    // state
    double *d_x = nullptr, *d_q = nullptr, *d_xpos0 = nullptr, *d_xn = nullptr;
    double4 *d_pos64 = nullptr;
    float4 *d_pos32 = nullptr, *d_pos32lo = nullptr;   // FP32 positions as hi + lo
    float *d_aa_te2 = nullptr;   // per replica: squared exact radius of the FP32 monomer kernel
    double *d_chain = nullptr;      // chain id per bead (monomers), -1-c for colloid c
    int *d_coll_rep = nullptr;      // replica of each colloid
    int *d_fresh = nullptr;         // per replica: 1 if it starts fresh (trap centres from its colloids)
    double *d_chs = nullptr;        // per colloid: its colloid-monomer HS sum (3 doubles)
    double *d_time = nullptr;       // per replica time
    double *d_ktrap = nullptr;      // per replica (weaken_trap mutates it)
    double *d_trapinfo = nullptr;   // per replica: tstop, weaken_trap, unused

    // far-field pair work lists
    Tile *d_aa_tiles = nullptr, *d_ab_tiles = nullptr, *d_bb_tiles = nullptr;
    int n_aa_tiles = 0, n_ab_tiles = 0, n_bb_tiles = 0, nch_aa = 1, nch_bb = 1;
    long part_stride = 0;
    double *d_partAA = nullptr, *d_partAB = nullptr, *d_partBB = nullptr, *d_partBA = nullptr;
    long nba = 0;

    // reference-mode AB translational block and its carried state
    double *d_tab = nullptr, *d_stale = nullptr;
    int *d_aa_last = nullptr;       // per replica: (i,j) of the last AA pair, -1 if none

    // arrowhead Schur floor (shell path)
    long nschur = 0;
    double *d_delta = nullptr, *d_schurQ = nullptr, *d_schurL = nullptr;
    int *d_schur_reps = nullptr; int n_schur_reps = 0;
    int *d_ss_reps = nullptr; int n_ss_reps = 0;   // replicas whose stresslet block is solved densely
    // Schur Lanczos noise of shell replicas above the dense Schur limit (slip_vel.cpp:283-288, 351-477)
    int n_sl_reps = 0;
    int *d_sl_reps = nullptr;        // slot -> replica
    int *d_sl_skip = nullptr;        // per replica: 1 = skip in the operator applies of the Lanczos loop
    double *d_slV = nullptr;         // per slot: basis, (SL_KMAX + 1) x nc11 (the last row is the residual)
    double *d_slT = nullptr;         // per slot: alpha[SL_KMAX], beta[SL_KMAX]
    void *d_sl_sc = nullptr;         // per slot: scalars (b0, m, done, nneg)
    double *d_sl_u = nullptr, *d_sl_y = nullptr, *d_sl_y2 = nullptr;   // mobility-layout work vectors
    int n_ss_polish = 0;                           // replicas with colloids beyond the dense limit

    // bonds (per-bead CSR: partner, sign)
    int *d_bond_ptr = nullptr, *d_bond_nbr = nullptr;
    double *d_bond_sgn = nullptr;

    // cell list / pair lists
    int *d_cell = nullptr, *d_cell_start = nullptr, *d_cell_sorted = nullptr, *d_cell_count = nullptr;
    int *d_cell_big = nullptr, *d_cell_nbig = nullptr, *d_cell_tmp = nullptr;   // cells of more than 64 members
    long ncell_cap = 0;
    double *d_cellgeo = nullptr;     // per replica: org[3], size[3], nc[3] (as double), periodic
    long *d_cell_offs = nullptr;     // per replica: first cell
    long ncells = 0;
    bool need_cells = false;
    int *d_nbr_ptr = nullptr, *d_nbr = nullptr;   // CSR neighbour lists (i<j pairs per i)
    long nbr_cap = 0;
    int *d_nbr_count = nullptr;
    int *d_scan_sums = nullptr; long scan_cap = 0;   // block totals of exclusive_scan

    // lubrication
    double *d_lubtab = nullptr; int lub_nrow = 0;
    double *d_luby = nullptr, *d_lub_diag = nullptr, *d_tmp_vel = nullptr, *d_tmp_vel2 = nullptr;
    double *d_zlub = nullptr; long zlub_cap = 0;
    int *d_lub_ptr = nullptr, *d_lub_nbr = nullptr; long lub_cap = 0; long lub_npairs = 0;
    int *d_lub_cidx = nullptr;       // per symmetric-list entry: its canonical pair index (-1: none)
    int *d_lubc_ptr = nullptr, *d_lubc_nbr = nullptr; int2 *d_lub_pairs = nullptr; long lubc_cap = 0;  // canonical
    // pair-space lubricated solve: per pair K^{1/2} and preconditioner blocks (12x12), CG vectors (12 per pair)
    double *d_pS = nullptr, *d_pP = nullptr, *d_py_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double *d_ppart = nullptr; long pair_cap = 0;
    // pair blocks d_pS / d_pP hold the setup of the current staged positions
    // (cleared by every packing, table change and reallocation)
    bool ps_setup_valid = false;
    // stresslet unknowns of replicas without a dense stresslet inverse (mobility layout), per-bead partials
    double *d_sv[5] = {nullptr, nullptr, nullptr, nullptr, nullptr}, *d_sbead[2] = {nullptr, nullptr};
    // pair-space MINRES: 10 pair-storage vectors (3 r, 3 w, v, z, x, Az), 9 stresslet-storage vectors, scalars
    double *d_pmp[10] = {}, *d_pms[9] = {}, *d_ppart2 = nullptr;
    MinresScal *d_pmr = nullptr;
    bool any_indef = false;          // some replica's far field may be indefinite: pair-space MINRES

    // trajectory observables (observe.cu)
    double *d_obs_acc = nullptr, *d_obs_prev = nullptr, *d_obs_ring = nullptr, *d_obs_msd = nullptr;
    int *d_obs_hasprev = nullptr;
    unsigned long long *d_obs_hb = nullptr, *d_obs_ht = nullptr, *d_obs_msdn = nullptr;
    int obs_nbins = 0, obs_lags = 0;
    double obs_bmax = 0.0, obs_tmax = 0.0;
    long obs_n = 0;
    RedTable red_bead;               // over beads (pair-space sums by lower bead)

    // Krylov workspace
    RedTable red;                    // over saddle vectors
    RedTable red_top;                // over mobility vectors
    RedTable red_vel;                // over velocity vectors (lubricated PCG)
    // lubricated structured solve: inverse stresslet blocks, PCG state (velocity layout)
    double *d_ssinv = nullptr; long n_ssinv = 0;
    PcgScal *d_pcg = nullptr;
    double *d_pV = nullptr, *d_pr = nullptr, *d_pz = nullptr, *d_pp = nullptr, *d_ps = nullptr, *d_pAp = nullptr,
           *d_pg = nullptr;
    double *d_pu = nullptr, *d_py = nullptr, *d_pu2 = nullptr, *d_py2 = nullptr;   // mobility layout
    double *d_D = nullptr, *d_z = nullptr, *d_v = nullptr, *d_xw = nullptr;
    double *d_Rr[3] = {nullptr, nullptr, nullptr}, *d_W[3] = {nullptr, nullptr, nullptr};
    MinresScal *d_mr = nullptr;
    double *d_sinv = nullptr;
    int *d_nactive = nullptr;
    int *h_nactive = nullptr;        // pinned

    // step workspace
    double *d_rhs = nullptr, *d_X = nullptr, *d_Xd = nullptr, *d_Xdet = nullptr, *d_Wn = nullptr;
    double *d_vdn = nullptr, *d_vdc = nullptr, *d_vb = nullptr, *d_up = nullptr, *d_ud = nullptr;
    double *d_drift = nullptr, *d_sb = nullptr, *d_fext = nullptr, *d_fb = nullptr, *d_wr = nullptr;
    double *d_tmp_top = nullptr, *d_tmp_top2 = nullptr;
    double *d_ref_r = nullptr, *d_ref_d = nullptr;   // iterative refinement: residual, correction (allocated on first use)
    int *d_pm_cnt = nullptr;                         // pair-space MINRES: items finished per replica (first use)
    uint64_t seed = 12345, step_counter = 0;
    uint64_t *d_rseed = nullptr, *d_rstep = nullptr;   // per-replica Philox key and step counter

    // Lanczos workspace
    int lz_kmax = 0;
    double *d_lzV = nullptr, *d_lzT = nullptr, *d_lzw = nullptr, *d_lzq = nullptr;
    double *d_lzs = nullptr;

    cudaStream_t side = nullptr;                   // far field: small pair kernels beside the monomer kernel
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaStream_t side2 = nullptr;                  // Lanczos convergence checks beside the next basis vectors
    cudaEvent_t ev_fork2 = nullptr, ev_chk = nullptr;
    void *h_spec = nullptr;                        // pinned copy of the checks' outcomes
};

// monomer column chunk width of the far-field AA kernels: process-wide (every
// context of the process chunks a replica the same way, which keeps a replica's
// arithmetic independent of its batch); set by ps_autotune
extern int g_aa_chunk_cols;
int set_aa_chunking(Engine &E, int cols);

// true when p is host memory (pageable or pinned): the C-ABI accepts host
// pointers for state and noise arguments and copies them itself
bool is_host_ptr(const void *p);

// observe.cu: OBS_K doubles per bead -- bond count, sum b (3), sum |b|, sum |b|^2,
// increment count, sum db (3); trap count, sum d (3), sum |d|, sum |d|^2, sum d_a^2 (3); pad
constexpr int OBS_K = 20;
int obs_reset(Engine &E, int nbins, double bond_max, double trap_max, int lags);
int obs_sample(Engine &E, cudaStream_t st);
int obs_read(Engine &E, ps_obs_out *out, cudaStream_t st);

// rpy.cu
// done: optional per-replica int flags (base pointer + byte stride); replicas
// whose flag is nonzero are skipped by every kernel of the apply.
// skip_aa: leave out the monomer-monomer pairs -- exact for every colloid row,
// and for the monomer rows when the monomer inputs are zero.
void apply_operator(Engine &E, int mode, const double *x, double *y, const double *scale, bool fp32, cudaStream_t st,
                    const void *done = nullptr, int done_stride = 0, bool skip_aa = false);
int time_pairs(Engine &E, int which, int reps, const double *u, double *ms, cudaStream_t st);
int fma_peak(int fp64, double *tflops, cudaStream_t st);
int rsqrt_check(const double *a, long n, unsigned long long *max_ulp, cudaStream_t st);
// lub.cu
void lub_apply(Engine &E, const double *x_saddle, double *y_vel, cudaStream_t st);
void lub_apply_vel(Engine &E, const double *u_vel, double *y_vel, cudaStream_t st);
int lub_build(Engine &E, cudaStream_t st);
int lub_diag(Engine &E, cudaStream_t st);
int lub_noise(Engine &E, const double *z, double *rhs, cudaStream_t st);
// stage.cu
int stage_pack(Engine &E, cudaStream_t st);
int stage_pairs(Engine &E, cudaStream_t st);
int stage_rhs(Engine &E, int drift, const double *fext, double *rhs, cudaStream_t st);
int stage_assemble(Engine &E, cudaStream_t st);
int stage_schur(Engine &E, cudaStream_t st);
int diag_saddle(Engine &E, double *d, cudaStream_t st);
int pair_list(Engine &E, int which, int32_t *pi, int32_t *pj, int64_t maxp, int64_t *count, cudaStream_t st);
// out[0..n] = exclusive scan of in[0..n-1], out[n] = total (pairs.cu)
int exclusive_scan(Engine &E, const int *in, int *out, long n, cudaStream_t st);
int slip_noise(Engine &E, const double *fb, double *W, const ps_sqrt_opts *o, ps_sqrt_result *res, cudaStream_t st);
int step_all(Engine &E, const ps_step_inputs *in, ps_step_result *res, cudaStream_t st);
// krylov.cu
int minres_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res, cudaStream_t st);
// solve.cu
int structured_solve(Engine &E, const double *b, double *x, const ps_ksp_opts *o, ps_ksp_result *res,
                     cudaStream_t st);
int schur_lanczos_noise(Engine &E, const double *fb, const double *ymcm, double *W, int *nneg, cudaStream_t st);
int lanczos_sqrt(Engine &E, const double *z, double *w, const ps_sqrt_opts *o, ps_sqrt_result *res, cudaStream_t st);
int build_red_table(Engine &E, RedTable &T, int layout);   // 0 saddle, 1 top, 2 velocity, 3 beads
void free_red_table(RedTable &T);
void seg_dot(Engine &E, RedTable &T, const double *a, const double *b, double *out_per_rep, cudaStream_t st);

void set_error(const std::string &s);
#define PS_CK(call)                                                                    \
    do {                                                                               \
        cudaError_t _e = (call);                                                       \
        if (_e != cudaSuccess) {                                                       \
            ps::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));         \
            return PS_ERR_CUDA;                                                        \
        }                                                                              \
    } while (0)

}  // namespace ps
