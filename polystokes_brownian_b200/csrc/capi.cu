// capi.cu -- extern "C" entry points of include/polystokes_b200.h: context
// construction (segment table, work lists, device buffers) and thin wrappers
// over the engine functions.
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>
#include "ps_internal.h"
#include "ps_kernels.h"

unsigned long long ps_launch_count = 0;

struct ps_ctx {
    ps::Engine E;
};

namespace ps {
static thread_local std::string g_err;
void set_error(const std::string &s) { g_err = s; }
}  // namespace ps

using ps::Engine;



static cudaStream_t S(void *p) { return (cudaStream_t)p; }

#define TRY_ALLOC(ptr, bytes)                                                                  \
    do {                                                                                       \
        size_t _b = (size_t)(bytes);                                                           \
        if (_b == 0) _b = 8;                                                                   \
        cudaError_t _e = cudaMalloc((void **)&(ptr), _b);                                      \
        if (_e != cudaSuccess) {                                                               \
            ps::set_error(std::string("cudaMalloc ") + #ptr + ": " + cudaGetErrorString(_e));  \
            return PS_ERR_NOMEM;                                                               \
        }                                                                                      \
        cudaMemset((void *)(ptr), 0, _b);                                                      \
    } while (0)

template <class T>
static int upload(T *&dst, const std::vector<T> &v)
{
    TRY_ALLOC(dst, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) PS_CK(cudaMemcpy(dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return PS_OK;
}

static void free_engine(Engine &E)
{
    void *ptrs[] = {E.d_segs, E.d_vec_offs, E.d_top_offs, E.d_vel_offs, E.d_bead_offs, E.d_x, E.d_q, E.d_xpos0,
                    E.d_xn, E.d_pos64, E.d_pos32, E.d_pos32lo, E.d_aa_te2, E.d_chain, E.d_coll_rep, E.d_chs, E.d_time, E.d_ktrap, E.d_trapinfo,
                    E.d_aa_tiles, E.d_ab_tiles, E.d_bb_tiles, E.d_partAA, E.d_partAB, E.d_partBB, E.d_partBA,
                    E.d_tab, E.d_stale, E.d_aa_last, E.d_delta, E.d_schurQ, E.d_schurL, E.d_schur_reps, E.d_ss_reps,
                    E.d_bond_ptr, E.d_bond_nbr, E.d_bond_sgn, E.d_cell, E.d_cell_start, E.d_cell_sorted,
                    E.d_cell_count, E.d_cellgeo, E.d_cell_offs, E.d_nbr_ptr, E.d_nbr, E.d_nbr_count, E.d_lubtab,
                    E.d_luby, E.d_lub_diag, E.d_lub_ptr, E.d_lub_nbr, E.d_lub_cidx, E.d_tmp_vel, E.d_tmp_vel2, E.d_zlub, E.d_D, E.d_z, E.d_v, E.d_xw, E.d_Rr[0],
                    E.d_Rr[1], E.d_Rr[2], E.d_W[0], E.d_W[1], E.d_W[2], E.d_mr, E.d_sinv, E.d_nactive,
                    E.d_rhs, E.d_X, E.d_Xd, E.d_Xdet, E.d_Wn, E.d_vdn, E.d_vdc, E.d_vb, E.d_up, E.d_ud,
                    E.d_drift, E.d_sb, E.d_fext, E.d_fb, E.d_wr, E.d_tmp_top, E.d_tmp_top2, E.d_lzV, E.d_lzT,
                    E.d_lzw, E.d_lzq, E.d_lzs, E.d_ssinv, E.d_pcg, E.d_pV, E.d_pr, E.d_pz, E.d_pp, E.d_ps,
                    E.d_pAp, E.d_pg, E.d_pu, E.d_py, E.d_pu2, E.d_py2, E.d_rseed, E.d_rstep,
                    E.d_lubc_ptr, E.d_lubc_nbr, E.d_lub_pairs, E.d_pS, E.d_pP, E.d_py_[0], E.d_py_[1], E.d_py_[2],
                    E.d_py_[3], E.d_py_[4], E.d_ppart, E.d_scan_sums, E.d_sv[0], E.d_sv[1], E.d_sv[2],
                    E.d_sv[3], E.d_sv[4], E.d_sbead[0], E.d_sbead[1], E.d_ppart2, E.d_pmr,
                    E.d_pmp[0], E.d_pmp[1], E.d_pmp[2], E.d_pmp[3], E.d_pmp[4], E.d_pmp[5], E.d_pmp[6],
                    E.d_pmp[7], E.d_pmp[8], E.d_pmp[9], E.d_pms[0], E.d_pms[1], E.d_pms[2], E.d_pms[3],
                    E.d_pms[4], E.d_pms[5], E.d_pms[6], E.d_pms[7], E.d_pms[8], E.d_obs_acc, E.d_obs_prev,
                    E.d_obs_ring, E.d_obs_msd, E.d_obs_hasprev, E.d_obs_hb, E.d_obs_ht, E.d_obs_msdn,
                    E.d_sl_reps, E.d_sl_skip, E.d_slV, E.d_slT, E.d_sl_sc, E.d_sl_u, E.d_sl_y, E.d_sl_y2,
                    E.d_cell_big, E.d_cell_nbig, E.d_cell_tmp, E.d_ref_r, E.d_ref_d, E.d_pm_cnt, E.d_fresh};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (E.h_nactive) cudaFreeHost(E.h_nactive);
    if (E.ev_fork) cudaEventDestroy(E.ev_fork);
    if (E.ev_join) cudaEventDestroy(E.ev_join);
    if (E.side) cudaStreamDestroy(E.side);
    if (E.ev_fork2) cudaEventDestroy(E.ev_fork2);
    if (E.ev_chk) cudaEventDestroy(E.ev_chk);
    if (E.side2) cudaStreamDestroy(E.side2);
    if (E.h_spec) cudaFreeHost(E.h_spec);
    ps::free_red_table(E.red);
    ps::free_red_table(E.red_top);
    ps::free_red_table(E.red_vel);
    ps::free_red_table(E.red_bead);
}

static int build(Engine &E, const ps_desc *descs, int R, int precision)
{
    E.R = R;
    E.precision = precision;
    E.desc.assign(descs, descs + R);
    E.segs.resize(R);
    long bead = 0, coll = 0, vec = 0, top = 0, vel = 0, schur = 0, ba = 0, cells = 0, ssinv = 0;
    std::vector<int> bead_offs(R + 1), vec_offs(R + 1), top_offs(R + 1), vel_offs(R + 1);
    std::vector<long> cell_offs(R + 1);
    std::vector<Tile> aa, ab, bb;
    std::vector<int> schur_reps, ss_reps, sl_reps;
    long slv = 0;
    int ss_polish = 0;
    const int TR = 128;
    int kTpos = 0, kTzero = 0;
    for (int r = 0; r < R; r++) {
        const ps_desc &d = descs[r];
        if (d.Nm < 0 || d.Nc < 0 || d.Nm + d.Nc < 1 || d.beta <= 0 || d.dt <= 0) {
            ps::set_error("invalid descriptor (Nm, Nc, beta, dt) for replica " + std::to_string(r));
            return PS_ERR_ARG;
        }
        if (d.Npoly * d.Nmono_per_chain != d.Nm && d.Nm > 0) {
            ps::set_error("Npoly * Nmono_per_chain != Nm for replica " + std::to_string(r));
            return PS_ERR_ARG;
        }
        if (d.lub_on) E.any_lub = true;
        Seg s;
        memset(&s, 0, sizeof s);
        s.Nm = d.Nm; s.Nc = d.Nc; s.Np = d.Nm + d.Nc;
        s.bead_off = (int)bead; s.coll_off = (int)coll; s.vec_off = (int)vec; s.top_off = (int)top; s.vel_off = (int)vel;
        s.nm3 = 3 * d.Nm; s.nc3 = 3 * d.Nc; s.nc5 = 5 * d.Nc; s.nc6 = 6 * d.Nc; s.nc11 = 11 * d.Nc;
        s.nm3nc3 = s.nm3 + s.nc3; s.nm3nc6 = s.nm3 + s.nc6; s.nm3nc11 = s.nm3 + s.nc11;
        s.n = s.nm3nc11 + s.nm3nc6;
        s.mm_HI = d.mm_HI; s.chain_HI = d.chain_HI; s.ab_mode = d.ab_mode; s.box_on = d.box_on;
        s.fene = d.fene; s.mono_ev = d.mono_ev; s.lub_on = d.lub_on; s.tether = d.tether; s.aa_mode = d.aa_mode;
        s.beta = d.beta; s.beta_inv = 1.0 / d.beta; s.kT = d.kT; s.dt = d.dt; s.epsilon = d.epsilon;
        s.kbond = d.kbond; s.r0 = d.r0; s.Lmax = d.Lmax;
        for (int k = 0; k < 3; k++) s.L[k] = d.box_on ? d.box[k] : 0.0;
        if (d.box_on)
            for (int k = 0; k < 3; k++)
                if (!(d.box[k] > 0)) { ps::set_error("Box lengths must be positive"); return PS_ERR_ARG; }
        double kp = d.hs_kpref > 0 ? d.hs_kpref : 1.0;
        s.hs_k = (d.hs_kmode == 1) ? kp / (d.dt * d.beta) : kp / d.dt;
        double pref = std::pow(2.0, 1.0 / 6.0);
        s.rverl[0] = (float)(0.05 + 2 * d.beta); s.rverl[1] = (float)(1.5 + d.beta); s.rverl[2] = 2.5f;
        s.sig[0] = (float)(2. * d.beta); s.sig[1] = (float)(1. + d.beta); s.sig[2] = 2.0f;
        for (int k = 0; k < 3; k++) s.rcut[k] = (float)(pref * (double)s.sig[k]);
        s.lub_gap = d.lub_gap;
        s.lub_bonded = d.lub_bonded;
        s.nper = d.Nmono_per_chain > 0 ? d.Nmono_per_chain : 1;
        s.ss_off = -1;
        s.nch_aa = std::max(1, (d.Nm + ps::g_aa_chunk_cols - 1) / ps::g_aa_chunk_cols);
        s.nch_bb = std::max(1, std::min(BB_MAX_CHUNKS, (d.Nc + BB_CHUNK_COLS - 1) / BB_CHUNK_COLS));
        if (d.aa_mode == PS_AA_RPY) {
            double b = d.beta, b2 = b * b;
            const double c[8] = {1.5, -b2, 0.75, 0.5 * b2, 1.0 / b, -0.1875 / b2, 1.0 / b, -0.28125 / b2};
            for (int k = 0; k < 8; k++) s.aa_c[k] = (float)c[k];
        } else {
            const double c[8] = {0.375, -2.0, 0.75, -0.5, -1.0, 0.375, 1.0, -0.28125};
            for (int k = 0; k < 8; k++) s.aa_c[k] = (float)c[k];
        }
        // crossover of slip_vel.cpp:283-288 (POLYSTOKES_LANCZOS_NC; 0 forces the Lanczos noise)
        int lnc = d.lanczos_nc >= 0 ? d.lanczos_nc : 64;
        s.shell_schur = (!d.mm_HI && d.Nc > 0 && s.nc11 <= lnc && s.nc11 <= PS_MAX_NC11_SCHUR);
        s.sl_slot = -1; s.sl_off = 0;
        if (!d.mm_HI && d.Nc > 0 && !s.shell_schur && d.kT > 0) {
            s.sl_slot = (int)sl_reps.size(); s.sl_off = (int)slv; sl_reps.push_back(r);
            slv += (long)(SL_KMAX + 1) * s.nc11;
        }
        if (s.shell_schur) { s.schur_off = (int)schur; schur += (long)s.nc11 * s.nc11; schur_reps.push_back(r); }
        if (d.Nc > 0) {
            if (s.nc5 <= 64) { ss_reps.push_back(r); s.ss_off = (int)ssinv; ssinv += (long)s.nc5 * s.nc5; }
            else { ss_polish++; E.any_indef = true; }   // colloid suspensions: far-field FTS indefinite near contact
        }
        // the reference's own monomer pair scalars make the far-field mobility indefinite
        if (d.mm_HI && ((d.Nm >= 2 && d.aa_mode == PS_AA_REFERENCE) || (d.Nm >= 1 && d.Nc >= 1 && d.ab_mode == PS_AB_REFERENCE))) {
            E.any_indef = true;
        }
        // tiles
        s.n_mtiles = (d.Nm + TR - 1) / TR;
        s.ba_off = (int)ba;
        if (d.Nc > 0) ba += (long)s.n_mtiles * d.Nc;
        for (int t = 0; t < s.n_mtiles; t++) {
            Tile tl = {r, t * TR, std::min(TR, d.Nm - t * TR), t};
            if (d.mm_HI && d.Nm >= 2) aa.push_back(tl);
            if (d.Nc > 0) ab.push_back(tl);
        }
        if (d.Nc >= 2)
            for (int t = 0; t * TR < d.Nc; t++) bb.push_back({r, t * TR, std::min(TR, d.Nc - t * TR), t});
        bead_offs[r] = (int)bead; vec_offs[r] = (int)vec; top_offs[r] = (int)top; vel_offs[r] = (int)vel;
        cell_offs[r] = cells;
        cells += CELL_CAP_PER_MONO * d.Nm + CELL_CAP_BASE;
        bead += s.Np; coll += d.Nc; vec += s.n; top += s.nm3nc11; vel += s.nm3nc6;
        E.maxNp = std::max(E.maxNp, s.Np);
        if (d.kT > 0) kTpos++; else kTzero++;
        if (d.mm_HI) E.any_mmhi = true;
        if (d.mm_HI && d.Nm >= 2) (d.aa_mode == PS_AA_RPY ? E.any_aa_rpy : E.any_aa_ref) = true;
        E.segs[r] = s;
    }
    if (kTpos && kTzero) {
        ps::set_error("a batch must not mix kT > 0 and kT == 0 replicas");
        return PS_ERR_UNSUPPORTED;
    }
    if (vec > (long)INT32_MAX / 2) { ps::set_error("batch too large"); return PS_ERR_TOO_LARGE; }
    E.any_kT = kTpos > 0;
    bead_offs[R] = (int)bead; vec_offs[R] = (int)vec; top_offs[R] = (int)top; vel_offs[R] = (int)vel;
    cell_offs[R] = cells;
    E.ntot = bead; E.ncoll = coll; E.nvec = vec; E.ntop = top; E.nvel = vel; E.nschur = schur; E.nba = ba;
    E.ncells = cells;
    E.need_cells = true;
    E.n_schur_reps = (int)schur_reps.size();
    E.any_shell_schur = E.n_schur_reps > 0;
    // heavy tiles first (columns per tile ~ N of the replica)
    auto by_cost = [&](const Tile &a, const Tile &b) {
        return E.segs[a.rep].Np > E.segs[b.rep].Np || (E.segs[a.rep].Np == E.segs[b.rep].Np && a.rep < b.rep);
    };
    std::stable_sort(aa.begin(), aa.end(), by_cost);
    std::stable_sort(bb.begin(), bb.end(), by_cost);
    E.n_aa_tiles = (int)aa.size(); E.n_ab_tiles = (int)ab.size(); E.n_bb_tiles = (int)bb.size();
    // grid extent in chunks: the largest per-replica chunk count
    E.nch_aa = 1; E.nch_bb = 1;
    for (auto &s : E.segs) { E.nch_aa = std::max(E.nch_aa, s.nch_aa); E.nch_bb = std::max(E.nch_bb, s.nch_bb); }
    E.part_stride = top;
    int rc;
    if ((rc = upload(E.d_segs, E.segs))) return rc;
    if ((rc = upload(E.d_vec_offs, vec_offs))) return rc;
    if ((rc = upload(E.d_top_offs, top_offs))) return rc;
    if ((rc = upload(E.d_vel_offs, vel_offs))) return rc;
    if ((rc = upload(E.d_bead_offs, bead_offs))) return rc;
    if ((rc = upload(E.d_cell_offs, cell_offs))) return rc;
    if ((rc = upload(E.d_aa_tiles, aa))) return rc;
    if ((rc = upload(E.d_ab_tiles, ab))) return rc;
    if ((rc = upload(E.d_bb_tiles, bb))) return rc;
    if ((rc = upload(E.d_schur_reps, schur_reps))) return rc;
    if ((rc = upload(E.d_ss_reps, ss_reps))) return rc;
    E.n_ss_reps = (int)ss_reps.size();
    E.n_sl_reps = (int)sl_reps.size();
    if (E.n_sl_reps) {
        std::vector<int> skip(R, 1);
        for (int r : sl_reps) skip[r] = 0;
        if ((rc = upload(E.d_sl_reps, sl_reps))) return rc;
        if ((rc = upload(E.d_sl_skip, skip))) return rc;
        TRY_ALLOC(E.d_slV, sizeof(double) * slv);
        TRY_ALLOC(E.d_slT, sizeof(double) * 2 * SL_KMAX * E.n_sl_reps);
        TRY_ALLOC(E.d_sl_sc, 32 * E.n_sl_reps);
        TRY_ALLOC(E.d_sl_u, sizeof(double) * top);
        TRY_ALLOC(E.d_sl_y, sizeof(double) * top);
        TRY_ALLOC(E.d_sl_y2, sizeof(double) * top);
    }
    E.n_ss_polish = ss_polish;
    // per-bead chain ids, colloid -> replica, bonds
    std::vector<double> chain(bead);
    std::vector<int> coll_rep(std::max<long>(coll, 1));
    std::vector<std::vector<std::pair<int, double>>> bl(bead);
    std::vector<int> aa_last(2 * R, -1);
    std::vector<double> trapinfo(3 * R), ktrap(R), tinit(R), stale(9 * R, 0.0);
    for (int r = 0; r < R; r++) {
        const ps_desc &d = descs[r];
        const Seg &s = E.segs[r];
        std::vector<int> cid(d.Nm);
        for (int i = 0; i < d.Npoly; i++)
            for (int j = 0; j < d.Nmono_per_chain; j++) {
                int k = i * d.Nmono_per_chain + j;
                if (k < d.Nm) cid[k] = i;
            }
        for (int m = 0; m < d.Nm; m++) chain[s.bead_off + m] = cid[m];
        for (int c = 0; c < d.Nc; c++) { chain[s.bead_off + d.Nm + c] = -1.0 - c; coll_rep[s.coll_off + c] = r; }
        // bonds (init.cpp:296-321), per bead in bond-index order
        int nbp = d.Nmono_per_chain - 1;
        auto add_bond = [&](int k, int j) {
            bl[s.bead_off + k].push_back({s.bead_off + j, -1.0});
            bl[s.bead_off + j].push_back({s.bead_off + k, +1.0});
        };
        for (int i = 0; i < d.Npoly; i++)
            for (int j = 0; j < nbp; j++) add_bond(i * d.Nmono_per_chain + j, i * d.Nmono_per_chain + j + 1);
        if (d.tether) {
            int cpc = d.Nc ? d.Npoly / d.Nc : 1;
            if (cpc < 1) cpc = 1;
            for (int i = 0; i < d.Npoly; i++) {
                int host = d.Nm + i / cpc;
                if (host >= s.Np) host = s.Np - 1;
                add_bond(i * d.Nmono_per_chain, host);
            }
        }
        // last non-skipped AA pair in (i<j) lexicographic order (mob.cpp:845-851)
        bool have = false;
        for (int i = d.Nm - 2; i >= 0 && !have; i--)
            for (int j = d.Nm - 1; j > i; j--)
                if (!(d.chain_HI && cid[i] == cid[j])) { aa_last[2 * r] = i; aa_last[2 * r + 1] = j; have = true; break; }
        trapinfo[3 * r] = d.tstart + d.trun;
        trapinfo[3 * r + 1] = d.weaken_trap;
        ktrap[r] = d.ktrap;
        tinit[r] = d.t0;
        for (int a = 0; a < 3; a++) stale[9 * r + 4 * a] = 1.0;   // fill_self leaves mob_a = I
    }
    std::vector<int> bptr(bead + 1, 0), bnbr;
    std::vector<double> bsgn;
    for (long b = 0; b < bead; b++) {
        bptr[b] = (int)bnbr.size();
        for (auto &p : bl[b]) { bnbr.push_back(p.first); bsgn.push_back(p.second); }
    }
    bptr[bead] = (int)bnbr.size();
    if ((rc = upload(E.d_chain, chain))) return rc;
    if ((rc = upload(E.d_coll_rep, coll_rep))) return rc;
    std::vector<int> fresh(R);
    for (int r = 0; r < R; r++) fresh[r] = descs[r].restart ? 0 : 1;
    if ((rc = upload(E.d_fresh, fresh))) return rc;
    if ((rc = upload(E.d_bond_ptr, bptr))) return rc;
    if ((rc = upload(E.d_bond_nbr, bnbr))) return rc;
    if ((rc = upload(E.d_bond_sgn, bsgn))) return rc;
    if ((rc = upload(E.d_aa_last, aa_last))) return rc;
    if ((rc = upload(E.d_trapinfo, trapinfo))) return rc;
    if ((rc = upload(E.d_ktrap, ktrap))) return rc;
    if ((rc = upload(E.d_time, tinit))) return rc;
    if ((rc = upload(E.d_stale, stale))) return rc;
    TRY_ALLOC(E.d_tab, sizeof(double) * 9 * R);
    TRY_ALLOC(E.d_rseed, sizeof(uint64_t) * R);
    TRY_ALLOC(E.d_rstep, sizeof(uint64_t) * R);
    // state
    TRY_ALLOC(E.d_x, sizeof(double) * 3 * bead);
    TRY_ALLOC(E.d_xn, sizeof(double) * 3 * bead);
    TRY_ALLOC(E.d_q, sizeof(double) * 4 * std::max<long>(coll, 1));
    TRY_ALLOC(E.d_xpos0, sizeof(double) * 3 * std::max<long>(coll, 1));
    TRY_ALLOC(E.d_chs, sizeof(double) * 3 * std::max<long>(coll, 1));
    TRY_ALLOC(E.d_pos64, sizeof(double4) * bead);
    TRY_ALLOC(E.d_pos32, sizeof(float4) * bead);
    TRY_ALLOC(E.d_pos32lo, sizeof(float4) * bead);
    TRY_ALLOC(E.d_aa_te2, sizeof(float) * std::max<long>(R, 1));
    // pair partials
    TRY_ALLOC(E.d_partAA, sizeof(double) * top * E.nch_aa);
    TRY_ALLOC(E.d_partAB, sizeof(double) * top);
    TRY_ALLOC(E.d_partBB, sizeof(double) * top * E.nch_bb);
    TRY_ALLOC(E.d_partBA, sizeof(double) * 11 * std::max<long>(ba, 1));
    TRY_ALLOC(E.d_delta, sizeof(double) * std::max<long>(schur, 1));
    TRY_ALLOC(E.d_schurQ, sizeof(double) * std::max<long>(schur, 1));
    TRY_ALLOC(E.d_schurL, sizeof(double) * std::max<long>(schur, 1));
    // cells and pair lists
    TRY_ALLOC(E.d_cell, sizeof(int) * bead);
    TRY_ALLOC(E.d_cell_start, sizeof(int) * (cells + 1));
    TRY_ALLOC(E.d_cell_count, sizeof(int) * (cells + 1));
    TRY_ALLOC(E.d_cell_sorted, sizeof(int) * bead);
    TRY_ALLOC(E.d_cell_big, sizeof(int) * (bead / 64 + 1));
    TRY_ALLOC(E.d_cell_nbig, sizeof(int));
    TRY_ALLOC(E.d_cell_tmp, sizeof(int) * bead);
    TRY_ALLOC(E.d_cellgeo, sizeof(double) * 20 * R);
    TRY_ALLOC(E.d_nbr_ptr, sizeof(int) * (bead + 1));
    TRY_ALLOC(E.d_lub_ptr, sizeof(int) * (bead + 1));
    TRY_ALLOC(E.d_lubc_ptr, sizeof(int) * (bead + 1));
    TRY_ALLOC(E.d_nbr_count, sizeof(int) * (bead + 1));
    E.scan_cap = (std::max<long>(bead, cells) + 4095) / 4096 + 8;
    TRY_ALLOC(E.d_scan_sums, sizeof(int) * E.scan_cap);
    E.nbr_cap = 16 * bead + 1024;
    TRY_ALLOC(E.d_nbr, sizeof(int) * E.nbr_cap);
    // Krylov
    TRY_ALLOC(E.d_D, sizeof(double) * vec);
    TRY_ALLOC(E.d_z, sizeof(double) * vec);
    TRY_ALLOC(E.d_v, sizeof(double) * vec);
    for (int k = 0; k < 3; k++) { TRY_ALLOC(E.d_Rr[k], sizeof(double) * vec); TRY_ALLOC(E.d_W[k], sizeof(double) * vec); }
    TRY_ALLOC(E.d_mr, sizeof(ps::MinresScal) * R);
    TRY_ALLOC(E.d_sinv, sizeof(double) * R);
    TRY_ALLOC(E.d_nactive, sizeof(int));
    PS_CK(cudaMallocHost(&E.h_nactive, sizeof(int)));
    // side stream for the far field's small pair kernels (monomer-colloid, colloid-colloid),
    // which run beside the monomer pair kernel; non-blocking so that the legacy default
    // stream does not serialise it, ordered by the fork and join events only
    PS_CK(cudaStreamCreateWithFlags(&E.side, cudaStreamNonBlocking));
    PS_CK(cudaEventCreateWithFlags(&E.ev_fork, cudaEventDisableTiming));
    PS_CK(cudaEventCreateWithFlags(&E.ev_join, cudaEventDisableTiming));
    // the Lanczos convergence checks run on their own stream beside the next basis vectors
    PS_CK(cudaStreamCreateWithFlags(&E.side2, cudaStreamNonBlocking));
    PS_CK(cudaEventCreateWithFlags(&E.ev_fork2, cudaEventDisableTiming));
    PS_CK(cudaEventCreateWithFlags(&E.ev_chk, cudaEventDisableTiming));
    PS_CK(cudaMallocHost(&E.h_spec, 16 * (size_t)std::max(E.R, 1)));
    if ((rc = ps::build_red_table(E, E.red, 0))) return rc;
    if ((rc = ps::build_red_table(E, E.red_top, 1))) return rc;
    // step workspace
    TRY_ALLOC(E.d_rhs, sizeof(double) * vec);
    TRY_ALLOC(E.d_X, sizeof(double) * vec);
    TRY_ALLOC(E.d_Xd, sizeof(double) * vec);
    TRY_ALLOC(E.d_Xdet, sizeof(double) * vec);
    TRY_ALLOC(E.d_Wn, sizeof(double) * top);
    TRY_ALLOC(E.d_fb, sizeof(double) * top);
    TRY_ALLOC(E.d_tmp_top, sizeof(double) * top);
    TRY_ALLOC(E.d_tmp_top2, sizeof(double) * top);
    double **velbufs[] = {&E.d_vdn, &E.d_vdc, &E.d_vb, &E.d_up, &E.d_ud, &E.d_drift, &E.d_sb, &E.d_fext, &E.d_wr,
                          &E.d_luby, &E.d_lub_diag, &E.d_tmp_vel, &E.d_tmp_vel2};
    for (double **p : velbufs) TRY_ALLOC(*p, sizeof(double) * vel);
    // lubricated structured solve
    if (E.any_lub || ss_polish) {
        E.n_ssinv = ssinv;
        TRY_ALLOC(E.d_ssinv, sizeof(double) * std::max<long>(ssinv, 1));
        TRY_ALLOC(E.d_pcg, sizeof(ps::PcgScal) * R);
        double **pv[] = {&E.d_pV, &E.d_pr, &E.d_pz, &E.d_pp, &E.d_ps, &E.d_pAp, &E.d_pg};
        for (double **p : pv) TRY_ALLOC(*p, sizeof(double) * vel);
        double **pt[] = {&E.d_pu, &E.d_py, &E.d_pu2, &E.d_py2};
        for (double **p : pt) TRY_ALLOC(*p, sizeof(double) * top);
        if ((rc = ps::build_red_table(E, E.red_vel, 2))) return rc;
        if ((rc = ps::build_red_table(E, E.red_bead, 3))) return rc;
        for (auto &p : E.d_sv) TRY_ALLOC(p, sizeof(double) * top);
        for (auto &p : E.d_sbead) TRY_ALLOC(p, sizeof(double) * bead);
        for (auto &p : E.d_pms) TRY_ALLOC(p, sizeof(double) * top);
        TRY_ALLOC(E.d_pmr, sizeof(ps::MinresScal) * R);
    }
    // Lanczos
    if (E.any_mmhi) {
        const int KM = 64;
        TRY_ALLOC(E.d_lzV, sizeof(double) * top * (KM + 1));
        TRY_ALLOC(E.d_lzq, sizeof(double) * top);
        TRY_ALLOC(E.d_lzT, sizeof(double) * ((KM + 1) * R * 3 + KM * R * 2 + R));
        TRY_ALLOC(E.d_lzs, 96 * R);          // Lanczos scalars, their snapshot, the checks' speculative outcomes
    }
    return PS_OK;
}

extern "C" {

const char *ps_last_error(void) { return ps::g_err.c_str(); }

int ps_ctx_create(const ps_desc *descs, int32_t nrep, int32_t precision, ps_ctx **out)
{
    if (!descs || nrep < 1 || !out) { ps::set_error("ps_ctx_create: bad arguments"); return PS_ERR_ARG; }
    if (precision != PS_PREC_FP64 && precision != PS_PREC_MIXED) { ps::set_error("bad precision"); return PS_ERR_ARG; }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { ps::set_error("no CUDA device"); return PS_ERR_CUDA; }
    ps_ctx *c = new ps_ctx();
    int rc = build(c->E, descs, nrep, precision);
    if (!rc) rc = ps_set_seed(c, c->E.seed);   // per-replica streams from the default seed
    if (rc) { free_engine(c->E); delete c; return rc; }
    *out = c;
    return PS_OK;
}

int ps_ctx_destroy(ps_ctx *ctx)
{
    if (!ctx) return PS_ERR_ARG;
    cudaDeviceSynchronize();
    free_engine(ctx->E);
    delete ctx;
    return PS_OK;
}

int ps_ctx_sizes(const ps_ctx *ctx, int64_t *o)
{
    if (!ctx || !o) return PS_ERR_ARG;
    const Engine &E = ctx->E;
    o[0] = E.ntot; o[1] = E.nvec; o[2] = E.ntop; o[3] = E.nvel; o[4] = E.ncoll; o[5] = E.R; o[6] = 0; o[7] = 0;
    return PS_OK;
}

int ps_ctx_offsets(const ps_ctx *ctx, int32_t rep, int64_t *o)
{
    if (!ctx || !o || rep < 0 || rep >= ctx->E.R) return PS_ERR_ARG;
    const Seg &s = ctx->E.segs[rep];
    o[0] = s.bead_off; o[1] = s.vec_off; o[2] = s.top_off; o[3] = s.vel_off;
    return PS_OK;
}

int ps_set_lub_table(ps_ctx *ctx, const double *tab, int32_t nrow, int32_t ncol)
{
    // rows of r2babc.dat: r/a then X11A X12A Y11A Y12A Y11B Y12B X11C X12C Y11C Y12C
    if (!ctx || !tab || nrow < 2 || ncol < 11) { ps::set_error("ps_set_lub_table: need >= 2 rows of 11 columns"); return PS_ERR_ARG; }
    for (int i = 1; i < nrow; i++)
        if (!(tab[i * ncol] > tab[(i - 1) * ncol])) { ps::set_error("ps_set_lub_table: r must increase"); return PS_ERR_ARG; }
    Engine &E = ctx->E;
    std::vector<double> t((size_t)nrow * 11);
    for (int i = 0; i < nrow; i++)
        for (int c = 0; c < 11; c++) t[(size_t)i * 11 + c] = tab[(size_t)i * ncol + c];
    if (E.d_lubtab) cudaFree(E.d_lubtab);
    E.d_lubtab = nullptr;
    E.ps_setup_valid = false;
    int rc = upload(E.d_lubtab, t);
    if (rc) return rc;
    E.lub_nrow = nrow;
    return PS_OK;
}

static uint64_t splitmix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

int ps_set_seed(ps_ctx *ctx, uint64_t seed)
{
    if (!ctx) return PS_ERR_ARG;
    Engine &E = ctx->E;
    E.seed = seed;
    E.step_counter = 0;
    std::vector<uint64_t> sd(E.R), zero(E.R, 0);
    for (int r = 0; r < E.R; r++) sd[r] = splitmix64(seed + (uint64_t)r);
    PS_CK(cudaMemcpy(E.d_rseed, sd.data(), sizeof(uint64_t) * E.R, cudaMemcpyHostToDevice));
    PS_CK(cudaMemcpy(E.d_rstep, zero.data(), sizeof(uint64_t) * E.R, cudaMemcpyHostToDevice));
    return PS_OK;
}

int ps_set_replica_seeds(ps_ctx *ctx, const uint64_t *seeds, const uint64_t *steps)
{
    if (!ctx || !seeds) return PS_ERR_ARG;
    Engine &E = ctx->E;
    PS_CK(cudaDeviceSynchronize());
    PS_CK(cudaMemcpy(E.d_rseed, seeds, sizeof(uint64_t) * E.R, cudaMemcpyHostToDevice));
    if (steps) PS_CK(cudaMemcpy(E.d_rstep, steps, sizeof(uint64_t) * E.R, cudaMemcpyHostToDevice));
    return PS_OK;
}

int ps_get_aux(ps_ctx *ctx, double *time, double *ktrap, double *xpos0, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    Engine &E = ctx->E;
    cudaStream_t st = S(stream);
    if (time) PS_CK(cudaMemcpyAsync(time, E.d_time, sizeof(double) * E.R, cudaMemcpyDefault, st));
    if (ktrap) PS_CK(cudaMemcpyAsync(ktrap, E.d_ktrap, sizeof(double) * E.R, cudaMemcpyDefault, st));
    if (xpos0 && E.ncoll) PS_CK(cudaMemcpyAsync(xpos0, E.d_xpos0, sizeof(double) * 3 * E.ncoll, cudaMemcpyDefault, st));
    PS_CK(cudaStreamSynchronize(st));
    return PS_OK;
}

int ps_set_aux(ps_ctx *ctx, const double *time, const double *ktrap, const double *xpos0, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    Engine &E = ctx->E;
    cudaStream_t st = S(stream);
    if (time) PS_CK(cudaMemcpyAsync(E.d_time, time, sizeof(double) * E.R, cudaMemcpyDefault, st));
    if (ktrap) PS_CK(cudaMemcpyAsync(E.d_ktrap, ktrap, sizeof(double) * E.R, cudaMemcpyDefault, st));
    if (xpos0 && E.ncoll) PS_CK(cudaMemcpyAsync(E.d_xpos0, xpos0, sizeof(double) * 3 * E.ncoll, cudaMemcpyDefault, st));
    PS_CK(cudaStreamSynchronize(st));
    return PS_OK;
}

int ps_obs_reset(ps_ctx *ctx, int32_t nbins, double bond_max, double trap_max, int32_t lags)
{
    if (!ctx) return PS_ERR_ARG;
    return ps::obs_reset(ctx->E, nbins, bond_max, trap_max, lags);
}

int ps_observe(ps_ctx *ctx, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    return ps::obs_sample(ctx->E, S(stream));
}

int ps_obs_read(ps_ctx *ctx, ps_obs_out *out, void *stream)
{
    if (!ctx || !out) return PS_ERR_ARG;
    return ps::obs_read(ctx->E, out, S(stream));
}

int ps_get_replica_steps(ps_ctx *ctx, uint64_t *steps)
{
    if (!ctx || !steps) return PS_ERR_ARG;
    PS_CK(cudaDeviceSynchronize());
    PS_CK(cudaMemcpy(steps, ctx->E.d_rstep, sizeof(uint64_t) * ctx->E.R, cudaMemcpyDeviceToHost));
    return PS_OK;
}

// index of the first non-finite value of v[0, n), or -1; the exponent test runs
// over the whole array without a branch (it vectorises), the search only on failure
static long first_nonfinite(const double *v, long n)
{
    uint64_t bad = 0;
    for (long i = 0; i < n; i++) {
        uint64_t u;
        std::memcpy(&u, v + i, sizeof u);
        bad |= (uint64_t)(((u >> 52) & 0x7ff) == 0x7ff);
    }
    if (!bad) return -1;
    for (long i = 0; i < n; i++)
        if (!std::isfinite(v[i])) return i;
    return -1;
}

// trap centres from the colloids of the replicas that start fresh (Stokes.cpp:279-287)
__global__ void k_trap_centres(long ncoll, const int *__restrict__ coll_rep, const Seg *__restrict__ segs,
                               const int *__restrict__ fresh, const double *__restrict__ x, double *__restrict__ xpos0)
{
    pdl_enter();
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoll) return;
    const int r = coll_rep[c];
    if (!fresh[r]) return;
    const Seg &s = segs[r];
    const long b = s.bead_off + s.Nm + (c - s.coll_off);
    for (int d = 0; d < 3; d++) xpos0[3 * c + d] = x[3 * b + d];
}

__global__ void k_quat_identity(long ncoll, double *__restrict__ q)
{
    pdl_enter();
    const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoll) return;
    q[4 * c] = 1.0; q[4 * c + 1] = 0.0; q[4 * c + 2] = 0.0; q[4 * c + 3] = 0.0;
}

int ps_set_state(ps_ctx *ctx, const double *x, const double *q, void *stream)
{
    if (!ctx || !x) return PS_ERR_ARG;
    Engine &E = ctx->E;
    cudaStream_t st = S(stream);
    // host inputs are scanned before anything is copied or launched: a non-finite
    // coordinate would otherwise travel through the cell grid and every pair kernel
    if (ps::is_host_ptr(x)) {
        const long i = first_nonfinite(x, 3 * E.ntot);
        if (i >= 0) {
            ps::set_error("non-finite position at index " + std::to_string(i));
            return PS_ERR_ARG;
        }
    }
    if (q && ps::is_host_ptr(q)) {
        const long i = first_nonfinite(q, 4 * E.ncoll);
        if (i >= 0) {
            ps::set_error("non-finite quaternion at index " + std::to_string(i));
            return PS_ERR_ARG;
        }
    }
    PS_CK(cudaMemcpyAsync(E.d_x, x, sizeof(double) * 3 * E.ntot, cudaMemcpyDefault, st));
    const int thr = 128;
    const unsigned nbc = (unsigned)((E.ncoll + thr - 1) / thr);
    if (q) PS_CK(cudaMemcpyAsync(E.d_q, q, sizeof(double) * 4 * E.ncoll, cudaMemcpyDefault, st));
    else if (E.ncoll) ps_launch(k_quat_identity, nbc, thr, 0, st, E.ncoll, E.d_q);
    // trap centres from the colloids on a fresh start (Stokes.cpp:279-287), one launch for the batch
    if (E.ncoll)
        ps_launch(k_trap_centres, nbc, thr, 0, st, E.ncoll, E.d_coll_rep, E.d_segs, E.d_fresh, E.d_x,
                E.d_xpos0);
    PS_CK(cudaGetLastError());
    int rc = ps::stage_pack(E, st);
    return rc;
}

int ps_get_state(ps_ctx *ctx, double *x, double *q, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    Engine &E = ctx->E;
    cudaStream_t st = S(stream);
    if (x) PS_CK(cudaMemcpyAsync(x, E.d_x, sizeof(double) * 3 * E.ntot, cudaMemcpyDefault, st));
    if (q && E.ncoll) PS_CK(cudaMemcpyAsync(q, E.d_q, sizeof(double) * 4 * E.ncoll, cudaMemcpyDefault, st));
    if (ps::is_host_ptr(x) || ps::is_host_ptr(q)) PS_CK(cudaStreamSynchronize(st));   // host copies complete on return
    return PS_OK;
}

int ps_set_time(ps_ctx *ctx, double t)
{
    if (!ctx) return PS_ERR_ARG;
    std::vector<double> tv(ctx->E.R, t);
    PS_CK(cudaMemcpy(ctx->E.d_time, tv.data(), sizeof(double) * tv.size(), cudaMemcpyHostToDevice));
    return PS_OK;
}

int ps_build_pairs(ps_ctx *ctx, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    return ps::stage_pairs(ctx->E, S(stream));
}

int ps_pair_list(ps_ctx *ctx, int32_t which, int32_t *pi, int32_t *pj, int64_t maxp, int64_t *count, void *stream)
{
    if (!ctx || which < 0 || which > 2) return PS_ERR_ARG;
    if (which == 2 && !ctx->E.any_lub) { ps::set_error("no replica has lubrication on"); return PS_ERR_STATE; }
    return ps::pair_list(ctx->E, which, pi, pj, maxp, count, S(stream));
}

int ps_rhs(ps_ctx *ctx, int32_t drift, const double *fext, double *rhs, void *stream)
{
    if (!ctx || !rhs || (drift && !fext)) return PS_ERR_ARG;
    return ps::stage_rhs(ctx->E, drift, fext, rhs, S(stream));
}

int ps_assemble(ps_ctx *ctx, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    int rc = ps::stage_assemble(ctx->E, S(stream));
    if (rc) return rc;
    return ps::stage_schur(ctx->E, S(stream));
}

int ps_matmult(ps_ctx *ctx, const double *x, double *y, void *stream)
{
    if (!ctx || !x || !y) return PS_ERR_ARG;
    ps::apply_operator(ctx->E, 0, x, y, nullptr, ctx->E.precision == PS_PREC_MIXED, S(stream));
    PS_CK(cudaGetLastError());
    return PS_OK;
}

int ps_mobility_apply(ps_ctx *ctx, const double *u, double *y, void *stream)
{
    if (!ctx || !u || !y) return PS_ERR_ARG;
    ps::apply_operator(ctx->E, 1, u, y, nullptr, ctx->E.precision == PS_PREC_MIXED, S(stream));
    PS_CK(cudaGetLastError());
    return PS_OK;
}

int ps_get_diagonal(ps_ctx *ctx, double *d, void *stream)
{
    if (!ctx || !d) return PS_ERR_ARG;
    return ps::diag_saddle(ctx->E, d, S(stream));
}

int ps_ksp_solve(ps_ctx *ctx, const double *b, double *x, const ps_ksp_opts *opts, ps_ksp_result *res, void *stream)
{
    if (!ctx || !b || !x) return PS_ERR_ARG;
    if (opts && opts->method == PS_SOLVE_STRUCTURED) return ps::structured_solve(ctx->E, b, x, opts, res, S(stream));
    return ps::minres_solve(ctx->E, b, x, opts, res, S(stream));
}

int ps_sqrtm_apply(ps_ctx *ctx, const double *z, double *w, const ps_sqrt_opts *opts, ps_sqrt_result *res, void *stream)
{
    if (!ctx || !z || !w) return PS_ERR_ARG;
    return ps::slip_noise(ctx->E, z, w, opts, res, S(stream));
}

int ps_step(ps_ctx *ctx, const ps_step_inputs *in, ps_step_result *res, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    return ps::step_all(ctx->E, in, res, S(stream));
}

int ps_step_outputs(ps_ctx *ctx, double *up, double *udiff, double *sb, double *fext, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    Engine &E = ctx->E;
    cudaStream_t st = S(stream);
    if (up) PS_CK(cudaMemcpyAsync(up, E.d_up, sizeof(double) * E.nvel, cudaMemcpyDefault, st));
    if (udiff) PS_CK(cudaMemcpyAsync(udiff, E.d_ud, sizeof(double) * E.nvel, cudaMemcpyDefault, st));
    if (sb) PS_CK(cudaMemcpyAsync(sb, E.d_sb, sizeof(double) * E.nvel, cudaMemcpyDefault, st));
    if (fext) PS_CK(cudaMemcpyAsync(fext, E.d_fext, sizeof(double) * E.nvel, cudaMemcpyDefault, st));
    if (ps::is_host_ptr(up) || ps::is_host_ptr(udiff) || ps::is_host_ptr(sb) || ps::is_host_ptr(fext))
        PS_CK(cudaStreamSynchronize(st));
    return PS_OK;
}

int ps_time_kernel(ps_ctx *ctx, int32_t which, int32_t reps, const double *u, double *ms, void *stream)
{
    if (!ctx || !u || !ms || which < 0 || which > 3) return PS_ERR_ARG;
    return ps::time_pairs(ctx->E, which, reps, u, ms, S(stream));
}

uint64_t ps_kernel_launches(void) { return (uint64_t)ps_launch_count; }


int ps_autotune(ps_ctx *ctx, int32_t reps, int32_t *best_cols, double *ms, void *stream)
{
    if (!ctx) return PS_ERR_ARG;
    ps::Engine &E = ctx->E;
    const int cand[4] = {128, 256, 512, 1024};
    double t[4] = {0, 0, 0, 0};
    double *u = nullptr;
    PS_CK(cudaMalloc(&u, sizeof(double) * std::max<long>(E.ntop, 1)));
    PS_CK(cudaMemset(u, 0, sizeof(double) * std::max<long>(E.ntop, 1)));
    int best = ps::g_aa_chunk_cols, rc = PS_OK;
    double tbest = 1e300;
    for (int k = 0; k < 4 && rc == PS_OK; k++) {
        if ((rc = ps::set_aa_chunking(E, cand[k]))) break;
        rc = ps::time_pairs(E, 3, reps > 0 ? reps : 5, u, &t[k], S(stream));   // apply incl. combine
        if (rc == PS_OK && t[k] < tbest) { tbest = t[k]; best = cand[k]; }
    }
    cudaFree(u);
    if (rc) return rc;
    ps::g_aa_chunk_cols = best;
    if ((rc = ps::set_aa_chunking(E, best))) return rc;
    if (best_cols) *best_cols = best;
    if (ms) for (int k = 0; k < 4; k++) ms[k] = t[k];
    return PS_OK;
}

int ps_fma_peak(int32_t fp64, double *tflops, void *stream)
{
    if (!tflops) return PS_ERR_ARG;
    return ps::fma_peak(fp64, tflops, S(stream));
}

int ps_rsqrt_check(const double *a, int64_t n, uint64_t *max_ulp, void *stream)
{
    if ((!a && n > 0) || n < 0 || !max_ulp) return PS_ERR_ARG;
    unsigned long long m = 0;
    int rc = ps::rsqrt_check(a, (long)n, &m, S(stream));
    *max_ulp = (uint64_t)m;
    return rc;
}

}  // extern "C"
