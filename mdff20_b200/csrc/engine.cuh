// mdffgpu engine: device state of one system and the launchers of its kernels.
#pragma once

#include <functional>
#include <vector>

#include "common.cuh"

namespace mdffgpu {

// ---------------------------------------------------------------- per type-pair data
// n-m LJ constants of init_nmlj (src/nmlj.c:198-236) and the BHMFT(D) table
// (src/bhmftd.c:99-110), for the ordered pair (ti, tj).
struct PairSR {
    double sigsq, epsqp, fc, ptwo, qtwo, uc, plj, qlj;
    double A, B, C, D, BD;
    int ip, iq;   // ptwo/qtwo as integers when integral (fast power path), else -1
};
// Tang-Toennies damping of the charge->dipole field for the ordered pair (ita, jta)
// (src/ewald.c:505-516): D1 from pol_damp_*[ita][ita][jta], D2 from [jta][ita][jta].
struct PairDamp {
    int ldamp, k1, k2, pad;
    double b1, c1, b2, c2;
};

// one k-space row segment: up to KSEG consecutive nz values at fixed (nx, ny)
constexpr int KSEG = 16;
constexpr int RHO_MIN_BLOCKS = 4;   // resident k_rho blocks per SM (caps registers at 128)
constexpr int RHOR_K = 32;          // k per k_rho_reduce block
struct KSeg {
    int nx, ny, z0, cnt;
    int koff, pad0, pad1, pad2;
};
// one k-space row: all nz of a fixed (nx, ny)
struct KRow {
    int nx, ny, z0, cnt;
    int koff, pad0, pad1, pad2;
};

// scalar slots (device array `scal`) written by the reduction kernels
enum Slot : int {
    S_LJ_U = 0, S_LJ_TAU = 1,      // 6 entries xx xy xz yy yz zz
    S_BH_U = 7, S_BH_TAU = 8,
    S_DIR_U = 14, S_DIR_TAU = 15,
    S_REC_U = 21, S_REC_TAU = 22,
    S_Q2 = 28, S_MU2 = 29,         // adjacent: written together
    S_KIN = 30,
    S_UPOL = 31, S_RMSD2 = 32,     // adjacent
    S_RZ = 33, S_RR = 34,          // adjacent
    S_PAP = 35, S_RZOLD = 36,
    S_DISP1 = 37, S_DISP2 = 38,
    NSLOT = 40
};

// values the host reads back in one copy after a step
struct DevScalars {
    double u_lj, pvir_lj, tau_lj[9];
    double u_bh, pvir_bh, tau_bh[9];
    double u_coul, pvir_coul, tau_coul[9];
    double u_pol, e_kin, e_nvt, scf_rmsd;
    double xi[16], vxi[16];
    double nhc_s;
    int scf_iter, nbuilds, rebuild, status;
};

// the stopping test of a recorded CG loop, evaluated by the last block of k_cg_step (or by
// k_cg_test before the first iteration): mode 1, the induced-dipole test
// rmsd = sqrt(r.r / npol) > tol (the reference's residual measure, src/pim.c:431-449);
// mode 2, the adjoint test r.r > rtol2 r0.r0; mode 0, none (host-driven loops).  Sets the
// while node's condition; the iteration limit or a non-finite residual raise status bits.
struct CgTest {
    cudaGraphConditionalHandle h;
    int mode;
    DevScalars *out;       // mode 1: iteration count and rmsd
    int npol;
    double tol;
    double *rr0, *itc;     // mode 2: the initial r.r and the iteration count (fit slots)
    double rtol2;
    int maxit;
    unsigned *status;
    unsigned *guard;       // iterations counted by k_cg_dir, which ends the loop past maxit
                           // whatever k_cg_step did (a backstop of the while node)
};

struct Engine;

// zero-initialised device allocation; MDFFGPU_ERR_NOMEM on failure.  The zeroing runs on
// the legacy stream, which the engine's non-blocking stream does not wait for, so it is
// completed here before the buffer is handed out.
template <typename T>
inline T *dalloc(size_t count) {
    T *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)&p, sizeof(T) * count);
    if (e != cudaSuccess) throw Error(MDFFGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    e = cudaMemset(p, 0, sizeof(T) * count);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) throw Error(MDFFGPU_ERR_CUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
    return p;
}

// ---------------------------------------------------------------- launchers
// lists.cu
void launch_kardir(Engine &e, const double4 *r, double4 *s);
// sets e.d_rebuild on the device (and, given a handle, the condition of a recorded IF node)
void launch_check_list(Engine &e, const cudaGraphConditionalHandle *h = nullptr);
void launch_build_lists(Engine &e, bool force); // gated by d_rebuild unless force
// pair.cu
void launch_sr(Engine &e, bool lj);            // adds forces into e.d_f, partials into slots
// real-space multipole sum on e.d_s (fractional positions); q, mu per ion.  forces:
// per-ion force into out_f plus energy/virial partials (slots S_DIR_*); ef: field into
// out_ef; efg: EFG into out_efg (efg_q adds the charge part, src/ewald.c:724-729).
void launch_dir(Engine &e, const double *q, const double3 *mu, double alpha, bool lq, bool ld, bool damp,
                bool forces, bool ef, bool efg, bool efg_q, double3 *out_ef, double *out_efg, double3 *out_f);
// per list entry (F1/d^3, 3 F2/d^5) for the current positions, then the dipole-only
// field from them (the induced-dipole iterations of one force evaluation)
void launch_dir_prep(Engine &e, double alpha);
void launch_dir_field_cached(Engine &e, const double3 *mu, double3 *out_ef);
// kspace.cu
// CG product formed where T p is formed (mixed-precision k-space combine, polarisable
// ions): ap = invpol p - T p, block partials of p.ap into slot S_PAP of part, reduced
// into scal by the kernel's last block
struct CgAp {
    const double *invpol = nullptr;
    const double3 *p = nullptr;
    double3 *ap = nullptr;            // null: not formed
    double *part = nullptr;
    int stride = 0;
    double *scal = nullptr;
    unsigned *ticket = nullptr;
};
struct RecOut {
    double3 *ef = nullptr;            // self2*mu + ef_dir + E_rec
    const double3 *ef_dir = nullptr;
    double self2 = 0.0;
    const double *self_q = nullptr;   // charges and dipoles of the self terms
    const double3 *self_mu = nullptr;
    double3 *f = nullptr;             // f + f_dir*coul + F_rec*coul
    const double3 *f_dir = nullptr;
    double coul = 1.0;
    double *efg = nullptr;            // self + efg_dir + EFG_rec (upper triangle)
    const double *efg_dir = nullptr;
    double2 *rho_raw = nullptr;       // receives rho(k) of (q, mu) when set
    const double2 *rho_acc = nullptr; // rho(k) of (q, mu) given: the rho pass is skipped
    bool energy = true;               // false: skip the energy/virial reduction (field-only passes)
    const int *idx = nullptr;         // mixed precision: only these ions (q, mu zero elsewhere;
    int cnt = -1;                     // outputs written at these ions only), cnt of them
    const int *out_idx = nullptr;     // mixed precision: outputs at these ions only (the rho
    int out_cnt = -1;                 // pass still sums over idx / all ions), out_cnt of them
    CgAp cg;                          // mixed precision, field only: the CG product at the output ions
};
void launch_rec(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const RecOut &o);
// fit.cu: the status bits of a force-matching evaluation as an Error (none: returns)
void fit_status(unsigned status);
constexpr int FIT_NRES = 1 + MDFFGPU_FIT_NPARAM + 1;   // loss, gradient, status bits per evaluation
// integrate.cu
struct AspcCoef {
    int ne;          // values of the history used (order + 1)
    double c[6];     // their coefficients, newest first
};
AspcCoef aspc_coef(int e, bool poly);
// k_scale_kin: v *= nhc_s (scale), the kinetic sum into scal[S_KIN], then (energy) e_kin
// and e_nvt
struct ScaleKinArgs {
    int n, scale, energy, nn;
    double L, temp;
    const DevScalars *out_s;
    const double *mass, *nhc;
    double3 *v;
    double *part, *scal;
    int stride;
    unsigned *ticket;
    DevScalars *out;
};
void launch_reduce_slots(Engine &e, int first_slot, int nslots, int nparts);
// true once the FP32 pair/k-space kernels exist in this build
inline bool mixed_available() { return true; }
// real32.cu: mixed-precision real space.  launch_pair_prep32 once per force evaluation
// (in-cutoff list and dipole-field records); launch_dir32 as launch_dir (charges from
// the fractional coordinates' w; a field-only pass may take an ion subset idx[cnt],
// written there only); launch_pol_field32: T mu at the polarisable ions from the
// dipole-field records (zero at the others)
void launch_pair_prep32(Engine &e);
void launch_dir32(Engine &e, const double *q, const double3 *mu, double alpha, bool lq, bool ld, bool damp,
                  bool forces, bool ef, double3 *out_ef, double3 *out_f, const int *idx = nullptr, int cnt = 0);
void launch_pol_field32(Engine &e, const double3 *p, double3 *out_ef);
// kspace32.cu: per force evaluation, the phase tables of the current positions
void launch_coords32(Engine &e);
// kspace32.cu: FP32 phase tables and k-space passes (idx: optional ion subset of cnt ions)
void setup_kspace32(Engine &e, const std::vector<KRow> &rows);
void launch_phase32(Engine &e);
void launch_rho32(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt);
void launch_combine32(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx,
                      int cnt, int slices, bool wf);
// kspace_ion_tc.cu: the ion pass on the tensor cores (false: not applicable, nothing
// launched); launch_ion_tc_table writes its per-ion operand of the current positions
bool launch_ion_tc(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx,
                   int cnt);
void launch_ion_tc_table(Engine &e);
void setup_ion_tc(Engine &e);
// kspace_tc.cu: the same rho chunk partials from tcgen05 TF32 MMAs (false: not applicable,
// nothing launched); launch_rho_tc_tables lays out its per-stage inputs of the current
// positions (after the phase table)
bool launch_rho_tc(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt,
                   int z_off, int *chunks_used);
void launch_rho_tc_tables(Engine &e);
void setup_rho_tc(Engine &e, int lz);
void launch_ion32(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx, int cnt);

// ---------------------------------------------------------------- engine state
struct Engine {
    mdffgpu_params p;
    int n = 0, nt = 0, device = 0;
    int precision = MDFFGPU_FP64;
    int pim_solver = MDFFGPU_PIM_REFERENCE;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    std::string last_error;

    // units (src/constants.c:8-18, reduced units :38-45)
    double boltz_unit, time_unit, press_unit, coul_unit;
    Cell cell;
    // derived md parameters (check_md, src/md.c:120-141)
    double dt, temp, tauT, timesca;
    int lqch = 0, ldip = 0, lpol = 0, ldmp = 0, lpim = 0, npol = 0;
    int lpolar[NT] = {0};
    double srcutsq = 0, lrcutsq = 0;
    double utail = 0, ptail = 0;

    // ---- host copies of per-ion constants
    std::vector<int> h_typ;
    std::vector<double> h_q;
    double *d_soa = nullptr;     // per-component state arrays of host transfers, 9 doubles per ion
    // ---- device per-ion arrays
    double4 *d_r = nullptr;      // Cartesian x y z, w = charge
    double4 *d_s = nullptr;      // fractional (kardir) x y z, w = charge
    double3 *d_v = nullptr, *d_f = nullptr, *d_f2 = nullptr;
    double *d_mass = nullptr, *d_invmass = nullptr, *d_q = nullptr;
    int *d_typ = nullptr;
    double3 *d_mu_static = nullptr, *d_mu_ind = nullptr, *d_mu_tot = nullptr;
    double *d_pol = nullptr, *d_invpol = nullptr;  // [n][9], zero for non-polarisable
    int *d_polar = nullptr;
    double3 *d_ef_stat = nullptr, *d_ef_ind = nullptr, *d_ef = nullptr;
    double3 *d_cg_r = nullptr, *d_cg_p = nullptr, *d_cg_ap = nullptr, *d_mu_save = nullptr;
    double3 *d_rs = nullptr;     // leap-frog r(t-dt)
    double *d_hist = nullptr;    // ASPC history [n][6][3]
    double *d_efg = nullptr;     // [n][9]
    double3 *d_tmp3 = nullptr;   // scratch field / force
    double *d_qzero = nullptr;
    double3 *d_muzero = nullptr;
    // pair tables
    PairSR *d_pair = nullptr;
    std::vector<PairSR> h_pair;      // host copies (parameter updates of the force-matching fit)
    std::vector<PairDamp> h_damp;
    PairDamp *d_damp = nullptr;

    // ---- neighbour lists (full lists, row-major [n][cap])
    int cap_nb = 0, cap_co = 0;
    int *d_nb = nullptr, *d_nbn = nullptr, *d_co = nullptr, *d_con = nullptr;
    double2 *d_coef = nullptr;   // [n][cap_co] cached dipole-field pair factors
    bool use32 = false;          // mixed precision: FP32 Ewald kernels
    // parts of the mixed path (all on by default; MDFFGPU_MIXED_PARTS=real|rec keeps
    // only that part in FP32, MDFFGPU_PIM_SUBSET=0 runs the CG field over all ions)
    bool real32 = true, rec32 = true, subset32 = true;
    // mixed-precision real space (real32.cu), sized like the Coulomb list
    int *d_nl32 = nullptr, *d_nln32 = nullptr;   // in-cutoff neighbours [n][cap32]
    int *d_pl32 = nullptr, *d_pln32 = nullptr;   // polarisable neighbours of polarisable ions
    float4 *d_pu32 = nullptr;                    // their dipole-field records (u, c1)
    float4 *d_qm32 = nullptr;                    // per-ion dipole (FP32), w = type
    int cap32 = 0;
    bool coef_ready = false;     // d_coef matches the current positions
    double4 *d_svl = nullptr;    // fractional positions at the last build
    int nc[3] = {1, 1, 1}, ncell = 1, cell_cap = 4096;
    int *d_cell_of = nullptr, *d_cell_cnt = nullptr, *d_cell_start = nullptr, *d_cell_cur = nullptr,
        *d_cell_ions = nullptr;
    int *d_rebuild = nullptr;    // 1 when the lists must be rebuilt this step
    bool list_ready = false;

    // ---- k space
    int nk = 0, nseg = 0, nrow = 0, kmax[3] = {0, 0, 0};
    double *d_Ak = nullptr, *d_kcoe = nullptr;
    double3 *d_kvec = nullptr;
    KSeg *d_seg = nullptr;
    KRow *d_row = nullptr;
    std::vector<int> h_tile_row;   // first row of each ion-pass tile (+ end)
    std::vector<int> h_tile_k;     // first k of each tile (+ end)
    int *d_tile_row = nullptr, *d_tile_k = nullptr;
    int ntile = 0, tile_kmax = 0;
    double2 *d_rho_part = nullptr, *d_rho = nullptr;   // partial per ion chunk, total (Ak-scaled)
    double2 *d_rho_acc = nullptr, *d_rho_it = nullptr; // rho(k) of (q, mu) along the fused CG; of its p
    // mixed precision k space (kspace32.cu)
    KSeg *d_seg32 = nullptr;                            // rho segments: (row, block of |nz|), both signs
    int nseg32 = 0, tab_w = 0;
    float2 *d_tab32 = nullptr;                          // phase table rows [n][tab_w]
    int rho32_chunks = 0, rho32_chunks_max = 0;         // chunks of the rho pass; room for the most
    int ion_tc_slices_set = 0;                          // tensor-core ion pass slices (0: cost model)
    int rho_chunks_used = 0;                            // chunk partials the last rho pass wrote
    // rho pass on the tensor cores (kspace_tc.cu): per-stage E operand tiles and E0 | E1
    // rows of the current positions, the chunk count (0: two CTAs per SM)
    bool rho_tc = true;
    float4 *d_rho_btab = nullptr, *d_rho_etab = nullptr;
    int rho_tc_lz = 0, rho_tc_chunks_set = 0;
    // ion pass on the tensor cores (kspace_ion_tc.cu): positions in the order polarisable
    // ions first, the per-ion operand tiles of the current positions, per-pass weights
    bool ion_tc = true;
    int *d_ion_order = nullptr;
    float4 *d_ion_atab = nullptr, *d_ion_wtab = nullptr;
    // CG initial guess: polynomial extrapolation through the last extrapolate_order + 1
    // converged dipoles (false: the reference's ASPC coefficients)
    bool cg_poly = true;
    float4 *d_qm_tc = nullptr;                          // per position of the order: (q, 2 pi B mu)
    float2 *d_rho_part32 = nullptr;                     // [rho32_chunks][nk]
    int ion32_slices = 0, nsm = 148;                    // most ion-pass slices; SMs
    double *d_ion_part32 = nullptr;                     // [slices][n][6]
    int *d_pidx = nullptr;                              // polarisable ions, ascending
    bool rho_acc_ready = false;                         // d_rho_acc holds rho(k) of (q, mu_tot)
    double *d_ion_part = nullptr;                       // ion-pass partial sums [ntile][n][12]
    int rho_chunks = 0, rho_chunk = 0;

    // ---- reductions
    double *d_part = nullptr;    // [NSLOT][part_stride]
    int part_stride = 0;
    double *d_scal = nullptr;    // [NSLOT]
    DevScalars *d_out = nullptr; // composed results
    DevScalars *h_out = nullptr; // pinned mirror
    unsigned *d_status = nullptr;
    unsigned *d_ticket = nullptr;   // block-arrival counters of kernels that finish their own reductions
    double *d_nhc = nullptr;     // xi[16], vxi[16], Q[16]

    // per-kernel timing of one chosen kernel family (CUDA events on `stream`)
    std::string prof_name;
    std::vector<cudaEvent_t> prof_pool;
    std::vector<std::pair<int, int>> prof_pairs;   // indices into prof_pool
    double prof_flops = 0.0;
    int prof_next = 0;
    void prof_begin(const char *name, int *slot);
    void prof_end(const char *name, int slot, double flops);
    void prof_result(double *ms, long long *count, double *flops);

    // pim bookkeeping
    int istep = 0;
    int last_scf_iter = 0;
    double last_rmsd = 0.0;
    int nbuilds = 0;

    // force matching (fit.cu)
    double *d_fpart = nullptr, *d_fscal = nullptr;
    double3 *d_w = nullptr, *d_lam = nullptr, *d_sv = nullptr, *d_fa = nullptr, *d_fb = nullptr, *d_fc = nullptr;
    double *d_qw = nullptr, *d_efg_rec = nullptr;
    double3 *d_muw = nullptr;
    double2 *d_rw = nullptr;
    double3 *d_ft = nullptr;         // target forces
    double *d_theta = nullptr;       // theta on the device (read by the result assembly)
    double *d_fres = nullptr;        // [1 + NPARAM + 1]: the last evaluation's result and status
    int last_adj_iter = 0;
    // one force-matching evaluation recorded as a CUDA graph (fit batches): both CG
    // solves are while nodes, theta is read from a device buffer and the result is
    // assembled on the device, so a replay needs no host round trip
    cudaGraphExec_t fit_exec = nullptr;
    long long fit_graph_gen = -1;

    // one MD step as a CUDA graph (md_steps): the induced-dipole CG loop is a while node
    // whose condition a device kernel sets, so a step needs no host round trip
    bool graph_on = true;
    bool capturing = false;                 // launches are being recorded
    bool pdl = true;                        // launches may carry the programmatic-serialization attribute
    // launch priority (0: the stream's).  The tensor-core k-space passes launch at the
    // device's greatest priority (prio_high) so that, where a side branch runs beside
    // them, the block scheduler places their large-shared-memory CTAs first and the
    // side grid fills what is left; recorded graphs keep it per node.
    int prio = 0, prio_high = 0;
    struct HighPrio {
        Engine &e;
        explicit HighPrio(Engine &x) : e(x) { e.prio = e.prio_high; }
        ~HighPrio() { e.prio = 0; }
    };
    cudaStream_t body_stream = nullptr;     // records the CG loop body
    // Independent parts of a force evaluation run on side streams (in a recorded step:
    // parallel branches of the graph).  on_side(k, f) issues f on side stream k after
    // all that `stream` has issued and after what side k already holds; join_side(k)
    // makes `stream` wait for all of side k.  Forks are joined before the first reader
    // of what they write, inside the same evaluation.
    static constexpr int SIDE_SR = 0;       // short-range pair forces (add into d_f)
    static constexpr int SIDE_PREP = 1;     // FP32 in-cutoff lists and dipole-field records, then the
                                            // real-space part of the solve's first field pass (d_tmp3)
    static constexpr int SIDE_DIR = 2;      // real-space Ewald forces (d_tmp3, S_DIR_U slots)
    // the real-space field of a field pass (d_tmp3) beside its k-space passes: SIDE_BODY
    // while a loop body is recorded (a stream that joined one capture cannot join the
    // body's, which is recorded inside it), SIDE_FIELD otherwise
    static constexpr int SIDE_BODY = 3;
    static constexpr int SIDE_FIELD = 4;
    static constexpr int NSIDE = 5;
    cudaStream_t side[NSIDE] = {};
    cudaEvent_t ev_fork[NSIDE] = {}, ev_join[NSIDE] = {};
    bool side_open[NSIDE] = {};
    bool side_on = true;                    // MDFFGPU_SIDE_STREAMS=0: everything on `stream`
    bool prep_issued = false;               // this evaluation's FP32 lists are issued (SIDE_PREP)
    template <class F>
    void on_side(int k, F &&f) {
        if (!side_on) {
            f();
            return;
        }
        MDFF_CK(cudaEventRecord(ev_fork[k], stream));
        MDFF_CK(cudaStreamWaitEvent(side[k], ev_fork[k], 0));
        cudaStream_t main = stream;
        stream = side[k];
        try {
            f();
        } catch (...) {
            stream = main;
            if (cudaEventRecord(ev_join[k], side[k]) == cudaSuccess) cudaStreamWaitEvent(stream, ev_join[k], 0);
            throw;
        }
        stream = main;
        MDFF_CK(cudaEventRecord(ev_join[k], side[k]));
        side_open[k] = true;
    }
    void join_side(int k) {
        if (!side_open[k]) return;
        side_open[k] = false;
        MDFF_CK(cudaStreamWaitEvent(stream, ev_join[k], 0));
    }
    // after a recording that failed part way: its forks belong to the abandoned capture
    void forget_sides() {
        for (bool &o : side_open) o = false;
        prep_issued = false;
    }
    cudaGraphExec_t step_exec = nullptr;
    long long gen = 0, graph_gen = -1;      // gen: bumped when buffers or modes change
    long long graph_outer = 0, graph_body = 0, body_count = 0;   // kernels per replay / per CG iteration
    long long graph_if = 0, if_count = 0;   // kernels of the list rebuild (an IF node) per rebuild

    explicit Engine(const mdffgpu_params &prm, int dev);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    // set-up pieces
    void setup_units_and_cell();
    void setup_types();
    void setup_kspace();
    void alloc_lists(int cap_nb_, int cap_co_);
    void setup_cells();

    // operations (engine.cu)
    void set_positions(const double *rx, const double *ry, const double *rz);
    void set_velocities(const double *vx, const double *vy, const double *vz);
    void get_state(double *rx, double *ry, double *rz, double *vx, double *vy, double *vz, double *fx,
                   double *fy, double *fz);
    void gen_verletlist();
    int check_verletlist(bool reset_status = true);
    void ensure_lists();
    void engforce(bool check_finite = true);   // check_finite: ST_NONFINITE from r and f
    void sr_forces(bool lj, double *u, double *pvir, double *tau);
    void sr_finish(bool lj);   // reduce the short-range slot, u / virial / stress into d_out
    void multipole_es_dev(const double *d_qv, const double3 *d_muv, double alpha, int flags, double3 *d_ef_out,
                          double *d_efg_out, double3 *d_f_out);
    void field_of(const double *d_qv, const double3 *d_muv, bool lq, bool ld, bool damp, double3 *d_ef_out,
                  double2 *rho_raw = nullptr);
    void field_pol(const double3 *d_p, double3 *d_out, double2 *rho_raw, bool cg_ap = false);
    void ensure_real32();
    void dfree32();
    void get_dipoles();
    void pim_reference();
    void pim_cg(bool fused);
    void pim_ko();
    void ko_inner(double3 *d_dmu, const double3 *d_find);
    double rmsd_of(const double3 *d_mu, const double3 *d_ef, double *upol_sum);
    void prop_agate(int step);
    // in: 6 host arrays (rx..vz) copied in first, out: 9 host arrays (rx..fz) filled after
    // the last step; both optional, entries may be null (mdffgpu_md_steps_host)
    void md_steps(int first, int nsteps, double *thermo, const double *const *in = nullptr,
                  double *const *out = nullptr);
    // force matching: theta = (A, B, C of Si-O, A, B, C of O-O, q_Si, alpha_O, b, c);
    // force_match: res[0] = sum |F - F_t|^2, res[1..10] = dL/dtheta for
    // L = scale/2 sum |F - F_t|^2 (w = scale (F - F_t))
    void set_fit_params(int tSi, int tO, const double *theta);
    void fit_host_params(int tSi, int tO, const double *theta);
    void force_match(const double3 *d_ft, double scale, double *res, int tSi, int tO);
    // the pieces of force_match: buffers, the device-side parameter update from a device
    // theta (recorded evaluations), the evaluation itself into d_res[0..NPARAM] (+ status)
    void fit_alloc();
    void fit_apply_theta(const double *d_th, int tSi, int tO);
    void fit_issue(const double3 *d_ft, double scale, int tSi, int tO, const double *d_th, double *d_res);
    void capture_fit(const double *d_th, int tSi, int tO, double scale, double *d_res);
    void solve_pim(const double3 *d_b, double3 *d_x, double rtol, int maxit);
    void fit_reduce(int first, int cnt, int nparts);
    void coul_forces(const double *d_qv, const double3 *d_muv, bool lq, bool ld, double3 *out);
    // exact restart (state.cu): the complete MD state as one byte block
    size_t state_bytes() const;
    void save_state(unsigned char *buf);
    int load_state(const unsigned char *buf, size_t bytes);
    bool graph_ok(int step) const;
    void capture_step(int step);
    // launch shapes of the mixed k space timed on this system (the field pass of the CG):
    // choice = {tensor-core ion pass, rho chunks, ion-pass slices}, ms = its time
    void tune_launch(int reps, int *choice, double *ms);
    void record_if(const std::function<void(cudaGraphConditionalHandle)> &test, const std::function<void()> &body);
    void record_while(const std::function<void(cudaGraphConditionalHandle)> &first,
                      const std::function<void(cudaGraphConditionalHandle)> &body);
    void drop_graph();
    void sync_scalars();
    void check_status();
    void finalize_coul(bool stress);
    void reduce(int first_slot, int nslots, int nparts) { launch_reduce_slots(*this, first_slot, nslots, nparts); }
};

// Programmatic dependent launch: every kernel of this library opens with grid_dep()
// (wait for the grids it depends on, then release its dependents), so each launch may
// carry the programmatic-serialization attribute -- the grid is launched while the one
// before it in the stream drains (a recorded graph keeps this as a programmatic edge)
// and starts its work once that one has completed with its writes visible.  Engine::pdl
// (MDFFGPU_PDL=0 at creation: off) selects it; the force-matching evaluations launch
// fully serialised (many of them run concurrently, and blocks resident early while they
// wait for their prerequisite take SM slots from the other streams' grids: measured 2%
// fewer configurations per second with it).

// launch bookkeeping: every kernel launch goes through this
#define MDFF_LAUNCH(eng, kernel, grid, block, smem, ...)                               \
    do {                                                                               \
        cudaLaunchAttribute at_[2];                                                    \
        unsigned na_ = 0;                                                              \
        if ((eng).pdl) {                                                               \
            at_[na_].id = cudaLaunchAttributeProgrammaticStreamSerialization;          \
            at_[na_++].val.programmaticStreamSerializationAllowed = 1;                 \
        }                                                                              \
        if ((eng).prio) {                                                              \
            at_[na_].id = cudaLaunchAttributePriority;                                 \
            at_[na_++].val.priority = (eng).prio;                                      \
        }                                                                              \
        cudaLaunchConfig_t cfg_ = {};                                                  \
        cfg_.gridDim = dim3(grid);                                                     \
        cfg_.blockDim = dim3(block);                                                   \
        cfg_.dynamicSmemBytes = (smem);                                                \
        cfg_.stream = (eng).stream;                                                    \
        cfg_.attrs = at_;                                                              \
        cfg_.numAttrs = na_;                                                           \
        MDFF_CK(cudaLaunchKernelEx(&cfg_, kernel, __VA_ARGS__));                       \
        (eng).launches++;                                                              \
    } while (0)

}  // namespace mdffgpu
