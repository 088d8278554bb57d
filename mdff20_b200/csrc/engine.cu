// Engine set-up and orchestration: the reference's engforce / get_dipoles /
// prop_agate / check_verletlist sequences (src/field.c:352-407, src/coulombic.c:67-130,
// src/integration.c:22-333, src/verlet.c:124-170) as launches on one CUDA stream.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <functional>

#include "engine.cuh"

namespace mdffgpu {

// kernels defined in integrate.cu / lists.cu
__global__ void k_reduce_slots(const double *, int, int, int, double *);
__global__ void k_fill3(int n, double3 *a, double3 v);
__global__ void k_copy3(int n, const double3 *a, double3 *b);
__global__ void k_self_sums(int n, const double *q, const double3 *mu, double *part, int stride);
__global__ void k_self_plus_dir(int n, double self2, const double3 *mu, const double3 *efd, double3 *ef);
__global__ void k_axpy3(int n, double a, const double3 *x, double3 *y);
__global__ void k_efg_self_dir(int n, double self2, const double *q, const double *efgd, double *efg);
__global__ void k_finalize_sr(const double *scal, int slot, double inveOmegaPU, double *u, double *pvir,
                              double *tau);
struct CoulFin {
    double alpha, coul, inveOmegaPU, ttpiV;
    int do_dir, do_rec, do_stress;
};
__global__ void k_finalize_coul(const double *scal, CoulFin c, double *u, double *pvir, double *tau);
__global__ void k_induced(int n, const int *polar, const double *pol, const double3 *ef, double3 *mu);
__global__ void k_aspc_predict(int n, AspcCoef cf, int es, double *hist, double3 *mu);
__global__ void k_aspc_correct(int n, double W, const int *polar, const double *pol, const double3 *ef,
                               double3 *mu);
__global__ void k_add3(int n, const double3 *a, const double3 *b, double3 *c);
__global__ void k_pim_sums(int n, const int *polar, const double *pol, const double *invpol, const double3 *mu,
                           const double3 *ef, double *part, int stride);
__global__ void k_hist_store(int n, const double3 *mu, double *hist);
__global__ void k_ko_find(int n, const int *polar, const double *invpol, const double3 *ef, const double3 *mu,
                          double3 *find);
__global__ void k_scale_add3(int n, double a, const double3 *x, double b, double3 *y);
__global__ void k_cg_residual(int n, const int *polar, const double *invpol, const double3 *efs,
                              const double3 *tx, const double3 *x, double3 *r);
__global__ void k_cg_ap(int n, const int *polar, const double *invpol, const double3 *p, const double3 *tp,
                        double3 *ap, double *part, int stride, double *scal, unsigned *ticket);
__global__ void k_cg_rz(int n, const int *polar, const double *pol, const double3 *r, double3 *z, double *part,
                        int stride, double *scal, unsigned *ticket);
__global__ void k_cg_dir(int n, const double *scal, const double3 *z, double3 *p, CgTest t);
__global__ void k_cg_step(int n, int nk, const int *polar, const double *pol, double *scal, const double3 *p,
                          const double3 *ap, double3 *x, double3 *r, double3 *z, const double2 *rho_p, double2 *acc,
                          double *part, int stride, unsigned *ticket, CgTest test);
__global__ void k_cg_test(CgTest t, const double *scal);
__global__ void k_upol_final(const double *scal, double coul, DevScalars *out);
__global__ void k_vv1(int n, double dt, double dtsq2, const double *invm, double4 *r, const double3 *v,
                      const double3 *f, double3 *fs);
__global__ void k_vv2(int n, double dt2, const double *invm, const double *mass, double3 *v, const double3 *f,
                      const double3 *fs, double *part, int stride);
__global__ void k_pv1(int n, double dt, double dt2, const double *invm, double4 *r, double3 *v, const double3 *f);
__global__ void k_pv2(int n, double dt2, const double *invm, const double *mass, double3 *v, const double3 *f,
                      double *part, int stride, double *scal, unsigned *ticket, const double4 *r, unsigned *status);
__global__ void k_scale_kin(ScaleKinArgs a);
__global__ void k_lf(int n, double dtsq, double idt, const double *invm, const double *mass, double4 *r,
                     double3 *rs, double3 *v, const double3 *f, double *part, int stride);
struct NhcArgs {
    int nn, yo, mults;
    double dt, temp, L, w[7];
};
void launch_nhc_chain(Engine &e, const NhcArgs &a, double *nhc, const double *scal, DevScalars *out);
__global__ void k_set_ekin(const double *scal, DevScalars *out);
__global__ void k_check_finite(int n, const double4 *r, const double3 *f, unsigned *status);
__global__ void k_sort_cells(int ncell, int cell_cap, const int *start, const int *cnt, int *ions,
                             const int *rebuild);

template <typename T>
static void dfree(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// 3x3 inverse by Gauss-Jordan with partial pivoting (1/a_ii for a diagonal input),
// standing in for invertmatrix3x3 (src/inverse_matrix.c:5-20, src/config.c:171)
static void invert3(const double in[3][3], double out[3][3]) {
    double m[3][6];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            m[i][j] = in[i][j];
            m[i][j + 3] = (i == j);
        }
    for (int c = 0; c < 3; c++) {
        int p = c;
        for (int r = c + 1; r < 3; r++)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (m[p][c] == 0.0) continue;
        if (p != c)
            for (int j = 0; j < 6; j++) std::swap(m[c][j], m[p][j]);
        double inv = 1.0 / m[c][c];
        for (int j = 0; j < 6; j++) m[c][j] = (j == c) ? 1.0 : m[c][j] * inv;
        for (int r = 0; r < 3; r++) {
            if (r == c || m[r][c] == 0.0) continue;
            double f = m[r][c];
            for (int j = 0; j < 6; j++) m[r][j] -= f * m[c][j];
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) out[i][j] = m[i][j + 3];
}

// ---------------------------------------------------------------- set-up
Engine::Engine(const mdffgpu_params &prm, int dev) : p(prm) {
    if (p.nion <= 0 || p.ntype <= 0 || p.ntype > NT) throw Error(MDFFGPU_ERR_ARG, "bad nion/ntype");
    int sum = 0;
    for (int t = 0; t < p.ntype; t++) sum += p.nionit[t];
    if (sum != p.nion) throw Error(MDFFGPU_ERR_ARG, "nionit does not sum to nion");  // src/config.c:112-121
    n = p.nion;
    nt = p.ntype;
    if (dev >= 0) MDFF_CK(cudaSetDevice(dev));
    MDFF_CK(cudaGetDevice(&device));
    MDFF_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    MDFF_CK(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
    for (int k = 0; k < NSIDE; k++) {
        MDFF_CK(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
        MDFF_CK(cudaEventCreateWithFlags(&ev_fork[k], cudaEventDisableTiming));
        MDFF_CK(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
    }
    if (const char *v = getenv("MDFFGPU_SIDE_STREAMS")) side_on = atoi(v) != 0;
    if (const char *v = getenv("MDFFGPU_PDL")) pdl = atoi(v) != 0;
    {
        int least = 0, greatest = 0;
        MDFF_CK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        prio_high = greatest;
        if (const char *v = getenv("MDFFGPU_TC_PRIORITY")) prio_high = atoi(v) ? greatest : 0;
    }
    setup_units_and_cell();
    setup_types();
    // device buffers
    d_r = dalloc<double4>(n);
    d_s = dalloc<double4>(n);
    d_v = dalloc<double3>(n);
    d_f = dalloc<double3>(n);
    d_f2 = dalloc<double3>(n);
    d_rs = dalloc<double3>(n);
    d_mu_ind = dalloc<double3>(n);
    d_mu_tot = dalloc<double3>(n);
    d_ef_stat = dalloc<double3>(n);
    d_ef_ind = dalloc<double3>(n);
    d_ef = dalloc<double3>(n);
    d_cg_r = dalloc<double3>(n);
    d_cg_p = dalloc<double3>(n);
    d_cg_ap = dalloc<double3>(n);
    d_mu_save = dalloc<double3>(n);
    d_tmp3 = dalloc<double3>(n);
    d_hist = dalloc<double>((size_t)n * ASPC_DEPTH * 3);
    d_efg = dalloc<double>((size_t)n * 9);
    d_qzero = dalloc<double>(n);
    d_muzero = dalloc<double3>(n);
    d_svl = dalloc<double4>(n);
    d_rebuild = dalloc<int>(1);
    d_status = dalloc<unsigned>(1);
    d_ticket = dalloc<unsigned>(8);
    d_scal = dalloc<double>(NSLOT);
    d_out = dalloc<DevScalars>(1);
    d_nhc = dalloc<double>(48);
    MDFF_CK(cudaMallocHost((void **)&h_out, sizeof(DevScalars)));
    d_soa = dalloc<double>(9 * (size_t)n);
    memset(h_out, 0, sizeof(DevScalars));
    if (p.lcoulombic) setup_kspace();
    int nkb = nk > 0 ? ceil_div(nk, RHOR_K) : 1;
    part_stride = std::max(ceil_div(n, 8), nkb) + 8;
    d_part = dalloc<double>((size_t)NSLOT * part_stride);
    // neighbour lists: initial capacities from the number density
    double rho = n * cell.inveOmega;
    double cnb = p.cutshortrange + (p.lverletL ? p.skindiff : 0.0);
    double cco = p.cutlongrange + (p.lverletL ? p.skindiff : 0.0);
    auto cap_for = [&](double cut) {
        double e = rho * 4.0 / 3.0 * PI_D * cut * cut * cut;
        int c = (int)(1.4 * e) + 64;
        c = (c + 31) / 32 * 32;
        return std::max(32, std::min(c, ((n + 31) / 32) * 32));
    };
    setup_cells();
    alloc_lists(cap_for(cnb), cap_for(cco));
    // NHC masses Q (src/integration.c:146-150)
    double L = 3.0 * (double)n;
    std::vector<double> nhc(48, 0.0);
    for (int i = 0; i < p.nhc_n && i < 16; i++) nhc[32 + i] = timesca * timesca * temp;
    nhc[32] *= L;
    MDFF_CK(cudaMemcpy(d_nhc, nhc.data(), sizeof(double) * 48, cudaMemcpyHostToDevice));
    MDFF_CK(cudaDeviceSynchronize());
}

Engine::~Engine() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto ev : prof_pool) cudaEventDestroy(ev);
    double4 *d4[] = {d_r, d_s, d_svl};
    for (auto &x : d4) cudaFree(x);
    double3 *d3[] = {d_v, d_f, d_f2, d_rs, d_mu_static, d_mu_ind, d_mu_tot, d_ef_stat, d_ef_ind, d_ef, d_cg_r,
                     d_cg_p, d_cg_ap, d_mu_save, d_tmp3, d_muzero, d_kvec};
    for (auto &x : d3) cudaFree(x);
    double *dd[] = {d_mass, d_invmass, d_q, d_pol, d_invpol, d_hist, d_efg, d_qzero, d_Ak, d_kcoe, d_part, d_scal,
                    d_nhc};
    for (auto &x : dd) cudaFree(x);
    int *di[] = {d_typ, d_polar, d_nb, d_nbn, d_co, d_con, d_cell_of, d_cell_cnt, d_cell_start, d_cell_cur,
                 d_cell_ions, d_rebuild, d_tile_row, d_tile_k};
    for (auto &x : di) cudaFree(x);
    cudaFree(d_pair);
    cudaFree(d_damp);
    cudaFree(d_seg);
    cudaFree(d_row);
    cudaFree(d_rho_part);
    cudaFree(d_rho);
    cudaFree(d_rho_acc);
    cudaFree(d_rho_it);
    cudaFree(d_seg32);
    cudaFree(d_tab32);
    cudaFree(d_rho_part32);
    cudaFree(d_ion_part32);
    cudaFree(d_pidx);
    cudaFree(d_qm_tc);
    cudaFree(d_rho_btab);
    cudaFree(d_rho_etab);
    cudaFree(d_ion_order);
    cudaFree(d_ion_atab);
    cudaFree(d_ion_wtab);
    cudaFree(d_ion_part);
    cudaFree(d_coef);
    dfree32();
    for (void *x : {(void *)d_fpart, (void *)d_fscal, (void *)d_w, (void *)d_lam, (void *)d_sv, (void *)d_fa,
                    (void *)d_fb, (void *)d_fc, (void *)d_qw, (void *)d_efg_rec, (void *)d_muw, (void *)d_rw,
                    (void *)d_ft, (void *)d_theta, (void *)d_fres})
        cudaFree(x);
    cudaFree(d_out);
    cudaFree(d_status);
    cudaFree(d_ticket);
    if (h_out) cudaFreeHost(h_out);
    cudaFree(d_soa);
    if (step_exec) cudaGraphExecDestroy(step_exec);
    if (fit_exec) cudaGraphExecDestroy(fit_exec);
    if (body_stream) cudaStreamDestroy(body_stream);
    for (int k = 0; k < NSIDE; k++) {
        if (ev_fork[k]) cudaEventDestroy(ev_fork[k]);
        if (ev_join[k]) cudaEventDestroy(ev_join[k]);
        if (side[k]) cudaStreamDestroy(side[k]);
    }
    if (stream) cudaStreamDestroy(stream);
}

void Engine::setup_units_and_cell() {
    if (p.lreduced) {
        boltz_unit = time_unit = press_unit = coul_unit = 1.0;
    } else {
        boltz_unit = 8.61734229648141E-05;
        time_unit = 98.2269514139276;
        press_unit = 0.00624150964712042;
        coul_unit = 14.3996441494161;
    }
    // lattice(), src/cell.c:13-91
    Cell &c = cell;
    memcpy(c.A, p.cell, sizeof(c.A));
    auto cross = [](const double *a, const double *b, double *h) {
        h[0] = a[1] * b[2] - a[2] * b[1];
        h[1] = a[2] * b[0] - a[0] * b[2];
        h[2] = a[0] * b[1] - a[1] * b[0];
    };
    cross(c.A[1], c.A[2], c.B[0]);
    cross(c.A[2], c.A[0], c.B[1]);
    cross(c.A[0], c.A[1], c.B[2]);
    double omega = c.B[0][0] * c.A[0][0] + c.B[1][0] * c.A[1][0] + c.B[2][0] * c.A[2][0];
    if (!(omega > 0.0)) throw Error(MDFFGPU_ERR_ARG, "cell volume must be positive");
    c.omega = omega;
    c.inveOmega = 1.0 / omega;
    c.inveOmegaPU = 1.0 / (omega * press_unit);
    for (int i = 0; i < 3; i++)
        c.w[i] = omega / std::sqrt(c.B[0][i] * c.B[0][i] + c.B[1][i] * c.B[1][i] + c.B[2][i] * c.B[2][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.B[i][j] = c.B[i][j] * c.inveOmega;
    c.ortho = 1;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (i != j && (c.A[i][j] != 0.0)) c.ortho = 0;
    // check_md, src/md.c:120-127
    tauT = p.tauTberendsen;
    if (p.nequil > 0 && tauT == 0.0) tauT = p.dt;
    if (p.egrator == 0 && p.nequil > 0) p.egrator = 1;   // equilibration runs velocity Verlet
    temp = p.temp * boltz_unit;
    dt = p.dt * time_unit;
    tauT *= time_unit;
    timesca = p.timesca_thermo * time_unit;
    srcutsq = p.cutshortrange * p.cutshortrange;
    lrcutsq = p.cutlongrange * p.cutlongrange;
}

void Engine::setup_types() {
    // flags of read_field / info_field (src/field.c:97-108, 195-221)
    for (int t = 0; t < nt; t++) {
        lpolar[t] = 0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (p.polit[t][i][j] != 0.0) lpolar[t] = 1, lpol = 1;
        if (p.qit[t] != 0.0) lqch = 1;
        for (int j = 0; j < 3; j++)
            if (p.dipit[t][j] != 0.0) ldip = 1;
    }
    // the damping tables' in-place symmetrisation loop, src/field.c:209-219
    for (int it = 0; it < nt; it++)
        for (int jt = 0; jt < nt; jt++)
            for (int kt = 0; kt < nt; kt++) {
                if (p.lpoldamping[jt][it][kt]) ldmp = 1;
                p.lpoldamping[jt][kt][it] = p.lpoldamping[jt][it][kt];
                p.pol_damp_b[jt][kt][it] = p.pol_damp_b[jt][it][kt];
                p.pol_damp_c[jt][kt][it] = p.pol_damp_c[jt][it][kt];
                p.pol_damp_k[jt][kt][it] = p.pol_damp_k[jt][it][kt];
            }
    for (int t = 0; t < nt; t++)
        if (lpolar[t]) lpim = 1;
    if (!p.lcoulombic) lqch = ldip = lpol = ldmp = lpim = 0;
    for (int t = 0; t < nt; t++)
        for (int i = 0; i < nt; i++)
            for (int j = 0; j < nt; j++)
                if (p.pol_damp_k[t][i][j] < 0 || p.pol_damp_k[t][i][j] > 8)
                    throw Error(MDFFGPU_ERR_ARG, "pol_damp_k must be in 0..8 (MAX_TT_EXPANSION, src/tt_damp.h:3)");

    // per ion (init_config, src/config.c:124-198)
    h_typ.resize(n);
    std::vector<double> mass(n), invm(n), q(n, 0.0), pol((size_t)n * 9, 0.0), invpol((size_t)n * 9, 0.0);
    std::vector<double3> mus(n, make_double3(0, 0, 0));
    std::vector<int> polar(n, 0);
    int ia = 0;
    for (int t = 0; t < nt; t++) {
        double ip[3][3];
        if (lpolar[t]) invert3(p.polit[t], ip);
        for (int k = 0; k < p.nionit[t]; k++, ia++) {
            h_typ[ia] = t;
            mass[ia] = p.massit[t];
            invm[ia] = 1.0 / p.massit[t];
            if (p.lcoulombic) {
                q[ia] = p.qit[t];
                mus[ia] = make_double3(p.dipit[t][0], p.dipit[t][1], p.dipit[t][2]);
                if (lpolar[t]) {
                    polar[ia] = 1;
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) {
                            pol[(size_t)ia * 9 + 3 * i + j] = p.polit[t][i][j];
                            invpol[(size_t)ia * 9 + 3 * i + j] = ip[i][j];
                        }
                }
            }
        }
    }
    npol = 0;
    std::vector<int> pidx;
    for (int i = 0; i < n; i++)
        if (polar[i]) pidx.push_back(i);
    npol = (int)pidx.size();
    {   // all ions, polarisable ones first (the tensor-core ion pass's positions)
        std::vector<int> order(pidx);
        for (int i = 0; i < n; i++)
            if (!polar[i]) order.push_back(i);
        d_ion_order = dalloc<int>(n);
        MDFF_CK(cudaMemcpy(d_ion_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    }
    if (npol) {
        d_pidx = dalloc<int>(npol);
        MDFF_CK(cudaMemcpy(d_pidx, pidx.data(), sizeof(int) * npol, cudaMemcpyHostToDevice));
    }
    h_q = q;
    d_typ = dalloc<int>(n);
    d_mass = dalloc<double>(n);
    d_invmass = dalloc<double>(n);
    d_q = dalloc<double>(n);
    d_pol = dalloc<double>((size_t)n * 9);
    d_invpol = dalloc<double>((size_t)n * 9);
    d_polar = dalloc<int>(n);
    d_mu_static = dalloc<double3>(n);
    MDFF_CK(cudaMemcpy(d_typ, h_typ.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_mass, mass.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_invmass, invm.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_q, q.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_pol, pol.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_invpol, invpol.data(), sizeof(double) * 9 * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_polar, polar.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_mu_static, mus.data(), sizeof(double3) * n, cudaMemcpyHostToDevice));

    // pair tables: init_nmlj (src/nmlj.c:198-247) and init_bhmftd (src/bhmftd.c:99-110)
    std::vector<PairSR> pr((size_t)nt * nt);
    if (p.lnmlj) {
        double two16 = std::pow(2.0, 1.0 / 6.0);
        double srcut3 = srcutsq * p.cutshortrange;
        for (int it = 0; it < nt; it++)
            for (int jt = 0; jt < nt; jt++) {
                if (jt >= it) {
                    p.plj[jt][it] = p.plj[it][jt];
                    p.qlj[jt][it] = p.qlj[it][jt];
                    p.sigmalj[jt][it] = p.sigmalj[it][jt];
                    p.epslj[jt][it] = p.epslj[it][jt];
                }
                double pp = p.plj[it][jt], qq = p.qlj[it][jt];
                PairSR &P = pr[(size_t)it * nt + jt];
                P.epsqp = p.epslj[it][jt] / (qq - pp);
                P.sigsq = two16 * two16 * p.sigmalj[it][jt] * p.sigmalj[it][jt];
                P.fc = (pp * qq * P.epsqp) / P.sigsq;
                P.ptwo = pp * 0.5;
                P.qtwo = qq * 0.5;
                P.plj = pp;
                P.qlj = qq;
                double sr2 = P.sigsq / srcutsq, sr = std::sqrt(sr2);
                double srp = std::pow(sr, pp), srq = std::pow(sr, qq);
                P.uc = P.epsqp * (pp * srq - qq * srp);
                auto as_int = [](double x) { return (x == std::floor(x) && x >= 0 && x <= 64) ? (int)x : -1; };
                P.ip = as_int(P.ptwo);
                P.iq = as_int(P.qtwo);
                double ut = P.epsqp * (pp * srq / (qq - 3.0) - qq * srp / (pp - 3.0));
                double pt = pp * qq * P.epsqp * (srq / (qq - 3.0) - srp / (pp - 3.0));
                ut *= srcut3 * TPI_D;
                pt *= srcut3 * TPI_D;
                if (p.nionit[it] && p.nionit[jt]) {
                    utail += ut * p.nionit[it] * p.nionit[jt] * cell.inveOmega;
                    ptail += pt * p.nionit[it] * p.nionit[jt] * cell.inveOmega;
                }
            }
        ptail = ptail / (press_unit * 3.0);
    }
    if (p.lbhmft || p.lbhmftd) {
        for (int it = 0; it < nt; it++)
            for (int jt = it; jt < nt; jt++) {
                p.Abhmftd[jt][it] = p.Abhmftd[it][jt];
                p.Bbhmftd[jt][it] = p.Bbhmftd[it][jt];
                p.Cbhmftd[jt][it] = p.Cbhmftd[it][jt];
                p.Dbhmftd[jt][it] = p.Dbhmftd[it][jt];
                p.BDbhmftd[jt][it] = p.BDbhmftd[it][jt];
            }
        for (int it = 0; it < nt; it++)
            for (int jt = 0; jt < nt; jt++) {
                PairSR &P = pr[(size_t)it * nt + jt];
                P.A = p.Abhmftd[it][jt];
                P.B = p.Bbhmftd[it][jt];
                P.C = p.Cbhmftd[it][jt];
                P.D = p.Dbhmftd[it][jt];
                P.BD = p.BDbhmftd[it][jt];
            }
    }
    d_pair = dalloc<PairSR>((size_t)nt * nt);
    MDFF_CK(cudaMemcpy(d_pair, pr.data(), sizeof(PairSR) * nt * nt, cudaMemcpyHostToDevice));
    h_pair = pr;
    std::vector<PairDamp> dm((size_t)nt * nt);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            PairDamp &D = dm[(size_t)a * nt + b];
            D.ldamp = (p.lpoldamping[a][a][b] || p.lpoldamping[b][a][b]) ? 1 : 0;
            D.b1 = p.pol_damp_b[a][a][b];
            D.c1 = p.pol_damp_c[a][a][b];
            D.k1 = p.pol_damp_k[a][a][b];
            D.b2 = p.pol_damp_b[b][a][b];
            D.c2 = p.pol_damp_c[b][a][b];
            D.k2 = p.pol_damp_k[b][a][b];
            // which of the two directions is a declared damping (parameter updates)
            D.pad = (p.lpoldamping[a][a][b] ? 1 : 0) | (p.lpoldamping[b][a][b] ? 2 : 0);
        }
    d_damp = dalloc<PairDamp>((size_t)nt * nt);
    MDFF_CK(cudaMemcpy(d_damp, dm.data(), sizeof(PairDamp) * nt * nt, cudaMemcpyHostToDevice));
    h_damp = dm;
}

// k-vectors in the reference's generation order (set_param_kmesh, src/kspace.c:64-102),
// grouped in rows of fixed (nx, ny)
void Engine::setup_kspace() {
    for (int d = 0; d < 3; d++) {
        kmax[d] = p.kES[d];
        if (kmax[d] < 0) throw Error(MDFFGPU_ERR_ARG, "kES must be >= 0");
    }
    int K0 = kmax[0], K1 = kmax[1], K2 = kmax[2];
    nk = K2 + K1 * (2 * K2 + 1) + K0 * (2 * K1 + 1) * (2 * K2 + 1);
    if (nk <= 0) throw Error(MDFFGPU_ERR_ARG, "empty k mesh");
    std::vector<double3> kv(nk);
    std::vector<double> Ak(nk), kcoe(nk);
    std::vector<KRow> rows;
    std::vector<KSeg> segs;
    double alpha2 = p.alphaES * p.alphaES;
    const Cell &c = cell;
    int ik = 0;
    for (int nx = 0; nx < K0 + 1; nx++) {
        int nymin = (nx == 0) ? 0 : -K1;
        for (int ny = nymin; ny < K1 + 1; ny++) {
            int nzmin = (nx == 0 && ny == 0) ? 1 : -K2;
            KRow R;
            R.nx = nx;
            R.ny = ny;
            R.z0 = nzmin;
            R.cnt = K2 - nzmin + 1;
            R.koff = ik;
            R.pad0 = R.pad1 = R.pad2 = 0;
            if (R.cnt <= 0) continue;
            rows.push_back(R);
            for (int z0 = nzmin; z0 <= K2; z0 += KSEG) {
                KSeg S;
                S.nx = nx;
                S.ny = ny;
                S.z0 = z0;
                S.cnt = std::min(KSEG, K2 - z0 + 1);
                S.koff = ik + (z0 - nzmin);
                S.pad0 = S.pad1 = S.pad2 = 0;
                segs.push_back(S);
            }
            for (int nz = nzmin; nz < K2 + 1; nz++) {
                double kx = TPI_D * ((double)nx * c.B[0][0] + (double)ny * c.B[0][1] + (double)nz * c.B[0][2]);
                double ky = TPI_D * ((double)nx * c.B[1][0] + (double)ny * c.B[1][1] + (double)nz * c.B[1][2]);
                double kz = TPI_D * ((double)nx * c.B[2][0] + (double)ny * c.B[2][1] + (double)nz * c.B[2][2]);
                double kk = kx * kx + ky * ky + kz * kz;
                kv[ik] = make_double3(kx, ky, kz);
                Ak[ik] = std::exp(-kk * 0.25 / alpha2) / kk;
                kcoe[ik] = 2.0 * (1.0 / kk + 1.0 / alpha2 / 4.0);
                ik++;
            }
        }
    }
    nrow = (int)rows.size();
    nseg = (int)segs.size();
    // ion-pass k slices: whole rows, at most 512 k per slice (8 KB of shared memory);
    // the slices are the second grid dimension of the ion pass
    const int TILEK = 512;
    h_tile_row.clear();
    h_tile_k.clear();
    int r = 0;
    tile_kmax = 0;
    while (r < nrow) {
        int k0 = rows[r].koff, cnt = 0, r1 = r;
        while (r1 < nrow && cnt + rows[r1].cnt <= TILEK) {
            cnt += rows[r1].cnt;
            r1++;
        }
        if (r1 == r) throw Error(MDFFGPU_ERR_ARG, "k row longer than a tile");
        h_tile_row.push_back(r);
        h_tile_k.push_back(k0);
        tile_kmax = std::max(tile_kmax, cnt);
        r = r1;
    }
    h_tile_row.push_back(nrow);
    h_tile_k.push_back(nk);
    ntile = (int)h_tile_row.size() - 1;
    d_kvec = dalloc<double3>(nk);
    d_Ak = dalloc<double>(nk);
    d_kcoe = dalloc<double>(nk);
    d_row = dalloc<KRow>(nrow);
    d_seg = dalloc<KSeg>(nseg);
    d_tile_row = dalloc<int>(ntile + 1);
    d_tile_k = dalloc<int>(ntile + 1);
    MDFF_CK(cudaMemcpy(d_kvec, kv.data(), sizeof(double3) * nk, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_Ak, Ak.data(), sizeof(double) * nk, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_kcoe, kcoe.data(), sizeof(double) * nk, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_row, rows.data(), sizeof(KRow) * nrow, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_seg, segs.data(), sizeof(KSeg) * nseg, cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_tile_row, h_tile_row.data(), sizeof(int) * (ntile + 1), cudaMemcpyHostToDevice));
    MDFF_CK(cudaMemcpy(d_tile_k, h_tile_k.data(), sizeof(int) * (ntile + 1), cudaMemcpyHostToDevice));
    // rho pass grid: segment blocks x ion chunks filling `waves` full waves of
    // RHO_MIN_BLOCKS resident blocks per SM (MDFFGPU_RHO_WAVES overrides, default 1)
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    int segblocks = ceil_div(nseg, 128);
    double waves = 1.0;
    if (const char *w = getenv("MDFFGPU_RHO_WAVES")) waves = std::max(0.1, atof(w));
    int chunks = std::max(1, (int)(waves * RHO_MIN_BLOCKS * nsm) / segblocks);
    chunks = std::min(chunks, std::max(1, ceil_div(n, 32)));
    rho_chunk = ceil_div(n, chunks);
    rho_chunks = ceil_div(n, rho_chunk);
    d_rho_part = dalloc<double2>((size_t)rho_chunks * nk);
    d_rho = dalloc<double2>(nk);
    d_rho_acc = dalloc<double2>(nk);
    d_rho_it = dalloc<double2>(nk);
    d_ion_part = dalloc<double>((size_t)ntile * n * 12);
    setup_kspace32(*this, rows);
}

void Engine::setup_cells() {
    double cnb = p.cutshortrange + (p.lverletL ? p.skindiff : 0.0);
    double cco = p.cutlongrange + (p.lverletL ? p.skindiff : 0.0);
    double cut = std::max(cnb, cco);
    for (int d = 0; d < 3; d++) {
        int c = cut > 0 ? (int)std::floor(cell.w[d] / cut) : 1;
        nc[d] = (c >= 3 && cell.ortho) ? std::min(c, 64) : 1;
    }
    ncell = nc[0] * nc[1] * nc[2];
    int cap = 4096;
    if (ncell == 1) {
        cap = 1;
        while (cap < n) cap <<= 1;
        if (cap > 12288) throw Error(MDFFGPU_ERR_CELL, "cell too small for a cell list and too many ions to scan");
    }
    cell_cap = cap;
    if (cell_cap * sizeof(int) > 48 * 1024) {
        MDFF_CK(cudaFuncSetAttribute(k_sort_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(cell_cap * sizeof(int))));
    }
    d_cell_of = dalloc<int>(n);
    d_cell_cnt = dalloc<int>(ncell);
    d_cell_start = dalloc<int>(ncell);
    d_cell_cur = dalloc<int>(ncell);
    d_cell_ions = dalloc<int>(n);
}

void Engine::alloc_lists(int cnb, int cco) {
    dfree(d_nb);
    dfree(d_nbn);
    dfree(d_co);
    dfree(d_con);
    cap_nb = cnb;
    cap_co = cco;
    gen++;
    d_nb = dalloc<int>((size_t)n * cap_nb);
    d_nbn = dalloc<int>(n);
    d_co = dalloc<int>((size_t)n * cap_co);
    d_con = dalloc<int>(n);
    dfree(d_coef);
    if (p.lcoulombic && lpol) d_coef = dalloc<double2>((size_t)n * cap_co);
    list_ready = false;
    coef_ready = false;
}

// ---------------------------------------------------------------- state
// host<->device transfers of the reference's per-component arrays (rx[], ry[], ... ):
// one copy per array into (or out of) the device block d_soa, packed into (unpacked from)
// the engine's double4 / double3 arrays by a kernel.  From page-locked host arrays the
// copies are direct DMA; each call returns once its copies are done.
__global__ void k_pack_r(int n, const double *__restrict__ soa, const double *__restrict__ q, double4 *__restrict__ r) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = make_double4(soa[i], soa[n + i], soa[2 * (size_t)n + i], q[i]);
}
__global__ void k_pack_v(int n, const double *__restrict__ soa, double3 *__restrict__ v) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = make_double3(soa[3 * (size_t)n + i], soa[4 * (size_t)n + i], soa[5 * (size_t)n + i]);
}
__global__ void k_unpack_state(int n, const double4 *__restrict__ r, const double3 *__restrict__ v,
                               const double3 *__restrict__ f, double *__restrict__ soa) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 a = r[i];
    const double3 b = v[i], c = f[i];
    const double x[9] = {a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z};
#pragma unroll
    for (int k = 0; k < 9; k++) soa[(size_t)k * n + i] = x[k];
}
// component c of an array of `stride`-double records (positions double4, velocities
// double3) into one component slot
__global__ void k_unpack_comp(int n, int c, const double *__restrict__ src, int stride, double *__restrict__ dst) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[(size_t)i * stride + c];
}

void Engine::set_positions(const double *rx, const double *ry, const double *rz) {
    const double *src[3] = {rx, ry, rz};
    for (int k = 0; k < 3; k++)
        MDFF_CK(cudaMemcpyAsync(d_soa + (size_t)k * n, src[k], sizeof(double) * n, cudaMemcpyHostToDevice, stream));
    MDFF_LAUNCH(*this, k_pack_r, ceil_div(n, 256), 256, 0, n, d_soa, d_q, d_r);
    MDFF_CK(cudaStreamSynchronize(stream));
    if (!p.lverletL) list_ready = false;
}

void Engine::set_velocities(const double *vx, const double *vy, const double *vz) {
    const double *src[3] = {vx, vy, vz};
    for (int k = 0; k < 3; k++) {
        double *dst = d_soa + (size_t)(3 + k) * n;
        if (src[k]) MDFF_CK(cudaMemcpyAsync(dst, src[k], sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        else MDFF_CK(cudaMemsetAsync(dst, 0, sizeof(double) * n, stream));
    }
    MDFF_LAUNCH(*this, k_pack_v, ceil_div(n, 256), 256, 0, n, d_soa, d_v);
    MDFF_CK(cudaStreamSynchronize(stream));
}

void Engine::get_state(double *rx, double *ry, double *rz, double *vx, double *vy, double *vz, double *fx,
                       double *fy, double *fz) {
    MDFF_LAUNCH(*this, k_unpack_state, ceil_div(n, 256), 256, 0, n, d_r, d_v, d_f, d_soa);
    double *dst[9] = {rx, ry, rz, vx, vy, vz, fx, fy, fz};
    for (int k = 0; k < 9; k++)
        if (dst[k])
            MDFF_CK(cudaMemcpyAsync(dst[k], d_soa + (size_t)k * n, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
}

void Engine::sync_scalars() {
    MDFF_CK(cudaMemcpyAsync(h_out, d_out, sizeof(DevScalars), cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(&h_out->status, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
}

void Engine::check_status() {
    unsigned st = (unsigned)h_out->status;
    if (st & ST_CELL_OVERFLOW) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "a cell holds more ions than its capacity");
    if (st & ST_NONFINITE) throw Error(MDFFGPU_ERR_NONFINITE, "non-finite positions or forces");
    if (st & ST_TC_TIMEOUT) throw Error(MDFFGPU_ERR_TIMEOUT, "tensor-core k-space pass timed out waiting on its MMAs");
}

// ---------------------------------------------------------------- lists
// build (forced) and grow the capacities until nothing overflows
void Engine::gen_verletlist() {
    for (int attempt = 0; attempt < 8; attempt++) {
        MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
        launch_kardir(*this, d_r, d_s);
        launch_build_lists(*this, true);
        unsigned st = 0;
        MDFF_CK(cudaMemcpyAsync(&st, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
        MDFF_CK(cudaStreamSynchronize(stream));
        if (st & ST_CELL_OVERFLOW) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "cell capacity exceeded");
        if (!(st & ST_LIST_OVERFLOW)) {
            list_ready = true;
            return;
        }
        // read the largest counts and grow
        std::vector<int> a(n), b(n);
        MDFF_CK(cudaMemcpy(a.data(), d_nbn, sizeof(int) * n, cudaMemcpyDeviceToHost));
        MDFF_CK(cudaMemcpy(b.data(), d_con, sizeof(int) * n, cudaMemcpyDeviceToHost));
        int ma = *std::max_element(a.begin(), a.end()), mb = *std::max_element(b.begin(), b.end());
        int na = std::max(cap_nb, (ma * 5 / 4 + 63) / 32 * 32), nb = std::max(cap_co, (mb * 5 / 4 + 63) / 32 * 32);
        alloc_lists(na, nb);
    }
    throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "neighbour list capacity could not be grown");
}

int Engine::check_verletlist(bool reset_status) {
    if (!list_ready) {
        gen_verletlist();
        return 1;
    }
    if (reset_status) MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
    if (capturing) {
        // the rebuild as an IF node: on the steps without one its kernels do not launch
        record_if([&](cudaGraphConditionalHandle h) { launch_check_list(*this, &h); },
                  [&] { launch_build_lists(*this, false); });
        return 0;   // the host reads the rebuild flag and status after the step
    }
    launch_check_list(*this);
    launch_build_lists(*this, false);
    int rb = 0;
    unsigned st = 0;
    MDFF_CK(cudaMemcpyAsync(&rb, d_rebuild, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(&st, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    if (st & ST_LIST_OVERFLOW) {
        gen_verletlist();   // positions unchanged: rebuild with larger capacity
        return 1;
    }
    if (st & ST_CELL_OVERFLOW) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "cell capacity exceeded");
    return rb;
}

void Engine::ensure_lists() {
    if (!p.lverletL) {
        gen_verletlist();   // the reference scans all pairs each call: rebuild at the cutoff itself
        return;
    }
    if (!list_ready) throw Error(MDFFGPU_ERR_STATE, "no Verlet list: call gen_verletlist first");
}

// ---------------------------------------------------------------- force evaluation
void Engine::sr_forces(bool lj, double *u, double *pvir, double *tau) {
    launch_sr(*this, lj);
    sr_finish(lj);
    (void)u;
    (void)pvir;
    (void)tau;
}

void Engine::sr_finish(bool lj) {
    int slot = lj ? S_LJ_U : S_BH_U;
    reduce(slot, 7, ceil_div(n, 8));
    DevScalars *o = d_out;
    if (lj)
        MDFF_LAUNCH(*this, k_finalize_sr, 1, 1, 0, d_scal, slot, cell.inveOmegaPU, &o->u_lj, &o->pvir_lj, o->tau_lj);
    else
        MDFF_LAUNCH(*this, k_finalize_sr, 1, 1, 0, d_scal, slot, cell.inveOmegaPU, &o->u_bh, &o->pvir_bh, o->tau_bh);
}

static double self2_of(double alpha) {
    const double rpi = 1.7724538509055160273;
    double selfa = alpha / rpi, selfa2 = 2.0 * selfa * alpha * alpha / 3.0;
    return 2.0 * selfa2;
}

// electric field of (q, mu): self + direct + reciprocal, as multipole_ES with
// do_ef only (src/ewald.c:75-348); no energy, no forces
void Engine::field_of(const double *d_qv, const double3 *d_muv, bool lq, bool ld, bool damp, double3 *d_ef_out,
                      double2 *rho_raw) {
    if (!lq && ld && !damp && coef_ready) {
        // induced dipoles: nonzero at polarisable ions only, field needed there only
        if (use32 && real32) launch_pol_field32(*this, d_muv, d_tmp3);
        else launch_dir_field_cached(*this, d_muv, d_tmp3);
    } else if (use32 && real32) {
        launch_dir32(*this, d_qv, d_muv, p.alphaES, lq, ld, damp, false, true, d_tmp3, nullptr);
    } else {
        launch_dir(*this, d_qv, d_muv, p.alphaES, lq, ld, damp, false, true, false, false, d_tmp3, nullptr, nullptr);
    }
    RecOut o;
    o.ef = d_ef_out;
    o.ef_dir = d_tmp3;
    o.self2 = self2_of(p.alphaES);
    o.self_mu = d_muv;
    o.rho_raw = rho_raw;
    launch_rec(*this, d_qv, d_muv, lq, ld, o);
}

// field of a CG search direction p, which vanishes off the polarisable ions: the
// k-space passes run over those ions only and the field is written there only
void Engine::field_pol(const double3 *d_p, double3 *d_out, double2 *rho_raw, bool cg_ap) {
    auto real = [&] {
        if (use32 && real32) launch_pol_field32(*this, d_p, d_tmp3);
        else launch_dir_field_cached(*this, d_p, d_tmp3);
    };
    // beside the k-space passes when launch_combine32 reads d_tmp3 (mixed k space)
    if (use32 && rec32) on_side(stream == body_stream ? SIDE_BODY : SIDE_FIELD, real);
    else real();
    RecOut o;
    o.ef = d_out;
    o.ef_dir = d_tmp3;
    o.self2 = self2_of(p.alphaES);
    o.self_mu = d_p;
    o.rho_raw = rho_raw;
    o.idx = d_pidx;
    o.cnt = npol;
    o.energy = false;   // the matrix-vector product needs the field only
    if (cg_ap) {
        // the CG product (k_cg_ap) at the polarisable ions, in the same pass
        o.cg.invpol = d_invpol;
        o.cg.p = d_p;
        o.cg.ap = d_cg_ap;
        o.cg.part = d_part;
        o.cg.stride = part_stride;
        o.cg.scal = d_scal;
        o.cg.ticket = d_ticket;
    }
    launch_rec(*this, d_qzero, d_p, false, true, o);
}

// Launch shapes of the mixed k space timed on this system.  The pass timed is the CG
// field pass (the field of the current induced dipoles at the polarisable ions: rho pass
// over them, its reduction, ion pass, combine), run about three times per MD step; the
// candidates are {CUDA-core, tensor-core ion pass} x {0.5, 1, 2 x the default rho-pass ion
// chunks} x {tensor-core row slices: the cost model's, 1..4}; each is timed over `reps`
// passes with CUDA events after two untimed ones, and the fastest is kept.  A force
// evaluation runs first (phase tables, dipole-field records and dipoles of the current
// positions); the state of the system is not changed.
void Engine::tune_launch(int reps, int *choice, double *ms) {
    if (!(use32 && real32 && rec32 && p.lcoulombic && lpol && npol > 0))
        throw Error(MDFFGPU_ERR_STATE, "launch tuning applies to the mixed-precision polarisable k space");
    reps = std::max(reps, 1);
    engforce();
    struct Cand {
        int tc, chunks, slices, rtc;
    };
    std::vector<int> chunk_set;
    for (int c : {std::max(1, rho32_chunks / 2), rho32_chunks, std::min(rho32_chunks_max, 2 * rho32_chunks)})
        if (std::find(chunk_set.begin(), chunk_set.end(), c) == chunk_set.end()) chunk_set.push_back(c);
    // rho pass: the CUDA-core pass at each chunk count, or the tensor-core pass (its own
    // chunks); ion pass: the CUDA-core pass, or the tensor-core pass at 0 (cost model) to 4
    // row slices
    std::vector<Cand> cands;
    for (int rtc = 0; rtc < (d_rho_btab ? 2 : 1); rtc++)
        for (int c : (rtc ? std::vector<int>{rho32_chunks} : chunk_set))
            for (int tc = 0; tc < (d_ion_atab ? 2 : 1); tc++)
                for (int sl = 0; sl <= (tc ? 4 : 0); sl++) cands.push_back({tc, c, sl, rtc});
    cudaEvent_t t0, t1;
    MDFF_CK(cudaEventCreate(&t0));
    MDFF_CK(cudaEventCreate(&t1));
    struct EvScope {
        cudaEvent_t a, b;
        ~EvScope() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evs{t0, t1};
    Cand best{ion_tc ? 1 : 0, rho32_chunks, ion_tc_slices_set, rho_tc ? 1 : 0};
    double best_ms = 1e300;
    auto apply = [&](const Cand &c) {
        ion_tc = c.tc != 0;
        rho32_chunks = c.chunks;
        ion_tc_slices_set = c.slices;
        rho_tc = c.rtc != 0;
        if (ion_tc) launch_ion_tc_table(*this);
        if (rho_tc) launch_rho_tc_tables(*this);
    };
    for (const Cand &c : cands) {
        apply(c);
        for (int w = 0; w < 2; w++) field_pol(d_mu_ind, d_ef_ind, nullptr, false);
        MDFF_CK(cudaEventRecord(t0, stream));
        for (int r = 0; r < reps; r++) field_pol(d_mu_ind, d_ef_ind, nullptr, false);
        MDFF_CK(cudaEventRecord(t1, stream));
        MDFF_CK(cudaEventSynchronize(t1));
        float el = 0.f;
        MDFF_CK(cudaEventElapsedTime(&el, t0, t1));
        double t = el / reps;
        if (t < best_ms) {
            best_ms = t;
            best = c;
        }
    }
    apply(best);
    MDFF_CK(cudaStreamSynchronize(stream));
    gen++;   // recorded steps use the chosen shapes from now on
    if (choice) {
        choice[0] = best.tc;
        choice[1] = best.rtc ? 0 : best.chunks;
        choice[2] = best.slices;
        choice[3] = best.rtc;
    }
    if (ms) *ms = best_ms;
}

// momentpolaSCF (src/pim.c:177-306) with extrapolate_dipole_aspc (src/pim.c:314-424)
void Engine::pim_reference() {
    int nb = ceil_div(n, 256);
    field_of(d_q, d_mu_static, lqch != 0, ldip != 0, ldmp != 0, d_ef_stat);
    MDFF_CK(cudaMemcpyAsync(d_ef, d_ef_stat, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    int ord = p.extrapolate_order;
    int e = (istep >= ord + 1) ? ord : (!istep ? 0 : istep - 1);
    int es = (e != ord) ? e + 1 : e;
    static const double Wt[6] = {0.0, 2.0 / 3.0, 0.6, 4.0 / 7.0, 5.0 / 9.0, 6.0 / 11.0};
    if (ord < 0 || ord > 5) throw Error(MDFFGPU_ERR_ARG, "extrapolate_order must be 0..5");
    int iscf = 0;
    double rmsd = 1.0e300;
    double upol_pre = 0.0;
    while (((iscf < p.max_scf_pim_iter) && (rmsd > p.conv_tol_ind)) || (iscf < p.min_scf_pim_iter)) {
        MDFF_CK(cudaMemsetAsync(d_mu_ind, 0, sizeof(double3) * n, stream));
        if (!iscf) MDFF_LAUNCH(*this, k_aspc_predict, nb, 256, 0, n, aspc_coef(e, false), es, d_hist, d_mu_ind);
        else MDFF_LAUNCH(*this, k_induced, nb, 256, 0, n, d_polar, d_pol, d_ef, d_mu_ind);
        if (!iscf) {  // u_pol of the predicted dipoles (src/pim.c:253), kept if the loop ends here
            MDFF_LAUNCH(*this, k_pim_sums, nb, 256, 0, n, d_polar, d_pol, d_invpol, d_mu_ind, d_ef, d_part,
                        part_stride);
            reduce(S_UPOL, 1, nb);
            MDFF_CK(cudaMemcpyAsync(&h_out->u_pol, d_scal + S_UPOL, sizeof(double), cudaMemcpyDeviceToHost, stream));
        }
        field_of(d_qzero, d_mu_ind, false, true, false, d_ef_ind);
        MDFF_LAUNCH(*this, k_add3, nb, 256, 0, n, d_ef_stat, d_ef_ind, d_ef);
        if (!iscf) MDFF_LAUNCH(*this, k_aspc_correct, nb, 256, 0, n, Wt[e], d_polar, d_pol, d_ef, d_mu_ind);
        MDFF_LAUNCH(*this, k_pim_sums, nb, 256, 0, n, d_polar, d_pol, d_invpol, d_mu_ind, d_ef, d_part, part_stride);
        reduce(S_UPOL, 2, nb);
        double sc[2];
        MDFF_CK(cudaMemcpyAsync(sc, d_scal + S_UPOL, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
        MDFF_CK(cudaStreamSynchronize(stream));
        if (!iscf) upol_pre = h_out->u_pol;
        rmsd = std::sqrt(sc[1] / (double)std::max(npol, 1));
        if (!std::isfinite(rmsd)) throw Error(MDFFGPU_ERR_NONFINITE, "induced dipoles diverged");
        iscf++;
        h_out->u_pol = (iscf == 1) ? upol_pre : sc[0];
    }
    double upol = h_out->u_pol;
    MDFF_LAUNCH(*this, k_hist_store, nb, 256, 0, n, d_mu_ind, d_hist);
    last_scf_iter = iscf;
    last_rmsd = rmsd;
    double v = 0.5 * upol * coul_unit;   // get_upol returns 0.5*sum (src/pim.c:160)
    MDFF_CK(cudaMemcpyAsync(&d_out->u_pol, &v, sizeof(double), cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
}

// While recording: a device-controlled branch.  `test` issues the kernel that sets the
// condition through the handle, then an IF node is added and `body` is recorded into its
// body graph on body_stream (if_count receives its launches).
void Engine::record_if(const std::function<void(cudaGraphConditionalHandle)> &test,
                       const std::function<void()> &body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cgraph = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle h;
    MDFF_CK(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cgraph, nullptr, nullptr));
    MDFF_CK(cudaGraphConditionalHandleCreate(&h, cgraph, 0, 0));
    test(h);
    MDFF_CK(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cgraph, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MDFF_CK(cudaGraphAddNode(&node, cgraph, deps, ndeps, &cp));
    cudaGraph_t bgraph = cp.conditional.phGraph_out[0];
    MDFF_CK(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t outer = stream;
    stream = body_stream;
    MDFF_CK(cudaStreamBeginCaptureToGraph(stream, bgraph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        long long b0 = launches;
        body();
        if_count += launches - b0;
    } catch (...) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(stream, &g2);
        stream = outer;
        throw;
    }
    cudaGraph_t g2 = nullptr;
    MDFF_CK(cudaStreamEndCapture(stream, &g2));
    stream = outer;
}

// While recording: a device-controlled loop.  `first` issues the test that decides
// whether the loop runs at all (it sets the condition through the handle), then the
// while node is added and `body` (one iteration ending in the same test) is recorded
// into its body graph on body_stream.  body_count receives the launches of one
// iteration.
void Engine::record_while(const std::function<void(cudaGraphConditionalHandle)> &first,
                          const std::function<void(cudaGraphConditionalHandle)> &body) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cgraph = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle h;
    MDFF_CK(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cgraph, nullptr, nullptr));
    MDFF_CK(cudaGraphConditionalHandleCreate(&h, cgraph, 0, 0));
    first(h);
    MDFF_CK(cudaStreamGetCaptureInfo(stream, &cs, nullptr, &cgraph, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    MDFF_CK(cudaGraphAddNode(&node, cgraph, deps, ndeps, &cp));
    cudaGraph_t bgraph = cp.conditional.phGraph_out[0];
    MDFF_CK(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t outer = stream;
    stream = body_stream;
    MDFF_CK(cudaStreamBeginCaptureToGraph(stream, bgraph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        long long b0 = launches;
        body(h);
        body_count = launches - b0;
    } catch (...) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(stream, &g2);
        stream = outer;
        throw;
    }
    cudaGraph_t g2 = nullptr;
    MDFF_CK(cudaStreamEndCapture(stream, &g2));
    stream = outer;
}

// preconditioned conjugate gradient on (alpha^-1 - T) mu = E_stat, polarisable ions;
// initial guess extrapolated from the converged dipoles of the previous steps (the
// polynomial through the last extrapolate_order + 1 of them: the CG needs no corrector,
// so the more accurate predictor saves iterations; cg_poly false: ASPC coefficients);
// stops when the reference's residual measure
// sqrt(sum (mu/alpha - E)^2 / npol) (src/pim.c:431-449) is below conv_tol_ind
// fused: E_stat + T mu0 is one Ewald evaluation of (q, mu_static + mu0) (the residual
// needs only their sum), and rho(k) of (q, mu_static + mu) follows the iterates
// (rho is linear in mu: rho(x + a p) = rho(x) + a rho(p)), so the force evaluation
// that follows skips its rho pass (rho_acc_ready).
void Engine::pim_cg(bool fused) {
    int nb = ceil_div(n, 256);
    int ord = p.extrapolate_order;
    if (ord < 0 || ord > 5) throw Error(MDFFGPU_ERR_ARG, "extrapolate_order must be 0..5");
    int e = (istep >= ord + 1) ? ord : (!istep ? 0 : istep - 1);
    int es = (e != ord) ? e + 1 : e;
    if (fused) {
        MDFF_LAUNCH(*this, k_aspc_predict, nb, 256, 0, n, aspc_coef(e, cg_poly), es, d_hist, d_mu_ind);
        MDFF_LAUNCH(*this, k_add3, nb, 256, 0, n, d_mu_static, d_mu_ind, d_mu_tot);
        // the residual reads the field at the polarisable ions only (FP64 real space
        // evaluates every ion; the k-space ion pass and FP32 real space only those)
        bool sub = subset32 && npol > 0;
        if (use32 && real32) {
            // on the branch of the in-cutoff lists, beside the k-space passes below (the
            // FP32 k-space combine joins it)
            auto dir = [&] {
                launch_dir32(*this, d_q, d_mu_tot, p.alphaES, lqch != 0, true, ldmp != 0, false, true, d_tmp3,
                             nullptr, sub ? d_pidx : nullptr, npol);
            };
            if (rec32) on_side(SIDE_PREP, dir);
            else dir();
        } else {
            launch_dir(*this, d_q, d_mu_tot, p.alphaES, lqch != 0, true, ldmp != 0, false, true, false, false,
                       d_tmp3, nullptr, nullptr);
        }
        RecOut o;
        o.ef = d_ef_ind;
        o.ef_dir = d_tmp3;
        o.self2 = self2_of(p.alphaES);
        o.self_mu = d_mu_tot;
        o.rho_raw = d_rho_acc;
        if (sub) {
            o.out_idx = d_pidx;
            o.out_cnt = npol;
        }
        launch_rec(*this, d_q, d_mu_tot, lqch != 0, true, o);
        join_side(SIDE_PREP);   // (joined by the combine already; the loop below reads the records)
        MDFF_LAUNCH(*this, k_cg_residual, nb, 256, 0, n, d_polar, d_invpol, d_muzero, d_ef_ind, d_mu_ind, d_cg_r);
    } else {
        field_of(d_q, d_mu_static, lqch != 0, ldip != 0, ldmp != 0, d_ef_stat);
        MDFF_LAUNCH(*this, k_aspc_predict, nb, 256, 0, n, aspc_coef(e, cg_poly), es, d_hist, d_mu_ind);
        field_of(d_qzero, d_mu_ind, false, true, false, d_ef_ind);
        MDFF_LAUNCH(*this, k_cg_residual, nb, 256, 0, n, d_polar, d_invpol, d_ef_stat, d_ef_ind, d_mu_ind, d_cg_r);
    }
    MDFF_LAUNCH(*this, k_cg_rz, nb, 256, 0, n, d_polar, d_pol, d_cg_r, d_mu_save, d_part, part_stride, d_scal,
                d_ticket + 1);
    MDFF_CK(cudaMemcpyAsync(d_cg_p, d_mu_save, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    int maxit = std::max(p.max_scf_pim_iter, 1);
    // one CG iteration up to the new residual norm and, recorded, the loop test in the
    // same launch (p <- z + beta p follows the test)
    CgTest test{};
    test.mode = 1;
    test.out = d_out;
    test.npol = npol;
    test.tol = p.conv_tol_ind;
    test.maxit = maxit;
    test.status = d_status;
    test.guard = d_ticket + 4;
    auto iteration = [&](CgTest t) {
        if (fused && subset32 && npol > 0) {
            // T p over the polarisable ions; Ap and p.Ap in the FP32 k-space combine, or
            // by k_cg_ap after the FP64 one
            bool ap_in_combine = use32 && rec32;
            field_pol(d_cg_p, d_ef_ind, d_rho_it, ap_in_combine);
            if (!ap_in_combine)
                MDFF_LAUNCH(*this, k_cg_ap, nb, 256, 0, n, d_polar, d_invpol, d_cg_p, d_ef_ind, d_cg_ap, d_part,
                            part_stride, d_scal, d_ticket);
        } else {
            field_of(d_qzero, d_cg_p, false, true, false, d_ef_ind, fused ? d_rho_it : nullptr);
            MDFF_LAUNCH(*this, k_cg_ap, nb, 256, 0, n, d_polar, d_invpol, d_cg_p, d_ef_ind, d_cg_ap, d_part,
                        part_stride, d_scal, d_ticket);
        }
        // x, r update, rho(k) of the iterate, z = alpha r and the new r.z, r.r: one launch
        MDFF_LAUNCH(*this, k_cg_step, nb + (fused ? ceil_div(nk, 256) : 0), 256, 0, n, nk, d_polar, d_pol, d_scal,
                    d_cg_p, d_cg_ap, d_mu_ind, d_cg_r, d_mu_save, d_rho_it, fused ? d_rho_acc : nullptr, d_part,
                    part_stride, d_ticket + 1, t);
    };
    if (capturing) {
        // graph: the loop is a while node whose condition the device test sets
        record_while(
            [&](cudaGraphConditionalHandle h) {
                test.h = h;
                MDFF_LAUNCH(*this, k_cg_test, 1, 32, 0, test, d_scal);
            },
            [&](cudaGraphConditionalHandle h) {
                test.h = h;
                iteration(test);
                MDFF_LAUNCH(*this, k_cg_dir, nb, 256, 0, n, d_scal, d_mu_save, d_cg_p, test);
            });
    } else {
        double rr = 0.0;
        MDFF_CK(cudaMemcpyAsync(&rr, d_scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, stream));
        MDFF_CK(cudaStreamSynchronize(stream));
        double rmsd = std::sqrt(rr / (double)std::max(npol, 1));
        int it = 0;
        CgTest none{};
        while (rmsd > p.conv_tol_ind && it < maxit) {
            iteration(none);
            MDFF_CK(cudaMemcpyAsync(&rr, d_scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, stream));
            MDFF_CK(cudaStreamSynchronize(stream));
            rmsd = std::sqrt(rr / (double)std::max(npol, 1));
            if (!std::isfinite(rmsd)) throw Error(MDFFGPU_ERR_NONFINITE, "CG diverged");
            it++;
            if (rmsd <= p.conv_tol_ind) break;
            MDFF_LAUNCH(*this, k_cg_dir, nb, 256, 0, n, d_scal, d_mu_save, d_cg_p, none);
        }
        if (rmsd > p.conv_tol_ind) throw Error(MDFFGPU_ERR_SCF, "CG did not converge in max_scf_pim_iter");
        last_scf_iter = it;
        last_rmsd = rmsd;
    }
    MDFF_LAUNCH(*this, k_pim_sums, nb, 256, 0, n, d_polar, d_pol, d_invpol, d_mu_ind, d_ef_stat, d_part, part_stride);
    reduce(S_UPOL, 1, nb);
    MDFF_LAUNCH(*this, k_upol_final, 1, 32, 0, d_scal, coul_unit, d_out);
    MDFF_LAUNCH(*this, k_hist_store, nb, 256, 0, n, d_mu_ind, d_hist);
    rho_acc_ready = fused;
}

// get_rmsd_mu (src/pim.c:431-449) of (mu, ef); also returns sum mu.invpol.mu
double Engine::rmsd_of(const double3 *d_mu, const double3 *d_ef, double *upol_sum) {
    int nb = ceil_div(n, 256);
    MDFF_LAUNCH(*this, k_pim_sums, nb, 256, 0, n, d_polar, d_pol, d_invpol, d_mu, d_ef, d_part, part_stride);
    reduce(S_UPOL, 2, nb);
    double sc[2];
    MDFF_CK(cudaMemcpyAsync(sc, d_scal + S_UPOL, sizeof(double) * 2, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    if (upol_sum) *upol_sum = sc[0];
    double r = std::sqrt(sc[1] / (double)std::max(npol, 1));
    if (!std::isfinite(r)) throw Error(MDFFGPU_ERR_NONFINITE, "induced dipoles diverged");
    return r;
}

// induced_moment_inner_kO (src/pim.c:647-748): real-space-only relaxation of the
// dipole increment with alpha_Ewald = 0.001 (src/pim.c:694) and omegakO mixing
void Engine::ko_inner(double3 *d_dmu, const double3 *d_find) {
    int nb = ceil_div(n, 256);
    const double ak = 0.001, om = p.omegakO;
    double rmsd_ext = rmsd_of(d_muzero, d_find, nullptr);
    MDFF_LAUNCH(*this, k_induced, nb, 256, 0, n, d_polar, d_pol, d_find, d_dmu);
    MDFF_LAUNCH(*this, k_scale_add3, nb, 256, 0, n, 0.0, d_dmu, om, d_dmu);
    int it = 0;
    double rmsd_in = 1.0e300;
    while ((it <= 20) && (rmsd_in > 0.1 * rmsd_ext)) {
        it++;
        MDFF_CK(cudaMemcpyAsync(d_mu_save, d_dmu, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
        launch_dir(*this, d_qzero, d_dmu, ak, false, true, false, false, true, false, false, d_tmp3, nullptr,
                   nullptr);
        MDFF_LAUNCH(*this, k_self_plus_dir, nb, 256, 0, n, self2_of(ak), d_dmu, d_tmp3, d_ef_ind);
        MDFF_LAUNCH(*this, k_add3, nb, 256, 0, n, d_find, d_ef_ind, d_ef_ind);   // ef_tot = ef_ext + ef_ind
        rmsd_in = rmsd_of(d_dmu, d_ef_ind, nullptr);
        MDFF_LAUNCH(*this, k_induced, nb, 256, 0, n, d_polar, d_pol, d_ef_ind, d_dmu);
        MDFF_LAUNCH(*this, k_scale_add3, nb, 256, 0, n, 1.0 - om, d_mu_save, om, d_dmu);
    }
}

// momentpolaSCFkO (src/pim.c:457-603)
void Engine::pim_ko() {
    int nb = ceil_div(n, 256);
    field_of(d_q, d_mu_static, lqch != 0, ldip != 0, ldmp != 0, d_ef_stat);
    MDFF_CK(cudaMemcpyAsync(d_ef, d_ef_stat, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_cg_r, d_ef_stat, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));  // f_ind
    MDFF_CK(cudaMemsetAsync(d_mu_ind, 0, sizeof(double3) * n, stream));
    MDFF_CK(cudaMemsetAsync(d_cg_p, 0, sizeof(double3) * n, stream));   // dmu_ind
    int ord = p.extrapolate_order;
    if (ord < 0 || ord > 5) throw Error(MDFFGPU_ERR_ARG, "extrapolate_order must be 0..5");
    int e = (istep >= ord + 1) ? ord : (!istep ? 0 : istep - 1);
    int es = (e != ord) ? e + 1 : e;
    static const double Wt[6] = {0.0, 2.0 / 3.0, 0.6, 4.0 / 7.0, 5.0 / 9.0, 6.0 / 11.0};
    int iscf = 0;
    double rmsd = 1.0e300, upol = 0.0;
    while (((iscf < p.max_scf_pim_iter) && (rmsd > p.conv_tol_ind)) || (iscf < p.min_scf_pim_iter)) {
        if ((!iscf) && (istep > 1)) {
            MDFF_LAUNCH(*this, k_aspc_predict, nb, 256, 0, n, aspc_coef(e, false), es, d_hist, d_mu_ind);
        } else {
            ko_inner(d_cg_p, d_cg_r);
            MDFF_LAUNCH(*this, k_scale_add3, nb, 256, 0, n, 1.0, d_cg_p, 1.0, d_mu_ind);
        }
        rmsd_of(d_mu_ind, d_ef, &upol);   // u_pol of these dipoles (src/pim.c:539)
        field_of(d_qzero, d_mu_ind, false, true, false, d_ef_ind);
        MDFF_LAUNCH(*this, k_add3, nb, 256, 0, n, d_ef_stat, d_ef_ind, d_ef);
        if (!iscf) MDFF_LAUNCH(*this, k_aspc_correct, nb, 256, 0, n, Wt[e], d_polar, d_pol, d_ef, d_mu_ind);
        rmsd = rmsd_of(d_mu_ind, d_ef, nullptr);
        MDFF_LAUNCH(*this, k_ko_find, nb, 256, 0, n, d_polar, d_invpol, d_ef, d_mu_ind, d_cg_r);
        iscf++;
    }
    MDFF_LAUNCH(*this, k_hist_store, nb, 256, 0, n, d_mu_ind, d_hist);
    last_scf_iter = iscf;
    last_rmsd = rmsd;
    double v = 0.5 * upol * coul_unit;
    MDFF_CK(cudaMemcpyAsync(&d_out->u_pol, &v, sizeof(double), cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
}

// get_dipoles (src/coulombic.c:67-130): mu = static + induced
void Engine::get_dipoles() {
    // mixed precision: in-cutoff list and dipole-field records of these positions (the
    // real-space kernels of this force evaluation read them)
    if (use32 && real32) {
        // issued beside the k-space tables; the fused CG's first field pass continues that
        // branch with its real-space part and its k-space combine joins it
        const bool cont = lpol && pim_solver == MDFFGPU_PIM_CG_FUSED && rec32;
        if (!prep_issued) launch_pair_prep32(*this);
        else if (!cont) join_side(SIDE_PREP);
        prep_issued = false;
    }
    if (lpol) {
        // positions are fixed through the solve: cache the dipole-field pair factors
        struct CoefScope {
            bool &flag;
            ~CoefScope() { flag = false; }
        } scope{coef_ready};
        if (!(use32 && real32)) launch_dir_prep(*this, p.alphaES);
        coef_ready = true;
        if (pim_solver == MDFFGPU_PIM_CG || pim_solver == MDFFGPU_PIM_CG_FUSED)
            pim_cg(pim_solver == MDFFGPU_PIM_CG_FUSED);
        else if (p.algo_pim == 1) pim_ko();
        else pim_reference();
        int nb = ceil_div(n, 256);
        MDFF_LAUNCH(*this, k_add3, nb, 256, 0, n, d_mu_static, d_mu_ind, d_mu_tot);
    } else {
        MDFF_CK(cudaMemcpyAsync(d_mu_tot, d_mu_static, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    }
}

void Engine::finalize_coul(bool stress) {
    CoulFin cf;
    cf.alpha = p.alphaES;
    cf.coul = coul_unit;
    cf.inveOmegaPU = cell.inveOmegaPU;
    cf.ttpiV = 2.0 * TPI_D * cell.inveOmega;
    cf.do_dir = 1;
    cf.do_rec = 1;
    cf.do_stress = stress;
    MDFF_LAUNCH(*this, k_finalize_coul, 1, 1, 0, d_scal, cf, &d_out->u_coul, &d_out->pvir_coul, d_out->tau_coul);
}

// engforce, src/field.c:352-407
void Engine::engforce(bool check_finite) {
    ensure_lists();
    MDFF_CK(cudaMemsetAsync(d_f, 0, sizeof(double3) * n, stream));
    launch_kardir(*this, d_r, d_s);
    // side branches from here (they read the fractional coordinates): the short-range
    // pairs, which add into d_f (joined before the k-space force combine reads it), and
    // in mixed precision the in-cutoff lists (joined before the dipole solve)
    if (p.lnmlj || p.lbhmft || p.lbhmftd)
        on_side(SIDE_SR, [&] {
            if (p.lnmlj) sr_forces(true, nullptr, nullptr, nullptr);
            if (p.lbhmft || p.lbhmftd) sr_forces(false, nullptr, nullptr, nullptr);
        });
    if (p.lcoulombic && use32 && real32) {
        on_side(SIDE_PREP, [&] { launch_pair_prep32(*this); });
        prep_issued = true;
    }
    if (use32) launch_coords32(*this);
    if (p.lcoulombic) {
        rho_acc_ready = false;
        get_dipoles();
        bool ld = (ldip || lpol);
        // direct space: forces, energy, virial (do_forces, do_stress; src/field.c:381-383);
        // beside the k-space force pass in mixed precision (launch_combine32 joins it)
        auto direct = [&] {
            if (use32 && real32)
                launch_dir32(*this, d_q, d_mu_tot, p.alphaES, lqch != 0, ld, ldmp != 0, true, false, nullptr, d_tmp3);
            else
                launch_dir(*this, d_q, d_mu_tot, p.alphaES, lqch != 0, ld, ldmp != 0, true, false, false, false,
                           nullptr, nullptr, d_tmp3);
            reduce(S_DIR_U, 7, ceil_div(n, 8));
        };
        if (use32 && rec32) on_side(SIDE_DIR, direct);
        else direct();
        if (!(use32 && rec32)) join_side(SIDE_SR);
        RecOut o;
        o.f = d_f;
        o.f_dir = d_tmp3;
        o.coul = coul_unit;
        if (rho_acc_ready) o.rho_acc = d_rho_acc;   // rho(k) of (q, mu_tot) from the fused CG
        rho_acc_ready = false;
        launch_rec(*this, d_q, d_mu_tot, lqch != 0, ld, o);
        join_side(SIDE_DIR);
        int nb = ceil_div(n, 256);
        MDFF_LAUNCH(*this, k_self_sums, nb, 256, 0, n, d_q, d_mu_tot, d_part, part_stride);
        reduce(S_Q2, 2, nb);
        finalize_coul(true);
    }
    for (int k = 0; k < NSIDE; k++) join_side(k);
    prep_issued = false;
    if (check_finite) MDFF_LAUNCH(*this, k_check_finite, ceil_div(n, 256), 256, 0, n, d_r, d_f, d_status);
}

// multipole_ES on caller data (src/ewald.c:75-348)
void Engine::multipole_es_dev(const double *d_qv, const double3 *d_muv, double alpha, int flags, double3 *d_ef_out,
                              double *d_efg_out, double3 *d_f_out) {
    bool lq = flags & MDFFGPU_ES_LQ, ld = flags & MDFFGPU_ES_LD, damp = flags & MDFFGPU_ES_LDAMP;
    bool fo = flags & MDFFGPU_ES_FORCES, st = flags & MDFFGPU_ES_STRESS, ef = flags & MDFFGPU_ES_EF;
    bool efg = flags & MDFFGPU_ES_EFG, dir = flags & MDFFGPU_ES_DIR, rec = flags & MDFFGPU_ES_REC;
    ensure_lists();
    launch_kardir(*this, d_r, d_s);
    if (use32) launch_coords32(*this);
    int nb = ceil_div(n, 256);
    double self2 = self2_of(alpha);
    // efg_dir accumulates the charge part when do_efg and the dipole part when do_efg
    // or do_forces (src/ewald.c:724-757)
    bool want_efg_dir = efg || (fo && ld);
    double3 *efd = d_ef_ind, *fd = d_tmp3;
    double *egd = d_efg;
    MDFF_CK(cudaMemsetAsync(d_part + (size_t)S_DIR_U * part_stride, 0, sizeof(double) * 7 * part_stride, stream));
    MDFF_CK(cudaMemsetAsync(d_scal, 0, sizeof(double) * NSLOT, stream));
    MDFF_CK(cudaMemsetAsync(efd, 0, sizeof(double3) * n, stream));
    MDFF_CK(cudaMemsetAsync(fd, 0, sizeof(double3) * n, stream));
    MDFF_CK(cudaMemsetAsync(egd, 0, sizeof(double) * 9 * n, stream));
    if (dir) {
        launch_dir(*this, d_qv, d_muv, alpha, lq, ld, damp, fo || st, ef, want_efg_dir, efg, ef ? efd : nullptr,
                   want_efg_dir ? egd : nullptr, fd);
        reduce(S_DIR_U, 7, ceil_div(n, 8));
    }
    if (rec) {
        RecOut o;
        o.ef = ef ? d_ef_out : nullptr;   // without do_ef the field is the self term only
        o.ef_dir = efd;
        o.self2 = self2;
        o.f = fo ? d_f_out : nullptr;
        o.f_dir = fd;
        o.coul = coul_unit;
        o.efg = (d_efg_out && ef) ? d_efg_out : nullptr;   // do_ef passed as do_efg, src/ewald.c:169
        o.efg_dir = egd;
        o.self_q = d_qv;
        o.self_mu = d_muv;
        launch_rec(*this, d_qv, d_muv, lq, ld, o);
        if (!ef) MDFF_LAUNCH(*this, k_self_plus_dir, nb, 256, 0, n, self2, d_muv, efd, d_ef_out);
        if (d_efg_out && !ef) MDFF_LAUNCH(*this, k_efg_self_dir, nb, 256, 0, n, self2, d_qv, egd, d_efg_out);
    } else {
        MDFF_LAUNCH(*this, k_self_plus_dir, nb, 256, 0, n, self2, d_muv, efd, d_ef_out);
        if (fo) MDFF_LAUNCH(*this, k_axpy3, nb, 256, 0, n, coul_unit, fd, d_f_out);
        if (d_efg_out) MDFF_LAUNCH(*this, k_efg_self_dir, nb, 256, 0, n, self2, d_qv, egd, d_efg_out);
    }
    MDFF_LAUNCH(*this, k_self_sums, nb, 256, 0, n, d_qv, d_muv, d_part, part_stride);
    reduce(S_Q2, 2, nb);
    CoulFin cf;
    cf.alpha = alpha;
    cf.coul = coul_unit;
    cf.inveOmegaPU = cell.inveOmegaPU;
    cf.ttpiV = 2.0 * TPI_D * cell.inveOmega;
    cf.do_dir = dir;
    cf.do_rec = rec;
    cf.do_stress = st;
    MDFF_CK(cudaMemsetAsync(d_out->tau_coul, 0, sizeof(double) * 9, stream));
    MDFF_LAUNCH(*this, k_finalize_coul, 1, 1, 0, d_scal, cf, &d_out->u_coul, &d_out->pvir_coul, d_out->tau_coul);
}

// ---------------------------------------------------------------- kernel timing
void Engine::prof_begin(const char *name, int *slot) {
    *slot = -1;
    if (prof_name.empty() || prof_name != name) return;
    if (prof_next >= (int)prof_pool.size()) {
        cudaEvent_t ev;
        MDFF_CK(cudaEventCreate(&ev));
        prof_pool.push_back(ev);
    }
    *slot = prof_next++;
    MDFF_CK(cudaEventRecord(prof_pool[*slot], stream));
}

void Engine::prof_end(const char *name, int slot, double flops) {
    if (slot < 0) return;
    if (prof_next >= (int)prof_pool.size()) {
        cudaEvent_t ev;
        MDFF_CK(cudaEventCreate(&ev));
        prof_pool.push_back(ev);
    }
    int s2 = prof_next++;
    MDFF_CK(cudaEventRecord(prof_pool[s2], stream));
    prof_pairs.push_back({slot, s2});
    prof_flops += flops;
    (void)name;
}

void Engine::prof_result(double *ms, long long *count, double *flops) {
    MDFF_CK(cudaStreamSynchronize(stream));
    double t = 0.0;
    for (auto &pr : prof_pairs) {
        float m = 0.f;
        MDFF_CK(cudaEventElapsedTime(&m, prof_pool[pr.first], prof_pool[pr.second]));
        t += m;
    }
    *ms = t;
    *count = (long long)prof_pairs.size();
    *flops = prof_flops;
}

// ---------------------------------------------------------------- integration
void Engine::prop_agate(int step) {
    istep = step;
    int nb = ceil_div(n, 256);
    switch (p.egrator) {
    case 0: {  // prop_leap_frog, src/integration.c:93-137
        engforce();
        MDFF_LAUNCH(*this, k_lf, nb, 256, 0, n, dt * dt, 0.5 / dt, d_invmass, d_mass, d_r, d_rs, d_v, d_f, d_part,
                    part_stride);
        reduce(S_KIN, 1, nb);
        MDFF_LAUNCH(*this, k_set_ekin, 1, 1, 0, d_scal, d_out);
        break;
    }
    case 2: {  // nhcn, src/integration.c:140-182
        NhcArgs a;
        a.nn = p.nhc_n;
        a.yo = p.nhc_yosh_order;
        a.mults = p.nhc_mults;
        a.dt = dt;
        a.temp = temp;
        a.L = 3.0 * (double)n;
        for (int k = 0; k < 7; k++) a.w[k] = 0.0;
        switch (a.yo) {  // Yoshida weights, src/integration.c:205-236
        case 1: a.w[0] = 1.0; break;
        case 3:
            a.w[0] = 1.0 / (2.0 - std::pow(2.0, 1.0 / 3.0));
            a.w[1] = 1.0 - 2.0 * a.w[0];
            a.w[2] = a.w[0];
            break;
        case 5:
            a.w[0] = 1.0 / (4.0 - std::pow(4.0, 1.0 / 3.0));
            a.w[1] = a.w[2] = a.w[3] = a.w[0];
            a.w[4] = 1.0 - 4.0 * a.w[0];
            break;
        case 7:
            a.w[0] = .78451361047756;
            a.w[1] = .235573213359357;
            a.w[2] = -1.17767998417887;
            a.w[3] = 1.0 - 2.0 * (a.w[0] + a.w[1] + a.w[2]);
            a.w[4] = a.w[2];
            a.w[5] = a.w[1];
            a.w[6] = a.w[0];
            break;
        default: throw Error(MDFFGPU_ERR_ARG, "nhc_yosh_order must be 1, 3, 5 or 7");
        }
        if (a.nn < 2 || a.nn > 16) throw Error(MDFFGPU_ERR_ARG, "nhc_n must be in 2..16");
        // the kinetic sums are reduced by the last block of the kernel that forms them
        ScaleKinArgs sk;
        sk.n = n;
        sk.energy = 0;
        sk.nn = a.nn;
        sk.L = a.L;
        sk.temp = temp;
        sk.out_s = d_out;
        sk.mass = d_mass;
        sk.nhc = d_nhc;
        sk.v = d_v;
        sk.part = d_part;
        sk.scal = d_scal;
        sk.stride = part_stride;
        sk.ticket = d_ticket + 6;
        sk.out = d_out;
        sk.scale = 0;
        MDFF_LAUNCH(*this, k_scale_kin, nb, 256, 0, sk);
        launch_nhc_chain(*this, a, d_nhc, d_scal, d_out);
        sk.scale = 1;
        MDFF_LAUNCH(*this, k_scale_kin, nb, 256, 0, sk);
        MDFF_LAUNCH(*this, k_pv1, nb, 256, 0, n, dt, dt * 0.5, d_invmass, d_r, d_v, d_f);
        engforce(false);   // the finiteness check runs in k_pv2
        MDFF_LAUNCH(*this, k_pv2, nb, 256, 0, n, dt * 0.5, d_invmass, d_mass, d_v, d_f, d_part, part_stride,
                    d_scal, d_ticket + 6, d_r, d_status);
        launch_nhc_chain(*this, a, d_nhc, d_scal, d_out);
        sk.energy = 1;   // then e_kin and e_nvt
        MDFF_LAUNCH(*this, k_scale_kin, nb, 256, 0, sk);
        break;
    }
    default: {  // prop_velocity_verlet, src/integration.c:22-63
        double dtsq2 = dt * dt * 0.5, dt2 = dt * 0.5;
        MDFF_LAUNCH(*this, k_vv1, nb, 256, 0, n, dt, dtsq2, d_invmass, d_r, d_v, d_f, d_f2);
        engforce();
        MDFF_LAUNCH(*this, k_vv2, nb, 256, 0, n, dt2, d_invmass, d_mass, d_v, d_f, d_f2, d_part, part_stride);
        reduce(S_KIN, 1, nb);
        MDFF_LAUNCH(*this, k_set_ekin, 1, 1, 0, d_scal, d_out);
        break;
    }
    }
}

// a step can be replayed from a graph once nothing in it needs the host: Verlet lists
// (rebuilt on the device when due), a CG solver, the ASPC order at its final value
bool Engine::graph_ok(int step) const {
    if (!graph_on || !p.lverletL || !prof_name.empty()) return false;
    if (p.lcoulombic && lpol) {
        if (pim_solver != MDFFGPU_PIM_CG && pim_solver != MDFFGPU_PIM_CG_FUSED) return false;
        if (step < p.extrapolate_order + 1) return false;
    }
    return true;
}

void Engine::drop_graph() {
    if (step_exec) cudaGraphExecDestroy(step_exec);
    step_exec = nullptr;
    graph_gen = -1;
    if (fit_exec) cudaGraphExecDestroy(fit_exec);
    fit_exec = nullptr;
    fit_graph_gen = -1;
}

// record prop_agate + check_verletlist of one step (src/md.c:237-241) as a graph
void Engine::capture_step(int step) {
    drop_graph();
    if (use32 && real32 && p.lcoulombic) ensure_real32();   // no allocation while recording
    MDFF_CK(cudaStreamSynchronize(stream));
    long long l0 = launches;
    body_count = 0;
    if_count = 0;
    MDFF_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    cudaGraph_t graph = nullptr;
    try {
        MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
        prop_agate(step);
        check_verletlist(false);
    } catch (...) {
        capturing = false;
        forget_sides();
        cudaStreamEndCapture(stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        launches = l0;
        throw;
    }
    capturing = false;
    MDFF_CK(cudaStreamEndCapture(stream, &graph));
    cudaError_t err = cudaGraphInstantiate(&step_exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        step_exec = nullptr;
        MDFF_CK(err);
    }
    graph_body = body_count;
    graph_if = if_count;
    graph_outer = launches - l0 - body_count - if_count;
    launches = l0;
    graph_gen = gen;
}

// run_md's loop body (src/md.c:229-241)
void Engine::md_steps(int first, int nsteps, double *thermo, const double *const *in, double *const *out) {
    if (in) {
        // the caller's positions and velocities, packed on the device (no synchronisation:
        // the step's own one below, or the list build's, covers the copies)
        for (int k = 0; k < 6; k++) {
            double *dst = d_soa + (size_t)k * n;
            if (in[k]) MDFF_CK(cudaMemcpyAsync(dst, in[k], sizeof(double) * n, cudaMemcpyHostToDevice, stream));
        }
        if (in[0] || in[1] || in[2]) {
            // components not given keep their device values
            for (int k = 0; k < 3; k++)
                if (!in[k]) MDFF_LAUNCH(*this, k_unpack_comp, ceil_div(n, 256), 256, 0, n, k, (const double *)d_r, 4,
                                        d_soa + (size_t)k * n);
            MDFF_LAUNCH(*this, k_pack_r, ceil_div(n, 256), 256, 0, n, d_soa, d_q, d_r);
            if (!p.lverletL) list_ready = false;
        }
        if (in[3] || in[4] || in[5]) {
            for (int k = 3; k < 6; k++)
                if (!in[k]) MDFF_LAUNCH(*this, k_unpack_comp, ceil_div(n, 256), 256, 0, n, k - 3, (const double *)d_v,
                                        3, d_soa + (size_t)k * n);
            MDFF_LAUNCH(*this, k_pack_v, ceil_div(n, 256), 256, 0, n, d_soa, d_v);
        }
    }
    auto queue_out = [&] {
        if (!out) return;
        MDFF_LAUNCH(*this, k_unpack_state, ceil_div(n, 256), 256, 0, n, d_r, d_v, d_f, d_soa);
        for (int k = 0; k < 9; k++)
            if (out[k])
                MDFF_CK(cudaMemcpyAsync(out[k], d_soa + (size_t)k * n, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                        stream));
    };
    if (nsteps == 0) {
        queue_out();
        MDFF_CK(cudaStreamSynchronize(stream));
        return;
    }
    if (p.lverletL && !list_ready) gen_verletlist();
    for (int s = 0; s < nsteps; s++) {
        int step = first + s;
        bool graphed = graph_ok(step);
        if (graphed) {
            if (!step_exec || graph_gen != gen) capture_step(step);
            istep = step;
            MDFF_CK(cudaGraphLaunch(step_exec, stream));
        } else {
            MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
            prop_agate(step);
            if (p.lverletL) check_verletlist(false);
        }
        if (s == nsteps - 1) queue_out();   // on the last step's synchronisation
        sync_scalars();
        if (graphed) {
            launches += graph_outer + graph_body * std::max(h_out->scf_iter, 0) + (h_out->rebuild ? graph_if : 0);
            if (p.lcoulombic && lpol) {
                last_scf_iter = h_out->scf_iter;
                last_rmsd = h_out->scf_rmsd;
            }
            unsigned st = (unsigned)h_out->status;
            if (st & ST_SCF) throw Error(MDFFGPU_ERR_SCF, "CG did not converge in max_scf_pim_iter");
            if (st & ST_LIST_OVERFLOW) gen_verletlist();   // positions unchanged: rebuild larger
        }
        check_status();
        if (thermo) {
            double *t = thermo + 12 * (size_t)s;
            t[0] = h_out->e_kin;
            t[1] = h_out->u_lj;
            t[2] = h_out->u_bh;
            t[3] = h_out->u_coul;
            t[4] = h_out->u_pol;
            t[5] = h_out->e_nvt;
            t[6] = h_out->pvir_lj;
            t[7] = h_out->pvir_bh;
            t[8] = h_out->pvir_coul;
            t[9] = (double)h_out->nbuilds;
            t[10] = (double)last_scf_iter;
            t[11] = last_rmsd;
        }
    }
}

}  // namespace mdffgpu
