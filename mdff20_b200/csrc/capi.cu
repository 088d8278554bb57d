// extern "C" entry points of libmdffgpu (declared in include/mdffgpu.h): argument
// checks, host<->device transfer and conversion of engine exceptions to status codes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "engine.cuh"

using mdffgpu::Engine;
using mdffgpu::Error;

struct mdffgpu_ctx {
    Engine *e;
    std::string err;
};

mdffgpu::Engine *mdffgpu_engine_of(mdffgpu_ctx *ctx) { return ctx ? ctx->e : nullptr; }

namespace {

template <typename F>
int guarded(mdffgpu_ctx *ctx, F &&f) {
    if (!ctx || !ctx->e) return MDFFGPU_ERR_ARG;
    try {
        f(*ctx->e);
        return MDFFGPU_OK;
    } catch (const Error &x) {
        ctx->err = x.what();
        return x.code;
    } catch (const std::exception &x) {
        ctx->err = x.what();
        return MDFFGPU_ERR_CUDA;
    }
}

void upload(Engine &e, void *dst, const void *src, size_t bytes) {
    MDFF_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, e.stream));
}
void download(Engine &e, void *dst, const void *src, size_t bytes) {
    MDFF_CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, e.stream));
}

}  // namespace

// ions from which the mixed k space runs on the tensor cores by default (the batched fit's
// configurations of 96 to 1536 ions evaluate faster on the CUDA-core passes)
constexpr int TC_MIN_IONS = 4096;

struct mdffgpu_fit_plan {
    std::vector<mdffgpu_ctx *> ctx;
    int tSi = 0, tO = 0, device = 0;
    double scale = 0.0;
    double *d_theta = nullptr;   // shared by every recorded evaluation
    double *d_res = nullptr;     // [nconf][FIT_NRES]
    double *h_theta = nullptr, *h_res = nullptr;   // pinned staging
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_theta = nullptr;
    std::vector<cudaEvent_t> ev_done;
    std::string err;
    ~mdffgpu_fit_plan() {
        for (cudaEvent_t e : ev_done) cudaEventDestroy(e);
        if (ev_theta) cudaEventDestroy(ev_theta);
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_theta);
        cudaFree(d_res);
        if (h_theta) cudaFreeHost(h_theta);
        if (h_res) cudaFreeHost(h_res);
    }
};

namespace {
template <typename F>
int plan_guarded(mdffgpu_fit_plan *plan, F &&f) {
    if (!plan) return MDFFGPU_ERR_ARG;
    try {
        f(*plan);
        return MDFFGPU_OK;
    } catch (const Error &x) {
        plan->err = x.what();
        return x.code;
    } catch (const std::exception &x) {
        plan->err = x.what();
        return MDFFGPU_ERR_CUDA;
    }
}
}  // namespace

extern "C" {

int mdffgpu_create(const mdffgpu_params *p, const double *rx, const double *ry, const double *rz, const double *vx,
                   const double *vy, const double *vz, int device, mdffgpu_ctx **out) {
    if (!p || !rx || !ry || !rz || !out) return MDFFGPU_ERR_ARG;
    *out = nullptr;
    mdffgpu_ctx *c = new mdffgpu_ctx();
    c->e = nullptr;
    try {
        c->e = new Engine(*p, device);
        c->e->set_positions(rx, ry, rz);
        c->e->set_velocities(vx, vy, vz);
    } catch (const Error &x) {
        int code = x.code;
        delete c->e;
        delete c;
        return code;
    } catch (const std::exception &x) {
        delete c->e;
        delete c;
        return MDFFGPU_ERR_CUDA;
    }
    *out = c;
    return MDFFGPU_OK;
}

int mdffgpu_destroy(mdffgpu_ctx *ctx) {
    if (!ctx) return MDFFGPU_ERR_ARG;
    delete ctx->e;
    delete ctx;
    return MDFFGPU_OK;
}

const char *mdffgpu_last_error(const mdffgpu_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int mdffgpu_set_precision(mdffgpu_ctx *ctx, int precision) {
    return guarded(ctx, [&](Engine &e) {
        if (precision != MDFFGPU_FP64 && precision != MDFFGPU_MIXED) throw Error(MDFFGPU_ERR_ARG, "bad precision");
        if (precision == MDFFGPU_MIXED && !mdffgpu::mixed_available())
            throw Error(MDFFGPU_ERR_ARG, "mixed precision kernels are not built in this library");
        e.precision = precision;
        e.use32 = (precision == MDFFGPU_MIXED);
        e.gen++;
        e.real32 = e.rec32 = e.subset32 = true;
        if (const char *v = getenv("MDFFGPU_MIXED_PARTS")) {
            e.real32 = strstr(v, "real") != nullptr;
            e.rec32 = strstr(v, "rec") != nullptr;
        }
        if (const char *v = getenv("MDFFGPU_PIM_SUBSET")) e.subset32 = atoi(v) != 0;
        // the rho and ion passes on the tensor cores (kspace_tc.cu, kspace_ion_tc.cu) from
        // TC_MIN_IONS ions on; below, where a pass is a few microseconds, the CUDA-core passes
        // (fewer kernels per pass).  MDFFGPU_RHO_TC / MDFFGPU_ION_TC = 0 / 1 override.
        e.rho_tc = e.ion_tc = e.n >= TC_MIN_IONS;
        if (const char *v = getenv("MDFFGPU_RHO_TC")) e.rho_tc = atoi(v) != 0;
        if (const char *v = getenv("MDFFGPU_ION_TC")) e.ion_tc = atoi(v) != 0;
    });
}

int mdffgpu_tune_launch(mdffgpu_ctx *ctx, int reps, int *choice, double *ms) {
    return guarded(ctx, [&](Engine &e) { e.tune_launch(reps, choice, ms); });
}

int mdffgpu_set_pim_solver(mdffgpu_ctx *ctx, int solver) {
    return guarded(ctx, [&](Engine &e) {
        if (solver != MDFFGPU_PIM_REFERENCE && solver != MDFFGPU_PIM_CG && solver != MDFFGPU_PIM_CG_FUSED)
            throw Error(MDFFGPU_ERR_ARG, "bad solver");
        e.pim_solver = solver;
        e.gen++;
        e.cg_poly = true;   // MDFFGPU_CG_PREDICT=aspc: start the CG from the ASPC predictor instead
        if (const char *v = getenv("MDFFGPU_CG_PREDICT")) e.cg_poly = strcmp(v, "aspc") != 0;
    });
}

int mdffgpu_set_graph(mdffgpu_ctx *ctx, int on) {
    return guarded(ctx, [&](Engine &e) {
        e.graph_on = on != 0;
        if (!e.graph_on) e.drop_graph();
    });
}

int mdffgpu_set_positions(mdffgpu_ctx *ctx, const double *rx, const double *ry, const double *rz) {
    if (!rx || !ry || !rz) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) { e.set_positions(rx, ry, rz); });
}

int mdffgpu_set_velocities(mdffgpu_ctx *ctx, const double *vx, const double *vy, const double *vz) {
    return guarded(ctx, [&](Engine &e) { e.set_velocities(vx, vy, vz); });
}

int mdffgpu_get_state(mdffgpu_ctx *ctx, double *rx, double *ry, double *rz, double *vx, double *vy, double *vz,
                      double *fx, double *fy, double *fz) {
    return guarded(ctx, [&](Engine &e) { e.get_state(rx, ry, rz, vx, vy, vz, fx, fy, fz); });
}

int mdffgpu_set_dipole_history(mdffgpu_ctx *ctx, const double *hist) {
    if (!hist) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        upload(e, e.d_hist, hist, sizeof(double) * 18 * (size_t)e.n);
        MDFF_CK(cudaStreamSynchronize(e.stream));
    });
}

int mdffgpu_get_dipole_history(mdffgpu_ctx *ctx, double *hist) {
    if (!hist) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        download(e, hist, e.d_hist, sizeof(double) * 18 * (size_t)e.n);
        MDFF_CK(cudaStreamSynchronize(e.stream));
    });
}

int mdffgpu_set_nhc(mdffgpu_ctx *ctx, const double *xi, const double *vxi) {
    if (!xi || !vxi) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        int k = e.p.nhc_n < 16 ? e.p.nhc_n : 16;
        upload(e, e.d_nhc, xi, sizeof(double) * k);
        upload(e, e.d_nhc + 16, vxi, sizeof(double) * k);
        MDFF_CK(cudaStreamSynchronize(e.stream));
    });
}

int mdffgpu_get_nhc(mdffgpu_ctx *ctx, double *xi, double *vxi) {
    if (!xi || !vxi) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        int k = e.p.nhc_n < 16 ? e.p.nhc_n : 16;
        download(e, xi, e.d_nhc, sizeof(double) * k);
        download(e, vxi, e.d_nhc + 16, sizeof(double) * k);
        MDFF_CK(cudaStreamSynchronize(e.stream));
    });
}

int mdffgpu_state_size(const mdffgpu_ctx *ctx, size_t *bytes) {
    if (!ctx || !ctx->e || !bytes) return MDFFGPU_ERR_ARG;
    *bytes = ctx->e->state_bytes();
    return MDFFGPU_OK;
}

int mdffgpu_save_state(mdffgpu_ctx *ctx, void *buf, size_t bytes) {
    if (!ctx || !ctx->e || !buf) return MDFFGPU_ERR_ARG;
    if (bytes < ctx->e->state_bytes()) {
        ctx->err = "save_state: buffer smaller than mdffgpu_state_size";
        return MDFFGPU_ERR_ARG;
    }
    return guarded(ctx, [&](Engine &e) { e.save_state((unsigned char *)buf); });
}

int mdffgpu_load_state(mdffgpu_ctx *ctx, const void *buf, size_t bytes, int *istep) {
    if (!buf) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        int s = e.load_state((const unsigned char *)buf, bytes);
        if (istep) *istep = s;
    });
}

int mdffgpu_get_thermo(mdffgpu_ctx *ctx, mdffgpu_thermo *t) {
    if (!t) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        e.sync_scalars();
        const mdffgpu::DevScalars &o = *e.h_out;
        t->e_kin = o.e_kin;
        t->e_nvt = o.e_nvt;
        t->u_lj = o.u_lj;
        t->u_bhmftd = o.u_bh;
        t->u_coul = o.u_coul;
        t->u_pol = o.u_pol;
        t->pvir_lj = o.pvir_lj;
        t->pvir_bhmftd = o.pvir_bh;
        t->pvir_coul = o.pvir_coul;
        memcpy(t->tau_lj, o.tau_lj, sizeof(double) * 9);
        memcpy(t->tau_bhmftd, o.tau_bh, sizeof(double) * 9);
        memcpy(t->tau_coul, o.tau_coul, sizeof(double) * 9);
        t->utail = e.utail;
        t->ptail = e.ptail;
        t->scf_rmsd = e.last_rmsd;
        t->scf_iter = e.last_scf_iter;
        t->nlist_builds = o.nbuilds;
    });
}

int mdffgpu_gen_verletlist(mdffgpu_ctx *ctx) {
    return guarded(ctx, [&](Engine &e) { e.gen_verletlist(); });
}

int mdffgpu_check_verletlist(mdffgpu_ctx *ctx, int *rebuilt) {
    return guarded(ctx, [&](Engine &e) {
        int r = e.check_verletlist();
        if (rebuilt) *rebuilt = r;
    });
}

// the reference's half list from the full lists: keep (i, j) when the parity rule
// of src/verlet.c:82-83 holds, ascending j
int mdffgpu_get_verletlist(mdffgpu_ctx *ctx, int which, int *point, int *list, int cap, int *count) {
    if (!point || (which != 0 && which != 1)) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        if (!e.list_ready) throw Error(MDFFGPU_ERR_STATE, "no Verlet list built");
        int c = which ? e.cap_co : e.cap_nb;
        std::vector<int> L((size_t)e.n * c), m(e.n);
        download(e, L.data(), which ? e.d_co : e.d_nb, sizeof(int) * L.size());
        download(e, m.data(), which ? e.d_con : e.d_nbn, sizeof(int) * e.n);
        MDFF_CK(cudaStreamSynchronize(e.stream));
        int tot = 0;
        std::vector<int> row;
        for (int i = 0; i < e.n; i++) {
            point[i] = tot;
            row.clear();
            int mi = m[i] < c ? m[i] : c;
            for (int k = 0; k < mi; k++) {
                int j = L[(size_t)i * c + k];
                if (((i > j) && ((i + j) % 2 == 0)) || ((i < j) && ((i + j) % 2 != 0))) row.push_back(j);
            }
            std::sort(row.begin(), row.end());
            for (int j : row) {
                if (list && tot < cap) list[tot] = j;
                tot++;
            }
        }
        point[e.n] = tot;
        if (count) *count = tot;
        if (list && tot > cap) throw Error(MDFFGPU_ERR_ARG, "list buffer too small");
    });
}

int mdffgpu_engforce(mdffgpu_ctx *ctx) {
    return guarded(ctx, [&](Engine &e) {
        MDFF_CK(cudaMemsetAsync(e.d_status, 0, sizeof(unsigned), e.stream));
        e.engforce();
        e.sync_scalars();
        e.check_status();
    });
}

static int sr_call(mdffgpu_ctx *ctx, bool lj, double *u, double *pvir, double *tau) {
    return guarded(ctx, [&](Engine &e) {
        if (lj && !e.p.lnmlj) throw Error(MDFFGPU_ERR_STATE, "lnmlj is not set");
        if (!lj && !(e.p.lbhmft || e.p.lbhmftd)) throw Error(MDFFGPU_ERR_STATE, "lbhmft/lbhmftd is not set");
        e.ensure_lists();
        mdffgpu::launch_kardir(e, e.d_r, e.d_s);
        e.sr_forces(lj, nullptr, nullptr, nullptr);
        e.sync_scalars();
        const mdffgpu::DevScalars &o = *e.h_out;
        if (u) *u = lj ? o.u_lj : o.u_bh;
        if (pvir) *pvir = lj ? o.pvir_lj : o.pvir_bh;
        if (tau) memcpy(tau, lj ? o.tau_lj : o.tau_bh, sizeof(double) * 9);
    });
}

int mdffgpu_engforce_nmlj(mdffgpu_ctx *ctx, double *u, double *pvir, double *tau) {
    return sr_call(ctx, true, u, pvir, tau);
}

int mdffgpu_engforce_bhmftd(mdffgpu_ctx *ctx, double *u, double *pvir, double *tau) {
    return sr_call(ctx, false, u, pvir, tau);
}

int mdffgpu_multipole_es(mdffgpu_ctx *ctx, const double *q, const double *mu, int flags, double alpha, double *u,
                         double *pvir, double *tau, double *ef, double *efg, double *f) {
    if (!q || !mu) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        if (!e.p.lcoulombic) throw Error(MDFFGPU_ERR_STATE, "lcoulombic is not set");
        size_t n = e.n;
        double *dq = nullptr, *defg = nullptr;
        double3 *dmu = nullptr, *def = nullptr, *df = nullptr;
        MDFF_CK(cudaMalloc(&dq, sizeof(double) * n));
        MDFF_CK(cudaMalloc(&dmu, sizeof(double3) * n));
        MDFF_CK(cudaMalloc(&def, sizeof(double3) * n));
        MDFF_CK(cudaMalloc(&df, sizeof(double3) * n));
        MDFF_CK(cudaMalloc(&defg, sizeof(double) * 9 * n));
        try {
            upload(e, dq, q, sizeof(double) * n);
            upload(e, dmu, mu, sizeof(double3) * n);
            MDFF_CK(cudaMemsetAsync(df, 0, sizeof(double3) * n, e.stream));
            double a = alpha > 0.0 ? alpha : e.p.alphaES;
            e.multipole_es_dev(dq, dmu, a, flags, def, efg ? defg : nullptr, df);
            e.sync_scalars();
            if (ef) download(e, ef, def, sizeof(double3) * n);
            if (efg) download(e, efg, defg, sizeof(double) * 9 * n);
            if (f) download(e, f, df, sizeof(double3) * n);
            MDFF_CK(cudaStreamSynchronize(e.stream));
            if (u) *u = e.h_out->u_coul;
            if (pvir) *pvir = e.h_out->pvir_coul;
            if (tau) memcpy(tau, e.h_out->tau_coul, sizeof(double) * 9);
        } catch (...) {
            cudaFree(dq); cudaFree(dmu); cudaFree(def); cudaFree(df); cudaFree(defg);
            throw;
        }
        cudaFree(dq); cudaFree(dmu); cudaFree(def); cudaFree(df); cudaFree(defg);
    });
}

int mdffgpu_get_dipoles(mdffgpu_ctx *ctx, double *mu, double *upol) {
    return guarded(ctx, [&](Engine &e) {
        if (!e.p.lcoulombic) throw Error(MDFFGPU_ERR_STATE, "lcoulombic is not set");
        e.ensure_lists();
        mdffgpu::launch_kardir(e, e.d_r, e.d_s);
        if (e.use32) mdffgpu::launch_coords32(e);
        e.get_dipoles();
        e.sync_scalars();
        if (mu) download(e, mu, e.d_mu_tot, sizeof(double3) * e.n);
        MDFF_CK(cudaStreamSynchronize(e.stream));
        if (upol) *upol = e.h_out->u_pol;
    });
}

int mdffgpu_prop_agate(mdffgpu_ctx *ctx, int istep) {
    return guarded(ctx, [&](Engine &e) {
        MDFF_CK(cudaMemsetAsync(e.d_status, 0, sizeof(unsigned), e.stream));
        e.prop_agate(istep);
        e.sync_scalars();
        e.check_status();
    });
}

int mdffgpu_md_steps(mdffgpu_ctx *ctx, int first, int nsteps, double *thermo) {
    if (nsteps < 0) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) { e.md_steps(first, nsteps, thermo); });
}

int mdffgpu_md_steps_host(mdffgpu_ctx *ctx, int first, int nsteps, const double *const *in, double *thermo,
                          double *const *out) {
    if (nsteps < 0) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) { e.md_steps(first, nsteps, thermo, in, out); });
}

long long mdffgpu_launch_count(const mdffgpu_ctx *ctx) { return (ctx && ctx->e) ? ctx->e->launches : -1; }

void *mdffgpu_stream(const mdffgpu_ctx *ctx) { return (ctx && ctx->e) ? (void *)ctx->e->stream : nullptr; }

int mdffgpu_profile(mdffgpu_ctx *ctx, const char *kernel) {
    return guarded(ctx, [&](Engine &e) {
        MDFF_CK(cudaStreamSynchronize(e.stream));
        e.prof_name = kernel ? kernel : "";
        e.prof_pairs.clear();
        e.prof_next = 0;
        e.prof_flops = 0.0;
    });
}

int mdffgpu_profile_result(mdffgpu_ctx *ctx, double *ms, long long *count, double *flops) {
    if (!ms || !count || !flops) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) { e.prof_result(ms, count, flops); });
}

int mdffgpu_fit_set_params(mdffgpu_ctx *ctx, int tSi, int tO, const double *theta) {
    if (!theta) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) { e.set_fit_params(tSi, tO, theta); });
}

namespace {
// target forces (AoS) onto the device, then the force-matching evaluation
void force_match_aos(Engine &e, int tSi, int tO, const double *ft_aos, double scale, double *res) {
    if (!e.d_ft) e.d_ft = mdffgpu::dalloc<double3>(e.n);
    MDFF_CK(cudaMemcpyAsync(e.d_ft, ft_aos, sizeof(double3) * e.n, cudaMemcpyHostToDevice, e.stream));
    e.force_match(e.d_ft, scale, res, tSi, tO);
}
}  // namespace

int mdffgpu_force_match(mdffgpu_ctx *ctx, int tSi, int tO, const double *fx_t, const double *fy_t,
                        const double *fz_t, double scale, double *res) {
    if (!fx_t || !fy_t || !fz_t || !res) return MDFFGPU_ERR_ARG;
    return guarded(ctx, [&](Engine &e) {
        std::vector<double> a((size_t)3 * e.n);
        for (int i = 0; i < e.n; i++) {
            a[3 * i] = fx_t[i];
            a[3 * i + 1] = fy_t[i];
            a[3 * i + 2] = fz_t[i];
        }
        force_match_aos(e, tSi, tO, a.data(), scale, res);
    });
}

int mdffgpu_fit_batch(mdffgpu_ctx **ctx, int nconf, int tSi, int tO, const double *theta,
                      const double *const *targets, double scale, int nthreads, double *res) {
    if (!ctx || nconf <= 0 || !theta || !targets || !res) return MDFFGPU_ERR_ARG;
    for (int c = 0; c < nconf; c++)
        if (!ctx[c] || !ctx[c]->e || !targets[c]) return MDFFGPU_ERR_ARG;
    int nt = std::max(1, std::min(nthreads, nconf));
    std::vector<std::vector<double>> part(nconf, std::vector<double>(1 + MDFFGPU_FIT_NPARAM, 0.0));
    std::vector<int> rc(nconf, MDFFGPU_OK);
    int device = ctx[0]->e->device;
    auto work = [&](int t) {
        cudaSetDevice(device);
        for (int c = t; c < nconf; c += nt) {
            rc[c] = guarded(ctx[c], [&](Engine &e) {
                e.set_fit_params(tSi, tO, theta);
                force_match_aos(e, tSi, tO, targets[c], scale, part[c].data());
            });
            if (rc[c] != MDFFGPU_OK) return;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    for (int k = 0; k <= MDFFGPU_FIT_NPARAM; k++) res[k] = 0.0;
    for (int c = 0; c < nconf; c++) {
        if (rc[c] != MDFFGPU_OK) return rc[c];
        for (int k = 0; k <= MDFFGPU_FIT_NPARAM; k++) res[k] += part[c][k];   // configuration order
    }
    return MDFFGPU_OK;
}

int mdffgpu_fit_plan_create(mdffgpu_ctx **ctx, int nconf, int tSi, int tO, const double *const *targets,
                            double scale, mdffgpu_fit_plan **out) {
    if (!ctx || nconf <= 0 || !targets || !out) return MDFFGPU_ERR_ARG;
    *out = nullptr;
    for (int c = 0; c < nconf; c++)
        if (!ctx[c] || !ctx[c]->e || !targets[c] || ctx[c]->e->device != ctx[0]->e->device) return MDFFGPU_ERR_ARG;
    mdffgpu_fit_plan *plan = new mdffgpu_fit_plan();
    int rc = plan_guarded(plan, [&](mdffgpu_fit_plan &P) {
        P.ctx.assign(ctx, ctx + nconf);
        P.tSi = tSi;
        P.tO = tO;
        P.scale = scale;
        P.device = ctx[0]->e->device;
        MDFF_CK(cudaSetDevice(P.device));
        MDFF_CK(cudaStreamCreateWithFlags(&P.stream, cudaStreamNonBlocking));
        MDFF_CK(cudaEventCreateWithFlags(&P.ev_theta, cudaEventDisableTiming));
        P.ev_done.assign(nconf, nullptr);
        for (int c = 0; c < nconf; c++) MDFF_CK(cudaEventCreateWithFlags(&P.ev_done[c], cudaEventDisableTiming));
        P.d_theta = mdffgpu::dalloc<double>(MDFFGPU_FIT_NPARAM);
        P.d_res = mdffgpu::dalloc<double>((size_t)nconf * mdffgpu::FIT_NRES);
        MDFF_CK(cudaMallocHost((void **)&P.h_theta, sizeof(double) * MDFFGPU_FIT_NPARAM));
        MDFF_CK(cudaMallocHost((void **)&P.h_res, sizeof(double) * nconf * mdffgpu::FIT_NRES));
        for (int c = 0; c < nconf; c++) {
            Engine &e = *ctx[c]->e;
            if (!e.d_ft) e.d_ft = mdffgpu::dalloc<double3>(e.n);
            upload(e, e.d_ft, targets[c], sizeof(double3) * e.n);
            MDFF_CK(cudaStreamSynchronize(e.stream));
        }
    });
    if (rc != MDFFGPU_OK) {
        delete plan;
        return rc;
    }
    *out = plan;
    return MDFFGPU_OK;
}

int mdffgpu_fit_plan_eval(mdffgpu_fit_plan *plan, const double *theta, double *res) {
    if (!plan || !theta || !res) return MDFFGPU_ERR_ARG;
    for (int k = 0; k < MDFFGPU_FIT_NPARAM; k++)
        if (!std::isfinite(theta[k])) return MDFFGPU_ERR_ARG;
    if (!(theta[7] > 0.0)) return MDFFGPU_ERR_ARG;   // the O polarisability is inverted
    return plan_guarded(plan, [&](mdffgpu_fit_plan &P) {
        const int nconf = (int)P.ctx.size(), NR = mdffgpu::FIT_NRES;
        MDFF_CK(cudaSetDevice(P.device));
        // record what is missing or stale before anything is in flight
        for (int c = 0; c < nconf; c++) {
            Engine &e = *P.ctx[c]->e;
            if (!e.fit_exec || e.fit_graph_gen != e.gen) {
                try {
                    e.capture_fit(P.d_theta, P.tSi, P.tO, P.scale, P.d_res + (size_t)c * NR);
                } catch (const Error &x) {
                    throw Error(x.code, "configuration " + std::to_string(c) + ": " + x.what());
                }
            }
        }
        std::memcpy(P.h_theta, theta, sizeof(double) * MDFFGPU_FIT_NPARAM);
        MDFF_CK(cudaMemcpyAsync(P.d_theta, P.h_theta, sizeof(double) * MDFFGPU_FIT_NPARAM, cudaMemcpyHostToDevice,
                                P.stream));
        MDFF_CK(cudaEventRecord(P.ev_theta, P.stream));
        for (int c = 0; c < nconf; c++) {
            Engine &e = *P.ctx[c]->e;
            MDFF_CK(cudaStreamWaitEvent(e.stream, P.ev_theta, 0));
            MDFF_CK(cudaGraphLaunch(e.fit_exec, e.stream));
            MDFF_CK(cudaEventRecord(P.ev_done[c], e.stream));
            MDFF_CK(cudaStreamWaitEvent(P.stream, P.ev_done[c], 0));
        }
        MDFF_CK(cudaMemcpyAsync(P.h_res, P.d_res, sizeof(double) * nconf * NR, cudaMemcpyDeviceToHost, P.stream));
        MDFF_CK(cudaStreamSynchronize(P.stream));
        for (int c = 0; c < nconf; c++) {
            try {
                mdffgpu::fit_status((unsigned)P.h_res[(size_t)c * NR + NR - 1]);
            } catch (const Error &x) {
                throw Error(x.code, "configuration " + std::to_string(c) + ": " + x.what());
            }
        }
        for (int k = 0; k <= MDFFGPU_FIT_NPARAM; k++) res[k] = 0.0;
        for (int c = 0; c < nconf; c++)   // configuration order
            for (int k = 0; k <= MDFFGPU_FIT_NPARAM; k++) res[k] += P.h_res[(size_t)c * NR + k];
        // the contexts' host copies of the parameters follow the device tables
        for (int c = 0; c < nconf; c++) P.ctx[c]->e->fit_host_params(P.tSi, P.tO, theta);
    });
}

int mdffgpu_fit_plan_destroy(mdffgpu_fit_plan *plan) {
    if (!plan) return MDFFGPU_ERR_ARG;
    delete plan;
    return MDFFGPU_OK;
}

const char *mdffgpu_fit_plan_last_error(const mdffgpu_fit_plan *plan) {
    return plan ? plan->err.c_str() : "null fit plan";
}

}  // extern "C"
