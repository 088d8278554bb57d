// Per-ion vector kernels: reductions, integrators (velocity Verlet, leap-frog,
// Nose-Hoover chain), induced-dipole updates (Jacobi/ASPC, CG) and the composition of
// the reference's energy/virial/stress globals.
#include "engine.cuh"

namespace mdffgpu {

// ---------------------------------------------------------------- reductions
// one block per slot; fixed-order tree over the block partials
__global__ void k_reduce_slots(const double *__restrict__ part, int stride, int first, int nparts,
                               double *__restrict__ scal) {
    grid_dep();
    int slot = first + blockIdx.x;
    const double *p = part + (size_t)slot * stride;
    double a = 0.0;
    for (int k = threadIdx.x; k < nparts; k += blockDim.x) a += p[k];
    __shared__ double sh[32];
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x < 32) {
        double b = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
        b = warp_sum(b);
        if (threadIdx.x == 0) scal[slot] = b;
    }
}

void launch_reduce_slots(Engine &e, int first_slot, int nslots, int nparts) {
    MDFF_LAUNCH(e, k_reduce_slots, nslots, 256, 0, e.d_part, e.part_stride, first_slot, nparts, e.d_scal);
}

// ---------------------------------------------------------------- small helpers
__global__ void k_fill3(int n, double3 *a, double3 v) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

__global__ void k_copy3(int n, const double3 *__restrict__ a, double3 *__restrict__ b) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// sum q^2 and |mu|^2 for the self terms (src/ewald.c:198-214)
__global__ void k_self_sums(int n, const double *__restrict__ q, const double3 *__restrict__ mu, double *part,
                            int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        if (q) v[0] = q[i] * q[i];
        if (mu) {
            double3 m = mu[i];
            v[1] = m.x * m.x + m.y * m.y + m.z * m.z;
        }
    }
    block_sum_to_part<2>(v, part, S_Q2, stride);
}

// ef = self2*mu + ef_dir (used when the reciprocal part is skipped)
__global__ void k_self_plus_dir(int n, double self2, const double3 *__restrict__ mu, const double3 *__restrict__ efd,
                                double3 *__restrict__ ef) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 m = mu ? mu[i] : make_double3(0, 0, 0);
    double3 d = efd ? efd[i] : make_double3(0, 0, 0);
    ef[i] = make_double3(self2 * m.x + d.x, self2 * m.y + d.y, self2 * m.z + d.z);
}

// f += f_dir * coul (when the reciprocal part is skipped)
__global__ void k_axpy3(int n, double a, const double3 *__restrict__ x, double3 *__restrict__ y) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 u = x[i], v = y[i];
    y[i] = make_double3(v.x + u.x * a, v.y + u.y * a, v.z + u.z * a);
}

__global__ void k_efg_self_dir(int n, double self2, const double *__restrict__ q, const double *__restrict__ efgd,
                               double *__restrict__ efg) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int p = 0; p < 3; p++)
        for (int r = 0; r < 3; r++) {
            double b = (p == r && q) ? -self2 * q[i] : 0.0;
            if (efgd) b += efgd[(size_t)i * 9 + 3 * p + r];
            efg[(size_t)i * 9 + 3 * p + r] = b;
        }
}

// ---------------------------------------------------------------- composition
// u, pvir, tau of a short-range evaluator from its slots (src/nmlj.c:351-363):
// slot 0 holds the full-list energy sum (each pair twice), slots 1..6 the full-list
// sum of r_a f_b + r_b f_a.
__global__ void k_finalize_sr(const double *__restrict__ scal, int slot, double inveOmegaPU, double *u, double *pvir,
                              double *tau) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    *u = 0.5 * scal[slot];
    double t[6];
    for (int k = 0; k < 6; k++) t[k] = 0.25 * scal[slot + 1 + k] * inveOmegaPU;
    double full[9] = {t[0], t[1], t[2], t[1], t[3], t[4], t[2], t[4], t[5]};
    double pv = 0.0;
    for (int k = 0; k < 9; k++) tau[k] = full[k];
    for (int k = 0; k < 3; k++) pv += full[4 * k] * (1.0 / 3.0);
    *pvir = pv;
}

// u_coul, tau_coul (src/ewald.c:209-307): dir (full-list sums), rec, self
struct CoulFin {
    double alpha, coul, inveOmegaPU, ttpiV;
    int do_dir, do_rec, do_stress;
};
__global__ void k_finalize_coul(const double *__restrict__ scal, CoulFin c, double *u, double *pvir, double *tau) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    const double rpi = 1.7724538509055160273;
    double alpha2 = c.alpha * c.alpha, selfa = c.alpha / rpi, selfa2 = 2.0 * selfa * alpha2 / 3.0;
    double u_self = -selfa * scal[S_Q2] + -selfa2 * scal[S_MU2];
    double u_dir = c.do_dir ? 0.5 * scal[S_DIR_U] : 0.0;
    double u_rec = c.do_rec ? scal[S_REC_U] * c.ttpiV : 0.0;
    *u = (u_dir + u_rec + u_self) * c.coul;
    if (c.do_stress) {
        double td[6], tr[6];
        for (int k = 0; k < 6; k++) {
            td[k] = 0.25 * scal[S_DIR_TAU + k] * c.inveOmegaPU;
            tr[k] = scal[S_REC_TAU + k] * c.ttpiV * c.inveOmegaPU;
        }
        int map[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
        for (int k = 0; k < 9; k++) {
            double t = 0.0;
            if (c.do_dir) t += td[map[k]] * c.coul;
            if (c.do_rec) t += tr[map[k]] * c.coul;
            tau[k] = t;
        }
    }
    double pv = 0.0;
    for (int k = 0; k < 3; k++) pv += tau[4 * k] * (1.0 / 3.0);
    *pvir = pv;
}

// ---------------------------------------------------------------- PIM
// induced_moment (src/pim.c:617-641): mu_i = sum_j pol[j][i] E_j, polarisable ions only
__device__ __forceinline__ double3 pol_times(const double *P, double3 e) {
    return make_double3(P[0] * e.x + P[3] * e.y + P[6] * e.z, P[1] * e.x + P[4] * e.y + P[7] * e.z,
                        P[2] * e.x + P[5] * e.y + P[8] * e.z);
}

__global__ void k_induced(int n, const int *__restrict__ polar, const double *__restrict__ pol,
                          const double3 *__restrict__ ef, double3 *__restrict__ mu) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !polar[i]) return;
    mu[i] = pol_times(pol + (size_t)i * 9, ef[i]);
}

// extrapolate_dipole_aspc predictor coefficients (src/pim.c:381-400) of order e, or
// (poly) those of the polynomial through the last e + 1 values, (-1)^k C(e + 1, k + 1);
// computed here once per launch, so the kernel indexes no table by a runtime order
AspcCoef aspc_coef(int e, bool poly) {
    static const double Bt[6][6] = {{1.0, 0, 0, 0, 0, 0},
                                    {2.0, -1.0, 0, 0, 0, 0},
                                    {2.5, -2.0, 0.5, 0, 0, 0},
                                    {2.8, -2.8, 1.2, -0.2, 0, 0},
                                    {3.0, -24.0 / 7.0, 27.0 / 14.0, -4.0 / 7.0, 1.0 / 14.0, 0},
                                    {22.0 / 7.0, -55.0 / 14.0, 55.0 / 21.0, -22.0 / 21.0, 5.0 / 21.0, -1.0 / 42.0}};
    static const double Pt[6][6] = {{1.0, 0, 0, 0, 0, 0},
                                    {2.0, -1.0, 0, 0, 0, 0},
                                    {3.0, -3.0, 1.0, 0, 0, 0},
                                    {4.0, -6.0, 4.0, -1.0, 0, 0},
                                    {5.0, -10.0, 10.0, -5.0, 1.0, 0},
                                    {6.0, -15.0, 20.0, -15.0, 6.0, -1.0}};
    if (e < 0 || e > 5) throw Error(MDFFGPU_ERR_ARG, "extrapolate_order must be 0..5");
    AspcCoef a;
    a.ne = e + 1;
    for (int k = 0; k < 6; k++) a.c[k] = poly ? Pt[e][k] : Bt[e][k];
    return a;
}

// the predictor mu = sum_k c_k hist_k over the last cf.ne values, then the history
// shift by `es` places
__global__ void k_aspc_predict(int n, AspcCoef cf, int es, double *__restrict__ hist, double3 *__restrict__ mu) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *h = hist + (size_t)i * ASPC_DEPTH * 3;
    double m[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 6; k++)
        if (k < cf.ne)
            for (int c = 0; c < 3; c++) m[c] += cf.c[k] * h[3 * k + c];
    for (int k = es; k > 0; k--)
        for (int c = 0; c < 3; c++) h[3 * k + c] = h[3 * (k - 1) + c];
    mu[i] = make_double3(m[0], m[1], m[2]);
}

// corrector (src/pim.c:403-420): mu = W * alpha E + (1 - W) * mu_pred
__global__ void k_aspc_correct(int n, double W, const int *__restrict__ polar, const double *__restrict__ pol,
                               const double3 *__restrict__ ef, double3 *__restrict__ mu) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 s = mu[i];
    double3 m = polar[i] ? pol_times(pol + (size_t)i * 9, ef[i]) : s;
    mu[i] = make_double3(m.x * W + (1.0 - W) * s.x, m.y * W + (1.0 - W) * s.y, m.z * W + (1.0 - W) * s.z);
}

// ef = a + b
__global__ void k_add3(int n, const double3 *__restrict__ a, const double3 *__restrict__ b, double3 *__restrict__ c) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 x = a[i], y = b[i];
    c[i] = make_double3(x.x + y.x, x.y + y.y, x.z + y.z);
}

// get_upol (src/pim.c:145-161) and get_rmsd_mu (src/pim.c:431-449) partial sums
__global__ void k_pim_sums(int n, const int *__restrict__ polar, const double *__restrict__ pol,
                           const double *__restrict__ invpol, const double3 *__restrict__ mu,
                           const double3 *__restrict__ ef, double *part, int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        double3 m3 = mu[i];
        double m[3] = {m3.x, m3.y, m3.z};
        const double *I = invpol + (size_t)i * 9;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) v[0] += m[a] * I[3 * a + b] * m[b];
        if (polar[i]) {
            double3 e3 = ef[i];
            double e[3] = {e3.x, e3.y, e3.z};
            const double *P = pol + (size_t)i * 9;
            for (int a = 0; a < 3; a++)
                if (P[4 * a] != 0.0) {
                    double d = m[a] / P[4 * a] - e[a];
                    v[1] += d * d;
                }
        }
    }
    block_sum_to_part<2>(v, part, S_UPOL, stride);
}

__global__ void k_hist_store(int n, const double3 *__restrict__ mu, double *__restrict__ hist) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 m = mu[i];
    double *h = hist + (size_t)i * ASPC_DEPTH * 3;
    h[0] = m.x;
    h[1] = m.y;
    h[2] = m.z;
}

// kO: f_ind = ef - mu * invpol_ii on polarisable ions (src/pim.c:561-567)
__global__ void k_ko_find(int n, const int *__restrict__ polar, const double *__restrict__ invpol,
                          const double3 *__restrict__ ef, const double3 *__restrict__ mu, double3 *__restrict__ find) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !polar[i]) return;
    const double *I = invpol + (size_t)i * 9;
    double3 e = ef[i], m = mu[i];
    find[i] = make_double3(e.x - m.x * I[0], e.y - m.y * I[4], e.z - m.z * I[8]);
}

// kO inner loop updates (src/pim.c:684-729)
__global__ void k_scale_add3(int n, double a, const double3 *__restrict__ x, double b, double3 *__restrict__ y) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 u = x[i], v = y[i];
    y[i] = make_double3(a * u.x + b * v.x, a * u.y + b * v.y, a * u.z + b * v.z);
}

// ---- CG on (alpha^-1 - T) mu = E_stat over the polarisable ions (diagonal-alpha preconditioner)
// r = ef_stat + T x - alpha^-1 x   with  T x  = field of x (incl. self term)
__global__ void k_cg_residual(int n, const int *__restrict__ polar, const double *__restrict__ invpol,
                              const double3 *__restrict__ efs, const double3 *__restrict__ tx,
                              const double3 *__restrict__ x, double3 *__restrict__ r) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!polar[i]) {
        r[i] = make_double3(0, 0, 0);
        return;
    }
    double3 e = efs[i], t = tx[i], m = x[i];
    const double *I = invpol + (size_t)i * 9;
    double3 ax = make_double3(I[0] * m.x + I[1] * m.y + I[2] * m.z, I[3] * m.x + I[4] * m.y + I[5] * m.z,
                              I[6] * m.x + I[7] * m.y + I[8] * m.z);
    r[i] = make_double3(e.x + t.x - ax.x, e.y + t.y - ax.y, e.z + t.z - ax.z);
}

// Ap = alpha^-1 p - T p ; partial sums of p.Ap
__global__ void k_cg_ap(int n, const int *__restrict__ polar, const double *__restrict__ invpol,
                        const double3 *__restrict__ p, const double3 *__restrict__ tp, double3 *__restrict__ ap,
                        double *part, int stride, double *scal, unsigned *ticket) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        if (polar[i]) {
            double3 m = p[i], t = tp[i];
            const double *I = invpol + (size_t)i * 9;
            double3 a = make_double3(I[0] * m.x + I[1] * m.y + I[2] * m.z - t.x,
                                     I[3] * m.x + I[4] * m.y + I[5] * m.z - t.y,
                                     I[6] * m.x + I[7] * m.y + I[8] * m.z - t.z);
            ap[i] = a;
            v[0] = m.x * a.x + m.y * a.y + m.z * a.z;
        } else {
            ap[i] = make_double3(0, 0, 0);
        }
    }
    block_sum_to_part<1>(v, part, S_PAP, stride);
    last_block_slots(part, stride, S_PAP, 1, scal, ticket);
}

// z = alpha r ; partial sums of r.z and r.r
__global__ void k_cg_rz(int n, const int *__restrict__ polar, const double *__restrict__ pol,
                        const double3 *__restrict__ r, double3 *__restrict__ z, double *part, int stride,
                        double *scal, unsigned *ticket) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < n) {
        if (polar[i]) {
            double3 rr = r[i];
            double3 zz = pol_times(pol + (size_t)i * 9, rr);  // pol symmetric in practice
            z[i] = zz;
            v[0] = rr.x * zz.x + rr.y * zz.y + rr.z * zz.z;
            v[1] = rr.x * rr.x + rr.y * rr.y + rr.z * rr.z;
        } else {
            z[i] = make_double3(0, 0, 0);
        }
    }
    block_sum_to_part<2>(v, part, S_RZ, stride);  // r.z, r.r
    last_block_slots(part, stride, S_RZ, 2, scal, ticket);
}

// the loop test of CgTest (first: before the first iteration, iteration count 0)
__device__ void cg_test(const CgTest &t, const double *scal, int first) {
    const double rr = scal[S_RR];
    unsigned go = 0;
    if (t.mode == 1) {
        const double rmsd = sqrt(rr / (double)(t.npol > 1 ? t.npol : 1));
        const int it = first ? 0 : t.out->scf_iter + 1;
        t.out->scf_iter = it;
        t.out->scf_rmsd = rmsd;
        if (!isfinite(rmsd)) atomicOr(t.status, (unsigned)ST_NONFINITE);
        else if (rmsd > t.tol) {
            if (it < t.maxit) go = 1;
            else atomicOr(t.status, (unsigned)ST_SCF);
        }
    } else {
        if (first) {
            *t.rr0 = rr;
            *t.itc = 0.0;
        } else {
            *t.itc += 1.0;
        }
        const int it = (int)*t.itc;
        if (!isfinite(rr)) atomicOr(t.status, (unsigned)ST_NONFINITE);
        else if (rr > t.rtol2 * *t.rr0 && rr > 0.0) {
            if (it < t.maxit) go = 1;
            else atomicOr(t.status, (unsigned)ST_SCF);
        }
    }
    cudaGraphSetConditional(t.h, go);
}

// the test of a recorded loop before its first iteration
__global__ void k_cg_test(CgTest t, const double *scal) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    *t.guard = 0u;
    cg_test(t, scal, 1);
}

// One CG update in a single launch: x += a p, r -= a Ap (a = rz / pAp, rz kept as rz_old),
// z = alpha r and the partial sums of r.z and r.r (as k_cg_rz), and in
// blocks past the ions (when acc is set) the rho(k) of the iterate, acc += a rho(p) (rho
// is linear in the dipoles).  Those blocks add zero partials; the last block reduces the
// slots as k_cg_rz does, so the scalars are the same bits.
__global__ void k_cg_step(int n, int nk, const int *__restrict__ polar, const double *__restrict__ pol,
                          double *scal, const double3 *__restrict__ p, const double3 *__restrict__ ap,
                          double3 *__restrict__ x, double3 *__restrict__ r, double3 *__restrict__ z,
                          const double2 *__restrict__ rho_p, double2 *__restrict__ acc, double *part, int stride,
                          unsigned *ticket, CgTest test) {
    grid_dep();
    const double rz = scal[S_RZ];
    const double a = rz / scal[S_PAP];
    const int nbi = (n + blockDim.x - 1) / blockDim.x;
    double v[2] = {0.0, 0.0};
    if ((int)blockIdx.x < nbi) {
        int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i == 0) scal[S_RZOLD] = rz;
        if (i < n) {
            double3 pp = p[i], q = ap[i], xx = x[i], rr = r[i];
            x[i] = make_double3(xx.x + a * pp.x, xx.y + a * pp.y, xx.z + a * pp.z);
            rr = make_double3(rr.x - a * q.x, rr.y - a * q.y, rr.z - a * q.z);
            r[i] = rr;
            if (polar[i]) {
                double3 zz = pol_times(pol + (size_t)i * 9, rr);
                z[i] = zz;
                v[0] = rr.x * zz.x + rr.y * zz.y + rr.z * zz.z;
                v[1] = rr.x * rr.x + rr.y * rr.y + rr.z * rr.z;
            } else {
                z[i] = make_double3(0, 0, 0);
            }
        }
    } else {
        int k = (blockIdx.x - nbi) * blockDim.x + threadIdx.x;
        if (k < nk) {
            double2 w = rho_p[k], s = acc[k];
            acc[k] = make_double2(s.x + a * w.x, s.y + a * w.y);
        }
    }
    block_sum_to_part<2>(v, part, S_RZ, stride);  // r.z, r.r
    const bool last = last_block_slots(part, stride, S_RZ, 2, scal, ticket);
    if (last && threadIdx.x == 0 && test.mode) cg_test(test, scal, 0);
}

// p = z + beta p, beta = rz_new / rz_old; in a recorded loop (t.mode set) also the
// backstop of the loop: past maxit iterations it ends the loop and raises ST_SCF
__global__ void k_cg_dir(int n, const double *__restrict__ scal, const double3 *__restrict__ z,
                         double3 *__restrict__ p, CgTest t) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && t.mode && ++*t.guard > (unsigned)t.maxit) {
        atomicOr(t.status, (unsigned)ST_SCF);
        cudaGraphSetConditional(t.h, 0);
    }
    if (i >= n) return;
    double beta = scal[S_RZ] / scal[S_RZOLD];
    double3 zz = z[i], pp = p[i];
    p[i] = make_double3(zz.x + beta * pp.x, zz.y + beta * pp.y, zz.z + beta * pp.z);
}

// u_pol = 1/2 sum mu.alpha^-1.mu in energy units
__global__ void k_upol_final(const double *scal, double coul, DevScalars *out) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    out->u_pol = 0.5 * scal[S_UPOL] * coul;
}

// ---------------------------------------------------------------- integrators
// prop_velocity_verlet first half (src/integration.c:33-38)
__global__ void k_vv1(int n, double dt, double dtsq2, const double *__restrict__ invm, double4 *__restrict__ r,
                      const double3 *__restrict__ v, const double3 *__restrict__ f, double3 *__restrict__ fs) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 x = r[i];
    double3 vv = v[i], ff = f[i];
    double im = invm[i];
    fs[i] = ff;
    x.x += vv.x * dt + (ff.x * dtsq2) * im;
    x.y += vv.y * dt + (ff.y * dtsq2) * im;
    x.z += vv.z * dt + (ff.z * dtsq2) * im;
    r[i] = x;
}

// prop_velocity_verlet second half (src/integration.c:47-57) + kinetic partials
__global__ void k_vv2(int n, double dt2, const double *__restrict__ invm, const double *__restrict__ mass,
                      double3 *__restrict__ v, const double3 *__restrict__ f, const double3 *__restrict__ fs,
                      double *part, int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double k[1] = {0.0};
    if (i < n) {
        double3 vv = v[i], ff = f[i], f0 = fs[i];
        double im = invm[i];
        vv.x += (f0.x + ff.x) * dt2 * im;
        vv.y += (f0.y + ff.y) * dt2 * im;
        vv.z += (f0.z + ff.z) * dt2 * im;
        v[i] = vv;
        k[0] = (vv.x * vv.x + vv.y * vv.y + vv.z * vv.z) * mass[i];
    }
    block_sum_to_part<1>(k, part, S_KIN, stride);
}

// prop_pos_vel_verlet (src/integration.c:66-90): half kick + drift ...
__global__ void k_pv1(int n, double dt, double dt2, const double *__restrict__ invm, double4 *__restrict__ r,
                      double3 *__restrict__ v, const double3 *__restrict__ f) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 x = r[i];
    double3 vv = v[i], ff = f[i];
    double im = invm[i];
    vv.x += ff.x * dt2 * im;
    vv.y += ff.y * dt2 * im;
    vv.z += ff.z * dt2 * im;
    x.x += vv.x * dt;
    x.y += vv.y * dt;
    x.z += vv.z * dt;
    v[i] = vv;
    r[i] = x;
}

// ... and the second half kick + kinetic partials
// second half kick of prop_velocity_verlet within nhcn (src/integration.c:165-167), the
// kinetic sum reduced by the last block into scal[S_KIN]; with r: the finiteness check of
// positions and forces (ST_NONFINITE) in the same pass
__global__ void __launch_bounds__(256) k_pv2(int n, double dt2, const double *__restrict__ invm,
                                             const double *__restrict__ mass, double3 *__restrict__ v,
                                             const double3 *__restrict__ f, double *part, int stride,
                                             double *scal, unsigned *ticket, const double4 *__restrict__ r,
                                             unsigned *status) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double k[1] = {0.0};
    if (i < n) {
        double3 vv = v[i], ff = f[i];
        double im = invm[i];
        if (r) {
            double4 x = r[i];
            if (!isfinite(x.x + x.y + x.z + ff.x + ff.y + ff.z)) atomicOr(status, ST_NONFINITE);
        }
        vv.x += ff.x * dt2 * im;
        vv.y += ff.y * dt2 * im;
        vv.z += ff.z * dt2 * im;
        v[i] = vv;
        k[0] = (vv.x * vv.x + vv.y * vv.y + vv.z * vv.z) * mass[i];
    }
    block_sum_to_part<1>(k, part, S_KIN, stride);
    last_block_slots(part, stride, S_KIN, 1, scal, ticket);
}

// kinetic partials, optionally after scaling v by the NHC factor s (src/integration.c:281-287)
// e_kin and the NHC conserved-quantity term e_nvt (src/integration.c:156-176) from the
// kinetic sum in scal[S_KIN]; one thread
__device__ void nhc_energy(int nn, double L, double temp, const double *__restrict__ nhc,
                           const double *__restrict__ scal, DevScalars *out) {
    const double *xi = nhc, *vxi = nhc + 16, *Q = nhc + 32;
    out->e_kin = 0.5 * scal[S_KIN];
    double nvt1 = L * temp * xi[0], nvt2 = vxi[0] * vxi[0] * 0.5 / Q[0], nvt3 = 0.0, nvt4 = 0.0;
    for (int i = 1; i < nn; i++) {
        nvt3 += vxi[i] * vxi[i] * 0.5 / Q[i];
        nvt4 += temp * xi[i];
    }
    out->e_nvt = nvt1 + nvt2 + nvt3 + nvt4;
    for (int i = 0; i < 16; i++) {
        out->xi[i] = xi[i];
        out->vxi[i] = vxi[i];
    }
}

// v *= s (scale) and the kinetic sum sum m v^2: block partials in the S_KIN slot, which
// the last block reduces into scal[S_KIN] as k_reduce_slots does (256-thread blocks);
// energy: then e_kin and e_nvt (nhc_energy)
__global__ void __launch_bounds__(256) k_scale_kin(ScaleKinArgs a) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double k[1] = {0.0};
    if (i < a.n) {
        double3 vv = a.v[i];
        if (a.scale) {
            double s = a.out_s->nhc_s;
            vv.x *= s;
            vv.y *= s;
            vv.z *= s;
            a.v[i] = vv;
        }
        k[0] = (vv.x * vv.x + vv.y * vv.y + vv.z * vv.z) * a.mass[i];
    }
    block_sum_to_part<1>(k, a.part, S_KIN, a.stride);
    const bool last = last_block_slots(a.part, a.stride, S_KIN, 1, a.scal, a.ticket);
    if (last && a.energy && threadIdx.x == 0) nhc_energy(a.nn, a.L, a.temp, a.nhc, a.scal, a.out);
}

// leap-frog (src/integration.c:93-137)
__global__ void k_lf(int n, double dtsq, double idt, const double *__restrict__ invm, const double *__restrict__ mass,
                     double4 *__restrict__ r, double3 *__restrict__ rs, double3 *__restrict__ v,
                     const double3 *__restrict__ f, double *part, int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double k[1] = {0.0};
    if (i < n) {
        double4 x = r[i];
        double3 o = rs[i], ff = f[i];
        double im = invm[i];
        double ux = 2.0 * x.x - o.x + ff.x * dtsq * im;
        double uy = 2.0 * x.y - o.y + ff.y * dtsq * im;
        double uz = 2.0 * x.z - o.z + ff.z * dtsq * im;
        double3 vv = make_double3(idt * (ux - o.x), idt * (uy - o.y), idt * (uz - o.z));
        v[i] = vv;
        k[0] = (vv.x * vv.x + vv.y * vv.y + vv.z * vv.z) * mass[i];
        rs[i] = make_double3(x.x, x.y, x.z);
        r[i] = make_double4(ux, uy, uz, x.w);
    }
    block_sum_to_part<1>(k, part, S_KIN, stride);
}

// chain_nhcn (src/integration.c:189-294) on one thread: thermostat variables in
// d_nhc (xi[16], vxi[16]); kin from the S_KIN slot (sum m v^2); writes s.  The
// second sweep stops at nhc_n-2 as in the reference (src/integration.c:269).  NN > 0:
// the chain length known at compile time, the chain held in registers (the loops
// unrolled); NN = 0: any length up to 16, the chain in local memory.  Either way the
// variables are read once and written once, and the arithmetic is the same.
struct NhcArgs {
    int nn, yo, mults;
    double dt, temp, L, w[7];
};
template <int NN>
__global__ void k_nhc_chain(NhcArgs a, double *__restrict__ nhc, const double *__restrict__ scal, DevScalars *out) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    constexpr int M = NN > 0 ? NN : 16;
    const int nn = NN > 0 ? NN : a.nn;
    double xi[M], vxi[M], Q[M], G[M];
#pragma unroll
    for (int i = 0; i < M; i++) {
        const bool on = i < nn;
        xi[i] = on ? nhc[i] : 0.0;
        vxi[i] = on ? nhc[16 + i] : 0.0;
        Q[i] = on ? nhc[32 + i] : 1.0;
        G[i] = 0.0;
    }
    const double kin = 0.5 * scal[S_KIN];
    double s = 1.0;
    G[0] = 2.0 * kin - a.L * a.temp;
    for (int k = 0; k < a.mults; k++) {
        for (int j = 0; j < a.yo && j < 7; j++) {
            const double dts = a.w[j] * a.dt / ((double)a.mults);
            const double dts2 = dts * 0.5, dts4 = dts2 * 0.5, dts8 = dts4 * 0.5;
            G[nn - 1] = (vxi[nn - 2] * vxi[nn - 2] / Q[nn - 2] - a.temp);
            vxi[nn - 1] += G[nn - 1] * dts4;
#pragma unroll
            for (int inh = M - 2; inh > -1; inh--) {
                if (inh > nn - 2) continue;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] += G[inh] * dts4;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
            }
            s *= exp(-vxi[0] * dts2 / Q[0]);
#pragma unroll
            for (int i = 0; i < M; i++)
                if (i < nn) xi[i] += vxi[i] * dts2 / Q[i];
            G[0] = 2.0 * kin * s * s - a.L * a.temp;
#pragma unroll
            for (int inh = 0; inh < M - 2; inh++) {
                if (inh >= nn - 2) break;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                vxi[inh] += G[inh] * dts4;
                vxi[inh] *= exp(-vxi[inh + 1] * dts8 / Q[inh + 1]);
                G[inh + 1] = (vxi[inh] * vxi[inh] / Q[inh] - a.temp);
            }
            vxi[nn - 1] += G[nn - 1] * dts4;
        }
    }
#pragma unroll
    for (int i = 0; i < M; i++)
        if (i < nn) {
            nhc[i] = xi[i];
            nhc[16 + i] = vxi[i];
        }
    out->nhc_s = s;
}

void launch_nhc_chain(Engine &e, const NhcArgs &a, double *nhc, const double *scal, DevScalars *out) {
    switch (a.nn) {
    case 2: MDFF_LAUNCH(e, k_nhc_chain<2>, 1, 1, 0, a, nhc, scal, out); break;
    case 3: MDFF_LAUNCH(e, k_nhc_chain<3>, 1, 1, 0, a, nhc, scal, out); break;
    case 4: MDFF_LAUNCH(e, k_nhc_chain<4>, 1, 1, 0, a, nhc, scal, out); break;
    case 5: MDFF_LAUNCH(e, k_nhc_chain<5>, 1, 1, 0, a, nhc, scal, out); break;
    default: MDFF_LAUNCH(e, k_nhc_chain<0>, 1, 1, 0, a, nhc, scal, out); break;
    }
}

__global__ void k_set_ekin(const double *__restrict__ scal, DevScalars *out) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    out->e_kin = 0.5 * scal[S_KIN];
}

// non-finite guard on positions and forces (status word)
__global__ void k_check_finite(int n, const double4 *__restrict__ r, const double3 *__restrict__ f, unsigned *status) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 x = r[i];
    double3 g = f[i];
    if (!isfinite(x.x + x.y + x.z + g.x + g.y + g.z)) atomicOr(status, ST_NONFINITE);
}

}  // namespace mdffgpu
