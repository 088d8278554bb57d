// Force matching: loss L = scale/2 sum_i |F_i - F_i^target|^2 style sums and its exact
// gradient with respect to the force-field parameters of the polarisable silica model
// (Born-Mayer A, B and dispersion C for Si-O and O-O, q_Si with q_O = -q_Si/2, the O
// polarisability, the Tang-Toennies damping b and c of the charge-dipole terms).
//
// The forces F(theta, mu*) are taken at the converged induced dipoles mu*, which solve
// R(mu, theta) = alpha^-1 mu - E(mu, theta) = 0.  With w = dL/dF,
//     dL/dtheta = w . dF/dtheta|_mu  -  lambda . dR/dtheta|_mu,   A lambda = s,
//     s_j = d(w.F)/dmu_j,  A = alpha^-1 - T  (the PIM operator, symmetric),
// i.e. ONE extra linear solve with the induced-dipole operator instead of
// differentiating through the CG iterations.  The pieces:
//   s (real space)  : k_adj_dir, d/dmu_i of the pair forces contracted with w_i - w_j,
//                     recomputed from the geometry (nothing stored per pair);
//   s (k space)     : EFG_rec(q, mu) . w_i plus the field of the w-derivative of rho,
//                     drho_w(k) = i sum_a k_a rho(q w_a, mu w_a)  (three rho passes);
//   BHM parameters  : k_bhm_sens, d(pair force)/d(A, B, C) contracted with w_i - w_j;
//   q_Si            : the Coulomb force is bilinear in (q, mu): w.dF/dq_Si =
//                     (2 w.F(q,0) + w.(F(q,mu) - F(q,0) - F(0,mu))) / q_Si, and
//                     dR/dq_Si = -E(q, 0) / q_Si;
//   alpha_O         : dR/dalpha = -mu / alpha^2 on O;
//   b, c            : k_damp_sens, derivatives of the damped charge-dipole force and of
//                     the damped charge field (E_stat) through the TT function.
#include "engine.cuh"

namespace mdffgpu {

constexpr int FIT_WARPS = 8;

// partial-sum slots of the fit (e.d_fpart / e.d_fscal)
enum FitSlot : int {
    F_LOSS = 0,
    F_BHM = 1,          // 8: A B C (Si-O), A B C (O-O), D (Si-O), D (O-O)
    F_DAMP = 9,         // 4: w.dF/db, w.dF/dc, lambda.dE/db, lambda.dE/dc
    F_WFALL = 13, F_WFQ0 = 14, F_WF0M = 15,   // w.F_coul(q,mu), w.F_coul(q,0), w.F_coul(0,mu)
    F_LESTAT = 16,      // lambda . E(q, 0)
    F_LMU = 17,         // lambda . mu_ind on the polarisable ions
    F_ADJ_RR0 = 18, F_ADJ_IT = 19,   // adjoint CG: initial r.r and iteration count (recorded loop)
    NFSLOT = 20
};
constexpr int NRES = FIT_NRES;

__global__ void k_reduce_slots(const double *part, int stride, int first, int nparts, double *scal);
// preconditioned CG kernels of integrate.cu
__global__ void k_cg_ap(int n, const int *polar, const double *invpol, const double3 *p, const double3 *tp,
                        double3 *ap, double *part, int stride, double *scal, unsigned *ticket);
__global__ void k_cg_rz(int n, const int *polar, const double *pol, const double3 *r, double3 *z, double *part,
                        int stride, double *scal, unsigned *ticket);
__global__ void k_cg_step(int n, int nk, const int *polar, const double *pol, double *scal, const double3 *p,
                          const double3 *ap, double3 *x, double3 *r, double3 *z, const double2 *rho_p, double2 *acc,
                          double *part, int stride, unsigned *ticket, CgTest test);
__global__ void k_cg_test(CgTest t, const double *scal);
__global__ void k_cg_dir(int n, const double *scal, const double3 *z, double3 *p, CgTest t);

struct TTd {
    double E[9];   // 1/k!
};

template <int NV>
__device__ __forceinline__ void fit_block_sum(double (&v)[NV], double *part, int slot, int stride) {
    __shared__ double sh[32][NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < NV; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) a += sh[q][threadIdx.x];
        part[(size_t)(slot + threadIdx.x) * stride + blockIdx.x] = a;
    }
}

// w = scale (F - F_t); partial sums of |F - F_t|^2
__global__ void k_fm_seed(int n, const double3 *__restrict__ f, const double3 *__restrict__ ft, double scale,
                          double3 *__restrict__ w, double *part, int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < n) {
        double3 a = f[i], b = ft[i];
        double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        w[i] = make_double3(scale * dx, scale * dy, scale * dz);
        v[0] = dx * dx + dy * dy + dz * dz;
    }
    fit_block_sum<1>(v, part, F_LOSS, stride);
}

// partial sums of a.b over the ions (mask: only polarisable ions when non-null)
__global__ void k_dot3(int n, const double3 *__restrict__ a, const double3 *__restrict__ b,
                       const int *__restrict__ mask, double *part, int slot, int stride) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v[1] = {0.0};
    if (i < n && (!mask || mask[i])) {
        double3 x = a[i], y = b[i];
        v[0] = x.x * y.x + x.y * y.y + x.z * y.z;
    }
    fit_block_sum<1>(v, part, slot, stride);
}

// s = coul (s_dir + E_rec(drho_w) + EFG_rec . w) on polarisable ions (EFG_rec: upper
// triangle as the k-space combine writes it), zero elsewhere
__global__ void k_adj_rhs(int n, const int *__restrict__ polar, double coul, const double3 *__restrict__ sdir,
                          const double3 *__restrict__ erw, const double *__restrict__ efg,
                          const double3 *__restrict__ w, double3 *__restrict__ s) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!polar[i]) {
        s[i] = make_double3(0, 0, 0);
        return;
    }
    const double *G = efg + (size_t)i * 9;
    double g[3][3];
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) g[p][q] = (q >= p) ? G[3 * p + q] : G[3 * q + p];
    double3 ww = w[i], a = sdir[i], e = erw[i];
    double gw[3];
    for (int p = 0; p < 3; p++) gw[p] = g[p][0] * ww.x + g[p][1] * ww.y + g[p][2] * ww.z;
    s[i] = make_double3(coul * (a.x + e.x + gw[0]), coul * (a.y + e.y + gw[1]), coul * (a.z + e.z + gw[2]));
}

// drho_w(k) = i (kx rho_x + ky rho_y + kz rho_z)
__global__ void k_drho_w(int nk, const double3 *__restrict__ kv, const double2 *__restrict__ rx,
                         const double2 *__restrict__ ry, const double2 *__restrict__ rz, double2 *__restrict__ out) {
    grid_dep();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    double3 kk = kv[k];
    double2 a = rx[k], b = ry[k], c = rz[k];
    double re = kk.x * a.x + kk.y * b.x + kk.z * c.x, im = kk.x * a.y + kk.y * b.y + kk.z * c.y;
    out[k] = make_double2(-im, re);
}

// q w_a and mu w_a (a = 0, 1, 2): charges and dipoles of the rho passes of drho_w
__global__ void k_scale_by_w(int n, int comp, const double *__restrict__ q, const double3 *__restrict__ mu,
                             const double3 *__restrict__ w, double *__restrict__ qo, double3 *__restrict__ muo) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 ww = w[i];
    double a = comp == 0 ? ww.x : (comp == 1 ? ww.y : ww.z);
    double3 m = mu[i];
    qo[i] = a * q[i];
    muo[i] = make_double3(a * m.x, a * m.y, a * m.z);
}

struct AdjArgs {
    int n, nt, cap;
    Cell c;
    const double4 *s;
    const double *q;
    const double3 *mu;
    const int *typ, *polar;
    const PairDamp *damp;
    const int *col, *con;
    double lrcutsq, alpha;
    int ldamp;
    TTd tt;
    const double3 *w;
    const double3 *lambda;
    double3 *sdir;
    double *part;
    int stride;
};

// TT f_k(b r) (src/tt_damp.c:16-32), its r-derivative fd and the derivatives of f and fd
// with respect to b and c
__device__ __forceinline__ void tt_param(const TTd &tt, double b, double c, double r, int k, double &f, double &fd,
                                         double &df_db, double &df_dc, double &dfd_db, double &dfd_dc) {
    double x = b * r, ex = exp(-x);
    double s = tt.E[k];
    for (int m = k - 1; m > -1; m--) s = s * x + tt.E[m];
    double xk = tt.E[k];
    for (int m = 0; m < k; m++) xk *= x;   // x^k / k!
    f = 1.0 - c * ex * s;
    fd = c * b * ex * xk;
    df_dc = -ex * s;
    df_db = r * c * ex * xk;
    dfd_dc = b * ex * xk;
    dfd_db = c * ex * xk * (1.0 + (double)k - x);
}

// s_i (real space, electrostatic units) = - sum_j d/dmu_i [(w_i - w_j) . fij] at
// polarisable i, fij the pair term of k_dir (force on i = -fij)
__global__ void __launch_bounds__(FIT_WARPS * 32) k_adj_dir(AdjArgs a) {
    grid_dep();
    int i = blockIdx.x * FIT_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    double si3[3] = {0, 0, 0};
    const double alpha = a.alpha, alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha5 = alpha3 * alpha2;
    const double rpi = 1.7724538509055160273;
    if (i < a.n && a.polar[i]) {
        double4 si = a.s[i];
        double3 wi = a.w[i];
        int ti = a.typ[i];
        int m = min(a.con[i], a.cap);
        const int *L = a.col + (size_t)i * a.cap;
        for (int k = lane; k < m; k += 32) {
            int j = L[k];
            double4 sj = a.s[j];
            double3 r = pbc_frac(a.c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double d2 = norm2_exact(r);
            if (d2 > a.lrcutsq) continue;
            double qj = a.q[j];
            double3 mj = a.mu[j];
            bool dip_j = (mj.x != 0.0) || (mj.y != 0.0) || (mj.z != 0.0);
            double3 wj = a.w[j];
            double v[3] = {wi.x - wj.x, wi.y - wj.y, wi.z - wj.z};
            double rr[3] = {r.x, r.y, r.z}, mv[3] = {mj.x, mj.y, mj.z};
            double d = sqrt(d2), d3 = d2 * d, d5 = d3 * d2;
            double dm1 = 1.0 / d, dm3 = dm1 / d2, dm5 = dm3 / d2, dm7 = dm5 / d2;
            double expon = exp(-alpha2 * d2) / rpi;
            double F0 = erfc(alpha * d);
            double F1 = F0 + 2.0 * alpha * d * expon;
            double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
            double F3 = F2 + 8.0 * alpha5 * d5 * expon / 15.0;
            double F2_dm5 = 3.0 * F2 * dm5, F3_dm7 = F3 * dm7 * 15.0;
            double vr = v[0] * rr[0] + v[1] * rr[1] + v[2] * rr[2];
            double t[3] = {0, 0, 0};
            if (dip_j) {   // dipole-dipole
                double rmj = rr[0] * mv[0] + rr[1] * mv[1] + rr[2] * mv[2];
                double vm = v[0] * mv[0] + v[1] * mv[1] + v[2] * mv[2];
                for (int p = 0; p < 3; p++)
                    t[p] += -F3_dm7 * rmj * vr * rr[p] + F2_dm5 * (vr * mv[p] + rmj * v[p] + vm * rr[p]);
            }
            // charge-dipole, with the damped part of the field at i from charge j
            double F1d1 = 0.0, F2d1 = 0.0;
            if (a.ldamp) {
                const PairDamp &D = a.damp[ti * a.nt + a.typ[j]];
                if (D.ldamp) {
                    double f, fd, x1, x2, x3, x4;
                    tt_param(a.tt, D.b1, D.c1, d, D.k1, f, fd, x1, x2, x3, x4);
                    F1d1 = 1.0 - f;
                    F2d1 = F1d1 + (d / 3.0) * fd;
                }
            }
            double g1 = (F1 - F1d1) * dm3, g2 = 3.0 * (F2 - F2d1) * dm5;
            for (int p = 0; p < 3; p++) t[p] += qj * (g1 * v[p] - g2 * vr * rr[p]);
            si3[0] += t[0];
            si3[1] += t[1];
            si3[2] += t[2];
        }
    }
    for (int p = 0; p < 3; p++) si3[p] = warp_sum(si3[p]);
    if (i < a.n && lane == 0) a.sdir[i] = make_double3(si3[0], si3[1], si3[2]);
}

// damping-parameter sensitivities over the Coulomb list (full list: halves for the
// force terms), per block: w.dF/db, w.dF/dc (electrostatic units), lambda.dE_stat/db,
// lambda.dE_stat/dc; the fit's b and c are those of every damped direction
__global__ void __launch_bounds__(FIT_WARPS * 32) k_damp_sens(AdjArgs a) {
    grid_dep();
    int i = blockIdx.x * FIT_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    double acc[4] = {0, 0, 0, 0};
    if (i < a.n) {
        double4 si = a.s[i];
        double3 wi = a.w[i], li = a.lambda[i];
        double qi = a.q[i];
        double3 mi = a.mu[i];
        bool dip_i = (mi.x != 0.0) || (mi.y != 0.0) || (mi.z != 0.0);
        int ti = a.typ[i];
        int m = min(a.con[i], a.cap);
        const int *L = a.col + (size_t)i * a.cap;
        for (int k = lane; k < m; k += 32) {
            int j = L[k];
            const PairDamp &D = a.damp[ti * a.nt + a.typ[j]];
            if (!D.ldamp) continue;
            double4 sj = a.s[j];
            double3 r = pbc_frac(a.c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double d2 = norm2_exact(r);
            if (d2 > a.lrcutsq) continue;
            double qj = a.q[j];
            double3 mj = a.mu[j];
            bool dip_j = (mj.x != 0.0) || (mj.y != 0.0) || (mj.z != 0.0);
            double d = sqrt(d2), dm3 = 1.0 / (d2 * d), dm5 = dm3 / d2;
            // derivatives of F1d = 1 - f and F2d = F1d + d/3 fd for both directions
            double dF1[2][2] = {{0, 0}, {0, 0}}, dF2[2][2] = {{0, 0}, {0, 0}};   // [dir][b or c]
            for (int dir = 0; dir < 2; dir++) {
                if (!(D.pad & (1 << dir))) continue;   // this direction is not a fitted damping
                double b = dir ? D.b2 : D.b1, c = dir ? D.c2 : D.c1;
                int kk = dir ? D.k2 : D.k1;
                double f, fd, dfb, dfc, dfdb, dfdc;
                tt_param(a.tt, b, c, d, kk, f, fd, dfb, dfc, dfdb, dfdc);
                dF1[dir][0] = -dfb;
                dF1[dir][1] = -dfc;
                dF2[dir][0] = -dfb + (d / 3.0) * dfdb;
                dF2[dir][1] = -dfc + (d / 3.0) * dfdc;
            }
            double3 wj = a.w[j];
            double v[3] = {wi.x - wj.x, wi.y - wj.y, wi.z - wj.z};
            double rr[3] = {r.x, r.y, r.z};
            double vr = v[0] * rr[0] + v[1] * rr[1] + v[2] * rr[2];
            double rmi = rr[0] * mi.x + rr[1] * mi.y + rr[2] * mi.z;
            double rmj = rr[0] * mj.x + rr[1] * mj.y + rr[2] * mj.z;
            double vmi = v[0] * mi.x + v[1] * mi.y + v[2] * mi.z;
            double vmj = v[0] * mj.x + v[1] * mj.y + v[2] * mj.z;
            double lr = li.x * rr[0] + li.y * rr[1] + li.z * rr[2];
            for (int pth = 0; pth < 2; pth++) {
                // force: F_ij = -fij, fij_d = -qj (a1 rmi r - b1 mi) + qi (a2 rmj r - b2 mj)
                if (dip_i || dip_j) {
                    double da1 = 3.0 * dF2[0][pth] * dm5, db1 = dF1[0][pth] * dm3;
                    double da2 = 3.0 * dF2[1][pth] * dm5, db2 = dF1[1][pth] * dm3;
                    double vf = -qj * (da1 * rmi * vr - db1 * vmi) + qi * (da2 * rmj * vr - db2 * vmj);
                    acc[pth] += -0.5 * vf;
                }
                // field at i from charge j: cfe = qj dm3 (F1 - F1d1) r
                acc[2 + pth] += -qj * dm3 * dF1[0][pth] * lr;
            }
        }
    }
    fit_block_sum<4>(acc, a.part, F_DAMP, a.stride);
}

// Born-Mayer-Huggins sensitivities over the short-range list (src/bhmftd.c:117-271 pair
// force w r, w = (B A e^-Bd - 6 C / d^7) / d): 1/2 sum (w_i - w_j) . r dw/dtheta for the
// (tSi, tO) and (tO, tO) type pairs
__global__ void __launch_bounds__(FIT_WARPS * 32) k_bhm_sens(int n, Cell c, const double4 *__restrict__ s,
                                                             const int *__restrict__ typ, const PairSR *__restrict__ pr,
                                                             int nt, const int *__restrict__ nbl,
                                                             const int *__restrict__ nbn, int cap, double srcutsq,
                                                             int tSi, int tO, const double3 *__restrict__ w,
                                                             double *part, int stride) {
    grid_dep();
    int i = blockIdx.x * FIT_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // A B C (Si-O), A B C (O-O), D (Si-O), D (O-O)
    if (i < n) {
        double4 si = s[i];
        double3 wi = w[i];
        int ti = typ[i];
        int m = min(nbn[i], cap);
        const int *L = nbl + (size_t)i * cap;
        for (int k = lane; k < m; k += 32) {
            int j = L[k];
            int tj = typ[j];
            int slot;
            if ((ti == tSi && tj == tO) || (ti == tO && tj == tSi)) slot = 0;
            else if (ti == tO && tj == tO) slot = 3;
            else continue;
            const PairSR &P = pr[ti * nt + tj];
            if (P.A == 0.0) continue;
            double4 sj = s[j];
            double3 r = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double r2 = norm2_exact(r);
            if (!(r2 < srcutsq)) continue;
            double d = sqrt(r2), ex = exp(-P.B * d);
            double3 wj = w[j];
            double vr = (wi.x - wj.x) * r.x + (wi.y - wj.y) * r.y + (wi.z - wj.z) * r.z;
            double h = 0.5 * vr / d;
            double d8 = r2 * r2 * r2 * r2;
            acc[slot + 0] += h * P.B * ex;
            acc[slot + 1] += h * P.A * ex * (1.0 - P.B * d);
            acc[slot + 2] += h * (-6.0 / (d8 / d));   // d/dC of -6 C / d^7 (h holds the 1/d)
            acc[6 + slot / 3] += h * (-8.0 / (d8 * d));   // d/dD of -8 D / d^9
        }
    }
    fit_block_sum<8>(acc, part, F_BHM, stride);
}

// ------------------------------------------------------------------ engine side
// the device half of set_fit_params from a device theta (recorded evaluations): the
// Born-Mayer-Huggins entries of (Si, O), (O, Si), (O, O) and the damping b, c of every
// damped direction (one thread per type pair) ...
__global__ void k_fit_tables(const double *__restrict__ th, int tSi, int tO, int nt, PairSR *__restrict__ pair,
                             PairDamp *__restrict__ damp) {
    grid_dep();
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nt * nt) return;
    int x = e / nt, y = e - x * nt;
    PairSR &P = pair[e];
    if ((x == tSi && y == tO) || (x == tO && y == tSi)) {
        P.A = th[0];
        P.B = th[1];
        P.C = th[2];
        P.D = th[10];
    } else if (x == tO && y == tO) {
        P.A = th[3];
        P.B = th[4];
        P.C = th[5];
        P.D = th[11];
    }
    PairDamp &D = damp[e];
    if (D.pad & 1) {
        D.b1 = th[8];
        D.c1 = th[9];
    }
    if (D.pad & 2) {
        D.b2 = th[8];
        D.c2 = th[9];
    }
}

// ... and the charges (q_Si = theta_6, q_O = -theta_6 / 2) and O polarisabilities
__global__ void k_fit_ions(int n, const int *__restrict__ typ, const double *__restrict__ th, int tSi, int tO,
                           double *__restrict__ q, double4 *__restrict__ r, double *__restrict__ pol,
                           double *__restrict__ invpol) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = typ[i];
    double v = q[i];
    if (t == tSi) v = th[6];
    else if (t == tO) v = -0.5 * th[6];
    q[i] = v;
    double4 x = r[i];
    x.w = v;
    r[i] = x;
    if (t == tO) {
        double alpha = th[7];
        for (int k = 0; k < 9; k++) {
            pol[(size_t)i * 9 + k] = (k % 4 == 0) ? alpha : 0.0;
            invpol[(size_t)i * 9 + k] = (k % 4 == 0) ? 1.0 / alpha : 0.0;
        }
    }
}

// loss and gradient from the reduced slots (see the file comment for the q_Si, alpha_O,
// b and c terms); res[NRES - 1] = the context's status bits
__global__ void k_fm_result(const double *__restrict__ sc, const double *__restrict__ th, double coul,
                            const unsigned *__restrict__ status, double *__restrict__ res) {
    grid_dep();
    if (threadIdx.x || blockIdx.x) return;
    res[0] = sc[F_LOSS];
    for (int k = 0; k < 6; k++) res[1 + k] = sc[F_BHM + k];
    double wqq = sc[F_WFQ0], wqm = sc[F_WFALL] - sc[F_WFQ0] - sc[F_WF0M];
    res[7] = (2.0 * wqq + wqm + sc[F_LESTAT]) / th[6];
    res[8] = sc[F_LMU] / (th[7] * th[7]);
    res[9] = coul * sc[F_DAMP + 0] + sc[F_DAMP + 2];
    res[10] = coul * sc[F_DAMP + 1] + sc[F_DAMP + 3];
    res[11] = sc[F_BHM + 6];
    res[12] = sc[F_BHM + 7];
    res[NRES - 1] = (double)*status;
}

// theta into the host copies of the parameters (p, the pair and damping tables, the
// charges); set_fit_params then copies them to the device
void Engine::fit_host_params(int tSi, int tO, const double *th) {
    if (tSi < 0 || tO < 0 || tSi >= nt || tO >= nt || tSi == tO) throw Error(MDFFGPU_ERR_ARG, "bad fit types");
    if (!(th[7] > 0.0)) throw Error(MDFFGPU_ERR_ARG, "polarisability must be positive");
    // Born-Mayer-Huggins tables (symmetric)
    for (int pair = 0; pair < 2; pair++) {
        int a = pair == 0 ? tSi : tO, b = tO;
        for (int s = 0; s < 2; s++) {
            int x = s ? b : a, y = s ? a : b;
            p.Abhmftd[x][y] = th[3 * pair + 0];
            p.Bbhmftd[x][y] = th[3 * pair + 1];
            p.Cbhmftd[x][y] = th[3 * pair + 2];
            p.Dbhmftd[x][y] = th[10 + pair];
            PairSR &P = h_pair[(size_t)x * nt + y];
            P.A = th[3 * pair + 0];
            P.B = th[3 * pair + 1];
            P.C = th[3 * pair + 2];
            P.D = th[10 + pair];
        }
    }
    // charges: q_Si = theta, q_O = -theta / 2
    p.qit[tSi] = th[6];
    p.qit[tO] = -0.5 * th[6];
    for (int i = 0; i < n; i++)
        if (h_typ[i] == tSi) h_q[i] = th[6];
        else if (h_typ[i] == tO) h_q[i] = -0.5 * th[6];
    // isotropic O polarisability
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) p.polit[tO][a][b] = (a == b) ? th[7] : 0.0;
    // Tang-Toennies b and c of every damped direction
    for (int t = 0; t < nt; t++)
        for (int i = 0; i < nt; i++)
            for (int j = 0; j < nt; j++)
                if (p.lpoldamping[t][i][j]) {
                    p.pol_damp_b[t][i][j] = th[8];
                    p.pol_damp_c[t][i][j] = th[9];
                }
    for (int x = 0; x < nt; x++)
        for (int y = 0; y < nt; y++) {
            PairDamp &D = h_damp[(size_t)x * nt + y];
            if (D.pad & 1) {
                D.b1 = th[8];
                D.c1 = th[9];
            }
            if (D.pad & 2) {
                D.b2 = th[8];
                D.c2 = th[9];
            }
        }
}

void Engine::set_fit_params(int tSi, int tO, const double *th) {
    fit_host_params(tSi, tO, th);
    fit_alloc();
    MDFF_CK(cudaMemcpyAsync(d_theta, th, sizeof(double) * MDFFGPU_FIT_NPARAM, cudaMemcpyHostToDevice, stream));
    fit_apply_theta(d_theta, tSi, tO);
    MDFF_CK(cudaStreamSynchronize(stream));
    gen++;
}

void Engine::fit_apply_theta(const double *d_th, int tSi, int tO) {
    MDFF_LAUNCH(*this, k_fit_tables, 1, 256, 0, d_th, tSi, tO, nt, d_pair, d_damp);
    MDFF_LAUNCH(*this, k_fit_ions, ceil_div(n, 256), 256, 0, n, d_typ, d_th, tSi, tO, d_q, d_r, d_pol, d_invpol);
}

// CG on A x = b over the polarisable ions, x0 = 0, until |r| <= rtol |b|; while
// recording, the loop is a device-controlled while node (the test in k_cg_step)
void Engine::solve_pim(const double3 *d_b, double3 *d_x, double rtol, int maxit) {
    int nb = ceil_div(n, 256);
    MDFF_CK(cudaMemsetAsync(d_x, 0, sizeof(double3) * n, stream));
    MDFF_CK(cudaMemcpyAsync(d_cg_r, d_b, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    MDFF_LAUNCH(*this, k_cg_rz, nb, 256, 0, n, d_polar, d_pol, d_cg_r, d_mu_save, d_part, part_stride, d_scal,
                d_ticket + 1);
    MDFF_CK(cudaMemcpyAsync(d_cg_p, d_mu_save, sizeof(double3) * n, cudaMemcpyDeviceToDevice, stream));
    // A p: the search direction vanishes off the polarisable ions, so the field passes
    // run over those ions only; A p and p.A p in the FP32 k-space combine (or k_cg_ap),
    // then x, r, z and r.z, r.r in one launch, as the induced-dipole CG does
    CgTest test{};
    test.mode = 2;
    test.rr0 = d_fscal + F_ADJ_RR0;
    test.itc = d_fscal + F_ADJ_IT;
    test.rtol2 = rtol * rtol;
    test.maxit = maxit;
    test.status = d_status;
    test.guard = d_ticket + 4;
    auto iteration = [&](CgTest t) {
        const bool sub = subset32 && npol > 0, ap_in_combine = sub && use32 && rec32;
        if (sub) field_pol(d_cg_p, d_ef_ind, nullptr, ap_in_combine);
        else field_of(d_qzero, d_cg_p, false, true, false, d_ef_ind);
        if (!ap_in_combine)
            MDFF_LAUNCH(*this, k_cg_ap, nb, 256, 0, n, d_polar, d_invpol, d_cg_p, d_ef_ind, d_cg_ap, d_part,
                        part_stride, d_scal, d_ticket);
        MDFF_LAUNCH(*this, k_cg_step, nb, 256, 0, n, 0, d_polar, d_pol, d_scal, d_cg_p, d_cg_ap, d_x, d_cg_r,
                    d_mu_save, nullptr, nullptr, d_part, part_stride, d_ticket + 1, t);
    };
    if (capturing) {
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
        return;
    }
    double rr0 = 0.0, rr = 0.0;
    MDFF_CK(cudaMemcpyAsync(&rr0, d_scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    rr = rr0;
    int it = 0;
    CgTest none{};
    while (rr > rtol * rtol * rr0 && rr > 0.0 && it < maxit) {
        iteration(none);
        MDFF_CK(cudaMemcpyAsync(&rr, d_scal + S_RR, sizeof(double), cudaMemcpyDeviceToHost, stream));
        MDFF_CK(cudaStreamSynchronize(stream));
        if (!std::isfinite(rr)) throw Error(MDFFGPU_ERR_NONFINITE, "adjoint CG diverged");
        it++;
        MDFF_LAUNCH(*this, k_cg_dir, nb, 256, 0, n, d_scal, d_mu_save, d_cg_p, none);
    }
    if (rr > rtol * rtol * rr0 && rr > 0.0) throw Error(MDFFGPU_ERR_SCF, "adjoint CG did not converge");
    last_adj_iter = it;
}

void Engine::fit_reduce(int first, int cnt, int nparts) {
    MDFF_LAUNCH(*this, k_reduce_slots, cnt, 256, 0, d_fpart, part_stride, first, nparts, d_fscal);
}

// Coulomb forces (electrostatic part only, energy units) of (q, mu) into out
void Engine::coul_forces(const double *d_qv, const double3 *d_muv, bool lq, bool ld, double3 *out) {
    MDFF_CK(cudaMemsetAsync(out, 0, sizeof(double3) * n, stream));
    // mixed: the FP32 real-space pass reads the context's charges from the packed
    // fractional coordinates, so d_qv may only be the charges themselves or absent (lq)
    if (use32 && real32)
        launch_dir32(*this, d_qv, d_muv, p.alphaES, lq, ld, ldmp != 0, true, false, nullptr, d_tmp3);
    else
        launch_dir(*this, d_qv, d_muv, p.alphaES, lq, ld, ldmp != 0, true, false, false, false, nullptr, nullptr,
                   d_tmp3);
    RecOut o;
    o.f = out;
    o.f_dir = d_tmp3;
    o.coul = coul_unit;
    launch_rec(*this, d_qv, d_muv, lq, ld, o);
}

// the status bits of an evaluation as the C ABI's error codes
void fit_status(unsigned st) {
    if (st & ST_CELL_OVERFLOW) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "a cell holds more ions than its capacity");
    if (st & ST_NONFINITE) throw Error(MDFFGPU_ERR_NONFINITE, "non-finite forces or CG residual");
    if (st & ST_TC_TIMEOUT) throw Error(MDFFGPU_ERR_TIMEOUT, "tensor-core k-space pass timed out waiting on its MMAs");
    if (st & ST_SCF) throw Error(MDFFGPU_ERR_SCF, "induced-dipole or adjoint CG did not converge");
}

void Engine::fit_alloc() {
    if (d_fpart) return;
    d_fpart = dalloc<double>((size_t)NFSLOT * part_stride);
    d_fscal = dalloc<double>(NFSLOT);
    d_w = dalloc<double3>(n);
    d_lam = dalloc<double3>(n);
    d_sv = dalloc<double3>(n);
    d_fa = dalloc<double3>(n);
    d_fb = dalloc<double3>(n);
    d_fc = dalloc<double3>(n);
    d_qw = dalloc<double>(n);
    d_muw = dalloc<double3>(n);
    d_efg_rec = dalloc<double>((size_t)n * 9);
    d_rw = dalloc<double2>((size_t)4 * nk);
    d_theta = dalloc<double>(MDFFGPU_FIT_NPARAM);
    d_fres = dalloc<double>(NRES);
}

// one evaluation on the stream: forces at the converged dipoles, the adjoint solve and
// the parameter sensitivities; d_res[0..NPARAM] = (sum |F - F_t|^2, dL/dtheta) with the
// q_Si and alpha_O terms taken at d_th[6], d_th[7]; d_res[NPARAM + 1] = status bits
void Engine::fit_issue(const double3 *d_ft, double scale, int tSi, int tO, const double *d_th, double *d_res) {
    if (!p.lcoulombic || !lpol) throw Error(MDFFGPU_ERR_STATE, "force matching needs the polarisable Coulomb model");
    if (pim_solver != MDFFGPU_PIM_CG && pim_solver != MDFFGPU_PIM_CG_FUSED)
        throw Error(MDFFGPU_ERR_STATE, "force matching needs a CG induced-dipole solver");
    // fully serialised launches on the one stream while an evaluation is issued (many
    // evaluations run concurrently; measured: both overlaps cost configurations per second)
    struct Off {
        bool &f, old;
        explicit Off(bool &x) : f(x), old(x) { f = false; }
        ~Off() { f = old; }
    } no_pdl(pdl), no_side(side_on);
    fit_alloc();
    const double *q = d_q;
    int nb = ceil_div(n, 256), nbw = ceil_div(n, FIT_WARPS);
    MDFF_CK(cudaMemsetAsync(d_fpart, 0, sizeof(double) * NFSLOT * part_stride, stream));
    // forces at the converged dipoles
    engforce();
    MDFF_LAUNCH(*this, k_fm_seed, nb, 256, 0, n, d_f, d_ft, scale, d_w, d_fpart, part_stride);
    fit_reduce(F_LOSS, 1, nb);
    // fixed geometry for the adjoint: fractional coordinates and lists as in engforce
    launch_kardir(*this, d_r, d_s);
    AdjArgs a;
    a.n = n;
    a.nt = nt;
    a.cap = cap_co;
    a.c = cell;
    a.s = d_s;
    a.q = q;
    a.mu = d_mu_tot;
    a.typ = d_typ;
    a.polar = d_polar;
    a.damp = d_damp;
    a.col = d_co;
    a.con = d_con;
    a.lrcutsq = lrcutsq;
    a.alpha = p.alphaES;
    a.ldamp = ldmp;
    a.tt.E[0] = 1.0;
    for (int k = 1; k < 9; k++) a.tt.E[k] = a.tt.E[k - 1] / (double)k;
    a.w = d_w;
    a.lambda = d_lam;
    a.sdir = d_sv;
    a.part = d_fpart;
    a.stride = part_stride;
    // s: real space
    MDFF_LAUNCH(*this, k_adj_dir, nbw, FIT_WARPS * 32, 0, a);
    // s: k space, drho_w from three rho passes of (q w_a, mu w_a).  These passes, the
    // adjoint solve and the Coulomb force evaluations below run in the context's precision;
    // the EFG pass runs in FP64 (launch_rec routes EFG requests to the FP64 kernels)
    for (int comp = 0; comp < 3; comp++) {
        MDFF_LAUNCH(*this, k_scale_by_w, nb, 256, 0, n, comp, q, d_mu_tot, d_w, d_qw, d_muw);
        RecOut o;
        o.rho_raw = d_rw + (size_t)comp * nk;
        launch_rec(*this, d_qw, d_muw, true, true, o);
    }
    MDFF_LAUNCH(*this, k_drho_w, ceil_div(nk, 256), 256, 0, nk, d_kvec, d_rw, d_rw + nk, d_rw + 2 * (size_t)nk,
                d_rw + 3 * (size_t)nk);
    {
        RecOut o;
        o.ef = d_fa;   // E_rec of drho_w (no self, no direct part)
        o.rho_acc = d_rw + 3 * (size_t)nk;
        launch_rec(*this, q, d_mu_tot, false, true, o);
    }
    {
        RecOut o;   // EFG_rec of (q, mu)
        o.efg = d_efg_rec;
        o.ef = d_fb;
        launch_rec(*this, q, d_mu_tot, true, true, o);
    }
    MDFF_LAUNCH(*this, k_adj_rhs, nb, 256, 0, n, d_polar, coul_unit, d_sv, d_fa, d_efg_rec, d_w, d_sv);
    // adjoint solve A lambda = s: FP64 (cached dipole-field factors of these positions) to
    // a 1e-11 relative residual, or mixed (the FP32 dipole-field records and phase tables
    // of the force evaluation above) to 1e-6
    {
        struct CoefScope {
            bool &flag;
            ~CoefScope() { flag = false; }
        } scope{coef_ready};
        if (!(use32 && real32)) launch_dir_prep(*this, p.alphaES);
        coef_ready = true;
        solve_pim(d_sv, d_lam, use32 ? 1e-6 : 1e-11, 500);
    }
    // parameter sensitivities
    MDFF_LAUNCH(*this, k_bhm_sens, nbw, FIT_WARPS * 32, 0, n, cell, d_s, d_typ, d_pair, nt, d_nb, d_nbn, cap_nb,
                srcutsq, tSi, tO, d_w, d_fpart, part_stride);
    fit_reduce(F_BHM, 8, nbw);
    MDFF_LAUNCH(*this, k_damp_sens, nbw, FIT_WARPS * 32, 0, a);
    fit_reduce(F_DAMP, 4, nbw);
    coul_forces(q, d_mu_tot, true, true, d_fa);      // F(q, mu)
    coul_forces(q, d_muzero, true, false, d_fb);     // F(q, 0)
    coul_forces(d_qzero, d_mu_tot, false, true, d_fc);   // F(0, mu)
    MDFF_LAUNCH(*this, k_dot3, nb, 256, 0, n, d_w, d_fa, nullptr, d_fpart, (int)F_WFALL, part_stride);
    MDFF_LAUNCH(*this, k_dot3, nb, 256, 0, n, d_w, d_fb, nullptr, d_fpart, (int)F_WFQ0, part_stride);
    MDFF_LAUNCH(*this, k_dot3, nb, 256, 0, n, d_w, d_fc, nullptr, d_fpart, (int)F_WF0M, part_stride);
    field_of(q, d_muzero, true, false, ldmp != 0, d_fb);   // E(q, 0), the static field
    MDFF_LAUNCH(*this, k_dot3, nb, 256, 0, n, d_lam, d_fb, d_polar, d_fpart, (int)F_LESTAT, part_stride);
    MDFF_LAUNCH(*this, k_dot3, nb, 256, 0, n, d_lam, d_mu_ind, d_polar, d_fpart, (int)F_LMU, part_stride);
    fit_reduce(F_WFALL, 5, nb);
    MDFF_LAUNCH(*this, k_fm_result, 1, 32, 0, d_fscal, d_th, coul_unit, d_status, d_res);
}

void Engine::force_match(const double3 *d_ft, double scale, double *h_res, int tSi, int tO) {
    fit_alloc();
    // theta of the current parameters (set_fit_params keeps the device copy current;
    // here the q_Si and alpha_O the result assembly divides by)
    double th[MDFFGPU_FIT_NPARAM] = {p.Abhmftd[tSi][tO], p.Bbhmftd[tSi][tO], p.Cbhmftd[tSi][tO],
                                     p.Abhmftd[tO][tO],  p.Bbhmftd[tO][tO],  p.Cbhmftd[tO][tO],
                                     p.qit[tSi],         p.polit[tO][0][0],  0.0, 0.0,
                                     p.Dbhmftd[tSi][tO], p.Dbhmftd[tO][tO]};
    MDFF_CK(cudaMemcpyAsync(d_theta, th, sizeof(double) * 8, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
    fit_issue(d_ft, scale, tSi, tO, d_theta, d_fres);
    double res[NRES];
    MDFF_CK(cudaMemcpyAsync(res, d_fres, sizeof(double) * NRES, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    fit_status((unsigned)res[NRES - 1]);
    for (int k = 0; k <= MDFFGPU_FIT_NPARAM; k++) h_res[k] = res[k];
}

// record one evaluation (theta from d_th, result into d_res) as a CUDA graph: the
// parameter update, forces with the induced-dipole CG, adjoint CG and sensitivities
void Engine::capture_fit(const double *d_th, int tSi, int tO, double scale, double *d_res) {
    if (fit_exec) cudaGraphExecDestroy(fit_exec);
    fit_exec = nullptr;
    if (p.lverletL && !list_ready) gen_verletlist();
    fit_alloc();
    if (use32 && real32 && p.lcoulombic) ensure_real32();   // no allocation while recording
    MDFF_CK(cudaStreamSynchronize(stream));
    long long l0 = launches;
    MDFF_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    cudaGraph_t graph = nullptr;
    try {
        MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
        pdl = false;
        fit_apply_theta(d_th, tSi, tO);
        pdl = true;
        fit_issue(d_ft, scale, tSi, tO, d_th, d_res);
    } catch (...) {
        capturing = false;
        pdl = true;
        forget_sides();
        cudaStreamEndCapture(stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        launches = l0;
        throw;
    }
    capturing = false;
    MDFF_CK(cudaStreamEndCapture(stream, &graph));
    cudaError_t err = cudaGraphInstantiate(&fit_exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        fit_exec = nullptr;
        MDFF_CK(err);
    }
    launches = l0;
    fit_graph_gen = gen;
}

}  // namespace mdffgpu
