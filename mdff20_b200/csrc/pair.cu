// Real-space pair kernels: n-m Lennard-Jones, BHMFT(D) with Tang-Toennies damping and
// the real-space multipole Ewald sum (charges + dipoles).  One warp per ion over that
// ion's FULL neighbour list; each lane takes every 32nd neighbour, per-ion sums are
// combined with warp shuffles and written by lane 0 (no atomics); energies and
// virials go to per-block partial sums reduced in a fixed order.
#include "engine.cuh"
#include "sr_pair.cuh"

namespace mdffgpu {

constexpr int PAIR_WARPS = 8;  // warps (= ions) per block

// block-level sum of NV per-warp values into part[(slot+v)*stride + blockIdx.x]
template <int NV>
__device__ __forceinline__ void block_partials(const double (&v)[NV], double *part, int slot, int stride) {
    __shared__ double sh[PAIR_WARPS][NV];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < NV; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = 0.0;
        for (int k = 0; k < PAIR_WARPS; k++) a += sh[k][threadIdx.x];
        part[(size_t)(slot + threadIdx.x) * stride + blockIdx.x] = a;
    }
}

// ---------------------------------------------------------------- short range
// engforce_nmlj_pbc (src/nmlj.c:254-385) when LJ, engforce_bhmftd_pbc
// (src/bhmftd.c:117-271) otherwise.  Adds forces into f; slot gets u (x2) and the
// virial sum over the full list of (r_a f_b + r_b f_a).  FAST (mixed precision,
// Buckingham): bhm_pair_fast, the same function with fewer roundings and divisions, in
// FP64: in FP32 the repulsion A exp(-B r) carries the rounding of r times B r (about 8 at
// Si-O contact), which measured an 8e-6 relative force error on the bench system.
template <bool LJ, bool FAST = false>
__global__ void __launch_bounds__(PAIR_WARPS * 32, FAST ? 3 : 1) k_sr(int n, Cell c, const double4 *__restrict__ s,
                                                        const int *__restrict__ typ, const PairSR *__restrict__ pr,
                                                        int nt, const int *__restrict__ nbl,
                                                        const int *__restrict__ nbn, int cap, double srcutsq,
                                                        int trunctype, int damped, TT tt, double3 *__restrict__ f,
                                                        double *__restrict__ part, int slot, int stride) {
    grid_dep();
    int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};  // u, Vxx Vxy Vxz Vyy Vyz Vzz
    double fx = 0, fy = 0, fz = 0;
    if (i < n) {
        double4 si = s[i];
        int ti = typ[i];
        int m = nbn[i];
        if (m > cap) m = cap;
        const int *L = nbl + (size_t)i * cap;
        // neighbour types and positions one round ahead, indices two rounds ahead
        int jc = lane < m ? L[lane] : 0;
        int jn = lane + 32 < m ? L[lane + 32] : 0;
        int tc = lane < m ? typ[jc] : 0;
        double4 sc = lane < m ? s[jc] : si;
        for (int k = lane; k < m; k += 32) {
            int tj = tc;
            double4 sj = sc;
            if (k + 32 < m) {
                tc = typ[jn];
                sc = s[jn];
            }
            if (k + 64 < m) jn = L[k + 64];
            const PairSR &P = pr[ti * nt + tj];
            if (!LJ && P.A == 0.0) continue;
            double3 r = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double r2 = norm2_exact(r);
            if (!(r2 < srcutsq)) continue;
            double u, w;
            if (FAST && !LJ) bhm_pair_fast(P, r2, damped, u, w);
            else sr_pair<LJ>(P, r2, trunctype, damped, tt, u, w);
            sr_accumulate(r, u, w, fx, fy, fz, acc);
        }
    }
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
#pragma unroll
    for (int k = 0; k < 7; k++) acc[k] = warp_sum(acc[k]);
    if (i < n && lane == 0) {
        double3 o = f[i];
        f[i] = make_double3(o.x + fx, o.y + fy, o.z + fz);
    }
    if (i >= n) {
#pragma unroll
        for (int k = 0; k < 7; k++) acc[k] = 0.0;
    }
    block_partials<7>(acc, part, slot, stride);
}

void launch_sr(Engine &e, bool lj) {
    TT tt = make_tt();
    int nb = ceil_div(e.n, PAIR_WARPS);
    if (lj)
        MDFF_LAUNCH(e, k_sr<true>, nb, PAIR_WARPS * 32, 0, e.n, e.cell, e.d_s, e.d_typ, e.d_pair, e.nt, e.d_nb,
                    e.d_nbn, e.cap_nb, e.srcutsq, e.p.trunctype, 0, tt, e.d_f, e.d_part, (int)S_LJ_U,
                    e.part_stride);
    else if (e.use32)
        MDFF_LAUNCH(e, (k_sr<false, true>), nb, PAIR_WARPS * 32, 0, e.n, e.cell, e.d_s, e.d_typ, e.d_pair, e.nt,
                    e.d_nb, e.d_nbn, e.cap_nb, e.srcutsq, e.p.trunctype, e.p.lbhmftd, tt, e.d_f, e.d_part,
                    (int)S_BH_U, e.part_stride);
    else
        MDFF_LAUNCH(e, k_sr<false>, nb, PAIR_WARPS * 32, 0, e.n, e.cell, e.d_s, e.d_typ, e.d_pair, e.nt, e.d_nb,
                    e.d_nbn, e.cap_nb, e.srcutsq, e.p.trunctype, e.p.lbhmftd, tt, e.d_f, e.d_part, (int)S_BH_U,
                    e.part_stride);
}

// ---------------------------------------------------------------- real-space Ewald
// multipole_ES_dir (src/ewald.c:353-871) for charges and dipoles, from ion i's side.
// For each neighbour j within cutlongrange (d2 <= lrcutsq, src/ewald.c:486) the
// tensors T0..T3 (src/ewald.c:562-620) are contracted directly with q and mu:
//   field at i      : -qj T1 (+ qj T1D1 damped)  and  T2 mu_j (only if mu_i, mu_j != 0)
//   force on i      : -f_ij with f_ij as src/ewald.c:719-812
//   EFG at i        : -qj T2 + T3 . mu_j
//   energy, virial  : half of the pair value (each pair is seen from both ions)
// Template flags select what is computed; FORCES also computes energy and virial.
struct DirArgs {
    int n, nt, cap;
    Cell c;
    const double4 *s;
    const double *q;
    const double3 *mu;
    const int *typ;
    const PairDamp *damp;
    const int *col, *con;
    double lrcutsq, alpha;
    TT tt;
    int lq, ld, ldamp, efg_q;
    double3 *ef;
    double *efg;
    double3 *f;
    double *part;
    int slot, stride;
};

template <bool FORCES, bool EF, bool EFG>
__global__ void __launch_bounds__(PAIR_WARPS * 32) k_dir(DirArgs a) {
    grid_dep();
    int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};   // u, V6
    double fi[3] = {0, 0, 0}, ei[3] = {0, 0, 0};
    double gi[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double alpha = a.alpha, alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha5 = alpha3 * alpha2;
    const double rpi = 1.7724538509055160273;  // sqrt(pi), src/constants.c:20
    if (i < a.n) {
        double4 si = a.s[i];
        double qi = a.lq ? a.q[i] : 0.0;
        double3 mi = a.ld ? a.mu[i] : make_double3(0, 0, 0);
        bool dip_i = (mi.x != 0.0) || (mi.y != 0.0) || (mi.z != 0.0);
        int ti = a.typ[i];
        int m = a.con[i];
        if (m > a.cap) m = a.cap;
        const int *L = a.col + (size_t)i * a.cap;
        for (int k = lane; k < m; k += 32) {
            int j = L[k];
            double4 sj = a.s[j];
            double3 r = pbc_frac(a.c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double d2 = norm2_exact(r);
            if (d2 > a.lrcutsq) continue;
            double qj = a.lq ? a.q[j] : 0.0;
            double3 mj = a.ld ? a.mu[j] : make_double3(0, 0, 0);
            bool dip_j = (mj.x != 0.0) || (mj.y != 0.0) || (mj.z != 0.0);
            double d = sqrt(d2), d3 = d2 * d, d5 = d3 * d2;
            double dm1 = 1.0 / d, dm3 = dm1 / d2, dm5 = dm3 / d2, dm7 = dm5 / d2;
            double expon = exp(-alpha2 * d2) / rpi;
            double F0 = erfc(alpha * d);
            double F1 = F0 + 2.0 * alpha * d * expon;
            double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
            double F3 = F2 + 8.0 * alpha5 * d5 * expon / 15.0;
            // Tang-Toennies damping of the charge->dipole field, src/ewald.c:505-539
            double F1d1 = 0.0, F1d2 = 0.0, F2d1 = 0.0, F2d2 = 0.0;
            bool damp = false;
            if (a.ldamp) {
                const PairDamp &D = a.damp[ti * a.nt + a.typ[j]];
                if (D.ldamp) {
                    damp = true;
                    double fd1, fdd1, fd2, fdd2;
                    tt_damp(a.tt, D.b1, D.c1, d, D.k1, fd1, fdd1);
                    tt_damp(a.tt, D.b2, D.c2, d, D.k2, fd2, fdd2);
                    F1d1 = -fd1 + 1.0;
                    F1d2 = -fd2 + 1.0;
                    F2d1 = F1d1 + (d / 3.0) * fdd1;
                    F2d2 = F1d2 + (d / 3.0) * fdd2;
                }
            }
            double F1_dm3 = F1 * dm3, F2_dm5 = 3.0 * F2 * dm5;
            double u = 0.0;
            double fij[3] = {0, 0, 0};
            // charge-charge, src/ewald.c:703-731
            if (a.lq) {
                u += qi * qj * (dm1 * F0);
                if (EF) {
                    double cfe = qj * dm3 * (F1 - F1d1);   // -qj T1 + qj T1D1
                    ei[0] += cfe * r.x;
                    ei[1] += cfe * r.y;
                    ei[2] += cfe * r.z;
                }
                if (FORCES) {
                    double cf = -qi * qj * F1_dm3;        // qij T1
                    fij[0] = cf * r.x;
                    fij[1] = cf * r.y;
                    fij[2] = cf * r.z;
                }
                if (EFG && a.efg_q) {
                    double rr[3] = {r.x, r.y, r.z};
                    for (int p = 0; p < 3; p++)
                        for (int q = 0; q < 3; q++)
                            gi[3 * p + q] += -qj * (rr[p] * rr[q] * F2_dm5 - (p == q ? F1_dm3 : 0.0));
                }
            }
            double rmi = r.x * mi.x + r.y * mi.y + r.z * mi.z;
            double rmj = r.x * mj.x + r.y * mj.y + r.z * mj.z;
            // dipole-dipole, src/ewald.c:737-761 (both dipoles non-zero)
            if (a.ld && dip_i && dip_j) {
                double mm = mi.x * mj.x + mi.y * mj.y + mi.z * mj.z;
                u += F1_dm3 * mm - F2_dm5 * rmi * rmj;
                if (EF) {
                    ei[0] += F2_dm5 * rmj * r.x - F1_dm3 * mj.x;
                    ei[1] += F2_dm5 * rmj * r.y - F1_dm3 * mj.y;
                    ei[2] += F2_dm5 * rmj * r.z - F1_dm3 * mj.z;
                }
                double F3_dm7 = F3 * dm7 * 15.0;
                if (FORCES) {
                    double c1 = -F3_dm7 * rmi * rmj, c2 = F2_dm5;
                    fij[0] -= c1 * r.x + c2 * (mm * r.x + mi.x * rmj + mj.x * rmi);
                    fij[1] -= c1 * r.y + c2 * (mm * r.y + mi.y * rmj + mj.y * rmi);
                    fij[2] -= c1 * r.z + c2 * (mm * r.z + mi.z * rmj + mj.z * rmi);
                }
                if (EFG) {
                    double rr[3] = {r.x, r.y, r.z}, mv[3] = {mj.x, mj.y, mj.z};
                    for (int p = 0; p < 3; p++)
                        for (int q = 0; q < 3; q++)
                            gi[3 * p + q] += -F3_dm7 * rmj * rr[p] * rr[q] +
                                             F2_dm5 * ((p == q ? rmj : 0.0) + mv[p] * rr[q] + rr[p] * mv[q]);
                }
            }
            // charge-dipole, src/ewald.c:767-812
            if (a.lq && a.ld && (dip_i || dip_j)) {
                u += F1_dm3 * (qi * rmj - qj * rmi);
                if (FORCES) {
                    double wx = qj * mi.x - qi * mj.x, wy = qj * mi.y - qi * mj.y, wz = qj * mi.z - qi * mj.z;
                    double rw = r.x * wx + r.y * wy + r.z * wz;
                    fij[0] += F2_dm5 * rw * r.x - F1_dm3 * wx;
                    fij[1] += F2_dm5 * rw * r.y - F1_dm3 * wy;
                    fij[2] += F2_dm5 * rw * r.z - F1_dm3 * wz;
                }
                if (damp) {
                    u += dm3 * (-qi * F1d2 * rmj + qj * F1d1 * rmi);
                    if (FORCES) {
                        double a1 = 3.0 * F2d1 * dm5, b1 = F1d1 * dm3;
                        double a2 = 3.0 * F2d2 * dm5, b2 = F1d2 * dm3;
                        fij[0] += -qj * (a1 * rmi * r.x - b1 * mi.x) + qi * (a2 * rmj * r.x - b2 * mj.x);
                        fij[1] += -qj * (a1 * rmi * r.y - b1 * mi.y) + qi * (a2 * rmj * r.y - b2 * mj.y);
                        fij[2] += -qj * (a1 * rmi * r.z - b1 * mi.z) + qi * (a2 * rmj * r.z - b2 * mj.z);
                    }
                }
            }
            if (FORCES) {
                fi[0] -= fij[0];
                fi[1] -= fij[1];
                fi[2] -= fij[2];
                acc[0] += u;
                acc[1] += -(r.x * fij[0] + r.x * fij[0]);
                acc[2] += -(r.x * fij[1] + r.y * fij[0]);
                acc[3] += -(r.x * fij[2] + r.z * fij[0]);
                acc[4] += -(r.y * fij[1] + r.y * fij[1]);
                acc[5] += -(r.y * fij[2] + r.z * fij[1]);
                acc[6] += -(r.z * fij[2] + r.z * fij[2]);
            } else {
                acc[0] += u;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 7; k++) acc[k] = warp_sum(acc[k]);
    if (FORCES) {
        for (int k = 0; k < 3; k++) fi[k] = warp_sum(fi[k]);
    }
    if (EF) {
        for (int k = 0; k < 3; k++) ei[k] = warp_sum(ei[k]);
    }
    if (EFG) {
        for (int k = 0; k < 9; k++) gi[k] = warp_sum(gi[k]);
    }
    if (i < a.n && lane == 0) {
        if (FORCES && a.f) a.f[i] = make_double3(fi[0], fi[1], fi[2]);
        if (EF && a.ef) a.ef[i] = make_double3(ei[0], ei[1], ei[2]);
        if (EFG && a.efg)
            for (int k = 0; k < 9; k++) a.efg[(size_t)i * 9 + k] = gi[k];
    }
    if (i >= a.n) {
#pragma unroll
        for (int k = 0; k < 7; k++) acc[k] = 0.0;
    }
    if (a.part) block_partials<7>(acc, a.part, a.slot, a.stride);
}

void launch_dir(Engine &e, const double *q, const double3 *mu, double alpha, bool lq, bool ld, bool damp,
                bool forces, bool ef, bool efg, bool efg_q, double3 *out_ef, double *out_efg, double3 *out_f) {
    const double4 *s = e.d_s;
    DirArgs a;
    a.n = e.n;
    a.nt = e.nt;
    a.cap = e.cap_co;
    a.c = e.cell;
    a.s = s;
    a.q = q;
    a.mu = mu;
    a.typ = e.d_typ;
    a.damp = e.d_damp;
    a.col = e.d_co;
    a.con = e.d_con;
    a.lrcutsq = e.lrcutsq;
    a.alpha = alpha;
    a.tt.E[0] = 1.0;
    for (int k = 1; k < 9; k++) a.tt.E[k] = a.tt.E[k - 1] / (double)k;
    a.lq = lq;
    a.ld = ld;
    a.ldamp = damp;
    a.efg_q = efg_q;
    a.ef = out_ef;
    a.efg = out_efg;
    a.f = out_f;
    a.part = e.d_part;
    a.slot = S_DIR_U;
    a.stride = e.part_stride;
    int nb = ceil_div(e.n, PAIR_WARPS);
    if (efg || (ef && forces))
        MDFF_LAUNCH(e, (k_dir<true, true, true>), nb, PAIR_WARPS * 32, 0, a);
    else if (forces)
        MDFF_LAUNCH(e, (k_dir<true, false, false>), nb, PAIR_WARPS * 32, 0, a);
    else
        MDFF_LAUNCH(e, (k_dir<false, true, false>), nb, PAIR_WARPS * 32, 0, a);
}

// ---------------------------------------------------------------- cached dipole field
// Within one force evaluation the positions are fixed while the induced dipoles are
// iterated (src/pim.c:236-278), so the screened pair factors F1/d^3 and 3 F2/d^5 of
// the dipole field (the T2 tensor, src/ewald.c:581-603) are computed once per list
// entry and reused by every iteration: the iteration kernel then does no erfc/exp.
__global__ void __launch_bounds__(PAIR_WARPS * 32) k_dir_prep(int n, Cell c, const double4 *__restrict__ s,
                                                             const int *__restrict__ col,
                                                             const int *__restrict__ con, int cap, double lrcutsq,
                                                             double alpha, double2 *__restrict__ coef) {
    grid_dep();
    int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    const double rpi = 1.7724538509055160273;
    const double alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
    double4 si = s[i];
    int m = min(con[i], cap);
    const int *L = col + (size_t)i * cap;
    double2 *C = coef + (size_t)i * cap;
    for (int k = lane; k < m; k += 32) {
        double4 sj = s[L[k]];
        double3 r = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
        double d2 = norm2_exact(r);
        double2 out = make_double2(0.0, 0.0);
        if (!(d2 > lrcutsq)) {
            double d = sqrt(d2), d3 = d2 * d;
            double dm1 = 1.0 / d, dm3 = dm1 / d2, dm5 = dm3 / d2;
            double expon = exp(-alpha2 * d2) / rpi;
            double F0 = erfc(alpha * d);
            double F1 = F0 + 2.0 * alpha * d * expon;
            double F2 = F1 + 4.0 * alpha3 * d3 * expon / 3.0;
            out = make_double2(F1 * dm3, 3.0 * F2 * dm5);
        }
        C[k] = out;
    }
}

// field of the dipoles mu from the cached factors: E_i = sum_j (3F2/d^5 (r.mu_j) r - F1/d^3 mu_j),
// only when mu_i and mu_j are non-zero (src/ewald.c:737-749)
__global__ void __launch_bounds__(PAIR_WARPS * 32) k_dir_field_cached(int n, Cell c, const double4 *__restrict__ s,
                                                                     const int *__restrict__ col,
                                                                     const int *__restrict__ con, int cap,
                                                                     const double2 *__restrict__ coef,
                                                                     const double3 *__restrict__ mu,
                                                                     double3 *__restrict__ ef) {
    grid_dep();
    int i = blockIdx.x * PAIR_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    double3 mi = mu[i];
    bool dip_i = (mi.x != 0.0) || (mi.y != 0.0) || (mi.z != 0.0);
    double ex = 0.0, ey = 0.0, ez = 0.0;
    if (dip_i) {
        double4 si = s[i];
        int m = min(con[i], cap);
        const int *L = col + (size_t)i * cap;
        const double2 *C = coef + (size_t)i * cap;
        for (int k = lane; k < m; k += 32) {
            double2 cf = C[k];
            if (cf.x == 0.0 && cf.y == 0.0) continue;
            int j = L[k];
            double3 mj = mu[j];
            if (mj.x == 0.0 && mj.y == 0.0 && mj.z == 0.0) continue;
            double4 sj = s[j];
            double3 r = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double rmj = r.x * mj.x + r.y * mj.y + r.z * mj.z;
            ex += cf.y * rmj * r.x - cf.x * mj.x;
            ey += cf.y * rmj * r.y - cf.x * mj.y;
            ez += cf.y * rmj * r.z - cf.x * mj.z;
        }
    }
    ex = warp_sum(ex);
    ey = warp_sum(ey);
    ez = warp_sum(ez);
    if (lane == 0) ef[i] = make_double3(ex, ey, ez);
}

void launch_dir_prep(Engine &e, double alpha) {
    int nb = ceil_div(e.n, PAIR_WARPS);
    MDFF_LAUNCH(e, k_dir_prep, nb, PAIR_WARPS * 32, 0, e.n, e.cell, e.d_s, e.d_co, e.d_con, e.cap_co, e.lrcutsq,
                alpha, e.d_coef);
}

void launch_dir_field_cached(Engine &e, const double3 *mu, double3 *out_ef) {
    int nb = ceil_div(e.n, PAIR_WARPS);
    int pd = -1;
    e.prof_begin("k_dir", &pd);
    MDFF_LAUNCH(e, k_dir_field_cached, nb, PAIR_WARPS * 32, 0, e.n, e.cell, e.d_s, e.d_co, e.d_con, e.cap_co,
                e.d_coef, mu, out_ef);
    e.prof_end("k_dir", pd, 0.0);
}

}  // namespace mdffgpu
