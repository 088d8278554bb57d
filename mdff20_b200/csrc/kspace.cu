// Reciprocal-space multipole Ewald sum: multipole_ES_rec (src/ewald.c:876-1051) with
// the structure factors of struct_fact / charge_density_* (src/kspace.c:154-302).
//
// The reference tabulates cos/sin(k.r) for every (k, ion) pair (N*nk doubles twice,
// src/kspace.c:35-38).  Here no table exists: with k = 2*pi*B*n (n integer, the
// reference's own k-vectors, src/kspace.c:87-89) the phase factorises,
//     exp(i k.r) = E0[nx] * E1[ny] * E2[nz],   E_d[m] = exp(2*pi*i*m*t_d),  t = B^T r,
// and each factor table is built per ion from one exactly reduced sincospi plus a
// complex recurrence.  Two passes:
//   k_rho     : rho(k) = sum_i (q_i + i k.mu_i) exp(i k.r_i); threads own k-row
//               segments of up to KSEG values of nz, ions stream through shared memory
//               in tiles; per-ion-chunk partial sums, reduced in a fixed order;
//   k_rec_ion : per ion, the k sums for field, force and EFG, threads own ions, the
//               Ak-scaled rho(k) streams through shared memory in row-aligned tiles;
//               sums are kept in n-space and mapped to Cartesian k once per ion.
#include "engine.cuh"

namespace mdffgpu {

constexpr int RHO_THREADS = 128;
constexpr int RHO_TI = 32;          // ions per shared-memory tile
constexpr int ION_THREADS = 128;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(2*pi*i*t) with exact reduction of t to [-1/2, 1/2]
__device__ __forceinline__ double2 cis2pi(double t) {
    double x = t - rint(t);
    double sn, cs;
    sincospi(2.0 * x, &sn, &cs);
    return make_double2(cs, sn);
}

// phase coordinates t = B^T r (so that k.r = 2*pi*n.t for the reference's k)
__device__ __forceinline__ double3 phase_coord(const Cell &c, double x, double y, double z) {
    return make_double3(c.B[0][0] * x + c.B[1][0] * y + c.B[2][0] * z,
                        c.B[0][1] * x + c.B[1][1] * y + c.B[2][1] * z,
                        c.B[0][2] * x + c.B[1][2] * y + c.B[2][2] * z);
}

// ---------------------------------------------------------------- pass 1: rho(k)
template <bool LQ, bool LD>
__global__ void __launch_bounds__(RHO_THREADS) k_rho(int n, int chunk, Cell c, int K0, int K1, int K2,
                                                    const double4 *__restrict__ r, const double *__restrict__ q,
                                                    const double3 *__restrict__ mu, int nseg,
                                                    const KSeg *__restrict__ seg, double2 *__restrict__ part,
                                                    int nk) {
    extern __shared__ double2 sm[];
    const int W0 = K0 + 1, W1 = 2 * K1 + 1, W2 = 2 * K2 + 1, WT = W0 + W1 + W2;
    double2 *E = sm;                                   // [RHO_TI][WT]
    double *qs = (double *)(sm + RHO_TI * WT);         // [RHO_TI]
    double *ms = qs + RHO_TI;                          // [RHO_TI][3]
    int sid = blockIdx.x * RHO_THREADS + threadIdx.x;
    KSeg S;
    if (sid < nseg) S = seg[sid];
    else S.nx = S.ny = S.z0 = S.cnt = S.koff = 0;
    double2 acc[KSEG];
#pragma unroll
    for (int z = 0; z < KSEG; z++) acc[z] = make_double2(0.0, 0.0);
    int i0 = blockIdx.y * chunk, i1 = min(n, i0 + chunk);
    const double tpi = TPI_D;
    for (int t0 = i0; t0 < i1; t0 += RHO_TI) {
        int nt = min(RHO_TI, i1 - t0);
        // tables: thread (slot, dim) for slot < RHO_TI, dim < 3
        if (threadIdx.x < 3 * RHO_TI) {
            int slot = threadIdx.x % RHO_TI, dim = threadIdx.x / RHO_TI;
            if (slot < nt) {
                int ia = t0 + slot;
                double4 ri = r[ia];
                double3 t = phase_coord(c, ri.x, ri.y, ri.z);
                double td = dim == 0 ? t.x : (dim == 1 ? t.y : t.z);
                double2 e1 = cis2pi(td);
                double2 *T = E + slot * WT + (dim == 0 ? 0 : (dim == 1 ? W0 : W0 + W1));
                int K = dim == 0 ? K0 : (dim == 1 ? K1 : K2);
                int zero = dim == 0 ? 0 : K;  // index of m = 0
                double2 v = make_double2(1.0, 0.0);
                T[zero] = v;
                for (int m = 1; m <= K; m++) {
                    v = (m == 1) ? e1 : cmul(v, e1);
                    T[zero + m] = v;
                    if (dim != 0) T[zero - m] = make_double2(v.x, -v.y);
                }
                if (dim == 0) {
                    qs[slot] = LQ ? q[ia] : 0.0;
                    if (LD) {
                        double3 m3 = mu[ia];
                        double3 mm = phase_coord(c, m3.x, m3.y, m3.z);
                        ms[3 * slot] = mm.x;
                        ms[3 * slot + 1] = mm.y;
                        ms[3 * slot + 2] = mm.z;
                    }
                }
            }
        }
        __syncthreads();
        if (sid < nseg) {
            for (int a = 0; a < nt; a++) {
                const double2 *T = E + a * WT;
                double2 b = cmul(T[S.nx], T[W0 + K1 + S.ny]);
                const double2 *Z = T + W0 + W1 + K2 + S.z0;
                double qa = LQ ? qs[a] : 0.0;
                double c0 = 0.0, c1 = 0.0;
                if (LD) {
                    c0 = tpi * ((double)S.nx * ms[3 * a] + (double)S.ny * ms[3 * a + 1]);
                    c1 = tpi * ms[3 * a + 2];
                }
#pragma unroll
                for (int z = 0; z < KSEG; z++) {
                    if (z < S.cnt) {
                        double2 ph = cmul(b, Z[z]);
                        if (LQ) {
                            acc[z].x += qa * ph.x;
                            acc[z].y += qa * ph.y;
                        }
                        if (LD) {
                            double kmu = c0 + (double)(S.z0 + z) * c1;
                            acc[z].x -= kmu * ph.y;
                            acc[z].y += kmu * ph.x;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (sid < nseg) {
        double2 *P = part + (size_t)blockIdx.y * nk + S.koff;
#pragma unroll
        for (int z = 0; z < KSEG; z++)
            if (z < S.cnt) P[z] = acc[z];
    }
}

// sum the ion-chunk partials of rho(k) in a fixed order; store Ak*rho(k); block
// partials of u_rec = sum Ak|rho|^2 and of the k-space virial (src/ewald.c:945-1006)
__global__ void k_rho_reduce(int nk, int nchunks, const double2 *__restrict__ part, const double *__restrict__ Ak,
                             const double *__restrict__ kcoe, const double3 *__restrict__ kv,
                             double2 *__restrict__ rho_s, double *__restrict__ ppart, int slot, int stride) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (k < nk) {
        double2 rho = make_double2(0.0, 0.0);
        for (int c = 0; c < nchunks; c++) {
            double2 p = part[(size_t)c * nk + k];
            rho.x += p.x;
            rho.y += p.y;
        }
        double ak = Ak[k], co = kcoe[k];
        double3 kk = kv[k];
        double str = (rho.x * rho.x + rho.y * rho.y) * ak;
        rho_s[k] = make_double2(ak * rho.x, ak * rho.y);
        v[0] = str;
        v[1] = (1.0 - co * kk.x * kk.x) * str;
        v[2] = -co * kk.x * kk.y * str;
        v[3] = -co * kk.x * kk.z * str;
        v[4] = (1.0 - co * kk.y * kk.y) * str;
        v[5] = -co * kk.y * kk.z * str;
        v[6] = (1.0 - co * kk.z * kk.z) * str;
    }
    __shared__ double sh[8][7];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 7; q++) v[q] = warp_sum(v[q]);
    if (l == 0)
        for (int q = 0; q < 7; q++) sh[w][q] = v[q];
    __syncthreads();
    if (threadIdx.x < 7) {
        double a = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) a += sh[q][threadIdx.x];
        ppart[(size_t)(slot + threadIdx.x) * stride + blockIdx.x] = a;
    }
}

// ---------------------------------------------------------------- pass 2: per ion
struct IonArgs {
    int n, K0, K1, K2;
    Cell c;
    const double4 *r;
    const double *q;
    const double3 *mu;
    const KRow *row;
    const int *tile_row, *tile_k;
    int ntile;
    const double2 *rho_s;
    double tfpiV, self2;    // 8 pi / V, 2*selfa2 (self field coefficient)
    int ld, want_ef, want_f, want_efg;
    const double3 *ef_dir;  // added to the result when not null
    double3 *ef;
    double coul;            // force unit
    const double3 *f_dir;   // direct-space forces (added x coul) when not null
    double3 *f;             // f += f_dir*coul + f_rec*coul
    double *efg;            // [n][9], receives self + dir (efg_dir) + rec
    const double *efg_dir;
    const double *qself;     // self terms use q and mu whatever lq/ld (src/ewald.c:201-224)
    const double3 *muself;
};

template <bool WF, bool WEFG>
__global__ void __launch_bounds__(ION_THREADS) k_rec_ion(IonArgs a) {
    extern __shared__ double2 rk[];
    int i = blockIdx.x * ION_THREADS + threadIdx.x;
    bool act = i < a.n;
    double3 t = make_double3(0, 0, 0), m = make_double3(0, 0, 0);
    double qi = 0.0;
    if (act) {
        double4 ri = a.r[i];
        t = phase_coord(a.c, ri.x, ri.y, ri.z);
        qi = a.q ? a.q[i] : 0.0;
        if (WF && a.ld) {
            double3 mu = a.mu[i];
            m = phase_coord(a.c, mu.x, mu.y, mu.z);
        }
    }
    double2 e1 = cis2pi(t.y), e2 = cis2pi(t.z);
    double2 e2m = cis2pi(-(double)a.K2 * t.z);
    double S0 = 0, S1 = 0, S2 = 0;              // sum n recarg
    double P0 = 0, P1 = 0, P2 = 0;              // sum n (n.m) recarg2
    double H[6] = {0, 0, 0, 0, 0, 0};           // sum n n^T recarg2
    double2 base = make_double2(1.0, 0.0);
    int cur_nx = -1, last_ny = 0;
    for (int tl = 0; tl < a.ntile; tl++) {
        int r0 = a.tile_row[tl], r1 = a.tile_row[tl + 1];
        int k0 = a.tile_k[tl], k1 = a.tile_k[tl + 1];
        for (int k = k0 + threadIdx.x; k < k1; k += ION_THREADS) rk[k - k0] = a.rho_s[k];
        __syncthreads();
        for (int rr = r0; rr < r1; rr++) {
            KRow R = a.row[rr];
            if (R.nx != cur_nx) {
                cur_nx = R.nx;
                base = cis2pi((double)R.nx * t.x + (double)R.ny * t.y);
            } else {
                for (int s = last_ny; s < R.ny; s++) base = cmul(base, e1);
            }
            last_ny = R.ny;
            double2 ph = (R.z0 == 1) ? cmul(base, e2) : cmul(base, e2m);
            const double2 *rho = rk + (R.koff - k0);
            double R1 = 0, Rz = 0, T1 = 0, Tz = 0, Q0 = 0, Q1 = 0, Q2 = 0;
            double z = (double)R.z0;
            double c0 = (double)R.nx * m.x + (double)R.ny * m.y;
            for (int kz = 0; kz < R.cnt; kz++) {
                double2 rh = rho[kz];
                double recarg = rh.y * ph.x - rh.x * ph.y;
                R1 += recarg;
                Rz += z * recarg;
                if (WF || WEFG) {
                    double recarg2 = rh.x * ph.x + rh.y * ph.y;
                    if (WF) {
                        double tq = (c0 + z * m.z) * recarg2;
                        T1 += tq;
                        Tz += z * tq;
                    }
                    if (WEFG) {
                        Q0 += recarg2;
                        Q1 += z * recarg2;
                        Q2 += z * z * recarg2;
                    }
                }
                ph = cmul(ph, e2);
                z += 1.0;
            }
            double nx = (double)R.nx, ny = (double)R.ny;
            S0 += nx * R1;
            S1 += ny * R1;
            S2 += Rz;
            if (WF) {
                P0 += nx * T1;
                P1 += ny * T1;
                P2 += Tz;
            }
            if (WEFG) {
                H[0] += nx * nx * Q0;
                H[1] += nx * ny * Q0;
                H[2] += nx * Q1;
                H[3] += ny * ny * Q0;
                H[4] += ny * Q1;
                H[5] += Q2;
            }
        }
        __syncthreads();
    }
    if (!act) return;
    const Cell &c = a.c;
    const double tpi = TPI_D;
    // B S: sum_k k recarg = 2 pi B S
    double gS[3], gP[3];
    for (int q = 0; q < 3; q++) {
        gS[q] = tpi * (c.B[q][0] * S0 + c.B[q][1] * S1 + c.B[q][2] * S2);
        gP[q] = tpi * tpi * (c.B[q][0] * P0 + c.B[q][1] * P1 + c.B[q][2] * P2);
    }
    if (a.want_ef) {
        double3 mu = a.muself ? a.muself[i] : make_double3(0, 0, 0);
        double3 base_e = make_double3(a.self2 * mu.x, a.self2 * mu.y, a.self2 * mu.z);
        if (a.ef_dir) {
            double3 d = a.ef_dir[i];
            base_e.x += d.x;
            base_e.y += d.y;
            base_e.z += d.z;
        }
        a.ef[i] = make_double3(base_e.x + (-a.tfpiV * gS[0]), base_e.y + (-a.tfpiV * gS[1]),
                               base_e.z + (-a.tfpiV * gS[2]));
    }
    if (WF && a.want_f) {
        double3 fo = a.f[i];
        if (a.f_dir) {
            double3 d = a.f_dir[i];
            fo.x += d.x * a.coul;
            fo.y += d.y * a.coul;
            fo.z += d.z * a.coul;
        }
        double fr[3];
        for (int q = 0; q < 3; q++) fr[q] = a.tfpiV * (-qi * gS[q] + (a.ld ? gP[q] : 0.0));
        a.f[i] = make_double3(fo.x + fr[0] * a.coul, fo.y + fr[1] * a.coul, fo.z + fr[2] * a.coul);
    }
    if (WEFG && a.want_efg) {
        // (2 pi)^2 B H B^T, upper triangle only as in src/ewald.c:977-984
        double Hm[3][3] = {{H[0], H[1], H[2]}, {H[1], H[3], H[4]}, {H[2], H[4], H[5]}};
        double BH[3][3];
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++)
                BH[p][q] = c.B[p][0] * Hm[0][q] + c.B[p][1] * Hm[1][q] + c.B[p][2] * Hm[2][q];
        for (int p = 0; p < 3; p++)
            for (int q = 0; q < 3; q++) {
                double v = 0.0;
                if (q >= p)
                    v = a.tfpiV * tpi * tpi * (BH[p][0] * c.B[q][0] + BH[p][1] * c.B[q][1] + BH[p][2] * c.B[q][2]);
                double b0 = (p == q && a.qself) ? -a.self2 * a.qself[i] : 0.0;
                if (a.efg_dir) b0 += a.efg_dir[(size_t)i * 9 + 3 * p + q];
                a.efg[(size_t)i * 9 + 3 * p + q] = b0 + v;
            }
    }
}

// ---------------------------------------------------------------- launcher
// rho pass + reduction + ion pass.  `o` says where the per-ion results go:
//   o.ef  = self2*mu + o.ef_dir + E_rec          (when o.ef)
//   o.f   = o.f + o.f_dir*coul + F_rec*coul      (when o.f)
//   o.efg = self + o.efg_dir + EFG_rec (upper)   (when o.efg)
// Algorithmic flops per (ion, k) pair, counted from the loop bodies (FMA = 2 flops):
//   k_rho     : phase b*E2 6, charge term 4, dipole term (k.mu 2 + 4) 6
//   k_rec_ion : phase recurrence 6, recarg 3, R sums 3, z += 1 1           (field: 13)
//               + recarg2 3, (n.m) recarg2 3, P sums 3                      (force: 22)
//               + Q sums 7                                                  (EFG:   29)
double rho_flops_per_pair(bool lq, bool ld) { return (lq ? 4.0 : 0.0) + (ld ? 6.0 : 0.0) + 6.0; }
double ion_flops_per_pair(bool f, bool efg) { return 13.0 + (f ? 9.0 : 0.0) + (efg ? 7.0 : 0.0); }

template <typename K>
static void allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) MDFF_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

void launch_rec(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const RecOut &o) {
    int segblocks = ceil_div(e.nseg, RHO_THREADS);
    dim3 grid(segblocks, e.rho_chunks);
    int WT = (e.kmax[0] + 1) + (2 * e.kmax[1] + 1) + (2 * e.kmax[2] + 1);
    size_t smem = sizeof(double2) * RHO_TI * WT + sizeof(double) * RHO_TI * 4;
    int ps = -1;
    e.prof_begin("k_rho", &ps);
    if (lq && ld) {
        allow_smem(k_rho<true, true>, smem);
        MDFF_LAUNCH(e, (k_rho<true, true>), grid, RHO_THREADS, smem, e.n, e.rho_chunk, e.cell, e.kmax[0], e.kmax[1],
                    e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    } else if (lq) {
        allow_smem(k_rho<true, false>, smem);
        MDFF_LAUNCH(e, (k_rho<true, false>), grid, RHO_THREADS, smem, e.n, e.rho_chunk, e.cell, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    } else if (ld) {
        allow_smem(k_rho<false, true>, smem);
        MDFF_LAUNCH(e, (k_rho<false, true>), grid, RHO_THREADS, smem, e.n, e.rho_chunk, e.cell, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    } else {
        MDFF_CK(cudaMemsetAsync(e.d_rho_part, 0, sizeof(double2) * (size_t)e.nk * e.rho_chunks, e.stream));
    }
    e.prof_end("k_rho", ps, (lq || ld) ? rho_flops_per_pair(lq, ld) * (double)e.n * e.nk : 0.0);
    int nbr = ceil_div(e.nk, 256);
    MDFF_LAUNCH(e, k_rho_reduce, nbr, 256, 0, e.nk, e.rho_chunks, e.d_rho_part, e.d_Ak, e.d_kcoe, e.d_kvec,
                e.d_rho, e.d_part, (int)S_REC_U, e.part_stride);
    e.reduce(S_REC_U, 7, nbr);

    IonArgs a;
    a.n = e.n;
    a.K0 = e.kmax[0];
    a.K1 = e.kmax[1];
    a.K2 = e.kmax[2];
    a.c = e.cell;
    a.r = e.d_r;
    a.q = lq ? q : nullptr;
    a.mu = mu;
    a.row = e.d_row;
    a.tile_row = e.d_tile_row;
    a.tile_k = e.d_tile_k;
    a.ntile = e.ntile;
    a.rho_s = e.d_rho;
    a.tfpiV = 2.0 * 2.0 * TPI_D * e.cell.inveOmega;
    a.self2 = o.self2;
    a.qself = o.self_q;
    a.muself = o.self_mu;
    a.ld = ld;
    a.want_ef = o.ef != nullptr;
    a.want_f = o.f != nullptr;
    a.want_efg = o.efg != nullptr;
    a.ef_dir = o.ef_dir;
    a.ef = o.ef;
    a.coul = o.coul;
    a.f_dir = o.f_dir;
    a.f = o.f;
    a.efg = o.efg;
    a.efg_dir = o.efg_dir;
    if (!a.want_ef && !a.want_f && !a.want_efg) return;
    size_t smem2 = sizeof(double2) * e.tile_kmax;
    int nb = ceil_div(e.n, ION_THREADS);
    int pi = -1;
    e.prof_begin("k_rec_ion", &pi);
    if (a.want_efg)
        MDFF_LAUNCH(e, (k_rec_ion<true, true>), nb, ION_THREADS, smem2, a);
    else if (a.want_f)
        MDFF_LAUNCH(e, (k_rec_ion<true, false>), nb, ION_THREADS, smem2, a);
    else
        MDFF_LAUNCH(e, (k_rec_ion<false, false>), nb, ION_THREADS, smem2, a);
    e.prof_end("k_rec_ion", pi, ion_flops_per_pair(a.want_f || a.want_efg, a.want_efg) * (double)e.n * e.nk);
}

}  // namespace mdffgpu
