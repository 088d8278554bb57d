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
//               in tiles; per-ion-chunk partial sums, reduced in a fixed order.  With
//               b = E0[nx] E1[ny] and k.mu = c0 + nz c1 the summand is
//               (B1 + nz B2) E2[nz], B1 = (q + i c0) b, B2 = i c1 b: 6 FP64 ops per k.
//   k_rec_ion : per (ion, k-slice) the k sums for field, force and EFG; threads own
//               ions, blockIdx.y a row-aligned slice of k whose Ak*rho(k) sits in
//               shared memory; two independent phase recurrences (even and odd nz);
//               sums kept in n-space, combined over slices and mapped to Cartesian k
//               once per ion by k_rec_combine.
#include "engine.cuh"

namespace mdffgpu {

constexpr int RHO_THREADS = 128;
constexpr int RHO_TI = 32;          // ions per shared-memory tile
constexpr int ION_THREADS = 128;
constexpr int ION_NV = 12;          // per (ion, slice) partial sums: S[3] P[3] H[6]

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
__global__ void __launch_bounds__(RHO_THREADS, RHO_MIN_BLOCKS) k_rho(int n, int chunk, Cell c, int K0, int K1, int K2,
                                                    const double4 *__restrict__ r, const double *__restrict__ q,
                                                    const double3 *__restrict__ mu, int nseg,
                                                    const KSeg *__restrict__ seg, double2 *__restrict__ part,
                                                    int nk, const int *__restrict__ idx) {
    grid_dep();
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
                int ia = idx ? idx[t0 + slot] : t0 + slot;   // ion subset: q, mu vanish elsewhere
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
                        ms[3 * slot] = tpi * mm.x;
                        ms[3 * slot + 1] = tpi * mm.y;
                        ms[3 * slot + 2] = tpi * mm.z;
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
                // B1 = (q + i c0) b, B2 = i c1 b; summand (B1 + nz B2) E2[nz]
                double qa = LQ ? qs[a] : 0.0;
                double c0 = 0.0, c1 = 0.0;
                if (LD) {
                    c0 = (double)S.nx * ms[3 * a] + (double)S.ny * ms[3 * a + 1];
                    c1 = ms[3 * a + 2];
                }
                double2 B1 = make_double2(qa * b.x - c0 * b.y, qa * b.y + c0 * b.x);
                double2 B2 = make_double2(-c1 * b.y, c1 * b.x);
                double zf = (double)S.z0;
#pragma unroll
                for (int z = 0; z < KSEG; z++) {
                    if (z < S.cnt) {
                        double2 C = B1;
                        if (LD) {
                            C.x = B1.x + (zf + (double)z) * B2.x;
                            C.y = B1.y + (zf + (double)z) * B2.y;
                        }
                        double2 e = Z[z];
                        acc[z].x += C.x * e.x - C.y * e.y;
                        acc[z].y += C.x * e.y + C.y * e.x;
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

// one warp, one k per lane: store Ak*rho(k); warp partials of u_rec = sum Ak|rho|^2 and
// of the k-space virial (src/ewald.c:945-1006) into ppart[slot..slot+6][blockIdx.x]
__device__ __forceinline__ void rho_finish(int k, int nk, double2 rho, const double *__restrict__ Ak,
                                           const double *__restrict__ kcoe, const double3 *__restrict__ kv,
                                           double2 *__restrict__ rho_s, double *__restrict__ ppart, int slot,
                                           int stride) {
    int l = threadIdx.x & 31;
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    if (k < nk) {
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
#pragma unroll
    for (int q = 0; q < 7; q++) v[q] = warp_sum(v[q]);
    if (l < 7) {
        double a = v[0];
#pragma unroll
        for (int q = 1; q < 7; q++)
            if (l == q) a = v[q];
        ppart[(size_t)(slot + l) * stride + blockIdx.x] = a;
    }
}

// sum the ion-chunk partials of rho(k) in a fixed order, then rho_finish. A block owns
// RHOR_K consecutive k (one per lane); its 8 warps take every 8th chunk and warp 0 adds
// the 8 warp sums in warp order. rho_raw (optional) receives rho(k) itself.  Partials
// are FP64 (kspace.cu) or FP32 (kspace32.cu: sums over one chunk of ions), added in FP64.
template <typename PT>
__global__ void __launch_bounds__(256) k_rho_reduce(int nk, int nchunks, const PT *__restrict__ part,
                                                    const double *__restrict__ Ak, const double *__restrict__ kcoe,
                                                    const double3 *__restrict__ kv, double2 *__restrict__ rho_s,
                                                    double2 *__restrict__ rho_raw, double *__restrict__ ppart,
                                                    int slot, int stride) {
    grid_dep();
    __shared__ double2 ws[8][RHOR_K];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int k = blockIdx.x * RHOR_K + l;
    // chunks w, w + 8, ...: four loads in flight into four accumulators (fixed order)
    double2 a0 = make_double2(0.0, 0.0), a1 = a0, a2 = a0, a3 = a0;
    if (k < nk) {
        int c = w;
        for (; c + 24 < nchunks; c += 32) {
            PT p0 = part[(size_t)c * nk + k], p1 = part[(size_t)(c + 8) * nk + k];
            PT p2 = part[(size_t)(c + 16) * nk + k], p3 = part[(size_t)(c + 24) * nk + k];
            a0.x += (double)p0.x, a0.y += (double)p0.y;
            a1.x += (double)p1.x, a1.y += (double)p1.y;
            a2.x += (double)p2.x, a2.y += (double)p2.y;
            a3.x += (double)p3.x, a3.y += (double)p3.y;
        }
        for (; c < nchunks; c += 8) {
            PT p = part[(size_t)c * nk + k];
            a0.x += (double)p.x, a0.y += (double)p.y;
        }
    }
    double2 acc = make_double2((a0.x + a1.x) + (a2.x + a3.x), (a0.y + a1.y) + (a2.y + a3.y));
    ws[w][l] = acc;
    __syncthreads();
    if (w) return;
    double2 rho = ws[0][l];
#pragma unroll
    for (int q = 1; q < 8; q++) {
        rho.x += ws[q][l].x;
        rho.y += ws[q][l].y;
    }
    if (rho_raw && k < nk) rho_raw[k] = rho;
    rho_finish(k, nk, rho, Ak, kcoe, kv, rho_s, ppart, slot, stride);
}

// rho_finish on a rho(k) assembled elsewhere (one warp per RHOR_K k)
__global__ void __launch_bounds__(32) k_rho_from_acc(int nk, const double2 *__restrict__ acc,
                                                     const double *__restrict__ Ak, const double *__restrict__ kcoe,
                                                     const double3 *__restrict__ kv, double2 *__restrict__ rho_s,
                                                     double *__restrict__ ppart, int slot, int stride) {
    grid_dep();
    int k = blockIdx.x * RHOR_K + threadIdx.x;
    double2 rho = k < nk ? acc[k] : make_double2(0.0, 0.0);
    rho_finish(k, nk, rho, Ak, kcoe, kv, rho_s, ppart, slot, stride);
}

// ---------------------------------------------------------------- pass 2: per ion
struct IonArgs {
    int n, K0, K1, K2;      // n: ions in the pass (idx[n] when idx is set)
    const int *idx;         // output ions (null: 0..n-1); partials are indexed by position in idx
    Cell c;
    const double4 *r;
    const double *q;
    const double3 *mu;
    const KRow *row;
    const int *tile_row, *tile_k;
    int ntile;
    const double2 *rho_s;
    double *part;           // [ntile][n][ION_NV]
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

// one slice of rows: S = sum_k n recarg, P = sum_k n (n.m) recarg2, H = sum_k n n^T recarg2
template <bool WF, bool WEFG>
__global__ void __launch_bounds__(ION_THREADS) k_rec_ion(IonArgs a) {
    grid_dep();
    extern __shared__ double2 rk[];
    int ii = blockIdx.x * ION_THREADS + threadIdx.x;
    int tl = blockIdx.y;
    bool act = ii < a.n;
    int i = act ? (a.idx ? a.idx[ii] : ii) : 0;
    int r0 = a.tile_row[tl], r1 = a.tile_row[tl + 1];
    int k0 = a.tile_k[tl], k1 = a.tile_k[tl + 1];
    for (int k = k0 + threadIdx.x; k < k1; k += ION_THREADS) rk[k - k0] = a.rho_s[k];
    double3 t = make_double3(0, 0, 0), m = make_double3(0, 0, 0);
    if (act) {
        double4 ri = a.r[i];
        t = phase_coord(a.c, ri.x, ri.y, ri.z);
        if (WF && a.ld) {
            double3 mu = a.mu[i];
            m = phase_coord(a.c, mu.x, mu.y, mu.z);
        }
    }
    __syncthreads();
    double2 e1 = cis2pi(t.y), e2 = cis2pi(t.z);
    double2 e22 = cmul(e2, e2);
    double2 e2m = cis2pi(-(double)a.K2 * t.z);
    double S0 = 0, S1 = 0, S2 = 0, P0 = 0, P1 = 0, P2 = 0;
    double H[6] = {0, 0, 0, 0, 0, 0};
    double2 base = make_double2(1.0, 0.0);
    int cur_nx = -1, last_ny = 0;
    for (int rr = r0; rr < r1; rr++) {
        KRow R = a.row[rr];
        if (R.nx != cur_nx) {
            cur_nx = R.nx;
            base = cis2pi((double)R.nx * t.x + (double)R.ny * t.y);
        } else {
            for (int s = last_ny; s < R.ny; s++) base = cmul(base, e1);
        }
        last_ny = R.ny;
        // two independent chains: even offsets from ph0, odd from ph1, both stepping e2^2
        double2 ph0 = (R.z0 == 1) ? cmul(base, e2) : cmul(base, e2m);
        double2 ph1 = cmul(ph0, e2);
        const double2 *rho = rk + (R.koff - k0);
        double R1a = 0, Rza = 0, T1a = 0, Tza = 0, Q0a = 0, Q1a = 0, Q2a = 0;
        double R1b = 0, Rzb = 0, T1b = 0, Tzb = 0, Q0b = 0, Q1b = 0, Q2b = 0;
        double za = (double)R.z0, zb = za + 1.0;
        double c0 = (double)R.nx * m.x + (double)R.ny * m.y;
        int cnt = R.cnt;
        for (int kz = 0; kz < cnt; kz += 2) {
            double2 ra = rho[kz];
            double rca = ra.y * ph0.x - ra.x * ph0.y;
            R1a += rca;
            Rza += za * rca;
            if (WF || WEFG) {
                double rc2 = ra.x * ph0.x + ra.y * ph0.y;
                if (WF) {
                    double tq = (c0 + za * m.z) * rc2;
                    T1a += tq;
                    Tza += za * tq;
                }
                if (WEFG) {
                    Q0a += rc2;
                    Q1a += za * rc2;
                    Q2a += za * za * rc2;
                }
            }
            if (kz + 1 < cnt) {
                double2 rb = rho[kz + 1];
                double rcb = rb.y * ph1.x - rb.x * ph1.y;
                R1b += rcb;
                Rzb += zb * rcb;
                if (WF || WEFG) {
                    double rc2 = rb.x * ph1.x + rb.y * ph1.y;
                    if (WF) {
                        double tq = (c0 + zb * m.z) * rc2;
                        T1b += tq;
                        Tzb += zb * tq;
                    }
                    if (WEFG) {
                        Q0b += rc2;
                        Q1b += zb * rc2;
                        Q2b += zb * zb * rc2;
                    }
                }
            }
            ph0 = cmul(ph0, e22);
            ph1 = cmul(ph1, e22);
            za += 2.0;
            zb += 2.0;
        }
        double nx = (double)R.nx, ny = (double)R.ny;
        double R1 = R1a + R1b, Rz = Rza + Rzb;
        S0 += nx * R1;
        S1 += ny * R1;
        S2 += Rz;
        if (WF) {
            double T1 = T1a + T1b, Tz = Tza + Tzb;
            P0 += nx * T1;
            P1 += ny * T1;
            P2 += Tz;
        }
        if (WEFG) {
            double Q0 = Q0a + Q0b, Q1 = Q1a + Q1b, Q2 = Q2a + Q2b;
            H[0] += nx * nx * Q0;
            H[1] += nx * ny * Q0;
            H[2] += nx * Q1;
            H[3] += ny * ny * Q0;
            H[4] += ny * Q1;
            H[5] += Q2;
        }
    }
    if (!act) return;
    double *o = a.part + ((size_t)tl * a.n + ii) * ION_NV;
    o[0] = S0;
    o[1] = S1;
    o[2] = S2;
    if (WF) {
        o[3] = P0;
        o[4] = P1;
        o[5] = P2;
    }
    if (WEFG)
        for (int k = 0; k < 6; k++) o[6 + k] = H[k];
}

// sum the slices of each ion (fixed order) and write field, force and EFG
template <bool WF, bool WEFG>
__global__ void k_rec_combine(IonArgs a) {
    grid_dep();
    int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= a.n) return;
    int i = a.idx ? a.idx[ii] : ii;
    double S0 = 0, S1 = 0, S2 = 0, P0 = 0, P1 = 0, P2 = 0, H[6] = {0, 0, 0, 0, 0, 0};
    for (int tl = 0; tl < a.ntile; tl++) {
        const double *o = a.part + ((size_t)tl * a.n + ii) * ION_NV;
        S0 += o[0];
        S1 += o[1];
        S2 += o[2];
        if (WF) {
            P0 += o[3];
            P1 += o[4];
            P2 += o[5];
        }
        if (WEFG)
            for (int k = 0; k < 6; k++) H[k] += o[6 + k];
    }
    const Cell &c = a.c;
    const double tpi = TPI_D;
    double qi = a.q ? a.q[i] : 0.0;
    // sum_k k recarg = 2 pi B S ; sum_k k (k.mu) recarg2 = (2 pi)^2 B P
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
// Algorithmic flops per (ion, k) pair, counted from the loop bodies (FMA = 2 flops):
//   k_rho     : (B1 + nz B2) 4 when dipoles, complex multiply-accumulate 8
//   k_rec_ion : phase recurrence 6, recarg 3, R sums 4                     (field: 13)
//               + recarg2 3, (c0 + nz m) recarg2 3, T sums 4                (force: 23)
//               + Q sums 7                                                  (EFG:   30)
double rho_flops_per_pair(bool lq, bool ld) { return 8.0 + (ld ? 4.0 : 0.0) + (lq ? 0.0 : 0.0); }
double ion_flops_per_pair(bool f, bool efg) { return 13.0 + (f ? 10.0 : 0.0) + (efg ? 7.0 : 0.0); }

template <typename K>
static void allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        MDFF_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// rho pass + reduction + ion pass.  `o` says where the per-ion results go:
//   o.ef  = self2*mu + o.ef_dir + E_rec          (when o.ef)
//   o.f   = o.f + o.f_dir*coul + F_rec*coul      (when o.f)
//   o.efg = self + o.efg_dir + EFG_rec (upper)   (when o.efg)
// mixed precision: kspace32.cu passes, FP64 reduction of the FP32 chunk partials
static void launch_rec32(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const RecOut &o) {
    int nbr = ceil_div(e.nk, RHOR_K);
    int cnt = o.idx ? o.cnt : e.n;
    if (o.rho_acc) {
        MDFF_LAUNCH(e, k_rho_from_acc, nbr, 32, 0, e.nk, o.rho_acc, e.d_Ak, e.d_kcoe, e.d_kvec, e.d_rho, e.d_part,
                    (int)S_REC_U, e.part_stride);
    } else {
        launch_rho32(e, q, mu, lq, ld, o.idx, cnt);
        MDFF_LAUNCH(e, k_rho_reduce<float2>, nbr, 256, 0, e.nk, e.rho_chunks_used, e.d_rho_part32, e.d_Ak, e.d_kcoe,
                    e.d_kvec, e.d_rho, o.rho_raw, e.d_part, (int)S_REC_U, e.part_stride);
    }
    if (o.energy) e.reduce(S_REC_U, 7, nbr);
    if (!o.ef && !o.f) return;
    if (o.out_idx) launch_ion32(e, lq ? q : nullptr, mu, ld, o, o.out_idx, o.out_cnt);
    else launch_ion32(e, lq ? q : nullptr, mu, ld, o, o.idx, cnt);
}

void launch_rec(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const RecOut &o) {
    // FP32 passes in mixed precision (no FP32 EFG: EFG requests run in FP64)
    if (e.use32 && e.rec32 && o.efg == nullptr) {
        launch_rec32(e, q, mu, lq, ld, o);
        return;
    }
    // ion subsets: the rho pass sums over o.idx (all ions when null; q and mu vanish
    // elsewhere), the ion pass writes at o.out_idx, else at o.idx, else at every ion
    const int *rho_idx = o.idx;
    int rho_n = o.idx ? o.cnt : e.n;
    const int *out_idx = o.out_idx ? o.out_idx : o.idx;
    int out_n = o.out_idx ? o.out_cnt : (o.idx ? o.cnt : e.n);
    int chunk = std::max(1, ceil_div(rho_n, e.rho_chunks));   // the same chunk count, shorter chunks
    int segblocks = ceil_div(e.nseg, RHO_THREADS);
    dim3 grid(segblocks, e.rho_chunks);
    int WT = (e.kmax[0] + 1) + (2 * e.kmax[1] + 1) + (2 * e.kmax[2] + 1);
    size_t smem = sizeof(double2) * RHO_TI * WT + sizeof(double) * RHO_TI * 4;
    int ps = -1;
    int nbr = ceil_div(e.nk, RHOR_K);
    if (o.rho_acc) {   // rho(k) already known (linear in q and mu): no ion x k pass
        MDFF_LAUNCH(e, k_rho_from_acc, nbr, 32, 0, e.nk, o.rho_acc, e.d_Ak, e.d_kcoe, e.d_kvec, e.d_rho, e.d_part,
                    (int)S_REC_U, e.part_stride);
        e.reduce(S_REC_U, 7, nbr);
    }
    if (!o.rho_acc) e.prof_begin("k_rho", &ps);
    if (o.rho_acc) {
    } else if (lq && ld) {
        allow_smem(k_rho<true, true>, smem);
        MDFF_LAUNCH(e, (k_rho<true, true>), grid, RHO_THREADS, smem, rho_n, chunk, e.cell, e.kmax[0], e.kmax[1],
                    e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk, rho_idx);
    } else if (lq) {
        allow_smem(k_rho<true, false>, smem);
        MDFF_LAUNCH(e, (k_rho<true, false>), grid, RHO_THREADS, smem, rho_n, chunk, e.cell, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk, rho_idx);
    } else if (ld) {
        allow_smem(k_rho<false, true>, smem);
        MDFF_LAUNCH(e, (k_rho<false, true>), grid, RHO_THREADS, smem, rho_n, chunk, e.cell, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_r, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk, rho_idx);
    } else {
        MDFF_CK(cudaMemsetAsync(e.d_rho_part, 0, sizeof(double2) * (size_t)e.nk * e.rho_chunks, e.stream));
    }
    if (!o.rho_acc) {
        e.prof_end("k_rho", ps, (lq || ld) ? rho_flops_per_pair(lq, ld) * (double)rho_n * e.nk : 0.0);
        MDFF_LAUNCH(e, k_rho_reduce<double2>, nbr, 256, 0, e.nk, e.rho_chunks, e.d_rho_part, e.d_Ak, e.d_kcoe, e.d_kvec,
                    e.d_rho, o.rho_raw, e.d_part, (int)S_REC_U, e.part_stride);
        e.reduce(S_REC_U, 7, nbr);
    }

    IonArgs a;
    a.n = out_n;
    a.idx = out_idx;
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
    a.part = e.d_ion_part;
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
    dim3 g2(ceil_div(out_n, ION_THREADS), e.ntile);
    int nb = ceil_div(out_n, 256);
    int pi = -1;
    e.prof_begin("k_rec_ion", &pi);
    if (a.want_efg)
        MDFF_LAUNCH(e, (k_rec_ion<true, true>), g2, ION_THREADS, smem2, a);
    else if (a.want_f)
        MDFF_LAUNCH(e, (k_rec_ion<true, false>), g2, ION_THREADS, smem2, a);
    else
        MDFF_LAUNCH(e, (k_rec_ion<false, false>), g2, ION_THREADS, smem2, a);
    e.prof_end("k_rec_ion", pi, ion_flops_per_pair(a.want_f || a.want_efg, a.want_efg) * (double)out_n * e.nk);
    if (a.want_efg)
        MDFF_LAUNCH(e, (k_rec_combine<true, true>), nb, 256, 0, a);
    else if (a.want_f)
        MDFF_LAUNCH(e, (k_rec_combine<true, false>), nb, 256, 0, a);
    else
        MDFF_LAUNCH(e, (k_rec_combine<false, false>), nb, 256, 0, a);
}

}  // namespace mdffgpu
