// Reciprocal-space Ewald sum in mixed precision (MDFFGPU_MIXED): the sums of kspace.cu
// with FP32 arithmetic per (ion, k) and FP64 wherever a sum spans many terms.
//
// Phase tables.  With k = 2 pi B n the phase of ion i factorises into
// E0[nx] E1[ny] E2[nz], E_d[m] = exp(2 pi i m t_d), t = B^T r (kspace.cu).  k_phase32
// writes, once per force evaluation (positions are fixed through the induced-dipole
// solve), one row of FP32 complex values per ion:
//     [ E0[0..K0] | E1[-K1..K1] | pad | Z blocks of ZB values of E2, stride ZS ]
// every entry from its own FP64-reduced argument m t_d - rint(m t_d) (no recurrence,
// so each value carries one rounding).  The z range of a k-row is cut into blocks of
// ZB consecutive nz (negative half -K2..0 and positive half 1..K2 separately, zero
// padded), so that a thread owns one block of one row and reads it with 16-byte loads;
// the two extra entries per block put neighbouring blocks in different shared-memory
// banks (the lanes of a warp read two blocks of the same ion at once).  Within a block
// the values are stored as planar pairs, (Re E2[z], Re E2[z+1]) then (Im E2[z],
// Im E2[z+1]), the operand layout of the packed FP32x2 FMA (FFMA2) of k_rho32.
//
// k_rho32   : rho(k) = sum_i (q_i + i k.mu_i) E0 E1 E2.  Thread = one segment (a row
//             and RZP values of |nz|, both signs: E2[-nz] = conj E2[nz]); ions stream
//             through shared memory in tiles of table rows; eight weighted sums per
//             |nz| give rho(+nz) and rho(-nz), 4 FMA per k-vector (2 without dipoles),
//             issued as packed FP32x2 FMAs over pairs of |nz|.  FP32 sums over one
//             block's ion chunk, chunk partials summed in FP64 in a fixed order
//             (k_rho_reduce32).
// k_ion32   : per ion and k-slice the n-space sums of field (and force) terms.  Thread
//             = ion; per row the block stages the weights of Ak rho(+z) and Ak rho(-z)
//             folded over the sign of nz, E2[z] (z = 1..KZ) sits in registers, the row
//             sums cost 4 FMA per k-vector (6 with forces) and one product with the row
//             phase exp(2 pi i (nx tx + ny ty)), from an FP64-reduced argument every
//             ION32_RUN rows and by FP32 steps in ny between.  Row sums FP32, rows FP64.
// Both passes take an optional ion index list (the polarisable ions of an induced-
// dipole iteration, whose search directions vanish elsewhere).
#include "engine.cuh"

namespace mdffgpu {

constexpr int ZB = 16;              // nz per segment block (two complex per 16-byte load)
constexpr int ZS = ZB + 2;          // block stride: consecutive blocks start 4 banks apart
constexpr int RZP = 8;              // |nz| values per rho segment (each for +nz and -nz)
constexpr int RHO32_THREADS = 128;
constexpr int RHO32_TI = 32;        // ions per shared-memory tile (two tiles in flight)
constexpr int RHO32_MIN_BLOCKS = 5;
constexpr int ION32_THREADS = 128;
constexpr int ION32_MIN_BLOCKS = 5;
constexpr int ION32X2_MIN_BLOCKS = 4;   // field-only ion pass, two ions per thread
constexpr int ION32_RUN = 4;        // rows per exact row phase in the ion pass

// asynchronous global -> shared copy of 16 bytes (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------- phase tables
struct TabLayout {
    int K0, K1, K2, nzb_neg, nzb, e1, z, w;   // offsets in float2 units
};

// one thread per (ion, table entry)
__global__ void k_phase32(int n, Cell c, const double4 *__restrict__ r, TabLayout L, float2 *__restrict__ tab) {
    grid_dep();
    // one ion per warp row (threadIdx.y), its entries over the lanes
    const int i = blockIdx.x * blockDim.y + threadIdx.y;
    if (i >= n) return;
    const double4 ri = r[i];
    for (int e = threadIdx.x; e < L.w; e += blockDim.x) {
        const size_t g = (size_t)i * L.w + e;
        int d = -1, m = 0;
        if (e < L.K0 + 1) {
            d = 0;
            m = e;
        } else if (e < L.e1 + 2 * L.K1 + 1) {
            d = 1;
            m = e - L.e1 - L.K1;
        } else if (e >= L.z) {
            // z blocks hold planar pairs: entry 2p = (x of z_2p, x of z_2p+1), entry 2p + 1 =
            // their y; the thread of entry 2p writes both
            int b = (e - L.z) / ZS, j = (e - L.z) - b * ZS;
            if (j >= ZB) {
                tab[g] = make_float2(0.f, 0.f);
                continue;
            }
            if (j & 1) continue;
            int m0 = (b < L.nzb_neg) ? -L.K2 + ZB * b + j : 1 + ZB * (b - L.nzb_neg) + j;
            bool ok0 = (b < L.nzb_neg) ? m0 <= 0 : m0 <= L.K2, ok1 = (b < L.nzb_neg) ? m0 + 1 <= 0 : m0 + 1 <= L.K2;
            double t = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
            float2 v0 = ok0 ? cis2pi32((double)m0 * t) : make_float2(0.f, 0.f);
            float2 v1 = ok1 ? cis2pi32((double)(m0 + 1) * t) : make_float2(0.f, 0.f);
            *(float4 *)(tab + g) = make_float4(v0.x, v1.x, v0.y, v1.y);
            continue;
        }
        float2 v = make_float2(0.f, 0.f);
        if (d >= 0) {
            double t = c.B[0][d] * ri.x + c.B[1][d] * ri.y + c.B[2][d] * ri.z;
            v = cis2pi32((double)m * t);
        }
        tab[g] = v;
    }
}

// ---------------------------------------------------------------- pass 1: rho(k)
// The summand of k = (nx, ny, nz) is (B1 + nz B2) E2[nz] with B1 = (q + i c0) b,
// B2 = i c1 b, b = E0[nx] E1[ny], c0 = 2 pi (nx m0 + ny m1), c1 = 2 pi m2 (m = B^T mu).
// E2[-z] = conj E2[z], so with E2[z] = (c, d) the sums over ions of the eight products
//     Sa = B1x c, Sb = B1y d, Sc = B1x d, Sd = B1y c,  Ta..Td the same with B2
// give both rho(+z) and rho(-z):
//     rho(+z) = (Sa - Sb + z (Ta - Tb),  Sc + Sd + z (Tc + Td))
//     rho(-z) = (Sa + Sb - z (Ta + Tb),  Sd - Sc + z (Tc - Td))
// 4 FMA per k-vector (2 without dipoles), issued as packed FP32x2 FMAs over the z pairs
// of the table.  A thread owns one segment: a row (nx, ny) and RZP consecutive |nz|,
// both signs, plus nz = 0 in the segment that starts at |nz| = 1.  Only the E0, E1 and
// positive-z parts of a table row are staged in shared memory.
template <bool LQ, bool LD>
__global__ void __launch_bounds__(RHO32_THREADS, RHO32_MIN_BLOCKS)
    k_rho32(int cnt, const int *__restrict__ idx, int chunk, TabLayout L, const float2 *__restrict__ tab,
            Cell c, const double *__restrict__ q, const double3 *__restrict__ mu, int nseg,
            const KSeg *__restrict__ seg, float2 *__restrict__ part, int nk) {
    grid_dep();
    constexpr int NP = RZP / 2;
    extern __shared__ float4 sm4[];
    const int ha = L.z / 2, skip = (ZS / 2) * L.nzb_neg;   // 16-byte units
    const int hw = L.w / 2, cw = hw - skip;               // staged row: E0 E1 | z > 0 blocks
    // two stages: [2][RHO32_TI][cw] staged rows, then [2][RHO32_TI] (q, 2 pi m)
    float4 *QMs = sm4 + 2 * RHO32_TI * cw;
    int sid = blockIdx.x * RHO32_THREADS + threadIdx.x;
    KSeg S;
    if (sid < nseg) S = seg[sid];
    else S.nx = S.ny = S.z0 = S.cnt = S.koff = S.pad0 = S.pad1 = S.pad2 = 0;
    const float fnx = (float)S.nx, fny = (float)S.ny;
    const int o0 = S.nx, o1 = L.e1 + L.K1 + S.ny;
    float2 Sa[NP], Sb[NP], Sc[NP], Sd[NP], Ta[NP], Tb[NP], Tc[NP], Td[NP];
#pragma unroll
    for (int h = 0; h < NP; h++) Sa[h] = Sb[h] = Sc[h] = Sd[h] = Ta[h] = Tb[h] = Tc[h] = Td[h] = make_float2(0.f, 0.f);
    float2 acc0 = make_float2(0.f, 0.f);
    int a0 = blockIdx.y * chunk, a1 = min(cnt, a0 + chunk);
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double tpi = TPI_D;
    // staged rows of the tile at t0 into stage buffer `st` by asynchronous 16-byte copies
    // (warp w copies rows w, w+4, ...); every thread commits one group per tile
    auto issue = [&](int t0, int st) {
        int nt = min(RHO32_TI, a1 - t0);
        float4 *dst = sm4 + st * RHO32_TI * cw;
        for (int a = w; a < nt; a += RHO32_THREADS / 32) {
            int ion = idx ? idx[t0 + a] : t0 + a;
            const float4 *src = (const float4 *)(tab + (size_t)ion * L.w);
            for (int j = lane; j < cw; j += 32) cp_async16(dst + a * cw + j, src + (j < ha ? j : j + skip));
        }
        cp_async_commit();
    };
    int ntiles = a1 > a0 ? (a1 - a0 + RHO32_TI - 1) / RHO32_TI : 0;
    if (ntiles > 0) issue(a0, 0);
    for (int t = 0; t < ntiles; t++) {
        int t0 = a0 + t * RHO32_TI, nt = min(RHO32_TI, a1 - t0), st = t & 1;
        if (t + 1 < ntiles) {
            issue(t0 + RHO32_TI, st ^ 1);   // overlaps this tile's arithmetic
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        float4 *QM = QMs + st * RHO32_TI;
        if (threadIdx.x < nt) {
            int ion = idx ? idx[t0 + threadIdx.x] : t0 + threadIdx.x;
            float4 v = make_float4(LQ ? (float)q[ion] : 0.f, 0.f, 0.f, 0.f);
            if (LD) {
                double3 m3 = mu[ion];
                v.y = (float)(tpi * (c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z));
                v.z = (float)(tpi * (c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z));
                v.w = (float)(tpi * (c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z));
            }
            QM[threadIdx.x] = v;
        }
        __syncthreads();
        const float4 *cur = sm4 + st * RHO32_TI * cw;
        if (sid < nseg) {
            for (int a = 0; a < nt; a++) {
                const float2 *R = (const float2 *)(cur + a * cw);
                float2 b = cmul32(R[o0], R[o1]);
                float4 qm = QM[a];
                float2 B1, B2 = make_float2(0.f, 0.f);
                if (LD) {
                    float c0 = fnx * qm.y + fny * qm.z, c1 = qm.w;
                    B1 = LQ ? make_float2(qm.x * b.x - c0 * b.y, qm.x * b.y + c0 * b.x)
                            : make_float2(-c0 * b.y, c0 * b.x);
                    B2 = make_float2(-c1 * b.y, c1 * b.x);
                } else {
                    B1 = make_float2(qm.x * b.x, qm.x * b.y);
                }
                acc0.x += B1.x;
                acc0.y += B1.y;
                const float2 b1x = make_float2(B1.x, B1.x), b1y = make_float2(B1.y, B1.y);
                const float2 b2x = make_float2(B2.x, B2.x), b2y = make_float2(B2.y, B2.y);
                const float4 *Z = cur + a * cw + S.pad0;
#pragma unroll
                for (int h = 0; h < NP; h++) {
                    const float4 ee = Z[h];
                    const float2 cv = make_float2(ee.x, ee.y), dv = make_float2(ee.z, ee.w);
                    Sa[h] = __ffma2_rn(b1x, cv, Sa[h]);
                    Sb[h] = __ffma2_rn(b1y, dv, Sb[h]);
                    Sc[h] = __ffma2_rn(b1x, dv, Sc[h]);
                    Sd[h] = __ffma2_rn(b1y, cv, Sd[h]);
                    if (LD) {
                        Ta[h] = __ffma2_rn(b2x, cv, Ta[h]);
                        Tb[h] = __ffma2_rn(b2y, dv, Tb[h]);
                        Tc[h] = __ffma2_rn(b2x, dv, Tc[h]);
                        Td[h] = __ffma2_rn(b2y, cv, Td[h]);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (sid < nseg) {
        // k index of nz in this row: S.koff + nz
        float2 *P = part + (size_t)blockIdx.y * nk + S.koff;
        const bool neg = S.pad1 & 1;
        if (S.pad1 & 2) P[0] = acc0;
#pragma unroll
        for (int h = 0; h < NP; h++) {
#pragma unroll
            for (int l = 0; l < 2; l++) {
                if (2 * h + l >= S.cnt) continue;
                const int z = S.z0 + 2 * h + l;
                const float fz = (float)z;
                const float sa = l ? Sa[h].y : Sa[h].x, sb = l ? Sb[h].y : Sb[h].x;
                const float sc = l ? Sc[h].y : Sc[h].x, sd = l ? Sd[h].y : Sd[h].x;
                const float ta = l ? Ta[h].y : Ta[h].x, tb = l ? Tb[h].y : Tb[h].x;
                const float tc = l ? Tc[h].y : Tc[h].x, td = l ? Td[h].y : Td[h].x;
                P[z] = make_float2(sa - sb + fz * (ta - tb), sc + sd + fz * (tc + td));
                if (neg) P[-z] = make_float2(sa + sb - fz * (ta + tb), sd - sc + fz * (tc - td));
            }
        }
    }
}

// ---------------------------------------------------------------- pass 2: per ion
struct Ion32Args {
    int cnt, nrow, rows_per_slice, nk;
    const int *idx;
    Cell c;
    const double4 *r;
    const double3 *mu;
    const KRow *row;
    const double2 *rho_s;
    double *part;          // [slice][cnt][nv]
    int ld;
};

// float4 entries per z pair of a staged row: the G and H weights, and K with forces
__host__ __device__ constexpr int ion32_nv(bool wf) { return wf ? 6 : 4; }
static int ion32_row_bytes(int KZ, bool wf) {
    return (int)sizeof(float4) * (1 + (KZ / 2) * ion32_nv(wf)) + (int)sizeof(int2);
}

// With Y(k) = Ak rho(k) conj(exp(i k.r)), the field needs Im Y, the force Re Y, summed
// over k with weights 1, nz (and nz^2).  In a row, exp(i k.r) = w E2[nz] with the row
// phase w, and E2[-z] = conj E2[z] = (c, -d), so over the row
//     sum Y = conj(w) G,  sum nz Y = conj(w) H,  sum nz^2 Y = conj(w) K,
//     G = rho_0 + sum_z (a1 c + a2 d, a3 c + a4 d),   K = sum_z z^2 (same terms)
//     H = sum_z z (-a4 c + a3 d, a2 c - a1 d)
// with a1 = Re(rho_z + rho_-z), a2 = Im(rho_z - rho_-z), a3 = Im(rho_z + rho_-z),
// a4 = Re(rho_-z - rho_z) of Ak rho.  The block stages a1..a4 (and their z, z^2
// multiples) of its rows in shared memory as planar z pairs; per ion the sums cost
// 4 FMA per k-vector (6 with forces: G, H and K are complex, each |z| serves +z and -z),
// packed FP32x2 FMAs over the pairs.
// the slice's rows staged in shared memory: (nx, ny) of each row in rnxy, and per row
// entry 0 = (rho_0, 0, 0), then per z pair (z, z') = (2p+1, 2p+2) the weights
//   (a1, a1', a2, a2'), (a3, a3', a4, a4'), z (-a4, -a4', a3, a3'), z (a2, a2', -a1, -a1'),
//   [forces] z^2 (a1, a1', a2, a2'), z^2 (a3, a3', a4, a4')
template <int KZ, bool WF>
__device__ __forceinline__ void ion32_stage(const Ion32Args &a, float4 *rk4, int2 *rnxy, int r0, int nrs) {
    constexpr int NV = ion32_nv(WF), NP = KZ / 2, RS = 1 + NP * NV;
    for (int e = threadIdx.x; e < nrs; e += (int)blockDim.x) {
        KRow R = a.row[r0 + e];
        rnxy[e] = make_int2(R.nx, R.ny);
    }
    for (int e = threadIdx.x; e < nrs * (NP + 1); e += (int)blockDim.x) {
        int rr = e / (NP + 1), pe = e - rr * (NP + 1);
        KRow R = a.row[r0 + rr];
        int zlo = R.z0, zhi = R.z0 + R.cnt - 1;
        auto rho_at = [&](int z) {
            if (z < zlo || z > zhi) return make_float2(0.f, 0.f);
            double2 p = a.rho_s[R.koff + z - zlo];
            return make_float2((float)p.x, (float)p.y);
        };
        float4 *o = rk4 + rr * RS;
        if (pe == 0) {
            float2 p = rho_at(0);
            o[0] = make_float4(p.x, p.y, 0.f, 0.f);
            continue;
        }
        int pr = pe - 1;
        float A1[2], A2[2], A3[2], A4[2], zz[2];
#pragma unroll
        for (int l = 0; l < 2; l++) {
            int z = 2 * pr + 1 + l;
            float2 rp = rho_at(z), rn = rho_at(-z);
            A1[l] = rp.x + rn.x;
            A2[l] = rp.y - rn.y;
            A3[l] = rp.y + rn.y;
            A4[l] = rn.x - rp.x;
            zz[l] = (float)z;
        }
        float4 *q = o + 1 + NV * pr;
        q[0] = make_float4(A1[0], A1[1], A2[0], A2[1]);
        q[1] = make_float4(A3[0], A3[1], A4[0], A4[1]);
        q[2] = make_float4(-zz[0] * A4[0], -zz[1] * A4[1], zz[0] * A3[0], zz[1] * A3[1]);
        q[3] = make_float4(zz[0] * A2[0], zz[1] * A2[1], -zz[0] * A1[0], -zz[1] * A1[1]);
        if (WF) {
            float s0 = zz[0] * zz[0], s1 = zz[1] * zz[1];
            q[4] = make_float4(s0 * A1[0], s1 * A1[1], s0 * A2[0], s1 * A2[1]);
            q[5] = make_float4(s0 * A3[0], s1 * A3[1], s0 * A4[0], s1 * A4[1]);
        }
    }
}

template <int KZ, bool WF>
__global__ void __launch_bounds__(ION32_THREADS, ION32_MIN_BLOCKS) k_ion32(Ion32Args a) {
    grid_dep();
    constexpr int NV = ion32_nv(WF), NP = KZ / 2, RS = 1 + NP * NV;
    extern __shared__ float4 rk4[];          // [rows of the slice][RS]
    int2 *rnxy = (int2 *)(rk4 + a.rows_per_slice * RS);   // (nx, ny) of the slice's rows
    int li = blockIdx.x * ION32_THREADS + threadIdx.x;
    int sl = blockIdx.y;
    int r0 = sl * a.rows_per_slice, r1 = min(a.nrow, r0 + a.rows_per_slice);
    int nrs = r1 - r0;
    ion32_stage<KZ, WF>(a, rk4, rnxy, r0, nrs);
    bool act = li < a.cnt;
    int ion = act ? (a.idx ? a.idx[li] : li) : 0;
    double4 ri = a.r[ion];
    const Cell &c = a.c;
    double tx = c.B[0][0] * ri.x + c.B[1][0] * ri.y + c.B[2][0] * ri.z;
    double ty = c.B[0][1] * ri.x + c.B[1][1] * ri.y + c.B[2][1] * ri.z;
    double tz = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
    // E2[z], z = 1..KZ, as planar pairs over (2p+1, 2p+2)
    float2 Ex[NP], Ey[NP];
#pragma unroll
    for (int pr = 0; pr < NP; pr++) {
        float2 ea = cis2pi32((double)(2 * pr + 1) * tz), eb = cis2pi32((double)(2 * pr + 2) * tz);
        Ex[pr] = make_float2(ea.x, eb.x);
        Ey[pr] = make_float2(ea.y, eb.y);
    }
    float mz = 0.f;
    double mx = 0.0, my = 0.0;
    if (WF && a.ld) {
        double3 m3 = a.mu[ion];
        mx = c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z;
        my = c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z;
        mz = (float)(c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z);
    }
    // row phase: exact (FP64-reduced argument) at the start of a run of up to ION32_RUN
    // rows (nx, ny), (nx, ny + 1), ..., the next ones times exp(2 pi i ty) in FP32
    const float2 e1 = cis2pi32(ty);
    float2 w = make_float2(1.f, 0.f);
    int2 Rp = make_int2(0, 0);
    int run = ION32_RUN;
    __syncthreads();
    double S0 = 0, S1 = 0, S2 = 0, P0 = 0, P1 = 0, P2 = 0;
    for (int rr = 0; rr < nrs; rr++) {
        int2 R = rnxy[rr];
        if (run < ION32_RUN && R.x == Rp.x && R.y == Rp.y + 1) {
            w = cmul32(w, e1);
            run++;
        } else {
            w = cis2pi32((double)R.x * tx + (double)R.y * ty);
            run = 1;
        }
        Rp = R;
        const float4 *Q = rk4 + rr * RS;
        const float4 q0 = Q[0];
        // two accumulators per component (the c and the d terms) for independent chains
        const float2 zero = make_float2(0.f, 0.f);
        float2 gx0 = zero, gx1 = zero, gy0 = zero, gy1 = zero, hx0 = zero, hx1 = zero, hy0 = zero, hy1 = zero;
        float2 kx = zero, ky = zero;
#pragma unroll
        for (int pr = 0; pr < NP; pr++) {
            const float4 *q = Q + 1 + NV * pr;
            const float4 g1 = q[0], g2 = q[1], h1 = q[2], h2 = q[3];
            const float2 ex = Ex[pr], ey = Ey[pr];
            gx0 = __ffma2_rn(make_float2(g1.x, g1.y), ex, gx0);
            gx1 = __ffma2_rn(make_float2(g1.z, g1.w), ey, gx1);
            gy0 = __ffma2_rn(make_float2(g2.x, g2.y), ex, gy0);
            gy1 = __ffma2_rn(make_float2(g2.z, g2.w), ey, gy1);
            hx0 = __ffma2_rn(make_float2(h1.x, h1.y), ex, hx0);
            hx1 = __ffma2_rn(make_float2(h1.z, h1.w), ey, hx1);
            hy0 = __ffma2_rn(make_float2(h2.x, h2.y), ex, hy0);
            hy1 = __ffma2_rn(make_float2(h2.z, h2.w), ey, hy1);
            if (WF) {
                const float4 k1 = q[4], k2 = q[5];
                kx = __ffma2_rn(make_float2(k1.z, k1.w), ey, __ffma2_rn(make_float2(k1.x, k1.y), ex, kx));
                ky = __ffma2_rn(make_float2(k2.z, k2.w), ey, __ffma2_rn(make_float2(k2.x, k2.y), ex, ky));
            }
        }
        const float2 gx = __fadd2_rn(gx0, gx1), gy = __fadd2_rn(gy0, gy1);
        const float2 hx = __fadd2_rn(hx0, hx1), hy = __fadd2_rn(hy0, hy1);
        const float Gx = q0.x + (gx.x + gx.y), Gy = q0.y + (gy.x + gy.y);
        const float Hx = hx.x + hx.y, Hy = hy.x + hy.y;
        // Im conj(w) G and Im conj(w) H
        const float R1 = w.x * Gy - w.y * Gx, Rz = w.x * Hy - w.y * Hx;
        double fx = (double)R.x, fy = (double)R.y;
        S0 += fx * (double)R1;
        S1 += fy * (double)R1;
        S2 += (double)Rz;
        if (WF) {
            const float Kx = kx.x + kx.y, Ky = ky.x + ky.y;
            // Re conj(w) G, H, K: sum_k (n.m) Re(conj(rho) ph) per component weight n,
            // c0 = nx mx + ny my
            const float Q0 = w.x * Gx + w.y * Gy, Q1 = w.x * Hx + w.y * Hy, Q2 = w.x * Kx + w.y * Ky;
            double c0 = fx * mx + fy * my;
            double T1 = c0 * (double)Q0 + (double)mz * (double)Q1;
            double Tz = c0 * (double)Q1 + (double)mz * (double)Q2;
            P0 += fx * T1;
            P1 += fy * T1;
            P2 += Tz;
        }
    }
    if (!act) return;
    const int nv = WF ? 6 : 3;
    double *o = a.part + ((size_t)sl * a.cnt + li) * nv;
    o[0] = S0;
    o[1] = S1;
    o[2] = S2;
    if (WF) {
        o[3] = P0;
        o[4] = P1;
        o[5] = P2;
    }
}

// k_ion32 for a field-only pass with two ions per thread (ions li and li + ION32_THREADS
// of a block of 2 ION32_THREADS): each staged weight loaded from shared memory feeds both
// ions' packed FMAs, and the two ions' sums are independent chains.  Same arithmetic per
// ion as k_ion32<KZ, false>.
template <int KZ>
__global__ void __launch_bounds__(ION32_THREADS, ION32X2_MIN_BLOCKS) k_ion32x2(Ion32Args a) {
    grid_dep();
    constexpr int NV = ion32_nv(false), NP = KZ / 2, RS = 1 + NP * NV;
    extern __shared__ float4 rk4[];          // [rows of the slice][RS]
    int2 *rnxy = (int2 *)(rk4 + a.rows_per_slice * RS);
    int sl = blockIdx.y;
    int r0 = sl * a.rows_per_slice, r1 = min(a.nrow, r0 + a.rows_per_slice);
    int nrs = r1 - r0;
    ion32_stage<KZ, false>(a, rk4, rnxy, r0, nrs);
    const Cell &c = a.c;
    int li[2];
    double tx[2], ty[2];
    float2 Ex[2][NP], Ey[2][NP], e1[2], w[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
        li[u] = blockIdx.x * (2 * ION32_THREADS) + u * ION32_THREADS + threadIdx.x;
        int ion = li[u] < a.cnt ? (a.idx ? a.idx[li[u]] : li[u]) : 0;
        double4 ri = a.r[ion];
        tx[u] = c.B[0][0] * ri.x + c.B[1][0] * ri.y + c.B[2][0] * ri.z;
        ty[u] = c.B[0][1] * ri.x + c.B[1][1] * ri.y + c.B[2][1] * ri.z;
        double tz = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
#pragma unroll
        for (int pr = 0; pr < NP; pr++) {
            float2 ea = cis2pi32((double)(2 * pr + 1) * tz), eb = cis2pi32((double)(2 * pr + 2) * tz);
            Ex[u][pr] = make_float2(ea.x, eb.x);
            Ey[u][pr] = make_float2(ea.y, eb.y);
        }
        e1[u] = cis2pi32(ty[u]);
        w[u] = make_float2(1.f, 0.f);
    }
    int2 Rp = make_int2(0, 0);
    int run = ION32_RUN;
    __syncthreads();
    double S0[2] = {0, 0}, S1[2] = {0, 0}, S2[2] = {0, 0};
    for (int rr = 0; rr < nrs; rr++) {
        int2 R = rnxy[rr];
        const bool step = run < ION32_RUN && R.x == Rp.x && R.y == Rp.y + 1;
#pragma unroll
        for (int u = 0; u < 2; u++)
            w[u] = step ? cmul32(w[u], e1[u]) : cis2pi32((double)R.x * tx[u] + (double)R.y * ty[u]);
        run = step ? run + 1 : 1;
        Rp = R;
        const float4 *Q = rk4 + rr * RS;
        const float4 q0 = Q[0];
        const float2 zero = make_float2(0.f, 0.f);
        float2 gx[2] = {zero, zero}, gy[2] = {zero, zero}, hx[2] = {zero, zero}, hy[2] = {zero, zero};
#pragma unroll
        for (int pr = 0; pr < NP; pr++) {
            const float4 *q = Q + 1 + NV * pr;
            const float4 g1 = q[0], g2 = q[1], h1 = q[2], h2 = q[3];
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const float2 ex = Ex[u][pr], ey = Ey[u][pr];
                gx[u] = __ffma2_rn(make_float2(g1.z, g1.w), ey, __ffma2_rn(make_float2(g1.x, g1.y), ex, gx[u]));
                gy[u] = __ffma2_rn(make_float2(g2.z, g2.w), ey, __ffma2_rn(make_float2(g2.x, g2.y), ex, gy[u]));
                hx[u] = __ffma2_rn(make_float2(h1.z, h1.w), ey, __ffma2_rn(make_float2(h1.x, h1.y), ex, hx[u]));
                hy[u] = __ffma2_rn(make_float2(h2.z, h2.w), ey, __ffma2_rn(make_float2(h2.x, h2.y), ex, hy[u]));
            }
        }
        double fx = (double)R.x, fy = (double)R.y;
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const float Gx = q0.x + (gx[u].x + gx[u].y), Gy = q0.y + (gy[u].x + gy[u].y);
            const float Hx = hx[u].x + hx[u].y, Hy = hy[u].x + hy[u].y;
            // Im conj(w) G and Im conj(w) H
            const float R1 = w[u].x * Gy - w[u].y * Gx, Rz = w[u].x * Hy - w[u].y * Hx;
            S0[u] += fx * (double)R1;
            S1[u] += fy * (double)R1;
            S2[u] += (double)Rz;
        }
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
        if (li[u] >= a.cnt) continue;
        double *o = a.part + ((size_t)sl * a.cnt + li[u]) * 3;
        o[0] = S0[u];
        o[1] = S1[u];
        o[2] = S2[u];
    }
}

// slices summed in a fixed order; field / force / self terms as k_rec_combine (kspace.cu)
struct Comb32Args {
    int cnt, nslice;
    const int *idx;
    Cell c;
    const double *part;
    double tfpiV, self2, coul;
    int ld;
    const double *q;
    const double3 *muself;
    const double3 *ef_dir;
    double3 *ef;
    const double3 *f_dir;
    double3 *f;
    CgAp cg;
};

template <bool WF>
__global__ void k_combine32(Comb32Args a) {
    grid_dep();
    int li = blockIdx.x * blockDim.x + threadIdx.x;
    double pap[1] = {0.0};
    if (li < a.cnt) {
        int i = a.idx ? a.idx[li] : li;
        const int nv = WF ? 6 : 3;
        double S[3] = {0, 0, 0}, P[3] = {0, 0, 0};
        for (int s = 0; s < a.nslice; s++) {
            const double *o = a.part + ((size_t)s * a.cnt + li) * nv;
            for (int k = 0; k < 3; k++) S[k] += o[k];
            if (WF)
                for (int k = 0; k < 3; k++) P[k] += o[3 + k];
        }
        const Cell &c = a.c;
        const double tpi = TPI_D;
        double gS[3], gP[3];
        for (int k = 0; k < 3; k++) {
            gS[k] = tpi * (c.B[k][0] * S[0] + c.B[k][1] * S[1] + c.B[k][2] * S[2]);
            gP[k] = tpi * tpi * (c.B[k][0] * P[0] + c.B[k][1] * P[1] + c.B[k][2] * P[2]);
        }
        if (a.ef) {
            double3 mu = a.muself ? a.muself[i] : make_double3(0, 0, 0);
            double3 b = make_double3(a.self2 * mu.x, a.self2 * mu.y, a.self2 * mu.z);
            if (a.ef_dir) {
                double3 d = a.ef_dir[i];
                b.x += d.x;
                b.y += d.y;
                b.z += d.z;
            }
            const double3 t =
                make_double3(b.x + (-a.tfpiV * gS[0]), b.y + (-a.tfpiV * gS[1]), b.z + (-a.tfpiV * gS[2]));
            a.ef[i] = t;
            if (!WF && a.cg.ap) {
                // k_cg_ap at a polarisable ion: ap = invpol p - T p, and p.ap
                double3 m = a.cg.p[i];
                const double *I = a.cg.invpol + (size_t)i * 9;
                double3 ap = make_double3(I[0] * m.x + I[1] * m.y + I[2] * m.z - t.x,
                                          I[3] * m.x + I[4] * m.y + I[5] * m.z - t.y,
                                          I[6] * m.x + I[7] * m.y + I[8] * m.z - t.z);
                a.cg.ap[i] = ap;
                pap[0] = m.x * ap.x + m.y * ap.y + m.z * ap.z;
            }
        }
        if (WF && a.f) {
            double qi = a.q ? a.q[i] : 0.0;
            double3 fo = a.f[i];
            if (a.f_dir) {
                double3 d = a.f_dir[i];
                fo.x += d.x * a.coul;
                fo.y += d.y * a.coul;
                fo.z += d.z * a.coul;
            }
            double fr[3];
            for (int k = 0; k < 3; k++) fr[k] = a.tfpiV * (-qi * gS[k] + (a.ld ? gP[k] : 0.0));
            a.f[i] = make_double3(fo.x + fr[0] * a.coul, fo.y + fr[1] * a.coul, fo.z + fr[2] * a.coul);
        }
    }
    if (!WF && a.cg.ap) {
        block_sum_to_part<1>(pap, a.cg.part, S_PAP, a.cg.stride);
        last_block_slots(a.cg.part, a.cg.stride, S_PAP, 1, a.cg.scal, a.cg.ticket);
    }
}

// ---------------------------------------------------------------- set-up and launchers
static TabLayout layout_of(const Engine &e) {
    TabLayout L;
    L.K0 = e.kmax[0];
    L.K1 = e.kmax[1];
    L.K2 = e.kmax[2];
    L.nzb_neg = ceil_div(L.K2 + 1, ZB);
    L.nzb = L.nzb_neg + std::max(1, ceil_div(L.K2, ZB));   // at least one z > 0 block
    L.e1 = L.K0 + 1;
    L.z = L.e1 + 2 * L.K1 + 1;
    L.z += L.z & 1;
    L.w = L.z + ZS * L.nzb;
    return L;
}

static int kz_of(int K2) { return K2 <= 8 ? 8 : (K2 <= 14 ? 14 : (K2 <= 16 ? 16 : 32)); }

void setup_kspace32(Engine &e, const std::vector<KRow> &rows) {
    TabLayout L = layout_of(e);
    if (kz_of(L.K2) < L.K2) throw Error(MDFFGPU_ERR_ARG, "mixed precision k-space supports kmax_z <= 32");
    // rho segments: per row, |nz| blocks of RZP starting at 1; the row holds nz = -K2..K2,
    // or nz = 1..K2 for (nx, ny) = (0, 0)
    std::vector<KSeg> segs;
    for (const KRow &R : rows) {
        bool full = R.z0 == -L.K2;
        if ((!full && R.z0 != 1) || R.z0 + R.cnt - 1 != L.K2) throw Error(MDFFGPU_ERR_ARG, "unexpected k row extent");
        for (int z0 = 1; z0 <= std::max(L.K2, 1); z0 += RZP) {   // K2 = 0: one segment for nz = 0
            KSeg S;
            S.nx = R.nx;
            S.ny = R.ny;
            S.z0 = z0;
            S.cnt = std::max(0, std::min(RZP, L.K2 - z0 + 1));
            S.koff = R.koff - R.z0;
            // staged-row offset (16-byte units) of the pair (z0, z0 + 1) in the z > 0 blocks
            S.pad0 = L.z / 2 + (ZS / 2) * ((z0 - 1) / ZB) + ((z0 - 1) % ZB) / 2;
            S.pad1 = (full ? 1 : 0) | ((full && z0 == 1) ? 2 : 0);
            S.pad2 = 0;
            segs.push_back(S);
        }
    }
    e.nseg32 = (int)segs.size();
    e.d_seg32 = dalloc<KSeg>(e.nseg32);
    MDFF_CK(cudaMemcpy(e.d_seg32, segs.data(), sizeof(KSeg) * e.nseg32, cudaMemcpyHostToDevice));
    e.tab_w = L.w;
    e.d_tab32 = dalloc<float2>((size_t)e.n * L.w);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e.device);
    int segblocks = ceil_div(e.nseg32, RHO32_THREADS);
    int chunks = std::max(1, RHO32_MIN_BLOCKS * nsm / segblocks);
    chunks = std::min(chunks, std::max(1, ceil_div(e.n, RHO32_TI)));
    e.rho32_chunks = chunks;
    // room for twice the chunks: the launch tuner tries 0.5x, 1x and 2x
    e.rho32_chunks_max = std::max(chunks, std::min(2 * chunks, std::max(1, ceil_div(e.n, RHO32_TI))));
    e.d_rho_part32 = dalloc<float2>((size_t)e.rho32_chunks_max * e.nk);
    // ion-pass slices are chosen per launch (ion32_slicing); room for the largest count
    e.nsm = nsm;
    int maxrows = std::max(1, (48 * 1024) / ion32_row_bytes(kz_of(L.K2), true));
    e.ion32_slices = std::max(std::min(32, e.nrow), ceil_div(e.nrow, maxrows));
    e.d_ion_part32 = dalloc<double>((size_t)e.ion32_slices * e.n * 6);
    setup_ion_tc(e);
    setup_rho_tc(e, L.z);
}

// k-row slices of one ion pass over `cnt` ions: about two full waves of resident blocks,
// at most e.ion32_slices, each slice's staged rows within 48 KB of shared memory
// two ions per thread: field-only passes with nz up to 16 (register budget)
static bool ion32_x2(const Engine &e, bool wf) { return !wf && kz_of(e.kmax[2]) <= 16; }

static void ion32_slicing(const Engine &e, int cnt, bool wf, int &rows, int &slices) {
    int KZ = kz_of(e.kmax[2]);
    // two ions per thread: the blocks fill the GPU once; one ion per thread: twice
    const bool x2 = ion32_x2(e, wf);
    int iblocks = ceil_div(std::max(cnt, 1), x2 ? 2 * ION32_THREADS : ION32_THREADS);
    int s = std::max(1, (x2 ? ION32X2_MIN_BLOCKS : 2 * ION32_MIN_BLOCKS) * e.nsm / iblocks);
    s = std::min(s, std::min(e.nrow, e.ion32_slices));
    int maxrows = std::max(1, (48 * 1024) / ion32_row_bytes(KZ, wf));
    s = std::max(s, ceil_div(e.nrow, maxrows));
    rows = ceil_div(e.nrow, s);
    slices = ceil_div(e.nrow, rows);
}

void launch_phase32(Engine &e) {
    TabLayout L = layout_of(e);
    MDFF_LAUNCH(e, k_phase32, ceil_div(e.n, 8), dim3(32, 8), 0, e.n, e.cell, e.d_r, L, e.d_tab32);
}

void launch_coords32(Engine &e) {
    if (e.d_tab32) launch_phase32(e);
    if (e.ion_tc) launch_ion_tc_table(e);
    if (e.rho_tc && e.d_tab32) launch_rho_tc_tables(e);
}

// FLOPs per (ion, k-vector) of the paired-nz formulation: 4 FMA with dipoles, 2 without
static double rho32_flops_per_pair(bool ld) { return ld ? 8.0 : 4.0; }
// FLOPs per (ion, k-vector) of the folded ion pass, counted from the loop body: per z
// pair (z, z') a thread issues 8 packed FFMA2 for G and H (16 FMA) per ion, covering the
// four k-vectors +-z, +-z' of the row: 4 FMA = 8 flops per (ion, k) for the field; the
// force pass adds the two K sums (4 FFMA2 more): 6 FMA = 12 flops
static double ion32_flops_per_pair(bool f) { return f ? 12.0 : 8.0; }
void launch_rho_reduce32(Engine &e, const float2 *part, int nchunks, double2 *rho_raw);

template <bool LQ, bool LD>
static void rho32_launch(Engine &e, dim3 grid, size_t smem, int cnt, const int *idx, int chunk, const TabLayout &L,
                         const double *q, const double3 *mu) {
    if (smem > 48 * 1024)
        MDFF_CK(cudaFuncSetAttribute(k_rho32<LQ, LD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MDFF_LAUNCH(e, (k_rho32<LQ, LD>), grid, RHO32_THREADS, smem, cnt, idx, chunk, L, e.d_tab32, e.cell, q, mu,
                e.nseg32, e.d_seg32, e.d_rho_part32, e.nk);
}

// rho(k) of (q, mu) over `cnt` ions (all when idx is null) into e.d_rho_part32 partials
void launch_rho32(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt) {
    TabLayout L = layout_of(e);
    int segblocks = ceil_div(e.nseg32, RHO32_THREADS);
    int chunk = ceil_div(std::max(cnt, 1), e.rho32_chunks);
    chunk = ceil_div(chunk, 4) * 4;
    dim3 grid(segblocks, e.rho32_chunks);
    const int cw = L.w / 2 - (ZS / 2) * L.nzb_neg;
    size_t smem = 2 * (sizeof(float4) * RHO32_TI * cw + sizeof(float4) * RHO32_TI);
    int ps = -1;
    e.prof_begin("k_rho", &ps);
    e.rho_chunks_used = e.rho32_chunks;
    int used = 0;
    if ((lq || ld) && e.rho_tc && launch_rho_tc(e, q, mu, lq, ld, idx, cnt, L.z, &used)) {
        e.rho_chunks_used = used;
    } else if (lq && ld) rho32_launch<true, true>(e, grid, smem, cnt, idx, chunk, L, q, mu);
    else if (lq) rho32_launch<true, false>(e, grid, smem, cnt, idx, chunk, L, q, mu);
    else if (ld) rho32_launch<false, true>(e, grid, smem, cnt, idx, chunk, L, q, mu);
    else MDFF_CK(cudaMemsetAsync(e.d_rho_part32, 0, sizeof(float2) * (size_t)e.nk * e.rho32_chunks, e.stream));
    e.prof_end("k_rho", ps, (lq || ld) ? rho32_flops_per_pair(ld) * (double)cnt * e.nk : 0.0);
}

template <int KZ, bool WF>
static void ion32_launch(Engine &e, dim3 g, size_t smem, const Ion32Args &a) {
    MDFF_LAUNCH(e, (k_ion32<KZ, WF>), g, ION32_THREADS, smem, a);
}

template <int KZ>
static void ion32_dispatch(Engine &e, dim3 g, size_t smem, const Ion32Args &a, bool wf) {
    if (wf) ion32_launch<KZ, true>(e, g, smem, a);
    else if (KZ <= 16) MDFF_LAUNCH(e, k_ion32x2<KZ <= 16 ? KZ : 16>, g, ION32_THREADS, smem, a);
    else ion32_launch<KZ, false>(e, g, smem, a);
}

// field (and force) terms of Ak rho(k) (e.d_rho) at `cnt` ions, then slice sums + self/direct terms
void launch_ion32(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx, int cnt) {
    bool wf = o.f != nullptr;
    if (e.ion_tc && launch_ion_tc(e, q, mu, ld, o, idx, cnt)) return;   // tensor-core pass
    int rows = 1, slices = 1;
    ion32_slicing(e, cnt, wf, rows, slices);
    Ion32Args a;
    a.cnt = cnt;
    a.nrow = e.nrow;
    a.rows_per_slice = rows;
    a.nk = e.nk;
    a.idx = idx;
    a.c = e.cell;
    a.r = e.d_r;
    a.mu = mu;
    a.row = e.d_row;
    a.rho_s = e.d_rho;
    a.part = e.d_ion_part32;
    a.ld = ld;
    int KZ = kz_of(e.kmax[2]);
    size_t smem = (size_t)ion32_row_bytes(KZ, wf) * rows;
    dim3 g(ceil_div(std::max(cnt, 1), ion32_x2(e, wf) ? 2 * ION32_THREADS : ION32_THREADS), slices);
    int pi = -1;
    e.prof_begin("k_rec_ion", &pi);
    if (KZ == 8) ion32_dispatch<8>(e, g, smem, a, wf);
    else if (KZ == 14) ion32_dispatch<14>(e, g, smem, a, wf);
    else if (KZ == 16) ion32_dispatch<16>(e, g, smem, a, wf);
    else ion32_dispatch<32>(e, g, smem, a, wf);
    e.prof_end("k_rec_ion", pi, ion32_flops_per_pair(wf) * (double)cnt * e.nk);
    launch_combine32(e, q, mu, ld, o, idx, cnt, slices, wf);
}

// the slice partials of an ion pass (e.d_ion_part32, [slice][cnt][3 or 6]) summed per ion
// and turned into field / force / self terms at ion idx[li] (li when idx is null)
void launch_combine32(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx,
                      int cnt, int slices, bool wf) {
    // the real-space terms and the short-range forces it adds to, when they ran beside
    e.join_side(Engine::SIDE_DIR);
    e.join_side(Engine::SIDE_SR);
    e.join_side(Engine::SIDE_PREP);
    e.join_side(Engine::SIDE_BODY);
    e.join_side(Engine::SIDE_FIELD);
    Comb32Args b;
    b.cnt = cnt;
    b.nslice = slices;
    b.idx = idx;
    b.c = e.cell;
    b.part = e.d_ion_part32;
    b.tfpiV = 2.0 * 2.0 * TPI_D * e.cell.inveOmega;
    b.self2 = o.self2;
    b.coul = o.coul;
    b.ld = ld;
    b.q = q;
    b.muself = o.self_mu;
    b.ef_dir = o.ef_dir;
    b.ef = o.ef;
    b.f_dir = o.f_dir;
    b.f = o.f;
    b.cg = o.cg;
    if (b.cg.ap && (wf || !o.ef)) throw Error(MDFFGPU_ERR_STATE, "the CG product needs a field-only pass");
    int nb = ceil_div(std::max(cnt, 1), 256);
    if (wf) MDFF_LAUNCH(e, k_combine32<true>, nb, 256, 0, b);
    else MDFF_LAUNCH(e, k_combine32<false>, nb, 256, 0, b);
}

}  // namespace mdffgpu
