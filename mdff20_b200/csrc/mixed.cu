// Mixed-precision (MDFFGPU_MIXED) real-space and k-space Ewald kernels.
//
// Same sums as pair.cu / kspace.cu, with the per-pair and per-(ion, k) arithmetic in
// FP32 and every accumulation that spans many terms compensated by FP64: pair terms are
// summed in FP32 per lane (about a dozen terms) and combined in FP64 across the warp;
// rho(k) is summed in FP32 over one block's chunk of ions (a few hundred) and the chunks
// are combined in FP64; the ion pass sums one k-row (<= 2 kmax + 1 terms) in FP32 and
// the rows in FP64.
// Geometry keeps FP64 where it matters: fractional coordinates are wrapped in FP64
// before they are rounded to FP32 (|s| <= 1/2, so the minimum-image difference keeps
// ~1e-7 relative accuracy), and the row phase bases are reduced in FP64.
// Neighbour lists, short-range forces, integrators and all reductions stay FP64.
#include "engine.cuh"

namespace mdffgpu {

constexpr int PAIR_WARPS32 = 8;
constexpr int RHO32_THREADS = 128;
constexpr int RHO32_TI = 32;
constexpr int ION32_THREADS = 128;
constexpr int ION32_NV = 12;

struct TT32 {
    float E[9];
};

__device__ __forceinline__ float powif(float x, int k) {
    float r = 1.0f;
    while (k) {
        if (k & 1) r *= x;
        x *= x;
        k >>= 1;
    }
    return r;
}

// TT_damping_functions (src/tt_damp.c:16-32) in FP32
__device__ __forceinline__ void tt_damp32(const TT32 &tt, float b, float c, float r, int order, float &f, float &fd) {
    float br = b * r;
    float ex = expf(-br) * c;
    float ff = tt.E[order];
    for (int k = order - 1; k > -1; k--) ff = ff * br + tt.E[k];
    f = 1.0f - ff * ex;
    fd = tt.E[order] * powif(br, order) * ex * b;
}

// wrapped fractional (kardir) and phase (B^T r) coordinates in FP32, w = charge
__global__ void k_coords32(int n, Cell c, const double4 *__restrict__ r, float4 *__restrict__ s32,
                           float4 *__restrict__ t32) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 ri = r[i];
    double3 s = kardir(c, ri.x, ri.y, ri.z);
    s.x -= rint(s.x);
    s.y -= rint(s.y);
    s.z -= rint(s.z);
    s32[i] = make_float4((float)s.x, (float)s.y, (float)s.z, (float)ri.w);
    double tx = c.B[0][0] * ri.x + c.B[1][0] * ri.y + c.B[2][0] * ri.z;
    double ty = c.B[0][1] * ri.x + c.B[1][1] * ri.y + c.B[2][1] * ri.z;
    double tz = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
    t32[i] = make_float4((float)(tx - rint(tx)), (float)(ty - rint(ty)), (float)(tz - rint(tz)), 0.f);
}

struct CellF {
    float A[3][3];
    float B[3][3];
};

__device__ __forceinline__ float3 pbc32(const CellF &c, float dx, float dy, float dz) {
    dx -= rintf(dx);
    dy -= rintf(dy);
    dz -= rintf(dz);
    return make_float3(dx * c.A[0][0] + dy * c.A[1][0] + dz * c.A[2][0],
                       dx * c.A[0][1] + dy * c.A[1][1] + dz * c.A[2][1],
                       dx * c.A[0][2] + dy * c.A[1][2] + dz * c.A[2][2]);
}

// ---------------------------------------------------------------- real space
struct Dir32Args {
    int n, nt, cap;
    CellF c;
    const float4 *s;
    const double *q;
    const double3 *mu;
    const int *typ;
    const PairDamp *damp;
    const int *col, *con;
    float lrcutsq, alpha;
    TT32 tt;
    int lq, ld, ldamp;
    double3 *ef;
    double3 *f;
    double *part;
    int slot, stride;
};

// multipole_ES_dir for charges and dipoles (see k_dir in pair.cu), FP32 pair math
template <bool FORCES, bool EF>
__global__ void __launch_bounds__(PAIR_WARPS32 * 32) k_dir32(Dir32Args a) {
    int i = blockIdx.x * PAIR_WARPS32 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    float acc[7] = {0, 0, 0, 0, 0, 0, 0};
    float fi[3] = {0, 0, 0}, ei[3] = {0, 0, 0};
    const float alpha = a.alpha, alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
    const float rpi = 1.7724538509055160273f;
    if (i < a.n) {
        float4 si = a.s[i];
        float qi = a.lq ? (float)a.q[i] : 0.f;
        float3 mi = make_float3(0.f, 0.f, 0.f);
        if (a.ld) {
            double3 m = a.mu[i];
            mi = make_float3((float)m.x, (float)m.y, (float)m.z);
        }
        bool dip_i = (mi.x != 0.f) || (mi.y != 0.f) || (mi.z != 0.f);
        int ti = a.typ[i];
        int m = min(a.con[i], a.cap);
        const int *L = a.col + (size_t)i * a.cap;
        for (int k = lane; k < m; k += 32) {
            int j = L[k];
            float4 sj = a.s[j];
            float3 r = pbc32(a.c, si.x - sj.x, si.y - sj.y, si.z - sj.z);
            float d2 = r.x * r.x + r.y * r.y + r.z * r.z;
            if (d2 > a.lrcutsq) continue;
            float qj = a.lq ? (float)a.q[j] : 0.f;
            float3 mj = make_float3(0.f, 0.f, 0.f);
            if (a.ld) {
                double3 mm = a.mu[j];
                mj = make_float3((float)mm.x, (float)mm.y, (float)mm.z);
            }
            bool dip_j = (mj.x != 0.f) || (mj.y != 0.f) || (mj.z != 0.f);
            float dm1 = rsqrtf(d2), d = d2 * dm1;
            float dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2, dm7 = dm5 * dm2;
            float expon = expf(-alpha2 * d2) / rpi;
            float F0 = erfcf(alpha * d);
            float F1 = F0 + 2.f * alpha * d * expon;
            float F2 = F1 + (4.f / 3.f) * alpha3 * d2 * d * expon;
            float F1d1 = 0.f, F1d2 = 0.f, F2d1 = 0.f, F2d2 = 0.f;
            bool damp = false;
            if (a.ldamp) {
                const PairDamp &D = a.damp[ti * a.nt + a.typ[j]];
                if (D.ldamp) {
                    damp = true;
                    float fd1, fdd1, fd2, fdd2;
                    tt_damp32(a.tt, (float)D.b1, (float)D.c1, d, D.k1, fd1, fdd1);
                    tt_damp32(a.tt, (float)D.b2, (float)D.c2, d, D.k2, fd2, fdd2);
                    F1d1 = 1.f - fd1;
                    F1d2 = 1.f - fd2;
                    F2d1 = F1d1 + (d / 3.f) * fdd1;
                    F2d2 = F1d2 + (d / 3.f) * fdd2;
                }
            }
            float F1_dm3 = F1 * dm3, F2_dm5 = 3.f * F2 * dm5;
            float u = 0.f;
            float fij[3] = {0.f, 0.f, 0.f};
            if (a.lq) {
                u += qi * qj * (dm1 * F0);
                if (EF) {
                    float cfe = qj * dm3 * (F1 - F1d1);
                    ei[0] += cfe * r.x;
                    ei[1] += cfe * r.y;
                    ei[2] += cfe * r.z;
                }
                if (FORCES) {
                    float cf = -qi * qj * F1_dm3;
                    fij[0] = cf * r.x;
                    fij[1] = cf * r.y;
                    fij[2] = cf * r.z;
                }
            }
            float rmi = r.x * mi.x + r.y * mi.y + r.z * mi.z;
            float rmj = r.x * mj.x + r.y * mj.y + r.z * mj.z;
            if (a.ld && dip_i && dip_j) {
                float mmm = mi.x * mj.x + mi.y * mj.y + mi.z * mj.z;
                u += F1_dm3 * mmm - F2_dm5 * rmi * rmj;
                if (EF) {
                    ei[0] += F2_dm5 * rmj * r.x - F1_dm3 * mj.x;
                    ei[1] += F2_dm5 * rmj * r.y - F1_dm3 * mj.y;
                    ei[2] += F2_dm5 * rmj * r.z - F1_dm3 * mj.z;
                }
                if (FORCES) {
                    float F3 = F2 + (8.f / 15.f) * alpha3 * alpha2 * d2 * d2 * d * expon;
                    float c1 = -F3 * dm7 * 15.f * rmi * rmj, c2 = F2_dm5;
                    fij[0] -= c1 * r.x + c2 * (mmm * r.x + mi.x * rmj + mj.x * rmi);
                    fij[1] -= c1 * r.y + c2 * (mmm * r.y + mi.y * rmj + mj.y * rmi);
                    fij[2] -= c1 * r.z + c2 * (mmm * r.z + mi.z * rmj + mj.z * rmi);
                }
            }
            if (a.lq && a.ld && (dip_i || dip_j)) {
                u += F1_dm3 * (qi * rmj - qj * rmi);
                if (FORCES) {
                    float wx = qj * mi.x - qi * mj.x, wy = qj * mi.y - qi * mj.y, wz = qj * mi.z - qi * mj.z;
                    float rw = r.x * wx + r.y * wy + r.z * wz;
                    fij[0] += F2_dm5 * rw * r.x - F1_dm3 * wx;
                    fij[1] += F2_dm5 * rw * r.y - F1_dm3 * wy;
                    fij[2] += F2_dm5 * rw * r.z - F1_dm3 * wz;
                }
                if (damp) {
                    u += dm3 * (-qi * F1d2 * rmj + qj * F1d1 * rmi);
                    if (FORCES) {
                        float a1 = 3.f * F2d1 * dm5, b1 = F1d1 * dm3;
                        float a2 = 3.f * F2d2 * dm5, b2 = F1d2 * dm3;
                        fij[0] += -qj * (a1 * rmi * r.x - b1 * mi.x) + qi * (a2 * rmj * r.x - b2 * mj.x);
                        fij[1] += -qj * (a1 * rmi * r.y - b1 * mi.y) + qi * (a2 * rmj * r.y - b2 * mj.y);
                        fij[2] += -qj * (a1 * rmi * r.z - b1 * mi.z) + qi * (a2 * rmj * r.z - b2 * mj.z);
                    }
                }
            }
            acc[0] += u;
            if (FORCES) {
                fi[0] -= fij[0];
                fi[1] -= fij[1];
                fi[2] -= fij[2];
                acc[1] += -2.f * r.x * fij[0];
                acc[2] += -(r.x * fij[1] + r.y * fij[0]);
                acc[3] += -(r.x * fij[2] + r.z * fij[0]);
                acc[4] += -2.f * r.y * fij[1];
                acc[5] += -(r.y * fij[2] + r.z * fij[1]);
                acc[6] += -2.f * r.z * fij[2];
            }
        }
    }
    // FP64 across the warp
    double dacc[7], dfi[3], dei[3];
#pragma unroll
    for (int k = 0; k < 7; k++) dacc[k] = warp_sum((double)acc[k]);
    if (FORCES)
        for (int k = 0; k < 3; k++) dfi[k] = warp_sum((double)fi[k]);
    if (EF)
        for (int k = 0; k < 3; k++) dei[k] = warp_sum((double)ei[k]);
    if (i < a.n && lane == 0) {
        if (FORCES && a.f) a.f[i] = make_double3(dfi[0], dfi[1], dfi[2]);
        if (EF && a.ef) a.ef[i] = make_double3(dei[0], dei[1], dei[2]);
    }
    if (i >= a.n)
        for (int k = 0; k < 7; k++) dacc[k] = 0.0;
    if (a.part) {
        __shared__ double sh[PAIR_WARPS32][7];
        int w = threadIdx.x >> 5;
        if (lane == 0)
            for (int k = 0; k < 7; k++) sh[w][k] = dacc[k];
        __syncthreads();
        if (threadIdx.x < 7) {
            double t = 0.0;
            for (int k = 0; k < PAIR_WARPS32; k++) t += sh[k][threadIdx.x];
            a.part[(size_t)(a.slot + threadIdx.x) * a.stride + blockIdx.x] = t;
        }
    }
}

// cached dipole-field factors (F1/d^3, 3 F2/d^5) in FP32
__global__ void __launch_bounds__(PAIR_WARPS32 * 32) k_dir_prep32(int n, CellF c, const float4 *__restrict__ s,
                                                                 const int *__restrict__ col,
                                                                 const int *__restrict__ con, int cap,
                                                                 float lrcutsq, float alpha,
                                                                 float2 *__restrict__ coef) {
    int i = blockIdx.x * PAIR_WARPS32 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    const float rpi = 1.7724538509055160273f;
    const float alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
    float4 si = s[i];
    int m = min(con[i], cap);
    const int *L = col + (size_t)i * cap;
    float2 *C = coef + (size_t)i * cap;
    for (int k = lane; k < m; k += 32) {
        float4 sj = s[L[k]];
        float3 r = pbc32(c, si.x - sj.x, si.y - sj.y, si.z - sj.z);
        float d2 = r.x * r.x + r.y * r.y + r.z * r.z;
        float2 out = make_float2(0.f, 0.f);
        if (!(d2 > lrcutsq)) {
            float dm1 = rsqrtf(d2), d = d2 * dm1, dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2;
            float expon = expf(-alpha2 * d2) / rpi;
            float F0 = erfcf(alpha * d);
            float F1 = F0 + 2.f * alpha * d * expon;
            float F2 = F1 + (4.f / 3.f) * alpha3 * d2 * d * expon;
            out = make_float2(F1 * dm3, 3.f * F2 * dm5);
        }
        C[k] = out;
    }
}

__global__ void __launch_bounds__(PAIR_WARPS32 * 32) k_dir_field_cached32(int n, CellF c,
                                                                         const float4 *__restrict__ s,
                                                                         const int *__restrict__ col,
                                                                         const int *__restrict__ con, int cap,
                                                                         const float2 *__restrict__ coef,
                                                                         const double3 *__restrict__ mu,
                                                                         double3 *__restrict__ ef) {
    int i = blockIdx.x * PAIR_WARPS32 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    double3 mid = mu[i];
    bool dip_i = (mid.x != 0.0) || (mid.y != 0.0) || (mid.z != 0.0);
    float ex = 0.f, ey = 0.f, ez = 0.f;
    if (dip_i) {
        float4 si = s[i];
        int m = min(con[i], cap);
        const int *L = col + (size_t)i * cap;
        const float2 *C = coef + (size_t)i * cap;
        for (int k = lane; k < m; k += 32) {
            float2 cf = C[k];
            if (cf.x == 0.f && cf.y == 0.f) continue;
            int j = L[k];
            double3 mm = mu[j];
            if (mm.x == 0.0 && mm.y == 0.0 && mm.z == 0.0) continue;
            float3 mj = make_float3((float)mm.x, (float)mm.y, (float)mm.z);
            float4 sj = s[j];
            float3 r = pbc32(c, si.x - sj.x, si.y - sj.y, si.z - sj.z);
            float rmj = r.x * mj.x + r.y * mj.y + r.z * mj.z;
            ex += cf.y * rmj * r.x - cf.x * mj.x;
            ey += cf.y * rmj * r.y - cf.x * mj.y;
            ez += cf.y * rmj * r.z - cf.x * mj.z;
        }
    }
    double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
    if (lane == 0) ef[i] = make_double3(dx, dy, dz);
}

// ---------------------------------------------------------------- k space
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// exp(2 pi i u) for u already reduced to [-1/2, 1/2]
__device__ __forceinline__ float2 cis2pif(float u) {
    float sn, cs;
    sincospif(2.f * u, &sn, &cs);
    return make_float2(cs, sn);
}

template <bool LQ, bool LD>
__global__ void __launch_bounds__(RHO32_THREADS, 4) k_rho32(int n, int chunk, CellF c, int K0, int K1, int K2,
                                                          const float4 *__restrict__ t32,
                                                          const double *__restrict__ q,
                                                          const double3 *__restrict__ mu, int nseg,
                                                          const KSeg *__restrict__ seg, double2 *__restrict__ part,
                                                          int nk) {
    extern __shared__ float2 smf[];
    const int W0 = K0 + 1, W1 = 2 * K1 + 1, W2 = 2 * K2 + 1, WT = W0 + W1 + W2;
    float2 *E = smf;
    float *qs = (float *)(smf + RHO32_TI * WT);
    float *ms = qs + RHO32_TI;
    int sid = blockIdx.x * RHO32_THREADS + threadIdx.x;
    KSeg S;
    if (sid < nseg) S = seg[sid];
    else S.nx = S.ny = S.z0 = S.cnt = S.koff = 0;
    float2 acc[KSEG];   // FP32 over this block's ion chunk; chunks are combined in FP64
#pragma unroll
    for (int z = 0; z < KSEG; z++) acc[z] = make_float2(0.f, 0.f);
    int i0 = blockIdx.y * chunk, i1 = min(n, i0 + chunk);
    const float tpi = 6.2831853071795864770f;
    for (int t0 = i0; t0 < i1; t0 += RHO32_TI) {
        int nt = min(RHO32_TI, i1 - t0);
        if (threadIdx.x < 3 * RHO32_TI) {
            int slot = threadIdx.x % RHO32_TI, dim = threadIdx.x / RHO32_TI;
            if (slot < nt) {
                int ia = t0 + slot;
                float4 t = t32[ia];
                float td = dim == 0 ? t.x : (dim == 1 ? t.y : t.z);
                float2 e1 = cis2pif(td);
                float2 *T = E + slot * WT + (dim == 0 ? 0 : (dim == 1 ? W0 : W0 + W1));
                int K = dim == 0 ? K0 : (dim == 1 ? K1 : K2);
                int zero = dim == 0 ? 0 : K;
                float2 v = make_float2(1.f, 0.f);
                T[zero] = v;
                for (int m = 1; m <= K; m++) {
                    v = (m == 1) ? e1 : cmulf(v, e1);
                    T[zero + m] = v;
                    if (dim != 0) T[zero - m] = make_float2(v.x, -v.y);
                }
                if (dim == 0) {
                    qs[slot] = LQ ? (float)q[ia] : 0.f;
                    if (LD) {
                        double3 m3 = mu[ia];
                        double mx = c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z;
                        double my = c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z;
                        double mz = c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z;
                        ms[3 * slot] = tpi * (float)mx;
                        ms[3 * slot + 1] = tpi * (float)my;
                        ms[3 * slot + 2] = tpi * (float)mz;
                    }
                }
            }
        }
        __syncthreads();
        if (sid < nseg) {
            for (int a = 0; a < nt; a++) {
                const float2 *T = E + a * WT;
                float2 b = cmulf(T[S.nx], T[W0 + K1 + S.ny]);
                const float2 *Z = T + W0 + W1 + K2 + S.z0;
                float qa = LQ ? qs[a] : 0.f;
                float c0 = 0.f, c1 = 0.f;
                if (LD) {
                    c0 = (float)S.nx * ms[3 * a] + (float)S.ny * ms[3 * a + 1];
                    c1 = ms[3 * a + 2];
                }
                float2 B1 = make_float2(qa * b.x - c0 * b.y, qa * b.y + c0 * b.x);
                float2 B2 = make_float2(-c1 * b.y, c1 * b.x);
                float zf = (float)S.z0;
#pragma unroll
                for (int z = 0; z < KSEG; z++) {
                    if (z < S.cnt) {
                        float2 C = B1;
                        if (LD) {
                            C.x = B1.x + (zf + (float)z) * B2.x;
                            C.y = B1.y + (zf + (float)z) * B2.y;
                        }
                        float2 e = Z[z];
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
            if (z < S.cnt) P[z] = make_double2((double)acc[z].x, (double)acc[z].y);
    }
}

struct Ion32Args {
    int n, K2;
    Cell c;
    const float4 *t32;
    const double4 *r;
    const double3 *mu;
    const KRow *row;
    const int *tile_row, *tile_k;
    const double2 *rho_s;
    double *part;
    int ld;
};

template <bool WF>
__global__ void __launch_bounds__(ION32_THREADS) k_rec_ion32(Ion32Args a) {
    extern __shared__ float2 rkf[];
    int i = blockIdx.x * ION32_THREADS + threadIdx.x;
    int tl = blockIdx.y;
    bool act = i < a.n;
    int r0 = a.tile_row[tl], r1 = a.tile_row[tl + 1];
    int k0 = a.tile_k[tl], k1 = a.tile_k[tl + 1];
    for (int k = k0 + threadIdx.x; k < k1; k += ION32_THREADS) {
        double2 v = a.rho_s[k];
        rkf[k - k0] = make_float2((float)v.x, (float)v.y);
    }
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
    double tx = 0.0, ty = 0.0;
    float3 m = make_float3(0.f, 0.f, 0.f);
    if (act) {
        t = a.t32[i];
        double4 ri = a.r[i];
        tx = a.c.B[0][0] * ri.x + a.c.B[1][0] * ri.y + a.c.B[2][0] * ri.z;
        ty = a.c.B[0][1] * ri.x + a.c.B[1][1] * ri.y + a.c.B[2][1] * ri.z;
        if (WF && a.ld) {
            double3 mu = a.mu[i];
            m = make_float3((float)(a.c.B[0][0] * mu.x + a.c.B[1][0] * mu.y + a.c.B[2][0] * mu.z),
                            (float)(a.c.B[0][1] * mu.x + a.c.B[1][1] * mu.y + a.c.B[2][1] * mu.z),
                            (float)(a.c.B[0][2] * mu.x + a.c.B[1][2] * mu.y + a.c.B[2][2] * mu.z));
        }
    }
    __syncthreads();
    float2 e2 = cis2pif(t.z);
    float2 e22 = cmulf(e2, e2);
    float tzm = -(float)a.K2 * t.z;
    float2 e2m = cis2pif(tzm - rintf(tzm));
    double S0 = 0, S1 = 0, S2 = 0, P0 = 0, P1 = 0, P2 = 0;
    for (int rr = r0; rr < r1; rr++) {
        KRow R = a.row[rr];
        // row phase base reduced in FP64: exp(2 pi i (nx tx + ny ty))
        double u = (double)R.nx * tx + (double)R.ny * ty;
        float2 base = cis2pif((float)(u - rint(u)));
        float2 ph0 = (R.z0 == 1) ? cmulf(base, e2) : cmulf(base, e2m);
        float2 ph1 = cmulf(ph0, e2);
        const float2 *rho = rkf + (R.koff - k0);
        float R1 = 0.f, Rz = 0.f, T1 = 0.f, Tz = 0.f;
        float za = (float)R.z0, zb = za + 1.f;
        float c0 = (float)R.nx * m.x + (float)R.ny * m.y;
        int cnt = R.cnt;
        for (int kz = 0; kz < cnt; kz += 2) {
            float2 ra = rho[kz];
            float rca = ra.y * ph0.x - ra.x * ph0.y;
            R1 += rca;
            Rz += za * rca;
            if (WF) {
                float rc2 = ra.x * ph0.x + ra.y * ph0.y;
                float tq = (c0 + za * m.z) * rc2;
                T1 += tq;
                Tz += za * tq;
            }
            if (kz + 1 < cnt) {
                float2 rb = rho[kz + 1];
                float rcb = rb.y * ph1.x - rb.x * ph1.y;
                R1 += rcb;
                Rz += zb * rcb;
                if (WF) {
                    float rc2 = rb.x * ph1.x + rb.y * ph1.y;
                    float tq = (c0 + zb * m.z) * rc2;
                    T1 += tq;
                    Tz += zb * tq;
                }
            }
            ph0 = cmulf(ph0, e22);
            ph1 = cmulf(ph1, e22);
            za += 2.f;
            zb += 2.f;
        }
        double nx = (double)R.nx, ny = (double)R.ny;
        S0 += nx * (double)R1;
        S1 += ny * (double)R1;
        S2 += (double)Rz;
        if (WF) {
            P0 += nx * (double)T1;
            P1 += ny * (double)T1;
            P2 += (double)Tz;
        }
    }
    if (!act) return;
    double *o = a.part + ((size_t)tl * a.n + i) * ION32_NV;
    o[0] = S0;
    o[1] = S1;
    o[2] = S2;
    if (WF) {
        o[3] = P0;
        o[4] = P1;
        o[5] = P2;
    }
}

// ---------------------------------------------------------------- launchers
static CellF cellf(const Cell &c) {
    CellF f;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            f.A[i][j] = (float)c.A[i][j];
            f.B[i][j] = (float)c.B[i][j];
        }
    return f;
}

void launch_coords32(Engine &e) {
    MDFF_LAUNCH(e, k_coords32, ceil_div(e.n, 256), 256, 0, e.n, e.cell, e.d_r, e.d_s32, e.d_t32);
}

void launch_dir32(Engine &e, const double *q, const double3 *mu, double alpha, bool lq, bool ld, bool damp,
                  bool forces, bool ef, double3 *out_ef, double3 *out_f) {
    Dir32Args a;
    a.n = e.n;
    a.nt = e.nt;
    a.cap = e.cap_co;
    a.c = cellf(e.cell);
    a.s = e.d_s32;
    a.q = q;
    a.mu = mu;
    a.typ = e.d_typ;
    a.damp = e.d_damp;
    a.col = e.d_co;
    a.con = e.d_con;
    a.lrcutsq = (float)e.lrcutsq;
    a.alpha = (float)alpha;
    a.tt.E[0] = 1.f;
    for (int k = 1; k < 9; k++) a.tt.E[k] = a.tt.E[k - 1] / (float)k;
    a.lq = lq;
    a.ld = ld;
    a.ldamp = damp;
    a.ef = out_ef;
    a.f = out_f;
    a.part = e.d_part;
    a.slot = S_DIR_U;
    a.stride = e.part_stride;
    int nb = ceil_div(e.n, PAIR_WARPS32);
    int pd = -1;
    e.prof_begin("k_dir", &pd);
    if (forces)
        MDFF_LAUNCH(e, (k_dir32<true, false>), nb, PAIR_WARPS32 * 32, 0, a);
    else
        MDFF_LAUNCH(e, (k_dir32<false, true>), nb, PAIR_WARPS32 * 32, 0, a);
    e.prof_end("k_dir", pd, 0.0);
    (void)ef;
}

void launch_dir_prep32(Engine &e, double alpha) {
    int nb = ceil_div(e.n, PAIR_WARPS32);
    MDFF_LAUNCH(e, k_dir_prep32, nb, PAIR_WARPS32 * 32, 0, e.n, cellf(e.cell), e.d_s32, e.d_co, e.d_con, e.cap_co,
                (float)e.lrcutsq, (float)alpha, e.d_coef32);
}

void launch_dir_field_cached32(Engine &e, const double3 *mu, double3 *out_ef) {
    int nb = ceil_div(e.n, PAIR_WARPS32);
    int pd = -1;
    e.prof_begin("k_dir", &pd);
    MDFF_LAUNCH(e, k_dir_field_cached32, nb, PAIR_WARPS32 * 32, 0, e.n, cellf(e.cell), e.d_s32, e.d_co, e.d_con,
                e.cap_co, e.d_coef32, mu, out_ef);
    e.prof_end("k_dir", pd, 0.0);
}

// k_rec_combine and k_rho_reduce are shared with the FP64 path (kspace.cu)
struct IonArgs;
void launch_rec_tail(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const RecOut &o,
                     bool fp32_ion);
double rho_flops_per_pair(bool lq, bool ld);
double ion_flops_per_pair(bool f, bool efg);

void launch_rho32(Engine &e, const double *q, const double3 *mu, bool lq, bool ld) {
    int segblocks = ceil_div(e.nseg, RHO32_THREADS);
    dim3 grid(segblocks, e.rho_chunks);
    int WT = (e.kmax[0] + 1) + (2 * e.kmax[1] + 1) + (2 * e.kmax[2] + 1);
    size_t smem = sizeof(float2) * RHO32_TI * WT + sizeof(float) * RHO32_TI * 4;
    CellF cf = cellf(e.cell);
    int ps = -1;
    e.prof_begin("k_rho", &ps);
    if (lq && ld)
        MDFF_LAUNCH(e, (k_rho32<true, true>), grid, RHO32_THREADS, smem, e.n, e.rho_chunk, cf, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_t32, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    else if (lq)
        MDFF_LAUNCH(e, (k_rho32<true, false>), grid, RHO32_THREADS, smem, e.n, e.rho_chunk, cf, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_t32, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    else if (ld)
        MDFF_LAUNCH(e, (k_rho32<false, true>), grid, RHO32_THREADS, smem, e.n, e.rho_chunk, cf, e.kmax[0],
                    e.kmax[1], e.kmax[2], e.d_t32, q, mu, e.nseg, e.d_seg, e.d_rho_part, e.nk);
    else
        MDFF_CK(cudaMemsetAsync(e.d_rho_part, 0, sizeof(double2) * (size_t)e.nk * e.rho_chunks, e.stream));
    e.prof_end("k_rho", ps, (lq || ld) ? rho_flops_per_pair(lq, ld) * (double)e.n * e.nk : 0.0);
}

void launch_ion32(Engine &e, const double3 *mu, bool ld, bool want_f) {
    Ion32Args a;
    a.n = e.n;
    a.K2 = e.kmax[2];
    a.c = e.cell;
    a.t32 = e.d_t32;
    a.r = e.d_r;
    a.mu = mu;
    a.row = e.d_row;
    a.tile_row = e.d_tile_row;
    a.tile_k = e.d_tile_k;
    a.rho_s = e.d_rho;
    a.part = e.d_ion_part;
    a.ld = ld;
    size_t smem = sizeof(float2) * e.tile_kmax;
    dim3 g(ceil_div(e.n, ION32_THREADS), e.ntile);
    int pi = -1;
    e.prof_begin("k_rec_ion", &pi);
    if (want_f)
        MDFF_LAUNCH(e, (k_rec_ion32<true>), g, ION32_THREADS, smem, a);
    else
        MDFF_LAUNCH(e, (k_rec_ion32<false>), g, ION32_THREADS, smem, a);
    e.prof_end("k_rec_ion", pi, ion_flops_per_pair(want_f, false) * (double)e.n * e.nk);
}

}  // namespace mdffgpu
