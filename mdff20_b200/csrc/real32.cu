// Mixed-precision (MDFFGPU_MIXED) real-space Ewald sum: multipole_ES_dir
// (src/ewald.c:353-871) for charges and dipoles with Tang-Toennies damped charge-dipole
// terms, FP32 pair arithmetic.
//
// Per force evaluation k_pair_prep32 walks each ion's Coulomb Verlet list once and
//   * keeps the neighbours inside the real-space cutoff (the FP64 test of pair.cu on the
//     exact FP64 minimum image, so the pair set is the FP64 path's), in list order;
//   * for polarisable ion pairs stores the dipole-field tensor of the pair as
//     u = sqrt(3 F2/d^5) r and c1 = F1/d^3, so that T_ij p_j = (u.p_j) u - c1 p_j: the
//     induced-dipole iterations then cost one 16-byte record per pair.
// Every pair kernel forms the displacement from the FP64 fractional coordinates
// (exact minimum image, then one rounding to FP32), so positions carry no FP32 error;
// pair terms are summed in FP32 per lane and in FP64 across the warp.
#include "engine.cuh"

namespace mdffgpu {

constexpr int PW32 = 8;   // warps (= ions) per block

struct CellF3 {
    float A[3][3];
};

struct DampF {
    int ldamp, k1, k2, pad;
    float b1, c1, b2, c2;
};

// exact FP64 minimum image of s_i - s_j in fractional space, rounded once, times A (FP32)
__device__ __forceinline__ float3 disp32(const CellF3 &c, double4 si, double4 sj) {
    double dx = si.x - sj.x, dy = si.y - sj.y, dz = si.z - sj.z;
    float fx = (float)(dx - rint(dx)), fy = (float)(dy - rint(dy)), fz = (float)(dz - rint(dz));
    return make_float3(fx * c.A[0][0] + fy * c.A[1][0] + fz * c.A[2][0],
                       fx * c.A[0][1] + fy * c.A[1][1] + fz * c.A[2][1],
                       fx * c.A[0][2] + fy * c.A[1][2] + fz * c.A[2][2]);
}

// Tang-Toennies f_k(br) and its derivative (src/tt_damp.c:16-32) in FP32; K > 0 fixes
// the order at compile time, K = 0 reads it from `order`
template <int K>
__device__ __forceinline__ void tt32(float b, float c, float r, int order, float &f, float &fd) {
    float x = b * r;
    float ex = expf(-x) * c;
    float s, xk;
    if (K > 0) {
        float term = 1.f;
        s = 1.f;
#pragma unroll
        for (int m = 1; m <= K; m++) {
            term *= x * (1.f / (float)m);
            s += term;
        }
        xk = term;   // x^K / K!
    } else {
        float term = 1.f;
        s = 1.f;
        for (int m = 1; m <= order; m++) {
            term *= x / (float)m;
            s += term;
        }
        xk = term;
    }
    f = 1.f - s * ex;
    fd = xk * ex * b;
}

__global__ void k_pack_mu32(int n, const double3 *__restrict__ mu, const int *__restrict__ typ,
                            float4 *__restrict__ out) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double3 m = mu ? mu[i] : make_double3(0, 0, 0);
    out[i] = make_float4((float)m.x, (float)m.y, (float)m.z, (float)typ[i]);
}

struct Prep32Args {
    int n;
    Cell c;
    const double4 *s;
    const int *col, *con;    // Coulomb Verlet list
    int cap;
    double lrcutsq;
    float alpha;
    const int *polar;
    int *nl, *nln, *pl, *pln;
    float4 *pu;
};

// warp per ion: in-cutoff list nl (all ions) and dipole-field records (polarisable pairs).
// The neighbour positions of the next chunk of 32 and the indices of the one after are
// loaded while the current chunk is processed.
__global__ void __launch_bounds__(PW32 * 32) k_pair_prep32(Prep32Args a) {
    grid_dep();
    int i = blockIdx.x * PW32 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const float irpi = 0.56418958354775628695f;   // 1 / sqrt(pi): a product, not a division
    const float alpha = a.alpha, alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
    const Cell &c = a.c;
    double4 si = a.s[i];
    bool pi = a.polar && a.polar[i];
    int m = min(a.con[i], a.cap);
    const int *L = a.col + (size_t)i * a.cap;
    int *NL = a.nl + (size_t)i * a.cap;
    int *PL = a.pl ? a.pl + (size_t)i * a.cap : nullptr;
    float4 *PU = a.pu ? a.pu + (size_t)i * a.cap : nullptr;
    int cnt = 0, pcnt = 0;
    // software pipeline: positions one chunk ahead, indices two chunks ahead
    int jc = lane < m ? L[lane] : 0;
    int jn = lane + 32 < m ? L[lane + 32] : 0;
    double4 sc = lane < m ? a.s[jc] : si;
    for (int k0 = 0; k0 < m; k0 += 32) {
        int k = k0 + lane;
        int j = jc;
        double4 sj = sc;
        if (k + 32 < m) sc = a.s[jn];
        jc = jn;
        if (k + 64 < m) jn = L[k + 64];
        bool keep = false, kp = false;
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < m) {
            double3 r = pbc_frac(c, si.x - sj.x, si.y - sj.y, si.z - sj.z);
            double d2 = norm2_exact(r);
            keep = !(d2 > a.lrcutsq);
            if (keep && pi && a.polar[j]) {
                kp = true;
                float3 rf = make_float3((float)r.x, (float)r.y, (float)r.z);
                float fd2 = (float)d2;
                float dm1 = rsqrtf(fd2), d = fd2 * dm1, dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2;
                float expon = expf(-alpha2 * fd2) * irpi;
                float F0 = erfcf(alpha * d);
                float F1 = F0 + 2.f * alpha * d * expon;
                float F2 = F1 + (4.f / 3.f) * alpha3 * fd2 * d * expon;
                float g = sqrtf(3.f * F2 * dm5);
                rec = make_float4(g * rf.x, g * rf.y, g * rf.z, F1 * dm3);
            }
        }
        const unsigned below = (1u << lane) - 1u;
        unsigned bk = __ballot_sync(0xffffffffu, keep);
        if (keep) NL[cnt + __popc(bk & below)] = j;
        cnt += __popc(bk);
        if (PL) {
            unsigned bp = __ballot_sync(0xffffffffu, kp);
            if (kp) {
                int pos = pcnt + __popc(bp & below);
                PL[pos] = j;
                PU[pos] = rec;
            }
            pcnt += __popc(bp);
        }
    }
    if (lane == 0) {
        a.nln[i] = cnt;
        if (a.pln) a.pln[i] = pcnt;
    }
}

// induced-dipole field T p at ion i from the dipole-field records: sum_j (u.p_j) u - c1 p_j
__global__ void __launch_bounds__(PW32 * 32) k_pol_field32(int n, const int *__restrict__ pl,
                                                           const float4 *__restrict__ pu,
                                                           const int *__restrict__ pln, int cap,
                                                           const double3 *__restrict__ p,
                                                           double3 *__restrict__ ef) {
    grid_dep();
    int i = blockIdx.x * PW32 + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    int m = pln[i];
    const int *L = pl + (size_t)i * cap;
    const float4 *U = pu + (size_t)i * cap;
    float ex = 0.f, ey = 0.f, ez = 0.f;
    // four records per lane in flight: their indices, records and dipole gathers are
    // issued before any of them is used (the walk is bound by these loads)
    constexpr int R = 4;
    for (int k0 = lane; k0 < m; k0 += 32 * R) {
        int j[R];
        float4 u[R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int k = k0 + 32 * r;
            j[r] = k < m ? L[k] : -1;
            u[r] = k < m ? U[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        double3 pd[R];
#pragma unroll
        for (int r = 0; r < R; r++) pd[r] = j[r] >= 0 ? p[j[r]] : make_double3(0.0, 0.0, 0.0);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const float px = (float)pd[r].x, py = (float)pd[r].y, pz = (float)pd[r].z;
            const float up = u[r].x * px + u[r].y * py + u[r].z * pz;
            ex += up * u[r].x - u[r].w * px;
            ey += up * u[r].y - u[r].w * py;
            ez += up * u[r].z - u[r].w * pz;
        }
    }
    double dx = warp_sum((double)ex), dy = warp_sum((double)ey), dz = warp_sum((double)ez);
    if (lane == 0) ef[i] = make_double3(dx, dy, dz);
}

struct Dir32bArgs {
    int n, nt, cap;
    const int *idx;        // field only: these ions (cnt of them), all when null
    int cnt;
    CellF3 c;
    const double4 *s;      // fractional coordinates, w = charge
    const float4 *qm;      // dipole, w = type
    const int *typ;
    const PairDamp *damp;
    const int *nl, *nln;
    float alpha;
    int lq, ld, ldamp;
    double3 *ef, *f;
    double *part;
    int slot, stride;
};

// multipole_ES_dir over the in-cutoff list: field (EF) or forces + energy + virial (FORCES)
template <bool FORCES, bool EF, int KTT>
__global__ void __launch_bounds__(PW32 * 32) k_dir32b(Dir32bArgs a) {
    grid_dep();
    __shared__ DampF dt[NT * NT];
    for (int e = threadIdx.x; e < a.nt * a.nt; e += blockDim.x) {
        PairDamp D = a.damp[e];
        DampF F;
        F.ldamp = D.ldamp;
        F.k1 = D.k1;
        F.k2 = D.k2;
        F.pad = 0;
        F.b1 = (float)D.b1;
        F.c1 = (float)D.c1;
        F.b2 = (float)D.b2;
        F.c2 = (float)D.c2;
        dt[e] = F;
    }
    __syncthreads();
    int wi = blockIdx.x * PW32 + (threadIdx.x >> 5);
    int i = wi;
    if (a.idx) i = (wi < a.cnt) ? a.idx[wi] : a.n;
    int lane = threadIdx.x & 31;
    float acc[7] = {0, 0, 0, 0, 0, 0, 0};
    float fi[3] = {0, 0, 0}, ei[3] = {0, 0, 0};
    const float alpha = a.alpha, alpha2 = alpha * alpha, alpha3 = alpha2 * alpha;
    const float irpi = 0.56418958354775628695f;   // 1 / sqrt(pi): a product, not a division
    if (i < a.n) {
        double4 si = a.s[i];
        float qi = a.lq ? (float)si.w : 0.f;
        float3 mi = make_float3(0.f, 0.f, 0.f);
        if (a.ld) {
            float4 m4 = a.qm[i];
            mi = make_float3(m4.x, m4.y, m4.z);
        }
        bool dip_i = (mi.x != 0.f) || (mi.y != 0.f) || (mi.z != 0.f);
        const DampF *Drow = dt + a.typ[i] * a.nt;
        int m = a.nln[i];
        const int *L = a.nl + (size_t)i * a.cap;
        // neighbour positions and dipoles one round ahead, indices two rounds ahead
        int jc = lane < m ? L[lane] : 0;
        int jn = lane + 32 < m ? L[lane + 32] : 0;
        double4 sc = lane < m ? a.s[jc] : si;
        float4 qc = (a.ld && lane < m) ? a.qm[jc] : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int k = lane; k < m; k += 32) {
            int j = jc;
            double4 sj = sc;
            float4 m4 = qc;
            if (k + 32 < m) {
                sc = a.s[jn];
                if (a.ld) qc = a.qm[jn];
            }
            jc = jn;
            if (k + 64 < m) jn = L[k + 64];
            float3 r = disp32(a.c, si, sj);
            float d2 = r.x * r.x + r.y * r.y + r.z * r.z;
            float qj = a.lq ? (float)sj.w : 0.f;
            float3 mj = make_float3(0.f, 0.f, 0.f);
            int tj = 0;
            if (a.ld) {
                mj = make_float3(m4.x, m4.y, m4.z);
                tj = (int)m4.w;
            } else if (a.ldamp) {
                tj = a.typ[j];
            }
            bool dip_j = (mj.x != 0.f) || (mj.y != 0.f) || (mj.z != 0.f);
            float dm1 = rsqrtf(d2), d = d2 * dm1;
            float dm2 = dm1 * dm1, dm3 = dm1 * dm2, dm5 = dm3 * dm2;
            float expon = expf(-alpha2 * d2) * irpi;
            float F0 = erfcf(alpha * d);
            float F1 = F0 + 2.f * alpha * d * expon;
            float F2 = F1 + (4.f / 3.f) * alpha3 * d2 * d * expon;
            float F1d1 = 0.f, F1d2 = 0.f, F2d1 = 0.f, F2d2 = 0.f;
            bool damp = false;
            if (a.ldamp) {
                DampF D = Drow[tj];
                if (D.ldamp) {
                    damp = true;
                    float fd1, fdd1, fd2, fdd2;
                    tt32<KTT>(D.b1, D.c1, d, D.k1, fd1, fdd1);
                    tt32<KTT>(D.b2, D.c2, d, D.k2, fd2, fdd2);
                    F1d1 = 1.f - fd1;
                    F1d2 = 1.f - fd2;
                    F2d1 = F1d1 + (d * (1.f / 3.f)) * fdd1;
                    F2d2 = F1d2 + (d * (1.f / 3.f)) * fdd2;
                }
            }
            float F1_dm3 = F1 * dm3, F2_dm5 = 3.f * F2 * dm5;
            float u = 0.f;
            float fij[3] = {0.f, 0.f, 0.f};
            if (a.lq) {
                if (FORCES) u += qi * qj * (dm1 * F0);
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
                if (FORCES) u += F1_dm3 * mmm - F2_dm5 * rmi * rmj;
                if (EF) {
                    ei[0] += F2_dm5 * rmj * r.x - F1_dm3 * mj.x;
                    ei[1] += F2_dm5 * rmj * r.y - F1_dm3 * mj.y;
                    ei[2] += F2_dm5 * rmj * r.z - F1_dm3 * mj.z;
                }
                if (FORCES) {
                    float dm7 = dm5 * dm2;
                    float F3 = F2 + (8.f / 15.f) * alpha3 * alpha2 * d2 * d2 * d * expon;
                    float c1 = -F3 * dm7 * 15.f * rmi * rmj, c2 = F2_dm5;
                    fij[0] -= c1 * r.x + c2 * (mmm * r.x + mi.x * rmj + mj.x * rmi);
                    fij[1] -= c1 * r.y + c2 * (mmm * r.y + mi.y * rmj + mj.y * rmi);
                    fij[2] -= c1 * r.z + c2 * (mmm * r.z + mi.z * rmj + mj.z * rmi);
                }
            }
            if (FORCES && a.lq && a.ld && (dip_i || dip_j)) {
                u += F1_dm3 * (qi * rmj - qj * rmi);
                float wx = qj * mi.x - qi * mj.x, wy = qj * mi.y - qi * mj.y, wz = qj * mi.z - qi * mj.z;
                float rw = r.x * wx + r.y * wy + r.z * wz;
                fij[0] += F2_dm5 * rw * r.x - F1_dm3 * wx;
                fij[1] += F2_dm5 * rw * r.y - F1_dm3 * wy;
                fij[2] += F2_dm5 * rw * r.z - F1_dm3 * wz;
                if (damp) {
                    u += dm3 * (-qi * F1d2 * rmj + qj * F1d1 * rmi);
                    float a1 = 3.f * F2d1 * dm5, b1 = F1d1 * dm3;
                    float a2 = 3.f * F2d2 * dm5, b2 = F1d2 * dm3;
                    fij[0] += -qj * (a1 * rmi * r.x - b1 * mi.x) + qi * (a2 * rmj * r.x - b2 * mj.x);
                    fij[1] += -qj * (a1 * rmi * r.y - b1 * mi.y) + qi * (a2 * rmj * r.y - b2 * mj.y);
                    fij[2] += -qj * (a1 * rmi * r.z - b1 * mi.z) + qi * (a2 * rmj * r.z - b2 * mj.z);
                }
            }
            if (FORCES) {
                acc[0] += u;
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
    double dfi[3], dei[3];
    if (FORCES)
        for (int k = 0; k < 3; k++) dfi[k] = warp_sum((double)fi[k]);
    if (EF)
        for (int k = 0; k < 3; k++) dei[k] = warp_sum((double)ei[k]);
    if (i < a.n && lane == 0) {
        if (FORCES && a.f) a.f[i] = make_double3(dfi[0], dfi[1], dfi[2]);
        if (EF && a.ef) a.ef[i] = make_double3(dei[0], dei[1], dei[2]);
    }
    if (FORCES && a.part) {
        double dacc[7];
#pragma unroll
        for (int k = 0; k < 7; k++) dacc[k] = warp_sum((double)acc[k]);
        __shared__ double sh[PW32][7];
        int w = threadIdx.x >> 5;
        if (lane == 0)
            for (int k = 0; k < 7; k++) sh[w][k] = (i < a.n) ? dacc[k] : 0.0;
        __syncthreads();
        if (threadIdx.x < 7) {
            double t = 0.0;
            for (int k = 0; k < PW32; k++) t += sh[k][threadIdx.x];
            a.part[(size_t)(a.slot + threadIdx.x) * a.stride + blockIdx.x] = t;
        }
    }
}

// ---------------------------------------------------------------- launchers
static CellF3 cellf3(const Cell &c) {
    CellF3 f;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) f.A[i][j] = (float)c.A[i][j];
    return f;
}

void Engine::ensure_real32() {
    if (d_nl32 && cap32 == cap_co) return;
    if (capturing) throw Error(MDFFGPU_ERR_STATE, "mixed-precision pair buffers allocated while recording");
    dfree32();
    cap32 = cap_co;
    gen++;
    d_nl32 = dalloc<int>((size_t)n * cap_co);
    d_nln32 = dalloc<int>(n);
    d_qm32 = dalloc<float4>(n);
    if (lpol) {
        d_pl32 = dalloc<int>((size_t)n * cap_co);
        d_pu32 = dalloc<float4>((size_t)n * cap_co);
        d_pln32 = dalloc<int>(n);
    }
}

void Engine::dfree32() {
    cudaFree(d_nl32);
    cudaFree(d_nln32);
    cudaFree(d_qm32);
    cudaFree(d_pl32);
    cudaFree(d_pu32);
    cudaFree(d_pln32);
    d_nl32 = d_nln32 = d_pl32 = d_pln32 = nullptr;
    d_qm32 = d_pu32 = nullptr;
    cap32 = 0;
}

// per force evaluation, after the fractional coordinates e.d_s are current
void launch_pair_prep32(Engine &e) {
    e.ensure_real32();
    Prep32Args a;
    a.n = e.n;
    a.c = e.cell;
    a.s = e.d_s;
    a.col = e.d_co;
    a.con = e.d_con;
    a.cap = e.cap_co;
    a.lrcutsq = e.lrcutsq;
    a.alpha = (float)e.p.alphaES;
    a.polar = e.lpol ? e.d_polar : nullptr;
    a.nl = e.d_nl32;
    a.nln = e.d_nln32;
    a.pl = e.d_pl32;
    a.pln = e.d_pln32;
    a.pu = e.d_pu32;
    MDFF_LAUNCH(e, k_pair_prep32, ceil_div(e.n, PW32), PW32 * 32, 0, a);
}

void launch_pol_field32(Engine &e, const double3 *p, double3 *out_ef) {
    int nb = ceil_div(e.n, PW32);
    int pd = -1;
    e.prof_begin("k_dir", &pd);
    MDFF_LAUNCH(e, k_pol_field32, nb, PW32 * 32, 0, e.n, e.d_pl32, e.d_pu32, e.d_pln32, e.cap_co, p, out_ef);
    e.prof_end("k_dir", pd, 0.0);
}

// 4 when every Tang-Toennies function the pair kernel evaluates has order 4 or c = 0
// (then f = 1 and f' = 0 whatever the order), else 0 (order read per pair)
static int uniform_tt_order(const Engine &e) {
    for (int a = 0; a < e.nt; a++)
        for (int b = 0; b < e.nt; b++) {
            if (!(e.p.lpoldamping[a][a][b] || e.p.lpoldamping[b][a][b])) continue;
            if (e.p.pol_damp_c[a][a][b] != 0.0 && e.p.pol_damp_k[a][a][b] != 4) return 0;
            if (e.p.pol_damp_c[b][a][b] != 0.0 && e.p.pol_damp_k[b][a][b] != 4) return 0;
        }
    return 4;
}

template <bool FORCES, bool EF>
static void dir32_launch(Engine &e, const Dir32bArgs &a, int ktt) {
    int nb = ceil_div(a.idx ? a.cnt : e.n, PW32);
    if (ktt == 4) MDFF_LAUNCH(e, (k_dir32b<FORCES, EF, 4>), nb, PW32 * 32, 0, a);
    else MDFF_LAUNCH(e, (k_dir32b<FORCES, EF, 0>), nb, PW32 * 32, 0, a);
}

void launch_dir32(Engine &e, const double *q, const double3 *mu, double alpha, bool lq, bool ld, bool damp,
                  bool forces, bool ef, double3 *out_ef, double3 *out_f, const int *idx, int cnt) {
    if (idx && forces) throw Error(MDFFGPU_ERR_STATE, "ion subsets are for field-only passes");
    (void)q;   // charges travel in the w component of the fractional coordinates
    if (ld) MDFF_LAUNCH(e, k_pack_mu32, ceil_div(e.n, 256), 256, 0, e.n, mu, e.d_typ, e.d_qm32);
    Dir32bArgs a;
    a.n = e.n;
    a.idx = idx;
    a.cnt = idx ? cnt : e.n;
    a.nt = e.nt;
    a.cap = e.cap_co;
    a.c = cellf3(e.cell);
    a.s = e.d_s;
    a.qm = e.d_qm32;
    a.typ = e.d_typ;
    a.damp = e.d_damp;
    a.nl = e.d_nl32;
    a.nln = e.d_nln32;
    a.alpha = (float)alpha;
    a.lq = lq;
    a.ld = ld;
    a.ldamp = damp;
    a.ef = out_ef;
    a.f = out_f;
    a.part = e.d_part;
    a.slot = S_DIR_U;
    a.stride = e.part_stride;
    int ktt = uniform_tt_order(e);
    int pd = -1;
    e.prof_begin("k_dir", &pd);
    if (forces) dir32_launch<true, false>(e, a, ktt);
    else dir32_launch<false, true>(e, a, ktt);
    e.prof_end("k_dir", pd, 0.0);
    (void)ef;
}

}  // namespace mdffgpu
