// The ion pass of the mixed-precision reciprocal sum on the 5th-generation tensor cores
// (tcgen05, sm_100a): the field (and force) k-sums of kspace32.cu's k_ion32 as a TF32
// matrix product with FP32 accumulation in tensor memory.
//
// Per row (nx, ny) of the k-set the ion pass needs, for every ion, the complex z-sums
//     G = rho_0 + sum_z (a1 c_z + a2 d_z) + i (a3 c_z + a4 d_z)
//     H = sum_z z (-a4 c_z + a3 d_z) + i z (a2 c_z - a1 d_z)
//     K = sum_z z^2 (a1 c_z + a2 d_z) + i z^2 (a3 c_z + a4 d_z)        (forces only)
// with E2[z] = (c_z, d_z) = exp(2 pi i z t_z) of the ion and a1..a4 the weights of
// Ak rho(+z) and Ak rho(-z) folded over the sign of nz (kspace32.cu).  Their real and
// imaginary parts are one real product
//     D[ion][(row, comp)] = sum_k V[ion][k] W[(row, comp)][k],
//     V = (c_1..c_K2, d_1..d_K2, 1, 0 ...)   (32 values per ion, fixed while the
//                                             positions are: one table per force evaluation)
//     W = the matching weights of Gx, Gy, Hx, Hy (Kx, Ky)   (per pass, from Ak rho)
// Every value x is split as x = h + l, both TF32, and the product taken as
// V_h W_h + V_h W_l + V_l W_h (K = 96), the dropped l l term 2^-22 of it.
//
// CTA = 128 ions (one tensor-memory lane each) and a slice of rows; 10 warps.  Warp 8
// copies the ions' operand tile once and the weight chunks of IT_RPC rows into two
// shared-memory buffers (bulk copies completing on mbarriers), warp 9 issues the 12 MMAs
// (M = 128, N = IT_RPC x components, K = 8) of each chunk into one of two accumulators
// in tensor memory and commits them, warps 0-7 read an accumulator back (tcgen05.ld;
// warp w takes the lanes of quarter w % 4 and half w / 4 of the chunk's rows) while the
// next chunk's MMAs run, and finish the rows as the CUDA-core pass does: the row phase w
// (an FP64-reduced argument every IT_RUN rows, FP32 steps in ny between), Im conj(w) G and
// Im conj(w) H (and the Re parts with the ion's dipole for forces), FP32 sums over a
// warp's rows of a chunk, FP64 across chunks.  Each (slice, half) goes to the partial
// buffer of k_ion32 as a slice of its own, summed per ion by k_combine32.  The field pass
// (96 KB of shared memory) runs two CTAs per SM, 16 row warps per SM.
//
// Every mbarrier wait is bounded: on expiry the kernel sets ST_TC_TIMEOUT, stops issuing,
// waits (bounded) for the copies and MMAs it has in flight, frees its tensor memory and
// returns; the host turns the flag into MDFFGPU_ERR_TIMEOUT.
#include <mutex>

#include "engine.cuh"
#include "tc_common.cuh"

namespace mdffgpu {

constexpr int IT_M = 128;          // ions per tile: MMA M, one tensor-memory lane each
constexpr int IT_KV = 32;          // operand values per ion: c_1..c_K2, d_1..d_K2, 1, zeros
constexpr int IT_K = 3 * IT_KV;    // K of one chunk's product: (h, h, l) x (h, l, h)
constexpr int IT_RPC = 16;         // k-rows per weight chunk
constexpr int IT_EPI = 8;          // row warps: lane quarter w % 4, half w / 4 of a chunk's rows
constexpr int IT_HALF = IT_RPC / 2;
constexpr int IT_THREADS = 32 * (IT_EPI + 2);   // + one copy warp, one MMA warp
constexpr int IT_RUN = 4;          // rows per exact row phase, as in the CUDA-core pass
constexpr int IT_MAXK2 = (IT_KV - 1) / 2;            // nz up to 15
constexpr uint32_t IT_A_LBO = (IT_M / 8) * 128;      // 16-byte K chunk stride of the ion tile
constexpr uint32_t IT_A_BYTES = (IT_K / 4) * IT_A_LBO;   // 48 KB
constexpr uint32_t IT_COPY = 16384;                  // bytes per bulk copy

template <int NC>
struct ItShape {
    static constexpr int N = IT_RPC * NC;                        // MMA N: (row, component)
    static constexpr uint32_t LBO = (N / 8) * 128;
    static constexpr uint32_t BYTES = (IT_K / 4) * LBO;          // one weight chunk
    static constexpr uint32_t TMEM_COLS = (2 * N <= 128) ? 128u : ((2 * N <= 256) ? 256u : 512u);   // two accumulators
    static constexpr size_t SMEM = IT_A_BYTES + 2 * (size_t)BYTES;
    static constexpr int MINB = SMEM <= 100 * 1024 ? 2 : 1;      // resident CTAs per SM
};

// ---------------------------------------------------------------- operands
// per position j (ion order[j]): V of E2[z] = exp(2 pi i z t_z) from FP64-reduced
// arguments, split into TF32 h + l, stored as the K-major no-swizzle operand tile of its
// 128 positions with K = (h | h | l)
__global__ void k_ion_tc_table(int n, int K2, Cell c, const double4 *__restrict__ r, const int *__restrict__ order,
                               float4 *__restrict__ atab) {
    grid_dep();
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double4 ri = r[order[j]];
    double tz = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
    float h[IT_KV], l[IT_KV];
#pragma unroll
    for (int k = 0; k < IT_KV; k++) {
        float v = 0.f;
        if (k < 2 * K2) {
            int z = k < K2 ? k + 1 : k - K2 + 1;
            float2 e = cis2pi32((double)z * tz);
            v = k < K2 ? e.x : e.y;
        } else if (k == 2 * K2) {
            v = 1.f;
        }
        split2(v, h[k], l[k]);
    }
    unsigned char *T = (unsigned char *)atab + (size_t)(j / IT_M) * IT_A_BYTES;
    const int x = j % IT_M;
#pragma unroll
    for (int kg = 0; kg < IT_K / 4; kg++) {
        const int t = kg / (IT_KV / 4), v0 = (kg % (IT_KV / 4)) * 4;
        const float *s = t == 2 ? l : h;
        *(float4 *)(T + kmaj(x, 4 * kg, IT_A_LBO)) = make_float4(s[v0], s[v0 + 1], s[v0 + 2], s[v0 + 3]);
    }
}

// per pass: the weights of every (row, component) from Ak rho(k), as K-major chunks of
// IT_RPC rows with K = (h | l | h); rows past nrow are zero.  Components: Gx, Gy, Hx,
// Hy (and Kx, Ky): the coefficients of c_z, of d_z and of the constant 1 in the sums above.
// One thread per (chunk, row-component, group of 4 of the 32 values).
template <int NC>
__global__ void k_ion_tc_weights(int nrow, int nchunk, int K2, const KRow *__restrict__ row,
                                 const double2 *__restrict__ rho, float4 *__restrict__ wtab) {
    grid_dep();
    using S = ItShape<NC>;
    constexpr int G = IT_KV / 4;
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nchunk * S::N * G) return;
    const int grp = g % G, t = g / G;
    const int ch = t / S::N, nn = t - ch * S::N;
    const int rloc = nn / NC, comp = nn - rloc * NC, rr = ch * IT_RPC + rloc;
    KRow R;
    R.nx = R.ny = R.z0 = R.cnt = R.koff = 0;
    const bool ok = rr < nrow;
    if (ok) R = row[rr];
    const int zlo = R.z0, zhi = R.z0 + R.cnt - 1;
    auto rho_at = [&](int z) {
        if (!ok || z < zlo || z > zhi) return make_double2(0.0, 0.0);
        return rho[R.koff + z - zlo];
    };
    float h[4], l[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int k = grp * 4 + u;
        double v = 0.0;
        if (k < 2 * K2) {
            const bool cpart = k < K2;
            const int z = cpart ? k + 1 : k - K2 + 1;
            const double2 rp = rho_at(z), rn = rho_at(-z);
            const double a1 = rp.x + rn.x, a2 = rp.y - rn.y, a3 = rp.y + rn.y, a4 = rn.x - rp.x;
            const double fz = (double)z;
            switch (comp) {
            case 0: v = cpart ? a1 : a2; break;
            case 1: v = cpart ? a3 : a4; break;
            case 2: v = cpart ? -fz * a4 : fz * a3; break;
            case 3: v = cpart ? fz * a2 : -fz * a1; break;
            case 4: v = fz * fz * (cpart ? a1 : a2); break;
            default: v = fz * fz * (cpart ? a3 : a4); break;
            }
        } else if (k == 2 * K2 && comp < 2) {
            const double2 r0 = rho_at(0);
            v = comp == 0 ? r0.x : r0.y;
        }
        split2((float)v, h[u], l[u]);
    }
    unsigned char *T = (unsigned char *)wtab + (size_t)ch * S::BYTES;
    const float4 hv = make_float4(h[0], h[1], h[2], h[3]), lv = make_float4(l[0], l[1], l[2], l[3]);
    *(float4 *)(T + kmaj(nn, grp * 4, S::LBO)) = hv;
    *(float4 *)(T + kmaj(nn, IT_KV + grp * 4, S::LBO)) = lv;
    *(float4 *)(T + kmaj(nn, 2 * IT_KV + grp * 4, S::LBO)) = hv;
}

// ---------------------------------------------------------------- the pass
struct IonTcArgs {
    int cnt;                 // positions 0..cnt-1 of order
    int nrow, rows_per_slice;   // rows_per_slice: a multiple of IT_RPC
    int ld;
    const int *order;
    Cell c;
    const double4 *r;
    const double3 *mu;
    const KRow *row;
    const float4 *atab, *wtab;
    double *part;            // [slice][cnt][3 or 6], as k_ion32
    unsigned *status;
};

template <int NC>
__global__ void __launch_bounds__(IT_THREADS, ItShape<NC>::MINB) k_ion_tc(IonTcArgs a) {
    grid_dep();
    using S = ItShape<NC>;
    constexpr bool WF = NC == 6;
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm;                                   // the ion tile
    unsigned char *sB = sm + IT_A_BYTES;                      // [2] weight chunks
    // per row of the slice: (nx, ny, 1 when the row continues the one before it in its
    // row warp's group of IT_HALF -- same nx, ny one higher --, 0)
    float4 *rowf = (float4 *)(sB + 2 * S::BYTES);
    uint64_t *bar = (uint64_t *)(rowf + a.rows_per_slice);
    // bar: 0 tile landed, 1-2 chunk landed, 3-4 chunk consumed, 5-6 accumulator ready,
    // 7-8 accumulator read (one arrival per row warp)
    volatile int *abort_flag = (volatile int *)(bar + 9);
    uint32_t *tmem_slot = (uint32_t *)(bar + 10);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int sl = blockIdx.y;
    const int r0 = sl * a.rows_per_slice, nrs = max(0, min(a.nrow, r0 + a.rows_per_slice) - r0);
    const int nch = (nrs + IT_RPC - 1) / IT_RPC, ch0 = r0 / IT_RPC;

    for (int e = tid; e < nrs; e += IT_THREADS) {
        const KRow R = a.row[r0 + e];
        bool step = false;
        if (e % IT_HALF != 0) {
            const KRow Q = a.row[r0 + e - 1];
            step = R.nx == Q.nx && R.ny == Q.ny + 1;
        }
        rowf[e] = make_float4((float)R.nx, (float)R.ny, step ? 1.f : 0.f, 0.f);
    }
    if (tid == 0) {
        mbar_init(smem_u32(&bar[0]), 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&bar[1 + b]), 1);
            mbar_init(smem_u32(&bar[3 + b]), 1);
            mbar_init(smem_u32(&bar[5 + b]), 1);
            mbar_init(smem_u32(&bar[7 + b]), IT_EPI);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(S::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    auto fail = [&]() {
        if (!*abort_flag) atomicOr(a.status, (unsigned)ST_TC_TIMEOUT);
        *abort_flag = 1;
    };

    if (warp == IT_EPI) {
        // ------------------------------------------------ copies
        if (lane == 0) {
            const uint32_t ba = smem_u32(&bar[0]);
            mbar_expect_tx(ba, IT_A_BYTES);
            const unsigned char *gA = (const unsigned char *)a.atab + (size_t)blockIdx.x * IT_A_BYTES;
            for (uint32_t o = 0; o < IT_A_BYTES; o += IT_COPY) bulk_g2s(smem_u32(sA) + o, gA + o, IT_COPY, ba);
            int issued = 0;
            for (int c = 0; c < nch && !*abort_flag; c++) {
                const int b = c & 1;
                if (c >= 2 && !mbar_wait(smem_u32(&bar[3 + b]), ((c >> 1) - 1) & 1)) {
                    fail();
                    break;
                }
                const uint32_t bf = smem_u32(&bar[1 + b]);
                mbar_expect_tx(bf, S::BYTES);
                const unsigned char *gB = (const unsigned char *)a.wtab + (size_t)(ch0 + c) * S::BYTES;
                for (uint32_t o = 0; o < S::BYTES; o += IT_COPY) {
                    const uint32_t sz = S::BYTES - o < IT_COPY ? S::BYTES - o : IT_COPY;
                    bulk_g2s(smem_u32(sB + b * S::BYTES) + o, gB + o, sz, bf);
                }
                issued = c + 1;
            }
            // nothing may land after the CTA is gone: wait (bounded) for what is in flight
            mbar_wait(ba, 0);
            for (int c = max(0, issued - 2); c < issued; c++) mbar_wait(smem_u32(&bar[1 + (c & 1)]), (c >> 1) & 1);
        }
    } else if (warp == IT_EPI + 1) {
        // ------------------------------------------------ MMAs
        if (lane == 0) {
            const uint32_t idesc = idesc_tf32(IT_M, S::N);
            int last = -1;
            if (!mbar_wait(smem_u32(&bar[0]), 0)) fail();
            for (int c = 0; c < nch && !*abort_flag; c++) {
                const int b = c & 1;
                if (!mbar_wait(smem_u32(&bar[1 + b]), (c >> 1) & 1)) {
                    fail();
                    break;
                }
                if (c >= 2 && !mbar_wait(smem_u32(&bar[7 + b]), ((c >> 1) - 1) & 1)) {
                    fail();
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t ab = smem_u32(sA), bb = smem_u32(sB + b * S::BYTES);
                const uint32_t d = tmem + (uint32_t)(b * S::N);
#pragma unroll
                for (int q = 0; q < IT_K / 8; q++) {
                    const uint64_t da = smem_desc(ab + 2 * q * IT_A_LBO, IT_A_LBO, 128);
                    const uint64_t db = smem_desc(bb + 2 * q * S::LBO, S::LBO, 128);
                    mma_tf32(d, da, db, idesc, q > 0 ? 1u : 0u);
                }
                mma_commit(smem_u32(&bar[3 + b]));   // the weight buffer is free again
                mma_commit(smem_u32(&bar[5 + b]));   // the accumulator is ready
                last = c;
            }
            // every MMA issued must finish before the tensor memory is freed
            if (last >= 0) mbar_wait(smem_u32(&bar[5 + (last & 1)]), (last >> 1) & 1);
        }
    } else {
        // ------------------------------------------------ rows (lane = ion of the tile)
        const int qd = warp & 3, hsel = warp >> 2;
        const int pos = blockIdx.x * IT_M + qd * 32 + lane;
        const bool act = pos < a.cnt;
        const int ion = act ? a.order[pos] : 0;
        const Cell &c = a.c;
        double tx = 0.0, ty = 0.0;
        float mx = 0.f, my = 0.f, mz = 0.f;
        if (act) {
            const double4 ri = a.r[ion];
            tx = c.B[0][0] * ri.x + c.B[1][0] * ri.y + c.B[2][0] * ri.z;
            ty = c.B[0][1] * ri.x + c.B[1][1] * ri.y + c.B[2][1] * ri.z;
            if (WF && a.ld) {
                const double3 m3 = a.mu[ion];
                mx = (float)(c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z);
                my = (float)(c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z);
                mz = (float)(c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z);
            }
        }
        const float2 e1 = cis2pi32(ty);
        float2 w = make_float2(1.f, 0.f);
        double S0 = 0, S1 = 0, S2 = 0, P0 = 0, P1 = 0, P2 = 0;
        const uint32_t lanebase = tmem + ((uint32_t)(qd * 32) << 16);
        bool ok = true;
        for (int ch = 0; ch < nch; ch++) {
            const int b = ch & 1;
            int got = 1;
            if (lane == 0) got = (!*abort_flag && mbar_wait(smem_u32(&bar[5 + b]), (ch >> 1) & 1)) ? 1 : 0;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) {
                if (lane == 0) fail();
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float v[IT_HALF * NC];
#pragma unroll
            for (int q = 0; q < NC; q++)
                tmem_ld8(lanebase + (uint32_t)(b * S::N + hsel * IT_HALF * NC + 8 * q), v + 8 * q);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar[7 + b]));   // the accumulator is in registers
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, p0 = 0.f, p1 = 0.f, p2 = 0.f;
#pragma unroll
            for (int j = 0; j < IT_HALF; j++) {
                const int rr = ch * IT_RPC + hsel * IT_HALF + j;
                if (rr >= nrs) break;
                const float4 R = rowf[rr];
                // the row phase: from an FP64-reduced argument at rows 0 and IT_RUN of the
                // group and wherever the row does not continue the one before, else by
                // one FP32 step in ny
                if (j % IT_RUN != 0 && R.z != 0.f) w = cmul32(w, e1);
                else w = cis2pi32((double)R.x * tx + (double)R.y * ty);
                const float *g = v + j * NC;
                const float Gx = g[0], Gy = g[1], Hx = g[2], Hy = g[3];
                // Im conj(w) G and Im conj(w) H
                const float R1 = w.x * Gy - w.y * Gx, Rz = w.x * Hy - w.y * Hx;
                const float fx = R.x, fy = R.y;
                s0 = fmaf(fx, R1, s0);
                s1 = fmaf(fy, R1, s1);
                s2 += Rz;
                if (WF) {
                    const float Kx = g[4], Ky = g[5];
                    // Re conj(w) G, H, K with the ion's dipole, c0 = nx mx + ny my
                    const float Q0 = w.x * Gx + w.y * Gy, Q1 = w.x * Hx + w.y * Hy, Q2 = w.x * Kx + w.y * Ky;
                    const float c0 = fx * mx + fy * my;
                    const float T1 = c0 * Q0 + mz * Q1, Tz = c0 * Q1 + mz * Q2;
                    p0 = fmaf(fx, T1, p0);
                    p1 = fmaf(fy, T1, p1);
                    p2 += Tz;
                }
            }
            S0 += (double)s0;
            S1 += (double)s1;
            S2 += (double)s2;
            if (WF) {
                P0 += (double)p0;
                P1 += (double)p1;
                P2 += (double)p2;
            }
        }
        if (ok && act) {
            const int nv = WF ? 6 : 3;
            double *o = a.part + ((size_t)(2 * sl + hsel) * a.cnt + pos) * nv;
            o[0] = S0;
            o[1] = S1;
            o[2] = S2;
            if (WF) {
                o[3] = P0;
                o[4] = P1;
                o[5] = P2;
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------- host side
static int ion_tc_tiles(int n) { return ceil_div(n, IT_M); }

// buffers of the pass (at set-up: nothing may be allocated while steps are recorded)
void setup_ion_tc(Engine &e) {
    if (e.d_ion_atab || e.kmax[2] > IT_MAXK2) return;
    e.d_ion_atab = dalloc<float4>((size_t)ion_tc_tiles(e.n) * (IT_A_BYTES / 16));
    e.d_ion_wtab = dalloc<float4>((size_t)ceil_div(e.nrow, IT_RPC) * (ItShape<6>::BYTES / 16));
}

void launch_ion_tc_table(Engine &e) {
    if (!e.d_ion_atab) return;
    MDFF_LAUNCH(e, k_ion_tc_table, ceil_div(e.n, 128), 128, 0, e.n, e.kmax[2], e.cell, e.d_r, e.d_ion_order,
                e.d_ion_atab);
}

// slices of the rows over the CTAs (MINB resident per SM): the fewest waves of
// (tiles x slices), counting a fixed set-up per CTA against the chunks it runs; each slice
// writes two partial slices (the halves of its rows), within the partial buffer
static int ion_tc_slices(const Engine &e, int tiles, int nchunk, bool wf, int minb) {
    const double setup = 3.0, per_chunk = wf ? 0.7 : 0.5;   // relative costs
    int best = 1;
    double best_t = 1e300;
    for (int s = 1; s <= std::min(std::min(8, nchunk), e.ion32_slices / 2); s++) {
        int waves = ceil_div((long long)tiles * s, (long long)e.nsm * minb);
        double t = waves * (setup + per_chunk * ceil_div(nchunk, s));
        if (t < best_t - 1e-9) {
            best_t = t;
            best = s;
        }
    }
    return best;
}

template <int NC>
static void ion_tc_run(Engine &e, const IonTcArgs &a, int tiles, int slices, int nchunk) {
    using S = ItShape<NC>;
    MDFF_LAUNCH(e, k_ion_tc_weights<NC>, ceil_div(nchunk * S::N * (IT_KV / 4), 128), 128, 0, e.nrow, nchunk,
                e.kmax[2], e.d_row, e.d_rho, e.d_ion_wtab);
    size_t smem = S::SMEM + sizeof(float4) * a.rows_per_slice + 16 * sizeof(uint64_t);
    // the largest request once per process (the attribute call is not recorded in graphs)
    static std::once_flag once;
    std::call_once(once, [] {
        MDFF_CK(cudaFuncSetAttribute(k_ion_tc<NC>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    });
    Engine::HighPrio hp(e);
    MDFF_LAUNCH(e, k_ion_tc<NC>, dim3(tiles, slices), IT_THREADS, smem, a);
}

bool launch_ion_tc(Engine &e, const double *q, const double3 *mu, bool ld, const RecOut &o, const int *idx,
                   int cnt) {
    if (!e.d_ion_atab || cnt <= 0 || e.ion32_slices < 2) return false;
    // positions 0..cnt-1 of the order: every ion, or the polarisable ones
    if (!(idx == nullptr && cnt == e.n) && !(idx == e.d_pidx && cnt == e.npol)) return false;
    const bool wf = o.f != nullptr;
    const int nchunk = ceil_div(e.nrow, IT_RPC), tiles = ion_tc_tiles(cnt);
    int slices = e.ion_tc_slices_set > 0 ? std::min(std::min(e.ion_tc_slices_set, nchunk), e.ion32_slices / 2)
                                         : ion_tc_slices(e, tiles, nchunk, wf, wf ? ItShape<6>::MINB : ItShape<4>::MINB);
    IonTcArgs a;
    a.cnt = cnt;
    a.nrow = e.nrow;
    a.rows_per_slice = ceil_div(nchunk, slices) * IT_RPC;
    slices = ceil_div(e.nrow, a.rows_per_slice);
    a.ld = ld;
    a.order = e.d_ion_order;
    a.c = e.cell;
    a.r = e.d_r;
    a.mu = mu;
    a.row = e.d_row;
    a.atab = e.d_ion_atab;
    a.wtab = e.d_ion_wtab;
    a.part = e.d_ion_part32;
    a.status = e.d_status;
    int pi = -1;
    e.prof_begin("k_rec_ion", &pi);
    if (wf) ion_tc_run<6>(e, a, tiles, slices, nchunk);
    else ion_tc_run<4>(e, a, tiles, slices, nchunk);
    // the same algorithmic count as the CUDA-core pass (8 / 12 flops per ion and k)
    e.prof_end("k_rec_ion", pi, (wf ? 12.0 : 8.0) * (double)cnt * e.nk);
    launch_combine32(e, q, mu, ld, o, idx ? idx : e.d_ion_order, cnt, 2 * slices, wf);
    return true;
}

}  // namespace mdffgpu
