// rho(k) on the 5th-generation tensor cores (tcgen05, sm_100a): the mixed-precision
// structure-factor pass as a TF32 matrix product with FP32 accumulation in tensor memory.
//
// With e^{ik.r_i} = E0_i[nx] E1_i[ny] E2_i[nz] and E2_i[-z] = conj E2_i[z] = (c, -d), the
// summand of k = (nx, ny, nz) is (B1 + nz B2) E2[nz] with, per row (nx, ny) and ion,
//     b = E0[nx] E1[ny],  B1 = (q + i c0) b,  B2 = i c1 b,  c0 = nx m0 + ny m1,  c1 = m2
// (m = 2 pi B mu), and the eight sums over ions of B1x c, B1y d, B1x d, B1y c and the same
// with B2 give rho(+z) and rho(-z) (kspace32.cu).  So the pass is one real product
//     C[(coef, row)][col] = sum_i A[(coef, row)][i] E[col][i],
// A = (B1x, B1y, B2x, B2y) of each row and ion (M = 4 x 32 rows per CTA), E = (1, c_1..c_K2,
// d_1..d_K2) of each ion (N = 32, the 1 for nz = 0): only A depends on the row, one
// complex product per (row, ion) to form it.  Every value x is split as x = h + l, both
// TF32 (round to nearest), and the product taken as hh + hl + lh (the dropped ll is 2^-22
// of it): K = 3 per ion.
//
// CTA = 32 k-rows and a chunk of ions, 8 warps.  Per stage of 16 ions the phase-table
// rows are staged in shared memory (asynchronous copies, three stages ahead), all warps
// write the split operands into one of two K-major no-swizzle buffers, one thread issues
// the six tcgen05.mma (M=128, N=32, K=8) and commits them to the buffer's mbarrier, and
// the next stage is written while they run.  Every window of stages (about 200 ions) the
// accumulator is read back (tcgen05.ld), combined into rho(+z), rho(-z) and written as one
// FP32 chunk partial per k; partials are summed in FP64 in a fixed order (k_rho_reduce),
// as for the CUDA-core pass.
//
// Selected with MDFFGPU_KSPACE_TC=1; the CUDA-core pass (kspace32.cu) is the default.
// Measured on the bench system (24000 ions, 12194 k, B200): forces within 3.4e-6 of FP64
// (CUDA-core pass 2.6e-6) and 2.8 instead of 2.9 CG iterations per step, but 114 us per
// dipole pass against 71 us: each 16-ion stage costs two CTA-wide barriers and a short
// dependent chain (staged loads, complex product, split, store) with four warps per
// scheduler, so the tensor pipe idles most of the time.
//
// Every wait on an mbarrier is bounded: on expiry the kernel sets ST_TC_TIMEOUT in the
// status word, waits (bounded) for its MMAs once more, frees its tensor memory and
// returns; the host turns the flag into MDFFGPU_ERR_TIMEOUT.
#include <cstdint>

#include "engine.cuh"
#include "tc_common.cuh"

namespace mdffgpu {

constexpr int TC_M = 128;          // MMA M: 4 coefficients x 32 k-rows, m = coef * 32 + row
constexpr int TC_ROWS = 32;
constexpr int TC_N = 32;           // MMA N: nz = 0, c_1..c_K2, d_1..d_K2, zero padding
constexpr int TC_SI = 16;          // ions per stage
constexpr int TC_KS = 3 * TC_SI;   // K per stage: split terms (hh, hl, lh) x ions, term-major
constexpr int TC_THREADS = 256;
constexpr int TC_NSTG = 3;         // staged-row buffers: copies run TC_NSTG - 1 stages ahead
constexpr int TC_IDX = 2048;       // ion indices of a chunk kept in shared memory (larger
                                   // chunks read them from global memory)
constexpr int TC_ISSUER = 128;     // thread that issues the MMAs (warp 4: no B operand work)
constexpr int TC_WIN = 12;         // stages per partial sum, at least (192 ions)
constexpr uint32_t TC_A_LBO = (TC_M / 8) * 128;        // 2048: 16-byte K chunk stride of A
constexpr uint32_t TC_B_LBO = (TC_N / 8) * 128;        // 512
constexpr uint32_t TC_A_BYTES = (TC_KS / 4) * TC_A_LBO;
constexpr uint32_t TC_OP_BYTES = TC_A_BYTES + (TC_KS / 4) * TC_B_LBO;
constexpr int TC_XS = TC_N + 1;    // padded row of the read-back accumulator

__device__ __forceinline__ void cp_async16_tc(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}

// (q, 2 pi (B mu)) per listed ion, as the CUDA-core pass forms it
__global__ void k_qm_tc(int cnt, const int *__restrict__ idx, Cell c, const double *__restrict__ q,
                        const double3 *__restrict__ mu, int lq, int ld, float4 *__restrict__ out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    int ion = idx ? idx[t] : t;
    const double tpi = TPI_D;
    float4 v = make_float4(lq ? (float)q[ion] : 0.f, 0.f, 0.f, 0.f);
    if (ld) {
        double3 m3 = mu[ion];
        v.y = (float)(tpi * (c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z));
        v.z = (float)(tpi * (c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z));
        v.w = (float)(tpi * (c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z));
    }
    out[t] = v;
}

struct RhoTcArgs {
    int cnt, chunk, win, nwin, nrow, nk, K2;
    int tab_w;                 // float2 per table row
    int ha;                    // 16-byte units of E0 | E1 in a table row
    int skip;                  // 16-byte units of the nz <= 0 blocks (not staged)
    int cw;                    // staged 16-byte units per ion: E0 | E1 | nz > 0 blocks
    int e1, K1;                // float2 offset of E1[-K1]
    const int *idx;
    const float2 *tab;
    const float4 *qm;          // per listed ion: (q, 2 pi B0.mu, 2 pi B1.mu, 2 pi B2.mu)
    const KRow *row;
    float2 *part;              // [partial][nk]
    unsigned *status;
};

__global__ void __launch_bounds__(TC_THREADS, 2) k_rho_tc(RhoTcArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int cw = a.cw;
    unsigned char *op = sm;                                              // [2][TC_OP_BYTES]
    float4 *stg = (float4 *)(sm + 2 * TC_OP_BYTES);                      // [TC_NSTG][TC_SI][cw]
    float4 *stq = stg + TC_NSTG * TC_SI * cw;                            // [TC_NSTG][TC_SI]
    float *X = (float *)(stq + TC_NSTG * TC_SI);                         // [TC_M][TC_XS]
    int *sidx = (int *)(X + TC_M * TC_XS);                               // [TC_IDX]
    uint64_t *mbar = (uint64_t *)(sidx + TC_IDX);                        // [2]
    int *abort_flag = (int *)(mbar + 2);
    uint32_t *tmem_slot = (uint32_t *)(abort_flag + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * TC_ROWS;
    const int a0 = blockIdx.y * a.chunk, a1 = min(a.cnt, a0 + a.chunk);
    const int nstage = a1 > a0 ? (a1 - a0 + TC_SI - 1) / TC_SI : 0;

    const bool lidx = a.idx && a1 - a0 <= TC_IDX;   // chunk's ion list in shared memory
    if (lidx)
        for (int t = tid; t < a1 - a0; t += TC_THREADS) sidx[t] = __ldg(a.idx + a0 + t);
    if (tid == 0) {
        for (int b = 0; b < 2; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(32)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // operand roles: A unit (row r, coefficient pair cp, ion quad jq), B unit (column n, quad)
    const int r = tid & 31, jq = (tid >> 5) & 3, cp = tid >> 7;
    const bool rok = row0 + r < a.nrow;
    KRow R;
    R.nx = R.ny = R.z0 = R.cnt = R.koff = 0;
    if (rok) R = a.row[row0 + r];
    const float fnx = (float)R.nx, fny = (float)R.ny;
    const int o0 = R.nx, o1 = a.e1 + a.K1 + R.ny;
    const int mx = 2 * cp * 32 + r, my = mx + 32;
    const int n = tid & 31;   // B column (threads < 128)
    int zsrc = 0;   // B column n: float offset in a staged row (x, y: Re E2[z], Re E2[z+1]; z, w: Im)
    if (n >= 1 && n <= 2 * a.K2) {
        int z = n <= a.K2 ? n : n - a.K2;
        zsrc = 4 * (a.ha + 9 * ((z - 1) / 16) + ((z - 1) % 16) / 2) + ((z - 1) & 1) + (n <= a.K2 ? 0 : 2);
    }

    // staged rows of stage s into stage buffer s % TC_NSTG (16-byte asynchronous copies,
    // warp w copies rows w, w + 8); one commit group per stage, empty past the last
    auto issue = [&](int s) {
        if (s < nstage) {
            const int t0 = a0 + s * TC_SI, nt = min(TC_SI, a1 - t0);
            float4 *dst = stg + (s % TC_NSTG) * TC_SI * cw;
            for (int j = warp; j < nt; j += TC_THREADS / 32) {
                int ion = lidx ? sidx[t0 - a0 + j] : (a.idx ? __ldg(a.idx + t0 + j) : t0 + j);
                const float4 *src = (const float4 *)(a.tab + (size_t)ion * a.tab_w);
                for (int u = lane; u < cw; u += 32) cp_async16_tc(dst + j * cw + u, src + (u < a.ha ? u : u + a.skip));
            }
            if (tid < nt) cp_async16_tc(stq + (s % TC_NSTG) * TC_SI + tid, a.qm + t0 + tid);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };

    const uint32_t idesc = idesc_tf32(TC_M, TC_N);
    int done_win = 0, last = -1;
    for (int s = 0; s < TC_NSTG - 1; s++) issue(s);
    for (int s = 0; s < nstage; s++) {
        const int buf = s & 1;
        asm volatile("cp.async.wait_group %0;\n" ::"n"(TC_NSTG - 2) : "memory");   // stage s has landed
        if (tid == TC_ISSUER && s >= 2 && !mbar_wait(smem_u32(&mbar[buf]), ((s - 2) >> 1) & 1)) *abort_flag = 1;
        __syncthreads();
        if (*abort_flag) break;
        issue(s + TC_NSTG - 1);   // into the buffer that stage s - 1 read
        const int t0 = a0 + s * TC_SI;
        const float4 *cur = stg + (s % TC_NSTG) * TC_SI * cw;
        const float4 *cq = stq + (s % TC_NSTG) * TC_SI;
        unsigned char *A = op + buf * TC_OP_BYTES, *B = A + TC_A_BYTES;
        {
            // A: coefficients of 4 ions for one row and one coefficient pair
            float xv[4], yv[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int jj = jq * 4 + j;
                xv[j] = yv[j] = 0.f;
                if (rok && t0 + jj < a1) {
                    const float2 *Rw = (const float2 *)(cur + jj * cw);
                    const float2 e0 = Rw[o0], e1 = Rw[o1];
                    const float bx = e0.x * e1.x - e0.y * e1.y, by = e0.x * e1.y + e0.y * e1.x;
                    const float4 qm = cq[jj];
                    if (cp == 0) {
                        const float c0 = fnx * qm.y + fny * qm.z;
                        xv[j] = qm.x * bx - c0 * by;
                        yv[j] = qm.x * by + c0 * bx;
                    } else {
                        xv[j] = -qm.w * by;
                        yv[j] = qm.w * bx;
                    }
                }
            }
            float xh[4], xl[4], yh[4], yl[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                split2(xv[j], xh[j], xl[j]);
                split2(yv[j], yh[j], yl[j]);
            }
#pragma unroll
            for (int t = 0; t < 3; t++) {   // A terms h h l
                const int k = t * TC_SI + jq * 4;
                const float *x = t == 2 ? xl : xh, *y = t == 2 ? yl : yh;
                *(float4 *)(A + kmaj(mx, k, TC_A_LBO)) = make_float4(x[0], x[1], x[2], x[3]);
                *(float4 *)(A + kmaj(my, k, TC_A_LBO)) = make_float4(y[0], y[1], y[2], y[3]);
            }
        }
        if (tid < 128) {
            // B: column n of 4 ions
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int jj = jq * 4 + j;
                v[j] = 0.f;
                if (t0 + jj < a1) {
                    if (n == 0) {
                        v[j] = 1.f;
                    } else if (n <= 2 * a.K2) {
                        v[j] = ((const float *)(cur + jj * cw))[zsrc];
                    }
                }
            }
            float h[4], l[4];
#pragma unroll
            for (int j = 0; j < 4; j++) split2(v[j], h[j], l[j]);
#pragma unroll
            for (int t = 0; t < 3; t++) {   // B terms h l h
                const int k = t * TC_SI + jq * 4;
                const float *w = t == 1 ? l : h;
                *(float4 *)(B + kmaj(n, k, TC_B_LBO)) = make_float4(w[0], w[1], w[2], w[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        const bool first = s % a.win == 0, end = s % a.win == a.win - 1 || s == nstage - 1;
        if (tid == TC_ISSUER) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ab = smem_u32(A), bb = smem_u32(B);
#pragma unroll
            for (int q = 0; q < TC_KS / 8; q++) {
                uint64_t da = smem_desc(ab + 2 * q * TC_A_LBO, TC_A_LBO, 128);
                uint64_t db = smem_desc(bb + 2 * q * TC_B_LBO, TC_B_LBO, 128);
                mma_tf32(tmem, da, db, idesc, (first && q == 0) ? 0u : 1u);
            }
            mma_commit(smem_u32(&mbar[buf]));
        }
        last = s;
        if (!end) continue;
        // ------------------------------------------------ window end: read back, combine
        if (tid == TC_ISSUER && !mbar_wait(smem_u32(&mbar[buf]), (s >> 1) & 1)) *abort_flag = 1;
        __syncthreads();
        if (*abort_flag) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        {
            const int qd = warp & 3, ch = warp >> 2;
            float v[16];
            const uint32_t base = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(ch * 16);
            tmem_ld8(base, v);
            tmem_ld8(base + 8, v + 8);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float *xr = X + (qd * 32 + lane) * TC_XS + ch * 16;
#pragma unroll
            for (int c = 0; c < 16; c++) xr[c] = v[c];
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        {
            float2 *P0 = a.part + ((size_t)blockIdx.y * a.nwin + done_win) * a.nk;
            // item it: row it & 31 (= r, TC_THREADS being a multiple of 32), nz = it >> 5
            for (int it = tid; it < TC_ROWS * (a.K2 + 1) && rok; it += TC_THREADS) {
                const int rr = r, z = it >> 5;
                const bool full = R.z0 <= 0;
                float2 *P = P0 + (R.koff - R.z0);
                const float *x0 = X + rr * TC_XS, *x1 = X + (32 + rr) * TC_XS;
                const float *x2 = X + (64 + rr) * TC_XS, *x3 = X + (96 + rr) * TC_XS;
                if (z == 0) {
                    if (full) P[0] = make_float2(x0[0], x1[0]);
                    continue;
                }
                const int cz = z, dz = a.K2 + z;
                const float sa = x0[cz], sb = x1[dz], sc = x0[dz], sd = x1[cz];
                const float ta = x2[cz], tb = x3[dz], tc = x2[dz], td = x3[cz];
                const float fz = (float)z;
                P[z] = make_float2(sa - sb + fz * (ta - tb), sc + sd + fz * (tc + td));
                if (full) P[-z] = make_float2(sa + sb - fz * (ta + tb), sd - sc + fz * (tc - td));
            }
        }
        done_win++;
    }
    const bool aborted = *abort_flag != 0;
    if (!aborted) {
        // windows of this chunk without ions: zero partials
        for (; done_win < a.nwin; done_win++) {
            float2 *P0 = a.part + ((size_t)blockIdx.y * a.nwin + done_win) * a.nk;
            for (int it = tid; it < TC_ROWS * (a.K2 + 1) && rok; it += TC_THREADS) {
                const int z = it >> 5;
                const bool full = R.z0 <= 0;
                float2 *P = P0 + (R.koff - R.z0);
                if (z == 0) {
                    if (full) P[0] = make_float2(0.f, 0.f);
                    continue;
                }
                P[z] = make_float2(0.f, 0.f);
                if (full) P[-z] = make_float2(0.f, 0.f);
            }
        }
    } else {
        if (tid == TC_ISSUER) {
            atomicOr(a.status, (unsigned)ST_TC_TIMEOUT);
            // the last committed stage covers every MMA issued before it
            if (last >= 0) mbar_wait(smem_u32(&mbar[last & 1]), (last >> 1) & 1);
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32) : "memory");
    }
}

static size_t rho_tc_smem(int cw) {
    return 2 * (size_t)TC_OP_BYTES + sizeof(float4) * (TC_NSTG * TC_SI * (size_t)cw + TC_NSTG * TC_SI) +
           sizeof(float) * TC_M * TC_XS + sizeof(int) * TC_IDX + 2 * sizeof(uint64_t) + 16;
}

// rho(k) partials of `cnt` ions (idx: subset) into e.d_rho_part32 on the tensor cores;
// returns false (nothing launched) when the k box is outside the kernel's range.
bool launch_rho_tc(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt,
                   int tab_w, int z_off, int nzb_neg, int *chunks_used) {
    int K2 = e.kmax[2];
    if (2 * K2 + 1 > TC_N || cnt <= 0) return false;
    if (!e.d_qm_tc) e.d_qm_tc = dalloc<float4>(e.n);
    MDFF_LAUNCH(e, k_qm_tc, ceil_div(cnt, 256), 256, 0, cnt, idx, e.cell, q, mu, lq ? 1 : 0, ld ? 1 : 0, e.d_qm_tc);
    RhoTcArgs a;
    a.cnt = cnt;
    a.nrow = e.nrow;
    a.nk = e.nk;
    a.K2 = K2;
    a.tab_w = tab_w;
    a.ha = z_off / 2;
    a.skip = 9 * nzb_neg;
    a.cw = tab_w / 2 - a.skip;
    a.e1 = e.kmax[0] + 1;
    a.K1 = e.kmax[1];
    a.idx = idx;
    a.tab = e.d_tab32;
    a.qm = e.d_qm_tc;
    a.row = e.d_row;
    a.part = e.d_rho_part32;
    a.status = e.d_status;
    // two CTAs per SM; chunk partials (ion chunks x windows) within the partial buffer
    int mtiles = ceil_div(e.nrow, TC_ROWS);
    int chunks = std::max(1, std::min(2 * e.nsm / mtiles, ceil_div(cnt, TC_SI)));
    a.chunk = ceil_div(ceil_div(cnt, chunks), TC_SI) * TC_SI;
    chunks = ceil_div(cnt, a.chunk);
    int stages = a.chunk / TC_SI;
    int wmax = std::max(1, e.rho32_chunks_max / chunks);
    a.win = std::min(stages, std::max(TC_WIN, ceil_div(stages, wmax)));
    a.nwin = ceil_div(stages, a.win);
    if (chunks * a.nwin > e.rho32_chunks_max) return false;
    size_t smem = rho_tc_smem(a.cw);
    MDFF_CK(cudaFuncSetAttribute(k_rho_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MDFF_LAUNCH(e, k_rho_tc, dim3(mtiles, chunks), TC_THREADS, smem, a);
    *chunks_used = chunks * a.nwin;
    return true;
}

}  // namespace mdffgpu
