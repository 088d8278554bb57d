// The rho pass of the mixed-precision reciprocal sum on the 5th-generation tensor cores
// (tcgen05, sm_100a): kspace32.cu's k_rho32 as a TF32 matrix product with FP32
// accumulation in tensor memory.
//
// With e^{ik.r_i} = E0_i[nx] E1_i[ny] E2_i[nz] and E2_i[-z] = conj E2_i[z] = (c, -d), the
// summand of k = (nx, ny, nz) is (B1 + nz B2) E2[nz] with, per row (nx, ny) and ion,
//     b = E0[nx] E1[ny],  B1 = (q + i c0) b,  B2 = i c1 b,  c0 = nx m0 + ny m1,  c1 = m2
// (m = 2 pi B mu), and the eight sums over ions of B1x c, B1y d, B1x d, B1y c and the same
// with B2 give rho(+z) and rho(-z) (kspace32.cu).  So the pass is one real product
//     C[(coef, row)][col] = sum_i A[(coef, row)][i] E[col][i],
// A = (B1x, B1y, B2x, B2y) of each row and ion (M = 4 coefficients x 32 rows per MMA),
// E = (1, c_1..c_K2, d_1..d_K2, 0 ...) of each ion (N = 32; the 1 gives nz = 0).  Only A
// depends on the row: one complex product per (row, ion) forms it, the MMA does the nz
// sums.  Every value x is split as x = h + l, both TF32, and the product taken as
// A_h E_h + A_h E_l + A_l E_h (the dropped l l term is 2^-22 of it): three MMAs per
// K step, the A_h tile read by two of them, so a producer stores each value twice
// (h and l), not three times.
//
// CTA = 64 k-rows (two M = 128 MMA tiles sharing every staged ion) and a chunk of ions
// in stages of 16, 14 warps:
//   warp 8      bulk-copies each stage's inputs -- the ions' E0 | E1 phase rows, their
//               (q, 2 pi B mu) and the E operand tile, all three laid out per stage once
//               per force evaluation (k_rho_tc_tables) or per pass (k_qm_tc) -- into one
//               of four input slots, completing on mbarriers;
//   warps 0-7   form A (warp w: tile w % 2, ions 4 (w / 2) .. + 3 of the stage, lane =
//               row), split it and store it K-major into one of two A buffers;
//   warp 9      issues the 12 MMAs (M = 128, N = 32, K = 8) of a stage -- the A_h E_h
//               products into the current window's accumulator of each tile, the small
//               A_h E_l and A_l E_h products into one accumulator per tile for the whole
//               chunk -- and commits them to the buffers' barriers;
//   warps 10-13 read each finished window (RT_WIN stages, 32 ions) back (tcgen05.ld;
//               warp w takes lane quarter w % 4) while the next window accumulates, add
//               it to FP32 running sums kept in tensor memory, and at the end add the
//               small-product sums, combine into rho(+z), rho(-z) and write the chunk
//               partial.
// The chunk partials are summed in FP64 in a fixed order (k_rho_reduce32), as the
// CUDA-core pass's are.  The tensor cores' FP32 accumulation is not round-to-nearest: each
// MMA into an accumulator costs up to an ulp of it, toward zero, which shrinks |rho| and
// so the energy.  So the large products take 4 MMA steps per window before a
// round-to-nearest FP32 add, and the small ones (2^-11 of the sum) accumulate apart.
//
// Every mbarrier wait is bounded: on expiry the kernel sets ST_TC_TIMEOUT, stops issuing,
// waits (bounded) for the copies and MMAs it has in flight, frees its tensor memory and
// returns; the host turns the flag into MDFFGPU_ERR_TIMEOUT.
#include <mutex>

#include "engine.cuh"
#include "tc_common.cuh"

namespace mdffgpu {

constexpr int RT_MT = 2;                        // MMA tiles (32 k-rows each) per CTA
constexpr int RT_ROWS = 32 * RT_MT;
constexpr int RT_M = 128;                       // MMA M: m = coefficient * 32 + row
constexpr int RT_N = 32;                        // MMA N: 1, c_1..c_K2, d_1..d_K2, zeros
constexpr int RT_SI = 16;                       // ions per stage
constexpr int RT_NIN = 4;                       // input slots: copies run up to 3 stages ahead
constexpr int RT_PROD = 8;                      // producer warps
constexpr int RT_COPY = RT_PROD;                // copy warp
constexpr int RT_MMA = RT_PROD + 1;             // MMA warp
constexpr int RT_EPI0 = RT_PROD + 2;            // first of the 4 read-back warps
constexpr int RT_THREADS = 32 * (RT_PROD + 6);
constexpr int RT_WIN = 2;                       // stages per accumulation window (32 ions)
constexpr int RT_MAXK2 = (RT_N - 1) / 2;        // nz up to 15
constexpr uint32_t RT_A_LBO = (RT_M / 8) * 128;                    // 2048
constexpr uint32_t RT_A_TILE = (2 * RT_SI / 4) * RT_A_LBO;         // K = (h | l) x 16 ions: 16 KB
constexpr uint32_t RT_A_BYTES = RT_MT * RT_A_TILE;                 // 32 KB per buffer
constexpr uint32_t RT_B_LBO = (RT_N / 8) * 128;                    // 512
constexpr uint32_t RT_B_TERM = (RT_SI / 4) * RT_B_LBO;             // 2 KB
constexpr uint32_t RT_B_BYTES = 2 * RT_B_TERM;                     // (h | l): 4 KB per stage
constexpr uint32_t RT_Q_BYTES = RT_SI * 16;
constexpr int RT_XS = RT_N + 1;                                    // padded read-back row
// tensor memory: two windows x RT_MT accumulators of the large products, RT_MT
// accumulators of the small ones, RT_MT running sums
constexpr uint32_t RT_SMALL_COL = 2 * RT_MT * RT_N;
constexpr uint32_t RT_RUN_COL = RT_SMALL_COL + RT_MT * RT_N;
constexpr uint32_t RT_TMEM_COLS = 256;
static_assert(RT_RUN_COL + RT_MT * RT_N <= RT_TMEM_COLS, "tensor memory columns");
static_assert(RT_MT * RT_M * RT_XS * 4 <= 2 * RT_A_BYTES, "read-back buffer within the A buffers");

// shared memory of the pass: [2][A] [NIN][B] [NIN][E rows] [NIN][qm] barriers flags
struct RtSmem {
    uint32_t b, e, q, bar, total;
};
__host__ __device__ inline RtSmem rt_smem(int lz) {
    RtSmem s;
    s.b = 2 * RT_A_BYTES;
    s.e = s.b + RT_NIN * RT_B_BYTES;
    s.q = s.e + RT_NIN * (uint32_t)(RT_SI * lz * 8);
    s.bar = s.q + RT_NIN * RT_Q_BYTES;
    s.total = s.bar + 16 * 8 + 16;   // 16 barriers, the abort flag and the tensor-memory address
    return s;
}

// ---------------------------------------------------------------- per-stage tables
// Once per force evaluation, for position p of order (stage p / RT_SI, slot p % RT_SI):
// the E0 | E1 prefix of the ion's phase-table row (lz complex values, the ones k_rho32
// reads) into etab, interleaved by position pairs -- entry e of the pair (2m, 2m + 1) is
// (x_2m, x_2m+1, y_2m, y_2m+1), the operand order of the pass's packed FP32x2 arithmetic --
// and the E operand (1, c_z, d_z of E2[z] = exp(2 pi i z t_z), the values of the phase
// table's z blocks) split into TF32 h + l, K-major, into btab.  Positions past n are zero.
// One thread per (position pair, prefix entry) and per (position, column).
__global__ void k_rho_tc_tables(int n, int npad, int lz, int tab_w, int K2, Cell c, const double4 *__restrict__ r,
                                const int *__restrict__ order, const float2 *__restrict__ tab,
                                float4 *__restrict__ etab, float *__restrict__ btab) {
    grid_dep();
    // pair entries, then (position, column) items; below 2^31 in all (launch_rho_tc_tables)
    const int ne = (npad / 2) * lz;
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ne + npad * RT_N) return;
    if (g < ne) {
        const int m = g / lz, e = g - m * lz;
        const int ia = 2 * m < n ? order[2 * m] : -1, ib = 2 * m + 1 < n ? order[2 * m + 1] : -1;
        const float2 va = ia >= 0 ? tab[(size_t)ia * tab_w + e] : make_float2(0.f, 0.f);
        const float2 vb = ib >= 0 ? tab[(size_t)ib * tab_w + e] : make_float2(0.f, 0.f);
        etab[g] = make_float4(va.x, vb.x, va.y, vb.y);
        return;
    }
    g -= ne;
    const int p = g / RT_N, col = g - p * RT_N;
    const int ion = p < n ? order[p] : -1;
    float v = 0.f;
    if (ion >= 0) {
        if (col == 0) {
            v = 1.f;
        } else if (col <= 2 * K2) {
            const int z = col <= K2 ? col : col - K2;
            const double4 ri = r[ion];
            const double tz = c.B[0][2] * ri.x + c.B[1][2] * ri.y + c.B[2][2] * ri.z;
            const float2 e = cis2pi32((double)z * tz);
            v = col <= K2 ? e.x : e.y;
        }
    }
    float h, l;
    split2(v, h, l);
    unsigned char *T = (unsigned char *)btab + (size_t)(p / RT_SI) * RT_B_BYTES;
    const int j = p % RT_SI;
    *(float *)(T + kmaj(col, j, RT_B_LBO)) = h;
    *(float *)(T + RT_B_TERM + kmaj(col, j, RT_B_LBO)) = l;
}

// per pass: (q, 2 pi (B mu)) of positions 0..cnt-1 of order, as k_rho32 forms them, zero
// at the positions past them (their A values vanish without a test in the pass); stored by
// position pairs (2m, 2m + 1) as (q_a, q_b, m0_a, m0_b), (m1_a, m1_b, m2_a, m2_b).  One
// thread per pair.
__device__ __forceinline__ float4 qm_of(int t, int cnt, const int *__restrict__ order, const Cell &c,
                                        const double *__restrict__ q, const double3 *__restrict__ mu, int lq, int ld) {
    if (t >= cnt) return make_float4(0.f, 0.f, 0.f, 0.f);
    const int ion = order[t];
    const double tpi = TPI_D;
    float4 v = make_float4(lq ? (float)q[ion] : 0.f, 0.f, 0.f, 0.f);
    if (ld) {
        const double3 m3 = mu[ion];
        v.y = (float)(tpi * (c.B[0][0] * m3.x + c.B[1][0] * m3.y + c.B[2][0] * m3.z));
        v.z = (float)(tpi * (c.B[0][1] * m3.x + c.B[1][1] * m3.y + c.B[2][1] * m3.z));
        v.w = (float)(tpi * (c.B[0][2] * m3.x + c.B[1][2] * m3.y + c.B[2][2] * m3.z));
    }
    return v;
}
__global__ void k_qm_tc(int cnt, int npad, const int *__restrict__ order, Cell c, const double *__restrict__ q,
                        const double3 *__restrict__ mu, int lq, int ld, float4 *__restrict__ out) {
    grid_dep();
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * m >= npad) return;
    const float4 a = qm_of(2 * m, cnt, order, c, q, mu, lq, ld), b = qm_of(2 * m + 1, cnt, order, c, q, mu, lq, ld);
    out[2 * m] = make_float4(a.x, b.x, a.y, b.y);
    out[2 * m + 1] = make_float4(a.z, b.z, a.w, b.w);
}

// ---------------------------------------------------------------- the pass
struct RhoTcArgs {
    int cnt, chunk, nrow, nk, K2, K1, e1, lz;
    const float4 *etab;      // [stage][RT_SI / 2 position pairs][lz]
    const float4 *btab;      // [stage][RT_B_BYTES / 16]
    const float4 *qm;        // [position]
    const KRow *row;
    float2 *part;            // [chunk][nk]
    unsigned *status;
};

__device__ __forceinline__ void tmem_st8(uint32_t addr, const float *v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(addr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

// the 12 MMAs of a stage (tiles 0 and 1, K chunks 0 and 1 of 8 ions): large products
// A_h E_h into h0 / h1 (accumulating when acc_h), small products A_h E_l, A_l E_h into
// s0 / s1 (accumulating when acc_s); a: descriptors of the A buffer (tile-major: A_h and
// A_l of tile 0, then tile 1), e: of the E tile
__device__ __forceinline__ void mma_stage(uint32_t h0, uint32_t h1, uint32_t s0, uint32_t s1, uint64_t a, uint64_t e,
                                          uint32_t idesc, uint32_t acc_h, uint32_t acc_s) {
    // descriptor start addresses are in 16-byte units (shared-memory offsets stay far below
    // the field's 2^18 bytes, so the additions do not carry out of it)
    constexpr uint64_t LO = (RT_SI / 4) * RT_A_LBO / 16, Q1 = 2 * RT_A_LBO / 16, T1 = RT_A_TILE / 16;
    constexpr uint64_t EL = RT_B_TERM / 16, EQ1 = 2 * RT_B_LBO / 16;
    asm volatile(
        "{\n\t.reg .pred ph, ps, pt;\n\t"
        "setp.ne.b32 ph, %17, 0;\n\t"
        "setp.ne.b32 ps, %18, 0;\n\t"
        "setp.ne.b32 pt, %16, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %4, %12, %16, ph;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %6, %14, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%2], %4, %13, %16, ps;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%2], %5, %12, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%2], %6, %15, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%2], %7, %14, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%1], %8, %12, %16, ph;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%1], %10, %14, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%3], %8, %13, %16, ps;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%3], %9, %12, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%3], %10, %15, %16, pt;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%3], %11, %14, %16, pt;\n\t}"
        :
        : "r"(h0), "r"(h1), "r"(s0), "r"(s1), "l"(a), "l"(a + LO), "l"(a + Q1), "l"(a + LO + Q1), "l"(a + T1),
          "l"(a + T1 + LO), "l"(a + T1 + Q1), "l"(a + T1 + LO + Q1), "l"(e), "l"(e + EL), "l"(e + EQ1),
          "l"(e + EL + EQ1), "r"(idesc), "r"(acc_h), "r"(acc_s));
}

__global__ void __launch_bounds__(RT_THREADS, 2) k_rho_tc(RhoTcArgs a) {
    grid_dep();
    extern __shared__ __align__(1024) unsigned char sm[];
    const RtSmem L = rt_smem(a.lz);
    const uint32_t ebytes = (uint32_t)(RT_SI * a.lz * 8);
    unsigned char *sA = sm, *sB = sm + L.b, *sE = sm + L.e, *sQ = sm + L.q;
    uint64_t *bar = (uint64_t *)(sm + L.bar);
    // bar: 0-3 inputs landed, 4-7 inputs consumed (8 producer warps + the MMAs), 8-9 A
    // written (8 producer warps), 10-11 A consumed (MMAs), 12-13 window accumulated,
    // 14-15 window read back (4 warps)
    constexpr int IN_FULL = 0, IN_EMPTY = 4, A_FULL = 8, A_EMPTY = 10, ACC_FULL = 12, ACC_EMPTY = 14;
    volatile int *abort_flag = (volatile int *)(bar + 16);
    uint32_t *tmem_slot = (uint32_t *)(bar + 16) + 1;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * RT_ROWS;
    const int a0 = blockIdx.y * a.chunk, a1 = min(a.cnt, a0 + a.chunk);
    const int nst = a1 > a0 ? (a1 - a0 + RT_SI - 1) / RT_SI : 0;
    const int nwin = (nst + RT_WIN - 1) / RT_WIN;

    if (tid == 0) {
        for (int i = 0; i < RT_NIN; i++) {
            mbar_init(smem_u32(&bar[IN_FULL + i]), 1);
            mbar_init(smem_u32(&bar[IN_EMPTY + i]), RT_PROD + 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&bar[A_FULL + b]), RT_PROD);
            mbar_init(smem_u32(&bar[A_EMPTY + b]), 1);
            mbar_init(smem_u32(&bar[ACC_FULL + b]), 1);
            mbar_init(smem_u32(&bar[ACC_EMPTY + b]), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *abort_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(RT_TMEM_COLS)
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
    // a bounded wait that gives up at once when another warp has already given up
    auto wait = [&](int i, int parity) -> bool {
        const uint32_t ba = smem_u32(&bar[i]);
        if (mbar_test(ba, (uint32_t)parity)) return true;
        if (*abort_flag) return false;
        if (mbar_wait(ba, (uint32_t)parity)) return true;
        fail();
        return false;
    };

    if (warp == RT_COPY) {
        // ------------------------------------------------ copies (lane 0)
        if (lane == 0) {
            int issued = 0;
            for (int s = 0; s < nst; s++) {
                const int slot = s % RT_NIN, u = s / RT_NIN;
                if (u > 0 && !wait(IN_EMPTY + slot, (u - 1) & 1)) break;
                if (*abort_flag) break;
                const int st = (a0 + s * RT_SI) / RT_SI;
                const uint32_t bf = smem_u32(&bar[IN_FULL + slot]);
                mbar_expect_tx(bf, ebytes + RT_Q_BYTES + RT_B_BYTES);
                bulk_g2s(smem_u32(sE + slot * ebytes), a.etab + (size_t)st * (ebytes / 16), ebytes, bf);
                bulk_g2s(smem_u32(sQ + slot * RT_Q_BYTES), a.qm + (size_t)st * RT_SI, RT_Q_BYTES, bf);
                bulk_g2s(smem_u32(sB + slot * RT_B_BYTES), a.btab + (size_t)st * (RT_B_BYTES / 16), RT_B_BYTES, bf);
                issued = s + 1;
            }
            // nothing may land after the CTA is gone: wait (bounded) for what is in flight
            for (int s = max(0, issued - RT_NIN); s < issued; s++)
                mbar_wait(smem_u32(&bar[IN_FULL + s % RT_NIN]), (s / RT_NIN) & 1);
        }
    } else if (warp == RT_MMA) {
        // ------------------------------------------------ MMAs (lane 0)
        if (lane == 0) {
            const uint32_t idesc = idesc_tf32(RT_M, RT_N);
            // descriptors of A buffer 0 and input slot 0; the others differ only in the start address
            const uint64_t dA = smem_desc(smem_u32(sA), RT_A_LBO, 128), dB = smem_desc(smem_u32(sB), RT_B_LBO, 128);
            int last = -1;
            for (int s = 0; s < nst; s++) {
                const int b = s & 1, slot = s % RT_NIN, w = s / RT_WIN, sw = s % RT_WIN;
                if (sw == 0 && w >= 2 && !wait(ACC_EMPTY + (w & 1), ((w >> 1) - 1) & 1)) break;
                if (!wait(A_FULL + b, (s >> 1) & 1) || !wait(IN_FULL + slot, (s / RT_NIN) & 1)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t hb = tmem + (uint32_t)((w & 1) * RT_MT * RT_N);
                mma_stage(hb, hb + RT_N, tmem + RT_SMALL_COL, tmem + RT_SMALL_COL + RT_N,
                          dA + (uint64_t)(b * (RT_A_BYTES / 16)), dB + (uint64_t)(slot * (RT_B_BYTES / 16)), idesc,
                          sw != 0 ? 1u : 0u, s != 0 ? 1u : 0u);
                mma_commit(smem_u32(&bar[A_EMPTY + b]));        // the A buffer is free again
                mma_commit(smem_u32(&bar[IN_EMPTY + slot]));    // so is the E tile (with 8 arrivals)
                if (sw == RT_WIN - 1 || s == nst - 1) mma_commit(smem_u32(&bar[ACC_FULL + (w & 1)]));
                last = s;
            }
            // every MMA issued must finish before the tensor memory is freed
            if (last >= 0) mbar_wait(smem_u32(&bar[A_EMPTY + (last & 1)]), (last >> 1) & 1);
        }
    } else if (warp < RT_PROD) {
        // ------------------------------------------------ A operand (lane = row)
        const int mt = warp % RT_MT, g = warp / RT_MT;
        const int rr = row0 + mt * 32 + lane;
        const bool rok = rr < a.nrow;
        KRow R;
        R.nx = R.ny = R.z0 = R.cnt = R.koff = 0;
        if (rok) R = a.row[rr];
        const float fnx = (float)R.nx, fny = (float)R.ny;
        const float2 fnx2 = make_float2(fnx, fnx), fny2 = make_float2(fny, fny);
        const int o0 = R.nx, o1 = a.e1 + a.K1 + R.ny;
        for (int s = 0; s < nst; s++) {
            const int b = s & 1, slot = s % RT_NIN;
            if (!__all_sync(0xffffffffu, wait(IN_FULL + slot, (s / RT_NIN) & 1))) break;
            const float4 *E = (const float4 *)(sE + slot * ebytes);   // [pair][lz]
            const float4 *Q = (const float4 *)(sQ + slot * RT_Q_BYTES);  // [pair][2]
            float h[4][4], l[4][4];   // [coefficient][ion]
            // two ions per FP32x2 operation; positions past the pass's ions have q = mu = 0
            // (k_qm_tc), rows past nrow give accumulator rows the read-back skips: no tests
#pragma unroll
            for (int pp = 0; pp < 2; pp++) {
                const int P = 2 * g + pp;
                const float4 ea = E[P * a.lz + o0], eb = E[P * a.lz + o1];
                const float2 e0x = make_float2(ea.x, ea.y), e0y = make_float2(ea.z, ea.w);
                const float2 e1x = make_float2(eb.x, eb.y), e1y = make_float2(eb.z, eb.w);
                const float4 qa = Q[2 * P], qb = Q[2 * P + 1];
                const float2 qx = make_float2(qa.x, qa.y), qy = make_float2(qa.z, qa.w);
                const float2 qz = make_float2(qb.x, qb.y), qw = make_float2(qb.z, qb.w);
                const float2 bx = __ffma2_rn(make_float2(-e0y.x, -e0y.y), e1y, __fmul2_rn(e0x, e1x));
                const float2 by = __ffma2_rn(e0y, e1x, __fmul2_rn(e0x, e1y));
                const float2 c0 = __ffma2_rn(fny2, qz, __fmul2_rn(fnx2, qy));
                const float2 v[4] = {__ffma2_rn(make_float2(-c0.x, -c0.y), by, __fmul2_rn(qx, bx)),
                                     __ffma2_rn(c0, bx, __fmul2_rn(qx, by)),
                                     __fmul2_rn(make_float2(-qw.x, -qw.y), by), __fmul2_rn(qw, bx)};
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float hx = tf32_round(v[c].x), hy = tf32_round(v[c].y);
                    const float2 lv = __fadd2_rn(v[c], make_float2(-hx, -hy));
                    h[c][2 * pp] = hx;
                    h[c][2 * pp + 1] = hy;
                    l[c][2 * pp] = lv.x;
                    l[c][2 * pp + 1] = lv.y;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar[IN_EMPTY + slot]));   // E rows and qm read
            // the A buffer of stage s - 2 must have been consumed by its MMAs (the values
            // above are formed while those run)
            if (!__all_sync(0xffffffffu, s < 2 || wait(A_EMPTY + b, ((s >> 1) - 1) & 1))) break;
            unsigned char *A = sA + b * RT_A_BYTES + mt * RT_A_TILE;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                *(float4 *)(A + kmaj(c * 32 + lane, g * 4, RT_A_LBO)) = make_float4(h[c][0], h[c][1], h[c][2], h[c][3]);
                *(float4 *)(A + kmaj(c * 32 + lane, RT_SI + g * 4, RT_A_LBO)) =
                    make_float4(l[c][0], l[c][1], l[c][2], l[c][3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar[A_FULL + b]));
        }
    } else {
        // ------------------------------------------------ read-back (warps 10-13)
        const int qd = warp & 3;
        const uint32_t lanebase = tmem + ((uint32_t)(qd * 32) << 16);
        for (int w = 0; w < nwin; w++) {
            const int b = w & 1;
            if (!__all_sync(0xffffffffu, wait(ACC_FULL + b, (w >> 1) & 1))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int mt = 0; mt < RT_MT; mt++) {
#pragma unroll
                for (int c8 = 0; c8 < RT_N / 8; c8++) {
                    float v[8], s[8];
                    tmem_ld8(lanebase + (uint32_t)((b * RT_MT + mt) * RT_N + 8 * c8), v);
                    const uint32_t ra = lanebase + RT_RUN_COL + (uint32_t)(mt * RT_N + 8 * c8);
                    if (w > 0) tmem_ld8(ra, s);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int k = 0; k < 8; k++) s[k] = w > 0 ? s[k] + v[k] : v[k];
                    tmem_st8(ra, s);
                }
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar[ACC_EMPTY + b]));   // the window's columns are read
        }
        // every window read (or the pass abandoned): the A buffers are free for the sums
        asm volatile("bar.sync 1, 128;" ::: "memory");
        const bool done = !*abort_flag;
        float *X = (float *)sA;   // [RT_MT][RT_M][RT_XS]
        if (done) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int mt = 0; mt < RT_MT; mt++) {
                float *xr = X + ((size_t)mt * RT_M + qd * 32 + lane) * RT_XS;
#pragma unroll
                for (int c8 = 0; c8 < RT_N / 8; c8++) {
                    float s[8], v[8];
                    if (nwin > 0) {
                        tmem_ld8(lanebase + RT_RUN_COL + (uint32_t)(mt * RT_N + 8 * c8), s);
                        tmem_ld8(lanebase + RT_SMALL_COL + (uint32_t)(mt * RT_N + 8 * c8), v);
                        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                        for (int k = 0; k < 8; k++) s[k] += v[k];
                    } else {
#pragma unroll
                        for (int k = 0; k < 8; k++) s[k] = 0.f;
                    }
#pragma unroll
                    for (int k = 0; k < 8; k++) xr[8 * c8 + k] = s[k];
                }
            }
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (done) {
            // item it: row it % RT_ROWS of the CTA, nz = it / RT_ROWS
            const int et = tid - 32 * RT_EPI0;
            for (int it = et; it < RT_ROWS * (a.K2 + 1); it += 128) {
                const int rl = it % RT_ROWS, z = it / RT_ROWS;
                if (row0 + rl >= a.nrow) continue;
                const KRow R = a.row[row0 + rl];
                const bool full = R.z0 <= 0;
                float2 *P = a.part + (size_t)blockIdx.y * a.nk + (R.koff - R.z0);
                const float *xb = X + ((size_t)(rl / 32) * RT_M + rl % 32) * RT_XS;
                const float *x0 = xb, *x1 = xb + 32 * RT_XS, *x2 = xb + 64 * RT_XS, *x3 = xb + 96 * RT_XS;
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
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(RT_TMEM_COLS) : "memory");
    }
}

// ---------------------------------------------------------------- host side
static int rt_npad(const Engine &e) { return ceil_div(e.n, RT_SI) * RT_SI; }

// buffers of the pass (at set-up: nothing may be allocated while steps are recorded);
// lz: float2 entries of a phase-table row's E0 | E1 prefix (even)
void setup_rho_tc(Engine &e, int lz) {
    if (e.d_rho_btab || e.kmax[2] > RT_MAXK2 || rt_smem(lz).total > 227 * 1024) return;
    const int npad = rt_npad(e);
    e.rho_tc_lz = lz;
    e.d_rho_btab = dalloc<float4>((size_t)(npad / RT_SI) * (RT_B_BYTES / 16));
    e.d_rho_etab = dalloc<float4>((size_t)npad * (lz / 2));
    e.d_qm_tc = dalloc<float4>(npad);
}

void launch_rho_tc_tables(Engine &e) {
    if (!e.d_rho_btab) return;
    const int npad = rt_npad(e), lz = e.rho_tc_lz;
    const long long tot = (long long)(npad / 2) * lz + (long long)npad * RT_N;
    if (tot >= (1LL << 31)) throw Error(MDFFGPU_ERR_ARG, "system too large for the tensor-core rho tables");
    MDFF_LAUNCH(e, k_rho_tc_tables, (unsigned)((tot + 255) / 256), 256, 0, e.n, npad, lz, e.tab_w, e.kmax[2], e.cell,
                e.d_r, e.d_ion_order, e.d_tab32, e.d_rho_etab, (float *)e.d_rho_btab);
}

// ions per chunk of a pass over `cnt` ions: a whole number of stages; by default two
// resident CTAs per SM over the row tiles; never more chunks than the partial buffer holds
static int rho_tc_chunk(const Engine &e, int cnt) {
    const int tiles = ceil_div(e.nrow, RT_ROWS), stages = ceil_div(std::max(cnt, 1), RT_SI);
    int c = e.rho_tc_chunks_set > 0 ? e.rho_tc_chunks_set : std::max(1, 2 * e.nsm / tiles);
    c = std::max(1, std::min(c, std::min(stages, e.rho32_chunks_max)));
    return ceil_div(stages, c) * RT_SI;
}

// rho(k) partials of positions 0..cnt-1 of the order (every ion, or the polarisable
// ones) into e.d_rho_part32; false (nothing launched) for any other ion subset
bool launch_rho_tc(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt,
                   int z_off, int *chunks_used) {
    if (!e.d_rho_btab || cnt <= 0 || z_off != e.rho_tc_lz) return false;
    if (!(idx == nullptr && cnt == e.n) && !(idx == e.d_pidx && cnt == e.npol)) return false;
    MDFF_LAUNCH(e, k_qm_tc, ceil_div(rt_npad(e) / 2, 256), 256, 0, cnt, rt_npad(e), e.d_ion_order, e.cell, q, mu,
                lq ? 1 : 0, ld ? 1 : 0, e.d_qm_tc);
    RhoTcArgs a;
    a.cnt = cnt;
    a.chunk = rho_tc_chunk(e, cnt);
    const int chunks = ceil_div(cnt, a.chunk);
    a.nrow = e.nrow;
    a.nk = e.nk;
    a.K2 = e.kmax[2];
    a.K1 = e.kmax[1];
    a.e1 = e.kmax[0] + 1;
    a.lz = e.rho_tc_lz;
    a.etab = e.d_rho_etab;
    a.btab = e.d_rho_btab;
    a.qm = e.d_qm_tc;
    a.row = e.d_row;
    a.part = e.d_rho_part32;
    a.status = e.d_status;
    // the largest request once per process (the attribute call is not recorded in graphs)
    static std::once_flag once;
    std::call_once(once, [] {
        MDFF_CK(cudaFuncSetAttribute(k_rho_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    });
    Engine::HighPrio hp(e);
    MDFF_LAUNCH(e, k_rho_tc, dim3(ceil_div(e.nrow, RT_ROWS), chunks), RT_THREADS, rt_smem(a.lz).total, a);
    *chunks_used = chunks;
    return true;
}

}  // namespace mdffgpu
