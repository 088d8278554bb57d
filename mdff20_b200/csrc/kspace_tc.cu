// rho(k) on the 5th-generation tensor cores (tcgen05, sm_100a): the mixed-precision
// structure-factor pass as TF32 matrix products with FP32 accumulation in tensor memory.
// Selected with MDFFGPU_KSPACE_TC=1; the CUDA-core pass (kspace32.cu) is the default,
// being the faster of the two on the bench system (below).
//
// With the phases factorised, e^{ik.r_i} = E0_i[nx] E1_i[ny] E2_i[nz], and
// k.mu_i = nx m0_i + ny m1_i + nz m2_i (m = 2 pi B mu), one row (nx, ny) of rho is
//     rho(row, nz) = sum_i b_i (q_i + i nz m2_i) E2_i + nx b_i (i m0_i E2_i) + ny b_i (i m1_i E2_i),
// b_i = E0_i[nx] E1_i[ny]: a real matrix product D[row][2 zc + {re,im}] = sum_K A[row][K]
// B[n][K] with six K entries per ion, A = (b, nx b, ny b) and B the matching three
// factors of each nz, so the accumulator is rho itself.  Every value x is split as
// x = h + l, both TF32 (round to nearest), and the product is taken as hh + hl + lh
// (the dropped ll is 2^-22 of it): 18 K entries per ion.
//
// Warp-specialised CTA (128 rows, the MMA's M, and a chunk of ions): 11 producer warps
// write the operands of 4-ion stages into a 4-slot shared-memory ring (no-swizzle K-major
// core matrices), one warp issues the stage's nine tcgen05.mma (M=128, N=2 NZP, K=8)
// round-robin over four independent accumulators and commits them to mbarriers, 8 drain
// warps read each finished accumulator buffer (two buffers) with tcgen05.ld and sum it in
// FP32 registers, written as four sub-chunk partials per CTA and summed over chunks in
// FP64 afterwards (k_rho_reduce), as for the CUDA-core pass.
//
// Measured on the bench system (24000 ions, 12194 k, B200): forces within 1.4e-6 of FP64
// (the CUDA-core pass: 1.7e-6), but about 190 us per pass against 98 us: the producers
// stall on the dependent global loads of the phase-table rows (long-scoreboard stalls
// dominate, the tensor pipe is busy about 10% of the time).
//
// Every wait on an mbarrier is bounded: on expiry the kernel sets ST_TC_TIMEOUT in the
// status word, waits (bounded) for its MMAs once more, frees its tensor memory and
// returns; the host turns the flag into MDFFGPU_ERR_TIMEOUT.
#include <cstdint>

#include "engine.cuh"

namespace mdffgpu {

constexpr int TC_M = 128;          // rows per CTA (MMA M)
constexpr int TC_PW = 11;          // producer warps: write the A and B operands (20 warps in all: 96 registers)
constexpr int TC_DW = 8;           // drain warps: tensor memory -> registers
constexpr int TC_THREADS = 32 * (TC_PW + TC_DW + 1);   // + one MMA warp
constexpr int TC_SI = 4;           // ions per stage
constexpr int TC_V = 6;            // K values per ion and split term
constexpr int TC_T = 3;            // split products per value pair: hh, hl, lh
constexpr int TC_KSTAGE = TC_T * TC_SI * TC_V;   // 72: nine MMAs of K = 8
constexpr int TC_NSLOT = 4;        // operand ring depth
constexpr int TC_G = 2;            // stages accumulated per tensor-memory buffer
constexpr int TC_R = 4;            // independent accumulators per buffer (MMA k goes to k % TC_R)
constexpr int TC_SUB = 4;          // partial sums written per CTA (sub-chunks of its ions)
constexpr int TC_SPIN = 400;       // try_wait rounds (each suspends up to TC_SUSPEND_NS) before giving up
constexpr unsigned TC_SUSPEND_NS = 5000000u;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// x = h + l, both TF32 (round to nearest)
__device__ __forceinline__ void split2(float x, float &h, float &l) {
    h = tf32_rna(x);
    l = tf32_rna(x - h);
}

__device__ __forceinline__ void cp_async16_tc(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}

// the waiting thread is suspended (up to the hint) until the phase completes
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(TC_SUSPEND_NS)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < TC_SPIN; it++)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance between the
// two 16-byte K chunks of one MMA, sbo = byte distance between 8-row groups
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version of sm_100
    return d;                 // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor, kind::tf32: D FP32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float *v) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = __uint_as_float(r[k]);
}

struct RhoTcArgs {
    int cnt, chunk, nrow, nk, K2, tab_w;
    int z_off;                 // float2 offset of the first z block in a table row
    int nzb_neg;               // negative-z blocks
    int e1;                    // float2 offset of E1[-K1]
    int K1;
    const int *idx;
    const float2 *tab;
    const float4 *qm;          // per listed ion: (q, 2 pi B0.mu, 2 pi B1.mu, 2 pi B2.mu)
    const KRow *row;
    float2 *part;              // [chunk][nk]
    unsigned *status;
};

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

// byte offset of element (row or column x, K index k) in a K-major no-swizzle operand
// whose 16-byte K chunks lie `lbo` bytes apart
__device__ __forceinline__ uint32_t kmaj(int x, int k, uint32_t lbo) {
    return (uint32_t)(k >> 2) * lbo + (uint32_t)((x >> 3) * 128 + (x & 7) * 16 + (k & 3) * 4);
}

// one ion's six values for split term t, as (h | l) pairs at K = t*SI*V + j*V
__device__ __forceinline__ void store_terms(unsigned char *base, int x, int j, uint32_t lbo, const float *v,
                                            bool a_side) {
    float h[TC_V], l[TC_V];
#pragma unroll
    for (int k = 0; k < TC_V; k++) split2(v[k], h[k], l[k]);
#pragma unroll
    for (int t = 0; t < TC_T; t++) {
        // A terms h h l, B terms h l h: products hh + hl + lh
        const float *w = (a_side ? t == 2 : t == 1) ? l : h;
        int k0 = t * TC_SI * TC_V + j * TC_V;
#pragma unroll
        for (int k = 0; k < TC_V; k += 2)
            *(float2 *)(base + kmaj(x, k0 + k, lbo)) = make_float2(w[k], w[k + 1]);
    }
}

// rho(row, nz) = sum_i b_i (q_i E2 + i nz m2_i E2) + nx b_i (i m0_i E2) + ny b_i (i m1_i E2),
// b = E0[nx] E1[ny]: A holds (b, nx b, ny b), B holds the three E2 factors of each nz,
// so the accumulator is rho itself.  Stage = TC_SI ions, K = 72; producers fill ring slot
// s % TC_NSLOT, the MMA warp issues nine MMAs into accumulator region (s / TC_G) % 2,
// the drain warps add each finished region.  Barriers: full[slot] (producer arrivals),
// empty[slot] (MMA commit), tfull[region] (MMA commit), tempty[region] (drain arrivals).
template <int NZP>
__global__ void __launch_bounds__(TC_THREADS, 1) k_rho_tc(RhoTcArgs a) {
    constexpr int N = 2 * NZP;
    constexpr int CH = TC_KSTAGE / 4;                     // 16-byte K chunks per stage (18)
    constexpr uint32_t A_LBO = (TC_M / 8) * 128;
    constexpr uint32_t B_LBO = (N / 8) * 128;
    constexpr uint32_t SLOT = CH * (A_LBO + B_LBO);
    constexpr int TMEM_COLS = 2 * TC_R * N < 32 ? 32 : 2 * TC_R * N;   // two buffers of TC_R accumulators
    constexpr int NH = N / 2;                             // columns per drain thread
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t *full = (uint64_t *)(sm + TC_NSLOT * SLOT);
    uint64_t *empty = full + TC_NSLOT;
    uint64_t *tfull = empty + TC_NSLOT;
    uint64_t *tempty = tfull + 2;
    uint32_t *tmem_slot = (uint32_t *)(tempty + 2);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * TC_M;
    const int a0 = blockIdx.y * a.chunk, a1 = min(a.cnt, a0 + a.chunk);
    const int nstage = a1 > a0 ? (a1 - a0 + TC_SI - 1) / TC_SI : 0;
    const int ngroup = (nstage + TC_G - 1) / TC_G;

    if (tid == 0) {
        for (int b = 0; b < TC_NSLOT; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full[b])), "r"(32 * TC_PW)
                         : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[b])) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&tfull[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&tempty[b])), "r"(32 * TC_DW)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // B columns past the last nz stay zero in every slot
    for (int e = tid; e < TC_NSLOT * CH * (N / 8) * 8; e += TC_THREADS) {
        int slot = e / (CH * N), rem = e - slot * CH * N, c = rem / N, n = rem - c * N;
        if ((n >> 1) > 2 * a.K2)
            *(float4 *)(sm + slot * SLOT + CH * A_LBO + c * B_LBO + (n >> 3) * 128 + (n & 7) * 16) =
                make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    bool ok = true;

    if (warp < TC_PW) {
        // ---------------------------------------------------------------- producers
        // items per stage: A (row r, ion j) for it < 128 SI, B (nz slot zc, ion j) after;
        // each thread keeps its items over all stages
        constexpr int NA = TC_M * TC_SI;
        const int nB = (2 * a.K2 + 1) * TC_SI;
        constexpr int PT = 32 * TC_PW;
        for (int s = 0; s < nstage && ok; s++) {
            const int slot = s % TC_NSLOT, use = s / TC_NSLOT;
            if (use > 0 && !mbar_wait(smem_u32(&empty[slot]), (use - 1) & 1)) {
                ok = false;
                break;
            }
            unsigned char *A = sm + slot * SLOT, *B = A + CH * A_LBO;
            const int t0 = a0 + s * TC_SI;
            for (int it = tid; it < NA + nB; it += PT) {
                float v[TC_V];
                if (it < NA) {
                    const int r = it & (TC_M - 1), j = it >> 7, t = t0 + j;
#pragma unroll
                    for (int k = 0; k < TC_V; k++) v[k] = 0.f;
                    if (row0 + r < a.nrow && t < a1) {
                        const KRow R = a.row[row0 + r];
                        const int ion = a.idx ? __ldg(a.idx + t) : t;
                        const float2 *Rw = a.tab + (size_t)ion * a.tab_w;
                        const float2 e0 = __ldg(Rw + R.nx), e1 = __ldg(Rw + a.e1 + a.K1 + R.ny);
                        const float br = e0.x * e1.x - e0.y * e1.y, bi = e0.x * e1.y + e0.y * e1.x;
                        const float fx = (float)R.nx, fy = (float)R.ny;
                        v[0] = br, v[1] = bi, v[2] = fx * br, v[3] = fx * bi, v[4] = fy * br, v[5] = fy * bi;
                    }
                    store_terms(A, r, j, A_LBO, v, true);
                } else {
                    const int e = it - NA, zc = e % (2 * a.K2 + 1), j = e / (2 * a.K2 + 1), t = t0 + j;
                    const int z = zc - a.K2;
                    float x[TC_V];
#pragma unroll
                    for (int k = 0; k < TC_V; k++) x[k] = 0.f;
                    if (t < a1) {
                        const int ion = a.idx ? __ldg(a.idx + t) : t;
                        const int slotz = z <= 0 ? (z + a.K2) / 16 * 18 + (z + a.K2) % 16
                                                 : (a.nzb_neg + (z - 1) / 16) * 18 + (z - 1) % 16;
                        // planar z pairs: entry 2p = (x, x'), entry 2p + 1 = (y, y')
                        const float2 *zp = a.tab + (size_t)ion * a.tab_w + a.z_off + (slotz & ~1);
                        const float2 px = __ldg(zp), py = __ldg(zp + 1);
                        const float2 E = (slotz & 1) ? make_float2(px.y, py.y) : make_float2(px.x, py.x);
                        const float4 qm = __ldg(a.qm + t);
                        const float c2 = (float)z * qm.w;
                        // X = E (q + i nz m2), Y = i m0 E, Z = i m1 E
                        x[0] = qm.x * E.x - c2 * E.y, x[1] = qm.x * E.y + c2 * E.x;
                        x[2] = -qm.y * E.y, x[3] = qm.y * E.x;
                        x[4] = -qm.z * E.y, x[5] = qm.z * E.x;
                    }
                    // real column: (Xr, -Xi, Yr, -Yi, Zr, -Zi); imaginary: (Xi, Xr, Yi, Yr, Zi, Zr)
                    v[0] = x[0], v[1] = -x[1], v[2] = x[2], v[3] = -x[3], v[4] = x[4], v[5] = -x[5];
                    store_terms(B, 2 * zc, j, B_LBO, v, false);
                    v[0] = x[1], v[1] = x[0], v[2] = x[3], v[3] = x[2], v[4] = x[5], v[5] = x[4];
                    store_terms(B, 2 * zc + 1, j, B_LBO, v, false);
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&full[slot])) : "memory");
        }
    } else if (warp < TC_PW + TC_DW) {
        // ---------------------------------------------------------------- drain
        // FP32 sums over groups, written as TC_SUB sub-chunk partials per CTA (each over
        // about a quarter of the CTA's ions), summed in FP64 with the other chunks
        const int dw = warp - TC_PW, sub = warp & 3, half = dw >> 2;
        const int r = row0 + sub * 32 + lane;
        KRow Q;
        Q.z0 = Q.cnt = Q.koff = 0;
        if (r < a.nrow) Q = a.row[r];
        const int fg = max(1, (ngroup + TC_SUB - 1) / TC_SUB);
        float acc[NH];
#pragma unroll
        for (int k = 0; k < NH; k++) acc[k] = 0.f;
        int written = 0;
        auto flush = [&](int sc) {
            if (r < a.nrow) {
                float2 *P = a.part + ((size_t)blockIdx.y * TC_SUB + sc) * a.nk;
#pragma unroll
                for (int k = 0; k < NH / 2; k++) {
                    int zz = half * (NH / 2) + k - a.K2;
                    if (zz >= Q.z0 && zz < Q.z0 + Q.cnt) P[Q.koff + (zz - Q.z0)] = make_float2(acc[2 * k], acc[2 * k + 1]);
                }
            }
#pragma unroll
            for (int k = 0; k < NH; k++) acc[k] = 0.f;
        };
        for (int g = 0; g < ngroup && ok; g++) {
            const int reg = g & 1;
            if (!mbar_wait(smem_u32(&tfull[reg]), (g >> 1) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int q = 0; q < TC_R; q++) {
                uint32_t base = tmem + ((uint32_t)(sub * 32) << 16) + (uint32_t)((reg * TC_R + q) * N + half * NH);
                float v[NH];   // all loads of one accumulator in flight, one wait
#pragma unroll
                for (int c8 = 0; c8 < NH; c8 += 8) tmem_ld8(base + (uint32_t)c8, v + c8);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int k = 0; k < NH; k++) acc[k] += v[k];
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[reg])) : "memory");
            if ((g + 1) % fg == 0 || g == ngroup - 1) flush(written++);
        }
        if (ok)
            while (written < TC_SUB) flush(written++);   // sub-chunks without ions: zero
    } else {
        // ---------------------------------------------------------------- MMA issue
        const uint32_t idesc = idesc_tf32(TC_M, N);
        int last = -1;
        for (int s = 0; s < nstage && ok; s++) {
            const int slot = s % TC_NSLOT, use = s / TC_NSLOT;
            const int g = s / TC_G, reg = g & 1;
            if (!mbar_wait(smem_u32(&full[slot]), use & 1)) {
                ok = false;
                break;
            }
            if (s % TC_G == 0 && g >= 2 && !mbar_wait(smem_u32(&tempty[reg]), ((g >> 1) - 1) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (lane == 0) {
                uint32_t ab = smem_u32(sm + slot * SLOT), bb = ab + CH * A_LBO;
#pragma unroll
                for (int k = 0; k < CH / 2; k++) {   // consecutive MMAs into different accumulators
                    uint32_t dt = tmem + (uint32_t)((reg * TC_R + k % TC_R) * N);
                    uint64_t da = smem_desc(ab + 2 * k * A_LBO, A_LBO, 128);
                    uint64_t db = smem_desc(bb + 2 * k * B_LBO, B_LBO, 128);
                    mma_tf32(dt, da, db, idesc, (s % TC_G == 0 && k < TC_R) ? 0u : 1u);
                }
                mma_commit(smem_u32(&empty[slot]));
                if (s % TC_G == TC_G - 1 || s == nstage - 1) mma_commit(smem_u32(&tfull[reg]));
            }
            __syncwarp();
            last = s;
        }
        // every MMA of this CTA has completed once the last commit has arrived
        if (last >= 0) mbar_wait(smem_u32(&empty[last % TC_NSLOT]), (last / TC_NSLOT) & 1);
    }
    if (!ok) atomicOr(a.status, (unsigned)ST_TC_TIMEOUT);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

template <int NZP>
static size_t rho_tc_slot_bytes() {
    return (size_t)(TC_KSTAGE / 4) * ((TC_M / 8) * 128 + (2 * NZP / 8) * 128);
}

template <int NZP>
static void rho_tc_launch(Engine &e, RhoTcArgs a, int mtiles, int chunks) {
    size_t slot = rho_tc_slot_bytes<NZP>();
    size_t smem = TC_NSLOT * slot + (2 * TC_NSLOT + 4) * sizeof(uint64_t) + 16;
    MDFF_CK(cudaFuncSetAttribute(k_rho_tc<NZP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MDFF_LAUNCH(e, k_rho_tc<NZP>, dim3(mtiles, chunks), TC_THREADS, smem, a);
}

// rho(k) chunk partials of `cnt` ions (idx: subset) into e.d_rho_part32 on the tensor
// cores; returns false (nothing launched) when the k box is outside the kernel's range.
bool launch_rho_tc(Engine &e, const double *q, const double3 *mu, bool lq, bool ld, const int *idx, int cnt,
                   int tab_w, int z_off, int nzb_neg, int *chunks_used) {
    int K2 = e.kmax[2];
    int nz = 2 * K2 + 1;
    int NZP = nz <= 16 ? 16 : (nz <= 32 ? 32 : 0);
    if (!NZP || cnt <= 0) return false;
    if (!e.d_qm_tc) e.d_qm_tc = dalloc<float4>(e.n);
    MDFF_LAUNCH(e, k_qm_tc, ceil_div(cnt, 256), 256, 0, cnt, idx, e.cell, q, mu, lq ? 1 : 0, ld ? 1 : 0, e.d_qm_tc);
    int mtiles = ceil_div(e.nrow, TC_M);
    int chunks = std::max(1, std::min(e.rho32_chunks / TC_SUB, e.nsm / std::max(1, mtiles)));
    RhoTcArgs a;
    a.cnt = cnt;
    a.chunk = ceil_div(ceil_div(cnt, chunks), TC_SI) * TC_SI;
    chunks = ceil_div(cnt, a.chunk);
    a.nrow = e.nrow;
    a.nk = e.nk;
    a.K2 = K2;
    a.tab_w = tab_w;
    a.z_off = z_off;
    a.nzb_neg = nzb_neg;
    a.e1 = e.kmax[0] + 1;
    a.K1 = e.kmax[1];
    a.idx = idx;
    a.tab = e.d_tab32;
    a.qm = e.d_qm_tc;
    a.row = e.d_row;
    a.part = e.d_rho_part32;
    a.status = e.d_status;
    if (NZP == 16) rho_tc_launch<16>(e, a, mtiles, chunks);
    else rho_tc_launch<32>(e, a, mtiles, chunks);
    *chunks_used = chunks * TC_SUB;
    return true;
}

}  // namespace mdffgpu
