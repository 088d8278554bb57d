// Verlet neighbour lists on the GPU: gen_pbc_verletlist / check_verletlist
// (src/verlet.c:54-170) rebuilt as cell-binned, warp-per-ion FULL lists.
//
// The reference keeps a half list (each pair once, parity rule src/verlet.c:82-83)
// and scatters forces to both ions.  Here every ion keeps all its neighbours, so each
// force kernel writes only its own ion (no atomics, deterministic sums); the pair
// SET equals the reference's because every distance is computed with the reference's
// operation order (kardir, nearbyint minimum image, A-multiply, x^2+y^2+z^2, no FMA)
// and tested with the same inclusive `<= (rc+skin)^2` (src/verlet.c:90,99).
#include "engine.cuh"

namespace mdffgpu {

// s = kardir(r), w = charge
__global__ void k_kardir(int n, Cell c, const double4 *__restrict__ r, double4 *__restrict__ s) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 ri = r[i];
    double3 f = kardir(c, ri.x, ri.y, ri.z);
    s[i] = make_double4(f.x, f.y, f.z, ri.w);
}

void launch_kardir(Engine &e, const double4 *r, double4 *s) {
    MDFF_LAUNCH(e, k_kardir, ceil_div(e.n, 256), 256, 0, e.n, e.cell, r, s);
}

// ---------------------------------------------------------------- check_verletlist
// displacement since the last build, largest and second largest (src/verlet.c:134-147)
__device__ __forceinline__ void top2_insert(double &m1, double &m2, double d) {
    if (d > m1) {
        m2 = m1;
        m1 = d;
    } else if (d > m2) {
        m2 = d;
    }
}

// warp merge of per-lane top-2 pairs (the two largest values, whatever the order they
// are met in)
__device__ __forceinline__ void top2_warp(double &m1, double &m2) {
    for (int o = 16; o > 0; o >>= 1) {
        double o1 = __shfl_xor_sync(0xffffffffu, m1, o);
        double o2 = __shfl_xor_sync(0xffffffffu, m2, o);
        double n1 = fmax(m1, o1);
        double n2 = fmax(fmin(m1, o1), fmax(m2, o2));
        m1 = n1;
        m2 = n2;
    }
}

// check_verletlist in one launch: the fractional coordinates of the current positions
// (kardir, written to s for a rebuild), each ion's displacement since the last build and
// per block its two largest (src/verlet.c:134-147); the last block to finish merges the
// block pairs and tests them against the skin (src/verlet.c:148).  On a rebuild it also
// zeroes the cell counts the binning adds to, and in a recorded step it sets the
// condition of the IF node that holds the rebuild (use_h).
struct CheckArgs {
    int n, ncell;
    Cell c;
    const double4 *r;
    double4 *s;
    const double4 *svl;
    double *part1, *part2;
    unsigned *ticket;
    double skindiff;
    int *rebuild, *cell_cnt;
    DevScalars *out;
    cudaGraphConditionalHandle h;
    int use_h;
};
__global__ void __launch_bounds__(256) k_check_list(CheckArgs a) {
    grid_dep();
    __shared__ double sm1[8], sm2[8];
    __shared__ bool last;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double m1 = 0.0, m2 = 0.0;
    if (i < a.n) {
        const double4 ri = a.r[i];
        const double3 f = kardir(a.c, ri.x, ri.y, ri.z);
        a.s[i] = make_double4(f.x, f.y, f.z, ri.w);
        const double4 b = a.svl[i];
        const double3 d = pbc_frac(a.c, dsub(f.x, b.x), dsub(f.y, b.y), dsub(f.z, b.z));
        m1 = __dsqrt_rn(norm2_exact(d));
    }
    top2_warp(m1, m2);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sm1[w] = m1;
        sm2[w] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a1 = 0.0, a2 = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            top2_insert(a1, a2, sm1[k]);
            top2_insert(a1, a2, sm2[k]);
        }
        a.part1[blockIdx.x] = a1;
        a.part2[blockIdx.x] = a2;
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ int rb_s;
    if (w == 0) {
        const volatile double *p1 = a.part1, *p2 = a.part2;
        double b1 = 0.0, b2 = 0.0;
        for (int k = l; k < (int)gridDim.x; k += 32) {
            top2_insert(b1, b2, p1[k]);
            top2_insert(b1, b2, p2[k]);
        }
        top2_warp(b1, b2);
        if (l == 0) {
            const int rb = (b1 + b2 > a.skindiff) ? 1 : 0;   // src/verlet.c:148
            *a.rebuild = rb;
            a.out->rebuild = rb;
            if (rb) a.out->nbuilds += 1;
            if (a.use_h) cudaGraphSetConditional(a.h, rb ? 1u : 0u);
            *a.ticket = 0u;
            rb_s = rb;
        }
    }
    __syncthreads();
    if (rb_s)
        for (int k = threadIdx.x; k < a.ncell; k += blockDim.x) a.cell_cnt[k] = 0;
}

__global__ void k_force_rebuild(int *rebuild, DevScalars *out) {
    grid_dep();
    *rebuild = 1;
    out->rebuild = 1;
    out->nbuilds += 1;
}

void launch_check_list(Engine &e, const cudaGraphConditionalHandle *h) {
    CheckArgs a;
    a.n = e.n;
    a.ncell = e.ncell;
    a.c = e.cell;
    a.r = e.d_r;
    a.s = e.d_s;
    a.svl = e.d_svl;
    a.part1 = e.d_part + (size_t)S_DISP1 * e.part_stride;
    a.part2 = e.d_part + (size_t)S_DISP2 * e.part_stride;
    a.ticket = e.d_ticket + 5;
    a.skindiff = e.p.skindiff;
    a.rebuild = e.d_rebuild;
    a.cell_cnt = e.d_cell_cnt;
    a.out = e.d_out;
    a.h = h ? *h : cudaGraphConditionalHandle{};
    a.use_h = h != nullptr;
    MDFF_LAUNCH(e, k_check_list, ceil_div(e.n, 256), 256, 0, a);
}

// ---------------------------------------------------------------- cell binning
__device__ __forceinline__ int cell_coord(double s, int ncd) {
    double u = s - floor(s);
    int c = (int)(u * (double)ncd);
    return c < 0 ? 0 : (c >= ncd ? ncd - 1 : c);
}

__global__ void k_bin(int n, int3 nc, const double4 *__restrict__ s, int *__restrict__ cell_of,
                      int *__restrict__ cnt, const int *__restrict__ rebuild) {
    grid_dep();
    if (!*rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 si = s[i];
    int cx = cell_coord(si.x, nc.x), cy = cell_coord(si.y, nc.y), cz = cell_coord(si.z, nc.z);
    int c = (cx * nc.y + cy) * nc.z + cz;
    cell_of[i] = c;
    atomicAdd(&cnt[c], 1);
}

// exclusive scan of the cell counts (one block), resets the fill cursors
__global__ void k_scan_cells(int ncell, const int *__restrict__ cnt, int *__restrict__ start, int *__restrict__ cur,
                             int cell_cap, unsigned *status, const int *__restrict__ rebuild) {
    grid_dep();
    if (!*rebuild) return;
    __shared__ int carry;
    __shared__ int wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ncell; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = (i < ncell) ? cnt[i] : 0;
        if (i < ncell && v > cell_cap) atomicOr(status, ST_CELL_OVERFLOW);
        int x = v;
        int l = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (l >= o) x += y;
        }
        if (l == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            int t = (l < (int)(blockDim.x >> 5)) ? wsum[l] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, t, o);
                if (l >= o) t += y;
            }
            wsum[l] = t;
        }
        __syncthreads();
        int excl = x - v + (w > 0 ? wsum[w - 1] : 0) + carry;
        if (i < ncell) {
            start[i] = excl;
            cur[i] = 0;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + v;
        __syncthreads();
    }
}

__global__ void k_fill_cells(int n, const int *__restrict__ cell_of, const int *__restrict__ start,
                             int *__restrict__ cur, int *__restrict__ ions, const int *__restrict__ rebuild) {
    grid_dep();
    if (!*rebuild) return;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cell_of[i];
    int k = atomicAdd(&cur[c], 1);
    ions[start[c] + k] = i;
}

// sort each cell's ion indices ascending (bitonic in shared memory) so that the list
// order, hence every pair sum, is the same from run to run
__global__ void k_sort_cells(int ncell, int cell_cap, const int *__restrict__ start, const int *__restrict__ cnt,
                             int *__restrict__ ions, const int *__restrict__ rebuild) {
    grid_dep();
    if (!*rebuild) return;
    extern __shared__ int sh[];
    int c = blockIdx.x;
    if (c >= ncell) return;
    int m = cnt[c];
    if (m <= 1 || m > cell_cap) return;
    int b = start[c];
    int p2 = 1;
    while (p2 < m) p2 <<= 1;
    for (int k = threadIdx.x; k < p2; k += blockDim.x) sh[k] = (k < m) ? ions[b + k] : 0x7fffffff;
    __syncthreads();
    for (int size = 2; size <= p2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int k = threadIdx.x; k < p2; k += blockDim.x) {
                int j = k ^ stride;
                if (j > k) {
                    bool up = ((k & size) == 0);
                    int a = sh[k], bb = sh[j];
                    if ((a > bb) == up) {
                        sh[k] = bb;
                        sh[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int k = threadIdx.x; k < m; k += blockDim.x) ions[b + k] = sh[k];
}

// ---------------------------------------------------------------- list build
// one warp per ion: scan the 27 (or fewer, for thin cells) neighbour cells in a fixed
// order and append, in order, every j with |r_ij|^2 <= cut^2 to both lists.
__global__ void k_build(int n, Cell c, int3 nc, const double4 *__restrict__ s, const int *__restrict__ cell_of,
                        const int *__restrict__ start, const int *__restrict__ cnt, const int *__restrict__ ions,
                        double rsq_nb, double rsq_co, int cap_nb, int *__restrict__ nbl, int *__restrict__ nbn,
                        int cap_co, int *__restrict__ col, int *__restrict__ con, double4 *__restrict__ svl,
                        unsigned *status, const int *__restrict__ rebuild) {
    grid_dep();
    if (!*rebuild) return;
    int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (i >= n) return;
    double4 si = s[i];
    int ci = cell_of[i];
    int cx = ci / (nc.y * nc.z), cy = (ci / nc.z) % nc.y, cz = ci % nc.z;
    int rx = nc.x >= 3 ? 1 : 0, ry = nc.y >= 3 ? 1 : 0, rz = nc.z >= 3 ? 1 : 0;
    int knb = 0, kco = 0;
    int *mynb = nbl + (size_t)i * cap_nb;
    int *myco = col + (size_t)i * cap_co;
    unsigned lt = (1u << lane) - 1u;
    for (int dx = -rx; dx <= rx; dx++) {
        int x = (cx + dx + nc.x) % nc.x;
        for (int dy = -ry; dy <= ry; dy++) {
            int y = (cy + dy + nc.y) % nc.y;
            for (int dz = -rz; dz <= rz; dz++) {
                int z = (cz + dz + nc.z) % nc.z;
                int cc = (x * nc.y + y) * nc.z + z;
                int b = start[cc], e = b + cnt[cc];
                for (int base = b; base < e; base += 32) {
                    int idx = base + lane;
                    bool in_nb = false, in_co = false;
                    int j = -1;
                    if (idx < e) {
                        j = ions[idx];
                        if (j != i) {
                            double4 sj = s[j];
                            double3 d = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
                            double r2 = norm2_exact(d);
                            in_nb = (r2 <= rsq_nb);
                            in_co = (r2 <= rsq_co);
                        }
                    }
                    unsigned bnb = __ballot_sync(0xffffffffu, in_nb);
                    unsigned bco = __ballot_sync(0xffffffffu, in_co);
                    if (in_nb) {
                        int pos = knb + __popc(bnb & lt);
                        if (pos < cap_nb) mynb[pos] = j;
                    }
                    if (in_co) {
                        int pos = kco + __popc(bco & lt);
                        if (pos < cap_co) myco[pos] = j;
                    }
                    knb += __popc(bnb);
                    kco += __popc(bco);
                }
            }
        }
    }
    if (lane == 0) {
        nbn[i] = knb;
        con[i] = kco;
        svl[i] = si;
        if (knb > cap_nb || kco > cap_co) atomicOr(status, ST_LIST_OVERFLOW);
    }
}

void launch_build_lists(Engine &e, bool force) {
    if (force) MDFF_LAUNCH(e, k_force_rebuild, 1, 1, 0, e.d_rebuild, e.d_out);
    int3 nc = make_int3(e.nc[0], e.nc[1], e.nc[2]);
    // after k_check_list the counts are zero already when a rebuild is due
    if (force) MDFF_CK(cudaMemsetAsync(e.d_cell_cnt, 0, sizeof(int) * e.ncell, e.stream));
    MDFF_LAUNCH(e, k_bin, ceil_div(e.n, 256), 256, 0, e.n, nc, e.d_s, e.d_cell_of, e.d_cell_cnt, e.d_rebuild);
    MDFF_LAUNCH(e, k_scan_cells, 1, 1024, 0, e.ncell, e.d_cell_cnt, e.d_cell_start, e.d_cell_cur, e.cell_cap,
                e.d_status, e.d_rebuild);
    MDFF_LAUNCH(e, k_fill_cells, ceil_div(e.n, 256), 256, 0, e.n, e.d_cell_of, e.d_cell_start, e.d_cell_cur,
                e.d_cell_ions, e.d_rebuild);
    MDFF_LAUNCH(e, k_sort_cells, e.ncell, 256, sizeof(int) * e.cell_cap, e.ncell, e.cell_cap, e.d_cell_start,
                e.d_cell_cnt, e.d_cell_ions, e.d_rebuild);
    double cnb = e.p.cutshortrange + e.p.skindiff, cco = e.p.cutlongrange + e.p.skindiff;
    if (!e.p.lverletL) {  // no lists in the reference: every pair inside the cutoff itself
        cnb = e.p.cutshortrange;
        cco = e.p.cutlongrange;
    }
    MDFF_LAUNCH(e, k_build, ceil_div((long long)e.n * 32, 256), 256, 0, e.n, e.cell, nc, e.d_s, e.d_cell_of,
                e.d_cell_start, e.d_cell_cnt, e.d_cell_ions, cnb * cnb, cco * cco, e.cap_nb, e.d_nb, e.d_nbn,
                e.cap_co, e.d_co, e.d_con, e.d_svl, e.d_status, e.d_rebuild);
}

}  // namespace mdffgpu
