// Radial distribution function on the GPU: the pair histogram of get_gr
// (src/radial_distribution.c:180-230) for one configuration after another.
//
// get_gr counts every ordered pair (ia, ja != ia) whose minimum-image distance is below
// cutgr into bin (int)(r / resg) of gr[bin][type(ia)][type(ja)], with the distance
// computed as everywhere in the reference: positions to fractional coordinates
// (kardir), difference, nearbyint shift, back to Cartesian with A (pbc,
// src/pbc.c:7-14), r^2 = x^2 + y^2 + z^2, sqrt.  The kernel does the same FP64
// operations, each rounded once (no contraction), so every pair lands in the
// reference's bin and the integer counts are identical.  A pair's distance is the same
// both ways round (negation is exact through every step), so each unordered pair is
// evaluated once and counted for both orders.
//
// Layout: one block per (i tile, j tile) of the upper triangle of the pair matrix,
// GR_TILE ions a side; the j tile is staged in shared memory, each thread runs one i
// against it, and the counts go to a block-private shared histogram that is added to
// the global 64-bit histogram once at the end (global atomics directly when the
// histogram does not fit in shared memory).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "engine.cuh"

namespace mdffgpu {

constexpr int GR_TILE = 128;
constexpr int GR_SMEM_COUNTERS = 10240;   // 40 KB of 32-bit block counters (+ 4.5 KB of tile)

__global__ void k_kardir(int n, Cell c, const double4 *r, double4 *s);

__global__ void __launch_bounds__(GR_TILE)
    k_gr_pairs(int n, Cell c, const double4 *__restrict__ s, const int *__restrict__ typ, int nt, int nbins,
               double cut2, double resg, unsigned long long *__restrict__ hist, int private_hist) {
    grid_dep();
    extern __shared__ unsigned int h_sh[];
    __shared__ double4 tile[GR_TILE];
    __shared__ int ttile[GR_TILE];
    int bi = blockIdx.y, bj = blockIdx.x;
    if (bj < bi) return;
    int nh = nbins * nt * nt;
    if (private_hist)
        for (int k = threadIdx.x; k < nh; k += blockDim.x) h_sh[k] = 0u;
    int j0 = bj * GR_TILE;
    int jend = min(GR_TILE, n - j0);
    if (threadIdx.x < jend) {
        tile[threadIdx.x] = s[j0 + threadIdx.x];
        ttile[threadIdx.x] = typ[j0 + threadIdx.x];
    }
    __syncthreads();
    int i = bi * GR_TILE + threadIdx.x;
    if (i < n) {
        double4 si = s[i];
        int ti = typ[i];
        for (int jj = (bi == bj) ? threadIdx.x + 1 : 0; jj < jend; jj++) {
            double4 sj = tile[jj];
            double3 d = pbc_frac(c, dsub(si.x, sj.x), dsub(si.y, sj.y), dsub(si.z, sj.z));
            double r2 = norm2_exact(d);
            if (!(r2 < cut2)) continue;
            int b = (int)__ddiv_rn(sqrt(r2), resg);
            if (b < 0 || b >= nbins) continue;   // cannot happen for nbins > cutgr / resg
            int tj = ttile[jj];
            int k1 = (b * nt + ti) * nt + tj, k2 = (b * nt + tj) * nt + ti;
            if (private_hist) {
                atomicAdd(&h_sh[k1], 1u);
                atomicAdd(&h_sh[k2], 1u);
            } else {
                atomicAdd(&hist[k1], 1ull);
                atomicAdd(&hist[k2], 1ull);
            }
        }
    }
    if (!private_hist) return;
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += blockDim.x)
        if (h_sh[k]) atomicAdd(&hist[k], (unsigned long long)h_sh[k]);
}

// lattice (src/cell.c:13-91) as far as kardir and pbc need it: A, B = (A_j x A_k) / omega
static Cell cell_of(const double *A9) {
    Cell c;
    memset(&c, 0, sizeof c);
    memcpy(c.A, A9, sizeof(c.A));
    const int nx[3] = {1, 2, 0}, ny[3] = {2, 0, 1};
    for (int i = 0; i < 3; i++) {
        const double *u = c.A[nx[i]], *v = c.A[ny[i]];
        c.B[i][0] = u[1] * v[2] - u[2] * v[1];
        c.B[i][1] = u[2] * v[0] - u[0] * v[2];
        c.B[i][2] = u[0] * v[1] - u[1] * v[0];
    }
    double omega = c.B[0][0] * c.A[0][0] + c.B[1][0] * c.A[1][0] + c.B[2][0] * c.A[2][0];
    if (!(omega > 0.0)) throw Error(MDFFGPU_ERR_ARG, "cell volume must be positive");
    c.omega = omega;
    c.inveOmega = 1.0 / omega;
    for (int i = 0; i < 3; i++)
        c.w[i] = omega / std::sqrt(c.B[0][i] * c.B[0][i] + c.B[1][i] * c.B[1][i] + c.B[2][i] * c.B[2][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.B[i][j] = c.B[i][j] * c.inveOmega;
    return c;
}

}  // namespace mdffgpu

using mdffgpu::Engine;
using mdffgpu::Error;

struct mdffgpu_rdf {
    int n = 0, nt = 0, nbins = 0, device = 0, nconf = 0;
    double cut2 = 0.0, resg = 0.0;
    cudaStream_t stream = nullptr;
    double4 *d_r = nullptr, *d_s = nullptr;
    int *d_typ = nullptr;
    unsigned long long *d_hist = nullptr;
    double4 *h_r = nullptr;   // pinned staging
    long long launches = 0;
    std::string err;
};

namespace {

template <typename F>
int rdf_guarded(mdffgpu_rdf *r, F &&f) {
    if (!r) return MDFFGPU_ERR_ARG;
    try {
        MDFF_CK(cudaSetDevice(r->device));
        f(*r);
        return MDFFGPU_OK;
    } catch (const Error &x) {
        r->err = x.what();
        return x.code;
    } catch (const std::exception &x) {
        r->err = x.what();
        return MDFFGPU_ERR_CUDA;
    }
}

void launch_gr(mdffgpu_rdf &r, const mdffgpu::Cell &c, const double4 *d_s, const int *d_typ, cudaStream_t st) {
    int nb = mdffgpu::ceil_div(r.n, mdffgpu::GR_TILE);
    int nh = r.nbins * r.nt * r.nt;
    int priv = nh <= mdffgpu::GR_SMEM_COUNTERS ? 1 : 0;
    size_t smem = priv ? sizeof(unsigned int) * nh : 0;
    dim3 grid(nb, nb);
    mdffgpu::k_gr_pairs<<<grid, mdffgpu::GR_TILE, smem, st>>>(r.n, c, d_s, d_typ, r.nt, r.nbins, r.cut2, r.resg,
                                                              r.d_hist, priv);
    MDFF_CK(cudaGetLastError());
    r.launches++;
}

}  // namespace

mdffgpu::Engine *mdffgpu_engine_of(mdffgpu_ctx *ctx);

extern "C" {

int mdffgpu_rdf_create(int nion, int ntype, const int *nionit, double cutgr, double resg, int nbins, int device,
                       mdffgpu_rdf **out) {
    if (!out || !nionit || nion <= 0 || ntype <= 0 || ntype > MDFFGPU_NTMAX || !(resg > 0.0) || !(cutgr > 0.0) ||
        nbins <= 0)
        return MDFFGPU_ERR_ARG;
    *out = nullptr;
    long long tot = 0;
    for (int t = 0; t < ntype; t++) tot += nionit[t] < 0 ? -1000000000LL : nionit[t];
    if (tot != nion) return MDFFGPU_ERR_ARG;
    if ((long long)nbins * ntype * ntype > (1LL << 28)) return MDFFGPU_ERR_ARG;
    mdffgpu_rdf *r = new mdffgpu_rdf();
    r->n = nion;
    r->nt = ntype;
    r->nbins = nbins;
    r->device = device;
    r->cut2 = cutgr * cutgr;
    r->resg = resg;
    int rc = rdf_guarded(r, [&](mdffgpu_rdf &x) {
        MDFF_CK(cudaStreamCreateWithFlags(&x.stream, cudaStreamNonBlocking));
        x.d_r = mdffgpu::dalloc<double4>(nion);
        x.d_s = mdffgpu::dalloc<double4>(nion);
        x.d_typ = mdffgpu::dalloc<int>(nion);
        x.d_hist = mdffgpu::dalloc<unsigned long long>((size_t)nbins * ntype * ntype);
        MDFF_CK(cudaMallocHost((void **)&x.h_r, sizeof(double4) * nion));
        std::vector<int> typ(nion);
        for (int t = 0, ia = 0; t < ntype; t++)
            for (int k = 0; k < nionit[t]; k++) typ[ia++] = t;
        MDFF_CK(cudaMemcpy(x.d_typ, typ.data(), sizeof(int) * nion, cudaMemcpyHostToDevice));
    });
    if (rc != MDFFGPU_OK) {
        mdffgpu_rdf_destroy(r);
        return rc;
    }
    *out = r;
    return MDFFGPU_OK;
}

int mdffgpu_rdf_destroy(mdffgpu_rdf *r) {
    if (!r) return MDFFGPU_ERR_ARG;
    cudaSetDevice(r->device);
    cudaFree(r->d_r);
    cudaFree(r->d_s);
    cudaFree(r->d_typ);
    cudaFree(r->d_hist);
    if (r->h_r) cudaFreeHost(r->h_r);
    if (r->stream) cudaStreamDestroy(r->stream);
    delete r;
    return MDFFGPU_OK;
}

const char *mdffgpu_rdf_last_error(const mdffgpu_rdf *r) { return r ? r->err.c_str() : "null rdf"; }

int mdffgpu_rdf_reset(mdffgpu_rdf *r) {
    return rdf_guarded(r, [&](mdffgpu_rdf &x) {
        MDFF_CK(cudaMemsetAsync(x.d_hist, 0, sizeof(unsigned long long) * x.nbins * x.nt * x.nt, x.stream));
        MDFF_CK(cudaStreamSynchronize(x.stream));
        x.nconf = 0;
    });
}

int mdffgpu_rdf_add(mdffgpu_rdf *r, const double *cell, const double *rx, const double *ry, const double *rz) {
    if (!cell || !rx || !ry || !rz) return MDFFGPU_ERR_ARG;
    return rdf_guarded(r, [&](mdffgpu_rdf &x) {
        mdffgpu::Cell c = mdffgpu::cell_of(cell);
        for (int i = 0; i < x.n; i++) x.h_r[i] = make_double4(rx[i], ry[i], rz[i], 0.0);
        MDFF_CK(cudaMemcpyAsync(x.d_r, x.h_r, sizeof(double4) * x.n, cudaMemcpyHostToDevice, x.stream));
        mdffgpu::k_kardir<<<mdffgpu::ceil_div(x.n, 256), 256, 0, x.stream>>>(x.n, c, x.d_r, x.d_s);
        MDFF_CK(cudaGetLastError());
        x.launches++;
        launch_gr(x, c, x.d_s, x.d_typ, x.stream);
        MDFF_CK(cudaStreamSynchronize(x.stream));
        x.nconf++;
    });
}

int mdffgpu_rdf_add_ctx(mdffgpu_rdf *r, mdffgpu_ctx *ctx) {
    Engine *e = mdffgpu_engine_of(ctx);
    if (!e) return MDFFGPU_ERR_ARG;
    return rdf_guarded(r, [&](mdffgpu_rdf &x) {
        if (e->n != x.n || e->nt != x.nt || e->device != x.device)
            throw Error(MDFFGPU_ERR_ARG, "rdf_add_ctx: the context holds another system or device");
        // the context's positions and types, on its stream (one less host round trip)
        mdffgpu::k_kardir<<<mdffgpu::ceil_div(x.n, 256), 256, 0, e->stream>>>(x.n, e->cell, e->d_r, x.d_s);
        MDFF_CK(cudaGetLastError());
        x.launches++;
        launch_gr(x, e->cell, x.d_s, e->d_typ, e->stream);
        MDFF_CK(cudaStreamSynchronize(e->stream));
        x.nconf++;
    });
}

int mdffgpu_rdf_counts(mdffgpu_rdf *r, long long *pairs, int *nconf) {
    if (!pairs) return MDFFGPU_ERR_ARG;
    return rdf_guarded(r, [&](mdffgpu_rdf &x) {
        size_t nh = (size_t)x.nbins * x.nt * x.nt;
        MDFF_CK(cudaMemcpyAsync(pairs, x.d_hist, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, x.stream));
        MDFF_CK(cudaStreamSynchronize(x.stream));
        if (nconf) *nconf = x.nconf;
    });
}

}  // extern "C"
