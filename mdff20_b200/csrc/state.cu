// Exact restart: the complete MD state of a context as one byte block.
//
// The reference restarts from CONTFF (src/config.c:291-345): positions wrapped into the
// cell, velocities and forces at 12 decimals.  That drops the induced-dipole history of
// the ASPC predictor (dipia_ind, src/config.h:48), the Nose-Hoover chain (xi, vxi,
// src/md.h:26), the leap-frog r(t-dt) (rxs, src/config.h:39), the positions at the last
// neighbour-list build (xvl, src/verlet.c:124-170) and the step count that sets the
// ASPC order (src/pim.c:325-333), so a restarted run leaves the original trajectory.
// This block keeps all of them at full precision: a context loaded from it continues
// exactly as the saved one would have (same lists, same predictor, same thermostat).
//
// Layout (little endian, 8-byte words after a 64-byte header):
//   header  "MDFFST01", int32 version, nion, ntype, egrator, istep, nbuilds, nhc_n,
//           list_ready, extrapolate_order, lverletL, 4 x int32 spare; then cell[9]
//   r[n][3] unwrapped positions, v[n][3], f[n][3], rs[n][3], svl[n][3] fractional
//   positions at the last build, mu_ind[n][3], hist[n][6][3], xi[16], vxi[16]
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine.cuh"

namespace mdffgpu {

namespace {

struct StateHeader {
    char magic[8];
    int32_t version, nion, ntype, egrator, istep, nbuilds, nhc_n, list_ready, extrapolate_order, lverletL;
    int32_t spare[4];
};
static_assert(sizeof(StateHeader) == 64, "state header is 64 bytes");
constexpr char MAGIC[8] = {'M', 'D', 'F', 'F', 'S', 'T', '0', '1'};
constexpr int VERSION = 1;
constexpr size_t WORDS_PER_ION = 3 * 6 + 18;

__global__ void k_pack3(int n, const double4 *__restrict__ a, double *__restrict__ out) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double4 x = a[i];
        out[3 * i] = x.x, out[3 * i + 1] = x.y, out[3 * i + 2] = x.z;
    }
}

// xyz from `in`, w = charge (the layout of d_r and d_s)
__global__ void k_unpack4(int n, const double *__restrict__ in, const double *__restrict__ q,
                          double4 *__restrict__ a) {
    grid_dep();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = make_double4(in[3 * i], in[3 * i + 1], in[3 * i + 2], q[i]);
}

}  // namespace

size_t Engine::state_bytes() const {
    return sizeof(StateHeader) + sizeof(double) * (9 + WORDS_PER_ION * (size_t)n + 32);
}

void Engine::save_state(unsigned char *buf) {
    StateHeader h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, MAGIC, 8);
    h.version = VERSION;
    h.nion = n;
    h.ntype = nt;
    h.egrator = p.egrator;
    h.istep = istep;
    sync_scalars();
    h.nbuilds = h_out->nbuilds;
    h.nhc_n = p.nhc_n;
    h.list_ready = list_ready ? 1 : 0;
    h.extrapolate_order = p.extrapolate_order;
    h.lverletL = p.lverletL;
    memcpy(buf, &h, sizeof h);
    double *w = (double *)(buf + sizeof h);
    memcpy(w, cell.A, sizeof(double) * 9);
    w += 9;
    size_t n3 = 3 * (size_t)n;
    std::vector<double> packed(2 * n3);
    int nb = ceil_div(n, 256);
    // stream-ordered scratch, returned to the pool on every exit (errors throw)
    struct AsyncScratch {
        double *p;
        cudaStream_t s;
        ~AsyncScratch() {
            if (p) cudaFreeAsync(p, s);
        }
    } scratch{nullptr, stream};
    MDFF_CK(cudaMallocAsync((void **)&scratch.p, sizeof(double) * 2 * n3, stream));
    double *d_tmp = scratch.p;
    MDFF_LAUNCH(*this, k_pack3, nb, 256, 0, n, d_r, d_tmp);
    MDFF_LAUNCH(*this, k_pack3, nb, 256, 0, n, d_svl, d_tmp + n3);
    MDFF_CK(cudaMemcpyAsync(packed.data(), d_tmp, sizeof(double) * 2 * n3, cudaMemcpyDeviceToHost, stream));
    scratch.p = nullptr;
    MDFF_CK(cudaFreeAsync(d_tmp, stream));
    std::vector<double> v(n3), f(n3), rs(n3), mu(n3), hist(18 * (size_t)n), nhc(32);
    MDFF_CK(cudaMemcpyAsync(v.data(), d_v, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(f.data(), d_f, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(rs.data(), d_rs, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(mu.data(), d_mu_ind, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(hist.data(), d_hist, sizeof(double) * 18 * n, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaMemcpyAsync(nhc.data(), d_nhc, sizeof(double) * 32, cudaMemcpyDeviceToHost, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    memcpy(w, packed.data(), sizeof(double) * n3), w += n3;   // r
    memcpy(w, v.data(), sizeof(double) * n3), w += n3;
    memcpy(w, f.data(), sizeof(double) * n3), w += n3;
    memcpy(w, rs.data(), sizeof(double) * n3), w += n3;
    memcpy(w, packed.data() + n3, sizeof(double) * n3), w += n3;   // svl
    memcpy(w, mu.data(), sizeof(double) * n3), w += n3;
    memcpy(w, hist.data(), sizeof(double) * 18 * n), w += 18 * (size_t)n;
    memcpy(w, nhc.data(), sizeof(double) * 32);
}

// Returns the saved step number.  The block must come from a context of the same system
// (ion and type counts, cell, integrator, ASPC order, list mode).
int Engine::load_state(const unsigned char *buf, size_t bytes) {
    if (bytes < sizeof(StateHeader)) throw Error(MDFFGPU_ERR_ARG, "state block too short");
    StateHeader h;
    memcpy(&h, buf, sizeof h);
    if (memcmp(h.magic, MAGIC, 8) != 0 || h.version != VERSION)
        throw Error(MDFFGPU_ERR_ARG, "not an engine state block");
    if (bytes != state_bytes()) throw Error(MDFFGPU_ERR_ARG, "state block size does not match this system");
    const double *w = (const double *)(buf + sizeof h);
    if (h.nion != n || h.ntype != nt || h.egrator != p.egrator || h.nhc_n != p.nhc_n ||
        h.extrapolate_order != p.extrapolate_order || h.lverletL != p.lverletL ||
        memcmp(w, cell.A, sizeof(double) * 9) != 0)
        throw Error(MDFFGPU_ERR_ARG, "state block belongs to another system");
    w += 9;
    size_t n3 = 3 * (size_t)n;
    const double *r = w, *v = r + n3, *f = v + n3, *rs = f + n3, *svl = rs + n3, *mu = svl + n3, *hist = mu + n3,
                 *nhc = hist + 18 * (size_t)n;
    int nb = ceil_div(n, 256);
    // stream-ordered scratch, returned to the pool on every exit (errors throw)
    struct AsyncScratch {
        double *p;
        cudaStream_t s;
        ~AsyncScratch() {
            if (p) cudaFreeAsync(p, s);
        }
    } scratch{nullptr, stream};
    MDFF_CK(cudaMallocAsync((void **)&scratch.p, sizeof(double) * 2 * n3, stream));
    double *d_tmp = scratch.p;
    MDFF_CK(cudaMemcpyAsync(d_tmp, r, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_tmp + n3, svl, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_LAUNCH(*this, k_unpack4, nb, 256, 0, n, d_tmp, d_q, d_r);
    MDFF_LAUNCH(*this, k_unpack4, nb, 256, 0, n, d_tmp + n3, d_q, d_s);
    MDFF_CK(cudaMemcpyAsync(d_v, v, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_f, f, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_rs, rs, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_mu_ind, mu, sizeof(double) * n3, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_hist, hist, sizeof(double) * 18 * n, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemcpyAsync(d_nhc, nhc, sizeof(double) * 32, cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    // the lists of the saved context are a function of the fractional positions at its
    // last build: build them again from exactly those (d_s = svl), growing as needed
    list_ready = false;
    if (h.list_ready && p.lverletL) {
        for (int attempt = 0; attempt < 8 && !list_ready; attempt++) {
            MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
            MDFF_LAUNCH(*this, k_unpack4, nb, 256, 0, n, d_tmp + n3, d_q, d_s);
            launch_build_lists(*this, true);
            unsigned st = 0;
            MDFF_CK(cudaMemcpyAsync(&st, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
            MDFF_CK(cudaStreamSynchronize(stream));
            if (st & ST_CELL_OVERFLOW) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "cell capacity exceeded");
            if (!(st & ST_LIST_OVERFLOW)) {
                list_ready = true;
                break;
            }
            std::vector<int> a(n), b(n);
            MDFF_CK(cudaMemcpy(a.data(), d_nbn, sizeof(int) * n, cudaMemcpyDeviceToHost));
            MDFF_CK(cudaMemcpy(b.data(), d_con, sizeof(int) * n, cudaMemcpyDeviceToHost));
            int ma = *std::max_element(a.begin(), a.end()), mb = *std::max_element(b.begin(), b.end());
            alloc_lists(std::max(cap_nb, (ma * 5 / 4 + 63) / 32 * 32), std::max(cap_co, (mb * 5 / 4 + 63) / 32 * 32));
        }
        if (!list_ready) throw Error(MDFFGPU_ERR_LIST_OVERFLOW, "neighbour list capacity could not be grown");
        launch_kardir(*this, d_r, d_s);   // as a finished step leaves it
    }
    scratch.p = nullptr;
    MDFF_CK(cudaFreeAsync(d_tmp, stream));
    int nbuilds = h.nbuilds;
    MDFF_CK(cudaMemcpyAsync(&d_out->nbuilds, &nbuilds, sizeof(int), cudaMemcpyHostToDevice, stream));
    MDFF_CK(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
    MDFF_CK(cudaStreamSynchronize(stream));
    istep = h.istep;
    coef_ready = false;
    rho_acc_ready = false;
    gen++;
    return h.istep;
}

}  // namespace mdffgpu
