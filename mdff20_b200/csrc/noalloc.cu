// Neighbour-list build that allocates nothing: the cell-binning scratch of the list
// build (fractional positions, cell of each ion, cell counts/starts/cursors, sorted
// cell members, positions at build) lives in one file-scope __device__ array instead
// of context buffers, and the caller passes its own device buffers for positions and
// lists.  It runs the same kernels as mdffgpu_gen_verletlist (lists.cu).
//
// For callers that cannot allocate device memory: an application that owns all GPU
// memory through its own pool and forbids allocations once it has started (so a
// cudaMalloc from a library would either fail or break its accounting), or a host that
// runs the engine inside a fixed device-memory budget set at start-up.
#include <mutex>

#include "engine.cuh"

namespace mdffgpu {

__global__ void k_kardir(int n, Cell c, const double4 *r, double4 *s);
__global__ void k_bin(int n, int3 nc, const double4 *s, int *cell_of, int *cnt, const int *rebuild);
__global__ void k_scan_cells(int ncell, const int *cnt, int *start, int *cur, int cell_cap, unsigned *status,
                             const int *rebuild);
__global__ void k_fill_cells(int n, const int *cell_of, const int *start, int *cur, int *ions, const int *rebuild);
__global__ void k_sort_cells(int ncell, int cell_cap, const int *start, const int *cnt, int *ions,
                             const int *rebuild);
__global__ void k_build(int n, Cell c, int3 nc, const double4 *s, const int *cell_of, const int *start,
                        const int *cnt, const int *ions, double rsq_nb, double rsq_co, int cap_nb, int *nbl,
                        int *nbn, int cap_co, int *col, int *con, double4 *svl, unsigned *status,
                        const int *rebuild);

// limits of the static scratch
constexpr int NA_MAX_IONS = 65536;
constexpr int NA_MAX_CELLS = 32768;
constexpr int NA_CELL_CAP = 4096;   // members of one cell (bitonic sort in shared memory)

// scratch layout, in 8-byte words: s[N] double4, svl[N] double4, then ints
constexpr size_t NA_WORDS = (size_t)NA_MAX_IONS * 4 * 2 +                       // s, svl
                            ((size_t)NA_MAX_IONS * 2 + (size_t)NA_MAX_CELLS * 3 + 64) / 2;  // ints
static __device__ __align__(256) double g_noalloc_scratch[NA_WORDS];

struct NaPtrs {
    double4 *s, *svl;
    int *cell_of, *ions, *cnt, *start, *cur, *rebuild;
    unsigned *status;
};

// device address of the scratch array, fetched once per device with that device current
static std::mutex g_na_mutex;
static void *g_na_base[64] = {nullptr};

static int na_pointers(NaPtrs *p) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MDFFGPU_ERR_CUDA;
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_base[dev]) {
            void *ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return MDFFGPU_ERR_CUDA;
            g_na_base[dev] = ptr;
        }
        base = g_na_base[dev];
    }
    char *b = (char *)base;
    p->s = (double4 *)b;
    p->svl = p->s + NA_MAX_IONS;
    int *ib = (int *)(p->svl + NA_MAX_IONS);
    p->cell_of = ib;
    p->ions = ib + NA_MAX_IONS;
    p->cnt = p->ions + NA_MAX_IONS;
    p->start = p->cnt + NA_MAX_CELLS;
    p->cur = p->start + NA_MAX_CELLS;
    p->rebuild = p->cur + NA_MAX_CELLS;
    p->status = (unsigned *)(p->rebuild + 1);
    return MDFFGPU_OK;
}

}  // namespace mdffgpu

using namespace mdffgpu;

extern "C" int mdffgpu_build_lists_noalloc(const double *d_pos, int n, const double *cell, double cut_nb,
                                           double cut_co, int cap_nb, int *d_nb, int *d_nbn, int cap_co,
                                           int *d_co, int *d_con, void *stream, int *status_out) {
    if (!d_pos || !cell || !d_nb || !d_nbn || !d_co || !d_con || n <= 0 || cap_nb <= 0 || cap_co <= 0 ||
        !(cut_nb > 0.0) || !(cut_co > 0.0))
        return MDFFGPU_ERR_ARG;
    if (n > NA_MAX_IONS) return MDFFGPU_ERR_ARG;   // more ions than the static scratch holds
    if (((uintptr_t)d_pos) % 32 != 0) return MDFFGPU_ERR_ARG;
    // lattice as lattice() (src/cell.c:13-91)
    Cell c;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.A[i][j] = cell[3 * i + j];
    auto cross = [](const double *a, const double *b, double *h) {
        h[0] = a[1] * b[2] - a[2] * b[1];
        h[1] = a[2] * b[0] - a[0] * b[2];
        h[2] = a[0] * b[1] - a[1] * b[0];
    };
    cross(c.A[1], c.A[2], c.B[0]);
    cross(c.A[2], c.A[0], c.B[1]);
    cross(c.A[0], c.A[1], c.B[2]);
    double omega = c.B[0][0] * c.A[0][0] + c.B[1][0] * c.A[1][0] + c.B[2][0] * c.A[2][0];
    if (!(omega > 0.0)) return MDFFGPU_ERR_ARG;
    c.omega = omega;
    c.inveOmega = 1.0 / omega;
    c.inveOmegaPU = 0.0;
    for (int i = 0; i < 3; i++)
        c.w[i] = omega / std::sqrt(c.B[0][i] * c.B[0][i] + c.B[1][i] * c.B[1][i] + c.B[2][i] * c.B[2][i]);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) c.B[i][j] = c.B[i][j] * c.inveOmega;
    c.ortho = 1;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            if (i != j && c.A[i][j] != 0.0) c.ortho = 0;
    // cell grid as Engine::setup_cells, then coarsened to the scratch's cell limit: the
    // largest dimension loses one cell at a time, so every cell stays at least one list
    // radius wide and the pair sets are those of the finer grid (32768 = 32^3, so no
    // dimension drops below 3)
    double cut = cut_nb > cut_co ? cut_nb : cut_co;
    int nc[3];
    for (int d = 0; d < 3; d++) {
        int k = (int)std::floor(c.w[d] / cut);
        nc[d] = (k >= 3 && c.ortho) ? (k < 64 ? k : 64) : 1;
    }
    while ((long long)nc[0] * nc[1] * nc[2] > NA_MAX_CELLS) {
        int d = (nc[1] > nc[0]) ? 1 : 0;
        if (nc[2] > nc[d]) d = 2;
        nc[d]--;
    }
    int ncell = nc[0] * nc[1] * nc[2];
    if (ncell == 1 && n > NA_CELL_CAP) return MDFFGPU_ERR_CELL;   // one cell must hold every ion
    NaPtrs P;
    int rc = na_pointers(&P);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the array keeps the last call's contents: reset what must start at zero, and set
    // the build flag the kernels test (any non-zero value)
    if (cudaMemsetAsync(P.cnt, 0, sizeof(int) * ncell, st) != cudaSuccess) return MDFFGPU_ERR_CUDA;
    if (cudaMemsetAsync(P.status, 0, sizeof(unsigned), st) != cudaSuccess) return MDFFGPU_ERR_CUDA;
    if (cudaMemsetAsync(P.rebuild, 1, sizeof(int), st) != cudaSuccess) return MDFFGPU_ERR_CUDA;
    int3 g = make_int3(nc[0], nc[1], nc[2]);
    int nb = (n + 255) / 256;
    k_kardir<<<nb, 256, 0, st>>>(n, c, (const double4 *)d_pos, P.s);
    k_bin<<<nb, 256, 0, st>>>(n, g, P.s, P.cell_of, P.cnt, P.rebuild);
    k_scan_cells<<<1, 1024, 0, st>>>(ncell, P.cnt, P.start, P.cur, NA_CELL_CAP, P.status, P.rebuild);
    k_fill_cells<<<nb, 256, 0, st>>>(n, P.cell_of, P.start, P.cur, P.ions, P.rebuild);
    k_sort_cells<<<ncell, 256, sizeof(int) * NA_CELL_CAP, st>>>(ncell, NA_CELL_CAP, P.start, P.cnt, P.ions,
                                                              P.rebuild);
    k_build<<<(int)(((long long)n * 32 + 255) / 256), 256, 0, st>>>(n, c, g, P.s, P.cell_of, P.start, P.cnt,
                                                                    P.ions, cut_nb * cut_nb, cut_co * cut_co,
                                                                    cap_nb, d_nb, d_nbn, cap_co, d_co, d_con,
                                                                    P.svl, P.status, P.rebuild);
    if (cudaGetLastError() != cudaSuccess) return MDFFGPU_ERR_CUDA;
    unsigned s = 0;
    if (cudaMemcpyAsync(&s, P.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MDFFGPU_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MDFFGPU_ERR_CUDA;
    if (status_out) *status_out = (int)s;
    if (s & ST_CELL_OVERFLOW) return MDFFGPU_ERR_CELL;
    if (s & ST_LIST_OVERFLOW) return MDFFGPU_ERR_LIST_OVERFLOW;
    return MDFFGPU_OK;
}
