// Shared device helpers for the mdffgpu engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

#include "mdffgpu.h"

namespace mdffgpu {

constexpr int NT = MDFFGPU_NTMAX;
constexpr double PI_D = 3.1415926535897932385;   // src/constants.h:11
constexpr double TPI_D = 6.2831853071795864770;  // src/constants.h:12
constexpr int ASPC_DEPTH = 6;                    // MAX_EXTRAPOLATE_ORDER + 1, src/pim.h:4

// ------------------------------------------------------------------ errors
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define MDFF_CK(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::mdffgpu::Error(MDFFGPU_ERR_CUDA, std::string(#call) + ": " +               \
                                                         cudaGetErrorString(e_) + " at " +     \
                                                         __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

// device status word bits (set by kernels, read by the host after a step)
enum StatusBits : unsigned {
    ST_LIST_OVERFLOW = 1u,
    ST_CELL_OVERFLOW = 2u,
    ST_NONFINITE = 4u,
    ST_SCF = 8u,
    ST_TC_TIMEOUT = 16u,   // a tensor-core kernel gave up waiting on its MMAs
};

// ------------------------------------------------------------------ cell geometry
// Lattice as in lattice() (src/cell.c:13-91); passed by value to kernels.
struct Cell {
    double A[3][3];   // rows: lattice vectors
    double B[3][3];   // reciprocal rows, B[i] . A[j] = delta_ij
    double omega, inveOmega, inveOmegaPU;
    double w[3];      // perpendicular widths
    int ortho;        // A and B diagonal
};

// First statement of every kernel (programmatic dependent launch): wait until the grids
// this one depends on have completed and their writes are visible (returns at once for
// a launch without a programmatic edge), then let this grid's dependents be scheduled;
// a dependent grid runs nothing before its own wait, so only its launch overlaps this
// grid's tail
__device__ __forceinline__ void grid_dep() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Exactly-rounded FP64 products/sums: the reference's geometry is compiled without
// FMA contraction (src/Makefile:17, no -mfma), and the neighbour-list pair set must
// match it bit for bit, so these expressions are kept uncontracted.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// kardir (src/cell.c:125-143): fractional coordinates, v1 = x*B00 + y*B01 + z*B02
__device__ __forceinline__ double3 kardir(const Cell &c, double x, double y, double z) {
    double3 s;
    s.x = dadd(dadd(dmul(x, c.B[0][0]), dmul(y, c.B[0][1])), dmul(z, c.B[0][2]));
    s.y = dadd(dadd(dmul(x, c.B[1][0]), dmul(y, c.B[1][1])), dmul(z, c.B[1][2]));
    s.z = dadd(dadd(dmul(x, c.B[2][0]), dmul(y, c.B[2][1])), dmul(z, c.B[2][2]));
    return s;
}

// pbc (src/pbc.c:7-14): nearbyint in fractional space (round half to even = rint),
// then back to Cartesian with A; returns the Cartesian minimum-image vector.
__device__ __forceinline__ double3 pbc_frac(const Cell &c, double dx, double dy, double dz) {
    double sx = dsub(dx, rint(dx));
    double sy = dsub(dy, rint(dy));
    double sz = dsub(dz, rint(dz));
    double3 r;
    r.x = dadd(dadd(dmul(sx, c.A[0][0]), dmul(sy, c.A[1][0])), dmul(sz, c.A[2][0]));
    r.y = dadd(dadd(dmul(sx, c.A[0][1]), dmul(sy, c.A[1][1])), dmul(sz, c.A[2][1]));
    r.z = dadd(dadd(dmul(sx, c.A[0][2]), dmul(sy, c.A[1][2])), dmul(sz, c.A[2][2]));
    return r;
}

__device__ __forceinline__ double norm2_exact(double3 r) {
    return dadd(dadd(dmul(r.x, r.x), dmul(r.y, r.y)), dmul(r.z, r.z));
}

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// block sums of NV per-thread values
template <int NV>
__device__ __forceinline__ void block_sum_to_part(double (&v)[NV], double *part, int slot, int stride) {
    __shared__ double sh[32][NV];
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < NV; k++) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double a = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) a += sh[q][threadIdx.x];
        part[(size_t)(slot + threadIdx.x) * stride + blockIdx.x] = a;
    }
}

// The last block of a kernel to finish reduces the partials of slots first..first+nslots-1
// exactly as k_reduce_slots does (same order), so the separate reduction launch is not
// needed; ticket (zero between calls) counts the finished blocks.  The writers of the
// partials fence their writes before arriving.
__device__ __forceinline__ bool last_block_slots(const double *part, int stride, int first, int nslots,
                                                 double *scal, unsigned *ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return false;
    __threadfence();
    __shared__ double sh[32];
    for (int sl = first; sl < first + nslots; sl++) {
        const volatile double *p = part + (size_t)sl * stride;
        double a = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) a += p[k];
        a = warp_sum(a);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
        __syncthreads();
        if (threadIdx.x < 32) {
            double b = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
            b = warp_sum(b);
            if (threadIdx.x == 0) scal[sl] = b;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// Neumaier (compensated) summation for FP32 accumulations in the mixed path
struct KahanF {
    float s, c;
    __device__ __forceinline__ KahanF() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float x) {
        float t = s + x;
        if (fabsf(s) >= fabsf(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

// complex product in FP32
__device__ __forceinline__ float2 cmul32(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exp(2 pi i x) for an FP64 argument: exact reduction to [-1/2, 1/2], FP32 sincospi
__device__ __forceinline__ float2 cis2pi32(double x) {
    x -= rint(x);
    float sn, cs;
    sincospif((float)(2.0 * x), &sn, &cs);
    return make_float2(cs, sn);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace mdffgpu
