// FP64 short-range pair term shared by the FP64 pair kernel (pair.cu) and the mixed-
// precision pair preparation (real32.cu): n-m Lennard-Jones (src/nmlj.c:254-385) or
// BHMFT(D) with Tang-Toennies damped dispersion (src/bhmftd.c:117-271).
#pragma once
#include "engine.cuh"

namespace mdffgpu {

struct TT {
    double E[9];  // 1/k!, get_TT_damp src/tt_damp.c:34-40
};

inline TT make_tt() {
    TT tt;
    tt.E[0] = 1.0;
    for (int k = 1; k < 9; k++) tt.E[k] = tt.E[k - 1] / (double)k;
    return tt;
}

__device__ __forceinline__ double powi(double x, int k) {
    double r = 1.0;
    while (k) {
        if (k & 1) r *= x;
        x *= x;
        k >>= 1;
    }
    return r;
}

// TT_damping_functions, src/tt_damp.c:16-32
__device__ __forceinline__ void tt_damp(const TT &tt, double b, double c, double r, int order, double &f,
                                        double &fd) {
    double br = b * r;
    double ex = exp(-br) * c;
    double ff = tt.E[order];
    for (int k = order - 1; k > -1; k--) ff = ff * br + tt.E[k];
    f = 1.0 - ff * ex;
    fd = tt.E[order] * powi(br, order) * ex * b;
}

// pair energy u and w = -(du/dr)/r of one pair at squared distance r2 (inside the cut-off)
template <bool LJ>
__device__ __forceinline__ void sr_pair(const PairSR &P, double r2, int trunctype, int damped, const TT &tt,
                                        double &u, double &w) {
    if (LJ) {
        double sr2 = P.sigsq / r2;
        double srp = P.ip >= 0 ? powi(sr2, P.ip) : pow(sr2, P.ptwo);
        double srq = P.iq >= 0 ? powi(sr2, P.iq) : pow(sr2, P.qtwo);
        u = (trunctype == 2) ? 0.0 : P.epsqp * (P.plj * srq - P.qlj * srp) - (trunctype == 1 ? P.uc : 0.0);
        w = P.fc * (srq - srp) * sr2;
    } else {
        double ir2 = 1.0 / r2, d = sqrt(r2);
        double erh = P.A * exp(-P.B * d);
        double ir6 = ir2 * ir2 * ir2, ir8 = ir6 * ir2;
        ir6 *= P.C;
        ir8 *= P.D;
        double f6 = 1.0, f8 = 1.0, fd6 = 0.0, fd8 = 0.0;
        if (damped) {
            tt_damp(tt, P.BD, 1.0, d, 6, f6, fd6);
            tt_damp(tt, P.BD, 1.0, d, 8, f8, fd8);
        }
        double ir6d = ir6 * f6, ir8d = ir8 * f8;
        double ir7 = 6.0 * ir6d / d, ir9 = 8.0 * ir8d / d;
        u = erh - ir6d - ir8d;
        w = (P.B * erh - ir7 - ir9 + ir6 * fd6 + ir8 * fd8) / d;
    }
}

// BHMFT(D) pair term of sr_pair<false> with shared subexpressions, for the mixed-precision
// path: one FP64 reciprocal square root in place of the square root and four divisions,
// and one Tang-Toennies exponential and one set of powers of b r for both dispersion
// orders (f8's polynomial is f6's plus the k = 7, 8 terms).  Same function, other roundings.
__device__ __forceinline__ void bhm_pair_fast(const PairSR &P, double r2, int damped, double &u, double &w) {
    constexpr double E6 = 1.0 / 720.0, E7 = 1.0 / 5040.0, E8 = 1.0 / 40320.0;
    double id = rsqrt(r2), d = r2 * id, ir2 = id * id;
    double erh = P.A * exp(-P.B * d);
    double ir6 = ir2 * ir2 * ir2, ir8 = ir6 * ir2;
    ir6 *= P.C;
    ir8 *= P.D;
    double f6 = 1.0, f8 = 1.0, fd6 = 0.0, fd8 = 0.0;
    if (damped) {
        double br = P.BD * d, ex = exp(-br);
        double s6 = E6;
        s6 = s6 * br + 1.0 / 120.0;
        s6 = s6 * br + 1.0 / 24.0;
        s6 = s6 * br + 1.0 / 6.0;
        s6 = s6 * br + 0.5;
        s6 = s6 * br + 1.0;
        s6 = s6 * br + 1.0;
        double b2 = br * br, b4 = b2 * b2, b6 = b4 * b2;
        double s8 = s6 + b6 * br * (E7 + E8 * br);
        f6 = 1.0 - s6 * ex;
        f8 = 1.0 - s8 * ex;
        fd6 = E6 * b6 * ex * P.BD;
        fd8 = E8 * (b4 * b4) * ex * P.BD;
    }
    double ir6d = ir6 * f6, ir8d = ir8 * f8;
    u = erh - ir6d - ir8d;
    w = (P.B * erh - (6.0 * ir6d + 8.0 * ir8d) * id + ir6 * fd6 + ir8 * fd8) * id;
}

// pair contribution to the per-ion force and to (u, virial): acc = u, Vxx Vxy Vxz Vyy Vyz Vzz
// as sums over the full list of (r_a f_b + r_b f_a)
__device__ __forceinline__ void sr_accumulate(double3 r, double u, double w, double &fx, double &fy, double &fz,
                                              double (&acc)[7]) {
    double gx = w * r.x, gy = w * r.y, gz = w * r.z;
    fx += gx;
    fy += gy;
    fz += gz;
    acc[0] += u;
    acc[1] += r.x * gx + r.x * gx;
    acc[2] += r.x * gy + r.y * gx;
    acc[3] += r.x * gz + r.z * gx;
    acc[4] += r.y * gy + r.y * gy;
    acc[5] += r.y * gz + r.z * gy;
    acc[6] += r.z * gz + r.z * gz;
}

}  // namespace mdffgpu
