// common.cuh -- device-side constants, equation of state, face interpolants
// and periodic/wall index helpers shared by the dycore kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/erf_b200.h"

namespace erfb {

// Physical constants (reference: Source/ERF_Constants.H:10-30, 66-87)
constexpr double R_d = 287.0;
constexpr double R_v = 461.505;
constexpr double Cp_d = 1004.5;
constexpr double p_0 = 1.0e5;
constexpr double Gamma_ = 1.4;
constexpr double ip_0 = 1. / p_0;
constexpr double iR_d = 1. / R_d;
constexpr double iGamma = 1. / Gamma_;
constexpr double L_v = 2.5e6;
constexpr double lcond = 2.501e6;
constexpr double Rd_on_Rv = R_d / R_v;

// Status bits written by kernels (OR-ed into ctx->status)
constexpr int ST_BADSTATE = 1;
constexpr int ST_NAN = 2;
constexpr int ST_TIMEOUT = 4;   // a bounded tensor-core wait ran out
constexpr int ST_BOUNDS = 8;    // bounds-checked build: an index left its array

// ---------------------------------------------------------------------------
// Equation of state (reference: Source/Utils/ERF_EOS.H:42-151).  Same
// association of the operands as the reference; the per-cell powers
// x^y (x near 1, |y| < 2) are formed as exp(y log x), within a few ulps of
// pow and cheaper.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double powxy(double x, double y) { return exp(y * log(x)); }
__device__ __forceinline__ double eos_p(double rt, double qv) {
    return p_0 * powxy(R_d * rt * (1.0 + (R_v / R_d) * qv) * ip_0, Gamma_);
}
__device__ __forceinline__ double eos_exner(double rt, double rdOcp) {
    return powxy(R_d * rt * (1.0 + R_v / R_d * 0.0) * ip_0, Gamma_ * rdOcp);
}
__device__ __forceinline__ double eos_T(double rho, double rt, double qv) {
    double p_loc = p_0 * powxy(R_d * rt * (1.0 + R_v / R_d * qv) * ip_0, Gamma_);
    return p_loc / (R_d * rho * (1.0 + R_v / R_d * qv));
}
__device__ __forceinline__ double eos_rho_given_theta_p(double theta, double p, double rdOcp, double qv) {
    return pow(p_0, rdOcp) * pow(p, iGamma) / (R_d * theta * (1.0 + R_v / R_d * qv));
}
__device__ __forceinline__ double eos_exner_p(double P, double rdOcp) { return pow(P * ip_0, rdOcp); }
__device__ __forceinline__ double eos_rt_given_p(double p) {
    return pow(p * pow(p_0, Gamma_ - 1), iGamma) * iR_d / (1.0 + R_v / R_d * 0.0);
}

// ---------------------------------------------------------------------------
// Face interpolants (reference: Source/Utils/ERF_Interpolation_UPW.H:9-611,
// ERF_Interpolation_WENO.H:9-259).  s[0..5] = phi at offsets -3..+2 from the
// face's high-side cell; upw is the advecting momentum on the face.  V is
// the arithmetic type (double for the plain form, float for the mixed form).
// ---------------------------------------------------------------------------
template <int TYPE>
struct Interp;

template <>
struct Interp<ERF_ADV_CENTERED_2ND> {
    static constexpr int W = 1;
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V, V) { return V(0.5) * (s[3] + s[2]); }
};
template <>
struct Interp<ERF_ADV_UPWIND_3RD> {
    static constexpr int W = 2;
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V upw, V frac) {
        if (upw != V(0)) upw = (upw > V(0)) ? V(1) : V(-1);
        upw *= frac;
        V a1 = s[3] + s[2], d1 = s[3] - s[2], a2 = s[4] + s[1], d2 = s[4] - s[1];
        return V(7.0 / 12.0) * a1 - V(1.0 / 12.0) * a2 + upw * V(1.0 / 12.0) * (d2 - V(3) * d1);
    }
};
template <>
struct Interp<ERF_ADV_CENTERED_4TH> {
    static constexpr int W = 2;
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V, V) {
        V a1 = s[3] + s[2], a2 = s[4] + s[1];
        return V(7.0 / 12.0) * a1 - V(1.0 / 12.0) * a2;
    }
};
template <>
struct Interp<ERF_ADV_UPWIND_5TH> {
    static constexpr int W = 3;
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V upw, V frac) {
        if (upw != V(0)) upw = (upw > V(0)) ? V(1) : V(-1);
        upw *= frac;
        V a1 = s[3] + s[2], a2 = s[4] + s[1], a3 = s[5] + s[0];
        V d1 = s[3] - s[2], d2 = s[4] - s[1], d3 = s[5] - s[0];
        return V(37.0 / 60.0) * a1 - V(2.0 / 15.0) * a2 + V(1.0 / 60.0) * a3 -
               upw * V(1.0 / 60.0) * (d3 - V(5) * d2 + V(10) * d1);
    }
};
template <>
struct Interp<ERF_ADV_CENTERED_6TH> {
    static constexpr int W = 3;
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V, V) {
        V a1 = s[3] + s[2], a2 = s[4] + s[1], a3 = s[5] + s[0];
        return V(37.0 / 60.0) * a1 - V(2.0 / 15.0) * a2 + V(1.0 / 60.0) * a3;
    }
};
template <>
struct Interp<ERF_ADV_WENO_3> {
    static constexpr int W = 2;
    // WENO3 (ERF_Interpolation_WENO.H:9-124) with the weights normalised once.
    template <class V>
    __device__ static __forceinline__ V ev(V a, V b, V c) {
        const V eps = V(1.0e-6);
        V b1 = (b - a) * (b - a), b2 = (c - b) * (c - b);
        V e1 = (eps + b1) * (eps + b1), e2 = (eps + b2) * (eps + b2);
        V w1 = V(1.0 / 3.0) * e2;
        V w2 = V(2.0 / 3.0) * e1;
        V ws = w1 + w2;
        V v1 = -a + V(3) * b, v2 = b + c;
        return (w1 * v1 + w2 * v2) / (V(2) * ws);
    }
    // The upwind side is selected by operand choice rather than a branch, so
    // a warp whose faces have mixed signs evaluates the scheme once.
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V upw, V) {
        const V tol = V(1.0e-12);
        const bool pos = upw > tol;
        V r = ev<V>(pos ? s[1] : s[4], pos ? s[2] : s[3], pos ? s[3] : s[2]);
        return (upw > tol || upw < -tol) ? r : V(0.5) * (s[3] + s[2]);
    }
};
template <>
struct Interp<ERF_ADV_WENO_5> {
    static constexpr int W = 3;
    // Jiang-Shu WENO5 with the reference's smoothness indicators, linear
    // weights (1/10, 3/5, 3/10) and eps = 1e-6 (ERF_Interpolation_WENO.H:
    // 129-259).  The non-linear weights g_k / (eps + b_k)^2 are formed as
    // g_k * prod_{m != k} (eps + b_m)^2, which has the same ratios and needs
    // one division (the normalisation) instead of four.
    template <class V>
    __device__ static __forceinline__ V ev(V a, V b, V c, V d, V e) {
        const V c1 = V(13.0 / 12.0), eps = V(1.0e-6);
        V b1 = c1 * (a - V(2) * b + c) * (a - V(2) * b + c) + V(0.25) * (a - V(4) * b + V(3) * c) * (a - V(4) * b + V(3) * c);
        V b2 = c1 * (b - V(2) * c + d) * (b - V(2) * c + d) + V(0.25) * (b - d) * (b - d);
        V b3 = c1 * (c - V(2) * d + e) * (c - V(2) * d + e) + V(0.25) * (V(3) * c - V(4) * d + e) * (V(3) * c - V(4) * d + e);
        V e1 = (eps + b1) * (eps + b1), e2 = (eps + b2) * (eps + b2), e3 = (eps + b3) * (eps + b3);
        V w1 = V(1.0 / 10.0) * (e2 * e3);
        V w2 = V(3.0 / 5.0) * (e1 * e3);
        V w3 = V(3.0 / 10.0) * (e1 * e2);
        V ws = w1 + w2 + w3;
        V v1 = V(2) * a - V(7) * b + V(11) * c;
        V v2 = -b + V(5) * c + V(2) * d;
        V v3 = V(2) * c + V(5) * d - e;
        return (w1 * v1 + w2 * v2 + w3 * v3) / (V(6) * ws);
    }
    template <class V>
    __device__ static __forceinline__ V eval(const V* s, V upw, V) {
        const V tol = V(1.0e-12);
        const bool pos = upw > tol;
        V r = ev<V>(pos ? s[0] : s[5], pos ? s[1] : s[4], pos ? s[2] : s[3], pos ? s[3] : s[2], pos ? s[4] : s[1]);
        return (upw > tol || upw < -tol) ? r : V(0.5) * (s[3] + s[2]);
    }
};

// Runtime dispatch over the supported interpolant codes
template <class V>
__device__ __forceinline__ V interp_rt(int type, const V* s, V upw, V frac) {
    switch (type) {
    case ERF_ADV_CENTERED_2ND: return Interp<ERF_ADV_CENTERED_2ND>::eval<V>(s, upw, frac);
    case ERF_ADV_UPWIND_3RD: return Interp<ERF_ADV_UPWIND_3RD>::eval<V>(s, upw, frac);
    case ERF_ADV_CENTERED_4TH: return Interp<ERF_ADV_CENTERED_4TH>::eval<V>(s, upw, frac);
    case ERF_ADV_UPWIND_5TH: return Interp<ERF_ADV_UPWIND_5TH>::eval<V>(s, upw, frac);
    case ERF_ADV_CENTERED_6TH: return Interp<ERF_ADV_CENTERED_6TH>::eval<V>(s, upw, frac);
    case ERF_ADV_WENO_3: return Interp<ERF_ADV_WENO_3>::eval<V>(s, upw, frac);
    case ERF_ADV_WENO_5: return Interp<ERF_ADV_WENO_5>::eval<V>(s, upw, frac);
    default: return V(0);
    }
}
__host__ __device__ __forceinline__ int stencil_width(int type) {
    switch (type) {
    case ERF_ADV_CENTERED_2ND: return 1;
    case ERF_ADV_UPWIND_3RD: case ERF_ADV_CENTERED_4TH: case ERF_ADV_WENO_3: return 2;
    default: return 3;
    }
}

// Compile-time selection of the interpolant: T >= 0 is a fixed scheme code,
// T < 0 selects the scheme at run time from `rt`.
template <int T>
__device__ __forceinline__ int width_of(int rt) {
    if constexpr (T < 0) return stencil_width(rt);
    else return Interp<T>::W;
}
template <int T, class V>
__device__ __forceinline__ V interp_of(int rt, const V* s, V upw, V frac) {
    if constexpr (T < 0) return interp_rt<V>(rt, s, upw, frac);
    else return Interp<T>::template eval<V>(s, upw, frac);
}

// Wall-reduced vertical interpolant for w (UPWINDALL, reference
// ERF_Interpolation_UPW.H:528-611); s entries outside the scheme's width are
// ignored.
template <class V>
__device__ __forceinline__ V interp_all(int type, const V* s, V upw, V frac) {
    if (type == ERF_ADV_CENTERED_2ND) return V(0.5) * (s[3] + s[2]);
    bool wide = (type == ERF_ADV_UPWIND_5TH || type == ERF_ADV_CENTERED_6TH);
    V sm3 = wide ? s[0] : V(0), sp2 = wide ? s[5] : V(0);
    if (upw != V(0)) upw = (upw > V(0)) ? V(1) : V(-1);
    upw *= frac;
    V a1 = s[3] + s[2], a2 = s[4] + s[1], d1 = s[3] - s[2], d2 = s[4] - s[1];
    V a3 = sp2 + sm3, d3 = sp2 - sm3;
    if (type == ERF_ADV_UPWIND_3RD) return V(7.0 / 12.0) * a1 - V(1.0 / 12.0) * a2 + upw * V(1.0 / 12.0) * (d2 - V(3) * d1);
    if (type == ERF_ADV_CENTERED_4TH) return V(7.0 / 12.0) * a1 - V(1.0 / 12.0) * a2;
    if (type == ERF_ADV_UPWIND_5TH)
        return V(37.0 / 60.0) * a1 - V(2.0 / 15.0) * a2 + V(1.0 / 60.0) * a3 - upw * V(1.0 / 60.0) * (d3 - V(5) * d2 + V(10) * d1);
    return V(37.0 / 60.0) * a1 - V(2.0 / 15.0) * a2 + V(1.0 / 60.0) * a3;
}

// ---------------------------------------------------------------------------
// Saturation over water: Flatau et al. (1992) Table 4 polynomials in Horner
// form, as in the reference's Source/Utils/ERF_Microphysics_Utils.H:52-160.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double esatw(double t) {
    double dtt = fmin(t - 273.16, 70.);
    return 6.11239921 + dtt * (0.443987641 + dtt * (0.142986287e-1 + dtt * (0.264847430e-3 + dtt * (0.302950461e-5 + dtt * (0.206739458e-7 + dtt * (0.640689451e-10 + dtt * (-0.952447341e-13 + -0.976195544e-15 * dtt)))))));
}
__device__ __forceinline__ double dtesatw(double t) {
    double dtt = t - 273.16;
    if (dtt >= 70.) return 0.0;
    return 0.443956472 + dtt * (0.285976452e-1 + dtt * (0.794747212e-3 + dtt * (0.121167162e-4 + dtt * (0.103167413e-6 + dtt * (0.385208005e-9 + dtt * (-0.604119582e-12 + dtt * (-0.792933209e-14 + -0.599634321e-17 * dtt)))))));
}

// ---------------------------------------------------------------------------
// Geometry and array views.  Internal arrays hold the valid region only:
// cells and x/y faces are nx*ny*nz (periodic faces: face nx == face 0),
// z faces nx*ny*(nz+1).  Lateral neighbours wrap; vertical neighbours follow
// the wall conditions.
// ---------------------------------------------------------------------------
struct Geo {
    int nx, ny, nz;
    int64_t sk;        // nx*ny
    int64_t ncell;     // nx*ny*nz
    int64_t nzf;       // nx*ny*(nz+1)
    double dxi, dyi, dzi;
    int zlo_noslip, zhi_noslip;
#ifdef ERF_B200_BOUNDS
    int* oob = nullptr;   // status word the bounds checks OR ST_BOUNDS into
#endif
};

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
// Periodic index for offsets that may exceed one period (tile halos on grids
// narrower than a tile): the common one-period cases without a division.
__device__ __forceinline__ int wrap_far(int i, int n) {
    if (i < 0) i += n;
    if (i >= n) i -= n;
    if ((unsigned)i >= (unsigned)n) i = ((i % n) + n) % n;
    return i;
}
__device__ __forceinline__ int clampk(int k, int nz) { return k < 0 ? 0 : (k >= nz ? nz - 1 : k); }
// Linear index of (i, j, k).  In the bounds-checked build
// (-DERF_B200_BOUNDS=1) an index outside i in [0, nx), j in [0, ny),
// k in [0, nz] (the z-face arrays have nz+1 levels) sets ST_BOUNDS in the
// status word and is replaced by element 0, so the access stays inside the
// array and the run goes on (no trap).
__device__ __forceinline__ int64_t cidx(const Geo& g, int i, int j, int k) {
#ifdef ERF_B200_BOUNDS
    if ((unsigned)i >= (unsigned)g.nx || (unsigned)j >= (unsigned)g.ny || (unsigned)k > (unsigned)g.nz) {
        if (g.oob) atomicOr(g.oob, ST_BOUNDS);
        return 0;
    }
#endif
    return (int64_t)i + (int64_t)g.nx * j + g.sk * k;
}

}  // namespace erfb
